"""Image and long-slit data models on the drop-in driver.

The reference's 2-D and slit paths reuse the disk kernels of the spectral
path with other outputs (model/gmodels/intensity_2d.py, intensity_3d.py,
brightness_smdisk_2d.py, brightness_smdisk_3d.py, brightness_mcdisk_3d.py,
opacity_smdisk_3d.py; model/dmodels/image.py, lslit.py):

* a brightness component evaluates its disk into the spatial ``image``
  (per spaxel, the sum of its voxels' attenuated surface brightness,
  gmodels.hpp:930-940) and its brightness cube (``rdata``), with no spectral
  axis (spectral size 1, step 0);
* an opacity component evaluates an opacity disk into the shared 3-D opacity
  cube, which the brightness components of the same model then read
  (gmodels.hpp:933-937);
* DModelImage is a DCube of size (nx, ny, 1) with a PSF only: the image is
  convolved with the PSF on the padded grid, downscaled/cropped and masked
  like a cube;
* DModelLSlit is a DCube of size (nx, 1, nz): a spectral model evaluated on a
  slit one spatial pixel wide, convolved with the PSF and the LSF, and
  returned as its (nz, nx) plane.

Divergences from the reference at its HEAD (both are failures there): the
long-slit data is returned as the slit's (nz, nx) plane (the reference
indexes the cube as ``dcube()[0][:, 0, :]``, which fails on its 3-D array),
and its weight map is the weight cube (the reference returns the mask cube
there).
"""

import numpy as np

from .disk import Disk
from .model import DCube, _DiskComponent, _merge, _rnodes


def _lst(x):
    return [] if x is None else list(x) if isinstance(x, (list, tuple)) else [x]


class BrightnessSMDisk2D(_DiskComponent):
    """brightness_smdisk_2d.py: a thin smooth disk's surface brightness."""

    @staticmethod
    def type():
        return 'smdisk'

    def __init__(self, loose, tilted, bptraits, sptraits=None, wptraits=None, rnmin=None,
                 rnmax=None, rnsep=None, rnlen=None, rnodes=None, rstep=None, interp='linear'):
        disk = Disk(loose, tilted, _rnodes(rnmin, rnmax, rnsep, rnlen, rnodes), rstep, interp,
                    dict(rpt=_lst(bptraits), spt=_lst(sptraits), wpt=_lst(wptraits)))
        super().__init__(disk)

    def evaluate(self, driver, params, image, wdata, bdata, spat_size, spat_step, spat_zero,
                 spat_rota, dtype, out_extra):
        """brightness_smdisk_2d.py:97-113: spatial z of size 1, no spectrum."""
        _DiskComponent.evaluate(self, driver, params, None, image, None, wdata, bdata, None,
                                tuple(spat_size) + (1,), tuple(spat_step) + (0,),
                                tuple(spat_zero) + (0,), spat_rota, 1, 0.0, 0.0, dtype,
                                out_extra)


class BrightnessSMDisk3D(_DiskComponent):
    """brightness_smdisk_3d.py: a thick smooth disk's brightness."""

    @staticmethod
    def type():
        return 'smdisk'

    def __init__(self, loose, tilted, bptraits, bhtraits, zptraits=None, sptraits=None,
                 wptraits=None, rnmin=None, rnmax=None, rnsep=None, rnlen=None, rnodes=None,
                 rstep=None, interp='linear'):
        disk = Disk(loose, tilted, _rnodes(rnmin, rnmax, rnsep, rnlen, rnodes), rstep, interp,
                    dict(rpt=_lst(bptraits), rht=_lst(bhtraits), zpt=_lst(zptraits),
                         spt=_lst(sptraits), wpt=_lst(wptraits)))
        super().__init__(disk)

    def evaluate(self, driver, params, odata, image, wdata, bdata, obdata, spat_size, spat_step,
                 spat_zero, spat_rota, dtype, out_extra):
        """brightness_smdisk_3d.py:110-122."""
        _DiskComponent.evaluate(self, driver, params, odata, image, None, wdata, bdata, obdata,
                                spat_size, spat_step, spat_zero, spat_rota, 1, 0.0, 0.0, dtype,
                                out_extra)


class BrightnessMCDisk3D(BrightnessSMDisk3D):
    """brightness_mcdisk_3d.py: a thick cloud disk's brightness."""

    MC = True

    @staticmethod
    def type():
        return 'mcdisk'

    def __init__(self, cflux, *args, **kwargs):
        super().__init__(*args, **kwargs)
        self._cflux = float(cflux)

    def set_mcdisk(self, seed, mode=0):
        self._seed = (seed, mode)
        if self._backend is not None:
            self._backend.set_mcdisk(seed, mode)

    def _prepare(self, driver, dtype):
        super()._prepare(driver, dtype)
        if getattr(self, '_seed', None):
            self._backend.set_mcdisk(*self._seed)


class OpacitySMDisk3D(_DiskComponent):
    """opacity_smdisk_3d.py: a thick smooth disk of opacity (opacity traits:
    density uids + 1000, traits.py:71-101), evaluated into the model's
    opacity cube."""

    @staticmethod
    def type():
        return 'smdisk'

    def __init__(self, loose, tilted, optraits, ohtraits, zptraits=None, sptraits=None,
                 rnmin=None, rnmax=None, rnsep=None, rnlen=None, rnodes=None, rstep=None,
                 interp='linear'):
        disk = Disk(loose, tilted, _rnodes(rnmin, rnmax, rnsep, rnlen, rnodes), rstep, interp,
                    dict(rpt=_lst(optraits), rht=_lst(ohtraits), zpt=_lst(zptraits),
                         spt=_lst(sptraits)), opacity=True)
        super().__init__(disk)

    def evaluate(self, driver, params, odata, spat_size, spat_step, spat_zero, spat_rota, dtype,
                 out_extra):
        """opacity_smdisk_3d.py:97-109: the disk's density into odata."""
        _DiskComponent.evaluate(self, driver, params, None, None, None, None, odata, None,
                                spat_size, spat_step, spat_zero, spat_rota, 1, 0.0, 0.0, dtype,
                                out_extra)


class GModelIntensity2D:
    """intensity_2d.py: thin brightness components into an image."""

    @staticmethod
    def type():
        return 'intensity_2d'

    def __init__(self, components):
        self._components = _lst(components)
        if not self._components:
            raise RuntimeError("at least one component must be configured")
        self._pdescs, self._mappings = _merge([c.pdescs() for c in self._components], 'cmp')
        self._wdata = None
        self._size = None

    def pdescs(self):
        return self._pdescs

    def has_weights(self):
        return any(c.has_weights() for c in self._components)

    def evaluate_image(self, driver, params, image_d, image_w, size, step, zero, rota, dtype,
                       out_extra):
        """intensity_2d.py:76-116."""
        size, step, zero = tuple(size), tuple(step), tuple(zero)
        if image_w is not None and (self._wdata is None or self._size != size):
            self._wdata = driver.mem_alloc_d(size[::-1], dtype)
        self._size = size
        if self._wdata is not None:
            driver.mem_fill(self._wdata, 0)
        for i, (c, m) in enumerate(zip(self._components, self._mappings)):
            cp = {p: params[m[p]] for p in c.pdescs()}
            ce = {} if out_extra is not None else None
            c.evaluate(driver, cp, image_d, self._wdata, None, size, step, zero, rota, dtype, ce)
            if ce:
                out_extra.update({f'component{i}_{k}': v for k, v in ce.items()})
        if image_w is not None:
            self._components[0]._backend.wcube_evaluate(size + (1,), 1, self._wdata, image_w)


class GModelIntensity3D:
    """intensity_3d.py: thick brightness components, optionally behind
    opacity components, into an image.  The spatial z axis is sized like the
    longer of x and y, with that axis' step, centred (intensity_3d.py:88-110),
    unless given."""

    @staticmethod
    def type():
        return 'intensity_3d'

    def __init__(self, components, opacity_components=None, size_z=None, step_z=None,
                 zero_z=None):
        self._components = _lst(components)
        self._ocomponents = _lst(opacity_components)
        if not self._components:
            raise RuntimeError("at least one component must be configured")
        # intensity_3d.py / _detail.py:339-342: components as 'cmp<i>_' from the
        # second on, opacity components always prefixed ('ocmp_', 'ocmp1_', ...)
        p, self._mappings = _merge([c.pdescs() for c in self._components], 'cmp')
        op, self._omappings = _merge([c.pdescs() for c in self._ocomponents], 'ocmp', True)
        self._pdescs = dict(p, **op)
        self._z = (size_z, step_z, zero_z)
        self._key = None
        self._wdata = self._odata = None

    def pdescs(self):
        return self._pdescs

    def has_weights(self):
        return any(c.has_weights() for c in self._components)

    def spatial(self, size, step):
        sx, sy = size[0], size[1]
        i = int(sx < sy)
        sz = self._z[0] if self._z[0] is not None else (sx, sy)[i]
        stz = self._z[1] if self._z[1] is not None else (step[0], step[1])[i]
        zz = self._z[2] if self._z[2] is not None else -(sz / 2 - 0.5) * stz
        return sz, stz, zz

    def evaluate_image(self, driver, params, image_d, image_w, size, step, zero, rota, dtype,
                       out_extra):
        """intensity_3d.py:121-190 (the opacity cube is zeroed per call)."""
        sz, stz, zz = self.spatial(size, step)
        spat_size = (size[0], size[1], sz)
        spat_step = (step[0], step[1], stz)
        spat_zero = (zero[0], zero[1], zz)
        key = (spat_size, image_w is not None)
        if self._key != key:
            self._wdata = driver.mem_alloc_d(spat_size[::-1], dtype) if image_w is not None \
                else None
            self._odata = driver.mem_alloc_d(spat_size[::-1], dtype) if self._ocomponents \
                else None
            self._key = key
        if self._wdata is not None:
            driver.mem_fill(self._wdata, 0)
        if self._odata is not None:
            driver.mem_fill(self._odata, 0)
            for i, (c, m) in enumerate(zip(self._ocomponents, self._omappings)):
                cp = {p: params[m[p]] for p in c.pdescs()}
                ce = {} if out_extra is not None else None
                c.evaluate(driver, cp, self._odata, spat_size, spat_step, spat_zero, rota,
                           dtype, ce)
                if ce:
                    out_extra.update({f'opacity_component{i}_{k}': v for k, v in ce.items()})
        for i, (c, m) in enumerate(zip(self._components, self._mappings)):
            cp = {p: params[m[p]] for p in c.pdescs()}
            ce = {} if out_extra is not None else None
            c.evaluate(driver, cp, self._odata, image_d, self._wdata, None, None, spat_size,
                       spat_step, spat_zero, rota, dtype, ce)
            if ce:
                out_extra.update({f'component{i}_{k}': v for k, v in ce.items()})
        if image_w is not None:
            self._components[0]._backend.wcube_evaluate(spat_size, 1, self._wdata, image_w)


class DModelImage:
    """dmodels/image.py: a PSF-convolved image (DCube of size (nx, ny, 1))."""

    @staticmethod
    def type():
        return 'image'

    def __init__(self, size, step=(1, 1), rpix=None, rval=(0, 0), rota=0, scale=(1, 1),
                 psf=None, mask_cutoff=None, mask_apply=False, dtype='float32'):
        if rpix is None:
            rpix = tuple((np.array(size) / 2 - 0.5).tolist())
        self._dcube = DCube(tuple(size) + (1,), tuple(step) + (0,), tuple(rpix) + (0,),
                            tuple(rval) + (0,), rota, tuple(scale) + (1,), psf, None, False,
                            mask_cutoff, mask_apply, dtype)
        self._driver = self._gmodel = None

    def keys(self):
        return ['image']

    def size(self):
        return self._dcube.size()[:2]

    def step(self):
        return self._dcube.step()[:2]

    def zero(self):
        return self._dcube.zero()[:2]

    def dtype(self):
        return self._dcube.dtype()

    def dcube(self):
        return self._dcube

    def evaluate(self, driver, gmodel, params, out_extra=None):
        """image.py:91-123."""
        dc = self._dcube
        if self._driver is not driver or self._gmodel is not gmodel:
            dc.prepare(driver, gmodel.has_weights())
            self._driver, self._gmodel = driver, gmodel
        driver.mem_fill(dc.scratch_dcube(), 0)
        gmodel.evaluate_image(driver, params, dc.scratch_dcube(), dc.scratch_wcube(),
                              dc.scratch_size()[:2], dc.scratch_step()[:2],
                              dc.scratch_zero()[:2], dc.rota(), dc.dtype(), out_extra)
        dc.evaluate(out_extra)
        m, w = dc.mcube(), dc.wcube()
        return dict(image=dict(d=dc.dcube()[0], m=None if m is None else m[0],
                               w=None if w is None else w[0]))


class DModelLSlit:
    """dmodels/lslit.py: a long-slit spectrum, the spectral model on a slit
    one pixel wide (DCube of size (nx, 1, nz)), PSF x LSF convolved; the
    data are the slit's (nz, nx) plane."""

    @staticmethod
    def type():
        return 'lslit'

    def __init__(self, size, step=(1, 1, 1), rpix=None, rval=(0, 0, 0), rota=0,
                 scale=(1, 1, 1), psf=None, lsf=None, weight=1, mask_cutoff=None,
                 mask_apply=False, dtype='float32'):
        size = tuple(size)
        if rpix is None:
            rpix = (size[0] / 2 - 0.5, 0.0, size[1] / 2 - 0.5)
        self._dcube = DCube((size[0], 1, size[1]), tuple(step), tuple(rpix), tuple(rval), rota,
                            tuple(scale), psf, lsf, weight, mask_cutoff, mask_apply, dtype)
        self._driver = self._gmodel = None

    def keys(self):
        return ['lslit']

    def size(self):
        return self._dcube.size()

    def step(self):
        return self._dcube.step()

    def zero(self):
        return self._dcube.zero()

    def dtype(self):
        return self._dcube.dtype()

    def dcube(self):
        return self._dcube

    def evaluate(self, driver, gmodel, params, out_extra=None):
        """lslit.py:95-128."""
        dc = self._dcube
        if self._driver is not driver or self._gmodel is not gmodel:
            dc.prepare(driver, gmodel.has_weights())
            self._driver, self._gmodel = driver, gmodel
        driver.mem_fill(dc.scratch_dcube(), 0)
        gmodel.evaluate_scube(driver, params, dc.scratch_dcube(), dc.scratch_wcube(),
                              dc.scratch_size(), dc.scratch_step(), dc.scratch_zero(), dc.rota(),
                              dc.dtype(), out_extra)
        dc.evaluate(out_extra)
        m, w = dc.mcube(), dc.wcube()
        return dict(lslit=dict(d=dc.dcube()[:, 0, :], m=None if m is None else m[:, 0, :],
                               w=None if w is None else w[:, 0, :]))


__all__ = ['BrightnessSMDisk2D', 'BrightnessSMDisk3D', 'BrightnessMCDisk3D', 'OpacitySMDisk3D',
           'GModelIntensity2D', 'GModelIntensity3D', 'DModelImage', 'DModelLSlit']
