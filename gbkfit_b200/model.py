"""Galaxy models, data models and the objective on the B200 driver.

Host-side mirror of the reference's model-evaluation callers, kept to the
spectral-cube path:

* disk components ``SpectralSMDisk2D`` / ``SpectralSMDisk3D`` /
  ``SpectralMCDisk3D`` (gmodels/spectral_{smdisk_2d,smdisk_3d,mcdisk_3d}.py)
  on top of ``Disk`` packing (gmodels/_disk.py:377-613, _smdisk.py,
  _mcdisk.py);
* galaxy models ``GModelKinematics2D`` / ``GModelKinematics3D``
  (gmodels/kinematics_{2d,3d}.py), components merged with the 'cmp' prefix;
* ``DCube`` (dmodels/_dcube.py: padding, PSF x LSF cube, cached FFT
  convolution, crop/downscale, mask) and the data models ``DModelSCube``
  (dmodels/scube.py) and ``DModelMMaps`` (dmodels/mmaps.py);
* ``Model`` and ``Objective`` (model/model.py, objective/objective.py:
  residual, residual sum, log-likelihood = -chi^2 / 2).

The reference's own Python model path raises at HEAD (components call a
``params()`` method no class defines, _detail.py:392-430; DModelSCube passes
13 arguments to the 12-argument DCube, scube.py:61-63); these classes follow
the evident intent of that code.  Every evaluation is the plain per-call path:
one native call per stage, synchronous like the reference.
"""

import numpy as np
import torch

from . import traits as tr
from .disk import Disk, KINDS
from .workloads import fft_optimal_shape


def _merge(pdesc_list, prefix, zero_prefix=False):
    """utils/miscutils.py:70-95 with zero_index = False: component i > 0 gets
    '<prefix><i>_', component 0 gets '<prefix>_' with zero_prefix, else none."""
    merged, maps = {}, []
    for i, d in enumerate(pdesc_list):
        m = {}
        for name, v in d.items():
            new = f'{prefix}{i}_{name}' if i else (f'{prefix}_{name}' if zero_prefix else name)
            m[name] = new
            merged[new] = v
        maps.append(m)
    return merged, maps


class _DiskComponent:
    """Packs a disk's parameters into device arrays and calls the backend."""

    MC = False

    def __init__(self, disk, cflux=None):
        self._disk = disk
        self._cflux = cflux
        self._driver = None
        self._dev = None
        self._backend = None

    def pdescs(self):
        return self._disk.pdescs

    def has_weights(self):
        return bool(self._disk.traits['wpt'])

    def disk(self):
        return self._disk

    def _prepare(self, driver, dtype):
        self._driver = driver
        self._backend = driver.backends().gmodel(dtype)
        d = self._disk
        dev = {}
        dev['subrnodes'] = driver.mem_copy_h2d(d.subrnodes.astype(np.float32))
        # the per-call parameter arrays (common parameters, trait parameter
        # values) share one device buffer, filled from one pinned host buffer
        # by one copy per evaluation
        sizes = [(name, d.common_size(name)) for name in ('vsys', 'xpos', 'ypos', 'posa', 'incl')
                 if name in d.pdescs]
        sizes += [(k, max(d.tables[k]['npv'], 1)) for k in KINDS if d.tables[k] is not None]
        total = sum(n for _, n in sizes)
        self._flat_d = torch.empty(total, dtype=torch.float32, device=driver.stream.device)
        self._flat_h = torch.empty(total, dtype=torch.float32, pin_memory=True)
        views, off = {}, 0
        for name, n in sizes:
            views[name] = (self._flat_d[off:off + n], self._flat_h[off:off + n].numpy())
            off += n
        self._views = views
        for name in ('vsys', 'xpos', 'ypos', 'posa', 'incl'):
            dev[name] = views[name][0] if name in views else None
        for k in KINDS:
            t = d.tables[k]
            if t is None:
                dev[k] = None
                continue
            dev[k] = dict(uids=driver.mem_copy_h2d(t['uids']),
                          cvalues=driver.mem_copy_h2d(t['cvalues']) if len(t['cvalues'])
                          else driver.mem_alloc_d(1, np.float32),
                          ccounts=driver.mem_copy_h2d(t['ccounts']),
                          pvalues=views[k][0],
                          pcounts=driver.mem_copy_h2d(t['pcounts']))
        if self.MC:
            dev['hasordint'] = driver.mem_copy_h2d(d.hasordint())
            ncsum = sum(1 if h else d.nsub - 2 for h in d.hasordint())
            dev['ncloudscsum'] = driver.mem_alloc_d(ncsum, np.int32)
        self._dev = dev

    def evaluate(self, driver, params, odata, image, scube, wdata, rdata, ordata,
                 spat_size, spat_step, spat_zero, spat_rota, spec_size, spec_step, spec_zero,
                 dtype, out_extra):
        """_disk.py:466-613."""
        if self._driver is not driver:
            self._prepare(driver, dtype)
        d, dev = self._disk, self._dev
        packed = d.pack(params)
        for name in ('vsys', 'xpos', 'ypos', 'posa', 'incl'):
            if dev[name] is not None:
                self._views[name][1][:] = packed[name]
        for k in KINDS:
            if dev[k] is not None and packed[k]['pvalues'].size:
                self._views[k][1][:packed[k]['pvalues'].size] = packed[k]['pvalues']
        # one copy on the driver's stream, ahead of the native call on the same
        # stream; the call synchronises before returning, so the pinned buffer
        # is free again for the next evaluation
        with torch.cuda.stream(driver.stream):
            self._flat_d.copy_(self._flat_h, non_blocking=True)
        shape = tuple(spat_size[::-1])
        extra = {}
        if out_extra is not None:
            dv = dev['subrnodes'].device
            if d.traits['rpt']:
                extra['rdata_cmp'] = torch.zeros(shape, device=dv)
            if d.traits['vpt']:
                extra['vdata_cmp'] = torch.full(shape, np.nan, device=dv)
            if d.traits['dpt']:
                extra['ddata_cmp'] = torch.full(shape, np.nan, device=dv)
        tset = []
        for k in KINDS:
            t = dev[k]
            tset += [None] * 5 if t is None else [t['uids'], t['cvalues'], t['ccounts'],
                                                  t['pvalues'], t['pcounts']]
        common = (d.loose, d.tilted, dev['subrnodes'], dev['vsys'], dev['xpos'], dev['ypos'],
                  dev['posa'], dev['incl'], *tset, odata, spat_size, spat_step, spat_zero,
                  spat_rota, spec_size, spec_step, spec_zero, image, scube, wdata, None,
                  rdata, extra.get('rdata_cmp'), ordata, None, extra.get('vdata_cmp'),
                  extra.get('ddata_cmp'))
        if self.MC:
            csum = d.ncloudscsum(params, self._cflux)
            dev['ncloudscsum'].copy_(torch.from_numpy(csum))
            self._backend.mcdisk_evaluate(self._cflux, int(csum[-1]), dev['ncloudscsum'],
                                          dev['hasordint'], *common)
        else:
            self._backend.smdisk_evaluate(*common)
        if out_extra is not None:
            key = 'odata' if d.opacity else 'bdata'
            if 'rdata_cmp' in extra:
                out_extra[key] = extra['rdata_cmp'].cpu().numpy()
            if 'vdata_cmp' in extra:
                out_extra['vdata'] = extra['vdata_cmp'].cpu().numpy()
            if 'ddata_cmp' in extra:
                out_extra['ddata'] = extra['ddata_cmp'].cpu().numpy()


def _rnodes(rnmin, rnmax, rnsep, rnlen, rnodes):
    """gmodels/_detail.py:14-52."""
    if rnodes is not None:
        return np.asarray(rnodes, dtype=np.float64)
    if rnsep is not None:
        return np.arange(rnmin, rnmax + rnsep, rnsep)
    return np.linspace(rnmin, rnmax, rnlen)


class SpectralSMDisk2D(_DiskComponent):
    """gmodels/spectral_smdisk_2d.py: thin smooth disk."""

    @staticmethod
    def type():
        return 'smdisk'

    def __init__(self, loose, tilted, bptraits, vptraits, dptraits, sptraits=None,
                 wptraits=None, rnmin=None, rnmax=None, rnsep=None, rnlen=None, rnodes=None,
                 rstep=None, interp='linear'):
        lst = lambda x: [] if x is None else list(x) if isinstance(x, (list, tuple)) else [x]
        disk = Disk(loose, tilted, _rnodes(rnmin, rnmax, rnsep, rnlen, rnodes), rstep, interp,
                    dict(rpt=lst(bptraits), vpt=lst(vptraits), dpt=lst(dptraits),
                         spt=lst(sptraits), wpt=lst(wptraits)))
        super().__init__(disk)

    def evaluate(self, driver, params, scube, wdata, bdata, spat_size, spat_step, spat_zero,
                 spat_rota, spec_size, spec_step, spec_zero, dtype, out_extra):
        """spectral_smdisk_2d.py:135-148: spatial z of size 1."""
        super().evaluate(driver, params, None, None, scube, wdata, bdata, None,
                         tuple(spat_size) + (1,), tuple(spat_step) + (0,),
                         tuple(spat_zero) + (0,), spat_rota, spec_size, spec_step, spec_zero,
                         dtype, out_extra)


class SpectralSMDisk3D(_DiskComponent):
    """gmodels/spectral_smdisk_3d.py: thick smooth disk."""

    @staticmethod
    def type():
        return 'smdisk'

    def __init__(self, loose, tilted, bptraits, vptraits, dptraits, bhtraits, vhtraits=None,
                 dhtraits=None, zptraits=None, sptraits=None, wptraits=None, rnmin=None,
                 rnmax=None, rnsep=None, rnlen=None, rnodes=None, rstep=None, interp='linear'):
        lst = lambda x: [] if x is None else list(x) if isinstance(x, (list, tuple)) else [x]
        bp, bh = lst(bptraits), lst(bhtraits)
        vp, dp = lst(vptraits), lst(dptraits)
        vh = lst(vhtraits) or [tr.vht_one() for _ in vp]
        dh = lst(dhtraits) or [tr.dht_one() for _ in dp]
        disk = Disk(loose, tilted, _rnodes(rnmin, rnmax, rnsep, rnlen, rnodes), rstep, interp,
                    dict(rpt=bp, rht=bh, vpt=vp, vht=vh, dpt=dp, dht=dh, zpt=lst(zptraits),
                         spt=lst(sptraits), wpt=lst(wptraits)))
        super().__init__(disk)


class SpectralMCDisk3D(SpectralSMDisk3D):
    """gmodels/spectral_mcdisk_3d.py: Monte-Carlo cloud disk."""

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


class GModelKinematics2D:
    """gmodels/kinematics_2d.py."""

    @staticmethod
    def type():
        return 'kinematics_2d'

    def __init__(self, components):
        self._components = list(components) if isinstance(components, (list, tuple)) \
            else [components]
        self._pdescs, self._mappings = _merge([c.pdescs() for c in self._components], 'cmp')
        self._wdata = None
        self._size = None

    def pdescs(self):
        return self._pdescs

    def has_weights(self):
        return any(c.has_weights() for c in self._components)

    def evaluate_scube(self, driver, params, scube_d, scube_w, size, step, zero, rota, dtype,
                       out_extra):
        spat_size, spat_step, spat_zero = tuple(size[:2]), tuple(step[:2]), tuple(zero[:2])
        if scube_w is not None and (self._wdata is None or self._size != spat_size):
            self._wdata = driver.mem_alloc_d(spat_size[::-1], dtype)
        self._size = spat_size
        if self._wdata is not None:
            driver.mem_fill(self._wdata, 0)
        for i, (c, m) in enumerate(zip(self._components, self._mappings)):
            cp = {p: params[m[p]] for p in c.pdescs()}
            ce = {} if out_extra is not None else None
            c.evaluate(driver, cp, scube_d, self._wdata, None, spat_size, spat_step, spat_zero,
                       rota, size[2], step[2], zero[2], dtype, ce)
            if ce:
                out_extra.update({f'component{i}_{k}': v for k, v in ce.items()})
        if scube_w is not None:
            c0 = self._components[0]
            c0._backend.wcube_evaluate(spat_size + (1,), size[2], self._wdata, scube_w)


class GModelKinematics3D(GModelKinematics2D):
    """gmodels/kinematics_3d.py: spatial z sized like the longer of x and y,
    centred (kinematics_3d.py:96-109)."""

    @staticmethod
    def type():
        return 'kinematics_3d'

    def __init__(self, components, size_z=None, step_z=None, zero_z=None):
        super().__init__(components)
        self._z = (size_z, step_z, zero_z)

    def evaluate_scube(self, driver, params, scube_d, scube_w, size, step, zero, rota, dtype,
                       out_extra):
        sx, sy = size[0], size[1]
        i = int(sx < sy)
        sz = self._z[0] if self._z[0] is not None else (sx, sy)[i]
        stz = self._z[1] if self._z[1] is not None else (step[0], step[1])[i]
        zz = self._z[2] if self._z[2] is not None else -(sz / 2 - 0.5) * stz
        spat_size, spat_step, spat_zero = (sx, sy, sz), (step[0], step[1], stz), (zero[0],
                                                                                zero[1], zz)
        wdata = None
        if scube_w is not None:
            wdata = driver.mem_alloc_d(spat_size[::-1], dtype)
            driver.mem_fill(wdata, 0)
        for i, (c, m) in enumerate(zip(self._components, self._mappings)):
            cp = {p: params[m[p]] for p in c.pdescs()}
            ce = {} if out_extra is not None else None
            _DiskComponent.evaluate(c, driver, cp, None, None, scube_d, wdata, None, None,
                                    spat_size, spat_step, spat_zero, rota, size[2], step[2],
                                    zero[2], dtype, ce)
            if ce:
                out_extra.update({f'component{i}_{k}': v for k, v in ce.items()})
        if scube_w is not None:
            self._components[0]._backend.wcube_evaluate(spat_size, size[2], wdata, scube_w)


class DCube:
    """dmodels/_dcube.py:17-313."""

    def __init__(self, size, step, rpix, rval, rota, scale, psf, lsf, smooth_weights,
                 mask_cutoff, mask_apply, dtype):
        if mask_apply and mask_cutoff is None:
            mask_apply = False
        if smooth_weights and not (psf or lsf):
            smooth_weights = False
        self._size_lo = tuple(size)
        self._step_lo = tuple(step)
        self._zero_lo = tuple(rval[i] - rpix[i] * step[i] for i in range(3))
        self._rota = rota
        self._scale = tuple(scale)
        self._psf, self._lsf = psf, lsf
        self._smooth_weights = smooth_weights
        self._mask_cutoff = mask_cutoff
        self._mask_apply = mask_apply
        self._dtype = np.dtype(dtype)
        self._driver = None

    def size(self):
        return self._size_lo

    def step(self):
        return self._step_lo

    def zero(self):
        return self._zero_lo

    def rota(self):
        return self._rota

    def dtype(self):
        return self._dtype

    def dcube(self):
        return self._dcube_lo

    def wcube(self):
        return self._wcube_lo

    def mcube(self):
        return self._mcube_lo

    def scratch_size(self):
        return self._size_hi

    def scratch_step(self):
        return self._step_hi

    def scratch_zero(self):
        return self._zero_hi

    def scratch_edge(self):
        return self._edge_hi

    def scratch_dcube(self):
        return self._dcube_hi

    def scratch_wcube(self):
        return self._wcube_hi

    def pcube(self):
        return self._pcube_hi

    def prepare(self, driver, has_weights):
        """_dcube.py:128-243."""
        size_lo, step_lo, zero_lo, scale = self._size_lo, self._step_lo, self._zero_lo, \
            self._scale
        psf, lsf, dtype = self._psf, self._lsf, self._dtype
        self._backend_fft = driver.backends().fft(dtype)
        self._backend_dmodel = driver.backends().dmodel(dtype)
        size_hi = tuple(size_lo[i] * scale[i] for i in range(3))
        step_hi = tuple(step_lo[i] / scale[i] for i in range(3))
        edge_hi = (0, 0, 0)
        if psf or lsf:
            psf_size = psf.size(step_hi[:2]) if psf else (1, 1)
            lsf_size = lsf.size(step_hi[2]) if lsf else 1
            size_hi, edge_hi = self._backend_fft.fft_convolution_shape(
                size_hi, psf_size + (lsf_size,))
        zero_hi = tuple(zero_lo[i] - step_lo[i] / 2 - (edge_hi[i] - 0.5) * step_hi[i]
                        for i in range(3))
        self._pcube_hi = None
        if psf or lsf:
            from .psflsf import LSFPoint, PSFPoint
            off = [(n % 2) - 1 for n in size_hi]
            p = (psf or PSFPoint()).asarray(step_hi[:2], size_hi[:2], (off[0], off[1]))
            l_ = (lsf or LSFPoint()).asarray(step_hi[2], size_hi[2], off[2])
            pc = (p * l_[:, None, None]).astype(dtype)
            pc = self._backend_fft.fft_convolution_shift(pc)
            self._pcube_hi = driver.mem_copy_h2d(np.ascontiguousarray(pc))
        shape_lo, shape_hi = size_lo[::-1], size_hi[::-1]
        self._dcube_lo = driver.mem_alloc_d(shape_lo, dtype)
        driver.mem_fill(self._dcube_lo, 0)
        self._dcube_hi = self._dcube_lo
        if size_lo != size_hi:
            self._dcube_hi = driver.mem_alloc_d(shape_hi, dtype)
            driver.mem_fill(self._dcube_hi, 0)
        self._wcube_lo = self._wcube_hi = None
        if has_weights:
            self._wcube_lo = driver.mem_alloc_d(shape_lo, dtype)
            driver.mem_fill(self._wcube_lo, 1)
            self._wcube_hi = self._wcube_lo
            if size_lo != size_hi:
                self._wcube_hi = driver.mem_alloc_d(shape_hi, dtype)
                driver.mem_fill(self._wcube_hi, 1)
        self._mcube_lo = None
        if self._mask_cutoff:
            self._mcube_lo = driver.mem_alloc_d(shape_lo, dtype)
            driver.mem_fill(self._mcube_lo, 1)
        self._size_hi, self._step_hi, self._zero_hi, self._edge_hi = size_hi, step_hi, \
            zero_hi, edge_hi
        self._driver = driver

    def evaluate(self, out_extra):
        """_dcube.py:245-313."""
        if self._psf or self._lsf:
            self._backend_fft.fft_convolve_cached(self._dcube_hi, self._pcube_hi)
            if self._wcube_lo is not None:
                self._backend_fft.fft_convolve_cached(self._wcube_hi, self._pcube_hi)
        if self._dcube_lo is not self._dcube_hi:
            self._backend_dmodel.dcube_downscale(self._scale, self._edge_hi, self._dcube_hi,
                                                 self._dcube_lo)
            if self._wcube_lo is not None and self._smooth_weights:
                self._backend_dmodel.dcube_downscale(self._scale, self._edge_hi,
                                                     self._wcube_hi, self._wcube_lo)
        if self._mask_cutoff is not None:
            self._backend_dmodel.dcube_mask(self._mask_cutoff, self._mask_apply,
                                            self._mcube_lo, self._dcube_lo, self._wcube_lo)
        if out_extra is not None:
            out_extra.update(dcube_lo=self._dcube_lo.cpu().numpy(),
                             dcube_hi=self._dcube_hi.cpu().numpy())


class DModelSCube:
    """dmodels/scube.py."""

    @staticmethod
    def type():
        return 'scube'

    def __init__(self, size, step=(1, 1, 1), rpix=None, rval=(0, 0, 0), rota=0,
                 scale=(1, 1, 1), psf=None, lsf=None, weight=1, mask_cutoff=None,
                 mask_apply=False, dtype='float32'):
        if rpix is None:
            rpix = tuple((np.array(size) / 2 - 0.5).tolist())
        self._dcube = DCube(tuple(size), tuple(step), tuple(rpix), tuple(rval), rota,
                            tuple(scale), psf, lsf, weight, mask_cutoff, mask_apply, dtype)
        self._driver = self._gmodel = None

    def keys(self):
        return ['scube']

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
        """model/core.py:62-80 + scube.py:95-122."""
        if self._driver is not driver or self._gmodel is not gmodel:
            self._dcube.prepare(driver, gmodel.has_weights())
            self._driver, self._gmodel = driver, gmodel
        dc = self._dcube
        driver.mem_fill(dc.scratch_dcube(), 0)
        gmodel.evaluate_scube(driver, params, dc.scratch_dcube(), dc.scratch_wcube(),
                              dc.scratch_size(), dc.scratch_step(), dc.scratch_zero(), dc.rota(),
                              dc.dtype(), out_extra)
        dc.evaluate(out_extra)
        return dict(scube=dict(d=dc.dcube(), m=dc.mcube(), w=dc.wcube()))


class DModelMMaps:
    """dmodels/mmaps.py."""

    @staticmethod
    def type():
        return 'mmaps'

    def __init__(self, size, step=(1, 1), rpix=None, rval=(0, 0), rota=0, scale=(1, 1),
                 psf=None, lsf=None, mask_cutoff=1e-6, orders=(0, 1, 2), dtype='float32'):
        if rpix is None:
            rpix = tuple((np.array(size) / 2 - 0.5).tolist())
        size, step, rpix, rval, scale = (tuple(size), tuple(step), tuple(rpix), tuple(rval),
                                         tuple(scale))
        orders = tuple(sorted(set(orders)))
        if any(o < 0 or o > 7 for o in orders):
            raise RuntimeError("moment orders must be between 0 and 7")
        if len(step) == 2:
            step = step + (1,)
        if len(size) == 2:
            from .psflsf import _roundu_odd
            size = size + (int(_roundu_odd(1000 / step[2])),)
        if len(rpix) == 2:
            rpix = rpix + (size[2] / 2 - 0.5,)
        if len(rval) == 2:
            rval = rval + (0,)
        if len(scale) == 2:
            scale = scale + (1,)
        if mask_cutoff is None:
            raise RuntimeError("masking cannot be disabled for the mmaps dmodel")
        self._orders = orders
        self._mask_cutoff = mask_cutoff
        self._dcube = DCube(size, step, rpix, rval, rota, scale, psf, lsf, True, None, False,
                            dtype)
        self._driver = self._gmodel = None

    def keys(self):
        return tuple(f'mmap{i}' for i in self._orders)

    def size(self):
        return self._dcube.size()[:2]

    def orders(self):
        return self._orders

    def dcube(self):
        return self._dcube

    def evaluate(self, driver, gmodel, params, out_extra=None):
        """mmaps.py:139-201."""
        dc = self._dcube
        if self._driver is not driver or self._gmodel is not gmodel:
            dc.prepare(driver, gmodel.has_weights())
            self._backend = driver.backends().dmodel(dc.dtype())
            n = len(self._orders)
            ny, nx = self.size()[1], self.size()[0]
            self._o = driver.mem_copy_h2d(np.array(self._orders, np.int32))
            self._d = driver.mem_alloc_d((n, ny, nx), dc.dtype())
            self._m = driver.mem_alloc_d((ny, nx), dc.dtype())
            self._w = driver.mem_alloc_d((n, ny, nx), dc.dtype())
            driver.mem_fill(self._d, np.nan)
            driver.mem_fill(self._m, 0)
            driver.mem_fill(self._w, 1)
            self._driver, self._gmodel = driver, gmodel
        driver.mem_fill(dc.scratch_dcube(), 0)
        gmodel.evaluate_scube(driver, params, dc.scratch_dcube(), dc.scratch_wcube(),
                              dc.scratch_size(), dc.scratch_step(), dc.scratch_zero(), dc.rota(),
                              dc.dtype(), out_extra)
        dc.evaluate(out_extra)
        self._backend.mmaps_moments(dc.size(), dc.step(), dc.zero(), dc.dcube(), dc.wcube(),
                                    self._mask_cutoff, self._o, self._d, self._w, self._m)
        return {key: dict(d=self._d[i], m=self._m, w=self._w[i])
                for i, key in enumerate(self.keys())}


class Model:
    """model/model.py: a (driver, dmodel, gmodel) triple."""

    def __init__(self, driver, dmodel, gmodel):
        self._driver, self._dmodel, self._gmodel = driver, dmodel, gmodel

    def driver(self):
        return self._driver

    def dmodel(self):
        return self._dmodel

    def gmodel(self):
        return self._gmodel

    def pdescs(self):
        return self._gmodel.pdescs()

    def evaluate_d(self, params, out_extra=None):
        return self._dmodel.evaluate(self._driver, self._gmodel, params, out_extra)

    def evaluate_h(self, params, out_extra=None):
        out = self.evaluate_d(params, out_extra)
        return {k: {kk: (None if vv is None else vv.cpu().numpy()) for kk, vv in v.items()}
                for k, v in out.items()}


class Objective:
    """objective/objective.py:133-308 for one model and its data:
    residual = ((mdl - obs) / err) * w_mdl * m_obs * m_mdl * weight,
    chi^2 = sum residual^2, log-likelihood = -chi^2 / 2."""

    def __init__(self, model, data, error=None, mask=None, weight=1.0):
        self._model = model
        drv = model.driver()
        self._backend = drv.backends().objective(np.float32)
        key = model.dmodel().keys()[0]
        self._key = key
        self._obs_d = drv.mem_copy_h2d(np.ascontiguousarray(data, np.float32))
        self._obs_e = None if error is None else drv.mem_copy_h2d(
            np.ascontiguousarray(error, np.float32))
        self._obs_m = None if mask is None else drv.mem_copy_h2d(
            np.ascontiguousarray(mask, np.float32))
        self._weight = float(weight)
        self._res = drv.mem_alloc_d(self._obs_d.numel(), np.float32)
        self._sum = drv.mem_alloc_d(1, np.float32)

    def residual_vector_d(self, params):
        out = self._model.evaluate_d(params)[self._key]
        self._backend.residual(self._obs_d.reshape(-1), self._obs_e, self._obs_m,
                               out['d'].reshape(-1), out['w'], out['m'], self._weight,
                               self._res)
        return self._res

    def residual_scalar(self, params, squared=True):
        res = self.residual_vector_d(params)
        self._backend.residual_sum(res, squared, self._sum)
        return float(self._sum.item())

    def log_likelihood(self, params):
        return -0.5 * self.residual_scalar(params, True)
