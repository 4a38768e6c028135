"""Image and long-slit data models on the GPU (gbkfit_b200.imaging) against
the oracle's DCube chain (oracle.dcube_pipeline with image / opacity
outputs; _dcube.py:128-313, gmodels.hpp:646-958):

* DModelImage of a thin brightness disk (GModelIntensity2D), supersampled
  (scale 2, 2) and PSF-convolved, with a mask;
* DModelImage of a thick brightness disk behind a thick opacity disk
  (GModelIntensity3D with an opacity component);
* DModelLSlit of a thin spectral disk: the (nz, nx) plane of a slit one
  pixel wide, PSF x LSF convolved.

Tolerances as for the cubes: normwise <= max(1e-5, 1.5 x the fp32 CPU
chain's own error against fp64)."""

import numpy as np
import pytest

from tests.helpers import rel_err

pytestmark = pytest.mark.gpu


def _drv():
    from gbkfit_b200.driver import DriverB200
    return DriverB200(0)


def _check(got, c64, c32):
    fin = np.isfinite(c64)
    assert np.array_equal(np.isfinite(got), fin)
    cpu = rel_err(c32[fin], c64[fin])
    e = rel_err(got[fin], c64[fin])
    assert e <= max(1e-5, 1.5 * cpu), (e, cpu)


def test_image_thin_brightness_supersampled(gpu, oracle_built):
    from gbkfit_b200 import model as M, psflsf, traits as T
    from gbkfit_b200.imaging import BrightnessSMDisk2D, DModelImage, GModelIntensity2D
    from oracle.oracle import dcube_pipeline
    comp = BrightnessSMDisk2D(False, False, [T.bpt('exponential'), T.bpt('nw_harmonic', order=2)],
                              rnodes=np.linspace(0, 30, 20))
    gm = GModelIntensity2D([comp])
    psf = psflsf.PSFGauss(psflsf.gauss_fwhm_to_sigma(2.5))
    size, step, rpix, rval, scale = (40, 36), (1.0, 1.0), (0.0, 0.0), (0.0, 0.0), (2, 2)
    cutoff = 1e-3
    dm = DModelImage(size, step, rpix=rpix, rval=rval, scale=scale, psf=psf, mask_cutoff=cutoff,
                     mask_apply=True)
    rn = np.linspace(0, 30, 20)
    params = dict(xpos=20.3, ypos=17.6, posa=45.0, incl=60.0, bpt_a=1.0, bpt_s=8.0,
                  bpt1_a=0.2 * np.exp(-rn / 15), bpt1_p=30 + rn)
    out = M.Model(_drv(), dm, gm).evaluate_h(params)['image']
    p = comp.disk().pack(params)
    args = (p, size + (1,), step + (0.0,), rpix + (0.0,), rval + (0.0,), scale + (1,), psf, None)
    c64, m64 = dcube_pipeline(*args, 'f64', cutoff, True, image=True)
    c32, _ = dcube_pipeline(*args, 'f32', cutoff, True, image=True)
    assert out['d'].shape == (36, 40)
    assert 0 < m64.sum() < m64.size and np.nanmax(c64) > 100 * cutoff
    near = np.abs(np.abs(np.nan_to_num(c64[0])) - cutoff) <= 1e-5 * np.nanmax(c64)
    assert np.all((out['m'] == m64[0]) | near)
    _check(out['d'], c64[0], c32[0])


def test_image_thick_brightness_behind_opacity(gpu, oracle_built):
    from gbkfit_b200 import model as M, psflsf, traits as T
    from gbkfit_b200.imaging import (BrightnessSMDisk3D, DModelImage, GModelIntensity3D,
                                     OpacitySMDisk3D)
    from oracle.oracle import dcube_pipeline
    rn = np.linspace(0, 30, 20)
    comp = BrightnessSMDisk3D(False, False, T.bpt('exponential'), T.bht('sech2'), rnodes=rn)
    opc = OpacitySMDisk3D(False, False, T.opt('exponential'), T.oht('sech2'), rnodes=rn)
    gm = GModelIntensity3D([comp], [opc])
    assert set(gm.pdescs()) >= {'bpt_a', 'bht_s', 'ocmp_opt_a', 'ocmp_oht_s', 'ocmp_xpos'}
    psf = psflsf.PSFGauss(psflsf.gauss_fwhm_to_sigma(2.0))
    size, step = (40, 36), (1.0, 1.0)
    dm = DModelImage(size, step, rpix=(0.0, 0.0), rval=(0.0, 0.0), psf=psf)
    geo = dict(xpos=20.3, ypos=17.6, posa=45.0, incl=70.0)
    params = dict(geo, bpt_a=1.0, bpt_s=8.0, bht_s=1.5,
                  **{f'ocmp_{k}': v for k, v in dict(geo, opt_a=0.2, opt_s=10.0, oht_a=1.0,
                                                      oht_s=2.0).items()})
    drv = _drv()
    got = M.Model(drv, dm, gm).evaluate_h(params)['image']['d']
    bare = M.Model(drv, DModelImage(size, step, rpix=(0.0, 0.0), rval=(0.0, 0.0), psf=psf),
                   GModelIntensity3D([comp])).evaluate_h(
        {k: v for k, v in params.items() if not k.startswith('ocmp_')})['image']['d']
    pb = comp.disk().pack({k: v for k, v in params.items() if not k.startswith('ocmp_')})
    po = opc.disk().pack({k[5:]: v for k, v in params.items() if k.startswith('ocmp_')})
    args = (pb, size + (1,), step + (0.0,), (0.0, 0.0, 0.0), (0.0, 0.0, 0.0), (1, 1, 1), psf,
            None)
    c64, _ = dcube_pipeline(*args, 'f64', thick=True, image=True, opacity_packed=po)
    c32, _ = dcube_pipeline(*args, 'f32', thick=True, image=True, opacity_packed=po)
    _check(got, c64[0], c32[0])
    assert got.sum() < 0.97 * bare.sum()        # the opacity disk absorbs


def test_lslit_thin_spectral(gpu, oracle_built):
    from gbkfit_b200 import model as M, workloads
    from gbkfit_b200.imaging import DModelLSlit
    from oracle.oracle import dcube_pipeline
    w = workloads.smdisk_cube64()
    g = w.geom
    comp = M.SpectralSMDisk2D(False, False, w.disk.traits['rpt'], w.disk.traits['vpt'],
                              w.disk.traits['dpt'], rnodes=w.disk.rnodes)
    size, step = (40, 32), (1.0, 1.0, 10.0)
    rpix, rval = (0.0, 0.0, 15.5), (0.0, 0.0, 0.0)
    dm = DModelLSlit(size, step, rpix=rpix, rval=rval, psf=g.psf, lsf=g.lsf)
    # the slit runs along the major axis through the centre
    params = dict(w.params, xpos=20.3, ypos=0.2, posa=90.0)
    out = M.Model(_drv(), dm, M.GModelKinematics2D([comp])).evaluate_h(params)['lslit']
    p = w.disk.pack(params)
    c64, _ = dcube_pipeline(p, (40, 1, 32), step, rpix, rval, (1, 1, 1), g.psf, g.lsf, 'f64')
    c32, _ = dcube_pipeline(p, (40, 1, 32), step, rpix, rval, (1, 1, 1), g.psf, g.lsf, 'f32')
    assert out['d'].shape == (32, 40) and c64.max() > 0
    _check(out['d'], c64[:, 0, :], c32[:, 0, :])
