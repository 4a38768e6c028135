"""The data-model classes end to end on the GPU (gbkfit_b200.model, the
reference's dmodels/scube.py and mmaps.py on the drop-in driver), against the
oracle's restatement of the DCube chain (oracle.dcube_pipeline: padded
high-resolution grid, smdisk, FFT PSF x LSF convolution, downscale, mask;
_dcube.py:128-313, dmodels.hpp:8-74) and of the moments (dmodels.hpp:77-228):

* DModelSCube with supersampling (scale (2, 2, 1) and (1, 1, 2)) and a
  mask cutoff applied to the cube;
* DModelMMaps on the plain smdisk configuration (64^3 cube, Gaussian PSF
  FWHM 2.5 px x LSF FWHM 2 channels): moment 0/1/2 maps of the convolved,
  cropped cube, against the fp64 chain and the compiled reference's moments.

Tolerances: cubes normwise <= max(1e-5, 1.5 x the fp32 CPU chain's own error);
mask maps identical except where the fp64 value is within 1e-5 of the peak
of the cutoff; moment maps per order <= max(1e-5, 2 x the fp32 CPU chain's
error) on the unmasked spaxels, NaN elsewhere."""

import numpy as np
import pytest

from tests.helpers import rel_err

pytestmark = pytest.mark.gpu


def _model(dm, w):
    from gbkfit_b200 import model as M
    from gbkfit_b200.driver import DriverB200
    comp = M.SpectralSMDisk2D(False, False, w.disk.traits['rpt'], w.disk.traits['vpt'],
                              w.disk.traits['dpt'], rnodes=w.disk.rnodes)
    return M.Model(DriverB200(0), dm, M.GModelKinematics2D([comp]))


@pytest.mark.parametrize('scale', [(2, 2, 1), (1, 1, 2)])
def test_scube_supersampled_masked(gpu, oracle_built, scale):
    from gbkfit_b200 import model as M, workloads
    from oracle.oracle import dcube_pipeline
    w = workloads.smdisk_cube64()
    size, step = (40, 36, 32), (1.0, 1.0, 10.0)
    rpix, rval = (0.0, 0.0, 15.5), (0.0, 0.0, 0.0)
    params = dict(w.params, xpos=20.3, ypos=17.6)
    g = w.geom
    cutoff = 2e-4
    dm = M.DModelSCube(size, step, rpix=rpix, rval=rval, scale=scale, psf=g.psf, lsf=g.lsf,
                       mask_cutoff=cutoff, mask_apply=True)
    out = _model(dm, w).evaluate_h(params)['scube']
    p = w.disk.pack(params)
    d64, m64 = dcube_pipeline(p, size, step, rpix, rval, scale, g.psf, g.lsf, 'f64', cutoff, True)
    d32, m32 = dcube_pipeline(p, size, step, rpix, rval, scale, g.psf, g.lsf, 'f32', cutoff, True)
    near = np.abs(np.abs(np.nan_to_num(d64)) - cutoff) <= 1e-5 * np.nanmax(np.abs(d64))
    assert np.nanmax(d64) > 10 * cutoff and 0 < m64.sum() < m64.size
    assert np.all((out['m'] == m64) | near)
    fin = np.isfinite(out['d']) & np.isfinite(d64)
    assert np.all(np.isfinite(out['d']) == (out['m'] > 0))
    cpu = rel_err(d32[fin], d64[fin])
    assert rel_err(out['d'][fin], d64[fin]) <= max(1e-5, 1.5 * cpu)


def test_mmaps_c0_chain(gpu, oracle_built):
    """The plain smdisk configuration through DModelMMaps: smdisk on the
    padded 96^3 grid -> FFT convolution -> crop -> moments 0, 1, 2."""
    from gbkfit_b200 import model as M, workloads
    from oracle.oracle import Oracle, Reference, dcube_pipeline
    w = workloads.smdisk_cube64()
    g = w.geom
    size, step, rpix, rval = g.size, g.step, (0.0, 0.0, 31.5), (0.0, 0.0, 0.0)
    orders = (0, 1, 2)
    dm = M.DModelMMaps(size, step, rpix=rpix, rval=rval, psf=g.psf, lsf=g.lsf, orders=orders)
    out = _model(dm, w).evaluate_h(w.params)
    p = w.disk.pack(w.params)
    zero = tuple(rval[i] - rpix[i] * step[i] for i in range(3))
    o = np.array(orders, np.int32)
    c64, _ = dcube_pipeline(p, size, step, rpix, rval, (1, 1, 1), g.psf, g.lsf, 'f64')
    # the fp32 chain as the reference driver runs it: fp32 smdisk, FFTW-like
    # single-precision FFT, fp32 moments
    c32, _ = dcube_pipeline(p, size, step, rpix, rval, (1, 1, 1), g.psf, g.lsf, 'f32',
                            fft_f32=True)
    md64, mm64, _ = Oracle('f64').mmaps_moments(size, step, zero, c64, None, 1e-6, o)
    md32, _, _ = Oracle('f32').mmaps_moments(size, step, zero, c32, None, 1e-6, o)
    v = mm64 > 0
    assert v.sum() > 1000
    # moments 1 and 2 divide by m0: on spaxels with m0 near the cutoff (1e-6,
    # against a peak of ~1.6) the fp32 convolution's noise (~1e-8 a voxel)
    # dominates them in any fp32 chain, the reference's included; they are
    # compared where m0 >= 1e-3 of its peak
    m0 = np.where(v, md64[0], 0.0)
    strong = v & (np.abs(m0) >= 1e-3 * np.max(np.abs(m0)))
    assert strong.sum() > 1000
    for i, order in enumerate(orders):
        got = out[f'mmap{order}']['d']
        assert np.array_equal(np.isfinite(got[strong]), np.ones(strong.sum(), bool)), order
        sel = v if order == 0 else strong
        assert np.array_equal(np.isnan(got[~v]), np.ones((~v).sum(), bool)), order
        cpu = rel_err(md32[i][sel], md64[i][sel])
        assert rel_err(got[sel], md64[i][sel]) <= max(1e-5, 2 * cpu), (order, cpu)
    if Reference.available():
        rd, rm, _ = Reference().mmaps_moments(size, step, zero, c32, None, 1e-6, o)
        assert np.array_equal(rm > 0, v)
        for i, order in enumerate(orders):
            got = out[f'mmap{order}']['d']
            sel = v if order == 0 else strong
            cpu = rel_err(md32[i][sel], md64[i][sel])
            assert rel_err(got[sel], rd[i][sel]) <= max(1e-5, 3 * cpu), order
