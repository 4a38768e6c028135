"""The benchmarked configuration itself against the oracle.

The batched workload at full size (512 parameter sets, 128x128x96 cube, 30
rings, Gaussian PSF FWHM 3 px x Gaussian LSF FWHM 1.5 channels, chi^2 against
the seeded noisy data cube), evaluated by the evaluator the benchmark builds:
direct (separable FIR) convolution with the trimmed 17/9 taps, one 512-set
wave, replayed from a captured CUDA graph.  Sets spread over the wave are
checked against the fp64 oracle chain (smdisk on the padded grid, FFT
convolution with the reference's PSF x LSF cube, crop, chi^2:
gmodels.hpp:646-958, _dcube.py:245-313, objective.hpp:8-31):

* model cube: normwise relative error <= max(1e-5, 1.5 x the reference fp32
  path's own error against fp64);
* chi^2: relative error <= 1e-4.

Every other shape the autotuner can pick for this workload (sets per wave,
output rows per PSF block, PSF kernel variants)
gives the same chi^2 and model cubes within fp32 rounding.
"""

import numpy as np
import pytest

from tests.helpers import rel_err

pytestmark = pytest.mark.gpu

NSETS = 512
SAMPLED = (0, 37, 128, 255, 256, 383, 450, 511)


@pytest.fixture(scope='module')
def headline(gpu):
    import torch
    from gbkfit_b200 import workloads
    from gbkfit_b200.batched import BatchedSMDisk, synthetic_data
    w = workloads.smdisk_batch128(nsets=NSETS)
    data, err, _ = synthetic_data(w)
    ev = BatchedSMDisk(w.disk, w.geom, data, err, max_sets=NSETS, chunk=NSETS, conv='direct')
    bufs = ev.alloc_inputs(NSETS)
    ev.upload(ev.pack(w.params, NSETS), bufs, NSETS)
    ev.capture(bufs, NSETS)
    ev.chi2.zero_()
    ev.replay()
    torch.cuda.synchronize()
    chi2 = ev.chi2[:NSETS].cpu().numpy().copy()
    # the sampled sets' model cubes, from the same kernels (the model output
    # is an extra store of the cropped cube)
    nx, ny, nz = w.geom.size
    model = torch.zeros((NSETS, nz, ny, nx), device='cuda')
    chi2_m = ev.evaluate_device(bufs, NSETS, model=model).cpu().numpy().copy()
    cubes = {i: model[i].cpu().numpy() for i in SAMPLED}
    del model
    torch.cuda.empty_cache()
    return dict(w=w, data=data, err=err, ev=ev, bufs=bufs, chi2=chi2, chi2_m=chi2_m, cubes=cubes)


def test_headline_configuration(headline):
    """The wave is the benchmark's: direct mode, trimmed taps, one wave."""
    ev = headline['ev']
    assert ev.conv_mode == 'direct' and ev.psf_rank == 1 and ev.chunk == NSETS
    assert tuple(headline['w'].geom.size) == (128, 128, 96)
    assert len(headline['w'].disk.rnodes) == 30
    # the model output does not change chi^2
    assert np.array_equal(headline['chi2'], headline['chi2_m'])
    assert np.all(np.isfinite(headline['chi2'])) and np.all(headline['chi2'] > 0)


@pytest.mark.parametrize('i', SAMPLED)
def test_headline_set_vs_fp64_oracle(headline, oracle_built, i):
    from gbkfit_b200 import workloads
    from oracle.oracle import chi2, scube_pipeline
    w = headline['w']
    p = w.disk.pack(workloads.set_params(w, i))
    ref64 = scube_pipeline(p, w.geom, precision='f64')
    ref32 = scube_pipeline(p, w.geom, precision='f32')
    cpu = rel_err(ref32, ref64)
    e = rel_err(headline['cubes'][i], ref64)
    assert e <= max(1e-5, 1.5 * cpu), (i, e, cpu)
    c_ref = chi2(ref64, headline['data'], headline['err'])
    got = float(headline['chi2'][i])
    assert abs(got - c_ref) / c_ref <= 1e-4, (i, got, c_ref)


@pytest.mark.parametrize('cfg', [dict(chunk=32), dict(chunk=128), dict(chunk=256),
                                 dict(chunk=512, band=96), dict(chunk=512, band=64),
                                 dict(chunk=512, band=48), dict(chunk=512, band=32),
                                 dict(chunk=512, psf_variant=1), dict(chunk=512, psf_variant=2),
                                 dict(chunk=512, psf_variant=3), dict(chunk=512, psf_variant=4),
                                 dict(chunk=512, psf_variant=5),
                                 dict(chunk=512, band=64, psf_variant=2),
                                 dict(chunk=512, model_variant=0),
                                 dict(chunk=512, model_variant=1), dict(chunk=512, model_variant=2),
                                 dict(chunk=512, model_variant=3),
                                 dict(chunk=128, model_variant=2, psf_variant=6),
                                 dict(chunk=512, psf_variant=6), dict(chunk=512, band=48, psf_variant=6),
                                 dict(chunk=128, psf_variant=6), dict(chunk=512, psf_variant=7),
                                 dict(chunk=512, band=48, psf_variant=7)])
def test_headline_tuner_shapes_agree(headline, cfg):
    """The other direct-mode shapes of the autotuner's search give the same
    results: chi^2 of all 512 sets within 1e-6 relative, sampled cubes
    within 1e-6 normwise."""
    import torch
    from gbkfit_b200.batched import BatchedSMDisk
    w = headline['w']
    ev = BatchedSMDisk(w.disk, w.geom, headline['data'], headline['err'], max_sets=NSETS,
                       conv='direct', **cfg)
    bufs = ev.alloc_inputs(NSETS)
    ev.upload(ev.pack(w.params, NSETS), bufs, NSETS)
    nx, ny, nz = w.geom.size
    model = torch.zeros((NSETS, nz, ny, nx), device='cuda')
    got = ev.evaluate_device(bufs, NSETS, model=model).cpu().numpy()
    ref = headline['chi2']
    assert np.max(np.abs(got - ref) / ref) <= 1e-6, cfg
    for i in SAMPLED[::2]:
        assert rel_err(model[i].cpu().numpy(), headline['cubes'][i]) <= 1e-6, (cfg, i)
    ev.close()
