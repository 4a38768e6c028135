"""mcdisk at the configuration's full scale: 1e7 clouds of a thick
exponential disk (scale 20 px, sech2 height 2 px, lramp rotation 220 km/s,
dispersion 15 km/s, incl 70, PA 30) into the padded 320 x 320 x 160 grid of
the 256 x 256 x 128 cube (spatial z 320), through the drop-in gmodel backend.

* deterministic mode (64-bit fixed point): bit-identical run to run, the
  spatial flux cube holds whole clouds and every cloud lands in it, so its
  total is exactly nclouds x cflux / (dx dy);
* fast mode (fp32 atomics) agrees with it to fp32 accumulation error;
* against the reference's own compiled mcdisk (oracle/_ref, one thread: one
  mt19937 stream), the clouds agree within shot noise (tests/mcdisk_stats.py).
"""

import numpy as np
import pytest

from tests.helpers import gpu_mcdisk, rel_err, upload
from tests.mcdisk_stats import compare_clouds

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def c1(gpu):
    import torch
    from gbkfit_b200 import workloads
    from gbkfit_b200.driver import DriverB200
    w = workloads.mcdisk_cube256()
    csum = w.disk.ncloudscsum(w.params, w.cflux)
    hoi = w.disk.hasordint()
    n = int(csum[-1])
    g = w.geometry_args()
    nx, ny, sz = g['spat_size']
    nz = g['spec_size']
    packed = w.disk.pack(w.params)
    pd = upload(packed, 'cuda')
    gm = DriverB200(0).backends().gmodel(np.float32)
    cs, hs = torch.from_numpy(csum).cuda(), torch.from_numpy(hoi).cuda()

    def run(mode, seed=42):
        gm.set_mcdisk(seed=seed, mode=mode)
        outs = dict(scube=torch.zeros((nz, ny, nx), device='cuda'),
                    rdata=torch.zeros((sz, ny, nx), device='cuda'))
        gpu_mcdisk(gm, w.cflux, n, cs, hs, pd, g, outs)
        gm.set_mcdisk(seed=42, mode=0)
        return {k: v.cpu().numpy() for k, v in outs.items()}

    return dict(w=w, csum=csum, hoi=hoi, n=n, g=g, packed=packed, run=run,
                per_cloud=w.cflux / (g['spat_step'][0] * g['spat_step'][1]))


def test_c1_scale(c1):
    assert 0.9e7 <= c1['n'] <= 1.1e7
    assert tuple(c1['g']['spat_size']) == (320, 320, 320) and c1['g']['spec_size'] == 160


def test_c1_deterministic_flux_conservation(c1):
    a, b = c1['run'](1), c1['run'](1)
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    counts = a['rdata'].astype(np.float64) / c1['per_cloud']
    assert np.max(np.abs(counts - np.rint(counts))) <= 1e-6 * max(1.0, counts.max())
    # every cloud of the disk lands in the padded cube
    assert int(np.rint(counts.sum())) == c1['n']
    assert abs(a['rdata'].astype(np.float64).sum() - c1['n'] * c1['per_cloud']) <= \
        1e-6 * c1['n'] * c1['per_cloud']
    c1['det'] = a


def test_c1_fast_mode_matches_deterministic(c1):
    det = c1.get('det') or c1['run'](1)
    fast = c1['run'](0)
    assert rel_err(fast['rdata'], det['rdata']) <= 1e-4
    assert rel_err(fast['scube'], det['scube']) <= 1e-5
    assert abs(fast['scube'].astype(np.float64).sum() - det['scube'].astype(np.float64).sum()) \
        <= 1e-5 * det['scube'].astype(np.float64).sum()


@pytest.mark.parametrize('mode', [2, 3])
def test_c1_atomic_modes_match_deterministic(c1, mode):
    """Mode 2 (lines accumulated channel-contiguous with 16-byte vector
    atomics, then added to the cube: mode 0's path) and mode 3 (one fp32
    atomic per channel) sum the same contributions as the deterministic
    mode, to fp32 accumulation error."""
    det = c1.get('det') or c1['run'](1)
    v4 = c1['run'](mode)
    assert np.array_equal(v4['rdata'] != 0, det['rdata'] != 0)
    assert rel_err(v4['rdata'], det['rdata']) <= 1e-4
    assert rel_err(v4['scube'], det['scube']) <= 1e-5
    assert abs(v4['scube'].astype(np.float64).sum() - det['scube'].astype(np.float64).sum()) \
        <= 1e-5 * det['scube'].astype(np.float64).sum()


def test_c1_vs_compiled_reference_shot_noise(c1, oracle_built):
    from oracle.oracle import Reference
    if not Reference.available():
        pytest.skip('oracle/_ref not built')
    g = c1['g']
    nx, ny, sz = g['spat_size']
    nz = g['spec_size']
    ref = Reference()
    nthreads = ref.num_threads()
    ref.set_num_threads(1)
    try:
        a = dict(scube=np.zeros((nz, ny, nx), np.float32),
                 rdata=np.zeros((sz, ny, nx), np.float32))
        ref.mcdisk_evaluate(c1['w'].cflux, c1['n'], c1['csum'], c1['hoi'], c1['packed'], g, a)
    finally:
        ref.set_num_threads(nthreads)
    b = c1.get('det') or c1['run'](1)
    st = compare_clouds(a, b, c1['n'], c1['per_cloud'], sigma_min=c1['w'].params['dpt_a'],
                        spec_step=g['spec_step'])
    assert st['inside'][0] == c1['n'] and st['inside'][1] == c1['n']
