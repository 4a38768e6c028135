"""mcdisk parity with the reference's own compiled mcdisk
(gmodel_mcdisk_evaluate_cloud, gmodels.hpp:326-643, in oracle/_ref), run with
one OpenMP thread so that its clouds come from one mt19937 stream: the
oracle's Philox clouds of the same disk and budget agree with it within shot
noise (tests/mcdisk_stats.py), and both conserve the flux of the clouds that
land in the cube exactly."""

import numpy as np
import pytest

from tests.mcdisk_stats import compare_clouds


def _small_disk():
    from gbkfit_b200 import workloads
    w = workloads.mcdisk_cube256(nclouds=400_000)
    w.geom = workloads.Geometry((64, 64, 32), (1, 1, 10), (0, 0, 15.5), (0, 0, 0),
                                w.geom.psf, w.geom.lsf)
    w.params = dict(w.params, xpos=32.0, ypos=32.0, bpt_s=8.0)
    w.disk = workloads.Disk(False, False, np.linspace(0, 24, 13), traits=w.disk.traits)
    return w


def test_oracle_mcdisk_vs_compiled_reference(oracle_built):
    from oracle.oracle import Oracle, Reference
    if not Reference.available():
        pytest.skip('oracle/_ref not built')
    w = _small_disk()
    cflux = 1e-3
    csum = w.disk.ncloudscsum(w.params, cflux)
    hoi = w.disk.hasordint()
    n = int(csum[-1])
    g = w.geometry_args(spat_z=40)
    nx, ny, sz = g['spat_size']
    nz = g['spec_size']
    packed = w.disk.pack(w.params)

    def outs():
        return dict(scube=np.zeros((nz, ny, nx), np.float32),
                    rdata=np.zeros((sz, ny, nx), np.float32))

    ref = Reference()
    nthreads = ref.num_threads()
    ref.set_num_threads(1)
    try:
        a = outs()
        ref.mcdisk_evaluate(cflux, n, csum, hoi, packed, g, a)
    finally:
        ref.set_num_threads(nthreads)
    b = outs()
    Oracle('f32').mcdisk_evaluate(cflux, n, csum, hoi, 123, packed, g, b)
    per_cloud = cflux / (g['spat_step'][0] * g['spat_step'][1])
    st = compare_clouds(a, b, n, per_cloud, sigma_min=w.params['dpt_a'],
                        spec_step=g['spec_step'])
    # most clouds land in the cube (the spatial z range cuts the sech2 tails)
    assert min(st['inside']) > 0.95 * n


@pytest.mark.parametrize('mistake', [dict(incl=71.0), dict(vpt_vt=220.0 * 1.03)])
def test_shot_noise_comparison_detects_a_planted_mistake(oracle_built, mistake):
    """The comparison has power: the oracle's disk with its inclination off
    by 1 degree, or its rotation 3 % too fast (mistakes planted on the CPU),
    fails it.  (The density profile is carried by the per-ring cloud budget,
    not by the kernel's density trait, so it is not a mistake to plant.)"""
    from oracle.oracle import Oracle
    w = _small_disk()
    cflux = 1e-3
    csum = w.disk.ncloudscsum(w.params, cflux)
    hoi = w.disk.hasordint()
    n = int(csum[-1])
    g = w.geometry_args(spat_z=40)
    nx, ny, sz = g['spat_size']
    nz = g['spec_size']

    def run(params, seed):
        o = dict(scube=np.zeros((nz, ny, nx), np.float32),
                 rdata=np.zeros((sz, ny, nx), np.float32))
        Oracle('f32').mcdisk_evaluate(cflux, n, csum, hoi, seed, w.disk.pack(params), g, o)
        return o

    per_cloud = cflux / (g['spat_step'][0] * g['spat_step'][1])
    a = run(w.params, 1)
    compare_clouds(a, run(w.params, 2), n, per_cloud, w.params['dpt_a'], g['spec_step'])
    wrong = dict(w.params, **mistake)
    with pytest.raises(AssertionError):
        compare_clouds(a, run(wrong, 2), n, per_cloud, w.params['dpt_a'], g['spec_step'])
