"""CUDA path vs oracle, through the C ABI (libgbkb200.so via the driver
backends).

Tolerances (normwise relative, max|a - b| / max|b|):
* model cubes: <= 1e-5 against the fp32 restatement of the reference (which
  itself matches the compiled reference to ~2 ulp), and against the fp64
  oracle no worse than 3x the fp32 CPU path's own fp64 error (and <= 1e-4);
* FFT convolution: <= 1e-5 against numpy float64;
* mcdisk: per-cloud agreement with the oracle's identical Philox stream.
"""

import numpy as np
import pytest

from tests.helpers import gpu_mcdisk, gpu_smdisk, rel_err, upload

pytestmark = pytest.mark.gpu

TOL = 1e-5


@pytest.fixture(scope='module')
def be(gpu):
    from gbkfit_b200.driver import DriverB200
    drv = DriverB200(0)
    b = drv.backends()
    return dict(drv=drv, fft=b.fft(np.float32), dmodel=b.dmodel(np.float32),
                gmodel=b.gmodel(np.float32), objective=b.objective(np.float32))


def _smdisk_both(be, oracle_built, w, thick=False, spat_z=None, extra_outs=()):
    import torch
    from oracle.oracle import Oracle
    g = w.geometry_args(spat_z)
    nx, ny, nz = g['spat_size'][0], g['spat_size'][1], g['spec_size']
    sz = g['spat_size'][2]
    packed = w.disk.pack(w.params)
    pd = upload(packed, 'cuda')
    outs_d = dict(scube=torch.zeros((nz, ny, nx), device='cuda'))
    outs_h = dict(scube=np.zeros((nz, ny, nx)))
    for n in extra_outs:
        fill = np.nan if n in ('vdata_cmp', 'ddata_cmp') else 0.0
        outs_d[n] = torch.full((sz, ny, nx), fill, device='cuda')
        outs_h[n] = np.full((sz, ny, nx), fill)
    gpu_smdisk(be['gmodel'], pd, g, outs_d)
    outs_32 = {k: v.astype(np.float32) for k, v in outs_h.items()}
    Oracle('f64').smdisk_evaluate(packed, g, outs_h)
    Oracle('f32').smdisk_evaluate(packed, g, outs_32)
    gd = {k: v.cpu().numpy() for k, v in outs_d.items()}
    return gd, outs_h, outs_32


def _check_cube(gpu_cube, o64, o32):
    """GPU error vs fp64 <= max(1e-5, 1.5 x the fp32 CPU path's own error),
    and GPU vs the fp32 CPU path within the sum of both fp32 errors."""
    e32 = rel_err(gpu_cube, o32)
    e64 = rel_err(gpu_cube, o64)
    cpu64 = rel_err(o32, o64)
    assert e64 <= max(TOL, 1.5 * cpu64), (e32, e64, cpu64)
    assert e32 <= max(TOL, e64 + cpu64 + 1e-6), (e32, e64, cpu64)


def test_smdisk_thin_cube64(be, oracle_built):
    from gbkfit_b200 import workloads
    gd, gh, g32 = _smdisk_both(be, oracle_built, workloads.smdisk_cube64(),
                               extra_outs=('rdata', 'vdata_cmp', 'ddata_cmp'))
    assert gh['scube'].max() > 0
    _check_cube(gd['scube'], gh['scube'], g32['scube'])
    _check_cube(gd['rdata'], gh['rdata'], g32['rdata'])
    m = np.isfinite(gh['vdata_cmp'])
    assert np.array_equal(m, np.isfinite(gd['vdata_cmp']))
    assert rel_err(gd['vdata_cmp'][m], gh['vdata_cmp'][m]) < TOL


def test_smdisk_thin_nodewise_batchset(be, oracle_built):
    from gbkfit_b200 import workloads
    w = workloads.smdisk_batch128(nsets=4)
    for i in range(4):
        wi = workloads.Workload(w.name, w.disk, workloads.set_params(w, i), w.geom)
        gd, gh, g32 = _smdisk_both(be, oracle_built, wi)
        _check_cube(gd['scube'], gh['scube'], g32['scube'])


def test_smdisk_thick(be, oracle_built):
    from gbkfit_b200 import workloads
    w = workloads.mcdisk_cube256()
    w.geom = workloads.Geometry((64, 64, 48), (1, 1, 10), (0, 0, 23.5), (0, 0, 0),
                                w.geom.psf, w.geom.lsf)
    w.params = dict(w.params, xpos=32.0, ypos=32.0, bpt_s=8.0)
    gd, gh, g32 = _smdisk_both(be, oracle_built, w, thick=True, spat_z=40,
                               extra_outs=('rdata',))
    assert gh['scube'].max() > 0
    _check_cube(gd['scube'], gh['scube'], g32['scube'])
    _check_cube(gd['rdata'], gh['rdata'], g32['rdata'])


@pytest.mark.parametrize('shape', [(96, 96, 96), (35, 48, 21), (160, 160, 128), (8, 1, 16),
                                   (1, 12, 10), (22, 26, 33)])
def test_fft_convolve_cached(be, shape):
    import torch
    from oracle.oracle import fft_convolve_cached
    rng = np.random.default_rng(7)
    a = rng.standard_normal(shape).astype(np.float32)
    k = rng.random(shape).astype(np.float32)
    k /= k.sum()
    ref = fft_convolve_cached(a, k)
    ad = torch.from_numpy(a).cuda()
    kd = torch.from_numpy(k).cuda()
    be['fft'].fft_convolve_cached(ad, kd)
    assert rel_err(ad.cpu().numpy(), ref) < TOL
    # second call hits the cached kernel spectrum
    ad2 = torch.from_numpy(a).cuda()
    be['fft'].fft_convolve_cached(ad2, kd)
    assert np.array_equal(ad.cpu().numpy(), ad2.cpu().numpy())


@pytest.mark.parametrize('shape', [(64, 40, 48), (15, 9, 7)])
def test_fft_r2c_c2r(be, shape):
    import torch
    rng = np.random.default_rng(3)
    a = rng.standard_normal(shape).astype(np.float32)
    ad = torch.from_numpy(a).cuda()
    nz, ny, nx = shape
    c = torch.zeros((nz, ny, nx // 2 + 1), dtype=torch.complex64, device='cuda')
    be['fft'].fft_r2c(ad, c)
    ref = np.fft.rfftn(a.astype(np.float64))
    assert rel_err(c.cpu().numpy(), ref) < TOL
    back = torch.zeros_like(ad)
    be['fft'].fft_c2r(c, back)
    assert rel_err(back.cpu().numpy() / a.size, a) < TOL
    # the input spectrum is preserved by c2r
    assert rel_err(c.cpu().numpy(), ref) < TOL


def test_fft_convolve_uncached(be):
    import torch
    from oracle.oracle import fft_convolve_cached
    rng = np.random.default_rng(5)
    shape = (32, 20, 24)
    a = rng.standard_normal(shape).astype(np.float32)
    k = rng.random(shape).astype(np.float32)
    ref = fft_convolve_cached(a, k)
    kd = torch.from_numpy(k).cuda()
    kc = torch.zeros((32, 20, 13), dtype=torch.complex64, device='cuda')
    be['fft'].fft_r2c(kd, kc)
    ad = torch.from_numpy(a).cuda()
    ac = torch.zeros_like(kc)
    be['fft'].fft_convolve(ad, ac, kc)
    assert rel_err(ad.cpu().numpy(), ref) < TOL


def test_moments(be, oracle_built):
    import torch
    from oracle.oracle import Oracle, Reference
    from gbkfit_b200 import workloads
    w = workloads.smdisk_cube64()
    g = w.geometry_args()
    nx, ny, nz = g['spat_size'][0], g['spat_size'][1], g['spec_size']
    cube = np.zeros((nz, ny, nx))
    Oracle('f64').smdisk_evaluate(w.disk.pack(w.params), g, dict(scube=cube))
    cube = cube.astype(np.float32)
    rng = np.random.default_rng(1)
    wcube = rng.random(cube.shape).astype(np.float32)
    orders = np.array([0, 1, 2, 3, 4], np.int32)
    size = (nx, ny, nz)
    step = (1.0, 1.0, 10.0)
    zero = (0.0, 0.0, -385.0)
    md = torch.zeros((5, ny, nx), device='cuda')
    mm = torch.zeros((ny, nx), device='cuda')
    mw = torch.zeros((ny, nx), device='cuda')
    be['dmodel'].mmaps_moments(size, step, zero, torch.from_numpy(cube).cuda(),
                               torch.from_numpy(wcube).cuda(), 1e-6,
                               torch.from_numpy(orders).cuda(), md, mw, mm)
    od, om, ow = Oracle('f64').mmaps_moments(size, step, zero, cube, wcube, 1e-6, orders)
    o32, _, w32 = Oracle('f32').mmaps_moments(size, step, zero, cube, wcube, 1e-6, orders)
    md, mm, mw = md.cpu().numpy(), mm.cpu().numpy(), mw.cpu().numpy()
    assert np.array_equal(mm, om)
    v = om > 0
    assert v.sum() > 100
    # per order: <= max(1e-5, 2 x the fp32 CPU path's own fp64 error); the
    # third moment sums flux * (v - m1)^3 with heavy cancellation and is
    # ill-conditioned in fp32 (the reference's own fp32 result is ~30% off)
    for i in range(5):
        cpu = rel_err(o32[i][v], od[i][v])
        assert rel_err(md[i][v], od[i][v]) <= max(TOL, 2 * cpu), i
        assert np.all(np.isnan(md[i][~v]))
    assert rel_err(mw[v], ow[v]) <= max(TOL, 2 * rel_err(w32[v], ow[v]))
    if Reference.available():
        rd, rm, rw = Reference().mmaps_moments(size, step, zero, cube, wcube, 1e-6, orders)
        assert np.array_equal(mm, rm)
        for i in (0, 1, 2, 4):
            assert rel_err(md[i][v], rd[i][v]) <= TOL, i


def test_residual_and_sum(be, oracle_built):
    import torch
    from oracle.oracle import Oracle
    rng = np.random.default_rng(11)
    n = 1_000_003
    od, oe, md, mw = (rng.random(n).astype(np.float32) + 0.5 for _ in range(4))
    om = (rng.random(n) > 0.1).astype(np.float32)
    t = {k: torch.from_numpy(v).cuda() for k, v in dict(od=od, oe=oe, om=om, md=md, mw=mw).items()}
    res = torch.zeros(n, device='cuda')
    be['objective'].residual(t['od'], t['oe'], t['om'], t['md'], t['mw'], None, 0.7, res)
    ref = Oracle('f64').residual(od, oe, om, md, mw, None, 0.7)
    assert rel_err(res.cpu().numpy(), ref) < 1e-6
    s = torch.zeros(1, device='cuda')
    be['objective'].residual_sum(res, True, s)
    assert abs(s.item() - Oracle('f64').residual_sum(res.cpu().numpy())) / s.item() < 1e-6
    be['objective'].residual_sum(res, False, s)
    assert abs(s.item() - Oracle('f64').residual_sum(res.cpu().numpy(), False)) / s.item() < 1e-6


def test_downscale_mask_wcube(be, oracle_built):
    import torch
    from oracle.oracle import Oracle
    o = Oracle('f32')
    rng = np.random.default_rng(2)
    src = rng.standard_normal((30, 26, 22)).astype(np.float32)
    dst = torch.zeros((9, 8, 10), device='cuda')
    be['dmodel'].dcube_downscale((2, 3, 3), (1, 2, 3), torch.from_numpy(src).cuda(), dst)
    ref = o.dcube_downscale((2, 3, 3), (1, 2, 3), src, (9, 8, 10))
    assert rel_err(dst.cpu().numpy(), ref) < 1e-6
    d = torch.from_numpy(src).cuda()
    m = torch.zeros_like(d)
    be['dmodel'].dcube_mask(0.5, True, m, d, None)
    rd, rm = o.dcube_mask(0.5, True, src)
    assert np.array_equal(m.cpu().numpy(), rm)
    assert np.array_equal(np.isnan(d.cpu().numpy()), np.isnan(rd))
    spat = np.abs(rng.standard_normal((5, 7, 9))).astype(np.float32)
    spec = torch.zeros((11, 7, 9), device='cuda')
    be['gmodel'].wcube_evaluate((9, 7, 5), 11, torch.from_numpy(spat).cuda(), spec)
    assert rel_err(spec.cpu().numpy(), o.wcube_evaluate(spat, 11)) < 1e-6


def test_mcdisk_flux_and_clouds(be, oracle_built):
    """Same Philox clouds as the oracle: the spatial flux map agrees per
    voxel except for clouds that land on a rint boundary, and the total flux
    of the clouds that fall inside the cube is conserved."""
    import torch
    from oracle.oracle import Oracle
    from gbkfit_b200 import workloads
    w = workloads.mcdisk_cube256(nclouds=200_000)
    w.geom = workloads.Geometry((64, 64, 32), (1, 1, 10), (0, 0, 15.5), (0, 0, 0),
                                w.geom.psf, w.geom.lsf)
    w.params = dict(w.params, xpos=32.0, ypos=32.0, bpt_s=8.0)
    w.disk = workloads.Disk(False, False, np.linspace(0, 40, 21), traits=w.disk.traits)
    csum = w.disk.ncloudscsum(w.params, 1e-3)
    hoi = w.disk.hasordint()
    nclouds = int(csum[-1])
    g = w.geometry_args(spat_z=32)
    nx, ny, sz = g['spat_size']
    nz = g['spec_size']
    packed = w.disk.pack(w.params)
    pd = upload(packed, 'cuda')
    be['gmodel'].set_mcdisk(seed=123, mode=0)
    outs = dict(scube=torch.zeros((nz, ny, nx), device='cuda'),
                rdata=torch.zeros((sz, ny, nx), device='cuda'))
    gpu_mcdisk(be['gmodel'], 1e-3, nclouds, torch.from_numpy(csum).cuda(),
               torch.from_numpy(hoi).cuda(), pd, g, outs)
    oh = dict(scube=np.zeros((nz, ny, nx), np.float32), rdata=np.zeros((sz, ny, nx), np.float32))
    Oracle('f32').mcdisk_evaluate(1e-3, nclouds, csum, hoi, 123, packed, g, oh)
    rd = outs['rdata'].cpu().numpy()
    per_cloud = 1e-3 / (g['spat_step'][0] * g['spat_step'][1])
    n_gpu = rd.sum() / per_cloud
    n_orc = oh['rdata'].sum() / per_cloud
    assert n_gpu > 0.5 * nclouds
    assert abs(n_gpu - n_orc) <= 1e-4 * nclouds
    diff = np.abs(rd - oh['rdata'])
    moved = int(np.sum(diff > 0.5 * per_cloud))       # ~2 voxels per cloud that moved
    assert moved <= 1e-3 * nclouds
    # scube: a cloud that landed in another spaxel moves its whole line (its
    # spectral sum is at most 1.5 x per_cloud / dz for these line widths);
    # every other cloud differs by fp32 rounding of its line only
    sg = outs['scube'].cpu().numpy().astype(np.float64)
    so = oh['scube'].astype(np.float64)
    line_sum = 1.5 * per_cloud / g['spec_step']
    assert np.abs(sg - so).sum() <= moved * line_sum + 1e-5 * np.abs(so).sum()
    assert abs(sg.sum() - so.sum()) <= moved * line_sum + 1e-5 * abs(so.sum())


def test_mcdisk_deterministic_mode(be, oracle_built):
    """Mode 1 (64-bit fixed-point accumulation) gives bit-identical cubes and
    maps run to run, and agrees with the fast fp32-atomic modes (0 and 2:
    vector atomics into a channel-contiguous scratch cube; 3: one atomic per
    channel)."""
    import torch
    from gbkfit_b200 import workloads
    w = workloads.mcdisk_cube256(nclouds=300_000)
    w.geom = workloads.Geometry((64, 64, 32), (1, 1, 10), (0, 0, 15.5), (0, 0, 0),
                                w.geom.psf, w.geom.lsf)
    w.params = dict(w.params, xpos=32.0, ypos=32.0, bpt_s=8.0)
    w.disk = workloads.Disk(False, False, np.linspace(0, 40, 21), traits=w.disk.traits)
    csum = w.disk.ncloudscsum(w.params, 1e-3)
    hoi = w.disk.hasordint()
    g = w.geometry_args(spat_z=32)
    nx, ny, sz = g['spat_size']
    nz = g['spec_size']
    pd = upload(w.disk.pack(w.params), 'cuda')

    def run(mode):
        be['gmodel'].set_mcdisk(seed=7, mode=mode)
        outs = dict(scube=torch.zeros((nz, ny, nx), device='cuda'),
                    image=torch.zeros((ny, nx), device='cuda'),
                    rdata=torch.zeros((sz, ny, nx), device='cuda'))
        gpu_mcdisk(be['gmodel'], 1e-3, int(csum[-1]), torch.from_numpy(csum).cuda(),
                   torch.from_numpy(hoi).cuda(), pd, g, outs)
        return {k: v.cpu().numpy() for k, v in outs.items()}

    a, b, fast, v4, scalar = run(1), run(1), run(0), run(2), run(3)
    be['gmodel'].set_mcdisk(seed=42, mode=0)
    # mode 2 (vector atomics into a channel-contiguous scratch cube; mode 0's
    # path) and mode 3 (one atomic per channel) sum the same contributions
    for o in (v4, scalar):
        assert rel_err(o['scube'], a['scube']) <= 1e-5
        for k in ('image', 'rdata'):
            assert rel_err(o[k], a[k]) <= 1e-4, k
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    # every cloud adds cflux / (dx dy) to the maps: the fixed-point sums are
    # whole cloud counts; the fast mode's fp32 atomics lose ~n eps per element
    per_cloud = 1e-3 / (g['spat_step'][0] * g['spat_step'][1])
    for k in ('image', 'rdata'):
        n = a[k].astype(np.float64) / per_cloud
        assert np.all(np.abs(n - np.rint(n)) <= 1e-6 * np.maximum(1.0, n)), k
        assert rel_err(fast[k], a[k]) <= 1e-4, (k, rel_err(fast[k], a[k]))
    assert rel_err(fast['scube'], a['scube']) <= 1e-5
    assert abs(a['scube'].sum() - fast['scube'].sum()) <= 1e-5 * abs(a['scube'].sum())


def test_mcdisk_dense_clouds_replicated_scratch(be, oracle_built):
    """Dense clouds (over 1,000 per spaxel on the 64x64 padded grid of a
    48x48 cube): the fast mode's line scratch is replicated 8 times
    (gbkb200_mcdisk_scratch_bytes) and the copies are summed by the
    transpose-add; the cube and maps agree with the deterministic mode and
    with one atomic per channel (mode 3)."""
    import torch
    from gbkfit_b200 import _native, psflsf, workloads
    w = workloads.mcdisk_cube256(nclouds=3_000_000)
    w.geom = workloads.Geometry((48, 48, 32), (1, 1, 10), (0, 0, 15.5), (0, 0, 0),
                                psflsf.PSFGauss(1.0), w.geom.lsf)
    w.params = dict(w.params, xpos=24.0, ypos=24.0, bpt_s=6.0)
    w.disk = workloads.Disk(False, False, np.linspace(0, 30, 21), traits=w.disk.traits)
    cflux = 4.8e-5                    # about 4.5e6 clouds, 1,100 per spaxel
    csum = w.disk.ncloudscsum(w.params, cflux)
    n = int(csum[-1])
    hoi = w.disk.hasordint()
    g = w.geometry_args(spat_z=32)
    nx, ny, sz = g['spat_size']
    nz = g['spec_size']
    copies = _native.lib().gbkb200_mcdisk_scratch_bytes(n, nx, ny, nz) // (
        nx * ny * ((nz + 3) // 4 * 4) * 4)
    assert copies == 8, (n, copies)
    pd = upload(w.disk.pack(w.params), 'cuda')

    def run(mode):
        be['gmodel'].set_mcdisk(seed=11, mode=mode)
        outs = dict(scube=torch.zeros((nz, ny, nx), device='cuda'),
                    rdata=torch.zeros((sz, ny, nx), device='cuda'))
        gpu_mcdisk(be['gmodel'], cflux, n, torch.from_numpy(csum).cuda(),
                   torch.from_numpy(hoi).cuda(), pd, g, outs)
        return {k: v.cpu().numpy() for k, v in outs.items()}

    fast, det, scalar = run(0), run(1), run(3)
    be['gmodel'].set_mcdisk(seed=42, mode=0)
    assert det['scube'].sum() > 0
    for o in (fast, scalar):
        assert rel_err(o['scube'], det['scube']) <= 1e-5
        assert rel_err(o['rdata'], det['rdata']) <= 1e-4
    assert abs(fast['scube'].astype(np.float64).sum() - det['scube'].astype(np.float64).sum()) \
        <= 1e-5 * det['scube'].astype(np.float64).sum()
