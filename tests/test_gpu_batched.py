"""Batched evaluator (gbkb200_batch_*) against the oracle's DModelSCube +
Objective chain and against the drop-in per-call GPU path."""

import numpy as np
import pytest

from tests.helpers import rel_err

pytestmark = pytest.mark.gpu


def _small_batch_workload(nsets):
    from gbkfit_b200 import workloads
    return workloads.smdisk_batch128(nsets=nsets, size=(64, 60, 48), nnodes=16)


@pytest.mark.parametrize('conv', ['fft', 'direct'])
def test_batched_chi2_vs_oracle(gpu, oracle_built, conv):
    import torch
    from oracle.oracle import chi2, scube_pipeline
    from gbkfit_b200 import workloads
    from gbkfit_b200.batched import BatchedSMDisk, synthetic_data
    w = _small_batch_workload(6)
    data, err, truth_model = synthetic_data(w)
    ev = BatchedSMDisk(w.disk, w.geom, data, err, max_sets=6, chunk=4, conv=conv)
    assert ev.conv_mode == conv
    bufs = ev.alloc_inputs(6)
    ev.upload(ev.pack(w.params, 6), bufs, 6)
    model = torch.zeros((6,) + tuple(w.geom.size[::-1]), device='cuda')
    got = ev.evaluate_device(bufs, 6, model=model).cpu().numpy()
    model = model.cpu().numpy()
    for i in range(6):
        p = w.disk.pack(workloads.set_params(w, i))
        ref64 = scube_pipeline(p, w.geom, precision='f64')
        ref32 = scube_pipeline(p, w.geom, precision='f32')
        cpu = rel_err(ref32, ref64)
        e = rel_err(model[i], ref64)
        assert e <= max(1e-5, 1.5 * cpu), (i, e, cpu)
        c_ref = chi2(ref64, data, err)
        assert abs(got[i] - c_ref) / c_ref < 1e-4, (i, got[i], c_ref)
    # the truth parameters give chi^2 ~ number of voxels (noise only)
    truth = {k: np.asarray(v)[None] for k, v in w.extra['truth'].items()}
    ev.upload(ev.pack(truth, 1), bufs, 1)
    c = ev.evaluate_device(bufs, 1).cpu().numpy()[0]
    n = np.prod(w.geom.size)
    assert 0.9 * n < c < 1.1 * n


@pytest.mark.parametrize('conv', ['fft', 'direct'])
def test_batched_matches_dropin_path(gpu, conv):
    """Batched chi^2 == the per-call drop-in path (DModelSCube + Objective)."""
    from gbkfit_b200 import workloads
    from gbkfit_b200.batched import BatchedSMDisk, synthetic_data
    from gbkfit_b200.driver import DriverB200
    from gbkfit_b200 import model as M
    w = _small_batch_workload(3)
    data, err, _ = synthetic_data(w)
    ev = BatchedSMDisk(w.disk, w.geom, data, err, max_sets=3, conv=conv)
    got = ev.evaluate(w.params, 3)
    drv = DriverB200(0)
    comp = M.SpectralSMDisk2D(False, False, w.disk.traits['rpt'], w.disk.traits['vpt'],
                              w.disk.traits['dpt'], rnodes=w.disk.rnodes)
    gm = M.GModelKinematics2D([comp])
    g = w.geom
    dm = M.DModelSCube(g.size, g.step, rpix=(0, 0, (g.size[2] - 1) / 2), rval=(0, 0, 0),
                       psf=g.psf, lsf=g.lsf)
    obj = M.Objective(M.Model(drv, dm, gm), data, err)
    for i in range(3):
        ref = -2 * obj.log_likelihood(workloads.set_params(w, i))
        assert abs(got[i] - ref) / ref < 1e-4, (i, got[i], ref)


@pytest.mark.parametrize('conv', ['fft', 'direct'])
def test_batched_chunks_and_graph(gpu, conv):
    """Results do not depend on the chunk size; a captured graph replays them."""
    import torch
    from gbkfit_b200.batched import BatchedSMDisk, synthetic_data
    w = _small_batch_workload(10)
    data, err, _ = synthetic_data(w)
    outs = []
    for chunk in (1, 3, 10):
        ev = BatchedSMDisk(w.disk, w.geom, data, err, max_sets=10, chunk=chunk, conv=conv)
        bufs = ev.alloc_inputs(10)
        ev.upload(ev.pack(w.params, 10), bufs, 10)
        outs.append(ev.evaluate_device(bufs, 10).cpu().numpy().copy())
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2])
    ev.capture(bufs, 10)
    ev.chi2.zero_()
    ev.replay()
    torch.cuda.synchronize()
    assert np.array_equal(ev.chi2[:10].cpu().numpy(), outs[0])


def test_batched_direct_mode_selection(gpu):
    """Automatic mode: direct for a (rank-1) circular Gaussian PSF, FFT for a
    high-rank Moffat PSF; both agree with the oracle."""
    from oracle.oracle import scube_pipeline
    from gbkfit_b200 import psflsf, workloads
    from gbkfit_b200.batched import BatchedSMDisk, synthetic_data
    import torch
    w = _small_batch_workload(2)
    data, err, _ = synthetic_data(w)
    ev = BatchedSMDisk(w.disk, w.geom, data, err, max_sets=2)
    assert ev.conv_mode == 'direct' and ev.psf_rank == 1
    w.geom = workloads.Geometry(w.geom.size, w.geom.step, (0, 0, (w.geom.size[2] - 1) / 2),
                                (0, 0, 0), psflsf.PSFMoffat(1.2, 2.5), w.geom.lsf)
    ev = BatchedSMDisk(w.disk, w.geom, data, err, max_sets=2)
    assert ev.conv_mode == 'fft'
    bufs = ev.alloc_inputs(2)
    ev.upload(ev.pack(w.params, 2), bufs, 2)
    model = torch.zeros((2,) + tuple(w.geom.size[::-1]), device='cuda')
    ev.evaluate_device(bufs, 2, model=model)
    ref = scube_pipeline(w.disk.pack(workloads.set_params(w, 1)), w.geom)
    assert rel_err(model[1].cpu().numpy(), ref) < 2e-5


def test_batched_direct_bands_wide_psf(gpu, oracle_built):
    """Direct mode on a wide cube whose planes are split into bands of rows
    (shared memory) with a large PSF box (FWHM 4 px): cube, chi^2 and the
    zero model outside each plane's nonzero box agree with the oracle."""
    import torch
    from oracle.oracle import chi2, scube_pipeline
    from gbkfit_b200 import psflsf, workloads
    from gbkfit_b200.batched import BatchedSMDisk, synthetic_data
    w = workloads.smdisk_batch128(nsets=3, size=(200, 180, 24), nnodes=12)
    w.geom = workloads.Geometry(w.geom.size, w.geom.step, (0, 0, (w.geom.size[2] - 1) / 2),
                                (0, 0, 0), psflsf.PSFGauss(psflsf.gauss_fwhm_to_sigma(4.0)),
                                w.geom.lsf)
    w.params['xpos'] = np.array([100.0, 60.0, 150.0])
    w.params['ypos'] = np.array([90.0, 40.0, 120.0])
    w.extra['truth']['xpos'], w.extra['truth']['ypos'] = 100.0, 90.0
    assert w.geom.kernel_size[0] > 25
    data, err, _ = synthetic_data(w)
    ev = BatchedSMDisk(w.disk, w.geom, data, err, max_sets=3, chunk=2, conv='direct')
    bufs = ev.alloc_inputs(3)
    ev.upload(ev.pack(w.params, 3), bufs, 3)
    model = torch.full((3,) + tuple(w.geom.size[::-1]), 7.0, device='cuda')
    got = ev.evaluate_device(bufs, 3, model=model).cpu().numpy()
    model = model.cpu().numpy()
    for i in range(3):
        ref = scube_pipeline(w.disk.pack(workloads.set_params(w, i)), w.geom)
        ref32 = scube_pipeline(w.disk.pack(workloads.set_params(w, i)), w.geom, precision='f32')
        assert rel_err(model[i], ref) <= max(1e-5, 1.5 * rel_err(ref32, ref)), i
        assert not np.any(model[i] == 7.0), i     # every voxel written
        c_ref = chi2(ref, data, err)
        assert abs(got[i] - c_ref) / c_ref < 1e-4, (i, got[i], c_ref)


def test_batched_direct_empty_planes(gpu, oracle_built):
    """A disk whose lines fall outside most channels (large vsys): the empty
    planes' chi^2 comes from the data table alone and matches the oracle."""
    from oracle.oracle import chi2, scube_pipeline
    from gbkfit_b200 import workloads
    from gbkfit_b200.batched import BatchedSMDisk, synthetic_data
    w = _small_batch_workload(2)
    data, err, _ = synthetic_data(w)
    w.params['vsys'] = np.array([-300.0, 2000.0])
    ev = BatchedSMDisk(w.disk, w.geom, data, err, max_sets=2, conv='direct')
    got = ev.evaluate(w.params, 2)
    for i in range(2):
        ref = scube_pipeline(w.disk.pack(workloads.set_params(w, i)), w.geom)
        c_ref = chi2(ref, data, err)
        assert abs(got[i] - c_ref) / c_ref < 1e-4, (i, got[i], c_ref)
    assert abs(got[1] - chi2(0 * data, data, err)) / got[1] < 1e-6


def test_batched_nodewise_fast_path_matches_generic(gpu):
    """The node-wise spaxel fast path (rpt/vpt/dpt uid 101 only) gives the
    same bits as the generic trait dispatch: a weight trait (which does not
    touch the cube) forces the generic path on an otherwise identical disk."""
    import torch
    from gbkfit_b200 import traits
    from gbkfit_b200.batched import BatchedSMDisk, synthetic_data
    from gbkfit_b200.disk import Disk
    w = _small_batch_workload(4)
    data, err, _ = synthetic_data(w)
    d2 = Disk(False, False, w.disk.rnodes, traits=dict(
        rpt=w.disk.traits['rpt'], vpt=w.disk.traits['vpt'], dpt=w.disk.traits['dpt'],
        wpt=[traits.wpt_axis_range(0, 30.0, 0.5)]))
    out = []
    for disk in (w.disk, d2):
        ev = BatchedSMDisk(disk, w.geom, data, err, max_sets=4, conv='direct')
        bufs = ev.alloc_inputs(4)
        ev.upload(ev.pack(w.params, 4), bufs, 4)
        model = torch.zeros((4,) + tuple(w.geom.size[::-1]), device='cuda')
        c = ev.evaluate_device(bufs, 4, model=model).cpu().numpy().copy()
        out.append((c, model.cpu().numpy(), ev.evaluate(w.params, 4)))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2], out[1][2]) and np.array_equal(out[0][0], out[0][2])


@pytest.mark.parametrize('size,psf_fwhm,lsf_fwhm', [
    ((37, 33, 20), 2.0, 1.0),       # odd width: the scalar residual path, short FIRs
    ((90, 70, 40), 5.0, 3.0),       # long FIRs, boxes wider than 32 strips' worth of lanes
    ((61, 128, 28), 3.0, 2.0),      # tall planes, many row groups per y-FIR round
])
def test_batched_direct_box_shapes(gpu, oracle_built, size, psf_fwhm, lsf_fwhm):
    """Direct mode over box shapes that exercise the kernels' lane mappings
    (x FIR (row, strip) pairs, y FIR (row group, column) rounds, odd widths):
    model cube and chi^2 against the fp64 oracle."""
    import torch
    from oracle.oracle import chi2, scube_pipeline
    from gbkfit_b200 import psflsf, workloads
    from gbkfit_b200.batched import BatchedSMDisk, synthetic_data
    nx, ny, nz = size
    w = workloads.smdisk_batch128(nsets=3, size=size, nnodes=10)
    w.geom = workloads.Geometry(size, w.geom.step, (0, 0, (nz - 1) / 2), (0, 0, 0),
                                psflsf.PSFGauss(psflsf.gauss_fwhm_to_sigma(psf_fwhm)),
                                psflsf.LSFGauss(psflsf.gauss_fwhm_to_sigma(lsf_fwhm * 10.0)))
    w.params['xpos'] = np.array([nx / 2, nx / 3, 2 * nx / 3])
    w.params['ypos'] = np.array([ny / 2, 2 * ny / 3, ny / 3])
    w.extra['truth']['xpos'], w.extra['truth']['ypos'] = nx / 2, ny / 2
    data, err, _ = synthetic_data(w)
    ev = BatchedSMDisk(w.disk, w.geom, data, err, max_sets=3, conv='direct')
    assert ev.conv_mode == 'direct'
    bufs = ev.alloc_inputs(3)
    ev.upload(ev.pack(w.params, 3), bufs, 3)
    model = torch.full((3,) + tuple(size[::-1]), 7.0, device='cuda')
    got = ev.evaluate_device(bufs, 3, model=model).cpu().numpy()
    model = model.cpu().numpy()
    for i in range(3):
        p = w.disk.pack(workloads.set_params(w, i))
        ref = scube_pipeline(p, w.geom)
        ref32 = scube_pipeline(p, w.geom, precision='f32')
        assert rel_err(model[i], ref) <= max(1e-5, 1.5 * rel_err(ref32, ref)), i
        assert not np.any(model[i] == 7.0), i
        c_ref = chi2(ref, data, err)
        assert abs(got[i] - c_ref) / c_ref < 1e-4, (i, got[i], c_ref)


def test_batched_cubes_match_disk_path(gpu):
    """gbkb200_batch_evaluate_cubes: model cubes sampled on the evaluator's
    window (here the drop-in smdisk on that window) give the chi^2 and cropped
    models of the evaluator's own disk path within fp32 rounding (the two
    evaluate the line profile with different exponentials)."""
    import torch
    from gbkfit_b200 import workloads
    from gbkfit_b200.batched import BatchedSMDisk, synthetic_data
    from gbkfit_b200.driver import DriverB200
    from tests.helpers import gpu_smdisk, upload
    n = 5
    w = _small_batch_workload(n)
    data, err, _ = synthetic_data(w)
    ev = BatchedSMDisk(w.disk, w.geom, data, err, max_sets=n, chunk=4, conv='direct')
    (ox, oy, oz), (wx, wy, wz) = ev.window()
    g = w.geom
    assert wx > g.size[0] and wy > g.size[1] and wz > g.size[2]
    assert min(ox, oy, oz) >= 0 and all(g.size_hi[i] >= (ox, oy, oz)[i] + (wx, wy, wz)[i]
                                        for i in range(3))
    geo = dict(loose=False, tilted=False, spat_size=(wx, wy, 1),
               spat_step=(g.step[0], g.step[1], 0.0),
               spat_zero=(g.zero_hi[0] + ox * g.step[0], g.zero_hi[1] + oy * g.step[1], 0.0),
               spec_size=wz, spec_step=g.step[2], spec_zero=g.zero_hi[2] + oz * g.step[2])
    gm = DriverB200(0).backends().gmodel(np.float32)
    cubes = torch.zeros((n, wz, wy, wx), device='cuda')
    for i in range(n):
        gpu_smdisk(gm, upload(w.disk.pack(workloads.set_params(w, i)), 'cuda'), geo,
                   dict(scube=cubes[i]))
    torch.cuda.synchronize()
    nx, ny, nz = g.size
    m_cube = torch.zeros((n, nz, ny, nx), device='cuda')
    m_disk = torch.zeros((n, nz, ny, nx), device='cuda')
    got = ev.evaluate_cubes_device(cubes, n, model=m_cube).cpu().numpy().copy()
    bufs = ev.alloc_inputs(n)
    ev.upload(ev.pack(w.params, n), bufs, n)
    ref = ev.evaluate_device(bufs, n, model=m_disk).cpu().numpy().copy()
    assert np.all(ref > 0)
    assert np.max(np.abs(got - ref) / ref) <= 1e-5, (got, ref)
    for i in range(n):
        assert rel_err(m_cube[i].cpu().numpy(), m_disk[i].cpu().numpy()) <= 1e-5, i
    # an all-zero cube: the model is zero and chi^2 is the data's own sum
    cubes.zero_()
    z = ev.evaluate_cubes_device(cubes, 1, model=m_cube).cpu().numpy()[0]
    d = np.asarray(data, np.float64) / np.asarray(err, np.float64)
    assert abs(z - np.sum(d * d)) <= 1e-5 * np.sum(d * d)
    assert float(m_cube[0].abs().max()) == 0.0
    ev.close()


@pytest.mark.parametrize('nodewise,ny', [(True, 60), (False, 60), (True, 62)])
def test_batched_model_variant_identical(gpu, nodewise, ny):
    """The model kernel on two 32-column chunks per warp (packed FP32 pairs,
    each lane rounded as fmaf) and on 4 x 8 spaxel tiles (range-table masks
    from per-plane ballots or from bit transposes) give bit-identical
    chi^2 and models, with an odd number of chunks (the last warp's second
    chunk is absent), on the node-wise fast path and the generic trait path,
    and with a window height that is not a multiple of 4 (the last row
    group of the tiles is partial: 62 + 16 rows)."""
    import torch
    from gbkfit_b200 import traits as T
    from gbkfit_b200 import workloads
    from gbkfit_b200.batched import BatchedSMDisk, synthetic_data
    from gbkfit_b200.disk import Disk
    n = 6
    w = workloads.smdisk_batch128(nsets=n, size=(64, ny, 48), nnodes=16)
    if not nodewise:
        w.disk = Disk(False, False, w.disk.rnodes, traits=dict(
            rpt=[T.bpt('nw_uniform')], vpt=[T.vpt('nw_tan_uniform')], dpt=[T.dpt('nw_uniform')],
            spt=[T.spt('azrange')]))
        w.params = dict(w.params, spt_p=np.full(n, 30.0), spt_s=np.full(n, 300.0))
        w.extra = dict(w.extra, truth=dict(w.extra['truth'], spt_p=30.0, spt_s=300.0))
    data, err, _ = synthetic_data(w)
    out = []
    for variant in (0, 1, 2, 3):
        ev = BatchedSMDisk(w.disk, w.geom, data, err, max_sets=n, chunk=4, conv='direct',
                           model_variant=variant)
        bufs = ev.alloc_inputs(n)
        ev.upload(ev.pack(w.params, n), bufs, n)
        model = torch.zeros((n,) + tuple(w.geom.size[::-1]), device='cuda')
        chi2 = ev.evaluate_device(bufs, n, model=model).cpu().numpy().copy()
        out.append((chi2, model.cpu().numpy()))
        ev.close()
    nch = -(-(w.geom.size[0] + 16) // 32)
    assert nch % 2 == 1
    for o in out[1:]:
        assert np.array_equal(out[0][0], o[0]) and np.array_equal(out[0][1], o[1])
    assert np.all(out[0][0] > 0)


def test_batched_evaluate_pieces_identical(gpu):
    """End-to-end evaluate() in one, two (the default from 256 sets) or three
    equal pieces or pieces of given sizes, smaller than a chunk or not: the
    same chi^2, bit for bit, as the device-resident evaluation."""
    from gbkfit_b200.batched import BatchedSMDisk, synthetic_data
    n = 300
    w = _small_batch_workload(n)
    data, err, _ = synthetic_data(w)
    ev = BatchedSMDisk(w.disk, w.geom, data, err, max_sets=n, chunk=128, conv='direct')
    bufs = ev.alloc_inputs(n)
    ev.upload(ev.pack(w.params, n), bufs, n)
    ref = ev.evaluate_device(bufs, n).cpu().numpy().copy()
    for pieces in (None, 1, 3, (100, 200), (64, 236)):
        got = ev.evaluate(w.params, n, pieces=pieces)
        assert np.array_equal(got, ref), pieces
    ev.close()


def test_timing_modes_and_counters(gpu):
    """Timing without counters leaves the counters at zero and the chi^2
    unchanged; timing with counters counts the direct-mode kernels' work."""
    import torch
    from gbkfit_b200.batched import BatchedSMDisk, synthetic_data
    w = _small_batch_workload(4)
    data, err, _ = synthetic_data(w)
    ev = BatchedSMDisk(w.disk, w.geom, data, err, max_sets=4, conv='direct')
    bufs = ev.alloc_inputs(4)
    ev.upload(ev.pack(w.params, 4), bufs, 4)
    plain = ev.evaluate_device(bufs, 4).clone()
    ev.set_timing(True, counters=False)
    timed = ev.evaluate_device(bufs, 4).clone()
    stages = ev.stage_times()
    assert stages and all(t > 0 and n == 1 for t, n in stages.values()), stages
    assert all(v == 0 for v in ev.work_counters().values())
    ev.set_timing(True, counters=True)
    counted = ev.evaluate_device(bufs, 4).clone()
    ev.stage_times()
    c = ev.work_counters()
    ev.set_timing(False)
    assert c['psf_x_fma'] > 0 and c['psf_y_fma'] > 0 and c['residual_voxels'] > 0
    assert c['lsf_fma'] > 0 and c['lines'] > 0
    torch.testing.assert_close(timed, plain, rtol=0, atol=0)
    torch.testing.assert_close(counted, plain, rtol=0, atol=0)


@pytest.mark.parametrize('nodewise', [True, False])
def test_batched_model_variant_scaled_line(gpu, oracle_built, nodewise):
    """The tile model kernel with the line's exponent as -t^2 (t one
    multiply-add per channel) matches the kernel with the exponent from the
    velocity difference within fp32 rounding, and the fp64 oracle."""
    import torch
    from oracle.oracle import scube_pipeline
    from gbkfit_b200 import traits as T
    from gbkfit_b200 import workloads
    from gbkfit_b200.batched import BatchedSMDisk, synthetic_data
    from gbkfit_b200.disk import Disk
    n = 5
    w = workloads.smdisk_batch128(nsets=n, size=(64, 62, 48), nnodes=16)
    if not nodewise:
        w.disk = Disk(False, False, w.disk.rnodes, traits=dict(
            rpt=[T.bpt('nw_uniform')], vpt=[T.vpt('nw_tan_uniform')], dpt=[T.dpt('nw_uniform')],
            spt=[T.spt('azrange')]))
        w.params = dict(w.params, spt_p=np.full(n, 30.0), spt_s=np.full(n, 300.0))
        w.extra = dict(w.extra, truth=dict(w.extra['truth'], spt_p=30.0, spt_s=300.0))
    data, err, _ = synthetic_data(w)
    out = []
    for variant in (3, 4):
        ev = BatchedSMDisk(w.disk, w.geom, data, err, max_sets=n, chunk=4, conv='direct',
                           model_variant=variant)
        bufs = ev.alloc_inputs(n)
        ev.upload(ev.pack(w.params, n), bufs, n)
        model = torch.zeros((n,) + tuple(w.geom.size[::-1]), device='cuda')
        chi2 = ev.evaluate_device(bufs, n, model=model).cpu().numpy().copy()
        out.append((chi2, model.cpu().numpy()))
        ev.close()
    (c3, m3), (c4, m4) = out
    assert np.all(np.abs(c4 - c3) <= 1e-5 * np.abs(c3)), (c3, c4)
    for i in range(n):
        assert np.abs(m4[i] - m3[i]).max() <= 1e-5 * np.abs(m3[i]).max(), i
        p = w.disk.pack(workloads.set_params(w, i))
        ref64 = scube_pipeline(p, w.geom, precision='f64')
        ref32 = scube_pipeline(p, w.geom, precision='f32')
        assert rel_err(m4[i], ref64) <= max(1e-5, 1.5 * rel_err(ref32, ref64)), i


def test_evaluate_rows_from_nodes_matches_host_packing(gpu):
    """evaluate() with the input rows built on the device from the raw node
    values (linear interpolation) gives the chi^2 of the host-packed path,
    on repeated calls and on a batch smaller than the evaluator's capacity."""
    from gbkfit_b200.batched import BatchedSMDisk, synthetic_data
    n = 40
    w = _small_batch_workload(n)
    data, err, _ = synthetic_data(w)
    ev = BatchedSMDisk(w.disk, w.geom, data, err, max_sets=48, chunk=32, conv='direct')
    got = ev.evaluate(w.params, n)
    assert ev._node_rows() is not None
    assert ev.last_h2d_bytes == n * ev._node_rows()['nraw'] * 8
    ref = ev.evaluate(w.params, n, pieces=1)
    np.testing.assert_allclose(got, ref, rtol=1e-6, atol=0)
    assert np.array_equal(ev.evaluate(w.params, n), got)
    sub = {k: (np.asarray(v)[:9] if np.ndim(v) and np.shape(v)[0] == n else v)
           for k, v in w.params.items()}
    np.testing.assert_allclose(ev.evaluate(sub, 9), got[:9], rtol=1e-6, atol=0)
