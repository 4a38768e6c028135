"""Benchmark: batched smdisk + PSF/LSF + chi^2 cube evaluations per second on B200.

Workload (the batched objective configuration): 512 parameter sets of a thin
smooth disk with 30 radial nodes (node-wise surface brightness exp(N(0,0.5)),
rotation ~U(50,300) km/s, dispersion ~U(5,40) km/s; incl ~U(20,80),
PA ~U(0,360)), each evaluated on a 128x128x96 cube (10 km/s channels),
convolved with a Gaussian PSF (FWHM 3 px) x Gaussian LSF (FWHM 1.5 channels)
and scored with chi^2 against a seeded synthetic data cube with Gaussian noise
of sigma = 2% of the peak.  Synthetic data (no datasets).

A step is one evaluation of all 512 sets.  `value` is evals/s with the
parameter sets resident in HBM; `e2e` is the same through the public API
(host parameter dicts -> packing -> pinned H2D -> chi^2 D2H).  With
--gpus N (torchrun) every rank evaluates its own 512 sets (weak scaling).

--impl reference times the reference's own CPU implementation of the path
(its smdisk/residual templates compiled with OpenMP in oracle/_ref, with
scipy's FFT standing in for FFTW, which is not installed) on the host cores.
"""

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "smdisk+PSF/LSF cube evals/s (batched, 512 sets, 128x128x96)"
UNIT = "evals/s"


def staged_bytes_per_eval(geom):
    """Algorithmic bytes of one staged evaluation with the reference padding
    P: 12 V(P) + 40 C(P) + 12 V(N) + 4 (model write, r2c, spectrum multiply,
    c2r, crop + data + error reads, chi^2)."""
    px, py, pz = geom.size_hi
    vp = px * py * pz
    cp = (px // 2 + 1) * py * pz
    vn = int(np.prod(geom.size))
    return 12 * vp + 40 * cp + 12 * vn + 4


def fft_flops_per_eval(geom):
    px, py, pz = geom.size_hi
    vp = px * py * pz
    cp = (px // 2 + 1) * py * pz
    return 2 * 2.5 * vp * np.log2(vp) + 6 * cp


def direct_flops_per_eval(geom):
    """Dense FIR FLOPs of one direct-mode evaluation: LSF over the window
    columns, PSF x over the window rows, PSF y over the crop (2 per tap);
    the kernels skip the exact-zero part of this work."""
    nx, ny, nz = geom.size
    kx, ky, kz = geom.kernel_size
    wx, wy = nx + kx - 1, ny + ky - 1
    return 2 * (kz * nz * wx * wy + kx * nz * wy * nx + ky * nz * ny * nx)


# DRAM bytes (read + write) per parameter set of each direct-mode kernel, from
# one ncu capture (dram__bytes_read.sum + dram__bytes_write.sum) of a 128-set
# wave of this workload, divided by 128; a launch of n sets moves about n times
# this (the traffic grows with the sets processed).  Not measured by this run.
# The model kernel's figure is that of the 4x8-tile form (its variants 2 and
# 3 store the same bytes).
NCU_DRAM_BYTES_PER_SET = {
    'kb_psf_residual': 288.8e6 / 128,
    'ka_lines_lsf': 169.7e6 / 128,
}

# FLOPs of one residual voxel computed from the model: (m - d), x w, r^2 sum
RESIDUAL_FLOPS = 3


def fp32_peak_tflops(clocks):
    """Nominal FP32 CUDA-core peak at the sampled SM clock: 148 SMs x 128
    lanes x 2 FLOP (one fused multiply-add) per clock."""
    mhz = clocks.get('sm_mhz') or clocks.get('sm_max_mhz') or 1965.0
    return 148 * 128 * 2 * mhz * 1e6 / 1e12, mhz


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', f'--id={self.index}', f'--query-gpu={self.FIELDS}',
                 '--format=csv,noheader,nounits', '-lms', '200'],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return dict(sm_mhz=None, sm_max_mhz=None, reasons=['nvidia-smi unavailable'])
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], None, set()
        names = ('hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap')
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(',')]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == 'active':
                    reasons.add(n)
        return dict(sm_mhz=float(np.median(sm)) if sm else None, sm_max_mhz=smax,
                    reasons=sorted(reasons), samples=len(sm))


def peaks():
    p = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d['hbm_gbs'], 'measured'
    return 6650.0, 'fallback'


def setup_dist(args):
    import torch
    import torch.distributed as dist
    rank, world = int(os.environ.get('RANK', 0)), int(os.environ.get('WORLD_SIZE', 1))
    local = int(os.environ.get('LOCAL_RANK', 0))
    if world > 1:
        import datetime
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device('cuda', local))
    torch.cuda.set_device(local)
    return rank, world, local


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device='cuda')
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def roofline_direct(kernels, counters, steps, nsets, clocks, geom, ms_step):
    """Roofline of the dominant direct-mode kernel (the PSF FIR + residual
    kernel): the FLOPs it executed (PSF x and y FIR multiply-adds and residual
    voxels, counted inside the kernel over a second pass of the same launches)
    per launch, divided by its average launch time (CUDA events on its stream,
    measured in a pass without the counters), against
    the FP32 CUDA-core peak at the sampled clock.  The kernel computes in
    FP32 on CUDA cores and moves little DRAM traffic (see `hbm_view`)."""
    peak, mhz = fp32_peak_tflops(clocks)
    name = 'kb_psf_residual'
    k = kernels[name]
    launches = k['launches_per_step'] * steps
    fl_kb = (2 * (counters['psf_x_fma'] + counters['psf_y_fma'])
             + RESIDUAL_FLOPS * counters['residual_voxels']) / launches
    ach = fl_kb / (k['ms_per_launch'] / 1e3) / 1e12
    sets_per_launch = nsets / k['launches_per_step']
    traffic = NCU_DRAM_BYTES_PER_SET[name] * sets_per_launch
    ka = kernels.get('ka_lines_lsf')
    ka_view = None
    if ka:
        fl_ka = 2 * counters['lsf_fma'] / (ka['launches_per_step'] * steps)
        ka_view = dict(kernel='ka_lines_lsf', executed_flops_per_launch=int(fl_ka),
                       lines_per_launch=int(counters['lines'] / (ka['launches_per_step'] * steps)),
                       achieved=round(fl_ka / (ka['ms_per_launch'] / 1e3) / 1e12, 2),
                       frac=round(fl_ka / (ka['ms_per_launch'] / 1e3) / 1e12 / peak, 3))
    step_bytes = sum(NCU_DRAM_BYTES_PER_SET[n] * nsets for n in NCU_DRAM_BYTES_PER_SET
                     if n in kernels)
    hbm, hbm_kind = peaks()
    return dict(
        bound='fp32-issue', kernel=name, achieved=round(ach, 2), peak=round(peak, 1),
        unit='TFLOP/s', frac=round(ach / peak, 3),
        peak_kind=f'nominal FP32 CUDA-core peak at the sampled SM clock ({mhz:.0f} MHz): '
                  '148 SMs x 128 lanes x 2 FLOP',
        executed_flops_per_launch=int(fl_kb), ms_per_launch=k['ms_per_launch'],
        sets_per_launch=sets_per_launch,
        basis='PSF x and y FIR multiply-adds (2 FLOP each) and residual voxels (3 FLOP each) '
              'executed by the kernel, counted in-kernel over a second pass of the same '
              'launches (the timed pass runs without the counters)',
        traffic=round(traffic), traffic_unit='DRAM bytes per launch',
        traffic_source='ncu capture of a 128-set wave of this workload, scaled to the '
                       'sets of one launch (not measured by this run)',
        model_kernel=ka_view, kernels=kernels, dominant=name,
        hbm_view=dict(dram_bytes_per_step=round(step_bytes),
                      achieved=round(step_bytes / (ms_step / 1e3) / 1e9, 1), peak=hbm,
                      unit='GB/s', frac=round(step_bytes / (ms_step / 1e3) / 1e9 / hbm, 3),
                      peak_kind=hbm_kind),
        staged_equivalent=dict(
            bytes_per_eval=staged_bytes_per_eval(geom),
            basis='staged FFT pipeline with the reference padding '
                  f'{list(geom.size_hi)}; the direct path does not move these bytes',
            equivalent_gbs=round(staged_bytes_per_eval(geom) * nsets / (ms_step / 1e3) / 1e9, 1)),
        dense_fir_equivalent_tflops=round(direct_flops_per_eval(geom) * nsets
                                          / (ms_step / 1e3) / 1e12, 2))


def roofline_fft(kernels, nsets, geom, ms_step):
    """FFT mode: staged algorithmic bytes with the reference padding over
    the step time, against the measured HBM bandwidth."""
    hbm, peak_kind = peaks()
    b_eval = staged_bytes_per_eval(geom)
    achieved = b_eval * nsets / (ms_step / 1e3) / 1e9
    return dict(bound='hbm', achieved=round(achieved, 1), peak=hbm, unit='GB/s',
                frac=round(achieved / hbm, 3), traffic=None, peak_kind=peak_kind,
                basis=f'staged algorithmic bytes per evaluation ({b_eval} B, reference '
                      f'padding {list(geom.size_hi)}) x {nsets} / step time',
                kernels=kernels, dominant=max(kernels, key=lambda k: kernels[k]['share']),
                fft_tflops=round(fft_flops_per_eval(geom) * nsets / (ms_step / 1e3) / 1e12, 2))


def parity_sample(ev, w, bufs, nsets, data, err, sets=(0, 255, 511)):
    """Sampled parity of the benchmarked evaluator: model cubes and chi^2 of a
    few sets against the fp64 oracle chain (normwise relative errors)."""
    import torch
    from oracle import oracle
    from oracle.oracle import chi2 as chi2_ref, scube_pipeline
    from gbkfit_b200 import workloads
    if not os.path.exists(oracle.ORACLE_LIB):
        oracle.build()
    sets = [i for i in sets if i < nsets]
    nx, ny, nz = w.geom.size
    model = torch.zeros((nsets, nz, ny, nx), device=ev.dev)
    c = ev.evaluate_device(bufs, nsets, model=model).cpu().numpy()
    cubes = {i: model[i].cpu().numpy().astype(np.float64) for i in sets}
    del model
    errs, cerrs = [], []
    for i in sets:
        ref = scube_pipeline(w.disk.pack(workloads.set_params(w, i)), w.geom, precision='f64')
        errs.append(float(np.max(np.abs(cubes[i] - ref)) / np.max(np.abs(ref))))
        cr = chi2_ref(ref, data, err)
        cerrs.append(abs(float(c[i]) - cr) / cr)
    return dict(sets=sets, model_max_rel_err=max(errs), chi2_max_rel_err=max(cerrs),
                vs='fp64 oracle (smdisk on the padded grid, FFT convolution, crop, chi^2)')


def autotune(w, data, err, nsets, budget_s=60.0):
    """Time candidate pipeline shapes (chunk, rows per K1 group, FFT grid);
    returns the fastest configuration."""
    import torch
    from gbkfit_b200.autotune import tune_batched
    return tune_batched(w, data, err, nsets, budget_s=budget_s)


def run_e2e(args, w, data, err, cfg, nsets, total, world, local):
    """The same metric through the public API: every rank takes the whole batch
    of host parameter dicts, copies its share's raw parameter values (pinned
    H2D; the input rows are built on the device), evaluates it, reads its
    chi^2 back (D2H) and gathers all chi^2 values (NCCL all_gather across the
    ranks)."""
    import torch
    from gbkfit_b200.batched import BatchedSMDisk
    from gbkfit_b200.sharded import ShardedEvaluator
    ev_api = BatchedSMDisk(w.disk, w.geom, data, err, max_sets=nsets, device=local, **cfg)
    sharded = ShardedEvaluator(ev_api)
    d2h = nsets * 4
    try:
        for _ in range(max(1, args.warmup)):
            sharded.evaluate(w.params, total)
    except Exception:
        print(f'e2e diagnostics: world {sharded.world} rank {sharded.rank} share '
              f'{sharded.share(total)} max_sets {ev_api.max_sets} chunk {ev_api.chunk} '
              f'total {total} shapes { {k: np.shape(v) for k, v in w.params.items()} }',
              file=sys.stderr, flush=True)
        raise
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        chi2_all = sharded.evaluate(w.params, total)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks((time.perf_counter() - t0) / args.steps, world)
    assert len(chi2_all) == total and np.all(np.isfinite(chi2_all))
    h2d = int(ev_api.last_h2d_bytes)     # pinned input pieces copied per call
    e2e = dict(value=total / e2e_s, unit=UNIT, h2d_bytes_per_step=h2d,
               d2h_bytes_per_step=d2h, ms_per_step=e2e_s * 1e3,
               gather_bytes_per_step=sharded.last_gather_bytes,
               path='ShardedEvaluator(BatchedSMDisk).evaluate: host parameter dicts of all '
                    f'{total} sets in, chi^2 of all sets out on every rank')

    return e2e


def run_b200(args):
    import torch
    from gbkfit_b200 import workloads
    from gbkfit_b200.batched import BatchedSMDisk, synthetic_data
    from gbkfit_b200.sharded import ShardedEvaluator, shard_sets, slice_sets
    rank, world, local = setup_dist(args)
    nsets = args.nsets
    # one batch of nsets x world sets (the same seeded draw on every rank);
    # rank r evaluates its contiguous share of nsets sets
    total = nsets * world
    w = workloads.smdisk_batch128(nsets=total, seed=1234)
    lo, hi = shard_sets(total, rank, world)
    mine = slice_sets(w.params, total, lo, hi)
    data, err, _ = synthetic_data(w, device=local)
    cfg = autotune(w, data, err, nsets, budget_s=args.tune_budget) if args.tune else {}
    if args.conv:
        cfg['conv'] = args.conv
        if args.conv == 'direct':
            cfg['fft_size'] = (0, 0, 0)
    if args.chunk:
        cfg['chunk'] = args.chunk
    if args.band:
        cfg['band'] = args.band
    if args.psf_variant >= 0:
        cfg['psf_variant'] = args.psf_variant
    if args.model_variant >= 0:
        cfg['model_variant'] = args.model_variant
    ev = BatchedSMDisk(w.disk, w.geom, data, err, max_sets=nsets, device=local, **cfg)
    bufs = ev.alloc_inputs(nsets)
    ev.upload(ev.pack(mine, nsets), bufs, nsets)
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device='cuda')
    use_graph = not args.no_graph
    if use_graph:
        ev.capture(bufs, nsets)
        run = ev.replay
    else:
        run = lambda: ev.evaluate_device(bufs, nsets)
    for _ in range(args.warmup):
        run()
    torch.cuda.synchronize()
    barrier(world)
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    torch.cuda.synchronize()
    barrier(world)
    for i in range(args.steps):
        flush.fill_(float(i))            # evict L2 between timed steps
        ev0[i].record(stream)
        run()
        ev1[i].record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = [a.elapsed_time(b) for a, b in zip(ev0, ev1)]
    ms_step = max_over_ranks(float(np.mean(ms)), world)
    value = world * nsets / (ms_step / 1e3)
    chi2 = ev.chi2[:nsets].cpu().numpy()
    assert np.all(np.isfinite(chi2)) and np.all(chi2 > 0)

    # per-kernel device time: the same evaluation launched without the graph,
    # with a CUDA event pair around every launch on the evaluator's stream and
    # no work counters; then one more pass with the counters for the executed
    # work (their atomic adds would lengthen the timed launches)
    ev.set_timing(True, counters=False)
    ev.stage_times()
    for i in range(args.steps):
        flush.fill_(float(i))
        ev.evaluate_device(bufs, nsets)
    stages = ev.stage_times()
    ev.set_timing(True, counters=True)
    ev.work_counters()
    for i in range(args.steps):
        flush.fill_(float(i))
        ev.evaluate_device(bufs, nsets)
    ev.stage_times()
    counters = ev.work_counters()
    ev.set_timing(False)
    tsum = sum(t for t, _ in stages.values())
    kernels = {k: dict(launches_per_step=n / args.steps, ms_per_step=round(t / args.steps, 4),
                       ms_per_launch=round(t / n, 5), share=round(t / tsum, 4))
               for k, (t, n) in stages.items()}

    e2e = None
    if args.e2e:
        e2e = run_e2e(args, w, data, err, cfg, nsets, total, world, local)
    out = None
    if rank == 0:
        n_chunks = (nsets + ev.chunk - 1) // ev.chunk
        per_chunk = 2 if ev.conv_mode == 'direct' else 5
        plain = plain_per_call(w, data, err) if args.plain else None
        serving = serving_run() if args.serving else None
        cpu = cpu_baseline(w, data, err) if args.cpu_baseline else None
        parity = parity_sample(ev, w, bufs, nsets, data, err) if args.parity else None
        if ev.conv_mode == 'direct':
            roof = roofline_direct(kernels, counters, args.steps, nsets, clocks, w.geom, ms_step)
        else:
            roof = roofline_fft(kernels, nsets, w.geom, ms_step)
        out = dict(
            metric=METRIC, value=round(value, 1), unit=UNIT, n_gpus=world, steps=args.steps,
            warmup=args.warmup, ms_per_step=round(ms_step, 4), higher_is_better=True,
            scaling='weak', vs_baseline=None, dtype='f32', data='synthetic',
            config=dict(workload='smdisk_batch128: 512 sets x 128x128x96 cube, 30 rings, '
                                 'Gaussian PSF FWHM 3 px x Gaussian LSF FWHM 1.5 ch, chi^2',
                        nsets_per_gpu=nsets, conv=ev.conv_mode, psf_rank=ev.psf_rank,
                        fft_grid=list(ev.fft_size), chunk=ev.chunk,
                        tuned=cfg, cuda_graph=use_graph, l2='flushed between steps (256 MB write)',
                        parallelism=f'dp{world} (parameter sets sharded across GPUs, '
                                    'chi^2 all_gather)'),
            e2e=e2e,
            roofline=roof,
            parity=parity,
            clocks=clocks,
            gpu_launches=args.steps * (per_chunk * n_chunks + 1),
            plain_per_call=plain,
            serving=serving,
            cpu_baseline=cpu,
        )
    if world > 1:
        import torch.distributed as dist
        ev._graph = None
        dist.destroy_process_group()
    return out


def serving_run(nrequests=10000, slots=8, load=0.8, batch_sets=32, mc_sets=8):
    """The serving stream (workloads.serving_stream: 64 datasets, 70 % smdisk /
    30 % mcdisk, sides 32-256 px, 32-192 channels, 1e5-1e7 clouds): capacity
    with every request submitted at once, then Poisson arrivals at `load` x
    capacity; latency = completion - scheduled arrival, and includes the
    packing of the request's parameters (in submit).  Every dataset is
    registered with its smdisk disk, so its smdisk requests are coalesced
    into batched launches (direct separable convolution, up to batch_sets
    sets each) and its mcdisk requests into launches of up to mc_sets
    cloud cubes on the evaluator's window (the same direct convolution)."""
    import torch
    from gbkfit_b200 import workloads
    from gbkfit_b200.serving import ModelServer, Request
    st = workloads.serving_stream(nrequests=nrequests, ndatasets=64, rate=1.0, seed=7)

    def reqs():
        return [Request(q['dataset'], q['kind'], st.datasets[q['dataset']][q['kind']],
                        q['params'], cflux=q['cflux'], thick=q['thick']) for q in st.requests]

    with ModelServer(slots=slots, hbm_budget=40 << 30) as srv:
        for d in st.datasets:
            srv.register(d['key'], d['geom'], d['data'], d['error'], smdisk=d['smdisk'],
                         batch_sets=batch_sets, mc_sets=mc_sets)
        [f.result() for f in [srv.submit(r) for r in reqs()[:300]]]     # plans, allocator
        srv.stats(reset=True)
        [f.result() for f in [srv.submit(r) for r in reqs()]]
        cap = srv.stats(reset=True)['evals_per_s']
        rate = load * cap
        arr = np.cumsum(np.random.default_rng(1).exponential(1 / rate, nrequests))
        rs = reqs()
        t0 = time.perf_counter()
        futs = []
        for r, a in zip(rs, arr):
            now = time.perf_counter() - t0
            if a > now:
                time.sleep(a - now)
            r.arrival = t0 + a
            futs.append(srv.submit(r))
        [f.result() for f in futs]
        s = srv.stats(reset=True)
        resident = srv._resident
    return dict(requests=nrequests, slots=slots, batch_sets=batch_sets, mc_sets=mc_sets,
                max_group=s.get('max_group'), capacity_evals_per_s=round(cap, 1),
                offered_evals_per_s=round(rate, 1), evals_per_s=round(s['evals_per_s'], 1),
                p50_ms=round(s['p50_ms'], 3), p99_ms=round(s['p99_ms'], 3),
                max_ms=round(s['max_ms'], 3), resident_gb=round(resident / 1e9, 3),
                latency='completion - arrival, parameter packing included',
                workload='serving_stream: 64 datasets (sides log-U 32-256 px, channels '
                         'log-U 32-192, PSF FWHM U(1.5,4) px, LSF FWHM U(1,3) ch), '
                         '70% smdisk / 30% mcdisk (1e5-1e7 clouds), chi^2 per request')


def plain_per_call(w, data, err, nsets=16):
    """The reference-style per-call path on the GPU: one synchronous
    DModelSCube evaluation + Objective.log_likelihood per parameter set."""
    import torch
    from gbkfit_b200 import model as M, workloads
    from gbkfit_b200.driver import DriverB200
    drv = DriverB200(torch.cuda.current_device())
    comp = M.SpectralSMDisk2D(False, False, w.disk.traits['rpt'], w.disk.traits['vpt'],
                              w.disk.traits['dpt'], rnodes=w.disk.rnodes)
    g = w.geom
    dm = M.DModelSCube(g.size, g.step, rpix=(0, 0, (g.size[2] - 1) / 2), rval=(0, 0, 0),
                       psf=g.psf, lsf=g.lsf)
    obj = M.Objective(M.Model(drv, dm, M.GModelKinematics2D([comp])), data, err)
    for i in range(3):
        obj.log_likelihood(workloads.set_params(w, i))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(nsets):
        obj.log_likelihood(workloads.set_params(w, i % w.nsets))
    dt = time.perf_counter() - t0
    return dict(value=round(nsets / dt, 1), unit=UNIT, sets=nsets,
                path='DModelSCube + Objective.log_likelihood, one synchronous call chain per set')


def reference_eval(ref, w, data, err, i, workers):
    """One evaluation with the reference's own CPU code: smdisk and the
    residual/sum from oracle/_ref, FFT convolution with scipy (FFTW stand-in)."""
    from oracle.oracle import fft_convolve_cached
    from gbkfit_b200 import workloads
    g = w.geom
    p = w.disk.pack(workloads.set_params(w, i))
    ss, st, sz = g.spat(False)
    nz = g.size_hi[2]
    geo = dict(loose=False, tilted=False, spat_size=ss, spat_step=st, spat_zero=sz,
               spec_size=nz, spec_step=g.step[2], spec_zero=g.zero_hi[2], opacity=None)
    cube = np.zeros((nz, ss[1], ss[0]), np.float32)
    ref.smdisk_evaluate(p, geo, dict(scube=cube))
    conv = fft_convolve_cached(cube, w._pcube, dtype=np.float32, workers=workers)
    ex, ey, ez = g.edge
    nx, ny, nzl = g.size
    crop = np.ascontiguousarray(conv[ez:ez + nzl, ey:ey + ny, ex:ex + nx], np.float32)
    res = ref.residual(data, err, None, crop, None, None, 1.0)
    return ref.residual_sum(res, True)


def cpu_baseline(w, data, err, sample_sets=4):
    """Bounded sample of the workload on the reference CPU path."""
    from oracle.oracle import Reference, build
    if not Reference.available():
        build()
    ref = Reference()
    workers = os.cpu_count()
    w._pcube = w.geom.pcube(np.float32)
    reference_eval(ref, w, data, err, 0, workers)
    t0 = time.perf_counter()
    for i in range(sample_sets):
        reference_eval(ref, w, data, err, i, workers)
    dt = time.perf_counter() - t0
    return dict(value=round(sample_sets / dt, 2), unit=UNIT, cores=ref.num_threads(),
                kind='reference',
                sample=f'{sample_sets} of the 512 parameter sets; smdisk and residual sum '
                       f'from the reference templates (OpenMP, {ref.num_threads()} threads), '
                       f'FFT convolution with scipy.fft ({workers} workers) standing in for '
                       f'FFTW on the reference padded grid {list(w.geom.size_hi)}')


def run_reference(args):
    rank, world = int(os.environ.get('RANK', 0)), int(os.environ.get('WORLD_SIZE', 1))
    if rank != 0:
        return None
    from gbkfit_b200 import workloads
    from oracle.oracle import Reference, build, scube_pipeline
    if not Reference.available():
        build()
    ref = Reference()
    w = workloads.smdisk_batch128(nsets=args.nsets)
    # data: the fp64 oracle model of the truth parameters plus the seeded noise
    truth = w.disk.pack(w.extra['truth'])
    m = scube_pipeline(truth, w.geom)
    rng = np.random.default_rng(w.extra['noise_seed'])
    sigma = w.extra['noise_frac'] * float(np.max(m))
    data = (m + rng.normal(0.0, sigma, m.shape)).astype(np.float32)
    err = np.full(m.shape, sigma, np.float32)
    workers = os.cpu_count()
    w._pcube = w.geom.pcube(np.float32)
    per_step = 2
    for i in range(args.warmup):
        reference_eval(ref, w, data, err, i, workers)
    t0 = time.perf_counter()
    k = 0
    for s in range(args.steps):
        for j in range(per_step):
            reference_eval(ref, w, data, err, k % args.nsets, workers)
            k += 1
    dt = time.perf_counter() - t0
    value = k / dt
    cpu = dict(value=round(value, 2), unit=UNIT, cores=ref.num_threads(), kind='reference',
               sample=f'{per_step} parameter sets per step of the 512-set workload')
    return dict(metric=METRIC, value=round(value, 2), unit=UNIT, n_gpus=world,
                steps=args.steps, warmup=args.warmup,
                ms_per_step=round(dt / args.steps * 1e3, 2), higher_is_better=True,
                scaling='weak', vs_baseline=None, dtype='f32', data='synthetic',
                config=dict(workload='smdisk_batch128: 512 sets x 128x128x96 cube, 30 rings, '
                                     'Gaussian PSF FWHM 3 px x Gaussian LSF FWHM 1.5 ch, chi^2',
                            sets_per_step=per_step),
                impl='reference', cpu_baseline=cpu,
                e2e=dict(value=round(value, 2), unit=UNIT, h2d_bytes_per_step=0,
                         d2h_bytes_per_step=0))


# ---- secondary workloads (one JSON line each; not the headline metric) -------

KINDS = ('rpt', 'rht', 'vpt', 'vht', 'dpt', 'dht', 'zpt', 'spt', 'wpt')


def _device_packed(packed, dev):
    """Disk.pack() host arrays -> torch tensors on the device."""
    import torch
    out = {}
    for k, v in packed.items():
        if v is None:
            out[k] = None
        elif isinstance(v, dict):
            out[k] = {f: torch.from_numpy(np.ascontiguousarray(a)).to(dev) for f, a in v.items()}
        else:
            out[k] = torch.from_numpy(np.ascontiguousarray(v)).to(dev)
    return out


def _trait_args(pd):
    args = []
    for k in KINDS:
        t = pd[k]
        args += [None] * 5 if t is None else [t['uids'], t['cvalues'], t['ccounts'],
                                              t['pvalues'], t['pcounts']]
    return args


def _events_ms(fn, steps, warmup):
    """Mean device ms of fn() over `steps` calls (CUDA events on the current
    stream, L2 flushed before every call), after `warmup` calls."""
    import torch
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device='cuda')
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0 = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    e1 = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    stream = torch.cuda.current_stream()
    for i in range(steps):
        flush.fill_(float(i))
        e0[i].record(stream)
        fn()
        e1[i].record(stream)
    torch.cuda.synchronize()
    return float(np.mean([a.elapsed_time(b) for a, b in zip(e0, e1)]))


def run_mcdisk(args):
    """mcdisk_cube256: 1e7 clouds of a thick exponential disk into the
    320x320x320 (spatial) x 160 (channels) padded grid, through the drop-in
    gmodel backend (fast and deterministic modes); the reference's mcdisk
    template (OpenMP) on the host cores for the same call."""
    import torch
    from gbkfit_b200 import workloads
    from gbkfit_b200.driver import DriverB200
    w = workloads.mcdisk_cube256()
    csum = w.disk.ncloudscsum(w.params, w.cflux)
    hoi = w.disk.hasordint()
    n = int(csum[-1])
    g = w.geometry_args()
    nx, ny, _ = g['spat_size']
    nz = g['spec_size']
    packed = w.disk.pack(w.params)
    pd = _device_packed(packed, 'cuda')
    cs, hs = torch.from_numpy(csum).cuda(), torch.from_numpy(hoi).cuda()
    scube = torch.zeros((nz, ny, nx), device='cuda')
    gm = DriverB200(torch.cuda.current_device()).backends().gmodel(np.float32)

    def call():
        scube.zero_()
        gm.mcdisk_evaluate(w.cflux, n, cs, hs, g['loose'], g['tilted'], pd['subrnodes'],
                           pd['vsys'], pd['xpos'], pd['ypos'], pd['posa'], pd['incl'],
                           *_trait_args(pd), g.get('opacity'), g['spat_size'], g['spat_step'],
                           g['spat_zero'], 0.0, g['spec_size'], g['spec_step'],
                           g['spec_zero'], None, scube, None, None, None, None, None, None,
                           None, None)

    ms = {}
    for mode, name in ((0, 'fast'), (1, 'deterministic'), (3, 'scalar_atomics')):
        gm.set_mcdisk(seed=42, mode=mode)
        ms[name] = _events_ms(call, args.steps, args.warmup)
    gm.set_mcdisk(seed=42, mode=0)
    cpu = None
    if args.cpu_baseline:
        from oracle.oracle import Reference, build
        if not Reference.available():
            build()
        ref = Reference()
        h = np.zeros((nz, ny, nx), np.float32)
        t0 = time.perf_counter()
        ref.mcdisk_evaluate(w.cflux, n, csum, hoi, packed, g, dict(scube=h))
        dt = time.perf_counter() - t0
        cpu = dict(value=round(1 / dt, 3), unit='evals/s', cores=ref.num_threads(),
                   kind='reference', sample='one full call (1e7 clouds)')
    return dict(metric='mcdisk evals/s (1e7 clouds, thick disk, padded 320x320x320 x 160 grid)',
                value=round(1e3 / ms['fast'], 2), unit='evals/s', n_gpus=1, steps=args.steps,
                warmup=args.warmup, ms_per_step=round(ms['fast'], 4),
                ms_deterministic=round(ms['deterministic'], 4),
                ms_scalar_atomics=round(ms['scalar_atomics'], 4), higher_is_better=True,
                dtype='f32', data='synthetic', gpu_launches=args.steps,
                config=dict(workload='mcdisk_cube256', nclouds=n, grid=[nx, ny, g['spat_size'][2], nz],
                            l2='flushed before every call (256 MB write)'),
                cpu_baseline=cpu)


def _c0_reference_eval(ref, w0, pcube, workers):
    """One plain smdisk evaluation with the reference's own CPU code: smdisk
    (oracle/_ref, OpenMP) on the padded 96^3 grid, the FFT convolution with
    scipy (standing in for FFTW, which is not installed), the crop and the
    moment maps 0/1/2 (oracle/_ref).  Returns (maps, cube)."""
    from oracle.oracle import fft_convolve_cached
    g = w0.geom
    ga = w0.geometry_args()
    hh = np.zeros((ga['spec_size'], ga['spat_size'][1], ga['spat_size'][0]), np.float32)
    ref.smdisk_evaluate(w0.disk.pack(w0.params), ga, dict(scube=hh))
    conv = fft_convolve_cached(hh, pcube, dtype=np.float32, workers=workers)
    ex, ey, ez = g.edge
    nx, ny, nz = g.size
    cube = np.ascontiguousarray(conv[ez:ez + nz, ey:ey + ny, ex:ex + nx], np.float32)
    zero = (0.0, 0.0, -(nz - 1) / 2 * g.step[2])
    maps = ref.mmaps_moments(g.size, g.step, zero, cube, None, 1e-6, np.array([0, 1, 2], np.int32))
    return maps, cube


def run_smdisk64(args):
    """smdisk_cube64, the plain configuration end to end: thin smdisk on the
    64^3 cube -> PSF x LSF FFT convolution on the padded 96^3 grid -> crop ->
    moment maps 0, 1, 2 and the full cube, through the drop-in DModelMMaps
    (one synchronous call chain per evaluation, the reference's semantics),
    host parameters in, host maps and cube out.  The reference's CPU code for
    the same chain (OpenMP smdisk and moments from oracle/_ref, scipy's FFT
    standing in for FFTW) is timed beside it on the host cores."""
    import torch
    from gbkfit_b200 import model as M, workloads
    from gbkfit_b200.driver import DriverB200
    w0 = workloads.smdisk_cube64()
    drv = DriverB200(torch.cuda.current_device())
    comp = M.SpectralSMDisk2D(False, False, w0.disk.traits['rpt'], w0.disk.traits['vpt'],
                              w0.disk.traits['dpt'], rnodes=w0.disk.rnodes)
    g0 = w0.geom
    dm = M.DModelMMaps(g0.size, g0.step, rpix=(0, 0, (g0.size[2] - 1) / 2), rval=(0, 0, 0),
                       psf=g0.psf, lsf=g0.lsf, orders=(0, 1, 2))
    mdl = M.Model(drv, dm, M.GModelKinematics2D([comp]))

    def call():
        out = mdl.evaluate_d(w0.params)
        maps = [out[f'mmap{o}']['d'].cpu().numpy() for o in (0, 1, 2)]
        cube = dm.dcube().dcube().cpu().numpy()
        return maps, cube

    for _ in range(args.warmup):
        call()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        maps, cube = call()
    ms = (time.perf_counter() - t0) / args.steps * 1e3
    # device time of the same chain (CUDA events around the call, L2 flushed)
    dev_ms = _events_ms(lambda: mdl.evaluate_d(w0.params), args.steps, args.warmup)
    cpu = None
    parity = None
    if args.cpu_baseline:
        from oracle.oracle import Reference, build
        if not Reference.available():
            build()
        ref = Reference()
        workers = os.cpu_count()
        pcube = g0.pcube(np.float32)
        (rd, _, _), rcube = _c0_reference_eval(ref, w0, pcube, workers)
        n = max(3, args.steps)
        t0 = time.perf_counter()
        for _ in range(n):
            _c0_reference_eval(ref, w0, pcube, workers)
        dt = (time.perf_counter() - t0) / n
        cpu = dict(value=round(1 / dt, 2), unit='evals/s', cores=ref.num_threads(),
                   kind='reference', ms_per_eval=round(dt * 1e3, 3),
                   sample=f'{n} evaluations of the same chain: smdisk + moments from the '
                          'reference templates (OpenMP), scipy.fft (all cores) for the FFT')
        # moment 0 on the spaxels the reference keeps; moments 1 and 2 (ratios
        # to moment 0) where moment 0 is at least 1e-3 of its peak: near the
        # 1e-6 cutoff the fp32 convolution's noise dominates them in any fp32
        # chain, the reference's included
        v = np.isfinite(rd[0])
        m0 = np.where(v, rd[0], 0.0)
        strong = v & (np.abs(m0) >= 1e-3 * np.max(np.abs(m0)))
        sel = [v, strong, strong]
        nrm = lambda a: float(np.sqrt(np.sum(np.asarray(a, np.float64) ** 2)))
        parity = dict(vs='the reference CPU chain (fp32)',
                      cube_rel_err=nrm(cube - rcube) / nrm(rcube),
                      map_rel_err=[nrm(maps[i][sel[i]] - rd[i][sel[i]]) / nrm(rd[i][sel[i]])
                                   for i in range(3)],
                      norm='normwise (L2) relative; maps 1, 2 where map 0 >= 1e-3 of its peak '
                           f'({int(strong.sum())} of {int(v.sum())} spaxels)')
    return dict(metric='smdisk_cube64 evaluations/s (smdisk -> PSF/LSF FFT -> moments 0/1/2 '
                       '+ cube, per call, synchronous)',
                value=round(1e3 / ms, 1), unit='evals/s', n_gpus=1, steps=args.steps,
                warmup=args.warmup, ms_per_step=round(ms, 4), device_ms=round(dev_ms, 4),
                higher_is_better=True, dtype='f32', data='synthetic',
                config=dict(workload='smdisk_cube64: 64^3 cube, 20 nodes, Gaussian PSF FWHM 2.5 px '
                                     'x LSF FWHM 2 ch, padded 96^3, moments 0/1/2',
                            path='Model.evaluate_d (DModelMMaps), host maps + cube out'),
                e2e=dict(value=round(1e3 / ms, 1), unit='evals/s',
                         h2d_bytes_per_step=None,
                         d2h_bytes_per_step=int(3 * 64 * 64 * 4 + 64 ** 3 * 4)),
                cpu_baseline=cpu, parity=parity)


def run_grad96(args):
    """grad96: chi^2 and its gradient (66 parameters) of smdisk + PSF/LSF on a
    96x96x64 cube through the hand-written adjoint; the data are the GPU
    model of the truth parameters plus seeded noise of 2 % of the peak."""
    import torch
    from gbkfit_b200 import workloads
    from gbkfit_b200.adjoint import SMDiskChi2, to_vector
    w = workloads.smdisk_grad96()
    shape = tuple(w.geom.size[::-1])
    probe = SMDiskChi2(w.disk, w.geom, np.zeros(shape, np.float32), np.ones(shape, np.float32))
    probe.value(to_vector(w.extra['truth'], 1.0))
    ex, ey, ez = w.geom.edge
    nx, ny, nz = w.geom.size
    m = probe.scube[ez:ez + nz, ey:ey + ny, ex:ex + nx].double().cpu().numpy()
    rng = np.random.default_rng(w.extra['noise_seed'])
    sigma = w.extra['noise_frac'] * float(np.max(m))
    data = (m + rng.normal(0.0, sigma, m.shape)).astype(np.float32)
    err = np.full(m.shape, sigma, np.float32)
    model = SMDiskChi2(w.disk, w.geom, data, err)
    theta = to_vector(w.params, w.extra['scale'])
    for _ in range(args.warmup):
        model.value_and_grad(theta)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        model.value_and_grad(theta)
    ms = (time.perf_counter() - t0) / args.steps * 1e3
    return dict(metric='grad96 chi^2 + gradient evaluations/s (66 parameters)',
                value=round(1e3 / ms, 1), unit='evals/s', n_gpus=1, steps=args.steps,
                warmup=args.warmup, ms_per_step=round(ms, 4), higher_is_better=True,
                dtype='f32', data='synthetic',
                config=dict(workload='smdisk_grad96: 96x96x64 cube, 20 nodes, 66 parameters',
                            path='SMDiskChi2.value_and_grad (host vector in, host gradient out)'))


def run_fft_conv(args):
    """fft_conv: the drop-in FFT convolution (gbkb200_fft_convolve_cached:
    r2c, multiply by the cached PSF x LSF spectrum / N, c2r; fft.hpp:98-207)
    on the padded grids of the mcdisk configuration (320 x 320 x 160) and of
    the largest serving request (288 x 288 x 224), and the batched evaluator
    in FFT mode (a Moffat PSF, not separable) on the batched configuration's
    512 sets of 128 x 128 x 96.  The convolution's bytes are those of its own
    five passes over the cube: x r2c (4 V read, 8 C written), y (16 C), z with
    the multiply (24 C: read, spectrum, write), inverse y (16 C), x c2r (8 C
    read, 4 V written) = 8 V + 72 C, V = voxels, C = (nx/2 + 1) ny nz."""
    import torch
    from gbkfit_b200 import psflsf, workloads
    from gbkfit_b200.batched import BatchedSMDisk, synthetic_data
    from gbkfit_b200.driver import DriverB200
    hbm, peak_kind = peaks()
    fft = DriverB200(torch.cuda.current_device()).backends().fft(np.float32)
    grids = []
    for name, (nx, ny, nz) in (('mcdisk_cube256 padded', (320, 320, 160)),
                               ('serving max padded', (288, 288, 224))):
        g = torch.Generator(device='cuda').manual_seed(1)
        cube = torch.rand((nz, ny, nx), device='cuda', generator=g)
        kern = torch.rand((nz, ny, nx), device='cuda', generator=g)
        kern /= kern.sum()
        work = cube.clone()

        def call():
            work.copy_(cube)
            fft.fft_convolve_cached(work, kern)

        copy_ms = _events_ms(lambda: work.copy_(cube), args.steps, args.warmup)
        ms = _events_ms(call, args.steps, args.warmup) - copy_ms
        v, c = nx * ny * nz, (nx // 2 + 1) * ny * nz
        b = 8 * v + 72 * c
        grids.append(dict(grid=[nx, ny, nz], what=name, ms=round(ms, 4),
                          pass_bytes=b, achieved_gbs=round(b / (ms / 1e3) / 1e9, 1),
                          frac=round(b / (ms / 1e3) / 1e9 / hbm, 3),
                          minimal_bytes=8 * v + 8 * c,
                          note='ms excludes the copy that restores the input'))
    # batched FFT mode: Moffat PSF (FWHM 3 px, beta 2.5) on the batched cube
    w = workloads.smdisk_batch128(nsets=args.nsets)
    w.geom = workloads.Geometry(w.geom.size, w.geom.step, (0, 0, (w.geom.size[2] - 1) / 2),
                                (0, 0, 0), psflsf.PSFMoffat(psflsf.moffat_fwhm_beta_to_alpha(3.0, 2.5),
                                                            2.5), w.geom.lsf)
    data, err, _ = synthetic_data(w)
    ev = BatchedSMDisk(w.disk, w.geom, data, err, max_sets=args.nsets, chunk=16, conv='fft')
    bufs = ev.alloc_inputs(args.nsets)
    ev.upload(ev.pack(w.params, args.nsets), bufs, args.nsets)
    ev.capture(bufs, args.nsets)
    bms = _events_ms(ev.replay, args.steps, args.warmup)
    return dict(metric='drop-in FFT convolution GB/s (own passes) and batched FFT-mode evals/s',
                value=grids[0]['achieved_gbs'], unit='GB/s', n_gpus=1, steps=args.steps,
                warmup=args.warmup, higher_is_better=True, dtype='f32', data='synthetic',
                roofline=dict(bound='hbm', achieved=grids[0]['achieved_gbs'], peak=hbm,
                              unit='GB/s', frac=grids[0]['frac'], peak_kind=peak_kind,
                              kernel='fft_convolve_cached (5 passes)', traffic=None),
                grids=grids,
                batched_fft=dict(workload='smdisk_batch128 sets with a Moffat PSF (FWHM 3 px, '
                                          'beta 2.5): FFT mode', nsets=args.nsets,
                                 fft_grid=list(ev.fft_size), chunk=ev.chunk,
                                 ms_per_step=round(bms, 4),
                                 evals_per_s=round(args.nsets / (bms / 1e3), 1)))


def run_serving(args):
    out = serving_run(nrequests=args.requests)
    return dict(metric='serving capacity evals/s and latency (ms)',
                value=out['capacity_evals_per_s'], unit='evals/s', n_gpus=1,
                higher_is_better=True, dtype='f32', data='synthetic', serving=out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    ap.add_argument('--nsets', type=int, default=512)
    ap.add_argument('--no-graph', action='store_true')
    ap.add_argument('--no-tune', dest='tune', action='store_false')
    ap.add_argument('--tune-budget', type=float, default=40.0)
    ap.add_argument('--no-plain', dest='plain', action='store_false')
    ap.add_argument('--no-serving', dest='serving', action='store_false')
    ap.add_argument('--no-cpu-baseline', dest='cpu_baseline', action='store_false')
    ap.add_argument('--no-e2e', dest='e2e', action='store_false',
                    help='skip the end-to-end (public API) measurement')
    ap.add_argument('--no-parity', dest='parity', action='store_false',
                    help='skip the sampled parity check against the fp64 oracle')
    ap.add_argument('--conv', choices=['fft', 'direct'], default=None,
                    help='force the convolution mode (default: tuned)')
    ap.add_argument('--chunk', type=int, default=0, help='force the sets per wave (default: tuned)')
    ap.add_argument('--psf-variant', type=int, default=-1, choices=[-1, 0, 1, 2, 3, 4, 5, 6, 7],
                    help='PSF kernel variant of the direct mode (default: tuned)')
    ap.add_argument('--model-variant', type=int, default=-1, choices=[-1, 0, 1, 2, 3, 4],
                    help='model kernel of the direct mode: 0 one chunk per warp, 1 chunk '
                         'pairs, 2 4x8 spaxel tiles, 3 tiles with transposed range masks, '
                         '4 as 3 with the scaled line exponent (default: tuned)')
    ap.add_argument('--band', type=int, default=0,
                    help='force the output rows per PSF block of the direct mode (default: tuned)')
    ap.add_argument('--workload', default='smdisk_batch128',
                    choices=['smdisk_batch128', 'mcdisk_cube256', 'smdisk_cube64', 'grad96',
                             'serving', 'fft_conv'],
                    help='smdisk_batch128 is the headline; the others print their own line')
    ap.add_argument('--requests', type=int, default=10000, help='serving workload: requests')
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    other = dict(mcdisk_cube256=run_mcdisk, smdisk_cube64=run_smdisk64, grad96=run_grad96,
                 serving=run_serving, fft_conv=run_fft_conv)
    if args.workload in other and args.impl != 'reference':
        import torch
        torch.cuda.set_device(0)
        out = other[args.workload](args)
    elif args.impl == 'reference':
        out = run_reference(args)
    else:
        out = run_b200(args)
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == '__main__':
    main()
