"""Multi-process (gloo, world size 2, CPU) tests of the sharded objective:
parameter sets are split across ranks with shard_sets, every rank scores its
own sets (the oracle stands in for the GPU here), and gathering the chi^2
values reproduces the single-process result exactly.  A rank that fails
before joining the gather is detected by the others through the process
group's timeout."""

import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _chi2_of_sets(lo, hi):
    from oracle.oracle import chi2, scube_pipeline
    from gbkfit_b200 import workloads
    w = workloads.smdisk_batch128(nsets=6, size=(24, 20, 16), nnodes=8)
    truth = w.disk.pack(w.extra['truth'])
    m = scube_pipeline(truth, w.geom)
    rng = np.random.default_rng(w.extra['noise_seed'])
    sigma = 0.02 * float(np.max(m))
    data = m + rng.normal(0, sigma, m.shape)
    err = np.full(m.shape, sigma)
    return [chi2(scube_pipeline(w.disk.pack(workloads.set_params(w, i)), w.geom), data, err)
            for i in range(lo, hi)]


def _worker(rank, world, port, out, fail_rank):
    import torch
    import torch.distributed as dist
    import datetime
    from gbkfit_b200.batched import shard_sets
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=20))
    try:
        if rank == fail_rank:
            raise RuntimeError('injected failure before the gather')
        lo, hi = shard_sets(6, rank, world)
        mine = torch.tensor(_chi2_of_sets(lo, hi) + [0.0] * (3 - (hi - lo)), dtype=torch.float64)
        parts = [torch.zeros(3, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(parts, mine)
        vals = []
        for r in range(world):
            a, b = shard_sets(6, r, world)
            vals += parts[r][:b - a].tolist()
        out.put((rank, 'ok', vals))
    except Exception as e:
        out.put((rank, 'error', type(e).__name__))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _run(world, fail_rank=-1):
    import multiprocessing as mp
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, q, fail_rank)) for r in range(world)]
    for p in ps:
        p.start()
    res = [q.get(timeout=180) for _ in ps]
    for p in ps:
        p.join(timeout=60)
    return sorted(res)


def test_sharded_chi2_equals_single_process(oracle_built):
    res = _run(2)
    single = _chi2_of_sets(0, 6)
    for rank, status, vals in res:
        assert status == 'ok'
        assert np.allclose(vals, single, rtol=0, atol=0)


def test_failed_rank_is_detected(oracle_built):
    res = _run(2, fail_rank=1)
    assert res[1][1] == 'error'          # the failing rank
    assert res[0][1] == 'error'          # the survivor's gather ends with an error
