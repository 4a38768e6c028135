"""Multi-process (gloo, world size 2, CPU) tests of the sharded objective
(gbkfit_b200.sharded.ShardedEvaluator): every rank evaluates its share of
the parameter sets and the chi^2 of all sets is gathered to every rank.  On
the CPU an oracle-backed evaluator stands in for each rank's GPU evaluator
(the same interface as BatchedSMDisk: evaluate(params, nsets), max_sets);
the sharding, the slicing of the per-set parameters, the padding and the
gather are the product's.

* sharded chi^2 == the single-process chi^2, exactly, for uneven shares and
  batches larger than one rank's max_sets;
* emcee's vectorised log-probability (fitting.BatchedLogProbability) on top of
  the sharded evaluator gives every rank the same values;
* parameters held by one rank reach the others (broadcast_theta);
* a rank that fails before the gather is detected by the others through the
  process group's timeout."""

import os
import socket

import numpy as np


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _problem():
    from oracle.oracle import scube_pipeline
    from gbkfit_b200 import workloads
    w = workloads.smdisk_batch128(nsets=7, size=(24, 20, 16), nnodes=8)
    truth = w.disk.pack(w.extra['truth'])
    m = scube_pipeline(truth, w.geom)
    rng = np.random.default_rng(w.extra['noise_seed'])
    sigma = 0.02 * float(np.max(m))
    data = m + rng.normal(0, sigma, m.shape)
    err = np.full(m.shape, sigma)
    return w, data, err


class OracleEvaluator:
    """The per-rank evaluator interface of BatchedSMDisk, scored by the fp64
    oracle (test stand-in for a rank's GPU)."""

    def __init__(self, w, data, err, max_sets=2):
        self.w, self.data, self.err, self.max_sets = w, data, err, max_sets
        self.calls = []

    def evaluate(self, params, nsets):
        from oracle.oracle import chi2, scube_pipeline
        assert nsets <= self.max_sets
        self.calls.append(nsets)
        out = []
        for i in range(nsets):
            p = {k: (np.asarray(v)[i] if np.ndim(v) and np.shape(v)[0] == nsets else v)
                 for k, v in params.items()}
            out.append(chi2(scube_pipeline(self.w.disk.pack(p), self.w.geom), self.data,
                            self.err))
        return np.array(out)


def _worker(rank, world, port, out, fail_rank):
    import datetime
    import torch.distributed as dist
    from gbkfit_b200 import fitting
    from gbkfit_b200.sharded import ShardedEvaluator, broadcast_theta
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=20))
    try:
        if rank == fail_rank:
            raise RuntimeError('injected failure before the gather')
        w, data, err = _problem()
        local = OracleEvaluator(w, data, err, max_sets=2)
        sh = ShardedEvaluator(local)
        chi2 = sh.evaluate(w.params, 7)
        # the sampler-side objective over the sharded evaluator: theta held by
        # rank 0 only, broadcast to the others
        template = {k: (np.asarray(v)[0] if np.ndim(v) and np.shape(v)[0] == 7 else v)
                    for k, v in w.params.items()}
        fp = fitting.FreeParams(template, {'incl': fitting.PriorUniform(10, 85),
                                           'vpt_vt[3]': fitting.PriorUniform(0, 400)})
        theta = np.stack([w.params['incl'], w.params['vpt_vt'][:, 3]], axis=1) \
            if rank == 0 else None
        theta = broadcast_theta(theta, src=0, ndim=2)
        post, blobs = fitting.BatchedLogProbability(sh, fp)(theta)
        out.put((rank, 'ok', dict(chi2=chi2.tolist(), post=post.tolist(), calls=local.calls,
                                  share=sh.share(7), theta=theta.tolist())))
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
    return sorted(res, key=lambda r: r[0])


def test_sharded_chi2_equals_single_process(oracle_built):
    from gbkfit_b200 import fitting
    from gbkfit_b200.sharded import ShardedEvaluator
    w, data, err = _problem()
    single_ev = OracleEvaluator(w, data, err, max_sets=7)
    single = ShardedEvaluator(single_ev).evaluate(w.params, 7)     # world 1: no gather
    res = _run(2)
    for rank, status, got in res:
        assert status == 'ok', got
        assert np.array_equal(np.array(got['chi2']), single)
        assert got['share'] == [(0, 4), (4, 7)][rank]
        # shares of 4 and 3 sets, in calls of at most max_sets = 2
        assert got['calls'][:2] == ([2, 2] if rank == 0 else [2, 1])
    theta = np.stack([w.params['incl'], w.params['vpt_vt'][:, 3]], axis=1)
    assert np.array_equal(np.array(res[1][2]['theta']), theta)
    template = {k: (np.asarray(v)[0] if np.ndim(v) and np.shape(v)[0] == 7 else v)
                for k, v in w.params.items()}
    fp = fitting.FreeParams(template, {'incl': fitting.PriorUniform(10, 85),
                                       'vpt_vt[3]': fitting.PriorUniform(0, 400)})
    post_single, _ = fitting.BatchedLogProbability(single_ev, fp)(theta)
    for rank, status, got in res:
        assert np.allclose(got['post'], post_single, rtol=1e-12, atol=0)
    assert res[0][2]['post'] == res[1][2]['post']


def test_failed_rank_is_detected(oracle_built):
    res = _run(2, fail_rank=1)
    assert res[1][1] == 'error'          # the failing rank
    assert res[0][1] == 'error'          # the survivor's gather ends with an error
