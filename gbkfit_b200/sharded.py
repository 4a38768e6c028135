"""Multi-GPU batched objective: parameter sets sharded across the ranks of a
process group, one GPU per rank, chi^2 gathered back.

The model evaluation of one parameter set needs nothing from any other set,
so the sets of a batch (the walkers of an ensemble step, the points a nested
sampler queues) are split into contiguous shares, one per rank.  Every rank
holds its own replica of the data cube, the PSF/LSF spectra and the evaluator
(a ``BatchedSMDisk`` on its GPU), evaluates its share, and the per-set chi^2
values of all shares are gathered to every rank with one ``all_gather`` of
``ceil(nsets / world)`` floats per rank (NCCL over NVLink for GPU process
groups, gloo for CPU ones).  That gather is the only data exchanged.

The ranks run SPMD: every rank calls ``evaluate`` with the same full batch
(samplers started from the same seed propose the same walkers on every
rank, and every rank then accepts the same moves from the same gathered
values).  A caller whose parameters live on one rank only broadcasts them
first with ``broadcast_theta``.

The reference evaluates one set per call on one device (emcee and dynesty
call ``Objective.log_likelihood`` per point,
fitting/fitters/emcee/sampler.py:34-57, fitting/fitters/dynesty/dynesty.py:
26-39); there is no multi-device counterpart.
"""

import numpy as np


def shard_sets(nsets, rank, world):
    """Contiguous [lo, hi) share of nsets parameter sets for one rank."""
    base, extra = divmod(int(nsets), int(world))
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def slice_sets(params, nsets, lo, hi):
    """The per-set entries (leading dimension nsets) of a parameter dict cut
    to sets [lo, hi); shared entries pass through."""
    out = {}
    for k, v in params.items():
        a = np.asarray(v)
        out[k] = a[lo:hi] if a.ndim and a.shape[0] == nsets else v
    return out


class ShardedEvaluator:
    """evaluator: this rank's evaluator, with ``evaluate(params, nsets)``
    returning chi^2 per set (host array) and ``max_sets`` (a BatchedSMDisk);
    group: a torch.distributed process group (None: the default group, or a
    single process when torch.distributed is not initialised).

    ``evaluate(params, nsets)`` takes the full batch on every rank and returns
    the chi^2 of all nsets sets on every rank.  ``max_sets`` is the batch the
    ranks take together in one call."""

    def __init__(self, evaluator, group=None):
        import torch.distributed as dist
        self.evaluator = evaluator
        self.group = group
        self.distributed = dist.is_available() and dist.is_initialized()
        if self.distributed:
            self.rank = dist.get_rank(group)
            self.world = dist.get_world_size(group)
            self.backend = dist.get_backend(group)
        else:
            self.rank, self.world, self.backend = 0, 1, None
        self.max_sets = int(evaluator.max_sets) * self.world
        self.last_gather_bytes = 0

    def share(self, nsets):
        """This rank's [lo, hi) of a batch of nsets sets."""
        return shard_sets(nsets, self.rank, self.world)

    def _local(self, params, nsets):
        lo, hi = self.share(nsets)
        sub = slice_sets(params, nsets, lo, hi)
        n = hi - lo
        out = np.empty(n, np.float64)
        step = int(self.evaluator.max_sets)
        for a in range(0, n, step):
            b = min(n, a + step)
            out[a:b] = self.evaluator.evaluate(slice_sets(sub, n, a, b), b - a)
        return out

    def evaluate(self, params, nsets):
        if int(nsets) != nsets or nsets < 0:
            raise ValueError(f"a batch of {nsets!r} sets")
        nsets = int(nsets)
        mine = self._local(params, nsets)
        if self.world == 1:
            return mine
        import torch
        import torch.distributed as dist
        width = -(-nsets // self.world)
        dev = torch.device('cuda', torch.cuda.current_device()) if self.backend == 'nccl' \
            else torch.device('cpu')
        buf = torch.zeros(width, dtype=torch.float64, device=dev)
        buf[:len(mine)] = torch.from_numpy(mine).to(dev)
        parts = [torch.empty_like(buf) for _ in range(self.world)]
        dist.all_gather(parts, buf, group=self.group)
        self.last_gather_bytes = width * 8 * self.world
        out = np.empty(nsets, np.float64)
        for r, part in enumerate(parts):
            lo, hi = shard_sets(nsets, r, self.world)
            out[lo:hi] = part[:hi - lo].cpu().numpy()
        return out


def broadcast_theta(theta, src=0, group=None, ndim=None):
    """Parameter rows (n, ndim) held by rank src, on every rank (the other
    ranks pass None and the row width ndim).  Two small broadcasts (the row
    count, then the rows) on the group's device."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return np.atleast_2d(np.asarray(theta, np.float64))
    dev = torch.device('cuda', torch.cuda.current_device()) \
        if dist.get_backend(group) == 'nccl' else torch.device('cpu')
    rank = dist.get_rank(group)
    if rank == src:
        theta = np.atleast_2d(np.asarray(theta, np.float64))
        shape = torch.tensor(theta.shape, dtype=torch.int64, device=dev)
    else:
        shape = torch.zeros(2, dtype=torch.int64, device=dev)
    dist.broadcast(shape, src, group=group)
    n, d = (int(v) for v in shape.tolist())
    if ndim is not None and d != ndim:
        raise ValueError(f"broadcast rows have width {d}, expected {ndim}")
    buf = torch.from_numpy(theta).to(dev) if rank == src else \
        torch.zeros((n, d), dtype=torch.float64, device=dev)
    dist.broadcast(buf, src, group=group)
    return buf.cpu().numpy()
