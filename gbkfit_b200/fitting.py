"""Sampler-side batched objective: the log-probability of an ensemble sampler
and the likelihood of a nested sampler, evaluated as whole batches on the GPU.

The reference evaluates one parameter set per call from its samplers:

* emcee: ``log_probability(eparams, parameters, objective)``
  (fitting/fitters/emcee/sampler.py:34-57) returns
  ``(log_like + log_prior, log_like, log_prior)``, with ``-inf`` and NaN blobs
  when the prior is zero, ``log_like = sum(objective.log_likelihood(params))``
  and ``log_likelihood = -chi^2 / 2`` (objective/objective.py);
  ``EnsembleSampler(nwalkers, ndim, log_prob_fn, ..., blobs_dtype=[('log_like',
  float), ('log_prior', float)])`` (sampler.py:195-213).
* dynesty: ``_prior_transform_wrapper(theta, parameters)`` rescales the unit
  cube through the priors and ``_log_likelihood_wrapper(theta, parameters,
  objective)`` returns the log-likelihood of one point
  (fitting/fitters/dynesty/dynesty.py:26-39).

Here the same quantities come from ``gbkfit_b200.batched.BatchedSMDisk``: all
walkers of an ensemble step (emcee's ``vectorize=True`` contract: a 2-D array
of positions in, a 1-D array of log-probabilities and the blobs out), or all
points that dynesty queues for its pool (``BatchPool.map``), are one batched
evaluation.  Points outside the prior are not evaluated.
"""

import numpy as np

BLOBS_DTYPE = [('log_like', float), ('log_prior', float)]


class PriorUniform:
    """Uniform prior on [minimum, maximum] (fitting/prior: log_prob, rescale,
    sample)."""

    def __init__(self, minimum, maximum):
        if not maximum > minimum:
            raise ValueError("a uniform prior needs maximum > minimum")
        self.minimum, self.maximum = float(minimum), float(maximum)

    def log_prob(self, x):
        x = np.asarray(x, np.float64)
        inside = (x >= self.minimum) & (x <= self.maximum)
        return np.where(inside, -np.log(self.maximum - self.minimum), -np.inf)

    def rescale(self, u):
        return self.minimum + np.asarray(u, np.float64) * (self.maximum - self.minimum)

    def sample(self, n, rng=None):
        rng = np.random.default_rng() if rng is None else rng
        return rng.uniform(self.minimum, self.maximum, n)


class FreeParams:
    """The sampled parameters of one disk.

    template: the disk's parameter dict (scalars and node arrays), giving the
    values of every parameter that is not sampled; priors: {exploded name:
    prior} for the sampled ones, exploded names being ``'incl'`` for scalars
    and ``'vpt_vt[3]'`` for node ``3`` of an array (the reference's exploded
    naming, params/utils)."""

    def __init__(self, template, priors):
        self.template = {k: np.array(v, np.float64) for k, v in template.items()}
        self.names = list(priors)
        self.priors = [priors[n] for n in self.names]
        self._slots = []
        for n in self.names:
            key, idx = _split(n)
            if key not in self.template:
                raise KeyError(f"unknown parameter {key!r}")
            shape = self.template[key].shape
            if (idx is None) != (shape == ()):
                raise KeyError(f"parameter {n!r} does not match the shape {shape} of {key!r}")
            if idx is not None and not 0 <= idx < shape[0]:
                raise KeyError(f"node index of {n!r} out of range")
            self._slots.append((key, idx))

    @property
    def ndim(self):
        return len(self.names)

    def log_prior(self, theta):
        """Sum of the priors' log-densities per row of theta (n, ndim)."""
        theta = np.atleast_2d(np.asarray(theta, np.float64))
        lp = np.zeros(theta.shape[0])
        for j, p in enumerate(self.priors):
            lp = lp + p.log_prob(theta[:, j])
        return lp

    def rescale(self, u):
        """Unit cube -> parameter space (dynesty's prior transform), for one
        point (ndim,) or rows (n, ndim)."""
        u = np.asarray(u, np.float64)
        out = np.empty_like(u)
        for j, p in enumerate(self.priors):
            out[..., j] = p.rescale(u[..., j])
        return out

    def sample(self, n, rng=None):
        """n starting points drawn from the priors (n, ndim)."""
        rng = np.random.default_rng() if rng is None else rng
        return np.stack([p.sample(n, rng) for p in self.priors], axis=1)

    def batch(self, theta):
        """Rows of theta (n, ndim) -> the per-set parameter dict that
        BatchedSMDisk.evaluate takes (leading dimension n)."""
        theta = np.atleast_2d(np.asarray(theta, np.float64))
        n = theta.shape[0]
        out = {k: np.broadcast_to(v, (n,) + v.shape).copy() for k, v in self.template.items()}
        for j, (key, idx) in enumerate(self._slots):
            if idx is None:
                out[key][:] = theta[:, j]
            else:
                out[key][:, idx] = theta[:, j]
        return out


def _split(name):
    if name.endswith(']') and '[' in name:
        key, idx = name[:-1].split('[', 1)
        return key, int(idx)
    return name, None


class BatchedLogProbability:
    """emcee's log_prob_fn with ``vectorize=True`` and
    ``blobs_dtype=BLOBS_DTYPE``.

    evaluator: a BatchedSMDisk (its ``evaluate(params, nsets)`` returns chi^2
    per set; batches larger than its ``max_sets`` are split); params:
    FreeParams.  ``__call__(theta)`` with theta (nwalkers, ndim) returns
    ``(log_post, blobs)``: log_post = log_like + log_prior, and ``-inf`` with
    NaN blobs where the prior is zero (sampler.py:47-50)."""

    def __init__(self, evaluator, params):
        self.evaluator, self.params = evaluator, params
        self.evaluations = 0

    def log_likelihood(self, theta):
        """-chi^2 / 2 of every row of theta (n, ndim), in batches."""
        theta = np.atleast_2d(np.asarray(theta, np.float64))
        n = theta.shape[0]
        out = np.empty(n)
        step = int(self.evaluator.max_sets)
        for lo in range(0, n, step):
            hi = min(n, lo + step)
            chi2 = self.evaluator.evaluate(self.params.batch(theta[lo:hi]), hi - lo)
            out[lo:hi] = -0.5 * np.asarray(chi2, np.float64)
        self.evaluations += n
        return out

    def __call__(self, theta):
        theta = np.atleast_2d(np.asarray(theta, np.float64))
        lp = self.params.log_prior(theta)
        ok = np.isfinite(lp)
        ll = np.full(theta.shape[0], np.nan)
        if ok.any():
            ll[ok] = self.log_likelihood(theta[ok])
        post = np.where(ok, ll + lp, -np.inf)
        blobs = np.empty(theta.shape[0], dtype=BLOBS_DTYPE)
        blobs['log_like'] = np.where(ok, ll, np.nan)
        blobs['log_prior'] = np.where(ok, lp, np.nan)
        return post, blobs


class DynestyLikelihood:
    """dynesty's ``loglikelihood`` and ``prior_transform`` (dynesty.py:26-39)
    for one point, plus ``batch`` for many; use with BatchPool so that the
    points dynesty queues are evaluated as one batch."""

    def __init__(self, evaluator, params):
        self._lp = BatchedLogProbability(evaluator, params)
        self.params = params

    def __call__(self, theta):
        return float(self._lp.log_likelihood(np.asarray(theta)[None])[0])

    def batch(self, thetas):
        return self._lp.log_likelihood(thetas)

    def prior_transform(self, u):
        return self.params.rescale(u)


class BatchPool:
    """A pool for dynesty (``pool=BatchPool(size)``; dynesty queues ``size``
    points when no ``queue_size`` is given): ``map`` of a batched likelihood
    (a DynestyLikelihood, or a wrapper that holds one in ``.func``, as dynesty
    wraps its callables) is one batched evaluation; anything else is mapped
    point by point."""

    def __init__(self, size=512):
        self.size = int(size)

    def map(self, fn, iterable):
        pts = list(iterable)
        target = getattr(fn, 'func', fn)
        if isinstance(target, DynestyLikelihood) and pts:
            return list(target.batch(np.stack([np.asarray(p, np.float64) for p in pts])))
        return [fn(p) for p in pts]

    def close(self):
        pass

    def join(self):
        pass
