"""Sampler-side batched objective (gbkfit_b200.fitting) on the CPU, with a
stand-in evaluator: the emcee vectorised log-probability contract
(fitting/fitters/emcee/sampler.py:34-57), dynesty's prior transform and the
batching pool (fitting/fitters/dynesty/dynesty.py:26-39)."""

import numpy as np
import pytest

from gbkfit_b200.fitting import (BLOBS_DTYPE, BatchPool, BatchedLogProbability,
                                 DynestyLikelihood, FreeParams, PriorUniform)


class _Evaluator:
    """chi^2 = sum over a few parameters of ((value - centre) / 0.1)^2; records
    the batch sizes it was called with."""
    max_sets = 4

    def __init__(self):
        self.calls = []

    def evaluate(self, params, nsets):
        self.calls.append(nsets)
        for v in params.values():
            assert np.shape(v)[0] == nsets
        return (((params['incl'] - 50.0) / 0.1) ** 2 + ((params['vpt_vt'][:, 2] - 120.0) / 0.1) ** 2
                + ((params['xpos'] - 32.0) / 0.1) ** 2)


def _params():
    template = dict(vsys=0.0, xpos=32.0, ypos=32.0, posa=10.0, incl=45.0,
                    vpt_vt=np.linspace(0, 200, 5), bpt_a=np.ones(5))
    priors = {'incl': PriorUniform(20, 80), 'vpt_vt[2]': PriorUniform(0, 300),
              'xpos': PriorUniform(30, 34)}
    return FreeParams(template, priors)


def test_free_params_batch_and_priors():
    fp = _params()
    assert fp.ndim == 3 and fp.names == ['incl', 'vpt_vt[2]', 'xpos']
    theta = np.array([[50.0, 120.0, 31.0], [60.0, 10.0, 33.0]])
    b = fp.batch(theta)
    assert b['incl'].tolist() == [50.0, 60.0] and b['xpos'].tolist() == [31.0, 33.0]
    assert b['vpt_vt'].shape == (2, 5) and b['vpt_vt'][:, 2].tolist() == [120.0, 10.0]
    assert b['vpt_vt'][0, 1] == 50.0 and b['posa'].tolist() == [10.0, 10.0]
    lp = fp.log_prior(theta)
    assert np.allclose(lp, -np.log(60.0) - np.log(300.0) - np.log(4.0))
    assert fp.log_prior([[10.0, 120.0, 31.0]])[0] == -np.inf
    u = np.array([0.0, 0.5, 1.0])
    assert np.allclose(fp.rescale(u), [20.0, 150.0, 34.0])
    s = fp.sample(100, np.random.default_rng(1))
    assert s.shape == (100, 3) and np.all(np.isfinite(fp.log_prior(s)))
    with pytest.raises(KeyError):
        FreeParams(dict(incl=1.0), {'vpt_vt[0]': PriorUniform(0, 1)})
    with pytest.raises(KeyError):
        FreeParams(dict(vpt_vt=np.zeros(3)), {'vpt_vt[3]': PriorUniform(0, 1)})
    with pytest.raises(KeyError):
        FreeParams(dict(vpt_vt=np.zeros(3)), {'vpt_vt': PriorUniform(0, 1)})


def test_vectorised_log_probability_contract():
    fp = _params()
    ev = _Evaluator()
    lpf = BatchedLogProbability(ev, fp)
    rng = np.random.default_rng(2)
    theta = fp.sample(11, rng)
    theta[3, 0] = 90.0            # outside the incl prior
    theta[7, 2] = 29.0            # outside the xpos prior
    post, blobs = lpf(theta)
    assert post.shape == (11,) and blobs.shape == (11,) and blobs.dtype == np.dtype(BLOBS_DTYPE)
    bad = np.zeros(11, bool)
    bad[[3, 7]] = True
    assert np.all(post[bad] == -np.inf)
    assert np.all(np.isnan(blobs['log_like'][bad])) and np.all(np.isnan(blobs['log_prior'][bad]))
    # only the 9 points inside the prior were evaluated, in batches of <= max_sets
    assert sum(ev.calls) == 9 and max(ev.calls) <= 4
    good = theta[~bad]
    chi2 = ((good[:, 0] - 50) / 0.1) ** 2 + ((good[:, 1] - 120) / 0.1) ** 2 + \
        ((good[:, 2] - 32) / 0.1) ** 2
    assert np.allclose(blobs['log_like'][~bad], -0.5 * chi2)
    assert np.allclose(post[~bad], -0.5 * chi2 + fp.log_prior(good))


def test_dynesty_likelihood_and_batch_pool():
    fp = _params()
    ev = _Evaluator()
    like = DynestyLikelihood(ev, fp)
    x = fp.rescale(np.array([0.5, 0.4, 0.5]))
    assert like(x) == pytest.approx(-0.5 * (((x[0] - 50) / 0.1) ** 2 + ((x[1] - 120) / 0.1) ** 2))
    assert ev.calls == [1]

    class Wrapped:                # dynesty wraps its callables and keeps them in .func
        def __init__(self, f):
            self.func = f

        def __call__(self, v):
            return self.func(v)

    pts = [fp.rescale(u) for u in np.random.default_rng(3).uniform(size=(7, 3))]
    ev.calls.clear()
    got = BatchPool().map(Wrapped(like), pts)
    assert ev.calls == [4, 3]      # one batched evaluation, split at max_sets
    assert np.allclose(got, [like(p) for p in pts])
    # anything else is mapped point by point
    assert BatchPool().map(lambda v: 2 * v, [1, 2]) == [2, 4]
