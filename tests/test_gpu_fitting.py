"""Sampler-side batched objective on the GPU: the vectorised log-probability
of a whole ensemble equals the batched evaluator's chi^2 set by set and the
fp64 oracle's chi^2; a few steps of an affine-invariant ensemble (stretch
move, Goodman & Weare 2010, emcee's default move) run through it."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SCALES = np.array([3.0, 5.0, 10.0, 2.0])     # walker spread per free parameter


def _setup(max_sets):
    from gbkfit_b200 import workloads
    from gbkfit_b200.batched import BatchedSMDisk, synthetic_data
    from gbkfit_b200.fitting import FreeParams, PriorUniform
    w = workloads.smdisk_batch128(nsets=1, size=(64, 60, 48), nnodes=16)
    data, err, _ = synthetic_data(w)
    truth = {k: np.asarray(v, np.float64) for k, v in w.extra['truth'].items()}
    x0 = np.array([truth['incl'], truth['posa'], truth['vpt_vt'][5], truth['dpt_a'][2]])
    names = ['incl', 'posa', 'vpt_vt[5]', 'dpt_a[2]']
    fp = FreeParams(truth, {n: PriorUniform(x - 6 * s, x + 6 * s)
                            for n, x, s in zip(names, x0, SCALES)})
    ev = BatchedSMDisk(w.disk, w.geom, data, err, max_sets=max_sets, conv='direct')
    return w, data, err, x0, fp, ev


def test_ensemble_log_probability_matches_evaluator_and_oracle(gpu, oracle_built):
    from oracle.oracle import chi2, scube_pipeline
    from gbkfit_b200.fitting import BatchedLogProbability
    w, data, err, x0, fp, ev = _setup(max_sets=16)
    rng = np.random.default_rng(5)
    theta = x0 + np.clip(rng.normal(0, 1, (40, 4)), -3, 3) * SCALES
    theta[11, 0] = x0[0] + 7 * SCALES[0]                 # outside the incl prior
    lpf = BatchedLogProbability(ev, fp)
    post, blobs = lpf(theta)
    assert post[11] == -np.inf and np.isnan(blobs['log_like'][11])
    ok = np.isfinite(post)
    assert ok.sum() == 39 and lpf.evaluations == 39
    # the same sets through the evaluator directly
    direct = np.concatenate([ev.evaluate(fp.batch(theta[ok][i:i + 16]), len(theta[ok][i:i + 16]))
                             for i in range(0, 39, 16)])
    assert np.array_equal(blobs['log_like'][ok], -0.5 * direct.astype(np.float64))
    # the fp64 oracle for three of the walkers
    for i in (0, 17, 39):
        p = {k: v[0] for k, v in fp.batch(theta[i]).items()}
        c = chi2(scube_pipeline(w.disk.pack(p), w.geom, precision='f64'), data, err)
        assert abs(-2.0 * blobs['log_like'][i] - c) <= 1e-4 * c, (i, blobs['log_like'][i], c)
        assert post[i] == pytest.approx(blobs['log_like'][i] + fp.log_prior(theta[i])[0])


def test_stretch_move_ensemble_steps(gpu):
    from gbkfit_b200.fitting import BatchedLogProbability
    w, data, err, x0, fp, ev = _setup(max_sets=32)
    lpf = BatchedLogProbability(ev, fp)
    rng = np.random.default_rng(11)
    nw, nd, a = 32, fp.ndim, 2.0
    pos = x0 + np.clip(rng.normal(0, 1, (nw, nd)), -2, 2) * SCALES / 2
    lp, _ = lpf(pos)
    accepted = 0
    for _ in range(4):
        for half in (np.arange(nw // 2), np.arange(nw // 2, nw)):
            other = np.setdiff1d(np.arange(nw), half)
            z = ((a - 1) * rng.uniform(size=len(half)) + 1) ** 2 / a
            partner = pos[rng.choice(other, len(half))]
            prop = partner + z[:, None] * (pos[half] - partner)
            lnew, _ = lpf(prop)                           # one batched evaluation per half
            acc = np.log(rng.uniform(size=len(half))) < (nd - 1) * np.log(z) + lnew - lp[half]
            pos[half[acc]] = prop[acc]
            lp[half[acc]] = lnew[acc]
            accepted += int(acc.sum())
    assert np.all(np.isfinite(lp)) and accepted > 0
    assert np.all(np.isfinite(fp.log_prior(pos)))
    assert lpf.evaluations <= nw + 8 * (nw // 2)
