"""Shot-noise comparison of two mcdisk evaluations of the same disk and cloud
budget drawn from different random streams (the reference's mt19937 seeded
42, host/kernels.hpp:239-242, against the counter-based Philox stream of the
oracle and the GPU).

Every cloud adds cflux / (dx dy) to one voxel of the spatial flux cube
(gmodels.hpp:562-575) and rho x the sampled line to one spectral column of
scube (gmodels.hpp:92-116 via :600-614), so:

* voxel cloud counts are Poisson: sum (a - b)^2 / sum (a + b) ~ 1.  The
  budget fixes each sub-ring's cloud count (_mcdisk.py:69-110), a stratified
  draw whose bins vary a little less than Poisson, most visibly for coarse
  bins that hold a large share of an inner ring; two different distributions
  would raise the ratio instead.  So the ratio must stay below 1 + 5 sigma
  of its sampling spread (sqrt(2 / dof)) and above 0.8 (two identical
  streams would give 0);
* the counts of clouds that land inside the cube agree within 5 binomial
  sigma of the clouds outside;
* the per-spaxel spectral sum (moment 0 of scube) in units of one cloud's
  mean spectral sum is Poisson as the counts;
* per channel, the totals differ within var(T_k) <= T_k x max contribution.
"""

import numpy as np


def poisson_ratio(a, b):
    """sum (a - b)^2 / sum (a + b) over bins with a + b > 0, and the number
    of such bins."""
    m = (a + b) > 0
    return float(np.sum((a - b)[m] ** 2) / np.sum((a + b)[m])), int(m.sum())


def assert_poisson(a, b, what):
    r, dof = poisson_ratio(a, b)
    tol = 5 * np.sqrt(2.0 / dof)
    assert 0.8 <= r <= 1 + tol, (what, r, dof, tol)
    return r


def compare_clouds(a, b, nclouds, per_cloud, sigma_min, spec_step):
    """a, b: dicts with 'rdata' (spatial flux cube) and 'scube' of two
    evaluations; per_cloud = cflux / (dx dy); sigma_min: the smallest line
    width of the disk (km/s).  Returns the statistics."""
    ca = np.rint(np.asarray(a['rdata'], np.float64) / per_cloud)
    cb = np.rint(np.asarray(b['rdata'], np.float64) / per_cloud)
    # the flux cube holds whole clouds
    for x, c in ((a, ca), (b, cb)):
        assert np.max(np.abs(np.asarray(x['rdata'], np.float64) / per_cloud - c)) < 0.05
    na, nb = ca.sum(), cb.sum()
    out_a, out_b = nclouds - na, nclouds - nb
    assert abs(na - nb) <= 5 * np.sqrt(out_a + out_b + 1), (na, nb, nclouds)
    st = dict(inside=(na, nb))
    st['voxels'] = assert_poisson(ca, cb, 'voxel counts')
    st['spaxels'] = assert_poisson(ca.sum(0), cb.sum(0), 'spaxel counts')
    sa = np.asarray(a['scube'], np.float64)
    sb = np.asarray(b['scube'], np.float64)
    m0a, m0b = sa.sum(0), sb.sum(0)
    unit = m0a.sum() / na                    # one cloud's mean spectral sum
    st['moment0'] = assert_poisson(m0a / unit, m0b / unit, 'spectral sums')
    ta, tb = sa.sum((1, 2)), sb.sum((1, 2))
    xmax = per_cloud / (sigma_min * np.sqrt(2 * np.pi))       # largest line value
    m = (ta + tb) > 0
    st['channels'] = float(np.mean((ta - tb)[m] ** 2 / ((ta + tb)[m] * xmax)))
    assert st['channels'] <= 1 + 5 * np.sqrt(2.0 / m.sum()), st
    return st
