"""The fp64 reference gradient of the differentiable configuration (oracle
chi2_gradient_f64: the smdisk line model, circular PSF x LSF convolution and
chi^2 differentiated analytically in float64) against central finite
differences of the C oracle pipeline's chi^2.  CPU only.

At the specified step h = 1e-3 (relative) the finite differences carry an
O(h^2) truncation error that is largest for the centre position: a shift of
0.05 px moves the lines near the disk centre by ~1.5 km/s against a 20 km/s
dispersion, where the velocity field curves sharply.  The geometry is
therefore also checked at h = 1e-4, where the truncation error is small and
fp64 rounding still is."""

import numpy as np

from tests.helpers import (grad96_fd, grad96_groups, grad96_oracle_chi2, grad96_problem,
                           grad96_reference_gradient)


def test_reference_gradient_matches_finite_differences(oracle_built):
    w, data, err, theta = grad96_problem()
    c2, g = grad96_reference_gradient(w, theta, data, err)
    # the reference's forward model is the oracle's
    c2_oracle = grad96_oracle_chi2(w, theta, data, err)
    assert abs(c2 - c2_oracle) <= 1e-10 * c2_oracle
    fd = grad96_fd(w, theta, data, err, rel=1e-3)
    assert np.linalg.norm(g - fd) <= 1e-3 * np.linalg.norm(fd)
    for gs in grad96_groups(theta, len(w.disk.rnodes))[1:]:
        assert np.linalg.norm(g[gs] - fd[gs]) <= 1e-4 * np.linalg.norm(fd[gs]), gs
    geo = grad96_fd(w, theta, data, err, rel=1e-4, idx=range(5))
    assert np.all(np.abs(g[:5] - geo) <= 5e-4 * np.abs(geo)), (g[:5], geo)
