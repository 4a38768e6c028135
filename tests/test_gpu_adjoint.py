"""Hand-written adjoint of smdisk + PSF/LSF convolution + chi^2 on the
differentiable configuration (96x96x64 cube, 20 rings, 66 parameters): chi^2
against the fp64 oracle, the gradient against the fp64 reference gradient
(oracle.chi2_gradient_f64, itself checked against finite differences on the
CPU) and against central finite differences (h = 1e-3 relative) of the fp64
oracle's chi^2, and the torch.autograd.Function wrapper."""

import numpy as np
import pytest

from tests.helpers import (grad96_fd, grad96_groups, grad96_oracle_chi2, grad96_problem,
                           grad96_reference_gradient)

pytestmark = pytest.mark.gpu

# GPU (fp32 forward, fp64 sums) against the fp64 reference gradient
TOL_REF_ALL = 1e-5
TOL_REF_GROUP = 1e-4
# against the h = 1e-3 central differences (their own truncation error is up
# to ~3e-3 for the centre position, see tests/test_adjoint_reference.py)
TOL_FD_ALL = 1e-3


@pytest.fixture(scope='module')
def problem(oracle_built):
    from gbkfit_b200.adjoint import SMDiskChi2
    w, data, err, theta = grad96_problem()
    return w, SMDiskChi2(w.disk, w.geom, data, err), theta, data, err


def test_chi2_matches_fp64_oracle(problem):
    w, model, theta, data, err = problem
    got = model.value(theta)
    ref = grad96_oracle_chi2(w, theta, data, err)
    assert abs(got - ref) / ref < 1e-5, (got, ref)


def test_gradient_matches_fp64_reference(problem):
    w, model, theta, data, err = problem
    c2, g = model.value_and_grad(theta)
    c2r, gr = grad96_reference_gradient(w, theta, data, err)
    assert len(g) == 66 and np.all(np.isfinite(g))
    assert abs(c2 - c2r) <= 1e-5 * c2r
    assert np.linalg.norm(g - gr) <= TOL_REF_ALL * np.linalg.norm(gr)
    for gs in grad96_groups(theta, model.nnodes):
        assert np.linalg.norm(g[gs] - gr[gs]) <= TOL_REF_GROUP * np.linalg.norm(gr[gs]), gs


def test_gradient_matches_finite_differences(problem):
    w, model, theta, data, err = problem
    _, g = model.value_and_grad(theta)
    fd = grad96_fd(w, theta, data, err, rel=1e-3)
    report = '\n'.join(f'{n:12s} {a: .6e} {b: .6e}' for n, a, b in zip(model.names, g, fd))
    assert np.linalg.norm(g - fd) <= TOL_FD_ALL * np.linalg.norm(fd), report


def test_autograd_function(problem):
    import torch
    from gbkfit_b200.adjoint import SMDiskChi2Function
    w, model, theta, data, err = problem
    _, g_ref = model.value_and_grad(theta)
    for _ in range(2):
        th = torch.tensor(theta, dtype=torch.float64, requires_grad=True)
        c2 = SMDiskChi2Function.apply(th, model)
        (g,) = torch.autograd.grad(c2, th)
        assert np.linalg.norm(g.numpy() - g_ref) <= 1e-6 * np.linalg.norm(g_ref)
    # the upstream gradient scales the result
    th = torch.tensor(theta, dtype=torch.float64, requires_grad=True)
    (2.5 * SMDiskChi2Function.apply(th, model)).backward()
    assert np.linalg.norm(th.grad.numpy() - 2.5 * g_ref) <= 1e-6 * np.linalg.norm(2.5 * g_ref)
