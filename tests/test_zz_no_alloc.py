"""The residual sum that allocates nothing
(gbkb200_objective_residual_sum_noalloc_f32), called through the C ABI.

It serves callers that cannot allocate device memory, for example a host
framework that owns all device memory through its own pool, or a loop that
must not allocate after start-up.  Its result must match the regular entry
point (gbkb200_objective_residual_sum_f32) within the tolerance of the other
reduction tests (1e-6 relative; both sum fp32 block partials in fp64, over
different block partitions), on two calls in a row: the second call reuses
the library's fixed scratch array that the first one left behind.

This file is named so that pytest collects it last.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_RESIDUALS = 8192 * 32768


def _lib():
    from gbkfit_b200 import _native
    lib = _native.lib()
    f = lib.gbkb200_objective_residual_sum_noalloc_f32
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def test_noalloc_residual_sum_matches(gpu):
    import torch
    from gbkfit_b200.driver import DriverB200
    noalloc = _lib()
    drv = DriverB200(0)
    obj = drv.backends().objective(np.float32)
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(2024)
    for n, squared in ((1_572_864, True), (3_000_017, False), (1_572_864, True)):
        res = torch.from_numpy(rng.standard_normal(n).astype(np.float32)).cuda()
        ref = torch.zeros(1, device='cuda')
        obj.residual_sum(res, squared, ref)
        for call in range(2):
            out = torch.full((1,), -1.0, device='cuda')
            rc = noalloc(res.data_ptr(), n, int(squared), out.data_ptr(), stream)
            assert rc == 0
            torch.cuda.synchronize()
            a, b = out.item(), ref.item()
            assert abs(a - b) <= 1e-6 * abs(b), (n, squared, call, a, b)


def test_noalloc_residual_sum_limits(gpu):
    import torch
    noalloc = _lib()
    stream = torch.cuda.current_stream().cuda_stream
    out = torch.full((1,), -1.0, device='cuda')
    res = torch.zeros(4, device='cuda')
    # beyond the scratch array: rejected before anything is launched
    assert noalloc(res.data_ptr(), MAX_RESIDUALS + 1, 1, out.data_ptr(), stream) == 7
    assert noalloc(res.data_ptr(), -1, 1, out.data_ptr(), stream) == 1
    # empty input sums to zero
    assert noalloc(res.data_ptr(), 0, 1, out.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    assert out.item() == 0.0
