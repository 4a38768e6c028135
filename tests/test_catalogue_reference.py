"""The oracle's trait catalogue against the reference's own compiled
templates (oracle/_ref): every trait uid of every kind
(tests/trait_catalogue.py), thin and thick disks, all spatial outputs.

Tolerance: normwise relative 1e-5 per output (the fp32 restatement and the
compiled reference differ by a few ulp where FMA contraction differs).  The
height traits that meet the reference's stub ggauss/moffat cdfs and its stub
moffat pdf give non-finite or zero cubes in the reference; there the oracle
must give the same pattern."""

import numpy as np
import pytest

from tests import trait_catalogue as C
from tests.helpers import rel_err

CASES = C.cases()


def _compare(a, b, name, tol=1e-5):
    for k in C.OUTS:
        x, y = np.asarray(a[k], np.float64), np.asarray(b[k], np.float64)
        fx, fy = np.isfinite(x), np.isfinite(y)
        if name in C.STUB_HEIGHTS or k in ('vdata_cmp', 'ddata_cmp'):
            assert np.array_equal(fx, fy), (name, k)
            if name in C.STUB_HEIGHTS:
                assert np.array_equal(x[fx] == 0, y[fy] == 0), (name, k)
                continue
        m = fx & fy
        assert rel_err(x[m], y[m]) <= tol, (name, k, rel_err(x[m], y[m]))


@pytest.mark.parametrize('case', CASES, ids=[c[0] for c in CASES])
def test_oracle_catalogue_vs_compiled_reference(oracle_built, case):
    from oracle.oracle import Oracle, Reference
    if not Reference.available():
        pytest.skip('oracle/_ref not built')
    name, traits, params, thick = case
    geo = C.geometry(thick)
    packed = C.disk_of(case).pack(params)
    a = C.host_outputs(geo, np.float32)
    b = C.host_outputs(geo, np.float32)
    assert Oracle('f32').smdisk_evaluate(packed, geo, a) == 0
    Reference().smdisk_evaluate(packed, geo, b)
    if name not in C.STUB_HEIGHTS:
        assert np.max(b['scube']) > 0, name
    _compare(a, b, name)
