"""The device-side row assembly's tables (gbkfit_b200.batched.node_row_tables)
applied on the host reproduce Disk.pack_batch's rows, the layout the batched
evaluator reads."""

import numpy as np
import pytest

from gbkfit_b200 import traits as T
from gbkfit_b200 import workloads
from gbkfit_b200.batched import node_row_tables, row_plan
from gbkfit_b200.disk import Disk, KINDS


def _rows_from_tables(tb, params, n):
    raw = np.empty((n, tb['nraw']))
    for pname, (ro, nin) in tb['raw'].items():
        raw[:, ro:ro + nin] = np.asarray(params[pname], np.float64).reshape(n, nin)
    flat = np.full(n * tb['total'], np.nan, np.float32)
    b = np.arange(n)[:, None]
    v = tb['w0'] * raw[:, tb['k0']] + tb['w1'] * raw[:, tb['k1']]
    flat[tb['base'][None, :] + b * tb['stride'][None, :]] = v.astype(np.float32)
    return {name: flat[n * s0:n * (s0 + w)].reshape(n, w) for name, s0, w in tb['blocks']}


def _pack_rows(disk, params, n):
    p = disk.pack_batch(params, n)
    out = {}
    for name in ('vsys', 'xpos', 'ypos', 'posa', 'incl'):
        if p[name] is not None:
            out[name] = np.asarray(p[name], np.float32).reshape(n, -1)
    for kind in KINDS:
        if p[kind] is not None and p[kind]['pvalues'].size:
            out[kind] = np.asarray(p[kind]['pvalues'], np.float32).reshape(n, -1)
    return out


@pytest.mark.parametrize('nodewise', [True, False])
def test_node_row_tables_match_pack_batch(nodewise):
    n = 7
    w = workloads.smdisk_batch128(nsets=n, size=(32, 30, 24), nnodes=16)
    disk, params = w.disk, w.params
    if not nodewise:
        disk = Disk(False, False, disk.rnodes, traits=dict(
            rpt=[T.bpt('nw_uniform')], vpt=[T.vpt('nw_tan_uniform')], dpt=[T.dpt('nw_uniform')],
            spt=[T.spt('azrange')]))
        params = dict(params, spt_p=np.full(n, 30.0), spt_s=np.full(n, 300.0))
    # a buffer of n + 3 rows per name (the evaluator's capacity), the batch
    # in its first n rows
    tb = node_row_tables(disk, n + 3)
    assert tb is not None
    full = {k: (np.concatenate([np.asarray(v), np.asarray(v)[:3]]) if np.ndim(v) and
                np.shape(v)[0] == n else v) for k, v in params.items()}
    got = _rows_from_tables(tb, full, n + 3)
    want = _pack_rows(disk, params, n)
    assert set(got) == set(want) == {name for name, _, _ in row_plan(disk)}
    for name in want:
        np.testing.assert_allclose(got[name][:n], want[name], rtol=2e-7, atol=0, err_msg=name)


def test_node_row_tables_only_linear():
    w = workloads.smdisk_batch128(nsets=2, size=(32, 30, 24), nnodes=16)
    d = w.disk
    d2 = Disk(False, False, d.rnodes, interp='akima', traits=d.traits)
    assert node_row_tables(d2, 2) is None
