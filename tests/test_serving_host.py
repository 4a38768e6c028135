"""Host side of the serving loop on the CPU: a request's parameter blob and
its native argument block (gbkb200_serve_args) carry every packed array of
the disk at the recorded offsets."""

import collections

import numpy as np

from gbkfit_b200.disk import KINDS


class _Dataset:
    """What Request.serve_args reads of a registered dataset (no device
    buffers: their pointers stay null here)."""

    def __init__(self, geom):
        self.geom = geom
        self.size_hi = tuple(geom.size_hi)
        self.spectrum = self.obs = self.err = None
        self.args_cache = {}


def _stream():
    from gbkfit_b200 import workloads
    return workloads.serving_stream(nrequests=8, ndatasets=3, rate=1e4, seed=5, max_side=64,
                                    max_channels=32, max_clouds=2e5, nrings=8)


def _check_array(req, name, want):
    off, n = req.layout[name]
    if want is None:
        assert off is None and n == 0, name
        return
    want = np.ascontiguousarray(want)
    if want.dtype == np.float64:
        want = want.astype(np.float32)
    assert off % 16 == 0 and n == want.size, name
    got = req.blob[off:off + want.nbytes].view(want.dtype)
    assert np.array_equal(got, want.ravel()), name


def test_request_blob_and_argument_block():
    """Every array of the blob and every field of the argument block, for
    first requests of a disk (laid out in full) and later ones (written into
    the disk's cached blob and argument templates)."""
    from gbkfit_b200.serving import Request
    st = _stream()
    kinds = set()
    seen = collections.Counter((q['dataset'], q['kind']) for q in st.requests)
    assert max(seen.values()) > 1       # some requests take the cached path
    dsets = {}
    for q in st.requests:
        d = st.datasets[q['dataset']]
        r = Request(q['dataset'], q['kind'], d[q['kind']], q['params'], cflux=q['cflux'],
                    thick=q['thick'])
        r.prepare()
        kinds.add(r.kind)
        packed = r.disk.pack(r.params)
        for k in ('subrnodes', 'vsys', 'xpos', 'ypos', 'posa', 'incl'):
            _check_array(r, k, packed[k])
        for k in KINDS:
            for f in ('uids', 'cvalues', 'ccounts', 'pvalues', 'pcounts'):
                _check_array(r, k + '.' + f, None if packed[k] is None else packed[k][f])
        ds = dsets.setdefault(q['dataset'], _Dataset(d['geom']))
        a = r.serve_args(ds)
        assert bytes(a) == bytes(r._serve_args(ds, None))
        off = lambda name: -1 if r.layout[name][0] is None else r.layout[name][0]
        assert a.blob_bytes == r.blob.size and a.nrnodes == len(packed['subrnodes'])
        assert a.off_rnodes == off('subrnodes') and a.off_incl == off('incl')
        for i, k in enumerate(KINDS):
            assert a.ntraits[i] == r.layout[k + '.uids'][1]
            assert a.off_pvalues[i] == off(k + '.pvalues')
        assert list(a.size) == list(d['geom'].size) and list(a.edge) == list(d['geom'].edge)
        if r.kind == 'mcdisk':
            csum = r.disk.ncloudscsum(r.params, r.cflux)
            _check_array(r, 'csum', np.asarray(csum, np.int32))
            _check_array(r, 'hoi', np.asarray(r.disk.hasordint(), np.uint8))
            assert a.kind == 1 and a.nclouds == int(csum[-1]) and a.csum_len == len(csum)
        else:
            assert a.kind == 0 and a.off_csum == -1 and a.off_hasordint == -1
    assert kinds == {'smdisk', 'mcdisk'}


def test_pack_one_plan_equals_pack():
    """BatchedSMDisk.pack_one (filled from a per-disk row plan) gives the rows
    of pack() for one set, value for value, for node-wise, smooth, mixture,
    loose and tilted disks."""
    from gbkfit_b200 import traits as T
    from gbkfit_b200.batched import BatchedSMDisk
    from gbkfit_b200.disk import Disk
    from tests import trait_catalogue as C

    class _Ev:
        def __init__(self, disk):
            self.disk = disk

    disks = []
    disks.append(Disk(True, True, C.RNODES, traits=dict(
        rpt=[T.bpt('exponential'), T.bpt('mixture_gauss', nblobs=2)],
        vpt=[T.vpt('tan_arctan')], dpt=[T.dpt('nw_uniform')])))
    cases = [c for c in C.cases() if not c[3]][:12]
    items = [(d, C._params(d)) for d in [C.disk_of(c) for c in cases]]
    for d in disks:                     # loose and tilted: node-wise centre and angles
        params = C._params(d)
        params.update({k: np.full(len(C.RNODES), float(params[k]) + 0.1 * i)
                       for i, k in enumerate(('vsys', 'xpos', 'ypos', 'posa', 'incl'))})
        items.append((d, params))
    st = _stream()
    items += [(st.datasets[q['dataset']]['smdisk'], q['params']) for q in st.requests
              if q['kind'] == 'smdisk']
    for d, params in items:
        ev = _Ev(d)
        one = {k: np.asarray(v)[None] for k, v in params.items()}
        ref = {k: v[0] for k, v in BatchedSMDisk.pack(ev, one, 1).items() if v.size}
        got = BatchedSMDisk.pack_one(ev, params)
        assert sorted(got) == sorted(ref)
        for k in ref:
            assert got[k].dtype == np.float32 and np.array_equal(got[k], ref[k]), k
