"""Batched evaluation of many parameter sets of one thin smooth disk.

``BatchedSMDisk`` evaluates, per parameter set, smdisk -> PSF x LSF FFT
convolution -> crop -> residual -> chi^2 against one data cube, for up to
``max_sets`` sets per call (sampler walkers), through gbkb200_batch_* of
libgbkb200.so.  Per set the result equals the reference chain
``DModelSCube.evaluate`` + ``Objective.residual_scalar(squared=True)``
(dmodels/scube.py:95-122, objective/objective.py:187-206).

Inputs can be host parameter dicts (packed with ``Disk.pack_batch`` and
copied from pinned memory) or device tensors already resident in HBM.  A
fixed-size call can be captured once in a CUDA graph and replayed.
"""

import ctypes

import numpy as np
import torch

from . import _native
from ._native import c_int, c_float, c_void_p, check
from .disk import KINDS

_lib = _native.lib()


class BatchDesc(ctypes.Structure):
    """include/gbkb200.h gbkb200_batch_desc."""
    _fields_ = [
        ('size', c_int * 3), ('kernel_size', c_int * 3), ('fft_size', c_int * 3),
        ('spat_step', c_float * 2), ('spat_zero', c_float * 2),
        ('spec_step', c_float), ('spec_zero', c_float),
        ('loose', c_int), ('tilted', c_int), ('nrnodes', c_int), ('rnodes', c_void_p),
        ('ntraits', c_int * 9), ('uids', c_void_p * 9), ('cvalues', c_void_p * 9),
        ('ccounts', c_void_p * 9), ('pcounts', c_void_p * 9), ('npvalues', c_int * 9),
        ('psf', ctypes.POINTER(ctypes.c_double)), ('lsf', ctypes.POINTER(ctypes.c_double)),
        ('obs_d', c_void_p), ('obs_e', c_void_p), ('obs_m', c_void_p), ('weight', c_float),
        ('max_sets', c_int), ('chunk', c_int), ('rows_k1', c_int), ('rows_k5', c_int),
        ('conv_mode', c_int), ('psf_rank', c_int),
        ('psf_u', ctypes.POINTER(ctypes.c_double)), ('psf_v', ctypes.POINTER(ctypes.c_double)),
        ('psf_band', c_int), ('psf_variant', c_int), ('model_variant', c_int),
    ]

CONV_MODES = dict(auto=0, fft=1, direct=2)


_lib.gbkb200_batch_create.argtypes = [c_void_p, ctypes.POINTER(BatchDesc),
                                      ctypes.POINTER(c_void_p)]
_lib.gbkb200_batch_create.restype = c_int
_lib.gbkb200_batch_evaluate.argtypes = [c_void_p, c_int] + [c_void_p] * 5 + [
    c_void_p * 9, c_void_p, c_void_p]
_lib.gbkb200_batch_evaluate.restype = c_int
_lib.gbkb200_batch_info.argtypes = [c_void_p, c_int * 3, ctypes.POINTER(c_int),
                                    ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(c_int)]
_lib.gbkb200_batch_info.restype = c_int
_lib.gbkb200_batch_destroy.argtypes = [c_void_p]
_lib.gbkb200_batch_destroy.restype = c_int
_lib.gbkb200_batch_set_timing.argtypes = [c_void_p, c_int]
_lib.gbkb200_batch_set_timing.restype = c_int
_lib.gbkb200_batch_timing.argtypes = [c_void_p, ctypes.c_double * 6, c_int * 6]
_lib.gbkb200_batch_timing.restype = c_int
_lib.gbkb200_batch_counters.argtypes = [c_void_p, ctypes.c_ulonglong * 8]
_lib.gbkb200_batch_counters.restype = c_int

_lib.gbkb200_rows_from_nodes.argtypes = [c_void_p, c_int, c_int] + [c_void_p] * 6 + [
    c_int, c_void_p, c_void_p]
_lib.gbkb200_rows_from_nodes.restype = c_int

BATCH_EXPORTED = ['gbkb200_batch_create', 'gbkb200_batch_evaluate', 'gbkb200_batch_info',
                  'gbkb200_batch_destroy', 'gbkb200_batch_set_timing', 'gbkb200_batch_timing',
                  'gbkb200_batch_counters', 'gbkb200_rows_from_nodes']

# slots of gbkb200_batch_counters
COUNTERS = ('lsf_fma', 'lines', 'psf_x_fma', 'psf_y_fma', 'residual_voxels', 'spaxels')

# per-stage kernel names of gbkb200_batch_timing, by convolution mode
STAGE_KERNELS = {
    'direct': {0: 'ka_lines_lsf', 4: 'kb_psf_residual', 5: 'k6_sum'},
    'fft': {0: 'k1_model_xfft', 1: 'k_lines (y forward)', 2: 'k_lines (z convolution)',
            3: 'k_lines (y inverse)', 4: 'k5_c2r_residual', 5: 'k6_sum'},
}


from .sharded import shard_sets  # noqa: E402,F401  (the per-rank share; see sharded.py)


def kernel_boxes(geom):
    """PSF image (Ky, Kx) and LSF (Kz) on their own odd-sized boxes, with the
    reference's sampling, truncation and normalisation (psfs.py, lsfs.py)."""
    from .psflsf import LSFPoint, PSFPoint
    kx, ky, kz = geom.kernel_size
    psf = (geom.psf or PSFPoint()).asarray(geom.step[:2], (kx, ky), (0, 0))
    lsf = (geom.lsf or LSFPoint()).asarray(geom.step[2], kz, 0)
    return np.ascontiguousarray(psf, np.float64), np.ascontiguousarray(lsf, np.float64)


def separable_factors(psf, tol=1e-9, max_rank=8):
    """PSF image (Ky, Kx) = sum_r u_r[y] v_r[x], from its SVD, with the
    smallest rank whose reconstruction is within tol x max|psf|; (0, None,
    None) when no rank up to max_rank reaches it."""
    u, s, vt = np.linalg.svd(psf)
    peak = np.max(np.abs(psf))
    for r in range(1, min(max_rank, len(s)) + 1):
        uu = u[:, :r] * np.sqrt(s[:r])
        vv = vt[:r].T * np.sqrt(s[:r])
        if np.max(np.abs(psf - uu @ vv.T)) <= tol * peak:
            return r, np.ascontiguousarray(uu.T), np.ascontiguousarray(vv.T)
    return 0, None, None


class BatchedSMDisk:
    """One thin disk, one data cube, up to max_sets parameter sets per call.

    disk: gbkfit_b200.disk.Disk; geom: gbkfit_b200.workloads.Geometry;
    data/error/mask: (nz, ny, nx) arrays (host or device) or None."""

    def __init__(self, disk, geom, data, error=None, mask=None, weight=1.0, max_sets=512,
                 chunk=0, fft_size=(0, 0, 0), rows_k1=0, rows_k5=0, conv='auto', band=0, device=0,
                 stream=None, psf_variant=0, model_variant=None):
        # the direct mode's model kernel: by default the 4 x 8 tile kernel with
        # transposed range masks (3), which keeps 16 bytes per output plane in
        # shared memory (up to 2048 planes); beyond that one chunk per warp (0)
        if model_variant is None:
            model_variant = 3 if geom.size[2] * 16 <= 32 * 1024 else 0
        if disk.traits['rht']:
            raise ValueError("the batched evaluator takes thin disks only")
        self.disk = disk
        self.geom = geom
        self.max_sets = int(max_sets)
        self.dev = torch.device('cuda', device)
        self.stream = stream or torch.cuda.current_stream(self.dev)
        self.ctx = _native.Context(device=device, stream=self.stream, sync=False)
        dev = self.dev
        f32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32)).to(dev) \
            if not torch.is_tensor(a) else a.to(dev, torch.float32).contiguous()
        self._keep = []
        self.obs = f32(data)
        self.err = None if error is None else f32(error)
        self.msk = None if mask is None else f32(mask)
        self.rnodes = f32(disk.subrnodes)
        d = BatchDesc()
        d.size[:] = list(geom.size)
        d.kernel_size[:] = list(geom.kernel_size)
        d.fft_size[:] = list(fft_size)
        d.spat_step[:] = [geom.step[0], geom.step[1]]
        d.spat_zero[:] = [geom.zero_hi[0], geom.zero_hi[1]]
        d.spec_step = geom.step[2]
        d.spec_zero = geom.zero_hi[2]
        d.loose, d.tilted, d.nrnodes = int(disk.loose), int(disk.tilted), disk.nsub
        d.rnodes = self.rnodes.data_ptr()
        self.npv = []
        for k, kind in enumerate(KINDS):
            t = disk.tables[kind]
            if t is None:
                d.ntraits[k] = 0
                d.npvalues[k] = 0
                self.npv.append(0)
                continue
            arrs = [torch.as_tensor(t['uids']).to(dev),
                    torch.as_tensor(t['cvalues'] if len(t['cvalues']) else np.zeros(1, np.float32)).to(dev),
                    torch.as_tensor(t['ccounts']).to(dev), torch.as_tensor(t['pcounts']).to(dev)]
            self._keep += arrs
            d.ntraits[k] = len(t['uids'])
            d.uids[k], d.cvalues[k], d.ccounts[k], d.pcounts[k] = [a.data_ptr() for a in arrs]
            d.npvalues[k] = t['npv']
            self.npv.append(t['npv'])
        psf, lsf = kernel_boxes(geom)
        self._psf, self._lsf = psf, lsf
        d.psf = psf.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        d.lsf = lsf.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        d.obs_d = self.obs.data_ptr()
        d.obs_e = self.err.data_ptr() if self.err is not None else None
        d.obs_m = self.msk.data_ptr() if self.msk is not None else None
        d.weight = float(weight)
        d.max_sets, d.chunk, d.rows_k1, d.rows_k5 = self.max_sets, chunk, rows_k1, rows_k5
        d.conv_mode = CONV_MODES[conv]
        d.psf_band = int(band)
        d.psf_variant = int(psf_variant)
        d.model_variant = int(model_variant)
        rank, fu, fv = separable_factors(psf) if conv != 'fft' else (0, None, None)
        self._fu, self._fv = fu, fv
        d.psf_rank = rank
        if rank:
            d.psf_u = fu.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            d.psf_v = fv.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        h = c_void_p()
        check(_lib.gbkb200_batch_create(self.ctx.handle, ctypes.byref(d), ctypes.byref(h)),
              'gbkb200_batch_create')
        self.handle = h
        fs = (c_int * 3)()
        ch = c_int()
        wb = ctypes.c_size_t()
        cm = c_int()
        check(_lib.gbkb200_batch_info(h, fs, ctypes.byref(ch), ctypes.byref(wb),
                                      ctypes.byref(cm)), 'batch_info')
        self.fft_size, self.chunk, self.work_bytes = tuple(fs), ch.value, wb.value
        self.conv_mode = {1: 'fft', 2: 'direct'}[cm.value]
        self.psf_rank = rank
        self.chi2 = torch.zeros(self.max_sets, device=dev)
        self._graph = None
        self._inputs = None

    # ---- inputs -------------------------------------------------------------
    def pack(self, params, nsets):
        """Host parameter dict (per-set leading axis) -> dict of pinned host arrays."""
        p = self.disk.pack_batch(params, nsets)
        out = {}
        for name in ('vsys', 'xpos', 'ypos', 'posa', 'incl'):
            if p[name] is not None:
                out[name] = np.ascontiguousarray(p[name], np.float32).reshape(nsets, -1)
        for kind in KINDS:
            if p[kind] is not None:
                out[kind] = np.ascontiguousarray(p[kind]['pvalues'], np.float32).reshape(nsets, -1)
        return out

    def alloc_inputs(self, nsets=None):
        """Device input buffers (resident) for nsets sets."""
        n = self.max_sets if nsets is None else nsets
        d = self.disk
        bufs = {}
        for name in ('vsys', 'xpos', 'ypos', 'posa', 'incl'):
            if name in d.pdescs:
                bufs[name] = torch.zeros((n, d.common_size(name)), device=self.dev)
        for k, kind in enumerate(KINDS):
            if self.npv[k]:
                bufs[kind] = torch.zeros((n, self.npv[k]), device=self.dev)
        return bufs

    def upload(self, packed, bufs, nsets):
        for k, v in packed.items():
            if v.size:      # kinds without parameters have no buffer
                bufs[k][:nsets].copy_(torch.from_numpy(v), non_blocking=True)

    # ---- evaluation ---------------------------------------------------------
    def evaluate_device(self, bufs, nsets, chi2=None, model=None):
        """chi^2 of nsets resident parameter sets (enqueued, not synchronised)."""
        chi2 = self.chi2 if chi2 is None else chi2
        g = lambda n: bufs[n].data_ptr() if n in bufs else None
        pv = (c_void_p * 9)(*[bufs[k].data_ptr() if k in bufs else None for k in KINDS])
        check(_lib.gbkb200_batch_evaluate(self.handle, int(nsets), g('vsys'), g('xpos'),
                                          g('ypos'), g('posa'), g('incl'), pv, chi2.data_ptr(),
                                          model.data_ptr() if model is not None else None),
              'gbkb200_batch_evaluate')
        return chi2[:nsets]

    def evaluate(self, params, nsets, pieces=None):
        """Host parameters -> host chi^2 (numpy), end to end.

        With linear node interpolation (and pieces not given) the raw
        parameter values of all sets are copied to the device in one transfer
        and the input rows are built there (gbkb200_rows_from_nodes), so the
        whole batch is evaluated as one piece.  Otherwise the batch is split
        into pieces; each piece is packed into its own
        pinned host buffer, copied to the device in one transfer and
        evaluated asynchronously while the next piece is packed; chi^2 comes
        back through a pinned buffer and the call synchronises once.
        pieces: how many equal pieces, or the sizes of the pieces (default:
        for 256 sets or more a first piece of an eighth of the sets, at least
        32, then the rest: the device starts early and the large second
        piece's packing overlaps the first's evaluation; else one piece); a
        piece smaller than the chunk is evaluated as a smaller wave."""
        nsets = int(nsets)
        if nsets > self.max_sets:
            raise ValueError(f"nsets {nsets} > max_sets {self.max_sets}")
        nd = self._node_rows() if pieces is None else None
        if nd is not None and not all(np.ndim(params[p]) >= 1 and np.shape(params[p])[0] == nsets
                                      for p in nd['raw']):
            nd = None
        if pieces is None:
            if nsets >= 256:
                first = max(32, nsets // 8 // 32 * 32)
                pieces = (first, nsets - first)
            else:
                pieces = 1
        if np.ndim(pieces) == 0:
            piece = max(1, -(-nsets // int(pieces)))
            piece = min(self.max_sets, -(-piece // 32) * 32)
            sizes = [min(piece, nsets - lo) for lo in range(0, nsets, piece)] or [0]
        else:
            sizes = [int(s) for s in pieces]
            if sum(sizes) != nsets or min(sizes) < 1:
                raise ValueError(f"piece sizes {sizes} do not make {nsets} sets")
        if nd is not None:
            return self._evaluate_nodes(nd, params, nsets)
        bounds = np.concatenate([[0], np.cumsum(sizes)]).astype(int)
        st = self._e2e_buffers(max(sizes), len(sizes))
        per_set = {k: (np.ndim(v) > 0 and np.shape(v)[0] == nsets) for k, v in params.items()}
        self.last_h2d_bytes = 0
        with torch.cuda.stream(self.stream):
            for j in range(len(sizes)):
                lo, hi = int(bounds[j]), int(bounds[j + 1])
                if hi <= lo:
                    continue
                sub = {k: (v[lo:hi] if per_set[k] else v) for k, v in params.items()}
                hv, hflat, dflat, dv = st['pieces'][j]
                for name, arr in self.pack(sub, hi - lo).items():
                    if arr.size:
                        hv[name][:hi - lo] = arr
                dflat.copy_(hflat, non_blocking=True)
                self.last_h2d_bytes += hflat.numel() * 4
                self.evaluate_device(dv, hi - lo, chi2=self.chi2[lo:hi])
            out = st['chi2'][:nsets]
            out.copy_(self.chi2[:nsets], non_blocking=True)
        self.stream.synchronize()
        return out.numpy().copy()

    def _node_rows(self):
        """Tables (node_row_tables) and buffers of the device-side row
        assembly, built once; None unless the disk interpolates linearly."""
        if hasattr(self, '_nodes'):
            return self._nodes
        self._nodes = None
        n = self.max_sets
        tb = node_row_tables(self.disk, n)
        if tb is None:
            return None
        k0, k1, w0, w1, base, stride = (tb[k] for k in ('k0', 'k1', 'w0', 'w1', 'base', 'stride'))
        raw, nraw, blocks, start = tb['raw'], tb['nraw'], tb['blocks'], tb['total']
        dev = self.dev
        dflat = torch.empty(max(1, n * start), dtype=torch.float32, device=dev)
        dv = {name: dflat[n * s0:n * (s0 + w)].view(n, w) for name, s0, w in blocks}
        hraw = torch.empty((n, nraw), dtype=torch.float64, pin_memory=True)
        t = {k: torch.from_numpy(v) for k, v in
             dict(k0=k0, k1=k1, w0=w0, w1=w1, base=base, stride=stride).items()}
        self._nodes = dict(raw=raw, nraw=nraw, width=len(k0), hraw=hraw, hraw_np=hraw.numpy(),
                           draw=torch.empty((n, nraw), dtype=torch.float64, device=dev),
                           tables={k: v.to(dev) for k, v in t.items()}, host_tables=t,
                           dflat=dflat, dv=dv,
                           chi2=torch.empty(n, dtype=torch.float32, pin_memory=True))
        return self._nodes

    def _evaluate_nodes(self, nd, params, nsets):
        """evaluate() through the device-side row assembly (one piece)."""
        hr = nd['hraw_np'][:nsets]
        for pname, (ro, nin) in nd['raw'].items():
            hr[:, ro:ro + nin] = np.asarray(params[pname], np.float64).reshape(nsets, nin)
        t = nd['tables']
        with torch.cuda.stream(self.stream):
            nd['draw'][:nsets].copy_(nd['hraw'][:nsets], non_blocking=True)
            self.last_h2d_bytes = nsets * nd['nraw'] * 8
            check(_lib.gbkb200_rows_from_nodes(
                nd['draw'].data_ptr(), nd['nraw'], nsets, t['k0'].data_ptr(),
                t['k1'].data_ptr(), t['w0'].data_ptr(), t['w1'].data_ptr(),
                t['base'].data_ptr(), t['stride'].data_ptr(), nd['width'],
                nd['dflat'].data_ptr(), c_void_p(self.stream.cuda_stream)),
                'gbkb200_rows_from_nodes')
            self.evaluate_device(nd['dv'], nsets)
            out = nd['chi2'][:nsets]
            out.copy_(self.chi2[:nsets], non_blocking=True)
        self.stream.synchronize()
        return out.numpy().copy()

    def _e2e_buffers(self, piece, npieces):
        """Pinned host and device input buffers of npieces pieces of piece sets."""
        st = getattr(self, '_e2e', None)
        if st is not None and st['piece'] == piece and len(st['pieces']) >= npieces:
            return st
        names = [n for n in ('vsys', 'xpos', 'ypos', 'posa', 'incl') if n in self.disk.pdescs]
        widths = [(n, self.disk.common_size(n)) for n in names]
        widths += [(kind, self.npv[k]) for k, kind in enumerate(KINDS) if self.npv[k]]
        total = piece * sum(w for _, w in widths)
        pieces = []
        for _ in range(npieces):
            hflat = torch.empty(total, dtype=torch.float32, pin_memory=True)
            dflat = torch.empty(total, dtype=torch.float32, device=self.dev)
            hv, dv, off = {}, {}, 0
            for name, w in widths:
                hv[name] = hflat[off:off + piece * w].view(piece, w).numpy()
                dv[name] = dflat[off:off + piece * w].view(piece, w)
                off += piece * w
            pieces.append((hv, hflat, dflat, dv))
        st = dict(piece=piece, pieces=pieces,
                  chi2=torch.empty(self.max_sets, dtype=torch.float32, pin_memory=True))
        self._e2e = st
        return st

    # ---- asynchronous groups (serving) ----------------------------------------
    def pack_one(self, params):
        """One parameter set (host dict) -> {name: float32 row} in the layout
        of the evaluator's inputs: the values pack() gives for one set, filled
        from a per-disk plan of the rows (the serving loop packs every
        request with it)."""
        plan = getattr(self, '_row_plan', None)
        if plan is None:
            plan = self._row_plan = row_plan(self.disk)
        out = {}
        for name, entries, width in plan:
            row = np.empty(width, np.float32)
            off = 0
            for pname, size, nw, interp in entries:
                v = params[pname]
                if nw:
                    vals = interp(np.asarray(v, np.float64)[None])[0]
                    n = vals.shape[0]
                else:
                    vals, n = np.asarray(v, np.float64).reshape(size), size
                row[off:off + n] = vals
                off += n
            out[name] = row
        return out

    def _submit_args(self):
        """The per-evaluator arguments of gbkb200_batch_submit (built once):
        the pinned and device input buffers of max_sets sets and the
        pointers of their per-name views."""
        a = getattr(self, '_sub', None)
        if a is not None:
            return a
        st = self._e2e_buffers(self.max_sets, 1)
        hv, hflat, dflat, dv = st['pieces'][0]
        g = lambda n: c_void_p(dv[n].data_ptr()) if n in dv else None
        pv = (c_void_p * 9)(*[dv[k].data_ptr() if k in dv else None for k in KINDS])
        self._sub = a = dict(hv=hv, out=st['chi2'], pv=pv, args=(
            c_void_p(hflat.data_ptr()), c_void_p(dflat.data_ptr()),
            ctypes.c_size_t(hflat.numel() * 4), g('vsys'), g('xpos'), g('ypos'), g('posa'),
            g('incl'), pv, c_void_p(self.chi2.data_ptr()), c_void_p(st['chi2'].data_ptr())))
        return a

    def submit_rows(self, rows):
        """Enqueue one evaluation of len(rows) parameter sets (rows from
        pack_one) on the evaluator's stream in one native call: the rows are
        gathered into a pinned buffer, copied to the device in one transfer,
        evaluated, and chi^2 is copied back to pinned memory.  Returns (done,
        chi2 host tensor view): chi2 is valid once done.query() is true.  One
        submission may be in flight per evaluator (the next one reuses its
        buffers): the caller waits for it before submitting again."""
        n = len(rows)
        if not 0 < n <= self.max_sets:
            raise ValueError(f"a group of {n} sets (max_sets {self.max_sets})")
        a = self._submit_args()
        for name, arr in a['hv'].items():
            if n == 1:
                arr[0] = rows[0][name]
            else:
                arr[:n] = np.stack([r[name] for r in rows])
        check(_lib.gbkb200_batch_submit(self.handle, c_int(n), *a['args']), 'batch_submit')
        return self._done, a['out'][:n]

    def submit_cubes(self, cubes, n):
        """As submit_rows, for n model cubes already enqueued into `cubes` on
        the evaluator's stream: the convolution, residual and sum, and chi^2
        copied back to pinned memory.  Returns (done, chi2 host view)."""
        if not 0 < n <= self.max_sets:
            raise ValueError(f"a group of {n} sets (max_sets {self.max_sets})")
        a = self._submit_args()
        check(_lib.gbkb200_batch_submit_cubes(self.handle, c_int(n), c_void_p(cubes.data_ptr()),
                                              a['args'][9], a['args'][10]), 'batch_submit_cubes')
        return self._done, a['out'][:n]

    @property
    def _done(self):
        d = getattr(self, '_done_obj', None)
        if d is None:
            d = self._done_obj = _Done(self)
        return d

    # ---- given model cubes (direct mode) ---------------------------------------
    def window(self):
        """The model window of the direct mode: (offset, size), the voxel
        offset (x, y, z) of its first voxel in the padded grid (whose zero is
        geom.zero_hi) and its size (Wx, Wy, Wz)."""
        off, size = (c_int * 3)(), (c_int * 3)()
        check(_lib.gbkb200_batch_window(self.handle, off, size), 'batch_window')
        return tuple(off), tuple(size)

    def evaluate_cubes_device(self, cubes, nsets, chi2=None, model=None):
        """chi^2 of nsets model cubes (device (>= nsets, Wz, Wy, Wx) float32,
        any gmodel's output on the window) through the direct mode's
        convolution, residual and sum (enqueued on the evaluator's stream,
        not synchronised)."""
        chi2 = self.chi2 if chi2 is None else chi2
        check(_lib.gbkb200_batch_evaluate_cubes(
            self.handle, c_int(int(nsets)), c_void_p(cubes.data_ptr()), c_void_p(chi2.data_ptr()),
            c_void_p(model.data_ptr()) if model is not None else None), 'batch_evaluate_cubes')
        return chi2[:nsets]

    def capture(self, bufs, nsets):
        """Capture one evaluate_device call for nsets sets in a CUDA graph."""
        s = torch.cuda.Stream(self.dev)
        s.wait_stream(torch.cuda.current_stream(self.dev))
        self.ctx.set_stream(s)
        with torch.cuda.stream(s):
            self.evaluate_device(bufs, nsets)   # warm-up outside capture
        torch.cuda.current_stream(self.dev).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            self.evaluate_device(bufs, nsets)
        self.ctx.set_stream(self.stream)
        self._graph = g
        return g

    def replay(self):
        self._graph.replay()
        return self.chi2

    def set_timing(self, enable, counters=True):
        """Per-stage CUDA-event timing of subsequent (uncaptured) evaluations;
        with ``counters`` the direct-mode kernels also count their executed
        work (atomic adds that lengthen the timed launches)."""
        mode = 0 if not enable else (1 if counters else 2)
        check(_lib.gbkb200_batch_set_timing(self.handle, mode), 'batch_set_timing')

    def stage_times(self):
        """{kernel name: (summed ms, launches)} since the last call (synchronises)."""
        ms = (ctypes.c_double * 6)()
        n = (c_int * 6)()
        check(_lib.gbkb200_batch_timing(self.handle, ms, n), 'batch_timing')
        names = STAGE_KERNELS[self.conv_mode]
        return {names[i]: (ms[i], n[i]) for i in range(6) if n[i]}

    def work_counters(self):
        """{counter: executed work} of the direct-mode kernels since the last
        call, counted while timing is enabled with counters (synchronises)."""
        out = (ctypes.c_ulonglong * 8)()
        check(_lib.gbkb200_batch_counters(self.handle, out), 'batch_counters')
        return {n: int(out[i]) for i, n in enumerate(COUNTERS)}

    def close(self):
        """Frees the evaluator's device memory and its native context (with
        the context's scratch, e.g. the serving loop's mcdisk line cubes)."""
        if getattr(self, 'handle', None):
            _lib.gbkb200_batch_destroy(self.handle)
            self.handle = None
        ctx = getattr(self, 'ctx', None)
        if ctx is not None:
            ctx.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _Done:
    """Completion of an evaluator's last asynchronous submission."""

    def __init__(self, ev):
        self._ev = ev
        self._flag = c_int()

    def query(self):
        check(_lib.gbkb200_batch_query(self._ev.handle, ctypes.byref(self._flag)), 'batch_query')
        return bool(self._flag.value)


def row_plan(disk):
    """The per-set input rows of a disk's batched evaluation: [(name,
    [(parameter, size, node-wise, interpolation), ...], row width)] for the
    common parameters and each kind's trait parameters, in Disk.pack_batch's
    order; node-wise values go through the same node -> sub-node
    interpolation as pack_batch for one set."""
    from .disk import _interp, _linear_matrix
    if disk.interp == 'linear':
        # pack_batch's linear interpolation of a batch: y @ W, W fixed per disk
        W = _linear_matrix(disk.rnodes, disk.subrnodes)
        interp = lambda y: y @ W
    else:
        interp = lambda y: _interp(disk.interp, disk.rnodes, y, disk.subrnodes)
    plan = []
    for name in ('vsys', 'xpos', 'ypos', 'posa', 'incl'):
        if name in disk.pdescs:
            nw = disk.pdescs[name][1]
            plan.append((name, [(name, 1, nw, interp)], disk.common_size(name)))
    for kind in KINDS:
        tab = disk.tables[kind]
        if tab is None or not tab['npv']:
            continue
        plan.append((kind, [(pname, size, nw, interp) for pname, size, nw in tab['plist']],
                     tab['npv']))
    return plan


def node_row_tables(disk, n):
    """The device-side row assembly's tables for a disk and a flat buffer of
    n sets (None unless the disk interpolates linearly): the raw layout
    {parameter: (offset, values per set)} of nraw values per set, and per
    output column j its raw indices k0, k1 and weights w0, w1 (the two
    weights of a sub-node's linear interpolation, the matrix pack_batch
    multiplies by, or 1 and 0 for a value taken as it is), its flat offset
    base (the name's block of n rows, then the column) and row stride; the
    name blocks (name, first column, width) and the columns per set."""
    if disk.interp != 'linear':
        return None
    from .disk import _linear_matrix
    wm = _linear_matrix(disk.rnodes, disk.subrnodes)
    raw, nraw = {}, 0
    k0, k1, w0, w1, base, stride, blocks = [], [], [], [], [], [], []
    start = 0
    for name, entries, width in row_plan(disk):
        col = 0
        for pname, size, nw, _ in entries:
            nin = wm.shape[0] if nw else size
            if pname not in raw:
                raw[pname] = (nraw, nin)
                nraw += nin
            ro = raw[pname][0]
            if nw:
                cols = []
                for c in range(wm.shape[1]):
                    nz = np.nonzero(wm[:, c])[0]
                    if len(nz) > 2:
                        return None
                    i0 = int(nz[0]) if len(nz) else 0
                    i1 = int(nz[1]) if len(nz) > 1 else i0
                    cols.append((ro + i0, ro + i1, wm[i0, c] if len(nz) else 0.0,
                                 wm[i1, c] if len(nz) > 1 else 0.0))
            else:
                cols = [(ro + c, ro + c, 1.0, 0.0) for c in range(size)]
            for a, b, wa, wb in cols:
                k0.append(a)
                k1.append(b)
                w0.append(wa)
                w1.append(wb)
                base.append(n * start + col)
                stride.append(width)
                col += 1
        if col != width:
            return None
        blocks.append((name, start, width))
        start += width
    return dict(raw=raw, nraw=nraw, k0=np.asarray(k0, np.int32), k1=np.asarray(k1, np.int32),
                w0=np.asarray(w0, np.float64), w1=np.asarray(w1, np.float64),
                base=np.asarray(base, np.int64), stride=np.asarray(stride, np.int32),
                blocks=blocks, total=start)


def synthetic_data(w, device=0, seed=None):
    """Data cube of a batched workload: the model of w.extra['truth'] (cropped
    cube from the batched evaluator itself) plus Gaussian noise of sigma =
    noise_frac x peak (seeded)."""
    truth = w.extra['truth']
    zeros = np.zeros(w.geom.size[::-1], np.float32)
    ev = BatchedSMDisk(w.disk, w.geom, zeros, max_sets=1, device=device)
    bufs = ev.alloc_inputs(1)
    ev.upload(ev.pack({k: np.asarray(v)[None] for k, v in truth.items()}, 1), bufs, 1)
    model = torch.zeros((1,) + tuple(w.geom.size[::-1]), device=ev.dev)
    ev.evaluate_device(bufs, 1, model=model)
    m = model[0].cpu().numpy().astype(np.float64)
    ev.close()
    rng = np.random.default_rng(w.extra['noise_seed'] if seed is None else seed)
    sigma = w.extra['noise_frac'] * float(np.max(m))
    data = m + rng.normal(0.0, sigma, m.shape)
    return data.astype(np.float32), np.full(m.shape, sigma, np.float32), m
