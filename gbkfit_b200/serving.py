"""Serving loop: continuous batching of model evaluations of uneven sizes.

No reference counterpart (GBKFIT evaluates one model per call).  Samplers and
fitters register their datasets (cube geometry, PSF, LSF, data and error
cubes) and then submit model evaluations against them from any thread; each
submission returns a ``concurrent.futures.Future`` of its chi^2 (and,
optionally, its model cube).

* Resident state: per dataset the PSF x LSF spectrum on the FFT grid
  (computed once, _dcube.py:189-207 + fft.hpp:98-125), the data and error
  cubes; the FFT plans live in the slots' native contexts and are reused by
  every request of the same grid size.
* Continuous batching: a scheduler thread keeps up to ``slots`` requests in
  flight, one per CUDA stream (a native context per stream), so requests of
  different sizes overlap on the device.  A request is admitted, in arrival
  order, as soon as a slot is free and the in-flight HBM footprint plus its
  own fits the budget; completions are polled through CUDA events and the
  freed slot and memory are given to the next request at once.
* Per request, one native call (gbkb200_serve_scube_chi2_f32) enqueues on
  its slot's stream: the copy of the packed parameters from pinned memory,
  smdisk or mcdisk on the padded grid (gmodels.hpp), the FFT convolution with
  the dataset's spectrum, the crop (dmodels.hpp:7-46), the residual and its
  sum of squares (objective.hpp:7-31, host/kernels.hpp:502-514), and the
  copies of chi^2 and the kernel status word to pinned host memory; the
  argument block is filled in the submitting thread, so the scheduler only
  sets the slot's buffers and makes the call.
* Coalescing: a dataset registered with its smdisk disk and a separable
  (rank-1) PSF keeps a batched evaluator of that disk (direct separable
  convolution, gbkb200_batch_*).  Its queued smdisk requests are packed into
  per-set parameter rows when they are submitted and started together, up
  to the evaluator's batch, whenever the evaluator is idle: one H2D copy of
  the rows, one batched evaluation, one D2H copy of chi^2 on the dataset's
  own stream.  Each request's chi^2 does not depend on the others of its
  launch (per-set partial sums in a fixed order).  Its queued mcdisk
  requests are coalesced the same way, up to mc_sets per launch: each
  request's clouds are splatted into its own cube on the evaluator's model
  window (gbkb200_serve_model_f32), and one launch convolves all of them
  with the separable PSF and LSF and takes their residual sums
  (gbkb200_batch_evaluate_cubes), instead of an FFT convolution of the
  padded grid per request.
* Latency: completion minus arrival (the submit time, or the arrival time a
  caller passes); the packing of the parameters happens in submit, after
  the arrival.  ``ModelServer.stats()`` gives p50/p99 and throughput.
"""

import collections
import threading
import time
import weakref
from concurrent.futures import Future

import numpy as np
import torch

from . import _native
from ._native import c_int, check
from .disk import KINDS

c_int3 = c_int * 3
_lib = _native.lib()
# per disk: {kind: (blob template, layout)} of Request.prepare
_BLOBS = weakref.WeakKeyDictionary()


def _ptr(t):
    return None if t is None else t.data_ptr()


def _cbytes(size_hi):
    px, py, pz = size_hi
    return 8 * (px // 2 + 1) * py * pz


class Dataset:
    """A registered dataset: geometry (workloads.Geometry, with PSF/LSF),
    data and error cubes (nz, ny, nx); resident on the device with the
    PSF x LSF spectrum of its FFT grid.

    smdisk: optionally, the thin smooth disk (gbkfit_b200.disk.Disk) that
    smdisk requests against this dataset use; when its PSF is separable
    (rank 1, e.g. a circular Gaussian) the dataset keeps a batched evaluator
    of that disk (direct separable convolution, batch_sets sets per launch,
    its own stream) and queued smdisk requests of that disk are coalesced
    into its launches."""

    MC_STAGE = 1 << 16      # bytes of a coalesced mcdisk request's packed parameters at most

    def __init__(self, key, geom, data, error, ctx, dev, stream, smdisk=None, batch_sets=16,
                 mc_sets=4, mc_seed=42):
        self.key, self.geom = key, geom
        f32 = lambda a: None if a is None else torch.as_tensor(
            np.ascontiguousarray(a, np.float32)).to(dev)
        self.obs, self.err = f32(data), f32(error)
        self.size_hi = tuple(geom.size_hi)
        px, py, pz = self.size_hi
        pcube = f32(geom.pcube(np.float32))
        self.spectrum = torch.empty(_cbytes(self.size_hi) // 4, dtype=torch.float32, device=dev)
        with torch.cuda.stream(stream):
            check(_lib.gbkb200_fft_r2c_f32(ctx.handle, c_int3(*self.size_hi), _ptr(pcube),
                                           _ptr(self.spectrum)), 'fft_r2c')
        stream.synchronize()
        self.footprint = self.spectrum.numel() * 4 + 2 * 4 * int(np.prod(geom.size))
        self.args_cache = {}    # (layout id, thick, window) -> (layout, ServeArgs template)
        self.holders = 0        # submitted requests that have not completed
        self.released = False   # unregistered
        self.smdisk, self.batched = smdisk, None
        self.group = None       # (event, chi2 host view, requests) of the launch in flight
        self.window = None      # (size, zero) of the model window of coalesced mcdisk requests
        self.mc_sets = 0
        if smdisk is not None and not smdisk.traits['rht'] and batch_sets > 0:
            from .batched import BatchedSMDisk, kernel_boxes, separable_factors
            if separable_factors(kernel_boxes(geom)[0])[0] == 1:
                self.batched = BatchedSMDisk(
                    smdisk, geom, self.obs, self.err, max_sets=int(batch_sets),
                    chunk=int(batch_sets), conv='direct', device=dev.index,
                    stream=torch.cuda.Stream(dev))
                self.footprint += self.batched.work_bytes + 4 * self.batched.max_sets
        if self.batched is not None and mc_sets > 0:
            (ox, oy, oz), (wx, wy, wz) = self.batched.window()
            st, z = geom.step, geom.zero_hi
            self.window = ((wx, wy, wz), (z[0] + ox * st[0], z[1] + oy * st[1], z[2] + oz * st[2]))
            self.mc_sets = min(int(mc_sets), self.batched.max_sets)
            self.mc_cubes = torch.empty((self.mc_sets, wz, wy, wx), dtype=torch.float32,
                                        device=dev)
            self.mc_h = torch.empty((self.mc_sets, self.MC_STAGE), dtype=torch.uint8,
                                    pin_memory=True)
            self.mc_d = torch.empty((self.mc_sets, self.MC_STAGE), dtype=torch.uint8, device=dev)
            # fast mode: the clouds' lines go through a channel-contiguous
            # scratch cube of the window held by the evaluator's context
            self.batched.ctx.set_mcdisk(mc_seed, 0)
            # the fast mode's line scratch at its largest (densest clouds)
            scratch = int(_lib.gbkb200_mcdisk_scratch_bytes(2 ** 31 - 1, wx, wy, wz))
            self.batched.ctx.reserve_scratch(scratch)
            self.footprint += self.mc_cubes.numel() * 4 + self.mc_d.numel() + scratch

    def request_layout(self):
        """Byte offsets of one in-flight request's device buffers (padded
        cube, its spectrum, cropped model, chi^2), 256-byte
        aligned, and their total."""
        px, py, pz = self.size_hi
        n = int(np.prod(self.geom.size))
        off, lay = 0, {}
        for name, nb in (('scube', 4 * px * py * pz), ('work', _cbytes(self.size_hi)),
                         ('crop', 4 * n), ('chi2', 4)):
            lay[name] = off
            off += (nb + 255) // 256 * 256
        return lay, off

    def request_footprint(self):
        """Device bytes of one in-flight request."""
        return self.request_layout()[1]


class Request:
    """One model evaluation: kind 'smdisk' or 'mcdisk'; disk
    (gbkfit_b200.disk.Disk) and its parameter dict; for mcdisk the cloud
    flux; thick: evaluate on the 3-D spatial grid (thick disks)."""

    def __init__(self, dataset, kind, disk, params, cflux=None, thick=False, want_model=False,
                 arrival=None):
        if kind not in ('smdisk', 'mcdisk'):
            raise ValueError(f"unknown request kind '{kind}'")
        if kind == 'mcdisk' and not cflux:
            raise ValueError("an mcdisk request needs its cloud flux")
        self.dataset, self.kind, self.disk, self.params = dataset, kind, disk, params
        self.cflux, self.thick, self.want_model = cflux, thick, want_model
        self.arrival = arrival
        self.admit = self.done = None
        self.future = Future()
        self.blob = self.layout = self.args = self.ds = None
        self.rows = None        # packed parameter row of a coalesced smdisk request
        self.cube = False       # a coalesced mcdisk request (model on the dataset's window)

    @staticmethod
    def _varying(packed, csum):
        """The blob's arrays that change from request to request of one disk."""
        for k in ('vsys', 'xpos', 'ypos', 'posa', 'incl'):
            yield k, packed[k]
        for k in KINDS:
            t = packed[k]
            yield k + '.pvalues', None if t is None else t['pvalues']
        if csum is not None:
            yield 'csum', csum

    def prepare(self):
        """Pack the parameters (Disk.pack, and the cloud budget of mcdisk)
        into one byte blob: the arrays at 16-byte aligned offsets.  The
        layout and the arrays that do not depend on the parameters (nodes,
        trait uids, constants and counts) are kept per disk and kind, so a
        request of a disk seen before only writes its own values into a copy
        of that blob."""
        packed = self.disk.pack(self.params)
        csum = None
        if self.kind == 'mcdisk':
            csum = np.asarray(self.disk.ncloudscsum(self.params, self.cflux), np.int32)
            self.nclouds = int(csum[-1]) if csum.size else 0
        cache = _BLOBS.get(self.disk)
        if cache is None:
            cache = _BLOBS[self.disk] = {}
        ent = cache.get(self.kind)
        if ent is not None:
            template, layout = ent
            blob = template.copy()
            for name, a in self._varying(packed, csum):
                off, n = layout[name]
                if (a is None) != (off is None) or (a is not None and a.size != n):
                    break       # another shape: lay the blob out again
                if a is not None:
                    a = np.ascontiguousarray(a, np.int32 if name == 'csum' else np.float32)
                    blob[off:off + a.nbytes] = a.view(np.uint8).ravel()
            else:
                self.blob, self.layout = blob, layout
                return
        arrays = []
        for k in ('subrnodes', 'vsys', 'xpos', 'ypos', 'posa', 'incl'):
            arrays.append((k, packed[k]))
        for k in KINDS:
            t = packed[k]
            for f in ('uids', 'cvalues', 'ccounts', 'pvalues', 'pcounts'):
                arrays.append((k + '.' + f, None if t is None else t[f]))
        if csum is not None:
            arrays.append(('csum', csum))
            arrays.append(('hoi', np.asarray(self.disk.hasordint(), np.uint8)))
        layout, off, chunks = {}, 0, []
        for name, a in arrays:
            if a is None:
                layout[name] = (None, 0)
                continue
            a = np.ascontiguousarray(a)
            if a.dtype == np.float64:
                a = a.astype(np.float32)
            b = a.view(np.uint8).ravel()
            layout[name] = (off, a.size)
            chunks.append((off, b))
            off += (b.size + 15) // 16 * 16
        blob = np.zeros(max(off, 16), np.uint8)
        for o, b in chunks:
            blob[o:o + b.size] = b
        cache[self.kind] = (blob.copy(), layout)
        self.blob, self.layout = blob, layout

    def serve_args(self, ds, window=None):
        """The native argument block of this request against dataset ds
        (everything but the slot's buffers, which the scheduler sets); with
        window = (size, zero) of a batched evaluator's model window, the model
        is evaluated on that window instead of the padded grid.  The block
        depends on the request only through its cloud budget: the rest is
        built once per (layout, thick, window) and kept by the dataset."""
        lay = self.layout
        key = (id(lay), bool(self.thick), window is not None)
        ent = ds.args_cache.get(key)
        if ent is None or ent[0] is not lay:
            ent = ds.args_cache[key] = (lay, self._serve_args(ds, window))
        a = _native.ServeArgs.from_buffer_copy(ent[1])
        if a.kind == 1:
            a.cflux, a.nclouds = float(self.cflux), int(self.nclouds)
        return a

    def _serve_args(self, ds, window):
        lay, g = self.layout, ds.geom
        off = lambda name: -1 if lay[name][0] is None else lay[name][0]
        a = _native.ServeArgs()
        a.kind = 0 if self.kind == 'smdisk' else 1
        if a.kind == 1:
            a.cflux, a.nclouds = float(self.cflux), int(self.nclouds)
            a.off_csum, a.csum_len = off('csum'), lay['csum'][1]
            a.off_hasordint = off('hoi')
        else:
            a.off_csum = a.off_hasordint = -1
        a.loose, a.tilted = int(self.disk.loose), int(self.disk.tilted)
        a.blob_bytes = self.blob.size
        a.off_rnodes, a.nrnodes = off('subrnodes'), lay['subrnodes'][1]
        a.off_vsys, a.off_xpos, a.off_ypos = off('vsys'), off('xpos'), off('ypos')
        a.off_posa, a.off_incl = off('posa'), off('incl')
        for i, k in enumerate(KINDS):
            a.ntraits[i] = lay[k + '.uids'][1]
            a.off_uids[i], a.off_cvalues[i] = off(k + '.uids'), off(k + '.cvalues')
            a.off_ccounts[i], a.off_pvalues[i] = off(k + '.ccounts'), off(k + '.pvalues')
            a.off_pcounts[i] = off(k + '.pcounts')
        ss, st, sz = g.spat(self.thick)
        spec = g.spec()
        if window is not None:
            (wx, wy, wz), (zx, zy, zz) = window
            ss, sz = (wx, wy, ss[2]), (zx, zy, sz[2])
            spec = (wz, spec[1], zz)
        a.spat_size[:] = [int(v) for v in ss]
        a.spat_step[:] = [float(v) for v in st]
        a.spat_zero[:] = [float(v) for v in sz]
        a.spec_size, a.spec_step, a.spec_zero = int(spec[0]), float(spec[1]), float(spec[2])
        a.size_hi[:] = list(ds.size_hi)
        a.edge[:] = [int(v) for v in g.edge]
        a.size[:] = [int(v) for v in g.size]
        a.spectrum, a.obs, a.err = _ptr(ds.spectrum), _ptr(ds.obs), _ptr(ds.err)
        a.msk, a.weight = None, 1.0
        return a


class _Slot:
    STAGE = 1 << 20     # bytes of a request's packed parameters at most

    def __init__(self, dev, mc_seed):
        self.stream = torch.cuda.Stream(dev)
        self.h_stage = torch.empty(self.STAGE, dtype=torch.uint8, pin_memory=True)
        self.d_stage = torch.empty(self.STAGE, dtype=torch.uint8, device=dev)
        self.ctx = _native.Context(device=dev.index, stream=self.stream, sync=False)
        # one atomic per channel: no scratch cube outside the HBM budget
        self.ctx.set_mcdisk(mc_seed, 3)
        self.event = torch.cuda.Event()
        self.out = torch.empty(1, dtype=torch.float32, pin_memory=True)
        self.status = torch.zeros(1, dtype=torch.int32, pin_memory=True)
        self.req = None
        self.keep = None
        self.bytes = 0


class ModelServer:
    """Continuous-batching model-evaluation server on one GPU.

    hbm_budget: device bytes for the registered datasets plus the in-flight
    requests; slots: requests in flight at most (one CUDA stream each)."""

    def __init__(self, device=0, hbm_budget=8 << 30, slots=8, mc_seed=42):
        self.dev = torch.device('cuda', device)
        self.budget = int(hbm_budget)
        self.mc_seed = mc_seed
        self._setup_stream = torch.cuda.Stream(self.dev)
        self._setup_ctx = _native.Context(device=device, stream=self._setup_stream, sync=False)
        self.datasets = {}
        self._slots = [_Slot(self.dev, mc_seed) for _ in range(int(slots))]
        self._queue = collections.deque()
        self._cv = threading.Condition()
        self._stop = False
        self._resident = 0          # dataset bytes
        self._inflight = 0          # in-flight request bytes
        self.max_inflight_bytes = 0
        self.max_inflight = 0
        self.max_group = 0          # largest coalesced launch
        self._group_ds = []         # datasets with a batched evaluator
        self._done = []
        self._error = None
        self._thread = threading.Thread(target=self._run, name='gbkb200-serving', daemon=True)
        self._thread.start()

    # ---- datasets --------------------------------------------------------------
    def register(self, key, geom, data, error=None, smdisk=None, batch_sets=16, mc_sets=4):
        """Make a dataset resident (its spectrum is computed now).  smdisk:
        the thin disk of its smdisk requests, whose requests are then
        coalesced into batched launches of up to batch_sets sets, and its
        mcdisk requests into launches of up to mc_sets (see Dataset)."""
        with torch.cuda.device(self.dev):
            ds = Dataset(key, geom, data, error, self._setup_ctx, self.dev, self._setup_stream,
                         smdisk=smdisk, batch_sets=batch_sets, mc_sets=mc_sets,
                         mc_seed=self.mc_seed)
        with self._cv:
            if key in self.datasets:
                raise KeyError(f"dataset {key!r} is already registered")
            if self._resident + ds.footprint + ds.request_footprint() > self.budget:
                raise MemoryError(f"dataset {key!r} does not fit the HBM budget")
            self.datasets[key] = ds
            self._resident += ds.footprint
            if ds.batched is not None:
                self._group_ds.append(ds)
        return ds

    def unregister(self, key):
        """Drop a dataset; requests already submitted against it still run
        (each holds its dataset until it completes).  Its device bytes stay
        counted against the budget until the last of them completes."""
        with self._cv:
            ds = self.datasets.pop(key)
            ds.released = True
            if ds.holders == 0:
                self._release(ds)

    def _release(self, ds):
        """An unregistered dataset that no request holds any more (call with
        the lock held): its bytes leave the budget, its evaluator goes."""
        self._resident -= ds.footprint
        if ds in self._group_ds:
            self._group_ds.remove(ds)
        if ds.batched is not None:
            ds.batched.stream.synchronize()
            ds.batched.close()

    # ---- requests --------------------------------------------------------------
    def submit(self, request):
        """Queue a Request; returns its Future (result: dict(chi2=..., and
        model=(nz, ny, nx) array when want_model))."""
        ds = self.datasets.get(request.dataset)
        if ds is None:
            raise KeyError(f"unknown dataset {request.dataset!r}")
        if request.arrival is None:
            request.arrival = time.perf_counter()
        # packing happens here, in the caller's thread, after the arrival time
        request.ds = ds
        if (ds.batched is not None and request.kind == 'smdisk' and request.disk is ds.smdisk
                and not request.want_model and not request.thick):
            request.rows = ds.batched.pack_one(request.params)
        else:
            if request.blob is None:
                request.prepare()
            # mcdisk requests of a dataset with a batched evaluator are
            # coalesced: the model on the evaluator's window
            request.cube = bool(ds.mc_sets and request.kind == 'mcdisk' and
                                not request.want_model and request.blob.size <= ds.MC_STAGE)
        if request.cube:
            request.args = request.serve_args(ds, window=ds.window)
        elif request.rows is None:
            if request.blob.size > _Slot.STAGE:
                raise ValueError("the request's parameter arrays exceed the staging buffer")
            # the request holds its dataset: the native arguments point into the
            # dataset's device buffers until the request completes
            request.args = request.serve_args(ds)
        with self._cv:
            if self._error is not None:
                raise RuntimeError("the serving loop stopped") from self._error
            if self.datasets.get(request.dataset) is not ds:
                raise KeyError(f"dataset {request.dataset!r} was unregistered")
            ds.holders += 1
            self._queue.append(request)
            self._cv.notify()
        return request.future

    def evaluate(self, request):
        """Submit and wait."""
        return self.submit(request).result()

    def close(self):
        with self._cv:
            self._stop = True
            self._cv.notify()
        self._thread.join()
        for s in self._slots:
            s.stream.synchronize()
            s.ctx.close()
        for ds in self.datasets.values():
            if ds.batched is not None:
                ds.batched.stream.synchronize()
                ds.batched.close()
        self._setup_ctx.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def stats(self, reset=False):
        """Latency percentiles (ms), throughput and occupancy of the
        completed requests since the last reset."""
        with self._cv:
            done = list(self._done)
            if reset:
                self._done.clear()
        if not done:
            return dict(requests=0)
        lat = np.array([r.done - r.arrival for r in done]) * 1e3
        t0 = min(r.arrival for r in done)
        t1 = max(r.done for r in done)
        return dict(requests=len(done), p50_ms=float(np.percentile(lat, 50)),
                    p99_ms=float(np.percentile(lat, 99)), mean_ms=float(lat.mean()),
                    max_ms=float(lat.max()), evals_per_s=len(done) / max(t1 - t0, 1e-9),
                    max_inflight=self.max_inflight, max_inflight_bytes=self.max_inflight_bytes,
                    max_group=self.max_group)

    # ---- scheduler -------------------------------------------------------------
    SCAN = 64   # queued requests the scheduler looks at per pass
    # clouds of one coalesced mcdisk launch at most (beyond its first
    # request): the launch's requests all complete with its slowest splat
    MC_GROUP_CLOUDS = 15_000_000

    def _run(self):
        try:
            with torch.cuda.device(self.dev):
                while True:
                    with self._cv:
                        busy = [s for s in self._slots if s.req is not None]
                        groups = [d for d in self._group_ds if d.group is not None]
                        if self._stop and not busy and not groups and not self._queue:
                            return
                        if not busy and not groups and not self._queue:
                            self._cv.wait()
                            continue
                    progressed = False
                    for s in busy:
                        if s.event.query():
                            self._complete(s)
                            progressed = True
                    for d in groups:
                        if d.group[0].query():
                            self._complete_group(d)
                            progressed = True
                    progressed |= self._admit()
                    if not progressed:
                        time.sleep(2e-5)
        except BaseException as e:      # fail every pending future, not the process
            with self._cv:
                self._error = e
                pending = list(self._queue) + [s.req for s in self._slots if s.req is not None]
                for d in self._group_ds:
                    if d.group is not None:
                        pending += d.group[2]
                self._queue.clear()
            for r in pending:
                if not r.future.done():
                    r.future.set_exception(e)

    def _admit(self):
        """Starts what the queue allows, in arrival order among the first
        SCAN requests: a coalesced group for a request of a batched dataset
        whose evaluator is idle (with the dataset's other queued requests), a
        slot for any other request while a slot is free and the HBM budget
        holds.  Requests that cannot start yet are passed over."""
        launches = []
        with self._cv:
            q = [self._queue.popleft() for _ in range(min(len(self._queue), self.SCAN))]
            free = [s for s in self._slots if s.req is None]
            taken = set()
            for i in range(len(q)):
                if i in taken:
                    continue
                req = q[i]
                ds = req.ds
                if req.rows is not None or req.cube:
                    if ds.group is not None or ds in (g[0] for g in launches if g[1] == 'group'):
                        continue
                    # a group of the same kind: parameter rows or mcdisk cubes
                    cube = req.cube
                    cap = ds.mc_sets if cube else ds.batched.max_sets
                    group = [i]
                    clouds = req.nclouds if cube else 0
                    for j in range(i + 1, len(q)):
                        if len(group) >= cap:
                            break
                        if j not in taken and q[j].ds is ds and q[j].cube == cube and (
                                cube or q[j].rows is not None):
                            if cube and clouds + q[j].nclouds > self.MC_GROUP_CLOUDS:
                                continue
                            clouds += q[j].nclouds if cube else 0
                            group.append(j)
                    taken.update(group)
                    launches.append((ds, 'group', [q[j] for j in group]))
                    continue
                if not free:
                    continue
                need = ds.request_footprint()
                if self._resident + self._inflight + need > self.budget and self._inflight > 0:
                    continue
                self._inflight += need
                taken.add(i)
                slot = free.pop(0)
                slot.req = req      # reserved; _launch fills the rest
                launches.append((slot, 'slot', (req, need)))
                nbusy = len(self._slots) - len(free)
                self.max_inflight = max(self.max_inflight, nbusy)
                self.max_inflight_bytes = max(self.max_inflight_bytes, self._inflight)
            # the requests passed over go back to the front, in order
            self._queue.extendleft(reversed([r for k, r in enumerate(q) if k not in taken]))
        done = 0
        try:
            for target, kind, what in launches:
                if kind == 'group':
                    self._launch_group(target, what)
                else:
                    self._launch(target, *what)
                done += 1
        except BaseException as e:
            # the requests taken for launches that did not start are in no
            # queue, slot or group any more: fail their futures here
            for target, kind, what in launches[done:]:
                for r in (what if kind == 'group' else [what[0]]):
                    if not r.future.done():
                        r.future.set_exception(e)
            raise
        return bool(launches)

    def _launch_group(self, ds, reqs):
        now = time.perf_counter()
        for r in reqs:
            r.admit = now
        if reqs[0].cube:
            ev, out = self._launch_cubes(ds, reqs)
        else:
            ev, out = ds.batched.submit_rows([r.rows for r in reqs])
        ds.group = (ev, out, reqs)
        self.max_group = max(self.max_group, len(reqs))

    def _launch_cubes(self, ds, reqs):
        """The models of a group of mcdisk requests, each into its own cube of
        the window, then one convolution + residual + sum launch, all on the
        evaluator's stream.  The staging and cube buffers are the dataset's:
        its previous group has completed (one group in flight per dataset)."""
        bt = ds.batched
        cube_bytes = ds.mc_cubes[0].numel() * 4
        h, d = ds.mc_h.data_ptr(), ds.mc_d.data_ptr()
        hn = ds.mc_h.numpy()
        for i, r in enumerate(reqs):
            nb = r.blob.size
            hn[i, :nb] = r.blob
            a = r.args
            a.blob_host, a.blob_dev = h + i * ds.MC_STAGE, d + i * ds.MC_STAGE
            a.scube = ds.mc_cubes.data_ptr() + i * cube_bytes
            check(_lib.gbkb200_serve_model_f32(bt.ctx.handle, a), 'serve_model')
        return bt.submit_cubes(ds.mc_cubes, len(reqs))

    def _complete_group(self, ds):
        ev, out, reqs = ds.group
        chi2 = out.numpy().copy()
        # a kernel of the group raised the status word (unknown trait uid)
        rc = _lib.gbkb200_batch_take_status(ds.batched.handle)
        now = time.perf_counter()
        with self._cv:
            ds.group = None
            for r in reqs:
                r.done = now
                r.ds = r.args = None
                ds.holders -= 1
                self._done.append(r)
            if ds.released and ds.holders == 0:
                self._release(ds)
        for r, c in zip(reqs, chi2):
            if rc:
                r.future.set_exception(_native.NativeError(rc, 'serving group'))
            else:
                r.future.set_result(dict(chi2=float(c)))

    def _launch(self, slot, req, need):
        ds = req.ds
        req.admit = time.perf_counter()
        slot.req, slot.bytes = req, need
        lay, total = ds.request_layout()
        nb = req.blob.size
        slot.h_stage.numpy()[:nb] = req.blob
        # allocated on the scheduler's stream and released only after the
        # slot's event has completed, so the allocator never hands it out
        # while the slot's stream still uses it
        buf = torch.empty(total, dtype=torch.uint8, device=self.dev)
        b = buf.data_ptr()
        a = req.args
        a.blob_dev, a.blob_host = slot.d_stage.data_ptr(), slot.h_stage.data_ptr()
        a.scube, a.work, a.chi2_dev = b + lay['scube'], b + lay['work'], b + lay['chi2']
        a.crop = b + lay['crop'] if req.want_model else None
        a.chi2_host, a.status_host = slot.out.data_ptr(), slot.status.data_ptr()
        check(_lib.gbkb200_serve_scube_chi2_f32(slot.ctx.handle, a), 'serve_scube_chi2')
        slot.event.record(slot.stream)
        slot.keep = (buf, lay['crop'])

    def _complete(self, slot):
        req = slot.req
        out = dict(chi2=float(slot.out[0]))
        if req.want_model:
            buf, o = slot.keep
            n = int(np.prod(req.ds.geom.size))
            nx, ny, nz = req.ds.geom.size
            out['model'] = buf[o:o + 4 * n].view(torch.float32).reshape(nz, ny, nx).cpu().numpy()
        rc = 0
        if int(slot.status[0]):
            # a kernel of this request raised the status word (unknown trait
            # uid): the context's synchronize reports and clears it
            rc = _lib.gbkb200_ctx_synchronize(slot.ctx.handle)
        req.done = time.perf_counter()
        ds = req.ds
        req.ds = req.args = None        # the dataset may go once no request holds it
        with self._cv:
            ds.holders -= 1
            if ds.released and ds.holders == 0:
                self._release(ds)
            self._inflight -= slot.bytes
            slot.req, slot.keep, slot.bytes = None, None, 0
            self._done.append(req)
        if rc:
            req.future.set_exception(_native.NativeError(rc, 'serving request'))
        else:
            req.future.set_result(out)
