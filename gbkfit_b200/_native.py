"""ctypes binding of libgbkb200.so (the C ABI declared in include/gbkb200.h).

The library is built in-tree by ``gbkfit_b200.build`` and loaded from the
package directory.  There is no fallback: if the library is missing or fails
to load, importing this module raises.
"""

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# GBKB200_LIB selects another build of the same library (e.g. the bounds-
# checked debug build libgbkb200_checked.so)
LIB_PATH = os.environ.get('GBKB200_LIB') or os.path.join(_HERE, 'libgbkb200.so')

OK = 0
ERRORS = {
    1: 'invalid argument', 2: 'unsupported size or configuration', 3: 'CUDA runtime error',
    4: 'unknown trait uid', 5: 'device allocation failed', 6: 'device-side wait timed out',
    7: 'size exceeds the documented maximum'}


class NativeError(RuntimeError):
    def __init__(self, code, where):
        msg = ERRORS.get(code, f'error {code}')
        if code == 3:
            msg += ': ' + _lib.gbkb200_last_cuda_error().decode()
        super().__init__(f"{where}: {msg}")
        self.code = code


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"the CUDA library {LIB_PATH} is missing; build it with "
            f"`python -c 'import gbkfit_b200.build as b; b.build()'`")
    return ctypes.CDLL(LIB_PATH)


_lib = _load()

c_int, c_float, c_void_p = ctypes.c_int, ctypes.c_float, ctypes.c_void_p
c_int3 = ctypes.c_int * 3
c_float3 = ctypes.c_float * 3

TRAIT_KINDS = ('rpt', 'rht', 'vpt', 'vht', 'dpt', 'dht', 'zpt', 'spt', 'wpt')

# argument list of the disk entry points (include/gbkb200.h GBKB200_DISK_ARGS):
# (name, ctype) in order
DISK_ARGS = [('loose', c_int), ('tilted', c_int), ('nrnodes', c_int), ('rnodes', c_void_p),
             ('vsys', c_void_p), ('xpos', c_void_p), ('ypos', c_void_p), ('posa', c_void_p),
             ('incl', c_void_p)]
for _k, _cnt in (('rpt', 'nrt'), ('rht', None), ('vpt', 'nvt'), ('vht', None),
                 ('dpt', 'ndt'), ('dht', None), ('zpt', 'nzt'), ('spt', 'nst'), ('wpt', 'nwt')):
    if _cnt:
        DISK_ARGS.append((_cnt, c_int))
    DISK_ARGS += [(f'{_k}_{f}', c_void_p) for f in ('uids', 'cvalues', 'ccounts', 'pvalues',
                                                     'pcounts')]
DISK_ARGS += [('opacity', c_void_p),
              ('spat_size_x', c_int), ('spat_size_y', c_int), ('spat_size_z', c_int),
              ('spat_step_x', c_float), ('spat_step_y', c_float), ('spat_step_z', c_float),
              ('spat_zero_x', c_float), ('spat_zero_y', c_float), ('spat_zero_z', c_float),
              ('spec_size', c_int), ('spec_step', c_float), ('spec_zero', c_float)]
DISK_ARGS += [(n, c_void_p) for n in ('image', 'scube', 'wdata', 'wdata_cmp', 'rdata',
                                      'rdata_cmp', 'ordata', 'ordata_cmp', 'vdata_cmp',
                                      'ddata_cmp')]
DISK_TYPES = [t for _, t in DISK_ARGS]

c_ll = ctypes.c_longlong


class ServeArgs(ctypes.Structure):
    """gbkb200_serve_args (include/gbkb200.h): one serving request; the
    parameter arrays are byte offsets into the request's blob (-1 = absent)."""
    _fields_ = [('kind', c_int), ('cflux', c_float), ('nclouds', c_int), ('loose', c_int),
                ('tilted', c_int), ('blob_dev', c_void_p), ('blob_host', c_void_p),
                ('blob_bytes', c_ll), ('off_rnodes', c_ll), ('nrnodes', c_int),
                ('off_vsys', c_ll), ('off_xpos', c_ll), ('off_ypos', c_ll), ('off_posa', c_ll),
                ('off_incl', c_ll), ('ntraits', c_int * 9), ('off_uids', c_ll * 9),
                ('off_cvalues', c_ll * 9), ('off_ccounts', c_ll * 9),
                ('off_pvalues', c_ll * 9), ('off_pcounts', c_ll * 9), ('off_csum', c_ll),
                ('csum_len', c_int), ('off_hasordint', c_ll), ('spat_size', c_int * 3),
                ('spat_step', c_float * 3), ('spat_zero', c_float * 3), ('spec_size', c_int),
                ('spec_step', c_float), ('spec_zero', c_float), ('size_hi', c_int * 3),
                ('edge', c_int * 3), ('size', c_int * 3), ('scube', c_void_p),
                ('work', c_void_p), ('spectrum', c_void_p), ('crop', c_void_p),
                ('obs', c_void_p), ('err', c_void_p), ('msk', c_void_p),
                ('weight', c_float), ('chi2_dev', c_void_p), ('chi2_host', c_void_p),
                ('status_host', c_void_p)]


_SIGS = {
    'gbkb200_ctx_create': [ctypes.POINTER(c_void_p), c_int],
    'gbkb200_ctx_destroy': [c_void_p],
    'gbkb200_ctx_set_stream': [c_void_p, c_void_p],
    'gbkb200_ctx_set_sync': [c_void_p, c_int],
    'gbkb200_ctx_set_mcdisk': [c_void_p, ctypes.c_ulonglong, c_int],
    'gbkb200_ctx_reserve_scratch': [c_void_p, ctypes.c_size_t],
    'gbkb200_mcdisk_scratch_bytes': [c_int, c_int, c_int, c_int],
    'gbkb200_ctx_synchronize': [c_void_p],
    'gbkb200_fft_r2c_f32': [c_void_p, c_int3, c_void_p, c_void_p],
    'gbkb200_fft_c2r_f32': [c_void_p, c_int3, c_void_p, c_void_p],
    'gbkb200_fft_convolve_f32': [c_void_p, c_int3, c_void_p, c_void_p, c_void_p],
    'gbkb200_fft_convolve_cached_f32': [c_void_p, c_int3, c_void_p, c_void_p],
    'gbkb200_fft_clear_cache': [c_void_p],
    'gbkb200_dmodel_dcube_downscale_f32': [c_void_p, c_int3, c_int3, c_int3, c_int3, c_void_p,
                                           c_void_p],
    'gbkb200_dmodel_dcube_mask_f32': [c_void_p, c_float, c_int, c_int3, c_void_p, c_void_p,
                                      c_void_p],
    'gbkb200_dmodel_mmaps_moments_f32': [c_void_p, c_int3, c_float3, c_float3, c_void_p,
                                         c_void_p, c_float, c_int, c_void_p, c_void_p, c_void_p,
                                         c_void_p],
    'gbkb200_gmodel_wcube_evaluate_f32': [c_void_p, c_int, c_int, c_int, c_int, c_void_p,
                                          c_void_p],
    'gbkb200_gmodel_smdisk_evaluate_f32': [c_void_p] + DISK_TYPES,
    'gbkb200_gmodel_mcdisk_evaluate_f32': [c_void_p, c_float, c_int, c_void_p, c_int, c_void_p]
                                          + DISK_TYPES,
    'gbkb200_objective_residual_f32': [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                       c_void_p, c_void_p, c_int, c_float, c_void_p],
    'gbkb200_objective_residual_sum_f32': [c_void_p, c_void_p, c_int, c_int, c_void_p],
    'gbkb200_serve_scube_chi2_f32': [c_void_p, ctypes.POINTER(ServeArgs)],
    'gbkb200_serve_model_f32': [c_void_p, ctypes.POINTER(ServeArgs)],
}

EXPORTED = sorted(_SIGS) + ['gbkb200_error_string', 'gbkb200_last_cuda_error']

for _name, _args in _SIGS.items():
    _f = getattr(_lib, _name)
    _f.argtypes = _args
    _f.restype = c_int
_lib.gbkb200_mcdisk_scratch_bytes.restype = ctypes.c_size_t
_lib.gbkb200_error_string.argtypes = [c_int]
_lib.gbkb200_error_string.restype = ctypes.c_char_p
_lib.gbkb200_last_cuda_error.argtypes = []
_lib.gbkb200_last_cuda_error.restype = ctypes.c_char_p


def lib():
    return _lib


def check(code, where):
    if code != OK:
        raise NativeError(code, where)


def call(name, *args):
    check(getattr(_lib, name)(*args), name)


class Context:
    """One native context: stream, sync mode and FFT caches (gbkb200_ctx)."""

    def __init__(self, device=0, stream=None, sync=True):
        h = c_void_p()
        check(_lib.gbkb200_ctx_create(ctypes.byref(h), int(device)), 'gbkb200_ctx_create')
        self.handle = h
        self.device = device
        if stream is not None:
            self.set_stream(stream)
        self.set_sync(sync)

    def set_stream(self, stream):
        """stream: a torch.cuda.Stream, a raw cudaStream_t int, or None (default)."""
        ptr = getattr(stream, 'cuda_stream', stream) or 0
        check(_lib.gbkb200_ctx_set_stream(self.handle, c_void_p(ptr)), 'set_stream')

    def set_sync(self, sync):
        check(_lib.gbkb200_ctx_set_sync(self.handle, int(bool(sync))), 'set_sync')

    def set_mcdisk(self, seed, mode=0):
        check(_lib.gbkb200_ctx_set_mcdisk(self.handle, int(seed), int(mode)), 'set_mcdisk')

    def reserve_scratch(self, nbytes):
        check(_lib.gbkb200_ctx_reserve_scratch(self.handle, int(nbytes)), 'reserve_scratch')

    def synchronize(self):
        check(_lib.gbkb200_ctx_synchronize(self.handle), 'synchronize')

    def close(self):
        if getattr(self, 'handle', None):
            _lib.gbkb200_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
