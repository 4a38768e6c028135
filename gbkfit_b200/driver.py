"""The B200 driver: memory API plus the four native backends.

Mirrors the reference's driver plugin interface:

* ``Driver`` (gbkfit/driver/core.py:26-90): ``mem_alloc_{s,h,d}``,
  ``mem_copy_{h2d,d2h}``, ``mem_fill``, ``math_*`` and ``backends()``;
* ``DriverBackends`` and ``DriverBackend{FFT,DModel,GModel,Objective}``
  (gbkfit/driver/backend.py:18-158), realised like the reference's native
  backends (gbkfit/driver/drivers/_detail/native.py:214-513): every method
  turns arrays into (pointer, size, shape) and calls the native module, here
  the C ABI of libgbkb200.so.

Device arrays are ``torch`` CUDA tensors (buffers only); host arrays are
numpy arrays backed by pinned memory.  All work is ordered on the driver's
stream (torch's current stream when the driver is created); the native calls
are synchronous, like the reference's (gbkfit_cuda/src/wrapper.cu ends every
call with cudaDeviceSynchronize).
"""

import numpy as np
import torch

from . import _native
from ._native import c_int3, c_float3, call

__all__ = ['DriverB200', 'DriverBackendsB200', 'NativeMemoryB200',
           'DriverBackendFFTB200', 'DriverBackendDModelB200', 'DriverBackendGModelB200',
           'DriverBackendObjectiveB200']

_NP2TORCH = {
    np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64,
    np.dtype(np.int32): torch.int32, np.dtype(np.int64): torch.int64,
    np.dtype(np.bool_): torch.bool, np.dtype(np.uint8): torch.uint8,
    np.dtype(np.complex64): torch.complex64,
}


def torch_dtype(dtype):
    return _NP2TORCH[np.dtype(dtype)]


class NativeMemoryB200:
    """_detail/native.py:191-211 for torch CUDA tensors."""

    @staticmethod
    def ptr(x):
        return x.data_ptr() if x is not None else 0

    @staticmethod
    def size(x):
        return x.numel() if x is not None else 0

    @staticmethod
    def shape(x):
        return tuple(x.shape) if x is not None else None

    @staticmethod
    def dtype(x):
        return x.dtype if x is not None else None


_ptr = NativeMemoryB200.ptr
_size = NativeMemoryB200.size
_shape = NativeMemoryB200.shape


class DriverB200:
    """Driver of type 'b200' (gbkfit/driver/core.py:26-90)."""

    @staticmethod
    def type():
        return 'b200'

    @classmethod
    def load(cls, info, *args, **kwargs):
        return cls(device=info.get('device', 0) if info else 0)

    def dump(self):
        return dict(type=self.type(), device=self.device)

    def __init__(self, device=0):
        if not torch.cuda.is_available():
            raise RuntimeError("DriverB200 needs a CUDA device")
        self.device = int(device)
        self._dev = torch.device('cuda', self.device)
        with torch.cuda.device(self._dev):
            self.stream = torch.cuda.current_stream(self._dev)

    def mem_alloc_s(self, shape, dtype):
        return self.mem_alloc_h(shape, dtype), self.mem_alloc_d(shape, dtype)

    def mem_alloc_h(self, shape, dtype):
        t = torch.empty(tuple(np.atleast_1d(shape).tolist()) if np.ndim(shape) else (int(shape),),
                        dtype=torch_dtype(dtype), pin_memory=True)
        return t.numpy()

    def mem_alloc_d(self, shape, dtype):
        shp = tuple(np.atleast_1d(shape).tolist()) if np.ndim(shape) else (int(shape),)
        return torch.empty(shp, dtype=torch_dtype(dtype), device=self._dev)

    def mem_copy_h2d(self, h_src, d_dst=None):
        if d_dst is None:
            d_dst = self.mem_alloc_d(h_src.shape, h_src.dtype)
        if h_src is not d_dst:
            d_dst.copy_(torch.from_numpy(np.ascontiguousarray(h_src)).reshape(d_dst.shape))
        return d_dst

    def mem_copy_d2h(self, d_src, h_dst=None):
        if h_dst is None:
            h_dst = self.mem_alloc_h(tuple(d_src.shape), _torch2np(d_src.dtype))
        if d_src is not h_dst:
            h_dst[...] = d_src.cpu().numpy().reshape(h_dst.shape)
        return h_dst

    def mem_fill(self, x, value):
        x.fill_(value)

    def math_abs(self, x, out=None):
        return torch.abs(x, out=out)

    def math_sum(self, x, out=None):
        s = torch.nansum(x).reshape((1,) * x.dim())
        if out is not None:
            out.copy_(s)
            return out
        return s

    def math_add(self, x1, x2, out=None):
        return torch.add(x1, x2, out=out)

    def math_sub(self, x1, x2, out=None):
        return torch.sub(x1, x2, out=out)

    def math_mul(self, x1, x2, out=None):
        return torch.mul(x1, x2, out=out)

    def math_div(self, x1, x2, out=None):
        return torch.div(x1, x2, out=out)

    def math_pow(self, x1, x2, out=None):
        return torch.pow(x1, x2, out=out)

    def backends(self):
        return DriverBackendsB200(self.device, self.stream)


def _torch2np(dt):
    for k, v in _NP2TORCH.items():
        if v == dt:
            return k
    raise TypeError(dt)


def _check_dtype(cls, dtype):
    """_detail/native.py:180-188: only float32 is instantiated natively."""
    if np.dtype(dtype) != np.dtype(np.float32):
        raise RuntimeError(
            f"could not create native module wrapper of type '{cls}'; the requested dtype is "
            f"not supported by the native module (requested: {np.dtype(dtype).name}; "
            f"supported: float32)")


class DriverBackendsB200:
    """backend.py:18-34."""

    def __init__(self, device=0, stream=None):
        self._device = device
        self._stream = stream

    def fft(self, dtype):
        return DriverBackendFFTB200(dtype, self._device, self._stream)

    def dmodel(self, dtype):
        return DriverBackendDModelB200(dtype, self._device, self._stream)

    def gmodel(self, dtype):
        return DriverBackendGModelB200(dtype, self._device, self._stream)

    def objective(self, dtype):
        return DriverBackendObjectiveB200(dtype, self._device, self._stream)


class _Native:
    def __init__(self, dtype, device, stream):
        _check_dtype(self.__class__.__qualname__, dtype)
        self._dtype = dtype
        self._device = device
        self._stream = stream
        self._ctx = _native.Context(device=device, stream=stream, sync=True)

    def dtype(self):
        return self._dtype

    @property
    def ctx(self):
        return self._ctx.handle


class DriverBackendFFTB200(_Native):
    """backend.py:37-81 + _detail/native.py:214-250."""

    @staticmethod
    def fft_complex_shape(shape):
        return tuple(list(shape[:-1]) + [shape[-1] // 2 + 1])

    @staticmethod
    def fft_convolution_shift(data):
        """backend.py:43-46: roll the kernel centre to (0, 0, 0)."""
        axis = tuple(range(data.ndim))
        return np.roll(data, np.array(data.shape) // 2 + 1, axis=axis)

    def __init__(self, dtype, device=0, stream=None):
        super().__init__(dtype, device, stream)
        self._fft_shape_threshold = 32

    def fft_optimal_shape(self, shape):
        """backend.py:51-59: power of two up to the threshold, else the next
        multiple of it."""
        th = self._fft_shape_threshold
        out = []
        for dim in shape:
            po2 = 1
            while po2 < dim:
                po2 *= 2
            mul = dim - dim % th + th if dim % th else dim
            out.append(po2 if po2 <= th else mul)
        return np.array(out)

    def fft_convolution_shape(self, data1_shape, data2_shape):
        """backend.py:61-65."""
        shape = np.array(data1_shape) + np.array(data2_shape) - 1
        shape = self.fft_optimal_shape(shape)
        margin = np.array(data2_shape) // 2
        return tuple(int(v) for v in shape), tuple(int(v) for v in margin)

    def fft_r2c(self, data_r, data_c):
        call('gbkb200_fft_r2c_f32', self.ctx, c_int3(*_shape(data_r)[::-1]), _ptr(data_r),
             _ptr(data_c))

    def fft_c2r(self, data_c, data_r):
        call('gbkb200_fft_c2r_f32', self.ctx, c_int3(*_shape(data_r)[::-1]), _ptr(data_c),
             _ptr(data_r))

    def fft_convolve(self, data1_r, data1_c, data2_c):
        call('gbkb200_fft_convolve_f32', self.ctx, c_int3(*_shape(data1_r)[::-1]),
             _ptr(data1_r), _ptr(data1_c), _ptr(data2_c))

    def fft_convolve_cached(self, data1_r, data2_r):
        call('gbkb200_fft_convolve_cached_f32', self.ctx, c_int3(*_shape(data1_r)[::-1]),
             _ptr(data1_r), _ptr(data2_r))

    def clear_cache(self):
        call('gbkb200_fft_clear_cache', self.ctx)


class DriverBackendDModelB200(_Native):
    """backend.py:84-99 + _detail/native.py:253-289."""

    def dcube_downscale(self, scale, edge_hi, cube_hi, cube_lo):
        call('gbkb200_dmodel_dcube_downscale_f32', self.ctx, c_int3(*scale), c_int3(*edge_hi),
             c_int3(*_shape(cube_hi)[::-1]), c_int3(*_shape(cube_lo)[::-1]), _ptr(cube_hi),
             _ptr(cube_lo))

    def dcube_mask(self, cutoff, apply, mcube, dcube, wcube):
        call('gbkb200_dmodel_dcube_mask_f32', self.ctx, float(cutoff), int(bool(apply)),
             c_int3(*_shape(dcube)[::-1]), _ptr(dcube), _ptr(mcube), _ptr(wcube))

    def mmaps_moments(self, size, step, zero, dcube, wcube, cutoff, orders,
                      mmaps_d, mmaps_w, mmaps_m):
        # argument order as _detail/native.py:286-289: (..., d, w, m)
        call('gbkb200_dmodel_mmaps_moments_f32', self.ctx, c_int3(*size), c_float3(*step),
             c_float3(*zero), _ptr(dcube), _ptr(wcube), float(cutoff), _size(orders),
             _ptr(orders), _ptr(mmaps_d), _ptr(mmaps_w), _ptr(mmaps_m))


def _disk_call_args(rnodes, vsys, xpos, ypos, posa, incl, tr, opacity, spat_size, spat_step,
                    spat_zero, spec_size, spec_step, spec_zero, outs):
    """_detail/native.py:349-401: arrays -> (size, pointer) argument list."""
    args = [_size(rnodes), _ptr(rnodes), _ptr(vsys), _ptr(xpos), _ptr(ypos), _ptr(posa),
            _ptr(incl)]
    for kind, cnt in (('rpt', True), ('rht', False), ('vpt', True), ('vht', False),
                      ('dpt', True), ('dht', False), ('zpt', True), ('spt', True),
                      ('wpt', True)):
        uids, cv, cc, pv, pc = tr[kind]
        if cnt:
            args.append(_size(uids))
        args += [_ptr(uids), _ptr(cv), _ptr(cc), _ptr(pv), _ptr(pc)]
    args.append(_ptr(opacity))
    args += [int(spat_size[0]), int(spat_size[1]), int(spat_size[2]),
             float(spat_step[0]), float(spat_step[1]), float(spat_step[2]),
             float(spat_zero[0]), float(spat_zero[1]), float(spat_zero[2]),
             int(spec_size), float(spec_step), float(spec_zero)]
    args += [_ptr(o) for o in outs]
    return args


class DriverBackendGModelB200(_Native):
    """backend.py:102-151 + _detail/native.py:292-475."""

    def wcube_evaluate(self, spat_size, spec_size, spat_data, spec_data):
        call('gbkb200_gmodel_wcube_evaluate_f32', self.ctx, int(spat_size[0]),
             int(spat_size[1]), int(spat_size[2]), int(spec_size), _ptr(spat_data),
             _ptr(spec_data))

    def set_mcdisk(self, seed, mode=0):
        self._ctx.set_mcdisk(seed, mode)

    def mcdisk_evaluate(
            self,
            cflux, nclouds, ncloudspt, hasordint,
            loose, tilted, rnodes,
            vsys, xpos, ypos, posa, incl,
            rpt_uids, rpt_cvalues, rpt_ccounts, rpt_pvalues, rpt_pcounts,
            rht_uids, rht_cvalues, rht_ccounts, rht_pvalues, rht_pcounts,
            vpt_uids, vpt_cvalues, vpt_ccounts, vpt_pvalues, vpt_pcounts,
            vht_uids, vht_cvalues, vht_ccounts, vht_pvalues, vht_pcounts,
            dpt_uids, dpt_cvalues, dpt_ccounts, dpt_pvalues, dpt_pcounts,
            dht_uids, dht_cvalues, dht_ccounts, dht_pvalues, dht_pcounts,
            zpt_uids, zpt_cvalues, zpt_ccounts, zpt_pvalues, zpt_pcounts,
            spt_uids, spt_cvalues, spt_ccounts, spt_pvalues, spt_pcounts,
            wpt_uids, wpt_cvalues, wpt_ccounts, wpt_pvalues, wpt_pcounts,
            opacity,
            spat_size, spat_step, spat_zero, spat_rota,
            spec_size, spec_step, spec_zero,
            image, scube,
            wdata, wdata_cmp,
            rdata, rdata_cmp,
            ordata, ordata_cmp,
            vdata_cmp, ddata_cmp):
        tr = dict(
            rpt=(rpt_uids, rpt_cvalues, rpt_ccounts, rpt_pvalues, rpt_pcounts),
            rht=(rht_uids, rht_cvalues, rht_ccounts, rht_pvalues, rht_pcounts),
            vpt=(vpt_uids, vpt_cvalues, vpt_ccounts, vpt_pvalues, vpt_pcounts),
            vht=(vht_uids, vht_cvalues, vht_ccounts, vht_pvalues, vht_pcounts),
            dpt=(dpt_uids, dpt_cvalues, dpt_ccounts, dpt_pvalues, dpt_pcounts),
            dht=(dht_uids, dht_cvalues, dht_ccounts, dht_pvalues, dht_pcounts),
            zpt=(zpt_uids, zpt_cvalues, zpt_ccounts, zpt_pvalues, zpt_pcounts),
            spt=(spt_uids, spt_cvalues, spt_ccounts, spt_pvalues, spt_pcounts),
            wpt=(wpt_uids, wpt_cvalues, wpt_ccounts, wpt_pvalues, wpt_pcounts))
        outs = (image, scube, wdata, wdata_cmp, rdata, rdata_cmp, ordata, ordata_cmp,
                vdata_cmp, ddata_cmp)
        args = _disk_call_args(rnodes, vsys, xpos, ypos, posa, incl, tr, opacity, spat_size,
                               spat_step, spat_zero, spec_size, spec_step, spec_zero, outs)
        call('gbkb200_gmodel_mcdisk_evaluate_f32', self.ctx, float(cflux), int(nclouds),
             _ptr(ncloudspt), _size(ncloudspt), _ptr(hasordint), loose, tilted, *args)

    def smdisk_evaluate(
            self,
            loose, tilted, rnodes,
            vsys, xpos, ypos, posa, incl,
            rpt_uids, rpt_cvalues, rpt_ccounts, rpt_pvalues, rpt_pcounts,
            rht_uids, rht_cvalues, rht_ccounts, rht_pvalues, rht_pcounts,
            vpt_uids, vpt_cvalues, vpt_ccounts, vpt_pvalues, vpt_pcounts,
            vht_uids, vht_cvalues, vht_ccounts, vht_pvalues, vht_pcounts,
            dpt_uids, dpt_cvalues, dpt_ccounts, dpt_pvalues, dpt_pcounts,
            dht_uids, dht_cvalues, dht_ccounts, dht_pvalues, dht_pcounts,
            zpt_uids, zpt_cvalues, zpt_ccounts, zpt_pvalues, zpt_pcounts,
            spt_uids, spt_cvalues, spt_ccounts, spt_pvalues, spt_pcounts,
            wpt_uids, wpt_cvalues, wpt_ccounts, wpt_pvalues, wpt_pcounts,
            opacity,
            spat_size, spat_step, spat_zero, spat_rota,
            spec_size, spec_step, spec_zero,
            image, scube,
            wdata, wdata_cmp,
            rdata, rdata_cmp,
            ordata, ordata_cmp,
            vdata_cmp, ddata_cmp):
        tr = dict(
            rpt=(rpt_uids, rpt_cvalues, rpt_ccounts, rpt_pvalues, rpt_pcounts),
            rht=(rht_uids, rht_cvalues, rht_ccounts, rht_pvalues, rht_pcounts),
            vpt=(vpt_uids, vpt_cvalues, vpt_ccounts, vpt_pvalues, vpt_pcounts),
            vht=(vht_uids, vht_cvalues, vht_ccounts, vht_pvalues, vht_pcounts),
            dpt=(dpt_uids, dpt_cvalues, dpt_ccounts, dpt_pvalues, dpt_pcounts),
            dht=(dht_uids, dht_cvalues, dht_ccounts, dht_pvalues, dht_pcounts),
            zpt=(zpt_uids, zpt_cvalues, zpt_ccounts, zpt_pvalues, zpt_pcounts),
            spt=(spt_uids, spt_cvalues, spt_ccounts, spt_pvalues, spt_pcounts),
            wpt=(wpt_uids, wpt_cvalues, wpt_ccounts, wpt_pvalues, wpt_pcounts))
        outs = (image, scube, wdata, wdata_cmp, rdata, rdata_cmp, ordata, ordata_cmp,
                vdata_cmp, ddata_cmp)
        args = _disk_call_args(rnodes, vsys, xpos, ypos, posa, incl, tr, opacity, spat_size,
                               spat_step, spat_zero, spec_size, spec_step, spec_zero, outs)
        call('gbkb200_gmodel_smdisk_evaluate_f32', self.ctx, loose, tilted, *args)


class DriverBackendObjectiveB200(_Native):
    """backend.py:154-158 + _detail/native.py:478-513."""

    def residual(self, obs_d, obs_e, obs_m, mdl_d, mdl_w, mdl_m, weight, res):
        call('gbkb200_objective_residual_f32', self.ctx, _ptr(obs_d), _ptr(obs_e), _ptr(obs_m),
             _ptr(mdl_d), _ptr(mdl_w), _ptr(mdl_m), _size(obs_d), float(weight), _ptr(res))

    def residual_sum(self, residual, squared, sum_):
        call('gbkb200_objective_residual_sum_f32', self.ctx, _ptr(residual), _size(residual),
             int(bool(squared)), _ptr(sum_))

    def count_elements(self, array1, array2, threshold, counts):
        raise NotImplementedError("count_pixels is not on the model-evaluation path")

    def foo(self):
        pass
