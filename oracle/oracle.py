"""Python harness of the oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by the CPU-baseline leg of bench.py, as the checker.  The product
(gbkfit_b200) never imports it.

* ``Oracle(precision)`` wraps oracle/_build/liboracle.so, the C restatement
  of the reference arithmetic (oracle_impl.h), in float32 ("f32", the
  reference's precision) or float64 ("f64", the fp64 oracle).
* ``Reference()`` wraps oracle/_ref/libgbkfit_ref.so, the reference's own
  templates compiled from its sources (ref_shim.cpp), when it was built.
* ``fft_convolve_cached`` restates the reference FFT convolution
  (gbkfit_host/include/gbkfit/host/fft.hpp:98-207: r2c, multiply by the
  kernel spectrum and 1/N, c2r) with numpy's pocketfft in float64.  FFTW3,
  which the reference uses, is not installed; the identity of the two is
  checked against the reference's direct convolution (gmodels.hpp:9-50).
"""

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(_HERE, '_build', 'liboracle.so')
REF_LIB = os.path.join(_HERE, '_ref', 'libgbkfit_ref.so')

KINDS = ('rpt', 'rht', 'vpt', 'vht', 'dpt', 'dht', 'zpt', 'spt', 'wpt')
OUTS = ('image', 'scube', 'wdata', 'wdata_cmp', 'rdata', 'rdata_cmp', 'ordata', 'ordata_cmp',
        'vdata_cmp', 'ddata_cmp')


def build():
    """Compile the oracle (and oracle/_ref where the reference tree exists)."""
    import subprocess
    subprocess.run(['make', '-s', '-C', _HERE], check=True)


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _as(a, dt):
    return None if a is None else np.ascontiguousarray(a, dtype=dt)


def disk_arglist(packed, geom, outs, real, with_counts=True):
    """The reference's smdisk/mcdisk argument list (host/gmodels.hpp:82-135)
    from a gbkfit_b200.disk.Disk.pack() result.

    geom: dict(loose, tilted, spat_size, spat_step, spat_zero, spec_size,
    spec_step, spec_zero, opacity).  Returns (args, keepalive)."""
    keep = []

    def arr(a, dt):
        a = _as(a, dt)
        keep.append(a)
        return _p(a)

    args = [int(geom['loose']), int(geom['tilted'])]
    rn = _as(packed['subrnodes'], real)
    keep.append(rn)
    args += [len(rn), _p(rn)]
    for name in ('vsys', 'xpos', 'ypos', 'posa', 'incl'):
        args.append(arr(packed[name], real))
    for k, cnt in (('rpt', True), ('rht', False), ('vpt', True), ('vht', False),
                   ('dpt', True), ('dht', False), ('zpt', True), ('spt', True),
                   ('wpt', True)):
        t = packed[k]
        if cnt:
            args.append(0 if t is None else len(t['uids']))
        if t is None:
            args += [None] * 5
        else:
            args += [arr(t['uids'], np.int32), arr(t['cvalues'], real), arr(t['ccounts'], np.int32),
                     arr(t['pvalues'], real), arr(t['pcounts'], np.int32)]
    args.append(arr(geom.get('opacity'), real))
    ss, st, sz = geom['spat_size'], geom['spat_step'], geom['spat_zero']
    R = ctypes.c_float if real == np.float32 else ctypes.c_double
    args += [int(ss[0]), int(ss[1]), int(ss[2]), R(st[0]), R(st[1]), R(st[2]),
             R(sz[0]), R(sz[1]), R(sz[2]), int(geom['spec_size']), R(geom['spec_step']),
             R(geom['spec_zero'])]
    for name in OUTS:
        o = outs.get(name)
        args.append(None if o is None else _p(o))
    return args, keep


class _Lib:
    def __init__(self, path, real):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        self.real = real
        self.R = ctypes.c_float if real == np.float32 else ctypes.c_double


class Oracle(_Lib):
    """The C restatement in float32 ('f32') or float64 ('f64')."""

    def __init__(self, precision='f64'):
        super().__init__(ORACLE_LIB, np.float32 if precision == 'f32' else np.float64)
        self.sfx = '_' + precision
        for n in ('orc_smdisk_evaluate', 'orc_mcdisk_evaluate'):
            getattr(self.lib, n + self.sfx).restype = ctypes.c_int
        self.lib.orc_residual_sum_f32.restype = ctypes.c_double
        self.lib.orc_residual_sum_f64.restype = ctypes.c_double

    def zeros(self, shape):
        return np.zeros(shape, dtype=self.real)

    def smdisk_evaluate(self, packed, geom, outs):
        args, keep = disk_arglist(packed, geom, outs, self.real)
        return getattr(self.lib, 'orc_smdisk_evaluate' + self.sfx)(*args)

    def mcdisk_evaluate(self, cflux, nclouds, csum, hasordint, seed, packed, geom, outs):
        args, keep = disk_arglist(packed, geom, outs, self.real)
        csum = np.ascontiguousarray(csum, np.int32)
        hoi = np.ascontiguousarray(hasordint, np.uint8)
        return getattr(self.lib, 'orc_mcdisk_evaluate' + self.sfx)(
            self.R(cflux), int(nclouds), _p(csum), len(csum), _p(hoi),
            ctypes.c_ulonglong(seed), *args)

    def mmaps_moments(self, size, step, zero, dcube, wcube, cutoff, orders):
        """Returns (mmaps_d, mask map, weight map)."""
        nx, ny, nz = size
        d = _as(dcube, self.real)
        w = _as(wcube, self.real)
        o = np.ascontiguousarray(orders, np.int32)
        md = np.zeros((len(o), ny, nx), self.real)
        mm = np.zeros((ny, nx), self.real)
        mw = np.zeros((ny, nx), self.real)
        R = self.R
        getattr(self.lib, 'orc_mmaps_moments' + self.sfx)(
            nx, ny, nz, R(step[0]), R(step[1]), R(step[2]), R(zero[0]), R(zero[1]), R(zero[2]),
            _p(d), _p(w), R(cutoff), len(o), _p(o), _p(md), _p(mm), _p(mw))
        return md, mm, mw

    def residual(self, od, oe, om, md, mw, mm, weight):
        n = int(np.asarray(od).size)
        res = np.zeros(n, self.real)
        a = [_as(x, self.real) for x in (od, oe, om, md, mw, mm)]
        getattr(self.lib, 'orc_residual' + self.sfx)(
            *[_p(x) for x in a], ctypes.c_long(n), self.R(weight), _p(res))
        return res

    def residual_sum(self, res, squared=True):
        r = _as(res, self.real)
        return getattr(self.lib, 'orc_residual_sum' + self.sfx)(_p(r), ctypes.c_long(r.size),
                                                               int(squared))

    def dcube_downscale(self, scale, offset, src, dst_shape):
        src = _as(src, self.real)
        dst = np.zeros(dst_shape, self.real)
        sz, sy, sx = src.shape
        dz, dy, dx = dst_shape
        getattr(self.lib, 'orc_dcube_downscale' + self.sfx)(
            *[int(v) for v in scale], *[int(v) for v in offset], sx, sy, sz, dx, dy, dz,
            _p(src), _p(dst))
        return dst

    def dcube_mask(self, cutoff, apply, d, with_mask=True):
        d = _as(d, self.real).copy()
        m = np.zeros_like(d) if with_mask else None
        nz, ny, nx = d.shape
        getattr(self.lib, 'orc_dcube_mask' + self.sfx)(self.R(cutoff), int(apply), nx, ny, nz,
                                                      _p(d), _p(m), None)
        return d, m

    def wcube_evaluate(self, spat, spec_z):
        spat = _as(spat, self.real)
        sz, sy, sx = spat.shape
        spec = np.zeros((spec_z, sy, sx), self.real)
        getattr(self.lib, 'orc_wcube_evaluate' + self.sfx)(sx, sy, sz, spec_z, _p(spat), _p(spec))
        return spec

    def convolve(self, a, b):
        """gmodels.hpp:9-50: direct zero-padded convolution (kernel centred at size//2)."""
        a = _as(a, self.real)
        b = _as(b, self.real)
        out = np.zeros_like(a)
        az, ay, ax = a.shape
        bz, by, bx = b.shape
        getattr(self.lib, 'orc_convolve' + self.sfx)(ax, ay, az, bx, by, bz, _p(a), _p(b),
                                                    _p(out))
        return out

    def philox(self, ctr, key0, key1):
        c = (ctypes.c_uint * 4)(*ctr)
        o = (ctypes.c_uint * 4)()
        self.lib.orc_philox4x32(c, ctypes.c_uint(key0), ctypes.c_uint(key1), o)
        return list(o)


class Reference(_Lib):
    """The reference's own templates (float32), compiled in oracle/_ref."""

    def __init__(self):
        super().__init__(REF_LIB, np.float32)
        self.lib.ref_num_threads.restype = ctypes.c_int

    @staticmethod
    def available():
        return os.path.exists(REF_LIB)

    def num_threads(self):
        return self.lib.ref_num_threads()

    def set_num_threads(self, n):
        """OpenMP threads of the following calls (one thread: the reference's
        mcdisk draws all clouds from one mt19937 stream seeded 42)."""
        self.lib.ref_set_num_threads(int(n))

    def smdisk_evaluate(self, packed, geom, outs):
        args, keep = disk_arglist(packed, geom, outs, np.float32)
        self.lib.ref_smdisk_evaluate_f32(*args)

    def mcdisk_evaluate(self, cflux, nclouds, csum, hasordint, packed, geom, outs):
        args, keep = disk_arglist(packed, geom, outs, np.float32)
        csum = np.ascontiguousarray(csum, np.int32)
        hoi = np.ascontiguousarray(hasordint, np.uint8)
        self.lib.ref_mcdisk_evaluate_f32(ctypes.c_float(cflux), int(nclouds), _p(csum),
                                         len(csum), _p(hoi), *args)

    def mmaps_moments(self, size, step, zero, dcube, wcube, cutoff, orders):
        nx, ny, nz = size
        d = _as(dcube, np.float32)
        w = _as(wcube, np.float32)
        o = np.ascontiguousarray(orders, np.int32)
        md = np.zeros((len(o), ny, nx), np.float32)
        mm = np.zeros((ny, nx), np.float32)
        mw = np.zeros((ny, nx), np.float32)
        F = ctypes.c_float
        # native argument order: (..., mmaps_d, mmaps_m, mmaps_w) with the
        # kernel swap: the m slot receives the weights, the w slot the mask
        self.lib.ref_mmaps_moments_f32(nx, ny, nz, F(step[0]), F(step[1]), F(step[2]),
                                       F(zero[0]), F(zero[1]), F(zero[2]), _p(d), _p(w),
                                       F(cutoff), len(o), _p(o), _p(md), _p(mw), _p(mm))
        return md, mm, mw

    def residual(self, od, oe, om, md, mw, mm, weight):
        n = int(np.asarray(od).size)
        res = np.zeros(n, np.float32)
        a = [_as(x, np.float32) for x in (od, oe, om, md, mw, mm)]
        self.lib.ref_residual_f32(*[_p(x) for x in a], n, ctypes.c_float(weight), _p(res))
        return res

    def residual_sum(self, res, squared=True):
        r = _as(res, np.float32)
        out = np.zeros(1, np.float32)
        self.lib.ref_residual_sum_f32(_p(r), r.size, int(squared), _p(out))
        return float(out[0])

    def dcube_downscale(self, scale, offset, src, dst_shape):
        src = _as(src, np.float32)
        dst = np.zeros(dst_shape, np.float32)
        sz, sy, sx = src.shape
        dz, dy, dx = dst_shape
        self.lib.ref_dcube_downscale_f32(*[int(v) for v in scale], *[int(v) for v in offset],
                                         sx, sy, sz, dx, dy, dz, _p(src), _p(dst))
        return dst

    def dcube_mask(self, cutoff, apply, d):
        d = _as(d, np.float32).copy()
        m = np.zeros_like(d)
        nz, ny, nx = d.shape
        self.lib.ref_dcube_mask_f32(ctypes.c_float(cutoff), int(apply), nx, ny, nz, _p(d), _p(m),
                                    None)
        return d, m

    def wcube_evaluate(self, spat, spec_z):
        spat = _as(spat, np.float32)
        sz, sy, sx = spat.shape
        spec = np.zeros((spec_z, sy, sx), np.float32)
        self.lib.ref_wcube_evaluate_f32(sx, sy, sz, spec_z, _p(spat), _p(spec))
        return spec

    def convolve(self, a, b):
        a = _as(a, np.float32)
        b = _as(b, np.float32)
        out = np.zeros_like(a)
        az, ay, ax = a.shape
        bz, by, bx = b.shape
        self.lib.ref_convolve_f32(ax, ay, az, bx, by, bz, _p(a), _p(b), _p(out))
        return out


def fft_convolve_cached(data1, data2, dtype=np.float64, workers=1):
    """fft.hpp:98-207 in float64: irfftn(rfftn(data1) * rfftn(data2)) (the
    1/N normalisation of the reference is numpy's backward-norm inverse)."""
    import scipy.fft
    a = np.asarray(data1, dtype)
    b = np.asarray(data2, dtype)
    spec = scipy.fft.rfftn(a, workers=workers) * scipy.fft.rfftn(b, workers=workers)
    return scipy.fft.irfftn(spec, s=a.shape, workers=workers)


def scube_pipeline(packed, geom, loose=False, tilted=False, precision='f64', thick=False,
                   spat_z=None):
    """The reference's DModelSCube chain for one parameter set
    (dmodels/scube.py:95-122, _dcube.py:245-289): smdisk on the padded grid,
    FFT convolution with the rolled PSF x LSF cube, crop.  geom is a
    gbkfit_b200.workloads.Geometry (its padding follows backend.py:51-66)."""
    o = Oracle(precision)
    ss, st, sz = geom.spat(thick, spat_z)
    nz_hi = geom.size_hi[2]
    g = dict(loose=loose, tilted=tilted, spat_size=ss, spat_step=st, spat_zero=sz,
             spec_size=nz_hi, spec_step=geom.step[2], spec_zero=geom.zero_hi[2], opacity=None)
    cube = np.zeros((nz_hi, ss[1], ss[0]), o.real)
    o.smdisk_evaluate(packed, g, dict(scube=cube))
    conv = fft_convolve_cached(cube, geom.pcube(np.float64 if precision == 'f64' else np.float32))
    ex, ey, ez = geom.edge
    nx, ny, nz = geom.size
    return conv[ez:ez + nz, ey:ey + ny, ex:ex + nx]


def chi2(model, data, error):
    """objective.hpp:7-31 + host/kernels.hpp:502-514 in float64."""
    r = (np.asarray(model, np.float64) - data) / error
    return float(np.sum(r * r))


def chi2_gradient_f64(packed, geom, data, error, scale):
    """fp64 reference gradient of chi^2 for a thin flat disk with node-wise
    density (uid 101), rotation (uid 101) and dispersion (uid 101): the
    smdisk line model of gmodels.hpp:645-958 (sky -> disk, math.hpp:63-71;
    ring interpolation, traits.hpp:138-141, 999-1007; line, gmodels.hpp
    :92-116) on the padded grid, the circular convolution with geom.pcube()
    (fft.hpp:98-207), the crop, r = (scale conv - d) / e (objective.hpp:7-31),
    differentiated analytically in float64 (numpy), every spaxel's line
    window held fixed.  Returns (chi^2, d chi^2 / d sub-node and geometry
    values) in the layout of gbkb200_gmodel_smdisk_nw_adjoint_f32 (density,
    rotation, dispersion sub-nodes, vsys, xpos, ypos, posa, incl), and
    d chi^2 / d scale."""
    import scipy.fft
    f = np.float64
    sub = np.asarray(packed['subrnodes'], f)
    ns = len(sub)
    bs = np.asarray(packed['rpt']['pvalues'], f)
    vs = np.asarray(packed['vpt']['pvalues'], f)
    ds = np.asarray(packed['dpt']['pvalues'], f)
    vsys = float(packed['vsys'][0]) if packed['vsys'] is not None else 0.0
    xpos, ypos = float(packed['xpos'][0]), float(packed['ypos'][0])
    phi, inc = np.deg2rad(float(packed['posa'][0])), np.deg2rad(float(packed['incl'][0]))
    sp, cp, si, ci = np.sin(phi), np.cos(phi), np.sin(inc), np.cos(inc)
    px, py, pz = geom.size_hi
    (sx, sy, _), (stx, sty, _), (zx, zy, _) = geom.spat()
    nz, dz, z0 = geom.spec()
    X = zx + np.arange(sx) * stx
    Y = zy + np.arange(sy) * sty
    xn = X[None, :] - xpos + 0 * Y[:, None]
    yn = Y[:, None] - ypos + 0 * X[None, :]
    xr = -xn * sp + yn * cp
    yr = -xn * cp - yn * sp
    yd = yr / ci
    r = np.sqrt(xr * xr + yd * yd)
    on = (r >= sub[0]) & (r < sub[-1])
    k = np.clip(np.searchsorted(sub, r, side='right'), 1, ns - 1)
    s0, s1 = sub[k - 1], sub[k]
    t = (r - s0) / (s1 - s0)
    bl = bs[k - 1] + t * (bs[k] - bs[k - 1])
    on &= bl != 0
    rho = bl / ci
    rs = np.where(r > 0, r, 1.0)
    c = np.where(r > 0, xr / rs, 0.0)
    sn = np.where(r > 0, yd / rs, 0.0)
    vrot = vs[k - 1] + t * (vs[k] - vs[k - 1])
    vv = np.where(r > 0, vrot * c * si, 0.0) + vsys
    draw = ds[k - 1] + t * (ds[k] - ds[k - 1])
    sig = np.abs(draw)
    sgn = np.where(draw < 0, -1.0, 1.0)
    sig_s = np.where(on, sig, 1.0)
    lo = np.maximum(np.rint((vv - 5 * sig - z0) / dz), 0)
    hi = np.minimum(np.rint((vv + 5 * sig - z0) / dz), nz - 1)
    on &= lo <= hi
    zv = z0 + np.arange(nz)[:, None, None] * dz
    iz = np.arange(nz)[:, None, None]
    win = on[None] & (iz >= lo[None]) & (iz <= hi[None])
    d = zv - vv[None]
    L = np.where(win, np.exp(-d * d / (2 * sig_s[None] ** 2)) / (sig_s[None] * np.sqrt(2 * np.pi)),
                 0.0)
    model = np.zeros((pz, py, px), f)
    model[:nz] = rho[None] * L
    pc = np.asarray(geom.pcube(f), f)
    K = scipy.fft.rfftn(pc)
    conv = scipy.fft.irfftn(scipy.fft.rfftn(model) * K, s=model.shape)
    ex, ey, ez = geom.edge
    Nx, Ny, Nz = geom.size
    cc = conv[ez:ez + Nz, ey:ey + Ny, ex:ex + Nx]
    e = np.asarray(error, f)
    res = (scale * cc - np.asarray(data, f)) / e
    chi2 = float(np.sum(res * res))
    dscale = float(np.sum(2 * res / e * cc))
    gP = np.zeros_like(model)
    gP[ez:ez + Nz, ey:ey + Ny, ex:ex + Nx] = 2 * res / e * scale
    G = scipy.fft.irfftn(scipy.fft.rfftn(gP) * np.conj(K), s=model.shape)[:nz]
    GL = G * L
    S0 = GL.sum(0)
    S1 = (GL * d).sum(0)
    S2 = (GL * d * d).sum(0)
    drho = S0
    dvv = rho * S1 / sig_s ** 2
    dsig = rho * (S2 / sig_s ** 3 - S0 / sig_s)
    wb = np.where(on, drho / ci, 0.0)
    wv = np.where(on & (r > 0), dvv * c * si, 0.0)
    wd = np.where(on, dsig * sgn, 0.0)
    grad = np.zeros(3 * ns + 5)
    for j, w_ in enumerate((wb, wv, wd)):
        np.add.at(grad, (j * ns + k - 1)[on], ((1 - t) * w_)[on])
        np.add.at(grad, (j * ns + k)[on], (t * w_)[on])
    ds_ = s1 - s0
    dr = wb * (bs[k] - bs[k - 1]) / ds_ + wv * (vs[k] - vs[k - 1]) / ds_ + \
        wd * (ds[k] - ds[k - 1]) / ds_
    dc = np.where(r > 0, dvv * vrot * si, 0.0)
    ti = si / ci
    di = drho * rho * ti + np.where(r > 0, dvv * vrot * c * ci, 0.0)
    dxr = np.where(r > 0, dr * c + dc * sn * sn / rs, 0.0)
    dyd = np.where(r > 0, dr * sn - dc * c * sn / rs, 0.0)
    dyr = dyd / ci
    di = di + dyd * yd * ti
    dxn = -dxr * sp - dyr * cp
    dyn = dxr * cp - dyr * sp
    dphi = dxr * yr - dyr * xr
    g0 = 3 * ns
    grad[g0 + 0] = np.sum(np.where(on, dvv, 0.0))
    grad[g0 + 1] = -np.sum(np.where(on, dxn, 0.0))
    grad[g0 + 2] = -np.sum(np.where(on, dyn, 0.0))
    grad[g0 + 3] = np.deg2rad(np.sum(np.where(on, dphi, 0.0)))
    grad[g0 + 4] = np.deg2rad(np.sum(np.where(on, di, 0.0)))
    return chi2, grad, dscale


def dcube_pipeline(packed, size, step, rpix, rval, scale, psf, lsf, precision='f64',
                   mask_cutoff=None, mask_apply=False, thick=False, image=False,
                   opacity_packed=None, fft_f32=False):
    """The reference's DCube chain with supersampling and masking
    (_dcube.py:128-313): the padded high-resolution grid (size x scale +
    kernel - 1, padded by backend.py:51-66), smdisk on it, FFT convolution
    with the rolled PSF x LSF cube sampled at the high-resolution step, the
    downscale of the crop (dmodels.hpp:8-46, host/kernels.hpp:55-80) and the
    mask (dmodels.hpp:49-74).  psf/lsf are gbkfit_b200.psflsf objects (their
    arrays are pinned to the reference's by the golden fixtures).

    image: the disk is evaluated into the spatial image instead of the
    spectral cube (the intensity gmodels, intensity_2d/3d.py; size z is 1).
    opacity_packed: an opacity disk evaluated first into the 3-D spatial
    opacity cube (its density output), which the disk then reads
    (intensity_3d.py:154-167, gmodels.hpp:933-937).  fft_f32: the FFT in
    single precision (as FFTW's float plans of the reference driver) instead
    of float64.  Returns (dcube_lo, mcube_lo or None)."""
    from gbkfit_b200.workloads import dcube_geometry
    o = Oracle(precision)
    real = o.real
    zero, size_hi, step_hi, zero_hi, edge, ksize = dcube_geometry(size, step, rpix, rval, scale,
                                                                  psf, lsf)
    sx, sy, sz = size_hi
    if thick:
        i = int(sx < sy)
        spat = ((sx, sy, (sx, sy)[i]), (step_hi[0], step_hi[1], step_hi[i]),
                (zero_hi[0], zero_hi[1], -((sx, sy)[i] / 2 - 0.5) * step_hi[i]))
    else:
        spat = ((sx, sy, 1), (step_hi[0], step_hi[1], 0.0), (zero_hi[0], zero_hi[1], 0.0))
    g = dict(loose=False, tilted=False, spat_size=spat[0], spat_step=spat[1],
             spat_zero=spat[2], spec_size=sz, spec_step=step_hi[2], spec_zero=zero_hi[2],
             opacity=None)
    if opacity_packed is not None:
        op = np.zeros(tuple(spat[0])[::-1], real)
        o.smdisk_evaluate(opacity_packed, g, dict(rdata=op))
        g['opacity'] = op
    cube = np.zeros((sz, sy, sx), real)
    if image:
        g['spec_size'], g['spec_step'], g['spec_zero'] = 1, 0.0, 0.0
        o.smdisk_evaluate(packed, g, dict(image=cube[0]))
    else:
        o.smdisk_evaluate(packed, g, dict(scube=cube))
    if psf is not None or lsf is not None:
        from gbkfit_b200 import psflsf as P
        off = [(n % 2) - 1 for n in size_hi]
        p = (psf or P.PSFPoint()).asarray(step_hi[:2], (sx, sy), (off[0], off[1]))
        l_ = (lsf or P.LSFPoint()).asarray(step_hi[2], sz, off[2])
        pc = (p * l_[:, None, None]).astype(real)
        pc = np.roll(pc, np.array(pc.shape) // 2 + 1, axis=(0, 1, 2))
        cube = fft_convolve_cached(cube, pc, dtype=np.float32 if fft_f32 else np.float64)
        cube = cube.astype(real)
    nx, ny, nz = size
    lo = o.dcube_downscale(scale, edge, cube, (nz, ny, nx))
    mcube = None
    if mask_cutoff is not None:
        lo, mcube = o.dcube_mask(mask_cutoff, mask_apply, lo)
    return lo, mcube
