"""Differentiable chi^2 of a thin smooth disk with node-wise surface
brightness, rotation curve and dispersion, with a hand-written adjoint.

No reference counterpart: GBKFIT computes no gradients.  The forward pass is
the drop-in path (smdisk_evaluate on the padded DCube grid, gmodels.hpp
:645-958; fft_convolve_cached, fft.hpp:98-125; crop; residual and sum of
squares, objective.hpp:7-31) with a multiplicative ``scale`` on the convolved
model.  The backward pass (include/gbkb200.h):

1. ``gbkb200_objective_chi2_adjoint_f32`` gives chi^2, d(chi^2)/d(scale) and
   g = d(chi^2)/d(convolved cube) on the padded grid, in one pass;
2. the drop-in FFT convolves g with the point-reflected PSF x LSF cube (the
   adjoint of the circular convolution): G = d(chi^2)/d(model cube);
3. ``gbkb200_gmodel_smdisk_nw_adjoint_f32`` recomputes every spaxel's ring
   position, interpolation weights and line and chains G to the sub-node
   values and the geometry; the sub-node gradients are mapped to the node
   parameters through the Jacobian of the node -> sub-node interpolation
   (_disk.py:107-125).

Parameter vector (``SMDiskChi2.names``): vsys, xpos, ypos, posa, incl, the
node values of the density, rotation and dispersion traits, then scale.
"""

import ctypes

import numpy as np
import torch

from . import _native
from ._native import c_float, c_int, c_void_p, check
from .disk import KINDS, _interp
from .driver import _disk_call_args

c_int3 = c_int * 3
_lib = _native.lib()


class NwDesc(ctypes.Structure):
    """gbkb200_smdisk_nw_desc (include/gbkb200.h)."""
    _fields_ = [
        ('spat_size', c_int * 2), ('spat_step', c_float * 2), ('spat_zero', c_float * 2),
        ('spec_size', c_int), ('spec_step', c_float), ('spec_zero', c_float),
        ('nsub', c_int), ('subrnodes', c_void_p), ('vsys', c_void_p),
        ('xpos', c_void_p), ('ypos', c_void_p), ('posa', c_void_p), ('incl', c_void_p),
        ('bsub', c_void_p), ('vsub', c_void_p), ('dsub', c_void_p),
    ]


_lib.gbkb200_objective_chi2_adjoint_f32.argtypes = [
    c_void_p, c_int3, c_int3, c_int3, c_void_p, c_void_p, c_void_p, c_void_p, c_float, c_float,
    c_void_p, c_void_p]
_lib.gbkb200_objective_chi2_adjoint_f32.restype = c_int
_lib.gbkb200_gmodel_smdisk_nw_adjoint_f32.argtypes = [c_void_p, ctypes.POINTER(NwDesc), c_void_p,
                                                      c_void_p]
_lib.gbkb200_gmodel_smdisk_nw_adjoint_f32.restype = c_int

ADJOINT_EXPORTED = ['gbkb200_objective_chi2_adjoint_f32', 'gbkb200_gmodel_smdisk_nw_adjoint_f32']

GEOMETRY = ('vsys', 'xpos', 'ypos', 'posa', 'incl')
# supported traits: (kind, trait name, node-wise parameter)
NW_TRAITS = (('rpt', 'nw_uniform', 'bpt_a'), ('vpt', 'nw_tan_uniform', 'vpt_vt'),
             ('dpt', 'nw_uniform', 'dpt_a'))


def _ptr(t):
    return None if t is None else t.data_ptr()


def param_names(disk):
    """Names of the parameter vector: geometry, node values per trait, scale."""
    nn = len(disk.rnodes)
    return list(GEOMETRY) + [f'{p}[{i}]' for _, _, p in NW_TRAITS for i in range(nn)] + ['scale']


def to_vector(params, scale=1.0):
    """Disk parameter dict (+ scale) -> parameter vector."""
    out = [float(params[n]) for n in GEOMETRY]
    for _, _, pname in NW_TRAITS:
        out += list(np.asarray(params[pname], np.float64))
    return np.asarray(out + [float(scale)])


def from_vector(disk, theta):
    """Parameter vector -> (Disk parameter dict, scale)."""
    nn = len(disk.rnodes)
    th = np.asarray(theta, np.float64).ravel()
    if th.size != 5 + 3 * nn + 1:
        raise ValueError(f"expected {5 + 3 * nn + 1} parameters, got {th.size}")
    p = {n: float(th[i]) for i, n in enumerate(GEOMETRY)}
    for j, (_, _, pname) in enumerate(NW_TRAITS):
        p[pname] = th[5 + j * nn:5 + (j + 1) * nn].copy()
    return p, float(th[-1])


def interpolation_jacobian(disk):
    """J (nnodes, nsub): d(sub-node values)/d(node values) of the disk's
    node -> sub-node interpolation (linear in the node values)."""
    n = len(disk.rnodes)
    return np.asarray(_interp(disk.interp, disk.rnodes, np.eye(n), disk.subrnodes), np.float64)


def assemble_gradient(jac, gsub, dscale):
    """Sub-node and geometry gradient (the adjoint kernel's layout) + the
    scale derivative -> gradient of the parameter vector."""
    ns = jac.shape[1]
    g = list(gsub[3 * ns:3 * ns + 5])
    for j in range(3):
        g += list(jac @ gsub[j * ns:(j + 1) * ns])
    return np.asarray(g + [float(dscale)])


class SMDiskChi2:
    """chi^2(theta) of one thin disk against one data cube, and its gradient.

    disk: gbkfit_b200.disk.Disk with exactly one node-wise density trait
    (bpt nw_uniform), rotation curve (vpt nw_tan_uniform) and dispersion
    (dpt nw_uniform), neither loose nor tilted; geom: workloads.Geometry;
    data/error/mask: (nz, ny, nx) arrays."""

    def __init__(self, disk, geom, data, error=None, mask=None, weight=1.0, device=0):
        if disk.loose or disk.tilted:
            raise ValueError("the adjoint supports flat (neither loose nor tilted) disks")
        for kind in KINDS:
            want = [t for t in NW_TRAITS if t[0] == kind]
            have = disk.traits.get(kind) or []
            if want:
                if len(have) != 1 or have[0].name != want[0][1]:
                    raise ValueError(f"the adjoint needs one {want[0][1]} trait of kind {kind}")
            elif have:
                raise ValueError(f"the adjoint does not support {kind} traits")
        self.disk, self.geom = disk, geom
        self.dev = torch.device('cuda', device)
        self.stream = torch.cuda.current_stream(self.dev)
        self.ctx = _native.Context(device=device, stream=self.stream, sync=False)
        f32 = lambda a: None if a is None else torch.as_tensor(
            np.ascontiguousarray(a, np.float32)).to(self.dev)
        self.obs, self.err, self.msk = f32(data), f32(error), f32(mask)
        self.weight = float(weight)
        self.size_hi = tuple(geom.size_hi)
        px, py, pz = self.size_hi
        self.scube = torch.zeros((pz, py, px), device=self.dev)
        self.gcube = torch.zeros((pz, py, px), device=self.dev)
        pc = geom.pcube(np.float32)
        self.pcube = f32(pc)
        # adjoint of the circular convolution: convolution with k(-i mod P)
        self.pcube_adj = f32(np.roll(pc[::-1, ::-1, ::-1], 1, axis=(0, 1, 2)))
        self.out2 = torch.zeros(2, dtype=torch.float64, device=self.dev)
        self.nsub = len(disk.subrnodes)
        self.gsub = torch.zeros(3 * self.nsub + 5, dtype=torch.float64, device=self.dev)
        self.jac = interpolation_jacobian(disk)
        self.names = param_names(disk)
        self.nnodes = len(disk.rnodes)
        self._theta = None
        self._keep = None

    # ---- parameters ----------------------------------------------------------
    def params(self, theta):
        """Parameter vector -> (Disk parameter dict, scale)."""
        return from_vector(self.disk, theta)

    def vector(self, params, scale=1.0):
        """Disk parameter dict (+ scale) -> parameter vector."""
        return to_vector(params, scale)

    # ---- passes --------------------------------------------------------------
    def _forward(self, theta):
        p, scale = self.params(theta)
        packed = self.disk.pack(p)
        dev = {}
        for k, v in packed.items():
            if v is None:
                dev[k] = None
            elif isinstance(v, dict):
                dev[k] = {f: torch.from_numpy(np.ascontiguousarray(a)).to(self.dev)
                          for f, a in v.items()}
            else:
                dev[k] = torch.from_numpy(np.ascontiguousarray(v)).to(self.dev)
        self._keep = dev
        tr = {k: ((dev[k]['uids'], dev[k]['cvalues'], dev[k]['ccounts'], dev[k]['pvalues'],
                   dev[k]['pcounts']) if dev[k] is not None else (None,) * 5) for k in KINDS}
        ss, st, sz = self.geom.spat()
        nz, dz, z0 = self.geom.spec()
        outs = (None, self.scube) + (None,) * 8
        args = _disk_call_args(dev['subrnodes'], dev['vsys'], dev['xpos'], dev['ypos'],
                               dev['posa'], dev['incl'], tr, None, ss, st, sz, nz, dz, z0, outs)
        args = [_ptr(a) if isinstance(a, torch.Tensor) else a for a in args]
        with torch.cuda.stream(self.stream):
            self.scube.zero_()
        check(_lib.gbkb200_gmodel_smdisk_evaluate_f32(self.ctx.handle, 0, 0, *args),
              'smdisk_evaluate')
        shape = c_int3(*self.size_hi)
        check(_lib.gbkb200_fft_convolve_cached_f32(self.ctx.handle, shape, _ptr(self.scube),
                                                   _ptr(self.pcube)), 'fft_convolve_cached')
        check(_lib.gbkb200_objective_chi2_adjoint_f32(
            self.ctx.handle, shape, c_int3(*self.geom.edge), c_int3(*self.geom.size),
            _ptr(self.scube), _ptr(self.obs), _ptr(self.err), _ptr(self.msk), self.weight, scale,
            _ptr(self.gcube), _ptr(self.out2)), 'chi2_adjoint')
        self._theta = np.asarray(theta, np.float64).ravel().copy()

    def _backward(self):
        dev = self._keep
        check(_lib.gbkb200_fft_convolve_cached_f32(self.ctx.handle, c_int3(*self.size_hi),
                                                   _ptr(self.gcube), _ptr(self.pcube_adj)),
              'fft_convolve_cached (adjoint)')
        d = NwDesc()
        ss, st, sz = self.geom.spat()
        nz, dz, z0 = self.geom.spec()
        d.spat_size[:] = [ss[0], ss[1]]
        d.spat_step[:] = [st[0], st[1]]
        d.spat_zero[:] = [sz[0], sz[1]]
        d.spec_size, d.spec_step, d.spec_zero = nz, dz, z0
        d.nsub = self.nsub
        d.subrnodes = _ptr(dev['subrnodes'])
        d.vsys, d.xpos, d.ypos = _ptr(dev['vsys']), _ptr(dev['xpos']), _ptr(dev['ypos'])
        d.posa, d.incl = _ptr(dev['posa']), _ptr(dev['incl'])
        d.bsub, d.vsub, d.dsub = (_ptr(dev['rpt']['pvalues']), _ptr(dev['vpt']['pvalues']),
                                  _ptr(dev['dpt']['pvalues']))
        check(_lib.gbkb200_gmodel_smdisk_nw_adjoint_f32(self.ctx.handle, ctypes.byref(d),
                                                        _ptr(self.gcube), _ptr(self.gsub)),
              'smdisk_nw_adjoint')

    def _assemble(self, out2, gsub):
        return assemble_gradient(self.jac, gsub, out2[1])

    # ---- public --------------------------------------------------------------
    def value(self, theta):
        """chi^2 at theta (synchronises)."""
        self._forward(theta)
        self.stream.synchronize()
        return float(self.out2[0].item())

    def value_and_grad(self, theta):
        """(chi^2, d chi^2 / d theta) at theta (synchronises)."""
        self._forward(theta)
        self._backward()
        self.stream.synchronize()
        out2 = self.out2.cpu().numpy()
        return float(out2[0]), self._assemble(out2, self.gsub.cpu().numpy())

    def grad_after_forward(self, theta):
        """The gradient at theta, reusing the residual adjoint of the last
        forward pass when it was taken at the same theta."""
        th = np.asarray(theta, np.float64).ravel()
        if self._theta is None or not np.array_equal(th, self._theta):
            self._forward(th)
        self._backward()
        self.stream.synchronize()
        out2 = self.out2.cpu().numpy()
        return self._assemble(out2, self.gsub.cpu().numpy())


class SMDiskChi2Function(torch.autograd.Function):
    """chi^2 = SMDiskChi2Function.apply(theta, model): differentiable in theta
    (a 1-D tensor ordered as model.names); the backward pass runs the
    hand-written adjoint on the GPU."""

    @staticmethod
    def forward(ctx, theta, model):
        th = theta.detach().to('cpu', torch.float64).numpy().copy()
        chi2 = model.value(th)
        ctx.model = model
        ctx.th = th
        return torch.tensor(chi2, dtype=theta.dtype, device=theta.device)

    @staticmethod
    def backward(ctx, grad_out):
        g = ctx.model.grad_after_forward(ctx.th)
        gt = torch.as_tensor(g, dtype=grad_out.dtype, device=grad_out.device)
        return grad_out * gt, None
