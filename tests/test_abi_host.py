"""CPU tests of the boundary and the host logic: the C ABI library loads and
exports every function declared in include/gbkb200.h; DCube geometry, padding
and packing rules; parameter validation."""

import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    with open(os.path.join(ROOT, 'include', 'gbkb200.h')) as f:
        text = f.read()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'\b(gbkb200_\w+)\s*\(', text)))


def test_library_exports_every_declared_symbol():
    from gbkfit_b200 import build
    build.build()
    import ctypes
    lib = ctypes.CDLL(build.OUT)
    names = _declared()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_native_binding_loads_and_binds():
    from gbkfit_b200 import _native
    for n in _native.EXPORTED:
        assert hasattr(_native.lib(), n)
    assert _native.lib().gbkb200_error_string(4) == b'unknown trait uid'


def test_fft_optimal_shape_matches_reference_rule():
    """driver/backend.py:51-59: po2 up to 32, else the next multiple of 32."""
    from gbkfit_b200.workloads import fft_optimal_shape
    assert fft_optimal_shape([1, 2, 3, 17, 32, 33, 80, 96, 148, 290]) == \
        (1, 2, 4, 32, 32, 64, 96, 96, 160, 320)


def test_fft_index_division_multipliers_are_exact():
    """The FFT passes divide thread indices (< 2^24) by run-time lengths
    (<= 2^16) as (x * ceil(2^40 / d)) >> 40: exact on the whole range, checked
    at every divisor on the last multiple below 2^24 minus one, the largest
    index and a random sample."""
    d = np.arange(1, (1 << 16) + 1, dtype=np.uint64)
    m = ((np.uint64(1) << np.uint64(40)) + d - np.uint64(1)) // d
    top = np.uint64((1 << 24) - 1)
    rng = np.random.default_rng(0)
    cols = [(top // d) * d - np.uint64(1), np.full_like(d, top), (top // d) * d,
            np.ones_like(d), np.zeros_like(d)]
    cols += [rng.integers(0, 1 << 24, d.size).astype(np.uint64) for _ in range(64)]
    for x in cols:
        assert np.array_equal((x * m) >> np.uint64(40), x // d)


def test_dcube_geometry_reference_pins():
    """tests/unit/test_dmodel.py:102-170 of the reference: scratch size, step
    and zero of a DCube without PSF/LSF."""
    from gbkfit_b200.workloads import dcube_geometry
    size, step = (21, 30, 41), (0.5, 1.5, 2.0)
    rpix, rval, scale = (5.0, 6.5, 7.5), (1.0, 1.5, 2.0), (1, 2, 3)
    zero, size_hi, step_hi, zero_hi, edge, _ = dcube_geometry(size, step, rpix, rval, scale,
                                                              None, None)
    assert zero == tuple(rval[i] - rpix[i] * step[i] for i in range(3))
    assert size_hi == (21, 60, 123)
    assert step_hi == (0.5, 0.75, 2.0 / 3)
    assert edge == (0, 0, 0)
    assert zero_hi == tuple(zero[i] - step[i] / 2 - (0 - 0.5) * step_hi[i] for i in range(3))


def test_dcube_geometry_with_psf_lsf():
    """_dcube.py:158-179 for the 64^3 workload: kernel (17, 17, 15), padded
    grid 96^3, edge (8, 8, 7)."""
    from gbkfit_b200 import workloads
    g = workloads.smdisk_cube64().geom
    assert g.kernel_size == (17, 17, 15)
    assert g.size_hi == (96, 96, 96)
    assert g.edge == (8, 8, 7)
    assert np.allclose(g.zero_hi, (-8.0, -8.0, -385.0))
    pc = g.pcube()
    assert pc.shape == (96, 96, 96)
    assert abs(pc.sum() - 1) < 1e-5
    assert np.unravel_index(np.argmax(pc), pc.shape) == (0, 0, 0)


def test_subrnodes_rule():
    """_disk.py:151-154."""
    from gbkfit_b200.disk import make_subrnodes, default_rstep
    rn = np.linspace(0, 30, 20)
    h = default_rstep(rn)
    s = make_subrnodes(rn, h)
    assert s[0] == 0 and np.isclose(s[1], h / 2) and np.isclose(s[-1], s[-2] + h / 2)
    assert np.allclose(np.diff(s[1:-1]), h)


def test_disk_validation():
    from gbkfit_b200 import traits as T
    from gbkfit_b200.disk import Disk
    with pytest.raises(RuntimeError):
        Disk(False, False, [0.0])
    with pytest.raises(RuntimeError):
        Disk(False, False, [0.0, 2.0, 1.0])
    with pytest.raises(RuntimeError):
        Disk(False, False, [0.0, 1.0], rstep=0.8)
    with pytest.raises(RuntimeError):
        Disk(False, False, [0.0, 1.0, 2.0], traits=dict(rpt=[T.bpt('exponential')] * 5))


def test_pack_batch_equals_pack():
    """Disk.pack_batch row i == Disk.pack of parameter set i."""
    from gbkfit_b200 import workloads
    w = workloads.smdisk_batch128(nsets=5)
    pb = w.disk.pack_batch(w.params, 5)
    for i in range(5):
        p = w.disk.pack(workloads.set_params(w, i))
        for n in ('xpos', 'ypos', 'posa', 'incl', 'vsys'):
            assert np.allclose(pb[n][i], p[n]), n
        for k in ('rpt', 'vpt', 'dpt'):
            assert np.allclose(pb[k]['pvalues'][i], p[k]['pvalues'], rtol=1e-6), k


def test_shard_sets_partition():
    from gbkfit_b200.batched import shard_sets
    for n in (0, 1, 7, 512, 513):
        for world in (1, 2, 3, 8):
            parts = [shard_sets(n, r, world) for r in range(world)]
            idx = np.concatenate([np.arange(a, b) for a, b in parts])
            assert np.array_equal(idx, np.arange(n))


def test_adjoint_parameter_layout_and_interpolation_jacobian():
    """The differentiable configuration has 66 parameters; the node -> sub-node
    Jacobian reproduces the packed sub-node values (_disk.py:107-125)."""
    from gbkfit_b200 import workloads
    from gbkfit_b200.adjoint import NW_TRAITS, interpolation_jacobian
    w = workloads.smdisk_grad96()
    nn = len(w.disk.rnodes)
    assert 5 + 3 * nn + 1 == 66
    jac = interpolation_jacobian(w.disk)
    assert jac.shape == (nn, w.disk.nsub)
    packed = w.disk.pack(w.params)
    for kind, _, pname in NW_TRAITS:
        sub = np.asarray(w.params[pname], np.float64) @ jac
        assert np.allclose(sub, packed[kind]['pvalues'], rtol=1e-6, atol=1e-6)
    assert w.extra['truth']['bpt_a'][-1] == 0.0     # tapered edge


def test_adjoint_rejects_unsupported_disks():
    import pytest
    from gbkfit_b200 import traits
    from gbkfit_b200.adjoint import SMDiskChi2
    from gbkfit_b200.disk import Disk
    from gbkfit_b200 import workloads
    g = workloads.smdisk_grad96().geom
    rn = np.linspace(0, 10, 5)
    bad = [
        Disk(False, False, rn, traits=dict(rpt=[traits.bpt('exponential')],
                                           vpt=[traits.vpt('nw_tan_uniform')],
                                           dpt=[traits.dpt('nw_uniform')])),
        Disk(True, False, rn, traits=dict(rpt=[traits.bpt('nw_uniform')],
                                          vpt=[traits.vpt('nw_tan_uniform')],
                                          dpt=[traits.dpt('nw_uniform')])),
        Disk(False, False, rn, traits=dict(rpt=[traits.bpt('nw_uniform')],
                                           vpt=[traits.vpt('nw_tan_uniform')],
                                           dpt=[traits.dpt('nw_uniform')],
                                           wpt=[traits.wpt_axis_range(0, 10, 1)])),
    ]
    for d in bad:
        with pytest.raises(ValueError):
            SMDiskChi2(d, g, np.zeros(g.size[::-1], np.float32))


def test_serve_args_layout_matches_header(tmp_path):
    """The ctypes mirror of gbkb200_serve_args has the C struct's size and
    field offsets (a C program built from the header prints them)."""
    import ctypes
    import subprocess
    from gbkfit_b200._native import ServeArgs
    names = [f[0] for f in ServeArgs._fields_]
    src = tmp_path / 'layout.c'
    body = '\n'.join(f'  printf("{n} %zu\\n", offsetof(gbkb200_serve_args, {n}));' for n in names)
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "gbkb200.h"\n'
                   'int main(void) {\n' + body +
                   '\n  printf("sizeof %zu\\n", sizeof(gbkb200_serve_args));\n  return 0;\n}\n')
    exe = tmp_path / 'layout'
    subprocess.run(['gcc', '-I', os.path.join(ROOT, 'include'), str(src), '-o', str(exe)],
                   check=True)
    got = dict(line.split() for line in subprocess.run(
        [str(exe)], check=True, capture_output=True, text=True).stdout.splitlines())
    assert int(got.pop('sizeof')) == ctypes.sizeof(ServeArgs)
    for n in names:
        assert int(got[n]) == getattr(ServeArgs, n).offset, n


def test_serve_entry_rejects_missing_arguments():
    """The per-request serving call checks its arguments before touching the
    device: no context or no argument block is an invalid-argument error."""
    import ctypes
    from gbkfit_b200 import _native
    lib = _native.lib()
    assert lib.gbkb200_serve_scube_chi2_f32(None, None) == 1
    a = _native.ServeArgs()
    assert lib.gbkb200_serve_scube_chi2_f32(None, ctypes.byref(a)) == 1


def test_imaging_model_parameter_names():
    """intensity_3d.py / gmodels/_detail.py:339-342 and utils/miscutils.py:
    70-95: brightness components keep their names (the second and later get
    'cmp<i>_'), opacity components are always prefixed ('ocmp_', 'ocmp1_')."""
    from gbkfit_b200 import traits as T
    from gbkfit_b200.imaging import (BrightnessSMDisk2D, BrightnessSMDisk3D, GModelIntensity2D,
                                     GModelIntensity3D, OpacitySMDisk3D, DModelImage,
                                     DModelLSlit)
    rn = np.linspace(0, 20, 6)
    b2 = [BrightnessSMDisk2D(False, False, T.bpt('exponential'), rnodes=rn) for _ in range(2)]
    assert set(GModelIntensity2D(b2).pdescs()) == {
        'xpos', 'ypos', 'posa', 'incl', 'bpt_a', 'bpt_s', 'cmp1_xpos', 'cmp1_ypos', 'cmp1_posa',
        'cmp1_incl', 'cmp1_bpt_a', 'cmp1_bpt_s'}
    b3 = BrightnessSMDisk3D(False, False, T.bpt('gauss'), T.bht('sech2'), rnodes=rn)
    o3 = [OpacitySMDisk3D(False, False, T.opt('exponential'), T.oht('sech2'), rnodes=rn)
          for _ in range(2)]
    names = set(GModelIntensity3D([b3], o3).pdescs())
    assert {'bpt_a', 'bht_s', 'ocmp_opt_a', 'ocmp_oht_a', 'ocmp1_opt_s', 'ocmp1_xpos'} <= names
    assert o3[0].disk().tables['rpt']['uids'][0] == T.OPT_OFFSET + T.RPT['exponential']
    assert DModelImage((30, 20)).size() == (30, 20) and DModelImage((30, 20)).keys() == ['image']
    assert DModelLSlit((30, 40)).size() == (30, 1, 40)


def test_mcdisk_scratch_copies_rule():
    """The fast mcdisk modes' line scratch: one channel-contiguous copy up to
    256 clouds per spaxel, 2/4/8 copies at 256/512/1024 and more, within
    64 MB of copies."""
    from gbkfit_b200 import _native
    f = _native.lib().gbkb200_mcdisk_scratch_bytes
    one = lambda sx, sy, nz: sx * sy * ((nz + 3) // 4 * 4) * 4
    assert f(100_000, 65, 68, 47) == one(65, 68, 47)
    assert f(10_000_000, 65, 68, 47) == 8 * one(65, 68, 47)
    assert f(10_000_000, 244, 262, 80) == one(244, 262, 80)          # 156 per spaxel
    assert f(3_000_000, 89, 142, 48) == one(89, 142, 48)              # 237 per spaxel
    assert f(5_000_000, 89, 142, 48) == 2 * one(89, 142, 48)          # 396
    assert f(2 ** 31 - 1, 320, 320, 160) == one(320, 320, 160)        # 62.5 MB: one copy fits
