"""Host packing, PSF/LSF and the oracle against fixtures produced by the
reference itself (tests/golden/make_golden.py): the arrays the reference's
Disk.evaluate hands to its native module, the reference's PSF/LSF arrays and
the outputs of the reference's compiled templates."""

import os

import numpy as np
import pytest

from tests.helpers import rel_err

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


def _load(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def _cases():
    from gbkfit_b200 import traits as T
    rn = np.linspace(0, 30, 20)
    base = dict(xpos=16.3, ypos=14.1, posa=45.0, incl=60.0, vsys=3.0)
    return [
        ('thin_exp_arctan', dict(rpt=[T.bpt('exponential')], vpt=[T.vpt('tan_arctan')],
                                 dpt=[T.dpt('uniform')]),
         dict(base, bpt_a=1.0, bpt_s=8.0, vpt_rt=4.0, vpt_vt=200.0, dpt_a=20.0), False, False),
        ('thin_nodewise', dict(rpt=[T.bpt('nw_uniform')], vpt=[T.vpt('nw_tan_uniform')],
                               dpt=[T.dpt('nw_uniform')]),
         dict(base, bpt_a=np.exp(-rn / 9), vpt_vt=220 * np.tanh(rn / 5), dpt_a=15 + rn / 3),
         False, False),
        ('thin_two_traits_harmonic_sel',
         dict(rpt=[T.bpt('exponential'), T.bpt('nw_harmonic', order=2)],
              vpt=[T.vpt('tan_tanh'), T.vpt('nw_rad_uniform')], dpt=[T.dpt('gauss')],
              spt=[T.spt('azrange')]),
         dict(base, bpt_a=1.0, bpt_s=6.0, bpt1_a=0.2 * np.ones(20), bpt1_p=np.linspace(0, 90, 20),
              vpt_rt=3.0, vpt_vt=180.0, vpt1_vr=np.linspace(0, 20, 20), dpt_a=30.0,
              dpt_s=10.0, spt_p=30.0, spt_s=300.0), False, False),
        ('loose_tilted', dict(rpt=[T.bpt('exponential')], vpt=[T.vpt('tan_arctan')],
                              dpt=[T.dpt('uniform')]),
         dict(vsys=np.linspace(0, 5, 20), xpos=16.0 + np.linspace(0, 1, 20),
              ypos=14.0 - np.linspace(0, 1, 20), posa=40 + np.linspace(0, 10, 20),
              incl=55 + np.linspace(0, 10, 20), bpt_a=1.0, bpt_s=8.0, vpt_rt=4.0,
              vpt_vt=200.0, dpt_a=20.0), True, True),
        ('thick_sech2', dict(rpt=[T.bpt('exponential')], rht=[T.bht('sech2', trunc=0)],
                             vpt=[T.vpt('tan_lramp')], vht=[T.vht_one()],
                             dpt=[T.dpt('uniform')], dht=[T.dht_one()]),
         dict(base, bpt_a=1.0, bpt_s=8.0, bht_s=1.5, vpt_rt=5.0, vpt_vt=200.0, dpt_a=15.0),
         False, False),
        ('thick_gauss_trunc_nw', dict(rpt=[T.bpt('gauss')],
                                      rht=[T.bht('gauss', rnodes=True, trunc=2.0)],
                                      vpt=[T.vpt('tan_arctan')], vht=[T.vht_one()],
                                      dpt=[T.dpt('exponential')], dht=[T.dht_one()]),
         dict(base, bpt_a=1.0, bpt_s=12.0, bht_s=1 + rn / 20, vpt_rt=4.0, vpt_vt=210.0,
              dpt_a=25.0, dpt_s=30.0), False, False),
    ]


def _disk(traits, loose, tilted):
    from gbkfit_b200.disk import Disk
    return Disk(loose, tilted, np.linspace(0, 30, 20), traits=traits)


@pytest.mark.parametrize('case', [c[0] for c in _cases()])
def test_packing_matches_reference(case):
    """gbkfit_b200.disk packing == the arrays of the reference's Disk.evaluate."""
    g = _load('packing.npz')
    name, traits, params, loose, tilted = [c for c in _cases() if c[0] == case][0]
    p = _disk(traits, loose, tilted).pack(params)
    ref = {k.split('/', 1)[1]: v for k, v in g.items() if k.startswith(name + '/')}
    assert np.array_equal(p['subrnodes'], ref['rnodes'].astype(np.float32))
    for n in ('vsys', 'xpos', 'ypos', 'posa', 'incl'):
        assert np.allclose(p[n], ref[n], rtol=1e-7, atol=0), n
    for k in ('rpt', 'rht', 'vpt', 'vht', 'dpt', 'dht', 'zpt', 'spt', 'wpt'):
        if f'{k}_uids' not in ref:
            assert p[k] is None, k
            continue
        for f in ('uids', 'ccounts', 'pcounts'):
            assert np.array_equal(p[k][f], ref[f'{k}_{f}']), (k, f)
        assert np.allclose(p[k]['cvalues'], ref[f'{k}_cvalues']), k
        assert np.allclose(p[k]['pvalues'], ref[f'{k}_pvalues'], rtol=2e-7, atol=1e-12), k


def test_mcdisk_cloud_budget_matches_reference():
    """_mcdisk.py:180-216: cumulative cloud counts and analytic-integral flags."""
    g = _load('packing.npz')
    name, traits, params, loose, tilted = _cases()[4]
    d = _disk(traits, loose, tilted)
    pre = 'mc_' + name + '/'
    assert np.array_equal(d.ncloudscsum(params, float(g[pre + 'cflux'])), g[pre + 'ncloudscsum'])
    assert np.array_equal(d.hasordint(), g[pre + 'hasordint'])


def test_psflsf_match_reference():
    from gbkfit_b200 import psflsf as P
    g = _load('psflsf.npz')
    psfs = dict(gauss=P.PSFGauss(1.5), moffat=P.PSFMoffat(1.2, 2.5), lorentz=P.PSFLorentz(0.8),
                ggauss=P.PSFGGauss(1.5, 1.5), gauss_ell=P.PSFGauss(1.0, ratio=0.6, posa=30.0))
    for k, o in psfs.items():
        assert np.allclose(o.asarray((0.5, 0.4)), g[f'psf_{k}'], rtol=1e-12, atol=1e-15), k
        assert np.allclose(o.asarray((1.0, 1.0), (24, 20), (-1, -1)), g[f'psf_{k}_padded'],
                           rtol=1e-12, atol=1e-15), k
    lsfs = dict(gauss=P.LSFGauss(5.0), moffat=P.LSFMoffat(5.0, 2.5), lorentz=P.LSFLorentz(3.0),
                ggauss=P.LSFGGauss(5.0, 1.5))
    for k, o in lsfs.items():
        assert np.allclose(o.asarray(0.5), g[f'lsf_{k}'], rtol=1e-12, atol=1e-15), k
        assert np.allclose(o.asarray(2.0, 32, -1), g[f'lsf_{k}_padded'], rtol=1e-12,
                           atol=1e-15), k


def test_psflsf_reference_test_pins():
    """tests/unit/test_psflsf.py:13-86 of the reference: unit sum (1e-9), odd
    sizes, peak at the centre, for its parameters."""
    from gbkfit_b200 import psflsf as P
    for psf in (P.PSFPoint(), P.PSFGauss(5.0), P.PSFGGauss(5.0, 1.0), P.PSFLorentz(5.0),
                P.PSFMoffat(5.0, 1.0)):
        a = psf.asarray((0.5, 0.2))
        size = psf.size((0.5, 0.2))
        assert a.shape[::-1] == size
        assert size[0] % 2 == 1 and size[1] % 2 == 1
        assert abs(a.sum() - 1) < 1e-9
        peak = np.unravel_index(np.argmax(a), a.shape)[::-1]
        assert peak == (size[0] // 2, size[1] // 2)
    for lsf in (P.LSFPoint(), P.LSFGauss(5.0), P.LSFGGauss(5.0, 1.0), P.LSFLorentz(5.0),
                P.LSFMoffat(5.0, 1.0)):
        a = lsf.asarray(0.5)
        assert a.shape[0] == lsf.size(0.5) and a.shape[0] % 2 == 1
        assert abs(a.sum() - 1) < 1e-9
        assert int(np.argmax(a)) == a.shape[0] // 2


_GEOMS = dict(
    thin=dict(spat_size=(36, 32, 1), spat_step=(1, 1, 0), spat_zero=(-2.0, -1.5, 0),
              spec_size=40, spec_step=10.0, spec_zero=-200.0),
    thick=dict(spat_size=(32, 30, 20), spat_step=(1, 1, 1), spat_zero=(0.0, -0.5, -9.5),
               spec_size=40, spec_step=10.0, spec_zero=-200.0))


@pytest.mark.parametrize('precision', ['f32', 'f64'])
@pytest.mark.parametrize('case', [c[0] for c in _cases()])
def test_oracle_smdisk_matches_reference_outputs(oracle_built, case, precision):
    """The oracle restatement reproduces the reference's compiled templates
    (f32: <= a few ulp, normwise; f64: the fp32 rounding of the reference)."""
    from oracle.oracle import Oracle
    cubes = _load('cubes.npz')
    name, traits, params, loose, tilted = [c for c in _cases() if c[0] == case][0]
    thick = name.startswith('thick')
    geo = dict(_GEOMS['thick' if thick else 'thin'], loose=loose, tilted=tilted, opacity=None)
    packed = _disk(traits, loose, tilted).pack(params)
    o = Oracle(precision)
    sx, sy, sz = geo['spat_size']
    outs = dict(scube=o.zeros((geo['spec_size'], sy, sx)), rdata=o.zeros((sz, sy, sx)),
                vdata_cmp=np.full((sz, sy, sx), np.nan, o.real),
                ddata_cmp=np.full((sz, sy, sx), np.nan, o.real))
    assert o.smdisk_evaluate(packed, geo, outs) == 0
    tol = 1e-5 if precision == 'f32' else 5e-5
    ref = cubes[f'{name}/scube']
    assert ref.max() > 0
    assert rel_err(outs['scube'], ref) < tol
    assert rel_err(outs['rdata'], cubes[f'{name}/rdata']) < tol
    m = np.isfinite(cubes[f'{name}/vdata_cmp'])
    assert np.array_equal(m, np.isfinite(outs['vdata_cmp']))
    assert rel_err(outs['vdata_cmp'][m], cubes[f'{name}/vdata_cmp'][m]) < tol


def test_oracle_dmodel_objective_match_reference(oracle_built):
    from oracle.oracle import Oracle
    c = _load('cubes.npz')
    o = Oracle('f32')
    md, mm, mw = o.mmaps_moments((36, 32, 40), (1.0, 1.0, 10.0), (0.0, 0.0, -200.0),
                                 c['thin_exp_arctan/scube'], c['moments/wcube'], 1e-6,
                                 c['moments/orders'])
    assert np.array_equal(mm, c['moments/m'])
    v = mm > 0
    for i in range(len(c['moments/orders'])):
        assert rel_err(md[i][v], c['moments/d'][i][v]) < 1e-5, i
    assert rel_err(mw[v], c['moments/w'][v]) < 1e-5
    res = o.residual(c['residual/od'], c['residual/oe'], c['residual/om'], c['residual/md'],
                     None, None, 0.8)
    assert np.array_equal(res, c['residual/res'])
    assert abs(o.residual_sum(res, True) - c['residual/sum_sq']) < 1e-5 * c['residual/sum_sq']
    assert abs(o.residual_sum(res, False) - c['residual/sum_abs']) < 1e-5 * c['residual/sum_abs']
    dst = o.dcube_downscale((2, 3, 2), (1, 2, 3), c['downscale/src'], (8, 5, 10))
    assert rel_err(dst, c['downscale/dst']) < 1e-6
    d, m = o.dcube_mask(0.6, True, c['downscale/src'])
    assert np.array_equal(m, c['mask/m'])
    assert np.array_equal(np.isnan(d), np.isnan(c['mask/d']))
    assert np.array_equal(o.wcube_evaluate(c['wcube/spat'], 11), c['wcube/spec'])
    assert rel_err(o.convolve(c['convolve/a'], c['convolve/k']), c['convolve/out']) < 1e-6


def test_fft_standin_matches_reference_direct_convolution():
    """The float64 FFT standing in for FFTW reproduces the reference's direct
    convolution (gmodels.hpp:9-50) once the cube is zero-padded by the kernel
    size and the kernel is rolled to the origin, as DCube does.  The direct
    form indexes data1[x - K/2 + x2] * data2[x2], a correlation: the FFT path
    gets the kernel flipped (the two agree for the symmetric PSF x LSF)."""
    from oracle.oracle import fft_convolve_cached
    c = _load('cubes.npz')
    a, k = c['convolve/a'], c['convolve/k']
    nz, ny, nx = a.shape
    kz, ky, kx = k.shape
    pad = np.zeros((nz + kz - 1, ny + ky - 1, nx + kx - 1))
    pad[:nz, :ny, :nx] = a
    kern = np.zeros_like(pad)
    kern[:kz, :ky, :kx] = k[::-1, ::-1, ::-1]
    kern = np.roll(kern, (-(kz // 2), -(ky // 2), -(kx // 2)), axis=(0, 1, 2))
    out = fft_convolve_cached(pad, kern)[:nz, :ny, :nx]
    assert rel_err(out, c['convolve/out']) < 1e-5


def test_philox_known_answers(oracle_built):
    """Philox-4x32-10 known-answer vectors of Salmon et al. (Random123)."""
    from oracle.oracle import Oracle
    o = Oracle('f32')
    assert o.philox([0, 0, 0, 0], 0, 0) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert o.philox([0xffffffff] * 4, 0xffffffff, 0xffffffff) == \
        [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert o.philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], 0xa4093822, 0x299f31d0) == \
        [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def test_oracle_matches_compiled_reference_on_cube64(oracle_built):
    """Where oracle/_ref was built: oracle vs the compiled reference on the
    64^3 smdisk workload."""
    from oracle.oracle import Oracle, Reference
    from gbkfit_b200 import workloads
    if not Reference.available():
        pytest.skip('oracle/_ref not built')
    w = workloads.smdisk_cube64()
    g = w.geometry_args()
    nx, ny, nz = g['spat_size'][0], g['spat_size'][1], g['spec_size']
    p = w.disk.pack(w.params)
    a = np.zeros((nz, ny, nx), np.float32)
    b = np.zeros((nz, ny, nx), np.float32)
    Oracle('f32').smdisk_evaluate(p, g, dict(scube=a))
    Reference().smdisk_evaluate(p, g, dict(scube=b))
    assert rel_err(a, b) < 1e-6
