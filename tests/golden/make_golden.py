"""Generates the golden fixtures of tests/golden from the REFERENCE itself.

Run from the repository root where a GBKFIT checkout exists:

    python tests/golden/make_golden.py [/path/to/gbkfit/src]

* packing.npz: the arrays the reference's own ``Disk.evaluate``
  (src/gbkfit/model/gmodels/_disk.py:466-613) hands to the native
  ``smdisk_evaluate`` / ``mcdisk_evaluate`` (captured through a recording
  driver), for several trait configurations;
* psflsf.npz: the reference's PSF/LSF arrays (src/gbkfit/psflsf);
* cubes.npz: outputs of the reference's compiled templates (oracle/_ref) on
  those packed arrays: smdisk cubes and maps, moments, residual and its sum,
  downscale, mask, wcube and the direct convolution.

Fixtures are small (cubes of a few tens of voxels per side).
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)


class RecordingDriver:
    """Host memory driver whose gmodel backend records its calls."""

    class _GModel:
        def __init__(self, log):
            self.log = log

        def smdisk_evaluate(self, *args):
            self.log.append(('smdisk', args))

        def mcdisk_evaluate(self, *args):
            self.log.append(('mcdisk', args))

    class _Backends:
        def __init__(self, log):
            self.log = log

        def gmodel(self, dtype):
            return RecordingDriver._GModel(self.log)

    def __init__(self):
        self.log = []

    def mem_alloc_s(self, shape, dtype):
        h = np.zeros(shape, dtype)
        return h, h.copy()

    def mem_alloc_h(self, shape, dtype):
        return np.zeros(shape, dtype)

    def mem_alloc_d(self, shape, dtype):
        return np.zeros(shape, dtype)

    def mem_copy_h2d(self, h, d=None):
        if d is None:
            return h.copy()
        d[...] = h
        return d

    def mem_copy_d2h(self, d, h=None):
        return d.copy() if h is None else d

    def mem_fill(self, x, v):
        x.fill(v)

    def backends(self):
        return RecordingDriver._Backends(self.log)


NAMES = ['loose', 'tilted', 'rnodes', 'vsys', 'xpos', 'ypos', 'posa', 'incl']
for k in ('rpt', 'rht', 'vpt', 'vht', 'dpt', 'dht', 'zpt', 'spt', 'wpt'):
    NAMES += [f'{k}_{f}' for f in ('uids', 'cvalues', 'ccounts', 'pvalues', 'pcounts')]


def cases(T):
    """(name, constructor kwargs of the disk, params) of the packing cases."""
    rn = list(np.linspace(0, 30, 20))
    base = dict(xpos=16.3, ypos=14.1, posa=45.0, incl=60.0, vsys=3.0)
    return [
        ('thin_exp_arctan', dict(rptraits=[T.BPTraitExponential()], rhtraits=[],
                                 vptraits=[T.VPTraitTanArctan()], vhtraits=[],
                                 dptraits=[T.DPTraitUniform()], dhtraits=[]), rn,
         dict(base, bpt_a=1.0, bpt_s=8.0, vpt_rt=4.0, vpt_vt=200.0, dpt_a=20.0), False, False),
        ('thin_nodewise', dict(rptraits=[T.BPTraitNWUniform()], rhtraits=[],
                               vptraits=[T.VPTraitNWTanUniform()], vhtraits=[],
                               dptraits=[T.DPTraitNWUniform()], dhtraits=[]), rn,
         dict(base, bpt_a=np.exp(-np.array(rn) / 9), vpt_vt=220 * np.tanh(np.array(rn) / 5),
              dpt_a=15 + np.array(rn) / 3), False, False),
        ('thin_two_traits_harmonic_sel', dict(
            rptraits=[T.BPTraitExponential(), T.BPTraitNWHarmonic(order=2)], rhtraits=[],
            vptraits=[T.VPTraitTanTanh(), T.VPTraitNWRadUniform()], vhtraits=[],
            dptraits=[T.DPTraitGauss()], dhtraits=[], sptraits=[T.SPTraitAzimuthalRange()]), rn,
         dict(base, bpt_a=1.0, bpt_s=6.0, bpt1_a=0.2 * np.ones(20), bpt1_p=np.linspace(0, 90, 20),
              vpt_rt=3.0, vpt_vt=180.0, vpt1_vr=np.linspace(0, 20, 20), dpt_a=30.0,
              dpt_s=10.0, spt_p=30.0, spt_s=300.0), False, False),
        ('loose_tilted', dict(rptraits=[T.BPTraitExponential()], rhtraits=[],
                              vptraits=[T.VPTraitTanArctan()], vhtraits=[],
                              dptraits=[T.DPTraitUniform()], dhtraits=[]), rn,
         dict(vsys=np.linspace(0, 5, 20), xpos=16.0 + np.linspace(0, 1, 20),
              ypos=14.0 - np.linspace(0, 1, 20), posa=40 + np.linspace(0, 10, 20),
              incl=55 + np.linspace(0, 10, 20), bpt_a=1.0, bpt_s=8.0, vpt_rt=4.0,
              vpt_vt=200.0, dpt_a=20.0), True, True),
        ('thick_sech2', dict(rptraits=[T.BPTraitExponential()],
                             rhtraits=[T.BHTraitSech2(trunc=0)],
                             vptraits=[T.VPTraitTanLRamp()], vhtraits=[T.VHTraitOne()],
                             dptraits=[T.DPTraitUniform()], dhtraits=[T.DHTraitOne()]), rn,
         dict(base, bpt_a=1.0, bpt_s=8.0, bht_s=1.5, vpt_rt=5.0, vpt_vt=200.0, dpt_a=15.0),
         False, False),
        ('thick_gauss_trunc_nw', dict(rptraits=[T.BPTraitGauss()],
                                      rhtraits=[T.BHTraitGauss(rnodes=True, trunc=2.0)],
                                      vptraits=[T.VPTraitTanArctan()], vhtraits=[T.VHTraitOne()],
                                      dptraits=[T.DPTraitExponential()],
                                      dhtraits=[T.DHTraitOne()]), rn,
         dict(base, bpt_a=1.0, bpt_s=12.0, bht_s=1 + np.array(rn) / 20, vpt_rt=4.0,
              vpt_vt=210.0, dpt_a=25.0, dpt_s=30.0), False, False),
    ]


def capture(D, T, name, kw, rn, params, loose, tilted, mc=False):
    from gbkfit.model.gmodels import _smdisk, _mcdisk
    from gbkfit.math import interpolation
    rstep = min(1, min(np.diff(rn)) / 2)
    args = dict(loose=loose, tilted=tilted, rnodes=tuple(rn), rstep=rstep,
                interp=interpolation.InterpolatorLinear, vsys_nwmode=None, xpos_nwmode=None,
                ypos_nwmode=None, posa_nwmode=None, incl_nwmode=None,
                zptraits=kw.get('zptraits', []), sptraits=kw.get('sptraits', []),
                wptraits=kw.get('wptraits', []))
    args.update({k: v for k, v in kw.items() if k not in args})
    disk = _mcdisk.MCDisk(cflux=1e-3, **args) if mc else _smdisk.SMDisk(**args)
    drv = RecordingDriver()
    p = {k: np.array(v, dtype=np.float64) if np.ndim(v) else v for k, v in params.items()}
    disk.evaluate(drv, p, None, None, None, None, None, None,
                  (16, 16, 1), (1, 1, 0), (0, 0, 0), 0, 8, 10.0, -40.0, np.float32, None)
    kind, call = drv.log[0]
    out = {}
    if mc:
        cflux, nclouds, csum, hoi = call[:4]
        out['cflux'] = np.float32(cflux)
        out['nclouds'] = np.int64(nclouds)
        out['ncloudscsum'] = np.asarray(csum, np.int32)
        out['hasordint'] = np.asarray(hoi, np.uint8)
        call = call[4:]
    for n, v in zip(NAMES, call):
        if v is None:
            continue
        out[n] = np.asarray(v)
    return out


def main(src=None):
    from _refimport import import_reference
    import_reference(src)
    import gbkfit.model.gmodels._disk as D
    import gbkfit.model.gmodels.traits as T
    import gbkfit.psflsf.lsfs as L
    import gbkfit.psflsf.psfs as P

    packing = {}
    for name, kw, rn, params, loose, tilted in cases(T):
        for k, v in capture(D, T, name, kw, rn, params, loose, tilted).items():
            packing[f'{name}/{k}'] = v
    name, kw, rn, params, loose, tilted = cases(T)[4]
    for k, v in capture(D, T, name, kw, rn, params, loose, tilted, mc=True).items():
        packing[f'mc_{name}/{k}'] = v
    np.savez_compressed(os.path.join(HERE, 'packing.npz'), **packing)

    psf = {}
    for label, obj in (('gauss', P.PSFGauss(1.5)), ('moffat', P.PSFMoffat(1.2, 2.5)),
                       ('lorentz', P.PSFLorentz(0.8)), ('ggauss', P.PSFGGauss(1.5, 1.5)),
                       ('gauss_ell', P.PSFGauss(1.0, ratio=0.6, posa=30.0))):
        psf[f'psf_{label}'] = obj.asarray((0.5, 0.4))
        psf[f'psf_{label}_padded'] = obj.asarray((1.0, 1.0), (24, 20), (-1, -1))
    for label, obj in (('gauss', L.LSFGauss(5.0)), ('moffat', L.LSFMoffat(5.0, 2.5)),
                       ('lorentz', L.LSFLorentz(3.0)), ('ggauss', L.LSFGGauss(5.0, 1.5))):
        psf[f'lsf_{label}'] = obj.asarray(0.5)
        psf[f'lsf_{label}_padded'] = obj.asarray(2.0, 32, -1)
    np.savez_compressed(os.path.join(HERE, 'psflsf.npz'), **psf)

    # reference model outputs from the compiled templates
    from oracle.oracle import Reference, build
    if not Reference.available():
        build()
    ref = Reference()
    cubes = {}
    geoms = dict(
        thin=dict(spat_size=(36, 32, 1), spat_step=(1, 1, 0), spat_zero=(-2.0, -1.5, 0),
                  spec_size=40, spec_step=10.0, spec_zero=-200.0),
        thick=dict(spat_size=(32, 30, 20), spat_step=(1, 1, 1), spat_zero=(0.0, -0.5, -9.5),
                   spec_size=40, spec_step=10.0, spec_zero=-200.0))
    for name, kw, rn, params, loose, tilted in cases(T):
        pk = {k.split('/', 1)[1]: v for k, v in packing.items() if k.startswith(name + '/')}
        thick = name.startswith('thick')
        g = dict(geoms['thick' if thick else 'thin'], loose=loose, tilted=tilted, opacity=None)
        packed = packed_from_capture(pk)
        sx, sy, sz = g['spat_size']
        outs = dict(scube=np.zeros((g['spec_size'], sy, sx), np.float32),
                    rdata=np.zeros((sz, sy, sx), np.float32),
                    vdata_cmp=np.full((sz, sy, sx), np.nan, np.float32),
                    ddata_cmp=np.full((sz, sy, sx), np.nan, np.float32))
        ref.smdisk_evaluate(packed, g, outs)
        for k, v in outs.items():
            cubes[f'{name}/{k}'] = v
    rng = np.random.default_rng(5)
    cube = cubes['thin_exp_arctan/scube']
    wc = rng.random(cube.shape).astype(np.float32)
    orders = np.array([0, 1, 2, 4], np.int32)
    md, mm, mw = ref.mmaps_moments((36, 32, 40), (1.0, 1.0, 10.0), (0.0, 0.0, -200.0), cube, wc,
                                   1e-6, orders)
    cubes.update({'moments/wcube': wc, 'moments/orders': orders, 'moments/d': md,
                  'moments/m': mm, 'moments/w': mw})
    od = rng.standard_normal(5000).astype(np.float32)
    oe = (rng.random(5000) + 0.5).astype(np.float32)
    om = (rng.random(5000) > 0.2).astype(np.float32)
    mdl = rng.standard_normal(5000).astype(np.float32)
    res = ref.residual(od, oe, om, mdl, None, None, 0.8)
    cubes.update({'residual/od': od, 'residual/oe': oe, 'residual/om': om, 'residual/md': mdl,
                  'residual/res': res,
                  'residual/sum_sq': np.float64(ref.residual_sum(res, True)),
                  'residual/sum_abs': np.float64(ref.residual_sum(res, False))})
    src_c = rng.standard_normal((20, 18, 22)).astype(np.float32)
    cubes['downscale/src'] = src_c
    cubes['downscale/dst'] = ref.dcube_downscale((2, 3, 2), (1, 2, 3), src_c, (8, 5, 10))
    d, m = ref.dcube_mask(0.6, True, src_c)
    cubes['mask/d'] = d
    cubes['mask/m'] = m
    spat = np.abs(rng.standard_normal((6, 7, 9))).astype(np.float32)
    cubes['wcube/spat'] = spat
    cubes['wcube/spec'] = ref.wcube_evaluate(spat, 11)
    a = rng.standard_normal((12, 14, 16)).astype(np.float32)
    k = rng.random((5, 7, 9)).astype(np.float32)
    cubes['convolve/a'] = a
    cubes['convolve/k'] = k
    cubes['convolve/out'] = ref.convolve(a, k)
    np.savez_compressed(os.path.join(HERE, 'cubes.npz'), **cubes)


def packed_from_capture(pk):
    """Captured reference arrays -> the packed-dict layout of the oracle."""
    out = dict(subrnodes=pk['rnodes'])
    for n in ('vsys', 'xpos', 'ypos', 'posa', 'incl'):
        out[n] = pk.get(n)
    for k in ('rpt', 'rht', 'vpt', 'vht', 'dpt', 'dht', 'zpt', 'spt', 'wpt'):
        if f'{k}_uids' in pk:
            out[k] = {f: pk[f'{k}_{f}'] for f in ('uids', 'cvalues', 'ccounts', 'pvalues',
                                                   'pcounts')}
        else:
            out[k] = None
    return out


if __name__ == '__main__':
    main(*sys.argv[1:])
