"""Every trait of the reference's catalogue (traits.py:16-148 uids) as a small
disk case: one kind varies, the others keep a plain exponential disk with an
arctan rotation curve and a uniform dispersion.  Parameter values are
generic physical ones (scales of a few pixels, velocities of a few hundred
km/s, angles in degrees) chosen per parameter name.

Each case: (name, traits, params, thick) for the 20-ring disk on 0-30 px of
the golden-fixture geometries (thin 36x32, thick 32x30x20; 40 channels).
"""

import numpy as np

RNODES = np.linspace(0, 30, 20)
BASE = dict(xpos=16.3, ypos=14.1, posa=45.0, incl=60.0, vsys=3.0)


def _value(kind, name, size, nodewise):
    """A value for parameter `name` of a trait of `kind` (node-wise: one per ring)."""
    r = RNODES
    nb = size if not nodewise else None
    amp = dict(rpt=1.0, dpt=20.0, opt=0.5).get(kind, 1.0)
    table = {
        'a': (amp * np.exp(-r / 12) + (0.05 if kind == 'rpt' else 5.0)) if nodewise else amp,
        's': 8.0 if kind in ('rpt', 'dpt', 'opt') else 1.5,
        'b': 1.5,
        'p': 30.0 + r if nodewise else 30.0,
        'vt': 200.0 * np.tanh(r / 5) if nodewise else 200.0,
        'rt': 4.0, 'g': 2.0,
        'vr': 20 * np.tanh(r / 8), 'vv': 10 * np.tanh(r / 8), 'vl': 15 * np.tanh(r / 8),
    }
    if kind == 'vpt' and name == 'a':
        table['a'] = (30 * np.tanh(r / 8)) if nodewise else 1.5
    if kind == 'vpt' and name == 'b':
        table['b'] = 0.5
    if kind == 'zpt':
        table['a'] = 0.5 * np.tanh(r / 10)
    if kind == 'dpt' and nodewise and name == 'a':
        table['a'] = 8.0 * np.exp(-r / 12) + 2.0
    if kind == 'spt':
        table['p'] = 30.0 + 0 * r if nodewise else 30.0
        table['s'] = 220.0 + 0 * r if nodewise else 220.0
    if nb and nb > 1:     # mixture blobs
        blobs = dict(r=[6.0, 12.0], t=[30.0, 200.0], a=[1.0, 0.5], s=[4.0, 6.0],
                     b=[1.5, 1.2], q=[0.7, 0.9], p=[20.0, 60.0])
        v = np.asarray(blobs[name][:nb], np.float64)
        if kind == 'dpt' and name == 'a':
            v = v * 20
        return v
    v = table[name]
    if nodewise:
        return np.broadcast_to(np.asarray(v, np.float64), r.shape).copy()
    return float(np.asarray(v))


def _params(disk, extra_prefixes=()):
    p = dict(BASE)
    for name, (size, nw) in disk.pdescs.items():
        if name in p:
            continue
        pre, pname = name.split('_', 1)
        kind = pre.rstrip('0123456789')
        kind = dict(bpt='rpt', bht='rht', vpt='vpt', vht='vht', dpt='dpt', dht='dht',
                    zpt='zpt', spt='spt', wpt='wpt', opt='opt', oht='oht')[kind]
        p[name] = _value(kind, pname, size, nw)
    return p


def cases():
    from gbkfit_b200 import traits as T
    from gbkfit_b200.disk import Disk
    base = dict(rpt=[T.bpt('exponential')], vpt=[T.vpt('tan_arctan')], dpt=[T.dpt('uniform')])
    out = []

    def add(name, traits, thick=False, loose=False, tilted=False):
        d = Disk(loose, tilted, RNODES, traits=traits)
        out.append((name, traits, _params(d), thick))

    for n in T.RPT:
        kw = dict(nblobs=2) if n.startswith('mixture') else {}
        if n == 'nw_harmonic':
            for order in (0, 2):
                add(f'rpt_{n}{order}', dict(base, rpt=[T.bpt(n, order=order)]))
            continue
        add(f'rpt_{n}', dict(base, rpt=[T.bpt(n, **kw)]))
    for n in T.VPT:
        if n.endswith('harmonic'):
            for order in (0, 1, 3):
                add(f'vpt_{n}{order}', dict(base, vpt=[T.vpt(n, order=order)]))
            continue
        add(f'vpt_{n}', dict(base, vpt=[T.vpt(n)]))
    for n in T.DPT:
        kw = dict(nblobs=2) if n.startswith('mixture') else {}
        if n == 'nw_harmonic':
            kw = dict(order=2)
        # a uniform floor first: decaying profiles alone take the dispersion
        # to ~0 at large radii, where the reference's line pdf (no guard on
        # sigma, gmodels.hpp:886) is ill-conditioned in fp32
        traits = [T.dpt(n, **kw)] if n == 'uniform' else [T.dpt('uniform'), T.dpt(n, **kw)]
        add(f'dpt_{n}', dict(base, dpt=traits))
    thick = dict(base, rht=[T.bht('sech2')], vht=[T.vht_one()], dht=[T.dht_one()])
    for n in T.RHT:
        for trunc, rn in ((0, False), (2.0, False), (0, True)):
            add(f'rht_{n}_t{trunc:g}{"_nw" if rn else ""}',
                dict(thick, rht=[T.bht(n, rnodes=rn, trunc=trunc)]), thick=True)
    for n in T.ZPT:
        kw = dict(order=2) if n == 'nw_harmonic' else {}
        add(f'zpt_{n}', dict(thick, zpt=[T.zpt(n, **kw)]), thick=True)
    for n in T.SPT:
        add(f'spt_{n}', dict(base, spt=[T.spt(n)]))
    add('wpt_axis_range', dict(base, wpt=[T.wpt_axis_range(0, 30.0, 0.5)]))
    add('two_traits_each', dict(rpt=[T.bpt('exponential'), T.bpt('gauss')],
                                vpt=[T.vpt('tan_arctan'), T.vpt('nw_rad_uniform')],
                                dpt=[T.dpt('uniform'), T.dpt('exponential')]))
    return out


GEOMS = dict(
    thin=dict(spat_size=(36, 32, 1), spat_step=(1, 1, 0), spat_zero=(-2.0, -1.5, 0),
              spec_size=40, spec_step=10.0, spec_zero=-200.0),
    thick=dict(spat_size=(32, 30, 20), spat_step=(1, 1, 1), spat_zero=(0.0, -0.5, -9.5),
               spec_size=40, spec_step=10.0, spec_zero=-200.0))


def geometry(thick, loose=False, tilted=False):
    return dict(GEOMS['thick' if thick else 'thin'], loose=loose, tilted=tilted, opacity=None)


# height traits whose reference normalisation uses its stub cdfs (ggauss and
# moffat, truncated: inf / NaN) or its stub moffat pdf (0): the outputs are
# compared by pattern (finite where, zero where), not by value
STUB_HEIGHTS = ('rht_ggauss_t2', 'rht_moffat_t0', 'rht_moffat_t2', 'rht_moffat_t0_nw')


def disk_of(case):
    from gbkfit_b200.disk import Disk
    name, traits, params, thick = case
    return Disk(False, False, RNODES, traits=traits)


OUTS = ('scube', 'rdata', 'wdata', 'vdata_cmp', 'ddata_cmp')


def host_outputs(geo, real):
    sx, sy, sz = geo['spat_size']
    nz = geo['spec_size']
    return dict(scube=np.zeros((nz, sy, sx), real), rdata=np.zeros((sz, sy, sx), real),
                wdata=np.zeros((sz, sy, sx), real),
                vdata_cmp=np.full((sz, sy, sx), np.nan, real),
                ddata_cmp=np.full((sz, sy, sx), np.nan, real))
