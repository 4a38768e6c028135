"""Trait catalogue of the disk components (host side).

Mirrors ``gbkfit/model/gmodels/traits.py`` of the reference: every trait has a
``uid`` (the same integers as the native catalogue, traits.py:16-148), a tuple
of constants ``consts()`` (traits.py:317-318: the constructor keyword values in
order), smooth parameters ``params_sm()`` and node-wise parameters
``params_rnw(nnodes)``.  Density traits also provide the ring integrals used to
budget mcdisk clouds (traits.py:188-275).

Only what the model-evaluation path needs is kept: no parsers or dumping.
"""

import numpy as np

TRUNC_DEFAULT = 0

# uids (traits.py:16-148)
RPT = dict(uniform=1, exponential=2, gauss=3, ggauss=4, lorentz=5, moffat=6, sech2=7,
           mixture_exponential=51, mixture_gauss=52, mixture_ggauss=53,
           mixture_moffat=54, nw_uniform=101, nw_harmonic=102, nw_distortion=103)
RHT = dict(uniform=1, exponential=2, gauss=3, ggauss=4, lorentz=5, moffat=6, sech2=7)
VPT = dict(tan_uniform=1, tan_arctan=2, tan_boissier=3, tan_epinat=4, tan_lramp=5,
           tan_tanh=6, tan_polyex=7, tan_rix=8, nw_tan_uniform=101,
           nw_tan_harmonic=102, nw_rad_uniform=103, nw_rad_harmonic=104,
           nw_ver_uniform=105, nw_ver_harmonic=106, nw_los_uniform=107,
           nw_los_harmonic=108)
DPT = dict(uniform=1, exponential=2, gauss=3, ggauss=4, lorentz=5, moffat=6, sech2=7,
           mixture_exponential=51, mixture_gauss=52, mixture_ggauss=53,
           mixture_moffat=54, nw_uniform=101, nw_harmonic=102, nw_distortion=103)
ZPT = dict(nw_uniform=101, nw_harmonic=102)
SPT = dict(azrange=1, nw_azrange=101)
WPT = dict(axis_range=1)
OPT_OFFSET = 1000   # opacity traits: 1000 + density uid (traits.py:71-101)

# smooth parameters of the polar profiles (traits.py:446-640, 1240-1500)
_SM_PROFILE = dict(uniform=('a',), exponential=('a', 's'), gauss=('a', 's'),
                   ggauss=('a', 's', 'b'), lorentz=('a', 's'), moffat=('a', 's', 'b'),
                   sech2=('a', 's'))
_SM_VEL = dict(tan_uniform=('vt',), tan_arctan=('rt', 'vt'), tan_boissier=('rt', 'vt'),
               tan_epinat=('rt', 'vt', 'a', 'g'), tan_lramp=('rt', 'vt'),
               tan_tanh=('rt', 'vt'), tan_polyex=('rt', 'vt', 'a'),
               tan_rix=('rt', 'vt', 'b', 'g'))
_NW_VEL = dict(nw_tan_uniform=('vt',), nw_rad_uniform=('vr',), nw_ver_uniform=('vv',),
               nw_los_uniform=('vl',))


def _profile_fun(name):
    """1-D profiles of math/math.py used by the ring integrals."""
    def expon(x, a, b, c):
        return a * np.exp(-np.abs(x - b) / c)

    def gauss(x, a, b, c):
        return a * np.exp(-(x - b) * (x - b) / (2 * c * c))

    def ggauss(x, a, b, c, d):
        return a * np.exp(-np.power(np.abs(x - b) / c, d))

    def lorentz(x, a, b, c):
        return a * c * c / ((x - b) * (x - b) + c * c)

    def moffat(x, a, b, c, d):
        return a / np.power(1 + ((x - b) / c) ** 2, d)

    def sech2(x, a, b, c):
        return a / np.cosh((x - b) / c) ** 2

    return dict(exponential=expon, gauss=gauss, ggauss=ggauss, lorentz=lorentz,
                moffat=moffat, sech2=sech2)[name]


def _integrate_rings(rings, fun, *args):
    """traits.py:188-197: ring-centre amplitude times annulus area."""
    rings = np.asarray(rings, dtype=np.float64)
    rsep = rings[1] - rings[0]
    rmin = rings - rsep * 0.5
    rmax = rings + rsep * 0.5
    return fun(rings, *args) * np.pi * (rmax * rmax - rmin * rmin)


class Trait:
    """A trait: ``kind`` is one of rpt/rht/vpt/vht/dpt/dht/zpt/spt/wpt/opt/oht."""

    def __init__(self, kind, name, uid, consts=(), sm=(), nw=(), order=None, nblobs=None):
        self.kind = kind
        self.name = name
        self._uid = uid
        self._consts = tuple(float(c) for c in consts)
        self._sm = tuple(sm)
        self._nw = tuple(nw)
        self._nblobs = nblobs

    def uid(self):
        return self._uid

    def consts(self):
        return self._consts

    def params_sm(self):
        """[(name, size)] of the smooth parameters."""
        n = self._nblobs
        return [(p, n if n else 1) for p in self._sm]

    def params_rnw(self, nnodes):
        """[(name, nnodes)] of the node-wise parameters."""
        return [(p, nnodes) for p in self._nw]

    def has_analytical_integral(self):
        # traits.py:446-800: uniform and the mixtures integrate analytically
        return self.name == 'uniform' or self.name.startswith('mixture')

    def integrate(self, params, rings):
        """Cloud budget of a density trait (traits.py:188-275)."""
        rings = np.asarray(rings, dtype=np.float64)
        if self.name == 'uniform':
            a = params['a']
            rsep = rings[1] - rings[0]
            rmin = rings[0] - 0.5 * rsep
            rmax = rings[-1] + 0.5 * rsep
            return np.pi * a * (rmax * rmax - rmin * rmin)
        if self.name in ('nw_uniform', 'nw_harmonic'):
            a = np.asarray(params['a'], dtype=np.float64)
            return _integrate_rings(rings, lambda x, a_: a_ * np.ones_like(x), a)
        if self.name in _SM_PROFILE:
            fun = _profile_fun(self.name)
            args = [params[p] for p in self._sm]
            a, rest = args[0], args[1:]
            return _integrate_rings(rings, lambda x, *r: fun(x, a, 0, *r), *rest)
        raise NotImplementedError(f"no integral for density trait '{self.name}'")

    def __repr__(self):
        return f"Trait({self.kind}:{self.name})"


# ---- constructors (one per reference trait class) -------------------------------

def bpt(name, nblobs=None, order=None):
    """Surface-brightness polar trait (traits.py:428-800)."""
    uid = RPT[name]
    if name in _SM_PROFILE:
        return Trait('rpt', name, uid, sm=_SM_PROFILE[name])
    if name in ('mixture_exponential', 'mixture_ggauss', 'mixture_moffat'):
        return Trait('rpt', name, uid, consts=(nblobs,),
                     sm=('r', 't', 'a', 's', 'b', 'q', 'p'), nblobs=nblobs)
    if name == 'mixture_gauss':
        return Trait('rpt', name, uid, consts=(nblobs,),
                     sm=('r', 't', 'a', 's', 'q', 'p'), nblobs=nblobs)
    if name == 'nw_uniform':
        return Trait('rpt', name, uid, nw=('a',))
    if name == 'nw_harmonic':
        return Trait('rpt', name, uid, consts=(order,), nw=('a', 'p') if order else ('a',))
    if name == 'nw_distortion':
        return Trait('rpt', name, uid, nw=('a', 'p', 's'))
    raise ValueError(name)


def opt(name, **kw):
    """Opacity polar trait: a density trait with uid + 1000."""
    t = bpt(name, **kw)
    t.kind = 'opt'
    t._uid += OPT_OFFSET
    return t


def bht(name, rnodes=False, trunc=TRUNC_DEFAULT):
    """Surface-brightness height trait (traits.py:802-880): consts (trunc, rnodes)."""
    uid = RHT[name]
    p = ('s', 'b') if name in ('ggauss', 'moffat') else ('s',)
    return Trait('rht', name, uid, consts=(trunc, bool(rnodes)),
                 sm=() if rnodes else p, nw=p if rnodes else ())


def oht(name, rnodes=False, trunc=TRUNC_DEFAULT):
    """Opacity height trait: amplitude first (traits.py:2000-2119)."""
    uid = OPT_OFFSET + RHT[name]
    p = ('a', 's', 'b') if name in ('ggauss', 'moffat') else ('a', 's')
    return Trait('oht', name, uid, consts=(trunc, bool(rnodes)),
                 sm=() if rnodes else p, nw=p if rnodes else ())


def vpt(name, order=None):
    """Velocity polar trait (traits.py:882-1120)."""
    uid = VPT[name]
    if name in _SM_VEL:
        return Trait('vpt', name, uid, sm=_SM_VEL[name])
    if name in _NW_VEL:
        return Trait('vpt', name, uid, nw=_NW_VEL[name])
    return Trait('vpt', name, uid, consts=(order,), nw=('a', 'p') if order else ('a',))


def vht_one():
    """traits.py:1122-1135: consts (rnodes=False,)."""
    return Trait('vht', 'one', 1, consts=(False,))


def dht_one():
    return Trait('dht', 'one', 1, consts=(False,))


def dpt(name, nblobs=None, order=None):
    """Dispersion polar trait (traits.py:1137-1400)."""
    t = bpt(name, nblobs=nblobs, order=order)
    t.kind = 'dpt'
    t._uid = DPT[name]
    return t


def zpt(name, order=None):
    """Vertical distortion polar trait."""
    if name == 'nw_uniform':
        return Trait('zpt', name, ZPT[name], nw=('a',))
    return Trait('zpt', name, ZPT[name], consts=(order,), nw=('a', 'p') if order else ('a',))


def spt(name):
    """Selection polar trait."""
    if name == 'azrange':
        return Trait('spt', name, SPT[name], sm=('p', 's'))
    return Trait('spt', name, SPT[name], nw=('p', 's'))


def wpt_axis_range(axis, angle, weight):
    return Trait('wpt', 'axis_range', WPT['axis_range'], consts=(axis, angle, weight))
