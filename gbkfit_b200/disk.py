"""Host-side packing of a disk component's parameters into the native arrays.

Mirrors ``gbkfit/model/gmodels/_disk.py`` of the reference:

* radial sub-nodes ``[r0, r0 + h/2, r0 + 3h/2, ..., last + h/2]`` with
  ``h = rstep`` (_disk.py:151-154);
* per trait kind the arrays ``uids`` (int32), ``cvalues`` (float32),
  ``ccounts`` (int32), ``pvalues`` (float32) and ``pcounts`` (int32), where a
  trait's parameters are its smooth parameters followed by its node-wise
  parameters interpolated onto the sub-nodes (_disk.py:42-125);
* the common parameters vsys/xpos/ypos/posa/incl, one value each or one per
  sub-node for loose/tilted disks (_disk.py:377-391, 515-534).

Parameter names follow the reference: ``vsys, xpos, ypos, posa, incl`` and,
per trait kind prefix (``bpt, bht, vpt, vht, dpt, dht, zpt, spt, wpt`` or
``opt, oht`` for opacity disks), ``<prefix>_<name>`` for the first trait and
``<prefix><i>_<name>`` for the i-th (utils/miscutils.py:70-95).

``pack_batch`` packs B parameter sets at once into (B, n) arrays for the
batched evaluator.
"""

import numpy as np
import scipy.interpolate

KINDS = ('rpt', 'rht', 'vpt', 'vht', 'dpt', 'dht', 'zpt', 'spt', 'wpt')


def make_subrnodes(rnodes, rstep):
    """_disk.py:151-156."""
    rnodes = np.asarray(rnodes, dtype=np.float64)
    sub = np.arange(rnodes[0] + rstep / 2, rnodes[-1], rstep)
    sub = np.insert(sub, 0, rnodes[0])
    sub = np.append(sub, sub[-1] + rstep / 2)
    return sub


def default_rstep(rnodes):
    """_detail.py:52: min(1, smallest node separation / 2)."""
    return min(1.0, float(np.min(np.diff(np.asarray(rnodes, dtype=np.float64)))) / 2)


_LINEAR_CACHE = {}


def _linear_matrix(x, xnew):
    """(n, m) matrix W of linear interpolation from nodes x to points xnew
    (y_new = y @ W, clamped at the ends like numpy.interp); cached, since a
    disk's nodes and sub-nodes do not change."""
    key = (np.asarray(x, np.float64).tobytes(), np.asarray(xnew, np.float64).tobytes())
    hit = _LINEAR_CACHE.get(key)
    if hit is None:
        idx = np.clip(np.searchsorted(x, xnew, side='right') - 1, 0, len(x) - 2)
        x0, x1 = x[idx], x[idx + 1]
        t = np.clip((xnew - x0) / (x1 - x0), 0.0, 1.0)
        hit = np.zeros((len(x), len(xnew)))
        cols = np.arange(len(xnew))
        np.add.at(hit, (idx, cols), 1.0 - t)
        np.add.at(hit, (idx + 1, cols), t)
        if len(_LINEAR_CACHE) > 256:
            _LINEAR_CACHE.clear()
        _LINEAR_CACHE[key] = hit
    return hit


def _interp(kind, x, y, xnew):
    """Node -> sub-node interpolation (math/interpolation.py:16-50)."""
    y = np.asarray(y, dtype=np.float64)
    if kind == 'linear':
        if y.ndim == 1:
            return np.interp(xnew, x, y)
        # batched: y (B, n)
        return y @ _linear_matrix(x, xnew)
    if kind == 'akima':
        return scipy.interpolate.Akima1DInterpolator(x, y, axis=-1)(xnew)
    if kind == 'pchip':
        return scipy.interpolate.PchipInterpolator(x, y, axis=-1)(xnew)
    raise ValueError(f"unknown interpolation '{kind}'")


class Disk:
    """Layout of one disk component's native arrays.

    traits: dict kind -> list of gbkfit_b200.traits.Trait (kinds as in KINDS;
    'rpt'/'rht' hold the density traits, brightness or opacity).
    """

    def __init__(self, loose, tilted, rnodes, rstep=None, interp='linear', traits=None,
                 opacity=False):
        self.loose = bool(loose)
        self.tilted = bool(tilted)
        self.rnodes = np.asarray(rnodes, dtype=np.float64)
        if len(self.rnodes) < 2 or np.any(np.diff(self.rnodes) <= 0) or self.rnodes[0] < 0:
            raise RuntimeError("rnodes must be at least two ascending, unique, positive values")
        self.rstep = default_rstep(self.rnodes) if rstep is None else float(rstep)
        if self.rstep <= 0 or self.rstep > np.min(np.diff(self.rnodes)) / 2:
            raise RuntimeError("rstep must be in (0, min node separation / 2]")
        self.interp = interp
        self.subrnodes = make_subrnodes(self.rnodes, self.rstep)
        self.nsub = len(self.subrnodes)
        self.traits = {k: list((traits or {}).get(k, ())) for k in KINDS}
        self.opacity = bool(opacity)
        for k in KINDS:
            if len(self.traits[k]) > 4:
                raise RuntimeError(f"at most 4 {k} traits (TRAIT_NUM_MAX)")
        if self.traits['rht'] and len(self.traits['rht']) != len(self.traits['rpt']):
            raise RuntimeError("one density height trait per density polar trait")
        prefixes = dict(rpt='opt' if opacity else 'bpt', rht='oht' if opacity else 'bht',
                        vpt='vpt', vht='vht', dpt='dpt', dht='dht', zpt='zpt', spt='spt',
                        wpt='wpt')
        nn = len(self.rnodes)
        # parameter descriptors: name -> (size, nodewise)
        self.pdescs = {}
        if self.traits['vpt']:
            self.pdescs['vsys'] = (nn if self.loose else 1, self.loose)
        self.pdescs['xpos'] = (nn if self.loose else 1, self.loose)
        self.pdescs['ypos'] = (nn if self.loose else 1, self.loose)
        self.pdescs['posa'] = (nn if self.tilted else 1, self.tilted)
        self.pdescs['incl'] = (nn if self.tilted else 1, self.tilted)
        # per kind: static tables and the ordered parameter list
        self.tables = {}
        for k in KINDS:
            ts = self.traits[k]
            if not ts:
                self.tables[k] = None
                continue
            uids, cvals, ccnts, pcnts, plist = [], [], [], [], []
            for i, t in enumerate(ts):
                pre = prefixes[k] + (str(i) if i else '') + '_'
                sm = t.params_sm()
                nw = t.params_rnw(nn)
                uids.append(t.uid())
                cvals += list(t.consts())
                ccnts.append(len(t.consts()))
                pcnts.append(sum(s for _, s in sm) + len(nw) * self.nsub)
                for name, size in sm:
                    plist.append((pre + name, size, False))
                    self.pdescs[pre + name] = (size, False)
                for name, size in nw:
                    plist.append((pre + name, size, True))
                    self.pdescs[pre + name] = (size, True)
            self.tables[k] = dict(
                uids=np.asarray(uids, np.int32), cvalues=np.asarray(cvals, np.float32),
                ccounts=np.asarray(ccnts, np.int32), pcounts=np.asarray(pcnts, np.int32),
                plist=plist, npv=int(sum(pcnts)))

    def common_size(self, name):
        if name in ('vsys', 'xpos', 'ypos'):
            return self.nsub if self.loose else 1
        return self.nsub if self.tilted else 1

    def _common(self, params, name, nw, batch):
        v = np.asarray(params[name], dtype=np.float64)
        if nw:
            return _interp(self.interp, self.rnodes, v, self.subrnodes)
        return v.reshape(batch + (1,)) if batch else np.atleast_1d(v)

    def pack(self, params):
        """One parameter set -> dict of host arrays (float32/int32)."""
        return self._pack(params, ())

    def pack_batch(self, params, nbatch):
        """params[name]: (B,) for scalars, (B, n) for vectors -> (B, ...) arrays."""
        return self._pack(params, (nbatch,))

    def _pack(self, params, batch):
        out = dict(subrnodes=self.subrnodes.astype(np.float32))
        for name in ('vsys', 'xpos', 'ypos', 'posa', 'incl'):
            if name not in self.pdescs:
                out[name] = None
                continue
            nw = self.pdescs[name][1]
            out[name] = np.asarray(self._common(params, name, nw, batch), np.float32)
        for k in KINDS:
            tab = self.tables[k]
            if tab is None:
                out[k] = None
                continue
            chunks = []
            for pname, size, nw in tab['plist']:
                v = np.asarray(params[pname], dtype=np.float64)
                if nw:
                    chunks.append(_interp(self.interp, self.rnodes, v, self.subrnodes))
                else:
                    chunks.append(v.reshape(batch + (size,)))
            pv = np.concatenate(chunks, axis=-1) if chunks else np.zeros(batch + (0,))
            out[k] = dict(uids=tab['uids'], cvalues=tab['cvalues'], ccounts=tab['ccounts'],
                          pvalues=np.ascontiguousarray(pv, np.float32), pcounts=tab['pcounts'])
        return out

    # ---- mcdisk cloud budget (_mcdisk.py:159-216) --------------------------------
    def hasordint(self):
        return np.asarray([t.has_analytical_integral() for t in self.traits['rpt']], np.uint8)

    def ncloudscsum(self, params, cflux):
        """Cumulative cloud counts per trait (analytic) or per ring."""
        ring_centres = self.subrnodes[1:-1]
        counts = []
        prefix = 'opt' if self.opacity else 'bpt'
        for i, t in enumerate(self.traits['rpt']):
            pre = prefix + (str(i) if i else '') + '_'
            tp = {}
            for name, _ in t.params_sm():
                tp[name] = params[pre + name]
            for name, _ in t.params_rnw(len(self.rnodes)):
                sub = _interp(self.interp, self.rnodes, params[pre + name], self.subrnodes)
                tp[name] = sub[1:-1]
            integral = t.integrate(tp, ring_centres)
            counts.extend(np.atleast_1d(np.asarray(integral) / cflux).astype(np.int32))
        return np.cumsum(np.asarray(counts, np.int64)).astype(np.int32)
