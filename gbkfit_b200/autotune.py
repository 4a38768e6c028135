"""Autotuner of the batched pipeline's shape parameters.

Knobs (all change speed only, never results beyond fp32 rounding):
* ``conv``: direct separable FIR (low-rank PSFs) or FFT convolution;
* ``fft_size``: FFT grid per axis, any 2/3/5/7-smooth size >= the window
  (x even);
* ``chunk``: parameter sets per pipeline wave (the wave's intermediates
  should stay in L2);
* ``band``: output rows per PSF block of the direct mode (smaller bands: more
  resident blocks, more halo rows);
* ``psf_variant``: PSF kernel sized for 4 or 5 resident blocks per SM, with
  its residual in a separate pass or in the y-FIR items (data loaded after or
  before each item's FIR), or persistent over all (set, plane) items;
* ``model_variant``: the direct mode's model kernel (0: one 32-column chunk
  per warp; 1: two chunks per warp on packed FP32 pairs; 2: a 4 x 8 spaxel
  tile per warp; 3: 2 with the range-table masks by bit transposes; the
  same values; 4: 3 with the line exponent from one multiply-add, the same
  values up to fp32 rounding);
* ``rows_k1``: spectral rows per shared-memory group of the model kernel.

Coordinate descent from the defaults; every trial builds an evaluator and
times a few full evaluations with CUDA events.  Results are cached per
(problem, device) in ~/.cache/gbkfit_b200/autotune.json.
"""

import json
import os
import time

import numpy as np

CACHE = os.path.join(os.path.expanduser('~'), '.cache', 'gbkfit_b200', 'autotune.json')


def smooth_sizes(w, even=False, count=3):
    out = []
    n = w
    while len(out) < count:
        m = n
        for p in (2, 3, 5, 7):
            while m % p == 0:
                m //= p
        if m == 1 and (not even or n % 2 == 0):
            out.append(n)
        n += 1
    return out


def _key(w, nsets):
    import torch
    from .batched import kernel_boxes, separable_factors
    g = w.geom
    rank = separable_factors(kernel_boxes(g)[0])[0]
    return json.dumps(dict(size=g.size, kernel=g.kernel_size, nsets=nsets, psf_rank=rank,
                           nsub=w.disk.nsub, device=torch.cuda.get_device_name()))


def _load():
    try:
        with open(CACHE) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(key, cfg):
    try:
        os.makedirs(os.path.dirname(CACHE), exist_ok=True)
        d = _load()
        d[key] = cfg
        with open(CACHE, 'w') as f:
            json.dump(d, f, indent=1)
    except OSError:
        pass


def time_config(w, data, err, nsets, cfg, reps=3):
    import torch
    from .batched import BatchedSMDisk
    try:
        ev = BatchedSMDisk(w.disk, w.geom, data, err, max_sets=nsets, **cfg)
    except RuntimeError:
        return float('inf')
    bufs = ev.alloc_inputs(nsets)
    ev.upload(ev.pack(w.params, nsets), bufs, nsets)
    ev.evaluate_device(bufs, nsets)
    t = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        ev.evaluate_device(bufs, nsets)
        b.record()
        b.synchronize()
        t.append(a.elapsed_time(b))
    ev.close()
    return float(np.median(t))


def tune_batched(w, data, err, nsets, budget_s=60.0, use_cache=True):
    """Best {fft_size, chunk, rows_k1, conv, band} for workload w with nsets sets."""
    key = _key(w, nsets)
    if use_cache:
        c = _load().get(key)
        if c:
            return dict(fft_size=tuple(c['fft_size']), chunk=c['chunk'], rows_k1=c['rows_k1'],
                        conv=c['conv'], band=c.get('band', 0),
                        psf_variant=c.get('psf_variant', 0),
                        model_variant=c.get('model_variant', 0))
    g = w.geom
    t_end = time.time() + budget_s
    # direct separable convolution (when the PSF is rank 1): chunk, then band
    best_d, best_dt = None, float('inf')
    for chunk in (32, 64, 128, 256, 512):
        cfg = dict(fft_size=(0, 0, 0), chunk=chunk, rows_k1=16, conv='direct', band=0,
                   model_variant=0)
        t = time_config(w, data, err, nsets, cfg)
        if t < best_dt:
            best_d, best_dt = cfg, t
    if best_d is not None:
        for band in (96, 64, 48, 32):
            if band >= g.size[1]:
                continue
            cfg = dict(best_d, band=band)
            t = time_config(w, data, err, nsets, cfg)
            if t < best_dt:
                best_d, best_dt = cfg, t
        # the PSF kernel's variants (resident blocks per SM x epilogue)
        base = dict(best_d)
        for variant in range(1, 8):
            cfg = dict(base, psf_variant=variant)
            t = time_config(w, data, err, nsets, cfg)
            if t < best_dt:
                best_d, best_dt = cfg, t
        # the model kernel's variants
        base = dict(best_d)
        for mv in (1, 2, 3, 4):
            cfg = dict(base, model_variant=mv)
            t = time_config(w, data, err, nsets, cfg)
            if t < best_dt:
                best_d, best_dt = cfg, t
    win = [g.size[i] + g.kernel_size[i] - 1 for i in range(3)]
    cand = [smooth_sizes(win[0], even=True), smooth_sizes(win[1]), smooth_sizes(win[2])]
    best = dict(fft_size=(cand[0][0], cand[1][0], cand[2][0]), chunk=8, rows_k1=16, conv='fft',
                band=0)
    best_t = time_config(w, data, err, nsets, best)
    trials = []
    for knob, values in (('chunk', (2, 4, 8, 16, 32)), ('rows_k1', (8, 16, 32)),
                         ('fft_x', cand[0]), ('fft_y', cand[1]), ('fft_z', cand[2]),
                         ('chunk', (2, 4, 8, 16, 32))):
        for v in values:
            if time.time() > t_end:
                break
            cfg = dict(best)
            if knob.startswith('fft_'):
                fs = list(cfg['fft_size'])
                fs['xyz'.index(knob[-1])] = v
                cfg['fft_size'] = tuple(fs)
            else:
                cfg[knob] = v
            if cfg == best:
                continue
            t = time_config(w, data, err, nsets, cfg)
            trials.append((knob, v, t))
            if t < best_t:
                best, best_t = cfg, t
    if best_dt < best_t:
        best, best_t = best_d, best_dt
    out = dict(best)
    out['fft_size'] = tuple(out['fft_size'])
    if use_cache:
        _store(key, dict(out, fft_size=list(out['fft_size']), ms=best_t))
    return out
