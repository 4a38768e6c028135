"""Shared helpers of the test-suite."""

import numpy as np

KINDS = ('rpt', 'rht', 'vpt', 'vht', 'dpt', 'dht', 'zpt', 'spt', 'wpt')


def rel_err(a, b):
    """max |a - b| / max |b| (normwise relative error)."""
    a = np.asarray(a)
    b = np.asarray(b)
    a = a.astype(np.complex128 if np.iscomplexobj(a) else np.float64)
    b = b.astype(np.complex128 if np.iscomplexobj(b) else np.float64)
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (den if den > 0 else 1.0))


def upload(packed, dev):
    """Disk.pack() host arrays -> torch tensors on dev (None stays None)."""
    import torch
    out = {}
    for k, v in packed.items():
        if v is None:
            out[k] = None
        elif isinstance(v, dict):
            out[k] = {f: torch.from_numpy(np.ascontiguousarray(a)).to(dev) for f, a in v.items()}
        else:
            out[k] = torch.from_numpy(np.ascontiguousarray(v)).to(dev)
    return out


def trait_args(pd):
    """Per-kind (uids, cvalues, ccounts, pvalues, pcounts) in reference order."""
    args = []
    for k in KINDS:
        t = pd[k]
        if t is None:
            args += [None] * 5
        else:
            args += [t['uids'], t['cvalues'], t['ccounts'], t['pvalues'], t['pcounts']]
    return args


def gpu_smdisk(backend, pd, geom, outs):
    """DriverBackendGModelB200.smdisk_evaluate with the reference's argument
    order (_detail/native.py:403-475)."""
    o = [outs.get(n) for n in ('image', 'scube', 'wdata', 'wdata_cmp', 'rdata', 'rdata_cmp',
                               'ordata', 'ordata_cmp', 'vdata_cmp', 'ddata_cmp')]
    backend.smdisk_evaluate(
        geom['loose'], geom['tilted'], pd['subrnodes'],
        pd['vsys'], pd['xpos'], pd['ypos'], pd['posa'], pd['incl'],
        *trait_args(pd), geom.get('opacity'),
        geom['spat_size'], geom['spat_step'], geom['spat_zero'], 0.0,
        geom['spec_size'], geom['spec_step'], geom['spec_zero'], *o)


def gpu_mcdisk(backend, cflux, nclouds, csum_d, hoi_d, pd, geom, outs):
    o = [outs.get(n) for n in ('image', 'scube', 'wdata', 'wdata_cmp', 'rdata', 'rdata_cmp',
                               'ordata', 'ordata_cmp', 'vdata_cmp', 'ddata_cmp')]
    backend.mcdisk_evaluate(
        cflux, nclouds, csum_d, hoi_d,
        geom['loose'], geom['tilted'], pd['subrnodes'],
        pd['vsys'], pd['xpos'], pd['ypos'], pd['posa'], pd['incl'],
        *trait_args(pd), geom.get('opacity'),
        geom['spat_size'], geom['spat_step'], geom['spat_zero'], 0.0,
        geom['spec_size'], geom['spec_step'], geom['spec_zero'], *o)
