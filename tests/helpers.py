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


def grad96_problem():
    """The differentiable configuration: workload, data (fp64 oracle model of
    the truth + seeded Gaussian noise of 2 % of the peak), error cube, and the
    evaluation point as a parameter vector (gbkfit_b200.adjoint layout)."""
    from gbkfit_b200 import workloads
    from gbkfit_b200.adjoint import to_vector
    from oracle.oracle import scube_pipeline
    w = workloads.smdisk_grad96()
    truth = scube_pipeline(w.disk.pack(w.extra['truth']), w.geom, precision='f64')
    rng = np.random.default_rng(w.extra['noise_seed'])
    sig = w.extra['noise_frac'] * truth.max()
    data = (truth + rng.normal(0.0, sig, truth.shape)).astype(np.float32)
    err = np.full_like(data, sig, dtype=np.float32)
    return w, data, err, to_vector(w.params, w.extra['scale'])


def grad96_oracle_chi2(w, theta, data, err):
    """chi^2 of the fp64 oracle pipeline at a parameter vector."""
    from gbkfit_b200.adjoint import from_vector
    from oracle.oracle import chi2, scube_pipeline
    p, scale = from_vector(w.disk, theta)
    m = scube_pipeline(w.disk.pack(p), w.geom, precision='f64')
    return chi2(scale * m, data.astype(np.float64), err.astype(np.float64))


def grad96_groups(theta, nnodes):
    """Slices of the parameter vector: geometry, the three node groups, scale."""
    return [slice(0, 5)] + [slice(5 + j * nnodes, 5 + (j + 1) * nnodes) for j in range(3)] + \
        [slice(len(theta) - 1, len(theta))]


def grad96_fd(w, theta, data, err, rel=1e-3, idx=None):
    """Central differences of the fp64 oracle chi^2 with h_j = rel x
    max(|theta_j|, mean |theta| of j's group), for the parameters idx (all)."""
    groups = grad96_groups(theta, len(w.disk.rnodes))
    mag = np.empty_like(theta)
    for gs in groups:
        mag[gs] = np.mean(np.abs(theta[gs]))
    h = rel * np.maximum(np.abs(theta), mag)
    idx = range(len(theta)) if idx is None else idx
    g = {}
    for j in idx:
        tp, tm = theta.copy(), theta.copy()
        tp[j] += h[j]
        tm[j] -= h[j]
        g[j] = (grad96_oracle_chi2(w, tp, data, err) - grad96_oracle_chi2(w, tm, data, err)) \
            / (2 * h[j])
    return np.array([g[j] for j in idx])


def grad96_reference_gradient(w, theta, data, err):
    """(chi^2, gradient) of the fp64 analytic reference (oracle.chi2_gradient_f64)."""
    from gbkfit_b200.adjoint import assemble_gradient, from_vector, interpolation_jacobian
    from oracle.oracle import chi2_gradient_f64
    p, scale = from_vector(w.disk, theta)
    c2, gsub, dscale = chi2_gradient_f64(w.disk.pack(p), w.geom, data, err, scale)
    return c2, assemble_gradient(interpolation_jacobian(w.disk), gsub, dscale)
