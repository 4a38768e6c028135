"""Synthetic workloads of the model-evaluation path (seeded, no datasets).

Each builder returns a ``Workload``: a disk layout, one or more parameter
sets, the padded evaluation geometry computed with the reference's DCube rules
(gbkfit/model/dmodels/_dcube.py:128-243), the PSF x LSF kernel cube and, for
objective workloads, a seeded noisy data cube.

* ``smdisk_cube64``: thin smooth disk, 64x64x64 cube, 20 rings on 0-30 px,
  exponential surface brightness (scale 8 px), arctan rotation curve
  (vmax 200 km/s, r_t 4 px), dispersion 20 km/s, incl 60, PA 45, centre
  (32, 32), vsys 0; Gaussian PSF FWHM 2.5 px, Gaussian LSF FWHM 2 channels
  (10 km/s channels).
* ``mcdisk_cube256``: thick cloud disk, 256x256x128 cube, exponential disk
  (scale 20 px), sech2 height (z0 2 px), lramp rotation curve (220 km/s, 10 px),
  dispersion 15 km/s, incl 70, PA 30, ~1e7 clouds; Moffat PSF FWHM 3 px
  beta 2.5, Gaussian LSF FWHM 2 channels.
* ``smdisk_batch128``: B parameter sets on 128x128x96 cubes with 30 rings,
  node-wise vrot ~ U(50, 300), vdisp ~ U(5, 40), surface brightness
  exp(N(0, 0.5)), incl ~ U(20, 80), PA ~ U(0, 360); data = model + N(0, (2%
  peak)^2); Gaussian PSF FWHM 3 px, Gaussian LSF FWHM 1.5 channels.
* ``smdisk_grad96``: 96x96x64 cube, 20 rings, node-wise vrot/vdisp/surface
  brightness (the 66-parameter gradient workload).
* ``serving_stream``: Poisson-arriving requests, 70 % smdisk / 30 % mcdisk,
  against datasets with log-uniform sides 32-256 px and 32-192 channels, each
  with its own Gaussian PSF (FWHM 1.5-4 px) and LSF (FWHM 1-3 channels);
  mcdisk requests draw 1e5-1e7 clouds log-uniformly.
"""

import numpy as np

from . import psflsf, traits
from .disk import Disk


def _odd_offset(n):
    """_dcube.py:195: offset -1 for even sizes."""
    return (n % 2) - 1


def fft_optimal_shape(shape, threshold=32):
    """driver/backend.py:51-59."""
    out = []
    for dim in shape:
        po2 = 1
        while po2 < dim:
            po2 *= 2
        mul = dim - dim % threshold + threshold if dim % threshold else dim
        out.append(int(po2 if po2 <= threshold else mul))
    return tuple(out)


def dcube_geometry(size, step, rpix, rval, scale, psf, lsf, pad=None):
    """_dcube.py:128-179: (zero_lo, size_hi, step_hi, zero_hi, edge_hi,
    kernel_size) of a DCube."""
    zero = tuple(rval[i] - rpix[i] * step[i] for i in range(3))
    size_hi = tuple(int(size[i]) * int(scale[i]) for i in range(3))
    step_hi = tuple(step[i] / scale[i] for i in range(3))
    edge = (0, 0, 0)
    ksize = (1, 1, 1)
    if psf is not None or lsf is not None:
        ps = psf.size(step_hi[:2]) if psf else (1, 1)
        ls = lsf.size(step_hi[2]) if lsf else 1
        ksize = (ps[0], ps[1], ls)
        need = tuple(size_hi[i] + ksize[i] - 1 for i in range(3))
        size_hi = fft_optimal_shape(need) if pad is None else pad(need)
        edge = tuple(k // 2 for k in ksize)
    zero_hi = tuple(zero[i] - step[i] / 2 - (edge[i] - 0.5) * step_hi[i] for i in range(3))
    return zero, size_hi, step_hi, zero_hi, edge, ksize


class Geometry:
    """Low-res cube and its padded ("hi") evaluation grid (_dcube.py:128-243),
    for scale (1, 1, 1)."""

    def __init__(self, size, step, rpix, rval, psf, lsf, pad=None):
        self.size = tuple(int(v) for v in size)
        self.step = tuple(float(v) for v in step)
        self.psf, self.lsf = psf, lsf
        (self.zero, self.size_hi, _, self.zero_hi, self.edge,
         self.kernel_size) = dcube_geometry(self.size, self.step, rpix, rval, (1, 1, 1), psf, lsf,
                                            pad)

    def pcube(self, dtype=np.float32):
        """_dcube.py:189-207: PSF x LSF on the padded grid, rolled to (0,0,0)."""
        nx, ny, nz = self.size_hi
        off = [_odd_offset(n) for n in self.size_hi]
        psf = self.psf if self.psf else psflsf.PSFPoint()
        lsf = self.lsf if self.lsf else psflsf.LSFPoint()
        p = psf.asarray(self.step[:2], (nx, ny), (off[0], off[1]))
        l_ = lsf.asarray(self.step[2], nz, off[2])
        cube = (p * l_[:, None, None]).astype(dtype)
        return np.roll(cube, np.array(cube.shape) // 2 + 1, axis=(0, 1, 2))

    def spat(self, thick=False, spat_z=None):
        """(spat_size, spat_step, spat_zero) of the gmodel on the padded grid
        (kinematics_2d.py:76-91 / kinematics_3d.py:88-139)."""
        sx, sy = self.size_hi[0], self.size_hi[1]
        if not thick:
            return (sx, sy, 1), (self.step[0], self.step[1], 0.0), (self.zero_hi[0],
                                                                    self.zero_hi[1], 0.0)
        i = int(sx < sy)
        sz = spat_z if spat_z is not None else (sx, sy)[i]
        stz = (self.step[0], self.step[1])[i]
        zz = -(sz / 2 - 0.5) * stz
        return (sx, sy, sz), (self.step[0], self.step[1], stz), (self.zero_hi[0],
                                                                 self.zero_hi[1], zz)

    def spec(self):
        return self.size_hi[2], self.step[2], self.zero_hi[2]


class Workload:
    def __init__(self, name, disk, params, geom, thick=False, cflux=None, data=None,
                 error=None, nsets=1, extra=None):
        self.name = name
        self.disk = disk
        self.params = params
        self.geom = geom
        self.thick = thick
        self.cflux = cflux
        self.data = data
        self.error = error
        self.nsets = nsets
        self.extra = extra or {}

    def geometry_args(self, spat_z=None):
        ss, st, sz = self.geom.spat(self.thick, spat_z)
        n, s, z = self.geom.spec()
        return dict(loose=self.disk.loose, tilted=self.disk.tilted, spat_size=ss, spat_step=st,
                    spat_zero=sz, spec_size=n, spec_step=s, spec_zero=z, opacity=None)


def smdisk_cube64():
    rnodes = np.linspace(0, 30, 20)
    disk = Disk(False, False, rnodes, traits=dict(
        rpt=[traits.bpt('exponential')], vpt=[traits.vpt('tan_arctan')],
        dpt=[traits.dpt('uniform')]))
    params = dict(vsys=0.0, xpos=32.0, ypos=32.0, posa=45.0, incl=60.0,
                  bpt_a=1.0, bpt_s=8.0, vpt_rt=4.0, vpt_vt=200.0, dpt_a=20.0)
    psf = psflsf.PSFGauss(psflsf.gauss_fwhm_to_sigma(2.5))
    lsf = psflsf.LSFGauss(psflsf.gauss_fwhm_to_sigma(2 * 10.0))
    geom = Geometry((64, 64, 64), (1, 1, 10), (0, 0, 31.5), (0, 0, 0), psf, lsf)
    return Workload('smdisk_cube64', disk, params, geom)


def mcdisk_cube256(nclouds=10_000_000):
    rnodes = np.linspace(0, 120, 61)
    disk = Disk(False, False, rnodes, traits=dict(
        rpt=[traits.bpt('exponential')], rht=[traits.bht('sech2')],
        vpt=[traits.vpt('tan_lramp')], vht=[traits.vht_one()],
        dpt=[traits.dpt('uniform')], dht=[traits.dht_one()]))
    params = dict(vsys=0.0, xpos=128.0, ypos=128.0, posa=30.0, incl=70.0,
                  bpt_a=1.0, bpt_s=20.0, bht_s=2.0, vpt_rt=10.0, vpt_vt=220.0, dpt_a=15.0)
    psf = psflsf.PSFMoffat(psflsf.moffat_fwhm_beta_to_alpha(3.0, 2.5), 2.5)
    lsf = psflsf.LSFGauss(psflsf.gauss_fwhm_to_sigma(2 * 10.0))
    geom = Geometry((256, 256, 128), (1, 1, 10), (0, 0, 63.5), (0, 0, 0), psf, lsf)
    # cloud flux so that the ring integrals sum to about nclouds clouds
    total = np.sum(disk.traits['rpt'][0].integrate(dict(a=1.0, s=20.0), disk.subrnodes[1:-1]))
    cflux = float(total / nclouds)
    return Workload('mcdisk_cube256', disk, params, geom, thick=True, cflux=cflux)


def _batch_params(rng, nsets, nnodes):
    return dict(
        vsys=np.zeros(nsets), xpos=np.full(nsets, 64.0), ypos=np.full(nsets, 64.0),
        posa=rng.uniform(0, 360, nsets), incl=rng.uniform(20, 80, nsets),
        bpt_a=np.exp(rng.normal(0, 0.5, (nsets, nnodes))),
        vpt_vt=rng.uniform(50, 300, (nsets, nnodes)),
        dpt_a=rng.uniform(5, 40, (nsets, nnodes)))


def smdisk_batch128(nsets=512, seed=1234, size=(128, 128, 96), nnodes=30):
    """Node-wise surface brightness uses natural-log amplitudes exp(N(0, 0.5))."""
    rng = np.random.default_rng(seed)
    rnodes = np.linspace(0, 60, nnodes)
    disk = Disk(False, False, rnodes, traits=dict(
        rpt=[traits.bpt('nw_uniform')], vpt=[traits.vpt('nw_tan_uniform')],
        dpt=[traits.dpt('nw_uniform')]))
    params = _batch_params(rng, nsets, nnodes)
    psf = psflsf.PSFGauss(psflsf.gauss_fwhm_to_sigma(3.0))
    lsf = psflsf.LSFGauss(psflsf.gauss_fwhm_to_sigma(1.5 * 10.0))
    nx, ny, nz = size
    geom = Geometry(size, (1, 1, 10), (0, 0, (nz - 1) / 2), (0, 0, 0), psf, lsf)
    truth = _batch_params(np.random.default_rng(seed + 1), 1, nnodes)
    truth = {k: v[0] for k, v in truth.items()}
    return Workload('smdisk_batch128', disk, params, geom, nsets=nsets,
                    extra=dict(truth=truth, noise_seed=seed + 2, noise_frac=0.02))


def smdisk_grad96(seed=99):
    """The differentiable configuration: 96x96x64 cube, 20 rings on 0-40 px,
    node-wise surface brightness, rotation and dispersion, PSF FWHM 2.5 px,
    LSF FWHM 2 channels, 66 parameters (geometry 5, nodes 3 x 20, scale).

    The surface brightness is tapered to 0 at the last node: the disk edge
    (r = last node) cuts the emission off, and with zero brightness there the
    model is continuous in the geometry parameters, so finite differences
    see only the derivatives that the adjoint computes.  ``params`` is the
    evaluation point, ``extra['truth']`` the parameters of the data cube
    (noise of sigma = noise_frac x peak), ``extra['scale']`` the evaluation
    scale."""
    rng = np.random.default_rng(seed)
    nn = 20
    rnodes = np.linspace(0, 40, nn)
    disk = Disk(False, False, rnodes, traits=dict(
        rpt=[traits.bpt('nw_uniform')], vpt=[traits.vpt('nw_tan_uniform')],
        dpt=[traits.dpt('nw_uniform')]))
    taper = 1 - (rnodes / rnodes[-1]) ** 4
    truth = dict(vsys=5.0, xpos=48.3, ypos=47.6, posa=35.0, incl=55.0,
                 bpt_a=np.exp(-rnodes / 12.0) * (1 + 0.1 * rng.standard_normal(nn)) * taper,
                 vpt_vt=200 * np.tanh(rnodes / 6.0) + 5 * rng.standard_normal(nn),
                 dpt_a=20 + 3 * rng.standard_normal(nn))
    params = dict(vsys=8.0, xpos=48.7, ypos=47.3, posa=37.0, incl=52.0,
                  bpt_a=truth['bpt_a'] * (1 + 0.05 * rng.standard_normal(nn)),
                  vpt_vt=truth['vpt_vt'] + 4 * rng.standard_normal(nn),
                  dpt_a=truth['dpt_a'] + 2 * rng.standard_normal(nn))
    psf = psflsf.PSFGauss(psflsf.gauss_fwhm_to_sigma(2.5))
    lsf = psflsf.LSFGauss(psflsf.gauss_fwhm_to_sigma(2 * 10.0))
    geom = Geometry((96, 96, 64), (1, 1, 10), (0, 0, 31.5), (0, 0, 0), psf, lsf)
    return Workload('smdisk_grad96', disk, params, geom,
                    extra=dict(truth=truth, scale=1.1, noise_seed=seed + 1, noise_frac=0.02))


def set_params(w, i):
    """Parameter set i of a batched workload as a single-set dict."""
    return {k: (v[i] if np.ndim(v) and np.shape(v)[0] == w.nsets else v)
            for k, v in w.params.items()}


class ServingStream:
    """Datasets and requests of a serving run (see serving_stream)."""

    def __init__(self, datasets, requests, arrivals):
        self.datasets = datasets        # list of dict(key, geom, data, error, smdisk, mcdisk)
        self.requests = requests        # list of dict(dataset, kind, params, cflux, thick)
        self.arrivals = arrivals        # seconds from the start, increasing


def _loguniform(rng, lo, hi, n=None):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), n))


def serving_stream(nrequests=10000, ndatasets=64, rate=2000.0, seed=7, max_side=256,
                   max_channels=192, max_clouds=1e7, nrings=30):
    """A request stream of samplers and fitters: ndatasets datasets (cube
    sides log-uniform 32-max_side px, channels 32-max_channels, 10 km/s
    channels; Gaussian PSF FWHM U(1.5, 4) px, Gaussian LSF FWHM U(1, 3)
    channels; data and error: seeded noise), and nrequests requests arriving
    as a Poisson process of the given rate (1/s), each against a uniformly
    drawn dataset: 70 % smdisk (thin disk, node-wise surface brightness
    exp(N(0, 0.5)), rotation U(50, 300) km/s, dispersion U(5, 40) km/s,
    incl U(20, 80), PA U(0, 360), as the batched configuration) and 30 %
    mcdisk (thick exponential disk with a sech2 height profile, flat rotation
    beyond a linear rise, constant dispersion, clouds log-uniform 1e5 to
    max_clouds)."""
    rng = np.random.default_rng(seed)
    datasets = []
    for i in range(ndatasets):
        nx, ny = (int(round(v)) for v in _loguniform(rng, 32, max_side, 2))
        nz = int(round(_loguniform(rng, 32, max_channels)))
        psf = psflsf.PSFGauss(psflsf.gauss_fwhm_to_sigma(rng.uniform(1.5, 4.0)))
        lsf = psflsf.LSFGauss(psflsf.gauss_fwhm_to_sigma(rng.uniform(1.0, 3.0) * 10.0))
        geom = Geometry((nx, ny, nz), (1, 1, 10), (0, 0, (nz - 1) / 2), (0, 0, 0), psf, lsf)
        rmax = 0.45 * min(nx, ny)
        sm = Disk(False, False, np.linspace(0, rmax, nrings), traits=dict(
            rpt=[traits.bpt('nw_uniform')], vpt=[traits.vpt('nw_tan_uniform')],
            dpt=[traits.dpt('nw_uniform')]))
        mc = Disk(False, False, np.linspace(0, rmax, 21), traits=dict(
            rpt=[traits.bpt('exponential')], rht=[traits.bht('sech2')],
            vpt=[traits.vpt('tan_lramp')], vht=[traits.vht_one()],
            dpt=[traits.dpt('uniform')], dht=[traits.dht_one()]))
        sigma = 0.01
        data = rng.standard_normal((nz, ny, nx), dtype=np.float32) * np.float32(sigma)
        err = np.full((nz, ny, nx), sigma, np.float32)
        datasets.append(dict(key=i, geom=geom, data=data, error=err, smdisk=sm, mcdisk=mc,
                             centre=((nx - 1) / 2, (ny - 1) / 2)))
    requests = []
    for j in range(nrequests):
        d = datasets[int(rng.integers(ndatasets))]
        cx, cy = d['centre']
        if rng.uniform() < 0.7:
            disk = d['smdisk']
            nn = len(disk.rnodes)
            params = dict(vsys=0.0, xpos=cx, ypos=cy, posa=rng.uniform(0, 360),
                          incl=rng.uniform(20, 80), bpt_a=np.exp(rng.normal(0, 0.5, nn)),
                          vpt_vt=rng.uniform(50, 300, nn), dpt_a=rng.uniform(5, 40, nn))
            requests.append(dict(dataset=d['key'], kind='smdisk', params=params, cflux=None,
                                 thick=False))
        else:
            disk = d['mcdisk']
            rmax = disk.rnodes[-1]
            params = dict(vsys=0.0, xpos=cx, ypos=cy, posa=rng.uniform(0, 360),
                          incl=rng.uniform(20, 80), bpt_a=1.0, bpt_s=rmax / 4,
                          bht_s=rng.uniform(1, 3), vpt_rt=rmax / 10,
                          vpt_vt=rng.uniform(150, 300), dpt_a=rng.uniform(10, 30))
            n = _loguniform(rng, 1e5, max_clouds)
            total = np.sum(disk.traits['rpt'][0].integrate(dict(a=1.0, s=rmax / 4),
                                                           disk.subrnodes[1:-1]))
            requests.append(dict(dataset=d['key'], kind='mcdisk', params=params,
                                 cflux=float(total / n), thick=True))
    arrivals = np.cumsum(rng.exponential(1.0 / rate, nrequests))
    return ServingStream(datasets, requests, arrivals)
