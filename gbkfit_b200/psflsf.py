"""Point- and line-spread functions sampled on the data-cube grid.

Mirrors ``gbkfit/psflsf`` of the reference (core.py:18-118, psfs/psfs.py,
lsfs/lsfs.py): analytic profiles sampled on a centred grid, truncated at
8 scale lengths (PSFs: radially; LSFs: on the positive side only, as in
lsfs.py:96) and normalised to unit sum.  Sizes are rounded up to odd.
"""

import numpy as np

_CUTOFF = 8


def _roundu_odd(x):
    """math/math.py:25-36."""
    e = 2 * np.ceil(0.5 * x)
    return e + 1 if e - 1 < x else e - 1


def _rot_lh_z_py(x, y, theta):
    """math/math.py:85-90 (the Python convention, used for PSF position angles)."""
    s, c = np.sin(theta), np.cos(theta)
    return x * c + y * s, -x * s + y * c


def _grid_2d(size, step, offset, ratio, posa):
    """psfs.py:23-36."""
    cx = size[0] // 2 + offset[0]
    cy = size[1] // 2 + offset[1]
    x = (np.arange(size[0]) - cx) * step[0]
    y = (np.arange(size[1]) - cy) * step[1]
    x, y = _rot_lh_z_py(x[None, :], y[:, None], np.radians(posa))
    return np.sqrt(x * x + y * y / (ratio * ratio))


def _grid_1d(size, step, offset):
    """lsfs.py:23-25."""
    return (np.arange(size) - (size // 2 + offset)) * step


def _gauss(x, a, b, c):
    return a * np.exp(-(x - b) * (x - b) / (2 * c * c))


def _ggauss(x, a, b, c, d):
    return a * np.exp(-np.power(np.abs(x - b) / c, d))


def _lorentz(x, a, b, c):
    return a * c * c / ((x - b) * (x - b) + c * c)


def _moffat(x, a, b, c, d):
    return a / np.power(1 + ((x - b) / c) ** 2, d)


def gauss_fwhm_to_sigma(fwhm):
    return fwhm / np.sqrt(8 * np.log(2))


def moffat_fwhm_beta_to_alpha(fwhm, beta):
    return fwhm / (2 * np.sqrt(np.power(2, 1 / beta) - 1))


class PSF:
    """core.py:66-118."""

    def size(self, step, offset=(0, 0)):
        b = self._size_impl(step)
        return (int(_roundu_odd(b[0] + offset[0])), int(_roundu_odd(b[1] + offset[1])))

    def asarray(self, step, size=None, offset=(0, 0)):
        if size is None:
            size = self.size(step, offset)
        elif (size[0] + offset[0]) % 2 == 0 or (size[1] + offset[1]) % 2 == 0:
            raise RuntimeError(
                f"invalid PSF size: (size + offset) = ({size[0] + offset[0]}, "
                f"{size[1] + offset[1]}), but both values must be odd")
        return self._asarray_impl(step, size, offset)


class PSFPoint(PSF):
    def _size_impl(self, step):
        return 1, 1

    def _asarray_impl(self, step, size, offset):
        d = np.zeros((size[1], size[0]))
        d[size[1] // 2 + offset[1], size[0] // 2 + offset[0]] = 1
        return d


class _PSFAnalytic(PSF):
    _scale_attr = 'sigma'

    def _size_impl(self, step):
        s = getattr(self, self._scale_attr)
        return 2 * _CUTOFF * s / step[0], 2 * _CUTOFF * s / step[1]

    def _asarray_impl(self, step, size, offset):
        r = _grid_2d(size, step, offset, self.ratio, self.posa)
        d = self._fun(r)
        d[r > _CUTOFF * getattr(self, self._scale_attr)] = 0
        return d / np.sum(d)


class PSFGauss(_PSFAnalytic):
    """psfs.py:79-120."""

    def __init__(self, sigma, ratio=1.0, posa=0.0):
        self.sigma, self.ratio, self.posa = sigma, ratio, posa

    def _fun(self, r):
        return _gauss(r, 1, 0, self.sigma)


class PSFGGauss(_PSFAnalytic):
    _scale_attr = 'alpha'

    def __init__(self, alpha, beta, ratio=1.0, posa=0.0):
        self.alpha, self.beta, self.ratio, self.posa = alpha, beta, ratio, posa

    def _fun(self, r):
        return _ggauss(r, 1, 0, self.alpha, self.beta)


class PSFLorentz(_PSFAnalytic):
    _scale_attr = 'gamma'

    def __init__(self, gamma, ratio=1.0, posa=0.0):
        self.gamma, self.ratio, self.posa = gamma, ratio, posa

    def _fun(self, r):
        return _lorentz(r, 1, 0, self.gamma)


class PSFMoffat(_PSFAnalytic):
    """psfs.py:219-268."""
    _scale_attr = 'alpha'

    def __init__(self, alpha, beta, ratio=1.0, posa=0.0):
        self.alpha, self.beta, self.ratio, self.posa = alpha, beta, ratio, posa

    def _fun(self, r):
        return _moffat(r, 1, 0, self.alpha, self.beta)


class LSF:
    """core.py:18-63."""

    def size(self, step, offset=0):
        return int(_roundu_odd(self._size_impl(step) + offset))

    def asarray(self, step, size=None, offset=0):
        if size is None:
            size = self.size(step, offset)
        elif (size + offset) % 2 == 0:
            raise RuntimeError(
                f"invalid LSF size: (size + offset) = ({size} + {offset} = "
                f"{size + offset}), but it must be odd")
        return self._asarray_impl(step, size, offset)


class LSFPoint(LSF):
    def _size_impl(self, step):
        return 1

    def _asarray_impl(self, step, size, offset):
        d = np.zeros(size)
        d[size // 2 + offset] = 1
        return d


class _LSFAnalytic(LSF):
    _scale_attr = 'sigma'

    def _size_impl(self, step):
        return 2 * _CUTOFF * getattr(self, self._scale_attr) / step

    def _asarray_impl(self, step, size, offset):
        z = _grid_1d(size, step, offset)
        d = self._fun(z)
        d[z > _CUTOFF * getattr(self, self._scale_attr)] = 0   # lsfs.py:96 (one-sided)
        return d / np.sum(d)


class LSFGauss(_LSFAnalytic):
    """lsfs.py:64-97."""

    def __init__(self, sigma):
        self.sigma = sigma

    def _fun(self, z):
        return _gauss(z, 1, 0, self.sigma)


class LSFGGauss(_LSFAnalytic):
    _scale_attr = 'alpha'

    def __init__(self, alpha, beta):
        self.alpha, self.beta = alpha, beta

    def _fun(self, z):
        return _ggauss(z, 1, 0, self.alpha, self.beta)


class LSFLorentz(_LSFAnalytic):
    _scale_attr = 'gamma'

    def __init__(self, gamma):
        self.gamma = gamma

    def _fun(self, z):
        return _lorentz(z, 1, 0, self.gamma)


class LSFMoffat(_LSFAnalytic):
    _scale_attr = 'alpha'

    def __init__(self, alpha, beta):
        self.alpha, self.beta = alpha, beta

    def _fun(self, z):
        return _moffat(z, 1, 0, self.alpha, self.beta)
