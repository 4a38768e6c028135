"""Imports the reference's Python package from a GBKFIT checkout for fixture
generation, with stand-ins for the modules it imports but the model path does
not use (astropy, ruamel.yaml, pandas) and for its generated version file."""

import os
import sys
import types


def reference_src():
    """src/ of the GBKFIT checkout the fixtures are generated from:
    $GBKFIT_REFERENCE/src, else the checkout of the build container."""
    return os.path.join(os.environ.get('GBKFIT_REFERENCE', '/root/reference'), 'src')


def import_reference(src=None):
    src = src or reference_src()
    if src not in sys.path:
        sys.path.insert(0, src)

    class _Any:
        def __init__(self, *a, **k):
            pass

    def mod(name, **attrs):
        m = types.ModuleType(name)
        m.__dict__.update(attrs)
        sys.modules[name] = m
        return m

    astropy = mod('astropy')
    astropy.wcs = mod('astropy.wcs', WCS=_Any)
    astropy.io = mod('astropy.io')
    astropy.io.fits = mod('astropy.io.fits', Header=_Any, PrimaryHDU=_Any, HDUList=_Any)
    astropy.units = mod('astropy.units')
    ruamel = mod('ruamel')
    ruamel.yaml = mod('ruamel.yaml', YAML=_Any)
    mod('gbkfit._version', __version__='0')
    import gbkfit  # noqa: F401
    return gbkfit
