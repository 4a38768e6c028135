"""In-tree build of libgbkb200.so for sm_100a (explicit nvcc, no JIT cache)."""

import glob
import os
import subprocess
import sys

_HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(_HERE)
CSRC = os.path.join(_HERE, 'csrc')
OUT = os.path.join(_HERE, 'libgbkb200.so')

NVCC_FLAGS = ['-gencode', 'arch=compute_100a,code=sm_100a', '-O3', '-lineinfo', '-std=c++17',
              '-Xcompiler', '-fPIC', '-shared', '-diag-suppress', '39']


def sources():
    return sorted(glob.glob(os.path.join(CSRC, '*.cu')))


def _stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = sources() + glob.glob(os.path.join(CSRC, '*.cuh')) + [
        os.path.join(ROOT, 'include', 'gbkb200.h')]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, checked=False):
    """Compile every .cu under csrc/ into gbkfit_b200/libgbkb200.so, or with
    checked=True into the bounds-checked debug build libgbkb200_checked.so."""
    out = OUT.replace('.so', '_checked.so') if checked else OUT
    if not force and not checked and not _stale():
        return out
    nvcc = os.environ.get('NVCC', 'nvcc')
    cmd = [nvcc] + NVCC_FLAGS + (['-DGBK_CHECKED'] if checked else []) + \
        ['-o', out + '.tmp'] + sources()
    if verbose:
        print(' '.join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True, cwd=ROOT)
    os.replace(out + '.tmp', out)
    return out


if __name__ == '__main__':
    build(force='--force' in sys.argv, verbose=True, checked='--checked' in sys.argv)
