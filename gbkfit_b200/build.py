"""In-tree build of libgbkb200.so for sm_100a (explicit nvcc, no JIT cache)."""

import glob
import os
import shutil
import subprocess
import sys
import tempfile
from concurrent.futures import ThreadPoolExecutor

_HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(_HERE)
CSRC = os.path.join(_HERE, 'csrc')
OUT = os.path.join(_HERE, 'libgbkb200.so')

NVCC_FLAGS = ['-gencode', 'arch=compute_100a,code=sm_100a', '-O3', '-lineinfo', '-std=c++17',
              '-Xcompiler', '-fPIC', '-diag-suppress', '39']


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
    """Compile every .cu under csrc/ (one object per file, in parallel) and
    link gbkfit_b200/libgbkb200.so, or with checked=True the bounds-checked
    debug build libgbkb200_checked.so."""
    out = OUT.replace('.so', '_checked.so') if checked else OUT
    if not force and not checked and not _stale():
        return out
    nvcc = os.environ.get('NVCC', 'nvcc')
    flags = NVCC_FLAGS + (['-DGBK_CHECKED'] if checked else [])
    tmp = tempfile.mkdtemp(prefix='gbkb200_build_')
    try:
        objs = [os.path.join(tmp, os.path.basename(src)[:-3] + '.o') for src in sources()]

        def compile_one(src_obj):
            cmd = [nvcc] + flags + ['-c', '-o', src_obj[1], src_obj[0]]
            if verbose:
                print(' '.join(cmd), file=sys.stderr)
            return subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True)

        with ThreadPoolExecutor(max_workers=max(1, min(len(objs), os.cpu_count() or 1))) as ex:
            results = list(ex.map(compile_one, zip(sources(), objs)))
        for src, r in zip(sources(), results):
            if r.stderr.strip() and (verbose or r.returncode):
                print(r.stderr, file=sys.stderr)
            if r.returncode:
                raise subprocess.CalledProcessError(r.returncode, 'nvcc ' + src)
        cmd = [nvcc, '-gencode', 'arch=compute_100a,code=sm_100a', '-shared', '-o',
               out + '.tmp'] + objs
        if verbose:
            print(' '.join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True, cwd=ROOT)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    os.replace(out + '.tmp', out)
    return out


if __name__ == '__main__':
    build(force='--force' in sys.argv, verbose=True, checked='--checked' in sys.argv)
