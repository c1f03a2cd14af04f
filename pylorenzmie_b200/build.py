'''Build the in-tree CUDA library ``pylorenzmie_b200/_lib/liblmb200.so``.

    python -m pylorenzmie_b200.build            # build if sources changed
    python -m pylorenzmie_b200.build --force

The library is compiled for sm_100a only (``-gencode
arch=compute_100a,code=sm_100a``) with nvcc, as a plain shared object
whose C ABI is declared in ``include/lmb200.h``.  No GPU is needed to
build.
'''
import argparse
import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / 'csrc'
INCLUDE = ROOT / 'include'
LIBDIR = PKG / '_lib'
LIBRARY = LIBDIR / 'liblmb200.so'
SOURCES = ['lmb200.cu', 'lmb_host.cpp']
GENCODE = ['-gencode', 'arch=compute_100a,code=sm_100a']


def nvcc_path():
    for cand in (os.environ.get('NVCC'), shutil.which('nvcc'),
                 '/usr/local/cuda/bin/nvcc'):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError('nvcc not found: set NVCC or put CUDA on PATH')


def _inputs():
    files = [CSRC / s for s in SOURCES]
    files += sorted(CSRC.glob('*.cuh'))
    files += sorted(INCLUDE.glob('*.h'))
    return files


def up_to_date():
    if not LIBRARY.exists():
        return False
    t = LIBRARY.stat().st_mtime
    return all(f.stat().st_mtime <= t for f in _inputs())


def command(output=LIBRARY, extra=()):
    return [nvcc_path(), *GENCODE, '-lineinfo', '-O3', '-std=c++17',
            '-shared', '-Xcompiler', '-fPIC', '-Xcompiler', '-O3',
            f'-I{INCLUDE}', f'-I{CSRC}', *extra,
            *[str(CSRC / s) for s in SOURCES], '-o', str(output)]


def build(force=False, verbose=False):
    '''Compile the library if a source is newer than it; return its path.'''
    if not force and up_to_date():
        return LIBRARY
    LIBDIR.mkdir(exist_ok=True)
    tmp = LIBRARY.with_suffix('.so.tmp')
    cmd = command(tmp, ('-Xptxas', '-v') if verbose else ())
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError('nvcc failed:\n' + ' '.join(cmd) + '\n' +
                           proc.stdout + proc.stderr)
    if verbose:
        print(proc.stdout + proc.stderr)
    os.replace(tmp, LIBRARY)
    return LIBRARY


if __name__ == '__main__':
    ap = argparse.ArgumentParser()
    ap.add_argument('--force', action='store_true')
    ap.add_argument('--verbose', action='store_true')
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
