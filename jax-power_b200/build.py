"""Build the C-ABI CUDA library ``jaxpower_b200/libjaxpower_b200.so`` in-tree.

    python jax-power_b200/build.py [--verbose]

Compiles every ``csrc/*.cu`` for sm_100a with nvcc and links them, with cuFFT,
into one shared library next to the Python package.  Object files go to
``csrc/_build/`` (git-ignored); recompilation is skipped for up-to-date objects.
"""
import argparse
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
BUILD = os.path.join(CSRC, '_build')
INCLUDE = os.path.join(os.path.dirname(HERE), 'include')
OUT = os.path.join(HERE, 'jaxpower_b200', 'libjaxpower_b200.so')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']


def nvcc():
    path = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
    if not os.path.exists(path):
        raise RuntimeError('nvcc not found')
    return path


def cuda_lib_dir():
    return os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(nvcc()))), 'lib64')


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, '*.cu')))
    headers = glob.glob(os.path.join(CSRC, '*.cuh')) + glob.glob(os.path.join(INCLUDE, '*.h'))
    newest_header = max((os.path.getmtime(h) for h in headers), default=0.)
    objects = []
    flags = ARCH + ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC,-O3', '-I', INCLUDE]
    if verbose:
        flags += ['-Xptxas', '-v']
    for src in sources:
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + '.o')
        objects.append(obj)
        if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
                and os.path.getmtime(obj) >= newest_header):
            continue
        cmd = [nvcc(), '-c', src, '-o', obj] + flags
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError('nvcc failed for {}:\n{}{}'.format(src, res.stdout, res.stderr))
        if verbose:
            sys.stdout.write(res.stdout + res.stderr)
    libdir = cuda_lib_dir()
    cmd = [nvcc(), '-shared', '-o', OUT] + ARCH + objects + [
        '-L' + libdir, '-lcufft', '-Xlinker', '-rpath,' + libdir]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError('link failed:\n{}{}'.format(res.stdout, res.stderr))
    return OUT


if __name__ == '__main__':
    parser = argparse.ArgumentParser()
    parser.add_argument('--verbose', action='store_true')
    parser.add_argument('--force', action='store_true')
    args = parser.parse_args()
    print(build(verbose=args.verbose, force=args.force))
