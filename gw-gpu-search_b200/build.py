"""Builds libgwb200.so (every kernel and the C ABI) in-tree with nvcc for sm_100a.

    python gw-gpu-search_b200/build.py [--force] [-j N]

Objects go to gw-gpu-search_b200/_build/, the library to gw-gpu-search_b200/gwb200/lib/libgwb200.so. A source is
recompiled when it or any header is newer than its object. Only nvcc and the CUDA toolkit are needed (no GPU)."""
import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, 'csrc')
BUILD = os.path.join(HERE, '_build')
LIB = os.path.join(HERE, 'gwb200', 'lib', 'libgwb200.so')
INCLUDE = os.path.join(ROOT, 'include')
CUDA = os.environ.get('CUDA_HOME', '/usr/local/cuda')
NVCC = os.path.join(CUDA, 'bin', 'nvcc')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC', '-Xcompiler', '-fvisibility=hidden',
         '--expt-relaxed-constexpr', '-I', INCLUDE, '-I', CSRC]


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(('.cuh', '.h'))]
    return hs + [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith('.h')]


def _compile(src, force, verbose):
    obj = os.path.join(BUILD, os.path.basename(src) + '.o')
    newest = max(os.path.getmtime(p) for p in [src] + _headers())
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj
    cmd = [NVCC] + ARCH + FLAGS + ['-c', src, '-o', obj]
    if verbose:
        cmd.insert(1, '-Xptxas=-v')
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError('nvcc failed for %s:\n%s\n%s' % (src, r.stdout, r.stderr))
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


def build(force=False, jobs=8, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    srcs = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith('.cu'))
    with ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, verbose), srcs))
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ['-shared', '-o', LIB] + objs + ['-L' + os.path.join(CUDA, 'lib64'), '-lcufft',
                                                                 '-Xlinker', '-rpath=' + os.path.join(CUDA, 'lib64')]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError('link failed:\n%s\n%s' % (r.stdout, r.stderr))
    return LIB


if __name__ == '__main__':
    ap = argparse.ArgumentParser()
    ap.add_argument('--force', action='store_true')
    ap.add_argument('-j', type=int, default=8)
    ap.add_argument('-v', action='store_true', help='print ptxas register and shared-memory usage')
    a = ap.parse_args()
    print(build(a.force, a.j, a.v))
