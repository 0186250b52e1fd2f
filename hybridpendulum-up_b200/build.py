"""Build the sm_100a shared library libhp.so in-tree with nvcc.

Usage: python build.py [--jobs N] [--force]
The library is the product: every entry point of include/hp.h lives in it.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
OUT = os.path.join(HERE, 'libhp.so')
# the per-bandlimit transform kernels are split over transform_b0..3.cu (B mod 4)
# so that they compile in parallel; the longest units first
SOURCES = ['transform_b0.cu', 'transform_b1.cu', 'transform_b2.cu', 'transform_b3.cu', 'deriv.cu', 'adjoint.cu',
           'transform.cu', 'tables.cu', 'prod.cu', 'capi.cu', 'collision.cu', 'stats.cu', 'init.cu', 'batch.cu',
           'real.cu', 'tc_beta.cu', 'tune.cu']
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC', '--expt-relaxed-constexpr',
         '-Xptxas', '-warn-spills']


def nvcc() -> str:
    cand = os.path.join(os.environ.get('CUDA_HOME', '/usr/local/cuda'), 'bin', 'nvcc')
    return cand if os.path.exists(cand) else 'nvcc'


def _obj(src: str) -> str:
    return os.path.join(HERE, '_build', src.replace('.cu', '.o'))


def _stale(src: str) -> bool:
    o = _obj(src)
    if not os.path.exists(o):
        return True
    deps = [os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in os.listdir(CSRC)
                                          if h.endswith(('.cuh', '.hpp'))]
    deps.append(os.path.join(HERE, '..', 'include', 'hp.h'))
    return any(os.path.getmtime(d) > os.path.getmtime(o) for d in deps)


def build(jobs: int = 8, force: bool = False, verbose: bool = False) -> str:
    os.makedirs(os.path.join(HERE, '_build'), exist_ok=True)
    todo = [s for s in SOURCES if force or _stale(s)]

    def compile_one(src):
        cmd = [nvcc(), *ARCH, *FLAGS, '-c', os.path.join(CSRC, src), '-o', _obj(src)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f'nvcc failed for {src}:\n{r.stderr}')
        return src, r.stderr

    with ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
        for src, err in ex.map(compile_one, todo):
            if verbose and err.strip():
                print(f'[{src}]\n{err}', file=sys.stderr)
    if todo or not os.path.exists(OUT):
        cmd = [nvcc(), *ARCH, '-shared', '-o', OUT, *[_obj(s) for s in SOURCES], '-lcudart']
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f'link failed:\n{r.stderr}')
    return OUT


if __name__ == '__main__':
    ap = argparse.ArgumentParser()
    ap.add_argument('--jobs', type=int, default=8)
    ap.add_argument('--force', action='store_true')
    ap.add_argument('-v', '--verbose', action='store_true')
    a = ap.parse_args()
    print(build(a.jobs, a.force, a.verbose))
