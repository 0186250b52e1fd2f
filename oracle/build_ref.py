"""Recipe: the reference's own collision table builders, compiled from their
sources under the reference checkout into oracle/_ref/ (test infrastructure).

Builds, for the 2-D hybrid model of pendulum_reduced_hybrid.m:130-141:
  oracle/_ref/getOmega_mex.so  from propagation/discrete/mex/sources/
                               pendulum_reduced_collision/src/{setup.cpp, getOmega.cu, mexOmega.cpp}
  oracle/_ref/getFcL_mex.so    from .../src/{setup.cpp, getFcL.cu, mexFcL.cpp}
linked against the host-memory MEX runtime of tests/mex_stub (mx_runtime.c,
built here as tests/mex_stub/_build/libmxstub.so) so tests call their
mexFunction through ctypes.  Nothing is copied out of the reference: nvcc
reads the sources where they lie.  oracle/ref_shim/cutensor.h stands in for
the legacy cuTENSOR header that setup.hpp includes (no cuTENSOR call is made
by these two builders).

Not built:
  getLambda.cu  its compute_lambda kernel reads lambda_indR[ind_lambda] before
                the ind_lambda < numR test (getLambda.cu:218-223), so the last
                block reads past the end of a device array; it is not run on
                shared GPUs.
  propagate.cu  needs the legacy cuTENSOR 1.x library (propagate.cu:41-88).

Usage: python oracle/build_ref.py [--reference DIR]   (default /root/reference)
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, '_ref')
STUB_DIR = os.path.join(ROOT, 'tests', 'mex_stub')
STUB_LIB = os.path.join(STUB_DIR, '_build', 'libmxstub.so')
COLL = os.path.join('propagation', 'discrete', 'mex', 'sources', 'pendulum_reduced_collision')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']


def nvcc() -> str:
    cand = os.path.join(os.environ.get('CUDA_HOME', '/usr/local/cuda'), 'bin', 'nvcc')
    return cand if os.path.exists(cand) else 'nvcc'


def build_stub(force: bool = False) -> str:
    """tests/mex_stub/_build/libmxstub.so (the MEX runtime stand-in)."""
    src = os.path.join(STUB_DIR, 'mx_runtime.c')
    if force or not os.path.exists(STUB_LIB) or os.path.getmtime(src) > os.path.getmtime(STUB_LIB):
        os.makedirs(os.path.dirname(STUB_LIB), exist_ok=True)
        subprocess.run(['gcc', '-std=gnu11', '-O2', '-shared', '-fPIC', '-Wall', '-I', STUB_DIR, src,
                        '-o', STUB_LIB], check=True)
    return STUB_LIB


def build(reference: str, force: bool = False) -> list[str]:
    build_stub(force)
    src = os.path.join(reference, COLL, 'src')
    inc = os.path.join(reference, COLL, 'include')
    if not os.path.isdir(src):
        return []
    os.makedirs(OUT, exist_ok=True)
    made = []
    for name, files in (('getOmega_mex', ['setup.cpp', 'getOmega.cu', 'mexOmega.cpp']),
                        ('getFcL_mex', ['setup.cpp', 'getFcL.cu', 'mexFcL.cpp'])):
        out = os.path.join(OUT, name + '.so')
        paths = [os.path.join(src, f) for f in files]
        if not force and os.path.exists(out) and all(os.path.getmtime(p) < os.path.getmtime(out) for p in paths):
            made.append(out)
            continue
        cmd = [nvcc(), *ARCH, '-O2', '-std=c++14', '-shared', '-Xcompiler', '-fPIC', '-w',
               '-I', inc, '-I', os.path.join(HERE, 'ref_shim'), '-I', STUB_DIR, *paths,
               '-L', os.path.dirname(STUB_LIB), '-lmxstub', '-Xlinker', '-rpath=$ORIGIN/../../tests/mex_stub/_build',
               '-o', out]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f'building {name} from the reference failed:\n{r.stderr[-4000:]}')
        made.append(out)
    return made


if __name__ == '__main__':
    ap = argparse.ArgumentParser()
    ap.add_argument('--reference', default='/root/reference')
    ap.add_argument('--force', action='store_true')
    a = ap.parse_args()
    for p in build(a.reference, a.force):
        print(p)
    sys.exit(0)
