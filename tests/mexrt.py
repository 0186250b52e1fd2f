"""Runs MEX gateways without MATLAB: builds them against the host-memory MEX
runtime of tests/mex_stub (mx_runtime.c) and calls their mexFunction through
ctypes, with numpy arrays in and out (column-major, as MATLAB holds them).

Used for the library's own gateways (hybridpendulum-up_b200/mex/hp_mex.c,
linked against libhp.so) and for the reference's collision table builders
that oracle/build_ref.py compiles into oracle/_ref.  Test infrastructure."""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
STUB_DIR = os.path.join(HERE, 'mex_stub')
BUILD = os.path.join(STUB_DIR, '_build')
PKG = os.path.join(ROOT, 'hybridpendulum-up_b200')
GATEWAY_SRC = os.path.join(PKG, 'mex', 'hp_mex.c')

# class ids of the public matrix.h (mirrored in tests/mex_stub/mex.h)
CELL, LOGICAL, CHAR, DOUBLE, SINGLE, INT16, INT32 = 1, 3, 4, 6, 7, 10, 12
_NP = {DOUBLE: np.float64, SINGLE: np.float32, INT16: np.int16, INT32: np.int32, LOGICAL: np.bool_}

_stub = None


def stub():
    """The MEX runtime stand-in, loaded once with global symbols (the gateways
    resolve mx* and mex* against it)."""
    global _stub
    if _stub is None:
        import sys
        sys.path.insert(0, ROOT)
        try:
            from oracle import build_ref
        finally:
            sys.path.pop(0)
        path = build_ref.build_stub()
        lib = ctypes.CDLL(path, mode=ctypes.RTLD_GLOBAL)
        vp, sz = ctypes.c_void_p, ctypes.c_size_t
        lib.mxstub_new.restype = vp
        lib.mxstub_new.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(sz)]
        lib.mxstub_string.restype = vp
        lib.mxstub_string.argtypes = [ctypes.c_char_p]
        lib.mxstub_free.argtypes = [vp]
        lib.mxstub_data.restype = vp
        lib.mxstub_data.argtypes = [vp]
        for f in ('mxstub_class', 'mxstub_is_complex', 'mxstub_ndim'):
            getattr(lib, f).restype = ctypes.c_int
            getattr(lib, f).argtypes = [vp]
        lib.mxstub_dim.restype = sz
        lib.mxstub_dim.argtypes = [vp, ctypes.c_int]
        lib.mxstub_call.restype = ctypes.c_int
        lib.mxstub_call.argtypes = [vp, ctypes.c_int, ctypes.POINTER(vp), ctypes.c_int, ctypes.POINTER(vp)]
        lib.mxstub_last_error.restype = ctypes.c_char_p
        lib.mxstub_run_atexit.argtypes = []
        _stub = lib
    return _stub


def build_gateway(define: str, name: str, extra=()) -> str:
    """hp_mex.c compiled with -D<define> into tests/mex_stub/_build/<name>.so."""
    stub()
    out = os.path.join(BUILD, name + '.so')
    deps = [GATEWAY_SRC, os.path.join(ROOT, 'include', 'hp.h'), os.path.join(STUB_DIR, 'mex.h')]
    if os.path.exists(out) and all(os.path.getmtime(d) < os.path.getmtime(out) for d in deps):
        return out
    cmd = ['gcc', '-std=c99', '-O2', '-shared', '-fPIC', '-Wall', '-Werror', f'-D{define}', *extra,
           '-I', STUB_DIR, '-I', os.path.join(ROOT, 'include'), GATEWAY_SRC,
           '-L', PKG, '-lhp', '-L', BUILD, '-lmxstub', f'-Wl,-rpath,{PKG}:{BUILD}', '-lm', '-o', out]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return out


class MexError(RuntimeError):
    pass


def to_mx(v):
    lib = stub()
    if isinstance(v, str):
        return lib.mxstub_string(v.encode())
    if isinstance(v, (bool, np.bool_)):
        a = np.array([[bool(v)]])
    elif isinstance(v, (int, float)) and not isinstance(v, bool):
        a = np.array([[float(v)]])
    else:
        a = np.asarray(v)
    if a.ndim < 2:
        a = a.reshape(-1, 1)
    cplx = np.iscomplexobj(a)
    if a.dtype == np.bool_:
        cls = LOGICAL
    elif a.dtype == np.int32:
        cls = INT32
    elif a.dtype == np.int16:
        cls = INT16
    elif a.dtype == np.float32:
        cls = SINGLE
    else:
        cls = DOUBLE
        a = a.astype(np.complex128 if cplx else np.float64, copy=False)
    dims = (ctypes.c_size_t * a.ndim)(*a.shape)
    h = lib.mxstub_new(cls, int(cplx), a.ndim, dims)
    if not h:
        raise MemoryError('mxstub_new failed')
    raw = np.asfortranarray(a).tobytes(order='F')
    ctypes.memmove(lib.mxstub_data(h), raw, len(raw))
    return h


def from_mx(h):
    lib = stub()
    cls = lib.mxstub_class(h)
    cplx = lib.mxstub_is_complex(h)
    shape = tuple(lib.mxstub_dim(h, i) for i in range(lib.mxstub_ndim(h)))
    dt = np.complex128 if (cls == DOUBLE and cplx) else _NP[cls]
    n = int(np.prod(shape))
    buf = (ctypes.c_char * (n * np.dtype(dt).itemsize)).from_address(lib.mxstub_data(h))
    return np.frombuffer(bytes(buf), dtype=dt).reshape(shape, order='F').copy()


class Gateway:
    """One MEX file: call(*args, nlhs=k) -> list of k numpy outputs."""

    def __init__(self, path: str):
        stub()
        self.lib = ctypes.CDLL(path)
        self.fn = ctypes.cast(self.lib.mexFunction, ctypes.c_void_p)

    def call(self, *args, nlhs: int = 1):
        lib = stub()
        prhs = (ctypes.c_void_p * max(len(args), 1))(*[to_mx(a) for a in args])
        plhs = (ctypes.c_void_p * max(nlhs, 1))()
        try:
            rc = lib.mxstub_call(self.fn, nlhs, plhs, len(args), prhs)
            if rc != 0:
                raise MexError(lib.mxstub_last_error().decode())
            return [from_mx(plhs[i]) for i in range(nlhs)]
        finally:
            for i in range(len(args)):
                lib.mxstub_free(prhs[i])
            for i in range(nlhs):
                if plhs[i]:
                    lib.mxstub_free(plhs[i])


def clear_all():
    """What MATLAB's `clear mex` does: run the gateways' mexAtExit handlers
    (they destroy their cached plans)."""
    if _stub is not None:
        _stub.mxstub_run_atexit()
