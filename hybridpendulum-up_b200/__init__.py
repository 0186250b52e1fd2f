"""B200 (sm_100a) Fokker-Planck propagation on SO(3) x R^n.

Host-side mirror of the reference's MEX / MATLAB interface for the propagation
path (fdcl-gwu/hybridPendulum-UP): the functions below keep the reference's
names, argument order and array layouts, and call the CUDA library ``libhp.so``
through its C ABI (``include/hp.h``).  There is no CPU fallback: importing this
package fails if the library has not been built (``python build.py``).

Arrays are numpy (host, staged through the plan) or torch CUDA tensors
(device pointers, no copies).  Layouts are the MATLAB column-major ones:
    F  (2lmax+1, 2lmax+1, lmax+1, 2Bx, 2Bx[, 2Bx]) complex128
    f  (2B, 2B, 2B, 2Bx, 2Bx[, 2Bx])                float64 (complex128 for complex plans)
so a C-ordered numpy array of the reversed shape, or an F-ordered array of the
MATLAB shape, is passed as is.
"""
from __future__ import annotations

import ctypes
import math
import os
from functools import lru_cache

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, 'libhp.so')

HP_OK, HP_ERR_INVALID, HP_ERR_SHAPE, HP_ERR_ALLOC, HP_ERR_CUDA = 0, 1, 2, 3, 4
HP_ERR_UNSUPPORTED, HP_ERR_NONFINITE, HP_ERR_NO_MODEL, HP_ERR_MASS_DRIFT = 5, 6, 7, 8
HP_FP64, HP_MIXED = 0, 1
HP_REAL, HP_COMPLEX = 0, 1
HP_EULER, HP_MIDPOINT, HP_RK2, HP_RK4 = 0, 1, 2, 3
HP_DEVICE, HP_HOST = 0, 1
HP_BETA_AUTO, HP_BETA_SIMT, HP_BETA_TENSOR, HP_BETA_TENSOR_BF16 = 0, 1, 2, 3
METHODS = {'euler': HP_EULER, 'midpoint': HP_MIDPOINT, 'rk2': HP_RK2, 'rk4': HP_RK4}

EXPORTS = ['hp_plan_create', 'hp_plan_destroy', 'hp_plan_get_info', 'hp_plan_set_stream',
           'hp_last_error', 'hp_plan_set_model', 'hp_wigner_d', 'hp_quad_weights',
           'hp_fftSO3R_forward', 'hp_fftSO3R_backward', 'hp_pendulum_propagate',
           'hp_pendulum_derivative', 'hp_fftSO3_prod', 'hp_state_create', 'hp_state_destroy',
           'hp_state_load', 'hp_state_store', 'hp_state_step', 'hp_state_density',
           'hp_state_mass', 'hp_plan_profile', 'hp_plan_profile_get', 'hp_plan_launch_count',
           'hp_pendulum_derivative_noalloc', 'hp_state_normalize', 'hp_collision_create',
           'hp_collision_destroy', 'hp_collision_tables', 'hp_collision_df', 'hp_plan_set_den_model',
           'hp_pendulum_propagate_den', 'hp_state_hybrid_step', 'hp_pendulum_derivative_adjoint',
           'hp_pendulum_adjoint', 'hp_moments', 'hp_state_moments', 'hp_density_mf_gauss',
           'hp_state_init_mf_gauss', 'hp_state_load_density', 'hp_batch_create', 'hp_batch_destroy', 'hp_batch_step', 'hp_batch_info',
           'hp_plan_set_gyro_bias_model', 'hp_gyrobias_propagate', 'hp_fftSO3_real_forward',
           'hp_fftSO3_real_backward', 'hp_fftSO3_real_prod', 'hp_plan_set_beta_engine', 'hp_plan_tc_errors',
           'hp_collision_lambda', 'hp_collision_omega', 'hp_collision_fcL', 'hp_collision_create_from_tables',
           'hp_state_set_guard', 'hp_set_device_budget', 'hp_device_bytes', 'hp_plan_autotune',
           'hp_plan_set_tune', 'hp_plan_get_tune', 'hp_tune_cache_save', 'hp_tune_cache_load',
           'hp_batch_set_persistent']


class HPError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f'hp error {code}: {msg}')
        self.code = code


class hp_model(ctypes.Structure):
    _fields_ = [('L', ctypes.c_double), ('b', ctypes.c_double * 3), ('G', ctypes.c_double * 9),
                ('gyro', ctypes.c_double * 3)]


class hp_model_grad(ctypes.Structure):
    _fields_ = [('b', ctypes.c_double * 3), ('G', ctypes.c_double * 9), ('gyro', ctypes.c_double * 3),
                ('gscale', ctypes.c_double * 3)]


class hp_moments_t(ctypes.Structure):
    _fields_ = [('mass', ctypes.c_double), ('ER', ctypes.c_double * 9), ('ERR', ctypes.c_double * 81),
                ('Ex', ctypes.c_double * 3), ('Exx', ctypes.c_double * 9), ('ExR', ctypes.c_double * 27)]


def _moments_dict(m: 'hp_moments_t', nd: int, fx) -> dict:
    out = dict(mass=m.mass, ER=np.array(m.ER[:]).reshape(3, 3), ERR=np.array(m.ERR[:]).reshape(3, 3, 3, 3),
               Ex=np.array(m.Ex[:nd]), Exx=np.array(m.Exx[:]).reshape(3, 3)[:nd, :nd],
               ExR=np.array(m.ExR[:]).reshape(3, 3, 3)[:nd])
    if fx is not None:
        out['fx'] = fx
    return out


def _mfg_args(U, s, V, mu, Sigma, ndim):
    U = np.ascontiguousarray(U, float).reshape(3, 3)
    V = np.ascontiguousarray(V, float).reshape(3, 3)
    s = np.ascontiguousarray(s, float).reshape(3)
    mu = np.ascontiguousarray(np.asarray(mu, float).reshape(-1)[:ndim])
    Sg = np.zeros((3, 3))
    Sa = np.asarray(Sigma, float)
    Sg[:Sa.shape[0], :Sa.shape[1]] = Sa
    arrs = (U, s, V, mu, np.ascontiguousarray(Sg))
    return arrs, [ctypes.c_void_p(a.ctypes.data) for a in arrs]


class hp_collision_params(ctypes.Structure):
    _fields_ = [('d', ctypes.c_double), ('h', ctypes.c_double), ('r', ctypes.c_double),
                ('theta_t', ctypes.c_double), ('lambda_max', ctypes.c_double), ('epsilon', ctypes.c_double),
                ('L', ctypes.c_double), ('Gd', ctypes.c_double * 9), ('nD', ctypes.c_int)]


class hp_plan_info_t(ctypes.Structure):
    _fields_ = [('B', ctypes.c_int), ('lmax', ctypes.c_int), ('Bx', ctypes.c_int), ('N', ctypes.c_int),
                ('ndim', ctypes.c_int), ('precision', ctypes.c_int), ('symmetry', ctypes.c_int),
                ('nx', ctypes.c_longlong), ('nrows', ctypes.c_longlong), ('n_full', ctypes.c_longlong),
                ('n_grid', ctypes.c_longlong), ('state_bytes', ctypes.c_longlong)]


def _load():
    if not os.path.exists(_LIB_PATH):
        raise ImportError(f'{_LIB_PATH} is missing: build it with `python build.py` '
                          '(the CUDA library is the only implementation; there is no fallback)')
    lib = ctypes.CDLL(_LIB_PATH)
    vp, ip, dp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    sig = {
        'hp_plan_create': [ctypes.POINTER(vp), ip, ip, ip, ip, ip],
        'hp_plan_destroy': [vp], 'hp_plan_get_info': [vp, ctypes.POINTER(hp_plan_info_t)],
        'hp_plan_set_stream': [vp, vp], 'hp_plan_set_model': [vp, ctypes.POINTER(hp_model), vp, ip],
        'hp_wigner_d': [vp, vp, ip], 'hp_quad_weights': [vp, vp, ip],
        'hp_fftSO3R_forward': [vp, vp, vp, ip], 'hp_fftSO3R_backward': [vp, vp, vp, ip],
        'hp_pendulum_propagate': [vp, vp, vp, dp, ip, ip], 'hp_pendulum_derivative': [vp, vp, vp, ip],
        'hp_fftSO3_prod': [vp, vp, vp, vp, ip, ip],
        'hp_state_create': [vp, ctypes.POINTER(vp)], 'hp_state_destroy': [vp],
        'hp_state_load': [vp, vp, ip], 'hp_state_store': [vp, vp, ip],
        'hp_state_step': [vp, dp, ip, ip], 'hp_state_density': [vp, vp], 'hp_state_mass': [vp, ctypes.POINTER(dp)],
        'hp_plan_profile': [vp, ip],
        'hp_plan_profile_get': [vp, ip, ctypes.c_char_p, ip, ctypes.POINTER(dp), ctypes.POINTER(ctypes.c_longlong)],
        'hp_plan_launch_count': [vp, ctypes.POINTER(ctypes.c_longlong)],
        'hp_state_normalize': [vp, dp, ctypes.POINTER(dp)],
        'hp_collision_create': [vp, ctypes.POINTER(hp_collision_params), ctypes.POINTER(vp), ctypes.POINTER(ip)],
        'hp_collision_destroy': [vp],
        'hp_collision_tables': [vp, vp, vp, vp, vp, vp, vp, ip],
        'hp_collision_df': [vp, vp, vp, ip],
        'hp_plan_set_den_model': [vp, ctypes.POINTER(hp_model), vp, ip],
        'hp_pendulum_propagate_den': [vp, vp, vp, vp, dp, ip, ip],
        'hp_state_hybrid_step': [vp, vp, dp, ip, ip],
        'hp_pendulum_derivative_adjoint': [vp, vp, vp, ip],
        'hp_moments': [vp, vp, ip, ctypes.POINTER(hp_moments_t), vp],
        'hp_state_moments': [vp, ctypes.POINTER(hp_moments_t), vp],
        'hp_density_mf_gauss': [vp, vp, vp, vp, vp, vp, vp, ip],
        'hp_state_init_mf_gauss': [vp, vp, vp, vp, vp, vp],
        'hp_state_load_density': [vp, vp],
        'hp_batch_create': [vp, vp, ip, ctypes.POINTER(vp)],
        'hp_batch_destroy': [vp],
        'hp_batch_step': [vp, dp, ip, ip],
        'hp_batch_info': [vp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ip)],
        'hp_pendulum_adjoint': [vp, vp, vp, ip, dp, ip, ip, vp, ctypes.POINTER(hp_model_grad), ip],
        'hp_plan_set_gyro_bias_model': [vp, dp, vp, vp],
        'hp_gyrobias_propagate': [vp, vp, vp, dp, ip],
        'hp_fftSO3_real_forward': [vp, vp, vp, ip, ip],
        'hp_fftSO3_real_backward': [vp, vp, vp, ip, ip],
        'hp_fftSO3_real_prod': [vp, vp, vp, vp, ip, ip],
        'hp_plan_set_beta_engine': [vp, ip],
        'hp_plan_tc_errors': [vp, ctypes.POINTER(ip)],
        'hp_collision_lambda': [vp, ctypes.POINTER(hp_collision_params), ctypes.POINTER(ip), vp, vp, vp, ip],
        'hp_collision_omega': [vp, ctypes.POINTER(hp_collision_params), ip, vp, vp, ip],
        'hp_collision_fcL': [vp, ctypes.POINTER(hp_collision_params), ip, vp, vp, vp, vp, ip],
        'hp_collision_create_from_tables': [vp, ip, ip, vp, vp, vp, vp, ip, ctypes.POINTER(vp)],
        'hp_state_set_guard': [vp, ip, dp],
        'hp_set_device_budget': [ctypes.c_longlong],
        'hp_device_bytes': [ctypes.POINTER(ctypes.c_longlong)],
        'hp_plan_autotune': [vp, ctypes.POINTER(dp), ctypes.POINTER(dp)],
        'hp_plan_set_tune': [vp, ip, ip, ip, ip],
        'hp_plan_get_tune': [vp, ctypes.POINTER(ip), ctypes.POINTER(ip), ctypes.POINTER(ip), ctypes.POINTER(ip)],
        'hp_tune_cache_save': [ctypes.c_char_p],
        'hp_tune_cache_load': [ctypes.c_char_p],
        'hp_batch_set_persistent': [vp, ip],
        'hp_host_read_in_place': [vp, ctypes.c_longlong, ctypes.POINTER(ip)],
    }
    for name, args in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    lib.hp_last_error.restype = ctypes.c_char_p
    lib.hp_last_error.argtypes = []
    return lib


_lib = _load()


def _check(code: int):
    if code != HP_OK:
        raise HPError(code, _lib.hp_last_error().decode())


def _ptr(a, dtype):
    """(pointer, mem) of a numpy array or torch CUDA tensor with the required dtype."""
    if isinstance(a, np.ndarray):
        if a.dtype != dtype:
            raise TypeError(f'expected {dtype}, got {a.dtype}')
        if not (a.flags['F_CONTIGUOUS'] or a.flags['C_CONTIGUOUS']):
            raise ValueError('array must be contiguous')
        return a.ctypes.data, HP_HOST
    try:
        import torch
    except ImportError as e:  # pragma: no cover
        raise TypeError('expected a numpy array') from e
    if isinstance(a, torch.Tensor):
        tdt = {np.dtype(np.float64): torch.float64, np.dtype(np.complex128): torch.complex128,
               np.dtype(np.float32): torch.float32}[np.dtype(dtype)]
        if a.dtype != tdt or not a.is_contiguous():
            raise TypeError(f'expected a contiguous {tdt} tensor')
        return a.data_ptr(), (HP_DEVICE if a.is_cuda else HP_HOST)
    raise TypeError(f'unsupported array type {type(a)}')


def host_read_in_place(a) -> bool:
    """True when the library reads the host array `a` (an F input) in place:
    page-locked memory mapped into the device address space, such as a torch
    ``pin_memory`` tensor; only the entries the plan keeps then cross the bus.
    False when it is copied whole to the device first (e.g. a numpy array)."""
    if isinstance(a, np.ndarray):
        p, nb = a.ctypes.data, a.nbytes
    else:
        if a.is_cuda:
            raise ValueError('expected a host array')
        p, nb = a.data_ptr(), a.numel() * a.element_size()
    r = ctypes.c_int()
    _check(_lib.hp_host_read_in_place(ctypes.c_void_p(p), nb, ctypes.byref(r)))
    return bool(r.value)


# ------------------------------------------------------------------- plan ----
class Plan:
    """Tables and workspace for one (B, Bx, ndim, precision, symmetry)."""

    def __init__(self, B: int, Bx: int, ndim: int, precision: int = HP_FP64, symmetry: int = HP_REAL):
        h = ctypes.c_void_p()
        _check(_lib.hp_plan_create(ctypes.byref(h), B, Bx, ndim, precision, symmetry))
        self._h = h
        self.B, self.Bx, self.ndim, self.precision, self.symmetry = B, Bx, ndim, precision, symmetry
        info = hp_plan_info_t()
        _check(_lib.hp_plan_get_info(h, ctypes.byref(info)))
        self.info = info
        self.lmax, self.N, self.nx, self.nrows = B - 1, 2 * Bx, info.nx, info.nrows
        self.model = None

    def __del__(self):
        h = getattr(self, '_h', None)
        if h is not None and _lib is not None:
            _lib.hp_plan_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    # shapes (MATLAB order)
    @property
    def F_shape(self):
        return (2 * self.lmax + 1, 2 * self.lmax + 1, self.lmax + 1) + (self.N,) * self.ndim

    @property
    def f_shape(self):
        return (2 * self.B,) * 3 + (self.N,) * self.ndim

    def set_stream(self, stream_ptr: int):
        _check(_lib.hp_plan_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    def set_model(self, L: float, b, G, MR, gyro=(0.0, 0.0, 0.0)):
        m = hp_model()
        m.L = float(L)
        bb = list(np.asarray(b, float).ravel()) + [0.0] * 3
        for i in range(3):
            m.b[i] = bb[i]
        Gm = np.zeros((3, 3))
        Ga = np.asarray(G, float)
        Gm[:Ga.shape[0], :Ga.shape[1]] = Ga
        for i in range(9):
            m.G[i] = Gm.ravel()[i]
        for i in range(3):
            m.gyro[i] = float(gyro[i])
        MRc = _as_matlab(MR, np.complex128)
        p, mem = _ptr(MRc, np.complex128)
        _check(_lib.hp_plan_set_model(self._h, ctypes.byref(m), ctypes.c_void_p(p), mem))
        self.model = dict(L=float(L), b=np.array(bb[:3]), G=Gm, gyro=tuple(gyro))
        self._MR_keep = MRc

    def set_den_model(self, L: float, b, G, mR):
        """Density-gravity model of pendulum_reduced_den.m (2-D plans): the
        gravity term fftSO3R(f . mR_i) is formed on the grid.  mR: (2, 2B, 2B, 2B)
        real samples (pendulum_reduced_den.m:132)."""
        m = hp_model()
        m.L = float(L)
        bb = list(np.asarray(b, float).ravel()) + [0.0] * 3
        for i in range(3):
            m.b[i] = bb[i]
        Gm = np.zeros((3, 3))
        Ga = np.asarray(G, float)
        Gm[:Ga.shape[0], :Ga.shape[1]] = Ga
        for i in range(9):
            m.G[i] = Gm.ravel()[i]
        mRc = _as_matlab(mR, np.float64)
        if tuple(mRc.shape) != (2,) + (2 * self.B,) * 3:
            raise HPError(HP_ERR_SHAPE, f'mR must have shape (2, {2 * self.B}, {2 * self.B}, {2 * self.B})')
        p, mem = _ptr(mRc, np.float64)
        _check(_lib.hp_plan_set_den_model(self._h, ctypes.byref(m), ctypes.c_void_p(p), mem))
        self.model = dict(L=float(L), b=np.array(bb[:3]), G=Gm, gyro=(0.0, 0.0, 0.0))
        self._MR_keep = mRc

    def profile(self, enable: bool = True):
        """Start (and reset) or stop per-kernel-family CUDA-event timing."""
        _check(_lib.hp_plan_profile(self._h, int(enable)))

    def profile_read(self) -> dict:
        """{family: (total_ms, launches)} since the last profile(True)."""
        out, i = {}, 0
        buf = ctypes.create_string_buffer(64)
        while True:
            ms, cnt = ctypes.c_double(), ctypes.c_longlong()
            if _lib.hp_plan_profile_get(self._h, i, buf, 64, ctypes.byref(ms), ctypes.byref(cnt)) != HP_OK:
                break
            out[buf.value.decode()] = (ms.value, cnt.value)
            i += 1
        return out

    def set_beta_engine(self, engine: int):
        """Engine of the forward transform's beta contraction: HP_BETA_AUTO
        (tensor cores in HP_MIXED plans with B >= 15), HP_BETA_SIMT or
        HP_BETA_TENSOR (tensor cores in every HP_MIXED plan)."""
        _check(_lib.hp_plan_set_beta_engine(self._h, int(engine)))

    def autotune(self) -> dict:
        """Time the candidate launch shapes of this plan's transforms and keep
        the fastest (cached for later plans of the same key)."""
        b, f = ctypes.c_double(), ctypes.c_double()
        _check(_lib.hp_plan_autotune(self._h, ctypes.byref(b), ctypes.byref(f)))
        return dict(self.get_tune(), backward_ms=b.value, forward_ms=f.value)

    def set_tune(self, synth_pt: int = 0, synth_waves: int = 0, tc_waves: int = 0, tc_form: int = -1):
        _check(_lib.hp_plan_set_tune(self._h, int(synth_pt), int(synth_waves), int(tc_waves), int(tc_form)))

    def get_tune(self) -> dict:
        a, b, c, d = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(_lib.hp_plan_get_tune(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(d)))
        return dict(synth_pt=a.value, synth_waves=b.value, tc_waves=c.value, tc_form=d.value)

    def tc_errors(self) -> int:
        """Tensor-core launches of this plan whose wait gave up (0 normally)."""
        v = ctypes.c_int()
        _check(_lib.hp_plan_tc_errors(self._h, ctypes.byref(v)))
        return v.value

    def launch_count(self) -> int:
        v = ctypes.c_longlong()
        _check(_lib.hp_plan_launch_count(self._h, ctypes.byref(v)))
        return v.value

    def wigner_d(self) -> np.ndarray:
        d = np.zeros((2 * self.lmax + 1, 2 * self.lmax + 1, self.lmax + 1, 2 * self.B), order='F')
        _check(_lib.hp_wigner_d(self._h, ctypes.c_void_p(d.ctypes.data), HP_HOST))
        return d

    def quad_weights(self) -> np.ndarray:
        w = np.zeros(2 * self.B)
        _check(_lib.hp_quad_weights(self._h, ctypes.c_void_p(w.ctypes.data), HP_HOST))
        return w

    # transforms -----------------------------------------------------------
    def forward(self, f, out=None):
        cplx = self.symmetry == HP_COMPLEX
        fdt = np.complex128 if cplx else np.float64
        f = _as_matlab(f, fdt)
        if out is None:
            out = _empty_like_mem(f, self.F_shape, np.complex128)
        pi, mi = _ptr(f, fdt)
        po, mo = _ptr(out, np.complex128)
        if mi != mo:
            raise ValueError('input and output must live in the same memory space')
        _check(_lib.hp_fftSO3R_forward(self._h, ctypes.c_void_p(pi), ctypes.c_void_p(po), mi))
        return out

    def backward(self, F, out=None):
        cplx = self.symmetry == HP_COMPLEX
        fdt = np.complex128 if cplx else np.float64
        F = _as_matlab(F, np.complex128)
        if out is None:
            out = _empty_like_mem(F, self.f_shape, fdt)
        pi, mi = _ptr(F, np.complex128)
        po, mo = _ptr(out, fdt)
        if mi != mo:
            raise ValueError('input and output must live in the same memory space')
        _check(_lib.hp_fftSO3R_backward(self._h, ctypes.c_void_p(pi), ctypes.c_void_p(po), mi))
        return out

    def propagate(self, F, dt: float, method: str = 'euler', out=None):
        F = _as_matlab(F, np.complex128)
        if out is None:
            out = _empty_like_mem(F, self.F_shape, np.complex128)
        pi, mi = _ptr(F, np.complex128)
        po, _ = _ptr(out, np.complex128)
        _check(_lib.hp_pendulum_propagate(self._h, ctypes.c_void_p(pi), ctypes.c_void_p(po), float(dt),
                                          METHODS[method.lower()], mi))
        return out

    def propagate_den(self, F, f, dt: float, method: str = 'euler', out=None):
        """One step of the density-gravity model; f is the grid density of F
        (None: recomputed from F by the backward transform)."""
        F = _as_matlab(F, np.complex128)
        if out is None:
            out = _empty_like_mem(F, self.F_shape, np.complex128)
        pi, mi = _ptr(F, np.complex128)
        po, _ = _ptr(out, np.complex128)
        pf = None
        if f is not None:
            f = _as_matlab(f, np.float64)
            if tuple(f.shape) != tuple(self.f_shape):
                raise HPError(HP_ERR_SHAPE, f'f must have shape {self.f_shape}')
            pf, mf = _ptr(f, np.float64)
            if mf != mi:
                raise ValueError('F and f must live in the same memory space')
        _check(_lib.hp_pendulum_propagate_den(self._h, ctypes.c_void_p(pi), ctypes.c_void_p(pf),
                                              ctypes.c_void_p(po), float(dt), METHODS[method.lower()], mi))
        return out

    def set_gyro_bias_model(self, L: float, G1, G2):
        """Gyro-bias attitude model of gyro_bias.m:226-300 (3-D plans): bias
        drift, attitude diffusion G1 and bias random walk G2 on the bias grid of
        period L (2 in the reference driver)."""
        g1 = np.ascontiguousarray(np.asarray(G1, float).reshape(3, 3))
        g2 = np.ascontiguousarray(np.asarray(G2, float).reshape(3, 3))
        _check(_lib.hp_plan_set_gyro_bias_model(self._h, float(L), g1.ctypes.data, g2.ctypes.data))
        self.model = dict(L=float(L), G1=g1, G2=g2)

    def gyrobias_propagate(self, F, dt: float, out=None):
        """Fnew = F + dt dF of the gyro-bias model (one Euler step)."""
        F = _as_matlab(F, np.complex128)
        if out is None:
            out = _empty_like_mem(F, self.F_shape, np.complex128)
        pi, mi = _ptr(F, np.complex128)
        po, _ = _ptr(out, np.complex128)
        _check(_lib.hp_gyrobias_propagate(self._h, ctypes.c_void_p(pi), ctypes.c_void_p(po), float(dt), mi))
        return out

    def real_forward(self, f, out=None):
        """Real-harmonic coefficients F(m, n, l[, b]) of fftSO3(f, B, true)
        (fftSO3.m:61-119) for real SO(3) samples f(a, j, c[, b]) on this plan's
        grid; a trailing axis batches independent functions."""
        N, D = 2 * self.B, 2 * self.lmax + 1
        f = _as_matlab(f, np.float64)
        if isinstance(f, np.ndarray):
            if tuple(f.shape[:3]) != (N, N, N) or f.ndim > 4:
                raise HPError(HP_ERR_SHAPE, f'f must have shape ({N}, {N}, {N}[, nbatch])')
            nb = f.shape[3] if f.ndim == 4 else 1
        else:                                   # flat device tensor: nbatch from its size
            nb = f.numel() // N ** 3
            if nb * N ** 3 != f.numel() or nb < 1:
                raise HPError(HP_ERR_SHAPE, f'f must hold nbatch * {N ** 3} values')
        shape = (D, D, self.B) + ((nb,) if nb > 1 or getattr(f, 'ndim', 3) == 4 else ())
        if out is None:
            out = _empty_like_mem(f, shape, np.float64)
        pf, mf = _ptr(f, np.float64)
        po, _ = _ptr(out, np.float64)
        _check(_lib.hp_fftSO3_real_forward(self._h, ctypes.c_void_p(pf), ctypes.c_void_p(po), nb, mf))
        return out

    def real_backward(self, F, out=None):
        """Real samples f(a, j, c[, b]) of ifftSO3(F, true) (ifftSO3.m:24-84)."""
        N, D = 2 * self.B, 2 * self.lmax + 1
        F = _as_matlab(F, np.float64)
        if isinstance(F, np.ndarray):
            if tuple(F.shape[:3]) != (D, D, self.B) or F.ndim > 4:
                raise HPError(HP_ERR_SHAPE, f'F must have shape ({D}, {D}, {self.B}[, nbatch])')
            nb = F.shape[3] if F.ndim == 4 else 1
        else:
            nb = F.numel() // (D * D * self.B)
            if nb * D * D * self.B != F.numel() or nb < 1:
                raise HPError(HP_ERR_SHAPE, f'F must hold nbatch * {D * D * self.B} values')
        shape = (N, N, N) + ((nb,) if nb > 1 or getattr(F, 'ndim', 3) == 4 else ())
        if out is None:
            out = _empty_like_mem(F, shape, np.float64)
        pF, mF = _ptr(F, np.float64)
        po, _ = _ptr(out, np.float64)
        _check(_lib.hp_fftSO3_real_backward(self._h, ctypes.c_void_p(pF), ctypes.c_void_p(po), nb, mF))
        return out

    def real_prod(self, F, G, out=None):
        """Real-harmonic coefficients of the product f g (fftSO3_prod.m:97-205,
        isreal) from real coefficients F, G of shape (D, D, B[, batch])."""
        D = 2 * self.lmax + 1
        F = np.asfortranarray(np.asarray(F, dtype=np.float64))
        G = np.asfortranarray(np.asarray(G, dtype=np.float64))
        if F.shape != G.shape or tuple(F.shape[:3]) != (D, D, self.B) or F.ndim > 4:
            raise HPError(HP_ERR_SHAPE, f'F and G must have shape ({D}, {D}, {self.B}[, batch])')
        nb = F.shape[3] if F.ndim == 4 else 1
        out = np.zeros(F.shape, order='F') if out is None else out
        _check(_lib.hp_fftSO3_real_prod(self._h, F.ctypes.data, G.ctypes.data, out.ctypes.data, nb, HP_HOST))
        return out

    def density_mf_gauss(self, U, s, V, mu, Sigma):
        """Matrix Fisher(U diag(s) V^T) x N(mu, Sigma) on the grid (pendulum.m:210-220), FP64."""
        keep, ptrs = _mfg_args(U, s, V, mu, Sigma, self.ndim)
        f = np.zeros(self.f_shape, order='F')
        _check(_lib.hp_density_mf_gauss(self._h, *ptrs, ctypes.c_void_p(f.ctypes.data), HP_HOST))
        return f

    def moments(self, F, want_fx: bool = False) -> dict:
        """Raw moments of get_stat (mass, ER, ERR, Ex, Exx, ExR; fx on request)
        of the density with coefficients F, from the coefficients alone."""
        F = _as_matlab(F, np.complex128)
        pf, mf = _ptr(F, np.complex128)
        m = hp_moments_t()
        fx = np.zeros((self.N,) * self.ndim, order='F') if want_fx else None
        _check(_lib.hp_moments(self._h, ctypes.c_void_p(pf), mf, ctypes.byref(m),
                               ctypes.c_void_p(fx.ctypes.data if want_fx else None)))
        return _moments_dict(m, self.ndim, fx)

    def derivative_adjoint(self, lam, out=None):
        """A^H lam, the adjoint of ``derivative`` under <X, Y> = Re sum conj(X) Y."""
        lam = _as_matlab(lam, np.complex128)
        if out is None:
            out = _empty_like_mem(lam, self.F_shape, np.complex128)
        pi, mi = _ptr(lam, np.complex128)
        po, _ = _ptr(out, np.complex128)
        _check(_lib.hp_pendulum_derivative_adjoint(self._h, ctypes.c_void_p(pi), ctypes.c_void_p(po), mi))
        return out

    def adjoint(self, F0, lamT, nsteps: int, dt: float, checkpoint_every: int = 10, method: str = 'euler'):
        """Reverse pass of ``nsteps`` Euler steps from F0 for a loss with gradient
        lamT at F_T.  Returns (lam0, grads) with grads = dict(b, G, gyro, gscale)."""
        F0 = _as_matlab(F0, np.complex128)
        lamT = _as_matlab(lamT, np.complex128)
        lam0 = _empty_like_mem(F0, self.F_shape, np.complex128)
        pf, mf = _ptr(F0, np.complex128)
        pl, ml = _ptr(lamT, np.complex128)
        po, _ = _ptr(lam0, np.complex128)
        if mf != ml:
            raise ValueError('F0 and lamT must live in the same memory space')
        g = hp_model_grad()
        _check(_lib.hp_pendulum_adjoint(self._h, ctypes.c_void_p(pf), ctypes.c_void_p(pl), int(nsteps), float(dt),
                                        METHODS[method.lower()], int(checkpoint_every), ctypes.c_void_p(po),
                                        ctypes.byref(g), mf))
        grads = dict(b=np.array(g.b[:]), G=np.array(g.G[:]).reshape(3, 3), gyro=np.array(g.gyro[:]),
                     gscale=np.array(g.gscale[:]))
        return lam0, grads

    def derivative(self, F, out=None):
        F = _as_matlab(F, np.complex128)
        if out is None:
            out = _empty_like_mem(F, self.F_shape, np.complex128)
        pi, mi = _ptr(F, np.complex128)
        po, _ = _ptr(out, np.complex128)
        _check(_lib.hp_pendulum_derivative(self._h, ctypes.c_void_p(pi), ctypes.c_void_p(po), mi))
        return out

    def prod(self, F, G, out=None):
        F = _as_matlab(F, np.complex128)
        G = _as_matlab(G, np.complex128)
        batch = int(np.prod(F.shape[3:])) if F.ndim > 3 else 1
        if out is None:
            out = _empty_like_mem(F, F.shape, np.complex128)
        pf, mf = _ptr(F, np.complex128)
        pg, _ = _ptr(G, np.complex128)
        po, _ = _ptr(out, np.complex128)
        _check(_lib.hp_fftSO3_prod(self._h, ctypes.c_void_p(pf), ctypes.c_void_p(pg), ctypes.c_void_p(po),
                                   batch, mf))
        return out


class State:
    """Coefficients resident on the device across steps."""

    def __init__(self, plan: Plan):
        h = ctypes.c_void_p()
        _check(_lib.hp_state_create(plan.handle, ctypes.byref(h)))
        self._h, self.plan = h, plan

    def __del__(self):
        h = getattr(self, '_h', None)
        if h is not None and _lib is not None:
            _lib.hp_state_destroy(h)
            self._h = None

    def load(self, F):
        F = _as_matlab(F, np.complex128)
        p, m = _ptr(F, np.complex128)
        _check(_lib.hp_state_load(self._h, ctypes.c_void_p(p), m))

    def store(self, out=None):
        if out is None:
            out = np.zeros(self.plan.F_shape, np.complex128, order='F')
        p, m = _ptr(out, np.complex128)
        _check(_lib.hp_state_store(self._h, ctypes.c_void_p(p), m))
        return out

    def step(self, dt: float, method: str = 'euler', nsteps: int = 1):
        _check(_lib.hp_state_step(self._h, float(dt), METHODS[method.lower()], int(nsteps)))

    def hybrid_step(self, coll: 'Collision', dt: float, method: str = 'euler', nsteps: int = 1):
        """nsteps steps of pendulum_reduced_hybrid.m:224-234 (density-gravity
        propagation, backward transform, collision update, forward transform)."""
        if coll.plan is not self.plan:
            raise ValueError('the collision operator must be built on the state plan')
        _check(_lib.hp_state_hybrid_step(self._h, coll._h, float(dt), METHODS[method.lower()], int(nsteps)))

    def init_mf_gauss(self, U, s, V, mu, Sigma):
        """Load F = fftSO3R of the matrix Fisher x Gaussian density, built on the device."""
        keep, ptrs = _mfg_args(U, s, V, mu, Sigma, self.plan.ndim)
        _check(_lib.hp_state_init_mf_gauss(self._h, *ptrs))

    def moments(self, want_fx: bool = False) -> dict:
        """Raw moments of get_stat of the resident density (after hybrid steps:
        of the post-collision grid density)."""
        m = hp_moments_t()
        fx = np.zeros((self.plan.N,) * self.plan.ndim, order='F') if want_fx else None
        _check(_lib.hp_state_moments(self._h, ctypes.byref(m),
                                     ctypes.c_void_p(fx.ctypes.data if want_fx else None)))
        return _moments_dict(m, self.plan.ndim, fx)

    def density_into(self, dev_ptr: int):
        _check(_lib.hp_state_density(self._h, ctypes.c_void_p(dev_ptr)))

    def load_density(self, dev_ptr: int):
        """F = fftSO3R(f) from a device density in the plan's compute precision."""
        _check(_lib.hp_state_load_density(self._h, ctypes.c_void_p(dev_ptr)))

    def normalize(self, mass: float) -> float:
        """Scale the state so its l = 0 mass is `mass`; returns the factor."""
        f = ctypes.c_double()
        _check(_lib.hp_state_normalize(self._h, float(mass), ctypes.byref(f)))
        return f.value

    def mass(self) -> float:
        v = ctypes.c_double()
        _check(_lib.hp_state_mass(self._h, ctypes.byref(v)))
        return v.value

    def set_guard(self, check_every: int = 1, mass_rtol: float = 0.0):
        """Health check every check_every steps: NaN/Inf in the coefficients
        (HP_ERR_NONFINITE) and, with mass_rtol > 0, l = 0 mass drift from its
        value now (HP_ERR_MASS_DRIFT).  check_every = 0 turns it off."""
        _check(_lib.hp_state_set_guard(self._h, int(check_every), float(mass_rtol)))


def set_device_budget(nbytes: int):
    """Cap the device bytes the library may hold at once (0: no cap)."""
    _check(_lib.hp_set_device_budget(int(nbytes)))


def tune_cache_save(path: str):
    """Write the launch shapes found by Plan.autotune in this process to a text file."""
    _check(_lib.hp_tune_cache_save(os.fsencode(path)))


def tune_cache_load(path: str):
    """Read a file written by tune_cache_save; later plans of a listed key start from its shapes."""
    _check(_lib.hp_tune_cache_load(os.fsencode(path)))


def device_bytes() -> int:
    """Device bytes the library holds now."""
    v = ctypes.c_longlong()
    _check(_lib.hp_device_bytes(ctypes.byref(v)))
    return v.value


# ---------------------------------------------------------------- helpers ----
def _as_matlab(a, dtype):
    """Numpy arrays are taken in MATLAB (Fortran) order; torch tensors as given
    (their memory must already be in the MATLAB column-major order)."""
    if isinstance(a, np.ndarray):
        return np.asfortranarray(a, dtype=dtype)
    return a


def _empty_like_mem(ref, shape, dtype):
    if isinstance(ref, np.ndarray):
        return np.zeros(shape, dtype=dtype, order='F')
    import torch
    tdt = {np.dtype(np.float64): torch.float64, np.dtype(np.complex128): torch.complex128}[np.dtype(dtype)]
    return torch.zeros(int(np.prod(shape)), dtype=tdt, device=ref.device)


class Collision:
    """Hybrid collision operator of pendulum_reduced_hybrid on a 2-D plan:
    getLambda_mex + getOmega_mex('new') + getFcL_mex tables, and the per-step
    pendulum_reduced_discrete_propagate(true, f, ...).  On a 3-D plan the same
    operator on a 3-D Omega grid (Gd then 3x3)."""

    def __init__(self, plan: Plan, d, h, r, theta_t, lambda_max, epsilon, L, Gd, nD=10):
        p = _coll_params(plan.ndim, d=d, h=h, r=r, theta_t=theta_t, lambda_max=lambda_max, epsilon=epsilon,
                         L=L, Gd=Gd, nD=nD)
        hnd, n = ctypes.c_void_p(), ctypes.c_int()
        _check(_lib.hp_collision_create(plan.handle, ctypes.byref(p), ctypes.byref(hnd), ctypes.byref(n)))
        self._h, self.plan, self.numR, self.nD = hnd, plan, n.value, int(nD)
        self.from_tables = False

    @classmethod
    def from_tables(cls, plan: Plan, lambda_, indR, fcL, fcL_indx):
        """The operator from given tables ([ix][k], [k], [ix][k][d], [ix][k][d]
        as returned by tables()), e.g. tables saved by an earlier run."""
        lam = np.ascontiguousarray(lambda_, np.float64)
        ind = np.ascontiguousarray(indR, np.int32).ravel()
        fc = np.ascontiguousarray(fcL, np.float64)
        ix = np.ascontiguousarray(fcL_indx, np.int16)
        numR, nD = ind.size, fc.shape[-1]
        self = cls.__new__(cls)
        hnd = ctypes.c_void_p()
        _check(_lib.hp_collision_create_from_tables(plan.handle, numR, nD, ind.ctypes.data, lam.ctypes.data,
                                                    fc.ctypes.data, ix.ctypes.data, HP_HOST, ctypes.byref(hnd)))
        self._h, self.plan, self.numR, self.nD = hnd, plan, numR, nD
        self.from_tables = True
        return self

    def __del__(self):
        h = getattr(self, '_h', None)
        if h is not None and _lib is not None:
            _lib.hp_collision_destroy(h)
            self._h = None

    def tables(self):
        nx = self.plan.N ** self.plan.ndim
        k, nD = self.numR, self.nD
        lam = np.zeros((nx, k)); ind = np.zeros(k, np.int32); om = np.zeros((nx, k, self.plan.ndim))
        fcL = np.zeros((nx, k, nD)); idx = np.zeros((nx, k, nD), np.int16)
        PC = np.zeros((8 * self.plan.B ** 3, 3))
        if self.from_tables:
            om = PC = None
        ptrs = [ctypes.c_void_p(a.ctypes.data if a is not None else None) for a in (lam, ind, om, fcL, idx, PC)]
        _check(_lib.hp_collision_tables(self._h, *ptrs, HP_HOST))
        return dict(lambda_=lam, indR=ind, omega=om, fcL=fcL, fcL_indx=idx, PC=PC)

    def df(self, f, out=None):
        """f: density f(a,b,c,i,j) (MATLAB layout); returns df, same layout."""
        f = _as_matlab(f, np.float64)
        if out is None:
            out = _empty_like_mem(f, self.plan.f_shape, np.float64)
        pf, mf = _ptr(f, np.float64)
        po, _ = _ptr(out, np.float64)
        _check(_lib.hp_collision_df(self._h, ctypes.c_void_p(pf), ctypes.c_void_p(po), mf))
        return out


def _coll_params(ndim, d=0.0, h=0.0, r=0.0, theta_t=0.0, lambda_max=0.0, epsilon=0.0, L=0.0, Gd=None, nD=1):
    p = hp_collision_params()
    p.d, p.h, p.r, p.theta_t, p.lambda_max, p.epsilon, p.L = d, h, r, theta_t, lambda_max, epsilon, L
    if Gd is not None:
        g = np.asarray(Gd, float).reshape(ndim, ndim).ravel(order='F')
        for i in range(ndim * ndim):
            p.Gd[i] = g[i]
    p.nD = int(nD)
    return p


def _x_grid_of(x):
    """(ndim, Bx, L) of an omega grid x(n, 2Bx, 2Bx[, 2Bx]) (MATLAB layout)."""
    x = np.asarray(x)
    nd, N = x.shape[0], x.shape[1]
    L = -2.0 * float(x.reshape(nd, -1, order='F')[0, 0])
    ref = _grid(N // 2, L, nd)
    if x.shape != ref.shape or not np.allclose(x, ref, rtol=0, atol=1e-9 * max(L, 1.0)):
        raise HPError(HP_ERR_UNSUPPORTED, 'x must be the uniform grid -L/2 + L*(0:2Bx-1)/(2Bx)')
    return nd, N // 2, L


def collision_count(plan: Plan, d, h, r, theta_t, lambda_max, L) -> int:
    """Number of colliding attitudes of the collision operator on `plan` (the
    numR of getLambda_mex), without building any table."""
    p = _coll_params(plan.ndim, d=d, h=h, r=r, theta_t=theta_t, lambda_max=lambda_max, L=L)
    n = ctypes.c_int()
    _check(_lib.hp_collision_lambda(plan.handle, ctypes.byref(p), ctypes.byref(n), None, None, None, HP_HOST))
    return n.value


def getLambda_mex(R, x, d, h, r, theta_t, lambda_max, compact=False):
    """[lambda, indR, PC] = getLambda_mex(R, x, d, h, r, theta_t, lambda_max, false)
    (propagation/discrete/mex/sources/pendulum_reduced_collision/src/mexLambda.cpp):
    lambda (numR, 2Bx, 2Bx), indR int32 (numR,) 0-based, PC (3, 2B, 2B, 2B).
    R must be the Euler-angle grid (the library builds it on the device)."""
    if compact:
        raise HPError(HP_ERR_UNSUPPORTED, 'the compact form of the noise-free model is not provided')
    B = np.asarray(R).shape[2] // 2
    nd, Bx, L = _x_grid_of(x)
    plan = get_plan(B, Bx, nd)
    p = _coll_params(nd, d=d, h=h, r=r, theta_t=theta_t, lambda_max=lambda_max, L=L)
    n = ctypes.c_int()
    _check(_lib.hp_collision_lambda(plan.handle, ctypes.byref(p), ctypes.byref(n), None, None, None, HP_HOST))
    nx = (2 * Bx) ** nd
    lam = np.zeros((nx, n.value)); ind = np.zeros(n.value, np.int32); PC = np.zeros((8 * B ** 3, 3))
    _check(_lib.hp_collision_lambda(plan.handle, ctypes.byref(p), ctypes.byref(n), lam.ctypes.data, ind.ctypes.data,
                                    PC.ctypes.data, HP_HOST))
    return (lam.T.reshape((n.value,) + (2 * Bx,) * nd, order='F'), ind,
            PC.T.reshape((3,) + (2 * B,) * 3, order='F'))


def getOmega_mex(R, x, indR, epsilon, PC, direction='new'):
    """Omega_new = getOmega_mex(R, x, indR, epsilon, PC, 'new') (mexOmega.cpp):
    Omega+ as (ndim, numR, 2Bx, 2Bx)."""
    if str(direction).lower() != 'new':
        raise HPError(HP_ERR_UNSUPPORTED, "only the 'new' direction (the hybrid model's reset map) is provided")
    B = np.asarray(R).shape[2] // 2
    nd, Bx, L = _x_grid_of(x)
    plan = get_plan(B, Bx, nd)
    ind = np.ascontiguousarray(indR, np.int32).ravel()
    p = _coll_params(nd, epsilon=epsilon, L=L)
    om = np.zeros(((2 * Bx) ** nd, ind.size, nd))
    _check(_lib.hp_collision_omega(plan.handle, ctypes.byref(p), ind.size, ind.ctypes.data, om.ctypes.data, HP_HOST))
    return np.transpose(om, (2, 1, 0)).reshape((nd, ind.size) + (2 * Bx,) * nd, order='F')


def getFcL_mex(x, Omega, lambda_, Gd, nD):
    """[fcL, fcL_indx] = getFcL_mex(x, Omega_new, lambda, Gd, nD) (mexFcL.cpp):
    (nD, numR, 2Bx, 2Bx) float64 and int16."""
    nd, Bx, L = _x_grid_of(x)
    plan = get_plan(2, Bx, nd)
    Om = np.asarray(Omega, float)
    numR = Om.shape[1]
    om = np.ascontiguousarray(np.transpose(Om.reshape(nd, numR, -1, order='F'), (2, 1, 0)))
    lam = np.ascontiguousarray(np.asarray(lambda_, float).reshape(numR, -1, order='F').T)
    p = _coll_params(nd, L=L, Gd=Gd, nD=int(nD))
    nx = (2 * Bx) ** nd
    fcL = np.zeros((nx, numR, int(nD))); idx = np.zeros((nx, numR, int(nD)), np.int16)
    _check(_lib.hp_collision_fcL(plan.handle, ctypes.byref(p), numR, om.ctypes.data, lam.ctypes.data,
                                 fcL.ctypes.data, idx.ctypes.data, HP_HOST))
    shp = (int(nD), numR) + (2 * Bx,) * nd
    return (np.transpose(fcL, (2, 1, 0)).reshape(shp, order='F'), np.transpose(idx, (2, 1, 0)).reshape(shp, order='F'))


def pendulum_reduced_discrete_propagate(noise, f, lambda_, indR, fcL, fcL_indx):
    """df = pendulum_reduced_discrete_propagate(true, f, lambda, indR, fcL, fcL_indx)
    (mexPropagate.cpp:6-77, propagate.cu:6-121) with MATLAB-layout tables."""
    if not noise:
        raise HPError(HP_ERR_UNSUPPORTED, 'only the noisy form of the hybrid model is provided')
    f = np.asfortranarray(f, np.float64)
    B, Bx, nd = f.shape[0] // 2, f.shape[3] // 2, f.ndim - 3
    plan = get_plan(B, Bx, nd)
    lam = np.asarray(lambda_, float)
    numR = lam.shape[0]
    nD = np.asarray(fcL).shape[0]
    c = Collision.from_tables(plan, lam.reshape(numR, -1, order='F').T,
                              indR, np.transpose(np.asarray(fcL, float).reshape(nD, numR, -1, order='F'), (2, 1, 0)),
                              np.transpose(np.asarray(fcL_indx, np.int16).reshape(nD, numR, -1, order='F'), (2, 1, 0)))
    return c.df(f)


class Batch:
    """Independent densities advanced together: member states of any plans
    (uneven bandlimits and omega grids), each optionally with a collision
    operator (hybrid step).  Members on different plans run concurrently; the
    steps are replayed from a CUDA graph after one warm-up step."""

    def __init__(self, states, collisions=None, persistent: bool = False):
        n = len(states)
        self._states = list(states)
        self._colls = list(collisions) if collisions is not None else [None] * n
        arr = (ctypes.c_void_p * n)(*[st._h for st in self._states])
        carr = (ctypes.c_void_p * n)(*[c._h if c is not None else None for c in self._colls])
        h = ctypes.c_void_p()
        _check(_lib.hp_batch_create(arr, carr, n, ctypes.byref(h)))
        self._h = h
        if persistent:
            _check(_lib.hp_batch_set_persistent(h, 1))

    def __del__(self):
        h = getattr(self, '_h', None)
        if h is not None and _lib is not None:
            _lib.hp_batch_destroy(h)
            self._h = None

    def step(self, dt: float, method: str = 'euler', nsteps: int = 1):
        _check(_lib.hp_batch_step(self._h, float(dt), METHODS[method.lower()], int(nsteps)))

    def info(self) -> dict:
        g, s = ctypes.c_longlong(), ctypes.c_int()
        _check(_lib.hp_batch_info(self._h, ctypes.byref(g), ctypes.byref(s)))
        return dict(graph_launches=g.value, streams=s.value)


@lru_cache(maxsize=32)
def get_plan(B: int, Bx: int, ndim: int, precision: int = HP_FP64, symmetry: int = HP_REAL) -> Plan:
    return Plan(B, Bx, ndim, precision, symmetry)


# ------------------------------------------------- reference-shaped API ----
def getu(lmax: int) -> np.ndarray:
    """u^l_i of getu.m:132-163 (complex harmonics): F^l[E_i f] = F^l[f] (u^l_i)^T."""
    D = 2 * lmax + 1
    u = np.zeros((D, D, lmax + 1, 3), np.complex128)
    for l in range(lmax + 1):
        for n in range(-l, l + 1):
            if n > -l:
                a = math.sqrt((l + n) * (l - n + 1))
                u[n + lmax - 1, n + lmax, l, 0] = -0.5j * a
                u[n + lmax - 1, n + lmax, l, 1] = 0.5 * a
            if n < l:
                a = math.sqrt((l - n) * (l + n + 1))
                u[n + lmax + 1, n + lmax, l, 0] = -0.5j * a
                u[n + lmax + 1, n + lmax, l, 1] = -0.5 * a
        for m in range(-l, l + 1):
            u[m + lmax, m + lmax, l, 2] = -1j * m
    return u


def _grid(Bx: int, L: float, ndim: int) -> np.ndarray:
    N = 2 * Bx
    g = -L / 2 + L / N * np.arange(N)
    return np.stack(np.meshgrid(*([g] * ndim), indexing='ij'), 0)


def _check_X(X, Bx: int, L: float, ndim: int):
    """The MEX receives X = fftn(x) (pendulum.m:141-143); the library rebuilds x
    from L, so X must be that table."""
    x = _grid(Bx, L, ndim)
    X = np.asarray(X)
    for i in range(ndim):
        ref = np.fft.fftn(x[i])
        if not np.allclose(X[..., i], ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max()):
            raise HPError(HP_ERR_UNSUPPORTED, 'X is not fftn of the uniform grid over [-L/2, L/2)')


def _fit_gyro(OJO, Bx: int, L: float):
    """Coefficients (g1, g2, g3) with ifftn(OJO_i) = (g1 x2 x3, g2 x1 x3, g3 x1 x2),
    the form of J^-1(-x cross Jx) for a diagonal J (pendulum.m:145-158)."""
    x = _grid(Bx, L, 3)
    pairs = [(1, 2), (0, 2), (0, 1)]
    g = []
    for i in range(3):
        ojo = np.real(np.fft.ifftn(np.asarray(OJO)[..., i]))
        basis = x[pairs[i][0]] * x[pairs[i][1]]
        c = float(np.sum(ojo * basis) / np.sum(basis * basis))
        resid = np.abs(ojo - c * basis).max()
        if resid > 1e-8 * max(1.0, np.abs(ojo).max()):
            raise HPError(HP_ERR_UNSUPPORTED, 'OJO is not of the diagonal-J form (g1 x2 x3, g2 x1 x3, g3 x1 x2)')
        g.append(c)
    return tuple(g)


def _model_plan(F, X, OJO, MR, b, G, L, precision):
    F = np.asarray(F)
    lmax = F.shape[2] - 1
    B = lmax + 1
    ndim = F.ndim - 3
    Bx = F.shape[3] // 2
    _check_X(X, Bx, L, ndim)
    gyro = _fit_gyro(OJO, Bx, L) if ndim == 3 else (0.0, 0.0, 0.0)
    plan = get_plan(B, Bx, ndim, precision, HP_REAL)
    plan.set_model(L, b, G, MR, gyro)
    return plan


def pendulum_propagate(F, X, OJO, MR, bt, G, dt, L, u, CG, method='euler'):
    """Drop-in for the MEX pendulum_propagate(F,X,OJO,MR,bt,G,dt,L,u,CG,method)
    (propagation/mex/sources/pendulum_propagate/kernel.cu:9-519), FP64.
    u and CG are accepted for signature compatibility; the library uses its own
    device tables (getu.m / clebsch_gordan.m restated on the GPU)."""
    plan = _model_plan(F, X, OJO, MR, bt, G, L, HP_FP64)
    return plan.propagate(F, dt, method)


def pendulum_propagate32(F, X, OJO, MR, bt, G, dt, L, u, CG, method='euler'):
    """Mixed-precision twin of pendulum_propagate (FP32 operators, FP64 accumulation)."""
    plan = _model_plan(F, X, OJO, MR, bt, G, L, HP_MIXED)
    return plan.propagate(F, dt, method)


def pendulum_propagate_reduced(F, X, MR, bt, G, dt, L, u, CG, method='euler'):
    """Drop-in for pendulum_propagate_reduced(F,X,MR,bt,G,dt,L,u,CG,method)
    (propagation/mex/sources/pendulum_propagate_reduced/kernel.cu:9-262)."""
    plan = _model_plan(F, X, None, MR, bt, G, L, HP_FP64)
    return plan.propagate(F, dt, method)


def pendulum_propagate_reduced32(F, X, MR, bt, G, dt, L, u, CG, method='euler'):
    plan = _model_plan(F, X, None, MR, bt, G, L, HP_MIXED)
    return plan.propagate(F, dt, method)


def _den_plan(F, X, mR, b, G, L, precision):
    F = np.asarray(F)
    B, Bx, ndim = F.shape[2], F.shape[3] // 2, F.ndim - 3
    if ndim != 2:
        raise HPError(HP_ERR_SHAPE, 'the density-gravity model is the reduced (2-D) pendulum')
    _check_X(X, Bx, L, ndim)
    plan = get_plan(B, Bx, ndim, precision, HP_REAL)
    plan.set_den_model(L, b, G, mR)
    return plan


def pendulum_propagate_reduced_den(F, f, X, mR, bt, G, dt, L, u, d, w, method='euler'):
    """Drop-in for pendulum_propagate_reduced_den(F,f,X,mR,bt,G,dt,L,u,d,w,method)
    (propagation/mex/sources/pendulum_propagate_reduced_den/kernel.cu:9-325).
    u, d and w are accepted for signature compatibility; f may be None."""
    plan = _den_plan(F, X, mR, bt, G, L, HP_FP64)
    return plan.propagate_den(F, f, dt, method)


def pendulum_propagate_reduced_den32(F, f, X, mR, bt, G, dt, L, u, d, w, method='euler'):
    """Mixed-precision twin of pendulum_propagate_reduced_den."""
    plan = _den_plan(F, X, mR, bt, G, L, HP_MIXED)
    return plan.propagate_den(F, f, dt, method)


def _bias_period(X, Bx: int) -> float:
    """Period L of the bias grid behind X = fftn(x) (gyro_bias.m:57-99):
    x_1 at the first grid point is -L/2; X must be that table."""
    X = np.asarray(X)
    L = -2.0 * float(np.real(np.fft.ifftn(X[..., 0]))[0, 0, 0])
    if not L > 0:
        raise HPError(HP_ERR_UNSUPPORTED, 'X is not fftn of a uniform grid over [-L/2, L/2)')
    _check_X(X, Bx, L, 3)
    return L


def _gyrobias_plan(F, X, G1, G2, precision):
    F = np.asarray(F)
    if F.ndim != 6:
        raise HPError(HP_ERR_SHAPE, 'the gyro-bias model has a 3-D bias: F is (2B-1, 2B-1, B, N, N, N)')
    B, Bx = F.shape[2], F.shape[3] // 2
    plan = get_plan(B, Bx, 3, precision, HP_REAL)
    plan.set_gyro_bias_model(_bias_period(X, Bx), G1, G2)
    return plan


def gyrobias_propagate(F, X, dt, u, G1, G2):
    """Drop-in for the MEX gyrobias_propagate(F,X,dt,u,G1,G2)
    (propagation/mex/sources/gyrobias_propagate/kernel.cu:8-130) and the
    integrate function of gyro_bias.m:226-300, FP64.  u is accepted for
    signature compatibility (the library builds getu.m's matrices itself)."""
    return _gyrobias_plan(F, X, G1, G2, HP_FP64).gyrobias_propagate(F, dt)


def gyrobias_propagate32(F, X, dt, u, G1, G2):
    """Mixed-precision twin of gyrobias_propagate."""
    return _gyrobias_plan(F, X, G1, G2, HP_MIXED).gyrobias_propagate(F, dt)


def fftSO3R_mex(direction: str, A, d=None, w=None, precision: int = HP_FP64):
    """Drop-in for fftSO3R_mex('forward', f, d, w) / fftSO3R_mex('backward', F, d)
    (propagation/mex/sources/fftSO3R/kernel.cu:5-392).  d and w are accepted for
    signature compatibility (the plan builds them on the device)."""
    A = np.asarray(A)
    if direction == 'forward':
        B, Bx, ndim = A.shape[0] // 2, A.shape[3] // 2, A.ndim - 3
        return get_plan(B, Bx, ndim, precision, HP_REAL).forward(A)
    if direction == 'backward':
        B, Bx, ndim = A.shape[2], A.shape[3] // 2, A.ndim - 3
        return get_plan(B, Bx, ndim, precision, HP_REAL).backward(A)
    raise ValueError("direction must be 'forward' or 'backward'")


def fftSO3R(f, precision: int = HP_FP64):
    """F = fftSO3R(f) for grid samples f (fftSO3R.m:89-106); complex f gives a complex plan."""
    f = np.asarray(f)
    B, Bx, ndim = f.shape[0] // 2, f.shape[3] // 2, f.ndim - 3
    sym = HP_COMPLEX if np.iscomplexobj(f) else HP_REAL
    return get_plan(B, Bx, ndim, precision, sym).forward(f)


def ifftSO3R(F, isreal: bool = True, precision: int = HP_FP64):
    """f = ifftSO3R(F) (ifftSO3R.m:16-37); isreal=True returns the real density
    (the 'symmetric' inverse of pendulum.m:303), False the complex samples."""
    F = np.asarray(F)
    B, Bx, ndim = F.shape[2], F.shape[3] // 2, F.ndim - 3
    return get_plan(B, Bx, ndim, precision, HP_REAL if isreal else HP_COMPLEX).backward(F)


def fftSO3_real(f):
    """F = fftSO3(f, B, true): real-harmonic coefficients of real samples
    f(a, j, c[, b]) (fftSO3.m:61-119), B = size(f, 1) / 2."""
    B = np.asarray(f).shape[0] // 2
    return get_plan(B, 2, 2).real_forward(f)


def ifftSO3_real(F):
    """f = ifftSO3(F, true) (ifftSO3.m:24-84), B = size(F, 3)."""
    return get_plan(np.asarray(F).shape[2], 2, 2).real_backward(F)


def fftSO3_prod_real(F, G):
    """FG of fftSO3_prod(func1, func2, B, true) (fftSO3_prod.m:97-205) from the
    real-harmonic coefficients F, G of the two functions."""
    return get_plan(np.asarray(F).shape[2], 2, 2).real_prod(F, G)


def fftSO3_prod(F, G):
    """FG of fftSO3_prod.m:247-264 from coefficient arrays F, G of shape
    (2lmax+1, 2lmax+1, lmax+1[, batch...]).  A batch of 1 uses any omega plan
    of the same B; the grid product fg is not returned (no function handles)."""
    F = np.asarray(F)
    B = F.shape[2]
    return get_plan(B, 2, 2, HP_FP64, HP_REAL).prod(F, G)
