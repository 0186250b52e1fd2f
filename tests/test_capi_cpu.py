"""The C ABI without a GPU: the library loads, exports every symbol that
include/hp.h declares, validates arguments and reports errors; host-side logic
of the Python mirror (MEX-argument checks) against the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

from oracle import pendulum as pd
from oracle import so3

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    h = open(os.path.join(ROOT, 'include', 'hp.h')).read()
    return re.findall(r'^\s*(?:int|const char\*)\s+(hp_\w+)\s*\(', h, re.M)


def test_every_declared_symbol_is_exported(hp):
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(hp._lib, s), s


def test_argument_validation_without_gpu(hp):
    lib = hp._lib
    h = ctypes.c_void_p()
    assert lib.hp_plan_create(ctypes.byref(h), 33, 2, 3, 0, 0) == hp.HP_ERR_INVALID     # B above 32
    assert b'bandlimit' in lib.hp_last_error()
    assert lib.hp_plan_create(ctypes.byref(h), 1, 2, 3, 0, 0) == hp.HP_ERR_INVALID      # B below 2
    assert lib.hp_plan_create(ctypes.byref(h), 4, 33, 3, 0, 0) == hp.HP_ERR_INVALID     # 2Bx = 66
    assert lib.hp_plan_create(ctypes.byref(h), 4, 1, 3, 0, 0) == hp.HP_ERR_INVALID      # 2Bx = 2
    assert lib.hp_plan_create(ctypes.byref(h), 4, 2, 4, 0, 0) == hp.HP_ERR_INVALID      # ndim
    assert lib.hp_plan_create(ctypes.byref(h), 4, 2, 3, 5, 0) == hp.HP_ERR_INVALID      # precision
    assert lib.hp_plan_create(None, 4, 2, 3, 0, 0) == hp.HP_ERR_INVALID
    assert lib.hp_plan_destroy(None) == hp.HP_OK
    assert lib.hp_state_step(None, ctypes.c_double(1e-3), 0, 1) == hp.HP_ERR_INVALID
    assert lib.hp_pendulum_propagate(None, None, None, ctypes.c_double(1e-3), 0, 0) == hp.HP_ERR_INVALID
    assert lib.hp_plan_set_beta_engine(None, hp.HP_BETA_TENSOR) == hp.HP_ERR_INVALID
    cnt = ctypes.c_int(-1)
    assert lib.hp_plan_tc_errors(None, ctypes.byref(cnt)) == hp.HP_ERR_INVALID


def test_device_budget_and_guard_arguments(hp):
    lib = hp._lib
    assert lib.hp_set_device_budget(-5) == hp.HP_ERR_INVALID
    assert lib.hp_set_device_budget(1 << 20) == hp.HP_OK
    assert lib.hp_set_device_budget(0) == hp.HP_OK
    v = ctypes.c_longlong(-1)
    assert lib.hp_device_bytes(ctypes.byref(v)) == hp.HP_OK and v.value >= 0
    assert lib.hp_device_bytes(None) == hp.HP_ERR_INVALID
    assert lib.hp_state_set_guard(None, 1, 0.0) == hp.HP_ERR_INVALID
    assert lib.hp_collision_lambda(None, None, None, None, None, None, 1) == hp.HP_ERR_INVALID
    assert lib.hp_collision_create_from_tables(None, 0, 1, None, None, None, None, 1, None) == hp.HP_ERR_INVALID


def test_host_read_in_place_arguments(hp):
    lib = hp._lib
    r = ctypes.c_int(-1)
    a = np.zeros(16, np.complex128)
    assert lib.hp_host_read_in_place(None, 16, ctypes.byref(r)) == hp.HP_ERR_INVALID
    assert lib.hp_host_read_in_place(ctypes.c_void_p(a.ctypes.data), 0, ctypes.byref(r)) == hp.HP_ERR_INVALID
    assert lib.hp_host_read_in_place(ctypes.c_void_p(a.ctypes.data), a.nbytes, None) == hp.HP_ERR_INVALID
    # pageable memory is never read in place (copied whole), with or without a device
    assert lib.hp_host_read_in_place(ctypes.c_void_p(a.ctypes.data), a.nbytes, ctypes.byref(r)) == hp.HP_OK
    assert r.value == 0
    assert hp.host_read_in_place(a) is False


def test_tune_cache_file_round_trip(hp, tmp_path):
    """The autotuner's cache file format: lines read back and written again
    unchanged; malformed lines are reported."""
    src = tmp_path / 'tune.txt'
    src.write_text('# comment\n15 16 3 1 0 0 2 8 16 1\n30 30 2 1 0 2 4 16 32 0\n')
    hp.tune_cache_load(str(src))
    out = tmp_path / 'out.txt'
    hp.tune_cache_save(str(out))
    lines = [l for l in out.read_text().splitlines() if not l.startswith('#')]
    assert '15 16 3 1 0 0 2 8 16 1' in lines and '30 30 2 1 0 2 4 16 32 0' in lines
    bad = tmp_path / 'bad.txt'
    bad.write_text('15 16 3 1 0 0 3 8 16 1\n')        # synth_pt 3 is not a choice
    with pytest.raises(hp.HPError):
        hp.tune_cache_load(str(bad))
    assert hp._lib.hp_plan_set_tune(None, 1, 1, 1, 1) == hp.HP_ERR_INVALID


def test_plan_creation_fails_cleanly_without_device(hp):
    import torch
    if torch.cuda.is_available():
        pytest.skip('a GPU is present')
    with pytest.raises(hp.HPError) as e:
        hp.Plan(4, 2, 3)
    assert e.value.code == hp.HP_ERR_CUDA


def test_getu_mirror_matches_oracle(hp):
    assert np.abs(hp.getu(6) - so3.getu(6)).max() == 0.0


def test_mex_argument_checks(hp):
    P = pd.pendulum_3d(3, 3)
    hp._check_X(P.X, 3, P.L, 3)
    with pytest.raises(hp.HPError):
        hp._check_X(P.X * 1.01, 3, P.L, 3)
    g = hp._fit_gyro(P.OJO, 3, P.L)
    J = np.diag(P.params['J'])
    ref = ((J[1] - J[2]) / J[0], (J[2] - J[0]) / J[1], (J[0] - J[1]) / J[2])
    assert np.allclose(g, ref, rtol=1e-10, atol=1e-12)
    Jfull = np.array([[0.02, 0.001, 0.0], [0.001, 0.02, 0.0], [0.0, 0.0, 0.01]])
    x = pd.omega_grid(3, P.L, 3)
    with pytest.raises(hp.HPError):
        hp._fit_gyro(pd.make_OJO(x, Jfull), 3, P.L)


GATEWAYS = [('HP_MEX_PROPAGATE3', 'pendulum_propagate', 11), ('HP_MEX_PROPAGATE2', 'pendulum_propagate_reduced', 10),
            ('HP_MEX_FFTSO3R', 'fftSO3R_mex', None), ('HP_MEX_GYROBIAS', 'gyrobias_propagate', 6),
            ('HP_MEX_PROPAGATE_DEN', 'pendulum_propagate_reduced_den', 12),
            ('HP_MEX_DISCRETE', 'pendulum_reduced_discrete_propagate', 6), ('HP_MEX_GETLAMBDA', 'getLambda_mex', 8),
            ('HP_MEX_GETOMEGA', 'getOmega_mex', 6), ('HP_MEX_GETFCL', 'getFcL_mex', 5)]


@pytest.mark.parametrize('define,name,nrhs', GATEWAYS)
def test_mex_gateway_builds_and_checks_arguments(define, name, nrhs):
    """Every MATLAB gateway (one source, one define each) builds against
    include/hp.h, libhp.so and the host-memory MEX runtime of tests/mex_stub,
    loads, and reports a wrong argument count through mexErrMsgIdAndTxt before
    it touches the device."""
    import shutil
    if shutil.which('gcc') is None:
        pytest.skip('no C compiler')
    import mexrt
    gw = mexrt.Gateway(mexrt.build_gateway(define, name))
    if define == 'HP_MEX_PROPAGATE3':
        mexrt.Gateway(mexrt.build_gateway(define, name + '32', ['-DHP_MEX_MIXED']))
    with pytest.raises(mexrt.MexError) as e:
        gw.call()
    if nrhs is not None:
        assert f'expected {nrhs} inputs' in str(e.value)


def test_mex_gateways_reject_unsupported_forms():
    """The noise-free forms of the discrete-only study are refused with a message."""
    import mexrt
    om = mexrt.Gateway(mexrt.build_gateway('HP_MEX_GETOMEGA', 'getOmega_mex'))
    with pytest.raises(mexrt.MexError, match="'new' direction"):
        om.call(np.zeros((3, 3, 2, 2, 2)), np.zeros((2, 4, 4)), np.zeros(1, np.int32), 0.8, np.zeros((3, 8)), 'old')
    dp = mexrt.Gateway(mexrt.build_gateway('HP_MEX_DISCRETE', 'pendulum_reduced_discrete_propagate'))
    with pytest.raises(mexrt.MexError, match='noisy form'):
        dp.call(False, 0.0, 0.0, 0.0, 0.0, 0.0)
