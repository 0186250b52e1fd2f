"""Failure detection on the host side of the GPU path: the per-step health
guard of the resident state (NaN/Inf in the coefficients, l = 0 mass drift),
injected through host inputs, and device-allocation failure injected through
the library's device budget.  No kernel is made to fault: the failures are
made on the host and reported as status codes."""
import math

import numpy as np
import pytest

from oracle import pendulum as pd
from oracle import so3

pytestmark = pytest.mark.gpu

PRM = dict(d=0.12, h=0.2, r=0.025, theta_t=5 * math.pi / 180, lambda_max=100.0, epsilon=0.8)


def gyro_of(P):
    J = np.diag(P.params['J'])
    return ((J[1] - J[2]) / J[0], (J[2] - J[0]) / J[1], (J[0] - J[1]) / J[2])


def state3(hp, precision, B=4, Bx=3, seed=1):
    P = pd.pendulum_3d(B, Bx)
    plan = hp.Plan(B, Bx, 3, precision, hp.HP_REAL)
    plan.set_model(P.L, P.b, P.G, P.MR, gyro_of(P))
    f, _ = pd.seeded_density(B, Bx, 3, P.L, seed=seed)
    F = so3.fftSO3R_forward(f)
    st = hp.State(plan)
    st.load(F)
    return plan, st, F


@pytest.mark.parametrize('precision', [0, 1])
def test_guard_reports_nan_from_host_input(hp, precision):
    plan, st, F = state3(hp, precision)
    st.set_guard(1)
    st.step(1e-3, 'euler', 3)                    # healthy: no error
    Fbad = F.copy()
    Fbad[3, 3, 3, 1, 2, 0] = np.nan              # one poisoned coefficient (m = n = 0, l = 3)
    st.load(Fbad)
    with pytest.raises(hp.HPError) as e:
        st.step(1e-3, 'euler', 5)
    assert e.value.code == hp.HP_ERR_NONFINITE
    assert 'non-finite' in str(e.value) and 'step 4' in str(e.value)   # the first step after the load
    # without the guard the same state steps silently (the reference's behaviour)
    st.set_guard(0)
    st.step(1e-3, 'euler', 1)
    assert not np.isfinite(st.store()).all()


def test_guard_every_k_steps_and_mass_drift(hp):
    plan, st, F = state3(hp, 0)
    st.set_guard(4, mass_rtol=1e-12)
    st.step(1e-3, 'RK4', 7)                      # the derivative conserves F^0_00[0]: checks at 4 pass
    m = st.mass()
    st.normalize(1.5 * m)                        # a change made outside the propagation
    st.step(1e-3, 'euler', 0)
    with pytest.raises(hp.HPError) as e:
        st.step(1e-3, 'euler', 4)                # the next check is at step 8
    assert e.value.code == hp.HP_ERR_MASS_DRIFT
    assert 'step 8' in str(e.value)
    st.set_guard(1, mass_rtol=1e-12)             # re-arming takes the current mass as reference
    st.step(1e-3, 'euler', 2)


def test_guard_in_hybrid_step_and_batch(hp):
    B, Bx = 4, 3
    P = pd.pendulum_reduced(B, Bx, L=3.4)
    plan = hp.Plan(B, Bx, 2, hp.HP_FP64, hp.HP_REAL)
    plan.set_den_model(P.L, P.b, P.G, P.mR)
    c = hp.Collision(plan, L=3.4, Gd=0.0025 * np.eye(2), nD=10, **PRM)
    f, _ = pd.seeded_density(B, Bx, 2, P.L, seed=4, sigma=0.4)
    F = so3.fftSO3R_forward(f)
    st = hp.State(plan)
    st.load(F)
    st.set_guard(1)
    st.hybrid_step(c, 0.01, 'euler', 2)
    F[2 * (B - 1), 2 * (B - 1), B - 1, 0, 0] = np.inf      # m = n = l = lmax: a stored (m >= 0) row
    st.load(F)
    with pytest.raises(hp.HPError) as e:
        st.hybrid_step(c, 0.01, 'euler', 1)
    assert e.value.code == hp.HP_ERR_NONFINITE
    # a batch checks its guarded members after the replayed steps
    plan3, good, _ = state3(hp, 1, seed=5)
    plan3b, bad, Fb = state3(hp, 1, B=5, Bx=3, seed=6)
    good.set_guard(1)
    bad.set_guard(1)
    Fb[4, 4, 2, 0, 0, 0] = np.nan
    bad.load(Fb)
    batch = hp.Batch([good, bad])
    with pytest.raises(hp.HPError) as e:
        batch.step(1e-3, 'euler', 6)
    assert e.value.code == hp.HP_ERR_NONFINITE


def test_device_budget_makes_allocation_fail(hp):
    import gc
    gc.collect()
    base = hp.device_bytes()
    plan = hp.Plan(6, 4, 3, hp.HP_FP64, hp.HP_REAL)
    after_plan = hp.device_bytes()
    assert after_plan > base
    try:
        hp.set_device_budget(after_plan + 1024)          # no room for a state
        with pytest.raises(hp.HPError) as e:
            hp.State(plan)
        assert e.value.code == hp.HP_ERR_ALLOC
        with pytest.raises(hp.HPError) as e:
            hp.Plan(10, 8, 3, hp.HP_FP64, hp.HP_REAL)
        assert e.value.code == hp.HP_ERR_ALLOC
        assert hp.device_bytes() == after_plan          # the failed creations left nothing behind
    finally:
        hp.set_device_budget(0)
    st = hp.State(plan)
    assert hp.device_bytes() >= after_plan + plan.info.state_bytes
    del st
    gc.collect()
    assert hp.device_bytes() == after_plan
