"""Batched propagation (members of uneven bandlimit and omega grid, some
sharing a plan, some hybrid) against each member stepped on its own: the
batch replays a captured graph of the same kernels, so plain steps must be
bit-identical; hybrid steps are held to 1e-12 relative L2."""
import math

import numpy as np
import pytest

from oracle import pendulum as pd

pytestmark = pytest.mark.gpu


def make_member(hp, B, Bx, nd, precision, seed, plans):
    key = (B, Bx, nd, precision)
    if key not in plans:
        P = pd.pendulum_3d(B, Bx, L=8.0) if nd == 3 else pd.pendulum_reduced(B, Bx, L=8.0)
        plan = hp.Plan(B, Bx, nd, precision, hp.HP_REAL)
        gyro = (0.0, 0.0, 0.0)
        if nd == 3:
            J = np.diag(P.params['J'])
            gyro = ((J[1] - J[2]) / J[0], (J[2] - J[0]) / J[1], (J[0] - J[1]) / J[2])
        plan.set_model(P.L, P.b, P.G, P.MR, gyro)
        plans[key] = plan
    plan = plans[key]
    _, prm = pd.seeded_density(3, 2, nd, 8.0, seed=seed)   # seeded parameters only
    st = hp.State(plan)
    st.init_mf_gauss(prm['U'], prm['s'], prm['V'], prm['mu'], 0.25 * np.eye(nd))
    return st


@pytest.mark.parametrize('method,nsteps', [('euler', 7), ('RK4', 4)])
def test_batch_equals_members(hp, method, nsteps):
    shapes = [(4, 2, 3, 1), (6, 3, 3, 1), (4, 2, 3, 1), (5, 4, 3, 0), (8, 2, 2, 1)]
    plans, members = {}, []
    for k, (B, Bx, nd, prec) in enumerate(shapes):
        members.append(make_member(hp, B, Bx, nd, prec, 100 + k, plans))
    ref = []
    for st in members:            # each member alone, eager
        F0 = st.store()
        st.step(1e-3, method, nsteps)
        ref.append(st.store())
        st.load(F0)
    batch = hp.Batch(members)
    batch.step(1e-3, method, nsteps)
    info = batch.info()
    assert info['streams'] == len(plans)
    assert info['graph_launches'] >= 1
    for st, r in zip(members, ref):
        assert np.array_equal(st.store(), r)
    # a second call replays the graph without a new warm-up (after realigning
    # the ping-pong buffers with one eager step when the count so far is odd)
    batch.step(1e-3, method, 4)
    assert batch.info()['graph_launches'] > info['graph_launches']


def test_batch_hybrid_members(hp):
    prm = dict(d=0.12, h=0.2, r=0.025, theta_t=5 * math.pi / 180, lambda_max=100.0, epsilon=0.8)
    members, colls, plans = [], [], []
    for k, (B, Bx) in enumerate([(4, 3), (5, 4)]):
        P = pd.pendulum_reduced(B, Bx, L=3.4)
        plan = hp.Plan(B, Bx, 2, 0, hp.HP_REAL)
        plan.set_den_model(P.L, P.b, P.G, P.mR)
        plans.append(plan)
        c = hp.Collision(plan, L=P.L, Gd=0.0025 * np.eye(2), nD=10, **prm)
        _, q = pd.seeded_density(3, 2, 2, P.L, seed=7 + k)
        st = hp.State(plan)
        st.init_mf_gauss(q['U'], q['s'], q['V'], q['mu'], 0.25 * np.eye(2))
        members.append(st)
        colls.append(c)
    ref = []
    for st, c in zip(members, colls):
        F0 = st.store()
        st.hybrid_step(c, 1e-3, 'euler', 5)
        ref.append(st.store())
        st.load(F0)
    batch = hp.Batch(members, colls)
    batch.step(1e-3, 'euler', 5)
    for st, r in zip(members, ref):
        out = st.store()
        assert np.linalg.norm(out - r) <= 1e-12 * np.linalg.norm(r)


def test_persistent_plane_pass_equals_members(hp):
    """The plane passes of the plain Euler members on 3-D plans run as one
    persistent work-queue kernel per round of members (one member per plan and
    round); members of FP32 and FP64 plans, plans shared by several members, a
    grid outside the persistent kernel's set (2Bx = 4) and a 2-D member step
    beside them.  Every member ends as when stepped alone."""
    shapes = [(4, 4, 3, 1), (6, 6, 3, 1), (4, 4, 3, 1), (5, 4, 3, 0), (8, 8, 3, 1), (4, 4, 3, 1), (3, 2, 3, 1),
              (6, 2, 2, 1), (5, 4, 3, 0)]
    plans, members = {}, []
    for k, (B, Bx, nd, prec) in enumerate(shapes):
        members.append(make_member(hp, B, Bx, nd, prec, 200 + k, plans))
    ref = []
    for st in members:
        F0 = st.store()
        st.step(1e-3, 'euler', 9)
        ref.append(st.store())
        st.load(F0)
    batch = hp.Batch(members, persistent=True)
    batch.step(1e-3, 'euler', 5)
    batch.step(1e-3, 'euler', 4)
    assert batch.info()['graph_launches'] >= 1
    for st, r in zip(members, ref):
        out = st.store()
        assert np.linalg.norm(out - r) <= 1e-13 * np.linalg.norm(r)
