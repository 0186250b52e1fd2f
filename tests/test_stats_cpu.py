"""Host-side fit of get_stat (proper SVD, matrix-Fisher parameters, Gaussian
part) against the oracle's restatement, on moments computed by the oracle."""
import importlib

import numpy as np
import pytest

from oracle import pendulum as pd
from oracle import so3
from oracle import stats as ost

pytestmark = pytest.mark.filterwarnings('ignore::scipy.integrate.IntegrationWarning')


@pytest.fixture(scope='module')
def pst():
    return importlib.import_module('hybridpendulum-up_b200.stats')


@pytest.mark.parametrize('s', [(5.0, 3.0, 1.0), (14.0, 9.0, -3.0), (0.3, 0.2, 0.1)])
def test_mf_parameters_round_trip(pst, s):
    d = ost.mf_dlogc(s)
    assert np.abs(pst.mf_first_moments(s) - d).max() < 1e-11
    assert np.abs(pst.mf_parameters(d) - np.array(s)).max() < 1e-7 * max(1.0, max(abs(v) for v in s))


def test_psvd_proper(pst):
    rng = np.random.default_rng(0)
    for _ in range(5):
        F = rng.standard_normal((3, 3))
        U, S, V = pst.psvd(F)
        assert abs(np.linalg.det(U) - 1) < 1e-12 and abs(np.linalg.det(V) - 1) < 1e-12
        assert np.abs(U @ S @ V.T - F).max() < 1e-12


@pytest.mark.parametrize('nd', [2, 3])
def test_get_stat_matches_oracle(pst, nd):
    B, Bx, L = 5, 3, 4.0
    f, _ = pd.seeded_density(B, Bx, nd, L, seed=4)
    ref = ost.get_stat_grid(f, L)
    out = pst.get_stat(ost.raw_moments_grid(f, L))
    for k in ('ER', 'Ex', 'Varx', 'EvR', 'ExvR', 'EvRvR', 'U', 'S', 'V', 'P', 'Miu', 'Sigma'):
        assert np.abs(out[k] - ref[k]).max() < 1e-8 * max(1.0, np.abs(ref[k]).max()), k
