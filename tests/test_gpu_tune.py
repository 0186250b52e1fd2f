"""The launch-shape autotuner: every candidate shape of the synthesis and of
the tensor-core forward contraction gives the oracle's transforms (FP32 bar
1e-6), the tuner keeps one of them and later plans of the same key start from
it."""
import numpy as np
import pytest

from oracle import pendulum as pd
from oracle import so3

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


@pytest.mark.parametrize('B,Bx,ndim', [(15, 4, 3), (8, 6, 2), (30, 3, 2)])
def test_every_shape_matches_the_oracle(hp, B, Bx, ndim):
    f, _ = pd.seeded_density(B, Bx, ndim, 8.0, seed=B)
    F = so3.fftSO3R_forward(f)
    f_ref = so3.ifftSO3R_backward(F, real=True)
    plan = hp.Plan(B, Bx, ndim, hp.HP_MIXED, hp.HP_REAL)
    for pt in (1, 2, 4):
        for waves in (4, 16):
            for form in (0, 1):
                plan.set_tune(synth_pt=pt, synth_waves=waves, tc_waves=waves // 4 if form else waves * 2, tc_form=form)
                assert rel(plan.backward(F), f_ref) < 1e-6, (pt, waves, form)
                assert rel(plan.forward(f), F) < 1e-6, (pt, waves, form)
    assert plan.tc_errors() == 0


def test_autotune_keeps_a_candidate_and_caches_it(hp, tmp_path):
    plan = hp.Plan(15, 6, 2, hp.HP_MIXED, hp.HP_REAL)
    r = plan.autotune()
    assert r['synth_pt'] in (1, 2, 4) and r['synth_waves'] in (4, 8, 16) and r['tc_form'] in (0, 1)
    assert r['tc_waves'] in ((1, 2, 4) if r['tc_form'] else (8, 16, 32))
    assert r['backward_ms'] > 0 and r['forward_ms'] > 0
    again = hp.Plan(15, 6, 2, hp.HP_MIXED, hp.HP_REAL)
    assert again.get_tune() == plan.get_tune()
    path = tmp_path / 'tune.txt'
    hp.tune_cache_save(str(path))
    assert '15 6 2 1 0 0' in path.read_text()
    p64 = hp.Plan(15, 6, 2, hp.HP_FP64, hp.HP_REAL)
    r64 = p64.autotune()
    assert r64['synth_pt'] == 1 and r64['forward_ms'] == 0.0
