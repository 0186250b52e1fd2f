"""Generate the small golden fixtures of tests/golden/ from the FP64 oracle.

The reference ships no test vectors and its MATLAB code cannot run on these
machines, so the fixtures are outputs of the oracle's statement-by-statement
restatement (derivative_literal, the dense-CG product, the literal
transforms) on seeded inputs.  They pin the oracle against regressions and let
the GPU tests compare the CUDA path with stored vectors.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import pendulum as pd  # noqa: E402
from oracle import so3  # noqa: E402


def main():
    out = {}
    # 3-D pendulum, B=3, 4^3 omega grid
    P = pd.pendulum_3d(3, 2)
    f, _ = pd.seeded_density(3, 2, 3, P.L, seed=101)
    F = so3.fftSO3R_forward(f)
    out['p3_f'] = f
    out['p3_F'] = F
    out['p3_MR'] = P.MR
    out['p3_dF'] = pd.derivative_literal(F, P)
    for meth in ('euler', 'midpoint', 'RK2', 'RK4'):
        out[f'p3_Fnew_{meth}'] = pd.integrate(F, lambda G: pd.derivative_literal(G, P), 1e-3, meth)
    out['p3_fback'] = so3.ifftSO3R_backward(F, real=True)
    # 2-D reduced pendulum, B=3, 6^2 omega grid
    Q = pd.pendulum_reduced(3, 3)
    g, _ = pd.seeded_density(3, 3, 2, Q.L, seed=102)
    G = so3.fftSO3R_forward(g)
    out['p2_f'] = g
    out['p2_F'] = G
    out['p2_MR'] = Q.MR
    out['p2_dF'] = pd.derivative_literal(G, Q)
    out['p2_dF_den'] = pd.derivative_den(G, None, Q)
    # product rule, B=4
    rng = np.random.default_rng(103)
    lmax = 3
    A = np.zeros((7, 7, 4), np.complex128)
    C = np.zeros_like(A)
    for l in range(4):
        s = slice(lmax - l, lmax + l + 1)
        A[s, s, l] = rng.standard_normal((2 * l + 1,) * 2) + 1j * rng.standard_normal((2 * l + 1,) * 2)
        C[s, s, l] = rng.standard_normal((2 * l + 1,) * 2) + 1j * rng.standard_normal((2 * l + 1,) * 2)
    out['prod_F'] = A
    out['prod_G'] = C
    out['prod_FG'] = so3.fftSO3_prod(A, C)
    np.savez_compressed(os.path.join(HERE, 'pendulum_small.npz'), **out)
    print('wrote', os.path.join(HERE, 'pendulum_small.npz'), {k: v.shape for k, v in out.items()})


if __name__ == '__main__':
    main()
