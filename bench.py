#!/usr/bin/env python
"""Benchmark of the pendulum Fokker-Planck step on SO(3) x R^3.

Workload (one "FP step" = the body of the time loop of pendulum.m:269-315
without the moment statistics): one Euler propagation of the coefficients F
(Lie, damping, gyroscopic, gravity and diffusion terms) followed by the
backward transform to the density f on the (alpha, beta, gamma, omega) grid.
B = 15 (30^3 Euler grid), omega grid 32^3 over [-4, 4]^3, dt = 1e-3,
J = diag(0.02, 0.02, 0.01), rho = (0, 0, 0.1), m = 1, g = 9.8, b = 0.05,
H = 0.2 I, seeded matrix-Fisher x Gaussian initial density (synthetic data).

`value` is the mixed-precision step (FP32 operators and transforms, FP64
coefficient accumulation) in steps/s over all ranks; the FP64 step on the same
inputs is timed beside it and the two results are compared (relative L2).
Every rank runs an independent replica (the step does not shard).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import importlib
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FP steps/s at B=15, ω 32³: mixed-precision vs FP64 on GPU, at ≤1e-6 rel L2"
PEAKS_FALLBACK = {'hbm_gbs': 6650.0, 'bf16_tflops': 1590.0}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--B', type=int, default=15)
    ap.add_argument('--Bx', type=int, default=16)
    ap.add_argument('--e2e-steps', type=int, default=2)
    ap.add_argument('--no-e2e', action='store_true')
    ap.add_argument('--no-cpu', action='store_true')
    ap.add_argument('--fp64-steps', type=int, default=None)
    ap.add_argument('--workload', default='step', choices=['step', 'batch', 'transform', 'hybrid', 'forward', 'adjoint'],
                    help='step: the headline FP step; batch: uneven-bandlimit batch of densities; '
                         'transform: B=32 round-trip precision stress; hybrid: the loop of '
                         'pendulum_reduced_hybrid.m at its own sizes (B=30, 60x60 omega); '
                         'forward: one FP32 forward transform on a 2-D omega grid (--B, --Bx, --beta-engine); '
                         'adjoint: the gradient of a terminal loss through 50 Euler steps at B=12, 24^3')
    ap.add_argument('--members', type=int, default=64)
    ap.add_argument('--persistent', action='store_true',
                    help='batch workload: plane passes of the plain members in one persistent launch per round')
    ap.add_argument('--coll-gb', type=float, default=24.0,
                    help='batch workload: device memory for 3-D collision tables; the members whose plans fit '
                         '(smallest first) run the hybrid step with the collision reset map')
    ap.add_argument('--tc-form', type=int, default=-1, choices=[-1, 0, 1],
                    help='forward workload: tensor-core kernel form (1 warp-specialised TMA pipeline, 0 staged)')
    ap.add_argument('--no-autotune', action='store_true',
                    help='keep the hand-picked launch shapes instead of timing the candidates first')
    ap.add_argument('--beta-engine', default='auto', choices=['auto', 'simt', 'tensor', 'tensor_bf16'],
                    help='forward-transform beta contraction (transform, hybrid and forward workloads): '
                         'tensor = 3xTF32, tensor_bf16 = BF16x3 on the tcgen05 tensor cores')
    return ap.parse_args()


def load_peaks():
    p = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    try:
        with open(p) as fh:
            d = json.load(fh)
        return {'hbm_gbs': float(d['hbm_gbs']), 'bf16_tflops': float(d['bf16_tflops'])}, 'measured'
    except Exception:
        return dict(PEAKS_FALLBACK), 'fallback'


# ------------------------------------------------------------ physics ----
PARAMS = dict(J=(0.02, 0.02, 0.01), rho=(0.0, 0.0, 0.1), mass=1.0, g=9.8, b=0.05, H=0.2, L=8.0, dt=1e-3)


def rotation_grid(B):
    k = np.arange(2 * B)
    al, be, ga = np.pi / B * k, np.pi / (4 * B) * (2 * k + 1), np.pi / B * k

    def rz(t):
        c, s = np.cos(t), np.sin(t)
        z, o = np.zeros_like(t), np.ones_like(t)
        return np.stack([np.stack([c, -s, z], -1), np.stack([s, c, z], -1), np.stack([z, z, o], -1)], -2)

    def ry(t):
        c, s = np.cos(t), np.sin(t)
        z, o = np.zeros_like(t), np.ones_like(t)
        return np.stack([np.stack([c, z, s], -1), np.stack([z, o, z], -1), np.stack([-s, z, c], -1)], -2)

    return np.einsum('aij,bjk,ckl->abcil', rz(al), ry(be), rz(ga))   # [a, b, c, 3, 3]


def mf_normaliser(s):
    from scipy.integrate import quad
    from scipy.special import iv
    v, _ = quad(lambda u: 0.5 * math.exp(s[2] * u) * iv(0, 0.5 * (s[0] - s[1]) * (1 - u))
                * iv(0, 0.5 * (s[0] + s[1]) * (1 + u)), -1, 1, epsabs=0, epsrel=1e-13, limit=200)
    return v


def model_inputs(hp, B, Bx, seed=0):
    """MR (via the library's own forward transform of the gravity multiplier),
    gyro coefficients and the seeded initial density factors."""
    P = PARAMS
    J = np.diag(P['J'])
    rho = np.array(P['rho'])
    hat = np.array([[0, -rho[2], rho[1]], [rho[2], 0, -rho[0]], [-rho[1], rho[0], 0]])
    A = np.linalg.inv(J) @ (-P['mass'] * P['g'] * hat)
    R = rotation_grid(B)
    mR = np.einsum('ij,abcj->iabc', A, R[..., 2, :])                 # (3, a, b, c)
    # SO(3)-only transform through a 2-D plan with a constant omega profile
    aux = hp.Plan(B, 2, 2, hp.HP_FP64, hp.HP_REAL)
    MR = np.zeros((2 * B - 1, 2 * B - 1, B, 3), np.complex128)
    for i in range(3):
        f = np.broadcast_to(mR[i][..., None, None], mR[i].shape + (4, 4))
        MR[..., i] = aux.forward(np.ascontiguousarray(f))[..., 0, 0] / 16.0
    Jd = np.diag(J)
    gyro = ((Jd[1] - Jd[2]) / Jd[0], (Jd[2] - Jd[0]) / Jd[1], (Jd[0] - Jd[1]) / Jd[2])
    G = 0.5 * (P['H'] * np.eye(3)) @ (P['H'] * np.eye(3)).T
    b = np.full(3, P['b'])
    # seeded matrix-Fisher(R; U diag(s) V^T) x N(omega; mu, 0.5^2 I)
    rng = np.random.default_rng(seed)

    def haar():
        Q, Rr = np.linalg.qr(rng.standard_normal((3, 3)))
        Q = Q * np.sign(np.diag(Rr))
        if np.linalg.det(Q) < 0:
            Q[:, 0] = -Q[:, 0]
        return Q

    U, V = haar(), haar()
    s = np.sort(rng.uniform(5, 20, 3))[::-1]
    mu = rng.uniform(-1, 1, 3)
    Fm = U @ np.diag(s) @ V.T
    fR = np.exp(np.einsum('ij,abcij->abc', Fm, R)) / mf_normaliser(s)   # (a, b, c)
    return dict(MR=MR, gyro=gyro, G=G, b=b, fR=fR, mu=mu, sigma=0.5)


def initial_density_dev(torch, inp, B, Bx, L, dev):
    """f(a,b,c,w) in the MATLAB column-major layout, built on the device."""
    N = 2 * Bx
    g1 = -L / 2 + L / N * torch.arange(N, dtype=torch.float64, device=dev)
    x1, x2, x3 = torch.meshgrid(g1, g1, g1, indexing='ij')
    mu = inp['mu']
    r2 = (x1 - mu[0]) ** 2 + (x2 - mu[1]) ** 2 + (x3 - mu[2]) ** 2
    sig = inp['sigma']
    fx = torch.exp(-0.5 * r2 / sig ** 2) / math.sqrt((2 * math.pi * sig ** 2) ** 3)
    fx = fx.permute(2, 1, 0).reshape(-1)                               # omega index i + N j + N^2 k
    fR = torch.from_numpy(np.ascontiguousarray(np.transpose(inp['fR'], (2, 1, 0)))).to(dev).reshape(-1)
    return (fx[:, None] * fR[None, :]).reshape(-1)                      # [w][c][b][a]


# ------------------------------------------------------------- clocks ----
class Clocks:
    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.idx), f'--query-gpu={self.FIELDS}',
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['nvidia-smi unavailable']}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ''
        sm, smax, reasons = [], None, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(',')]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == 'active':
                    reasons.add(nm)
        return {'sm_mhz': float(np.median(sm)) if sm else None, 'sm_max_mhz': smax,
                'reasons': sorted(reasons), 'samples': len(sm)}


# ---------------------------------------------------------- roofline ----
def algorithmic_bytes(plan, family, mixed):
    """Compulsory bytes of one launch of a kernel family (each operand once)."""
    pts = plan.nrows * plan.nx                   # stored coefficient points
    c64, cT = 16, (8 if mixed else 16)
    rT = 4 if mixed else 8
    ngrid = (2 * plan.B) ** 3 * plan.nx
    return {
        'deriv.plane': pts * (c64 + cT + cT + c64),   # F in, P3 in, G in, F out
        'deriv.axis3': pts * (c64 + cT),
        'deriv.local': pts * (c64 + cT),
        'tf.wplane': pts * (c64 + cT),
        'tf.wline': pts * (cT + cT),
        'tf.transpose': pts * (cT + cT),
        'tf.synth': pts * cT + ngrid * rT,
    }.get(family)


# ------------------------------------------------------------ CPU leg ----
def cpu_sample(B, Bx_sample, nsteps, workers):
    """FP64 oracle (restatement) step on B, (2 Bx_sample)^3: Euler propagate +
    density synthesis.  Returns seconds per step."""
    from oracle import pendulum as pd
    from oracle import so3
    import scipy.fft
    P = pd.pendulum_3d(B, Bx_sample, J=PARAMS['J'], rho=PARAMS['rho'], mass=PARAMS['mass'], g=PARAMS['g'],
                       b=PARAMS['b'], H=PARAMS['H'], L=PARAMS['L'])
    f, _ = pd.seeded_density(B, Bx_sample, 3, P.L, seed=0)
    with scipy.fft.set_workers(workers):
        F = so3.fftSO3R_forward(f)
        pd.gravity_taps(B - 1, P.MR[B - 2:B + 1, B - 2:B + 1, 1, 0])   # warm the CG cache
        t0 = time.perf_counter()
        for _ in range(nsteps):
            F = pd.integrate(F, lambda G: pd.derivative_fast(G, P), PARAMS['dt'], 'euler')
            so3.ifftSO3R_backward(F, real=True)
        return (time.perf_counter() - t0) / nsteps


def cpu_baseline_obj(B, Bx, steps=1):
    Bs = 4                               # omega 8^3 sample
    workers = os.cpu_count() or 1
    sec = cpu_sample(B, Bs, steps, workers)
    scale = (Bx / Bs) ** 3               # omega points of the full grid per sample point
    val = 1.0 / (sec * scale)
    return {'value': val, 'unit': 'steps/s', 'cores': workers, 'kind': 'port',
            'sample': f'FP64 numpy oracle (restatement, fast form: omega FFTs, degree-1 CG gravity), '
                      f'B={B} on a {2 * Bs}^3 omega grid, {steps} step(s) of Euler propagate + density '
                      f'synthesis, {sec:.2f} s/step, scaled by omega points x{scale:.0f} to {2 * Bx}^3 '
                      f'(cost per omega point taken as constant in the grid size)'}


# ------------------------------------------------------------ replicas ----
def replica_seed(rank: int) -> int:
    """Each rank propagates its own independent density (no data exchange)."""
    return rank


def max_over_ranks(value: float, world: int, device=None) -> float:
    """Slowest rank's time: the job's time for weak-scaled replicas."""
    if world <= 1:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, steps: int, max_ms: float) -> float:
    """Steps/s of the whole job: every rank did `steps` steps in `max_ms`."""
    return world * steps / (max_ms / 1e3)


# ---------------------------------------------------------------- main ----
def main():
    args = parse()
    rank = int(os.environ.get('RANK', '0'))
    world = int(os.environ.get('WORLD_SIZE', '1'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    B, Bx = args.B, args.Bx

    if args.workload == 'batch':
        return bench_batch(args, rank, world, local)
    if args.workload == 'transform':
        return bench_transform(args, rank, local)
    if args.workload == 'hybrid':
        return bench_hybrid(args, rank, local)
    if args.workload == 'forward':
        return bench_forward(args, rank, local)
    if args.workload == 'adjoint':
        return bench_adjoint(args, rank, local)
    if args.impl == 'reference':
        if rank != 0:
            return 0
        cb = cpu_sample_loop(args, B, Bx)
        print(json.dumps(cb), flush=True)
        return 0

    import torch
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    if world > 1:
        import datetime
        torch.distributed.init_process_group('nccl', timeout=datetime.timedelta(seconds=600))
    hp = importlib.import_module('hybridpendulum-up_b200')
    stream = torch.cuda.current_stream(dev)
    inp = model_inputs(hp, B, Bx, seed=replica_seed(rank))
    L, dt = PARAMS['L'], PARAMS['dt']

    def make(prec):
        pl = hp.Plan(B, Bx, 3, prec, hp.HP_REAL)
        pl.set_stream(stream.cuda_stream)
        pl.set_model(L, inp['b'], inp['G'], inp['MR'], inp['gyro'])
        return pl

    pmix, p64 = make(hp.HP_MIXED), make(hp.HP_FP64)
    tunes = {}
    if not args.no_autotune:     # launch shapes timed on scratch, before (and outside) the timed region
        tunes = {'mixed': pmix.autotune(), 'fp64': p64.autotune()}
    f0 = initial_density_dev(torch, inp, B, Bx, L, dev)
    F0 = torch.zeros(int(np.prod(p64.F_shape)), dtype=torch.complex128, device=dev)
    p64.forward(f0, out=F0)
    del f0
    smix, s64 = hp.State(pmix), hp.State(p64)
    smix.load(F0)
    s64.load(F0)
    ngrid = (2 * B) ** 3 * pmix.nx
    fmix = torch.empty(ngrid, dtype=torch.float32, device=dev)
    f64 = torch.empty(ngrid, dtype=torch.float64, device=dev)
    mass0 = smix.mass()

    def step(state, fout):
        state.step(dt, 'euler', 1)
        state.density_into(fout.data_ptr())

    def barrier():
        torch.cuda.synchronize(dev)
        if world > 1:
            torch.distributed.barrier()

    def timed(state, fout, plan, K, W, profile=False):
        # the clock sampler (200 ms period) starts before the warm-up so that
        # its samples cover the whole timed region
        clk = Clocks(local)
        clk.start()
        for _ in range(W):
            step(state, fout)
        barrier()
        if profile:
            plan.profile(True)
        n0 = plan.launch_count()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(K):
            step(state, fout)
        ev1.record(stream)
        barrier()
        time.sleep(0.25)                 # one more sample after the timed region
        clocks = clk.stop()
        ms = ev0.elapsed_time(ev1)
        prof = plan.profile_read() if profile else {}
        if profile:
            plan.profile(False)
        launches = plan.launch_count() - n0
        return max_over_ranks(ms, world, dev), clocks, prof, launches

    K, W = args.steps, max(args.warmup, 3)
    ms_mix, clocks, prof, launches = timed(smix, fmix, pmix, K, W, profile=False)
    # per-kernel device time of the same timed loop, in a second pass with event brackets
    _, _, prof, _ = timed(smix, fmix, pmix, K, 1, profile=True)
    K64 = args.fp64_steps or K
    ms_64, clocks64, _, _ = timed(s64, f64, p64, K64, W, profile=False)
    _, _, prof64, _ = timed(s64, f64, p64, K64, 1, profile=True)

    # accuracy of the mixed step against the FP64 step from the same state
    ta = hp.State(pmix)
    tb = hp.State(p64)
    Fs = torch.zeros_like(F0)
    s64.store(Fs)
    ta.load(Fs)
    tb.load(Fs)
    ta.step(dt, 'euler', 1)
    tb.step(dt, 'euler', 1)
    Fa = torch.zeros_like(F0)
    Fb = torch.zeros_like(F0)
    ta.store(Fa)
    tb.store(Fb)
    dF = (Fa - Fs) - (Fb - Fs)
    err_step = float(torch.linalg.vector_norm(dF) / torch.linalg.vector_norm(Fb - Fs))
    err_F = float(torch.linalg.vector_norm(Fa - Fb) / torch.linalg.vector_norm(Fb))
    ta.density_into(fmix.data_ptr())
    tb.density_into(f64.data_ptr())
    err_f = float(torch.linalg.vector_norm(fmix.double() - f64) / torch.linalg.vector_norm(f64))
    err_fmax = float((fmix.double() - f64).abs().max() / f64.abs().max())
    mass_drift = abs(smix.mass() - mass0) / abs(mass0)
    del ta, tb, Fs, Fa, Fb, dF

    value = whole_job_rate(world, K, ms_mix)
    value64 = whole_job_rate(world, K64, ms_64)

    # roofline of the dominant kernel family
    peaks, peak_src = load_peaks()
    fam = max(prof, key=lambda k: prof[k][0]) if prof else None
    roof = None
    if fam:
        tot_ms, cnt = prof[fam]
        per = tot_ms / max(cnt, 1)
        ab = algorithmic_bytes(pmix, fam, True)
        if ab:
            ach = ab / (per / 1e3) / 1e9
            traffic = None
            try:
                with open(os.path.join(ROOT, 'profiles', 'traffic.json')) as fh:
                    tj = json.load(fh).get(fam)
                if tj and B == 15 and Bx == 16:
                    traffic = int(tj['bytes_per_launch'])
            except Exception:
                traffic = None
            roof = {'bound': 'hbm', 'kernel': fam, 'achieved': round(ach, 1), 'peak': peaks['hbm_gbs'],
                    'unit': 'GB/s', 'frac': round(ach / peaks['hbm_gbs'], 4), 'traffic': traffic,
                    'peak_source': peak_src, 'ms_per_launch': round(per, 4),
                    'algorithmic_bytes_per_launch': int(ab)}
    kernel_ms = {k: round(v[0] / max(v[1], 1), 4) for k, v in prof.items()}
    step_share = {k: round(v[0] / sum(x[0] for x in prof.values()), 4) for k, v in prof.items()} if prof else {}

    # end to end through the MEX-shaped C ABI with pinned host buffers
    e2e = None
    if not args.no_e2e and args.e2e_steps > 0:
        Fh = torch.empty(int(np.prod(pmix.F_shape)), dtype=torch.complex128, pin_memory=True)
        Fh.copy_(F0.cpu())
        Fn = torch.empty_like(Fh).pin_memory()
        fh = torch.empty(ngrid, dtype=torch.float64, pin_memory=True)
        del F0
        torch.cuda.empty_cache()
        pmix.propagate(Fh, dt, 'euler', out=Fn)     # warm-up: workspace allocation
        pmix.backward(Fn, out=fh)
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            pmix.propagate(Fh, dt, 'euler', out=Fn)
            pmix.backward(Fn, out=fh)
            Fh, Fn = Fn, Fh
        barrier()
        dt_e2e = max_over_ranks(time.perf_counter() - t0, world, dev)
        # two F inputs per step: read in place from the pinned buffers (only the
        # entries the plan keeps cross the bus) or copied whole
        in_place = hp.host_read_in_place(Fh) and hp.host_read_in_place(Fn)
        bi = 2 * (pmix.nrows * pmix.nx if in_place else Fh.numel()) * 16
        bo = Fh.numel() * 16 + fh.numel() * 8
        e2e = {'value': whole_job_rate(world, args.e2e_steps, dt_e2e * 1e3), 'unit': 'steps/s',
               'h2d_bytes_per_step': bi, 'd2h_bytes_per_step': bo,
               'h2d': ('kept entries read in place from the pinned MATLAB-layout F buffers (full buffers: '
                       f'{2 * Fh.numel() * 16} bytes)') if in_place else 'full MATLAB-layout F buffers copied',
               'api': 'hp_pendulum_propagate + hp_fftSO3R_backward, host (pinned) MATLAB-layout buffers'}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            cpu = cpu_baseline_obj(B, Bx)
        except Exception as e:   # the GPU number stands without it
            cpu = {'value': None, 'error': str(e)[:200]}

    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        'metric': METRIC, 'value': round(value, 3), 'unit': 'steps/s', 'n_gpus': world, 'steps': K,
        'warmup': W, 'ms_per_step': round(ms_mix / K, 4), 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'f32 (f64 accumulation)', 'data': 'synthetic',
        'config': {'workload': f'pendulum FP step: Euler propagate + density synthesis, B={B}, '
                               f'omega {2 * Bx}^3, dt={dt}',
                   'B': B, 'omega_grid': f'{2 * Bx}^3', 'ndim': 3, 'dt': dt, 'method': 'euler',
                   'parallelism': f'replicas x{world}', 'l2': 'inputs larger than L2 (F state 1.24 GB)',
                   'step_includes': ['derivative (Lie, damping, gyroscopic, CG gravity, diffusion)',
                                     'Euler update (FP64)', 'inverse omega FFT', 'SO(3) synthesis to f'],
                   'launch_shapes': tunes or 'hand-picked (--no-autotune)'},
        'fp64': {'value': round(value64, 3), 'ms_per_step': round(ms_64 / K64, 4), 'steps': K64,
                 'clocks_sm_mhz': clocks64.get('sm_mhz'),
                 'kernel_ms_per_launch': {k: round(v[0] / max(v[1], 1), 4) for k, v in prof64.items()}},
        'speedup_mixed_vs_fp64': round(value / value64, 3),
        'accuracy_mixed_vs_fp64': {'step_increment_rel_l2': err_step, 'F_rel_l2': err_F,
                                   'density_rel_l2': err_f, 'density_max_rel': err_fmax,
                                   'mass_drift_rel': mass_drift},
        'roofline': roof,
        'kernel_ms_per_launch': kernel_ms,
        'kernel_time_share': step_share,
        'cpu_baseline': cpu,
        'e2e': e2e,
        'gpu_launches': launches,
        'clocks': clocks,
    }
    print(json.dumps(line), flush=True)
    return 0


def bench_batch(args, rank, world, local):
    """Independent seeded densities with bandlimits B in {8, 12, 16, 20} and
    omega grids {16^3, 24^3, 32^3} mixed by the seed, advanced together in
    mixed precision (one CUDA graph per two batch steps, members on distinct
    plans concurrent, launch shapes autotuned per plan), against the
    per-density FP64 loop.  Members whose plans' collision tables fit in
    --coll-gb (smallest plans first; the 3-D tables hold numR x nx x nD taps)
    take the hybrid step of pendulum_reduced_hybrid.m:224-234 with the 3-D
    collision reset map (propagate, backward transform, collision update,
    forward transform); the others the plain propagation.  Prints one JSON
    line (not the headline)."""
    import torch
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    hp = importlib.import_module('hybridpendulum-up_b200')
    rng = np.random.default_rng(1000 + rank)
    Bs, Bxs = [8, 12, 16, 20], [8, 12, 16]
    shapes = [(int(rng.choice(Bs)), int(rng.choice(Bxs))) for _ in range(args.members)]
    L, dt = PARAMS['L'], PARAMS['dt']
    inputs, plans = {}, {}
    for B, _ in shapes:
        if B not in inputs:
            inputs[B] = model_inputs(hp, B, 2, seed=0)

    def plan(B, Bx, prec):
        pl = hp.Plan(B, Bx, 3, prec, hp.HP_REAL)
        inp = inputs[B]
        pl.set_model(L, inp['b'], inp['G'], inp['MR'], inp['gyro'])
        return pl

    def params(k):
        r = np.random.default_rng(5000 + k)
        Q = []
        for _ in range(2):
            q, rr = np.linalg.qr(r.standard_normal((3, 3)))
            q = q * np.sign(np.diag(rr))
            if np.linalg.det(q) < 0:
                q[:, 0] = -q[:, 0]
            Q.append(q)
        return Q[0], np.sort(r.uniform(5, 20, 3))[::-1], Q[1], r.uniform(-1, 1, 3)

    # which plans take the collision reset map: count the colliding attitudes
    # (cheap), then admit plans smallest-table first within the memory budget
    CPRM = dict(d=0.12, h=0.2, r=0.025, theta_t=5 * math.pi / 180, lambda_max=100.0, epsilon=0.8)
    Gd3 = (0.05 * np.eye(3)) @ (0.05 * np.eye(3)).T
    nD = 10
    table_bytes = {}
    for key in sorted(set(shapes)):
        numR = hp.collision_count(plan(key[0], key[1], hp.HP_FP64), L=L, **{k: CPRM[k] for k in
                                                                          ('d', 'h', 'r', 'theta_t', 'lambda_max')})
        nx = (2 * key[1]) ** 3
        # FP64 tables (lambda, Omega+, fcL, 16-bit indices) + transposed copies in the compute precision
        table_bytes[key] = numR * nx * (8 + 24 + nD * 10 + (nD * 6 + 4))
    hybrid_plans, used = set(), 0
    for key in sorted(table_bytes, key=lambda k: table_bytes[k]):
        if used + table_bytes[key] <= args.coll_gb * 1e9:
            hybrid_plans.add(key)
            used += table_bytes[key]

    def stepper(st, c):
        return (lambda n: st.hybrid_step(c, dt, 'euler', n)) if c is not None else (lambda n: st.step(dt, 'euler', n))

    # per-density FP64 loop (timed on every member, a few steps each)
    k64 = 3
    t64 = 0.0
    ref = {}
    nsample = 2
    for key in sorted(set(shapes)):
        p64 = plan(key[0], key[1], hp.HP_FP64)
        c64 = hp.Collision(p64, L=L, Gd=Gd3, nD=nD, **CPRM) if key in hybrid_plans else None
        st = hp.State(p64)
        adv = stepper(st, c64)
        for k, sh in enumerate(shapes):
            if sh != key:
                continue
            U, s_, V, mu = params(k)
            st.init_mf_gauss(U, s_, V, mu, 0.25 * np.eye(3))
            adv(1)
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            adv(k64)
            e1.record()
            torch.cuda.synchronize(dev)
            t64 += e0.elapsed_time(e1)
            if k < nsample:
                st.init_mf_gauss(U, s_, V, mu, 0.25 * np.eye(3))
                adv(args.warmup + args.steps)
                ref[k] = st.store()
        del st, c64, p64
        torch.cuda.empty_cache()
    rate64 = args.members * k64 / (t64 / 1e3)
    # the batch (mixed precision)
    for key in sorted(set(shapes)):
        plans[key] = plan(key[0], key[1], hp.HP_MIXED)
        if not args.no_autotune:
            plans[key].autotune()
    colls = {key: hp.Collision(plans[key], L=L, Gd=Gd3, nD=nD, **CPRM) for key in hybrid_plans}
    states, member_colls = [], []
    for k, sh in enumerate(shapes):
        st = hp.State(plans[sh])
        U, s_, V, mu = params(k)
        st.init_mf_gauss(U, s_, V, mu, 0.25 * np.eye(3))
        states.append(st)
        member_colls.append(colls.get(sh))
    batch = hp.Batch(states, member_colls, persistent=args.persistent)
    batch.step(dt, 'euler', args.warmup)          # warm-up and graph capture
    torch.cuda.synchronize(dev)
    accuracy = None
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record()
    batch.step(dt, 'euler', args.steps)
    e1.record()
    torch.cuda.synchronize(dev)
    wall = time.perf_counter() - t0
    ms = e0.elapsed_time(e1)
    info = batch.info()
    errs = [float(np.linalg.norm(states[k].store() - ref[k]) / np.linalg.norm(ref[k])) for k in ref]
    accuracy = max(errs)
    rate = args.members * args.steps / (ms / 1e3)
    hist = {}
    for B, Bx in shapes:
        hist[f'B{B}_omega{2 * Bx}^3'] = hist.get(f'B{B}_omega{2 * Bx}^3', 0) + 1
    out = {'metric': 'batched FP member-steps/s (uneven bandlimits and omega grids)', 'value': round(rate, 2),
           'unit': 'member-steps/s', 'n_gpus': 1, 'steps': args.steps, 'warmup': args.warmup,
           'ms_per_batch_step': round(ms / args.steps, 3), 'host_wall_s': round(wall, 3),
           'higher_is_better': True, 'dtype': 'f32 (f64 accumulation)', 'data': 'synthetic',
           'config': {'workload': 'batch of pendulum FP steps (Euler, dt=1e-3): hybrid steps with the 3-D collision '
                                  'reset map for the members whose tables fit, plain propagation for the rest',
                      'members': args.members, 'shapes': hist, 'distinct_plans': len(plans),
                      'hybrid_members': sum(1 for c in member_colls if c is not None),
                      'collision_table_gb': round(used / 1e9, 2), 'persistent_plane_pass': args.persistent,
                      'launch_shapes': 'autotuned per plan' if not args.no_autotune else 'hand-picked'},
           'fp64_per_density_loop': {'value': round(rate64, 2), 'unit': 'member-steps/s', 'steps_each': k64},
           'speedup_vs_fp64_loop': round(rate / rate64, 3),
           'graph_launches': info['graph_launches'], 'concurrent_streams': info['streams'],
           'max_rel_l2_vs_fp64_loop': accuracy}
    if rank == 0:
        print(json.dumps(out), flush=True)
    return 0


def bench_transform(args, rank, local):
    """ifftSO3R -> fftSO3R round trip at B=32 (64^3 Euler grid) on a 24^3 omega
    grid, complex coefficients i.i.d. N(0,1)/(2l+1) per degree (seeded), in FP64
    and in mixed precision; errors are relative L2 against the input (the FP64
    round trip is the identity up to rounding) and against the FP64 density.
    Prints one JSON line (not the headline)."""
    import torch
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    hp = importlib.import_module('hybridpendulum-up_b200')
    B, Bx = 32, 12
    lmax = B - 1
    D = 2 * lmax + 1
    N = 2 * Bx
    g = torch.Generator(device=dev).manual_seed(7 + rank)
    shape = (N, N, N, lmax + 1, D, D)        # reversed MATLAB order, C-contiguous
    F = torch.empty(shape, dtype=torch.complex128, device=dev)
    Fr = torch.view_as_real(F)
    Fr.normal_(generator=g)
    l = torch.arange(lmax + 1, device=dev).view(-1, 1, 1)
    m = (torch.arange(D, device=dev) - lmax).view(1, 1, -1)
    n = (torch.arange(D, device=dev) - lmax).view(1, -1, 1)
    scale = (((m.abs() <= l) & (n.abs() <= l)).to(torch.float64) / (2 * l + 1)).view(1, lmax + 1, D, D, 1)
    Fr.view(N * N * N, lmax + 1, D, D, 2).mul_(scale)
    del Fr
    torch.cuda.empty_cache()       # the library allocates with cudaMalloc, outside torch's cache
    nF = torch.linalg.vector_norm(F).item()
    out = {}
    fsample = None
    ns = (2 * B) ** 3 * N * N * 2            # first two omega planes of the density
    for name, prec in (('fp64', hp.HP_FP64), ('mixed', hp.HP_MIXED)):
        plan = hp.Plan(B, Bx, 3, prec, hp.HP_COMPLEX)
        plan.set_beta_engine(beta_engine(hp, args))
        st = hp.State(plan)
        cdt = torch.complex128 if prec == hp.HP_FP64 else torch.complex64
        f = torch.empty((2 * B) ** 3 * N ** 3, dtype=cdt, device=dev)
        st.load(F)
        st.density_into(f.data_ptr())
        st.load_density(f.data_ptr())
        torch.cuda.synchronize(dev)
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        st.load(F)
        torch.cuda.synchronize(dev)
        e[0].record()
        st.density_into(f.data_ptr())
        e[1].record()
        st.load_density(f.data_ptr())
        e[2].record()
        torch.cuda.synchronize(dev)
        r = {'backward_ms': round(e[0].elapsed_time(e[1]), 2), 'forward_ms': round(e[1].elapsed_time(e[2]), 2)}
        if fsample is None:
            fsample = f[:ns].clone()
        else:
            r['density_rel_l2_vs_fp64'] = (torch.linalg.vector_norm(f[:ns].to(torch.complex128) - fsample) /
                                           torch.linalg.vector_norm(fsample)).item()
        del f
        torch.cuda.empty_cache()
        F2 = torch.empty_like(F)
        st.store(F2)
        F2.sub_(F)
        r['round_trip_rel_l2'] = (torch.linalg.vector_norm(F2) / nF).item()
        del F2
        out[name] = r
        del st, plan
        torch.cuda.empty_cache()
    line = {'metric': 'fftSO3R round trip at B=32, omega 24^3 (complex coefficients)', 'unit': 'ms',
            'value': round(out['mixed']['backward_ms'] + out['mixed']['forward_ms'], 2), 'higher_is_better': False,
            'n_gpus': 1, 'dtype': 'f32 (mixed) and f64', 'data': 'synthetic',
            'config': {'workload': 'transform precision stress', 'B': B, 'omega_grid': '24^3',
                       'coefficients': 'i.i.d. N(0,1)/(2l+1), complex', 'beta_engine': args.beta_engine},
            'fp64': out['fp64'], 'mixed': out['mixed'],
            'beta_contraction': {'forward': {'auto': 'tcgen05 tensor cores, 3xTF32 split (B >= 15)',
                                             'tensor': 'tcgen05 tensor cores, 3xTF32 split',
                                             'tensor_bf16': 'tcgen05 tensor cores, BF16x3 split',
                                             'simt': 'CUDA-core FP32 FMAs'}[args.beta_engine],
                                 'backward': 'CUDA cores, fused with the gamma/alpha FFTs'}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def bench_forward(args, rank, local):
    """One forward transform (fftSO3R) of a random FP32 density on a 2-D omega
    grid, B = --B, 2Bx = 2 * --Bx, mixed plan, through the state API
    (hp_state_load_density): the small case the beta-contraction profiles are
    captured on.  Prints one JSON line (not the headline)."""
    import torch
    torch.cuda.set_device(local)
    hp = importlib.import_module('hybridpendulum-up_b200')
    B, Bx = args.B, args.Bx
    plan = hp.Plan(B, Bx, 2, hp.HP_MIXED, hp.HP_REAL)
    plan.set_beta_engine(beta_engine(hp, args))
    if args.tc_form >= 0:
        plan.set_tune(tc_form=args.tc_form)
    g = torch.Generator(device='cuda').manual_seed(11 + rank)
    f = torch.rand((2 * B) ** 3 * (2 * Bx) ** 2, dtype=torch.float32, device='cuda', generator=g)
    st = hp.State(plan)
    for _ in range(max(args.warmup, 1)):
        st.load_density(f.data_ptr())
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        st.load_density(f.data_ptr())
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    plan.profile(True)
    for _ in range(2):
        st.load_density(f.data_ptr())
    torch.cuda.synchronize()
    fam = {k: round(v[0] / v[1], 4) for k, v in plan.profile_read().items()}
    plan.profile(False)
    line = {'metric': f'fftSO3R forward, B={B}, omega {2 * Bx}x{2 * Bx}, FP32 plan', 'value': round(ms, 4),
            'unit': 'ms', 'higher_is_better': False, 'n_gpus': 1, 'steps': args.steps, 'warmup': args.warmup,
            'dtype': 'f32', 'data': 'synthetic (uniform random density)',
            'config': {'workload': 'forward transform', 'B': B, 'omega_grid': f'{2 * Bx}x{2 * Bx}',
                       'beta_engine': args.beta_engine},
            'kernel_ms_per_launch': fam, 'tc_errors': plan.tc_errors(), 'launch_shapes': plan.get_tune()}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def bench_adjoint(args, rank, local):
    """The differentiation workload: gradients of a terminal loss
    <lamT, F_T> with respect to the initial coefficients and the damping,
    gyroscopic, noise and gravity parameters through 50 Euler steps
    (dt = 1e-3) at B=12 on a 24^3 omega grid, FP64 plan, checkpoints every
    10 steps (hp_pendulum_adjoint: forward sweep keeping checkpoints, then
    the reverse sweep recomputing each segment), device-resident.  Timed with
    CUDA events beside the plain 50-step forward propagation it
    differentiates.  Prints one JSON line (not the headline)."""
    import torch
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    hp = importlib.import_module('hybridpendulum-up_b200')
    B, Bx, nsteps, ckpt = 12, 12, 50, 10
    inp = model_inputs(hp, B, Bx, seed=replica_seed(rank))
    L, dt = PARAMS['L'], PARAMS['dt']
    stream = torch.cuda.current_stream(dev)
    plan = hp.Plan(B, Bx, 3, hp.HP_FP64, hp.HP_REAL)
    plan.set_stream(stream.cuda_stream)
    plan.set_model(L, inp['b'], inp['G'], inp['MR'], inp['gyro'])
    f0 = initial_density_dev(torch, inp, B, Bx, L, dev)
    n = int(np.prod(plan.F_shape))
    F0 = torch.zeros(n, dtype=torch.complex128, device=dev)
    plan.forward(f0, out=F0)
    del f0
    g = torch.Generator(device=dev).manual_seed(5 + rank)
    lamT = torch.randn(n, dtype=torch.complex128, device=dev, generator=g)
    st = hp.State(plan)

    def forward_only():
        st.load(F0)
        st.step(dt, 'euler', nsteps)

    def timed(fn, K, W):
        for _ in range(W):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(K):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / K

    K, W = max(1, min(args.steps, 5)), max(args.warmup, 1)
    ms_adj = timed(lambda: plan.adjoint(F0, lamT, nsteps, dt, ckpt), K, W)
    ms_fwd = timed(forward_only, K, W)
    plan.profile(True)
    lam0, grads = plan.adjoint(F0, lamT, nsteps, dt, ckpt)
    torch.cuda.synchronize()
    fam = {k: round(v[0], 2) for k, v in plan.profile_read().items()}   # ms per gradient by kernel family
    plan.profile(False)
    line = {'metric': 'gradient of a terminal loss through 50 Euler steps, B=12, omega 24^3, FP64',
            'value': round(ms_adj, 3), 'unit': 'ms per gradient', 'higher_is_better': False, 'n_gpus': 1,
            'steps': K, 'warmup': W, 'dtype': 'f64', 'data': 'synthetic',
            'config': {'workload': 'adjoint (config 4)', 'B': B, 'omega_grid': '24^3', 'nsteps': nsteps,
                       'checkpoint_every': ckpt, 'gradients': ['F0', 'b', 'G', 'gyro', 'gscale']},
            'forward_50_steps_ms': round(ms_fwd, 3), 'reverse_over_forward': round(ms_adj / ms_fwd, 2),
            'kernel_ms_per_gradient': fam,
            'grad_b': [float(x) for x in grads['b']]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def beta_engine(hp, args):
    return {'auto': hp.HP_BETA_AUTO, 'simt': hp.HP_BETA_SIMT, 'tensor': hp.HP_BETA_TENSOR,
            'tensor_bf16': hp.HP_BETA_TENSOR_BF16}[args.beta_engine]


def bench_hybrid(args, rank, local):
    """The time loop of pendulum_reduced_hybrid.m:224-238 at its own sizes and
    parameters (BR = Bx = 30, L = 3.4, scaled time, wall collision with
    restitution 0.8, nD = 10; pendulum_reduced_hybrid.m:28-128): per step the
    density-gravity propagation (Euler), backward transform, collision update,
    forward transform and the get_stat moments, all on the device.  Prints one
    JSON line (not the headline)."""
    import torch
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    hp = importlib.import_module('hybridpendulum-up_b200')
    B, Bx, L = 30, 30, 3.4
    J, rho, mass, g = 0.01436, 0.1, 1.0642, 9.8
    tscale = math.sqrt(J / (mass * g * rho))
    dt = 1 / 400 / tscale
    coll = dict(d=0.12, h=0.2, r=0.025, theta_t=5 * math.pi / 180, lambda_max=100 * tscale, epsilon=0.8)
    Gd = (0.05 * np.eye(2)) @ (0.05 * np.eye(2)).T
    b = np.array([0.2, 0.2]) * tscale
    Ht = np.eye(2) * tscale ** 1.5
    G = 0.5 * Ht @ Ht.T
    R = rotation_grid(B)
    mR = np.stack([R[..., 2, 1], -R[..., 2, 0]])                      # [R32; -R31] (pendulum_reduced_hybrid.m:118)
    th = -2 * math.pi / 3
    U = np.array([[math.cos(th), 0, math.sin(th)], [0, 1, 0], [-math.sin(th), 0, math.cos(th)]])
    Sigma = (2 * tscale) ** 2 * np.eye(2)
    out = {}
    for name, prec in (('mixed', hp.HP_MIXED), ('fp64', hp.HP_FP64)):
        plan = hp.Plan(B, Bx, 2, prec, hp.HP_REAL)
        plan.set_beta_engine(beta_engine(hp, args))
        plan.set_den_model(L, b, G, mR)
        t0 = time.perf_counter()
        c = hp.Collision(plan, L=L, Gd=Gd, nD=10, **coll)
        torch.cuda.synchronize(dev)
        t_tables = time.perf_counter() - t0
        st = hp.State(plan)
        st.init_mf_gauss(U, (15.0, 15.0, 15.0), np.eye(3), np.zeros(2), Sigma)
        for _ in range(args.warmup):
            st.hybrid_step(c, dt, 'euler', 1)
            st.moments()
        torch.cuda.synchronize(dev)
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        for _ in range(args.steps):
            st.hybrid_step(c, dt, 'euler', 1)
        e1.record()
        torch.cuda.synchronize(dev)
        tm = time.perf_counter()
        for _ in range(args.steps):
            st.moments()
        t_mom = (time.perf_counter() - tm) / args.steps
        ms = e0.elapsed_time(e1) / args.steps
        plan.profile(True)
        for _ in range(2):
            st.hybrid_step(c, dt, 'euler', 1)
        torch.cuda.synchronize(dev)
        fam = {k: round(v[0] / 2, 3) for k, v in plan.profile_read().items()}
        plan.profile(False)
        mo = st.moments()
        out[name] = {'ms_per_step': round(ms, 3), 'steps_per_s': round(1000.0 / (ms + 1000 * t_mom), 3),
                     'moments_ms': round(1000 * t_mom, 3), 'colliding_attitudes': c.numR,
                     'tables_s': round(t_tables, 2), 'mass': mo['mass'], 'ER': mo['ER'].tolist(),
                     'kernel_ms_per_step': fam}
        del st, c, plan
        torch.cuda.empty_cache()
    er = np.array(out['mixed']['ER']) - np.array(out['fp64']['ER'])
    line = {'metric': 'hybrid FP steps/s, pendulum_reduced_hybrid sizes (B=30, omega 60x60)',
            'value': out['mixed']['steps_per_s'], 'unit': 'steps/s', 'higher_is_better': True, 'n_gpus': 1,
            'steps': args.steps, 'warmup': args.warmup, 'dtype': 'f32 (f64 accumulation)', 'data': 'synthetic',
            'config': {'workload': 'hybrid loop body incl. get_stat moments', 'B': B, 'omega_grid': '60x60',
                       'dt': dt, 'method': 'euler', 'beta_engine': args.beta_engine},
            'mixed': out['mixed'], 'fp64': out['fp64'],
            'ER_max_abs_diff_mixed_vs_fp64': float(np.abs(er).max())}
    for k in ('mixed', 'fp64'):
        line[k].pop('ER')
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def cpu_sample_loop(args, B, Bx):
    """--impl reference: the FP64 oracle port on the host cores, each step a
    bounded sample of the workload (omega 8^3), reported per full-size step."""
    workers = os.cpu_count() or 1
    Bs = 4
    for _ in range(max(args.warmup, 0)):
        cpu_sample(B, Bs, 1, workers)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cpu_sample(B, Bs, 1, workers)
    sec = (time.perf_counter() - t0) / max(args.steps, 1)
    scale = (Bx / Bs) ** 3
    val = 1.0 / (sec * scale)
    return {'metric': METRIC, 'impl': 'reference', 'value': val, 'unit': 'steps/s', 'n_gpus': args.gpus,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': sec * scale * 1e3,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
            'data': 'synthetic',
            'config': {'workload': f'pendulum FP step: Euler propagate + density synthesis, B={B}, '
                                   f'omega {2 * Bx}^3, dt={PARAMS["dt"]}'},
            'cpu_baseline': {'value': val, 'unit': 'steps/s', 'cores': workers, 'kind': 'port',
                             'sample': f'FP64 numpy oracle, B={B}, omega {2 * Bs}^3 per step, scaled by '
                                       f'omega points x{scale:.0f}'},
            'e2e': {'value': val, 'unit': 'steps/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}


if __name__ == '__main__':
    sys.exit(main())
