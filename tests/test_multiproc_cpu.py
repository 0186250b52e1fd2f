"""Multi-process replicas on CPU (gloo, world size 2): the propagation step does
not shard, so bench.py --gpus N runs N independent replicas.  Checks the host
logic of that path: per-rank seeds give different densities, each rank steps
its own replica (oracle step on CPU), the job time is the max over ranks and
the whole-job rate counts every rank's steps."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    import time
    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world)
    import bench
    from oracle import pendulum as pd
    from oracle import so3
    P = pd.pendulum_3d(3, 2)
    f, meta = pd.seeded_density(3, 2, 3, P.L, seed=bench.replica_seed(rank))
    F = so3.fftSO3R_forward(f)
    t0 = time.perf_counter()
    steps = 2
    for _ in range(steps):
        F = pd.integrate(F, lambda G: pd.derivative_fast(G, P), 1e-3, 'euler')
    ms = (time.perf_counter() - t0) * 1e3 * (1 + rank)       # rank 1 reports the slower time
    mx = bench.max_over_ranks(ms, world)
    rate = bench.whole_job_rate(world, steps, mx)
    mass = float(F[2, 2, 0, 0, 0, 0].real)
    allm = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(allm, torch.tensor([mass], dtype=torch.float64))
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, ms, mx, rate, [float(a.item()) for a in allm], meta['mu'].tolist()))


def test_two_rank_replicas():
    import multiprocessing as mp
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    (_, ms0, mx0, r0, m0, mu0), (_, ms1, mx1, r1, m1, mu1) = res
    assert mx0 == mx1 == pytest.approx(max(ms0, ms1))
    assert r0 == r1 == pytest.approx(2 * 2 / (max(ms0, ms1) / 1e3))
    assert mu0 != mu1                       # independent replicas
    assert m0 == m1 and len(m0) == 2         # gathered masses agree across ranks
