"""The rank-sharded calibration on CPU (two gloo ranks, no GPU): a quadratic stand-in for
the gauge misfit whose elements are split between the ranks; the ranks' summed J and zone
gradient drive identical L-BFGS steps on both ranks and reach the single-process fit of
the union; the scenario partition is balanced and covers every scenario once."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest


def _problem(seed=3, ne=400):
    rng = np.random.default_rng(seed)
    zones = rng.integers(0, 16, ne)
    target = rng.uniform(0.02, 0.06, 16)[zones] * np.exp(rng.normal(0, 0.05, ne))
    wts = rng.uniform(0.5, 2.0, ne)
    return zones, target, wts


def _objective(torch, target, wts):
    t = torch.as_tensor(target)
    w = torch.as_tensor(wts)

    def f(n_el):
        return (w * (n_el - t) ** 2).sum() * 1e3
    return f


def _fit(rank, world, port, out):
    import torch
    import torch.distributed as dist

    from dgrain.calibration import ZonalCalibration

    zones, target, wts = _problem()
    group = None
    sel = np.arange(len(zones))
    if world > 1:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world)
        group = dist.group.WORLD
        sel = np.arange(rank, len(zones), world)  # this rank's share of the elements
    cal = ZonalCalibration(None, None, zones[sel], 16, group=group,
                           objective_fn=_objective(torch, target[sel], wts[sel]))
    n = cal.fit(np.full(16, 0.04), 15)
    out.put((rank, n.tolist(), cal.evals))
    if world > 1:
        dist.destroy_process_group()


def test_sharded_fit_equals_single_process():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    _fit(0, 1, 0, q)
    _, single, _ = q.get()
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = [ctx.Process(target=_fit, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, n0, e0), (_, n1, e1) = res
    assert n0 == n1 and e0 == e1  # identical steps on both ranks
    np.testing.assert_allclose(n0, single, rtol=1e-7)
    _, target, _ = _problem()
    assert np.all(np.isfinite(n0))


def test_partition_is_balanced():
    from dgrain.calibration import partition, workload_counts

    counts = workload_counts(64)
    for world in (1, 2, 3, 8):
        shares = partition(counts, world)
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(64))
        loads = [counts[s].sum() for s in shares]
        assert max(loads) - min(loads) <= counts.max()
