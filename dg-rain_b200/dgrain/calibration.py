"""Calibration of a shared zonal Manning n field over a batched ensemble.

Every scenario's elements are assigned to one of nzx x nzy zones by their centroid in the
scenario's normalised domain coordinates; one n value per zone is shared by all
scenarios.  The objective is the ensemble's gauge misfit (GaugeMisfit on an Ensemble, J
summed over the scenarios); torch.optim.LBFGS minimises it over theta = log n (so n stays
positive), with gradients from the discrete adjoint through the torch.autograd.Function
(adjoint.gauge_misfit): the per-element gradient is gathered to the zones by autograd's
transpose of the zone lookup.

Across GPUs the scenarios are independent units: each rank owns a share of them
(partition, balanced by element count) in its own Ensemble, and every evaluation sums J
and the 16 zone-gradient values over the ranks with one all-reduce, so every rank takes the
same L-BFGS steps.  Nothing else is exchanged.
"""
from __future__ import annotations

import time

import numpy as np

from .adjoint import GaugeMisfit, gauge_misfit
from .mesh import Mesh


def zone_index(mesh: Mesh, nzx: int = 4, nzy: int = 4) -> np.ndarray:
    """zone [num_el] of every element: the nzx x nzy tiling of the normalised domain
    coordinates of its centroid, row-major in y"""
    v = mesh.el2v
    cx = mesh.x[v].mean(axis=1)
    cy = mesh.y[v].mean(axis=1)
    u = (cx - mesh.x.min()) / (mesh.x.max() - mesh.x.min())
    w = (cy - mesh.y.min()) / (mesh.y.max() - mesh.y.min())
    ix = np.clip((u * nzx).astype(np.int64), 0, nzx - 1)
    iy = np.clip((w * nzy).astype(np.int64), 0, nzy - 1)
    return iy * nzx + ix


class ZonalCalibration:
    """J(n_zone) of an ensemble misfit from a fixed initial state, and its L-BFGS fit.

    group: a torch.distributed process group (or None) whose ranks hold the other
    scenarios; objective_fn(n_el) -> torch scalar replaces the gauge misfit (tests)."""

    def __init__(self, misfit: GaugeMisfit | None, state, zones: np.ndarray, nzones: int, group=None,
                 objective_fn=None):
        import torch

        self.torch = torch
        self.misfit = misfit
        self.state = state
        self.zones = torch.as_tensor(np.ascontiguousarray(zones, dtype=np.int64))
        if misfit is not None:
            assert self.zones.shape == (misfit.ne,)
        self.nzones = int(nzones)
        self.group = group
        self.objective_fn = objective_fn
        self.evals = 0
        self.fwd_ms = 0.0
        self.bwd_ms = 0.0

    def n_elements(self, n_zone) -> np.ndarray:
        return np.asarray(n_zone, dtype=np.float64)[self.zones.numpy()]

    def objective(self, theta):
        """torch scalar J(exp(theta)) of this rank's scenarios, differentiable with respect
        to theta [nzones]"""
        n_el = self.torch.exp(theta)[self.zones]
        if self.objective_fn is not None:
            return self.objective_fn(n_el)
        return gauge_misfit(n_el, None, self.misfit, self.state)

    def set_target_from(self, n_zone_true) -> np.ndarray:
        """records the gauge series of the field n_zone_true as the target; returns it"""
        self.misfit.solver.set_element_manning(self.n_elements(n_zone_true))
        _, vals = self.misfit.forward(self.state)
        self.misfit.set_target(vals)
        return vals

    def _sum_over_ranks(self, J, grad):
        """J and the zone gradient summed over the group's ranks (one all-reduce)"""
        torch = self.torch
        import torch.distributed as dist

        buf = torch.cat([J.detach().reshape(1), grad]).to(torch.float64)
        dev = None
        if dist.get_backend(self.group) == "nccl":
            dev = torch.device("cuda", torch.cuda.current_device())
            buf = buf.to(dev)
        dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=self.group)
        buf = buf.cpu()
        return buf[0], buf[1:].clone()

    def fit(self, n_zone0, iterations: int = 20, history: list | None = None):
        """L-BFGS (strong Wolfe line search) over log n from n_zone0; returns the fitted
        zone values.  history, when given, receives (J, n_zone) at every evaluation."""
        torch = self.torch
        theta = torch.tensor(np.log(np.asarray(n_zone0, dtype=np.float64)), dtype=torch.float64, requires_grad=True)
        opt = torch.optim.LBFGS([theta], lr=1.0, max_iter=iterations, max_eval=int(iterations * 1.5) + 1,
                                tolerance_grad=0.0, tolerance_change=0.0, history_size=20,
                                line_search_fn="strong_wolfe")

        def closure():
            opt.zero_grad()
            J = self.objective(theta)
            J.backward()
            if self.group is not None:
                Jt, gt = self._sum_over_ranks(J, theta.grad)
                theta.grad.copy_(gt)
                J = Jt
            if self.misfit is not None:
                f, b, _ = self.misfit.timing()
                self.fwd_ms += f
                self.bwd_ms += b
            self.evals += 1
            if history is not None:
                history.append((float(J.detach()), np.exp(theta.detach().numpy()).copy()))
            return J.detach()

        t0 = time.perf_counter()
        opt.step(closure)
        self.wall_s = time.perf_counter() - t0
        self.iterations = int(opt.state[opt._params[0]]["n_iter"])
        return np.exp(theta.detach().numpy())


def partition(counts, world: int) -> list:
    """scenario indices of each rank: largest first to the least loaded rank (ties to the
    lower rank), each rank's share in ascending scenario order"""
    load = [0.0] * world
    share: list = [[] for _ in range(world)]
    for k in sorted(range(len(counts)), key=lambda i: (-counts[i], i)):
        r = min(range(world), key=lambda j: (load[j], j))
        share[r].append(k)
        load[r] += counts[k]
    return [sorted(s) for s in share]


def relative_error(n_zone, n_zone_true) -> float:
    a, b = np.asarray(n_zone, dtype=np.float64), np.asarray(n_zone_true, dtype=np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _workload_draws(nscen, lo, hi, seed, ngauges):
    """the workload's random draws, in their fixed order: element counts, then per basin the
    hump centre and the gauge points (the basins' extents follow from their cell counts),
    then the generating zone field"""
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(lo), np.log(hi), nscen))
    per = []
    for c in counts:
        nx = max(2, int(round(np.sqrt(float(c)))))
        ny = max(1, nx // 2)
        x0, y0 = 0.0, 0.0
        x1 = float(np.float64(nx) * (10000.0 / nx))  # the generator's largest x (cell * count)
        y1 = float(np.float64(ny) * (5000.0 / ny))
        cx = rng.uniform(x0 + 0.2 * (x1 - x0), x1 - 0.2 * (x1 - x0))
        cy = rng.uniform(y0 + 0.2 * (y1 - y0), y1 - 0.2 * (y1 - y0))
        px = rng.uniform(x0 + 0.02 * (x1 - x0), x1 - 0.02 * (x1 - x0), ngauges)
        py = rng.uniform(y0 + 0.02 * (y1 - y0), y1 - 0.02 * (y1 - y0), ngauges)
        per.append((cx, cy, 0.08 * (x1 - x0), px, py))
    n_true = rng.uniform(0.02, 0.06, 16)
    return counts, per, n_true


def workload_counts(nscen: int = 64, lo: float = 20000, hi: float = 150000, seed: int = 5) -> np.ndarray:
    """element-count targets of the workload's basins (for partitioning)"""
    return _workload_draws(nscen, lo, hi, seed, 1)[0]


def ensemble_workload(nscen: int = 64, lo: float = 20000, hi: float = 150000, seed: int = 5, ngauges: int = 32,
                      amp: float = 1.0, subset=None):
    """The batched calibration workload: nscen submerged basins (10 km x 5 km, datum 7 m,
    tide on the x = 0 side) of log-uniform element counts in [lo, hi], each with a 1 m
    Gaussian hump as its initial elevation (projected onto the p = 2 basis) and ngauges
    gauges uniform over its domain; the generating 16-zone n field U(0.02, 0.06).
    subset: the basins to build (default all), e.g. one rank's share.
    Returns (meshes, scenario params, states, [(gauge elements, weights)], zones, n_true)."""
    from . import p2
    from .mesh import rectangle_with_elements

    counts, per, n_true = _workload_draws(nscen, lo, hi, seed, ngauges)
    idx = range(nscen) if subset is None else subset
    meshes, params, states, gauges, zones = [], [], [], [], []
    for k in idx:
        m = rectangle_with_elements(float(counts[k]), seed=seed * 1000 + k, datum=7.0)
        cx, cy, wid, px, py = per[k]
        hump = lambda x, y: amp * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * wid * wid))  # noqa: E731
        z = np.zeros(p2.NM * m.num_el)
        meshes.append(m)
        params.append(dict(tide_on=1, tide_amp=0.5, tide_period=44712.0, rain=0.0, n_el=None))
        states.append((p2.project(m, hump), z, z.copy(), np.zeros(m.num_el, dtype=np.int32)))
        gauges.append(p2.gauge_weights(m, list(zip(px, py))))
        zones.append(zone_index(m))
    return meshes, params, states, gauges, zones, n_true


def setup(ensemble, states, gauges, zones, nsteps: int, ckpt_every: int, group=None) -> ZonalCalibration:
    """GaugeMisfit over the whole ensemble (flattened gauges) and its ZonalCalibration"""
    el = np.concatenate([g[0] + ensemble.el_off[k] for k, g in enumerate(gauges)]).astype(np.int32)
    w = np.concatenate([g[1] for g in gauges])
    mis = GaugeMisfit(ensemble, nsteps, ckpt_every, el, w)
    return ZonalCalibration(mis, ensemble.flatten_states(states), np.concatenate(zones), 16, group=group)


def main(argv=None):
    """python -m dgrain.calibration: the batched p = 2 SSP(3,3) calibration; prints one JSON
    line (recovered-n error, objective, adjoint-to-forward time ratio, device times).
    Under torchrun each rank (one GPU) owns a share of the scenarios (partition) and the
    ranks sum J and the zone gradient with NCCL."""
    import argparse
    import datetime
    import json
    import os

    import torch

    from .solver import Ensemble

    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--scenarios", type=int, default=64)
    ap.add_argument("--lo", type=float, default=20000)
    ap.add_argument("--hi", type=float, default=150000)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--ckpt", type=int, default=50)
    ap.add_argument("--iterations", type=int, default=20)
    ap.add_argument("--seed", type=int, default=5)
    a = ap.parse_args(argv)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    group = None
    if world > 1:
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
        group = dist.group.WORLD
    share = partition(workload_counts(a.scenarios, a.lo, a.hi, a.seed), world)[rank]
    t0 = time.perf_counter()
    meshes, params, states, gauges, zones, n_true = ensemble_workload(a.scenarios, a.lo, a.hi, a.seed, subset=share)
    t_mesh = time.perf_counter() - t0
    with Ensemble(meshes, params, order=2, wet_dry=0, cfl=0.1, rk_stages=3, device=local) as e:
        cal = setup(e, states, gauges, zones, a.steps, a.ckpt, group=group)
        cal.set_target_from(n_true)
        f_target, _, _ = cal.misfit.timing()
        n0 = np.full(16, 0.04)
        hist: list = []
        n_fit = cal.fit(n0, a.iterations, hist)
        stats = np.array([cal.fwd_ms, cal.bwd_ms, float(e.ne)])
        if group is not None:
            import torch.distributed as dist

            t = torch.tensor(stats[:2], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
            n = torch.tensor(stats[2:], dtype=torch.float64, device="cuda")
            dist.all_reduce(n, op=dist.ReduceOp.SUM, group=group)
            stats = np.concatenate([t.cpu().numpy(), n.cpu().numpy()])
        out = {"workload": f"{a.scenarios} p=2 SSP(3,3) basins, {int(stats[2])} elements "
                           f"(log-uniform [{a.lo:g}, {a.hi:g}]), {a.steps} steps, checkpoint every {a.ckpt}, "
                           f"{len(gauges[0][0])} gauges each, 16-zone n, torch L-BFGS",
               "ranks": world, "elements": int(stats[2]), "iterations": cal.iterations, "evaluations": cal.evals,
               "n_error_initial": relative_error(n0, n_true), "n_error": relative_error(n_fit, n_true),
               "J_initial": hist[0][0], "J_final": hist[-1][0],
               "forward_ms_per_eval": stats[0] / cal.evals, "backward_ms_per_eval": stats[1] / cal.evals,
               "adjoint_to_forward": stats[1] / stats[0], "target_forward_ms": f_target,
               "wall_s": cal.wall_s, "mesh_s": t_mesh,
               "n_true": [round(float(v), 5) for v in n_true], "n_fit": [round(float(v), 5) for v in n_fit]}
    if group is not None:
        import torch.distributed as dist

        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))
    return out


if __name__ == "__main__":
    main()
