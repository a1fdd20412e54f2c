"""Calibration of a shared zonal Manning n field over a batched ensemble.

Every scenario's elements are assigned to one of nzx x nzy zones by their centroid in the
scenario's normalised domain coordinates; one n value per zone is shared by all
scenarios.  The objective is the ensemble's gauge misfit (GaugeMisfit on an Ensemble, J
summed over the scenarios); torch.optim.LBFGS minimises it over theta = log n (so n stays
positive), with gradients from the discrete adjoint through the torch.autograd.Function
(adjoint.gauge_misfit): the per-element gradient is gathered to the zones by autograd's
transpose of the zone lookup.
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
    """J(n_zone) of an ensemble misfit from a fixed initial state, and its L-BFGS fit."""

    def __init__(self, misfit: GaugeMisfit, state, zones: np.ndarray, nzones: int):
        import torch

        self.torch = torch
        self.misfit = misfit
        self.state = state
        self.zones = torch.as_tensor(np.ascontiguousarray(zones, dtype=np.int64))
        assert self.zones.shape == (misfit.ne,)
        self.nzones = int(nzones)
        self.evals = 0
        self.fwd_ms = 0.0
        self.bwd_ms = 0.0

    def n_elements(self, n_zone) -> np.ndarray:
        return np.asarray(n_zone, dtype=np.float64)[self.zones.numpy()]

    def objective(self, theta):
        """torch scalar J(exp(theta)) differentiable with respect to theta [nzones]"""
        n_el = self.torch.exp(theta)[self.zones]
        return gauge_misfit(n_el, None, self.misfit, self.state)

    def set_target_from(self, n_zone_true) -> np.ndarray:
        """records the gauge series of the field n_zone_true as the target; returns it"""
        self.misfit.solver.set_element_manning(self.n_elements(n_zone_true))
        _, vals = self.misfit.forward(self.state)
        self.misfit.set_target(vals)
        return vals

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
            f, b, _ = self.misfit.timing()
            self.evals += 1
            self.fwd_ms += f
            self.bwd_ms += b
            if history is not None:
                history.append((float(J.detach()), np.exp(theta.detach().numpy()).copy()))
            return J

        t0 = time.perf_counter()
        opt.step(closure)
        self.wall_s = time.perf_counter() - t0
        self.iterations = int(opt.state[opt._params[0]]["n_iter"])
        return np.exp(theta.detach().numpy())


def relative_error(n_zone, n_zone_true) -> float:
    a, b = np.asarray(n_zone, dtype=np.float64), np.asarray(n_zone_true, dtype=np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def ensemble_workload(nscen: int = 64, lo: float = 20000, hi: float = 150000, seed: int = 5, ngauges: int = 32,
                      amp: float = 1.0):
    """The batched calibration workload: nscen submerged basins (10 km x 5 km, datum 7 m,
    tide on the x = 0 side) of log-uniform element counts in [lo, hi], each with a 1 m
    Gaussian hump as its initial elevation (projected onto the p = 2 basis) and ngauges
    gauges uniform over its domain; the generating 16-zone n field U(0.02, 0.06).
    Returns (meshes, scenario params, states, [(gauge elements, weights)], zones, n_true)."""
    from . import p2
    from .mesh import rectangle_with_elements

    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(lo), np.log(hi), nscen))
    meshes = [rectangle_with_elements(float(c), seed=seed * 1000 + k, datum=7.0) for k, c in enumerate(counts)]
    params = [dict(tide_on=1, tide_amp=0.5, tide_period=44712.0, rain=0.0, n_el=None) for _ in meshes]
    states, gauges, zones = [], [], []
    for m in meshes:
        x0, x1, y0, y1 = m.x.min(), m.x.max(), m.y.min(), m.y.max()
        cx, cy = rng.uniform(x0 + 0.2 * (x1 - x0), x1 - 0.2 * (x1 - x0)), rng.uniform(y0 + 0.2 * (y1 - y0),
                                                                                    y1 - 0.2 * (y1 - y0))
        wid = 0.08 * (x1 - x0)
        hump = lambda x, y: amp * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * wid * wid))  # noqa: E731
        z = np.zeros(p2.NM * m.num_el)
        states.append((p2.project(m, hump), z, z.copy(), np.zeros(m.num_el, dtype=np.int32)))
        pts = list(zip(rng.uniform(x0 + 0.02 * (x1 - x0), x1 - 0.02 * (x1 - x0), ngauges),
                       rng.uniform(y0 + 0.02 * (y1 - y0), y1 - 0.02 * (y1 - y0), ngauges)))
        gauges.append(p2.gauge_weights(m, pts))
        zones.append(zone_index(m))
    n_true = rng.uniform(0.02, 0.06, 16)
    return meshes, params, states, gauges, zones, n_true


def setup(ensemble, states, gauges, zones, nsteps: int, ckpt_every: int) -> ZonalCalibration:
    """GaugeMisfit over the whole ensemble (flattened gauges) and its ZonalCalibration"""
    el = np.concatenate([g[0] + ensemble.el_off[k] for k, g in enumerate(gauges)]).astype(np.int32)
    w = np.concatenate([g[1] for g in gauges])
    mis = GaugeMisfit(ensemble, nsteps, ckpt_every, el, w)
    return ZonalCalibration(mis, ensemble.flatten_states(states), np.concatenate(zones), 16)


def main(argv=None):
    """python -m dgrain.calibration: the batched p = 2 SSP(3,3) calibration; prints one JSON
    line (recovered-n error, objective, adjoint-to-forward time ratio, device times)."""
    import argparse
    import json

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
    t0 = time.perf_counter()
    meshes, params, states, gauges, zones, n_true = ensemble_workload(a.scenarios, a.lo, a.hi, a.seed)
    t_mesh = time.perf_counter() - t0
    with Ensemble(meshes, params, order=2, wet_dry=0, cfl=0.1, rk_stages=3) as e:
        cal = setup(e, states, gauges, zones, a.steps, a.ckpt)
        cal.set_target_from(n_true)
        f_target, _, _ = cal.misfit.timing()
        n0 = np.full(16, 0.04)
        hist: list = []
        n_fit = cal.fit(n0, a.iterations, hist)
        out = {"workload": f"{a.scenarios} p=2 SSP(3,3) basins, {e.ne} elements (log-uniform [{a.lo:g}, {a.hi:g}]), "
                           f"{a.steps} steps, checkpoint every {a.ckpt}, {len(gauges[0][0])} gauges each, "
                           "16-zone n, torch L-BFGS",
               "elements": e.ne, "iterations": cal.iterations, "evaluations": cal.evals,
               "n_error_initial": relative_error(n0, n_true), "n_error": relative_error(n_fit, n_true),
               "J_initial": hist[0][0], "J_final": hist[-1][0],
               "forward_ms_per_eval": cal.fwd_ms / cal.evals, "backward_ms_per_eval": cal.bwd_ms / cal.evals,
               "adjoint_to_forward": cal.bwd_ms / cal.fwd_ms, "target_forward_ms": f_target,
               "wall_s": cal.wall_s, "mesh_s": t_mesh,
               "n_true": [round(float(v), 5) for v in n_true], "n_fit": [round(float(v), 5) for v in n_fit]}
    print(json.dumps(out))
    return out


if __name__ == "__main__":
    main()
