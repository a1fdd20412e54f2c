"""Gauge-misfit objectives of the device time loop and their derivatives: discrete adjoint
(gradients with respect to per-element Manning n, node depth and the initial state),
tangent-linear directional derivatives, and a torch.autograd.Function over them.

The objective of a run of nsteps steps from a given state is
    J = sum_n sum_g (zeta_g(u^{n+1}) - target[n, g])^2,
zeta_g the elevation at gauge g's point: the Crouzeix-Raviart interpolation of the midpoint
values at p = 1 (place_gauges), the modal expansion at p = 2 (p2.gauge_weights).  On an
Ensemble the state, gauges and gradients use the flattened numbering (Ensemble.el_off /
nd_off) and J sums over the scenarios.  Derivatives
are those of the discrete scheme with its decisions and dt sequence frozen at the recorded
forward run (the C ABI's dgr_adjoint_* / dgr_tlm); finite differences that should agree
with them use the same dt sequence (forward(..., replay_dt=True)).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .mesh import Mesh, _dp, _ip
from .solver import Solver


def barycentric(mesh: Mesh, px: float, py: float):
    """(element, barycentric coordinates) of the element containing the point, or (-1, None)."""
    v = mesh.el2v
    x0, y0 = mesh.x[v[:, 0]], mesh.y[v[:, 0]]
    x1, y1 = mesh.x[v[:, 1]], mesh.y[v[:, 1]]
    x2, y2 = mesh.x[v[:, 2]], mesh.y[v[:, 2]]
    det = (y1 - y2) * (x0 - x2) + (x2 - x1) * (y0 - y2)
    l0 = ((y1 - y2) * (px - x2) + (x2 - x1) * (py - y2)) / det
    l1 = ((y2 - y0) * (px - x2) + (x0 - x2) * (py - y2)) / det
    l2 = 1.0 - l0 - l1
    inside = np.nonzero((l0 >= -1e-12) & (l1 >= -1e-12) & (l2 >= -1e-12))[0]
    if inside.size == 0:
        return -1, None
    e = int(inside[0])
    return e, np.array([l0[e], l1[e], l2[e]])


def cr_weights(lam: np.ndarray) -> np.ndarray:
    """Crouzeix-Raviart basis at a point with barycentric coordinates lam: midpoint k lies on
    the edge (v_k, v_{k+1}), psi_k = 1 - 2 lam_{k+2}."""
    return np.array([1.0 - 2.0 * lam[2], 1.0 - 2.0 * lam[0], 1.0 - 2.0 * lam[1]])


def place_gauges(mesh: Mesh, points) -> tuple[np.ndarray, np.ndarray]:
    """Elements and Crouzeix-Raviart weights [ng, 3] of gauge points [(x, y), ...]."""
    els, ws = [], []
    for px, py in points:
        e, lam = barycentric(mesh, px, py)
        if e < 0:
            raise ValueError(f"gauge ({px}, {py}) lies outside the mesh")
        els.append(e)
        ws.append(cr_weights(lam))
    return np.asarray(els, dtype=np.int32), np.ascontiguousarray(np.asarray(ws, dtype=np.float64))


def intertidal_points(mesh: Mesh, n: int, amp: float, seed: int, max_tries: int = 200000):
    """n points uniform over the part of the domain whose bed elevation (-z, linear over each
    element) lies in [-amp, amp]; rejection sampling from a seeded generator."""
    rng = np.random.default_rng(seed)
    lo = np.array([mesh.x.min(), mesh.y.min()])
    hi = np.array([mesh.x.max(), mesh.y.max()])
    pts = []
    for _ in range(max_tries):
        p = rng.uniform(lo, hi)
        e, lam = barycentric(mesh, p[0], p[1])
        if e < 0:
            continue
        elev = -float(lam @ mesh.z[mesh.el2v[e]])
        if -amp <= elev <= amp:
            pts.append((float(p[0]), float(p[1])))
            if len(pts) == n:
                return pts
    raise ValueError("no intertidal zone found for the gauges")


class GaugeMisfit:
    """J and its derivatives for one Solver or Ensemble over nsteps steps, with a checkpoint
    every ckpt_every steps."""

    def __init__(self, solver, nsteps: int, ckpt_every: int, gauge_el, gauge_w, target=None):
        self.solver = solver
        self.lib = solver.lib
        self.nsteps = int(nsteps)
        self.nm = solver.nm
        self.ne = solver.ne
        self.nn = solver.mesh.num_nodes if isinstance(solver, Solver) else solver.nn
        self.el = np.ascontiguousarray(gauge_el, dtype=np.int32)
        self.w = np.ascontiguousarray(gauge_w, dtype=np.float64).reshape(-1, self.nm)
        self.ng = int(self.el.shape[0])
        tgt = None if target is None else self._target(target)
        _lib.check(self.lib.dgr_adjoint_setup(solver.ctx, self.nsteps, int(ckpt_every), self.ng, _ip(self.el),
                                              _dp(self.w), None if tgt is None else _dp(tgt)), "dgr_adjoint_setup")
        self.state = None

    def _target(self, target) -> np.ndarray:
        t = np.ascontiguousarray(target, dtype=np.float64).reshape(-1)
        assert t.shape == (self.nsteps * self.ng,)
        return t

    def set_target(self, target) -> None:
        t = self._target(target)
        _lib.check(self.lib.dgr_adjoint_set_target(self.solver.ctx, _dp(t)), "dgr_adjoint_set_target")

    def _state(self, state):
        z, x, y = (np.ascontiguousarray(a, dtype=np.float64) for a in state[:3])
        assert z.shape == x.shape == y.shape == (self.nm * self.ne,)
        wd = np.ascontiguousarray(state[3] if len(state) > 3 else np.full(self.ne, -1), dtype=np.int32)
        return z, x, y, wd

    def forward(self, state, time: float = -1.0, dt: float = 0.0, replay_dt: bool = False):
        """Runs nsteps steps from state = (zeta, Qx, Qy[, WD]); returns (J, gauge values
        [nsteps, ng])."""
        z, x, y, wd = self._state(state)
        self.state = (z, x, y, wd)
        J = C.c_double()
        vals = np.empty(self.nsteps * self.ng)
        self.solver._status(self.lib.dgr_adjoint_forward(self.solver.ctx, _dp(z), _dp(x), _dp(y), _ip(wd), time, dt,
                                                         int(replay_dt), C.byref(J), _dp(vals)), "dgr_adjoint_forward")
        return J.value, vals.reshape(self.nsteps, self.ng)

    def backward(self) -> dict:
        """Gradient of the last forward run's J."""
        ne, nn, nm = self.ne, self.nn, self.nm
        g = {"n_el": np.empty(ne), "z": np.empty(nn), "zeta0": np.empty(nm * ne), "qx0": np.empty(nm * ne),
             "qy0": np.empty(nm * ne)}
        self.solver._status(self.lib.dgr_adjoint_backward(self.solver.ctx, _dp(g["n_el"]), _dp(g["z"]),
                                                          _dp(g["zeta0"]), _dp(g["qx0"]), _dp(g["qy0"])),
                            "dgr_adjoint_backward")
        return g

    def tlm(self, state, dn_el=None, dz=None, dstate=None):
        """(J, dJ) along the direction (dn_el, dz, dstate) with the recorded dt sequence."""
        z, x, y, wd = self._state(state)
        opt = lambda a: None if a is None else _dp(np.ascontiguousarray(a, dtype=np.float64))  # noqa: E731
        keep = [None if a is None else np.ascontiguousarray(a, dtype=np.float64)
                for a in ((dstate or (None, None, None))[:3] + (dn_el, dz))]
        J, dJ = C.c_double(), C.c_double()
        self.solver._status(self.lib.dgr_tlm(self.solver.ctx, _dp(z), _dp(x), _dp(y), _ip(wd), *[opt(a) for a in keep],
                                             C.byref(J), C.byref(dJ)), "dgr_tlm")
        return J.value, dJ.value

    def frozen(self, state, n_el=None, z=None, state_p=None):
        """(J, J_p): J at the recorded point and J_p at the perturbed point (n_el, z, state_p;
        None = unperturbed) with the recorded run's decisions and dt sequence frozen."""
        zz, x, y, wd = self._state(state)
        opt = lambda a: None if a is None else _dp(np.ascontiguousarray(a, dtype=np.float64))  # noqa: E731
        keep = [None if a is None else np.ascontiguousarray(a, dtype=np.float64)
                for a in ((state_p or (None, None, None))[:3] + (n_el, z))]
        J, Jp = C.c_double(), C.c_double()
        self.solver._status(self.lib.dgr_fd_frozen(self.solver.ctx, _dp(zz), _dp(x), _dp(y), _ip(wd),
                                                   *[opt(a) for a in keep], C.byref(J), C.byref(Jp)),
                            "dgr_fd_frozen")
        return J.value, Jp.value

    def dt_history(self):
        """recorded dt and boundary time per step ([nsteps], or [nsteps, scenarios] for an
        Ensemble)"""
        nsc = getattr(self.solver, "n", 1) if not isinstance(self.solver, Solver) else 1
        dt = np.empty(self.nsteps * nsc)
        t = np.empty(self.nsteps * nsc)
        _lib.check(self.lib.dgr_adjoint_dt(self.solver.ctx, _dp(dt), _dp(t)), "dgr_adjoint_dt")
        if nsc == 1:
            return dt, t
        return dt.reshape(self.nsteps, nsc), t.reshape(self.nsteps, nsc)

    def timing(self):
        """device ms of the last forward, backward and tangent-linear runs"""
        f, b, t = C.c_double(), C.c_double(), C.c_double()
        _lib.check(self.lib.dgr_adjoint_timing(self.solver.ctx, C.byref(f), C.byref(b), C.byref(t)),
                   "dgr_adjoint_timing")
        return f.value, b.value, t.value


def _torch_function():
    import torch

    class MisfitFunction(torch.autograd.Function):
        """J(n_el, z) of a GaugeMisfit from a fixed initial state; backward is the discrete
        adjoint.  z None keeps the depths (the only choice on an Ensemble).  Each backward
        must follow its own forward (the adjoint replays the last recorded run)."""

        @staticmethod
        def forward(ctx, n_el, z, misfit, state, time, dt):
            s = misfit.solver
            s.set_element_manning(n_el.detach().cpu().numpy().astype(np.float64))
            if z is not None:
                s.set_bathymetry(z.detach().cpu().numpy().astype(np.float64))
            J, _ = misfit.forward(state, time, dt)
            ctx.misfit = misfit
            ctx.dev = (n_el.device, None if z is None else z.device)
            return torch.tensor(J, dtype=torch.float64, device=n_el.device)

        @staticmethod
        def backward(ctx, gJ):
            g = ctx.misfit.backward()
            gn = torch.from_numpy(g["n_el"]).to(ctx.dev[0]) * gJ
            gz = None if ctx.dev[1] is None else torch.from_numpy(g["z"]).to(ctx.dev[1]) * gJ
            return gn, gz, None, None, None, None

    return MisfitFunction


_FN = None


def gauge_misfit(n_el, z, misfit: GaugeMisfit, state, time: float = -1.0, dt: float = 0.0):
    """torch scalar J(n_el, z) differentiable with respect to the float64 tensors n_el
    (per element) and z (per node, or None to keep the depths)."""
    global _FN
    if _FN is None:
        _FN = _torch_function()
    return _FN.apply(n_el, z, misfit, state, time, dt)
