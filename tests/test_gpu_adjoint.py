"""Discrete adjoint and tangent-linear model of the device time loop, on the GPU.

Gauge-misfit objective over a run with checkpoints (ragged last segment), gradients with
respect to per-element Manning n, node depth and the initial state:
  * the recorded forward run is dgr_run's run bit for bit, and the TLM's primal is too;
  * adjoint . direction == TLM directional derivative to round-off (dot-product test),
    with wet/dry off and on (shoreline, limiter and PDop branches active);
  * central finite differences with the recorded dt sequence agree with the TLM to 1e-6
    on a smooth, fully submerged case;
  * gradients are bitwise reproducible; the torch.autograd.Function returns them.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import land_film_state

pytestmark = pytest.mark.gpu

NSTEPS, CKPT = 40, 16


def basin_case(dgrain, nx=24, ny=12, seed=5):
    """Submerged basin (depth 4.5-12.5 m), a Gaussian hump of 0.3 m, tide at x = 0."""
    m = dgrain.rectangle(nx, ny, jitter=0.15, seed=seed, datum=7.0)
    rng = np.random.default_rng(seed)
    cx, cy = rng.uniform(3000, 7000), rng.uniform(1500, 3500)
    zn = 0.3 * np.exp(-((m.x - cx) ** 2 + (m.y - cy) ** 2) / (2 * 1200.0 ** 2))
    state = dgrain.initial_state(m, zn)
    n_el = rng.uniform(0.02, 0.05, m.num_el)
    pts = list(zip(rng.uniform(500, 9500, 8), rng.uniform(500, 4500, 8)))
    return m, state, n_el, pts


def coastal_case(dgrain, nx=32, ny=16, seed=7):
    """The coastal rectangle with a land film: wet/dry shoreline, gauges in the intertidal band."""
    m = dgrain.rectangle(nx, ny, jitter=0.1, seed=seed)
    state = land_film_state(dgrain, m)
    rng = np.random.default_rng(seed)
    n_el = rng.uniform(0.02, 0.05, m.num_el)
    pts = dgrain.intertidal_points(m, 8, 0.5, seed)
    return m, state, n_el, pts


def make(dgrain, case, wet_dry, target_from=None):
    m, state, n_el, pts = case
    s = dgrain.Solver(m, wet_dry=wet_dry, cfl=0.3, tide_on=1, tide_amp=0.5)
    s.set_element_manning(n_el)
    el, w = dgrain.place_gauges(m, pts)
    mis = dgrain.GaugeMisfit(s, NSTEPS, CKPT, el, w)
    # synthetic target: the same run with n perturbed by +-20 % log-normal noise
    rng = np.random.default_rng(99)
    s.set_element_manning(n_el * np.exp(rng.normal(0.0, 0.2, n_el.shape)))
    _, vals = mis.forward(state)
    mis.set_target(vals + 0.0)
    s.set_element_manning(n_el)
    return s, mis


def directions(m, seed):
    rng = np.random.default_rng(seed)
    dn = rng.normal(size=m.num_el)
    dz = rng.normal(size=m.num_nodes)
    ds = tuple(rng.normal(size=3 * m.num_el) for _ in range(3))
    return dn / np.linalg.norm(dn), dz / np.linalg.norm(dz), tuple(d / np.linalg.norm(d) for d in ds)


def test_forward_is_the_plain_run(dgrain):
    case = basin_case(dgrain)
    s, mis = make(dgrain, case, 1)
    J, vals = mis.forward(case[1])
    want_state = s.download_state()
    with dgrain.Solver(case[0], wet_dry=1, cfl=0.3, tide_on=1, tide_amp=0.5) as r:
        r.set_element_manning(case[2])
        r.upload_state(*case[1])
        t, dt, n = r.time_evolution(1e300, NSTEPS)
        for a, b in zip(r.download_state(), want_state):
            assert np.array_equal(a, b)
    dts, times = mis.dt_history()
    assert n == NSTEPS and times[-1] + dts[-1] == t
    assert J > 0 and np.isfinite(vals).all()
    Jt, _ = mis.tlm(case[1])
    assert Jt == J  # the TLM's primal is the forward run, bit for bit
    s.close()


@pytest.mark.parametrize("which", ["basin_wd_off", "basin", "coastal"])
def test_adjoint_is_transpose_of_tlm(dgrain, which):
    case = coastal_case(dgrain) if which == "coastal" else basin_case(dgrain)
    s, mis = make(dgrain, case, 0 if which == "basin_wd_off" else 1)
    J, _ = mis.forward(case[1])
    g = mis.backward()
    dn, dz, ds = directions(case[0], 1)
    for kw, adj in ((dict(dn_el=dn), g["n_el"] @ dn), (dict(dz=dz), g["z"] @ dz),
                    (dict(dstate=ds), g["zeta0"] @ ds[0] + g["qx0"] @ ds[1] + g["qy0"] @ ds[2])):
        Jt, dJ = mis.tlm(case[1], **kw)
        assert Jt == J
        assert abs(dJ - adj) <= 1e-10 * max(abs(dJ), abs(adj)) + 1e-14 * J, (which, kw.keys(), dJ, adj)
    s.close()


def test_gradients_match_finite_differences(dgrain):
    """Central differences with the recorded dt sequence (frozen), 16 random directions in
    n, depth and the initial state.  Steps of 1e-4 relative keep J's round-off (about 1e-18
    here) far below the change of J; Richardson extrapolation of steps h and h/2 removes the
    O(h^2) term, and the agreement of the two steps shows that no decision flips inside the
    interval."""
    case = basin_case(dgrain)
    m, state, n_el, _ = case
    s, mis = make(dgrain, case, 1)
    J0, _ = mis.forward(state)
    g = mis.backward()
    z0 = m.z.copy()
    worst = 0.0
    for k in range(16):
        dn, dz, ds = directions(m, 100 + k)
        kind = k % 3
        if kind == 0:
            h = 1e-4 * np.abs(n_el).max() / np.abs(dn).max()
            J = lambda e: _run_n(s, mis, state, n_el + e * dn)  # noqa: E731
            adj = g["n_el"] @ dn
        elif kind == 1:
            h = 1e-4 * np.abs(z0).max() / np.abs(dz).max()
            J = lambda e: _run_z(s, mis, state, z0 + e * dz)  # noqa: E731
            adj = g["z"] @ dz
        else:
            h = 1e-4 * np.abs(state[0]).max() / max(np.abs(d).max() for d in ds)
            J = lambda e: mis.forward(tuple(a + e * d for a, d in zip(state[:3], ds)) + (state[3],),  # noqa: E731
                                      replay_dt=True)[0]
            adj = g["zeta0"] @ ds[0] + g["qx0"] @ ds[1] + g["qy0"] @ ds[2]
        d1 = (J(h) - J(-h)) / (2 * h)
        d2 = (J(h / 2) - J(-h / 2)) / h
        s.set_element_manning(n_el)
        s.set_bathymetry(z0)
        fd = (4 * d2 - d1) / 3
        _, dJ = mis.tlm(state, **({0: dict(dn_el=dn), 1: dict(dz=dz), 2: dict(dstate=ds)}[kind]))
        assert abs(d2 - d1) <= 1e-3 * abs(dJ), (k, kind, d1, d2)  # smooth over the interval
        rel = abs(fd - dJ) / max(abs(dJ), 1e-300)
        worst = max(worst, rel)
        assert rel < 1e-6, (k, kind, fd, dJ, adj)
        assert abs(adj - dJ) <= 1e-10 * abs(dJ)
    mis.forward(state)  # the recorded run again
    assert worst < 1e-6
    s.close()


def _run_n(s, mis, state, n):
    s.set_element_manning(n)
    return mis.forward(state, replay_dt=True)[0]


def _run_z(s, mis, state, z):
    s.set_bathymetry(z)
    return mis.forward(state, replay_dt=True)[0]


def test_gradients_are_reproducible(dgrain):
    case = coastal_case(dgrain)
    s, mis = make(dgrain, case, 1)
    mis.forward(case[1])
    g1 = mis.backward()
    mis.forward(case[1])
    g2 = mis.backward()
    for k in g1:
        assert np.array_equal(g1[k], g2[k]), k
    assert np.abs(g1["n_el"]).max() > 0 and np.abs(g1["z"]).max() > 0
    s.close()


def test_torch_function(dgrain):
    torch = pytest.importorskip("torch")
    case = basin_case(dgrain)
    m, state, n_el, _ = case
    s, mis = make(dgrain, case, 1)
    n_t = torch.tensor(n_el, dtype=torch.float64, requires_grad=True)
    z_t = torch.tensor(m.z, dtype=torch.float64, requires_grad=True)
    J = dgrain.gauge_misfit(n_t, z_t, mis, state)
    J.backward()
    J0, _ = mis.forward(state)
    g = mis.backward()
    assert float(J.detach()) == J0
    assert np.array_equal(n_t.grad.numpy(), g["n_el"])
    assert np.array_equal(z_t.grad.numpy(), g["z"])
    # a small step against the n gradient lowers the misfit
    step = 1e-3 * n_el.max() / np.abs(g["n_el"]).max()
    with torch.no_grad():
        J1 = dgrain.gauge_misfit(n_t - step * n_t.grad, z_t, mis, state)
    assert float(J1) < float(J)
    s.close()
