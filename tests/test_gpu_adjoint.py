"""Discrete adjoint and tangent-linear model of the device time loop, on the GPU.

Gauge-misfit objective over a run with checkpoints (ragged last segment), gradients with
respect to per-element Manning n, node depth and the initial state:
  * the recorded forward run is dgr_run's run bit for bit, and the TLM's primal is too;
  * adjoint . direction == TLM directional derivative to round-off (dot-product test),
    with wet/dry off and on (shoreline, limiter and PDop branches active);
  * central finite differences with frozen masks and dt agree with the TLM to 1e-6 along
    random directions in n, depth and state; so do finite differences of the plain run (dt
    frozen) along n and depth on a smooth, fully submerged case; the Taylor remainder is
    second order;
  * gradients are bitwise reproducible; the torch.autograd.Function returns them.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import bits_equal, land_film_state

pytestmark = pytest.mark.gpu

NSTEPS, CKPT = 40, 16


def midpoints(m):
    v = m.el2v
    return (0.5 * (m.x[v] + m.x[np.roll(v, -1, axis=1)])).reshape(-1), \
        (0.5 * (m.y[v] + m.y[np.roll(v, -1, axis=1)])).reshape(-1)


def basin_case(dgrain, nx=24, ny=12, seed=5):
    """Submerged basin (depth 4.5-12.5 m), tide at x = 0; the initial state has structure
    everywhere (a Gaussian hump of 0.3 m on a basin-wide 5 cm tilt, a smooth background
    discharge), so no decision sits at a flat, zero-flow tie."""
    m = dgrain.rectangle(nx, ny, jitter=0.15, seed=seed, datum=7.0)
    rng = np.random.default_rng(seed)
    cx, cy = rng.uniform(3000, 7000), rng.uniform(1500, 3500)
    zn = 0.3 * np.exp(-((m.x - cx) ** 2 + (m.y - cy) ** 2) / (2 * 1200.0 ** 2)) + \
        0.05 * np.sin(2 * np.pi * m.x / 10000.0 + 0.3) * np.cos(np.pi * m.y / 5000.0 + 0.2)
    zeta, _, _, wd = dgrain.initial_state(m, zn)
    mx, my = midpoints(m)
    qx = 0.2 * np.sin(np.pi * mx / 10000.0 + 0.4) * np.cos(2 * np.pi * my / 5000.0 + 0.1)
    qy = 0.15 * np.cos(np.pi * mx / 5000.0 + 0.7) * np.sin(np.pi * my / 5000.0 + 0.5)
    n_el = rng.uniform(0.02, 0.05, m.num_el)
    pts = list(zip(rng.uniform(500, 9500, 8), rng.uniform(500, 4500, 8)))
    return m, (zeta, qx, qy, wd), n_el, pts


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


def smooth_field(m, rng, n_bumps=6, width=1500.0):
    """random smooth field at the element midpoints [3*el+k]: a sum of Gaussian bumps"""
    mx, my = midpoints(m)
    f = np.zeros(mx.shape)
    for _ in range(n_bumps):
        cx, cy = rng.uniform(m.x.min(), m.x.max()), rng.uniform(m.y.min(), m.y.max())
        f += rng.normal() * np.exp(-((mx - cx) ** 2 + (my - cy) ** 2) / (2 * width ** 2))
    return f


def directions(m, seed):
    """random directions: per-element n and per-node depth noise; smooth state fields (state
    noise would put the limiter's decisions at the scale of the perturbation itself)"""
    rng = np.random.default_rng(seed)
    dn = rng.normal(size=m.num_el)
    dz = rng.normal(size=m.num_nodes)
    ds = tuple(smooth_field(m, rng) for _ in range(3))
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
            assert bits_equal(a, b)
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


def _fd_ladder(J, h0):
    """central differences for steps h0 * 10^(-k/2), k = 0..4: round-off grows as the step
    shrinks, decision kinks crossed inside the interval as it grows"""
    return [(h0 * 10 ** (-k / 2), (J(h0 * 10 ** (-k / 2)) - J(-h0 * 10 ** (-k / 2))) / (2 * h0 * 10 ** (-k / 2)))
            for k in range(5)]


def test_gradients_match_frozen_finite_differences(dgrain):
    """Central finite differences with frozen masks and dt (dgr_fd_frozen: the recorded
    run's decisions and dt sequence held at the perturbed points) along 16 random directions
    in n, depth and the initial state (raw per-entry noise included) agree with the
    tangent-linear model, and with the adjoint, to 1e-6."""
    case = basin_case(dgrain)
    m, state, n_el, _ = case
    s, mis = make(dgrain, case, 1)
    J0, _ = mis.forward(state)
    g = mis.backward()
    mis.forward(state)  # recorded run again (the backward leaves the context's state spent)
    assert mis.frozen(state) == (J0, J0)
    z0 = m.z.copy()
    rng = np.random.default_rng(17)
    worst = 0.0
    for k in range(16):
        dn, dz, ds = directions(m, 200 + k)
        kind = k % 3
        if kind == 2 and k % 2:
            ds = tuple(rng.normal(size=3 * m.num_el) for _ in range(3))  # raw noise
            ds = tuple(d / np.linalg.norm(d) for d in ds)
        if kind == 0:
            h0 = 1e-4 * np.abs(n_el).max() / np.abs(dn).max()
            J = lambda e: mis.frozen(state, n_el=n_el + e * dn)[1]  # noqa: E731
            adj, kw = g["n_el"] @ dn, dict(dn_el=dn)
        elif kind == 1:
            h0 = 1e-4 * np.abs(z0).max() / np.abs(dz).max()
            J = lambda e: mis.frozen(state, z=z0 + e * dz)[1]  # noqa: E731
            adj, kw = g["z"] @ dz, dict(dz=dz)
        else:
            h0 = 1e-4 * np.abs(state[0]).max() / max(np.abs(d).max() for d in ds)
            J = lambda e: mis.frozen(state, state_p=tuple(a + e * d for a, d in zip(state[:3], ds)))[1]  # noqa
            adj = g["zeta0"] @ ds[0] + g["qx0"] @ ds[1] + g["qy0"] @ ds[2]
            kw = dict(dstate=ds)
        ladder = _fd_ladder(J, h0)
        _, dJ = mis.tlm(state, **kw)
        rel = min(abs(fd - dJ) for _, fd in ladder) / abs(dJ)
        worst = max(worst, rel)
        assert rel < 1e-6, (k, kind, dJ, ladder)
        assert abs(adj - dJ) <= 1e-10 * abs(dJ)
    assert worst < 1e-6
    s.close()


def test_gradients_match_finite_differences_of_the_run(dgrain):
    """Central differences of the plain forward run (dt sequence frozen, decisions taken
    afresh) along random directions in n and depth agree with the tangent-linear model to
    1e-6 wherever the run is smooth along the direction.  The reference limiter's
    redistribution jumps where a vertex's deviation from the element mean changes sign, so
    some directions cross a jump within every step size: their difference quotients
    scatter as 1/h along the ladder and they are left out; most directions are smooth."""
    case = basin_case(dgrain)
    m, state, n_el, _ = case
    s, mis = make(dgrain, case, 1)
    mis.forward(state)
    z0 = m.z.copy()
    smooth = 0
    for k in range(8):
        dn, dz, _ = directions(m, 100 + k)
        if k % 2 == 0:
            h0 = 1e-4 * np.abs(n_el).max() / np.abs(dn).max()
            J = lambda e: _run_n(s, mis, state, n_el + e * dn)  # noqa: E731
            kw = dict(dn_el=dn)
        else:
            h0 = 1e-4 * np.abs(z0).max() / np.abs(dz).max()
            J = lambda e: _run_z(s, mis, state, z0 + e * dz)  # noqa: E731
            kw = dict(dz=dz)
        ladder = _fd_ladder(J, h0)
        s.set_element_manning(n_el)
        s.set_bathymetry(z0)
        mis.forward(state)
        _, dJ = mis.tlm(state, **kw)
        fds = np.array([fd for _, fd in ladder])
        if np.abs(np.diff(fds[:4])).max() > 1e-4 * abs(dJ):
            continue  # a jump inside the interval
        smooth += 1
        rel = np.abs(fds - dJ).min() / abs(dJ)
        assert rel < 1e-6, (k, dJ, ladder)
    assert smooth >= 4
    s.close()


def test_taylor_remainder_is_second_order(dgrain):
    """|J(p + h d) - J(p) - h J'(p) d| falls as h^2 along one direction in n, depth and state
    together (perturbations of 1 % down to 0.1 %): the gradient is the derivative."""
    case = basin_case(dgrain)
    m, state, n_el, _ = case
    s, mis = make(dgrain, case, 1)
    J0, _ = mis.forward(state)
    g = mis.backward()
    dn, dz, ds = directions(m, 7)
    dn *= 0.01 * np.abs(n_el).max() / np.abs(dn).max()
    dz *= 0.01 * np.abs(m.z).max() / np.abs(dz).max()
    ds = tuple(d * 0.01 * np.abs(state[0]).max() / np.abs(d).max() for d in ds)
    slope = g["n_el"] @ dn + g["z"] @ dz + g["zeta0"] @ ds[0] + g["qx0"] @ ds[1] + g["qy0"] @ ds[2]
    rem = []
    hs = (1.0, 0.3, 0.1)
    for h in hs:
        s.set_element_manning(n_el + h * dn)
        s.set_bathymetry(m.z + h * dz)
        Jh = mis.forward(tuple(a + h * d for a, d in zip(state[:3], ds)) + (state[3],), replay_dt=True)[0]
        rem.append(abs(Jh - J0 - h * slope))
    s.set_element_manning(n_el)
    s.set_bathymetry(m.z)
    rates = [np.log(rem[i] / rem[i + 1]) / np.log(hs[i] / hs[i + 1]) for i in range(2)]
    assert all(1.8 < r < 2.2 for r in rates), (rem, rates)
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
        assert bits_equal(g1[k], g2[k]), k
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
    assert bits_equal(n_t.grad.numpy(), g["n_el"])
    assert bits_equal(z_t.grad.numpy(), g["z"])
    # a small step against the n gradient lowers the misfit
    step = 1e-3 * n_el.max() / np.abs(g["n_el"]).max()
    with torch.no_grad():
        J1 = dgrain.gauge_misfit(n_t - step * n_t.grad, z_t, mis, state)
    assert float(J1) < float(J)
    s.close()
