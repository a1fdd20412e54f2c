"""Discrete adjoint and tangent-linear model of the p = 2 modal step (dgr_params.order = 2),
on the GPU: a submerged tidal basin with per-element Manning n, gauges evaluating the modal
elevation at their points.
  * the recorded forward run is dgr_run's run bit for bit, and the TLM's primal is too;
  * adjoint . direction == TLM directional derivative to round-off (dot-product test) for
    n, depth and state directions, with SSP-RK2 and SSP(3,3);
  * central finite differences with frozen dt agree with the TLM to 1e-6;
  * gradients are bitwise reproducible.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import bits_equal

pytestmark = pytest.mark.gpu

NSTEPS, CKPT = 30, 8  # ragged last segment


def p2_case(dgrain, nx=16, ny=8, seed=11):
    m = dgrain.rectangle(nx, ny, jitter=0.15, seed=seed, datum=7.0)
    rng = np.random.default_rng(seed)
    cx, cy = rng.uniform(3000, 7000), rng.uniform(1500, 3500)
    hump = lambda x, y: 0.3 * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * 1500.0 ** 2))  # noqa: E731
    qx = lambda x, y: 0.2 * np.sin(np.pi * x / 10000.0 + 0.4) * np.cos(2 * np.pi * y / 5000.0 + 0.1)  # noqa: E731
    qy = lambda x, y: 0.15 * np.cos(np.pi * x / 5000.0 + 0.7) * np.sin(np.pi * y / 5000.0 + 0.5)  # noqa: E731
    state = (dgrain.p2.project(m, hump), dgrain.p2.project(m, qx), dgrain.p2.project(m, qy),
             np.zeros(m.num_el, dtype=np.int32))
    n_el = rng.uniform(0.02, 0.05, m.num_el)
    pts = list(zip(rng.uniform(500, 9500, 8), rng.uniform(500, 4500, 8)))
    return m, state, n_el, pts


def solver(dgrain, m, rk_stages):
    return dgrain.Solver(m, order=2, wet_dry=0, cfl=0.1, tide_on=1, tide_amp=0.5, rk_stages=rk_stages)


def make(dgrain, case, rk_stages=3):
    m, state, n_el, pts = case
    s = solver(dgrain, m, rk_stages)
    el, w = dgrain.p2.gauge_weights(m, pts)
    mis = dgrain.GaugeMisfit(s, NSTEPS, CKPT, el, w)
    rng = np.random.default_rng(99)
    s.set_element_manning(n_el * np.exp(rng.normal(0.0, 0.2, n_el.shape)))
    _, vals = mis.forward(state)
    mis.set_target(vals)
    s.set_element_manning(n_el)
    return s, mis


def directions(dgrain, m, seed):
    rng = np.random.default_rng(seed)
    dn = rng.normal(size=m.num_el)
    dz = rng.normal(size=m.num_nodes)
    ds = []
    for _ in range(3):
        cx, cy, a = rng.uniform(0, 10000), rng.uniform(0, 5000), rng.normal()
        ds.append(dgrain.p2.project(m, lambda x, y: a * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * 1500.0 ** 2))))
    return dn / np.linalg.norm(dn), dz / np.linalg.norm(dz), tuple(d / np.linalg.norm(d) for d in ds)


def test_p2_forward_is_the_plain_run(dgrain):
    case = p2_case(dgrain)
    s, mis = make(dgrain, case)
    J, vals = mis.forward(case[1])
    want = s.download_state()
    with solver(dgrain, case[0], 3) as r:
        r.set_element_manning(case[2])
        r.upload_state(*case[1])
        t, dt, n = r.time_evolution(1e300, NSTEPS)
        for a, b in zip(r.download_state()[:3], want[:3]):
            assert bits_equal(a, b)
    dts, times = mis.dt_history()
    assert n == NSTEPS and times[-1] + dts[-1] == t
    # the gauge values are the modal elevation at the gauge points
    el, w = dgrain.p2.gauge_weights(case[0], case[3])
    z = want[0].reshape(-1, 6)
    assert np.allclose(vals[-1], (w * z[el]).sum(axis=1), rtol=0, atol=1e-14)
    assert J > 0 and np.isfinite(vals).all()
    Jt, _ = mis.tlm(case[1])
    assert Jt == J
    s.close()


@pytest.mark.parametrize("rk_stages", [2, 3])
def test_p2_adjoint_is_transpose_of_tlm(dgrain, rk_stages):
    case = p2_case(dgrain)
    s, mis = make(dgrain, case, rk_stages)
    J, _ = mis.forward(case[1])
    g = mis.backward()
    dn, dz, ds = directions(dgrain, case[0], 1)
    for kw, adj in ((dict(dn_el=dn), g["n_el"] @ dn), (dict(dz=dz), g["z"] @ dz),
                    (dict(dstate=ds), g["zeta0"] @ ds[0] + g["qx0"] @ ds[1] + g["qy0"] @ ds[2])):
        Jt, dJ = mis.tlm(case[1], **kw)
        assert Jt == J
        assert abs(dJ - adj) <= 1e-10 * max(abs(dJ), abs(adj)) + 1e-14 * J, (rk_stages, kw.keys(), dJ, adj)
    s.close()


def test_p2_gradients_match_frozen_finite_differences(dgrain):
    case = p2_case(dgrain)
    m, state, n_el, _ = case
    s, mis = make(dgrain, case)
    J0, _ = mis.forward(state)
    g = mis.backward()
    mis.forward(state)
    assert mis.frozen(state) == (J0, J0)
    z0 = m.z.copy()
    for k in range(6):
        dn, dz, ds = directions(dgrain, m, 300 + k)
        kind = k % 3
        if kind == 0:
            h0 = 1e-4 * np.abs(n_el).max() / np.abs(dn).max()
            J = lambda e: mis.frozen(state, n_el=n_el + e * dn)[1]  # noqa: E731
            adj, kw = g["n_el"] @ dn, dict(dn_el=dn)
        elif kind == 1:
            h0 = 1e-4 * np.abs(z0).max() / np.abs(dz).max()
            J = lambda e: mis.frozen(state, z=z0 + e * dz)[1]  # noqa: E731
            adj, kw = g["z"] @ dz, dict(dz=dz)
        else:
            h0 = 1e-3 * np.abs(state[0]).max() / max(np.abs(d).max() for d in ds)
            J = lambda e: mis.frozen(state, state_p=tuple(a + e * d for a, d in zip(state[:3], ds)))[1]  # noqa
            adj = g["zeta0"] @ ds[0] + g["qx0"] @ ds[1] + g["qy0"] @ ds[2]
            kw = dict(dstate=ds)
        fds = [(J(h) - J(-h)) / (2 * h) for h in (h0, h0 / 10 ** 0.5, h0 / 10)]
        _, dJ = mis.tlm(state, **kw)
        assert min(abs(f - dJ) for f in fds) <= 1e-6 * abs(dJ), (k, dJ, fds)
        assert abs(adj - dJ) <= 1e-10 * abs(dJ)
    s.close()


def test_p2_gradients_are_reproducible(dgrain):
    case = p2_case(dgrain)
    s, mis = make(dgrain, case)
    mis.forward(case[1])
    g1 = mis.backward()
    mis.forward(case[1])
    g2 = mis.backward()
    for k in g1:
        assert bits_equal(g1[k], g2[k]), k
    s.close()
