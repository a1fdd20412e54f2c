"""Discrete adjoint of the batched ensemble: one recorded run over all scenarios (each with
its own CFL dt and forcing), checkpoints, one backward sweep.
  * each scenario's gradients are those of the scenario run alone, bit for bit, and J is the
    sum of the scenarios' objectives; the dt histories are the scenarios' own;
  * adjoint . direction == TLM directional derivative over the whole ensemble;
at p = 1 with wet/dry on and at p = 2 with SSP(3,3).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import bits_equal, land_film_state

pytestmark = pytest.mark.gpu

NSTEPS, CKPT = 24, 10


def scenarios(dgrain, order):
    meshes = [dgrain.rectangle_with_elements(n, seed=60 + k, cell=5.0, datum=7.0 if order == 2 else 0.0)
              for k, n in enumerate((600, 1500, 1100))]
    params = [dict(tide_on=1, tide_amp=0.3 + 0.2 * k, tide_period=44712.0, rain=1e-6 * k, n_el=None)
              for k in range(len(meshes))]
    rng = np.random.default_rng(5)
    n_el = [rng.uniform(0.02, 0.05, m.num_el) for m in meshes]
    if order == 2:
        states = []
        for m in meshes:
            cx, cy = m.x.mean(), m.y.mean()
            w = 0.2 * (m.x.max() - m.x.min())
            hump = lambda x, y: 0.2 * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * w * w))  # noqa: E731
            zero = np.zeros(6 * m.num_el)
            states.append((dgrain.p2.project(m, hump), zero, zero.copy(), np.zeros(m.num_el, dtype=np.int32)))
    else:
        states = [land_film_state(dgrain, m) for m in meshes]
    gauges = []
    for k, m in enumerate(meshes):
        pts = list(zip(rng.uniform(m.x.min(), m.x.max(), 4), rng.uniform(m.y.min(), m.y.max(), 4)))
        gauges.append(dgrain.p2.gauge_weights(m, pts) if order == 2 else dgrain.place_gauges(m, pts))
    return meshes, params, n_el, states, gauges


def common(order):
    return dict(order=2, wet_dry=0, cfl=0.1, rk_stages=3) if order == 2 else dict(wet_dry=1, cfl=0.3)


def perturbed(n_el):
    """the target's n: each scenario's n with +-20 % log-normal noise (scenario seeds)"""
    return [n * np.exp(np.random.default_rng(99 + k).normal(0.0, 0.2, n.shape)) for k, n in enumerate(n_el)]


def targets(dgrain, mis, setn, n_el, n_target, state):
    setn(n_target)
    _, vals = mis.forward(state)
    mis.set_target(vals)
    setn(n_el)


@pytest.mark.parametrize("order", [1, 2])
def test_ensemble_gradients_equal_alone(dgrain, order):
    meshes, params, n_el, states, gauges = scenarios(dgrain, order)
    alone = []
    for k, m in enumerate(meshes):
        p = params[k]
        with dgrain.Solver(m, tide_on=1, tide_amp=p["tide_amp"], rain=p["rain"], **common(order)) as s:
            mis = dgrain.GaugeMisfit(s, NSTEPS, CKPT, *gauges[k])
            targets(dgrain, mis, s.set_element_manning, n_el[k], perturbed(n_el)[k], states[k])
            J, vals = mis.forward(states[k])
            g = mis.backward()
            alone.append((J, vals, g, mis.dt_history()))
    with dgrain.Ensemble(meshes, params, **common(order)) as e:
        el = np.concatenate([gauges[k][0] + e.el_off[k] for k in range(len(meshes))]).astype(np.int32)
        w = np.concatenate([gauges[k][1] for k in range(len(meshes))])
        mis = dgrain.GaugeMisfit(e, NSTEPS, CKPT, el, w)
        n_flat = np.concatenate(n_el)
        state = e.flatten_states(states)
        targets(dgrain, mis, e.set_element_manning, n_flat, np.concatenate(perturbed(n_el)), state)
        J, vals = mis.forward(state)
        g = mis.backward()
        dt, t = mis.dt_history()
    assert abs(J - sum(a[0] for a in alone)) <= 1e-13 * J
    ng = [len(gg[0]) for gg in gauges]
    off = np.concatenate([[0], np.cumsum(ng)])
    for k in range(len(meshes)):
        assert bits_equal(vals[:, off[k]:off[k + 1]], alone[k][1])
        assert bits_equal(dt[:, k], alone[k][3][0]) and bits_equal(t[:, k], alone[k][3][1])
        e0, e1 = e.el_off[k], e.el_off[k + 1]
        n0, n1 = e.nd_off[k], e.nd_off[k + 1]
        nm = 6 if order == 2 else 3
        ga = alone[k][2]
        assert bits_equal(g["n_el"][e0:e1], ga["n_el"]), k
        assert bits_equal(g["z"][n0:n1], ga["z"]), k
        for key in ("zeta0", "qx0", "qy0"):
            assert bits_equal(g[key][nm * e0:nm * e1], ga[key]), (k, key)
    assert np.abs(g["n_el"]).max() > 0


@pytest.mark.parametrize("order", [1, 2])
def test_ensemble_adjoint_is_transpose_of_tlm(dgrain, order):
    meshes, params, n_el, states, gauges = scenarios(dgrain, order)
    with dgrain.Ensemble(meshes, params, **common(order)) as e:
        el = np.concatenate([gauges[k][0] + e.el_off[k] for k in range(len(meshes))]).astype(np.int32)
        w = np.concatenate([gauges[k][1] for k in range(len(meshes))])
        mis = dgrain.GaugeMisfit(e, NSTEPS, CKPT, el, w)
        n_flat = np.concatenate(n_el)
        state = e.flatten_states(states)
        targets(dgrain, mis, e.set_element_manning, n_flat, np.concatenate(perturbed(n_el)), state)
        J, _ = mis.forward(state)
        g = mis.backward()
        rng = np.random.default_rng(3)
        dn = rng.normal(size=e.ne)
        Jt, dJ = mis.tlm(state, dn_el=dn)
        assert Jt == J
        adj = g["n_el"] @ dn
        assert abs(dJ - adj) <= 1e-10 * max(abs(dJ), abs(adj)), (dJ, adj)
