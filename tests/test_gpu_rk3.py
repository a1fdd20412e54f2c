"""SSP(3,3) time stepping (rk_stages = 3; coefficients of DG-SWEM src/prep_DG.F:1253-1270,
an extension of 2DCode's SSP-RK2): the device loop against the oracle's restatement
(bit-identical with Manning n = 0), every schedule, the ensemble, and the adjoint of the
three-stage step."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import bits_equal, land_film_state

pytestmark = pytest.mark.gpu


def coastal(dgrain, nx=40, ny=20, seed=3, nfric=0.0):
    m = dgrain.rectangle(nx, ny, jitter=0.1, seed=seed)
    m.nfric[:] = nfric
    return m, land_film_state(dgrain, m)


@pytest.mark.parametrize("schedule", [(128, 0), (64, 1), (256, 2)])
def test_rk3_run_matches_oracle(dgrain, oracle_mod, schedule):
    m, st = coastal(dgrain)
    o = oracle_mod.Oracle(m)
    o.set_state(*st)
    rc, t_o, dt_o, n_o, hist = o.run(40, 1e9, 0.3, wet_dry=1, tide_on=1, amp=0.5, rk_stages=3, want_dt=True)
    assert rc == 0 and n_o == 40
    with dgrain.Solver(m, wet_dry=1, cfl=0.3, tide_on=1, tide_amp=0.5, rk_stages=3) as s:
        s.set_schedule(*schedule)
        s.upload_state(*st)
        assert s.time_evolution(1e9, 40) == (t_o, dt_o, n_o)
        for a, b in zip(s.download_state(), o.get_state()):
            assert bits_equal(a, b), schedule


def test_rk3_host_step_matches_device_loop(dgrain):
    """oneTimeStep2D-style stepping (dgr_step) runs the same three stages"""
    m, st = coastal(dgrain, nfric=0.03)
    with dgrain.Solver(m, wet_dry=1, cfl=0.3, tide_on=0, rk_stages=3) as s:
        s.upload_state(*st)
        t, dt, n = s.time_evolution(1e9, 10)
        want = s.download_state()
        s.upload_state(*st)
        tt, d = 0.0, 1e-7
        for _ in range(10):
            s.boundary_conditions(tt)
            tt = tt + d
            lam = s.oneTimeStep2D(tt, d)
            d = 0.3 * m.min_edge / lam
        assert (tt, d) == (t, dt)
        for a, b in zip(s.download_state(), want):
            assert bits_equal(a, b)


def test_rk3_ensemble_equals_alone(dgrain):
    meshes = [dgrain.rectangle_with_elements(n, seed=50 + k, cell=5.0, datum=7.0) for k, n in enumerate((700, 2300))]
    params = [dict(tide_on=1, tide_amp=0.4 + 0.3 * k, tide_period=44712.0, rain=0.0, n_el=None) for k in range(2)]
    states = [land_film_state(dgrain, mm) for mm in meshes]
    alone = []
    for mm, p, st in zip(meshes, params, states):
        with dgrain.Solver(mm, wet_dry=1, cfl=0.3, tide_on=1, tide_amp=p["tide_amp"], rk_stages=3) as s:
            s.upload_state(*st)
            clock = s.time_evolution(1e300, 15)
            alone.append((clock, s.download_state()))
    with dgrain.Ensemble(meshes, params, wet_dry=1, cfl=0.3, rk_stages=3) as e:
        for k, st in enumerate(states):
            e.upload_state(k, *st)
        t, dt, n = e.run(15)
        for k in range(2):
            assert (t[k], dt[k], n[k]) == alone[k][0]
            for a, b in zip(e.download_state(k), alone[k][1]):
                assert bits_equal(a, b)


def test_rk3_adjoint(dgrain):
    """adjoint . d == TLM for n, depth and state directions; the TLM primal is the forward
    run; central differences with frozen masks and dt agree with the TLM to 1e-6"""
    m, st = coastal(dgrain, nx=32, ny=16, seed=7, nfric=0.03)
    rng = np.random.default_rng(1)
    n_el = rng.uniform(0.02, 0.05, m.num_el)
    el, w = dgrain.place_gauges(m, dgrain.intertidal_points(m, 6, 0.5, 7))
    with dgrain.Solver(m, wet_dry=1, cfl=0.3, tide_on=1, tide_amp=0.5, rk_stages=3) as s:
        mis = dgrain.GaugeMisfit(s, 30, 8, el, w)
        s.set_element_manning(n_el * np.exp(rng.normal(0.0, 0.2, m.num_el)))
        _, vals = mis.forward(st)
        mis.set_target(vals)
        s.set_element_manning(n_el)
        J, _ = mis.forward(st)
        g = mis.backward()
        dn = rng.normal(size=m.num_el)
        dz = rng.normal(size=m.num_nodes)
        ds = tuple(rng.normal(size=3 * m.num_el) for _ in range(3))
        mis.forward(st)
        for kw, adj in ((dict(dn_el=dn), g["n_el"] @ dn), (dict(dz=dz), g["z"] @ dz),
                        (dict(dstate=ds), g["zeta0"] @ ds[0] + g["qx0"] @ ds[1] + g["qy0"] @ ds[2])):
            Jt, dJ = mis.tlm(st, **kw)
            assert Jt == J
            assert abs(dJ - adj) <= 1e-10 * abs(dJ), (kw.keys(), dJ, adj)
        _, dJ = mis.tlm(st, dn_el=dn)
        fds = []
        for rel in (1e-4, 1e-5, 1e-6):
            h = rel * n_el.max() / np.abs(dn).max()
            Jp = mis.frozen(st, n_el=n_el + h * dn)[1]
            Jm = mis.frozen(st, n_el=n_el - h * dn)[1]
            fds.append((Jp - Jm) / (2 * h))
        assert min(abs(f - dJ) for f in fds) <= 1e-6 * abs(dJ), (dJ, fds)
