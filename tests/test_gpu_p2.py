"""The p = 2 modal step (dgr_params.order = 2; an extension without a 2DCode counterpart,
so it is checked by the properties of the discrete scheme and by convergence):
  * a lake at rest over varying depth stays at rest (well-balanced);
  * the water volume of a closed basin is conserved to round-off;
  * a linear standing wave converges at third order in space and time (SSP(3,3));
  * the result does not depend on the orientation of the elements' vertex lists;
  * an ensemble of p = 2 meshes gives each scenario's bits alone."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import bits_equal

pytestmark = pytest.mark.gpu

G = 9.81


def basin(dgrain, nx, ny, seed=2, jitter=0.15, flat=None):
    m = dgrain.rectangle(nx, ny, jitter=jitter, seed=seed, datum=7.0, ocean=False)
    if flat is not None:
        m.z[:] = flat
        m.nfric[:] = 0.0
    return m


def solver(dgrain, m, **kw):
    kw.setdefault("rk_stages", 3)
    return dgrain.Solver(m, order=2, wet_dry=0, cfl=0.1, tide_on=0, **kw)


def p2_state(dgrain, m, fz, fqx=None, fqy=None):
    zero = lambda x, y: np.zeros_like(x)  # noqa: E731
    return (dgrain.p2.project(m, fz), dgrain.p2.project(m, fqx or zero), dgrain.p2.project(m, fqy or zero),
            np.zeros(m.num_el, dtype=np.int32))


def test_lake_at_rest(dgrain):
    m = basin(dgrain, 16, 8)
    st = p2_state(dgrain, m, lambda x, y: np.full_like(x, 0.1))
    with solver(dgrain, m) as s:
        s.upload_state(*st)
        rz, rx, ry, _ = s.compute2DL(0.0)
        assert max(np.abs(rz).max(), np.abs(rx).max(), np.abs(ry).max()) < 1e-12
        s.time_evolution(1e300, 50)
        z, qx, qy, _ = s.download_state()
    assert np.abs(z - st[0]).max() < 1e-12 and np.abs(qx).max() < 1e-10 and np.abs(qy).max() < 1e-10


def test_closed_basin_conserves_volume(dgrain):
    m = basin(dgrain, 16, 8)
    hump = lambda x, y: 0.3 * np.exp(-((x - 4000) ** 2 + (y - 2500) ** 2) / (2 * 900.0 ** 2))  # noqa: E731
    st = p2_state(dgrain, m, hump)
    v0 = dgrain.p2.volume(m, st[0])
    with solver(dgrain, m) as s:
        s.upload_state(*st)
        t, dt, n = s.time_evolution(1e300, 100)
        z, qx, _, _ = s.download_state()
    assert n == 100 and np.abs(qx).max() > 1e-3  # the hump has spread
    assert abs(dgrain.p2.volume(m, z) - v0) <= 1e-12 * abs(v0)


def standing_wave_error(dgrain, nx, t_end=250.0, amp=1e-5, depth=10.0, lx=10000.0, rk_stages=3):
    """L2 error of zeta against A cos(kx) cos(wt), the linear standing wave of a closed
    flat basin (relative to the L2 norm of zeta at t = 0)"""
    m = basin(dgrain, nx, nx // 2, flat=depth, jitter=0.1)
    k = np.pi / lx
    w = k * np.sqrt(G * depth)
    st = p2_state(dgrain, m, lambda x, y: amp * np.cos(k * x))
    with solver(dgrain, m, rk_stages=rk_stages) as s:
        s.upload_state(*st)
        t, dt, n = s.time_evolution(t_end, 10 ** 6)
        z = s.download_state()[0]
    assert t == t_end
    exact = lambda x, y: amp * np.cos(k * x) * np.cos(w * t_end)  # noqa: E731
    norm = dgrain.p2.l2_error(m, np.zeros_like(z), lambda x, y: amp * np.cos(k * x))
    return dgrain.p2.l2_error(m, z, exact) / norm


def test_standing_wave_converges_at_third_order(dgrain):
    e = [standing_wave_error(dgrain, nx) for nx in (8, 16, 32)]
    rates = [np.log2(e[i] / e[i + 1]) for i in range(2)]
    assert e[-1] < 1e-3 and rates[-1] > 2.5, (e, rates)


def test_orientation_does_not_matter(dgrain):
    """elements listed clockwise (every other one) run the shared edges in the same direction
    as their neighbours; the Gauss points are paired by the edge's direction bit"""
    m1 = basin(dgrain, 12, 6)
    m2 = dgrain.rectangle(12, 6, jitter=0.15, seed=2, datum=7.0, ocean=False, connect=False)
    m2.el2v[1::2] = m2.el2v[1::2][:, ::-1].copy()
    dgrain.build_connectivity(m2)
    hump = lambda x, y: 0.2 * np.exp(-((x - 5000) ** 2 + (y - 2000) ** 2) / (2 * 1200.0 ** 2))  # noqa: E731
    out = []
    for m in (m1, m2):
        st = p2_state(dgrain, m, hump)
        with solver(dgrain, m) as s:
            s.upload_state(*st)
            s.time_evolution(1e300, 40)
            out.append((m, s.download_state()[0]))
    # compare the fields at the centroids (element order is the same; the centroid is the
    # first point of the area rule, the same point for either vertex order)
    c1 = dgrain.p2.evaluate(m1, out[0][1])[:, 0]
    c2 = dgrain.p2.evaluate(m2, out[1][1])[:, 0]
    assert np.abs(c1 - c2).max() <= 1e-10 * np.abs(c1).max()


def test_p2_ensemble_equals_alone(dgrain):
    meshes = [dgrain.rectangle_with_elements(n, seed=80 + k, cell=5.0, datum=7.0) for k, n in enumerate((500, 1800))]
    params = [dict(tide_on=1, tide_amp=0.3 + 0.4 * k, tide_period=44712.0, rain=1e-6 * k, n_el=None) for k in range(2)]
    states = [p2_state(dgrain, mm, lambda x, y: np.zeros_like(x)) for mm in meshes]
    alone = []
    for mm, p, st in zip(meshes, params, states):
        with dgrain.Solver(mm, order=2, wet_dry=0, cfl=0.1, rk_stages=3, tide_on=1, tide_amp=p["tide_amp"],
                           rain=p["rain"]) as s:
            s.upload_state(*st)
            clock = s.time_evolution(1e300, 20)
            alone.append((clock, s.download_state()))
    with dgrain.Ensemble(meshes, params, order=2, wet_dry=0, cfl=0.1, rk_stages=3) as e:
        for k, st in enumerate(states):
            e.upload_state(k, *st)
        t, dt, n = e.run(20)
        for k in range(2):
            assert (t[k], dt[k], n[k]) == alone[k][0]
            for a, b in zip(e.download_state(k)[:3], alone[k][1][:3]):
                assert bits_equal(a, b)
            assert np.abs(alone[k][1][1]).max() > 0  # the tide drives a flow
