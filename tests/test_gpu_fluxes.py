"""DG-SWEM's local Lax-Friedrichs (dgr_params.flux = 1, src/numerical_flux.F:887-1141) and
HLLC (flux = 2, :1154-1400) fluxes, extensions with no 2DCode counterpart, so checked by the
scheme's properties, each flux:
  * a lake at rest stays at rest and a closed basin conserves its volume (p = 1 and p = 2);
  * a submerged tidal basin stays finite with positive depths and differs from the Roe run
    by a discretisation-sized amount;
  * p = 2 converges at third order;
  * the adjoint is the transpose of the tangent-linear model (p = 1 with wet/dry, p = 2)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import land_film_state

pytestmark = pytest.mark.gpu


def areas(m):
    v = m.el2v
    x, y = m.x[v], m.y[v]
    return 0.5 * np.abs((x[:, 1] - x[:, 0]) * (y[:, 2] - y[:, 0]) - (x[:, 2] - x[:, 0]) * (y[:, 1] - y[:, 0]))


def midpoint_field(m, f):
    v = m.el2v
    mx = 0.5 * (m.x[v] + m.x[np.roll(v, -1, axis=1)])
    my = 0.5 * (m.y[v] + m.y[np.roll(v, -1, axis=1)])
    return np.ascontiguousarray(f(mx, my).reshape(-1))


@pytest.fixture(params=[1, 2], ids=["llf", "hllc"])
def flux(request):
    return request.param


def test_p1_lake_at_rest_and_volume(dgrain, flux):
    m = dgrain.rectangle(24, 12, jitter=0.15, seed=4, datum=7.0, ocean=False)
    zero = np.zeros(3 * m.num_el)
    rest = (np.full(3 * m.num_el, 0.1), zero, zero.copy())
    with dgrain.Solver(m, wet_dry=0, cfl=0.3, tide_on=0, flux=flux) as s:
        s.upload_state(*rest)
        s.time_evolution(1e300, 50)
        z, qx, qy, _ = s.download_state()
        assert np.abs(z - 0.1).max() < 1e-12 and max(np.abs(qx).max(), np.abs(qy).max()) < 1e-10
        hump = midpoint_field(m, lambda x, y: 0.3 * np.exp(-((x - 4000) ** 2 + (y - 2500) ** 2) / (2 * 900.0 ** 2)))
        s.upload_state(hump, zero, zero.copy())
        s.time_evolution(1e300, 100)
        z, qx, _, _ = s.download_state()
    a = areas(m)
    v0 = (a * hump.reshape(-1, 3).mean(axis=1)).sum()
    v1 = (a * z.reshape(-1, 3).mean(axis=1)).sum()
    assert np.abs(qx).max() > 1e-3 and abs(v1 - v0) <= 1e-12 * abs(v0)


def test_p1_tidal_basin_vs_roe(dgrain, flux):
    """a submerged tidal basin (wet/dry on, every element wet): finite, positive depths,
    and within a discretisation-sized distance of the Roe run"""
    m = dgrain.rectangle(40, 20, jitter=0.1, seed=3, datum=7.0)
    st = dgrain.initial_state(m, np.zeros(m.num_nodes))
    out = []
    for f in (0, flux):
        with dgrain.Solver(m, wet_dry=1, cfl=0.3, tide_on=1, tide_amp=0.5, flux=f) as s:
            s.upload_state(*st)
            t, dt, n = s.time_evolution(1e300, 300)
            assert n == 300
            out.append(s.download_state())
    z0, z1 = out[0][0], out[1][0]
    assert np.isfinite(z1).all()
    H = z1.reshape(-1, 3) + 0.5 * (m.z[m.el2v] + m.z[np.roll(m.el2v, -1, axis=1)])
    assert H.min() > 0
    d = np.abs(z1 - z0).max()
    assert 0 < d < 0.05 * np.abs(z0).max(), (d, np.abs(z0).max())


def test_p2_well_balanced_and_convergent(dgrain, flux):
    m = dgrain.rectangle(16, 8, jitter=0.15, seed=2, datum=7.0, ocean=False)
    c = dgrain.p2.project(m, lambda x, y: np.full_like(x, 0.1))
    zero = np.zeros_like(c)
    with dgrain.Solver(m, order=2, wet_dry=0, cfl=0.1, rk_stages=3, tide_on=0, flux=flux) as s:
        s.upload_state(c, zero, zero.copy(), np.zeros(m.num_el, dtype=np.int32))
        s.time_evolution(1e300, 50)
        z, qx, qy, _ = s.download_state()
    assert np.abs(z - c).max() < 1e-12 and max(np.abs(qx).max(), np.abs(qy).max()) < 1e-10
    errs = []
    for nx in (8, 16, 32):
        mm = dgrain.rectangle(nx, nx // 2, jitter=0.1, seed=2, datum=7.0, ocean=False)
        mm.z[:] = 10.0
        mm.nfric[:] = 0.0
        k = np.pi / 10000.0
        w = k * np.sqrt(9.81 * 10.0)
        c0 = dgrain.p2.project(mm, lambda x, y: 1e-5 * np.cos(k * x))
        zz = np.zeros_like(c0)
        with dgrain.Solver(mm, order=2, wet_dry=0, cfl=0.1, rk_stages=3, tide_on=0, flux=flux) as s:
            s.upload_state(c0, zz, zz.copy(), np.zeros(mm.num_el, dtype=np.int32))
            t, _, _ = s.time_evolution(250.0, 10 ** 6)
            z = s.download_state()[0]
        norm = dgrain.p2.l2_error(mm, np.zeros_like(z), lambda x, y: 1e-5 * np.cos(k * x))
        errs.append(dgrain.p2.l2_error(mm, z, lambda x, y: 1e-5 * np.cos(k * x) * np.cos(w * t)) / norm)
    rate = np.log2(errs[1] / errs[2])
    assert errs[-1] < 1e-3 and rate > 2.5, (errs, rate)


@pytest.mark.parametrize("order", [1, 2])
def test_adjoint_is_transpose_of_tlm(dgrain, flux, order):
    rng = np.random.default_rng(8)
    if order == 1:
        m = dgrain.rectangle(32, 16, jitter=0.1, seed=7)
        st = land_film_state(dgrain, m)
        kw = dict(wet_dry=1, cfl=0.3)
        el, w = dgrain.place_gauges(m, dgrain.intertidal_points(m, 6, 0.5, 7))
        nm = 3
    else:
        m = dgrain.rectangle(16, 8, jitter=0.15, seed=11, datum=7.0)
        hump = lambda x, y: 0.3 * np.exp(-((x - 5000) ** 2 + (y - 2500) ** 2) / (2 * 1500.0 ** 2))  # noqa: E731
        c = dgrain.p2.project(m, hump)
        st = (c, np.zeros_like(c), np.zeros_like(c), np.zeros(m.num_el, dtype=np.int32))
        kw = dict(order=2, wet_dry=0, cfl=0.1, rk_stages=3)
        el, w = dgrain.p2.gauge_weights(m, list(zip(rng.uniform(500, 9500, 6), rng.uniform(500, 4500, 6))))
        nm = 6
    n_el = rng.uniform(0.02, 0.05, m.num_el)
    with dgrain.Solver(m, tide_on=1, tide_amp=0.5, flux=flux, **kw) as s:
        mis = dgrain.GaugeMisfit(s, 24, 8, el, w)
        s.set_element_manning(n_el * np.exp(rng.normal(0.0, 0.2, m.num_el)))
        _, vals = mis.forward(st)
        mis.set_target(vals)
        s.set_element_manning(n_el)
        J, _ = mis.forward(st)
        g = mis.backward()
        dn = rng.normal(size=m.num_el)
        dz = rng.normal(size=m.num_nodes)
        mis.forward(st)
        for kwd, adj in ((dict(dn_el=dn), g["n_el"] @ dn), (dict(dz=dz), g["z"] @ dz)):
            Jt, dJ = mis.tlm(st, **kwd)
            assert Jt == J
            assert abs(dJ - adj) <= 1e-10 * max(abs(dJ), abs(adj)) + 1e-14 * J, (kwd.keys(), dJ, adj)
    assert g["zeta0"].shape == (nm * m.num_el,)
