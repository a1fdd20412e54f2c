"""Gauge series recorded by the device loop (dgr_set_gauges): identical to the gauge values
of the recorded adjoint forward run (the same steps and the same functional), under every
fused schedule, and for an ensemble identical to each scenario run alone (p = 2)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import bits_equal, land_film_state

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("schedule", [(128, 0), (256, 1), (64, 2)])
def test_series_equals_recorded_run(dgrain, schedule):
    m = dgrain.rectangle(40, 20, jitter=0.1, seed=5)
    st = land_film_state(dgrain, m)
    el, w = dgrain.place_gauges(m, dgrain.intertidal_points(m, 6, 0.5, 5))
    with dgrain.Solver(m, wet_dry=1, cfl=0.3, tide_on=1, tide_amp=0.5) as s:
        mis = dgrain.GaugeMisfit(s, 30, 10, el, w)  # target 0: the gauge values themselves
        _, want = mis.forward(st)
        s.set_schedule(*schedule)
        s.set_gauges(el, w, 40)
        s.upload_state(*st)
        t, dt, n = s.time_evolution(1e300, 30)
        got = s.gauge_series()
    assert n == 30 and got.shape == (40, 6)
    assert bits_equal(got[:30], want)
    assert not got[30:].any()  # rows past the run untouched


def test_ensemble_series_equal_alone(dgrain):
    meshes = [dgrain.rectangle_with_elements(n, seed=70 + k, cell=5.0, datum=7.0) for k, n in enumerate((600, 1400))]
    params = [dict(tide_on=1, tide_amp=0.3 + 0.3 * k, tide_period=44712.0, rain=0.0, n_el=None) for k in range(2)]
    rng = np.random.default_rng(2)
    gauges, states = [], []
    for mm in meshes:
        pts = list(zip(rng.uniform(mm.x.min(), mm.x.max(), 3), rng.uniform(mm.y.min(), mm.y.max(), 3)))
        gauges.append(dgrain.p2.gauge_weights(mm, pts))
        hump = lambda x, y: 0.2 * np.exp(-((x - x.mean()) ** 2 + (y - y.mean()) ** 2) / 2e3)  # noqa: E731
        zero = np.zeros(6 * mm.num_el)
        states.append((dgrain.p2.project(mm, hump), zero, zero.copy()))
    common = dict(order=2, wet_dry=0, cfl=0.1, rk_stages=3)
    alone = []
    for k, mm in enumerate(meshes):
        with dgrain.Solver(mm, tide_on=1, tide_amp=params[k]["tide_amp"], **common) as s:
            s.set_gauges(*gauges[k], 20)
            s.upload_state(*states[k])
            s.time_evolution(1e300, 20)
            alone.append(s.gauge_series())
    with dgrain.Ensemble(meshes, params, **common) as e:
        el = np.concatenate([gauges[k][0] + e.el_off[k] for k in range(2)]).astype(np.int32)
        e.set_gauges(el, np.concatenate([gauges[k][1] for k in range(2)]), 20)
        for k in range(2):
            e.upload_state(k, *states[k])
        t, dt, n = e.run(20, final_time=np.array([1e300, 1e300]))
        got = e.gauge_series()
    assert (n == 20).all()
    assert bits_equal(got[:, :3], alone[0]) and bits_equal(got[:, 3:], alone[1])
    assert np.abs(got).max() > 0
