"""Resume from a restart file (dgr_save_restart / dgr_load_restart).

The reference has no restart: 2DCode writes .dat snapshots at FinalTime only
(2DCode/time_evolution.c:324-390).  Here a run saved after N steps (state, wet/dry flags,
time and the next dt, in the .dat row layout with values that read back exactly) and
loaded into a fresh context continues bit for bit as the run that never stopped.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import bits_equal, land_film_state

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["coastal_wet_dry", "p2_basin"])
def test_restart_continues_bit_identically(dgrain, tmp_path, case):
    if case == "coastal_wet_dry":
        m = dgrain.rectangle(60, 30, jitter=0.1, seed=7)
        st = land_film_state(dgrain, m)
        kw = dict(wet_dry=1, cfl=0.3, tide_on=1, tide_amp=0.5)
    else:
        m = dgrain.rectangle(30, 15, jitter=0.1, seed=7, datum=7.0)
        hump = lambda x, y: 0.3 * np.exp(-((x - 5000.0) ** 2 + (y - 2500.0) ** 2) / 1e6)  # noqa: E731
        zero = lambda x, y: np.zeros_like(x)  # noqa: E731
        st = (dgrain.p2.project(m, hump), dgrain.p2.project(m, zero), dgrain.p2.project(m, zero),
              np.zeros(m.num_el, dtype=np.int32))
        kw = dict(wet_dry=0, cfl=0.1, order=2, rk_stages=3, tide_on=1, tide_amp=0.3)
    with dgrain.Solver(m, **kw) as s:
        s.upload_state(*st)
        want_clock = s.time_evolution(1e9, 40)
        want = s.download_state()
    path = tmp_path / "run.rst"
    with dgrain.Solver(m, **kw) as s:
        s.upload_state(*st)
        t, dt, n = s.time_evolution(1e9, 25)
        assert n == 25
        s.save_restart(path, t, dt)
    with dgrain.Solver(m, **kw) as s2:  # a fresh context on the same mesh
        t, dt = s2.load_restart(path)
        t2, dt2, n2 = s2.time_evolution(1e9, 15, t, dt)
        got = s2.download_state()
    assert n2 == 15 and (t2, dt2) == want_clock[:2]
    for a, b in zip(got, want):
        assert bits_equal(a, b)
