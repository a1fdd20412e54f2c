"""Host side of the zonal calibration (no GPU): the 4 x 4 zone tiling of normalised
coordinates, the seeded workload's shapes and determinism, p = 2 gauge weights reproducing
the modal elevation at the gauge points."""
from __future__ import annotations

import numpy as np


def test_zone_index_tiles_normalised_coordinates(dgrain):
    from dgrain import calibration as cb

    m = dgrain.rectangle(16, 8, jitter=0.2, seed=1)
    z = cb.zone_index(m)
    assert z.shape == (m.num_el,) and z.min() == 0 and z.max() == 15
    cx = m.x[m.el2v].mean(axis=1)
    cy = m.y[m.el2v].mean(axis=1)
    ix, iy = z % 4, z // 4
    assert np.all(cx[ix == 0] < 2500 + 1e-9) and np.all(cx[ix == 3] >= 7500 - 1e-9)
    assert np.all(cy[iy == 0] < 1250 + 1e-9) and np.all(cy[iy == 3] >= 3750 - 1e-9)
    assert np.bincount(z, minlength=16).min() > 0


def test_workload_is_seeded(dgrain):
    from dgrain import calibration as cb

    a = cb.ensemble_workload(3, 800, 2000, seed=4)
    b = cb.ensemble_workload(3, 800, 2000, seed=4)
    meshes, params, states, gauges, zones, n_true = a
    assert len(meshes) == len(params) == len(states) == len(gauges) == len(zones) == 3
    assert n_true.shape == (16,) and np.all((0.02 <= n_true) & (n_true <= 0.06))
    for k, m in enumerate(meshes):
        assert 700 <= m.num_el <= 2400
        assert states[k][0].shape == (6 * m.num_el,)
        assert gauges[k][1].shape == (32, 6)
        assert np.array_equal(states[k][0], b[2][k][0]) and np.array_equal(gauges[k][0], b[3][k][0])
        # the hump's crest is the highest modal elevation
        assert states[k][0].reshape(-1, 6)[:, 0].max() > 0.5
    assert np.array_equal(n_true, b[5])


def test_relative_error():
    from dgrain import calibration as cb

    assert cb.relative_error([1.0, 2.0], [1.0, 2.0]) == 0.0
    assert abs(cb.relative_error([1.1, 2.0], [1.0, 2.0]) - 0.1 / np.sqrt(5)) < 1e-15
