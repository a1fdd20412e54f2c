"""The device-side .dat writer (dgr_write_state_dat): byte-identical to the host writer
(printf "%1.15f\\t\\t", the reference's snapshot format) on the state after a wet/dry run,
at p = 2 (six coefficients per line) against Python's correctly rounded formatting, for an
ensemble scenario, and across chunk boundaries."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import land_film_state

pytestmark = pytest.mark.gpu


def test_state_dat_matches_host_writer(dgrain, tmp_path):
    m = dgrain.rectangle(400, 400, jitter=0.1, seed=3)  # 320,000 triangles: two chunks
    with dgrain.Solver(m, wet_dry=1, cfl=0.3, tide_on=1, tide_amp=0.5) as s:
        s.upload_state(*land_film_state(dgrain, m))
        s.time_evolution(1e9, 20)
        z, qx, qy, _ = s.download_state()
        s.write_state_dat(tmp_path / "H.dat", tmp_path / "Qx.dat", tmp_path / "Qy.dat")
        s.write_state_dat(None, tmp_path / "Qx2.dat", None)
    lib = dgrain.load()
    for name, v in (("H", z), ("Qx", qx), ("Qy", qy)):
        ref = tmp_path / f"{name}_host.dat"
        assert lib.dgr_write_dat(str(ref).encode(), m.num_el, v.ctypes.data_as(dgrain._lib.dptr)) == 0
        assert (tmp_path / f"{name}.dat").read_bytes() == ref.read_bytes(), name
    assert (tmp_path / "Qx2.dat").read_bytes() == (tmp_path / "Qx.dat").read_bytes()
    assert not (tmp_path / "Qy2.dat").exists()


def test_p2_and_ensemble_dat(dgrain, tmp_path):
    meshes = [dgrain.rectangle_with_elements(n, seed=90 + k, cell=5.0, datum=7.0) for k, n in enumerate((700, 1600))]
    params = [dict(tide_on=1, tide_amp=0.4, tide_period=44712.0, rain=0.0, n_el=None) for _ in meshes]
    with dgrain.Ensemble(meshes, params, order=2, wet_dry=0, cfl=0.1, rk_stages=3) as e:
        for k, mm in enumerate(meshes):
            hump = lambda x, y: 0.3 * np.exp(-((x - x.mean()) ** 2 + (y - y.mean()) ** 2) / 2e3)  # noqa: E731
            zero = np.zeros(6 * mm.num_el)
            e.upload_state(k, dgrain.p2.project(mm, hump), zero, zero.copy())
        e.run(10)
        z, qx, qy, _ = e.download_state(1)
        e.write_state_dat(1, tmp_path / "z.dat", tmp_path / "qx.dat", None)
    for name, v in (("z", z), ("qx", qx)):
        want = "".join("".join("%1.15f\t\t" % x for x in row) + "\n" for row in v.reshape(-1, 6))
        assert (tmp_path / f"{name}.dat").read_text() == want, name


def test_unformattable_value_is_refused(dgrain, tmp_path):
    """a value of magnitude >= 2^63 is refused with DGR_ERR_INVALID and its file removed"""
    m = dgrain.rectangle(6, 3, seed=1)
    z = np.zeros(3 * m.num_el)
    qx = z.copy()
    qx[4] = 1e19
    with dgrain.Solver(m, wet_dry=0) as s:
        s.upload_state(z, qx, z.copy())
        with pytest.raises(dgrain.DgrError) as ei:
            s.write_state_dat(tmp_path / "z.dat", tmp_path / "qx.dat")
        assert ei.value.code == dgrain._lib.DGR_ERR_INVALID
    assert (tmp_path / "z.dat").exists() and not (tmp_path / "qx.dat").exists()
