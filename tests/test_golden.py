"""The oracle restatement against golden vectors that the unmodified reference wrote
(tests/golden/make_golden.py).  Runs everywhere: no reference tree, no GPU needed."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import bits_equal, load_golden, mesh_from_golden


@pytest.mark.parametrize("flag", [0, 1])
def test_oracle_compute2DL_golden(dgrain, oracle_mod, flag):
    g = load_golden("compute2DL_jittered576.npz")
    m = mesh_from_golden(dgrain, g)
    # the generator and the native connectivity builder still give the stored mesh
    m2 = dgrain.rectangle(24, 12, jitter=0.1, seed=5)
    for k in ("x", "y", "z", "el2v", "ed2v", "ed2el", "bdry"):
        assert bits_equal(getattr(m2, k), g[k]), k
    orc = oracle_mod.Oracle(m)
    wd = g["wd_rand"] if flag else np.full(m.num_el, -1, dtype=np.int32)
    orc.set_state(g["zeta"], g["qx"], g["qy"], wd)
    orc.set_bc(g["bzeta"], g["bqn"])
    rc, rz, rx, ry, lam = orc.compute_L(flag)
    assert rc == 0
    assert bits_equal(rz, g[f"wd{flag}_rhs_zeta"])
    assert bits_equal(rx, g[f"wd{flag}_rhs_qx"])
    assert bits_equal(ry, g[f"wd{flag}_rhs_qy"])
    assert lam == float(g[f"wd{flag}_max_lambda"])
    for a, k in zip(orc.fhat(), ("f1", "f2", "f3")):
        assert bits_equal(a, g[f"wd{flag}_{k}"])


def test_oracle_run_golden(dgrain, oracle_mod):
    g = load_golden("run120_wd_tide_rect1600.npz")
    m = mesh_from_golden(dgrain, g)
    orc = oracle_mod.Oracle(m)
    orc.set_state(g["zeta0"], g["qx0"], g["qy0"], g["wd0"])
    rc, t, dt, n, hist = orc.run(120, 1e9, 0.3, wet_dry=1, tide_on=1, amp=0.5, want_dt=True)
    assert rc == 0 and n == 120
    z, qx, qy, wd = orc.get_state()
    assert bits_equal(z, g["zeta"]) and bits_equal(qx, g["qx"]) and bits_equal(qy, g["qy"])
    assert bits_equal(wd, g["wd"])
    assert t == float(g["time"]) and dt == float(g["dt_next"])
    assert bits_equal(hist, g["dt_hist"])


def test_oracle_failure_golden(dgrain, oracle_mod):
    g = load_golden("failure_film_h0_rect1600.npz")
    m = mesh_from_golden(dgrain, g)
    orc = oracle_mod.Oracle(m)
    orc.set_state(g["zeta0"], g["qx0"], g["qy0"], g["wd0"])
    rc, t, dt, n, _ = orc.run(50, 1e9, 0.3, wet_dry=1, tide_on=1, amp=0.5)
    code, idx = orc.last_error()
    assert rc == code == 1
    assert idx == int(g["fail_edge"]) and n == int(g["steps_done"])


def test_numpy_mesh_setup_golden(dgrain):
    """The oracle's numpy mesh set-up (oracle/mesh_setup.py, used where the reference step
    runs on meshes too large for its own set-up) gives the arrays the reference wrote."""
    from oracle import mesh_setup

    for name in ("compute2DL_jittered576.npz", "run120_wd_tide_rect1600.npz"):
        g = load_golden(name)
        ed2v, ed2el, bdry, min_edge = mesh_setup.connectivity(g["el2v"], g["x"], g["y"], g["inflow1"],
                                                              g["inflow2"], g["outflow"])
        assert bits_equal(ed2v, g["ed2v"]) and bits_equal(ed2el, g["ed2el"]) and bits_equal(bdry, g["bdry"]), name
        assert min_edge == float(g["min_edge"]), name


@pytest.mark.parametrize("nx,ny,jitter,seed", [(40, 20, 0.0, 1), (57, 31, 0.1, 4), (200, 100, 0.1, 2)])
def test_numpy_mesh_setup_equals_native_builder(dgrain, nx, ny, jitter, seed):
    """The numpy set-up against the library's hashed builder and initial state, with every
    boundary type present."""
    from oracle import mesh_setup

    m = dgrain.rectangle(nx, ny, jitter=jitter, seed=seed, connect=False)
    bottom = np.stack([np.arange(nx), np.arange(1, nx + 1)], 1).astype(np.int32)
    m.inflow1 = np.ascontiguousarray(bottom[: nx // 2])
    m.inflow2 = np.ascontiguousarray(np.concatenate([bottom[nx // 2:], bottom[:2]]))
    dgrain.build_connectivity(m)
    ed2v, ed2el, bdry, min_edge = mesh_setup.connectivity(m.el2v, m.x, m.y, m.inflow1, m.inflow2, m.outflow)
    assert bits_equal(ed2v, m.ed2v) and bits_equal(ed2el, m.ed2el) and bits_equal(bdry, m.bdry)
    assert min_edge == m.min_edge
    zn = np.maximum(0.0, 0.5e-3 - m.z)
    for a, b in zip(mesh_setup.initial_state(m.el2v, zn), dgrain.initial_state(m, zn)):
        assert bits_equal(a, b)
