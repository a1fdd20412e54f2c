"""Pins the oracle: the C restatement (oracle/dgr_oracle.c) against the UNMODIFIED
reference 2DCode compiled into oracle/_ref, bit for bit, and the native mesh ingest
(dgr_read_fort14 / dgr_build_connectivity) against the reference's store_mesh /
extract_mesh_attributes.  Skipped where oracle/_ref was not built (no reference tree);
test_golden.py covers the same ground from committed fixtures."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import bits_equal, land_film_state, moving_state, negative_zeros, signed_zero_state

pytestmark = pytest.mark.skipif(
    not __import__("oracle.oracle", fromlist=["x"]).have_reference(),
    reason="oracle/_ref not built (reference tree absent)")


def _same(a, b):
    return bits_equal(a, b)


@pytest.mark.parametrize("jitter,seed,nx,ny", [(0.0, 1, 40, 20), (0.1, 3, 30, 17), (0.1, 9, 13, 29)])
def test_connectivity_matches_reference(dgrain, oracle_mod, tmp_path, jitter, seed, nx, ny):
    m = dgrain.rectangle(nx, ny, jitter=jitter, seed=seed)
    # add inflow lists on the y = 0 and y = Ly sides so every boundary type appears
    bottom = np.stack([np.arange(nx), np.arange(1, nx + 1)], 1).astype(np.int32)
    top = bottom + ny * (nx + 1)
    m.inflow1 = np.ascontiguousarray(bottom[: nx // 2])
    m.inflow2 = np.ascontiguousarray(np.concatenate([top[: nx // 3], bottom[:2]]))  # overlap: type 3 wins
    dgrain.build_connectivity(m)
    path = str(tmp_path / "m.14")
    dgrain.write_fort14(m, path)
    ref = oracle_mod.Reference(wet_dry=False)
    ref.load_fort14(path)
    rm = ref.get_mesh()
    m2 = dgrain.read_fort14(path)
    for k in ("x", "y", "z", "nfric", "el2v"):
        assert _same(getattr(m2, k), rm[k]), k
        assert _same(getattr(m, k), rm[k]), k
    for k in ("ed2v", "ed2el", "bdry"):
        assert _same(getattr(m, k), rm[k]), k
        assert _same(getattr(m2, k), rm[k]), k
    assert m.min_edge == rm["min_edge"] == m2.min_edge
    assert set(np.unique(m.bdry)) == {0, 1, 2, 3}
    # the numpy restatement that lets the reference step run on meshes too large for its
    # own set-up (bench.py's reference arm)
    from oracle import mesh_setup

    ed2v, ed2el, bdry, min_edge = mesh_setup.connectivity(m.el2v, m.x, m.y, m.inflow1, m.inflow2, m.outflow)
    assert _same(ed2v, rm["ed2v"]) and _same(ed2el, rm["ed2el"]) and _same(bdry, rm["bdry"])
    assert min_edge == rm["min_edge"]


def _pair(dgrain, oracle_mod, mesh, wet_dry, state):
    ref = oracle_mod.Reference(wet_dry=bool(wet_dry))
    ref.set_mesh(mesh)
    ref.initialize()
    ref.set_state(*state)
    ref.boundary_conditions()
    orc = oracle_mod.Oracle(mesh)
    orc.set_state(*state)
    orc.boundary_conditions()
    bz, bq = ref.get_bc()
    orc.set_bc(bz, bq)  # identical boundary arrays (the reference leaves land entries unset)
    return ref, orc


@pytest.mark.parametrize("wet_dry", [0, 1])
@pytest.mark.parametrize("kind", ["film", "moving"])
def test_compute2DL_bitexact(dgrain, oracle_mod, mesh_c1, wet_dry, kind):
    st = land_film_state(dgrain, mesh_c1) if kind == "film" else moving_state(dgrain, mesh_c1, seed=4)
    if wet_dry:
        st = list(st)
        st[3] = np.random.default_rng(1).integers(0, 2, mesh_c1.num_el).astype(np.int32)
    ref, orc = _pair(dgrain, oracle_mod, mesh_c1, wet_dry, st)
    r1 = ref.compute2DL()
    r2 = orc.compute_L(wet_dry)
    assert r1[0] == 0 and r2[0] == 0
    for a, b in zip(r1[1:4], r2[1:4]):
        assert _same(a, b)
    assert r1[4] == r2[4]
    for a, b in zip(ref.fhat(), orc.fhat()):
        assert _same(a, b)


def test_roe_flux_and_inner_products_bitexact(dgrain, oracle_mod, mesh_j):
    ref = oracle_mod.Reference(wet_dry=False)
    ref.set_mesh(mesh_j)
    ref.initialize()
    st = moving_state(dgrain, mesh_j, seed=2)
    ref.set_state(*st)
    ref.compute2DL()
    orc = oracle_mod.Oracle(mesh_j)
    orc.set_state(*st)
    orc.set_bc(*ref.get_bc())
    orc.compute_L(0)
    import ctypes as C

    rng = np.random.default_rng(0)
    for _ in range(200):
        a = list(rng.uniform(0.2, 3.0, 2)) + list(rng.normal(0, 1, 4)) + [rng.uniform(0, 2)]
        th = rng.uniform(0, 2 * np.pi)
        nx, ny = np.cos(th), np.sin(th)
        lg = [0.0, 9.81][rng.integers(0, 2)]
        o1, o2 = np.zeros(3), np.zeros(3)
        l1 = ref.lib.ref_roe_flux(oracle_mod._d(o1), a[0], a[1], a[2], a[3], a[4], a[5], a[6], nx, ny, lg)
        l2 = orc.lib.orc_roe_flux(oracle_mod._d(o2), a[0], a[1], a[2], a[3], a[4], a[5], a[6], nx, ny, lg, 9.81)
        assert l1 == l2 and _same(o1, o2)
    for el in range(0, mesh_j.num_el, 7):
        s1, v1 = np.zeros(9), np.zeros(21)
        s2, v2 = np.zeros(9), np.zeros(21)
        ref.lib.ref_inner_products(el, oracle_mod._d(s1), oracle_mod._d(v1))
        orc.lib.orc_inner_products(C.c_void_p(orc.h), el, oracle_mod._d(s2), oracle_mod._d(v2))
        assert _same(s1, s2) and _same(v1, v2)


@pytest.mark.parametrize("wet_dry", [0, 1])
def test_limiter_pdop_status_bitexact(dgrain, oracle_mod, mesh_c1, wet_dry):
    # a rough state: film initial condition plus noise, so limiter and PDop branches fire
    rng = np.random.default_rng(11)
    z, qx, qy, wd = land_film_state(dgrain, mesh_c1)
    z = z + 0.002 * rng.standard_normal(z.shape)
    qx = 0.01 * rng.standard_normal(qx.shape)
    qy = 0.01 * rng.standard_normal(qy.shape)
    ref, orc = _pair(dgrain, oracle_mod, mesh_c1, wet_dry, (z, qx, qy, wd))
    assert ref.slope_limiter() == 0 and orc.slope_limiter() == 0
    for a, b in zip(ref.get_state()[:3], orc.get_state()[:3]):
        assert _same(a, b)
    assert ref.pdop() == 0 and orc.pdop() == 0
    for a, b in zip(ref.get_state()[:3], orc.get_state()[:3]):
        assert _same(a, b)
    lim, pd = orc.decisions()
    assert lim.sum() > 0 and (pd > 0).sum() > 0
    ref.wd_status()
    orc.wd_status()
    assert _same(ref.get_state()[3], orc.get_state()[3])
    ref.wd_status()
    orc.wd_status()  # second call exercises the hysteresis branch
    assert _same(ref.get_state()[3], orc.get_state()[3])


def test_driver_sequence_equals_reference_oneTimeStep2D(dgrain, oracle_mod, mesh_j):
    """The driver's gsl sequence with wet/dry off and no rain is the reference's own
    oneTimeStep2D (2DCode/time_evolution.c:10-246)."""
    st = moving_state(dgrain, mesh_j, seed=3, qscale=0.05)
    a = oracle_mod.Reference(wet_dry=False)
    a.set_mesh(mesh_j)
    a.initialize()
    a.set_state(*st)
    a.boundary_conditions()
    assert a.step(5.0, 0.5, use_reference_step=True) == 0
    s_ref = a.get_state()
    a.set_state(*st)
    assert a.step(5.0, 0.5, use_reference_step=False) == 0
    for x, y in zip(s_ref[:3], a.get_state()[:3]):
        assert _same(x, y)


@pytest.mark.parametrize("wet_dry", [0, 1])
def test_run_bitexact_with_tide_and_failure(dgrain, oracle_mod, mesh_c1, wet_dry):
    """Long runs: identical states and dt sequences, and identical failure (code, edge)
    when the reference stops on a NaN flux."""
    st = land_film_state(dgrain, mesh_c1)
    ref = oracle_mod.Reference(wet_dry=bool(wet_dry))
    ref.set_mesh(mesh_c1)
    ref.initialize()
    ref.set_state(*st)
    orc = oracle_mod.Oracle(mesh_c1)
    orc.set_state(*st)
    r1 = ref.run(400, 1e9, 0.3, tide_on=1, amp=0.5, want_dt=True)
    r2 = orc.run(400, 1e9, 0.3, wet_dry=wet_dry, tide_on=1, amp=0.5, want_dt=True)
    s1, s2 = ref.get_state(), orc.get_state()
    for x, y in zip(s1, s2):
        assert _same(x, y)
    if r1[0] != 0:
        code, idx = orc.last_error()
        assert r2[0] == code != 0
        assert f"edge {idx} " in ref.message() or f"el {idx} " in ref.message() or f"element {idx} " in ref.message()
        assert r1[3] == r2[3]  # same number of completed steps
    else:
        assert r2[0] == 0 and r1[1] == r2[1] and r1[2] == r2[2]
        assert _same(r1[4], r2[4])


def test_time_loop_matches_reference_time_evolution(dgrain, oracle_mod, mesh_j, tmp_path):
    """ref_run / orc_run (CFL 0.1, no tide, wet/dry off) reproduce the reference's own
    time_evolution(), compared through its .dat output at FinalTime."""
    st = moving_state(dgrain, mesh_j, seed=8, qscale=0.01)
    ref = oracle_mod.Reference(wet_dry=False)
    ref.set_mesh(mesh_j)
    ref.initialize()
    ref.set_state(*st)
    final = 60.0
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        assert ref.time_evolution(final) == 0
    finally:
        os.chdir(cwd)
    got = [np.loadtxt(tmp_path / f"001_{n}.dat").ravel() for n in ("H", "Qx", "Qy")]
    orc = oracle_mod.Oracle(mesh_j)
    orc.set_state(*st)
    rc, t, dt, n, _ = orc.run(10**6, final, 0.1, wet_dry=0)
    assert rc == 0 and t == final
    s = orc.get_state()
    for a, b in zip(got, s[:3]):
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-15 * (1 + np.abs(b).max()) + 1e-15)


@pytest.mark.parametrize("seed", [1, 2])
def test_limiter_signed_zero_bounds_bitexact(dgrain, oracle_mod, seed):
    """Node bounds that are zeros of either sign, and the limiter's clamp on them: the
    restatement gives the reference build's bits, signs of zeros included (the reference
    binary's fmax returns its second operand on a tie)."""
    m = dgrain.rectangle(60, 30, jitter=0.1, seed=13)
    st = signed_zero_state(dgrain, m, seed, nx=60)
    o = oracle_mod.Oracle(m)
    o.set_state(*st)
    o.slope_limiter()
    r = oracle_mod.Reference(wet_dry=True)
    r.set_mesh(m)
    r.initialize()
    r.set_state(*st)
    r.slope_limiter()
    got, want = o.get_state(), r.get_state()
    for a, b in zip(got[:3], want[:3]):
        assert _same(a, b)
    assert negative_zeros(want[1]) > 0  # the case reaches the sign of a zero
