"""Parity of the sm_100a kernels (through the C ABI) with the oracle restatement, which
tests/test_oracle_pin.py and tests/test_golden.py pin to the reference.

Tolerances.  Every kernel evaluates the reference's expressions in the reference's order
with separately rounded IEEE operations, so results are bit-identical except through
pow(H, 4/3) in the Manning friction: the device evaluates it correctly rounded, glibc's
pow is not correctly rounded for ~0.1% of arguments, and there the two differ by one ulp.
Hence:
  * Manning n = 0 (friction term exactly 0): bit-identical, states and flags;
  * n > 0: wet/dry flags and limiter/PDop decisions identical, FP64 state within
    RTOL_RUN = 1e-11 relative to the largest magnitude of each variable (the target stated
    for this port), single operators within RTOL_OP = 1e-13.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import (bits_equal, land_film_state, load_golden, mesh_from_golden, moving_state, negative_zeros,
                      signed_zero_state)

pytestmark = pytest.mark.gpu

RTOL_RUN = 1e-11
RTOL_OP = 1e-13


def rel_err(a, b):
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / scale)


def same(a, b):
    return bits_equal(a, b)


def no_friction(dgrain, m):
    m2 = dgrain.Mesh(**{f.name: getattr(m, f.name) for f in __import__("dataclasses").fields(m)})
    m2.nfric = np.zeros_like(m.nfric)
    return m2


def expect_same_run(dgrain, s, o, rc, t_o, dt_o, n_o, nsteps):
    """The device loop repeats the oracle's run bit for bit: the same clock and state, or,
    when the reference scheme stops on a NaN, the same failure (code, index, step)."""
    if rc == 0:
        t_g, dt_g, n_g = s.time_evolution(1e9, nsteps)
        assert (t_g, dt_g, n_g) == (t_o, dt_o, n_o)
        for a, b in zip(s.download_state(), o.get_state()):
            assert same(a, b)
    else:
        with pytest.raises(dgrain.StepError) as ei:
            s.time_evolution(1e9, nsteps)
        code, idx = o.last_error()
        assert (ei.value.code, ei.value.index, ei.value.step) == (code, idx, n_o)


def make_pair(dgrain, oracle_mod, m, state, wet_dry=1, **params):
    s = dgrain.Solver(m, wet_dry=wet_dry, record_decisions=1, **params)
    s.upload_state(*state)
    o = oracle_mod.Oracle(m)
    o.set_state(*state)
    return s, o


@pytest.mark.parametrize("wet_dry", [0, 1])
@pytest.mark.parametrize("friction", [False, True])
def test_compute2DL(dgrain, oracle_mod, mesh_j, wet_dry, friction):
    m = mesh_j if friction else no_friction(dgrain, mesh_j)
    st = list(moving_state(dgrain, m, seed=4))
    if wet_dry:
        st[3] = np.random.default_rng(1).integers(0, 2, m.num_el).astype(np.int32)
    s, o = make_pair(dgrain, oracle_mod, m, st, wet_dry)
    o.boundary_conditions()
    s.set_boundary(*o.get_bc())
    rz, rx, ry, lam = s.compute2DL()
    rc, oz, ox, oy, olam = o.compute_L(wet_dry)
    assert rc == 0
    assert lam == olam
    for a, b in zip(s.fhat(), o.fhat()):
        assert same(a, b)  # the edge flux has no pow: always bit-identical
    if friction:
        for a, b in zip((rz, rx, ry), (oz, ox, oy)):
            assert rel_err(a, b) <= RTOL_OP
        assert same(rz, oz)  # the elevation equation has no friction term
    else:
        for a, b in zip((rz, rx, ry), (oz, ox, oy)):
            assert same(a, b)


def test_compute2DL_golden(dgrain):
    g = load_golden("compute2DL_jittered576.npz")
    m = mesh_from_golden(dgrain, g)
    for flag in (0, 1):
        wd = g["wd_rand"] if flag else np.full(m.num_el, -1, dtype=np.int32)
        with dgrain.Solver(m, wet_dry=flag) as s:
            s.upload_state(g["zeta"], g["qx"], g["qy"], wd)
            s.set_boundary(g["bzeta"], g["bqn"])
            rz, rx, ry, lam = s.compute2DL()
            assert lam == float(g[f"wd{flag}_max_lambda"])
            assert same(rz, g[f"wd{flag}_rhs_zeta"])
            assert rel_err(rx, g[f"wd{flag}_rhs_qx"]) <= RTOL_OP
            assert rel_err(ry, g[f"wd{flag}_rhs_qy"]) <= RTOL_OP
            for a, k in zip(s.fhat(), ("f1", "f2", "f3")):
                assert same(a, g[f"wd{flag}_{k}"])


def test_limiter_pdop_status(dgrain, oracle_mod, mesh_c1):
    rng = np.random.default_rng(11)
    z, qx, qy, wd = land_film_state(dgrain, mesh_c1)
    z = z + 0.002 * rng.standard_normal(z.shape)
    qx = 0.01 * rng.standard_normal(qx.shape)
    qy = 0.01 * rng.standard_normal(qy.shape)
    s, o = make_pair(dgrain, oracle_mod, mesh_c1, (z, qx, qy, wd))
    s.SlopeLimiter()
    o.slope_limiter()
    gs, os_ = s.download_state(), o.get_state()
    for a, b in zip(gs[:3], os_[:3]):
        assert same(a, b)
    lim_g, _ = s.decisions(0)
    lim_o, _ = o.decisions()
    assert same(lim_g, lim_o) and lim_o.sum() > 0
    s.PDop2D()
    o.pdop()
    gs, os_ = s.download_state(), o.get_state()
    for a, b in zip(gs[:3], os_[:3]):
        assert same(a, b)
    _, pd_g = s.decisions(0)
    _, pd_o = o.decisions()
    assert same(pd_g, pd_o) and (pd_o > 0).sum() > 0
    for _ in range(2):  # the second call takes the hysteresis branch
        s.wetDryStatus2D()
        o.wd_status()
        assert same(s.download_state()[3], o.get_state()[3])


@pytest.mark.parametrize("wet_dry", [0, 1])
def test_single_step_decisions(dgrain, oracle_mod, mesh_c1, wet_dry):
    m = no_friction(dgrain, mesh_c1)
    st = land_film_state(dgrain, m)
    s, o = make_pair(dgrain, oracle_mod, m, st, wet_dry)
    o.boundary_conditions(0.0, 1, 0.5, 44712.0)
    s.set_boundary(*o.get_bc())
    t, dt = 0.0, 1e-7
    for n in range(3):
        t += dt
        lam = s.oneTimeStep2D(t, dt)
        rc, dec = o.step(t, dt, wet_dry, 0.0, want_decisions=True)
        assert rc == 0
        assert lam == o.max_lambda()
        gs, os_ = s.download_state(), o.get_state()
        for a, b in zip(gs, os_):
            assert same(a, b)
        l0, p0 = s.decisions(0)
        l1, p1 = s.decisions(1)
        assert same(l0, dec[0]) and same(l1, dec[2])
        if wet_dry:
            assert same(p0, dec[1]) and same(p1, dec[3])
        o.boundary_conditions(t, 1, 0.5, 44712.0)
        s.set_boundary(*o.get_bc())
        dt = 0.3 * m.min_edge / lam


def test_run_bitexact_without_friction(dgrain, oracle_mod, mesh_c1):
    """Device-resident loop (CUDA graph, device CFL dt and tide) against the oracle's time
    loop: bit-identical for 150 wet/dry steps when the friction term is zero."""
    m = no_friction(dgrain, mesh_c1)
    st = land_film_state(dgrain, m)
    s, o = make_pair(dgrain, oracle_mod, m, st, 1, cfl=0.3, tide_on=1, tide_amp=0.5)
    rc, t_o, dt_o, n_o, _ = o.run(150, 1e9, 0.3, wet_dry=1, tide_on=1, amp=0.5)
    expect_same_run(dgrain, s, o, rc, t_o, dt_o, n_o, 150)


@pytest.mark.parametrize("block_size", [64, 128, 256])
def test_run_partial_tiles_and_blocks(dgrain, oracle_mod, block_size):
    """A jittered 23 x 11-cell mesh (506 triangles: not a whole number of the geometry's
    32-element tiles, nor of any block size) repeats the oracle bit for bit over 60 wet/dry
    steps with every block size of the element and limiter kernels."""
    m = no_friction(dgrain, dgrain.rectangle(23, 11, jitter=0.1, seed=4))
    assert m.num_el % 32 != 0
    st = land_film_state(dgrain, m)
    s, o = make_pair(dgrain, oracle_mod, m, st, 1, cfl=0.3, tide_on=1, tide_amp=0.5)
    s.set_schedule(block_size, 0)
    rc, t_o, dt_o, n_o, _ = o.run(60, 1e9, 0.3, wet_dry=1, tide_on=1, amp=0.5)
    expect_same_run(dgrain, s, o, rc, t_o, dt_o, n_o, 60)


def test_run_golden_with_friction(dgrain):
    """120 wet/dry steps with tide and friction against the reference's own output."""
    g = load_golden("run120_wd_tide_rect1600.npz")
    m = mesh_from_golden(dgrain, g)
    with dgrain.Solver(m, wet_dry=1, cfl=0.3, tide_on=1, tide_amp=0.5) as s:
        s.upload_state(g["zeta0"], g["qx0"], g["qy0"], g["wd0"])
        t, dt, n = s.time_evolution(1e9, 120)
        assert n == 120
        z, qx, qy, wd = s.download_state()
    assert same(wd, g["wd"])
    assert rel_err(z, g["zeta"]) <= RTOL_RUN
    assert rel_err(qx, g["qx"]) <= RTOL_RUN
    assert rel_err(qy, g["qy"]) <= RTOL_RUN
    assert abs(t - float(g["time"])) <= RTOL_RUN * float(g["time"])
    assert abs(dt - float(g["dt_next"])) <= RTOL_RUN * float(g["dt_next"])


def test_failure_parity_golden(dgrain):
    """Land film at exactly H0: the reference stops with 'both elements wet flux not a
    number, edge N'; the GPU reports the same code, edge and step."""
    g = load_golden("failure_film_h0_rect1600.npz")
    m = mesh_from_golden(dgrain, g)
    with dgrain.Solver(m, wet_dry=1, cfl=0.3, tide_on=1, tide_amp=0.5) as s:
        s.upload_state(g["zeta0"], g["qx0"], g["qy0"], g["wd0"])
        with pytest.raises(dgrain.StepError) as ei:
            s.time_evolution(1e9, 50)
        assert ei.value.code == 1
        assert ei.value.index == int(g["fail_edge"])
        assert ei.value.step == int(g["steps_done"])
        # the context stays usable after the failure
        s.upload_state(g["zeta0"], g["qx0"], g["qy0"], g["wd0"])
        t, dt, n = s.time_evolution(1e9, 1)
        assert n == 1


def test_nan_injection_reports_reference_edge(dgrain, oracle_mod, mesh_j):
    """A NaN planted in the host state: GPU and oracle name the same first edge."""
    st = list(moving_state(dgrain, mesh_j, seed=6, qscale=0.01))
    st[0] = st[0].copy()
    st[0][3 * 100 + 1] = np.nan
    s, o = make_pair(dgrain, oracle_mod, mesh_j, st, 0)
    o.boundary_conditions()
    s.set_boundary(*o.get_bc())
    rc, *_ = o.compute_L(0)
    code, idx = o.last_error()
    assert rc == code == 1
    with pytest.raises(dgrain.StepError) as ei:
        s.compute2DL()
    assert (ei.value.code, ei.value.index) == (code, idx)


@pytest.mark.parametrize("rain", [0.0, 1.0e-6, 2.0e-5])
def test_extensions_rain_element_manning(dgrain, oracle_mod, mesh_j, rain):
    """Rain and per-element Manning n (extensions, same definition on both sides)."""
    m = no_friction(dgrain, mesh_j)
    st = land_film_state(dgrain, m)
    n_el = np.zeros(m.num_el)
    s, o = make_pair(dgrain, oracle_mod, m, st, 1, cfl=0.3, tide_on=1, tide_amp=0.8, rain=rain)
    s.set_element_manning(n_el)
    o.set_element_manning(n_el)
    rc, t_o, dt_o, n_o, _ = o.run(40, 1e9, 0.3, wet_dry=1, rain=rain, tide_on=1, amp=0.8)
    expect_same_run(dgrain, s, o, rc, t_o, dt_o, n_o, 40)


def test_large_mesh_one_step(dgrain, oracle_mod):
    """One wet/dry step on a 400,000-triangle jittered mesh, GPU against the oracle."""
    m = dgrain.rectangle(632, 316, jitter=0.1, seed=21)
    st = land_film_state(dgrain, m)
    s, o = make_pair(dgrain, oracle_mod, m, st, 1, cfl=0.3, tide_on=1, tide_amp=0.5)
    rc, *_ = o.run(2, 1e9, 0.3, wet_dry=1, tide_on=1, amp=0.5)
    assert rc == 0
    t, dt, n = s.time_evolution(1e9, 2)
    gs, os_ = s.download_state(), o.get_state()
    assert same(gs[3], os_[3])
    for a, b in zip(gs[:3], os_[:3]):
        assert rel_err(a, b) <= RTOL_RUN


@pytest.mark.parametrize("friction", [False, True])
def test_million_triangle_wet_dry_run(dgrain, oracle_mod, friction):
    """Six wet/dry steps with the tide on the benchmark's generator at 1,000,000 triangles
    (1,000 x 500 cells, jitter 0.1, land film H0/2, CFL 0.3), device loop against the
    oracle: the same clock and wet/dry flags; without friction the state bit for bit, with
    Manning n = 0.03 within RTOL_RUN of each field's largest magnitude."""
    m = dgrain.rectangle(1000, 500, jitter=0.1, seed=2)
    if not friction:
        m = no_friction(dgrain, m)
    st = land_film_state(dgrain, m)
    s, o = make_pair(dgrain, oracle_mod, m, st, 1, cfl=0.3, tide_on=1, tide_amp=0.5)
    rc, t_o, dt_o, n_o, _ = o.run(6, 1e9, 0.3, wet_dry=1, tide_on=1, amp=0.5)
    assert rc == 0 and n_o == 6
    t, dt, n = s.time_evolution(1e9, 6)
    assert n == 6
    # the clock follows the max wave speed, which friction's last-bit differences can move
    assert t == t_o if not friction else abs(t - t_o) <= RTOL_RUN * abs(t_o)
    gs, os_ = s.download_state(), o.get_state()
    assert same(gs[3], os_[3])
    for a, b in zip(gs[:3], os_[:3]):
        if friction:
            assert rel_err(a, b) <= RTOL_RUN
        else:
            assert same(a, b)
    if not friction:
        assert dt == dt_o
    s.close()


def test_manning_power_correctly_rounded(dgrain):
    """The device x^(4./3) against 60-digit decimal values rounded once to double."""
    import ctypes as C

    g = load_golden("pow43_cr.npz")
    x = np.ascontiguousarray(g["x"])
    y = np.empty_like(x)
    lib = dgrain.load()
    assert lib.dgr_pow43_batch(x.ctypes.data_as(dgrain._lib.dptr), y.ctypes.data_as(dgrain._lib.dptr),
                               len(x), 0) == 0
    assert bits_equal(y, g["cr"])
    # glibc's pow (the reference's) agrees wherever glibc is correctly rounded
    agree = (y == g["glibc"]).mean()
    assert agree > 0.998, agree


def test_manning_power_fast_phase_equals_exact(dgrain):
    """The device evaluates x^(4./3) in two phases (a float-seeded fast value kept only when
    its error interval rounds to one double, else the exact path); the host compiles the
    exact path alone.  On 4 million seeded depths, both ends of the fast domain and the
    rare fallback arguments included, the two agree bit for bit."""
    import ctypes as C

    from test_adjoint_cores import LIB as CORES_LIB, _build as build_cores

    rng = np.random.default_rng(2024)
    n = 1 << 20
    x = np.concatenate([
        np.exp(rng.uniform(np.log(1e-6), np.log(1e3), n)),          # depths of the runs
        1e-3 + rng.uniform(-2e-5, 2e-5, n),                          # around the wet/dry film H0
        np.exp(rng.uniform(-90.0, 90.0, n)),                         # across the fast domain's ends
        rng.uniform(0.5, 20.0, n),
        np.array([2.0 ** -120, np.nextafter(2.0 ** -120, 0), 2.0 ** 120, np.nextafter(2.0 ** 120, 0),
                  1e-200, 1e200, 1.0, 8.0, 27.0, 0.125]),
    ])
    y = np.empty_like(x)
    lib = dgrain.load()
    assert lib.dgr_pow43_batch(x.ctypes.data_as(dgrain._lib.dptr), y.ctypes.data_as(dgrain._lib.dptr),
                               len(x), 0) == 0
    build_cores()
    host = C.CDLL(CORES_LIB)
    dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
    host.dgr_t_pow43.argtypes = [dp, dp, C.c_int]
    want = np.empty_like(x)
    host.dgr_t_pow43(x, want, len(x))
    bad = np.flatnonzero(y != want)
    assert bad.size == 0, (bad.size, x[bad[:5]], y[bad[:5]], want[bad[:5]])


@pytest.mark.parametrize("seed", [1, 2])
def test_limiter_signed_zero_bounds(dgrain, oracle_mod, seed):
    """Node bounds that are zeros of either sign: the device limiter keeps the sign of the
    first zero mean in element order and clamps as the reference build does (its fmax
    returns the second operand on a tie), bit for bit with the oracle."""
    m = dgrain.rectangle(60, 30, jitter=0.1, seed=13)
    st = signed_zero_state(dgrain, m, seed, nx=60)
    s, o = make_pair(dgrain, oracle_mod, m, st)
    s.SlopeLimiter()
    o.slope_limiter()
    got, want = s.download_state(), o.get_state()
    for a, b in zip(got, want):
        assert same(a, b)
    assert negative_zeros(want[1]) > 0
    s.close()


def _division_cases(n, seed):
    """operand pairs for the shared-reciprocal division: random within its valid range,
    exact and near-exact quotients, all-ones divisors, quotients near powers of two,
    zeros of both signs, and the sizes of the RT0 fits"""
    rng = np.random.default_rng(seed)

    def rand(k, lo, hi):
        m = rng.integers(0, 1 << 52, k, dtype=np.uint64)
        e = rng.integers(lo, hi + 1, k).astype(np.uint64) + np.uint64(1023)
        s = rng.integers(0, 2, k).astype(np.uint64) << np.uint64(63)
        return (s | (e << np.uint64(52)) | m).view(np.float64)

    k = n // 6
    b = rand(6 * k, -100, 100)
    a = np.empty(6 * k)
    a[:k] = rand(k, -900, 900)
    a[k:2 * k] = b[k:2 * k] * rng.integers(-2048, 2048, k)
    near = (rand(k, -20, 20) * b[2 * k:3 * k]).view(np.int64) + rng.integers(-2, 3, k)
    a[2 * k:3 * k] = near.view(np.float64)
    b[3 * k:4 * k] = np.where(rng.random(k) < 0.5, 1.0, -1.0) * np.ldexp(
        np.nextafter(2.0, 0.0), rng.integers(-100, 100, k))
    a[3 * k:4 * k] = rand(k, -100, 100)
    a[4 * k:5 * k] = np.where(rng.random(k) < 0.5, -0.0, 0.0)
    a[5 * k:] = rand(k, -40, 15)
    b[5 * k:] = rand(k, -10, 10)
    return np.ascontiguousarray(a), np.ascontiguousarray(b)


def test_shared_reciprocal_division_on_device(dgrain):
    """The element kernel's divisions by the fit determinant (one reciprocal per element and
    Markstein's correction) equal the IEEE division bit for bit, on 6 million pairs."""
    a, b = _division_cases(6_000_000, 11)
    q = np.empty_like(a)
    valid = np.empty(len(a), dtype=np.int32)
    lib = dgrain.load()
    dp, ip = dgrain._lib.dptr, dgrain._lib.iptr
    assert lib.dgr_div_rcp_batch(a.ctypes.data_as(dp), b.ctypes.data_as(dp), q.ctypes.data_as(dp),
                                 valid.ctypes.data_as(ip), len(a), 0) == 0
    v = valid == 1
    assert v.mean() > 0.99
    with np.errstate(all="ignore"):
        assert bits_equal(q[v], (a / b)[v])
