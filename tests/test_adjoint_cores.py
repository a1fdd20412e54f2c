"""Derivative cores of the adjoint, on the CPU: the forward arithmetic of one edge, element or
limiter pass (dgr_scheme.cuh) in dual numbers (the tangent-linear model) against the
hand-written reverse (dgr_reverse.cuh).

  * dot-product test: <J xd, yb> == <xd, J^T yb> to round-off, for random inputs covering
    every branch (wet/dry edge cases, boundary kinds and sentinels, RK modes, limiter clamps
    and redistribution, PDop mass and momentum branches);
  * finite differences: central differences agree with the tangent to 1e-6 where no
    decision changes within the step (one-sided differences agree).

The cores are compiled for the host from the library's own headers (tests/cores_host.cu)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "cores_host.cu")
CSRC = os.path.join(HERE, "..", "dg-rain_b200", "csrc")
LIB = os.path.join(HERE, "_build", "libdgr_cores_host.so")
G = 9.81
H0 = 1e-3
VELZERO = 1e-10

dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def _build():
    deps = [SRC] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(d) for d in deps):
        return
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-x", "c++", "-D__host__=", "-D__device__=",
                    "-D__forceinline__=inline", "-o", LIB, SRC], check=True)


@pytest.fixture(scope="module")
def cores():
    _build()
    lib = C.CDLL(LIB)
    d = C.c_double
    lib.dgr_t_set_flux.argtypes = [C.c_int]
    lib.dgr_t_pow43.argtypes = [dp, dp, C.c_int]
    lib.dgr_t_roe.argtypes = [dp, d, d, d, d, dp, dp, dp, dp, dp]
    lib.dgr_t_edge.argtypes = [C.c_int] * 5 + [d, d, dp, d, d, d, dp, dp, dp, dp, dp]
    lib.dgr_t_element.argtypes = ([C.c_int, dp, dp, dp, d, d, d, d, d] + [dp] * 7 + [d, dp, dp, dp, dp, dp, dp, dp,
                                                                                    dp])
    lib.dgr_t_limit.argtypes = [C.c_int, dp, dp, dp, dp, d, d, dp, dp, dp, dp, dp, dp, dp, dp, dp, dp, dp, ip]
    return lib


def _dot_ok(yd, yb, xd, xb, tol=1e-12):
    """<yd, yb> == <xd, xb> relative to the larger side, or, when both sides are round-off
    (a derivative that vanishes identically, e.g. the mirrored dry-dry flux), to the scale
    |xd| |yb| of an O(1) Jacobian"""
    a, b = yd @ yb, xd @ xb
    return abs(a - b) <= tol * max(abs(a), abs(b)) + 1e-13 * np.linalg.norm(xd) * np.linalg.norm(yb)


# --------------------------------------------------------------------------- Roe ---

def _roe_inputs(rng):
    z_edge = rng.uniform(0.5, 4.0)
    h = rng.uniform(0.2, 3.0, 2)
    x = np.array([h[0] - z_edge, h[1] - z_edge, *rng.uniform(-2, 2, 4), z_edge])
    x = x[[0, 1, 2, 3, 4, 5, 6]]
    th = rng.uniform(0, 2 * np.pi)
    return x, np.cos(th), np.sin(th)


def _roe(cores, x, nx, ny, lg, xd=None, yb=None):
    xd = np.zeros(7) if xd is None else xd
    yb = np.zeros(3) if yb is None else yb
    y, yd, xb = np.zeros(3), np.zeros(3), np.zeros(7)
    cores.dgr_t_roe(x, nx, ny, lg, G, xd, yb, y, yd, xb)
    return y, yd, xb


@pytest.fixture(params=[0, 1, 2], ids=["roe", "llf", "hllc"])
def flux(request, cores):
    """numerical flux of the edge cases: the Roe flux of 2DCode, the local Lax-Friedrichs
    and HLLC fluxes of DG-SWEM"""
    cores.dgr_t_set_flux(request.param)
    yield request.param
    cores.dgr_t_set_flux(0)


@pytest.mark.parametrize("lg", [G, 0.0])
def test_roe_dot_product(cores, flux, lg):
    rng = np.random.default_rng(1)
    for _ in range(400):
        x, nx, ny = _roe_inputs(rng)
        xd, yb = rng.normal(size=7), rng.normal(size=3)
        _, yd, xb = _roe(cores, x, nx, ny, lg, xd, yb)
        assert _dot_ok(yd, yb, xd, xb), (x, nx, ny)


def _fd_check(f, x, xd, yd, rel=1e-6, h=1e-6):
    """central difference of f along xd against yd, to rel of the tangent plus the
    difference's own round-off (eps |f| / step); None when a kink lies within the step
    (the one-sided differences disagree)"""
    s = h * max(1.0, np.max(np.abs(x)))
    fp, f0, fm = f(x + s * xd), f(x), f(x - s * xd)
    fwd, bwd = (fp - f0) / s, (f0 - fm) / s
    scale = max(np.max(np.abs(yd)), 1e-8)
    noise = 20 * np.finfo(float).eps * max(np.max(np.abs(f0)), 1.0) / s
    if np.max(np.abs(fwd - bwd)) > 1e-3 * scale + noise:
        return None
    cen = (fp - fm) / (2 * s)
    return np.max(np.abs(cen - yd)) <= rel * scale + noise


def test_roe_tangent_matches_finite_differences(cores, flux):
    rng = np.random.default_rng(2)
    checked = 0
    for _ in range(200):
        x, nx, ny = _roe_inputs(rng)
        xd = rng.normal(size=7)
        _, yd, _ = _roe(cores, x, nx, ny, G, xd)
        ok = _fd_check(lambda xx: _roe(cores, xx, nx, ny, G)[0], x, xd, yd)
        if ok is None:
            continue
        assert ok
        checked += 1
    assert checked > 150


# -------------------------------------------------------------------------- edges ---

EDGE_CASES = [  # (wd_on, kind, bd, wdi, wde, bz, bq)
    (0, 0, 0, 1, 1, 0, 0),
    (1, 0, 0, 1, 1, 0, 0),
    (1, 0, 0, 0, 1, 0, 0),
    (1, 0, 0, 1, 0, 0, 0),
    (1, 0, 0, 0, 0, 0, 0),
    (1, 1, 0, 1, 1, 0, 0),
    (1, 1, 0, 0, 0, 0, 0),
    (1, 2, 2, 1, 1, 0.3, 1e6),
    (1, 2, 2, 1, 1, -1000.0, 1e6),
    (1, 2, 1, 1, 1, 0.2, 0.5),
    (1, 2, 2, 0, 0, 0.3, 1e6),
]


def _edge(cores, case, x, nx, ny, xd=None, yb=None):
    wd_on, kind, bd, wdi, wde, bz, bq = case
    xd = np.zeros(7) if xd is None else xd
    yb = np.zeros(6) if yb is None else yb
    y, yd, xb = np.zeros(6), np.zeros(6), np.zeros(7)
    cores.dgr_t_edge(wd_on, kind, bd, wdi, wde, bz, bq, x, nx, ny, G, xd, yb, y, yd, xb)
    return y, yd, xb


def _edge_inputs(rng):
    z_edge = rng.uniform(0.5, 4.0)
    h = rng.uniform(0.2, 3.0, 2)
    x = np.array([h[0] - z_edge, *rng.uniform(-2, 2, 2), h[1] - z_edge, *rng.uniform(-2, 2, 2), z_edge])
    th = rng.uniform(0, 2 * np.pi)
    return x, np.cos(th), np.sin(th)


@pytest.mark.parametrize("case", EDGE_CASES)
def test_edge_dot_product_and_fd(cores, flux, case):
    rng = np.random.default_rng(3)
    checked = 0
    for _ in range(150):
        x, nx, ny = _edge_inputs(rng)
        xd, yb = rng.normal(size=7), rng.normal(size=6)
        if case[1]:
            xd[3:6] = 0.0  # boundary: the exterior slot is not an input
        _, yd, xb = _edge(cores, case, x, nx, ny, xd, yb)
        assert _dot_ok(yd, yb, xd, xb), (case, x)
        ok = _fd_check(lambda xx: _edge(cores, case, xx, nx, ny)[0], x, xd, yd)
        if ok is not None:
            assert ok, (case, x)
            checked += 1
    assert checked > 100


# ----------------------------------------------------------------------- elements ---

def _tri(rng):
    base = rng.uniform(0, 1000, 2)
    pts = base + np.array([[0, 0], [50, 0], [0, 50]]) + rng.uniform(-10, 10, (3, 2))
    return np.ascontiguousarray(pts[:, 0]), np.ascontiguousarray(pts[:, 1])


def _element(cores, mode, geom, p, lg, rain, dt, xd=None, wb=None):
    """p = concatenation F[9], S[9], U[9], zv[3], nel -> w[9]"""
    xv, yv = geom
    F, S, U, zv, nel = p[:9], p[9:18], p[18:27], p[27:30], p[30]
    xd = np.zeros(31) if xd is None else xd
    wb = np.zeros(9) if wb is None else wb
    w, wdot = np.zeros(9), np.zeros(9)
    Fb, Sb, Ub, zvb, nelb = np.zeros(9), np.zeros(9), np.zeros(9), np.zeros(3), np.zeros(1)
    cores.dgr_t_element(mode, xv, yv, np.ascontiguousarray(zv), nel, G, lg, rain, dt,
                        np.ascontiguousarray(F), np.ascontiguousarray(S), np.ascontiguousarray(U),
                        np.ascontiguousarray(xd[:9]), np.ascontiguousarray(xd[9:18]),
                        np.ascontiguousarray(xd[18:27]), np.ascontiguousarray(xd[27:30]), xd[30], wb, w, wdot,
                        Fb, Sb, Ub, zvb, nelb)
    return w, wdot, np.concatenate([Fb, Sb, Ub, zvb, nelb])


def _element_inputs(rng):
    zv = rng.uniform(1.0, 4.0, 3)
    midz = 0.5 * (zv + np.roll(zv, -1))
    S = np.concatenate([rng.uniform(0.1, 1.0, 3) - 0.0 * midz, rng.uniform(-1, 1, 6)])
    U = np.concatenate([rng.uniform(0.1, 1.0, 3), rng.uniform(-1, 1, 6)])
    F = rng.normal(size=9)
    return np.concatenate([F, S, U, zv, [rng.uniform(0.01, 0.08)]])


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("lg", [G, 0.0])
def test_element_dot_product_and_fd(cores, mode, lg):
    rng = np.random.default_rng(4 + mode)
    checked = 0
    for _ in range(120):
        geom = _tri(rng)
        p = _element_inputs(rng)
        xd, wb = rng.normal(size=31), rng.normal(size=9)
        if mode != 2:
            xd[18:27] = 0.0
        _, wdot, pb = _element(cores, mode, geom, p, lg, 1e-6, 0.7, xd, wb)
        assert _dot_ok(wdot, wb, xd, pb, 1e-11), (mode, lg)
        ok = _fd_check(lambda pp: _element(cores, mode, geom, pp, lg, 1e-6, 0.7)[0], p, xd, wdot)
        if ok is not None:
            assert ok
            checked += 1
    assert checked > 100


def test_element_friction_at_rest(cores):
    """zero discharge: the speed in the Manning term has no derivative, its product with
    the discharge does (0); tangent and adjoint stay finite and transposed"""
    rng = np.random.default_rng(9)
    geom = _tri(rng)
    p = _element_inputs(rng)
    p[12:18] = 0.0
    xd, wb = rng.normal(size=31), rng.normal(size=9)
    _, wdot, pb = _element(cores, 1, geom, p, G, 0.0, 0.5, xd, wb)
    assert np.all(np.isfinite(wdot)) and np.all(np.isfinite(pb))
    assert _dot_ok(wdot, wb, xd, pb, 1e-11)


# ----------------------------------------------------------------------- limiter ---

def _limit(cores, pdop, p, xd=None, wb=None):
    """p = w[9], bmax[9], bmin[9], zn[3]"""
    w, bmax, bmin, zn = (np.ascontiguousarray(a) for a in (p[:9], p[9:18], p[18:27], p[27:30]))
    xd = np.zeros(30) if xd is None else xd
    wb = np.zeros(9) if wb is None else wb
    out, outd, wbo, bxb, bnb, znb = (np.zeros(n) for n in (9, 9, 9, 9, 9, 3))
    dec = np.zeros(5, dtype=np.int32)
    cores.dgr_t_limit(pdop, w, bmax, bmin, zn, H0, VELZERO, np.ascontiguousarray(xd[:9]),
                      np.ascontiguousarray(xd[9:18]), np.ascontiguousarray(xd[18:27]),
                      np.ascontiguousarray(xd[27:30]), wb, out, outd, wbo, bxb, bnb, znb, dec)
    return out, outd, np.concatenate([wbo, bxb, bnb, znb]), dec


def _limit_inputs(rng, regime):
    """regime 0: wet, limiter active; 1: near dry (PDop mass and momentum branches)"""
    zn = rng.uniform(0.2, 2.0, 3) if regime == 0 else rng.uniform(-0.05, 0.05, 3)
    w = np.zeros(9)
    if regime == 0:
        w[:3] = rng.uniform(-0.1, 0.1, 3)
    else:
        w[:3] = rng.uniform(-0.02, 0.03, 3) + 0.5 * H0
    w[3:] = rng.uniform(-0.5, 0.5, 6)
    # vertex values and bounds around them, some tight enough to clamp
    vx = np.stack([w[3 * v] - w[3 * v + 1] + w[3 * v + 2] for v in range(3)])
    bmax, bmin = np.zeros(9), np.zeros(9)
    for v in range(3):
        wv = w[3 * v:3 * v + 3]
        verts = np.array([wv[0] - wv[1] + wv[2], wv[0] + wv[1] - wv[2], -wv[0] + wv[1] + wv[2]])
        avg = wv.mean()
        spread = np.abs(verts - avg).max() + 1e-3
        bmax[3 * v:3 * v + 3] = avg + rng.uniform(0.2, 1.5, 3) * spread
        bmin[3 * v:3 * v + 3] = avg - rng.uniform(0.2, 1.5, 3) * spread
    del vx
    return np.concatenate([w, bmax, bmin, zn])


@pytest.mark.parametrize("pdop", [0, 1])
def test_limiter_dot_product_and_fd(cores, pdop):
    rng = np.random.default_rng(11 + pdop)
    seen = set()
    checked = 0
    for it in range(600):
        p = _limit_inputs(rng, it % 2)
        xd, wb = rng.normal(size=30), rng.normal(size=9)
        _, outd, pb, dec = _limit(cores, pdop, p, xd, wb)
        assert dec[4] == 1  # the reverse took the forward's branches
        seen.add((int(dec[0]), int(dec[1]), int(dec[2])))
        if dec[3]:
            continue  # NaN branch: no derivative
        assert _dot_ok(outd, wb, xd, pb, 1e-11), (p, dec)
        ok = _fd_check(lambda pp: _limit(cores, pdop, pp)[0], p, xd, outd, h=1e-9)
        if ok is not None:
            assert ok, (p, dec)
            checked += 1
    assert checked > 300
    assert any(s[0] == 1 for s in seen)  # limited elements
    if pdop:
        for b in (1, 2):
            assert any(s[1] == b for s in seen), seen  # PDop mass branches
            assert any(s[2] == b for s in seen), seen  # PDop momentum branches


def _hllc_branch(x, nx, ny, g=G):
    """HLLC branch of DG-SWEM's order (0 in, 1 in star, 2 ex star, 3 ex) for x = (zin, zex,
    qxin, qxex, qyin, qyex, zedge)"""
    h_in, h_ex = x[0] + x[6], x[1] + x[6]
    un_in = (x[2] * nx + x[4] * ny) / h_in
    un_ex = (x[3] * nx + x[5] * ny) / h_ex
    c_in, c_ex = np.sqrt(g * h_in), np.sqrt(g * h_ex)
    hs = (0.5 * (c_in + c_ex) + 0.25 * (un_in - un_ex)) ** 2 / g
    l_in = np.sqrt((hs * hs + hs * h_in) / (2 * h_in * h_in)) if hs > h_in else 1.0
    l_ex = np.sqrt((hs * hs + hs * h_ex) / (2 * h_ex * h_ex)) if hs > h_ex else 1.0
    s_in, s_ex = un_in - c_in * l_in, un_ex + c_ex * l_ex
    a, b = un_ex - s_ex, un_in - s_in
    s_st = (s_in * h_ex * a - s_ex * h_in * b) / (h_ex * a - h_in * b)
    return 0 if s_in >= 0 else (1 if s_st >= 0 else (2 if s_ex >= 0 else 3))


def test_hllc_inputs_cover_every_branch():
    """the random inputs of the flux tests reach all four HLLC branches"""
    rng = np.random.default_rng(1)
    seen = set()
    for _ in range(400):
        x, nx, ny = _roe_inputs(rng)
        seen.add(_hllc_branch(x, nx, ny))
    assert seen == {0, 1, 2, 3}, seen


def test_host_manning_power_is_correctly_rounded(cores):
    """pow43 as the host compiles it against the 60-digit decimal values of the golden file;
    the device's two-phase evaluation is checked against this one (test_gpu_parity)."""
    g = np.load(os.path.join(HERE, "golden", "pow43_cr.npz"))
    x = np.ascontiguousarray(g["x"])
    y = np.empty_like(x)
    cores.dgr_t_pow43(x, y, len(x))
    assert np.array_equal(y, g["cr"])


def test_manning_power_fast_phase_error_analysis(tmp_path):
    """The device's fast phase of x^(4./3), restated with host stand-ins for its float
    intrinsics (tests/pow43_sim.c), with the seed and the log pushed to the ends of their
    error bounds: every value its rounding test keeps equals the exact phase's."""
    exe = str(tmp_path / "pow43_sim")
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-o", exe, os.path.join(HERE, "pow43_sim.c"), "-lm"],
                   check=True)
    res = subprocess.run([exe, "2000000"], capture_output=True, text=True)
    assert res.returncode == 0, res.stdout
    lines = res.stdout.strip().splitlines()
    assert len(lines) == 3 and all(" 0 differ" in ln for ln in lines), lines


def test_shared_reciprocal_division_is_ieee_division(tmp_path):
    """div_rcp (the element kernel's divisions by the fit determinant through one shared
    reciprocal and Markstein's correction) equals the IEEE division bit for bit wherever it
    reports itself valid, on 4 million seeded operand pairs: random, exact and near-exact
    quotients, all-ones and one-bit divisors, quotients near powers of two, the edges of its
    valid range, signed zeros, and the sizes the fits meet."""
    lib_path = str(tmp_path / "libdiv_host.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-x", "c++",
                    "-D__host__=", "-D__device__=", "-D__forceinline__=inline", "-o", lib_path,
                    os.path.join(HERE, "div_host.cpp")], check=True)
    lib = C.CDLL(lib_path)
    lib.dgr_t_div_rcp.restype = C.c_longlong
    lib.dgr_t_div_rcp.argtypes = [C.c_longlong, C.c_ulonglong, C.POINTER(C.c_longlong)]
    valid = C.c_longlong()
    bad = lib.dgr_t_div_rcp(4_000_000, 20240917, C.byref(valid))
    assert bad == 0
    assert valid.value > 3_900_000
