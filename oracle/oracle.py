"""ORACLE — test infrastructure only.

ctypes bindings of
  * oracle/_build/liboracle.so  — the C restatement (dgr_oracle.c), and
  * oracle/_ref/libref2d.so / libref2d_wd.so — the unmodified reference 2DCode built by
    oracle/Makefile (present only where the reference tree was available at build time),
  * oracle/_ref/librefchan.so — the unmodified ChanNet/internal_BC.c (channel coupling).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref2d.so")
REF_LIB_WD = os.path.join(HERE, "_ref", "libref2d_wd.so")
REF_LIB_WD_O3 = os.path.join(HERE, "_ref", "libref2d_wd_o3.so")  # -O3 -march=x86-64-v3, timing only
REF_CHAN_LIB = os.path.join(HERE, "_ref", "librefchan.so")

dptr = C.POINTER(C.c_double)
iptr = C.POINTER(C.c_int)


def _d(a):
    return a.ctypes.data_as(dptr)


def _i(a):
    return a.ctypes.data_as(iptr)


# Where the reference tree is mounted in the build container (DGR_REFERENCE overrides it);
# hosts without it build the restatement only and use the prebuilt reference files.
REFERENCE_TREE = os.environ.get("DGR_REFERENCE", "/root/reference")


def build() -> None:
    """make -C oracle (restatement always; the reference only where its tree exists)."""
    cmd = ["make", "-s", "-C", HERE]
    ref2d = os.path.join(REFERENCE_TREE, "2DCode")
    if os.path.exists(os.path.join(ref2d, "compute2DL.c")):
        cmd.append(f"REF={ref2d}")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + res.stdout + res.stderr)


def have_reference() -> bool:
    return os.path.exists(REF_LIB) and os.path.exists(REF_LIB_WD)


# --------------------------------------------------------------------------- restatement --

_olib = None


def _oracle_lib():
    global _olib
    if _olib is None:
        if not os.path.exists(ORACLE_LIB):
            build()
        lib = C.CDLL(ORACLE_LIB)
        lib.orc_create.restype = C.c_void_p
        lib.orc_create.argtypes = [C.c_int, C.c_int, C.c_int, dptr, dptr, dptr, dptr, iptr, iptr, iptr, iptr, C.c_double]
        lib.orc_destroy.argtypes = [C.c_void_p]
        lib.orc_set_constants.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double]
        lib.orc_set_element_manning.argtypes = [C.c_void_p, dptr]
        lib.orc_set_state.argtypes = [C.c_void_p, dptr, dptr, dptr, iptr]
        lib.orc_get_state.argtypes = [C.c_void_p, dptr, dptr, dptr, iptr]
        lib.orc_set_bc.argtypes = [C.c_void_p, dptr, dptr]
        lib.orc_get_bc.argtypes = [C.c_void_p, dptr, dptr]
        lib.orc_get_rhs.argtypes = [C.c_void_p, dptr, dptr, dptr]
        lib.orc_get_fhat.argtypes = [C.c_void_p, dptr, dptr, dptr]
        lib.orc_max_lambda.restype = C.c_double
        lib.orc_max_lambda.argtypes = [C.c_void_p]
        lib.orc_last_error.argtypes = [C.c_void_p, iptr, iptr]
        lib.orc_initial_state.argtypes = [C.c_void_p, dptr]
        lib.orc_get_decisions.argtypes = [C.c_void_p, iptr, iptr]
        lib.orc_boundary_conditions.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_double, C.c_double]
        lib.orc_compute_L.argtypes = [C.c_void_p, C.c_int, C.c_double]
        lib.orc_slope_limiter.argtypes = [C.c_void_p]
        lib.orc_pdop.argtypes = [C.c_void_p]
        lib.orc_wd_status.argtypes = [C.c_void_p]
        lib.orc_roe_flux.restype = C.c_double
        lib.orc_roe_flux.argtypes = [dptr] + [C.c_double] * 11
        lib.orc_inner_products.argtypes = [C.c_void_p, C.c_int, dptr, dptr]
        lib.orc_step.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_double, iptr, iptr, iptr, iptr]
        lib.orc_run.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, C.c_double,
                                C.c_int, C.c_double, C.c_double, dptr, dptr, dptr, iptr]
        lib.orc_run_rk.argtypes = lib.orc_run.argtypes + [C.c_int]
        lib.orc_internal_bc.argtypes = _INTERNAL_BC_ARGS
        _olib = lib
    return _olib


_INTERNAL_BC_ARGS = ([C.c_int, C.c_int, dptr, dptr, dptr, iptr, iptr, iptr, dptr, dptr, dptr, dptr, dptr, C.c_int]
                     + [iptr] * 6 + [dptr, dptr])
_clib = None


def have_reference_coupling() -> bool:
    return os.path.exists(REF_CHAN_LIB)


def internal_bc(mesh, zeta, qx, qy, bzeta, bqn, channels, reference=False, repeats=0):
    """ChanNet/internal_BC.c on one junction mesh, by the restatement (dgr_oracle.c) or by the
    reference build.  zeta/qx/qy: reference layout [3*el+k]; bzeta/bqn [nf] (copied);
    channels: list of (A, Q, inflow_edges, outflow_edges), A and Q the channel's traces
    (2 per node, copied).  Returns (bzeta, bqn, [(A, Q)...]) after the coupling pass; with
    repeats > 0 the pass runs that many more times on the same inputs and the seconds per
    pass of the C call alone come last."""
    global _clib
    if reference:
        if _clib is None:
            _clib = C.CDLL(REF_CHAN_LIB, mode=os.RTLD_LOCAL)
            _clib.ref_internal_bc.argtypes = _INTERNAL_BC_ARGS
            _clib.ref_internal_bc.restype = C.c_int
        fn = _clib.ref_internal_bc
    else:
        fn = _oracle_lib().orc_internal_bc
        fn.restype = C.c_int
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)  # noqa: E731
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)  # noqa: E731
    nodes = i32([len(c[0]) // 2 for c in channels])
    off = i32(np.concatenate([[0], np.cumsum(nodes)[:-1]]) if len(channels) else [0])
    A = f64(np.concatenate([c[0] for c in channels]) if channels else [0.0])
    Q = f64(np.concatenate([c[1] for c in channels]) if channels else [0.0])
    in_ptr = i32(np.concatenate([[0], np.cumsum([len(c[2]) for c in channels])]))
    out_ptr = i32(np.concatenate([[0], np.cumsum([len(c[3]) for c in channels])]))
    in_e = i32(np.concatenate([np.asarray(c[2], dtype=np.int32) for c in channels] + [np.zeros(1, np.int32)]))
    out_e = i32(np.concatenate([np.asarray(c[3], dtype=np.int32) for c in channels] + [np.zeros(1, np.int32)]))
    bz, bq = f64(bzeta).copy(), f64(bqn).copy()
    zt, qxx, qyy = f64(zeta), f64(qx), f64(qy)
    x, y, z = f64(mesh.x), f64(mesh.y), f64(mesh.z)
    el2v, ed2v, ed2el = i32(mesh.el2v.ravel()), i32(mesh.ed2v.ravel()), i32(mesh.ed2el.ravel())
    args = (mesh.num_el, mesh.num_edges, _d(x), _d(y), _d(z), _i(el2v), _i(ed2v), _i(ed2el), _d(zt), _d(qxx),
            _d(qyy), _d(bz), _d(bq), len(channels), _i(in_ptr), _i(in_e), _i(out_ptr), _i(out_e), _i(nodes),
            _i(off), _d(A), _d(Q))
    rc = fn(*args)
    if rc != 0:
        raise ValueError("internal_bc: bad coupled edge")
    out, o = [], 0
    for n in nodes:
        out.append((A[2 * o:2 * (o + n)].copy(), Q[2 * o:2 * (o + n)].copy()))
        o += n
    if repeats > 0:
        import time

        t0 = time.perf_counter()
        for _ in range(repeats):
            fn(*args)
        return bz, bq, out, (time.perf_counter() - t0) / repeats
    return bz, bq, out


class Oracle:
    """The C restatement on one mesh (arrays in the reference layout)."""

    def __init__(self, mesh, n_el=None):
        self.lib = _oracle_lib()
        self.ne, self.nn, self.nf = mesh.num_el, mesh.num_nodes, mesh.num_edges
        self.h = self.lib.orc_create(self.ne, self.nn, self.nf, _d(mesh.x), _d(mesh.y), _d(mesh.z), _d(mesh.nfric),
                                     _i(mesh.el2v), _i(mesh.ed2el), _i(mesh.ed2v), _i(mesh.bdry), mesh.min_edge)
        self.min_edge = mesh.min_edge
        if n_el is not None:
            self.set_element_manning(n_el)

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_element_manning(self, n_el):
        if n_el is None:
            self.lib.orc_set_element_manning(self.h, None)
        else:
            self._nel = np.ascontiguousarray(n_el, dtype=np.float64)
            self.lib.orc_set_element_manning(self.h, _d(self._nel))

    def set_state(self, zeta, qx, qy, wd=None):
        z, x, y = (np.ascontiguousarray(a, dtype=np.float64) for a in (zeta, qx, qy))
        w = None if wd is None else np.ascontiguousarray(wd, dtype=np.int32)
        self.lib.orc_set_state(self.h, _d(z), _d(x), _d(y), None if w is None else _i(w))

    def get_state(self):
        z, x, y = (np.empty(3 * self.ne) for _ in range(3))
        w = np.empty(self.ne, dtype=np.int32)
        self.lib.orc_get_state(self.h, _d(z), _d(x), _d(y), _i(w))
        return z, x, y, w

    def set_bc(self, bz, bq):
        bz, bq = (np.ascontiguousarray(a, dtype=np.float64) for a in (bz, bq))
        self.lib.orc_set_bc(self.h, _d(bz), _d(bq))

    def get_bc(self):
        bz, bq = np.empty(self.nf), np.empty(self.nf)
        self.lib.orc_get_bc(self.h, _d(bz), _d(bq))
        return bz, bq

    def boundary_conditions(self, t=0.0, tide_on=0, amp=0.0, period=44712.0):
        self.lib.orc_boundary_conditions(self.h, t, tide_on, amp, period)

    def compute_L(self, wet_dry, rain=0.0):
        rc = self.lib.orc_compute_L(self.h, wet_dry, rain)
        r = [np.empty(3 * self.ne) for _ in range(3)]
        self.lib.orc_get_rhs(self.h, *[_d(a) for a in r])
        return rc, r[0], r[1], r[2], self.lib.orc_max_lambda(self.h)

    def fhat(self):
        f = [np.empty(3 * self.ne) for _ in range(3)]
        self.lib.orc_get_fhat(self.h, *[_d(a) for a in f])
        return f

    def slope_limiter(self):
        return self.lib.orc_slope_limiter(self.h)

    def pdop(self):
        return self.lib.orc_pdop(self.h)

    def wd_status(self):
        self.lib.orc_wd_status(self.h)

    def decisions(self):
        lim = np.empty(self.ne, dtype=np.int32)
        pd = np.empty(self.ne, dtype=np.int32)
        self.lib.orc_get_decisions(self.h, _i(lim), _i(pd))
        return lim, pd

    def last_error(self):
        c, i = C.c_int(), C.c_int()
        self.lib.orc_last_error(self.h, C.byref(c), C.byref(i))
        return c.value, i.value

    def step(self, time, dt, wet_dry=1, rain=0.0, want_decisions=False):
        if want_decisions:
            d = [np.zeros(self.ne, dtype=np.int32) for _ in range(4)]
            rc = self.lib.orc_step(self.h, time, dt, wet_dry, rain, *[_i(a) for a in d])
            return rc, d
        rc = self.lib.orc_step(self.h, time, dt, wet_dry, rain, None, None, None, None)
        return rc, None

    def max_lambda(self):
        return self.lib.orc_max_lambda(self.h)

    def run(self, nsteps, final_time, cfl, dt0=1e-7, wet_dry=1, rain=0.0, tide_on=0, amp=0.0, period=44712.0,
            time=-1.0, dt=0.0, want_dt=False, rk_stages=2):
        t, d, n = C.c_double(time), C.c_double(dt), C.c_int(0)
        hist = np.zeros(max(nsteps, 1)) if want_dt else None
        rc = self.lib.orc_run_rk(self.h, nsteps, final_time, cfl, dt0, wet_dry, rain, tide_on, amp, period,
                                 C.byref(t), C.byref(d), None if hist is None else _d(hist), C.byref(n), rk_stages)
        return rc, t.value, d.value, n.value, (hist[: n.value] if hist is not None else None)


# ------------------------------------------------------------------ compiled reference --

class Reference:
    """The unmodified reference 2DCode (process-wide globals: one mesh per library).
    wet_dry selects the -DWDON build (compute2DL's wet/dry flux branch)."""

    _libs: dict = {}

    def __init__(self, wet_dry: bool, optimised: bool = False):
        path = (REF_LIB_WD_O3 if optimised else REF_LIB_WD) if wet_dry else REF_LIB
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (the reference tree was not available)")
        if path not in Reference._libs:
            lib = C.CDLL(path, mode=os.RTLD_LOCAL)
            lib.ref_load_fort14.argtypes = [C.c_char_p]
            lib.ref_set_mesh.argtypes = [C.c_int, C.c_int, C.c_int, dptr, dptr, dptr, dptr, iptr, iptr, iptr, iptr,
                                         C.c_double]
            lib.ref_get_counts.argtypes = [iptr, iptr, iptr, dptr]
            lib.ref_get_mesh.argtypes = [dptr, dptr, dptr, dptr, iptr, iptr, iptr, iptr]
            lib.ref_set_state.argtypes = [dptr, dptr, dptr, iptr]
            lib.ref_get_state.argtypes = [dptr, dptr, dptr, iptr]
            lib.ref_get_rhs.argtypes = [dptr, dptr, dptr]
            lib.ref_get_fhat.argtypes = [dptr, dptr, dptr]
            lib.ref_set_bc.argtypes = [dptr, dptr]
            lib.ref_get_bc.argtypes = [dptr, dptr]
            lib.ref_max_lambda.restype = C.c_double
            lib.ref_compute2DL.argtypes = [C.c_double]
            lib.ref_roe_flux.restype = C.c_double
            lib.ref_roe_flux.argtypes = [dptr] + [C.c_double] * 10
            lib.ref_inner_products.argtypes = [C.c_int, dptr, dptr]
            lib.ref_step.argtypes = [C.c_double, C.c_double, C.c_int, C.c_double, C.c_int]
            lib.ref_run.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, C.c_double, C.c_int,
                                    C.c_double, C.c_double, dptr, dptr, dptr, iptr]
            lib.ref_time_evolution.argtypes = [C.c_double]
            lib.ref_last_message.restype = C.c_char_p
            Reference._libs[path] = lib
        self.lib = Reference._libs[path]
        self.wet_dry = wet_dry

    def load_fort14(self, path):
        rc = self.lib.ref_load_fort14(os.fsencode(path))
        if rc:
            raise RuntimeError("reference store_mesh/extract_mesh_attributes failed: " + self.message())
        self._counts()
        return rc

    def set_mesh(self, mesh):
        self.lib.ref_set_mesh(mesh.num_el, mesh.num_nodes, mesh.num_edges, _d(mesh.x), _d(mesh.y), _d(mesh.z),
                              _d(mesh.nfric), _i(mesh.el2v), _i(mesh.ed2el), _i(mesh.ed2v), _i(mesh.bdry),
                              mesh.min_edge)
        self._counts()

    def _counts(self):
        ne, nn, nf, me = C.c_int(), C.c_int(), C.c_int(), C.c_double()
        self.lib.ref_get_counts(C.byref(ne), C.byref(nn), C.byref(nf), C.byref(me))
        self.ne, self.nn, self.nf, self.min_edge = ne.value, nn.value, nf.value, me.value

    def get_mesh(self):
        x, y, z, n = (np.empty(self.nn) for _ in range(4))
        el2v = np.empty((self.ne, 3), dtype=np.int32)
        ed2el = np.empty((self.nf, 2), dtype=np.int32)
        ed2v = np.empty((self.nf, 2), dtype=np.int32)
        bdry = np.empty(self.nf, dtype=np.int32)
        self.lib.ref_get_mesh(_d(x), _d(y), _d(z), _d(n), _i(el2v), _i(ed2el), _i(ed2v), _i(bdry))
        return dict(x=x, y=y, z=z, nfric=n, el2v=el2v, ed2el=ed2el, ed2v=ed2v, bdry=bdry, min_edge=self.min_edge)

    def initialize(self):
        self.lib.ref_initialize()

    def set_state(self, zeta, qx, qy, wd=None):
        z, x, y = (np.ascontiguousarray(a, dtype=np.float64) for a in (zeta, qx, qy))
        w = None if wd is None else np.ascontiguousarray(wd, dtype=np.int32)
        self.lib.ref_set_state(_d(z), _d(x), _d(y), None if w is None else _i(w))

    def get_state(self):
        z, x, y = (np.empty(3 * self.ne) for _ in range(3))
        w = np.empty(self.ne, dtype=np.int32)
        self.lib.ref_get_state(_d(z), _d(x), _d(y), _i(w))
        return z, x, y, w

    def set_bc(self, bz, bq):
        bz, bq = (np.ascontiguousarray(a, dtype=np.float64) for a in (bz, bq))
        self.lib.ref_set_bc(_d(bz), _d(bq))

    def get_bc(self):
        bz, bq = np.empty(self.nf), np.empty(self.nf)
        self.lib.ref_get_bc(_d(bz), _d(bq))
        return bz, bq

    def boundary_conditions(self):
        return self.lib.ref_boundary_conditions()

    def compute2DL(self, time=0.0):
        rc = self.lib.ref_compute2DL(time)
        r = [np.empty(3 * self.ne) for _ in range(3)]
        self.lib.ref_get_rhs(*[_d(a) for a in r])
        return rc, r[0], r[1], r[2], self.lib.ref_max_lambda()

    def fhat(self):
        f = [np.empty(3 * self.ne) for _ in range(3)]
        self.lib.ref_get_fhat(*[_d(a) for a in f])
        return f

    def slope_limiter(self):
        return self.lib.ref_slope_limiter()

    def pdop(self):
        return self.lib.ref_pdop()

    def wd_status(self):
        return self.lib.ref_wd_status()

    def step(self, time, dt, rain=0.0, use_reference_step=False):
        return self.lib.ref_step(time, dt, 1 if self.wet_dry else 0, rain, 1 if use_reference_step else 0)

    def max_lambda(self):
        return self.lib.ref_max_lambda()

    def message(self):
        return self.lib.ref_last_message().decode(errors="replace")

    def run(self, nsteps, final_time, cfl, dt0=1e-7, rain=0.0, tide_on=0, amp=0.0, period=44712.0, time=-1.0,
            dt=0.0, want_dt=False):
        t, d, n = C.c_double(time), C.c_double(dt), C.c_int(0)
        hist = np.zeros(max(nsteps, 1)) if want_dt else None
        rc = self.lib.ref_run(nsteps, final_time, cfl, dt0, 1 if self.wet_dry else 0, rain, tide_on, amp, period,
                              C.byref(t), C.byref(d), None if hist is None else _d(hist), C.byref(n))
        return rc, t.value, d.value, n.value, (hist[: n.value] if hist is not None else None)

    def time_evolution(self, final_time):
        return self.lib.ref_time_evolution(final_time)
