"""Python mirror of the reference 2DCode call surface over the C ABI.

Method names follow the reference functions they replace (2DCode/compute2DL.c:12,
SlopeLimiter2D.c:10, wetDry2D.c:16 and :63, time_evolution.c:10 and :248,
boundary_conditions.c:9); arrays use the reference layout [3*el+k].  Where the reference
prints a message and exits, these methods raise StepError carrying the same code and the
edge or element index the reference would have printed.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .mesh import Mesh, _dp, _ip


class StepError(RuntimeError):
    def __init__(self, code: int, index: int, step: int, where: str):
        self.code, self.index, self.step = code, index, step
        super().__init__(f"{where}: {_lib.status_string(code)} (code {code}) at index {index}, step {step}")


def default_params(**overrides) -> _lib.DgrParams:
    p = _lib.DgrParams()
    _lib.check(_lib.load().dgr_params_default(C.byref(p)), "dgr_params_default")
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise KeyError(f"unknown parameter {k}")
        setattr(p, k, v)
    return p


class Solver:
    """One mesh on one GPU (a dgr_ctx)."""

    def __init__(self, mesh: Mesh, params: _lib.DgrParams | None = None, **overrides):
        self.lib = _lib.load()
        self.mesh = mesh
        self.params = params if params is not None else default_params(**overrides)
        self._view = mesh.view()
        h = C.c_void_p()
        _lib.check(self.lib.dgr_create(C.byref(self._view), C.byref(self.params), C.byref(h)), "dgr_create")
        self.ctx = h
        self.ne = mesh.num_el
        self.nf = mesh.num_edges
        self.nm = 6 if self.params.order == 2 else 3  # state coefficients per element and variable

    # ------------------------------------------------------------------ life ----
    def close(self) -> None:
        if self.ctx:
            self.lib.dgr_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, **kw) -> None:
        for k, v in kw.items():
            setattr(self.params, k, v)
        _lib.check(self.lib.dgr_set_params(self.ctx, C.byref(self.params)), "dgr_set_params")

    def set_element_manning(self, n_el: np.ndarray | None) -> None:
        if n_el is None:
            _lib.check(self.lib.dgr_set_element_manning(self.ctx, None), "dgr_set_element_manning")
            return
        n_el = np.ascontiguousarray(n_el, dtype=np.float64)
        assert n_el.shape == (self.ne,)
        _lib.check(self.lib.dgr_set_element_manning(self.ctx, _dp(n_el)), "dgr_set_element_manning")

    def set_bathymetry(self, z: np.ndarray) -> None:
        """Node depths (the fort.14 depth column); every depth-dependent factor is
        recomputed on the device."""
        z = np.ascontiguousarray(z, dtype=np.float64)
        assert z.shape == (self.mesh.num_nodes,)
        _lib.check(self.lib.dgr_set_bathymetry(self.ctx, _dp(z)), "dgr_set_bathymetry")

    # ----------------------------------------------------------------- state ----
    def upload_state(self, zeta, qx, qy, wd=None) -> None:
        z = np.ascontiguousarray(zeta, dtype=np.float64)
        x = np.ascontiguousarray(qx, dtype=np.float64)
        y = np.ascontiguousarray(qy, dtype=np.float64)
        assert z.shape == x.shape == y.shape == (self.nm * self.ne,)
        w = None if wd is None else np.ascontiguousarray(wd, dtype=np.int32)
        _lib.check(self.lib.dgr_upload_state(self.ctx, _dp(z), _dp(x), _dp(y), None if w is None else _ip(w)),
                   "dgr_upload_state")

    def download_state(self):
        z = np.empty(self.nm * self.ne)
        x = np.empty(self.nm * self.ne)
        y = np.empty(self.nm * self.ne)
        w = np.empty(self.ne, dtype=np.int32)
        _lib.check(self.lib.dgr_download_state(self.ctx, _dp(z), _dp(x), _dp(y), _ip(w)), "dgr_download_state")
        return z, x, y, w

    def set_gauges(self, gauge_el, gauge_w, capacity: int) -> None:
        """record the elevation at the gauges after every step of the device loop (up to
        `capacity` steps per run); gauge_el None removes them"""
        if gauge_el is None:
            _lib.check(self.lib.dgr_set_gauges(self.ctx, 0, None, None, 0), "dgr_set_gauges")
            self._gauges = None
            return
        el = np.ascontiguousarray(gauge_el, dtype=np.int32)
        w = np.ascontiguousarray(gauge_w, dtype=np.float64).reshape(len(el), self.nm)
        _lib.check(self.lib.dgr_set_gauges(self.ctx, len(el), _ip(el), _dp(w), int(capacity)), "dgr_set_gauges")
        self._gauges = (len(el), int(capacity))

    def gauge_series(self) -> np.ndarray:
        """[capacity, ngauges] values recorded by the last run"""
        ng, cap = self._gauges
        out = np.empty((cap, ng))
        _lib.check(self.lib.dgr_get_gauge_series(self.ctx, _dp(out)), "dgr_get_gauge_series")
        return out

    def save_restart(self, path, time: float, dt: float) -> None:
        """state, wet/dry flags and clock (time, next dt) to a restart file (dgr_save_restart)"""
        _lib.check(self.lib.dgr_save_restart(self.ctx, str(path).encode(), time, dt), "dgr_save_restart")

    def load_restart(self, path):
        """a restart file into this context; returns (time, dt) to continue with"""
        t, d = C.c_double(), C.c_double()
        _lib.check(self.lib.dgr_load_restart(self.ctx, str(path).encode(), C.byref(t), C.byref(d)),
                   "dgr_load_restart")
        return t.value, d.value

    def write_state_dat(self, zeta_path=None, qx_path=None, qy_path=None) -> None:
        """the current state as the reference's .dat snapshot files, formatted on the device"""
        enc = lambda p: None if p is None else str(p).encode()  # noqa: E731
        _lib.check(self.lib.dgr_write_state_dat(self.ctx, enc(zeta_path), enc(qx_path), enc(qy_path)),
                   "dgr_write_state_dat")

    def set_boundary(self, bzeta, bqn) -> None:
        bz = np.ascontiguousarray(bzeta, dtype=np.float64)
        bq = np.ascontiguousarray(bqn, dtype=np.float64)
        _lib.check(self.lib.dgr_set_boundary(self.ctx, _dp(bz), _dp(bq)), "dgr_set_boundary")

    def boundary_conditions(self, time: float = 0.0) -> None:
        _lib.check(self.lib.dgr_boundary_conditions(self.ctx, time), "dgr_boundary_conditions")

    def get_boundary(self):
        """(bzeta, bQn) of every edge as the device holds them"""
        bz, bq = np.empty(self.nf), np.empty(self.nf)
        _lib.check(self.lib.dgr_get_boundary(self.ctx, _dp(bz), _dp(bq)), "dgr_get_boundary")
        return bz, bq

    # ----------------------------------------------------- channel coupling ----
    def set_channel_ends(self, ends) -> None:
        """ends: list of (edges, outflow) — the mesh edges a channel end is attached to, in
        the order of the reference's junction-edge list, and whether it is the channel's
        last node (outflow, 1) or its first (inflow, 0); see dgr_set_channel_ends"""
        ptr = np.concatenate([[0], np.cumsum([len(e) for e, _ in ends])]).astype(np.int32)
        edges = np.ascontiguousarray(np.concatenate([np.asarray(e, dtype=np.int32) for e, _ in ends]
                                                    + [np.zeros(0, np.int32)]), dtype=np.int32)
        out = np.ascontiguousarray([int(o) for _, o in ends], dtype=np.int32)
        rc = self.lib.dgr_set_channel_ends(self.ctx, len(ends), _ip(ptr), _ip(edges if edges.size else ptr),
                                           _ip(out if out.size else ptr))
        _lib.check(rc, "dgr_set_channel_ends")
        self._nends = len(ends)

    def stream(self) -> int:
        """the context's cudaStream_t as an integer (torch.cuda.ExternalStream accepts it)"""
        s = C.c_void_p()
        _lib.check(self.lib.dgr_get_stream(self.ctx, C.byref(s)), "dgr_get_stream")
        return int(s.value or 0)

    def couple_channel_ends_device(self, a_end, q_end, a_ghost, q_ghost) -> None:
        """the coupling pass on device buffers (torch CUDA float64 tensors of the ends'
        count, or raw device addresses), enqueued on the solver's stream"""
        ptr = [int(t.data_ptr()) if hasattr(t, "data_ptr") else int(t) for t in (a_end, q_end, a_ghost, q_ghost)]
        _lib.check(self.lib.dgr_couple_channel_ends_device(self.ctx, *[C.c_void_p(p) for p in ptr]),
                   "dgr_couple_channel_ends_device")

    def couple_channel_ends(self, a_end, q_end):
        """one coupling pass (internal_BC): returns the ends' ghost (A, Q)"""
        n = getattr(self, "_nends", 0)
        a = np.ascontiguousarray(a_end, dtype=np.float64).reshape(n)
        q = np.ascontiguousarray(q_end, dtype=np.float64).reshape(n)
        ag, qg = np.empty(n), np.empty(n)
        if n:
            _lib.check(self.lib.dgr_couple_channel_ends(self.ctx, _dp(a), _dp(q), _dp(ag), _dp(qg)),
                       "dgr_couple_channel_ends")
        return ag, qg

    # ------------------------------------------------------------- operators ----
    def _status(self, rc: int, where: str) -> None:
        if rc == _lib.DGR_OK:
            return
        if 1 <= rc <= 7:
            code, index, step = C.c_int(), C.c_int(), C.c_int()
            self.lib.dgr_last_error(self.ctx, C.byref(code), C.byref(index), C.byref(step))
            raise StepError(code.value, index.value, step.value, where)
        _lib.check(rc, where)

    def compute2DL(self, time: float = 0.0):
        rz = np.empty(self.nm * self.ne)
        rx = np.empty(self.nm * self.ne)
        ry = np.empty(self.nm * self.ne)
        lam = C.c_double()
        self._status(self.lib.dgr_compute_L(self.ctx, time, _dp(rz), _dp(rx), _dp(ry), C.byref(lam)), "compute2DL")
        return rz, rx, ry, lam.value

    def SlopeLimiter(self) -> None:  # noqa: N802 (reference name)
        self._status(self.lib.dgr_slope_limiter(self.ctx), "SlopeLimiter")

    def PDop2D(self) -> None:  # noqa: N802
        self._status(self.lib.dgr_pdop(self.ctx), "PDop2D")

    def wetDryStatus2D(self) -> None:  # noqa: N802
        self._status(self.lib.dgr_wet_dry_status(self.ctx), "wetDryStatus2D")

    def oneTimeStep2D(self, time: float, dt: float) -> float:  # noqa: N802
        lam = C.c_double()
        self._status(self.lib.dgr_step(self.ctx, time, dt, C.byref(lam)), "oneTimeStep2D")
        return lam.value

    def time_evolution(self, final_time: float, nsteps: int, time: float = -1.0, dt: float = 0.0):
        """Device-resident loop; returns (time, next dt, steps done)."""
        t = C.c_double(time)
        d = C.c_double(dt)
        n = C.c_int(0)
        self._status(self.lib.dgr_run(self.ctx, nsteps, final_time, C.byref(t), C.byref(d), C.byref(n)),
                     "time_evolution")
        return t.value, d.value, n.value

    # ------------------------------------------------------------ diagnostics ----
    def last_error(self):
        code, index, step = C.c_int(), C.c_int(), C.c_int()
        _lib.check(self.lib.dgr_last_error(self.ctx, C.byref(code), C.byref(index), C.byref(step)),
                   "dgr_last_error")
        return code.value, index.value, step.value

    def decisions(self, stage: int):
        lim = np.empty(self.ne, dtype=np.int32)
        pd = np.empty(self.ne, dtype=np.int32)
        _lib.check(self.lib.dgr_get_decisions(self.ctx, stage, _ip(lim), _ip(pd)), "dgr_get_decisions")
        return lim, pd

    def fhat(self):
        f = [np.empty(3 * self.ne) for _ in range(3)]
        _lib.check(self.lib.dgr_get_fhat(self.ctx, *[_dp(a) for a in f]), "dgr_get_fhat")
        return tuple(f)

    def kernel_launches(self) -> int:
        return int(self.lib.dgr_kernel_launches(self.ctx))

    def last_device_ms(self) -> float:
        return float(self.lib.dgr_last_device_ms(self.ctx))

    def profile_step(self, nsteps: int = 3):
        """Average device ms per launch of (edge flux, element, node bounds, limiter)."""
        out = (C.c_double * 4)()
        self._status(self.lib.dgr_profile_step(self.ctx, nsteps, out, 4), "dgr_profile_step")
        return list(out)


def _schedule_methods(cls):
    """Schedule controls shared by Solver and Ensemble (dgr_set_schedule / dgr_autotune)."""

    def set_schedule(self, block_size: int = 64, fusion: int = 0) -> None:
        _lib.check(self.lib.dgr_set_schedule(self.ctx, block_size, fusion), "dgr_set_schedule")

    def get_schedule(self):
        b, f = C.c_int(), C.c_int()
        _lib.check(self.lib.dgr_get_schedule(self.ctx, C.byref(b), C.byref(f)), "dgr_get_schedule")
        return b.value, f.value

    def autotune(self, trial_steps: int = 5):
        """Times every schedule from the current state (restored afterwards) and keeps the
        fastest; returns (block_size, fusion, {(block_size, fusion): ms per step})."""
        b, f = C.c_int(), C.c_int()
        ms = (C.c_double * 9)()
        _lib.check(self.lib.dgr_autotune(self.ctx, trial_steps, C.byref(b), C.byref(f), ms), "dgr_autotune")
        table = {(bs, fu): ms[3 * i + fu] for i, bs in enumerate((64, 128, 256)) for fu in range(3)}
        return b.value, f.value, table

    def set_barrier_wait(self, max_polls: int = 1 << 24, phantom_blocks: int = 0) -> None:
        """Bound of the persistent kernels' grid-barrier wait; phantom_blocks = 1 makes the
        wait run out on purpose (DGR_ERR_TIMEOUT), a test of that path."""
        _lib.check(self.lib.dgr_set_barrier_wait(self.ctx, max_polls, phantom_blocks), "dgr_set_barrier_wait")

    cls.set_schedule = set_schedule
    cls.get_schedule = get_schedule
    cls.autotune = autotune
    cls.set_barrier_wait = set_barrier_wait
    return cls


_schedule_methods(Solver)


@_schedule_methods
class Ensemble:
    """Many meshes advanced together by one context (dgr_ensemble_*): each scenario with
    its own CFL dt, forcing and results, identical to running it alone."""

    def __init__(self, meshes, scenarios=None, **common):
        self.lib = _lib.load()
        self.meshes = list(meshes)
        n = len(self.meshes)
        self.params = default_params(**common)
        self.nm = 6 if self.params.order == 2 else 3  # state coefficients per element and variable
        self._views = (_lib.DgrMeshView * n)(*[m.view() for m in self.meshes])
        sp = (_lib.DgrScenarioParams * n)()
        self._keep = []
        for k in range(n):
            d = dict(tide_on=self.params.tide_on, tide_amp=self.params.tide_amp,
                     tide_period=self.params.tide_period, rain=self.params.rain, n_el=None)
            if scenarios is not None:
                d.update(scenarios[k])
            sp[k].tide_on, sp[k].tide_amp = int(d["tide_on"]), float(d["tide_amp"])
            sp[k].tide_period, sp[k].rain = float(d["tide_period"]), float(d["rain"])
            if d["n_el"] is not None:
                a = np.ascontiguousarray(d["n_el"], dtype=np.float64)
                assert a.shape == (self.meshes[k].num_el,)
                self._keep.append(a)
                sp[k].n_el = _dp(a)
        h = C.c_void_p()
        _lib.check(self.lib.dgr_ensemble_create(n, self._views, sp, C.byref(self.params), C.byref(h)),
                   "dgr_ensemble_create")
        self.ctx = h
        self.n = n
        # flattened numbering: scenario s's element i is el_off[s] + i (nodes likewise)
        self.el_off = np.concatenate([[0], np.cumsum([m.num_el for m in self.meshes])]).astype(np.int64)
        self.nd_off = np.concatenate([[0], np.cumsum([m.num_nodes for m in self.meshes])]).astype(np.int64)
        self.ne = int(self.el_off[-1])
        self.nn = int(self.nd_off[-1])

    def close(self) -> None:
        if self.ctx:
            self.lib.dgr_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload_state(self, s: int, zeta, qx, qy, wd=None) -> None:
        ne = self.meshes[s].num_el
        z, x, y = (np.ascontiguousarray(a, dtype=np.float64) for a in (zeta, qx, qy))
        assert z.shape == x.shape == y.shape == (self.nm * ne,)
        w = None if wd is None else np.ascontiguousarray(wd, dtype=np.int32)
        _lib.check(self.lib.dgr_ensemble_upload_state(self.ctx, s, _dp(z), _dp(x), _dp(y),
                                                      None if w is None else _ip(w)), "dgr_ensemble_upload_state")

    def download_state(self, s: int):
        ne = self.meshes[s].num_el
        z, x, y = np.empty(self.nm * ne), np.empty(self.nm * ne), np.empty(self.nm * ne)
        w = np.empty(ne, dtype=np.int32)
        _lib.check(self.lib.dgr_ensemble_download_state(self.ctx, s, _dp(z), _dp(x), _dp(y), _ip(w)),
                   "dgr_ensemble_download_state")
        return z, x, y, w

    def run(self, nsteps: int, final_time=1e300, time=None, dt=None, check=True):
        """Advances every scenario up to nsteps steps; returns (time[], dt[], steps[])."""
        fin = np.ascontiguousarray(np.broadcast_to(np.asarray(final_time, dtype=np.float64), (self.n,)))
        t = np.full(self.n, -1.0) if time is None else np.ascontiguousarray(time, dtype=np.float64).copy()
        d = np.zeros(self.n) if dt is None else np.ascontiguousarray(dt, dtype=np.float64).copy()
        steps = np.zeros(self.n, dtype=np.int32)
        rc = self.lib.dgr_ensemble_run(self.ctx, nsteps, _dp(fin), _dp(t), _dp(d), _ip(steps))
        if rc != _lib.DGR_OK and (check or not 1 <= rc <= 7):
            if 1 <= rc <= 7:
                for s in range(self.n):
                    code, index, step = self.last_error(s)
                    if code:
                        raise StepError(code, index, step, f"ensemble scenario {s}")
            _lib.check(rc, "dgr_ensemble_run")
        return t, d, steps

    def set_gauges(self, gauge_el, gauge_w, capacity: int) -> None:
        """record the elevation at the gauges after every step of the device loop (up to
        `capacity` steps per run); gauge_el None removes them"""
        if gauge_el is None:
            _lib.check(self.lib.dgr_set_gauges(self.ctx, 0, None, None, 0), "dgr_set_gauges")
            self._gauges = None
            return
        el = np.ascontiguousarray(gauge_el, dtype=np.int32)
        w = np.ascontiguousarray(gauge_w, dtype=np.float64).reshape(len(el), self.nm)
        _lib.check(self.lib.dgr_set_gauges(self.ctx, len(el), _ip(el), _dp(w), int(capacity)), "dgr_set_gauges")
        self._gauges = (len(el), int(capacity))

    def gauge_series(self) -> np.ndarray:
        """[capacity, ngauges] values recorded by the last run"""
        ng, cap = self._gauges
        out = np.empty((cap, ng))
        _lib.check(self.lib.dgr_get_gauge_series(self.ctx, _dp(out)), "dgr_get_gauge_series")
        return out

    def write_state_dat(self, s: int, zeta_path=None, qx_path=None, qy_path=None) -> None:
        """scenario s's current state as .dat snapshot files, formatted on the device"""
        enc = lambda p: None if p is None else str(p).encode()  # noqa: E731
        _lib.check(self.lib.dgr_ensemble_write_state_dat(self.ctx, s, enc(zeta_path), enc(qx_path), enc(qy_path)),
                   "dgr_ensemble_write_state_dat")

    def set_element_manning(self, n_el) -> None:
        """per-element Manning n of every scenario, flattened (scenario order); None: the
        node-averaged n of each mesh"""
        if n_el is None:
            _lib.check(self.lib.dgr_set_element_manning(self.ctx, None), "dgr_set_element_manning")
            return
        a = np.ascontiguousarray(n_el, dtype=np.float64)
        assert a.shape == (self.ne,)
        _lib.check(self.lib.dgr_set_element_manning(self.ctx, _dp(a)), "dgr_set_element_manning")

    def flatten_states(self, states):
        """one state per scenario -> the flattened (zeta, Qx, Qy, WD) of the whole ensemble"""
        parts = [[np.asarray(st[v]) for st in states] for v in range(3)]
        wd = [np.asarray(st[3], dtype=np.int32) if len(st) > 3 else np.full(m.num_el, -1, dtype=np.int32)
              for st, m in zip(states, self.meshes)]
        return tuple(np.ascontiguousarray(np.concatenate(p), dtype=np.float64) for p in parts) + \
            (np.ascontiguousarray(np.concatenate(wd)),)

    def _status(self, rc: int, where: str) -> None:
        if rc == _lib.DGR_OK:
            return
        if 1 <= rc <= 7:
            for s in range(self.n):
                code, index, step = self.last_error(s)
                if code:
                    raise StepError(code, index, step, f"{where}, ensemble scenario {s}")
        _lib.check(rc, where)

    def last_error(self, s: int):
        code, index, step = C.c_int(), C.c_int(), C.c_int()
        _lib.check(self.lib.dgr_ensemble_last_error(self.ctx, s, C.byref(code), C.byref(index), C.byref(step)),
                   "dgr_ensemble_last_error")
        return code.value, index.value, step.value

    def kernel_launches(self) -> int:
        return int(self.lib.dgr_kernel_launches(self.ctx))

    def last_device_ms(self) -> float:
        return float(self.lib.dgr_last_device_ms(self.ctx))
