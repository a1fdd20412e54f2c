"""ctypes binding of libdgrain.so (the C ABI declared in include/dgrain.h).

There is no CPU fallback: if the library is missing this module raises, and every
device call returns DGR_ERR_NO_DEVICE when no GPU is visible.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# DGRAIN_LIBRARY=checked selects the build whose kernels test every gathered index
# (libdgrain_checked.so, compiled with -DDGR_CHECKED by build.py --checked); a path to a
# .so selects that build of the same sources (build.py's `out`, e.g. for tuning sweeps)
_choice = os.environ.get("DGRAIN_LIBRARY", "")
LIB_PATH = (os.path.join(_HERE, "libdgrain_checked.so") if _choice == "checked"
            else os.path.abspath(_choice) if _choice.endswith(".so") else os.path.join(_HERE, "libdgrain.so"))

DGR_OK = 0
DGR_ERR_NAN_FLUX = 1
DGR_ERR_NAN_FLUX_IN = 2
DGR_ERR_NAN_FLUX_EX = 3
DGR_ERR_NEG_DEPTH = 4
DGR_ERR_NAN_VELOCITY = 5
DGR_ERR_EDGE_MATCH = 6
DGR_ERR_BAD_INDEX = 7
DGR_ERR_INVALID = 10
DGR_ERR_MESH = 11
DGR_ERR_IO = 12
DGR_ERR_CUDA = 13
DGR_ERR_NO_DEVICE = 14
DGR_ERR_TOO_LARGE = 15
DGR_ERR_TIMEOUT = 16

dptr = C.POINTER(C.c_double)
iptr = C.POINTER(C.c_int)


class DgrParams(C.Structure):
    _fields_ = [
        ("g", C.c_double),
        ("H0", C.c_double),
        ("VELZERO", C.c_double),
        ("cfl", C.c_double),
        ("dt0", C.c_double),
        ("wet_dry", C.c_int),
        ("tide_on", C.c_int),
        ("tide_amp", C.c_double),
        ("tide_period", C.c_double),
        ("rain", C.c_double),
        ("device", C.c_int),
        ("record_decisions", C.c_int),
        ("rk_stages", C.c_int),
        ("order", C.c_int),
        ("flux", C.c_int),
    ]


class DgrMeshView(C.Structure):
    _fields_ = [
        ("num_el", C.c_int),
        ("num_nodes", C.c_int),
        ("num_edges", C.c_int),
        ("x_coord", dptr),
        ("y_coord", dptr),
        ("z", dptr),
        ("nFriction", dptr),
        ("EltoVert", iptr),
        ("EdgtoEls", iptr),
        ("EdgtoVert", iptr),
        ("BdryPrescribed", iptr),
        ("minEdgLength", C.c_double),
    ]


class DgrScenarioParams(C.Structure):
    _fields_ = [
        ("tide_amp", C.c_double),
        ("tide_period", C.c_double),
        ("rain", C.c_double),
        ("tide_on", C.c_int),
        ("n_el", dptr),
    ]


class DgrFort14(C.Structure):
    _fields_ = [
        ("num_el", C.c_int),
        ("num_nodes", C.c_int),
        ("x_coord", dptr),
        ("y_coord", dptr),
        ("z", dptr),
        ("nFriction", dptr),
        ("EltoVert", iptr),
        ("num_inflow1", C.c_int),
        ("num_inflow2", C.c_int),
        ("num_outflow", C.c_int),
        ("inflow1", iptr),
        ("inflow2", iptr),
        ("outflow", iptr),
    ]


# (name, restype, argtypes) of every exported entry point of include/dgrain.h
SIGNATURES = [
    ("dgr_status_string", C.c_char_p, [C.c_int]),
    ("dgr_abi_version", C.c_int, []),
    ("dgr_read_fort14", C.c_int, [C.c_char_p, C.POINTER(C.POINTER(DgrFort14))]),
    ("dgr_fort14_free", None, [C.POINTER(DgrFort14)]),
    ("dgr_count_edges", C.c_int, [C.c_int, C.c_int, iptr, iptr]),
    ("dgr_build_connectivity", C.c_int,
     [C.c_int, C.c_int, iptr, dptr, dptr, C.c_int, iptr, C.c_int, iptr, C.c_int, iptr, iptr, iptr, iptr, dptr]),
    ("dgr_build_connectivity_device", C.c_int,
     [C.c_int, C.c_int, iptr, dptr, dptr, C.c_int, iptr, C.c_int, iptr, C.c_int, iptr, iptr, iptr, iptr, dptr]),
    ("dgr_initial_state", C.c_int, [C.c_int, iptr, dptr, dptr, dptr, dptr, iptr]),
    ("dgr_write_dat", C.c_int, [C.c_char_p, C.c_int, dptr]),
    ("dgr_write_state_dat", C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_char_p]),
    ("dgr_set_gauges", C.c_int, [C.c_void_p, C.c_int, iptr, dptr, C.c_int]),
    ("dgr_get_gauge_series", C.c_int, [C.c_void_p, dptr]),
    ("dgr_ensemble_write_state_dat", C.c_int, [C.c_void_p, C.c_int, C.c_char_p, C.c_char_p, C.c_char_p]),
    ("dgr_host_alloc", C.c_void_p, [C.c_size_t]),
    ("dgr_host_free", None, [C.c_void_p]),
    ("dgr_params_default", C.c_int, [C.POINTER(DgrParams)]),
    ("dgr_create", C.c_int, [C.POINTER(DgrMeshView), C.POINTER(DgrParams), C.POINTER(C.c_void_p)]),
    ("dgr_destroy", C.c_int, [C.c_void_p]),
    ("dgr_get_params", C.c_int, [C.c_void_p, C.POINTER(DgrParams)]),
    ("dgr_set_params", C.c_int, [C.c_void_p, C.POINTER(DgrParams)]),
    ("dgr_set_element_manning", C.c_int, [C.c_void_p, dptr]),
    ("dgr_upload_state", C.c_int, [C.c_void_p, dptr, dptr, dptr, iptr]),
    ("dgr_download_state", C.c_int, [C.c_void_p, dptr, dptr, dptr, iptr]),
    ("dgr_set_boundary", C.c_int, [C.c_void_p, dptr, dptr]),
    ("dgr_boundary_conditions", C.c_int, [C.c_void_p, C.c_double]),
    ("dgr_compute_L", C.c_int, [C.c_void_p, C.c_double, dptr, dptr, dptr, dptr]),
    ("dgr_slope_limiter", C.c_int, [C.c_void_p]),
    ("dgr_pdop", C.c_int, [C.c_void_p]),
    ("dgr_wet_dry_status", C.c_int, [C.c_void_p]),
    ("dgr_step", C.c_int, [C.c_void_p, C.c_double, C.c_double, dptr]),
    ("dgr_run", C.c_int, [C.c_void_p, C.c_int, C.c_double, dptr, dptr, iptr]),
    ("dgr_last_error", C.c_int, [C.c_void_p, iptr, iptr, iptr]),
    ("dgr_last_cuda_error", C.c_char_p, []),
    ("dgr_get_decisions", C.c_int, [C.c_void_p, C.c_int, iptr, iptr]),
    ("dgr_get_fhat", C.c_int, [C.c_void_p, dptr, dptr, dptr]),
    ("dgr_kernel_launches", C.c_longlong, [C.c_void_p]),
    ("dgr_last_device_ms", C.c_double, [C.c_void_p]),
    ("dgr_profile_step", C.c_int, [C.c_void_p, C.c_int, dptr, C.c_int]),
    ("dgr_pow43_batch", C.c_int, [dptr, dptr, C.c_int, C.c_int]),
    ("dgr_div_rcp_batch", C.c_int, [dptr, dptr, dptr, iptr, C.c_int, C.c_int]),
    ("dgr_set_channel_ends", C.c_int, [C.c_void_p, C.c_int, iptr, iptr, iptr]),
    ("dgr_couple_channel_ends", C.c_int, [C.c_void_p, dptr, dptr, dptr, dptr]),
    ("dgr_get_boundary", C.c_int, [C.c_void_p, dptr, dptr]),
    ("dgr_couple_channel_ends_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("dgr_get_stream", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    ("dgr_ensemble_create", C.c_int, [C.c_int, C.POINTER(DgrMeshView), C.POINTER(DgrScenarioParams),
                                      C.POINTER(DgrParams), C.POINTER(C.c_void_p)]),
    ("dgr_ensemble_size", C.c_int, [C.c_void_p]),
    ("dgr_ensemble_upload_state", C.c_int, [C.c_void_p, C.c_int, dptr, dptr, dptr, iptr]),
    ("dgr_ensemble_download_state", C.c_int, [C.c_void_p, C.c_int, dptr, dptr, dptr, iptr]),
    ("dgr_ensemble_run", C.c_int, [C.c_void_p, C.c_int, dptr, dptr, dptr, iptr]),
    ("dgr_ensemble_last_error", C.c_int, [C.c_void_p, C.c_int, iptr, iptr, iptr]),
    ("dgr_set_schedule", C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    ("dgr_get_schedule", C.c_int, [C.c_void_p, iptr, iptr]),
    ("dgr_write_restart", C.c_int, [C.c_char_p, C.c_int, C.c_int, dptr, dptr, dptr, iptr, C.c_double, C.c_double]),
    ("dgr_read_restart", C.c_int, [C.c_char_p, C.c_int, C.c_int, dptr, dptr, dptr, iptr, dptr, dptr]),
    ("dgr_save_restart", C.c_int, [C.c_void_p, C.c_char_p, C.c_double, C.c_double]),
    ("dgr_load_restart", C.c_int, [C.c_void_p, C.c_char_p, dptr, dptr]),
    ("dgr_set_barrier_wait", C.c_int, [C.c_void_p, C.c_uint, C.c_uint]),
    ("dgr_autotune", C.c_int, [C.c_void_p, C.c_int, iptr, iptr, dptr]),
    ("dgr_slope_limiter_noalloc", C.c_int,
     [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]),
    ("dgr_adjoint_setup", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, iptr, dptr, dptr]),
    ("dgr_adjoint_set_target", C.c_int, [C.c_void_p, dptr]),
    ("dgr_adjoint_forward", C.c_int,
     [C.c_void_p, dptr, dptr, dptr, iptr, C.c_double, C.c_double, C.c_int, dptr, dptr]),
    ("dgr_adjoint_backward", C.c_int, [C.c_void_p, dptr, dptr, dptr, dptr, dptr]),
    ("dgr_tlm", C.c_int, [C.c_void_p, dptr, dptr, dptr, iptr, dptr, dptr, dptr, dptr, dptr, dptr, dptr]),
    ("dgr_fd_frozen", C.c_int, [C.c_void_p, dptr, dptr, dptr, iptr, dptr, dptr, dptr, dptr, dptr, dptr, dptr]),
    ("dgr_adjoint_dt", C.c_int, [C.c_void_p, dptr, dptr]),
    ("dgr_adjoint_timing", C.c_int, [C.c_void_p, dptr, dptr, dptr]),
    ("dgr_set_bathymetry", C.c_int, [C.c_void_p, dptr]),
    ("dgr_p2_reference", C.c_int, [dptr, C.c_int]),
]

_lib = None


def load() -> C.CDLL:
    """Load libdgrain.so once; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python dg-rain_b200/build.py` "
            "(there is no CPU fallback for the DG-RAIN step)")
    lib = C.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def status_string(code: int) -> str:
    return load().dgr_status_string(code).decode()


class DgrError(RuntimeError):
    def __init__(self, code: int, where: str, detail: str = ""):
        self.code = code
        msg = f"{where}: {status_string(code)} ({code})"
        if code == DGR_ERR_CUDA:
            msg += f": {load().dgr_last_cuda_error().decode()}"
        if detail:
            msg += f" {detail}"
        super().__init__(msg)


def check(code: int, where: str) -> None:
    if code != DGR_OK:
        raise DgrError(code, where)
