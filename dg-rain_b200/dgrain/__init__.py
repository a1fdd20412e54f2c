"""dgrain — B200-native DG-RAIN 2D shallow-water step (sm_100a FP64 kernels behind the
C ABI of include/dgrain.h).  This package is the Python side of that ABI: ctypes
bindings, the synthetic mesh generator and a mirror of the reference call surface."""
from . import _lib, p2
from ._lib import DgrError, load
from .mesh import (Mesh, build_connectivity, initial_state, read_fort14, rectangle,
                   rectangle_with_elements, write_fort14)
from .solver import Ensemble, Solver, StepError, default_params
from .adjoint import GaugeMisfit, cr_weights, gauge_misfit, intertidal_points, place_gauges
from . import calibration

__all__ = [
    "_lib", "p2", "calibration", "DgrError", "load", "Mesh", "build_connectivity", "initial_state", "read_fort14",
    "rectangle", "rectangle_with_elements", "write_fort14", "Ensemble", "Solver", "StepError", "default_params",
    "GaugeMisfit", "cr_weights", "gauge_misfit", "intertidal_points", "place_gauges",
]
