"""The device .dat writer's number formatting (dgr_format.cuh), compiled for the host and
compared byte for byte with the C library's printf("%1.15f"), the format of the
reference's snapshot files, on values of every magnitude, exact decimal ties (odd
multiples of 2^-16 sit exactly half-way at the 15th decimal), carries into the integer
part, negative zero, subnormals, nan and inf."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "format_host.cpp")
HDR = os.path.join(HERE, "..", "dg-rain_b200", "csrc", "dgr_format.cuh")
LIB = os.path.join(HERE, "_build", "libdgr_format_host.so")


def _lib():
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(SRC), os.path.getmtime(HDR)):
        os.makedirs(os.path.dirname(LIB), exist_ok=True)
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", LIB, SRC], check=True)
    lib = C.CDLL(LIB)
    lib.dgr_t_format_mismatches.restype = C.c_longlong
    lib.dgr_t_format_mismatches.argtypes = [np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS"), C.c_longlong,
                                            C.POINTER(C.c_longlong)]
    return lib


def _check(lib, v):
    v = np.ascontiguousarray(v, dtype=np.float64)
    first = C.c_longlong()
    bad = lib.dgr_t_format_mismatches(v, v.size, C.byref(first))
    assert bad == 0, (bad, repr(v[first.value]), "%1.15f" % v[first.value])


def test_format_matches_printf():
    lib = _lib()
    rng = np.random.default_rng(0)
    parts = [
        rng.normal(size=200000),
        rng.normal(size=200000) * 10.0 ** rng.uniform(-20, 18, 200000),
        rng.uniform(-1e-15, 1e-15, 50000),
        (rng.integers(-2 ** 40, 2 ** 40, 100000) * 2 + 1) / 2.0 ** 16,   # exact ties at the 15th decimal
        (rng.integers(-2 ** 30, 2 ** 30, 50000) * 2 + 1) / 2.0 ** 16 + rng.integers(-1000, 1000, 50000),
        np.array([0.0, -0.0, 1.0, -1.0, 0.9999999999999999, 0.99999999999999995, 1 - 2 ** -53, 5e-16, -5e-16,
                  4.9999999999999996e-16, 1.5e-15, 2.5e-15, 2 ** -1074, -2 ** -1074, 2 ** -1022, 2.0 ** 62,
                  2.0 ** 63 - 1024, 9.5, 123456789.123456789, np.nan, -np.nan, np.inf, -np.inf]),
        rng.integers(0, 2 ** 63, 100000, dtype=np.int64).view(np.float64),  # random bit patterns (|v| < 2)
    ]
    for p in parts:
        _check(lib, p)
