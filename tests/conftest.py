"""Shared fixtures.  Tests marked `gpu` need a CUDA device; everything else runs on CPU."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "dg-rain_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and runs the sm_100a kernels")


def _ensure_built():
    import importlib

    sys.path.insert(0, PKG)
    build = importlib.import_module("build")
    build.build()
    from oracle import oracle as orc

    orc.build()


_ensure_built()


@pytest.fixture(scope="session")
def dgrain():
    import dgrain as d

    return d


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as o

    return o


def bits_equal(a, b) -> bool:
    """Equal bit for bit: float arrays are compared as their bit patterns, so the signs of
    zeros count; NaNs match NaNs whatever their payload (x86 and the GPU make different
    default NaNs).  Other arrays compare by value."""
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape:
        return False
    if a.dtype.kind != "f" and b.dtype.kind != "f":
        return bool(np.array_equal(a, b))
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    na, nb = np.isnan(a), np.isnan(b)
    return bool(np.array_equal(na, nb) and np.array_equal(a.view(np.int64)[~na], b.view(np.int64)[~nb]))


def land_film_state(dgrain_mod, mesh, film=0.5e-3):
    """Surface 0 at rest; dry land holds a film of depth `film` (below H0 = 1e-3 so the
    reference's wetDryStatus2D classifies it dry without rounding ties)."""
    zn = np.maximum(0.0, film - mesh.z)
    return dgrain_mod.initial_state(mesh, zn)


def signed_zero_state(dgrain_mod, mesh, seed, nx):
    """A land-film state with noise, plus a patch of wet (ocean-side) cells whose Qx and Qy
    element means are +0 or -0 (random signs), a few of them negative (Qx) or positive (Qy):
    inside the patch the limiter's node max (Qx) or min (Qy) is then a zero, whose sign is
    that of the first zero mean in element order, and its clamp meets zeros of both signs.
    `mesh` is a rectangle of nx cells per row (two triangles per cell)."""
    rng = np.random.default_rng(seed)
    z, qx, qy, wd = land_film_state(dgrain_mod, mesh)
    z = z + 0.002 * rng.standard_normal(z.shape)
    qx = 0.01 * rng.standard_normal(qx.shape)
    qy = 0.01 * rng.standard_normal(qy.shape)
    cell = np.arange(mesh.num_el) // 2
    patch = np.flatnonzero((cell % nx < nx // 6) & (cell // nx >= 5) & (cell // nx < 20))
    for q, sign_of_nonzero in ((qx, -1.0), (qy, 1.0)):
        v = q.reshape(-1, 3)
        v[patch] = np.where(rng.random(len(patch)) < 0.5, -0.0, 0.0)[:, None]
        few = patch[rng.random(len(patch)) < 0.1]
        v[few] = sign_of_nonzero * 0.01 * rng.random((len(few), 3))
    return z, qx, qy, wd


def negative_zeros(a) -> int:
    """how many entries of a are -0.0"""
    a = np.ascontiguousarray(a, dtype=np.float64)
    return int(((a == 0.0) & np.signbit(a)).sum())


def moving_state(dgrain_mod, mesh, seed=0, depth=2.0, qscale=0.5):
    """A fully wet random state with momentum, exercising every flux branch."""
    rng = np.random.default_rng(seed)
    zn = depth - mesh.z + 0.05 * rng.standard_normal(mesh.num_nodes)
    zeta, qx, qy, wd = dgrain_mod.initial_state(mesh, zn)
    qx = qscale * rng.standard_normal(qx.shape)
    qy = qscale * rng.standard_normal(qy.shape)
    return zeta, qx, qy, wd


@pytest.fixture(scope="session")
def mesh_c1(dgrain):
    """The 10 km x 5 km, 40 x 20-cell split rectangle (1,600 triangles)."""
    return dgrain.rectangle(40, 20, jitter=0.0, seed=1)


@pytest.fixture(scope="session")
def mesh_j(dgrain):
    """A jittered 24 x 12-cell mesh (576 triangles)."""
    return dgrain.rectangle(24, 12, jitter=0.1, seed=5)


def has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name), allow_pickle=False))


def mesh_from_golden(dgrain_mod, g):
    """Mesh object from the arrays stored in a golden fixture (no generator involved)."""
    m = dgrain_mod.Mesh(x=g["x"], y=g["y"], z=g["z"], nfric=g["nfric"], el2v=g["el2v"],
                        inflow1=g["inflow1"], inflow2=g["inflow2"], outflow=g["outflow"])
    m.ed2v, m.ed2el, m.bdry, m.min_edge = g["ed2v"], g["ed2el"], g["bdry"], float(g["min_edge"])
    return m
