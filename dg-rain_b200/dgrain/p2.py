"""Fields of the p = 2 modal step (dgr_params.order = 2): L2 projection onto DG-SWEM's
orthogonal basis and evaluation, with the reference-element tables the kernels use
(dgr_p2_reference).  Coefficients are laid out [6*el + m] per variable."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .mesh import Mesh

NM = 6


def reference() -> dict:
    t = np.empty(234)
    _lib.check(_lib.load().dgr_p2_reference(t.ctypes.data_as(_lib.dptr), C.c_int(234)), "dgr_p2_reference")
    return {"wq": t[0:7], "lam": t[7:28].reshape(7, 3), "phi": t[28:70].reshape(7, 6),
            "dr": t[70:112].reshape(7, 6), "ds": t[112:154].reshape(7, 6), "te": t[154:157], "wg": t[157:160],
            "phie": t[160:214].reshape(3, 3, 6), "mass": t[214:220], "rs": t[220:234].reshape(7, 2)}


def basis(r, s) -> np.ndarray:
    """the six basis functions [..., 6] at reference coordinates (r, s) (closed forms of
    DG-SWEM src/orthobasis_area.F:18-175 at p = 2, hierarchical order)"""
    r, s = np.asarray(r, dtype=np.float64), np.asarray(s, dtype=np.float64)
    A = r + (1.0 + s) / 2
    B = (1.0 - s) / 2
    return np.stack([np.ones_like(r), (3 * s + 1) / 2, A, (5 * s * s + 2 * s - 1) / 2, A * (5 * s + 3) / 2,
                     (3 * A * A - B * B) / 2], axis=-1)


def gauge_weights(mesh: Mesh, points) -> tuple[np.ndarray, np.ndarray]:
    """elements and weights [ng, 6] of gauge points [(x, y), ...]: the basis at the point, so
    that sum_m w_m zeta_m is the p = 2 elevation there"""
    from .adjoint import barycentric

    els, ws = [], []
    for px, py in points:
        e, lam = barycentric(mesh, px, py)
        if e < 0:
            raise ValueError(f"gauge ({px}, {py}) lies outside the mesh")
        # vertices (-1,-1), (1,-1), (-1,1) of the reference triangle
        r = -lam[0] + lam[1] - lam[2]
        s = -lam[0] - lam[1] + lam[2]
        els.append(e)
        ws.append(basis(r, s))
    return np.asarray(els, dtype=np.int32), np.ascontiguousarray(np.asarray(ws, dtype=np.float64))


def quadrature_points(mesh: Mesh, ref: dict | None = None):
    """physical coordinates [ne, 7] of every element's area quadrature points and the weights
    [ne, 7] of the physical integral (2 |J| w_q)"""
    ref = ref or reference()
    v = mesh.el2v
    X = mesh.x[v] @ ref["lam"].T
    Y = mesh.y[v] @ ref["lam"].T
    xr, xs = (mesh.x[v[:, 1]] - mesh.x[v[:, 0]]) / 2, (mesh.x[v[:, 2]] - mesh.x[v[:, 0]]) / 2
    yr, ys = (mesh.y[v[:, 1]] - mesh.y[v[:, 0]]) / 2, (mesh.y[v[:, 2]] - mesh.y[v[:, 0]]) / 2
    detj = np.abs(xr * ys - xs * yr)
    return X, Y, 2.0 * detj[:, None] * ref["wq"][None, :]


def project(mesh: Mesh, f, ref: dict | None = None) -> np.ndarray:
    """L2 projection of f(x, y) (vectorised) onto the basis: coefficients [6*el + m]"""
    ref = ref or reference()
    X, Y, W = quadrature_points(mesh, ref)
    F = np.asarray(f(X, Y), dtype=np.float64)
    c = (W * F) @ ref["phi"] / (W.sum(axis=1)[:, None] / 2.0) / ref["mass"][None, :]
    return np.ascontiguousarray(c.reshape(-1))


def evaluate(mesh: Mesh, coeffs: np.ndarray, ref: dict | None = None) -> np.ndarray:
    """values [ne, 7] at the area quadrature points"""
    ref = ref or reference()
    return coeffs.reshape(-1, NM) @ ref["phi"].T


def l2_error(mesh: Mesh, coeffs: np.ndarray, f, ref: dict | None = None) -> float:
    ref = ref or reference()
    X, Y, W = quadrature_points(mesh, ref)
    d = evaluate(mesh, coeffs, ref) - f(X, Y)
    return float(np.sqrt((W * d * d).sum()))


def volume(mesh: Mesh, zeta: np.ndarray, ref: dict | None = None) -> float:
    """integral of the elevation over the mesh (only mode 0 contributes)"""
    ref = ref or reference()
    _, _, W = quadrature_points(mesh, ref)
    return float((W.sum(axis=1) * zeta.reshape(-1, NM)[:, 0]).sum())
