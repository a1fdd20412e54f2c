"""Meshes in the 2DCode layout: fort.14 I/O, connectivity, and the seeded synthetic
coastal-watershed generator used by the tests and the benchmark.

The reference ships no 2D mesh, so every workload here comes from `rectangle()`:
  * a Lx x Ly rectangle of nx x ny cells, each split into two triangles along the same
    diagonal, counter-clockwise; interior nodes jittered by U(-j, j) * cell size per axis,
    boundary nodes only along their side, corners fixed;
  * land elevation rising linearly from -5 m at x = 0 to +2 m at x = Lx, plus 8 Gaussian
    bumps (amplitude U(-0.5, 0.5) m, width U(300, 800) m, centres uniform); the mesh
    stores depth z = -elevation (the reference's convention, H = zeta + z);
  * Manning n per node; the x = 0 side goes in the outflow list (type-2 edges,
    elevation-specified, the ocean), every other boundary edge is land;
  * node ids row-major, elements cell by cell.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os

import numpy as np

from . import _lib


@dataclasses.dataclass
class Mesh:
    x: np.ndarray          # [nn] float64
    y: np.ndarray          # [nn]
    z: np.ndarray          # [nn] depth, positive down
    nfric: np.ndarray      # [nn] Manning n
    el2v: np.ndarray       # [ne, 3] int32, 0-based
    inflow1: np.ndarray    # [k, 2] int32 node pairs
    inflow2: np.ndarray
    outflow: np.ndarray
    ed2v: np.ndarray | None = None   # [nf, 2]
    ed2el: np.ndarray | None = None  # [nf, 2]
    bdry: np.ndarray | None = None   # [nf]
    min_edge: float = 0.0

    @property
    def num_el(self) -> int:
        return int(self.el2v.shape[0])

    @property
    def num_nodes(self) -> int:
        return int(self.x.shape[0])

    @property
    def num_edges(self) -> int:
        return int(self.ed2v.shape[0]) if self.ed2v is not None else self.num_nodes + self.num_el - 1

    def view(self) -> "_lib.DgrMeshView":
        """dgr_mesh_view over this mesh's arrays (kept alive by the mesh object)."""
        if self.ed2v is None:
            build_connectivity(self)
        v = _lib.DgrMeshView()
        v.num_el, v.num_nodes, v.num_edges = self.num_el, self.num_nodes, self.num_edges
        v.x_coord = _dp(self.x)
        v.y_coord = _dp(self.y)
        v.z = _dp(self.z)
        v.nFriction = _dp(self.nfric)
        v.EltoVert = _ip(self.el2v)
        v.EdgtoEls = _ip(self.ed2el)
        v.EdgtoVert = _ip(self.ed2v)
        v.BdryPrescribed = _ip(self.bdry)
        v.minEdgLength = self.min_edge
        return v


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_lib.dptr)


def _ip(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_lib.iptr)


def _pairs(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).reshape(-1, 2))


def rectangle(nx: int, ny: int, lx: float = 10000.0, ly: float = 5000.0, jitter: float = 0.0,
              seed: int = 0, n_bumps: int = 8, manning: float = 0.03, connect: bool = True,
              datum: float = 0.0, ocean: bool = True) -> Mesh:
    """The synthetic coastal rectangle; `datum` lowers the whole land surface by that many
    metres (datum = 3 gives a basin that is under water everywhere); ocean = False closes
    the x = 0 side (every boundary edge is land)."""
    rng = np.random.default_rng(seed)
    amp = rng.uniform(-0.5, 0.5, n_bumps)
    sig = rng.uniform(300.0, 800.0, n_bumps)
    cx = rng.uniform(0.0, lx, n_bumps)
    cy = rng.uniform(0.0, ly, n_bumps)
    dx, dy = lx / nx, ly / ny
    ii, jj = np.meshgrid(np.arange(nx + 1, dtype=np.float64), np.arange(ny + 1, dtype=np.float64))
    x = ii * dx
    y = jj * dy
    if jitter > 0.0:
        jx = rng.uniform(-jitter, jitter, x.shape) * dx
        jy = rng.uniform(-jitter, jitter, y.shape) * dy
        left_right = (ii == 0) | (ii == nx)
        bottom_top = (jj == 0) | (jj == ny)
        jx[left_right] = 0.0     # x fixed on the vertical sides
        jy[bottom_top] = 0.0     # y fixed on the horizontal sides
        x = x + jx
        y = y + jy
    x = x.ravel()
    y = y.ravel()
    elev = -5.0 + 7.0 * x / lx - datum
    for k in range(n_bumps):
        elev = elev + amp[k] * np.exp(-((x - cx[k]) ** 2 + (y - cy[k]) ** 2) / (2.0 * sig[k] ** 2))
    z = -elev
    nfric = np.full(x.shape, manning)

    node = lambda i, j: j * (nx + 1) + i  # noqa: E731
    I, J = np.meshgrid(np.arange(nx, dtype=np.int64), np.arange(ny, dtype=np.int64))
    I, J = I.ravel(), J.ravel()
    a, b, c, d = node(I, J), node(I + 1, J), node(I + 1, J + 1), node(I, J + 1)
    el2v = np.empty((2 * nx * ny, 3), dtype=np.int32)
    el2v[0::2] = np.stack([a, b, c], axis=1)
    el2v[1::2] = np.stack([a, c, d], axis=1)
    jj_ = np.arange(ny)
    outflow = np.stack([node(0, jj_), node(0, jj_ + 1)], axis=1).astype(np.int32)
    if not ocean:
        outflow = _pairs([])
    m = Mesh(x=np.ascontiguousarray(x), y=np.ascontiguousarray(y), z=np.ascontiguousarray(z),
             nfric=np.ascontiguousarray(nfric), el2v=np.ascontiguousarray(el2v),
             inflow1=_pairs([]), inflow2=_pairs([]), outflow=np.ascontiguousarray(outflow))
    if connect:
        build_connectivity(m)
    return m


def build_connectivity(m: Mesh, device: bool = False) -> Mesh:
    """EdgtoVert/EdgtoEls/BdryPrescribed/minEdgLength exactly as
    2DCode/extract_mesh_attributes.c:143-361 numbers them (native, hashed; device=True:
    sorted on the current GPU, same arrays)."""
    lib = _lib.load()
    if device:
        nf = m.num_nodes + m.num_el - 1  # Euler's relation, checked by the builder
    else:
        nf = C.c_int(0)
        _lib.check(lib.dgr_count_edges(m.num_el, m.num_nodes, _ip(m.el2v), C.byref(nf)), "dgr_count_edges")
        nf = nf.value
    ed2v = np.zeros((nf, 2), dtype=np.int32)
    ed2el = np.zeros((nf, 2), dtype=np.int32)
    bdry = np.zeros(nf, dtype=np.int32)
    me = C.c_double(0.0)
    fn = lib.dgr_build_connectivity_device if device else lib.dgr_build_connectivity
    _lib.check(fn(
        m.num_el, m.num_nodes, _ip(m.el2v), _dp(m.x), _dp(m.y),
        len(m.inflow1), _ip(m.inflow1), len(m.inflow2), _ip(m.inflow2), len(m.outflow), _ip(m.outflow),
        _ip(ed2v), _ip(ed2el), _ip(bdry), C.byref(me)), "dgr_build_connectivity")
    m.ed2v, m.ed2el, m.bdry, m.min_edge = ed2v, ed2el, bdry, me.value
    return m


def write_fort14(m: Mesh, path: str, title: str = "DG-RAIN synthetic mesh") -> None:
    """fort.14 in the 2DCode dialect (2DCode/extract_mesh_attributes.c:39-141); floats are
    written with 17 significant digits so that reading them back is exact."""
    with open(path, "w") as f:
        f.write(title + "\n")
        f.write(f"{m.num_el} {m.num_nodes}\n")
        ids = np.arange(1, m.num_nodes + 1)
        np.savetxt(f, np.column_stack([ids, m.x, m.y, m.z, m.nfric]),
                   fmt=["%d", "%.17g", "%.17g", "%.17g", "%.17g"])
        eids = np.arange(1, m.num_el + 1)
        np.savetxt(f, np.column_stack([eids, np.full(m.num_el, 3), m.el2v + 1]), fmt="%d")
        f.write("boundaries\n")
        for lst in (m.inflow1, m.inflow2, m.outflow):
            f.write(f"{len(lst)}\n")
            if len(lst):
                np.savetxt(f, lst + 1, fmt="%d")


def read_fort14(path: str, connect: bool = True) -> Mesh:
    """store_mesh (2DCode/extract_mesh_attributes.c:39-141), native reader."""
    lib = _lib.load()
    p = C.POINTER(_lib.DgrFort14)()
    _lib.check(lib.dgr_read_fort14(os.fsencode(path), C.byref(p)), f"dgr_read_fort14({path})")
    try:
        f = p.contents
        nn, ne = f.num_nodes, f.num_el
        arr = lambda ptr, n, dt: np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt, copy=True)  # noqa: E731
        m = Mesh(x=arr(f.x_coord, nn, np.float64), y=arr(f.y_coord, nn, np.float64),
                 z=arr(f.z, nn, np.float64), nfric=arr(f.nFriction, nn, np.float64),
                 el2v=arr(f.EltoVert, 3 * ne, np.int32).reshape(ne, 3),
                 inflow1=_pairs(arr(f.inflow1, 2 * f.num_inflow1, np.int32)) if f.num_inflow1 else _pairs([]),
                 inflow2=_pairs(arr(f.inflow2, 2 * f.num_inflow2, np.int32)) if f.num_inflow2 else _pairs([]),
                 outflow=_pairs(arr(f.outflow, 2 * f.num_outflow, np.int32)) if f.num_outflow else _pairs([]))
    finally:
        lib.dgr_fort14_free(p)
    if connect:
        build_connectivity(m)
    return m


def initial_state(m: Mesh, zeta_nodal: np.ndarray | None = None, h0: float = 1e-3):
    """2DCode/initialize.c:117-126 from nodal elevations.  Default nodal elevation is the
    synthetic workloads' 'surface 0 at rest': zeta = max(0, H0 - z), so dry land holds a
    film of depth H0.  Returns (zeta, Qx, Qy, WD) in the reference layout."""
    if zeta_nodal is None:
        zeta_nodal = np.maximum(0.0, h0 - m.z)
    zeta_nodal = np.ascontiguousarray(zeta_nodal, dtype=np.float64)
    ne = m.num_el
    zeta = np.zeros(3 * ne)
    qx = np.zeros(3 * ne)
    qy = np.zeros(3 * ne)
    wd = np.zeros(ne, dtype=np.int32)
    lib = _lib.load()
    _lib.check(lib.dgr_initial_state(ne, _ip(m.el2v), _dp(zeta_nodal), _dp(zeta), _dp(qx), _dp(qy), _ip(wd)),
               "dgr_initial_state")
    return zeta, qx, qy, wd


def log_uniform_sizes(n: int, lo: int, hi: int, seed: int) -> np.ndarray:
    """Element counts log-uniform in [lo, hi] (ensemble workloads)."""
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(lo), np.log(hi), n))


def rectangle_with_elements(n_el: float, seed: int, jitter: float = 0.1, cell: float | None = None, **kw) -> Mesh:
    """Rectangle mesh with about n_el triangles: nx = round(sqrt(n_el)), ny = nx // 2.
    With `cell` (metres) the domain is nx*cell by ny*cell instead of 10 km x 5 km, so the
    resolution, and with it the CFL time step, stays that of the large workload."""
    nx = max(2, int(round(np.sqrt(n_el))))
    ny = max(1, nx // 2)
    if cell is not None:
        kw.setdefault("lx", nx * cell)
        kw.setdefault("ly", ny * cell)
    return rectangle(nx, ny, jitter=jitter, seed=seed, **kw)
