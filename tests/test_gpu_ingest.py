"""Mesh ingest on the GPU (dgr_build_connectivity_device): EdgtoVert, EdgtoEls,
BdryPrescribed and minEdgLength identical to the host builder (itself pinned to
2DCode/extract_mesh_attributes.c) on jittered rectangles with every boundary kind, with
the elements shuffled and their vertex lists rotated or reversed, on the golden fort.14
mesh, and on a 1M-triangle mesh; invalid meshes are refused."""
from __future__ import annotations

import copy
import time

import numpy as np
import pytest

from conftest import load_golden, mesh_from_golden

pytestmark = pytest.mark.gpu


def both(dgrain, m):
    a = dgrain.build_connectivity(copy.deepcopy(m))
    t0 = time.perf_counter()
    b = dgrain.build_connectivity(copy.deepcopy(m), device=True)
    return a, b, time.perf_counter() - t0


def same(a, b):
    assert np.array_equal(a.ed2v, b.ed2v)
    assert np.array_equal(a.ed2el, b.ed2el)
    assert np.array_equal(a.bdry, b.bdry)
    assert a.min_edge == b.min_edge


@pytest.mark.parametrize("nx,ny,jitter", [(3, 2, 0.0), (40, 20, 0.0), (57, 31, 0.2)])
def test_device_connectivity_equals_host(dgrain, nx, ny, jitter):
    m = dgrain.rectangle(nx, ny, jitter=jitter, seed=nx, connect=False)
    # every boundary kind, with overlaps between the lists (priority rule)
    rng = np.random.default_rng(nx)
    bnd = np.concatenate([m.inflow1, m.inflow2, m.outflow]) if len(m.outflow) else None
    if bnd is not None and len(bnd) > 4:
        m.inflow2 = np.ascontiguousarray(bnd[rng.choice(len(bnd), 3, replace=False)])
        m.inflow1 = np.ascontiguousarray(np.concatenate([m.inflow1, bnd[:2]]).astype(np.int32))
    a, b, _ = both(dgrain, m)
    same(a, b)
    assert (b.bdry > 0).any()


def test_shuffled_and_reoriented(dgrain):
    m = dgrain.rectangle(30, 15, jitter=0.15, seed=4, connect=False)
    rng = np.random.default_rng(0)
    m.el2v = np.ascontiguousarray(m.el2v[rng.permutation(m.num_el)])
    rot = rng.integers(0, 3, m.num_el)
    for k in range(m.num_el):
        m.el2v[k] = np.roll(m.el2v[k], rot[k])
    flip = rng.random(m.num_el) < 0.3
    m.el2v[flip] = m.el2v[flip][:, ::-1]
    m.el2v = np.ascontiguousarray(m.el2v)
    same(*both(dgrain, m)[:2])


@pytest.mark.parametrize("fixture", ["compute2DL_jittered576.npz", "run120_wd_tide_rect1600.npz"])
def test_golden_meshes(dgrain, fixture):
    """against the connectivity the reference's own extract_mesh_attributes produced"""
    g = mesh_from_golden(dgrain, load_golden(fixture))
    b = dgrain.build_connectivity(copy.deepcopy(g), device=True)
    same(g, b)


def test_large_mesh(dgrain):
    m = dgrain.rectangle(1000, 500, jitter=0.1, seed=3, connect=False)
    t0 = time.perf_counter()
    a = dgrain.build_connectivity(copy.deepcopy(m))
    host_s = time.perf_counter() - t0
    dgrain.build_connectivity(copy.deepcopy(m), device=True)  # warm-up (context, module load)
    t0 = time.perf_counter()
    b = dgrain.build_connectivity(copy.deepcopy(m), device=True)
    dev_s = time.perf_counter() - t0
    same(a, b)
    print(f"connectivity of {m.num_el} triangles: host {host_s:.3f} s, device {dev_s:.3f} s")


def test_invalid_meshes_refused(dgrain):
    m = dgrain.rectangle(4, 2, connect=False)
    bad = copy.deepcopy(m)
    bad.el2v = bad.el2v.copy()
    bad.el2v[0, 1] = bad.el2v[0, 0]  # repeated vertex
    with pytest.raises(dgrain.DgrError):
        dgrain.build_connectivity(bad, device=True)
    bad = copy.deepcopy(m)
    bad.el2v = bad.el2v.copy()
    bad.el2v[1, 2] = m.num_nodes  # out of range
    with pytest.raises(dgrain.DgrError):
        dgrain.build_connectivity(bad, device=True)
