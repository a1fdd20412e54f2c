"""ORACLE — test infrastructure only.

A numpy restatement of the reference's mesh set-up, for meshes far too large for the
reference's own O(E*N) search (2DCode/extract_mesh_attributes.c), so that the unmodified
reference step can run on the 4,000,000-triangle workload without this repository's
library:

  * connectivity(): EdgtoVert, EdgtoEls, BdryPrescribed and minEdgLength numbered as
    2DCode/extract_mesh_attributes.c:143-361 numbers them;
  * initial_state(): the midpoint state of 2DCode/initialize.c:117-126 from nodal
    elevations, at rest, WD = -1.

The numbering rules, each restated here by sorting instead of the reference's nested loops:
  1. node adjacency in first-seen order: elements in index order, for local vertex n the
     neighbours v[(n+1)%3] then v[(n+2)%3] appended when not yet listed (:166-212);
  2. edges numbered by their lower node, then by the position of the higher node in the
     lower node's adjacency list (:225-250);
  3. EdgtoEls: the first two elements, in index order, that own the edge; an edge with one
     element repeats it (:259-295);
  4. BdryPrescribed: 3 if the edge is in the second inflow list, else 1 if in the first,
     else 2 if in the outflow list, else 0 (:297-354);
  5. minEdgLength: the least edge length, from 9999999 (:25, :302-303).
Elements with a repeated vertex are refused.  Checked against the reference's own arrays
(tests/test_oracle_pin.py, tests/test_golden.py) and against the library's builders.

Only tests/ and bench.py's reference arm use this module.
"""
from __future__ import annotations

import numpy as np


def _pair_keys(pairs, nn):
    p = np.asarray(pairs, dtype=np.int64).reshape(-1, 2)
    return np.minimum(p[:, 0], p[:, 1]) * nn + np.maximum(p[:, 0], p[:, 1])


def connectivity(el2v, x, y, inflow1=(), inflow2=(), outflow=()):
    """Returns (ed2v [nf, 2], ed2el [nf, 2], bdry [nf]) as int32 and min_edge (float)."""
    v = np.asarray(el2v, dtype=np.int64).reshape(-1, 3)
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    ne, nn = len(v), len(x)
    if ((v < 0) | (v >= nn)).any():
        raise ValueError("vertex index out of range")
    if ((v[:, 0] == v[:, 1]) | (v[:, 1] == v[:, 2]) | (v[:, 2] == v[:, 0])).any():
        raise ValueError("element with a repeated vertex")

    # rule 1: incidence records in the reference's visiting order (element, local vertex,
    # then its two neighbours); a stable sort by (node, neighbour) keeps each pair's records
    # in that order, so the head of each run is the pair's first sighting
    node = np.repeat(v, 2, axis=1).ravel()
    nb = v[:, [1, 2, 2, 0, 0, 1]].ravel()
    key = node * nn + nb
    order = np.argsort(key, kind="stable")
    ks = key[order]
    head = np.ones(len(ks), dtype=bool)
    head[1:] = ks[1:] != ks[:-1]
    first = order[head]
    pn, pb = node[first], nb[first]

    # rule 2: from each node, the neighbours above it in first-seen order
    up = pb > pn
    pn, pb, first = pn[up], pb[up], first[up]
    o2 = np.lexsort((first, pn))
    ed2v = np.stack([pn[o2], pb[o2]], axis=1)
    nf = len(ed2v)
    if nf != nn + ne - 1:  # Euler's relation, as the reference requires (:218-256)
        raise ValueError(f"{nf} edges, Euler's relation gives {nn + ne - 1}")

    # rule 3: owners of each edge, first two in element order
    ekey = ed2v[:, 0] * nn + ed2v[:, 1]
    srt = np.argsort(ekey)
    a, b = v, v[:, [1, 2, 0]]
    q = (np.minimum(a, b) * nn + np.maximum(a, b)).ravel()
    pos = np.searchsorted(ekey[srt], q)
    e_of = srt[pos]
    el_of = np.repeat(np.arange(ne, dtype=np.int64), 3)
    o3 = np.argsort(e_of, kind="stable")  # records are already in element order
    es, els = e_of[o3], el_of[o3]
    start = np.flatnonzero(np.r_[True, es[1:] != es[:-1]])
    ed2el = np.empty((nf, 2), dtype=np.int64)
    ed2el[es[start], 0] = els[start]
    ed2el[:, 1] = ed2el[:, 0]
    nxt = start + 1
    has2 = nxt < len(es)
    has2[has2] = es[nxt[has2]] == es[start[has2]]
    ed2el[es[start[has2]], 1] = els[nxt[has2]]

    # rule 4: boundary lists, second inflow first
    bdry = np.zeros(nf, dtype=np.int32)
    for lst, typ in ((outflow, 2), (inflow1, 1), (inflow2, 3)):
        if len(lst):
            bdry[np.isin(ekey, _pair_keys(lst, nn))] = typ

    # rule 5: the reference's length expression
    n0, n1 = ed2v[:, 0], ed2v[:, 1]
    dx, dy = x[n1] - x[n0], y[n1] - y[n0]
    length = np.sqrt(dx * dx + dy * dy)
    min_edge = float(min(9999999.0, length.min()))
    return ed2v.astype(np.int32), ed2el.astype(np.int32), bdry, min_edge


def initial_state(el2v, zeta_nodal):
    """(zeta, Qx, Qy, WD) in the reference layout: zeta at each edge midpoint the mean of
    its two nodal values (0.5 * (a + b), as the reference writes it), at rest, WD = -1."""
    v = np.asarray(el2v, dtype=np.int64).reshape(-1, 3)
    nz = np.asarray(zeta_nodal, dtype=np.float64)[v]
    zeta = np.empty((len(v), 3))
    zeta[:, 0] = 0.5 * (nz[:, 0] + nz[:, 1])
    zeta[:, 1] = 0.5 * (nz[:, 1] + nz[:, 2])
    zeta[:, 2] = 0.5 * (nz[:, 2] + nz[:, 0])
    n3 = 3 * len(v)
    return zeta.ravel(), np.zeros(n3), np.zeros(n3), np.full(len(v), -1, dtype=np.int32)
