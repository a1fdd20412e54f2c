"""Channel <-> junction coupling (ChanNet/internal_BC.c) on the CPU: the oracle's C
restatement (oracle/dgr_oracle.c, orc_internal_bc) against the UNMODIFIED reference
internal_BC.c compiled into oracle/_ref (oracle/chan_driver.c), bit for bit, on random
junction states and channel-end edge lists.  The device coupling is checked against the
restatement in test_gpu_coupling.py."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import bits_equal

oracle = pytest.importorskip("oracle.oracle")


def boundary_edges(m):
    e = np.flatnonzero(m.ed2el[:, 0] == m.ed2el[:, 1])
    return e.astype(np.int32)


def coupling_case(dgrain, nx=20, ny=10, seed=0, nchan=4, overlap=False, datum=0.0):
    """A jittered junction mesh with a random state and `nchan` channels, each with a few
    boundary edges at its inflow and/or outflow end (disjoint unless overlap)."""
    m = dgrain.rectangle(nx, ny, jitter=0.1, seed=seed, datum=datum)
    rng = np.random.default_rng(seed)
    ne, nf = m.num_el, m.num_edges
    zeta = rng.uniform(-0.5, 0.5, 3 * ne)
    qx = rng.normal(0.0, 0.3, 3 * ne)
    qy = rng.normal(0.0, 0.3, 3 * ne)
    bz = rng.normal(size=nf)
    bq = rng.normal(size=nf)
    be = rng.permutation(boundary_edges(m))
    channels, used = [], 0
    for c in range(nchan):
        nodes = int(rng.integers(2, 12))
        A = rng.uniform(0.5, 40.0, 2 * nodes)
        Q = rng.normal(0.0, 5.0, 2 * nodes)
        ends = []
        for side in range(2):
            n = int(rng.integers(0, 4)) if c else int(rng.integers(1, 4))
            if overlap and used >= 2:
                ends.append(be[used - 2:used - 2 + n])
            else:
                ends.append(be[used:used + n])
                used += n
        channels.append((A, Q, ends[0], ends[1]))
    return m, (zeta, qx, qy), bz, bq, channels


@pytest.mark.skipif(not oracle.have_reference_coupling(), reason="oracle/_ref not built (reference tree absent)")
@pytest.mark.parametrize("seed,overlap", [(0, False), (1, False), (2, False), (3, True), (4, True)])
def test_internal_bc_restatement_matches_reference(dgrain, seed, overlap):
    m, (zeta, qx, qy), bz, bq, chans = coupling_case(dgrain, seed=seed, overlap=overlap)
    got = oracle.internal_bc(m, zeta, qx, qy, bz, bq, chans)
    want = oracle.internal_bc(m, zeta, qx, qy, bz, bq, chans, reference=True)
    assert bits_equal(got[0], want[0]) and bits_equal(got[1], want[1])
    for (a, q), (ar, qr) in zip(got[2], want[2]):
        assert bits_equal(a, ar) and bits_equal(q, qr)
    # the pass did something: coupled edges rewritten, ghost traces set
    coupled = np.concatenate([np.concatenate([c[2], c[3]]) for c in chans]).astype(int)
    assert not bits_equal(got[0][coupled], bz[coupled])


def test_internal_bc_lake_at_rest(dgrain):
    """A junction at rest (flat surface 0.2 m, no discharge) and channels holding the same
    surface at rest: every coupled edge gets bzeta = 0.2 and bQn = 0, and each channel's
    ghost area is the wetted length-weighted depth of its edges (a basin 7 m below datum)."""
    m, _, bz, bq, chans = coupling_case(dgrain, seed=7, datum=7.0)
    ne = m.num_el
    zeta = np.full(3 * ne, 0.2)
    zero = np.zeros(3 * ne)
    rest = []
    for A, Q, e_in, e_out in chans:
        A = A.copy()
        Q = np.zeros_like(Q)
        for side, edges in ((0, e_in), (1, e_out)):
            if len(edges) == 0:
                continue
            # channel trace at the junction node = surface depth x the edges' total length
            idx = 1 if side == 0 else len(A) - 2
            e = edges[0]
            v = m.ed2v[e]
            zm = 0.5 * (m.z[v[0]] + m.z[v[1]])
            L = np.hypot(*(np.array([m.x[v[0]] - m.x[v[1]], m.y[v[0]] - m.y[v[1]]])))
            A[idx] = (0.2 + zm) * len(edges) * L
        rest.append((A, Q, e_in, e_out))
    bz2, bq2, out = oracle.internal_bc(m, zeta, zero, zero, bz, bq, rest)
    for (A, Q, e_in, e_out), (A2, Q2) in zip(rest, out):
        if len(e_in):
            e = e_in[0]
            assert abs(bz2[e] - 0.2) < 1e-12 and bq2[e] == 0.0
            assert Q2[0] == 0.0 and A2[0] > 0
        if len(e_out):
            assert Q2[-1] == 0.0 and A2[-1] > 0


def test_internal_bc_restatement_matches_golden(dgrain):
    """The restatement against the reference internal_BC's own outputs committed in
    tests/golden/coupling_internal_bc.npz (tests/golden/make_coupling_golden.py), so the
    pin holds where oracle/_ref was not built."""
    from conftest import load_golden, mesh_from_golden

    g = load_golden("coupling_internal_bc.npz")
    m = mesh_from_golden(dgrain, g)
    chans, off = [], 0
    for k, n in enumerate(g["nodes"]):
        chans.append((g["A"][2 * off:2 * (off + n)], g["Q"][2 * off:2 * (off + n)],
                      g["in_edges"][g["in_ptr"][k]:g["in_ptr"][k + 1]],
                      g["out_edges"][g["out_ptr"][k]:g["out_ptr"][k + 1]]))
        off += n
    bz, bq, out = oracle.internal_bc(m, g["zeta"], g["qx"], g["qy"], g["bz"], g["bq"], chans)
    assert bits_equal(bz, g["bz_out"]) and bits_equal(bq, g["bq_out"])
    assert bits_equal(np.concatenate([o[0] for o in out]), g["A_out"])
    assert bits_equal(np.concatenate([o[1] for o in out]), g["Q_out"])
