"""Writes the golden vectors of ChanNet's channel <-> junction coupling by running the
UNMODIFIED reference internal_BC.c (oracle/_ref/librefchan.so, built by `make -C oracle`
from the reference tree) on a seeded junction mesh, state and channel lists (overlapping
lists included, so the write order is pinned too).

    python tests/golden/make_coupling_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "dg-rain_b200"))

import dgrain  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main():
    m = dgrain.rectangle(24, 12, jitter=0.1, seed=17)
    rng = np.random.default_rng(17)
    ne, nf = m.num_el, m.num_edges
    zeta, qx, qy = rng.uniform(-0.5, 0.5, 3 * ne), rng.normal(0, 0.3, 3 * ne), rng.normal(0, 0.3, 3 * ne)
    bz, bq = rng.normal(size=nf), rng.normal(size=nf)
    be = rng.permutation(np.flatnonzero(m.ed2el[:, 0] == m.ed2el[:, 1])).astype(np.int32)
    chans, used = [], 0
    for c in range(5):
        nodes = int(rng.integers(2, 9))
        A, Q = rng.uniform(0.5, 40.0, 2 * nodes), rng.normal(0.0, 5.0, 2 * nodes)
        ends = []
        for side in range(2):
            n = int(rng.integers(1, 4))
            start = used - 1 if c == 4 else used  # the last channel reuses an edge
            ends.append(be[start:start + n])
            used = max(used, start + n)
        chans.append((A, Q, ends[0], ends[1]))
    bz2, bq2, out = O.internal_bc(m, zeta, qx, qy, bz, bq, chans, reference=True)
    cat = lambda xs, dt: np.concatenate([np.asarray(x, dtype=dt) for x in xs])  # noqa: E731
    np.savez_compressed(
        os.path.join(HERE, "coupling_internal_bc.npz"),
        x=m.x, y=m.y, z=m.z, nfric=m.nfric, el2v=m.el2v, ed2v=m.ed2v, ed2el=m.ed2el, bdry=m.bdry,
        min_edge=np.array(m.min_edge), inflow1=m.inflow1, inflow2=m.inflow2, outflow=m.outflow,
        zeta=zeta, qx=qx, qy=qy, bz=bz, bq=bq,
        nodes=np.array([len(c[0]) // 2 for c in chans], dtype=np.int32),
        A=cat([c[0] for c in chans], np.float64), Q=cat([c[1] for c in chans], np.float64),
        in_ptr=np.concatenate([[0], np.cumsum([len(c[2]) for c in chans])]).astype(np.int32),
        in_edges=cat([c[2] for c in chans], np.int32),
        out_ptr=np.concatenate([[0], np.cumsum([len(c[3]) for c in chans])]).astype(np.int32),
        out_edges=cat([c[3] for c in chans], np.int32),
        bz_out=bz2, bq_out=bq2, A_out=cat([o[0] for o in out], np.float64), Q_out=cat([o[1] for o in out], np.float64))
    print("written coupling_internal_bc.npz:", len(chans), "channels,", used, "junction edges")


if __name__ == "__main__":
    main()
