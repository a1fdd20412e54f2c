"""Writes the golden vectors in this folder by running the UNMODIFIED reference 2DCode
(oracle/_ref, built by `make -C oracle` from the reference tree).

    python tests/golden/make_golden.py

Each fixture stores its mesh arrays and inputs together with the reference's outputs,
so the tests do not depend on the mesh generator or on the reference being present.
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


def mesh_arrays(m):
    return dict(x=m.x, y=m.y, z=m.z, nfric=m.nfric, el2v=m.el2v, ed2v=m.ed2v, ed2el=m.ed2el, bdry=m.bdry,
                min_edge=np.array(m.min_edge), inflow1=m.inflow1, inflow2=m.inflow2, outflow=m.outflow)


def film_state(m, film):
    return dgrain.initial_state(m, np.maximum(0.0, film - m.z))


def moving(m, seed):
    rng = np.random.default_rng(seed)
    zn = 2.0 - m.z + 0.05 * rng.standard_normal(m.num_nodes)
    z, qx, qy, wd = dgrain.initial_state(m, zn)
    return z, 0.5 * rng.standard_normal(qx.shape), 0.5 * rng.standard_normal(qy.shape), wd


def main():
    O.build()
    assert O.have_reference(), "needs oracle/_ref (reference tree)"

    # 1. compute2DL on a jittered mesh with a moving state, wet/dry off and on
    m = dgrain.rectangle(24, 12, jitter=0.1, seed=5)
    z, qx, qy, wd = moving(m, 4)
    wd_rand = np.random.default_rng(1).integers(0, 2, m.num_el).astype(np.int32)
    out = dict(mesh_arrays(m), zeta=z, qx=qx, qy=qy, wd_rand=wd_rand)
    for flag, w in ((0, wd), (1, wd_rand)):
        ref = O.Reference(wet_dry=bool(flag))
        ref.set_mesh(m)
        ref.initialize()
        ref.set_state(z, qx, qy, w)
        ref.boundary_conditions()
        rc, rz, rx, ry, lam = ref.compute2DL()
        assert rc == 0
        bz, bq = ref.get_bc()
        f1, f2, f3 = ref.fhat()
        out.update({f"wd{flag}_rhs_zeta": rz, f"wd{flag}_rhs_qx": rx, f"wd{flag}_rhs_qy": ry,
                    f"wd{flag}_max_lambda": np.array(lam), f"wd{flag}_f1": f1, f"wd{flag}_f2": f2,
                    f"wd{flag}_f3": f3})
        out["bzeta"], out["bqn"] = bz, bq
    np.savez_compressed(os.path.join(HERE, "compute2DL_jittered576.npz"), **out)

    # 2. 120 wet/dry steps with tide on the 1,600-triangle rectangle (land film H0/2)
    m = dgrain.rectangle(40, 20, jitter=0.0, seed=1)
    z, qx, qy, wd = film_state(m, 0.5e-3)
    ref = O.Reference(wet_dry=True)
    ref.set_mesh(m)
    ref.initialize()
    ref.set_state(z, qx, qy, wd)
    rc, t, dt, n, hist = ref.run(120, 1e9, 0.3, tide_on=1, amp=0.5, want_dt=True)
    assert rc == 0 and n == 120
    s = ref.get_state()
    np.savez_compressed(os.path.join(HERE, "run120_wd_tide_rect1600.npz"),
                        **mesh_arrays(m), zeta0=z, qx0=qx, qy0=qy, wd0=wd, zeta=s[0], qx=s[1], qy=s[2], wd=s[3],
                        time=np.array(t), dt_next=np.array(dt), dt_hist=hist)

    # 3. the land film at exactly H0: the reference stops on a NaN flux
    z, qx, qy, wd = film_state(m, 1e-3)
    ref = O.Reference(wet_dry=True)
    ref.set_mesh(m)
    ref.initialize()
    ref.set_state(z, qx, qy, wd)
    rc, t, dt, n, hist = ref.run(50, 1e9, 0.3, tide_on=1, amp=0.5, want_dt=True)
    msg = ref.message()
    assert rc != 0
    edge = int(msg.split("edge")[1].split()[0])
    np.savez_compressed(os.path.join(HERE, "failure_film_h0_rect1600.npz"),
                        **mesh_arrays(m), zeta0=z, qx0=qx, qy0=qy, wd0=wd, steps_done=np.array(n),
                        fail_edge=np.array(edge), message=np.array(msg))
    print("written:", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))


if __name__ == "__main__":
    main()
