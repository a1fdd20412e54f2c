"""Channel <-> junction coupling on the device (dgr_set_channel_ends / dgr_couple_channel_ends,
ChanNet/internal_BC.c) against the oracle's restatement, which test_coupling.py pins to the
reference build:
  * one coupling pass: the coupled edges' bzeta / bQn and the channel ends' ghost (A, Q)
    bit for bit, on random states;
  * a coupled run: per step, the ends' traces follow a hydrograph, the coupling pass feeds
    the junction's prescribed edges and the junction takes a wet/dry step (the ChanNet
    order); ghosts and the junction state stay bit-identical to the oracle's loop;
  * invalid channel-end lists are refused.
"""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from conftest import bits_equal
from test_coupling import coupling_case

pytestmark = pytest.mark.gpu


def prescribed(dgrain, m, chans, friction=True):
    """the mesh with the channels' edges marked as the reference marks them
    (BdryPrescribed 1: inflow channel, 2: outflow channel)"""
    m2 = dgrain.Mesh(**{f.name: getattr(m, f.name) for f in dataclasses.fields(m)})
    m2.bdry = m.bdry.copy()
    for _, _, e_in, e_out in chans:
        m2.bdry[np.asarray(e_in, dtype=int)] = 1
        m2.bdry[np.asarray(e_out, dtype=int)] = 2
    if not friction:
        m2.nfric = np.zeros_like(m.nfric)
    return m2


def ends_of(chans):
    """(edges, outflow) per channel end, and the channel index and trace slot of each"""
    ends, where = [], []
    for ch, (A, _, e_in, e_out) in enumerate(chans):
        if len(e_in):
            ends.append((e_in, 0))
            where.append((ch, 1, 0))
        if len(e_out):
            ends.append((e_out, 1))
            where.append((ch, len(A) - 2, len(A) - 1))
    return ends, where


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_coupling_pass_equals_oracle(dgrain, oracle_mod, seed):
    m0, (zeta, qx, qy), bz, bq, chans = coupling_case(dgrain, seed=seed, nchan=5)
    m = prescribed(dgrain, m0, chans)
    ends, where = ends_of(chans)
    bz2, bq2, outs = oracle_mod.internal_bc(m, zeta, qx, qy, bz, bq, chans)
    with dgrain.Solver(m, wet_dry=1) as s:
        s.upload_state(zeta, qx, qy)
        s.set_boundary(bz, bq)
        s.set_channel_ends(ends)
        a_end = np.array([chans[ch][0][i] for ch, i, _ in where])
        q_end = np.array([chans[ch][1][i] for ch, i, _ in where])
        ag, qg = s.couple_channel_ends(a_end, q_end)
        dbz, dbq = s.get_boundary()
    for k, (ch, _, g) in enumerate(where):
        assert ag[k] == outs[ch][0][g] and qg[k] == outs[ch][1][g], k
    coupled = np.concatenate([np.asarray(e, dtype=int) for e, _ in ends])
    assert bits_equal(dbz[coupled], bz2[coupled])
    assert bits_equal(dbq[coupled], bq2[coupled])
    # the other prescribed edges keep what dgr_set_boundary gave them
    other = np.setdiff1d(np.flatnonzero(m.bdry != 0), coupled)
    assert bits_equal(dbz[other], bz[other]) and bits_equal(dbq[other], bq[other])


@pytest.mark.parametrize("friction", [False, True])
def test_coupled_run_matches_oracle(dgrain, oracle_mod, friction):
    m0, _, _, _, chans = coupling_case(dgrain, nx=24, ny=12, seed=11, nchan=3, datum=7.0)
    m = prescribed(dgrain, m0, chans, friction=friction)
    ends, where = ends_of(chans)
    cx, cy = m.x.mean(), m.y.mean()
    st = dgrain.initial_state(m, 0.3 * np.exp(-((m.x - cx) ** 2 + (m.y - cy) ** 2) / (2 * 1500.0 ** 2)))
    o = oracle_mod.Oracle(m)
    o.set_state(*st)
    o.boundary_conditions()
    chans = [(A.copy(), Q.copy(), e_in, e_out) for A, Q, e_in, e_out in chans]
    base = [(chans[ch][0][i], chans[ch][1][i]) for ch, i, _ in where]
    time, dt, nsteps = 0.0, 2.0, 40
    with dgrain.Solver(m, wet_dry=1) as s:
        s.upload_state(*st)
        s.set_boundary(*o.get_bc())
        s.set_channel_ends(ends)
        for n in range(nsteps):
            time += dt
            # the channels' traces at the junction: a hydrograph in place of the 1D solver
            a_end = np.array([a * (1.0 + 0.1 * np.sin(0.05 * time + k)) for k, (a, _) in enumerate(base)])
            q_end = np.array([q * np.cos(0.03 * time + k) for k, (_, q) in enumerate(base)])
            for k, (ch, i, _) in enumerate(where):
                chans[ch][0][i] = a_end[k]
                chans[ch][1][i] = q_end[k]
            ag, qg = s.couple_channel_ends(a_end, q_end)
            s.oneTimeStep2D(time, dt)
            z, x, y, _ = o.get_state()
            bz, bq = o.get_bc()
            bz, bq, outs = oracle_mod.internal_bc(m, z, x, y, bz, bq, chans)
            o.set_bc(bz, bq)
            rc, _ = o.step(time, dt, wet_dry=1)
            assert rc == 0
            for k, (ch, _, g) in enumerate(where):
                if friction:
                    assert abs(ag[k] - outs[ch][0][g]) <= 1e-11 * abs(outs[ch][0][g])
                else:
                    assert ag[k] == outs[ch][0][g] and qg[k] == outs[ch][1][g], (n, k)
        got, want = s.download_state(), o.get_state()
    assert bits_equal(got[3], want[3])
    for a, b in zip(got[:3], want[:3]):
        if friction:
            assert np.abs(a - b).max() <= 1e-11 * max(np.abs(b).max(), 1e-300)
        else:
            assert bits_equal(a, b)
    # the channels moved water: the junction is no longer the initial state
    assert not bits_equal(got[1], st[1])


def test_channel_end_lists_are_checked(dgrain):
    m0, _, _, _, chans = coupling_case(dgrain, seed=4)
    m = prescribed(dgrain, m0, chans)
    ends, _ = ends_of(chans)
    land = np.flatnonzero((m.ed2el[:, 0] == m.ed2el[:, 1]) & (m.bdry == 0))
    interior = np.flatnonzero(m.ed2el[:, 0] != m.ed2el[:, 1])
    e0 = np.asarray(ends[0][0], dtype=np.int32)
    with dgrain.Solver(m, wet_dry=1) as s:
        for bad in ([(np.array([land[0]]), 0)],          # not a prescribed edge
                    [(np.array([interior[0]]), 1)],      # interior edge
                    [(e0, 0), (e0[:1], 1)],              # one edge on two ends
                    [(np.array([m.num_edges]), 0)],      # out of range
                    [(e0, 2)],                           # end kind
                    [(np.zeros(0, np.int32), 0)]):       # empty end
            with pytest.raises(Exception):
                s.set_channel_ends(bad)
        s.set_channel_ends(ends)
        s.set_channel_ends([])      # removes the coupling
        assert s.couple_channel_ends(np.zeros(0), np.zeros(0))[0].size == 0


def test_device_buffer_pass_equals_host_pass(dgrain):
    """dgr_couple_channel_ends_device on torch CUDA buffers, ordered through the context's
    stream, gives the host-array pass's ghosts and boundary values bit for bit."""
    import torch

    m0, (zeta, qx, qy), bz, bq, chans = coupling_case(dgrain, seed=5, nchan=5)
    m = prescribed(dgrain, m0, chans)
    ends, where = ends_of(chans)
    a_end = np.array([chans[ch][0][i] for ch, i, _ in where])
    q_end = np.array([chans[ch][1][i] for ch, i, _ in where])
    with dgrain.Solver(m, wet_dry=1) as s:
        s.upload_state(zeta, qx, qy)
        s.set_boundary(bz, bq)
        s.set_channel_ends(ends)
        ag, qg = s.couple_channel_ends(a_end, q_end)
        hb = s.get_boundary()
        s.set_boundary(bz, bq)
        dev = torch.device("cuda", 0)
        da, dq = torch.tensor(a_end, device=dev), torch.tensor(q_end, device=dev)
        dga, dgq = torch.empty_like(da), torch.empty_like(dq)
        torch.cuda.synchronize()
        s.couple_channel_ends_device(da, dq, dga, dgq)
        torch.cuda.ExternalStream(s.stream()).synchronize()
        db = s.get_boundary()
    assert bits_equal(dga.cpu().numpy(), ag) and bits_equal(dgq.cpu().numpy(), qg)
    assert bits_equal(db[0], hb[0]) and bits_equal(db[1], hb[1])


def test_device_buffer_pass_accepts_pinned_host_memory(dgrain):
    """Pinned host buffers are addressable by the kernel (unified addressing), so the
    device-buffer pass takes them and gives the host pass's ghosts."""
    import torch

    m0, (zeta, qx, qy), bz, bq, chans = coupling_case(dgrain, seed=6, nchan=4)
    m = prescribed(dgrain, m0, chans)
    ends, where = ends_of(chans)
    a_end = np.array([chans[ch][0][i] for ch, i, _ in where])
    q_end = np.array([chans[ch][1][i] for ch, i, _ in where])
    with dgrain.Solver(m, wet_dry=1) as s:
        s.upload_state(zeta, qx, qy)
        s.set_channel_ends(ends)
        ag, qg = s.couple_channel_ends(a_end, q_end)
        pa = torch.tensor(a_end).pin_memory()
        pq = torch.tensor(q_end).pin_memory()
        ga, gq = torch.empty_like(pa).pin_memory(), torch.empty_like(pq).pin_memory()
        s.couple_channel_ends_device(pa, pq, ga, gq)
        torch.cuda.ExternalStream(s.stream()).synchronize()
    assert bits_equal(ga.numpy(), ag) and bits_equal(gq.numpy(), qg)
