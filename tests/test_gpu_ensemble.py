"""Batched ensemble (many meshes of uneven size in one context) and the schedules of the
device loop (block size x fusion depth).  Every scenario of an ensemble must give the
bits it gives alone, under every schedule; a failing scenario stops alone.

Scenarios are basins at 5 m resolution under water everywhere (the ensemble workload): the reference
wet/dry scheme runs them for thousands of steps with rain, whereas rain on dry land makes
it stop on a NaN flux within tens of steps."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import bits_equal, land_film_state

pytestmark = pytest.mark.gpu


def scenarios(dgrain, sizes=(600, 1900, 350, 4100, 1200), seed=0):
    rng = np.random.default_rng(seed)
    meshes, params, states = [], [], []
    for k, n in enumerate(sizes):
        m = dgrain.rectangle_with_elements(n, seed=100 + k, cell=5.0, datum=7.0)
        n_el = rng.uniform(0.02, 0.06, m.num_el) if k % 2 == 0 else None
        p = dict(tide_on=1, tide_amp=float(rng.uniform(0.2, 1.5)), tide_period=44712.0,
                 rain=float(rng.uniform(0, 100) / 3.6e6), n_el=n_el)
        meshes.append(m)
        params.append(p)
        states.append(land_film_state(dgrain, m))
    return meshes, params, states


def alone(dgrain, m, p, st, nsteps, schedule=(128, 0)):
    with dgrain.Solver(m, wet_dry=1, cfl=0.3, tide_on=p["tide_on"], tide_amp=p["tide_amp"],
                       tide_period=p["tide_period"], rain=p["rain"]) as s:
        if p["n_el"] is not None:
            s.set_element_manning(p["n_el"])
        s.set_schedule(*schedule)
        s.upload_state(*st)
        t, dt, n = s.time_evolution(1e300, nsteps)
        return (t, dt, n), s.download_state()


def test_ensemble_equals_scenarios_alone(dgrain):
    meshes, params, states = scenarios(dgrain)
    ref = [alone(dgrain, m, p, st, 25) for m, p, st in zip(meshes, params, states)]
    with dgrain.Ensemble(meshes, params, wet_dry=1, cfl=0.3) as e:
        for k, st in enumerate(states):
            e.upload_state(k, *st)
        t, dt, n = e.run(25)
        for k in range(len(meshes)):
            assert (t[k], dt[k], n[k]) == ref[k][0]
            for a, b in zip(e.download_state(k), ref[k][1]):
                assert bits_equal(a, b), k


@pytest.mark.parametrize("block_size", [64, 128, 256])
@pytest.mark.parametrize("fusion", [0, 1, 2])
def test_schedules_give_identical_bits(dgrain, block_size, fusion):
    meshes, params, states = scenarios(dgrain, sizes=(900, 2500, 400))
    base = None
    for sched in ((128, 0), (block_size, fusion)):
        with dgrain.Ensemble(meshes, params, wet_dry=1, cfl=0.3) as e:
            e.set_schedule(*sched)
            for k, st in enumerate(states):
                e.upload_state(k, *st)
            clock = e.run(12)
            out = [e.download_state(k) for k in range(len(meshes))]
        if base is None:
            base = (clock, out)
            continue
        for a, b in zip(clock, base[0]):
            assert bits_equal(a, b)
        for k in range(len(meshes)):
            for a, b in zip(out[k], base[1][k]):
                assert bits_equal(a, b), (sched, k)


def test_single_mesh_schedules_match_oracle(dgrain, oracle_mod, mesh_c1):
    """Fused single-mesh schedules against the oracle restatement (friction term zero, so
    bit-identical)."""
    m = dgrain.Mesh(**{f.name: getattr(mesh_c1, f.name) for f in __import__("dataclasses").fields(mesh_c1)})
    m.nfric = np.zeros_like(m.nfric)
    st = land_film_state(dgrain, m)
    o = oracle_mod.Oracle(m)
    o.set_state(*st)
    rc, t_o, dt_o, n_o, _ = o.run(60, 1e9, 0.3, wet_dry=1, tide_on=1, amp=0.5)
    assert rc == 0
    want = o.get_state()
    for sched in ((64, 2), (256, 1)):
        with dgrain.Solver(m, wet_dry=1, cfl=0.3, tide_on=1, tide_amp=0.5) as s:
            s.set_schedule(*sched)
            s.upload_state(*st)
            assert s.time_evolution(1e9, 60) == (t_o, dt_o, n_o)
            for a, b in zip(s.download_state(), want):
                assert bits_equal(a, b), sched


def test_autotune_keeps_state_and_picks_a_schedule(dgrain):
    meshes, params, states = scenarios(dgrain, sizes=(1500, 800))
    with dgrain.Ensemble(meshes, params, wet_dry=1, cfl=0.3) as e:
        for k, st in enumerate(states):
            e.upload_state(k, *st)
        t, dt, n = e.run(3)
        before = [e.download_state(k) for k in range(2)]
        bs, fu, table = e.autotune(trial_steps=3)
        assert bs in (64, 128, 256) and fu in (0, 1, 2)
        assert table[(bs, fu)] == min(v for v in table.values() if v > 0)
        assert e.get_schedule() == (bs, fu)
        for k in range(2):
            for a, b in zip(e.download_state(k), before[k]):
                assert bits_equal(a, b)
        t2, dt2, n2 = e.run(5, time=t, dt=dt)
        assert (n2 == 5).all()


def test_failing_scenario_stops_alone(dgrain):
    """A scenario that the reference scheme cannot run (land film at exactly H0) stops
    with the same failure as alone; the other scenarios finish every step."""
    meshes, params, states = scenarios(dgrain, sizes=(700, 1600, 900))
    m = dgrain.rectangle(40, 20, jitter=0.0, seed=1)
    bad_state = dgrain.initial_state(m, np.maximum(0.0, 1e-3 - m.z))
    pbad = dict(tide_on=1, tide_amp=0.5, tide_period=44712.0, rain=0.0, n_el=None)
    with dgrain.Solver(m, wet_dry=1, cfl=0.3, tide_on=1, tide_amp=0.5) as s:
        s.upload_state(*bad_state)
        with pytest.raises(dgrain.StepError) as ei:
            s.time_evolution(1e300, 20)
        want = (ei.value.code, ei.value.index, ei.value.step)
    meshes.insert(1, m)
    params.insert(1, pbad)
    states.insert(1, bad_state)
    with dgrain.Ensemble(meshes, params, wet_dry=1, cfl=0.3) as e:
        for k, st in enumerate(states):
            e.upload_state(k, *st)
        t, dt, n = e.run(20, check=False)
        assert e.last_error(1) == want
        assert n[1] == want[2]
        for k in (0, 2, 3):
            assert n[k] == 20 and e.last_error(k)[0] == 0
