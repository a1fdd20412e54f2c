"""The bounded wait of the persistent kernels' grid barrier (fusion 1 and 2).

Every wait on the device is bounded: a block that polls the barrier max_polls times gives
up, every block leaves the launch, and the run returns DGR_ERR_TIMEOUT instead of hanging
the GPU (the reference has no device waits; its failures end the process,
2DCode/compute2DL.c:245-302, and here they are statuses).  These tests make the wait run
out on purpose through dgr_set_barrier_wait's phantom block (a barrier that also waits for
a block that never arrives), which faults nothing, and check that the context stays
usable: the next run, back at the default bound, is bit-identical to a run that never
timed out.
"""
from __future__ import annotations

import time

import numpy as np
import pytest

from conftest import bits_equal, land_film_state

pytestmark = pytest.mark.gpu

POLLS = 1000  # about a millisecond of polling per wait, against the default second


def _reference_run(dgrain, m, st, steps):
    with dgrain.Solver(m, wet_dry=1, cfl=0.3, tide_on=1, tide_amp=0.5) as s:
        s.upload_state(*st)
        clock = s.time_evolution(1e9, steps)
        return clock, s.download_state()


@pytest.mark.parametrize("fusion", [1, 2])
def test_barrier_wait_runs_out_and_context_recovers(dgrain, fusion):
    m = dgrain.rectangle(60, 30, jitter=0.1, seed=3)
    st = land_film_state(dgrain, m)
    want_clock, want = _reference_run(dgrain, m, st, 12)
    with dgrain.Solver(m, wet_dry=1, cfl=0.3, tide_on=1, tide_amp=0.5) as s:
        s.set_schedule(128, fusion)
        s.upload_state(*st)
        s.time_evolution(1e9, 1)  # builds and warms the fused launch
        s.set_barrier_wait(POLLS, 1)
        s.upload_state(*st)
        t0 = time.perf_counter()
        with pytest.raises(dgrain.DgrError) as ei:
            s.time_evolution(1e9, 3)
        elapsed = time.perf_counter() - t0
        assert ei.value.code == dgrain._lib.DGR_ERR_TIMEOUT
        assert elapsed < 2.0  # the bounded wait, not the default bound of about a second per wait
        s.set_barrier_wait()  # back to the default bound, no phantom block
        s.upload_state(*st)
        assert s.time_evolution(1e9, 12) == want_clock
        for a, b in zip(s.download_state(), want):
            assert bits_equal(a, b)


def test_ensemble_barrier_wait_runs_out_and_recovers(dgrain):
    meshes = [dgrain.rectangle(40, 20, jitter=0.1, seed=k, datum=7.0) for k in (1, 2)]
    states = [dgrain.initial_state(m, np.maximum(0.0, 0.5e-3 - m.z)) for m in meshes]

    def run(e, steps):
        for k, st in enumerate(states):
            e.upload_state(k, *st)
        clock = e.run(steps)
        return clock, [e.download_state(k) for k in range(len(meshes))]

    with dgrain.Ensemble(meshes, wet_dry=1, cfl=0.3) as e:
        want_clock, want = run(e, 8)
    with dgrain.Ensemble(meshes, wet_dry=1, cfl=0.3) as e:
        e.set_schedule(64, 1)
        e.set_barrier_wait(POLLS, 1)
        with pytest.raises(dgrain.DgrError) as ei:
            run(e, 2)
        assert ei.value.code == dgrain._lib.DGR_ERR_TIMEOUT
        e.set_barrier_wait()
        got_clock, got = run(e, 8)
    for a, b in zip(got_clock, want_clock):
        assert bits_equal(a, b)
    for a, b in zip(got, want):
        for x, y in zip(a, b):
            assert bits_equal(x, y)
