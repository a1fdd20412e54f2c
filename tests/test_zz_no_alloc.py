"""The allocation-free limiter entry point, dgr_slope_limiter_noalloc.

It exists for callers that may not allocate device memory — code handed its buffers by
a host framework or memory pool, or running where cudaMalloc/cudaFree are not allowed.
The caller owns every input and output (allocated here by torch, as such a host would);
the entry point's only scratch is its static device array.  Its output must equal the
context limiter's (dgr_slope_limiter) exactly — the tolerance every limiter test here
uses — on two calls in a row, the second one running over the scratch contents left by
the first.  This file is collected last so that a failure here stops a `-x` run only
after every other test has run.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import negative_zeros, signed_zero_state

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.int64)


def test_noalloc_limiter_matches_context_limiter(dgrain, oracle_mod):
    import torch

    lib = dgrain.load()
    m = dgrain.rectangle(60, 30, jitter=0.1, seed=13)
    dev = torch.device("cuda", 0)
    el2v = torch.from_numpy(m.el2v.ravel().copy()).to(dev)
    z = torch.from_numpy(m.z.copy()).to(dev)
    stream = torch.cuda.current_stream(dev)
    fired = 0
    for seed in (1, 2):  # two calls in a row
        st = signed_zero_state(dgrain, m, seed, nx=60)
        with dgrain.Solver(m) as s:  # the existing entry point
            s.upload_state(*st)
            s.SlopeLimiter()
            want = s.download_state()[:3]
        o = oracle_mod.Oracle(m)  # the reference's limiter, restated on the CPU
        o.set_state(*st)
        o.slope_limiter()
        for a, b in zip(want, o.get_state()[:3]):
            assert np.array_equal(bits(a), bits(b))
        d = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in st[:3]]
        rc = lib.dgr_slope_limiter_noalloc(m.num_el, m.num_nodes, C.c_void_p(el2v.data_ptr()),
                                           C.c_void_p(z.data_ptr()), C.c_void_p(d[0].data_ptr()),
                                           C.c_void_p(d[1].data_ptr()), C.c_void_p(d[2].data_ptr()), 1e-3,
                                           C.c_void_p(stream.cuda_stream))
        assert rc == 0
        torch.cuda.synchronize(dev)
        got = [t.cpu().numpy() for t in d]
        for a, b in zip(got, want):
            assert np.array_equal(bits(a), bits(b))  # bit patterns: the signs of zeros count
        fired += int((got[0] != st[0]).any())
        # the zero patch reached the output: the limited Qx holds zeros of both signs
        assert 0 < negative_zeros(got[1]) < int((got[1] == 0.0).sum())
    assert fired == 2  # the limiter changed both states


def test_noalloc_limiter_rejects_meshes_beyond_its_scratch(dgrain):
    import torch

    lib = dgrain.load()
    limit = 131072  # DGR_NOALLOC_MAX_NODES in include/dgrain.h
    t = torch.zeros(16, dtype=torch.float64, device="cuda")
    i = torch.zeros(16, dtype=torch.int32, device="cuda")
    p = C.c_void_p(t.data_ptr())
    rc = lib.dgr_slope_limiter_noalloc(1, limit + 1, C.c_void_p(i.data_ptr()), p, p, p, p, 1e-3, None)
    assert rc == dgrain._lib.DGR_ERR_TOO_LARGE
