"""The C ABI without a GPU: the library loads, exports every entry point that
include/dgrain.h declares, and its host-side functions (fort.14 reader, connectivity,
initial state, .dat writer) behave like the reference's."""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, has_gpu


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "dgrain.h")).read()
    return sorted(set(re.findall(r"^DGR_API [^;(]*?\b(dgr_\w+)\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol(dgrain):
    lib = dgrain.load()
    names = declared_symbols()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n
    bound = {n for n, _, _ in dgrain._lib.SIGNATURES}
    assert set(names) == bound, set(names) ^ bound
    assert lib.dgr_abi_version() == 1
    assert dgrain._lib.status_string(1) == "numerical flux not a number"


def test_fort14_roundtrip_and_connectivity(dgrain, tmp_path):
    m = dgrain.rectangle(9, 5, jitter=0.1, seed=2)
    p = str(tmp_path / "a.14")
    dgrain.write_fort14(m, p)
    m2 = dgrain.read_fort14(p)
    for k in ("x", "y", "z", "nfric", "el2v", "outflow", "ed2v", "ed2el", "bdry"):
        assert np.array_equal(getattr(m, k), getattr(m2, k)), k
    assert m.min_edge == m2.min_edge
    assert m.num_edges == m.num_nodes + m.num_el - 1
    # boundary edges repeat their element; interior edges list the lower element first
    bd = m.ed2el[:, 0] == m.ed2el[:, 1]
    assert bd.sum() == 2 * (9 + 5)
    assert np.all(m.ed2el[~bd, 0] < m.ed2el[~bd, 1])
    assert (m.bdry == 2).sum() == 5


def test_fort14_errors(dgrain, tmp_path):
    p = tmp_path / "bad.14"
    p.write_text("title\n2 3\n1 0 0 0 0.03\n")
    with pytest.raises(dgrain.DgrError) as ei:
        dgrain.read_fort14(str(p))
    assert ei.value.code == dgrain._lib.DGR_ERR_IO
    with pytest.raises(dgrain.DgrError):
        dgrain.read_fort14(str(tmp_path / "missing.14"))


def test_mesh_breaking_euler_relation_is_rejected(dgrain):
    # two separate triangles: NumEdges (6) != NumNodes + NumEl - 1 (7)
    m = dgrain.Mesh(x=np.array([0, 1, 0, 5, 6, 5.0]), y=np.array([0, 0, 1, 0, 0, 1.0]), z=np.zeros(6),
                    nfric=np.zeros(6), el2v=np.array([[0, 1, 2], [3, 4, 5]], dtype=np.int32),
                    inflow1=np.zeros((0, 2), np.int32), inflow2=np.zeros((0, 2), np.int32),
                    outflow=np.zeros((0, 2), np.int32))
    with pytest.raises(dgrain.DgrError) as ei:
        dgrain.build_connectivity(m)
    assert ei.value.code == dgrain._lib.DGR_ERR_MESH


def test_initial_state_and_dat_writer(dgrain, tmp_path):
    m = dgrain.rectangle(4, 2, seed=1)
    z, qx, qy, wd = dgrain.initial_state(m, np.arange(m.num_nodes, dtype=np.float64))
    el = 3
    v = m.el2v[el]
    assert z[3 * el] == 0.5 * (v[0] + v[1]) and z[3 * el + 2] == 0.5 * (v[2] + v[0])
    assert not qx.any() and not qy.any() and (wd == -1).all()
    lib = dgrain.load()
    p = str(tmp_path / "001_H.dat")
    assert lib.dgr_write_dat(p.encode(), m.num_el, z.ctypes.data_as(dgrain._lib.dptr)) == 0
    lines = open(p).read().splitlines()
    assert len(lines) == m.num_el
    assert lines[0] == "\t\t".join("%1.15f" % x for x in z[:3]) + "\t\t"


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU path")
def test_device_calls_fail_loudly_without_gpu(dgrain):
    m = dgrain.rectangle(4, 2, seed=1)
    with pytest.raises(dgrain.DgrError) as ei:
        dgrain.Solver(m)
    assert ei.value.code == dgrain._lib.DGR_ERR_NO_DEVICE
    p = dgrain.default_params()
    assert p.g == 9.81 and p.H0 == 1e-3 and p.VELZERO == 1e-2 and p.cfl == 0.1 and p.dt0 == 1e-7


def test_coupling_entry_points_check_their_arguments(dgrain):
    """The coupling entry points refuse a missing context or missing arrays before any
    device work (no GPU needed)."""
    lib = dgrain.load()
    inv = dgrain._lib.DGR_ERR_INVALID
    one = (C.c_int * 2)(0, 1)
    d = (C.c_double * 1)(0.0)
    assert lib.dgr_set_channel_ends(None, 1, one, one, one) == inv
    assert lib.dgr_couple_channel_ends(None, d, d, d, d) == inv
    assert lib.dgr_couple_channel_ends_device(None, None, None, None, None) == inv
    assert lib.dgr_get_boundary(None, d, d) == inv
    p = C.c_void_p()
    assert lib.dgr_get_stream(None, C.byref(p)) == inv
    assert lib.dgr_set_barrier_wait(None, 1000, 0) == inv


def test_pointer_rule_of_the_device_buffer_entry_points(tmp_path):
    """The rule dgr_couple_channel_ends_device and dgr_slope_limiter_noalloc apply to a
    caller's pointer before launching (dg-rain_b200/csrc/dgr_ptr.h), on attribute values a
    one-GPU machine cannot produce: another GPU's buffer is refused even though it is
    device memory, and so are unmapped or pageable host memory."""
    import subprocess

    here = os.path.dirname(os.path.abspath(__file__))
    lib_path = str(tmp_path / "libptr_host.so")
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", cuda_inc, "-o", lib_path,
                    os.path.join(here, "ptr_host.cpp")], check=True)
    lib = C.CDLL(lib_path)
    lib.dgr_t_may_access.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int]
    types = (C.c_int * 4)()
    lib.dgr_t_memory_types(types)
    unregistered, host, device, managed = list(types)
    p = 0x7f0000001000
    ok = lambda t, owner, dptr, dev: bool(lib.dgr_t_may_access(t, owner, dptr, p, dev))  # noqa: E731
    assert ok(device, 0, p, 0) and ok(device, 3, p, 3)
    assert not ok(device, 1, p, 0)          # another GPU's memory
    assert not ok(device, 0, p + 256, 0)    # not addressable at this address
    assert ok(managed, 0, p, 2)             # managed memory, mapped where the kernel runs
    assert ok(host, 0, p, 0)                # pinned and mapped (unified addressing)
    assert not ok(host, 0, None, 0)         # pinned but not mapped
    assert not ok(unregistered, 0, None, 0) and not ok(unregistered, 0, p, 0)  # pageable memory


def test_restart_file_round_trip_and_errors(dgrain, tmp_path):
    """dgr_write_restart / dgr_read_restart: every value comes back with the same bits
    (signed zeros, subnormals, the extremes), the flags and the clock too; a file of another
    mesh size or order, or a damaged one, is refused."""
    lib = dgrain.load()
    from dgrain.mesh import _dp, _ip

    rng = np.random.default_rng(4)
    for ne, nm in ((7, 3), (5, 6)):
        n = ne * nm
        vals = [rng.standard_normal(n) * 10.0 ** rng.integers(-300, 300, n) for _ in range(3)]
        vals[0][:4] = [-0.0, 0.0, 5e-324, -1.7976931348623157e308]
        vals[1][:2] = [1 / 3, -2.2250738585072014e-308]
        wd = rng.integers(-1, 2, ne).astype(np.int32)
        path = str(tmp_path / f"r{nm}.rst").encode()
        assert lib.dgr_write_restart(path, ne, nm, *[_dp(v) for v in vals], _ip(wd), 1234.5678, 0.1 / 3) == 0
        got = [np.empty(n) for _ in range(3)]
        gwd = np.empty(ne, dtype=np.int32)
        t, d = C.c_double(), C.c_double()
        assert lib.dgr_read_restart(path, ne, nm, *[_dp(g) for g in got], _ip(gwd), C.byref(t), C.byref(d)) == 0
        for a, b in zip(got, vals):
            assert np.array_equal(a.view(np.int64), b.view(np.int64))
        assert np.array_equal(gwd, wd) and t.value == 1234.5678 and d.value == 0.1 / 3
        # another mesh size or order
        assert lib.dgr_read_restart(path, ne + 1, nm, *[_dp(g) for g in got], _ip(gwd), C.byref(t),
                                    C.byref(d)) == dgrain._lib.DGR_ERR_MESH
        # a file cut short
        text = open(path, "rb").read()
        bad = str(tmp_path / "cut.rst").encode()
        open(bad, "wb").write(text[: len(text) // 2])
        assert lib.dgr_read_restart(bad, ne, nm, *[_dp(g) for g in got], _ip(gwd), C.byref(t),
                                    C.byref(d)) == dgrain._lib.DGR_ERR_IO
    assert lib.dgr_read_restart(str(tmp_path / "none.rst").encode(), 7, 3, *[_dp(g) for g in got[:3]], _ip(gwd),
                                C.byref(t), C.byref(d)) in (dgrain._lib.DGR_ERR_IO, dgrain._lib.DGR_ERR_INVALID)
