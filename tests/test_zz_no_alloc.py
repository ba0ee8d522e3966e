"""mdb_kinetic_sum_noalloc, the allocation-free thermo reduction.

It serves callers that own their device arrays and may not let a library
allocate device memory (a framework whose allocator has reserved the device's
memory, or a timed loop in which cudaMalloc would synchronise the device).
This test feeds it velocities that the test itself placed on the device and
checks, on two calls in a row with different states, that its sum gives the
same temperature as mdb_thermo on the same state, to 1e-12 relative (the two
reductions add in different orders). It lives in its own file, collected
last, so a failure here cannot hide failures of the other tests.
"""
import ctypes as C

import numpy as np
import pytest

import mdb

pytestmark = pytest.mark.gpu

REL = 1e-12


def _noalloc_temperature(torch, lib, v, natoms, mass=1.0):
    d_v = torch.from_numpy(np.ascontiguousarray(v, dtype=np.float64).reshape(-1)).cuda()
    d_out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.mdb_kinetic_sum_noalloc(C.c_void_p(d_v.data_ptr()), len(v), mass,
                                     C.c_void_p(d_out.data_ptr()), C.c_void_p(stream))
    assert rc == 0, lib.mdb_status_string(rc)
    torch.cuda.synchronize()
    return float(d_out.item()) / (natoms * 3 - 3)   # LJ: mvv2e = 1, dof = 3N - 3


def test_noalloc_kinetic_sum_matches_thermo_twice():
    torch = pytest.importorskip("torch")
    lib = mdb.load()
    hp = mdb.host_params(nx=12, ny=12, nz=12)
    x, v, t = mdb.create_fcc(hp)
    s = mdb.system_from_host(hp, len(t))
    s.set_atoms(x, v, t)
    s.setup()
    n = len(t)

    # call 1: the initial state
    _, v1, _, _ = s.atoms()
    T_ref = s.thermo()["T"]
    assert _noalloc_temperature(torch, lib, v1, n) == pytest.approx(T_ref, rel=REL)

    # call 2, right after, on a different state: the shared scratch must not
    # carry anything over from call 1
    s.run(25)
    _, v2, _, _ = s.atoms()
    T_ref2 = s.thermo()["T"]
    assert abs(T_ref2 - T_ref) > 1e-3
    assert _noalloc_temperature(torch, lib, v2, n) == pytest.approx(T_ref2, rel=REL)


def test_noalloc_rejects_more_atoms_than_its_scratch():
    torch = pytest.importorskip("torch")
    lib = mdb.load()
    d_out = torch.zeros(1, dtype=torch.float64, device="cuda")
    d_v = torch.zeros(3, dtype=torch.float64, device="cuda")
    # the size check fails before any device access
    rc = lib.mdb_kinetic_sum_noalloc(C.c_void_p(d_v.data_ptr()), 8388609, 1.0,
                                     C.c_void_p(d_out.data_ptr()), None)
    assert rc == 1  # MDB_ERR_ARG


def test_noalloc_many_partials_and_empty():
    """More than 1024 block partials (2.2M atoms: the final kernel's strided
    loop runs) against a float64 numpy sum, then n = 0, which must give 0 even
    though the shared scratch still holds the previous call's partials."""
    torch = pytest.importorskip("torch")
    lib = mdb.load()
    n = 2_200_000                      # 1,075 partials of 2,048 atoms
    rng = np.random.default_rng(7)
    v = rng.standard_normal((n, 3))
    mass = 1.5
    d_v = torch.from_numpy(v.reshape(-1)).cuda()
    d_out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        rc = lib.mdb_kinetic_sum_noalloc(C.c_void_p(d_v.data_ptr()), n, mass,
                                         C.c_void_p(d_out.data_ptr()), C.c_void_p(stream))
        assert rc == 0, lib.mdb_status_string(rc)
        torch.cuda.synchronize()
        want = float(np.sum(v * v) * mass)
        assert float(d_out.item()) == pytest.approx(want, rel=REL)
    rc = lib.mdb_kinetic_sum_noalloc(None, 0, mass, C.c_void_p(d_out.data_ptr()),
                                     C.c_void_p(stream))
    assert rc == 0, lib.mdb_status_string(rc)
    torch.cuda.synchronize()
    assert float(d_out.item()) == 0.0
