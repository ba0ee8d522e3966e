"""Pins the cluster-pair oracle (oracle/mdb_oracle_cp.c) to the reference.

The reference's cluster-pair sources are compiled here three times by
oracle/Makefile: the scalar reference kernel (M x N = 1 x 2, exact FP64
forces), the AVX2 build (4 x 4) and the AVX-512 build (4 x 8); the SIMD builds'
forces use approximate reciprocals and serve only as cluster/list oracles. The
oracle must reproduce each build bit for bit: clusters (column order of equal-z
atoms included), j-clusters, ghost clusters, slot positions, j-cluster
columns and lists with their masks, on the lattice start and on disordered
states read from a dump; forces and whole trajectories against the exact 1x2
build. The reference's own tests/test_neighbor.c property (every j-cluster
whose box is within cutneigh is listed, none much farther) is checked too.
"""
import os

import numpy as np
import pytest

import mdb
import oracle as O

SHAPES = ["1x2", "4x4", "4x8"]


def need_ref(shape):
    if not O.ref_cp_available(shape):
        pytest.skip("reference cluster-pair build not available (oracle/_ref)")


def shape_mn(shape):
    return tuple(int(v) for v in shape.split("x"))


def oracle_like(ref, x, v, t, half=0, prune_every=1000):
    M, N = shape_mn_of(ref)
    p = ref.params()
    o = O.OracleCP(x, v, t, M=M, N=N, half=half, natoms=ref.counts()["natoms"],
                   prune_every=prune_every, **p)
    o.setup()
    o.force()  # the reference computes the force before its loop (the shim does too)
    return o


def shape_mn_of(ref):
    return ref.M, ref.N


def assert_same(ref, o, M):
    assert ref.counts() == o.counts()
    for a, b in zip(ref.iclusters(), o.iclusters()):
        assert np.array_equal(a, b)
    for a, b in zip(ref.jclusters(), o.jclusters()):
        assert np.array_equal(a, b)
    for a, b in zip(ref.ghosts(), o.ghosts()):
        assert np.array_equal(a, b)
    xs, vs, _, ts = ref.slots()
    xo, vo, _, to = o.slots()
    assert np.array_equal(xs, xo)
    assert np.array_equal(ts, to)
    nat, _, _ = o.iclusters()
    valid = np.concatenate([np.arange(M) < k for k in nat])
    assert np.array_equal(vs[:len(valid)][valid], vo[:len(valid)][valid])
    nn, nm, nb, im = ref.neighbor_list()
    nn2, nm2, nb2, im2 = o.neighbor_list()
    assert np.array_equal(nn, nn2) and np.array_equal(nm, nm2)
    for i in range(len(nn)):
        assert np.array_equal(nb[i, :nn[i]], nb2[i, :nn[i]]), i
        assert np.array_equal(im[i, :nn[i]], im2[i, :nn[i]]), i


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("half", [0, 1])
def test_lattice_setup_matches_reference(shape, half):
    need_ref(shape)
    ref = O.RefCP(shape, 8, 8, 8, half=half)
    x, v, t = ref.atoms()
    # the cluster-pair createAtom is the Verlet-list one: same lattice, same
    # seeded velocities, same rand() types
    vl = O.Oracle(nx=8, ny=8, nz=8)
    vl.lattice()
    xv, vv, _, tv = vl.atoms()
    assert np.array_equal(x, xv) and np.array_equal(v, vv) and np.array_equal(t, tv)
    o = oracle_like(ref, x, v, t, half=half)
    assert_same(ref, o, ref.M)


def _thermalised_dump(tmp_path, n, steps=150):
    vl = O.Oracle(nx=n, ny=n, nz=n)
    vl.lattice()
    vl.setup()
    vl.run(steps)
    x, v, _, t = vl.atoms()
    p = vl.params()
    path = str(tmp_path / f"state_{n}.dmp")
    mdb.write_dmp(path, x, v, t, (p["xprd"], p["yprd"], p["zprd"]))
    return path, x, v, t


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("half,n", [(0, 6), (1, 7)])
def test_disordered_state_matches_reference(tmp_path, shape, half, n):
    need_ref(shape)
    path, x, v, t = _thermalised_dump(tmp_path, n)
    ref = O.RefCP(shape, n, n, n, half=half, input_file=path)
    rx, rv, rt = ref.atoms()
    assert np.array_equal(rx, x) and np.array_equal(rv, v) and np.array_equal(rt, t)
    o = oracle_like(ref, rx, rv, rt, half=half)
    assert_same(ref, o, ref.M)
    nat, _, _ = o.iclusters()
    assert (nat < ref.M).any() or ref.M == 1


@pytest.mark.parametrize("half", [0, 1])
def test_exact_build_forces_and_trajectory(half):
    need_ref("1x2")
    ref = O.RefCP("1x2", 6, 6, 6, half=half)
    x, v, t = ref.atoms()
    o = oracle_like(ref, x, v, t, half=half)
    ref.force()
    o.force()
    nat, _, _ = o.iclusters()
    valid = np.concatenate([np.arange(1) < k for k in nat])
    fs = ref.slots()[2][:len(valid)][valid]
    fo = o.slots()[2][:len(valid)][valid]
    assert np.array_equal(fs, fo)
    for n in range(60):
        ref.step(n)
        o.step(n)
        if (n + 1) % 20 == 0:
            assert ref.thermo()["T"] == o.thermo()["T"]
            assert ref.thermo()["P"] == o.thermo()["P"]
    assert_same(ref, o, 1)


def test_prune_matches_reference():
    need_ref("1x2")
    ref = O.RefCP("1x2", 6, 6, 6, prune_every=7)
    x, v, t = ref.atoms()
    o = oracle_like(ref, x, v, t, prune_every=7)
    for n in range(30):
        ref.step(n)
        o.step(n)
    assert_same(ref, o, 1)


@pytest.mark.parametrize("shape", ["4x4", "4x8"])
def test_list_acceptance_rule(shape):
    """The list holds exactly the j-clusters whose box is within cutneigh and
    that are either within rbb or have an atom pair inside cutneigh
    (buildNeighborCPU, clusterpair/neighbor.c:423-483), checked by brute force
    on the 4x4x4 lattice of the reference's tests/test_neighbor.c. (That test's
    own claim, every box-close j-cluster listed, does not hold for the
    reference's lists: box-close clusters without a close atom pair are left
    out by the reference too.)"""
    M, N = shape_mn(shape)
    vl = O.Oracle(nx=4, ny=4, nz=4)
    vl.lattice()
    x, v, _, t = vl.atoms()
    p = vl.params()
    o = O.OracleCP(x, v, t, M=M, N=N, natoms=len(t), xprd=p["xprd"], yprd=p["yprd"],
                   zprd=p["zprd"], cutforce=p["cutforce"], cutneigh=p["cutneigh"])
    o.setup()
    _, _, ibb = o.iclusters()
    _, jbb = o.jclusters()
    nn, _, nb, _ = o.neighbor_list()
    xs = o.slots()[0]
    cut2 = p["cutneigh"] ** 2
    rbb2 = o.bin_geometry()["rbb_sq"]

    def d2(a, b):
        s = 0.0
        for lo, hi in ((4, 5), (2, 3), (0, 1)):
            dm = max(a[lo] - b[hi], b[lo] - a[hi], 0.0)
            s += dm * dm
        return s

    for ci in range(len(nn)):
        listed = set(nb[ci, :nn[ci]].tolist())
        xi = xs[ci * M:(ci + 1) * M]
        for cj in range(len(jbb)):
            dd = d2(ibb[ci], jbb[cj])
            want = False
            if dd < cut2:
                xj = xs[cj * N:(cj + 1) * N]
                r2 = ((xi[:, None, :] - xj[None, :, :]) ** 2).sum(-1)
                want = dd < rbb2 or bool((r2 < cut2).any())
            assert (cj in listed) == want, (ci, cj)


def test_scheme_equivalence_with_verlet_list():
    """tests/regression_scheme_equiv.sh: the cluster-pair scheme's T and P at
    step 200 within 2% / 5% of the Verlet-list scheme's on the same system."""
    vl = O.Oracle(nx=8, ny=8, nz=8)
    vl.lattice()
    x, v, _, t = vl.atoms()
    p = vl.params()
    vl.setup()
    vl.run(200)
    tv = vl.thermo()
    for M, N in ((4, 4), (4, 8)):
        o = O.OracleCP(x, v, t, M=M, N=N, natoms=len(t), xprd=p["xprd"], yprd=p["yprd"],
                       zprd=p["zprd"], cutforce=p["cutforce"], cutneigh=p["cutneigh"],
                       dt=p["dt"], dtforce=p["dtforce"])
        o.setup()
        o.force()
        o.run(200)
        o.lib.orccp_update_single_atoms(o.h)  # the reference's final updateAtoms
        tc = o.thermo()
        assert abs(tc["T"] - tv["T"]) <= 0.02 * abs(tv["T"])
        assert abs(tc["P"] - tv["P"]) <= 0.05 * abs(tv["P"])
