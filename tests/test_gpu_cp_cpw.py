"""Several i-clusters per warp in the mixed cluster-pair kernel (force_cpw).

force_cpw 2, 4 and 8 give each i-cluster a segment of 16, 8 or 4 lanes
instead of a warp (8: 4x4 clusters only). They evaluate the same pairs of the same list, so their forces equal
force_cpw 1's up to FP32 summation order (the split of a row among lanes
differs), for 4x4 and 4x8 clusters, half and full lists, one and four atom
types, with energies; trajectories stay within the mixed path's budget of the
FP64 oracle's forces. Ensemble members keep their setting in batched
launches.
"""
import numpy as np
import pytest

import mdb
import oracle as O
from test_gpu_cp_pairs import MIXED_RMS, SUM_ORDER, rel, system, valid_forces

pytestmark = pytest.mark.gpu

C5_TYPES = ([0.5, 1.5, 0.8, 1.2], [0.8, 1.2, 1.0, 0.9])


def forces(s, cpw, energy=True, jpl=1):
    s.tune("force_cpw", cpw)
    s.tune("force_jpl", jpl)
    s.compute_force(energy=energy)
    return valid_forces(s), (s.thermo()["PE"] if energy else None)


@pytest.mark.parametrize("N", [4, 8])
@pytest.mark.parametrize("half", [0, 1])
@pytest.mark.parametrize("types", [None, C5_TYPES], ids=["one_type", "four_types"])
def test_cpw_matches_one_cluster_per_warp(N, half, types):
    s, _ = system(7, N, half, steps=120, types=types)
    f1, e1 = forces(s, 1)
    for cpw, jpl in ((2, 1), (4, 1), (4, 2)) + (((8, 1),) if N == 4 else ()):
        f, e = forces(s, cpw, jpl=jpl)
        r, m = rel(f, f1)
        assert r <= SUM_ORDER and m <= 10 * SUM_ORDER, (cpw, jpl, r, m)
        assert e == pytest.approx(e1, rel=1e-6)


@pytest.mark.parametrize("half", [0, 1])
def test_cpw_against_fp64_oracle(half):
    """force_cpw 2 and 4 on a melted state against the FP64 oracle's forces."""
    n = 8
    o0 = O.Oracle(nx=n, ny=n, nz=n)
    o0.lattice()
    o0.setup()
    o0.run(200)
    x, v, _, t = o0.atoms()
    hp = mdb.host_params(nx=n, ny=n, nz=n)
    mdb.create_fcc(hp)
    common = dict(xprd=hp.xprd, yprd=hp.yprd, zprd=hp.zprd, cutforce=hp.cutforce,
                  cutneigh=hp.cutneigh, dt=hp.dt, dtforce=hp.dtforce, mass=hp.mass,
                  epsilon=hp.epsilon, sigma=hp.sigma, ntypes=hp.ntypes)
    o = O.OracleCP(x, v, t, M=4, N=4, half=half, natoms=len(t), **common)
    o.setup()
    o.force()
    nat = o.iclusters()[0]
    ok = np.concatenate([np.arange(4) < k for k in nat])
    fo = o.slots()[2][:len(ok)][ok]
    s = mdb.ClusterSystem(natoms=len(t), cluster_n=4, half_neigh=half, precision="mixed",
                          **common)
    s.set_atoms(x, v, t)
    s.setup()
    for cpw, jpl in ((2, 1), (4, 1), (4, 2), (8, 1)):
        f, _ = forces(s, cpw, energy=False, jpl=jpl)
        r, m = rel(f, fo)
        assert r <= MIXED_RMS and m <= 20 * MIXED_RMS, (cpw, jpl, r, m)


def test_cpw_trajectory_tracks_one_cluster_per_warp():
    """100 steps from the lattice (five rebuilds) with force_cpw 1 and 2: the
    temperatures agree as two mixed runs that differ in summation order."""
    a, _ = system(6, 4, 1)
    b, _ = system(6, 4, 1)
    a.tune("force_cpw", 1)
    b.tune("force_cpw", 2)
    a.run(100, max_samples=0)
    b.run(100, max_samples=0)
    assert b.thermo()["T"] == pytest.approx(a.thermo()["T"], rel=1e-3)


def test_ensemble_members_keep_their_cpw():
    """A batched ensemble whose members run 1, 2, 4 and 8 i-clusters per warp
    (four force groups): full-list members follow their solo twins with the
    same setting bit for bit."""
    from test_gpu_cp import replica
    cfg = [(4, 0.84, 1.44, 1), (5, 0.80, 1.0, 2), (4, 0.90, 1.6, 4), (6, 0.76, 0.8, 8)]
    pairs = []
    for n, rho, T, cpw in cfg:
        a, b = replica(n, rho, T, 4, "mixed")
        a.tune("force_cpw", cpw)
        b.tune("force_cpw", cpw)
        pairs.append((a, b))
    ens = mdb.Ensemble([p[0] for p in pairs])
    got = ens.run(45, max_samples=8)
    for k, (a, b) in enumerate(pairs):
        want = b.run(45, max_samples=8)
        assert got[k] == want, k
        xa, va, _ = a.atoms()
        xb, vb, _ = b.atoms()
        assert np.array_equal(xa, xb) and np.array_equal(va, vb), k
    ens.close()


def test_cpw_rejects_bad_values():
    s, _ = system(4, 4, 0)
    for bad in (0, 3, 16):
        with pytest.raises(mdb.MdbError):
            s.tune("force_cpw", bad)
    s.tune("force_cpw", 8)
    w, _ = system(4, 8, 0)
    with pytest.raises(mdb.MdbError):  # a 4-lane segment is narrower than a 4x8 j-cluster
        w.tune("force_cpw", 8)
