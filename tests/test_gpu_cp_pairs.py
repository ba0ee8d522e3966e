"""The pair-list force path of the mixed cluster-pair scheme (force_path 1).

It evaluates only the pairs of the listed cluster pairs that were within
r_c + buffer of each other when their codes were last derived, and re-derives
inside the timestep whenever an atom has moved more than buffer / 2 since. The
pairs inside r_c are then exactly those the cluster-pair kernel (force_path 0)
evaluates, so on the same state and list the two paths agree up to FP32
summation order; a missed pair would show as an error of order 1e-3 of the
force scale on its atoms. Checked here on thermalised and hot systems, after
runs long enough to need several re-derivations, for 4x4 and 4x8 clusters,
half and full lists, one and four atom types; and against the FP64 oracle
within the mixed path's error budget.
"""
import numpy as np
import pytest

import mdb
import oracle as O

pytestmark = pytest.mark.gpu

SUM_ORDER = 2e-6   # FP32 summation order: RMS and max relative to the RMS force
MIXED_RMS = 1e-5


def system(n, N, half, rho=0.8442, temp=1.44, types=None, precision="mixed", steps=0):
    extra = {}
    if types is not None:
        import workloads as W
        extra = dict(types=types, cutforce=W.c5_cutoff(types[1]))
    hp = mdb.host_params(nx=n, ny=n, nz=n, rho=rho, temp=temp, **extra)
    x, v, t = mdb.create_fcc(hp)
    kw = dict(xprd=hp.xprd, yprd=hp.yprd, zprd=hp.zprd, cutforce=hp.cutforce,
              cutneigh=hp.cutneigh, dt=hp.dt, dtforce=hp.dtforce, mass=hp.mass,
              reneigh_every=hp.reneigh_every, nstat=hp.nstat, natoms=len(t), cluster_n=N,
              half_neigh=half, ntypes=hp.ntypes)
    if types is not None:
        kw.update(epsilon_per_type=list(types[0]), sigma_per_type=list(types[1]))
    s = mdb.ClusterSystem(precision=precision, **kw)
    s.set_atoms(x, v, t)
    s.setup()
    if steps:
        s.run(steps, max_samples=0)
        xa, va, ta = s.atoms()
        s.set_atoms(xa, va, ta)
        s.setup()
    return s, kw


def valid_forces(s):
    nat = s.iclusters()[0]
    ok = np.concatenate([np.arange(4) < k for k in nat])
    return s.slots()[2][:len(ok)][ok]


def rel(f, fref):
    rms = np.sqrt(np.mean(np.sum(fref * fref, axis=1)))
    d = np.sqrt(np.sum((f - fref) ** 2, axis=1))
    return np.sqrt(np.mean(d * d)) / rms, d.max() / rms


def both_paths(s, energy=False):
    """Forces of the current state and list from the pair path, then from the
    cluster-pair kernel (the context is left on the cluster-pair kernel)."""
    s.tune("force_path", 1)
    s.compute_force(energy=energy)
    fp = valid_forces(s)
    pe_p = s.thermo()["PE"] if energy else None
    s.tune("force_path", 0)
    s.compute_force(energy=energy)
    fc = valid_forces(s)
    pe_c = s.thermo()["PE"] if energy else None
    return fp, fc, pe_p, pe_c


@pytest.mark.parametrize("N", [4, 8])
@pytest.mark.parametrize("half", [0, 1])
def test_pair_path_matches_cluster_kernel(N, half):
    s, _ = system(8, N, half, steps=150)
    fp, fc, pe_p, pe_c = both_paths(s, energy=True)
    r, m = rel(fp, fc)
    assert r <= SUM_ORDER and m <= 20 * SUM_ORDER, (r, m)
    assert pe_p == pytest.approx(pe_c, rel=1e-6)


@pytest.mark.parametrize("N", [4, 8])
def test_pair_path_multitype(N):
    import workloads as W
    s, _ = system(7, N, 1, types=W.c5_types(), steps=100)
    fp, fc, pe_p, pe_c = both_paths(s, energy=True)
    r, m = rel(fp, fc)
    assert r <= SUM_ORDER and m <= 20 * SUM_ORDER, (r, m)
    assert pe_p == pytest.approx(pe_c, rel=1e-6)


@pytest.mark.parametrize("N,half", [(4, 1), (4, 0), (8, 1)])
def test_pair_path_no_pair_missed_over_a_hot_run(N, half):
    """A hot dense liquid (rho 0.95, T 2.0): atoms cross half the buffer within a
    few steps, so the codes are re-derived many times between rebuilds. At
    several points of the run (inside rebuild periods, where the codes are
    oldest) the forces the run computed equal the cluster-pair kernel's on the
    same state and list."""
    s, _ = system(8, N, half, rho=0.95, temp=2.0)
    s.tune("force_path", 1)
    d0, _ = s.pair_stats()
    done = 0
    for k in (7, 12, 26, 39):
        s.run(k - done, first_step=done, max_samples=0)
        done = k
        fp = valid_forces(s)
        s.tune("force_path", 0)
        s.compute_force()
        fc = valid_forces(s)
        s.tune("force_path", 1)
        r, m = rel(fp, fc)
        assert r <= SUM_ORDER and m <= 20 * SUM_ORDER, (k, r, m)
    d1, codes = s.pair_stats()
    assert d1 > d0 and codes > 0
    # with a small buffer (limit 0.05 per atom) the integrator's test triggers
    # derivations inside the rebuild period, and forces stay the same
    s.set_pair_buffer(0.1)
    s.run(1, first_step=done, max_samples=0)
    d2, _ = s.pair_stats()
    s.run(15, first_step=done + 1, max_samples=0)
    d3, _ = s.pair_stats()
    assert d3 - d2 >= 5, (d2, d3)
    fp = valid_forces(s)
    s.tune("force_path", 0)
    s.compute_force()
    r, m = rel(fp, valid_forces(s))
    assert r <= SUM_ORDER and m <= 20 * SUM_ORDER, (r, m)


@pytest.mark.parametrize("half", [0, 1])
def test_pair_path_against_fp64_oracle(half):
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
    s = mdb.ClusterSystem(natoms=len(t), cluster_n=4, half_neigh=half, precision="mixed",
                          **common)
    s.tune("force_path", 1)
    s.set_atoms(x, v, t)
    s.setup()
    o = O.OracleCP(x, v, t, M=4, N=4, half=half, natoms=len(t), **common)
    o.setup()
    o.force()
    nat = o.iclusters()[0]
    ok = np.concatenate([np.arange(4) < k for k in nat])
    fo = o.slots()[2][:len(ok)][ok]
    r, m = rel(valid_forces(s), fo)
    assert r <= MIXED_RMS and m <= 20 * MIXED_RMS, (r, m)


def test_pair_path_trajectory_tracks_cluster_kernel():
    """100 steps from the lattice on both paths: temperatures agree as the
    cluster-pair kernel's own mixed run tracks FP64."""
    a, _ = system(6, 4, 1)
    b, _ = system(6, 4, 1)
    b.tune("force_path", 1)
    ta = a.run(100)
    tb = b.run(100)
    for p, q in zip(ta, tb):
        assert abs(p["T"] - q["T"]) <= 1e-3 * p["T"]


def test_pair_path_timing_and_buffer():
    s, _ = system(8, 4, 1, steps=50)
    s.tune("force_path", 1)
    t = s.time_force(reps=5)
    assert t > 0
    fp = valid_forces(s)  # time_force leaves the state's forces
    s.tune("force_path", 0)
    s.compute_force()
    r, m = rel(fp, valid_forces(s))
    assert r <= SUM_ORDER, r
    # a smaller buffer re-derives more often and keeps the same forces
    s.tune("force_path", 1)
    s.set_pair_buffer(0.1)
    s.compute_force()
    r, m = rel(valid_forces(s), fp)
    assert r <= SUM_ORDER and m <= 20 * SUM_ORDER, (r, m)
    with pytest.raises(mdb.MdbError):
        f64, _ = system(5, 4, 1, precision="fp64")
        f64.tune("force_path", 1)


# ---- MDB_PREC_MIXED_COMP: compensated sums, exact cutoff decisions ------------

def oracle_state(n, types=None, steps=150):
    """A thermalised state from the Verlet-list oracle, with its parameters."""
    kw = {}
    okw = {}
    if types is not None:
        import workloads as W
        kw = dict(types=types, cutforce=W.c5_cutoff(types[1]))
        okw = dict(epsilon_per_type=types[0], sigma_per_type=types[1], ntypes=len(types[0]),
                   cutforce=kw["cutforce"])
    o = O.Oracle(nx=n, ny=n, nz=n, **okw)
    o.lattice()
    o.setup()
    o.run(steps)
    x, v, _, t = o.atoms()
    hp = mdb.host_params(nx=n, ny=n, nz=n, **kw)
    mdb.create_fcc(hp)
    return hp, x, v, t


@pytest.mark.parametrize("N,half", [(4, 1), (4, 0), (8, 1)])
def test_comp_against_fp64_oracle_multitype(N, half):
    """4 types, geometric mixing, cutoff 2.5 sigma_max: the compensated path
    takes exactly the FP64 path's pairs (no outliers from pairs within an FP32
    rounding of the cutoff, where the unshifted potential jumps) and carries
    compensated sums, so both its RMS and its max per-atom error stay far
    below the mixed path's budget."""
    import workloads as W
    types = W.c5_types()
    hp, x, v, t = oracle_state(7, types)
    common = dict(xprd=hp.xprd, yprd=hp.yprd, zprd=hp.zprd, cutforce=hp.cutforce,
                  cutneigh=hp.cutneigh, dt=hp.dt, dtforce=hp.dtforce, mass=hp.mass,
                  ntypes=4, epsilon_per_type=list(types[0]), sigma_per_type=list(types[1]))
    o = O.OracleCP(x, v, t, M=4, N=N, half=half, natoms=len(t), **common)
    o.setup()
    o.force()
    nat = o.iclusters()[0]
    ok = np.concatenate([np.arange(4) < k for k in nat])
    fo = o.slots()[2][:len(ok)][ok]
    errs = {}
    for prec in ("mixed", "mixed_comp"):
        s = mdb.ClusterSystem(natoms=len(t), cluster_n=N, half_neigh=half, precision=prec,
                              **common)
        s.set_atoms(x, v, t)
        s.setup()
        errs[prec] = rel(valid_forces(s), fo)
        s.close()
    r, m = errs["mixed_comp"]
    assert r <= 2e-6 and m <= 5e-5, errs
    assert r <= errs["mixed"][0], errs


def test_comp_runs_and_rejects_the_cluster_kernel():
    s, _ = system(6, 4, 1, precision="mixed_comp")
    with pytest.raises(mdb.MdbError):
        s.tune("force_path", 0)
    t0 = s.thermo()["T"]
    samples = s.run(100)
    assert samples and abs(samples[-1]["T"] - t0) < 0.5 * t0
