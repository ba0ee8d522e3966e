"""The cluster-pair scheme's bin size as a tuning choice (``column_edge``, the
autotuner's bin-size knob): a column grid other than setupNeighbor's
(clusterpair/neighbor.c:128-145) gives other clusters and lists, but the same
pairs inside the list cutoff. So FP64 full-list forces equal the default
grid's (and the oracle's) up to summation order, mixed forces stay within the
budget, lists rebuilt inside a run stay complete, and an ensemble member on
such a grid still follows its solo run bit for bit. The
default (100) is the reference's grid, which the other tests pin bit for bit.
"""
import numpy as np
import pytest

import mdb

from test_gpu_cp import MIXED_RMS, SHAPES, assert_forces_close, local_forces, pair, \
    thermalised, valid_slots

pytestmark = pytest.mark.gpu


def build(hp, x, v, t, N, edge, half=0, precision="fp64"):
    s = mdb.ClusterSystem(natoms=len(t), cluster_n=N, half_neigh=half, precision=precision,
                          column_edge=edge, xprd=hp.xprd, yprd=hp.yprd, zprd=hp.zprd,
                          cutforce=hp.cutforce, cutneigh=hp.cutneigh, dt=hp.dt,
                          dtforce=hp.dtforce, mass=hp.mass, epsilon=hp.epsilon,
                          sigma=hp.sigma, reneigh_every=hp.reneigh_every, nstat=hp.nstat,
                          ntypes=hp.ntypes)
    s.set_atoms(x, v, t)
    s.setup()
    return s


def by_position(s):
    """Positions and forces of the local atoms, in the lexicographic order of
    their positions (cluster order differs between grids)."""
    c = s.counts()
    x, _, f, t = s.slots()
    n = c["ncl"] * 4
    keep = t[:n] >= 0
    x, f = x[:n][keep], f[:n][keep]
    o = np.lexsort((x[:, 2], x[:, 1], x[:, 0]))
    return x[o], f[o]


@pytest.mark.parametrize("N", SHAPES)
@pytest.mark.parametrize("edge", [80, 125])
def test_other_grid_same_fp64_forces(N, edge):
    hp, x, v, t = thermalised(8)
    ref, o = pair(hp, x, v, t, N)
    s = build(hp, x, v, t, N, edge)
    assert s.geometry()["nbinx"] != ref.geometry()["nbinx"]
    assert s.counts()["nlocal"] == len(t)
    xs, fs = by_position(s)
    xr, fr = by_position(ref)
    assert np.array_equal(xs, xr)
    assert_forces_close(fs, fr)
    # the default grid's forces are the oracle's (the reference's grid)
    assert_forces_close(local_forces(ref, valid_slots(o)), local_forces(o, valid_slots(o)), 0.0)
    s.close()
    ref.close()


@pytest.mark.parametrize("N", SHAPES)
@pytest.mark.parametrize("half", [0, 1])
def test_other_grid_mixed_within_budget(N, half):
    hp, x, v, t = thermalised(8)
    ref = build(hp, x, v, t, N, 100, half)
    s = build(hp, x, v, t, N, 125, half, "mixed")
    _, fr = by_position(ref)
    _, fs = by_position(s)
    scale = np.sqrt(np.mean(np.sum(fr * fr, axis=1)))
    rms = np.sqrt(np.mean(np.sum((fs - fr) ** 2, axis=1))) / scale
    assert rms <= MIXED_RMS, rms
    s.close()
    ref.close()


def missing_pairs(s, cutneigh):
    """Atom pairs closer than cutneigh that no listed cluster pair covers."""
    from scipy.spatial import cKDTree
    c = s.counts()
    x, _, _, t = s.slots()
    nn, _, nb = s.neighbor_list()
    N = s.N
    covered = set()
    for ci in range(c["ncl"]):
        for cj in nb[ci, :nn[ci]]:
            covered.update((ci * 4 + a, int(cj) * N + b) for a in range(4) for b in range(N))
    valid = np.isfinite(x[:, 0]) & (t >= 0)
    idx = np.nonzero(valid)[0]
    tree = cKDTree(x[idx])
    missing = 0
    for i in range(c["ncl"] * 4):
        if valid[i]:
            for jj in tree.query_ball_point(x[i], cutneigh * (1.0 - 1e-12)):
                j = int(idx[jj])
                if j != i and (i, j) not in covered and (j, i) not in covered:
                    missing += 1
    return missing


@pytest.mark.parametrize("edge", [80, 125])
def test_other_grid_rebuilds_stay_complete(edge):
    """40 steps (rebuilds with re-clustering at steps 20 and 40) on another
    grid: the last build's list covers every atom pair within cutneigh, and
    its forces equal a fresh build's on the reference grid from the same
    positions. (Trajectories of two grids are not compared step by step: the
    summation order differs, and with the reference's unshifted potential a
    pair whose distance sits within a rounding of r_c may be inside in one run
    and outside in the other, a force jump of F(r_c).)"""
    hp, x, v, t = thermalised(7, nstat=10)
    b = build(hp, x, v, t, 4, edge)
    b.run(40, max_samples=0)
    assert missing_pairs(b, hp.cutneigh) == 0
    xb, vb, tb = b.atoms()
    a = build(hp, xb, vb, tb, 4, 100)
    assert missing_pairs(a, hp.cutneigh) == 0
    pa, fa = by_position(a)
    pb, fb = by_position(b)
    assert np.array_equal(pa, pb)
    assert_forces_close(fb, fa)
    a.close()
    b.close()


def test_ensemble_member_on_other_grid_matches_solo():
    """Members on different grids in one batched ensemble follow their solo
    runs bit for bit (full lists, mixed)."""
    runs = []
    for n, rho, T, edge in ((5, 0.85, 1.2, 125), (4, 0.8, 0.9, 100), (6, 0.9, 1.5, 80)):
        hp = mdb.host_params(nx=n, ny=n, nz=n, rho=rho, temp=T, nstat=10)
        x, v, t = mdb.create_fcc(hp)
        runs.append([build(hp, x, v, t, 4, edge, precision="mixed") for _ in range(2)])
    ens = mdb.Ensemble([r[0] for r in runs])
    got = ens.run(45, max_samples=8)
    for k, (a, b) in enumerate(runs):
        want = b.run(45, max_samples=8)
        assert got[k] == want, k
        for u, w in zip(a.slots(), b.slots()):
            assert np.array_equal(u, w)
    ens.close()
    for r in runs:
        for s in r:
            s.close()


def test_column_edge_rejected_after_atoms_and_out_of_range():
    hp = mdb.host_params(nx=4, ny=4, nz=4)
    x, v, t = mdb.create_fcc(hp)
    s = build(hp, x, v, t, 4, 100)
    with pytest.raises(mdb.MdbError):
        s.tune("column_edge", 125)
    s.close()
    with pytest.raises(mdb.MdbError):
        build(hp, x, v, t, 4, 49)
    with pytest.raises(mdb.MdbError):
        build(hp, x, v, t, 4, 201)
