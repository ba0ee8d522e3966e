"""Parity at the benchmark configurations' own sizes.

The other GPU tests pin every kernel against the oracle on small systems; these
repeat the comparisons at the sizes the benchmark runs, where capacities grow,
columns are long, ghost counts are large and overflow replays happen:

* LJ fcc 64^3 (1,048,576 atoms), cluster-pair scheme, 4x4 and 4x8 clusters,
  half and full lists: clusters, j-clusters, ghost clusters, columns, the
  ordered list rows with their masks and the FP64 forces against the oracle
  (bit-identical for full lists, 1e-12 of the force scale for half lists,
  whose reactions are added by atomics), on the perfect lattice (equal z
  values: the swap-sort replay) and on a disordered state; a 20-step FP64
  trajectory across a rebuild, bit for bit; the mixed forces against the
  oracle's FP64 forces within the error budget.
* The same workload in the Verlet-list scheme: ordered lists and FP64 forces.
* EAM copper, fcc 32^3 (131,072 atoms, a = 3.615 A, 1600 K, Cu_u3 funcfl):
  lists, forces and F'(rho) after setup and after 5 steps bit for bit against
  the oracle, and against the reference itself reading the same state from a
  dump file; thermo to 1e-10.
* Multi-type liquid (4 types, geometric mixing, cutoff 2.5 sigma_max) at 64^3:
  cluster-pair build and FP64 forces against the oracle.

The oracle (oracle/, a C restatement pinned to the reference by
tests/test_oracle*.py) runs each of these in seconds.
"""
import os

import numpy as np
import pytest

import mdb
import oracle as O
from conftest import EAM_FILE

pytestmark = pytest.mark.gpu

FP64_REL = 1e-12
THERMO_REL = 1e-10
MIXED_RMS = 1e-5
CELLS = 64
EAM_CELLS = 32
EAM_A = 3.615
EAM_T = 1600.0


def _common(hp):
    return dict(xprd=hp.xprd, yprd=hp.yprd, zprd=hp.zprd, cutforce=hp.cutforce,
                cutneigh=hp.cutneigh, dt=hp.dt, dtforce=hp.dtforce, mass=hp.mass,
                epsilon=hp.epsilon, sigma=hp.sigma, reneigh_every=hp.reneigh_every,
                nstat=hp.nstat, ntypes=hp.ntypes)


def _types(hp):
    if not hp.has_types:
        return None, None
    return list(hp.epsilon_per_type)[:hp.ntypes], list(hp.sigma_per_type)[:hp.ntypes]


def cp_gpu(hp, x, v, t, N, half, precision="fp64"):
    eps, sig = _types(hp)
    s = mdb.ClusterSystem(natoms=len(t), cluster_n=N, half_neigh=half, precision=precision,
                          epsilon_per_type=eps, sigma_per_type=sig, **_common(hp))
    s.set_atoms(x, v, t)
    s.setup()
    return s


def cp_oracle(hp, x, v, t, N, half):
    eps, sig = _types(hp)
    o = O.OracleCP(x, v, t, M=4, N=N, half=half, natoms=len(t), epsilon_per_type=eps,
                   sigma_per_type=sig, **_common(hp))
    o.setup()
    o.force()
    return o


def assert_same_rows(nn, nb, nn2, nb2):
    """Ordered rows equal: entries past each row's length are ignored."""
    assert np.array_equal(nn, nn2)
    w = int(nn.max()) if len(nn) else 0
    a, b = nb[:, :w], nb2[:, :w]
    used = np.arange(w)[None, :] < nn[:, None]
    assert np.array_equal(a[used], b[used])


def assert_same_build(s, o):
    cs, co = s.counts(), o.counts()
    for k in ("nlocal", "ncl", "ncj", "ngc", "nghost", "dummy", "maxneighs"):
        assert cs[k] == co[k], (k, cs[k], co[k])
    for a, b in zip(s.iclusters(), o.iclusters()):
        assert np.array_equal(a, b)
    for a, b in zip(s.jclusters(), o.jclusters()):
        assert np.array_equal(a, b)
    for a, b in zip(s.ghosts(), o.ghosts()):
        assert np.array_equal(a, b)
    xs, _, _, ts = s.slots()
    xo, _, _, to = o.slots()
    assert np.array_equal(xs, xo)
    real = np.isfinite(xo[:, 0])
    assert np.array_equal(ts[real], to[real])
    for a, b in zip(s.columns(), o.columns()):
        assert np.array_equal(a, b)
    nn, nm, nb = s.neighbor_list()
    nn2, nm2, nb2, _ = o.neighbor_list()
    assert np.array_equal(nm, nm2)
    assert_same_rows(nn, nb, nn2, nb2)


def valid_slots(o):
    nat, _, _ = o.iclusters()
    return np.concatenate([np.arange(4) < k for k in nat])


def local_forces(sys_or_orc, valid):
    return sys_or_orc.slots()[2][:len(valid)][valid]


def force_scale(f):
    return max(np.sqrt(np.mean(np.sum(f * f, axis=1))), 1.0)


def assert_forces_close(f, fref, tol=FP64_REL):
    err = np.abs(f - fref).max()
    assert err <= tol * force_scale(fref), (err, force_scale(fref))


def rel_rms(f, fref):
    rms = np.sqrt(np.mean(np.sum(fref * fref, axis=1)))
    return np.sqrt(np.mean(np.sum((f - fref) ** 2, axis=1))) / rms


@pytest.fixture(scope="module")
def lattice64():
    hp = mdb.host_params(nx=CELLS, ny=CELLS, nz=CELLS)
    x, v, t = mdb.create_fcc(hp)
    assert len(t) == 1048576
    return hp, x, v, t


@pytest.fixture(scope="module")
def melted64(lattice64):
    """The lattice after 60 FP64 steps on the GPU (3 rebuilds; bit-identical to
    the oracle's trajectory, see test_c2_cp_trajectory_bit_exact): no equal z
    values, ragged clusters."""
    hp, x, v, t = lattice64
    s = cp_gpu(hp, x, v, t, 4, 0)
    s.run(60, max_samples=0)
    xa, va, ta = s.atoms()
    s.close()
    return hp, xa, va, ta


@pytest.mark.parametrize("N", [4, 8])
@pytest.mark.parametrize("half", [0, 1])
def test_c2_cp_lattice_build_and_forces(lattice64, N, half):
    hp, x, v, t = lattice64
    s = cp_gpu(hp, x, v, t, N, half)
    o = cp_oracle(hp, x, v, t, N, half)
    assert_same_build(s, o)
    valid = valid_slots(o)
    fs, fo = local_forces(s, valid), local_forces(o, valid)
    if half:
        assert_forces_close(fs, fo)
    else:
        assert np.array_equal(fs, fo)
    s.close()


@pytest.mark.parametrize("N,half", [(4, 1), (4, 0), (8, 1)])
def test_c2_cp_melted_build_forces_and_mixed(melted64, N, half):
    hp, x, v, t = melted64
    s = cp_gpu(hp, x, v, t, N, half)
    o = cp_oracle(hp, x, v, t, N, half)
    assert_same_build(s, o)
    nat = o.iclusters()[0]
    assert (nat < 4).any()
    valid = valid_slots(o)
    fo = local_forces(o, valid)
    fs = local_forces(s, valid)
    if half:
        assert_forces_close(fs, fo)
    else:
        assert np.array_equal(fs, fo)
    s.close()
    m = cp_gpu(hp, x, v, t, N, half, precision="mixed")
    assert rel_rms(local_forces(m, valid), fo) <= MIXED_RMS
    m.close()


def test_c2_cp_trajectory_bit_exact(lattice64):
    """20 FP64 steps (the rebuild of step 19 included) through the hooks and
    through the graph-captured loop, 4x4 full lists, against the oracle."""
    hp, x, v, t = lattice64
    s = cp_gpu(hp, x, v, t, 4, 0)
    o = cp_oracle(hp, x, v, t, 4, 0)
    g = cp_gpu(hp, x, v, t, 4, 0)
    for n in range(20):
        s.step_hooks(n)
        o.step(n)
    g.run(20, max_samples=0)
    valid = valid_slots(o)
    xo, vo, _, _ = o.slots()
    for sys_ in (s, g):
        xs, vs, _, _ = sys_.slots()
        assert np.array_equal(xs[:len(valid)][valid], xo[:len(valid)][valid])
        assert np.array_equal(vs[:len(valid)][valid], vo[:len(valid)][valid])
    assert_same_build(s, o)
    T = o.thermo()["T"]
    assert abs(s.thermo()["T"] - T) <= THERMO_REL * T
    s.close()
    g.close()


@pytest.mark.parametrize("half", [0, 1])
def test_c2_vl_lists_and_forces(half):
    hp = mdb.host_params(nx=CELLS, ny=CELLS, nz=CELLS, half_neigh=half)
    x, v, t = mdb.create_fcc(hp)
    s = mdb.system_from_host(hp, len(t))
    s.set_atoms(x, v, t)
    s.setup()
    o = O.Oracle(nx=CELLS, ny=CELLS, nz=CELLS, half_neigh=half)
    o.lattice()
    o.setup()
    o.force()
    bs, ps = s.ghosts()
    bo, po = o.ghosts()
    assert np.array_equal(bs, bo) and np.array_equal(ps, po)
    ns, ls = s.neighbor_list()
    no, lo = o.neighbor_list()
    assert_same_rows(ns, ls, no, lo)
    fs, fo = s.atoms()[2], o.atoms()[2]
    if half:
        assert_forces_close(fs, fo)
    else:
        assert np.array_equal(fs, fo)
    s.close()


def copper():
    tab = mdb.read_funcfl(EAM_FILE)
    hp = mdb.host_params(eam=tab, nx=EAM_CELLS, ny=EAM_CELLS, nz=EAM_CELLS,
                         rho=4.0 / EAM_A ** 3, temp=EAM_T)
    x, v, t = mdb.create_fcc(hp)
    hp.from_file = 1  # the reference reads this configuration from a dump: cutneigh/2 bins
    return tab, hp, x, v, t


def test_c3_eam_copper_against_oracle():
    tab, hp, x, v, t = copper()
    assert len(t) == 131072
    s = mdb.system_from_host(hp, len(t), eam=tab)
    s.set_atoms(x, v, t)
    s.setup()
    o = O.Oracle(eam_file=EAM_FILE, force_field=1, from_file=1, xprd=hp.xprd, yprd=hp.yprd,
                 zprd=hp.zprd)
    o.set_atoms(x, v, t)
    o.setup()
    o.force()
    n = len(t)
    ns, ls = s.neighbor_list()
    no, lo = o.neighbor_list()
    assert_same_rows(ns, ls, no, lo)
    assert np.array_equal(s.atoms()[2], o.atoms()[2])
    assert np.array_equal(s.eam_fp()[:n], o.eam_fp()[:n])
    for k in range(5):
        s.step(k)
        o.step(k)
    xs, vs, fs, _ = s.atoms()
    xo, vo, fo, _ = o.atoms()
    assert np.array_equal(xs, xo) and np.array_equal(vs, vo) and np.array_equal(fs, fo)
    assert np.array_equal(s.eam_fp()[:n], o.eam_fp()[:n])
    s.compute_force(energy=True)  # PE is reported after an energy evaluation
    ts, to = s.thermo(), o.thermo()
    for key in ("T", "P", "PE"):
        assert ts[key] == pytest.approx(to[key], rel=THERMO_REL), key
    s.close()


@pytest.mark.parametrize("precision", ["mixed", "mixed_comp"])
def test_c3_eam_copper_mixed_against_oracle(precision):
    """The mixed EAM passes (in-cutoff rows from the density pass, F'(rho)
    gathered with the position) on the copper state after 100 FP64 steps,
    against the oracle's FP64 forces on the same state: within the mixed
    path's budget, with one and with two lanes per atom in the density pass
    (the same rows; only the FP64 density sum's order differs)."""
    tab, hp, x, v, t = copper()
    s = mdb.system_from_host(hp, len(t), eam=tab)
    s.set_atoms(x, v, t)
    s.setup()
    s.run(100, max_samples=0)
    xa, va, _, ta = s.atoms()
    s.close()
    o = O.Oracle(eam_file=EAM_FILE, force_field=1, from_file=1, xprd=hp.xprd, yprd=hp.yprd,
                 zprd=hp.zprd)
    o.set_atoms(xa, va, ta)
    o.setup()
    o.force()
    m = mdb.system_from_host(hp, len(t), eam=tab, precision=precision)
    m.set_atoms(xa, va, ta)
    m.setup()
    f1 = m.atoms()[2]
    assert rel_rms(f1, o.atoms()[2]) <= MIXED_RMS
    m.compute_force(energy=True)
    assert m.thermo()["PE"] == pytest.approx(o.thermo()["PE"], rel=1e-6)
    m.tune("eam_rho_lanes", 2)
    m.compute_force(energy=True)
    assert m.thermo()["PE"] == pytest.approx(o.thermo()["PE"], rel=1e-6)
    f2 = m.atoms()[2]
    assert rel_rms(f2, f1) <= 1e-6 and rel_rms(f2, o.atoms()[2]) <= MIXED_RMS
    with pytest.raises(mdb.MdbError):
        m.tune("eam_rho_lanes", 3)
    m.close()


@pytest.mark.skipif(not O.ref_available(), reason="reference build absent")
def test_c3_eam_copper_against_reference(tmp_path):
    """The reference itself (its own sources, strict FP64 build) reads the
    generated copper state from a dump file (-i, -f eam): the same lists, the
    same forces and the same positions after 5 steps."""
    tab, hp, x, v, t = copper()
    path = str(tmp_path / "cu32.dmp")
    mdb.write_dmp(path, x, v, t, (hp.xprd, hp.yprd, hp.zprd))
    r = O.RefVL(force_field=1, input_file=path, eam_file=EAM_FILE)
    assert r.nlocal == len(t)
    s = mdb.system_from_host(hp, len(t), eam=tab)
    s.set_atoms(x, v, t)
    s.setup()
    r.force()
    ns, ls = s.neighbor_list()
    nr, lr = r.neighbor_list()
    assert_same_rows(ns, ls, nr, lr)
    assert np.array_equal(s.atoms()[2], r.atoms()[2])
    for k in range(5):
        s.step(k)
        r.step(k)
    xs, vs, _, _ = s.atoms()
    xr, vr, _, _ = r.atoms()
    assert np.array_equal(xs, xr) and np.array_equal(vs, vr)
    assert s.thermo()["T"] == pytest.approx(r.thermo()["T"], rel=THERMO_REL)
    s.close()


@pytest.mark.parametrize("N", [4, 8])
def test_c5_multitype_build_and_forces(N):
    import workloads as W
    eps, sig = W.c5_types()
    hp = mdb.host_params(nx=CELLS, ny=CELLS, nz=CELLS, types=(eps, sig),
                         cutforce=W.c5_cutoff(sig))
    x, v, t = mdb.create_fcc(hp)
    assert hp.ntypes == 4 and set(np.unique(t).tolist()) == {0, 1, 2, 3}
    s = cp_gpu(hp, x, v, t, N, 1)
    o = cp_oracle(hp, x, v, t, N, 1)
    assert_same_build(s, o)
    valid = valid_slots(o)
    assert_forces_close(local_forces(s, valid), local_forces(o, valid))
    s.close()
