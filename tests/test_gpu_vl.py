"""Parity of the CUDA Verlet-list path (libmdb through its C ABI) with the oracle
and with fixtures produced by the reference itself.

FP64 path: binning geometry, ghost map, neighbour lists (as ordered rows) and
full-list forces are bit-identical; trajectories through the hooks and through
the graph-captured loop stay bit-identical for tens of steps across rebuilds;
half-list forces (atomics, different summation order) agree to 1e-12 of the
force scale (see assert_forces_close); thermo to 1e-10. Mixed path: force
error against FP64 within the stated budget (RMS <= 1e-5 of the RMS force).
"""
import os

import numpy as np
import pytest

import mdb
import oracle as O
from conftest import EAM_FILE, GOLDEN

pytestmark = pytest.mark.gpu

FP64_REL = 1e-12     # per-atom force tolerance (relative to RMS |f|) when order differs
THERMO_REL = 1e-10
MIXED_RMS = 1e-5     # RMS force error budget of the mixed path, relative to RMS |f|


def rel_err(a, b):
    rms = np.sqrt(np.mean(np.sum(b * b, axis=1)))
    d = np.sqrt(np.sum((a - b) ** 2, axis=1))
    return d.max() / rms, np.sqrt(np.mean(d * d)) / rms


def assert_forces_close(f, fref, tol=FP64_REL):
    """|f - fref| <= tol * max(RMS |fref|, 1): at a perfect-lattice start the net
    forces cancel to ~1e-14 while each pair term is O(1) (reduced LJ units,
    eV/A for EAM), so a different summation order is judged against the pair
    force scale, not against the near-zero net force."""
    scale = max(np.sqrt(np.mean(np.sum(fref * fref, axis=1))), 1.0)
    err = np.abs(f - fref).max()
    assert err <= tol * scale, (err, scale)


def lj_system(precision="fp64", **kw):
    hp = mdb.host_params(**kw)
    x, v, t = mdb.create_fcc(hp)
    s = mdb.system_from_host(hp, len(t), precision=precision)
    s.set_atoms(x, v, t)
    s.setup()
    return s, hp


def lj_oracle(**kw):
    o = O.Oracle(**kw)
    o.lattice()
    o.setup()
    o.force()
    return o


def eam_pair(g, precision="fp64", nstat=100):
    tab = mdb.read_funcfl(EAM_FILE)
    hp = mdb.host_params(eam=tab, nstat=nstat)
    hp.from_file = 1
    hp.xprd, hp.yprd, hp.zprd = (float(b) for b in g["box"])
    s = mdb.system_from_host(hp, len(g["type"]), eam=tab, precision=precision)
    s.set_atoms(g["x0"], g["v0"], g["type"])
    s.setup()
    return s


@pytest.mark.parametrize("cells", [(5, 5, 5), (8, 8, 8), (7, 6, 5), (16, 16, 16)])
def test_bin_geometry_and_ghosts(cells):
    nx, ny, nz = cells
    s, _ = lj_system(nx=nx, ny=ny, nz=nz)
    o = lj_oracle(nx=nx, ny=ny, nz=nz)
    gs, go = s.bin_geometry(), o.bin_geometry()
    for k in go:
        if k == "stencil":
            assert np.array_equal(gs[k], go[k])
        else:
            assert gs[k] == go[k], k
    bs, ps = s.ghosts()
    bo, po = o.ghosts()
    assert np.array_equal(bs, bo) and np.array_equal(ps, po)
    assert np.array_equal(s.positions_all(), o.positions_all())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("half", [0, 1])
def test_lists_bit_exact_in_reference_order(half, precision):
    s, _ = lj_system(precision=precision, nx=8, ny=7, nz=9, half_neigh=half)
    o = lj_oracle(nx=8, ny=7, nz=9, half_neigh=half)
    ns, ls = s.neighbor_list()
    no, lo = o.neighbor_list()
    assert np.array_equal(ns, no)
    for i in range(len(ns)):
        assert np.array_equal(ls[i, :ns[i]], lo[i, :no[i]])


@pytest.mark.parametrize("half", [0, 1])
def test_against_reference_fixture(half):
    g = dict(np.load(os.path.join(GOLDEN, "lj_half_5x5x5.npz" if half else
                                  "lj_full_5x5x5.npz")))
    s, _ = lj_system(nx=5, ny=5, nz=5, half_neigh=half)
    ns, ls = s.neighbor_list()
    assert np.array_equal(ns, g["numneigh"])
    for i in range(len(ns)):
        assert np.array_equal(ls[i, :ns[i]], g["neighbors"][i, :ns[i]])
    _, _, f, _ = s.atoms()
    if half:
        assert_forces_close(f, g["f0"])
    else:
        assert np.array_equal(f, g["f0"])
    for n in range(45):
        s.step(n)
    x, v, f, _ = s.atoms()
    if half:
        assert np.abs(x - g["x45"]).max() < 1e-9
    else:
        assert np.array_equal(x, g["x45"]) and np.array_equal(v, g["v45"])
    assert s.thermo()["T"] == pytest.approx(float(g["T45"]), rel=1e-9 if half else THERMO_REL)


def test_full_list_force_and_trajectory_bit_exact_hooks_and_graphs():
    kw = dict(nx=9, ny=8, nz=10, nstat=43)
    o = lj_oracle(**kw)
    s1, _ = lj_system(**kw)
    s2, _ = lj_system(**kw)
    _, _, f, _ = s1.atoms()
    assert np.array_equal(f, o.atoms()[2])
    th0 = s1.thermo()
    tho = o.thermo()
    assert th0["T"] == pytest.approx(tho["T"], rel=THERMO_REL)
    assert th0["PE"] == pytest.approx(tho["PE"], rel=THERMO_REL)
    for n in range(43):
        o.step(n)
        s1.step(n)
    samples = s2.run(43)
    xo, vo, fo, _ = o.atoms()
    for s in (s1, s2):
        x, v, f, _ = s.atoms()
        assert np.array_equal(x, xo) and np.array_equal(v, vo) and np.array_equal(f, fo)
    th = o.thermo()
    last = samples[-1]
    assert last["step"] == 43
    for k in ("T", "P", "PE", "E"):
        assert last[k] == pytest.approx(th[k], rel=THERMO_REL)


def test_sort_atoms_bit_exact():
    """sortAtom on the GPU after 33 steps: the same permutation of positions,
    velocities, types and forces as the oracle (itself pinned to the
    reference's sortAtom), then a rebuild and the same forces."""
    kw = dict(nx=7, ny=6, nz=5)
    o = lj_oracle(**kw)
    s, _ = lj_system(**kw)
    for n in range(33):
        o.step(n)
        s.step(n)
    o.sort_atoms()
    s.sort_atoms()
    xo, vo, fo, to = o.atoms()
    x, v, f, t = s.atoms()
    assert np.array_equal(x, xo) and np.array_equal(v, vo)
    assert np.array_equal(t, to) and np.array_equal(f, fo)
    o.reghost()
    o.force()
    s.setup_pbc()
    s.update_pbc()
    s.build_neighbor()
    s.compute_force()
    assert np.array_equal(s.atoms()[2], o.atoms()[2])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_resort_run(precision):
    """mdb_run with a resort period follows the oracle's SORT_ATOMS loop bit for
    bit in FP64 (full lists), and the mixed path stays within its budget."""
    kw = dict(nx=8, ny=8, nz=8, nstat=50)
    o = lj_oracle(**kw)
    o.set_resort(40)
    s, _ = lj_system(precision=precision, **kw)
    s.set_resort(40)
    samples = s.run(100)
    o.run(100)
    xo, vo, fo, to = o.atoms()
    x, v, f, t = s.atoms()
    assert np.array_equal(t, to)
    if precision == "fp64":
        assert np.array_equal(x, xo) and np.array_equal(v, vo) and np.array_equal(f, fo)
    else:
        assert np.abs(x - xo).max() < 1e-3
    assert samples[-1]["step"] == 100
    assert samples[-1]["T"] == pytest.approx(o.thermo()["T"], rel=THERMO_REL if precision == "fp64" else 1e-3)


def test_half_list_forces_and_steps():
    kw = dict(nx=8, ny=8, nz=8, half_neigh=1)
    o = lj_oracle(**kw)
    s, _ = lj_system(**kw)
    assert_forces_close(s.atoms()[2], o.atoms()[2])
    assert s.thermo()["PE"] == pytest.approx(o.thermo()["PE"], rel=THERMO_REL)
    full, _ = lj_system(nx=8, ny=8, nz=8)
    assert_forces_close(s.atoms()[2], full.atoms()[2])
    for n in range(5):
        o.step(n)
        s.step(n)
    assert_forces_close(s.atoms()[2], o.atoms()[2], 1e-10)
    assert s.thermo()["T"] == pytest.approx(o.thermo()["T"], rel=THERMO_REL)


def test_multitype_geometric_rule():
    eps, sig = [1.0, 0.6, 1.4, 0.9], [1.0, 0.85, 1.1, 0.95]
    kw = dict(nx=6, ny=6, nz=6)
    hp = mdb.host_params(types=(eps, sig), **kw)
    x, v, t = mdb.create_fcc(hp)
    s = mdb.system_from_host(hp, len(t))
    s.set_atoms(x, v, t)
    s.setup()
    o = O.Oracle(epsilon_per_type=eps, sigma_per_type=sig, **kw)
    o.lattice()
    o.setup()
    o.force()
    assert np.array_equal(s.atoms()[2], o.atoms()[2])
    for n in range(21):
        o.step(n)
        s.step(n)
    assert np.array_equal(s.atoms()[0], o.atoms()[0])


def test_list_capacity_grows_on_overflow():
    hp = mdb.host_params(nx=6, ny=6, nz=6)
    x, v, t = mdb.create_fcc(hp)
    s = mdb.system_from_host(hp, len(t), maxneighs=8)
    s.set_atoms(x, v, t)
    s.setup()
    o = lj_oracle(nx=6, ny=6, nz=6)
    assert s.counts()[2] > 78
    assert np.array_equal(s.atoms()[2], o.atoms()[2])


def test_small_box_and_multiple_images():
    """Box shorter than twice the cutoff: an atom meets several images of the
    same neighbour. Both paths keep every image like the reference (ghosts
    carry their own positions)."""
    s, _ = lj_system(nx=3, ny=3, nz=3)
    o = lj_oracle(nx=3, ny=3, nz=3)
    assert np.array_equal(s.atoms()[2], o.atoms()[2])
    o.run(60)
    x, v, _, t = o.atoms()
    o.set_state(x, v)
    o.setup()
    o.force()
    m, _ = lj_system(precision="mixed", nx=3, ny=3, nz=3)
    m.set_atoms(x, v, t)
    m.setup()
    assert rel_err(m.atoms()[2], o.atoms()[2])[1] <= MIXED_RMS


def test_eam_fp64_bit_exact_against_reference_fixture():
    g = dict(np.load(os.path.join(GOLDEN, "eam_cu_6x6x6.npz")))
    s = eam_pair(g)
    ns, ls = s.neighbor_list()
    assert np.array_equal(ns, g["numneigh"])
    assert np.array_equal(s.atoms()[2], g["f0"])
    for n in range(25):
        s.step(n)
    x, v, f, _ = s.atoms()
    assert np.array_equal(x, g["x25"]) and np.array_equal(v, g["v25"])
    assert np.array_equal(f, g["f25"])
    assert s.thermo()["T"] == pytest.approx(float(g["T25"]), rel=THERMO_REL)


def test_eam_fp_and_graph_loop_match_oracle():
    g = dict(np.load(os.path.join(GOLDEN, "eam_cu_6x6x6.npz")))
    box = g["box"]
    o = O.Oracle(eam_file=EAM_FILE, force_field=1, from_file=1, xprd=box[0], yprd=box[1],
                 zprd=box[2])
    o.set_atoms(g["x0"], g["v0"], g["type"])
    o.setup()
    o.force()
    s = eam_pair(g, nstat=30)
    assert np.array_equal(s.eam_fp()[:len(g["type"])], o.eam_fp()[:len(g["type"])])
    assert s.thermo()["PE"] == pytest.approx(o.thermo()["PE"], rel=THERMO_REL)
    samples = s.run(30)
    o.run(30)
    assert np.array_equal(s.atoms()[0], o.atoms()[0])
    th = o.thermo()
    for k in ("T", "P", "PE", "E"):
        assert samples[-1][k] == pytest.approx(th[k], rel=THERMO_REL)


@pytest.mark.parametrize("precision", ["mixed", "mixed_comp"])
@pytest.mark.parametrize("half", [0, 1])
def test_mixed_lj_force_error_budget(precision, half):
    """Mixed forces against FP64 on a melted (non-lattice) snapshot."""
    kw = dict(nx=8, ny=8, nz=8, half_neigh=half)
    ref, _ = lj_system(**kw)
    ref.run(200)
    x, v, _, t = ref.atoms()
    ref.set_atoms(x, v, t)
    ref.setup()
    mx, _ = lj_system(precision=precision, **kw)
    mx.set_atoms(x, v, t)
    mx.setup()
    emax, erms = rel_err(mx.atoms()[2], ref.atoms()[2])
    assert erms <= MIXED_RMS, (emax, erms)
    assert mx.thermo()["PE"] == pytest.approx(ref.thermo()["PE"], rel=1e-6)


@pytest.mark.parametrize("precision", ["mixed", "mixed_comp"])
def test_mixed_eam_force_error_budget(precision):
    """On a thermalised state: the fixture starts on a perfect lattice, where
    net forces cancel to rounding level and no relative measure is meaningful."""
    g = dict(np.load(os.path.join(GOLDEN, "eam_cu_6x6x6.npz")))
    ref = eam_pair(g)
    ref.run(300)
    x, v, _, t = ref.atoms()
    ref.set_atoms(x, v, t)
    ref.setup()
    mx = eam_pair(g, precision=precision)
    mx.set_atoms(x, v, t)
    mx.setup()
    emax, erms = rel_err(mx.atoms()[2], ref.atoms()[2])
    assert erms <= MIXED_RMS, (emax, erms)


def test_full_size_properties():
    """64^3 cells (1,048,576 atoms): size-independent checks where the oracle is
    too slow: zero net force, FP64 determinism, half == full, mixed budget."""
    kw = dict(nx=64, ny=64, nz=64)
    a, _ = lj_system(**kw)
    b, _ = lj_system(**kw)
    fa = a.atoms()[2]
    assert np.array_equal(fa, b.atoms()[2])
    rms = np.sqrt(np.mean(np.sum(fa * fa, axis=1)))
    a.run(40)
    b.run(40)
    xa, va, fa, _ = a.atoms()
    assert np.array_equal(xa, b.atoms()[0]) and np.array_equal(va, b.atoms()[1])
    assert np.abs(fa.sum(axis=0)).max() <= 1e-9 * max(rms, 1.0) * len(fa)
    x, v, _, t = a.atoms()
    h, _ = lj_system(half_neigh=1, **kw)
    h.set_atoms(x, v, t)
    h.setup()
    a.set_atoms(x, v, t)
    a.setup()
    assert_forces_close(h.atoms()[2], a.atoms()[2])
    m, _ = lj_system(precision="mixed", **kw)
    m.set_atoms(x, v, t)
    m.setup()
    assert rel_err(m.atoms()[2], a.atoms()[2])[1] <= MIXED_RMS


def test_launches_are_counted():
    s, _ = lj_system(nx=6, ny=6, nz=6)
    n0 = s.launches
    s.run(20)
    assert s.launches - n0 >= 19 * 4


# ---- the stub gather benchmark (verletlist/main-stub.c) -------------------------

@pytest.mark.parametrize("pattern", ["seq", "fix", "rand"])
@pytest.mark.parametrize("half", [0, 1])
def test_stub_list_forces(pattern, half):
    """Forces on the stub's synthetic lists: bit-identical to the oracle with
    full lists, within the atomics tolerance with half lists."""
    x, v, t, num, nb = mdb.stub_system(3000, pattern, 76, nreps=2)
    s, box, cut = mdb.stub_context(x, v, t, num, nb, half=half)
    s.compute_force()
    o = O.Oracle(nx=1, ny=1, nz=1, from_file=1, xprd=box, yprd=box, zprd=box, cutforce=cut,
                 skin=0.0, half_neigh=half)
    o.set_atoms(x, v, t)
    o.set_list(num, nb)
    o.force()
    f, fo = s.atoms()[2], o.atoms()[2]
    # the fix pattern lists atom i itself for i < 76 (as the reference's
    # does): those forces are NaN on both sides
    if half:
        ok = np.isfinite(fo).all(axis=1)
        assert np.array_equal(np.isfinite(f).all(axis=1), ok)
        scale = np.abs(fo[ok]).max()
        assert np.abs(f[ok] - fo[ok]).max() <= 1e-12 * scale
    else:
        assert np.array_equal(f, fo, equal_nan=True)
    s.close()


def test_stub_list_rejected_for_mixed_and_bad_entries():
    x, v, t, num, nb = mdb.stub_system(500, "seq", 8)
    s, _, _ = mdb.stub_context(x, v, t, num, nb)
    bad = nb.copy()
    bad[3, 2] = 500
    with pytest.raises(mdb.MdbError):
        s.set_neighbor_list(num, bad)
    s.close()
