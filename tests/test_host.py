"""Host side of the product without a GPU: the C-ABI library loads and exports
every symbol its headers declare, and the host setup (lattice, dump reader,
EAM splines, parameters) reproduces the oracle bit for bit."""
import os
import re

import numpy as np
import pytest

import mdb
import oracle as O
from conftest import EAM_FILE, GOLDEN, ROOT


def declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mdbh?_[a-z0-9_]+)\s*\(", src)))


@pytest.mark.parametrize("header,exports", [("mdb.h", mdb.EXPORTS),
                                            ("mdb_cp.h", mdb.CP_EXPORTS),
                                            ("mdb_host.h", mdb.HOST_EXPORTS)])
def test_library_exports_every_declared_symbol(header, exports):
    lib = mdb.load()
    names = declared(header)
    assert sorted(exports) == names
    for n in names:
        assert hasattr(lib, n), n


def test_status_strings():
    lib = mdb.load()
    assert lib.mdb_status_string(0) == b"ok"
    assert lib.mdb_status_string(3) == b"buffer overflow"


@pytest.mark.parametrize("cells", [(8, 8, 8), (5, 7, 6), (3, 3, 3), (12, 4, 9)])
def test_fcc_matches_oracle(cells):
    nx, ny, nz = cells
    hp = mdb.host_params(nx=nx, ny=ny, nz=nz)
    x, v, t = mdb.create_fcc(hp)
    o = O.Oracle(nx=nx, ny=ny, nz=nz)
    o.lattice()
    xo, vo, _, to = o.atoms()
    assert np.array_equal(x, xo) and np.array_equal(v, vo) and np.array_equal(t, to)
    p = o.params()
    assert hp.xprd == p["xprd"] and hp.cutneigh == p["cutneigh"] and hp.dtforce == p["dtforce"]


def test_fcc_matches_reference_fixture():
    g = dict(np.load(os.path.join(GOLDEN, "lj_full_5x5x5.npz")))
    x, v, t = mdb.create_fcc(mdb.host_params(nx=5, ny=5, nz=5))
    assert np.array_equal(x, g["x0"]) and np.array_equal(v, g["v0"])
    assert np.array_equal(t, g["type"])


def test_eam_splines_match_oracle():
    t = mdb.read_funcfl(EAM_FILE)
    o = O.Oracle(eam_file=EAM_FILE, force_field=1)
    ot = o.eam_tables()
    for k in ("frho_spline", "rhor_spline", "z2r_spline"):
        assert np.array_equal(t[k], ot[k])
    for k in ("nrho", "nr", "nrho_tot", "nr_tot", "mass"):
        assert t[k] == ot[k]


def test_eam_params_follow_initeam():
    t = mdb.read_funcfl(EAM_FILE)
    hp = mdb.host_params(eam=t, nx=4, ny=4, nz=4)
    mdb.load().mdbh_finalize(hp)
    o = O.Oracle(eam_file=EAM_FILE, force_field=1, nx=4, ny=4, nz=4)
    o.lattice()
    p = o.params()
    assert hp.cutneigh == p["cutneigh"] and hp.dtforce == p["dtforce"]
    assert hp.xprd == p["xprd"] and hp.mass == p["mass"]


def test_dump_roundtrip_and_reader(tmp_path):
    g = dict(np.load(os.path.join(GOLDEN, "eam_cu_6x6x6.npz")))
    path = str(tmp_path / "cu.dmp")
    mdb.write_dmp(path, g["x0"], g["v0"], g["type"], tuple(g["box"]))
    hp = mdb.host_params()
    x, v, t = mdb.read_dmp(hp, path)
    assert np.array_equal(x, g["x0"]) and np.array_equal(v, g["v0"])
    assert np.array_equal(t, g["type"]) and hp.from_file == 1
    assert hp.xprd == g["box"][0]


def test_dump_reader_rejects_truncated_file(tmp_path):
    path = tmp_path / "bad.dmp"
    path.write_text("ITEM: TIMESTEP\n0\nITEM: NUMBER OF ATOMS\n4\nITEM: BOX BOUNDS pp pp pp\n"
                    "0 1\n0 1\n0 1\nITEM: ATOMS id type x y z vx vy vz\n1 1 0 0 0 0 0 0\n")
    with pytest.raises(mdb.MdbError):
        mdb.read_dmp(mdb.host_params(), str(path))


def test_reference_dump_files_parse():
    """The reference's copper inputs use the same dump layout (1-based types)."""
    import oracle as O
    tree = O.reference_tree()
    if tree is None:
        pytest.skip("reference tree not present")
    ref = os.path.join(tree, "data", "copper_melting", "input_eam_cu_one_atomtype_20x20x20.dmp")
    hp = mdb.host_params()
    x, v, t = mdb.read_dmp(hp, ref)
    assert len(t) == 32000 and hp.xprd == pytest.approx(72.3) and set(t.tolist()) == {1}


def test_param_and_types_files(tmp_path):
    (tmp_path / "types.dat").write_text("# eps sigma\n1.0 1.0\n4.0 2.0\n")
    (tmp_path / "p.conf").write_text(f"types_file {tmp_path / 'types.dat'}\nnx 10\n"
                                     "dt 0.001\ncutforce 2.0 # comment\nskin 0.2\n")
    hp = mdb.host_params()
    assert mdb.load().mdbh_read_params(hp, str(tmp_path / "p.conf").encode()) == 0
    mdb.load().mdbh_finalize(hp)
    assert hp.ntypes == 2 and hp.has_types == 1 and hp.nx == 10
    assert list(hp.sigma_per_type)[:2] == [1.0, 2.0]
    assert hp.cutneigh == 2.0 + 0.2 and hp.dtforce == 0.5 * 0.001
    (tmp_path / "bad.conf").write_text(f"types_file {tmp_path / 'types.dat'}\nepsilon 2\n")
    assert mdb.load().mdbh_read_params(mdb.host_params(), str(tmp_path / "bad.conf").encode())


# ---- the other input formats of readAtom, and the writers ----------------------

def _argon_state(n=400, box=(16.0, 17.5, 15.25), seed=3):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.0, 1.0, (n, 3)) * np.array(box)
    v = rng.normal(0.0, 0.3, (n, 3))
    return np.round(x, 3), np.round(v, 4), box


def _write_gro(path, x, v, box):
    with open(path, "w") as f:
        f.write("Liquid argon test state\n")
        f.write(f" {len(x)}\n")
        for i, (p, q) in enumerate(zip(x, v)):
            f.write(f"{i + 1:5d}Ar      Ar {i + 1:4d} {p[0]:7.3f} {p[1]:7.3f} {p[2]:7.3f}"
                    f" {q[0]:7.4f} {q[1]:7.4f} {q[2]:7.4f}\n")
        f.write(f" {box[0]:9.5f} {box[1]:9.5f} {box[2]:9.5f}\n")


def _write_pdb(path, x, box):
    with open(path, "w") as f:
        f.write("HEADER    test\nREMARK    argon\n")
        f.write(f"CRYST1 {box[0]:.3f} {box[1]:.3f} {box[2]:.3f} 90.00 90.00 90.00 P 1 1\n")
        f.write("MODEL 1\n")
        for i, p in enumerate(x):
            f.write(f"ATOM {i + 1} Ar AR {i + 1} {p[0]:.3f} {p[1]:.3f} {p[2]:.3f} 1.00 0.00\n")
        f.write("TER\nENDMDL\n")


def _write_in(path, x, v, box, mass=39.94):
    with open(path, "w") as f:
        f.write(f"{len(x)} 0.0 {box[0]} 0.0 {box[1]} 0.0 {box[2]}\n")
        for k, (p, q) in enumerate(zip(x, v)):
            m = "inf" if k == 0 else f"{mass}"
            f.write(f"{m} {p[0]} {p[1]} {p[2]} {q[0]} {q[1]} {q[2]}\n")


@pytest.mark.parametrize("ext", ["gro", "pdb", "in"])
def test_readers_parse_formats(tmp_path, ext):
    x, v, box = _argon_state()
    path = str(tmp_path / f"argon.{ext}")
    {"gro": lambda: _write_gro(path, x, v, box), "pdb": lambda: _write_pdb(path, x, box),
     "in": lambda: _write_in(path, x, v, box)}[ext]()
    hp = mdb.host_params()
    xr, vr, tr = mdb.read_atoms(hp, path)
    assert xr.shape == x.shape and np.allclose(xr, x, atol=5e-4)
    if ext == "pdb":
        assert np.all(vr == 0.0)
    else:
        assert np.allclose(vr, v, atol=5e-5)
    assert set(tr.tolist()) == {0} and hp.ntypes == 1 and hp.from_file == 1
    assert (hp.xprd, hp.yprd, hp.zprd) == pytest.approx(box, abs=1e-3)
    if ext == "in":
        assert hp.mass == pytest.approx(39.94)


@pytest.mark.skipif(not O.ref_available(), reason="reference not compiled here")
@pytest.mark.parametrize("ext", ["gro", "pdb", "in"])
def test_readers_match_reference_readers(tmp_path, ext):
    """The same file read by the reference's readAtom (compiled from its
    sources) and by mdbh_read_atoms: identical positions, velocities, types,
    box (and mass)."""
    x, v, box = _argon_state(n=300, box=(14.0, 14.5, 15.0))
    path = str(tmp_path / f"argon.{ext}")
    {"gro": lambda: _write_gro(path, x, v, box), "pdb": lambda: _write_pdb(path, x, box),
     "in": lambda: _write_in(path, x, v, box)}[ext]()
    hp = mdb.host_params()
    xr, vr, tr = mdb.read_atoms(hp, path)
    r = O.RefVL(input_file=path)
    assert r.nlocal == len(tr)
    xo, vo, _, to = r.atoms()
    assert np.array_equal(xr, xo) and np.array_equal(vr, vo) and np.array_equal(tr, to)
    d = r.params()
    assert (hp.xprd, hp.yprd, hp.zprd) == (d["xprd"], d["yprd"], d["zprd"])
    if ext == "in":
        assert hp.mass == d["mass"]


def test_readers_reject_bad_input(tmp_path):
    bad = tmp_path / "bad.pdb"
    bad.write_text("CRYST1 10 10 10\nATOM 1 Xe XE 1 1.0 1.0 1.0 1.00 0.00\n")
    with pytest.raises(mdb.MdbError):
        mdb.read_atoms(mdb.host_params(), str(bad))
    short = tmp_path / "short.gro"
    short.write_text("t\n 3\n    1Ar      Ar    1   1.0 1.0 1.0 0 0 0\n")
    with pytest.raises(mdb.MdbError):
        mdb.read_atoms(mdb.host_params(), str(short))
    with pytest.raises(mdb.MdbError):
        mdb.read_atoms(mdb.host_params(), str(tmp_path / "atoms.xyz"))


def test_atom_and_vtk_writers(tmp_path):
    x, v, box = _argon_state(n=5)
    t = np.array([0, 1, 0, 2, 0], dtype=np.int32)
    mdb.write_atoms(str(tmp_path / "w.csv"), x, v, t)
    lines = (tmp_path / "w.csv").read_text().splitlines()
    assert len(lines) == 5
    f = lines[3].split(",")
    assert f[0] == "2" and f[1] == "1.000000" and f[-1] == "0" and len(f) == 9
    assert float(f[2]) == pytest.approx(x[3, 0], abs=1e-6)
    mdb.write_vtk(str(tmp_path / "traj"), 7, x)
    vtk = (tmp_path / "traj_7.vtk").read_text().splitlines()
    assert vtk[0] == "# vtk DataFile Version 2.0" and vtk[4] == "POINTS 5 double"
    assert "CELLS 5 10" in vtk and "CELL_TYPES 5" in vtk and "POINT_DATA 5" in vtk
    assert vtk[5] == "%.4f %.4f %.4f" % tuple(x[0])


# ---- the stub gather benchmark's inputs (verletlist/main-stub.c) ----------------

def test_stub_patterns():
    n, nn = 300, 16
    x, v, t, num, nb = mdb.stub_system(n, "seq", nn, nreps=2)
    assert np.all(num == 2 * nn) and nb.shape == (n, 2 * nn)
    i = np.arange(n)[:, None]
    assert np.array_equal(nb[:, :nn], (i + 1 + np.arange(nn)[None, :]) % n)
    assert np.array_equal(nb[:, nn:], nb[:, :nn])
    assert np.array_equal(x[:, 0], np.arange(n) * 0.00001) and np.all(v == 0)
    assert t.min() >= 0 and t.max() < 4
    _, _, _, _, fix = mdb.stub_system(n, "fix", nn)
    assert np.all(fix == np.arange(nn)[None, :])
    _, _, t1, _, rnd = mdb.stub_system(n, "rand", nn)
    assert np.all((rnd >= 0) & (rnd < n)) and np.all(rnd != i)
    assert all(len(set(r)) == nn for r in rnd.tolist())
    _, _, t2, _, rnd2 = mdb.stub_system(n, "rand", nn)
    assert np.array_equal(rnd, rnd2) and np.array_equal(t1, t2)  # seeded
    with pytest.raises(mdb.MdbError):
        mdb.stub_system(10, "rand", 16)  # the reference's own precondition


def test_stub_force_oracle_matches_direct_sum():
    """The oracle's computeForceLJFullNeigh on a stub list equals a direct
    double-precision sum of the same pairs, to 1e-13 of the sum of the terms'
    magnitudes (the pair terms span many orders and cancel)."""
    n, nn = 200, 12
    x, v, t, num, nb = mdb.stub_system(n, "rand", nn)
    o = O.Oracle(nx=1, ny=1, nz=1, from_file=1, xprd=2.0, yprd=2.0, zprd=2.0, cutforce=10.0,
                 skin=0.0)
    o.set_atoms(x, v, t)
    o.set_list(num, nb)
    o.force()
    f = o.atoms()[2]
    d = x[:, None, :] - x[nb]
    r2 = np.sum(d * d, axis=2)
    sr2 = 1.0 / r2
    sr6 = sr2 ** 3
    fr = 48.0 * sr6 * (sr6 - 0.5) * sr2
    terms = d * fr[:, :, None]
    fd = np.sum(terms, axis=1)
    scale = np.sum(np.abs(terms), axis=1)
    assert np.all(np.abs(f - fd) <= 1e-13 * scale)
