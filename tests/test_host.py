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
    ref = "/root/reference/data/copper_melting/input_eam_cu_one_atomtype_20x20x20.dmp"
    if not os.path.exists(ref):
        pytest.skip("reference tree not present")
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
