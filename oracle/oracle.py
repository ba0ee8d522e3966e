"""ctypes front end for the CPU checkers (TEST INFRASTRUCTURE ONLY).

* ``Oracle``  wraps ``liboracle.so``, the plain-C restatement of the MD-Bench
  Verlet-list timestep (oracle/mdb_oracle.c).
* ``RefVL``   wraps ``_ref/libmdbref_vl.so``, the reference's own sources
  compiled here with a small driver shim (oracle/ref_vl_shim.c). It exists only
  where the reference tree was present at build time.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
use this module, and only as the checker.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmdbref_vl.so")
REF_BIN = os.path.join(HERE, "_ref", "MDBench-VL")
REF_TREE_FILE = os.path.join(HERE, "_ref", "reference_tree.txt")


def reference_tree():
    """The MD-Bench source tree the checkers were built from (recorded by
    oracle/Makefile), or None where it is absent (e.g. on a GPU host)."""
    try:
        with open(REF_TREE_FILE) as f:
            path = f.read().strip()
    except OSError:
        return None
    return path if path and os.path.isdir(path) else None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


class OrcParams(C.Structure):
    _fields_ = [
        ("force_field", C.c_int), ("half_neigh", C.c_int),
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("ntypes", C.c_int), ("from_file", C.c_int),
        ("pbc_x", C.c_int), ("pbc_y", C.c_int), ("pbc_z", C.c_int),
        ("reneigh_every", C.c_int), ("nstat", C.c_int),
        ("rho", C.c_double), ("temp", C.c_double), ("mass", C.c_double),
        ("dt", C.c_double), ("cutforce", C.c_double), ("skin", C.c_double),
        ("epsilon", C.c_double), ("sigma", C.c_double),
        ("xprd", C.c_double), ("yprd", C.c_double), ("zprd", C.c_double),
        ("epsilon_per_type", C.POINTER(C.c_double)),
        ("sigma_per_type", C.POINTER(C.c_double)),
    ]


def default_params(**kw):
    """Reference defaults, common/parameter.c:73-124 (geometric rule, 4 types)."""
    p = dict(force_field=0, half_neigh=0, nx=32, ny=32, nz=32, ntypes=4, from_file=0,
             pbc_x=1, pbc_y=1, pbc_z=1, reneigh_every=20, nstat=100, rho=0.8442,
             temp=1.44, mass=1.0, dt=0.005, cutforce=2.5, skin=0.3, epsilon=1.0,
             sigma=1.0, xprd=0.0, yprd=0.0, zprd=0.0)
    p.update(kw)
    return p


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError(f"{ORACLE_SO} missing: run `make -C oracle`")
        lib = C.CDLL(ORACLE_SO)
        lib.orc_create.restype = C.c_void_p
        lib.orc_create.argtypes = [C.POINTER(OrcParams)]
        lib.orc_destroy.argtypes = [C.c_void_p]
        for name in ("orc_lattice", "orc_setup", "orc_build_neighbor", "orc_setup_pbc",
                     "orc_nlocal", "orc_nghost", "orc_maxneighs"):
            getattr(lib, name).argtypes = [C.c_void_p]
            getattr(lib, name).restype = C.c_int
        for name in ("orc_update_pbc", "orc_update_atoms_pbc", "orc_initial_integrate",
                     "orc_final_integrate", "orc_sort_atoms"):
            getattr(lib, name).argtypes = [C.c_void_p]
            getattr(lib, name).restype = None
        lib.orc_compute_force.argtypes = [C.c_void_p]
        lib.orc_compute_force.restype = C.c_double
        lib.orc_step.argtypes = [C.c_void_p, C.c_int]
        lib.orc_set_resort.argtypes = [C.c_void_p, C.c_int]
        lib.orc_set_list.argtypes = [C.c_void_p, _ip, _ip, C.c_int]
        lib.orc_load_eam.argtypes = [C.c_void_p, C.c_char_p]
        lib.orc_load_eam.restype = C.c_int
        lib.orc_eam_info.argtypes = [C.c_void_p] + [C.POINTER(C.c_int)] * 4 + \
            [C.POINTER(C.c_double)] * 4
        lib.orc_eam_tables.argtypes = [C.c_void_p, _dp, _dp, _dp]
        lib.orc_set_atoms.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _ip]
        lib.orc_set_atoms.restype = C.c_int
        lib.orc_thermo.argtypes = [C.c_void_p] + [C.POINTER(C.c_double)] * 4
        lib.orc_get_atoms.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p]
        lib.orc_get_positions_all.argtypes = [C.c_void_p, _dp]
        lib.orc_set_state.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        lib.orc_get_ghosts.argtypes = [C.c_void_p, _ip, _ip]
        lib.orc_get_list.argtypes = [C.c_void_p, _ip, _ip, C.c_int]
        lib.orc_get_eam_fp.argtypes = [C.c_void_p, _dp]
        lib.orc_bin_geometry.argtypes = [C.c_void_p, _ip, _dp, _ip]
        lib.orc_get_params.argtypes = [C.c_void_p, _dp]
        _lib = lib
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Oracle:
    """One Verlet-list system held by the C restatement."""

    def __init__(self, eam_file=None, epsilon_per_type=None, sigma_per_type=None, **kw):
        self.lib = _load()
        self.pd = default_params(**kw)
        self._keep = []
        p = OrcParams(**{k: v for k, v in self.pd.items()})
        if epsilon_per_type is not None:
            e = np.ascontiguousarray(epsilon_per_type, dtype=np.float64)
            s = np.ascontiguousarray(sigma_per_type, dtype=np.float64)
            self._keep += [e, s]
            p.epsilon_per_type = e.ctypes.data_as(C.POINTER(C.c_double))
            p.sigma_per_type = s.ctypes.data_as(C.POINTER(C.c_double))
        self.h = self.lib.orc_create(C.byref(p))
        if eam_file is not None:
            rc = self.lib.orc_load_eam(self.h, eam_file.encode())
            if rc != 0:
                raise RuntimeError(f"oracle: cannot read EAM file {eam_file} ({rc})")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    # -- construction -------------------------------------------------------
    def lattice(self):
        return self.lib.orc_lattice(self.h)

    def set_atoms(self, x, v, type_):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
        v = np.ascontiguousarray(v, dtype=np.float64).reshape(-1)
        t = np.ascontiguousarray(type_, dtype=np.int32)
        return self.lib.orc_set_atoms(self.h, len(t), x, v, t)

    def setup(self):
        return self.lib.orc_setup(self.h)

    # -- hooks --------------------------------------------------------------
    def force(self):
        return self.lib.orc_compute_force(self.h)

    def step(self, n):
        self.lib.orc_step(self.h, n)

    def run(self, nsteps, start=0):
        for n in range(start, start + nsteps):
            self.lib.orc_step(self.h, n)

    def rebuild(self):
        self.lib.orc_update_atoms_pbc(self.h)
        self.lib.orc_setup_pbc(self.h)
        self.lib.orc_update_pbc(self.h)
        self.lib.orc_build_neighbor(self.h)

    def sort_atoms(self):
        """sortAtom; ghosts and lists are cleared (rebuild before a force)."""
        self.lib.orc_sort_atoms(self.h)

    def set_resort(self, every):
        self.lib.orc_set_resort(self.h, every)

    def set_list(self, numneigh, neighbors):
        """A caller's list of locals (rows of neighbors.shape[1] entries)."""
        nb = np.ascontiguousarray(neighbors, dtype=np.int32)
        self.lib.orc_set_list(self.h, np.ascontiguousarray(numneigh, dtype=np.int32), nb,
                              nb.shape[1])

    def reghost(self):
        """setupPbc + updatePbc + buildNeighbor without the wrap."""
        self.lib.orc_setup_pbc(self.h)
        self.lib.orc_update_pbc(self.h)
        self.lib.orc_build_neighbor(self.h)

    # -- state --------------------------------------------------------------
    @property
    def nlocal(self):
        return self.lib.orc_nlocal(self.h)

    @property
    def nghost(self):
        return self.lib.orc_nghost(self.h)

    @property
    def maxneighs(self):
        return self.lib.orc_maxneighs(self.h)

    def atoms(self):
        n = self.nlocal
        x = np.zeros((n, 3)); v = np.zeros((n, 3)); f = np.zeros((n, 3))
        t = np.zeros(n + self.nghost, dtype=np.int32)
        self.lib.orc_get_atoms(self.h, _ptr(x), _ptr(v), _ptr(f), _ptr(t))
        return x, v, f, t[:n]

    def positions_all(self):
        x = np.zeros((self.nlocal + self.nghost, 3))
        self.lib.orc_get_positions_all(self.h, x.reshape(-1))
        return x

    def set_state(self, x=None, v=None):
        xs = None if x is None else np.ascontiguousarray(x, dtype=np.float64)
        vs = None if v is None else np.ascontiguousarray(v, dtype=np.float64)
        self.lib.orc_set_state(self.h, _ptr(xs), _ptr(vs))

    def ghosts(self):
        ng = self.nghost
        bm = np.zeros(max(ng, 1), dtype=np.int32)
        pb = np.zeros(max(3 * ng, 3), dtype=np.int32)
        self.lib.orc_get_ghosts(self.h, bm, pb)
        return bm[:ng], pb[:3 * ng].reshape(ng, 3)

    def neighbor_list(self):
        n = self.nlocal
        ld = self.maxneighs
        nn = np.zeros(n, dtype=np.int32)
        nb = np.zeros(n * ld, dtype=np.int32)
        self.lib.orc_get_list(self.h, nn, nb, ld)
        return nn, nb.reshape(n, ld)

    def eam_fp(self):
        fp = np.zeros(self.nlocal + self.nghost)
        self.lib.orc_get_eam_fp(self.h, fp)
        return fp

    def eam_tables(self):
        ints = [C.c_int() for _ in range(4)]
        dbls = [C.c_double() for _ in range(4)]
        rc = self.lib.orc_eam_info(self.h, *[C.byref(i) for i in ints],
                                   *[C.byref(d) for d in dbls])
        if rc:
            raise RuntimeError("oracle: no EAM tables loaded")
        nrho, nr, nrho_tot, nr_tot = [i.value for i in ints]
        drho, dr, cut, mass = [d.value for d in dbls]
        fr = np.zeros(nrho_tot); rr = np.zeros(nr_tot); zr = np.zeros(nr_tot)
        self.lib.orc_eam_tables(self.h, fr, rr, zr)
        return dict(nrho=nrho, nr=nr, nrho_tot=nrho_tot, nr_tot=nr_tot, drho=drho, dr=dr,
                    cut=cut, mass=mass, frho_spline=fr, rhor_spline=rr, z2r_spline=zr)

    def bin_geometry(self):
        ints = np.zeros(10, dtype=np.int32)
        dbls = np.zeros(7)
        st = np.zeros(4096, dtype=np.int32)
        self.lib.orc_bin_geometry(self.h, ints, dbls, st)
        keys_i = ["nbinx", "nbiny", "nbinz", "mbinx", "mbiny", "mbinz", "pad_x", "pad_y",
                  "pad_z", "nstencil"]
        keys_d = ["binsizex", "binsizey", "binsizez", "bininvx", "bininvy", "bininvz",
                  "cutneigh"]
        g = {k: int(v) for k, v in zip(keys_i, ints)}
        g.update({k: float(v) for k, v in zip(keys_d, dbls)})
        g["stencil"] = st[:g["nstencil"]].copy()
        return g

    def params(self):
        d = np.zeros(8)
        self.lib.orc_get_params(self.h, d)
        return dict(zip(["xprd", "yprd", "zprd", "dt", "dtforce", "mass", "cutforce",
                         "cutneigh"], d.tolist()))

    def thermo(self):
        vals = [C.c_double() for _ in range(4)]
        self.lib.orc_thermo(self.h, *[C.byref(v) for v in vals])
        T, P, KE, PE = [v.value for v in vals]
        return dict(T=T, P=P, KE=KE, PE=PE, E=KE + PE)


# ----------------------------------------------------------------------------
_ref = None


def ref_available():
    return os.path.exists(REF_SO)


def _load_ref():
    global _ref
    if _ref is None:
        lib = C.CDLL(REF_SO)
        lib.ref_vl_setup.argtypes = [C.c_int] * 5 + [C.c_char_p] * 3
        lib.ref_vl_setup.restype = C.c_int
        for n in ("ref_vl_nlocal", "ref_vl_nghost", "ref_vl_maxneighs"):
            getattr(lib, n).restype = C.c_int
        lib.ref_vl_params.argtypes = [_dp]
        lib.ref_vl_get_atoms.argtypes = [C.c_void_p] * 4 + [C.c_int]
        lib.ref_vl_set_state.argtypes = [C.c_void_p, C.c_void_p]
        lib.ref_vl_get_ghosts.argtypes = [_ip, _ip]
        lib.ref_vl_get_list.argtypes = [_ip, _ip, C.c_int]
        lib.ref_vl_force.restype = C.c_double
        lib.ref_vl_step.argtypes = [C.c_int]
        lib.ref_vl_sort.argtypes = []
        lib.ref_vl_thermo.argtypes = [C.POINTER(C.c_double)] * 2
        lib.ref_vl_set_threads.argtypes = [C.c_int]
        _ref = lib
    return _ref


class RefVL:
    """The reference itself (one system per process: its state is global)."""

    def __init__(self, nx=8, ny=8, nz=8, half=0, force_field=0, param_file=None,
                 input_file=None, eam_file=None):
        self.lib = _load_ref()
        self.lib.ref_vl_set_threads(1 if half else os.cpu_count())
        enc = lambda s: None if s is None else s.encode()
        self.lib.ref_vl_setup(nx, ny, nz, half, force_field, enc(param_file),
                              enc(input_file), enc(eam_file))

    @property
    def nlocal(self):
        return self.lib.ref_vl_nlocal()

    @property
    def nghost(self):
        return self.lib.ref_vl_nghost()

    def atoms(self, include_ghosts=False):
        n = self.nlocal + (self.nghost if include_ghosts else 0)
        x = np.zeros((n, 3)); v = np.zeros((n, 3)); f = np.zeros((n, 3))
        t = np.zeros(n, dtype=np.int32)
        self.lib.ref_vl_get_atoms(_ptr(x), _ptr(v), _ptr(f), _ptr(t), n)
        return x, v, f, t

    def set_state(self, x=None, v=None):
        xs = None if x is None else np.ascontiguousarray(x, dtype=np.float64)
        vs = None if v is None else np.ascontiguousarray(v, dtype=np.float64)
        self.lib.ref_vl_set_state(_ptr(xs), _ptr(vs))

    def ghosts(self):
        ng = self.nghost
        bm = np.zeros(max(ng, 1), dtype=np.int32)
        pb = np.zeros(max(3 * ng, 3), dtype=np.int32)
        self.lib.ref_vl_get_ghosts(bm, pb)
        return bm[:ng], pb[:3 * ng].reshape(ng, 3)

    def neighbor_list(self):
        n = self.nlocal
        ld = self.lib.ref_vl_maxneighs()
        nn = np.zeros(n, dtype=np.int32)
        nb = np.zeros(n * ld, dtype=np.int32)
        self.lib.ref_vl_get_list(nn, nb, ld)
        return nn, nb.reshape(n, ld)

    def force(self):
        return self.lib.ref_vl_force()

    def step(self, n):
        self.lib.ref_vl_step(n)

    def sort_atoms(self):
        """The reference's sortAtom (moves positions and velocities only)."""
        self.lib.ref_vl_sort()

    def params(self):
        d = np.zeros(8)
        self.lib.ref_vl_params(d)
        return dict(zip(["xprd", "yprd", "zprd", "dt", "dtforce", "mass", "cutforce",
                         "cutneigh"], d.tolist()))

    def thermo(self):
        T = C.c_double(); P = C.c_double()
        self.lib.ref_vl_thermo(C.byref(T), C.byref(P))
        return dict(T=T.value, P=P.value)


# ---------------------------------------------------------------------------
# cluster-pair scheme
REF_CP_SO = {shape: os.path.join(HERE, "_ref", f"libmdbref_cp_{shape}.so")
             for shape in ("1x2", "4x4", "4x8")}
REF_CP_BIN = {shape: os.path.join(HERE, "_ref", f"MDBench-CP-{shape}")
              for shape in ("4x4", "4x8")}


class OrcCpParams(C.Structure):
    _fields_ = [
        ("cluster_m", C.c_int), ("cluster_n", C.c_int), ("fma_rsq", C.c_int),
        ("half_neigh", C.c_int), ("ntypes", C.c_int), ("natoms", C.c_int),
        ("reneigh_every", C.c_int), ("prune_every", C.c_int), ("nstat", C.c_int),
        ("xprd", C.c_double), ("yprd", C.c_double), ("zprd", C.c_double),
        ("dt", C.c_double), ("dtforce", C.c_double), ("mass", C.c_double),
        ("cutforce", C.c_double), ("cutneigh", C.c_double),
        ("epsilon", C.c_double), ("sigma", C.c_double),
        ("epsilon_per_type", C.POINTER(C.c_double)),
        ("sigma_per_type", C.POINTER(C.c_double)),
    ]


_cp_lib = None


def _load_cp():
    global _cp_lib
    if _cp_lib is None:
        lib = _load()
        lib.orccp_create.restype = C.c_void_p
        lib.orccp_create.argtypes = [C.POINTER(OrcCpParams)]
        lib.orccp_destroy.argtypes = [C.c_void_p]
        lib.orccp_set_atoms.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _ip]
        for n in ("orccp_setup", "orccp_build_clusters", "orccp_setup_pbc",
                  "orccp_build_neighbor"):
            getattr(lib, n).argtypes = [C.c_void_p]
            getattr(lib, n).restype = C.c_int
        for n in ("orccp_define_jclusters", "orccp_bin_jclusters", "orccp_prune_neighbor",
                  "orccp_update_single_atoms", "orccp_update_atoms_pbc",
                  "orccp_initial_integrate", "orccp_final_integrate"):
            getattr(lib, n).argtypes = [C.c_void_p]
            getattr(lib, n).restype = None
        lib.orccp_update_pbc.argtypes = [C.c_void_p, C.c_int]
        lib.orccp_compute_force.argtypes = [C.c_void_p]
        lib.orccp_compute_force.restype = C.c_double
        lib.orccp_step.argtypes = [C.c_void_p, C.c_int]
        lib.orccp_thermo.argtypes = [C.c_void_p] + [C.POINTER(C.c_double)] * 2
        lib.orccp_energy.argtypes = [C.c_void_p] + [C.POINTER(C.c_double)] * 2
        lib.orccp_counts.argtypes = [C.c_void_p, _ip]
        lib.orccp_get_atoms.argtypes = [C.c_void_p] + [C.c_void_p] * 3
        lib.orccp_get_slots.argtypes = [C.c_void_p] + [C.c_void_p] * 4 + [C.c_int]
        lib.orccp_set_slots.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        lib.orccp_get_iclusters.argtypes = [C.c_void_p, _ip, C.c_void_p, C.c_void_p]
        lib.orccp_get_jclusters.argtypes = [C.c_void_p, _ip, C.c_void_p, C.c_int]
        lib.orccp_get_ghosts.argtypes = [C.c_void_p, _ip, _ip]
        lib.orccp_get_list.argtypes = [C.c_void_p, _ip, C.c_void_p, _ip, C.c_void_p, C.c_int]
        lib.orccp_bin_geometry.argtypes = [C.c_void_p, _ip, _dp, C.c_void_p]
        lib.orccp_get_columns.argtypes = [C.c_void_p, _ip, _ip, C.c_int]
        lib.orccp_get_columns.restype = C.c_int
        _cp_lib = lib
    return _cp_lib


def _cp_counts(c):
    return dict(zip(["nlocal", "natoms", "ncl", "ncj", "ngc", "nghost", "dummy",
                     "maxneighs"], [int(v) for v in c]))


class _CpViews:
    """Shared getters of the cluster-pair oracle and the reference shim."""

    def nslots(self):
        c = self.counts()
        return (c["ncj"] + c["ngc"] + 1) * self.N

    def slots(self):
        ns = self.nslots()
        x = np.zeros((ns, 3)); v = np.zeros((ns, 3)); f = np.zeros((ns, 3))
        t = np.zeros(ns, dtype=np.int32)
        self._get_slots(_ptr(x), _ptr(v), _ptr(f), _ptr(t), ns)
        return x, v, f, t

    def neighbor_list(self):
        c = self.counts()
        n, ld = c["ncl"], c["maxneighs"]
        nn = np.zeros(max(n, 1), dtype=np.int32)
        nm = np.zeros(max(n, 1), dtype=np.int32)
        nb = np.zeros(max(n * ld, 1), dtype=np.int32)
        im = np.zeros(max(n * ld, 1), dtype=np.uint32)
        self._get_list(nn, nm, nb, im, ld)
        return nn[:n], nm[:n], nb[:n * ld].reshape(n, ld), im[:n * ld].reshape(n, ld)

    def ghosts(self):
        ng = self.counts()["ngc"]
        bm = np.zeros(max(ng, 1), dtype=np.int32)
        pb = np.zeros(max(3 * ng, 3), dtype=np.int32)
        self._get_ghosts(bm, pb)
        return bm[:ng], pb[:3 * ng].reshape(ng, 3)


class OracleCP(_CpViews):
    """One cluster-pair system held by the C restatement. Atoms come from the
    caller (normally the Verlet-list oracle's lattice, pinned to the reference's
    createAtom)."""

    def __init__(self, x, v, type_, M=4, N=4, fma_rsq=None, half=0, ntypes=4, natoms=None,
                 xprd=None, yprd=None, zprd=None, dt=0.005, dtforce=None, mass=1.0,
                 cutforce=2.5, cutneigh=2.8, epsilon=1.0, sigma=1.0, reneigh_every=20,
                 prune_every=1000, nstat=100, epsilon_per_type=None, sigma_per_type=None):
        self.lib = _load_cp()
        self.M, self.N = M, N
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)
        v = np.ascontiguousarray(v, dtype=np.float64).reshape(-1, 3)
        t = np.ascontiguousarray(type_, dtype=np.int32)
        n = len(x)
        p = OrcCpParams(cluster_m=M, cluster_n=N,
                        fma_rsq=int(M > 1 if fma_rsq is None else fma_rsq), half_neigh=half,
                        ntypes=ntypes, natoms=n if natoms is None else natoms,
                        reneigh_every=reneigh_every, prune_every=prune_every, nstat=nstat,
                        xprd=xprd, yprd=yprd, zprd=zprd, dt=dt,
                        dtforce=0.5 * dt if dtforce is None else dtforce, mass=mass,
                        cutforce=cutforce, cutneigh=cutneigh, epsilon=epsilon, sigma=sigma)
        self._keep = []
        if epsilon_per_type is not None:
            e = np.ascontiguousarray(epsilon_per_type, dtype=np.float64)
            s = np.ascontiguousarray(sigma_per_type, dtype=np.float64)
            self._keep += [e, s]
            p.epsilon_per_type = e.ctypes.data_as(C.POINTER(C.c_double))
            p.sigma_per_type = s.ctypes.data_as(C.POINTER(C.c_double))
        self.h = self.lib.orccp_create(C.byref(p))
        if not self.h:
            raise ValueError("oracle: unsupported cluster shape or types")
        self.lib.orccp_set_atoms(self.h, n, x.reshape(-1), v.reshape(-1), t)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orccp_destroy(self.h)
            self.h = None

    def setup(self):
        rc = self.lib.orccp_setup(self.h)
        if rc != 0:
            raise RuntimeError("oracle: atom outside the column grid")

    def counts(self):
        c = np.zeros(8, dtype=np.int32)
        self.lib.orccp_counts(self.h, c)
        return _cp_counts(c)

    def _get_slots(self, *a):
        self.lib.orccp_get_slots(self.h, *a)

    def _get_list(self, nn, nm, nb, im, ld):
        self.lib.orccp_get_list(self.h, nn, _ptr(nm), nb, _ptr(im), ld)

    def _get_ghosts(self, *a):
        self.lib.orccp_get_ghosts(self.h, *a)

    def set_slots(self, x=None, v=None):
        xs = None if x is None else np.ascontiguousarray(x, dtype=np.float64)
        vs = None if v is None else np.ascontiguousarray(v, dtype=np.float64)
        self.lib.orccp_set_slots(self.h, _ptr(xs), _ptr(vs))

    def iclusters(self):
        n = self.counts()["ncl"]
        nat = np.zeros(max(n, 1), dtype=np.int32); b = np.zeros(max(n, 1), dtype=np.int32)
        bb = np.zeros(max(6 * n, 6))
        self.lib.orccp_get_iclusters(self.h, nat, _ptr(b), _ptr(bb))
        return nat[:n], b[:n], bb[:6 * n].reshape(n, 6)

    def jclusters(self):
        c = self.counts()
        n = c["ncj"] + c["ngc"]
        nat = np.zeros(max(n, 1), dtype=np.int32); bb = np.zeros(max(6 * n, 6))
        self.lib.orccp_get_jclusters(self.h, nat, _ptr(bb), n)
        return nat[:n], bb[:6 * n].reshape(n, 6)

    def atoms(self):
        n = self.counts()["nlocal"]
        x = np.zeros((n, 3)); v = np.zeros((n, 3)); t = np.zeros(n, dtype=np.int32)
        self.lib.orccp_get_atoms(self.h, _ptr(x), _ptr(v), _ptr(t))
        return x, v, t

    def bin_geometry(self):
        ints = np.zeros(7, dtype=np.int32); d = np.zeros(3)
        self.lib.orccp_bin_geometry(self.h, ints, d, None)
        st = np.zeros(int(ints[6]), dtype=np.int32)
        self.lib.orccp_bin_geometry(self.h, ints, d, _ptr(st))
        keys = ["nbinx", "nbiny", "mbinx", "mbiny", "mbinxlo", "mbinylo", "nstencil"]
        g = dict(zip(keys, [int(i) for i in ints]))
        g.update(binsizex=d[0], binsizey=d[1], rbb_sq=d[2], stencil=st)
        return g

    def columns(self):
        g = self.bin_geometry()
        mb = g["mbinx"] * g["mbiny"]
        start = np.zeros(mb + 1, dtype=np.int32)
        n = self.lib.orccp_get_columns(self.h, start, np.zeros(1, dtype=np.int32), 0)
        lst = np.zeros(max(n, 1), dtype=np.int32)
        self.lib.orccp_get_columns(self.h, start, lst, n)
        return start, lst[:n]

    def force(self):
        return self.lib.orccp_compute_force(self.h)

    def prune(self):
        self.lib.orccp_prune_neighbor(self.h)

    def update_pbc(self, first=0):
        self.lib.orccp_update_pbc(self.h, first)

    def step(self, n):
        self.lib.orccp_step(self.h, n)

    def run(self, nsteps, start=0):
        for n in range(start, start + nsteps):
            self.step(n)

    def thermo(self):
        T = C.c_double(); P = C.c_double(); KE = C.c_double(); PE = C.c_double()
        self.lib.orccp_thermo(self.h, C.byref(T), C.byref(P))
        self.lib.orccp_energy(self.h, C.byref(KE), C.byref(PE))
        return dict(T=T.value, P=P.value, KE=KE.value, PE=PE.value, E=KE.value + PE.value)


_ref_cp = {}


def ref_cp_available(shape="4x4"):
    return os.path.exists(REF_CP_SO[shape])


def _load_ref_cp(shape):
    if shape not in _ref_cp:
        lib = C.CDLL(REF_CP_SO[shape])
        lib.ref_cp_shape.argtypes = [C.POINTER(C.c_int)] * 2
        lib.ref_cp_shape.restype = C.c_int
        lib.ref_cp_setup.argtypes = [C.c_int] * 4 + [C.c_char_p] * 2 + [C.c_int]
        lib.ref_cp_setup.restype = C.c_int
        lib.ref_cp_counts.argtypes = [_ip]
        lib.ref_cp_params.argtypes = [_dp]
        lib.ref_cp_get_atoms.argtypes = [C.c_void_p] * 3
        lib.ref_cp_get_slots.argtypes = [C.c_void_p] * 4 + [C.c_int]
        lib.ref_cp_get_iclusters.argtypes = [_ip, _ip, _dp]
        lib.ref_cp_get_jclusters.argtypes = [_ip, _dp, C.c_int]
        lib.ref_cp_get_ghosts.argtypes = [_ip, _ip]
        lib.ref_cp_get_list.argtypes = [_ip, _ip, _ip, C.c_void_p, C.c_int]
        lib.ref_cp_force.restype = C.c_double
        lib.ref_cp_step.argtypes = [C.c_int]
        lib.ref_cp_thermo.argtypes = [C.POINTER(C.c_double)] * 2
        lib.ref_cp_set_threads.argtypes = [C.c_int]
        _ref_cp[shape] = lib
    return _ref_cp[shape]


class RefCP(_CpViews):
    """The reference cluster-pair scheme itself, one build per cluster shape
    (one system per build and process: its state is global)."""

    def __init__(self, shape="4x4", nx=8, ny=8, nz=8, half=0, param_file=None,
                 input_file=None, prune_every=0, threads=1):
        self.lib = _load_ref_cp(shape)
        m = C.c_int(); n = C.c_int()
        self.lib.ref_cp_shape(C.byref(m), C.byref(n))
        self.M, self.N = m.value, n.value
        self.lib.ref_cp_set_threads(threads)
        enc = lambda s: None if s is None else s.encode()
        self.lib.ref_cp_setup(nx, ny, nz, half, enc(param_file), enc(input_file), prune_every)

    def counts(self):
        c = np.zeros(8, dtype=np.int32)
        self.lib.ref_cp_counts(c)
        return _cp_counts(c)

    def _get_slots(self, *a):
        self.lib.ref_cp_get_slots(*a)

    def _get_list(self, nn, nm, nb, im, ld):
        self.lib.ref_cp_get_list(nn, nm, nb, _ptr(im), ld)

    def _get_ghosts(self, *a):
        self.lib.ref_cp_get_ghosts(*a)

    def iclusters(self):
        n = self.counts()["ncl"]
        nat = np.zeros(max(n, 1), dtype=np.int32); b = np.zeros(max(n, 1), dtype=np.int32)
        bb = np.zeros(max(6 * n, 6))
        self.lib.ref_cp_get_iclusters(nat, b, bb)
        return nat[:n], b[:n], bb[:6 * n].reshape(n, 6)

    def jclusters(self):
        c = self.counts()
        n = c["ncj"] + c["ngc"]
        nat = np.zeros(max(n, 1), dtype=np.int32); bb = np.zeros(max(6 * n, 6))
        self.lib.ref_cp_get_jclusters(nat, bb, n)
        return nat[:n], bb[:6 * n].reshape(n, 6)

    def atoms(self):
        n = self.counts()["nlocal"]
        x = np.zeros((n, 3)); v = np.zeros((n, 3)); t = np.zeros(n, dtype=np.int32)
        self.lib.ref_cp_get_atoms(_ptr(x), _ptr(v), _ptr(t))
        return x, v, t

    def params(self):
        d = np.zeros(8)
        self.lib.ref_cp_params(d)
        return dict(zip(["xprd", "yprd", "zprd", "dt", "dtforce", "mass", "cutforce",
                         "cutneigh"], d.tolist()))

    def force(self):
        return self.lib.ref_cp_force()

    def step(self, n):
        self.lib.ref_cp_step(n)

    def thermo(self):
        T = C.c_double(); P = C.c_double()
        self.lib.ref_cp_thermo(C.byref(T), C.byref(P))
        return dict(T=T.value, P=P.value)
