"""Python binding of libmdb (the B200 MD-Bench timestep) over its C ABI.

This mirrors the reference's plugin surface (computeForce, buildNeighbor,
updatePbc, updateAtomsPbc, initialIntegrate, finalIntegrate, computeThermo)
one call per hook, plus the whole graph-captured loop (``System.run``).
Everything runs on the GPU; there is no CPU fallback: importing this module
without the built ``libmdb.so`` or calling it without a CUDA device raises.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmdb.so")

FF_LJ, FF_EAM = 0, 1
PREC_FP64, PREC_MIXED, PREC_MIXED_COMP = 0, 1, 2
BINS_LATTICE, BINS_FILE = 0, 1
PRECISIONS = {"fp64": PREC_FP64, "mixed": PREC_MIXED, "mixed_comp": PREC_MIXED_COMP}


class MdbError(RuntimeError):
    pass


class MdbParams(C.Structure):
    _fields_ = [
        ("force_field", C.c_int), ("half_neigh", C.c_int), ("precision", C.c_int),
        ("bin_rule", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("pbc_x", C.c_int), ("pbc_y", C.c_int), ("pbc_z", C.c_int), ("ntypes", C.c_int),
        ("reneigh_every", C.c_int), ("nstat", C.c_int), ("maxneighs", C.c_int),
        ("natoms", C.c_int), ("device", C.c_int),
        ("xprd", C.c_double), ("yprd", C.c_double), ("zprd", C.c_double),
        ("dt", C.c_double), ("dtforce", C.c_double), ("mass", C.c_double),
        ("cutforce", C.c_double), ("cutneigh", C.c_double),
        ("epsilon", C.c_double), ("sigma", C.c_double),
        ("epsilon_per_type", C.POINTER(C.c_double)),
        ("sigma_per_type", C.POINTER(C.c_double)),
    ]


class MdbEamTables(C.Structure):
    _fields_ = [
        ("nrho", C.c_int), ("nr", C.c_int), ("nrho_tot", C.c_int), ("nr_tot", C.c_int),
        ("rdr", C.c_double), ("rdrho", C.c_double), ("cut", C.c_double), ("mass", C.c_double),
        ("frho_spline", C.POINTER(C.c_double)), ("rhor_spline", C.POINTER(C.c_double)),
        ("z2r_spline", C.POINTER(C.c_double)),
    ]


class MdbHostParams(C.Structure):
    _fields_ = [
        ("force_field", C.c_int), ("half_neigh", C.c_int), ("precision", C.c_int),
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("ntypes", C.c_int),
        ("ntimes", C.c_int), ("nstat", C.c_int), ("reneigh_every", C.c_int),
        ("pbc_x", C.c_int), ("pbc_y", C.c_int), ("pbc_z", C.c_int), ("has_types", C.c_int),
        ("epsilon", C.c_double), ("sigma", C.c_double), ("rho", C.c_double),
        ("temp", C.c_double), ("mass", C.c_double), ("dt", C.c_double),
        ("cutforce", C.c_double), ("skin", C.c_double),
        ("epsilon_per_type", C.c_double * 8), ("sigma_per_type", C.c_double * 8),
        ("xprd", C.c_double), ("yprd", C.c_double), ("zprd", C.c_double),
        ("from_file", C.c_int),
        ("lattice", C.c_double), ("cutneigh", C.c_double), ("dtforce", C.c_double),
    ]


class MdbThermo(C.Structure):
    _fields_ = [("step", C.c_int), ("temperature", C.c_double), ("pressure", C.c_double),
                ("ke", C.c_double), ("pe", C.c_double), ("etotal", C.c_double)]

    def as_dict(self):
        return dict(step=self.step, T=self.temperature, P=self.pressure, KE=self.ke,
                    PE=self.pe, E=self.etotal)


# every symbol include/mdb.h declares
EXPORTS = [
    "mdb_create", "mdb_destroy", "mdb_status_string", "mdb_last_error", "mdb_stream",
    "mdb_synchronize", "mdb_set_eam", "mdb_eam_read_funcfl", "mdb_eam_free", "mdb_set_atoms",
    "mdb_get_atoms", "mdb_setup_pbc", "mdb_update_pbc", "mdb_update_atoms_pbc",
    "mdb_build_neighbor", "mdb_compute_force", "mdb_compute_force_energy",
    "mdb_initial_integrate", "mdb_final_integrate", "mdb_thermo", "mdb_setup", "mdb_run", "mdb_get_counts",
    "mdb_get_positions_all", "mdb_get_ghosts", "mdb_get_neighbor_list",
    "mdb_get_bin_geometry", "mdb_get_eam_fp", "mdb_launch_count", "mdb_kinetic_sum_noalloc",
    "mdb_fp32_fma_rate",
    "mdb_set_owned", "mdb_gather_positions", "mdb_set_halo_positions",
    "mdb_sort_atoms", "mdb_set_resort", "mdb_tune", "mdb_set_neighbor_list",
]
# every symbol include/mdb_cp.h declares
CP_EXPORTS = [
    "mdb_cp_create", "mdb_cp_destroy", "mdb_cp_last_error", "mdb_cp_stream", "mdb_cp_synchronize", "mdb_cp_tune",
    "mdb_cp_launch_count", "mdb_cp_set_atoms", "mdb_cp_get_atoms", "mdb_cp_build_clusters",
    "mdb_cp_define_jclusters", "mdb_cp_setup_pbc", "mdb_cp_update_pbc", "mdb_cp_bin_jclusters",
    "mdb_cp_build_neighbor", "mdb_cp_prune_neighbor", "mdb_cp_update_single_atoms",
    "mdb_cp_update_atoms_pbc", "mdb_cp_compute_force", "mdb_cp_compute_force_energy",
    "mdb_cp_initial_integrate", "mdb_cp_final_integrate", "mdb_cp_thermo", "mdb_cp_setup",
    "mdb_cp_run", "mdb_cp_get_counts", "mdb_cp_get_slots", "mdb_cp_get_iclusters",
    "mdb_cp_get_jclusters", "mdb_cp_get_ghosts", "mdb_cp_get_neighbor_list",
    "mdb_cp_get_columns", "mdb_cp_get_geometry", "mdb_cp_time_force", "mdb_cp_ensemble_create",
    "mdb_cp_ensemble_destroy", "mdb_cp_ensemble_last_error", "mdb_cp_ensemble_stream",
    "mdb_cp_ensemble_launch_count", "mdb_cp_ensemble_run", "mdb_cp_ensemble_tune",
    "mdb_cp_set_rebuild_check", "mdb_cp_get_rebuilds", "mdb_cp_set_pair_buffer",
    "mdb_cp_get_pair_stats", "mdb_cp_get_check_stats", "mdb_cp_ensemble_check_stats",
]
# every symbol include/mdb_host.h declares
HOST_EXPORTS = [
    "mdbh_defaults", "mdbh_read_params", "mdbh_read_types", "mdbh_apply_eam",
    "mdbh_finalize", "mdbh_create_fcc", "mdbh_read_dmp", "mdbh_write_dmp", "mdbh_mdb_params",
    "mdbh_read_pdb", "mdbh_read_gro", "mdbh_read_in", "mdbh_read_atoms", "mdbh_write_atoms",
    "mdbh_write_vtk", "mdbh_stub_atoms", "mdbh_stub_neighbors",
]

_lib = None
_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def load():
    """Load libmdb.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise MdbError(f"{LIB_PATH} is missing: build it with `make -C md-bench_b200`")
    lib = C.CDLL(LIB_PATH)
    vp, ip = C.c_void_p, C.c_int
    sig = {
        "mdb_create": ([C.POINTER(MdbParams), C.POINTER(vp)], ip),
        "mdb_destroy": ([vp], ip),
        "mdb_status_string": ([ip], C.c_char_p),
        "mdb_last_error": ([vp], C.c_char_p),
        "mdb_stream": ([vp], vp),
        "mdb_synchronize": ([vp], ip),
        "mdb_set_eam": ([vp, C.POINTER(MdbEamTables)], ip),
        "mdb_eam_read_funcfl": ([C.c_char_p, C.POINTER(MdbEamTables)], ip),
        "mdb_eam_free": ([C.POINTER(MdbEamTables)], None),
        "mdb_set_atoms": ([vp, ip, _dp, _dp, _ip], ip),
        "mdb_get_atoms": ([vp, vp, vp, vp, vp], ip),
        "mdb_thermo": ([vp, C.POINTER(MdbThermo)], ip),
        "mdb_run": ([vp, ip, ip, C.POINTER(MdbThermo), ip, C.POINTER(ip)], ip),
        "mdb_get_counts": ([vp, C.POINTER(ip), C.POINTER(ip), C.POINTER(ip)], ip),
        "mdb_get_positions_all": ([vp, _dp], ip),
        "mdb_get_ghosts": ([vp, _ip, _ip], ip),
        "mdb_get_neighbor_list": ([vp, _ip, vp, ip], ip),
        "mdb_get_bin_geometry": ([vp, _ip, _dp, _ip, ip], ip),
        "mdb_get_eam_fp": ([vp, _dp], ip),
        "mdb_launch_count": ([vp], C.c_longlong),
        "mdb_kinetic_sum_noalloc": ([vp, ip, C.c_double, vp, vp], ip),
        "mdb_fp32_fma_rate": ([ip, C.POINTER(C.c_double)], ip),
        "mdb_set_owned": ([vp, ip], ip),
        "mdb_gather_positions": ([vp, vp, ip, C.c_double, C.c_double, C.c_double, vp], ip),
        "mdb_set_halo_positions": ([vp, vp, ip], ip),
    }
    for name in ("mdb_setup_pbc", "mdb_update_pbc", "mdb_update_atoms_pbc",
                 "mdb_build_neighbor", "mdb_compute_force", "mdb_compute_force_energy",
                 "mdb_initial_integrate", "mdb_final_integrate", "mdb_setup",
                 "mdb_sort_atoms"):
        sig[name] = ([vp], ip)
    sig["mdb_set_resort"] = ([vp, ip], ip)
    sig["mdb_tune"] = ([vp, C.c_char_p, ip], ip)
    sig["mdb_set_neighbor_list"] = ([vp, _ip, _ip, ip], ip)
    sig.update({
        "mdb_cp_create": ([C.POINTER(MdbParams), ip, ip, C.POINTER(vp)], ip),
        "mdb_cp_destroy": ([vp], ip),
        "mdb_cp_last_error": ([vp], C.c_char_p),
        "mdb_cp_stream": ([vp], vp),
        "mdb_cp_launch_count": ([vp], C.c_longlong),
        "mdb_cp_set_atoms": ([vp, ip, _dp, _dp, _ip], ip),
        "mdb_cp_get_atoms": ([vp, vp, vp, vp], ip),
        "mdb_cp_thermo": ([vp, C.POINTER(MdbThermo)], ip),
        "mdb_cp_run": ([vp, ip, ip, C.POINTER(MdbThermo), ip, C.POINTER(ip)], ip),
        "mdb_cp_get_counts": ([vp, _ip], ip),
        "mdb_cp_get_slots": ([vp, vp, vp, vp, vp, ip], ip),
        "mdb_cp_get_iclusters": ([vp, vp, vp, vp], ip),
        "mdb_cp_get_jclusters": ([vp, vp, vp, ip], ip),
        "mdb_cp_get_ghosts": ([vp, vp, vp], ip),
        "mdb_cp_get_neighbor_list": ([vp, vp, vp, vp, ip], ip),
        "mdb_cp_get_columns": ([vp, vp, vp, ip], ip),
        "mdb_cp_get_geometry": ([vp, vp, vp, vp, ip], ip),
        "mdb_cp_tune": ([vp, C.c_char_p, ip], ip),
        "mdb_cp_time_force": ([vp, ip, C.POINTER(C.c_double)], ip),
        "mdb_cp_set_rebuild_check": ([vp, C.c_double], ip),
        "mdb_cp_set_pair_buffer": ([vp, C.c_double], ip),
        "mdb_cp_get_pair_stats": ([vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)], ip),
        "mdb_cp_get_rebuilds": ([vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)], ip),
        "mdb_cp_get_check_stats": ([vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)], ip),
        "mdb_cp_ensemble_check_stats": ([vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)],
                                        ip),
        "mdb_cp_ensemble_create": ([C.POINTER(vp), ip, C.POINTER(vp)], ip),
        "mdb_cp_ensemble_destroy": ([vp], ip),
        "mdb_cp_ensemble_last_error": ([vp], C.c_char_p),
        "mdb_cp_ensemble_stream": ([vp], vp),
        "mdb_cp_ensemble_launch_count": ([vp], C.c_longlong),
        "mdb_cp_ensemble_run": ([vp, ip, ip, C.POINTER(MdbThermo), ip, C.POINTER(ip)], ip),
        "mdb_cp_ensemble_tune": ([vp, C.c_char_p, ip], ip),
    })
    for name in ("mdb_cp_synchronize", "mdb_cp_build_clusters", "mdb_cp_define_jclusters",
                 "mdb_cp_setup_pbc",
                 "mdb_cp_update_pbc", "mdb_cp_bin_jclusters", "mdb_cp_build_neighbor",
                 "mdb_cp_prune_neighbor", "mdb_cp_update_single_atoms",
                 "mdb_cp_update_atoms_pbc", "mdb_cp_compute_force",
                 "mdb_cp_compute_force_energy", "mdb_cp_initial_integrate",
                 "mdb_cp_final_integrate", "mdb_cp_setup"):
        sig[name] = ([vp], ip)
    hp = C.POINTER(MdbHostParams)
    pd, pi = C.POINTER(C.POINTER(C.c_double)), C.POINTER(C.POINTER(C.c_int))
    sig.update({
        "mdbh_defaults": ([hp], None),
        "mdbh_read_params": ([hp, C.c_char_p], ip),
        "mdbh_read_types": ([hp, C.c_char_p], ip),
        "mdbh_apply_eam": ([hp, C.POINTER(MdbEamTables)], None),
        "mdbh_finalize": ([hp], None),
        "mdbh_create_fcc": ([hp, pd, pd, pi], ip),
        "mdbh_read_dmp": ([hp, C.c_char_p, pd, pd, pi], ip),
        "mdbh_read_pdb": ([hp, C.c_char_p, pd, pd, pi], ip),
        "mdbh_read_gro": ([hp, C.c_char_p, pd, pd, pi], ip),
        "mdbh_read_in": ([hp, C.c_char_p, pd, pd, pi], ip),
        "mdbh_read_atoms": ([hp, C.c_char_p, pd, pd, pi], ip),
        "mdbh_write_atoms": ([C.c_char_p, ip, _dp, _dp, _ip], ip),
        "mdbh_write_vtk": ([C.c_char_p, ip, ip, _dp], ip),
        "mdbh_stub_atoms": ([ip, ip, C.c_uint, _dp, _dp, _ip], ip),
        "mdbh_stub_neighbors": ([ip, ip, ip, ip, _ip, _ip], ip),
        "mdbh_write_dmp": ([C.c_char_p, ip, _dp, _dp, _ip, C.c_double, C.c_double,
                            C.c_double], ip),
        "mdbh_mdb_params": ([hp, ip, C.POINTER(MdbParams)], None),
    })
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


_libc = C.CDLL(None)
_libc.free.argtypes = [C.c_void_p]


def host_params(**kw):
    """Reference defaults (mdbh_defaults) with overrides, e.g. nx=64, half_neigh=1.

    ``eam`` (tables from :func:`read_funcfl`) applies initEam's overrides;
    ``types`` = (epsilon_per_type, sigma_per_type) sets a types file's content.
    Call :func:`finalize` (done by the builders below) before use."""
    lib = load()
    p = MdbHostParams()
    lib.mdbh_defaults(C.byref(p))
    eam = kw.pop("eam", None)
    types = kw.pop("types", None)
    if isinstance(kw.get("precision"), str):
        kw["precision"] = PRECISIONS[kw["precision"]]
    if eam is not None:
        t, _keep = _eam_struct(eam)
        lib.mdbh_apply_eam(C.byref(p), C.byref(t))
    for k, v in kw.items():
        setattr(p, k, v)
    if types is not None:
        eps, sig = types
        p.ntypes = len(eps)
        p.has_types = 1
        for i, (e, s) in enumerate(zip(eps, sig)):
            p.epsilon_per_type[i] = e
            p.sigma_per_type[i] = s
    return p


def _take(ptr, n, dtype, shape):
    a = np.ctypeslib.as_array(ptr, (n,)).astype(dtype, copy=True).reshape(shape)
    _libc.free(C.cast(ptr, C.c_void_p))
    return a


def create_fcc(hp):
    """createAtom + adjustThermo on the host: (x, v, type) as numpy arrays."""
    lib = load()
    lib.mdbh_finalize(C.byref(hp))
    xp, vp, tp = C.POINTER(C.c_double)(), C.POINTER(C.c_double)(), C.POINTER(C.c_int)()
    n = lib.mdbh_create_fcc(C.byref(hp), C.byref(xp), C.byref(vp), C.byref(tp))
    if n < 0:
        raise MdbError(f"mdbh_create_fcc failed ({-n})")
    return (_take(xp, 3 * n, np.float64, (n, 3)), _take(vp, 3 * n, np.float64, (n, 3)),
            _take(tp, n, np.int32, (n,)))


def read_dmp(hp, path):
    """readAtom_dmp: sets hp's box and from_file; returns (x, v, type)."""
    lib = load()
    xp, vp, tp = C.POINTER(C.c_double)(), C.POINTER(C.c_double)(), C.POINTER(C.c_int)()
    n = lib.mdbh_read_dmp(C.byref(hp), path.encode(), C.byref(xp), C.byref(vp), C.byref(tp))
    if n < 0:
        raise MdbError(f"cannot read dump {path}")
    lib.mdbh_finalize(C.byref(hp))
    return (_take(xp, 3 * n, np.float64, (n, 3)), _take(vp, 3 * n, np.float64, (n, 3)),
            _take(tp, n, np.int32, (n,)))


def read_atoms(hp, path):
    """readAtom: .pdb / .gro / .dmp / .in by extension; sets hp's box, ntypes,
    from_file (and mass for .in); returns (x, v, type)."""
    lib = load()
    xp, vp, tp = C.POINTER(C.c_double)(), C.POINTER(C.c_double)(), C.POINTER(C.c_int)()
    n = lib.mdbh_read_atoms(C.byref(hp), path.encode(), C.byref(xp), C.byref(vp), C.byref(tp))
    if n < 0:
        raise MdbError(f"cannot read atoms from {path}")
    lib.mdbh_finalize(C.byref(hp))
    return (_take(xp, 3 * n, np.float64, (n, 3)), _take(vp, 3 * n, np.float64, (n, 3)),
            _take(tp, n, np.int32, (n,)))


def write_atoms(path, x, v, t):
    """writeAtom (-w): one "type,1.0,x,y,z,vx,vy,vz,0" line per atom."""
    rc = load().mdbh_write_atoms(path.encode(), len(t),
                                 np.ascontiguousarray(x, np.float64).ravel(),
                                 np.ascontiguousarray(v, np.float64).ravel(),
                                 np.ascontiguousarray(t, np.int32))
    if rc:
        raise MdbError(f"cannot write {path}")


def write_vtk(base, timestep, x):
    """write_atoms_to_vtk_file: <base>_<timestep>.vtk."""
    x = np.ascontiguousarray(x, np.float64).ravel()
    rc = load().mdbh_write_vtk(base.encode(), int(timestep), len(x) // 3, x)
    if rc:
        raise MdbError(f"cannot write {base}_{timestep}.vtk")


STUB_PATTERNS = {"seq": 0, "fix": 1, "rand": 2}


def stub_system(natoms, pattern="seq", nneighs=76, nreps=1, ntypes=4, seed=1):
    """The stub gather benchmark's input (verletlist/main-stub.c): atoms on a
    diagonal at rest and a synthetic list. Returns (x, v, type, numneigh,
    neighbors) with neighbors of shape (natoms, nneighs * nreps)."""
    lib = load()
    x = np.zeros((natoms, 3)); v = np.zeros((natoms, 3))
    t = np.zeros(natoms, dtype=np.int32)
    if lib.mdbh_stub_atoms(natoms, ntypes, seed, x.reshape(-1), v.reshape(-1), t):
        raise MdbError("mdbh_stub_atoms: bad arguments")
    nn = np.zeros(natoms, dtype=np.int32)
    nb = np.zeros((natoms, nneighs * nreps), dtype=np.int32)
    if lib.mdbh_stub_neighbors(natoms, STUB_PATTERNS[pattern], nneighs, nreps, nn,
                               nb.reshape(-1)):
        raise MdbError("mdbh_stub_neighbors: bad arguments")
    return x, v, t, nn, nb


def stub_context(x, v, t, numneigh, neighbors, half=0, ntypes=4, device=0):
    """An FP64 LJ :class:`System` holding a stub list. The reference's stub sets
    the cutoff to 1e6 so that every listed pair interacts; here the cutoff is
    just above the diagonal's length (the same pairs interact) and the box its
    length, which keeps the bin grid small."""
    n = len(t)
    box = max(n * 1e-5, 1.0)
    cut = np.sqrt(3.0) * box * 1.001 + 1.0
    s = System(xprd=box, yprd=box, zprd=box, cutforce=cut, cutneigh=cut, dt=0.005,
               dtforce=0.0025, natoms=n, half_neigh=half, bin_rule=BINS_FILE, ntypes=ntypes,
               maxneighs=neighbors.shape[1], device=device)
    s.set_atoms(x, v, t)
    s.set_neighbor_list(numneigh, neighbors)
    return s, box, cut


def write_dmp(path, x, v, t, box):
    lib = load()
    rc = lib.mdbh_write_dmp(path.encode(), len(t), np.ascontiguousarray(x, np.float64).ravel(),
                            np.ascontiguousarray(v, np.float64).ravel(),
                            np.ascontiguousarray(t, np.int32), *box)
    if rc:
        raise MdbError(f"cannot write dump {path}")


def _eam_struct(t):
    keep = [np.ascontiguousarray(t[k], dtype=np.float64)
            for k in ("frho_spline", "rhor_spline", "z2r_spline")]
    ptr = [a.ctypes.data_as(C.POINTER(C.c_double)) for a in keep]
    s = MdbEamTables(nrho=t["nrho"], nr=t["nr"], nrho_tot=t["nrho_tot"], nr_tot=t["nr_tot"],
                     rdr=t["rdr"], rdrho=t["rdrho"], cut=t["cut"], mass=t["mass"],
                     frho_spline=ptr[0], rhor_spline=ptr[1], z2r_spline=ptr[2])
    return s, keep


def system_from_host(hp, natoms, eam=None, device=0, **overrides):
    """A :class:`System` configured exactly as the reference configures itself."""
    lib = load()
    lib.mdbh_finalize(C.byref(hp))
    mp = MdbParams()
    lib.mdbh_mdb_params(C.byref(hp), natoms, C.byref(mp))
    kw = {f: getattr(mp, f) for f, _ in MdbParams._fields_
          if f not in ("epsilon_per_type", "sigma_per_type")}
    kw["pbc"] = (kw.pop("pbc_x"), kw.pop("pbc_y"), kw.pop("pbc_z"))
    kw["device"] = device
    if hp.has_types:
        kw["epsilon_per_type"] = list(hp.epsilon_per_type)[:hp.ntypes]
        kw["sigma_per_type"] = list(hp.sigma_per_type)[:hp.ntypes]
    kw.update(overrides)
    return System(eam=eam, **kw)


def fp32_fma_rate(device=0):
    """The device's packed FP32 FMA rate in flops per second (mdb_fp32_fma_rate)."""
    lib = load()
    r = C.c_double()
    rc = lib.mdb_fp32_fma_rate(int(device), C.byref(r))
    if rc:
        raise MdbError(f"mdb_fp32_fma_rate: {lib.mdb_status_string(rc).decode()}")
    return r.value


def read_funcfl(path):
    """EAM tables from a funcfl file (mdb_eam_read_funcfl) as numpy arrays."""
    lib = load()
    t = MdbEamTables()
    rc = lib.mdb_eam_read_funcfl(path.encode(), C.byref(t))
    if rc:
        raise MdbError(f"cannot read EAM file {path}: {lib.mdb_status_string(rc).decode()}")
    out = dict(nrho=t.nrho, nr=t.nr, nrho_tot=t.nrho_tot, nr_tot=t.nr_tot, rdr=t.rdr,
               rdrho=t.rdrho, cut=t.cut, mass=t.mass,
               frho_spline=np.ctypeslib.as_array(t.frho_spline, (t.nrho_tot,)).copy(),
               rhor_spline=np.ctypeslib.as_array(t.rhor_spline, (t.nr_tot,)).copy(),
               z2r_spline=np.ctypeslib.as_array(t.z2r_spline, (t.nr_tot,)).copy())
    lib.mdb_eam_free(C.byref(t))
    return out


class System:
    """One device-resident MD system (an ``MdbCtx``)."""

    def __init__(self, *, xprd, yprd, zprd, cutforce, cutneigh, dt, dtforce, natoms,
                 mass=1.0, force_field=FF_LJ, half_neigh=0, precision=PREC_FP64,
                 bin_rule=BINS_LATTICE, nx=0, ny=0, nz=0, ntypes=1, epsilon=1.0, sigma=1.0,
                 epsilon_per_type=None, sigma_per_type=None, reneigh_every=20, nstat=100,
                 maxneighs=100, pbc=(1, 1, 1), device=0, eam=None):
        self.lib = load()
        if isinstance(precision, str):
            precision = PRECISIONS[precision]
        p = MdbParams(force_field=force_field, half_neigh=half_neigh, precision=precision,
                      bin_rule=bin_rule, nx=nx, ny=ny, nz=nz, pbc_x=pbc[0], pbc_y=pbc[1],
                      pbc_z=pbc[2], ntypes=ntypes, reneigh_every=reneigh_every, nstat=nstat,
                      maxneighs=maxneighs, natoms=natoms, device=device, xprd=xprd,
                      yprd=yprd, zprd=zprd, dt=dt, dtforce=dtforce, mass=mass,
                      cutforce=cutforce, cutneigh=cutneigh, epsilon=epsilon, sigma=sigma)
        keep = []
        if epsilon_per_type is not None:
            e = np.ascontiguousarray(epsilon_per_type, dtype=np.float64)
            s = np.ascontiguousarray(sigma_per_type, dtype=np.float64)
            keep += [e, s]
            p.epsilon_per_type = e.ctypes.data_as(C.POINTER(C.c_double))
            p.sigma_per_type = s.ctypes.data_as(C.POINTER(C.c_double))
        h = C.c_void_p()
        rc = self.lib.mdb_create(C.byref(p), C.byref(h))
        if rc:
            raise MdbError(f"mdb_create failed: {self.lib.mdb_status_string(rc).decode()}")
        self.h = h
        self.params = p
        self.nlocal = 0
        if eam is not None:
            self.set_eam(eam)

    def close(self):
        if getattr(self, "h", None):
            self.lib.mdb_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _ck(self, rc, what):
        if rc:
            msg = self.lib.mdb_last_error(self.h)
            raise MdbError(f"{what}: {self.lib.mdb_status_string(rc).decode()}"
                           f" ({msg.decode() if msg else ''})")

    # -- data ---------------------------------------------------------------
    def set_eam(self, t):
        self._eam_keep = [np.ascontiguousarray(t[k], dtype=np.float64)
                          for k in ("frho_spline", "rhor_spline", "z2r_spline")]
        ptr = [a.ctypes.data_as(C.POINTER(C.c_double)) for a in self._eam_keep]
        tab = MdbEamTables(nrho=t["nrho"], nr=t["nr"], nrho_tot=t["nrho_tot"],
                           nr_tot=t["nr_tot"], rdr=t["rdr"], rdrho=t["rdrho"], cut=t["cut"],
                           mass=t["mass"], frho_spline=ptr[0], rhor_spline=ptr[1],
                           z2r_spline=ptr[2])
        self._ck(self.lib.mdb_set_eam(self.h, C.byref(tab)), "mdb_set_eam")

    def set_atoms(self, x, v, type_):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
        v = np.ascontiguousarray(v, dtype=np.float64).reshape(-1)
        t = np.ascontiguousarray(type_, dtype=np.int32)
        self._ck(self.lib.mdb_set_atoms(self.h, len(t), x, v, t), "mdb_set_atoms")
        self.nlocal = len(t)

    def atoms(self):
        n = self.nlocal
        x = np.zeros((n, 3)); v = np.zeros((n, 3)); f = np.zeros((n, 3))
        t = np.zeros(n, dtype=np.int32)
        ptr = lambda a: a.ctypes.data_as(C.c_void_p)
        self._ck(self.lib.mdb_get_atoms(self.h, ptr(x), ptr(v), ptr(f), ptr(t)),
                 "mdb_get_atoms")
        return x, v, f, t

    def set_atoms_ptr(self, n, x, v, type_):
        """set_atoms from raw pointers (host or device memory of the context's
        device): n AoS position and velocity triples, n int32 types."""
        if not hasattr(self, "_set_ptr"):
            fn = self.lib._FuncPtr(("mdb_set_atoms", self.lib))
            fn.argtypes, fn.restype = [C.c_void_p, C.c_int] + [C.c_void_p] * 3, C.c_int
            type(self)._set_ptr = fn
        self._ck(self._set_ptr(self.h, int(n), C.c_void_p(x), C.c_void_p(v),
                               C.c_void_p(type_)), "mdb_set_atoms")
        self.nlocal = int(n)

    def atoms_ptr(self, x=None, v=None, f=None, type_=None):
        """mdb_get_atoms into raw pointers (host or device memory; None: skipped)."""
        cv = lambda p: C.c_void_p(p) if p else None
        self._ck(self.lib.mdb_get_atoms(self.h, cv(x), cv(v), cv(f), cv(type_)),
                 "mdb_get_atoms")

    def counts(self):
        nl, ng, mx = C.c_int(), C.c_int(), C.c_int()
        self._ck(self.lib.mdb_get_counts(self.h, C.byref(nl), C.byref(ng), C.byref(mx)),
                 "mdb_get_counts")
        return nl.value, ng.value, mx.value

    def positions_all(self):
        nl, ng, _ = self.counts()
        x = np.zeros((nl + ng) * 3)
        self._ck(self.lib.mdb_get_positions_all(self.h, x), "mdb_get_positions_all")
        return x.reshape(-1, 3)

    def ghosts(self):
        _, ng, _ = self.counts()
        bm = np.zeros(max(ng, 1), dtype=np.int32)
        pb = np.zeros(max(3 * ng, 3), dtype=np.int32)
        self._ck(self.lib.mdb_get_ghosts(self.h, bm, pb), "mdb_get_ghosts")
        return bm[:ng], pb[:3 * ng].reshape(ng, 3)

    def neighbor_list(self):
        nl, _, mx = self.counts()
        nn = np.zeros(nl, dtype=np.int32)
        nb = np.zeros(nl * mx, dtype=np.int32)
        self._ck(self.lib.mdb_get_neighbor_list(self.h, nn, nb.ctypes.data_as(C.c_void_p), mx),
                 "mdb_get_neighbor_list")
        return nn, nb.reshape(nl, mx)

    def numneigh(self):
        nl, _, _ = self.counts()
        nn = np.zeros(nl, dtype=np.int32)
        self._ck(self.lib.mdb_get_neighbor_list(self.h, nn, None, 0), "mdb_get_neighbor_list")
        return nn

    def bin_geometry(self):
        ints = np.zeros(10, dtype=np.int32)
        dbls = np.zeros(7)
        st = np.zeros(4096, dtype=np.int32)
        self._ck(self.lib.mdb_get_bin_geometry(self.h, ints, dbls, st, 4096),
                 "mdb_get_bin_geometry")
        keys_i = ["nbinx", "nbiny", "nbinz", "mbinx", "mbiny", "mbinz", "pad_x", "pad_y",
                  "pad_z", "nstencil"]
        keys_d = ["binsizex", "binsizey", "binsizez", "bininvx", "bininvy", "bininvz",
                  "cutneigh"]
        g = {k: int(v) for k, v in zip(keys_i, ints)}
        g.update({k: float(v) for k, v in zip(keys_d, dbls)})
        g["stencil"] = st[:g["nstencil"]].copy()
        return g

    def eam_fp(self):
        nl, ng, _ = self.counts()
        fp = np.zeros(nl + ng)
        self._ck(self.lib.mdb_get_eam_fp(self.h, fp), "mdb_get_eam_fp")
        return fp

    # -- hooks --------------------------------------------------------------
    def setup(self):
        self._ck(self.lib.mdb_setup(self.h), "mdb_setup")

    def setup_pbc(self):
        self._ck(self.lib.mdb_setup_pbc(self.h), "mdb_setup_pbc")

    def update_pbc(self):
        self._ck(self.lib.mdb_update_pbc(self.h), "mdb_update_pbc")

    def update_atoms_pbc(self):
        self._ck(self.lib.mdb_update_atoms_pbc(self.h), "mdb_update_atoms_pbc")

    def set_neighbor_list(self, numneigh, neighbors):
        """A caller's list of locals (FP64 contexts; the stub benchmark)."""
        nb = np.ascontiguousarray(neighbors, dtype=np.int32)
        self._ck(self.lib.mdb_set_neighbor_list(self.h, np.ascontiguousarray(
            numneigh, dtype=np.int32), nb.reshape(-1), nb.shape[1]), "mdb_set_neighbor_list")

    def sort_atoms(self):
        """sortAtom: locals bin by bin; ghosts and lists must be rebuilt."""
        self._ck(self.lib.mdb_sort_atoms(self.h), "mdb_sort_atoms")

    def set_resort(self, every):
        self._ck(self.lib.mdb_set_resort(self.h, int(every)), "mdb_set_resort")

    def tune(self, key, value):
        """Launch tuning (``eam_rho_lanes``: 1 or 2)."""
        self._ck(self.lib.mdb_tune(self.h, key.encode(), int(value)), "mdb_tune")

    def build_neighbor(self):
        self._ck(self.lib.mdb_build_neighbor(self.h), "mdb_build_neighbor")

    def compute_force(self, energy=False):
        if energy:
            self._ck(self.lib.mdb_compute_force_energy(self.h), "mdb_compute_force_energy")
        else:
            self._ck(self.lib.mdb_compute_force(self.h), "mdb_compute_force")

    def initial_integrate(self):
        self._ck(self.lib.mdb_initial_integrate(self.h), "mdb_initial_integrate")

    def final_integrate(self):
        self._ck(self.lib.mdb_final_integrate(self.h), "mdb_final_integrate")

    def thermo(self):
        t = MdbThermo()
        self._ck(self.lib.mdb_thermo(self.h, C.byref(t)), "mdb_thermo")
        return t.as_dict()

    def step(self, n):
        """One timestep with index n through the individual hooks."""
        reneigh = (n + 1) % self.params.reneigh_every == 0
        self.initial_integrate()
        if reneigh:
            self.update_atoms_pbc()
            self.setup_pbc()
            self.update_pbc()
            self.build_neighbor()
        else:
            self.update_pbc()
        self.compute_force()
        self.final_integrate()

    def run(self, nsteps, first_step=0, max_samples=64):
        """Graph-captured loop; returns the thermo samples."""
        buf = (MdbThermo * max(max_samples, 1))()
        ns = C.c_int()
        self._ck(self.lib.mdb_run(self.h, first_step, nsteps, buf, max_samples, C.byref(ns)),
                 "mdb_run")
        return [buf[k].as_dict() for k in range(ns.value)]

    # -- domain decomposition (halo atoms) ------------------------------------
    def set_owned(self, nown):
        """Atoms [nown, nlocal) of the last set_atoms are halo atoms."""
        self._ck(self.lib.mdb_set_owned(self.h, int(nown)), "mdb_set_owned")

    def gather_positions(self, d_idx, n, shift, d_out):
        """Device AoS positions of atoms d_idx[0..n) plus shift into d_out
        (device pointers as ints), on the context's stream."""
        self._ck(self.lib.mdb_gather_positions(self.h, C.c_void_p(d_idx), int(n),
                                               float(shift[0]), float(shift[1]),
                                               float(shift[2]), C.c_void_p(d_out)),
                 "mdb_gather_positions")

    def set_halo_positions(self, d_x, n):
        """The halo atoms' positions from device AoS triples, on the context's stream."""
        self._ck(self.lib.mdb_set_halo_positions(self.h, C.c_void_p(d_x), int(n)),
                 "mdb_set_halo_positions")

    def synchronize(self):
        self._ck(self.lib.mdb_synchronize(self.h), "mdb_synchronize")

    @property
    def stream(self):
        return self.lib.mdb_stream(self.h)

    @property
    def launches(self):
        return self.lib.mdb_launch_count(self.h)


def _vp(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class ClusterSystem:
    """One device-resident system in the cluster-pair scheme (an ``MdbCp``):
    GROMACS-style 4x4 (``cluster_n=4``) or 4x8 (``cluster_n=8``) clusters."""

    def __init__(self, *, xprd, yprd, zprd, cutforce, cutneigh, dt, dtforce, natoms,
                 cluster_n=4, prune_every=0, mass=1.0, half_neigh=0, precision=PREC_FP64,
                 ntypes=1, epsilon=1.0, sigma=1.0, epsilon_per_type=None, sigma_per_type=None,
                 reneigh_every=20, nstat=100, maxneighs=0, device=0, column_edge=100,
                 **_ignored):
        self.lib = load()
        if isinstance(precision, str):
            precision = PRECISIONS[precision]
        p = MdbParams(force_field=FF_LJ, half_neigh=half_neigh, precision=precision,
                      ntypes=ntypes, reneigh_every=reneigh_every, nstat=nstat,
                      maxneighs=maxneighs, natoms=natoms, device=device, xprd=xprd,
                      yprd=yprd, zprd=zprd, dt=dt, dtforce=dtforce, mass=mass,
                      cutforce=cutforce, cutneigh=cutneigh, epsilon=epsilon, sigma=sigma,
                      pbc_x=1, pbc_y=1, pbc_z=1)
        self._keep = []
        if epsilon_per_type is not None:
            e = np.ascontiguousarray(epsilon_per_type, dtype=np.float64)
            s = np.ascontiguousarray(sigma_per_type, dtype=np.float64)
            self._keep += [e, s]
            p.epsilon_per_type = e.ctypes.data_as(C.POINTER(C.c_double))
            p.sigma_per_type = s.ctypes.data_as(C.POINTER(C.c_double))
        h = C.c_void_p()
        rc = self.lib.mdb_cp_create(C.byref(p), cluster_n, prune_every, C.byref(h))
        if rc:
            raise MdbError(f"mdb_cp_create failed: {self.lib.mdb_status_string(rc).decode()}")
        self.h = h
        self.params = p
        self.M, self.N = 4, cluster_n
        self.nlocal = 0
        self.column_edge = column_edge
        if column_edge != 100:
            # the column grid (bin size) in percent of the reference's
            self._ck(self.lib.mdb_cp_tune(h, b"column_edge", int(column_edge)), "column_edge")

    def close(self):
        if getattr(self, "h", None):
            self.lib.mdb_cp_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _ck(self, rc, what):
        if rc:
            msg = self.lib.mdb_cp_last_error(self.h)
            raise MdbError(f"{what}: {self.lib.mdb_status_string(rc).decode()}"
                           f" ({msg.decode() if msg else ''})")

    def _call(self, name):
        self._ck(getattr(self.lib, name)(self.h), name)

    # -- data ---------------------------------------------------------------
    def set_atoms(self, x, v, type_):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
        v = np.ascontiguousarray(v, dtype=np.float64).reshape(-1)
        t = np.ascontiguousarray(type_, dtype=np.int32)
        self._ck(self.lib.mdb_cp_set_atoms(self.h, len(t), x, v, t), "mdb_cp_set_atoms")
        self.nlocal = len(t)

    def atoms(self, out=None):
        """(x, v, type) as updateSingleAtoms last wrote them; out: arrays of those
        shapes to fill (pinned host memory makes the copy a DMA at full speed)."""
        n = self.nlocal
        if out is None:
            out = (np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n, dtype=np.int32))
        x, v, t = out
        self._ck(self.lib.mdb_cp_get_atoms(self.h, _vp(x), _vp(v), _vp(t)), "mdb_cp_get_atoms")
        return x, v, t

    def counts(self):
        c = np.zeros(8, dtype=np.int32)
        self._ck(self.lib.mdb_cp_get_counts(self.h, c), "mdb_cp_get_counts")
        return dict(zip(["nlocal", "natoms", "ncl", "ncj", "ngc", "nghost", "dummy",
                         "maxneighs"], [int(v) for v in c]))

    def nslots(self):
        c = self.counts()
        return (c["ncj"] + c["ngc"] + 1) * self.N

    def slots(self):
        ns = self.nslots()
        x = np.zeros((ns, 3)); v = np.zeros((ns, 3)); f = np.zeros((ns, 3))
        t = np.zeros(ns, dtype=np.int32)
        self._ck(self.lib.mdb_cp_get_slots(self.h, _vp(x), _vp(v), _vp(f), _vp(t), ns),
                 "mdb_cp_get_slots")
        return x, v, f, t

    def iclusters(self):
        n = self.counts()["ncl"]
        nat = np.zeros(max(n, 1), dtype=np.int32); b = np.zeros(max(n, 1), dtype=np.int32)
        bb = np.zeros(max(6 * n, 6))
        self._ck(self.lib.mdb_cp_get_iclusters(self.h, _vp(nat), _vp(b), _vp(bb)),
                 "mdb_cp_get_iclusters")
        return nat[:n], b[:n], bb[:6 * n].reshape(n, 6)

    def jclusters(self):
        c = self.counts()
        n = c["ncj"] + c["ngc"]
        nat = np.zeros(max(n, 1), dtype=np.int32); bb = np.zeros(max(6 * n, 6))
        self._ck(self.lib.mdb_cp_get_jclusters(self.h, _vp(nat), _vp(bb), n),
                 "mdb_cp_get_jclusters")
        return nat[:n], bb[:6 * n].reshape(n, 6)

    def ghosts(self):
        ng = self.counts()["ngc"]
        bm = np.zeros(max(ng, 1), dtype=np.int32); pb = np.zeros(max(3 * ng, 3), dtype=np.int32)
        self._ck(self.lib.mdb_cp_get_ghosts(self.h, _vp(bm), _vp(pb)), "mdb_cp_get_ghosts")
        return bm[:ng], pb[:3 * ng].reshape(ng, 3)

    def neighbor_list(self):
        c = self.counts()
        n, ld = c["ncl"], c["maxneighs"]
        nn = np.zeros(max(n, 1), dtype=np.int32); nm = np.zeros(max(n, 1), dtype=np.int32)
        nb = np.zeros(max(n * ld, 1), dtype=np.int32)
        self._ck(self.lib.mdb_cp_get_neighbor_list(self.h, _vp(nn), _vp(nm), _vp(nb), ld),
                 "mdb_cp_get_neighbor_list")
        return nn[:n], nm[:n], nb[:n * ld].reshape(n, ld)

    def numneigh(self):
        n = self.counts()["ncl"]
        nn = np.zeros(max(n, 1), dtype=np.int32)
        self._ck(self.lib.mdb_cp_get_neighbor_list(self.h, _vp(nn), None, None, 0),
                 "mdb_cp_get_neighbor_list")
        return nn[:n]

    def columns(self):
        g = self.geometry()
        mb = g["mbinx"] * g["mbiny"]
        start = np.zeros(mb + 1, dtype=np.int32)
        n = self.lib.mdb_cp_get_columns(self.h, _vp(start), None, 0)
        lst = np.zeros(max(n, 1), dtype=np.int32)
        self.lib.mdb_cp_get_columns(self.h, _vp(start), _vp(lst), n)
        return start, lst[:n]

    def geometry(self):
        ints = np.zeros(7, dtype=np.int32); d = np.zeros(3); st = np.zeros(4096, dtype=np.int32)
        self._ck(self.lib.mdb_cp_get_geometry(self.h, _vp(ints), _vp(d), _vp(st), 4096),
                 "mdb_cp_get_geometry")
        keys = ["nbinx", "nbiny", "mbinx", "mbiny", "mbinxlo", "mbinylo", "nstencil"]
        g = dict(zip(keys, [int(i) for i in ints]))
        g.update(binsizex=d[0], binsizey=d[1], rbb_sq=d[2], stencil=st[:g["nstencil"]].copy())
        return g

    # -- hooks --------------------------------------------------------------
    def setup(self):
        self._call("mdb_cp_setup")

    def build_clusters(self):
        self._call("mdb_cp_build_clusters")
        self._call("mdb_cp_define_jclusters")

    def setup_pbc(self):
        self._call("mdb_cp_setup_pbc")

    def update_pbc(self):
        self._call("mdb_cp_update_pbc")

    def bin_jclusters(self):
        self._call("mdb_cp_bin_jclusters")

    def build_neighbor(self):
        self._call("mdb_cp_build_neighbor")

    def prune(self):
        self._call("mdb_cp_prune_neighbor")

    def update_single_atoms(self):
        self._call("mdb_cp_update_single_atoms")

    def update_atoms_pbc(self):
        self._call("mdb_cp_update_atoms_pbc")

    def compute_force(self, energy=False):
        self._call("mdb_cp_compute_force_energy" if energy else "mdb_cp_compute_force")

    def initial_integrate(self):
        self._call("mdb_cp_initial_integrate")

    def final_integrate(self):
        self._call("mdb_cp_final_integrate")

    def step_hooks(self, n, prune_every=1000):
        """One timestep of clusterpair/main.c:326-362 through the single hooks."""
        p = self.params
        self.initial_integrate()
        if (n + 1) % p.reneigh_every:
            if not (n + 1) % prune_every:
                self.prune()
            self.update_pbc()
        else:
            self.update_single_atoms()
            self.update_atoms_pbc()
            self.build_clusters()
            self.setup_pbc()
            self.bin_jclusters()
            self.build_neighbor()
        self.compute_force()
        self.final_integrate()

    def run(self, nsteps, first_step=0, max_samples=64):
        samples = (MdbThermo * max(max_samples, 1))()
        ns = C.c_int()
        self._ck(self.lib.mdb_cp_run(self.h, first_step, nsteps, samples, max_samples,
                                     C.byref(ns)), "mdb_cp_run")
        return [samples[i].as_dict() for i in range(ns.value)]

    def thermo(self):
        t = MdbThermo()
        self._ck(self.lib.mdb_cp_thermo(self.h, C.byref(t)), "mdb_cp_thermo")
        return t.as_dict()

    def synchronize(self):
        self._call("mdb_cp_synchronize")

    def tune(self, key, value):
        self._ck(self.lib.mdb_cp_tune(self.h, key.encode(), int(value)), "mdb_cp_tune")

    def set_rebuild_check(self, max_displacement):
        """Also rebuild whenever an atom moved farther than max_displacement
        since the last build (0: the fixed schedule alone)."""
        self._ck(self.lib.mdb_cp_set_rebuild_check(self.h, float(max_displacement)),
                 "mdb_cp_set_rebuild_check")

    def set_pair_buffer(self, buffer):
        """r_in - r_c of the pair-list path (force_path 1); negative: the skin."""
        self._ck(self.lib.mdb_cp_set_pair_buffer(self.h, float(buffer)),
                 "mdb_cp_set_pair_buffer")

    def pair_stats(self):
        """(derivations run, j atoms listed over all i pairs) of the pair-list path."""
        a, b = C.c_longlong(), C.c_longlong()
        self._ck(self.lib.mdb_cp_get_pair_stats(self.h, C.byref(a), C.byref(b)),
                 "mdb_cp_get_pair_stats")
        return a.value, b.value

    def rebuilds(self):
        """(scheduled, displacement-triggered) rebuilds of checked runs."""
        a, b = C.c_longlong(), C.c_longlong()
        self._ck(self.lib.mdb_cp_get_rebuilds(self.h, C.byref(a), C.byref(b)),
                 "mdb_cp_get_rebuilds")
        return a.value, b.value

    def check_stats(self):
        """(checked steps decided on the device, overflowed rebuilds among them
        replayed by the host)."""
        a, b = C.c_longlong(), C.c_longlong()
        self._ck(self.lib.mdb_cp_get_check_stats(self.h, C.byref(a), C.byref(b)),
                 "mdb_cp_get_check_stats")
        return a.value, b.value

    def time_force(self, reps=20):
        """Seconds per force launch (CUDA events on the context's stream)."""
        t = C.c_double()
        self._ck(self.lib.mdb_cp_time_force(self.h, int(reps), C.byref(t)), "mdb_cp_time_force")
        return t.value

    @property
    def stream(self):
        return int(self.lib.mdb_cp_stream(self.h) or 0)

    @property
    def launches(self):
        return int(self.lib.mdb_cp_launch_count(self.h))


class Ensemble:
    """Independent cluster-pair systems advanced together, one CUDA graph launch
    per timestep for all of them (an ``MdbCpEnsemble``). Members must be set up."""

    def __init__(self, members, batched=None):
        self.lib = load()
        self.members = list(members)
        arr = (C.c_void_p * len(self.members))(*[m.h.value for m in self.members])
        h = C.c_void_p()
        rc = self.lib.mdb_cp_ensemble_create(arr, len(self.members), C.byref(h))
        if rc:
            raise MdbError(f"mdb_cp_ensemble_create failed: "
                           f"{self.lib.mdb_status_string(rc).decode()}")
        self.h = h
        if batched is not None:
            self.tune("batched", int(batched))

    def tune(self, key, value):
        rc = self.lib.mdb_cp_ensemble_tune(self.h, key.encode(), int(value))
        if rc:
            msg = self.lib.mdb_cp_ensemble_last_error(self.h)
            raise MdbError(f"mdb_cp_ensemble_tune: {msg.decode() if msg else rc}")

    def check_stats(self):
        """(checked steps decided on the device, overflowed rebuilds replayed)."""
        a, b = C.c_longlong(), C.c_longlong()
        rc = self.lib.mdb_cp_ensemble_check_stats(self.h, C.byref(a), C.byref(b))
        if rc:
            raise MdbError("mdb_cp_ensemble_check_stats")
        return a.value, b.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.mdb_cp_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def run(self, nsteps, first_step=0, max_samples=16):
        """Returns one list of thermo samples per member."""
        n = len(self.members)
        buf = (MdbThermo * max(n * max_samples, 1))()
        ns = C.c_int()
        rc = self.lib.mdb_cp_ensemble_run(self.h, first_step, nsteps, buf, max_samples,
                                          C.byref(ns))
        if rc:
            msg = self.lib.mdb_cp_ensemble_last_error(self.h)
            raise MdbError(f"mdb_cp_ensemble_run: {self.lib.mdb_status_string(rc).decode()}"
                           f" ({msg.decode() if msg else ''})")
        return [[buf[k * max_samples + j].as_dict() for j in range(ns.value)]
                for k in range(n)]

    @property
    def stream(self):
        return int(self.lib.mdb_cp_ensemble_stream(self.h) or 0)

    @property
    def launches(self):
        return int(self.lib.mdb_cp_ensemble_launch_count(self.h))
