/*
 * CPU oracle for the MD-Bench short-range timestep (Verlet-list scheme, LJ and EAM).
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain-C restatement of the reference
 * algorithm, used by tests/, by __graft_entry__.smoke() and by bench.py's
 * CPU-baseline leg as the checker. The product (libmdb, the CUDA path) never
 * links, loads or calls it.
 *
 * Parity of this oracle is pinned against (a) the reference's own golden thermo
 * values (tests/sim_copper_fcc_regression.sh:23-26) and (b) the reference itself
 * compiled from its sources into oracle/_ref (oracle/Makefile), whose outputs the
 * tests compare bit-for-bit with this restatement.
 *
 * All floating point in this file is IEEE double, compiled with
 * -ffp-contract=off -fno-fast-math so that every expression rounds exactly as
 * the reference's strict build does.
 */
#ifndef MDB_ORACLE_H
#define MDB_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OrcSys OrcSys;

/* Flat parameter block (mirrors the reference Parameter fields this path uses,
 * common/parameter.h:76-119). */
typedef struct {
    int force_field;     /* 0 = LJ, 1 = EAM */
    int half_neigh;      /* 0 = full list, 1 = half list */
    int nx, ny, nz;      /* unit cells (lattice input) */
    int ntypes;          /* number of LJ types (reference default 4) */
    int from_file;       /* 1: atoms supplied by caller (dmp input) -> cutneigh/2 bins */
    int pbc_x, pbc_y, pbc_z;
    int reneigh_every;
    int nstat;
    double rho, temp, mass, dt, cutforce, skin, epsilon, sigma;
    double xprd, yprd, zprd; /* box lengths for from_file (xlo = 0) */
    const double* epsilon_per_type; /* NULL: all types use epsilon */
    const double* sigma_per_type;   /* NULL: all types use sigma */
} OrcParams;

OrcSys* orc_create(const OrcParams* p);
void orc_destroy(OrcSys* s);

/* EAM funcfl file -> grid arrays -> 7-coefficient splines (common/eam_utils.c). */
int orc_load_eam(OrcSys* s, const char* path);
int orc_eam_info(OrcSys* s, int* nrho, int* nr, int* nrho_tot, int* nr_tot, double* drho,
    double* dr, double* cut, double* mass);
void orc_eam_tables(OrcSys* s, double* frho_spline, double* rhor_spline, double* z2r_spline);

/* fcc lattice + thermo setup + COM removal/rescale (verletlist/main.c:46-113). */
int orc_lattice(OrcSys* s);
/* Atoms from the caller (as read from a .dmp file); no velocity rescale. */
int orc_set_atoms(OrcSys* s, int n, const double* x, const double* v, const int* type);

/* setupNeighbor + setupPbc + updatePbc + buildNeighbor. */
int orc_setup(OrcSys* s);
/* Individual hooks (reference names in the .c file). */
void orc_update_atoms_pbc(OrcSys* s);
int orc_setup_pbc(OrcSys* s);
void orc_update_pbc(OrcSys* s);
int orc_build_neighbor(OrcSys* s);
double orc_compute_force(OrcSys* s); /* returns potential energy (total) */
void orc_initial_integrate(OrcSys* s);
void orc_final_integrate(OrcSys* s);
/* One timestep with index n (0-based), exactly as the main loop runs it. */
void orc_step(OrcSys* s, int n);
/* sortAtom (locals bin by bin; ghosts cleared: call orc_setup_pbc,
 * orc_update_pbc, orc_build_neighbor before the next force) and the SORT_ATOMS
 * resort period used by orc_step (0: never). */
void orc_sort_atoms(OrcSys* s);
void orc_set_resort(OrcSys* s, int every);
/* A caller's list (row-major, ld entries per row) of locals, no ghosts: the
 * stub gather benchmark's input to computeForce. */
void orc_set_list(OrcSys* s, const int* numneigh, const int* neighbors, int ld);

/* Thermo of the current state: T and P as the reference prints them,
 * KE, PE (from the last force call) and E = KE + PE, all totals. */
void orc_thermo(OrcSys* s, double* T, double* P, double* KE, double* PE);

int orc_nlocal(OrcSys* s);
int orc_nghost(OrcSys* s);
int orc_maxneighs(OrcSys* s);
/* x, v, f: 3*n doubles (AoS), locals only unless n_out > nlocal. */
void orc_get_atoms(OrcSys* s, double* x, double* v, double* f, int* type);
void orc_get_positions_all(OrcSys* s, double* x); /* nlocal+nghost */
void orc_set_state(OrcSys* s, const double* x, const double* v);
void orc_get_ghosts(OrcSys* s, int* border_map, int* pbc_xyz);
void orc_get_list(OrcSys* s, int* numneigh, int* neighbors, int ld);
void orc_get_eam_fp(OrcSys* s, double* fp);
/* ints: nbinx nbiny nbinz mbinx mbiny mbinz pad_x pad_y pad_z nstencil
 * doubles: binsizex binsizey binsizez bininvx bininvy bininvz cutneigh */
void orc_bin_geometry(OrcSys* s, int* ints, double* dbls, int* stencil);
void orc_get_params(OrcSys* s, double* dbls); /* xprd yprd zprd dt dtforce mass cutforce cutneigh */

#ifdef __cplusplus
}
#endif
#endif
