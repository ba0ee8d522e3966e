/*
 * mdb_host.h - host-side setup of an MD-Bench run for libmdb: parameters,
 * the fcc lattice generator, the LAMMPS-style dump reader/writer and the
 * translation into MdbParams. These restate the reference's setup code
 * (common/parameter.c, verletlist/atom.c, common/thermo.c, verletlist/main.c)
 * so a caller that drives the GPU path starts from the reference's exact
 * initial state. Plain C, no CUDA types; exported by libmdb.so.
 */
#ifndef MDB_HOST_H
#define MDB_HOST_H

#include "mdb.h"

#ifdef __cplusplus
extern "C" {
#endif

#define MDBH_MAX_TYPES 8

/* The Parameter fields (common/parameter.h:76-119) this path reads. */
typedef struct {
    int force_field;  /* MDB_FF_LJ / MDB_FF_EAM */
    int half_neigh;
    int precision;    /* MDB_PREC_* (not a reference parameter) */
    int nx, ny, nz;
    int ntypes;
    int ntimes, nstat, reneigh_every;
    int pbc_x, pbc_y, pbc_z;
    int has_types;    /* epsilon_per_type / sigma_per_type valid */
    double epsilon, sigma, rho, temp, mass, dt, cutforce, skin;
    double epsilon_per_type[MDBH_MAX_TYPES];
    double sigma_per_type[MDBH_MAX_TYPES];
    /* box: set by the lattice (nx*lattice) or by an input file */
    double xprd, yprd, zprd;
    int from_file;    /* atoms came from a file: bins of cutneigh/2, no rescale */
    /* derived (mdbh_finalize) */
    double lattice, cutneigh, dtforce;
} MdbHostParams;

/* initParameter defaults, common/parameter.c:73-124 (geometric rule). */
void mdbh_defaults(MdbHostParams* p);
/* readParameter: "key value" lines, '#' comments (common/parameter.c:186-279).
 * Returns MDB_OK or MDB_ERR_ARG (unreadable file, bad types file). */
int mdbh_read_params(MdbHostParams* p, const char* path);
/* readTypesFile: one "epsilon sigma" pair per line (common/parameter.c:126-184). */
int mdbh_read_types(MdbHostParams* p, const char* path);
/* initEam overrides (common/eam_utils.c:22-40): mass, cutoff, T, dt, rho. */
void mdbh_apply_eam(MdbHostParams* p, const MdbEamTables* t);
/* lattice constant, box, cutneigh = cutforce + skin (EAM: + 1.0), dtforce. */
void mdbh_finalize(MdbHostParams* p);

/* createAtom (verletlist/atom.c:104-246) followed by adjustThermo
 * (common/thermo.c:102-159). Allocates *x, *v (3n, AoS) and *type (n) with
 * malloc; returns n or a negative status. Types are drawn from rand() after
 * srand(1), the state a fresh reference process starts in. */
int mdbh_create_fcc(const MdbHostParams* p, double** x, double** v, int** type);

/* readAtom_dmp (verletlist/atom.c:529-656): sets the box in p, from_file = 1.
 * Returns n or a negative status. */
int mdbh_read_dmp(MdbHostParams* p, const char* path, double** x, double** v, int** type);
/* Writes a dump the reader above accepts (ids 1-based, types as given). */
int mdbh_write_dmp(const char* path, int n, const double* x, const double* v, const int* type,
    double xprd, double yprd, double zprd);

/* The other input formats of readAtom (verletlist/atom.c:260-760); each sets
 * the box, ntypes (max type + 1) and from_file like mdbh_read_dmp and returns
 * the atom count, or -MDB_ERR_ARG where the reference would exit. Arrays are
 * malloc'd (free with free()).
 * readAtom_pdb (:296-410): CRYST1 box, ATOM records, zero velocities. */
int mdbh_read_pdb(MdbHostParams* p, const char* path, double** x, double** v, int** type);
/* readAtom_gro (:412-527): title, count, atom lines with velocities, box. */
int mdbh_read_gro(MdbHostParams* p, const char* path, double** x, double** v, int** type);
/* readAtom_in (:658-760): "natoms xlo xhi ylo yhi zlo zhi", then
 * "mass x y z vx vy vz" lines (sets p->mass). */
int mdbh_read_in(MdbHostParams* p, const char* path, double** x, double** v, int** type);
/* readAtom (:260-294): dispatch on .pdb / .gro / .dmp / .in. */
int mdbh_read_atoms(MdbHostParams* p, const char* path, double** x, double** v, int** type);
/* writeAtom (-w, :762-786): "type,1.0,x,y,z,vx,vy,vz,0" per atom. */
int mdbh_write_atoms(const char* path, int n, const double* x, const double* v,
    const int* type);
/* write_atoms_to_vtk_file (verletlist/vtk.c:21-71): "<base>_<timestep>.vtk". */
int mdbh_write_vtk(const char* base, int timestep, int n, const double* x);

/* The stub gather benchmark (verletlist/main-stub.c): synthetic atoms and
 * neighbour patterns that feed the force kernels alone. Atoms: atom i at
 * (i, i, i) * 1e-5, at rest, type rand() % ntypes after srand(seed) (1: a fresh
 * process, as the reference). Patterns (createNeighbors, :60-113), row-major
 * rows of nneighs * nreps entries: SEQ the atoms after i (cyclically; the
 * reference's last atom points one past the end), FIX atoms 0..nneighs-1, RAND
 * distinct random atoms other than i (rand(), continuing the atoms' stream),
 * each row repeated nreps times. */
#define MDBH_STUB_SEQ  0
#define MDBH_STUB_FIX  1
#define MDBH_STUB_RAND 2
int mdbh_stub_atoms(int natoms, int ntypes, unsigned seed, double* x, double* v, int* type);
int mdbh_stub_neighbors(int natoms, int pattern, int nneighs, int nreps, int* numneigh,
    int* neighbors);

/* Fill MdbParams for an n-atom system described by p. */
void mdbh_mdb_params(const MdbHostParams* p, int natoms, MdbParams* out);

#ifdef __cplusplus
}
#endif
#endif /* MDB_HOST_H */
