/*
 * CPU oracle for MD-Bench's cluster-pair (GROMACS-style) scheme: cluster build,
 * j-clusters, cluster ghosts, column binning of j-clusters, the bounding-box
 * cluster-pair list, pruning, the exact reference force kernel, the
 * cluster-layout integrator and the scatter back to atoms.
 *
 * TEST INFRASTRUCTURE ONLY: a plain-C restatement of the reference algorithm
 * (reference files clusterpair/neighbor.c, pbc.c, force_lj.c, integrate.c,
 * cited per function in the .c file), used by tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg as the checker. The product (libmdb) never
 * links or calls it.
 *
 * Parity is pinned by tests against the reference compiled from its own
 * sources into oracle/_ref: the scalar reference-kernel build (M x N = 1 x 2)
 * for clusters, lists, forces and trajectories bit for bit, and the AVX2 (4 x 4)
 * and AVX-512 (4 x 8) builds for clusters, ghosts and lists bit for bit (their
 * SIMD force kernels use approximate reciprocals and are not oracles).
 *
 * Slots: atom cjj of j-cluster cj lives in slot cj*N + cjj (locals, ghost
 * clusters, then one dummy cluster); with M <= N this is also slot ci*M + cii
 * of atom cii of i-cluster ci.
 */
#ifndef MDB_ORACLE_CP_H
#define MDB_ORACLE_CP_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OrcCp OrcCp;

typedef struct {
    int cluster_m, cluster_n; /* 1x2, 4x4 or 4x8 */
    int fma_rsq;              /* list/prune pair test as fma(dx,dx,fma(dy,dy,dz*dz)) (SIMD
                                 builds) instead of dx*dx+dy*dy+dz*dz (scalar build) */
    int half_neigh;
    int ntypes;
    int natoms;               /* Natoms for the bin density and the thermo dof */
    int reneigh_every, prune_every, nstat;
    double xprd, yprd, zprd;
    double dt, dtforce, mass, cutforce, cutneigh;
    double epsilon, sigma;
    const double* epsilon_per_type; /* NULL: all types use epsilon */
    const double* sigma_per_type;   /* NULL: all types use sigma */
} OrcCpParams;

OrcCp* orccp_create(const OrcCpParams* p);
void orccp_destroy(OrcCp* s);

/* Atom arrays (AoS triples), e.g. from the Verlet-list oracle's lattice. */
int orccp_set_atoms(OrcCp* s, int n, const double* x, const double* v, const int* type);

/* setupNeighbor, buildClusters, defineJClusters, setupPbc, binJClusters,
 * buildNeighbor (clusterpair/main.c:44-97). */
int orccp_setup(OrcCp* s);
int orccp_build_clusters(OrcCp* s);
void orccp_define_jclusters(OrcCp* s);
int orccp_setup_pbc(OrcCp* s);
void orccp_update_pbc(OrcCp* s, int first);
void orccp_bin_jclusters(OrcCp* s);
int orccp_build_neighbor(OrcCp* s);
void orccp_prune_neighbor(OrcCp* s);
void orccp_update_single_atoms(OrcCp* s);
void orccp_update_atoms_pbc(OrcCp* s);
double orccp_compute_force(OrcCp* s); /* returns the potential energy */
void orccp_initial_integrate(OrcCp* s);
void orccp_final_integrate(OrcCp* s);
void orccp_step(OrcCp* s, int n);
/* T and P as computeThermo prints them, from the atom arrays. */
void orccp_thermo(OrcCp* s, double* T, double* P);
/* Kinetic and potential energy of the cluster state (not in the reference). */
void orccp_energy(OrcCp* s, double* KE, double* PE);

/* counts: Nlocal Natoms Nclusters_local ncj Nclusters_ghost Nghost dummy_cj
 *         maxneighs (the layout of the reference shim's ref_cp_counts) */
void orccp_counts(OrcCp* s, int* c);
void orccp_get_atoms(OrcCp* s, double* x, double* v, int* type);
void orccp_get_slots(OrcCp* s, double* x, double* v, double* f, int* type, int nslots);
void orccp_set_slots(OrcCp* s, const double* x, const double* v);
void orccp_get_iclusters(OrcCp* s, int* natoms, int* bin, double* bb);
void orccp_get_jclusters(OrcCp* s, int* natoms, double* bb, int count);
void orccp_get_ghosts(OrcCp* s, int* border_map, int* pbc);
void orccp_get_list(OrcCp* s, int* numneigh, int* nmasked, int* neighbors, unsigned* imask,
    int ld);
/* ints: nbinx nbiny mbinx mbiny mbinxlo mbinylo nstencil; dbls: binsizex
 * binsizey rbb_sq */
void orccp_bin_geometry(OrcCp* s, int* ints, double* dbls, int* stencil);
/* j-cluster columns as CSR: start[mbins + 1], list[start[mbins]] */
int orccp_get_columns(OrcCp* s, int* start, int* list, int cap);

#ifdef __cplusplus
}
#endif
#endif
