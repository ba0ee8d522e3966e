/*
 * mdb.h - C ABI of libmdb, the B200 (sm_100a) implementation of MD-Bench's
 * short-range timestep: binning and Verlet lists, ghost/PBC setup and update,
 * Lennard-Jones (full/half lists, single and multi-type) and three-pass EAM
 * forces, the velocity-Verlet integrator and the thermo reductions.
 *
 * The reference binds its kernels through global function pointers
 * (verletlist/force.h:16-17, neighbor.h:80-81, pbc.h:15-17, integrate.h:12-14)
 * and a CUDA shim (common/device.h:26-50). Each hook below names the reference
 * interface it replaces. All state lives in an opaque context that owns its
 * device memory and one CUDA stream; every call is stream-ordered on that
 * stream and returns an int status (0 = success) instead of exiting the
 * process as the reference's cuda_assert does (common/deviceCuda.cu:14-20).
 * A context is not thread-safe; distinct contexts are independent.
 *
 * Arrays crossing this boundary are plain host pointers in the reference's
 * default layout: positions, velocities and forces as AoS triples
 * (verletlist/atom.h:78-88, ATOM_POSITION_AOS), types as int.
 */
#ifndef MDB_H
#define MDB_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define MDB_OK           0
#define MDB_ERR_ARG      1 /* invalid argument or unsupported configuration */
#define MDB_ERR_CUDA     2 /* a CUDA runtime call failed (context unusable) */
#define MDB_ERR_OVERFLOW 3 /* a device buffer overflowed and could not grow */
#define MDB_ERR_TIMEOUT  4 /* a bounded device wait expired */
#define MDB_ERR_NOMEM    5 /* device or host allocation failed */
#define MDB_ERR_STATE    6 /* call out of order (e.g. force before atoms) */

/* ---- enumerations ---------------------------------------------------------- */
#define MDB_FF_LJ  0 /* enum forcetype FF_LJ, verletlist/force.h:20 */
#define MDB_FF_EAM 1 /* FF_EAM */

#define MDB_PREC_FP64       0 /* FP64 throughout; reproduces the reference bit for bit */
#define MDB_PREC_MIXED      1 /* FP32 pair forces on exact relative coordinates, FP32 sums */
#define MDB_PREC_MIXED_COMP 2 /* as MIXED with compensated (two-float) force sums */

#define MDB_BINS_LATTICE 0 /* nbin = max(1, 5/6 * n cells), verletlist/neighbor.c:67-69 */
#define MDB_BINS_FILE    1 /* bin size = cutneigh/2, verletlist/neighbor.c:123-141 */

/* ---- parameters (the subset of Parameter, common/parameter.h:76-119, that
 *      the timestep reads) -------------------------------------------------- */
typedef struct {
    int force_field;   /* MDB_FF_LJ or MDB_FF_EAM */
    int half_neigh;    /* 0 full list, 1 half list (LJ only) */
    int precision;     /* MDB_PREC_* */
    int bin_rule;      /* MDB_BINS_* */
    int nx, ny, nz;    /* unit cells (MDB_BINS_LATTICE) */
    int pbc_x, pbc_y, pbc_z;
    int ntypes;        /* LJ types; per-type tables below (NULL: epsilon, sigma) */
    int reneigh_every; /* rebuild period in steps (reference default 20) */
    int nstat;         /* thermo sample period in steps (reference default 100) */
    int maxneighs;     /* initial list capacity per atom; 0 -> 100 as the reference */
    int natoms;        /* total atoms for the thermo degrees of freedom */
    int device;        /* CUDA device ordinal */
    double xprd, yprd, zprd; /* box lengths; the box starts at the origin */
    double dt;
    double dtforce;    /* as the reference computes it (0.5*dt, EAM: /mass/mvv2e) */
    double mass;
    double cutforce;
    double cutneigh;   /* cutforce + skin */
    double epsilon, sigma;
    const double* epsilon_per_type; /* ntypes entries or NULL */
    const double* sigma_per_type;   /* ntypes entries or NULL */
} MdbParams;

/* EAM tables: 7-coefficient cubic rows as common/eam_utils.c:224-284 lays them
 * out (coefficients 0..2 derivative, 3..6 value); one element. */
typedef struct {
    int nrho, nr;
    int nrho_tot, nr_tot;
    double rdr, rdrho;
    double cut, mass;
    const double* frho_spline; /* nrho_tot */
    const double* rhor_spline; /* nr_tot */
    const double* z2r_spline;  /* nr_tot */
} MdbEamTables;

/* Thermo sample: T and P exactly as computeThermo prints them
 * (common/thermo.c:60-100; P is the reference's kinetic-only pressure), plus
 * totals of kinetic, potential and total energy (not in the reference). */
typedef struct {
    int step;
    double temperature;
    double pressure;
    double ke;
    double pe;
    double etotal;
} MdbThermo;

typedef struct MdbCtx MdbCtx;

/* ---- context ----------------------------------------------------------------
 * Replaces initDevice (verletlist/device_spec.c:12-48) and the allocateGPU /
 * memcpyToGPU family (common/device.h:26-50). */
int mdb_create(const MdbParams* params, MdbCtx** out);
int mdb_destroy(MdbCtx* ctx);
const char* mdb_status_string(int status);
const char* mdb_last_error(const MdbCtx* ctx);
void* mdb_stream(MdbCtx* ctx); /* the context's cudaStream_t */
int mdb_synchronize(MdbCtx* ctx);

/* EAM tables (from mdb_eam_read_funcfl or any other source). */
int mdb_set_eam(MdbCtx* ctx, const MdbEamTables* tables);

/* Reads a funcfl file and builds the splines as initEam does
 * (common/eam_utils.c:22-284). Arrays are malloc'd; free with
 * mdb_eam_free. */
int mdb_eam_read_funcfl(const char* path, MdbEamTables* out);
void mdb_eam_free(MdbEamTables* t);

/* Local atoms, AoS arrays. Replaces copyDataToCUDADevice /
 * copyDataFromCUDADevice (verletlist/forceCuda.cu:331-343). The arrays may be
 * host or device memory of the context's device (unified addressing), so a
 * caller that keeps its atoms on the GPU moves them without a host copy (the
 * types of device arrays are copied to the host once, to be checked). */
int mdb_set_atoms(MdbCtx* ctx, int nlocal, const double* x, const double* v, const int* type);
int mdb_get_atoms(MdbCtx* ctx, double* x, double* v, double* f, int* type);

/* ---- hooks ------------------------------------------------------------------ */
/* setupPbc (verletlist/pbc.c:103-232): ghost map in the reference order. */
int mdb_setup_pbc(MdbCtx* ctx);
/* updatePbc (verletlist/pbc.c:42-58, pbcCuda.cu:51-74): ghost positions. */
int mdb_update_pbc(MdbCtx* ctx);
/* updateAtomsPbc (verletlist/pbc.c:62-87): wrap local atoms into the box. */
int mdb_update_atoms_pbc(MdbCtx* ctx);
/* buildNeighbor (verletlist/neighbor.c:260-352, neighborCuda.cu:259-364):
 * binning + list, growing the list capacity on overflow. */
int mdb_build_neighbor(MdbCtx* ctx);
/* computeForce (verletlist/force.h:16-17): LJ full/half or EAM per params. */
int mdb_compute_force(MdbCtx* ctx);
/* The same forces plus the potential energy that mdb_thermo then reports (the
 * reference computes no energy; this variant is not part of its hook set). */
int mdb_compute_force_energy(MdbCtx* ctx);
/* initialIntegrate / finalIntegrate (verletlist/integrate.c:21-42). */
int mdb_initial_integrate(MdbCtx* ctx);
int mdb_final_integrate(MdbCtx* ctx);
/* computeThermo (common/thermo.c:60-100) of the current state. */
int mdb_thermo(MdbCtx* ctx, MdbThermo* out);

/* sortAtom (verletlist/neighbor.c:466-536): local atoms reordered bin by bin,
 * each bin's atoms in index order, for locality of the list build and force
 * gathers. Positions, types, velocities and forces move together (the
 * reference moves positions and velocities only). Ghosts and lists are invalid
 * afterwards, as in the reference (which clears Nghost first): run
 * mdb_setup_pbc + mdb_update_pbc + mdb_build_neighbor, or mdb_setup, before
 * the next force. */
int mdb_sort_atoms(MdbCtx* ctx);
/* SORT_ATOMS builds (verletlist/main.c:92-95, 372-381; Parameter.resort_every,
 * reference default 400): mdb_run sorts before the initial integration of
 * every step n with (n+1) % resort_every == 0 and rebuilds in that step.
 * 0 (the default, as SORT_ATOMS ?= false) disables. */
int mdb_set_resort(MdbCtx* ctx, int resort_every);
/* Launch tuning (no counterpart in the reference): "eam_rho_lanes" = 1 or 2
 * lanes per atom in the mixed EAM density pass (2: the lanes take alternate
 * list entries and append the in-cutoff ones in list order; the force pass
 * reads the same rows either way, only the FP64 density sum's order
 * changes; default 1, measured faster at 131k atoms). */
int mdb_tune(MdbCtx* ctx, const char* key, int value);

/* A caller-made neighbour list (row-major, row i = numneigh[i] local atom
 * indices, leading dimension ld) for the force kernels, with no ghosts, as the
 * stub gather benchmark feeds computeForce (verletlist/main-stub.c:60-113,
 * 250-262). Valid until the next list build. FP64 contexts only (the mixed
 * kernels need the cell codes of a built list). */
int mdb_set_neighbor_list(MdbCtx* ctx, const int* numneigh, const int* neighbors, int ld);

/* setup tail of verletlist/main.c:96-111 for atoms already set:
 * setupPbc, updatePbc, buildNeighbor, computeForce. */
int mdb_setup(MdbCtx* ctx);

/* The timestep loop of verletlist/main.c:371-419 for steps
 * first_step .. first_step+nsteps-1, each step captured in CUDA graphs.
 * A thermo sample (with potential energy) is taken after every step n with
 * (n+1) % nstat == 0, as the reference prints them; up to max_samples (at most
 * 64 per call) are returned in samples. */
int mdb_run(MdbCtx* ctx, int first_step, int nsteps, MdbThermo* samples, int max_samples,
    int* nsamples);

/* ---- domain decomposition ----------------------------------------------------
 * The reference's MPI halo (forward(), common/shell_methods.h:28-54, with
 * ghostNeighbor/exchangeComm of common/comm.c:233-631) as building blocks for
 * a caller that splits the box into slabs over GPUs and moves the halo with
 * its own transport (NCCL, gloo, device copies): the context holds the
 * domain's own atoms first and then the halo atoms received from the
 * neighbouring domains, already shifted into this domain's periodic frame.
 * Halo atoms are binned, listed and imaged by the periodic directions like
 * owned atoms but get no force row, no integration and no thermo; the caller
 * refreshes their positions before every force evaluation and runs the
 * per-step hooks (mdb_run refuses a context with halo atoms). LJ only (EAM
 * would need a mid-step F'(rho) exchange, which the reference's EAM does not
 * have either). Full and half lists: the halo covers both z faces, as the
 * reference's fullShell method, whose reverse() moves nothing
 * (common/shell_methods.h:59-88): with half lists a halo atom is listed like
 * a ghost and gets no reaction, so each domain computes the pairs across its
 * faces for its own atoms. */
/* Atoms [nown, nlocal) of the last mdb_set_atoms are halo atoms (nown =
 * nlocal: none); mdb_set_atoms resets it. */
int mdb_set_owned(MdbCtx* ctx, int nown);
/* Device AoS triples d_out[3k..3k+2] = position of atom d_idx[k] + shift,
 * k < n (the positions another domain receives as its halo). Asynchronous on
 * the context's stream. */
int mdb_gather_positions(MdbCtx* ctx, const int* d_idx, int n, double shift_x,
    double shift_y, double shift_z, double* d_out);
/* The halo atoms' positions from device AoS triples (n = nlocal - nown).
 * Asynchronous on the context's stream; follow with mdb_update_pbc. */
int mdb_set_halo_positions(MdbCtx* ctx, const double* d_x, int n);

/* ---- allocation-free entry point -------------------------------------------
 * No counterpart in the reference. For callers that keep their own device
 * arrays and cannot let a library allocate device memory (a framework whose
 * allocator has reserved the device's memory, a timed loop in which
 * cudaMalloc would synchronise the device, a plugin host that forbids it):
 * sum over n atoms of mass * (vx^2 + vy^2 + vz^2), the sum that
 * computeThermo turns into T (common/thermo.c:74-77; T = sum * mvv2e / dof).
 * d_v: n AoS velocity triples in device memory; d_out: one double in device
 * memory; stream: a cudaStream_t (NULL = legacy default stream). Asynchronous.
 * Allocates nothing: partial sums go to a static 32 KiB device array that
 * every call on a device shares (overlapping calls on the GPU race; each call
 * rewrites every slot it reads, so no clearing is needed). At most 8,388,608
 * atoms per call (MDB_ERR_ARG beyond). The first call on a device looks up the
 * array's device address; make that first call before any stream capture. The
 * address is cached per device and CUDA context: the first call under another
 * context of the device (a non-primary driver-API context, or the new primary
 * context after cudaDeviceReset) looks it up again, so make that call before
 * any capture too. */
int mdb_kinetic_sum_noalloc(const double* d_v, int n, double mass, double* d_out, void* stream);

/* ---- device probe -------------------------------------------------------------
 * No counterpart in the reference. The packed FP32 FMA rate of a device, in
 * FP32 flops per second (one fused multiply-add = 2 flops): every thread of a
 * grid filling all SMs runs eight independent chains of fma.rn.f32x2, timed
 * with CUDA events on a stream of its own, best of five launches after a
 * warm-up. The roofline denominator of the mixed cluster-pair force kernels,
 * whose pair arithmetic runs on that pipe. Synchronous; allocates and frees a
 * small output buffer. */
int mdb_fp32_fma_rate(int device, double* flops_per_s);

/* ---- introspection (tests, tools) ----------------------------------------- */
int mdb_get_counts(MdbCtx* ctx, int* nlocal, int* nghost, int* maxneighs);
int mdb_get_positions_all(MdbCtx* ctx, double* x); /* (nlocal+nghost) x 3 */
int mdb_get_ghosts(MdbCtx* ctx, int* border_map, int* pbc_xyz);
/* Row-major copy: neighbors[i*ld + k], k < numneigh[i], in build order. */
int mdb_get_neighbor_list(MdbCtx* ctx, int* numneigh, int* neighbors, int ld);
/* ints: nbinx nbiny nbinz mbinx mbiny mbinz pad_x pad_y pad_z nstencil;
 * dbls: binsizex binsizey binsizez bininvx bininvy bininvz cutneigh. */
int mdb_get_bin_geometry(MdbCtx* ctx, int* ints, double* dbls, int* stencil, int max_stencil);
int mdb_get_eam_fp(MdbCtx* ctx, double* fp); /* nlocal + nghost */
/* Kernel launches issued by this context since creation (instrumentation). */
long long mdb_launch_count(const MdbCtx* ctx);

#ifdef __cplusplus
}
#endif
#endif /* MDB_H */
