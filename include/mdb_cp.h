/*
 * mdb_cp.h - C ABI of libmdb's cluster-pair scheme: MD-Bench's GROMACS-style
 * 4xN cluster-pair path (clusterpair/ in the reference) on B200 (sm_100a).
 *
 * The reference builds this scheme as a separate executable with its own
 * Atom (clusterpair/atom.h:39-90) and binds its kernels through global function
 * pointers: BuildClustersFunction, BuildNeighborFunction, PruneNeighborFunction
 * (clusterpair/neighbor.h:56-61), UpdatePbcFunction (clusterpair/pbc.h),
 * IntegrationFunction (clusterpair/integrate.h:14-16) and
 * ComputeForceFunction (clusterpair/force.h:16-17). Each hook below names the
 * function it replaces. As in mdb.h, all state lives in an opaque context that
 * owns its device memory and one CUDA stream, every call is stream-ordered and
 * returns an int status (MDB_OK = 0), and a context is not thread-safe.
 *
 * Cluster shapes: M x N = 4 x 4 (the reference's AVX2 build) or 4 x 8 (its
 * AVX-512 build). LJ only (the reference's cluster-pair EAM is a stub).
 *
 * Layout of arrays crossing this boundary: atoms as AoS triples in atom order;
 * "slots" in the reference's cluster order, slot cj*N + cjj = atom cjj of
 * j-cluster cj (locals, then ghost clusters, then the dummy cluster), which is
 * slot ci*M + cii of atom cii of i-cluster ci; bounding boxes as
 * (minx maxx miny maxy minz maxz).
 */
#ifndef MDB_CP_H
#define MDB_CP_H

#include "mdb.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct MdbCp MdbCp;

/* Context for the parameters of mdb.h (force_field must be MDB_FF_LJ;
 * precision MDB_PREC_FP64 or MDB_PREC_MIXED; maxneighs 0 -> 200 as
 * initNeighbor, clusterpair/neighbor.c:73-77) and cluster width
 * cluster_n = 4 or 8; prune_every <= 0 keeps the reference's 1000. The column
 * grid of setupNeighbor (clusterpair/neighbor.c:108-215) is fixed here from
 * params->natoms and the box. Replaces initDevice + initNeighbor. */
int mdb_cp_create(const MdbParams* params, int cluster_n, int prune_every, MdbCp** out);
int mdb_cp_destroy(MdbCp* ctx);
const char* mdb_cp_last_error(const MdbCp* ctx);
void* mdb_cp_stream(MdbCp* ctx);
int mdb_cp_synchronize(MdbCp* ctx);
/* Launch tuning (no counterpart in the reference; results are unchanged
 * except where noted):
 * "force_cpw" = i-clusters per warp of the mixed cluster-pair kernel: 1, 2, 4,
 * or 8 with 4x4 clusters (default 4). Each i-cluster gets 32 / force_cpw
 * lanes; the rows of a warp's clusters run side by side. The same pairs are
 * evaluated, but a row's split among the lanes, and so the FP32 rounding of
 * the i sums, depends on the setting. Ensemble members keep theirs;
 * "force_jpl" = j atoms per lane of the mixed cluster-pair kernel: 1, or 2
 * with force_cpw 4 (two consecutive atoms of an entry share a lane's list,
 * anchor and loop work; FP32 rounding changes as for force_cpw; default 2
 * for one atom type, 1 for several types and for 4x8 half lists; ensemble
 * members keep theirs);
 * "force_block" = threads per block of the mixed force kernel (32..512, a
 * multiple of 32; default 128); "force_variant" = 0..3: 0 and 1 prefetch the
 * j data one or two list blocks ahead with no register budget, 2 and 3 the same
 * with a budget for 8 resident blocks of 128 threads per SM (these run blocks
 * of 128 threads; default 2; with force_cpw > 1 the prefetch is one block,
 * 1 runs as 0 and 3 asks a budget for 6 blocks instead of 8);
 * "force_swizzle" = 1: the blocks one resident
 * slot runs in turn take neighbouring i-clusters (L1 reuse of j data; default
 * 0, measured within 2 % either way); "force_path" (mixed contexts) = 0: the
 * cluster-pair kernel evaluates every pair slot of the listed cluster pairs,
 * as the reference's computeForceLJ kernels do (clusterpair/force_lj.c);
 * 1: the pair-list kernel evaluates only the listed cluster pairs' pairs
 * within r_c + buffer of each other when last derived (see
 * mdb_cp_set_pair_buffer), re-derived inside the timestep whenever an atom
 * has moved more than buffer / 2 since: the same pairs inside r_c, so the
 * same forces up to FP32 summation order; "pair_variant" = 0..3: launch
 * shape of the pair-list kernel (j loads in flight per lane and register
 * budget: 0 = 4 loads, 1 = 2, 2 = 3 with a budget for 6 blocks of 128
 * threads per SM, 3 = 2 with a budget for 8; default 0);
 * "column_edge" = 50..200: the xy edge of the column grid in percent of
 * setupNeighbor's (max(M, N) / rho)^(1/3) (clusterpair/neighbor.c:128-145),
 * the scheme's bin size; accepted only before mdb_cp_set_atoms. 100 (the
 * default) is the reference's grid and lists; any other value gives other
 * clusters and lists with the same pairs inside cutneigh, so the same forces
 * up to summation order. */
int mdb_cp_tune(MdbCp* ctx, const char* key, int value);
/* Buffer of the pair-list path (force_path 1; no counterpart in the
 * reference): pairs are kept within r_c + buffer, and any atom moving more
 * than buffer / 2 since the last derivation triggers a new one in the next
 * force evaluation. Negative (the default): the list skin, cutneigh -
 * cutforce. */
int mdb_cp_set_pair_buffer(MdbCp* ctx, double buffer);
/* Pair-list path statistics: derivations run so far, and the j atoms listed
 * by the last derivation over all i pairs (each stands for two pair slots). */
int mdb_cp_get_pair_stats(MdbCp* ctx, long long* derivations, long long* codes);
/* Device time of one force evaluation (no energy) on the context's stream:
 * the mean over reps back-to-back launches after two untimed ones, from CUDA
 * events. For launch tuning; the force array is overwritten with the same
 * values. */
int mdb_cp_time_force(MdbCp* ctx, int reps, double* seconds);
long long mdb_cp_launch_count(const MdbCp* ctx);

/* Atom arrays (createAtom / readAtom output, or any state). */
int mdb_cp_set_atoms(MdbCp* ctx, int nlocal, const double* x, const double* v, const int* type);
/* Atom arrays as updateSingleAtoms last wrote them (cluster order after a rebuild). */
int mdb_cp_get_atoms(MdbCp* ctx, double* x, double* v, int* type);

/* ---- hooks ---------------------------------------------------------------- */
/* buildClusters (clusterpair/neighbor.c:1513-1611): binAtoms, sortAtomsByZCoord,
 * clusters and boxes; the GPU builds the j-cluster boxes in the same pass. */
int mdb_cp_build_clusters(MdbCp* ctx);
/* defineJClusters (clusterpair/neighbor.c:1807-1915): done by
 * mdb_cp_build_clusters; kept so callers can keep the reference's sequence. */
int mdb_cp_define_jclusters(MdbCp* ctx);
/* setupPbc + updatePbc(first) (clusterpair/pbc.c:184-331). */
int mdb_cp_setup_pbc(MdbCp* ctx);
/* updatePbc (clusterpair/pbc.c:43-113): ghost positions from their owners. */
int mdb_cp_update_pbc(MdbCp* ctx);
/* binJClusters (clusterpair/neighbor.c:1917-2094). */
int mdb_cp_bin_jclusters(MdbCp* ctx);
/* buildNeighbor (clusterpair/neighbor.c:282-529), growing maxneighs by 1.2x
 * the longest row when a row reaches it, as the reference does. */
int mdb_cp_build_neighbor(MdbCp* ctx);
/* pruneNeighbor (clusterpair/neighbor.c:1098-1264). */
int mdb_cp_prune_neighbor(MdbCp* ctx);
/* updateSingleAtoms (clusterpair/neighbor.c:2096-2149). */
int mdb_cp_update_single_atoms(MdbCp* ctx);
/* updateAtomsPbc (clusterpair/pbc.c:116-143). */
int mdb_cp_update_atoms_pbc(MdbCp* ctx);
/* computeForce: computeForceLJRef semantics (clusterpair/force_lj.c:23-189) in
 * FP64, or FP32 pair forces on cluster-relative coordinates (MIXED). */
int mdb_cp_compute_force(MdbCp* ctx);
/* The same plus the potential energy (not computed by the reference). */
int mdb_cp_compute_force_energy(MdbCp* ctx);
/* initialIntegrate / finalIntegrate (clusterpair/integrate.c:29-86). */
int mdb_cp_initial_integrate(MdbCp* ctx);
int mdb_cp_final_integrate(MdbCp* ctx);
/* computeThermo (common/thermo.c:60-100): T and P from the atom arrays, as
 * the reference prints them (velocities as of the last updateSingleAtoms); ke,
 * pe and etotal from the cluster state. pe: of the last energy evaluation; when
 * the last force evaluation (mdb_cp_setup, mdb_cp_compute_force, the last step
 * of mdb_cp_run) had none and the slots have not moved since, one force
 * evaluation with the energy runs first (the same forces; half lists sum them
 * in another atomic order); otherwise NaN. */
int mdb_cp_thermo(MdbCp* ctx, MdbThermo* out);

/* setup() of clusterpair/main.c:44-97 for atoms already set: buildClusters,
 * defineJClusters, setupPbc, binJClusters, buildNeighbor, then computeForce
 * (no energy: mdb_cp_thermo evaluates it when asked). */
int mdb_cp_setup(MdbCp* ctx);
/* The timestep loop of clusterpair/main.c:326-362 for steps first_step ..
 * first_step+nsteps-1 (prune every prune_every steps, rebuild every
 * reneigh_every), plain steps as CUDA graphs. Thermo samples after every step
 * n with (n+1) % nstat == 0, up to max_samples (at most 64 per call). */
int mdb_cp_run(MdbCp* ctx, int first_step, int nsteps, MdbThermo* samples, int max_samples,
    int* nsamples);

/* Displacement-checked rebuilds (no counterpart in the reference, which only
 * rebuilds every reneigh_every steps). With max_displacement > 0, mdb_cp_run
 * also rebuilds in any step in which some atom has moved farther than
 * max_displacement since the last build (skin / 2 keeps every list complete
 * whatever the motion); the integrator tests the displacement and raises a
 * device flag. The decision is taken on the device: each such step is one
 * CUDA graph whose conditional nodes run updateAtoms and the whole rebuild
 * when the flag is up, else updatePbc, then the force, with no host
 * synchronisation. A rebuild there that overflows a buffer stops the call's
 * later steps on the device; the host then grows the buffer, replays that
 * build and resumes from the next step, so the result is that of growing
 * the buffer at once. Scheduled rebuilds, pruning, thermo samples, a call's
 * first and last step, the pair-list path and the tuning key
 * "check_on_host" = 1 read the flag on the host after the integration
 * instead (the same decisions, so the same trajectory). 0 (the default)
 * restores the fixed schedule alone. After a change the next step rebuilds
 * first. */
int mdb_cp_set_rebuild_check(MdbCp* ctx, double max_displacement);
/* Rebuilds performed by mdb_cp_run with the check on: on the fixed schedule,
 * and triggered by the displacement test. */
int mdb_cp_get_rebuilds(MdbCp* ctx, long long* scheduled, long long* checked);
/* Checked steps decided on the device so far, and rebuilds among them that
 * overflowed a buffer and were replayed by the host (no counterpart in the
 * reference). */
int mdb_cp_get_check_stats(MdbCp* ctx, long long* graph_steps, long long* replays);

/* ---- ensembles ----------------------------------------------------------------
 * No counterpart in the reference (which runs one system per process). Many
 * independent systems, each an MdbCp already set up with mdb_cp_setup, of any
 * sizes and temperatures but the same reneigh_every, nstat and prune_every,
 * advance together: every timestep of all members is one CUDA graph launch
 * whose branches are the members' own kernel sequences, so small replicas run
 * concurrently and fill the GPU. Rebuild steps synchronise once for all
 * members. Thermo samples after every step n with (n+1) % nstat == 0, up to
 * max_samples per member: samples[member * max_samples + k]. The members stay
 * usable on their own between runs; do not use them while a run is active.
 * Members must run the cluster-pair force kernel (force_path 0): MDB_ERR_ARG
 * otherwise. */
typedef struct MdbCpEnsemble MdbCpEnsemble;
int mdb_cp_ensemble_create(MdbCp* const* members, int n, MdbCpEnsemble** out);
int mdb_cp_ensemble_destroy(MdbCpEnsemble* ens);
const char* mdb_cp_ensemble_last_error(const MdbCpEnsemble* ens);
void* mdb_cp_ensemble_stream(MdbCpEnsemble* ens);
long long mdb_cp_ensemble_launch_count(const MdbCpEnsemble* ens);
/* "batched" = 1 (the default when every member is MDB_PREC_MIXED): the
 * integrator, the ghost update and the force kernel each run as one launch
 * over all members (members grouped by cluster shape, list form, types and
 * launch settings); 0: every member runs its own kernel sequence on its own
 * graph branch. Results are the same either way.
 * "check_on_host" = 1: members with the displacement check
 * (mdb_cp_set_rebuild_check; batched ensembles only) have the host read their
 * flags after every integration; 0 (the default): each checked step is one
 * CUDA graph launch whose conditional nodes rebuild the members whose flag is
 * up (the others update their ghosts, so each member follows its own checked
 * run alone), with no host synchronisation, and a rebuild there that
 * overflows a member's buffer is replayed by the host at its next
 * synchronisation, as for a single system. The same decisions either way. */
int mdb_cp_ensemble_tune(MdbCpEnsemble* ens, const char* key, int value);
int mdb_cp_ensemble_run(MdbCpEnsemble* ens, int first_step, int nsteps, MdbThermo* samples,
    int max_samples, int* nsamples);
/* Checked steps decided on the device so far, and overflowed rebuilds among
 * them replayed by the host (no counterpart in the reference). */
int mdb_cp_ensemble_check_stats(MdbCpEnsemble* ens, long long* graph_steps, long long* replays);

/* ---- introspection (tests, tools) ----------------------------------------- */
/* counts: Nlocal Natoms Nclusters_local ncj Nclusters_ghost Nghost dummy_cj
 * maxneighs */
int mdb_cp_get_counts(MdbCp* ctx, int* counts);
/* nslots slots of x, type; v and f for the local slots (others untouched). */
int mdb_cp_get_slots(MdbCp* ctx, double* x, double* v, double* f, int* type, int nslots);
int mdb_cp_get_iclusters(MdbCp* ctx, int* natoms, int* bin, double* bb);
int mdb_cp_get_jclusters(MdbCp* ctx, int* natoms, double* bb, int count);
int mdb_cp_get_ghosts(MdbCp* ctx, int* border_map, int* pbc_xyz);
/* Row-major copy: neighbors[ci*ld + k], k < numneigh[ci], in list order. */
int mdb_cp_get_neighbor_list(MdbCp* ctx, int* numneigh, int* nmasked, int* neighbors, int ld);
/* j-cluster columns: start[mbins + 1], list[start[mbins]]; returns the count. */
int mdb_cp_get_columns(MdbCp* ctx, int* start, int* list, int cap);
/* ints: nbinx nbiny mbinx mbiny mbinxlo mbinylo nstencil; dbls: binsizex
 * binsizey rbb_sq; stencil: nstencil flat offsets */
int mdb_cp_get_geometry(MdbCp* ctx, int* ints, double* dbls, int* stencil, int max_stencil);

#ifdef __cplusplus
}
#endif
#endif /* MDB_CP_H */
