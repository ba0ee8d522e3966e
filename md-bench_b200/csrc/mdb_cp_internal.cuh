// Cluster-pair (GROMACS-style) scheme: device layout and launch helpers shared
// by mdb_cp_build.cu, mdb_cp_force.cu and mdb_cp_api.cu.
//
// Device data layout (HBM), per context, for cluster shape M x N (4x4 or 4x8):
//   atom arrays (atom order, what updateSingleAtoms writes):
//     ax double4[nlocal] (.w = type bits), av double4[nlocal]
//   slots (cluster order): slot cj*N + cjj = atom cjj of j-cluster cj; locals
//   first (slot ci*M + cii = atom cii of i-cluster ci), then ghost j-clusters,
//   then one dummy cluster:
//     cx  double4[slot_cap]  FP64 positions, .w = type bits, -1 for padding
//                            (padding positions are +INF as in the reference)
//     cv  double4 (locals), cf double4 (FP64 forces, locals + ghosts)
//     xr  float4             mixed path: position relative to the anchor of the
//                            slot's j-cluster, .w = type bits (-1 for padding,
//                            whose position holds a large finite sentinel)
//     cf32 float4            mixed path forces
//   per i-cluster: inat, cbin, cl_first (atom index of its first atom in the
//     next updateSingleAtoms), ibbmin/ibbmax double4 (bbox)
//   per j-cluster (locals + ghosts): jnat, jbbmin/jbbmax double4, anchor float4
//     (mixed: a multiple of 1/8 near the box centre, so anchor differences are
//     exact in FP32)
//   ghosts: border (owner j-cluster), pbc code ((dx+1) | (dy+1)<<2 | (dz+1)<<4)
//   columns: j-clusters per xy column as CSR (jcol_start, jcol), sorted by
//     bbminz as binJClusters leaves them, with their boxes copied in column
//     order (jcbbmin/jcbbmax) for the list build's window search
//   list: entry k of i-cluster ci at list[k * ks + ci * cs]: k-major (ks =
//     capacity of i-clusters, cs = 1) for the FP64 kernel's thread-per-atom
//     reads, row-major (ks = 1, cs = maxneighs) for the mixed kernel's
//     warp-per-cluster reads; numneigh[ci]; the diagonal (masked) entry first
//     as the reference puts it
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "mdb_internal.cuh"

#define CP_M            4    /* i-cluster size of the GPU shapes */
#define CP_COL_SMEM     1024 /* column sort in shared memory up to this many atoms */
#define CP_PAD_F        1.0e18f
#define CP_ANCHOR_STEP  0.125

// device counters of the cluster-pair scheme (int slots)
enum {
    CP_NCL          = 0,  // local i-clusters
    CP_NCJ          = 1,  // local j-clusters
    CP_NGC          = 2,  // ghost j-clusters in use (clamped to capacity)
    CP_NGC_TOTAL    = 3,  // ghost j-clusters requested by setupPbc
    CP_NGHOST_ATOMS = 4,
    CP_MAXNEED      = 5,  // largest list length seen (>= maxneighs means regrow)
    CP_BADBIN       = 6,  // atoms outside the column grid
    CP_SLOTS        = 7
};

namespace mdb {
namespace cp {

struct Geom {
    int nbinx, nbiny, mbinx, mbiny, mbinxlo, mbinylo, mbins, nstencil;
    double binsizex, binsizey, bininvx, bininvy;
    double xprd, yprd, zprd;
    double cutneigh, cutneighsq, rbb_sq;
    // bound on |FP32 - FP64| of a squared distance or box distance computed
    // from coordinates rounded to FP32 (the list build's prefilter)
    float list_margin;
    // z buckets of the list build's window table: bucket of z =
    // clamp(floor((z - z0) * zinv), 0, zq); per column zq + 2 entries
    int zq;
    double z0, zinv;
};

// the window table's bucket of a z coordinate (monotone in z; NaN -> 0)
__host__ __device__ __forceinline__ int zbucket(const Geom& g, double z)
{
    double q = floor((z - g.z0) * g.zinv);
    q        = fmin(fmax(q, 0.0), (double)g.zq);
    return (int)q;
}

struct Types {
    int ntypes, uniform;
    double sqrt_eps[MDB_MAX_TYPES], sigma3[MDB_MAX_TYPES];
    float sqrt_eps_f[MDB_MAX_TYPES], sigma3_f[MDB_MAX_TYPES];
    double eps0, sigma6_0; // uniform case
    int force_block;       // threads per block of the mixed force kernel (tunable)
    int force_variant;     // mixed force kernel: bit 0 prefetch 2 ahead, bit 1 register budget
    int force_swizzle;     // mixed force kernel: blocks walk contiguous cluster ranges (0/1)
    int force_cpw;         // mixed force kernel: i-clusters per warp (1, 2, 4, 8)
    int force_jpl;         // mixed force kernel: j atoms per lane (1, or 2 with force_cpw 4)
    int pair_variant;      // pair-list force kernel: launch shape (0..3)
};

__device__ __forceinline__ int slot_type(const double4& p) { return (int)__double_as_longlong(p.w); }

__device__ __forceinline__ double type_bits(int t) { return __longlong_as_double((long long)t); }

// mixed-path position of one slot, relative to the anchor a of its j-cluster;
// b = the slot's index in its j-cluster. mode 1: .w holds the type bits;
// mode 2 (one atom type, no type needed): slots 0, 1, 2 of a j-cluster carry
// the anchor's x, y, z in .w instead, so the force kernel reads a j atom and
// its cluster's anchor in one load (padding is told by its position).
__device__ __forceinline__ void put_rel(float4* xr, int slot, const double4& p, const float4& a,
    int mode, int b)
{
    const int t = slot_type(p);
    float w     = __int_as_float(t < 0 ? -1 : t);
    if (mode == 2 && b < 3) w = b == 0 ? a.x : (b == 1 ? a.y : a.z);
    if (t < 0) {
        xr[slot] = make_float4(CP_PAD_F, CP_PAD_F, CP_PAD_F, w);
    } else {
        xr[slot] = make_float4((float)(p.x - (double)a.x), (float)(p.y - (double)a.y),
            (float)(p.z - (double)a.z), w);
    }
}

// coord2bin / coord2bin2D, clusterpair/neighbor.c:1366-1407
__device__ __forceinline__ void coord2bin2d(const Geom& g, double x, double y, int& ix, int& iy)
{
    if (x >= g.xprd) ix = (int)((x - g.xprd) * g.bininvx) + g.nbinx - g.mbinxlo;
    else if (x >= 0.0) ix = (int)(x * g.bininvx) - g.mbinxlo;
    else ix = (int)(x * g.bininvx) - g.mbinxlo - 1;
    if (y >= g.yprd) iy = (int)((y - g.yprd) * g.bininvy) + g.nbiny - g.mbinylo;
    else if (y >= 0.0) iy = (int)(y * g.bininvy) - g.mbinylo;
    else iy = (int)(y * g.bininvy) - g.mbinylo - 1;
}

// ---- launch helpers ---------------------------------------------------------
// build (mdb_cp_build.cu)
void launch_gather(cudaStream_t s, int M, int ncl_cap, const int* cnt, const double4* cx,
    const double4* cv, const int* cl_first, double4* ax, double4* av, int wrap, double xprd,
    double yprd, double zprd);
void launch_bin_atoms(cudaStream_t s, int n, const double4* ax, const Geom& g, int* atom_col,
    int* col_count, int* cnt);
void launch_scatter_atoms(cudaStream_t s, int n, const int* atom_col, const int* col_start,
    int* col_fill, int* col_atoms);
void launch_sort_columns(cudaStream_t s, const Geom& g, int M, int N, const int* col_start,
    int* col_atoms, const double4* ax, int* col_sorted, int* gidx, double* gz, int* ncl_col);
void launch_build_clusters(cudaStream_t s, const Geom& g, int M, int N, int mixed,
    const int* col_start, const int* col_sorted, const int* cl_start, const double4* ax,
    const double4* av, double4* cx, double4* cv, int* inat, int* cbin, int* cl_first,
    double4* ibbmin, double4* ibbmax, int* jnat, double4* jbbmin, double4* jbbmax,
    float4* anchor, float4* xr, int* cnt, unsigned long long* zext);
void launch_ghost_count(cudaStream_t s, int ncj_cap, const int* cnt, const int* jnat,
    const double4* jbbmin, const double4* jbbmax, const Geom& g, int* gcount);
void launch_ghost_write(cudaStream_t s, int ncj_cap, int ngc_cap, int* cnt, const int* jnat,
    const double4* jbbmin, const double4* jbbmax, const Geom& g, const int* gstart,
    int* border, int* pbc);
void launch_ghost_first(cudaStream_t s, int N, int ngc_cap, int mixed, int* cnt,
    const int* border, const int* pbc, const Geom& g, double4* cx, int* jnat, double4* jbbmin,
    double4* jbbmax, float4* anchor, float4* xr, unsigned long long* zext);
void launch_ghost_update(cudaStream_t s, int N, int ngc_cap, int mixed, const int* cnt,
    const int* border, const int* pbc, const int* jnat, const Geom& g, double4* cx,
    const float4* anchor, float4* xr);
void launch_ghost_columns(cudaStream_t s, int N, int ngc_cap, const int* cnt, const int* pbc,
    const int* jnat, const double4* cx, const Geom& g, int* gcolumn, int* gcol_count);
void launch_column_sizes(cudaStream_t s, int mbins1, int jfac, const int* ncl_col,
    const int* gcol_count, int* jcol_n);
void launch_ghost_scatter(cudaStream_t s, int ngc_cap, const int* cnt, const int* gcolumn,
    const int* jcol_start, const int* ncl_col, int jfac, int* gfill, int* gtmp);
void launch_merge_columns(cudaStream_t s, int mbins1, int jfac, const int* ncl_col,
    const int* cl_start, const int* gcol_count, const int* jcol_start, const int* gtmp,
    const double4* jbbmin, const double4* jbbmax, int* jcol, double4* jcbbmin, double4* jcbbmax);
// FP32 copies for the list build's prefilter: the column-ordered j boxes
// (jcbbf[2m] min, [2m+1] max) and the slot positions (all j-clusters)
void launch_list_prep(cudaStream_t s, int N, int slot_cap, const Geom& g, const int* cnt,
    const int* jcol_start, const double4* jcbbmin, const double4* jcbbmax, const double4* cx,
    float4* jcbbf, float4* cxf, int* ztab);
void launch_build_list(cudaStream_t s, int M, int N, int half, int ncl_cap, const int* cnt,
    const Geom& g, const int* stencil, const int* cbin, const double4* ibbmin,
    const double4* ibbmax, const double4* jcbbmin, const double4* jcbbmax, const double4* cx,
    const float4* jcbbf, const float4* cxf, const int* jcol, const int* ztab,
    const unsigned long long* zext, int maxneighs, int ks, int cs, int* list, int* numneigh,
    int* nmasked, int* cnt_out);
void launch_prune(cudaStream_t s, int M, int N, int ncl_cap, const int* cnt, const double4* cx,
    double cutneighsq, int maxneighs, int ks, int cs, int* list, int* numneigh, int* nmasked);

// force / integrate / thermo (mdb_cp_force.cu)
int force_blocks(int ncl_cap);
void launch_force_fp64(cudaStream_t s, int M, int N, int half, int energy, int ncl_cap,
    const int* cnt, const double4* cx, const Types& ty, double cutforcesq, const int* list,
    int ks, int cs, const int* numneigh, double4* cf, double* epart);
// returns the number of blocks launched (= energy partials written)
int launch_force_mixed(cudaStream_t s, int N, int half, int energy, int ncl_cap,
    const int* cnt, const float4* xr, const float4* anchor, const Types& ty, float cutforcesq,
    const int* list, int ks, int cs, const int* numneigh, float4* cf32, double* epart);
// threads per block and block count of a mixed force launch
int force_mixed_threads(const Types& ty);
int force_mixed_grid(int ncl_cap, const Types& ty);
// xmode: the put_rel mode of xr (ignored when xr is null)
// xb (null: no check): slot positions at the last build; a slot farther than
// sqrt(lim2) from it sets *flag (the displacement check of a rebuild policy)
// xq (null: no check): the mixed positions the pair codes were derived from;
// a slot farther than sqrt(qlim2) from it sets *qflag (the pair-list path)
void launch_cp_initial(cudaStream_t s, int M, int N, int ncl_cap, const int* cnt, double dtf,
    double dt, double4* cx, double4* cv, const double4* cf, const float4* cf32,
    const float4* anchor, float4* xr, int xmode, const double4* xb, double lim2, int* flag,
    const float4* xq = nullptr, float qlim2 = 0.f, int* qflag = nullptr);
void launch_cp_final(cudaStream_t s, int M, int ncl_cap, const int* cnt, double dtf,
    const double4* cx, double4* cv, const double4* cf, const float4* cf32);
void launch_cp_final_initial(cudaStream_t s, int M, int N, int ncl_cap, const int* cnt,
    double dtf, double dt, double4* cx, double4* cv, const double4* cf, const float4* cf32,
    const float4* anchor, float4* xr, int xmode, const double4* xb, double lim2, int* flag,
    const float4* xq = nullptr, float qlim2 = 0.f, int* qflag = nullptr);
int ke_blocks(int n);

// ---- pair-list force path (mdb_cp_pairs.cu) ---------------------------------
// LJ constants per (type i, type j): x = 48 eps s^2, y = 24 eps s, z = s, w = eps
// with s = sigma_ij^6 = sigma_i^3 sigma_j^3 and eps = sqrt(eps_i eps_j) (the
// reference's geometric rule, clusterpair/force_lj.c:130-132); one-type
// systems use a0, b0, sig6_0, eps0
struct PairTypes {
    float4 tab[MDB_MAX_TYPES * MDB_MAX_TYPES];
    float a0, b0, sig6_0;
    double eps0;
};
// chunks of a list row of maxneighs entries (256 / N entries each)
int pair_chunks(int maxneighs, int N);
// blocks of the derivation and force launches (one warp per i-cluster)
int pair_grid(int ncl_cap);
// codes of every i pair (j atoms within sqrt(rin2)) and the positions they
// were derived from (xq); returns at once unless qflag[0] or force is set;
// qflag[1] counts the derivations that ran
void launch_pair_derive(cudaStream_t s, int N, int half, int uniform, int ncl_cap,
    const int* cnt, const float4* xr, const float4* anchor, const int* list, int cs,
    const int* numneigh, float rin2, int* qflag, int force, unsigned char* pcode,
    unsigned short* pcnt, int chmax, float4* xq);
// MDB_PREC_MIXED_COMP: FP64 slot positions for the exact cutoff decision, the
// FP64 force slots that receive the forces, FP64 r_c^2 (cf64 null: plain mixed)
struct CompArgs {
    const double4* cx = nullptr;
    double4* cf64     = nullptr;
    double cutsq      = 0.0;
};
// forces from the codes; clears qflag[0]; variant: launch shape (0..3);
// returns the blocks launched (= energy partials written)
int launch_force_pairs(cudaStream_t s, int N, int half, int energy, int uniform, int variant,
    int ncl_cap,
    const int* cnt, const float4* xr, const float4* anchor, const PairTypes& pt,
    float cutforcesq, const int* list, int cs, const int* numneigh,
    const unsigned char* pcode, const unsigned short* pcnt, int chmax, float4* cf32,
    double* epart, int* qflag, const CompArgs& ca = CompArgs());

// ---- batched launches over the members of an ensemble -----------------------
// One launch covers every member: block b of the launch runs block bmap[b].y
// of member bmap[b].x, whose buffers come from a device table. The block maps
// are built on the host from the members' capacities, so a captured graph
// stays valid until a member's buffers move.
struct CpStepMember { // integrator and ghost update
    const int* cnt;
    double4* cx;
    double4* cv;
    const double4* cf;
    float4* cf32;
    const float4* anchor;
    float4* xr;
    const int* border;
    const int* pbc;
    const int* jnat;
    double dtf, dt, xprd, yprd, zprd;
    int M, N, mixed; // mixed: 0 FP64, else the xr mode of put_rel
    int zero_f; // half lists: the force slots are cleared before each force evaluation
    const double4* xb; // displacement check (null: off), see launch_cp_initial
    double lim2;
    int* flag;
};
struct CpForceMember { // mixed force kernel (row-major lists)
    const int* cnt;
    const float4* xr;
    const float4* anchor;
    const int* list;
    const int* numneigh;
    float4* cf32;
    double* epart;
    int cs, pad;
};
// Every buffer and size the rebuild kernels of one member use.
struct CpBuildMember {
    Geom g;
    int M, N, jfac, mixed, half, nlocal, ncl_cap, ncj_cap, ngc_cap, maxneighs, ks, cs;
    int* cnt;
    unsigned long long* zext;
    double4 *ax, *av, *cx, *cv;
    int *cl_first, *atom_col, *col_count, *col_start, *col_fill, *col_atoms, *col_sorted, *gidx;
    double* gz;
    int *ncl_col, *cl_start, *inat, *cbin;
    double4 *ibbmin, *ibbmax;
    int* jnat;
    double4 *jbbmin, *jbbmax;
    float4 *anchor, *xr;
    int *gcount, *gstart, *border, *pbc, *gcolumn, *gcol_count, *jcol_n, *jcol_start, *gfill;
    int *gtmp, *jcol;
    double4 *jcbbmin, *jcbbmax;
    float4 *jcbbf, *cxf;
    int* ztab;
    int slot_cap;
    const int* stencil;
    int *list, *numneigh, *nmasked;
};
// stages of a batched rebuild, in order; the block-map entry of each stage
// covers every member's grid of the single-member launch
enum CpBuildStage {
    CB_RESET,    // counters and column counts to zero
    CB_GATHER,   // updateSingleAtoms + updateAtomsPbc
    CB_BIN,      // binAtoms
    CB_SCATTER,  // column lists
    CB_SORT,     // sortAtomsByZCoord
    CB_CLUSTERS, // buildClusters + defineJClusters
    CB_GCOUNT,   // setupPbc: images per j-cluster
    CB_GWRITE,   // setupPbc: ghost table
    CB_GFIRST,   // updatePbc(first)
    CB_GCOLS,    // binJClusters: ghost columns
    CB_CSIZES,   // binJClusters: column sizes
    CB_GSCATTER, // binJClusters: ghosts into columns
    CB_MERGE,    // binJClusters: merge by bbminz
    CB_PREP,     // buildNeighbor: FP32 copies of boxes and positions, window table
    CB_LIST,     // buildNeighbor
    CB_COUNT
};
// blocks (and threads per block) of a stage for one member
int cp_build_stage_blocks(int stage, const CpBuildMember& m, int* threads);
// the stage over all members: nblocks entries of bmap (only: null, or a flag
// per member, 0 = the member skips it)
void launch_build_stage_batch(cudaStream_t s, int stage, int nblocks,
    const CpBuildMember* tab, const int2* bmap, const int* only);
// the column scans of the rebuild (which: 0 col_count, 1 ncl_col, 2 gcount,
// 3 jcol_n), one block per member (only: as above)
void launch_scan_batch(cudaStream_t s, int which, int nmem, const CpBuildMember* tab,
    const int* only);
// the displacement check's reference positions of the members whose flag in
// only is set (slots as built), over the integrator's block map
void launch_snapshot_batch(cudaStream_t s, int nblocks, const CpStepMember* tab,
    const int2* bmap, const int* only);
// every member's CP_SLOTS counters into out[member * CP_SLOTS + k]
void launch_counters_batch(cudaStream_t s, int nmem, const CpBuildMember* tab, int* out);

void launch_cp_integrate_batch(cudaStream_t s, bool final_, bool initial, int nblocks,
    const CpStepMember* tab, const int2* bmap);
// half-list members (zero_f): force slots [0, ncl * M) to zero, over the
// integrator's block map; launched right before the force evaluation
void launch_zero_forces_batch(cudaStream_t s, int nblocks, const CpStepMember* tab,
    const int2* bmap);
// skip: null, or a flag per member (set = the member skips the update)
void launch_ghost_update_batch(cudaStream_t s, int nblocks, const CpStepMember* tab,
    const int2* bmap, const int* skip);
void launch_force_mixed_batch(cudaStream_t s, int N, int half, int energy, const Types& ty,
    float cutforcesq, int nblocks, const CpForceMember* tab, const int2* bmap);
void launch_ke_atoms(cudaStream_t s, int n, const double4* av, double mass, double* partials);
void launch_ke_slots(cudaStream_t s, int M, int ncl_cap, const int* cnt, const double4* cx,
    const double4* cv, double mass, double* partials);

} // namespace cp
} // namespace mdb
