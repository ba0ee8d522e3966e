// Internal declarations shared by the libmdb translation units.
// Device data layout (HBM), per context:
//   x        double4[nall_cap]  positions of locals then ghosts; .w holds the type
//                               id as raw int bits (never used arithmetically)
//   xr       float4[nall_cap]   mixed path: position relative to the centre of the
//                               atom's cell (cells of edge G, a power of two, fixed at
//                               each rebuild), .w type bits
//   qcell    int[nall_cap]      mixed path: the cell of each atom, 10 bits per axis
//   vx,vy,vz / fx,fy,fz         SoA doubles over locals
//   neighbors int32 [maxneighs][ld]  SoA (k-major), row t belongs to atom
//                               local_order[t] (atoms of one bin are adjacent rows);
//                               mixed path: bits 0-24 index, bits 25-31 cell-offset code
//   numneigh  int32 [nlocal]    indexed by row t
//   bins: CSR (bin_start[mbins+1], bin_atoms[nall]) with atoms of a bin in
//         ascending index order, so lists come out in the reference order
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "mdb.h"

#define MDB_MAX_TYPES   8
#define MDB_MAX_STENCIL 1331 /* (2*5+1)^3 */
#define MDB_IDX_BITS    26   /* mixed-path list entries: index bits (6 code bits above) */
#define MDB_IDX_MASK    ((1 << MDB_IDX_BITS) - 1)

// device counters (int slots)
enum {
    CNT_NGHOST       = 0, // ghosts in use (clamped to capacity)
    CNT_NGHOST_TOTAL = 1, // ghosts requested by the last setupPbc
    CNT_MAXNEED      = 2, // largest numneigh seen when a row overflowed
    CNT_BADBIN       = 3, // atoms found outside the bin grid
    CNT_BADCELL      = 4, // mixed path: neighbour farther than two cells
    CNT_SLOTS        = 8
};

struct BinGeom {
    int nbinx, nbiny, nbinz;
    int mbinx, mbiny, mbinz;
    int pad_x, pad_y, pad_z;
    int nstencil, mbins;
    double binsizex, binsizey, binsizez;
    double bininvx, bininvy, bininvz;
    double xlo, ylo, zlo; // fabs(0 - pad*binsize) + 1e-9, verletlist/neighbor.c:361-366
};

struct LJTable {
    int ntypes;
    int uniform; // every type pair has the same epsilon and sigma6
    double eps[MDB_MAX_TYPES * MDB_MAX_TYPES];
    double sig6[MDB_MAX_TYPES * MDB_MAX_TYPES];
};

struct LJTableF {
    int ntypes;
    int uniform;
    float eps[MDB_MAX_TYPES * MDB_MAX_TYPES];
    float sig6[MDB_MAX_TYPES * MDB_MAX_TYPES];
};

// Mixed-path cells: edge G, the smallest power of two >= cutneigh, so the
// cells of a listed pair differ by -1, 0 or +1 per axis and offset * G is
// exact in FP32. A list entry stores the three offsets + 1 as 2-bit fields
// above the index bits.
struct CellFrame {
    double g;
    double ginv;
};

struct CellShift {
    float g;
};

// cell offset (-1, 0 or +1) of 2-bit field f, as an exact float without an
// int->float conversion: 0x4B400000 is 1.5 * 2^23, so OR-ing f into the
// mantissa gives 12582912 + f exactly
__device__ __forceinline__ float cell_offset(unsigned f)
{
    return __int_as_float(0x4B400000 | (int)f) - 12582913.0f;
}

// pair difference p_i - p_j - offset * G on the mixed path; a fused multiply-add
// with the exact product offset * G rounds once
__device__ __forceinline__ void cell_delta(const float4& pi, const float4& pj, unsigned code,
    float g, float& dx, float& dy, float& dz)
{
    dx = __fmaf_rn(-cell_offset(code & 3u), g, pi.x - pj.x);
    dy = __fmaf_rn(-cell_offset((code >> 2) & 3u), g, pi.y - pj.y);
    dz = __fmaf_rn(-cell_offset((code >> 4) & 3u), g, pi.z - pj.z);
}

struct EamDev {
    int nrho, nr;
    double rdr, rdrho;
    const double* frho; // rows of 8 doubles (coefficients 0..6 + pad)
    const double* rhor;
    const double* z2r;
    const float* frho32;
    // mixed path, FP32 rows: dens32[m] = rho coefficients 3..6 (the density
    // pass); pair32[2m], pair32[2m + 1] = z2r coefficients 3..6, then rho
    // coefficients 0..2 and z2r coefficient 0 (the force pass: z2r 1 and 2
    // are 2 c4 / dr and c5 / dr of the spline, formed in the kernel)
    const float4* dens32;
    const float4* pair32;
};

namespace mdb {

// ---- small device helpers ---------------------------------------------------
__device__ __forceinline__ int type_of(const double4& p) { return (int)__double_as_longlong(p.w); }

// read-only 32-byte position load as two 16-byte non-coherent loads of one sector
// a double4 in one 256-bit read-only load (sm_100; p 32-byte aligned, as
// every double4 array from cudaMalloc is)
__device__ __forceinline__ double4 ldg4(const double4* p)
{
    double4 r;
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
        : "=d"(r.x), "=d"(r.y), "=d"(r.z), "=d"(r.w)
        : "l"(p));
    return r;
}

__device__ __forceinline__ int pack_cell(int cx, int cy, int cz)
{
    return (cx + 512) | ((cy + 512) << 10) | ((cz + 512) << 20);
}

__device__ __forceinline__ int cell_axis(int q, int a) { return ((q >> (10 * a)) & 1023) - 512; }

// position relative to the centre of cell q, FP32
__device__ __forceinline__ float4 rel_position(const double4& p, int q, const CellFrame& cf)
{
    float4 r;
    r.x = (float)(p.x - ((double)cell_axis(q, 0) + 0.5) * cf.g);
    r.y = (float)(p.y - ((double)cell_axis(q, 1) + 0.5) * cf.g);
    r.z = (float)(p.z - ((double)cell_axis(q, 2) + 0.5) * cf.g);
    r.w = __int_as_float(type_of(p));
    return r;
}

// block-wide sum; the result is valid in thread 0 (all threads must call)
__device__ __forceinline__ double block_sum(double v)
{
    __shared__ double ws[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) ws[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (warp == 0) {
        t = lane < (int)(blockDim.x >> 5) ? ws[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1)
            t += __shfl_down_sync(0xffffffffu, t, o);
    }
    __syncthreads();
    return t;
}

// ---- launch helpers (implemented in the .cu files) --------------------------

// scan: out[0..n] exclusive prefix sums of in[0..n-1]; out[n] = total.
// scratch must hold scan_scratch_ints(n) ints.
int scan_scratch_ints(int n);
void scan_exclusive(const int* in, int* out, int n, int* scratch, cudaStream_t s);

// integrator / pbc / thermo (mdb_vl.cu). xr/qcell are null on the FP64 path.
void launch_initial_integrate(cudaStream_t s, int n, double dtf, double dt, double4* x,
    double* vx, double* vy, double* vz, const double* fx, const double* fy, const double* fz,
    float4* xr, const int* qcell, CellFrame cf);
void launch_final_integrate(cudaStream_t s, int n, double dtf, double* vx, double* vy,
    double* vz, const double* fx, const double* fy, const double* fz);
// finalIntegrate of step n followed by initialIntegrate of step n+1 in one pass
void launch_final_initial_integrate(cudaStream_t s, int n, double dtf, double dt, double4* x,
    double* vx, double* vy, double* vz, const double* fx, const double* fy, const double* fz,
    float4* xr, const int* qcell, CellFrame cf);
void launch_pack_atoms(cudaStream_t s, int n, const double* xa, const double* va,
    const int* ta, double4* x, double* vx, double* vy, double* vz);
void launch_unpack_atoms(cudaStream_t s, int n, const double4* x, const double* vx,
    const double* vy, const double* vz, const double* fx, const double* fy, const double* fz,
    double* xa, double* va, double* fa, int* ta);
void launch_wrap(cudaStream_t s, int n, double4* x, double xprd, double yprd, double zprd);
// gathers of sortAtom: out[k] = in[order[k]] (three SoA arrays into out[0..3n))
void launch_permute4(cudaStream_t s, int n, const int* order, const double4* in, double4* out);
void launch_permute3(cudaStream_t s, int n, const int* order, const double* a, const double* b,
    const double* c, double* out);
void launch_ghost_count(cudaStream_t s, int n, const double4* x, double cut, double xprd,
    double yprd, double zprd, int px, int py, int pz, int* cnt);
void launch_ghost_write(cudaStream_t s, int n, int ghost_cap, double4* x, double cut,
    double xprd, double yprd, double zprd, int px, int py, int pz, const int* off,
    int* border_map, int* pbc_code, int* counters);
// ghost positions from their owners; with xr/qcell also the mixed-path copies
// (then x of the ghosts is not written: only the rebuild needs it)
void launch_ghost_update(cudaStream_t s, int nlocal, int ghost_cap, double4* x,
    const int* border_map, const int* pbc_code, double xprd, double yprd, double zprd,
    const int* counters, float4* xr, const int* qcell, CellFrame cf);
// cells and relative positions of atoms [first, first + count) (count may be
// read from counters: pass count < 0 to use nlocal + counters[CNT_NGHOST])
void launch_cells(cudaStream_t s, int nlocal, int nall_cap, const double4* x, float4* xr,
    int* qcell, CellFrame cf, const int* counters, int locals_only);
void launch_bin_count(cudaStream_t s, int nlocal, int nall_cap, const double4* x, BinGeom g,
    int* atom_bin, int* atom_slot, int* bin_count, int* bin_lcount, int* counters);
void launch_bin_scatter(cudaStream_t s, int nlocal, int nall_cap, const int* atom_bin,
    const int* atom_slot, const int* bin_start, int* bin_atoms, const int* counters);
void launch_bin_sort(cudaStream_t s, int mbins, const int* bin_start, int* bin_atoms,
    const int* loc_start, int* local_order);
// stencil entries: {flat bin offset, dx, dy, dz}; qcell non-null packs cell codes
// positions of the binned atoms in bin order (atom index bits in .w), FP64
// and rounded to FP32
void launch_bin_positions(cudaStream_t s, int nall_cap, int mbins, const double4* x,
    const int* bin_start, const int* bin_atoms, double4* bin_x, float4* bin_xf);
// the Verlet list from the bin-ordered positions; margin bounds the FP32
// prefilter's rsq error (only candidates within it take the exact FP64 test)
void launch_build_list(cudaStream_t s, int nlocal, const double4* x, BinGeom g,
    const int4* stencil, const int* atom_bin, const int* bin_start,
    const double4* bin_x, const float4* bin_xf, double cutneighsq, float margin, int half,
    int maxneighs, int ld, int* neighbors, int* numneigh, int* counters, const int* qcell);
int ke_partial_blocks(int n);
void launch_ke_partial(cudaStream_t s, int n, const double* vx, const double* vy,
    const double* vz, double mass, double* partials);
void launch_reduce_partials(cudaStream_t s, int nparts, const double* partials, double* out);

// forces (mdb_force_lj.cu, mdb_force_eam.cu); thread t handles atom order[t]
int force_partial_blocks(int n);
void launch_lj_fp64(cudaStream_t s, int half, int energy, int nlocal, const int* order,
    const double4* x, const int* numneigh, const int* neighbors, int ld, double cutforcesq,
    const LJTable& tab, double* fx, double* fy, double* fz, double* epart);
void launch_lj_mixed(cudaStream_t s, int comp, int half, int energy, int nlocal,
    const int* order, const float4* xr, const CellShift& sh, const int* numneigh,
    const int* neighbors, int ld, float cutforcesq, const LJTableF& tab, double* fx,
    double* fy, double* fz, double* epart);
void launch_eam_fp64(cudaStream_t s, int energy, int nlocal, int ghost_cap, const int* order,
    const double4* x, const int* numneigh, const int* neighbors, int ld, double cutforcesq,
    EamDev eam, const int* border_map, const int* counters, double* fp, double* fx,
    double* fy, double* fz, double* epart_rho, double* epart_pair);
// mixed EAM: four threads per atom; xe (nlocal + ghost_cap) receives
// (position, F'(rho)) of every atom for the force pass; comp: two-sum
// compensated force sums; returns the energy partials written per pass
int launch_eam_mixed(cudaStream_t s, int energy, int comp, int rho_lanes, int nlocal,
    int ghost_cap,
    const float4* xr, const CellShift& sh, const int* numneigh, const int* neighbors, int ld,
    float cutforcesq, EamDev eam, const int* border_map, const int* counters, int* cut,
    int* ncut, double* fp, float4* xe, double* fx, double* fy, double* fz, double* epart_rho,
    double* epart_pair);
int eam_mixed_blocks(int nlocal);

// domain-decomposed runs: positions of atoms idx[0..n) plus a shift, AoS
// triples (the halo another domain receives); and the positions of halo
// atoms [first, first + n) from AoS triples (mixed: relative copies too)
void launch_gather_positions(cudaStream_t s, int n, const int* idx, const double4* x, double sx,
    double sy, double sz, double* out);
void launch_set_halo(cudaStream_t s, int first, int n, const double* in, double4* x, float4* xr,
    const int* qcell, const CellFrame& cf);

// launches issued through these helpers by the calling host thread (per
// thread, so that contexts driven from different threads count their own:
// a context is used by one thread at a time)
extern thread_local long long g_launches;

} // namespace mdb

#define MDB_NTHREADS 256
static inline int mdb_blocks(long long n, int t) { return (int)((n + t - 1) / t); }
