// Cluster-pair scheme, the rebuild path: updateSingleAtoms/updateAtomsPbc,
// binAtoms + sortAtomsByZCoord + buildClusters + defineJClusters, setupPbc +
// updatePbc, binJClusters and buildNeighbor (4xN, bounding-box pruned), plus
// pruneNeighbor. Every result is the reference's, bit for bit: the same FP64
// expressions in the same order, and the same orders of atoms in columns, of
// j-clusters in columns and of entries in the lists.
#include <math.h>

#include "mdb_cp_f2.cuh"
#include "mdb_cp_internal.cuh"

namespace mdb {
namespace cp {

static __device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// ---- updateSingleAtoms + updateAtomsPbc --------------------------------------
// clusterpair/neighbor.c:2096-2149 (slot -> atom index = atoms of the clusters
// before it) and clusterpair/pbc.c:116-143 (wrap into the box)
__device__ __forceinline__ void gather_blk(int bid, int M, const int* __restrict__ cnt,
    const double4* __restrict__ cx,
    const double4* __restrict__ cv, const int* __restrict__ cl_first, double4* __restrict__ ax,
    double4* __restrict__ av, int wrap, double xprd, double yprd, double zprd)
{
    const int s = bid * blockDim.x + threadIdx.x;
    if (s >= cnt[CP_NCL] * M) return;
    double4 p = cx[s];
    if (slot_type(p) < 0) return;
    const int a = cl_first[s / M] + s % M;
    if (wrap) {
        if (p.x < 0.0) p.x += xprd;
        else if (p.x >= xprd) p.x -= xprd;
        if (p.y < 0.0) p.y += yprd;
        else if (p.y >= yprd) p.y -= yprd;
        if (p.z < 0.0) p.z += zprd;
        else if (p.z >= zprd) p.z -= zprd;
    }
    ax[a] = p;
    av[a] = cv[s];
}

__global__ void k_gather(int M, const int* __restrict__ cnt, const double4* __restrict__ cx,
    const double4* __restrict__ cv, const int* __restrict__ cl_first, double4* __restrict__ ax,
    double4* __restrict__ av, int wrap, double xprd, double yprd, double zprd)
{
    gather_blk(blockIdx.x, M, cnt, cx, cv, cl_first, ax, av, wrap, xprd, yprd, zprd);
}

void launch_gather(cudaStream_t s, int M, int ncl_cap, const int* cnt, const double4* cx,
    const double4* cv, const int* cl_first, double4* ax, double4* av, int wrap, double xprd,
    double yprd, double zprd)
{
    long long n = (long long)ncl_cap * M;
    k_gather<<<mdb_blocks(n, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(M, cnt, cx, cv, cl_first, ax,
        av, wrap, xprd, yprd, zprd);
    g_launches++;
}

// ---- binAtoms (clusterpair/neighbor.c:1409-1449) -----------------------------
// Atoms arrive in cluster order from the last build, so the lanes of a warp
// mostly share a column: one atomic per distinct column of the warp
// (__match_any_sync). The order in which a column's atoms are appended does
// not matter: the column sort orders them by z and atom index.
__device__ __forceinline__ void bin_atoms_blk(int bid, int n, const double4* __restrict__ ax,
    Geom g, int* atom_col,
    int* col_count, int* cnt)
{
    const int i = bid * blockDim.x + threadIdx.x;
    int b       = -1;
    if (i < n) {
        double4 p = ax[i];
        int ix, iy;
        coord2bin2d(g, p.x, p.y, ix, iy);
        b = iy * g.mbinx + ix + 1;
        if (b < 0 || b >= g.mbins) {
            atomicAdd(&cnt[CP_BADBIN], 1);
            b = -1;
        }
        atom_col[i] = b;
    }
    const unsigned peers = __match_any_sync(0xffffffffu, b);
    if (b >= 0 && (threadIdx.x & 31) == __ffs(peers) - 1)
        atomicAdd(&col_count[b], __popc(peers));
}

__global__ void k_bin_atoms(int n, const double4* __restrict__ ax, Geom g, int* atom_col,
    int* col_count, int* cnt)
{
    bin_atoms_blk(blockIdx.x, n, ax, g, atom_col, col_count, cnt);
}

void launch_bin_atoms(cudaStream_t s, int n, const double4* ax, const Geom& g, int* atom_col,
    int* col_count, int* cnt)
{
    if (n <= 0) return;
    k_bin_atoms<<<mdb_blocks(n, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(n, ax, g, atom_col,
        col_count, cnt);
    g_launches++;
}

__device__ __forceinline__ void scatter_atoms_blk(int bid, int n, const int* __restrict__ atom_col,
    const int* __restrict__ col_start, int* col_fill, int* col_atoms)
{
    const int i          = bid * blockDim.x + threadIdx.x;
    const int lane       = threadIdx.x & 31;
    const int b          = i < n ? atom_col[i] : -1;
    const unsigned peers = __match_any_sync(0xffffffffu, b);
    const int leader     = __ffs(peers) - 1;
    int base             = 0;
    if (b >= 0 && lane == leader) base = atomicAdd(&col_fill[b], __popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (b >= 0) col_atoms[col_start[b] + base + __popc(peers & ((1u << lane) - 1u))] = i;
}

__global__ void k_scatter_atoms(int n, const int* __restrict__ atom_col,
    const int* __restrict__ col_start, int* col_fill, int* col_atoms)
{
    scatter_atoms_blk(blockIdx.x, n, atom_col, col_start, col_fill, col_atoms);
}

void launch_scatter_atoms(cudaStream_t s, int n, const int* atom_col, const int* col_start,
    int* col_fill, int* col_atoms)
{
    if (n <= 0) return;
    k_scatter_atoms<<<mdb_blocks(n, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(n, atom_col, col_start,
        col_fill, col_atoms);
    g_launches++;
}

// ---- sortAtomsByZCoord (clusterpair/neighbor.c:1452-1481) ----------------------
// One warp per column. The column's atoms arrive in arbitrary order from the
// atomic scatter; a bitonic sort by atom index restores binAtoms' order (atoms
// appended in index order). The reference then runs a selection sort that, for
// each position a, swaps in the first minimum of z among positions a..c-1.
// Without equal z values the result is the unique ascending order, which a
// bitonic sort by z gives directly. Equal z values (a perfect lattice) make the
// result depend on the swaps: such columns go back to index order and the warp
// replays the selection sort exactly, each step a warp-wide (z, position)
// minimum and one swap.
template <bool BY_Z>
__device__ void bitonic(int* idx, double* z, int P)
{
    const int lane = lane_id();
    for (int size = 2; size <= P; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = lane; t < (P >> 1); t += 32) {
                int i   = 2 * t - (t & (stride - 1));
                int j   = i + stride;
                bool up = (i & size) == 0;
                int a = idx[i], b = idx[j];
                double za = z[i], zb = z[j];
                bool gt = BY_Z ? (za > zb || (za == zb && a > b)) : (a > b);
                if (gt == up) {
                    idx[i] = b;
                    idx[j] = a;
                    z[i]   = zb;
                    z[j]   = za;
                }
            }
            __syncwarp();
        }
    }
}

__device__ void sort_column(int* idx, double* z, int c, int P, const double4* __restrict__ ax)
{
    const int lane = lane_id();
    for (int k = lane; k < P; k += 32) {
        if (k >= c) idx[k] = 0x7fffffff;
        z[k] = k < c ? ax[idx[k]].z : INFINITY;
    }
    __syncwarp();
    bitonic<true>(idx, z, P);
    bool tie = false;
    for (int k = lane; k + 1 < c; k += 32)
        tie |= z[k] == z[k + 1];
    if (!__any_sync(0xffffffffu, tie)) return;
    // equal z: back to binAtoms' order, then replay the selection sort
    bitonic<false>(idx, z, P);
    for (int a = 0; a < c; a++) {
        double bz = INFINITY;
        int bp    = 0x7fffffff;
        for (int p = a + lane; p < c; p += 32) {
            double zp = z[p];
            if (zp < bz || bp == 0x7fffffff) {
                bz = zp;
                bp = p;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            double oz = __shfl_xor_sync(0xffffffffu, bz, o);
            int op    = __shfl_xor_sync(0xffffffffu, bp, o);
            if (op != 0x7fffffff && (bp == 0x7fffffff || oz < bz || (oz == bz && op < bp))) {
                bz = oz;
                bp = op;
            }
        }
        if (lane == 0 && bp != a) {
            int ta = idx[a];
            idx[a] = idx[bp];
            idx[bp] = ta;
            double tz = z[a];
            z[a]      = z[bp];
            z[bp]     = tz;
        }
        __syncwarp();
    }
}

#define CP_SORT_WARPS 4

__device__ __forceinline__ void sort_columns_blk(int bid, int mbins, int M, int N,
    const int* __restrict__ col_start, int* col_atoms, const double4* __restrict__ ax,
    int* col_sorted, int* gidx, double* gz, int* ncl_col)
{
    __shared__ int s_idx[CP_SORT_WARPS][CP_COL_SMEM];
    __shared__ double s_z[CP_SORT_WARPS][CP_COL_SMEM];
    const int w    = threadIdx.x >> 5;
    const int b    = bid * CP_SORT_WARPS + w;
    const int lane = lane_id();
    if (b >= mbins) return;
    const int start = col_start[b];
    const int c     = col_start[b + 1] - start;
    int P           = 1;
    while (P < c) P <<= 1;
    int* idx;
    double* z;
    if (P <= CP_COL_SMEM) {
        idx = s_idx[w];
        z   = s_z[w];
    } else {
        // 2 * start leaves room for the power-of-two padding of every column
        idx = gidx + 2 * (size_t)start;
        z   = gz + 2 * (size_t)start;
    }
    for (int k = lane; k < c; k += 32)
        idx[k] = col_atoms[start + k];
    __syncwarp();
    if (c > 0) sort_column(idx, z, c, P, ax);
    for (int k = lane; k < c; k += 32)
        col_sorted[start + k] = idx[k];
    if (lane == 0) {
        int nc = (c + M - 1) / M;
        if (N > M && (nc & 1)) nc++;
        ncl_col[b] = nc;
    }
}

__global__ void __launch_bounds__(32 * CP_SORT_WARPS) k_sort_columns(int mbins, int M, int N,
    const int* __restrict__ col_start, int* col_atoms, const double4* __restrict__ ax,
    int* col_sorted, int* gidx, double* gz, int* ncl_col)
{
    sort_columns_blk(blockIdx.x, mbins, M, N, col_start, col_atoms, ax, col_sorted, gidx, gz,
        ncl_col);
}

void launch_sort_columns(cudaStream_t s, const Geom& g, int M, int N, const int* col_start,
    int* col_atoms, const double4* ax, int* col_sorted, int* gidx, double* gz, int* ncl_col)
{
    // gidx / gz: 2 * nlocal entries each, used by columns longer than CP_COL_SMEM
    int blocks = (g.mbins + CP_SORT_WARPS - 1) / CP_SORT_WARPS;
    k_sort_columns<<<blocks, 32 * CP_SORT_WARPS, 0, s>>>(g.mbins, M, N, col_start, col_atoms, ax,
        col_sorted, gidx, gz, ncl_col);
    g_launches++;
}

// ---- buildClustersCPU + defineJClusters (clusterpair/neighbor.c:1513-1611, :1807-1915)
// One warp per column: slots filled from the z-sorted column in chunks of M
// (padding +INF, type -1), then per cluster its atom count, column and bounding
// box with the reference's compare-and-replace order, then the j-cluster boxes
// (M < N: the union of the two i-clusters of a pair). Mixed path: anchors and
// anchor-relative FP32 positions.
__device__ __forceinline__ float4 anchor_of(const double4& mn, const double4& mx)
{
    const double st = CP_ANCHOR_STEP;
    float4 a;
    a.x = (float)(rint(0.5 * (mn.x + mx.x) / st) * st);
    a.y = (float)(rint(0.5 * (mn.y + mx.y) / st) * st);
    a.z = (float)(rint(0.5 * (mn.z + mx.z) / st) * st);
    a.w = 0.0f;
    return a;
}

__device__ __forceinline__ void zext_max(unsigned long long* zext, double e)
{
    // non-negative doubles order like their bit patterns
    unsigned long long v = (unsigned long long)__double_as_longlong(e > 0.0 ? e : 0.0);
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long u = __shfl_xor_sync(0xffffffffu, v, o);
        v                    = u > v ? u : v;
    }
    if (lane_id() == 0) atomicMax(zext, v);
}

template <int M, int N>
__device__ __forceinline__ void build_clusters_blk(int bid, int mbins, int mixed,
    const int* __restrict__ col_start,
    const int* __restrict__ col_sorted, const int* __restrict__ cl_start,
    const double4* __restrict__ ax, const double4* __restrict__ av, double4* cx, double4* cv,
    int* inat, int* cbin, int* cl_first, double4* ibbmin, double4* ibbmax, int* jnat,
    double4* jbbmin, double4* jbbmax, float4* anchor, float4* xr, int* cnt,
    unsigned long long* zext)
{
    const int b    = (bid * blockDim.x + threadIdx.x) >> 5;
    const int lane = lane_id();
    if (b == 0 && lane == 0) {
        cnt[CP_NCL] = cl_start[mbins];
        cnt[CP_NCJ] = cl_start[mbins] / (N / M);
    }
    if (b >= mbins) return;
    const int start = col_start[b];
    const int c     = col_start[b + 1] - start;
    const int k0    = cl_start[b];
    const int nclu  = cl_start[b + 1] - k0;
    for (int j = lane; j < nclu * M; j += 32) {
        const int slot = k0 * M + j;
        if (j < c) {
            int i     = col_sorted[start + j];
            cx[slot]  = ax[i];
            cv[slot]  = av[i];
        } else {
            cx[slot] = make_double4(INFINITY, INFINITY, INFINITY, type_bits(-1));
            cv[slot] = make_double4(0.0, 0.0, 0.0, 0.0);
        }
    }
    __syncwarp();
    double ext = 0.0;
    for (int k = lane; k < nclu; k += 32) {
        const int ci = k0 + k;
        int nat      = c - k * M;
        nat          = nat < 0 ? 0 : (nat > M ? M : nat);
        double4 mn   = make_double4(INFINITY, INFINITY, INFINITY, 0.0);
        double4 mx   = make_double4(-INFINITY, -INFINITY, -INFINITY, 0.0);
        for (int a = 0; a < nat; a++) {
            double4 p = cx[ci * M + a];
            if (mn.x > p.x) mn.x = p.x;
            if (mx.x < p.x) mx.x = p.x;
            if (mn.y > p.y) mn.y = p.y;
            if (mx.y < p.y) mx.y = p.y;
            if (mn.z > p.z) mn.z = p.z;
            if (mx.z < p.z) mx.z = p.z;
        }
        inat[ci]     = nat;
        cbin[ci]     = b;
        cl_first[ci] = start + k * M;
        ibbmin[ci]   = mn;
        ibbmax[ci]   = mx;
        if (N == M) {
            jnat[ci]   = nat;
            jbbmin[ci] = mn;
            jbbmax[ci] = mx;
            if (nat > 0 && mx.z - mn.z > ext) ext = mx.z - mn.z;
        }
    }
    __syncwarp();
    if (N == 2 * M) {
        for (int kk = lane; kk < (nclu >> 1); kk += 32) {
            const int ci = k0 + 2 * kk, cj = ci >> 1;
            double4 a0 = ibbmin[ci], a1 = ibbmax[ci], b0 = ibbmin[ci + 1], b1 = ibbmax[ci + 1];
            double4 mn, mx;
            mn.x = a0.x < b0.x ? a0.x : b0.x;
            mx.x = a1.x > b1.x ? a1.x : b1.x;
            mn.y = a0.y < b0.y ? a0.y : b0.y;
            mx.y = a1.y > b1.y ? a1.y : b1.y;
            mn.z = a0.z < b0.z ? a0.z : b0.z;
            mx.z = a1.z > b1.z ? a1.z : b1.z;
            mn.w = mx.w = 0.0;
            jbbmin[cj] = mn;
            jbbmax[cj] = mx;
            jnat[cj]   = inat[ci] + inat[ci + 1];
            if (mx.z - mn.z > ext) ext = mx.z - mn.z;
        }
        __syncwarp();
    }
    zext_max(zext, ext);
    if (mixed) {
        const int jfac = N / M;
        const int j0 = k0 / jfac, nj = nclu / jfac;
        for (int k = lane; k < nj; k += 32)
            anchor[j0 + k] = anchor_of(jbbmin[j0 + k], jbbmax[j0 + k]);
        __syncwarp();
        for (int j = lane; j < nclu * M; j += 32) {
            const int slot = k0 * M + j;
            put_rel(xr, slot, cx[slot], anchor[slot / N], mixed, slot % N);
        }
    }
}

template <int M, int N>
__global__ void k_build_clusters(int mbins, int mixed, const int* __restrict__ col_start,
    const int* __restrict__ col_sorted, const int* __restrict__ cl_start,
    const double4* __restrict__ ax, const double4* __restrict__ av, double4* cx, double4* cv,
    int* inat, int* cbin, int* cl_first, double4* ibbmin, double4* ibbmax, int* jnat,
    double4* jbbmin, double4* jbbmax, float4* anchor, float4* xr, int* cnt,
    unsigned long long* zext)
{
    build_clusters_blk<M, N>(blockIdx.x, mbins, mixed, col_start, col_sorted, cl_start, ax, av,
        cx, cv, inat, cbin, cl_first, ibbmin, ibbmax, jnat, jbbmin, jbbmax, anchor, xr, cnt, zext);
}

void launch_build_clusters(cudaStream_t s, const Geom& g, int M, int N, int mixed,
    const int* col_start, const int* col_sorted, const int* cl_start, const double4* ax,
    const double4* av, double4* cx, double4* cv, int* inat, int* cbin, int* cl_first,
    double4* ibbmin, double4* ibbmax, int* jnat, double4* jbbmin, double4* jbbmax,
    float4* anchor, float4* xr, int* cnt, unsigned long long* zext)
{
    long long threads = (long long)g.mbins * 32;
    int blocks        = mdb_blocks(threads, 128);
    if (N == 4)
        k_build_clusters<4, 4><<<blocks, 128, 0, s>>>(g.mbins, mixed, col_start, col_sorted,
            cl_start, ax, av, cx, cv, inat, cbin, cl_first, ibbmin, ibbmax, jnat, jbbmin, jbbmax,
            anchor, xr, cnt, zext);
    else
        k_build_clusters<4, 8><<<blocks, 128, 0, s>>>(g.mbins, mixed, col_start, col_sorted,
            cl_start, ax, av, cx, cv, inat, cbin, cl_first, ibbmin, ibbmax, jnat, jbbmin, jbbmax,
            anchor, xr, cnt, zext);
    g_launches++;
}

// ---- setupPbc (clusterpair/pbc.c:184-331) -------------------------------------
// The 26 images of a j-cluster in the reference's order: 6 faces, 8 corners,
// 12 edges, each present when the box is within cutneigh of that side.
__device__ __forceinline__ int ghost_images(const double4& mn, const double4& mx, const Geom& g,
    int* codes)
{
    const double cut = g.cutneigh;
    const bool lx = mn.x < cut, hx = mx.x >= (g.xprd - cut);
    const bool ly = mn.y < cut, hy = mx.y >= (g.yprd - cut);
    const bool lz = mn.z < cut, hz = mx.z >= (g.zprd - cut);
    int n = 0;
#define CP_IMG(c, dx, dy, dz)                                                            \
    if (c) {                                                                             \
        if (codes) codes[n] = ((dx) + 1) | (((dy) + 1) << 2) | (((dz) + 1) << 4);        \
        n++;                                                                             \
    }
    CP_IMG(lx, +1, 0, 0)
    CP_IMG(hx, -1, 0, 0)
    CP_IMG(ly, 0, +1, 0)
    CP_IMG(hy, 0, -1, 0)
    CP_IMG(lz, 0, 0, +1)
    CP_IMG(hz, 0, 0, -1)
    CP_IMG(lx && ly && lz, +1, +1, +1)
    CP_IMG(lx && hy && lz, +1, -1, +1)
    CP_IMG(lx && ly && hz, +1, +1, -1)
    CP_IMG(lx && hy && hz, +1, -1, -1)
    CP_IMG(hx && ly && lz, -1, +1, +1)
    CP_IMG(hx && hy && lz, -1, -1, +1)
    CP_IMG(hx && ly && hz, -1, +1, -1)
    CP_IMG(hx && hy && hz, -1, -1, -1)
    CP_IMG(lx && lz, +1, 0, +1)
    CP_IMG(lx && hz, +1, 0, -1)
    CP_IMG(hx && lz, -1, 0, +1)
    CP_IMG(hx && hz, -1, 0, -1)
    CP_IMG(ly && lz, 0, +1, +1)
    CP_IMG(ly && hz, 0, +1, -1)
    CP_IMG(hy && lz, 0, -1, +1)
    CP_IMG(hy && hz, 0, -1, -1)
    CP_IMG(ly && lx, +1, +1, 0)
    CP_IMG(ly && hx, -1, +1, 0)
    CP_IMG(hy && lx, +1, -1, 0)
    CP_IMG(hy && hx, -1, -1, 0)
#undef CP_IMG
    return n;
}

__device__ __forceinline__ void ghost_count_blk(int bid, int ncj_cap, const int* __restrict__ cnt,
    const int* __restrict__ jnat, const double4* __restrict__ jbbmin,
    const double4* __restrict__ jbbmax, Geom g, int* gcount)
{
    const int cj = bid * blockDim.x + threadIdx.x;
    if (cj >= ncj_cap) return;
    int n = 0;
    if (cj < cnt[CP_NCJ] && jnat[cj] > 0) n = ghost_images(jbbmin[cj], jbbmax[cj], g, nullptr);
    gcount[cj] = n;
}

__global__ void k_ghost_count(int ncj_cap, const int* __restrict__ cnt,
    const int* __restrict__ jnat, const double4* __restrict__ jbbmin,
    const double4* __restrict__ jbbmax, Geom g, int* gcount)
{
    ghost_count_blk(blockIdx.x, ncj_cap, cnt, jnat, jbbmin, jbbmax, g, gcount);
}

void launch_ghost_count(cudaStream_t s, int ncj_cap, const int* cnt, const int* jnat,
    const double4* jbbmin, const double4* jbbmax, const Geom& g, int* gcount)
{
    k_ghost_count<<<mdb_blocks(ncj_cap, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(ncj_cap, cnt, jnat,
        jbbmin, jbbmax, g, gcount);
    g_launches++;
}

__device__ __forceinline__ void ghost_write_blk(int bid, int ncj_cap, int ngc_cap, int* cnt,
    const int* __restrict__ jnat,
    const double4* __restrict__ jbbmin, const double4* __restrict__ jbbmax, Geom g,
    const int* __restrict__ gstart, int* border, int* pbc)
{
    const int cj = bid * blockDim.x + threadIdx.x;
    if (cj == 0) {
        int total          = gstart[ncj_cap];
        cnt[CP_NGC_TOTAL]  = total;
        cnt[CP_NGC]        = total < ngc_cap ? total : ngc_cap;
    }
    if (cj >= ncj_cap || cj >= cnt[CP_NCJ] || jnat[cj] <= 0) return;
    int codes[26];
    int n  = ghost_images(jbbmin[cj], jbbmax[cj], g, codes);
    int g0 = gstart[cj];
    for (int k = 0; k < n; k++) {
        if (g0 + k >= ngc_cap) break;
        border[g0 + k] = cj;
        pbc[g0 + k]    = codes[k];
    }
}

__global__ void k_ghost_write(int ncj_cap, int ngc_cap, int* cnt, const int* __restrict__ jnat,
    const double4* __restrict__ jbbmin, const double4* __restrict__ jbbmax, Geom g,
    const int* __restrict__ gstart, int* border, int* pbc)
{
    ghost_write_blk(blockIdx.x, ncj_cap, ngc_cap, cnt, jnat, jbbmin, jbbmax, g, gstart, border,
        pbc);
}

void launch_ghost_write(cudaStream_t s, int ncj_cap, int ngc_cap, int* cnt, const int* jnat,
    const double4* jbbmin, const double4* jbbmax, const Geom& g, const int* gstart, int* border,
    int* pbc)
{
    k_ghost_write<<<mdb_blocks(ncj_cap, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(ncj_cap, ngc_cap,
        cnt, jnat, jbbmin, jbbmax, g, gstart, border, pbc);
    g_launches++;
}

// updatePbcCPU(first = 1), clusterpair/pbc.c:43-113: ghost positions, padding,
// boxes; one thread per ghost j-cluster, plus one for the dummy cluster
__device__ __forceinline__ void ghost_first_blk(int bid, int N, int* cnt,
    const int* __restrict__ border,
    const int* __restrict__ pbc, int mixed, Geom g, double4* cx, int* jnat, double4* jbbmin,
    double4* jbbmax, float4* anchor, float4* xr, unsigned long long* zext)
{
    const int gi  = bid * blockDim.x + threadIdx.x;
    const int ngc = cnt[CP_NGC], ncj = cnt[CP_NCJ];
    double ext    = 0.0;
    if (gi < ngc) {
        const int cg = ncj + gi, o = border[gi], code = pbc[gi];
        const double sx = (double)((code & 3) - 1) * g.xprd;
        const double sy = (double)(((code >> 2) & 3) - 1) * g.yprd;
        const double sz = (double)(((code >> 4) & 3) - 1) * g.zprd;
        const int nat   = jnat[o];
        jnat[cg]        = nat;
        atomicAdd(&cnt[CP_NGHOST_ATOMS], nat);
        double4 mn = make_double4(INFINITY, INFINITY, INFINITY, 0.0);
        double4 mx = make_double4(-INFINITY, -INFINITY, -INFINITY, 0.0);
        for (int k = 0; k < N; k++) {
            double4 q;
            if (k < nat) {
                double4 p = cx[o * N + k];
                q         = make_double4(p.x + sx, p.y + sy, p.z + sz, p.w);
                if (mn.x > q.x) mn.x = q.x;
                if (mx.x < q.x) mx.x = q.x;
                if (mn.y > q.y) mn.y = q.y;
                if (mx.y < q.y) mx.y = q.y;
                if (mn.z > q.z) mn.z = q.z;
                if (mx.z < q.z) mx.z = q.z;
            } else {
                q = make_double4(INFINITY, INFINITY, INFINITY, type_bits(-1));
            }
            cx[cg * N + k] = q;
        }
        jbbmin[cg] = mn;
        jbbmax[cg] = mx;
        if (nat > 0) ext = mx.z - mn.z;
        if (mixed) {
            float4 a   = anchor_of(mn, mx);
            anchor[cg] = a;
            for (int k = 0; k < N; k++)
                put_rel(xr, cg * N + k, cx[cg * N + k], a, mixed, k);
        }
    } else if (gi == ngc) {
        const int cd = ncj + ngc; // dummy cluster
        for (int k = 0; k < N; k++) {
            cx[cd * N + k] = make_double4(INFINITY, INFINITY, INFINITY, type_bits(-1));
            if (mixed)
                put_rel(xr, cd * N + k,
                    make_double4(INFINITY, INFINITY, INFINITY, type_bits(-1)),
                    make_float4(0.f, 0.f, 0.f, 0.f), mixed, k);
        }
        if (mixed) anchor[cd] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    zext_max(zext, ext);
}

__global__ void k_ghost_first(int N, int* cnt, const int* __restrict__ border,
    const int* __restrict__ pbc, int mixed, Geom g, double4* cx, int* jnat, double4* jbbmin,
    double4* jbbmax, float4* anchor, float4* xr, unsigned long long* zext)
{
    ghost_first_blk(blockIdx.x, N, cnt, border, pbc, mixed, g, cx, jnat, jbbmin, jbbmax, anchor,
        xr, zext);
}

void launch_ghost_first(cudaStream_t s, int N, int ngc_cap, int mixed, int* cnt,
    const int* border, const int* pbc, const Geom& g, double4* cx, int* jnat, double4* jbbmin,
    double4* jbbmax, float4* anchor, float4* xr, unsigned long long* zext)
{
    k_ghost_first<<<mdb_blocks(ngc_cap + 1, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(N, cnt, border,
        pbc, mixed, g, cx, jnat, jbbmin, jbbmax, anchor, xr, zext);
    g_launches++;
}

// updatePbcCPU(first = 0): ghost positions from their owners every step
__device__ __forceinline__ void ghost_update_slot(int s, int N, int mixed,
    const int* __restrict__ cnt, const int* __restrict__ border, const int* __restrict__ pbc,
    const int* __restrict__ jnat, double xprd, double yprd, double zprd, double4* cx,
    const float4* __restrict__ anchor, float4* xr)
{
    const int gi = s / N, k = s - gi * N;
    if (gi >= cnt[CP_NGC]) return;
    const int cg = cnt[CP_NCJ] + gi;
    if (k >= jnat[cg]) return;
    const int code = pbc[gi];
    double4 p      = cx[border[gi] * N + k];
    p.x += (double)((code & 3) - 1) * xprd;
    p.y += (double)(((code >> 2) & 3) - 1) * yprd;
    p.z += (double)(((code >> 4) & 3) - 1) * zprd;
    cx[cg * N + k] = p;
    if (mixed) put_rel(xr, cg * N + k, p, anchor[cg], mixed, k);
}

__global__ void k_ghost_update(int N, int mixed, const int* __restrict__ cnt,
    const int* __restrict__ border, const int* __restrict__ pbc, const int* __restrict__ jnat,
    Geom g, double4* cx, const float4* __restrict__ anchor, float4* xr)
{
    ghost_update_slot(blockIdx.x * blockDim.x + threadIdx.x, N, mixed, cnt, border, pbc, jnat,
        g.xprd, g.yprd, g.zprd, cx, anchor, xr);
}

// skip: null, or a flag per member (the members whose flag is set skip it)
__global__ void k_ghost_update_batch(const CpStepMember* __restrict__ tab,
    const int2* __restrict__ bmap, const int* __restrict__ skip)
{
    const int2 bm = __ldg(&bmap[blockIdx.x]);
    if (bm.x < 0 || (skip && skip[bm.x])) return;
    const CpStepMember& m = tab[bm.x];
    ghost_update_slot(bm.y * blockDim.x + threadIdx.x, m.N, m.mixed, m.cnt, m.border, m.pbc,
        m.jnat, m.xprd, m.yprd, m.zprd, m.cx, m.anchor, m.xr);
}

void launch_ghost_update_batch(cudaStream_t s, int nblocks, const CpStepMember* tab,
    const int2* bmap, const int* skip)
{
    if (nblocks <= 0) return;
    k_ghost_update_batch<<<nblocks, MDB_NTHREADS, 0, s>>>(tab, bmap, skip);
    g_launches++;
}

void launch_ghost_update(cudaStream_t s, int N, int ngc_cap, int mixed, const int* cnt,
    const int* border, const int* pbc, const int* jnat, const Geom& g, double4* cx,
    const float4* anchor, float4* xr)
{
    long long n = (long long)ngc_cap * N;
    k_ghost_update<<<mdb_blocks(n, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(N, mixed, cnt, border, pbc,
        jnat, g, cx, anchor, xr);
    g_launches++;
}

// ---- binJClusters (clusterpair/neighbor.c:1917-2094) ------------------------------
// Ghost j-clusters go to the column of their innermost atom (per image
// direction, indexes clamped to the grid) and are inserted before the first
// entry with a larger bbminz. Local j-clusters come first in cluster order and
// are already ordered by bbminz, so the final column is the stable merge of the
// locals and of the ghosts sorted by (bbminz, index).
__device__ __forceinline__ void ghost_columns_blk(int bid, int N, const int* __restrict__ cnt,
    const int* __restrict__ pbc,
    const int* __restrict__ jnat, const double4* __restrict__ cx, Geom g, int* gcolumn,
    int* gcol_count)
{
    const int gi = bid * blockDim.x + threadIdx.x;
    if (gi >= cnt[CP_NGC]) return;
    const int cg = cnt[CP_NCJ] + gi, code = pbc[gi];
    const int dx = (code & 3) - 1, dy = ((code >> 2) & 3) - 1;
    int ix, iy;
    double4 p = cx[cg * N];
    coord2bin2d(g, p.x, p.y, ix, iy);
    ix = max(min(ix, g.mbinx - 1), 0);
    iy = max(min(iy, g.mbiny - 1), 0);
    for (int k = 1; k < jnat[cg]; k++) {
        int nix, niy;
        p = cx[cg * N + k];
        coord2bin2d(g, p.x, p.y, nix, niy);
        nix = max(min(nix, g.mbinx - 1), 0);
        niy = max(min(niy, g.mbiny - 1), 0);
        if (dx > 0 && ix > nix) ix = nix;
        if (dx < 0 && ix < nix) ix = nix;
        if (dy > 0 && iy > niy) iy = niy;
        if (dy < 0 && iy < niy) iy = niy;
    }
    int b       = iy * g.mbinx + ix + 1;
    gcolumn[gi] = b;
    atomicAdd(&gcol_count[b], 1);
}

__global__ void k_ghost_columns(int N, const int* __restrict__ cnt, const int* __restrict__ pbc,
    const int* __restrict__ jnat, const double4* __restrict__ cx, Geom g, int* gcolumn,
    int* gcol_count)
{
    ghost_columns_blk(blockIdx.x, N, cnt, pbc, jnat, cx, g, gcolumn, gcol_count);
}

void launch_ghost_columns(cudaStream_t s, int N, int ngc_cap, const int* cnt, const int* pbc,
    const int* jnat, const double4* cx, const Geom& g, int* gcolumn, int* gcol_count)
{
    k_ghost_columns<<<mdb_blocks(ngc_cap, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(N, cnt, pbc, jnat,
        cx, g, gcolumn, gcol_count);
    g_launches++;
}

__device__ __forceinline__ void column_sizes_blk(int bid, int mbins1, int jfac,
    const int* __restrict__ ncl_col,
    const int* __restrict__ gcol_count, int* jcol_n)
{
    const int b = bid * blockDim.x + threadIdx.x;
    if (b < mbins1) jcol_n[b] = ncl_col[b] / jfac + gcol_count[b];
}

__global__ void k_column_sizes(int mbins1, int jfac, const int* __restrict__ ncl_col,
    const int* __restrict__ gcol_count, int* jcol_n)
{
    column_sizes_blk(blockIdx.x, mbins1, jfac, ncl_col, gcol_count, jcol_n);
}

void launch_column_sizes(cudaStream_t s, int mbins1, int jfac, const int* ncl_col,
    const int* gcol_count, int* jcol_n)
{
    k_column_sizes<<<mdb_blocks(mbins1, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(mbins1, jfac, ncl_col,
        gcol_count, jcol_n);
    g_launches++;
}

__device__ __forceinline__ void ghost_scatter_blk(int bid, const int* __restrict__ cnt,
    const int* __restrict__ gcolumn,
    const int* __restrict__ jcol_start, const int* __restrict__ ncl_col, int jfac, int* gfill,
    int* gtmp)
{
    const int gi = bid * blockDim.x + threadIdx.x;
    if (gi >= cnt[CP_NGC]) return;
    const int b = gcolumn[gi];
    gtmp[jcol_start[b] + ncl_col[b] / jfac + atomicAdd(&gfill[b], 1)] = cnt[CP_NCJ] + gi;
}

__global__ void k_ghost_scatter(const int* __restrict__ cnt, const int* __restrict__ gcolumn,
    const int* __restrict__ jcol_start, const int* __restrict__ ncl_col, int jfac, int* gfill,
    int* gtmp)
{
    ghost_scatter_blk(blockIdx.x, cnt, gcolumn, jcol_start, ncl_col, jfac, gfill, gtmp);
}

void launch_ghost_scatter(cudaStream_t s, int ngc_cap, const int* cnt, const int* gcolumn,
    const int* jcol_start, const int* ncl_col, int jfac, int* gfill, int* gtmp)
{
    k_ghost_scatter<<<mdb_blocks(ngc_cap, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(cnt, gcolumn,
        jcol_start, ncl_col, jfac, gfill, gtmp);
    g_launches++;
}

__device__ __forceinline__ void merge_columns_blk(int bid, int mbins1, int jfac,
    const int* __restrict__ ncl_col,
    const int* __restrict__ cl_start, const int* __restrict__ gcol_count,
    const int* __restrict__ jcol_start, const int* __restrict__ gtmp,
    const double4* __restrict__ jbbmin, const double4* __restrict__ jbbmax, int* jcol,
    double4* jcbbmin, double4* jcbbmax)
{
    const int b    = (bid * blockDim.x + threadIdx.x) >> 5;
    const int lane = lane_id();
    if (b >= mbins1) return;
    const int start = jcol_start[b];
    const int nl = ncl_col[b] / jfac, ng = gcol_count[b];
    const int cj0 = b < mbins1 - 1 ? cl_start[b] / jfac : 0;
    const int* gl = gtmp + start + nl;
    for (int i = lane; i < nl; i += 32) {
        const double key = jbbmin[cj0 + i].z;
        int before       = 0;
        for (int e = 0; e < ng; e++)
            before += jbbmin[gl[e]].z < key;
        const int m = start + i + before;
        jcol[m]     = cj0 + i;
        jcbbmin[m]  = jbbmin[cj0 + i];
        jcbbmax[m]  = jbbmax[cj0 + i];
    }
    for (int e = lane; e < ng; e += 32) {
        const int gj     = gl[e];
        const double key = jbbmin[gj].z;
        int pos          = 0;
        for (int i = 0; i < nl; i++)
            pos += jbbmin[cj0 + i].z <= key;
        for (int f = 0; f < ng; f++) {
            const int gf  = gl[f];
            const double kf = jbbmin[gf].z;
            pos += kf < key || (kf == key && gf < gj);
        }
        jcol[start + pos]    = gj;
        jcbbmin[start + pos] = jbbmin[gj];
        jcbbmax[start + pos] = jbbmax[gj];
    }
}

__global__ void k_merge_columns(int mbins1, int jfac, const int* __restrict__ ncl_col,
    const int* __restrict__ cl_start, const int* __restrict__ gcol_count,
    const int* __restrict__ jcol_start, const int* __restrict__ gtmp,
    const double4* __restrict__ jbbmin, const double4* __restrict__ jbbmax, int* jcol,
    double4* jcbbmin, double4* jcbbmax)
{
    merge_columns_blk(blockIdx.x, mbins1, jfac, ncl_col, cl_start, gcol_count, jcol_start, gtmp,
        jbbmin, jbbmax, jcol, jcbbmin, jcbbmax);
}

void launch_merge_columns(cudaStream_t s, int mbins1, int jfac, const int* ncl_col,
    const int* cl_start, const int* gcol_count, const int* jcol_start, const int* gtmp,
    const double4* jbbmin, const double4* jbbmax, int* jcol, double4* jcbbmin, double4* jcbbmax)
{
    long long threads = (long long)mbins1 * 32;
    k_merge_columns<<<mdb_blocks(threads, 128), 128, 0, s>>>(mbins1, jfac, ncl_col, cl_start,
        gcol_count, jcol_start, gtmp, jbbmin, jbbmax, jcol, jcbbmin, jcbbmax);
    g_launches++;
}

// ---- buildNeighborCPU (clusterpair/neighbor.c:282-529) ---------------------------
// One warp per i-cluster. Within a column the j-clusters are sorted by bbminz,
// so the candidates of each stencil column form a window [lo, hi): lane k
// finds column k's window by two binary searches, skipping below the clusters
// whose box lies more than cutneigh under the i box (with the largest z extent
// of any j-cluster and a margin) and above those starting more than cutneigh
// over it; both skipped groups fail the reference's test exactly. The windows
// are then concatenated in stencil order and the warp tests 32 candidates at a
// time, one per lane, with the reference's test: box distance squared (z, y,
// x) below cutneigh^2, accepted below rbb^2, else if any atom pair has
// fma(dx,dx,fma(dy,dy,dz*dz)) below cutneigh^2. A ballot keeps the accepted
// ones in candidate order, so a row is stencil order, then column order; the
// diagonal entry is then swapped to the front as the reference's masked
// entries are.
template <int M, int N>
__device__ __forceinline__ bool any_pair(const double3* xi, const double4* __restrict__ cj_x,
    double cutsq)
{
    bool hit = false;
#pragma unroll
    for (int b = 0; b < N; b++) {
        double4 xj = cj_x[b];
#pragma unroll
        for (int a = 0; a < M; a++) {
            double dx = xi[a].x - xj.x, dy = xi[a].y - xj.y, dz = xi[a].z - xj.z;
            double rsq = __fma_rn(dx, dx, __fma_rn(dy, dy, dz * dz));
            hit |= rsq < cutsq;
        }
    }
    return hit;
}

__device__ __forceinline__ double bb_axis(double imin, double imax, double jmin, double jmax)
{
    double dl = imin - jmax, dh = jmin - imax;
    double dm = dl > dh ? dl : dh;
    return dm > 0.0 ? dm : 0.0;
}

#define CP_LIST_WARPS 4
// resident blocks of 4 warps asked of the register allocator for the list
// build (latency-bound: occupancy pays more than registers for its rare
// exact fallbacks)
#define CP_LIST_MINB 8
#define CP_LIST_EXPAND 256

// FP32 copies for the prefilter: thread t rounds slot t's position and, if t
// is a column entry, that entry's box. Window table: entry q of column c
// (t = c * (zq + 2) + q) is the first entry of the column whose bbminz lies
// in bucket q or above (the column end for q = zq + 1), so that the entries
// of buckets [qa, qb] are [ztab[qa], ztab[qb + 1]).
__host__ __device__ __forceinline__ int list_prep_threads(const Geom& g, int slot_cap)
{
    const int zt = g.mbins * (g.zq + 2);
    return slot_cap > zt ? slot_cap : zt;
}

__device__ __forceinline__ void list_prep_blk(int bid, int N, int slot_cap, const Geom& g,
    const int* __restrict__ cnt, const int* __restrict__ jcol_start,
    const double4* __restrict__ jcbbmin, const double4* __restrict__ jcbbmax,
    const double4* __restrict__ cx, float4* jcbbf, float4* cxf, int* ztab)
{
    const int t = bid * blockDim.x + threadIdx.x;
    if (t < (cnt[CP_NCJ] + cnt[CP_NGC] + 1) * N && t < slot_cap) {
        const double4 p = cx[t];
        cxf[t]          = make_float4((float)p.x, (float)p.y, (float)p.z, 0.f);
    }
    if (t < jcol_start[g.mbins + 1]) {
        const double4 a = jcbbmin[t], b = jcbbmax[t];
        jcbbf[2 * t]     = make_float4((float)a.x, (float)a.y, (float)a.z, 0.f);
        jcbbf[2 * t + 1] = make_float4((float)b.x, (float)b.y, (float)b.z, 0.f);
    }
    const int zn = g.zq + 2;
    if (t < g.mbins * zn) {
        const int c = t / zn, q = t - c * zn;
        int L = jcol_start[c], R = jcol_start[c + 1];
        while (L < R) {
            const int mid = (L + R) >> 1;
            if (zbucket(g, jcbbmin[mid].z) < q) L = mid + 1;
            else R = mid;
        }
        ztab[t] = L;
    }
}

__global__ void k_list_prep(int N, int slot_cap, Geom g, const int* __restrict__ cnt,
    const int* __restrict__ jcol_start, const double4* __restrict__ jcbbmin,
    const double4* __restrict__ jcbbmax, const double4* __restrict__ cx, float4* jcbbf,
    float4* cxf, int* ztab)
{
    list_prep_blk(blockIdx.x, N, slot_cap, g, cnt, jcol_start, jcbbmin, jcbbmax, cx, jcbbf, cxf,
        ztab);
}

void launch_list_prep(cudaStream_t s, int N, int slot_cap, const Geom& g, const int* cnt,
    const int* jcol_start, const double4* jcbbmin, const double4* jcbbmax, const double4* cx,
    float4* jcbbf, float4* cxf, int* ztab)
{
    const long long zt = (long long)g.mbins * (g.zq + 2);
    k_list_prep<<<mdb_blocks(slot_cap > zt ? slot_cap : zt, MDB_NTHREADS), MDB_NTHREADS, 0,
        s>>>(N, slot_cap, g, cnt, jcol_start, jcbbmin, jcbbmax, cx, jcbbf, cxf, ztab);
    g_launches++;
}

__device__ __forceinline__ float bb_axis_f(float imin, float imax, float jmin, float jmax)
{
    float dl = imin - jmax, dh = jmin - imax;
    float dm = dl > dh ? dl : dh;
    return dm > 0.f ? dm : 0.f;
}

// The exact FP64 tests, taken only near a threshold: kept out of line so that
// their registers do not weigh on the FP32 path.
template <int M, int N>
__device__ __noinline__ bool exact_any_pair(const double4* __restrict__ ci_x,
    const double4* __restrict__ cj_x, double cutsq)
{
    double3 xi[M];
#pragma unroll
    for (int a = 0; a < M; a++) {
        const double4 p = ci_x[a];
        xi[a]           = make_double3(p.x, p.y, p.z);
    }
    return any_pair<M, N>(xi, cj_x, cutsq);
}

// the reference's box distance (z, y, x); returns d < cutsq, *in_rbb = d < rbbsq
__device__ __noinline__ bool exact_box(const double4* __restrict__ imn_p,
    const double4* __restrict__ imx_p, const double4* __restrict__ jn_p,
    const double4* __restrict__ jx_p, double cutsq, double rbbsq, bool* in_rbb)
{
    const double4 imn = *imn_p, imx = *imx_p, jn = *jn_p, jx = *jx_p;
    double d = bb_axis(imn.z, imx.z, jn.z, jx.z);
    d        = d * d;
    double e = bb_axis(imn.y, imx.y, jn.y, jx.y);
    d += e * e;
    e = bb_axis(imn.x, imx.x, jn.x, jx.x);
    d += e * e;
    *in_rbb = d < rbbsq;
    return d < cutsq;
}

// the i-cluster's 4 FP32 positions as packed pairs (atoms 0,1 and 2,3)
struct IPairs {
    f2 x[2], y[2], z[2];
};

// The reference's pair test decided in FP32 where the rounding margin allows
// (some pair surely inside cutneigh, or every pair surely outside), else by
// the exact FP64 test on the i-cluster's slots ci*M.. and the j-cluster's.
// Two pairs per packed instruction; each squared distance rounds exactly as
// (dx dx + dy dy) + dz dz in scalar FP32, and "some pair below lo" / "some pair
// at or below hi" are decided on the smallest of them.
template <int M, int N>
__device__ __forceinline__ bool any_pair_f(const IPairs& ip, const float4* __restrict__ cjf,
    float lo, float hi, const double4* __restrict__ ci_x, const double4* __restrict__ cj_x,
    double cutsq)
{
    static_assert(M == 4, "i-clusters of 4 atoms");
    float mn = 3.0e38f;
    // the j-cluster's slots two per 256-bit load (cjf is 32-byte aligned: N even)
#pragma unroll
    for (int b = 0; b < N; b += 2) {
        float4 xjp[2];
        ldg_pair4(&cjf[b], xjp[0], xjp[1]);
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const float4 xj = xjp[u];
            const f2 XJ = f2_pack(xj.x, xj.x), YJ = f2_pack(xj.y, xj.y), ZJ = f2_pack(xj.z, xj.z);
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const f2 dx = f2_sub(ip.x[h], XJ), dy = f2_sub(ip.y[h], YJ),
                         dz = f2_sub(ip.z[h], ZJ);
                const f2 r2 = f2_add(f2_add(f2_mul(dx, dx), f2_mul(dy, dy)), f2_mul(dz, dz));
                float r0, r1;
                f2_unpack(r2, r0, r1);
                mn = fminf(mn, fminf(r0, r1));
            }
        }
    }
    if (mn < lo) return true;
    if (!(mn <= hi)) return false;
    return exact_any_pair<M, N>(ci_x, cj_x, cutsq);
}

template <int M, int N>
__device__ __forceinline__ void build_list_blk(int bid, int half, int* cnt, Geom g,
    const int* __restrict__ stencil,
    const int* __restrict__ cbin, const double4* __restrict__ ibbmin,
    const double4* __restrict__ ibbmax, const double4* __restrict__ jcbbmin,
    const double4* __restrict__ jcbbmax, const double4* __restrict__ cx,
    const float4* __restrict__ jcbbf, const float4* __restrict__ cxf,
    const int* __restrict__ jcol, const int* __restrict__ ztab,
    const unsigned long long* __restrict__ zext, int maxneighs, int ks, int cs, int* list,
    int* numneigh, int* nmasked)
{
    __shared__ int s_lo[CP_LIST_WARPS][32];
    __shared__ int s_ws[CP_LIST_WARPS][32];
    // the flattened windows' column-list indices, when they fit (else each
    // candidate finds its column by a binary search over s_ws)
    __shared__ int s_m[CP_LIST_WARPS][CP_LIST_EXPAND];
    const int w    = threadIdx.x >> 5;
    const int ci   = (bid * blockDim.x + threadIdx.x) >> 5;
    const int lane = lane_id();
    if (ci >= cnt[CP_NCL]) return;
    const int ci_cj0 = ci / (N / M);
    const double imnz = ibbmin[ci].z, imxz = ibbmax[ci].z;
    float3 xif[M];
#pragma unroll
    for (int a = 0; a < M; a++) {
        const float4 p = cxf[ci * M + a];
        xif[a]         = make_float3(p.x, p.y, p.z);
    }
    IPairs ipf;
#pragma unroll
    for (int h = 0; h < 2; h++) {
        ipf.x[h] = f2_pack(xif[2 * h].x, xif[2 * h + 1].x);
        ipf.y[h] = f2_pack(xif[2 * h].y, xif[2 * h + 1].y);
        ipf.z[h] = f2_pack(xif[2 * h].z, xif[2 * h + 1].z);
    }
    // FP32 decisions are taken only outside +-margin of the thresholds
    const float mg     = g.list_margin;
    const float cut_lo = (float)g.cutneighsq - mg, cut_hi = (float)g.cutneighsq + mg;
    const float rbb_lo = (float)g.rbb_sq - mg, rbb_hi = (float)g.rbb_sq + mg;
    const float imnxf = (float)ibbmin[ci].x, imnyf = (float)ibbmin[ci].y;
    const float imxxf = (float)ibbmax[ci].x, imxyf = (float)ibbmax[ci].y;
    const float imnzf = (float)imnz, imxzf = (float)imxz;
    const double zx  = __longlong_as_double((long long)*zext);
    const double zlo = imnz - g.cutneigh - zx - 1.0e-6;
    // window of a column: the entries of buckets [qa, qb], a superset of those
    // with zlo <= bbminz <= imxz + cutneigh (zbucket is monotone); all others
    // fail the box test
    const int zn = g.zq + 2;
    const int qa = zbucket(g, zlo), qb1 = zbucket(g, imxz + g.cutneigh + 1.0e-6) + 1;
    const int ib     = cbin[ci];
    int* row         = list + (size_t)ci * cs;
    int total = 0, diag_pos = -1;
    for (int kb = 0; kb < g.nstencil; kb += 32) {
        const int k = kb + lane;
        int lo = 0, wn = 0;
        if (k < g.nstencil) {
            const int* zt = ztab + (size_t)(ib + stencil[k]) * zn;
            lo            = __ldg(&zt[qa]);
            const int hi  = __ldg(&zt[qb1]);
            wn            = hi > lo ? hi - lo : 0;
        }
        int incl = wn;
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        const int W     = __shfl_sync(0xffffffffu, incl, 31);
        s_lo[w][lane]   = lo;
        s_ws[w][lane]   = incl - wn;
        const bool expanded = W <= CP_LIST_EXPAND;
        if (expanded)
            for (int q = 0; q < wn; q++)
                s_m[w][incl - wn + q] = lo + q;
        __syncwarp();
        for (int t0 = 0; t0 < W; t0 += 32) {
            const int t = t0 + lane;
            bool ok     = false;
            int cj      = -1;
            if (t < W) {
                int m;
                if (expanded) {
                    m = s_m[w][t];
                } else {
                    int a = 0, z = 31; // last column whose window starts at or before t
                    while (a < z) {
                        int mid = (a + z + 1) >> 1;
                        if (s_ws[w][mid] <= t) a = mid;
                        else z = mid - 1;
                    }
                    m = s_lo[w][a] + (t - s_ws[w][a]);
                }
                cj          = jcol[m];
                if (!(half && ci_cj0 > cj)) {
                    float4 fn, fx;
                    ldg_pair4(&jcbbf[2 * m], fn, fx); // the box's min and max
                    float df = bb_axis_f(imnzf, imxzf, fn.z, fx.z);
                    df       = df * df;
                    float ef = bb_axis_f(imnyf, imxyf, fn.y, fx.y);
                    df += ef * ef;
                    ef = bb_axis_f(imnxf, imxxf, fn.x, fx.x);
                    df += ef * ef;
                    if (df <= cut_hi) {
                        bool in_cut = true, in_rbb = df < rbb_lo;
                        if (df >= cut_lo || (df >= rbb_lo && df <= rbb_hi))
                            in_cut = exact_box(&ibbmin[ci], &ibbmax[ci], &jcbbmin[m],
                                &jcbbmax[m], g.cutneighsq, g.rbb_sq, &in_rbb);
                        if (in_cut)
                            ok = in_rbb || any_pair_f<M, N>(ipf, cxf + (size_t)cj * N, cut_lo,
                                               cut_hi, cx + (size_t)ci * M,
                                               cx + (size_t)cj * N, g.cutneighsq);
                    }
                }
            }
            const unsigned bal = __ballot_sync(0xffffffffu, ok);
            if (ok) {
                const int p = total + __popc(bal & ((1u << lane) - 1u));
                if (p < maxneighs) row[(size_t)p * ks] = cj;
                if (cj == ci_cj0) diag_pos = p;
            }
            total += __popc(bal);
        }
        __syncwarp();
    }
    // the diagonal entry (mask != all) goes to the front, clusterpair/neighbor.c:599-649
    diag_pos = __reduce_max_sync(0xffffffffu, diag_pos);
    __syncwarp();
    if (lane == 0) {
        if (diag_pos > 0 && diag_pos < maxneighs) {
            int first                  = row[0];
            row[0]                     = row[(size_t)diag_pos * ks];
            row[(size_t)diag_pos * ks] = first;
        }
        numneigh[ci] = total < maxneighs ? total : maxneighs;
        nmasked[ci]  = diag_pos >= 0 ? 1 : 0;
        if (total >= maxneighs) atomicMax(&cnt[CP_MAXNEED], total);
    }
}

template <int M, int N>
__global__ void __launch_bounds__(32 * CP_LIST_WARPS, CP_LIST_MINB) k_build_list(int half, int* cnt, Geom g,
    const int* __restrict__ stencil,
    const int* __restrict__ cbin, const double4* __restrict__ ibbmin,
    const double4* __restrict__ ibbmax, const double4* __restrict__ jcbbmin,
    const double4* __restrict__ jcbbmax, const double4* __restrict__ cx,
    const float4* __restrict__ jcbbf, const float4* __restrict__ cxf,
    const int* __restrict__ jcol, const int* __restrict__ ztab,
    const unsigned long long* __restrict__ zext, int maxneighs, int ks, int cs, int* list,
    int* numneigh, int* nmasked)
{
    build_list_blk<M, N>(blockIdx.x, half, cnt, g, stencil, cbin, ibbmin, ibbmax, jcbbmin,
        jcbbmax, cx, jcbbf, cxf, jcol, ztab, zext, maxneighs, ks, cs, list, numneigh,
        nmasked);
}

void launch_build_list(cudaStream_t s, int M, int N, int half, int ncl_cap, const int* cnt,
    const Geom& g, const int* stencil, const int* cbin, const double4* ibbmin,
    const double4* ibbmax, const double4* jcbbmin, const double4* jcbbmax, const double4* cx,
    const float4* jcbbf, const float4* cxf, const int* jcol, const int* ztab,
    const unsigned long long* zext, int maxneighs, int ks, int cs, int* list, int* numneigh,
    int* nmasked, int* cnt_out)
{
    long long threads = (long long)ncl_cap * 32;
    int blocks        = mdb_blocks(threads, 32 * CP_LIST_WARPS);
    (void)M;
    (void)cnt;
    if (N == 4)
        k_build_list<4, 4><<<blocks, 32 * CP_LIST_WARPS, 0, s>>>(half, cnt_out, g, stencil, cbin,
            ibbmin, ibbmax, jcbbmin, jcbbmax, cx, jcbbf, cxf, jcol, ztab, zext, maxneighs,
            ks, cs, list, numneigh, nmasked);
    else
        k_build_list<4, 8><<<blocks, 32 * CP_LIST_WARPS, 0, s>>>(half, cnt_out, g, stencil, cbin,
            ibbmin, ibbmax, jcbbmin, jcbbmax, cx, jcbbf, cxf, jcol, ztab, zext, maxneighs,
            ks, cs, list, numneigh, nmasked);
    g_launches++;
}

// ---- pruneNeighborCPU (clusterpair/neighbor.c:1098-1264) -------------------------
// Entries are tested in parallel (any atom pair inside cutneigh, the SIMD
// builds' fma form over all M x N slots); lane 0 then replays the reference's
// compaction, which moves the last entry into each freed place.
template <int M, int N>
__global__ void k_prune(const int* __restrict__ cnt, const double4* __restrict__ cx,
    double cutneighsq, int maxneighs, int ks, int cs, int* list, int* numneigh, int* nmasked)
{
    extern __shared__ unsigned char s_flags_raw[];
    const int w    = threadIdx.x >> 5;
    const int ci   = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = lane_id();
    if (ci >= cnt[CP_NCL]) return;
    const int nn = numneigh[ci];
    unsigned char* flag = s_flags_raw + (size_t)w * maxneighs;
    double3 xi[M];
#pragma unroll
    for (int a = 0; a < M; a++) {
        double4 p = cx[ci * M + a];
        xi[a]     = make_double3(p.x, p.y, p.z);
    }
    int* row = list + (size_t)ci * cs;
    for (int k = lane; k < nn; k += 32) {
        int cj  = row[(size_t)k * ks];
        flag[k] = any_pair<M, N>(xi, cx + (size_t)cj * N, cutneighsq) ? 1 : 0;
    }
    __syncwarp();
    if (lane == 0) {
        int n = nn, nm = nmasked[ci], k = 0;
        while (k < n) {
            if (flag[k]) {
                k++;
            } else {
                n--;
                if (k < nm) nm--;
                row[(size_t)k * ks] = row[(size_t)n * ks];
                flag[k]                   = flag[n];
            }
        }
        numneigh[ci] = n;
        nmasked[ci]  = nm;
    }
}

void launch_prune(cudaStream_t s, int M, int N, int ncl_cap, const int* cnt, const double4* cx,
    double cutneighsq, int maxneighs, int ks, int cs, int* list, int* numneigh, int* nmasked)
{
    (void)M;
    // one flag byte per list entry and warp (the caller keeps maxneighs
    // below 12,288 so that 4 warps fit in 48 KB)
    long long threads = (long long)ncl_cap * 32;
    int blocks        = mdb_blocks(threads, 128);
    size_t smem       = 4 * (size_t)maxneighs;
    if (N == 4)
        k_prune<4, 4><<<blocks, 128, smem, s>>>(cnt, cx, cutneighsq, maxneighs, ks, cs, list,
            numneigh, nmasked);
    else
        k_prune<4, 8><<<blocks, 128, smem, s>>>(cnt, cx, cutneighsq, maxneighs, ks, cs, list,
            numneigh, nmasked);
    g_launches++;
}

// ---- batched rebuild over the members of an ensemble ------------------------------
// Each stage runs the single-member block bodies above; block b of a launch is
// block bmap[b].y of member bmap[b].x.
int cp_build_stage_blocks(int stage, const CpBuildMember& m, int* threads)
{
    const int T = MDB_NTHREADS, mb1 = m.g.mbins + 1;
    *threads    = T;
    switch (stage) {
    case CB_RESET: return mdb_blocks(mb1, T);
    case CB_GATHER: return mdb_blocks((long long)m.ncl_cap * m.M, T);
    case CB_BIN:
    case CB_SCATTER: return m.nlocal > 0 ? mdb_blocks(m.nlocal, T) : 0;
    case CB_SORT: *threads = 32 * CP_SORT_WARPS; return mdb_blocks(m.g.mbins, CP_SORT_WARPS);
    case CB_CLUSTERS: *threads = 128; return mdb_blocks((long long)m.g.mbins * 32, 128);
    case CB_GCOUNT:
    case CB_GWRITE: return mdb_blocks(m.ncj_cap, T);
    case CB_GFIRST: return mdb_blocks(m.ngc_cap + 1, T);
    case CB_GCOLS:
    case CB_GSCATTER: return mdb_blocks(m.ngc_cap, T);
    case CB_CSIZES: return mdb_blocks(mb1, T);
    case CB_MERGE: *threads = 128; return mdb_blocks((long long)mb1 * 32, 128);
    case CB_PREP: return mdb_blocks(list_prep_threads(m.g, m.slot_cap), T);
    case CB_LIST:
        *threads = 32 * CP_LIST_WARPS;
        return mdb_blocks((long long)m.ncl_cap * 32, 32 * CP_LIST_WARPS);
    }
    return 0;
}

__device__ __forceinline__ void reset_blk(int bid, const CpBuildMember& m)
{
    const int t = bid * blockDim.x + threadIdx.x;
    if (t <= m.g.mbins) {
        m.col_count[t]  = 0;
        m.col_fill[t]   = 0;
        m.ncl_col[t]    = 0;
        m.gcol_count[t] = 0;
        m.gfill[t]      = 0;
    }
    if (t == 0) {
        *m.zext                  = 0ull;
        m.cnt[CP_MAXNEED]        = 0;
        m.cnt[CP_BADBIN]         = 0;
        m.cnt[CP_NGHOST_ATOMS]   = 0;
    }
}

// only: null, or a flag per member (the members whose flag is 0 skip the stage)
template <int STAGE>
__global__ void __launch_bounds__(256, STAGE == CB_LIST ? 3 : 1)
    k_build_stage_batch(const CpBuildMember* __restrict__ tab,
    const int2* __restrict__ bmap, const int* __restrict__ only)
{
    const int2 bm          = __ldg(&bmap[blockIdx.x]);
    if (only && !only[bm.x]) return;
    const CpBuildMember& m = tab[bm.x];
    const int b            = bm.y;
    switch (STAGE) {
    case CB_RESET: reset_blk(b, m); break;
    case CB_GATHER:
        gather_blk(b, m.M, m.cnt, m.cx, m.cv, m.cl_first, m.ax, m.av, 1, m.g.xprd, m.g.yprd,
            m.g.zprd);
        break;
    case CB_BIN: bin_atoms_blk(b, m.nlocal, m.ax, m.g, m.atom_col, m.col_count, m.cnt); break;
    case CB_SCATTER:
        scatter_atoms_blk(b, m.nlocal, m.atom_col, m.col_start, m.col_fill, m.col_atoms);
        break;
    case CB_SORT:
        sort_columns_blk(b, m.g.mbins, m.M, m.N, m.col_start, m.col_atoms, m.ax, m.col_sorted,
            m.gidx, m.gz, m.ncl_col);
        break;
    case CB_CLUSTERS:
        if (m.N == 4)
            build_clusters_blk<4, 4>(b, m.g.mbins, m.mixed, m.col_start, m.col_sorted,
                m.cl_start, m.ax, m.av, m.cx, m.cv, m.inat, m.cbin, m.cl_first, m.ibbmin,
                m.ibbmax, m.jnat, m.jbbmin, m.jbbmax, m.anchor, m.xr, m.cnt, m.zext);
        else
            build_clusters_blk<4, 8>(b, m.g.mbins, m.mixed, m.col_start, m.col_sorted,
                m.cl_start, m.ax, m.av, m.cx, m.cv, m.inat, m.cbin, m.cl_first, m.ibbmin,
                m.ibbmax, m.jnat, m.jbbmin, m.jbbmax, m.anchor, m.xr, m.cnt, m.zext);
        break;
    case CB_GCOUNT:
        ghost_count_blk(b, m.ncj_cap, m.cnt, m.jnat, m.jbbmin, m.jbbmax, m.g, m.gcount);
        break;
    case CB_GWRITE:
        ghost_write_blk(b, m.ncj_cap, m.ngc_cap, m.cnt, m.jnat, m.jbbmin, m.jbbmax, m.g, m.gstart,
            m.border, m.pbc);
        break;
    case CB_GFIRST:
        ghost_first_blk(b, m.N, m.cnt, m.border, m.pbc, m.mixed, m.g, m.cx, m.jnat, m.jbbmin,
            m.jbbmax, m.anchor, m.xr, m.zext);
        break;
    case CB_GCOLS:
        ghost_columns_blk(b, m.N, m.cnt, m.pbc, m.jnat, m.cx, m.g, m.gcolumn, m.gcol_count);
        break;
    case CB_CSIZES:
        column_sizes_blk(b, m.g.mbins + 1, m.jfac, m.ncl_col, m.gcol_count, m.jcol_n);
        break;
    case CB_GSCATTER:
        ghost_scatter_blk(b, m.cnt, m.gcolumn, m.jcol_start, m.ncl_col, m.jfac, m.gfill, m.gtmp);
        break;
    case CB_MERGE:
        merge_columns_blk(b, m.g.mbins + 1, m.jfac, m.ncl_col, m.cl_start, m.gcol_count,
            m.jcol_start, m.gtmp, m.jbbmin, m.jbbmax, m.jcol, m.jcbbmin, m.jcbbmax);
        break;
    case CB_LIST:
        if (m.N == 4)
            build_list_blk<4, 4>(b, m.half, m.cnt, m.g, m.stencil, m.cbin, m.ibbmin, m.ibbmax,
                m.jcbbmin, m.jcbbmax, m.cx, m.jcbbf, m.cxf, m.jcol, m.ztab, m.zext,
                m.maxneighs, m.ks, m.cs, m.list, m.numneigh, m.nmasked);
        else
            build_list_blk<4, 8>(b, m.half, m.cnt, m.g, m.stencil, m.cbin, m.ibbmin, m.ibbmax,
                m.jcbbmin, m.jcbbmax, m.cx, m.jcbbf, m.cxf, m.jcol, m.ztab, m.zext,
                m.maxneighs, m.ks, m.cs, m.list, m.numneigh, m.nmasked);
        break;
    case CB_PREP:
        list_prep_blk(b, m.N, m.slot_cap, m.g, m.cnt, m.jcol_start, m.jcbbmin, m.jcbbmax, m.cx,
            m.jcbbf, m.cxf, m.ztab);
        break;
    }
}

void launch_build_stage_batch(cudaStream_t s, int stage, int nblocks, const CpBuildMember* tab,
    const int2* bmap, const int* only)
{
    if (nblocks <= 0) return;
    CpBuildMember probe{};
    probe.M = 4, probe.N = 4;
    int T = 0;
    cp_build_stage_blocks(stage, probe, &T);
    switch (stage) {
#define CP_STAGE(S)                                                                      \
    case S: k_build_stage_batch<S><<<nblocks, T, 0, s>>>(tab, bmap, only); break;
        CP_STAGE(CB_RESET)
        CP_STAGE(CB_GATHER)
        CP_STAGE(CB_BIN)
        CP_STAGE(CB_SCATTER)
        CP_STAGE(CB_SORT)
        CP_STAGE(CB_CLUSTERS)
        CP_STAGE(CB_GCOUNT)
        CP_STAGE(CB_GWRITE)
        CP_STAGE(CB_GFIRST)
        CP_STAGE(CB_GCOLS)
        CP_STAGE(CB_CSIZES)
        CP_STAGE(CB_GSCATTER)
        CP_STAGE(CB_MERGE)
        CP_STAGE(CB_PREP)
        CP_STAGE(CB_LIST)
#undef CP_STAGE
    default: return;
    }
    g_launches++;
}

// exclusive scan of one member's array by one block of 1024 threads (4 items
// per thread per pass), out[n] = total
#define CP_SCAN_T 1024
__global__ void __launch_bounds__(CP_SCAN_T) k_scan_batch(const CpBuildMember* __restrict__ tab,
    int which, const int* __restrict__ only)
{
    __shared__ int s_w[CP_SCAN_T / 32];
    if (only && !only[blockIdx.x]) return;
    const CpBuildMember& m = tab[blockIdx.x];
    const int* in;
    int* out;
    int n;
    switch (which) {
    case 0: in = m.col_count, out = m.col_start, n = m.g.mbins; break;
    case 1: in = m.ncl_col, out = m.cl_start, n = m.g.mbins + 1; break;
    case 2: in = m.gcount, out = m.gstart, n = m.ncj_cap; break;
    default: in = m.jcol_n, out = m.jcol_start, n = m.g.mbins + 1; break;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int carry = 0;
    for (int base = 0; base < n; base += 4 * CP_SCAN_T) {
        const int i0 = base + 4 * threadIdx.x;
        int v[4], t = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            v[k] = i0 + k < n ? in[i0 + k] : 0;
            t += v[k];
        }
        int inc = t;
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += u;
        }
        if (lane == 31) s_w[w] = inc;
        __syncthreads();
        if (w == 0) {
            int x = s_w[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += u;
            }
            s_w[lane] = x;
        }
        __syncthreads();
        int run = carry + (w > 0 ? s_w[w - 1] : 0) + inc - t;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (i0 + k < n) out[i0 + k] = run;
            run += v[k];
        }
        carry += s_w[CP_SCAN_T / 32 - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[n] = carry;
}

void launch_scan_batch(cudaStream_t s, int which, int nmem, const CpBuildMember* tab,
    const int* only)
{
    if (nmem <= 0) return;
    k_scan_batch<<<nmem, CP_SCAN_T, 0, s>>>(tab, which, only);
    g_launches++;
}

__global__ void k_counters_batch(const CpBuildMember* __restrict__ tab, int* out)
{
    if (threadIdx.x < CP_SLOTS) out[blockIdx.x * CP_SLOTS + threadIdx.x] = tab[blockIdx.x].cnt[threadIdx.x];
}

// the displacement check's reference positions (slots as built) of the
// members whose flag is set, over the integrator's block map
__global__ void k_snapshot_batch(const CpStepMember* __restrict__ tab,
    const int2* __restrict__ bmap, const int* __restrict__ only)
{
    const int2 bm = __ldg(&bmap[blockIdx.x]);
    if (bm.x < 0 || !only[bm.x]) return;
    const CpStepMember& m = tab[bm.x];
    const int k           = bm.y * blockDim.x + threadIdx.x;
    if (m.xb && k < m.cnt[CP_NCL] * m.M) const_cast<double4*>(m.xb)[k] = m.cx[k];
}

void launch_snapshot_batch(cudaStream_t s, int nblocks, const CpStepMember* tab,
    const int2* bmap, const int* only)
{
    if (nblocks <= 0) return;
    k_snapshot_batch<<<nblocks, MDB_NTHREADS, 0, s>>>(tab, bmap, only);
    g_launches++;
}

void launch_counters_batch(cudaStream_t s, int nmem, const CpBuildMember* tab, int* out)
{
    if (nmem <= 0) return;
    k_counters_batch<<<nmem, 32, 0, s>>>(tab, out);
    g_launches++;
}

} // namespace cp
} // namespace mdb
