// Device-wide exclusive prefix sum over int32 (three passes: tile sums,
// scan of tile sums, tile rescan with offsets). Used for the ghost-map
// offsets (one count per local atom) and for the bin CSR (one count per bin).
#include "mdb_internal.cuh"

namespace mdb {

static constexpr int SCAN_THREADS = 1024;
static constexpr int SCAN_ITEMS   = 4;
static constexpr int SCAN_TILE    = SCAN_THREADS * SCAN_ITEMS;

int scan_scratch_ints(int n) { return (n + SCAN_TILE - 1) / SCAN_TILE + 1; }

// Inclusive block scan of one value per thread; returns the inclusive prefix,
// *total receives the block sum.
__device__ __forceinline__ int block_inclusive_scan(int v, int* total)
{
    __shared__ int warp_sums[SCAN_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    if (lane == 31) warp_sums[warp] = v;
    __syncthreads();
    if (warp == 0) {
        int w = (lane < (int)(blockDim.x >> 5)) ? warp_sums[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        warp_sums[lane] = w;
    }
    __syncthreads();
    int prefix = warp > 0 ? warp_sums[warp - 1] : 0;
    *total     = warp_sums[(blockDim.x >> 5) - 1];
    __syncthreads();
    return v + prefix;
}

__global__ void k_scan_tiles(const int* __restrict__ in, int n, int* __restrict__ tile_sums)
{
    long long base = (long long)blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    int s          = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++)
        if (base + k < n) s += in[base + k];
    int total;
    block_inclusive_scan(s, &total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// One block: exclusive scan of the tile sums in place; tile_sums[ntiles] = total.
__global__ void k_scan_tile_sums(int* tile_sums, int ntiles)
{
    int carry = 0;
    for (int base = 0; base < ntiles; base += SCAN_THREADS) {
        int idx = base + threadIdx.x;
        int v   = idx < ntiles ? tile_sums[idx] : 0;
        int total;
        int inc = block_inclusive_scan(v, &total);
        if (idx < ntiles) tile_sums[idx] = carry + inc - v;
        carry += total;
    }
    if (threadIdx.x == 0) tile_sums[ntiles] = carry;
}

__global__ void k_scan_apply(const int* __restrict__ in, int* __restrict__ out, int n,
    const int* __restrict__ tile_sums, int ntiles)
{
    long long base = (long long)blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    int s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        v[k] = (base + k < n) ? in[base + k] : 0;
        s += v[k];
    }
    int total;
    int inc  = block_inclusive_scan(s, &total);
    int run  = tile_sums[blockIdx.x] + inc - s;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = tile_sums[ntiles];
}

void scan_exclusive(const int* in, int* out, int n, int* scratch, cudaStream_t s)
{
    int ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (ntiles == 0) ntiles = 1;
    k_scan_tiles<<<ntiles, SCAN_THREADS, 0, s>>>(in, n, scratch);
    k_scan_tile_sums<<<1, SCAN_THREADS, 0, s>>>(scratch, ntiles);
    k_scan_apply<<<ntiles, SCAN_THREADS, 0, s>>>(in, out, n, scratch, ntiles);
    g_launches += 3;
}

} // namespace mdb
