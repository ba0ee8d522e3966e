// mdb_kinetic_sum_noalloc: the thermo velocity reduction for callers that own
// their device buffers and cannot allocate device memory.
//
// Who needs it: code that keeps its own MD state on the GPU and may not let a
// library allocate device memory - a framework whose caching allocator or
// memory pool has reserved the device's memory up front (a cudaMalloc from
// here would fail or fragment that pool), a timed or latency-critical loop
// in which cudaMalloc / cudaFree would synchronise the device, or a plugin
// host that forbids its libraries to own device memory. mdb_thermo needs a
// context, and creating a context allocates; this entry point only reads the
// caller's velocities and writes the caller's output.
//
// Scratch: the per-block partial sums live in a file-scope __device__ array of
// NOALLOC_MAX_PARTIALS doubles (32 KiB on every device that loads this
// library, held until the process exits). One partial covers a fixed chunk of
// NOALLOC_CHUNK atoms, so a call accepts at most
// NOALLOC_MAX_PARTIALS * NOALLOC_CHUNK = 8,388,608 atoms and rejects more.
// Host code must not pass the array's name to a kernel (in host code it is a
// host-side shadow, not a device address): the device address is looked up
// with cudaGetSymbolAddress, with the device current, once per device and
// CUDA context, and cached. The cache is keyed on the current context as well
// as the device number, so a call made under another context of the same
// device (a driver-API context that is not the primary one, or the new
// primary context after cudaDeviceReset) looks the address up again instead
// of using one that belongs to a module of a context that is gone. Such a
// look-up is part of that call: make the first call under each context before
// any stream capture.
#include <stdio.h>

#include <mutex>

#include "mdb_internal.cuh"

namespace {

constexpr int NOALLOC_CHUNK        = 2048; // atoms per partial (one block of 256 threads)
constexpr int NOALLOC_MAX_PARTIALS = 4096;
constexpr int NOALLOC_THREADS      = 256;
constexpr int NOALLOC_MAX_DEVICES  = 64;

static __device__ __align__(256) double g_noalloc_partials[NOALLOC_MAX_PARTIALS];

std::mutex g_noalloc_lock;
struct ScratchAddr {
    void* ctx    = nullptr; // the CUDA context the address belongs to
    double* addr = nullptr;
};
ScratchAddr g_noalloc_addr[NOALLOC_MAX_DEVICES];

// cuCtxGetCurrent through the runtime's driver entry point (no link-time
// dependency on the driver library)
typedef int (*CtxGetCurrentFn)(void** pctx);

static int current_context(void** ctx)
{
    static CtxGetCurrentFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !p)
            return -1;
        fn = reinterpret_cast<CtxGetCurrentFn>(p);
    }
    return fn(ctx) == 0 && *ctx ? 0 : -1;
}

// Each block sums (vx^2 + vy^2 + vz^2) * mass over its chunk of AoS velocities
// (verletlist/atom.h:78-88 layout) and writes one partial; every partial slot
// in [0, nparts) is written by this launch, so nothing needs clearing.
__global__ void __launch_bounds__(NOALLOC_THREADS) k_ke_chunks(const double* __restrict__ v,
    int n, double mass, double* __restrict__ partials)
{
    double t   = 0.0;
    long long b = (long long)blockIdx.x * NOALLOC_CHUNK;
    for (int k = threadIdx.x; k < NOALLOC_CHUNK; k += blockDim.x) {
        long long i = b + k;
        if (i < n) {
            double a = v[3 * i], c = v[3 * i + 1], d = v[3 * i + 2];
            t += (a * a + c * c + d * d) * mass;
        }
    }
    t = mdb::block_sum(t);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

__global__ void __launch_bounds__(1024) k_ke_final(const double* __restrict__ partials,
    int nparts, double* __restrict__ out)
{
    double t = 0.0;
    for (int k = threadIdx.x; k < nparts; k += blockDim.x)
        t += partials[k];
    t = mdb::block_sum(t);
    if (threadIdx.x == 0) *out = t;
}

} // namespace

extern "C" int mdb_kinetic_sum_noalloc(const double* d_v, int n, double mass, double* d_out,
    void* stream)
{
    if (n < 0 || !d_out || (n > 0 && !d_v)) return MDB_ERR_ARG;
    if ((long long)n > (long long)NOALLOC_MAX_PARTIALS * NOALLOC_CHUNK) {
        fprintf(stderr,
            "mdb_kinetic_sum_noalloc: %d atoms exceed the static scratch capacity of %d atoms\n",
            n, NOALLOC_MAX_PARTIALS * NOALLOC_CHUNK);
        return MDB_ERR_ARG;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES)
        return MDB_ERR_CUDA;
    // no current context yet (a caller whose first runtime call this is): the
    // symbol look-up below makes the device's primary context current
    void* ctx = nullptr;
    if (current_context(&ctx) != 0) ctx = nullptr;
    double* scratch = nullptr;
    {
        // once per device and context, with that device current: the device
        // address of the static array (the first call under a context does
        // this look-up, so make that call before any stream capture)
        std::lock_guard<std::mutex> lock(g_noalloc_lock);
        ScratchAddr& c = g_noalloc_addr[dev];
        if (!ctx || !c.addr || c.ctx != ctx) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_partials) != cudaSuccess || !p)
                return MDB_ERR_CUDA;
            if (!ctx && current_context(&ctx) != 0) return MDB_ERR_CUDA;
            c.addr = static_cast<double*>(p);
            c.ctx  = ctx;
        }
        scratch = c.addr;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int nparts     = n > 0 ? (n + NOALLOC_CHUNK - 1) / NOALLOC_CHUNK : 1;
    k_ke_chunks<<<nparts, NOALLOC_THREADS, 0, s>>>(d_v, n, mass, scratch);
    k_ke_final<<<1, 1024, 0, s>>>(scratch, nparts, d_out);
    mdb::g_launches += 2;
    return cudaGetLastError() == cudaSuccess ? MDB_OK : MDB_ERR_CUDA;
}
