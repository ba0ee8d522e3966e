// mdb_fp32_fma_rate: the device's packed FP32 FMA throughput, measured.
//
// The mixed cluster-pair force kernels evaluate their pair forces with packed
// two-lane FP32 instructions (fma.rn.f32x2 and friends), so the roofline that
// bounds them is the FP32 pipe's. No library routine reports that rate, and a
// figure derived from the clock assumes a lane count; this entry point
// measures it instead: every thread of a grid that fills all SMs runs eight
// independent chains of packed FMAs (two FMAs, four flops, per instruction),
// timed with CUDA events on a stream of its own after a warm-up launch. The
// result is the best of several launches, in FP32 flops per second.
#include <cuda_runtime.h>

#include "mdb.h"
#include "mdb_cp_f2.cuh"

namespace {

using mdb::cp::f2;
using mdb::cp::f2_fma;
using mdb::cp::f2_pack;
using mdb::cp::f2_unpack;

constexpr int PROBE_CHAINS  = 8;
constexpr int PROBE_THREADS = 256;

// a = a * m + c on PROBE_CHAINS independent packed chains; m and c keep the
// values bounded (|m| < 1), the sum written at the end keeps the work alive
__global__ void __launch_bounds__(PROBE_THREADS) k_fp32_fma_chains(int iters, float m, float c,
    float* out)
{
    f2 a[PROBE_CHAINS];
#pragma unroll
    for (int k = 0; k < PROBE_CHAINS; k++)
        a[k] = f2_pack(0.001f * (threadIdx.x + k), 0.002f * (blockIdx.x + k));
    const f2 M = f2_pack(m, m), C = f2_pack(c, c);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < PROBE_CHAINS; k++) a[k] = f2_fma(a[k], M, C);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < PROBE_CHAINS; k++) {
        float lo, hi;
        f2_unpack(a[k], lo, hi);
        s += lo + hi;
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

} // namespace

extern "C" int mdb_fp32_fma_rate(int device, double* flops_per_s)
{
    if (!flops_per_s) return MDB_ERR_ARG;
    *flops_per_s = 0.0;
    cudaError_t e = cudaSetDevice(device);
    int sms = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess || sms < 1) return MDB_ERR_CUDA;
    // 8 resident blocks of 256 threads per SM (64 warps), 4 waves
    const int blocks = sms * 8 * 4, iters = 4096;
    float* out       = nullptr;
    cudaStream_t s   = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if ((e = cudaMalloc((void**)&out, sizeof(float) * blocks * PROBE_THREADS)) == cudaSuccess &&
        (e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) == cudaSuccess &&
        (e = cudaEventCreate(&e0)) == cudaSuccess && (e = cudaEventCreate(&e1)) == cudaSuccess) {
        double best = 0.0;
        for (int rep = 0; rep < 6 && e == cudaSuccess; rep++) {
            cudaEventRecord(e0, s);
            k_fp32_fma_chains<<<blocks, PROBE_THREADS, 0, s>>>(iters, 0.999f, 0.001f, out);
            cudaEventRecord(e1, s);
            e = cudaEventSynchronize(e1);
            float ms = 0.f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            // rep 0 is the warm-up
            if (e == cudaSuccess && rep > 0 && ms > 0.f) {
                const double flops =
                    (double)blocks * PROBE_THREADS * iters * PROBE_CHAINS * 2.0 * 2.0;
                if (flops / (ms * 1e-3) > best) best = flops / (ms * 1e-3);
            }
        }
        *flops_per_s = best;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    if (out) cudaFree(out);
    return e == cudaSuccess ? MDB_OK : MDB_ERR_CUDA;
}
