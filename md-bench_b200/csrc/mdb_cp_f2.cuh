// Packed two-lane FP32 arithmetic and the reduction helpers shared by the
// mixed cluster-pair force kernels (mdb_cp_force.cu, mdb_cp_pairs.cu).
#pragma once

#include <cuda_runtime.h>

namespace mdb {
namespace cp {

// one vector reduction (red.global.add.v4.f32, sm_90+) instead of three
// scalar atomics for a force update
__device__ __forceinline__ void red_add4(float4* dst, float x, float y, float z)
{
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(dst), "f"(x), "f"(y),
                 "f"(z), "f"(0.0f)
                 : "memory");
}

// two consecutive float4 in one 256-bit load (sm_100); p 32-byte aligned
__device__ __forceinline__ void ldg_pair4(const float4* p, float4& a, float4& b)
{
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z),
          "=f"(b.w)
        : "l"(p));
}

// PTX rcp.approx.ftz.f32: at most 1 ulp from 1/x, one MUFU operation
__device__ __forceinline__ float rcp_approx(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Packed FP32 pairs: sm_100 executes add/sub/mul/fma on two f32 lanes of a
// 64-bit register in one instruction (PTX .f32x2), so each thread carries its
// 4 i atoms as two packed pairs (atoms 0,1 and 2,3) and computes two pairs per
// instruction.
typedef unsigned long long f2;

__device__ __forceinline__ f2 f2_pack(float lo, float hi)
{
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void f2_unpack(f2 v, float& lo, float& hi)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f2 f2_add(f2 a, f2 b)
{
    f2 r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f2 f2_sub(f2 a, f2 b)
{
    f2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f2 f2_mul(f2 a, f2 b)
{
    f2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f2 f2_fma(f2 a, f2 b, f2 c)
{
    f2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}

} // namespace cp
} // namespace mdb
