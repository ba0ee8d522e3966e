// Cluster-pair scheme: Lennard-Jones forces (FP64 reference-exact and FP32
// mixed), the cluster-layout integrator and the thermo partial sums.
#include <math.h>

#include <algorithm>

#include "mdb_cp_f2.cuh"
#include "mdb_cp_internal.cuh"

namespace mdb {
namespace cp {

#define CP_FORCE_THREADS 128

int force_blocks(int ncl_cap)
{
    // the FP64 kernel runs one thread per slot, the mixed one a warp per
    // i-cluster; both size their partial-energy arrays by this count
    long long t = (long long)ncl_cap * 32;
    return mdb_blocks(t, CP_FORCE_THREADS);
}

// ---- FP64: computeForceLJRef (clusterpair/force_lj.c:23-189) -----------------
// One thread per i slot. For each list entry the sum over the N j atoms is
// formed first and then added to the atom's force, exactly the reference's
// order, so full-list forces are bit-identical. Self pairs (and, for half
// lists, the lower triangle) of the diagonal entry are excluded by cluster
// index as the reference does; half lists subtract the reaction from local j
// slots with atomics (the reference drops ghost reactions: without MPI its
// reverse communication does nothing).
template <int M, int N, bool HALF, bool ENERGY>
__global__ void __launch_bounds__(CP_FORCE_THREADS) k_force_fp64(const int* __restrict__ cnt,
    const double4* __restrict__ cx, Types ty, double cutforcesq, const int* __restrict__ list,
    int ks, int cs, const int* __restrict__ numneigh, double4* cf, double* epart)
{
    __shared__ double s_se[MDB_MAX_TYPES], s_s3[MDB_MAX_TYPES];
    if (threadIdx.x < MDB_MAX_TYPES) {
        s_se[threadIdx.x] = ty.sqrt_eps[threadIdx.x];
        s_s3[threadIdx.x] = ty.sigma3[threadIdx.x];
    }
    __syncthreads();
    const int s    = blockIdx.x * blockDim.x + threadIdx.x;
    const int ncl  = cnt[CP_NCL];
    const int nloc = ncl * M; // local slots (= ncj * N)
    double epot    = 0.0;
    if (s < nloc) {
        const double4 pi = cx[s];
        const int ti     = slot_type(pi);
        if (ti >= 0) {
            const int ci = s / M, a = s - ci * M;
            const int ci_cj0 = ci / (N / M);
            const int ai     = a + M * (ci % (N / M));
            const double se_i = s_se[ti], s3_i = s_s3[ti];
            double fx = 0.0, fy = 0.0, fz = 0.0;
            const int nn = numneigh[ci];
            for (int k = 0; k < nn; k++) {
                const int cj = __ldg(&list[(size_t)k * ks + (size_t)ci * cs]);
                double fix = 0.0, fiy = 0.0, fiz = 0.0;
#pragma unroll
                for (int b = 0; b < N; b++) {
                    const bool cond = HALF ? (ci_cj0 != cj || ai < b) : (ci_cj0 != cj || ai != b);
                    if (!cond) continue;
                    const int sj     = cj * N + b;
                    const double4 pj = ldg4(&cx[sj]);
                    const double delx = pi.x - pj.x;
                    const double dely = pi.y - pj.y;
                    const double delz = pi.z - pj.z;
                    const double rsq  = delx * delx + dely * dely + delz * delz;
                    if (rsq < cutforcesq) {
                        int tj            = slot_type(pj);
                        tj                = tj < 0 ? 0 : tj;
                        const double sig6 = s3_i * s_s3[tj];
                        const double eps  = se_i * s_se[tj];
                        const double sr2  = 1.0 / rsq;
                        const double sr6  = sr2 * sr2 * sr2 * sig6;
                        const double force = 48.0 * sr6 * (sr6 - 0.5) * sr2 * eps;
                        if (HALF && sj < nloc) {
                            atomicAdd(&cf[sj].x, -(delx * force));
                            atomicAdd(&cf[sj].y, -(dely * force));
                            atomicAdd(&cf[sj].z, -(delz * force));
                        }
                        fix += delx * force;
                        fiy += dely * force;
                        fiz += delz * force;
                        if (ENERGY) {
                            double e = 4.0 * eps * sr6 * (sr6 - 1.0);
                            epot += (HALF && sj < nloc) ? e : 0.5 * e;
                        }
                    }
                }
                fx += fix;
                fy += fiy;
                fz += fiz;
            }
            if (HALF) {
                atomicAdd(&cf[s].x, fx);
                atomicAdd(&cf[s].y, fy);
                atomicAdd(&cf[s].z, fz);
            } else {
                cf[s] = make_double4(fx, fy, fz, 0.0);
            }
        }
    }
    if (ENERGY) {
        double t = block_sum(epot);
        if (threadIdx.x == 0) epart[blockIdx.x] = t;
    }
}

template <int N, bool HALF, bool ENERGY>
static void run_fp64(cudaStream_t s, int blocks, const int* cnt, const double4* cx,
    const Types& ty, double cutforcesq, const int* list, int ks, int cs, const int* numneigh,
    double4* cf, double* epart)
{
    k_force_fp64<4, N, HALF, ENERGY><<<blocks, CP_FORCE_THREADS, 0, s>>>(cnt, cx, ty, cutforcesq,
        list, ks, cs, numneigh, cf, epart);
}

void launch_force_fp64(cudaStream_t s, int M, int N, int half, int energy, int ncl_cap,
    const int* cnt, const double4* cx, const Types& ty, double cutforcesq, const int* list,
    int ks, int cs, const int* numneigh, double4* cf, double* epart)
{
    (void)M;
    // one thread per slot: ncl_cap * 4 threads; energy partials sized by
    // force_blocks (ncl_cap * 32 threads) cover it
    int blocks = mdb_blocks((long long)ncl_cap * 4, CP_FORCE_THREADS);
    if (N == 4) {
        if (half) energy ? run_fp64<4, true, true>(s, blocks, cnt, cx, ty, cutforcesq, list, ks, cs, numneigh, cf, epart)
                         : run_fp64<4, true, false>(s, blocks, cnt, cx, ty, cutforcesq, list, ks, cs, numneigh, cf, epart);
        else energy ? run_fp64<4, false, true>(s, blocks, cnt, cx, ty, cutforcesq, list, ks, cs, numneigh, cf, epart)
                    : run_fp64<4, false, false>(s, blocks, cnt, cx, ty, cutforcesq, list, ks, cs, numneigh, cf, epart);
    } else {
        if (half) energy ? run_fp64<8, true, true>(s, blocks, cnt, cx, ty, cutforcesq, list, ks, cs, numneigh, cf, epart)
                         : run_fp64<8, true, false>(s, blocks, cnt, cx, ty, cutforcesq, list, ks, cs, numneigh, cf, epart);
        else energy ? run_fp64<8, false, true>(s, blocks, cnt, cx, ty, cutforcesq, list, ks, cs, numneigh, cf, epart)
                    : run_fp64<8, false, false>(s, blocks, cnt, cx, ty, cutforcesq, list, ks, cs, numneigh, cf, epart);
    }
    g_launches++;
}

// ---- mixed: FP32 pair forces on anchor-relative coordinates ------------------------
// One warp per i-cluster (M = 4 atoms, held by every lane). The warp takes
// 32 / N list entries at a time; lane (e, b) owns atom b of entry e and
// computes its pairs with the 4 i atoms. Positions are relative to per-cluster
// anchors on a 1/8 grid: the anchor difference is exact in FP32 and is added
// to the j position once per entry. Full lists reduce the i forces across the
// warp once per i-cluster; half lists also accumulate each j atom's reaction
// over the 4 i atoms in the lane and add it with one atomic per component.
// Padding slots sit at +1e18 (j) and invalid i atoms are moved to -1e18, so
// they fall outside the cutoff without INF arithmetic.
// Sum of 12 partial sums over the L lanes of one i-cluster's segment (l =
// the lane's index in it). Transpose-reduce: after the xor-L/2 and xor-L/4
// steps each lane holds 3 partial sums of i atom l / (L/4); plain xor steps
// L/8 .. 1 finish them.
template <int L>
__device__ __forceinline__ void seg_reduce_12(float (&v)[12], int l)
{
    float h[6];
    const bool up = l & (L / 2);
#pragma unroll
    for (int i = 0; i < 6; i++) {
        float send = up ? v[i] : v[i + 6];
        float keep = up ? v[i + 6] : v[i];
        h[i]       = keep + __shfl_xor_sync(0xffffffffu, send, L / 2);
    }
    float q[3];
    const bool up2 = l & (L / 4);
#pragma unroll
    for (int i = 0; i < 3; i++) {
        float send = up2 ? h[i] : h[i + 3];
        float keep = up2 ? h[i + 3] : h[i];
        q[i]       = keep + __shfl_xor_sync(0xffffffffu, send, L / 4);
    }
#pragma unroll
    for (int o = L / 8; o > 0; o >>= 1)
#pragma unroll
        for (int i = 0; i < 3; i++)
            q[i] += __shfl_xor_sync(0xffffffffu, q[i], o);
    v[0] = q[0];
    v[1] = q[1];
    v[2] = q[2];
}

// The i side of one i-cluster: coordinates and type parameters of atoms
// (0,1) and (2,3) packed.
struct IPack {
    f2 x[2], y[2], z[2];
    f2 se[2], s3[2];
};

// Pairs of one j atom with the 4 i atoms, two per packed instruction. With
// u = 1/r^2 (0 outside the cutoff) and s = sigma^6, the LJ force over r is
// 48 eps s u^4 (s u^3 - 1/2) = u^4 (A u^3 - B), A = 48 eps s^2, B = 24 eps s,
// for uniform types. The i forces accumulate in fx/fy/fz (packed like the i
// atoms); half lists also accumulate sum(d * force) for the j atom in g (its
// reaction is minus the sum of both halves).
template <bool HALF, bool ENERGY, bool UNIFORM>
__device__ __forceinline__ void mixed_entry(const IPack& ip, const float4& xj, float sej,
    float s3j, unsigned excl, float cutforcesq, f2 A2, f2 mB2, float sig6u, double eps0,
    double ew, f2 (&fx)[2], f2 (&fy)[2], f2 (&fz)[2], f2& gx, f2& gy, f2& gz, double& e)
{
    const f2 XJ = f2_pack(xj.x, xj.x), YJ = f2_pack(xj.y, xj.y), ZJ = f2_pack(xj.z, xj.z);
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const f2 DX  = f2_sub(ip.x[h], XJ);
        const f2 DY  = f2_sub(ip.y[h], YJ);
        const f2 DZ  = f2_sub(ip.z[h], ZJ);
        const f2 RSQ = f2_fma(DX, DX, f2_fma(DY, DY, f2_mul(DZ, DZ)));
        float r0, r1;
        f2_unpack(RSQ, r0, r1);
        // excl: bit a set when pair (i atom a, this j atom) is excluded
        const bool in0 = r0 < cutforcesq && !((excl >> (2 * h)) & 1u);
        const bool in1 = r1 < cutforcesq && !((excl >> (2 * h + 1)) & 1u);
        float u0 = rcp_approx(r0), u1 = rcp_approx(r1);
        u0          = in0 ? u0 : 0.0f;
        u1          = in1 ? u1 : 0.0f;
        const f2 U  = f2_pack(u0, u1);
        const f2 U2 = f2_mul(U, U);
        const f2 U3 = f2_mul(U2, U);
        f2 F, SR6 = 0, EP = 0;
        if (UNIFORM) {
            F = f2_mul(f2_mul(U2, U2), f2_fma(A2, U3, mB2));
            if (ENERGY) SR6 = f2_mul(f2_pack(sig6u, sig6u), U3);
        } else {
            SR6 = f2_mul(f2_mul(ip.s3[h], f2_pack(s3j, s3j)), U3);
            EP  = f2_mul(ip.se[h], f2_pack(sej, sej));
            F   = f2_mul(f2_mul(U, SR6),
                f2_mul(EP, f2_fma(f2_pack(48.0f, 48.0f), SR6, f2_pack(-24.0f, -24.0f))));
        }
        fx[h] = f2_fma(DX, F, fx[h]);
        fy[h] = f2_fma(DY, F, fy[h]);
        fz[h] = f2_fma(DZ, F, fz[h]);
        if (HALF) {
            gx = f2_fma(DX, F, gx);
            gy = f2_fma(DY, F, gy);
            gz = f2_fma(DZ, F, gz);
        }
        if (ENERGY) {
            float s0, s1, e0, e1;
            f2_unpack(SR6, s0, s1);
            f2_unpack(EP, e0, e1);
            const double E0 = UNIFORM ? eps0 : (double)e0, E1 = UNIFORM ? eps0 : (double)e1;
            if (in0) e += ew * 4.0 * E0 * (double)s0 * ((double)s0 - 1.0);
            if (in1) e += ew * 4.0 * E1 * (double)s1 * ((double)s1 - 1.0);
        }
    }
}

// j data of one list entry: the atom's position moved into the i-cluster's
// anchor frame (the anchor difference is exact), its type bits in .w. Lanes
// past the end of a row read the dummy j-cluster (padding at +1e18, anchor 0),
// so no lane branches.
template <int JPL>
struct JEntry {
    float4 x[JPL]; // atoms b0 .. b0 + JPL - 1 of the entry
    int cj;
};

// the j position moved from its cluster's anchor a into the i frame (anchors
// are multiples of 1/8 of magnitude < 2^17: a - ai is exact; x and y as one
// packed pair)
__device__ __forceinline__ void to_i_frame(float4& x, float ax, float ay, float az,
    const float4& ai)
{
    const f2 dxy = f2_sub(f2_pack(ax, ay), f2_pack(ai.x, ai.y));
    const f2 jxy = f2_add(f2_pack(x.x, x.y), dxy);
    f2_unpack(jxy, x.x, x.y);
    x.z += az - ai.z;
}

// AW (one atom type): the anchor travels in .w of the entry's slots 0..2 and
// is applied when the entry is used (after its load has landed); otherwise
// it is loaded here and applied at once.
template <int N, bool AW, int JPL>
__device__ __forceinline__ JEntry<JPL> load_entry(int cj, int b0, const float4* __restrict__ xr,
    const float4* __restrict__ anchor, const float4& ai)
{
    JEntry<JPL> j;
    j.cj = cj;
    if (JPL == 2) {
        // slots cj * N + b0, b0 even: a 32-byte aligned pair
        ldg_pair4(&xr[cj * N + b0], j.x[0], j.x[JPL - 1]);
    } else {
#pragma unroll
        for (int u = 0; u < JPL; u++)
            j.x[u] = __ldg(&xr[cj * N + b0 + u]);
    }
    if (!AW) {
        const float4 a = __ldg(&anchor[cj]);
#pragma unroll
        for (int u = 0; u < JPL; u++)
            to_i_frame(j.x[u], a.x, a.y, a.z, ai);
    }
    return j;
}

// A segment of L = 32 / CPW lanes per i-cluster (M = 4 atoms, held by every
// lane of the segment as two packed pairs): CPW i-clusters per warp. The
// segment takes L / N list entries at a time; lane (e, b) owns atom b of entry
// e and computes its pairs with the 4 i atoms, two per packed instruction. The
// list is read in coalesced blocks of L entries (the next block in flight) and
// the j data of the next iteration is loaded while the current one computes.
// Full lists reduce the i forces across the segment once per i-cluster; half
// lists also accumulate each j atom's reaction over the 4 i atoms in the lane
// and add it with one atomic per component. Padding slots sit at +1e18 (j) and
// invalid i atoms are moved to -1e18, so they fall outside the cutoff without
// INF arithmetic.
// CPW > 1 shares the per-cluster set-up (i atoms, row pointers, the first
// loads) and the final reduction of a warp among CPW clusters, a fixed cost
// per i-cluster that is otherwise as large as four or five iterations over
// the row; a warp runs as many iterations as its longest row (the shorter
// rows compute the padding cluster meanwhile). The split of a row among the
// lanes, and so the FP32 rounding of the i sums, depends on CPW.
// PF: j data prefetched 1 or 2 iterations ahead; MINB: minimum resident blocks
// of 128 threads per SM asked of the register allocator (0: no request; 8
// caps a thread at 64 registers, measured best against 6, 7, 9 and 10).
// Both are launch-shape choices of the autotuner; results do not depend on them.
// JPL: j atoms per lane (consecutive atoms of one entry; 2 shares a lane's
// list handling, anchor and loop work between two atoms).
// The work of block bid (warps x CPW = i-clusters); s_se / s_s3: the type
// tables in shared memory.
template <int N, bool HALF, bool ENERGY, bool UNIFORM, int PF, int CPW, int JPL>
__device__ __forceinline__ void force_mixed_block(int bid, const int* __restrict__ cnt,
    const float4* __restrict__ xr, const float4* __restrict__ anchor, const Types& ty,
    float cutforcesq, const int* __restrict__ list, int ks, int cs,
    const int* __restrict__ numneigh, float4* cf32, double* epart, const float* s_se,
    const float* s_s3)
{
    constexpr int L   = 32 / CPW;  // lanes per i-cluster
    constexpr int LPE = N / JPL;   // lanes per list entry
    constexpr int JPW = L / LPE;   // entries per segment iteration
    static_assert(JPW >= 1, "a segment holds at least one list entry");
    const int lane = threadIdx.x & 31;
    const int l    = lane & (L - 1);
    const int ci   = ((bid * blockDim.x + threadIdx.x) >> 5) * CPW + lane / L;
    const int ncl  = cnt[CP_NCL];
    const bool act = ci < ncl;
    double e       = 0.0;
    if (__any_sync(0xffffffffu, act)) {
        const int cic    = act ? ci : 0; // address arithmetic of inactive segments
        const int jfac   = N / 4;
        const int ci_cj0 = cic / jfac;
        const int ai0    = 4 * (cic % jfac);
        const int nloc   = ncl * 4;
        // i atoms relative to their j-cluster's anchor; j positions are moved
        // into that frame by adding (anchor_j - anchor_i), exact in FP32
        const float4 ai = anchor[ci_cj0];
        float4 xi[4];
        float sei[4], s3i[4];
#pragma unroll
        for (int a = 0; a < 4; a++) {
            xi[a] = xr[cic * 4 + a];
            // padding: type -1, or (one type: .w carries the anchor) the
            // +1e18 position; every atom of an inactive segment
            int t          = UNIFORM ? 0 : __float_as_int(xi[a].w);
            const bool pad = !act || (UNIFORM ? !(xi[a].x < 0.1f * CP_PAD_F) : t < 0);
            if (pad) {
                xi[a].x = xi[a].y = xi[a].z = -CP_PAD_F;
                t                           = 0;
            }
            sei[a] = UNIFORM ? 0.f : s_se[t];
            s3i[a] = UNIFORM ? 0.f : s_s3[t];
        }
        IPack ip;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            ip.x[h]  = f2_pack(xi[2 * h].x, xi[2 * h + 1].x);
            ip.y[h]  = f2_pack(xi[2 * h].y, xi[2 * h + 1].y);
            ip.z[h]  = f2_pack(xi[2 * h].z, xi[2 * h + 1].z);
            ip.se[h] = f2_pack(sei[2 * h], sei[2 * h + 1]);
            ip.s3[h] = f2_pack(s3i[2 * h], s3i[2 * h + 1]);
        }
        const float cA    = (float)(48.0 * ty.eps0 * ty.sigma6_0 * ty.sigma6_0);
        const float cB    = (float)(24.0 * ty.eps0 * ty.sigma6_0);
        const float sig6u = (float)ty.sigma6_0;
        const f2 A2 = f2_pack(cA, cA), mB2 = f2_pack(-cB, -cB);
        f2 fx[2] = {0, 0}, fy[2] = {0, 0}, fz[2] = {0, 0};
        const int eidx = l / LPE, bq = l - eidx * LPE, b0 = bq * JPL;
        // pairs of the diagonal entry (cj == ci_cj0) excluded as the
        // reference's cond (clusterpair/force_lj.c:108-123): the self pair, and
        // for half lists every pair with the i atom at or after the j atom
        unsigned diag_excl[JPL];
#pragma unroll
        for (int u = 0; u < JPL; u++) {
            diag_excl[u] = 0;
#pragma unroll
            for (int a = 0; a < 4; a++)
                if (HALF ? (ai0 + a >= b0 + u) : (ai0 + a == b0 + u)) diag_excl[u] |= 1u << a;
        }
        const int nn    = act ? numneigh[ci] : 0;
        const int dummy = cnt[CP_NCJ] + cnt[CP_NGC]; // the dummy j-cluster
        const int* row  = list + (size_t)cic * cs;
        int lst_cur = l < nn ? __ldg(&row[(size_t)l * ks]) : dummy;
        int lst_nxt = L + l < nn ? __ldg(&row[(size_t)(L + l) * ks]) : dummy;
        JEntry<JPL> cur = load_entry<N, UNIFORM, JPL>(
            __shfl_sync(0xffffffffu, lst_cur, eidx, L), b0, xr, anchor, ai);
        JEntry<JPL> nx1;
        if (PF == 2) {
            const int c1 = __shfl_sync(0xffffffffu, lst_cur, JPW + eidx, L);
            nx1 = load_entry<N, UNIFORM, JPL>(JPW < nn ? c1 : dummy, b0, xr, anchor, ai);
        }
        // one segment iteration: JPW entries, lane (eidx, bq) on atoms b0 ..
        // b0 + JPL - 1 of entry kb + eidx; masked: the iteration may hold the
        // diagonal entry
        auto step = [&](int kb, bool masked) {
            // the entry block holding kn is rotated in when kn reaches it
            const int kn = kb + PF * JPW;
            if ((kn & (L - 1)) == 0) {
                lst_cur = lst_nxt;
                lst_nxt = kn + L + l < nn ? __ldg(&row[(size_t)(kn + L + l) * ks]) : dummy;
            }
            const int cjn = __shfl_sync(0xffffffffu, lst_cur, (kn & (L - 1)) + eidx, L);
            const JEntry<JPL> nx =
                load_entry<N, UNIFORM, JPL>(kn < nn ? cjn : dummy, b0, xr, anchor, ai);
            const int cj = cur.cj;
            float ax = 0.f, ay = 0.f, az = 0.f;
            if (UNIFORM) {
                // the anchor of this entry's j-cluster from .w of its slots
                // 0..2, held by the entry's lanes JPL slots each
                const int base = lane - bq;
                ax = __shfl_sync(0xffffffffu, cur.x[0 % JPL].w, base + 0 / JPL);
                ay = __shfl_sync(0xffffffffu, cur.x[1 % JPL].w, base + 1 / JPL);
                az = __shfl_sync(0xffffffffu, cur.x[2 % JPL].w, base + 2 / JPL);
            }
#pragma unroll
            for (int u = 0; u < JPL; u++) {
                const int b = b0 + u;
                float4 xj   = cur.x[u];
                if (UNIFORM) to_i_frame(xj, ax, ay, az, ai);
                float sej = 0.f, s3j = 0.f;
                if (!UNIFORM) {
                    int t = __float_as_int(cur.x[u].w);
                    t     = t < 0 ? 0 : t;
                    sej   = s_se[t];
                    s3j   = s_s3[t];
                }
                f2 gx = 0, gy = 0, gz = 0;
                // energy weight: full lists see every pair twice; half lists
                // once, except pairs with ghost atoms, which both owners list
                const double ew = (!HALF || cj * N + b >= nloc) ? 0.5 : 1.0;
                mixed_entry<HALF, ENERGY, UNIFORM>(ip, xj, sej, s3j,
                    (masked && cj == ci_cj0) ? diag_excl[u] : 0u, cutforcesq, A2, mB2, sig6u,
                    ty.eps0, ew, fx, fy, fz, gx, gy, gz, e);
                // reactions on local j atoms only (the reference drops ghost
                // reactions; the dummy cluster lies past the ghosts); padding
                // j slots get exact zeros
                if (HALF && cj * N + b < nloc) {
                    float gx0, gx1, gy0, gy1, gz0, gz1;
                    f2_unpack(gx, gx0, gx1);
                    f2_unpack(gy, gy0, gy1);
                    f2_unpack(gz, gz0, gz1);
                    red_add4(&cf32[cj * N + b], -(gx0 + gx1), -(gy0 + gy1), -(gz0 + gz1));
                }
            }
            if (PF == 2) {
                cur = nx1;
                nx1 = nx;
            } else {
                cur = nx;
            }
        };
        // the warp runs its longest row; the diagonal entry is the first of
        // its row (the list build swaps it to the front and pruning never
        // removes it), so only the first iteration tests for it
        const int nmax = CPW > 1 ? __reduce_max_sync(0xffffffffu, nn) : nn;
        if (nmax > 0) {
            step(0, true);
#pragma unroll((HALF && (CPW == 1 || JPL == 2)) ? 1 : 2)
            for (int kb = JPW; kb < nmax; kb += JPW) step(kb, false);
        }
        float f[12];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            f2_unpack(fx[h], f[6 * h + 0], f[6 * h + 3]);
            f2_unpack(fy[h], f[6 * h + 1], f[6 * h + 4]);
            f2_unpack(fz[h], f[6 * h + 2], f[6 * h + 5]);
        }
        seg_reduce_12<L>(f, l);
        if (act && (l & (L / 4 - 1)) == 0) {
            const int a     = l / (L / 4);
            const float4 xa = xr[ci * 4 + a];
            if (UNIFORM ? xa.x < 0.1f * CP_PAD_F : __float_as_int(xa.w) >= 0) {
                float4* dst = &cf32[ci * 4 + a];
                if (HALF) red_add4(dst, f[0], f[1], f[2]);
                else *dst = make_float4(f[0], f[1], f[2], 0.f);
            }
        }
    }
    if (ENERGY) {
        double t = block_sum(e);
        if (threadIdx.x == 0) epart[bid] = t;
    }
}

__device__ __forceinline__ void load_type_tables(const Types& ty, float* s_se, float* s_s3)
{
    if (threadIdx.x < MDB_MAX_TYPES) {
        s_se[threadIdx.x] = ty.sqrt_eps_f[threadIdx.x];
        s_s3[threadIdx.x] = ty.sigma3_f[threadIdx.x];
    }
    __syncthreads();
}

// slots > 0: the grid is slots x K blocks and block b works on block
// (b % slots) * K + b / slots, so that the blocks one resident slot runs one
// after another take neighbouring i-clusters, whose j data is then still in
// that SM's L1 (blocks of a launch start in index order)
template <int N, bool HALF, bool ENERGY, bool UNIFORM, int PF, int MINB, int CPW, int JPL>
__global__ void __launch_bounds__(MINB ? 128 : 512, MINB ? MINB : 1) k_force_mixed(
    const int* __restrict__ cnt,
    const float4* __restrict__ xr, const float4* __restrict__ anchor, Types ty,
    float cutforcesq, const int* __restrict__ list, int ks, int cs,
    const int* __restrict__ numneigh, float4* cf32, double* epart, int slots)
{
    __shared__ float s_se[MDB_MAX_TYPES], s_s3[MDB_MAX_TYPES];
    load_type_tables(ty, s_se, s_s3);
    int bid = blockIdx.x;
    if (slots > 0) bid = (blockIdx.x % slots) * (gridDim.x / slots) + blockIdx.x / slots;
    force_mixed_block<N, HALF, ENERGY, UNIFORM, PF, CPW, JPL>(bid, cnt, xr, anchor, ty, cutforcesq,
        list, ks, cs, numneigh, cf32, epart, s_se, s_s3);
}

// all members of an ensemble group (same shape, list form, types and launch)
template <int N, bool HALF, bool ENERGY, bool UNIFORM, int PF, int MINB, int CPW, int JPL>
__global__ void __launch_bounds__(MINB ? 128 : 512, MINB ? MINB : 1) k_force_mixed_batch(
    const CpForceMember* __restrict__ tab, const int2* __restrict__ bmap, Types ty,
    float cutforcesq)
{
    __shared__ float s_se[MDB_MAX_TYPES], s_s3[MDB_MAX_TYPES];
    const int2 bm = __ldg(&bmap[blockIdx.x]);
    if (bm.x < 0) return; // an unused entry of a map sized for the capacities
    load_type_tables(ty, s_se, s_s3);
    const CpForceMember& m = tab[bm.x];
    force_mixed_block<N, HALF, ENERGY, UNIFORM, PF, CPW, JPL>(bm.y, m.cnt, m.xr, m.anchor, ty, cutforcesq,
        m.list, 1, m.cs, m.numneigh, m.cf32, m.epart, s_se, s_s3);
}

int force_mixed_threads(const Types& ty)
{
    // blocks of ty.force_block threads (128 when a register budget is asked)
    return (ty.force_variant & 2) ? 128 : ty.force_block;
}

int force_mixed_grid(int ncl_cap, const Types& ty)
{
    const int nt = force_mixed_threads(ty);
    return (int)(((long long)ncl_cap * 32 / ty.force_cpw + nt - 1) / nt);
}

template <int N, bool HALF, bool ENERGY, bool UNIFORM>
static void run_mixed_batch(cudaStream_t s, int nblocks, const CpForceMember* tab,
    const int2* bmap, const Types& ty, float cutforcesq)
{
    const int nt = force_mixed_threads(ty);
#define CP_RUN(PF, MB, C) CP_RUNJ(PF, MB, C, 1)
#define CP_RUNJ(PF, MB, C, J)                                                            \
    k_force_mixed_batch<N, HALF, ENERGY, UNIFORM, PF, MB, C, J><<<nblocks, nt, 0, s>>>(tab,   \
        bmap, ty, cutforcesq)
    const int v = ty.force_variant;
    if (ty.force_cpw == 4 && ty.force_jpl == 2) {
        if (v & 2) CP_RUNJ(1, 8, 4, 2);
        else CP_RUNJ(1, 0, 4, 2);
    } else if (ty.force_cpw == 2) {
        if (v == 3) CP_RUN(1, 6, 2);
        else if (v & 2) CP_RUN(1, 8, 2);
        else CP_RUN(1, 0, 2);
    } else if (ty.force_cpw == 4) {
        if (v == 3) CP_RUN(1, 6, 4);
        else if (v & 2) CP_RUN(1, 8, 4);
        else CP_RUN(1, 0, 4);
    } else if (ty.force_cpw == 8) {
        if constexpr (N == 4) {
            if (v == 3) CP_RUN(1, 6, 8);
            else if (v & 2) CP_RUN(1, 8, 8);
            else CP_RUN(1, 0, 8);
        }
    } else {
        switch (v) {
        case 1: CP_RUN(2, 0, 1); break;
        case 2: CP_RUN(1, 8, 1); break;
        case 3: CP_RUN(2, 8, 1); break;
        default: CP_RUN(1, 0, 1); break;
        }
    }
#undef CP_RUN
#undef CP_RUNJ
}

template <int N, bool HALF>
static void run_mixed_batch_e(cudaStream_t s, int energy, int nblocks,
    const CpForceMember* tab, const int2* bmap, const Types& ty, float cutforcesq)
{
    if (ty.uniform) {
        if (energy) run_mixed_batch<N, HALF, true, true>(s, nblocks, tab, bmap, ty, cutforcesq);
        else run_mixed_batch<N, HALF, false, true>(s, nblocks, tab, bmap, ty, cutforcesq);
    } else {
        if (energy) run_mixed_batch<N, HALF, true, false>(s, nblocks, tab, bmap, ty, cutforcesq);
        else run_mixed_batch<N, HALF, false, false>(s, nblocks, tab, bmap, ty, cutforcesq);
    }
}

void launch_force_mixed_batch(cudaStream_t s, int N, int half, int energy, const Types& ty,
    float cutforcesq, int nblocks, const CpForceMember* tab, const int2* bmap)
{
    if (nblocks <= 0) return;
    if (N == 4) {
        if (half) run_mixed_batch_e<4, true>(s, energy, nblocks, tab, bmap, ty, cutforcesq);
        else run_mixed_batch_e<4, false>(s, energy, nblocks, tab, bmap, ty, cutforcesq);
    } else {
        if (half) run_mixed_batch_e<8, true>(s, energy, nblocks, tab, bmap, ty, cutforcesq);
        else run_mixed_batch_e<8, false>(s, energy, nblocks, tab, bmap, ty, cutforcesq);
    }
    g_launches++;
}

template <int N, bool HALF, bool ENERGY, bool UNIFORM>
static void run_mixed(cudaStream_t s, int blocks, const int* cnt, const float4* xr,
    const float4* anchor, const Types& ty, float cutforcesq, const int* list, int ks, int cs,
    const int* numneigh, float4* cf32, double* epart)
{
    const int v  = ty.force_variant;
    const int nt = force_mixed_threads(ty);
    int nb = blocks, slots = 0;
    if (!ENERGY && ty.force_swizzle) {
        // resident blocks of the whole GPU: the SM count times the blocks of
        // this shape one SM holds
        static int nsm = 0;
        if (!nsm) {
            int dev = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        }
        const int per_sm =
            (v & 2) ? ((v == 3 && ty.force_cpw > 1) ? 6 : 8) : std::max(1, 2048 / nt);
        slots            = nsm * per_sm;
        if (nb > slots) nb = (nb + slots - 1) / slots * slots;
        else slots = 0;
    }
#define CP_RUN(PF, MB, C) CP_RUNJ(PF, MB, C, 1)
#define CP_RUNJ(PF, MB, C, J)                                                            \
    k_force_mixed<N, HALF, ENERGY, UNIFORM, PF, MB, C, J><<<nb, nt, 0, s>>>(cnt, xr, anchor, \
        ty, cutforcesq, list, ks, cs, numneigh, cf32, epart, slots)
    // several clusters per warp: prefetch depth 1; bit 0 of the variant
    // lowers the register budget's block count from 8 to 6
    if (ty.force_cpw == 2) {
        if (v == 3) CP_RUN(1, 6, 2);
        else if (v & 2) CP_RUN(1, 8, 2);
        else CP_RUN(1, 0, 2);
    } else if (ty.force_cpw == 4 && ty.force_jpl == 2) {
        if (v & 2) CP_RUNJ(1, 8, 4, 2);
        else CP_RUNJ(1, 0, 4, 2);
    } else if (ty.force_cpw == 4) {
        if (v == 3) CP_RUN(1, 6, 4);
        else if (v & 2) CP_RUN(1, 8, 4);
        else CP_RUN(1, 0, 4);
    } else if (ty.force_cpw == 8) {
        // a segment of 4 lanes: one entry of a 4-wide j-cluster at a time
        if constexpr (N == 4) {
            if (v == 3) CP_RUN(1, 6, 8);
            else if (v & 2) CP_RUN(1, 8, 8);
            else CP_RUN(1, 0, 8);
        }
    } else {
        switch (v) {
        case 1: CP_RUN(2, 0, 1); break;
        case 2: CP_RUN(1, 8, 1); break;
        case 3: CP_RUN(2, 8, 1); break;
        default: CP_RUN(1, 0, 1); break;
        }
    }
#undef CP_RUN
#undef CP_RUNJ
}

template <int N, bool HALF>
static void run_mixed_e(cudaStream_t s, int blocks, int energy, const int* cnt, const float4* xr,
    const float4* anchor, const Types& ty, float cutforcesq, const int* list, int ks, int cs,
    const int* numneigh, float4* cf32, double* epart)
{
    if (ty.uniform) {
        if (energy) run_mixed<N, HALF, true, true>(s, blocks, cnt, xr, anchor, ty, cutforcesq, list, ks, cs, numneigh, cf32, epart);
        else run_mixed<N, HALF, false, true>(s, blocks, cnt, xr, anchor, ty, cutforcesq, list, ks, cs, numneigh, cf32, epart);
    } else {
        if (energy) run_mixed<N, HALF, true, false>(s, blocks, cnt, xr, anchor, ty, cutforcesq, list, ks, cs, numneigh, cf32, epart);
        else run_mixed<N, HALF, false, false>(s, blocks, cnt, xr, anchor, ty, cutforcesq, list, ks, cs, numneigh, cf32, epart);
    }
}

int launch_force_mixed(cudaStream_t s, int N, int half, int energy, int ncl_cap,
    const int* cnt, const float4* xr, const float4* anchor, const Types& ty, float cutforcesq,
    const int* list, int ks, int cs, const int* numneigh, float4* cf32, double* epart)
{
    const int blocks = force_mixed_grid(ncl_cap, ty);
    if (N == 4) {
        if (half) run_mixed_e<4, true>(s, blocks, energy, cnt, xr, anchor, ty, cutforcesq, list, ks, cs, numneigh, cf32, epart);
        else run_mixed_e<4, false>(s, blocks, energy, cnt, xr, anchor, ty, cutforcesq, list, ks, cs, numneigh, cf32, epart);
    } else {
        if (half) run_mixed_e<8, true>(s, blocks, energy, cnt, xr, anchor, ty, cutforcesq, list, ks, cs, numneigh, cf32, epart);
        else run_mixed_e<8, false>(s, blocks, energy, cnt, xr, anchor, ty, cutforcesq, list, ks, cs, numneigh, cf32, epart);
    }
    g_launches++;
    return blocks;
}

// ---- integrator: initialIntegrateCPU / finalIntegrateCPU (clusterpair/integrate.c:29-86)
__device__ __forceinline__ double3 slot_force(int s, const double4* cf, const float4* cf32)
{
    if (cf32) {
        float4 f = cf32[s];
        return make_double3((double)f.x, (double)f.y, (double)f.z);
    }
    double4 f = cf[s];
    return make_double3(f.x, f.y, f.z);
}

// zero_f: clear the force slot after its use (half lists accumulate into it;
// only when a force evaluation follows before anything reads the forces)
// xb (displacement check, null: off): positions at the last build; a slot
// that moved farther than sqrt(lim2) since then sets *flag.
template <bool FINAL, bool INITIAL>
__device__ __forceinline__ void cp_integrate_slot(int s, int M, int N,
    const int* __restrict__ cnt, double dtf, double dt, double4* cx, double4* cv,
    const double4* __restrict__ cf, float4* cf32, const float4* __restrict__ anchor, float4* xr,
    bool zero_f, int xmode, const double4* __restrict__ xb = nullptr, double lim2 = 0.0,
    int* flag = nullptr, const float4* __restrict__ xq = nullptr, float qlim2 = 0.f,
    int* qflag = nullptr)
{
    if (s >= cnt[CP_NCL] * M) return;
    double4 p = cx[s];
    if (slot_type(p) < 0) return;
    double4 v       = cv[s];
    const double3 f = slot_force(s, cf, cf32);
    if (INITIAL && zero_f) {
        if (cf32) cf32[s] = make_float4(0.f, 0.f, 0.f, 0.f);
        else const_cast<double4*>(cf)[s] = make_double4(0.0, 0.0, 0.0, 0.0);
    }
    if (FINAL) {
        v.x += dtf * f.x;
        v.y += dtf * f.y;
        v.z += dtf * f.z;
    }
    if (INITIAL) {
        v.x += dtf * f.x;
        v.y += dtf * f.y;
        v.z += dtf * f.z;
        p.x += dt * v.x;
        p.y += dt * v.y;
        p.z += dt * v.z;
        cx[s] = p;
        if (xr) put_rel(xr, s, p, anchor[s / N], xmode, s % N);
        if (xq) {
            const float4 r = xr[s], q = xq[s];
            const float dx = r.x - q.x, dy = r.y - q.y, dz = r.z - q.z;
            if (dx * dx + dy * dy + dz * dz > qlim2) *qflag = 1;
        }
        if (xb) {
            const double4 q = xb[s];
            const double dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
            if (dx * dx + dy * dy + dz * dz > lim2) *flag = 1;
        }
    }
    cv[s] = v;
}

template <bool FINAL, bool INITIAL>
__global__ void k_cp_integrate(int M, int N, const int* __restrict__ cnt, double dtf, double dt,
    double4* cx, double4* cv, const double4* __restrict__ cf, const float4* __restrict__ cf32,
    const float4* __restrict__ anchor, float4* xr, int xmode, const double4* __restrict__ xb,
    double lim2, int* flag, const float4* __restrict__ xq, float qlim2, int* qflag)
{
    cp_integrate_slot<FINAL, INITIAL>(blockIdx.x * blockDim.x + threadIdx.x, M, N, cnt, dtf, dt,
        cx, cv, cf, const_cast<float4*>(cf32), anchor, xr, false, xmode, xb, lim2, flag, xq,
        qlim2, qflag);
}

template <bool FINAL, bool INITIAL>
__global__ void k_cp_integrate_batch(const CpStepMember* __restrict__ tab,
    const int2* __restrict__ bmap)
{
    const int2 bm = __ldg(&bmap[blockIdx.x]);
    if (bm.x < 0) return;
    const CpStepMember& m = tab[bm.x];
    cp_integrate_slot<FINAL, INITIAL>(bm.y * blockDim.x + threadIdx.x, m.M, m.N, m.cnt, m.dtf,
        m.dt, m.cx, m.cv, m.cf, m.cf32, m.anchor, m.xr, false, m.mixed, m.xb, m.lim2, m.flag);
}

// Clearing the half-list force slots right before the force kernel (rather
// than in the integrator, which streams positions and velocities through L2
// after it) leaves the slots in L2 when the kernel's reduction atomics arrive.
__global__ void k_zero_forces_batch(const CpStepMember* __restrict__ tab,
    const int2* __restrict__ bmap)
{
    const int2 bm = __ldg(&bmap[blockIdx.x]);
    if (bm.x < 0) return;
    const CpStepMember& m = tab[bm.x];
    const int s           = bm.y * blockDim.x + threadIdx.x;
    if (!m.zero_f || s >= m.cnt[CP_NCL] * m.M) return;
    if (m.cf32) m.cf32[s] = make_float4(0.f, 0.f, 0.f, 0.f);
    else const_cast<double4*>(m.cf)[s] = make_double4(0.0, 0.0, 0.0, 0.0);
}

void launch_zero_forces_batch(cudaStream_t s, int nblocks, const CpStepMember* tab,
    const int2* bmap)
{
    if (nblocks <= 0) return;
    k_zero_forces_batch<<<nblocks, MDB_NTHREADS, 0, s>>>(tab, bmap);
    g_launches++;
}

void launch_cp_integrate_batch(cudaStream_t s, bool final_, bool initial, int nblocks,
    const CpStepMember* tab, const int2* bmap)
{
    if (nblocks <= 0) return;
    if (final_ && initial)
        k_cp_integrate_batch<true, true><<<nblocks, MDB_NTHREADS, 0, s>>>(tab, bmap);
    else if (initial) k_cp_integrate_batch<false, true><<<nblocks, MDB_NTHREADS, 0, s>>>(tab, bmap);
    else k_cp_integrate_batch<true, false><<<nblocks, MDB_NTHREADS, 0, s>>>(tab, bmap);
    g_launches++;
}

void launch_cp_initial(cudaStream_t s, int M, int N, int ncl_cap, const int* cnt, double dtf,
    double dt, double4* cx, double4* cv, const double4* cf, const float4* cf32,
    const float4* anchor, float4* xr, int xmode, const double4* xb, double lim2, int* flag,
    const float4* xq, float qlim2, int* qflag)
{
    long long n = (long long)ncl_cap * M;
    k_cp_integrate<false, true><<<mdb_blocks(n, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(M, N, cnt,
        dtf, dt, cx, cv, cf, cf32, anchor, xr, xmode, xb, lim2, flag, xq, qlim2, qflag);
    g_launches++;
}

void launch_cp_final(cudaStream_t s, int M, int ncl_cap, const int* cnt, double dtf,
    const double4* cx, double4* cv, const double4* cf, const float4* cf32)
{
    long long n = (long long)ncl_cap * M;
    k_cp_integrate<true, false><<<mdb_blocks(n, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(M, M, cnt,
        dtf, 0.0, const_cast<double4*>(cx), cv, cf, cf32, nullptr, nullptr, 0, nullptr, 0.0,
        nullptr, nullptr, 0.f, nullptr);
    g_launches++;
}

void launch_cp_final_initial(cudaStream_t s, int M, int N, int ncl_cap, const int* cnt,
    double dtf, double dt, double4* cx, double4* cv, const double4* cf, const float4* cf32,
    const float4* anchor, float4* xr, int xmode, const double4* xb, double lim2, int* flag,
    const float4* xq, float qlim2, int* qflag)
{
    long long n = (long long)ncl_cap * M;
    k_cp_integrate<true, true><<<mdb_blocks(n, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(M, N, cnt,
        dtf, dt, cx, cv, cf, cf32, anchor, xr, xmode, xb, lim2, flag, xq, qlim2, qflag);
    g_launches++;
}

// ---- thermo: computeThermo (common/thermo.c:60-100) over the atom arrays ------------
int ke_blocks(int n) { return mdb_blocks(n > 0 ? n : 1, MDB_NTHREADS); }

__global__ void k_ke_atoms(int n, const double4* __restrict__ av, double mass, double* partials)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double t    = 0.0;
    if (i < n) {
        double4 v = av[i];
        t         = (v.x * v.x + v.y * v.y + v.z * v.z) * mass;
    }
    t = block_sum(t);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

void launch_ke_atoms(cudaStream_t s, int n, const double4* av, double mass, double* partials)
{
    k_ke_atoms<<<ke_blocks(n), MDB_NTHREADS, 0, s>>>(n, av, mass, partials);
    g_launches++;
}

// kinetic energy sum of the cluster state (locals): the same sum over slots
__global__ void k_ke_slots(int M, const int* __restrict__ cnt, const double4* __restrict__ cx,
    const double4* __restrict__ cv, double mass, double* partials)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    double t    = 0.0;
    if (s < cnt[CP_NCL] * M && slot_type(cx[s]) >= 0) {
        double4 v = cv[s];
        t         = (v.x * v.x + v.y * v.y + v.z * v.z) * mass;
    }
    t = block_sum(t);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

void launch_ke_slots(cudaStream_t s, int M, int ncl_cap, const int* cnt, const double4* cx,
    const double4* cv, double mass, double* partials)
{
    long long n = (long long)ncl_cap * M;
    k_ke_slots<<<mdb_blocks(n, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(M, cnt, cx, cv, mass, partials);
    g_launches++;
}

} // namespace cp
} // namespace mdb
