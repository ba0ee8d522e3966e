// Cluster-pair scheme, mixed precision: the pair-list force path.
//
// The cluster-pair list (built bit-exactly as the reference's
// buildNeighborCPU, clusterpair/neighbor.c:282-765) lists whole 4 x N
// cluster pairs: on the LJ liquid about a quarter of their pair slots lie
// inside the cutoff, and the cluster-pair force kernel (mdb_cp_force.cu) pays
// for all of them. This path derives from that list, per pair of i atoms
// (atoms 0,1 and 2,3 of an i-cluster), the j atoms of its listed cluster
// pairs that lie within r_in = r_c + buffer of either atom, and evaluates
// only those: each lane holds one i pair packed in .f32x2 registers and
// computes both pairs of a j atom per packed instruction.
//
// Exactness of the pair set: a pair left out had r > r_in when the codes
// were derived; it can come inside r_c only after one of its atoms moved more
// than buffer / 2. The integrator compares every atom's position with its
// position at the last derivation and raises a device flag past that limit;
// the derivation kernel runs at every force evaluation but returns at once
// unless the flag is set (or a list build asked for it), so the pairs
// evaluated are exactly the listed cluster pairs' pairs within r_c, as in the
// cluster-pair kernels, with no host round trip inside the captured timestep.
//
// Codes: for i pair h of i-cluster ci and chunk c of its list row (chunks of
// 256 / N entries), one byte per j atom, e * N + b (entry e of the chunk, atom
// b of that j-cluster); pcnt holds the count. Storage is fixed at 256 bytes
// per (i pair, chunk), so a derivation can never overflow it.
#include <algorithm>

#include "mdb_cp_f2.cuh"
#include "mdb_cp_internal.cuh"

namespace mdb {
namespace cp {

#define PAIR_THREADS 128
#define PAIR_WARPS (PAIR_THREADS / 32)
// launch shapes of the force kernel (tuning key pair_variant; results do not
// depend on them): codes a lane has in flight, and the minimum resident blocks
// of 128 threads per SM asked of the register allocator (0: no request)
static constexpr int PAIR_VARIANTS[4][2] = {{4, 0}, {2, 0}, {3, 6}, {2, 8}};

template <int N> struct PairChunk {
    static constexpr int CH   = 256 / N; // list entries per chunk: codes e * N + b < 256
    static constexpr int LOGN = N == 4 ? 2 : 3;
};

int pair_chunks(int maxneighs, int N) { return (maxneighs + 256 / N - 1) / (256 / N); }

// i atom of an i-cluster in its cluster frame; padding (type -1, or with one
// atom type the +1e18 position) reported invalid and moved to -1e18, where it
// pairs with nothing
template <bool UNIFORM>
__device__ __forceinline__ float4 i_atom(const float4* __restrict__ xr, int slot, bool& valid,
    int& type)
{
    float4 p = __ldg(&xr[slot]);
    type     = UNIFORM ? 0 : __float_as_int(p.w);
    valid    = UNIFORM ? p.x < 0.1f * CP_PAD_F : type >= 0;
    if (!valid) {
        p.x = p.y = p.z = -CP_PAD_F;
        type            = 0;
    }
    return p;
}

// ---- one code: a j atom against the lane's i pair ------------------------------
// Packed FP32: both pairs per instruction, the cutoff and the exclusion bits
// ex (bit k: pair with i atom 2h + k excluded) as select masks. The j
// position is already in the i frame. Half lists add the reaction on local j
// atoms (summed over the pair) with one vector reduction.
// COMP (MDB_PREC_MIXED_COMP): a pair whose FP32 distance lies within an FP32
// rounding margin of r_c is tested again in FP64 on the positions the FP64
// path uses (cx, the same expression), so both paths take the same pairs; the
// i sums carry two-sum compensation terms (c*) and half-list reactions go to
// the FP64 force slots by FP64 atomics.
struct CompState {
    const double4* cx;
    double cutsq;
    int si0;  // slot of i atom 2h
    f2 cx_, cy_, cz_;
};

__device__ __forceinline__ void two_sum2(f2& s, f2& c, const f2& v)
{
    const f2 t  = f2_add(s, v);
    const f2 bp = f2_sub(t, s);
    c           = f2_add(c, f2_add(f2_sub(s, f2_sub(t, bp)), f2_sub(v, bp)));
    s           = t;
}

template <bool HALF, bool ENERGY, bool UNIFORM, bool COMP>
__device__ __forceinline__ void pair2(const f2& XI, const f2& YI, const f2& ZI,
    const float4& xj, int sj, unsigned ex, int t0, int t1, const float4* s_tab,
    const PairTypes& pt, float cutforcesq, const f2& A2, const f2& mB2, int nloc, f2& fx,
    f2& fy, f2& fz, float4* cf32, double4* cf64, CompState& cs, double& e)
{
    const f2 DX  = f2_sub(XI, f2_pack(xj.x, xj.x));
    const f2 DY  = f2_sub(YI, f2_pack(xj.y, xj.y));
    const f2 DZ  = f2_sub(ZI, f2_pack(xj.z, xj.z));
    const f2 RSQ = f2_fma(DX, DX, f2_fma(DY, DY, f2_mul(DZ, DZ)));
    float r0, r1;
    f2_unpack(RSQ, r0, r1);
    bool in0 = r0 < cutforcesq && !(ex & 1u);
    bool in1 = r1 < cutforcesq && !(ex & 2u);
    if (COMP) {
        // FP32 distances are within ~1e-6 relative of the exact ones here
        const float band = 1e-5f * cutforcesq;
        const bool b0 = fabsf(r0 - cutforcesq) < band, b1 = fabsf(r1 - cutforcesq) < band;
        if (b0 || b1) {
            const double4 pj = cs.cx[sj];
#pragma unroll
            for (int k = 0; k < 2; k++) {
                if (!(k ? b1 : b0)) continue;
                const double4 pi  = cs.cx[cs.si0 + k];
                const double delx = pi.x - pj.x, dely = pi.y - pj.y, delz = pi.z - pj.z;
                const double rsq  = delx * delx + dely * dely + delz * delz;
                const bool in     = rsq < cs.cutsq && !((ex >> k) & 1u);
                if (k) in1 = in;
                else in0 = in;
            }
        }
    }
    float u0 = rcp_approx(r0), u1 = rcp_approx(r1);
    u0          = in0 ? u0 : 0.0f;
    u1          = in1 ? u1 : 0.0f;
    const f2 U  = f2_pack(u0, u1);
    const f2 U2 = f2_mul(U, U);
    const f2 U3 = f2_mul(U2, U);
    f2 F;
    float4 ta = make_float4(0.f, 0.f, 0.f, 0.f), tb = ta;
    if (UNIFORM) {
        F = f2_mul(f2_mul(U2, U2), f2_fma(A2, U3, mB2));
    } else {
        int tj = __float_as_int(xj.w);
        tj     = tj < 0 ? 0 : tj;
        ta     = s_tab[t0 * MDB_MAX_TYPES + tj];
        tb     = s_tab[t1 * MDB_MAX_TYPES + tj];
        F = f2_mul(f2_mul(U2, U2), f2_fma(f2_pack(ta.x, tb.x), U3, f2_pack(-ta.y, -tb.y)));
    }
    if (COMP) {
        const f2 GX = f2_mul(DX, F), GY = f2_mul(DY, F), GZ = f2_mul(DZ, F);
        two_sum2(fx, cs.cx_, GX);
        two_sum2(fy, cs.cy_, GY);
        two_sum2(fz, cs.cz_, GZ);
        if (HALF && sj < nloc) {
            float gx0, gx1, gy0, gy1, gz0, gz1;
            f2_unpack(GX, gx0, gx1);
            f2_unpack(GY, gy0, gy1);
            f2_unpack(GZ, gz0, gz1);
            atomicAdd(&cf64[sj].x, -((double)gx0 + (double)gx1));
            atomicAdd(&cf64[sj].y, -((double)gy0 + (double)gy1));
            atomicAdd(&cf64[sj].z, -((double)gz0 + (double)gz1));
        }
    } else {
        fx = f2_fma(DX, F, fx);
        fy = f2_fma(DY, F, fy);
        fz = f2_fma(DZ, F, fz);
        if (HALF && sj < nloc) {
            float gx0, gx1, gy0, gy1, gz0, gz1;
            f2_unpack(f2_mul(DX, F), gx0, gx1);
            f2_unpack(f2_mul(DY, F), gy0, gy1);
            f2_unpack(f2_mul(DZ, F), gz0, gz1);
            red_add4(&cf32[sj], -(gx0 + gx1), -(gy0 + gy1), -(gz0 + gz1));
        }
    }
    if (ENERGY) {
        // full lists see every pair twice; half lists once, except pairs
        // with ghost atoms, which both owners list
        const double ew = (!HALF || sj >= nloc) ? 0.5 : 1.0;
        float s0, s1;
        f2_unpack(f2_mul(UNIFORM ? f2_pack(pt.sig6_0, pt.sig6_0) : f2_pack(ta.z, tb.z), U3), s0,
            s1);
        const double E0 = UNIFORM ? pt.eps0 : (double)ta.w;
        const double E1 = UNIFORM ? pt.eps0 : (double)tb.w;
        if (in0) e += ew * 4.0 * E0 * (double)s0 * ((double)s0 - 1.0);
        if (in1) e += ew * 4.0 * E1 * (double)s1 * ((double)s1 - 1.0);
    }
}

// ---- derivation ----------------------------------------------------------------
// Runs before every force evaluation and returns at once unless the flag is
// set (an atom moved past half the buffer since the last derivation, or a
// build asked for it) or force is given; its grid is one wave of resident
// blocks that loops over the clusters, so the common case costs one wave of
// early exits. One warp per i-cluster at a time: the warp caches the chunk's
// entries (slot base, anchor offset) in shared memory, then tests every atom
// of them against the cluster's 4 i atoms, two candidate passes in flight,
// with the reference's exclusions on the diagonal entry
// (clusterpair/force_lj.c:108-123); ballots keep the list order; the codes of
// both i pairs, their counts and the i atoms' positions (for the
// integrator's test) are written.
template <int N, bool HALF, bool UNIFORM>
__global__ void __launch_bounds__(PAIR_THREADS) k_pair_derive(const int* __restrict__ cnt,
    const float4* __restrict__ xr, const float4* __restrict__ anchor,
    const int* __restrict__ list, int cs, const int* __restrict__ numneigh, float rin2,
    int* qflag, int force, unsigned char* __restrict__ pcode,
    unsigned short* __restrict__ pcnt, int chmax, float4* __restrict__ xq)
{
    if (!force && *(volatile int*)qflag == 0) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) qflag[1] += 1; // derivations run
    constexpr int CH = PairChunk<N>::CH, LOGN = PairChunk<N>::LOGN;
    __shared__ float4 s_row[PAIR_WARPS][CH];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ncl  = cnt[CP_NCL];
    const int jfac = N / 4;
    const unsigned lt = (1u << lane) - 1u;
    for (int ci = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; ci < ncl;
         ci += (gridDim.x * blockDim.x) >> 5) {
        const int ci_cj0 = ci / jfac, ai0 = 4 * (ci % jfac);
        const int nn     = __ldg(&numneigh[ci]);
        const int* row   = list + (size_t)ci * cs;
        const float4 ai  = __ldg(&anchor[ci_cj0]);
        float xi[4], yi[4], zi[4];
        unsigned vmask = 0;
#pragma unroll
        for (int a = 0; a < 4; a++) {
            bool v;
            int t;
            const float4 p = i_atom<UNIFORM>(xr, ci * 4 + a, v, t);
            xi[a] = p.x, yi[a] = p.y, zi[a] = p.z;
            vmask |= (v ? 1u : 0u) << a;
        }
        if (lane < 4) xq[ci * 4 + lane] = __ldg(&xr[ci * 4 + lane]);
        const int nch = (nn + CH - 1) / CH;
        for (int c = 0; c < nch; c++) {
            const int ne = min(CH, nn - c * CH);
            const int ns = ne * N;
            for (int k = lane; k < ne; k += 32) {
                const int cj   = __ldg(&row[c * CH + k]);
                const float4 a = __ldg(&anchor[cj]);
                s_row[warp][k] = make_float4(a.x - ai.x, a.y - ai.y, a.z - ai.z,
                    __int_as_float(cj * N));
            }
            __syncwarp();
            unsigned char* o0 = pcode + ((size_t)(2 * ci) * chmax + c) * 256;
            unsigned char* o1 = o0 + (size_t)chmax * 256;
            int n0 = 0, n1 = 0;
            for (int q0 = 0; q0 < ns; q0 += 64) {
                float4 xa[2], da[2];
                int qa[2];
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    qa[u]          = q0 + 32 * u + lane;
                    const bool act = qa[u] < ns;
                    da[u]          = s_row[warp][act ? qa[u] >> LOGN : 0];
                    xa[u] = act ? __ldg(&xr[__float_as_int(da[u].w) + (qa[u] & (N - 1))])
                                : make_float4(CP_PAD_F, CP_PAD_F, CP_PAD_F, 0.f);
                }
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    const int b    = qa[u] & (N - 1);
                    const float jx = xa[u].x + da[u].x, jy = xa[u].y + da[u].y,
                                jz = xa[u].z + da[u].z;
                    const bool dg  = __float_as_int(da[u].w) == ci_cj0 * N;
                    bool in0 = false, in1 = false;
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        const float dx = xi[k] - jx, dy = yi[k] - jy, dz = zi[k] - jz;
                        const float r2 = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz)));
                        const bool ex  = dg && (HALF ? (ai0 + k >= b) : (ai0 + k == b));
                        const bool ok  = ((vmask >> k) & 1u) && !ex && r2 < rin2;
                        if (k < 2) in0 |= ok;
                        else in1 |= ok;
                    }
                    const unsigned m0 = __ballot_sync(0xffffffffu, in0);
                    const unsigned m1 = __ballot_sync(0xffffffffu, in1);
                    if (in0) o0[n0 + __popc(m0 & lt)] = (unsigned char)qa[u];
                    if (in1) o1[n1 + __popc(m1 & lt)] = (unsigned char)qa[u];
                    n0 += __popc(m0);
                    n1 += __popc(m1);
                }
            }
            if (lane == 0) {
                pcnt[(size_t)(2 * ci) * chmax + c]     = (unsigned short)n0;
                pcnt[(size_t)(2 * ci + 1) * chmax + c] = (unsigned short)n1;
            }
            __syncwarp(); // the cached row is rewritten for the next chunk
        }
    }
}

// ---- force -------------------------------------------------------------------
// One warp per i-cluster; lanes 16h..16h+15 own i pair h (atoms 2h, 2h+1,
// packed). Every load that depends on no other is issued first (row length,
// first list entries, first codes and their count, i atoms, anchor); per
// chunk the warp then caches the entries in shared memory (each j-cluster's
// slot base and its anchor offset from the i-cluster's anchor, a difference
// of multiples of 1/8 and so exact in FP32), and each lane takes its codes
// PAIR_BATCH at a time with all their j loads in flight together. Thread 0
// of block 0 clears the derivation flag (the derivation kernel of this
// evaluation has completed before this kernel starts).
template <int N, bool HALF, bool ENERGY, bool UNIFORM, int PAIR_BATCH, int MINB, bool COMP>
__global__ void __launch_bounds__(PAIR_THREADS, MINB ? MINB : 1) k_force_pairs(const int* __restrict__ cnt,
    const float4* __restrict__ xr, const float4* __restrict__ anchor, PairTypes pt,
    float cutforcesq, const int* __restrict__ list, int cs, const int* __restrict__ numneigh,
    const unsigned char* __restrict__ pcode, const unsigned short* __restrict__ pcnt, int chmax,
    float4* cf32, double* epart, int* qflag, const double4* __restrict__ cx, double4* cf64,
    double cutsq64)
{
    constexpr int CH = PairChunk<N>::CH, LOGN = PairChunk<N>::LOGN;
    __shared__ float4 s_row[PAIR_WARPS][CH];
    __shared__ float4 s_tab[UNIFORM ? 1 : MDB_MAX_TYPES * MDB_MAX_TYPES];
    if (!UNIFORM) {
        for (int k = threadIdx.x; k < MDB_MAX_TYPES * MDB_MAX_TYPES; k += blockDim.x)
            s_tab[k] = pt.tab[k];
        __syncthreads();
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) qflag[0] = 0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ci   = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int ncl  = cnt[CP_NCL];
    double e       = 0.0;
    if (ci < ncl) {
        const int h = lane >> 4, s = lane & 15;
        const int jfac = N / 4, ci_cj0 = ci / jfac, ai0 = 4 * (ci % jfac);
        const int nloc = ncl * 4;
        // loads that depend on nothing else
        const int nn          = __ldg(&numneigh[ci]);
        const int* row        = list + (size_t)ci * cs;
        int rw0               = lane < cs ? __ldg(&row[lane]) : 0;
        int rw1               = (CH > 32 && lane + 32 < cs) ? __ldg(&row[lane + 32]) : 0;
        const unsigned char* mycode = pcode + (size_t)(2 * ci + h) * chmax * 256;
        int ncode             = pcnt[(size_t)(2 * ci + h) * chmax];
        int cw[PAIR_BATCH];
#pragma unroll
        for (int m = 0; m < PAIR_BATCH; m++)
            cw[m] = mycode[s + 16 * m];
        const float4 ai = __ldg(&anchor[ci_cj0]);
        bool v0, v1;
        int t0, t1;
        const float4 p0 = i_atom<UNIFORM>(xr, ci * 4 + 2 * h, v0, t0);
        const float4 p1 = i_atom<UNIFORM>(xr, ci * 4 + 2 * h + 1, v1, t1);
        const f2 XI = f2_pack(p0.x, p1.x), YI = f2_pack(p0.y, p1.y), ZI = f2_pack(p0.z, p1.z);
        // exclusion bits of the diagonal entry for the lane's pair: bit 2b + k
        // for i atom 2h + k and atom b of the i-cluster's own j-cluster
        unsigned xtab = 0;
#pragma unroll
        for (int b = 0; b < N; b++)
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const int ia = ai0 + 2 * h + k;
                if (HALF ? (ia >= b) : (ia == b)) xtab |= 1u << (2 * b + k);
            }
        const f2 A2 = f2_pack(pt.a0, pt.a0), mB2 = f2_pack(-pt.b0, -pt.b0);
        f2 fx = 0, fy = 0, fz = 0;
        CompState cst;
        cst.cx = cx, cst.cutsq = cutsq64, cst.si0 = ci * 4 + 2 * h;
        cst.cx_ = cst.cy_ = cst.cz_ = 0;
        const int nch    = (nn + CH - 1) / CH;
        const bool diag0 = nn > 0 && __shfl_sync(0xffffffffu, rw0, 0) == ci_cj0;
        for (int c = 0; c < nch; c++) {
            const int ne = min(CH, nn - c * CH);
            const int ns = ne * N;
            if (c > 0) {
                rw0 = lane < ne ? __ldg(&row[c * CH + lane]) : 0;
                rw1 = (CH > 32 && lane + 32 < ne) ? __ldg(&row[c * CH + lane + 32]) : 0;
                ncode = pcnt[(size_t)(2 * ci + h) * chmax + c];
#pragma unroll
                for (int m = 0; m < PAIR_BATCH; m++)
                    cw[m] = mycode[c * 256 + s + 16 * m];
            }
            if (lane < ne) {
                const float4 a = __ldg(&anchor[rw0]);
                s_row[warp][lane] = make_float4(a.x - ai.x, a.y - ai.y, a.z - ai.z,
                    __int_as_float(rw0 * N));
            }
            if (CH > 32 && lane + 32 < ne) {
                const float4 a = __ldg(&anchor[rw1]);
                s_row[warp][lane + 32] = make_float4(a.x - ai.x, a.y - ai.y, a.z - ai.z,
                    __int_as_float(rw1 * N));
            }
            __syncwarp();
            // codes and counts come from a derivation on the current rows;
            // the clamps keep every access inside this chunk regardless
            ncode = min(ncode, ns);
            for (int base = 0; base < ncode; base += 16 * PAIR_BATCH) {
                if (base > 0) {
#pragma unroll
                    for (int m = 0; m < PAIR_BATCH; m++) {
                        const int k = base + s + 16 * m;
                        cw[m]       = k < ncode ? mycode[c * 256 + k] : 0;
                    }
                }
                float4 xj[PAIR_BATCH], dj[PAIR_BATCH];
                bool ok[PAIR_BATCH];
#pragma unroll
                for (int m = 0; m < PAIR_BATCH; m++) {
                    ok[m] = base + s + 16 * m < ncode && cw[m] < ns;
                    dj[m] = s_row[warp][ok[m] ? cw[m] >> LOGN : 0];
                }
#pragma unroll
                for (int m = 0; m < PAIR_BATCH; m++)
                    if (ok[m]) xj[m] = __ldg(&xr[__float_as_int(dj[m].w) + (cw[m] & (N - 1))]);
#pragma unroll
                for (int m = 0; m < PAIR_BATCH; m++) {
                    if (!ok[m]) continue;
                    const int q  = cw[m];
                    const int sj = __float_as_int(dj[m].w) + (q & (N - 1));
                    // into the i frame: the same roundings as the cluster-pair kernel
                    float4 x     = xj[m];
                    const f2 jxy = f2_add(f2_pack(x.x, x.y), f2_pack(dj[m].x, dj[m].y));
                    f2_unpack(jxy, x.x, x.y);
                    x.z += dj[m].z;
                    const unsigned ex = (c == 0 && diag0 && q < N) ? (xtab >> (2 * q)) & 3u : 0u;
                    pair2<HALF, ENERGY, UNIFORM, COMP>(XI, YI, ZI, x, sj, ex, t0, t1, s_tab, pt,
                        cutforcesq, A2, mB2, nloc, fx, fy, fz, cf32, cf64, cst, e);
                }
            }
            __syncwarp();
        }
        if (COMP) {
            // each lane's sum and compensation in FP64, reduced over the 16
            // lanes of the pair in FP64
            float a0, a1, b0, b1;
            double d[6];
            f2_unpack(fx, a0, a1);
            f2_unpack(cst.cx_, b0, b1);
            d[0] = (double)a0 + (double)b0, d[3] = (double)a1 + (double)b1;
            f2_unpack(fy, a0, a1);
            f2_unpack(cst.cy_, b0, b1);
            d[1] = (double)a0 + (double)b0, d[4] = (double)a1 + (double)b1;
            f2_unpack(fz, a0, a1);
            f2_unpack(cst.cz_, b0, b1);
            d[2] = (double)a0 + (double)b0, d[5] = (double)a1 + (double)b1;
#pragma unroll
            for (int o = 8; o > 0; o >>= 1)
#pragma unroll
                for (int k = 0; k < 6; k++)
                    d[k] += __shfl_xor_sync(0xffffffffu, d[k], o);
            if (s == 0) {
                double4* dst = &cf64[ci * 4 + 2 * h];
                if (HALF) {
                    if (v0) atomicAdd(&dst[0].x, d[0]), atomicAdd(&dst[0].y, d[1]),
                        atomicAdd(&dst[0].z, d[2]);
                    if (v1) atomicAdd(&dst[1].x, d[3]), atomicAdd(&dst[1].y, d[4]),
                        atomicAdd(&dst[1].z, d[5]);
                } else {
                    if (v0) dst[0] = make_double4(d[0], d[1], d[2], 0.0);
                    if (v1) dst[1] = make_double4(d[3], d[4], d[5], 0.0);
                }
            }
        }
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) {
            fx = f2_add(fx, __shfl_xor_sync(0xffffffffu, fx, o));
            fy = f2_add(fy, __shfl_xor_sync(0xffffffffu, fy, o));
            fz = f2_add(fz, __shfl_xor_sync(0xffffffffu, fz, o));
        }
        if (!COMP && s == 0) {
            float ax, bx, ay, by, az, bz;
            f2_unpack(fx, ax, bx);
            f2_unpack(fy, ay, by);
            f2_unpack(fz, az, bz);
            float4* dst = &cf32[ci * 4 + 2 * h];
            if (HALF) {
                if (v0) red_add4(dst, ax, ay, az);
                if (v1) red_add4(dst + 1, bx, by, bz);
            } else {
                if (v0) dst[0] = make_float4(ax, ay, az, 0.f);
                if (v1) dst[1] = make_float4(bx, by, bz, 0.f);
            }
        }
    }
    if (ENERGY) {
        const double t = block_sum(e);
        if (threadIdx.x == 0) epart[blockIdx.x] = t;
    }
}

int pair_grid(int ncl_cap) { return (int)(((long long)ncl_cap * 32 + PAIR_THREADS - 1) / PAIR_THREADS); }

// one wave of resident derivation blocks (at most the clusters' own grid)
static int derive_grid(int ncl_cap)
{
    static int nsm = 0;
    if (!nsm) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if (nsm < 1) nsm = 1;
    }
    return std::max(1, std::min(pair_grid(ncl_cap), nsm * (2048 / PAIR_THREADS)));
}

template <int N, bool HALF>
static void derive_n(cudaStream_t s, int uniform, int grid, const int* cnt, const float4* xr,
    const float4* anchor, const int* list, int cs, const int* numneigh, float rin2, int* qflag,
    int force, unsigned char* pcode, unsigned short* pcnt, int chmax, float4* xq)
{
    if (uniform)
        k_pair_derive<N, HALF, true><<<grid, PAIR_THREADS, 0, s>>>(cnt, xr, anchor, list, cs,
            numneigh, rin2, qflag, force, pcode, pcnt, chmax, xq);
    else
        k_pair_derive<N, HALF, false><<<grid, PAIR_THREADS, 0, s>>>(cnt, xr, anchor, list, cs,
            numneigh, rin2, qflag, force, pcode, pcnt, chmax, xq);
}

void launch_pair_derive(cudaStream_t s, int N, int half, int uniform, int ncl_cap,
    const int* cnt, const float4* xr, const float4* anchor, const int* list, int cs,
    const int* numneigh, float rin2, int* qflag, int force, unsigned char* pcode,
    unsigned short* pcnt, int chmax, float4* xq)
{
    const int grid = derive_grid(ncl_cap);
    if (N == 4) {
        if (half) derive_n<4, true>(s, uniform, grid, cnt, xr, anchor, list, cs, numneigh, rin2, qflag, force, pcode, pcnt, chmax, xq);
        else derive_n<4, false>(s, uniform, grid, cnt, xr, anchor, list, cs, numneigh, rin2, qflag, force, pcode, pcnt, chmax, xq);
    } else {
        if (half) derive_n<8, true>(s, uniform, grid, cnt, xr, anchor, list, cs, numneigh, rin2, qflag, force, pcode, pcnt, chmax, xq);
        else derive_n<8, false>(s, uniform, grid, cnt, xr, anchor, list, cs, numneigh, rin2, qflag, force, pcode, pcnt, chmax, xq);
    }
    g_launches++;
}

template <int N, bool HALF, bool ENERGY, bool UNIFORM>
static void pairs_v(cudaStream_t s, int variant, int grid, const int* cnt, const float4* xr,
    const float4* anchor, const PairTypes& pt, float cutforcesq, const int* list, int cs,
    const int* numneigh, const unsigned char* pcode, const unsigned short* pcnt, int chmax,
    float4* cf32, double* epart, int* qflag, const CompArgs& ca)
{
    if (ca.cf64) { // compensated: the default shape
        k_force_pairs<N, HALF, ENERGY, UNIFORM, PAIR_VARIANTS[0][0], PAIR_VARIANTS[0][1], true>
            <<<grid, PAIR_THREADS, 0, s>>>(cnt, xr, anchor, pt, cutforcesq, list, cs, numneigh,
                pcode, pcnt, chmax, cf32, epart, qflag, ca.cx, ca.cf64, ca.cutsq);
        return;
    }
#define PAIR_RUN(V)                                                                      \
    k_force_pairs<N, HALF, ENERGY, UNIFORM, PAIR_VARIANTS[V][0], PAIR_VARIANTS[V][1], false> \
        <<<grid, PAIR_THREADS, 0, s>>>(cnt, xr, anchor, pt, cutforcesq, list, cs, numneigh, \
            pcode, pcnt, chmax, cf32, epart, qflag, nullptr, nullptr, 0.0)
    // energy evaluations (every nstat steps) use the default shape
    switch (ENERGY ? 0 : variant) {
    case 1: PAIR_RUN(1); break;
    case 2: PAIR_RUN(2); break;
    case 3: PAIR_RUN(3); break;
    default: PAIR_RUN(0); break;
    }
#undef PAIR_RUN
}

template <int N, bool HALF, bool ENERGY>
static void pairs_e(cudaStream_t s, int uniform, int variant, int grid, const int* cnt,
    const float4* xr, const float4* anchor, const PairTypes& pt, float cutforcesq,
    const int* list, int cs, const int* numneigh, const unsigned char* pcode,
    const unsigned short* pcnt, int chmax, float4* cf32, double* epart, int* qflag,
    const CompArgs& ca)
{
    if (uniform)
        pairs_v<N, HALF, ENERGY, true>(s, variant, grid, cnt, xr, anchor, pt, cutforcesq, list,
            cs, numneigh, pcode, pcnt, chmax, cf32, epart, qflag, ca);
    else
        pairs_v<N, HALF, ENERGY, false>(s, variant, grid, cnt, xr, anchor, pt, cutforcesq, list,
            cs, numneigh, pcode, pcnt, chmax, cf32, epart, qflag, ca);
}

template <int N>
static void pairs_n(cudaStream_t s, int half, int energy, int uniform, int variant, int grid,
    const int* cnt, const float4* xr, const float4* anchor, const PairTypes& pt,
    float cutforcesq, const int* list, int cs, const int* numneigh,
    const unsigned char* pcode, const unsigned short* pcnt, int chmax, float4* cf32,
    double* epart, int* qflag, const CompArgs& ca)
{
    if (half) {
        if (energy) pairs_e<N, true, true>(s, uniform, variant, grid, cnt, xr, anchor, pt, cutforcesq, list, cs, numneigh, pcode, pcnt, chmax, cf32, epart, qflag, ca);
        else pairs_e<N, true, false>(s, uniform, variant, grid, cnt, xr, anchor, pt, cutforcesq, list, cs, numneigh, pcode, pcnt, chmax, cf32, epart, qflag, ca);
    } else {
        if (energy) pairs_e<N, false, true>(s, uniform, variant, grid, cnt, xr, anchor, pt, cutforcesq, list, cs, numneigh, pcode, pcnt, chmax, cf32, epart, qflag, ca);
        else pairs_e<N, false, false>(s, uniform, variant, grid, cnt, xr, anchor, pt, cutforcesq, list, cs, numneigh, pcode, pcnt, chmax, cf32, epart, qflag, ca);
    }
}

int launch_force_pairs(cudaStream_t s, int N, int half, int energy, int uniform, int variant,
    int ncl_cap, const int* cnt, const float4* xr, const float4* anchor, const PairTypes& pt,
    float cutforcesq, const int* list, int cs, const int* numneigh,
    const unsigned char* pcode, const unsigned short* pcnt, int chmax, float4* cf32,
    double* epart, int* qflag, const CompArgs& ca)
{
    const int grid = pair_grid(ncl_cap);
    if (N == 4)
        pairs_n<4>(s, half, energy, uniform, variant, grid, cnt, xr, anchor, pt, cutforcesq,
            list, cs, numneigh, pcode, pcnt, chmax, cf32, epart, qflag, ca);
    else
        pairs_n<8>(s, half, energy, uniform, variant, grid, cnt, xr, anchor, pt, cutforcesq,
            list, cs, numneigh, pcode, pcnt, chmax, cf32, epart, qflag, ca);
    g_launches++;
    return grid;
}

} // namespace cp
} // namespace mdb
