// EAM forces over Verlet lists (computeForceEam, verletlist/force_eam.c:19-228)
// as three kernels: (1) density rho_i and fp_i = F'(rho_i) per local atom,
// (2) fp copied to the ghosts through the ghost map (the mid-step halo),
// (3) pair forces from rho', phi' and fp_i + fp_j.
//
// Thread t handles atom t (or order[t]). Spline tables are re-laid out as rows of 8
// coefficients (one 64-byte row per grid point instead of 56 bytes) so a row
// is two aligned sectors.
// FP64 path: -fmad=false, bit-identical to the reference's strict build.
// Mixed path: pair terms and spline rows in FP32 on cell-relative FP32
// positions (see mdb_force_lj.cu); the density (embedding) sum, F'(rho) and
// all energy sums in FP64.
#include "mdb_internal.cuh"

namespace mdb {

static constexpr int EAM_THREADS = 128;

// one 32-byte row (two float4) in one 256-bit load (sm_100); p 32-byte aligned
__device__ __forceinline__ void ldg_row32(const float4* p, float4& a, float4& b)
{
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z),
          "=f"(b.w)
        : "l"(p));
}
static constexpr int EUNROLL     = 4;

template <bool ENERGY>
__global__ void __launch_bounds__(EAM_THREADS) k_eam_rho_fp64(int nlocal,
    const int* __restrict__ order, const double4* __restrict__ x,
    const int* __restrict__ numneigh, const int* __restrict__ neighbors, int ld,
    double cutforcesq, EamDev e, double* __restrict__ fp, double* __restrict__ epart)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double eng  = 0.0;
    if (t < nlocal) {
        const int i      = order ? order[t] : t;
        const double4 xi = x[i];
        const int n      = numneigh[t];
        const int* nb    = neighbors + t;
        double rhoi      = 0.0;
        auto pair        = [&](const double4& xj) {
            double delx = xi.x - xj.x;
            double dely = xi.y - xj.y;
            double delz = xi.z - xj.z;
            double rsq  = delx * delx + dely * dely + delz * delz;
            if (rsq < cutforcesq) {
                double p = sqrt(rsq) * e.rdr + 1.0;
                int m    = (int)(p);
                m        = m < e.nr - 1 ? m : e.nr - 1;
                p -= m;
                p               = p < 1.0 ? p : 1.0;
                const double* c = e.rhor + 8 * m;
                rhoi += ((__ldg(c + 3) * p + __ldg(c + 4)) * p + __ldg(c + 5)) * p + __ldg(c + 6);
            }
        };
        int k = 0;
        for (; k + EUNROLL <= n; k += EUNROLL) {
            int j[EUNROLL];
            double4 xj[EUNROLL];
#pragma unroll
            for (int u = 0; u < EUNROLL; u++)
                j[u] = __ldcs(nb + (size_t)(k + u) * ld);
#pragma unroll
            for (int u = 0; u < EUNROLL; u++)
                xj[u] = ldg4(x + j[u]);
#pragma unroll
            for (int u = 0; u < EUNROLL; u++)
                pair(xj[u]);
        }
        for (; k < n; k++)
            pair(ldg4(x + __ldcs(nb + (size_t)k * ld)));
        double p = 1.0 * rhoi * e.rdrho + 1.0;
        int m    = (int)(p);
        m        = m < e.nrho - 1 ? m : e.nrho - 1;
        m        = m > 1 ? m : 1;
        p -= m;
        p               = p < 1.0 ? p : 1.0;
        const double* c = e.frho + 8 * m;
        fp[i]           = (__ldg(c + 0) * p + __ldg(c + 1)) * p + __ldg(c + 2);
        if (ENERGY) eng = ((__ldg(c + 3) * p + __ldg(c + 4)) * p + __ldg(c + 5)) * p + __ldg(c + 6);
    }
    if (ENERGY) {
        double s = block_sum(eng);
        if (threadIdx.x == 0) epart[blockIdx.x] = s;
    }
}

__global__ void k_eam_fp_ghost(int nlocal, double* __restrict__ fp,
    const int* __restrict__ border_map, const int* __restrict__ counters)
{
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= counters[CNT_NGHOST]) return;
    fp[nlocal + g] = fp[border_map[g]];
}

template <bool ENERGY>
__global__ void __launch_bounds__(EAM_THREADS) k_eam_force_fp64(int nlocal,
    const int* __restrict__ order, const double4* __restrict__ x,
    const int* __restrict__ numneigh, const int* __restrict__ neighbors, int ld,
    double cutforcesq, EamDev e, const double* __restrict__ fp, double* __restrict__ fx,
    double* __restrict__ fy, double* __restrict__ fz, double* __restrict__ epart)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double eng  = 0.0;
    if (t < nlocal) {
        const int i      = order ? order[t] : t;
        const double4 xi = x[i];
        const int n      = numneigh[t];
        const int* nb    = neighbors + t;
        const double fpi = fp[i];
        double fix = 0.0, fiy = 0.0, fiz = 0.0;
        auto pair = [&](int j, const double4& xj) {
            double delx = xi.x - xj.x;
            double dely = xi.y - xj.y;
            double delz = xi.z - xj.z;
            double rsq  = delx * delx + dely * dely + delz * delz;
            if (rsq < cutforcesq) {
                double r = sqrt(rsq);
                double p = r * e.rdr + 1.0;
                int m    = (int)(p);
                m        = m < e.nr - 1 ? m : e.nr - 1;
                p -= m;
                p                = p < 1.0 ? p : 1.0;
                const double* cr = e.rhor + 8 * m;
                const double* cz = e.z2r + 8 * m;
                double rhoip     = (__ldg(cr + 0) * p + __ldg(cr + 1)) * p + __ldg(cr + 2);
                double z2p       = (__ldg(cz + 0) * p + __ldg(cz + 1)) * p + __ldg(cz + 2);
                double z2 = ((__ldg(cz + 3) * p + __ldg(cz + 4)) * p + __ldg(cz + 5)) * p +
                            __ldg(cz + 6);
                double recip = 1.0 / r;
                double phi   = z2 * recip;
                double phip  = z2p * recip - phi * recip;
                double psip  = fpi * rhoip + __ldg(fp + j) * rhoip + phip;
                double fpair = -psip * recip;
                fix += delx * fpair;
                fiy += dely * fpair;
                fiz += delz * fpair;
                if (ENERGY) eng += 0.5 * phi;
            }
        };
        int k = 0;
        for (; k + EUNROLL <= n; k += EUNROLL) {
            int j[EUNROLL];
            double4 xj[EUNROLL];
#pragma unroll
            for (int u = 0; u < EUNROLL; u++)
                j[u] = __ldcs(nb + (size_t)(k + u) * ld);
#pragma unroll
            for (int u = 0; u < EUNROLL; u++)
                xj[u] = ldg4(x + j[u]);
#pragma unroll
            for (int u = 0; u < EUNROLL; u++)
                pair(j[u], xj[u]);
        }
        for (; k < n; k++) {
            int j = __ldcs(nb + (size_t)k * ld);
            pair(j, ldg4(x + j));
        }
        fx[i] = fix;
        fy[i] = fiy;
        fz[i] = fiz;
    }
    if (ENERGY) {
        double s = block_sum(eng);
        if (threadIdx.x == 0) epart[blockIdx.x] = s;
    }
}

// ---- mixed ------------------------------------------------------------------
// Thread t handles atom t. The density pass also writes, per atom, the list
// entries inside the cutoff in list order (cut, laid out like the list, and
// their count ncut), and xe = (position, F'(rho)) of the atom; k_eam_xe_ghost
// writes xe of every ghost. The force pass then runs over the in-cutoff
// entries only and gathers a neighbour's position and F'(rho_j) in one
// 16-byte load: the same pairs in the same order as a pass over the whole list
// that skips the rest, without the skin entries (about 40 % of a list at
// r_c + 1 A) and without a cutoff branch that diverges inside a warp. The two
// passes compute rsq from the same FP32 values with the same operations, so
// every entry of cut is inside the cutoff in the force pass too.
int eam_mixed_blocks(int nlocal) { return mdb_blocks(nlocal, EAM_THREADS); }

template <bool ENERGY>
__global__ void __launch_bounds__(EAM_THREADS) k_eam_rho_mixed(int nlocal,
    const float4* __restrict__ xr, CellShift sh, const int* __restrict__ numneigh,
    const int* __restrict__ neighbors, int ld, float cutforcesq, EamDev e,
    int* __restrict__ cut, int* __restrict__ ncut, double* __restrict__ fp,
    float4* __restrict__ xe, double* __restrict__ epart)
{
    const float cg = sh.g;
    const int i    = blockIdx.x * blockDim.x + threadIdx.x;
    double eng     = 0.0;
    if (i < nlocal) {
        const float4 pi = xr[i];
        const int n     = numneigh[i];
        const int* nb   = neighbors + i;
        int* out        = cut + i;
        int c           = 0;
        double rhoi     = 0.0; // FP64 embedding (density) sum
        const float rdr = (float)e.rdr;
        auto pair       = [&](int en, const float4& pj) {
            float dx, dy, dz;
            cell_delta(pi, pj, (unsigned)en >> MDB_IDX_BITS, cg, dx, dy, dz);
            float rsq = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, dz * dz));
            if (rsq < cutforcesq) {
                float p = __fmaf_rn(sqrtf(rsq), rdr, 1.0f);
                int m   = (int)p;
                m       = m < e.nr - 1 ? m : e.nr - 1;
                p -= (float)m;
                p              = p < 1.0f ? p : 1.0f;
                const float4 a = __ldg(e.dens32 + m); // coefficients 3..6
                rhoi += (double)__fmaf_rn(__fmaf_rn(__fmaf_rn(a.x, p, a.y), p, a.z), p, a.w);
                __stcg(out + (size_t)c * ld, en);
                c++;
            }
        };
        int k = 0;
        for (; k + EUNROLL <= n; k += EUNROLL) {
            int en[EUNROLL];
            float4 pj[EUNROLL];
#pragma unroll
            for (int v = 0; v < EUNROLL; v++)
                en[v] = __ldcs(nb + (size_t)(k + v) * ld);
#pragma unroll
            for (int v = 0; v < EUNROLL; v++)
                pj[v] = __ldg(xr + (en[v] & MDB_IDX_MASK));
#pragma unroll
            for (int v = 0; v < EUNROLL; v++)
                pair(en[v], pj[v]);
        }
        for (; k < n; k++) {
            const int en = __ldcs(nb + (size_t)k * ld);
            pair(en, __ldg(xr + (en & MDB_IDX_MASK)));
        }
        ncut[i]   = c;
        double p = 1.0 * rhoi * e.rdrho + 1.0;
        int m    = (int)(p);
        m        = m < e.nrho - 1 ? m : e.nrho - 1;
        m        = m > 1 ? m : 1;
        p -= m;
        p                = p < 1.0 ? p : 1.0;
        const double* cf = e.frho + 8 * m;
        const double fpi = (__ldg(cf + 0) * p + __ldg(cf + 1)) * p + __ldg(cf + 2);
        fp[i]            = fpi;
        xe[i]            = make_float4(pi.x, pi.y, pi.z, (float)fpi);
        if (ENERGY) eng = ((__ldg(cf + 3) * p + __ldg(cf + 4)) * p + __ldg(cf + 5)) * p + __ldg(cf + 6);
    }
    if (ENERGY) {
        double s = block_sum(eng);
        if (threadIdx.x == 0) epart[blockIdx.x] = s;
    }
}

// The density pass with two lanes per atom (lanes 2q and 2q + 1 of a warp on
// atom 16 w + q): the lanes take list entries k and k + 1 of each pair and
// append the in-cutoff ones to cut in list order (the lower lane's first), so
// the force pass reads the same rows as after the one-lane pass; the two FP64
// partial densities are added at the end. Twice the warps of the one-lane pass
// keep more gathers in flight on a 131k-atom system. Blocks of 2 x EAM_THREADS
// threads cover the same EAM_THREADS atoms as a block of the one-lane pass, so
// both write the same energy partials.
template <bool ENERGY>
__global__ void __launch_bounds__(2 * EAM_THREADS) k_eam_rho_mixed2(int nlocal,
    const float4* __restrict__ xr, CellShift sh, const int* __restrict__ numneigh,
    const int* __restrict__ neighbors, int ld, float cutforcesq, EamDev e,
    int* __restrict__ cut, int* __restrict__ ncut, double* __restrict__ fp,
    float4* __restrict__ xe, double* __restrict__ epart)
{
    const float cg  = sh.g;
    const int lane  = threadIdx.x & 31;
    const int u     = lane & 1;
    const int i     = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 16 + (lane >> 1);
    const bool act  = i < nlocal;
    const int ia    = act ? i : 0;
    const float4 pi = act ? xr[ia] : make_float4(0.f, 0.f, 0.f, 0.f);
    const int n     = act ? numneigh[ia] : 0;
    const int* nb   = neighbors + ia;
    int* out        = cut + ia;
    int c           = 0;     // entries appended so far (both lanes)
    double rhoi     = 0.0;   // this lane's FP64 partial density
    double eng      = 0.0;
    const float rdr = (float)e.rdr;
    const unsigned pairmask = 3u << (lane & ~1);
    auto pair = [&](int en, const float4& pj, bool valid) {
        bool in = false;
        if (valid) {
            float dx, dy, dz;
            cell_delta(pi, pj, (unsigned)en >> MDB_IDX_BITS, cg, dx, dy, dz);
            const float rsq = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, dz * dz));
            in              = rsq < cutforcesq;
            if (in) {
                float p = __fmaf_rn(sqrtf(rsq), rdr, 1.0f);
                int m   = (int)p;
                m       = m < e.nr - 1 ? m : e.nr - 1;
                p -= (float)m;
                p              = p < 1.0f ? p : 1.0f;
                const float4 a = __ldg(e.dens32 + m); // coefficients 3..6
                rhoi += (double)__fmaf_rn(__fmaf_rn(__fmaf_rn(a.x, p, a.y), p, a.z), p, a.w);
            }
        }
        const unsigned bal = __ballot_sync(0xffffffffu, in) & pairmask;
        if (in) __stcg(out + (size_t)(c + (u ? __popc(bal) - 1 : 0)) * ld, en);
        c += __popc(bal);
    };
    // a warp runs as many pair steps as its longest row
    int nmax = n;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nmax = max(nmax, __shfl_xor_sync(0xffffffffu, nmax, o));
    int k = 0;
    for (; k + 2 * EUNROLL <= nmax; k += 2 * EUNROLL) {
        int en[EUNROLL];
        float4 pj[EUNROLL];
#pragma unroll
        for (int v = 0; v < EUNROLL; v++) {
            const int kk = k + 2 * v + u;
            en[v]        = kk < n ? __ldcs(nb + (size_t)kk * ld) : 0;
        }
#pragma unroll
        for (int v = 0; v < EUNROLL; v++)
            pj[v] = k + 2 * v + u < n ? __ldg(xr + (en[v] & MDB_IDX_MASK)) : pi;
#pragma unroll
        for (int v = 0; v < EUNROLL; v++)
            pair(en[v], pj[v], k + 2 * v + u < n);
    }
    for (; k < nmax; k += 2) {
        const bool valid = k + u < n;
        const int en     = valid ? __ldcs(nb + (size_t)(k + u) * ld) : 0;
        pair(en, valid ? __ldg(xr + (en & MDB_IDX_MASK)) : pi, valid);
    }
    rhoi += __shfl_xor_sync(0xffffffffu, rhoi, 1);
    if (act && u == 0) {
        ncut[i]  = c;
        double p = 1.0 * rhoi * e.rdrho + 1.0;
        int m    = (int)(p);
        m        = m < e.nrho - 1 ? m : e.nrho - 1;
        m        = m > 1 ? m : 1;
        p -= m;
        p                = p < 1.0 ? p : 1.0;
        const double* cf = e.frho + 8 * m;
        const double fpi = (__ldg(cf + 0) * p + __ldg(cf + 1)) * p + __ldg(cf + 2);
        fp[i]            = fpi;
        xe[i]            = make_float4(pi.x, pi.y, pi.z, (float)fpi);
        if (ENERGY) eng = ((__ldg(cf + 3) * p + __ldg(cf + 4)) * p + __ldg(cf + 5)) * p + __ldg(cf + 6);
    }
    if (ENERGY) {
        double s = block_sum(eng);
        if (threadIdx.x == 0) epart[blockIdx.x] = s;
    }
}

// F'(rho) of the ghosts from their owners (the mid-step halo of
// computeForceEam, verletlist/force_eam.c:120-130), with their positions
__global__ void k_eam_xe_ghost(int nlocal, const float4* __restrict__ xr,
    double* __restrict__ fp, float4* __restrict__ xe, const int* __restrict__ border_map,
    const int* __restrict__ counters)
{
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= counters[CNT_NGHOST]) return;
    const double f   = fp[border_map[g]];
    const float4 p   = xr[nlocal + g];
    fp[nlocal + g]   = f;
    xe[nlocal + g]   = make_float4(p.x, p.y, p.z, (float)f);
}

// COMP: Knuth two-sum compensated force sums (MDB_PREC_MIXED_COMP)
template <bool ENERGY, bool COMP>
__global__ void __launch_bounds__(EAM_THREADS) k_eam_force_mixed(int nlocal,
    const float4* __restrict__ xe, CellShift sh, const int* __restrict__ ncut,
    const int* __restrict__ cut, int ld, EamDev e, double* __restrict__ fx,
    double* __restrict__ fy, double* __restrict__ fz, double* __restrict__ epart)
{
    const float cg = sh.g;
    const int i    = blockIdx.x * blockDim.x + threadIdx.x;
    double eng     = 0.0;
    if (i < nlocal) {
        const float4 pi = xe[i];
        const int n     = ncut[i];
        const int* nb   = cut + i;
        const float fpi = pi.w;
        const float rdr = (float)e.rdr;
        const float rdr2 = 2.0f * rdr;
        float fix = 0.f, fiy = 0.f, fiz = 0.f;
        float cx = 0.f, cy = 0.f, cz = 0.f; // compensation terms
        auto acc = [&](float& s, float& c, float d, float f) {
            if (COMP) { // s + c carries the running sum exactly
                float v  = d * f;
                float w  = s + v;
                float bp = w - s;
                float r  = (s - (w - bp)) + (v - bp);
                s        = w;
                c += r;
            } else {
                s = __fmaf_rn(d, f, s);
            }
        };
        auto pair = [&](int en, const float4& pj) {
            float dx, dy, dz;
            cell_delta(pi, pj, (unsigned)en >> MDB_IDX_BITS, cg, dx, dy, dz);
            const float rsq = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, dz * dz));
            const float r   = sqrtf(rsq);
            float p         = __fmaf_rn(r, rdr, 1.0f);
            int m           = (int)p;
            m               = m < e.nr - 1 ? m : e.nr - 1;
            p -= (float)m;
            p               = p < 1.0f ? p : 1.0f;
            // z2r coefficients 3..6, then rho 0..2 and z2r 0; z2r 1 and 2 are
            // 2 c4 / dr and c5 / dr (spline7's derivative rows)
            float4 za, rb;
            ldg_row32(e.pair32 + 2 * m, za, rb);
            float rhoip = __fmaf_rn(__fmaf_rn(rb.x, p, rb.y), p, rb.z);
            float z2p   = __fmaf_rn(__fmaf_rn(rb.w, p, za.y * rdr2), p, za.z * rdr);
            float z2    = __fmaf_rn(__fmaf_rn(__fmaf_rn(za.x, p, za.y), p, za.z), p, za.w);
            float recip = __fdividef(1.0f, r);
            float phi   = z2 * recip;
            float phip  = __fmaf_rn(z2p, recip, -phi * recip);
            float psip  = __fmaf_rn(fpi + pj.w, rhoip, phip);
            float fpair = -psip * recip;
            acc(fix, cx, dx, fpair);
            acc(fiy, cy, dy, fpair);
            acc(fiz, cz, dz, fpair);
            if (ENERGY) eng += 0.5 * (double)phi;
        };
        int k = 0;
        for (; k + EUNROLL <= n; k += EUNROLL) {
            int en[EUNROLL];
            float4 pj[EUNROLL];
#pragma unroll
            for (int v = 0; v < EUNROLL; v++)
                en[v] = __ldcs(nb + (size_t)(k + v) * ld);
#pragma unroll
            for (int v = 0; v < EUNROLL; v++)
                pj[v] = __ldg(xe + (en[v] & MDB_IDX_MASK));
#pragma unroll
            for (int v = 0; v < EUNROLL; v++)
                pair(en[v], pj[v]);
        }
        for (; k < n; k++) {
            const int en = __ldcs(nb + (size_t)k * ld);
            pair(en, __ldg(xe + (en & MDB_IDX_MASK)));
        }
        fx[i] = (double)fix + (double)cx;
        fy[i] = (double)fiy + (double)cy;
        fz[i] = (double)fiz + (double)cz;
    }
    if (ENERGY) {
        double s = block_sum(eng);
        if (threadIdx.x == 0) epart[blockIdx.x] = s;
    }
}

static void fp_ghost(cudaStream_t s, int nlocal, int ghost_cap, double* fp,
    const int* border_map, const int* counters)
{
    if (ghost_cap <= 0) return;
    k_eam_fp_ghost<<<mdb_blocks(ghost_cap, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(nlocal, fp,
        border_map, counters);
    g_launches++;
}

void launch_eam_fp64(cudaStream_t s, int energy, int nlocal, int ghost_cap, const int* order,
    const double4* x, const int* numneigh, const int* neighbors, int ld, double cutforcesq,
    EamDev eam, const int* border_map, const int* counters, double* fp, double* fx,
    double* fy, double* fz, double* epart_rho, double* epart_pair)
{
    if (nlocal <= 0) return;
    int nb = mdb_blocks(nlocal, EAM_THREADS);
    if (energy)
        k_eam_rho_fp64<true><<<nb, EAM_THREADS, 0, s>>>(nlocal, order, x, numneigh, neighbors,
            ld, cutforcesq, eam, fp, epart_rho);
    else
        k_eam_rho_fp64<false><<<nb, EAM_THREADS, 0, s>>>(nlocal, order, x, numneigh, neighbors,
            ld, cutforcesq, eam, fp, epart_rho);
    g_launches++;
    fp_ghost(s, nlocal, ghost_cap, fp, border_map, counters);
    if (energy)
        k_eam_force_fp64<true><<<nb, EAM_THREADS, 0, s>>>(nlocal, order, x, numneigh,
            neighbors, ld, cutforcesq, eam, fp, fx, fy, fz, epart_pair);
    else
        k_eam_force_fp64<false><<<nb, EAM_THREADS, 0, s>>>(nlocal, order, x, numneigh,
            neighbors, ld, cutforcesq, eam, fp, fx, fy, fz, epart_pair);
    g_launches++;
}

int launch_eam_mixed(cudaStream_t s, int energy, int comp, int rho_lanes, int nlocal,
    int ghost_cap,
    const float4* xr, const CellShift& sh, const int* numneigh, const int* neighbors, int ld,
    float cutforcesq, EamDev eam, const int* border_map, const int* counters, int* cut,
    int* ncut, double* fp, float4* xe, double* fx, double* fy, double* fz, double* epart_rho,
    double* epart_pair)
{
    if (nlocal <= 0) return 0;
    const int nb = eam_mixed_blocks(nlocal);
    if (rho_lanes == 2) {
        if (energy)
            k_eam_rho_mixed2<true><<<nb, 2 * EAM_THREADS, 0, s>>>(nlocal, xr, sh, numneigh,
                neighbors, ld, cutforcesq, eam, cut, ncut, fp, xe, epart_rho);
        else
            k_eam_rho_mixed2<false><<<nb, 2 * EAM_THREADS, 0, s>>>(nlocal, xr, sh, numneigh,
                neighbors, ld, cutforcesq, eam, cut, ncut, fp, xe, epart_rho);
    } else if (energy)
        k_eam_rho_mixed<true><<<nb, EAM_THREADS, 0, s>>>(nlocal, xr, sh, numneigh, neighbors,
            ld, cutforcesq, eam, cut, ncut, fp, xe, epart_rho);
    else
        k_eam_rho_mixed<false><<<nb, EAM_THREADS, 0, s>>>(nlocal, xr, sh, numneigh, neighbors,
            ld, cutforcesq, eam, cut, ncut, fp, xe, epart_rho);
    g_launches++;
    if (ghost_cap > 0) {
        k_eam_xe_ghost<<<mdb_blocks(ghost_cap, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(nlocal, xr,
            fp, xe, border_map, counters);
        g_launches++;
    }
#define EAM_FM(E, C)                                                                     \
    k_eam_force_mixed<E, C><<<nb, EAM_THREADS, 0, s>>>(nlocal, xe, sh, ncut, cut, ld, eam, fx, \
        fy, fz, epart_pair)
    if (energy) {
        if (comp) EAM_FM(true, true);
        else EAM_FM(true, false);
    } else {
        if (comp) EAM_FM(false, true);
        else EAM_FM(false, false);
    }
#undef EAM_FM
    g_launches++;
    return nb;
}

} // namespace mdb
