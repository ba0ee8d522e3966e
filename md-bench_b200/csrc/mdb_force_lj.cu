// Lennard-Jones forces over Verlet lists (computeForceLJFullNeigh /
// computeForceLJHalfNeigh, verletlist/force_lj.c:17-206).
//
// Thread t handles atom i = t (or order[t] when an order is given) and reads
// row t of the list. The list is k-major, so each step of the k loop is one 128-byte coalesced
// read per warp; neighbour positions are 32-byte (FP64) or 16-byte (mixed)
// gathers that mostly hit L1/L2. The k loop is unrolled by UNROLL with all
// list reads and gathers of a batch issued before any arithmetic, which keeps
// enough bytes in flight for the HBM-bound list stream. Pairs are summed in
// list order.
//
// FP64 path: -fmad=false keeps every product and sum rounded as the
// reference's strict build rounds them, so full-list forces are bit-identical.
// Mixed path: FP32 positions relative to the centre of each atom's cell (edge
// G, a power of two) plus the cell offset of the pair (-1, 0, +1 per axis,
// 2-bit fields of the list entry): dx = (p_i - p_j) - offset * G, the offset
// decoded into an exact float with integer bit operations. No int->float
// conversions, no shared-memory table, one approximate reciprocal per pair;
// FP32 force sums (or two-sum compensated sums), FP64 energy sums.
#include "mdb_internal.cuh"

namespace mdb {

static constexpr int LJ_THREADS = 128;
static constexpr int UNROLL     = 8;

int force_partial_blocks(int n) { return mdb_blocks(n > 0 ? n : 1, LJ_THREADS); }

template <bool HALF, bool UNIFORM, bool ENERGY>
__global__ void __launch_bounds__(LJ_THREADS) k_lj_fp64(int nlocal,
    const int* __restrict__ order, const double4* __restrict__ x,
    const int* __restrict__ numneigh, const int* __restrict__ neighbors, int ld,
    double cutforcesq, LJTable tab, double* __restrict__ fx, double* __restrict__ fy,
    double* __restrict__ fz, double* __restrict__ epart)
{
    __shared__ double s_eps[MDB_MAX_TYPES * MDB_MAX_TYPES];
    __shared__ double s_sig6[MDB_MAX_TYPES * MDB_MAX_TYPES];
    const int nt = tab.ntypes;
    if (!UNIFORM) {
        for (int k = threadIdx.x; k < nt * nt; k += blockDim.x) {
            s_eps[k]  = tab.eps[k];
            s_sig6[k] = tab.sig6[k];
        }
        __syncthreads();
    }
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double epot = 0.0;
    if (t < nlocal) {
        const int i      = order ? order[t] : t;
        const double4 xi = x[i];
        const int ti     = type_of(xi);
        const int n      = numneigh[t];
        const int* nb    = neighbors + t;
        double fix = 0.0, fiy = 0.0, fiz = 0.0;
        const double eps0 = tab.eps[0], sig0 = tab.sig6[0];

        auto pair = [&](int j, const double4& xj) {
            double delx = xi.x - xj.x;
            double dely = xi.y - xj.y;
            double delz = xi.z - xj.z;
            double rsq  = delx * delx + dely * dely + delz * delz;
            double sigma6 = sig0, epsilon = eps0;
            if (!UNIFORM) {
                int tij = ti * nt + type_of(xj);
                sigma6  = s_sig6[tij];
                epsilon = s_eps[tij];
            }
            if (rsq < cutforcesq) {
                double sr2   = 1.0 / rsq;
                double sr6   = sr2 * sr2 * sr2 * sigma6;
                double force = 48.0 * sr6 * (sr6 - 0.5) * sr2 * epsilon;
                fix += delx * force;
                fiy += dely * force;
                fiz += delz * force;
                if (HALF && j < nlocal) {
                    atomicAdd(&fx[j], -(delx * force));
                    atomicAdd(&fy[j], -(dely * force));
                    atomicAdd(&fz[j], -(delz * force));
                }
                if (ENERGY) {
                    double e = 4.0 * epsilon * sr6 * (sr6 - 1.0);
                    epot += (HALF && j < nlocal) ? e : 0.5 * e;
                }
            }
        };

        int k = 0;
        for (; k + UNROLL <= n; k += UNROLL) {
            int j[UNROLL];
            double4 xj[UNROLL];
#pragma unroll
            for (int u = 0; u < UNROLL; u++)
                j[u] = __ldcs(nb + (size_t)(k + u) * ld);
#pragma unroll
            for (int u = 0; u < UNROLL; u++)
                xj[u] = ldg4(x + j[u]);
#pragma unroll
            for (int u = 0; u < UNROLL; u++)
                pair(j[u], xj[u]);
        }
        for (; k < n; k++) {
            int j = __ldcs(nb + (size_t)k * ld);
            pair(j, ldg4(x + j));
        }
        if (HALF) {
            atomicAdd(&fx[i], fix);
            atomicAdd(&fy[i], fiy);
            atomicAdd(&fz[i], fiz);
        } else {
            fx[i] = fix;
            fy[i] = fiy;
            fz[i] = fiz;
        }
    }
    if (ENERGY) {
        double e = block_sum(epot);
        if (threadIdx.x == 0) epart[blockIdx.x] = e;
    }
}

template <bool HALF, bool UNIFORM, bool ENERGY, bool COMP>
__global__ void __launch_bounds__(LJ_THREADS) k_lj_mixed(int nlocal,
    const int* __restrict__ order, const float4* __restrict__ xr, CellShift sh,
    const int* __restrict__ numneigh, const int* __restrict__ neighbors, int ld,
    float cutforcesq, LJTableF tab, double* __restrict__ fx, double* __restrict__ fy,
    double* __restrict__ fz, double* __restrict__ epart)
{
    __shared__ float s_eps[MDB_MAX_TYPES * MDB_MAX_TYPES];
    __shared__ float s_sig6[MDB_MAX_TYPES * MDB_MAX_TYPES];
    const int nt = tab.ntypes;
    if (!UNIFORM) {
        for (int k = threadIdx.x; k < nt * nt; k += blockDim.x) {
            s_eps[k]  = tab.eps[k];
            s_sig6[k] = tab.sig6[k];
        }
        __syncthreads();
    }
    const float cg = sh.g;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double epot = 0.0;
    if (t < nlocal) {
        const int i     = order ? order[t] : t;
        const float4 pi = xr[i];
        const int ti    = __float_as_int(pi.w);
        const int n     = numneigh[t];
        const int* nb   = neighbors + t;
        float fix = 0.f, fiy = 0.f, fiz = 0.f;
        float cx = 0.f, cy = 0.f, cz = 0.f; // compensation terms
        const float eps0 = tab.eps[0], sig0 = tab.sig6[0];
        // one type: force / r = sr2 s (A s - B), s = 1 / r^6, A = 48 eps sigma^12,
        // B = 24 eps sigma^6
        const float cA = 48.0f * eps0 * sig0 * sig0, cB = 24.0f * eps0 * sig0;

        auto acc = [&](float& s, float& c, float d, float f) {
            if (COMP) { // Knuth two-sum: s + c carries the running sum exactly
                float v  = d * f;
                float u  = s + v;
                float bp = u - s;
                float e  = (s - (u - bp)) + (v - bp);
                s        = u;
                c += e;
            } else {
                s = __fmaf_rn(d, f, s);
            }
        };

        auto pair = [&](int e, const float4& pj) {
            const int j = e & MDB_IDX_MASK;
            float delx, dely, delz;
            cell_delta(pi, pj, (unsigned)e >> MDB_IDX_BITS, cg, delx, dely, delz);
            float rsq = __fmaf_rn(delx, delx, __fmaf_rn(dely, dely, delz * delz));
            float sigma6 = sig0, epsilon = eps0;
            if (!UNIFORM) {
                int tij = ti * nt + __float_as_int(pj.w);
                sigma6  = s_sig6[tij];
                epsilon = s_eps[tij];
            }
            if (UNIFORM && !HALF && !ENERGY && !COMP) {
                // one type, full lists: no branch; pairs outside the cutoff
                // add exact zeros (the same sums as the branch)
                const float sr2 = __fdividef(1.0f, rsq);
                const float s3  = sr2 * sr2 * sr2;
                float force     = sr2 * s3 * __fmaf_rn(cA, s3, -cB);
                force           = rsq < cutforcesq ? force : 0.0f;
                fix             = __fmaf_rn(delx, force, fix);
                fiy             = __fmaf_rn(dely, force, fiy);
                fiz             = __fmaf_rn(delz, force, fiz);
            } else if (rsq < cutforcesq) {
                float sr2 = __fdividef(1.0f, rsq);
                float sr6, force;
                if (UNIFORM) {
                    const float s3 = sr2 * sr2 * sr2;
                    sr6            = s3 * sigma6;
                    force          = sr2 * s3 * __fmaf_rn(cA, s3, -cB);
                } else {
                    sr6   = sr2 * sr2 * sr2 * sigma6;
                    force = 48.0f * sr6 * (sr6 - 0.5f) * sr2 * epsilon;
                }
                acc(fix, cx, delx, force);
                acc(fiy, cy, dely, force);
                acc(fiz, cz, delz, force);
                if (HALF && j < nlocal) {
                    atomicAdd(&fx[j], -(double)(delx * force));
                    atomicAdd(&fy[j], -(double)(dely * force));
                    atomicAdd(&fz[j], -(double)(delz * force));
                }
                if (ENERGY) {
                    double en = (double)(4.0f * epsilon * sr6 * (sr6 - 1.0f));
                    epot += (HALF && j < nlocal) ? en : 0.5 * en;
                }
            }
        };

        int k = 0;
        for (; k + UNROLL <= n; k += UNROLL) {
            int e[UNROLL];
            float4 pj[UNROLL];
#pragma unroll
            for (int u = 0; u < UNROLL; u++)
                e[u] = __ldcs(nb + (size_t)(k + u) * ld);
#pragma unroll
            for (int u = 0; u < UNROLL; u++)
                pj[u] = __ldg(xr + (e[u] & MDB_IDX_MASK));
#pragma unroll
            for (int u = 0; u < UNROLL; u++)
                pair(e[u], pj[u]);
        }
        for (; k < n; k++) {
            int e = __ldcs(nb + (size_t)k * ld);
            pair(e, __ldg(xr + (e & MDB_IDX_MASK)));
        }
        double rx = (double)fix + (double)cx;
        double ry = (double)fiy + (double)cy;
        double rz = (double)fiz + (double)cz;
        if (HALF) {
            atomicAdd(&fx[i], rx);
            atomicAdd(&fy[i], ry);
            atomicAdd(&fz[i], rz);
        } else {
            fx[i] = rx;
            fy[i] = ry;
            fz[i] = rz;
        }
    }
    if (ENERGY) {
        double e = block_sum(epot);
        if (threadIdx.x == 0) epart[blockIdx.x] = e;
    }
}

template <bool HALF, bool UNIFORM>
static void lj64(cudaStream_t s, int energy, int nb, int nlocal, const int* order,
    const double4* x, const int* numneigh, const int* neighbors, int ld, double cut,
    const LJTable& tab, double* fx, double* fy, double* fz, double* epart)
{
    if (energy)
        k_lj_fp64<HALF, UNIFORM, true><<<nb, LJ_THREADS, 0, s>>>(nlocal, order, x, numneigh,
            neighbors, ld, cut, tab, fx, fy, fz, epart);
    else
        k_lj_fp64<HALF, UNIFORM, false><<<nb, LJ_THREADS, 0, s>>>(nlocal, order, x, numneigh,
            neighbors, ld, cut, tab, fx, fy, fz, epart);
}

void launch_lj_fp64(cudaStream_t s, int half, int energy, int nlocal, const int* order,
    const double4* x, const int* numneigh, const int* neighbors, int ld, double cutforcesq,
    const LJTable& tab, double* fx, double* fy, double* fz, double* epart)
{
    if (nlocal <= 0) return;
    int nb = force_partial_blocks(nlocal);
    if (half) {
        if (tab.uniform)
            lj64<true, true>(s, energy, nb, nlocal, order, x, numneigh, neighbors, ld,
                cutforcesq, tab, fx, fy, fz, epart);
        else
            lj64<true, false>(s, energy, nb, nlocal, order, x, numneigh, neighbors, ld,
                cutforcesq, tab, fx, fy, fz, epart);
    } else {
        if (tab.uniform)
            lj64<false, true>(s, energy, nb, nlocal, order, x, numneigh, neighbors, ld,
                cutforcesq, tab, fx, fy, fz, epart);
        else
            lj64<false, false>(s, energy, nb, nlocal, order, x, numneigh, neighbors, ld,
                cutforcesq, tab, fx, fy, fz, epart);
    }
    g_launches++;
}

template <bool HALF, bool UNIFORM, bool COMP>
static void ljmx(cudaStream_t s, int energy, int nb, int nlocal, const int* order,
    const float4* xr, const CellShift& sh, const int* numneigh, const int* neighbors, int ld,
    float cut, const LJTableF& tab, double* fx, double* fy, double* fz, double* epart)
{
    if (energy)
        k_lj_mixed<HALF, UNIFORM, true, COMP><<<nb, LJ_THREADS, 0, s>>>(nlocal, order, xr, sh,
            numneigh, neighbors, ld, cut, tab, fx, fy, fz, epart);
    else
        k_lj_mixed<HALF, UNIFORM, false, COMP><<<nb, LJ_THREADS, 0, s>>>(nlocal, order, xr, sh,
            numneigh, neighbors, ld, cut, tab, fx, fy, fz, epart);
}

template <bool HALF, bool COMP>
static void ljmx_u(cudaStream_t s, int energy, int nb, int nlocal, const int* order,
    const float4* xr, const CellShift& sh, const int* numneigh, const int* neighbors, int ld,
    float cut, const LJTableF& tab, double* fx, double* fy, double* fz, double* epart)
{
    if (tab.uniform)
        ljmx<HALF, true, COMP>(s, energy, nb, nlocal, order, xr, sh, numneigh, neighbors, ld,
            cut, tab, fx, fy, fz, epart);
    else
        ljmx<HALF, false, COMP>(s, energy, nb, nlocal, order, xr, sh, numneigh, neighbors, ld,
            cut, tab, fx, fy, fz, epart);
}

void launch_lj_mixed(cudaStream_t s, int comp, int half, int energy, int nlocal,
    const int* order, const float4* xr, const CellShift& sh, const int* numneigh,
    const int* neighbors, int ld, float cutforcesq, const LJTableF& tab, double* fx,
    double* fy, double* fz, double* epart)
{
    if (nlocal <= 0) return;
    int nb = force_partial_blocks(nlocal);
    if (half) {
        if (comp)
            ljmx_u<true, true>(s, energy, nb, nlocal, order, xr, sh, numneigh, neighbors, ld,
                cutforcesq, tab, fx, fy, fz, epart);
        else
            ljmx_u<true, false>(s, energy, nb, nlocal, order, xr, sh, numneigh, neighbors, ld,
                cutforcesq, tab, fx, fy, fz, epart);
    } else {
        if (comp)
            ljmx_u<false, true>(s, energy, nb, nlocal, order, xr, sh, numneigh, neighbors, ld,
                cutforcesq, tab, fx, fy, fz, epart);
        else
            ljmx_u<false, false>(s, energy, nb, nlocal, order, xr, sh, numneigh, neighbors, ld,
                cutforcesq, tab, fx, fy, fz, epart);
    }
    g_launches++;
}

} // namespace mdb
