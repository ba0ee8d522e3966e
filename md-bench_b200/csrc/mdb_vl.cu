// Verlet-list scheme kernels other than the forces: integrator, periodic
// images (ghost map and update), binning, list build and the thermo sums.
// Compiled with -fmad=false: every FP64 expression rounds exactly as the
// reference's strict build evaluates it, which keeps the FP64 path
// bit-identical to the reference (see the parity tests).
#include "mdb_internal.cuh"

namespace mdb {

thread_local long long g_launches = 0;

// ---- integrator: verletlist/integrate.c:21-42 -------------------------------
__device__ __forceinline__ void initial_step(int i, double dtf, double dt, double4* x,
    double& a, double& b, double& c, const double* fx, const double* fy, const double* fz,
    float4* xr, const int* qcell, const CellFrame& cf)
{
    a = a + dtf * fx[i];
    b = b + dtf * fy[i];
    c = c + dtf * fz[i];
    double4 p = x[i];
    p.x       = p.x + dt * a;
    p.y       = p.y + dt * b;
    p.z       = p.z + dt * c;
    x[i]      = p;
    if (xr) xr[i] = rel_position(p, qcell[i], cf);
}

__global__ void k_initial_integrate(int n, double dtf, double dt, double4* __restrict__ x,
    double* __restrict__ vx, double* __restrict__ vy, double* __restrict__ vz,
    const double* __restrict__ fx, const double* __restrict__ fy,
    const double* __restrict__ fz, float4* __restrict__ xr, const int* __restrict__ qcell,
    CellFrame cf)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double a = vx[i], b = vy[i], c = vz[i];
    initial_step(i, dtf, dt, x, a, b, c, fx, fy, fz, xr, qcell, cf);
    vx[i] = a;
    vy[i] = b;
    vz[i] = c;
}

__global__ void k_final_integrate(int n, double dtf, double* __restrict__ vx,
    double* __restrict__ vy, double* __restrict__ vz, const double* __restrict__ fx,
    const double* __restrict__ fy, const double* __restrict__ fz)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    vx[i] = vx[i] + dtf * fx[i];
    vy[i] = vy[i] + dtf * fy[i];
    vz[i] = vz[i] + dtf * fz[i];
}

// finalIntegrate(n) then initialIntegrate(n+1): two separately rounded
// velocity updates, exactly as the two reference calls, in one pass
__global__ void k_final_initial_integrate(int n, double dtf, double dt,
    double4* __restrict__ x, double* __restrict__ vx, double* __restrict__ vy,
    double* __restrict__ vz, const double* __restrict__ fx, const double* __restrict__ fy,
    const double* __restrict__ fz, float4* __restrict__ xr, const int* __restrict__ qcell,
    CellFrame cf)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double a = vx[i] + dtf * fx[i];
    double b = vy[i] + dtf * fy[i];
    double c = vz[i] + dtf * fz[i];
    initial_step(i, dtf, dt, x, a, b, c, fx, fy, fz, xr, qcell, cf);
    vx[i] = a;
    vy[i] = b;
    vz[i] = c;
}

void launch_initial_integrate(cudaStream_t s, int n, double dtf, double dt, double4* x,
    double* vx, double* vy, double* vz, const double* fx, const double* fy, const double* fz,
    float4* xr, const int* qcell, CellFrame cf)
{
    if (n <= 0) return;
    k_initial_integrate<<<mdb_blocks(n, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(n, dtf, dt, x,
        vx, vy, vz, fx, fy, fz, xr, qcell, cf);
    g_launches++;
}

void launch_final_integrate(cudaStream_t s, int n, double dtf, double* vx, double* vy,
    double* vz, const double* fx, const double* fy, const double* fz)
{
    if (n <= 0) return;
    k_final_integrate<<<mdb_blocks(n, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(n, dtf, vx, vy, vz,
        fx, fy, fz);
    g_launches++;
}

void launch_final_initial_integrate(cudaStream_t s, int n, double dtf, double dt, double4* x,
    double* vx, double* vy, double* vz, const double* fx, const double* fy, const double* fz,
    float4* xr, const int* qcell, CellFrame cf)
{
    if (n <= 0) return;
    k_final_initial_integrate<<<mdb_blocks(n, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(n, dtf, dt,
        x, vx, vy, vz, fx, fy, fz, xr, qcell, cf);
    g_launches++;
}

// ---- host-layout transfer: AoS triples <-> device layout ---------------------
__global__ void k_pack_atoms(int n, const double* __restrict__ xa, const double* __restrict__ va,
    const int* __restrict__ ta, double4* __restrict__ x, double* __restrict__ vx,
    double* __restrict__ vy, double* __restrict__ vz)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    x[i]  = make_double4(xa[3 * i], xa[3 * i + 1], xa[3 * i + 2],
         __longlong_as_double((long long)ta[i]));
    vx[i] = va[3 * i];
    vy[i] = va[3 * i + 1];
    vz[i] = va[3 * i + 2];
}

__global__ void k_unpack_atoms(int n, const double4* __restrict__ x,
    const double* __restrict__ vx, const double* __restrict__ vy,
    const double* __restrict__ vz, const double* __restrict__ fx,
    const double* __restrict__ fy, const double* __restrict__ fz, double* __restrict__ xa,
    double* __restrict__ va, double* __restrict__ fa, int* __restrict__ ta)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 p     = x[i];
    xa[3 * i]     = p.x;
    xa[3 * i + 1] = p.y;
    xa[3 * i + 2] = p.z;
    ta[i]         = type_of(p);
    va[3 * i]     = vx[i];
    va[3 * i + 1] = vy[i];
    va[3 * i + 2] = vz[i];
    fa[3 * i]     = fx[i];
    fa[3 * i + 1] = fy[i];
    fa[3 * i + 2] = fz[i];
}

void launch_pack_atoms(cudaStream_t s, int n, const double* xa, const double* va,
    const int* ta, double4* x, double* vx, double* vy, double* vz)
{
    if (n <= 0) return;
    k_pack_atoms<<<mdb_blocks(n, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(n, xa, va, ta, x, vx, vy,
        vz);
    g_launches++;
}

void launch_unpack_atoms(cudaStream_t s, int n, const double4* x, const double* vx,
    const double* vy, const double* vz, const double* fx, const double* fy, const double* fz,
    double* xa, double* va, double* fa, int* ta)
{
    if (n <= 0) return;
    k_unpack_atoms<<<mdb_blocks(n, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(n, x, vx, vy, vz, fx,
        fy, fz, xa, va, fa, ta);
    g_launches++;
}

// ---- wrap: updateAtomsPbcCPU, verletlist/pbc.c:62-87 ------------------------
__global__ void k_wrap(int n, double4* __restrict__ x, double xprd, double yprd, double zprd)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 p = x[i];
    if (p.x < 0.0) p.x += xprd;
    else if (p.x >= xprd) p.x -= xprd;
    if (p.y < 0.0) p.y += yprd;
    else if (p.y >= yprd) p.y -= yprd;
    if (p.z < 0.0) p.z += zprd;
    else if (p.z >= zprd) p.z -= zprd;
    x[i] = p;
}

void launch_wrap(cudaStream_t s, int n, double4* x, double xprd, double yprd, double zprd)
{
    if (n <= 0) return;
    k_wrap<<<mdb_blocks(n, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(n, x, xprd, yprd, zprd);
    g_launches++;
}

// ---- sortAtom, verletlist/neighbor.c:466-536 ----------------------------------
// New atom k is old atom order[k] (the locals bin by bin, each bin's atoms in
// index order); positions carry the type bits, so types move with them.
__global__ void k_permute4(int n, const int* __restrict__ order, const double4* __restrict__ in,
    double4* __restrict__ out)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) out[k] = in[order[k]];
}

// three SoA arrays a, b, c into out[0..n), out[n..2n), out[2n..3n)
__global__ void k_permute3(int n, const int* __restrict__ order, const double* __restrict__ a,
    const double* __restrict__ b, const double* __restrict__ c, double* __restrict__ out)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int o = order[k];
    out[k]         = a[o];
    out[n + k]     = b[o];
    out[2 * n + k] = c[o];
}

void launch_permute4(cudaStream_t s, int n, const int* order, const double4* in, double4* out)
{
    if (n <= 0) return;
    k_permute4<<<mdb_blocks(n, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(n, order, in, out);
    g_launches++;
}

void launch_permute3(cudaStream_t s, int n, const int* order, const double* a, const double* b,
    const double* c, double* out)
{
    if (n <= 0) return;
    k_permute3<<<mdb_blocks(n, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(n, order, a, b, c, out);
    g_launches++;
}

// ---- ghost map: setupPbc, verletlist/pbc.c:103-232 ---------------------------
// The 26 image candidates of one atom, enumerated in the reference's order
// (6 faces, 8 corners, 12 edges). For each candidate `visit(sx, sy, sz)` is
// called when the atom lies within cutneigh of the faces it crosses.
template <typename F>
__device__ __forceinline__ void for_each_image(double x, double y, double z, double c,
    double xp, double yp, double zp, int px, int py, int pz, F visit)
{
    const bool xl = x < c, xh = x >= (xp - c);
    const bool yl = y < c, yh = y >= (yp - c);
    const bool zl = z < c, zh = z >= (zp - c);
    if (px) {
        if (xl) visit(+1, 0, 0);
        if (xh) visit(-1, 0, 0);
    }
    if (py) {
        if (yl) visit(0, +1, 0);
        if (yh) visit(0, -1, 0);
    }
    if (pz) {
        if (zl) visit(0, 0, +1);
        if (zh) visit(0, 0, -1);
    }
    if (px && py && pz) {
        if (xl && yl && zl) visit(+1, +1, +1);
        if (xl && yh && zl) visit(+1, -1, +1);
        if (xl && yl && zh) visit(+1, +1, -1);
        if (xl && yh && zh) visit(+1, -1, -1);
        if (xh && yl && zl) visit(-1, +1, +1);
        if (xh && yh && zl) visit(-1, -1, +1);
        if (xh && yl && zh) visit(-1, +1, -1);
        if (xh && yh && zh) visit(-1, -1, -1);
    }
    if (px && pz) {
        if (xl && zl) visit(+1, 0, +1);
        if (xl && zh) visit(+1, 0, -1);
        if (xh && zl) visit(-1, 0, +1);
        if (xh && zh) visit(-1, 0, -1);
    }
    if (py && pz) {
        if (yl && zl) visit(0, +1, +1);
        if (yl && zh) visit(0, +1, -1);
        if (yh && zl) visit(0, -1, +1);
        if (yh && zh) visit(0, -1, -1);
    }
    if (px && py) {
        if (yl && xl) visit(+1, +1, 0);
        if (yl && xh) visit(-1, +1, 0);
        if (yh && xl) visit(+1, -1, 0);
        if (yh && xh) visit(-1, -1, 0);
    }
}

__global__ void k_ghost_count(int n, const double4* __restrict__ x, double c, double xp,
    double yp, double zp, int px, int py, int pz, int* __restrict__ cnt)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 p = x[i];
    int k     = 0;
    for_each_image(p.x, p.y, p.z, c, xp, yp, zp, px, py, pz, [&](int, int, int) { k++; });
    cnt[i] = k;
}

__device__ __forceinline__ int pack_shift(int sx, int sy, int sz)
{
    return (sx + 1) | ((sy + 1) << 2) | ((sz + 1) << 4);
}

__global__ void k_ghost_write(int n, int ghost_cap, double4* __restrict__ x, double c,
    double xp, double yp, double zp, int px, int py, int pz, const int* __restrict__ off,
    int* __restrict__ border_map, int* __restrict__ pbc_code)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 p = x[i];
    int g     = off[i];
    for_each_image(p.x, p.y, p.z, c, xp, yp, zp, px, py, pz, [&](int sx, int sy, int sz) {
        if (g < ghost_cap) {
            border_map[g] = i;
            pbc_code[g]   = pack_shift(sx, sy, sz);
            double4 gp;
            gp.x     = p.x + sx * xp;
            gp.y     = p.y + sy * yp;
            gp.z     = p.z + sz * zp;
            gp.w     = p.w;
            x[n + g] = gp;
        }
        g++;
    });
}

__global__ void k_ghost_finalize(int n, int ghost_cap, const int* __restrict__ off,
    int* __restrict__ counters)
{
    int total                  = off[n];
    counters[CNT_NGHOST_TOTAL] = total;
    counters[CNT_NGHOST]       = total < ghost_cap ? total : ghost_cap;
}

void launch_ghost_count(cudaStream_t s, int n, const double4* x, double cut, double xprd,
    double yprd, double zprd, int px, int py, int pz, int* cnt)
{
    if (n <= 0) return;
    k_ghost_count<<<mdb_blocks(n, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(n, x, cut, xprd, yprd,
        zprd, px, py, pz, cnt);
    g_launches++;
}

void launch_ghost_write(cudaStream_t s, int n, int ghost_cap, double4* x, double cut,
    double xprd, double yprd, double zprd, int px, int py, int pz, const int* off,
    int* border_map, int* pbc_code, int* counters)
{
    k_ghost_finalize<<<1, 1, 0, s>>>(n, ghost_cap, off, counters);
    g_launches++;
    if (n <= 0) return;
    k_ghost_write<<<mdb_blocks(n, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(n, ghost_cap, x, cut,
        xprd, yprd, zprd, px, py, pz, off, border_map, pbc_code);
    g_launches++;
}

// ---- ghost update: updatePbcCPU, verletlist/pbc.c:42-58 ----------------------
__global__ void k_ghost_update(int nlocal, double4* __restrict__ x,
    const int* __restrict__ border_map, const int* __restrict__ pbc_code, double xp,
    double yp, double zp, const int* __restrict__ counters, float4* __restrict__ xr,
    const int* __restrict__ qcell, CellFrame cf)
{
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= counters[CNT_NGHOST]) return;
    int b     = border_map[g];
    int code  = pbc_code[g];
    int sx    = (code & 3) - 1, sy = ((code >> 2) & 3) - 1, sz = ((code >> 4) & 3) - 1;
    double4 p = x[b];
    double4 q;
    q.x = p.x + sx * xp;
    q.y = p.y + sy * yp;
    q.z = p.z + sz * zp;
    q.w = p.w;
    if (xr) xr[nlocal + g] = rel_position(q, qcell[nlocal + g], cf);
    else x[nlocal + g] = q;
}

void launch_ghost_update(cudaStream_t s, int nlocal, int ghost_cap, double4* x,
    const int* border_map, const int* pbc_code, double xprd, double yprd, double zprd,
    const int* counters, float4* xr, const int* qcell, CellFrame cf)
{
    if (ghost_cap <= 0) return;
    k_ghost_update<<<mdb_blocks(ghost_cap, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(nlocal, x,
        border_map, pbc_code, xprd, yprd, zprd, counters, xr, qcell, cf);
    g_launches++;
}

// ---- mixed-path cells: qcell = floor(x / G) per axis, xr relative to its centre
__global__ void k_cells(int nlocal, const double4* __restrict__ x, float4* __restrict__ xr,
    int* __restrict__ qcell, CellFrame cf, const int* __restrict__ counters, int locals_only)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int n = locals_only ? nlocal : nlocal + counters[CNT_NGHOST];
    if (i >= n) return;
    double4 p = x[i];
    int q     = pack_cell((int)floor(p.x * cf.ginv), (int)floor(p.y * cf.ginv),
            (int)floor(p.z * cf.ginv));
    qcell[i]  = q;
    xr[i]     = rel_position(p, q, cf);
}

void launch_cells(cudaStream_t s, int nlocal, int nall_cap, const double4* x, float4* xr,
    int* qcell, CellFrame cf, const int* counters, int locals_only)
{
    int n = locals_only ? nlocal : nall_cap;
    if (n <= 0) return;
    k_cells<<<mdb_blocks(n, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(nlocal, x, xr, qcell, cf,
        counters, locals_only);
    g_launches++;
}

// ---- binning: coord2bin + binatoms, verletlist/neighbor.c:355-464 ------------
__device__ __forceinline__ int coord2bin(const double4& p, const BinGeom& g)
{
    int ix = (int)((p.x + g.xlo) * g.bininvx);
    int iy = (int)((p.y + g.ylo) * g.bininvy);
    int iz = (int)((p.z + g.zlo) * g.bininvz);
    if (ix < 0 || iy < 0 || iz < 0 || ix >= g.mbinx || iy >= g.mbiny || iz >= g.mbinz)
        return -1;
    return iz * g.mbiny * g.mbinx + iy * g.mbinx + ix;
}

// bin_count[b]: atoms in bin b; bin_lcount[b]: local atoms in bin b
__global__ void k_bin_count(int nlocal, const double4* __restrict__ x, BinGeom g,
    int* __restrict__ atom_bin, int* __restrict__ atom_slot, int* __restrict__ bin_count,
    int* __restrict__ bin_lcount, int* __restrict__ counters)
{
    int i    = blockIdx.x * blockDim.x + threadIdx.x;
    int nall = nlocal + counters[CNT_NGHOST];
    if (i >= nall) return;
    int b = coord2bin(x[i], g);
    if (b < 0) {
        atomicAdd(&counters[CNT_BADBIN], 1);
        atom_bin[i] = -1;
        return;
    }
    atom_bin[i]  = b;
    atom_slot[i] = atomicAdd(&bin_count[b], 1);
    if (i < nlocal) atomicAdd(&bin_lcount[b], 1);
}

__global__ void k_bin_scatter(int nlocal, const int* __restrict__ atom_bin,
    const int* __restrict__ atom_slot, const int* __restrict__ bin_start,
    int* __restrict__ bin_atoms, const int* __restrict__ counters)
{
    int i    = blockIdx.x * blockDim.x + threadIdx.x;
    int nall = nlocal + counters[CNT_NGHOST];
    if (i >= nall) return;
    int b = atom_bin[i];
    if (b < 0) return;
    bin_atoms[bin_start[b] + atom_slot[i]] = i;
}

// Atoms of a bin in ascending index order: the order binatoms produces when it
// fills bins in one serial pass (verletlist/neighbor.c:443-454). Locals have
// the smaller indices, so they form the head of each sorted bin; the heads of
// all bins, concatenated in bin order, give local_order (the order in which
// sortAtom places the local atoms).
__global__ void k_bin_sort(int mbins, const int* __restrict__ bin_start,
    int* __restrict__ bin_atoms, const int* __restrict__ loc_start,
    int* __restrict__ local_order)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= mbins) return;
    int s = bin_start[b], e = bin_start[b + 1];
    for (int k = s + 1; k < e; k++) {
        int v = bin_atoms[k];
        int m = k - 1;
        while (m >= s && bin_atoms[m] > v) {
            bin_atoms[m + 1] = bin_atoms[m];
            m--;
        }
        bin_atoms[m + 1] = v;
    }
    int o = loc_start[b], nl = loc_start[b + 1] - o;
    for (int k = 0; k < nl; k++)
        local_order[o + k] = bin_atoms[s + k];
}

void launch_bin_count(cudaStream_t s, int nlocal, int nall_cap, const double4* x, BinGeom g,
    int* atom_bin, int* atom_slot, int* bin_count, int* bin_lcount, int* counters)
{
    k_bin_count<<<mdb_blocks(nall_cap, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(nlocal, x, g,
        atom_bin, atom_slot, bin_count, bin_lcount, counters);
    g_launches++;
}

void launch_bin_scatter(cudaStream_t s, int nlocal, int nall_cap, const int* atom_bin,
    const int* atom_slot, const int* bin_start, int* bin_atoms, const int* counters)
{
    k_bin_scatter<<<mdb_blocks(nall_cap, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(nlocal, atom_bin,
        atom_slot, bin_start, bin_atoms, counters);
    g_launches++;
}

void launch_bin_sort(cudaStream_t s, int mbins, const int* bin_start, int* bin_atoms,
    const int* loc_start, int* local_order)
{
    k_bin_sort<<<mdb_blocks(mbins, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(mbins, bin_start,
        bin_atoms, loc_start, local_order);
    g_launches++;
}

// ---- list build: buildNeighborCPU, verletlist/neighbor.c:260-352 -------------
// One thread per local atom i (atom order, so the k-major row writes of a warp
// are coalesced). The stencil is walked in the reference order and each bin's
// atoms in index order, so row i holds exactly the reference's neighbours of i
// in the reference's order. A stencil bin is skipped when its box lies farther
// than cutneigh from the atom (a lower bound on every distance to its atoms,
// with a relative margin: skipping only removes candidates that would fail the
// test). The candidate loop handles two candidates per iteration so their
// loads overlap. On the mixed path each entry also carries the cell offset of
// the pair (2 bits per axis, bits 26-31).
__global__ void k_bin_positions(int mbins, const double4* __restrict__ x,
    const int* __restrict__ bin_start, const int* __restrict__ bin_atoms,
    double4* __restrict__ bin_x, float4* __restrict__ bin_xf)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= bin_start[mbins]) return;
    const int j     = bin_atoms[m];
    const double4 p = x[j];
    bin_x[m]  = make_double4(p.x, p.y, p.z, __longlong_as_double((long long)j));
    bin_xf[m] = make_float4((float)p.x, (float)p.y, (float)p.z, __int_as_float(j));
}

void launch_bin_positions(cudaStream_t s, int nall_cap, int mbins, const double4* x,
    const int* bin_start, const int* bin_atoms, double4* bin_x, float4* bin_xf)
{
    k_bin_positions<<<mdb_blocks(nall_cap, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(mbins, x,
        bin_start, bin_atoms, bin_x, bin_xf);
    g_launches++;
}

// Candidates come from the bin-ordered copies (a bin's atoms contiguous, in
// index order): the FP32 copy decides every candidate whose FP32 distance lies
// more than `margin` (a bound on its rounding error) from cutneigh^2; the few
// within it take the reference's exact FP64 test on the FP64 copy. Accepted
// sets and their order are therefore exactly the reference's.
__global__ void __launch_bounds__(128) k_build_list(int nlocal, const double4* __restrict__ x,
    BinGeom g, const int4* __restrict__ stencil, const int* __restrict__ atom_bin,
    const int* __restrict__ bin_start, const double4* __restrict__ bin_x,
    const float4* __restrict__ bin_xf, double cutneighsq, float margin, int half,
    int maxneighs, int ld, int* __restrict__ neighbors, int* __restrict__ numneigh,
    int* __restrict__ counters, const int* __restrict__ qcell)
{
    extern __shared__ int4 st[];
    for (int k = threadIdx.x; k < g.nstencil; k += blockDim.x)
        st[k] = stencil[k];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nlocal) return;
    const double4 xi = x[i];
    const int ibin   = atom_bin[i];
    const int qi     = qcell ? qcell[i] : 0;
    const double ux  = (xi.x + g.xlo) * g.bininvx;
    const double uy  = (xi.y + g.ylo) * g.bininvy;
    const double uz  = (xi.z + g.zlo) * g.bininvz;
    const float fx   = (float)(ux - (double)(int)ux);
    const float fy   = (float)(uy - (double)(int)uy);
    const float fz   = (float)(uz - (double)(int)uz);
    const float bx = (float)g.binsizex, by = (float)g.binsizey, bz = (float)g.binsizez;
    const float skip2 = (float)cutneighsq * 1.0001f + 1e-4f;
    const float xif = (float)xi.x, yif = (float)xi.y, zif = (float)xi.z;
    const float lo = (float)cutneighsq - margin, hi = (float)cutneighsq + margin;
    int n = 0, bad = 0;

    auto consider = [&](int m, const float4& c) {
        const int j = __float_as_int(c.w);
        if (j == i || (half && j < i)) return;
        const float dx = xif - c.x, dy = yif - c.y, dz = zif - c.z;
        const float r2 = dx * dx + dy * dy + dz * dz;
        if (r2 > hi) return;
        if (r2 >= lo) {
            // the reference's test, verletlist/neighbor.c:320-330
            const double4 xj = ldg4(&bin_x[m]);
            double delx      = xi.x - xj.x;
            double dely      = xi.y - xj.y;
            double delz      = xi.z - xj.z;
            double rsq       = delx * delx + dely * dely + delz * delz;
            if (!(rsq <= cutneighsq)) return;
        }
        int e = j;
        if (qcell) {
            int qj = __ldg(&qcell[j]);
            int cx = cell_axis(qj, 0) - cell_axis(qi, 0);
            int cy = cell_axis(qj, 1) - cell_axis(qi, 1);
            int cz = cell_axis(qj, 2) - cell_axis(qi, 2);
            if (cx < -1 || cx > 1 || cy < -1 || cy > 1 || cz < -1 || cz > 1) bad = 1;
            int code = ((cx + 1) & 3) | (((cy + 1) & 3) << 2) | (((cz + 1) & 3) << 4);
            e        = j | (code << MDB_IDX_BITS);
        }
        if (n < maxneighs) neighbors[(size_t)n * ld + i] = e;
        n++;
    };

    if (ibin >= 0) {
        for (int k = 0; k < g.nstencil; k++) {
            const int4 sk = st[k];
            const int jbin = ibin + sk.x;
            if (jbin < 0 || jbin >= g.mbins) continue;
            float gx = sk.y > 0 ? (sk.y - fx) : (sk.y < 0 ? (fx - (sk.y + 1)) : 0.f);
            float gy = sk.z > 0 ? (sk.z - fy) : (sk.z < 0 ? (fy - (sk.z + 1)) : 0.f);
            float gz = sk.w > 0 ? (sk.w - fz) : (sk.w < 0 ? (fz - (sk.w + 1)) : 0.f);
            gx *= bx;
            gy *= by;
            gz *= bz;
            if (gx * gx + gy * gy + gz * gz > skip2) continue;
            const int beg = __ldg(&bin_start[jbin]);
            const int end = __ldg(&bin_start[jbin + 1]);
            int m         = beg;
            for (; m + 1 < end; m += 2) {
                const float4 ca = __ldg(&bin_xf[m]);
                const float4 cb = __ldg(&bin_xf[m + 1]);
                consider(m, ca);
                consider(m + 1, cb);
            }
            if (m < end) consider(m, __ldg(&bin_xf[m]));
        }
    }
    // the stored count never exceeds the row capacity, so no consumer can read
    // past the list; the true count of an overflowing row goes to the host,
    // which grows the list and rebuilds before any force is computed
    numneigh[i] = n < maxneighs ? n : maxneighs;
    if (n > maxneighs) atomicMax(&counters[CNT_MAXNEED], n);
    if (bad) atomicAdd(&counters[CNT_BADCELL], 1);
}

void launch_build_list(cudaStream_t s, int nlocal, const double4* x, BinGeom g,
    const int4* stencil, const int* atom_bin, const int* bin_start,
    const double4* bin_x, const float4* bin_xf, double cutneighsq, float margin, int half,
    int maxneighs, int ld, int* neighbors, int* numneigh, int* counters, const int* qcell)
{
    if (nlocal <= 0) return;
    size_t smem = sizeof(int4) * g.nstencil;
    k_build_list<<<mdb_blocks(nlocal, 128), 128, smem, s>>>(nlocal, x, g, stencil, atom_bin,
        bin_start, bin_x, bin_xf, cutneighsq, margin, half, maxneighs, ld, neighbors, numneigh,
        counters, qcell);
    g_launches++;
}

// ---- thermo: sum of m v.v per block, then one fixed-order reduction ----------
static constexpr int KE_THREADS    = 256;
static constexpr int KE_MAX_BLOCKS = 1184; // 8 x 148 SMs

int ke_partial_blocks(int n)
{
    int b = mdb_blocks(n, KE_THREADS);
    return b < KE_MAX_BLOCKS ? (b > 0 ? b : 1) : KE_MAX_BLOCKS;
}

__global__ void k_ke_partial(int n, const double* __restrict__ vx,
    const double* __restrict__ vy, const double* __restrict__ vz, double mass,
    double* __restrict__ part)
{
    // sum of (vx^2 + vy^2 + vz^2) * mass, common/thermo.c:74-77
    double t = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double a = vx[i], b = vy[i], c = vz[i];
        t += (a * a + b * b + c * c) * mass;
    }
    t = block_sum(t);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

__global__ void k_reduce_partials(int nparts, const double* __restrict__ part,
    double* __restrict__ out)
{
    double t = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x)
        t += part[i];
    t = block_sum(t);
    if (threadIdx.x == 0) *out = t;
}

void launch_ke_partial(cudaStream_t s, int n, const double* vx, const double* vy,
    const double* vz, double mass, double* partials)
{
    k_ke_partial<<<ke_partial_blocks(n), KE_THREADS, 0, s>>>(n, vx, vy, vz, mass, partials);
    g_launches++;
}

void launch_reduce_partials(cudaStream_t s, int nparts, const double* partials, double* out)
{
    k_reduce_partials<<<1, 1024, 0, s>>>(nparts, partials, out);
    g_launches++;
}

// ---- halo atoms of a domain-decomposed run ------------------------------------
// out[3k..3k+2] = position of atom idx[k] plus shift (the periodic image a
// neighbouring domain sees across the global box boundary; one FP64 addition
// per coordinate, as a ghost image is made)
__global__ void k_gather_positions(int n, const int* __restrict__ idx,
    const double4* __restrict__ x, double sx, double sy, double sz, double* __restrict__ out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double4 p = x[idx[k]];
    out[3 * k]      = p.x + sx;
    out[3 * k + 1]  = p.y + sy;
    out[3 * k + 2]  = p.z + sz;
}

void launch_gather_positions(cudaStream_t s, int n, const int* idx, const double4* x, double sx,
    double sy, double sz, double* out)
{
    if (n <= 0) return;
    k_gather_positions<<<mdb_blocks(n, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(n, idx, x, sx, sy,
        sz, out);
    g_launches++;
}

// halo atoms [first, first + n) take positions from in (AoS triples); their
// type bits stay; the mixed path's relative copy follows (cells fixed at the
// last build, as for the atoms the integrator moves)
__global__ void k_set_halo(int first, int n, const double* __restrict__ in, double4* x,
    float4* xr, const int* __restrict__ qcell, CellFrame cf)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int i = first + k;
    double4 p   = x[i];
    p.x = in[3 * k], p.y = in[3 * k + 1], p.z = in[3 * k + 2];
    x[i] = p;
    if (xr) xr[i] = rel_position(p, qcell[i], cf);
}

void launch_set_halo(cudaStream_t s, int first, int n, const double* in, double4* x, float4* xr,
    const int* qcell, const CellFrame& cf)
{
    if (n <= 0) return;
    k_set_halo<<<mdb_blocks(n, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(first, n, in, x, xr, qcell,
        cf);
    g_launches++;
}

} // namespace mdb
