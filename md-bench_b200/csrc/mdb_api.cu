// libmdb C ABI: context, memory, the reference hooks, and the graph-captured
// timestep loop. See include/mdb.h for the contract of every entry point.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "mdb_internal.cuh"

using namespace mdb;

struct Graph {
    cudaGraphExec_t exec = nullptr;
    long long kernels    = 0;
};

struct MdbCtx {
    MdbParams p;
    std::vector<double> eps_t, sig_t;
    int dev          = 0;
    cudaStream_t s   = nullptr;
    std::string err;
    long long launches = 0;

    // sizes; atoms [nown, nlocal) are halo copies from neighbouring domains
    // (binned, imaged and listed, but without force row, integration or
    // thermo); nown = 0: every atom is owned
    int nlocal = 0, ntypes = 1, nown = 0;
    // capacities: atom_cap local atoms (the atom-sized arrays and the list's
    // leading dimension), nall_cap positions (locals then ghosts), border_cap
    // ghost maps; ghost_cap = the ghosts the current nlocal leaves room for
    int ghost_cap = 0, nall_cap = 0, atom_cap = 0, border_cap = 0;
    int maxneighs = 100, ld = 0;
    bool have_atoms = false, have_list = false, have_ghosts = false, mixed = false;
    bool have_eam = false;

    BinGeom g;
    std::vector<int> stencil;
    std::vector<int4> stencil4;
    LJTable tab;
    LJTableF tabf;
    CellFrame cf;
    CellShift shift;
    double cutforcesq = 0, cutneighsq = 0;
    // |FP32 rsq - exact rsq| bound of the list build's prefilter (box size)
    float list_margin = 0;
    double mvv2e = 1, dof_boltz = 1, t_scale = 1, p_scale = 1;

    // device buffers
    double4* x  = nullptr;
    float4* xr  = nullptr; // mixed path: cell-relative FP32 positions
    int* qcell  = nullptr; // mixed path: cell of each atom
    double *vx = nullptr, *vy = nullptr, *vz = nullptr;
    double *fx = nullptr, *fy = nullptr, *fz = nullptr;
    int *border_map = nullptr, *pbc_code = nullptr;
    int *ghost_cnt = nullptr, *ghost_off = nullptr;
    int *atom_bin = nullptr, *atom_slot = nullptr;
    int *bin_count = nullptr, *bin_start = nullptr, *bin_atoms = nullptr;
    double4* bin_x = nullptr; // positions in bin order, atom index bits in .w
    float4* bin_xf = nullptr; // the same rounded to FP32 (list build prefilter)
    int *bin_lcount = nullptr, *loc_start = nullptr; // locals per bin, their offsets
    int* local_order = nullptr; // local atoms bin by bin (the order sortAtom gives)
    int4* stencil_d  = nullptr;                      // {flat offset, dx, dy, dz}
    int *numneigh = nullptr, *neighbors = nullptr;
    int* counters = nullptr;
    int* scan_scratch = nullptr;
    int scan_scratch_n = 0;
    double* partials = nullptr; // 3 regions of npart doubles
    int npart = 0;
    double* red = nullptr; // reductions: [slot*4 + {ke, pe_a, pe_b}]
    int nred_slots = 0;
    double* fp = nullptr;
    float4* xe = nullptr; // mixed EAM: (cell-relative position, F'(rho)) of every atom
    // mixed EAM: the list entries inside the cutoff (laid out like the list)
    // and their count per atom, written by the density pass
    int *eam_cutlist = nullptr, *eam_ncut = nullptr;
    double* stage  = nullptr; // 9 * nlocal doubles: AoS x, v, f for host transfers
    int* stage_t   = nullptr; // nlocal types
    double *eam_frho = nullptr, *eam_rhor = nullptr, *eam_z2r = nullptr;
    float* eam_frho32 = nullptr;
    float4 *eam_dens32 = nullptr, *eam_pair32 = nullptr;
    EamDev eam;
    double eam_cut = 0;

    // pinned host mirrors
    int* h_counters = nullptr;
    double* h_red   = nullptr;

    Graph g_plain, g_rebuild;
    bool energy_valid = false;
    int resort_every  = 0; // SORT_ATOMS builds: sortAtom every resort_every steps
    int eam_rho_lanes = 1; // mixed EAM density pass: lanes per atom (1 or 2)
};

// ---------------------------------------------------------------------------
#define CK(call)                                                                         \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) return fail(ctx, MDB_ERR_CUDA, #call, e_);                \
    } while (0)

static int fail(MdbCtx* ctx, int code, const char* what, cudaError_t e = cudaSuccess)
{
    if (ctx) {
        char buf[512];
        if (e != cudaSuccess)
            snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
        else
            snprintf(buf, sizeof buf, "%s", what);
        ctx->err = buf;
    }
    return code;
}

template <typename T> static cudaError_t dalloc(T** p, size_t n)
{
    *p = nullptr;
    if (n == 0) n = 1;
    return cudaMalloc((void**)p, n * sizeof(T));
}

template <typename T> static void dfree(T*& p)
{
    if (p) cudaFree(p);
    p = nullptr;
}

// atoms this context integrates and computes forces for
static int owned(const MdbCtx* ctx) { return ctx->nown > 0 ? ctx->nown : ctx->nlocal; }

static void destroy_graph(Graph& g)
{
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g.exec    = nullptr;
    g.kernels = 0;
}

static void drop_graphs(MdbCtx* ctx)
{
    destroy_graph(ctx->g_plain);
    destroy_graph(ctx->g_rebuild);
}

// Launch count bookkeeping: direct launches add to g_launches; launches
// recorded during a capture are moved to the graph and replayed per launch.
static long long launch_mark() { return mdb::g_launches; }
static void launch_account(MdbCtx* ctx, long long mark) { ctx->launches += mdb::g_launches - mark; }

// ---------------------------------------------------------------------------
// Bin geometry: setupNeighbor, verletlist/neighbor.c:101-258
static double bindist(const BinGeom& g, int i, int j, int k)
{
    double dx, dy, dz;
    if (i > 0) dx = (i - 1) * g.binsizex;
    else if (i == 0) dx = 0.0;
    else dx = (i + 1) * g.binsizex;
    if (j > 0) dy = (j - 1) * g.binsizey;
    else if (j == 0) dy = 0.0;
    else dy = (j + 1) * g.binsizey;
    if (k > 0) dz = (k - 1) * g.binsizez;
    else if (k == 0) dz = 0.0;
    else dz = (k + 1) * g.binsizez;
    return (dx * dx + dy * dy + dz * dz);
}

static int setup_bins(MdbCtx* ctx)
{
    const MdbParams& p = ctx->p;
    BinGeom& g         = ctx->g;
    const double cut   = p.cutneigh;
    const double fac   = 0.999;
    if (p.bin_rule == MDB_BINS_FILE) {
        g.binsizex = cut * 0.5;
        g.binsizey = cut * 0.5;
        g.binsizez = cut * 0.5;
        g.nbinx    = (int)(p.xprd / g.binsizex);
        g.nbiny    = (int)(p.yprd / g.binsizey);
        g.nbinz    = (int)(p.zprd / g.binsizez);
        if (g.nbinx == 0) g.nbinx = 1;
        if (g.nbiny == 0) g.nbiny = 1;
        if (g.nbinz == 0) g.nbinz = 1;
        g.bininvx = g.nbinx / p.xprd;
        g.bininvy = g.nbiny / p.yprd;
        g.bininvz = g.nbinz / p.zprd;
    } else {
        const double scale = 5.0 / 6.0;
        double bx = scale * p.nx, by = scale * p.ny, bz = scale * p.nz;
        g.nbinx    = (int)(1 > bx ? 1 : bx);
        g.nbiny    = (int)(1 > by ? 1 : by);
        g.nbinz    = (int)(1 > bz ? 1 : bz);
        g.binsizex = p.xprd / g.nbinx;
        g.binsizey = p.yprd / g.nbiny;
        g.binsizez = p.zprd / g.nbinz;
        g.bininvx  = 1.0 / g.binsizex;
        g.bininvy  = 1.0 / g.binsizey;
        g.bininvz  = 1.0 / g.binsizez;
    }
    g.pad_x = (int)(cut * g.bininvx);
    while (g.pad_x * g.binsizex < fac * cut)
        g.pad_x++;
    g.pad_y = (int)(cut * g.bininvy);
    while (g.pad_y * g.binsizey < fac * cut)
        g.pad_y++;
    g.pad_z = (int)(cut * g.bininvz);
    while (g.pad_z * g.binsizez < fac * cut)
        g.pad_z++;
    int nextx = (int)(cut * g.bininvx);
    while (nextx * g.binsizex < fac * cut) {
        nextx++;
        g.pad_x++;
    }
    int nexty = (int)(cut * g.bininvy);
    while (nexty * g.binsizey < fac * cut) {
        nexty++;
        g.pad_y++;
    }
    int nextz = (int)(cut * g.bininvz);
    while (nextz * g.binsizez < fac * cut) {
        nextz++;
        g.pad_z++;
    }
    g.mbinx = std::max(1, g.nbinx + 4 * g.pad_x);
    g.mbiny = std::max(1, g.nbiny + 4 * g.pad_y);
    g.mbinz = std::max(1, g.nbinz + 4 * g.pad_z);
    long long mb = (long long)g.mbinx * g.mbiny * g.mbinz;
    if (mb > (1LL << 30)) return fail(ctx, MDB_ERR_ARG, "bin grid too large");
    g.mbins = (int)mb;
    ctx->stencil.clear();
    ctx->stencil4.clear();
    double cutsq = cut * cut;
    for (int k = -nextz; k <= nextz; k++)
        for (int j = -nexty; j <= nexty; j++)
            for (int i = -nextx; i <= nextx; i++)
                if (bindist(g, i, j, k) < cutsq) {
                    int flat = k * g.mbiny * g.mbinx + j * g.mbinx + i;
                    ctx->stencil.push_back(flat);
                    ctx->stencil4.push_back(make_int4(flat, i, j, k));
                }
    g.nstencil = (int)ctx->stencil.size();
    if (g.nstencil > MDB_MAX_STENCIL) return fail(ctx, MDB_ERR_ARG, "stencil too large");
    g.xlo = fabs(0.0 - g.pad_x * g.binsizex) + 1e-9;
    g.ylo = fabs(0.0 - g.pad_y * g.binsizey) + 1e-9;
    g.zlo = fabs(0.0 - g.pad_z * g.binsizez) + 1e-9;
    return MDB_OK;
}

// LJ type-pair tables: computePerTypeLJParameters + computeTypePairLJParameters
// (common/parameter.c:31-71); types beyond the given tables use epsilon/sigma.
static int setup_types(MdbCtx* ctx, int ntypes)
{
    if (ntypes < 1) ntypes = 1;
    if (ntypes > MDB_MAX_TYPES) return fail(ctx, MDB_ERR_ARG, "more than 8 atom types");
    ctx->ntypes = ntypes;
    std::vector<double> sq(ntypes), s3(ntypes);
    for (int t = 0; t < ntypes; t++) {
        double e = t < (int)ctx->eps_t.size() ? ctx->eps_t[t] : ctx->p.epsilon;
        double s = t < (int)ctx->sig_t.size() ? ctx->sig_t[t] : ctx->p.sigma;
        sq[t]    = sqrt(e);
        s3[t]    = s * s * s;
    }
    LJTable& T  = ctx->tab;
    LJTableF& F = ctx->tabf;
    memset(&T, 0, sizeof T);
    memset(&F, 0, sizeof F);
    T.ntypes = F.ntypes = ntypes;
    bool uniform        = true;
    for (int i = 0; i < ntypes; i++)
        for (int j = 0; j < ntypes; j++) {
            int k     = i * ntypes + j;
            T.eps[k]  = sq[i] * sq[j];
            T.sig6[k] = s3[i] * s3[j];
            F.eps[k]  = (float)T.eps[k];
            F.sig6[k] = (float)T.sig6[k];
            if (T.eps[k] != T.eps[0] || T.sig6[k] != T.sig6[0]) uniform = false;
        }
    T.uniform = F.uniform = uniform ? 1 : 0;
    return MDB_OK;
}

static void setup_thermo_constants(MdbCtx* ctx)
{
    // setupThermo, common/thermo.c:35-58
    const MdbParams& p = ctx->p;
    if (p.force_field == MDB_FF_EAM) {
        ctx->mvv2e     = 1.036427e-04;
        ctx->dof_boltz = (p.natoms * 3 - 3) * 8.617343e-05;
        ctx->t_scale   = ctx->mvv2e / ctx->dof_boltz;
        ctx->p_scale   = 1.602176e+06 / 3 / p.xprd / p.yprd / p.zprd;
    } else {
        ctx->mvv2e     = 1.0;
        ctx->dof_boltz = (p.natoms * 3 - 3);
        ctx->t_scale   = ctx->mvv2e / ctx->dof_boltz;
        ctx->p_scale   = 1.0 / 3 / p.xprd / p.yprd / p.zprd;
    }
}

// ---------------------------------------------------------------------------
extern "C" const char* mdb_status_string(int st)
{
    switch (st) {
    case MDB_OK: return "ok";
    case MDB_ERR_ARG: return "invalid argument";
    case MDB_ERR_CUDA: return "CUDA error";
    case MDB_ERR_OVERFLOW: return "buffer overflow";
    case MDB_ERR_TIMEOUT: return "device wait timed out";
    case MDB_ERR_NOMEM: return "out of memory";
    case MDB_ERR_STATE: return "call out of order";
    default: return "unknown status";
    }
}

extern "C" const char* mdb_last_error(const MdbCtx* ctx) { return ctx ? ctx->err.c_str() : ""; }
extern "C" void* mdb_stream(MdbCtx* ctx) { return ctx ? (void*)ctx->s : nullptr; }
extern "C" long long mdb_launch_count(const MdbCtx* ctx) { return ctx ? ctx->launches : 0; }

extern "C" int mdb_create(const MdbParams* params, MdbCtx** out)
{
    if (!params || !out) return MDB_ERR_ARG;
    *out         = nullptr;
    MdbCtx* ctx  = new MdbCtx();
    ctx->p       = *params;
    MdbParams& p = ctx->p;
    if (p.ntypes < 1) p.ntypes = 1;
    if (p.epsilon_per_type) ctx->eps_t.assign(p.epsilon_per_type, p.epsilon_per_type + p.ntypes);
    if (p.sigma_per_type) ctx->sig_t.assign(p.sigma_per_type, p.sigma_per_type + p.ntypes);
    p.epsilon_per_type = nullptr;
    p.sigma_per_type   = nullptr;
    if (p.reneigh_every < 1) p.reneigh_every = 20;
    if (p.nstat < 1) p.nstat = 100;
    if (p.maxneighs < 1) p.maxneighs = 100;
    ctx->maxneighs = p.maxneighs;
    int rc         = MDB_OK;
    if (!(p.xprd > 0 && p.yprd > 0 && p.zprd > 0) || !(p.cutneigh > 0) || !(p.cutforce > 0) ||
        p.cutforce > p.cutneigh || (p.force_field != MDB_FF_LJ && p.force_field != MDB_FF_EAM) ||
        p.precision < MDB_PREC_FP64 || p.precision > MDB_PREC_MIXED_COMP ||
        (p.force_field == MDB_FF_EAM && p.half_neigh)) {
        rc = fail(ctx, MDB_ERR_ARG, "invalid parameters");
        goto bad;
    }
    ctx->mixed = p.precision != MDB_PREC_FP64;
    ctx->cutforcesq = p.cutforce * p.cutforce;
    ctx->cutneighsq = p.cutneigh * p.cutneigh;
    {
        // coordinates (ghosts included) lie within the box grown by cutneigh;
        // rounding each to FP32 moves a difference by at most 2 e, e = |x|max
        // 2^-24, and rsq by at most 2 e (|dx| + |dy| + |dz|) + 3 (2e)^2 with
        // |d| <= cutneigh near the threshold, plus the FP32 rounding of the
        // three products and two sums; a factor 4 covers the rest
        const double xmax = std::max(p.xprd, std::max(p.yprd, p.zprd)) + 2.0 * p.cutneigh;
        const double e    = xmax * 0x1p-24;
        const double bnd  = 2.0 * e * 3.0 * p.cutneigh + 12.0 * e * e +
                           8.0 * ctx->cutneighsq * 0x1p-24;
        ctx->list_margin = (float)(4.0 * bnd);
    }
    {
        // mixed-path cells: the smallest power of two G >= cutneigh, so the
        // cells of any listed pair differ by at most one per axis
        double g = 1.0 / 1024;
        while (g < p.cutneigh)
            g *= 2;
        ctx->cf.g    = g;
        ctx->cf.ginv = 1.0 / g;
        ctx->shift.g = (float)g;
        double lmax = std::max(p.xprd, std::max(p.yprd, p.zprd)) + 2 * p.cutneigh;
        if (ctx->mixed && lmax * ctx->cf.ginv > 1000) {
            rc = fail(ctx, MDB_ERR_ARG, "box too large for the mixed path's cell index");
            goto bad;
        }
    }
    if ((rc = setup_bins(ctx)) != MDB_OK) goto bad;
    if ((rc = setup_types(ctx, p.ntypes)) != MDB_OK) goto bad;
    setup_thermo_constants(ctx);
    {
        cudaError_t e;
        if ((e = cudaSetDevice(p.device)) != cudaSuccess) {
            rc = fail(ctx, MDB_ERR_CUDA, "cudaSetDevice", e);
            goto bad;
        }
        ctx->dev = p.device;
        if ((e = cudaStreamCreateWithFlags(&ctx->s, cudaStreamNonBlocking)) != cudaSuccess) {
            rc = fail(ctx, MDB_ERR_CUDA, "cudaStreamCreate", e);
            goto bad;
        }
        if ((e = dalloc(&ctx->counters, CNT_SLOTS)) != cudaSuccess ||
            (e = dalloc(&ctx->stencil_d, ctx->g.nstencil)) != cudaSuccess ||
            (e = dalloc(&ctx->bin_count, ctx->g.mbins)) != cudaSuccess ||
            (e = dalloc(&ctx->bin_start, ctx->g.mbins + 1)) != cudaSuccess ||
            (e = cudaMallocHost((void**)&ctx->h_counters, CNT_SLOTS * sizeof(int))) !=
                cudaSuccess) {
            rc = fail(ctx, MDB_ERR_NOMEM, "device allocation", e);
            goto bad;
        }
        if ((e = dalloc(&ctx->bin_lcount, ctx->g.mbins)) != cudaSuccess ||
            (e = dalloc(&ctx->loc_start, ctx->g.mbins + 1)) != cudaSuccess) {
            rc = fail(ctx, MDB_ERR_NOMEM, "device allocation", e);
            goto bad;
        }
        cudaMemset(ctx->counters, 0, CNT_SLOTS * sizeof(int));
        cudaMemcpy(ctx->stencil_d, ctx->stencil4.data(), sizeof(int4) * ctx->g.nstencil,
            cudaMemcpyHostToDevice);
        if ((e = cudaGetLastError()) != cudaSuccess) {
            rc = fail(ctx, MDB_ERR_CUDA, "setup copy", e);
            goto bad;
        }
    }
    *out = ctx;
    return MDB_OK;
bad:
    fprintf(stderr, "mdb_create: %s\n", ctx->err.c_str());
    mdb_destroy(ctx);
    return rc;
}

static void free_atom_buffers(MdbCtx* ctx)
{
    dfree(ctx->x);
    dfree(ctx->xr);
    dfree(ctx->qcell);
    dfree(ctx->local_order);
    dfree(ctx->vx);
    dfree(ctx->vy);
    dfree(ctx->vz);
    dfree(ctx->fx);
    dfree(ctx->fy);
    dfree(ctx->fz);
    dfree(ctx->border_map);
    dfree(ctx->pbc_code);
    dfree(ctx->ghost_cnt);
    dfree(ctx->ghost_off);
    dfree(ctx->atom_bin);
    dfree(ctx->atom_slot);
    dfree(ctx->bin_atoms);
    dfree(ctx->bin_x);
    dfree(ctx->bin_xf);
    dfree(ctx->numneigh);
    dfree(ctx->neighbors);
    dfree(ctx->eam_cutlist);
    dfree(ctx->eam_ncut);
    dfree(ctx->scan_scratch);
    dfree(ctx->partials);
    dfree(ctx->red);
    dfree(ctx->fp);
    dfree(ctx->xe);
    dfree(ctx->stage);
    dfree(ctx->stage_t);
    if (ctx->h_red) cudaFreeHost(ctx->h_red);
    ctx->h_red = nullptr;
}

extern "C" int mdb_destroy(MdbCtx* ctx)
{
    if (!ctx) return MDB_OK;
    if (ctx->s) cudaStreamSynchronize(ctx->s);
    drop_graphs(ctx);
    free_atom_buffers(ctx);
    dfree(ctx->counters);
    dfree(ctx->stencil_d);
    dfree(ctx->bin_count);
    dfree(ctx->bin_start);
    dfree(ctx->bin_lcount);
    dfree(ctx->loc_start);
    dfree(ctx->eam_frho);
    dfree(ctx->eam_rhor);
    dfree(ctx->eam_z2r);
    dfree(ctx->eam_frho32);
    dfree(ctx->eam_dens32);
    dfree(ctx->eam_pair32);
    if (ctx->h_counters) cudaFreeHost(ctx->h_counters);
    if (ctx->s) cudaStreamDestroy(ctx->s);
    delete ctx;
    return MDB_OK;
}

extern "C" int mdb_synchronize(MdbCtx* ctx)
{
    if (!ctx) return MDB_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->s));
    return MDB_OK;
}

// (Re)allocate everything sized by nall_cap, preserving local positions.
static int alloc_ghost_sized(MdbCtx* ctx, int ghost_cap)
{
    cudaStream_t s = ctx->s;
    CK(cudaStreamSynchronize(s));
    drop_graphs(ctx);
    int nall = ctx->nlocal + ghost_cap;
    double4* nx;
    CK(dalloc(&nx, nall));
    if (ctx->x) {
        CK(cudaMemcpyAsync(nx, ctx->x, sizeof(double4) * ctx->nlocal, cudaMemcpyDeviceToDevice, s));
        CK(cudaStreamSynchronize(s));
    }
    dfree(ctx->x);
    ctx->x = nx;
    if (ctx->mixed) {
        if ((long long)nall > (long long)MDB_IDX_MASK)
            return fail(ctx, MDB_ERR_ARG, "mixed path limited to 2^25 atoms including ghosts");
        // cells and relative positions are recomputed by every rebuild
        dfree(ctx->xr);
        dfree(ctx->qcell);
        CK(dalloc(&ctx->xr, nall));
        CK(dalloc(&ctx->qcell, nall));
    }
    dfree(ctx->border_map);
    dfree(ctx->pbc_code);
    dfree(ctx->atom_bin);
    dfree(ctx->atom_slot);
    dfree(ctx->bin_atoms);
    dfree(ctx->bin_x);
    dfree(ctx->bin_xf);
    dfree(ctx->fp);
    dfree(ctx->xe);
    CK(dalloc(&ctx->border_map, ghost_cap));
    CK(dalloc(&ctx->pbc_code, ghost_cap));
    ctx->border_cap = ghost_cap;
    CK(dalloc(&ctx->atom_bin, nall));
    CK(dalloc(&ctx->atom_slot, nall));
    CK(dalloc(&ctx->bin_atoms, nall));
    CK(dalloc(&ctx->bin_x, nall));
    CK(dalloc(&ctx->bin_xf, nall));
    if (ctx->p.force_field == MDB_FF_EAM) CK(dalloc(&ctx->fp, nall));
    if (ctx->p.force_field == MDB_FF_EAM && ctx->mixed) CK(dalloc(&ctx->xe, nall));
    ctx->ghost_cap   = ghost_cap;
    ctx->nall_cap    = nall;
    ctx->have_ghosts = false;
    ctx->have_list   = false;
    return MDB_OK;
}

static int alloc_list(MdbCtx* ctx, int maxneighs)
{
    CK(cudaStreamSynchronize(ctx->s));
    drop_graphs(ctx);
    dfree(ctx->neighbors);
    dfree(ctx->eam_cutlist);
    CK(dalloc(&ctx->neighbors, (size_t)maxneighs * ctx->ld));
    if (ctx->p.force_field == MDB_FF_EAM && ctx->mixed)
        CK(dalloc(&ctx->eam_cutlist, (size_t)maxneighs * ctx->ld));
    ctx->maxneighs = maxneighs;
    ctx->have_list = false;
    return MDB_OK;
}

extern "C" int mdb_set_atoms(MdbCtx* ctx, int nlocal, const double* x, const double* v,
    const int* type)
{
    if (!ctx || nlocal < 0 || (nlocal > 0 && (!x || !v || !type))) return MDB_ERR_ARG;
    CK(cudaSetDevice(ctx->dev));
    ctx->nown = 0; // new atoms: all owned until mdb_set_owned
    // host or device arrays (unified addressing); the types are checked here
    std::vector<int> htype;
    const int* th = type;
    if (nlocal > 0) {
        cudaPointerAttributes pa;
        if (cudaPointerGetAttributes(&pa, type) == cudaSuccess &&
            (pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged)) {
            htype.resize(nlocal);
            CK(cudaMemcpy(htype.data(), type, sizeof(int) * nlocal, cudaMemcpyDefault));
            th = htype.data();
        }
        cudaGetLastError();
    }
    int maxt = 0;
    for (int i = 0; i < nlocal; i++) {
        if (th[i] < 0) return fail(ctx, MDB_ERR_ARG, "negative atom type");
        maxt = std::max(maxt, th[i] + 1);
    }
    int rc = setup_types(ctx, std::max(ctx->p.ntypes, maxt));
    if (rc) return rc;
    // the buffers are kept while the atom count stays within the capacity
    // (a domain's atom count changes a little at every rebuild)
    bool realloc_all = nlocal > ctx->atom_cap || !ctx->x;
    if (!realloc_all && nlocal != ctx->nlocal) {
        CK(cudaStreamSynchronize(ctx->s));
        drop_graphs(ctx);
        ctx->nlocal      = nlocal;
        ctx->ghost_cap   = std::min(ctx->border_cap, ctx->nall_cap - nlocal);
        ctx->have_ghosts = ctx->have_list = false;
    }
    if (realloc_all) {
        CK(cudaStreamSynchronize(ctx->s));
        drop_graphs(ctx);
        free_atom_buffers(ctx);
        ctx->nlocal   = nlocal;
        const int cap = nlocal + nlocal / 32 + 64;
        ctx->atom_cap = cap;
        ctx->ld       = ((cap + 31) / 32) * 32;
        CK(dalloc(&ctx->vx, cap));
        CK(dalloc(&ctx->vy, cap));
        CK(dalloc(&ctx->vz, cap));
        CK(dalloc(&ctx->fx, cap));
        CK(dalloc(&ctx->fy, cap));
        CK(dalloc(&ctx->fz, cap));
        CK(cudaMemset(ctx->fx, 0, sizeof(double) * cap));
        CK(cudaMemset(ctx->fy, 0, sizeof(double) * cap));
        CK(cudaMemset(ctx->fz, 0, sizeof(double) * cap));
        CK(dalloc(&ctx->ghost_cnt, cap + 1));
        CK(dalloc(&ctx->ghost_off, cap + 1));
        CK(dalloc(&ctx->numneigh, cap));
        if (ctx->p.force_field == MDB_FF_EAM && ctx->mixed) CK(dalloc(&ctx->eam_ncut, cap));
        CK(dalloc(&ctx->local_order, cap));
        CK(dalloc(&ctx->stage, 9 * (size_t)cap));
        CK(dalloc(&ctx->stage_t, cap));
        int nscan         = std::max(scan_scratch_ints(cap), scan_scratch_ints(ctx->g.mbins));
        ctx->scan_scratch_n = nscan;
        CK(dalloc(&ctx->scan_scratch, nscan));
        ctx->npart = std::max(std::max(force_partial_blocks(cap), ke_partial_blocks(cap)),
            eam_mixed_blocks(cap));
        CK(dalloc(&ctx->partials, 3 * (size_t)ctx->npart));
        ctx->nred_slots = 64;
        CK(dalloc(&ctx->red, 4 * (size_t)ctx->nred_slots));
        CK(cudaMallocHost((void**)&ctx->h_red, 4 * sizeof(double) * ctx->nred_slots));
        // initial ghost capacity: surface shell estimate, grown on demand
        double vol   = ctx->p.xprd * ctx->p.yprd * ctx->p.zprd;
        double dens  = vol > 0 ? nlocal / vol : 0;
        double c     = ctx->p.cutneigh;
        double shell = (ctx->p.xprd + 2 * c) * (ctx->p.yprd + 2 * c) * (ctx->p.zprd + 2 * c) - vol;
        // an atom has at most 7 images (3 faces, 3 edges, 1 corner)
        int gcap = (int)std::min(7.0 * nlocal + 1024, 1.25 * dens * shell + 1024);
        ctx->x       = nullptr;
        if ((rc = alloc_ghost_sized(ctx, gcap)) != MDB_OK) return rc;
        if ((rc = alloc_list(ctx, ctx->maxneighs)) != MDB_OK) return rc;
    }
    // AoS host arrays go up as they are; a kernel packs them into the device
    // layout (double4 with the type bits in .w, SoA velocities)
    cudaStream_t s = ctx->s;
    size_t n3      = 3 * (size_t)nlocal;
    CK(cudaMemcpyAsync(ctx->stage, x, sizeof(double) * n3, cudaMemcpyDefault, s));
    CK(cudaMemcpyAsync(ctx->stage + n3, v, sizeof(double) * n3, cudaMemcpyDefault, s));
    CK(cudaMemcpyAsync(ctx->stage_t, type, sizeof(int) * nlocal, cudaMemcpyDefault, s));
    {
        long long m = launch_mark();
        launch_pack_atoms(s, nlocal, ctx->stage, ctx->stage + n3, ctx->stage_t, ctx->x, ctx->vx,
            ctx->vy, ctx->vz);
        launch_account(ctx, m);
    }
    if (ctx->mixed) {
        long long m = launch_mark();
        launch_cells(s, nlocal, ctx->nall_cap, ctx->x, ctx->xr, ctx->qcell, ctx->cf,
            ctx->counters, 1);
        launch_account(ctx, m);
    }
    CK(cudaStreamSynchronize(s));
    ctx->have_atoms   = true;
    ctx->have_ghosts  = false;
    ctx->have_list    = false;
    ctx->energy_valid = false;
    return MDB_OK;
}

extern "C" int mdb_get_atoms(MdbCtx* ctx, double* x, double* v, double* f, int* type)
{
    if (!ctx || !ctx->have_atoms) return MDB_ERR_STATE;
    int n          = ctx->nlocal;
    size_t n3      = 3 * (size_t)n;
    cudaStream_t s = ctx->s;
    long long m    = launch_mark();
    launch_unpack_atoms(s, n, ctx->x, ctx->vx, ctx->vy, ctx->vz, ctx->fx, ctx->fy, ctx->fz,
        ctx->stage, ctx->stage + n3, ctx->stage + 2 * n3, ctx->stage_t);
    launch_account(ctx, m);
    if (x) CK(cudaMemcpyAsync(x, ctx->stage, sizeof(double) * n3, cudaMemcpyDefault, s));
    if (v) CK(cudaMemcpyAsync(v, ctx->stage + n3, sizeof(double) * n3, cudaMemcpyDefault, s));
    if (f) CK(cudaMemcpyAsync(f, ctx->stage + 2 * n3, sizeof(double) * n3, cudaMemcpyDefault, s));
    if (type) CK(cudaMemcpyAsync(type, ctx->stage_t, sizeof(int) * n, cudaMemcpyDefault, s));
    CK(cudaStreamSynchronize(s));
    return MDB_OK;
}

// ---------------------------------------------------------------------------
// enqueue helpers (no host synchronisation; safe inside stream capture)
static void enq_initial(MdbCtx* ctx)
{
    launch_initial_integrate(ctx->s, owned(ctx), ctx->p.dtforce, ctx->p.dt, ctx->x, ctx->vx,
        ctx->vy, ctx->vz, ctx->fx, ctx->fy, ctx->fz, ctx->mixed ? ctx->xr : nullptr,
        ctx->qcell, ctx->cf);
}

static void enq_final(MdbCtx* ctx)
{
    launch_final_integrate(ctx->s, owned(ctx), ctx->p.dtforce, ctx->vx, ctx->vy, ctx->vz,
        ctx->fx, ctx->fy, ctx->fz);
}

// finalIntegrate of the previous step fused with initialIntegrate of this one
static void enq_final_initial(MdbCtx* ctx)
{
    launch_final_initial_integrate(ctx->s, owned(ctx), ctx->p.dtforce, ctx->p.dt, ctx->x,
        ctx->vx, ctx->vy, ctx->vz, ctx->fx, ctx->fy, ctx->fz, ctx->mixed ? ctx->xr : nullptr,
        ctx->qcell, ctx->cf);
}

// Mixed path: only the cell-relative FP32 ghost positions are refreshed
// between rebuilds (the FP64 ghost positions are rebuilt with the ghost map).
static void enq_ghost_update(MdbCtx* ctx)
{
    launch_ghost_update(ctx->s, ctx->nlocal, ctx->ghost_cap, ctx->x, ctx->border_map,
        ctx->pbc_code, ctx->p.xprd, ctx->p.yprd, ctx->p.zprd, ctx->counters,
        ctx->mixed ? ctx->xr : nullptr, ctx->qcell, ctx->cf);
}

static void enq_force(MdbCtx* ctx, bool energy)
{
    cudaStream_t s = ctx->s;
    int n          = owned(ctx); // rows of the owned atoms (full lists with halos)
    double* ep0    = ctx->partials;
    double* ep1    = ctx->partials + ctx->npart;
    if (ctx->p.force_field == MDB_FF_EAM) {
        if (ctx->mixed) {
            launch_eam_mixed(s, energy, ctx->p.precision == MDB_PREC_MIXED_COMP,
                ctx->eam_rho_lanes, n, ctx->ghost_cap, ctx->xr, ctx->shift, ctx->numneigh, ctx->neighbors, ctx->ld,
                (float)ctx->cutforcesq, ctx->eam, ctx->border_map, ctx->counters,
                ctx->eam_cutlist, ctx->eam_ncut, ctx->fp, ctx->xe, ctx->fx, ctx->fy, ctx->fz, ep0,
                ep1);
        } else {
            launch_eam_fp64(s, energy, n, ctx->ghost_cap, nullptr,ctx->x,
                ctx->numneigh, ctx->neighbors, ctx->ld, ctx->cutforcesq, ctx->eam,
                ctx->border_map, ctx->counters, ctx->fp, ctx->fx, ctx->fy, ctx->fz, ep0, ep1);
        }
        return;
    }
    if (ctx->p.half_neigh) {
        cudaMemsetAsync(ctx->fx, 0, sizeof(double) * n, s);
        cudaMemsetAsync(ctx->fy, 0, sizeof(double) * n, s);
        cudaMemsetAsync(ctx->fz, 0, sizeof(double) * n, s);
    }
    if (ctx->mixed)
        launch_lj_mixed(s, ctx->p.precision == MDB_PREC_MIXED_COMP, ctx->p.half_neigh, energy, n,
            nullptr, ctx->xr, ctx->shift, ctx->numneigh, ctx->neighbors, ctx->ld,
            (float)ctx->cutforcesq, ctx->tabf, ctx->fx, ctx->fy, ctx->fz, ep0);
    else
        launch_lj_fp64(s, ctx->p.half_neigh, energy, n, nullptr, ctx->x, ctx->numneigh,
            ctx->neighbors, ctx->ld, ctx->cutforcesq, ctx->tab, ctx->fx, ctx->fy, ctx->fz, ep0);
}

// Rebuild sequence after the initial integration of a reneighbour step:
// updateAtomsPbc, setupPbc, updatePbc, buildNeighbor. Idempotent, so it can be
// replayed after growing a buffer.
static void enq_ghosts(MdbCtx* ctx)
{
    cudaStream_t s = ctx->s;
    const MdbParams& p = ctx->p;
    launch_ghost_count(s, ctx->nlocal, ctx->x, p.cutneigh, p.xprd, p.yprd, p.zprd, p.pbc_x,
        p.pbc_y, p.pbc_z, ctx->ghost_cnt);
    scan_exclusive(ctx->ghost_cnt, ctx->ghost_off, ctx->nlocal, ctx->scan_scratch, s);
    launch_ghost_write(s, ctx->nlocal, ctx->ghost_cap, ctx->x, p.cutneigh, p.xprd, p.yprd,
        p.zprd, p.pbc_x, p.pbc_y, p.pbc_z, ctx->ghost_off, ctx->border_map, ctx->pbc_code,
        ctx->counters);
    // mixed path: cells (fixed until the next rebuild) of locals and ghosts
    if (ctx->mixed)
        launch_cells(s, ctx->nlocal, ctx->nall_cap, ctx->x, ctx->xr, ctx->qcell, ctx->cf,
            ctx->counters, 0);
}

static void enq_list(MdbCtx* ctx)
{
    cudaStream_t s = ctx->s;
    cudaMemsetAsync(ctx->bin_count, 0, sizeof(int) * ctx->g.mbins, s);
    cudaMemsetAsync(ctx->bin_lcount, 0, sizeof(int) * ctx->g.mbins, s);
    cudaMemsetAsync(ctx->local_order, 0xff, sizeof(int) * std::max(ctx->nlocal, 1), s);
    launch_bin_count(s, ctx->nlocal, ctx->nall_cap, ctx->x, ctx->g, ctx->atom_bin,
        ctx->atom_slot, ctx->bin_count, ctx->bin_lcount, ctx->counters);
    scan_exclusive(ctx->bin_count, ctx->bin_start, ctx->g.mbins, ctx->scan_scratch, s);
    scan_exclusive(ctx->bin_lcount, ctx->loc_start, ctx->g.mbins, ctx->scan_scratch, s);
    launch_bin_scatter(s, ctx->nlocal, ctx->nall_cap, ctx->atom_bin, ctx->atom_slot,
        ctx->bin_start, ctx->bin_atoms, ctx->counters);
    launch_bin_sort(s, ctx->g.mbins, ctx->bin_start, ctx->bin_atoms, ctx->loc_start,
        ctx->local_order);
    launch_bin_positions(s, ctx->nall_cap, ctx->g.mbins, ctx->x, ctx->bin_start, ctx->bin_atoms,
        ctx->bin_x, ctx->bin_xf);
    launch_build_list(s, ctx->nlocal, ctx->x, ctx->g, ctx->stencil_d, ctx->atom_bin,
        ctx->bin_start, ctx->bin_x, ctx->bin_xf, ctx->cutneighsq, ctx->list_margin,
        ctx->p.half_neigh, ctx->maxneighs, ctx->ld, ctx->neighbors, ctx->numneigh,
        ctx->counters, ctx->mixed ? ctx->qcell : nullptr);
}

static void clear_rebuild_counters(MdbCtx* ctx)
{
    // CNT_MAXNEED, CNT_BADBIN, CNT_BADCELL
    cudaMemsetAsync(ctx->counters + CNT_MAXNEED, 0, 3 * sizeof(int), ctx->s);
}

static void enq_rebuild(MdbCtx* ctx)
{
    clear_rebuild_counters(ctx);
    launch_wrap(ctx->s, ctx->nlocal, ctx->x, ctx->p.xprd, ctx->p.yprd, ctx->p.zprd);
    enq_ghosts(ctx);
    enq_list(ctx);
}

// setup() of verletlist/main.c:96-111 builds ghosts and lists without wrapping.
static void enq_rebuild_nowrap(MdbCtx* ctx)
{
    clear_rebuild_counters(ctx);
    enq_ghosts(ctx);
    enq_list(ctx);
}

// Reads the device counters and grows whatever overflowed. Returns 1 when the
// rebuild must be replayed, 0 when it is complete, <0 on error (negated status).
static int check_rebuild(MdbCtx* ctx)
{
    cudaStream_t s = ctx->s;
    cudaError_t e  = cudaMemcpyAsync(ctx->h_counters, ctx->counters, CNT_SLOTS * sizeof(int),
        cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return -fail(ctx, MDB_ERR_CUDA, "rebuild check", e);
    const int* h = ctx->h_counters;
    if (h[CNT_BADBIN] > 0) return -fail(ctx, MDB_ERR_OVERFLOW, "atom outside the bin grid");
    if (h[CNT_BADCELL] > 0)
        return -fail(ctx, MDB_ERR_OVERFLOW, "mixed path: listed pair more than two cells apart");
    int again = 0;
    if (h[CNT_NGHOST_TOTAL] > ctx->ghost_cap) {
        int rc = alloc_ghost_sized(ctx, (int)(h[CNT_NGHOST_TOTAL] * 1.2) + 1024);
        if (rc) return -rc;
        again = 1;
    } else if (h[CNT_MAXNEED] > ctx->maxneighs) {
        int rc = alloc_list(ctx, (int)(h[CNT_MAXNEED] * 1.2));
        if (rc) return -rc;
        again = 1;
    }
    return again;
}


static int capture(MdbCtx* ctx, Graph& g, void (*body)(MdbCtx*))
{
    cudaGraph_t graph;
    long long mark = launch_mark();
    CK(cudaStreamBeginCapture(ctx->s, cudaStreamCaptureModeThreadLocal));
    body(ctx);
    cudaError_t e = cudaStreamEndCapture(ctx->s, &graph);
    g.kernels     = mdb::g_launches - mark;
    mdb::g_launches = mark;
    if (e != cudaSuccess) return fail(ctx, MDB_ERR_CUDA, "stream capture", e);
    e = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(ctx, MDB_ERR_CUDA, "graph instantiate", e);
    return MDB_OK;
}

static int launch_graph(MdbCtx* ctx, Graph& g)
{
    CK(cudaGraphLaunch(g.exec, ctx->s));
    ctx->launches += g.kernels;
    return MDB_OK;
}

static int do_rebuild(MdbCtx* ctx, bool use_graph, bool wrap = true)
{
    for (int attempt = 0; attempt < 8; attempt++) {
        if (use_graph) {
            if (!ctx->g_rebuild.exec) {
                int rc = capture(ctx, ctx->g_rebuild, enq_rebuild);
                if (rc) return rc;
            }
            int rc = launch_graph(ctx, ctx->g_rebuild);
            if (rc) return rc;
        } else {
            long long m = launch_mark();
            if (wrap) enq_rebuild(ctx);
            else enq_rebuild_nowrap(ctx);
            launch_account(ctx, m);
        }
        int r = check_rebuild(ctx);
        if (r < 0) return -r;
        if (r == 0) {
            ctx->have_ghosts = ctx->have_list = true;
            return MDB_OK;
        }
    }
    return fail(ctx, MDB_ERR_OVERFLOW, "rebuild did not converge");
}

// sortAtom (verletlist/neighbor.c:466-536): the reference clears the ghosts,
// bins the locals (binatoms: a bin's atoms in index order) and rewrites the
// atom arrays bin by bin. Positions (with their type bits), velocities and
// forces move together here; the reference moves only positions and
// velocities. Ghosts and lists are left invalid, as in the reference.
static int sort_atoms(MdbCtx* ctx)
{
    cudaStream_t s = ctx->s;
    const int n    = ctx->nlocal;
    long long m    = launch_mark();
    cudaMemsetAsync(ctx->counters + CNT_NGHOST, 0, sizeof(int), s);
    cudaMemsetAsync(ctx->counters + CNT_BADBIN, 0, sizeof(int), s);
    cudaMemsetAsync(ctx->bin_count, 0, sizeof(int) * ctx->g.mbins, s);
    cudaMemsetAsync(ctx->bin_lcount, 0, sizeof(int) * ctx->g.mbins, s);
    cudaMemsetAsync(ctx->local_order, 0xff, sizeof(int) * std::max(n, 1), s);
    launch_bin_count(s, n, ctx->nall_cap, ctx->x, ctx->g, ctx->atom_bin, ctx->atom_slot,
        ctx->bin_count, ctx->bin_lcount, ctx->counters);
    scan_exclusive(ctx->bin_count, ctx->bin_start, ctx->g.mbins, ctx->scan_scratch, s);
    scan_exclusive(ctx->bin_lcount, ctx->loc_start, ctx->g.mbins, ctx->scan_scratch, s);
    launch_bin_scatter(s, n, ctx->nall_cap, ctx->atom_bin, ctx->atom_slot, ctx->bin_start,
        ctx->bin_atoms, ctx->counters);
    launch_bin_sort(s, ctx->g.mbins, ctx->bin_start, ctx->bin_atoms, ctx->loc_start,
        ctx->local_order);
    // stage: 9 n doubles; positions as double4 [0, 4n), velocities [4n, 7n)
    double4* sx = reinterpret_cast<double4*>(ctx->stage);
    double* sv  = ctx->stage + 4 * (size_t)n;
    launch_permute4(s, n, ctx->local_order, ctx->x, sx);
    launch_permute3(s, n, ctx->local_order, ctx->vx, ctx->vy, ctx->vz, sv);
    CK(cudaMemcpyAsync(ctx->x, sx, sizeof(double4) * n, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(ctx->vx, sv, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(ctx->vy, sv + n, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(ctx->vz, sv + 2 * (size_t)n, sizeof(double) * n,
        cudaMemcpyDeviceToDevice, s));
    launch_permute3(s, n, ctx->local_order, ctx->fx, ctx->fy, ctx->fz, ctx->stage);
    CK(cudaMemcpyAsync(ctx->fx, ctx->stage, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(ctx->fy, ctx->stage + n, sizeof(double) * n, cudaMemcpyDeviceToDevice,
        s));
    CK(cudaMemcpyAsync(ctx->fz, ctx->stage + 2 * (size_t)n, sizeof(double) * n,
        cudaMemcpyDeviceToDevice, s));
    launch_account(ctx, m);
    CK(cudaMemcpyAsync(ctx->h_counters, ctx->counters, CNT_SLOTS * sizeof(int),
        cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    ctx->have_ghosts = ctx->have_list = false;
    if (ctx->h_counters[CNT_BADBIN] > 0)
        return fail(ctx, MDB_ERR_OVERFLOW, "atom outside the bin grid");
    return MDB_OK;
}

// ---------------------------------------------------------------------------
// hooks
#define NEED_ATOMS()                                                                     \
    do {                                                                                 \
        if (!ctx) return MDB_ERR_ARG;                                                    \
        if (!ctx->have_atoms) return fail(ctx, MDB_ERR_STATE, "no atoms set");           \
    } while (0)

extern "C" int mdb_setup_pbc(MdbCtx* ctx)
{
    NEED_ATOMS();
    for (int attempt = 0; attempt < 4; attempt++) {
        long long m = launch_mark();
        enq_ghosts(ctx);
        launch_account(ctx, m);
        int r = check_rebuild(ctx);
        if (r < 0) return -r;
        if (r == 0) {
            ctx->have_ghosts = true;
            ctx->have_list   = false;
            return MDB_OK;
        }
    }
    return fail(ctx, MDB_ERR_OVERFLOW, "ghost map did not converge");
}

extern "C" int mdb_update_pbc(MdbCtx* ctx)
{
    NEED_ATOMS();
    if (!ctx->have_ghosts) return fail(ctx, MDB_ERR_STATE, "setup_pbc not run");
    long long m = launch_mark();
    // FP64 ghost positions, and on the mixed path also their relative copies
    launch_ghost_update(ctx->s, ctx->nlocal, ctx->ghost_cap, ctx->x, ctx->border_map,
        ctx->pbc_code, ctx->p.xprd, ctx->p.yprd, ctx->p.zprd, ctx->counters, nullptr, nullptr,
        ctx->cf);
    if (ctx->mixed) enq_ghost_update(ctx);
    launch_account(ctx, m);
    return MDB_OK;
}

extern "C" int mdb_update_atoms_pbc(MdbCtx* ctx)
{
    NEED_ATOMS();
    long long m = launch_mark();
    launch_wrap(ctx->s, ctx->nlocal, ctx->x, ctx->p.xprd, ctx->p.yprd, ctx->p.zprd);
    if (ctx->mixed)
        launch_cells(ctx->s, ctx->nlocal, ctx->nall_cap, ctx->x, ctx->xr, ctx->qcell, ctx->cf,
            ctx->counters, 1);
    launch_account(ctx, m);
    return MDB_OK;
}

extern "C" int mdb_build_neighbor(MdbCtx* ctx)
{
    NEED_ATOMS();
    if (!ctx->have_ghosts) return fail(ctx, MDB_ERR_STATE, "setup_pbc not run");
    for (int attempt = 0; attempt < 8; attempt++) {
        long long m = launch_mark();
        clear_rebuild_counters(ctx);
        enq_list(ctx);
        launch_account(ctx, m);
        int r = check_rebuild(ctx);
        if (r < 0) return -r;
        if (r == 0) {
            ctx->have_list = true;
            return MDB_OK;
        }
        if (!ctx->have_ghosts) { // ghost buffers were regrown: rebuild the map too
            int rc = mdb_setup_pbc(ctx);
            if (rc) return rc;
        }
    }
    return fail(ctx, MDB_ERR_OVERFLOW, "list build did not converge");
}

static int compute_force(MdbCtx* ctx, bool energy)
{
    NEED_ATOMS();
    if (!ctx->have_list) return fail(ctx, MDB_ERR_STATE, "no neighbour list");
    if (ctx->p.force_field == MDB_FF_EAM && !ctx->have_eam)
        return fail(ctx, MDB_ERR_STATE, "EAM tables not set");
    long long m = launch_mark();
    enq_force(ctx, energy);
    launch_account(ctx, m);
    ctx->energy_valid = energy;
    CK(cudaGetLastError());
    return MDB_OK;
}

extern "C" int mdb_compute_force(MdbCtx* ctx) { return compute_force(ctx, false); }
extern "C" int mdb_compute_force_energy(MdbCtx* ctx) { return compute_force(ctx, true); }

extern "C" int mdb_initial_integrate(MdbCtx* ctx)
{
    NEED_ATOMS();
    long long m = launch_mark();
    enq_initial(ctx);
    launch_account(ctx, m);
    ctx->energy_valid = false;
    return MDB_OK;
}

extern "C" int mdb_final_integrate(MdbCtx* ctx)
{
    NEED_ATOMS();
    long long m = launch_mark();
    enq_final(ctx);
    launch_account(ctx, m);
    return MDB_OK;
}

static void enq_thermo(MdbCtx* ctx, int slot, bool with_pe)
{
    cudaStream_t s = ctx->s;
    double* r      = ctx->red + 4 * slot;
    int nke        = ke_partial_blocks(owned(ctx));
    launch_ke_partial(s, owned(ctx), ctx->vx, ctx->vy, ctx->vz, ctx->p.mass,
        ctx->partials + 2 * (size_t)ctx->npart);
    launch_reduce_partials(s, nke, ctx->partials + 2 * (size_t)ctx->npart, r + 0);
    if (with_pe) {
        // the mixed EAM passes write eam_mixed_blocks partials, the rest one
        // per block of the force kernels
        int nf = ctx->p.force_field == MDB_FF_EAM && ctx->mixed ? eam_mixed_blocks(owned(ctx))
                                                               : force_partial_blocks(owned(ctx));
        launch_reduce_partials(s, nf, ctx->partials, r + 1);
        if (ctx->p.force_field == MDB_FF_EAM)
            launch_reduce_partials(s, nf, ctx->partials + ctx->npart, r + 2);
        else
            cudaMemsetAsync(r + 2, 0, sizeof(double), s);
    } else {
        cudaMemsetAsync(r + 1, 0, 2 * sizeof(double), s);
    }
}

static void finish_thermo(MdbCtx* ctx, const double* r, int step, MdbThermo* out)
{
    double t      = r[0];
    out->step     = step;
    out->ke       = 0.5 * t * ctx->mvv2e;
    double T      = t * ctx->t_scale;
    out->temperature = T;
    out->pressure = (T * ctx->dof_boltz) * ctx->p_scale;
    out->pe       = r[1] + r[2];
    out->etotal   = out->ke + out->pe;
}

extern "C" int mdb_thermo(MdbCtx* ctx, MdbThermo* out)
{
    NEED_ATOMS();
    if (!out) return MDB_ERR_ARG;
    long long m = launch_mark();
    enq_thermo(ctx, 0, ctx->energy_valid);
    launch_account(ctx, m);
    CK(cudaMemcpyAsync(ctx->h_red, ctx->red, 4 * sizeof(double), cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    finish_thermo(ctx, ctx->h_red, -1, out);
    if (!ctx->energy_valid) out->pe = out->etotal = NAN;
    return MDB_OK;
}

extern "C" int mdb_setup(MdbCtx* ctx)
{
    NEED_ATOMS();
    if (ctx->p.force_field == MDB_FF_EAM && !ctx->have_eam)
        return fail(ctx, MDB_ERR_STATE, "EAM tables not set");
    int rc = do_rebuild(ctx, false, false); // setupPbc + updatePbc + buildNeighbor
    if (rc) return rc;
    return compute_force(ctx, true);
}

// A plain step (no rebuild, no sample) whose predecessor left its final
// integration pending: finalIntegrate(n-1) + initialIntegrate(n) in one
// kernel, ghost update, force. Its own final integration is left pending.
static void enq_plain_step(MdbCtx* ctx)
{
    enq_final_initial(ctx);
    enq_ghost_update(ctx);
    enq_force(ctx, false);
}

extern "C" int mdb_set_neighbor_list(MdbCtx* ctx, const int* numneigh, const int* neighbors,
    int ld)
{
    NEED_ATOMS();
    if (!numneigh || !neighbors || ld < 1) return MDB_ERR_ARG;
    if (ctx->mixed) return fail(ctx, MDB_ERR_ARG, "caller lists need an FP64 context");
    const int n = ctx->nlocal;
    int maxn    = 0;
    for (int i = 0; i < n; i++) {
        if (numneigh[i] < 0 || numneigh[i] > ld) return fail(ctx, MDB_ERR_ARG, "row length");
        maxn = std::max(maxn, numneigh[i]);
        for (int k = 0; k < numneigh[i]; k++) {
            const int j = neighbors[(size_t)i * ld + k];
            if (j < 0 || j >= n) return fail(ctx, MDB_ERR_ARG, "entry is not a local atom");
        }
    }
    CK(cudaSetDevice(ctx->dev));
    if (maxn > ctx->maxneighs) {
        int rc = alloc_list(ctx, maxn);
        if (rc) return rc;
    }
    // k-major on the device: entry k of atom i at k * ld + i
    std::vector<int> all((size_t)ctx->maxneighs * ctx->ld, 0);
    for (int i = 0; i < n; i++)
        for (int k = 0; k < numneigh[i]; k++)
            all[(size_t)k * ctx->ld + i] = neighbors[(size_t)i * ld + k];
    CK(cudaStreamSynchronize(ctx->s));
    CK(cudaMemcpy(ctx->neighbors, all.data(), sizeof(int) * all.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->numneigh, numneigh, sizeof(int) * n, cudaMemcpyHostToDevice));
    CK(cudaMemset(ctx->counters + CNT_NGHOST, 0, sizeof(int)));
    ctx->have_ghosts = ctx->have_list = true;
    return MDB_OK;
}

extern "C" int mdb_sort_atoms(MdbCtx* ctx)
{
    NEED_ATOMS();
    CK(cudaSetDevice(ctx->dev));
    return sort_atoms(ctx);
}

extern "C" int mdb_tune(MdbCtx* ctx, const char* key, int value)
{
    if (!ctx || !key) return MDB_ERR_ARG;
    if (!strcmp(key, "eam_rho_lanes")) {
        if (value != 1 && value != 2) return MDB_ERR_ARG;
        drop_graphs(ctx);
        ctx->eam_rho_lanes = value;
        return MDB_OK;
    }
    return fail(ctx, MDB_ERR_ARG, "unknown tuning key");
}

extern "C" int mdb_set_resort(MdbCtx* ctx, int resort_every)
{
    if (!ctx || resort_every < 0) return MDB_ERR_ARG;
    ctx->resort_every = resort_every;
    return MDB_OK;
}

// ---- domain decomposition -------------------------------------------------------
extern "C" int mdb_set_owned(MdbCtx* ctx, int nown)
{
    NEED_ATOMS();
    if (nown < 1 || nown > ctx->nlocal) return fail(ctx, MDB_ERR_ARG, "owned count out of range");
    // half lists: a halo atom is listed like a ghost (index past every owned
    // atom) and gets no reaction, so each domain computes the pairs across its
    // faces for its own atoms, with no reverse exchange of forces
    if (nown < ctx->nlocal && ctx->p.force_field != MDB_FF_LJ)
        return fail(ctx, MDB_ERR_ARG, "halo atoms need LJ forces");
    ctx->nown = nown == ctx->nlocal ? 0 : nown;
    drop_graphs(ctx);
    return MDB_OK;
}

extern "C" int mdb_gather_positions(MdbCtx* ctx, const int* d_idx, int n, double shift_x,
    double shift_y, double shift_z, double* d_out)
{
    NEED_ATOMS();
    if (n < 0 || (n > 0 && (!d_idx || !d_out))) return MDB_ERR_ARG;
    long long m = launch_mark();
    launch_gather_positions(ctx->s, n, d_idx, ctx->x, shift_x, shift_y, shift_z, d_out);
    launch_account(ctx, m);
    CK(cudaGetLastError());
    return MDB_OK;
}

extern "C" int mdb_set_halo_positions(MdbCtx* ctx, const double* d_x, int n)
{
    NEED_ATOMS();
    const int first = owned(ctx), nhalo = ctx->nown > 0 ? ctx->nlocal - ctx->nown : 0;
    if (n != nhalo || (n > 0 && !d_x)) return fail(ctx, MDB_ERR_ARG, "halo size mismatch");
    long long m = launch_mark();
    launch_set_halo(ctx->s, first, n, d_x, ctx->x, ctx->mixed ? ctx->xr : nullptr, ctx->qcell,
        ctx->cf);
    launch_account(ctx, m);
    CK(cudaGetLastError());
    return MDB_OK;
}

extern "C" int mdb_run(MdbCtx* ctx, int first_step, int nsteps, MdbThermo* samples,
    int max_samples, int* nsamples)
{
    NEED_ATOMS();
    if (!ctx->have_list) return fail(ctx, MDB_ERR_STATE, "mdb_setup not run");
    if (ctx->nown > 0)
        return fail(ctx, MDB_ERR_STATE,
            "halo atoms are refreshed between steps by the caller: drive the steps by the hooks");
    if (nsteps < 0 || (max_samples > 0 && !samples)) return MDB_ERR_ARG;
    if (nsamples) *nsamples = 0;
    int nslot = 0;
    std::vector<int> slot_step;
    const int last = first_step + nsteps - 1;
    // finalIntegrate of step n is deferred and fused with initialIntegrate of
    // step n+1 unless a thermo sample, a rebuild step or the end of the run
    // needs it on its own
    bool pending_final = false;
    for (int n = first_step; n <= last; n++) {
        // SORT_ATOMS builds resort before the step's initial integration
        // (verletlist/main.c:372-381); the step then rebuilds ghosts and lists
        const bool resort = ctx->resort_every > 0 && (n + 1) % ctx->resort_every == 0;
        bool reneigh      = resort || (n + 1) % ctx->p.reneigh_every == 0;
        bool sample       = max_samples > 0 && (n + 1) % ctx->p.nstat == 0;
        if (resort) {
            if (pending_final) {
                long long m0 = launch_mark();
                enq_final(ctx);
                launch_account(ctx, m0);
                pending_final = false;
            }
            int rc = sort_atoms(ctx);
            if (rc) return rc;
        }
        if (!reneigh && !sample && pending_final) {
            if (!ctx->g_plain.exec) {
                int rc = capture(ctx, ctx->g_plain, enq_plain_step);
                if (rc) return rc;
            }
            int rc = launch_graph(ctx, ctx->g_plain);
            if (rc) return rc;
            if (n == last) {
                long long m = launch_mark();
                enq_final(ctx);
                launch_account(ctx, m);
            }
            continue;
        }
        long long m = launch_mark();
        if (pending_final) enq_final_initial(ctx);
        else enq_initial(ctx);
        pending_final = false;
        launch_account(ctx, m);
        if (reneigh) {
            int rc = do_rebuild(ctx, true);
            if (rc) return rc;
        } else {
            m = launch_mark();
            enq_ghost_update(ctx);
            launch_account(ctx, m);
        }
        m = launch_mark();
        enq_force(ctx, sample);
        if (sample || n == last) {
            enq_final(ctx);
        } else {
            pending_final = true;
        }
        if (sample && nslot < ctx->nred_slots && nslot < max_samples) {
            enq_thermo(ctx, nslot, true);
            slot_step.push_back(n + 1);
            nslot++;
        }
        launch_account(ctx, m);
    }
    ctx->energy_valid = nsteps > 0 && max_samples > 0;
    CK(cudaGetLastError());
    if (nslot > 0) {
        CK(cudaMemcpyAsync(ctx->h_red, ctx->red, 4 * sizeof(double) * nslot,
            cudaMemcpyDeviceToHost, ctx->s));
    }
    CK(cudaStreamSynchronize(ctx->s));
    for (int k = 0; k < nslot; k++)
        finish_thermo(ctx, ctx->h_red + 4 * k, slot_step[k], &samples[k]);
    if (nsamples) *nsamples = nslot;
    return MDB_OK;
}

// ---------------------------------------------------------------------------
extern "C" int mdb_set_eam(MdbCtx* ctx, const MdbEamTables* t)
{
    if (!ctx || !t || !t->frho_spline || !t->rhor_spline || !t->z2r_spline || t->nr < 3 ||
        t->nrho < 3)
        return MDB_ERR_ARG;
    if (ctx->p.force_field != MDB_FF_EAM) return fail(ctx, MDB_ERR_ARG, "not an EAM context");
    CK(cudaSetDevice(ctx->dev));
    CK(cudaStreamSynchronize(ctx->s));
    drop_graphs(ctx);
    auto relayout = [](const double* src, int n, int tot, std::vector<double>& d,
                        std::vector<float>& f) {
        int rows = std::min(n + 1, tot / 7);
        d.assign((size_t)(n + 1) * 8, 0.0);
        f.assign((size_t)(n + 1) * 8, 0.0f);
        for (int m = 0; m < rows; m++)
            for (int c = 0; c < 7; c++) {
                d[(size_t)m * 8 + c] = src[(size_t)m * 7 + c];
                f[(size_t)m * 8 + c] = (float)src[(size_t)m * 7 + c];
            }
    };
    std::vector<double> fr, rr, zr;
    std::vector<float> fr32, rr32, zr32;
    relayout(t->frho_spline, t->nrho, t->nrho_tot, fr, fr32);
    relayout(t->rhor_spline, t->nr, t->nr_tot, rr, rr32);
    relayout(t->z2r_spline, t->nr, t->nr_tot, zr, zr32);
    // the mixed passes' rows (see EamDev)
    const size_t nrow = (size_t)t->nr + 1;
    std::vector<float4> dens32(nrow), pair32(2 * nrow);
    for (size_t m = 0; m < nrow; m++) {
        const float* r = &rr32[m * 8];
        const float* z = &zr32[m * 8];
        dens32[m]         = make_float4(r[3], r[4], r[5], r[6]);
        pair32[2 * m]     = make_float4(z[3], z[4], z[5], z[6]);
        pair32[2 * m + 1] = make_float4(r[0], r[1], r[2], z[0]);
    }
    dfree(ctx->eam_frho);
    dfree(ctx->eam_rhor);
    dfree(ctx->eam_z2r);
    dfree(ctx->eam_frho32);
    dfree(ctx->eam_dens32);
    dfree(ctx->eam_pair32);
    CK(dalloc(&ctx->eam_frho, fr.size()));
    CK(dalloc(&ctx->eam_rhor, rr.size()));
    CK(dalloc(&ctx->eam_z2r, zr.size()));
    CK(dalloc(&ctx->eam_frho32, fr32.size()));
    CK(dalloc(&ctx->eam_dens32, dens32.size()));
    CK(dalloc(&ctx->eam_pair32, pair32.size()));
    CK(cudaMemcpy(ctx->eam_frho, fr.data(), fr.size() * 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->eam_rhor, rr.data(), rr.size() * 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->eam_z2r, zr.data(), zr.size() * 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->eam_frho32, fr32.data(), fr32.size() * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->eam_dens32, dens32.data(), dens32.size() * sizeof(float4),
        cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->eam_pair32, pair32.data(), pair32.size() * sizeof(float4),
        cudaMemcpyHostToDevice));
    ctx->eam.nrho   = t->nrho;
    ctx->eam.nr     = t->nr;
    ctx->eam.rdr    = t->rdr;
    ctx->eam.rdrho  = t->rdrho;
    ctx->eam.frho   = ctx->eam_frho;
    ctx->eam.rhor   = ctx->eam_rhor;
    ctx->eam.z2r    = ctx->eam_z2r;
    ctx->eam.frho32 = ctx->eam_frho32;
    ctx->eam.dens32 = ctx->eam_dens32;
    ctx->eam.pair32 = ctx->eam_pair32;
    ctx->have_eam   = true;
    return MDB_OK;
}

// ---------------------------------------------------------------------------
// introspection
extern "C" int mdb_get_counts(MdbCtx* ctx, int* nlocal, int* nghost, int* maxneighs)
{
    if (!ctx) return MDB_ERR_ARG;
    CK(cudaMemcpyAsync(ctx->h_counters, ctx->counters, CNT_SLOTS * sizeof(int),
        cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    if (nlocal) *nlocal = ctx->nlocal;
    if (nghost) *nghost = ctx->have_ghosts ? ctx->h_counters[CNT_NGHOST] : 0;
    if (maxneighs) *maxneighs = ctx->maxneighs;
    return MDB_OK;
}

extern "C" int mdb_get_positions_all(MdbCtx* ctx, double* x)
{
    NEED_ATOMS();
    int nl, ng;
    int rc = mdb_get_counts(ctx, &nl, &ng, nullptr);
    if (rc) return rc;
    std::vector<double4> h(nl + ng);
    CK(cudaMemcpy(h.data(), ctx->x, sizeof(double4) * (nl + ng), cudaMemcpyDeviceToHost));
    for (int i = 0; i < nl + ng; i++) {
        x[3 * i]     = h[i].x;
        x[3 * i + 1] = h[i].y;
        x[3 * i + 2] = h[i].z;
    }
    return MDB_OK;
}

extern "C" int mdb_get_ghosts(MdbCtx* ctx, int* border_map, int* pbc_xyz)
{
    NEED_ATOMS();
    int ng;
    int rc = mdb_get_counts(ctx, nullptr, &ng, nullptr);
    if (rc) return rc;
    std::vector<int> bm(ng), code(ng);
    if (ng > 0) {
        CK(cudaMemcpy(bm.data(), ctx->border_map, sizeof(int) * ng, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(code.data(), ctx->pbc_code, sizeof(int) * ng, cudaMemcpyDeviceToHost));
    }
    for (int g = 0; g < ng; g++) {
        if (border_map) border_map[g] = bm[g];
        if (pbc_xyz) {
            pbc_xyz[3 * g + 0] = (code[g] & 3) - 1;
            pbc_xyz[3 * g + 1] = ((code[g] >> 2) & 3) - 1;
            pbc_xyz[3 * g + 2] = ((code[g] >> 4) & 3) - 1;
        }
    }
    return MDB_OK;
}

extern "C" int mdb_get_neighbor_list(MdbCtx* ctx, int* numneigh, int* neighbors, int ld)
{
    NEED_ATOMS();
    if (!ctx->have_list) return fail(ctx, MDB_ERR_STATE, "no neighbour list");
    // row i (column i of the k-major list) belongs to atom i. Mixed-path
    // entries carry a cell-offset code above the index bits, masked off here.
    int n = ctx->nlocal;
    std::vector<int> nn(n), order(n);
    CK(cudaStreamSynchronize(ctx->s));
    CK(cudaMemcpy(nn.data(), ctx->numneigh, sizeof(int) * n, cudaMemcpyDeviceToHost));
    for (int t = 0; t < n; t++)
        order[t] = t;
    if (numneigh)
        for (int t = 0; t < n; t++)
            numneigh[order[t]] = nn[t];
    if (neighbors) {
        const int mask = ctx->mixed ? MDB_IDX_MASK : -1;
        std::vector<int> all((size_t)ctx->maxneighs * ctx->ld);
        CK(cudaMemcpy(all.data(), ctx->neighbors, sizeof(int) * all.size(), cudaMemcpyDeviceToHost));
        for (int t = 0; t < n; t++)
            for (int k = 0; k < nn[t] && k < ld && k < ctx->maxneighs; k++)
                neighbors[(size_t)order[t] * ld + k] = all[(size_t)k * ctx->ld + t] & mask;
    }
    return MDB_OK;
}

extern "C" int mdb_get_bin_geometry(MdbCtx* ctx, int* ints, double* dbls, int* stencil,
    int max_stencil)
{
    if (!ctx) return MDB_ERR_ARG;
    const BinGeom& g = ctx->g;
    int iv[10]       = { g.nbinx, g.nbiny, g.nbinz, g.mbinx, g.mbiny, g.mbinz, g.pad_x, g.pad_y,
        g.pad_z, g.nstencil };
    double dv[7] = { g.binsizex, g.binsizey, g.binsizez, g.bininvx, g.bininvy, g.bininvz,
        ctx->p.cutneigh };
    if (ints) memcpy(ints, iv, sizeof iv);
    if (dbls) memcpy(dbls, dv, sizeof dv);
    if (stencil)
        memcpy(stencil, ctx->stencil.data(), sizeof(int) * std::min(max_stencil, g.nstencil));
    return MDB_OK;
}

extern "C" int mdb_get_eam_fp(MdbCtx* ctx, double* fp)
{
    NEED_ATOMS();
    if (!ctx->fp) return fail(ctx, MDB_ERR_STATE, "not an EAM context");
    int nl, ng;
    int rc = mdb_get_counts(ctx, &nl, &ng, nullptr);
    if (rc) return rc;
    CK(cudaMemcpy(fp, ctx->fp, sizeof(double) * (nl + ng), cudaMemcpyDeviceToHost));
    return MDB_OK;
}
