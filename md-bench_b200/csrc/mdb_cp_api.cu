// libmdb cluster-pair C ABI (include/mdb_cp.h): context, buffers, the
// reference hooks and the graph-captured timestep loop of clusterpair/main.c.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "mdb_cp.h"
#include "mdb_cp_internal.cuh"

using namespace mdb;
using namespace mdb::cp;

struct CpGraph {
    cudaGraphExec_t exec = nullptr;
    long long kernels    = 0;
};

struct MdbCp {
    MdbParams p;
    std::vector<double> eps_t, sig_t;
    int M = CP_M, N = 4, jfac = 1, prune_every = 1000;
    bool mixed = false;
    // MDB_PREC_MIXED_COMP: the pair-list kernel with compensated sums and
    // exact cutoff decisions, forces in the FP64 slots cf
    bool comp = false;
    int dev        = 0;
    cudaStream_t s = nullptr;
    std::string err;
    long long launches = 0;

    int nlocal = 0, maxneighs = 200;
    // column edge in percent of setupNeighbor's (max(M, N) / rho)^(1/3); 100
    // keeps the reference's grid, so its lists (tuning key "column_edge")
    int col_edge_pct = 100;
    Geom g;
    std::vector<int> stencil;
    Types ty;
    double cutforcesq = 0;
    double t_scale = 1, dof_boltz = 1, p_scale = 1;

    // capacities
    int atom_cap = 0, ncl_cap = 0, ncj_cap = 0, ngc_cap = 0, slot_cap = 0, ld = 0;

    // atom arrays and columns
    double4 *ax = nullptr, *av = nullptr;
    int *atom_col = nullptr, *col_count = nullptr, *col_start = nullptr, *col_fill = nullptr;
    int *col_atoms = nullptr, *col_sorted = nullptr, *gidx = nullptr;
    double* gz    = nullptr;
    int *ncl_col = nullptr, *cl_start = nullptr;
    // slots
    double4 *cx = nullptr, *cv = nullptr, *cf = nullptr;
    float4 *xr = nullptr, *cf32 = nullptr, *anchor = nullptr;
    // clusters
    int *inat = nullptr, *cbin = nullptr, *cl_first = nullptr, *jnat = nullptr;
    double4 *ibbmin = nullptr, *ibbmax = nullptr, *jbbmin = nullptr, *jbbmax = nullptr;
    // ghosts and j columns
    int *gcount = nullptr, *gstart = nullptr, *border = nullptr, *pbc = nullptr;
    int *gcolumn = nullptr, *gcol_count = nullptr, *gfill = nullptr, *jcol_n = nullptr;
    int *jcol_start = nullptr, *gtmp = nullptr, *jcol = nullptr;
    int* ztab = nullptr; // the list build's window table (Geom zq, z0, zinv)
    double4 *jcbbmin = nullptr, *jcbbmax = nullptr;
    float4 *jcbbf = nullptr, *cxf = nullptr; // FP32 copies for the list build
    int* stencil_d = nullptr;
    // list
    int *list = nullptr, *numneigh = nullptr, *nmasked = nullptr;
    // counters, scratch, reductions
    int* cnt                 = nullptr;
    unsigned long long* zext = nullptr;
    int* scan_scratch        = nullptr;
    int scan_scratch_n       = 0;
    double* partials         = nullptr; // npart for energy + npart for ke
    int npart                = 0;
    double* red              = nullptr; // 64 slots x {ke_atoms, pe, ke_slots, pad}
    double* stage            = nullptr;
    int* stage_i             = nullptr;
    size_t stage_n           = 0;
    int* h_cnt               = nullptr;
    double* h_red            = nullptr;

    bool have_atoms = false, have_clusters = false, have_ghosts = false, have_list = false;
    bool energy_valid = false;
    // the slot forces belong to the current slot positions (a force evaluation
    // since the last integration or cluster build), so thermo can evaluate
    // the energy on demand
    bool force_current = false;
    int energy_blocks = 0; // partial-energy blocks of the last energy evaluation
    CpGraph g_plain;
    unsigned gen = 0; // bumped whenever buffers move (graphs that hold them are stale)
    // displacement-checked rebuilds (0: the reference's fixed schedule only):
    // slot positions at the last build, a device flag set by the integrator
    double disp_max    = 0.0;
    double4* xbuild    = nullptr;
    int xbuild_n       = 0;
    int* dflag         = nullptr;
    int* h_dflag       = nullptr;
    bool snap_valid    = false;
    long long rebuilds_sched = 0, rebuilds_check = 0;
    // the check decided on the device (default; "check_on_host" 1: the host
    // reads the flag every step): one graph per step with conditional nodes
    // that rebuild when the flag is up, and skip the force and every later
    // step of the call once such a rebuild overflowed a buffer (the host
    // grows it, replays that build and resumes). dstate: {stopped, steps
    // run, rebuilds} on the device, h_dstate its pinned copy
    bool check_host    = false;
    int* dstate        = nullptr;
    int* h_dstate      = nullptr;
    cudaStream_t s_cap[2] = {nullptr, nullptr}; // capture streams of the bodies
    CpGraph g_chk;
    // kernels of the checked step graph's parts, for the launch count: the
    // step's fixed part, the ghost update, the rebuild, the force
    long long chk_k[4] = {0, 0, 0, 0};
    long long chk_steps = 0, chk_replays = 0; // graph steps run, overflowed rebuilds replayed
    // pair-list force path of the mixed scheme (force_path 1, mdb_cp_pairs.cu):
    // codes per (i pair, chunk), their counts, the positions they were
    // derived from, and {derive flag, derivations run}
    int force_path        = 0;
    double pair_buffer    = -1.0; // r_in - r_c; < 0: the list's skin
    PairTypes pt;
    unsigned char* pcode  = nullptr;
    unsigned short* pcnt  = nullptr;
    float4* xq            = nullptr;
    int* qflag            = nullptr;
    int pair_ncl = 0, pair_chmax = 0;
};

#define RED_SLOTS 64

#define CK(call)                                                                         \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) return fail(ctx, MDB_ERR_CUDA, #call, e_);                \
    } while (0)

static int fail(MdbCp* ctx, int code, const char* what, cudaError_t e = cudaSuccess)
{
    if (ctx) {
        char buf[512];
        if (e != cudaSuccess) snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
        else snprintf(buf, sizeof buf, "%s", what);
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

static void drop_graph(MdbCp* ctx)
{
    ctx->gen++;
    if (ctx->g_plain.exec) cudaGraphExecDestroy(ctx->g_plain.exec);
    ctx->g_plain.exec    = nullptr;
    ctx->g_plain.kernels = 0;
    if (ctx->g_chk.exec) cudaGraphExecDestroy(ctx->g_chk.exec);
    ctx->g_chk.exec    = nullptr;
    ctx->g_chk.kernels = 0;
}

static int ensure_pairs(MdbCp* ctx);
static int mark_derive(MdbCp* ctx);
static void setup_columns(MdbCp* ctx);
static int alloc_columns(MdbCp* ctx);

static long long mark() { return mdb::g_launches; }
static void account(MdbCp* ctx, long long m) { ctx->launches += mdb::g_launches - m; }

// ---------------------------------------------------------------------------
// setupNeighbor, clusterpair/neighbor.c:108-215 (box at the origin)
static double bindist2(const Geom& g, int i, int j)
{
    double dx, dy;
    if (i > 0) dx = (i - 1) * g.binsizex;
    else if (i == 0) dx = 0.0;
    else dx = (i + 1) * g.binsizex;
    if (j > 0) dy = (j - 1) * g.binsizey;
    else if (j == 0) dy = 0.0;
    else dy = (j + 1) * g.binsizey;
    return dx * dx + dy * dy;
}

static void setup_columns(MdbCp* ctx)
{
    const MdbParams& p = ctx->p;
    Geom& g            = ctx->g;
    const double xprd = p.xprd, yprd = p.yprd, zprd = p.zprd, cut = p.cutneigh;
    double density  = ((double)p.natoms) / ((xprd - 0.0) * (yprd - 0.0) * (zprd - 0.0));
    double in_cell  = (double)std::max(ctx->M, ctx->N);
    double tx       = cbrt(in_cell / density);
    double ty       = cbrt(in_cell / density);
    if (ctx->col_edge_pct != 100) {
        tx *= ctx->col_edge_pct / 100.0;
        ty *= ctx->col_edge_pct / 100.0;
    }
    g.nbinx         = std::max(1, (int)ceil((xprd - 0.0) / tx));
    g.nbiny         = std::max(1, (int)ceil((yprd - 0.0) / ty));
    g.binsizex      = (xprd - 0.0) / g.nbinx;
    g.binsizey      = (yprd - 0.0) / g.nbiny;
    g.bininvx       = 1.0 / g.binsizex;
    g.bininvy       = 1.0 / g.binsizey;
    g.xprd          = xprd;
    g.yprd          = yprd;
    g.zprd          = zprd;
    g.cutneigh      = cut;
    g.cutneighsq    = cut * cut;
    double coord    = 0.0 - cut - 1.0e-6 * xprd;
    g.mbinxlo       = (int)(coord * g.bininvx);
    if (coord < 0.0) g.mbinxlo = g.mbinxlo - 1;
    coord       = xprd + cut + 1.0e-6 * xprd;
    int mbinxhi = (int)(coord * g.bininvx);
    coord       = 0.0 - cut - 1.0e-6 * yprd;
    g.mbinylo   = (int)(coord * g.bininvy);
    if (coord < 0.0) g.mbinylo = g.mbinylo - 1;
    coord       = yprd + cut + 1.0e-6 * yprd;
    int mbinyhi = (int)(coord * g.bininvy);
    g.mbinxlo   = g.mbinxlo - 1;
    mbinxhi     = mbinxhi + 1;
    g.mbinx     = mbinxhi - g.mbinxlo + 1;
    g.mbinylo   = g.mbinylo - 1;
    mbinyhi     = mbinyhi + 1;
    g.mbiny     = mbinyhi - g.mbinylo + 1;
    int nextx   = (int)(cut * g.bininvx);
    int nexty   = (int)(cut * g.bininvy);
    if (nextx * g.binsizex < 0.999 * cut) nextx++;
    if (nexty * g.binsizey < 0.999 * cut) nexty++;
    ctx->stencil.clear();
    for (int j = -nexty; j <= nexty; j++)
        for (int i = -nextx; i <= nextx; i++)
            if (bindist2(g, i, j) < g.cutneighsq) ctx->stencil.push_back(j * g.mbinx + i);
    g.nstencil = (int)ctx->stencil.size();
    g.mbins    = g.mbinx * g.mbiny;
    // buildNeighborCPU, clusterpair/neighbor.c:300-303
    double bbx = 0.5 * (g.binsizex + g.binsizex);
    double bby = 0.5 * (g.binsizey + g.binsizey);
    double rbb = std::max(0.0, cut - 0.5 * sqrt(bbx * bbx + bby * bby));
    g.rbb_sq   = rbb * rbb;
    // coordinates (ghosts included) lie within the box grown by cutneigh;
    // rounding each to FP32 moves a difference by at most 2e, e = |x|max
    // 2^-24, and a squared distance (or box distance) by at most
    // 4e (|dx| + |dy| + |dz|) + 12 e^2 with |d| <= cutneigh near a threshold,
    // plus the FP32 rounding of three products and two sums; doubled
    {
        const double xmax = std::max(g.xprd, std::max(g.yprd, g.zprd)) + 2.0 * cut;
        const double e    = xmax * 0x1p-24;
        const double bnd  = 4.0 * e * 3.0 * cut + 12.0 * e * e + 8.0 * g.cutneighsq * 0x1p-24;
        g.list_margin     = (float)(2.0 * bnd);
    }
    // window table of the list build: buckets of about a quarter of a
    // j-cluster's height over the z range of local and ghost j-clusters
    {
        const double per_col = (double)p.natoms / ((double)ctx->N * g.nbinx * g.nbiny);
        const double span    = zprd + 2.0 * cut + 2.0;
        double dz            = 0.25 * zprd / std::max(per_col, 1.0);
        if (!(dz > span / 8192.0)) dz = span / 8192.0;
        g.z0   = -cut - 1.0;
        g.zinv = 1.0 / dz;
        g.zq   = std::max(1, (int)ceil(span * g.zinv));
    }
}

// computePerTypeLJParameters (common/parameter.c:31-45): per-type sqrt(eps)
// and sigma^3; pairs mix geometrically (clusterpair/force_lj.c:130-132)
static int setup_types(MdbCp* ctx)
{
    int nt = std::max(1, ctx->p.ntypes);
    if (nt > MDB_MAX_TYPES) return fail(ctx, MDB_ERR_ARG, "more than 8 atom types");
    Types& t = ctx->ty;
    memset(&t, 0, sizeof t);
    t.ntypes     = nt;
    bool uniform = true;
    for (int k = 0; k < nt; k++) {
        double e = k < (int)ctx->eps_t.size() ? ctx->eps_t[k] : ctx->p.epsilon;
        double s = k < (int)ctx->sig_t.size() ? ctx->sig_t[k] : ctx->p.sigma;
        t.sqrt_eps[k]   = sqrt(e);
        t.sigma3[k]     = s * s * s;
        t.sqrt_eps_f[k] = (float)t.sqrt_eps[k];
        t.sigma3_f[k]   = (float)t.sigma3[k];
        if (t.sqrt_eps[k] != t.sqrt_eps[0] || t.sigma3[k] != t.sigma3[0]) uniform = false;
    }
    t.uniform     = uniform ? 1 : 0;
    t.force_block   = 128;
    t.force_variant = 2; // measured fastest on B200 at 1M atoms (4x4 and 4x8, full and half)
    t.force_swizzle = 0;
    // four i-clusters per warp: measured fastest on B200 at 1M atoms (4x4 and
    // 4x8, full and half; 170 us against 229 us per launch for one per warp)
    t.force_cpw     = 4;
    // two j atoms per lane (one 256-bit load), one atom type: at 1M atoms 189
    // against 200 us per launch for 4x4 full lists, 159 against 164 us for
    // 4x4 half lists; 4x8 half lists 188 against 182 us; several types (their
    // per-atom tables take the registers) 2.83e9 against 3.65e9 atom-steps/s
    // on the 4-type liquid
    t.force_jpl     = (t.uniform && (ctx->N == 4 || !ctx->p.half_neigh)) ? 2 : 1;
    t.eps0        = t.sqrt_eps[0] * t.sqrt_eps[0];
    t.sigma6_0 = t.sigma3[0] * t.sigma3[0];
    // the pair-list path's constants (geometric mixing, in FP64 then rounded)
    PairTypes& pt = ctx->pt;
    memset(&pt, 0, sizeof pt);
    for (int a = 0; a < MDB_MAX_TYPES; a++)
        for (int b = 0; b < MDB_MAX_TYPES; b++) {
            const int ta = a < nt ? a : 0, tb = b < nt ? b : 0;
            const double e  = t.sqrt_eps[ta] * t.sqrt_eps[tb];
            const double s6 = t.sigma3[ta] * t.sigma3[tb];
            pt.tab[a * MDB_MAX_TYPES + b] =
                make_float4((float)(48.0 * e * s6 * s6), (float)(24.0 * e * s6), (float)s6, (float)e);
        }
    pt.a0     = (float)(48.0 * t.eps0 * t.sigma6_0 * t.sigma6_0);
    pt.b0     = (float)(24.0 * t.eps0 * t.sigma6_0);
    pt.sig6_0 = (float)t.sigma6_0;
    pt.eps0   = t.eps0;
    return MDB_OK;
}

extern "C" const char* mdb_cp_last_error(const MdbCp* ctx) { return ctx ? ctx->err.c_str() : ""; }
extern "C" void* mdb_cp_stream(MdbCp* ctx) { return ctx ? (void*)ctx->s : nullptr; }
extern "C" long long mdb_cp_launch_count(const MdbCp* ctx) { return ctx ? ctx->launches : 0; }

extern "C" int mdb_cp_tune(MdbCp* ctx, const char* key, int value)
{
    if (!ctx || !key) return MDB_ERR_ARG;
    if (!strcmp(key, "force_block")) {
        if (value < 32 || value > 512 || value % 32) return MDB_ERR_ARG;
        drop_graph(ctx);
        ctx->ty.force_block = value;
        return MDB_OK;
    }
    if (!strcmp(key, "force_swizzle")) {
        if (value < 0 || value > 1) return MDB_ERR_ARG;
        drop_graph(ctx);
        ctx->ty.force_swizzle = value;
        return MDB_OK;
    }
    if (!strcmp(key, "force_cpw")) {
        // 8: 4x4 clusters only (a segment of 4 lanes holds one j-cluster)
        if (value != 1 && value != 2 && value != 4 && !(value == 8 && ctx->N == 4))
            return MDB_ERR_ARG;
        drop_graph(ctx);
        ctx->ty.force_cpw = value;
        return MDB_OK;
    }
    if (!strcmp(key, "force_jpl")) {
        // 2: single systems with force_cpw 4
        if (value != 1 && value != 2) return MDB_ERR_ARG;
        drop_graph(ctx);
        ctx->ty.force_jpl = value;
        return MDB_OK;
    }
    if (!strcmp(key, "force_variant")) {
        if (value < 0 || value > 3) return MDB_ERR_ARG;
        drop_graph(ctx);
        ctx->ty.force_variant = value;
        return MDB_OK;
    }
    if (!strcmp(key, "pair_variant")) {
        if (value < 0 || value > 3) return MDB_ERR_ARG;
        drop_graph(ctx);
        ctx->ty.pair_variant = value;
        return MDB_OK;
    }
    if (!strcmp(key, "check_on_host")) {
        // 1: the displacement check's flag is read by the host every step
        if (value < 0 || value > 1) return MDB_ERR_ARG;
        drop_graph(ctx);
        ctx->check_host = value != 0;
        return MDB_OK;
    }
    if (!strcmp(key, "column_edge")) {
        // the column grid sizes the atom and cluster buffers: only before atoms
        if (value < 50 || value > 200) return fail(ctx, MDB_ERR_ARG, "column_edge: 50..200");
        if (ctx->atom_cap != 0)
            return fail(ctx, MDB_ERR_ARG, "column_edge is set before mdb_cp_set_atoms");
        CK(cudaSetDevice(ctx->dev));
        drop_graph(ctx);
        ctx->col_edge_pct = value;
        setup_columns(ctx);
        return alloc_columns(ctx);
    }
    if (!strcmp(key, "force_path")) {
        // compensated contexts run the pair-list kernel only
        if (value < 0 || value > 1 || (value == 1 && !ctx->mixed) || (value == 0 && ctx->comp))
            return MDB_ERR_ARG;
        drop_graph(ctx);
        ctx->force_path = value;
        return ensure_pairs(ctx);
    }
    return fail(ctx, MDB_ERR_ARG, "unknown tuning key");
}

extern "C" int mdb_cp_set_pair_buffer(MdbCp* ctx, double buffer)
{
    if (!ctx || !(buffer == buffer)) return MDB_ERR_ARG;
    drop_graph(ctx);
    ctx->pair_buffer = buffer;
    return mark_derive(ctx);
}

extern "C" int mdb_cp_get_pair_stats(MdbCp* ctx, long long* derivations, long long* codes)
{
    if (!ctx) return MDB_ERR_ARG;
    if (derivations) *derivations = 0;
    if (codes) *codes = 0;
    if (!ctx->qflag) return MDB_OK;
    CK(cudaSetDevice(ctx->dev));
    int q[2] = {0, 0};
    CK(cudaMemcpyAsync(q, ctx->qflag, sizeof q, cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    if (derivations) *derivations = q[1];
    if (codes && ctx->pcnt) {
        // codes of the current clusters (two i pairs per i-cluster)
        CK(cudaMemcpyAsync(ctx->h_cnt, ctx->cnt, CP_SLOTS * sizeof(int), cudaMemcpyDeviceToHost,
            ctx->s));
        CK(cudaStreamSynchronize(ctx->s));
        const size_t n = (size_t)ctx->h_cnt[CP_NCL] * 2 * ctx->pair_chmax;
        std::vector<unsigned short> h(n);
        if (n) {
            CK(cudaMemcpy(h.data(), ctx->pcnt, n * sizeof(unsigned short), cudaMemcpyDeviceToHost));
        }
        long long t = 0;
        for (unsigned short v : h) t += v;
        *codes = t;
    }
    return MDB_OK;
}

extern "C" int mdb_cp_synchronize(MdbCp* ctx)
{
    if (!ctx) return MDB_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->s));
    return MDB_OK;
}

static void free_all(MdbCp* ctx)
{
    dfree(ctx->ax), dfree(ctx->av), dfree(ctx->atom_col), dfree(ctx->col_count);
    dfree(ctx->col_start), dfree(ctx->col_fill), dfree(ctx->col_atoms), dfree(ctx->col_sorted);
    dfree(ctx->gidx), dfree(ctx->gz), dfree(ctx->ncl_col), dfree(ctx->cl_start);
    dfree(ctx->cx), dfree(ctx->cv), dfree(ctx->cf), dfree(ctx->xr), dfree(ctx->cf32);
    dfree(ctx->anchor), dfree(ctx->inat), dfree(ctx->cbin), dfree(ctx->cl_first);
    dfree(ctx->jnat), dfree(ctx->ibbmin), dfree(ctx->ibbmax), dfree(ctx->jbbmin);
    dfree(ctx->jbbmax), dfree(ctx->gcount), dfree(ctx->gstart), dfree(ctx->border);
    dfree(ctx->pbc), dfree(ctx->gcolumn), dfree(ctx->gcol_count), dfree(ctx->gfill);
    dfree(ctx->jcol_n), dfree(ctx->jcol_start), dfree(ctx->gtmp), dfree(ctx->jcol);
    dfree(ctx->ztab);
    dfree(ctx->jcbbmin), dfree(ctx->jcbbmax), dfree(ctx->jcbbf), dfree(ctx->cxf);
    dfree(ctx->stencil_d), dfree(ctx->list), dfree(ctx->numneigh), dfree(ctx->nmasked);
    dfree(ctx->xbuild), dfree(ctx->dflag);
    dfree(ctx->pcode), dfree(ctx->pcnt), dfree(ctx->xq), dfree(ctx->qflag);
    ctx->pair_ncl = ctx->pair_chmax = 0;
    if (ctx->h_dflag) cudaFreeHost(ctx->h_dflag);
    ctx->h_dflag  = nullptr;
    dfree(ctx->dstate);
    if (ctx->h_dstate) cudaFreeHost(ctx->h_dstate);
    ctx->h_dstate = nullptr;
    ctx->xbuild_n = 0;
    dfree(ctx->cnt), dfree(ctx->zext), dfree(ctx->scan_scratch), dfree(ctx->partials);
    dfree(ctx->red), dfree(ctx->stage), dfree(ctx->stage_i);
    if (ctx->h_cnt) cudaFreeHost(ctx->h_cnt);
    if (ctx->h_red) cudaFreeHost(ctx->h_red);
    ctx->h_cnt = nullptr;
    ctx->h_red = nullptr;
}

extern "C" int mdb_cp_destroy(MdbCp* ctx)
{
    if (!ctx) return MDB_ERR_ARG;
    cudaSetDevice(ctx->dev);
    if (ctx->s) cudaStreamSynchronize(ctx->s);
    drop_graph(ctx);
    free_all(ctx);
    if (ctx->s) cudaStreamDestroy(ctx->s);
    for (cudaStream_t c : ctx->s_cap)
        if (c) cudaStreamDestroy(c);
    delete ctx;
    return MDB_OK;
}

// arrays sized by the column grid (setup_columns), with the stencil copied
static int alloc_columns(MdbCp* ctx)
{
    cudaError_t e;
    const int mb1 = ctx->g.mbins + 1;
    dfree(ctx->stencil_d), dfree(ctx->col_count), dfree(ctx->col_start), dfree(ctx->col_fill);
    dfree(ctx->ncl_col), dfree(ctx->cl_start), dfree(ctx->gcol_count), dfree(ctx->gfill);
    dfree(ctx->jcol_n), dfree(ctx->jcol_start), dfree(ctx->ztab);
    if ((e = dalloc(&ctx->stencil_d, ctx->g.nstencil)) != cudaSuccess ||
        (e = dalloc(&ctx->col_count, mb1)) != cudaSuccess ||
        (e = dalloc(&ctx->col_start, mb1 + 1)) != cudaSuccess ||
        (e = dalloc(&ctx->col_fill, mb1)) != cudaSuccess ||
        (e = dalloc(&ctx->ncl_col, mb1)) != cudaSuccess ||
        (e = dalloc(&ctx->cl_start, mb1 + 1)) != cudaSuccess ||
        (e = dalloc(&ctx->gcol_count, mb1)) != cudaSuccess ||
        (e = dalloc(&ctx->gfill, mb1)) != cudaSuccess ||
        (e = dalloc(&ctx->jcol_n, mb1)) != cudaSuccess ||
        (e = dalloc(&ctx->jcol_start, mb1 + 1)) != cudaSuccess ||
        (e = dalloc(&ctx->ztab, (size_t)ctx->g.mbins * (ctx->g.zq + 2))) != cudaSuccess)
        return fail(ctx, MDB_ERR_NOMEM, "device allocation (columns)", e);
    if ((e = cudaMemcpy(ctx->stencil_d, ctx->stencil.data(), sizeof(int) * ctx->g.nstencil,
             cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(ctx, MDB_ERR_CUDA, "stencil copy", e);
    return MDB_OK;
}

extern "C" int mdb_cp_create(const MdbParams* params, int cluster_n, int prune_every, MdbCp** out)
{
    if (!params || !out) return MDB_ERR_ARG;
    *out        = nullptr;
    MdbCp* ctx  = new MdbCp();
    ctx->p      = *params;
    MdbParams& p = ctx->p;
    int rc       = MDB_OK;
    if (p.ntypes < 1) p.ntypes = 1;
    if (p.epsilon_per_type) ctx->eps_t.assign(p.epsilon_per_type, p.epsilon_per_type + p.ntypes);
    if (p.sigma_per_type) ctx->sig_t.assign(p.sigma_per_type, p.sigma_per_type + p.ntypes);
    p.epsilon_per_type = nullptr;
    p.sigma_per_type   = nullptr;
    if (p.reneigh_every < 1) p.reneigh_every = 20;
    if (p.nstat < 1) p.nstat = 100;
    ctx->maxneighs   = p.maxneighs > 0 ? p.maxneighs : 200;
    ctx->prune_every = prune_every > 0 ? prune_every : 1000;
    ctx->N           = cluster_n;
    ctx->jfac        = cluster_n / CP_M;
    ctx->mixed       = p.precision == MDB_PREC_MIXED || p.precision == MDB_PREC_MIXED_COMP;
    ctx->comp        = p.precision == MDB_PREC_MIXED_COMP;
    ctx->force_path  = ctx->comp ? 1 : 0;
    ctx->cutforcesq  = p.cutforce * p.cutforce;
    if ((cluster_n != 4 && cluster_n != 8) || p.force_field != MDB_FF_LJ ||
        !(p.precision == MDB_PREC_FP64 || p.precision == MDB_PREC_MIXED ||
            p.precision == MDB_PREC_MIXED_COMP) ||
        !(p.xprd > 0 && p.yprd > 0 && p.zprd > 0) || !(p.cutforce > 0) ||
        !(p.cutneigh >= p.cutforce) || p.natoms < 1 || ctx->maxneighs > 12288) {
        rc = fail(ctx, MDB_ERR_ARG, "invalid parameters for the cluster-pair scheme");
        goto bad;
    }
    // the mixed path's anchors are multiples of 1/8 held in FP32
    if (ctx->mixed && std::max(p.xprd, std::max(p.yprd, p.zprd)) > 1.0e5) {
        rc = fail(ctx, MDB_ERR_ARG, "box too large for FP32 cluster anchors");
        goto bad;
    }
    setup_columns(ctx);
    if ((rc = setup_types(ctx)) != MDB_OK) goto bad;
    // setupThermo, common/thermo.c:35-58 (LJ units)
    ctx->dof_boltz = (p.natoms * 3 - 3);
    ctx->t_scale   = 1.0 / ctx->dof_boltz;
    ctx->p_scale   = 1.0 / 3 / p.xprd / p.yprd / p.zprd;
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
        if ((e = dalloc(&ctx->cnt, CP_SLOTS)) != cudaSuccess ||
            (e = dalloc(&ctx->zext, 1)) != cudaSuccess ||
            (e = dalloc(&ctx->red, 4 * RED_SLOTS)) != cudaSuccess ||
            (e = cudaMallocHost((void**)&ctx->h_cnt, CP_SLOTS * sizeof(int))) != cudaSuccess ||
            (e = cudaMallocHost((void**)&ctx->h_red, 4 * RED_SLOTS * sizeof(double))) !=
                cudaSuccess) {
            rc = fail(ctx, MDB_ERR_NOMEM, "device allocation", e);
            goto bad;
        }
        cudaMemset(ctx->cnt, 0, CP_SLOTS * sizeof(int));
        if ((rc = alloc_columns(ctx)) != MDB_OK) goto bad;
    }
    *out = ctx;
    return MDB_OK;
bad:
    fprintf(stderr, "mdb_cp_create: %s\n", ctx->err.c_str());
    mdb_cp_destroy(ctx);
    return rc;
}

// ---------------------------------------------------------------------------
// buffers sized by the atom count (clusters) and by the ghost capacity
static int alloc_atoms(MdbCp* ctx, int n)
{
    cudaError_t e;
    const int mb = ctx->g.mbins;
    // clusters: ceil(c / M) per column, +1 per column for even pairs (M < N)
    ctx->ncl_cap  = n / ctx->M + 2 * mb + 8;
    ctx->ncj_cap  = ctx->ncl_cap / ctx->jfac + 1;
    ctx->ld       = ctx->ncl_cap;
    ctx->atom_cap = n;
    dfree(ctx->ax), dfree(ctx->av), dfree(ctx->atom_col), dfree(ctx->col_atoms);
    dfree(ctx->col_sorted), dfree(ctx->gidx), dfree(ctx->gz), dfree(ctx->inat), dfree(ctx->cbin);
    dfree(ctx->cl_first), dfree(ctx->ibbmin), dfree(ctx->ibbmax), dfree(ctx->gcount);
    dfree(ctx->gstart), dfree(ctx->numneigh), dfree(ctx->nmasked), dfree(ctx->list);
    dfree(ctx->scan_scratch), dfree(ctx->partials), dfree(ctx->stage), dfree(ctx->stage_i);
    int scan_n          = std::max(std::max(mb + 2, ctx->ncj_cap + 1), 1);
    ctx->scan_scratch_n = scan_scratch_ints(scan_n);
    // energy partials: one per force block (mixed blocks of 32 threads at the least)
    ctx->npart = std::max(4 * force_blocks(ctx->ncl_cap), ke_blocks(ctx->ncl_cap * ctx->M));
    ctx->stage_n = (size_t)3 * std::max(n, 1) * 3;
    if ((e = dalloc(&ctx->ax, n)) != cudaSuccess || (e = dalloc(&ctx->av, n)) != cudaSuccess ||
        (e = dalloc(&ctx->atom_col, n)) != cudaSuccess ||
        (e = dalloc(&ctx->col_atoms, n)) != cudaSuccess ||
        (e = dalloc(&ctx->col_sorted, n)) != cudaSuccess ||
        (e = dalloc(&ctx->gidx, 2 * (size_t)n + 2)) != cudaSuccess ||
        (e = dalloc(&ctx->gz, 2 * (size_t)n + 2)) != cudaSuccess ||
        (e = dalloc(&ctx->inat, ctx->ncl_cap)) != cudaSuccess ||
        (e = dalloc(&ctx->cbin, ctx->ncl_cap)) != cudaSuccess ||
        (e = dalloc(&ctx->cl_first, ctx->ncl_cap)) != cudaSuccess ||
        (e = dalloc(&ctx->ibbmin, ctx->ncl_cap)) != cudaSuccess ||
        (e = dalloc(&ctx->ibbmax, ctx->ncl_cap)) != cudaSuccess ||
        (e = dalloc(&ctx->gcount, ctx->ncj_cap)) != cudaSuccess ||
        (e = dalloc(&ctx->gstart, ctx->ncj_cap + 1)) != cudaSuccess ||
        (e = dalloc(&ctx->numneigh, ctx->ncl_cap)) != cudaSuccess ||
        (e = dalloc(&ctx->nmasked, ctx->ncl_cap)) != cudaSuccess ||
        (e = dalloc(&ctx->list, (size_t)ctx->maxneighs * ctx->ld)) != cudaSuccess ||
        (e = dalloc(&ctx->scan_scratch, ctx->scan_scratch_n)) != cudaSuccess ||
        (e = dalloc(&ctx->partials, 2 * (size_t)ctx->npart)) != cudaSuccess ||
        (e = dalloc(&ctx->stage, ctx->stage_n)) != cudaSuccess ||
        (e = dalloc(&ctx->stage_i, std::max(n, 1))) != cudaSuccess)
        return fail(ctx, MDB_ERR_NOMEM, "device allocation (atoms)", e);
    cudaMemsetAsync(ctx->numneigh, 0, sizeof(int) * ctx->ncl_cap, ctx->s);
    return MDB_OK;
}

static int alloc_ghosts(MdbCp* ctx, int ngc_cap)
{
    cudaError_t e;
    drop_graph(ctx);
    ctx->ngc_cap  = ngc_cap;
    const int nj  = ctx->ncj_cap + ngc_cap + 1;
    ctx->slot_cap = nj * ctx->N;
    dfree(ctx->cx), dfree(ctx->cv), dfree(ctx->cf), dfree(ctx->xr), dfree(ctx->cf32);
    dfree(ctx->anchor), dfree(ctx->jnat), dfree(ctx->jbbmin), dfree(ctx->jbbmax);
    dfree(ctx->border), dfree(ctx->pbc), dfree(ctx->gcolumn), dfree(ctx->gtmp), dfree(ctx->jcol);
    dfree(ctx->jcbbmin), dfree(ctx->jcbbmax), dfree(ctx->jcbbf), dfree(ctx->cxf);
    if ((e = dalloc(&ctx->cx, ctx->slot_cap)) != cudaSuccess ||
        (e = dalloc(&ctx->jcbbmin, nj)) != cudaSuccess ||
        (e = dalloc(&ctx->jcbbf, 2 * (size_t)nj)) != cudaSuccess ||
        (e = dalloc(&ctx->cxf, ctx->slot_cap)) != cudaSuccess ||
        (e = dalloc(&ctx->jcbbmax, nj)) != cudaSuccess ||
        (e = dalloc(&ctx->cv, ctx->slot_cap)) != cudaSuccess ||
        (e = dalloc(&ctx->cf, ctx->slot_cap)) != cudaSuccess ||
        (e = dalloc(&ctx->jnat, nj)) != cudaSuccess ||
        (e = dalloc(&ctx->jbbmin, nj)) != cudaSuccess ||
        (e = dalloc(&ctx->jbbmax, nj)) != cudaSuccess ||
        (e = dalloc(&ctx->border, ngc_cap)) != cudaSuccess ||
        (e = dalloc(&ctx->pbc, ngc_cap)) != cudaSuccess ||
        (e = dalloc(&ctx->gcolumn, ngc_cap)) != cudaSuccess ||
        (e = dalloc(&ctx->gtmp, nj)) != cudaSuccess || (e = dalloc(&ctx->jcol, nj)) != cudaSuccess)
        return fail(ctx, MDB_ERR_NOMEM, "device allocation (ghosts)", e);
    if (ctx->mixed) {
        if ((e = dalloc(&ctx->xr, ctx->slot_cap)) != cudaSuccess ||
            (e = dalloc(&ctx->cf32, ctx->slot_cap)) != cudaSuccess ||
            (e = dalloc(&ctx->anchor, nj)) != cudaSuccess)
            return fail(ctx, MDB_ERR_NOMEM, "device allocation (ghosts)", e);
    }
    cudaMemsetAsync(ctx->cf, 0, sizeof(double4) * ctx->slot_cap, ctx->s);
    if (ctx->cf32) cudaMemsetAsync(ctx->cf32, 0, sizeof(float4) * ctx->slot_cap, ctx->s);
    ctx->have_clusters = ctx->have_ghosts = ctx->have_list = false;
    return MDB_OK;
}

static int alloc_list(MdbCp* ctx, int maxneighs)
{
    if (maxneighs > 12288) return fail(ctx, MDB_ERR_OVERFLOW, "cluster list longer than 12288");
    drop_graph(ctx);
    dfree(ctx->list);
    ctx->maxneighs = maxneighs;
    CK(dalloc(&ctx->list, (size_t)maxneighs * ctx->ld));
    return MDB_OK;
}

// r_in - r_c of the pair-list path
static double pair_buffer(const MdbCp* ctx)
{
    return ctx->pair_buffer >= 0.0 ? ctx->pair_buffer : ctx->p.cutneigh - ctx->p.cutforce;
}

// the next force evaluation derives the pair codes again
static int mark_derive(MdbCp* ctx)
{
    if (!ctx->qflag) return MDB_OK;
    CK(cudaMemsetAsync(ctx->qflag, 1, sizeof(int), ctx->s)); // any non-zero value
    return MDB_OK;
}

// Buffers of the pair-list path for the current cluster and list capacities
// (called after builds, never inside a capture: buffers that move drop the
// captured graphs), then a derivation is due.
static int ensure_pairs(MdbCp* ctx)
{
    if (!ctx->mixed || ctx->force_path != 1 || ctx->ncl_cap <= 0) return MDB_OK;
    const int chmax = pair_chunks(ctx->maxneighs, ctx->N);
    if (!ctx->qflag) {
        CK(dalloc(&ctx->qflag, 3));
        CK(cudaMemsetAsync(ctx->qflag, 0, 3 * sizeof(int), ctx->s));
    }
    if (ctx->pair_ncl < ctx->ncl_cap || ctx->pair_chmax != chmax) {
        drop_graph(ctx);
        dfree(ctx->pcode), dfree(ctx->pcnt), dfree(ctx->xq);
        ctx->pair_ncl = ctx->pair_chmax = 0;
        const size_t n2 = (size_t)ctx->ncl_cap * 2 * chmax;
        CK(dalloc(&ctx->pcode, n2 * 256));
        CK(dalloc(&ctx->pcnt, n2));
        CK(dalloc(&ctx->xq, (size_t)ctx->ncl_cap * 4));
        ctx->pair_ncl   = ctx->ncl_cap;
        ctx->pair_chmax = chmax;
    }
    return mark_derive(ctx);
}

#define NEED_ATOMS()                                                                     \
    do {                                                                                 \
        if (!ctx) return MDB_ERR_ARG;                                                    \
        if (!ctx->have_atoms) return fail(ctx, MDB_ERR_STATE, "no atoms set");           \
    } while (0)

// AoS host triples <-> double4 atom arrays, converted on the device so that
// pinned host buffers move by DMA at full speed
__global__ void k_cp_pack_atoms(int n, const double* __restrict__ xa,
    const double* __restrict__ va, const int* __restrict__ ta, int has_t, double4* ax,
    double4* av, int ntypes, int* bad)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int t = has_t ? ta[i] : 0;
    if (t < 0 || t >= ntypes) atomicAdd(bad, 1);
    ax[i] = make_double4(xa[3 * i], xa[3 * i + 1], xa[3 * i + 2], type_bits(t));
    av[i] = make_double4(va[3 * i], va[3 * i + 1], va[3 * i + 2], 0.0);
}

__global__ void k_cp_unpack_atoms(int n, const double4* __restrict__ ax,
    const double4* __restrict__ av, double* xa, double* va, int* ta)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 p = ax[i], q = av[i];
    xa[3 * i] = p.x, xa[3 * i + 1] = p.y, xa[3 * i + 2] = p.z;
    va[3 * i] = q.x, va[3 * i + 1] = q.y, va[3 * i + 2] = q.z;
    ta[i] = slot_type(p);
}

extern "C" int mdb_cp_set_atoms(MdbCp* ctx, int nlocal, const double* x, const double* v,
    const int* type)
{
    if (!ctx || nlocal < 1 || !x || !v) return MDB_ERR_ARG;
    CK(cudaSetDevice(ctx->dev));
    if (nlocal != ctx->atom_cap) {
        CK(cudaStreamSynchronize(ctx->s));
        drop_graph(ctx);
        int rc = alloc_atoms(ctx, nlocal);
        if (rc) return rc;
        // ghost j-clusters: start from the surface layer estimate (grown on
        // overflow); the slot arrays depend on the local cluster capacity too
        const MdbParams& p = ctx->p;
        double vol   = p.xprd * p.yprd * p.zprd;
        double shell = (p.xprd + 2 * p.cutneigh + 4) * (p.yprd + 2 * p.cutneigh + 4) *
                           (p.zprd + 2 * p.cutneigh + 4) -
                       vol;
        double est = 1.5 * shell / vol * nlocal / ctx->N + 1024;
        est        = std::max(est, (double)ctx->ngc_cap);
        rc         = alloc_ghosts(ctx, (int)std::min(est, 2.0e9 / ctx->N));
        if (rc) return rc;
    }
    ctx->nlocal       = nlocal;
    cudaStream_t s    = ctx->s;
    const size_t n3   = 3 * (size_t)nlocal;
    double* sx        = ctx->stage;
    double* sv        = ctx->stage + n3;
    int* bad          = ctx->cnt + CP_BADBIN; // reused as a scratch flag here
    CK(cudaMemsetAsync(bad, 0, sizeof(int), s));
    CK(cudaMemcpyAsync(sx, x, sizeof(double) * n3, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(sv, v, sizeof(double) * n3, cudaMemcpyHostToDevice, s));
    if (type)
        CK(cudaMemcpyAsync(ctx->stage_i, type, sizeof(int) * nlocal, cudaMemcpyHostToDevice, s));
    k_cp_pack_atoms<<<mdb_blocks(nlocal, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(nlocal, sx, sv,
        ctx->stage_i, type ? 1 : 0, ctx->ax, ctx->av, ctx->ty.ntypes, bad);
    ctx->launches++;
    int hbad = 0;
    CK(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (hbad) return fail(ctx, MDB_ERR_ARG, "atom type out of range");
    ctx->have_atoms    = true;
    ctx->have_clusters = ctx->have_ghosts = ctx->have_list = false;
    ctx->energy_valid = ctx->force_current = false;
    return MDB_OK;
}

extern "C" int mdb_cp_get_atoms(MdbCp* ctx, double* x, double* v, int* type)
{
    NEED_ATOMS();
    const int n       = ctx->nlocal;
    const size_t n3   = 3 * (size_t)n;
    cudaStream_t s    = ctx->s;
    k_cp_unpack_atoms<<<mdb_blocks(n, MDB_NTHREADS), MDB_NTHREADS, 0, s>>>(n, ctx->ax, ctx->av,
        ctx->stage, ctx->stage + n3, ctx->stage_i);
    ctx->launches++;
    if (x) CK(cudaMemcpyAsync(x, ctx->stage, sizeof(double) * n3, cudaMemcpyDeviceToHost, s));
    if (v) CK(cudaMemcpyAsync(v, ctx->stage + n3, sizeof(double) * n3, cudaMemcpyDeviceToHost, s));
    if (type) CK(cudaMemcpyAsync(type, ctx->stage_i, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return MDB_OK;
}

// ---------------------------------------------------------------------------
// enqueue helpers (stream-ordered, graph-capturable)
// put_rel mode of xr: 0 FP64 (no xr), 1 mixed with type bits, 2 mixed with one
// atom type (anchor components in .w, read by the UNIFORM force kernels)
static int xr_mode(const MdbCp* ctx) { return ctx->mixed ? (ctx->ty.uniform ? 2 : 1) : 0; }

static void enq_clusters(MdbCp* ctx)
{
    cudaStream_t s = ctx->s;
    const Geom& g  = ctx->g;
    const int mb1  = g.mbins + 1;
    cudaMemsetAsync(ctx->col_count, 0, sizeof(int) * mb1, s);
    cudaMemsetAsync(ctx->col_fill, 0, sizeof(int) * mb1, s);
    cudaMemsetAsync(ctx->ncl_col, 0, sizeof(int) * mb1, s);
    cudaMemsetAsync(ctx->zext, 0, sizeof(unsigned long long), s);
    launch_bin_atoms(s, ctx->nlocal, ctx->ax, g, ctx->atom_col, ctx->col_count, ctx->cnt);
    scan_exclusive(ctx->col_count, ctx->col_start, g.mbins, ctx->scan_scratch, s);
    launch_scatter_atoms(s, ctx->nlocal, ctx->atom_col, ctx->col_start, ctx->col_fill,
        ctx->col_atoms);
    launch_sort_columns(s, g, ctx->M, ctx->N, ctx->col_start, ctx->col_atoms, ctx->ax,
        ctx->col_sorted, ctx->gidx, ctx->gz, ctx->ncl_col);
    scan_exclusive(ctx->ncl_col, ctx->cl_start, mb1, ctx->scan_scratch, s);
    launch_build_clusters(s, g, ctx->M, ctx->N, xr_mode(ctx), ctx->col_start, ctx->col_sorted,
        ctx->cl_start, ctx->ax, ctx->av, ctx->cx, ctx->cv, ctx->inat, ctx->cbin, ctx->cl_first,
        ctx->ibbmin, ctx->ibbmax, ctx->jnat, ctx->jbbmin, ctx->jbbmax, ctx->anchor, ctx->xr,
        ctx->cnt, ctx->zext);
}

static void enq_setup_pbc(MdbCp* ctx)
{
    cudaStream_t s = ctx->s;
    cudaMemsetAsync(ctx->cnt + CP_NGHOST_ATOMS, 0, sizeof(int), s);
    launch_ghost_count(s, ctx->ncj_cap, ctx->cnt, ctx->jnat, ctx->jbbmin, ctx->jbbmax, ctx->g,
        ctx->gcount);
    scan_exclusive(ctx->gcount, ctx->gstart, ctx->ncj_cap, ctx->scan_scratch, s);
    launch_ghost_write(s, ctx->ncj_cap, ctx->ngc_cap, ctx->cnt, ctx->jnat, ctx->jbbmin,
        ctx->jbbmax, ctx->g, ctx->gstart, ctx->border, ctx->pbc);
    launch_ghost_first(s, ctx->N, ctx->ngc_cap, xr_mode(ctx), ctx->cnt, ctx->border, ctx->pbc,
        ctx->g, ctx->cx, ctx->jnat, ctx->jbbmin, ctx->jbbmax, ctx->anchor, ctx->xr, ctx->zext);
}

static void enq_bin_j(MdbCp* ctx)
{
    cudaStream_t s = ctx->s;
    const int mb1  = ctx->g.mbins + 1;
    cudaMemsetAsync(ctx->gcol_count, 0, sizeof(int) * mb1, s);
    cudaMemsetAsync(ctx->gfill, 0, sizeof(int) * mb1, s);
    launch_ghost_columns(s, ctx->N, ctx->ngc_cap, ctx->cnt, ctx->pbc, ctx->jnat, ctx->cx, ctx->g,
        ctx->gcolumn, ctx->gcol_count);
    launch_column_sizes(s, mb1, ctx->jfac, ctx->ncl_col, ctx->gcol_count, ctx->jcol_n);
    scan_exclusive(ctx->jcol_n, ctx->jcol_start, mb1, ctx->scan_scratch, s);
    launch_ghost_scatter(s, ctx->ngc_cap, ctx->cnt, ctx->gcolumn, ctx->jcol_start, ctx->ncl_col,
        ctx->jfac, ctx->gfill, ctx->gtmp);
    launch_merge_columns(s, mb1, ctx->jfac, ctx->ncl_col, ctx->cl_start, ctx->gcol_count,
        ctx->jcol_start, ctx->gtmp, ctx->jbbmin, ctx->jbbmax, ctx->jcol, ctx->jcbbmin,
        ctx->jcbbmax);
}

// list layout: row-major for the mixed kernel, k-major for the FP64 one
static int lks(const MdbCp* ctx) { return ctx->mixed ? 1 : ctx->ld; }
static int lcs(const MdbCp* ctx) { return ctx->mixed ? ctx->maxneighs : 1; }

static void enq_list(MdbCp* ctx)
{
    launch_list_prep(ctx->s, ctx->N, ctx->slot_cap, ctx->g, ctx->cnt, ctx->jcol_start,
        ctx->jcbbmin, ctx->jcbbmax, ctx->cx, ctx->jcbbf, ctx->cxf, ctx->ztab);
    launch_build_list(ctx->s, ctx->M, ctx->N, ctx->p.half_neigh, ctx->ncl_cap, ctx->cnt, ctx->g,
        ctx->stencil_d, ctx->cbin, ctx->ibbmin, ctx->ibbmax, ctx->jcbbmin, ctx->jcbbmax, ctx->cx,
        ctx->jcbbf, ctx->cxf, ctx->jcol, ctx->ztab, ctx->zext, ctx->maxneighs, lks(ctx),
        lcs(ctx), ctx->list, ctx->numneigh, ctx->nmasked, ctx->cnt);
}

static void clear_build_counters(MdbCp* ctx)
{
    // CP_MAXNEED, CP_BADBIN
    cudaMemsetAsync(ctx->cnt + CP_MAXNEED, 0, 2 * sizeof(int), ctx->s);
}

// buildClusters .. buildNeighbor from the atom arrays (idempotent)
static void enq_build(MdbCp* ctx)
{
    clear_build_counters(ctx);
    enq_clusters(ctx);
    enq_setup_pbc(ctx);
    enq_bin_j(ctx);
    enq_list(ctx);
}

static void enq_gather(MdbCp* ctx, int wrap)
{
    launch_gather(ctx->s, ctx->M, ctx->ncl_cap, ctx->cnt, ctx->cx, ctx->cv, ctx->cl_first,
        ctx->ax, ctx->av, wrap, ctx->p.xprd, ctx->p.yprd, ctx->p.zprd);
}

// Reads the counters; grows what overflowed. 1: replay the build, 0: done,
// <0: error (negated status). what: the stages that ran.
enum { CHK_CLUSTERS = 1, CHK_GHOSTS = 2, CHK_LIST = 4, CHK_ALL = 7 };

// evaluates counters already copied to ctx->h_cnt
static int eval_build(MdbCp* ctx, int what)
{
    const int* h = ctx->h_cnt;
    if (h[CP_BADBIN] > 0) return -fail(ctx, MDB_ERR_OVERFLOW, "atom outside the column grid");
    if ((what & CHK_GHOSTS) && h[CP_NGC_TOTAL] > ctx->ngc_cap) {
        int rc = alloc_ghosts(ctx, (int)(h[CP_NGC_TOTAL] * 1.2) + 1024);
        if (rc) return -rc;
        return 1;
    }
    if ((what & CHK_LIST) && h[CP_MAXNEED] >= ctx->maxneighs) {
        // buildNeighborCPU: maxneighs = 1.2 x the longest row, then rebuild
        int rc = alloc_list(ctx, (int)(h[CP_MAXNEED] * 1.2));
        if (rc) return -rc;
        return 1;
    }
    return 0;
}

static int check_build(MdbCp* ctx, int what)
{
    cudaError_t e = cudaMemcpyAsync(ctx->h_cnt, ctx->cnt, CP_SLOTS * sizeof(int),
        cudaMemcpyDeviceToHost, ctx->s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->s);
    if (e != cudaSuccess) return -fail(ctx, MDB_ERR_CUDA, "rebuild check", e);
    return eval_build(ctx, what);
}

// positions of the slots as built, for the displacement check
static int snapshot(MdbCp* ctx)
{
    if (ctx->disp_max <= 0.0) return MDB_OK;
    const int n = ctx->ncl_cap * ctx->M;
    if (ctx->xbuild_n < n) {
        dfree(ctx->xbuild);
        CK(dalloc(&ctx->xbuild, n));
        ctx->xbuild_n = n;
        drop_graph(ctx);
    }
    if (!ctx->dflag) {
        CK(dalloc(&ctx->dflag, 1));
        CK(cudaMallocHost((void**)&ctx->h_dflag, sizeof(int)));
    }
    CK(cudaMemcpyAsync(ctx->xbuild, ctx->cx, sizeof(double4) * n, cudaMemcpyDeviceToDevice,
        ctx->s));
    CK(cudaMemsetAsync(ctx->dflag, 0, sizeof(int), ctx->s));
    ctx->snap_valid = true;
    return MDB_OK;
}

static int do_build(MdbCp* ctx)
{
    ctx->force_current = false;
    for (int attempt = 0; attempt < 8; attempt++) {
        long long m = mark();
        enq_build(ctx);
        account(ctx, m);
        int r = check_build(ctx, CHK_ALL);
        if (r < 0) return -r;
        if (r == 0) {
            ctx->have_clusters = ctx->have_ghosts = ctx->have_list = true;
            int rc = ensure_pairs(ctx);
            if (rc) return rc;
            return snapshot(ctx);
        }
    }
    return fail(ctx, MDB_ERR_OVERFLOW, "rebuild did not converge");
}

static bool pair_path(const MdbCp* ctx) { return ctx->mixed && ctx->force_path == 1 && ctx->qflag; }

// pair codes, when an atom moved past half the buffer, a build asked for it,
// or force
static void enq_derive(MdbCp* ctx, int force)
{
    const double rin = ctx->p.cutforce + pair_buffer(ctx);
    launch_pair_derive(ctx->s, ctx->N, ctx->p.half_neigh, ctx->ty.uniform, ctx->ncl_cap, ctx->cnt,
        ctx->xr, ctx->anchor, ctx->list, lcs(ctx), ctx->numneigh, (float)(rin * rin), ctx->qflag,
        force, ctx->pcode, ctx->pcnt, ctx->pair_chmax, ctx->xq);
}

static int enq_force_pairs(MdbCp* ctx, bool energy)
{
    CompArgs ca;
    if (ctx->comp) ca.cx = ctx->cx, ca.cf64 = ctx->cf, ca.cutsq = ctx->cutforcesq;
    return launch_force_pairs(ctx->s, ctx->N, ctx->p.half_neigh, energy, ctx->ty.uniform,
        ctx->ty.pair_variant, ctx->ncl_cap, ctx->cnt, ctx->xr, ctx->anchor, ctx->pt,
        (float)ctx->cutforcesq, ctx->list, lcs(ctx), ctx->numneigh, ctx->pcode, ctx->pcnt,
        ctx->pair_chmax, ctx->cf32, ctx->partials, ctx->qflag, ca);
}

// the FP32 force slots the integrator reads (null: it reads the FP64 slots,
// as FP64 and compensated contexts keep their forces there)
static float4* f32_slots(const MdbCp* ctx) { return ctx->mixed && !ctx->comp ? ctx->cf32 : nullptr; }

// the integrator's test of the pair-list path: half the buffer, less a
// margin for the FP32 rounding of the positions it compares
static float pair_qlim2(const MdbCp* ctx)
{
    const double q = 0.5 * pair_buffer(ctx) * 0.999;
    return (float)(q * q);
}

static void enq_force(MdbCp* ctx, bool energy)
{
    cudaStream_t s = ctx->s;
    const int nloc_slots = ctx->ncl_cap * ctx->M;
    if (pair_path(ctx)) {
        if (ctx->p.half_neigh && ctx->comp)
            cudaMemsetAsync(ctx->cf, 0, sizeof(double4) * (size_t)nloc_slots, s);
        else if (ctx->p.half_neigh)
            cudaMemsetAsync(ctx->cf32, 0, sizeof(float4) * (size_t)nloc_slots, s);
        enq_derive(ctx, 0);
        const int nb = enq_force_pairs(ctx, energy);
        if (energy) ctx->energy_blocks = nb;
    } else if (ctx->mixed) {
        if (ctx->p.half_neigh)
            cudaMemsetAsync(ctx->cf32, 0, sizeof(float4) * (size_t)nloc_slots, s);
        const int nb = launch_force_mixed(s, ctx->N, ctx->p.half_neigh, energy, ctx->ncl_cap,
            ctx->cnt, ctx->xr, ctx->anchor, ctx->ty, (float)ctx->cutforcesq, ctx->list, lks(ctx),
            lcs(ctx), ctx->numneigh, ctx->cf32, ctx->partials);
        if (energy) ctx->energy_blocks = nb;
    } else {
        if (ctx->p.half_neigh)
            cudaMemsetAsync(ctx->cf, 0, sizeof(double4) * (size_t)nloc_slots, s);
        launch_force_fp64(s, ctx->M, ctx->N, ctx->p.half_neigh, energy, ctx->ncl_cap, ctx->cnt,
            ctx->cx, ctx->ty, ctx->cutforcesq, ctx->list, lks(ctx), lcs(ctx), ctx->numneigh,
            ctx->cf, ctx->partials);
        if (energy) ctx->energy_blocks = mdb_blocks((long long)ctx->ncl_cap * 4, 128);
    }
}

// the displacement check's arguments for the integrator (none when off)
static const double4* check_xb(const MdbCp* ctx)
{
    return ctx->disp_max > 0.0 && ctx->snap_valid ? ctx->xbuild : nullptr;
}

static void enq_initial(MdbCp* ctx)
{
    const bool pq = pair_path(ctx);
    launch_cp_initial(ctx->s, ctx->M, ctx->N, ctx->ncl_cap, ctx->cnt, ctx->p.dtforce, ctx->p.dt,
        ctx->cx, ctx->cv, ctx->cf, f32_slots(ctx), ctx->anchor,
        ctx->mixed ? ctx->xr : nullptr, xr_mode(ctx), check_xb(ctx),
        ctx->disp_max * ctx->disp_max, ctx->dflag, pq ? ctx->xq : nullptr, pair_qlim2(ctx),
        pq ? ctx->qflag : nullptr);
}

static void enq_final(MdbCp* ctx)
{
    launch_cp_final(ctx->s, ctx->M, ctx->ncl_cap, ctx->cnt, ctx->p.dtforce, ctx->cx, ctx->cv,
        ctx->cf, f32_slots(ctx));
}

static void enq_final_initial(MdbCp* ctx)
{
    const bool pq = pair_path(ctx);
    launch_cp_final_initial(ctx->s, ctx->M, ctx->N, ctx->ncl_cap, ctx->cnt, ctx->p.dtforce,
        ctx->p.dt, ctx->cx, ctx->cv, ctx->cf, f32_slots(ctx), ctx->anchor,
        ctx->mixed ? ctx->xr : nullptr, xr_mode(ctx), check_xb(ctx),
        ctx->disp_max * ctx->disp_max, ctx->dflag, pq ? ctx->xq : nullptr, pair_qlim2(ctx),
        pq ? ctx->qflag : nullptr);
}

static void enq_ghost_update(MdbCp* ctx)
{
    launch_ghost_update(ctx->s, ctx->N, ctx->ngc_cap, xr_mode(ctx), ctx->cnt, ctx->border,
        ctx->pbc, ctx->jnat, ctx->g, ctx->cx, ctx->anchor, ctx->xr);
}

static void enq_prune(MdbCp* ctx)
{
    launch_prune(ctx->s, ctx->M, ctx->N, ctx->ncl_cap, ctx->cnt, ctx->cx, ctx->g.cutneighsq,
        ctx->maxneighs, lks(ctx), lcs(ctx), ctx->list, ctx->numneigh, ctx->nmasked);
    if (pair_path(ctx)) mark_derive(ctx); // the rows moved: codes index list entries
}

// T and P from the atom arrays (as computeThermo reads them), KE of the
// cluster state, PE from the last energy evaluation
static void enq_thermo(MdbCp* ctx, int slot, bool with_pe)
{
    cudaStream_t s = ctx->s;
    double* r      = ctx->red + 4 * slot;
    double* pk     = ctx->partials + ctx->npart;
    launch_ke_atoms(s, ctx->nlocal, ctx->av, ctx->p.mass, pk);
    launch_reduce_partials(s, ke_blocks(ctx->nlocal), pk, r + 0);
    launch_ke_slots(s, ctx->M, ctx->ncl_cap, ctx->cnt, ctx->cx, ctx->cv, ctx->p.mass, pk);
    launch_reduce_partials(s, ke_blocks(ctx->ncl_cap * ctx->M), pk, r + 2);
    if (with_pe) launch_reduce_partials(s, ctx->energy_blocks, ctx->partials, r + 1);
    else cudaMemsetAsync(r + 1, 0, sizeof(double), s);
}

static void finish_thermo(MdbCp* ctx, const double* r, int step, MdbThermo* out)
{
    out->step        = step;
    double T         = r[0] * ctx->t_scale;
    out->temperature = T;
    out->pressure    = (T * ctx->dof_boltz) * ctx->p_scale;
    out->ke          = 0.5 * r[2];
    out->pe          = r[1];
    out->etotal      = out->ke + out->pe;
}

// ---------------------------------------------------------------------------
// hooks
extern "C" int mdb_cp_build_clusters(MdbCp* ctx)
{
    NEED_ATOMS();
    long long m = mark();
    clear_build_counters(ctx);
    enq_clusters(ctx);
    account(ctx, m);
    int r = check_build(ctx, CHK_CLUSTERS);
    if (r < 0) return -r;
    ctx->have_clusters = true;
    ctx->have_ghosts = ctx->have_list = false;
    ctx->force_current = false;
    return MDB_OK;
}

extern "C" int mdb_cp_define_jclusters(MdbCp* ctx)
{
    NEED_ATOMS();
    if (!ctx->have_clusters) return fail(ctx, MDB_ERR_STATE, "buildClusters not run");
    return MDB_OK;
}

extern "C" int mdb_cp_setup_pbc(MdbCp* ctx)
{
    NEED_ATOMS();
    if (!ctx->have_clusters) return fail(ctx, MDB_ERR_STATE, "buildClusters not run");
    for (int attempt = 0; attempt < 4; attempt++) {
        long long m = mark();
        enq_setup_pbc(ctx);
        account(ctx, m);
        int r = check_build(ctx, CHK_GHOSTS);
        if (r < 0) return -r;
        if (r == 0) {
            ctx->have_ghosts = true;
            return MDB_OK;
        }
        // ghost capacity grew: the slot arrays are new, rebuild the clusters
        m = mark();
        enq_clusters(ctx);
        account(ctx, m);
    }
    return fail(ctx, MDB_ERR_OVERFLOW, "setupPbc did not converge");
}

extern "C" int mdb_cp_update_pbc(MdbCp* ctx)
{
    NEED_ATOMS();
    if (!ctx->have_ghosts) return fail(ctx, MDB_ERR_STATE, "setupPbc not run");
    long long m = mark();
    enq_ghost_update(ctx);
    account(ctx, m);
    return MDB_OK;
}

extern "C" int mdb_cp_bin_jclusters(MdbCp* ctx)
{
    NEED_ATOMS();
    if (!ctx->have_ghosts) return fail(ctx, MDB_ERR_STATE, "setupPbc not run");
    long long m = mark();
    enq_bin_j(ctx);
    account(ctx, m);
    return MDB_OK;
}

extern "C" int mdb_cp_build_neighbor(MdbCp* ctx)
{
    NEED_ATOMS();
    if (!ctx->have_ghosts) return fail(ctx, MDB_ERR_STATE, "setupPbc not run");
    for (int attempt = 0; attempt < 8; attempt++) {
        long long m = mark();
        clear_build_counters(ctx);
        enq_list(ctx);
        account(ctx, m);
        int r = check_build(ctx, CHK_LIST);
        if (r < 0) return -r;
        if (r == 0) {
            ctx->have_list = true;
            return ensure_pairs(ctx);
        }
        if (!ctx->have_ghosts) return do_build(ctx); // capacity change dropped the clusters
    }
    return fail(ctx, MDB_ERR_OVERFLOW, "buildNeighbor did not converge");
}

extern "C" int mdb_cp_prune_neighbor(MdbCp* ctx)
{
    NEED_ATOMS();
    if (!ctx->have_list) return fail(ctx, MDB_ERR_STATE, "buildNeighbor not run");
    long long m = mark();
    enq_prune(ctx);
    account(ctx, m);
    return MDB_OK;
}

extern "C" int mdb_cp_update_single_atoms(MdbCp* ctx)
{
    NEED_ATOMS();
    if (!ctx->have_clusters) return fail(ctx, MDB_ERR_STATE, "buildClusters not run");
    long long m = mark();
    enq_gather(ctx, 0);
    account(ctx, m);
    return MDB_OK;
}

__global__ void k_wrap_atoms(int n, double4* ax, double xprd, double yprd, double zprd)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 p = ax[i];
    if (p.x < 0.0) p.x += xprd;
    else if (p.x >= xprd) p.x -= xprd;
    if (p.y < 0.0) p.y += yprd;
    else if (p.y >= yprd) p.y -= yprd;
    if (p.z < 0.0) p.z += zprd;
    else if (p.z >= zprd) p.z -= zprd;
    ax[i] = p;
}

extern "C" int mdb_cp_update_atoms_pbc(MdbCp* ctx)
{
    NEED_ATOMS();
    k_wrap_atoms<<<mdb_blocks(ctx->nlocal, MDB_NTHREADS), MDB_NTHREADS, 0, ctx->s>>>(ctx->nlocal,
        ctx->ax, ctx->p.xprd, ctx->p.yprd, ctx->p.zprd);
    ctx->launches++;
    CK(cudaGetLastError());
    return MDB_OK;
}

static int compute_force(MdbCp* ctx, bool energy)
{
    NEED_ATOMS();
    if (!ctx->have_list) return fail(ctx, MDB_ERR_STATE, "buildNeighbor not run");
    long long m = mark();
    enq_force(ctx, energy);
    account(ctx, m);
    CK(cudaGetLastError());
    ctx->energy_valid  = energy;
    ctx->force_current = true;
    return MDB_OK;
}

extern "C" int mdb_cp_compute_force(MdbCp* ctx) { return compute_force(ctx, false); }
extern "C" int mdb_cp_compute_force_energy(MdbCp* ctx) { return compute_force(ctx, true); }

extern "C" int mdb_cp_initial_integrate(MdbCp* ctx)
{
    NEED_ATOMS();
    if (!ctx->have_clusters) return fail(ctx, MDB_ERR_STATE, "buildClusters not run");
    long long m = mark();
    enq_initial(ctx);
    account(ctx, m);
    ctx->force_current = false;
    return MDB_OK;
}

extern "C" int mdb_cp_final_integrate(MdbCp* ctx)
{
    NEED_ATOMS();
    if (!ctx->have_clusters) return fail(ctx, MDB_ERR_STATE, "buildClusters not run");
    long long m = mark();
    enq_final(ctx);
    account(ctx, m);
    return MDB_OK;
}

extern "C" int mdb_cp_time_force(MdbCp* ctx, int reps, double* seconds)
{
    NEED_ATOMS();
    if (!ctx->have_list) return fail(ctx, MDB_ERR_STATE, "mdb_cp_setup not run");
    if (reps < 1 || !seconds) return MDB_ERR_ARG;
    CK(cudaSetDevice(ctx->dev));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    cudaError_t e = cudaEventCreate(&e1);
    if (e != cudaSuccess) {
        cudaEventDestroy(e0);
        return fail(ctx, MDB_ERR_CUDA, "event", e);
    }
    long long m = mark();
    // the pair-list path: the codes once, then the force kernel on them
    // alone (half lists accumulate: the forces are restored below)
    const bool pq = pair_path(ctx);
    if (pq) enq_derive(ctx, 1);
    for (int k = 0; k < 2; k++) pq ? (void)enq_force_pairs(ctx, false) : enq_force(ctx, false);
    cudaEventRecord(e0, ctx->s);
    for (int k = 0; k < reps; k++) pq ? (void)enq_force_pairs(ctx, false) : enq_force(ctx, false);
    cudaEventRecord(e1, ctx->s);
    if (pq) enq_force(ctx, false); // the state's forces again (half lists accumulated)
    account(ctx, m);
    e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return fail(ctx, MDB_ERR_CUDA, "force timing", e);
    *seconds = ms * 1e-3 / reps;
    return MDB_OK;
}

extern "C" int mdb_cp_thermo(MdbCp* ctx, MdbThermo* out)
{
    NEED_ATOMS();
    if (!out) return MDB_ERR_ARG;
    long long m = mark();
    if (!ctx->energy_valid && ctx->force_current && ctx->have_list) {
        // the energy of the current state: one force evaluation with it (the
        // same forces; half lists sum them in another atomic order)
        enq_force(ctx, true);
        ctx->energy_valid = true;
    }
    bool pe     = ctx->energy_valid && ctx->have_clusters;
    if (ctx->have_clusters) {
        enq_thermo(ctx, 0, pe);
    } else {
        double* pk = ctx->partials + ctx->npart;
        launch_ke_atoms(ctx->s, ctx->nlocal, ctx->av, ctx->p.mass, pk);
        launch_reduce_partials(ctx->s, ke_blocks(ctx->nlocal), pk, ctx->red);
        cudaMemsetAsync(ctx->red + 1, 0, 3 * sizeof(double), ctx->s);
    }
    account(ctx, m);
    CK(cudaMemcpyAsync(ctx->h_red, ctx->red, 4 * sizeof(double), cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    finish_thermo(ctx, ctx->h_red, -1, out);
    if (!pe) out->pe = out->etotal = NAN;
    return MDB_OK;
}

extern "C" int mdb_cp_setup(MdbCp* ctx)
{
    NEED_ATOMS();
    CK(cudaSetDevice(ctx->dev));
    int rc = do_build(ctx);
    if (rc) return rc;
    // the energy is evaluated when mdb_cp_thermo asks for it
    return compute_force(ctx, false);
}

// A plain step whose predecessor left its final integration pending:
// finalIntegrate(n-1) + initialIntegrate(n), updatePbc, force.
static void enq_plain_step(MdbCp* ctx)
{
    enq_final_initial(ctx);
    enq_ghost_update(ctx);
    enq_force(ctx, false);
}

static int capture_plain(MdbCp* ctx)
{
    cudaGraph_t graph;
    long long m0 = mark();
    CK(cudaStreamBeginCapture(ctx->s, cudaStreamCaptureModeThreadLocal));
    enq_plain_step(ctx);
    cudaError_t e = cudaStreamEndCapture(ctx->s, &graph);
    ctx->g_plain.kernels = mdb::g_launches - m0;
    mdb::g_launches      = m0;
    if (e != cudaSuccess) return fail(ctx, MDB_ERR_CUDA, "stream capture", e);
    e = cudaGraphInstantiate(&ctx->g_plain.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(ctx, MDB_ERR_CUDA, "graph instantiate", e);
    return MDB_OK;
}

// ---- displacement check decided on the device --------------------------------
// dstate = {stopped, steps run, rebuilds}: a step's graph opens with a gate
// (the step runs unless a rebuild earlier in the call overflowed a buffer),
// rebuilds when the integrator raised the displacement flag, and runs the
// force unless that rebuild overflowed.
__global__ void k_chk_gate(cudaGraphConditionalHandle h, int* st)
{
    const bool go = st[0] == 0;
    if (go) st[1]++;
    cudaGraphSetConditional(h, go ? 1u : 0u);
}

__global__ void k_chk_reb(cudaGraphConditionalHandle h, const int* dflag, int* st)
{
    const bool reb = *dflag != 0;
    if (reb) st[2]++;
    cudaGraphSetConditional(h, reb ? 1u : 0u);
}

// what eval_build would grow (or reject) stops the call
__global__ void k_chk_built(const int* cnt, int ngc_cap, int maxneighs, int* st)
{
    if (cnt[CP_BADBIN] > 0 || cnt[CP_NGC_TOTAL] > ngc_cap || cnt[CP_MAXNEED] >= maxneighs)
        st[0] = 1;
}

__global__ void k_chk_force(cudaGraphConditionalHandle h, const int* st)
{
    cudaGraphSetConditional(h, st[0] == 0 ? 1u : 0u);
}

// An "if" node (size 2: if / else) on handle h after the current capture
// point of stream s; its body graphs in bodies[0..size).
static cudaError_t cap_conditional(cudaStream_t s, cudaGraphConditionalHandle h, unsigned size,
    cudaGraph_t* bodies)
{
    cudaStreamCaptureStatus st;
    cudaGraph_t g                = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd                    = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd);
    if (e != cudaSuccess) return e;
    cudaGraphNodeParams p = {};
    p.type                = cudaGraphNodeTypeConditional;
    p.conditional.handle  = h;
    p.conditional.type    = cudaGraphCondTypeIf;
    p.conditional.size    = size;
    cudaGraphNode_t node;
    if ((e = cudaGraphAddNode(&node, g, deps, nd, &p)) != cudaSuccess) return e;
    for (unsigned k = 0; k < size; k++) bodies[k] = p.conditional.phGraph_out[k];
    return cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies);
}

static cudaError_t cap_handle(cudaStream_t s, cudaGraphConditionalHandle* h)
{
    cudaStreamCaptureStatus st;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamGetCaptureInfo(s, &st, nullptr, &g, nullptr, nullptr);
    if (e != cudaSuccess) return e;
    return cudaGraphConditionalHandleCreate(h, g, 0, 0);
}

// One checked step as a graph: finalIntegrate(n-1) + initialIntegrate(n) with
// the displacement test, then either updateAtoms + the whole rebuild (an atom
// moved past the limit) or updatePbc, then the force; all of it only while no
// rebuild of this call has overflowed a buffer. The bodies are captured on two
// further streams (enq_* enqueue on ctx->s, which points at the capturing one).
static int capture_chk(MdbCp* ctx)
{
    cudaError_t e = cudaSuccess;
    for (cudaStream_t& c : ctx->s_cap)
        if (!c && (e = cudaStreamCreateWithFlags(&c, cudaStreamNonBlocking)) != cudaSuccess)
            return fail(ctx, MDB_ERR_CUDA, "capture stream", e);
    const cudaStream_t s0 = ctx->s, s1 = ctx->s_cap[0], s2 = ctx->s_cap[1];
    const cudaStreamCaptureMode mode = cudaStreamCaptureModeThreadLocal;
    cudaGraphConditionalHandle h_step = 0, h_reb = 0, h_force = 0;
    cudaGraph_t step[1] = {nullptr}, reb[2] = {nullptr, nullptr}, frc[1] = {nullptr};
    cudaGraph_t graph = nullptr;
    const long long m0 = mark();
    long long* k = ctx->chk_k;
    bool cap1 = false, cap2 = false;
    auto body2 = [&](cudaGraph_t g, int what) -> cudaError_t {
        // one body of the inner conditionals, captured on s2
        cudaError_t r = cudaStreamBeginCaptureToGraph(s2, g, nullptr, nullptr, 0, mode);
        if (r != cudaSuccess) return r;
        cap2 = true;
        ctx->s = s2;
        long long m = mark();
        if (what == 0) {
            enq_gather(ctx, 1);
            enq_build(ctx);
            k_chk_built<<<1, 1, 0, s2>>>(ctx->cnt, ctx->ngc_cap, ctx->maxneighs, ctx->dstate);
            cudaMemcpyAsync(ctx->xbuild, ctx->cx, sizeof(double4) * ctx->ncl_cap * ctx->M,
                cudaMemcpyDeviceToDevice, s2);
            cudaMemsetAsync(ctx->dflag, 0, sizeof(int), s2);
            k[2] = mark() - m + 1;
        } else if (what == 1) {
            enq_ghost_update(ctx);
            k[1] = mark() - m;
        } else {
            enq_force(ctx, false);
            k[3] = mark() - m;
        }
        ctx->s = s1;
        r = cudaGetLastError();
        cudaGraph_t out = nullptr;
        cudaError_t r2 = cudaStreamEndCapture(s2, &out);
        cap2 = false;
        return r != cudaSuccess ? r : r2;
    };
    e = cudaStreamBeginCapture(s0, mode);
    if (e == cudaSuccess) e = cap_handle(s0, &h_step);
    if (e == cudaSuccess) {
        k_chk_gate<<<1, 1, 0, s0>>>(h_step, ctx->dstate);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cap_conditional(s0, h_step, 1, step);
    if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(s1, step[0], nullptr, nullptr, 0, mode);
    if (e == cudaSuccess) {
        cap1   = true;
        ctx->s = s1;
        long long m = mark();
        enq_final_initial(ctx);
        k[0] = mark() - m + 2;
        e = cap_handle(s1, &h_reb);
    }
    if (e == cudaSuccess) {
        k_chk_reb<<<1, 1, 0, s1>>>(h_reb, ctx->dflag, ctx->dstate);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cap_conditional(s1, h_reb, 2, reb);
    if (e == cudaSuccess) e = body2(reb[0], 0);
    if (e == cudaSuccess) e = body2(reb[1], 1);
    if (e == cudaSuccess) e = cap_handle(s1, &h_force);
    if (e == cudaSuccess) {
        k_chk_force<<<1, 1, 0, s1>>>(h_force, ctx->dstate);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cap_conditional(s1, h_force, 1, frc);
    if (e == cudaSuccess) e = body2(frc[0], 2);
    ctx->s = s0;
    mdb::g_launches = m0;
    if (cap2) {
        cudaGraph_t g2 = nullptr;
        cudaStreamEndCapture(s2, &g2);
    }
    if (cap1) {
        cudaGraph_t g1       = nullptr;
        const cudaError_t e1 = cudaStreamEndCapture(s1, &g1);
        if (e == cudaSuccess) e = e1;
    }
    const cudaError_t e0 = cudaStreamEndCapture(s0, &graph);
    if (e == cudaSuccess) e = e0;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&ctx->g_chk.exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, MDB_ERR_CUDA, "checked step graph", e);
    }
    ctx->g_chk.kernels = 1;
    return MDB_OK;
}

// The device's record of the graph steps launched since the last call (their
// step indices in `launched`): counts their rebuilds and kernels and, when a
// rebuild overflowed a buffer, grows it, replays that build (from the atom
// arrays its updateAtoms wrote: the build is idempotent) and evaluates that
// step's force. *resume = that step (the later ones did nothing), else -1.
static int chk_resolve(MdbCp* ctx, std::vector<int>& launched, int* resume)
{
    *resume = -1;
    if (launched.empty()) return MDB_OK;
    CK(cudaMemcpyAsync(ctx->h_dstate, ctx->dstate, 3 * sizeof(int), cudaMemcpyDeviceToHost,
        ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    const int stopped = ctx->h_dstate[0], ran = ctx->h_dstate[1], reb = ctx->h_dstate[2];
    CK(cudaMemsetAsync(ctx->dstate, 0, 3 * sizeof(int), ctx->s));
    const long long* k = ctx->chk_k;
    ctx->rebuilds_check += reb;
    ctx->chk_steps += ran;
    ctx->chk_replays += stopped ? 1 : 0;
    ctx->launches += (long long)launched.size() + ran * k[0] + (ran - reb) * k[1] + reb * k[2] +
                     (ran - stopped) * k[3];
    if (stopped) {
        if (ran < 1 || ran > (int)launched.size())
            return fail(ctx, MDB_ERR_CUDA, "checked steps: inconsistent device record");
        const int n = launched[ran - 1];
        CK(cudaMemcpyAsync(ctx->h_cnt, ctx->cnt, CP_SLOTS * sizeof(int), cudaMemcpyDeviceToHost,
            ctx->s));
        CK(cudaStreamSynchronize(ctx->s));
        const int r = eval_build(ctx, CHK_ALL);
        if (r < 0) return -r;
        int rc = do_build(ctx);
        if (rc) return rc;
        long long m = mark();
        enq_force(ctx, false);
        account(ctx, m);
        *resume = n;
    }
    launched.clear();
    return MDB_OK;
}

// The timestep loop with the displacement check: each step's initial
// integration also tests every atom's displacement since the last build, and
// the step rebuilds when an atom moved farther than disp_max, besides the
// reference's fixed schedule. Lists are then complete at every step for any
// motion. The decision is taken on the device (a conditional graph per step,
// no host synchronisation) except at scheduled rebuilds, pruning, thermo
// samples, a call's first and last step and with the pair-list path, where
// (as with "check_on_host") the host reads the flag after the integration.
static int run_checked(MdbCp* ctx, int first_step, int nsteps, MdbThermo* samples,
    int max_samples, int* nsamples)
{
    int nslot = 0;
    std::vector<int> slot_step, launched;
    const int last       = first_step + nsteps - 1;
    bool pending_final   = false;
    const bool on_device = !ctx->check_host && !pair_path(ctx);
    if (on_device && !ctx->dstate) {
        CK(dalloc(&ctx->dstate, 3));
        CK(cudaMallocHost((void**)&ctx->h_dstate, 3 * sizeof(int)));
        CK(cudaMemsetAsync(ctx->dstate, 0, 3 * sizeof(int), ctx->s));
    }
    for (int n = first_step; n <= last; n++) {
        const bool sched  = (n + 1) % ctx->p.reneigh_every == 0;
        const bool prune  = !sched && (n + 1) % ctx->prune_every == 0;
        const bool sample = max_samples > 0 && (n + 1) % ctx->p.nstat == 0;
        if (on_device && pending_final && ctx->snap_valid && !sched && !prune && !sample &&
            n != last) {
            if (!ctx->g_chk.exec) {
                int rc = capture_chk(ctx);
                if (rc) return rc;
            }
            CK(cudaGraphLaunch(ctx->g_chk.exec, ctx->s));
            launched.push_back(n);
            continue; // the step leaves its final integration pending
        }
        if (!launched.empty()) {
            int resume = -1;
            int rc     = chk_resolve(ctx, launched, &resume);
            if (rc) return rc;
            if (resume >= 0) {
                n = resume; // steps after it did nothing: run them again
                continue;
            }
        }
        const bool had = ctx->snap_valid;
        long long m    = mark();
        if (pending_final) enq_final_initial(ctx);
        else enq_initial(ctx);
        pending_final = false;
        account(ctx, m);
        bool reneigh = sched || !had;
        if (!reneigh) {
            CK(cudaMemcpyAsync(ctx->h_dflag, ctx->dflag, sizeof(int), cudaMemcpyDeviceToHost,
                ctx->s));
            CK(cudaStreamSynchronize(ctx->s));
            reneigh = *ctx->h_dflag != 0;
            if (reneigh) ctx->rebuilds_check++;
        } else if (sched) {
            ctx->rebuilds_sched++;
        }
        if (reneigh) {
            m = mark();
            enq_gather(ctx, 1);
            account(ctx, m);
            int rc = do_build(ctx);
            if (rc) return rc;
        } else {
            m = mark();
            if (prune) enq_prune(ctx);
            enq_ghost_update(ctx);
            account(ctx, m);
        }
        m = mark();
        enq_force(ctx, sample);
        if (sample || n == last) enq_final(ctx);
        else pending_final = true;
        if (sample && nslot < RED_SLOTS && nslot < max_samples) {
            enq_thermo(ctx, nslot, true);
            slot_step.push_back(n + 1);
            nslot++;
        }
        account(ctx, m);
    }
    ctx->energy_valid = nsteps > 0 && max_samples > 0 && ((last + 1) % ctx->p.nstat == 0);
    if (nsteps > 0) ctx->force_current = true;
    CK(cudaGetLastError());
    if (nslot > 0)
        CK(cudaMemcpyAsync(ctx->h_red, ctx->red, 4 * sizeof(double) * nslot,
            cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    for (int k = 0; k < nslot; k++)
        finish_thermo(ctx, ctx->h_red + 4 * k, slot_step[k], &samples[k]);
    if (nsamples) *nsamples = nslot;
    return MDB_OK;
}

extern "C" int mdb_cp_set_rebuild_check(MdbCp* ctx, double max_displacement)
{
    if (!ctx || !(max_displacement >= 0.0)) return MDB_ERR_ARG;
    CK(cudaSetDevice(ctx->dev));
    CK(cudaStreamSynchronize(ctx->s));
    drop_graph(ctx);
    ctx->disp_max   = max_displacement;
    ctx->snap_valid = false; // the next step rebuilds (and snapshots) first
    return MDB_OK;
}

extern "C" int mdb_cp_get_check_stats(MdbCp* ctx, long long* graph_steps, long long* replays)
{
    if (!ctx) return MDB_ERR_ARG;
    if (graph_steps) *graph_steps = ctx->chk_steps;
    if (replays) *replays = ctx->chk_replays;
    return MDB_OK;
}

extern "C" int mdb_cp_get_rebuilds(MdbCp* ctx, long long* scheduled, long long* checked)
{
    if (!ctx) return MDB_ERR_ARG;
    if (scheduled) *scheduled = ctx->rebuilds_sched;
    if (checked) *checked = ctx->rebuilds_check;
    return MDB_OK;
}

extern "C" int mdb_cp_run(MdbCp* ctx, int first_step, int nsteps, MdbThermo* samples,
    int max_samples, int* nsamples)
{
    NEED_ATOMS();
    if (!ctx->have_list) return fail(ctx, MDB_ERR_STATE, "mdb_cp_setup not run");
    if (nsteps < 0 || (max_samples > 0 && !samples)) return MDB_ERR_ARG;
    CK(cudaSetDevice(ctx->dev));
    if (ctx->disp_max > 0.0) {
        if (nsamples) *nsamples = 0;
        return run_checked(ctx, first_step, nsteps, samples, max_samples, nsamples);
    }
    if (nsamples) *nsamples = 0;
    int nslot = 0;
    std::vector<int> slot_step;
    const int last     = first_step + nsteps - 1;
    bool pending_final = false;
    for (int n = first_step; n <= last; n++) {
        const bool reneigh = (n + 1) % ctx->p.reneigh_every == 0;
        const bool prune   = !reneigh && (n + 1) % ctx->prune_every == 0;
        const bool sample  = max_samples > 0 && (n + 1) % ctx->p.nstat == 0;
        if (!reneigh && !prune && !sample && pending_final && n != last) {
            if (!ctx->g_plain.exec) {
                int rc = capture_plain(ctx);
                if (rc) return rc;
            }
            CK(cudaGraphLaunch(ctx->g_plain.exec, ctx->s));
            ctx->launches += ctx->g_plain.kernels;
            continue;
        }
        long long m = mark();
        if (pending_final) enq_final_initial(ctx);
        else enq_initial(ctx);
        pending_final = false;
        account(ctx, m);
        if (reneigh) {
            // updateAtoms (updateSingleAtoms + updateAtomsPbc), then reneighbour
            m = mark();
            enq_gather(ctx, 1);
            account(ctx, m);
            int rc = do_build(ctx);
            if (rc) return rc;
        } else {
            m = mark();
            if (prune) enq_prune(ctx);
            enq_ghost_update(ctx);
            account(ctx, m);
        }
        m = mark();
        enq_force(ctx, sample);
        if (sample || n == last) enq_final(ctx);
        else pending_final = true;
        if (sample && nslot < RED_SLOTS && nslot < max_samples) {
            enq_thermo(ctx, nslot, true);
            slot_step.push_back(n + 1);
            nslot++;
        }
        account(ctx, m);
    }
    if (pending_final) {
        long long m = mark();
        enq_final(ctx);
        account(ctx, m);
    }
    ctx->energy_valid = nsteps > 0 && max_samples > 0 && ((last + 1) % ctx->p.nstat == 0);
    if (nsteps > 0) ctx->force_current = true;
    CK(cudaGetLastError());
    if (nslot > 0)
        CK(cudaMemcpyAsync(ctx->h_red, ctx->red, 4 * sizeof(double) * nslot,
            cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    for (int k = 0; k < nslot; k++)
        finish_thermo(ctx, ctx->h_red + 4 * k, slot_step[k], &samples[k]);
    if (nsamples) *nsamples = nslot;
    return MDB_OK;
}

// ---------------------------------------------------------------------------
// introspection
extern "C" int mdb_cp_get_counts(MdbCp* ctx, int* c)
{
    NEED_ATOMS();
    if (!c) return MDB_ERR_ARG;
    CK(cudaMemcpyAsync(ctx->h_cnt, ctx->cnt, CP_SLOTS * sizeof(int), cudaMemcpyDeviceToHost,
        ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    const int* h = ctx->h_cnt;
    c[0]         = ctx->nlocal;
    c[1]         = ctx->p.natoms;
    c[2]         = h[CP_NCL];
    c[3]         = h[CP_NCJ];
    c[4]         = h[CP_NGC];
    c[5]         = h[CP_NGHOST_ATOMS];
    c[6]         = h[CP_NCJ] + h[CP_NGC];
    c[7]         = ctx->maxneighs;
    return MDB_OK;
}

template <typename T>
static int copy_back(MdbCp* ctx, std::vector<T>& h, const T* d, size_t n)
{
    h.resize(n);
    if (n == 0) return MDB_OK;
    CK(cudaMemcpyAsync(h.data(), d, sizeof(T) * n, cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    return MDB_OK;
}

extern "C" int mdb_cp_get_slots(MdbCp* ctx, double* x, double* v, double* f, int* type, int nslots)
{
    NEED_ATOMS();
    if (nslots < 0 || nslots > ctx->slot_cap) return MDB_ERR_ARG;
    int c[8];
    int rc = mdb_cp_get_counts(ctx, c);
    if (rc) return rc;
    const int nloc = c[2] * ctx->M;
    std::vector<double4> hx, hv, hf;
    std::vector<float4> hf32;
    if ((rc = copy_back(ctx, hx, ctx->cx, nslots))) return rc;
    if (v && (rc = copy_back(ctx, hv, ctx->cv, std::min(nslots, nloc)))) return rc;
    if (f) {
        if (f32_slots(ctx)) rc = copy_back(ctx, hf32, ctx->cf32, std::min(nslots, nloc));
        else rc = copy_back(ctx, hf, ctx->cf, std::min(nslots, nloc));
        if (rc) return rc;
    }
    for (int s = 0; s < nslots; s++) {
        if (x) {
            x[3 * s] = hx[s].x, x[3 * s + 1] = hx[s].y, x[3 * s + 2] = hx[s].z;
        }
        if (type) {
            long long t;
            memcpy(&t, &hx[s].w, sizeof t);
            type[s] = (int)t;
        }
        if (s < nloc) {
            if (v) v[3 * s] = hv[s].x, v[3 * s + 1] = hv[s].y, v[3 * s + 2] = hv[s].z;
            if (f && f32_slots(ctx))
                f[3 * s] = hf32[s].x, f[3 * s + 1] = hf32[s].y, f[3 * s + 2] = hf32[s].z;
            else if (f)
                f[3 * s] = hf[s].x, f[3 * s + 1] = hf[s].y, f[3 * s + 2] = hf[s].z;
        }
    }
    return MDB_OK;
}

static void bb_out(const double4& mn, const double4& mx, double* b)
{
    b[0] = mn.x, b[1] = mx.x, b[2] = mn.y, b[3] = mx.y, b[4] = mn.z, b[5] = mx.z;
}

extern "C" int mdb_cp_get_iclusters(MdbCp* ctx, int* natoms, int* bin, double* bb)
{
    NEED_ATOMS();
    int c[8], rc = mdb_cp_get_counts(ctx, c);
    if (rc) return rc;
    const int n = c[2];
    std::vector<int> hn, hb;
    std::vector<double4> h0, h1;
    if ((rc = copy_back(ctx, hn, ctx->inat, n)) || (rc = copy_back(ctx, hb, ctx->cbin, n)) ||
        (rc = copy_back(ctx, h0, ctx->ibbmin, n)) || (rc = copy_back(ctx, h1, ctx->ibbmax, n)))
        return rc;
    for (int i = 0; i < n; i++) {
        if (natoms) natoms[i] = hn[i];
        if (bin) bin[i] = hb[i];
        if (bb) bb_out(h0[i], h1[i], bb + 6 * i);
    }
    return MDB_OK;
}

extern "C" int mdb_cp_get_jclusters(MdbCp* ctx, int* natoms, double* bb, int count)
{
    NEED_ATOMS();
    if (count < 0 || count > ctx->ncj_cap + ctx->ngc_cap) return MDB_ERR_ARG;
    std::vector<int> hn;
    std::vector<double4> h0, h1;
    int rc;
    if ((rc = copy_back(ctx, hn, ctx->jnat, count)) ||
        (rc = copy_back(ctx, h0, ctx->jbbmin, count)) ||
        (rc = copy_back(ctx, h1, ctx->jbbmax, count)))
        return rc;
    for (int i = 0; i < count; i++) {
        if (natoms) natoms[i] = hn[i];
        if (bb) bb_out(h0[i], h1[i], bb + 6 * i);
    }
    return MDB_OK;
}

extern "C" int mdb_cp_get_ghosts(MdbCp* ctx, int* border_map, int* pbc_xyz)
{
    NEED_ATOMS();
    int c[8], rc = mdb_cp_get_counts(ctx, c);
    if (rc) return rc;
    std::vector<int> hb, hp;
    if ((rc = copy_back(ctx, hb, ctx->border, c[4])) || (rc = copy_back(ctx, hp, ctx->pbc, c[4])))
        return rc;
    for (int g = 0; g < c[4]; g++) {
        if (border_map) border_map[g] = hb[g];
        if (pbc_xyz) {
            pbc_xyz[3 * g]     = (hp[g] & 3) - 1;
            pbc_xyz[3 * g + 1] = ((hp[g] >> 2) & 3) - 1;
            pbc_xyz[3 * g + 2] = ((hp[g] >> 4) & 3) - 1;
        }
    }
    return MDB_OK;
}

extern "C" int mdb_cp_get_neighbor_list(MdbCp* ctx, int* numneigh, int* nmasked, int* neighbors,
    int ld)
{
    NEED_ATOMS();
    if (!ctx->have_list) return fail(ctx, MDB_ERR_STATE, "buildNeighbor not run");
    int c[8], rc = mdb_cp_get_counts(ctx, c);
    if (rc) return rc;
    const int n = c[2];
    std::vector<int> hn, hm, hl;
    if ((rc = copy_back(ctx, hn, ctx->numneigh, n)) || (rc = copy_back(ctx, hm, ctx->nmasked, n)))
        return rc;
    if (neighbors && (rc = copy_back(ctx, hl, ctx->list, (size_t)ctx->maxneighs * ctx->ld)))
        return rc;
    for (int i = 0; i < n; i++) {
        if (numneigh) numneigh[i] = hn[i];
        if (nmasked) nmasked[i] = hm[i];
        if (neighbors)
            for (int k = 0; k < hn[i] && k < ld; k++)
                neighbors[(size_t)i * ld + k] =
                    hl[(size_t)k * lks(ctx) + (size_t)i * lcs(ctx)];
    }
    return MDB_OK;
}

extern "C" int mdb_cp_get_columns(MdbCp* ctx, int* start, int* list, int cap)
{
    NEED_ATOMS();
    const int mb = ctx->g.mbins;
    std::vector<int> hs, hl;
    int rc;
    if ((rc = copy_back(ctx, hs, ctx->jcol_start, mb + 1))) return rc;
    const int n = hs[mb];
    if ((rc = copy_back(ctx, hl, ctx->jcol, n))) return rc;
    if (start) memcpy(start, hs.data(), sizeof(int) * (mb + 1));
    if (list)
        for (int i = 0; i < n && i < cap; i++)
            list[i] = hl[i];
    return n;
}

extern "C" int mdb_cp_get_geometry(MdbCp* ctx, int* ints, double* dbls, int* stencil,
    int max_stencil)
{
    if (!ctx) return MDB_ERR_ARG;
    const Geom& g = ctx->g;
    if (ints) {
        ints[0] = g.nbinx, ints[1] = g.nbiny, ints[2] = g.mbinx, ints[3] = g.mbiny;
        ints[4] = g.mbinxlo, ints[5] = g.mbinylo, ints[6] = g.nstencil;
    }
    if (dbls) dbls[0] = g.binsizex, dbls[1] = g.binsizey, dbls[2] = g.rbb_sq;
    if (stencil)
        for (int k = 0; k < g.nstencil && k < max_stencil; k++)
            stencil[k] = ctx->stencil[k];
    return MDB_OK;
}

// ---------------------------------------------------------------------------
// Ensemble of independent cluster-pair systems (replicas of uneven size and
// temperature). Every timestep of all members is one CUDA graph launch: the
// graph forks one branch per member (each branch is that member's own kernel
// sequence on its own buffers) and joins them, so the replicas' kernels run
// concurrently and fill the GPU even when single replicas are small. Rebuild
// steps launch the members' rebuilds as one graph, read all their overflow
// counters with one synchronisation, and redo only members that grew.
struct MdbCpEnsemble {
    std::vector<MdbCp*> m;
    std::vector<cudaEvent_t> join;
    cudaEvent_t fork = nullptr;
    cudaStream_t s   = nullptr;
    int dev          = 0;
    std::string err;
    long long launches = 0;
    // graphs of the step parts (see the EG_ kinds), valid for the members'
    // buffer generations in gen
    CpGraph g[16];
    std::vector<unsigned> gen;
    double* h_red = nullptr; // 4 doubles per member
    // batched launches (every member mixed): the integrator, the ghost update
    // and each force group run as one launch over all members; the members'
    // own streams only carry the rebuild and the thermo sums
    bool batched   = false;
    bool tables_ok = false;
    CpStepMember* d_step   = nullptr;
    CpForceMember* d_force = nullptr;
    int2* d_bmap           = nullptr;
    size_t bmap_cap        = 0;
    int nb_integ = 0, nb_ghost = 0;
    size_t off_integ = 0, off_ghost = 0;
    // batched rebuild: member table, block map per stage, counters of all members
    CpBuildMember* d_build = nullptr;
    int nb_stage[CB_COUNT]     = {};
    size_t off_stage[CB_COUNT] = {};
    int* d_cnt_all = nullptr;
    int* h_cnt_all = nullptr;
    // displacement check: one flag per member (set by the batched integrator)
    int* d_flags = nullptr;
    int* h_flags = nullptr;
    // the check decided on the device (default; "check_on_host" 1: the host
    // reads the flags every step): one graph per step whose conditional nodes
    // rebuild the members whose flag is up (the others update their ghosts);
    // dstate = {stopped, steps run, steps with a rebuild} as for a single
    // system
    bool check_host = false;
    int* dstate     = nullptr;
    int* h_dstate   = nullptr;
    int* d_rebcnt   = nullptr; // per member: checked rebuilds on the device
    int* h_rebcnt   = nullptr;
    cudaStream_t s_cap[2] = {nullptr, nullptr};
    long long chk_k[4]    = {0, 0, 0, 0}; // kernels: fixed part, ghost update, rebuild, force
    long long chk_steps = 0, chk_replays = 0;
    // per member {M, N, force group, i-clusters per warp, force threads}, for
    // the block maps that a rebuild inside the checked step graph refreshes
    int* d_mapinfo = nullptr;
    size_t* d_goff = nullptr; // per force group: its region of the maps and size
    int* d_gnb     = nullptr;
    struct Group { // members sharing cluster shape, list form, types and launch shape
        int N, half;
        Types ty;
        float cutsq;
        int nblocks;
        size_t off, off_dyn;
    };
    // block maps of the integrator, the ghost update and the force groups that
    // cover only the members' current clusters (the rest of each region is
    // unused entries); refreshed from the counters after every rebuild.
    // Energy evaluations use the capacity maps, so that every energy partial
    // of a member is written.
    size_t off_integ_dyn = 0, off_ghost_dyn = 0, dyn_begin = 0, dyn_end = 0;
    int2* h_dyn = nullptr;
    std::vector<int> gid;
    std::vector<Group> groups;
};

// step parts captured per ensemble: FI = final integration of the previous
// step fused with the initial one of this step, I = initial only
enum {
    EG_PLAIN_FI, // FI, ghost update, force
    EG_PLAIN_I,  // I, ghost update, force
    EG_FRONT_FI, // FI, ghost update (a sample step follows with EG_SAMPLE)
    EG_FRONT_I,  // I, ghost update
    EG_REB_FI,   // FI, updateSingleAtoms + wrap, rebuild, counters to the host
    EG_REB_I,    // I, the same
    EG_FORCE,    // force
    EG_SAMPLE,   // force with energy, final integration, thermo to the host
    EG_FINAL,    // the final integration left pending by the last step
    // displacement-checked steps (batched ensembles)
    EG_CK_FI,     // FI with the check, flags to the host
    EG_CK_I,      // I with the check, flags to the host
    EG_REB_NOINT, // the rebuild of EG_REB_* without the integration
    EG_GHOST,     // ghost update
    EG_CHK,       // a whole checked step, the rebuild decided on the device
    EG_COUNT
};
static_assert(EG_COUNT <= 16, "graph slots of MdbCpEnsemble");

static void ens_drop(MdbCpEnsemble* e)
{
    e->tables_ok = false;
    for (size_t k = 0; k < e->m.size(); k++) e->gen[k] = e->m[k]->gen;
    for (auto& g : e->g) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g.exec    = nullptr;
        g.kernels = 0;
    }
}

static int ens_fail(MdbCpEnsemble* e, int code, const char* what, cudaError_t ce = cudaSuccess)
{
    char buf[512];
    if (ce != cudaSuccess) snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(ce));
    else snprintf(buf, sizeof buf, "%s", what);
    e->err = buf;
    return code;
}

static void ens_body(MdbCp* c, int kind)
{
    switch (kind) {
    case EG_PLAIN_FI: enq_plain_step(c); break;
    case EG_PLAIN_I:
        enq_initial(c);
        enq_ghost_update(c);
        enq_force(c, false);
        break;
    case EG_FRONT_FI:
        enq_final_initial(c);
        enq_ghost_update(c);
        break;
    case EG_FRONT_I:
        enq_initial(c);
        enq_ghost_update(c);
        break;
    case EG_REB_FI:
    case EG_REB_I:
        if (kind == EG_REB_FI) enq_final_initial(c);
        else enq_initial(c);
        enq_gather(c, 1);
        enq_build(c);
        cudaMemcpyAsync(c->h_cnt, c->cnt, CP_SLOTS * sizeof(int), cudaMemcpyDeviceToHost, c->s);
        break;
    case EG_FORCE: enq_force(c, false); break;
    case EG_SAMPLE:
        enq_force(c, true);
        enq_final(c);
        enq_thermo(c, 0, true);
        cudaMemcpyAsync(c->h_red, c->red, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->s);
        break;
    case EG_FINAL: enq_final(c); break;
    }
}

static bool same_types(const Types& a, const Types& b)
{
    if (a.ntypes != b.ntypes || a.uniform != b.uniform || a.eps0 != b.eps0 ||
        a.sigma6_0 != b.sigma6_0 || a.force_block != b.force_block ||
        a.force_variant != b.force_variant || a.force_cpw != b.force_cpw ||
        a.force_jpl != b.force_jpl)
        return false;
    for (int t = 0; t < MDB_MAX_TYPES; t++)
        if (a.sqrt_eps_f[t] != b.sqrt_eps_f[t] || a.sigma3_f[t] != b.sigma3_f[t]) return false;
    return true;
}

// the dynamic block maps from the members' counters as the last build left
// them (host copies in h_cnt); stream-ordered before the next graph launch
static int ens_dyn_maps(MdbCpEnsemble* e)
{
    if (!e->batched || !e->tables_ok) return MDB_OK;
    int2* h  = e->h_dyn;
    size_t w = e->dyn_begin;
    const int n = (int)e->m.size();
    auto fill = [&](size_t cap, auto blocks_of) {
        const size_t end = w + cap;
        for (int k = 0; k < n; k++) {
            const int nb = blocks_of(e->m[k]);
            for (int b = 0; b < nb && w < end; b++) h[w++] = make_int2(k, b);
        }
        while (w < end) h[w++] = make_int2(-1, 0);
    };
    fill(e->nb_integ, [](const MdbCp* c) {
        return mdb_blocks((long long)c->h_cnt[CP_NCL] * c->M, MDB_NTHREADS);
    });
    fill(e->nb_ghost, [](const MdbCp* c) {
        return mdb_blocks((long long)c->h_cnt[CP_NGC] * c->N, MDB_NTHREADS);
    });
    for (size_t q = 0; q < e->groups.size(); q++) {
        const size_t end = w + e->groups[q].nblocks;
        for (int k = 0; k < n; k++) {
            if (e->gid[k] != (int)q) continue;
            const MdbCp* c = e->m[k];
            const int nb   = force_mixed_grid(c->h_cnt[CP_NCL], c->ty);
            for (int b = 0; b < nb && w < end; b++) h[w++] = make_int2(k, b);
        }
        while (w < end) h[w++] = make_int2(-1, 0);
    }
    cudaError_t ce = cudaMemcpyAsync(e->d_bmap + e->dyn_begin, h + e->dyn_begin,
        sizeof(int2) * (e->dyn_end - e->dyn_begin), cudaMemcpyHostToDevice, e->s);
    if (ce != cudaSuccess) return ens_fail(e, MDB_ERR_CUDA, "ensemble block maps", ce);
    return MDB_OK;
}

// member tables and block maps of the batched launches, from the members'
// current buffers and capacities
static int ens_tables(MdbCpEnsemble* e)
{
    if (e->tables_ok) return MDB_OK;
    // graphs launched earlier may still read the old tables
    cudaError_t ce = cudaStreamSynchronize(e->s);
    if (ce != cudaSuccess) return ens_fail(e, MDB_ERR_CUDA, "ensemble tables (sync)", ce);
    const int n = (int)e->m.size();
    std::vector<CpStepMember> st(n);
    std::vector<CpForceMember> fo(n);
    std::vector<int2> maps;
    auto add = [&](int k, int nb) {
        for (int b = 0; b < nb; b++) maps.push_back(make_int2(k, b));
    };
    for (int k = 0; k < n; k++) {
        const MdbCp* c = e->m[k];
        CpStepMember& a = st[k];
        a.cnt = c->cnt, a.cx = c->cx, a.cv = c->cv, a.cf = c->cf, a.cf32 = c->cf32;
        a.anchor = c->anchor, a.xr = c->xr, a.border = c->border, a.pbc = c->pbc;
        a.jnat = c->jnat, a.dtf = c->p.dtforce, a.dt = c->p.dt, a.xprd = c->g.xprd;
        a.yprd = c->g.yprd, a.zprd = c->g.zprd, a.M = c->M, a.N = c->N, a.mixed = xr_mode(c);
        a.zero_f = c->p.half_neigh;
        a.xb     = c->disp_max > 0.0 ? c->xbuild : nullptr;
        a.lim2   = c->disp_max * c->disp_max;
        a.flag   = nullptr; // set once the flags exist, below
        CpForceMember& f = fo[k];
        f.cnt = c->cnt, f.xr = c->xr, f.anchor = c->anchor, f.list = c->list;
        f.numneigh = c->numneigh, f.cf32 = c->cf32, f.epart = c->partials, f.cs = lcs(c);
        f.pad = 0;
    }
    std::vector<CpBuildMember> bt(n);
    for (int k = 0; k < n; k++) {
        const MdbCp* c   = e->m[k];
        CpBuildMember& b = bt[k];
        b.g = c->g, b.M = c->M, b.N = c->N, b.jfac = c->jfac, b.mixed = xr_mode(c);
        b.half = c->p.half_neigh, b.nlocal = c->nlocal, b.ncl_cap = c->ncl_cap;
        b.ncj_cap = c->ncj_cap, b.ngc_cap = c->ngc_cap, b.maxneighs = c->maxneighs;
        b.ks = lks(c), b.cs = lcs(c), b.cnt = c->cnt, b.zext = c->zext;
        b.ax = c->ax, b.av = c->av, b.cx = c->cx, b.cv = c->cv, b.cl_first = c->cl_first;
        b.atom_col = c->atom_col, b.col_count = c->col_count, b.col_start = c->col_start;
        b.col_fill = c->col_fill, b.col_atoms = c->col_atoms, b.col_sorted = c->col_sorted;
        b.gidx = c->gidx, b.gz = c->gz, b.ncl_col = c->ncl_col, b.cl_start = c->cl_start;
        b.inat = c->inat, b.cbin = c->cbin, b.ibbmin = c->ibbmin, b.ibbmax = c->ibbmax;
        b.jnat = c->jnat, b.jbbmin = c->jbbmin, b.jbbmax = c->jbbmax, b.anchor = c->anchor;
        b.xr = c->xr, b.gcount = c->gcount, b.gstart = c->gstart, b.border = c->border;
        b.pbc = c->pbc, b.gcolumn = c->gcolumn, b.gcol_count = c->gcol_count;
        b.jcol_n = c->jcol_n, b.jcol_start = c->jcol_start, b.gfill = c->gfill;
        b.gtmp = c->gtmp, b.jcol = c->jcol, b.jcbbmin = c->jcbbmin, b.jcbbmax = c->jcbbmax;
        b.jcbbf = c->jcbbf, b.cxf = c->cxf, b.slot_cap = c->slot_cap, b.ztab = c->ztab;
        b.stencil = c->stencil_d, b.list = c->list, b.numneigh = c->numneigh;
        b.nmasked = c->nmasked;
    }
    for (int st = 0; st < CB_COUNT; st++) {
        e->off_stage[st] = maps.size();
        for (int k = 0; k < n; k++) {
            int threads;
            add(k, cp_build_stage_blocks(st, bt[k], &threads));
        }
        e->nb_stage[st] = (int)(maps.size() - e->off_stage[st]);
    }
    e->off_integ = maps.size();
    for (int k = 0; k < n; k++)
        add(k, mdb_blocks((long long)e->m[k]->ncl_cap * e->m[k]->M, MDB_NTHREADS));
    e->nb_integ  = (int)(maps.size() - e->off_integ);
    e->off_ghost = maps.size();
    for (int k = 0; k < n; k++)
        add(k, mdb_blocks((long long)e->m[k]->ngc_cap * e->m[k]->N, MDB_NTHREADS));
    e->nb_ghost = (int)(maps.size() - e->off_ghost);
    e->groups.clear();
    std::vector<int> gid(n, -1);
    for (int k = 0; k < n; k++) {
        const MdbCp* c    = e->m[k];
        const float cutsq = (float)c->cutforcesq;
        for (size_t q = 0; q < e->groups.size() && gid[k] < 0; q++) {
            const auto& gr = e->groups[q];
            if (gr.N == c->N && gr.half == c->p.half_neigh && gr.cutsq == cutsq &&
                same_types(gr.ty, c->ty))
                gid[k] = (int)q;
        }
        if (gid[k] < 0) {
            gid[k] = (int)e->groups.size();
            e->groups.push_back({c->N, c->p.half_neigh, c->ty, cutsq, 0, 0});
        }
    }
    for (size_t q = 0; q < e->groups.size(); q++) {
        auto& gr = e->groups[q];
        gr.off   = maps.size();
        for (int k = 0; k < n; k++)
            if (gid[k] == (int)q) {
                MdbCp* c         = e->m[k];
                const int nb     = force_mixed_grid(c->ncl_cap, c->ty);
                c->energy_blocks = nb; // the partials a batched energy launch writes
                add(k, nb);
            }
        gr.nblocks = (int)(maps.size() - gr.off);
    }
    e->gid = gid;
    // dynamic regions, same sizes (contents written by ens_dyn_maps)
    e->dyn_begin     = maps.size();
    e->off_integ_dyn = maps.size();
    maps.resize(maps.size() + e->nb_integ, make_int2(-1, 0));
    e->off_ghost_dyn = maps.size();
    maps.resize(maps.size() + e->nb_ghost, make_int2(-1, 0));
    for (auto& gr : e->groups) {
        gr.off_dyn = maps.size();
        maps.resize(maps.size() + gr.nblocks, make_int2(-1, 0));
    }
    e->dyn_end = maps.size();
    if (!e->d_step) {
        ce = cudaMalloc((void**)&e->d_step, sizeof(CpStepMember) * n);
        if (ce == cudaSuccess) ce = cudaMalloc((void**)&e->d_force, sizeof(CpForceMember) * n);
        if (ce == cudaSuccess) ce = cudaMalloc((void**)&e->d_build, sizeof(CpBuildMember) * n);
        if (ce == cudaSuccess) ce = cudaMalloc((void**)&e->d_cnt_all, sizeof(int) * CP_SLOTS * n);
        if (ce == cudaSuccess)
            ce = cudaMallocHost((void**)&e->h_cnt_all, sizeof(int) * CP_SLOTS * n);
        if (ce == cudaSuccess) ce = cudaMalloc((void**)&e->d_flags, sizeof(int) * n);
        if (ce == cudaSuccess) ce = cudaMallocHost((void**)&e->h_flags, sizeof(int) * n);
        if (ce == cudaSuccess) ce = cudaMemset(e->d_flags, 0, sizeof(int) * n);
        if (ce != cudaSuccess) return ens_fail(e, MDB_ERR_NOMEM, "ensemble tables", ce);
    }
    if (maps.size() > e->bmap_cap) {
        if (e->d_bmap) cudaFree(e->d_bmap);
        if (e->h_dyn) cudaFreeHost(e->h_dyn);
        e->d_bmap   = nullptr;
        e->h_dyn    = nullptr;
        e->bmap_cap = maps.size() + maps.size() / 4;
        ce          = cudaMalloc((void**)&e->d_bmap, sizeof(int2) * e->bmap_cap);
        if (ce == cudaSuccess) ce = cudaMallocHost((void**)&e->h_dyn, sizeof(int2) * e->bmap_cap);
        if (ce != cudaSuccess) {
            e->bmap_cap = 0;
            return ens_fail(e, MDB_ERR_NOMEM, "ensemble block maps", ce);
        }
    }
    for (int k = 0; k < n; k++) st[k].flag = e->d_flags + k;
    const char* what = "member table";
    ce = cudaMemcpy(e->d_step, st.data(), sizeof(CpStepMember) * n, cudaMemcpyHostToDevice);
    if (ce == cudaSuccess)
        ce = cudaMemcpy(e->d_force, fo.data(), sizeof(CpForceMember) * n, cudaMemcpyHostToDevice);
    if (ce == cudaSuccess) {
        what = "rebuild table";
        ce = cudaMemcpy(e->d_build, bt.data(), sizeof(CpBuildMember) * n, cudaMemcpyHostToDevice);
    }
    if (ce == cudaSuccess && !maps.empty()) {
        what = "block maps";
        ce   = cudaMemcpy(e->d_bmap, maps.data(), sizeof(int2) * maps.size(),
            cudaMemcpyHostToDevice);
    }
    if (ce != cudaSuccess) return ens_fail(e, MDB_ERR_CUDA, what, ce);
    e->tables_ok = true;
    return ens_dyn_maps(e);
}

static void ens_integ(MdbCpEnsemble* e, bool final_, bool initial)
{
    launch_cp_integrate_batch(e->s, final_, initial, e->nb_integ, e->d_step,
        e->d_bmap + e->off_integ_dyn);
}

static void ens_forces(MdbCpEnsemble* e, bool energy)
{
    launch_zero_forces_batch(e->s, e->nb_integ, e->d_step, e->d_bmap + e->off_integ_dyn);
    for (const auto& gr : e->groups)
        launch_force_mixed_batch(e->s, gr.N, gr.half, energy, gr.ty, gr.cutsq, gr.nblocks,
            e->d_force, e->d_bmap + (energy ? gr.off : gr.off_dyn));
}

// per-member work on the members' streams, forked from and joined to e->s
template <class F> static void ens_fork(MdbCpEnsemble* e, F&& body)
{
    cudaEventRecord(e->fork, e->s);
    for (size_t k = 0; k < e->m.size(); k++) {
        MdbCp* c = e->m[k];
        cudaStreamWaitEvent(c->s, e->fork, 0);
        body(c);
        cudaEventRecord(e->join[k], c->s);
        cudaStreamWaitEvent(e->s, e->join[k], 0);
    }
}

// updateAtoms + the whole rebuild of the members (every member, or with only
// those whose flag in only is set), stage by stage (block maps of the
// capacities), then every member's counters into d_cnt_all
static void ens_rebuild_stages(MdbCpEnsemble* e, const int* only)
{
    const int n = (int)e->m.size();
    auto stage  = [e, only](int st) {
        launch_build_stage_batch(e->s, st, e->nb_stage[st], e->d_build,
            e->d_bmap + e->off_stage[st], only);
    };
    stage(CB_RESET);
    stage(CB_GATHER);
    stage(CB_BIN);
    launch_scan_batch(e->s, 0, n, e->d_build, only);
    stage(CB_SCATTER);
    stage(CB_SORT);
    launch_scan_batch(e->s, 1, n, e->d_build, only);
    stage(CB_CLUSTERS);
    stage(CB_GCOUNT);
    launch_scan_batch(e->s, 2, n, e->d_build, only);
    stage(CB_GWRITE);
    stage(CB_GFIRST);
    stage(CB_GCOLS);
    stage(CB_CSIZES);
    launch_scan_batch(e->s, 3, n, e->d_build, only);
    stage(CB_GSCATTER);
    stage(CB_MERGE);
    stage(CB_PREP);
    stage(CB_LIST);
    launch_counters_batch(e->s, n, e->d_build, e->d_cnt_all);
}

// positions as built, for the members' displacement checks
static void ens_snapshots(MdbCpEnsemble* e)
{
    for (MdbCp* c : e->m)
        if (c->disp_max > 0.0 && c->xbuild)
            cudaMemcpyAsync(c->xbuild, c->cx, sizeof(double4) * c->ncl_cap * c->M,
                cudaMemcpyDeviceToDevice, e->s);
}

static void ens_body_batched(MdbCpEnsemble* e, int kind)
{
    const bool fi = kind == EG_PLAIN_FI || kind == EG_FRONT_FI || kind == EG_REB_FI;
    switch (kind) {
    case EG_PLAIN_FI:
    case EG_PLAIN_I:
    case EG_FRONT_FI:
    case EG_FRONT_I:
        ens_integ(e, fi, true);
        launch_ghost_update_batch(e->s, e->nb_ghost, e->d_step, e->d_bmap + e->off_ghost_dyn,
            nullptr);
        if (kind == EG_PLAIN_FI || kind == EG_PLAIN_I) ens_forces(e, false);
        break;
    case EG_REB_FI:
    case EG_REB_I:
    case EG_REB_NOINT: {
        // updateAtoms + the whole rebuild, stage by stage: of every member on
        // the schedule; of the members whose displacement flag is up in a
        // checked step (EG_REB_NOINT), the others' ghosts updated instead
        if (kind != EG_REB_NOINT) {
            ens_integ(e, fi, true);
            ens_rebuild_stages(e, nullptr);
        } else {
            launch_ghost_update_batch(e->s, e->nb_ghost, e->d_step,
                e->d_bmap + e->off_ghost_dyn, e->d_flags);
            ens_rebuild_stages(e, e->d_flags);
        }
        cudaMemcpyAsync(e->h_cnt_all, e->d_cnt_all, sizeof(int) * CP_SLOTS * e->m.size(),
            cudaMemcpyDeviceToHost, e->s);
        // positions as built, for the members' displacement checks (the
        // flags are cleared by the host after the rebuild)
        if (kind != EG_REB_NOINT) ens_snapshots(e);
        else
            launch_snapshot_batch(e->s, e->nb_integ, e->d_step, e->d_bmap + e->off_integ,
                e->d_flags);
        break;
    }
    case EG_CK_FI:
    case EG_CK_I:
        ens_integ(e, kind == EG_CK_FI, true);
        cudaMemcpyAsync(e->h_flags, e->d_flags, sizeof(int) * e->m.size(),
            cudaMemcpyDeviceToHost, e->s);
        break;
    case EG_GHOST:
        launch_ghost_update_batch(e->s, e->nb_ghost, e->d_step, e->d_bmap + e->off_ghost_dyn,
            nullptr);
        break;
    case EG_FORCE: ens_forces(e, false); break;
    case EG_SAMPLE:
        ens_forces(e, true);
        ens_integ(e, true, false);
        ens_fork(e, [](MdbCp* c) {
            enq_thermo(c, 0, true);
            cudaMemcpyAsync(c->h_red, c->red, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->s);
        });
        break;
    case EG_FINAL: ens_integ(e, true, false); break;
    }
}

// rebuild every member when some member's displacement flag is up
__global__ void k_ens_chk_reb(cudaGraphConditionalHandle h, const int* flags, int n, int* st,
    int* rebuilds)
{
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x)
        if (flags[k]) {
            any = 1;
            if (st[0] == 0) rebuilds[k]++; // the member's own rebuild count
        }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (any) st[2]++;
        cudaGraphSetConditional(h, any ? 1u : 0u);
    }
}

// after a device rebuild: a member whose counters eval_build would grow (or
// reject) stops the call
__global__ void k_ens_chk_built(const CpBuildMember* __restrict__ tab, int n, int* st)
{
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int* c = tab[k].cnt;
        if (c[CP_BADBIN] > 0 || c[CP_NGC_TOTAL] > tab[k].ngc_cap ||
            c[CP_MAXNEED] >= tab[k].maxneighs)
            st[0] = 1;
    }
}

// The block maps of the members' current clusters (ens_dyn_maps' layout: per
// region the members in order, each with its blocks, then unused entries),
// from the device counters after a rebuild inside the checked step graph.
// One block; a member's block count as launch_* computes it.
template <class F>
__device__ void fill_map_region(int2* out, int cap, int n, F blocks_of)
{
    __shared__ int s_scan[256];
    __shared__ int s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (int base = 0; base < n; base += blockDim.x) {
        const int k = base + threadIdx.x;
        const int c = k < n ? blocks_of(k) : 0;
        s_scan[threadIdx.x] = c;
        __syncthreads();
        for (int o = 1; o < (int)blockDim.x; o <<= 1) {
            const int v = threadIdx.x >= o ? s_scan[threadIdx.x - o] : 0;
            __syncthreads();
            s_scan[threadIdx.x] += v;
            __syncthreads();
        }
        const int start = s_carry + s_scan[threadIdx.x] - c;
        for (int b = 0; b < c && start + b < cap; b++) out[start + b] = make_int2(k, b);
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) s_carry += s_scan[threadIdx.x];
        __syncthreads();
    }
    for (int w = min(s_carry, cap) + threadIdx.x; w < cap; w += blockDim.x)
        out[w] = make_int2(-1, 0);
    __syncthreads();
}

__global__ void __launch_bounds__(256) k_ens_dyn_maps(const CpBuildMember* __restrict__ tab,
    const int* __restrict__ info, int n, int2* bmap, size_t off_integ, int nb_integ,
    size_t off_ghost, int nb_ghost, const size_t* __restrict__ goff,
    const int* __restrict__ gnb, int ngroups)
{
    fill_map_region(bmap + off_integ, nb_integ, n, [&](int k) {
        return (int)(((long long)tab[k].cnt[CP_NCL] * info[5 * k] + MDB_NTHREADS - 1) /
                     MDB_NTHREADS);
    });
    fill_map_region(bmap + off_ghost, nb_ghost, n, [&](int k) {
        return (int)(((long long)tab[k].cnt[CP_NGC] * info[5 * k + 1] + MDB_NTHREADS - 1) /
                     MDB_NTHREADS);
    });
    for (int q = 0; q < ngroups; q++)
        fill_map_region(bmap + goff[q], gnb[q], n, [&](int k) {
            if (info[5 * k + 2] != q) return 0;
            const int nt = info[5 * k + 4];
            return (int)(((long long)tab[k].cnt[CP_NCL] * 32 / info[5 * k + 3] + nt - 1) / nt);
        });
}

// the member table of k_ens_dyn_maps for the current groups
static int ens_map_info(MdbCpEnsemble* e)
{
    const int n = (int)e->m.size(), ng = (int)e->groups.size();
    std::vector<int> info(5 * (size_t)n);
    for (int k = 0; k < n; k++) {
        const MdbCp* c = e->m[k];
        info[5 * k]     = c->M;
        info[5 * k + 1] = c->N;
        info[5 * k + 2] = e->gid[k];
        info[5 * k + 3] = c->ty.force_cpw;
        info[5 * k + 4] = force_mixed_threads(c->ty);
    }
    std::vector<size_t> goff(std::max(ng, 1));
    std::vector<int> gnb(std::max(ng, 1));
    for (int q = 0; q < ng; q++) goff[q] = e->groups[q].off_dyn, gnb[q] = e->groups[q].nblocks;
    cudaError_t ce = cudaSuccess;
    if (!e->d_mapinfo) {
        ce = cudaMalloc((void**)&e->d_mapinfo, sizeof(int) * info.size());
        if (ce == cudaSuccess) ce = cudaMalloc((void**)&e->d_goff, sizeof(size_t) * 64);
        if (ce == cudaSuccess) ce = cudaMalloc((void**)&e->d_gnb, sizeof(int) * 64);
        if (ce != cudaSuccess) return ens_fail(e, MDB_ERR_NOMEM, "ensemble map table", ce);
    }
    if (ng > 64) return ens_fail(e, MDB_ERR_ARG, "more than 64 force groups");
    ce = cudaMemcpy(e->d_mapinfo, info.data(), sizeof(int) * info.size(), cudaMemcpyHostToDevice);
    if (ce == cudaSuccess)
        ce = cudaMemcpy(e->d_goff, goff.data(), sizeof(size_t) * goff.size(), cudaMemcpyHostToDevice);
    if (ce == cudaSuccess)
        ce = cudaMemcpy(e->d_gnb, gnb.data(), sizeof(int) * gnb.size(), cudaMemcpyHostToDevice);
    if (ce != cudaSuccess) return ens_fail(e, MDB_ERR_CUDA, "ensemble map table", ce);
    return MDB_OK;
}

// One checked step of a batched ensemble as a graph, as capture_chk for a
// single system: gate; the fused integration with every member's test; if a
// flag is up, updateAtoms + the rebuild of every member, the overflow test,
// the snapshots and the flags cleared, else the ghost update; then the force.
// Every launch uses the block maps of the current clusters, which the rebuild
// refreshes on the device from the members' new counters.
static int ens_capture_chk(MdbCpEnsemble* e)
{
    int rc = ens_map_info(e);
    if (rc) return rc;
    cudaError_t ce = cudaSuccess;
    for (cudaStream_t& c : e->s_cap)
        if (!c && (ce = cudaStreamCreateWithFlags(&c, cudaStreamNonBlocking)) != cudaSuccess)
            return ens_fail(e, MDB_ERR_CUDA, "capture stream", ce);
    const cudaStream_t s0 = e->s, s1 = e->s_cap[0], s2 = e->s_cap[1];
    const cudaStreamCaptureMode mode = cudaStreamCaptureModeThreadLocal;
    const int n = (int)e->m.size();
    cudaGraphConditionalHandle h_step = 0, h_reb = 0, h_force = 0;
    cudaGraph_t step[1] = {nullptr}, reb[2] = {nullptr, nullptr}, frc[1] = {nullptr};
    cudaGraph_t graph = nullptr;
    const long long m0 = mark();
    long long* k = e->chk_k;
    bool cap1 = false, cap2 = false;
    auto body2 = [&](cudaGraph_t g, int what) -> cudaError_t {
        cudaError_t r = cudaStreamBeginCaptureToGraph(s2, g, nullptr, nullptr, 0, mode);
        if (r != cudaSuccess) return r;
        cap2 = true;
        e->s = s2;
        long long m = mark();
        if (what == 0) {
            // the members whose flag is up rebuild, the others update their
            // ghosts as in a plain step
            launch_ghost_update_batch(s2, e->nb_ghost, e->d_step, e->d_bmap + e->off_ghost_dyn,
                e->d_flags);
            ens_rebuild_stages(e, e->d_flags);
            k_ens_chk_built<<<1, 128, 0, s2>>>(e->d_build, n, e->dstate);
            k_ens_dyn_maps<<<1, 256, 0, s2>>>(e->d_build, e->d_mapinfo, n, e->d_bmap,
                e->off_integ_dyn, e->nb_integ, e->off_ghost_dyn, e->nb_ghost, e->d_goff,
                e->d_gnb, (int)e->groups.size());
            launch_snapshot_batch(s2, e->nb_integ, e->d_step, e->d_bmap + e->off_integ,
                e->d_flags);
            cudaMemsetAsync(e->d_flags, 0, sizeof(int) * n, s2);
            k[2] = mark() - m + 2;
        } else if (what == 1) {
            launch_ghost_update_batch(s2, e->nb_ghost, e->d_step, e->d_bmap + e->off_ghost_dyn,
                nullptr);
            k[1] = mark() - m;
        } else {
            ens_forces(e, false);
            k[3] = mark() - m;
        }
        e->s = s1;
        r = cudaGetLastError();
        cudaGraph_t out = nullptr;
        cudaError_t r2  = cudaStreamEndCapture(s2, &out);
        cap2            = false;
        return r != cudaSuccess ? r : r2;
    };
    ce = cudaStreamBeginCapture(s0, mode);
    if (ce == cudaSuccess) ce = cap_handle(s0, &h_step);
    if (ce == cudaSuccess) {
        k_chk_gate<<<1, 1, 0, s0>>>(h_step, e->dstate);
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cap_conditional(s0, h_step, 1, step);
    if (ce == cudaSuccess) ce = cudaStreamBeginCaptureToGraph(s1, step[0], nullptr, nullptr, 0, mode);
    if (ce == cudaSuccess) {
        cap1   = true;
        e->s   = s1;
        long long m = mark();
        ens_integ(e, true, true);
        k[0] = mark() - m + 2;
        ce   = cap_handle(s1, &h_reb);
    }
    if (ce == cudaSuccess) {
        k_ens_chk_reb<<<1, 128, 0, s1>>>(h_reb, e->d_flags, n, e->dstate, e->d_rebcnt);
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cap_conditional(s1, h_reb, 2, reb);
    if (ce == cudaSuccess) ce = body2(reb[0], 0);
    if (ce == cudaSuccess) ce = body2(reb[1], 1);
    if (ce == cudaSuccess) ce = cap_handle(s1, &h_force);
    if (ce == cudaSuccess) {
        k_chk_force<<<1, 1, 0, s1>>>(h_force, e->dstate);
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cap_conditional(s1, h_force, 1, frc);
    if (ce == cudaSuccess) ce = body2(frc[0], 2);
    e->s            = s0;
    mdb::g_launches = m0;
    if (cap2) {
        cudaGraph_t g2 = nullptr;
        cudaStreamEndCapture(s2, &g2);
    }
    if (cap1) {
        cudaGraph_t g1        = nullptr;
        const cudaError_t ce1 = cudaStreamEndCapture(s1, &g1);
        if (ce == cudaSuccess) ce = ce1;
    }
    const cudaError_t ce0 = cudaStreamEndCapture(s0, &graph);
    if (ce == cudaSuccess) ce = ce0;
    if (ce == cudaSuccess) ce = cudaGraphInstantiate(&e->g[EG_CHK].exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (ce != cudaSuccess) {
        cudaGetLastError();
        return ens_fail(e, MDB_ERR_CUDA, "checked ensemble step graph", ce);
    }
    e->g[EG_CHK].kernels = 1;
    return MDB_OK;
}

static int ens_capture(MdbCpEnsemble* e, int kind)
{
    CpGraph& g = e->g[kind];
    if (g.exec) return MDB_OK;
    if (e->batched) {
        int rc = ens_tables(e);
        if (rc) return rc;
    }
    if (kind == EG_CHK) return ens_capture_chk(e);
    cudaGraph_t graph;
    long long m0 = mark();
    cudaError_t ce = cudaStreamBeginCapture(e->s, cudaStreamCaptureModeThreadLocal);
    if (ce != cudaSuccess) return ens_fail(e, MDB_ERR_CUDA, "ensemble capture", ce);
    if (e->batched) ens_body_batched(e, kind);
    else ens_fork(e, [kind](MdbCp* c) { ens_body(c, kind); });
    ce        = cudaStreamEndCapture(e->s, &graph);
    g.kernels = mdb::g_launches - m0;
    mdb::g_launches = m0;
    if (ce != cudaSuccess) return ens_fail(e, MDB_ERR_CUDA, "ensemble capture", ce);
    ce = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return ens_fail(e, MDB_ERR_CUDA, "ensemble graph instantiate", ce);
    return MDB_OK;
}

static int ens_launch(MdbCpEnsemble* e, int kind)
{
    for (size_t k = 0; k < e->m.size(); k++)
        if (e->gen[k] != e->m[k]->gen) {
            ens_drop(e);
            break;
        }
    int rc = ens_capture(e, kind);
    if (rc) return rc;
    cudaError_t ce = cudaGraphLaunch(e->g[kind].exec, e->s);
    if (ce != cudaSuccess) return ens_fail(e, MDB_ERR_CUDA, "ensemble graph launch", ce);
    e->launches += e->g[kind].kernels;
    return MDB_OK;
}

extern "C" int mdb_cp_ensemble_create(MdbCp* const* members, int n, MdbCpEnsemble** out)
{
    if (!members || n < 1 || !out) return MDB_ERR_ARG;
    *out = nullptr;
    for (int k = 0; k < n; k++) {
        MdbCp* c = members[k];
        if (!c || !c->have_list) return MDB_ERR_STATE;
        if (c->dev != members[0]->dev || c->p.reneigh_every != members[0]->p.reneigh_every ||
            c->p.nstat != members[0]->p.nstat || c->prune_every != members[0]->prune_every)
            return MDB_ERR_ARG;
        // the batched rebuild does not derive pair codes: members run the
        // cluster-pair kernel
        if (c->force_path != 0) return fail(c, MDB_ERR_ARG, "ensemble member on force_path 1");
    }
    MdbCpEnsemble* e = new MdbCpEnsemble();
    e->m.assign(members, members + n);
    e->gen.assign(n, 0);
    for (int k = 0; k < n; k++) e->gen[k] = members[k]->gen;
    e->dev = members[0]->dev;
    cudaError_t ce = cudaSetDevice(e->dev);
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&e->s, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming);
    e->join.assign(n, nullptr);
    for (int k = 0; k < n && ce == cudaSuccess; k++)
        ce = cudaEventCreateWithFlags(&e->join[k], cudaEventDisableTiming);
    if (ce == cudaSuccess) ce = cudaMallocHost((void**)&e->h_red, 4 * sizeof(double) * n);
    e->batched = true;
    for (int k = 0; k < n; k++) e->batched = e->batched && members[k]->mixed;
    if (ce != cudaSuccess) {
        mdb_cp_ensemble_destroy(e);
        return MDB_ERR_CUDA;
    }
    *out = e;
    return MDB_OK;
}

extern "C" int mdb_cp_ensemble_destroy(MdbCpEnsemble* e)
{
    if (!e) return MDB_ERR_ARG;
    cudaSetDevice(e->dev);
    if (e->s) cudaStreamSynchronize(e->s);
    ens_drop(e);
    for (auto ev : e->join)
        if (ev) cudaEventDestroy(ev);
    if (e->fork) cudaEventDestroy(e->fork);
    if (e->h_red) cudaFreeHost(e->h_red);
    if (e->d_step) cudaFree(e->d_step);
    if (e->d_force) cudaFree(e->d_force);
    if (e->d_bmap) cudaFree(e->d_bmap);
    if (e->d_build) cudaFree(e->d_build);
    if (e->d_cnt_all) cudaFree(e->d_cnt_all);
    if (e->h_cnt_all) cudaFreeHost(e->h_cnt_all);
    if (e->h_dyn) cudaFreeHost(e->h_dyn);
    if (e->d_flags) cudaFree(e->d_flags);
    if (e->h_flags) cudaFreeHost(e->h_flags);
    if (e->dstate) cudaFree(e->dstate);
    if (e->h_dstate) cudaFreeHost(e->h_dstate);
    if (e->d_rebcnt) cudaFree(e->d_rebcnt);
    if (e->h_rebcnt) cudaFreeHost(e->h_rebcnt);
    if (e->d_mapinfo) cudaFree(e->d_mapinfo);
    if (e->d_goff) cudaFree(e->d_goff);
    if (e->d_gnb) cudaFree(e->d_gnb);
    for (cudaStream_t c : e->s_cap)
        if (c) cudaStreamDestroy(c);
    if (e->s) cudaStreamDestroy(e->s);
    delete e;
    return MDB_OK;
}

extern "C" const char* mdb_cp_ensemble_last_error(const MdbCpEnsemble* e)
{
    return e ? e->err.c_str() : "";
}
extern "C" void* mdb_cp_ensemble_stream(MdbCpEnsemble* e) { return e ? (void*)e->s : nullptr; }

extern "C" int mdb_cp_ensemble_tune(MdbCpEnsemble* e, const char* key, int value)
{
    if (!e || !key) return MDB_ERR_ARG;
    if (!strcmp(key, "batched")) {
        bool all_mixed = true;
        for (MdbCp* c : e->m) all_mixed = all_mixed && c->mixed;
        if (value && !all_mixed) return ens_fail(e, MDB_ERR_ARG, "batched needs mixed members");
        cudaStreamSynchronize(e->s);
        e->batched = value != 0;
        ens_drop(e);
        return MDB_OK;
    }
    if (!strcmp(key, "check_on_host")) {
        if (value < 0 || value > 1) return MDB_ERR_ARG;
        e->check_host = value != 0;
        return MDB_OK;
    }
    return ens_fail(e, MDB_ERR_ARG, "unknown tuning key");
}
extern "C" long long mdb_cp_ensemble_launch_count(const MdbCpEnsemble* e)
{
    return e ? e->launches : 0;
}

// rebuild: one graph for all members, one synchronisation, then members whose
// buffers overflowed grow and rebuild on their own (their atom arrays already
// hold the wrapped state, so the rebuild is idempotent)
static int ens_rebuild(MdbCpEnsemble* e, int kind)
{
    int rc = ens_launch(e, kind);
    if (rc) return rc;
    cudaError_t ce = cudaStreamSynchronize(e->s);
    if (ce == cudaSuccess && e->d_flags)
        ce = cudaMemsetAsync(e->d_flags, 0, sizeof(int) * e->m.size(), e->s);
    if (ce != cudaSuccess) return ens_fail(e, MDB_ERR_CUDA, "ensemble rebuild", ce);
    for (size_t k = 0; k < e->m.size(); k++) {
        MdbCp* c = e->m[k];
        if (e->batched)
            memcpy(c->h_cnt, e->h_cnt_all + k * CP_SLOTS, sizeof(int) * CP_SLOTS);
        int r = eval_build(c, CHK_ALL);
        if (r < 0) return ens_fail(e, -r, c->err.c_str());
        if (r > 0) {
            // grown buffers bump the member's generation: graphs are recaptured
            rc = do_build(c);
            if (rc) return ens_fail(e, rc, c->err.c_str());
            // its snapshot copy ran on the member's stream
            ce = cudaStreamSynchronize(c->s);
            if (ce != cudaSuccess) return ens_fail(e, MDB_ERR_CUDA, "member rebuild", ce);
        }
        c->have_clusters = c->have_ghosts = c->have_list = true;
        if (c->disp_max > 0.0 && c->xbuild) c->snap_valid = true;
    }
    return ens_dyn_maps(e);
}

// The device's record of the checked step graphs launched since the last call
// (their steps in `launched`), as chk_resolve for a single system: counts
// rebuilds and kernels, refreshes the counters and block maps after device
// rebuilds, and when a rebuild overflowed a member's buffer grows it, replays
// that member's build, runs the step's force and sets *resume to the step.
static int ens_chk_resolve(MdbCpEnsemble* e, std::vector<int>& launched, int* resume)
{
    *resume = -1;
    if (launched.empty()) return MDB_OK;
    const int n    = (int)e->m.size();
    cudaError_t ce = cudaMemcpyAsync(e->h_dstate, e->dstate, 3 * sizeof(int),
        cudaMemcpyDeviceToHost, e->s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->s);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(e->dstate, 0, 3 * sizeof(int), e->s);
    if (ce != cudaSuccess) return ens_fail(e, MDB_ERR_CUDA, "checked steps", ce);
    const int stopped = e->h_dstate[0], ran = e->h_dstate[1], reb = e->h_dstate[2];
    const long long* k = e->chk_k;
    e->launches += (long long)launched.size() + ran * k[0] + (ran - reb) * k[1] + reb * k[2] +
                   (ran - stopped) * k[3];
    e->chk_steps += ran;
    e->chk_replays += stopped ? 1 : 0;
    if (reb > 0) {
        ce = cudaMemcpyAsync(e->h_rebcnt, e->d_rebcnt, sizeof(int) * n, cudaMemcpyDeviceToHost,
            e->s);
        if (ce == cudaSuccess) ce = cudaMemsetAsync(e->d_rebcnt, 0, sizeof(int) * n, e->s);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->s);
        if (ce != cudaSuccess) return ens_fail(e, MDB_ERR_CUDA, "checked steps (rebuilds)", ce);
        for (int q = 0; q < n; q++) e->m[q]->rebuilds_check += e->h_rebcnt[q];
    }
    int rc = MDB_OK;
    if (reb > 0) {
        ce = cudaMemcpyAsync(e->h_cnt_all, e->d_cnt_all, sizeof(int) * CP_SLOTS * n,
            cudaMemcpyDeviceToHost, e->s);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->s);
        if (ce != cudaSuccess) return ens_fail(e, MDB_ERR_CUDA, "checked steps (counters)", ce);
        for (int q = 0; q < n; q++)
            memcpy(e->m[q]->h_cnt, e->h_cnt_all + (size_t)q * CP_SLOTS, sizeof(int) * CP_SLOTS);
    }
    if (stopped) {
        if (ran < 1 || ran > (int)launched.size())
            return ens_fail(e, MDB_ERR_CUDA, "checked steps: inconsistent device record");
        for (MdbCp* c : e->m) {
            const int r = eval_build(c, CHK_ALL);
            if (r < 0) return ens_fail(e, -r, c->err.c_str());
            if (r > 0) {
                // grown buffers bump the member's generation: graphs are recaptured
                if ((rc = do_build(c))) return ens_fail(e, rc, c->err.c_str());
                if ((ce = cudaStreamSynchronize(c->s)) != cudaSuccess)
                    return ens_fail(e, MDB_ERR_CUDA, "member rebuild", ce);
            }
        }
        if ((rc = ens_dyn_maps(e)) || (rc = ens_launch(e, EG_FORCE))) return rc;
        *resume = launched[ran - 1];
    } else if (reb > 0 && (rc = ens_dyn_maps(e))) {
        return rc;
    }
    launched.clear();
    return MDB_OK;
}

extern "C" int mdb_cp_ensemble_check_stats(MdbCpEnsemble* e, long long* graph_steps,
    long long* replays)
{
    if (!e) return MDB_ERR_ARG;
    if (graph_steps) *graph_steps = e->chk_steps;
    if (replays) *replays = e->chk_replays;
    return MDB_OK;
}

extern "C" int mdb_cp_ensemble_run(MdbCpEnsemble* e, int first_step, int nsteps,
    MdbThermo* samples, int max_samples, int* nsamples)
{
    if (!e || nsteps < 0 || (max_samples > 0 && !samples)) return MDB_ERR_ARG;
    cudaSetDevice(e->dev);
    const int n = (int)e->m.size();
    MdbCp* c0   = e->m[0];
    if (nsamples) *nsamples = 0;
    for (MdbCp* c : e->m)
        if (!c->have_list) return ens_fail(e, MDB_ERR_STATE, "a member is not set up");
    // members' own streams may still hold work: order the ensemble after it
    for (MdbCp* c : e->m) cudaStreamSynchronize(c->s);
    cudaStreamSynchronize(e->s);
    int nslot = 0, rc;
    // displacement check (batched ensembles): a member that moved too far
    // since the last build makes every member rebuild in that step
    bool checked = false, force_reb = false;
    for (MdbCp* c : e->m) {
        if (c->disp_max <= 0.0) continue;
        if (!e->batched) return ens_fail(e, MDB_ERR_ARG, "the check needs a batched ensemble");
        checked = true;
        if (!c->snap_valid) {
            // no positions of the last build: rebuild first (this allocates)
            if ((rc = snapshot(c))) return ens_fail(e, rc, c->err.c_str());
            cudaStreamSynchronize(c->s);
            force_reb = true;
        }
    }
    // members may have been rebuilt on their own since the last run
    if ((rc = ens_dyn_maps(e))) return rc;
    const bool on_device = checked && !e->check_host;
    if (on_device && !e->dstate) {
        cudaError_t ce = cudaMalloc((void**)&e->dstate, 3 * sizeof(int));
        if (ce == cudaSuccess) ce = cudaMallocHost((void**)&e->h_dstate, 3 * sizeof(int));
        if (ce == cudaSuccess) ce = cudaMalloc((void**)&e->d_rebcnt, n * sizeof(int));
        if (ce == cudaSuccess) ce = cudaMallocHost((void**)&e->h_rebcnt, n * sizeof(int));
        if (ce == cudaSuccess) ce = cudaMemsetAsync(e->dstate, 0, 3 * sizeof(int), e->s);
        if (ce == cudaSuccess) ce = cudaMemsetAsync(e->d_rebcnt, 0, n * sizeof(int), e->s);
        if (ce != cudaSuccess) return ens_fail(e, MDB_ERR_NOMEM, "checked steps", ce);
    }
    std::vector<int> launched;
    const int last     = first_step + nsteps - 1;
    bool pending_final = false;
    for (int step = first_step; step <= last; step++) {
        const bool reneigh = (step + 1) % c0->p.reneigh_every == 0;
        const bool prune   = !reneigh && (step + 1) % c0->prune_every == 0;
        const bool sample  = max_samples > 0 && (step + 1) % c0->p.nstat == 0 && nslot < max_samples;
        // a checked step decided on the device: one graph launch, no synchronisation
        if (on_device && pending_final && !prune && !reneigh && !force_reb && !sample &&
            step != last) {
            if ((rc = ens_launch(e, EG_CHK))) return rc;
            launched.push_back(step);
            continue;
        }
        if (!launched.empty()) {
            int resume = -1;
            if ((rc = ens_chk_resolve(e, launched, &resume))) return rc;
            if (resume >= 0) {
                step = resume; // the steps after it did nothing: run them again
                continue;
            }
        }
        if (checked && !prune && !reneigh && !force_reb) {
            if ((rc = ens_launch(e, pending_final ? EG_CK_FI : EG_CK_I))) return rc;
            pending_final  = false;
            cudaError_t ce = cudaStreamSynchronize(e->s);
            if (ce != cudaSuccess) return ens_fail(e, MDB_ERR_CUDA, "ensemble check", ce);
            bool any = false;
            for (int k = 0; k < n; k++) any = any || e->h_flags[k] != 0;
            if (any) {
                // the members whose flag is up rebuild, the others update ghosts
                if ((rc = ens_rebuild(e, EG_REB_NOINT))) return rc;
                for (int k = 0; k < n; k++)
                    if (e->h_flags[k]) e->m[k]->rebuilds_check++;
            } else if ((rc = ens_launch(e, EG_GHOST))) {
                return rc;
            }
            if ((rc = ens_launch(e, sample ? EG_SAMPLE : EG_FORCE))) return rc;
            pending_final = !sample;
        } else if (checked && !prune) {
            // scheduled (or first) rebuild
            if ((rc = ens_rebuild(e, pending_final ? EG_REB_FI : EG_REB_I))) return rc;
            for (MdbCp* c : e->m) (reneigh ? c->rebuilds_sched : c->rebuilds_check)++;
            force_reb = false;
            if ((rc = ens_launch(e, sample ? EG_SAMPLE : EG_FORCE))) return rc;
            pending_final = !sample;
        } else if (prune) {
            // rare (default never): direct launches on the members' streams
            cudaStreamSynchronize(e->s);
            const long long m0 = mark();
            for (MdbCp* c : e->m) {
                if (pending_final) enq_final_initial(c);
                else enq_initial(c);
                enq_prune(c);
                enq_ghost_update(c);
                enq_force(c, false);
                cudaStreamSynchronize(c->s);
            }
            e->launches += mark() - m0;
            pending_final = true;
        } else if (reneigh) {
            if ((rc = ens_rebuild(e, pending_final ? EG_REB_FI : EG_REB_I))) return rc;
            if ((rc = ens_launch(e, sample ? EG_SAMPLE : EG_FORCE))) return rc;
            pending_final = !sample;
        } else {
            if (sample) {
                if ((rc = ens_launch(e, pending_final ? EG_FRONT_FI : EG_FRONT_I))) return rc;
                if ((rc = ens_launch(e, EG_SAMPLE))) return rc;
                pending_final = false;
            } else {
                if ((rc = ens_launch(e, pending_final ? EG_PLAIN_FI : EG_PLAIN_I))) return rc;
                pending_final = true;
            }
        }
        if (sample) {
            cudaError_t ce = cudaStreamSynchronize(e->s);
            if (ce != cudaSuccess) return ens_fail(e, MDB_ERR_CUDA, "ensemble sample", ce);
            for (int k = 0; k < n; k++) {
                MdbCp* c = e->m[k];
                finish_thermo(c, c->h_red, step + 1, &samples[(size_t)k * max_samples + nslot]);
                c->energy_valid = true;
            }
            nslot++;
        }
    }
    if (pending_final && (rc = ens_launch(e, EG_FINAL))) return rc;
    cudaError_t ce = cudaStreamSynchronize(e->s);
    if (ce != cudaSuccess) return ens_fail(e, MDB_ERR_CUDA, "ensemble run", ce);
    if (nsamples) *nsamples = nslot;
    return MDB_OK;
}
