/*
 * CPU oracle, cluster-pair scheme. TEST INFRASTRUCTURE ONLY (see
 * mdb_oracle_cp.h). Plain C, IEEE double, compiled with -ffp-contract=off
 * -fno-fast-math; fma() appears only where the reference's SIMD builds use an
 * explicit fused multiply-add.
 */
#include "mdb_oracle_cp.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define ORC_MIN(a, b) ((a) < (b) ? (a) : (b)) /* common/util.h:12 */
#define ORC_MAX(a, b) ((a) > (b) ? (a) : (b)) /* common/util.h:16 */

/* interaction masks, clusterpair/neighbor.h:21-30 */
#define MASK_ALL     0xffffffffu
#define MASK_DIAG    0x08ceu
#define MASK_J2_0    0x0002u
#define MASK_J2_1    0x002fu
#define MASK_J8_0    0xf0f8fcfeu
#define MASK_J8_1    0x0080c0e0u

struct OrcCp {
    OrcCpParams p;
    int M, N, jfac;
    double sqrt_eps_t[64], sigma3_t[64];

    /* atom arrays */
    int nlocal;
    double *ax, *av;
    int* at;

    /* xy columns (setupNeighbor, clusterpair/neighbor.c:108-215) */
    int nbinx, nbiny, mbinx, mbiny, mbinxlo, mbinylo, mbins;
    double binsizex, binsizey, bininvx, bininvy, cutneighsq, rbb_sq;
    int nstencil;
    int* stencil;
    int* col_count;
    int col_cap;
    int* col_atoms; /* mbins * col_cap */

    /* clusters */
    int ncl, ncj, ngc, dummy, nghost_atoms;
    int slot_cap, clu_cap;
    double *cx, *cv, *cf, *cse, *cs3;
    int* ct;
    int *inat, *cbin, *jnat;
    double *ibb, *jbb;
    int *border, *pbc;
    int gcap;

    /* j-cluster columns */
    int* jcol_count;
    int jcol_cap;
    int* jcol; /* (mbins + 1) * jcol_cap */

    /* list (AoS, neighbors[ci * maxneighs + k]) */
    int maxneighs, list_rows;
    int *numneigh, *nmasked, *neigh;
    unsigned* imask;

    double epot;
};

static void* orc_grow(void* p, size_t n)
{
    void* q = realloc(p, n ? n : 1);
    if (!q) {
        fprintf(stderr, "oracle: out of memory\n");
        exit(1);
    }
    return q;
}

OrcCp* orccp_create(const OrcCpParams* p)
{
    if (!p || p->cluster_m < 1 || (p->cluster_n != p->cluster_m && p->cluster_n != 2 * p->cluster_m))
        return NULL;
    if (p->ntypes < 1 || p->ntypes > 64) return NULL;
    OrcCp* s = (OrcCp*)calloc(1, sizeof(OrcCp));
    s->p     = *p;
    s->M     = p->cluster_m;
    s->N     = p->cluster_n;
    s->jfac  = s->N / s->M;
    /* computePerTypeLJParameters, common/parameter.c:31-45 */
    for (int t = 0; t < p->ntypes; t++) {
        double eps = p->epsilon_per_type ? p->epsilon_per_type[t] : p->epsilon;
        double sig = p->sigma_per_type ? p->sigma_per_type[t] : p->sigma;
        s->sqrt_eps_t[t] = sqrt(eps);
        s->sigma3_t[t]   = sig * sig * sig;
    }
    s->maxneighs = 200; /* initNeighbor, clusterpair/neighbor.c:73-77 */
    return s;
}

void orccp_destroy(OrcCp* s)
{
    if (!s) return;
    free(s->ax), free(s->av), free(s->at);
    free(s->stencil), free(s->col_count), free(s->col_atoms);
    free(s->cx), free(s->cv), free(s->cf), free(s->cse), free(s->cs3), free(s->ct);
    free(s->inat), free(s->cbin), free(s->jnat), free(s->ibb), free(s->jbb);
    free(s->border), free(s->pbc);
    free(s->jcol_count), free(s->jcol);
    free(s->numneigh), free(s->nmasked), free(s->neigh), free(s->imask);
    free(s);
}

int orccp_set_atoms(OrcCp* s, int n, const double* x, const double* v, const int* type)
{
    s->nlocal = n;
    s->ax     = (double*)orc_grow(s->ax, sizeof(double) * 3 * (size_t)n);
    s->av     = (double*)orc_grow(s->av, sizeof(double) * 3 * (size_t)n);
    s->at     = (int*)orc_grow(s->at, sizeof(int) * (size_t)n);
    memcpy(s->ax, x, sizeof(double) * 3 * (size_t)n);
    memcpy(s->av, v, sizeof(double) * 3 * (size_t)n);
    for (int i = 0; i < n; i++)
        s->at[i] = type ? type[i] : 0;
    return 0;
}

/* ---- columns ----------------------------------------------------------- */

/* bindist, clusterpair/neighbor.c:1343-1364 (2-D) */
static double orc_bindist2(OrcCp* s, int i, int j)
{
    double delx, dely;
    if (i > 0) delx = (i - 1) * s->binsizex;
    else if (i == 0) delx = 0.0;
    else delx = (i + 1) * s->binsizex;
    if (j > 0) dely = (j - 1) * s->binsizey;
    else if (j == 0) dely = 0.0;
    else dely = (j + 1) * s->binsizey;
    return delx * delx + dely * dely;
}

/* setupNeighbor, clusterpair/neighbor.c:108-215 (box at the origin) */
static void orc_setup_columns(OrcCp* s)
{
    const double xprd = s->p.xprd, yprd = s->p.yprd, zprd = s->p.zprd;
    const double cutneigh = s->p.cutneigh;
    double density  = ((double)s->p.natoms) / ((xprd - 0.0) * (yprd - 0.0) * (zprd - 0.0));
    double in_cell  = (double)ORC_MAX(s->M, s->N);
    double target_x = cbrt(in_cell / density);
    double target_y = cbrt(in_cell / density);
    s->nbinx        = ORC_MAX(1, (int)ceil((xprd - 0.0) / target_x));
    s->nbiny        = ORC_MAX(1, (int)ceil((yprd - 0.0) / target_y));
    s->binsizex     = (xprd - 0.0) / s->nbinx;
    s->binsizey     = (yprd - 0.0) / s->nbiny;
    s->bininvx      = 1.0 / s->binsizex;
    s->bininvy      = 1.0 / s->binsizey;
    s->cutneighsq   = cutneigh * cutneigh;

    double coord = 0.0 - cutneigh - 1.0e-6 * xprd;
    s->mbinxlo   = (int)(coord * s->bininvx);
    if (coord < 0.0) s->mbinxlo = s->mbinxlo - 1;
    coord       = xprd + cutneigh + 1.0e-6 * xprd;
    int mbinxhi = (int)(coord * s->bininvx);
    coord       = 0.0 - cutneigh - 1.0e-6 * yprd;
    s->mbinylo  = (int)(coord * s->bininvy);
    if (coord < 0.0) s->mbinylo = s->mbinylo - 1;
    coord       = yprd + cutneigh + 1.0e-6 * yprd;
    int mbinyhi = (int)(coord * s->bininvy);
    s->mbinxlo  = s->mbinxlo - 1;
    mbinxhi     = mbinxhi + 1;
    s->mbinx    = mbinxhi - s->mbinxlo + 1;
    s->mbinylo  = s->mbinylo - 1;
    mbinyhi     = mbinyhi + 1;
    s->mbiny    = mbinyhi - s->mbinylo + 1;

    int nextx = (int)(cutneigh * s->bininvx);
    int nexty = (int)(cutneigh * s->bininvy);
    if (nextx * s->binsizex < 0.999 * cutneigh) nextx++;
    if (nexty * s->binsizey < 0.999 * cutneigh) nexty++;
    s->stencil  = (int*)orc_grow(s->stencil, sizeof(int) * (2 * nexty + 1) * (2 * nextx + 1));
    s->nstencil = 0;
    for (int j = -nexty; j <= nexty; j++)
        for (int i = -nextx; i <= nextx; i++)
            if (orc_bindist2(s, i, j) < s->cutneighsq) s->stencil[s->nstencil++] = j * s->mbinx + i;
    s->mbins = s->mbinx * s->mbiny;

    /* buildNeighborCPU, clusterpair/neighbor.c:300-303 */
    double bbx = 0.5 * (s->binsizex + s->binsizex);
    double bby = 0.5 * (s->binsizey + s->binsizey);
    double rbb = ORC_MAX(0.0, cutneigh - 0.5 * sqrt(bbx * bbx + bby * bby));
    s->rbb_sq  = rbb * rbb;
    (void)zprd;
}

/* coord2bin2D, clusterpair/neighbor.c:1390-1407 (bin = iy * mbinx + ix + 1) */
static void orc_coord2bin2d(OrcCp* s, double x, double y, int* ix, int* iy)
{
    if (x >= s->p.xprd) *ix = (int)((x - s->p.xprd) * s->bininvx) + s->nbinx - s->mbinxlo;
    else if (x >= 0.0) *ix = (int)(x * s->bininvx) - s->mbinxlo;
    else *ix = (int)(x * s->bininvx) - s->mbinxlo - 1;
    if (y >= s->p.yprd) *iy = (int)((y - s->p.yprd) * s->bininvy) + s->nbiny - s->mbinylo;
    else if (y >= 0.0) *iy = (int)(y * s->bininvy) - s->mbinylo;
    else *iy = (int)(y * s->bininvy) - s->mbinylo - 1;
}

/* binAtoms (clusterpair/neighbor.c:1409-1449): atoms appended to their column
 * in index order */
static int orc_bin_atoms(OrcCp* s)
{
    s->col_count = (int*)orc_grow(s->col_count, sizeof(int) * s->mbins);
    memset(s->col_count, 0, sizeof(int) * s->mbins);
    int* bin_of = (int*)malloc(sizeof(int) * (size_t)(s->nlocal ? s->nlocal : 1));
    int cmax    = 1;
    for (int i = 0; i < s->nlocal; i++) {
        int ix, iy;
        orc_coord2bin2d(s, s->ax[3 * i], s->ax[3 * i + 1], &ix, &iy);
        int b = iy * s->mbinx + ix + 1;
        if (b < 0 || b >= s->mbins) {
            free(bin_of);
            return -1;
        }
        bin_of[i] = b;
        if (++s->col_count[b] > cmax) cmax = s->col_count[b];
    }
    s->col_cap   = cmax;
    s->col_atoms = (int*)orc_grow(s->col_atoms, sizeof(int) * (size_t)s->mbins * cmax);
    memset(s->col_count, 0, sizeof(int) * s->mbins);
    for (int i = 0; i < s->nlocal; i++) {
        int b                                               = bin_of[i];
        s->col_atoms[(size_t)b * s->col_cap + s->col_count[b]++] = i;
    }
    free(bin_of);
    return 0;
}

/* sortAtomsByZCoord (clusterpair/neighbor.c:1452-1481): selection sort that
 * swaps the first minimum into place, so equal z keep the order this swapping
 * produces */
static void orc_sort_columns(OrcCp* s)
{
    for (int b = 0; b < s->mbins; b++) {
        int c    = s->col_count[b];
        int* col = &s->col_atoms[(size_t)b * s->col_cap];
        for (int a = 0; a < c; a++) {
            int i = col[a], min_a = a, min_i = i;
            double min_z = s->ax[3 * i + 2];
            for (int k = a + 1; k < c; k++) {
                int j = col[k];
                if (s->ax[3 * j + 2] < min_z) {
                    min_a = k;
                    min_i = j;
                    min_z = s->ax[3 * j + 2];
                }
            }
            col[a]     = min_i;
            col[min_a] = i;
        }
    }
}

static void orc_reserve_clusters(OrcCp* s, int nclu_j)
{
    /* nclu_j: j-cluster slots needed (locals + ghosts + dummy) */
    int nslots = nclu_j * s->N;
    if (nslots > s->slot_cap) {
        int cap    = nslots + nslots / 2 + 64;
        s->cx      = (double*)orc_grow(s->cx, sizeof(double) * 3 * (size_t)cap);
        s->cv      = (double*)orc_grow(s->cv, sizeof(double) * 3 * (size_t)cap);
        s->cf      = (double*)orc_grow(s->cf, sizeof(double) * 3 * (size_t)cap);
        s->cse     = (double*)orc_grow(s->cse, sizeof(double) * (size_t)cap);
        s->cs3     = (double*)orc_grow(s->cs3, sizeof(double) * (size_t)cap);
        s->ct      = (int*)orc_grow(s->ct, sizeof(int) * (size_t)cap);
        s->slot_cap = cap;
    }
    int nclu = nslots / s->M + 2;
    if (nclu > s->clu_cap) {
        int cap    = nclu + nclu / 2 + 64;
        s->inat    = (int*)orc_grow(s->inat, sizeof(int) * (size_t)cap);
        s->cbin    = (int*)orc_grow(s->cbin, sizeof(int) * (size_t)cap);
        s->jnat    = (int*)orc_grow(s->jnat, sizeof(int) * (size_t)cap);
        s->ibb     = (double*)orc_grow(s->ibb, sizeof(double) * 6 * (size_t)cap);
        s->jbb     = (double*)orc_grow(s->jbb, sizeof(double) * 6 * (size_t)cap);
        s->clu_cap = cap;
    }
}

/* buildClustersCPU, clusterpair/neighbor.c:1513-1611 */
int orccp_build_clusters(OrcCp* s)
{
    const int M = s->M, N = s->N;
    if (orc_bin_atoms(s)) return -1;
    orc_sort_columns(s);
    int total = 0;
    for (int b = 0; b < s->mbins; b++) {
        int nc = (s->col_count[b] + M - 1) / M;
        if (N > M && nc % 2) nc++;
        total += nc;
    }
    orc_reserve_clusters(s, total / s->jfac + 1);
    s->ncl = 0;
    for (int b = 0; b < s->mbins; b++) {
        int c  = s->col_count[b];
        int nc = (c + M - 1) / M;
        if (N > M && nc % 2) nc++;
        int a = 0;
        for (int k = 0; k < nc; k++) {
            const int ci = s->ncl;
            double bb[6] = {INFINITY, -INFINITY, INFINITY, -INFINITY, INFINITY, -INFINITY};
            int nat      = 0;
            for (int cii = 0; cii < M; cii++) {
                int sl = ci * M + cii;
                if (a < c) {
                    int i   = s->col_atoms[(size_t)b * s->col_cap + a];
                    double x = s->ax[3 * i], y = s->ax[3 * i + 1], z = s->ax[3 * i + 2];
                    s->cx[3 * sl]     = x;
                    s->cx[3 * sl + 1] = y;
                    s->cx[3 * sl + 2] = z;
                    s->cv[3 * sl]     = s->av[3 * i];
                    s->cv[3 * sl + 1] = s->av[3 * i + 1];
                    s->cv[3 * sl + 2] = s->av[3 * i + 2];
                    if (bb[0] > x) bb[0] = x;
                    if (bb[1] < x) bb[1] = x;
                    if (bb[2] > y) bb[2] = y;
                    if (bb[3] < y) bb[3] = y;
                    if (bb[4] > z) bb[4] = z;
                    if (bb[5] < z) bb[5] = z;
                    int t       = s->at[i];
                    s->ct[sl]   = t;
                    s->cse[sl]  = s->sqrt_eps_t[t];
                    s->cs3[sl]  = s->sigma3_t[t];
                    nat++;
                } else {
                    s->cx[3 * sl] = s->cx[3 * sl + 1] = s->cx[3 * sl + 2] = INFINITY;
                    s->ct[sl]                                           = 0;
                    s->cse[sl]                                          = 0.0;
                    s->cs3[sl]                                          = 0.0;
                }
                a++;
            }
            s->cbin[ci] = b;
            s->inat[ci] = nat;
            memcpy(&s->ibb[6 * ci], bb, sizeof(bb));
            s->ncl++;
        }
    }
    return 0;
}

/* defineJClusters, clusterpair/neighbor.c:1807-1915 (M == N and M < N) */
void orccp_define_jclusters(OrcCp* s)
{
    s->ncj = s->ncl / s->jfac;
    if (s->jfac == 1) {
        memcpy(s->jbb, s->ibb, sizeof(double) * 6 * (size_t)s->ncl);
        memcpy(s->jnat, s->inat, sizeof(int) * (size_t)s->ncl);
        return;
    }
    for (int ci = 0; ci < s->ncl; ci += 2) {
        const double* a = &s->ibb[6 * ci];
        const double* b = &s->ibb[6 * (ci + 1)];
        double* j       = &s->jbb[6 * (ci >> 1)];
        j[0]            = ORC_MIN(a[0], b[0]);
        j[1]            = ORC_MAX(a[1], b[1]);
        j[2]            = ORC_MIN(a[2], b[2]);
        j[3]            = ORC_MAX(a[3], b[3]);
        j[4]            = ORC_MIN(a[4], b[4]);
        j[5]            = ORC_MAX(a[5], b[5]);
        s->jnat[ci >> 1] = s->inat[ci] + s->inat[ci + 1];
    }
}

/* ---- cluster ghosts (clusterpair/pbc.c) --------------------------------- */

static void orc_add_ghost(OrcCp* s, int cj, int dx, int dy, int dz)
{
    int g = s->ngc++;
    if (g >= s->gcap) {
        s->gcap   = 2 * s->gcap + 1024;
        s->border = (int*)orc_grow(s->border, sizeof(int) * (size_t)s->gcap);
        s->pbc    = (int*)orc_grow(s->pbc, sizeof(int) * 3 * (size_t)s->gcap);
    }
    orc_reserve_clusters(s, s->ncj + s->ngc + 1);
    const int cg   = s->ncj + g;
    const int nat  = s->jnat[cj];
    s->border[g]   = cj;
    s->pbc[3 * g]  = dx;
    s->pbc[3 * g + 1] = dy;
    s->pbc[3 * g + 2] = dz;
    s->jnat[cg]    = nat;
    s->nghost_atoms += nat;
    for (int k = 0; k < nat; k++) {
        s->ct[cg * s->N + k]  = s->ct[cj * s->N + k];
        s->cse[cg * s->N + k] = s->cse[cj * s->N + k];
        s->cs3[cg * s->N + k] = s->cs3[cj * s->N + k];
    }
}

/* updatePbcCPU, clusterpair/pbc.c:43-113 */
void orccp_update_pbc(OrcCp* s, int first)
{
    const int N = s->N;
    for (int g = 0; g < s->ngc; g++) {
        const int cj = s->ncj + g, o = s->border[g];
        double bb[6] = {INFINITY, -INFINITY, INFINITY, -INFINITY, INFINITY, -INFINITY};
        for (int k = 0; k < s->jnat[cj]; k++) {
            const double* src = &s->cx[3 * (o * N + k)];
            double* dst       = &s->cx[3 * (cj * N + k)];
            double x          = src[0] + s->pbc[3 * g] * s->p.xprd;
            double y          = src[1] + s->pbc[3 * g + 1] * s->p.yprd;
            double z          = src[2] + s->pbc[3 * g + 2] * s->p.zprd;
            dst[0] = x, dst[1] = y, dst[2] = z;
            s->ct[cj * N + k] = s->ct[o * N + k];
            if (first) {
                if (bb[0] > x) bb[0] = x;
                if (bb[1] < x) bb[1] = x;
                if (bb[2] > y) bb[2] = y;
                if (bb[3] < y) bb[3] = y;
                if (bb[4] > z) bb[4] = z;
                if (bb[5] < z) bb[5] = z;
            }
        }
        if (first) {
            for (int k = s->jnat[cj]; k < N; k++) {
                double* dst = &s->cx[3 * (cj * N + k)];
                dst[0] = dst[1] = dst[2] = INFINITY;
                s->ct[cj * N + k]        = 0;
            }
            memcpy(&s->jbb[6 * cj], bb, sizeof(bb));
        }
    }
}

/* setupPbc, clusterpair/pbc.c:184-331: ghost j-clusters in the reference order
 * (6 faces, 8 corners, 12 edges per j-cluster), then the dummy cluster */
int orccp_setup_pbc(OrcCp* s)
{
    const double cut = s->p.cutneigh, xh = s->p.xprd - cut, yh = s->p.yprd - cut,
                 zh = s->p.zprd - cut;
    s->ngc          = 0;
    s->nghost_atoms = 0;
    for (int cj = 0; cj < s->ncj; cj++) {
        if (s->jnat[cj] <= 0) continue;
        const double* b = &s->jbb[6 * cj];
        const int lx = b[0] < cut, hx = b[1] >= xh, ly = b[2] < cut, hy = b[3] >= yh,
                  lz = b[4] < cut, hz = b[5] >= zh;
        if (lx) orc_add_ghost(s, cj, +1, 0, 0);
        if (hx) orc_add_ghost(s, cj, -1, 0, 0);
        if (ly) orc_add_ghost(s, cj, 0, +1, 0);
        if (hy) orc_add_ghost(s, cj, 0, -1, 0);
        if (lz) orc_add_ghost(s, cj, 0, 0, +1);
        if (hz) orc_add_ghost(s, cj, 0, 0, -1);
        if (lx && ly && lz) orc_add_ghost(s, cj, +1, +1, +1);
        if (lx && hy && lz) orc_add_ghost(s, cj, +1, -1, +1);
        if (lx && ly && hz) orc_add_ghost(s, cj, +1, +1, -1);
        if (lx && hy && hz) orc_add_ghost(s, cj, +1, -1, -1);
        if (hx && ly && lz) orc_add_ghost(s, cj, -1, +1, +1);
        if (hx && hy && lz) orc_add_ghost(s, cj, -1, -1, +1);
        if (hx && ly && hz) orc_add_ghost(s, cj, -1, +1, -1);
        if (hx && hy && hz) orc_add_ghost(s, cj, -1, -1, -1);
        if (lx && lz) orc_add_ghost(s, cj, +1, 0, +1);
        if (lx && hz) orc_add_ghost(s, cj, +1, 0, -1);
        if (hx && lz) orc_add_ghost(s, cj, -1, 0, +1);
        if (hx && hz) orc_add_ghost(s, cj, -1, 0, -1);
        if (ly && lz) orc_add_ghost(s, cj, 0, +1, +1);
        if (ly && hz) orc_add_ghost(s, cj, 0, +1, -1);
        if (hy && lz) orc_add_ghost(s, cj, 0, -1, +1);
        if (hy && hz) orc_add_ghost(s, cj, 0, -1, -1);
        if (ly && lx) orc_add_ghost(s, cj, +1, +1, 0);
        if (ly && hx) orc_add_ghost(s, cj, -1, +1, 0);
        if (hy && lx) orc_add_ghost(s, cj, +1, -1, 0);
        if (hy && hx) orc_add_ghost(s, cj, -1, -1, 0);
    }
    orc_reserve_clusters(s, s->ncj + s->ngc + 1);
    s->dummy = s->ncj + s->ngc;
    for (int k = 0; k < s->N; k++) {
        double* d = &s->cx[3 * (s->dummy * s->N + k)];
        d[0] = d[1] = d[2]            = INFINITY;
        s->ct[s->dummy * s->N + k]    = 0;
    }
    orccp_update_pbc(s, 1);
    return 0;
}

/* binJClusters, clusterpair/neighbor.c:1917-2094: local j-clusters appended in
 * cluster order, then each ghost j-cluster put in the column of its innermost
 * atom and inserted before the first entry whose bbminz is larger */
void orccp_bin_jclusters(OrcCp* s)
{
    const int N = s->N;
    int nb      = s->mbins + 1; /* a clamped ghost can address bin mbins */
    int* cnt    = (int*)calloc((size_t)nb, sizeof(int));
    int* gbin   = (int*)malloc(sizeof(int) * (size_t)(s->ngc ? s->ngc : 1));
    for (int ci = 0; ci < s->ncl; ci++)
        if (s->M >= N || ci % 2 == 0) cnt[s->cbin[ci]]++;
    for (int g = 0; g < s->ngc; g++) {
        const int cj = s->ncj + g;
        gbin[g]      = -1;
        if (s->jnat[cj] <= 0) continue;
        int ix, iy;
        orc_coord2bin2d(s, s->cx[3 * (cj * N)], s->cx[3 * (cj * N) + 1], &ix, &iy);
        ix = ORC_MAX(ORC_MIN(ix, s->mbinx - 1), 0);
        iy = ORC_MAX(ORC_MIN(iy, s->mbiny - 1), 0);
        for (int k = 1; k < s->jnat[cj]; k++) {
            int nix, niy;
            orc_coord2bin2d(s, s->cx[3 * (cj * N + k)], s->cx[3 * (cj * N + k) + 1], &nix, &niy);
            nix = ORC_MAX(ORC_MIN(nix, s->mbinx - 1), 0);
            niy = ORC_MAX(ORC_MIN(niy, s->mbiny - 1), 0);
            if (s->pbc[3 * g] > 0 && ix > nix) ix = nix;
            if (s->pbc[3 * g] < 0 && ix < nix) ix = nix;
            if (s->pbc[3 * g + 1] > 0 && iy > niy) iy = niy;
            if (s->pbc[3 * g + 1] < 0 && iy < niy) iy = niy;
        }
        gbin[g] = iy * s->mbinx + ix + 1;
        cnt[gbin[g]]++;
    }
    int cap = 1;
    for (int b = 0; b < nb; b++)
        cap = ORC_MAX(cap, cnt[b]);
    s->jcol_cap   = cap;
    s->jcol       = (int*)orc_grow(s->jcol, sizeof(int) * (size_t)nb * cap);
    s->jcol_count = (int*)orc_grow(s->jcol_count, sizeof(int) * (size_t)nb);
    memset(s->jcol_count, 0, sizeof(int) * (size_t)nb);
    for (int ci = 0; ci < s->ncl; ci++) {
        if (!(s->M >= N || ci % 2 == 0)) continue;
        int b                                          = s->cbin[ci];
        s->jcol[(size_t)b * cap + s->jcol_count[b]++] = ci / s->jfac;
    }
    for (int g = 0; g < s->ngc; g++) {
        if (gbin[g] < 0) continue;
        const int cj = s->ncj + g, b = gbin[g];
        int* col     = &s->jcol[(size_t)b * cap];
        int c        = s->jcol_count[b];
        double minz  = s->jbb[6 * cj + 4];
        int at       = c;
        for (int i = 0; i < c; i++)
            if (s->jbb[6 * col[i] + 4] > minz) {
                at = i;
                break;
            }
        for (int i = c; i > at; i--)
            col[i] = col[i - 1];
        col[at] = cj;
        s->jcol_count[b]++;
    }
    free(cnt);
    free(gbin);
}

/* ---- cluster-pair list --------------------------------------------------- */

/* get_imask_simd_j2/j4/j8, clusterpair/neighbor.c:245-267, selected by the
 * build's VECTOR_WIDTH (= N in the three builds used here) with rdiag = 1 */
static unsigned orc_imask(OrcCp* s, int ci, int cj)
{
    switch (s->N) {
    case 2:
        return ci * 2 == cj ? MASK_J2_0 : (ci * 2 + 1 == cj ? MASK_J2_1 : MASK_ALL);
    case 4:
        return ci == cj ? MASK_DIAG : MASK_ALL;
    default:
        return ci == cj * 2 ? MASK_J8_0 : (ci == cj * 2 + 1 ? MASK_J8_1 : MASK_ALL);
    }
}

static double orc_bb_axis(double imin, double imax, double jmin, double jmax)
{
    double dl = imin - jmax, dh = jmin - imax;
    double dm = ORC_MAX(dl, dh);
    return ORC_MAX(dm, 0.0);
}

/* any atom pair of (ci, cj) closer than cutsq; i atoms are the M slots of ci,
 * j atoms the N slots of cj (padding slots hold INF and never match) */
static int orc_any_pair(OrcCp* s, int ci, int cj, double cutsq)
{
    const int M = s->M, N = s->N;
    for (int a = 0; a < M; a++) {
        const double* xi = &s->cx[3 * (ci * M + a)];
        for (int b = 0; b < N; b++) {
            const double* xj = &s->cx[3 * (cj * N + b)];
            double dx = xi[0] - xj[0], dy = xi[1] - xj[1], dz = xi[2] - xj[2];
            double rsq = s->p.fma_rsq ? fma(dx, dx, fma(dy, dy, dz * dz))
                                      : dx * dx + dy * dy + dz * dz;
            if (rsq < cutsq) return 1;
        }
    }
    return 0;
}

/* buildNeighborCPU, clusterpair/neighbor.c:282-529: per i-cluster, the stencil
 * columns in order, each column's j-clusters in order (half lists skip
 * cj < ci_cj0); bounding-box distance (z, y, x) below cutneigh^2, accepted
 * outright below rbb^2, else if any atom pair is inside cutneigh; entries with
 * a diagonal mask are moved to the front. Grows maxneighs to 1.2x the largest
 * count and rebuilds when a row reaches maxneighs. */
int orccp_build_neighbor(OrcCp* s)
{
    const int half = s->p.half_neigh;
    for (;;) {
        const int ld = s->maxneighs;
        if (s->ncl > s->list_rows || !s->neigh) {
            s->list_rows = s->ncl;
            s->numneigh  = (int*)orc_grow(s->numneigh, sizeof(int) * (size_t)s->ncl);
            s->nmasked   = (int*)orc_grow(s->nmasked, sizeof(int) * (size_t)s->ncl);
        }
        s->neigh = (int*)orc_grow(s->neigh, sizeof(int) * (size_t)s->list_rows * ld);
        s->imask = (unsigned*)orc_grow(s->imask, sizeof(unsigned) * (size_t)s->list_rows * ld);
        int newmax = ld, resize = 0;
        for (int ci = 0; ci < s->ncl; ci++) {
            const int ci_cj0 = ci / s->jfac;
            const double* ib = &s->ibb[6 * ci];
            int n = 0, nm = 0;
            int* row     = &s->neigh[(size_t)ci * ld];
            unsigned* mr = &s->imask[(size_t)ci * ld];
            for (int k = 0; k < s->nstencil; k++) {
                const int jb = s->cbin[ci] + s->stencil[k];
                const int* col = &s->jcol[(size_t)jb * s->jcol_cap];
                for (int m = 0; m < s->jcol_count[jb]; m++) {
                    const int cj = col[m];
                    if (half && ci_cj0 > cj) continue;
                    const double* jbx = &s->jbb[6 * cj];
                    double d = orc_bb_axis(ib[4], ib[5], jbx[4], jbx[5]);
                    d        = d * d;
                    double e = orc_bb_axis(ib[2], ib[3], jbx[2], jbx[3]);
                    d += e * e;
                    e = orc_bb_axis(ib[0], ib[1], jbx[0], jbx[1]);
                    d += e * e;
                    if (!(d < s->cutneighsq)) continue;
                    int ok = d < s->rbb_sq;
                    if (!ok) ok = orc_any_pair(s, ci, cj, s->cutneighsq);
                    if (!ok) continue;
                    unsigned im = orc_imask(s, ci, cj);
                    if (n < ld) {
                        if (im == MASK_ALL) {
                            row[n] = cj;
                            mr[n]  = im;
                        } else {
                            row[n]  = row[nm];
                            mr[n]   = mr[nm];
                            row[nm] = cj;
                            mr[nm]  = im;
                            nm++;
                        }
                    }
                    n++;
                }
            }
            s->numneigh[ci] = n;
            s->nmasked[ci]  = nm;
            if (n >= ld) {
                resize = 1;
                if (n > newmax) newmax = n;
            }
        }
        if (!resize) break;
        s->maxneighs = (int)(newmax * 1.2);
    }
    return 0;
}

/* pruneNeighborCPU, clusterpair/neighbor.c:1098-1264: drop j-clusters with no
 * atom pair inside cutneigh (the list's own cutoff), moving the last entry into
 * the freed place */
void orccp_prune_neighbor(OrcCp* s)
{
    const int ld = s->maxneighs;
    for (int ci = 0; ci < s->ncl; ci++) {
        int nn = s->numneigh[ci], nm = s->nmasked[ci], k = 0;
        int* row = &s->neigh[(size_t)ci * ld];
        while (k < nn) {
            int cj = row[k], in_range;
            if (s->p.fma_rsq) {
                in_range = orc_any_pair(s, ci, cj, s->cutneighsq);
            } else {
                /* scalar build: only the real atoms of both clusters */
                in_range = 0;
                for (int a = 0; a < s->inat[ci] && !in_range; a++) {
                    const double* xi = &s->cx[3 * (ci * s->M + a)];
                    for (int b = 0; b < s->jnat[cj]; b++) {
                        const double* xj = &s->cx[3 * (cj * s->N + b)];
                        double dx = xi[0] - xj[0], dy = xi[1] - xj[1], dz = xi[2] - xj[2];
                        if (dx * dx + dy * dy + dz * dz < s->cutneighsq) {
                            in_range = 1;
                            break;
                        }
                    }
                }
            }
            if (in_range) {
                k++;
            } else {
                nn--;
                if (k < nm) nm--;
                row[k] = row[nn];
            }
        }
        s->numneigh[ci] = nn;
        s->nmasked[ci]  = nm;
    }
}

/* ---- force, integrator, atoms -------------------------------------------- */

/* computeForceLJRef, clusterpair/force_lj.c:23-189: per i-cluster, per list
 * entry, per i atom, the sum over the N j atoms is added to the atom's force;
 * exclusion of self pairs (and of the lower triangle for half lists) by the
 * cluster indices; sigma6 and epsilon by geometric mixing of the per-atom
 * sigma^3 and sqrt(epsilon). Half lists subtract the reaction from every j slot
 * (ghost reactions are discarded). The potential energy 4 eps sr6 (sr6 - 1)
 * (not computed by the reference) is summed per pair, halved for full lists. */
double orccp_compute_force(OrcCp* s)
{
    const int M = s->M, N = s->N, half = s->p.half_neigh;
    const double cutforcesq = s->p.cutforce * s->p.cutforce;
    const int nsl           = (s->ncj + s->ngc) * N;
    for (int ci = 0; ci < s->ncl; ci++)
        for (int a = 0; a < s->inat[ci]; a++) {
            double* f = &s->cf[3 * (ci * M + a)];
            f[0] = f[1] = f[2] = 0.0;
        }
    for (int sl = s->ncl * M; sl < nsl; sl++) {
        double* f = &s->cf[3 * sl];
        f[0] = f[1] = f[2] = 0.0;
    }
    double epot = 0.0;
    const int ld = s->maxneighs;
    for (int ci = 0; ci < s->ncl; ci++) {
        const int ci_cj0 = ci / s->jfac;
        for (int k = 0; k < s->numneigh[ci]; k++) {
            const int cj = s->neigh[(size_t)ci * ld + k];
            for (int a = 0; a < M; a++) {
                const int si     = ci * M + a;
                const double* xi = &s->cx[3 * si];
                const int ai     = a + M * (ci % s->jfac); /* position inside j-cluster ci_cj0 */
                double fix = 0, fiy = 0, fiz = 0;
                for (int b = 0; b < N; b++) {
                    int cond = half ? (ci_cj0 != cj || ai < b) : (ci_cj0 != cj || ai != b);
                    if (!cond) continue;
                    const int sj     = cj * N + b;
                    const double* xj = &s->cx[3 * sj];
                    double delx = xi[0] - xj[0];
                    double dely = xi[1] - xj[1];
                    double delz = xi[2] - xj[2];
                    double rsq  = delx * delx + dely * dely + delz * delz;
                    double sigma6 = s->cs3[si] * s->cs3[sj];
                    double eps    = s->cse[si] * s->cse[sj];
                    if (rsq < cutforcesq) {
                        double sr2   = 1.0 / rsq;
                        double sr6   = sr2 * sr2 * sr2 * sigma6;
                        double force = 48.0 * sr6 * (sr6 - 0.5) * sr2 * eps;
                        if (half) {
                            s->cf[3 * sj] -= delx * force;
                            s->cf[3 * sj + 1] -= dely * force;
                            s->cf[3 * sj + 2] -= delz * force;
                        }
                        fix += delx * force;
                        fiy += dely * force;
                        fiz += delz * force;
                        double e = 4.0 * eps * sr6 * (sr6 - 1.0);
                        if (half) {
                            epot += sj < s->ncl * M ? e : 0.5 * e;
                        } else {
                            epot += 0.5 * e;
                        }
                    }
                }
                s->cf[3 * si] += fix;
                s->cf[3 * si + 1] += fiy;
                s->cf[3 * si + 2] += fiz;
            }
        }
    }
    s->epot = epot;
    return epot;
}

/* initialIntegrateCPU, clusterpair/integrate.c:29-61 */
void orccp_initial_integrate(OrcCp* s)
{
    for (int ci = 0; ci < s->ncl; ci++)
        for (int a = 0; a < s->inat[ci]; a++) {
            int sl    = ci * s->M + a;
            double* v = &s->cv[3 * sl];
            double* x = &s->cx[3 * sl];
            double* f = &s->cf[3 * sl];
            v[0] += s->p.dtforce * f[0];
            v[1] += s->p.dtforce * f[1];
            v[2] += s->p.dtforce * f[2];
            x[0] += s->p.dt * v[0];
            x[1] += s->p.dt * v[1];
            x[2] += s->p.dt * v[2];
        }
}

/* finalIntegrateCPU, clusterpair/integrate.c:64-86 */
void orccp_final_integrate(OrcCp* s)
{
    for (int ci = 0; ci < s->ncl; ci++)
        for (int a = 0; a < s->inat[ci]; a++) {
            int sl    = ci * s->M + a;
            double* v = &s->cv[3 * sl];
            double* f = &s->cf[3 * sl];
            v[0] += s->p.dtforce * f[0];
            v[1] += s->p.dtforce * f[1];
            v[2] += s->p.dtforce * f[2];
        }
}

/* updateSingleAtoms, clusterpair/neighbor.c:2096-2149: atoms renumbered in
 * cluster order */
void orccp_update_single_atoms(OrcCp* s)
{
    int n = 0;
    for (int ci = 0; ci < s->ncl; ci++)
        for (int a = 0; a < s->inat[ci]; a++) {
            int sl = ci * s->M + a;
            memcpy(&s->ax[3 * n], &s->cx[3 * sl], sizeof(double) * 3);
            memcpy(&s->av[3 * n], &s->cv[3 * sl], sizeof(double) * 3);
            s->at[n] = s->ct[sl];
            n++;
        }
}

/* updateAtomsPbcCPU, clusterpair/pbc.c:116-143 */
void orccp_update_atoms_pbc(OrcCp* s)
{
    const double prd[3] = {s->p.xprd, s->p.yprd, s->p.zprd};
    for (int i = 0; i < s->nlocal; i++)
        for (int d = 0; d < 3; d++) {
            double* x = &s->ax[3 * i + d];
            if (*x < 0.0) *x += prd[d];
            else if (*x >= prd[d]) *x -= prd[d];
        }
}

int orccp_setup(OrcCp* s)
{
    orc_setup_columns(s);
    if (orccp_build_clusters(s)) return -1;
    orccp_define_jclusters(s);
    orccp_setup_pbc(s);
    orccp_bin_jclusters(s);
    return orccp_build_neighbor(s);
}

/* the timestep of clusterpair/main.c:326-362 without MPI */
void orccp_step(OrcCp* s, int n)
{
    orccp_initial_integrate(s);
    if ((n + 1) % s->p.reneigh_every) {
        if (!((n + 1) % s->p.prune_every)) orccp_prune_neighbor(s);
        orccp_update_pbc(s, 0);
    } else {
        orccp_update_single_atoms(s);
        orccp_update_atoms_pbc(s);
        orccp_build_clusters(s);
        orccp_define_jclusters(s);
        orccp_setup_pbc(s);
        orccp_bin_jclusters(s);
        orccp_build_neighbor(s);
    }
    orccp_compute_force(s);
    orccp_final_integrate(s);
}

/* computeThermo (common/thermo.c:60-100) over the atom arrays */
void orccp_thermo(OrcCp* s, double* T, double* P)
{
    double dof    = (s->p.natoms * 3 - 3);
    double pscale = 1.0 / 3 / s->p.xprd / s->p.yprd / s->p.zprd;
    double t      = 0.0;
    for (int i = 0; i < s->nlocal; i++) {
        const double* v = &s->av[3 * i];
        t += (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) * s->p.mass;
    }
    t  = t * (1.0 / dof);
    *T = t;
    *P = (t * dof) * pscale;
}

void orccp_energy(OrcCp* s, double* KE, double* PE)
{
    double t = 0.0;
    for (int ci = 0; ci < s->ncl; ci++)
        for (int a = 0; a < s->inat[ci]; a++) {
            const double* v = &s->cv[3 * (ci * s->M + a)];
            t += (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) * s->p.mass;
        }
    if (KE) *KE = 0.5 * t;
    if (PE) *PE = s->epot;
}

/* ---- getters ------------------------------------------------------------- */

void orccp_counts(OrcCp* s, int* c)
{
    c[0] = s->nlocal;
    c[1] = s->p.natoms;
    c[2] = s->ncl;
    c[3] = s->ncj;
    c[4] = s->ngc;
    c[5] = s->nghost_atoms;
    c[6] = s->dummy;
    c[7] = s->maxneighs;
}

void orccp_get_atoms(OrcCp* s, double* x, double* v, int* type)
{
    if (x) memcpy(x, s->ax, sizeof(double) * 3 * (size_t)s->nlocal);
    if (v) memcpy(v, s->av, sizeof(double) * 3 * (size_t)s->nlocal);
    if (type) memcpy(type, s->at, sizeof(int) * (size_t)s->nlocal);
}

void orccp_get_slots(OrcCp* s, double* x, double* v, double* f, int* type, int nslots)
{
    int nloc = s->ncl * s->M;
    for (int sl = 0; sl < nslots; sl++) {
        if (x) memcpy(&x[3 * sl], &s->cx[3 * sl], sizeof(double) * 3);
        if (type) type[sl] = s->ct[sl];
        if (sl < nloc) {
            if (v) memcpy(&v[3 * sl], &s->cv[3 * sl], sizeof(double) * 3);
            if (f) memcpy(&f[3 * sl], &s->cf[3 * sl], sizeof(double) * 3);
        }
    }
}

void orccp_set_slots(OrcCp* s, const double* x, const double* v)
{
    int nloc = s->ncl * s->M;
    for (int ci = 0; ci < s->ncl; ci++)
        for (int a = 0; a < s->inat[ci]; a++) {
            int sl = ci * s->M + a;
            if (x) memcpy(&s->cx[3 * sl], &x[3 * sl], sizeof(double) * 3);
            if (v) memcpy(&s->cv[3 * sl], &v[3 * sl], sizeof(double) * 3);
        }
    (void)nloc;
}

void orccp_get_iclusters(OrcCp* s, int* natoms, int* bin, double* bb)
{
    memcpy(natoms, s->inat, sizeof(int) * (size_t)s->ncl);
    if (bin) memcpy(bin, s->cbin, sizeof(int) * (size_t)s->ncl);
    if (bb) memcpy(bb, s->ibb, sizeof(double) * 6 * (size_t)s->ncl);
}

void orccp_get_jclusters(OrcCp* s, int* natoms, double* bb, int count)
{
    memcpy(natoms, s->jnat, sizeof(int) * (size_t)count);
    if (bb) memcpy(bb, s->jbb, sizeof(double) * 6 * (size_t)count);
}

void orccp_get_ghosts(OrcCp* s, int* border_map, int* pbc)
{
    memcpy(border_map, s->border, sizeof(int) * (size_t)s->ngc);
    memcpy(pbc, s->pbc, sizeof(int) * 3 * (size_t)s->ngc);
}

void orccp_get_list(OrcCp* s, int* numneigh, int* nmasked, int* neighbors, unsigned* imask,
    int ld)
{
    for (int ci = 0; ci < s->ncl; ci++) {
        int nn       = s->numneigh[ci];
        numneigh[ci] = nn;
        if (nmasked) nmasked[ci] = s->nmasked[ci];
        for (int k = 0; k < nn && k < ld; k++) {
            neighbors[(size_t)ci * ld + k] = s->neigh[(size_t)ci * s->maxneighs + k];
            if (imask) imask[(size_t)ci * ld + k] = s->imask[(size_t)ci * s->maxneighs + k];
        }
    }
}

void orccp_bin_geometry(OrcCp* s, int* ints, double* dbls, int* stencil)
{
    ints[0] = s->nbinx;
    ints[1] = s->nbiny;
    ints[2] = s->mbinx;
    ints[3] = s->mbiny;
    ints[4] = s->mbinxlo;
    ints[5] = s->mbinylo;
    ints[6] = s->nstencil;
    dbls[0] = s->binsizex;
    dbls[1] = s->binsizey;
    dbls[2] = s->rbb_sq;
    if (stencil) memcpy(stencil, s->stencil, sizeof(int) * (size_t)s->nstencil);
}

int orccp_get_columns(OrcCp* s, int* start, int* list, int cap)
{
    int n = 0;
    for (int b = 0; b <= s->mbins; b++) {
        start[b] = n;
        if (b == s->mbins) break;
        for (int i = 0; i < s->jcol_count[b]; i++) {
            if (n < cap) list[n] = s->jcol[(size_t)b * s->jcol_cap + i];
            n++;
        }
    }
    return n;
}
