/*
 * CPU oracle for the MD-Bench Verlet-list timestep (LJ full/half, EAM).
 *
 * TEST INFRASTRUCTURE ONLY (see mdb_oracle.h). Each function below names the
 * reference file:line it restates; paths are relative to the MD-Bench tree.
 * Single-threaded on purpose: the reference's half-list kernel races under
 * OpenMP (verletlist/force_lj.c:183-187), and a fixed summation order keeps
 * this oracle deterministic.
 */
#include "mdb_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define ORC_MAX(a, b) ((a) > (b) ? (a) : (b))
#define ORC_MIN(a, b) ((a) < (b) ? (a) : (b))

typedef struct {
    int nrho, nr;
    double drho, dr, cut, mass;
    double *frho, *rhor, *zr;
} OrcFuncfl;

struct OrcSys {
    OrcParams p;
    double* eps_t;   /* per-type epsilon (ntypes) */
    double* sig_t;   /* per-type sigma (ntypes) */
    /* derived parameters */
    double lattice, xprd, yprd, zprd, cutneigh, dtforce, mass, dt, cutforce;
    double temp;
    /* type-pair tables (geometric rule, common/parameter.c:48-71) */
    int ntypes;
    double *epsilon, *sigma6, *cutforcesq, *cutneighsq;
    /* atoms: AoS x/v/f, capacity nmax */
    int natoms, nlocal, nghost, nmax;
    double *x, *v, *f;
    int* type;
    /* ghosts */
    int nmaxghost;
    int *border_map, *pbcx, *pbcy, *pbcz;
    /* binning (verletlist/neighbor.c:29-45) */
    int nbinx, nbiny, nbinz, mbinx, mbiny, mbinz, pad_x, pad_y, pad_z;
    double binsizex, binsizey, binsizez, bininvx, bininvy, bininvz;
    int nstencil;
    int* stencil;
    int mbins, atoms_per_bin;
    int *bincount, *bins;
    /* neighbor list, AoS rows of maxneighs */
    int maxneighs, listcap;
    int *numneigh, *neighbors;
    /* thermo constants (common/thermo.c:35-58) */
    double mvv2e, dof_boltz, t_scale, p_scale;
    double epot;
    /* EAM */
    int has_eam;
    OrcFuncfl file;
    int eam_nrho, eam_nr, nrho_tot, nr_tot;
    double eam_dr, eam_rdr, eam_drho, eam_rdrho;
    double *frho, *rhor, *z2r;
    double *frho_spline, *rhor_spline, *z2r_spline;
    double *fp, *rho;
    int resort_every; /* SORT_ATOMS builds: sortAtom period (0: never) */
};

/* ------------------------------------------------------------------------- */
/* Park-Miller minimal standard generator, common/util.c:24-33.               */
static double orc_myrandom(int* seed)
{
    const int ia = 16807, im = 2147483647, iq = 127773, ir = 2836;
    int k  = (*seed) / iq;
    *seed  = ia * (*seed - k * iq) - ir * k;
    if (*seed < 0) *seed += im;
    return (1.0 / im) * (*seed);
}

static void* orc_alloc(size_t n)
{
    void* p = calloc(1, n ? n : 1);
    if (!p) {
        fprintf(stderr, "oracle: out of memory\n");
        abort();
    }
    return p;
}

static void orc_grow_atoms(OrcSys* s, int need)
{
    if (need <= s->nmax) return;
    int nmax = s->nmax;
    while (nmax < need)
        nmax += 20000; /* verletlist/atom.c:20 DELTA */
    s->x    = realloc(s->x, sizeof(double) * 3 * nmax);
    s->v    = realloc(s->v, sizeof(double) * 3 * nmax);
    s->f    = realloc(s->f, sizeof(double) * 3 * nmax);
    s->type = realloc(s->type, sizeof(int) * nmax);
    memset(s->x + 3 * s->nmax, 0, sizeof(double) * 3 * (nmax - s->nmax));
    memset(s->v + 3 * s->nmax, 0, sizeof(double) * 3 * (nmax - s->nmax));
    memset(s->f + 3 * s->nmax, 0, sizeof(double) * 3 * (nmax - s->nmax));
    memset(s->type + s->nmax, 0, sizeof(int) * (nmax - s->nmax));
    s->nmax = nmax;
}

OrcSys* orc_create(const OrcParams* p)
{
    OrcSys* s = orc_alloc(sizeof(OrcSys));
    s->p      = *p;
    s->ntypes = p->ntypes > 0 ? p->ntypes : 1;
    s->eps_t  = orc_alloc(sizeof(double) * s->ntypes);
    s->sig_t  = orc_alloc(sizeof(double) * s->ntypes);
    for (int t = 0; t < s->ntypes; t++) {
        s->eps_t[t] = p->epsilon_per_type ? p->epsilon_per_type[t] : p->epsilon;
        s->sig_t[t] = p->sigma_per_type ? p->sigma_per_type[t] : p->sigma;
    }
    s->p.epsilon_per_type = NULL;
    s->p.sigma_per_type   = NULL;
    s->dt                 = p->dt;
    s->mass               = p->mass;
    s->cutforce           = p->cutforce;
    s->temp               = p->temp;
    s->maxneighs          = 100; /* verletlist/neighbor.c:76 */
    s->atoms_per_bin      = 8;   /* verletlist/neighbor.c:72 */
    return s;
}

void orc_destroy(OrcSys* s)
{
    if (!s) return;
    free(s->eps_t);
    free(s->sig_t);
    free(s->epsilon);
    free(s->sigma6);
    free(s->cutforcesq);
    free(s->cutneighsq);
    free(s->x);
    free(s->v);
    free(s->f);
    free(s->type);
    free(s->border_map);
    free(s->pbcx);
    free(s->pbcy);
    free(s->pbcz);
    free(s->stencil);
    free(s->bincount);
    free(s->bins);
    free(s->numneigh);
    free(s->neighbors);
    free(s->file.frho);
    free(s->file.rhor);
    free(s->file.zr);
    free(s->frho);
    free(s->rhor);
    free(s->z2r);
    free(s->frho_spline);
    free(s->rhor_spline);
    free(s->z2r_spline);
    free(s->fp);
    free(s->rho);
    free(s);
}

/* ------------------------------------------------------------------------- */
/* EAM: common/eam_utils.c:42-284                                              */
static int orc_readline(char* line, int n, FILE* fp) { return fgets(line, n, fp) != NULL; }

static void orc_grab(FILE* fp, int n, double* list)
{
    /* common/eam_utils.c:286-299 */
    char line[4096];
    int i = 0;
    while (i < n && orc_readline(line, sizeof line, fp)) {
        char* tok = strtok(line, " \t\n\r\f");
        while (tok && i < n) {
            list[i++] = atof(tok);
            tok       = strtok(NULL, " \t\n\r\f");
        }
    }
}

static void orc_interpolate(int n, double delta, const double* f, double* spline)
{
    /* common/eam_utils.c:253-284 */
    for (int m = 1; m <= n; m++)
        spline[m * 7 + 6] = f[m];
    spline[1 * 7 + 5]       = spline[2 * 7 + 6] - spline[1 * 7 + 6];
    spline[2 * 7 + 5]       = 0.5 * (spline[3 * 7 + 6] - spline[1 * 7 + 6]);
    spline[(n - 1) * 7 + 5] = 0.5 * (spline[n * 7 + 6] - spline[(n - 2) * 7 + 6]);
    spline[n * 7 + 5]       = spline[n * 7 + 6] - spline[(n - 1) * 7 + 6];
    for (int m = 3; m <= n - 2; m++)
        spline[m * 7 + 5] = ((spline[(m - 2) * 7 + 6] - spline[(m + 2) * 7 + 6]) +
                                8.0 * (spline[(m + 1) * 7 + 6] - spline[(m - 1) * 7 + 6])) /
                            12.0;
    for (int m = 1; m <= n - 1; m++) {
        spline[m * 7 + 4] = 3.0 * (spline[(m + 1) * 7 + 6] - spline[m * 7 + 6]) -
                            2.0 * spline[m * 7 + 5] - spline[(m + 1) * 7 + 5];
        spline[m * 7 + 3] = spline[m * 7 + 5] + spline[(m + 1) * 7 + 5] -
                            2.0 * (spline[(m + 1) * 7 + 6] - spline[m * 7 + 6]);
    }
    spline[n * 7 + 4] = 0.0;
    spline[n * 7 + 3] = 0.0;
    for (int m = 1; m <= n; m++) {
        spline[m * 7 + 2] = spline[m * 7 + 5] / delta;
        spline[m * 7 + 1] = 2.0 * spline[m * 7 + 4] / delta;
        spline[m * 7 + 0] = 3.0 * spline[m * 7 + 3] / delta;
    }
}

/* 4-point Lagrange resample of one funcfl array onto the common grid,
 * common/eam_utils.c:95-112 (the same stencil is used three times there). */
static double orc_lagrange(const double* arr, int nfile, double dfile, double r)
{
    const double sixth = 1.0 / 6.0;
    double p           = r / dfile + 1.0;
    int k              = (int)(p);
    k                  = ORC_MIN(k, nfile - 2);
    k                  = ORC_MAX(k, 2);
    p -= k;
    p           = ORC_MIN(p, 2.0);
    double cof1 = -sixth * p * (p - 1.0) * (p - 2.0);
    double cof2 = 0.5 * (p * p - 1.0) * (p - 2.0);
    double cof3 = -0.5 * p * (p + 1.0) * (p - 2.0);
    double cof4 = sixth * p * (p * p - 1.0);
    return cof1 * arr[k - 1] + cof2 * arr[k] + cof3 * arr[k + 1] + cof4 * arr[k + 2];
}

int orc_load_eam(OrcSys* s, const char* path)
{
    /* readEamFile, common/eam_utils.c:42-85 */
    FILE* fp = fopen(path, "r");
    if (!fp) return -1;
    char line[4096];
    int tmp;
    OrcFuncfl* file = &s->file;
    if (!orc_readline(line, sizeof line, fp)) goto bad;
    if (!orc_readline(line, sizeof line, fp)) goto bad;
    if (sscanf(line, "%d %lg", &tmp, &file->mass) != 2) goto bad;
    if (!orc_readline(line, sizeof line, fp)) goto bad;
    if (sscanf(line, "%d %lg %d %lg %lg", &file->nrho, &file->drho, &file->nr, &file->dr,
            &file->cut) != 5)
        goto bad;
    file->frho = orc_alloc(sizeof(double) * (file->nrho + 1));
    file->rhor = orc_alloc(sizeof(double) * (file->nr + 1));
    file->zr   = orc_alloc(sizeof(double) * (file->nr + 1));
    orc_grab(fp, file->nrho, file->frho);
    orc_grab(fp, file->nr, file->zr);
    orc_grab(fp, file->nr, file->rhor);
    for (int i = file->nrho; i > 0; i--)
        file->frho[i] = file->frho[i - 1];
    for (int i = file->nr; i > 0; i--)
        file->rhor[i] = file->rhor[i - 1];
    for (int i = file->nr; i > 0; i--)
        file->zr[i] = file->zr[i - 1];
    fclose(fp);

    /* file2array, common/eam_utils.c:87-222 (one funcfl file) */
    double rmax = 0.0, rhomax = 0.0;
    s->eam_dr   = ORC_MAX(0.0, file->dr);
    s->eam_drho = ORC_MAX(0.0, file->drho);
    rmax        = ORC_MAX(rmax, (file->nr - 1) * file->dr);
    rhomax      = ORC_MAX(rhomax, (file->nrho - 1) * file->drho);
    s->eam_nr   = (int)(rmax / s->eam_dr + 0.5);
    s->eam_nrho = (int)(rhomax / s->eam_drho + 0.5);
    s->frho     = orc_alloc(sizeof(double) * (s->eam_nrho + 1));
    for (int m = 1; m <= s->eam_nrho; m++)
        s->frho[m] = orc_lagrange(file->frho, file->nrho, file->drho, (m - 1) * s->eam_drho);
    s->rhor = orc_alloc(sizeof(double) * (s->eam_nr + 1));
    for (int m = 1; m <= s->eam_nr; m++)
        s->rhor[m] = orc_lagrange(file->rhor, file->nr, file->dr, (m - 1) * s->eam_dr);
    s->z2r = orc_alloc(sizeof(double) * (s->eam_nr + 1));
    for (int m = 1; m <= s->eam_nr; m++) {
        double r   = (m - 1) * s->eam_dr;
        double zri = orc_lagrange(file->zr, file->nr, file->dr, r);
        double zrj = orc_lagrange(file->zr, file->nr, file->dr, r);
        s->z2r[m]  = 27.2 * 0.529 * zri * zrj;
    }

    /* array2spline, common/eam_utils.c:224-251 (tables are identical for every
     * type pair, so one copy serves all type indices) */
    s->eam_rdr   = 1.0 / s->eam_dr;
    s->eam_rdrho = 1.0 / s->eam_drho;
    s->nrho_tot  = (s->eam_nrho + 1) * 7 + 64;
    s->nr_tot    = (s->eam_nr + 1) * 7 + 64;
    s->nrho_tot -= s->nrho_tot % 64;
    s->nr_tot -= s->nr_tot % 64;
    s->frho_spline = orc_alloc(sizeof(double) * s->nrho_tot);
    s->rhor_spline = orc_alloc(sizeof(double) * s->nr_tot);
    s->z2r_spline  = orc_alloc(sizeof(double) * s->nr_tot);
    orc_interpolate(s->eam_nrho, s->eam_drho, s->frho, s->frho_spline);
    orc_interpolate(s->eam_nr, s->eam_dr, s->rhor, s->rhor_spline);
    orc_interpolate(s->eam_nr, s->eam_dr, s->z2r, s->z2r_spline);

    /* initEam parameter overrides, common/eam_utils.c:29-35 */
    s->has_eam  = 1;
    s->mass     = file->mass;
    s->cutforce = file->cut;
    s->temp     = 600.0;
    s->dt       = 0.001;
    s->p.rho    = 0.07041125;
    return 0;
bad:
    fclose(fp);
    return -2;
}

int orc_eam_info(OrcSys* s, int* nrho, int* nr, int* nrho_tot, int* nr_tot, double* drho,
    double* dr, double* cut, double* mass)
{
    if (!s->has_eam) return -1;
    *nrho     = s->eam_nrho;
    *nr       = s->eam_nr;
    *nrho_tot = s->nrho_tot;
    *nr_tot   = s->nr_tot;
    *drho     = s->eam_drho;
    *dr       = s->eam_dr;
    *cut      = s->file.cut;
    *mass     = s->file.mass;
    return 0;
}

void orc_eam_tables(OrcSys* s, double* frho_spline, double* rhor_spline, double* z2r_spline)
{
    memcpy(frho_spline, s->frho_spline, sizeof(double) * s->nrho_tot);
    memcpy(rhor_spline, s->rhor_spline, sizeof(double) * s->nr_tot);
    memcpy(z2r_spline, s->z2r_spline, sizeof(double) * s->nr_tot);
}

/* ------------------------------------------------------------------------- */
/* Type tables: computePerTypeLJParameters + computeTypePairLJParameters,
 * common/parameter.c:31-71, with cutoffs from verletlist/atom.c:150-153.      */
static void orc_type_tables(OrcSys* s, int ntypes)
{
    free(s->epsilon);
    free(s->sigma6);
    free(s->cutforcesq);
    free(s->cutneighsq);
    s->epsilon    = orc_alloc(sizeof(double) * ntypes * ntypes);
    s->sigma6     = orc_alloc(sizeof(double) * ntypes * ntypes);
    s->cutforcesq = orc_alloc(sizeof(double) * ntypes * ntypes);
    s->cutneighsq = orc_alloc(sizeof(double) * ntypes * ntypes);
    for (int i = 0; i < ntypes; i++) {
        for (int j = 0; j < ntypes; j++) {
            double ei = i < s->p.ntypes ? s->eps_t[i] : s->p.epsilon;
            double ej = j < s->p.ntypes ? s->eps_t[j] : s->p.epsilon;
            double si = i < s->p.ntypes ? s->sig_t[i] : s->p.sigma;
            double sj = j < s->p.ntypes ? s->sig_t[j] : s->p.sigma;
            double s3i = si * si * si, s3j = sj * sj * sj;
            s->epsilon[i * ntypes + j]    = sqrt(ei) * sqrt(ej);
            s->sigma6[i * ntypes + j]     = s3i * s3j;
            s->cutneighsq[i * ntypes + j] = s->cutneigh * s->cutneigh;
            s->cutforcesq[i * ntypes + j] = s->cutforce * s->cutforce;
        }
    }
    s->ntypes = ntypes;
}

static void orc_setup_thermo(OrcSys* s)
{
    /* common/thermo.c:35-58 */
    if (s->p.force_field == 0) {
        s->mvv2e     = 1.0;
        s->dof_boltz = (s->natoms * 3 - 3);
        s->t_scale   = s->mvv2e / s->dof_boltz;
        s->p_scale   = 1.0 / 3 / s->xprd / s->yprd / s->zprd;
    } else {
        s->mvv2e     = 1.036427e-04;
        s->dof_boltz = (s->natoms * 3 - 3) * 8.617343e-05;
        s->t_scale   = s->mvv2e / s->dof_boltz;
        s->p_scale   = 1.602176e+06 / 3 / s->xprd / s->yprd / s->zprd;
        s->dtforce /= s->mvv2e;
    }
}

static void orc_adjust_thermo(OrcSys* s)
{
    /* common/thermo.c:102-159 */
    double vxtot = 0.0, vytot = 0.0, vztot = 0.0;
    for (int i = 0; i < s->nlocal; i++) {
        vxtot += s->v[3 * i + 0];
        vytot += s->v[3 * i + 1];
        vztot += s->v[3 * i + 2];
    }
    vxtot = vxtot / s->natoms;
    vytot = vytot / s->natoms;
    vztot = vztot / s->natoms;
    for (int i = 0; i < s->nlocal; i++) {
        s->v[3 * i + 0] -= vxtot;
        s->v[3 * i + 1] -= vytot;
        s->v[3 * i + 2] -= vztot;
    }
    double t = 0.0;
    for (int i = 0; i < s->nlocal; i++) {
        const double* vi = &s->v[3 * i];
        t += (vi[0] * vi[0] + vi[1] * vi[1] + vi[2] * vi[2]) * s->mass;
    }
    t *= s->t_scale;
    double factor = sqrt(s->temp / t);
    for (int i = 0; i < s->nlocal; i++) {
        s->v[3 * i + 0] *= factor;
        s->v[3 * i + 1] *= factor;
        s->v[3 * i + 2] *= factor;
    }
}

static void orc_common_params(OrcSys* s)
{
    /* verletlist/main.c:54-62 and :305 */
    s->cutneigh = s->cutforce + s->p.skin;
    if (s->has_eam) s->cutneigh = s->cutforce + 1.0; /* common/eam_utils.c:31 */
    s->lattice = pow((4.0 / s->p.rho), (1.0 / 3.0));
    if (!s->p.from_file) {
        s->xprd = s->p.nx * s->lattice;
        s->yprd = s->p.ny * s->lattice;
        s->zprd = s->p.nz * s->lattice;
    } else {
        s->xprd = s->p.xprd;
        s->yprd = s->p.yprd;
        s->zprd = s->p.zprd;
    }
    s->dtforce = 0.5 * s->dt;
    if (s->has_eam) s->dtforce = 0.5 * s->dt / s->mass; /* common/eam_utils.c:35 */
}

int orc_lattice(OrcSys* s)
{
    /* createAtom, verletlist/atom.c:104-246 */
    orc_common_params(s);
    orc_type_tables(s, s->p.ntypes);
    const double xlo = 0.0, ylo = 0.0, zlo = 0.0;
    const double xhi = s->xprd, yhi = s->yprd, zhi = s->zprd;
    const int nx = s->p.nx, ny = s->p.ny, nz = s->p.nz;
    s->natoms   = 4 * nx * ny * nz;
    s->nlocal   = 0;
    double alat = pow((4.0 / s->p.rho), (1.0 / 3.0));
    int ilo     = (int)(xlo / (0.5 * alat) - 1);
    int ihi     = (int)(xhi / (0.5 * alat) + 1);
    int jlo     = (int)(ylo / (0.5 * alat) - 1);
    int jhi     = (int)(yhi / (0.5 * alat) + 1);
    int klo     = (int)(zlo / (0.5 * alat) - 1);
    int khi     = (int)(zhi / (0.5 * alat) + 1);
    ilo         = ORC_MAX(ilo, 0);
    ihi         = ORC_MIN(ihi, 2 * nx - 1);
    jlo         = ORC_MAX(jlo, 0);
    jhi         = ORC_MIN(jhi, 2 * ny - 1);
    klo         = ORC_MAX(klo, 0);
    khi         = ORC_MIN(khi, 2 * nz - 1);

    srand(1); /* the reference draws types from glibc rand() in its default state */
    int sx = 0, sy = 0, sz = 0, ox = 0, oy = 0, oz = 0;
    const int sub = 8;
    while (oz * sub <= khi) {
        int k = oz * sub + sz;
        int j = oy * sub + sy;
        int i = ox * sub + sx;
        if (((i + j + k) % 2 == 0) && (i >= ilo) && (i <= ihi) && (j >= jlo) && (j <= jhi) &&
            (k >= klo) && (k <= khi)) {
            double xt = 0.5 * alat * i;
            double yt = 0.5 * alat * j;
            double zt = 0.5 * alat * k;
            if (xt >= xlo && xt < xhi && yt >= ylo && yt < yhi && zt >= zlo && zt < zhi) {
                int n = k * (2 * ny) * (2 * nx) + j * (2 * nx) + i + 1;
                double vv[3];
                for (int d = 0; d < 3; d++) {
                    for (int m = 0; m < 5; m++)
                        orc_myrandom(&n);
                    vv[d] = orc_myrandom(&n);
                }
                orc_grow_atoms(s, s->nlocal + 1);
                int idx              = s->nlocal;
                s->x[3 * idx + 0]    = xt;
                s->x[3 * idx + 1]    = yt;
                s->x[3 * idx + 2]    = zt;
                s->v[3 * idx + 0]    = vv[0];
                s->v[3 * idx + 1]    = vv[1];
                s->v[3 * idx + 2]    = vv[2];
                s->type[idx]         = rand() % s->p.ntypes;
                s->nlocal++;
            }
        }
        sx++;
        if (sx == sub) { sx = 0; sy++; }
        if (sy == sub) { sy = 0; sz++; }
        if (sz == sub) { sz = 0; ox++; }
        if (ox * sub > ihi) { ox = 0; oy++; }
        if (oy * sub > jhi) { oy = 0; oz++; }
    }
    orc_setup_thermo(s);
    orc_adjust_thermo(s);
    return s->nlocal;
}

int orc_set_atoms(OrcSys* s, int n, const double* x, const double* v, const int* type)
{
    /* readAtom_dmp, verletlist/atom.c:529-656: types are taken as given and the
     * type table spans max(type)+1 entries; no thermo adjustment follows
     * (verletlist/main.c:88-90). */
    orc_common_params(s);
    orc_grow_atoms(s, n + 1);
    int ntypes = 0;
    for (int i = 0; i < n; i++) {
        memcpy(&s->x[3 * i], &x[3 * i], 3 * sizeof(double));
        memcpy(&s->v[3 * i], &v[3 * i], 3 * sizeof(double));
        s->type[i] = type[i];
        ntypes     = ORC_MAX(type[i] + 1, ntypes);
    }
    s->natoms = s->nlocal = n;
    orc_type_tables(s, ntypes);
    orc_setup_thermo(s);
    return n;
}

/* ------------------------------------------------------------------------- */
/* Binning, verletlist/neighbor.c:62-258 and :355-400.                         */
static double orc_bindist(OrcSys* s, int i, int j, int k)
{
    double dx, dy, dz;
    if (i > 0) dx = (i - 1) * s->binsizex;
    else if (i == 0) dx = 0.0;
    else dx = (i + 1) * s->binsizex;
    if (j > 0) dy = (j - 1) * s->binsizey;
    else if (j == 0) dy = 0.0;
    else dy = (j + 1) * s->binsizey;
    if (k > 0) dz = (k - 1) * s->binsizez;
    else if (k == 0) dz = 0.0;
    else dz = (k + 1) * s->binsizez;
    return (dx * dx + dy * dy + dz * dz);
}

static int orc_coord2bin(OrcSys* s, double xin, double yin, double zin)
{
    const double eps = 1e-9;
    double xlo       = fabs(0.0 - s->pad_x * s->binsizex) + eps;
    double ylo       = fabs(0.0 - s->pad_y * s->binsizey) + eps;
    double zlo       = fabs(0.0 - s->pad_z * s->binsizez) + eps;
    int ix           = (int)((xin + xlo) * s->bininvx);
    int iy           = (int)((yin + ylo) * s->bininvy);
    int iz           = (int)((zin + zlo) * s->bininvz);
    return (iz * s->mbiny * s->mbinx + iy * s->mbinx + ix);
}

static void orc_setup_neighbor(OrcSys* s)
{
    const double factor = 0.999;
    double cutneigh     = s->cutneigh;
    double cutneighsq   = cutneigh * cutneigh;
    if (s->p.from_file) {
        s->binsizex = cutneigh * 0.5;
        s->binsizey = cutneigh * 0.5;
        s->binsizez = cutneigh * 0.5;
        s->nbinx    = (int)(s->xprd / s->binsizex);
        s->nbiny    = (int)(s->yprd / s->binsizey);
        s->nbinz    = (int)(s->zprd / s->binsizez);
        if (s->nbinx == 0) s->nbinx = 1;
        if (s->nbiny == 0) s->nbiny = 1;
        if (s->nbinz == 0) s->nbinz = 1;
        s->bininvx = s->nbinx / s->xprd;
        s->bininvy = s->nbiny / s->yprd;
        s->bininvz = s->nbinz / s->zprd;
    } else {
        const double neighscale = 5.0 / 6.0;
        double bx               = neighscale * s->p.nx;
        double by               = neighscale * s->p.ny;
        double bz               = neighscale * s->p.nz;
        s->nbinx                = (int)(1 > bx ? 1 : bx);
        s->nbiny                = (int)(1 > by ? 1 : by);
        s->nbinz                = (int)(1 > bz ? 1 : bz);
        s->binsizex             = s->xprd / s->nbinx;
        s->binsizey             = s->yprd / s->nbiny;
        s->binsizez             = s->zprd / s->nbinz;
        s->bininvx              = 1.0 / s->binsizex;
        s->bininvy              = 1.0 / s->binsizey;
        s->bininvz              = 1.0 / s->binsizez;
    }
    /* pad is incremented in two loops (neighbor.c:151-158 and :200-216) */
    s->pad_x = (int)(cutneigh * s->bininvx);
    while (s->pad_x * s->binsizex < factor * cutneigh)
        s->pad_x++;
    s->pad_y = (int)(cutneigh * s->bininvy);
    while (s->pad_y * s->binsizey < factor * cutneigh)
        s->pad_y++;
    s->pad_z = (int)(cutneigh * s->bininvz);
    while (s->pad_z * s->binsizez < factor * cutneigh)
        s->pad_z++;
    int nextx = (int)(cutneigh * s->bininvx);
    while (nextx * s->binsizex < factor * cutneigh) {
        nextx++;
        s->pad_x++;
    }
    int nexty = (int)(cutneigh * s->bininvy);
    while (nexty * s->binsizey < factor * cutneigh) {
        nexty++;
        s->pad_y++;
    }
    int nextz = (int)(cutneigh * s->bininvz);
    while (nextz * s->binsizez < factor * cutneigh) {
        nextz++;
        s->pad_z++;
    }
    s->mbinx = ORC_MAX(1, s->nbinx + 4 * s->pad_x);
    s->mbiny = ORC_MAX(1, s->nbiny + 4 * s->pad_y);
    s->mbinz = ORC_MAX(1, s->nbinz + 4 * s->pad_z);
    free(s->stencil);
    s->stencil  = orc_alloc(sizeof(int) * (2 * nextz + 1) * (2 * nexty + 1) * (2 * nextx + 1));
    s->nstencil = 0;
    for (int k = -nextz; k <= nextz; k++)
        for (int j = -nexty; j <= nexty; j++)
            for (int i = -nextx; i <= nextx; i++)
                if (orc_bindist(s, i, j, k) < cutneighsq)
                    s->stencil[s->nstencil++] = k * s->mbiny * s->mbinx + j * s->mbinx + i;
    s->mbins = s->mbinx * s->mbiny * s->mbinz;
    free(s->bincount);
    free(s->bins);
    s->bincount = orc_alloc(sizeof(int) * s->mbins);
    s->bins     = orc_alloc(sizeof(int) * s->mbins * s->atoms_per_bin);
}

static void orc_binatoms(OrcSys* s)
{
    /* verletlist/neighbor.c:431-464 */
    int nall   = s->nlocal + s->nghost;
    int resize = 1;
    while (resize) {
        resize = 0;
        memset(s->bincount, 0, sizeof(int) * s->mbins);
        for (int i = 0; i < nall; i++) {
            int ib = orc_coord2bin(s, s->x[3 * i], s->x[3 * i + 1], s->x[3 * i + 2]);
            if (ib < 0 || ib >= s->mbins) {
                fprintf(stderr, "oracle: atom %d outside the bin grid\n", i);
                abort();
            }
            if (s->bincount[ib] < s->atoms_per_bin) {
                int ac                                = s->bincount[ib]++;
                s->bins[ib * s->atoms_per_bin + ac] = i;
            } else {
                resize = 1;
            }
        }
        if (resize) {
            free(s->bins);
            s->atoms_per_bin *= 2;
            s->bins = orc_alloc(sizeof(int) * s->mbins * s->atoms_per_bin);
        }
    }
}

int orc_build_neighbor(OrcSys* s)
{
    /* buildNeighborCPU, verletlist/neighbor.c:260-352 (full shell, no half stencil) */
    int nall = s->nlocal + s->nghost;
    if (s->listcap < nall * s->maxneighs) {
        free(s->numneigh);
        free(s->neighbors);
        s->numneigh  = orc_alloc(sizeof(int) * nall);
        s->neighbors = orc_alloc(sizeof(int) * (size_t)nall * s->maxneighs);
        s->listcap   = nall * s->maxneighs;
    }
    orc_binatoms(s);
    int resize = 1;
    while (resize) {
        int new_maxneighs = s->maxneighs;
        resize            = 0;
        for (int i = 0; i < s->nlocal; i++) {
            int n       = 0;
            double xtmp = s->x[3 * i], ytmp = s->x[3 * i + 1], ztmp = s->x[3 * i + 2];
            int ibin    = orc_coord2bin(s, xtmp, ytmp, ztmp);
            int type_i  = s->type[i];
            int* row    = &s->neighbors[(size_t)i * s->maxneighs];
            for (int k = 0; k < s->nstencil; k++) {
                int jbin = ibin + s->stencil[k];
                int* loc = &s->bins[jbin * s->atoms_per_bin];
                for (int m = 0; m < s->bincount[jbin]; m++) {
                    int j = loc[m];
                    if (i == j) continue;
                    if (s->p.half_neigh && j < i) continue;
                    double delx = xtmp - s->x[3 * j];
                    double dely = ytmp - s->x[3 * j + 1];
                    double delz = ztmp - s->x[3 * j + 2];
                    double rsq  = delx * delx + dely * dely + delz * delz;
                    double cut  = s->cutneighsq[type_i * s->ntypes + s->type[j]];
                    if (rsq <= cut) {
                        if (n < s->maxneighs) row[n] = j;
                        n++;
                    }
                }
            }
            s->numneigh[i] = n;
            if (n >= s->maxneighs) {
                resize = 1;
                if (n > new_maxneighs) new_maxneighs = n;
            }
        }
        if (resize) {
            s->maxneighs = new_maxneighs * 1.2;
            free(s->neighbors);
            s->neighbors = orc_alloc(sizeof(int) * (size_t)nall * s->maxneighs);
            s->listcap   = nall * s->maxneighs;
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* PBC, verletlist/pbc.c:42-232                                               */
void orc_update_atoms_pbc(OrcSys* s)
{
    for (int i = 0; i < s->nlocal; i++) {
        double* xi = &s->x[3 * i];
        if (xi[0] < 0.0) xi[0] += s->xprd;
        else if (xi[0] >= s->xprd) xi[0] -= s->xprd;
        if (xi[1] < 0.0) xi[1] += s->yprd;
        else if (xi[1] >= s->yprd) xi[1] -= s->yprd;
        if (xi[2] < 0.0) xi[2] += s->zprd;
        else if (xi[2] >= s->zprd) xi[2] -= s->zprd;
    }
}

void orc_update_pbc(OrcSys* s)
{
    int nl = s->nlocal;
    for (int g = 0; g < s->nghost; g++) {
        int b                  = s->border_map[g];
        s->x[3 * (nl + g) + 0] = s->x[3 * b + 0] + s->pbcx[g] * s->xprd;
        s->x[3 * (nl + g) + 1] = s->x[3 * b + 1] + s->pbcy[g] * s->yprd;
        s->x[3 * (nl + g) + 2] = s->x[3 * b + 2] + s->pbcz[g] * s->zprd;
    }
}

static void orc_addghost(OrcSys* s, int* ng, int i, int dx, int dy, int dz)
{
    int g = (*ng)++;
    if (g >= s->nmaxghost) {
        int nm         = s->nmaxghost + 20000;
        s->border_map  = realloc(s->border_map, sizeof(int) * nm);
        s->pbcx        = realloc(s->pbcx, sizeof(int) * nm);
        s->pbcy        = realloc(s->pbcy, sizeof(int) * nm);
        s->pbcz        = realloc(s->pbcz, sizeof(int) * nm);
        s->nmaxghost   = nm;
    }
    orc_grow_atoms(s, s->nlocal + g + 1);
    s->border_map[g]       = i;
    s->pbcx[g]             = dx;
    s->pbcy[g]             = dy;
    s->pbcz[g]             = dz;
    s->type[s->nlocal + g] = s->type[i];
}

int orc_setup_pbc(OrcSys* s)
{
    int ng          = 0;
    const double c  = s->cutneigh;
    const double xp = s->xprd, yp = s->yprd, zp = s->zprd;
    const int px = s->p.pbc_x, py = s->p.pbc_y, pz = s->p.pbc_z;
    for (int i = 0; i < s->nlocal; i++) {
        double x = s->x[3 * i], y = s->x[3 * i + 1], z = s->x[3 * i + 2];
        /* 6 planes */
        if (px) {
            if (x < c) orc_addghost(s, &ng, i, +1, 0, 0);
            if (x >= (xp - c)) orc_addghost(s, &ng, i, -1, 0, 0);
        }
        if (py) {
            if (y < c) orc_addghost(s, &ng, i, 0, +1, 0);
            if (y >= (yp - c)) orc_addghost(s, &ng, i, 0, -1, 0);
        }
        if (pz) {
            if (z < c) orc_addghost(s, &ng, i, 0, 0, +1);
            if (z >= (zp - c)) orc_addghost(s, &ng, i, 0, 0, -1);
        }
        /* 8 corners */
        if (px && py && pz) {
            if (x < c && y < c && z < c) orc_addghost(s, &ng, i, +1, +1, +1);
            if (x < c && y >= (yp - c) && z < c) orc_addghost(s, &ng, i, +1, -1, +1);
            if (x < c && y < c && z >= (zp - c)) orc_addghost(s, &ng, i, +1, +1, -1);
            if (x < c && y >= (yp - c) && z >= (zp - c)) orc_addghost(s, &ng, i, +1, -1, -1);
            if (x >= (xp - c) && y < c && z < c) orc_addghost(s, &ng, i, -1, +1, +1);
            if (x >= (xp - c) && y >= (yp - c) && z < c) orc_addghost(s, &ng, i, -1, -1, +1);
            if (x >= (xp - c) && y < c && z >= (zp - c)) orc_addghost(s, &ng, i, -1, +1, -1);
            if (x >= (xp - c) && y >= (yp - c) && z >= (zp - c))
                orc_addghost(s, &ng, i, -1, -1, -1);
        }
        /* 12 edges */
        if (px && pz) {
            if (x < c && z < c) orc_addghost(s, &ng, i, +1, 0, +1);
            if (x < c && z >= (zp - c)) orc_addghost(s, &ng, i, +1, 0, -1);
            if (x >= (xp - c) && z < c) orc_addghost(s, &ng, i, -1, 0, +1);
            if (x >= (xp - c) && z >= (zp - c)) orc_addghost(s, &ng, i, -1, 0, -1);
        }
        if (py && pz) {
            if (y < c && z < c) orc_addghost(s, &ng, i, 0, +1, +1);
            if (y < c && z >= (zp - c)) orc_addghost(s, &ng, i, 0, +1, -1);
            if (y >= (yp - c) && z < c) orc_addghost(s, &ng, i, 0, -1, +1);
            if (y >= (yp - c) && z >= (zp - c)) orc_addghost(s, &ng, i, 0, -1, -1);
        }
        if (px && py) {
            if (y < c && x < c) orc_addghost(s, &ng, i, +1, +1, 0);
            if (y < c && x >= (xp - c)) orc_addghost(s, &ng, i, -1, +1, 0);
            if (y >= (yp - c) && x < c) orc_addghost(s, &ng, i, +1, -1, 0);
            if (y >= (yp - c) && x >= (xp - c)) orc_addghost(s, &ng, i, -1, -1, 0);
        }
    }
    s->nghost = ng;
    return ng;
}

/* ------------------------------------------------------------------------- */
/* Forces                                                                     */
static double orc_force_lj(OrcSys* s)
{
    /* computeForceLJFullNeigh / computeForceLJHalfNeigh, verletlist/force_lj.c:17-206.
     * The potential energy is not computed by the reference; it is accumulated
     * here from the same sr6 as 4*eps*sr6*(sr6-1) per pair (unshifted), halved
     * for pairs that are visited twice. */
    int nl       = s->nlocal;
    int half     = s->p.half_neigh;
    int nzero    = half ? nl + s->nghost : nl;
    double epot  = 0.0;
    memset(s->f, 0, sizeof(double) * 3 * nzero);
    for (int i = 0; i < nl; i++) {
        int nn      = s->numneigh[i];
        double xtmp = s->x[3 * i], ytmp = s->x[3 * i + 1], ztmp = s->x[3 * i + 2];
        double fix = 0, fiy = 0, fiz = 0;
        int type_i = s->type[i];
        const int* row = &s->neighbors[(size_t)i * s->maxneighs];
        for (int k = 0; k < nn; k++) {
            int j        = row[k];
            double delx  = xtmp - s->x[3 * j];
            double dely  = ytmp - s->x[3 * j + 1];
            double delz  = ztmp - s->x[3 * j + 2];
            double rsq   = delx * delx + dely * dely + delz * delz;
            int tij      = type_i * s->ntypes + s->type[j];
            double cutsq = s->cutforcesq[tij];
            double sig6  = s->sigma6[tij];
            double eps   = s->epsilon[tij];
            if (rsq < cutsq) {
                double sr2   = 1.0 / rsq;
                double sr6   = sr2 * sr2 * sr2 * sig6;
                double force = 48.0 * sr6 * (sr6 - 0.5) * sr2 * eps;
                fix += delx * force;
                fiy += dely * force;
                fiz += delz * force;
                double e = 4.0 * eps * sr6 * (sr6 - 1.0);
                if (half && j < nl) {
                    s->f[3 * j + 0] -= delx * force;
                    s->f[3 * j + 1] -= dely * force;
                    s->f[3 * j + 2] -= delz * force;
                    epot += e;
                } else {
                    epot += 0.5 * e;
                }
            }
        }
        s->f[3 * i + 0] += fix;
        s->f[3 * i + 1] += fiy;
        s->f[3 * i + 2] += fiz;
    }
    return epot;
}

static double orc_force_eam(OrcSys* s)
{
    /* computeForceEam, verletlist/force_eam.c:19-228 (one element; every type
     * pair indexes an identical table copy). The embedding energy F(rho_i) and
     * the pair energy phi = z2/r use the value coefficients 3..6 of the same
     * splines; they are not computed by the reference. */
    int nl  = s->nlocal;
    int cap = s->nmax;
    free(s->fp);
    free(s->rho);
    s->fp  = orc_alloc(sizeof(double) * cap);
    s->rho = orc_alloc(sizeof(double) * cap);
    const double* rs = s->rhor_spline;
    const double* fs = s->frho_spline;
    const double* zs = s->z2r_spline;
    const double rdr = s->eam_rdr, rdrho = s->eam_rdrho;
    const int nr = s->eam_nr, nrho = s->eam_nrho;
    double epot = 0.0;
    for (int i = 0; i < nl; i++) {
        int nn      = s->numneigh[i];
        double xtmp = s->x[3 * i], ytmp = s->x[3 * i + 1], ztmp = s->x[3 * i + 2];
        double rhoi = 0;
        int type_i  = s->type[i];
        const int* row = &s->neighbors[(size_t)i * s->maxneighs];
        for (int k = 0; k < nn; k++) {
            int j       = row[k];
            double delx = xtmp - s->x[3 * j];
            double dely = ytmp - s->x[3 * j + 1];
            double delz = ztmp - s->x[3 * j + 2];
            double rsq  = delx * delx + dely * dely + delz * delz;
            if (rsq < s->cutforcesq[type_i * s->ntypes + s->type[j]]) {
                double p = sqrt(rsq) * rdr + 1.0;
                int m    = (int)(p);
                m        = m < nr - 1 ? m : nr - 1;
                p -= m;
                p = p < 1.0 ? p : 1.0;
                rhoi += ((rs[m * 7 + 3] * p + rs[m * 7 + 4]) * p + rs[m * 7 + 5]) * p +
                        rs[m * 7 + 6];
            }
        }
        double p = 1.0 * rhoi * rdrho + 1.0;
        int m    = (int)(p);
        m        = ORC_MAX(1, ORC_MIN(m, nrho - 1));
        p -= m;
        p         = ORC_MIN(p, 1.0);
        s->fp[i]  = (fs[m * 7 + 0] * p + fs[m * 7 + 1]) * p + fs[m * 7 + 2];
        s->rho[i] = rhoi;
        epot += ((fs[m * 7 + 3] * p + fs[m * 7 + 4]) * p + fs[m * 7 + 5]) * p + fs[m * 7 + 6];
    }
    for (int g = 0; g < s->nghost; g++)
        s->fp[nl + g] = s->fp[s->border_map[g]];
    for (int i = 0; i < nl; i++) {
        int nn      = s->numneigh[i];
        double xtmp = s->x[3 * i], ytmp = s->x[3 * i + 1], ztmp = s->x[3 * i + 2];
        double fix = 0, fiy = 0, fiz = 0;
        int type_i = s->type[i];
        const int* row = &s->neighbors[(size_t)i * s->maxneighs];
        for (int k = 0; k < nn; k++) {
            int j       = row[k];
            double delx = xtmp - s->x[3 * j];
            double dely = ytmp - s->x[3 * j + 1];
            double delz = ztmp - s->x[3 * j + 2];
            double rsq  = delx * delx + dely * dely + delz * delz;
            if (rsq < s->cutforcesq[type_i * s->ntypes + s->type[j]]) {
                double r = sqrt(rsq);
                double p = r * rdr + 1.0;
                int m    = (int)(p);
                m        = m < nr - 1 ? m : nr - 1;
                p -= m;
                p = p < 1.0 ? p : 1.0;
                double rhoip = (rs[m * 7 + 0] * p + rs[m * 7 + 1]) * p + rs[m * 7 + 2];
                double z2p   = (zs[m * 7 + 0] * p + zs[m * 7 + 1]) * p + zs[m * 7 + 2];
                double z2 = ((zs[m * 7 + 3] * p + zs[m * 7 + 4]) * p + zs[m * 7 + 5]) * p +
                            zs[m * 7 + 6];
                double recip = 1.0 / r;
                double phi   = z2 * recip;
                double phip  = z2p * recip - phi * recip;
                double psip  = s->fp[i] * rhoip + s->fp[j] * rhoip + phip;
                double fpair = -psip * recip;
                fix += delx * fpair;
                fiy += dely * fpair;
                fiz += delz * fpair;
                epot += 0.5 * phi;
            }
        }
        s->f[3 * i + 0] = fix;
        s->f[3 * i + 1] = fiy;
        s->f[3 * i + 2] = fiz;
    }
    return epot;
}

double orc_compute_force(OrcSys* s)
{
    s->epot = s->p.force_field == 1 ? orc_force_eam(s) : orc_force_lj(s);
    return s->epot;
}

/* ------------------------------------------------------------------------- */
/* Integrator, verletlist/integrate.c:21-42                                    */
void orc_initial_integrate(OrcSys* s)
{
    for (int i = 0; i < s->nlocal; i++) {
        double *x = &s->x[3 * i], *v = &s->v[3 * i], *f = &s->f[3 * i];
        v[0] += s->dtforce * f[0];
        v[1] += s->dtforce * f[1];
        v[2] += s->dtforce * f[2];
        x[0] = x[0] + s->dt * v[0];
        x[1] = x[1] + s->dt * v[1];
        x[2] = x[2] + s->dt * v[2];
    }
}

void orc_final_integrate(OrcSys* s)
{
    for (int i = 0; i < s->nlocal; i++) {
        double *v = &s->v[3 * i], *f = &s->f[3 * i];
        v[0] += s->dtforce * f[0];
        v[1] += s->dtforce * f[1];
        v[2] += s->dtforce * f[2];
    }
}

/* ------------------------------------------------------------------------- */
int orc_setup(OrcSys* s)
{
    /* verletlist/main.c:46-113 tail: setupNeighbor, setupPbc, updatePbc,
     * buildNeighbor (thermo was set up by orc_lattice / orc_set_atoms). */
    orc_setup_neighbor(s);
    orc_setup_pbc(s);
    orc_update_pbc(s);
    return orc_build_neighbor(s);
}

void orc_sort_atoms(OrcSys* s)
{
    /* sortAtom, verletlist/neighbor.c:466-536: no ghosts, binatoms, then the
     * atoms bin by bin (each bin's atoms in index order). The reference
     * rewrites positions and velocities only; types and forces move here too. */
    s->nghost = 0;
    orc_binatoms(s);
    const int n = s->nlocal;
    double* nx  = orc_alloc(sizeof(double) * 3 * (size_t)s->nmax);
    double* nv  = orc_alloc(sizeof(double) * 3 * (size_t)s->nmax);
    double* nf  = orc_alloc(sizeof(double) * 3 * (size_t)s->nmax);
    int* nt     = orc_alloc(sizeof(int) * (size_t)s->nmax);
    int k       = 0;
    for (int b = 0; b < s->mbins; b++)
        for (int c = 0; c < s->bincount[b]; c++, k++) {
            const int o = s->bins[b * s->atoms_per_bin + c];
            for (int d = 0; d < 3; d++) {
                nx[3 * k + d] = s->x[3 * o + d];
                nv[3 * k + d] = s->v[3 * o + d];
                nf[3 * k + d] = s->f[3 * o + d];
            }
            nt[k] = s->type[o];
        }
    if (k != n) {
        fprintf(stderr, "oracle: sort lost atoms (%d of %d)\n", k, n);
        abort();
    }
    free(s->x);
    free(s->v);
    free(s->f);
    free(s->type);
    s->x    = nx;
    s->v    = nv;
    s->f    = nf;
    s->type = nt;
}

void orc_set_resort(OrcSys* s, int every) { s->resort_every = every > 0 ? every : 0; }

void orc_set_list(OrcSys* s, const int* numneigh, const int* neighbors, int ld)
{
    /* the stub benchmark's createNeighbors (verletlist/main-stub.c:60-113)
     * hands computeForce a list of locals with no ghosts */
    const int n = s->nlocal;
    s->nghost   = 0;
    free(s->numneigh);
    free(s->neighbors);
    s->numneigh  = orc_alloc(sizeof(int) * (size_t)(n + 1));
    s->neighbors = orc_alloc(sizeof(int) * (size_t)n * (size_t)ld + 1);
    s->maxneighs = ld;
    s->listcap   = n * ld;
    memcpy(s->numneigh, numneigh, sizeof(int) * (size_t)n);
    memcpy(s->neighbors, neighbors, sizeof(int) * (size_t)n * (size_t)ld);
}

void orc_step(OrcSys* s, int n)
{
    /* verletlist/main.c:371-419 (no MPI: forward/reverse reduce to updatePbc);
     * SORT_ATOMS: sortAtom first (main.c:372-381), and the step rebuilds */
    const int resort = s->resort_every > 0 && (n + 1) % s->resort_every == 0;
    int reneigh      = resort || (n + 1) % s->p.reneigh_every == 0;
    if (resort) orc_sort_atoms(s);
    orc_initial_integrate(s);
    if (reneigh) {
        orc_update_atoms_pbc(s);
        orc_setup_pbc(s);
        orc_update_pbc(s);
        orc_build_neighbor(s);
    } else {
        orc_update_pbc(s);
    }
    orc_compute_force(s);
    orc_final_integrate(s);
}

void orc_thermo(OrcSys* s, double* T, double* P, double* KE, double* PE)
{
    /* computeThermo, common/thermo.c:60-100; KE = 1/2 sum m v^2 * mvv2e */
    double t = 0.0;
    for (int i = 0; i < s->nlocal; i++) {
        const double* v = &s->v[3 * i];
        t += (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) * s->mass;
    }
    double ke = 0.5 * t * s->mvv2e;
    t         = t * s->t_scale;
    if (T) *T = t;
    if (P) *P = (t * s->dof_boltz) * s->p_scale;
    if (KE) *KE = ke;
    if (PE) *PE = s->epot;
}

int orc_nlocal(OrcSys* s) { return s->nlocal; }
int orc_nghost(OrcSys* s) { return s->nghost; }
int orc_maxneighs(OrcSys* s) { return s->maxneighs; }

void orc_get_atoms(OrcSys* s, double* x, double* v, double* f, int* type)
{
    if (x) memcpy(x, s->x, sizeof(double) * 3 * s->nlocal);
    if (v) memcpy(v, s->v, sizeof(double) * 3 * s->nlocal);
    if (f) memcpy(f, s->f, sizeof(double) * 3 * s->nlocal);
    if (type) memcpy(type, s->type, sizeof(int) * (s->nlocal + s->nghost));
}

void orc_get_positions_all(OrcSys* s, double* x)
{
    memcpy(x, s->x, sizeof(double) * 3 * (s->nlocal + s->nghost));
}

void orc_set_state(OrcSys* s, const double* x, const double* v)
{
    if (x) memcpy(s->x, x, sizeof(double) * 3 * s->nlocal);
    if (v) memcpy(s->v, v, sizeof(double) * 3 * s->nlocal);
}

void orc_get_ghosts(OrcSys* s, int* border_map, int* pbc_xyz)
{
    for (int g = 0; g < s->nghost; g++) {
        if (border_map) border_map[g] = s->border_map[g];
        if (pbc_xyz) {
            pbc_xyz[3 * g + 0] = s->pbcx[g];
            pbc_xyz[3 * g + 1] = s->pbcy[g];
            pbc_xyz[3 * g + 2] = s->pbcz[g];
        }
    }
}

void orc_get_list(OrcSys* s, int* numneigh, int* neighbors, int ld)
{
    for (int i = 0; i < s->nlocal; i++) {
        int nn      = s->numneigh[i];
        numneigh[i] = nn;
        if (neighbors)
            for (int k = 0; k < nn && k < ld; k++)
                neighbors[(size_t)i * ld + k] = s->neighbors[(size_t)i * s->maxneighs + k];
    }
}

void orc_get_eam_fp(OrcSys* s, double* fp)
{
    if (s->fp) memcpy(fp, s->fp, sizeof(double) * (s->nlocal + s->nghost));
}

void orc_bin_geometry(OrcSys* s, int* ints, double* dbls, int* stencil)
{
    int iv[10] = { s->nbinx, s->nbiny, s->nbinz, s->mbinx, s->mbiny, s->mbinz, s->pad_x,
        s->pad_y, s->pad_z, s->nstencil };
    double dv[7] = { s->binsizex, s->binsizey, s->binsizez, s->bininvx, s->bininvy,
        s->bininvz, s->cutneigh };
    if (ints) memcpy(ints, iv, sizeof iv);
    if (dbls) memcpy(dbls, dv, sizeof dv);
    if (stencil) memcpy(stencil, s->stencil, sizeof(int) * s->nstencil);
}

void orc_get_params(OrcSys* s, double* d)
{
    d[0] = s->xprd;
    d[1] = s->yprd;
    d[2] = s->zprd;
    d[3] = s->dt;
    d[4] = s->dtforce;
    d[5] = s->mass;
    d[6] = s->cutforce;
    d[7] = s->cutneigh;
}
