/*
 * Host-side setup for libmdb (see include/mdb_host.h). Compiled with
 * -ffp-contract=off so that the generated lattice and velocities are the
 * reference's to the last bit.
 */
#include "mdb_host.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define HMAX(a, b) ((a) > (b) ? (a) : (b))
#define HMIN(a, b) ((a) < (b) ? (a) : (b))

void mdbh_defaults(MdbHostParams* p)
{
    memset(p, 0, sizeof *p);
    p->force_field   = MDB_FF_LJ;
    p->precision     = MDB_PREC_FP64;
    p->epsilon       = 1.0;
    p->sigma         = 1.0;
    p->rho           = 0.8442;
    p->ntypes        = 4;
    p->ntimes        = 200;
    p->dt            = 0.005;
    p->nx = p->ny = p->nz = 32;
    p->pbc_x = p->pbc_y = p->pbc_z = 1;
    p->cutforce      = 2.5;
    p->skin          = 0.3;
    p->temp          = 1.44;
    p->nstat         = 100;
    p->mass          = 1.0;
    p->reneigh_every = 20;
}

static char* trim_comment(char* line)
{
    char* h = strchr(line, '#');
    if (h) *h = '\0';
    return line;
}

int mdbh_read_types(MdbHostParams* p, const char* path)
{
    FILE* fp = fopen(path, "r");
    if (!fp) return MDB_ERR_ARG;
    char line[4096];
    int t = 0;
    while (fgets(line, sizeof line, fp)) {
        char* save = NULL;
        char* e    = strtok_r(trim_comment(line), " \t\n\r", &save);
        if (!e) continue;
        char* s = strtok_r(NULL, " \t\n\r", &save);
        if (!s || t >= MDBH_MAX_TYPES) {
            fclose(fp);
            return MDB_ERR_ARG;
        }
        p->epsilon_per_type[t] = atof(e);
        p->sigma_per_type[t]   = atof(s);
        t++;
    }
    fclose(fp);
    if (t == 0) return MDB_ERR_ARG;
    p->ntypes    = t;
    p->has_types = 1;
    return MDB_OK;
}

int mdbh_read_params(MdbHostParams* p, const char* path)
{
    FILE* fp = fopen(path, "r");
    if (!fp) return MDB_ERR_ARG;
    char line[4096];
    char types_file[4096] = { 0 };
    int explicit_lj       = 0;
    while (fgets(line, sizeof line, fp)) {
        char* save = NULL;
        char* key  = strtok_r(trim_comment(line), " \t\n\r", &save);
        char* val  = key ? strtok_r(NULL, " \t\n\r", &save) : NULL;
        if (!key || !val) continue;
#define RP(name, conv)                                                                  \
    if (strcmp(key, #name) == 0) {                                                      \
        p->name = conv(val);                                                            \
        continue;                                                                       \
    }
        if (strcmp(key, "force_field") == 0) {
            p->force_field = strncmp(val, "eam", 3) == 0 ? MDB_FF_EAM : MDB_FF_LJ;
            continue;
        }
        if (strcmp(key, "types_file") == 0) {
            snprintf(types_file, sizeof types_file, "%s", val);
            continue;
        }
        if (!strcmp(key, "epsilon") || !strcmp(key, "sigma") || !strcmp(key, "ntypes"))
            explicit_lj = 1;
        RP(epsilon, atof)
        RP(sigma, atof)
        RP(rho, atof)
        RP(dt, atof)
        RP(cutforce, atof)
        RP(skin, atof)
        RP(temp, atof)
        RP(mass, atof)
        RP(ntypes, atoi)
        RP(ntimes, atoi)
        RP(nx, atoi)
        RP(ny, atoi)
        RP(nz, atoi)
        RP(pbc_x, atoi)
        RP(pbc_y, atoi)
        RP(pbc_z, atoi)
        RP(nstat, atoi)
        RP(reneigh_every, atoi)
        RP(half_neigh, atoi)
#undef RP
    }
    fclose(fp);
    /* common/parameter.c:262-273: a types file excludes epsilon/sigma/ntypes */
    if (types_file[0]) {
        if (explicit_lj) return MDB_ERR_ARG;
        return mdbh_read_types(p, types_file);
    }
    return MDB_OK;
}

void mdbh_apply_eam(MdbHostParams* p, const MdbEamTables* t)
{
    p->force_field = MDB_FF_EAM;
    p->mass        = t->mass;
    p->cutforce    = t->cut;
    p->temp        = 600.0;
    p->dt          = 0.001;
    p->rho         = 0.07041125;
}

void mdbh_finalize(MdbHostParams* p)
{
    p->lattice = pow((4.0 / p->rho), (1.0 / 3.0));
    if (!p->from_file) {
        p->xprd = p->nx * p->lattice;
        p->yprd = p->ny * p->lattice;
        p->zprd = p->nz * p->lattice;
    }
    if (p->force_field == MDB_FF_EAM) {
        p->cutneigh = p->cutforce + 1.0;                /* common/eam_utils.c:31 */
        p->dtforce  = 0.5 * p->dt / p->mass;            /* common/eam_utils.c:35 */
        p->dtforce /= 1.036427e-04;                     /* common/thermo.c:56 */
    } else {
        p->cutneigh = p->cutforce + p->skin;            /* verletlist/main.c:305 */
        p->dtforce  = 0.5 * p->dt;                      /* common/parameter.c:276 */
    }
}

/* Park-Miller minimal standard generator (Schrage), common/util.c:24-33. */
static double park_miller(int* seed)
{
    const int a = 16807, m = 2147483647, q = 127773, r = 2836;
    int k       = (*seed) / q;
    *seed       = a * (*seed - k * q) - r * k;
    if (*seed < 0) *seed += m;
    return (1.0 / m) * (*seed);
}

int mdbh_create_fcc(const MdbHostParams* p, double** xo, double** vo, int** to)
{
    const int nx = p->nx, ny = p->ny, nz = p->nz;
    if (nx < 1 || ny < 1 || nz < 1 || p->ntypes < 1) return -MDB_ERR_ARG;
    long long natoms = 4LL * nx * ny * nz;
    if (natoms > 0x7fffffffLL) return -MDB_ERR_ARG;
    double* x = malloc(sizeof(double) * 3 * natoms);
    double* v = malloc(sizeof(double) * 3 * natoms);
    int* type = malloc(sizeof(int) * natoms);
    if (!x || !v || !type) {
        free(x);
        free(v);
        free(type);
        return -MDB_ERR_NOMEM;
    }
    const double xhi = p->xprd, yhi = p->yprd, zhi = p->zprd;
    double alat      = pow((4.0 / p->rho), (1.0 / 3.0));
    int ilo = HMAX((int)(0.0 / (0.5 * alat) - 1), 0);
    int ihi = HMIN((int)(xhi / (0.5 * alat) + 1), 2 * nx - 1);
    int jlo = HMAX((int)(0.0 / (0.5 * alat) - 1), 0);
    int jhi = HMIN((int)(yhi / (0.5 * alat) + 1), 2 * ny - 1);
    int klo = HMAX((int)(0.0 / (0.5 * alat) - 1), 0);
    int khi = HMIN((int)(zhi / (0.5 * alat) + 1), 2 * nz - 1);

    /* traversal in 8x8x8 sub-boxes, verletlist/atom.c:170-245 */
    srand(1);
    int n = 0, sx = 0, sy = 0, sz = 0, ox = 0, oy = 0, oz = 0;
    const int sub = 8;
    while (oz * sub <= khi) {
        int k = oz * sub + sz, j = oy * sub + sy, i = ox * sub + sx;
        if (((i + j + k) % 2 == 0) && i >= ilo && i <= ihi && j >= jlo && j <= jhi && k >= klo &&
            k <= khi) {
            double xt = 0.5 * alat * i, yt = 0.5 * alat * j, zt = 0.5 * alat * k;
            if (xt >= 0.0 && xt < xhi && yt >= 0.0 && yt < yhi && zt >= 0.0 && zt < zhi &&
                n < natoms) {
                int seed = k * (2 * ny) * (2 * nx) + j * (2 * nx) + i + 1;
                for (int d = 0; d < 3; d++) {
                    for (int m = 0; m < 5; m++)
                        park_miller(&seed);
                    v[3 * n + d] = park_miller(&seed);
                }
                x[3 * n + 0] = xt;
                x[3 * n + 1] = yt;
                x[3 * n + 2] = zt;
                type[n]      = rand() % p->ntypes;
                n++;
            }
        }
        if (++sx == sub) { sx = 0; sy++; }
        if (sy == sub) { sy = 0; sz++; }
        if (sz == sub) { sz = 0; ox++; }
        if (ox * sub > ihi) { ox = 0; oy++; }
        if (oy * sub > jhi) { oy = 0; oz++; }
    }

    /* adjustThermo: remove centre-of-mass motion, rescale to temp */
    double mvv2e = p->force_field == MDB_FF_EAM ? 1.036427e-04 : 1.0;
    double dof   = p->force_field == MDB_FF_EAM ? (natoms * 3 - 3) * 8.617343e-05
                                                : (double)(natoms * 3 - 3);
    double t_scale = mvv2e / dof;
    double vt[3]   = { 0.0, 0.0, 0.0 };
    for (int i = 0; i < n; i++)
        for (int d = 0; d < 3; d++)
            vt[d] += v[3 * i + d];
    for (int d = 0; d < 3; d++)
        vt[d] = vt[d] / natoms;
    for (int i = 0; i < n; i++)
        for (int d = 0; d < 3; d++)
            v[3 * i + d] -= vt[d];
    double t = 0.0;
    for (int i = 0; i < n; i++)
        t += (v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2]) *
             p->mass;
    t *= t_scale;
    double factor = sqrt(p->temp / t);
    for (int i = 0; i < 3 * n; i++)
        v[i] *= factor;
    *xo = x;
    *vo = v;
    *to = type;
    return n;
}

int mdbh_read_dmp(MdbHostParams* p, const char* path, double** xo, double** vo, int** to)
{
    FILE* fp = fopen(path, "r");
    if (!fp) return -MDB_ERR_ARG;
    char line[4096];
    int natoms = 0, read = 0, have_ts = 0;
    double lo[3] = { 0, 0, 0 }, hi[3] = { 0, 0, 0 };
    double *x = NULL, *v = NULL;
    int* type = NULL;
    int bad   = 0;
    while (!bad && fgets(line, sizeof line, fp)) {
        if (strncmp(line, "ITEM: ", 6) != 0) {
            bad = 1;
            break;
        }
        const char* item = line + 6;
        if (strncmp(item, "TIMESTEP", 8) == 0) {
            bad     = !fgets(line, sizeof line, fp);
            have_ts = 1;
        } else if (strncmp(item, "NUMBER OF ATOMS", 15) == 0) {
            bad    = !fgets(line, sizeof line, fp);
            natoms = atoi(line);
            if (natoms <= 0) bad = 1;
        } else if (strncmp(item, "BOX BOUNDS pp pp pp", 19) == 0) {
            for (int d = 0; d < 3 && !bad; d++) {
                if (!fgets(line, sizeof line, fp) || sscanf(line, "%lf %lf", &lo[d], &hi[d]) != 2)
                    bad = 1;
            }
        } else if (strncmp(item, "ATOMS id type x y z vx vy vz", 28) == 0) {
            if (natoms <= 0) {
                bad = 1;
                break;
            }
            x    = calloc(3 * (size_t)natoms, sizeof(double));
            v    = calloc(3 * (size_t)natoms, sizeof(double));
            type = calloc((size_t)natoms, sizeof(int));
            for (int i = 0; i < natoms && !bad; i++) {
                int id, t;
                double a[6];
                if (!fgets(line, sizeof line, fp) ||
                    sscanf(line, "%d %d %lf %lf %lf %lf %lf %lf", &id, &t, &a[0], &a[1], &a[2],
                        &a[3], &a[4], &a[5]) != 8 ||
                    id < 1 || id > natoms) {
                    bad = 1;
                    break;
                }
                id--;
                type[id] = t;
                for (int d = 0; d < 3; d++) {
                    x[3 * id + d] = a[d];
                    v[3 * id + d] = a[3 + d];
                }
                read++;
            }
            break;
        } else {
            bad = 1;
        }
    }
    fclose(fp);
    if (bad || !have_ts || read != natoms) {
        free(x);
        free(v);
        free(type);
        return -MDB_ERR_ARG;
    }
    p->xprd      = hi[0] - lo[0];
    p->yprd      = hi[1] - lo[1];
    p->zprd      = hi[2] - lo[2];
    p->from_file = 1;
    *xo          = x;
    *vo          = v;
    *to          = type;
    return natoms;
}

int mdbh_write_dmp(const char* path, int n, const double* x, const double* v, const int* type,
    double xprd, double yprd, double zprd)
{
    FILE* fp = fopen(path, "w");
    if (!fp) return MDB_ERR_ARG;
    fprintf(fp, "ITEM: TIMESTEP\n0\nITEM: NUMBER OF ATOMS\n%d\nITEM: BOX BOUNDS pp pp pp\n", n);
    fprintf(fp, "0.0 %.17g\n0.0 %.17g\n0.0 %.17g\n", xprd, yprd, zprd);
    fprintf(fp, "ITEM: ATOMS id type x y z vx vy vz\n");
    for (int i = 0; i < n; i++)
        fprintf(fp, "%d %d %.17g %.17g %.17g %.17g %.17g %.17g\n", i + 1, type[i], x[3 * i],
            x[3 * i + 1], x[3 * i + 2], v[3 * i], v[3 * i + 1], v[3 * i + 2]);
    return fclose(fp) == 0 ? MDB_OK : MDB_ERR_ARG;
}

/* ---- other input formats (readAtom, verletlist/atom.c:260-760) -------------- */

/* growable atom arrays of the readers */
typedef struct {
    int n, cap;
    double *x, *v;
    int* type;
} HostAtoms;

static int ha_reserve(HostAtoms* a, int need)
{
    if (need <= a->cap) return 1;
    int cap = a->cap ? a->cap : 1024;
    while (cap < need) cap *= 2;
    double* x = realloc(a->x, sizeof(double) * 3 * (size_t)cap);
    if (x) a->x = x;
    double* v = realloc(a->v, sizeof(double) * 3 * (size_t)cap);
    if (v) a->v = v;
    int* t = realloc(a->type, sizeof(int) * (size_t)cap);
    if (t) a->type = t;
    if (!x || !v || !t) return 0;
    memset(a->x + 3 * (size_t)a->cap, 0, sizeof(double) * 3 * (size_t)(cap - a->cap));
    memset(a->v + 3 * (size_t)a->cap, 0, sizeof(double) * 3 * (size_t)(cap - a->cap));
    memset(a->type + a->cap, 0, sizeof(int) * (size_t)(cap - a->cap));
    a->cap = cap;
    return 1;
}

static void ha_free(HostAtoms* a)
{
    free(a->x);
    free(a->v);
    free(a->type);
    memset(a, 0, sizeof *a);
}

static int ha_finish(HostAtoms* a, MdbHostParams* p, double** x, double** v, int** type)
{
    int tmax = 0;
    for (int i = 0; i < a->n; i++) tmax = HMAX(tmax, a->type[i]);
    p->ntypes    = tmax + 1; /* atom->ntypes = max type + 1 */
    p->from_file = 1;
    *x           = a->x;
    *v           = a->v;
    *type        = a->type;
    return a->n;
}

/* the readers split lines at single spaces as strtok(line, " ") does */
static char* next_tok(char** save) { return strtok_r(NULL, " ", save); }

/* type names: only argon is known (type_str2int, verletlist/atom.c:248-258) */
static int type_of_name(const char* name)
{
    return (name && strncmp(name, "Ar", 2) == 0) ? 0 : -1;
}

int mdbh_read_pdb(MdbHostParams* p, const char* path, double** x, double** v, int** type)
{
    /* readAtom_pdb, verletlist/atom.c:296-410: CRYST1 gives the box (lower
     * corner at the origin); ATOM lines: serial, name, residue, residue id,
     * x y z, occupancy, charge; velocities zero */
    FILE* fp = fopen(path, "r");
    if (!fp) return -MDB_ERR_ARG;
    char line[4096];
    HostAtoms a = { 0 };
    int bad     = 0;
    while (!bad && fgets(line, sizeof line, fp)) {
        char* save = NULL;
        char* item = strtok_r(line, " ", &save);
        if (!item) continue;
        if (!strncmp(item, "CRYST1", 6)) {
            char *a1 = next_tok(&save), *a2 = next_tok(&save), *a3 = next_tok(&save);
            if (!a1 || !a2 || !a3) {
                bad = 1;
                break;
            }
            p->xprd = atof(a1);
            p->yprd = atof(a2);
            p->zprd = atof(a3);
        } else if (!strncmp(item, "ATOM", 4)) {
            char* f[9];
            for (int k = 0; k < 9; k++) f[k] = next_tok(&save);
            if (!f[8]) {
                bad = 1;
                break;
            }
            const int id = atoi(f[0]) - 1;
            const int t  = type_of_name(f[1]);
            if (id < 0 || t < 0 || !ha_reserve(&a, id + 2)) {
                bad = 1;
                break;
            }
            a.type[id] = t;
            for (int d = 0; d < 3; d++) {
                a.x[3 * id + d] = atof(f[4 + d]);
                a.v[3 * id + d] = 0.0;
            }
            a.n++;
        } else if (strncmp(item, "HEADER", 6) && strncmp(item, "REMARK", 6) &&
                   strncmp(item, "MODEL", 5) && strncmp(item, "TER", 3) &&
                   strncmp(item, "ENDMDL", 6)) {
            bad = 1; /* the reference stops on any other record */
        }
    }
    fclose(fp);
    if (bad || a.n == 0) {
        ha_free(&a);
        return -MDB_ERR_ARG;
    }
    return ha_finish(&a, p, x, v, type);
}

int mdbh_read_gro(MdbHostParams* p, const char* path, double** x, double** v, int** type)
{
    /* readAtom_gro, verletlist/atom.c:412-527: title, atom count, one line per
     * atom (residue+name, atom name, number, x y z, vx vy vz; atoms stored in
     * file order), then the box line */
    FILE* fp = fopen(path, "r");
    if (!fp) return -MDB_ERR_ARG;
    char line[4096];
    HostAtoms a = { 0 };
    int bad = 0, want = 0;
    if (!fgets(line, sizeof line, fp) || !fgets(line, sizeof line, fp)) bad = 1;
    if (!bad) {
        char* save = NULL;
        char* c    = strtok_r(line, " ", &save);
        want       = c ? atoi(c) : 0;
        if (want <= 0 || !ha_reserve(&a, want + 1)) bad = 1;
    }
    while (!bad && a.n < want && fgets(line, sizeof line, fp)) {
        char* save = NULL;
        char* f[9];
        f[0] = strtok_r(line, " ", &save);
        for (int k = 1; k < 9; k++) f[k] = next_tok(&save);
        const int t = type_of_name(f[1]);
        if (!f[8] || t < 0) {
            bad = 1;
            break;
        }
        a.type[a.n] = t;
        for (int d = 0; d < 3; d++) {
            a.x[3 * a.n + d] = atof(f[3 + d]);
            a.v[3 * a.n + d] = atof(f[6 + d]);
        }
        a.n++;
    }
    if (!bad && fgets(line, sizeof line, fp)) {
        char* save = NULL;
        char* b0   = strtok_r(line, " ", &save);
        char* b1   = next_tok(&save);
        char* b2   = next_tok(&save);
        if (b0 && b1 && b2) {
            p->xprd = atof(b0);
            p->yprd = atof(b1);
            p->zprd = atof(b2);
        }
    }
    fclose(fp);
    if (bad || a.n != want) {
        ha_free(&a);
        return -MDB_ERR_ARG;
    }
    return ha_finish(&a, p, x, v, type);
}

int mdbh_read_in(MdbHostParams* p, const char* path, double** x, double** v, int** type)
{
    /* readAtom_in, verletlist/atom.c:658-760: "natoms xlo xhi ylo yhi zlo zhi",
     * then "mass x y z vx vy vz" per atom (the last finite mass becomes the
     * mass; "inf" is skipped); one atom type */
    FILE* fp = fopen(path, "r");
    if (!fp) return -MDB_ERR_ARG;
    char line[4096];
    HostAtoms a = { 0 };
    int bad = 0, natoms = 0;
    double b[6] = { 0 };
    if (!fgets(line, sizeof line, fp)) bad = 1;
    if (!bad) {
        char* save = NULL;
        char* c    = strtok_r(line, " ", &save);
        natoms     = c ? atoi(c) : 0;
        for (int k = 0; k < 6 && !bad; k++) {
            char* t = next_tok(&save);
            if (!t) bad = 1;
            else b[k] = atof(t);
        }
        if (natoms <= 0 || !ha_reserve(&a, natoms + 1)) bad = 1;
    }
    for (int i = 0; i < natoms && !bad; i++) {
        char* save = NULL;
        if (!fgets(line, sizeof line, fp)) {
            bad = 1;
            break;
        }
        char* f[7];
        f[0] = strtok_r(line, " ", &save);
        for (int k = 1; k < 7; k++) f[k] = next_tok(&save);
        if (!f[6]) {
            bad = 1;
            break;
        }
        if (strncmp(f[0], "inf", 3) != 0) p->mass = atof(f[0]);
        a.type[i] = 0;
        for (int d = 0; d < 3; d++) {
            a.x[3 * i + d] = atof(f[1 + d]);
            a.v[3 * i + d] = atof(f[4 + d]);
        }
        a.n++;
    }
    fclose(fp);
    if (bad) {
        ha_free(&a);
        return -MDB_ERR_ARG;
    }
    p->xprd = b[1] - b[0];
    p->yprd = b[3] - b[2];
    p->zprd = b[5] - b[4];
    return ha_finish(&a, p, x, v, type);
}

int mdbh_read_atoms(MdbHostParams* p, const char* path, double** x, double** v, int** type)
{
    /* readAtom, verletlist/atom.c:260-294: by file extension */
    const size_t n = strlen(path);
    if (n >= 4 && !strcmp(path + n - 4, ".pdb")) return mdbh_read_pdb(p, path, x, v, type);
    if (n >= 4 && !strcmp(path + n - 4, ".gro")) return mdbh_read_gro(p, path, x, v, type);
    if (n >= 4 && !strcmp(path + n - 4, ".dmp")) return mdbh_read_dmp(p, path, x, v, type);
    if (n >= 3 && !strcmp(path + n - 3, ".in")) return mdbh_read_in(p, path, x, v, type);
    return -MDB_ERR_ARG;
}

int mdbh_write_atoms(const char* path, int n, const double* x, const double* v, const int* type)
{
    /* writeAtom (-w), verletlist/atom.c:762-786: "type,1.0,x,y,z,vx,vy,vz,0" */
    FILE* fp = fopen(path, "w");
    if (!fp) return MDB_ERR_ARG;
    for (int i = 0; i < n; i++)
        fprintf(fp, "%d,%f,%f,%f,%f,%f,%f,%f,0\n", type[i], 1.0, x[3 * i], x[3 * i + 1],
            x[3 * i + 2], v[3 * i], v[3 * i + 1], v[3 * i + 2]);
    return fclose(fp) == 0 ? MDB_OK : MDB_ERR_ARG;
}

int mdbh_write_vtk(const char* base, int timestep, int n, const double* x)
{
    /* write_atoms_to_vtk_file, verletlist/vtk.c:21-71: "<base>_<step>.vtk",
     * legacy ASCII unstructured grid of vertex cells, unit masses */
    char path[4096];
    snprintf(path, sizeof path, "%s_%d.vtk", base, timestep);
    FILE* fp = fopen(path, "wb");
    if (!fp) return MDB_ERR_ARG;
    fprintf(fp, "# vtk DataFile Version 2.0\nParticle data\nASCII\nDATASET UNSTRUCTURED_GRID\n");
    fprintf(fp, "POINTS %d double\n", n);
    for (int i = 0; i < n; i++)
        fprintf(fp, "%.4f %.4f %.4f\n", x[3 * i], x[3 * i + 1], x[3 * i + 2]);
    fprintf(fp, "\n\nCELLS %d %d\n", n, 2 * n);
    for (int i = 0; i < n; i++) fprintf(fp, "1 %d\n", i);
    fprintf(fp, "\n\nCELL_TYPES %d\n", n);
    for (int i = 0; i < n; i++) fprintf(fp, "1\n");
    fprintf(fp, "\n\nPOINT_DATA %d\nSCALARS mass double\nLOOKUP_TABLE default\n", n);
    for (int i = 0; i < n; i++) fprintf(fp, "1.0\n");
    fprintf(fp, "\n\n");
    return fclose(fp) == 0 ? MDB_OK : MDB_ERR_ARG;
}

/* ---- the stub gather benchmark (verletlist/main-stub.c) --------------------- */

int mdbh_stub_atoms(int natoms, int ntypes, unsigned seed, double* x, double* v, int* type)
{
    /* main-stub.c:221-234: atom i at (i, i, i) * 1e-5 at rest, type rand() %
     * ntypes from the process's rand() stream (a fresh process: seed 1) */
    if (natoms < 1 || ntypes < 1 || !x || !v || !type) return MDB_ERR_ARG;
    srand(seed);
    for (int i = 0; i < natoms; i++) {
        type[i] = rand() % ntypes;
        for (int d = 0; d < 3; d++) {
            x[3 * i + d] = (double)i * 0.00001;
            v[3 * i + d] = 0.0;
        }
    }
    return MDB_OK;
}

int mdbh_stub_neighbors(int natoms, int pattern, int nneighs, int nreps, int* numneigh,
    int* neighbors)
{
    /* createNeighbors, main-stub.c:60-113, row-major rows of nneighs * nreps:
     * seq: the nneighs atoms after i (cyclically), fix: atoms 0 .. nneighs-1,
     * rand: distinct random atoms other than i, drawn from rand() (continuing
     * the stream of mdbh_stub_atoms); the row is then repeated nreps times. */
    if (natoms < 1 || nneighs < 1 || nreps < 1 || !numneigh || !neighbors) return MDB_ERR_ARG;
    if (pattern < MDBH_STUB_SEQ || pattern > MDBH_STUB_RAND) return MDB_ERR_ARG;
    if (pattern == MDBH_STUB_RAND && natoms <= nneighs) return MDB_ERR_ARG;
    if (pattern == MDBH_STUB_FIX && natoms < nneighs) return MDB_ERR_ARG;
    const size_t row = (size_t)nneighs * nreps;
    for (int i = 0; i < natoms; i++) {
        int* r = neighbors + (size_t)i * row;
        for (int k = 0; k < nneighs; k++) {
            int j;
            if (pattern == MDBH_STUB_SEQ) {
                j = (int)(((long long)i + 1 + k) % natoms);
            } else if (pattern == MDBH_STUB_FIX) {
                j = k;
            } else {
                int again;
                do {
                    j     = rand() % natoms;
                    again = j == i;
                    for (int l = 0; l < k && !again; l++) again = r[l] == j;
                } while (again);
            }
            r[k] = j;
        }
        for (int q = 1; q < nreps; q++) memcpy(r + (size_t)q * nneighs, r, sizeof(int) * nneighs);
        numneigh[i] = (int)row;
    }
    return MDB_OK;
}

void mdbh_mdb_params(const MdbHostParams* p, int natoms, MdbParams* o)
{
    memset(o, 0, sizeof *o);
    o->force_field      = p->force_field;
    o->half_neigh       = p->half_neigh;
    o->precision        = p->precision;
    o->bin_rule         = p->from_file ? MDB_BINS_FILE : MDB_BINS_LATTICE;
    o->nx               = p->nx;
    o->ny               = p->ny;
    o->nz               = p->nz;
    o->pbc_x            = p->pbc_x;
    o->pbc_y            = p->pbc_y;
    o->pbc_z            = p->pbc_z;
    o->ntypes           = p->ntypes;
    o->reneigh_every    = p->reneigh_every;
    o->nstat            = p->nstat;
    o->maxneighs        = 100;
    o->natoms           = natoms;
    o->xprd             = p->xprd;
    o->yprd             = p->yprd;
    o->zprd             = p->zprd;
    o->dt               = p->dt;
    o->dtforce          = p->dtforce;
    o->mass             = p->mass;
    o->cutforce         = p->cutforce;
    o->cutneigh         = p->cutneigh;
    o->epsilon          = p->epsilon;
    o->sigma            = p->sigma;
    o->epsilon_per_type = p->has_types ? p->epsilon_per_type : NULL;
    o->sigma_per_type   = p->has_types ? p->sigma_per_type : NULL;
}
