// EAM funcfl reader and spline construction for libmdb (host code).
// Follows initEam / readEamFile / file2array / array2spline / interpolate of
// the reference (common/eam_utils.c:22-284) for a single element: the funcfl
// arrays are resampled onto a common grid with 4-point Lagrange weights and
// turned into rows of 7 cubic coefficients (0..2: derivative, 3..6: value).
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "mdb.h"

namespace {

bool read_values(FILE* fp, int n, std::vector<double>& out)
{
    out.assign(n + 1, 0.0);
    int i = 0;
    char line[4096];
    while (i < n && fgets(line, sizeof line, fp)) {
        char* save = nullptr;
        for (char* tok = strtok_r(line, " \t\n\r\f", &save); tok && i < n;
             tok       = strtok_r(nullptr, " \t\n\r\f", &save))
            out[++i] = atof(tok); // 1-based like the reference after its shift
    }
    return i == n;
}

double lagrange4(const std::vector<double>& a, int nfile, double dfile, double r)
{
    const double sixth = 1.0 / 6.0;
    double p           = r / dfile + 1.0;
    int k              = (int)(p);
    k                  = k < nfile - 2 ? k : nfile - 2;
    k                  = k > 2 ? k : 2;
    p -= k;
    p           = p < 2.0 ? p : 2.0;
    double cof1 = -sixth * p * (p - 1.0) * (p - 2.0);
    double cof2 = 0.5 * (p * p - 1.0) * (p - 2.0);
    double cof3 = -0.5 * p * (p + 1.0) * (p - 2.0);
    double cof4 = sixth * p * (p * p - 1.0);
    return cof1 * a[k - 1] + cof2 * a[k] + cof3 * a[k + 1] + cof4 * a[k + 2];
}

void spline7(int n, double delta, const std::vector<double>& f, double* s)
{
    for (int m = 1; m <= n; m++)
        s[m * 7 + 6] = f[m];
    s[1 * 7 + 5]       = s[2 * 7 + 6] - s[1 * 7 + 6];
    s[2 * 7 + 5]       = 0.5 * (s[3 * 7 + 6] - s[1 * 7 + 6]);
    s[(n - 1) * 7 + 5] = 0.5 * (s[n * 7 + 6] - s[(n - 2) * 7 + 6]);
    s[n * 7 + 5]       = s[n * 7 + 6] - s[(n - 1) * 7 + 6];
    for (int m = 3; m <= n - 2; m++)
        s[m * 7 + 5] = ((s[(m - 2) * 7 + 6] - s[(m + 2) * 7 + 6]) +
                           8.0 * (s[(m + 1) * 7 + 6] - s[(m - 1) * 7 + 6])) /
                       12.0;
    for (int m = 1; m <= n - 1; m++) {
        s[m * 7 + 4] = 3.0 * (s[(m + 1) * 7 + 6] - s[m * 7 + 6]) - 2.0 * s[m * 7 + 5] -
                       s[(m + 1) * 7 + 5];
        s[m * 7 + 3] = s[m * 7 + 5] + s[(m + 1) * 7 + 5] - 2.0 * (s[(m + 1) * 7 + 6] - s[m * 7 + 6]);
    }
    s[n * 7 + 4] = 0.0;
    s[n * 7 + 3] = 0.0;
    for (int m = 1; m <= n; m++) {
        s[m * 7 + 2] = s[m * 7 + 5] / delta;
        s[m * 7 + 1] = 2.0 * s[m * 7 + 4] / delta;
        s[m * 7 + 0] = 3.0 * s[m * 7 + 3] / delta;
    }
}

} // namespace

extern "C" void mdb_eam_free(MdbEamTables* t)
{
    if (!t) return;
    free((void*)t->frho_spline);
    free((void*)t->rhor_spline);
    free((void*)t->z2r_spline);
    memset(t, 0, sizeof *t);
}

extern "C" int mdb_eam_read_funcfl(const char* path, MdbEamTables* out)
{
    if (!path || !out) return MDB_ERR_ARG;
    memset(out, 0, sizeof *out);
    FILE* fp = fopen(path, "r");
    if (!fp) return MDB_ERR_ARG;
    char line[4096];
    int tmp, nrho_f, nr_f;
    double mass, drho_f, dr_f, cut;
    bool ok = fgets(line, sizeof line, fp) && fgets(line, sizeof line, fp) &&
              sscanf(line, "%d %lg", &tmp, &mass) == 2 && fgets(line, sizeof line, fp) &&
              sscanf(line, "%d %lg %d %lg %lg", &nrho_f, &drho_f, &nr_f, &dr_f, &cut) == 5 &&
              nrho_f > 4 && nr_f > 4 && drho_f > 0 && dr_f > 0;
    std::vector<double> frho_f, zr_f, rhor_f;
    if (ok) ok = read_values(fp, nrho_f, frho_f) && read_values(fp, nr_f, zr_f) &&
                 read_values(fp, nr_f, rhor_f);
    fclose(fp);
    if (!ok) return MDB_ERR_ARG;

    // common grid (file2array): one file, so the grid is the file's own
    double rmax   = (nr_f - 1) * dr_f;
    double rhomax = (nrho_f - 1) * drho_f;
    int nr        = (int)(rmax / dr_f + 0.5);
    int nrho      = (int)(rhomax / drho_f + 0.5);
    std::vector<double> frho(nrho + 1), rhor(nr + 1), z2r(nr + 1);
    for (int m = 1; m <= nrho; m++)
        frho[m] = lagrange4(frho_f, nrho_f, drho_f, (m - 1) * drho_f);
    for (int m = 1; m <= nr; m++)
        rhor[m] = lagrange4(rhor_f, nr_f, dr_f, (m - 1) * dr_f);
    for (int m = 1; m <= nr; m++) {
        double r   = (m - 1) * dr_f;
        double zri = lagrange4(zr_f, nr_f, dr_f, r);
        double zrj = lagrange4(zr_f, nr_f, dr_f, r);
        z2r[m]     = 27.2 * 0.529 * zri * zrj;
    }
    int nrho_tot = (nrho + 1) * 7 + 64;
    int nr_tot   = (nr + 1) * 7 + 64;
    nrho_tot -= nrho_tot % 64;
    nr_tot -= nr_tot % 64;
    double* fs = (double*)calloc(nrho_tot, sizeof(double));
    double* rs = (double*)calloc(nr_tot, sizeof(double));
    double* zs = (double*)calloc(nr_tot, sizeof(double));
    if (!fs || !rs || !zs) {
        free(fs);
        free(rs);
        free(zs);
        return MDB_ERR_NOMEM;
    }
    spline7(nrho, drho_f, frho, fs);
    spline7(nr, dr_f, rhor, rs);
    spline7(nr, dr_f, z2r, zs);
    out->nrho        = nrho;
    out->nr          = nr;
    out->nrho_tot    = nrho_tot;
    out->nr_tot      = nr_tot;
    out->rdr         = 1.0 / dr_f;
    out->rdrho       = 1.0 / drho_f;
    out->cut         = cut;
    out->mass        = mass;
    out->frho_spline = fs;
    out->rhor_spline = rs;
    out->z2r_spline  = zs;
    return MDB_OK;
}
