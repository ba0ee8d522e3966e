/*
 * Test-only shim that drives the MD-Bench reference's own Verlet-list sources
 * (compiled from the reference tree by oracle/Makefile into oracle/_ref/) so
 * that tests can compare the oracle restatement, and through it the CUDA path,
 * with the reference itself on identical inputs. Not part of the product.
 *
 * The call sequence mirrors setup() and the timestep loop of
 * verletlist/main.c:46-113 and :371-419 of the reference.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <atom.h>
#include <device.h>
#include <eam.h>
#include <force.h>
#include <integrate.h>
#include <neighbor.h>
#include <parameter.h>
#include <pbc.h>
#include <stats.h>
#include <thermo.h>
#include <util.h>
#ifdef _OPENMP
#include <omp.h>
#endif

extern int *PBCx, *PBCy, *PBCz;

/* The reference half-list kernel updates f[j] without atomics inside an
 * OpenMP loop (verletlist/force_lj.c:183-187); comparisons run it with one
 * thread. */
void ref_vl_set_threads(int n)
{
#ifdef _OPENMP
    omp_set_num_threads(n);
#else
    (void)n;
#endif
}

static Parameter g_param;
static Atom g_atom;
static Neighbor g_neighbor;
static Stats g_stats;

/* Returns Nlocal. param_file / input_file / eam_file may be NULL. */
int ref_vl_setup(int nx, int ny, int nz, int half, int force_field, const char* param_file,
    const char* input_file, const char* eam_file)
{
    initParameter(&g_param);
    if (param_file) readParameter(&g_param, param_file);
    g_param.nx          = nx;
    g_param.ny          = ny;
    g_param.nz          = nz;
    g_param.half_neigh  = half;
    g_param.force_field = force_field;
    if (input_file) g_param.input_file = strdup(input_file);
    if (eam_file) g_param.eam_file = strdup(eam_file);
    g_param.cutneigh = g_param.cutforce + g_param.skin;

    /* setup(), verletlist/main.c:46-113 */
    if (g_param.force_field == FF_EAM) initEam(&g_param);
    g_param.lattice = pow((4.0 / g_param.rho), (1.0 / 3.0));
    g_param.xprd    = g_param.nx * g_param.lattice;
    g_param.yprd    = g_param.ny * g_param.lattice;
    g_param.zprd    = g_param.nz * g_param.lattice;
    initAtom(&g_atom);
    initPbc(&g_atom);
    initStats(&g_stats);
    initNeighbor(&g_neighbor, &g_param);
    /* a fresh reference process draws types from rand() in its default state */
    srand(1);
    if (g_param.input_file == NULL) createAtom(&g_atom, &g_param);
    else readAtom(&g_atom, &g_param);
    setupNeighbor(&g_param);
    setupThermo(&g_param, g_atom.Natoms);
    if (g_param.input_file == NULL) adjustThermo(&g_param, &g_atom);
    setupPbc(&g_atom, &g_param);
    initDevice(&g_param, &g_atom, &g_neighbor);
    updatePbc(&g_atom, &g_param, true);
    buildNeighbor(&g_atom, &g_neighbor);
    initForce(&g_param);
    return g_atom.Nlocal;
}

int ref_vl_nlocal(void) { return g_atom.Nlocal; }
int ref_vl_nghost(void) { return g_atom.Nghost; }
int ref_vl_maxneighs(void) { return g_neighbor.maxneighs; }

void ref_vl_params(double* d)
{
    d[0] = g_param.xprd;
    d[1] = g_param.yprd;
    d[2] = g_param.zprd;
    d[3] = g_param.dt;
    d[4] = g_param.dtforce;
    d[5] = g_param.mass;
    d[6] = g_param.cutforce;
    d[7] = g_param.cutneigh;
}

void ref_vl_get_atoms(double* x, double* v, double* f, int* type, int nall)
{
    for (int i = 0; i < nall; i++) {
        for (int d = 0; d < 3; d++) {
            if (x) x[3 * i + d] = g_atom.x[3 * i + d];
            if (v) v[3 * i + d] = g_atom.vx[3 * i + d];
            if (f) f[3 * i + d] = g_atom.fx[3 * i + d];
        }
        if (type) type[i] = g_atom.type[i];
    }
}

void ref_vl_set_state(const double* x, const double* v)
{
    for (int i = 0; i < 3 * g_atom.Nlocal; i++) {
        if (x) g_atom.x[i] = x[i];
        if (v) g_atom.vx[i] = v[i];
    }
}

void ref_vl_get_ghosts(int* border_map, int* pbc)
{
    for (int g = 0; g < g_atom.Nghost; g++) {
        border_map[g]  = g_atom.border_map[g];
        pbc[3 * g + 0] = PBCx[g];
        pbc[3 * g + 1] = PBCy[g];
        pbc[3 * g + 2] = PBCz[g];
    }
}

void ref_vl_get_list(int* numneigh, int* neighbors, int ld)
{
    for (int i = 0; i < g_atom.Nlocal; i++) {
        int nn      = g_neighbor.numneigh[i];
        numneigh[i] = nn;
        for (int k = 0; k < nn && k < ld; k++)
            neighbors[(size_t)i * ld + k] = neighs(g_neighbor.neighbors, i, k,
                g_atom.Nlocal, g_neighbor.maxneighs);
    }
}

double ref_vl_force(void) { return computeForce(&g_param, &g_atom, &g_neighbor, &g_stats); }

void ref_vl_rebuild(void)
{
    updateAtomsPbc(&g_atom, &g_param, true);
    setupPbc(&g_atom, &g_param);
    updatePbc(&g_atom, &g_param, true);
    buildNeighbor(&g_atom, &g_neighbor);
}

/* sortAtom as the SORT_ATOMS build calls it (verletlist/main.c:92-95) */
void ref_vl_sort(void)
{
    g_atom.Nghost = 0;
    sortAtom(&g_atom);
}

void ref_vl_step(int n)
{
    /* verletlist/main.c:371-419 without MPI */
    int reneigh = (n + 1) % g_param.reneigh_every == 0;
    initialIntegrate(reneigh, &g_param, &g_atom);
    if (reneigh) {
        ref_vl_rebuild();
    } else {
        updatePbc(&g_atom, &g_param, false);
    }
    computeForce(&g_param, &g_atom, &g_neighbor, &g_stats);
    finalIntegrate(reneigh, &g_param, &g_atom);
}

/* Temperature and (kinetic) pressure exactly as computeThermo prints them
 * (common/thermo.c:35-100), summed in index order. */
void ref_vl_thermo(double* T, double* P)
{
    double mvv2e, dof;
    if (g_param.force_field == FF_EAM) {
        mvv2e = 1.036427e-04;
        dof   = (g_atom.Natoms * 3 - 3) * 8.617343e-05;
    } else {
        mvv2e = 1.0;
        dof   = (g_atom.Natoms * 3 - 3);
    }
    double pscale = (g_param.force_field == FF_EAM ? 1.602176e+06 : 1.0) / 3 / g_param.xprd /
                    g_param.yprd / g_param.zprd;
    double t = 0.0;
    for (int i = 0; i < g_atom.Nlocal; i++) {
        double* v = &g_atom.vx[3 * i];
        t += (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) * g_param.mass;
    }
    t  = t * (mvv2e / dof);
    *T = t;
    *P = (t * dof) * pscale;
}
