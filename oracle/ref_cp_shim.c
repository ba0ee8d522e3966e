/*
 * Test-only shim that drives the MD-Bench reference's own cluster-pair sources
 * (compiled from the reference tree by oracle/Makefile into oracle/_ref/, once
 * per cluster shape: the scalar reference kernel with M x N = 1 x 2, the AVX2
 * build with 4 x 4 and the AVX-512 build with 4 x 8). Tests compare the oracle
 * restatement, and through it the CUDA path, with the reference itself on
 * identical inputs. Not part of the product.
 *
 * The call sequence mirrors setup(), reneighbour() and the timestep loop of
 * clusterpair/main.c:44-127 and :326-362 without MPI.
 *
 * Cluster data is exported in "slot" order: slot cj*N + cjj holds atom cjj of
 * j-cluster cj (locals, then ghost clusters, then the dummy cluster), which for
 * M <= N is also slot ci*M + cii of atom cii of i-cluster ci.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <atom.h>
#include <device.h>
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

void ref_cp_set_threads(int n)
{
#ifdef _OPENMP
    omp_set_num_threads(n);
#else
    (void)n;
#endif
}

static Parameter g_param;
static Atom g_atom;
static Neighbor g_nb;
static Stats g_stats;

int ref_cp_shape(int* m, int* n)
{
    *m = CLUSTER_M;
    *n = CLUSTER_N;
    return VECTOR_WIDTH;
}

/* Returns Nclusters_local. param_file / input_file may be NULL;
 * prune_every <= 0 keeps the reference default. */
int ref_cp_setup(int nx, int ny, int nz, int half, const char* param_file,
    const char* input_file, int prune_every)
{
    initParameter(&g_param);
    if (param_file) readParameter(&g_param, param_file);
    g_param.nx         = nx;
    g_param.ny         = ny;
    g_param.nz         = nz;
    g_param.half_neigh = half;
    if (input_file) g_param.input_file = strdup(input_file);
    if (prune_every > 0) g_param.prune_every = prune_every;
    g_param.cutneigh = g_param.cutforce + g_param.skin;

    /* setup(), clusterpair/main.c:44-97 */
    g_param.lattice = pow((4.0 / g_param.rho), (1.0 / 3.0));
    g_param.xprd    = g_param.nx * g_param.lattice;
    g_param.yprd    = g_param.ny * g_param.lattice;
    g_param.zprd    = g_param.nz * g_param.lattice;
    initAtom(&g_atom);
    initForce(&g_param);
    initPbc(&g_atom);
    initStats(&g_stats);
    initNeighbor(&g_nb, &g_param);
    srand(1);
    if (g_param.input_file == NULL) createAtom(&g_atom, &g_param);
    else readAtom(&g_atom, &g_param);
    setupNeighbor(&g_param, &g_atom);
    setupThermo(&g_param, g_atom.Natoms);
    if (g_param.input_file == NULL) adjustThermo(&g_param, &g_atom);
    buildClusters(&g_atom);
    defineJClusters(&g_param, &g_atom);
    setupPbc(&g_atom, &g_param);
    binJClusters(&g_param, &g_atom);
    buildNeighbor(&g_atom, &g_nb);
    initDevice(&g_param, &g_atom, &g_nb);
    /* the force before the loop, clusterpair/main.c:310 */
    computeForce(&g_param, &g_atom, &g_nb, &g_stats);
    return g_atom.Nclusters_local;
}

/* counts: Nlocal Natoms Nclusters_local ncj Nclusters_ghost Nghost dummy_cj
 *         maxneighs */
void ref_cp_counts(int* c)
{
    c[0] = g_atom.Nlocal;
    c[1] = g_atom.Natoms;
    c[2] = g_atom.Nclusters_local;
    c[3] = get_ncj_from_nci(g_atom.Nclusters_local);
    c[4] = g_atom.Nclusters_ghost;
    c[5] = g_atom.Nghost;
    c[6] = g_atom.dummy_cj;
    c[7] = g_nb.maxneighs;
}

void ref_cp_params(double* d)
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

/* Atom arrays (atom order, as updateSingleAtoms last wrote them). */
void ref_cp_get_atoms(double* x, double* v, int* type)
{
    for (int i = 0; i < g_atom.Nlocal; i++) {
        if (x) {
            /* ATOM_POSITION_AOS: x[3i + d] (clusterpair/atom.h:121-125) */
            x[3 * i + 0] = g_atom.x[3 * i + 0];
            x[3 * i + 1] = g_atom.x[3 * i + 1];
            x[3 * i + 2] = g_atom.x[3 * i + 2];
        }
        if (v) {
            v[3 * i + 0] = g_atom.vx[i];
            v[3 * i + 1] = g_atom.vy[i];
            v[3 * i + 2] = g_atom.vz[i];
        }
        if (type) type[i] = g_atom.type[i];
    }
}

/* nslots = (ncj + Nclusters_ghost + 1) * N slots of x (and of v, f, type for
 * the local slots; ghost and dummy slots of v and f are left untouched). */
void ref_cp_get_slots(double* x, double* v, double* f, int* type, int nslots)
{
    for (int s = 0; s < nslots; s++) {
        int cj   = s / CLUSTER_N;
        int cjj  = s % CLUSTER_N;
        int base = CJ_VECTOR_BASE_INDEX(cj);
        if (x) {
            x[3 * s + 0] = g_atom.cl_x[base + CL_X_INDEX(cjj)];
            x[3 * s + 1] = g_atom.cl_x[base + CL_Y_INDEX(cjj)];
            x[3 * s + 2] = g_atom.cl_x[base + CL_Z_INDEX(cjj)];
        }
        if (type) type[s] = g_atom.cl_t[CJ_SCALAR_BASE_INDEX(cj) + cjj];
    }
    int nloc = g_atom.Nclusters_local * CLUSTER_M;
    for (int s = 0; s < nloc && s < nslots; s++) {
        int cj   = s / CLUSTER_N;
        int cjj  = s % CLUSTER_N;
        int base = CJ_VECTOR3_BASE_INDEX(cj);
        if (v) {
            v[3 * s + 0] = g_atom.cl_v[base + CL_X_INDEX_3D(cjj)];
            v[3 * s + 1] = g_atom.cl_v[base + CL_Y_INDEX_3D(cjj)];
            v[3 * s + 2] = g_atom.cl_v[base + CL_Z_INDEX_3D(cjj)];
        }
        if (f) {
            f[3 * s + 0] = g_atom.cl_f[base + CL_X_INDEX_3D(cjj)];
            f[3 * s + 1] = g_atom.cl_f[base + CL_Y_INDEX_3D(cjj)];
            f[3 * s + 2] = g_atom.cl_f[base + CL_Z_INDEX_3D(cjj)];
        }
    }
}

/* Per i-cluster: natoms, bin, bbox (minx maxx miny maxy minz maxz). */
void ref_cp_get_iclusters(int* natoms, int* bin, double* bb)
{
    for (int ci = 0; ci < g_atom.Nclusters_local; ci++) {
        Cluster* c = &g_atom.iclusters[ci];
        natoms[ci] = c->natoms;
        bin[ci]    = g_atom.cluster_bin[ci];
        double* b  = &bb[6 * ci];
        b[0]       = c->bbminx;
        b[1]       = c->bbmaxx;
        b[2]       = c->bbminy;
        b[3]       = c->bbmaxy;
        b[4]       = c->bbminz;
        b[5]       = c->bbmaxz;
    }
}

/* Per j-cluster (locals then ghosts): natoms and bbox. */
void ref_cp_get_jclusters(int* natoms, double* bb, int count)
{
    for (int cj = 0; cj < count; cj++) {
        Cluster* c = &g_atom.jclusters[cj];
        natoms[cj] = c->natoms;
        double* b  = &bb[6 * cj];
        b[0]       = c->bbminx;
        b[1]       = c->bbmaxx;
        b[2]       = c->bbminy;
        b[3]       = c->bbmaxy;
        b[4]       = c->bbminz;
        b[5]       = c->bbmaxz;
    }
}

void ref_cp_get_ghosts(int* border_map, int* pbc)
{
    for (int g = 0; g < g_atom.Nclusters_ghost; g++) {
        border_map[g]  = g_atom.border_map[g];
        pbc[3 * g + 0] = g_atom.PBCx[g];
        pbc[3 * g + 1] = g_atom.PBCy[g];
        pbc[3 * g + 2] = g_atom.PBCz[g];
    }
}

void ref_cp_get_list(int* numneigh, int* nmasked, int* neighbors, unsigned* imask, int ld)
{
    const int nbM = g_atom.Nclusters_local;
    const int nbN = g_nb.maxneighs;
    for (int ci = 0; ci < g_atom.Nclusters_local; ci++) {
        int nn       = g_nb.numneigh[ci];
        numneigh[ci] = nn;
        nmasked[ci]  = g_nb.numneigh_masked[ci];
        for (int k = 0; k < nn && k < ld; k++) {
            neighbors[(size_t)ci * ld + k] = neighs(g_nb.neighbors, ci, k, nbM, nbN);
            if (imask) imask[(size_t)ci * ld + k] = neighs(g_nb.neighbors_imask, ci, k, nbM, nbN);
        }
    }
}

double ref_cp_force(void) { return computeForce(&g_param, &g_atom, &g_nb, &g_stats); }

void ref_cp_prune(void) { pruneNeighbor(&g_param, &g_atom, &g_nb); }

/* updateAtoms() + reneighbour(), clusterpair/main.c:99-127 */
void ref_cp_rebuild(void)
{
    updateSingleAtoms(&g_param, &g_atom);
    updateAtomsPbc(&g_atom, &g_param, false);
    buildClusters(&g_atom);
    defineJClusters(&g_param, &g_atom);
    setupPbc(&g_atom, &g_param);
    binJClusters(&g_param, &g_atom);
    buildNeighbor(&g_atom, &g_nb);
}

void ref_cp_step(int n)
{
    /* clusterpair/main.c:326-362 without MPI */
    initialIntegrate(&g_param, &g_atom);
    if ((n + 1) % g_param.reneigh_every) {
        if (!((n + 1) % g_param.prune_every)) pruneNeighbor(&g_param, &g_atom, &g_nb);
        updatePbc(&g_atom, &g_param, false);
    } else {
        ref_cp_rebuild();
    }
    computeForce(&g_param, &g_atom, &g_nb, &g_stats);
    finalIntegrate(&g_param, &g_atom);
}

/* Temperature and (kinetic) pressure exactly as computeThermo prints them
 * (common/thermo.c:60-100): from the atom arrays, which updateSingleAtoms
 * last refreshed. */
void ref_cp_thermo(double* T, double* P)
{
    double dof    = (g_atom.Natoms * 3 - 3);
    double pscale = 1.0 / 3 / g_param.xprd / g_param.yprd / g_param.zprd;
    double t      = 0.0;
    for (int i = 0; i < g_atom.Nlocal; i++) {
        t += (g_atom.vx[i] * g_atom.vx[i] + g_atom.vy[i] * g_atom.vy[i] +
                 g_atom.vz[i] * g_atom.vz[i]) *
             g_param.mass;
    }
    t  = t * (1.0 / dof);
    *T = t;
    *P = (t * dof) * pscale;
}
