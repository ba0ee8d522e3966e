/* MD-Bench's Verlet-list hooks bound to libmdb (include/mdb.h).
 *
 * The drop-in a maintainer adds to the reference: compiled with the
 * reference's own headers and flags and linked with its sources in place of
 * three of them, which this file replaces:
 *
 *   common/device.c      initDevice and the device-memory shim of the CPU
 *                        build (:12-20; libmdb owns its device memory, so the
 *                        shim stays a set of no-ops; the CUDA build's
 *                        initDevice is verletlist/device_spec.c:12-48)
 *   verletlist/force.c   computeForce, initForce          (:11-42)
 *   verletlist/pbc.c     updatePbc, updateAtomsPbc, initPbc, setupPbc,
 *                        NmaxGhost, PBCx/y/z              (:17-232)
 *
 * The reference's main.c, Atom, Neighbor, Parameter, thermo and the rest stay
 * as they are. Its hook pointers (verletlist/force.h:16-17, neighbor.h:80-81,
 * pbc.h:15-17, integrate.h:12-14) end up on libmdb's entry points, which keep
 * the atoms on the GPU between calls; the host arrays are refreshed before
 * every thermo sample, which is all the reference's loop reads from them
 * (computeThermo, common/thermo.c:60-100, sums the host velocities).
 *
 * Build (oracle/Makefile, target _ref/MDBench-VL-libmdb): the reference's
 * verletlist and common sources without the three files above, its main.c
 * and this file, -I<include>, -lmdb. Errors print libmdb's message and
 * exit, as the reference's cuda_assert does (common/deviceCuda.cu:14-20). */
#include <stdbool.h>
#include <stdio.h>
#include <stdlib.h>

#include <atom.h>
#include <device.h>
#include <eam.h>
#include <force.h>
#include <integrate.h>
#include <neighbor.h>
#include <parameter.h>
#include <pbc.h>
#include <stats.h>

#include "mdb.h"

static MdbCtx* g_ctx;
static int g_steps; /* timesteps completed (finalIntegrate calls) */

static void ck(int rc, const char* what)
{
    if (rc != MDB_OK) {
        fprintf(stderr, "%s: %s (%s)\n", what, mdb_status_string(rc),
            g_ctx ? mdb_last_error(g_ctx) : "no context");
        exit(EXIT_FAILURE);
    }
}

/* ---- verletlist/pbc.c ------------------------------------------------------ */
int NmaxGhost;
int *PBCx, *PBCy, *PBCz;

static void updatePbcB200(Atom* atom, Parameter* param, bool reneigh)
{
    (void)atom, (void)param, (void)reneigh;
    ck(mdb_update_pbc(g_ctx), "updatePbc");
}

static void updateAtomsPbcB200(Atom* atom, Parameter* param, bool reneigh)
{
    (void)atom, (void)param, (void)reneigh;
    ck(mdb_update_atoms_pbc(g_ctx), "updateAtomsPbc");
}

UpdatePbcFunction updatePbc      = updatePbcB200;
UpdatePbcFunction updateAtomsPbc = updateAtomsPbcB200;

void initPbc(Atom* atom)
{
    NmaxGhost        = 0;
    atom->border_map = NULL;
    PBCx = PBCy = PBCz = NULL;
}

/* setup() calls this once before initDevice (no context yet: initDevice sets
 * the ghosts up) and reneighbour() at every rebuild */
void setupPbc(Atom* atom, Parameter* param)
{
    (void)atom, (void)param;
    if (g_ctx) ck(mdb_setup_pbc(g_ctx), "setupPbc");
}

/* ---- verletlist/force.c and the other hooks ---------------------------------- */
ComputeForceFunction computeForce;

static double computeForceB200(Parameter* param, Atom* atom, Neighbor* neighbor, Stats* stats)
{
    (void)param, (void)atom, (void)neighbor, (void)stats;
    ck(mdb_compute_force(g_ctx), "computeForce");
    return 0.0;
}

static void buildNeighborB200(Atom* atom, Neighbor* neighbor)
{
    (void)atom, (void)neighbor;
    ck(mdb_build_neighbor(g_ctx), "buildNeighbor");
}

static void initialIntegrateB200(bool reneigh, Parameter* param, Atom* atom)
{
    (void)reneigh, (void)param, (void)atom;
    ck(mdb_initial_integrate(g_ctx), "initialIntegrate");
}

/* the loop samples thermo after step n when (n + 1) % nstat == 0 and after
 * the last step: the host arrays are brought up to date for those */
static void finalIntegrateB200(bool reneigh, Parameter* param, Atom* atom)
{
    (void)reneigh;
    ck(mdb_final_integrate(g_ctx), "finalIntegrate");
    g_steps++;
    if (g_steps % param->nstat == 0 || g_steps == param->ntimes)
        ck(mdb_get_atoms(g_ctx, atom->x, atom->vx, atom->fx, atom->type), "mdb_get_atoms");
}

void initForce(Parameter* param)
{
    (void)param;
    computeForce = computeForceB200;
}

/* ---- common/device.c ---------------------------------------------------------------
 * The device-memory shim (common/device.h:26-50) is not needed: the
 * reference's growAtom (verletlist/atom.c:788-866) still calls it for its
 * unused device mirror. */
void GPUfree(void* any) { (void)any; }
void* allocateGPU(size_t bytesize)
{
    (void)bytesize;
    return NULL;
}
void* reallocateGPU(void* ptr, size_t new_bytesize)
{
    (void)ptr, (void)new_bytesize;
    return NULL;
}
void memcpyToGPU(void* d_ptr, void* h_ptr, size_t bytesize) { (void)d_ptr, (void)h_ptr, (void)bytesize; }
void memcpyFromGPU(void* h_ptr, void* d_ptr, size_t bytesize) { (void)h_ptr, (void)d_ptr, (void)bytesize; }
void memsetGPU(void* d_ptr, int value, size_t bytesize) { (void)d_ptr, (void)value, (void)bytesize; }

/* initDevice: setup() calls it after createAtom/readAtom, adjustThermo and the first
 * setupPbc, before updatePbc and buildNeighbor: the atoms go to the GPU and
 * every hook is bound here, so the first list is already libmdb's. */
void initDevice(Parameter* param, Atom* atom, Neighbor* neighbor)
{
    MdbParams p = { 0 };
    p.force_field      = param->force_field == FF_EAM ? MDB_FF_EAM : MDB_FF_LJ;
    p.half_neigh       = param->half_neigh;
    p.precision        = getenv("MDB_MIXED") ? MDB_PREC_MIXED : MDB_PREC_FP64;
    p.bin_rule         = param->input_file ? MDB_BINS_FILE : MDB_BINS_LATTICE;
    p.nx               = param->nx;
    p.ny               = param->ny;
    p.nz               = param->nz;
    p.pbc_x            = param->pbc_x;
    p.pbc_y            = param->pbc_y;
    p.pbc_z            = param->pbc_z;
    p.ntypes           = atom->ntypes;
    p.reneigh_every    = param->reneigh_every;
    p.nstat            = param->nstat;
    p.maxneighs        = neighbor->maxneighs;
    p.natoms           = atom->Natoms;
    p.xprd             = param->xprd;
    p.yprd             = param->yprd;
    p.zprd             = param->zprd;
    p.dt               = param->dt;
    p.dtforce          = param->dtforce;
    p.mass             = param->mass;
    p.cutforce         = param->cutforce;
    p.cutneigh         = param->cutneigh;
    p.epsilon          = param->epsilon;
    p.sigma            = param->sigma;
    p.epsilon_per_type = param->epsilon_per_type;
    p.sigma_per_type   = param->sigma_per_type;
    ck(mdb_create(&p, &g_ctx), "mdb_create");
    if (param->force_field == FF_EAM) {
        /* the tables initEam built (common/eam_utils.c:22-284) */
        MdbEamTables t = { eam.nrho, eam.nr, eam.nrho_tot, eam.nr_tot, eam.rdr, eam.rdrho,
            eam.file.cut, eam.file.mass, eam.frho_spline, eam.rhor_spline, eam.z2r_spline };
        ck(mdb_set_eam(g_ctx, &t), "mdb_set_eam");
    }
    ck(mdb_set_atoms(g_ctx, atom->Nlocal, atom->x, atom->vx, atom->type), "mdb_set_atoms");
    ck(mdb_setup_pbc(g_ctx), "setupPbc");
    buildNeighbor    = buildNeighborB200;
    initialIntegrate = initialIntegrateB200;
    finalIntegrate   = finalIntegrateB200;
    computeForce     = computeForceB200;
    g_steps          = 0;
}
