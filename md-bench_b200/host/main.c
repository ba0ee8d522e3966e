/*
 * MDBench-B200: the Verlet-list driver of MD-Bench (verletlist/main.c:187-529)
 * on libmdb. Same command line and the same thermo and performance lines, so
 * the reference's regression scripts (tests/sim_copper_fcc_regression.sh) can
 * run it unchanged. The timestep loop runs either as the reference's
 * per-hook sequence (--hooks) or as the graph-captured loop (default).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "mdb.h"
#include "mdb_host.h"

static double now(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + (double)ts.tv_nsec * 1.e-9;
}

#define CHECK(call)                                                                     \
    do {                                                                                \
        int rc_ = (call);                                                               \
        if (rc_ != MDB_OK) {                                                            \
            fprintf(stderr, "%s failed: %s (%s)\n", #call, mdb_status_string(rc_),      \
                ctx ? mdb_last_error(ctx) : "");                                        \
            exit(EXIT_FAILURE);                                                         \
        }                                                                               \
    } while (0)

static void usage(void)
{
    printf("MDBench-B200: MD-Bench's Verlet-list timestep on a B200\n"
           "-p / --params <file>   parameter file (key value)\n"
           "-f <lj|eam>            force field\n"
           "-i <file>              input atoms (.pdb, .gro, .dmp or .in, as readAtom)\n"
           "-e <file>              EAM funcfl file\n"
           "-n / --nsteps <int>    timesteps\n"
           "-nx/-ny/-nz <int>      unit cells\n"
           "-half <0|1>            half (1) or full (0) neighbour lists\n"
           "-r / --radius <real>   force cutoff\n"
           "-s / --skin <real>     Verlet skin\n"
           "--prec <fp64|mixed|mixed_comp>  precision of the force kernels\n"
           "--hooks                run the per-hook loop instead of CUDA graphs\n"
           "-w <file>              write the initial atoms (writeAtom's format; .dmp: a dump)\n");
}

int main(int argc, char** argv)
{
    MdbHostParams hp;
    MdbCtx* ctx = NULL;
    mdbh_defaults(&hp);
    const char *input = NULL, *eam_file = NULL, *write_file = NULL;
    int hooks = 0, ff = -1;
    double cutforce = -1, skin = -1;
    for (int i = 1; i < argc; i++) {
        const char* a = argv[i];
        const char* v = i + 1 < argc ? argv[i + 1] : NULL;
        if ((!strcmp(a, "-p") || !strcmp(a, "--params")) && v) {
            if (mdbh_read_params(&hp, v) != MDB_OK) {
                fprintf(stderr, "Could not read parameter file: %s\n", v);
                return EXIT_FAILURE;
            }
            i++;
        } else if (!strcmp(a, "-f") && v) {
            ff = !strncmp(v, "eam", 3) ? MDB_FF_EAM : (!strncmp(v, "lj", 2) ? MDB_FF_LJ : -2);
            if (ff == -2) {
                fprintf(stderr, "Invalid force field!\n");
                return EXIT_FAILURE;
            }
            i++;
        } else if (!strcmp(a, "-i") && v) {
            input = v;
            i++;
        } else if (!strcmp(a, "-e") && v) {
            eam_file = v;
            i++;
        } else if ((!strcmp(a, "-n") || !strcmp(a, "--nsteps")) && v) {
            hp.ntimes = atoi(v);
            i++;
        } else if (!strcmp(a, "-nx") && v) {
            hp.nx = atoi(v);
            i++;
        } else if (!strcmp(a, "-ny") && v) {
            hp.ny = atoi(v);
            i++;
        } else if (!strcmp(a, "-nz") && v) {
            hp.nz = atoi(v);
            i++;
        } else if (!strcmp(a, "-half") && v) {
            hp.half_neigh = atoi(v);
            i++;
        } else if ((!strcmp(a, "-r") || !strcmp(a, "--radius")) && v) {
            cutforce = atof(v);
            i++;
        } else if ((!strcmp(a, "-s") || !strcmp(a, "--skin")) && v) {
            skin = atof(v);
            i++;
        } else if (!strcmp(a, "--prec") && v) {
            hp.precision = !strcmp(v, "mixed") ? MDB_PREC_MIXED
                           : !strcmp(v, "mixed_comp") ? MDB_PREC_MIXED_COMP
                                                      : MDB_PREC_FP64;
            i++;
        } else if (!strcmp(a, "-w") && v) {
            write_file = v;
            i++;
        } else if (!strcmp(a, "--hooks")) {
            hooks = 1;
        } else if (!strcmp(a, "-h") || !strcmp(a, "--help")) {
            usage();
            return EXIT_SUCCESS;
        }
    }
    if (ff >= 0) hp.force_field = ff;
    if (cutforce > 0) hp.cutforce = cutforce;
    if (skin >= 0) hp.skin = skin;

    double t0 = now();
    MdbEamTables eam;
    memset(&eam, 0, sizeof eam);
    if (hp.force_field == MDB_FF_EAM) {
        if (!eam_file || mdb_eam_read_funcfl(eam_file, &eam) != MDB_OK) {
            fprintf(stderr, "Can't open EAM Potential file: %s\n", eam_file ? eam_file : "");
            return EXIT_FAILURE;
        }
        mdbh_apply_eam(&hp, &eam);
    }
    double *x = NULL, *v = NULL;
    int* type = NULL;
    int n;
    if (input) {
        n = mdbh_read_atoms(&hp, input, &x, &v, &type);
        if (n < 0) {
            fprintf(stderr, "Input error: atom data was not read from %s\n", input);
            return EXIT_FAILURE;
        }
        mdbh_finalize(&hp);
        printf("Read %d atoms from %s\n", n, input);
    } else {
        mdbh_finalize(&hp);
        n = mdbh_create_fcc(&hp, &x, &v, &type);
        if (n < 0) {
            fprintf(stderr, "Could not create the lattice\n");
            return EXIT_FAILURE;
        }
    }
    if (write_file) {
        const size_t wl = strlen(write_file);
        if (wl >= 4 && !strcmp(write_file + wl - 4, ".dmp"))
            mdbh_write_dmp(write_file, n, x, v, type, hp.xprd, hp.yprd, hp.zprd);
        else
            mdbh_write_atoms(write_file, n, x, v, type);
    }

    MdbParams mp;
    mdbh_mdb_params(&hp, n, &mp);
    CHECK(mdb_create(&mp, &ctx));
    if (hp.force_field == MDB_FF_EAM) CHECK(mdb_set_eam(ctx, &eam));
    CHECK(mdb_set_atoms(ctx, n, x, v, type));
    CHECK(mdb_setup(ctx));
    double tsetup = now() - t0;

    static const char* prec_name[] = { "fp64", "mixed", "mixed_comp" };
    printf("SIMULATION PARAMETERS\n"
           "-------------------------------------------------------------------------------\n");
    printf("    Force field:                       %s\n", hp.force_field ? "eam" : "lj");
    printf("    Kernel:                            CUDA sm_100a (%s)\n", prec_name[hp.precision]);
    printf("    Unit cells (nx,ny,nz):             %d x %d x %d\n", hp.nx, hp.ny, hp.nz);
    printf("    Domain box sizes:                  %.2e x %.2e x %.2e\n", hp.xprd, hp.yprd, hp.zprd);
    printf("    Lattice constant:                  %.6e\n", hp.lattice);
    printf("    Timesteps:                         %d\n", hp.ntimes);
    printf("    Timestep (dt):                     %.6e\n", hp.dt);
    printf("    Cutoff radius:                     %.6e\n", hp.cutforce);
    printf("    Skin distance:                     %.6e\n", hp.cutneigh - hp.cutforce);
    printf("    Half neighbor-lists:               %s\n", hp.half_neigh ? "yes" : "no");
    printf("    Reneighbor every:                  %d steps\n", hp.reneigh_every);
    printf("\nSIMULATION PROGRESS\n"
           "-------------------------------------------------------------------------------\n");
    printf("  %-10s %15s %15s\n", "Step", "Temperature", "Pressure");
    MdbThermo th;
    CHECK(mdb_thermo(ctx, &th));
    printf("  %-10d %15.6e %15.6e\n", 0, th.temperature, th.pressure);
    fflush(stdout);

    double tstart = now();
    if (hooks) {
        for (int s = 0; s < hp.ntimes; s++) {
            int reneigh = (s + 1) % hp.reneigh_every == 0;
            CHECK(mdb_initial_integrate(ctx));
            if (reneigh) {
                CHECK(mdb_update_atoms_pbc(ctx));
                CHECK(mdb_setup_pbc(ctx));
                CHECK(mdb_update_pbc(ctx));
                CHECK(mdb_build_neighbor(ctx));
            } else {
                CHECK(mdb_update_pbc(ctx));
            }
            CHECK(mdb_compute_force(ctx));
            CHECK(mdb_final_integrate(ctx));
            if ((s + 1) % hp.nstat == 0 || s + 1 == hp.ntimes) {
                CHECK(mdb_thermo(ctx, &th));
                printf("  %-10d %15.6e %15.6e\n", s + 1, th.temperature, th.pressure);
            }
        }
        CHECK(mdb_synchronize(ctx));
    } else {
        MdbThermo samples[64];
        int done = 0;
        while (done < hp.ntimes) {
            int chunk = hp.ntimes - done;
            if (chunk > 60 * hp.nstat) chunk = 60 * hp.nstat;
            int ns = 0;
            CHECK(mdb_run(ctx, done, chunk, samples, 64, &ns));
            for (int k = 0; k < ns; k++)
                printf("  %-10d %15.6e %15.6e\n", samples[k].step, samples[k].temperature,
                    samples[k].pressure);
            done += chunk;
        }
    }
    double ttotal = now() - tstart;
    printf("-------------------------------------------------------------------------------\n"
           "\nPERFORMANCE REPORT\n"
           "-------------------------------------------------------------------------------\n");
    printf("    Setup                    %8.2f s\n", tsetup);
    int nl = 0, ng = 0, mx = 0;
    CHECK(mdb_get_counts(ctx, &nl, &ng, &mx));
    printf("\n  System: %d atoms (%d ghost) | %d timesteps\n", n, ng, hp.ntimes);
    printf("  Performance: %.2fs total | %.2f atom updates/us | %.2f steps/s\n", ttotal,
        (double)n * hp.ntimes / (ttotal * 1e6), hp.ntimes / ttotal);
    printf("-------------------------------------------------------------------------------\n");
    mdb_destroy(ctx);
    if (hp.force_field == MDB_FF_EAM) mdb_eam_free(&eam);
    free(x);
    free(v);
    free(type);
    return EXIT_SUCCESS;
}
