/* periodic_driver.c -- TEST INFRASTRUCTURE ONLY (never shipped, never measured).
 *
 * A small application driver written against the reference's lattice API (lb.h) alone, for
 * the functions the reference's own driver leaves unused or untested: makePeriodic
 * (lb.c:1783-1817), saveVel (lb.c:1822-1850) and saveF (lb.c:1853-1866).  oracle/Makefile
 * builds it twice from this one file:
 *   _ref/periodic_ref   with the reference's unmodified lb.c and boundaries.c;
 *   _ref/periodic_gpu   against include/lb.h and the GPU library (-DLBREF_GPU).
 * The tests run both and require identical output files.
 *
 * Scenario: a box periodic in x and y (every interior node BGK, a bounce-back disk inside),
 * every node -- ghost ring included -- initialised to the equilibrium of a smooth
 * position-dependent state.  makePeriodic runs once on that initial state (before any step:
 * the GPU library wraps its host arrays) and then after every stream (on the device).
 *
 * usage: periodic_<ref|gpu> lx ly steps variant outdir
 *   variant 0: collide + propagate (origin), 1: collide_with_stream + finalize_stream (combine)
 * writes outdir/lattice.bin (the final lattice, ghost ring included, raw doubles in
 * [X][Y][9] order), outdir/vel.dat (saveVel) and outdir/f<i>.dat (saveF, i = 0..8).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include "lb.h"
#include "boundaries.h"
#ifdef LBREF_GPU
#include "lbgpu.h"
#endif

/* Globals lb.c reads (declared extern at lb.c:30-38); an application driver defines them. */
PressureBCData *pressureBoundary;
int blk_size = 1;
double *myrho1, *myrho2;
int iT = 0, count = 0;
int thread_block = 1;
int NUM_THREADS = 1;
long long global_CM[NUM_EVENTS];

static const double kPi = 3.14159265358979323846;

int main(int argc, char **argv)
{
    Simulation sim;
    Dynamics bulk, wall;
    double omega = 1.7;
    int lx, ly, steps, variant, X, Y, i, t;
    char path[4096];
    FILE *f;
    if (argc != 6) {
        fprintf(stderr, "usage: %s lx ly steps variant outdir\n", argv[0]);
        return 2;
    }
    lx = atoi(argv[1]); ly = atoi(argv[2]); steps = atoi(argv[3]); variant = atoi(argv[4]);
    bulk.dynamicsFun = &bgk; bulk.selfData = (void *)&omega;
    wall.dynamicsFun = &bounceBack; wall.selfData = 0;
    myrho1 = (double *)calloc(ly + 2, sizeof(double));
    myrho2 = (double *)calloc(ly + 2, sizeof(double));

    constructSim(&sim, lx, ly);
    for (X = 0; X <= lx + 1; ++X)
        for (Y = 0; Y <= ly + 1; ++Y) {
            double rho = 1. + 0.01 * sin(2. * kPi * X / lx) * cos(2. * kPi * Y / ly);
            double ux = 0.03 * sin(2. * kPi * Y / ly);
            double uy = 0.02 * cos(2. * kPi * X / lx);
            iniEquilibrium(&sim.lattice[X][Y], rho, ux, uy);
        }
    for (X = 1; X <= lx; ++X)
        for (Y = 1; Y <= ly; ++Y) {
            int dx = X - lx / 3, dy = Y - ly / 2, r = ly / 8 + 1;
            setDynamics(&sim, X, Y, (dx * dx + dy * dy <= r * r) ? &wall : &bulk);
        }

    makePeriodic(&sim);   /* on the initial state: before the first step */
    for (t = 0; t < steps; ++t) {
        if (variant == 0) {
            collide(&sim);
            propagate(&sim);
        } else {
            collide_with_stream(&sim);
            finalize_stream(&sim);
        }
        makePeriodic(&sim);
    }

    snprintf(path, sizeof path, "%s/vel.dat", argv[5]);
    saveVel(&sim, path);
    for (i = 0; i < 9; ++i) {
        snprintf(path, sizeof path, "%s/f%d.dat", argv[5], i);
        saveF(&sim, i, path);
    }
#ifdef LBREF_GPU
    lbSyncToHost(&sim);
    if (lbGetLastError()) {
        fprintf(stderr, "liblbgpu error %d: %s\n", lbGetLastError(), lbGetLastErrorString());
        return 1;
    }
#endif
    snprintf(path, sizeof path, "%s/lattice.bin", argv[5]);
    f = fopen(path, "wb");
    if (!f) return 1;
    for (X = 0; X < lx + 2; ++X)
        for (Y = 0; Y < ly + 2; ++Y) fwrite(sim.lattice[X][Y].fPop, sizeof(double), 9, f);
    fclose(f);
    destructSim(&sim);
    free(myrho1); free(myrho2);
    return 0;
}
