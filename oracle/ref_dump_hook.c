/* ref_dump_hook.c -- TEST INFRASTRUCTURE ONLY.
 *
 * Lets the UNMODIFIED application driver unsteady.c write its final lattice to a file.
 * oracle/Makefile compiles unsteady.c with -DdestructSim=lbref_dump_then_destruct and
 * -DconstructSim=lbref_construct_hook, so the driver's own calls (unsteady.c:376, :563) land
 * here; lb.c itself is compiled without those renames and provides the real functions.
 *
 *   LBREF_DUMP=<path>   write the populations of sim->lattice, ghost ring included, as raw
 *                       little-endian doubles in [X][Y][9] order (X = 0..lx+1, Y = 0..ly+1).
 *   LBREF_POISON=1      fill the second buffer with NaN right after construction.
 *
 * With -DLBREF_GPU the same hook serves the driver linked against this repository's GPU
 * library: it first asks the library to copy the device state back (lbSyncToHost).
 */
#include <stdio.h>
#include <stdlib.h>
#include <math.h>
#include "lb.h"
#ifdef LBREF_GPU
#include "lbgpu.h"
#endif

void lbref_construct_hook(Simulation *sim, int lx, int ly)
{
    const char *p = getenv("LBREF_POISON");
    constructSim(sim, lx, ly);
    if (p && p[0] == '1') {
        size_t n = (size_t)(lx + 2) * (size_t)(ly + 2), k;
        int i;
        for (k = 0; k < n; ++k)
            for (i = 0; i < 9; ++i) sim->tmpMemoryChunk[k].fPop[i] = NAN;
    }
}

void lbref_dump_then_destruct(Simulation *sim)
{
    const char *path = getenv("LBREF_DUMP");
    if (path) {
        FILE *f;
        int X, Y;
#ifdef LBREF_GPU
        lbSyncToHost(sim);
#endif
        f = fopen(path, "wb");
        if (f) {
            for (X = 0; X < sim->lx + 2; ++X)
                for (Y = 0; Y < sim->ly + 2; ++Y)
                    fwrite(sim->lattice[X][Y].fPop, sizeof(double), 9, f);
            fclose(f);
        }
    }
    destructSim(sim);
}
