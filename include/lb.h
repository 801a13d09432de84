/* lb.h -- drop-in C interface of the B200 lattice-Boltzmann library (liblbgpu.so).
 *
 * Source-compatible with the reference's lattice header (lb.h of memory-aware-LBM): the same
 * types with the same member order and the same function prototypes, so a C driver written
 * against the reference (its application driver unsteady.c included) compiles unchanged
 * against this header and links with -llbgpu instead of the reference's lb.c/boundaries.c.
 * Each declaration cites the reference interface it replaces.
 *
 * What changes behind the interface:
 *   - constructSim still allocates the two host node arrays the driver reads and writes;
 *     the lattice also gets a device copy (structure-of-arrays populations, a per-node
 *     dynamics tag, per-row/column boundary tables) created at the first step call.
 *   - every collide/propagate entry point runs CUDA kernels for sm_100a on that device copy;
 *     there is no CPU fallback.  Results are bit-identical to the reference's FP64 CPU code.
 *   - after each entry point the library copies back to the host what the driver reads
 *     (see lbSetSyncMode in lbgpu.h); lbSyncToHost copies the whole current lattice.
 *   - errors never abort: entry points keep their void signatures and record the first
 *     error of the calling thread, readable with lbGetLastError (lbgpu.h).
 */
#ifndef LB_H
#define LB_H

#include "stddef.h"

#ifdef _OPENMP
#include <omp.h>   /* the reference header pulls this in for its drivers (reference lb.h:36-38) */
#endif

/* The application driver computes a zero-gradient outlet before each call (reference
 * lb.h:34); the two-step entry points do it themselves for their second step. */
#define ZGB

/* Size of the cache-miss counter array the reference's drivers define (reference lb.h:40);
 * kept so drivers that declare `long long global_CM[NUM_EVENTS]` still compile. */
#define NUM_EVENTS 4

#ifdef __cplusplus
extern "C" {
#endif

/* A node's collision rule: function plus its parameter block (reference lb.h:59-62).
 * The library identifies the rule by the function's address, so only the dynamics
 * functions exported below (bgk, bounceBack and the boundaries.h functions) run on the GPU. */
typedef struct {
    void (*dynamicsFun)(double *fPop, void *selfData);
    void *selfData;
} Dynamics;

/* One lattice node: nine populations and its dynamics (reference lb.h:72-75). */
typedef struct {
    double fPop[9];
    Dynamics *dynamics;
} Node;

void constructNode(Node *node);                                   /* reference lb.h:77 */
void iniEquilibrium(Node *node, double rho, double ux, double uy); /* reference lb.h:78 */

/* The simulation: sizes, two host node arrays and their column tables (reference
 * lb.h:87-93).  `device` is appended for the GPU copy; drivers embed Simulation by value and
 * must leave it alone (it is zero for a lattice that has not run a step yet). */
typedef struct {
    int lx, ly;
    Node *memoryChunk;
    Node *tmpMemoryChunk;
    Node **lattice;
    Node **tmpLattice;
    void *device;
} Simulation;

/* Defined by the application driver, as in the reference (reference lb.h:97). */
void updateZeroGradientBoundary();

/* One-step form: in-place collision, then propagation and buffer swap
 * (reference lb.h:100-104, lb.c:172-348). */
void collide(Simulation *sim);
void collide_openmp(Simulation *sim);
void propagate(Simulation *sim);
void propagate_openmp(Simulation *sim);
void finalize_stream(Simulation *sim);

/* Fused collision + propagation; finalize_stream then swaps (reference lb.h:107-108,
 * lb.c:353-437). */
void collide_with_stream(Simulation *sim);
void collide_with_stream_openmp(Simulation *sim);

/* Two time steps per call, result left in `lattice` with no swap (reference lb.h:111-122,
 * lb.c:442-1779).  tight_block needs lx and ly to be multiples of blk_size and the panel
 * forms need ly (panel_iy) or lx (panel_ix) to be one; otherwise the call records
 * LB_ERR_BLOCK_SIZE and leaves the lattice unchanged. */
void collide_tight(Simulation *sim);
void collide_tight2(Simulation *sim);
void collide_tight_openmp(Simulation *sim);
void collide_tight_block(Simulation *sim);
void collide_tight_block_openmp(Simulation *sim);
void collide_tight_panel_ix(Simulation *sim);
void collide_tight_panel_iy(Simulation *sim);
void collide_tight_panel_iy_openmp(Simulation *sim);

/* Construction (reference lb.h:125-127, lb.c:85-121).  constructSim accepts
 * 1 <= lx <= LBGPU_MAX_LX and 1 <= ly <= LBGPU_MAX_LY (lbgpu.h: 2^20 and 65533, CUDA's grid
 * limit); other sizes leave *sim zeroed and record LB_ERR_ARG. */
void constructSim(Simulation *sim, int lx, int ly);
void destructSim(Simulation *sim);
void setDynamics(Simulation *sim, int iX, int iY, Dynamics *dyn);

/* Periodic wrap of the populations streamed into the ghost ring (reference lb.h:129,
 * lb.c:1783-1817) and text output of the current lattice (reference lb.h:130-131,
 * lb.c:1822-1866); the output functions first copy the device lattice back. */
void makePeriodic(Simulation *sim);
void saveVel(Simulation *sim, char fName[]);
void saveF(Simulation *sim, int iPop, char fName[]);

/* Host helpers drivers call directly (reference lb.h:137-143, lb.c:134-166). */
void computeMacros(double *f, double *rho, double *ux, double *uy);
double computeEquilibrium(int iPop, double rho, double ux, double uy, double uSqr);
void bgk(double *fPop, void *selfData);

#ifdef __cplusplus
}
#endif
#endif
