/* lbdriver.h -- cylinder-channel host driver on the drop-in interface (liblbgpu.so).
 *
 * No counterpart function in the reference: it packages what the reference's application
 * driver unsteady.c does (channel set-up and time loop, unsteady.c:84-199 and :424-531) as a
 * callable function, so the drop-in interface can be driven from tests and benchmarks.
 */
#ifndef LBDRIVER_H
#define LBDRIVER_H

#ifdef __cplusplus
extern "C" {
#endif

enum { LBDRV_ORIGIN = 0, LBDRV_COMBINE = 1, LBDRV_TIGHT = 2, LBDRV_TIGHT_BLOCK = 3,
       LBDRV_PANEL = 4 };

typedef struct {
    int lx, ly;                  /* interior size */
    int obst_x, obst_y, obst_r;  /* obstacle disk, 1-based node coordinates */
    double umax, re;             /* Poiseuille peak velocity and Reynolds number */
    int wall;                    /* LBGPU_WALL_REGULARIZED or LBGPU_WALL_BOUNCEBACK */
    int outlet;                  /* LBGPU_OUTLET_ZGB or LBGPU_OUTLET_CONST */
    int variant;                 /* LBDRV_* entry-point family */
    int blk;                     /* blk_size for tight_block / panel */
    int sync_mode;               /* LB_SYNC_* or -1 for the library default */
} lbdrv_config;

/* Build the channel, run `nsteps` steps (two-step variants round up to even), copy the final
 * lattice into out[((X*(ly+2))+Y)*9+i] when out is not NULL and the loop's wall time into
 * *seconds.  Returns the number of steps run, or -LB_ERR_* on failure. */
int lbdrv_run(const lbdrv_config *cfg, int nsteps, double *out, double *seconds);

/* Bytes copied host->device and device->host by the calling thread's last lbdrv_run, from
 * its first step through the final copy-back (lbGetTransferBytes of its simulation). */
void lbdrv_last_transfer_bytes(unsigned long long *h2d, unsigned long long *d2h);

/* Steps advanced by one call of the variant's collision function (1 or 2). */
int lbdrv_variant_steps(int variant);

#ifdef __cplusplus
}
#endif
#endif
