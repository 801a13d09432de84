/* lbdriver.c -- cylinder-channel host driver written against the drop-in lb.h/boundaries.h
 * interface only, the way the reference's application driver unsteady.c is.
 *
 * It builds the channel through constructSim / iniEquilibrium / setDynamics with Dynamics and
 * boundary-data objects it owns (unsteady.c:62-79, :113-199), then runs the reference's time
 * loop (unsteady.c:424-531): before each call the zero-gradient outlet update when the outlet
 * is extrapolated (unsteady.c:205-214), then the variant's collision function and, for the
 * one-step variants, its stream function.  Two-step variants advance two steps per call.
 *
 * Options beyond the application driver: bounce-back walls instead of regularized ones, and
 * a constant-density outlet whose data live outside `pressureBoundary` (so the two-step
 * variants' extrapolation, which writes that global, leaves it alone).
 *
 * Used by the command-line driver (lbgpu_unsteady), by bench.py's end-to-end leg and by the
 * drop-in tests; lbdrv_run reports the wall time of the loop, which includes the first
 * upload of the host lattice and the final copy back (lbSyncToHost).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>
#include "lb.h"
#include "boundaries.h"
#include "lbgpu.h"
#include "lbdriver.h"

/* Driver globals of the drop-in interface (the reference's lb.c reads them, lb.c:30-38). */
extern PressureBCData *pressureBoundary;
extern double *myrho1, *myrho2;
extern int blk_size;

static double now_s(void)
{
    struct timeval tv;
    gettimeofday(&tv, 0);
    return (double)tv.tv_sec + (double)tv.tv_usec * 1e-6;
}

typedef struct {
    Simulation sim;
    int lx, ly, outlet;
    double omega, umax;
    Dynamics bulk, bounce, upper, lower;
    VelocityBCData wall;
    VelocityBCData *inlet;
    PressureBCData *outlet_data;   /* constant-density outlet */
    PressureBCData *zgb_data;      /* becomes `pressureBoundary` for the extrapolated outlet */
    Dynamics *left, *right;
    double *rho1, *rho2;
} Channel;

static double poiseuille(const Channel *ch, int iY)
{
    double y = (double)(iY - 1);
    double L = (double)(ch->ly - 1);
    return 4. * ch->umax / (L * L) * (L * y - y * y);
}

static void zgb_update(Channel *ch)
{
    int iY;
    double rho1, ux1, uy1, rho2, ux2, uy2;
    for (iY = 2; iY <= ch->ly - 1; ++iY) {
        computeMacros(ch->sim.lattice[ch->lx - 1][iY].fPop, &rho1, &ux1, &uy1);
        computeMacros(ch->sim.lattice[ch->lx - 2][iY].fPop, &rho2, &ux2, &uy2);
        pressureBoundary[iY].rho = 4. / 3. * rho1 - 1. / 3. * rho2;
        pressureBoundary[iY].uPar = 0.;
    }
}

static void channel_free(Channel *ch)
{
    destructSim(&ch->sim);
    if (pressureBoundary == ch->zgb_data) pressureBoundary = 0;
    if (myrho1 == ch->rho1) myrho1 = 0;
    if (myrho2 == ch->rho2) myrho2 = 0;
    free(ch->inlet); free(ch->outlet_data); free(ch->zgb_data);
    free(ch->left); free(ch->right); free(ch->rho1); free(ch->rho2);
    free(ch);
}

static Channel *channel_build(const lbdrv_config *c)
{
    int iX, iY;
    Channel *ch = (Channel *)calloc(1, sizeof(Channel));
    double nu;
    if (!ch) return 0;
    ch->lx = c->lx; ch->ly = c->ly; ch->umax = c->umax; ch->outlet = c->outlet;
    nu = c->umax * 2. * c->obst_r / c->re;
    ch->omega = 1. / (3 * nu + 1. / 2.);
    ch->bulk.dynamicsFun = &bgk;          ch->bulk.selfData = (void *)&ch->omega;
    ch->bounce.dynamicsFun = &bounceBack; ch->bounce.selfData = 0;
    ch->wall.bulkDynamics = &ch->bulk;    ch->wall.ux = 0.; ch->wall.uy = 0.;
    ch->upper.dynamicsFun = &upperRegularized; ch->upper.selfData = (void *)&ch->wall;
    ch->lower.dynamicsFun = &lowerRegularized; ch->lower.selfData = (void *)&ch->wall;
    ch->inlet = (VelocityBCData *)calloc(c->ly + 2, sizeof(VelocityBCData));
    ch->outlet_data = (PressureBCData *)calloc(c->ly + 2, sizeof(PressureBCData));
    ch->zgb_data = (PressureBCData *)calloc(c->ly + 2, sizeof(PressureBCData));
    ch->left = (Dynamics *)calloc(c->ly + 2, sizeof(Dynamics));
    ch->right = (Dynamics *)calloc(c->ly + 2, sizeof(Dynamics));
    ch->rho1 = (double *)calloc(c->ly + 2, sizeof(double));
    ch->rho2 = (double *)calloc(c->ly + 2, sizeof(double));
    if (!ch->inlet || !ch->outlet_data || !ch->zgb_data || !ch->left || !ch->right || !ch->rho1 ||
        !ch->rho2) {
        channel_free(ch);
        return 0;
    }
    pressureBoundary = ch->zgb_data;
    myrho1 = ch->rho1;
    myrho2 = ch->rho2;
    blk_size = c->blk > 0 ? c->blk : 1;
    for (iY = 2; iY <= c->ly - 1; ++iY) {
        ch->inlet[iY].bulkDynamics = &ch->bulk; ch->inlet[iY].uy = 0.;
        ch->zgb_data[iY].bulkDynamics = &ch->bulk;
        ch->zgb_data[iY].rho = 1.; ch->zgb_data[iY].uPar = 0.;
        ch->outlet_data[iY].bulkDynamics = &ch->bulk;
        ch->outlet_data[iY].rho = 1.; ch->outlet_data[iY].uPar = 0.;
        ch->left[iY].dynamicsFun = &leftRegularized;
        ch->left[iY].selfData = (void *)&ch->inlet[iY];
        ch->right[iY].dynamicsFun = &rightPressureRegularized;
        ch->right[iY].selfData = (c->outlet == LBGPU_OUTLET_ZGB) ? (void *)&ch->zgb_data[iY]
                                                                 : (void *)&ch->outlet_data[iY];
    }
    constructSim(&ch->sim, c->lx, c->ly);
    if (!ch->sim.memoryChunk) { channel_free(ch); return 0; }
    if (c->sync_mode >= 0) lbSetSyncMode(&ch->sim, c->sync_mode);
    for (iX = 1; iX <= c->lx; ++iX)
        for (iY = 1; iY <= c->ly; ++iY) {
            iniEquilibrium(&ch->sim.lattice[iX][iY], 1., poiseuille(ch, iY), 0.);
            if ((iX - c->obst_x) * (iX - c->obst_x) + (iY - c->obst_y) * (iY - c->obst_y) <=
                c->obst_r * c->obst_r)
                setDynamics(&ch->sim, iX, iY, &ch->bounce);
            else
                setDynamics(&ch->sim, iX, iY, &ch->bulk);
        }
    for (iX = 1; iX <= c->lx; ++iX) {
        if (c->wall == LBGPU_WALL_BOUNCEBACK) {
            setDynamics(&ch->sim, iX, 1, &ch->bounce);
            setDynamics(&ch->sim, iX, c->ly, &ch->bounce);
        } else {
            setDynamics(&ch->sim, iX, 1, &ch->lower);
            setDynamics(&ch->sim, iX, c->ly, &ch->upper);
        }
    }
    for (iY = 2; iY <= c->ly - 1; ++iY) {
        ch->inlet[iY].ux = poiseuille(ch, iY);
        setDynamics(&ch->sim, 1, iY, &ch->left[iY]);
        setDynamics(&ch->sim, c->lx, iY, &ch->right[iY]);
    }
    return ch;
}

static __thread unsigned long long g_h2d, g_d2h;

void lbdrv_last_transfer_bytes(unsigned long long *h2d, unsigned long long *d2h)
{
    if (h2d) *h2d = g_h2d;
    if (d2h) *d2h = g_d2h;
}

int lbdrv_variant_steps(int variant)
{
    return (variant >= LBDRV_TIGHT) ? 2 : 1;
}

int lbdrv_run(const lbdrv_config *c, int nsteps, double *out, double *seconds)
{
    void (*collision_func)(Simulation *) = 0;
    void (*stream_func)(Simulation *) = 0;
    int two = 0, done = 0, X, Y, rc, t;
    double t0, t1;
    Channel *ch;
    if (!c || c->lx < 1 || c->ly < 1 || nsteps < 0) return -LB_ERR_ARG;
    switch (c->variant) {
    case LBDRV_ORIGIN: collision_func = &collide; stream_func = &propagate; break;
    case LBDRV_COMBINE: collision_func = &collide_with_stream; stream_func = &finalize_stream; break;
    case LBDRV_TIGHT: collision_func = &collide_tight; two = 1; break;
    case LBDRV_TIGHT_BLOCK: collision_func = &collide_tight_block; two = 1; break;
    case LBDRV_PANEL: collision_func = &collide_tight_panel_iy; two = 1; break;
    default: return -LB_ERR_ARG;
    }
    lbClearError();
    g_h2d = g_d2h = 0;
    ch = channel_build(c);
    if (!ch) {   /* constructSim records why (a size out of range, no host memory) */
        rc = lbGetLastError();
        return -(rc ? rc : LB_ERR_ALLOC);
    }
    t0 = now_s();
    for (t = 0; t < nsteps; t += two ? 2 : 1) {
        if (c->outlet == LBGPU_OUTLET_ZGB) zgb_update(ch);
        collision_func(&ch->sim);
        if (!two) stream_func(&ch->sim);
        done += two ? 2 : 1;
        if (lbGetLastError()) break;
    }
    lbSyncToHost(&ch->sim);
    t1 = now_s();
    lbGetTransferBytes(&ch->sim, &g_h2d, &g_d2h);
    if (seconds) *seconds = t1 - t0;
    rc = lbGetLastError();
    if (out && rc == LB_OK)
        for (X = 0; X < c->lx + 2; ++X)
            for (Y = 0; Y < c->ly + 2; ++Y)
                memcpy(&out[((size_t)X * (c->ly + 2) + Y) * 9], ch->sim.lattice[X][Y].fPop,
                       9 * sizeof(double));
    channel_free(ch);
    return rc == LB_OK ? done : -rc;
}
