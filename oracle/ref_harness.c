/* ref_harness.c -- TEST INFRASTRUCTURE ONLY (never shipped, never measured as the product).
 *
 * A small host driver for the reference implementation's own lattice API.  oracle/Makefile
 * compiles this file together with the UNMODIFIED reference sources lb.c and boundaries.c
 * (read where they lie in the reference checkout) into oracle/_ref/libref_lb_{serial,omp}.so.
 * The tests use those libraries to produce golden populations, and bench.py's reference arm
 * uses the OpenMP one as the timed CPU baseline.
 *
 * What the driver does mirrors the reference's application driver unsteady.c:
 *   - the global variables lb.c declares extern (lb.c:30-38) are defined here, as the
 *     application driver defines them (unsteady.c:41-54);
 *   - the flow constants follow setConstants (unsteady.c:91-103): nu = uMax*2*r/Re,
 *     omega = 1/(3 nu + 1/2);
 *   - the boundary data follow iniData (unsteady.c:113-142) and the geometry follows
 *     iniGeometry (unsteady.c:162-199), with two options the reference driver hard-codes:
 *     the wall kind (regularized u=0, unsteady.c:185-188, or full-way bounce-back) and the
 *     outlet kind (zero-gradient extrapolated density through the `pressureBoundary`
 *     global, unsteady.c:205-214, or a constant density kept in a private array);
 *   - the time loop follows unsteady.c:424-531: per call ZGB update (when the outlet is
 *     ZGB), collision_func, then stream_func for the one-step variants.
 * Everything here is plain C in this repository's own words; no reference code is copied.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include "lb.h"
#include "boundaries.h"
#ifdef _OPENMP
#include <omp.h>
#endif

/* Globals the reference library reads (declared extern at lb.c:30-38). */
PressureBCData *pressureBoundary;
int blk_size = 1;
double *myrho1, *myrho2;
int iT = 0, count = 0;
int thread_block = 1;
int NUM_THREADS = 1;
long long global_CM[NUM_EVENTS];

enum { REF_WALL_REGULARIZED = 0, REF_WALL_BOUNCEBACK = 1 };
enum { REF_OUTLET_ZGB = 0, REF_OUTLET_CONST = 1 };
enum { REF_ORIGIN = 0, REF_COMBINE = 1, REF_TIGHT = 2, REF_TIGHT_BLOCK = 3, REF_PANEL = 4 };

static Simulation g_sim;
static int g_lx, g_ly, g_outlet, g_ready;
static double g_omega, g_umax;
static Dynamics g_bulk, g_bounce, g_upper, g_lower;
static VelocityBCData g_wall;
static VelocityBCData *g_inlet;
static PressureBCData *g_const_outlet;
static Dynamics *g_left, *g_right;

/* Poiseuille inflow profile, same expression as the application driver
 * (unsteady.c:155-159): 4 uMax / L^2 * (L y - y^2), y = iY-1, L = ly-1. */
static double ref_poiseuille(int iY)
{
    double y = (double)(iY - 1);
    double L = (double)(g_ly - 1);
    return 4. * g_umax / (L * L) * (L * y - y * y);
}

/* Zero-gradient outlet update of the application driver (unsteady.c:205-214). */
static void ref_zgb_update(void)
{
    int iY;
    double rho1, ux1, uy1, rho2, ux2, uy2;
    for (iY = 2; iY <= g_ly - 1; ++iY) {
        computeMacros(g_sim.lattice[g_lx - 1][iY].fPop, &rho1, &ux1, &uy1);
        computeMacros(g_sim.lattice[g_lx - 2][iY].fPop, &rho2, &ux2, &uy2);
        pressureBoundary[iY].rho = 4. / 3. * rho1 - 1. / 3. * rho2;
        pressureBoundary[iY].uPar = 0.;
    }
}

static void custom_free(void);

void ref_free(void)
{
    custom_free();
    if (!g_ready) return;
    destructSim(&g_sim);
    free(g_inlet); free(g_const_outlet); free(pressureBoundary);
    free(g_left); free(g_right); free(myrho1); free(myrho2);
    g_inlet = 0; g_const_outlet = 0; pressureBoundary = 0; g_left = g_right = 0;
    myrho1 = myrho2 = 0;
    g_ready = 0;
}

/* Build the channel.  poison_tmp != 0 fills every population of the second buffer with NaN
 * right after construction (the corner stale-slot probe). Returns omega. */
double ref_setup(int lx, int ly, int obst_x, int obst_y, int obst_r, double uMax, double Re,
                 int wall_kind, int outlet_kind, int poison_tmp)
{
    int iX, iY;
    double nu;
    ref_free();
    g_lx = lx; g_ly = ly; g_umax = uMax; g_outlet = outlet_kind;
    nu = uMax * 2. * obst_r / Re;
    g_omega = 1. / (3 * nu + 1. / 2.);

    g_bulk.dynamicsFun = &bgk;          g_bulk.selfData = (void *)&g_omega;
    g_bounce.dynamicsFun = &bounceBack; g_bounce.selfData = 0;
    g_wall.bulkDynamics = &g_bulk; g_wall.ux = 0.; g_wall.uy = 0.;
    g_upper.dynamicsFun = &upperRegularized; g_upper.selfData = (void *)&g_wall;
    g_lower.dynamicsFun = &lowerRegularized; g_lower.selfData = (void *)&g_wall;

    g_inlet = (VelocityBCData *)calloc(ly + 2, sizeof(VelocityBCData));
    g_const_outlet = (PressureBCData *)calloc(ly + 2, sizeof(PressureBCData));
    pressureBoundary = (PressureBCData *)calloc(ly + 2, sizeof(PressureBCData));
    g_left = (Dynamics *)calloc(ly + 2, sizeof(Dynamics));
    g_right = (Dynamics *)calloc(ly + 2, sizeof(Dynamics));
    myrho1 = (double *)calloc(ly + 2, sizeof(double));
    myrho2 = (double *)calloc(ly + 2, sizeof(double));
    for (iY = 2; iY <= ly - 1; ++iY) {
        g_inlet[iY].bulkDynamics = &g_bulk; g_inlet[iY].uy = 0.;
        pressureBoundary[iY].bulkDynamics = &g_bulk;
        pressureBoundary[iY].rho = 1.; pressureBoundary[iY].uPar = 0.;
        g_const_outlet[iY].bulkDynamics = &g_bulk;
        g_const_outlet[iY].rho = 1.; g_const_outlet[iY].uPar = 0.;
        g_left[iY].dynamicsFun = &leftRegularized;
        g_left[iY].selfData = (void *)&g_inlet[iY];
        g_right[iY].dynamicsFun = &rightPressureRegularized;
        g_right[iY].selfData = (outlet_kind == REF_OUTLET_ZGB) ? (void *)&pressureBoundary[iY]
                                                               : (void *)&g_const_outlet[iY];
    }

    constructSim(&g_sim, lx, ly);
    if (poison_tmp) {
        size_t n = (size_t)(lx + 2) * (size_t)(ly + 2), k;
        int i;
        for (k = 0; k < n; ++k)
            for (i = 0; i < 9; ++i) g_sim.tmpMemoryChunk[k].fPop[i] = NAN;
    }

    for (iX = 1; iX <= lx; ++iX) {
        for (iY = 1; iY <= ly; ++iY) {
            iniEquilibrium(&g_sim.lattice[iX][iY], 1., ref_poiseuille(iY), 0.);
            if ((iX - obst_x) * (iX - obst_x) + (iY - obst_y) * (iY - obst_y) <= obst_r * obst_r)
                setDynamics(&g_sim, iX, iY, &g_bounce);
            else
                setDynamics(&g_sim, iX, iY, &g_bulk);
        }
    }
    for (iX = 1; iX <= lx; ++iX) {
        if (wall_kind == REF_WALL_BOUNCEBACK) {
            setDynamics(&g_sim, iX, 1, &g_bounce);
            setDynamics(&g_sim, iX, ly, &g_bounce);
        } else {
            setDynamics(&g_sim, iX, 1, &g_lower);
            setDynamics(&g_sim, iX, ly, &g_upper);
        }
    }
    for (iY = 2; iY <= ly - 1; ++iY) {
        g_inlet[iY].ux = ref_poiseuille(iY);
        setDynamics(&g_sim, 1, iY, &g_left[iY]);
        setDynamics(&g_sim, lx, iY, &g_right[iY]);
    }
    iT = 0;
    g_ready = 1;
    return g_omega;
}

/* ---------------------------------------------------------------------------------------
 * Generic lattice: any per-node dynamics assignment expressed in the oracle's tag and table
 * form (lbm_oracle.h), so every boundary function of boundaries.h can be pinned.  One
 * Dynamics object and one VelocityBCData/PressureBCData per (table, coordinate); the
 * right-side pressure table IS the `pressureBoundary` global, so zero-gradient rows update
 * the data their outlet nodes read, as in the application driver.
 * ------------------------------------------------------------------------------------- */
static VelocityBCData *g_vel[4];
static PressureBCData *g_prs[4];
static Dynamics *g_kind_dyn[19];
static unsigned char *g_zgb_rows;
static int g_custom;

static void custom_free(void)
{
    int k;
    for (k = 0; k < 4; ++k) { free(g_vel[k]); g_vel[k] = 0; }
    for (k = 0; k < 3; ++k) { free(g_prs[k]); g_prs[k] = 0; }
    g_prs[3] = 0;
    for (k = 0; k < 19; ++k) { free(g_kind_dyn[k]); g_kind_dyn[k] = 0; }
    free(g_zgb_rows); g_zgb_rows = 0;
    g_custom = 0;
}

int ref_setup_custom(int lx, int ly, double omega, const unsigned char *tag, const double *bc,
                     const unsigned char *zgb_row, const double *lat0, const double *tmp0)
{
    static void (*const kind_fun[19])(double *, void *) = {
        0, &bgk, &bounceBack,
        &upperZouHe, &lowerZouHe, &leftZouHe, &rightZouHe,
        &upperPressureZouHe, &lowerPressureZouHe, &leftPressureZouHe, &rightPressureZouHe,
        &upperRegularized, &lowerRegularized, &leftRegularized, &rightRegularized,
        &upperPressureRegularized, &lowerPressureRegularized, &leftPressureRegularized,
        &rightPressureRegularized };
    const int nb = (lx > ly ? lx : ly) + 2, ny2 = ly + 2;
    int k, c, X, Y, i;
    ref_free();
    custom_free();
    g_lx = lx; g_ly = ly; g_omega = omega; g_outlet = REF_OUTLET_CONST;
    g_bulk.dynamicsFun = &bgk; g_bulk.selfData = (void *)&g_omega;
    for (k = 0; k < 4; ++k) {
        g_vel[k] = (VelocityBCData *)calloc(nb, sizeof(VelocityBCData));
        for (c = 0; c < nb; ++c) {
            g_vel[k][c].bulkDynamics = &g_bulk;
            g_vel[k][c].ux = bc[((0 * 4 + k) * 2 + 0) * nb + c];
            g_vel[k][c].uy = bc[((0 * 4 + k) * 2 + 1) * nb + c];
        }
    }
    pressureBoundary = (PressureBCData *)calloc(nb, sizeof(PressureBCData));
    for (k = 0; k < 4; ++k) {
        g_prs[k] = (k == 3) ? pressureBoundary : (PressureBCData *)calloc(nb, sizeof(PressureBCData));
        for (c = 0; c < nb; ++c) {
            g_prs[k][c].bulkDynamics = &g_bulk;
            g_prs[k][c].rho = bc[((1 * 4 + k) * 2 + 0) * nb + c];
            g_prs[k][c].uPar = bc[((1 * 4 + k) * 2 + 1) * nb + c];
        }
    }
    for (k = 3; k < 19; ++k) {
        int j = k - 3, side = j % 4, pressure = (j / 4) & 1;
        g_kind_dyn[k] = (Dynamics *)calloc(nb, sizeof(Dynamics));
        for (c = 0; c < nb; ++c) {
            g_kind_dyn[k][c].dynamicsFun = kind_fun[k];
            g_kind_dyn[k][c].selfData = pressure ? (void *)&g_prs[side][c] : (void *)&g_vel[side][c];
        }
    }
    g_bounce.dynamicsFun = &bounceBack; g_bounce.selfData = 0;
    myrho1 = (double *)calloc(ny2, sizeof(double));
    myrho2 = (double *)calloc(ny2, sizeof(double));
    g_zgb_rows = (unsigned char *)calloc(ny2, 1);
    for (Y = 0; Y < ny2; ++Y) g_zgb_rows[Y] = zgb_row ? zgb_row[Y] : 0;

    constructSim(&g_sim, lx, ly);
    for (X = 0; X < lx + 2; ++X)
        for (Y = 0; Y < ny2; ++Y)
            for (i = 0; i < 9; ++i) {
                g_sim.lattice[X][Y].fPop[i] = lat0[((size_t)X * ny2 + Y) * 9 + i];
                g_sim.tmpLattice[X][Y].fPop[i] = tmp0[((size_t)X * ny2 + Y) * 9 + i];
            }
    for (X = 1; X <= lx; ++X)
        for (Y = 1; Y <= ly; ++Y) {
            int t = tag[X * ny2 + Y];
            if (t == 1) setDynamics(&g_sim, X, Y, &g_bulk);
            else if (t == 2) setDynamics(&g_sim, X, Y, &g_bounce);
            else if (t >= 3 && t < 19) {
                int side = (t - 3) % 4;
                setDynamics(&g_sim, X, Y, &g_kind_dyn[t][side <= 1 ? X : Y]);
            }
        }
    iT = 0;
    g_custom = 1;
    g_ready = 1;
    return 0;
}

/* Zero-gradient update restricted to the flagged rows of a generic lattice. */
static void custom_zgb_update(void)
{
    int Y;
    double rho1, ux1, uy1, rho2, ux2, uy2;
    for (Y = 0; Y < g_ly + 2; ++Y) {
        if (!g_zgb_rows[Y]) continue;
        computeMacros(g_sim.lattice[g_lx - 1][Y].fPop, &rho1, &ux1, &uy1);
        computeMacros(g_sim.lattice[g_lx - 2][Y].fPop, &rho2, &ux2, &uy2);
        pressureBoundary[Y].rho = 4. / 3. * rho1 - 1. / 3. * rho2;
        pressureBoundary[Y].uPar = 0.;
    }
}

/* Block sizes read by the tight_block / panel variants and by the OpenMP schedules. */
void ref_set_blocking(int blk, int tblock, int nthreads)
{
    blk_size = blk;
    thread_block = tblock;
#ifdef _OPENMP
    if (nthreads > 0) { omp_set_num_threads(nthreads); NUM_THREADS = nthreads; }
#else
    (void)nthreads;
#endif
}

int ref_has_openmp(void)
{
#ifdef _OPENMP
    return 1;
#else
    return 0;
#endif
}

int ref_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Run `nsteps` time steps with the chosen variant through the reference entry points.
 * Two-step variants advance 2 steps per call; nsteps is rounded up to an even count exactly
 * as the application loop does (unsteady.c:425-429). Returns the steps actually run. */
int ref_run(int variant, int use_openmp, int nsteps)
{
    void (*collision_func)(Simulation *) = 0;
    void (*stream_func)(Simulation *) = 0;
    int two = 0, done = 0;
    if (!g_ready) return -1;
    switch (variant) {
    case REF_ORIGIN:
        collision_func = use_openmp ? &collide_openmp : &collide;
        stream_func = use_openmp ? &propagate_openmp : &propagate;
        break;
    case REF_COMBINE:
        collision_func = use_openmp ? &collide_with_stream_openmp : &collide_with_stream;
        stream_func = &finalize_stream;
        break;
    case REF_TIGHT:
        collision_func = use_openmp ? &collide_tight_openmp : &collide_tight; two = 1; break;
    case REF_TIGHT_BLOCK:
        collision_func = use_openmp ? &collide_tight_block_openmp : &collide_tight_block; two = 1; break;
    case REF_PANEL:
        collision_func = use_openmp ? &collide_tight_panel_iy_openmp : &collide_tight_panel_iy; two = 1; break;
    default:
        return -2;
    }
    for (iT = 0; iT < nsteps; iT += two ? 2 : 1) {
        if (g_custom) custom_zgb_update();
        else if (g_outlet == REF_OUTLET_ZGB) ref_zgb_update();
        collision_func(&g_sim);
        if (!two) stream_func(&g_sim);
        done += two ? 2 : 1;
    }
    return done;
}

/* Copy populations of the current `lattice` (which_buf 0) or `tmpLattice` (1) into
 * out[((X*(ly+2)) + Y)*9 + i], ghost ring included. */
void ref_dump(int which_buf, double *out)
{
    int X, Y, i;
    Node **lat = which_buf ? g_sim.tmpLattice : g_sim.lattice;
    for (X = 0; X < g_lx + 2; ++X)
        for (Y = 0; Y < g_ly + 2; ++Y)
            for (i = 0; i < 9; ++i)
                out[((size_t)X * (g_ly + 2) + Y) * 9 + i] = lat[X][Y].fPop[i];
}

/* Outlet densities, and the two-step variants' density scratch (lb.c:471-480, :527-531). */
void ref_outlet_state(double *press_rho, double *rho1, double *rho2)
{
    int Y;
    for (Y = 0; Y < g_ly + 2; ++Y) {
        press_rho[Y] = pressureBoundary[Y].rho;
        rho1[Y] = myrho1[Y];
        rho2[Y] = myrho2[Y];
    }
}
