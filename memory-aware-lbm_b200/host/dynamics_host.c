/* dynamics_host.c -- host implementations of the per-node functions of lb.h/boundaries.h.
 *
 * Drivers call these directly on single nodes (the application driver's zero-gradient update
 * calls computeMacros, unsteady.c:209-210; a custom driver may collide a node by hand), and
 * the GPU library reads a node's rule from the *address* of the function in its Dynamics.
 * The arithmetic follows the reference's expressions and order (lb.c:62-166,
 * boundaries.c:48-414) so that host and device results agree bit for bit; this file is
 * compiled without FMA contraction.  bounceBack keeps its scratch on the stack (the
 * reference uses a static array, boundaries.c:49, which races under OpenMP).
 */
#include <stddef.h>
#include "lb.h"
#include "boundaries.h"

static const double T[9] = { 4. / 9., 1. / 9., 1. / 9., 1. / 9., 1. / 9.,
                             1. / 36., 1. / 36., 1. / 36., 1. / 36. };
static const int C[9][2] = { { 0, 0 }, { 1, 0 }, { 0, 1 }, { -1, 0 }, { 0, -1 },
                             { 1, 1 }, { -1, 1 }, { -1, -1 }, { 1, -1 } };

enum { UP = 0, LO = 1, LE = 2, RI = 3 };

void constructNode(Node *node)
{
    int i;
    for (i = 0; i < 9; ++i) node->fPop[i] = 0.;
    node->dynamics = 0;
}

void computeMacros(double *f, double *rho, double *ux, double *uy)
{
    double top = f[2] + f[5] + f[6];
    double mid = f[0] + f[1] + f[3];
    double bot = f[4] + f[7] + f[8];
    *rho = top + mid + bot;
    *ux = (f[1] + f[5] + f[8] - (f[3] + f[6] + f[7])) / (*rho);
    *uy = (top - bot) / (*rho);
}

double computeEquilibrium(int iPop, double rho, double ux, double uy, double uSqr)
{
    double cu = C[iPop][0] * ux + C[iPop][1] * uy;
    return rho * T[iPop] * (1. + 3. * cu + 4.5 * cu * cu - 1.5 * uSqr);
}

void iniEquilibrium(Node *node, double rho, double ux, double uy)
{
    double usqr = ux * ux + uy * uy;
    int i;
    for (i = 0; i < 9; ++i) node->fPop[i] = computeEquilibrium(i, rho, ux, uy, usqr);
}

void bgk(double *fPop, void *selfData)
{
    double omega = *(double *)selfData;
    double rho, ux, uy, usqr;
    int i;
    computeMacros(fPop, &rho, &ux, &uy);
    usqr = ux * ux + uy * uy;
    for (i = 0; i < 9; ++i) {
        fPop[i] *= (1 - omega);
        fPop[i] += omega * computeEquilibrium(i, rho, ux, uy, usqr);
    }
}

void bounceBack(double *fPop, void *selfData)
{
    double t;
    (void)selfData;
    t = fPop[1]; fPop[1] = fPop[3]; fPop[3] = t;
    t = fPop[2]; fPop[2] = fPop[4]; fPop[4] = t;
    t = fPop[5]; fPop[5] = fPop[7]; fPop[7] = t;
    t = fPop[6]; fPop[6] = fPop[8]; fPop[8] = t;
}

static double known_sum(const double *f, int side)
{
    switch (side) {
    case UP: return f[0] + f[3] + f[1] + 2 * (f[6] + f[2] + f[5]);
    case LO: return f[0] + f[3] + f[1] + 2 * (f[8] + f[4] + f[7]);
    case RI: return f[0] + f[2] + f[4] + 2 * (f[1] + f[5] + f[8]);
    default: return f[0] + f[2] + f[4] + 2 * (f[3] + f[6] + f[7]);
    }
}

static double wall_rho(const double *f, int side, double un)
{
    double s = known_sum(f, side);
    return (side == UP || side == RI) ? 1. / (1. + un) * s : 1. / (1. - un) * s;
}

static double wall_u(const double *f, int side, double rho)
{
    double s = known_sum(f, side);
    return (side == UP || side == RI) ? -1. + 1. / rho * s : 1. - 1. / rho * s;
}

static void zouhe(double *f, int side, double ux, double uy, double rho)
{
    switch (side) {
    case UP:
        f[7] = f[5] + 0.5 * (f[1] - f[3]) - rho * uy / 6 - rho * ux / 2.;
        f[8] = f[6] + 0.5 * (f[3] - f[1]) - rho * uy / 6 + rho * ux / 2.;
        f[4] = f[2] - 2. / 3. * rho * uy;
        break;
    case LO:
        f[6] = f[8] + 0.5 * (f[1] - f[3]) + rho * uy / 6 - rho * ux / 2.;
        f[5] = f[7] + 0.5 * (f[3] - f[1]) + rho * uy / 6 + rho * ux / 2.;
        f[2] = f[4] + 2. / 3. * rho * uy;
        break;
    case RI:
        f[6] = f[8] + 0.5 * (f[4] - f[2]) - rho * ux / 6 + rho * uy / 2.;
        f[7] = f[5] + 0.5 * (f[2] - f[4]) - rho * ux / 6 - rho * uy / 2.;
        f[3] = f[1] - 2. / 3. * rho * ux;
        break;
    default:
        f[5] = f[7] + 0.5 * (f[4] - f[2]) + rho * ux / 6. + rho * uy / 2.;
        f[8] = f[6] + 0.5 * (f[2] - f[4]) + rho * ux / 6. - rho * uy / 2.;
        f[1] = f[3] + 2. / 3. * rho * ux;
        break;
    }
}

static void regularize(double *f, int side, double rho, double ux, double uy)
{
    double fe[9], n[9], pxx, pyy, pxy;
    int i;
    for (i = 0; i < 9; ++i) {
        fe[i] = computeEquilibrium(i, rho, ux, uy, ux * ux + uy * uy);
        n[i] = f[i] - fe[i];
    }
    switch (side) {
    case UP:
        pxx = n[1] + n[3] + 2. * (n[5] + n[6]);
        pyy = 2. * (n[6] + n[2] + n[5]);
        pxy = 2. * (n[5] - n[6]);
        break;
    case LO:
        pxx = n[1] + n[3] + 2. * (n[7] + n[8]);
        pyy = 2. * (n[4] + n[7] + n[8]);
        pxy = 2. * (n[7] - n[8]);
        break;
    case RI:
        pxx = 2. * (n[1] + n[5] + n[8]);
        pyy = n[2] + n[4] + 2. * (n[5] + n[8]);
        pxy = 2. * (n[5] - n[8]);
        break;
    default:
        pxx = 2. * (n[3] + n[6] + n[7]);
        pyy = n[2] + n[4] + 2. * (n[6] + n[7]);
        pxy = 2. * (n[7] - n[6]);
        break;
    }
    for (i = 0; i < 9; ++i)
        f[i] = fe[i] + 9. / 2. * T[i] *
               ((C[i][0] * C[i][0] - 1. / 3.) * pxx + (C[i][1] * C[i][1] - 1. / 3.) * pyy +
                2. * C[i][0] * C[i][1] * pxy);
}

static void chain_bulk(double *f, Dynamics *bulk)
{
    bulk->dynamicsFun(f, bulk->selfData);
}

static void velocity_rule(double *f, void *selfData, int side, int regularized)
{
    VelocityBCData *d = (VelocityBCData *)selfData;
    double rho = wall_rho(f, side, (side == UP || side == LO) ? d->uy : d->ux);
    if (regularized) regularize(f, side, rho, d->ux, d->uy);
    else zouhe(f, side, d->ux, d->uy, rho);
    chain_bulk(f, d->bulkDynamics);
}

static void pressure_rule(double *f, void *selfData, int side, int regularized)
{
    PressureBCData *d = (PressureBCData *)selfData;
    double u = wall_u(f, side, d->rho);
    double ux = (side == UP || side == LO) ? d->uPar : u;
    double uy = (side == UP || side == LO) ? u : d->uPar;
    if (regularized) regularize(f, side, d->rho, ux, uy);
    else zouhe(f, side, ux, uy, d->rho);
    chain_bulk(f, d->bulkDynamics);
}

void upperZouHe(double *f, void *s) { velocity_rule(f, s, UP, 0); }
void lowerZouHe(double *f, void *s) { velocity_rule(f, s, LO, 0); }
void leftZouHe(double *f, void *s) { velocity_rule(f, s, LE, 0); }
void rightZouHe(double *f, void *s) { velocity_rule(f, s, RI, 0); }
void upperPressureZouHe(double *f, void *s) { pressure_rule(f, s, UP, 0); }
void lowerPressureZouHe(double *f, void *s) { pressure_rule(f, s, LO, 0); }
void leftPressureZouHe(double *f, void *s) { pressure_rule(f, s, LE, 0); }
void rightPressureZouHe(double *f, void *s) { pressure_rule(f, s, RI, 0); }
void upperRegularized(double *f, void *s) { velocity_rule(f, s, UP, 1); }
void lowerRegularized(double *f, void *s) { velocity_rule(f, s, LO, 1); }
void leftRegularized(double *f, void *s) { velocity_rule(f, s, LE, 1); }
void rightRegularized(double *f, void *s) { velocity_rule(f, s, RI, 1); }
void upperPressureRegularized(double *f, void *s) { pressure_rule(f, s, UP, 1); }
void lowerPressureRegularized(double *f, void *s) { pressure_rule(f, s, LO, 1); }
void leftPressureRegularized(double *f, void *s) { pressure_rule(f, s, LE, 1); }
void rightPressureRegularized(double *f, void *s) { pressure_rule(f, s, RI, 1); }

/* ---- cylinder channel builder (native interface) --------------------------------------
 * The application driver's geometry (unsteady.c:155-199) expressed as tags and tables:
 * obstacle disk of bounce-back nodes, walls on rows 1 and ly (regularized u = 0 or
 * bounce-back, corners included), regularized Poiseuille inlet on column 1 and regularized
 * pressure outlet on column lx for rows 2..ly-1.  omega = 1/(3 nu + 1/2), nu = uMax 2r/Re
 * (unsteady.c:100-103). */
#include <string.h>
#include <stdint.h>

static double poiseuille(int iY, int ly, double uMax)
{
    double y = (double)(iY - 1);
    double L = (double)(ly - 1);
    return 4. * uMax / (L * L) * (L * y - y * y);
}

double lbgpu_build_cylinder(int lx, int ly, int obst_x, int obst_y, int obst_r, double umax,
                            double re, int wall_kind, int outlet_kind, uint8_t *tag,
                            double *bc, uint8_t *zgb_row, double *f)
{
    const int ny2 = ly + 2;
    const int nb = (lx > ly ? lx : ly) + 2;
    double nu = umax * 2. * obst_r / re;
    double omega = 1. / (3 * nu + 1. / 2.);
    int X, Y;
    if (tag) memset(tag, 0, (size_t)(lx + 2) * ny2);
    if (bc) memset(bc, 0, sizeof(double) * 16 * (size_t)nb);
    if (zgb_row) memset(zgb_row, 0, (size_t)ny2);
    if (f) memset(f, 0, sizeof(double) * 9 * (size_t)(lx + 2) * ny2);
    for (X = 1; X <= lx; ++X)
        for (Y = 1; Y <= ly; ++Y) {
            if (f) {
                Node nd;
                iniEquilibrium(&nd, 1., poiseuille(Y, ly, umax), 0.);
                memcpy(&f[((size_t)X * ny2 + Y) * 9], nd.fPop, sizeof nd.fPop);
            }
            if (tag)
                tag[(size_t)X * ny2 + Y] =
                    ((X - obst_x) * (X - obst_x) + (Y - obst_y) * (Y - obst_y) <= obst_r * obst_r)
                        ? 2 : 1;
        }
    if (tag)
        for (X = 1; X <= lx; ++X) {
            tag[(size_t)X * ny2 + 1] = (wall_kind == 1) ? 2 : 12;    /* lower regularized */
            tag[(size_t)X * ny2 + ly] = (wall_kind == 1) ? 2 : 11;   /* upper regularized */
        }
    for (Y = 2; Y <= ly - 1; ++Y) {
        if (tag) {
            tag[(size_t)1 * ny2 + Y] = 13;                           /* left regularized */
            tag[(size_t)lx * ny2 + Y] = 18;                          /* right pressure reg. */
        }
        if (bc) {
            bc[(LE * 2 + 0) * nb + Y] = poiseuille(Y, ly, umax);     /* velocity-left ux */
            bc[(LE * 2 + 1) * nb + Y] = 0.;
            bc[((4 + RI) * 2 + 0) * nb + Y] = 1.;                    /* pressure-right rho */
            bc[((4 + RI) * 2 + 1) * nb + Y] = 0.;
        }
        if (zgb_row) zgb_row[Y] = (outlet_kind == 0) ? 1 : 0;
    }
    return omega;
}
