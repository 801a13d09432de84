/* lbm_oracle.c -- TEST INFRASTRUCTURE ONLY: CPU restatement of the reference's D2Q9 step.
 *
 * Every function below states, in this repository's own code, what one reference function
 * computes, cited by file:line.  Arithmetic is IEEE double evaluated in the reference's
 * expression order (left-to-right sums, the same grouping of products and quotients) and is
 * compiled without FMA contraction (oracle/Makefile), so results are bit-identical to the
 * reference built the same way.  The product never links this file.
 */
#include <stdlib.h>
#include <string.h>
#include "lbm_oracle.h"

/* D2Q9 lattice: weights, velocities and opposite directions (lb.c:48-55, boundaries.c:32-42).
 * Direction order 0:(0,0) 1:(1,0) 2:(0,1) 3:(-1,0) 4:(0,-1) 5:(1,1) 6:(-1,1) 7:(-1,-1) 8:(1,-1). */
static const double W[9] = { 4. / 9., 1. / 9., 1. / 9., 1. / 9., 1. / 9.,
                             1. / 36., 1. / 36., 1. / 36., 1. / 36. };
static const int CX[9] = { 0, 1, 0, -1, 0, 1, -1, -1, 1 };
static const int CY[9] = { 0, 0, 1, 0, -1, 1, 1, -1, -1 };
static const int OPP[9] = { 0, 3, 4, 1, 2, 7, 8, 5, 6 };

enum { SIDE_UPPER = 0, SIDE_LOWER = 1, SIDE_LEFT = 2, SIDE_RIGHT = 3 };

/* Density and velocity from the three horizontal line sums (lb.c:134-141). */
void orc_macros(const double *f, double *rho, double *ux, double *uy)
{
    double top = f[2] + f[5] + f[6];
    double mid = f[0] + f[1] + f[3];
    double bot = f[4] + f[7] + f[8];
    double r = top + mid + bot;
    *rho = r;
    *ux = (f[1] + f[5] + f[8] - (f[3] + f[6] + f[7])) / r;
    *uy = (top - bot) / r;
}

/* Second-order equilibrium for one direction (lb.c:144-151). */
double orc_equilibrium(int i, double rho, double ux, double uy, double usqr)
{
    double cu = CX[i] * ux + CY[i] * uy;
    return rho * W[i] * (1. + 3. * cu + 4.5 * cu * cu - 1.5 * usqr);
}

/* All nine directions at (rho, ux, uy) (lb.c:71-78). */
void orc_init_equilibrium(double *f, double rho, double ux, double uy)
{
    double usqr = ux * ux + uy * uy;
    int i;
    for (i = 0; i < 9; ++i) f[i] = orc_equilibrium(i, rho, ux, uy, usqr);
}

/* BGK relaxation: two roundings per direction, f*(1-omega) then + omega*feq (lb.c:154-166). */
static void bgk_relax(double *f, double omega)
{
    double rho, ux, uy, usqr;
    int i;
    orc_macros(f, &rho, &ux, &uy);
    usqr = ux * ux + uy * uy;
    for (i = 0; i < 9; ++i) {
        f[i] *= (1 - omega);
        f[i] += omega * orc_equilibrium(i, rho, ux, uy, usqr);
    }
}

/* Full-way bounce-back: every direction takes its opposite's value (boundaries.c:48-59). */
static void bounce_back(double *f)
{
    double g[9];
    int i;
    for (i = 0; i < 9; ++i) g[i] = f[OPP[i]];
    for (i = 0; i < 9; ++i) f[i] = g[i];
}

/* Sum of the populations known on a straight wall: rest + tangential + twice the ones
 * pointing out of the fluid (boundaries.c:66-126 use these sums inline). */
static double known_sum(const double *f, int side)
{
    switch (side) {
    case SIDE_UPPER: return f[0] + f[3] + f[1] + 2 * (f[6] + f[2] + f[5]);
    case SIDE_LOWER: return f[0] + f[3] + f[1] + 2 * (f[8] + f[4] + f[7]);
    case SIDE_RIGHT: return f[0] + f[2] + f[4] + 2 * (f[1] + f[5] + f[8]);
    default:         return f[0] + f[2] + f[4] + 2 * (f[3] + f[6] + f[7]);
    }
}

/* Wall density from the prescribed normal velocity (upperRho/lowerRho/rightRho/leftRho,
 * boundaries.c:66-118). */
static double wall_rho(const double *f, int side, double un)
{
    double s = known_sum(f, side);
    switch (side) {
    case SIDE_UPPER: return 1. / (1. + un) * s;
    case SIDE_LOWER: return 1. / (1. - un) * s;
    case SIDE_RIGHT: return 1. / (1. + un) * s;
    default:         return 1. / (1. - un) * s;
    }
}

/* Normal velocity from the prescribed density (upperU/lowerU/rightU/leftU,
 * boundaries.c:74-126). */
static double wall_u(const double *f, int side, double rho)
{
    double s = known_sum(f, side);
    switch (side) {
    case SIDE_UPPER: return -1. + 1. / rho * s;
    case SIDE_LOWER: return 1. - 1. / rho * s;
    case SIDE_RIGHT: return -1. + 1. / rho * s;
    default:         return 1. - 1. / rho * s;
    }
}

/* Zou/He completion of the three unknown populations (completeUpper/Lower/Right/Left,
 * boundaries.c:131-169). */
static void zouhe_complete(double *f, int side, double ux, double uy, double rho)
{
    switch (side) {
    case SIDE_UPPER:
        f[7] = f[5] + 0.5 * (f[1] - f[3]) - rho * uy / 6 - rho * ux / 2.;
        f[8] = f[6] + 0.5 * (f[3] - f[1]) - rho * uy / 6 + rho * ux / 2.;
        f[4] = f[2] - 2. / 3. * rho * uy;
        break;
    case SIDE_LOWER:
        f[6] = f[8] + 0.5 * (f[1] - f[3]) + rho * uy / 6 - rho * ux / 2.;
        f[5] = f[7] + 0.5 * (f[3] - f[1]) + rho * uy / 6 + rho * ux / 2.;
        f[2] = f[4] + 2. / 3. * rho * uy;
        break;
    case SIDE_RIGHT:
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

/* Regularized reconstruction: split f into equilibrium and non-equilibrium parts
 * (splitEqNeq, boundaries.c:239-249), take the side's non-equilibrium stress from its known
 * populations (upper/lower/right/leftNeqPi, boundaries.c:266-302) and rebuild
 * f = feq + 9/2 t_i Q_i:Pi (regularizedF, boundaries.c:251-262). */
static void regularize(double *f, int side, double rho, double ux, double uy)
{
    double feq[9], fneq[9], pxx, pyy, pxy;
    int i;
    for (i = 0; i < 9; ++i) {
        feq[i] = orc_equilibrium(i, rho, ux, uy, ux * ux + uy * uy);
        fneq[i] = f[i] - feq[i];
    }
    switch (side) {
    case SIDE_UPPER:
        pxx = fneq[1] + fneq[3] + 2. * (fneq[5] + fneq[6]);
        pyy = 2. * (fneq[6] + fneq[2] + fneq[5]);
        pxy = 2. * (fneq[5] - fneq[6]);
        break;
    case SIDE_LOWER:
        pxx = fneq[1] + fneq[3] + 2. * (fneq[7] + fneq[8]);
        pyy = 2. * (fneq[4] + fneq[7] + fneq[8]);
        pxy = 2. * (fneq[7] - fneq[8]);
        break;
    case SIDE_RIGHT:
        pxx = 2. * (fneq[1] + fneq[5] + fneq[8]);
        pyy = fneq[2] + fneq[4] + 2. * (fneq[5] + fneq[8]);
        pxy = 2. * (fneq[5] - fneq[8]);
        break;
    default:
        pxx = 2. * (fneq[3] + fneq[6] + fneq[7]);
        pyy = fneq[2] + fneq[4] + 2. * (fneq[6] + fneq[7]);
        pxy = 2. * (fneq[7] - fneq[6]);
        break;
    }
    for (i = 0; i < 9; ++i)
        f[i] = feq[i] + 9. / 2. * W[i] *
               ((CX[i] * CX[i] - 1. / 3.) * pxx + (CY[i] * CY[i] - 1. / 3.) * pyy +
                2. * CX[i] * CY[i] * pxy);
}

/* One node's collision through its dynamics (collideNode, lb.c:125-128).  Boundary kinds
 * chain to bulk BGK as every boundary function of boundaries.c:171-414 does.  param2 holds
 * the node's boundary data: (ux, uy) for velocity kinds, (rho, uPar) for pressure kinds. */
void orc_collide_node(int tag, double *f, double omega, const double *param2)
{
    int k, side, pressure;
    double rho, u;
    if (tag == ORC_BGK) { bgk_relax(f, omega); return; }
    if (tag == ORC_BOUNCE_BACK) { bounce_back(f); return; }
    if (tag < ORC_UPPER_ZOUHE || tag >= ORC_NUM_TAGS) return;
    k = tag - ORC_UPPER_ZOUHE;
    side = k % 4;
    pressure = (k / 4) & 1;
    if (tag < ORC_UPPER_REGULARIZED) {
        /* Zou/He: velocity kinds boundaries.c:171-201, pressure kinds boundaries.c:203-233 */
        if (!pressure) {
            double ux = param2[0], uy = param2[1];
            rho = wall_rho(f, side, (side <= SIDE_LOWER) ? uy : ux);
            zouhe_complete(f, side, ux, uy, rho);
        } else {
            rho = param2[0];
            u = wall_u(f, side, rho);
            if (side <= SIDE_LOWER) zouhe_complete(f, side, param2[1], u, rho);
            else                    zouhe_complete(f, side, u, param2[1], rho);
        }
    } else {
        /* regularized: velocity kinds boundaries.c:304-358, pressure kinds :360-414 */
        if (!pressure) {
            double ux = param2[0], uy = param2[1];
            rho = wall_rho(f, side, (side <= SIDE_LOWER) ? uy : ux);
            regularize(f, side, rho, ux, uy);
        } else {
            rho = param2[0];
            u = wall_u(f, side, rho);
            if (side <= SIDE_LOWER) regularize(f, side, rho, param2[1], u);
            else                    regularize(f, side, rho, u, param2[1]);
        }
    }
    bgk_relax(f, omega);
}

static int table_of(int tag)
{
    int k = tag - ORC_UPPER_ZOUHE;
    return ((k / 4) & 1) * 4 + (k % 4);
}

int orc_run(int lx, int ly, double omega, const unsigned char *tag, double *bc,
            const unsigned char *zgb_row, double *lat, double *tmp, int nsteps)
{
    const int ny2 = ly + 2;
    const int nb = (lx > ly ? lx : ly) + 2;
    const int right_prs = 1 * 4 + SIDE_RIGHT;
    double *a = lat, *b = tmp, *sw;
    int s, X, Y, i;
    for (s = 0; s < nsteps; ++s) {
        /* zero-gradient outlet: rho = 4/3 rho(lx-1) - 1/3 rho(lx-2) of the pre-collision
         * populations of this step, uPar = 0 (unsteady.c:205-214) */
        if (zgb_row) {
            for (Y = 0; Y < ny2; ++Y) {
                double rho1, ux1, uy1, rho2, ux2, uy2;
                if (!zgb_row[Y]) continue;
                orc_macros(&a[((size_t)(lx - 1) * ny2 + Y) * 9], &rho1, &ux1, &uy1);
                orc_macros(&a[((size_t)(lx - 2) * ny2 + Y) * 9], &rho2, &ux2, &uy2);
                bc[(right_prs * 2 + 0) * nb + Y] = 4. / 3. * rho1 - 1. / 3. * rho2;
                bc[(right_prs * 2 + 1) * nb + Y] = 0.;
            }
        }
        /* in-place collision of the interior (lb.c:181-185) */
        for (X = 1; X <= lx; ++X) {
            for (Y = 1; Y <= ly; ++Y) {
                int t = tag[X * ny2 + Y];
                double p[2] = { 0., 0. };
                if (t == ORC_NONE || t >= ORC_NUM_TAGS) return -1;
                if (t >= ORC_UPPER_ZOUHE) {
                    int tb = table_of(t);
                    int coord = ((t - ORC_UPPER_ZOUHE) % 4 <= SIDE_LOWER) ? X : Y;
                    p[0] = bc[(tb * 2 + 0) * nb + coord];
                    p[1] = bc[(tb * 2 + 1) * nb + coord];
                }
                orc_collide_node(t, &a[((size_t)X * ny2 + Y) * 9], omega, p);
            }
        }
        /* propagation into the second buffer; ghost destinations are written, ghost sources
         * are never read, so ghost-sourced slots keep the second buffer's old content
         * (lb.c:258-267), then the swap (lb.c:269-271) */
        for (X = 1; X <= lx; ++X)
            for (Y = 1; Y <= ly; ++Y)
                for (i = 0; i < 9; ++i)
                    b[((size_t)(X + CX[i]) * ny2 + (Y + CY[i])) * 9 + i] =
                        a[((size_t)X * ny2 + Y) * 9 + i];
        sw = a; a = b; b = sw;
    }
    if (a != lat) {
        size_t n = (size_t)(lx + 2) * ny2 * 9, k;
        for (k = 0; k < n; ++k) { double v = lat[k]; lat[k] = tmp[k]; tmp[k] = v; }
    }
    return 0;
}

/* Sums of a lattice state, the checker of the GPU reductions (no reference counterpart: the
 * reference computes no forces).  out[0] mass, [1..2] momentum, [3..4] momentum-exchange force
 * on bounce-back nodes strictly inside the lattice (2 c_i f_i over links entering them from
 * non-bounce-back nodes), [5] kinetic energy |j|^2/(2 rho) of BGK nodes, [6] nodes with a
 * non-finite population, [7] mass of BGK nodes.  Plain left-to-right sums. */
void orc_moments(int lx, int ly, const unsigned char *tag, const double *lat, double *out)
{
    const int ny2 = ly + 2;
    int X, Y, i, k;
    for (k = 0; k < 8; ++k) out[k] = 0.;
    for (X = 1; X <= lx; ++X)
        for (Y = 1; Y <= ly; ++Y) {
            const double *f = &lat[((size_t)X * ny2 + Y) * 9];
            double rho = 0., jx = 0., jy = 0.;
            int bad = 0;
            for (i = 0; i < 9; ++i) {
                rho += f[i];
                jx += CX[i] * f[i];
                jy += CY[i] * f[i];
                bad |= !(f[i] - f[i] == 0.);
            }
            out[0] += rho; out[1] += jx; out[2] += jy;
            out[6] += bad ? 1. : 0.;
            if (tag[X * ny2 + Y] == ORC_BGK) {
                out[5] += (jx * jx + jy * jy) / (2. * rho);
                out[7] += rho;
            } else if (tag[X * ny2 + Y] == ORC_BOUNCE_BACK && X >= 2 && X <= lx - 1 && Y >= 2 &&
                       Y <= ly - 1) {
                for (i = 1; i < 9; ++i)
                    if (tag[(X - CX[i]) * ny2 + (Y - CY[i])] != ORC_BOUNCE_BACK) {
                        out[3] += 2. * CX[i] * f[i];
                        out[4] += 2. * CY[i] * f[i];
                    }
            }
        }
}

/* Poiseuille profile of the application driver (unsteady.c:155-159). */
static double poiseuille(int iY, int ly, double uMax)
{
    double y = (double)(iY - 1);
    double L = (double)(ly - 1);
    return 4. * uMax / (L * L) * (L * y - y * y);
}

double orc_build_cylinder(int lx, int ly, int obst_x, int obst_y, int obst_r, double uMax,
                          double Re, int wall_kind, int outlet_kind, unsigned char *tag,
                          double *bc, unsigned char *zgb_row, double *lat, double *tmp)
{
    const int ny2 = ly + 2;
    const int nb = (lx > ly ? lx : ly) + 2;
    const int vel_up = SIDE_UPPER, vel_lo = SIDE_LOWER, vel_left = SIDE_LEFT;
    const int prs_right = 4 + SIDE_RIGHT;
    double nu = uMax * 2. * obst_r / Re;
    double omega = 1. / (3 * nu + 1. / 2.);
    int X, Y;
    size_t n = (size_t)(lx + 2) * ny2;
    memset(tag, 0, n);
    memset(bc, 0, sizeof(double) * 16 * (size_t)nb);
    memset(zgb_row, 0, (size_t)ny2);
    memset(lat, 0, sizeof(double) * 9 * n);
    memset(tmp, 0, sizeof(double) * 9 * n);
    /* bulk and obstacle (unsteady.c:164-182) */
    for (X = 1; X <= lx; ++X)
        for (Y = 1; Y <= ly; ++Y) {
            orc_init_equilibrium(&lat[((size_t)X * ny2 + Y) * 9], 1., poiseuille(Y, ly, uMax), 0.);
            tag[X * ny2 + Y] =
                ((X - obst_x) * (X - obst_x) + (Y - obst_y) * (Y - obst_y) <= obst_r * obst_r)
                    ? ORC_BOUNCE_BACK : ORC_BGK;
        }
    /* walls, corners included (unsteady.c:185-188) */
    for (X = 1; X <= lx; ++X) {
        if (wall_kind == 1) {
            tag[X * ny2 + 1] = ORC_BOUNCE_BACK;
            tag[X * ny2 + ly] = ORC_BOUNCE_BACK;
        } else {
            tag[X * ny2 + 1] = ORC_LOWER_REGULARIZED;
            tag[X * ny2 + ly] = ORC_UPPER_REGULARIZED;
            bc[(vel_lo * 2 + 0) * nb + X] = 0.; bc[(vel_lo * 2 + 1) * nb + X] = 0.;
            bc[(vel_up * 2 + 0) * nb + X] = 0.; bc[(vel_up * 2 + 1) * nb + X] = 0.;
        }
    }
    /* inlet and outlet (unsteady.c:193-198, iniData unsteady.c:128-141) */
    for (Y = 2; Y <= ly - 1; ++Y) {
        tag[1 * ny2 + Y] = ORC_LEFT_REGULARIZED;
        bc[(vel_left * 2 + 0) * nb + Y] = poiseuille(Y, ly, uMax);
        bc[(vel_left * 2 + 1) * nb + Y] = 0.;
        tag[lx * ny2 + Y] = ORC_RIGHT_PRESSURE_REGULARIZED;
        bc[(prs_right * 2 + 0) * nb + Y] = 1.;
        bc[(prs_right * 2 + 1) * nb + Y] = 0.;
        zgb_row[Y] = (outlet_kind == 0) ? 1 : 0;
    }
    return omega;
}
