/* lbm_oracle.h -- TEST INFRASTRUCTURE ONLY: the CPU oracle for the D2Q9 cylinder step.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may load this; the
 * product never links it.  It restates, in plain C, the reference's one-step ("origin")
 * algorithm: in-place collision of every interior node through its dynamics
 * (lb.c:172-185, lb.c:125-128), then propagation into the second buffer that never reads
 * ghost sources (lb.c:246-271), then the buffer swap.  The zero-gradient outlet update of
 * the application driver (unsteady.c:205-214) runs before each step for flagged rows.
 *
 * Parity is pinned against the reference itself: tests/test_oracle_pins.py compares this
 * oracle with the reference's own lb.c/boundaries.c compiled into oracle/_ref, and
 * tests/golden/ holds digests of the reference's outputs made by tests/golden/make_golden.py.
 *
 * Layout (the reference's own): populations f[((X*(ly+2)) + Y)*9 + i] for X = 0..lx+1,
 * Y = 0..ly+1 (ghost ring included), lattice directions in the reference order
 * (lb.c:48-55).  Per-node dynamics are a tag byte tag[X*(ly+2)+Y] with the values below;
 * boundary parameters live in per-side tables bc[((table*2)+component)*nb + coord] with
 * nb = max(lx, ly) + 2, table = family*4 + side (family 0 velocity (ux, uy), 1 pressure
 * (rho, uPar); side 0 upper, 1 lower, 2 left, 3 right), coord = X for upper/lower and Y
 * for left/right.
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ORC_NONE = 0, ORC_BGK = 1, ORC_BOUNCE_BACK = 2,
    ORC_UPPER_ZOUHE = 3, ORC_LOWER_ZOUHE = 4, ORC_LEFT_ZOUHE = 5, ORC_RIGHT_ZOUHE = 6,
    ORC_UPPER_PRESSURE_ZOUHE = 7, ORC_LOWER_PRESSURE_ZOUHE = 8,
    ORC_LEFT_PRESSURE_ZOUHE = 9, ORC_RIGHT_PRESSURE_ZOUHE = 10,
    ORC_UPPER_REGULARIZED = 11, ORC_LOWER_REGULARIZED = 12,
    ORC_LEFT_REGULARIZED = 13, ORC_RIGHT_REGULARIZED = 14,
    ORC_UPPER_PRESSURE_REGULARIZED = 15, ORC_LOWER_PRESSURE_REGULARIZED = 16,
    ORC_LEFT_PRESSURE_REGULARIZED = 17, ORC_RIGHT_PRESSURE_REGULARIZED = 18,
    ORC_NUM_TAGS = 19
};

/* Advance `nsteps` steps.  lat holds L_0 on entry and L_nsteps on return; tmp holds the
 * second buffer (its ghost-sourced slots are what the first step's stream leaves behind) and
 * on return holds the final second buffer.  bc is updated in place by the ZGB rows.
 * Returns 0, or -1 when an interior node has no dynamics (the reference would crash). */
int orc_run(int lx, int ly, double omega, const unsigned char *tag, double *bc,
            const unsigned char *zgb_row, double *lat, double *tmp, int nsteps);

/* Single-node pieces, exported so tests can compare the product's host helpers with them. */
void orc_macros(const double *f, double *rho, double *ux, double *uy);
double orc_equilibrium(int i, double rho, double ux, double uy, double usqr);
void orc_collide_node(int tag, double *f, double omega, const double *param2);
void orc_init_equilibrium(double *f, double rho, double ux, double uy);

/* Sums of a state (mass, momentum, obstacle force, kinetic energy, non-finite nodes, bulk
 * mass) -- the checker of the GPU reductions; see lbm_oracle.c. */
void orc_moments(int lx, int ly, const unsigned char *tag, const double *lat, double *out);

/* Cylinder geometry builder used by the tests (the application driver's iniGeometry,
 * unsteady.c:162-199, with the wall/outlet options of the harness).  Fills tag, bc,
 * zgb_row and the initial populations of lat; tmp is zeroed.  Returns omega. */
double orc_build_cylinder(int lx, int ly, int obst_x, int obst_y, int obst_r, double uMax,
                          double Re, int wall_kind, int outlet_kind, unsigned char *tag,
                          double *bc, unsigned char *zgb_row, double *lat, double *tmp);

#ifdef __cplusplus
}
#endif
#endif
