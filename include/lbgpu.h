/* lbgpu.h -- native C interface of liblbgpu.so beyond the drop-in lb.h / boundaries.h.
 *
 * Two groups of functions:
 *
 *  1. Companions of the drop-in interface (no counterpart in the reference, whose lattice
 *     lives in host memory only): copying the device lattice back, telling the library the
 *     host copy changed, choosing what is copied back after each entry point, and reading
 *     the error the last entry point recorded.
 *
 *  2. The lattice object used by benchmarks, batching and serving: populations stored in
 *     FP64, FP32, or FP16/BF16 offsets, stepped by the two-buffer pull kernel or the in-place
 *     AA kernel.  Geometry is given in the same per-node tag / per-side table form the
 *     drop-in interface derives from Dynamics pointers:
 *       tag[X*(ly+2) + Y]          X = 0..lx+1, Y = 0..ly+1 (ghost ring tag LBGPU_TAG_NONE)
 *       bc[((t*2)+k)*nb + coord]   nb = max(lx,ly)+2; table t = family*4 + side with family
 *                                  0 velocity (k: ux, uy) or 1 pressure (k: rho, uPar), side
 *                                  0 upper, 1 lower, 2 left, 3 right; coord = X for upper and
 *                                  lower, Y for left and right
 *       populations f[((X*(ly+2)) + Y)*9 + i], the reference's node order and direction order.
 *
 * All functions return LB_OK (0) or an LB_ERR_* code and never abort; the message of the
 * last failure on the calling thread is lbGetLastErrorString().
 */
#ifndef LBGPU_H
#define LBGPU_H

#include <stddef.h>
#include <stdint.h>
#include "lb.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes ------------------------------------------------------------------- */
enum {
    LB_OK = 0,
    LB_ERR_CUDA = 1,          /* a CUDA call failed (message has the CUDA error string)  */
    LB_ERR_ALLOC = 2,         /* device or pinned-host allocation refused                 */
    LB_ERR_ARG = 3,           /* invalid argument (size, pointer, enum value)             */
    LB_ERR_BLOCK_SIZE = 4,    /* blk_size does not divide the swept extent                */
    LB_ERR_DYNAMICS = 5,      /* a node uses a dynamics function the GPU cannot run       */
    LB_ERR_LAYOUT = 6,        /* two boundary nodes share a table slot with different data */
    LB_ERR_STATE = 7,         /* call not valid in the lattice's current state            */
    LB_ERR_NO_DEVICE = 8,     /* no CUDA device                                           */
    LB_ERR_TIMEOUT = 9,       /* a bounded device wait gave up                            */
    LB_ERR_CAPACITY = 10      /* a request exceeds a fixed capacity (budget, slots)       */
};

/* Error recorded by the calling thread's most recent failing call (0 when none), and
 * its message.  lbClearError resets both. No counterpart in the reference (void API). */
int lbGetLastError(void);
const char *lbGetLastErrorString(void);
void lbClearError(void);

/* ---- drop-in companions ---------------------------------------------------------- */
/* What the drop-in entry points copy back to the host lattice after running:
 *   LB_SYNC_NONE     nothing; call lbSyncToHost before reading sim->lattice.
 *   LB_SYNC_OUTLET   columns lx-1 and lx-2 (interior rows), which the application driver's
 *                    zero-gradient update reads before every step (default).
 *   LB_SYNC_FULL     the whole current lattice, ghost ring included.
 * The environment variable LBGPU_SYNC=none|outlet|full sets the default. */
enum { LB_SYNC_NONE = 0, LB_SYNC_OUTLET = 1, LB_SYNC_FULL = 2 };
void lbSetSyncMode(Simulation *sim, int mode);

/* Copy the current lattice (post-stream state, ghost ring included) into the host
 * arrays sim->lattice points to.  The host copy of tmpLattice is not maintained. */
void lbSyncToHost(Simulation *sim);

/* The driver wrote populations of sim->lattice directly: upload them before the next
 * entry point.  (setDynamics marks the dynamics dirty by itself.) */
void lbMarkHostDirty(Simulation *sim);

/* Bytes the library has copied host->device and device->host for this simulation since
 * constructSim (populations, dynamics, tables, outlet columns, read-outs).  No counterpart in
 * the reference: it lets a benchmark declare the transfers of the drop-in path. */
void lbGetTransferBytes(const Simulation *sim, unsigned long long *h2d, unsigned long long *d2h);

/* ---- lattice object ------------------------------------------------------------------ */
enum { LBGPU_F64 = 0, LBGPU_F32 = 1, LBGPU_F16 = 2, LBGPU_BF16 = 3 };
enum { LBGPU_PULL = 0, LBGPU_AA = 1 };

enum {
    LBGPU_TAG_NONE = 0, LBGPU_TAG_BGK = 1, LBGPU_TAG_BOUNCE_BACK = 2,
    LBGPU_TAG_UPPER_ZOUHE = 3, LBGPU_TAG_LOWER_ZOUHE = 4,
    LBGPU_TAG_LEFT_ZOUHE = 5, LBGPU_TAG_RIGHT_ZOUHE = 6,
    LBGPU_TAG_UPPER_PRESSURE_ZOUHE = 7, LBGPU_TAG_LOWER_PRESSURE_ZOUHE = 8,
    LBGPU_TAG_LEFT_PRESSURE_ZOUHE = 9, LBGPU_TAG_RIGHT_PRESSURE_ZOUHE = 10,
    LBGPU_TAG_UPPER_REGULARIZED = 11, LBGPU_TAG_LOWER_REGULARIZED = 12,
    LBGPU_TAG_LEFT_REGULARIZED = 13, LBGPU_TAG_RIGHT_REGULARIZED = 14,
    LBGPU_TAG_UPPER_PRESSURE_REGULARIZED = 15, LBGPU_TAG_LOWER_PRESSURE_REGULARIZED = 16,
    LBGPU_TAG_LEFT_PRESSURE_REGULARIZED = 17, LBGPU_TAG_RIGHT_PRESSURE_REGULARIZED = 18,
    LBGPU_NUM_TAGS = 19
};

enum { LBGPU_WALL_REGULARIZED = 0, LBGPU_WALL_BOUNCEBACK = 1 };
enum { LBGPU_OUTLET_ZGB = 0, LBGPU_OUTLET_CONST = 1 };

typedef struct lbgpu_lattice lbgpu_lattice;

/* Select the CUDA device used by this thread's later lbgpu_create / constructSim calls (the
 * library carries its own CUDA runtime, so a device chosen through another runtime, such as
 * the one PyTorch loads, does not carry over).  Returns LB_ERR_NO_DEVICE for a bad index. */
int lbgpu_set_device(int device);
int lbgpu_device_count(void);

/* Allocate a lattice on the current CUDA device: two population buffers for
 * LBGPU_PULL, one for LBGPU_AA, plus tags and tables.  1 <= lx <= LBGPU_MAX_LX and
 * 1 <= ly <= LBGPU_MAX_LY, else LB_ERR_ARG: the row-wise kernels launch one grid row per
 * lattice row including the two ghost rows, and CUDA allows at most 65535 grid rows. */
enum { LBGPU_MAX_LX = 1 << 20, LBGPU_MAX_LY = 65533 };
int lbgpu_create(int lx, int ly, int precision, int scheme, lbgpu_lattice **out);
int lbgpu_destroy(lbgpu_lattice *lat);

/* Geometry and boundary data (layouts above).  zgb_row may be NULL; rows flagged there take
 * their right-side pressure density from the zero-gradient extrapolation
 * 4/3 rho(lx-1) - 1/3 rho(lx-2) of the populations entering each step. */
int lbgpu_set_geometry(lbgpu_lattice *lat, double omega, const uint8_t *tag, const double *bc,
                       const uint8_t *zgb_row);

/* Initial populations of the first and second buffers (tmp may be NULL for zeros); resets
 * the step count.  For FP16/BF16 storage, `scale_log2` in lbgpu_set_offset_scale applies. */
int lbgpu_set_populations(lbgpu_lattice *lat, const double *f, const double *tmp);

/* Power-of-two scale s of the FP16/BF16 offset storage: stored = (f_i - w_i) * 2^s. */
int lbgpu_set_offset_scale(lbgpu_lattice *lat, int scale_log2);

/* FP16/BF16 storage only: store offsets from the equilibrium of a per-row shift velocity
 * instead of from the lattice weights: stored_i = (f_i - f_eq_i(1, (u_row[Y], 0))) * 2^s, where
 * Y is the row that consumes the value (the receiving row after streaming).  For a channel whose
 * flow stays close to a known profile (the Poiseuille inflow of lbgpu_setup_cylinder, 4 uMax
 * (L y - y^2) / L^2 with y = Y - 1, L = ly - 1, and 0 in the ghost rows), the stored values are
 * small deviations, which the 16-bit significand resolves far better than offsets from w_i; it
 * removes the slow drift of the smooth far field.  u_row has ly + 2 values (|u| < 0.5); NULL
 * returns to offsets from w_i.  Set it, like the scale, before the initial state is written.
 * LB_ERR_STATE for FP64/FP32 lattices.  No counterpart in the reference (FP64 only). */
int lbgpu_set_offset_shift(lbgpu_lattice *lat, const double *u_row);

/* FP16/BF16 storage only: round stored post-collision values stochastically (on = 1) instead
 * of to nearest (on = 0, the default).  Rounding to nearest drops every change of a stored value
 * below half its quantum, so a slow transient stalls in 16-bit storage; stochastic rounding keeps
 * the stored value unbiased (sm_100a hardware conversion `cvt.rs`).  The random bits of a value
 * are a function of (seed, collision number, node, direction) only: results are deterministic for
 * a seed and identical across the pull scheme, the AA scheme and two steps per sweep.  Initial
 * states and uploads still round to nearest.  Lattices with it on step alone (a batch refuses
 * them, LB_ERR_STATE).  LB_ERR_STATE for FP64/FP32 lattices.  No counterpart in the reference. */
int lbgpu_set_stochastic_rounding(lbgpu_lattice *lat, int on, unsigned seed);

/* Cylinder channel on the device without host population arrays: tags and tables as the
 * application driver builds them (obstacle disk, walls, Poiseuille inlet, pressure outlet)
 * and equilibrium populations at rho = 1 and the Poiseuille profile.  Returns omega through
 * omega_out when not NULL. */
int lbgpu_setup_cylinder(lbgpu_lattice *lat, int obst_x, int obst_y, int obst_r, double umax,
                         double re, int wall_kind, int outlet_kind, double *omega_out);

/* The same geometry into host arrays (tag, bc, zgb_row, f as laid out above); f may be NULL. */
double lbgpu_build_cylinder(int lx, int ly, int obst_x, int obst_y, int obst_r, double umax,
                            double re, int wall_kind, int outlet_kind, uint8_t *tag,
                            double *bc, uint8_t *zgb_row, double *f);

/* Steps per sweep of the pull scheme: 1 (default) or 2.  With 2, lbgpu_step advances pairs of
 * steps in one kernel that keeps the intermediate state on chip (in registers, shifted across
 * lanes by warp shuffles, for FP64/FP32; in shared memory for 16-bit storage), the GPU form of
 * the reference's collide_tight two-steps-per-sweep idea (lb.c:442-572): one read and one write
 * of the lattice per two steps.  Results are identical to single steps; on B200 it runs at 0.85
 * of one step per sweep, which already streams at the copy bandwidth.
 * Lattices with an extrapolated outlet (a pass between every two steps) and the first step of
 * a fresh lattice still run single steps.  LB_ERR_STATE for the AA scheme. */
int lbgpu_set_sweep_steps(lbgpu_lattice *lat, int steps);

/* Advance `nsteps` time steps; asynchronous on the lattice's stream. */
int lbgpu_step(lbgpu_lattice *lat, int nsteps);

/* Advance `nsteps` steps and report their device time in milliseconds (CUDA events on the
 * lattice's stream); synchronous. */
int lbgpu_step_timed(lbgpu_lattice *lat, int nsteps, float *ms);

/* Current post-stream populations as FP64, ghost ring included (layout above). */
int lbgpu_get_populations(lbgpu_lattice *lat, double *f);

/* Density and velocity of the current state for the interior, [Y-1][X-1] row-major
 * (ly rows of lx values), computed on the device. Any pointer may be NULL. */
int lbgpu_get_macros(lbgpu_lattice *lat, double *rho, double *ux, double *uy);

/* lbgpu_get_macros for callers that cannot allocate device memory while the solver runs (a
 * serving loop reading one simulation while others step: cudaMalloc/cudaFree would stall every
 * stream; a process whose device memory another allocator has reserved).  No counterpart in
 * the reference.  Allocates nothing: the device scratch is a fixed array of 3 x 262,144
 * doubles (6 MiB, held by every GPU that loads the library), so lattices above 262,144
 * interior nodes get LB_ERR_CAPACITY.  The first call on a device looks up that array's
 * address; make it before any stream capture.  Later calls look it up again unless the
 * lattice's stream is capturing, so a device reset (cudaDeviceReset) between calls is safe.
 * All calls share the array: calls that overlap on the GPU race. */
int lbgpu_get_macros_noalloc(lbgpu_lattice *lat, double *rho, double *ux, double *uy);

/* FP64 sums over the current state, computed on the device in a fixed order (bitwise
 * reproducible): out[0] mass (sum of rho over interior nodes), out[1..2] momentum, out[3..4]
 * force on the obstacle by momentum exchange (2 c_i f_i over every link entering a bounce-back
 * node strictly inside the lattice from a non-bounce-back node), out[5] kinetic energy of bulk
 * nodes, out[6] number of nodes with a non-finite population, out[7] mass of bulk nodes.
 * No counterpart in the reference (it computes no forces). */
int lbgpu_moments(lbgpu_lattice *lat, double out[8]);

/* Time averages of the velocity field: accumulate adds the current (ux, uy) of every interior
 * node to FP64 running sums on the device; average copies sum/samples into [ly][lx] host arrays;
 * reset clears the sums. */
int lbgpu_velocity_accumulate(lbgpu_lattice *lat);
int lbgpu_velocity_average(lbgpu_lattice *lat, double *ux, double *uy, long long *samples);
int lbgpu_velocity_reset(lbgpu_lattice *lat);

int lbgpu_synchronize(lbgpu_lattice *lat);

/* ---- batches: many independent lattices in one launch per step --------------------------
 * No counterpart in the reference (one lattice per process).  Members are lattices of the
 * batch's precision, pull or AA, with constant-density outlets (an extrapolated outlet is
 * stepped on its own).  lbgpu_batch_step advances every member by nsteps: per step one launch
 * for the pull members and one for each phase of the AA members walks a work list of 128-node
 * tiles; chunks of 50 steps are replayed as a CUDA graph.  Each member's result is bit-identical to stepping it alone.  The batch does not
 * own its members; remove a member before destroying it.  Steps are asynchronous on the batch's
 * stream and ordered with the members' own streams. */
typedef struct lbgpu_batch lbgpu_batch;
int lbgpu_batch_create(int precision, lbgpu_batch **out);
int lbgpu_batch_destroy(lbgpu_batch *b);
int lbgpu_batch_add(lbgpu_batch *b, lbgpu_lattice *lat, int *slot);
int lbgpu_batch_remove(lbgpu_batch *b, int slot);
int lbgpu_batch_size(lbgpu_batch *b);
int lbgpu_batch_step(lbgpu_batch *b, int nsteps);
int lbgpu_batch_step_timed(lbgpu_batch *b, int nsteps, float *ms);
int lbgpu_batch_synchronize(lbgpu_batch *b);
int lbgpu_batch_last_launches(lbgpu_batch *b);

/* Tile shape of a size class (class of a lattice = lbgpu_batch_size_class(lx*ly), 0..5 for
 * < 16K, 64K, 256K, 1M, 4M nodes and above): nodes_per_thread 1: tiles tile_width (32, 64,
 * 128) nodes wide and threads / tile_width rows high, one node per thread of a block of
 * `threads` threads; nodes_per_thread 4 (16-bit storage, tile_width 128, pull members): each
 * warp one row of 128 nodes, four per thread.  Defaults: 128 wide, one node per thread; four
 * nodes per thread for 16-bit lattices of 64K nodes and more. */
int lbgpu_batch_size_class(long long nodes);
int lbgpu_batch_set_shape(lbgpu_batch *b, int size_class, int tile_width, int nodes_per_thread);
int lbgpu_batch_get_shape(lbgpu_batch *b, int size_class, int *tile_width, int *nodes_per_thread);
/* Strip length of a size class: one block steps `passes` (1..64, default 4) tiles of a member
 * stacked in y, one after another down the lattice, and reads the member's descriptor once. */
int lbgpu_batch_set_passes(lbgpu_batch *b, int size_class, int passes);
int lbgpu_batch_get_passes(lbgpu_batch *b, int size_class);
/* Launch form: 1 = a persistent grid (resident blocks per SM x SMs) strides through the work
 * list, 0 = one block per tile (the default). */
int lbgpu_batch_set_persistent(lbgpu_batch *b, int persistent);
int lbgpu_batch_get_persistent(lbgpu_batch *b);
/* Threads per tile (= nodes per tile, one block per tile): 128 (default), 256 or 512. */
int lbgpu_batch_set_threads(lbgpu_batch *b, int threads);
int lbgpu_batch_get_threads(lbgpu_batch *b);

/* Autotuner: times `steps` batch steps (after one untimed step) with each threads-per-tile and
 * launch-form pair, then, for each size class present, with each tile shape (three widths, and
 * four nodes per thread for 16-bit storage), keeping the fastest at each stage (the members
 * really advance 6 x (steps + 1) plus 3 or 4 x (steps + 1) per class present); best_ms[6]
 * receives each class's best time (0 for classes not present) when not NULL. */
int lbgpu_batch_autotune(lbgpu_batch *b, int steps, float *best_ms);

/* Device bytes a lattice of this size, precision and scheme allocates. */
size_t lbgpu_lattice_bytes(int lx, int ly, int precision, int scheme);

/* ---- serving: continuous batching of simulation requests --------------------------------
 * No counterpart in the reference.  A request is a cylinder channel (bounce-back walls,
 * constant-density outlet) with a step cap (a multiple of the server's check interval) and a
 * steady-state tolerance: it retires when the largest velocity change over one check interval
 * falls below `tol` (0: never) or at the cap; a request whose velocity becomes non-finite
 * retires at that check with converged = -1.  lbgpu_server_run serves every submitted request,
 * honouring arrival times (seconds after the run starts) in wall-clock time: batched = 1 admits
 * requests in arrival order while their lattices fit the budget and steps all resident ones
 * together (lbgpu_batch); batched = 0 solves them one at a time on their own (plain solves). */
typedef struct {
    int lx, ly, obst_x, obst_y, obst_r;
    double umax, re;
    int max_steps;
    double tol;
    double arrival;
    int want_fields;       /* keep the final velocity field for lbgpu_server_result */
} lbgpu_request;

typedef struct {
    double arrival, admit, finish;  /* seconds after the run's start */
    long long steps, nodes;
    int converged, done;            /* converged: 1 steady, 0 step cap, -1 diverged */
    double last_change;             /* velocity change over the last check interval */
    int solo;                       /* 1: stepped on its own, not as a batch member */
} lbgpu_result;

typedef struct lbgpu_server lbgpu_server;
int lbgpu_server_create(int precision, size_t budget_bytes, int check_every, lbgpu_server **out);
int lbgpu_server_destroy(lbgpu_server *s);
int lbgpu_server_set_scheme(lbgpu_server *s, int size_class, int scheme);
int lbgpu_server_set_shape(lbgpu_server *s, int size_class, int tile_width, int nodes_per_thread);
int lbgpu_server_set_persistent(lbgpu_server *s, int persistent);
int lbgpu_server_set_threads(lbgpu_server *s, int threads);
/* Requests of at least `nodes` lattice nodes (default 2^20) are not batch members: they fill
 * the GPU on their own and step with the single-lattice kernels on their own streams,
 * concurrently with the batch; 0 batches every request. */
int lbgpu_server_set_solo_nodes(lbgpu_server *s, long long nodes);
int lbgpu_server_set_offset_scale(lbgpu_server *s, int scale_log2);
/* FP16/BF16 servers: store each request's offsets from its inflow profile's equilibrium per
 * row (lbgpu_set_offset_shift) instead of from w_i. */
int lbgpu_server_set_offset_shift(lbgpu_server *s, int on);
/* FP16/BF16 servers: round each request's stored values stochastically
 * (lbgpu_set_stochastic_rounding, seeded with the request id). */
int lbgpu_server_set_stochastic_rounding(lbgpu_server *s, int on);
int lbgpu_server_submit(lbgpu_server *s, const lbgpu_request *r, int *id);
int lbgpu_server_run(lbgpu_server *s, int batched);
int lbgpu_server_result(lbgpu_server *s, int id, lbgpu_result *out, double *ux, double *uy);
/* out[0] makespan (s), out[1] lattice updates, out[2] peak resident requests, out[3] peak bytes */
int lbgpu_server_stats(lbgpu_server *s, double out[4]);

/* Autotuner for the scheme of batch members of one size: copies of a cylinder channel of
 * lx x ly (enough for about 8M nodes, at most 64) step together in a batch, once in the pull
 * and once in the AA scheme; returns the faster one (*scheme) and both timings of `steps`
 * batch steps. */
int lbgpu_tune_scheme(int precision, int lx, int ly, int steps, int *scheme, float *ms_pull,
                      float *ms_aa);
void *lbgpu_stream(lbgpu_lattice *lat);           /* the lattice's cudaStream_t            */
long long lbgpu_steps_done(lbgpu_lattice *lat);
size_t lbgpu_device_bytes(lbgpu_lattice *lat);     /* device memory held by the lattice     */
int lbgpu_last_kernel_launches(lbgpu_lattice *lat); /* kernels launched by the last step call */

#ifdef __cplusplus
}
#endif
#endif
