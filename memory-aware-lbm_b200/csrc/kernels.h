// kernels.h -- host launchers of the device kernels (all asynchronous on `s`).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "layout.cuh"

namespace lbgpu {

// Device-side view of one lattice's data, passed by value to the launchers.
struct DevLattice {
    Geo g;
    int precision;       // LBGPU_F64 / F32 / F16 / BF16: element type of buf and side
    void *buf[2];        // population buffers (buf[1] unused by the AA scheme)
    void *side;          // stale-slot store [2][9][nper] (+ a scratch [9][nper] for pull lattices)
    void *ghost2;        // AA only: the second buffer's ghost ring [9][nghost] (see logical())
    const uint8_t *tag;  // tag plane
    double *bc;          // boundary tables [8][2][nb]
    const int *zgb_src;  // [4][nb]: pressure-table slot -> source row of its ZGB density, or -1
    double *zrho;        // [2*(ly+2)]: rho(lx-1, Y), rho(lx-2, Y) of the last ZGB pass
    double omega;
    float scale, inv_scale;  // FP16/BF16 offset storage: stored = (f - w) * scale
};

// How the post-stream state is read from a buffer:
//   VIEW_DIRECT        the buffer holds it (pull form L, or a collided state read as is)
//   VIEW_PULL_PENDING  the buffer holds C_n; the state is C_n streamed (side store: C_{n-1})
//   VIEW_AA_NATURAL    AA buffer in natural slots; stale slots in the side store
//   VIEW_AA_SWAPPED    AA buffer holds C_n in the opposite slots of each node
enum { VIEW_DIRECT = 0, VIEW_PULL_PENDING = 1, VIEW_AA_NATURAL = 2, VIEW_AA_SWAPPED = 3 };

void launch_collide_inplace(const DevLattice &d, int cur, int side_par, cudaStream_t s);
void launch_pull(const DevLattice &d, int src, int side_par, bool ghosts, cudaStream_t s);
// Kernels launch_pull launches (16-bit storage without the ghost ring: the quad kernel and the
// perimeter kernel).
int pull_launches(const DevLattice &d, bool ghosts);
void launch_stream(const DevLattice &d, int src, int side_par, cudaStream_t s);
// Two pull steps in one sweep (temporal blocking): C_n in buffer src (n_par = n & 1) ->
// C_{n+2} in buffer 1 - src, then the stale-slot scratch into parity n+1 and the two buffers'
// ghost rings exchanged.  Pull lattices without ghost-ring output only.
void launch_pull2(const DevLattice &d, int src, int n_par, cudaStream_t s);
void launch_side_from_buf(const DevLattice &d, int b, int side_par, cudaStream_t s);
// AA only: keep buffer b's ghost ring as the second buffer's (d.ghost2).
void launch_ghost_copy(const DevLattice &d, int b, cudaStream_t s);
void launch_readout(const DevLattice &d, int view, int cur, int side_par, int X0, int X1,
                    double *out, int rec_stride, const uint64_t *dynp, cudaStream_t s);
// Records of columns X0..X1-1, rows Y0..Y0+H-1 (in: [X - X0][Y - Y0][rec_stride] doubles) into
// buffer b.
void launch_upload(const DevLattice &d, int b, const double *in, int rec_stride, int X0, int X1,
                   int Y0, int H, cudaStream_t s);
// Tag plane from a device copy of a host-order tag array tag_xy[X * (ly + 2) + Y].
void launch_tags_from_xy(const DevLattice &d, const uint8_t *in, cudaStream_t s);
void launch_zgb_rho(const DevLattice &d, int view, int cur, int side_par, cudaStream_t s);
void launch_zgb_apply(const DevLattice &d, cudaStream_t s);
void launch_periodic(const DevLattice &d, int b, cudaStream_t s);
// Tag plane of the cylinder channel (obstacle disk, walls of wall_kind, regularized inlet,
// pressure-regularized outlet) written on the device.
void launch_cylinder_tags(const DevLattice &d, int ox, int oy, int r, int wall_kind, cudaStream_t s);
void launch_init_cylinder(const DevLattice &d, int b, double umax, cudaStream_t s);
void launch_macros(const DevLattice &d, int view, int cur, int side_par, double *rho, double *ux,
                   double *uy, cudaStream_t s);
// FP64 reductions of the current state (mass, momentum, obstacle force, kinetic energy,
// non-finite nodes, fluid mass) into out[8]; `partial` is scratch of (ly+2)*8 doubles.
void launch_moments(const DevLattice &d, int view, int cur, int side_par, double *partial,
                    double *out, cudaStream_t s);
// acc[0..lx*ly) += ux, acc[lx*ly..2*lx*ly) += uy of the current state.
void launch_accumulate_velocity(const DevLattice &d, int view, int cur, int side_par, double *acc,
                                cudaStream_t s);
// max over the interior of |u - u_prev| into *out (float bits, cleared by the caller);
// prev (lx*ly float2, [Y-1][X-1]) receives the current velocity.
void launch_velocity_change(const DevLattice &d, int view, int cur, int side_par, void *prev,
                            unsigned *out, cudaStream_t s);
// ---- batches: many lattices per launch ------------------------------------------------
// threads per block = nodes per tile: 128, 256 or 512
// Kinds of batch step: pull (one node per thread), AA even and odd, the 16-bit pull with four
// nodes per thread (each warp one row of 128 nodes, see pull_quad), which leaves each member's
// perimeter nodes to BATCH_PERIM: the pull step of those nodes, one per thread, one block a run
// of `threads` perimeter nodes of a member (work item: the member, x0 = the run's first number).
enum { BATCH_PULL = 0, BATCH_AA_EVEN = 1, BATCH_AA_ODD = 2, BATCH_PULL4 = 3, BATCH_PERIM = 4 };
constexpr int BATCH_KINDS = 5;

// One lattice of a batch, with its state at the start of the current chunk of steps:
// pull scheme: the buffer holding C_n is buf[cur0]; AA: phase0 0 = natural form, 1 = swapped;
// tau0 = the time step the chunk's first launch executes (its side parity is tau0 & 1).
struct BatchInst {
    Geo g;
    void *buf[2];
    void *side;
    const uint8_t *tag;
    const double *bc;
    double omega;
    float scale, inv_scale;
    int scheme, cur0, phase0, tau0;   // tau0 + k: the collision number of step k of a chunk
    unsigned rs_seed;                 // 16-bit members: stochastic rounding seed (rs != 0)
    int rs;
};

// A strip of `passes` tiles of a lattice stacked in y, stepped by one block from the top down.
// A tile: nodes x0 .. x0 + (32 << shape) - 1 and threads / (32 << shape) rows (BATCH_PULL4:
// x0 .. x0 + 127 and threads / 32 rows); pass p covers the tile starting at row
// y0 + p * (rows of a tile).  `sp` packs shape (bits 0..7) and passes (bits 8..).
struct BatchWork {
    int inst, x0, y0, sp;
};
__host__ __device__ inline int batch_shape(int sp) { return sp & 0xff; }
__host__ __device__ inline int batch_passes(int sp) { return sp >> 8; }
__host__ __device__ inline int batch_sp(int shape, int passes) { return shape | (passes << 8); }

// Step k of a chunk, of kind BATCH_PULL / AA_EVEN / AA_ODD / PULL4 (16-bit only), for every tile of a
// work list of `nwork` tiles of `threads` nodes: `persistent` grids of `grid` blocks stride
// through the list, otherwise `grid` must equal nwork (one block per tile).
// flags (16-bit batches): bit 0 -- some member rounds stochastically, bit 1 -- some member stores
// row-shifted offsets; the kernels then carry those paths.
void launch_batch(int precision, int kind, int threads, bool persistent, int flags, const BatchInst *insts,
                  const BatchWork *work, int nwork, int grid, int k, cudaStream_t s);
// Resident blocks per SM of the persistent kernel of a kind and block size.
int batch_blocks_per_sm(int precision, int kind, int threads);

// AA scheme (buffer 0): the even step collides every node in place into the opposite slots,
// the odd step gathers from the neighbours' opposite slots and scatters to their natural slots.
void launch_aa_even(const DevLattice &d, int side_par, cudaStream_t s);
void launch_aa_odd(const DevLattice &d, int side_par, cudaStream_t s);

}  // namespace lbgpu
