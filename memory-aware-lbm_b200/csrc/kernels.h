// kernels.h -- host launchers of the device kernels (all asynchronous on `s`).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "layout.cuh"

namespace lbgpu {

// Device-side view of one lattice's data, passed by value to the launchers.
struct DevLattice {
    Geo g;
    void *buf[2];        // population buffers (buf[1] unused by the AA scheme)
    void *side;          // stale-slot store [2][9][nper]
    const uint8_t *tag;  // tag plane
    double *bc;          // boundary tables [8][2][nb]
    const int *zgb_src;  // [4][nb]: pressure-table slot -> source row of its ZGB density, or -1
    double *zrho;        // [2*(ly+2)]: rho(lx-1, Y), rho(lx-2, Y) of the last ZGB pass
    double omega;
    float scale, inv_scale;  // FP16/BF16 offset storage: stored = (f - w) * scale
};

// ---- exact FP64 kernels (reference arithmetic, bit-exact) ------------------------------
void launch_collide_inplace_f64(const DevLattice &d, int cur, int side_par, cudaStream_t s);
void launch_pull_f64(const DevLattice &d, int src, int side_par, bool ghosts, cudaStream_t s);
void launch_stream_f64(const DevLattice &d, int src, int side_par, cudaStream_t s);
void launch_side_from_buf_f64(const DevLattice &d, int b, int side_par, cudaStream_t s);
void launch_readout_f64(const DevLattice &d, int cur, int pending, int side_par, int X0, int X1,
                        double *out, int rec_stride, const uint64_t *dynp, cudaStream_t s);
void launch_upload_f64(const DevLattice &d, int b, const double *in, int rec_stride, int X0,
                       int X1, cudaStream_t s);
void launch_zgb_rho_f64(const DevLattice &d, int cur, int pending, int side_par, cudaStream_t s);
void launch_zgb_apply(const DevLattice &d, cudaStream_t s);
void launch_periodic_f64(const DevLattice &d, int b, cudaStream_t s);
void launch_init_cylinder_f64(const DevLattice &d, int b, double umax, cudaStream_t s);
void launch_macros_f64(const DevLattice &d, int cur, int pending, int side_par, double *rho,
                       double *ux, double *uy, cudaStream_t s);

}  // namespace lbgpu
