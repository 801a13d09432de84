// lattice.h -- the device lattice object behind both C interfaces.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>
#include <vector>
#include "kernels.h"

namespace lbgpu {

// Thread-local error state of the C interfaces (LB_ERR_* codes of include/lbgpu.h).
int set_error(int code, const char *fmt, ...);
int cuda_error(cudaError_t e, const char *what);
int last_error();
const char *last_error_string();
void clear_error();

enum { FORM_L = 0, FORM_C = 1 };

// CUDA's limit on gridDim.y (kernels that launch one grid row a lattice row or column).
constexpr size_t kMaxGridY = 65535;

struct Lattice {
    int lx = 0, ly = 0;
    int precision = 0;   // LBGPU_F64 / F32 / F16 / BF16
    int scheme = 0;      // LBGPU_PULL / LBGPU_AA
    DevLattice d{};
    size_t elem = 8;     // bytes per stored population
    int cur = 0;         // buffer holding the state
    int form = FORM_L;   // see kernels.cu
    int pending = 0;     // form C only: 1 when the post-stream state is the current one
    long long n = 0;     // index of the last collision (form C) or of the state (form L)
    bool ghosts = false; // keep the ghost ring exact (drop-in interface)
    bool zgb_each_step = false;  // native: extrapolated outlet before every step
    int sweep_steps = 1;         // pull scheme: 2 = two steps per sweep where eligible (k_sweep2)
    cudaStream_t stream = nullptr;
    size_t bytes = 0;
    int launches = 0;    // kernels launched by the last public call
    unsigned long long h2d_bytes = 0, d2h_bytes = 0;  // bytes copied host<->device so far
    int device = 0;      // CUDA device the lattice lives on

    std::vector<double> bc_host;   // [16*nb] last uploaded boundary tables
    std::vector<int> zgb_src_host; // [4*nb]
    double *stage = nullptr;       // device staging for record transfers
    size_t stage_bytes = 0;

    int create(int lx, int ly, int precision, int scheme);
    void destroy();

    // per-step operations (asynchronous on `stream`)
    int op_collide();        // collide the current state in place or through the pull kernel
    int op_propagate();      // mark (or perform) the stream
    int materialize();       // form C + pending -> form L
    int zgb_pass();          // extrapolated outlet densities into the tables (zgb_src slots)
    int aa_step();           // one AA time step (even or odd kernel)
    int step(int nsteps);    // full native steps
    void view(int &v, int &par) const;  // read-out view and stale side parity of the state
    long long steps_done() const;

    // data movement
    int upload_bc(const double *bc);      // host [16*nb]
    int upload_zgb_src(const int *src);   // host [4*nb]
    int upload_tags(const uint8_t *tag_xy);  // host tag[X*(ly+2)+Y], validated here
    int upload_tag_plane(const uint8_t *plane);  // host plane in device layout
    int upload_records(int b, const double *host, int rs, int X0, int X1);
    // rows Y0..Y0+H-1 of columns X0..X1-1 from host records laid out like upload_records' (host
    // points at column X0, row 0)
    int upload_record_rows(int b, const double *host, int rs, int X0, int X1, int Y0, int H);
    // the stale-slot and ghost-ring sources of buffer b only: columns 0, 1, lx, lx+1 and rows
    // 0, 1, ly, ly+1 (the pull kernel writes the rest before anything reads it)
    int upload_records_edges(int b, const double *host, int rs);
    int upload_tags_xy(const uint8_t *tag_xy);   // host order, already validated
    int readout_records(double *host, int rs, const uint64_t *dynp_dev, int X0, int X1);
    int init_side_from(int b, int par);
    int init_cylinder(double umax);  // equilibrium Poiseuille populations into buffer 0
    int get_macros(double *rho, double *ux, double *uy);  // host [ly][lx] arrays
    int moments(double out[8]);                           // FP64 sums (kernels.h)
    int velocity_accumulate();
    int velocity_average(double *ux, double *uy, long long *samples);
    double *red_scratch = nullptr;  // (ly+2)*8 partial sums + 8 results
    double *vel_acc = nullptr;      // 2*lx*ly running velocity sums
    float *shift = nullptr;         // 16-bit storage: per-row shift velocity [ly+2] (d.g.shift_u)
    bool rs = false;                // 16-bit storage: stochastic rounding of stored values
    unsigned rs_seed = 0;
    // the keys of collision k (and k + 1, two-step sweep) into d.g before a collision launch
    void set_rs_keys(long long k);
    long long vel_samples = 0;
    int check(const char *what);   // cudaGetLastError -> error code
    int side_par_stale() const { return (int)((n + 1) & 1); }
    size_t stage_cols(int rs) const;
    int ensure_stage(size_t bytes_needed);
};

}  // namespace lbgpu

// The opaque handle of include/lbgpu.h.
struct lbgpu_lattice {
    lbgpu::Lattice L;
};
