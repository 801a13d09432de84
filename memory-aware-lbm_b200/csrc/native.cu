// native.cu -- the lbgpu_* functions of include/lbgpu.h (lattice object interface).
#include <cstring>
#include <vector>
#include "d2q9.cuh"
#include "lattice.h"
#include "lbgpu.h"

using lbgpu::Lattice;
using lbgpu::set_error;

namespace {

int bad_handle(const lbgpu_lattice *h, const char *fn)
{
    if (!h) return set_error(LB_ERR_ARG, "%s: null lattice", fn);
    return LB_OK;
}

// zgb_src for the native interface: right-side pressure slot Y takes row Y's extrapolation.
void zgb_slots_from_rows(const Lattice &L, const uint8_t *zgb_row, std::vector<int> &src,
                         bool &any)
{
    const int nb = L.d.g.nb;
    src.assign(4 * (size_t)nb, -1);
    any = false;
    if (!zgb_row) return;
    for (int Y = 0; Y < L.ly + 2; ++Y)
        if (zgb_row[Y]) {
            src[(size_t)3 * nb + Y] = Y;   // table 4 + right side -> index 3 of the 4 pressure tables
            any = true;
        }
}

bool zgb_wanted(const uint8_t *zgb_row, int ly)
{
    if (zgb_row)
        for (int Y = 0; Y < ly + 2; ++Y)
            if (zgb_row[Y]) return true;
    return false;
}

// Boundary tables, ZGB slots and omega of a geometry whose tags are already on the device.
int set_tables(Lattice &L, double omega, const double *bc, const uint8_t *zgb_row)
{
    std::vector<int> src;
    bool any = false;
    zgb_slots_from_rows(L, zgb_row, src, any);
    if (int rc = L.upload_bc(bc)) return rc;
    if (int rc = L.upload_zgb_src(src.data())) return rc;
    L.zgb_each_step = any;
    L.d.omega = omega;
    return LB_OK;
}

}  // namespace

extern "C" {

int lbGetLastError(void) { return lbgpu::last_error(); }
const char *lbGetLastErrorString(void) { return lbgpu::last_error_string(); }
void lbClearError(void) { lbgpu::clear_error(); }

int lbgpu_set_device(int device)
{
    int n = 0;
    if (int rc = lbgpu::cuda_error(cudaGetDeviceCount(&n), "cudaGetDeviceCount")) return rc;
    if (device < 0 || device >= n)
        return set_error(LB_ERR_NO_DEVICE, "device %d requested, %d present", device, n);
    return lbgpu::cuda_error(cudaSetDevice(device), "cudaSetDevice");
}

int lbgpu_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

int lbgpu_create(int lx, int ly, int precision, int scheme, lbgpu_lattice **out)
{
    if (!out) return set_error(LB_ERR_ARG, "lbgpu_create: null output pointer");
    *out = nullptr;
    lbgpu_lattice *h = new lbgpu_lattice;
    int rc = h->L.create(lx, ly, precision, scheme);
    if (rc != LB_OK) {
        h->L.destroy();
        delete h;
        return rc;
    }
    *out = h;
    return LB_OK;
}

int lbgpu_destroy(lbgpu_lattice *h)
{
    if (!h) return LB_OK;
    h->L.destroy();
    delete h;
    return LB_OK;
}

int lbgpu_set_geometry(lbgpu_lattice *h, double omega, const uint8_t *tag, const double *bc,
                       const uint8_t *zgb_row)
{
    if (int rc = bad_handle(h, "lbgpu_set_geometry")) return rc;
    if (!tag || !bc) return set_error(LB_ERR_ARG, "lbgpu_set_geometry: null tag or table");
    Lattice &L = h->L;
    if (zgb_wanted(zgb_row, L.ly) && L.lx < 2)
        return set_error(LB_ERR_ARG, "extrapolated outlet needs lx >= 2");
    if (int rc = L.upload_tags(tag)) return rc;
    return set_tables(L, omega, bc, zgb_row);
}

int lbgpu_set_offset_scale(lbgpu_lattice *h, int scale_log2)
{
    if (int rc = bad_handle(h, "lbgpu_set_offset_scale")) return rc;
    if (scale_log2 < -30 || scale_log2 > 30)
        return set_error(LB_ERR_ARG, "offset scale 2^%d out of range", scale_log2);
    h->L.d.scale = ldexpf(1.0f, scale_log2);
    h->L.d.inv_scale = ldexpf(1.0f, -scale_log2);
    return LB_OK;
}

int lbgpu_set_offset_shift(lbgpu_lattice *h, const double *u_row)
{
    if (int rc = bad_handle(h, "lbgpu_set_offset_shift")) return rc;
    Lattice &L = h->L;
    if (L.precision != LBGPU_F16 && L.precision != LBGPU_BF16)
        return set_error(LB_ERR_STATE, "lbgpu_set_offset_shift: FP16/BF16 storage only");
    if (!u_row) {
        if (L.shift) {
            if (int rc = lbgpu::cuda_error(cudaStreamSynchronize(L.stream), "lbgpu_set_offset_shift")) return rc;
            cudaFree(L.shift);
        }
        L.shift = nullptr;
        L.d.g.shift_u = nullptr;
        return LB_OK;
    }
    // the table of Geo::shift_u: u_s[Y], S_i(Y), S_i(Y) - S_i(Y + c_iy) (layout.cuh), in FP64
    // from the float velocities, then rounded once, so every kernel reads the same values
    const int ny2 = L.ly + 2;
    std::vector<float> u(20 * (size_t)ny2, 0.0f);
    for (int Y = 0; Y < ny2; ++Y) {
        if (!(u_row[Y] > -0.5 && u_row[Y] < 0.5))
            return set_error(LB_ERR_ARG, "lbgpu_set_offset_shift: u[%d] = %g out of range", Y, u_row[Y]);
        u[Y] = (float)u_row[Y];
    }
    auto S = [&](int i, int Y) {
        const double v = (double)u[Y], c = (double)lbgpu::cx(i), w = (double)lbgpu::wgtf(i);
        return w * (1.0 + 3.0 * c * v + 4.5 * c * c * v * v - 1.5 * v * v);
    };
    for (int Y = 0; Y < ny2; ++Y)
        for (int i = 0; i < 9; ++i) {
            u[ny2 + 9 * Y + i] = (float)S(i, Y);
            const int Yc = Y + lbgpu::cy(i);
            if (lbgpu::cy(i) != 0 && Yc >= 0 && Yc < ny2) u[10 * ny2 + 9 * Y + i] = (float)(S(i, Y) - S(i, Yc));
            if (u[10 * ny2 + 9 * Y + i] != 0.0f) u[19 * ny2 + Y] = 1.0f;
        }
    if (!L.shift) {
        void *p = nullptr;
        if (int rc = lbgpu::cuda_error(cudaMalloc(&p, u.size() * sizeof(float)), "cudaMalloc(offset shift)")) return rc;
        L.shift = static_cast<float *>(p);
    }
    if (int rc = lbgpu::cuda_error(cudaMemcpyAsync(L.shift, u.data(), u.size() * sizeof(float),
                                                   cudaMemcpyHostToDevice, L.stream), "upload offset shift"))
        return rc;
    if (int rc = lbgpu::cuda_error(cudaStreamSynchronize(L.stream), "upload offset shift")) return rc;
    L.d.g.shift_u = L.shift;
    return LB_OK;
}

int lbgpu_set_stochastic_rounding(lbgpu_lattice *h, int on, unsigned seed)
{
    if (int rc = bad_handle(h, "lbgpu_set_stochastic_rounding")) return rc;
    Lattice &L = h->L;
    if (L.precision != LBGPU_F16 && L.precision != LBGPU_BF16)
        return set_error(LB_ERR_STATE, "lbgpu_set_stochastic_rounding: FP16/BF16 storage only");
    if (on != 0 && on != 1) return set_error(LB_ERR_ARG, "lbgpu_set_stochastic_rounding: on = %d", on);
    L.rs = on != 0;
    L.rs_seed = seed;
    L.d.g.rs_key = 0;
    L.d.g.rs_key2 = 0;
    return LB_OK;
}

int lbgpu_set_populations(lbgpu_lattice *h, const double *f, const double *tmp)
{
    if (int rc = bad_handle(h, "lbgpu_set_populations")) return rc;
    if (!f) return set_error(LB_ERR_ARG, "lbgpu_set_populations: null populations");
    Lattice &L = h->L;
    L.launches = 0;
    if (L.scheme == LBGPU_AA) {
        // one buffer: the second buffer only matters through its stale slots (side parity 1,
        // read by the first odd step); the first buffer's own stale slots go to parity 0
        // and, for odd step counts, through the ghost slots nothing streams into (ghost2)
        if (tmp) {
            if (int rc = L.upload_records(0, tmp, 9, 0, L.lx + 2)) return rc;
            if (int rc = L.init_side_from(0, 1)) return rc;
            lbgpu::launch_ghost_copy(L.d, 0, L.stream);
        } else {
            if (int rc = lbgpu::cuda_error(cudaMemsetAsync(L.d.side, 0, 2 * 9 * (size_t)L.d.g.nper * L.elem,
                                                           L.stream), "clear side store"))
                return rc;
            if (int rc = lbgpu::cuda_error(cudaMemsetAsync(L.d.ghost2, 0, 9 * (size_t)L.d.g.nghost() * L.elem,
                                                           L.stream), "clear ghost ring"))
                return rc;
        }
        if (int rc = L.upload_records(0, f, 9, 0, L.lx + 2)) return rc;
        if (int rc = L.init_side_from(0, 0)) return rc;
    } else {
        if (int rc = L.upload_records(0, f, 9, 0, L.lx + 2)) return rc;
        if (tmp) {
            if (int rc = L.upload_records(1, tmp, 9, 0, L.lx + 2)) return rc;
        } else {
            if (int rc = lbgpu::cuda_error(cudaMemsetAsync(L.d.buf[1], 0, 9 * (size_t)L.d.g.plane * L.elem,
                                                           L.stream), "clear second buffer"))
                return rc;
        }
        // the first stream leaves the second buffer's content in the stale slots: side parity 1
        if (int rc = L.init_side_from(1, 1)) return rc;
    }
    L.cur = 0; L.form = lbgpu::FORM_L; L.pending = 0; L.n = 0;
    return lbgpu::cuda_error(cudaStreamSynchronize(L.stream), "lbgpu_set_populations");
}

int lbgpu_setup_cylinder(lbgpu_lattice *h, int obst_x, int obst_y, int obst_r, double umax,
                         double re, int wall_kind, int outlet_kind, double *omega_out)
{
    if (int rc = bad_handle(h, "lbgpu_setup_cylinder")) return rc;
    Lattice &L = h->L;
    // the tag plane is written on the device (O(nodes)); the boundary tables, O(perimeter),
    // come from the host builder
    std::vector<uint8_t> zgb(L.ly + 2);
    std::vector<double> bc(16 * (size_t)L.d.g.nb);
    const double omega = lbgpu_build_cylinder(L.lx, L.ly, obst_x, obst_y, obst_r, umax, re,
                                              wall_kind, outlet_kind, nullptr, bc.data(),
                                              zgb.data(), nullptr);
    if (omega_out) *omega_out = omega;
    if (zgb_wanted(zgb.data(), L.ly) && L.lx < 2)
        return set_error(LB_ERR_ARG, "extrapolated outlet needs lx >= 2");
    lbgpu::launch_cylinder_tags(L.d, obst_x, obst_y, obst_r, wall_kind, L.stream);
    if (int rc = lbgpu::cuda_error(cudaGetLastError(), "cylinder tags")) return rc;
    if (int rc = set_tables(L, omega, bc.data(), zgb.data())) return rc;
    L.launches = 0;
    for (int b = 0; b < 2; ++b)
        if (L.d.buf[b])
            if (int rc = lbgpu::cuda_error(cudaMemsetAsync(L.d.buf[b], 0, 9 * (size_t)L.d.g.plane * L.elem,
                                                           L.stream), "clear populations"))
                return rc;
    if (int rc = lbgpu::cuda_error(cudaMemsetAsync(L.d.side, 0, 2 * 9 * (size_t)L.d.g.nper * L.elem,
                                                   L.stream), "clear side store"))
        return rc;
    if (int rc = L.init_cylinder(umax)) return rc;
    // second buffer zero (reference calloc, lb.c:91-92): side parity 1 stays zero; the AA scheme
    // reads the initial state's own stale slots from parity 0
    if (L.scheme == LBGPU_AA) {
        if (int rc = L.init_side_from(0, 0)) return rc;
        if (int rc = lbgpu::cuda_error(cudaMemsetAsync(L.d.ghost2, 0, 9 * (size_t)L.d.g.nghost() * L.elem,
                                                       L.stream), "clear ghost ring"))
            return rc;
    }
    L.cur = 0; L.form = lbgpu::FORM_L; L.pending = 0; L.n = 0;
    return lbgpu::cuda_error(cudaStreamSynchronize(L.stream), "lbgpu_setup_cylinder");
}

int lbgpu_set_sweep_steps(lbgpu_lattice *h, int steps)
{
    if (int rc = bad_handle(h, "lbgpu_set_sweep_steps")) return rc;
    if (steps != 1 && steps != 2) return set_error(LB_ERR_ARG, "lbgpu_set_sweep_steps: %d (1 or 2)", steps);
    if (steps == 2 && h->L.scheme != LBGPU_PULL)
        return set_error(LB_ERR_STATE, "two steps per sweep needs the pull scheme");
    h->L.sweep_steps = steps;
    return LB_OK;
}

int lbgpu_step(lbgpu_lattice *h, int nsteps)
{
    if (int rc = bad_handle(h, "lbgpu_step")) return rc;
    return h->L.step(nsteps);
}

int lbgpu_step_timed(lbgpu_lattice *h, int nsteps, float *ms)
{
    if (int rc = bad_handle(h, "lbgpu_step_timed")) return rc;
    Lattice &L = h->L;
    cudaEvent_t e0, e1;
    if (int rc = lbgpu::cuda_error(cudaEventCreate(&e0), "cudaEventCreate")) return rc;
    if (int rc = lbgpu::cuda_error(cudaEventCreate(&e1), "cudaEventCreate")) {
        cudaEventDestroy(e0);
        return rc;
    }
    int rc = lbgpu::cuda_error(cudaEventRecord(e0, L.stream), "cudaEventRecord");
    if (rc == LB_OK) rc = L.step(nsteps);
    if (rc == LB_OK) rc = lbgpu::cuda_error(cudaEventRecord(e1, L.stream), "cudaEventRecord");
    if (rc == LB_OK) rc = lbgpu::cuda_error(cudaEventSynchronize(e1), "cudaEventSynchronize");
    float t = 0.f;
    if (rc == LB_OK) rc = lbgpu::cuda_error(cudaEventElapsedTime(&t, e0, e1), "cudaEventElapsedTime");
    if (ms) *ms = t;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

int lbgpu_get_populations(lbgpu_lattice *h, double *f)
{
    if (int rc = bad_handle(h, "lbgpu_get_populations")) return rc;
    if (!f) return set_error(LB_ERR_ARG, "lbgpu_get_populations: null output");
    return h->L.readout_records(f, 9, nullptr, 0, h->L.lx + 2);
}

int lbgpu_get_macros(lbgpu_lattice *h, double *rho, double *ux, double *uy)
{
    if (int rc = bad_handle(h, "lbgpu_get_macros")) return rc;
    return h->L.get_macros(rho, ux, uy);
}

int lbgpu_moments(lbgpu_lattice *h, double out[8])
{
    if (int rc = bad_handle(h, "lbgpu_moments")) return rc;
    if (!out) return set_error(LB_ERR_ARG, "lbgpu_moments: null output");
    return h->L.moments(out);
}

int lbgpu_velocity_accumulate(lbgpu_lattice *h)
{
    if (int rc = bad_handle(h, "lbgpu_velocity_accumulate")) return rc;
    return h->L.velocity_accumulate();
}

int lbgpu_velocity_average(lbgpu_lattice *h, double *ux, double *uy, long long *samples)
{
    if (int rc = bad_handle(h, "lbgpu_velocity_average")) return rc;
    return h->L.velocity_average(ux, uy, samples);
}

int lbgpu_velocity_reset(lbgpu_lattice *h)
{
    if (int rc = bad_handle(h, "lbgpu_velocity_reset")) return rc;
    lbgpu::Lattice &L = h->L;
    L.vel_samples = 0;
    if (!L.vel_acc) return LB_OK;
    return lbgpu::cuda_error(cudaMemsetAsync(L.vel_acc, 0, 2 * (size_t)L.lx * L.ly * sizeof(double), L.stream),
                             "lbgpu_velocity_reset");
}

int lbgpu_synchronize(lbgpu_lattice *h)
{
    if (int rc = bad_handle(h, "lbgpu_synchronize")) return rc;
    return lbgpu::cuda_error(cudaStreamSynchronize(h->L.stream), "lbgpu_synchronize");
}

void *lbgpu_stream(lbgpu_lattice *h) { return h ? (void *)h->L.stream : nullptr; }
long long lbgpu_steps_done(lbgpu_lattice *h)
{
    return h ? h->L.steps_done() : 0;
}
size_t lbgpu_device_bytes(lbgpu_lattice *h) { return h ? h->L.bytes : 0; }
int lbgpu_last_kernel_launches(lbgpu_lattice *h) { return h ? h->L.launches : 0; }

}  // extern "C"
