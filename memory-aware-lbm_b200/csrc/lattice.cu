// lattice.cu -- allocation, state machine and data movement of a device lattice.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include "codec.cuh"
#include "lattice.h"
#include "lbgpu.h"

namespace lbgpu {

// ---- thread-local error state ---------------------------------------------------------
namespace {
thread_local int g_err = 0;
thread_local char g_msg[512] = "";
}  // namespace

int set_error(int code, const char *fmt, ...)
{
    if (g_err == 0) {  // keep the first error until cleared
        g_err = code;
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(g_msg, sizeof g_msg, fmt, ap);
        va_end(ap);
    }
    return code;
}

int cuda_error(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return LB_OK;
    if (e == cudaErrorMemoryAllocation)
        return set_error(LB_ERR_ALLOC, "%s: %s", what, cudaGetErrorString(e));
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        return set_error(LB_ERR_NO_DEVICE, "%s: %s", what, cudaGetErrorString(e));
    return set_error(LB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

int last_error() { return g_err; }
const char *last_error_string() { return g_msg; }
void clear_error() { g_err = 0; g_msg[0] = 0; }

#define LB_TRY(expr)                                \
    do {                                            \
        int rc_ = (expr);                           \
        if (rc_ != LB_OK) return rc_;               \
    } while (0)
#define LB_CUDA(call, what) LB_TRY(cuda_error((call), (what)))

// ---- lifetime -------------------------------------------------------------------------
static size_t elem_bytes(int precision)
{
    switch (precision) {
    case LBGPU_F64: return 8;
    case LBGPU_F32: return 4;
    default: return 2;
    }
}

int Lattice::create(int lx_, int ly_, int precision_, int scheme_)
{
    // The row-wise kernels launch one grid row per lattice row, ghost rows included, and CUDA
    // caps gridDim.y at 65535: hence ly <= LBGPU_MAX_LY.
    if (lx_ < 1 || ly_ < 1 || lx_ > LBGPU_MAX_LX || ly_ > LBGPU_MAX_LY)
        return set_error(LB_ERR_ARG, "lattice size %d x %d out of range (1..%d x 1..%d)", lx_, ly_,
                         LBGPU_MAX_LX, LBGPU_MAX_LY);
    if (precision_ < LBGPU_F64 || precision_ > LBGPU_BF16)
        return set_error(LB_ERR_ARG, "unknown precision %d", precision_);
    if (scheme_ != LBGPU_PULL && scheme_ != LBGPU_AA)
        return set_error(LB_ERR_ARG, "unknown scheme %d", scheme_);
    lx = lx_; ly = ly_; precision = precision_; scheme = scheme_;
    elem = elem_bytes(precision);
    d.g = make_geo(lx, ly, (int)elem);
    d.precision = precision;
    d.omega = 1.0;
    d.scale = 1.0f; d.inv_scale = 1.0f;
    int ndev = 0;
    LB_CUDA(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
    if (ndev == 0) return set_error(LB_ERR_NO_DEVICE, "no CUDA device");
    LB_CUDA(cudaGetDevice(&device), "cudaGetDevice");
    LB_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");

    const size_t nbuf = (scheme == LBGPU_AA) ? 1 : 2;
    const size_t pbytes = 9 * (size_t)d.g.plane * elem;
    // two parities, and for the pull scheme the scratch of the two-step kernel
    const size_t sbytes = (scheme == LBGPU_PULL ? 3 : 2) * 9 * (size_t)d.g.nper * elem;
    void *p = nullptr;
    for (size_t b = 0; b < nbuf; ++b) {
        LB_CUDA(cudaMalloc(&p, pbytes), "cudaMalloc(populations)");
        d.buf[b] = p;
        LB_CUDA(cudaMemsetAsync(p, 0, pbytes, stream), "cudaMemset(populations)");
    }
    if (scheme == LBGPU_AA) {
        const size_t gbytes = 9 * (size_t)d.g.nghost() * elem;
        LB_CUDA(cudaMalloc(&p, gbytes), "cudaMalloc(ghost ring)");
        d.ghost2 = p;
        LB_CUDA(cudaMemsetAsync(p, 0, gbytes, stream), "cudaMemset(ghost ring)");
        bytes += gbytes;
    }
    LB_CUDA(cudaMalloc(&p, sbytes), "cudaMalloc(side store)");
    d.side = p;
    LB_CUDA(cudaMemsetAsync(p, 0, sbytes, stream), "cudaMemset(side store)");
    LB_CUDA(cudaMalloc(&p, (size_t)d.g.plane), "cudaMalloc(tags)");
    d.tag = static_cast<const uint8_t *>(p);
    LB_CUDA(cudaMemsetAsync(p, 0, (size_t)d.g.plane, stream), "cudaMemset(tags)");
    LB_CUDA(cudaMalloc(&p, 16 * (size_t)d.g.nb * sizeof(double)), "cudaMalloc(tables)");
    d.bc = static_cast<double *>(p);
    LB_CUDA(cudaMemsetAsync(p, 0, 16 * (size_t)d.g.nb * sizeof(double), stream), "cudaMemset");
    LB_CUDA(cudaMalloc(&p, 4 * (size_t)d.g.nb * sizeof(int)), "cudaMalloc(zgb slots)");
    d.zgb_src = static_cast<const int *>(p);
    LB_CUDA(cudaMemsetAsync(p, 0xff, 4 * (size_t)d.g.nb * sizeof(int), stream), "cudaMemset");
    LB_CUDA(cudaMalloc(&p, 2 * (size_t)(ly + 2) * sizeof(double)), "cudaMalloc(zgb rho)");
    d.zrho = static_cast<double *>(p);
    LB_CUDA(cudaMemsetAsync(p, 0, 2 * (size_t)(ly + 2) * sizeof(double), stream), "cudaMemset");
    bytes += nbuf * pbytes + sbytes + (size_t)d.g.plane + 16 * (size_t)d.g.nb * 8 +
            4 * (size_t)d.g.nb * 4 + 2 * (size_t)(ly + 2) * 8;
    bc_host.assign(16 * (size_t)d.g.nb, 0.0);
    zgb_src_host.assign(4 * (size_t)d.g.nb, -1);
    cur = 0; form = FORM_L; pending = 0; n = 0;
    return check("lattice create");
}

void Lattice::destroy()
{
    if (stream) cudaStreamSynchronize(stream);
    for (int b = 0; b < 2; ++b) if (d.buf[b]) cudaFree(d.buf[b]);
    if (d.side) cudaFree(d.side);
    if (d.ghost2) cudaFree(d.ghost2);
    if (d.tag) cudaFree(const_cast<uint8_t *>(d.tag));
    if (d.bc) cudaFree(d.bc);
    if (d.zgb_src) cudaFree(const_cast<int *>(d.zgb_src));
    if (d.zrho) cudaFree(d.zrho);
    if (stage) cudaFree(stage);
    if (red_scratch) cudaFree(red_scratch);
    if (vel_acc) cudaFree(vel_acc);
    if (shift) cudaFree(shift);
    red_scratch = nullptr; vel_acc = nullptr; vel_samples = 0; shift = nullptr;
    if (stream) cudaStreamDestroy(stream);
    d = DevLattice{};
    stage = nullptr; stage_bytes = 0; stream = nullptr;
}

int Lattice::check(const char *what)
{
    return cuda_error(cudaGetLastError(), what);
}

// How the post-stream state is read, and which side parity holds its stale slots.
void Lattice::view(int &v, int &par) const
{
    if (scheme == LBGPU_AA) {
        if (form == FORM_L) { v = VIEW_AA_NATURAL; par = (int)(n & 1); }
        else { v = VIEW_AA_SWAPPED; par = (int)((n + 1) & 1); }
        return;
    }
    par = (int)((n + 1) & 1);
    v = (form == FORM_C && pending) ? VIEW_PULL_PENDING : VIEW_DIRECT;
}

// Collision k produces the post-collision state C_k; its stored values round with key k.
void Lattice::set_rs_keys(long long k)
{
    d.g.rs_key = rs ? rs_key(rs_seed, (unsigned long long)k) : 0u;
    d.g.rs_key2 = rs ? rs_key(rs_seed, (unsigned long long)(k + 1)) : 0u;
}

// ---- state machine (pull scheme) ------------------------------------------------------
int Lattice::op_collide()
{
    if (scheme != LBGPU_PULL) return set_error(LB_ERR_STATE, "collide/propagate need the pull scheme");
    if (form == FORM_C && pending) {
        set_rs_keys(n + 1);
        launch_pull(d, cur, (int)((n + 1) & 1), ghosts, stream);
        launches += pull_launches(d, ghosts) - 1;
        cur = 1 - cur;
        ++n;
    } else {
        set_rs_keys(n);
        launch_collide_inplace(d, cur, (int)(n & 1), stream);
        form = FORM_C;
    }
    pending = 0;
    ++launches;
    return check("collide");
}

int Lattice::materialize()
{
    if (scheme != LBGPU_PULL) return set_error(LB_ERR_STATE, "materialize needs the pull scheme");
    if (form == FORM_C && pending) {
        launch_stream(d, cur, (int)((n + 1) & 1), stream);
        cur = 1 - cur;
        ++n;
        form = FORM_L;
        pending = 0;
        ++launches;
    }
    return check("stream");
}

int Lattice::op_propagate()
{
    if (scheme != LBGPU_PULL) return set_error(LB_ERR_STATE, "collide/propagate need the pull scheme");
    if (form == FORM_C && !pending) {
        pending = 1;
        return LB_OK;
    }
    LB_TRY(materialize());
    // stream of an uncollided state: it acts as its own post-collision state
    launch_side_from_buf(d, cur, (int)(n & 1), stream);
    ++launches;
    form = FORM_C;
    pending = 1;
    return check("propagate");
}

int Lattice::zgb_pass()
{
    if (lx < 2) return set_error(LB_ERR_ARG, "the extrapolated outlet needs lx >= 2");
    if (scheme == LBGPU_PULL && form == FORM_C && !pending)
        return set_error(LB_ERR_STATE, "extrapolated outlet requested on a collided state");
    int v, par;
    view(v, par);
    launch_zgb_rho(d, v, cur, par, stream);
    launch_zgb_apply(d, stream);
    launches += 2;
    return check("zgb pass");
}

// One AA time step: natural form -> even kernel (C_m into the opposite slots); swapped form ->
// odd kernel (gather, collide, scatter), leaving the natural form two steps on.
int Lattice::aa_step()
{
    if (form == FORM_L) {
        set_rs_keys(n);
        launch_aa_even(d, (int)(n & 1), stream);
        form = FORM_C;
        pending = 1;
    } else {
        set_rs_keys(n + 1);
        launch_aa_odd(d, (int)((n + 1) & 1), stream);
        n += 2;
        form = FORM_L;
        pending = 0;
    }
    ++launches;
    return check("aa step");
}

int Lattice::step(int nsteps)
{
    if (nsteps < 0) return set_error(LB_ERR_ARG, "negative step count");
    launches = 0;
    for (int s = 0; s < nsteps; ++s) {
        if (zgb_each_step) LB_TRY(zgb_pass());
        if (scheme == LBGPU_AA) {
            LB_TRY(aa_step());
        } else if (sweep_steps == 2 && nsteps - s >= 2 && !zgb_each_step && !ghosts && form == FORM_C && pending) {
            // two steps in one sweep: C_n -> C_{n+2} in the other buffer, still pending
            set_rs_keys(n + 1);
            launch_pull2(d, cur, (int)(n & 1), stream);
            launches += 2;
            cur = 1 - cur;
            n += 2;
            ++s;
            LB_TRY(check("two-step pull"));
        } else {
            LB_TRY(op_collide());
            LB_TRY(op_propagate());
        }
    }
    return LB_OK;
}

long long Lattice::steps_done() const
{
    if (form == FORM_C && pending) return n + 1;
    return n;
}

// ---- data movement --------------------------------------------------------------------
int Lattice::ensure_stage(size_t need)
{
    if (stage_bytes >= need) return LB_OK;
    if (stage) { cudaStreamSynchronize(stream); cudaFree(stage); stage = nullptr; stage_bytes = 0; }
    void *p = nullptr;
    LB_CUDA(cudaMalloc(&p, need), "cudaMalloc(staging)");
    stage = static_cast<double *>(p);
    stage_bytes = need;
    return LB_OK;
}

size_t Lattice::stage_cols(int rs) const
{
    const size_t col = (size_t)(ly + 2) * rs * sizeof(double);
    size_t cols = ((size_t)64 << 20) / col;
    if (cols < 1) cols = 1;
    if (cols > (size_t)(lx + 2)) cols = (size_t)(lx + 2);
    if (cols > kMaxGridY) cols = kMaxGridY;   // one grid row a column in the copy kernels
    return cols;
}

int Lattice::upload_records(int b, const double *host, int rs, int X0, int X1)
{
    const size_t col = (size_t)(ly + 2) * rs;
    const size_t cols = stage_cols(rs);
    LB_TRY(ensure_stage(cols * col * sizeof(double)));
    for (int c0 = X0; c0 < X1; c0 += (int)cols) {
        const int c1 = (c0 + (int)cols < X1) ? c0 + (int)cols : X1;
        LB_CUDA(cudaMemcpyAsync(stage, host + (size_t)(c0 - X0) * col,
                                (size_t)(c1 - c0) * col * sizeof(double),
                                cudaMemcpyHostToDevice, stream), "upload populations");
        h2d_bytes += (size_t)(c1 - c0) * col * sizeof(double);
        launch_upload(d, b, stage, rs, c0, c1, 0, ly + 2, stream);
        ++launches;
    }
    return check("upload");
}

int Lattice::upload_record_rows(int b, const double *host, int rs, int X0, int X1, int Y0, int H)
{
    if (X1 <= X0 || H <= 0) return LB_OK;
    const size_t col = (size_t)(ly + 2) * rs, band = (size_t)H * rs;
    size_t cols = ((size_t)64 << 20) / (band * sizeof(double));
    if (cols < 1) cols = 1;
    if (cols > (size_t)(X1 - X0)) cols = (size_t)(X1 - X0);
    if (cols > kMaxGridY) cols = kMaxGridY;
    LB_TRY(ensure_stage(cols * band * sizeof(double)));
    for (int c0 = X0; c0 < X1; c0 += (int)cols) {
        const int c1 = (c0 + (int)cols < X1) ? c0 + (int)cols : X1;
        LB_CUDA(cudaMemcpy2DAsync(stage, band * sizeof(double), host + (size_t)(c0 - X0) * col + (size_t)Y0 * rs,
                                  col * sizeof(double), band * sizeof(double), (size_t)(c1 - c0),
                                  cudaMemcpyHostToDevice, stream), "upload population rows");
        h2d_bytes += (size_t)(c1 - c0) * band * sizeof(double);
        launch_upload(d, b, stage, rs, c0, c1, Y0, H, stream);
        ++launches;
    }
    return check("upload rows");
}

int Lattice::upload_records_edges(int b, const double *host, int rs)
{
    if (lx < 4 || ly < 4) return upload_records(b, host, rs, 0, lx + 2);
    const size_t col = (size_t)(ly + 2) * rs;
    LB_TRY(upload_records(b, host, rs, 0, 2));
    LB_TRY(upload_records(b, host + (size_t)lx * col, rs, lx, lx + 2));
    LB_TRY(upload_record_rows(b, host + 2 * col, rs, 2, lx, 0, 2));
    return upload_record_rows(b, host + 2 * col, rs, 2, lx, ly, 2);
}

int Lattice::readout_records(double *host, int rs, const uint64_t *dynp_dev, int X0, int X1)
{
    const size_t col = (size_t)(ly + 2) * rs;
    const size_t cols = stage_cols(rs);
    LB_TRY(ensure_stage(cols * col * sizeof(double)));
    int v, par;
    view(v, par);
    for (int c0 = X0; c0 < X1; c0 += (int)cols) {
        const int c1 = (c0 + (int)cols < X1) ? c0 + (int)cols : X1;
        launch_readout(d, v, cur, par, c0, c1, stage, rs, dynp_dev, stream);
        ++launches;
        LB_CUDA(cudaMemcpyAsync(host + (size_t)(c0 - X0) * col, stage,
                                (size_t)(c1 - c0) * col * sizeof(double),
                                cudaMemcpyDeviceToHost, stream), "download populations");
        d2h_bytes += (size_t)(c1 - c0) * col * sizeof(double);
    }
    LB_CUDA(cudaStreamSynchronize(stream), "readout");
    return check("readout");
}

int Lattice::init_side_from(int b, int par)
{
    launch_side_from_buf(d, b, par, stream);
    ++launches;
    return check("side store init");
}

int Lattice::init_cylinder(double umax)
{
    launch_init_cylinder(d, 0, umax, stream);
    ++launches;
    return check("init cylinder");
}

int Lattice::get_macros(double *rho, double *ux, double *uy)
{
    const size_t nn = (size_t)lx * ly;
    double *dev = nullptr;
    LB_CUDA(cudaMalloc(&dev, 3 * nn * sizeof(double)), "cudaMalloc(macros)");
    int v, par;
    view(v, par);
    launch_macros(d, v, cur, par, dev, dev + nn, dev + 2 * nn, stream);
    int rc = check("macros");
    if (rc == LB_OK && rho) rc = cuda_error(cudaMemcpyAsync(rho, dev, nn * 8, cudaMemcpyDeviceToHost, stream), "macros");
    if (rc == LB_OK && ux) rc = cuda_error(cudaMemcpyAsync(ux, dev + nn, nn * 8, cudaMemcpyDeviceToHost, stream), "macros");
    if (rc == LB_OK && uy) rc = cuda_error(cudaMemcpyAsync(uy, dev + 2 * nn, nn * 8, cudaMemcpyDeviceToHost, stream), "macros");
    if (rc == LB_OK) rc = cuda_error(cudaStreamSynchronize(stream), "macros");
    d2h_bytes += nn * 8 * ((rho != nullptr) + (ux != nullptr) + (uy != nullptr));
    cudaFree(dev);
    return rc;
}

int Lattice::moments(double out[8])
{
    if (!red_scratch) {
        void *p = nullptr;
        LB_CUDA(cudaMalloc(&p, ((size_t)(ly + 2) * 8 + 8) * sizeof(double)), "cudaMalloc(reduction)");
        red_scratch = static_cast<double *>(p);
    }
    int v, par;
    view(v, par);
    double *res = red_scratch + (size_t)(ly + 2) * 8;
    launch_moments(d, v, cur, par, red_scratch, res, stream);
    LB_TRY(check("moments"));
    LB_CUDA(cudaMemcpyAsync(out, res, 8 * sizeof(double), cudaMemcpyDeviceToHost, stream), "moments");
    d2h_bytes += 8 * sizeof(double);
    LB_CUDA(cudaStreamSynchronize(stream), "moments");
    return LB_OK;
}

int Lattice::velocity_accumulate()
{
    const size_t bytes = 2 * (size_t)lx * ly * sizeof(double);
    if (!vel_acc) {
        void *p = nullptr;
        LB_CUDA(cudaMalloc(&p, bytes), "cudaMalloc(velocity sums)");
        vel_acc = static_cast<double *>(p);
        LB_CUDA(cudaMemsetAsync(vel_acc, 0, bytes, stream), "clear velocity sums");
        vel_samples = 0;
    }
    int v, par;
    view(v, par);
    launch_accumulate_velocity(d, v, cur, par, vel_acc, stream);
    ++vel_samples;
    return check("velocity accumulate");
}

int Lattice::velocity_average(double *ux, double *uy, long long *samples)
{
    const size_t nn = (size_t)lx * ly;
    if (samples) *samples = vel_samples;
    if (!vel_acc || vel_samples == 0) return set_error(LB_ERR_STATE, "no velocity samples accumulated");
    if (ux) LB_CUDA(cudaMemcpyAsync(ux, vel_acc, nn * 8, cudaMemcpyDeviceToHost, stream), "velocity average");
    if (uy) LB_CUDA(cudaMemcpyAsync(uy, vel_acc + nn, nn * 8, cudaMemcpyDeviceToHost, stream), "velocity average");
    LB_CUDA(cudaStreamSynchronize(stream), "velocity average");
    d2h_bytes += nn * 8 * ((ux != nullptr) + (uy != nullptr));
    const double k = 1.0 / (double)vel_samples;
    for (size_t i = 0; i < nn; ++i) {
        if (ux) ux[i] *= k;
        if (uy) uy[i] *= k;
    }
    return LB_OK;
}

int Lattice::upload_bc(const double *bc)
{
    std::memcpy(bc_host.data(), bc, bc_host.size() * sizeof(double));
    LB_CUDA(cudaMemcpyAsync(d.bc, bc_host.data(), bc_host.size() * sizeof(double),
                            cudaMemcpyHostToDevice, stream), "upload tables");
    h2d_bytes += bc_host.size() * sizeof(double);
    // the copy reads bc_host asynchronously: wait so the caller may reuse its array and
    // the next refresh may overwrite bc_host
    LB_CUDA(cudaStreamSynchronize(stream), "upload tables");
    return LB_OK;
}

int Lattice::upload_zgb_src(const int *src)
{
    std::memcpy(zgb_src_host.data(), src, zgb_src_host.size() * sizeof(int));
    LB_CUDA(cudaMemcpyAsync(const_cast<int *>(d.zgb_src), zgb_src_host.data(),
                            zgb_src_host.size() * sizeof(int), cudaMemcpyHostToDevice, stream),
            "upload zgb slots");
    h2d_bytes += zgb_src_host.size() * sizeof(int);
    LB_CUDA(cudaStreamSynchronize(stream), "upload zgb slots");
    return LB_OK;
}

int Lattice::upload_tag_plane(const uint8_t *plane)
{
    LB_CUDA(cudaMemcpyAsync(const_cast<uint8_t *>(d.tag), plane, (size_t)d.g.plane,
                            cudaMemcpyHostToDevice, stream), "upload tags");
    h2d_bytes += (size_t)d.g.plane;
    LB_CUDA(cudaStreamSynchronize(stream), "upload tags");
    return LB_OK;
}

int Lattice::upload_tags(const uint8_t *tag_xy)
{
    for (int X = 0; X < lx + 2; ++X)
        for (int Y = 0; Y < ly + 2; ++Y) {
            const int t = tag_xy[(size_t)X * (ly + 2) + Y];
            if (t >= LBGPU_NUM_TAGS)
                return set_error(LB_ERR_ARG, "tag %d at (%d,%d) out of range", t, X, Y);
            if (d.g.interior(X, Y) && t == LBGPU_TAG_NONE)
                return set_error(LB_ERR_DYNAMICS, "interior node (%d,%d) has no dynamics", X, Y);
        }
    return upload_tags_xy(tag_xy);
}

// The host array in its own order to the device, transposed there (a host transpose writes one
// byte a cache line).
int Lattice::upload_tags_xy(const uint8_t *tag_xy)
{
    const size_t n = (size_t)(lx + 2) * (ly + 2);
    LB_TRY(ensure_stage(n));
    LB_CUDA(cudaMemcpyAsync(stage, tag_xy, n, cudaMemcpyHostToDevice, stream), "upload tags");
    h2d_bytes += n;
    launch_tags_from_xy(d, reinterpret_cast<const uint8_t *>(stage), stream);
    LB_TRY(check("tags"));
    LB_CUDA(cudaStreamSynchronize(stream), "upload tags");
    return LB_OK;
}

}  // namespace lbgpu
