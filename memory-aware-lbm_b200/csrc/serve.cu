// serve.cu -- continuous-batching request loop (lbgpu_server_* of include/lbgpu.h).
//
// Requests (a cylinder channel, a step cap and a steady-state tolerance) arrive over wall-clock
// time.  The loop admits them in arrival order while their lattices fit the HBM budget, keeps
// every admitted lattice resident, advances them `check_every` steps at a time, and after each
// advance retires every member that reached its step cap or whose largest velocity change over
// those steps fell below its tolerance (device reduction, one copy back for all members).
// Retiring frees the member's memory, which admits waiting requests before the next advance.
// Lattices below the solo size are members of one batch (one launch per step for all of them);
// larger ones, which fill the GPU on their own, step with the single-lattice kernels on their
// own streams, concurrently with the batch.
//
// The sequential mode serves the same requests one at a time, each stepped on its own
// (plain solves: the single-lattice kernels, no batch, no graphs), as the comparison.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <thread>
#include <vector>
#include "lattice.h"
#include "lbgpu.h"

using lbgpu::set_error;

namespace {

struct Req {
    lbgpu_request spec{};
    lbgpu_lattice *lat = nullptr;
    void *prev = nullptr;        // FP32 velocity at the last check
    int slot = -1;
    size_t bytes = 0;
    double admit = -1.0, finish = -1.0;
    long long steps = 0;
    int converged = 0;
    float change = -1.0f;
    bool active = false, done = false;
    bool solo = false;           // stepped on its own stream instead of in the batch
    std::vector<double> ux, uy;
};

// The velocity-change kernel reports a non-finite velocity as 3e38: such a request has
// diverged and retires at once.
constexpr float kDiverged = 1e30f;

double now_s(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

struct lbgpu_server {
    int precision = LBGPU_F32;
    int scheme[6] = {0, 0, 0, 0, 0, 0};      // per batch size class: LBGPU_PULL or LBGPU_AA
    int shape_w[6] = {0, 0, 0, 0, 0, 0};     // per size class: batch tile width, 0 = default
    int shape_n[6] = {1, 1, 1, 1, 1, 1};     // and nodes per thread
    int persistent = -1;                     // batch launch form, -1 = default
    int threads = 0;                         // batch threads per tile, 0 = default
    long long solo_nodes = 1LL << 20;        // requests of this many nodes or more step on their own
    size_t budget = 0;
    int check_every = 100;
    int scale_log2 = 10;
    bool shift = false;                      // 16-bit offsets from each request's inflow profile
    bool rs = false;                         // 16-bit stochastic rounding, seeded by request id
    std::vector<Req> reqs;
    unsigned *d_change = nullptr;
    int cap_change = 0;
    cudaStream_t stream = nullptr;
    double makespan = 0.0;
    long long lups = 0;
    int peak_active = 0;
    size_t peak_bytes = 0;
};

namespace {

int serr(cudaError_t e, const char *what) { return lbgpu::cuda_error(e, what); }

size_t request_bytes(const lbgpu_server *s, const lbgpu_request &r, int scheme)
{
    return lbgpu_lattice_bytes(r.lx, r.ly, s->precision, scheme) + 8 * (size_t)r.lx * r.ly;
}

int scheme_of(const lbgpu_server *s, const lbgpu_request &r)
{
    return s->scheme[lbgpu_batch_size_class((long long)r.lx * r.ly)];
}

// Allocate and set up a request's lattice and its velocity snapshot.
int start(lbgpu_server *s, Req &q, int id)
{
    const lbgpu_request &r = q.spec;
    const int sch = scheme_of(s, r);
    if (int rc = lbgpu_create(r.lx, r.ly, s->precision, sch, &q.lat)) return rc;
    if (s->precision == LBGPU_F16 || s->precision == LBGPU_BF16) {
        if (int rc = lbgpu_set_offset_scale(q.lat, s->scale_log2)) return rc;
        if (s->shift) {   // the channel's Poiseuille inflow profile, as lbgpu_setup_cylinder writes it
            std::vector<double> u(r.ly + 2, 0.0);
            const double L = r.ly - 1.0;
            for (int Y = 1; Y <= r.ly; ++Y) {
                const double y = Y - 1.0;
                u[Y] = 4.0 * r.umax / (L * L) * (L * y - y * y);
            }
            if (int rc = lbgpu_set_offset_shift(q.lat, u.data())) return rc;
        }
        if (s->rs)
            if (int rc = lbgpu_set_stochastic_rounding(q.lat, 1, (unsigned)id)) return rc;
    }
    if (int rc = lbgpu_setup_cylinder(q.lat, r.obst_x, r.obst_y, r.obst_r, r.umax, r.re,
                                      LBGPU_WALL_BOUNCEBACK, LBGPU_OUTLET_CONST, nullptr))
        return rc;
    if (int rc = serr(cudaMalloc(&q.prev, 8 * (size_t)r.lx * r.ly), "cudaMalloc(velocity snapshot)")) return rc;
    // the snapshot starts as the initial velocity (the first check compares against it)
    lbgpu::Lattice &L = q.lat->L;
    int v, par;
    L.view(v, par);
    lbgpu::launch_velocity_change(L.d, v, L.cur, par, q.prev, s->d_change, L.stream);
    if (int rc = serr(cudaStreamSynchronize(L.stream), "request set-up")) return rc;
    q.bytes = request_bytes(s, r, sch);
    q.active = true;
    return LB_OK;
}

void release(Req &q)
{
    if (q.prev) cudaFree(q.prev);
    q.prev = nullptr;
    if (q.lat) lbgpu_destroy(q.lat);
    q.lat = nullptr;
    q.active = false;
}

int ensure_change(lbgpu_server *s, int n)
{
    if (n <= s->cap_change) return LB_OK;
    if (s->d_change) cudaFree(s->d_change);
    s->cap_change = std::max(n, 2 * s->cap_change);
    void *p = nullptr;
    if (int rc = serr(cudaMalloc(&p, (size_t)s->cap_change * sizeof(unsigned)), "cudaMalloc(residuals)")) return rc;
    s->d_change = static_cast<unsigned *>(p);
    return LB_OK;
}

}  // namespace

extern "C" {

size_t lbgpu_lattice_bytes(int lx, int ly, int precision, int scheme)
{
    const int elem = precision == LBGPU_F64 ? 8 : (precision == LBGPU_F32 ? 4 : 2);
    const lbgpu::Geo g = lbgpu::make_geo(lx, ly, elem);
    const size_t nbuf = scheme == LBGPU_AA ? 1 : 2;
    const size_t nside = scheme == LBGPU_AA ? 2 : 3;
    size_t b = nbuf * 9 * (size_t)g.plane * elem + nside * 9 * (size_t)g.nper * elem + (size_t)g.plane +
               16 * (size_t)g.nb * 8 + 4 * (size_t)g.nb * 4 + 2 * (size_t)(ly + 2) * 8;
    if (scheme == LBGPU_AA) b += 9 * (size_t)g.nghost() * elem;
    return b;
}

int lbgpu_server_create(int precision, size_t budget_bytes, int check_every, lbgpu_server **out)
{
    if (!out || check_every < 1 || budget_bytes == 0)
        return set_error(LB_ERR_ARG, "lbgpu_server_create: bad arguments");
    *out = nullptr;
    if (precision < LBGPU_F64 || precision > LBGPU_BF16)
        return set_error(LB_ERR_ARG, "lbgpu_server_create: precision %d", precision);
    lbgpu_server *s = new lbgpu_server;
    s->precision = precision;
    s->budget = budget_bytes;
    s->check_every = check_every;
    if (int rc = serr(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "server stream")) {
        delete s;
        return rc;
    }
    *out = s;
    return LB_OK;
}

int lbgpu_server_destroy(lbgpu_server *s)
{
    if (!s) return LB_OK;
    for (Req &q : s->reqs) release(q);
    if (s->d_change) cudaFree(s->d_change);
    cudaStreamDestroy(s->stream);
    delete s;
    return LB_OK;
}

int lbgpu_server_set_scheme(lbgpu_server *s, int size_class, int scheme)
{
    if (!s || size_class < 0 || size_class >= 6 || (scheme != LBGPU_PULL && scheme != LBGPU_AA))
        return set_error(LB_ERR_ARG, "lbgpu_server_set_scheme: bad arguments");
    s->scheme[size_class] = scheme;
    return LB_OK;
}

int lbgpu_server_set_shape(lbgpu_server *s, int size_class, int tile_width, int nodes_per_thread)
{
    if (!s || size_class < 0 || size_class >= 6 || (tile_width != 32 && tile_width != 64 && tile_width != 128) ||
        (nodes_per_thread != 1 && nodes_per_thread != 4))
        return set_error(LB_ERR_ARG, "lbgpu_server_set_shape: bad arguments");
    s->shape_w[size_class] = tile_width;
    s->shape_n[size_class] = nodes_per_thread;
    return LB_OK;
}

int lbgpu_server_set_persistent(lbgpu_server *s, int persistent)
{
    if (!s) return set_error(LB_ERR_ARG, "lbgpu_server_set_persistent: null server");
    s->persistent = persistent ? 1 : 0;
    return LB_OK;
}

int lbgpu_server_set_threads(lbgpu_server *s, int threads)
{
    if (!s || (threads != 128 && threads != 256 && threads != 512))
        return set_error(LB_ERR_ARG, "lbgpu_server_set_threads: %d (128, 256, 512)", threads);
    s->threads = threads;
    return LB_OK;
}

int lbgpu_server_set_solo_nodes(lbgpu_server *s, long long nodes)
{
    if (!s || nodes < 0) return set_error(LB_ERR_ARG, "lbgpu_server_set_solo_nodes: bad arguments");
    s->solo_nodes = nodes;
    return LB_OK;
}

int lbgpu_server_set_offset_shift(lbgpu_server *s, int on)
{
    if (!s) return set_error(LB_ERR_ARG, "lbgpu_server_set_offset_shift: null server");
    if (on && s->precision != LBGPU_F16 && s->precision != LBGPU_BF16)
        return set_error(LB_ERR_STATE, "lbgpu_server_set_offset_shift: FP16/BF16 storage only");
    s->shift = on != 0;
    return LB_OK;
}

int lbgpu_server_set_stochastic_rounding(lbgpu_server *s, int on)
{
    if (!s) return set_error(LB_ERR_ARG, "lbgpu_server_set_stochastic_rounding: null server");
    if (on && s->precision != LBGPU_F16 && s->precision != LBGPU_BF16)
        return set_error(LB_ERR_STATE, "lbgpu_server_set_stochastic_rounding: FP16/BF16 storage only");
    s->rs = on != 0;
    return LB_OK;
}

int lbgpu_server_set_offset_scale(lbgpu_server *s, int scale_log2)
{
    if (!s || scale_log2 < -30 || scale_log2 > 30) return set_error(LB_ERR_ARG, "lbgpu_server_set_offset_scale");
    s->scale_log2 = scale_log2;
    return LB_OK;
}

int lbgpu_server_submit(lbgpu_server *s, const lbgpu_request *r, int *id)
{
    if (!s || !r) return set_error(LB_ERR_ARG, "lbgpu_server_submit: null argument");
    if (r->lx < 4 || r->ly < 4 || r->max_steps < 1 || r->max_steps % s->check_every)
        return set_error(LB_ERR_ARG, "lbgpu_server_submit: size %d x %d or step cap %d (a multiple of %d)",
                         r->lx, r->ly, r->max_steps, s->check_every);
    if (request_bytes(s, *r, scheme_of(s, *r)) > s->budget)
        return set_error(LB_ERR_CAPACITY, "lbgpu_server_submit: a %d x %d lattice exceeds the budget", r->lx, r->ly);
    Req q;
    q.spec = *r;
    s->reqs.push_back(q);
    if (id) *id = (int)s->reqs.size() - 1;
    return LB_OK;
}

int lbgpu_server_run(lbgpu_server *s, int batched)
{
    if (!s) return set_error(LB_ERR_ARG, "lbgpu_server_run: null server");
    const int n = (int)s->reqs.size();
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return s->reqs[a].spec.arrival < s->reqs[b].spec.arrival; });
    if (int rc = ensure_change(s, std::max(1, n))) return rc;
    lbgpu_batch *batch = nullptr;
    if (batched) {
        if (int rc = lbgpu_batch_create(s->precision, &batch)) return rc;
        for (int c = 0; c < 6; ++c)
            if (s->shape_w[c])
                if (int rc = lbgpu_batch_set_shape(batch, c, s->shape_w[c], s->shape_n[c])) {
                    lbgpu_batch_destroy(batch);
                    return rc;
                }
        if (s->persistent >= 0) lbgpu_batch_set_persistent(batch, s->persistent);
        if (s->threads) lbgpu_batch_set_threads(batch, s->threads);
    }
    std::vector<int> active;
    size_t used = 0;
    int qi = 0, rc = LB_OK;
    s->lups = 0;
    s->peak_active = 0;
    s->peak_bytes = 0;
    const auto t0 = std::chrono::steady_clock::now();
    while (rc == LB_OK && (qi < n || !active.empty())) {
        // admit in arrival order while memory allows (sequential: one request at a time)
        while (qi < n && s->reqs[order[qi]].spec.arrival <= now_s(t0)) {
            Req &q = s->reqs[order[qi]];
            const size_t need = request_bytes(s, q.spec, scheme_of(s, q.spec));
            if (used + need > s->budget || (!batched && !active.empty())) break;
            if ((rc = start(s, q, order[qi]))) break;
            q.admit = now_s(t0);
            used += need;
            q.solo = batched && (long long)q.spec.lx * q.spec.ly >= s->solo_nodes && s->solo_nodes > 0;
            if (batched && !q.solo && (rc = lbgpu_batch_add(batch, q.lat, &q.slot))) break;
            active.push_back(order[qi]);
            ++qi;
        }
        if (rc) break;
        s->peak_active = std::max(s->peak_active, (int)active.size());
        s->peak_bytes = std::max(s->peak_bytes, used);
        if (active.empty()) {   // idle until the next arrival
            const double wait = s->reqs[order[qi]].spec.arrival - now_s(t0);
            if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 0.001)));
            continue;
        }
        // advance every active request by check_every steps
        if (batched) {
            if ((rc = lbgpu_batch_step(batch, s->check_every))) break;
            for (int i : active)
                if (s->reqs[i].solo && (rc = lbgpu_step(s->reqs[i].lat, s->check_every))) break;
            if (rc) break;
        } else {
            if ((rc = lbgpu_step(s->reqs[active[0]].lat, s->check_every))) break;
        }
        if ((rc = serr(cudaMemsetAsync(s->d_change, 0, active.size() * sizeof(unsigned), s->stream), "clear residuals"))) break;
        if ((rc = serr(cudaStreamSynchronize(s->stream), "clear residuals"))) break;
        for (size_t k = 0; k < active.size(); ++k) {
            Req &q = s->reqs[active[k]];
            lbgpu::Lattice &L = q.lat->L;
            int v, par;
            L.view(v, par);
            lbgpu::launch_velocity_change(L.d, v, L.cur, par, q.prev, s->d_change + k, L.stream);
            q.steps += s->check_every;
            s->lups += (long long)s->check_every * q.spec.lx * q.spec.ly;
        }
        for (int i : active)
            if ((rc = serr(cudaStreamSynchronize(s->reqs[i].lat->L.stream), "residuals"))) break;
        if (rc) break;
        std::vector<float> change(active.size());
        if ((rc = serr(cudaMemcpy(change.data(), s->d_change, active.size() * sizeof(float), cudaMemcpyDeviceToHost),
                       "residuals")))
            break;
        std::vector<int> keep;
        for (size_t k = 0; k < active.size(); ++k) {
            Req &q = s->reqs[active[k]];
            q.change = change[k];
            const bool conv = q.spec.tol > 0.0 && change[k] < q.spec.tol;
            const bool diverged = !(change[k] < kDiverged);
            if (q.steps >= q.spec.max_steps || conv || diverged) {
                q.converged = diverged ? -1 : (conv ? 1 : 0);
                if (q.spec.want_fields) {
                    q.ux.resize((size_t)q.spec.lx * q.spec.ly);
                    q.uy.resize((size_t)q.spec.lx * q.spec.ly);
                    if ((rc = lbgpu_get_macros(q.lat, nullptr, q.ux.data(), q.uy.data()))) break;
                }
                if (batched && !q.solo && (rc = lbgpu_batch_remove(batch, q.slot))) break;
                q.finish = now_s(t0);
                used -= q.bytes;
                release(q);
                q.done = true;
            } else {
                keep.push_back(active[k]);
            }
        }
        active.swap(keep);
    }
    s->makespan = now_s(t0);
    if (batch) lbgpu_batch_destroy(batch);
    for (int i : active) release(s->reqs[i]);
    return rc;
}

int lbgpu_server_result(lbgpu_server *s, int id, lbgpu_result *out, double *ux, double *uy)
{
    if (!s || id < 0 || id >= (int)s->reqs.size() || !out) return set_error(LB_ERR_ARG, "lbgpu_server_result");
    const Req &q = s->reqs[id];
    out->arrival = q.spec.arrival;
    out->admit = q.admit;
    out->finish = q.finish;
    out->steps = q.steps;
    out->converged = q.converged;
    out->last_change = q.change;
    out->nodes = (long long)q.spec.lx * q.spec.ly;
    out->done = q.done ? 1 : 0;
    out->solo = q.solo ? 1 : 0;
    if (ux && !q.ux.empty()) std::memcpy(ux, q.ux.data(), q.ux.size() * sizeof(double));
    if (uy && !q.uy.empty()) std::memcpy(uy, q.uy.data(), q.uy.size() * sizeof(double));
    return LB_OK;
}

int lbgpu_server_stats(lbgpu_server *s, double out[4])
{
    if (!s || !out) return set_error(LB_ERR_ARG, "lbgpu_server_stats");
    out[0] = s->makespan;
    out[1] = (double)s->lups;
    out[2] = (double)s->peak_active;
    out[3] = (double)s->peak_bytes;
    return LB_OK;
}

}  // extern "C"
