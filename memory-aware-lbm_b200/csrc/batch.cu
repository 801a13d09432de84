// batch.cu -- many independent lattices advanced together (lbgpu_batch_* of include/lbgpu.h).
//
// Every step of every member runs in one persistent launch per scheme: a grid of
// (blocks per SM x SMs) blocks walks a work list of tiles (member, x0, y0, tile shape).  Steps
// are grouped in chunks of 50 (an even count) captured once as a CUDA graph: the kernels read
// each member's buffers and parities from a device descriptor array, so the same graph
// replays chunk after chunk; it is re-captured only when the membership changes.  Tile shapes
// are chosen per size class of member (node count), by hand or by lbgpu_batch_autotune.
#include <algorithm>
#include <cstring>
#include <vector>
#include "lattice.h"
#include "lbgpu.h"

using lbgpu::BatchInst;
using lbgpu::BatchWork;
using lbgpu::Lattice;
using lbgpu::set_error;

namespace {

constexpr int kClasses = 6;     // node-count classes: < 16K, 64K, 256K, 1M, 4M, above
constexpr int kChunk = 50;      // steps per captured graph (even: buffer parities repeat)

int size_class(long long nodes)
{
    int c = 0;
    for (long long lim = 16384; c < kClasses - 1 && nodes >= lim; lim *= 4) ++c;
    return c;
}

// Tiles of width 32 << (shape & 3) and (128 / width) << (shape >> 2) rows.
int tile_w(int shape) { return 32 << (shape & 3); }
int tile_h(int shape) { return (lbgpu::BATCH_THREADS / tile_w(shape)) << (shape >> 2); }

}  // namespace

struct lbgpu_batch {
    int precision = 0;
    cudaStream_t stream = nullptr;
    std::vector<lbgpu_lattice *> members;   // slot -> lattice (null: free slot)
    int shape[kClasses] = {2, 2, 2, 2, 2, 2};  // 128 wide, one row per thread
    BatchInst *d_inst = nullptr;
    int cap_inst = 0;
    BatchWork *d_work[2] = {nullptr, nullptr};
    int cap_work[2] = {0, 0};
    int *d_nwork = nullptr;                  // [2]
    int nwork[2] = {0, 0};
    int grid[2] = {0, 0};
    std::vector<BatchInst> h_inst;
    bool dirty = true;                       // descriptors or work lists must be rebuilt
    cudaEvent_t order = nullptr;             // orders the batch stream against members' streams
    cudaGraphExec_t graph = nullptr;
    int graph_grid[2] = {0, 0};               // values the captured graph has baked in
    BatchWork *graph_work[2] = {nullptr, nullptr};
    BatchInst *graph_inst = nullptr;
    bool graph_has[2] = {false, false};
    int launches = 0;
};

namespace {

int batch_error(cudaError_t e, const char *what) { return lbgpu::cuda_error(e, what); }

// Descriptor of a member from its lattice state (see kernels.h BatchInst).
BatchInst describe(const Lattice &L)
{
    BatchInst b;
    b.g = L.d.g;
    b.buf[0] = L.d.buf[0];
    b.buf[1] = L.d.buf[1];
    b.side = L.d.side;
    b.tag = L.d.tag;
    b.bc = L.d.bc;
    b.omega = L.d.omega;
    b.scale = L.d.scale;
    b.inv_scale = L.d.inv_scale;
    b.scheme = L.scheme;
    if (L.scheme == LBGPU_PULL) {
        b.cur0 = L.cur;
        b.phase0 = 0;
        b.tau0 = (int)(L.n + 1);
    } else {
        b.cur0 = 0;
        b.phase0 = (L.form == lbgpu::FORM_L) ? 0 : 1;
        b.tau0 = (int)((L.form == lbgpu::FORM_L) ? L.n : L.n + 1);
    }
    return b;
}

// A member's host-side state after `m` batch steps (no launches).
void advance(Lattice &L, int m)
{
    for (int s = 0; s < m; ++s) {
        if (L.scheme == LBGPU_PULL) {
            L.cur = 1 - L.cur;
            ++L.n;
        } else if (L.form == lbgpu::FORM_L) {
            L.form = lbgpu::FORM_C;
            L.pending = 1;
        } else {
            L.n += 2;
            L.form = lbgpu::FORM_L;
            L.pending = 0;
        }
    }
}

int ensure_capacity(lbgpu_batch *b, int ninst, int nw0, int nw1)
{
    if (ninst > b->cap_inst) {
        if (b->d_inst) cudaFree(b->d_inst);
        b->cap_inst = std::max(ninst, 2 * b->cap_inst);
        void *p = nullptr;
        if (int rc = batch_error(cudaMalloc(&p, (size_t)b->cap_inst * sizeof(BatchInst)), "cudaMalloc(batch members)")) return rc;
        b->d_inst = static_cast<BatchInst *>(p);
    }
    const int need[2] = {nw0, nw1};
    for (int s = 0; s < 2; ++s)
        if (need[s] > b->cap_work[s]) {
            if (b->d_work[s]) cudaFree(b->d_work[s]);
            b->cap_work[s] = std::max(need[s], 2 * b->cap_work[s]);
            void *p = nullptr;
            if (int rc = batch_error(cudaMalloc(&p, (size_t)b->cap_work[s] * sizeof(BatchWork)), "cudaMalloc(batch tiles)")) return rc;
            b->d_work[s] = static_cast<BatchWork *>(p);
        }
    if (!b->d_nwork) {
        void *p = nullptr;
        if (int rc = batch_error(cudaMalloc(&p, 2 * sizeof(int)), "cudaMalloc(batch counts)")) return rc;
        b->d_nwork = static_cast<int *>(p);
    }
    return LB_OK;
}

void drop_graph(lbgpu_batch *b)
{
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
}

// Rebuild descriptors and work lists from the members' current states.
int rebuild(lbgpu_batch *b)
{
    std::vector<BatchWork> work[2];
    b->h_inst.assign(b->members.size(), BatchInst{});
    for (size_t i = 0; i < b->members.size(); ++i) {
        lbgpu_lattice *m = b->members[i];
        if (!m) continue;
        const Lattice &L = m->L;
        b->h_inst[i] = describe(L);
        const int sh = b->shape[size_class((long long)L.lx * L.ly)];
        const int tw = tile_w(sh), th = tile_h(sh);
        const int s = (L.scheme == LBGPU_AA) ? 1 : 0;
        for (int y0 = 1; y0 <= L.ly; y0 += th)
            for (int x0 = 1; x0 <= L.lx; x0 += tw) work[s].push_back(BatchWork{(int)i, x0, y0, sh});
    }
    if (int rc = ensure_capacity(b, (int)std::max<size_t>(b->h_inst.size(), 1), (int)work[0].size(), (int)work[1].size())) return rc;
    for (int s = 0; s < 2; ++s) {
        b->nwork[s] = (int)work[s].size();
        if (b->nwork[s])
            if (int rc = batch_error(cudaMemcpyAsync(b->d_work[s], work[s].data(), work[s].size() * sizeof(BatchWork),
                                                     cudaMemcpyHostToDevice, b->stream), "upload batch tiles"))
                return rc;
    }
    if (!b->h_inst.empty())
        if (int rc = batch_error(cudaMemcpyAsync(b->d_inst, b->h_inst.data(), b->h_inst.size() * sizeof(BatchInst),
                                                 cudaMemcpyHostToDevice, b->stream), "upload batch members"))
            return rc;
    if (int rc = batch_error(cudaMemcpyAsync(b->d_nwork, b->nwork, 2 * sizeof(int), cudaMemcpyHostToDevice, b->stream),
                             "upload batch counts"))
        return rc;
    // the host arrays are read asynchronously: keep them alive until the copies finish
    if (int rc = batch_error(cudaStreamSynchronize(b->stream), "batch rebuild")) return rc;
    int sms = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    for (int s = 0; s < 2; ++s) {
        const int per_sm = std::max(1, lbgpu::batch_blocks_per_sm(b->precision, s == 1 ? LBGPU_AA : LBGPU_PULL));
        b->grid[s] = per_sm * sms;   // fixed: surplus blocks find no tile and exit
    }
    if (b->grid[0] != b->graph_grid[0] || b->grid[1] != b->graph_grid[1] ||
        b->d_work[0] != b->graph_work[0] || b->d_work[1] != b->graph_work[1] || b->d_inst != b->graph_inst ||
        (b->nwork[0] > 0) != b->graph_has[0] || (b->nwork[1] > 0) != b->graph_has[1])
        drop_graph(b);
    b->dirty = false;
    return LB_OK;
}

// k-th step of a chunk for both schemes.
void launch_step(lbgpu_batch *b, int k)
{
    for (int s = 0; s < 2; ++s)
        if (b->nwork[s]) {
            lbgpu::launch_batch(b->precision, s == 1 ? LBGPU_AA : LBGPU_PULL, b->d_inst, b->d_work[s],
                                b->d_nwork + s, b->grid[s], k, b->stream);
            ++b->launches;
        }
}

int capture_chunk(lbgpu_batch *b)
{
    cudaGraph_t g = nullptr;
    if (int rc = batch_error(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "begin capture")) return rc;
    const int before = b->launches;
    for (int k = 0; k < kChunk; ++k) launch_step(b, k);
    b->launches = before;
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (e != cudaSuccess) return batch_error(e, "end capture");
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return batch_error(e, "graph instantiate");
    for (int s = 0; s < 2; ++s) {
        b->graph_grid[s] = b->grid[s];
        b->graph_work[s] = b->d_work[s];
        b->graph_has[s] = b->nwork[s] > 0;
    }
    b->graph_inst = b->d_inst;
    return LB_OK;
}

// Members whose lattice holds an uncollided pull state get their first step on their own
// (the in-place collision), as do members with an extrapolated outlet (the batch kernel has
// no outlet pass).
bool needs_own_step(const Lattice &L)
{
    return L.zgb_each_step || (L.scheme == LBGPU_PULL && !(L.form == lbgpu::FORM_C && L.pending));
}

// The batch stream waits for work queued on the members' own streams, and they for the batch.
int order_before(lbgpu_batch *b)
{
    for (lbgpu_lattice *m : b->members) {
        if (!m) continue;
        if (int rc = batch_error(cudaEventRecord(b->order, m->L.stream), "order")) return rc;
        if (int rc = batch_error(cudaStreamWaitEvent(b->stream, b->order, 0), "order")) return rc;
    }
    return LB_OK;
}

int order_after(lbgpu_batch *b)
{
    if (int rc = batch_error(cudaEventRecord(b->order, b->stream), "order")) return rc;
    for (lbgpu_lattice *m : b->members)
        if (m)
            if (int rc = batch_error(cudaStreamWaitEvent(m->L.stream, b->order, 0), "order")) return rc;
    return LB_OK;
}

}  // namespace

extern "C" {

int lbgpu_batch_create(int precision, lbgpu_batch **out)
{
    if (!out) return set_error(LB_ERR_ARG, "lbgpu_batch_create: null output");
    *out = nullptr;
    if (precision < LBGPU_F64 || precision > LBGPU_BF16)
        return set_error(LB_ERR_ARG, "lbgpu_batch_create: precision %d", precision);
    lbgpu_batch *b = new lbgpu_batch;
    b->precision = precision;
    if (int rc = batch_error(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "batch stream")) {
        delete b;
        return rc;
    }
    if (int rc = batch_error(cudaEventCreateWithFlags(&b->order, cudaEventDisableTiming), "batch event")) {
        cudaStreamDestroy(b->stream);
        delete b;
        return rc;
    }
    *out = b;
    return LB_OK;
}

int lbgpu_batch_destroy(lbgpu_batch *b)
{
    if (!b) return LB_OK;
    cudaStreamSynchronize(b->stream);
    drop_graph(b);
    if (b->d_inst) cudaFree(b->d_inst);
    for (int s = 0; s < 2; ++s) if (b->d_work[s]) cudaFree(b->d_work[s]);
    if (b->d_nwork) cudaFree(b->d_nwork);
    cudaEventDestroy(b->order);
    cudaStreamDestroy(b->stream);
    delete b;
    return LB_OK;
}

int lbgpu_batch_add(lbgpu_batch *b, lbgpu_lattice *lat, int *slot)
{
    if (!b || !lat) return set_error(LB_ERR_ARG, "lbgpu_batch_add: null argument");
    if (lat->L.precision != b->precision)
        return set_error(LB_ERR_ARG, "lbgpu_batch_add: lattice precision %d, batch precision %d",
                         lat->L.precision, b->precision);
    if (lat->L.zgb_each_step)
        return set_error(LB_ERR_ARG, "lbgpu_batch_add: extrapolated outlets are stepped on their own, not in a batch");
    for (lbgpu_lattice *m : b->members)
        if (m == lat) return set_error(LB_ERR_ARG, "lbgpu_batch_add: lattice already in the batch");
    // the member's own stream may still be writing its initial state
    if (int rc = batch_error(cudaStreamSynchronize(lat->L.stream), "lbgpu_batch_add")) return rc;
    size_t k = 0;
    while (k < b->members.size() && b->members[k]) ++k;
    if (k == b->members.size()) b->members.push_back(lat);
    else b->members[k] = lat;
    if (slot) *slot = (int)k;
    b->dirty = true;
    return LB_OK;
}

int lbgpu_batch_remove(lbgpu_batch *b, int slot)
{
    if (!b || slot < 0 || slot >= (int)b->members.size() || !b->members[slot])
        return set_error(LB_ERR_ARG, "lbgpu_batch_remove: bad slot %d", slot);
    if (int rc = batch_error(cudaStreamSynchronize(b->stream), "lbgpu_batch_remove")) return rc;
    b->members[slot] = nullptr;
    while (!b->members.empty() && !b->members.back()) b->members.pop_back();
    b->dirty = true;
    return LB_OK;
}

int lbgpu_batch_size(lbgpu_batch *b)
{
    if (!b) return 0;
    int n = 0;
    for (lbgpu_lattice *m : b->members) n += m ? 1 : 0;
    return n;
}

int lbgpu_batch_set_shape(lbgpu_batch *b, int size_class_, int tile_width, int rows_per_thread)
{
    if (!b || size_class_ < 0 || size_class_ >= kClasses)
        return set_error(LB_ERR_ARG, "lbgpu_batch_set_shape: size class %d", size_class_);
    int ws = -1, rs = -1;
    for (int k = 0; k < 3; ++k) if ((32 << k) == tile_width) ws = k;
    for (int k = 0; k < 3; ++k) if ((1 << k) == rows_per_thread) rs = k;
    if (ws < 0 || rs < 0)
        return set_error(LB_ERR_ARG, "lbgpu_batch_set_shape: tile width %d (32, 64, 128), rows %d (1, 2, 4)",
                         tile_width, rows_per_thread);
    b->shape[size_class_] = ws | (rs << 2);
    b->dirty = true;
    return LB_OK;
}

int lbgpu_batch_get_shape(lbgpu_batch *b, int size_class_, int *tile_width, int *rows_per_thread)
{
    if (!b || size_class_ < 0 || size_class_ >= kClasses)
        return set_error(LB_ERR_ARG, "lbgpu_batch_get_shape: size class %d", size_class_);
    if (tile_width) *tile_width = tile_w(b->shape[size_class_]);
    if (rows_per_thread) *rows_per_thread = 1 << (b->shape[size_class_] >> 2);
    return LB_OK;
}

int lbgpu_batch_size_class(long long nodes) { return size_class(nodes); }

int lbgpu_batch_step(lbgpu_batch *b, int nsteps)
{
    if (!b || nsteps < 0) return set_error(LB_ERR_ARG, "lbgpu_batch_step: bad arguments");
    b->launches = 0;
    if (nsteps == 0 || lbgpu_batch_size(b) == 0) return LB_OK;
    // A member that needs its first step on its own (see needs_own_step) makes every member
    // take that step on its own path (the same per-node arithmetic as the batch kernel).
    bool own = false;
    for (lbgpu_lattice *m : b->members)
        if (m && needs_own_step(m->L)) own = true;
    if (own) {
        for (lbgpu_lattice *m : b->members) {
            if (!m) continue;
            if (int rc = m->L.step(1)) return rc;
            b->launches += m->L.launches;
        }
        for (lbgpu_lattice *m : b->members)
            if (m)
                if (int rc = batch_error(cudaStreamSynchronize(m->L.stream), "member step")) return rc;
        --nsteps;
        b->dirty = true;
    }
    if (b->dirty)
        if (int rc = rebuild(b)) return rc;
    if (int rc = order_before(b)) return rc;
    int done = 0;
    while (nsteps - done >= kChunk) {
        if (!b->graph)
            if (int rc = capture_chunk(b)) return rc;
        if (int rc = batch_error(cudaGraphLaunch(b->graph, b->stream), "graph launch")) return rc;
        b->launches += kChunk * ((b->nwork[0] ? 1 : 0) + (b->nwork[1] ? 1 : 0));
        done += kChunk;
    }
    const int rem = nsteps - done;
    for (int k = 0; k < rem; ++k) launch_step(b, k);
    if (int rc = lbgpu::cuda_error(cudaGetLastError(), "batch step")) return rc;
    for (lbgpu_lattice *m : b->members)
        if (m) advance(m->L, nsteps);
    if (int rc = order_after(b)) return rc;
    if (rem & 1) {
        // parities changed: new descriptors before the next call (a chunk's graph reads them)
        for (size_t i = 0; i < b->members.size(); ++i)
            if (b->members[i]) b->h_inst[i] = describe(b->members[i]->L);
        if (int rc = batch_error(cudaMemcpyAsync(b->d_inst, b->h_inst.data(), b->h_inst.size() * sizeof(BatchInst),
                                                 cudaMemcpyHostToDevice, b->stream), "update batch members"))
            return rc;
        if (int rc = batch_error(cudaStreamSynchronize(b->stream), "update batch members")) return rc;
    }
    return LB_OK;
}

int lbgpu_batch_step_timed(lbgpu_batch *b, int nsteps, float *ms)
{
    if (!b) return set_error(LB_ERR_ARG, "lbgpu_batch_step_timed: null batch");
    cudaEvent_t e0, e1;
    if (int rc = batch_error(cudaEventCreate(&e0), "cudaEventCreate")) return rc;
    if (int rc = batch_error(cudaEventCreate(&e1), "cudaEventCreate")) { cudaEventDestroy(e0); return rc; }
    int rc = batch_error(cudaEventRecord(e0, b->stream), "cudaEventRecord");
    if (rc == LB_OK) rc = lbgpu_batch_step(b, nsteps);
    if (rc == LB_OK) rc = batch_error(cudaEventRecord(e1, b->stream), "cudaEventRecord");
    if (rc == LB_OK) rc = batch_error(cudaEventSynchronize(e1), "cudaEventSynchronize");
    float t = 0.f;
    if (rc == LB_OK) rc = batch_error(cudaEventElapsedTime(&t, e0, e1), "cudaEventElapsedTime");
    if (ms) *ms = t;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

int lbgpu_batch_synchronize(lbgpu_batch *b)
{
    if (!b) return set_error(LB_ERR_ARG, "lbgpu_batch_synchronize: null batch");
    return batch_error(cudaStreamSynchronize(b->stream), "lbgpu_batch_synchronize");
}

int lbgpu_batch_last_launches(lbgpu_batch *b) { return b ? b->launches : 0; }

// For every size class present, time `steps` batch steps with each tile shape and keep the
// fastest.  The members really step (3 x 3 shapes x `steps` steps per class).
int lbgpu_batch_autotune(lbgpu_batch *b, int steps, float *best_ms_out)
{
    if (!b || steps < 1) return set_error(LB_ERR_ARG, "lbgpu_batch_autotune: bad arguments");
    bool present[kClasses] = {false};
    for (lbgpu_lattice *m : b->members)
        if (m) present[size_class((long long)m->L.lx * m->L.ly)] = true;
    for (int c = 0; c < kClasses; ++c) {
        if (!present[c]) continue;
        float best = 1e30f;
        int best_shape = b->shape[c];
        for (int ws = 0; ws < 3; ++ws)
            for (int rs = 0; rs < 3; ++rs) {
                b->shape[c] = ws | (rs << 2);
                b->dirty = true;
                float ms = 0.f;
                if (int rc = lbgpu_batch_step_timed(b, steps, &ms)) return rc;
                if (ms < best) { best = ms; best_shape = b->shape[c]; }
            }
        b->shape[c] = best_shape;
        b->dirty = true;
        if (best_ms_out) best_ms_out[c] = best;
    }
    return LB_OK;
}

// Choose between the two-buffer pull scheme and the in-place AA scheme for lattices of one
// size: time `steps` steps of a cylinder channel of that size in each scheme on their own.
int lbgpu_tune_scheme(int precision, int lx, int ly, int steps, int *scheme, float *ms_pull, float *ms_aa)
{
    float t[2] = {0.f, 0.f};
    for (int s = 0; s < 2; ++s) {
        lbgpu_lattice *h = nullptr;
        if (int rc = lbgpu_create(lx, ly, precision, s == 0 ? LBGPU_PULL : LBGPU_AA, &h)) return rc;
        int rc = lbgpu_setup_cylinder(h, lx / 5 + 1, ly / 2 + 1, ly / 10 + 1, 0.02, 100.0,
                                      LBGPU_WALL_BOUNCEBACK, LBGPU_OUTLET_CONST, nullptr);
        if (rc == LB_OK) rc = lbgpu_step(h, 2);
        if (rc == LB_OK) rc = lbgpu_step_timed(h, steps, &t[s]);
        lbgpu_destroy(h);
        if (rc) return rc;
    }
    if (ms_pull) *ms_pull = t[0];
    if (ms_aa) *ms_aa = t[1];
    if (scheme) *scheme = (t[1] < t[0]) ? LBGPU_AA : LBGPU_PULL;
    return LB_OK;
}

}  // extern "C"
