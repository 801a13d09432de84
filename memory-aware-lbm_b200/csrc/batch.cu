// batch.cu -- many independent lattices advanced together (lbgpu_batch_* of include/lbgpu.h).
//
// Every step of every member runs in at most four launches, one per kind of step: the pull step
// of the two-buffer members (one node per thread, or for 16-bit storage optionally four nodes
// per thread), and the even and the odd AA step of the in-place members (AA members are kept in
// two lists by the parity of their phase, so each list runs one kind at a time).  A launch
// walks a work list of tiles (member, x0, y0, shape) of 128, 256 or 512 nodes, one per thread
// (or four per thread): either one block per tile, or a persistent grid of (blocks per SM x
// SMs) blocks strides through it.  Steps are grouped in chunks of 50 (an even count) captured
// once as a CUDA graph: the kernels read each member's buffers and parities from a device
// descriptor array, so the same graph replays chunk after chunk; it is re-captured when the
// membership or the launch form changes.
// A work item is a strip of tiles of one member stacked in y: its block reads the member's
// descriptor once and steps the tiles one after another down the lattice, so the descriptor's
// dependent loads are spread over the strip.  Tile widths and strip lengths are chosen per size
// class of member (node count), the threads per tile and the launch form per batch, by hand or by
// lbgpu_batch_autotune.
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
constexpr int kLists = 5;       // pull, pull four nodes a thread; AA of phase parity 0, 1 at rebuild;
                                // the perimeters of the four-nodes-a-thread members
constexpr int kQuad = 3;        // shape of the four-nodes-a-thread pull tiles (16-bit storage)
constexpr int kMaxPasses = 64;  // tiles a block may step down one member

int size_class(long long nodes)
{
    int c = 0;
    for (long long lim = 16384; c < kClasses - 1 && nodes >= lim; lim *= 4) ++c;
    return c;
}

// Tiles of width 32 << shape and threads / width rows; quad tiles 128 wide, threads / 32 rows.
int tile_w(int shape) { return shape == kQuad ? 128 : 32 << shape; }
int tile_h(int shape, int threads) { return shape == kQuad ? threads / 32 : threads / tile_w(shape); }

}  // namespace

struct lbgpu_batch {
    int precision = 0;
    cudaStream_t stream = nullptr;
    std::vector<lbgpu_lattice *> members;   // slot -> lattice (null: free slot)
    int shape[kClasses] = {2, 2, 2, 2, 2, 2};  // 0..2: 32 << shape wide; kQuad: 16-bit quad pull
    int passes[kClasses] = {4, 4, 4, 4, 4, 4}; // tiles a block steps down the lattice (4 measured
                                               // best on the 512-channel mix, FP32 and FP16)
    int threads = 128;                       // nodes per tile = threads per block
    bool persistent = false;
    BatchInst *d_inst = nullptr;
    int cap_inst = 0;
    BatchWork *d_work[kLists] = {};
    int cap_work[kLists] = {};
    int nwork[kLists] = {};
    int per_sm[lbgpu::BATCH_KINDS][3] = {};  // resident blocks per SM, [kind][threads 128/256/512]
    int sms = 0;
    int aa_phase = 0;                        // phase parity of list 2 now (list 3: the other)
    std::vector<BatchInst> h_inst;
    bool dirty = true;                       // descriptors or work lists must be rebuilt
    cudaEvent_t order = nullptr;             // orders the batch stream against members' streams
    cudaGraphExec_t graph[2] = {nullptr, nullptr};   // one chunk, by aa_phase
    int launches = 0;
    bool rs = false;                         // some member rounds stochastically (set at rebuild)
    bool shift = false;                      // some member stores row-shifted offsets (set at rebuild)
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
    b.rs = L.rs ? 1 : 0;
    b.rs_seed = L.rs_seed;
    return b;
}

// Stochastically rounded members key their collisions by number (tau0 + k), which a replayed
// chunk cannot advance: before each chunk after the first of a call the descriptors are
// uploaded again with tau0 moved on by the steps done (an even number: parities unchanged).
int refresh_collision_numbers(lbgpu_batch *b, int done)
{
    for (size_t i = 0; i < b->members.size(); ++i)
        if (b->members[i]) {
            b->h_inst[i] = describe(b->members[i]->L);
            b->h_inst[i].tau0 += done;
        }
    return batch_error(cudaMemcpyAsync(b->d_inst, b->h_inst.data(), b->h_inst.size() * sizeof(BatchInst),
                                       cudaMemcpyHostToDevice, b->stream), "update batch collision numbers");
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

int ensure_capacity(lbgpu_batch *b, int ninst, const int *need)
{
    if (ninst > b->cap_inst) {
        if (b->d_inst) cudaFree(b->d_inst);
        b->d_inst = nullptr;
        b->cap_inst = std::max(ninst, 2 * b->cap_inst);
        void *p = nullptr;
        if (int rc = batch_error(cudaMalloc(&p, (size_t)b->cap_inst * sizeof(BatchInst)), "cudaMalloc(batch members)")) return rc;
        b->d_inst = static_cast<BatchInst *>(p);
    }
    for (int s = 0; s < kLists; ++s)
        if (need[s] > b->cap_work[s]) {
            if (b->d_work[s]) cudaFree(b->d_work[s]);
            b->d_work[s] = nullptr;
            b->cap_work[s] = std::max(need[s], 2 * b->cap_work[s]);
            void *p = nullptr;
            if (int rc = batch_error(cudaMalloc(&p, (size_t)b->cap_work[s] * sizeof(BatchWork)), "cudaMalloc(batch tiles)")) return rc;
            b->d_work[s] = static_cast<BatchWork *>(p);
        }
    return LB_OK;
}

void drop_graphs(lbgpu_batch *b)
{
    for (cudaGraphExec_t &g : b->graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

// Rebuild descriptors and work lists from the members' current states.
int rebuild(lbgpu_batch *b)
{
    std::vector<BatchWork> work[kLists];
    b->h_inst.assign(b->members.size(), BatchInst{});
    for (size_t i = 0; i < b->members.size(); ++i) {
        lbgpu_lattice *m = b->members[i];
        if (!m) continue;
        const Lattice &L = m->L;
        b->h_inst[i] = describe(L);
        int sh = b->shape[size_class((long long)L.lx * L.ly)];
        if (sh == kQuad && L.scheme == LBGPU_AA) sh = 2;   // AA steps run one node per thread
        const int np = b->passes[size_class((long long)L.lx * L.ly)];
        const int tw = tile_w(sh), th = tile_h(sh, b->threads) * np;
        const int s = (L.scheme == LBGPU_AA) ? 2 + b->h_inst[i].phase0 : (sh == kQuad ? 1 : 0);
        for (int y0 = 1; y0 <= L.ly; y0 += th)
            for (int x0 = 1; x0 <= L.lx; x0 += tw)
                work[s].push_back(BatchWork{(int)i, x0, y0, lbgpu::batch_sp(sh, np)});
        if (s == 1)   // its perimeter, one block a run of `threads` perimeter nodes
            for (int p0 = 0; p0 < 2 * L.lx + 2 * L.ly; p0 += b->threads)
                work[4].push_back(BatchWork{(int)i, p0, 1, lbgpu::batch_sp(sh, 1)});
    }
    b->aa_phase = 0;
    b->rs = false;
    b->shift = false;
    for (const BatchInst &d : b->h_inst) {
        b->rs = b->rs || d.rs;
        b->shift = b->shift || d.g.shift_u != nullptr;
    }
    int need[kLists];
    for (int s = 0; s < kLists; ++s) need[s] = (int)work[s].size();
    if (int rc = ensure_capacity(b, (int)std::max<size_t>(b->h_inst.size(), 1), need)) return rc;
    for (int s = 0; s < kLists; ++s) {
        b->nwork[s] = need[s];
        if (need[s])
            if (int rc = batch_error(cudaMemcpyAsync(b->d_work[s], work[s].data(), work[s].size() * sizeof(BatchWork),
                                                     cudaMemcpyHostToDevice, b->stream), "upload batch tiles"))
                return rc;
    }
    if (!b->h_inst.empty())
        if (int rc = batch_error(cudaMemcpyAsync(b->d_inst, b->h_inst.data(), b->h_inst.size() * sizeof(BatchInst),
                                                 cudaMemcpyHostToDevice, b->stream), "upload batch members"))
            return rc;
    // the host arrays are read asynchronously: keep them alive until the copies finish
    if (int rc = batch_error(cudaStreamSynchronize(b->stream), "batch rebuild")) return rc;
    if (!b->sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
        for (int kind = 0; kind < lbgpu::BATCH_KINDS; ++kind)
            for (int t = 0; t < 3; ++t)
                b->per_sm[kind][t] = std::max(1, lbgpu::batch_blocks_per_sm(b->precision, kind, 128 << t));
    }
    drop_graphs(b);
    b->dirty = false;
    return LB_OK;
}

// k-th step of a chunk: one launch per non-empty work list.
void launch_step(lbgpu_batch *b, int k)
{
    for (int s = 0; s < kLists; ++s) {
        if (!b->nwork[s]) continue;
        int kind = s == 0 ? lbgpu::BATCH_PULL : (s == 1 ? lbgpu::BATCH_PULL4 : lbgpu::BATCH_PERIM);
        if (s == 2 || s == 3) {
            const int phase = (s == 2) ? b->aa_phase : 1 - b->aa_phase;
            kind = ((phase + k) & 1) ? lbgpu::BATCH_AA_ODD : lbgpu::BATCH_AA_EVEN;
        }
        const int t = b->threads == 512 ? 2 : (b->threads == 256 ? 1 : 0);
        const int grid = b->persistent ? std::min(b->per_sm[kind][t] * b->sms, b->nwork[s]) : b->nwork[s];
        lbgpu::launch_batch(b->precision, kind, b->threads, b->persistent, (b->rs ? 1 : 0) | (b->shift ? 2 : 0),
                            b->d_inst, b->d_work[s],
                            b->nwork[s], grid, k, b->stream);
        ++b->launches;
    }
}

int launches_per_step(const lbgpu_batch *b)
{
    int n = 0;
    for (int s = 0; s < kLists; ++s) n += b->nwork[s] ? 1 : 0;
    return n;
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
    e = cudaGraphInstantiate(&b->graph[b->aa_phase], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return batch_error(e, "graph instantiate");
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
    if (precision == LBGPU_F16 || precision == LBGPU_BF16)
        for (int c = 2; c < kClasses; ++c) b->shape[c] = kQuad;   // lattices of 64K nodes and more
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
    drop_graphs(b);
    if (b->d_inst) cudaFree(b->d_inst);
    for (int s = 0; s < kLists; ++s) if (b->d_work[s]) cudaFree(b->d_work[s]);
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

int lbgpu_batch_set_shape(lbgpu_batch *b, int size_class_, int tile_width, int nodes_per_thread)
{
    if (!b || size_class_ < 0 || size_class_ >= kClasses)
        return set_error(LB_ERR_ARG, "lbgpu_batch_set_shape: size class %d", size_class_);
    int ws = -1;
    for (int k = 0; k < 3; ++k) if ((32 << k) == tile_width) ws = k;
    const bool quad_ok = (b->precision == LBGPU_F16 || b->precision == LBGPU_BF16) && tile_width == 128;
    if (ws < 0 || (nodes_per_thread != 1 && !(nodes_per_thread == 4 && quad_ok)))
        return set_error(LB_ERR_ARG, "lbgpu_batch_set_shape: tile width %d (32, 64, 128), nodes per thread %d "
                         "(1; 4 with width 128 and 16-bit storage)", tile_width, nodes_per_thread);
    b->shape[size_class_] = nodes_per_thread == 4 ? kQuad : ws;
    b->dirty = true;
    return LB_OK;
}

int lbgpu_batch_get_shape(lbgpu_batch *b, int size_class_, int *tile_width, int *nodes_per_thread)
{
    if (!b || size_class_ < 0 || size_class_ >= kClasses)
        return set_error(LB_ERR_ARG, "lbgpu_batch_get_shape: size class %d", size_class_);
    if (tile_width) *tile_width = tile_w(b->shape[size_class_]);
    if (nodes_per_thread) *nodes_per_thread = b->shape[size_class_] == kQuad ? 4 : 1;
    return LB_OK;
}

int lbgpu_batch_set_passes(lbgpu_batch *b, int size_class_, int passes)
{
    if (!b || size_class_ < 0 || size_class_ >= kClasses || passes < 1 || passes > kMaxPasses)
        return set_error(LB_ERR_ARG, "lbgpu_batch_set_passes: size class %d, passes %d (1..%d)",
                         size_class_, passes, kMaxPasses);
    if (b->passes[size_class_] != passes) {
        b->passes[size_class_] = passes;
        b->dirty = true;
    }
    return LB_OK;
}

int lbgpu_batch_get_passes(lbgpu_batch *b, int size_class_)
{
    return (b && size_class_ >= 0 && size_class_ < kClasses) ? b->passes[size_class_] : 0;
}

int lbgpu_batch_set_persistent(lbgpu_batch *b, int persistent)
{
    if (!b) return set_error(LB_ERR_ARG, "lbgpu_batch_set_persistent: null batch");
    if (b->persistent != (persistent != 0)) {
        b->persistent = persistent != 0;
        drop_graphs(b);
    }
    return LB_OK;
}

int lbgpu_batch_get_persistent(lbgpu_batch *b) { return b && b->persistent ? 1 : 0; }

int lbgpu_batch_set_threads(lbgpu_batch *b, int threads)
{
    if (!b || (threads != 128 && threads != 256 && threads != 512))
        return set_error(LB_ERR_ARG, "lbgpu_batch_set_threads: %d threads per tile (128, 256, 512)", threads);
    if (b->threads != threads) {
        b->threads = threads;
        b->dirty = true;
    }
    return LB_OK;
}

int lbgpu_batch_get_threads(lbgpu_batch *b) { return b ? b->threads : 0; }

int lbgpu_batch_size_class(long long nodes) { return size_class(nodes); }

int lbgpu_batch_step(lbgpu_batch *b, int nsteps)
{
    if (!b || nsteps < 0) return set_error(LB_ERR_ARG, "lbgpu_batch_step: bad arguments");
    b->launches = 0;
    if (nsteps == 0 || lbgpu_batch_size(b) == 0) return LB_OK;
    bool any_rs = false;
    for (lbgpu_lattice *m : b->members)
        if (m && m->L.rs) any_rs = true;
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
    // rounding switched (or reseeded), or a row shift set or cleared, on a member since the
    // descriptors were written
    for (size_t i = 0; i < b->members.size() && !b->dirty; ++i)
        if (b->members[i] && (i >= b->h_inst.size() || b->h_inst[i].rs != (b->members[i]->L.rs ? 1 : 0) ||
                              b->h_inst[i].rs_seed != b->members[i]->L.rs_seed ||
                              b->h_inst[i].g.shift_u != b->members[i]->L.d.g.shift_u))
            b->dirty = true;
    if (b->dirty)
        if (int rc = rebuild(b)) return rc;
    if (int rc = order_before(b)) return rc;
    int done = 0;
    while (nsteps - done >= kChunk) {
        if (any_rs && done)
            if (int rc = refresh_collision_numbers(b, done)) return rc;
        if (!b->graph[b->aa_phase])
            if (int rc = capture_chunk(b)) return rc;
        if (int rc = batch_error(cudaGraphLaunch(b->graph[b->aa_phase], b->stream), "graph launch")) return rc;
        b->launches += kChunk * launches_per_step(b);
        done += kChunk;
    }
    const int rem = nsteps - done;
    if (any_rs && done && rem)
        if (int rc = refresh_collision_numbers(b, done)) return rc;
    for (int k = 0; k < rem; ++k) launch_step(b, k);
    if (int rc = lbgpu::cuda_error(cudaGetLastError(), "batch step")) return rc;
    for (lbgpu_lattice *m : b->members)
        if (m) advance(m->L, nsteps);
    if (int rc = order_after(b)) return rc;
    if ((rem & 1) || any_rs) {
        // parities changed (or stochastically rounded members count collisions): new
        // descriptors before the next call (a chunk's graph reads them); on odd remainders the
        // AA lists swap their kind of step
        if (rem & 1) b->aa_phase ^= 1;
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

// One candidate setting: an untimed batch step first (work-list rebuild, first-step path), so
// that the timed steps hold only the launches the setting makes.
static int time_setting(lbgpu_batch *b, int steps, float *ms)
{
    if (int rc = lbgpu_batch_step(b, 1)) return rc;
    return lbgpu_batch_step_timed(b, steps, ms);
}

// Threads per tile and launch form first (six combinations, shapes as set), then for every size
// class present the three tile widths (and for 16-bit storage the four-nodes-a-thread pull),
// each timed over `steps` batch steps after one untimed step; the fastest is kept at each
// stage.  The members really step (6 x (steps + 1), then 3 or 4 x (steps + 1) per class).
int lbgpu_batch_autotune(lbgpu_batch *b, int steps, float *best_ms_out)
{
    if (!b || steps < 1) return set_error(LB_ERR_ARG, "lbgpu_batch_autotune: bad arguments");
    bool present[kClasses] = {false};
    for (lbgpu_lattice *m : b->members)
        if (m) present[size_class((long long)m->L.lx * m->L.ly)] = true;
    {
        float best = 1e30f;
        int best_t = b->threads, best_p = b->persistent ? 1 : 0;
        for (int t = 128; t <= 512; t *= 2)
            for (int p = 0; p < 2; ++p) {
                lbgpu_batch_set_threads(b, t);
                lbgpu_batch_set_persistent(b, p);
                float ms = 0.f;
                if (int rc = time_setting(b, steps, &ms)) return rc;
                if (ms < best) { best = ms; best_t = t; best_p = p; }
            }
        lbgpu_batch_set_threads(b, best_t);
        lbgpu_batch_set_persistent(b, best_p);
    }
    for (int c = 0; c < kClasses; ++c) {
        if (best_ms_out) best_ms_out[c] = 0.f;
        if (!present[c]) continue;
        float best = 1e30f;
        int best_shape = b->shape[c];
        const int nshapes = (b->precision == LBGPU_F16 || b->precision == LBGPU_BF16) ? 4 : 3;
        for (int ws = 0; ws < nshapes; ++ws) {
            b->shape[c] = ws;
            b->dirty = true;
            float ms = 0.f;
            if (int rc = time_setting(b, steps, &ms)) return rc;
            if (ms < best) { best = ms; best_shape = ws; }
        }
        b->shape[c] = best_shape;
        b->dirty = true;
        // then the strip length: how many tiles of the class one block steps
        int best_np = b->passes[c];
        for (int np = 1; np <= 16; np *= 2) {
            if (np == best_np) continue;
            const int keep = b->passes[c];
            b->passes[c] = np;
            b->dirty = true;
            float ms = 0.f;
            if (int rc = time_setting(b, steps, &ms)) return rc;
            if (ms < best) { best = ms; best_np = np; }
            b->passes[c] = keep;
        }
        b->passes[c] = best_np;
        b->dirty = true;
        if (best_ms_out) best_ms_out[c] = best;
    }
    return LB_OK;
}

// Choose between the two-buffer pull scheme and the in-place AA scheme for lattices of one
// size as batch members: for each scheme, copies of a cylinder channel of that size (enough for
// about 8M nodes, at most 64) step together in a batch, and `steps` batch steps are timed.
int lbgpu_tune_scheme(int precision, int lx, int ly, int steps, int *scheme, float *ms_pull, float *ms_aa)
{
    if (lx < 4 || ly < 4 || steps < 1) return set_error(LB_ERR_ARG, "lbgpu_tune_scheme: bad arguments");
    const long long nodes = (long long)lx * ly;
    const int copies = (int)std::max(1LL, std::min(64LL, (8LL << 20) / nodes));
    float t[2] = {0.f, 0.f};
    for (int s = 0; s < 2; ++s) {
        std::vector<lbgpu_lattice *> lats;
        lbgpu_batch *b = nullptr;
        int rc = lbgpu_batch_create(precision, &b);
        for (int c = 0; c < copies && rc == LB_OK; ++c) {
            lbgpu_lattice *h = nullptr;
            rc = lbgpu_create(lx, ly, precision, s == 0 ? LBGPU_PULL : LBGPU_AA, &h);
            if (rc) break;
            lats.push_back(h);
            rc = lbgpu_setup_cylinder(h, lx / 5 + 1, ly / 2 + 1, ly / 10 + 1, 0.02, 100.0,
                                      LBGPU_WALL_BOUNCEBACK, LBGPU_OUTLET_CONST, nullptr);
            if (rc == LB_OK) rc = lbgpu_batch_add(b, h, nullptr);
        }
        if (rc == LB_OK) rc = lbgpu_batch_step(b, 2);
        if (rc == LB_OK) rc = lbgpu_batch_step_timed(b, steps, &t[s]);
        if (b) lbgpu_batch_destroy(b);
        for (lbgpu_lattice *h : lats) lbgpu_destroy(h);
        if (rc) return rc;
    }
    if (ms_pull) *ms_pull = t[0];
    if (ms_aa) *ms_aa = t[1];
    if (scheme) *scheme = (t[1] < t[0]) ? LBGPU_AA : LBGPU_PULL;
    return LB_OK;
}

}  // extern "C"
