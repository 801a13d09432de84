// dropin.cu -- the lb.h / boundaries.h entry points on the GPU (drop-in for the reference's
// lb.c collide/propagate functions).
//
// The host Simulation keeps the reference's two node arrays; the library adds a device
// lattice (exact FP64, pull kernel, ghost ring kept) created at the first step call.
//   * Dynamics -> tags: the function address of every node's Dynamics picks the rule
//     (bgk, bounceBack, 16 boundary rules); boundary data come from the per-side tables,
//     slot (side, coordinate), re-read from the driver's VelocityBCData/PressureBCData at
//     every entry because drivers change them between steps (unsteady.c:211-212).
//   * entry points map onto the lattice's state machine (lattice.cu): collide collides,
//     propagate / finalize_stream mark the stream (performed by the next collision's pull
//     kernel or by a read-out), the two-step functions run two steps with the second step's
//     outlet densities extrapolated on the device (lb.c:471-480, :527-531).
//   * after each entry point the sync mode decides what is copied back to the host arrays.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#include "d2q9.cuh"
#include "lattice.h"
#include "lb.h"
#include "boundaries.h"
#include "lbgpu.h"

using lbgpu::Lattice;
using lbgpu::set_error;

// Globals the reference's lattice code reads from its driver (reference lb.c:30-38).  A
// driver that defines them (the application driver does, unsteady.c:41-54) takes
// precedence at dynamic-link time; these definitions let drivers that do not use them link.
extern "C" {
PressureBCData *pressureBoundary = nullptr;
int blk_size = 1;
double *myrho1 = nullptr, *myrho2 = nullptr;
int iT = 0, count = 0;
int thread_block = 1;
int NUM_THREADS = 1;
long long global_CM[NUM_EVENTS] = {0, 0, 0, 0};
}

namespace {

typedef void (*DynFun)(double *, void *);

struct DropIn {
    Lattice L;
    bool created = false;
    bool uploaded = false;
    bool tags_dirty = true;
    bool pops_dirty = false;
    bool dynp_dirty = true;
    bool bc_force = true;       // upload tables at the next refresh even if unchanged
    bool tmp_is_stream = false; // tmpLattice holds the stream of lattice (collide_with_stream)
    int sync_mode = LB_SYNC_OUTLET;
    bool pinned[3] = {false, false, false};         // host arrays, then the dynamics pointers
    void *pinned_ptr[3] = {nullptr, nullptr, nullptr};
    std::vector<uint64_t> dynp;          // host Dynamics* of every node, [X*(ly+2)+Y]
    uint64_t *dynp_dev = nullptr;
    std::vector<const void *> slot_src;  // [8*nb] boundary data object of each table slot
    std::vector<int> active_slots;
    // per active slot: the two values' addresses in the driver's data object and their table
    // offsets (set at each rescan, so a refresh does no index arithmetic)
    struct SlotRead { const double *src[2]; size_t off[2]; };
    std::vector<SlotRead> slot_reads;
    std::vector<const double *> omegas;  // distinct omega pointers of bgk / bulk dynamics
    std::vector<double> bc_new;
    const PressureBCData *zgb_base = nullptr;
    int zgb_base_ly = -1;
};

DropIn *ctx_of(Simulation *sim) { return sim ? static_cast<DropIn *>(sim->device) : nullptr; }

// Function address -> tag, in the LBGPU_TAG_* order.
const DynFun kRules[LBGPU_NUM_TAGS] = {
    nullptr, &bgk, &bounceBack,
    &upperZouHe, &lowerZouHe, &leftZouHe, &rightZouHe,
    &upperPressureZouHe, &lowerPressureZouHe, &leftPressureZouHe, &rightPressureZouHe,
    &upperRegularized, &lowerRegularized, &leftRegularized, &rightRegularized,
    &upperPressureRegularized, &lowerPressureRegularized, &leftPressureRegularized,
    &rightPressureRegularized};

int rule_tag(DynFun f)
{
    for (int t = 1; t < LBGPU_NUM_TAGS; ++t)
        if (kRules[t] == f) return t;
    return -1;
}

Node *chunk_of(Node **cols) { return cols ? cols[0] : nullptr; }

void add_omega(DropIn *c, const double *p)
{
    if (std::find(c->omegas.begin(), c->omegas.end(), p) == c->omegas.end()) c->omegas.push_back(p);
}

// Read every node's Dynamics into the tag plane and the table-slot map.
int scan_dynamics(Simulation *sim, DropIn *c)
{
    Lattice &L = c->L;
    const int lx = sim->lx, ly = sim->ly, nb = L.d.g.nb;
    // tags in the host's own node order (sequential reads and writes; the device transposes)
    std::vector<uint8_t> txy((size_t)(lx + 2) * (ly + 2), 0);
    c->slot_src.assign(8 * (size_t)nb, nullptr);
    c->active_slots.clear();
    c->omegas.clear();
    const Dynamics *last = nullptr;
    int last_tag = 0;
    for (int X = 1; X <= lx; ++X) {
        const uint64_t *col = c->dynp.data() + (size_t)X * (ly + 2);
        uint8_t *tcol = txy.data() + (size_t)X * (ly + 2);
        for (int Y = 1; Y <= ly; ++Y) {
            const Dynamics *dyn = reinterpret_cast<const Dynamics *>(col[Y]);
            if (!dyn)
                return set_error(LB_ERR_DYNAMICS, "node (%d,%d) has no dynamics (setDynamics was not called)", X, Y);
            if (dyn != last) {
                const int t = rule_tag(dyn->dynamicsFun);
                if (t < 0)
                    return set_error(LB_ERR_DYNAMICS,
                                     "node (%d,%d): dynamics function %p is not one of the library's rules",
                                     X, Y, (void *)dyn->dynamicsFun);
                if (t == LBGPU_TAG_BGK) {
                    if (!dyn->selfData)
                        return set_error(LB_ERR_DYNAMICS, "node (%d,%d): bgk without omega", X, Y);
                    add_omega(c, static_cast<const double *>(dyn->selfData));
                } else if (t >= LBGPU_TAG_UPPER_ZOUHE) {
                    const VelocityBCData *vd = static_cast<const VelocityBCData *>(dyn->selfData);
                    if (!vd || !vd->bulkDynamics || vd->bulkDynamics->dynamicsFun != &bgk ||
                        !vd->bulkDynamics->selfData)
                        return set_error(LB_ERR_DYNAMICS,
                                         "node (%d,%d): boundary data must chain to a bgk bulk dynamics", X, Y);
                    add_omega(c, static_cast<const double *>(vd->bulkDynamics->selfData));
                }
                last = dyn;
                last_tag = t;
            }
            tcol[Y] = (uint8_t)last_tag;
            if (last_tag >= LBGPU_TAG_UPPER_ZOUHE) {
                const int tb = lbgpu::tag_table(last_tag);
                const int coord = (lbgpu::tag_side(last_tag) <= lbgpu::SIDE_LOWER) ? X : Y;
                const size_t k = (size_t)tb * nb + coord;
                if (!c->slot_src[k]) {
                    c->slot_src[k] = dyn->selfData;
                    c->active_slots.push_back((int)k);
                } else if (c->slot_src[k] != dyn->selfData) {
                    return set_error(LB_ERR_LAYOUT,
                                     "node (%d,%d): two %s boundary nodes on the same %s use different data objects",
                                     X, Y, lbgpu::tag_pressure(last_tag) ? "pressure" : "velocity",
                                     coord == X ? "column" : "row");
                }
            }
        }
    }
    c->slot_reads.clear();
    for (int k : c->active_slots) {
        const int tb = k / nb, coord = k % nb;
        DropIn::SlotRead r;
        if (tb < 4) {
            const VelocityBCData *vd = static_cast<const VelocityBCData *>(c->slot_src[k]);
            r.src[0] = &vd->ux; r.src[1] = &vd->uy;
        } else {
            const PressureBCData *pd = static_cast<const PressureBCData *>(c->slot_src[k]);
            r.src[0] = &pd->rho; r.src[1] = &pd->uPar;
        }
        r.off[0] = (size_t)(tb * 2 + 0) * nb + coord;
        r.off[1] = (size_t)(tb * 2 + 1) * nb + coord;
        c->slot_reads.push_back(r);
    }
    c->bc_force = true;
    c->zgb_base = nullptr;
    c->zgb_base_ly = -1;
    return L.upload_tags_xy(txy.data());
}

// Re-read boundary data and omega from the driver's objects; upload what changed.
int refresh_params(DropIn *c)
{
    Lattice &L = c->L;
    if (c->omegas.empty()) {
        L.d.omega = 1.0;
    } else {
        const double w = *c->omegas[0];
        for (size_t k = 1; k < c->omegas.size(); ++k)
            if (*c->omegas[k] != w)
                return set_error(LB_ERR_DYNAMICS, "bgk dynamics with different omega values (%g, %g)",
                                 w, *c->omegas[k]);
        L.d.omega = w;
    }
    // bc_new mirrors the last uploaded tables; each active slot is compared with the driver's
    // object (bitwise, as a memcmp would) and the tables go up only when one changed or a pass
    // forced it (a rescan, or device-side writes of the two-step outlet)
    if (c->bc_new.size() != L.bc_host.size()) c->bc_new = L.bc_host;
    bool changed = c->bc_force;
    double *bcn = c->bc_new.data();
    for (const DropIn::SlotRead &r : c->slot_reads)
        for (int j = 0; j < 2; ++j) {
            const double v = *r.src[j];
            if (std::memcmp(&bcn[r.off[j]], &v, sizeof(double)) != 0) {
                bcn[r.off[j]] = v;
                changed = true;
            }
        }
    if (changed) {
        if (int rc = L.upload_bc(c->bc_new.data())) return rc;
        c->bc_force = false;
    }
    return LB_OK;
}

int upload_dynp(DropIn *c)
{
    if (!c->dynp_dirty) return LB_OK;
    const size_t bytes = c->dynp.size() * sizeof(uint64_t);
    if (!c->dynp_dev) {
        void *p = nullptr;
        if (int rc = lbgpu::cuda_error(cudaMalloc(&p, bytes), "cudaMalloc(dynamics pointers)")) return rc;
        c->dynp_dev = static_cast<uint64_t *>(p);
    }
    if (int rc = lbgpu::cuda_error(cudaMemcpyAsync(c->dynp_dev, c->dynp.data(), bytes,
                                                   cudaMemcpyHostToDevice, c->L.stream), "upload dynamics pointers"))
        return rc;
    c->L.h2d_bytes += bytes;
    if (int rc = lbgpu::cuda_error(cudaStreamSynchronize(c->L.stream), "upload dynamics pointers")) return rc;
    c->dynp_dirty = false;
    return LB_OK;
}

void pin_host(Simulation *sim, DropIn *c)
{
    const char *e = getenv("LBGPU_PIN");
    if (e && e[0] == '0') return;
    const size_t nodes = (size_t)(sim->lx + 2) * (sim->ly + 2);
    // the dynamics pointers too: the first read-out uploads them (the vector never reallocates)
    void *chunks[3] = {sim->memoryChunk, sim->tmpMemoryChunk, c->dynp.data()};
    const size_t bytes[3] = {nodes * sizeof(Node), nodes * sizeof(Node), c->dynp.size() * sizeof(uint64_t)};
    for (int k = 0; k < 3; ++k) {
        if (c->pinned[k] || !chunks[k] || !bytes[k]) continue;
        if (cudaHostRegister(chunks[k], bytes[k], cudaHostRegisterPortable) == cudaSuccess) {
            c->pinned[k] = true;
            c->pinned_ptr[k] = chunks[k];
        } else {
            cudaGetLastError();  // pageable transfers still work
        }
    }
}

// Create the device lattice and pin the host arrays (once).
int create_device(Simulation *sim, DropIn *c)
{
    if (c->created) return LB_OK;
    Lattice &L = c->L;
    if (int rc = L.create(sim->lx, sim->ly, LBGPU_F64, LBGPU_PULL)) {
        L.destroy();
        return rc;
    }
    L.ghosts = true;
    c->created = true;
    pin_host(sim, c);
    return LB_OK;
}

// Bring the device copy up to date before an entry point runs (`tables`: the entry collides,
// so omega and the boundary data objects are re-read; a pure stream never reads them).
DropIn *prepare(Simulation *sim, const char *fn, bool tables = true)
{
    DropIn *c = ctx_of(sim);
    if (!c) {
        set_error(LB_ERR_STATE, "%s: the simulation was not created by constructSim", fn);
        return nullptr;
    }
    Lattice &L = c->L;
    if (!c->created && create_device(sim, c) != LB_OK) return nullptr;
    // The population uploads go first: they are asynchronous copies from the pinned host
    // arrays, so the host's scan of the dynamics pointers below runs while they transfer.
    if (!c->uploaded) {
        L.launches = 0;
        if (L.upload_records(0, reinterpret_cast<const double *>(chunk_of(sim->lattice)), 10, 0, sim->lx + 2) ||
            L.upload_records_edges(1, reinterpret_cast<const double *>(chunk_of(sim->tmpLattice)), 10) ||
            L.init_side_from(1, 1))
            return nullptr;
        L.cur = 0; L.form = lbgpu::FORM_L; L.pending = 0; L.n = 0;
        c->uploaded = true;
        c->pops_dirty = false;
    } else if (c->pops_dirty) {
        // the host lattice is the current state: put it where that state lives
        const double *src = reinterpret_cast<const double *>(chunk_of(sim->lattice));
        if (L.form == lbgpu::FORM_C && L.pending) {
            if (L.upload_records(1 - L.cur, src, 10, 0, sim->lx + 2)) return nullptr;
            L.cur = 1 - L.cur; ++L.n; L.form = lbgpu::FORM_L; L.pending = 0;
        } else {
            if (L.upload_records(L.cur, src, 10, 0, sim->lx + 2)) return nullptr;
        }
        c->pops_dirty = false;
    }
    if (c->tags_dirty) {
        if (scan_dynamics(sim, c) != LB_OK) return nullptr;
        c->tags_dirty = false;
    }
    if (tables && refresh_params(c) != LB_OK) return nullptr;
    return c;
}

// Copy back what the sync mode asks for.
void finish(Simulation *sim, DropIn *c)
{
    Lattice &L = c->L;
    if (c->sync_mode == LB_SYNC_NONE) return;
    if (upload_dynp(c) != LB_OK) return;
    Node *host = chunk_of(sim->lattice);
    const size_t col = (size_t)(sim->ly + 2);
    if (c->sync_mode == LB_SYNC_FULL) {
        L.readout_records(reinterpret_cast<double *>(host), 10, c->dynp_dev, 0, sim->lx + 2);
        return;
    }
    // columns lx-2 and lx-1 are adjacent in the host's y-contiguous node array: one read-out
    const int X0 = sim->lx >= 2 ? sim->lx - 2 : 0;
    L.readout_records(reinterpret_cast<double *>(host + (size_t)X0 * col), 10, c->dynp_dev, X0, sim->lx);
}

void swap_host(Simulation *sim)
{
    Node **t = sim->lattice;
    sim->lattice = sim->tmpLattice;
    sim->tmpLattice = t;
}

// Pressure-table slots whose data object is an element 2..ly-1 of the driver's
// pressureBoundary array: the two-step entry points overwrite those elements with the
// extrapolated density before their second step (lb.c:527-531).
int refresh_zgb_slots(Simulation *sim, DropIn *c)
{
    if (c->zgb_base == pressureBoundary && c->zgb_base_ly == sim->ly) return LB_OK;
    Lattice &L = c->L;
    const int nb = L.d.g.nb, ly = sim->ly;
    std::vector<int> src(4 * (size_t)nb, -1);
    if (pressureBoundary) {
        const char *lo = reinterpret_cast<const char *>(&pressureBoundary[2]);
        const char *hi = reinterpret_cast<const char *>(&pressureBoundary[ly - 1]);
        for (int k : c->active_slots) {
            const int tb = k / nb;
            if (tb < 4) continue;
            const char *p = static_cast<const char *>(c->slot_src[k]);
            if (p >= lo && p <= hi && (p - lo) % (long)sizeof(PressureBCData) == 0) {
                const int row = 2 + (int)((p - lo) / (long)sizeof(PressureBCData));
                src[(size_t)(tb - 4) * nb + (k % nb)] = row;
            }
        }
    }
    if (int rc = L.upload_zgb_src(src.data())) return rc;
    c->zgb_base = pressureBoundary;
    c->zgb_base_ly = ly;
    return LB_OK;
}

bool blocks_ok(Simulation *sim, int need_x, int need_y, const char *fn)
{
    if (blk_size < 1 || (need_x && sim->lx % blk_size) || (need_y && sim->ly % blk_size)) {
        set_error(LB_ERR_BLOCK_SIZE, "%s: blk_size %d does not divide the lattice (%d x %d)", fn,
                  blk_size, sim->lx, sim->ly);
        return false;
    }
    return true;
}

// Two steps per call; the second step's outlet density is extrapolated on the device from the
// populations entering that step, and the driver's globals get what the reference leaves there.
void two_steps(Simulation *sim, const char *fn, int need_x, int need_y)
{
    if ((need_x || need_y) && !blocks_ok(sim, need_x, need_y, fn)) return;
    DropIn *c = prepare(sim, fn);
    if (!c) return;
    Lattice &L = c->L;
    L.launches = 0;
    c->tmp_is_stream = false;
    if (L.op_collide() || L.op_propagate()) return;
    if (refresh_zgb_slots(sim, c)) return;
    if (sim->lx >= 2) {
        if (L.zgb_pass()) return;
    }
    if (L.op_collide() || L.op_propagate()) return;
    c->bc_force = true;  // the tables now hold the extrapolated densities
    if (sim->lx >= 2 && (pressureBoundary || myrho1 || myrho2)) {
        std::vector<double> zr(2 * (size_t)(sim->ly + 2));
        if (lbgpu::cuda_error(cudaMemcpyAsync(zr.data(), L.d.zrho, zr.size() * 8, cudaMemcpyDeviceToHost,
                                              L.stream), fn) ||
            lbgpu::cuda_error(cudaStreamSynchronize(L.stream), fn))
            return;
        L.d2h_bytes += zr.size() * 8;
        for (int k = 1; k <= sim->ly - 1; ++k) {
            if (myrho1) myrho1[k] = zr[2 * k];
            if (myrho2 && sim->lx >= 3) myrho2[k] = zr[2 * k + 1];
        }
        if (pressureBoundary)
            for (int Y = 2; Y <= sim->ly - 1; ++Y) {
                pressureBoundary[Y].rho = 4. / 3. * zr[2 * Y] - 1. / 3. * zr[2 * Y + 1];
                pressureBoundary[Y].uPar = 0.;
            }
    }
    finish(sim, c);
}

}  // namespace

extern "C" {

// ---- construction ---------------------------------------------------------------------
void constructSim(Simulation *sim, int lx, int ly)
{
    if (!sim) { set_error(LB_ERR_ARG, "constructSim: null simulation"); return; }
    std::memset(sim, 0, sizeof *sim);
    if (lx < 1 || ly < 1 || lx > LBGPU_MAX_LX || ly > LBGPU_MAX_LY) {
        set_error(LB_ERR_ARG, "constructSim: size %d x %d out of range (1..%d x 1..%d)", lx, ly,
                  LBGPU_MAX_LX, LBGPU_MAX_LY);
        return;
    }
    const size_t nodes = (size_t)(lx + 2) * (ly + 2);
    sim->lx = lx;
    sim->ly = ly;
    sim->memoryChunk = static_cast<Node *>(calloc(nodes, sizeof(Node)));
    sim->tmpMemoryChunk = static_cast<Node *>(calloc(nodes, sizeof(Node)));
    sim->lattice = static_cast<Node **>(calloc(lx + 2, sizeof(Node *)));
    sim->tmpLattice = static_cast<Node **>(calloc(lx + 2, sizeof(Node *)));
    if (!sim->memoryChunk || !sim->tmpMemoryChunk || !sim->lattice || !sim->tmpLattice) {
        set_error(LB_ERR_ALLOC, "constructSim: host allocation of %zu nodes failed", nodes);
        free(sim->memoryChunk); free(sim->tmpMemoryChunk); free(sim->lattice); free(sim->tmpLattice);
        std::memset(sim, 0, sizeof *sim);
        return;
    }
    for (int X = 0; X < lx + 2; ++X) {
        sim->lattice[X] = sim->memoryChunk + (size_t)X * (ly + 2);
        sim->tmpLattice[X] = sim->tmpMemoryChunk + (size_t)X * (ly + 2);
    }
    DropIn *c = new DropIn;
    c->dynp.assign(nodes, 0);
    const char *m = getenv("LBGPU_SYNC");
    if (m) {
        if (!strcmp(m, "none")) c->sync_mode = LB_SYNC_NONE;
        else if (!strcmp(m, "full")) c->sync_mode = LB_SYNC_FULL;
        else c->sync_mode = LB_SYNC_OUTLET;
    }
    sim->device = c;
    // Allocate the device lattice and pin the host arrays now, as part of construction (the
    // reference's drivers time the steps only).  Without a usable device this is retried at
    // the first step, where a failure is reported.
    if (lbgpu::last_error() == LB_OK && lbgpu_device_count() > 0) {
        if (create_device(sim, c) != LB_OK) lbgpu::clear_error();
    }
}

void destructSim(Simulation *sim)
{
    if (!sim) return;
    DropIn *c = ctx_of(sim);
    if (c) {
        if (c->created) {
            if (c->dynp_dev) cudaFree(c->dynp_dev);
            c->L.destroy();
        }
        for (int k = 0; k < 3; ++k)   // before the dynamics-pointer vector goes with c
            if (c->pinned[k]) cudaHostUnregister(c->pinned_ptr[k]);
        delete c;
    }
    free(sim->lattice);
    free(sim->memoryChunk);
    free(sim->tmpLattice);
    free(sim->tmpMemoryChunk);
    std::memset(sim, 0, sizeof *sim);
}

void setDynamics(Simulation *sim, int iX, int iY, Dynamics *dyn)
{
    sim->lattice[iX][iY].dynamics = dyn;
    sim->tmpLattice[iX][iY].dynamics = dyn;
    DropIn *c = ctx_of(sim);
    if (c) {
        c->dynp[(size_t)iX * (sim->ly + 2) + iY] = reinterpret_cast<uint64_t>(dyn);
        c->tags_dirty = true;
        c->dynp_dirty = true;
    }
}

// ---- one-step form ---------------------------------------------------------------------
void collide(Simulation *sim)
{
    DropIn *c = prepare(sim, "collide");
    if (!c) return;
    c->L.launches = 0;
    c->tmp_is_stream = false;
    if (c->L.op_collide()) return;
    finish(sim, c);
}
void collide_openmp(Simulation *sim) { collide(sim); }

void propagate(Simulation *sim)
{
    DropIn *c = prepare(sim, "propagate", false);
    if (!c) return;
    c->L.launches = 0;
    c->tmp_is_stream = false;
    if (c->L.op_propagate()) return;
    swap_host(sim);
    finish(sim, c);
}
void propagate_openmp(Simulation *sim) { propagate(sim); }

void collide_with_stream(Simulation *sim)
{
    DropIn *c = prepare(sim, "collide_with_stream");
    if (!c) return;
    c->L.launches = 0;
    if (c->L.op_collide()) return;
    c->tmp_is_stream = true;
    finish(sim, c);
}
void collide_with_stream_openmp(Simulation *sim) { collide_with_stream(sim); }

// The reference only swaps the two arrays (lb.c:344-348); what the swapped-in array holds
// depends on the call before it.
void finalize_stream(Simulation *sim)
{
    DropIn *c = ctx_of(sim);
    if (!c || !c->uploaded) {
        swap_host(sim);  // nothing on the device yet: the host arrays are the state
        return;
    }
    c = prepare(sim, "finalize_stream", false);
    if (!c) return;
    Lattice &L = c->L;
    L.launches = 0;
    if (c->tmp_is_stream) {
        if (L.op_propagate()) return;  // the second array holds the stream of the collided state
    } else if (L.form == lbgpu::FORM_C && L.pending) {
        L.pending = 0;                 // the second array holds the collided state
    } else {
        // the second array holds the previous collided state (or, before any step, the
        // second array the driver filled)
        L.cur = 1 - L.cur;
        L.form = lbgpu::FORM_C;
        L.pending = 0;
        --L.n;
    }
    c->tmp_is_stream = false;
    swap_host(sim);
    finish(sim, c);
}

// ---- two-step forms (lb.c:442-1779) -------------------------------------------------------
void collide_tight(Simulation *sim) { two_steps(sim, "collide_tight", 0, 0); }
void collide_tight2(Simulation *sim) { two_steps(sim, "collide_tight2", 0, 0); }
void collide_tight_openmp(Simulation *sim) { two_steps(sim, "collide_tight_openmp", 0, 0); }
void collide_tight_block(Simulation *sim) { two_steps(sim, "collide_tight_block", 1, 1); }
void collide_tight_block_openmp(Simulation *sim) { two_steps(sim, "collide_tight_block_openmp", 1, 1); }
void collide_tight_panel_ix(Simulation *sim) { two_steps(sim, "collide_tight_panel_ix", 1, 0); }
void collide_tight_panel_iy(Simulation *sim) { two_steps(sim, "collide_tight_panel_iy", 0, 1); }
void collide_tight_panel_iy_openmp(Simulation *sim) { two_steps(sim, "collide_tight_panel_iy_openmp", 0, 1); }

// ---- periodic wrap and output ---------------------------------------------------------------
void makePeriodic(Simulation *sim)
{
    DropIn *c = ctx_of(sim);
    if (c && !c->uploaded) {
        // before the first step the host arrays are the state: wrap them on the host
        Node **lat = sim->lattice;
        const int lx = sim->lx, ly = sim->ly;
        for (int X = 1; X <= lx; ++X) {
            lat[X][ly].fPop[4] = lat[X][0].fPop[4]; lat[X][ly].fPop[7] = lat[X][0].fPop[7];
            lat[X][ly].fPop[8] = lat[X][0].fPop[8];
            lat[X][1].fPop[2] = lat[X][ly + 1].fPop[2]; lat[X][1].fPop[5] = lat[X][ly + 1].fPop[5];
            lat[X][1].fPop[6] = lat[X][ly + 1].fPop[6];
        }
        for (int Y = 1; Y <= ly; ++Y) {
            lat[1][Y].fPop[1] = lat[lx + 1][Y].fPop[1]; lat[1][Y].fPop[5] = lat[lx + 1][Y].fPop[5];
            lat[1][Y].fPop[8] = lat[lx + 1][Y].fPop[8];
            lat[lx][Y].fPop[3] = lat[0][Y].fPop[3]; lat[lx][Y].fPop[6] = lat[0][Y].fPop[6];
            lat[lx][Y].fPop[7] = lat[0][Y].fPop[7];
        }
        lat[1][1].fPop[5] = lat[lx + 1][ly + 1].fPop[5];
        lat[lx][1].fPop[6] = lat[0][ly + 1].fPop[6];
        lat[lx][ly].fPop[7] = lat[0][0].fPop[7];
        lat[1][ly].fPop[8] = lat[lx + 1][0].fPop[8];
        return;
    }
    c = prepare(sim, "makePeriodic");
    if (!c) return;
    Lattice &L = c->L;
    L.launches = 0;
    c->tmp_is_stream = false;
    if (L.materialize()) return;
    lbgpu::launch_periodic(L.d, L.cur, L.stream);
    ++L.launches;
    if (L.form == lbgpu::FORM_C) {
        // the wrap rewrote stale slots of a collided state: refresh their record
        if (L.init_side_from(L.cur, (int)(L.n & 1))) return;
    }
    if (L.check("makePeriodic")) return;
    finish(sim, c);
}

void lbSyncToHost(Simulation *sim)
{
    DropIn *c = ctx_of(sim);
    if (!c || !c->uploaded) return;  // the host arrays are the state
    if (upload_dynp(c) != LB_OK) return;
    c->L.readout_records(reinterpret_cast<double *>(chunk_of(sim->lattice)), 10, c->dynp_dev, 0,
                         sim->lx + 2);
}

void lbGetTransferBytes(const Simulation *sim, unsigned long long *h2d, unsigned long long *d2h)
{
    DropIn *c = sim ? static_cast<DropIn *>(sim->device) : nullptr;
    if (h2d) *h2d = (c && c->created) ? c->L.h2d_bytes : 0;
    if (d2h) *d2h = (c && c->created) ? c->L.d2h_bytes : 0;
}

void lbMarkHostDirty(Simulation *sim)
{
    DropIn *c = ctx_of(sim);
    if (c && c->uploaded) c->pops_dirty = true;
}

void lbSetSyncMode(Simulation *sim, int mode)
{
    DropIn *c = ctx_of(sim);
    if (!c) { set_error(LB_ERR_STATE, "lbSetSyncMode: simulation not constructed"); return; }
    if (mode < LB_SYNC_NONE || mode > LB_SYNC_FULL) { set_error(LB_ERR_ARG, "lbSetSyncMode: mode %d", mode); return; }
    c->sync_mode = mode;
}

void saveVel(Simulation *sim, char fName[])
{
    lbSyncToHost(sim);
    FILE *f = fopen(fName, "w");
    if (!f) { set_error(LB_ERR_ARG, "saveVel: cannot open %s", fName); return; }
    for (int Y = 1; Y <= sim->ly; ++Y)
        for (int X = 1; X <= sim->lx; ++X) {
            double rho, ux, uy;
            computeMacros(sim->lattice[X][Y].fPop, &rho, &ux, &uy);
            fprintf(f, "%f,%f,%f\n", ux, 1.0, uy);
        }
    fclose(f);
}

void saveF(Simulation *sim, int iPop, char fName[])
{
    lbSyncToHost(sim);
    FILE *f = fopen(fName, "w");
    if (!f) { set_error(LB_ERR_ARG, "saveF: cannot open %s", fName); return; }
    for (int Y = 1; Y <= sim->ly; ++Y) {
        for (int X = 1; X <= sim->lx; ++X) fprintf(f, "%f ", sim->lattice[X][Y].fPop[iPop]);
        fprintf(f, "\n");
    }
    fclose(f);
}

}  // extern "C"
