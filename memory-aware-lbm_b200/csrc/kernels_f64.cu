// kernels_f64.cu -- exact FP64 kernels for sm_100a.
//
// State convention shared by every kernel here (n = index of the last collision):
//   form L : buffer `cur` holds the post-stream populations L_m, stale slots included.
//   form C : buffer `cur` holds the post-collision populations C_n; the post-stream state
//            L_{n+1} is "C_n streamed", read through logical_value().
//   side store parity p = k & 1 holds the post-collision values C_k of the perimeter
//            nodes' stale slots, which the stream two steps later must leave in place
//            (reference: in-place collision lb.c:181-185 + propagation that never reads
//            ghost sources lb.c:258-267 on a second buffer that is reused every other step).
#include "d2q9.cuh"
#include "kernels.h"

namespace lbgpu {

namespace {

constexpr int BX = 128;  // threads along x per block (coalesced axis)

__device__ __forceinline__ const double *plane(const double *b, const Geo &g, int i)
{
    return b + (size_t)i * (size_t)g.plane;
}
__device__ __forceinline__ double *plane(double *b, const Geo &g, int i)
{
    return b + (size_t)i * (size_t)g.plane;
}

// Table entry (p0, p1) of a boundary node (ux, uy) or (rho, uPar).
__device__ __forceinline__ void node_params(const double *__restrict__ bc, const Geo &g, int t,
                                            int X, int Y, double &p0, double &p1)
{
    p0 = 0.0; p1 = 0.0;
    if (t >= TAG_ZOUHE_FIRST && t < TAG_COUNT) {
        const int tb = tag_table(t);
        const int coord = (tag_side(t) <= SIDE_LOWER) ? X : Y;
        p0 = bc[(tb * 2 + 0) * g.nb + coord];
        p1 = bc[(tb * 2 + 1) * g.nb + coord];
    }
}

// Post-stream value of slot i at node (X, Y), for any node of the lattice including the
// ghost ring: the materialized buffer in form L (or a bare collided state), else the
// value streamed from the source node, the side store for an interior node's stale slot,
// or the second buffer's untouched content for a ghost slot with no source.
__device__ __forceinline__ double logical_value(const Geo &g, int pending,
                                                const double *__restrict__ cur,
                                                const double *__restrict__ other,
                                                const double *__restrict__ side, int X, int Y,
                                                int i)
{
    if (!pending) return plane(cur, g, i)[g.idx(X, Y)];
    const int sx = X - cx(i), sy = Y - cy(i);
    if (g.interior(sx, sy)) return plane(cur, g, i)[g.idx(sx, sy)];
    if (g.interior(X, Y)) return side[(size_t)i * g.nper + g.pidx(X, Y)];
    return plane(other, g, i)[g.idx(X, Y)];
}

// In-place collision of every interior node (form L -> form C); the perimeter nodes also
// record their stale slots' post-collision values in side parity `sp`.
__global__ void __launch_bounds__(BX) k_collide_inplace(Geo g, double *__restrict__ buf,
                                                        const uint8_t *__restrict__ tag,
                                                        const double *__restrict__ bc,
                                                        double omega, double *__restrict__ side)
{
    const int X = blockIdx.x * BX + threadIdx.x + 1;
    const int Y = blockIdx.y + 1;
    if (X > g.lx) return;
    const long long o = g.idx(X, Y);
    double f[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) f[i] = plane(buf, g, i)[o];
    const int t = tag[o];
    double p0, p1;
    node_params(bc, g, t, X, Y, p0, p1);
    ex::collide(t, f, omega, p0, p1);
#pragma unroll
    for (int i = 0; i < 9; ++i) plane(buf, g, i)[o] = f[i];
    if (g.perimeter(X, Y)) {
        const int p = g.pidx(X, Y);
#pragma unroll
        for (int i = 0; i < 9; ++i)
            if (!g.interior(X - cx(i), Y - cy(i))) side[(size_t)i * g.nper + p] = f[i];
    }
}

// Fused stream + collide (form C_n in `src` -> form C_{n+1} in `dst`): each interior
// node gathers L_{n+1} from its neighbours (stale slots from side parity (n+1)&1, which
// holds C_{n-1}), collides, writes C_{n+1}, and refreshes the same side parity.  With
// `ghosts`, ghost-ring nodes of `dst` receive the values streamed out of the lattice, as
// the reference's propagation writes them (lb.c:258-267).
template <bool GHOSTS>
__global__ void __launch_bounds__(BX) k_pull(Geo g, const double *__restrict__ src,
                                             double *__restrict__ dst,
                                             const uint8_t *__restrict__ tag,
                                             const double *__restrict__ bc, double omega,
                                             double *__restrict__ side)
{
    const int X = blockIdx.x * BX + threadIdx.x + (GHOSTS ? 0 : 1);
    const int Y = blockIdx.y + (GHOSTS ? 0 : 1);
    if (X > g.lx + (GHOSTS ? 1 : 0)) return;
    const long long o = g.idx(X, Y);
    if (GHOSTS && !g.interior(X, Y)) {
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            const int sx = X - cx(i), sy = Y - cy(i);
            if (g.interior(sx, sy)) plane(dst, g, i)[o] = plane(src, g, i)[g.idx(sx, sy)];
        }
        return;
    }
    double f[9];
    const bool edge = g.perimeter(X, Y);
    if (!edge) {
#pragma unroll
        for (int i = 0; i < 9; ++i)
            f[i] = plane(src, g, i)[o - cx(i) - (long long)cy(i) * g.pitch];
    } else {
        const int p = g.pidx(X, Y);
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            const int sx = X - cx(i), sy = Y - cy(i);
            f[i] = g.interior(sx, sy) ? plane(src, g, i)[g.idx(sx, sy)]
                                      : side[(size_t)i * g.nper + p];
        }
    }
    const int t = tag[o];
    double p0, p1;
    node_params(bc, g, t, X, Y, p0, p1);
    ex::collide(t, f, omega, p0, p1);
#pragma unroll
    for (int i = 0; i < 9; ++i) plane(dst, g, i)[o] = f[i];
    if (edge) {
        const int p = g.pidx(X, Y);
#pragma unroll
        for (int i = 0; i < 9; ++i)
            if (!g.interior(X - cx(i), Y - cy(i))) side[(size_t)i * g.nper + p] = f[i];
    }
}

// Propagation of C_n in `src` into `dst` (form C -> form L), ghost ring included; stale
// slots of interior nodes come from side parity (n-1)&1, ghost slots with no source keep
// `dst`'s content (lb.c:258-267).
__global__ void __launch_bounds__(BX) k_stream(Geo g, const double *__restrict__ src,
                                               double *__restrict__ dst,
                                               const double *__restrict__ side)
{
    const int X = blockIdx.x * BX + threadIdx.x;
    const int Y = blockIdx.y;
    if (X > g.lx + 1) return;
    const long long o = g.idx(X, Y);
    const bool in = g.interior(X, Y);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const int sx = X - cx(i), sy = Y - cy(i);
        if (g.interior(sx, sy)) plane(dst, g, i)[o] = plane(src, g, i)[g.idx(sx, sy)];
        else if (in) plane(dst, g, i)[o] = side[(size_t)i * g.nper + g.pidx(X, Y)];
    }
}

// Copy the stale slots of the perimeter nodes of buffer b into side parity sp.
__global__ void k_side_from_buf(Geo g, const double *__restrict__ buf, double *__restrict__ side)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int nrow = 2 * g.lx, ncol = g.ly > 2 ? 2 * (g.ly - 2) : 0;
    if (k >= nrow + ncol) return;
    int X, Y;
    if (k < g.lx) { X = k + 1; Y = 1; }
    else if (k < nrow) { X = k - g.lx + 1; Y = g.ly; }
    else if (k < nrow + ncol / 2) { X = 1; Y = k - nrow + 2; }
    else { X = g.lx; Y = k - nrow - ncol / 2 + 2; }
    const long long o = g.idx(X, Y);
    const int p = g.pidx(X, Y);
#pragma unroll
    for (int i = 0; i < 9; ++i)
        if (!g.interior(X - cx(i), Y - cy(i))) side[(size_t)i * g.nper + p] = plane(buf, g, i)[o];
}

// Current state of columns [X0, X1) (all rows) as node records of `rs` doubles:
// populations in slots 0..8 and, when `dynp` is given, the host dynamics pointer bits
// in slot 9 (the host Node layout).
__global__ void __launch_bounds__(BX) k_readout(Geo g, const double *__restrict__ cur,
                                                const double *__restrict__ other,
                                                const double *__restrict__ side, int pending,
                                                int X0, int X1, double *__restrict__ out,
                                                int rs, const uint64_t *__restrict__ dynp)
{
    const int Y = blockIdx.x * BX + threadIdx.x;
    const int X = X0 + blockIdx.y;
    if (Y > g.ly + 1 || X >= X1) return;
    const size_t r = ((size_t)(X - X0) * (g.ly + 2) + Y) * rs;
#pragma unroll
    for (int i = 0; i < 9; ++i) out[r + i] = logical_value(g, pending, cur, other, side, X, Y, i);
    if (dynp) {
        const uint64_t v = dynp[(size_t)X * (g.ly + 2) + Y];
        out[r + 9] = __longlong_as_double((long long)v);
    }
}

// Node records of columns [X0, X1) into buffer b (inverse of k_readout).
__global__ void __launch_bounds__(BX) k_upload(Geo g, const double *__restrict__ in, int rs,
                                               int X0, int X1, double *__restrict__ buf)
{
    const int Y = blockIdx.x * BX + threadIdx.x;
    const int X = X0 + blockIdx.y;
    if (Y > g.ly + 1 || X >= X1) return;
    const size_t r = ((size_t)(X - X0) * (g.ly + 2) + Y) * rs;
    const long long o = g.idx(X, Y);
#pragma unroll
    for (int i = 0; i < 9; ++i) plane(buf, g, i)[o] = in[r + i];
}

// Density of the post-stream state at columns lx-1 and lx-2 for every row (the inputs of
// the zero-gradient outlet, unsteady.c:205-214 and lb.c:471-480).
__global__ void k_zgb_rho(Geo g, const double *__restrict__ cur, const double *__restrict__ other,
                          const double *__restrict__ side, int pending, double *__restrict__ zrho)
{
    const int Y = blockIdx.x * blockDim.x + threadIdx.x;
    if (Y > g.ly + 1) return;
    double f[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) f[i] = logical_value(g, pending, cur, other, side, g.lx - 1, Y, i);
    zrho[2 * Y] = ex::density(f);
#pragma unroll
    for (int i = 0; i < 9; ++i) f[i] = logical_value(g, pending, cur, other, side, g.lx - 2, Y, i);
    zrho[2 * Y + 1] = ex::density(f);
}

// Pressure-table slots fed by the extrapolation: rho = 4/3 rho1 - 1/3 rho2, uPar = 0.
__global__ void k_zgb_apply(int nb, const int *__restrict__ zgb_src, const double *__restrict__ zrho,
                            double *__restrict__ bc)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= 4 * nb) return;
    const int src = zgb_src[k];
    if (src < 0) return;
    const int tb = 4 + k / nb, c = k % nb;
    bc[(tb * 2 + 0) * nb + c] = ex::S(ex::M(4. / 3., zrho[2 * src]), ex::M(1. / 3., zrho[2 * src + 1]));
    bc[(tb * 2 + 1) * nb + c] = 0.0;
}

// Periodic wrap of buffer b (form L): the slots a boundary node would receive from across the
// lattice take the values streamed into the opposite ghost ring (lb.c:1783-1817).  The
// three phases run in the reference's order so that later writes win.
__global__ void k_periodic(Geo g, double *__restrict__ buf)
{
    const int lx = g.lx, ly = g.ly;
#define P(i, X, Y) plane(buf, g, (i))[g.idx((X), (Y))]
    for (int X = 1 + threadIdx.x; X <= lx; X += blockDim.x) {
        P(4, X, ly) = P(4, X, 0); P(7, X, ly) = P(7, X, 0); P(8, X, ly) = P(8, X, 0);
        P(2, X, 1) = P(2, X, ly + 1); P(5, X, 1) = P(5, X, ly + 1); P(6, X, 1) = P(6, X, ly + 1);
    }
    __syncthreads();
    for (int Y = 1 + threadIdx.x; Y <= ly; Y += blockDim.x) {
        P(1, 1, Y) = P(1, lx + 1, Y); P(5, 1, Y) = P(5, lx + 1, Y); P(8, 1, Y) = P(8, lx + 1, Y);
        P(3, lx, Y) = P(3, 0, Y); P(6, lx, Y) = P(6, 0, Y); P(7, lx, Y) = P(7, 0, Y);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        P(5, 1, 1) = P(5, lx + 1, ly + 1);
        P(6, lx, 1) = P(6, 0, ly + 1);
        P(7, lx, ly) = P(7, 0, 0);
        P(8, 1, ly) = P(8, lx + 1, 0);
    }
#undef P
}

// Equilibrium at rho = 1 and the Poiseuille velocity of row Y, ux = 4 uMax/L^2 (L y - y^2)
// with y = Y-1, L = ly-1 (unsteady.c:155-159, :169-170); ghost ring zero (lb.c:62-68).
__global__ void __launch_bounds__(BX) k_init_cylinder(Geo g, double *__restrict__ buf, double umax)
{
    const int X = blockIdx.x * BX + threadIdx.x;
    const int Y = blockIdx.y;
    if (X > g.lx + 1) return;
    const long long o = g.idx(X, Y);
    double f[9];
    if (g.interior(X, Y)) {
        const double y = (double)(Y - 1), L = (double)(g.ly - 1);
        const double u = ex::M(ex::D(ex::M(4.0, umax), ex::M(L, L)), ex::S(ex::M(L, y), ex::M(y, y)));
        ex::equilibrium(f, 1.0, u, 0.0);
    } else {
#pragma unroll
        for (int i = 0; i < 9; ++i) f[i] = 0.0;
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) plane(buf, g, i)[o] = f[i];
}

__global__ void __launch_bounds__(BX) k_macros(Geo g, const double *__restrict__ cur,
                                               const double *__restrict__ other,
                                               const double *__restrict__ side, int pending,
                                               double *__restrict__ rho, double *__restrict__ ux,
                                               double *__restrict__ uy)
{
    const int X = blockIdx.x * BX + threadIdx.x + 1;
    const int Y = blockIdx.y + 1;
    if (X > g.lx) return;
    double f[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) f[i] = logical_value(g, pending, cur, other, side, X, Y, i);
    double r, u, v;
    ex::macros(f, r, u, v);
    const size_t k = (size_t)(Y - 1) * g.lx + (X - 1);
    if (rho) rho[k] = r;
    if (ux) ux[k] = u;
    if (uy) uy[k] = v;
}

inline double *B(const DevLattice &d, int b) { return static_cast<double *>(d.buf[b]); }
inline double *SIDE(const DevLattice &d, int p)
{
    return static_cast<double *>(d.side) + (size_t)(p & 1) * 9 * (size_t)d.g.nper;
}
inline unsigned cdiv(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

}  // namespace

void launch_collide_inplace_f64(const DevLattice &d, int cur, int side_par, cudaStream_t s)
{
    dim3 grid(cdiv(d.g.lx, BX), d.g.ly);
    k_collide_inplace<<<grid, BX, 0, s>>>(d.g, B(d, cur), d.tag, d.bc, d.omega, SIDE(d, side_par));
}

void launch_pull_f64(const DevLattice &d, int src, int side_par, bool ghosts, cudaStream_t s)
{
    if (ghosts) {
        dim3 grid(cdiv(d.g.lx + 2, BX), d.g.ly + 2);
        k_pull<true><<<grid, BX, 0, s>>>(d.g, B(d, src), B(d, 1 - src), d.tag, d.bc, d.omega,
                                         SIDE(d, side_par));
    } else {
        dim3 grid(cdiv(d.g.lx, BX), d.g.ly);
        k_pull<false><<<grid, BX, 0, s>>>(d.g, B(d, src), B(d, 1 - src), d.tag, d.bc, d.omega,
                                          SIDE(d, side_par));
    }
}

void launch_stream_f64(const DevLattice &d, int src, int side_par, cudaStream_t s)
{
    dim3 grid(cdiv(d.g.lx + 2, BX), d.g.ly + 2);
    k_stream<<<grid, BX, 0, s>>>(d.g, B(d, src), B(d, 1 - src), SIDE(d, side_par));
}

void launch_side_from_buf_f64(const DevLattice &d, int b, int side_par, cudaStream_t s)
{
    const int n = 2 * d.g.lx + (d.g.ly > 2 ? 2 * (d.g.ly - 2) : 0);
    k_side_from_buf<<<cdiv(n, 256), 256, 0, s>>>(d.g, B(d, b), SIDE(d, side_par));
}

void launch_readout_f64(const DevLattice &d, int cur, int pending, int side_par, int X0, int X1,
                        double *out, int rec_stride, const uint64_t *dynp, cudaStream_t s)
{
    if (X1 <= X0) return;
    dim3 grid(cdiv(d.g.ly + 2, BX), X1 - X0);
    k_readout<<<grid, BX, 0, s>>>(d.g, B(d, cur), B(d, 1 - cur), SIDE(d, side_par), pending, X0,
                                  X1, out, rec_stride, dynp);
}

void launch_upload_f64(const DevLattice &d, int b, const double *in, int rec_stride, int X0,
                       int X1, cudaStream_t s)
{
    if (X1 <= X0) return;
    dim3 grid(cdiv(d.g.ly + 2, BX), X1 - X0);
    k_upload<<<grid, BX, 0, s>>>(d.g, in, rec_stride, X0, X1, B(d, b));
}

void launch_zgb_rho_f64(const DevLattice &d, int cur, int pending, int side_par, cudaStream_t s)
{
    k_zgb_rho<<<cdiv(d.g.ly + 2, 128), 128, 0, s>>>(d.g, B(d, cur), B(d, 1 - cur),
                                                     SIDE(d, side_par), pending, d.zrho);
}

void launch_zgb_apply(const DevLattice &d, cudaStream_t s)
{
    k_zgb_apply<<<cdiv(4LL * d.g.nb, 256), 256, 0, s>>>(d.g.nb, d.zgb_src, d.zrho, d.bc);
}

void launch_periodic_f64(const DevLattice &d, int b, cudaStream_t s)
{
    k_periodic<<<1, 1024, 0, s>>>(d.g, B(d, b));
}

void launch_init_cylinder_f64(const DevLattice &d, int b, double umax, cudaStream_t s)
{
    dim3 grid(cdiv(d.g.lx + 2, BX), d.g.ly + 2);
    k_init_cylinder<<<grid, BX, 0, s>>>(d.g, B(d, b), umax);
}

void launch_macros_f64(const DevLattice &d, int cur, int pending, int side_par, double *rho,
                       double *ux, double *uy, cudaStream_t s)
{
    dim3 grid(cdiv(d.g.lx, BX), d.g.ly);
    k_macros<<<grid, BX, 0, s>>>(d.g, B(d, cur), B(d, 1 - cur), SIDE(d, side_par), pending, rho,
                                 ux, uy);
}

}  // namespace lbgpu
