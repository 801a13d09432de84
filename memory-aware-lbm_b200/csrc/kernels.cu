// kernels.cu -- step, read-out and set-up kernels for sm_100a, for every storage type.
//
// State convention shared by every kernel here (n = index of the last collision):
//   pull form L : buffer `cur` holds the post-stream populations L_m, stale slots included.
//   pull form C : buffer `cur` holds the post-collision populations C_n; the post-stream state
//                 L_{n+1} is "C_n streamed", read through logical().
//   AA natural  : the AA buffer holds L_m in each node's own slots (stale slots in the side store).
//   AA swapped  : the AA buffer holds C_n of direction i in slot opp(i) of each node.
//   side store parity p = k & 1 holds the post-collision values C_k of the perimeter nodes'
//   stale slots, which the stream two steps later must leave in place (reference: in-place
//   collision lb.c:181-185 + propagation that never reads ghost sources lb.c:258-267 into a
//   second buffer that is reused every other step).
//
// Storage types: double (exact FP64 arithmetic), float, __half / __nv_bfloat16 offsets
// (codec.cuh; optionally offset from a per-row equilibrium and stochastically rounded), all with
// the same index space (layout.cuh).
//
// Memory system: the step kernels stream the lattice once per step from HBM; one thread a block
// prefetches into L2 the rows a block a few rows further down will read
// (cp.async.bulk.prefetch.L2, distances measured per kernel); the two-step sweep moves its next
// row into shared memory with cp.async while it computes.
#include <algorithm>
#include "codec.cuh"
#include "kernels.h"
#include "lbgpu.h"

namespace lbgpu {

namespace {

constexpr int BX = 128;  // threads along x per block (coalesced axis)

template <class S>
__device__ __forceinline__ const S *plane(const S *b, const Geo &g, int i)
{
    return b + (size_t)i * (size_t)g.plane;
}
template <class S>
__device__ __forceinline__ S *plane(S *b, const Geo &g, int i)
{
    return b + (size_t)i * (size_t)g.plane;
}

// Table entry (p0, p1) of a boundary node: (ux, uy) or (rho, uPar).
__device__ __forceinline__ void node_params(const double *__restrict__ bc, int nb, int t, int X, int Y,
                                            double &p0, double &p1)
{
    p0 = 0.0; p1 = 0.0;
    if (t >= TAG_ZOUHE_FIRST && t < TAG_COUNT) {
        const int tb = tag_table(t);
        const int coord = (tag_side(t) <= SIDE_LOWER) ? X : Y;
        p0 = bc[(tb * 2 + 0) * nb + coord];
        p1 = bc[(tb * 2 + 1) * nb + coord];
    }
}

__device__ __forceinline__ void node_params(const double *__restrict__ bc, const Geo &g, int t,
                                            int X, int Y, double &p0, double &p1)
{
    node_params(bc, g.nb, t, X, Y, p0, p1);
}

template <class S>
__device__ __forceinline__ void collide_node(const double *__restrict__ bc, const Geo &g, int t,
                                             int X, int Y, typename Codec<S>::R f[9], double omega)
{
    using R = typename Codec<S>::R;
    double p0, p1;
    node_params(bc, g, t, X, Y, p0, p1);
    rules::collide<R>(t, f, (R)omega, (R)p0, (R)p1);
}

template <class S>
__device__ __forceinline__ typename Codec<S>::R dec_row(const Geo &g, S v, int i, float inv, int Y);

// Post-stream value of slot i at node (X, Y), any node of the lattice including the ghost
// ring, under each view (kernels.h).  Ghost slots that no interior node streams into keep the
// content of the buffer the state lives in, as in the reference: for the pull scheme `other`
// is the second buffer; for the AA scheme's swapped view (an odd step count, which the
// reference leaves in its second buffer) `other` is that buffer's saved ghost ring
// [9][nghost].
template <class S>
__device__ __forceinline__ typename Codec<S>::R logical(const Geo &g, int view, const S *__restrict__ cur,
                                                        const S *__restrict__ other,
                                                        const S *__restrict__ side, int X, int Y,
                                                        int i, float inv)
{
    using C = Codec<S>;
    const int sx = X - cx(i), sy = Y - cy(i);
    switch (view) {
    case VIEW_PULL_PENDING:
        if (g.interior(sx, sy)) return dec_row<S>(g, plane(cur, g, i)[g.idx(sx, sy)], i, inv, Y);
        if (g.interior(X, Y)) return dec_row<S>(g, side[(size_t)i * g.nper + g.pidx(X, Y)], i, inv, Y);
        return dec_row<S>(g, plane(other, g, i)[g.idx(X, Y)], i, inv, Y);
    case VIEW_AA_NATURAL:
        if (g.interior(X, Y) && !g.interior(sx, sy))
            return dec_row<S>(g, side[(size_t)i * g.nper + g.pidx(X, Y)], i, inv, Y);
        return dec_row<S>(g, plane(cur, g, i)[g.idx(X, Y)], i, inv, Y);
    case VIEW_AA_SWAPPED:
        if (g.interior(sx, sy)) return dec_row<S>(g, plane(cur, g, opp(i))[g.idx(sx, sy)], i, inv, Y);
        if (g.interior(X, Y)) return dec_row<S>(g, side[(size_t)i * g.nper + g.pidx(X, Y)], i, inv, Y);
        return dec_row<S>(g, other[(size_t)i * g.nghost() + g.gidx(X, Y)], i, inv, Y);
    default:
        return dec_row<S>(g, plane(cur, g, i)[g.idx(X, Y)], i, inv, Y);
    }
}

// ---- 16-bit storage, four nodes per thread ------------------------------------------------
//
// Stored value D_i = (f_i - w_i) 2^s.  With sum(w) = 1 and sum(c w) = 0 the BGK step works on
// D directly: rho = 1 + 2^-s sum(D), j = 2^-s sum(c D), and
//   D_i' = D_i + omega (E_i - D_i),  E_i = 2^s w_i (rho (1 + 3 cu + 4.5 cu^2 - 1.5 u^2) - 1),
// so there is no per-population decode or encode arithmetic, only the conversions (two per
// instruction when packing).  Boundary rules decode to f and use the generic path.

template <class S> struct Half2Ops;
template <> struct Half2Ops<__half> {
    static __device__ __forceinline__ float lo(unsigned w) { return __half2float(__ushort_as_half((unsigned short)(w & 0xffffu))); }
    static __device__ __forceinline__ float hi(unsigned w) { return __half2float(__ushort_as_half((unsigned short)(w >> 16))); }
    static __device__ __forceinline__ unsigned pack(float a, float b)
    {
        const __half2 h = __floats2half2_rn(a, b);
        return *reinterpret_cast<const unsigned *>(&h);
    }
};
template <> struct Half2Ops<__nv_bfloat16> {
    static __device__ __forceinline__ float lo(unsigned w) { return __uint_as_float(w << 16); }
    static __device__ __forceinline__ float hi(unsigned w) { return __uint_as_float(w & 0xffff0000u); }
    static __device__ __forceinline__ unsigned pack(float a, float b)
    {
        const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
        return *reinterpret_cast<const unsigned *>(&h);
    }
};

// BGK on scaled offsets D[9] of one node (sc = 2^s, inv = 2^-s).  With d = rho - 1 =
// inv sum(D) and j = rho u = inv sum(c D), rho c.u = c.j and rho u^2 = j.u give
//   E_i = sc w_i (A + 3 c.j + 4.5 (c.u)(c.j)),  A = d - 1.5 j.u,
// and the relaxation is D_i' = (1 - omega) D_i + omega E_i.  Opposite directions i, opp(i)
// share c.u and c.j up to sign: omega E_i, omega E_opp = a +- b with
// a = k (A + 4.5 (c.u)(c.j)), b = 3 k c.j, k = omega sc w.
// With a row shift (SHIFT, offsets relative to S_i = f_eq_i(1, (us, 0)) instead of w_i):
// j = (us, 0) + inv J, E_i = sc (f_eq_i(rho, u) - S_i), so A gains -1.5 us (ux - us) and a gains
// 4.5 k (c.us)(c.u - c.us); b is unchanged.  Without it the arithmetic is exactly the unshifted one.
// 1/rho uses the hardware reciprocal (the 16-bit path is held to a tolerance, not bit-exact).
template <bool SHIFT>
__device__ __forceinline__ void bgk_offsets(float D[9], float omega, float sc, float inv, float us)
{
    // J = 2^s (j - us): scaled sums; u = J inv / rho (+ us / rho), inv folded into constants
    const float sum = ((D[0] + D[1]) + (D[2] + D[3])) + ((D[4] + D[5]) + (D[6] + D[7])) + D[8];
    const float d = inv * sum;
    const float Jx = (D[1] - D[3]) + (D[5] - D[6]) + (D[8] - D[7]);
    const float Jy = (D[2] - D[4]) + (D[5] - D[8]) + (D[6] - D[7]);
    const float ir = __fdividef(1.0f, 1.0f + d);
    const float q = inv * ir;
    const float ux = SHIFT ? fmaf(Jx, q, __fmul_rn(us, ir)) : Jx * q, uy = Jy * q;
    float A = fmaf(-1.5f * inv, fmaf(Jx, ux, Jy * uy), d);
    // shifted terms: t = ux - us; 4.5 (c.us)(c.u - c.us) is e1 = 4.5 us t for (1, 3) and
    // e1 +- 4.5 us uy for (5, 7) and (6, 8), folded into the pair's constant term: A1 = A + e1,
    // A1 +- 4.5 us uy
    const float t = SHIFT ? __fsub_rn(ux, us) : 0.0f;
    if (SHIFT) A = fmaf(-1.5f * us, t, A);
    const float ux45 = (4.5f * inv) * ux, uy45 = (4.5f * inv) * uy;
    const float hs = 4.5f * us;
    const float A1 = SHIFT ? fmaf(hs, t, A) : A, ev = SHIFT ? __fmul_rn(hs, uy) : 0.0f;
    const float A5 = SHIFT ? __fadd_rn(A1, ev) : A, A6 = SHIFT ? __fsub_rn(A1, ev) : A;
    const float om1 = 1.0f - omega;
    const float k0 = omega * sc * (4.f / 9.f), k1 = omega * sc * (1.f / 9.f), k2 = omega * sc * (1.f / 36.f);
    D[0] = fmaf(om1, D[0], k0 * A);
    // The shifted terms use explicitly rounded operations: no multiply-add contraction may
    // differ between the kernels that inline this, so every scheme stays bit-identical.
#define LBGPU_PAIR(I, J, K, CU45, CJ, AP)                              \
    {                                                                  \
        const float cj = (CJ);                                         \
        if (SHIFT) {                                                   \
            const float a = __fmul_rn(K, fmaf(CU45, cj, (AP)));        \
            const float b = __fmul_rn((3.0f * inv) * K, cj);          \
            D[I] = fmaf(om1, D[I], __fadd_rn(a, b));                   \
            D[J] = fmaf(om1, D[J], __fsub_rn(a, b));                   \
        } else {                                                       \
            const float a = K * fmaf(CU45, cj, A);                     \
            const float b = ((3.0f * inv) * K) * cj;                   \
            D[I] = fmaf(om1, D[I], a + b);                             \
            D[J] = fmaf(om1, D[J], a - b);                             \
        }                                                              \
    }
    LBGPU_PAIR(1, 3, k1, ux45, Jx, A1)
    LBGPU_PAIR(2, 4, k1, uy45, Jy, A)
    LBGPU_PAIR(5, 7, k2, __fadd_rn(ux45, uy45), __fadd_rn(Jx, Jy), A5)
    LBGPU_PAIR(6, 8, k2, __fsub_rn(uy45, ux45), __fsub_rn(Jy, Jx), A6)
#undef LBGPU_PAIR
}


// Working values of a kernel: decoded populations f for FP64/FP32, the stored offsets D as
// float for 16-bit storage (see bgk_offsets); collide_w applies a node's rule to them.  Every
// kernel of one storage type uses these, so all schemes agree bit for bit.
template <class S> struct Work {
    using W = typename Codec<S>::R;
    static __device__ __forceinline__ W load(S v, int i, float inv) { return Codec<S>::dec(v, i, inv); }
    static __device__ __forceinline__ S store(W w, int i, float sc) { return Codec<S>::enc(w, i, sc); }
};
template <> struct Work<__half> {
    using W = float;
    static __device__ __forceinline__ float load(__half v, int, float) { return __half2float(v); }
    static __device__ __forceinline__ __half store(float w, int, float) { return __float2half_rn(w); }
};
template <> struct Work<__nv_bfloat16> {
    using W = float;
    static __device__ __forceinline__ float load(__nv_bfloat16 v, int, float) { return __bfloat162float(v); }
    static __device__ __forceinline__ __nv_bfloat16 store(float w, int, float) { return __float2bfloat16_rn(w); }
};

// Stochastic rounding (codec.cuh) is a compile-time choice of a kernel (RS), so no store
// carries a branch: RS kernels run only for 16-bit lattices with it on, whose collision key is
// then never 0.
// The random word of node (X, Y) for a collision key.
template <class S, bool RS>
__device__ __forceinline__ RsNode rs_node(const Geo &g, unsigned key, int X, int Y)
{
    if constexpr (RS && sizeof(S) == 2) {
        const int q = (X - 1) & 3;
        return RsNode{rs_mix(((unsigned)Y * (unsigned)(g.lx + 2) + (unsigned)(X - q)) ^ key), q};
    }
    return RsNode{0u, 0};
}

// A post-collision working value of direction i as stored: rounded to nearest, or (RS)
// stochastically with the node's random word h.
template <class S, bool RS>
__device__ __forceinline__ S put(typename Work<S>::W w, int i, float sc, RsNode h)
{
    if constexpr (RS && sizeof(S) == 2) {
        const unsigned p = rs_pair(h.hq, h.q >> 1, i);
        return RsOps<S>::one(w, (h.q & 1) ? (p >> 16) : p);
    }
    return Work<S>::store(w, i, sc);
}

// Decode / encode of a value consumed at row Y (read-outs, uploads, initial states).
template <class S>
__device__ __forceinline__ typename Codec<S>::R dec_row(const Geo &g, S v, int i, float inv, int Y)
{
    if constexpr (sizeof(S) == 2) {
        if (g.shift_u) return fmaf(Work<S>::load(v, i, inv), inv, g.shift_base(Y)[i]);
    }
    return Codec<S>::dec(v, i, inv);
}

template <class S>
__device__ __forceinline__ S enc_row(const Geo &g, typename Codec<S>::R f, int i, float sc, int Y)
{
    if constexpr (sizeof(S) == 2) {
        if (g.shift_u) return Work<S>::store(__fmul_rn(__fsub_rn(f, g.shift_base(Y)[i]), sc), i, sc);
    }
    return Codec<S>::enc(f, i, sc);
}

// A post-collision value of direction i at row Y, as stored in a population plane: with a row
// shift it is relative to the row that consumes it after streaming, Y + c_iy (stale-slot copies
// in the side store are consumed by the node itself and stay relative to row Y).
// SH: 0 no shift, 1 shift (known at compile time), 2 decided by g.shift_u at run time.
// Rows whose rebase values are all zero (shift_rebased false) store unchanged in every kernel.
template <class S, int SH = 2>
__device__ __forceinline__ typename Work<S>::W stored_out(const Geo &g, int Y, int i, typename Work<S>::W w,
                                                          float sc)
{
    if constexpr (sizeof(S) == 2 && SH != 0) {
        if (cy(i) != 0 && (SH == 1 || g.shift_u) && g.shift_rebased(Y))
            return __fadd_rn(w, __fmul_rn(g.shift_rebase(Y)[i], sc));
    }
    return w;
}

// A non-BGK rule on one node's 16-bit offsets: decode, the generic rule, encode.  Out of line so
// the bulk path keeps its registers (it runs for boundary and obstacle nodes only); the shifted
// form is a separate function, because a larger callee costs the 64-register quad kernel spills.
template <class S>
static __device__ __noinline__ void boundary_offsets(const double *__restrict__ bc, Geo g, int t, int X,
                                                     int Y, float D[9], double omega, float sc, float inv)
{
    float f[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) f[i] = fmaf(D[i], inv, wgtf(i));
    collide_node<S>(bc, g, t, X, Y, f, omega);
#pragma unroll
    for (int i = 0; i < 9; ++i) D[i] = (f[i] - wgtf(i)) * sc;
}

// The same with offsets from the row's shift equilibrium (base: S_i of the row).
template <class S>
static __device__ __noinline__ void boundary_offsets_shifted(const double *__restrict__ bc, int nb,
                                                             const float *__restrict__ base, int t, int X, int Y,
                                                             float D[9], double omega, float sc, float inv)
{
    float f[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) f[i] = fmaf(D[i], inv, base[i]);
    double p0, p1;
    node_params(bc, nb, t, X, Y, p0, p1);
    rules::collide<float>(t, f, (float)omega, (float)p0, (float)p1);
#pragma unroll
    for (int i = 0; i < 9; ++i) D[i] = (f[i] - base[i]) * sc;
}

template <class S, int SH = 2>
__device__ __forceinline__ void collide_w(const double *__restrict__ bc, const Geo &g, int t, int X,
                                          int Y, typename Work<S>::W w[9], double omega, float sc,
                                          float inv)
{
    if constexpr (sizeof(S) == 2) {
        if (t == TAG_BGK) {
            if constexpr (SH == 1) bgk_offsets<true>(w, (float)omega, sc, inv, g.shift_u[Y]);
            else if constexpr (SH == 0) bgk_offsets<false>(w, (float)omega, sc, inv, 0.0f);
            else if (g.shift_u) bgk_offsets<true>(w, (float)omega, sc, inv, g.shift_u[Y]);
            else bgk_offsets<false>(w, (float)omega, sc, inv, 0.0f);
        } else {
            float tmp[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) tmp[i] = w[i];
            if (SH == 1 || (SH == 2 && g.shift_u))
                boundary_offsets_shifted<S>(bc, g.nb, g.shift_base(Y), t, X, Y, tmp, omega, sc, inv);
            else
                boundary_offsets<S>(bc, g, t, X, Y, tmp, omega, sc, inv);
#pragma unroll
            for (int i = 0; i < 9; ++i) w[i] = tmp[i];
        }
    } else {
        collide_node<S>(bc, g, t, X, Y, w, omega);
    }
}

// L2 prefetch for the block a few rows further down the grid (blocks run roughly in row order,
// so those rows are read soon after, from L2): one thread a block issues the nine row segments
// that block reads, nodes x0 .. x0 + NW - 1 of rows Y - c_iy widened by 16 bytes a side
// (cp.async.bulk.prefetch.L2: no completion to wait for).  A segment starts on a 16-byte boundary
// (the layout puts X = 1 on a 128-byte line and x0 - 1 is a multiple of NW) and is a multiple of
// 16 bytes long; blocks whose segment would pass the row's pitch skip it, as do rows past ly, so
// every prefetched byte is inside its plane.
// Distances measured on the 16384x4096 channel (GLUPS without -> with): 16-bit pull 16 rows
// (157.7 -> 170.9 FP16, 157.7 -> 171.7 BF16); FP32 pull 8 rows (88.0 -> 90.3); FP64 pull none (it
// runs at the copy bandwidth already, and 8 / 16 / 32 rows cost 1 / 10 / 29 %: rows fetched that
// early are evicted before they are read).
#ifndef LBGPU_PF_ROWS
#define LBGPU_PF_ROWS 16       // 16-bit pull kernel
#endif
#ifndef LBGPU_PF_TAGS
#define LBGPU_PF_TAGS 1        // the 16-bit pull kernel's tag row as well (167.4 -> 169.5 FP16)
#endif
// The tag row is prefetched with the population rows by the AA kernels too (about 2 % each:
// FP16 149.3 -> 152.1, FP32 83.7 -> 85.4, FP64 44.5 -> 45.4), not by the FP32 pull kernel
// (no change there).
#ifndef LBGPU_PF_ROWS_F32
#define LBGPU_PF_ROWS_F32 8    // FP32 pull kernel
#endif
#ifndef LBGPU_PF_ROWS_AA
#define LBGPU_PF_ROWS_AA 16    // 16-bit AA kernels (140.4 -> 150.8 FP16)
#endif
template <class S>
constexpr int pf_rows_wide() { return sizeof(S) == 4 ? LBGPU_PF_ROWS_F32 : 0; }
#ifndef LBGPU_PF_ROWS_AA_F32
#define LBGPU_PF_ROWS_AA_F32 8    // FP32 AA kernels (78.8 -> 86.1)
#endif
#ifndef LBGPU_PF_ROWS_AA_F64
#define LBGPU_PF_ROWS_AA_F64 4    // FP64 AA kernels (42.6 -> 45.7)
#endif
template <class S>
constexpr int pf_rows_aa_wide() { return sizeof(S) == 4 ? LBGPU_PF_ROWS_AA_F32 : (sizeof(S) == 8 ? LBGPU_PF_ROWS_AA_F64 : 0); }
// ROWS: which row of plane i a node of row Y reads: 0 row Y - c_iy (pull), 1 row Y (AA even
// step), 2 row Y + c_iy (AA odd step, whose direction i comes from plane opp(i) at row Y - c_iy).
template <class S, int NW, int ROWS = 0>
__device__ __forceinline__ void prefetch_rows_l2(const Geo &g, const S *__restrict__ src, int x0, int Y,
                                                 const uint8_t *__restrict__ tag = nullptr)
{
    constexpr int H = 16 / (int)sizeof(S);                          // halo elements a side
    constexpr unsigned BYTES = (unsigned)((NW + 2 * H) * sizeof(S));
    if (Y > g.ly || (long long)(x0 + NW + H - 1) + g.xoff - 1 >= g.pitch) return;
    if (tag)   // the block's tag row: one byte a node, 16-byte aligned like the rows
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(tag + g.idx(x0, Y)), "n"(NW) : "memory");
#pragma unroll
    for (int i = 0; i < 9; ++i)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;"
                     ::"l"(plane(src, g, i) + g.idx(x0 - H, ROWS == 0 ? Y - cy(i) : (ROWS == 1 ? Y : Y + cy(i)))),
                     "n"(BYTES)
                     : "memory");
}

// ---- pull scheme --------------------------------------------------------------------------

// In-place collision of every interior node (form L -> form C); the perimeter nodes also
// record their stale slots' post-collision values in the side parity given.
template <class S, bool RS>
__global__ void __launch_bounds__(BX) k_collide_inplace(Geo g, S *__restrict__ buf,
                                                        const uint8_t *__restrict__ tag,
                                                        const double *__restrict__ bc, double omega,
                                                        S *__restrict__ side, float sc, float inv)
{
    using C = Codec<S>;
    using R = typename C::R;
    const int X = blockIdx.x * BX + threadIdx.x + 1;
    const int Y = blockIdx.y + 1;
    if (X > g.lx) return;
    const long long o = g.idx(X, Y);
    typename Work<S>::W f[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) f[i] = Work<S>::load(plane(buf, g, i)[o], i, inv);
    collide_w<S>(bc, g, tag[o], X, Y, f, omega, sc, inv);
    const RsNode h = rs_node<S, RS>(g, g.rs_key, X, Y);
#pragma unroll
    for (int i = 0; i < 9; ++i) plane(buf, g, i)[o] = put<S, RS>(stored_out<S>(g, Y, i, f[i], sc), i, sc, h);
    if (g.perimeter(X, Y)) {
        const int p = g.pidx(X, Y);
#pragma unroll
        for (int i = 0; i < 9; ++i)
            if (!g.interior(X - cx(i), Y - cy(i))) side[(size_t)i * g.nper + p] = put<S, RS>(f[i], i, sc, h);
    }
}

// Fused stream + collide (form C_n in `src` -> form C_{n+1} in `dst`): each interior node
// gathers L_{n+1} from its neighbours (stale slots from the side parity holding C_{n-1}),
// collides, writes C_{n+1} and refreshes the same side parity.  With GHOSTS, ghost-ring nodes
// of `dst` receive the values streamed out of the lattice, as the reference's propagation
// writes them (lb.c:258-267).  Lanes map X = 1, 2, ... as without the ring, so every warp's
// rows start on a 128-byte line; the thread of column lx+1 also takes ghost column 0.
template <class S>
__device__ __forceinline__ void ring_node(const Geo &g, const S *__restrict__ src, S *__restrict__ dst, int X,
                                          int Y)
{
    const long long o = g.idx(X, Y);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const int sx = X - cx(i), sy = Y - cy(i);
        if (g.interior(sx, sy)) plane(dst, g, i)[o] = plane(src, g, i)[g.idx(sx, sy)];
    }
}

template <class S, bool GHOSTS>
__global__ void __launch_bounds__(BX) k_pull(Geo g, const S *__restrict__ src, S *__restrict__ dst,
                                             const uint8_t *__restrict__ tag,
                                             const double *__restrict__ bc, double omega,
                                             S *__restrict__ side, float sc, float inv)
{
    using C = Codec<S>;
    using R = typename C::R;
    const int X = blockIdx.x * BX + threadIdx.x + 1;
    const int Y = blockIdx.y + (GHOSTS ? 0 : 1);
    if (!GHOSTS && pf_rows_wide<S>() > 0 && threadIdx.x == 0)
        prefetch_rows_l2<S, BX>(g, src, 1 + BX * (int)blockIdx.x, Y + pf_rows_wide<S>());
    if (X > g.lx + (GHOSTS ? 1 : 0)) return;
    const long long o = g.idx(X, Y);
    if (GHOSTS && !g.interior(X, Y)) {
        ring_node(g, src, dst, X, Y);
        if (X == g.lx + 1) ring_node(g, src, dst, 0, Y);
        return;
    }
    typename Work<S>::W f[9];
    const bool edge = g.perimeter(X, Y);
    if (!edge) {
#pragma unroll
        for (int i = 0; i < 9; ++i)
            f[i] = Work<S>::load(plane(src, g, i)[o - cx(i) - (long long)cy(i) * g.pitch], i, inv);
    } else {
        const int p = g.pidx(X, Y);
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            const int sx = X - cx(i), sy = Y - cy(i);
            f[i] = Work<S>::load(g.interior(sx, sy) ? plane(src, g, i)[g.idx(sx, sy)]
                                             : side[(size_t)i * g.nper + p], i, inv);
        }
    }
    collide_w<S>(bc, g, tag[o], X, Y, f, omega, sc, inv);
#pragma unroll
    for (int i = 0; i < 9; ++i) plane(dst, g, i)[o] = Work<S>::store(stored_out<S>(g, Y, i, f[i], sc), i, sc);
    if (edge) {
        const int p = g.pidx(X, Y);
#pragma unroll
        for (int i = 0; i < 9; ++i)
            if (!g.interior(X - cx(i), Y - cy(i))) side[(size_t)i * g.nper + p] = Work<S>::store(f[i], i, sc);
    }
}

// Pull step of one node, any storage type (the general path of every pull kernel).
template <class S, int SH = 2, bool RS = false>
__device__ __forceinline__ void pull_node(const Geo &g, const S *__restrict__ src, S *__restrict__ dst,
                                          const uint8_t *__restrict__ tag, const double *__restrict__ bc,
                                          double omega, S *__restrict__ side, float sc, float inv,
                                          int X, int Y, unsigned key = 0u)
{
    const long long o = g.idx(X, Y);
    typename Work<S>::W f[9];
    const bool edge = g.perimeter(X, Y);
    const int p = edge ? g.pidx(X, Y) : 0;
    if (!edge) {
#pragma unroll
        for (int i = 0; i < 9; ++i)
            f[i] = Work<S>::load(plane(src, g, i)[o - cx(i) - (long long)cy(i) * g.pitch], i, inv);
    } else {
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            const int sx = X - cx(i), sy = Y - cy(i);
            f[i] = Work<S>::load(g.interior(sx, sy) ? plane(src, g, i)[g.idx(sx, sy)]
                                                    : side[(size_t)i * g.nper + p], i, inv);
        }
    }
    collide_w<S, SH>(bc, g, tag[o], X, Y, f, omega, sc, inv);
    const RsNode h = rs_node<S, RS>(g, key, X, Y);
#pragma unroll
    for (int i = 0; i < 9; ++i) plane(dst, g, i)[o] = put<S, RS>(stored_out<S, SH>(g, Y, i, f[i], sc), i, sc, h);
    if (edge) {
#pragma unroll
        for (int i = 0; i < 9; ++i)
            if (!g.interior(X - cx(i), Y - cy(i))) side[(size_t)i * g.nper + p] = put<S, RS>(f[i], i, sc, h);
    }
}

// Perimeter node number p (Geo::pidx numbering: row 1, row ly, then columns 1 and lx without
// their corners) -> its coordinates; false for numbers that name no node, or a node a second
// time where the lattice is one row or one column wide.
__device__ __forceinline__ bool perim_node(const Geo &g, int p, int &X, int &Y)
{
    if (p < g.lx) { X = p + 1; Y = 1; return true; }
    if (p < 2 * g.lx) { X = p - g.lx + 1; Y = g.ly; return g.ly > 1; }
    const int q = p - 2 * g.lx;
    if (q < g.ly - 2) { X = 1; Y = q + 2; return true; }
    if (q >= g.ly && q < 2 * g.ly - 2) { X = g.lx; Y = q - g.ly + 2; return g.lx > 1; }
    return false;
}

// The pull step of every perimeter node, one a thread (the 16-bit quad kernels leave them out,
// see pull_quad's PERIM_APART).
template <class S, int SH, bool RS>
__global__ void __launch_bounds__(256) k_perim_pull(Geo g, const S *__restrict__ src, S *__restrict__ dst,
                                                    const uint8_t *__restrict__ tag, const double *__restrict__ bc,
                                                    double omega, S *__restrict__ side, float sc, float inv)
{
    int X, Y;
    if (perim_node(g, (int)(blockIdx.x * 256 + threadIdx.x), X, Y))
        pull_node<S, SH, RS>(g, src, dst, tag, bc, omega, side, sc, inv, X, Y, g.rs_key);
}

// The hash of the quad x0..x0+3 (RS only).
template <class S, bool RS>
__device__ __forceinline__ unsigned quad_hash(const Geo &g, unsigned key, int x0, int Y)
{
    return RS ? rs_mix(((unsigned)Y * (unsigned)(g.lx + 2) + (unsigned)x0) ^ key) : 0u;
}

// Direction i of a quad's four working values as the stored aligned word pair.
template <class S, bool RS>
__device__ __forceinline__ uint2 pack_quad(const float D[4][9], int i, unsigned hq)
{
    uint2 w;
    if constexpr (RS) {
        w.x = RsOps<S>::pack(D[0][i], D[1][i], rs_pair(hq, 0, i));
        w.y = RsOps<S>::pack(D[2][i], D[3][i], rs_pair(hq, 1, i));
    } else {
        w.x = Half2Ops<S>::pack(D[0][i], D[1][i]);
        w.y = Half2Ops<S>::pack(D[2][i], D[3][i]);
    }
    return w;
}

// Pull step for 16-bit storage, four nodes per thread (X = x0..x0+3 with x0 = 1 mod 4, so a
// quad is one aligned 8-byte word pair).  Per direction one aligned 8-byte load; an x-shifted
// quad is assembled by byte permutes from that word pair and the neighbouring 4-byte word,
// loaded by every lane (the adjacent lane's data, so an L1 hit).  The kernel is bounded by
// instruction issue, so the collision is written for few instructions (bgk_offsets) and the
// boundary rules stay out of line.
//
// pull_quad runs the four nodes x0..x0+3 of row Y for one lane.  Rows 1 and ly run the per-node
// path.  On every other row each lane runs the vector path; a quad whose nodes are all inside
// 2..lx-1 stores its word pairs, a quad at either end of the row (a row's first quad holds the
// perimeter column 1, its last the column lx and possibly nodes past the row) stores its inner
// nodes one by one and recomputes its perimeter node with the per-node path.  So only the one
// or two edge lanes of a row do extra work, instead of whole edge warps running per node.  The
// vector loads of an edge quad stay inside the allocation: left of column 1 they reach the row
// padding and ghost column (x0 - 2 >= -1), past lx they reach at most five elements into the
// row padding or the next row, which exists because Y <= ly - 1.
// PERIM_APART: the perimeter nodes are stepped by another kernel (the batch's BATCH_PERIM
// list): rows 1 and ly are skipped, and an edge quad stores its inner nodes only, so no lane of
// a quad warp runs the per-node path while the others wait.
template <class S, bool SHIFT, bool RS = false, bool PERIM_APART = false>
__device__ __forceinline__ void pull_quad(const Geo &g, const S *__restrict__ src, S *__restrict__ dst,
                                          const uint8_t *__restrict__ tag, const double *__restrict__ bc,
                                          double omega, S *__restrict__ side, float sc, float inv, int x0,
                                          int Y, int lane, unsigned key = 0u)
{
    using H = Half2Ops<S>;
    (void)lane;
    if (Y < 2 || Y > g.ly - 1) {
        if constexpr (!PERIM_APART) {
            for (int k = 0; k < 4; ++k)
                if (x0 + k <= g.lx) pull_node<S, SHIFT ? 1 : 0, RS>(g, src, dst, tag, bc, omega, side, sc, inv, x0 + k, Y, key);
        }
        return;
    }
    if (x0 > g.lx) return;
    const long long o = g.idx(x0, Y);
    uint2 v[9];
    unsigned e[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const S *row = plane(src, g, i) + (o - (long long)cy(i) * g.pitch);
        v[i] = *reinterpret_cast<const uint2 *>(row);
        // the word holding the shifted quad's outer source (the neighbouring lane's data:
        // an L1 hit, no extra DRAM traffic, and no shuffle)
        if (cx(i) == 1) e[i] = *reinterpret_cast<const unsigned *>(row - 2);
        if (cx(i) == -1) e[i] = *reinterpret_cast<const unsigned *>(row + 4);
    }
    const unsigned tq = *reinterpret_cast<const unsigned *>(tag + o);
    float D[4][9];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        unsigned w0 = v[i].x, w1 = v[i].y;
        if (cx(i) == 1) {            // quad of sources x0-1..x0+2
            const unsigned n0 = __byte_perm(e[i], w0, 0x5432), n1 = __byte_perm(w0, w1, 0x5432);
            w0 = n0; w1 = n1;
        } else if (cx(i) == -1) {    // quad of sources x0+1..x0+4
            const unsigned n0 = __byte_perm(w0, w1, 0x5432), n1 = __byte_perm(w1, e[i], 0x5432);
            w0 = n0; w1 = n1;
        }
        D[0][i] = H::lo(w0); D[1][i] = H::hi(w0);
        D[2][i] = H::lo(w1); D[3][i] = H::hi(w1);
    }
    if (tq == 0x01010101u) {         // four bulk nodes
        const float om = (float)omega;
        const float us = SHIFT ? g.shift_u[Y] : 0.0f;
#pragma unroll
        for (int k = 0; k < 4; ++k) bgk_offsets<SHIFT>(D[k], om, sc, inv, us);
    } else {
#pragma unroll
        for (int k = 0; k < 4; ++k)
            collide_w<S, SHIFT ? 1 : 0>(bc, g, (int)((tq >> (8 * k)) & 0xff), x0 + k, Y, D[k], omega, sc, inv);
    }
    const unsigned hq = quad_hash<S, RS>(g, key, x0, Y);
    if (SHIFT && g.shift_rebased(Y)) {
#pragma unroll
        for (int i = 0; i < 9; ++i)
#pragma unroll
            for (int k = 0; k < 4; ++k) D[k][i] = stored_out<S, 1>(g, Y, i, D[k][i], sc);
    }
    if (x0 >= 2 && x0 + 3 <= g.lx - 1) {
#pragma unroll
        for (int i = 0; i < 9; ++i)
            *reinterpret_cast<uint2 *>(plane(dst, g, i) + o) = pack_quad<S, RS>(D, i, hq);
    } else {                         // a row's first or last quad: its inner nodes one by one
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (x0 + k < 2 || x0 + k > g.lx - 1) continue;
#pragma unroll
            for (int i = 0; i < 9; ++i) plane(dst, g, i)[o + k] = put<S, RS>(D[k][i], i, sc, RsNode{hq, k});
        }
        if constexpr (PERIM_APART) return;
        if (x0 == 1) pull_node<S, SHIFT ? 1 : 0, RS>(g, src, dst, tag, bc, omega, side, sc, inv, 1, Y, key);
        if (g.lx >= x0 && g.lx <= x0 + 3 && g.lx >= 2)
            pull_node<S, SHIFT ? 1 : 0, RS>(g, src, dst, tag, bc, omega, side, sc, inv, g.lx, Y, key);
    }
}

// Perimeter nodes stepped apart from the quads (see k_pull4h): 1 for the row-shifted forms only,
// 2 for every form, 0 for none.  Measured on one B200 at 16384 x 4096 (GLUPS, apart / in the
// quad warps): banded shift + stochastic 155-158 / 148-151, banded shift 161 / 158; FP16 170 /
// 174, FP16 stochastic 166 / 172, BF16 171 / 174.
#ifndef LBGPU_PULL4H_PERIM_APART
#define LBGPU_PULL4H_PERIM_APART 1
#endif
template <bool SHIFT>
constexpr bool pull4h_perim_apart() { return LBGPU_PULL4H_PERIM_APART == 2 || (LBGPU_PULL4H_PERIM_APART == 1 && SHIFT); }
// Resident blocks of the row-shifted form: 8 (64 registers) since its perimeter runs apart from
// the quads (the quad path then spills 28-48 bytes); measured on one B200 at 16384 x 4096, banded
// shift + stochastic 165.4-165.8 GLUPS against 162.3-162.4 at 7 blocks (72 registers), exact
// profile + stochastic 151-153 against 143-144.
#ifndef LBGPU_PULL4H_SHIFT_MINB
#define LBGPU_PULL4H_SHIFT_MINB 8
#endif
// PERIM_APART: the quads leave the perimeter to another pass (see pull_quad); PERIM_ROWS: that pass
// is the grid rows past the lattice's ly rows, one perimeter node a thread, so it runs inside the
// same launch (in its tail) instead of as a launch of its own.
template <class S, bool SHIFT, bool RS, bool PERIM_APART = false, bool PERIM_ROWS = false>
__global__ void __launch_bounds__(BX, SHIFT ? LBGPU_PULL4H_SHIFT_MINB : 8) k_pull4h(Geo g, const S *__restrict__ src, S *__restrict__ dst,
                                               const uint8_t *__restrict__ tag,
                                               const double *__restrict__ bc, double omega,
                                               S *__restrict__ side, float sc, float inv)
{
    if (LBGPU_PF_ROWS > 0 && threadIdx.x == 0)
        prefetch_rows_l2<S, 4 * BX>(g, src, 1 + 4 * BX * (int)blockIdx.x, (int)blockIdx.y + 1 + LBGPU_PF_ROWS,
                                    LBGPU_PF_TAGS ? tag : nullptr);
    if (PERIM_ROWS && (int)blockIdx.y >= g.ly) {   // the grid rows past the lattice: perimeter nodes
        int X, Y;
        const int p = (int)(((blockIdx.y - g.ly) * gridDim.x + blockIdx.x) * BX + threadIdx.x);
        if (perim_node(g, p, X, Y))
            pull_node<S, SHIFT ? 1 : 0, RS>(g, src, dst, tag, bc, omega, side, sc, inv, X, Y, g.rs_key);
        return;
    }
    const int t = blockIdx.x * BX + threadIdx.x;
    pull_quad<S, SHIFT, RS, PERIM_APART>(g, src, dst, tag, bc, omega, side, sc, inv, 1 + 4 * t, blockIdx.y + 1,
                                         threadIdx.x & 31, g.rs_key);
}

// Propagation of C_n in `src` into `dst` (form C -> form L), ghost ring included; stale
// slots of interior nodes come from the side parity holding C_{n-1}; ghost slots with no
// source keep `dst`'s content (lb.c:258-267).  Stored values move unchanged.
template <class S>
__global__ void __launch_bounds__(BX) k_stream(Geo g, const S *__restrict__ src, S *__restrict__ dst,
                                               const S *__restrict__ side)
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

// ---- two steps per sweep (temporal blocking) ----------------------------------------------
//
// The GPU form of the reference's two-steps-per-sweep ("tight") idea (lb.c:442-572).  Each node
// runs pull_node's arithmetic on the same inputs and the intermediate state is kept in the
// storage type, so the result is identical to two single pull steps.
//
// Stale slots: step n+1 reads side parity (n+1)&1 (C_{n-1}); its new values go to the scratch
// slot `side_tmp`, not to that parity, because neighbouring blocks may still read it for their
// halo.  Step n+2 reads and writes parity n&1 for its own nodes only.  launch_pull2_finish then
// moves the scratch into parity (n+1)&1 and swaps the two buffers' ghost rings: the state ends
// in the buffer two single steps would not have left it in, and the read-outs take ghost values
// from the other buffer.
//
// The kernel is a sweep (the shape of the reference's tight variants): a block of W + 2 threads
// owns a strip of W columns and a segment of H rows and walks down it, keeping four rows of C_n
// (W + 4 wide) and three rows of C_{n+1} (W + 2 wide) in shared memory.  Iteration t has C_n row
// YL = y0 - 2 + t (fetched asynchronously during the previous iteration), fetches row YL + 1,
// computes C_{n+1} on row YL - 1 (W + 2 nodes: one a thread) and C_{n+2} on row YL - 2, which it
// writes.  Halo work is two columns a side and two rows a segment end (a few percent), and the
// shared memory a block needs is small enough for several blocks a SM.
template <class S, int W>
constexpr size_t sweep2_r0_bytes() { return (4 * 9 * (size_t)(W + 4) * sizeof(S) + 15) / 16 * 16; }
template <class S, int W>
constexpr size_t sweep2_smem_bytes() { return sweep2_r0_bytes<S, W>() + 3 * 9 * (size_t)(W + 2) * sizeof(S); }

template <class S, int W, int H, bool RS>
__global__ void __launch_bounds__(W + 2) k_sweep2(Geo g, const S *__restrict__ src, S *__restrict__ dst,
                                             const uint8_t *__restrict__ tag, const double *__restrict__ bc,
                                             double omega, const S *__restrict__ side_a,
                                             S *__restrict__ side_tmp, S *__restrict__ side_b, float sc,
                                             float inv)
{
    constexpr int W0 = W + 4, W1 = W + 2;
    extern __shared__ __align__(16) unsigned char sweep_smem[];
    auto r0 = reinterpret_cast<S (*)[9][W0]>(sweep_smem);                 // C_n rows [4], slot = row mod 4
    auto r1 = reinterpret_cast<S (*)[9][W1]>(sweep_smem + sweep2_r0_bytes<S, W>());   // C_{n+1} rows [3]
    const int x0 = 1 + blockIdx.x * W, y0 = 1 + blockIdx.y * H;
    const int tx = threadIdx.x;
    const int yend = min(y0 + H, g.ly + 1);           // rows y0 .. yend-1 are this block's
    // C_n row YL into ring slot YL mod 4 by asynchronous copies (cp.async; one commit group a row,
    // empty for rows outside the array).  A copy unit is one element of 4 or 8 bytes, or two
    // 2-byte elements from an even k (element x0-2+k of the row sits at an even index then, so
    // the pair is 4-byte aligned); units may cover the row's padding (X = -1 or lx + 2), which is
    // inside the allocation and never read back.
    constexpr int E = sizeof(S) >= 4 ? 1 : 2;
    constexpr unsigned UB = E * sizeof(S);
    auto fetch = [&](int YL) {
        if (YL >= 0 && YL <= g.ly + 1) {
            const int sl = (YL + 4) % 4;
            for (int u = tx; u < W0 / E; u += W + 2) {
                const int k = u * E, X = x0 - 2 + k;
                if (X + E - 1 >= 0 && X <= g.lx + 1) {
                    const long long o = g.idx(X, YL);
#pragma unroll
                    for (int i = 0; i < 9; ++i) {
                        const unsigned d = (unsigned)__cvta_generic_to_shared(&r0[sl][i][k]);
                        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(d), "l"(plane(src, g, i) + o),
                                     "n"(UB) : "memory");
                    }
                }
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    fetch(y0 - 2);
    for (int t = 0; y0 - 2 + t - 2 < yend; ++t) {
        const int YL = y0 - 2 + t;
        // row YL + 1 flies while rows YL - 1 and YL - 2 are computed; its slot held row YL - 3,
        // last read before the previous iteration's second barrier
        fetch(YL + 1);
        asm volatile("cp.async.wait_group 1;" ::: "memory");   // this thread's copies of row YL landed
        __syncthreads();                                      // everyone's
        // step n+1 on row YL - 1, columns x0-1 .. x0+W
        const int Y1 = YL - 1;
        if (Y1 >= y0 - 1 && Y1 >= 1 && Y1 <= g.ly && Y1 <= yend) {
            for (int k = tx; k < W1; k += W + 2) {
                const int X = x0 - 1 + k;
                if (X < 1 || X > g.lx) continue;
                const bool edge = g.perimeter(X, Y1);
                const int p = edge ? g.pidx(X, Y1) : 0;
                typename Work<S>::W f[9];
#pragma unroll
                for (int i = 0; i < 9; ++i) {
                    const int sx = X - cx(i), sy = Y1 - cy(i);
                    f[i] = Work<S>::load(g.interior(sx, sy) ? r0[(sy + 4) % 4][i][sx - x0 + 2]
                                                            : side_a[(size_t)i * g.nper + p], i, inv);
                }
                collide_w<S>(bc, g, tag[g.idx(X, Y1)], X, Y1, f, omega, sc, inv);
                const int sl = (Y1 + 3) % 3;
                const RsNode h = rs_node<S, RS>(g, g.rs_key, X, Y1);
#pragma unroll
                for (int i = 0; i < 9; ++i) r1[sl][i][k] = put<S, RS>(stored_out<S>(g, Y1, i, f[i], sc), i, sc, h);
                if (edge && X >= x0 && X < x0 + W && Y1 >= y0 && Y1 < yend) {
#pragma unroll
                    for (int i = 0; i < 9; ++i)
                        if (!g.interior(X - cx(i), Y1 - cy(i)))
                            side_tmp[(size_t)i * g.nper + p] = put<S, RS>(f[i], i, sc, h);
                }
            }
        }
        __syncthreads();
        // step n+2 on row YL - 2, columns x0 .. x0+W-1, to the other buffer
        const int Y2 = YL - 2;
        const int X = x0 + tx;
        if (tx < W && Y2 >= y0 && Y2 < yend && X <= g.lx) {
            const bool edge = g.perimeter(X, Y2);
            const int p = edge ? g.pidx(X, Y2) : 0;
            typename Work<S>::W f[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                const int sx = X - cx(i), sy = Y2 - cy(i);
                f[i] = Work<S>::load(g.interior(sx, sy) ? r1[(sy + 3) % 3][i][sx - x0 + 1]
                                                        : side_b[(size_t)i * g.nper + p], i, inv);
            }
            const long long o = g.idx(X, Y2);
            collide_w<S>(bc, g, tag[o], X, Y2, f, omega, sc, inv);
            const RsNode h = rs_node<S, RS>(g, g.rs_key2, X, Y2);
#pragma unroll
            for (int i = 0; i < 9; ++i) plane(dst, g, i)[o] = put<S, RS>(stored_out<S>(g, Y2, i, f[i], sc), i, sc, h);
            if (edge) {
#pragma unroll
                for (int i = 0; i < 9; ++i)
                    if (!g.interior(X - cx(i), Y2 - cy(i))) side_b[(size_t)i * g.nper + p] = put<S, RS>(f[i], i, sc, h);
            }
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");   // the last prefetch lands before the block ends
}

// ---- two steps per sweep, register form ---------------------------------------------------
//
// The same two steps as k_sweep2 (same node arithmetic, same stale-slot and scratch handling,
// finished by k_pull2_finish), with both steps kept in registers: each warp owns a strip of
// SW2_OUT = 28 columns and a segment of H rows and walks down it.  Lane l holds column
// X = x0 - 2 + l (x0 - 2 .. x0 + 29); one iteration loads row R of C_n (nine populations of the
// lane's column), shifts directions with c_ix = +-1 one lane across by shuffles, computes step
// n+1 on row R - 1 (lanes 1..30 are valid) and step n+2 on row R - 2 (lanes 2..29, written).  A
// population's row shift c_iy is the walk itself: directions with c_iy = +1 come from the row
// two iterations back, c_iy = 0 from the previous one, c_iy = -1 from the current one, so each
// step holds nine values of the rows behind it.  No shared memory and no block barrier: warps
// are independent, the halo (two columns a side, shared with the neighbouring strips, and two
// rows a segment end) is re-read from L2.
constexpr int SW2_OUT = 28;   // output columns a warp

// Direction groups of the walk (D2Q9 order of lb.c:48-55): c_iy = +1 {2, 5, 6}, 0 {0, 1, 3},
// -1 {4, 7, 8}.
template <class W>
__device__ __forceinline__ W lane_shift(W v, int i)
{
    if (cx(i) == 1) return __shfl_up_sync(0xffffffffu, v, 1);     // from lane - 1
    if (cx(i) == -1) return __shfl_down_sync(0xffffffffu, v, 1);  // from lane + 1
    return v;
}

// One pull step of the walk on row Y at column X of this lane: the gathered populations from the
// held rows (up: c_iy = +1, mid: c_iy = 0) and the current one (cur, already lane-shifted),
// stale slots from `side` on the perimeter; collides into f.
template <class S>
__device__ __forceinline__ void walk_gather(const Geo &g, const typename Work<S>::W up[3],
                                            const typename Work<S>::W mid[3],
                                            const typename Work<S>::W cur[9], const S *__restrict__ side,
                                            float inv, int X, int Y, bool edge, int p,
                                            typename Work<S>::W f[9])
{
    f[2] = up[0]; f[5] = up[1]; f[6] = up[2];
    f[0] = mid[0]; f[1] = mid[1]; f[3] = mid[2];
    f[4] = cur[4]; f[7] = cur[7]; f[8] = cur[8];
    if (edge) {
#pragma unroll
        for (int i = 0; i < 9; ++i)
            if (!g.interior(X - cx(i), Y - cy(i))) f[i] = Work<S>::load(side[(size_t)i * g.nper + p], i, inv);
    }
}

template <class S>
__device__ __forceinline__ void walk_hold(typename Work<S>::W up_next[3], typename Work<S>::W up[3],
                                          typename Work<S>::W mid[3], const typename Work<S>::W cur[9])
{
    up[0] = up_next[0]; up[1] = up_next[1]; up[2] = up_next[2];
    up_next[0] = cur[2]; up_next[1] = cur[5]; up_next[2] = cur[6];
    mid[0] = cur[0]; mid[1] = cur[1]; mid[2] = cur[3];
}

// Rows ahead of the walk prefetched into L2 (0: none), measured on the 16384 x 4096 channel
// (GLUPS of two steps per sweep at 0 / 4 / 8 rows): FP64 29.7 / 38.8 / 33.3, FP32 77.3 / 62.1 / 62.0.
#ifndef LBGPU_SWEEP2W_PF64
#define LBGPU_SWEEP2W_PF64 4
#endif
#ifndef LBGPU_SWEEP2W_PF32
#define LBGPU_SWEEP2W_PF32 0
#endif
template <class S>
constexpr int sweep2w_pf() { return sizeof(S) == 8 ? LBGPU_SWEEP2W_PF64 : (sizeof(S) == 4 ? LBGPU_SWEEP2W_PF32 : 0); }
#ifndef LBGPU_SWEEP2W_MINB64
#define LBGPU_SWEEP2W_MINB64 4    // blocks of 4 warps a SM for FP64 (at most 128 registers)
#endif
#ifndef LBGPU_SWEEP2W_MINB32
#define LBGPU_SWEEP2W_MINB32 6    // FP32 (at most 80 registers)
#endif
template <class S>
constexpr int sweep2w_min_blocks()
{
    return sizeof(S) == 8 ? LBGPU_SWEEP2W_MINB64 : (sizeof(S) == 4 ? LBGPU_SWEEP2W_MINB32 : 5);
}

template <class S, int H, bool RS>
__global__ void __launch_bounds__(128, sweep2w_min_blocks<S>()) k_sweep2w(Geo g, const S *__restrict__ src, S *__restrict__ dst,
                                                 const uint8_t *__restrict__ tag, const double *__restrict__ bc,
                                                 double omega, const S *__restrict__ side_a,
                                                 S *__restrict__ side_tmp, S *__restrict__ side_b, float sc,
                                                 float inv)
{
    using W = typename Work<S>::W;
    const int lane = threadIdx.x & 31;
    const int x0 = 1 + ((int)blockIdx.x * 4 + (int)(threadIdx.x >> 5)) * SW2_OUT;
    if (x0 > g.lx) return;                                 // the whole warp
    const int X = x0 - 2 + lane;
    const int y0 = 1 + (int)blockIdx.y * H;
    const int yend = min(y0 + H, g.ly + 1);                // rows y0 .. yend-1 are this warp's
    const bool col_in = X >= 0 && X <= g.lx + 1;           // a column of the arrays
    const bool x_int = X >= 1 && X <= g.lx;
    const bool own_a = lane >= 2 && lane < 2 + SW2_OUT && x_int;   // owned columns (either step)
    W a_up[3] = {}, a_upn[3] = {}, a_mid[3] = {};          // C_n rows behind the walk
    W b_up[3] = {}, b_upn[3] = {}, b_mid[3] = {};          // C_{n+1} rows behind the walk
    // Row R + 1 is loaded while row R is computed (its values are first used one iteration
    // later), and with sweep2w_pf > 0 lane 0 prefetches into L2 the strip's row that many rows
    // ahead: 32 elements from column x0 - 2, widened to 16-byte boundaries and by 16 bytes,
    // skipped where the segment would pass the row's pitch (every byte inside its plane).
    S raw[9];
    auto fetch = [&](int R) {
        if (col_in && R >= 0 && R <= g.ly + 1) {
            const long long o = g.idx(X, R);
#pragma unroll
            for (int i = 0; i < 9; ++i) raw[i] = plane(src, g, i)[o];
        } else {
#pragma unroll
            for (int i = 0; i < 9; ++i) raw[i] = S(0);
        }
    };
    fetch(y0 - 2);
    for (int R = y0 - 2; R <= yend + 1; ++R) {
        // C_n row R, lane-shifted
        W cur[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) cur[i] = Work<S>::load(raw[i], i, inv);
        fetch(R + 1);
        if (sweep2w_pf<S>() > 0 && lane == 0) {
            const int Rp = R + 1 + sweep2w_pf<S>();
            constexpr int EB = (int)sizeof(S);
            const long long e0 = g.idx(x0 - 2, Rp);                       // element of column x0 - 2
            const long long b0 = (e0 * EB) & ~15LL, b1 = ((e0 + 32) * EB + 31) & ~15LL;
            if (Rp <= g.ly + 1 && b1 <= ((long long)Rp + 1) * g.pitch * EB)
#pragma unroll
                for (int i = 0; i < 9; ++i)
                    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(
                                     reinterpret_cast<const char *>(plane(src, g, i)) + b0),
                                 "r"((unsigned)(b1 - b0)) : "memory");
        }
#pragma unroll
        for (int i = 0; i < 9; ++i) cur[i] = lane_shift(cur[i], i);
        // step n+1 on row Y1 = R - 1: its C_{n+1} values in the storage type, lane-shifted
        const int Y1 = R - 1;
        W nxt[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) nxt[i] = W(0);
        if (R >= y0 && x_int && Y1 >= 1 && Y1 <= g.ly) {
            const bool edge = g.perimeter(X, Y1);
            const int p = edge ? g.pidx(X, Y1) : 0;
            W f[9];
            walk_gather<S>(g, a_up, a_mid, cur, side_a, inv, X, Y1, edge, p, f);
            collide_w<S>(bc, g, tag[g.idx(X, Y1)], X, Y1, f, omega, sc, inv);
            const RsNode h = rs_node<S, RS>(g, g.rs_key, X, Y1);
#pragma unroll
            for (int i = 0; i < 9; ++i)
                nxt[i] = Work<S>::load(put<S, RS>(stored_out<S>(g, Y1, i, f[i], sc), i, sc, h), i, inv);
            if (edge && own_a && lane < 2 + SW2_OUT && Y1 >= y0 && Y1 < yend) {
#pragma unroll
                for (int i = 0; i < 9; ++i)
                    if (!g.interior(X - cx(i), Y1 - cy(i)))
                        side_tmp[(size_t)i * g.nper + p] = put<S, RS>(f[i], i, sc, h);
            }
        }
        walk_hold<S>(a_upn, a_up, a_mid, cur);
#pragma unroll
        for (int i = 0; i < 9; ++i) nxt[i] = lane_shift(nxt[i], i);
        // step n+2 on row Y2 = R - 2, written for the owned columns
        const int Y2 = R - 2;
        if (R >= y0 + 2 && own_a && Y2 < yend) {
            const bool edge = g.perimeter(X, Y2);
            const int p = edge ? g.pidx(X, Y2) : 0;
            W f[9];
            walk_gather<S>(g, b_up, b_mid, nxt, side_b, inv, X, Y2, edge, p, f);
            const long long o = g.idx(X, Y2);
            collide_w<S>(bc, g, tag[o], X, Y2, f, omega, sc, inv);
            const RsNode h = rs_node<S, RS>(g, g.rs_key2, X, Y2);
#pragma unroll
            for (int i = 0; i < 9; ++i) plane(dst, g, i)[o] = put<S, RS>(stored_out<S>(g, Y2, i, f[i], sc), i, sc, h);
            if (edge) {
#pragma unroll
                for (int i = 0; i < 9; ++i)
                    if (!g.interior(X - cx(i), Y2 - cy(i))) side_b[(size_t)i * g.nper + p] = put<S, RS>(f[i], i, sc, h);
            }
        }
        walk_hold<S>(b_upn, b_up, b_mid, nxt);
    }
}

// After k_sweep2: the scratch stale slots into parity (n+1)&1, and the ghost rings of the two
// buffers exchanged (one thread per perimeter node and per ghost-ring node).
template <class S>
__global__ void k_pull2_finish(Geo g, S *__restrict__ b0, S *__restrict__ b1, const S *__restrict__ side_tmp,
                               S *__restrict__ side_a)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < g.nper) {
#pragma unroll
        for (int i = 0; i < 9; ++i) side_a[(size_t)i * g.nper + k] = side_tmp[(size_t)i * g.nper + k];
    }
    const int ng = g.nghost();
    if (k < ng) {
        int X, Y;
        if (k < g.lx + 2) { X = k; Y = 0; }
        else if (k < 2 * (g.lx + 2)) { X = k - (g.lx + 2); Y = g.ly + 1; }
        else if (k < 2 * (g.lx + 2) + g.ly) { X = 0; Y = k - 2 * (g.lx + 2) + 1; }
        else { X = g.lx + 1; Y = k - 2 * (g.lx + 2) - g.ly + 1; }
        const long long o = g.idx(X, Y);
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            const S t = plane(b0, g, i)[o];
            plane(b0, g, i)[o] = plane(b1, g, i)[o];
            plane(b1, g, i)[o] = t;
        }
    }
}

// ---- AA scheme ----------------------------------------------------------------------------

// Even step at node (X, Y): own natural slots (stale ones from the side store) -> collide ->
// own opposite slots.
template <class S, int SH = 2, bool RS = false>
__device__ __forceinline__ void aa_even_node(const Geo &g, S *__restrict__ a, const uint8_t *__restrict__ tag,
                                             const double *__restrict__ bc, double omega,
                                             S *__restrict__ side, float sc, float inv, int X, int Y, unsigned key = 0u)
{
    const long long o = g.idx(X, Y);
    const bool edge = g.perimeter(X, Y);
    const int p = edge ? g.pidx(X, Y) : 0;
    typename Work<S>::W f[9];
    if (!edge) {   // the nine loads back to back (a per-slot address choice serialises them)
#pragma unroll
        for (int i = 0; i < 9; ++i) f[i] = Work<S>::load(plane(a, g, i)[o], i, inv);
    } else {
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            const bool stale = !g.interior(X - cx(i), Y - cy(i));
            f[i] = Work<S>::load(stale ? side[(size_t)i * g.nper + p] : plane(a, g, i)[o], i, inv);
        }
    }
    collide_w<S, SH>(bc, g, tag[o], X, Y, f, omega, sc, inv);
    const RsNode h = rs_node<S, RS>(g, key, X, Y);
#pragma unroll
    for (int i = 0; i < 9; ++i) plane(a, g, opp(i))[o] = put<S, RS>(stored_out<S, SH>(g, Y, i, f[i], sc), i, sc, h);
    if (edge) {
#pragma unroll
        for (int i = 0; i < 9; ++i)
            if (!g.interior(X - cx(i), Y - cy(i))) side[(size_t)i * g.nper + p] = put<S, RS>(f[i], i, sc, h);
    }
}

// Odd step at node (X, Y): gather direction i from the source neighbour's opposite slot (stale
// slots from the side store) -> collide -> scatter direction i to the destination neighbour's
// natural slot.  Slot A[i][x + c_i] is read (as opp of the neighbour's gather) and written by
// the same thread, so the in-place update is race-free.  Destinations in the ghost ring are
// written too, so the natural form carries the values streamed out of the lattice.
template <class S, int SH = 2, bool RS = false>
__device__ __forceinline__ void aa_odd_node(const Geo &g, S *__restrict__ a, const uint8_t *__restrict__ tag,
                                            const double *__restrict__ bc, double omega,
                                            S *__restrict__ side, float sc, float inv, int X, int Y, unsigned key = 0u)
{
    const long long o = g.idx(X, Y);
    const bool edge = g.perimeter(X, Y);
    const int p = edge ? g.pidx(X, Y) : 0;
    typename Work<S>::W f[9];
    if (!edge) {
#pragma unroll
        for (int i = 0; i < 9; ++i)
            f[i] = Work<S>::load(plane(a, g, opp(i))[o - cx(i) - (long long)cy(i) * g.pitch], i, inv);
    } else {
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            const int sx = X - cx(i), sy = Y - cy(i);
            f[i] = Work<S>::load(g.interior(sx, sy) ? plane(a, g, opp(i))[g.idx(sx, sy)]
                                                    : side[(size_t)i * g.nper + p], i, inv);
        }
    }
    collide_w<S, SH>(bc, g, tag[o], X, Y, f, omega, sc, inv);
    const RsNode h = rs_node<S, RS>(g, key, X, Y);
#pragma unroll
    for (int i = 0; i < 9; ++i)
        plane(a, g, i)[o + cx(i) + (long long)cy(i) * g.pitch] = put<S, RS>(stored_out<S, SH>(g, Y, i, f[i], sc), i, sc, h);
    if (edge) {
#pragma unroll
        for (int i = 0; i < 9; ++i)
            if (!g.interior(X - cx(i), Y - cy(i))) side[(size_t)i * g.nper + p] = put<S, RS>(f[i], i, sc, h);
    }
}

template <class S>
__global__ void __launch_bounds__(BX) k_aa_even(Geo g, S *__restrict__ a,
                                                const uint8_t *__restrict__ tag,
                                                const double *__restrict__ bc, double omega,
                                                S *__restrict__ side, float sc, float inv)
{
    const int X = blockIdx.x * BX + threadIdx.x + 1;
    const int Y = blockIdx.y + 1;
    if (pf_rows_aa_wide<S>() > 0 && threadIdx.x == 0)
        prefetch_rows_l2<S, BX, 1>(g, a, 1 + BX * (int)blockIdx.x, Y + pf_rows_aa_wide<S>(),
                                   tag);
    if (X <= g.lx) aa_even_node<S>(g, a, tag, bc, omega, side, sc, inv, X, Y);
}

template <class S>
__global__ void __launch_bounds__(BX) k_aa_odd(Geo g, S *__restrict__ a,
                                               const uint8_t *__restrict__ tag,
                                               const double *__restrict__ bc, double omega,
                                               S *__restrict__ side, float sc, float inv)
{
    const int X = blockIdx.x * BX + threadIdx.x + 1;
    const int Y = blockIdx.y + 1;
    if (pf_rows_aa_wide<S>() > 0 && threadIdx.x == 0)
        prefetch_rows_l2<S, BX, 2>(g, a, 1 + BX * (int)blockIdx.x, Y + pf_rows_aa_wide<S>(),
                                   tag);
    if (X <= g.lx) aa_odd_node<S>(g, a, tag, bc, omega, side, sc, inv, X, Y);
}

// AA steps for 16-bit storage, four nodes per thread (the layout of pull_quad: x0 = 1 mod 4,
// each warp one row of 128 nodes; warps touching the perimeter or the row's end run the
// per-node functions).  Even step: the quad's natural slots in, its opposite slots out, both
// aligned.  Odd step: sources gathered as in pull_quad; the scatter to x + c_i shifts the quad by
// one element, so for c_ix = +-1 the aligned word pair is assembled from the neighbouring lane's
// value (one shuffle), and the element that belongs to the next (previous) warp is written by
// its own lane with a 2-byte store.  Every slot is read only by the node whose result is written
// into it (aa_odd_node), and each lane has consumed its loads before the shuffles that precede
// the stores, so the in-place update stays race-free.
template <class S, bool SHIFT>
__device__ __forceinline__ bool aa_quad_vec(const Geo &g, int x0, int Y, int lane)
{
    const int xw0 = x0 - 4 * lane;
    return (xw0 >= 2) && (xw0 + 127 <= g.lx - 1) && (Y >= 2) && (Y <= g.ly - 1);
}

template <class S, bool SHIFT>
__device__ __forceinline__ void aa_collide_quad(const Geo &g, const uint8_t *__restrict__ tag,
                                                const double *__restrict__ bc, double omega, float sc,
                                                float inv, int x0, int Y, long long o, float D[4][9])
{
    const unsigned tq = *reinterpret_cast<const unsigned *>(tag + o);
    if (tq == 0x01010101u) {
        const float om = (float)omega;
        const float us = SHIFT ? g.shift_u[Y] : 0.0f;
#pragma unroll
        for (int k = 0; k < 4; ++k) bgk_offsets<SHIFT>(D[k], om, sc, inv, us);
    } else {
#pragma unroll
        for (int k = 0; k < 4; ++k)
            collide_w<S, SHIFT ? 1 : 0>(bc, g, (int)((tq >> (8 * k)) & 0xff), x0 + k, Y, D[k], omega, sc, inv);
    }
    if (SHIFT && g.shift_rebased(Y)) {
#pragma unroll
        for (int i = 0; i < 9; ++i)
#pragma unroll
            for (int k = 0; k < 4; ++k) D[k][i] = stored_out<S, 1>(g, Y, i, D[k][i], sc);
    }
}

template <class S, bool SHIFT, bool RS>
__global__ void __launch_bounds__(BX, SHIFT ? 7 : 8) k_aa4_even(Geo g, S *__restrict__ a, const uint8_t *__restrict__ tag,
                                                  const double *__restrict__ bc, double omega,
                                                  S *__restrict__ side, float sc, float inv)
{
    using H = Half2Ops<S>;
    const int x0 = 1 + 4 * (blockIdx.x * BX + threadIdx.x), Y = blockIdx.y + 1, lane = threadIdx.x & 31;
    if (LBGPU_PF_ROWS_AA > 0 && threadIdx.x == 0)
        prefetch_rows_l2<S, 4 * BX, 1>(g, a, 1 + 4 * BX * (int)blockIdx.x, Y + LBGPU_PF_ROWS_AA,
                                       tag);
    const unsigned key = g.rs_key;
    if (!aa_quad_vec<S, SHIFT>(g, x0, Y, lane)) {
        for (int k = 0; k < 4; ++k)
            if (x0 + k <= g.lx) aa_even_node<S, SHIFT ? 1 : 0, RS>(g, a, tag, bc, omega, side, sc, inv, x0 + k, Y, key);
        return;
    }
    const long long o = g.idx(x0, Y);
    float D[4][9];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const uint2 v = *reinterpret_cast<const uint2 *>(plane(a, g, i) + o);
        D[0][i] = H::lo(v.x); D[1][i] = H::hi(v.x);
        D[2][i] = H::lo(v.y); D[3][i] = H::hi(v.y);
    }
    aa_collide_quad<S, SHIFT>(g, tag, bc, omega, sc, inv, x0, Y, o, D);
    const unsigned hq = quad_hash<S, RS>(g, key, x0, Y);
#pragma unroll
    for (int i = 0; i < 9; ++i) *reinterpret_cast<uint2 *>(plane(a, g, opp(i)) + o) = pack_quad<S, RS>(D, i, hq);
}

#ifndef LBGPU_AA4_ODD_MINB
#define LBGPU_AA4_ODD_MINB 7        // resident blocks of the odd AA step (72 registers)
#endif
template <class S, bool SHIFT, bool RS>
__global__ void __launch_bounds__(BX, SHIFT ? LBGPU_AA4_ODD_MINB - 1 : LBGPU_AA4_ODD_MINB) k_aa4_odd(Geo g, S *__restrict__ a, const uint8_t *__restrict__ tag,
                                                 const double *__restrict__ bc, double omega,
                                                 S *__restrict__ side, float sc, float inv)
{
    using H = Half2Ops<S>;
    const int x0 = 1 + 4 * (blockIdx.x * BX + threadIdx.x), Y = blockIdx.y + 1, lane = threadIdx.x & 31;
    if (LBGPU_PF_ROWS_AA > 0 && threadIdx.x == 0)
        prefetch_rows_l2<S, 4 * BX, 2>(g, a, 1 + 4 * BX * (int)blockIdx.x, Y + LBGPU_PF_ROWS_AA,
                                       tag);
    const unsigned key = g.rs_key;
    if (!aa_quad_vec<S, SHIFT>(g, x0, Y, lane)) {
        for (int k = 0; k < 4; ++k)
            if (x0 + k <= g.lx) aa_odd_node<S, SHIFT ? 1 : 0, RS>(g, a, tag, bc, omega, side, sc, inv, x0 + k, Y, key);
        return;
    }
    const long long o = g.idx(x0, Y);
    float D[4][9];
#pragma unroll
    for (int i = 0; i < 9; ++i) {   // direction i gathered from the opposite slots of x - c_i
        const S *row = plane(a, g, opp(i)) + (o - (long long)cy(i) * g.pitch);
        const uint2 v = *reinterpret_cast<const uint2 *>(row);
        unsigned w0 = v.x, w1 = v.y;
        if (cx(i) == 1) {            // sources x0-1..x0+2
            const unsigned e = *reinterpret_cast<const unsigned *>(row - 2);
            const unsigned n0 = __byte_perm(e, w0, 0x5432), n1 = __byte_perm(w0, w1, 0x5432);
            w0 = n0; w1 = n1;
        } else if (cx(i) == -1) {    // sources x0+1..x0+4
            const unsigned e = *reinterpret_cast<const unsigned *>(row + 4);
            const unsigned n0 = __byte_perm(w0, w1, 0x5432), n1 = __byte_perm(w1, e, 0x5432);
            w0 = n0; w1 = n1;
        }
        D[0][i] = H::lo(w0); D[1][i] = H::hi(w0);
        D[2][i] = H::lo(w1); D[3][i] = H::hi(w1);
    }
    aa_collide_quad<S, SHIFT>(g, tag, bc, omega, sc, inv, x0, Y, o, D);
    const unsigned hw = quad_hash<S, RS>(g, key, x0, Y);
#pragma unroll
    for (int i = 0; i < 9; ++i) {    // direction i scattered to the natural slots of x + c_i
        const uint2 wq = pack_quad<S, RS>(D, i, hw);
        const unsigned w0 = wq.x, w1 = wq.y;
        S *drow = plane(a, g, i) + (o + (long long)cy(i) * g.pitch);
        unsigned short *h = reinterpret_cast<unsigned short *>(drow);
        if (cx(i) == 0) {
            *reinterpret_cast<uint2 *>(drow) = make_uint2(w0, w1);
        } else if (cx(i) == 1) {     // positions x0..x0+3 take nodes x0-1 (previous lane), x0, x0+1, x0+2
            const unsigned pw = __shfl_up_sync(0xffffffffu, w1, 1);
            const unsigned n0 = __byte_perm(pw, w0, 0x5432), n1 = __byte_perm(w0, w1, 0x5432);
            if (lane != 0) {
                *reinterpret_cast<uint2 *>(drow) = make_uint2(n0, n1);
            } else {                 // position x0 belongs to the previous warp's last lane
                h[1] = (unsigned short)(w0 & 0xffffu);
                *reinterpret_cast<unsigned *>(drow + 2) = n1;
            }
            if (lane == 31) h[4] = (unsigned short)(w1 >> 16);
        } else {                     // positions x0..x0+3 take nodes x0+1, x0+2, x0+3, x0+4 (next lane)
            const unsigned nw = __shfl_down_sync(0xffffffffu, w0, 1);
            const unsigned n0 = __byte_perm(w0, w1, 0x5432), n1 = __byte_perm(w1, nw, 0x5432);
            if (lane != 31) {
                *reinterpret_cast<uint2 *>(drow) = make_uint2(n0, n1);
            } else {                 // position x0+3 belongs to the next warp's first lane
                *reinterpret_cast<unsigned *>(drow) = n0;
                h[2] = (unsigned short)(w1 >> 16);
            }
            if (lane == 0) h[-1] = (unsigned short)(w0 & 0xffffu);
        }
    }
}

// ---- many lattices in one launch ----------------------------------------------------------
//
// One time step of every lattice of a batch: one launch per kind of step (pull, AA even, AA
// odd) over a work list of tiles (lattice, x0, y0, tile width).  A tile is BT nodes, one per
// thread of a BT-thread block (BT = 128, 256 or 512): 32 << shape nodes wide and BT / width
// rows high.  The launch is either persistent (a grid of blocks-per-SM x SMs blocks strides
// through the list) or one block per tile.  A lattice's buffers and parities at step k of a
// chunk follow from its state at the chunk's start (BatchInst), so a CUDA graph of the chunk's
// launches replays unchanged.  Each node runs the same function as the single-lattice kernels,
// so a lattice's result is the same in the batch and alone.
//
// One node per thread is deliberate: a loop over several nodes per thread lets the compiler keep
// the nine source and nine destination plane addresses live across iterations, which doubled the
// registers per thread (and halved the resident warps) of the loop form.  Larger tiles instead
// spread the two dependent descriptor loads at the start of a tile over more nodes.  The kernel
// is bound by memory latency at the occupancy its registers allow (ncu, FP32 pull list: 62 % of
// warps active at 40 registers before the cap, 84 % at 32 with it, against 86 % for the
// single-lattice pull kernel), so the minimum blocks per SM below cap the registers as far as
// that costs no (or a few bytes of) spills: 2048 threads a SM leave 32 registers a thread, 1280
// leave 48, 1024 leave 64, 768 leave 80.
// The 16-bit quad list: 8 blocks of 128 threads (64 registers, with spills) measured 96.8 GLUPS
// on the 512-channel batch against 95.5 at 6 blocks (80 registers), 88.5 at 5 and 79.4 at 4
// (127 registers, no spills): occupancy beats the spills here.
#ifndef LBGPU_PULL4_MINB
#define LBGPU_PULL4_MINB 8
#endif
template <class S, int KIND, bool PERSIST, int BT>
constexpr int batch_min_blocks()
{
    int b128 = 0;   // blocks of 128 threads
    if (sizeof(S) == 8) b128 = KIND == BATCH_PULL ? (PERSIST ? 6 : 10) : (KIND == BATCH_AA_EVEN ? 6 : 5);
    else if (KIND == BATCH_PULL) b128 = PERSIST ? 8 : 16;
    else if (KIND == BATCH_AA_EVEN) b128 = PERSIST ? 8 : 10;
    else if (KIND == BATCH_PULL4) b128 = LBGPU_PULL4_MINB;
    else if (KIND == BATCH_PERIM) b128 = 8;
    else b128 = (sizeof(S) == 4 && !PERSIST) ? 6 : 8;
    return b128 * 128 / BT > 0 ? b128 * 128 / BT : 1;
}

// One strip of tiles (BatchWork): the member's descriptor is read once, then the block walks its
// passes down the lattice; every node runs the single-lattice node function.  With
// LBGPU_BATCH_PF > 0 the rows of the tile that many passes ahead are prefetched into L2 at the
// start of each pass (lane 0 of each warp for the warp's row segment, with prefetch_rows_l2's
// alignment and bounds rules: tile widths and x0 - 1 are multiples of 32 nodes).  Off by
// default: one and two passes ahead measured slower on the 512-channel mix (FP32 60-66 against
// 66-75 GLUPS, FP16 80-100 against 85-97).
#ifndef LBGPU_BATCH_PF
#define LBGPU_BATCH_PF 0
#endif
template <class S, int NW, int ROWS>
__device__ __forceinline__ void batch_prefetch(const Geo &g, const S *src, int x0, int Y, const uint8_t *tag)
{
    if constexpr (LBGPU_BATCH_PF > 0) prefetch_rows_l2<S, NW, ROWS>(g, src, x0, Y, tag);
}

// F: bit 0 -- some member rounds stochastically (RS paths compiled in); bit 1 -- some member
// stores 16-bit offsets with a row shift (the shifted quad path compiled in).  Batches without
// either keep kernels without that code, whose registers it would otherwise raise.
template <class S, int KIND, int BT, int F>
__device__ __forceinline__ void batch_strip(const BatchInst *__restrict__ insts, const BatchWork it, int k)
{
    constexpr bool RS = (F & 1) != 0, SHQ = (F & 2) != 0;
    const BatchInst &d = insts[it.inst];
    const Geo g = d.g;
    const int passes = batch_passes(it.sp);
    S *side = static_cast<S *>(d.side) + (size_t)((d.tau0 + k) & 1) * 9 * (size_t)g.nper;
    const double omega = d.omega;
    const float sc = d.scale, inv = d.inv_scale;
    if constexpr (KIND == BATCH_PULL4) {
        if constexpr (sizeof(S) == 2) {
            // warp w of the block: row y0 + w of each pass, lanes x0 + 4 lane .. x0 + 4 lane + 3
            const int lane = threadIdx.x & 31;
            const int src = d.cur0 ^ (k & 1);
            const S *sb = static_cast<const S *>(d.buf[src]);
            S *db = static_cast<S *>(d.buf[src ^ 1]);
            const int x0 = it.x0 + 4 * lane;
            int Y = it.y0 + (int)(threadIdx.x >> 5);
            const bool rs = RS && d.rs;
            const unsigned key = rs ? rs_key(d.rs_seed, (unsigned long long)(d.tau0 + k)) : 0u;
            for (int p = 0; p < passes && Y <= g.ly; ++p, Y += BT / 32) {   // uniform over the warp
                if (LBGPU_BATCH_PF > 0 && lane == 0 && p + LBGPU_BATCH_PF < passes)
                    batch_prefetch<S, 128, 0>(g, sb, it.x0, Y + LBGPU_BATCH_PF * (BT / 32), d.tag);
                if (RS && rs) {
                    if (SHQ && g.shift_u) pull_quad<S, true, true, true>(g, sb, db, d.tag, d.bc, omega, side, sc, inv, x0, Y, lane, key);
                    else pull_quad<S, false, true, true>(g, sb, db, d.tag, d.bc, omega, side, sc, inv, x0, Y, lane, key);
                } else if (SHQ && g.shift_u) {
                    pull_quad<S, true, false, true>(g, sb, db, d.tag, d.bc, omega, side, sc, inv, x0, Y, lane);
                } else {
                    pull_quad<S, false, false, true>(g, sb, db, d.tag, d.bc, omega, side, sc, inv, x0, Y, lane);
                }
            }
        }
        return;
    }
    if constexpr (KIND == BATCH_PERIM) {
        if constexpr (sizeof(S) == 2) {
            // a run of BT of the member's perimeter nodes (perim_node numbering)
            const int src = d.cur0 ^ (k & 1);
            const S *sb = static_cast<const S *>(d.buf[src]);
            S *db = static_cast<S *>(d.buf[src ^ 1]);
            const bool rs = RS && d.rs;
            const unsigned key = rs ? rs_key(d.rs_seed, (unsigned long long)(d.tau0 + k)) : 0u;
            {   // perimeter nodes it.x0 .. it.x0 + BT - 1, one a thread
                int X, Y;
                if (!perim_node(g, it.x0 + (int)threadIdx.x, X, Y)) return;
                if (RS && rs) {
                    if (SHQ && g.shift_u) pull_node<S, 1, true>(g, sb, db, d.tag, d.bc, omega, side, sc, inv, X, Y, key);
                    else pull_node<S, 0, true>(g, sb, db, d.tag, d.bc, omega, side, sc, inv, X, Y, key);
                } else if (SHQ && g.shift_u) {
                    pull_node<S, 1>(g, sb, db, d.tag, d.bc, omega, side, sc, inv, X, Y);
                } else {
                    pull_node<S, 0>(g, sb, db, d.tag, d.bc, omega, side, sc, inv, X, Y);
                }
            }
        }
        return;
    }
    const int lw = 5 + batch_shape(it.sp);             // log2 of the tile width
    const int X = it.x0 + (int)(threadIdx.x & ((1u << lw) - 1));
    if (X > g.lx) return;
    const int rows = BT >> lw;
    int Y = it.y0 + (int)(threadIdx.x >> lw);
    if constexpr (RS && sizeof(S) == 2) {
        if (d.rs) {   // the single-lattice arithmetic with the member's collision key
            const unsigned key = rs_key(d.rs_seed, (unsigned long long)(d.tau0 + k));
            for (int p = 0; p < passes && Y <= g.ly; ++p, Y += rows) {
                if (KIND == BATCH_PULL) {
                    const int src = d.cur0 ^ (k & 1);
                    pull_node<S, 2, true>(g, static_cast<const S *>(d.buf[src]), static_cast<S *>(d.buf[src ^ 1]),
                                          d.tag, d.bc, omega, side, sc, inv, X, Y, key);
                } else if (KIND == BATCH_AA_EVEN) {
                    aa_even_node<S, 2, true>(g, static_cast<S *>(d.buf[0]), d.tag, d.bc, omega, side, sc, inv, X, Y, key);
                } else {
                    aa_odd_node<S, 2, true>(g, static_cast<S *>(d.buf[0]), d.tag, d.bc, omega, side, sc, inv, X, Y, key);
                }
            }
            return;
        }
    }
    const bool pf_lane = LBGPU_BATCH_PF > 0 && (threadIdx.x & 31) == 0;   // a warp's 32 nodes
    for (int p = 0; p < passes && Y <= g.ly; ++p, Y += rows) {
        if (LBGPU_BATCH_PF > 0 && pf_lane && p + LBGPU_BATCH_PF < passes) {
            const int Yp = Y + LBGPU_BATCH_PF * rows;
            if (KIND == BATCH_PULL)
                batch_prefetch<S, 32, 0>(g, static_cast<const S *>(d.buf[d.cur0 ^ (k & 1)]), X, Yp, nullptr);
            else if (KIND == BATCH_AA_EVEN)
                batch_prefetch<S, 32, 1>(g, static_cast<const S *>(d.buf[0]), X, Yp, nullptr);
            else
                batch_prefetch<S, 32, 2>(g, static_cast<const S *>(d.buf[0]), X, Yp, nullptr);
        }
        if (KIND == BATCH_PULL) {
            const int src = d.cur0 ^ (k & 1);
            pull_node<S>(g, static_cast<const S *>(d.buf[src]), static_cast<S *>(d.buf[src ^ 1]), d.tag,
                         d.bc, omega, side, sc, inv, X, Y);
        } else if (KIND == BATCH_AA_EVEN) {
            aa_even_node<S>(g, static_cast<S *>(d.buf[0]), d.tag, d.bc, omega, side, sc, inv, X, Y);
        } else {
            aa_odd_node<S>(g, static_cast<S *>(d.buf[0]), d.tag, d.bc, omega, side, sc, inv, X, Y);
        }
    }
}

template <class S, int KIND, bool PERSIST, int BT, int F = 0>
__global__ void __launch_bounds__(BT, (batch_min_blocks<S, KIND, PERSIST, BT>()))
    k_batch(const BatchInst *__restrict__ insts, const BatchWork *__restrict__ work, int nwork, int k)
{
    if (PERSIST) {
        for (int w = blockIdx.x; w < nwork; w += gridDim.x) batch_strip<S, KIND, BT, F>(insts, work[w], k);
    } else if ((int)blockIdx.x < nwork) {
        batch_strip<S, KIND, BT, F>(insts, work[blockIdx.x], k);
    }
}

// ---- side store, read-out, upload ----------------------------------------------------------

// Copy the stale slots of the perimeter nodes of buffer b into a side parity.
template <class S>
__global__ void k_side_from_buf(Geo g, const S *__restrict__ buf, S *__restrict__ side)
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

// Ghost ring of buffer b into the AA scheme's copy of the second buffer's ring.
template <class S>
__global__ void k_ghost_copy(Geo g, const S *__restrict__ buf, S *__restrict__ ring)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int ng = g.nghost();
    if (k >= ng) return;
    int X, Y;
    if (k < g.lx + 2) { X = k; Y = 0; }
    else if (k < 2 * (g.lx + 2)) { X = k - (g.lx + 2); Y = g.ly + 1; }
    else if (k < 2 * (g.lx + 2) + g.ly) { X = 0; Y = k - 2 * (g.lx + 2) + 1; }
    else { X = g.lx + 1; Y = k - 2 * (g.lx + 2) - g.ly + 1; }
#pragma unroll
    for (int i = 0; i < 9; ++i) ring[(size_t)i * ng + k] = plane(buf, g, i)[g.idx(X, Y)];
}

// Current state of columns [X0, X1) (all rows) as FP64 node records of `rs` doubles:
// populations in slots 0..8 and, when `dynp` is given, the host dynamics pointer bits in
// slot 9 (the host Node layout).
template <class S>
__global__ void __launch_bounds__(BX) k_readout(Geo g, int view, const S *__restrict__ cur,
                                                const S *__restrict__ other,
                                                const S *__restrict__ side, int X0, int X1,
                                                double *__restrict__ out, int rs,
                                                const uint64_t *__restrict__ dynp, float inv)
{
    const int Y = blockIdx.x * BX + threadIdx.x;
    const int X = X0 + blockIdx.y;
    if (Y > g.ly + 1 || X >= X1) return;
    const size_t r = ((size_t)(X - X0) * (g.ly + 2) + Y) * rs;
#pragma unroll
    for (int i = 0; i < 9; ++i) out[r + i] = (double)logical(g, view, cur, other, side, X, Y, i, inv);
    if (dynp) out[r + 9] = __longlong_as_double((long long)dynp[(size_t)X * (g.ly + 2) + Y]);
}

// FP64 node records of columns [X0, X1) into buffer b (inverse of k_readout).
template <class S>
__global__ void __launch_bounds__(BX) k_upload(Geo g, const double *__restrict__ in, int rs, int X0,
                                               int X1, int Y0, int H, S *__restrict__ buf, float sc)
{
    const int Y = Y0 + blockIdx.x * BX + threadIdx.x;
    const int X = X0 + blockIdx.y;
    if (Y >= Y0 + H || X >= X1) return;
    const size_t r = ((size_t)(X - X0) * H + (Y - Y0)) * rs;
    const long long o = g.idx(X, Y);
#pragma unroll
    for (int i = 0; i < 9; ++i)
        plane(buf, g, i)[o] = enc_row<S>(g, (typename Codec<S>::R)in[r + i], i, sc, Y);
}

// ---- outlet extrapolation, periodic wrap, initial state, macroscopic fields ---------------

// Density of the post-stream state at columns lx-1 and lx-2 for every row (the inputs of the
// zero-gradient outlet, unsteady.c:205-214 and lb.c:471-480).
template <class S>
__global__ void k_zgb_rho(Geo g, int view, const S *__restrict__ cur, const S *__restrict__ other,
                          const S *__restrict__ side, double *__restrict__ zrho, float inv)
{
    using R = typename Codec<S>::R;
    const int Y = blockIdx.x * blockDim.x + threadIdx.x;
    if (Y > g.ly + 1) return;
    R f[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) f[i] = logical(g, view, cur, other, side, g.lx - 1, Y, i, inv);
    zrho[2 * Y] = (double)rules::density(f);
#pragma unroll
    for (int i = 0; i < 9; ++i) f[i] = logical(g, view, cur, other, side, g.lx - 2, Y, i, inv);
    zrho[2 * Y + 1] = (double)rules::density(f);
}

// Pressure-table slots fed by the extrapolation: rho = 4/3 rho1 - 1/3 rho2, uPar = 0.
__global__ void k_zgb_apply(int nb, const int *__restrict__ zgb_src, const double *__restrict__ zrho,
                            double *__restrict__ bc)
{
    using O = Ar<double>;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= 4 * nb) return;
    const int src = zgb_src[k];
    if (src < 0) return;
    const int tb = 4 + k / nb, c = k % nb;
    bc[(tb * 2 + 0) * nb + c] = O::S(O::M(4. / 3., zrho[2 * src]), O::M(1. / 3., zrho[2 * src + 1]));
    bc[(tb * 2 + 1) * nb + c] = 0.0;
}

// Periodic wrap of buffer b (pull form L): the slots a boundary node would receive from across
// the lattice take the values streamed into the opposite ghost ring (lb.c:1783-1817).  The
// three phases run in the reference's order so that later writes win.
template <class S>
__global__ void k_periodic(Geo g, S *__restrict__ buf)
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
// with y = Y-1, L = ly-1 (unsteady.c:155-159, :169-170), computed in exact FP64 and encoded;
// ghost ring zero (lb.c:62-68).
template <class S>
__global__ void __launch_bounds__(BX) k_init_cylinder(Geo g, S *__restrict__ buf, double umax, float sc)
{
    using O = Ar<double>;
    const int X = blockIdx.x * BX + threadIdx.x;
    const int Y = blockIdx.y;
    if (X > g.lx + 1) return;
    const long long o = g.idx(X, Y);
    double f[9];
    if (g.interior(X, Y)) {
        const double y = (double)(Y - 1), L = (double)(g.ly - 1);
        const double u = O::M(O::D(O::M(4.0, umax), O::M(L, L)), O::S(O::M(L, y), O::M(y, y)));
        rules::equilibrium<double>(f, 1.0, u, 0.0);
#pragma unroll
        for (int i = 0; i < 9; ++i)
            plane(buf, g, i)[o] = enc_row<S>(g, (typename Codec<S>::R)f[i], i, sc, Y);
    } else {
#pragma unroll
        for (int i = 0; i < 9; ++i) plane(buf, g, i)[o] = S(0);
    }
}

// Tag plane of the cylinder channel, the same assignment order as the host builder
// (dynamics_host.c lbgpu_build_cylinder, after unsteady.c:162-199): bulk or obstacle disk,
// then the lower and upper wall rows, then the inlet and outlet columns of rows 2..ly-1.
__global__ void __launch_bounds__(BX) k_cylinder_tags(Geo g, uint8_t *__restrict__ tag, int ox, int oy,
                                                      int r, int lower, int upper)
{
    const int X = blockIdx.x * BX + threadIdx.x;
    const int Y = blockIdx.y;
    if (X > g.lx + 1) return;
    int t = LBGPU_TAG_NONE;
    if (g.interior(X, Y)) {
        const long long dx = X - ox, dy = Y - oy;
        t = dx * dx + dy * dy <= (long long)r * r ? LBGPU_TAG_BOUNCE_BACK : LBGPU_TAG_BGK;
        if (Y == 1) t = lower;
        if (Y == g.ly) t = upper;
        if (Y >= 2 && Y <= g.ly - 1) {
            if (X == 1) t = LBGPU_TAG_LEFT_REGULARIZED;
            if (X == g.lx) t = LBGPU_TAG_RIGHT_PRESSURE_REGULARIZED;
        }
    }
    tag[g.idx(X, Y)] = (uint8_t)t;
}

template <class S>
__global__ void __launch_bounds__(BX) k_macros(Geo g, int view, const S *__restrict__ cur,
                                               const S *__restrict__ other,
                                               const S *__restrict__ side, double *__restrict__ rho,
                                               double *__restrict__ ux, double *__restrict__ uy,
                                               float inv)
{
    using R = typename Codec<S>::R;
    const int X = blockIdx.x * BX + threadIdx.x + 1;
    const int Y = blockIdx.y + 1;
    if (X > g.lx) return;
    R f[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) f[i] = logical(g, view, cur, other, side, X, Y, i, inv);
    R r, u, v;
    rules::macros<R>(f, r, u, v);
    const size_t k = (size_t)(Y - 1) * g.lx + (X - 1);
    if (rho) rho[k] = (double)r;
    if (ux) ux[k] = (double)u;
    if (uy) uy[k] = (double)v;
}

// ---- FP64 reductions of the current state ----------------------------------------------
//
// One block per interior row sums, in a fixed order, eight quantities over the row into
// partial[Y][8]; k_moments_final sums the rows in a fixed order.  Results are bitwise
// reproducible for a given lattice and state.
//   0 mass            sum of rho over every interior node
//   1, 2 momentum     sum of (jx, jy)
//   3, 4 force        momentum exchange on the obstacle: 2 sum c_i f_i over every link that
//                     enters a bounce-back node strictly inside the lattice (rows 2..ly-1,
//                     columns 2..lx-1) from a non-bounce-back node, f_i being the population
//                     that arrived at the solid node this step (full-way bounce-back returns
//                     it reversed: momentum 2 c_i f_i per link and step)
//   5 kinetic energy  sum of |j|^2 / (2 rho) over bulk (BGK) nodes
//   6 non-finite      number of nodes with a NaN or infinite population
//   7 fluid mass      sum of rho over bulk (BGK) nodes
constexpr int RED_THREADS = 256;

template <class S>
__global__ void __launch_bounds__(RED_THREADS) k_moments_rows(Geo g, int view, const S *__restrict__ cur,
                                                              const S *__restrict__ other,
                                                              const S *__restrict__ side,
                                                              const uint8_t *__restrict__ tag,
                                                              double *__restrict__ partial, float inv)
{
    const int Y = blockIdx.x + 1;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int X = 1 + threadIdx.x; X <= g.lx; X += RED_THREADS) {
        double f[9];
        bool bad = false;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            f[i] = (double)logical(g, view, cur, other, side, X, Y, i, inv);
            bad |= !isfinite(f[i]);
        }
        const double rho = ((f[0] + f[1]) + (f[2] + f[3])) + ((f[4] + f[5]) + (f[6] + f[7])) + f[8];
        const double jx = (f[1] - f[3]) + (f[5] - f[6]) + (f[8] - f[7]);
        const double jy = (f[2] - f[4]) + (f[5] - f[8]) + (f[6] - f[7]);
        acc[0] += rho; acc[1] += jx; acc[2] += jy;
        acc[6] += bad ? 1.0 : 0.0;
        const int t = tag[g.idx(X, Y)];
        if (t == TAG_BGK) {
            acc[5] += (jx * jx + jy * jy) / (2.0 * rho);
            acc[7] += rho;
        } else if (t == TAG_BOUNCE && X >= 2 && X <= g.lx - 1 && Y >= 2 && Y <= g.ly - 1) {
#pragma unroll
            for (int i = 1; i < 9; ++i) {
                if (tag[g.idx(X - cx(i), Y - cy(i))] != TAG_BOUNCE) {
                    acc[3] += 2.0 * cx(i) * f[i];
                    acc[4] += 2.0 * cy(i) * f[i];
                }
            }
        }
    }
    __shared__ double red[8][RED_THREADS];
#pragma unroll
    for (int k = 0; k < 8; ++k) red[k][threadIdx.x] = acc[k];
    __syncthreads();
    for (int w = RED_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
#pragma unroll
            for (int k = 0; k < 8; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 8) partial[(size_t)Y * 8 + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void __launch_bounds__(RED_THREADS) k_moments_final(int ly, const double *__restrict__ partial,
                                                               double *__restrict__ out)
{
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int Y = 1 + threadIdx.x; Y <= ly; Y += RED_THREADS)
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] += partial[(size_t)Y * 8 + k];
    __shared__ double red[8][RED_THREADS];
#pragma unroll
    for (int k = 0; k < 8; ++k) red[k][threadIdx.x] = acc[k];
    __syncthreads();
    for (int w = RED_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
#pragma unroll
            for (int k = 0; k < 8; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 8) out[threadIdx.x] = red[threadIdx.x][0];
}

// Running sums of the velocity field (time averages): acc[0][.] += ux, acc[1][.] += uy.
template <class S>
__global__ void __launch_bounds__(BX) k_accumulate_velocity(Geo g, int view, const S *__restrict__ cur,
                                                            const S *__restrict__ other,
                                                            const S *__restrict__ side,
                                                            double *__restrict__ acc, float inv)
{
    const int X = blockIdx.x * BX + threadIdx.x + 1;
    const int Y = blockIdx.y + 1;
    if (X > g.lx) return;
    double f[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) f[i] = (double)logical(g, view, cur, other, side, X, Y, i, inv);
    const double rho = ((f[0] + f[1]) + (f[2] + f[3])) + ((f[4] + f[5]) + (f[6] + f[7])) + f[8];
    const double jx = (f[1] - f[3]) + (f[5] - f[6]) + (f[8] - f[7]);
    const double jy = (f[2] - f[4]) + (f[5] - f[8]) + (f[6] - f[7]);
    const size_t k = (size_t)(Y - 1) * g.lx + (X - 1);
    const size_t n = (size_t)g.lx * g.ly;
    acc[k] += jx / rho;
    acc[n + k] += jy / rho;
}

// Steady-state residual: the largest |u - u_prev| over the interior (u_prev: the velocity at
// the previous check, FP32 pairs, replaced by the current one).  *out holds the bits of a
// non-negative float, so an integer atomicMax orders it; the caller clears it first.
template <class S>
__global__ void __launch_bounds__(BX) k_velocity_change(Geo g, int view, const S *__restrict__ cur,
                                                        const S *__restrict__ other,
                                                        const S *__restrict__ side,
                                                        float2 *__restrict__ prev,
                                                        unsigned *__restrict__ out, float inv)
{
    const int X = blockIdx.x * BX + threadIdx.x + 1;
    const int Y = blockIdx.y + 1;
    float d = 0.0f;
    if (X <= g.lx) {
        double f[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) f[i] = (double)logical(g, view, cur, other, side, X, Y, i, inv);
        const double rho = ((f[0] + f[1]) + (f[2] + f[3])) + ((f[4] + f[5]) + (f[6] + f[7])) + f[8];
        const float ux = (float)(((f[1] - f[3]) + (f[5] - f[6]) + (f[8] - f[7])) / rho);
        const float uy = (float)(((f[2] - f[4]) + (f[5] - f[8]) + (f[6] - f[7])) / rho);
        const size_t k = (size_t)(Y - 1) * g.lx + (X - 1);
        const float2 p = prev[k];
        d = sqrtf((ux - p.x) * (ux - p.x) + (uy - p.y) * (uy - p.y));
        if (!(d == d)) d = 3.0e38f;   // a NaN counts as not converged
        prev[k] = make_float2(ux, uy);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d = fmaxf(d, __shfl_xor_sync(0xffffffffu, d, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(d));
}

inline unsigned cdiv(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

template <class S> S *B(const DevLattice &d, int b) { return static_cast<S *>(d.buf[b]); }
// The `other` argument of logical(): the pull scheme's second buffer, or the AA ring copy.
template <class S> S *OTHER(const DevLattice &d, int cur)
{
    return d.buf[1] ? static_cast<S *>(d.buf[1 - cur]) : static_cast<S *>(d.ghost2);
}
template <class S> S *SIDE(const DevLattice &d, int p)
{
    return static_cast<S *>(d.side) + (size_t)(p & 1) * 9 * (size_t)d.g.nper;
}
// Pull scheme only: the scratch slot after the two parities (see k_sweep2).
template <class S> S *SIDE_TMP(const DevLattice &d)
{
    return static_cast<S *>(d.side) + 2 * 9 * (size_t)d.g.nper;
}

}  // namespace

// Run F<S>() with S the lattice's storage type.
#define LBGPU_DISPATCH(d, BODY)                                        \
    switch ((d).precision) {                                          \
    case LBGPU_F64: { using S = double; BODY; } break;                \
    case LBGPU_F32: { using S = float; BODY; } break;                 \
    case LBGPU_F16: { using S = __half; BODY; } break;                \
    default: { using S = __nv_bfloat16; BODY; } break;                \
    }

void launch_collide_inplace(const DevLattice &d, int cur, int side_par, cudaStream_t s)
{
    dim3 grid(cdiv(d.g.lx, BX), d.g.ly);
    if (d.g.rs_key && d.precision == LBGPU_F16)
        k_collide_inplace<__half, true><<<grid, BX, 0, s>>>(d.g, B<__half>(d, cur), d.tag, d.bc, d.omega,
                                                           SIDE<__half>(d, side_par), d.scale, d.inv_scale);
    else if (d.g.rs_key && d.precision == LBGPU_BF16)
        k_collide_inplace<__nv_bfloat16, true><<<grid, BX, 0, s>>>(d.g, B<__nv_bfloat16>(d, cur), d.tag, d.bc,
                                                                  d.omega, SIDE<__nv_bfloat16>(d, side_par),
                                                                  d.scale, d.inv_scale);
    else
        LBGPU_DISPATCH(d, (k_collide_inplace<S, false><<<grid, BX, 0, s>>>(d.g, B<S>(d, cur), d.tag, d.bc,
                           d.omega, SIDE<S>(d, side_par), d.scale, d.inv_scale)));
}

template <class S, bool SHIFT, bool RS>
static void launch_pull4h_t(const DevLattice &d, dim3 grid, int src, int side_par, cudaStream_t s)
{
    if (!pull4h_perim_apart<SHIFT>()) {
        k_pull4h<S, SHIFT, RS><<<grid, BX, 0, s>>>(d.g, B<S>(d, src), B<S>(d, 1 - src), d.tag, d.bc, d.omega,
                                                   SIDE<S>(d, side_par), d.scale, d.inv_scale);
        return;
    }
    // the perimeter as extra grid rows of the same launch where CUDA's 65535 grid rows allow,
    // else as a launch of its own after the quads
    const int pblocks = cdiv(2 * d.g.lx + 2 * d.g.ly, BX);
    const int prows = cdiv(pblocks, (int)grid.x);
    if ((long long)grid.y + prows <= 65535) {
        dim3 g2(grid.x, grid.y + prows);
        k_pull4h<S, SHIFT, RS, true, true><<<g2, BX, 0, s>>>(d.g, B<S>(d, src), B<S>(d, 1 - src), d.tag, d.bc,
                                                             d.omega, SIDE<S>(d, side_par), d.scale, d.inv_scale);
    } else {
        k_pull4h<S, SHIFT, RS, true, false><<<grid, BX, 0, s>>>(d.g, B<S>(d, src), B<S>(d, 1 - src), d.tag, d.bc,
                                                                d.omega, SIDE<S>(d, side_par), d.scale, d.inv_scale);
        k_perim_pull<S, SHIFT ? 1 : 0, RS><<<cdiv(2 * d.g.lx + 2 * d.g.ly, 256), 256, 0, s>>>(
            d.g, B<S>(d, src), B<S>(d, 1 - src), d.tag, d.bc, d.omega, SIDE<S>(d, side_par), d.scale, d.inv_scale);
    }
}

template <class S>
static void launch_pull4h(const DevLattice &d, dim3 grid, int src, int side_par, cudaStream_t s)
{
    if (d.g.shift_u) {
        if (d.g.rs_key) launch_pull4h_t<S, true, true>(d, grid, src, side_par, s);
        else launch_pull4h_t<S, true, false>(d, grid, src, side_par, s);
    } else {
        if (d.g.rs_key) launch_pull4h_t<S, false, true>(d, grid, src, side_par, s);
        else launch_pull4h_t<S, false, false>(d, grid, src, side_par, s);
    }
}

int pull_launches(const DevLattice &d, bool ghosts)
{
    const bool half = d.precision == LBGPU_F16 || d.precision == LBGPU_BF16;
    const bool apart = d.g.shift_u ? pull4h_perim_apart<true>() : pull4h_perim_apart<false>();
    if (ghosts || !half || !apart) return 1;
    const int gx = cdiv((d.g.lx + 3) / 4, BX);
    const int prows = cdiv(cdiv(2 * d.g.lx + 2 * d.g.ly, BX), gx);
    return (long long)d.g.ly + prows <= 65535 ? 1 : 2;
}

void launch_pull(const DevLattice &d, int src, int side_par, bool ghosts, cudaStream_t s)
{
    if (ghosts) {
        dim3 grid(cdiv(d.g.lx + 1, BX), d.g.ly + 2);
        LBGPU_DISPATCH(d, (k_pull<S, true><<<grid, BX, 0, s>>>(d.g, B<S>(d, src), B<S>(d, 1 - src),
                           d.tag, d.bc, d.omega, SIDE<S>(d, side_par), d.scale, d.inv_scale)));
    } else if (d.precision == LBGPU_F16 || d.precision == LBGPU_BF16) {
        dim3 grid(cdiv((d.g.lx + 3) / 4, BX), d.g.ly);
        if (d.precision == LBGPU_F16) launch_pull4h<__half>(d, grid, src, side_par, s);
        else launch_pull4h<__nv_bfloat16>(d, grid, src, side_par, s);
    } else {
        dim3 grid(cdiv(d.g.lx, BX), d.g.ly);
        LBGPU_DISPATCH(d, (k_pull<S, false><<<grid, BX, 0, s>>>(d.g, B<S>(d, src), B<S>(d, 1 - src),
                           d.tag, d.bc, d.omega, SIDE<S>(d, side_par), d.scale, d.inv_scale)));
    }
}

template <class S, int W, int H, bool RS = false>
static void launch_sweep2_t(const DevLattice &d, int src, int n_par, cudaStream_t s)
{
    constexpr size_t smem = sweep2_smem_bytes<S, W>();
    cudaFuncSetAttribute(k_sweep2<S, W, H, RS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 grid(cdiv(d.g.lx, W), cdiv(d.g.ly, H));
    k_sweep2<S, W, H, RS><<<grid, W + 2, smem, s>>>(d.g, B<S>(d, src), B<S>(d, 1 - src), d.tag, d.bc, d.omega,
                                         SIDE<S>(d, n_par + 1), SIDE_TMP<S>(d), SIDE<S>(d, n_par), d.scale,
                                         d.inv_scale);
}

// The register form (k_sweep2w) of the two-step sweep for the storage types whose bit is set in
// LBGPU_SWEEP2_REG (1 FP64, 2 FP32, 4 FP16 / BF16); the others use the shared-memory form.
// Measured on the 16384 x 4096 channel (GLUPS, register / shared-memory form): FP64 38.8 / 37.4,
// FP32 77.3 / 70.4, FP16 58.1 / 63.0.
#ifndef LBGPU_SWEEP2_REG
#define LBGPU_SWEEP2_REG 3
#endif
#ifndef LBGPU_SWEEP2W_H
#define LBGPU_SWEEP2W_H 128     // rows a warp walks
#endif
template <class S, bool RS = false>
static void launch_sweep2w_t(const DevLattice &d, int src, int n_par, cudaStream_t s)
{
    const int strips = cdiv(d.g.lx, SW2_OUT);
    dim3 grid(cdiv(strips, 4), cdiv(d.g.ly, LBGPU_SWEEP2W_H));
    k_sweep2w<S, LBGPU_SWEEP2W_H, RS><<<grid, 128, 0, s>>>(d.g, B<S>(d, src), B<S>(d, 1 - src), d.tag, d.bc,
                                                          d.omega, SIDE<S>(d, n_par + 1), SIDE_TMP<S>(d),
                                                          SIDE<S>(d, n_par), d.scale, d.inv_scale);
}

void launch_pull2(const DevLattice &d, int src, int n_par, cudaStream_t s)
{
    constexpr bool reg64 = (LBGPU_SWEEP2_REG & 1) != 0, reg32 = (LBGPU_SWEEP2_REG & 2) != 0,
                   reg16 = (LBGPU_SWEEP2_REG & 4) != 0;
    switch (d.precision) {
    case LBGPU_F64:
        if (reg64) launch_sweep2w_t<double>(d, src, n_par, s);
        else launch_sweep2_t<double, 126, 128>(d, src, n_par, s);
        break;
    case LBGPU_F32:
        if (reg32) launch_sweep2w_t<float>(d, src, n_par, s);
        else launch_sweep2_t<float, 126, 128>(d, src, n_par, s);
        break;
    case LBGPU_F16:
        if (reg16) {
            if (d.g.rs_key) launch_sweep2w_t<__half, true>(d, src, n_par, s);
            else launch_sweep2w_t<__half>(d, src, n_par, s);
        } else if (d.g.rs_key) {
            launch_sweep2_t<__half, 126, 128, true>(d, src, n_par, s);
        } else {
            launch_sweep2_t<__half, 126, 128>(d, src, n_par, s);
        }
        break;
    default:
        if (reg16) {
            if (d.g.rs_key) launch_sweep2w_t<__nv_bfloat16, true>(d, src, n_par, s);
            else launch_sweep2w_t<__nv_bfloat16>(d, src, n_par, s);
        } else if (d.g.rs_key) {
            launch_sweep2_t<__nv_bfloat16, 126, 128, true>(d, src, n_par, s);
        } else {
            launch_sweep2_t<__nv_bfloat16, 126, 128>(d, src, n_par, s);
        }
        break;
    }
    const int nthreads = std::max(d.g.nper, d.g.nghost());
    LBGPU_DISPATCH(d, (k_pull2_finish<S><<<cdiv(nthreads, 256), 256, 0, s>>>(d.g, B<S>(d, 0), B<S>(d, 1),
                       SIDE_TMP<S>(d), SIDE<S>(d, n_par + 1))));
}

void launch_stream(const DevLattice &d, int src, int side_par, cudaStream_t s)
{
    dim3 grid(cdiv(d.g.lx + 2, BX), d.g.ly + 2);
    LBGPU_DISPATCH(d, (k_stream<S><<<grid, BX, 0, s>>>(d.g, B<S>(d, src), B<S>(d, 1 - src),
                       SIDE<S>(d, side_par))));
}

template <class S, bool SHIFT, bool RS>
static void launch_aa4_t(const DevLattice &d, bool odd, int side_par, cudaStream_t s)
{
    dim3 grid(cdiv((d.g.lx + 3) / 4, BX), d.g.ly);
    if (odd)
        k_aa4_odd<S, SHIFT, RS><<<grid, BX, 0, s>>>(d.g, B<S>(d, 0), d.tag, d.bc, d.omega,
                                                    SIDE<S>(d, side_par), d.scale, d.inv_scale);
    else
        k_aa4_even<S, SHIFT, RS><<<grid, BX, 0, s>>>(d.g, B<S>(d, 0), d.tag, d.bc, d.omega,
                                                     SIDE<S>(d, side_par), d.scale, d.inv_scale);
}

template <class S>
static void launch_aa4(const DevLattice &d, bool odd, int side_par, cudaStream_t s)
{
    if (d.g.shift_u) {
        if (d.g.rs_key) launch_aa4_t<S, true, true>(d, odd, side_par, s);
        else launch_aa4_t<S, true, false>(d, odd, side_par, s);
    } else {
        if (d.g.rs_key) launch_aa4_t<S, false, true>(d, odd, side_par, s);
        else launch_aa4_t<S, false, false>(d, odd, side_par, s);
    }
}

void launch_aa_even(const DevLattice &d, int side_par, cudaStream_t s)
{
    if (d.precision == LBGPU_F16) return launch_aa4<__half>(d, false, side_par, s);
    if (d.precision == LBGPU_BF16) return launch_aa4<__nv_bfloat16>(d, false, side_par, s);
    dim3 grid(cdiv(d.g.lx, BX), d.g.ly);
    LBGPU_DISPATCH(d, (k_aa_even<S><<<grid, BX, 0, s>>>(d.g, B<S>(d, 0), d.tag, d.bc, d.omega,
                       SIDE<S>(d, side_par), d.scale, d.inv_scale)));
}

void launch_aa_odd(const DevLattice &d, int side_par, cudaStream_t s)
{
    if (d.precision == LBGPU_F16) return launch_aa4<__half>(d, true, side_par, s);
    if (d.precision == LBGPU_BF16) return launch_aa4<__nv_bfloat16>(d, true, side_par, s);
    dim3 grid(cdiv(d.g.lx, BX), d.g.ly);
    LBGPU_DISPATCH(d, (k_aa_odd<S><<<grid, BX, 0, s>>>(d.g, B<S>(d, 0), d.tag, d.bc, d.omega,
                       SIDE<S>(d, side_par), d.scale, d.inv_scale)));
}

template <class S, int KIND, int BT, int F>
static void launch_batch_r(bool persistent, const BatchInst *insts, const BatchWork *work, int nwork, int grid,
                           int k, cudaStream_t s)
{
    if (persistent) k_batch<S, KIND, true, BT, F><<<grid, BT, 0, s>>>(insts, work, nwork, k);
    else k_batch<S, KIND, false, BT, F><<<grid, BT, 0, s>>>(insts, work, nwork, k);
}

// flags: bit 0 stochastic rounding, bit 1 row shift (kernels.h launch_batch); the shift matters
// to the quad kind only.
template <class S, int KIND, int BT>
static void launch_batch_b(bool persistent, int flags, const BatchInst *insts, const BatchWork *work, int nwork,
                           int grid, int k, cudaStream_t s)
{
    if constexpr (sizeof(S) == 2) {
        const int f = (KIND == BATCH_PULL4 || KIND == BATCH_PERIM) ? (flags & 3) : (flags & 1);
        if (f == 1) return launch_batch_r<S, KIND, BT, 1>(persistent, insts, work, nwork, grid, k, s);
        if constexpr (KIND == BATCH_PULL4 || KIND == BATCH_PERIM) {
            if (f == 2) return launch_batch_r<S, KIND, BT, 2>(persistent, insts, work, nwork, grid, k, s);
            if (f == 3) return launch_batch_r<S, KIND, BT, 3>(persistent, insts, work, nwork, grid, k, s);
        }
    }
    launch_batch_r<S, KIND, BT, 0>(persistent, insts, work, nwork, grid, k, s);
}

template <class S, int KIND>
static void launch_batch_k(int bt, bool persistent, int rs, const BatchInst *insts, const BatchWork *work,
                           int nwork, int grid, int k, cudaStream_t s)
{
    if (bt == 512) launch_batch_b<S, KIND, 512>(persistent, rs, insts, work, nwork, grid, k, s);
    else if (bt == 256) launch_batch_b<S, KIND, 256>(persistent, rs, insts, work, nwork, grid, k, s);
    else launch_batch_b<S, KIND, 128>(persistent, rs, insts, work, nwork, grid, k, s);
}

template <class S>
static void launch_batch_t(int kind, int bt, bool persistent, int rs, const BatchInst *insts,
                           const BatchWork *work, int nwork, int grid, int k, cudaStream_t s)
{
    if (kind == BATCH_PULL) launch_batch_k<S, BATCH_PULL>(bt, persistent, rs, insts, work, nwork, grid, k, s);
    else if (kind == BATCH_AA_EVEN)
        launch_batch_k<S, BATCH_AA_EVEN>(bt, persistent, rs, insts, work, nwork, grid, k, s);
    else if (kind == BATCH_AA_ODD)
        launch_batch_k<S, BATCH_AA_ODD>(bt, persistent, rs, insts, work, nwork, grid, k, s);
    else if constexpr (sizeof(S) == 2) {
        if (kind == BATCH_PULL4) launch_batch_k<S, BATCH_PULL4>(bt, persistent, rs, insts, work, nwork, grid, k, s);
        else launch_batch_k<S, BATCH_PERIM>(bt, persistent, rs, insts, work, nwork, grid, k, s);
    }
}

void launch_batch(int precision, int kind, int threads, bool persistent, int rs, const BatchInst *insts,
                  const BatchWork *work, int nwork, int grid, int k, cudaStream_t s)
{
    switch (precision) {
    case LBGPU_F64: launch_batch_t<double>(kind, threads, persistent, 0, insts, work, nwork, grid, k, s); break;
    case LBGPU_F32: launch_batch_t<float>(kind, threads, persistent, 0, insts, work, nwork, grid, k, s); break;
    case LBGPU_F16: launch_batch_t<__half>(kind, threads, persistent, rs, insts, work, nwork, grid, k, s); break;
    default: launch_batch_t<__nv_bfloat16>(kind, threads, persistent, rs, insts, work, nwork, grid, k, s); break;
    }
}

template <class S, int KIND>
static int blocks_k(int bt)
{
    int n = 0;
    if (bt == 512) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch<S, KIND, true, 512>, 512, 0);
    else if (bt == 256) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch<S, KIND, true, 256>, 256, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch<S, KIND, true, 128>, 128, 0);
    return n;
}

template <class S>
static int blocks_t(int kind, int bt)
{
    if (kind == BATCH_PULL) return blocks_k<S, BATCH_PULL>(bt);
    if (kind == BATCH_AA_EVEN) return blocks_k<S, BATCH_AA_EVEN>(bt);
    if (kind == BATCH_AA_ODD) return blocks_k<S, BATCH_AA_ODD>(bt);
    if constexpr (sizeof(S) == 2) {
        if (kind == BATCH_PULL4) return blocks_k<S, BATCH_PULL4>(bt);
        return blocks_k<S, BATCH_PERIM>(bt);
    }
    return 0;
}

int batch_blocks_per_sm(int precision, int kind, int threads)
{
    switch (precision) {
    case LBGPU_F64: return blocks_t<double>(kind, threads);
    case LBGPU_F32: return blocks_t<float>(kind, threads);
    case LBGPU_F16: return blocks_t<__half>(kind, threads);
    default: return blocks_t<__nv_bfloat16>(kind, threads);
    }
}

void launch_side_from_buf(const DevLattice &d, int b, int side_par, cudaStream_t s)
{
    const int n = 2 * d.g.lx + (d.g.ly > 2 ? 2 * (d.g.ly - 2) : 0);
    LBGPU_DISPATCH(d, (k_side_from_buf<S><<<cdiv(n, 256), 256, 0, s>>>(d.g, B<S>(d, b),
                       SIDE<S>(d, side_par))));
}

void launch_ghost_copy(const DevLattice &d, int b, cudaStream_t s)
{
    if (!d.ghost2) return;
    LBGPU_DISPATCH(d, (k_ghost_copy<S><<<cdiv(d.g.nghost(), 256), 256, 0, s>>>(d.g, B<S>(d, b),
                       static_cast<S *>(d.ghost2))));
}

void launch_readout(const DevLattice &d, int view, int cur, int side_par, int X0, int X1,
                    double *out, int rec_stride, const uint64_t *dynp, cudaStream_t s)
{
    if (X1 <= X0) return;
    dim3 grid(cdiv(d.g.ly + 2, BX), X1 - X0);
    LBGPU_DISPATCH(d, (k_readout<S><<<grid, BX, 0, s>>>(d.g, view, B<S>(d, cur), OTHER<S>(d, cur),
                       SIDE<S>(d, side_par), X0, X1, out, rec_stride, dynp, d.inv_scale)));
}

void launch_upload(const DevLattice &d, int b, const double *in, int rec_stride, int X0, int X1,
                   int Y0, int H, cudaStream_t s)
{
    if (X1 <= X0 || H <= 0) return;
    dim3 grid(cdiv(H, BX), X1 - X0);
    LBGPU_DISPATCH(d, (k_upload<S><<<grid, BX, 0, s>>>(d.g, in, rec_stride, X0, X1, Y0, H, B<S>(d, b),
                       d.scale)));
}

// Tag plane from a host-order array tag_xy[X * (ly + 2) + Y] (ghost ring included): 32 x 32
// tiles through shared memory, read along y and written along x.
__global__ void k_tags_from_xy(Geo g, const uint8_t *__restrict__ in, uint8_t *__restrict__ tag)
{
    __shared__ uint8_t t[32][33];
    const int Y0 = blockIdx.x * 32, X0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
#pragma unroll
    for (int j = 0; j < 32; j += 8) {
        const int X = X0 + ty + j, Y = Y0 + tx;
        if (X < g.lx + 2 && Y < g.ly + 2) t[ty + j][tx] = in[(size_t)X * (g.ly + 2) + Y];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 32; j += 8) {
        const int Y = Y0 + ty + j, X = X0 + tx;
        if (X < g.lx + 2 && Y < g.ly + 2) tag[g.idx(X, Y)] = t[tx][ty + j];
    }
}

void launch_tags_from_xy(const DevLattice &d, const uint8_t *in, cudaStream_t s)
{
    dim3 grid(cdiv(d.g.ly + 2, 32), cdiv(d.g.lx + 2, 32));
    k_tags_from_xy<<<grid, dim3(32, 8), 0, s>>>(d.g, in, const_cast<uint8_t *>(d.tag));
}

void launch_zgb_rho(const DevLattice &d, int view, int cur, int side_par, cudaStream_t s)
{
    LBGPU_DISPATCH(d, (k_zgb_rho<S><<<cdiv(d.g.ly + 2, 128), 128, 0, s>>>(d.g, view, B<S>(d, cur),
                       OTHER<S>(d, cur), SIDE<S>(d, side_par), d.zrho, d.inv_scale)));
}

void launch_zgb_apply(const DevLattice &d, cudaStream_t s)
{
    k_zgb_apply<<<cdiv(4LL * d.g.nb, 256), 256, 0, s>>>(d.g.nb, d.zgb_src, d.zrho, d.bc);
}

void launch_periodic(const DevLattice &d, int b, cudaStream_t s)
{
    LBGPU_DISPATCH(d, (k_periodic<S><<<1, 1024, 0, s>>>(d.g, B<S>(d, b))));
}

void launch_init_cylinder(const DevLattice &d, int b, double umax, cudaStream_t s)
{
    dim3 grid(cdiv(d.g.lx + 2, BX), d.g.ly + 2);
    LBGPU_DISPATCH(d, (k_init_cylinder<S><<<grid, BX, 0, s>>>(d.g, B<S>(d, b), umax, d.scale)));
}

void launch_cylinder_tags(const DevLattice &d, int ox, int oy, int r, int wall_kind, cudaStream_t s)
{
    dim3 grid(cdiv(d.g.lx + 2, BX), d.g.ly + 2);
    const bool bb = wall_kind == LBGPU_WALL_BOUNCEBACK;
    k_cylinder_tags<<<grid, BX, 0, s>>>(d.g, const_cast<uint8_t *>(d.tag), ox, oy, r,
                                        bb ? LBGPU_TAG_BOUNCE_BACK : LBGPU_TAG_LOWER_REGULARIZED,
                                        bb ? LBGPU_TAG_BOUNCE_BACK : LBGPU_TAG_UPPER_REGULARIZED);
}

void launch_moments(const DevLattice &d, int view, int cur, int side_par, double *partial,
                    double *out, cudaStream_t s)
{
    LBGPU_DISPATCH(d, (k_moments_rows<S><<<d.g.ly, RED_THREADS, 0, s>>>(d.g, view, B<S>(d, cur),
                       OTHER<S>(d, cur), SIDE<S>(d, side_par), d.tag, partial, d.inv_scale)));
    k_moments_final<<<1, RED_THREADS, 0, s>>>(d.g.ly, partial, out);
}

void launch_velocity_change(const DevLattice &d, int view, int cur, int side_par, void *prev,
                            unsigned *out, cudaStream_t s)
{
    dim3 grid(cdiv(d.g.lx, BX), d.g.ly);
    LBGPU_DISPATCH(d, (k_velocity_change<S><<<grid, BX, 0, s>>>(d.g, view, B<S>(d, cur),
                       OTHER<S>(d, cur), SIDE<S>(d, side_par), static_cast<float2 *>(prev), out,
                       d.inv_scale)));
}

void launch_accumulate_velocity(const DevLattice &d, int view, int cur, int side_par, double *acc,
                                cudaStream_t s)
{
    dim3 grid(cdiv(d.g.lx, BX), d.g.ly);
    LBGPU_DISPATCH(d, (k_accumulate_velocity<S><<<grid, BX, 0, s>>>(d.g, view, B<S>(d, cur),
                       OTHER<S>(d, cur), SIDE<S>(d, side_par), acc, d.inv_scale)));
}

void launch_macros(const DevLattice &d, int view, int cur, int side_par, double *rho, double *ux,
                   double *uy, cudaStream_t s)
{
    dim3 grid(cdiv(d.g.lx, BX), d.g.ly);
    LBGPU_DISPATCH(d, (k_macros<S><<<grid, BX, 0, s>>>(d.g, view, B<S>(d, cur), OTHER<S>(d, cur),
                       SIDE<S>(d, side_par), rho, ux, uy, d.inv_scale)));
}

}  // namespace lbgpu
