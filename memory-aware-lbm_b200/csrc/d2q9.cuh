// d2q9.cuh -- D2Q9 lattice constants and per-node collision rules for the device.
//
// The rules are templates over the arithmetic type T:
//   * T = double, exact: the reference's expressions evaluated in its order with explicit
//     round-to-nearest IEEE intrinsics (__dadd_rn, __dmul_rn, __ddiv_rn), which the compiler
//     never fuses into FMAs.  A node collided here is bit-identical to the reference's CPU
//     code built without FMA contraction.
//   * T = float, fast: the same physics with plain operators (FMA contraction allowed), and a
//     BGK written for throughput (one reciprocal of rho, factored equilibrium).  Used by the
//     FP32 and FP16/BF16-storage kernels and held to a stated tolerance.
//
// Direction order (reference lb.c:48-55): 0:(0,0) 1:(1,0) 2:(0,1) 3:(-1,0) 4:(0,-1)
// 5:(1,1) 6:(-1,1) 7:(-1,-1) 8:(1,-1); weights 4/9, 1/9 x4, 1/36 x4; opposite
// {0,3,4,1,2,7,8,5,6} (boundaries.c:32).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace lbgpu {

__host__ __device__ constexpr int cx(int i) { return (i == 1 || i == 5 || i == 8) ? 1 : ((i == 3 || i == 6 || i == 7) ? -1 : 0); }
__host__ __device__ constexpr int cy(int i) { return (i == 2 || i == 5 || i == 6) ? 1 : ((i == 4 || i == 7 || i == 8) ? -1 : 0); }
__host__ __device__ constexpr int opp(int i) { return i == 0 ? 0 : (i <= 4 ? ((i + 1) % 4) + 1 : ((i - 3) % 4) + 5); }
__host__ __device__ constexpr double wgt(int i) { return i == 0 ? 4. / 9. : (i < 5 ? 1. / 9. : 1. / 36.); }
__host__ __device__ constexpr float wgtf(int i) { return i == 0 ? 4.f / 9.f : (i < 5 ? 1.f / 9.f : 1.f / 36.f); }

// Dynamics tags (values shared with include/lbgpu.h LBGPU_TAG_*).
enum : int {
    TAG_NONE = 0, TAG_BGK = 1, TAG_BOUNCE = 2,
    TAG_ZOUHE_FIRST = 3, TAG_REG_FIRST = 11, TAG_COUNT = 19
};
enum : int { SIDE_UPPER = 0, SIDE_LOWER = 1, SIDE_LEFT = 2, SIDE_RIGHT = 3 };

// A boundary tag's side (0 upper, 1 lower, 2 left, 3 right), family (0 velocity,
// 1 pressure) and table index family*4 + side into the per-side parameter tables.
__host__ __device__ inline int tag_side(int t) { return (t - TAG_ZOUHE_FIRST) & 3; }
__host__ __device__ inline int tag_pressure(int t) { return ((t - TAG_ZOUHE_FIRST) >> 2) & 1; }
__host__ __device__ inline int tag_table(int t) { return tag_pressure(t) * 4 + tag_side(t); }

// ----------------------------------------------------------------------------------------
// Arithmetic policies.
// ----------------------------------------------------------------------------------------
template <class T> struct Ar;
template <> struct Ar<double> {
    static __device__ __forceinline__ double A(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double S(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double M(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double D(double a, double b) { return __ddiv_rn(a, b); }
};
template <> struct Ar<float> {
    static __device__ __forceinline__ float A(float a, float b) { return a + b; }
    static __device__ __forceinline__ float S(float a, float b) { return a - b; }
    static __device__ __forceinline__ float M(float a, float b) { return a * b; }
    static __device__ __forceinline__ float D(float a, float b) { return __fdiv_rn(a, b); }
};

// ----------------------------------------------------------------------------------------
// Rules (reference lb.c:134-166, boundaries.c:48-414), written once for both types.
// ----------------------------------------------------------------------------------------
namespace rules {

// density and velocity from the three line sums (lb.c:134-141)
template <class T>
__device__ __forceinline__ void macros(const T f[9], T &rho, T &ux, T &uy)
{
    using O = Ar<T>;
    T top = O::A(O::A(f[2], f[5]), f[6]);
    T mid = O::A(O::A(f[0], f[1]), f[3]);
    T bot = O::A(O::A(f[4], f[7]), f[8]);
    rho = O::A(O::A(top, mid), bot);
    ux = O::D(O::S(O::A(O::A(f[1], f[5]), f[8]), O::A(O::A(f[3], f[6]), f[7])), rho);
    uy = O::D(O::S(top, bot), rho);
}

template <class T>
__device__ __forceinline__ T density(const T f[9])
{
    using O = Ar<T>;
    T top = O::A(O::A(f[2], f[5]), f[6]);
    T mid = O::A(O::A(f[0], f[1]), f[3]);
    T bot = O::A(O::A(f[4], f[7]), f[8]);
    return O::A(O::A(top, mid), bot);
}

// equilibrium of direction I: rho t_I (1 + 3cu + 4.5cu^2 - 1.5u^2), left to right (lb.c:144-151)
template <int I, class T>
__device__ __forceinline__ T feq(T rho, T ux, T uy, T usqr)
{
    using O = Ar<T>;
    T cu = O::A(O::M((T)cx(I), ux), O::M((T)cy(I), uy));
    return O::M(O::M(rho, (T)wgt(I)), O::S(O::A(O::A((T)1, O::M((T)3, cu)), O::M(O::M((T)4.5, cu), cu)),
                                         O::M((T)1.5, usqr)));
}

template <int I, class T>
__device__ __forceinline__ void relax_one(T f[9], T omega, T om1, T rho, T ux, T uy, T usqr)
{
    using O = Ar<T>;
    f[I] = O::M(f[I], om1);
    f[I] = O::A(f[I], O::M(omega, feq<I>(rho, ux, uy, usqr)));
}

// BGK: f *= (1-omega); f += omega feq (lb.c:154-166)
template <class T>
__device__ __forceinline__ void bgk(T f[9], T omega)
{
    using O = Ar<T>;
    T rho, ux, uy;
    macros(f, rho, ux, uy);
    const T usqr = O::A(O::M(ux, ux), O::M(uy, uy));
    const T om1 = O::S((T)1, omega);
    relax_one<0>(f, omega, om1, rho, ux, uy, usqr);
    relax_one<1>(f, omega, om1, rho, ux, uy, usqr);
    relax_one<2>(f, omega, om1, rho, ux, uy, usqr);
    relax_one<3>(f, omega, om1, rho, ux, uy, usqr);
    relax_one<4>(f, omega, om1, rho, ux, uy, usqr);
    relax_one<5>(f, omega, om1, rho, ux, uy, usqr);
    relax_one<6>(f, omega, om1, rho, ux, uy, usqr);
    relax_one<7>(f, omega, om1, rho, ux, uy, usqr);
    relax_one<8>(f, omega, om1, rho, ux, uy, usqr);
}

// Throughput form of BGK in FP32: one reciprocal of rho, equilibrium factored as
// w rho (1 - 1.5u^2) + w rho cu (3 + 4.5 cu), relaxation as f + omega (feq - f).
template <>
__device__ __forceinline__ void bgk<float>(float f[9], float omega)
{
    const float rho = ((f[0] + f[1]) + (f[2] + f[3])) + ((f[4] + f[5]) + (f[6] + f[7])) + f[8];
    const float inv = __frcp_rn(rho);
    const float jx = (f[1] - f[3]) + (f[5] - f[6]) + (f[8] - f[7]);
    const float jy = (f[2] - f[4]) + (f[5] - f[8]) + (f[6] - f[7]);
    const float ux = jx * inv, uy = jy * inv;
    const float base = 1.0f - 1.5f * (ux * ux + uy * uy);
    const float r0 = (4.f / 9.f) * rho, r1 = (1.f / 9.f) * rho, r2 = (1.f / 36.f) * rho;
#define LBGPU_RELAX(I, W, CU)                                         \
    {                                                                 \
        const float cu = (CU);                                        \
        const float fe = W * (base + cu * (3.0f + 4.5f * cu));        \
        f[I] = fmaf(omega, fe - f[I], f[I]);                          \
    }
    LBGPU_RELAX(0, r0, 0.0f)
    LBGPU_RELAX(1, r1, ux)
    LBGPU_RELAX(2, r1, uy)
    LBGPU_RELAX(3, r1, -ux)
    LBGPU_RELAX(4, r1, -uy)
    LBGPU_RELAX(5, r2, ux + uy)
    LBGPU_RELAX(6, r2, uy - ux)
    LBGPU_RELAX(7, r2, -ux - uy)
    LBGPU_RELAX(8, r2, ux - uy)
#undef LBGPU_RELAX
}

// full-way bounce-back (boundaries.c:48-59)
template <class T>
__device__ __forceinline__ void bounce(T f[9])
{
    T t;
    t = f[1]; f[1] = f[3]; f[3] = t;
    t = f[2]; f[2] = f[4]; f[4] = t;
    t = f[5]; f[5] = f[7]; f[7] = t;
    t = f[6]; f[6] = f[8]; f[8] = t;
}

// rest + tangential + 2 x outgoing populations of a straight wall (sums inside
// boundaries.c:66-126)
template <class T>
__device__ __forceinline__ T known_sum(const T f[9], int side)
{
    using O = Ar<T>;
    switch (side) {
    case SIDE_UPPER: return O::A(O::A(O::A(f[0], f[3]), f[1]), O::M((T)2, O::A(O::A(f[6], f[2]), f[5])));
    case SIDE_LOWER: return O::A(O::A(O::A(f[0], f[3]), f[1]), O::M((T)2, O::A(O::A(f[8], f[4]), f[7])));
    case SIDE_RIGHT: return O::A(O::A(O::A(f[0], f[2]), f[4]), O::M((T)2, O::A(O::A(f[1], f[5]), f[8])));
    default:         return O::A(O::A(O::A(f[0], f[2]), f[4]), O::M((T)2, O::A(O::A(f[3], f[6]), f[7])));
    }
}

// wall density from the normal velocity (upperRho..leftRho, boundaries.c:66-118)
template <class T>
__device__ __forceinline__ T wall_rho(const T f[9], int side, T un)
{
    using O = Ar<T>;
    const T s = known_sum(f, side);
    return (side == SIDE_UPPER || side == SIDE_RIGHT) ? O::M(O::D((T)1, O::A((T)1, un)), s)
                                                      : O::M(O::D((T)1, O::S((T)1, un)), s);
}

// normal velocity from the wall density (upperU..leftU, boundaries.c:74-126)
template <class T>
__device__ __forceinline__ T wall_u(const T f[9], int side, T rho)
{
    using O = Ar<T>;
    const T s = known_sum(f, side);
    return (side == SIDE_UPPER || side == SIDE_RIGHT) ? O::A((T)-1, O::M(O::D((T)1, rho), s))
                                                      : O::S((T)1, O::M(O::D((T)1, rho), s));
}

// Zou/He completion of the unknown populations (boundaries.c:131-169)
template <class T>
__device__ __forceinline__ void zouhe_complete(T f[9], int side, T ux, T uy, T rho)
{
    using O = Ar<T>;
    const T ruy6 = O::D(O::M(rho, uy), (T)6), rux2 = O::D(O::M(rho, ux), (T)2);
    const T rux6 = O::D(O::M(rho, ux), (T)6), ruy2 = O::D(O::M(rho, uy), (T)2);
    const T two3 = (T)(2. / 3.);
    switch (side) {
    case SIDE_UPPER:
        f[7] = O::S(O::S(O::A(f[5], O::M((T)0.5, O::S(f[1], f[3]))), ruy6), rux2);
        f[8] = O::A(O::S(O::A(f[6], O::M((T)0.5, O::S(f[3], f[1]))), ruy6), rux2);
        f[4] = O::S(f[2], O::M(O::M(two3, rho), uy));
        break;
    case SIDE_LOWER:
        f[6] = O::S(O::A(O::A(f[8], O::M((T)0.5, O::S(f[1], f[3]))), ruy6), rux2);
        f[5] = O::A(O::A(O::A(f[7], O::M((T)0.5, O::S(f[3], f[1]))), ruy6), rux2);
        f[2] = O::A(f[4], O::M(O::M(two3, rho), uy));
        break;
    case SIDE_RIGHT:
        f[6] = O::A(O::S(O::A(f[8], O::M((T)0.5, O::S(f[4], f[2]))), rux6), ruy2);
        f[7] = O::S(O::S(O::A(f[5], O::M((T)0.5, O::S(f[2], f[4]))), rux6), ruy2);
        f[3] = O::S(f[1], O::M(O::M(two3, rho), ux));
        break;
    default:
        f[5] = O::A(O::A(O::A(f[7], O::M((T)0.5, O::S(f[4], f[2]))), rux6), ruy2);
        f[8] = O::S(O::A(O::A(f[6], O::M((T)0.5, O::S(f[2], f[4]))), rux6), ruy2);
        f[1] = O::A(f[3], O::M(O::M(two3, rho), ux));
        break;
    }
}

template <int I, class T>
__device__ __forceinline__ void reg_one(T f[9], const T fe[9], T pxx, T pyy, T pxy)
{
    using O = Ar<T>;
    const T qxx = O::S((T)(cx(I) * cx(I)), (T)(1. / 3.));
    const T qyy = O::S((T)(cy(I) * cy(I)), (T)(1. / 3.));
    const T qxy = O::M(O::M((T)2, (T)cx(I)), (T)cy(I));
    f[I] = O::A(fe[I], O::M(O::M((T)4.5, (T)wgt(I)), O::A(O::A(O::M(qxx, pxx), O::M(qyy, pyy)), O::M(qxy, pxy))));
}

// regularized reconstruction: splitEqNeq + side NeqPi + regularizedF (boundaries.c:239-302)
template <class T>
__device__ __forceinline__ void regularize(T f[9], int side, T rho, T ux, T uy)
{
    using O = Ar<T>;
    T fe[9], n[9];
    const T usqr = O::A(O::M(ux, ux), O::M(uy, uy));
    fe[0] = feq<0>(rho, ux, uy, usqr); fe[1] = feq<1>(rho, ux, uy, usqr);
    fe[2] = feq<2>(rho, ux, uy, usqr); fe[3] = feq<3>(rho, ux, uy, usqr);
    fe[4] = feq<4>(rho, ux, uy, usqr); fe[5] = feq<5>(rho, ux, uy, usqr);
    fe[6] = feq<6>(rho, ux, uy, usqr); fe[7] = feq<7>(rho, ux, uy, usqr);
    fe[8] = feq<8>(rho, ux, uy, usqr);
#pragma unroll
    for (int i = 0; i < 9; ++i) n[i] = O::S(f[i], fe[i]);
    T pxx, pyy, pxy;
    switch (side) {
    case SIDE_UPPER:
        pxx = O::A(O::A(n[1], n[3]), O::M((T)2, O::A(n[5], n[6])));
        pyy = O::M((T)2, O::A(O::A(n[6], n[2]), n[5]));
        pxy = O::M((T)2, O::S(n[5], n[6]));
        break;
    case SIDE_LOWER:
        pxx = O::A(O::A(n[1], n[3]), O::M((T)2, O::A(n[7], n[8])));
        pyy = O::M((T)2, O::A(O::A(n[4], n[7]), n[8]));
        pxy = O::M((T)2, O::S(n[7], n[8]));
        break;
    case SIDE_RIGHT:
        pxx = O::M((T)2, O::A(O::A(n[1], n[5]), n[8]));
        pyy = O::A(O::A(n[2], n[4]), O::M((T)2, O::A(n[5], n[8])));
        pxy = O::M((T)2, O::S(n[5], n[8]));
        break;
    default:
        pxx = O::M((T)2, O::A(O::A(n[3], n[6]), n[7]));
        pyy = O::A(O::A(n[2], n[4]), O::M((T)2, O::A(n[6], n[7])));
        pxy = O::M((T)2, O::S(n[7], n[6]));
        break;
    }
    reg_one<0>(f, fe, pxx, pyy, pxy); reg_one<1>(f, fe, pxx, pyy, pxy);
    reg_one<2>(f, fe, pxx, pyy, pxy); reg_one<3>(f, fe, pxx, pyy, pxy);
    reg_one<4>(f, fe, pxx, pyy, pxy); reg_one<5>(f, fe, pxx, pyy, pxy);
    reg_one<6>(f, fe, pxx, pyy, pxy); reg_one<7>(f, fe, pxx, pyy, pxy);
    reg_one<8>(f, fe, pxx, pyy, pxy);
}

// Any non-BGK rule; (p0, p1) are the node's table entry: (ux, uy) or (rho, uPar).
// Boundary rules chain to bulk BGK like every function of boundaries.c:171-414.
template <class T>
static __device__ __noinline__ void collide_boundary(int t, T f[9], T omega, T p0, T p1)
{
    if (t == TAG_BOUNCE) { bounce(f); return; }
    if (t < TAG_ZOUHE_FIRST || t >= TAG_COUNT) return;
    const int side = tag_side(t);
    const bool tb = side <= SIDE_LOWER;
    T rho, ux, uy;
    if (!tag_pressure(t)) {
        ux = p0; uy = p1;
        rho = wall_rho(f, side, tb ? uy : ux);
    } else {
        rho = p0;
        const T u = wall_u(f, side, rho);
        ux = tb ? p1 : u;
        uy = tb ? u : p1;
    }
    if (t < TAG_REG_FIRST) zouhe_complete(f, side, ux, uy, rho);
    else regularize(f, side, rho, ux, uy);
    bgk(f, omega);
}

// The boundary rules run out of line on a private copy, so the bulk path's populations stay
// in registers (a warp whose lanes are all bulk nodes never enters the call).
template <class T>
__device__ __forceinline__ void collide(int t, T f[9], T omega, T p0, T p1)
{
    if (t == TAG_BGK) {
        bgk(f, omega);
    } else {
        T g[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) g[i] = f[i];
        collide_boundary<T>(t, g, omega, p0, p1);
#pragma unroll
        for (int i = 0; i < 9; ++i) f[i] = g[i];
    }
}

// equilibrium at (rho, ux, uy) for initialisation (lb.c:71-78)
template <class T>
__device__ __forceinline__ void equilibrium(T f[9], T rho, T ux, T uy)
{
    using O = Ar<T>;
    const T usqr = O::A(O::M(ux, ux), O::M(uy, uy));
    f[0] = feq<0>(rho, ux, uy, usqr); f[1] = feq<1>(rho, ux, uy, usqr);
    f[2] = feq<2>(rho, ux, uy, usqr); f[3] = feq<3>(rho, ux, uy, usqr);
    f[4] = feq<4>(rho, ux, uy, usqr); f[5] = feq<5>(rho, ux, uy, usqr);
    f[6] = feq<6>(rho, ux, uy, usqr); f[7] = feq<7>(rho, ux, uy, usqr);
    f[8] = feq<8>(rho, ux, uy, usqr);
}

}  // namespace rules
}  // namespace lbgpu
