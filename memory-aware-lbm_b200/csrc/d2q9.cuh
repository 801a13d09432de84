// d2q9.cuh -- D2Q9 lattice constants and per-node collision rules for the device.
//
// Two arithmetic forms:
//   * exact FP64 (namespace ex): the reference's expressions evaluated in its order with
//     explicit round-to-nearest IEEE intrinsics (__dadd_rn, __dmul_rn, __ddiv_rn), which the
//     compiler never fuses into FMAs.  A node collided here is bit-identical to the
//     reference's CPU code built without FMA contraction.
//   * fast FP32 (namespace fs): the same physics written for throughput (one reciprocal of
//     rho, FMA-friendly grouping), used by the FP32 and FP16/BF16-storage kernels and held to
//     a stated tolerance instead of bit-exactness.
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
// Exact FP64 rules (reference lb.c:134-166, boundaries.c:48-414).
// ----------------------------------------------------------------------------------------
namespace ex {

__device__ __forceinline__ double A(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double S(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double M(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double D(double a, double b) { return __ddiv_rn(a, b); }

// density and velocity from the three line sums (lb.c:134-141)
__device__ __forceinline__ void macros(const double f[9], double &rho, double &ux, double &uy)
{
    double top = A(A(f[2], f[5]), f[6]);
    double mid = A(A(f[0], f[1]), f[3]);
    double bot = A(A(f[4], f[7]), f[8]);
    rho = A(A(top, mid), bot);
    ux = D(S(A(A(f[1], f[5]), f[8]), A(A(f[3], f[6]), f[7])), rho);
    uy = D(S(top, bot), rho);
}

__device__ __forceinline__ double density(const double f[9])
{
    double top = A(A(f[2], f[5]), f[6]);
    double mid = A(A(f[0], f[1]), f[3]);
    double bot = A(A(f[4], f[7]), f[8]);
    return A(A(top, mid), bot);
}

// equilibrium of direction i: rho t_i (1 + 3cu + 4.5cu^2 - 1.5u^2), left to right (lb.c:144-151)
template <int I>
__device__ __forceinline__ double feq(double rho, double ux, double uy, double usqr)
{
    double cu = A(M((double)cx(I), ux), M((double)cy(I), uy));
    return M(M(rho, wgt(I)), S(A(A(1.0, M(3.0, cu)), M(M(4.5, cu), cu)), M(1.5, usqr)));
}

template <int I>
__device__ __forceinline__ void relax_one(double f[9], double omega, double om1, double rho,
                                          double ux, double uy, double usqr)
{
    f[I] = M(f[I], om1);
    f[I] = A(f[I], M(omega, feq<I>(rho, ux, uy, usqr)));
}

// BGK: f *= (1-omega); f += omega feq (lb.c:154-166)
__device__ __forceinline__ void bgk(double f[9], double omega)
{
    double rho, ux, uy;
    macros(f, rho, ux, uy);
    const double usqr = A(M(ux, ux), M(uy, uy));
    const double om1 = S(1.0, omega);
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

// full-way bounce-back (boundaries.c:48-59)
__device__ __forceinline__ void bounce(double f[9])
{
    double t;
    t = f[1]; f[1] = f[3]; f[3] = t;
    t = f[2]; f[2] = f[4]; f[4] = t;
    t = f[5]; f[5] = f[7]; f[7] = t;
    t = f[6]; f[6] = f[8]; f[8] = t;
}

// rest + tangential + 2 x outgoing populations of a straight wall (sums inside
// boundaries.c:66-126)
__device__ __forceinline__ double known_sum(const double f[9], int side)
{
    switch (side) {
    case SIDE_UPPER: return A(A(A(f[0], f[3]), f[1]), M(2.0, A(A(f[6], f[2]), f[5])));
    case SIDE_LOWER: return A(A(A(f[0], f[3]), f[1]), M(2.0, A(A(f[8], f[4]), f[7])));
    case SIDE_RIGHT: return A(A(A(f[0], f[2]), f[4]), M(2.0, A(A(f[1], f[5]), f[8])));
    default:         return A(A(A(f[0], f[2]), f[4]), M(2.0, A(A(f[3], f[6]), f[7])));
    }
}

// wall density from the normal velocity (upperRho..leftRho, boundaries.c:66-118)
__device__ __forceinline__ double wall_rho(const double f[9], int side, double un)
{
    const double s = known_sum(f, side);
    return (side == SIDE_UPPER || side == SIDE_RIGHT) ? M(D(1.0, A(1.0, un)), s)
                                                      : M(D(1.0, S(1.0, un)), s);
}

// normal velocity from the wall density (upperU..leftU, boundaries.c:74-126)
__device__ __forceinline__ double wall_u(const double f[9], int side, double rho)
{
    const double s = known_sum(f, side);
    return (side == SIDE_UPPER || side == SIDE_RIGHT) ? A(-1.0, M(D(1.0, rho), s))
                                                      : S(1.0, M(D(1.0, rho), s));
}

// Zou/He completion of the unknown populations (boundaries.c:131-169)
__device__ __forceinline__ void zouhe_complete(double f[9], int side, double ux, double uy,
                                               double rho)
{
    const double ruy6 = D(M(rho, uy), 6.0), rux2 = D(M(rho, ux), 2.0);
    const double rux6 = D(M(rho, ux), 6.0), ruy2 = D(M(rho, uy), 2.0);
    switch (side) {
    case SIDE_UPPER:
        f[7] = S(S(A(f[5], M(0.5, S(f[1], f[3]))), ruy6), rux2);
        f[8] = A(S(A(f[6], M(0.5, S(f[3], f[1]))), ruy6), rux2);
        f[4] = S(f[2], M(M(2. / 3., rho), uy));
        break;
    case SIDE_LOWER:
        f[6] = S(A(A(f[8], M(0.5, S(f[1], f[3]))), ruy6), rux2);
        f[5] = A(A(A(f[7], M(0.5, S(f[3], f[1]))), ruy6), rux2);
        f[2] = A(f[4], M(M(2. / 3., rho), uy));
        break;
    case SIDE_RIGHT:
        f[6] = A(S(A(f[8], M(0.5, S(f[4], f[2]))), rux6), ruy2);
        f[7] = S(S(A(f[5], M(0.5, S(f[2], f[4]))), rux6), ruy2);
        f[3] = S(f[1], M(M(2. / 3., rho), ux));
        break;
    default:
        f[5] = A(A(A(f[7], M(0.5, S(f[4], f[2]))), rux6), ruy2);
        f[8] = S(A(A(f[6], M(0.5, S(f[2], f[4]))), rux6), ruy2);
        f[1] = A(f[3], M(M(2. / 3., rho), ux));
        break;
    }
}

template <int I>
__device__ __forceinline__ void reg_one(double f[9], const double fe[9], double pxx, double pyy,
                                        double pxy)
{
    const double qxx = S((double)(cx(I) * cx(I)), 1. / 3.);
    const double qyy = S((double)(cy(I) * cy(I)), 1. / 3.);
    const double qxy = M(M(2.0, (double)cx(I)), (double)cy(I));
    f[I] = A(fe[I], M(M(9. / 2., wgt(I)), A(A(M(qxx, pxx), M(qyy, pyy)), M(qxy, pxy))));
}

// regularized reconstruction: splitEqNeq + side NeqPi + regularizedF (boundaries.c:239-302)
__device__ __forceinline__ void regularize(double f[9], int side, double rho, double ux, double uy)
{
    double fe[9], n[9];
    const double usqr = A(M(ux, ux), M(uy, uy));
    fe[0] = feq<0>(rho, ux, uy, usqr); fe[1] = feq<1>(rho, ux, uy, usqr);
    fe[2] = feq<2>(rho, ux, uy, usqr); fe[3] = feq<3>(rho, ux, uy, usqr);
    fe[4] = feq<4>(rho, ux, uy, usqr); fe[5] = feq<5>(rho, ux, uy, usqr);
    fe[6] = feq<6>(rho, ux, uy, usqr); fe[7] = feq<7>(rho, ux, uy, usqr);
    fe[8] = feq<8>(rho, ux, uy, usqr);
#pragma unroll
    for (int i = 0; i < 9; ++i) n[i] = S(f[i], fe[i]);
    double pxx, pyy, pxy;
    switch (side) {
    case SIDE_UPPER:
        pxx = A(A(n[1], n[3]), M(2.0, A(n[5], n[6])));
        pyy = M(2.0, A(A(n[6], n[2]), n[5]));
        pxy = M(2.0, S(n[5], n[6]));
        break;
    case SIDE_LOWER:
        pxx = A(A(n[1], n[3]), M(2.0, A(n[7], n[8])));
        pyy = M(2.0, A(A(n[4], n[7]), n[8]));
        pxy = M(2.0, S(n[7], n[8]));
        break;
    case SIDE_RIGHT:
        pxx = M(2.0, A(A(n[1], n[5]), n[8]));
        pyy = A(A(n[2], n[4]), M(2.0, A(n[5], n[8])));
        pxy = M(2.0, S(n[5], n[8]));
        break;
    default:
        pxx = M(2.0, A(A(n[3], n[6]), n[7]));
        pyy = A(A(n[2], n[4]), M(2.0, A(n[6], n[7])));
        pxy = M(2.0, S(n[7], n[6]));
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
static __device__ __noinline__ void collide_boundary(int t, double f[9], double omega,
                                                     double p0, double p1)
{
    if (t == TAG_BOUNCE) { bounce(f); return; }
    if (t < TAG_ZOUHE_FIRST || t >= TAG_COUNT) return;
    const int side = tag_side(t);
    const bool tb = side <= SIDE_LOWER;
    double rho, ux, uy;
    if (!tag_pressure(t)) {
        ux = p0; uy = p1;
        rho = wall_rho(f, side, tb ? uy : ux);
    } else {
        rho = p0;
        const double u = wall_u(f, side, rho);
        ux = tb ? p1 : u;
        uy = tb ? u : p1;
    }
    if (t < TAG_REG_FIRST) zouhe_complete(f, side, ux, uy, rho);
    else regularize(f, side, rho, ux, uy);
    bgk(f, omega);
}

// The boundary rules run out of line on a private copy, so the bulk path's populations stay
// in registers (a warp whose lanes are all bulk nodes never enters the call).
__device__ __forceinline__ void collide(int t, double f[9], double omega, double p0, double p1)
{
    if (t == TAG_BGK) {
        bgk(f, omega);
    } else {
        double g[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) g[i] = f[i];
        collide_boundary(t, g, omega, p0, p1);
#pragma unroll
        for (int i = 0; i < 9; ++i) f[i] = g[i];
    }
}

// equilibrium at (rho, ux, uy) for initialisation (lb.c:71-78)
__device__ __forceinline__ void equilibrium(double f[9], double rho, double ux, double uy)
{
    const double usqr = A(M(ux, ux), M(uy, uy));
    f[0] = feq<0>(rho, ux, uy, usqr); f[1] = feq<1>(rho, ux, uy, usqr);
    f[2] = feq<2>(rho, ux, uy, usqr); f[3] = feq<3>(rho, ux, uy, usqr);
    f[4] = feq<4>(rho, ux, uy, usqr); f[5] = feq<5>(rho, ux, uy, usqr);
    f[6] = feq<6>(rho, ux, uy, usqr); f[7] = feq<7>(rho, ux, uy, usqr);
    f[8] = feq<8>(rho, ux, uy, usqr);
}

}  // namespace ex
}  // namespace lbgpu
