// codec.cuh -- how populations are stored in HBM.
//
//   double          FP64 as is (the exact path)
//   float           FP32 as is
//   __half          FP16 offset: stored = (f_i - w_i) * 2^s, decoded to FP32 as
//   __nv_bfloat16   BF16 offset   w_i + stored * 2^-s
//
// Removing the lattice weight w_i leaves the small deviation from rest, whose magnitude
// (about 3 w_i |u|) the 11-bit (FP16) or 8-bit (BF16) mantissa resolves relatively; the
// power-of-two scale 2^s keeps those deviations out of the FP16 subnormal range and is exact
// to apply.  Opposite directions share a weight, so a value may move between the planes of
// i and opp(i) (the AA scheme does) without re-encoding.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include "d2q9.cuh"

namespace lbgpu {

template <class S> struct Codec;

template <> struct Codec<double> {
    using R = double;
    static __device__ __forceinline__ double dec(double v, int, float) { return v; }
    static __device__ __forceinline__ double enc(double v, int, float) { return v; }
};

template <> struct Codec<float> {
    using R = float;
    static __device__ __forceinline__ float dec(float v, int, float) { return v; }
    static __device__ __forceinline__ float enc(float v, int, float) { return v; }
};

template <> struct Codec<__half> {
    using R = float;
    static __device__ __forceinline__ float dec(__half v, int i, float inv)
    {
        return fmaf(__half2float(v), inv, wgtf(i));
    }
    static __device__ __forceinline__ __half enc(float v, int i, float sc)
    {
        return __float2half_rn((v - wgtf(i)) * sc);
    }
};

template <> struct Codec<__nv_bfloat16> {
    using R = float;
    static __device__ __forceinline__ float dec(__nv_bfloat16 v, int i, float inv)
    {
        return fmaf(__bfloat162float(v), inv, wgtf(i));
    }
    static __device__ __forceinline__ __nv_bfloat16 enc(float v, int i, float sc)
    {
        return __float2bfloat16_rn((v - wgtf(i)) * sc);
    }
};

// ---- stochastic rounding of 16-bit stores --------------------------------------------------
//
// Round to nearest loses every change of a stored value smaller than half its quantum: in a slow
// transient (a channel building its pressure gradient, a wake drifting) the 16-bit state stalls
// where the FP64 one moves on.  Stochastic rounding (Croci & Giles, "Effects of round-to-nearest
// and stochastic rounding in the numerical solution of the heat equation in low precision", 2020)
// rounds up with probability equal to the discarded fraction, so the stored value is unbiased.
// sm_100a converts with it in hardware: `cvt.rs.f16x2.f32 d, a, b, rbits` (and `.bf16x2`) adds
// random bits to the discarded mantissa bits and truncates.  The operand a goes to the upper half
// of d and takes its random bits from bits 16.. of rbits, b to the lower half with bits 0..
// (13 bits a value for FP16, 16 for BF16).
//
// The random bits of a value depend only on (seed, collision number k, node, direction), so every
// scheme that produces the same post-collision value stores the same bits:
//   key_k = rs_key(seed, k)                              per collision (host), never 0
//   H     = rs_mix((Y (lx + 2) + x0) ^ key_k)            per quad of nodes x0..x0+3 of a row,
//                                                        x0 = X - ((X - 1) mod 4)
//   P     = H * M(p, i),  p = (X - x0) / 2               per pair of nodes and direction, M odd
//   node x0 + 2p takes bits 0..15 of P, node x0 + 2p + 1 bits 16..31
// which is the operand layout of cvt.rs.f16x2: a quad's direction-i pair converts with P as
// rbits as it is, one hash a quad and one multiply a stored pair.  rs_mix is the 32-bit integer
// hash "lowbias32" (C. Wellons, hash-prospector).
__host__ __device__ __forceinline__ unsigned rs_mix(unsigned x)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

__host__ __device__ __forceinline__ unsigned rs_key(unsigned seed, unsigned long long k)
{
    const unsigned lo = (unsigned)k, hi = (unsigned)(k >> 32);
    return rs_mix(seed ^ rs_mix(lo ^ rs_mix(hi + 0x9e3779b9u))) | 1u;
}

__host__ __device__ __forceinline__ unsigned rs_pair(unsigned hq, int p, int i)
{
    return hq * (0x9e3779b9u * (unsigned)(2 * (9 * p + i) + 1));   // odd multiplier: a bijection of hq
}

// A node's place in its quad and the quad's hash (RS kernels; zero otherwise).
struct RsNode {
    unsigned hq;
    int q;
};

template <class S> struct RsOps;
template <> struct RsOps<__half> {
    // two values (lo -> bits 0..15 of the result with the random bits 0..15 of r, hi -> bits
    // 16..31 with r's bits 16..31)
    static __device__ __forceinline__ unsigned pack(float lo, float hi, unsigned r)
    {
        unsigned d;
        asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(r));
        return d;
    }
    // one value with the random bits 0..15 of r
    static __device__ __forceinline__ __half one(float v, unsigned r)
    {
        return __ushort_as_half((unsigned short)(pack(v, 0.0f, r & 0xffffu) & 0xffffu));
    }
};
template <> struct RsOps<__nv_bfloat16> {
    static __device__ __forceinline__ unsigned pack(float lo, float hi, unsigned r)
    {
        unsigned d;
        asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(r));
        return d;
    }
    static __device__ __forceinline__ __nv_bfloat16 one(float v, unsigned r)
    {
        return __ushort_as_bfloat16((unsigned short)(pack(v, 0.0f, r & 0xffffu) & 0xffffu));
    }
};

}  // namespace lbgpu
