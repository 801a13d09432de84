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

}  // namespace lbgpu
