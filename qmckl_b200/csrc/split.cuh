// Operand pieces of the mixed-form MO contraction on the tensor cores.
//
//   3 pieces: bfloat16, x = x1 + x2 + x3 (round to nearest at each step); the
//             six products of total order <= 2 are accumulated.
//   2 pieces: float16 of x / s, s a power of two, x / s = x1 + x2 (round to
//             nearest); the three products x1 y1, x1 y2, x2 y1 are
//             accumulated.  float16 keeps 11 significant bits per piece (22
//             for the pair, against 24 for three bfloat16 pieces) but needs
//             the scale s to keep values inside its range (6e-8 .. 65504):
//             one per AO component for the AO matrix (value, gradient,
//             Laplacian: an upper bound of the component over the basis,
//             brought to 2^10), one per MO for the coefficients (its largest
//             coefficient brought to 2^10).  Scales are powers of two, so
//             scaling and unscaling are exact.
// The scale block (doubles) stored after the coefficient pieces: [0..4] the
// AO-component scales, [kScaleCols + mo] the MO scales (all 1 for 3 pieces).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdint>

namespace qb {

constexpr int kScaleCols = 8;

// Two FP32 values -> PIECES packed pieces (element 0 in the low half).
template <int PIECES>
__device__ __forceinline__ void split_pair(float v0, float v1, float inv_scale, uint32_t (&pk)[3]) {
  if constexpr (PIECES == 2) {
    const float a0 = v0 * inv_scale, a1 = v1 * inv_scale;
    const __half2 h2 = __floats2half2_rn(a0, a1);
    const float2 hf = __half22float2(h2);
    const __half2 m2 = __floats2half2_rn(a0 - hf.x, a1 - hf.y);
    pk[0] = *reinterpret_cast<const uint32_t*>(&h2);
    pk[1] = *reinterpret_cast<const uint32_t*>(&m2);
    pk[2] = 0u;
  } else {
    const __nv_bfloat162 h2 = __floats2bfloat162_rn(v0, v1);
    const float2 hf = __bfloat1622float2(h2);
    const float r0 = v0 - hf.x, r1 = v1 - hf.y;
    const __nv_bfloat162 m2 = __floats2bfloat162_rn(r0, r1);
    const float2 mf = __bfloat1622float2(m2);
    const __nv_bfloat162 l2 = __floats2bfloat162_rn(r0 - mf.x, r1 - mf.y);
    pk[0] = *reinterpret_cast<const uint32_t*>(&h2);
    pk[1] = *reinterpret_cast<const uint32_t*>(&m2);
    pk[2] = *reinterpret_cast<const uint32_t*>(&l2);
  }
}

// One FP32 value -> PIECES 16-bit pieces.
template <int PIECES>
__device__ __forceinline__ void split_one(float v, float inv_scale, uint16_t (&o)[3]) {
  if constexpr (PIECES == 2) {
    const float a = v * inv_scale;
    const __half h = __float2half_rn(a);
    const __half m = __float2half_rn(a - __half2float(h));
    o[0] = __half_as_ushort(h);
    o[1] = __half_as_ushort(m);
    o[2] = 0;
  } else {
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    const float r = v - __bfloat162float(h);
    const __nv_bfloat16 m = __float2bfloat16_rn(r);
    o[0] = __bfloat16_as_ushort(h);
    o[1] = __bfloat16_as_ushort(m);
    o[2] = __bfloat16_as_ushort(__float2bfloat16_rn(r - __bfloat162float(m)));
  }
}

// One FP64 value -> 3 bfloat16 pieces, each the rounding of the remainder
// (formed exactly in FP64): x = x1 + x2 + x3 to ~2^-24 relative.
__device__ __forceinline__ void split3_bf16(double v, uint16_t (&o)[3]) {
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const __nv_bfloat16 h = __double2bfloat16(v);
    o[q] = __bfloat16_as_ushort(h);
    v -= (double)__bfloat162float(h);
  }
}

// Reciprocal AO-component scales (exact: powers of two) for the producers;
// all 1 when no scale block is given (3 bfloat16 pieces need none).
template <int COMPS>
__device__ __forceinline__ void load_inv_scales(const double* scales, float (&inv)[5]) {
#pragma unroll
  for (int c = 0; c < 5; ++c) inv[c] = scales ? (float)(1.0 / scales[c < COMPS ? c : 0]) : 1.f;
}

}  // namespace qb
