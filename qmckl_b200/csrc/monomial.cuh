// FP32 cartesian monomials of l <= 3 by Horner, shared by the mixed-form AO
// producers (fused_common.cuh, ao_tile.cu).
#pragma once

#include <cuda_runtime.h>

namespace qb {

// (c0, c1, c2, c3) with r^a = c0 + c1 r + c2 r^2 + c3 r^3, a = 0..3.
static __constant__ float4 kAxisHot[4] = {{1.f, 0.f, 0.f, 0.f}, {0.f, 1.f, 0.f, 0.f}, {0.f, 0.f, 1.f, 0.f},
                                          {0.f, 0.f, 0.f, 1.f}};

// One axis of a cartesian monomial, exponent a <= 3 given by its one-hot
// coefficients h: F0 = r^a, F1 = a r^(a-1), G = a (a-1) r^(a-2) / 2.  With
// t2 = c3 r + c2 and t1 = t2 r + c1: F0 = t1 r + c0, F1 = (t2 + c3 r) r + t1,
// G = 3 c3 r + c2.
__device__ __forceinline__ void axis_factors(float r, float4 h, float& F0, float& F1, float& G) {
  const float t2 = fmaf(h.w, r, h.z);
  const float t1 = fmaf(t2, r, h.y);
  F0 = fmaf(t1, r, h.x);
  const float u = fmaf(h.w, r, t2);
  F1 = fmaf(u, r, t1);
  G = fmaf(h.w, r, u);
}

// x^a y^b z^c (a, b, c <= 3) and its gradient and Laplacian: P[0] the value,
// P[1..3] the gradient, P[4] the Laplacian.  The exponents index a
// warp-uniform table lookup: no selects, no branches.
__device__ __forceinline__ void monomial_horner(int a, int b, int c, float x, float y, float z, float (&P)[5]) {
  float X0, X1, XG, Y0, Y1, YG, Z0, Z1, ZG;
  axis_factors(x, kAxisHot[a & 3], X0, X1, XG);
  axis_factors(y, kAxisHot[b & 3], Y0, Y1, YG);
  axis_factors(z, kAxisHot[c & 3], Z0, Z1, ZG);
  const float xy = X0 * Y0, yz = Y0 * Z0, xz = X0 * Z0;
  P[0] = xy * Z0;
  P[1] = X1 * yz;
  P[2] = Y1 * xz;
  P[3] = Z1 * xy;
  P[4] = 2.f * (XG * yz + YG * xz + ZG * xy);
}

}  // namespace qb
