// Derivative kernels of the AO VGL: the AO Hessian getter and the adjoint of
// MO VGL with respect to the nuclear and point coordinates.
//
// Quantities (derivatives with respect to the point coordinates r; an AO
// centred on nucleus A depends on r - R_A, so d/dR_A = -d/dr):
//   radial part  R(s) = sum_j c_j exp(-a_j s), s = r^2, and its s-derivatives
//                R1 = -sum a c e, R2 = sum a^2 c e, R3 = -sum a^3 c e
//                d_d R = 2 x_d R1,  d_d d_e R = 4 x_d x_e R2 + 2 delta_de R1,
//                lap R = 4 s R2 + 6 R1,  d_d lap R = x_d (20 R2 + 8 s R3)
//   monomial     P = x^a y^b z^c with all derivatives up to third order
//   AO           chi = f P R;  H_de = d_d d_e chi;  T_d = d_d lap chi
// The reference forms the same quantities from the shell Hessian
// (qmckl_compute_ao_basis_shell_gaussian_hessian, org/qmckl_ao.org:5480-5580),
// the polynomial Hessian (qmckl_compute_ao_polynomial_hessian_doc, 7113-7236)
// and the AO Hessian (qmckl_compute_ao_hessian_doc, 9590-9720); its orbital
// forces (org/qmckl_forces.org:5688-6772) contract them with the MO
// coefficients.  Screening follows the forward kernels: nucleus skipped when
// r^2 > cutoff * range, primitives sorted by exponent with a break at
// a r^2 > cutoff, AO skipped when its contracted radial value is zero.
//
// Work decomposition: one warp per (point, nucleus block), as in the forward
// AO kernel: lanes stage the block's displacements and radial derivative sets
// in shared memory, then sweep the block's contiguous AO range.
//   MODE_HESSIAN  writes ao_hessian[3][point][4][ao] (coalesced rows).
//   MODE_ADJOINT  reads G[point][5][ao] = (W . C)[point][comp][ao], the loss
//                 weights pulled back through the MO coefficients, and forms
//                 q_d = G0 d_d chi + sum_e G_{1+e} H_ed + G4 T_d per AO.  A
//                 segmented warp reduction over the (contiguous) AOs of each
//                 nucleus feeds per-CTA shared accumulators of dL/dR (one
//                 device atomic per nucleus and CTA at the end); the sum over
//                 all AOs gives dL/dr of the point.
#include <algorithm>
#include <type_traits>

#include "kernels.cuh"

namespace qb {
namespace {

constexpr int kWarpsD = 8;
constexpr double kShiftD = 1.e-20;
constexpr int MODE_HESSIAN = 0, MODE_ADJOINT = 1;

struct DerivSmem {
  double rad[kBlockSlots][4];   // R, R1, R2, R3 of the block's shells
  double nuc[kBlockNuc][4];     // displacement, r^2 (negative when screened out)
  uint8_t act[kBlockSlots];     // the shells whose nucleus is in range
};

// x^a and its first three derivatives (Leibniz, one factor x at a time)
template <typename F>
__device__ __forceinline__ void pow_derivs(F x, int a, F (&q)[4]) {
  if (a <= 3) {
    // without branches (lanes of a warp hold different exponents): with
    // f_i = x for i <= a, 1 otherwise, x^a = f1 f2 f3, and the derivatives
    // a x^(a-1), a (a-1) x^(a-2), a (a-1) (a-2) vanish where they must
    const F f1 = a >= 1 ? x : F(1), f2 = a >= 2 ? x : F(1), f3 = a >= 3 ? x : F(1);
    const F fa = F(a);
    q[2] = fa * (fa - F(1)) * f3;
    q[1] = fa * (f2 * f3);
    q[0] = f1 * (f2 * f3);
    q[3] = fa * (fa - F(1)) * (fa - F(2));
    return;
  }
  q[0] = F(1); q[1] = F(0); q[2] = F(0); q[3] = F(0);
  for (int i = 0; i < a; ++i) {
    q[3] = q[3] * x + F(3) * q[2];
    q[2] = q[2] * x + F(2) * q[1];
    q[1] = q[1] * x + q[0];
    q[0] = q[0] * x;
  }
}

template <bool MIXED>
__device__ __forceinline__ void stage_deriv(const DevTables& T, DerivSmem& sm, const int4 blk, const int2 slots,
                                            double px, double py, double pz, double cutoff, int lane) {
  const int nn = blk.y - blk.x;
  if (lane < nn) {
    const int n = blk.x + lane;
    const int N = T.nucl_num;
    const double x = px - T.nucl_coord[n];
    const double y = py - T.nucl_coord[n + N];
    const double z = pz - T.nucl_coord[n + 2 * N];
    const double r2 = x * x + y * y + z * z;
    const bool in = !(r2 > cutoff * T.nucleus_range[n]);
    sm.nuc[lane][0] = x;
    sm.nuc[lane][1] = y;
    sm.nuc[lane][2] = z;
    sm.nuc[lane][3] = in ? r2 : -1.0;
  }
  __syncwarp();
  // shells of screened-out nuclei are not staged (the AO loop tests the nucleus first)
  const int nlive = pack_live_slots(T.slot_nuc, blk.x, slots, sm.nuc, sm.act, lane);
  for (int i = lane; i < nlive; i += 32) {
    const int ls = sm.act[i];
    const int s = slots.x + ls;
    const int nucl = T.slot_nuc[s];
    const double r2 = sm.nuc[nucl - blk.x][3];
    double acc[4] = {0., 0., 0., 0.};
    {
      const int2 cr = T.slot_coef[s];
      const int p0 = T.nuc_prim_start[nucl];
      for (int j = cr.x; j < cr.y; ++j) {
        const double a = T.expo[p0 + T.coef_prim[j]];
        const double ar2 = a * r2;
        if (ar2 > cutoff) break;   // primitives sorted by exponent
        const double e = (MIXED && ar2 <= 30.0) ? (double)expf(-(float)ar2) : exp(-ar2);
        const double ce = T.coef_val[j] * e;
        acc[0] += ce;
        acc[1] -= a * ce;
        acc[2] += a * a * ce;
        acc[3] -= a * a * a * ce;
      }
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) sm.rad[ls][c] = acc[c];
  }
  __syncwarp();
}

// Hessian H[d][e] and gradient of the Laplacian T[d] of one AO (times its
// factor f), plus its gradient g[d], in arithmetic F.  The radial
// combinations that cancel near their zeros, lap R = 4 s R2 + 6 R1 and
// k3 = 20 R2 + 8 s R3, come in formed in FP64.
template <typename F>
__device__ __forceinline__ void ao_derivs(int code, F f, const F (&v)[3], const F (&R)[3], F lapR, F k3,
                                          F (&g)[3], F (&H)[3][3], F (&Tl)[3]) {
  const int ax = code & 15, by = (code >> 4) & 15, cz = (code >> 8) & 15, l = (code >> 12) & 15;
  F X[4], Y[4], Z[4];
  pow_derivs<F>(v[0], ax, X);
  pow_derivs<F>(v[1], by, Y);
  pow_derivs<F>(v[2], cz, Z);
  const F P = X[0] * Y[0] * Z[0] + (l >= 1 ? F(kShiftD) : F(0));
  const F Pd[3] = {X[1] * Y[0] * Z[0], X[0] * Y[1] * Z[0], X[0] * Y[0] * Z[1]};
  F Pdd[3][3];
  Pdd[0][0] = X[2] * Y[0] * Z[0];
  Pdd[1][1] = X[0] * Y[2] * Z[0];
  Pdd[2][2] = X[0] * Y[0] * Z[2];
  Pdd[0][1] = Pdd[1][0] = X[1] * Y[1] * Z[0];
  Pdd[0][2] = Pdd[2][0] = X[1] * Y[0] * Z[1];
  Pdd[1][2] = Pdd[2][1] = X[0] * Y[1] * Z[1];
  const F lapP = Pdd[0][0] + Pdd[1][1] + Pdd[2][2];
  const F dlapP[3] = {X[3] * Y[0] * Z[0] + X[1] * Y[2] * Z[0] + X[1] * Y[0] * Z[2],
                      X[2] * Y[1] * Z[0] + X[0] * Y[3] * Z[0] + X[0] * Y[1] * Z[2],
                      X[2] * Y[0] * Z[1] + X[0] * Y[2] * Z[1] + X[0] * Y[0] * Z[3]};
  const F Rd[3] = {F(2) * v[0] * R[1], F(2) * v[1] * R[1], F(2) * v[2] * R[1]};
  F Rdd[3][3];
#pragma unroll
  for (int d = 0; d < 3; ++d)
#pragma unroll
    for (int e = 0; e < 3; ++e) Rdd[d][e] = F(4) * v[d] * v[e] * R[2] + (d == e ? F(2) * R[1] : F(0));
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    g[d] = f * (Pd[d] * R[0] + P * Rd[d]);
#pragma unroll
    for (int e = 0; e < 3; ++e) H[d][e] = f * (Pdd[d][e] * R[0] + Pd[d] * Rd[e] + Pd[e] * Rd[d] + P * Rdd[d][e]);
    F t = F(0);
#pragma unroll
    for (int e = 0; e < 3; ++e) t += Pdd[d][e] * Rd[e] + Pd[e] * Rdd[d][e];
    Tl[d] = f * (dlapP[d] * R[0] + lapP * Rd[d] + F(2) * t + Pd[d] * lapR + P * v[d] * k3);
  }
}

// MODE_HESSIAN: out = ao_hessian[3][point_num][4][ao] (point_num points from
//   coord [3][cstride], cstride >= point_num).
// MODE_ADJOINT: G = [point_num][5][ao]; grad_nucl [nucl][3] -= sum q (per-CTA
//   shared accumulators when use_smem, else device atomics); grad_coord
//   ([3][gstride], may be null) += sum q.
// MIXED: FP32 exponentials where a r^2 <= 30; in MODE_ADJOINT also G in FP32
//   and the per-AO derivative arithmetic in FP32 (displacements, r^2, radial
//   sums and the cancelling radial combinations in FP64; q summed in FP64).
template <int MODE, bool MIXED>
__global__ void __launch_bounds__(kWarpsD * 32)
deriv_kernel(const DevTables T, const int64_t point_num, const double* __restrict__ coord, const int64_t cstride,
             const double cutoff, double* __restrict__ out, const void* __restrict__ Gv,
             double* __restrict__ grad_nucl, double* __restrict__ grad_coord, const int64_t gstride,
             const bool use_smem, const double* __restrict__ cusp_r) {
  using F = typename std::conditional<MIXED && MODE == MODE_ADJOINT, float, double>::type;
  const F* __restrict__ G = (const F*)Gv;
  __shared__ DerivSmem smem[kWarpsD];
  extern __shared__ double sacc[];   // [nucl][3] (MODE_ADJOINT with use_smem)
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  DerivSmem& sm = smem[warp];
  const int64_t A = T.ao_num;
  if (MODE == MODE_ADJOINT && use_smem) {
    for (int i = threadIdx.x; i < 3 * T.nucl_num; i += blockDim.x) sacc[i] = 0.0;
    __syncthreads();
  }
  const int64_t stride = (int64_t)gridDim.x * kWarpsD;
  // one warp per point, through its nucleus blocks (as the FP64 AO kernel)
  for (int64_t p = (int64_t)blockIdx.x * kWarpsD + warp; p < point_num; p += stride) {
   double pg[3] = {0., 0., 0.};
   for (int b = 0; b < T.nblock; ++b) {
    const int4 blk = T.block[b];
    const int2 slots = T.block_slots[b];
    stage_deriv<MIXED>(T, sm, blk, slots, coord[p], coord[p + cstride], coord[p + 2 * cstride], cutoff, lane);
    for (int k0 = blk.z; k0 < blk.w; k0 += 32) {
      const int k = k0 + lane;
      const bool valid = k < blk.w;
      int nl = kBlockNuc;   // past-the-end lanes form their own (last) segment
      F g[3] = {F(0), F(0), F(0)}, H[3][3] = {{F(0), F(0), F(0)}, {F(0), F(0), F(0)}, {F(0), F(0), F(0)}},
        Tl[3] = {F(0), F(0), F(0)};
      if (valid) {
        const int code = T.ao_code[k];
        const int slot = (code >> 16) & 255;
        nl = (code >> 24) & 31;
        const double r2 = sm.nuc[nl][3];
        const double* Rs = sm.rad[slot];
        if (r2 >= 0.0 && Rs[0] != 0.0 && !cusp_masked(cusp_r, (code >> 12) & 15, blk.x + nl, r2, false)) {
          const double lapR = 4.0 * r2 * Rs[2] + 6.0 * Rs[1];
          const double k3 = 20.0 * Rs[2] + 8.0 * r2 * Rs[3];
          const F v[3] = {(F)sm.nuc[nl][0], (F)sm.nuc[nl][1], (F)sm.nuc[nl][2]};
          const F R[3] = {(F)Rs[0], (F)Rs[1], (F)Rs[2]};
          ao_derivs<F>(code, (F)T.ao_factor[k], v, R, (F)lapR, (F)k3, g, H, Tl);
        }
      }
      if (MODE == MODE_HESSIAN) {
        if (valid) {
#pragma unroll
          for (int i = 0; i < 3; ++i) {
            double* o = out + ((int64_t)i * point_num + p) * 4 * A;
            o[k] = H[i][0];
            o[A + k] = H[i][1];
            o[2 * A + k] = H[i][2];
            o[3 * A + k] = Tl[i];
          }
        }
      } else {
        double q[3] = {0., 0., 0.};
        if (valid) {
          const F* gr = G + p * 5 * A + k;
          const F G0 = gr[0], G1 = gr[A], G2 = gr[2 * A], G3 = gr[3 * A], G4 = gr[4 * A];
#pragma unroll
          for (int d = 0; d < 3; ++d)
            q[d] = (double)(G0 * g[d] + G1 * H[0][d] + G2 * H[1][d] + G3 * H[2][d] + G4 * Tl[d]);
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) pg[d] += q[d];
        // segmented sum over lanes of the same nucleus (AOs of a nucleus are
        // contiguous, so segments are runs of lanes): the first lane of each
        // run ends up with the run's sum
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
          const int ko = __shfl_down_sync(0xffffffffu, nl, off);
          double o[3];
#pragma unroll
          for (int d = 0; d < 3; ++d) o[d] = __shfl_down_sync(0xffffffffu, q[d], off);
          if (lane + off < 32 && ko == nl) {
#pragma unroll
            for (int d = 0; d < 3; ++d) q[d] += o[d];
          }
        }
        const int kprev = __shfl_up_sync(0xffffffffu, nl, 1);
        if ((lane == 0 || kprev != nl) && nl < kBlockNuc) {
          const int n = blk.x + nl;
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            if (use_smem) atomicAdd(&sacc[n * 3 + d], q[d]);
            else if (grad_nucl != nullptr) atomicAdd(&grad_nucl[n * 3 + d], -q[d]);
          }
        }
      }
    }
    __syncwarp();
   }
    if (MODE == MODE_ADJOINT && grad_coord != nullptr) {
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        double s = pg[d];
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        pg[d] = s;
      }
      if (lane == 0) {
#pragma unroll
        for (int d = 0; d < 3; ++d) atomicAdd(&grad_coord[p + d * gstride], pg[d]);
      }
    }
    __syncwarp();
  }
  if (MODE == MODE_ADJOINT && use_smem && grad_nucl != nullptr) {
    __syncthreads();
    for (int i = threadIdx.x; i < 3 * T.nucl_num; i += blockDim.x)
      if (sacc[i] != 0.0) atomicAdd(&grad_nucl[i], -sacc[i]);
  }
}

template <int MODE>
cudaError_t launch_deriv(const DevTables& T, int64_t point_num, const double* coord, int64_t cstride, double cutoff,
                         bool mixed, double* out, const void* G, double* grad_nucl, double* grad_coord,
                         int64_t gstride, cudaStream_t s, const double* cusp_r = nullptr) {
  if (point_num <= 0) return cudaSuccess;
  const int grid = (int)std::min<int64_t>((point_num + kWarpsD - 1) / kWarpsD, 148 * 8);   // warps = points
  size_t dyn = 0;
  bool use_smem = false;
  if (MODE == MODE_ADJOINT) {
    dyn = sizeof(double) * 3 * (size_t)T.nucl_num;
    use_smem = dyn <= 64 * 1024;
    if (!use_smem) dyn = 0;
  }
  cudaError_t e = cudaSuccess;
  if (mixed) {
    auto k = deriv_kernel<MODE, true>;
    if (dyn > 48 * 1024) e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
    if (e != cudaSuccess) return e;
    k<<<grid, kWarpsD * 32, dyn, s>>>(T, point_num, coord, cstride, cutoff, out, G, grad_nucl, grad_coord, gstride,
                                      use_smem, cusp_r);
  } else {
    auto k = deriv_kernel<MODE, false>;
    if (dyn > 48 * 1024) e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
    if (e != cudaSuccess) return e;
    k<<<grid, kWarpsD * 32, dyn, s>>>(T, point_num, coord, cstride, cutoff, out, G, grad_nucl, grad_coord, gstride,
                                      use_smem, cusp_r);
  }
  count_launch();
  return cudaGetLastError();
}

// Orbital forces (derivatives with respect to the nuclear coordinates; the
// reference's qmckl_get_forces_* getters, org/qmckl_forces.org:5129-6880).
// Only the AOs of nucleus a depend on R_a, so each force is a contraction
// over that nucleus's AO range [nuc_ao[a].x, nuc_ao[a].y):
//   out[(a * R + r) * M + i] = -sum_k X_r[k] * Ct[k][i]
// with the row r and its source row X_r:
//   MODE 0 forces_mo_value [a][p][n][i]: R = 3P, r = 3p + n,         X_r = ao_vgl[p][1+n]
//   MODE 1 forces_mo_g [a][n][p][m][i]:  R = 9P, r = 3(nP + p) + m,  X_r = ao_hessian[n][p][m]
//   MODE 2 forces_mo_l [a][n][p][i]:     R = 3P, r = nP + p,         X_r = ao_hessian[n][p][3]
// One thread per output element, MOs fastest (coalesced Ct reads and stores).
template <int MODE>
__global__ void forces_mo_kernel(const int64_t P, const int64_t A, const int64_t M, const int N,
                                 const int2* __restrict__ nuc_ao, const double* __restrict__ X,
                                 const double* __restrict__ Ct, double* __restrict__ out) {
  const int64_t R = (MODE == 1 ? 9 : 3) * P;
  const int64_t total = (int64_t)N * R * M;
  for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < total; u += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = u % M;
    const int64_t ar = u / M;
    const int a = (int)(ar / R);
    const int64_t r = ar - (int64_t)a * R;
    const double* xr;
    if (MODE == 0) {
      const int64_t p = r / 3, n = r - 3 * p;
      xr = X + (p * 5 + 1 + n) * A;
    } else if (MODE == 1) {
      const int64_t np = r / 3, m = r - 3 * np;
      xr = X + (np * 4 + m) * A;
    } else {
      xr = X + (r * 4 + 3) * A;
    }
    const int2 kr = nuc_ao[a];
    double acc = 0.0;
    for (int k = kr.x; k < kr.y; ++k) acc -= Ct[(int64_t)k * M + i] * xr[k];
    out[u] = acc;
  }
}

// forces_ao_value[a][p][n][k] = -ao_vgl[p][1+n][k] for the AOs of nucleus a, 0 elsewhere
__global__ void forces_ao_kernel(const int64_t P, const int64_t A, const int N, const int2* __restrict__ nuc_ao,
                                 const double* __restrict__ X, double* __restrict__ out) {
  const int64_t total = (int64_t)N * P * 3 * A;
  for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < total; u += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = u % A;
    const int64_t apn = u / A;
    const int64_t n = apn % 3, ap = apn / 3;
    const int64_t p = ap % P;
    const int a = (int)(ap / P);
    const int2 kr = nuc_ao[a];
    out[u] = (k >= kr.x && k < kr.y) ? -X[(p * 5 + 1 + n) * A + k] : 0.0;
  }
}

}  // namespace

cudaError_t launch_forces(int which, int64_t P, int64_t A, int64_t M, int N, const int2* nuc_ao, const double* X,
                          const double* Ct, double* out, cudaStream_t s) {
  if (P <= 0 || N <= 0) return cudaSuccess;
  const int64_t total = which == 3 ? (int64_t)N * P * 3 * A : (int64_t)N * (which == 1 ? 9 : 3) * P * M;
  const int grid = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
  switch (which) {
    case 0: forces_mo_kernel<0><<<grid, 256, 0, s>>>(P, A, M, N, nuc_ao, X, Ct, out); break;
    case 1: forces_mo_kernel<1><<<grid, 256, 0, s>>>(P, A, M, N, nuc_ao, X, Ct, out); break;
    case 2: forces_mo_kernel<2><<<grid, 256, 0, s>>>(P, A, M, N, nuc_ao, X, Ct, out); break;
    case 3: forces_ao_kernel<<<grid, 256, 0, s>>>(P, A, N, nuc_ao, X, out); break;
    default: return cudaErrorInvalidValue;
  }
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_ao_hessian(const DevTables& T, int64_t point_num, const double* coord, double cutoff, bool mixed,
                              double* ao_hessian, cudaStream_t s, const double* cusp_r) {
  return launch_deriv<MODE_HESSIAN>(T, point_num, coord, point_num, cutoff, mixed, ao_hessian, nullptr, nullptr,
                                    nullptr, 0, s, cusp_r);
}

cudaError_t launch_mo_adjoint_nuclear(const DevTables& T, int64_t point_num, const double* coord, int64_t cstride,
                                      double cutoff, bool mixed, const void* G, double* grad_nucl,
                                      double* grad_coord, int64_t gstride, cudaStream_t s) {
  return launch_deriv<MODE_ADJOINT>(T, point_num, coord, cstride, cutoff, mixed, nullptr, G, grad_nucl, grad_coord,
                                    gstride, s);
}

}  // namespace qb
