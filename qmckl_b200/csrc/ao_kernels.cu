// AO kernels: FP64 AO VGL / AO value, the primitive and shell VGL getters, and
// the mixed-precision AO VGL kernel that feeds the tensor-core MO contraction.
//
// Arithmetic follows the reference's production kernel
// qmckl_compute_ao_vgl_hpc_gaussian (org/qmckl_ao.org:8601-8973):
//   * nucleus screened when r^2 > cutoff * nucleus_range          (8707)
//   * per nucleus, primitives sorted by exponent; a primitive and all
//     following ones are skipped once a*r^2 > cutoff                (8756-8766)
//   * radial VGL: e = exp(-a r^2), f = -2 a e,
//     (e, f x, f y, f z, f (3 - 2 a r^2)) contracted with the merged
//     normalized coefficients                                         (8798-8828)
//   * shell skipped when its contracted value is exactly zero         (8850)
//   * product rule with the cartesian monomials of
//     qmckl_ao_polynomial_transp_vgl_hpc (6624-6914), 1e-20 shift on the value.
//
// Work decomposition (B200): one warp evaluates one (point, nucleus block)
// pair.  Lanes first form the displacements of the block's nuclei, then the
// radial VGL of the block's shells into shared memory, then sweep the block's
// contiguous AO range with consecutive lanes on consecutive AOs, so every
// store of ao_vgl[point][comp][k] is a 256-byte coalesced row segment.
#include <cuda_bf16.h>

#include "kernels.cuh"
#include "split.cuh"

namespace qb {

namespace {

constexpr int kWarps = 8;
constexpr double kShift = 1.e-20;

__device__ __forceinline__ double ipow(double x, int n) {
  double r = 1.0;
  for (int i = 0; i < n; ++i) r = r * x;
  return r;
}

// Cartesian monomial x^a y^b z^c with gradient and Laplacian, as formed by the
// reference's HPC polynomial routine (l >= 2 branch; l <= 1 handled by caller).
template <typename R>
__device__ __forceinline__ void monomial_vgl(int a, int b, int c, R x, R y, R z, R out[5]) {
  const R pa = (R)ipow(x, a), pb = (R)ipow(y, b), pc = (R)ipow(z, c);
  const R pa1 = a >= 1 ? (R)ipow(x, a - 1) : R(1), pb1 = b >= 1 ? (R)ipow(y, b - 1) : R(1),
          pc1 = c >= 1 ? (R)ipow(z, c - 1) : R(1);
  const R pa2 = a >= 2 ? (R)ipow(x, a - 2) : R(1), pb2 = b >= 2 ? (R)ipow(y, b - 2) : R(1),
          pc2 = c >= 2 ? (R)ipow(z, c - 2) : R(1);
  R xy = pa * pb, yz = pb * pc, xz = pa * pc;
  out[0] = xy * pc + R(kShift);
  xy *= R(c);
  xz *= R(b);
  yz *= R(a);
  out[1] = pa1 * yz;
  out[2] = pb1 * xz;
  out[3] = pc1 * xy;
  out[4] = R(a - 1) * pa2 * yz + R(b - 1) * pb2 * xz + R(c - 1) * pc2 * xy;
}

// x^n, x^(n-1) and x^(n-2) for 0 <= n <= 3 without branches; a missing power
// is 1 (it is multiplied by n or n - 1 = 0).
__device__ __forceinline__ void pows3(double x, int n, double& p0, double& p1, double& p2) {
  const double f1 = n >= 1 ? x : 1.0, f2 = n >= 2 ? x : 1.0, f3 = n >= 3 ? x : 1.0;
  p2 = f3;
  p1 = f2 * f3;
  p0 = f1 * p1;
}

struct WarpSmem {
  double rad[kBlockSlots][5];   // radial VGL of the block's shells
  double nuc[kBlockNuc][4];     // x, y, z displacement, r^2 (negative when screened out)
  uint8_t act[kBlockSlots];     // the shells whose nucleus is in range
};

// Radial part of one shell (slot) for one point; FP64 throughout.
template <int COMPS>
__device__ __forceinline__ void shell_radial(const DevTables& T, int slot, int nucl, double x, double y,
                                             double z, double r2, double cutoff, bool dp_exp,
                                             double out[5]) {
  double acc[5] = {0., 0., 0., 0., 0.};
  const int2 cr = T.slot_coef[slot];
  (void)nucl;
  for (int j = cr.x; j < cr.y; ++j) {
    const double2 ac = T.coef_ac[j];
    const double a = ac.x;
    const double ar2 = a * r2;
    if (ar2 > cutoff) break;   // primitives are sorted by exponent
    const double e = dp_exp ? exp(-ar2) : (double)expf(-(float)ar2);
    const double cv = ac.y;
    acc[0] += cv * e;
    if (COMPS == 5) {
      double f = a * e;
      f = -f - f;
      acc[1] += cv * (f * x);
      acc[2] += cv * (f * y);
      acc[3] += cv * (f * z);
      acc[4] += cv * (f * (3.0 - 2.0 * ar2));
    }
  }
#pragma unroll
  for (int c = 0; c < 5; ++c) out[c] = acc[c];
}

// Stages 1 and 2 of a (point, block) item: displacements and radial VGL in smem.
template <int COMPS>
__device__ __forceinline__ void stage_block(const DevTables& T, WarpSmem& sm, const int4 blk,
                                            const int2 slots, double px, double py, double pz,
                                            double cutoff, bool dp_exp, int lane) {
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
  // shells of screened-out nuclei are not staged: the AO loop tests the
  // nucleus before it reads sm.rad
  const int nlive = pack_live_slots(T.slot_nuc, blk.x, slots, sm.nuc, sm.act, lane);
  for (int i = lane; i < nlive; i += 32) {
    const int ls = sm.act[i];
    const int s = slots.x + ls;
    const int nucl = T.slot_nuc[s];
    const int nl = nucl - blk.x;
    double out[5];
    shell_radial<COMPS>(T, s, nucl, sm.nuc[nl][0], sm.nuc[nl][1], sm.nuc[nl][2], sm.nuc[nl][3], cutoff, dp_exp, out);
#pragma unroll
    for (int c = 0; c < 5; ++c) sm.rad[ls][c] = out[c];
  }
  __syncwarp();
}

// FP64 AO VGL (COMPS = 5) or AO value (COMPS = 1).  SPLIT: each value
// stored as 3 bfloat16 pieces (split.cuh) at pieces[q * pstride + row * lda
// + ao], rows p * COMPS + c, instead of FP64 in `out`.
template <int COMPS, bool SPLIT = false>
__global__ void __launch_bounds__(kWarps * 32)
ao_f64_kernel(const DevTables T, const int64_t point_num, const double* __restrict__ coord,
              const double cutoff, const bool dp_exp, double* __restrict__ out,
              uint16_t* __restrict__ pieces = nullptr, const int64_t lda = 0, const int64_t pstride = 0,
              const double* __restrict__ cusp_r = nullptr) {
  __shared__ WarpSmem smem[kWarps];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  WarpSmem& sm = smem[warp];
  const int64_t A = T.ao_num;
  const int64_t stride = (int64_t)gridDim.x * kWarps;
  // one warp per point, through its nucleus blocks in order: the point's
  // rows are written in sequence (faster than spreading a point's blocks
  // over warps: 2.9 against 3.1 ms on the config-1 molecule)
  for (int64_t p = (int64_t)blockIdx.x * kWarps + warp; p < point_num; p += stride)
  for (int b = 0; b < T.nblock; ++b) {
    const int4 blk = T.block[b];
    const int2 slots = T.block_slots[b];
    const double px = coord[p], py = coord[p + point_num], pz = coord[p + 2 * point_num];
    stage_block<COMPS>(T, sm, blk, slots, px, py, pz, cutoff, dp_exp, lane);
    double* __restrict__ row = out + p * COMPS * A;
    // The lanes' 32-AO groups start on a 128-byte boundary of the output
    // (64 bytes of the bfloat16 pieces): a group that straddles it writes
    // partial sectors and ~20% fewer bytes per second (2.87 ms against 2.37
    // for the 13 GB of the config-1 molecule's AO VGL, stores alone).
    const int sh = SPLIT ? (int)((reinterpret_cast<uintptr_t>(pieces + p * COMPS * lda + blk.z) >> 1) & 31)
                         : (int)((reinterpret_cast<uintptr_t>(row + blk.z) >> 3) & 15);
    for (int k = blk.z - sh + lane; k < blk.w; k += 32) {
      if (k < blk.z) continue;
      const int code = T.ao_code[k];
      const int a = code & 15, bb = (code >> 4) & 15, c = (code >> 8) & 15, l = (code >> 12) & 15;
      const int slot = (code >> 16) & 255, nl = (code >> 24) & 31;
      double v[5] = {0., 0., 0., 0., 0.};
      const double s1 = sm.rad[slot][0];
      if (sm.nuc[nl][3] >= 0.0 && s1 != 0.0 && !cusp_masked(cusp_r, l, blk.x + nl, sm.nuc[nl][3], COMPS == 1)) {
        const double f = T.ao_factor[k];
        const double s2 = sm.rad[slot][1], s3 = sm.rad[slot][2], s4 = sm.rad[slot][3], s5 = sm.rad[slot][4];
        if (l <= 3) {
          // one formula for every l <= 3 (the l = 0 and l = 1 cases of the
          // reference are its special values): no divergence between lanes
          double xa, xa1, xa2, yb, yb1, yb2, zc, zc1, zc2;
          pows3(sm.nuc[nl][0], a, xa, xa1, xa2);
          pows3(sm.nuc[nl][1], bb, yb, yb1, yb2);
          pows3(sm.nuc[nl][2], c, zc, zc1, zc2);
          const double da = (double)a, db = (double)bb, dc = (double)c;
          const double yz = yb * zc, xz = xa * zc, xy = xa * yb;
          const double P0 = xa * yz + (l >= 1 ? kShift : 0.0);
          const double P1 = da * xa1 * yz, P2 = db * yb1 * xz, P3 = dc * zc1 * xy;
          v[0] = P0 * s1 * f;
          if (COMPS == 5) {
            const double P4 = da * (da - 1.0) * xa2 * yz + db * (db - 1.0) * yb2 * xz + dc * (dc - 1.0) * zc2 * xy;
            v[1] = (P1 * s1 + P0 * s2) * f;
            v[2] = (P2 * s1 + P0 * s3) * f;
            v[3] = (P3 * s1 + P0 * s4) * f;
            v[4] = (P4 * s1 + P0 * s5 + 2.0 * (P1 * s2 + P2 * s3 + P3 * s4)) * f;
          }
        } else {   // l >= 4
          double P[5];
          monomial_vgl<double>(a, bb, c, sm.nuc[nl][0], sm.nuc[nl][1], sm.nuc[nl][2], P);
          v[0] = P[0] * s1 * f;
          if (COMPS == 5) {
            v[1] = (P[1] * s1 + P[0] * s2) * f;
            v[2] = (P[2] * s1 + P[0] * s3) * f;
            v[3] = (P[3] * s1 + P[0] * s4) * f;
            v[4] = (P[4] * s1 + P[0] * s5 + 2.0 * (P[1] * s2 + P[2] * s3 + P[3] * s4)) * f;
          }
        }
      }
      if constexpr (SPLIT) {
#pragma unroll
        for (int c = 0; c < COMPS; ++c) {
          uint16_t pc[3];
          split3_bf16(v[c], pc);
          uint16_t* dst = pieces + (p * COMPS + c) * lda + k;
          dst[0] = pc[0];
          dst[pstride] = pc[1];
          dst[2 * pstride] = pc[2];
        }
      } else {
        // streaming stores: the array is written once and not read back here
        __stcs(&row[k], v[0]);
        if (COMPS == 5) {
          __stcs(&row[A + k], v[1]);
          __stcs(&row[2 * A + k], v[2]);
          __stcs(&row[3 * A + k], v[3]);
          __stcs(&row[4 * A + k], v[4]);
        }
      }
    }
    __syncwarp();
  }
}

// qmckl_compute_ao_basis_primitive_gaussian_vgl (org/qmckl_ao.org:4468-4520):
// one thread per (point, primitive), primitive fastest for coalesced stores.
__global__ void primitive_vgl_kernel(const DevTables T, const int64_t point_num,
                                     const double* __restrict__ coord, const double cutoff,
                                     double* __restrict__ out) {
  const int64_t Pn = T.prim_num;
  const int64_t total = point_num * Pn;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = i / Pn;
    const int64_t q = i - p * Pn;
    const int n = T.prim_nuc[q];
    const int N = T.nucl_num;
    const double x = coord[p] - T.nucl_coord[n];
    const double y = coord[p + point_num] - T.nucl_coord[n + N];
    const double z = coord[p + 2 * point_num] - T.nucl_coord[n + 2 * N];
    const double r2 = x * x + y * y + z * z;
    const double a = T.prim_expo[q];
    const double ar2 = a * r2;
    double* o = out + p * 5 * Pn + q;
    if (ar2 > cutoff) {
      o[0] = 0.0; o[Pn] = 0.0; o[2 * Pn] = 0.0; o[3 * Pn] = 0.0; o[4 * Pn] = 0.0;
      continue;
    }
    const double v = exp(-ar2);
    const double two_a = -2.0 * a * v;
    o[0] = v;
    o[Pn] = two_a * x;
    o[2 * Pn] = two_a * y;
    o[3 * Pn] = two_a * z;
    o[4 * Pn] = two_a * (3.0 - 2.0 * ar2);
  }
}

// qmckl_compute_ao_basis_shell_gaussian_vgl (org/qmckl_ao.org:4769-4868):
// one thread per (point, shell); primitives in the user's order.
__global__ void shell_vgl_kernel(const DevTables T, const int64_t point_num,
                                 const double* __restrict__ coord, const double cutoff,
                                 double* __restrict__ out) {
  const int64_t S = T.shell_num;
  const int64_t total = point_num * S;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = i / S;
    const int64_t s = i - p * S;
    const int n = T.shell_nuc[s];
    const int N = T.nucl_num;
    const double x = coord[p] - T.nucl_coord[n];
    const double y = coord[p + point_num] - T.nucl_coord[n + N];
    const double z = coord[p + 2 * point_num] - T.nucl_coord[n + 2 * N];
    const double r2 = x * x + y * y + z * z;
    double acc[5] = {0., 0., 0., 0., 0.};
    if (!(r2 > cutoff * T.nucleus_range[n])) {
      const int2 pr = T.shell_prims[s];
      for (int q = pr.x; q < pr.y; ++q) {
        const double a = T.prim_expo[q];
        const double ar2 = a * r2;
        if (ar2 > cutoff) continue;
        const double v = T.prim_coef[q] * exp(-ar2);
        const double two_a = -2.0 * a * v;
        acc[0] += v;
        acc[1] += two_a * x;
        acc[2] += two_a * y;
        acc[3] += two_a * z;
        acc[4] += two_a * (3.0 - 2.0 * ar2);
      }
    }
    double* o = out + p * 5 * S + s;
#pragma unroll
    for (int c = 0; c < 5; ++c) o[c * S] = acc[c];
  }
}

int grid_for(int64_t items_per_warp_unit) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t want = (items_per_warp_unit + kWarps - 1) / kWarps;
  const int64_t cap = (int64_t)sms * 8;
  return (int)(want < cap ? (want > 0 ? want : 1) : cap);
}

}  // namespace

cudaError_t launch_ao_vgl_f64(const DevTables& T, int64_t point_num, const double* coord,
                              double cutoff, bool dp_exp, double* ao_vgl, cudaStream_t s, const double* cusp_r) {
  if (point_num <= 0) return cudaSuccess;
  const int grid = grid_for(point_num);   // one warp per point
  ao_f64_kernel<5><<<grid, kWarps * 32, 0, s>>>(T, point_num, coord, cutoff, dp_exp, ao_vgl, nullptr, 0, 0, cusp_r);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_ao_vgl_pieces(const DevTables& T, int64_t point_num, const double* coord, double cutoff,
                                 bool dp_exp, void* pieces, int64_t lda, int64_t pstride, cudaStream_t s) {
  if (point_num <= 0) return cudaSuccess;
  if (lda < T.ao_num || lda % 8 != 0 || pstride % 8 != 0) return cudaErrorInvalidValue;
  const int grid = grid_for(point_num);   // one warp per point
  ao_f64_kernel<5, true><<<grid, kWarps * 32, 0, s>>>(T, point_num, coord, cutoff, dp_exp, nullptr,
                                                      (uint16_t*)pieces, lda, pstride);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_ao_value_f64(const DevTables& T, int64_t point_num, const double* coord,
                                double cutoff, bool dp_exp, double* ao_value, cudaStream_t s, const double* cusp_r) {
  if (point_num <= 0) return cudaSuccess;
  const int grid = grid_for(point_num);   // one warp per point
  ao_f64_kernel<1><<<grid, kWarps * 32, 0, s>>>(T, point_num, coord, cutoff, dp_exp, ao_value, nullptr, 0, 0,
                                                cusp_r);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_primitive_vgl(const DevTables& T, int64_t point_num, const double* coord,
                                 double cutoff, double* prim_vgl, cudaStream_t s) {
  if (point_num <= 0) return cudaSuccess;
  const int64_t total = point_num * T.prim_num;
  const int grid = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
  primitive_vgl_kernel<<<grid, 256, 0, s>>>(T, point_num, coord, cutoff, prim_vgl);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_shell_vgl(const DevTables& T, int64_t point_num, const double* coord,
                             double cutoff, double* shell_vgl, cudaStream_t s) {
  if (point_num <= 0) return cudaSuccess;
  const int64_t total = point_num * T.shell_num;
  const int grid = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
  shell_vgl_kernel<<<grid, 256, 0, s>>>(T, point_num, coord, cutoff, shell_vgl);
  count_launch();
  return cudaGetLastError();
}

}  // namespace qb
