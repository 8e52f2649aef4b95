// Tiled AO kernels: one CTA evaluates a tile of 32 points x one AO tile
// (64 AOs, 32 where a 64-AO window holds more than 32 shells).
//
// Phase 0  the tile's points, nuclei and shells are staged in shared memory
// Phase R  the radial VGL of every (point, shell) of the tile, once, into
//          shared memory (consecutive threads = consecutive points of one
//          shell, so a warp runs the same primitive loop)
// Phase A  one thread per (point, 8 consecutive AOs): monomials with
//          branch-free power selection, the product rule, and 16-byte stores
//          of whole 8-AO row segments
// Output modes: FP64 ao_vgl[point][5][ao] / ao_value[point][ao] (arithmetic
// of qmckl_compute_ao_vgl_hpc_gaussian, org/qmckl_ao.org:8601-8973, as in
// ao_kernels.cu), or the bfloat16 pieces of the mixed form (FP64 radial part
// with FP32 exponentials for a r^2 <= 30, FP32 monomials and product rule).
#include <cuda_bf16.h>

#include "ao_tile.cuh"
#include "monomial.cuh"
#include "split.cuh"

namespace qb {
namespace {

constexpr int TP = kTilePoints;
constexpr int kThreads = 256;
constexpr double kShift = 1.e-20;

template <typename R>
struct RadT;
template <>
struct RadT<double> { using T = double; };
template <>
struct RadT<float> { using T = float; };

__device__ __forceinline__ double sel_pow(int n, double x, double x2, double x3) {
  return n == 0 ? 1.0 : (n == 1 ? x : (n == 2 ? x2 : x3));
}
__device__ __forceinline__ float sel_pow(int n, float x, float x2, float x3) {
  return n == 0 ? 1.f : (n == 1 ? x : (n == 2 ? x2 : x3));
}
template <typename R>
__device__ __forceinline__ R loop_pow(R x, int n) {
  R r = R(1);
  for (int i = 0; i < n; ++i) r = r * x;
  return r;
}

// Monomial VGL for l >= 2, the generic formula of the reference's HPC
// polynomial routine (org/qmckl_ao.org:6840-6880).  Powers are formed as
// 1, x, x*x, (x*x)*x like its running products.
template <typename R>
__device__ __forceinline__ void monomial(int a, int b, int c, R x, R y, R z, R shift, R (&P)[5]) {
  R pa, pb, pc, pa1, pb1, pc1, pa2, pb2, pc2;
  if (a <= 3 && b <= 3 && c <= 3) {
    const R x2 = x * x, y2 = y * y, z2 = z * z;
    const R x3 = x2 * x, y3 = y2 * y, z3 = z2 * z;
    pa = sel_pow(a, x, x2, x3); pb = sel_pow(b, y, y2, y3); pc = sel_pow(c, z, z2, z3);
    pa1 = sel_pow(a > 0 ? a - 1 : 0, x, x2, x3); pb1 = sel_pow(b > 0 ? b - 1 : 0, y, y2, y3);
    pc1 = sel_pow(c > 0 ? c - 1 : 0, z, z2, z3);
    pa2 = sel_pow(a > 1 ? a - 2 : 0, x, x2, x3); pb2 = sel_pow(b > 1 ? b - 2 : 0, y, y2, y3);
    pc2 = sel_pow(c > 1 ? c - 2 : 0, z, z2, z3);
  } else {
    pa = loop_pow(x, a); pb = loop_pow(y, b); pc = loop_pow(z, c);
    pa1 = a >= 1 ? loop_pow(x, a - 1) : R(1); pb1 = b >= 1 ? loop_pow(y, b - 1) : R(1);
    pc1 = c >= 1 ? loop_pow(z, c - 1) : R(1);
    pa2 = a >= 2 ? loop_pow(x, a - 2) : R(1); pb2 = b >= 2 ? loop_pow(y, b - 2) : R(1);
    pc2 = c >= 2 ? loop_pow(z, c - 2) : R(1);
  }
  R xy = pa * pb, yz = pb * pc, xz = pa * pc;
  P[0] = xy * pc + shift;
  xy *= R(c);
  xz *= R(b);
  yz *= R(a);
  P[1] = pa1 * yz;
  P[2] = pb1 * xz;
  P[3] = pc1 * xy;
  P[4] = R(a - 1) * pa2 * yz + R(b - 1) * pb2 * xz + R(c - 1) * pc2 * xy;
}

// AO value/gradient/Laplacian from its shell radial VGL s[] (product rule of
// org/qmckl_ao.org:8913-8950; a zero contracted value gives a zero AO, 8850).
template <typename R, int COMPS>
__device__ __forceinline__ void ao_vgl_one(int code, R f, const R* s, R x, R y, R z, R shift, R (&v)[5]) {
#pragma unroll
  for (int c = 0; c < 5; ++c) v[c] = R(0);
  const R s1 = s[0];
  if (s1 == R(0)) return;
  const int a = code & 15, b = (code >> 4) & 15, c = (code >> 8) & 15, l = (code >> 12) & 15;
  if (l == 0) {
    v[0] = s1 * f;
    if (COMPS == 5) { v[1] = s[1] * f; v[2] = s[2] * f; v[3] = s[3] * f; v[4] = s[4] * f; }
    return;
  }
  R P[5];
  if (l == 1) {
    P[0] = (a ? x : (b ? y : z)) + shift;
    P[1] = R(a); P[2] = R(b); P[3] = R(c); P[4] = R(0);
  } else if (std::is_same<R, float>::value && l <= 3) {
    // FP32 (mixed form): the three cubics by Horner of monomial.cuh
    float Pf[5];
    monomial_horner(a, b, c, (float)x, (float)y, (float)z, Pf);
#pragma unroll
    for (int q = 0; q < 5; ++q) P[q] = (R)Pf[q];
    P[0] += shift;
  } else {
    monomial<R>(a, b, c, x, y, z, shift, P);
  }
  v[0] = P[0] * s1 * f;
  if (COMPS == 5) {
    v[1] = (P[1] * s1 + P[0] * s[1]) * f;
    v[2] = (P[2] * s1 + P[0] * s[2]) * f;
    v[3] = (P[3] * s1 + P[0] * s[3]) * f;
    if (l == 1) v[4] = (P[0] * s[4] + R(2) * (P[1] * s[1] + P[2] * s[2] + P[3] * s[3])) * f;
    else v[4] = (P[4] * s1 + P[0] * s[4] + R(2) * (P[1] * s[1] + P[2] * s[2] + P[3] * s[3])) * f;
  }
}

// MODE 0: FP64 output (exponentials in FP64 when dp_exp, else FP32 as the
// reference's single-precision branch); MODE 2 / 3: mixed form, 2 / 3 pieces.
template <int MODE, int COMPS>
__global__ void __launch_bounds__(kThreads)
ao_tile_kernel(const DevTables T, const AoTiles Tl, const int64_t P, const double* __restrict__ coord,
               const double cutoff, const bool dp_exp, void* __restrict__ out, const int64_t ld,
               const int64_t piece_stride, const double* __restrict__ scales) {
  using R = typename RadT<typename std::conditional<MODE == 0, double, float>::type>::T;
  __shared__ double s_pts[3][TP];
  __shared__ double s_nuc[kTileNuc][4];          // x, y, z, cutoff * range
  __shared__ int s_sh_nuc[kTileShells];
  __shared__ int2 s_sh_coef[kTileShells];
  __shared__ int s_sh_p0[kTileShells];
  __shared__ R s_rad[TP][kTileShells][5];

  const int tid = threadIdx.x;
  const int64_t p0 = (int64_t)blockIdx.x * TP;
  const int4 tile = Tl.tile[blockIdx.y];        // (k_begin, k_end, shell_begin, shell_end)
  const int2 tnuc = Tl.tile_nuc[blockIdx.y];    // (nuc_begin, nuc_end)
  const int nsh = tile.w - tile.z, nnu = tnuc.y - tnuc.x;
  const int N = T.nucl_num;

  if (tid < 3 * TP) {
    const int d = tid / TP, i = tid - d * TP;
    s_pts[d][i] = (p0 + i < P) ? coord[(p0 + i) + d * P] : 1.0e30;
  }
  if (tid < nnu) {
    const int n = tnuc.x + tid;
    s_nuc[tid][0] = T.nucl_coord[n];
    s_nuc[tid][1] = T.nucl_coord[n + N];
    s_nuc[tid][2] = T.nucl_coord[n + 2 * N];
    s_nuc[tid][3] = cutoff * T.nucleus_range[n];
  }
  if (tid < nsh) {
    const int sh = tile.z + tid;
    const int n = T.shell_nuc[sh];
    s_sh_nuc[tid] = n - tnuc.x;
    s_sh_coef[tid] = T.shell_coef[sh];
    s_sh_p0[tid] = T.nuc_prim_start[n];
  }
  __syncthreads();

  // ---- Phase R: radial VGL of (point, shell)
  for (int u = tid; u < nsh * TP; u += kThreads) {
    const int sl = u / TP, i = u - sl * TP;
    const int nl = s_sh_nuc[sl];
    const double x = s_pts[0][i] - s_nuc[nl][0];
    const double y = s_pts[1][i] - s_nuc[nl][1];
    const double z = s_pts[2][i] - s_nuc[nl][2];
    const double r2 = x * x + y * y + z * z;
    double acc[5] = {0., 0., 0., 0., 0.};
    if (!(r2 > s_nuc[nl][3])) {
      const int2 cr = s_sh_coef[sl];
      const int pb = s_sh_p0[sl];
      for (int j = cr.x; j < cr.y; ++j) {
        const double al = T.expo[pb + T.coef_prim[j]];
        const double ar2 = al * r2;
        if (ar2 > cutoff) break;   // primitives sorted by exponent
        const double cv = T.coef_val[j];
        if (MODE == 0) {
          const double e = dp_exp ? exp(-ar2) : (double)expf(-(float)ar2);
          acc[0] += cv * e;
          if (COMPS == 5) {
            double f = al * e;
            f = -f - f;
            acc[1] += cv * (f * x);
            acc[2] += cv * (f * y);
            acc[3] += cv * (f * z);
            acc[4] += cv * (f * (3.0 - 2.0 * ar2));
          }
        } else {
          const double e = ar2 > 30.0 ? exp(-ar2) : (double)expf(-(float)ar2);
          acc[0] += cv * e;
          if (COMPS == 5) {
            const double f = -2.0 * al * e;
            acc[1] += cv * (f * x);
            acc[2] += cv * (f * y);
            acc[3] += cv * (f * z);
            acc[4] += cv * (f * (3.0 - 2.0 * ar2));
          }
        }
      }
    }
#pragma unroll
    for (int c = 0; c < 5; ++c) s_rad[i][sl][c] = (R)acc[c];
  }
  __syncthreads();

  // ---- Phase A: one thread per (point, 8-AO chunk)
  const int width = tile.y - tile.x;
  const int chunks = (width + 7) >> 3;
  for (int u = tid; u < TP * chunks; u += kThreads) {
    const int i = u / chunks, j = u - i * chunks;
    const int64_t p = p0 + i;
    if (p >= P) continue;
    const int k0 = tile.x + 8 * j;
    if constexpr (MODE == 0) {
      // FP64: two AOs at a time, stored as double2 per component row
      double* o = (double*)out;
      const bool vec = ((ld & 1) == 0);
#pragma unroll
      for (int t = 0; t < 8; t += 2) {
        R v0[5] = {R(0), R(0), R(0), R(0), R(0)}, v1[5] = {R(0), R(0), R(0), R(0), R(0)};
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int k = k0 + t + h;
          if (k < tile.y) {
            const int code = Tl.ao_tcode[k];
            const int sl = (code >> 16) & 31, nl = (code >> 21) & 31;
            const double dx = s_pts[0][i] - s_nuc[nl][0];
            const double dy = s_pts[1][i] - s_nuc[nl][1];
            const double dz = s_pts[2][i] - s_nuc[nl][2];
            ao_vgl_one<R, COMPS>(code, (R)T.ao_factor[k], &s_rad[i][sl][0], (R)dx, (R)dy, (R)dz, R(kShift),
                                 h ? v1 : v0);
          }
        }
        const int k = k0 + t;
#pragma unroll
        for (int c = 0; c < COMPS; ++c) {
          double* row = o + (p * COMPS + c) * ld + k;
          if (vec && k + 1 < tile.y) {
            *reinterpret_cast<double2*>(row) = make_double2((double)v0[c], (double)v1[c]);
          } else {
            if (k < tile.y) row[0] = (double)v0[c];
            if (k + 1 < tile.y) row[1] = (double)v1[c];
          }
        }
      }
    } else {
    R vals[8][COMPS];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      const int k = k0 + t;
      R v[5] = {R(0), R(0), R(0), R(0), R(0)};
      if (k < tile.y) {
        const int code = Tl.ao_tcode[k];
        const int sl = (code >> 16) & 31, nl = (code >> 21) & 31;
        const double dx = s_pts[0][i] - s_nuc[nl][0];
        const double dy = s_pts[1][i] - s_nuc[nl][1];
        const double dz = s_pts[2][i] - s_nuc[nl][2];
        ao_vgl_one<R, COMPS>(code, (R)T.ao_factor[k], &s_rad[i][sl][0], (R)dx, (R)dy, (R)dz, R(0), v);
      }
#pragma unroll
      for (int c = 0; c < COMPS; ++c) vals[t][c] = v[c];
    }
    {
      constexpr int PIECES = MODE == 0 ? 2 : MODE;
      uint16_t* a = (uint16_t*)out;
      float inv[5];
      load_inv_scales<COMPS>(scales, inv);
#pragma unroll
      for (int c = 0; c < COMPS; ++c) {
        uint32_t pk[PIECES][4];
#pragma unroll
        for (int t = 0; t < 8; t += 2) {
          uint32_t q3[3];
          split_pair<PIECES>((float)vals[t][c], (float)vals[t + 1][c], inv[c], q3);
#pragma unroll
          for (int q = 0; q < PIECES; ++q) pk[q][t >> 1] = q3[q];
        }
        const int64_t off = (p * COMPS + c) * ld + k0;   // k0 multiple of 8, ld multiple of 64
#pragma unroll
        for (int q = 0; q < PIECES; ++q)
          *reinterpret_cast<uint4*>(a + q * piece_stride + off) = make_uint4(pk[q][0], pk[q][1], pk[q][2], pk[q][3]);
      }
    }
    }
  }
}

template <int MODE, int COMPS>
cudaError_t launch(const DevTables& T, const AoTiles& Tl, int64_t P, const double* coord, double cutoff, bool dp_exp,
                   void* out, int64_t ld, int64_t piece_stride, const double* scales, cudaStream_t s) {
  if (P <= 0) return cudaSuccess;
  const int64_t ptiles = (P + TP - 1) / TP;
  if (ptiles > 0x7fffffff || Tl.ntiles > 65535) return cudaErrorInvalidValue;
  dim3 grid((unsigned)ptiles, (unsigned)Tl.ntiles);
  ao_tile_kernel<MODE, COMPS><<<grid, kThreads, 0, s>>>(T, Tl, P, coord, cutoff, dp_exp, out, ld, piece_stride, scales);
  count_launch();
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_ao_tile_f64(const DevTables& T, const AoTiles& Tl, int64_t P, const double* coord, double cutoff,
                               bool dp_exp, int comps, double* out, cudaStream_t s) {
  const int64_t ld = T.ao_num;
  return comps == 5 ? launch<0, 5>(T, Tl, P, coord, cutoff, dp_exp, out, ld, 0, nullptr, s)
                    : launch<0, 1>(T, Tl, P, coord, cutoff, dp_exp, out, ld, 0, nullptr, s);
}

cudaError_t launch_ao_tile_split(const DevTables& T, const AoTiles& Tl, int64_t P, const double* coord, double cutoff,
                                 int comps, int pieces, const double* scales, void* a, int64_t lda,
                                 int64_t piece_stride, cudaStream_t s) {
  if (pieces != 3) return cudaErrorInvalidValue;   // 3 bfloat16 pieces (unfused organisation)
  return comps == 5 ? launch<3, 5>(T, Tl, P, coord, cutoff, false, a, lda, piece_stride, scales, s)
                    : launch<3, 1>(T, Tl, P, coord, cutoff, false, a, lda, piece_stride, scales, s);
}

}  // namespace qb
