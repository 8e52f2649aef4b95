// Cusp adjustment of the MOs and point-nucleus distances.
//
// With radii r_cusp set (qmckl_set_mo_basis_r_cusp, org/qmckl_mo.org:479-700)
// the MO of a point closer to nucleus A than r_cusp[A] leaves out A's s AOs
// (the AO producers zero them, cusp_masked in kernels.cuh) and gains A's
// cubic  c0 + c1 r + c2 r^2 + c3 r^3  with c = cusp_param[A][0..3][mo]:
//   value      (qmckl_compute_mo_basis_mo_value_cusp_doc, 2807-2860, r <= r_cusp)
//   VGL        (qmckl_compute_mo_basis_mo_vgl_cusp_doc, 3099-3185, r < r_cusp):
//              gradient (c1/r + 2 c2 + 3 c3 r) (r - R_A),
//              Laplacian 2 c1/r + 6 c2 + 12 c3 r
//   Hessian    (qmckl_compute_mo_basis_mo_hessian_cusp_doc_f, 2629-2697):
//              d_k d_j = -c1 x_k x_j / r^3 + 3 c3 x_k x_j / r
//                        + delta_kj (c1 / r + 2 c2 + 3 c3 r)
// These kernels add the cubics after the MO contraction, nucleus by nucleus
// in ascending order as the reference does.  One warp per point: the lanes
// test 32 nuclei at a time, then sweep the MOs of each nucleus in range.
#include <algorithm>
#include <cmath>

#include "kernels.cuh"

namespace qb {
namespace {

constexpr int kCuspWarps = 8;

// distance from nucleus n to the point (the reference's en_distance: x = R - r)
__device__ __forceinline__ double en_dist(const double* nucl, int N, int n, double px, double py, double pz) {
  const double x = nucl[n] - px, y = nucl[n + N] - py, z = nucl[n + 2 * N] - pz;
  return sqrt(x * x + y * y + z * z);
}

template <int COMPS>
__global__ void __launch_bounds__(kCuspWarps * 32)
cusp_mo_kernel(const int64_t P, const double* __restrict__ coord, const int64_t cstride, const int N,
               const double* __restrict__ nucl, const double* __restrict__ r_cusp, const double* __restrict__ prm,
               const int M, double* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * kCuspWarps;
  for (int64_t p = (int64_t)blockIdx.x * kCuspWarps + (threadIdx.x >> 5); p < P; p += warps) {
    const double px = coord[p], py = coord[p + cstride], pz = coord[p + 2 * cstride];
    double* o = out + p * COMPS * M;
    for (int n0 = 0; n0 < N; n0 += 32) {
      const int n = n0 + lane;
      double r = 0.0;
      bool in = false;
      if (n < N) {
        r = en_dist(nucl, N, n, px, py, pz);
        in = COMPS == 1 ? (r <= r_cusp[n]) : (r < r_cusp[n]);
      }
      unsigned int hits = __ballot_sync(0xffffffffu, in);
      while (hits != 0u) {
        const int src = __ffs(hits) - 1;
        hits &= hits - 1u;
        const int a = n0 + src;
        const double ra = __shfl_sync(0xffffffffu, r, src);
        const double* c = prm + (int64_t)a * 4 * M;
        if (COMPS == 1) {
          for (int i = lane; i < M; i += 32) o[i] += c[i] + ra * (c[M + i] + ra * (c[2 * M + i] + ra * c[3 * M + i]));
        } else {
          const double vx = px - nucl[a], vy = py - nucl[a + N], vz = pz - nucl[a + 2 * N];
          const double rinv = 1.0 / ra;
          for (int i = lane; i < M; i += 32) {
            const double c0 = c[i], c1 = c[M + i], c2 = c[2 * M + i], c3 = c[3 * M + i];
            o[i] += c0 + ra * (c1 + ra * (c2 + ra * c3));
            const double g = rinv * c1 + 2.0 * c2 + ra * 3.0 * c3;
            o[M + i] += vx * g;
            o[2 * M + i] += vy * g;
            o[3 * M + i] += vz * g;
            o[4 * M + i] += 2.0 * c1 * rinv + 6.0 * c2 + 12.0 * c3 * ra;
          }
        }
      }
    }
  }
}

__global__ void __launch_bounds__(kCuspWarps * 32)
cusp_hessian_kernel(const int64_t P, const double* __restrict__ coord, const int N, const double* __restrict__ nucl,
                    const double* __restrict__ r_cusp, const double* __restrict__ prm, const int M,
                    double* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * kCuspWarps;
  for (int64_t p = (int64_t)blockIdx.x * kCuspWarps + (threadIdx.x >> 5); p < P; p += warps) {
    const double pt[3] = {coord[p], coord[p + P], coord[p + 2 * P]};
    for (int n0 = 0; n0 < N; n0 += 32) {
      const int n = n0 + lane;
      double r = 0.0;
      bool in = false;
      if (n < N) {
        r = en_dist(nucl, N, n, pt[0], pt[1], pt[2]);
        in = r < r_cusp[n];
      }
      unsigned int hits = __ballot_sync(0xffffffffu, in);
      while (hits != 0u) {
        const int src = __ffs(hits) - 1;
        hits &= hits - 1u;
        const int a = n0 + src;
        const double ra = __shfl_sync(0xffffffffu, r, src);
        const double rv[3] = {pt[0] - nucl[a], pt[1] - nucl[a + N], pt[2] - nucl[a + 2 * N]};
        const double rinv = 1.0 / ra;
        const double rinv3 = rinv * rinv * rinv;
        const double* c = prm + (int64_t)a * 4 * M;
        for (int jj = 0; jj < 3; ++jj)
          for (int kk = 0; kk < 3; ++kk) {
            double* o = out + ((int64_t)(jj * P + p) * 3 + kk) * M;
            for (int i = lane; i < M; i += 32) {
              const double c1 = c[M + i], c3 = c[3 * M + i];
              double v = o[i] - c1 * rv[kk] * rv[jj] * rinv3 + c3 * 3.0 * rv[kk] * rv[jj] * rinv;
              if (kk == jj) v = v + c1 * rinv + c[2 * M + i] * 2.0 + c3 * 3.0 * ra;
              o[i] = v;
            }
          }
      }
    }
  }
}

__global__ void en_distance_kernel(const int64_t P, const double* __restrict__ coord, const int N,
                                   const double* __restrict__ nucl, double* __restrict__ out) {
  const int64_t total = P * (int64_t)N;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = i / N;
    const int n = (int)(i - p * N);
    out[i] = en_dist(nucl, N, n, coord[p], coord[p + P], coord[p + 2 * P]);
  }
}

int warp_grid(int64_t P) { return (int)std::min<int64_t>((P + kCuspWarps - 1) / kCuspWarps, 148 * 16); }

}  // namespace

cudaError_t launch_cusp_mo(int64_t P, int comps, const double* coord, int64_t cstride, int N, const double* nucl,
                           const double* r_cusp, const double* prm, int M, double* out, cudaStream_t s) {
  if (P <= 0 || N <= 0 || M <= 0) return cudaSuccess;
  if (comps != 1 && comps != 5) return cudaErrorInvalidValue;
  if (cstride < P) cstride = P;
  if (comps == 1)
    cusp_mo_kernel<1><<<warp_grid(P), kCuspWarps * 32, 0, s>>>(P, coord, cstride, N, nucl, r_cusp, prm, M, out);
  else
    cusp_mo_kernel<5><<<warp_grid(P), kCuspWarps * 32, 0, s>>>(P, coord, cstride, N, nucl, r_cusp, prm, M, out);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_cusp_hessian(int64_t P, const double* coord, int N, const double* nucl, const double* r_cusp,
                                const double* prm, int M, double* out, cudaStream_t s) {
  if (P <= 0 || N <= 0 || M <= 0) return cudaSuccess;
  cusp_hessian_kernel<<<warp_grid(P), kCuspWarps * 32, 0, s>>>(P, coord, N, nucl, r_cusp, prm, M, out);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_en_distance(int64_t P, const double* coord, int N, const double* nucl, double* out,
                               cudaStream_t s) {
  if (P <= 0 || N <= 0) return cudaSuccess;
  const int64_t total = P * (int64_t)N;
  const int grid = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
  en_distance_kernel<<<grid, 256, 0, s>>>(P, coord, N, nucl, out);
  count_launch();
  return cudaGetLastError();
}

}  // namespace qb
