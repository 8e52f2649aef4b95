// FP64 MO contraction: C[M][N] = A[M][K] * B[K][N] (row-major).
//
// For MO VGL, A is ao_vgl viewed as a (5*point_num) x ao_num matrix, B is
// coefficient_t [ao][mo] and C is mo_vgl viewed as (5*point_num) x mo_num; for
// MO value the same with ao_value / mo_value.  This is the dense form of
// qmckl_compute_mo_basis_mo_vgl_hpc (org/qmckl_mo.org:2015-2163): the
// reference skips AOs whose value is exactly zero, whose products are exact
// zeros, so only the summation order differs.
//
// The FP64 form runs on the FP64 tensor pipe (mma.sync m8n8k4 f64, the only
// FP64 MMA on sm_100a; tcgen05 has no FP64 kind).  CTA tile 128 x (8*NT*2),
// BK = 16, 8 warps as 4 (M) x 2 (N), each warp 32 x 8*NT, operands staged in
// shared memory by a 3-stage cp.async pipeline with zero-filled edges.
#include <algorithm>

#include "kernels.cuh"

namespace qb {
namespace {

constexpr int BM = 128, BK = 16, STAGES = 3;
constexpr int LDA_S = BK + 4;  // padded smem row stride (doubles) of the A tile

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src), "r"(bytes));
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src, int bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_u32(dst)), "l"(src), "r"(bytes));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// TA: A is stored transposed (element (m, k) at A[k * lda + m]); its shared
// tile is then kept k-major ([BK][BM + 4]).  Split K (TA only): CTA z of the
// grid covers k in [z * k_split, (z + 1) * k_split) and writes C + z * c_split.
template <int NT, int VA, int VB, bool TA>
__global__ void __launch_bounds__(256)
dgemm_kernel(int64_t M, int64_t N, int64_t K, const double* __restrict__ A_, int64_t lda,
             const double* __restrict__ B_, int64_t ldb, double* __restrict__ C_, int64_t ldc, int64_t k_split,
             int64_t c_split) {
  constexpr int BN = 16 * NT;
  constexpr int LDB_S = BN + 4;
  constexpr int LDT = BM + 4;                      // row stride of the k-major A tile (TA)
  extern __shared__ __align__(16) double smem[];
  double* As = smem;                               // [STAGES][BM][LDA_S] or [STAGES][BK][LDT]
  double* Bs = smem + STAGES * BM * LDA_S;         // [STAGES][BK][LDB_S]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp & 3, wn = warp >> 2;
  const int g = lane >> 2, t = lane & 3;
  const int64_t n0 = (int64_t)blockIdx.x * BN;
  const double* __restrict__ A = A_;
  const double* __restrict__ B = B_;
  double* __restrict__ C = C_;
  if constexpr (TA) {   // split K (used with the transposed form only)
    const int64_t kz0 = (int64_t)blockIdx.z * k_split;
    // an empty K range (last splits of a short K) still writes its zero slice
    K = kz0 >= K ? 0 : ((K - kz0) < k_split ? (K - kz0) : k_split);
    A = A_ + kz0 * lda;
    B = B_ + kz0 * ldb;
    C = C_ + (int64_t)blockIdx.z * c_split;
  }
  const int ktiles = (int)((K + BK - 1) / BK);

  for (int64_t mt = blockIdx.y; mt * BM < M; mt += gridDim.y) {
    const int64_t m0 = mt * BM;
    double acc[4][NT][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < NT; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    auto load_tile = [&](int kt, int st) {
      const int64_t k0 = (int64_t)kt * BK;
      double* as = As + st * BM * LDA_S;
      double* bs = Bs + st * BK * LDB_S;
      // A tile: BM x BK
      constexpr int ACH = BM * BK / VA;
      if constexpr (TA) {
#pragma unroll
        for (int i = 0; i < ACH / 256; ++i) {
          const int c = tid + i * 256;
          const int kr = c / (BM / VA), mc = (c % (BM / VA)) * VA;
          const int64_t gm = m0 + mc, gk = k0 + kr;
          int bytes = 0;
          if (gm < M && gk < K) bytes = (int)((M - gm) < VA ? (M - gm) : VA) * 8;
          const double* src = bytes ? A + gk * lda + gm : A;
          if (VA == 2) cp_async16(as + kr * LDT + mc, src, bytes);
          else cp_async8(as + kr * LDT + mc, src, bytes);
        }
      } else {
#pragma unroll
        for (int i = 0; i < ACH / 256; ++i) {
          const int c = tid + i * 256;
          const int row = c / (BK / VA), col = (c % (BK / VA)) * VA;
          const int64_t gm = m0 + row, gk = k0 + col;
          int bytes = 0;
          if (gm < M && gk < K) bytes = (int)((K - gk) < VA ? (K - gk) : VA) * 8;
          const double* src = bytes ? A + gm * lda + gk : A;
          if (VA == 2) cp_async16(as + row * LDA_S + col, src, bytes);
          else cp_async8(as + row * LDA_S + col, src, bytes);
        }
      }
      // B tile: BK x BN
      constexpr int BCH = BK * BN / VB;
      for (int c = tid; c < BCH; c += 256) {
        const int row = c / (BN / VB), col = (c % (BN / VB)) * VB;
        const int64_t gk = k0 + row, gn = n0 + col;
        int bytes = 0;
        if (gk < K && gn < N) bytes = (int)((N - gn) < VB ? (N - gn) : VB) * 8;
        const double* src = bytes ? B + gk * ldb + gn : B;
        if (VB == 2) cp_async16(bs + row * LDB_S + col, src, bytes);
        else cp_async8(bs + row * LDB_S + col, src, bytes);
      }
    };

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
      if (s < ktiles) load_tile(s, s);
      cp_commit();
    }
    for (int kt = 0; kt < ktiles; ++kt) {
      cp_wait<STAGES - 2>();
      __syncthreads();
      const int nk = kt + STAGES - 1;
      if (nk < ktiles) load_tile(nk, nk % STAGES);
      cp_commit();
      const double* as = As + (kt % STAGES) * BM * LDA_S;
      const double* bs = Bs + (kt % STAGES) * BK * LDB_S + wn * (8 * NT);
#pragma unroll
      for (int kk = 0; kk < BK; kk += 4) {
        double af[4], bf[NT];
#pragma unroll
        for (int i = 0; i < 4; ++i)
          af[i] = TA ? as[(kk + t) * LDT + wm * 32 + i * 8 + g] : as[(wm * 32 + i * 8 + g) * LDA_S + kk + t];
#pragma unroll
        for (int j = 0; j < NT; ++j) bf[j] = bs[(kk + t) * LDB_S + j * 8 + g];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < NT; ++j) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
      }
    }
    cp_wait<0>();
    __syncthreads();
    // epilogue: each thread owns rows g of 8-row tiles, columns 2t, 2t+1
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int64_t m = m0 + wm * 32 + i * 8 + g;
      if (m >= M) continue;
      double* crow = C + m * ldc;
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        const int64_t n = n0 + wn * (8 * NT) + j * 8 + 2 * t;
        if (n + 1 < N && ((ldc & 1) == 0)) {
          *reinterpret_cast<double2*>(crow + n) = make_double2(acc[i][j][0], acc[i][j][1]);
        } else {
          if (n < N) crow[n] = acc[i][j][0];
          if (n + 1 < N) crow[n + 1] = acc[i][j][1];
        }
      }
    }
  }
}

template <int NT, int VA, int VB, bool TA>
cudaError_t run(int64_t M, int64_t N, int64_t K, const double* A, int64_t lda, const double* B,
                int64_t ldb, double* C, int64_t ldc, int splits, cudaStream_t s) {
  constexpr int BN = 16 * NT;
  const size_t smem = sizeof(double) * STAGES * (BM * LDA_S + BK * (BN + 4));
  auto kern = dgemm_kernel<NT, VA, VB, TA>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int64_t mt = (M + BM - 1) / BM;
  const int64_t k_split = ((K + splits - 1) / splits + BK - 1) / BK * BK;
  dim3 grid((unsigned)((N + BN - 1) / BN), (unsigned)std::min<int64_t>(mt, 65535), (unsigned)splits);
  kern<<<grid, 256, smem, s>>>(M, N, K, A, lda, B, ldb, C, ldc, k_split, M * ldc);
  count_launch();
  return cudaGetLastError();
}

template <int NT, bool TA>
cudaError_t run_nt(int64_t M, int64_t N, int64_t K, const double* A, int64_t lda, const double* B,
                   int64_t ldb, double* C, int64_t ldc, int splits, cudaStream_t s) {
  const bool va = (lda % 2 == 0) && ((uintptr_t)A % 16 == 0);
  const bool vb = (ldb % 2 == 0) && ((uintptr_t)B % 16 == 0);
  if (va && vb) return run<NT, 2, 2, TA>(M, N, K, A, lda, B, ldb, C, ldc, splits, s);
  if (va) return run<NT, 2, 1, TA>(M, N, K, A, lda, B, ldb, C, ldc, splits, s);
  if (vb) return run<NT, 1, 2, TA>(M, N, K, A, lda, B, ldb, C, ldc, splits, s);
  return run<NT, 1, 1, TA>(M, N, K, A, lda, B, ldb, C, ldc, splits, s);
}

template <bool TA>
cudaError_t run_any(int64_t M, int64_t N, int64_t K, const double* A, int64_t lda, const double* B, int64_t ldb,
                    double* C, int64_t ldc, int splits, cudaStream_t s) {
  if (M <= 0 || N <= 0) return cudaSuccess;
  if (!TA && splits != 1) return cudaErrorInvalidValue;
  // pick the N tile (64 or 80 columns) that wastes fewer padded columns
  const int64_t w64 = ((N + 63) / 64) * 64 - N, w80 = ((N + 79) / 80) * 80 - N;
  if (w80 < w64) return run_nt<5, TA>(M, N, K, A, lda, B, ldb, C, ldc, splits, s);
  return run_nt<4, TA>(M, N, K, A, lda, B, ldb, C, ldc, splits, s);
}

// Tile-sparse FP64 MO contraction.  Rows are (point, component) pairs of
// tiles of PTS points in the spatial order perm (125 of the 128 tile rows
// for VGL, 128 for values).  The K dimension of a tile is its list of live
// AOs (tlist, made by f64_plan_kernel): the AOs of the shells that do not
// vanish at some point of the tile, in the basis order, padded with -1 to a
// multiple of 16.  An AO left out is an exact zero at every point of the
// tile, so the sum is the dense one in the basis order, without its zero
// terms (the order of the reference's own contraction,
// org/qmckl_mo.org:2015-2163, which skips the zero AOs of each point).
//   ao    [P][COMPS][lda]    the AO matrix in the basis order (FP64 kernel)
//   tlist [tiles][kmax]      live AOs of each tile, tcount[tile] entries
//   Bt    [ao][ldb]          coefficient_t (ldb even, 16-byte aligned rows)
//   out   [P][COMPS][ldc]
// A and B tiles are gathered by the list with cp.async (8-byte elements for
// A, 16-byte pairs of B rows); 128 x (16 NT) tiles, BK = 16, 3 stages, 8
// warps as 4 (M) x 2 (N), mma.sync m8n8k4 f64 as the dense kernel.
template <int NT, int COMPS>
__global__ void __launch_bounds__(256)
sparse_dgemm_kernel(int64_t P, int64_t N, const double* __restrict__ ao, int64_t lda, const int* __restrict__ perm,
                    const int* __restrict__ tlist, const int* __restrict__ tcount, int64_t kmax,
                    const double* __restrict__ Bt, int64_t ldb, double* __restrict__ C, int64_t ldc, int64_t ntiles) {
  constexpr int PTS = BM / COMPS;
  constexpr int BN = 16 * NT;
  constexpr int LDB_S = BN + 4;
  extern __shared__ __align__(16) double smem[];
  double* As = smem;                               // [STAGES][BM][LDA_S]
  double* Bs = smem + STAGES * BM * LDA_S;         // [STAGES][BK][LDB_S]
  __shared__ const double* rowp[BM];               // source row of each tile row (null: padding)
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp & 3, wn = warp >> 2;
  const int g = lane >> 2, t = lane & 3;
  const int64_t n0 = (int64_t)blockIdx.x * BN;

  for (int64_t tile = blockIdx.y; tile < ntiles; tile += gridDim.y) {
    const int64_t p0 = tile * PTS;
    const int* kl = tlist + tile * kmax;
    if (tid < BM) {
      const int i = tid / COMPS, c = tid - i * COMPS;
      const double* r = nullptr;
      if (i < PTS && p0 + i < P) r = ao + ((int64_t)perm[p0 + i] * COMPS + c) * lda;
      rowp[tid] = r;
    }
    __syncthreads();
    const int ktiles = tcount[tile] / BK;
    double acc[4][NT][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < NT; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    auto load_tile = [&](int kt, int st) {
      const int* kk = kl + kt * BK;
      double* as = As + st * BM * LDA_S;
      double* bs = Bs + st * BK * LDB_S;
#pragma unroll
      for (int i = 0; i < BM * BK / 256; ++i) {
        const int c = tid + i * 256;
        const int row = c / BK, col = c % BK;
        const double* r = rowp[row];
        const int k = kk[col];
        const bool ok = r != nullptr && k >= 0;
        cp_async8(as + row * LDA_S + col, ok ? r + k : ao, ok ? 8 : 0);
      }
      constexpr int BCH = BK * BN / 2;
      for (int c = tid; c < BCH; c += 256) {
        const int row = c / (BN / 2), col = (c % (BN / 2)) * 2;
        const int64_t gn = n0 + col;
        const int k = kk[row];
        const int bytes = (k >= 0 && gn < N) ? (int)((N - gn) < 2 ? (N - gn) : 2) * 8 : 0;
        cp_async16(bs + row * LDB_S + col, bytes ? Bt + (int64_t)k * ldb + gn : Bt, bytes);
      }
    };

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
      if (s < ktiles) load_tile(s, s);
      cp_commit();
    }
    for (int kt = 0; kt < ktiles; ++kt) {
      cp_wait<STAGES - 2>();
      __syncthreads();
      const int nk = kt + STAGES - 1;
      if (nk < ktiles) load_tile(nk, nk % STAGES);
      cp_commit();
      const double* as = As + (kt % STAGES) * BM * LDA_S;
      const double* bs = Bs + (kt % STAGES) * BK * LDB_S + wn * (8 * NT);
#pragma unroll
      for (int kk = 0; kk < BK; kk += 4) {
        double af[4], bf[NT];
#pragma unroll
        for (int i = 0; i < 4; ++i) af[i] = as[(wm * 32 + i * 8 + g) * LDA_S + kk + t];
#pragma unroll
        for (int j = 0; j < NT; ++j) bf[j] = bs[(kk + t) * LDB_S + j * 8 + g];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < NT; ++j) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
      }
    }
    cp_wait<0>();
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = wm * 32 + i * 8 + g;
      if (rowp[r] == nullptr) continue;
      const int ip = r / COMPS, c = r - ip * COMPS;
      double* crow = C + ((int64_t)perm[p0 + ip] * COMPS + c) * ldc;
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        const int64_t n = n0 + wn * (8 * NT) + j * 8 + 2 * t;
        if (n + 1 < N && ((ldc & 1) == 0)) {
          *reinterpret_cast<double2*>(crow + n) = make_double2(acc[i][j][0], acc[i][j][1]);
        } else {
          if (n < N) crow[n] = acc[i][j][0];
          if (n + 1 < N) crow[n + 1] = acc[i][j][1];
        }
      }
    }
    __syncthreads();   // rowp is rewritten for the next tile
  }
}

// The live-AO list of each tile of PTS points (in the order perm): one CTA
// per tile tests every shell's screening sphere (sph[s] = nucleus, squared
// radius beyond which the shell's AOs are exact zeros) against the tile's
// points, then writes the AOs of the live shells in the basis order
// (shell_ao[s] = first AO, AO count), padded with -1 to a multiple of 16.
// Scratch: dynamic shared memory of 2 * shell_num ints.
template <int PTS>
__global__ void __launch_bounds__(256)
f64_plan_kernel(int64_t P, const double* __restrict__ coord, int64_t cstride, const int* __restrict__ perm,
                int shell_num, const double4* __restrict__ sph, const int2* __restrict__ shell_ao,
                int* __restrict__ tlist, int* __restrict__ tcount, int64_t kmax) {
  __shared__ double spts[3 * PTS];
  __shared__ int wsum[8];
  extern __shared__ int sbuf[];   // [shell_num] live AO counts, then [shell_num] list positions
  int* cnt = sbuf;
  int* pos = sbuf + shell_num;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t tile = blockIdx.x;
  const int64_t p0 = tile * PTS;
  const int np = (int)(P - p0 < PTS ? P - p0 : PTS);
  for (int t = tid; t < 3 * PTS; t += blockDim.x) {
    const int d = t / PTS, i = t - d * PTS;
    spts[t] = i < np ? coord[(int64_t)perm[p0 + i] + d * cstride] : 0.0;
  }
  __syncthreads();
  for (int s = tid; s < shell_num; s += blockDim.x) {
    const double4 c = sph[s];
    bool live = false;
    for (int i = 0; i < np && !live; ++i) {
      const double x = spts[i] - c.x, y = spts[PTS + i] - c.y, z = spts[2 * PTS + i] - c.z;
      live = x * x + y * y + z * z <= c.w;
    }
    cnt[s] = live ? shell_ao[s].y : 0;
  }
  __syncthreads();
  // exclusive scan of cnt: thread tid owns shells [tid * per, (tid + 1) * per)
  const int per = (shell_num + 255) / 256;
  const int s0 = tid * per, s1 = min(shell_num, s0 + per);
  int local = 0;
  for (int s = s0; s < s1; ++s) local += cnt[s];
  int incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  int base = 0;
  for (int w = 0; w < warp; ++w) base += wsum[w];
  int total = 0;
  for (int w = 0; w < 8; ++w) total += wsum[w];
  int run = base + incl - local;
  for (int s = s0; s < s1; ++s) {
    pos[s] = run;
    run += cnt[s];
  }
  __syncthreads();
  int* out = tlist + tile * kmax;
  for (int s = tid; s < shell_num; s += blockDim.x) {
    const int n = cnt[s], a0 = shell_ao[s].x, q = pos[s];
    for (int k = 0; k < n; ++k) out[q + k] = a0 + k;
  }
  const int padded = (total + 15) / 16 * 16;
  for (int q = total + tid; q < padded; q += blockDim.x) out[q] = -1;
  if (tid == 0) tcount[tile] = padded;
}

template <int NT, int COMPS>
cudaError_t run_sparse(int64_t P, int64_t N, const double* ao, int64_t lda, const int* perm, const int* tlist,
                       const int* tcount, int64_t kmax, const double* Bt, int64_t ldb, double* C, int64_t ldc,
                       cudaStream_t s) {
  constexpr int BN = 16 * NT;
  constexpr int PTS = BM / COMPS;
  const size_t smem = sizeof(double) * STAGES * (BM * LDA_S + BK * (BN + 4));
  auto kern = sparse_dgemm_kernel<NT, COMPS>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int64_t ntiles = (P + PTS - 1) / PTS;
  dim3 grid((unsigned)((N + BN - 1) / BN), (unsigned)std::min<int64_t>(ntiles, 65535));
  kern<<<grid, 256, smem, s>>>(P, N, ao, lda, perm, tlist, tcount, kmax, Bt, ldb, C, ldc, ntiles);
  count_launch();
  return cudaGetLastError();
}

// out[n][m] (+)= sum_z part[z][m][n], through 32 x 32 shared tiles
__global__ void add_transposed_kernel(const double* __restrict__ part, int splits, int64_t M, int64_t N,
                                      double* __restrict__ out, bool accumulate) {
  __shared__ double tile[32][33];
  const int64_t m0 = (int64_t)blockIdx.y * 32, n0 = (int64_t)blockIdx.x * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int64_t m = m0 + r, n = n0 + threadIdx.x;
    double v = 0.0;
    if (m < M && n < N)
      for (int z = 0; z < splits; ++z) v += part[((int64_t)z * M + m) * N + n];
    tile[r][threadIdx.x] = v;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int64_t n = n0 + r, m = m0 + threadIdx.x;
    if (m < M && n < N) {
      double* o = out + n * M + m;
      *o = accumulate ? *o + tile[threadIdx.x][r] : tile[threadIdx.x][r];
    }
  }
}

}  // namespace

cudaError_t launch_gemm_f64(int64_t M, int64_t N, int64_t K, const double* A, int64_t lda,
                            const double* B, int64_t ldb, double* C, int64_t ldc, cudaStream_t s) {
  return run_any<false>(M, N, K, A, lda, B, ldb, C, ldc, 1, s);
}

cudaError_t launch_gemm_f64_tn_split(int64_t M, int64_t N, int64_t K, const double* A, int64_t lda, const double* B,
                                     int64_t ldb, double* part, int splits, cudaStream_t s) {
  if (splits < 1) return cudaErrorInvalidValue;
  return run_any<true>(M, N, K, A, lda, B, ldb, part, N, splits, s);
}

int64_t f64_plan_kmax(int64_t ao_num) { return (ao_num + 15) / 16 * 16; }

size_t f64_plan_bytes(int64_t point_num, int comps, int64_t ao_num) {
  const int pts = BM / comps;
  const int64_t tiles = (point_num + pts - 1) / pts;
  return sizeof(int) * (size_t)tiles * (size_t)(f64_plan_kmax(ao_num) + 1);
}

cudaError_t launch_f64_plan(int64_t point_num, int comps, const double* coord, int64_t cstride, const int* perm,
                            int shell_num, const void* sph, const void* shell_ao, int64_t ao_num, void* plan,
                            cudaStream_t s) {
  if (point_num <= 0) return cudaSuccess;
  if (comps != 1 && comps != 5) return cudaErrorInvalidValue;
  if (cstride < point_num) cstride = point_num;
  const int pts = BM / comps;
  const int64_t tiles = (point_num + pts - 1) / pts;
  const int64_t kmax = f64_plan_kmax(ao_num);
  int* tcount = (int*)plan;
  int* tlist = tcount + tiles;
  const size_t sm = sizeof(int) * 2 * (size_t)shell_num;
  if (sm > 200 * 1024) return cudaErrorInvalidValue;
  auto kern5 = f64_plan_kernel<BM / 5>;
  auto kern1 = f64_plan_kernel<BM>;
  cudaError_t e = cudaFuncSetAttribute(comps == 5 ? kern5 : kern1, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)std::max<size_t>(sm, 1));
  if (e != cudaSuccess) return e;
  if (comps == 5)
    kern5<<<(unsigned)tiles, 256, sm, s>>>(point_num, coord, cstride, perm, shell_num, (const double4*)sph,
                                           (const int2*)shell_ao, tlist, tcount, kmax);
  else
    kern1<<<(unsigned)tiles, 256, sm, s>>>(point_num, coord, cstride, perm, shell_num, (const double4*)sph,
                                           (const int2*)shell_ao, tlist, tcount, kmax);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_gemm_f64_sparse(int64_t point_num, int comps, int64_t N, const double* ao, int64_t lda,
                                   const int* perm, const void* plan, int64_t ao_num, const double* Bt, int64_t ldb,
                                   double* C, int64_t ldc, cudaStream_t s) {
  if (point_num <= 0 || N <= 0) return cudaSuccess;
  if ((ldb & 1) != 0 || (reinterpret_cast<uintptr_t>(Bt) & 15) != 0) return cudaErrorInvalidValue;
  const int pts = BM / comps;
  const int64_t tiles = (point_num + pts - 1) / pts;
  const int* tcount = (const int*)plan;
  const int* tlist = tcount + tiles;
  const int64_t kmax = f64_plan_kmax(ao_num);
  // the N tile (64 or 80 columns) that wastes fewer padded columns
  const bool nt5 = ((N + 79) / 80) * 80 - N < ((N + 63) / 64) * 64 - N;
  if (comps == 5)
    return nt5 ? run_sparse<5, 5>(point_num, N, ao, lda, perm, tlist, tcount, kmax, Bt, ldb, C, ldc, s)
               : run_sparse<4, 5>(point_num, N, ao, lda, perm, tlist, tcount, kmax, Bt, ldb, C, ldc, s);
  if (comps == 1)
    return nt5 ? run_sparse<5, 1>(point_num, N, ao, lda, perm, tlist, tcount, kmax, Bt, ldb, C, ldc, s)
               : run_sparse<4, 1>(point_num, N, ao, lda, perm, tlist, tcount, kmax, Bt, ldb, C, ldc, s);
  return cudaErrorInvalidValue;
}

cudaError_t launch_add_transposed(const double* part, int splits, int64_t M, int64_t N, double* out, bool accumulate,
                                  cudaStream_t s) {
  if (M <= 0 || N <= 0) return cudaSuccess;
  dim3 grid((unsigned)((N + 31) / 32), (unsigned)((M + 31) / 32));
  add_transposed_kernel<<<grid, dim3(32, 8), 0, s>>>(part, splits, M, N, out, accumulate);
  count_launch();
  return cudaGetLastError();
}

}  // namespace qb
