// Mixed-precision MO contraction on tcgen05 tensor cores.
//
// mo[(p,c)][i] = sum_k A[(p,c)][k] * C[i][k], with A = ao_vgl viewed as a
// (comps*point_num) x ao_num matrix (qmckl_compute_mo_basis_mo_vgl_hpc,
// org/qmckl_mo.org:2015-2163, in dense form) and C = coefficient[mo][ao].
//
// Both operands are split into 16-bit pieces (split.cuh: 3 bfloat16 pieces,
// or 2 float16 pieces of power-of-two scaled values), the pieces of A
// produced by the mixed AO kernel and those of C once per coefficient
// update.  Products X_i*Y_j with i + j < pieces are accumulated in FP32 in
// tensor memory: 6 products for 3 bfloat16 pieces, 3 for 2 float16 pieces
// (both ~2^-22..2^-24 relative, below the FP32 rounding of the AOs).
// The rounding of the FP32 accumulation grows with the number of
// accumulation steps, so the leading product A1*C1 is accumulated in two
// accumulators (first and second half of K) and the correction products,
// 2^-8 smaller, in a third; the epilogue adds the three in FP64.
//
// GEMM kernel (one 128 x n_tile output tile per CTA):
//   warp 4      TMA producer: all A and C pieces of a 64-wide K block into a
//               stage (128B-swizzled, K-major), completion on full[stage]
//   warp 5      allocates TMEM, then one thread issues the tcgen05.mma chain
//               (4 K steps x products) and commits to empty[stage]; after the
//               last K block it commits to acc_full
//   warps 0..3  epilogue: tcgen05.ld 32 lanes each, FP32 -> FP64, staged in
//               shared memory and written as contiguous output rows
// Every mbarrier wait is bounded by a %globaltimer deadline; a timeout sets an
// error word that the host turns into QMCKL_FAILURE, and the CTA still frees
// its TMEM and exits.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ao_tile.cuh"
#include "mo_tc.cuh"
#include "split.cuh"
#include "tc_ptx.cuh"

namespace qb {

namespace {
using namespace tcx;

constexpr int BM = 128;          // rows per tile (tcgen05 M)
constexpr int BK = 64;           // K per stage: one 128-byte swizzle row of bf16
constexpr int UMMA_K = 16;       // K per tcgen05.mma of kind::f16
constexpr int kEpiWarps = 4;
constexpr int kThreads = 32 * (kEpiWarps + 2);


// ------------------------------------------------------------ GEMM kernel

// TWO_ACC: one accumulator for the leading product and one for the
// corrections (short K: the split of the leading product over two halves of
// K is not needed), so that a 128-column tile needs 256 TMEM columns and two
// CTAs share an SM.
template <int PIECES, int STAGES, typename OutT = double, bool TWO_ACC = false>
__global__ void __launch_bounds__(kThreads, TWO_ACC ? 2 : 1)
tc_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
               const int64_t M, const int n_out, const int n_tile, const int kblocks, const int comps,
               const double* __restrict__ scales, OutT* __restrict__ out, const int64_t ldo,
               int* __restrict__ err) {
  constexpr int NPROD = PIECES == 3 ? 6 : 3;
  constexpr int A_TILE = BM * BK * 2;             // bytes of one A piece tile
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // 1024-byte aligned base for the swizzled tiles
  // 1024-byte aligned base, kept as pointer arithmetic on the __shared__
  // array so that accesses compile to shared-memory (not generic) loads
  uint8_t* smem = smem_raw + ((1024u - (tcx::smem_addr(smem_raw) & 1023u)) & 1023u);
  const int B_TILE = n_tile * BK * 2;
  const int STAGE = PIECES * (A_TILE + B_TILE);
  uint64_t* full = (uint64_t*)(smem + STAGES * STAGE);
  uint64_t* empty = full + STAGES;
  uint64_t* acc_full = empty + STAGES;
  uint32_t* tmem_slot = (uint32_t*)(acc_full + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t m0 = (int64_t)blockIdx.x * BM;
  const int n0 = blockIdx.y * n_tile;
  // three accumulators of n_tile columns: A1*C1 (first half of K), A1*C1
  // (second half), corrections
  constexpr int NACC = TWO_ACC ? 2 : 3;
  uint32_t tmem_cols = 32;
  while ((int)tmem_cols < NACC * n_tile) tmem_cols <<= 1;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(acc_full, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == kEpiWarps + 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                 "r"(tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == kEpiWarps) {
    // ---------------- TMA producer
    if (lane == 0) {
      for (int kb = 0; kb < kblocks; ++kb) {
        const int s = kb % STAGES;
        const uint32_t phase = (uint32_t)(kb / STAGES) & 1u;
        if (!mbar_wait(&empty[s], phase ^ 1u, err, 1)) break;
        uint8_t* st = smem + s * STAGE;
        mbar_expect_tx(&full[s], (uint32_t)STAGE);
        for (int p = 0; p < PIECES; ++p) {
          tma_load_3d(st + p * A_TILE, &tmA, &full[s], kb * BK, (int)m0, p);
          tma_load_3d(st + PIECES * A_TILE + p * B_TILE, &tmB, &full[s], kb * BK, n0, p);
        }
      }
    }
  } else if (warp == kEpiWarps + 1) {
    // ---------------- MMA issuer
    if (lane == 0) {
      const uint32_t fmt = PIECES == 3 ? 1u : 0u;   // bfloat16 or float16 operands
      const uint32_t idesc = (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(n_tile >> 3) << 17) |
                             ((uint32_t)(BM >> 4) << 24);
      // products (i, j) with i + j < PIECES, smallest terms first
      constexpr int pa3[6] = {2, 1, 0, 1, 0, 0}, pb3[6] = {0, 1, 2, 0, 1, 0};
      constexpr int pa2[3] = {1, 0, 0}, pb2[3] = {0, 1, 0};
      bool ok = true;
      for (int kb = 0; kb < kblocks && ok; ++kb) {
        const int s = kb % STAGES;
        const uint32_t phase = (uint32_t)(kb / STAGES) & 1u;
        if (!mbar_wait(&full[s], phase, err, 2)) { ok = false; break; }
        tc_fence_after();
        const uint32_t base = smem_addr(smem + s * STAGE);
        for (int kk = 0; kk < BK / UMMA_K; ++kk) {
#pragma unroll
          for (int t = 0; t < NPROD; ++t) {
            const int ia = PIECES == 3 ? pa3[t] : pa2[t];
            const int ib = PIECES == 3 ? pb3[t] : pb2[t];
            const uint32_t a_addr = base + ia * A_TILE + kk * UMMA_K * 2;
            const uint32_t b_addr = base + PIECES * A_TILE + ib * B_TILE + kk * UMMA_K * 2;
            const bool lead = (t == NPROD - 1);                 // A1*C1
            const bool second = !TWO_ACC && lead && (2 * kb >= kblocks);
            const uint32_t d = tmem + (uint32_t)((lead ? (second ? 1 : 0) : NACC - 1) * n_tile);
            const bool first_use = lead ? (second ? (kb == (kblocks + 1) / 2 && kk == 0) : (kb == 0 && kk == 0))
                                        : (kb == 0 && kk == 0 && t == 0);
            umma_bf16(d, smem_desc(a_addr), smem_desc(b_addr), idesc, first_use ? 0u : 1u);
          }
        }
        umma_commit(&empty[s]);
      }
      umma_commit(acc_full);
    }
  } else {
    // ---------------- epilogue (warps 0..3, TMEM lanes 32*warp ..)
    bool ok = mbar_wait(acc_full, 0, err, 3);
    ok = __all_sync(0xffffffffu, ok && *(volatile int*)err == 0);   // warp-uniform for tcgen05.ld
    tc_fence_after();
    // When the tile's rows fit in the idle stage memory and are 16-byte
    // aligned in `out`, they are staged there (rows padded by 16 bytes, so a
    // warp's 16-byte stores fall on distinct banks) and each row leaves in
    // one bulk copy; otherwise each warp writes its rows through a small
    // staging buffer.
    constexpr int kPadT = 16 / (int)sizeof(OutT);
    const int ldst = n_tile + kPadT;
    const int ncols = n_out - n0 < n_tile ? n_out - n0 : n_tile;
    const bool bulk = (size_t)BM * ldst * sizeof(OutT) <= (size_t)STAGES * STAGE &&
                      ((size_t)ncols * sizeof(OutT)) % 16 == 0 && ((size_t)ldo * sizeof(OutT)) % 16 == 0 &&
                      (reinterpret_cast<uintptr_t>(out) & 15) == 0;
    if (bulk) {
      OutT* stg = (OutT*)smem;
      const int r = warp * 32 + lane;   // this thread's TMEM lane = tile row
      const int64_t row = m0 + r;
      const bool has_second = !TWO_ACC && kblocks >= 2;
      if (ok) {
        for (int c0 = 0; c0 < n_tile; c0 += 16) {
          uint32_t r0[16], r1[16], r2[16];
          const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
          tmem_ld16(ta, r0);
          if (has_second) tmem_ld16(ta + (uint32_t)n_tile, r1);
          tmem_ld16(ta + (uint32_t)((NACC - 1) * n_tile), r2);
          OutT vals[16];
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            double v = (double)__uint_as_float(r0[j]) + (double)__uint_as_float(r2[j]);
            if (has_second) v += (double)__uint_as_float(r1[j]);
            if constexpr (PIECES == 2) {
              const int col = n0 + c0 + j;
              v *= scales[(int)(row % comps)] * (col < n_out ? scales[kScaleCols + col] : 1.0);
            }
            vals[j] = (OutT)v;
          }
          uint4* dst = reinterpret_cast<uint4*>(stg + (size_t)r * ldst + c0);
          if constexpr (sizeof(OutT) == 4) {
#pragma unroll
            for (int q = 0; q < 4; ++q)
              dst[q] = make_uint4(__float_as_uint(vals[4 * q]), __float_as_uint(vals[4 * q + 1]),
                                  __float_as_uint(vals[4 * q + 2]), __float_as_uint(vals[4 * q + 3]));
          } else {
#pragma unroll
            for (int q = 0; q < 8; ++q) {
              const unsigned long long a = __double_as_longlong(vals[2 * q]), b = __double_as_longlong(vals[2 * q + 1]);
              dst[q] = make_uint4((uint32_t)a, (uint32_t)(a >> 32), (uint32_t)b, (uint32_t)(b >> 32));
            }
          }
        }
      }
      fence_async_smem();
      named_bar_sync(1, kEpiWarps * 32);   // all epilogue warps arrive, whatever their `ok`
      if (ok && row < M) {
        bulk_store(out + row * ldo + n0, stg + (size_t)r * ldst, (uint32_t)(ncols * sizeof(OutT)));
        bulk_commit();
        bulk_wait_read();
      }
    } else if (ok) {
      double* stage = (double*)smem + warp * 32 * 16;     // [32 rows][16 cols] per warp; stages are idle now
      const int row_base = warp * 32;
      const bool has_second = !TWO_ACC && kblocks >= 2;
      for (int c0 = 0; c0 < n_tile; c0 += 16) {
        uint32_t r0[16], r1[16], r2[16];
        const uint32_t ta = tmem + ((uint32_t)row_base << 16) + (uint32_t)c0;
        tmem_ld16(ta, r0);
        if (has_second) tmem_ld16(ta + (uint32_t)n_tile, r1);
        tmem_ld16(ta + (uint32_t)((NACC - 1) * n_tile), r2);
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          double v = (double)__uint_as_float(r0[j]) + (double)__uint_as_float(r2[j]);
          if (has_second) v += (double)__uint_as_float(r1[j]);
          stage[lane * 16 + ((j + lane) & 15)] = v;
        }
        __syncwarp();
        // two rows per pass: lanes 0-15 row 2q, lanes 16-31 row 2q+1
        for (int q = 0; q < 16; ++q) {
          const int rr = 2 * q + (lane >> 4);
          const int cc = lane & 15;
          const int64_t row = m0 + row_base + rr;
          const int col = n0 + c0 + cc;
          if (row < M && col < n_out) {
            double v = stage[rr * 16 + ((cc + rr) & 15)];
            // float16 operands carry power-of-two component and MO scales
            if constexpr (PIECES == 2) v *= scales[(int)(row % comps)] * scales[kScaleCols + col];
            out[row * ldo + col] = (OutT)v;
          }
        }
        __syncwarp();
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kEpiWarps + 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols));
  }
}

// ------------------------------------------------------------ TN GEMM, split K
//
// part[z][a][b] = sum over the rows r of K slice z of X[r][a] * Y[r][b]: the
// contraction over the rows of two row-major matrices (the coefficient
// gradient of the adjoint, AO^T W).  Both operands are read as they lie,
// MN-major: a stage holds BKR rows of 64-column boxes (128B swizzle), and the
// shared-memory descriptors step from one 64-column box to the next by the
// leading byte offset (one box) and from one 8-row group to the next by the
// stride byte offset (1024 B).  The K range is cut into slices of kps stages
// (one CTA each); the slices' FP32 accumulators are written as FP64 partials
// and summed in a fixed order by the caller, so the FP32 accumulation of a
// CTA stays short.
constexpr int BKR = 32;                 // rows (K) per stage of the MN-major kernel
constexpr int MN_BOX = 64 * BKR * 2;    // one {64 columns, BKR rows} bf16 box: 4 KB
constexpr int kMnStages = 3;

__device__ __forceinline__ uint64_t smem_desc_mn(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)(MN_BOX >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__global__ void __launch_bounds__(kThreads, 1)
tc_gemm_mn_kernel(const __grid_constant__ CUtensorMap tmX, const __grid_constant__ CUtensorMap tmY,
                  const int64_t a_num, const int b_num, const int n_tile, const int kblocks, const int kps,
                  double* __restrict__ part, int* __restrict__ err) {
  constexpr int PIECES = 3, NPROD = 6, STAGES = kMnStages;
  constexpr int A_BOXES = BM / 64;
  constexpr int A_T = A_BOXES * MN_BOX;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = smem_raw + ((1024u - (tcx::smem_addr(smem_raw) & 1023u)) & 1023u);
  const int b_boxes = n_tile / 64;
  const int B_T = b_boxes * MN_BOX;
  const int STAGE = PIECES * (A_T + B_T);
  uint64_t* full = (uint64_t*)(smem + STAGES * STAGE);
  uint64_t* empty = full + STAGES;
  uint64_t* acc_full = empty + STAGES;
  uint32_t* tmem_slot = (uint32_t*)(acc_full + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t a0 = (int64_t)blockIdx.x * BM;
  const int n0 = blockIdx.y * n_tile;
  const int kb0 = blockIdx.z * kps;
  const int nk = min(kps, kblocks - kb0);          // >= 1: the host sizes the grid
  // accumulators: A1*Y1 in two halves of the slice when three fit in TMEM
  // (n_tile <= 128), else one; the corrections in the last
  const bool halves = 3 * n_tile <= 512;
  const uint32_t corr = (uint32_t)((halves ? 2 : 1) * n_tile);
  uint32_t tmem_cols = 32;
  while (tmem_cols < corr + (uint32_t)n_tile) tmem_cols <<= 1;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(acc_full, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == kEpiWarps + 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                 "r"(tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == kEpiWarps) {
    // ---------------- TMA producer
    if (lane == 0) {
      for (int j = 0; j < nk; ++j) {
        const int s = j % STAGES;
        const uint32_t phase = (uint32_t)(j / STAGES) & 1u;
        if (!mbar_wait(&empty[s], phase ^ 1u, err, 1)) break;
        uint8_t* st = smem + s * STAGE;
        mbar_expect_tx(&full[s], (uint32_t)STAGE);
        const int r = (kb0 + j) * BKR;
        for (int p = 0; p < PIECES; ++p) {
          for (int q = 0; q < A_BOXES; ++q)
            tma_load_3d(st + p * A_T + q * MN_BOX, &tmX, &full[s], (int)a0 + 64 * q, r, p);
          for (int q = 0; q < b_boxes; ++q)
            tma_load_3d(st + PIECES * A_T + p * B_T + q * MN_BOX, &tmY, &full[s], n0 + 64 * q, r, p);
        }
      }
    }
  } else if (warp == kEpiWarps + 1) {
    // ---------------- MMA issuer (both operands MN-major: bits 15 and 16)
    if (lane == 0) {
      const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) |
                             ((uint32_t)(n_tile >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
      constexpr int pa[6] = {2, 1, 0, 1, 0, 0}, pb[6] = {0, 1, 2, 0, 1, 0};
      for (int j = 0; j < nk; ++j) {
        const int s = j % STAGES;
        const uint32_t phase = (uint32_t)(j / STAGES) & 1u;
        if (!mbar_wait(&full[s], phase, err, 2)) break;
        tc_fence_after();
        const uint32_t base = smem_addr(smem + s * STAGE);
        for (int kk = 0; kk < BKR / UMMA_K; ++kk) {
#pragma unroll
          for (int t = 0; t < NPROD; ++t) {
            // UMMA_K rows of 128 bytes per K step
            const uint32_t a_addr = base + pa[t] * A_T + kk * UMMA_K * 128;
            const uint32_t b_addr = base + PIECES * A_T + pb[t] * B_T + kk * UMMA_K * 128;
            const bool lead = (t == NPROD - 1);
            const bool second = halves && lead && (2 * j >= nk);
            const uint32_t d = tmem + (lead ? (second ? (uint32_t)n_tile : 0u) : corr);
            const bool first_use = lead ? (second ? (j == (nk + 1) / 2 && kk == 0) : (j == 0 && kk == 0))
                                        : (j == 0 && kk == 0 && t == 0);
            umma_bf16(d, smem_desc_mn(a_addr), smem_desc_mn(b_addr), idesc, first_use ? 0u : 1u);
          }
        }
        umma_commit(&empty[s]);
      }
      umma_commit(acc_full);
    }
  } else {
    // ---------------- epilogue (warps 0..3: TMEM lanes = rows a of the tile)
    bool ok = mbar_wait(acc_full, 0, err, 3);
    ok = __all_sync(0xffffffffu, ok && *(volatile int*)err == 0);
    tc_fence_after();
    if (ok) {
      double* stage = (double*)smem + warp * 32 * 16;
      const int row_base = warp * 32;
      const bool has_second = halves && nk >= 2;
      double* out = part + (int64_t)blockIdx.z * a_num * b_num;
      for (int c0 = 0; c0 < n_tile && n0 + c0 < b_num; c0 += 16) {
        uint32_t r0[16], r1[16], r2[16];
        const uint32_t ta = tmem + ((uint32_t)row_base << 16) + (uint32_t)c0;
        tmem_ld16(ta, r0);
        if (has_second) tmem_ld16(ta + (uint32_t)n_tile, r1);
        tmem_ld16(ta + corr, r2);
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          double v = (double)__uint_as_float(r0[j]) + (double)__uint_as_float(r2[j]);
          if (has_second) v += (double)__uint_as_float(r1[j]);
          stage[lane * 16 + ((j + lane) & 15)] = v;
        }
        __syncwarp();
        for (int q = 0; q < 16; ++q) {
          const int rr = 2 * q + (lane >> 4);
          const int cc = lane & 15;
          const int64_t row = a0 + row_base + rr;
          const int col = n0 + c0 + cc;
          if (row < a_num && col < b_num) out[row * b_num + col] = stage[rr * 16 + ((cc + rr) & 15)];
        }
        __syncwarp();
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kEpiWarps + 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols));
  }
}

// FP64 rows -> 3 bfloat16 pieces (x = x1 + x2 + x3, each the rounding of the
// remainder, formed in FP64), zero beyond `cols` up to the pitch ldo.
__global__ void split_rows_kernel(const double* __restrict__ x, int64_t rows, int cols, int64_t ldx,
                                  uint16_t* __restrict__ out, int ldo, int64_t pstride) {
  const int64_t total = rows * (int64_t)ldo;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / ldo;
    const int c = (int)(i - r * ldo);
    uint16_t p[3];
    split3_bf16(c < cols ? x[r * ldx + c] : 0.0, p);
    out[i] = p[0];
    out[pstride + i] = p[1];
    out[2 * pstride + i] = p[2];
  }
}

// ------------------------------------------------------------ A pieces

constexpr int kAoWarps = 8;

struct MixSmem {
  float rad[kBlockSlots][5];
  double nuc[kBlockNuc][4];
};

// Mixed-form AO VGL: radial part with FP64 displacement, r^2, exponent
// argument, radial Laplacian factor and FP64 accumulation (FP32 exponential
// when a r^2 <= 30, FP64 above); monomials and the product rule in FP32; the
// five components of each AO written as 16-bit pieces (split.cuh) of rows
// p*comps + c.
template <int PIECES, int COMPS>
__global__ void __launch_bounds__(kAoWarps * 32)
ao_split_kernel(const DevTables T, const int64_t point_num, const double* __restrict__ coord, const double cutoff,
                const double* __restrict__ scales, uint16_t* __restrict__ a, const int64_t lda,
                const int64_t piece_stride, const double* __restrict__ cusp_r) {
  __shared__ MixSmem smem[kAoWarps];
  float inv[5];
  load_inv_scales<COMPS>(scales, inv);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  MixSmem& sm = smem[warp];
  const int64_t items = point_num * (int64_t)T.nblock;
  const int64_t stride = (int64_t)gridDim.x * kAoWarps;
  for (int64_t it = (int64_t)blockIdx.x * kAoWarps + warp; it < items; it += stride) {
    const int64_t p = it / T.nblock;
    const int b = (int)(it - p * T.nblock);
    const int4 blk = T.block[b];
    const int2 slots = T.block_slots[b];
    const double px = coord[p], py = coord[p + point_num], pz = coord[p + 2 * point_num];
    const int nn = blk.y - blk.x;
    if (lane < nn) {
      const int n = blk.x + lane;
      const int N = T.nucl_num;
      const double x = px - T.nucl_coord[n];
      const double y = py - T.nucl_coord[n + N];
      const double z = pz - T.nucl_coord[n + 2 * N];
      const double r2 = x * x + y * y + z * z;
      sm.nuc[lane][0] = x;
      sm.nuc[lane][1] = y;
      sm.nuc[lane][2] = z;
      sm.nuc[lane][3] = (r2 > cutoff * T.nucleus_range[n]) ? -1.0 : r2;
    }
    __syncwarp();
    for (int s = slots.x + lane; s < slots.y; s += 32) {
      const int nucl = T.slot_nuc[s];
      const int nl = nucl - blk.x;
      const double r2 = sm.nuc[nl][3];
      double acc[5] = {0., 0., 0., 0., 0.};
      if (r2 >= 0.0) {
        const double x = sm.nuc[nl][0], y = sm.nuc[nl][1], z = sm.nuc[nl][2];
        const int2 cr = T.slot_coef[s];
        const int p0 = T.nuc_prim_start[nucl];
        for (int j = cr.x; j < cr.y; ++j) {
          const double al = T.expo[p0 + T.coef_prim[j]];
          const double ar2 = al * r2;
          if (ar2 > cutoff) break;
          const double e = ar2 > 30.0 ? exp(-ar2) : (double)expf(-(float)ar2);
          const double cv = T.coef_val[j];
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
      const int ls = s - slots.x;
#pragma unroll
      for (int c = 0; c < 5; ++c) sm.rad[ls][c] = (float)acc[c];
    }
    __syncwarp();
    for (int k = blk.z + lane; k < blk.w; k += 32) {
      const int code = T.ao_code[k];
      const int ax = code & 15, by = (code >> 4) & 15, cz = (code >> 8) & 15, l = (code >> 12) & 15;
      const int slot = (code >> 16) & 255, nl = (code >> 24) & 31;
      float v[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
      const float s1 = sm.rad[slot][0];
      if (sm.nuc[nl][3] >= 0.0 && s1 != 0.0f && !cusp_masked(cusp_r, l, blk.x + nl, sm.nuc[nl][3], COMPS == 1)) {
        const float f = (float)T.ao_factor[k];
        const float s2 = sm.rad[slot][1], s3 = sm.rad[slot][2], s4 = sm.rad[slot][3], s5 = sm.rad[slot][4];
        if (l == 0) {
          v[0] = s1 * f; v[1] = s2 * f; v[2] = s3 * f; v[3] = s4 * f; v[4] = s5 * f;
        } else {
          const float x = (float)sm.nuc[nl][0], y = (float)sm.nuc[nl][1], z = (float)sm.nuc[nl][2];
          float P0, P1, P2, P3, P4;
          if (l == 1) {
            P0 = ax ? x : (by ? y : z);
            P1 = (float)ax; P2 = (float)by; P3 = (float)cz; P4 = 0.f;
          } else {
            float pa = 1.f, pb = 1.f, pc = 1.f, pa1 = 1.f, pb1 = 1.f, pc1 = 1.f, pa2 = 1.f, pb2 = 1.f, pc2 = 1.f;
            for (int i = 0; i < ax; ++i) { pa2 = pa1; pa1 = pa; pa *= x; }
            for (int i = 0; i < by; ++i) { pb2 = pb1; pb1 = pb; pb *= y; }
            for (int i = 0; i < cz; ++i) { pc2 = pc1; pc1 = pc; pc *= z; }
            if (ax < 2) pa2 = 1.f;
            if (by < 2) pb2 = 1.f;
            if (cz < 2) pc2 = 1.f;
            float xy = pa * pb, yz = pb * pc, xz = pa * pc;
            P0 = xy * pc;
            xy *= (float)cz; xz *= (float)by; yz *= (float)ax;
            P1 = pa1 * yz; P2 = pb1 * xz; P3 = pc1 * xy;
            P4 = (float)(ax - 1) * pa2 * yz + (float)(by - 1) * pb2 * xz + (float)(cz - 1) * pc2 * xy;
          }
          v[0] = P0 * s1 * f;
          v[1] = (P1 * s1 + P0 * s2) * f;
          v[2] = (P2 * s1 + P0 * s3) * f;
          v[3] = (P3 * s1 + P0 * s4) * f;
          v[4] = (P4 * s1 + P0 * s5 + 2.f * (P1 * s2 + P2 * s3 + P3 * s4)) * f;
        }
      }
#pragma unroll
      for (int c = 0; c < COMPS; ++c) {
        uint16_t pcs[3];
        split_one<PIECES>(v[c], inv[c], pcs);
        const int64_t off = (p * COMPS + c) * lda + k;
#pragma unroll
        for (int q = 0; q < PIECES; ++q) a[q * piece_stride + off] = pcs[q];
      }
    }
    __syncwarp();
  }
}

// ------------------------------------------------------------ host side

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

// 3-D bf16 map {K, rows, pieces}, box {64, box_rows, 1}, 128B swizzle.
bool make_map(CUtensorMap* map, const void* base, int64_t k, int64_t rows, int64_t ld, int pieces, int64_t piece_stride,
              int box_rows) {
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[3] = {(cuuint64_t)k, (cuuint64_t)rows, (cuuint64_t)pieces};
  cuuint64_t strides[2] = {(cuuint64_t)(ld * 2), (cuuint64_t)(piece_stride * 2)};
  cuuint32_t box[3] = {(cuuint32_t)BK, (cuuint32_t)box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

int sm_count() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

template <int PIECES, int STAGES, typename OutT = double, bool TWO_ACC = false>
cudaError_t launch_gemm(const CUtensorMap& ta, const CUtensorMap& tb, int64_t M, int n_out, int n_tile, int n_tiles,
                        int kblocks, int comps, const double* scales, OutT* out, int64_t ldo, int* err,
                        cudaStream_t s) {
  const size_t stage = (size_t)PIECES * (BM * BK * 2 + (size_t)n_tile * BK * 2);
  const size_t smem = 1024 + STAGES * stage + (2 * STAGES + 1) * 8 + 16;
  auto kern = tc_gemm_kernel<PIECES, STAGES, OutT, TWO_ACC>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)((M + BM - 1) / BM), (unsigned)n_tiles);
  kern<<<grid, kThreads, smem, s>>>(ta, tb, M, n_out, n_tile, kblocks, comps, scales, out, ldo, err);
  count_launch();
  return cudaGetLastError();
}

}  // namespace

TcPlan tc_plan(int64_t ao_num, int64_t mo_num, int pieces) {
  TcPlan p;
  p.ao_num = ao_num;
  p.mo_num = mo_num;
  p.pieces = pieces;
  p.k_pad = (ao_num + BK - 1) / BK * BK;
  // N tiles of at most 256 columns (one tcgen05.mma N), multiples of 16
  p.n_tiles = (int)((mo_num + 255) / 256);
  const int64_t per = (mo_num + p.n_tiles - 1) / p.n_tiles;
  p.n_tile = (int)((per + 15) / 16 * 16);
  // the pipeline stages (pieces x (A 16 KB + B n_tile*128 B), 2 stages for 3
  // pieces, 3 for 2) must fit in 227 KB of shared memory: n_tile <= 160
  while (p.n_tile > 160) {
    p.n_tiles += 1;
    const int64_t q = (mo_num + p.n_tiles - 1) / p.n_tiles;
    p.n_tile = (int)((q + 15) / 16 * 16);
  }
  p.n_pad = (int64_t)p.n_tile * p.n_tiles;
  p.scale_off = ((size_t)pieces * p.n_pad * p.k_pad * 2 + 255) / 256 * 256;
  p.coef_bytes = p.scale_off + sizeof(double) * (kScaleCols + (size_t)p.n_pad);
  return p;
}

TcPlan tc_plan_fused(int64_t ao_num, int64_t mo_num, int pieces) {
  TcPlan p = tc_plan(ao_num, mo_num, pieces);
  // QMCKL_B200_WIDE_TILES: unset, wide tiles when they take fewer MO tiles,
  // or as many with three A stages; "0", never; "1", whenever they fit
  const char* env = std::getenv("QMCKL_B200_WIDE_TILES");
  const bool never = env != nullptr && std::strcmp(env, "0") == 0;
  const bool always = env != nullptr && std::strcmp(env, "1") == 0;
  if (pieces != 3 || never) return p;
  // two accumulators of up to 256 columns fit TMEM (512); the single
  // coefficient tile (3 x 128 B per MO) fits beside the 48 KB A stages
  const int n_tiles = (int)((mo_num + 255) / 256);
  if (n_tiles > p.n_tiles && !always) return p;
  const int64_t per = (mo_num + n_tiles - 1) / n_tiles;
  const int n_tile = (int)((per + 15) / 16 * 16);
  // shared memory: the A stages (48 KB each), the coefficient tile
  // (384 B per MO), room for a K-block record per stage (4 KB each) and
  // the rest (alignment, barriers, points, lists: 3 KB)
  auto bytes = [&](int nst) { return 1024 + (size_t)nst * (49152 + 4096) + (size_t)384 * n_tile + 3072; };
  int nst = 0;
  if (bytes(3) <= 232448) nst = 3;
  else if (bytes(2) <= 232448) nst = 2;
  if (nst == 0) return p;
  // As many tiles either way: the wide form wins only with its third stage
  // (config-1 molecule, 160 MOs: 2.52 against 2.67 ms); with two it
  // reloads its single coefficient tile between blocks for nothing.
  if (n_tiles == p.n_tiles && nst < 3 && !always) return p;
  p.n_tiles = n_tiles;
  p.n_tile = n_tile;
  p.nacc = 2;
  p.nst = nst;
  p.n_pad = (int64_t)p.n_tile * p.n_tiles;
  p.scale_off = ((size_t)pieces * p.n_pad * p.k_pad * 2 + 255) / 256 * 256;
  p.coef_bytes = p.scale_off + sizeof(double) * (kScaleCols + (size_t)p.n_pad);
  return p;
}

size_t tc_a_bytes(const TcPlan& plan, int64_t rows) { return (size_t)plan.pieces * (size_t)rows * plan.k_pad * 2; }

cudaError_t tc_prepare_coef(const TcPlan& plan, const double* coefficient_host, void* d_coef, cudaStream_t s) {
  const int64_t A = plan.ao_num, M = plan.mo_num, KP = plan.k_pad, NP = plan.n_pad;
  std::vector<uint8_t> h(plan.coef_bytes, 0);
  uint16_t* pc = (uint16_t*)h.data();
  double* sc = (double*)(h.data() + plan.scale_off);
  for (int i = 0; i < kScaleCols + NP; ++i) sc[i] = 1.0;
  if (plan.pieces == 3) {
    auto to_bf16 = [](double x) -> uint16_t {   // round to nearest even of the FP32 rounding
      float f = (float)x;
      uint32_t u;
      std::memcpy(&u, &f, 4);
      if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t)(u >> 16);
      u += 0x7fffu + ((u >> 16) & 1u);
      return (uint16_t)(u >> 16);
    };
    auto from_bf16 = [](uint16_t b) -> double {
      uint32_t u = (uint32_t)b << 16;
      float f;
      std::memcpy(&f, &u, 4);
      return (double)f;
    };
    for (int64_t i = 0; i < M; ++i)
      for (int64_t k = 0; k < A; ++k) {
        double r = coefficient_host[i * A + k];
        for (int p = 0; p < 3; ++p) {
          const uint16_t b = to_bf16(r);
          pc[((size_t)p * NP + i) * KP + k] = b;
          r -= from_bf16(b);
        }
      }
  } else {
    for (int64_t i = 0; i < M; ++i) {
      double mx = 0.0;
      for (int64_t k = 0; k < A; ++k) mx = std::max(mx, std::fabs(coefficient_host[i * A + k]));
      // per-MO power of two bringing the largest coefficient to 2^10
      const double tau = mx > 0.0 ? std::ldexp(1.0, (int)std::ceil(std::log2(mx / 1024.0))) : 1.0;
      sc[kScaleCols + i] = tau;
      for (int64_t k = 0; k < A; ++k) {
        const double x = coefficient_host[i * A + k] / tau;
        const __half x1 = __float2half_rn((float)x);
        const __half x2 = __float2half_rn((float)(x - (double)__half2float(x1)));
        pc[((size_t)0 * NP + i) * KP + k] = __half_as_ushort(x1);
        pc[((size_t)1 * NP + i) * KP + k] = __half_as_ushort(x2);
      }
    }
  }
  cudaError_t e = cudaMemcpyAsync(d_coef, h.data(), h.size(), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(s);   // the host staging buffer goes out of scope
}

void tc_envelope(const ShellBound* shells, int nshell, double r_max, float r0, float inv_log2q, float* env) {
  using fz::kEnvCells;
  // Upper bounds, with |x^a y^b z^c| <= r^l, |grad P| <= l r^(l-1),
  // |lap P| <= l(l-1) r^(l-2) and, for R(r) = sum c exp(-a r^2) with
  // S_n = sum c a^n exp(-a r^2): |grad R| = 2 r |S1|, lap R = 4 r^2 S2 - 6 S1.
  // Sampled 16 times per radial cell; the envelope of a cell is the maximum
  // over it and every later cell (suffix maximum), doubled for the sampling.
  constexpr int kSub = 16;
  double cell[3][kEnvCells];
  for (int q = 0; q < 3; ++q)
    for (int g = 0; g < kEnvCells; ++g) cell[q][g] = 0.0;
  auto start = [&](int g) { return g == 0 ? 0.0 : (double)r0 * std::exp2((double)(g - 1) / inv_log2q); };
  for (int g = 0; g < kEnvCells; ++g) {
    const double a0 = start(g);
    const double a1 = g + 1 < kEnvCells ? start(g + 1) : std::max(a0, r_max);
    for (int t = 0; t <= kSub; ++t) {
      const double r = a0 + (a1 - a0) * t / kSub;
      if (r > r_max) break;
      for (int s = 0; s < nshell; ++s) {
        const ShellBound& S = shells[s];
        double S0 = 0.0, S1 = 0.0, S2 = 0.0;
        for (int j = 0; j < S.nprim; ++j) {
          const double e = S.coef[j] * std::exp(-S.expo[j] * r * r);
          S0 += e;
          S1 += S.expo[j] * e;
          S2 += S.expo[j] * S.expo[j] * e;
        }
        const int l = S.l;
        const double rl = std::pow(r, l), rl1 = l >= 1 ? l * std::pow(r, l - 1) : 0.0,
                     rl2 = l >= 2 ? l * (l - 1) * std::pow(r, l - 2) : 0.0;
        const double gR = 2.0 * r * std::fabs(S1), lR = std::fabs(4.0 * r * r * S2 - 6.0 * S1);
        cell[0][g] = std::max(cell[0][g], S.factor * rl * std::fabs(S0));
        cell[1][g] = std::max(cell[1][g], S.factor * (rl1 * std::fabs(S0) + rl * gR));
        cell[2][g] = std::max(cell[2][g], S.factor * (rl2 * std::fabs(S0) + 2.0 * rl1 * gR + rl * lR));
      }
    }
  }
  for (int q = 0; q < 3; ++q) {
    double m = 0.0;
    for (int g = kEnvCells - 1; g >= 0; --g) {
      m = std::max(m, cell[q][g]);
      env[q * kEnvCells + g] = (float)(2.0 * m);
    }
  }
}

cudaError_t tc_run(const DevTables& T, const TcPlan& plan, int64_t point_num, int comps, const double* coord,
                   double cutoff, const void* d_coef, void* d_a, double* out, int* err, cudaStream_t s,
                   const AoTiles* tiles, const double* cusp_r) {
  if (point_num <= 0) return cudaSuccess;
  if (plan.pieces != 3) return cudaErrorInvalidValue;   // the unfused kernels take 3 bfloat16 pieces
  const int64_t rows = (int64_t)comps * point_num;
  const int64_t lda = plan.k_pad;
  const int64_t pstride = rows * lda;
  uint16_t* a = (uint16_t*)d_a;
  const double* sc = tc_scales(plan, d_coef);
  // 1) AO pieces
  if (tiles != nullptr && cusp_r == nullptr) {   // the tiled producer knows no cusp adjustment
    cudaError_t e =
        launch_ao_tile_split(T, *tiles, point_num, coord, cutoff, comps, plan.pieces, sc, a, lda, pstride, s);
    if (e != cudaSuccess) return e;
  } else {
    const int64_t items = point_num * T.nblock;
    const int grid = (int)std::min<int64_t>((items + kAoWarps - 1) / kAoWarps, (int64_t)sm_count() * 8);
    if (comps == 5)
      ao_split_kernel<3, 5><<<grid, kAoWarps * 32, 0, s>>>(T, point_num, coord, cutoff, sc, a, lda, pstride, cusp_r);
    else
      ao_split_kernel<3, 1><<<grid, kAoWarps * 32, 0, s>>>(T, point_num, coord, cutoff, sc, a, lda, pstride, cusp_r);
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  // 2) tensor-core contraction
  CUtensorMap ta, tb;
  if (!make_map(&ta, a, plan.ao_num, rows, lda, plan.pieces, pstride, BM)) return cudaErrorInvalidValue;
  if (!make_map(&tb, d_coef, plan.ao_num, plan.n_pad, plan.k_pad, plan.pieces, plan.n_pad * plan.k_pad, plan.n_tile))
    return cudaErrorInvalidValue;
  if (!err) return cudaErrorInvalidValue;
  const int kblocks = (int)((plan.ao_num + BK - 1) / BK);
  // a timed-out barrier wait stays in *err for the caller's next synchronization
  return launch_gemm<3, 2>(ta, tb, rows, (int)plan.mo_num, plan.n_tile, plan.n_tiles, kblocks, comps, sc, out,
                           plan.mo_num, err, s);
}

cudaError_t tc_prime_unfused() {
  cudaFuncAttributes a;
  cudaError_t e = cudaFuncGetAttributes(&a, ao_split_kernel<3, 5>);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, ao_split_kernel<3, 1>);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, tc_gemm_kernel<3, 2, double, false>);
  return e;
}

cudaError_t tc_run_scratch(const DevTables& T, const TcPlan& plan, int64_t point_num, int comps,
                           const double* coord, double cutoff, const void* d_coef, void* d_a, int* d_err,
                           double* out, cudaStream_t s, const double* cusp_r) {
  if (point_num <= 0) return cudaSuccess;
  if (plan.pieces != 3 || d_err == nullptr) return cudaErrorInvalidValue;   // 3 bfloat16 pieces
  const int64_t rows = (int64_t)comps * point_num;
  const int64_t lda = plan.k_pad;
  const int64_t pstride = rows * lda;
  uint16_t* a = (uint16_t*)d_a;
  const double* sc = tc_scales(plan, d_coef);
  const int64_t items = point_num * T.nblock;
  const int grid = (int)std::min<int64_t>((items + kAoWarps - 1) / kAoWarps, (int64_t)sm_count() * 8);
  if (comps == 5)
    ao_split_kernel<3, 5><<<grid, kAoWarps * 32, 0, s>>>(T, point_num, coord, cutoff, sc, a, lda, pstride, cusp_r);
  else
    ao_split_kernel<3, 1><<<grid, kAoWarps * 32, 0, s>>>(T, point_num, coord, cutoff, sc, a, lda, pstride, cusp_r);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  CUtensorMap ta, tb;
  if (!make_map(&ta, a, plan.ao_num, rows, lda, plan.pieces, pstride, BM)) return cudaErrorInvalidValue;
  if (!make_map(&tb, d_coef, plan.ao_num, plan.n_pad, plan.k_pad, plan.pieces, plan.n_pad * plan.k_pad, plan.n_tile))
    return cudaErrorInvalidValue;
  const int kblocks = (int)((plan.ao_num + BK - 1) / BK);
  return launch_gemm<3, 2>(ta, tb, rows, (int)plan.mo_num, plan.n_tile, plan.n_tiles, kblocks, comps, sc, out,
                           plan.mo_num, d_err, s);
}

// ------------------------------------------------------------ adjoint contractions

cudaError_t tc_split_rows(const double* x, int64_t rows, int cols, int64_t ldx, void* pieces, int ldp,
                          int64_t pstride, cudaStream_t s) {
  if (rows <= 0) return cudaSuccess;
  if (ldp < cols || ldp % 8 != 0 || pstride % 8 != 0) return cudaErrorInvalidValue;
  const int64_t total = rows * (int64_t)ldp;
  const int grid = (int)std::min<int64_t>((total + 255) / 256, (int64_t)sm_count() * 16);
  split_rows_kernel<<<grid, 256, 0, s>>>(x, rows, cols, ldx, (uint16_t*)pieces, ldp, pstride);
  count_launch();
  return cudaGetLastError();
}

int tc_tn_splits(int64_t rows, int kps) {
  const int64_t kblocks = (rows + BKR - 1) / BKR;
  return (int)((kblocks + kps - 1) / kps);
}

cudaError_t tc_gemm_tn_split(const void* x, int64_t ldx, int64_t x_pstride, int64_t a_num, const void* y, int64_t ldy,
                             int64_t y_pstride, int b_num, int64_t rows, int kps, double* part, int* err,
                             cudaStream_t s) {
  if (rows <= 0 || a_num <= 0 || b_num <= 0) return cudaSuccess;
  if (kps < 1 || ldx % 8 != 0 || ldy % 8 != 0 || x_pstride % 8 != 0 || y_pstride % 8 != 0)
    return cudaErrorInvalidValue;
  // N tiles of at most 192 columns, multiples of the 64-column box
  const int n_tiles = (b_num + 191) / 192;
  const int n_tile = ((b_num + n_tiles - 1) / n_tiles + 63) / 64 * 64;
  const int64_t kblocks64 = (rows + BKR - 1) / BKR;
  if (kblocks64 > (int64_t)1 << 30) return cudaErrorInvalidValue;
  const int kblocks = (int)kblocks64;
  const int splits = (kblocks + kps - 1) / kps;
  CUtensorMap tx, ty;
  if (!make_map(&tx, x, a_num, rows, ldx, 3, x_pstride, BKR)) return cudaErrorInvalidValue;
  if (!make_map(&ty, y, b_num, rows, ldy, 3, y_pstride, BKR)) return cudaErrorInvalidValue;
  const size_t stage = (size_t)3 * ((BM / 64) * MN_BOX + (size_t)(n_tile / 64) * MN_BOX);
  const size_t smem = 1024 + kMnStages * stage + (2 * kMnStages + 1) * 8 + 16;
  cudaError_t e = cudaFuncSetAttribute(tc_gemm_mn_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)((a_num + BM - 1) / BM), (unsigned)n_tiles, (unsigned)splits);
  tc_gemm_mn_kernel<<<grid, kThreads, smem, s>>>(tx, ty, a_num, b_num, n_tile, kblocks, kps, part, err);
  count_launch();
  return cudaGetLastError();
}

cudaError_t tc_gemm_nt(const void* x, int64_t ldx, int64_t x_pstride, int64_t rows, int64_t k, const void* y,
                       int64_t ldy, int64_t y_pstride, int64_t n, float* out, int64_t ldo, int* err, cudaStream_t s) {
  if (rows <= 0 || n <= 0) return cudaSuccess;
  if (ldx % 8 != 0 || ldy % 8 != 0 || x_pstride % 8 != 0 || y_pstride % 8 != 0) return cudaErrorInvalidValue;
  // 128-column MO tiles, one stage, two accumulators: ~99 KB of shared
  // memory and 256 TMEM columns, two CTAs per SM (one's epilogue overlaps
  // the other's loads and MMAs); K (the MO count) is short
  const int n_tile = 128;
  const int n_tiles = (int)((n + n_tile - 1) / n_tile);
  CUtensorMap tx, ty;
  if (!make_map(&tx, x, k, rows, ldx, 3, x_pstride, BM)) return cudaErrorInvalidValue;
  if (!make_map(&ty, y, k, n, ldy, 3, y_pstride, n_tile)) return cudaErrorInvalidValue;
  const int kblocks = (int)((k + BK - 1) / BK);
  return launch_gemm<3, 1, float, true>(tx, ty, rows, (int)n, n_tile, n_tiles, kblocks, 1, nullptr, out, ldo, err, s);
}

}  // namespace qb
