// Fused mixed-form AO -> MO evaluation: the AO matrix never leaves the SM.
//
// One CTA owns a tile of points and one N tile of MOs.  Its 128 accumulator
// rows are (point, component) pairs: 25 points x 5 components (+3 zero rows)
// for MO VGL, 128 points for MO value.  For every 64-wide K block (64 AOs):
//   warps 0..7  (producers) evaluate the AOs of the block at the tile's points
//               and write them as bfloat16 pieces straight into the 128B-
//               swizzled K-major shared-memory tile the tensor core reads
//               (one 16-byte store per (row, 8 AOs, piece)); then
//               fence.proxy.async + arrive on full[stage]
//   warp 8      TMA-loads the coefficient pieces of the block (full[stage])
//   warp 9      allocates TMEM; one thread issues the split-BF16 tcgen05.mma
//               chain into three FP32 accumulators (leading product in two
//               K halves, corrections in the third) and commits empty[stage]
//   warps 0..3  epilogue: sum of the three accumulators in FP64, written as
//               contiguous rows of mo_vgl[point][5][mo] (or mo_value)
// AO arithmetic (mixed form): FP64 displacement, r^2, exponent argument and
// radial Laplacian factor, FP32 exponential when a r^2 <= 30 (FP64 above),
// FP64 radial accumulation, FP32 monomials and product rule; the screening
// follows qmckl_compute_ao_vgl_hpc_gaussian (org/qmckl_ao.org:8601-8973).
// Every mbarrier wait is bounded (2 s of %globaltimer); a timeout sets the
// error word and the CTA still releases its TMEM.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>

#include "mo_tc.cuh"
#include "tc_ptx.cuh"

namespace qb {
namespace {

using namespace tcx;

constexpr int BM = 128, BK = 64, UMMA_K = 16;
constexpr int kProdWarps = 8;
constexpr int kProd = kProdWarps * 32;
constexpr int kTmaWarp = kProdWarps;
constexpr int kMmaWarp = kProdWarps + 1;
constexpr int kThreadsF = (kProdWarps + 2) * 32;
constexpr int A_TILE = BM * BK * 2;
constexpr int STAGES = 2;

__device__ __forceinline__ uint32_t bf16_bits(__nv_bfloat16 h) { return (uint32_t)__bfloat16_as_ushort(h); }

// Radial VGL of one shell at one point (mixed form).
__device__ __forceinline__ void radial_mixed(const DevTables& T, int sh, double px, double py, double pz,
                                             double cutoff, float (&s)[5], float& fx, float& fy, float& fz,
                                             bool& live) {
  const int n = T.shell_nuc[sh];
  const int N = T.nucl_num;
  const double x = px - T.nucl_coord[n];
  const double y = py - T.nucl_coord[n + N];
  const double z = pz - T.nucl_coord[n + 2 * N];
  const double r2 = x * x + y * y + z * z;
  fx = (float)x;
  fy = (float)y;
  fz = (float)z;
  double acc[5] = {0., 0., 0., 0., 0.};
  live = !(r2 > cutoff * T.nucleus_range[n]);
  if (live) {
    const int2 cr = T.shell_coef[sh];
    const int p0 = T.nuc_prim_start[n];
    for (int j = cr.x; j < cr.y; ++j) {
      const double al = T.expo[p0 + T.coef_prim[j]];
      const double ar2 = al * r2;
      if (ar2 > cutoff) break;   // sorted by exponent
      const double e = ar2 > 30.0 ? exp(-ar2) : (double)expf(-(float)ar2);
      const double cv = T.coef_val[j];
      const double f = -2.0 * al * e;
      acc[0] += cv * e;
      acc[1] += cv * (f * x);
      acc[2] += cv * (f * y);
      acc[3] += cv * (f * z);
      acc[4] += cv * (f * (3.0 - 2.0 * ar2));
    }
  }
#pragma unroll
  for (int c = 0; c < 5; ++c) s[c] = (float)acc[c];
}

// Value, gradient and Laplacian of one AO from its shell's radial VGL (FP32).
__device__ __forceinline__ void ao_product(int code, float f, const float (&s)[5], float x, float y, float z,
                                           float (&v)[5]) {
  const int ax = code & 15, by = (code >> 4) & 15, cz = (code >> 8) & 15, l = (code >> 12) & 15;
  if (l == 0) {
#pragma unroll
    for (int c = 0; c < 5; ++c) v[c] = s[c] * f;
    return;
  }
  float P0, P1, P2, P3, P4;
  if (l == 1) {
    P0 = ax ? x : (by ? y : z);
    P1 = (float)ax; P2 = (float)by; P3 = (float)cz; P4 = 0.f;
  } else {
    float pa = 1.f, pb = 1.f, pc = 1.f, pa1 = 1.f, pb1 = 1.f, pc1 = 1.f, pa2 = 1.f, pb2 = 1.f, pc2 = 1.f;
    for (int i = 0; i < ax; ++i) { pa2 = pa1; pa1 = pa; pa *= x; }
    for (int i = 0; i < by; ++i) { pb2 = pb1; pb1 = pb; pb *= y; }
    for (int i = 0; i < cz; ++i) { pc2 = pc1; pc1 = pc; pc *= z; }
    float xy = pa * pb, yz = pb * pc, xz = pa * pc;
    P0 = xy * pc;
    xy *= (float)cz; xz *= (float)by; yz *= (float)ax;
    P1 = pa1 * yz; P2 = pb1 * xz; P3 = pc1 * xy;
    P4 = (float)(ax - 1) * pa2 * yz + (float)(by - 1) * pb2 * xz + (float)(cz - 1) * pc2 * xy;
  }
  v[0] = P0 * s[0] * f;
  v[1] = (P1 * s[0] + P0 * s[1]) * f;
  v[2] = (P2 * s[0] + P0 * s[2]) * f;
  v[3] = (P3 * s[0] + P0 * s[3]) * f;
  v[4] = (P4 * s[0] + P0 * s[4] + 2.f * (P1 * s[1] + P2 * s[2] + P3 * s[3])) * f;
}

template <int PIECES, int COMPS>
__global__ void __launch_bounds__(kThreadsF, 1)
fused_mo_kernel(const DevTables T, const __grid_constant__ CUtensorMap tmB, const int64_t P,
                const double* __restrict__ coord, const double cutoff, const int n_out, const int n_tile,
                const int kblocks, double* __restrict__ out, int* __restrict__ err) {
  constexpr int NPROD = PIECES == 3 ? 6 : 3;
  constexpr int PTS = BM / COMPS;            // 25 points (VGL) or 128 (value)
  constexpr int UNITS = PTS * (BK / 8);      // (point, 8-AO chunk) units per K block
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int B_TILE = n_tile * BK * 2;
  const int A_BYTES = PIECES * A_TILE;
  const int STAGE = PIECES * (A_TILE + B_TILE);
  uint64_t* full = (uint64_t*)(smem + STAGES * STAGE);
  uint64_t* empty = full + STAGES;
  uint64_t* acc_full = empty + STAGES;
  uint32_t* tmem_slot = (uint32_t*)(acc_full + 1);
  double* pts = (double*)(acc_full + 2);      // [3][PTS]

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t p0 = (int64_t)blockIdx.x * PTS;
  const int n0 = blockIdx.y * n_tile;
  const int A = T.ao_num;
  uint32_t tmem_cols = 32;
  while ((int)tmem_cols < 3 * n_tile) tmem_cols <<= 1;

  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], kProd + 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(acc_full, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int t = tid; t < 3 * PTS; t += kThreadsF) {
    const int d = t / PTS, i = t - d * PTS;
    pts[t] = (p0 + i < P) ? coord[(p0 + i) + d * P] : 0.0;
  }
  // rows PTS*COMPS .. 127 of the A tiles stay zero for the whole kernel
  constexpr int PAD = BM - PTS * COMPS;
  if constexpr (PAD > 0) {
    for (int t = tid; t < STAGES * PIECES * PAD * 8; t += kThreadsF) {
      const int chunk = t & 7;
      const int rr = (t >> 3) % PAD;
      const int tile = (t >> 3) / PAD;   // stage * PIECES + piece
      const int r = PTS * COMPS + rr;
      uint8_t* base = smem + (tile / PIECES) * STAGE + (tile % PIECES) * A_TILE;
      st_shared_v4(smem_addr(base + r * 128 + ((chunk ^ (r & 7)) << 4)), 0u, 0u, 0u, 0u);
    }
  }
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                 "r"(tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp < kProdWarps) {
    // ---------------- AO producers
    for (int kb = 0; kb < kblocks; ++kb) {
      const int s = kb & 1;
      const uint32_t phase = (uint32_t)(kb >> 1) & 1u;
      if (!mbar_wait(&empty[s], phase ^ 1u, err, 11)) break;
      const uint32_t a_base = smem_addr(smem + s * STAGE);
      for (int u = tid; u < UNITS; u += kProd) {
        const int i = u >> 3, j = u & 7;
        const bool active = p0 + i < P;
        const double px = pts[i], py = pts[PTS + i], pz = pts[2 * PTS + i];
        uint32_t pk[PIECES][COMPS][4];
        int prev = -1;
        float rs[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
        float fx = 0.f, fy = 0.f, fz = 0.f;
        bool live = false;
#pragma unroll
        for (int t = 0; t < 8; ++t) {
          const int k = kb * BK + j * 8 + t;
          float v[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
          if (active && k < A) {
            const int sh = T.ao_shell[k];
            if (sh != prev) {
              radial_mixed(T, sh, px, py, pz, cutoff, rs, fx, fy, fz, live);
              prev = sh;
            }
            if (live && rs[0] != 0.f) ao_product(T.ao_code[k], (float)T.ao_factor[k], rs, fx, fy, fz, v);
          }
#pragma unroll
          for (int c = 0; c < COMPS; ++c) {
            const __nv_bfloat16 h = __float2bfloat16_rn(v[c]);
            float r = v[c] - __bfloat162float(h);
            const __nv_bfloat16 m = __float2bfloat16_rn(r);
            uint32_t bits[3] = {bf16_bits(h), bf16_bits(m), 0u};
            if (PIECES == 3) {
              r = r - __bfloat162float(m);
              bits[2] = bf16_bits(__float2bfloat16_rn(r));
            }
#pragma unroll
            for (int q = 0; q < PIECES; ++q) {
              if (t & 1) pk[q][c][t >> 1] |= bits[q] << 16;
              else pk[q][c][t >> 1] = bits[q];
            }
          }
        }
#pragma unroll
        for (int c = 0; c < COMPS; ++c) {
          const int r = i * COMPS + c;
          const uint32_t off = (uint32_t)(r * 128 + ((j ^ (r & 7)) << 4));
#pragma unroll
          for (int q = 0; q < PIECES; ++q)
            st_shared_v4(a_base + q * A_TILE + off, pk[q][c][0], pk[q][c][1], pk[q][c][2], pk[q][c][3]);
        }
      }
      fence_async_smem();
      mbar_arrive(&full[s]);
    }
  } else if (warp == kTmaWarp) {
    // ---------------- coefficient pieces
    if (lane == 0) {
      for (int kb = 0; kb < kblocks; ++kb) {
        const int s = kb & 1;
        const uint32_t phase = (uint32_t)(kb >> 1) & 1u;
        if (!mbar_wait(&empty[s], phase ^ 1u, err, 12)) break;
        uint8_t* st = smem + s * STAGE + A_BYTES;
        mbar_expect_tx(&full[s], (uint32_t)(PIECES * B_TILE));
        for (int q = 0; q < PIECES; ++q) tma_load_3d(st + q * B_TILE, &tmB, &full[s], kb * BK, n0, q);
      }
    }
  } else {
    // ---------------- MMA issuer
    if (lane == 0) {
      const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n_tile >> 3) << 17) |
                             ((uint32_t)(BM >> 4) << 24);
      constexpr int pa3[6] = {2, 1, 0, 1, 0, 0}, pb3[6] = {0, 1, 2, 0, 1, 0};
      constexpr int pa2[3] = {1, 0, 0}, pb2[3] = {0, 1, 0};
      for (int kb = 0; kb < kblocks; ++kb) {
        const int s = kb & 1;
        const uint32_t phase = (uint32_t)(kb >> 1) & 1u;
        if (!mbar_wait(&full[s], phase, err, 13)) break;
        tc_fence_after();
        const uint32_t base = smem_addr(smem + s * STAGE);
        for (int kk = 0; kk < BK / UMMA_K; ++kk) {
#pragma unroll
          for (int t = 0; t < NPROD; ++t) {
            const int ia = PIECES == 3 ? pa3[t] : pa2[t];
            const int ib = PIECES == 3 ? pb3[t] : pb2[t];
            const uint32_t a_addr = base + ia * A_TILE + kk * UMMA_K * 2;
            const uint32_t b_addr = base + A_BYTES + ib * B_TILE + kk * UMMA_K * 2;
            const bool lead = (t == NPROD - 1);
            const bool second = lead && (2 * kb >= kblocks);
            const uint32_t d = tmem + (uint32_t)((lead ? (second ? 1 : 0) : 2) * n_tile);
            const bool first_use = lead ? (second ? (kb == (kblocks + 1) / 2 && kk == 0) : (kb == 0 && kk == 0))
                                        : (kb == 0 && kk == 0 && t == 0);
            umma_bf16(d, smem_desc(a_addr), smem_desc(b_addr), idesc, first_use ? 0u : 1u);
          }
        }
        umma_commit(&empty[s]);
      }
      umma_commit(acc_full);
    }
  }

  if (warp < 4) {
    // ---------------- epilogue: TMEM lanes 32*warp .. 32*warp+31
    bool ok = mbar_wait(acc_full, 0, err, 14);
    ok = __all_sync(0xffffffffu, ok && *(volatile int*)err == 0);
    tc_fence_after();
    if (ok) {
      double* stage = (double*)smem + warp * 32 * 16;
      const int row_base = warp * 32;
      const bool has_second = kblocks >= 2;
      const int64_t rows_total = P * COMPS;
      for (int c0 = 0; c0 < n_tile; c0 += 16) {
        uint32_t r0[16], r1[16], r2[16];
        const uint32_t ta = tmem + ((uint32_t)row_base << 16) + (uint32_t)c0;
        tmem_ld16(ta, r0);
        tmem_ld16(ta + (uint32_t)n_tile, r1);
        tmem_ld16(ta + (uint32_t)(2 * n_tile), r2);
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
          const int r = row_base + rr;
          const int64_t row = p0 * COMPS + r;
          const int col = n0 + c0 + cc;
          if (r < PTS * COMPS && row < rows_total && col < n_out)
            out[row * n_out + col] = stage[rr * 16 + ((cc + rr) & 15)];
        }
        __syncwarp();
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols));
  }
}

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

int* fused_err_word() {
  static int* words[64] = {nullptr};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  if (!words[dev]) {
    int* d = nullptr;
    if (cudaMalloc(&d, sizeof(int)) != cudaSuccess) return nullptr;
    if (cudaMemset(d, 0, sizeof(int)) != cudaSuccess) return nullptr;
    words[dev] = d;
  }
  return words[dev];
}

template <int PIECES, int COMPS>
cudaError_t launch_fused(const DevTables& T, const CUtensorMap& tb, int64_t P, const double* coord, double cutoff,
                         int n_out, int n_tile, int n_tiles, int kblocks, double* out, int* err, cudaStream_t s) {
  constexpr int PTS = BM / COMPS;
  const size_t stage = (size_t)PIECES * (A_TILE + (size_t)n_tile * BK * 2);
  const size_t smem = 1024 + STAGES * stage + (2 * STAGES + 2) * 8 + 3 * PTS * 8 + 16;
  auto kern = fused_mo_kernel<PIECES, COMPS>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)((P + PTS - 1) / PTS), (unsigned)n_tiles);
  kern<<<grid, kThreadsF, smem, s>>>(T, tb, P, coord, cutoff, n_out, n_tile, kblocks, out, err);
  count_launch();
  return cudaGetLastError();
}

}  // namespace

cudaError_t tc_run_fused(const DevTables& T, const TcPlan& plan, int64_t point_num, int comps, const double* coord,
                         double cutoff, const void* d_coef, double* out, cudaStream_t s) {
  if (point_num <= 0) return cudaSuccess;
  auto fn = encode_fn();
  if (!fn) return cudaErrorNotSupported;
  CUtensorMap tb;
  {
    cuuint64_t dims[3] = {(cuuint64_t)plan.ao_num, (cuuint64_t)plan.n_pad, (cuuint64_t)plan.pieces};
    cuuint64_t strides[2] = {(cuuint64_t)(plan.k_pad * 2), (cuuint64_t)(plan.n_pad * plan.k_pad * 2)};
    cuuint32_t box[3] = {(cuuint32_t)BK, (cuuint32_t)plan.n_tile, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(&tb, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(d_coef), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
  }
  int* err = fused_err_word();
  if (!err) return cudaErrorMemoryAllocation;
  const int kblocks = (int)((plan.ao_num + BK - 1) / BK);
  cudaError_t e;
  if (plan.pieces == 3)
    e = comps == 5 ? launch_fused<3, 5>(T, tb, point_num, coord, cutoff, (int)plan.mo_num, plan.n_tile, plan.n_tiles,
                                        kblocks, out, err, s)
                   : launch_fused<3, 1>(T, tb, point_num, coord, cutoff, (int)plan.mo_num, plan.n_tile, plan.n_tiles,
                                        kblocks, out, err, s);
  else
    e = comps == 5 ? launch_fused<2, 5>(T, tb, point_num, coord, cutoff, (int)plan.mo_num, plan.n_tile, plan.n_tiles,
                                        kblocks, out, err, s)
                   : launch_fused<2, 1>(T, tb, point_num, coord, cutoff, (int)plan.mo_num, plan.n_tile, plan.n_tiles,
                                        kblocks, out, err, s);
  if (e != cudaSuccess) return e;
  int h = 0;
  e = cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return e;
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  if (h != 0) {
    cudaMemsetAsync(err, 0, sizeof(int), s);
    return cudaErrorLaunchTimeout;
  }
  return cudaSuccess;
}

}  // namespace qb
