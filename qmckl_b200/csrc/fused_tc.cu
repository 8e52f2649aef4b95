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
constexpr int kProdWarps = 16;   // one warp per 4-AO chunk of the 64-AO K block
constexpr int kChunk = BK / kProdWarps;
constexpr int kProd = kProdWarps * 32;
constexpr int kTmaWarp = kProdWarps;
constexpr int kMmaWarp = kProdWarps + 1;
constexpr int kThreadsF = (kProdWarps + 2) * 32;
constexpr int A_TILE = BM * BK * 2;
constexpr int STAGES = 2;

// Per-K-block record (built on the host, see device.cu): everything the
// producers need for the block's 64 AOs, so they never read device memory.
//   [0]    int32 nsh, nprim, 0, 0
//   [16]   64 x {int32 code (a|b<<4|c<<8|l<<12|local_shell<<16, -1 past ao_num), float ao_factor}
//   [528]  nsh x KRecShell
//   [...]  nprim x {double exponent, double coefficient} (sorted per shell)
struct KRecShell {
  double x, y, z, range;
  int32_t pb, pe, pad0, pad1;
};
constexpr int kRecAoOff = 16;
constexpr int kRecShellOff = 16 + 64 * 8;

// Radial VGL of one shell at one point from a K-block record in shared memory.
__device__ __forceinline__ void radial_rec(const KRecShell& S, const double2* prm, double px, double py, double pz,
                                           double cutoff, float (&s)[5], float& fx, float& fy, float& fz,
                                           bool& live) {
  const double x = px - S.x;
  const double y = py - S.y;
  const double z = pz - S.z;
  const double r2 = x * x + y * y + z * z;
  fx = (float)x;
  fy = (float)y;
  fz = (float)z;
  double acc[5] = {0., 0., 0., 0., 0.};
  live = !(r2 > cutoff * S.range);
  if (live) {
    for (int j = S.pb; j < S.pe; ++j) {
      const double2 pc = prm[j];
      const double ar2 = pc.x * r2;
      if (ar2 > cutoff) break;   // sorted by exponent
      const double e = ar2 > 30.0 ? exp(-ar2) : (double)expf(-(float)ar2);
      const double f = -2.0 * pc.x * e;
      acc[0] += pc.y * e;
      acc[1] += pc.y * (f * x);
      acc[2] += pc.y * (f * y);
      acc[3] += pc.y * (f * z);
      acc[4] += pc.y * (f * (3.0 - 2.0 * ar2));
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
    if (l <= 3) {   // branch-free powers
      const float x2 = x * x, y2 = y * y, z2 = z * z;
      const float xs[4] = {1.f, x, x2, x2 * x}, ys[4] = {1.f, y, y2, y2 * y}, zs[4] = {1.f, z, z2, z2 * z};
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (ax == q) { pa = xs[q]; pa1 = q >= 1 ? xs[q - 1] : 1.f; pa2 = q >= 2 ? xs[q - 2] : 1.f; }
        if (by == q) { pb = ys[q]; pb1 = q >= 1 ? ys[q - 1] : 1.f; pb2 = q >= 2 ? ys[q - 2] : 1.f; }
        if (cz == q) { pc = zs[q]; pc1 = q >= 1 ? zs[q - 1] : 1.f; pc2 = q >= 2 ? zs[q - 2] : 1.f; }
      }
    } else {
      for (int i = 0; i < ax; ++i) { pa2 = pa1; pa1 = pa; pa *= x; }
      for (int i = 0; i < by; ++i) { pb2 = pb1; pb1 = pb; pb *= y; }
      for (int i = 0; i < cz; ++i) { pc2 = pc1; pc1 = pc; pc *= z; }
    }
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
                const int kblocks, const uint8_t* __restrict__ krec, const int rec_bytes,
                const int* __restrict__ perm, double* __restrict__ out, int* __restrict__ err) {
  constexpr int NPROD = PIECES == 3 ? 6 : 3;
  constexpr int PTS = BM / COMPS;            // 25 points (VGL) or 128 (value)
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // 1024-byte aligned base, kept as pointer arithmetic on the __shared__
  // array so that accesses compile to shared-memory (not generic) loads
  uint8_t* smem = smem_raw + ((1024u - (tcx::smem_addr(smem_raw) & 1023u)) & 1023u);
  const int B_TILE = n_tile * BK * 2;
  const int A_BYTES = PIECES * A_TILE;
  const int STAGE = PIECES * (A_TILE + B_TILE);
  uint8_t* recs = smem + STAGES * STAGE;      // STAGES K-block records
  uint64_t* full = (uint64_t*)(recs + STAGES * rec_bytes);
  uint64_t* empty = full + STAGES;
  uint64_t* rec_full = empty + STAGES;
  uint64_t* acc_full = rec_full + STAGES;
  uint32_t* tmem_slot = (uint32_t*)(acc_full + 1);
  double* pts = (double*)(acc_full + 2);      // [3][PTS]
  int64_t* pidx = (int64_t*)(pts + 3 * PTS);  // [PTS] original index of each tile point

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t p0 = (int64_t)blockIdx.x * PTS;
  const int n0 = blockIdx.y * n_tile;
  uint32_t tmem_cols = 32;
  while ((int)tmem_cols < 3 * n_tile) tmem_cols <<= 1;

  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], kProd + 1);
      mbar_init(&empty[s], 1);
      mbar_init(&rec_full[s], 1);
    }
    mbar_init(acc_full, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int t = tid; t < 3 * PTS; t += kThreadsF) {
    const int d = t / PTS, i = t - d * PTS;
    const int64_t q = (p0 + i < P) ? (perm ? (int64_t)perm[p0 + i] : p0 + i) : -1;
    pts[t] = q >= 0 ? coord[q + d * P] : 0.0;
    if (d == 0) pidx[i] = q;
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
    // ---------------- AO producers: warp w owns AOs [4w, 4w+4) of each K block,
    // its lanes are the tile's points (uniform control flow within the warp)
    const int j = warp;
    for (int kb = 0; kb < kblocks; ++kb) {
      const int s = kb & 1;
      const uint32_t phase = (uint32_t)(kb >> 1) & 1u;
      // warp-uniform outcome: every lane must take the same path
      bool ok = mbar_wait(&empty[s], phase ^ 1u, err, 11);
      ok = ok && mbar_wait(&rec_full[s], phase, err, 15);
      if (!__all_sync(0xffffffffu, ok)) break;
      const uint32_t a_base = smem_addr(smem + s * STAGE);
      const uint8_t* rec = recs + s * rec_bytes;
      const int2* rao = (const int2*)(rec + kRecAoOff) + j * kChunk;
      const KRecShell* rsh = (const KRecShell*)(rec + kRecShellOff);
      const double2* rprm = (const double2*)(rec + kRecShellOff + ((const int*)rec)[0] * (int)sizeof(KRecShell));
      for (int g = 0; g < (PTS + 31) / 32; ++g) {
        const int i = lane + 32 * g;
        const int ic = i < PTS ? i : PTS - 1;
        const bool active = i < PTS && p0 + i < P;
        const double px = pts[ic], py = pts[PTS + ic], pz = pts[2 * PTS + ic];
        uint32_t pk[PIECES][COMPS][kChunk / 2];
        int prev = -1;
        float rs[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
        float fx = 0.f, fy = 0.f, fz = 0.f;
        bool live = false;
#pragma unroll
        for (int t = 0; t < kChunk; t += 2) {
          float v[2][5];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int2 e = rao[t + h];                 // same address in every lane: broadcast
            const int code = e.x;
            const int sh = code < 0 ? -1 : (code >> 16);
            const float f = __int_as_float(e.y);
#pragma unroll
            for (int c = 0; c < 5; ++c) v[h][c] = 0.f;
            if (sh >= 0) {
              if (sh != prev) {   // sh is warp-uniform
                if (active) radial_rec(rsh[sh], rprm, px, py, pz, cutoff, rs, fx, fy, fz, live);
                prev = sh;
              }
              if (active && live && rs[0] != 0.f) ao_product(code & 0xFFFF, f, rs, fx, fy, fz, v[h]);
            }
          }
          bool nz = false;
#pragma unroll
          for (int c = 0; c < COMPS; ++c) nz = nz || v[0][c] != 0.f || v[1][c] != 0.f;
          if (!__any_sync(0xffffffffu, nz)) {   // both AOs zero at every point of the warp
#pragma unroll
            for (int c = 0; c < COMPS; ++c)
#pragma unroll
              for (int q = 0; q < PIECES; ++q) pk[q][c][t >> 1] = 0u;
            continue;
          }
#pragma unroll
          for (int c = 0; c < COMPS; ++c) {
            // round-to-nearest bf16 pieces of the two AOs, packed as bf16x2
            const __nv_bfloat162 h2 = __floats2bfloat162_rn(v[0][c], v[1][c]);
            const float2 hf = __bfloat1622float2(h2);
            const float r0 = v[0][c] - hf.x, r1 = v[1][c] - hf.y;
            const __nv_bfloat162 m2 = __floats2bfloat162_rn(r0, r1);
            pk[0][c][t >> 1] = *reinterpret_cast<const uint32_t*>(&h2);
            pk[1][c][t >> 1] = *reinterpret_cast<const uint32_t*>(&m2);
            if (PIECES == 3) {
              const float2 mf = __bfloat1622float2(m2);
              const __nv_bfloat162 l2 = __floats2bfloat162_rn(r0 - mf.x, r1 - mf.y);
              pk[PIECES - 1][c][t >> 1] = *reinterpret_cast<const uint32_t*>(&l2);
            }
          }
        }
        if (i < PTS) {
#pragma unroll
          for (int c = 0; c < COMPS; ++c) {
            const int r = i * COMPS + c;
            // 16-byte chunk j/2 of the 128-byte row (swizzled), 8-byte half j&1
            const uint32_t off = (uint32_t)(r * 128 + (((j >> 1) ^ (r & 7)) << 4) + ((j & 1) << 3));
#pragma unroll
            for (int q = 0; q < PIECES; ++q) st_shared_v2(a_base + q * A_TILE + off, pk[q][c][0], pk[q][c][1]);
          }
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
        mbar_expect_tx(&rec_full[s], (uint32_t)rec_bytes);
        bulk_load(recs + s * rec_bytes, krec + (size_t)kb * rec_bytes, (uint32_t)rec_bytes, &rec_full[s]);
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
          const int col = n0 + c0 + cc;
          if (r < PTS * COMPS && col < n_out) {
            const int64_t q = pidx[r / COMPS];
            if (q >= 0) out[(q * COMPS + r % COMPS) * n_out + col] = stage[rr * 16 + ((cc + rr) & 15)];
          }
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
size_t fused_smem(int n_tile, int rec_bytes) {
  constexpr int PTS = BM / COMPS;
  const size_t stage = (size_t)PIECES * (A_TILE + (size_t)n_tile * BK * 2);
  return 1024 + STAGES * stage + (size_t)STAGES * rec_bytes + (3 * STAGES + 2) * 8 + 4 * PTS * 8 + 16;
}

template <int PIECES, int COMPS>
cudaError_t launch_fused(const DevTables& T, const CUtensorMap& tb, int64_t P, const double* coord, double cutoff,
                         int n_out, int n_tile, int n_tiles, int kblocks, const uint8_t* krec, int rec_bytes,
                         const int* perm, double* out, int* err, cudaStream_t s) {
  constexpr int PTS = BM / COMPS;
  const size_t smem = fused_smem<PIECES, COMPS>(n_tile, rec_bytes);
  auto kern = fused_mo_kernel<PIECES, COMPS>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)((P + PTS - 1) / PTS), (unsigned)n_tiles);
  kern<<<grid, kThreadsF, smem, s>>>(T, tb, P, coord, cutoff, n_out, n_tile, kblocks, krec, rec_bytes, perm, out, err);
  count_launch();
  return cudaGetLastError();
}

}  // namespace

size_t tc_fused_smem(const TcPlan& plan, int comps, int rec_bytes) {
  if (plan.pieces == 3) return comps == 5 ? fused_smem<3, 5>(plan.n_tile, rec_bytes) : fused_smem<3, 1>(plan.n_tile, rec_bytes);
  return comps == 5 ? fused_smem<2, 5>(plan.n_tile, rec_bytes) : fused_smem<2, 1>(plan.n_tile, rec_bytes);
}

cudaError_t tc_run_fused(const DevTables& T, const TcPlan& plan, int64_t point_num, int comps, const double* coord,
                         double cutoff, const void* d_coef, const void* krec, int rec_bytes, const int* perm,
                         double* out, cudaStream_t s) {
  if (point_num <= 0) return cudaSuccess;
  if (rec_bytes <= 0 || rec_bytes % 128 != 0) return cudaErrorInvalidValue;
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
                                        kblocks, (const uint8_t*)krec, rec_bytes, perm, out, err, s)
                   : launch_fused<3, 1>(T, tb, point_num, coord, cutoff, (int)plan.mo_num, plan.n_tile, plan.n_tiles,
                                        kblocks, (const uint8_t*)krec, rec_bytes, perm, out, err, s);
  else
    e = comps == 5 ? launch_fused<2, 5>(T, tb, point_num, coord, cutoff, (int)plan.mo_num, plan.n_tile, plan.n_tiles,
                                        kblocks, (const uint8_t*)krec, rec_bytes, perm, out, err, s)
                   : launch_fused<2, 1>(T, tb, point_num, coord, cutoff, (int)plan.mo_num, plan.n_tile, plan.n_tiles,
                                        kblocks, (const uint8_t*)krec, rec_bytes, perm, out, err, s);
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

// ---------------------------------------------------------------- point order
//
// Tiles of spatially close points share their zero AOs, which the producers
// of the fused kernel skip a pair of AOs at a time.  Points are bucketed into
// the cells of a 32^3 grid over the box of the nuclei (coordinates clamped),
// ordered by Morton code.
// The order within a cell does not affect any result: every output row is a
// function of its own point only.
namespace qb {
namespace {

__device__ __forceinline__ unsigned int spread5(unsigned int x) {   // 5 bits -> every third bit
  x &= 31u;
  x = (x | (x << 8)) & 0x0300F00Fu;
  x = (x | (x << 4)) & 0x030C30C3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}

__global__ void point_keys_kernel(const double* __restrict__ coord, int64_t P, double3 origin, double inv_cell,
                                  int* __restrict__ keys, unsigned int* __restrict__ counts) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < P; p += (int64_t)gridDim.x * blockDim.x) {
    int c[3];
    const double o[3] = {origin.x, origin.y, origin.z};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double v = floor((coord[p + d * P] - o[d]) * inv_cell);
      c[d] = (int)fmin(31.0, fmax(0.0, v));
    }
    const int key = (int)(spread5(c[0]) | (spread5(c[1]) << 1) | (spread5(c[2]) << 2));
    keys[p] = key;
    atomicAdd(&counts[key], 1u);
  }
}

// exclusive scan of kSortCells counts in one CTA of 1024 threads
__global__ void __launch_bounds__(1024) scan_cells_kernel(unsigned int* counts) {
  constexpr int PER = kSortCells / 1024;
  __shared__ unsigned int part[1024];
  unsigned int local[PER];
  unsigned int sum = 0;
  const int base = threadIdx.x * PER;
#pragma unroll
  for (int i = 0; i < PER; ++i) { local[i] = counts[base + i]; sum += local[i]; }
  part[threadIdx.x] = sum;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const unsigned int v = threadIdx.x >= off ? part[threadIdx.x - off] : 0u;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  unsigned int run = part[threadIdx.x] - sum;
#pragma unroll
  for (int i = 0; i < PER; ++i) { counts[base + i] = run; run += local[i]; }
}

__global__ void scatter_points_kernel(const int* __restrict__ keys, int64_t P, unsigned int* __restrict__ offsets,
                                      int* __restrict__ perm) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < P; p += (int64_t)gridDim.x * blockDim.x) {
    const unsigned int pos = atomicAdd(&offsets[keys[p]], 1u);
    perm[pos] = (int)p;
  }
}

}  // namespace

cudaError_t point_order(const double* coord, int64_t point_num, const double* box_lo, const double* box_hi,
                        int* keys, unsigned int* counts, int* perm, cudaStream_t s) {
  // 32 cells per axis over the box of the nuclei (cells at least 1 bohr wide)
  double ext = 0.0;
  for (int d = 0; d < 3; ++d) ext = std::max(ext, box_hi[d] - box_lo[d]);
  const double cell = std::max(1.0, ext / 32.0);
  const double3 origin = make_double3(box_lo[0], box_lo[1], box_lo[2]);
  if (point_num <= 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(counts, 0, sizeof(unsigned int) * kSortCells, s);
  if (e != cudaSuccess) return e;
  const int grid = (int)std::min<int64_t>((point_num + 255) / 256, 148 * 8);
  point_keys_kernel<<<grid, 256, 0, s>>>(coord, point_num, origin, 1.0 / cell, keys, counts);
  scan_cells_kernel<<<1, 1024, 0, s>>>(counts);
  scatter_points_kernel<<<grid, 256, 0, s>>>(keys, point_num, counts, perm);
  count_launch(3);
  return cudaGetLastError();
}

}  // namespace qb
