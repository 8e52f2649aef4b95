// Device pieces shared by the fused AO -> MO kernels (fused_tc.cu: one
// system, one tile per CTA; batch_tc.cu: many systems, persistent CTAs fed by
// a device work queue).
//
// A CTA owns a tile of points and an N tile of MOs.  Its 128 accumulator rows
// are (point, component) pairs: 25 points x 5 components (+3 zero rows) for
// MO VGL, 128 points for MO value.  Per 64-AO K block, producer warps evaluate
// the block's AOs at the tile's points and write them as 16-bit split pieces
// straight into the 128B-swizzled K-major shared-memory tile the tensor core
// reads; the coefficient pieces arrive by TMA; one thread issues the
// split tcgen05.mma chain into three FP32 TMEM accumulators (leading product
// in two K halves, corrections in the third); the epilogue sums them in FP64
// and undoes the power-of-two scales.
//
// AO arithmetic (mixed form): FP64 displacement, r^2, exponent argument and
// radial Laplacian factor, FP32 exponential when a r^2 <= 30 (FP64 above),
// FP64 radial accumulation, FP32 monomials and product rule; the screening
// follows qmckl_compute_ao_vgl_hpc_gaussian (org/qmckl_ao.org:8601-8973).
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>

#include "monomial.cuh"
#include "split.cuh"
#include "tc_ptx.cuh"

namespace qb {
namespace fz {

using namespace tcx;

constexpr int BM = 128, BK = 64, UMMA_K = 16;
constexpr int A_TILE = BM * BK * 2;

// Per-K-block record (built on the host): everything the producers need for
// the block's 64 AOs, so they never read device memory.
//   [0]    int32 nsh, nprim, 0, 0
//   [16]   64 x {int32 code (a|b<<4|c<<8|l<<12|local_shell<<16, -1 past ao_num), float ao_factor}
//   [528]  nsh x KRecShell
//   [...]  nprim x {double exponent, double coefficient} (sorted per shell)
// cusp_r2: the squared cusp radius of the shell's nucleus when the shell is
// an s shell that the cusp adjustment leaves out of the MOs within it
// (kernels.cuh cusp_masked; compared with r^2 <= cusp_r2), else -1.
struct KRecShell {
  double x, y, z, range;
  int32_t pb, pe;
  float cusp_r2;
  int32_t pad;
};
// Tile-skipping tables of the K blocks (built by build_fused_records in
// device.cu): int2 kb_sh[kblocks], the range of shell spheres of each K
// block, then, from byte kskip_sph_offset(kblocks) on, double4 sph[] (the
// shell's nucleus and the squared radius beyond which its AOs vanish in the
// producers).
__host__ __device__ constexpr int kskip_sph_offset(int kblocks) { return (kblocks * 8 + 31) / 32 * 32; }
// After the spheres: int2 kpos[shell_num], the K position of the first AO of
// each sphere's shell and its AO count (the 16-AO k-steps a live shell
// occupies).  shell_num is kb_sh[kblocks - 1].y, the end of the last block's
// range.
__host__ __device__ constexpr int kskip_kpos_offset(int kblocks, int shell_num) {
  return kskip_sph_offset(kblocks) + 32 * shell_num;
}

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
  // With S_n = sum_j c_j a_j^n e_j:  value S0, gradient -2 S1 (x, y, z),
  // Laplacian sum_j c_j (-2 a_j e_j)(3 - 2 a_j r^2) = 4 r^2 S2 - 6 S1, all in
  // FP64 (the Laplacian's cancellation happens before the FP32 rounding).
  double S0 = 0.0, S1 = 0.0, S2 = 0.0;
  live = !(r2 > cutoff * S.range) && !(r2 <= (double)S.cusp_r2);
  if (live) {
    for (int j = S.pb; j < S.pe; ++j) {
      const double2 pc = prm[j];
      const double ar2 = pc.x * r2;
      if (ar2 > cutoff) break;   // sorted by exponent
      const double e = ar2 > 30.0 ? exp(-ar2) : (double)expf(-(float)ar2);
      const double ce = pc.y * e;
      const double ace = pc.x * ce;
      S0 += ce;
      S1 += ace;
      S2 = fma(pc.x, ace, S2);
    }
  }
  const double g = -2.0 * S1;
  s[0] = (float)S0;
  s[1] = (float)(g * x);
  s[2] = (float)(g * y);
  s[3] = (float)(g * z);
  s[4] = (float)(fma(4.0 * r2, S2, -6.0 * S1));
}

// Per-row power-of-two scales of the 2-piece float16 operands (split.cuh).
// Each accumulator row (point i, component c) is scaled by 2^-e so that its
// AO values stay below 2^10 in magnitude; e comes from an upper bound of the
// row's AOs: max over the nuclei of a per-nucleus envelope of |AO|, |grad AO|
// or |lap AO| at the point's distance (RowBound.env, a suffix maximum over
// geometric radial cells: cell 0 = [0, r0), cell g >= 1 starts at
// r0 * 2^((g-1)/inv_log2q); built on the host).  Scales are exact, the
// epilogue multiplies the row by 2^e again.
constexpr int kEnvCells = 64;
constexpr int kExpMin = -60, kExpMax = 60;
struct RowBound {
  const double* nucl;   // [3][nucl_num]
  const float* env;     // [nucl_num][3][kEnvCells]: value, gradient, Laplacian envelopes
  int nucl_num;
  float r0, inv_log2q;
};

// 2^e for |e| <= 60, built from the exponent bits
__device__ __forceinline__ float pow2f(int e) { return __int_as_float((127 + e) << 23); }
__device__ __forceinline__ double pow2d(int e) { return __longlong_as_double((long long)(1023 + e) << 52); }

// envelope group of a component: value 0, gradient 1, Laplacian 2
template <int COMPS>
__device__ __forceinline__ int comp_group(int c) {
  return COMPS == 1 ? 0 : (c == 0 ? 0 : (c == 4 ? 2 : 1));
}

// rexp[3][PTS] (shared, preset to kExpMin) <- the scale exponents of the
// tile's rows; all threads of the CTA take part (then a barrier).
template <int PTS>
__device__ __forceinline__ void row_exponents(const RowBound& RB, const double* pts, const int64_t* pidx, int* rexp,
                                              int tid, int nthreads) {
  const int N = RB.nucl_num;
  for (int u = tid; u < PTS * N; u += nthreads) {
    const int i = u % PTS, n = u / PTS;
    if (pidx[i] < 0) continue;
    const double dx = pts[i] - RB.nucl[n], dy = pts[PTS + i] - RB.nucl[n + N], dz = pts[2 * PTS + i] - RB.nucl[n + 2 * N];
    const float r = sqrtf((float)(dx * dx + dy * dy + dz * dz));
    int g = 0;
    if (r >= RB.r0) {
      // lower cell on a rounding tie: a larger (still valid) bound
      const float x = log2f(r / RB.r0) * RB.inv_log2q - 1.0e-3f;
      g = x < 0.f ? 1 : min(kEnvCells - 1, 1 + (int)x);
    }
    const float* e = RB.env + (size_t)n * 3 * kEnvCells + g;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const float b = e[q * kEnvCells];
      if (b > 0.f) {
        int ex;
        frexpf(b * (1.0f / 1024.0f), &ex);
        atomicMax(&rexp[q * PTS + i], min(ex, kExpMax));
      }
    }
  }
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
  } else if (l <= 3) {
    // Per axis, r^a and its first two derivatives as one cubic each, by
    // Horner from the exponent's one-hot coefficients (a warp-uniform table
    // lookup, monomial.cuh): no selects, no branches.
    float X0, X1, XG, Y0, Y1, YG, Z0, Z1, ZG;
    axis_factors(x, kAxisHot[ax & 3], X0, X1, XG);
    axis_factors(y, kAxisHot[by & 3], Y0, Y1, YG);
    axis_factors(z, kAxisHot[cz & 3], Z0, Z1, ZG);
    const float xy = X0 * Y0, yz = Y0 * Z0, xz = X0 * Z0;
    P0 = xy * Z0;
    P1 = X1 * yz; P2 = Y1 * xz; P3 = Z1 * xy;
    P4 = 2.f * (XG * yz + YG * xz + ZG * xy);
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

// One producer warp's share of a K block: AOs [CHUNK*j, CHUNK*j + CHUNK) of
// the block (record `rec`) at the tile's points (pts [3][PTS] in shared
// memory; lanes are points), scaled by 2^-rexp[group][point] (2 pieces) and
// written as PIECES 16-bit pieces (split.cuh) into the
// swizzled A tiles at a_base (shared address; pieces A_TILE bytes apart).
// p_first: index of the tile's first point among the P points (rows past P
// are written as zeros).  Pairs of AOs that are zero at every point of the
// warp skip the split arithmetic.
// Tile skipping.  flags[kb] = 1 when some shell of K block kb reaches one of
// the tile's np points (pts: [3][PTS]), by the kskip tables (null: every
// block).  Warp w of nwarps takes blocks w, w + nwarps, ...; its lanes take
// the block's screening spheres, each tested against the points in shared
// memory (one load per lane, no chain of dependent loads).
template <int PTS>
__device__ __forceinline__ void tile_kblock_flags(const uint8_t* kskip, int kblocks, const double* pts, int np,
                                                  int* flags, int warp, int lane, int nwarps, bool ksteps = false) {
  // ksteps: the flag is the mask of the block's 16-AO k-steps that hold an AO
  // of a live shell (kpos table); otherwise 1 for a live block
  const int2* kb_sh = (const int2*)kskip;
  const double4* sph = kskip ? (const double4*)(kskip + kskip_sph_offset(kblocks)) : nullptr;
  const int2* kpos = (kskip && ksteps) ? (const int2*)(kskip + kskip_kpos_offset(kblocks, kb_sh[kblocks - 1].y))
                                       : nullptr;
  for (int kb = warp; kb < kblocks; kb += nwarps) {
    unsigned int mask = kskip == nullptr ? (ksteps ? 0xFu : 1u) : 0u;
    if (kskip != nullptr) {
      const int2 r = kb_sh[kb];
      for (int q0 = r.x; q0 < r.y && (kpos != nullptr || mask == 0u); q0 += 32) {
        const int q = q0 + lane;
        bool l = false;
        if (q < r.y) {
          const double4 c = sph[q];
          for (int i = 0; i < np && !l; ++i) {
            const double x = pts[i] - c.x, y = pts[PTS + i] - c.y, z = pts[2 * PTS + i] - c.z;
            l = x * x + y * y + z * z <= c.w;
          }
        }
        unsigned int m = 0u;
        if (l) {
          if (kpos != nullptr) {
            const int2 kp = kpos[q];
            const int k0 = max(kp.x, kb * 64) - kb * 64, k1 = min(kp.x + kp.y, kb * 64 + 64) - kb * 64;
            for (int kk = k0 >> 4; kk <= (k1 - 1) >> 4; ++kk) m |= 1u << kk;
          } else {
            m = 1u;
          }
        }
        mask |= __reduce_or_sync(0xffffffffu, m);
      }
    }
    if (lane == 0) flags[kb] = (int)mask;
  }
}

// One warp: the 16-AO k-steps that the MMAs of a tile issue, from the flags
// of tile_kblock_flags (k-step masks): the sum of their bits, or the four
// k-steps of the zero block that stands in when no block is alive.
__device__ __forceinline__ int tile_kstep_count(const int* flags, int kblocks, int lane) {
  int n = 0;
  for (int kb = lane; kb < kblocks; kb += 32) n += __popc((unsigned int)flags[kb]);
  n = __reduce_add_sync(0xffffffffu, n);
  return n == 0 ? BK / UMMA_K : n;
}

// One warp: the flagged K blocks in order into act[], and cnt[0..3] = their
// count, the first block of each half of K (-1: none) and the first block.
// With no block alive, one (zero) block 0 initialises the accumulators.
// Returns the count.
// With masks, each entry of act[] is kb | (k-step mask << 16).
__device__ __forceinline__ int tile_kblock_list(const int* flags, int kblocks, int* act, int* cnt, int lane,
                                                bool masks = false) {
  int n = 0, lo = -1, hi = -1, first = -1;
  for (int kb0 = 0; kb0 < kblocks; kb0 += 32) {
    const int kb = kb0 + lane;
    const bool f = kb < kblocks && flags[kb] != 0;
    const unsigned int m = __ballot_sync(0xffffffffu, f);
    const unsigned int mlo = __ballot_sync(0xffffffffu, f && 2 * kb < kblocks);
    const unsigned int mhi = __ballot_sync(0xffffffffu, f && 2 * kb >= kblocks);
    if (f) act[n + __popc(m & ((1u << lane) - 1u))] = kb | (masks ? (flags[kb] << 16) : 0);
    if (first < 0 && m != 0u) first = kb0 + __ffs(m) - 1;
    if (lo < 0 && mlo != 0u) lo = kb0 + __ffs(mlo) - 1;
    if (hi < 0 && mhi != 0u) hi = kb0 + __ffs(mhi) - 1;
    n += __popc(m);
  }
  if (n == 0) {
    if (lane == 0) act[0] = masks ? (0xF << 16) : 0;
    n = 1;
    lo = 0;
    first = 0;
  }
  if (lane == 0) {
    cnt[0] = n;
    cnt[1] = lo;
    cnt[2] = hi;
    cnt[3] = first;
  }
  return n;
}

template <int PIECES, int COMPS, int CHUNK>
__device__ __forceinline__ void produce_kblock(const uint8_t* rec, const double* pts, int64_t p_first, int64_t P,
                                               double cutoff, const int* rexp, uint32_t a_base, int j, int lane) {
  static_assert(CHUNK == 4 || CHUNK == 8, "a producer warp covers a half or a whole 16-byte chunk");
  constexpr int PTS = BM / COMPS;
  const int2* rao = (const int2*)(rec + kRecAoOff) + j * CHUNK;
  const KRecShell* rsh = (const KRecShell*)(rec + kRecShellOff);
  const double2* rprm = (const double2*)(rec + kRecShellOff + ((const int*)rec)[0] * (int)sizeof(KRecShell));
  for (int g = 0; g < (PTS + 31) / 32; ++g) {
    const int i = lane + 32 * g;
    const int ic = i < PTS ? i : PTS - 1;
    const bool active = i < PTS && p_first + i < P;
    const double px = pts[ic], py = pts[PTS + ic], pz = pts[2 * PTS + ic];
    float inv[COMPS];
#pragma unroll
    for (int c = 0; c < COMPS; ++c) inv[c] = PIECES == 2 ? pow2f(-rexp[comp_group<COMPS>(c) * PTS + ic]) : 1.0f;
    uint32_t pk[PIECES][COMPS][CHUNK / 2];
    int prev = -1;
    float rs[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    float fx = 0.f, fy = 0.f, fz = 0.f;
    bool live = false;
#pragma unroll
    for (int t = 0; t < CHUNK; t += 2) {
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
        // pieces of the two AOs, packed two per 32-bit word (split.cuh)
        uint32_t q3[3];
        split_pair<PIECES>(v[0][c], v[1][c], inv[c], q3);
#pragma unroll
        for (int q = 0; q < PIECES; ++q) pk[q][c][t >> 1] = q3[q];
      }
    }
    if (i < PTS) {
#pragma unroll
      for (int c = 0; c < COMPS; ++c) {
        const int r = i * COMPS + c;
        if (CHUNK == 4) {
          // 16-byte chunk j/2 of the 128-byte row (swizzled), 8-byte half j&1
          const uint32_t off = (uint32_t)(r * 128 + (((j >> 1) ^ (r & 7)) << 4) + ((j & 1) << 3));
#pragma unroll
          for (int q = 0; q < PIECES; ++q) st_shared_v2(a_base + q * A_TILE + off, pk[q][c][0], pk[q][c][1]);
        } else {
          const uint32_t off = (uint32_t)(r * 128 + ((j ^ (r & 7)) << 4));
#pragma unroll
          for (int q = 0; q < PIECES; ++q)
            st_shared_v4(a_base + q * A_TILE + off, pk[q][c][0], pk[q][c][1], pk[q][c][CHUNK / 2 - 2],
                         pk[q][c][CHUNK / 2 - 1]);
        }
      }
    }
  }
}

// The split-BF16 MMA chain of one K block from the stage at shared address
// `base` (A pieces, then B pieces): per 16-AO k-step the products of total
// order <= 2, the leading product A1 B1 into accumulator 0 for the first
// half of the K blocks and 1 for the second, whatever blocks a tile skips
// (so that a row's sums never depend on the other rows of its tile), the
// corrections into accumulator 2.  The products are issued A piece by A
// piece, each piece read once into the tensor core's collector buffer and
// kept for the products that follow with it (3 pieces: A1 B3, A1 B2, A1 B1,
// A2 B2, A2 B1, A3 B1; 2 pieces: A1 B2, A1 B1, A2 B1), so the MMAs read 12 KB
// less shared memory per k-step than with A read for every product.  The
// k-steps that vanish over the tile are skipped.  kmask: bit kk set when
// k-step kk (AOs [16 kk, 16 kk + 16) of the block) holds an AO of a live
// shell (0: all four); a skipped k-step would add exact zeros, so the sums
// are those of the full chain.  init[3]: whether accumulator 0 (leading
// product, first half of K), 1 (leading product, second half) or 2
// (corrections) holds a sum yet; the first MMA into each overwrites it.
// One k-step kk of that chain.  NACC = 3: the accumulators above; NACC = 2
// (wide MO tiles): the leading product in accumulator 0 for all of K, the
// corrections in accumulator 1 (li must be 0).
template <int PIECES, int NACC = 3>
__device__ __forceinline__ void mma_kstep(uint32_t base, uint32_t a_bytes, uint32_t b_tile, uint32_t tmem, int n_tile,
                                          uint32_t idesc, int li, int kk, bool (&init)[3]) {
  static_assert(NACC == 2 || NACC == 3, "two or three accumulators");
  const uint32_t dl = tmem + (uint32_t)(li * n_tile), dc = tmem + (uint32_t)((NACC - 1) * n_tile);
  const uint32_t a0 = base + kk * UMMA_K * 2, b0 = base + a_bytes + kk * UMMA_K * 2;
  const uint64_t A1 = smem_desc(a0), A2 = smem_desc(a0 + A_TILE);
  const uint64_t B1 = smem_desc(b0), B2 = smem_desc(b0 + b_tile);
  const uint32_t ic = init[NACC - 1] ? 1u : 0u, il = init[li] ? 1u : 0u;
  if constexpr (PIECES == 3) {
    const uint64_t A3 = smem_desc(a0 + 2 * A_TILE), B3 = smem_desc(b0 + 2 * b_tile);
    umma_bf16_ca<1>(dc, A1, B3, idesc, ic);
    umma_bf16_ca<2>(dc, A1, B2, idesc, 1u);
    umma_bf16_ca<3>(dl, A1, B1, idesc, il);
    umma_bf16_ca<1>(dc, A2, B2, idesc, 1u);
    umma_bf16_ca<3>(dc, A2, B1, idesc, 1u);
    umma_bf16(dc, A3, B1, idesc, 1u);
  } else {
    umma_bf16_ca<1>(dc, A1, B2, idesc, ic);
    umma_bf16_ca<3>(dl, A1, B1, idesc, il);
    umma_bf16(dc, A2, B1, idesc, 1u);
  }
  init[NACC - 1] = true;
  init[li] = true;
}

// Accumulator of the leading product for K block kb: 0 in the first half of
// the blocks, 1 in the second.
__device__ __forceinline__ int lead_acc(int kb, int kblocks) { return 2 * kb >= kblocks ? 1 : 0; }

template <int PIECES>
__device__ __forceinline__ void mma_kblock_masked(uint32_t base, uint32_t a_bytes, uint32_t b_tile, uint32_t tmem,
                                                  int n_tile, uint32_t idesc, int kb, int kblocks, uint32_t kmask,
                                                  bool (&init)[3]) {
  if (kmask == 0u) kmask = 0xFu;
  const int li = lead_acc(kb, kblocks);
  for (int kk = 0; kk < BK / UMMA_K; ++kk)
    if ((kmask >> kk) & 1u) mma_kstep<PIECES>(base, a_bytes, b_tile, tmem, n_tile, idesc, li, kk, init);
}

// Whether producer warp `warp` (AOs [chunk * warp, chunk * warp + chunk) of
// a K block) has work in a block whose act[] entry is `entry`: not when
// its k-step is skipped by the MMAs (its A tile is then never read).
__device__ __forceinline__ bool kstep_live(int entry, int warp, int chunk) {
  const uint32_t m = (uint32_t)entry >> 16;
  return m == 0u || ((m >> ((warp * chunk) >> 4)) & 1u) != 0u;
}

// Instruction descriptor of tcgen05.mma kind::f16: FP32 accumulator, A and B
// both bfloat16 (3 pieces) or both float16 (2 pieces), K-major, M = 128.
template <int PIECES>
__device__ __forceinline__ uint32_t mma_idesc(int n_tile) {
  const uint32_t fmt = PIECES == 3 ? 1u : 0u;
  return (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(n_tile >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

// Epilogue of one warp (TMEM lanes 32*(warp%4) .. +31, 16-column chunks
// chunk0, chunk0 + chunk_step, ...): FP64 sum of the three
// accumulators times the row scale 2^rexp and the MO scale (split.cuh), rows
// (tile point i, component c) written to out[(pidx[i] * COMPS + c) * n_out +
// col] for the MO columns [n0, n0 + n_tile).
// stage: 32 x 16 doubles of shared scratch for this warp.
template <int PIECES, int COMPS, int NACC = 3>
__device__ __forceinline__ void epilogue_warp(uint32_t tmem, int n_tile, int n0, int n_out, bool has_second,
                                              const int64_t* pidx, const int* rexp, const double* scales,
                                              double* out, double* stage, int warp, int lane, int chunk0 = 0,
                                              int chunk_step = 1, bool has_first = true) {
  constexpr int PTS = BM / COMPS;
  const int row_base = (warp & 3) * 32;   // a warp reads the TMEM lanes of its quadrant
  for (int c0 = 16 * chunk0; c0 < n_tile; c0 += 16 * chunk_step) {
    uint32_t r0[16], r1[16], r2[16];
    const uint32_t ta = tmem + ((uint32_t)row_base << 16) + (uint32_t)c0;
    tmem_ld16(ta, r0);
    tmem_ld16(ta + (uint32_t)n_tile, r1);
    if (NACC == 3) tmem_ld16(ta + (uint32_t)(2 * n_tile), r2);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      double v;
      if (NACC == 2) {   // leading product + corrections
        v = (double)__uint_as_float(r0[j]) + (double)__uint_as_float(r1[j]);
      } else {
        v = has_first ? (double)__uint_as_float(r0[j]) + (double)__uint_as_float(r2[j])
                      : (double)__uint_as_float(r2[j]);
        if (has_second) v += (double)__uint_as_float(r1[j]);
      }
      stage[lane * 16 + ((j + lane) & 15)] = v;
    }
    __syncwarp();
    const int cc = lane & 15;
    const int col = n0 + c0 + cc;
    const double cs = (PIECES == 2 && col < n_out) ? scales[kScaleCols + col] : 1.0;
    for (int q = 0; q < 16; ++q) {
      const int rr = 2 * q + (lane >> 4);
      const int r = row_base + rr;
      if (r < PTS * COMPS && col < n_out) {
        const int64_t pq = pidx[r / COMPS];
        if (pq >= 0) {
          const int c = r % COMPS, i = r / COMPS;
          double v = stage[rr * 16 + ((cc + rr) & 15)];
          if (PIECES == 2) v *= cs * pow2d(rexp[comp_group<COMPS>(c) * PTS + i]);
          out[(pq * COMPS + c) * n_out + col] = v;
        }
      }
    }
    __syncwarp();
  }
}

// Epilogue into shared memory: TMEM lane quadrant warp % 4, a share of the
// 16-column chunks, as epilogue_warp; row r (= point * COMPS + component) of
// the tile goes to stg + r * ldst in the same arithmetic.  ldst = n_tile + 2
// puts the 16-byte stores of a warp's 32 rows on 8 distinct bank groups.  The
// caller copies each row to its place in global memory with one bulk copy.
// Only the columns [col_lo, col_hi) of the tile (multiples of 16; column
// col_lo lands at stg + r * ldst), so that a wide tile can go out in passes.
template <int PIECES, int COMPS, int NACC = 3>
__device__ __forceinline__ void epilogue_stage_warp(uint32_t tmem, int n_tile, int n0, int n_out, bool has_second,
                                                    const int* rexp, const double* scales, double* stg, int ldst,
                                                    int warp, int lane, int chunk0, int chunk_step, bool has_first,
                                                    int col_lo = 0, int col_hi = 1 << 30) {
  constexpr int PTS = BM / COMPS;
  const int row_base = (warp & 3) * 32;
  const int r = row_base + lane;
  const bool row_ok = r < PTS * COMPS;
  const double rs = (PIECES == 2 && row_ok) ? pow2d(rexp[comp_group<COMPS>(r % COMPS) * PTS + r / COMPS]) : 1.0;
  const int c_end = min(n_tile, col_hi);
  for (int c0 = col_lo + 16 * chunk0; c0 < c_end; c0 += 16 * chunk_step) {
    uint32_t r0[16], r1[16], r2[16];
    const uint32_t ta = tmem + ((uint32_t)row_base << 16) + (uint32_t)c0;
    tmem_ld16(ta, r0);
    tmem_ld16(ta + (uint32_t)n_tile, r1);
    if (NACC == 3) tmem_ld16(ta + (uint32_t)(2 * n_tile), r2);
    if (row_ok) {
      double* dst = stg + (size_t)r * ldst + (c0 - col_lo);
#pragma unroll
      for (int j = 0; j < 16; j += 2) {
        double v[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          double x;
          if (NACC == 2) {   // leading product + corrections
            x = (double)__uint_as_float(r0[j + h]) + (double)__uint_as_float(r1[j + h]);
          } else {
            x = has_first ? (double)__uint_as_float(r0[j + h]) + (double)__uint_as_float(r2[j + h])
                          : (double)__uint_as_float(r2[j + h]);
            if (has_second) x += (double)__uint_as_float(r1[j + h]);
          }
          if (PIECES == 2) {
            const int col = n0 + c0 + j + h;
            x *= (col < n_out ? scales[kScaleCols + col] : 1.0) * rs;
          }
          v[h] = x;
        }
        *reinterpret_cast<double2*>(dst + j) = make_double2(v[0], v[1]);
      }
    }
  }
}

// Zero the rows PTS*COMPS .. 127 of every A tile (they stay zero).
template <int PIECES, int COMPS, int STAGES>
__device__ __forceinline__ void zero_pad_rows(uint8_t* smem, int stage_bytes, int tid, int nthreads) {
  constexpr int PTS = BM / COMPS;
  constexpr int PAD = BM - PTS * COMPS;
  if constexpr (PAD > 0) {
    for (int t = tid; t < STAGES * PIECES * PAD * 8; t += nthreads) {
      const int chunk = t & 7;
      const int rr = (t >> 3) % PAD;
      const int tile = (t >> 3) / PAD;   // stage * PIECES + piece
      const int r = PTS * COMPS + rr;
      uint8_t* base = smem + (tile / PIECES) * stage_bytes + (tile % PIECES) * A_TILE;
      st_shared_v4(smem_addr(base + r * 128 + ((chunk ^ (r & 7)) << 4)), 0u, 0u, 0u, 0u);
    }
  }
}

}  // namespace fz
}  // namespace qb
