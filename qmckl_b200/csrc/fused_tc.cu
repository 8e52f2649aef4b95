// Fused mixed-form AO -> MO evaluation of one system: the AO matrix never
// leaves the SM.  One CTA per (tile of points, N tile of MOs); the shared
// device pieces (AO production into swizzled split-BF16 tiles, MMA chain,
// epilogue) and their arithmetic are described in fused_common.cuh.
// Warp roles: warps 0..15 produce the AO pieces of the 64-AO K blocks (4-AO
// chunks claimed in order from a shared counter, lanes = points); warp 16
// bulk-copies the blocks' records, TMA-loads the coefficient pieces and
// publishes the count of blocks whose MMAs are done; warp 17 owns TMEM and
// issues the MMAs; the 16 producer warps then run the epilogue (4 per TMEM
// lane quadrant).  Every wait is bounded (2 s of %globaltimer); a timeout
// sets the error word and the CTA still releases its TMEM.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>

#include "fused_common.cuh"
#include "mo_tc.cuh"

namespace qb {
namespace {

using namespace tcx;

using namespace fz;

constexpr int kChunks = 16;      // 4-AO chunks of a 64-AO K block, 4 per 16-AO k-step
constexpr int kChunk = BK / kChunks;
constexpr int kProdWarps = 16;   // producer warps (a multiple of 4: the epilogue splits them by TMEM quadrant)
constexpr int kProd = kProdWarps * 32;
constexpr int kTmaWarp = kProdWarps;
constexpr int kMmaWarp = kProdWarps + 1;
constexpr int kThreadsF = (kProdWarps + 2) * 32;
constexpr int STAGES = 2;
constexpr int kKsteps = BK / UMMA_K;   // 16-AO k-steps per K block, 4 chunks each

// Tile skipping: kskip (optional; layout in fused_common.cuh) lists, per K
// block, the screening spheres of its shells.  A K block whose shells are
// all beyond their radius at every point of the tile contributes exact zeros
// and is left out of the producer, TMA and MMA loops.

// Test hook (qmckl_b200_inject_late_warps): nanoseconds that every producer
// warp holding a chunk of a skipped k-step sleeps before its stage wait, so
// that the MMAs of its block can complete first.  Non-zero selects the LATE
// instantiation of the kernel (3 pieces, VGL); the others compile it out.
std::atomic<unsigned int> g_late_warp_ns{0u};

// NACC = 3: three accumulators of n_tile <= 160 columns (the leading
// product in two halves of K, the corrections), each stage holding its A
// and coefficient tiles.  NACC = 2 (wide MO tiles, n_tile <= 256, with a tile
// plan only): the leading product in one accumulator, the corrections in the
// other, and a single coefficient tile after the NST A stages (three where
// they fit, else two), loaded for block it once the MMAs of block it - 1 are
// done; the epilogue writes the tile in column passes that fit the idle
// stage memory.
template <int PIECES, int COMPS, int NACC, int NST, bool LATE = false>
__global__ void __launch_bounds__(kThreadsF, 1)
fused_mo_kernel(const DevTables T, const __grid_constant__ CUtensorMap tmB, const int64_t P,
                const double* __restrict__ coord, const double cutoff, const int n_out, const int n_tile,
                const int kblocks, const uint8_t* __restrict__ krec, const int rec_bytes,
                const int* __restrict__ perm, const double* __restrict__ scales, const RowBound rb,
                double* __restrict__ out, int* __restrict__ err, const int64_t cstride,
                const uint8_t* __restrict__ kskip, unsigned long long* __restrict__ kstat,
                const double* __restrict__ tpts, const int* __restrict__ tinfo, const unsigned int late_ns) {
  constexpr int PTS = BM / COMPS;            // 25 points (VGL) or 128 (value)
  // NST stages of the A tiles: 2 for NACC = 3 (each with its coefficient
  // tile), 2 or 3 for wide MO tiles
  static_assert(NACC == 2 || NST == STAGES, "three accumulators: two stages");
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // 1024-byte aligned base, kept as pointer arithmetic on the __shared__
  // array so that accesses compile to shared-memory (not generic) loads
  uint8_t* smem = smem_raw + ((1024u - (tcx::smem_addr(smem_raw) & 1023u)) & 1023u);
  const int B_TILE = n_tile * BK * 2;
  const int A_BYTES = PIECES * A_TILE;
  const int STAGE = NACC == 3 ? PIECES * (A_TILE + B_TILE) : A_BYTES;
  // offset of the coefficient tile from the start of stage s
  auto b_off = [&](int s) { return NACC == 3 ? A_BYTES : (NST - s) * STAGE; };
  const int STAGE_MEM = NST * STAGE + (NACC == 3 ? 0 : PIECES * B_TILE);
  uint8_t* recs = smem + STAGE_MEM;           // NST K-block records
  // Barriers: full[4 s + kk], k-step kk of the block in stage s produced (its
  // four chunks, or the MMA thread in their place when the k-step is
  // skipped); bfull[s], the block's coefficient pieces landed; empty[s], all
  // the block's MMAs done (the stage and its record slot free); rec_full[s],
  // its record landed.
  uint64_t* full = (uint64_t*)(recs + NST * rec_bytes);
  uint64_t* bfull = full + NST * kKsteps;
  uint64_t* empty = bfull + NST;
  uint64_t* rec_full = empty + NST;
  uint64_t* acc_full = rec_full + NST;
  uint32_t* tmem_slot = (uint32_t*)(acc_full + 1);
  double* pts = (double*)(acc_full + 2);      // [3][PTS]
  int64_t* pidx = (int64_t*)(pts + 3 * PTS);  // [PTS] original index of each tile point
  int* rexp = (int*)(pidx + PTS);             // [3][PTS] row scale exponents (2 pieces)
  int* act = rexp + 3 * PTS;                  // [kblocks] the K blocks of this tile, [kblocks] flags,
  int* kflag = act + kblocks;                 // then: count, first block of each half, first block
  int* nact_p = kflag + kblocks;
  int* claim = nact_p + 4;                    // chunks claimed by the producer warps after their first
  int* released = claim + 1;                  // K blocks whose MMAs the TMA thread has seen done

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t p0 = (int64_t)blockIdx.x * PTS;
  const int n0 = blockIdx.y * n_tile;
  uint32_t tmem_cols = 32;
  while ((int)tmem_cols < NACC * n_tile) tmem_cols <<= 1;

  // loads of K block kb (the it-th of the tile) into stage it % NST: the
  // block's record and its coefficient pieces
  auto load_record = [&](int it, int kb) {
    const int s = it % NST;
    mbar_expect_tx(&rec_full[s], (uint32_t)rec_bytes);
    bulk_load(recs + s * rec_bytes, krec + (size_t)kb * rec_bytes, (uint32_t)rec_bytes, &rec_full[s]);
  };
  auto load_coef = [&](int it, int kb) {
    const int s = it % NST;
    uint8_t* st = smem + s * STAGE + b_off(s);
    mbar_expect_tx(&bfull[s], (uint32_t)(PIECES * B_TILE));
    for (int q = 0; q < PIECES; ++q) tma_load_3d(st + q * B_TILE, &tmB, &bfull[s], kb * BK, n0, q);
  };
  int tma_pre = 0;   // K blocks whose loads the TMA thread issued during the prologue
  if (tid == kTmaWarp * 32) {
    for (int s = 0; s < NST; ++s) {
      for (int kk = 0; kk < kKsteps; ++kk) mbar_init(&full[s * kKsteps + kk], kChunks / kKsteps * 32);
      mbar_init(&bfull[s], 1);
      mbar_init(&empty[s], 1);
      mbar_init(&rec_full[s], 1);
    }
    mbar_init(acc_full, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (tinfo != nullptr) {
      // with a tile plan the first K blocks are known at once: their loads
      // (into stages not used yet, nothing to wait for) run under the prologue
      const int* ti = tinfo + (size_t)blockIdx.x * (kblocks + 4);
      const int n = ti[0];
      tma_pre = n < NST ? n : NST;
      for (int it = 0; it < tma_pre; ++it) {
        load_record(it, ti[4 + it] & 0xFFFF);
        if (NACC == 3 || it == 0) load_coef(it, ti[4 + it] & 0xFFFF);   // one coefficient tile (NACC 2)
      }
    }
  }
  for (int t = tid; t < 3 * PTS; t += kThreadsF) {
    const int d = t / PTS, i = t - d * PTS;
    const int64_t q = (p0 + i < P) ? (perm ? (int64_t)perm[p0 + i] : p0 + i) : -1;
    // with a tile plan the coordinates come gathered in tile order
    pts[t] = tpts != nullptr ? tpts[(size_t)blockIdx.x * 3 * PTS + t] : (q >= 0 ? coord[q + d * cstride] : 0.0);
    if (d == 0) pidx[i] = q;
    rexp[t] = PIECES == 2 ? kExpMin : 0;
  }
  if (tid == 0) {
    *claim = 0;
    *released = 0;
  }
  if (tinfo != nullptr) {   // the tile's K-block list, made by tile_plan_kernel
    const int* ti = tinfo + (size_t)blockIdx.x * (kblocks + 4);
    for (int t = tid; t < kblocks + 4; t += kThreadsF) {
      if (t < 4) nact_p[t] = ti[t];
      else act[t - 4] = ti[t];
    }
  }
  __syncthreads();
  if (PIECES == 2) row_exponents<PTS>(rb, pts, pidx, rexp, tid, kThreadsF);
  // K blocks that are not identically zero over the tile's points
  if (tinfo == nullptr) {
    tile_kblock_flags<PTS>(kskip, kblocks, pts, (int)(P - p0 < PTS ? P - p0 : PTS), kflag, warp, lane, kThreadsF / 32,
                           true);
    __syncthreads();
    if (warp == 0) {
      tile_kblock_list(kflag, kblocks, act, nact_p, lane, true);
      if (kstat != nullptr) {   // 16-AO k-steps issued / in the dense contraction, summed over CTAs
        const int ks = tile_kstep_count(kflag, kblocks, lane);
        if (lane == 0) {
          atomicAdd(&kstat[0], (unsigned long long)ks);
          atomicAdd(&kstat[1], (unsigned long long)kblocks * (BK / UMMA_K));
        }
      }
    }
  }
  // rows PTS*COMPS .. 127 of the A tiles stay zero for the whole kernel
  zero_pad_rows<PIECES, COMPS, NST>(smem, STAGE, tid, kThreadsF);
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
  const int nact = *nact_p;

  if (warp < kProdWarps) {
    // ---------------- AO producers.  The work comes in chunks of 4 AOs of a K
    // block (chunk c: AOs [4c, 4c+4), lanes = the tile's points, so control
    // flow is uniform within the warp), numbered block by block; each warp
    // takes the next unclaimed chunk from a shared counter (its first one is
    // chunk `warp` of the first block).  A warp done early goes on with the
    // next chunks, into the next block's stage once that stage is free,
    // instead of waiting for the slowest warp of its block.  Chunks are
    // claimed in order, so every chunk of a block is taken before any chunk
    // of a later block: a warp waiting for a stage waits only for blocks
    // whose chunks are all in progress.
    // A chunk of a skipped k-step is never read by the MMAs: it waits only
    // until the MMAs of the block NST back are done (as every chunk does,
    // which keeps any warp from claiming a chunk NST blocks past a stage
    // still in use) and does not arrive; the MMA thread arrives for the
    // whole skipped k-step.  Since the block's MMAs need none of its
    // arrivals, they may finish before such a warp reaches its wait: a
    // parity wait on the stage barrier alone would then read the barrier a
    // phase late and wait for the stage's next use.  So its wait also ends
    // when the count of blocks released (published by the TMA thread after
    // its own waits on the same barriers, and only growing) shows the block
    // NST back done.
    const int total = nact * kChunks;
    for (int q = warp; q < total;) {
      const int it = q / kChunks, c = q - it * kChunks;
      const int s = it % NST;
      const uint32_t phase = (uint32_t)(it / NST) & 1u;
      const bool live = kstep_live(act[it], c, kChunk);
      // warp-uniform outcome: every lane must take the same path.  A
      // produced chunk also waits for the block's record.  Its arrival comes
      // after the stage's release, that is after the MMA thread has waited
      // for the same full[] barrier's phase of the block NST back, so no
      // phase of a barrier mixes the arrivals of two blocks and no parity
      // wait falls two phases behind.
      bool ok;
      if (live) {
        ok = mbar_wait(&empty[s], phase ^ 1u, err, 11) && mbar_wait(&rec_full[s], phase, err, 15);
      } else {
        if constexpr (LATE)
          for (unsigned int t = 0; t < late_ns; t += 1000u) __nanosleep(1000u);
        ok = mbar_wait_or_count(&empty[s], phase ^ 1u, released, it - NST + 1, err, 16);
      }
      if (!__all_sync(0xffffffffu, ok)) break;
      if (live) {
        const uint32_t a_base = smem_addr(smem + s * STAGE);
        produce_kblock<PIECES, COMPS, kChunk>(recs + s * rec_bytes, pts, p0, P, cutoff, rexp, a_base, c, lane);
        fence_async_smem();
        mbar_arrive(&full[s * kKsteps + c / (kChunks / kKsteps)]);
      }
      int nq = 0;
      if (lane == 0) nq = atomicAdd(claim, 1) + kProdWarps;
      q = __shfl_sync(0xffffffffu, nq, 0);
    }
  } else if (warp == kTmaWarp) {
    // ---------------- records and coefficient pieces
    if (lane == 0) {
      if (NACC == 3) {
        for (int it = tma_pre; it < nact; ++it) {
          const int s = it % NST;
          const uint32_t phase = (uint32_t)(it / NST) & 1u;
          // the stage, its record slot included: every MMA of block it - NST done
          if (!mbar_wait(&empty[s], phase ^ 1u, err, 12)) break;
          if (it >= NST) *(volatile int*)released = it - NST + 1;
          load_record(it, act[it] & 0xFFFF);
          load_coef(it, act[it] & 0xFFFF);
        }
      } else {
        // the single coefficient tile of block it once the MMAs of block
        // it - 1 are done; then the record of block it + 2, whose slot (block
        // it - 1's) is free by the same wait (the prologue loaded records 0
        // to 2 and the coefficients of block 0)
        for (int it = 1; it < nact; ++it) {
          const int b = it - 1;
          if (!mbar_wait(&empty[b % NST], (uint32_t)(b / NST) & 1u, err, 12)) break;
          *(volatile int*)released = it;
          load_coef(it, act[it] & 0xFFFF);
          const int r = it + NST - 1;   // its record slot is block it - 1's
          if (r < nact && r >= tma_pre) load_record(r, act[r] & 0xFFFF);
        }
      }
    }
  } else {
    // ---------------- MMA issuer
    if (lane == 0) {
      const uint32_t idesc = mma_idesc<PIECES>(n_tile);
      bool init[3] = {false, false, false};   // accumulators written so far
      for (int it = 0; it < nact; ++it) {
        const int s = it % NST;
        const uint32_t phase = (uint32_t)(it / NST) & 1u;
        // each k-step's MMAs go out as soon as its four chunks are produced;
        // for a skipped k-step this thread arrives in place of its chunks
        // (it waited for that barrier's phase of the block NST back itself)
        if (!mbar_wait(&bfull[s], phase, err, 13)) break;
        const int kb = act[it] & 0xFFFF;
        uint32_t kmask = (uint32_t)act[it] >> 16;
        if (kmask == 0u) kmask = 0xFu;
        const int li = NACC == 3 ? lead_acc(kb, kblocks) : 0;
        bool ok = true;
        for (int kk = 0; kk < kKsteps; ++kk) {
          const bool kl = ((kmask >> kk) & 1u) != 0u;
          if (!kl) mbar_arrive_n(&full[s * kKsteps + kk], (uint32_t)(kChunks / kKsteps * 32));
          if (!mbar_wait(&full[s * kKsteps + kk], phase, err, 13)) {
            ok = false;
            break;
          }
          if (!kl) continue;
          tc_fence_after();
          mma_kstep<PIECES, NACC>(smem_addr(smem + s * STAGE), (uint32_t)b_off(s), (uint32_t)B_TILE, tmem, n_tile,
                                  idesc, li, kk, init);
        }
        if (!ok) break;
        umma_commit(&empty[s]);
      }
      umma_commit(acc_full);
    }
  }

  if (warp < kProdWarps) {
    // ---------------- epilogue: every producer warp, TMEM lane quadrant warp % 4,
    // a quarter of the 16-column chunks.  When the tile's rows fit in the idle
    // stage memory (and are 16-byte aligned in `out`), they are staged there
    // and each row leaves in one bulk copy (global stores of 256 bytes from
    // every warp ran at ~17 GB/s per SM); otherwise each warp writes its rows
    // through a small staging buffer.
    bool ok = mbar_wait(acc_full, 0, err, 14);
    ok = __all_sync(0xffffffffu, ok && *(volatile int*)err == 0);
    tc_fence_after();
    // the tile goes out in column passes of `pw` columns (a multiple of 16),
    // as few as the idle stage memory allows (one for NACC = 3)
    int npass = 1, pw = n_tile;
    if constexpr (NACC == 2) {
      const int max_pw = ((int)(STAGE_MEM / (BM * sizeof(double))) - 2) / 16 * 16;
      npass = max_pw >= 16 ? (n_tile + max_pw - 1) / max_pw : 0;
      pw = npass > 0 ? ((n_tile + npass - 1) / npass + 15) / 16 * 16 : 0;
    }
    const int ldst = pw + 2;
    const bool bulk = npass > 0 && (size_t)BM * ldst * sizeof(double) <= (size_t)STAGE_MEM && (n_out & 1) == 0 &&
                      (reinterpret_cast<uintptr_t>(out) & 15) == 0;
    if (NACC == 3 && bulk) {
      // one pass: the whole tile fits the idle stage memory
      double* stg = (double*)smem;
      if (ok)
        epilogue_stage_warp<PIECES, COMPS, NACC>(tmem, n_tile, n0, n_out, nact_p[2] >= 0, rexp, scales, stg, ldst,
                                                 warp, lane, warp >> 2, kProdWarps / 4, nact_p[1] >= 0);
      fence_async_smem();
      named_bar_sync(1, kProd);   // all producer warps arrive, whatever their `ok`
      if (ok) {
        const int ncols = min(n_tile, n_out - n0);   // even: n_out even, n0 a multiple of 16
        for (int r = tid; r < PTS * COMPS; r += kProd) {
          const int64_t pq = pidx[r / COMPS];
          if (pq >= 0)
            bulk_store(out + (pq * COMPS + r % COMPS) * n_out + n0, stg + (size_t)r * ldst, (uint32_t)ncols * 8u);
        }
        bulk_commit();
        bulk_wait_read();
      }
    } else if (bulk) {
      double* stg = (double*)smem;
      for (int c_lo = 0; c_lo < n_tile; c_lo += pw) {
        if (c_lo > 0) named_bar_sync(1, kProd);   // the previous pass's rows have left the staging memory
        if (ok)
          epilogue_stage_warp<PIECES, COMPS, NACC>(tmem, n_tile, n0, n_out, nact_p[2] >= 0, rexp, scales, stg, ldst,
                                                   warp, lane, warp >> 2, kProdWarps / 4, nact_p[1] >= 0, c_lo,
                                                   c_lo + pw);
        fence_async_smem();
        named_bar_sync(1, kProd);   // all producer warps arrive, whatever their `ok`
        if (ok) {
          // even: n_out even, n0 and c_lo multiples of 16
          const int ncols = min(min(pw, n_tile - c_lo), n_out - n0 - c_lo);
          if (ncols > 0) {
            for (int r = tid; r < PTS * COMPS; r += kProd) {
              const int64_t pq = pidx[r / COMPS];
              if (pq >= 0)
                bulk_store(out + (pq * COMPS + r % COMPS) * n_out + n0 + c_lo, stg + (size_t)r * ldst,
                           (uint32_t)ncols * 8u);
            }
          }
          bulk_commit();
          bulk_wait_read();
        }
      }
    } else if (ok) {
      epilogue_warp<PIECES, COMPS, NACC>(tmem, n_tile, n0, n_out, nact_p[2] >= 0, pidx, rexp, scales, out,
                                         (double*)smem + warp * 32 * 16, warp, lane, warp >> 2, kProdWarps / 4,
                                         nact_p[1] >= 0);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols));
  }
}

// Tile plan: per tile of PTS points (in the order perm), the coordinates
// gathered in tile order (tpts[tile][3][PTS]) and the K blocks that do not
// vanish over the tile (tinfo[tile][kblocks + 4]: count, first block of each
// half of K, first block, then the list, padded with 0), exactly as the fused
// kernel's own prologue finds them.  One CTA per tile: the warps take K
// blocks, the lanes the block's screening spheres, each tested against the
// tile's points in shared memory (no chains of dependent loads).
template <int PTS>
__global__ void __launch_bounds__(256)
tile_plan_kernel(const int64_t P, const double* __restrict__ coord, const int64_t cstride, const int* __restrict__ perm,
                 const int kblocks, const uint8_t* __restrict__ kskip, double* __restrict__ tpts,
                 int* __restrict__ tinfo, unsigned long long* __restrict__ kstat, const int n_tiles) {
  __shared__ double spts[3 * PTS];
  extern __shared__ int sflag[];   // [kblocks]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t tile = blockIdx.x;
  const int64_t p0 = tile * PTS;
  const int np = (int)(P - p0 < PTS ? P - p0 : PTS);
  for (int t = tid; t < 3 * PTS; t += blockDim.x) {
    const int d = t / PTS, i = t - d * PTS;
    const int64_t q = i < np ? (perm ? (int64_t)perm[p0 + i] : p0 + i) : -1;
    const double v = q >= 0 ? coord[q + d * cstride] : 0.0;
    spts[t] = v;
    tpts[tile * 3 * PTS + t] = v;
  }
  __syncthreads();
  tile_kblock_flags<PTS>(kskip, kblocks, spts, np, sflag, warp, lane, (int)(blockDim.x >> 5), true);
  __syncthreads();
  if (warp != 0) return;
  int* ti = tinfo + tile * (kblocks + 4);
  const int n = tile_kblock_list(sflag, kblocks, ti + 4, ti, lane, true);
  for (int t = n + lane; t < kblocks; t += 32) ti[4 + t] = 0;
  if (kstat != nullptr) {   // counted per CTA of the fused kernel: once per MO tile
    const int ks = tile_kstep_count(sflag, kblocks, lane);
    if (lane == 0) {
      atomicAdd(&kstat[0], (unsigned long long)ks * n_tiles);
      atomicAdd(&kstat[1], (unsigned long long)kblocks * (BK / UMMA_K) * n_tiles);
    }
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

size_t tile_plan_pts_bytes(int64_t tiles, int pts) { return ((size_t)tiles * 3 * pts * sizeof(double) + 255) / 256 * 256; }

template <int PIECES, int COMPS, int NACC, int NST>
size_t fused_smem(int n_tile, int rec_bytes, int kblocks) {
  constexpr int PTS = BM / COMPS;
  const size_t b_tile = (size_t)PIECES * n_tile * BK * 2;
  const size_t stage_mem = NACC == 3 ? NST * ((size_t)PIECES * A_TILE + b_tile) : NST * (size_t)PIECES * A_TILE + b_tile;
  return 1024 + stage_mem + (size_t)NST * rec_bytes + ((kKsteps + 3) * NST + 2) * 8 + 4 * PTS * 8 +
         3 * PTS * 4 +
         (size_t)(2 * kblocks + 6) * 4 + 16;
}

template <int PIECES, int COMPS, int NACC, int NST>
cudaError_t launch_fused(const DevTables& T, const CUtensorMap& tb, int64_t P, const double* coord, double cutoff,
                         int n_out, int n_tile, int n_tiles, int kblocks, const uint8_t* krec, int rec_bytes,
                         const int* perm, const double* scales, const RowBound& rb, double* out, int* err,
                         int64_t cstride, const uint8_t* kskip, unsigned long long* kstat, void* tplan,
                         cudaStream_t s) {
  constexpr int PTS = BM / COMPS;
  const size_t smem = fused_smem<PIECES, COMPS, NACC, NST>(n_tile, rec_bytes, kblocks);
  auto kern = fused_mo_kernel<PIECES, COMPS, NACC, NST>;
  const unsigned int late_ns = g_late_warp_ns.load(std::memory_order_relaxed);
  if constexpr (PIECES == 3 && COMPS == 5)
    if (late_ns != 0u) kern = fused_mo_kernel<PIECES, COMPS, NACC, NST, true>;
  if (NACC == 2 && tplan == nullptr) return cudaErrorInvalidValue;   // the wide form needs a tile plan
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int64_t tiles = (P + PTS - 1) / PTS;
  double* tpts = nullptr;
  int* tinfo = nullptr;
  if (tplan != nullptr) {
    tpts = (double*)tplan;
    tinfo = (int*)((uint8_t*)tplan + tile_plan_pts_bytes(tiles, PTS));
    tile_plan_kernel<PTS><<<(unsigned)tiles, 256, sizeof(int) * (size_t)kblocks, s>>>(
        P, coord, cstride, perm, kblocks, kskip, tpts, tinfo, kstat, n_tiles);
    count_launch();
    kstat = nullptr;   // counted by the plan
  }
  dim3 grid((unsigned)tiles, (unsigned)n_tiles);
  kern<<<grid, kThreadsF, smem, s>>>(T, tb, P, coord, cutoff, n_out, n_tile, kblocks, krec, rec_bytes, perm, scales,
                                     rb, out, err, cstride, kskip, kstat, tpts, tinfo, late_ns);
  count_launch();
  return cudaGetLastError();
}

}  // namespace

size_t tc_fused_smem(const TcPlan& plan, int comps, int rec_bytes) {
  const int kb = (int)((plan.ao_num + BK - 1) / BK);
  const int n = plan.n_tile;
  if (plan.pieces == 3 && plan.nacc == 2 && plan.nst == 3)
    return comps == 5 ? fused_smem<3, 5, 2, 3>(n, rec_bytes, kb) : fused_smem<3, 1, 2, 3>(n, rec_bytes, kb);
  if (plan.pieces == 3 && plan.nacc == 2)
    return comps == 5 ? fused_smem<3, 5, 2, 2>(n, rec_bytes, kb) : fused_smem<3, 1, 2, 2>(n, rec_bytes, kb);
  if (plan.pieces == 3)
    return comps == 5 ? fused_smem<3, 5, 3, 2>(n, rec_bytes, kb) : fused_smem<3, 1, 3, 2>(n, rec_bytes, kb);
  return comps == 5 ? fused_smem<2, 5, 3, 2>(n, rec_bytes, kb) : fused_smem<2, 1, 3, 2>(n, rec_bytes, kb);
}

size_t tc_tile_plan_bytes(const TcPlan& plan, int64_t point_num, int comps) {
  const int pts = BM / comps;
  const int64_t tiles = (point_num + pts - 1) / pts;
  const int kb = (int)((plan.ao_num + BK - 1) / BK);
  return tile_plan_pts_bytes(tiles, pts) + sizeof(int) * (size_t)tiles * (kb + 4);
}

size_t tc_kskip_bytes(int64_t ao_num, int64_t shell_num) {
  const int kb = (int)((ao_num + BK - 1) / BK);
  return (size_t)kskip_kpos_offset(kb, (int)shell_num) + sizeof(int2) * (size_t)shell_num;
}

cudaError_t tc_encode_coef_map(const TcPlan& plan, const void* d_coef, CUtensorMap* map) {
  auto fn = encode_fn();
  if (!fn) return cudaErrorNotSupported;
  cuuint64_t dims[3] = {(cuuint64_t)plan.ao_num, (cuuint64_t)plan.n_pad, (cuuint64_t)plan.pieces};
  cuuint64_t strides[2] = {(cuuint64_t)(plan.k_pad * 2), (cuuint64_t)(plan.n_pad * plan.k_pad * 2)};
  cuuint32_t box[3] = {(cuuint32_t)BK, (cuuint32_t)plan.n_tile, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(d_coef), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t tc_launch_fused(const TcPlan& plan, int64_t point_num, int comps, const double* coord, double cutoff,
                            const CUtensorMap& tb, const void* krec, int rec_bytes, const int* perm, const void* d_coef,
                            const RowBound& rb, double* out, int* err, cudaStream_t s, int64_t cstride,
                            const void* kskip, unsigned long long* kstat, void* tplan) {
  if (point_num <= 0) return cudaSuccess;
  if (cstride < point_num) cstride = point_num;
  if (rec_bytes <= 0 || rec_bytes % 128 != 0) return cudaErrorInvalidValue;
  const DevTables T{};   // the fused kernel reads the records only
  const int kblocks = (int)((plan.ao_num + BK - 1) / BK);
  const uint8_t* kr = (const uint8_t*)krec;
  const int M = (int)plan.mo_num;
  const double* sc = tc_scales(plan, d_coef);
  const uint8_t* ks = (const uint8_t*)kskip;
  auto run = [&](auto launch) {
    return launch(T, tb, point_num, coord, cutoff, M, plan.n_tile, plan.n_tiles, kblocks, kr, rec_bytes, perm, sc, rb,
                  out, err, cstride, ks, kstat, tplan, s);
  };
  if (plan.pieces == 3 && plan.nacc == 2 && plan.nst == 3)
    return comps == 5 ? run(launch_fused<3, 5, 2, 3>) : run(launch_fused<3, 1, 2, 3>);
  if (plan.pieces == 3 && plan.nacc == 2)
    return comps == 5 ? run(launch_fused<3, 5, 2, 2>) : run(launch_fused<3, 1, 2, 2>);
  if (plan.pieces == 3)
    return comps == 5 ? run(launch_fused<3, 5, 3, 2>) : run(launch_fused<3, 1, 3, 2>);
  return comps == 5 ? run(launch_fused<2, 5, 3, 2>) : run(launch_fused<2, 1, 3, 2>);
}

cudaError_t tc_run_fused(const DevTables& T, const TcPlan& plan, int64_t point_num, int comps, const double* coord,
                         double cutoff, const void* d_coef, const void* krec, int rec_bytes, const int* perm,
                         const RowBound& rb, double* out, int* err, cudaStream_t s, int64_t cstride,
                         const void* kskip, unsigned long long* kstat, void* tplan) {
  (void)T;
  if (point_num <= 0) return cudaSuccess;
  if (err == nullptr) return cudaErrorInvalidValue;
  CUtensorMap tb;
  cudaError_t e = tc_encode_coef_map(plan, d_coef, &tb);
  if (e != cudaSuccess) return e;
  // a timed-out barrier wait stays in *err for the caller's next synchronization
  return tc_launch_fused(plan, point_num, comps, coord, cutoff, tb, krec, rec_bytes, perm, d_coef, rb, out, err, s,
                         cstride, kskip, kstat, tplan);
}

cudaError_t tc_set_late_warps(unsigned int ns) {
  g_late_warp_ns.store(ns, std::memory_order_relaxed);
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

__global__ void point_keys_kernel(const double* __restrict__ coord, int64_t P, int64_t cstride, double3 origin,
                                  double inv_cell, int* __restrict__ keys, unsigned int* __restrict__ counts) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < P; p += (int64_t)gridDim.x * blockDim.x) {
    int c[3];
    const double o[3] = {origin.x, origin.y, origin.z};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double v = floor((coord[p + d * cstride] - o[d]) * inv_cell);
      c[d] = (int)fmin(31.0, fmax(0.0, v));
    }
    const int key = (int)(spread5(c[0]) | (spread5(c[1]) << 1) | (spread5(c[2]) << 2));
    keys[p] = key;
    atomicAdd(&counts[key], 1u);
  }
}

// exclusive scan of kSortCells counts in one CTA of 1024 threads: warp w
// scans cells [1024 w, 1024 w + 1024) as 32 rows of 32 (coalesced loads and
// stores, shuffles within a row, a carry from row to row), then the warps'
// totals are scanned and added
__global__ void __launch_bounds__(1024) scan_cells_kernel(unsigned int* counts) {
  static_assert(kSortCells == 32 * 1024, "32 warps x 32 rows x 32 cells");
  __shared__ unsigned int wbase[32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned int* c = counts + warp * 1024;
  unsigned int v[32];
  unsigned int carry = 0u;
#pragma unroll
  for (int i = 0; i < 32; ++i) {
    const unsigned int x = c[32 * i + lane];
    unsigned int y = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned int t = __shfl_up_sync(0xffffffffu, y, o);
      if (lane >= o) y += t;
    }
    v[i] = carry + y - x;
    carry += __shfl_sync(0xffffffffu, y, 31);
  }
  if (lane == 0) wbase[warp] = carry;
  __syncthreads();
  if (warp == 0) {
    const unsigned int x = wbase[lane];
    unsigned int y = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned int t = __shfl_up_sync(0xffffffffu, y, o);
      if (lane >= o) y += t;
    }
    wbase[lane] = y - x;
  }
  __syncthreads();
  const unsigned int base = wbase[warp];
#pragma unroll
  for (int i = 0; i < 32; ++i) c[32 * i + lane] = base + v[i];
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
                        int* keys, unsigned int* counts, int* perm, cudaStream_t s, int64_t cstride) {
  if (cstride < point_num) cstride = point_num;
  // 32 cells per axis over the box of the nuclei (cells at least 1 bohr wide)
  double ext = 0.0;
  for (int d = 0; d < 3; ++d) ext = std::max(ext, box_hi[d] - box_lo[d]);
  const double cell = std::max(1.0, ext / 32.0);
  const double3 origin = make_double3(box_lo[0], box_lo[1], box_lo[2]);
  if (point_num <= 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(counts, 0, sizeof(unsigned int) * kSortCells, s);
  if (e != cudaSuccess) return e;
  const int grid = (int)std::min<int64_t>((point_num + 255) / 256, 148 * 8);
  point_keys_kernel<<<grid, 256, 0, s>>>(coord, point_num, cstride, origin, 1.0 / cell, keys, counts);
  scan_cells_kernel<<<1, 1024, 0, s>>>(counts);
  scatter_points_kernel<<<grid, 256, 0, s>>>(keys, point_num, counts, perm);
  count_launch(3);
  return cudaGetLastError();
}

}  // namespace qb
