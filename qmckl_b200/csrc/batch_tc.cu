// Batched MO VGL (mixed form) of many independent systems in one persistent
// launch, driven by a device work queue.
//
// A batch snapshots N contexts (basis, nuclei, MO coefficients, precision)
// and a point count per system.  Points and results are packed: system s
// reads its [3][P_s] coordinates at d_coord + coord_offset[s] and writes its
// mo_vgl[P_s][5][mo_s] at d_mo_vgl + out_offset[s].
//
// Device work queue.  One CTA per SM loops: one thread takes the next item
// with an atomic increment of the queue head, the CTA runs it, and so on.
//   prep item  (system s): the CTA orders the system's points spatially
//              (counting sort over 16^3 cells of the nuclei's box, in shared
//              memory) into the permutation buffer, then publishes
//              ready[s] with a release store.
//   tile item  (system s, point tile t, MO tile j): 25 points x n_tile MOs of
//              s, through the fused AO -> split-BF16 tcgen05 pipeline of
//              fused_common.cuh.  It first waits (acquire loads, bounded by
//              an iteration cap or 2 s) until ready[s] is set.
// All prep items precede all tile items in the queue, and a prep item never
// waits, so every wait ends.  Pipeline barrier phases run on across items
// (K blocks counted per CTA); TMEM is allocated once per CTA.
// A failed wait sets the error word; every CTA then stops taking items.
//
// Tile shapes come from a small autotuner (qmckl_b200_batch_tune): producer
// warps per CTA (16 warps x 4 AOs or 8 warps x 8 AOs per K block) and the
// queue order (largest work per tile first, system by system, or round
// robin over systems), timed on the batch itself.  The choice can be kept in
// a tuning file named by QMCKL_B200_TUNE_FILE and is applied to batches of
// the same shape.  The launch sequence (queue reset + kernel) is captured in
// a CUDA graph and replayed while the buffers stay the same.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "fused_common.cuh"
#include "internal.h"
#include "mo_tc.cuh"
#include "qmckl_b200.h"

namespace qb {
namespace {

using namespace fz;

constexpr int kStages = 2;
constexpr int kPieces = 3;   // bfloat16 x 3 operands (split.cuh), as the single-system default
constexpr int kCellsAxis = 16;
constexpr int kCells = kCellsAxis * kCellsAxis * kCellsAxis;
constexpr int kPts = BM / 5;   // 25 points per tile (MO VGL)

struct alignas(64) BatchDesc {
  int64_t coord_off;   // element offset of the system's [3][P] coordinates
  int64_t out_off;     // element offset of its [P][5][mo] output
  int64_t perm_off;    // offset of its point order in the permutation buffer
  int64_t P;
  const uint8_t* krec;
  const uint8_t* kskip;   // tile-skipping tables of the K blocks (fused_tc.cu)
  const double* scales;   // scale block of the system's coefficient pieces
  RowBound rb;            // row bounds of the float16 operands
  double cutoff;
  double lo[3];
  double inv_cell;
  int32_t rec_bytes, kblocks, n_out, n_tile;
  int32_t n_tiles, ptiles, pad0, pad1;
};

struct BatchCtl {                 // shared-memory control block of a CTA
  uint64_t full[kStages], empty[kStages], rec_full[kStages], acc_full;
  uint32_t tmem_slot;
  int item[4];
  int ok;
  int claim;   // chunks of the current item claimed by the producer warps after their first
  double pts[3 * kPts];
  int64_t pidx[kPts];
  int rexp[3 * kPts];
  // followed in shared memory by the tile's K blocks, their flags and the
  // counts (batch_smem): int act[kb_max], flag[kb_max], n, lo, hi, first
};

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Wait until *flag != 0: at most `limit` polls when limit > 0, else 2 s.
__device__ bool wait_flag(const int* flag, long long limit, int* err) {
  const uint64_t t0 = globaltimer();
  for (long long i = 0;; ++i) {
    if (ld_acquire(flag) != 0) return true;
    if (*(volatile int*)err != 0) return false;
    if ((limit > 0 && i + 1 >= limit) || (limit <= 0 && globaltimer() - t0 > kWaitNs)) {
      atomicCAS(err, 0, 26);
      return false;
    }
    __nanosleep(128);
  }
}

__device__ __forceinline__ int cell_key(const double* crd, int64_t p, int64_t P, const BatchDesc& D) {
  int c[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double v = floor((crd[p + d * P] - D.lo[d]) * D.inv_cell);
    c[d] = (int)fmin((double)(kCellsAxis - 1), fmax(0.0, v));
  }
  int key = 0;
#pragma unroll
  for (int b = 0; b < 4; ++b)
    key |= (((c[0] >> b) & 1) << (3 * b)) | (((c[1] >> b) & 1) << (3 * b + 1)) | (((c[2] >> b) & 1) << (3 * b + 2));
  return key;
}

// Spatial order of one system's points by a counting sort in shared memory
// (scratch: kCells + nthreads words).  The order inside a cell is arbitrary:
// every output row depends on its own point only.
__device__ void order_system(const BatchDesc& D, const double* coord, int* perm, uint8_t* scratch, int tid,
                             int nthreads) {
  unsigned* cnt = (unsigned*)scratch;
  unsigned* part = cnt + kCells;
  const double* crd = coord + D.coord_off;
  const int64_t P = D.P;
  for (int i = tid; i < kCells; i += nthreads) cnt[i] = 0u;
  __syncthreads();
  for (int64_t p = tid; p < P; p += nthreads) atomicAdd(&cnt[cell_key(crd, p, P, D)], 1u);
  __syncthreads();
  const int per = (kCells + nthreads - 1) / nthreads;
  const int c0 = min(tid * per, kCells), c1 = min(c0 + per, kCells);
  unsigned local = 0u;
  for (int i = c0; i < c1; ++i) local += cnt[i];
  part[tid] = local;
  __syncthreads();
  for (int off = 1; off < nthreads; off <<= 1) {
    const unsigned v = tid >= off ? part[tid - off] : 0u;
    __syncthreads();
    part[tid] += v;
    __syncthreads();
  }
  unsigned run = part[tid] - local;
  for (int i = c0; i < c1; ++i) {
    const unsigned c = cnt[i];
    cnt[i] = run;
    run += c;
  }
  __syncthreads();
  int* pm = perm + D.perm_off;
  for (int64_t p = tid; p < P; p += nthreads) pm[atomicAdd(&cnt[cell_key(crd, p, P, D)], 1u)] = (int)p;
  __syncthreads();
}

template <int PRODW>
__global__ void __launch_bounds__((PRODW + 2) * 32, 1)
batch_mo_kernel(const BatchDesc* __restrict__ desc, const CUtensorMap* __restrict__ tmaps,
                const int4* __restrict__ items, const int n_items, int* __restrict__ ctl_words,
                const double* __restrict__ coord, double* __restrict__ out, int* __restrict__ perm,
                const int n_tile_max, const int rec_max, const int kb_max, const long long wait_limit,
                const int publish) {
  constexpr int COMPS = 5;
  constexpr int PIECES = kPieces;
  constexpr int CHUNK = BK / PRODW;
  constexpr int NPROD = PRODW * 32;
  constexpr int NTHREADS = (PRODW + 2) * 32;
  constexpr int TMA_WARP = PRODW, MMA_WARP = PRODW + 1;
  int* err = ctl_words;           // [0] error word, [1] queue head, [2..] ready flags
  int* head = ctl_words + 1;
  int* ready = ctl_words + 2;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = smem_raw + ((1024u - (smem_addr(smem_raw) & 1023u)) & 1023u);
  const int B_MAX = n_tile_max * BK * 2;
  const int STAGE = PIECES * (A_TILE + B_MAX);
  uint8_t* recs = smem + kStages * STAGE;
  BatchCtl& C = *(BatchCtl*)(recs + kStages * rec_max);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint32_t tmem_cols = 32;
  while ((int)tmem_cols < 3 * n_tile_max) tmem_cols <<= 1;

  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&C.full[s], NPROD + 1);
      mbar_init(&C.empty[s], 1);
      mbar_init(&C.rec_full[s], 1);
    }
    mbar_init(&C.acc_full, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  zero_pad_rows<PIECES, COMPS, kStages>(smem, STAGE, tid, NTHREADS);
  if (warp == MMA_WARP) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&C.tmem_slot)),
                 "r"(tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = C.tmem_slot;

  uint32_t kbase = 0;    // K blocks run by this CTA so far: pipeline stage and phase
  uint32_t ntiles = 0;   // tile items run so far: accumulator phase
  for (;;) {
    if (tid == 0) {
      int4 it = make_int4(-1, 0, 0, 0);
      if (*(volatile int*)err == 0) {
        const int idx = atomicAdd(head, 1);
        if (idx < n_items) it = items[idx];
      }
      C.item[0] = it.x;
      C.item[1] = it.y;
      C.item[2] = it.z;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const int sys = C.item[0], ptile = C.item[1], ntile = C.item[2];
    if (sys < 0) break;
    const BatchDesc& D = desc[sys];
    if (ptile < 0) {
      // ---------------- prep item: point order of the system (stage memory as scratch)
      order_system(D, coord, perm, smem, tid, NTHREADS);
      zero_pad_rows<PIECES, COMPS, kStages>(smem, STAGE, tid, NTHREADS);
      fence_async_smem();
      __syncthreads();
      if (tid == 0) {
        __threadfence();
        if (publish) st_release(&ready[sys], 1);
      }
      continue;
    }
    // ---------------- tile item
    if (tid == 0) C.ok = wait_flag(&ready[sys], wait_limit, err) ? 1 : 0;
    __syncthreads();
    if (!C.ok) continue;
    const int64_t P = D.P;
    const int64_t p0 = (int64_t)ptile * kPts;
    const double* crd = coord + D.coord_off;
    const int* pm = perm + D.perm_off;
    for (int t = tid; t < 3 * kPts; t += NTHREADS) {
      const int d = t / kPts, i = t - d * kPts;
      const int64_t q = (p0 + i < P) ? (int64_t)__ldcg(pm + p0 + i) : -1;
      C.pts[t] = q >= 0 ? crd[q + d * P] : 0.0;
      if (d == 0) C.pidx[i] = q;
      C.rexp[t] = PIECES == 2 ? kExpMin : 0;
    }
    __syncthreads();
    if (PIECES == 2) {
      row_exponents<kPts>(D.rb, C.pts, C.pidx, C.rexp, tid, NTHREADS);
      __syncthreads();
    }
    const int kblocks = D.kblocks, n_tile = D.n_tile, rec_bytes = D.rec_bytes;
    const int n0 = ntile * n_tile;
    const int B_TILE = n_tile * BK * 2;
    // K blocks that are not identically zero over the tile's points (as in
    // the single-system fused kernel, fused_tc.cu)
    int* act = (int*)(&C + 1);
    int* kflag = act + kb_max;
    int* kcnt = kflag + kb_max;
    tile_kblock_flags<kPts>(D.kskip, kblocks, C.pts, (int)(P - p0 < kPts ? P - p0 : kPts), kflag, warp, lane,
                            NTHREADS / 32, true);
    __syncthreads();
    if (warp == 0) tile_kblock_list(kflag, kblocks, act, kcnt, lane, true);
    if (tid == 0) C.claim = 0;
    __syncthreads();
    const int nact = kcnt[0];
    if (warp < PRODW) {
      // the item's PRODW chunks per K block, claimed in order from a shared
      // counter (first: chunk `warp` of the first block), as in the
      // single-system kernel (fused_tc.cu): a warp done early goes on with
      // the next chunks instead of waiting for its block's slowest warp.
      // Every chunk waits for its stage and record and arrives (one barrier
      // per stage, as many chunks as warps), so no wait falls two phases
      // behind.
      const int total = nact * PRODW;
      for (int q = warp; q < total;) {
        const int it = q / PRODW, c = q - it * PRODW;
        const uint32_t g = kbase + (uint32_t)it;
        const int s = (int)(g & 1u);
        const uint32_t phase = (g >> 1) & 1u;
        bool ok = mbar_wait(&C.empty[s], phase ^ 1u, err, 21);
        ok = ok && mbar_wait(&C.rec_full[s], phase, err, 25);
        if (!__all_sync(0xffffffffu, ok)) break;
        if (kstep_live(act[it], c, CHUNK))
          produce_kblock<PIECES, COMPS, CHUNK>(recs + s * rec_max, C.pts, p0, P, D.cutoff, C.rexp,
                                               smem_addr(smem + s * STAGE), c, lane);
        fence_async_smem();
        mbar_arrive(&C.full[s]);
        int nq = 0;
        if (lane == 0) nq = atomicAdd(&C.claim, 1) + PRODW;
        q = __shfl_sync(0xffffffffu, nq, 0);
      }
    } else if (warp == TMA_WARP) {
      if (lane == 0) {
        const CUtensorMap* map = tmaps + sys;
        for (int it = 0; it < nact; ++it) {
          const int kb = act[it] & 0xFFFF;
          const uint32_t g = kbase + (uint32_t)it;
          const int s = (int)(g & 1u);
          const uint32_t phase = (g >> 1) & 1u;
          if (!mbar_wait(&C.empty[s], phase ^ 1u, err, 22)) break;
          mbar_expect_tx(&C.rec_full[s], (uint32_t)rec_bytes);
          bulk_load(recs + s * rec_max, D.krec + (size_t)kb * rec_bytes, (uint32_t)rec_bytes, &C.rec_full[s]);
          uint8_t* st = smem + s * STAGE + PIECES * A_TILE;
          mbar_expect_tx(&C.full[s], (uint32_t)(PIECES * B_TILE));
          for (int q = 0; q < PIECES; ++q) tma_load_3d(st + q * B_TILE, map, &C.full[s], kb * BK, n0, q);
        }
      }
    } else {
      if (lane == 0) {
        const uint32_t idesc = mma_idesc<PIECES>(n_tile);
        bool init[3] = {false, false, false};   // accumulators written in this item
        for (int it = 0; it < nact; ++it) {
          const uint32_t g = kbase + (uint32_t)it;
          const int s = (int)(g & 1u);
          const uint32_t phase = (g >> 1) & 1u;
          if (!mbar_wait(&C.full[s], phase, err, 23)) break;
          tc_fence_after();
          mma_kblock_masked<PIECES>(smem_addr(smem + s * STAGE), (uint32_t)(PIECES * A_TILE), (uint32_t)B_TILE, tmem,
                                    n_tile, idesc, act[it] & 0xFFFF, kblocks, (uint32_t)act[it] >> 16, init);
          umma_commit(&C.empty[s]);
        }
        umma_commit(&C.acc_full);
      }
    }
    if (warp < PRODW) {
      // epilogue: every producer warp, TMEM lane quadrant warp % 4.  The
      // stage memory is idle until the next item: the tile's rows are staged
      // there and each leaves in one bulk copy when they fit and are 16-byte
      // aligned in global memory, else each warp writes its rows through a
      // small staging buffer.  Either staging overwrites the zero rows of
      // the A tiles; those rows only feed accumulator rows that are never
      // stored.
      bool ok = mbar_wait(&C.acc_full, ntiles & 1u, err, 24);
      ok = __all_sync(0xffffffffu, ok && *(volatile int*)err == 0);
      tc_fence_after();
      double* o = out + D.out_off;
      const int ldst = n_tile + 2;
      const bool bulk = (size_t)BM * ldst * sizeof(double) <= (size_t)kStages * STAGE && (D.n_out & 1) == 0 &&
                        (reinterpret_cast<uintptr_t>(o) & 15) == 0;
      if (bulk) {
        double* stg = (double*)smem;
        if (ok)
          epilogue_stage_warp<PIECES, COMPS>(tmem, n_tile, n0, D.n_out, kcnt[2] >= 0, C.rexp, D.scales, stg, ldst,
                                             warp, lane, warp >> 2, PRODW / 4, kcnt[1] >= 0);
        fence_async_smem();
        named_bar_sync(1, NPROD);   // all producer warps arrive, whatever their `ok`
        if (ok) {
          const int ncols = min(n_tile, D.n_out - n0);
          for (int r = tid; r < kPts * COMPS; r += NPROD) {
            const int64_t pq = C.pidx[r / COMPS];
            if (pq >= 0)
              bulk_store(o + (pq * COMPS + r % COMPS) * D.n_out + n0, stg + (size_t)r * ldst, (uint32_t)ncols * 8u);
          }
          bulk_commit();
          bulk_wait_read();
        }
      } else if (ok) {
        epilogue_warp<PIECES, COMPS>(tmem, n_tile, n0, D.n_out, kcnt[2] >= 0, C.pidx, C.rexp, D.scales, o,
                                     (double*)smem + warp * 32 * 16, warp, lane, warp >> 2, PRODW / 4,
                                     kcnt[1] >= 0);
      }
    }
    kbase += (uint32_t)nact;
    ++ntiles;
  }
  tc_fence_before();
  __syncthreads();
  if (tid == 0 && *(volatile int*)err != 0) {
    // after a failure, give copies already issued time to land before exit
    const uint64_t t0 = globaltimer();
    while (globaltimer() - t0 < 20000ull) __nanosleep(1000);
  }
  __syncthreads();
  if (warp == MMA_WARP) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols));
  }
}

size_t batch_smem(int n_tile_max, int rec_max, int kb_max) {
  return 1024 + (size_t)kStages * kPieces * (A_TILE + (size_t)n_tile_max * BK * 2) + (size_t)kStages * rec_max +
         sizeof(BatchCtl) + (size_t)(2 * kb_max + 4) * 4;
}

struct BatchSys {
  int64_t P = 0, A = 0, M = 0;
  TcPlan plan;
  size_t coef_off = 0, krec_off = 0, kskip_off = 0;
  int rec_bytes = 0;
  std::vector<int64_t> ao_perm;   // the AO at each K position of the records
  double cutoff = 0.0;
  double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  int64_t coord_off = 0, out_off = 0, perm_off = 0;
  CUtensorMap map;
  RowBound rb{};
};

struct DBuf {
  void* p = nullptr;
  size_t cap = 0;
};

cudaError_t dalloc(DBuf& b, size_t bytes) {
  if (b.cap >= bytes && b.p) return cudaSuccess;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
  cudaError_t e = cudaMalloc(&b.p, std::max<size_t>(bytes, 256));
  if (e == cudaSuccess) b.cap = std::max<size_t>(bytes, 256);
  return e;
}

}  // namespace

struct Batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::vector<BatchSys> sys;
  int64_t coord_total = 0, out_total = 0, perm_total = 0;
  int n_tile_max = 0, rec_max = 0, kb_max = 0;
  DBuf coef, krec, kskip, desc, tmaps, items, ctl, perm, keys, counts, loop_err, nucl, env;
  int n_items = 0;
  // tuning
  int prod_warps = 16;
  int order = 0;
  uint64_t signature = 0;
  // graph
  bool use_graph = true;
  cudaGraphExec_t exec = nullptr;
  const double* g_coord = nullptr;
  double* g_out = nullptr;
  int g_prod = 0, g_order = -1;
  long long wait_limit = 0;
  int publish = 1;
  int* h_err = nullptr;   // pinned
};

namespace {

constexpr uint64_t kBatchTag = 0xBA7C4B200ull;

struct BatchHandle {
  uint64_t tag;
  Batch* b;
};

Batch* batch_of(qmckl_b200_batch h) {
  BatchHandle* bh = (BatchHandle*)h;
  if (bh == nullptr || bh->tag != kBatchTag) return nullptr;
  return bh->b;
}

// queue: prep items (largest systems first), then the tile items in the
// chosen order
cudaError_t build_items(Batch* B) {
  const int n = (int)B->sys.size();
  std::vector<int> by_cost(n);
  for (int s = 0; s < n; ++s) by_cost[s] = s;
  auto tile_cost = [&](int s) { return (double)B->sys[s].plan.k_pad * (B->sys[s].plan.n_tile + 64); };
  std::stable_sort(by_cost.begin(), by_cost.end(), [&](int a, int b) {
    const double ca = tile_cost(a) * B->sys[a].P, cb = tile_cost(b) * B->sys[b].P;
    return ca > cb;
  });
  std::vector<int4> it;
  for (int s : by_cost)
    if (B->sys[s].P > 0) it.push_back(make_int4(s, -1, 0, 0));
  auto tiles_of = [&](int s, std::vector<int4>& v) {
    const BatchSys& S = B->sys[s];
    const int pt = (int)((S.P + kPts - 1) / kPts);
    for (int t = 0; t < pt; ++t)
      for (int j = 0; j < S.plan.n_tiles; ++j) v.push_back(make_int4(s, t, j, 0));
  };
  if (B->order == 0) {   // largest work per tile first
    std::vector<int> o(n);
    for (int s = 0; s < n; ++s) o[s] = s;
    std::stable_sort(o.begin(), o.end(), [&](int a, int b) { return tile_cost(a) > tile_cost(b); });
    for (int s : o) tiles_of(s, it);
  } else if (B->order == 1) {   // system by system, largest systems first
    for (int s : by_cost) tiles_of(s, it);
  } else {   // round robin over the systems
    std::vector<std::vector<int4>> per(n);
    size_t longest = 0;
    for (int s = 0; s < n; ++s) {
      tiles_of(s, per[s]);
      longest = std::max(longest, per[s].size());
    }
    for (size_t k = 0; k < longest; ++k)
      for (int s : by_cost)
        if (k < per[s].size()) it.push_back(per[s][k]);
  }
  B->n_items = (int)it.size();
  cudaError_t e = dalloc(B->items, sizeof(int4) * std::max<size_t>(it.size(), 1));
  if (e != cudaSuccess) return e;
  if (!it.empty()) e = cudaMemcpy(B->items.p, it.data(), sizeof(int4) * it.size(), cudaMemcpyHostToDevice);
  return e;
}

cudaError_t set_kernel_attrs(Batch* B) {
  const size_t smem = batch_smem(B->n_tile_max, B->rec_max, B->kb_max);
  cudaError_t e = cudaFuncSetAttribute(batch_mo_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(batch_mo_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  return e;
}

cudaError_t enqueue(Batch* B, const double* coord, double* out) {
  const size_t smem = batch_smem(B->n_tile_max, B->rec_max, B->kb_max);
  cudaError_t e = cudaMemsetAsync(B->ctl.p, 0, sizeof(int) * (2 + B->sys.size()), B->stream);
  if (e != cudaSuccess) return e;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, B->device);
  const int grid = std::max(1, std::min(sms, B->n_items));
  if (B->prod_warps == 8)
    batch_mo_kernel<8><<<grid, 10 * 32, smem, B->stream>>>(
        (const BatchDesc*)B->desc.p, (const CUtensorMap*)B->tmaps.p, (const int4*)B->items.p, B->n_items,
        (int*)B->ctl.p, coord, out, (int*)B->perm.p, B->n_tile_max, B->rec_max, B->kb_max, B->wait_limit,
        B->publish);
  else
    batch_mo_kernel<16><<<grid, 18 * 32, smem, B->stream>>>(
        (const BatchDesc*)B->desc.p, (const CUtensorMap*)B->tmaps.p, (const int4*)B->items.p, B->n_items,
        (int*)B->ctl.p, coord, out, (int*)B->perm.p, B->n_tile_max, B->rec_max, B->kb_max, B->wait_limit,
        B->publish);
  return cudaGetLastError();
}

void drop_graph(Batch* B) {
  if (B->exec) cudaGraphExecDestroy(B->exec);
  B->exec = nullptr;
}

cudaError_t run(Batch* B, const double* coord, double* out) {
  if (B->n_items == 0) return cudaSuccess;
  if (!B->use_graph || B->stream == nullptr) {
    count_launch();
    return enqueue(B, coord, out);
  }
  if (!B->exec || B->g_coord != coord || B->g_out != out || B->g_prod != B->prod_warps || B->g_order != B->order) {
    drop_graph(B);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    cudaError_t e1 = enqueue(B, coord, out);
    e = cudaStreamEndCapture(B->stream, &g);
    if (e1 != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return e1;
    }
    if (e != cudaSuccess) return e;
    e = cudaGraphInstantiate(&B->exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      B->exec = nullptr;
      return e;
    }
    B->g_coord = coord;
    B->g_out = out;
    B->g_prod = B->prod_warps;
    B->g_order = B->order;
  }
  count_launch();   // the kernel of the replayed graph
  return cudaGraphLaunch(B->exec, B->stream);
}

uint64_t fnv(uint64_t h, int64_t v) {
  for (int i = 0; i < 8; ++i) {
    h ^= (uint64_t)((v >> (8 * i)) & 0xFF);
    h *= 1099511628211ull;
  }
  return h;
}

void load_tuning(Batch* B) {
  const char* f = std::getenv("QMCKL_B200_TUNE_FILE");
  if (!f) return;
  FILE* fp = std::fopen(f, "r");
  if (!fp) return;
  char line[256];
  while (std::fgets(line, sizeof line, fp)) {
    unsigned long long sig = 0;
    int pw = 0, ord = 0;
    if (std::sscanf(line, "batch %llx %d %d", &sig, &pw, &ord) == 3 && sig == B->signature &&
        (pw == 8 || pw == 16) && ord >= 0 && ord <= 2) {
      B->prod_warps = pw;
      B->order = ord;
    }
  }
  std::fclose(fp);
}

qmckl_exit_code fail(qmckl_context ctx0, const char* fname, const char* msg) {
  return qmckl_failwith(ctx0, QMCKL_FAILURE, fname, msg);
}

}  // namespace
}  // namespace qb

using namespace qb;

extern "C" {

qmckl_exit_code qmckl_b200_batch_create(const qmckl_context* contexts, const int64_t* point_num, const int64_t num,
                                        qmckl_b200_batch* batch) {
  const char* fname = "qmckl_b200_batch_create";
  if (batch == nullptr) return QMCKL_INVALID_ARG_4;
  *batch = 0;
  if (contexts == nullptr || num <= 0) return QMCKL_INVALID_ARG_1;
  if (point_num == nullptr) return QMCKL_INVALID_ARG_2;
  const qmckl_context c0 = contexts[0];
  for (int64_t s = 0; s < num; ++s) {
    if (qmckl_context_check(contexts[s]) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
    const Context* ctx = ctx_of(contexts[s]);
    if (!ctx->ao_basis.provided || !ctx->mo_basis.provided)
      return qmckl_failwith(c0, QMCKL_NOT_PROVIDED, fname, "a context has no AO or MO basis");
    if (ctx->ao_basis.type != 'G') return fail(c0, fname, "only Gaussian basis sets are implemented");
    if (point_num[s] < 0) return qmckl_failwith(c0, QMCKL_INVALID_ARG_2, fname, "negative point count");
    if (!ctx->mo_basis.r_cusp.empty())
      return qmckl_failwith(c0, QMCKL_INVALID_ARG_1, fname, "cusp-adjusted MOs (r_cusp set) are not batched");
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(c0, fname, "no CUDA device: qmckl_b200 computes on the GPU only");
  }
  Batch* B = new Batch();
  cudaGetDevice(&B->device);
  auto bail = [&](const char* msg) {
    qmckl_b200_batch h = (qmckl_b200_batch)(new BatchHandle{kBatchTag, B});
    qmckl_b200_batch_destroy(h);
    return fail(c0, fname, msg);
  };
  B->sys.resize((size_t)num);
  size_t coef_total = 0, krec_total = 0, nucl_total = 0, env_total = 0, kskip_total = 0;
  std::vector<std::vector<uint8_t>> recs((size_t)num), kskips((size_t)num);
  std::vector<std::vector<float>> envs((size_t)num);
  std::vector<float> env_r0((size_t)num), env_il((size_t)num);
  std::vector<size_t> nucl_off((size_t)num), env_off((size_t)num);
  uint64_t sig = 1469598103934665603ull;
  sig = fnv(sig, num);
  // the kernel's shared memory follows the largest MO tile and K-block count
  // of the batch: known before the records are built, so that each system's
  // records can take what is left
  for (int64_t s = 0; s < num; ++s) {
    const Context* ctx = ctx_of(contexts[s]);
    const TcPlan pl = tc_plan(ctx->ao_basis.ao_num, ctx->mo_basis.mo_num, kPieces);
    B->n_tile_max = std::max(B->n_tile_max, pl.n_tile);
    B->kb_max = std::max(B->kb_max, (int)((ctx->ao_basis.ao_num + BK - 1) / BK));
  }
  size_t max_rec = 128;
  while (batch_smem(B->n_tile_max, (int)max_rec + 128, B->kb_max) <= 232448) max_rec += 128;
  for (int64_t s = 0; s < num; ++s) {
    const Context* ctx = ctx_of(contexts[s]);
    BatchSys& S = B->sys[s];
    S.P = point_num[s];
    S.A = ctx->ao_basis.ao_num;
    S.M = ctx->mo_basis.mo_num;
    S.plan = tc_plan(S.A, S.M, kPieces);
    S.cutoff = std::log((double)(((uint64_t)1) << (ctx->precision - 1)));
    if (!build_fused_records(ctx, S.cutoff, max_rec, recs[s], S.rec_bytes, kskips[s], S.ao_perm))
      return bail("AOs are not numbered shell by shell");
    build_envelopes(ctx, envs[s], env_r0[s], env_il[s]);
    nucl_off[s] = nucl_total;
    nucl_total += 3 * (size_t)ctx->nucleus.num;
    env_off[s] = env_total;
    env_total += envs[s].size();
    const int64_t N = ctx->nucleus.num;
    for (int d = 0; d < 3; ++d) {
      S.lo[d] = 1e300;
      S.hi[d] = -1e300;
      for (int64_t n = 0; n < N; ++n) {
        S.lo[d] = std::min(S.lo[d], ctx->nucleus.coord[n + d * N] - 4.0);
        S.hi[d] = std::max(S.hi[d], ctx->nucleus.coord[n + d * N] + 4.0);
      }
    }
    S.coef_off = coef_total;
    coef_total += (S.plan.coef_bytes + 1023) / 1024 * 1024;
    S.krec_off = krec_total;
    krec_total += recs[s].size();
    S.kskip_off = kskip_total;
    kskip_total += (kskips[s].size() + 255) / 256 * 256;
    S.coord_off = B->coord_total;
    B->coord_total += 3 * S.P;
    S.out_off = B->out_total;
    B->out_total += 5 * S.P * S.M;
    S.perm_off = B->perm_total;
    B->perm_total += S.P;
    B->n_tile_max = std::max(B->n_tile_max, S.plan.n_tile);
    B->rec_max = std::max(B->rec_max, S.rec_bytes);
    sig = fnv(fnv(fnv(sig, S.P), S.A), S.M);
  }
  B->signature = sig;
  if (batch_smem(B->n_tile_max, B->rec_max, B->kb_max) > 232448) return bail("basis too large for the batched kernel");
  if (dalloc(B->coef, coef_total) != cudaSuccess || dalloc(B->krec, krec_total) != cudaSuccess ||
      dalloc(B->kskip, std::max<size_t>(kskip_total, 256)) != cudaSuccess ||
      dalloc(B->desc, sizeof(BatchDesc) * num) != cudaSuccess ||
      dalloc(B->tmaps, sizeof(CUtensorMap) * num) != cudaSuccess ||
      dalloc(B->ctl, sizeof(int) * (2 + num)) != cudaSuccess ||
      dalloc(B->perm, sizeof(int) * std::max<int64_t>(B->perm_total, 1)) != cudaSuccess ||
      dalloc(B->nucl, sizeof(double) * std::max<size_t>(nucl_total, 1)) != cudaSuccess ||
      dalloc(B->env, sizeof(float) * std::max<size_t>(env_total, 1)) != cudaSuccess ||
      cudaMallocHost(&B->h_err, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    return bail("device allocation failed");
  }
  if (cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking) != cudaSuccess) return bail("stream creation failed");
  B->own_stream = true;
  std::vector<BatchDesc> hd((size_t)num);
  std::vector<CUtensorMap> hm((size_t)num);
  for (int64_t s = 0; s < num; ++s) {
    const Context* ctx = ctx_of(contexts[s]);
    BatchSys& S = B->sys[s];
    void* dcoef = (char*)B->coef.p + S.coef_off;
    {
      // coefficient columns in the K order of the records
      std::vector<double> cp((size_t)(S.M * S.A));
      const std::vector<double>& c = ctx->mo_basis.coefficient;
      for (int64_t i = 0; i < S.M; ++i)
        for (int64_t k = 0; k < S.A; ++k) cp[i * S.A + k] = c[i * S.A + S.ao_perm[k]];
      if (tc_prepare_coef(S.plan, cp.data(), dcoef, B->stream) != cudaSuccess) return bail("coefficient upload failed");
    }
    if (cudaMemcpyAsync((char*)B->kskip.p + S.kskip_off, kskips[s].data(), kskips[s].size(), cudaMemcpyHostToDevice,
                        B->stream) != cudaSuccess)
      return bail("record upload failed");
    double* dn = (double*)B->nucl.p + nucl_off[s];
    float* de = (float*)B->env.p + env_off[s];
    if (cudaMemcpyAsync(dn, ctx->nucleus.coord.data(), sizeof(double) * 3 * ctx->nucleus.num, cudaMemcpyHostToDevice,
                        B->stream) != cudaSuccess ||
        (!envs[s].empty() && cudaMemcpyAsync(de, envs[s].data(), sizeof(float) * envs[s].size(),
                                             cudaMemcpyHostToDevice, B->stream) != cudaSuccess))
      return bail("nuclear data upload failed");
    if (tc_encode_coef_map(S.plan, dcoef, &S.map) != cudaSuccess) return bail("tensor map encoding failed");
    hm[s] = S.map;
    if (!recs[s].empty() &&
        cudaMemcpyAsync((char*)B->krec.p + S.krec_off, recs[s].data(), recs[s].size(), cudaMemcpyHostToDevice,
                        B->stream) != cudaSuccess)
      return bail("record upload failed");
    BatchDesc& D = hd[s];
    std::memset(&D, 0, sizeof D);
    D.coord_off = S.coord_off;
    D.out_off = S.out_off;
    D.perm_off = S.perm_off;
    D.P = S.P;
    D.krec = (const uint8_t*)B->krec.p + S.krec_off;
    D.kskip = (const uint8_t*)B->kskip.p + S.kskip_off;
    D.scales = tc_scales(S.plan, dcoef);
    D.rb = RowBound{dn, de, (int)ctx->nucleus.num, env_r0[s], env_il[s]};
    S.rb = D.rb;
    D.cutoff = S.cutoff;
    double ext = 0.0;
    for (int d = 0; d < 3; ++d) {
      D.lo[d] = S.lo[d];
      ext = std::max(ext, S.hi[d] - S.lo[d]);
    }
    D.inv_cell = 1.0 / std::max(1.0, ext / kCellsAxis);
    D.rec_bytes = S.rec_bytes;
    D.kblocks = (int)((S.A + BK - 1) / BK);
    D.n_out = (int)S.M;
    D.n_tile = S.plan.n_tile;
    D.n_tiles = S.plan.n_tiles;
    D.ptiles = (int)((S.P + kPts - 1) / kPts);
  }
  if (cudaMemcpyAsync(B->desc.p, hd.data(), sizeof(BatchDesc) * num, cudaMemcpyHostToDevice, B->stream) != cudaSuccess ||
      cudaMemcpyAsync(B->tmaps.p, hm.data(), sizeof(CUtensorMap) * num, cudaMemcpyHostToDevice, B->stream) != cudaSuccess ||
      cudaStreamSynchronize(B->stream) != cudaSuccess)
    return bail("descriptor upload failed");
  load_tuning(B);
  if (build_items(B) != cudaSuccess || set_kernel_attrs(B) != cudaSuccess) return bail("work queue setup failed");
  *batch = (qmckl_b200_batch)(new BatchHandle{kBatchTag, B});
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_b200_batch_destroy(qmckl_b200_batch batch) {
  Batch* B = batch_of(batch);
  if (!B) return QMCKL_INVALID_ARG_1;
  cudaSetDevice(B->device);
  if (B->stream) cudaStreamSynchronize(B->stream);
  drop_graph(B);
  for (DBuf* b : {&B->coef, &B->krec, &B->kskip, &B->desc, &B->tmaps, &B->items, &B->ctl, &B->perm, &B->keys, &B->counts,
                  &B->loop_err, &B->nucl, &B->env})
    if (b->p) cudaFree(b->p);
  if (B->h_err) cudaFreeHost(B->h_err);
  if (B->own_stream && B->stream) cudaStreamDestroy(B->stream);
  delete B;
  BatchHandle* bh = (BatchHandle*)batch;
  bh->tag = 0;
  delete bh;
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_b200_batch_layout(qmckl_b200_batch batch, int64_t* coord_offset, int64_t* out_offset,
                                        int64_t* totals) {
  Batch* B = batch_of(batch);
  if (!B) return QMCKL_INVALID_ARG_1;
  for (size_t s = 0; s < B->sys.size(); ++s) {
    if (coord_offset) coord_offset[s] = B->sys[s].coord_off;
    if (out_offset) out_offset[s] = B->sys[s].out_off;
  }
  if (totals) {
    totals[0] = B->coord_total;
    totals[1] = B->out_total;
  }
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_b200_batch_set_stream(qmckl_b200_batch batch, void* stream) {
  Batch* B = batch_of(batch);
  if (!B) return QMCKL_INVALID_ARG_1;
  cudaSetDevice(B->device);
  drop_graph(B);
  if (B->own_stream && B->stream) {
    cudaStreamSynchronize(B->stream);
    cudaStreamDestroy(B->stream);
  }
  B->stream = (cudaStream_t)stream;
  B->own_stream = false;
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_b200_batch_set_graph(qmckl_b200_batch batch, const int32_t enable) {
  Batch* B = batch_of(batch);
  if (!B) return QMCKL_INVALID_ARG_1;
  B->use_graph = enable != 0;
  if (!B->use_graph) drop_graph(B);
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_b200_batch_set_tuning(qmckl_b200_batch batch, const int32_t producer_warps, const int32_t order) {
  Batch* B = batch_of(batch);
  if (!B) return QMCKL_INVALID_ARG_1;
  if (producer_warps != 8 && producer_warps != 16) return QMCKL_INVALID_ARG_2;
  if (order < 0 || order > 2) return QMCKL_INVALID_ARG_3;
  cudaSetDevice(B->device);
  B->prod_warps = producer_warps;
  if (B->order != order) {
    B->order = order;
    if (B->stream) cudaStreamSynchronize(B->stream);
    if (build_items(B) != cudaSuccess) return QMCKL_FAILURE;
  }
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_b200_batch_get_tuning(qmckl_b200_batch batch, int32_t* producer_warps, int32_t* order) {
  Batch* B = batch_of(batch);
  if (!B) return QMCKL_INVALID_ARG_1;
  if (producer_warps) *producer_warps = B->prod_warps;
  if (order) *order = B->order;
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_b200_batch_set_wait_limit(qmckl_b200_batch batch, const int64_t polls, const int32_t publish) {
  Batch* B = batch_of(batch);
  if (!B) return QMCKL_INVALID_ARG_1;
  B->wait_limit = (long long)polls;
  B->publish = publish != 0;
  drop_graph(B);
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_b200_batch_mo_vgl_device(qmckl_b200_batch batch, const double* d_coord, double* d_mo_vgl) {
  Batch* B = batch_of(batch);
  if (!B) return QMCKL_INVALID_ARG_1;
  if (B->coord_total > 0 && d_coord == nullptr) return QMCKL_INVALID_ARG_2;
  if (B->out_total > 0 && d_mo_vgl == nullptr) return QMCKL_INVALID_ARG_3;
  cudaSetDevice(B->device);
  cudaError_t e = run(B, d_coord, d_mo_vgl);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return QMCKL_FAILURE;
  }
  return QMCKL_SUCCESS;
}

// The same evaluation as a per-system loop of the single-system kernels
// (point order + fused kernel per system), for comparison.
qmckl_exit_code qmckl_b200_batch_mo_vgl_loop_device(qmckl_b200_batch batch, const double* d_coord,
                                                    double* d_mo_vgl) {
  Batch* B = batch_of(batch);
  if (!B) return QMCKL_INVALID_ARG_1;
  cudaSetDevice(B->device);
  int64_t pmax = 0;
  for (auto& S : B->sys) pmax = std::max(pmax, S.P);
  if (dalloc(B->keys, sizeof(int) * std::max<int64_t>(pmax, 1)) != cudaSuccess ||
      dalloc(B->counts, sizeof(unsigned) * (kSortCells + 1)) != cudaSuccess ||
      dalloc(B->loop_err, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    return QMCKL_ALLOCATION_FAILED;
  }
  cudaError_t e = cudaMemsetAsync(B->loop_err.p, 0, sizeof(int), B->stream);
  for (auto& S : B->sys) {
    if (e != cudaSuccess) break;
    if (S.P == 0) continue;
    const double* c = d_coord + S.coord_off;
    int* pm = (int*)B->perm.p + S.perm_off;
    e = point_order(c, S.P, S.lo, S.hi, (int*)B->keys.p, (unsigned*)B->counts.p, pm, B->stream);
    if (e == cudaSuccess)
      e = tc_launch_fused(S.plan, S.P, 5, c, S.cutoff, S.map, (const char*)B->krec.p + S.krec_off, S.rec_bytes, pm,
                          (const char*)B->coef.p + S.coef_off, S.rb, d_mo_vgl + S.out_off, (int*)B->loop_err.p,
                          B->stream, -1, (const char*)B->kskip.p + S.kskip_off);
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(B->h_err, B->loop_err.p, sizeof(int), cudaMemcpyDeviceToHost, B->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(B->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return QMCKL_FAILURE;
  }
  return *B->h_err == 0 ? QMCKL_SUCCESS : QMCKL_FAILURE;
}

// Waits for the batch's stream and reports a failed wait in the last
// persistent launch (error word != 0) as QMCKL_FAILURE.
qmckl_exit_code qmckl_b200_batch_synchronize(qmckl_b200_batch batch, int32_t* status) {
  Batch* B = batch_of(batch);
  if (!B) return QMCKL_INVALID_ARG_1;
  cudaSetDevice(B->device);
  cudaError_t e = cudaMemcpyAsync(B->h_err, B->ctl.p, sizeof(int), cudaMemcpyDeviceToHost, B->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(B->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return QMCKL_FAILURE;
  }
  if (status) *status = *B->h_err;
  return *B->h_err == 0 ? QMCKL_SUCCESS : QMCKL_FAILURE;
}

// Autotuner: times every (producer warps, queue order) candidate on the
// batch itself (`reps` launches each after one warm-up) and keeps the
// fastest; appends the choice to QMCKL_B200_TUNE_FILE when set.
qmckl_exit_code qmckl_b200_batch_tune(qmckl_b200_batch batch, const double* d_coord, double* d_mo_vgl,
                                      const int32_t reps, double* best_ms) {
  Batch* B = batch_of(batch);
  if (!B) return QMCKL_INVALID_ARG_1;
  if (reps <= 0) return QMCKL_INVALID_ARG_4;
  cudaSetDevice(B->device);
  const bool graph = B->use_graph;
  B->use_graph = false;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  int bp = B->prod_warps, bo = B->order;
  qmckl_exit_code rc = QMCKL_SUCCESS;
  for (int pw : {16, 8}) {
    for (int ord = 0; ord <= 2 && rc == QMCKL_SUCCESS; ++ord) {
      rc = qmckl_b200_batch_set_tuning(batch, pw, ord);
      if (rc != QMCKL_SUCCESS) break;
      if (run(B, d_coord, d_mo_vgl) != cudaSuccess) { rc = QMCKL_FAILURE; break; }
      cudaEventRecord(e0, B->stream);
      for (int r = 0; r < reps; ++r) run(B, d_coord, d_mo_vgl);
      cudaEventRecord(e1, B->stream);
      if (cudaEventSynchronize(e1) != cudaSuccess) { rc = QMCKL_FAILURE; break; }
      if (qmckl_b200_batch_synchronize(batch, nullptr) != QMCKL_SUCCESS) { rc = QMCKL_FAILURE; break; }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      ms /= (float)reps;
      if (ms < best) {
        best = ms;
        bp = pw;
        bo = ord;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  B->use_graph = graph;
  if (rc != QMCKL_SUCCESS) {
    cudaGetLastError();
    return rc;
  }
  rc = qmckl_b200_batch_set_tuning(batch, bp, bo);
  if (best_ms) *best_ms = best;
  const char* f = std::getenv("QMCKL_B200_TUNE_FILE");
  if (f && rc == QMCKL_SUCCESS) {
    FILE* fp = std::fopen(f, "a");
    if (fp) {
      std::fprintf(fp, "batch %llx %d %d %.4f\n", (unsigned long long)B->signature, bp, bo, best);
      std::fclose(fp);
    }
  }
  return rc;
}

}  // extern "C"
