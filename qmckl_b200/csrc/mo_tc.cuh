// Mixed-precision MO contraction on tcgen05 tensor cores (mo_tc.cu).
//
// A (the AO matrix, rows = (point, component), columns = AOs) and C (the MO
// coefficients) are split into `pieces` bfloat16 matrices whose sum is the
// FP32 value; the products of total order < pieces are accumulated in FP32 in
// tensor memory (pieces = 2: hi*hi + hi*lo + lo*hi; pieces = 3: the six
// products of order <= 2).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "fused_common.cuh"
#include "kernels.cuh"

namespace qb {

struct TcPlan {
  int64_t ao_num = 0, mo_num = 0;
  int pieces = 3;
  int64_t k_pad = 0;     // AO count padded to the K block (64)
  int64_t n_pad = 0;     // MO count padded to a multiple of 16 (one tile <= 256)
  int n_tiles = 0;       // number of N tiles of n_tile columns
  int n_tile = 0;
  size_t scale_off = 0;  // byte offset of the scale block (split.cuh) after the pieces
  size_t coef_bytes = 0; // pieces * n_pad * k_pad 16-bit values + the scale block
  int nacc = 3;          // fused kernel: 3 accumulators (n_tile <= 160) or 2 (wide tiles, n_tile <= 256)
  int nst = 2;           // fused kernel: stages of the A tiles (3 for wide tiles when they fit)
};

// Device pointer to the scale block of a plan's coefficient buffer.
inline const double* tc_scales(const TcPlan& plan, const void* d_coef) {
  return (const double*)((const char*)d_coef + plan.scale_off);
}

TcPlan tc_plan(int64_t ao_num, int64_t mo_num, int pieces);
// The fused kernel's plan (3 pieces): tiles of up to 256 MOs with two
// accumulators when they take fewer MO tiles than tc_plan's, or as many with
// three A stages (up to 176 MOs a tile); tc_plan's otherwise
// (QMCKL_B200_WIDE_TILES=0: never; =1: whenever they fit).
TcPlan tc_plan_fused(int64_t ao_num, int64_t mo_num, int pieces);
size_t tc_a_bytes(const TcPlan& plan, int64_t rows);
// coefficient [mo][ao] (host, FP64) -> split pieces and the scale block on
// the device (per-MO scales for 2 pieces).
cudaError_t tc_prepare_coef(const TcPlan& plan, const double* coefficient_host, void* d_coef, cudaStream_t s);
// Envelopes of the row bounds (fused_common.cuh RowBound) for one nucleus:
// env[3][kEnvCells] <- suffix maxima over the radial cells of upper bounds
// of |AO|, |grad AO| and |lap AO| over the nucleus's shells (shells: l, AO
// factor bound, primitive exponents / coefficients; AOs vanish beyond r_max).
struct ShellBound {
  int l;
  double factor;
  const double* expo;
  const double* coef;
  int nprim;
};
void tc_envelope(const ShellBound* shells, int nshell, double r_max, float r0, float inv_log2q, float* env);
// AO (mixed) -> A pieces -> tensor-core GEMM -> out[(point*comps + c)][mo] FP64
// `tiles` selects the tiled AO kernel (ao_tile.cu) for the pieces when given;
// cusp_r ([nucl], optional) leaves out the AOs of the cusp adjustment
// (kernels.cuh cusp_masked; the untiled producer is used then).
// err: a device word that a bounded barrier wait of the GEMM sets when it
// gives up; it is left on the device for the caller to read at its next
// synchronization point (the call itself does not synchronize).
struct AoTiles;
cudaError_t tc_run(const DevTables& T, const TcPlan& plan, int64_t point_num, int comps, const double* coord,
                   double cutoff, const void* d_coef, void* d_a, double* out, int* err, cudaStream_t s,
                   const AoTiles* tiles = nullptr, const double* cusp_r = nullptr);

// Fused form of tc_run: the AO pieces are produced in shared memory by the
// GEMM kernel itself and never written to device memory (fused_tc.cu).
// krec: one record of rec_bytes per 64-AO K block (see fused_tc.cu); perm
// (optional): order in which the points are grouped into tiles.
// rb: the per-row scale bounds of 2-piece float16 operands (fused_common.cuh).
// kskip (optional): the tile-skipping tables of the K blocks (fused_tc.cu),
// tc_kskip_bytes long; kstat (optional): two device counters to which every
// tile adds the 16-AO k-steps its MMAs issue and the dense count.  tplan (optional,
// tc_tile_plan_bytes of scratch): a small kernel first gathers each tile's
// coordinates and finds its K blocks, so that the fused kernel's CTAs start
// on their pipeline at once (the same blocks, the same results).
cudaError_t tc_run_fused(const DevTables& T, const TcPlan& plan, int64_t point_num, int comps, const double* coord,
                         double cutoff, const void* d_coef, const void* krec, int rec_bytes, const int* perm,
                         const fz::RowBound& rb, double* out, int* err, cudaStream_t s, int64_t cstride = -1,
                         const void* kskip = nullptr, unsigned long long* kstat = nullptr, void* tplan = nullptr);
size_t tc_kskip_bytes(int64_t ao_num, int64_t shell_num);
size_t tc_tile_plan_bytes(const TcPlan& plan, int64_t point_num, int comps);
// TMA map of a plan's coefficient pieces (box: 64 AOs x n_tile MOs x 1 piece,
// 128B swizzle) and a launch of the fused kernel that does not wait for it
// (err: device error word, left for the caller to check).
cudaError_t tc_encode_coef_map(const TcPlan& plan, const void* d_coef, CUtensorMap* map);
cudaError_t tc_launch_fused(const TcPlan& plan, int64_t point_num, int comps, const double* coord, double cutoff,
                            const CUtensorMap& map, const void* krec, int rec_bytes, const int* perm, const void* d_coef,
                            const fz::RowBound& rb, double* out, int* err, cudaStream_t s, int64_t cstride = -1,
                            const void* kskip = nullptr, unsigned long long* kstat = nullptr, void* tplan = nullptr);
// Test hook of the fused kernel (3 pieces, VGL), for the launches that follow
// in this process: producer warps holding a chunk of a skipped k-step sleep
// `ns` nanoseconds before their stage wait (0: off, the kernel without it).
cudaError_t tc_set_late_warps(unsigned int ns);
// Spatial order of points (32^3 cells over [box_lo, box_hi], Morton order) by
// a counting sort: perm[P]; keys[P] and counts[kSortCells + 1] are scratch.
// cstride: distance between the x, y and z blocks of coord (default
// point_num; larger for a slice of a bigger [3][N] array).  The fused
// kernels take the same stride.
constexpr int kSortCells = 1 << 15;
cudaError_t point_order(const double* coord, int64_t point_num, const double* box_lo, const double* box_hi,
                        int* keys, unsigned int* counts, int* perm, cudaStream_t s, int64_t cstride = -1);
// dynamic shared memory of the fused kernel (must stay <= 227 KB)
size_t tc_fused_smem(const TcPlan& plan, int comps, int rec_bytes);

// Same evaluation with caller-provided scratch: the A pieces in d_a.  Makes
// no device allocation.
cudaError_t tc_run_scratch(const DevTables& T, const TcPlan& plan, int64_t point_num, int comps,
                           const double* coord, double cutoff, const void* d_coef, void* d_a, int* d_err,
                           double* out, cudaStream_t s, const double* cusp_r = nullptr);

// Contractions of the mixed-form adjoint on the tensor cores (3 bfloat16
// pieces, FP32 accumulation in TMEM, FP64 results).  Piece buffers are
// [3][rows][ld] 16-bit values (ld and pstride multiples of 8, 16-byte
// aligned base); columns beyond the logical width read as zero.
//   tc_split_rows : FP64 x[rows][cols] (pitch ldx) -> pieces [3][rows][ldp]
//   tc_gemm_tn_split : part[z][a][b] = sum over the rows of K slice z of
//                   X[r][a] Y[r][b], z < tc_tn_splits(rows, kps); slices of
//                   kps * 32 rows (the caller sums the partials)
//   tc_gemm_nt    : out[r][j] (FP32, pitch ldo) = sum_k X[r][k] Y[j][k]
// err: a device error word set by a timed-out barrier wait.
cudaError_t tc_split_rows(const double* x, int64_t rows, int cols, int64_t ldx, void* pieces, int ldp,
                          int64_t pstride, cudaStream_t s);
int tc_tn_splits(int64_t rows, int kps);
cudaError_t tc_gemm_tn_split(const void* x, int64_t ldx, int64_t x_pstride, int64_t a_num, const void* y, int64_t ldy,
                             int64_t y_pstride, int b_num, int64_t rows, int kps, double* part, int* err,
                             cudaStream_t s);
cudaError_t tc_gemm_nt(const void* x, int64_t ldx, int64_t x_pstride, int64_t rows, int64_t k, const void* y,
                       int64_t ldy, int64_t y_pstride, int64_t n, float* out, int64_t ldo, int* err, cudaStream_t s);

// What the fixed-scratch entry point needs from a context whose basis and
// coefficient pieces are already on the device (device.cu).
struct PreparedMixed {
  DevTables T;
  TcPlan plan;
  const void* coef = nullptr;
  cudaStream_t stream = nullptr;
  double cutoff = 0.0;
  // cusp adjustment (null when the context has none): radii [nucl] and the
  // cubics' parameters [nucl][4][mo] on the device
  const double* cusp_r = nullptr;
  const double* cusp_prm = nullptr;
  int* err = nullptr;   // the context's error word of the tensor-core kernels
};

// Load, during a regular evaluation, the device code and data the
// allocation-free entry point uses later (lazy module loading would
// otherwise allocate device memory at its first call): the unfused kernels
// (mo_tc.cu) and the fixed scratch array (noalloc.cu).
cudaError_t tc_prime_unfused();
cudaError_t noalloc_prime();

}  // namespace qb
