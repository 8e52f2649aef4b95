// Device-side tables and kernel launchers of the orbital-evaluation path.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace qb {

// Limits of the per-warp shared-memory staging in the AO kernels.  A nucleus
// block holds at most kBlockNuc nuclei and kBlockSlots shells; finalization
// rejects a basis with more than kBlockSlots shells on one nucleus.
constexpr int kBlockNuc = 32;
constexpr int kBlockSlots = 64;

// Basis tables in device memory (one allocation; see device.cu).
//
// Nuclei are grouped into blocks of consecutive nuclei.  A block's AOs are
// contiguous ([ao_begin, ao_end)) because AOs are numbered nucleus by nucleus.
// The block's shells are its "slots" (block-local shell numbering) and each AO
// carries its slot, its block-local nucleus and its cartesian powers.
struct DevTables {
  int32_t nucl_num, shell_num, prim_num, ao_num, nblock, nslot;
  const double* nucl_coord;       // [3][nucl]
  const double* nucleus_range;    // [nucl]
  const int32_t* nuc_prim_start;  // [nucl+1] into expo (sorted, de-duplicated per nucleus)
  const double* expo;             // [sum of unique primitives]
  const int4* block;              // [nblock] (nuc_begin, nuc_end, ao_begin, ao_end)
  const int2* block_slots;        // [nblock] (slot_begin, slot_end)
  const int32_t* slot_nuc;        // [nslot] global nucleus of a slot
  const int2* slot_coef;          // [nslot] (begin, end) into coef_prim / coef_val
  const int32_t* coef_prim;       // nucleus-local index of the sorted primitive
  const double* coef_val;         // normalized, merged coefficient
  const int32_t* ao_code;         // [ao] a | b<<4 | c<<8 | l<<12 | slot<<16 | nuc_local<<24
  const double* ao_factor;        // [ao]
  // tables of the primitive / shell getters (unsorted, as set by the user)
  const int32_t* prim_nuc;        // [prim]
  const double* prim_expo;        // [prim]
  const double* prim_coef;        // [prim] normalized coefficient
  const int32_t* shell_nuc;       // [shell]
  const int2* shell_prims;        // [shell] (prim_begin, prim_end)
  // tables of the fused AO -> MO kernel (global shell numbering)
  const int32_t* ao_shell;        // [ao] shell of each AO
  const int2* shell_coef;         // [shell] (begin, end) into coef_prim / coef_val
  const double2* coef_ac;         // [coefficient entry] (exponent, coefficient): coef_val with its exponent
};

// Global count of kernels launched by this library.
void count_launch(int n = 1);

// Cusp adjustment of the MOs (org/qmckl_mo.org:2839, 3133, 2659): the s AOs
// of a nucleus are left out of the MO sums at points closer to it than its
// radius cusp_r[nucl] (strictly for MO values, r <= r_cusp for the VGL and the
// Hessian).  r2 < 0 marks a nucleus screened out (its AOs vanish anyway).
__device__ __forceinline__ bool cusp_masked(const double* cusp_r, int l, int nucl, double r2, bool strict) {
  if (cusp_r == nullptr || l != 0 || r2 < 0.0) return false;
  const double r = sqrt(r2), R = cusp_r[nucl];
  return strict ? (r < R) : (r <= R);
}

// Whole warp: the positions (relative to slots.x) of a nucleus block's shells
// whose nucleus is in range of the point (nuc[.][3] >= 0), packed in slot
// order into act; returns their count.  The radial staging then runs over
// the live shells only, in as few 32-lane passes as they need.
__device__ __forceinline__ int pack_live_slots(const int32_t* __restrict__ slot_nuc, int blk_first, int2 slots,
                                               const double (*nuc)[4], uint8_t* act, int lane) {
  int n = 0;
  for (int s0 = slots.x; s0 < slots.y; s0 += 32) {
    const int s = s0 + lane;
    const bool live = s < slots.y && nuc[slot_nuc[s] - blk_first][3] >= 0.0;
    const unsigned int m = __ballot_sync(0xffffffffu, live);
    if (live) act[n + __popc(m & ((1u << lane) - 1u))] = (uint8_t)(s - slots.x);
    n += __popc(m);
  }
  __syncwarp();
  return n;
}

// AO kernels (ao_kernels.cu).  coord is [3][point_num].  All return
// cudaGetLastError() after the launch.
// cusp_r (optional, [nucl]): the AOs that the cusp adjustment leaves out of
// the MO sums are written as zero (the arrays then only feed the MO step).
cudaError_t launch_ao_vgl_f64(const DevTables& T, int64_t point_num, const double* coord,
                              double cutoff, bool dp_exp, double* ao_vgl, cudaStream_t s,
                              const double* cusp_r = nullptr);
// The same FP64 AO VGL stored as 3 bfloat16 pieces (split.cuh) of rows
// p*5 + c: pieces[q * pstride + row * lda + ao] (lda, pstride multiples of 8).
cudaError_t launch_ao_vgl_pieces(const DevTables& T, int64_t point_num, const double* coord, double cutoff,
                                 bool dp_exp, void* pieces, int64_t lda, int64_t pstride, cudaStream_t s);
cudaError_t launch_ao_value_f64(const DevTables& T, int64_t point_num, const double* coord,
                                double cutoff, bool dp_exp, double* ao_value, cudaStream_t s,
                                const double* cusp_r = nullptr);
// Cusp adjustment (cusp.cu, org/qmckl_mo.org:2807-2860, 3099-3185,
// 2629-2697): adds, for every nucleus closer to a point than its radius, the
// cubic c0 + c1 r + c2 r^2 + c3 r^3 (prm [nucl][4][mo]) to the point's MO
// values (comps 1, r <= r_cusp) or its value, gradient and Laplacian
// (comps 5, r < r_cusp) in out[point][comps][mo]; its Hessian to
// out[3][point][3][mo].  coord [3][cstride].
cudaError_t launch_cusp_mo(int64_t P, int comps, const double* coord, int64_t cstride, int N, const double* nucl,
                           const double* r_cusp, const double* prm, int M, double* out, cudaStream_t s);
cudaError_t launch_cusp_hessian(int64_t P, const double* coord, int N, const double* nucl, const double* r_cusp,
                                const double* prm, int M, double* out, cudaStream_t s);
// en_distance[point][nucl] (org/qmckl_electron.org:1357-1393)
cudaError_t launch_en_distance(int64_t P, const double* coord, int N, const double* nucl, double* out,
                               cudaStream_t s);
cudaError_t launch_primitive_vgl(const DevTables& T, int64_t point_num, const double* coord,
                                 double cutoff, double* prim_vgl, cudaStream_t s);
cudaError_t launch_shell_vgl(const DevTables& T, int64_t point_num, const double* coord,
                             double cutoff, double* shell_vgl, cudaStream_t s);

// Mixed-form AO kernel: writes the AO matrix A[(point,comp)][k] as `pieces`
// bfloat16 matrices (A = sum of pieces), each [5*point_num][lda], lda >= ao_num,
// pieces at stride piece_stride elements.
cudaError_t launch_ao_vgl_split(const DevTables& T, int64_t point_num, const double* coord,
                                double cutoff, int pieces, void* a_pieces, int64_t lda,
                                int64_t piece_stride, cudaStream_t s);

// FP64 GEMM C[M][N] = A[M][K] * B[K][N], row-major with leading dimensions (gemm_f64.cu).
cudaError_t launch_gemm_f64(int64_t M, int64_t N, int64_t K, const double* A, int64_t lda,
                            const double* B, int64_t ldb, double* C, int64_t ldc, cudaStream_t s);

// Tile-sparse FP64 MO contraction (gemm_f64.cu).  launch_f64_plan writes,
// for tiles of 128 / comps points in the order perm, the list of AOs whose
// shell reaches some point of the tile (basis order; sph[s] = double4 of the
// shell's nucleus and squared screening radius, shell_ao[s] = int2 first AO
// and AO count) into plan (f64_plan_bytes); launch_gemm_f64_sparse then
// computes out[p][c][n] = sum over the tile's list of ao[p][c][k] * Bt[k][n]
// (Bt: coefficient_t with ldb even and 16-byte aligned rows).
size_t f64_plan_bytes(int64_t point_num, int comps, int64_t ao_num);
cudaError_t launch_f64_plan(int64_t point_num, int comps, const double* coord, int64_t cstride, const int* perm,
                            int shell_num, const void* sph, const void* shell_ao, int64_t ao_num, void* plan,
                            cudaStream_t s);
cudaError_t launch_gemm_f64_sparse(int64_t point_num, int comps, int64_t N, const double* ao, int64_t lda,
                                   const int* perm, const void* plan, int64_t ao_num, const double* Bt, int64_t ldb,
                                   double* C, int64_t ldc, cudaStream_t s);

// Split-K FP64 GEMM with A transposed: part[z][m][n] = sum over the z-th K
// range of A[k][m] * B[k][n] (A element (m, k) at A[k * lda + m]), for
// z < splits; part is [splits][M][N].
cudaError_t launch_gemm_f64_tn_split(int64_t M, int64_t N, int64_t K, const double* A, int64_t lda, const double* B,
                                     int64_t ldb, double* part, int splits, cudaStream_t s);
// out[n][m] = (out[n][m] +) sum_z part[z][m][n]  (fixed summation order)
cudaError_t launch_add_transposed(const double* part, int splits, int64_t M, int64_t N, double* out, bool accumulate,
                                  cudaStream_t s);

// Derivative kernels (adjoint.cu).  ao_hessian: [3][point_num][4][ao]
// (coord [3][point_num]).  Adjoint: G [point_num][5][ao]; grad_nucl
// [nucl][3] -= and grad_coord [3][gstride] += (may be null); coord
// [3][cstride].  `mixed` selects FP32 exponentials where a r^2 <= 30; for
// the adjoint it also means G in FP32 (float*, else double*) and FP32
// per-AO derivative arithmetic.
cudaError_t launch_ao_hessian(const DevTables& T, int64_t point_num, const double* coord, double cutoff, bool mixed,
                              double* ao_hessian, cudaStream_t s, const double* cusp_r = nullptr);
// Orbital forces (adjoint.cu): which = 0 forces_mo_value, 1 forces_mo_g,
// 2 forces_mo_l (from X = ao_vgl for 0, ao_hessian for 1 and 2, and
// Ct = coefficient_t [ao][mo]), 3 forces_ao_value (from X = ao_vgl).
// nuc_ao[a] = AO range of nucleus a.
cudaError_t launch_forces(int which, int64_t P, int64_t A, int64_t M, int N, const int2* nuc_ao, const double* X,
                          const double* Ct, double* out, cudaStream_t s);
cudaError_t launch_mo_adjoint_nuclear(const DevTables& T, int64_t point_num, const double* coord, int64_t cstride,
                                      double cutoff, bool mixed, const void* G, double* grad_nucl,
                                      double* grad_coord, int64_t gstride, cudaStream_t s);

}  // namespace qb
