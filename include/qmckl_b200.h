/*
 * qmckl_b200.h -- B200 extensions beside the unchanged qmckl.h surface.
 *
 * The reference library has no device interface; these entry points have no
 * counterpart in it.  They give callers that keep their electron coordinates
 * and results in GPU memory a way to run the same evaluation without host
 * copies, and expose the knobs of the device implementation.  Every function
 * returns a qmckl_exit_code and records failures with qmckl_failwith, like
 * the reference's own functions (org/qmckl_error.org:539-598).
 */
#ifndef QMCKL_B200_H
#define QMCKL_B200_H

#include "qmckl.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Arithmetic form of the device kernels.
 *  AUTO : FP64 when the context precision is > 26 bits, else MIXED.  The
 *         threshold is where the reference switches its MO contraction to
 *         single precision (org/qmckl_mo.org:2028-2039).
 *  FP64 : all arithmetic in FP64 (parity form).
 *  MIXED: FP32 AO arithmetic (FP64 displacements, r^2, tight exponents and the
 *         Laplacian radial factor) and the MO contraction on tcgen05 tensor
 *         cores as split-BF16 products accumulated in FP32. */
#define QMCKL_B200_FORM_AUTO  0
#define QMCKL_B200_FORM_FP64  1
#define QMCKL_B200_FORM_MIXED 2

qmckl_exit_code qmckl_b200_set_form(qmckl_context context, const int32_t form);
qmckl_exit_code qmckl_b200_get_form(const qmckl_context context, int32_t* const form);

/* Operand split of the fused mixed MO contraction: 3 (default) = three
 * bfloat16 pieces, six products (all pairs of total order <= 2); 2 = two
 * float16 pieces of values scaled by powers of two (per accumulator row from
 * a bound of the row's AOs, per MO from its largest coefficient), three
 * products.  The unfused organisation (qmckl_b200_set_mixed_kernel(ctx, 0))
 * and qmckl_b200_mo_vgl_device_noalloc always use three bfloat16 pieces. */
qmckl_exit_code qmckl_b200_set_split_terms(qmckl_context context, const int32_t pieces);

/* Kernel organisation of the mixed form: 1 (default) runs the fused kernel
 * that produces the bfloat16 AO pieces in shared memory next to the tensor
 * cores (no AO matrix in device memory); 0 writes the AO pieces to device
 * memory and runs the tensor-core contraction on them. */
qmckl_exit_code qmckl_b200_set_mixed_kernel(qmckl_context context, const int32_t fused);

/* The CUDA device and stream (cudaStream_t passed as void*) the context uses.
 * Default: the current device at the first evaluation, and a non-blocking
 * stream owned by the context.  A stream handle of 0 selects the legacy
 * default stream.  Set the device before the first evaluation.
 * qmckl_b200_synchronize waits for the context's stream and returns
 * QMCKL_FAILURE when a bounded barrier wait of a mixed-form tensor-core
 * kernel gave up since the last synchronization point (the host getters
 * check the same at their end). */
qmckl_exit_code qmckl_b200_set_device(qmckl_context context, const int32_t device);
qmckl_exit_code qmckl_b200_set_stream(qmckl_context context, void* stream);
qmckl_exit_code qmckl_b200_synchronize(qmckl_context context);

/* Device-resident evaluation.  d_coord is device memory holding point_num
 * points as [3][point_num] (the 'T' layout of qmckl_set_point); outputs are
 * device memory in the reference layouts ao_vgl[point][5][ao],
 * ao_value[point][ao], mo_vgl[point][5][mo], mo_value[point][mo].  The basis
 * and MO coefficients come from the context.  Work is enqueued on the
 * context's stream; the call returns without synchronizing (the first call
 * of a context, or one after the basis, coefficients or precision changed,
 * first uploads its tables, which waits for the copies). */
qmckl_exit_code qmckl_b200_ao_vgl_device(qmckl_context context, const int64_t point_num,
                                         const double* d_coord, double* d_ao_vgl);
qmckl_exit_code qmckl_b200_ao_value_device(qmckl_context context, const int64_t point_num,
                                           const double* d_coord, double* d_ao_value);
qmckl_exit_code qmckl_b200_mo_vgl_device(qmckl_context context, const int64_t point_num,
                                         const double* d_coord, double* d_mo_vgl);
qmckl_exit_code qmckl_b200_mo_value_device(qmckl_context context, const int64_t point_num,
                                           const double* d_coord, double* d_mo_value);
/* AO Hessian into device memory, layout of qmckl_get_ao_basis_ao_hessian
 * ([3][point][4][ao], org/qmckl_ao.org:9400-9404). */
qmckl_exit_code qmckl_b200_ao_hessian_device(qmckl_context context, const int64_t point_num,
                                             const double* d_coord, double* d_ao_hessian);

/* Adjoint of MO VGL (no counterpart in the reference, which offers the
 * orbital forces qmckl_get_forces_mo_value / _mo_g / _mo_l of
 * org/qmckl_forces.org:5550-6880 as full tensors instead).  For the scalar
 * L = sum_{p,c,i} d_weight[p][c][i] * mo_vgl[p][c][i] (d_weight in the
 * mo_vgl layout [point][5][mo]) it writes, each output optional (NULL):
 *   d_grad_coef  [mo][ao]  dL/d coefficient (the qmckl_set_mo_basis_coefficient layout)
 *   d_grad_nucl  [nucl][3] dL/d nuclear coordinates
 *   d_grad_coord [3][point] dL/d point coordinates (the d_coord layout)
 * Outputs are overwritten.  Nothing of a forward evaluation is reused: the
 * AOs and their derivatives are recomputed.  The context's form selects the
 * arithmetic: FP64 throughout, or mixed: the contractions dL/dC = AO^T W and
 * W C^T on the tensor cores as split-bfloat16 products accumulated in FP32
 * over slices of 2048 rows summed in FP64, FP32 exponentials and FP32
 * per-AO derivative arithmetic (gradients within ~4e-7 of the FP64 form's
 * largest entries).  Both forms return without synchronizing; a bounded
 * wait of the mixed form's kernels that gives up is reported by the next
 * qmckl_b200_synchronize. */
qmckl_exit_code qmckl_b200_mo_vgl_adjoint_device(qmckl_context context, const int64_t point_num,
                                                 const double* d_coord, const double* d_weight,
                                                 double* d_grad_coef, double* d_grad_nucl, double* d_grad_coord);

/* Batched MO VGL (mixed form) of many independent systems in one persistent
 * launch driven by a device work queue (no counterpart in the reference,
 * which evaluates one context at a time).  A batch snapshots, at creation,
 * the basis, nuclei, MO coefficients and precision of each context and takes
 * the number of points of each system; re-create it after changing a
 * context.  Coordinates and results are packed device buffers: system s
 * reads [3][point_num[s]] doubles at d_coord + coord_offset[s] and writes
 * mo_vgl[point_num[s]][5][mo_num_s] at d_mo_vgl + out_offset[s]
 * (qmckl_b200_batch_layout; totals[0], totals[1] = buffer lengths in
 * doubles).  qmckl_b200_batch_mo_vgl_device enqueues one persistent launch
 * (replayed from a CUDA graph while the buffers and tuning stay the same;
 * qmckl_b200_batch_set_graph(b, 0) launches directly) on the batch's own
 * stream or the one set by qmckl_b200_batch_set_stream (graph capture needs
 * a stream other than the legacy default one); qmckl_b200_batch_synchronize
 * waits and returns QMCKL_FAILURE when a bounded wait of the launch gave up
 * (*status = its code).  qmckl_b200_batch_mo_vgl_loop_device computes the
 * same with one launch sequence per system (synchronous).
 * qmckl_b200_batch_tune times the kernel variants (producer warps 16 or 8,
 * queue order 0: largest work per tile first, 1: system by system, 2: round
 * robin) on the given buffers and keeps the fastest (*best_ms: its time);
 * QMCKL_B200_TUNE_FILE names a file where choices are appended and read back
 * for batches of the same shape.  qmckl_b200_batch_set_wait_limit bounds the
 * dependency waits of tile items to `polls` polls (0: 2 s); publish = 0 keeps
 * the point-order items from releasing their systems (test hook: every wait
 * then fails and the launch ends with an error status). */
typedef int64_t qmckl_b200_batch;
qmckl_exit_code qmckl_b200_batch_create(const qmckl_context* contexts, const int64_t* point_num, const int64_t num,
                                        qmckl_b200_batch* batch);
qmckl_exit_code qmckl_b200_batch_destroy(qmckl_b200_batch batch);
qmckl_exit_code qmckl_b200_batch_layout(qmckl_b200_batch batch, int64_t* coord_offset, int64_t* out_offset,
                                        int64_t* totals);
qmckl_exit_code qmckl_b200_batch_set_stream(qmckl_b200_batch batch, void* stream);
qmckl_exit_code qmckl_b200_batch_set_graph(qmckl_b200_batch batch, const int32_t enable);
qmckl_exit_code qmckl_b200_batch_mo_vgl_device(qmckl_b200_batch batch, const double* d_coord, double* d_mo_vgl);
qmckl_exit_code qmckl_b200_batch_mo_vgl_loop_device(qmckl_b200_batch batch, const double* d_coord,
                                                    double* d_mo_vgl);
qmckl_exit_code qmckl_b200_batch_synchronize(qmckl_b200_batch batch, int32_t* status);
qmckl_exit_code qmckl_b200_batch_tune(qmckl_b200_batch batch, const double* d_coord, double* d_mo_vgl,
                                      const int32_t reps, double* best_ms);
qmckl_exit_code qmckl_b200_batch_set_tuning(qmckl_b200_batch batch, const int32_t producer_warps, const int32_t order);
qmckl_exit_code qmckl_b200_batch_get_tuning(qmckl_b200_batch batch, int32_t* producer_warps, int32_t* order);
qmckl_exit_code qmckl_b200_batch_set_wait_limit(qmckl_b200_batch batch, const int64_t polls, const int32_t publish);

/* Mixed-form MO VGL that allocates no device memory.  No counterpart in the
 * reference library.
 *
 * For callers that cannot allocate device memory when they evaluate the
 * orbitals: codes whose device memory is held by a pool allocator that has
 * already reserved the free memory (cudaMalloc would fail, and memory freed
 * with cudaFree would escape the pool).  Same arguments, result and
 * arithmetic as qmckl_b200_mo_vgl_device in the mixed form with the unfused
 * kernels (it always evaluates the mixed form, whatever qmckl_b200_set_form
 * says), but the scratch it needs lives in one fixed 32 MiB array inside the
 * library, held by every GPU that loads the library until the process exits.
 * The caller passes the coordinates and the output buffer (device memory).
 *   - Limit: point_num * 5 rows of the AO matrix in 3 bfloat16 pieces
 *     of ao_num rounded up to 64 columns must fit in the 32 MiB; larger
 *     point_num is rejected with QMCKL_INVALID_ARG_2 and a message giving the
 *     largest point count for the basis (546 points for 2000 AOs).
 *   - The basis tables, the split MO coefficients and the context's error
 *     word must already be on the device: run one regular mixed-form
 *     evaluation of the context first (that one allocates, and it also loads
 *     the kernels and the fixed array this call uses); otherwise
 *     QMCKL_NOT_PROVIDED.
 *   - Every call uses the same array and it keeps the previous call's
 *     contents (every byte a call reads was written by that call).  Calls
 *     whose GPU work overlaps (other streams, other host threads, other
 *     contexts) race on the array: order them on one stream.
 *   - The work is enqueued on the context's stream and the call returns
 *     without synchronizing; a bounded wait of its kernels that gives up is
 *     reported by the context's next synchronization point
 *     (qmckl_b200_synchronize or a host getter) as QMCKL_FAILURE. */
qmckl_exit_code qmckl_b200_mo_vgl_device_noalloc(qmckl_context context, const int64_t point_num,
                                                 const double* d_coord, double* d_mo_vgl);

/* Tile skipping of the fused mixed-form kernel: the 16-AO k-steps (a
 * quarter of a 64-AO K block) whose MMAs it issued, and the k-steps of the
 * dense contraction, summed over its launches
 * (one count per CTA: tile of points x MO tile) since the context's first
 * fused evaluation or the last reset (reset != 0 clears them after reading).
 * Both 0 before any fused evaluation.  Synchronizes the context's stream. */
qmckl_exit_code qmckl_b200_get_kblock_stats(qmckl_context context, int64_t* evaluated, int64_t* total,
                                           const int32_t reset);

/* Test hook: write `code` into the context's error word of the mixed-form
 * tensor-core kernels, as a bounded barrier wait that gave up would, so that
 * the next synchronization point reports QMCKL_FAILURE.  Needs one mixed-form
 * evaluation of the context first (QMCKL_NOT_PROVIDED otherwise). */
qmckl_exit_code qmckl_b200_inject_wait_failure(qmckl_context context, const int32_t code);

/* The MO tiling of the fused mixed-form kernel for ao_num AOs, mo_num MOs and
 * `pieces` (2 or 3) split pieces: tile width, tile count, FP32 accumulators
 * per tile (3, or 2 for wide tiles) and pipeline stages (2 or 3), as the
 * library chooses them (QMCKL_B200_WIDE_TILES included).  Host only: needs
 * no device and no context. */
qmckl_exit_code qmckl_b200_get_fused_plan(const int64_t ao_num, const int64_t mo_num, const int32_t pieces,
                                          int32_t* n_tile, int32_t* n_tiles, int32_t* accumulators,
                                          int32_t* stages);

/* Test hook: in the fused mixed-form VGL kernel (3 pieces) launched after
 * this call, in this process, every producer warp holding a chunk of a
 * skipped 16-AO k-step sleeps `ns` nanoseconds (0 <= ns <= 1e7; 0 = off, the
 * default, which launches the kernel without the sleep) before it waits for
 * its pipeline stage, so that its block's MMAs can complete before that wait
 * starts.  The results must not change. */
qmckl_exit_code qmckl_b200_inject_late_warps(const int64_t ns);

/* Number of kernels this library launched since the process started. */
int64_t qmckl_b200_kernel_launch_count(void);

/* Fault-injection hook for tests: make the n-th next allocation (host
 * registry or device) fail with QMCKL_ALLOCATION_FAILED; n < 0 disables. */
void qmckl_b200_inject_alloc_failure(const int64_t n);

#ifdef __cplusplus
}
#endif
#endif /* QMCKL_B200_H */
