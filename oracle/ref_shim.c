/*
 * Support code of oracle/_ref/libqmckl_ref.so (TEST INFRASTRUCTURE ONLY):
 * the memory, matrix and context calls that the reference's extracted HPC
 * kernels and basis finalization make, and the library's entry points.  See
 * ref_shim.h.
 */
#include <stdio.h>

#include "ref_shim.h"

void* qmckl_malloc(qmckl_context context, const qmckl_memory_info_struct info) {
  (void)context;
  return calloc(1, info.size > 0 ? info.size : 1);
}

qmckl_matrix qmckl_matrix_alloc(qmckl_context context, const int64_t size1, const int64_t size2) {
  (void)context;
  qmckl_matrix m;
  m.size[0] = size1;
  m.size[1] = size2;
  const int64_t n = size1 * size2;
  m.data = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
  return m;
}

qmckl_matrix qmckl_matrix_set(qmckl_matrix matrix, double value) {
  for (int64_t i = 0; i < matrix.size[0] * matrix.size[1]; ++i) matrix.data[i] = value;
  return matrix;
}

qmckl_tensor qmckl_tensor_alloc(qmckl_context context, const int32_t order, const int64_t* size) {
  (void)context;
  qmckl_tensor t;
  memset(&t, 0, sizeof t);
  t.order = order;
  int64_t n = 1;
  for (int32_t i = 0; i < order; ++i) {
    t.size[i] = size[i];
    n *= size[i];
  }
  t.data = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
  return t;
}

qmckl_tensor qmckl_tensor_set(qmckl_tensor tensor, double value) {
  int64_t n = 1;
  for (int32_t i = 0; i < tensor.order; ++i) n *= tensor.size[i];
  for (int64_t i = 0; i < n; ++i) tensor.data[i] = value;
  return tensor;
}

qmckl_context qmckl_context_check(const qmckl_context context) { return context; }

qmckl_exit_code qmckl_context_touch(const qmckl_context context) {
  (void)context;
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_failwith(qmckl_context context, const qmckl_exit_code exit_code, const char* function,
                               const char* message) {
  (void)context;
  fprintf(stderr, "libqmckl_ref: %s failed (%d)%s%s\n", function ? function : "?", (int)exit_code,
          message ? ": " : "", message ? message : "");
  return exit_code;
}

qmckl_exit_code qmckl_get_nucleus_num(const qmckl_context context, int64_t* const num) {
  *num = ((const qmckl_context_struct*)context)->nucleus.num;
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_set_ao_basis_r_power(qmckl_context context, const int32_t* r_power, const int64_t size_max) {
  qmckl_context_struct* ctx = (qmckl_context_struct*)context;
  if (size_max < ctx->ao_basis.shell_num) return QMCKL_INVALID_ARG_3;
  free(ctx->ao_basis.r_power);
  ctx->ao_basis.r_power = (int32_t*)malloc(sizeof(int32_t) * (size_t)ctx->ao_basis.shell_num);
  memcpy(ctx->ao_basis.r_power, r_power, sizeof(int32_t) * (size_t)ctx->ao_basis.shell_num);
  return QMCKL_SUCCESS;
}

#define DUP(dst, src, n, T)                                                   \
  do {                                                                        \
    dst = (T*)malloc(sizeof(T) * (size_t)((n) > 0 ? (n) : 1));                \
    memcpy(dst, src, sizeof(T) * (size_t)(n));                                \
  } while (0)

qmckl_context_struct* ref_system_create(const ref_system_in* in) {
  qmckl_context_struct* ctx = (qmckl_context_struct*)calloc(1, sizeof(qmckl_context_struct));
  ctx->num_threads = in->num_threads > 0 ? in->num_threads : 1;
  ctx->numprec.precision = in->precision;
  ctx->numprec.range = 11;
  ctx->nucleus.num = in->nucl_num;
  ctx->nucleus.coord = qmckl_matrix_alloc(0, in->nucl_num, 3);
  memcpy(ctx->nucleus.coord.data, in->nucl_coord, sizeof(double) * 3 * (size_t)in->nucl_num);
  ref_ao_basis* b = &ctx->ao_basis;
  b->type = 'G';
  b->shell_num = in->shell_num;
  b->prim_num = in->prim_num;
  b->ao_num = in->ao_num;
  DUP(b->nucleus_index, in->nucleus_index, in->nucl_num, int64_t);
  DUP(b->nucleus_shell_num, in->nucleus_shell_num, in->nucl_num, int64_t);
  DUP(b->shell_ang_mom, in->shell_ang_mom, in->shell_num, int32_t);
  DUP(b->shell_prim_num, in->shell_prim_num, in->shell_num, int64_t);
  DUP(b->shell_prim_index, in->shell_prim_index, in->shell_num, int64_t);
  DUP(b->shell_factor, in->shell_factor, in->shell_num, double);
  DUP(b->exponent, in->exponent, in->prim_num, double);
  DUP(b->coefficient, in->coefficient, in->prim_num, double);
  DUP(b->prim_factor, in->prim_factor, in->prim_num, double);
  DUP(b->ao_factor, in->ao_factor, in->ao_num, double);
  if (qmckl_finalize_basis((qmckl_context)ctx) != QMCKL_SUCCESS) {
    ref_system_destroy(ctx);
    return NULL;
  }
  return ctx;
}

void ref_system_destroy(qmckl_context_struct* ctx) {
  if (ctx == NULL) return;
  ref_ao_basis* b = &ctx->ao_basis;
  void* arrays[] = {b->nucleus_index, b->nucleus_shell_num, b->shell_ang_mom, b->shell_prim_num, b->shell_prim_index,
                    b->shell_factor, b->exponent, b->coefficient, b->prim_factor, b->ao_factor, b->r_power,
                    b->nucleus_prim_index, b->ao_ang_mom, b->ao_nucl, b->coefficient_normalized,
                    b->nucleus_max_ang_mom, b->nucleus_range, b->prim_num_per_nucleus, b->coef_per_nucleus.data,
                    b->expo_per_nucleus.data, ctx->nucleus.coord.data};
  for (size_t i = 0; i < sizeof arrays / sizeof arrays[0]; ++i) free(arrays[i]);
  free(ctx);
}

void ref_system_set(qmckl_context_struct* ctx, int32_t precision, int32_t num_threads) {
  if (precision > 0) ctx->numprec.precision = precision;
  if (num_threads > 0) ctx->num_threads = num_threads;
}

qmckl_exit_code ref_ao_vgl(qmckl_context_struct* ctx, int64_t point_num, const double* coord, double* ao_vgl) {
  const ref_ao_basis* b = &ctx->ao_basis;
  return qmckl_compute_ao_vgl_hpc_gaussian(
      (qmckl_context)ctx, b->ao_num, b->shell_num, b->prim_num_per_nucleus, point_num, ctx->nucleus.num, coord,
      ctx->nucleus.coord.data, b->nucleus_index, b->nucleus_shell_num, b->nucleus_range, b->nucleus_max_ang_mom,
      b->shell_ang_mom, b->ao_factor, b->expo_per_nucleus, b->coef_per_nucleus, ao_vgl);
}

qmckl_exit_code ref_ao_value(qmckl_context_struct* ctx, int64_t point_num, const double* coord, double* ao_value) {
  const ref_ao_basis* b = &ctx->ao_basis;
  return qmckl_compute_ao_value_hpc_gaussian(
      (qmckl_context)ctx, b->ao_num, b->shell_num, b->prim_num_per_nucleus, point_num, ctx->nucleus.num, coord,
      ctx->nucleus.coord.data, b->nucleus_index, b->nucleus_shell_num, b->nucleus_range, b->nucleus_max_ang_mom,
      b->shell_ang_mom, b->ao_factor, b->expo_per_nucleus, b->coef_per_nucleus, ao_value);
}

qmckl_exit_code ref_mo_vgl(qmckl_context_struct* ctx, int64_t mo_num, const double* coefficient_t, int64_t point_num,
                           const double* ao_vgl, double* mo_vgl) {
  return qmckl_compute_mo_basis_mo_vgl_hpc((qmckl_context)ctx, ctx->ao_basis.ao_num, mo_num, point_num,
                                           coefficient_t, ao_vgl, mo_vgl);
}

qmckl_exit_code ref_mo_value(qmckl_context_struct* ctx, int64_t mo_num, const double* coefficient_t,
                             int64_t point_num, const double* ao_value, double* mo_value) {
  return qmckl_compute_mo_basis_mo_value_hpc((qmckl_context)ctx, ctx->ao_basis.ao_num, mo_num, point_num,
                                             coefficient_t, ao_value, mo_value);
}
