/*
 * Stand-in for the parts of the reference library that its HPC orbital
 * kernels touch, so that those kernels -- extracted verbatim from the
 * reference's org sources by oracle/build_ref.py -- compile on their own into
 * oracle/_ref/libqmckl_ref.so.  TEST INFRASTRUCTURE ONLY: the reference's own
 * CPU path, used as the checker of the oracle and as the timed CPU baseline;
 * the product library never links it.
 *
 * What is stood in for, and where the reference defines it:
 *   - the context: only the fields the kernels read or the basis finalization
 *     writes (org/qmckl_context.org:183-198 holds the real struct; the
 *     nucleus, AO basis and numerical-precision sub-structs are in
 *     org/qmckl_nucleus.org, org/qmckl_ao.org:330-420, org/qmckl_numprec.org);
 *   - matrix and tensor values and their index macros (column-major, as
 *     org/qmckl_blas.org:197-300 and 576-579 define them);
 *   - memory allocation (org/qmckl_memory.org) by plain malloc, and the few
 *     API calls qmckl_finalize_basis makes (oracle/ref_shim.c).
 * Exit codes and the public prototypes come from include/qmckl.h.
 */
#ifndef QMCKL_B200_REF_SHIM_H
#define QMCKL_B200_REF_SHIM_H

#include <assert.h>
#include <math.h>
#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/qmckl.h"

#define QMCKL_TENSOR_ORDER_MAX 16

typedef struct qmckl_matrix {
  double* restrict data;
  int64_t size[2];
} qmckl_matrix;

typedef struct qmckl_tensor {
  double* restrict data;
  int32_t order;
  int32_t unused;
  int64_t size[QMCKL_TENSOR_ORDER_MAX];
} qmckl_tensor;

/* element (i, j) of a column-major matrix, (i, j, k) of a column-major tensor */
#define qmckl_mat(m, i, j) m.data[(i) + (j) * m.size[0]]
#define qmckl_ten3(t, i, j, k) t.data[(i) + t.size[0] * ((j) + t.size[1] * (k))]

typedef struct qmckl_memory_info_struct {
  size_t size;
} qmckl_memory_info_struct;
static const qmckl_memory_info_struct qmckl_memory_info_struct_zero = {0};

void* qmckl_malloc(qmckl_context context, const qmckl_memory_info_struct info);
qmckl_matrix qmckl_matrix_alloc(qmckl_context context, const int64_t size1, const int64_t size2);
qmckl_matrix qmckl_matrix_set(qmckl_matrix matrix, double value);
qmckl_tensor qmckl_tensor_alloc(qmckl_context context, const int32_t order, const int64_t* size);
qmckl_tensor qmckl_tensor_set(qmckl_tensor tensor, double value);

typedef struct ref_ao_basis {
  char type;
  int64_t shell_num, prim_num, ao_num;
  int64_t* nucleus_index;
  int64_t* nucleus_shell_num;
  int32_t* shell_ang_mom;
  int64_t* shell_prim_num;
  int64_t* shell_prim_index;
  double* shell_factor;
  double* exponent;
  double* coefficient;
  double* prim_factor;
  double* ao_factor;
  int32_t* r_power;
  /* written by qmckl_finalize_basis / qmckl_finalize_basis_hpc */
  int64_t* nucleus_prim_index;
  int32_t* ao_ang_mom;
  int64_t* ao_nucl;
  double* coefficient_normalized;
  int32_t* nucleus_max_ang_mom;
  double* nucleus_range;
  int32_t* prim_num_per_nucleus;
  qmckl_tensor coef_per_nucleus;
  qmckl_matrix expo_per_nucleus;
} ref_ao_basis;

typedef struct ref_nucleus {
  int64_t num;
  qmckl_matrix coord; /* [3][num] as the kernels read it: coord.data[n + d * num] */
} ref_nucleus;

typedef struct ref_numprec {
  int32_t precision;
  int32_t range;
} ref_numprec;

typedef struct qmckl_context_struct {
  int32_t num_threads;
  ref_numprec numprec;
  ref_nucleus nucleus;
  ref_ao_basis ao_basis;
} qmckl_context_struct;

/* extracted functions called before the block that defines them */
qmckl_exit_code qmckl_finalize_basis_hpc(qmckl_context context);
qmckl_exit_code qmckl_compute_mo_basis_mo_vgl_hpc_sp(const qmckl_context context, const int64_t ao_num,
                                                     const int64_t mo_num, const int64_t point_num,
                                                     const double* coefficient_t, const double* ao_vgl,
                                                     double* const mo_vgl);
qmckl_exit_code qmckl_compute_mo_basis_mo_value_hpc_sp(const qmckl_context context, const int64_t ao_num,
                                                       const int64_t mo_num, const int64_t point_num,
                                                       const double* coefficient_t, const double* ao_value,
                                                       double* const mo_value);
qmckl_exit_code qmckl_compute_ao_vgl_hpc_gaussian(
    const qmckl_context context, const int64_t ao_num, const int64_t shell_num,
    const int32_t* prim_num_per_nucleus, const int64_t point_num, const int64_t nucl_num, const double* coord,
    const double* nucl_coord, const int64_t* nucleus_index, const int64_t* nucleus_shell_num,
    const double* nucleus_range, const int32_t* nucleus_max_ang_mom, const int32_t* shell_ang_mom,
    const double* ao_factor, const qmckl_matrix expo_per_nucleus, const qmckl_tensor coef_per_nucleus,
    double* const ao_vgl);
qmckl_exit_code qmckl_compute_ao_value_hpc_gaussian(
    const qmckl_context context, const int64_t ao_num, const int64_t shell_num,
    const int32_t* prim_num_per_nucleus, const int64_t point_num, const int64_t nucl_num, const double* coord,
    const double* nucl_coord, const int64_t* nucleus_index, const int64_t* nucleus_shell_num,
    const double* nucleus_range, const int32_t* nucleus_max_ang_mom, const int32_t* shell_ang_mom,
    const double* ao_factor, const qmckl_matrix expo_per_nucleus, const qmckl_tensor coef_per_nucleus,
    double* const ao_value);
qmckl_exit_code qmckl_compute_mo_basis_mo_vgl_hpc(const qmckl_context context, const int64_t ao_num,
                                                  const int64_t mo_num, const int64_t point_num,
                                                  const double* coefficient_t, const double* ao_vgl,
                                                  double* const mo_vgl);
qmckl_exit_code qmckl_compute_mo_basis_mo_value_hpc(const qmckl_context context, const int64_t ao_num,
                                                    const int64_t mo_num, const int64_t point_num,
                                                    const double* coefficient_t, const double* ao_value,
                                                    double* const mo_value);
qmckl_exit_code qmckl_finalize_basis(qmckl_context context);

/* ---- entry points of libqmckl_ref.so for the tests and the CPU baseline ---- */

/* The arrays handed to the reference's qmckl_set_ao_basis_* setters, the
 * nuclei ([3][nucl_num]), the precision and the thread count. */
typedef struct ref_system_in {
  int64_t nucl_num, shell_num, prim_num, ao_num;
  const double* nucl_coord;
  const int64_t* nucleus_index;
  const int64_t* nucleus_shell_num;
  const int32_t* shell_ang_mom;
  const int64_t* shell_prim_num;
  const int64_t* shell_prim_index;
  const double* shell_factor;
  const double* exponent;
  const double* coefficient;
  const double* prim_factor;
  const double* ao_factor;
  int32_t precision, num_threads;
} ref_system_in;

/* A context finalized by the reference's own qmckl_finalize_basis (NULL on
 * failure). */
qmckl_context_struct* ref_system_create(const ref_system_in* in);
void ref_system_destroy(qmckl_context_struct* ctx);
void ref_system_set(qmckl_context_struct* ctx, int32_t precision, int32_t num_threads);
/* coord [3][point_num]; outputs in the reference layouts */
qmckl_exit_code ref_ao_vgl(qmckl_context_struct* ctx, int64_t point_num, const double* coord, double* ao_vgl);
qmckl_exit_code ref_ao_value(qmckl_context_struct* ctx, int64_t point_num, const double* coord, double* ao_value);
/* coefficient_t [ao_num][mo_num] */
qmckl_exit_code ref_mo_vgl(qmckl_context_struct* ctx, int64_t mo_num, const double* coefficient_t, int64_t point_num,
                           const double* ao_vgl, double* mo_vgl);
qmckl_exit_code ref_mo_value(qmckl_context_struct* ctx, int64_t mo_num, const double* coefficient_t,
                             int64_t point_num, const double* ao_value, double* mo_value);

#endif
