// MO basis: setters, getters, finalization, MO selection, rescaling and the
// MO array getters.
//
// Follows org/qmckl_mo.org: setters 192-290 (mo_num once, coefficient may be
// replaced), finalize 316-373 (coefficient_t = transpose, cached MO arrays
// dropped, context touched), getters 483-560, select_mo 874-966, rescale
// 3479-3529, mo_value get/inplace 988-1112, mo_vgl get/inplace 1626-1747.
#include "internal.h"

using namespace qb;

namespace qb {

qmckl_exit_code finalize_mo_basis(qmckl_context context) {
  Context* ctx = ctx_of(context);
  const int64_t A = ctx->ao_basis.ao_num, M = ctx->mo_basis.mo_num;
  if (alloc_should_fail()) return qmckl_failwith(context, QMCKL_ALLOCATION_FAILED, "qmckl_finalize_mo_basis", NULL);
  std::vector<double>& c = ctx->mo_basis.coefficient;
  std::vector<double> t((size_t)(A * M));
  for (int64_t i = 0; i < A; ++i)
    for (int64_t j = 0; j < M; ++j) t[i * M + j] = c[j * A + i];
  ctx->mo_basis.coefficient_t = std::move(t);
  ctx->mo_basis.coef_version += 1;
  ctx->mo_basis.mo_vgl_date = 0;
  ctx->mo_basis.mo_value_date = 0;
  dev_invalidate_mo(context);
  return qmckl_context_touch(context);
}

}  // namespace qb

extern "C" {

qmckl_exit_code qmckl_set_mo_basis_mo_num(qmckl_context context, const int64_t mo_num) {
  const int32_t mask = 1;
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_NULL_CONTEXT;
  Context* ctx = ctx_of(context);
  if (!(ctx->mo_basis.uninitialized & mask))
    return qmckl_failwith(context, QMCKL_ALREADY_SET, "qmckl_set_mo_*", NULL);
  if (mo_num <= 0) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_set_mo_basis_mo_num", "mo_num <= 0");
  ctx->mo_basis.mo_num = mo_num;
  ctx->mo_basis.uninitialized &= ~mask;
  ctx->mo_basis.provided = (ctx->mo_basis.uninitialized == 0);
  if (ctx->mo_basis.provided) return finalize_mo_basis(context);
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_set_mo_basis_coefficient(qmckl_context context, const double* coefficient, const int64_t size_max) {
  const int32_t mask = 1 << 1;
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_NULL_CONTEXT;
  Context* ctx = ctx_of(context);
  const int64_t n = ctx->ao_basis.ao_num * ctx->mo_basis.mo_num;
  if (size_max < n) return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_set_mo_basis_coefficient", "Array too small");
  if (n <= 0) return qmckl_failwith(context, QMCKL_FAILURE, "qmckl_set_mo_basis_coefficient", "ao_num or mo_num is not set");
  if (coefficient == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_set_mo_basis_coefficient", "NULL pointer");
  if (alloc_should_fail()) return qmckl_failwith(context, QMCKL_ALLOCATION_FAILED, "qmckl_set_mo_basis_coefficient", NULL);
  ctx->mo_basis.coefficient.assign(coefficient, coefficient + n);
  ctx->mo_basis.uninitialized &= ~mask;
  ctx->mo_basis.provided = (ctx->mo_basis.uninitialized == 0);
  if (ctx->mo_basis.provided) return finalize_mo_basis(context);
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_get_mo_basis_mo_num(const qmckl_context context, int64_t* mo_num) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT)
    return qmckl_failwith(context, QMCKL_INVALID_CONTEXT, "qmckl_get_mo_basis_mo_num", NULL);
  Context* ctx = ctx_of(context);
  if (ctx->mo_basis.uninitialized & 1) return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_get_mo_basis_mo_num", NULL);
  if (mo_num == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_mo_basis_mo_num", "NULL pointer");
  *mo_num = ctx->mo_basis.mo_num;
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_get_mo_basis_coefficient(const qmckl_context context, double* const coefficient, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT)
    return qmckl_failwith(context, QMCKL_INVALID_CONTEXT, "qmckl_get_mo_basis_coefficient", NULL);
  Context* ctx = ctx_of(context);
  if (ctx->mo_basis.uninitialized & (1 << 1)) return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_get_mo_basis_coefficient", NULL);
  if (coefficient == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_mo_basis_coefficient", "NULL pointer");
  const int64_t n = ctx->ao_basis.ao_num * ctx->mo_basis.mo_num;
  if (size_max < n)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_get_mo_basis_coefficient", "Array too small: expected mo_num * ao_num.");
  std::memcpy(coefficient, ctx->mo_basis.coefficient.data(), sizeof(double) * n);
  return QMCKL_SUCCESS;
}

bool qmckl_mo_basis_provided(const qmckl_context context) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return false;
  return ctx_of(context)->mo_basis.provided;
}

qmckl_exit_code qmckl_mo_basis_select_mo(const qmckl_context context, const int32_t* keep, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT)
    return qmckl_failwith(context, QMCKL_INVALID_CONTEXT, "qmckl_get_mo_basis_select_mo", NULL);
  Context* ctx = ctx_of(context);
  if (!qmckl_mo_basis_provided(context)) return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_get_mo_basis_select_mo", NULL);
  if (keep == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_mo_basis_select_mo", "NULL pointer");
  const int64_t M = ctx->mo_basis.mo_num, A = ctx->ao_basis.ao_num;
  if (size_max < M) return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_get_mo_basis_select_mo", "Array too small: expected mo_num.");
  int64_t m_new = 0;
  for (int64_t i = 0; i < M; ++i) m_new += (keep[i] != 0);
  if (alloc_should_fail()) return qmckl_failwith(context, QMCKL_ALLOCATION_FAILED, "qmckl_get_mo_basis_select_mo", NULL);
  std::vector<double> c((size_t)(A * m_new));
  int64_t k = 0;
  for (int64_t i = 0; i < M; ++i)
    if (keep[i] != 0) {
      std::memcpy(&c[k * A], &ctx->mo_basis.coefficient[i * A], sizeof(double) * A);
      ++k;
    }
  ctx->mo_basis.coefficient = std::move(c);
  ctx->mo_basis.mo_num = m_new;
  return finalize_mo_basis(context);
}

qmckl_exit_code qmckl_mo_basis_rescale(qmckl_context context, const double scaling_factor) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT)
    return qmckl_failwith(context, QMCKL_NULL_CONTEXT, "qmckl_mo_basis_rescale", NULL);
  if (scaling_factor == 0.)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_mo_basis_rescale", "scaling factor can't be zero");
  Context* ctx = ctx_of(context);
  if (!ctx->mo_basis.provided) return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_mo_basis_rescale", NULL);
  const int64_t n = ctx->ao_basis.ao_num * ctx->mo_basis.mo_num;
  for (int64_t i = 0; i < n; ++i) {
    ctx->mo_basis.coefficient[i] *= scaling_factor;
    ctx->mo_basis.coefficient_t[i] *= scaling_factor;
  }
  ctx->mo_basis.coef_version += 1;
  dev_invalidate_mo(context);
  return qmckl_context_touch(context);
}

/* ------------------------------------------------- computed array getters */

qmckl_exit_code qmckl_get_mo_basis_mo_value(qmckl_context context, double* const mo_value, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_NULL_CONTEXT;
  Context* ctx = ctx_of(context);
  if (!ctx->mo_basis.provided) return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_provide_mo_basis_mo_value", NULL);
  const int64_t sze = ctx->point.num * ctx->mo_basis.mo_num;
  if (size_max < sze) return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_get_mo_basis_mo_value", "input array too small");
  if (mo_value == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_mo_basis_mo_value", "NULL pointer");
  return dev_provide_mo_value(context, mo_value);
}

qmckl_exit_code qmckl_get_mo_basis_mo_value_inplace(qmckl_context context, double* const mo_value, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT)
    return qmckl_failwith(context, QMCKL_INVALID_CONTEXT, "qmckl_get_mo_basis_mo_value", NULL);
  Context* ctx = ctx_of(context);
  const int64_t sze = ctx->mo_basis.mo_num * ctx->point.num;
  if (size_max < sze) return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_get_mo_basis_mo_value", "input array too small");
  if (!ctx->mo_basis.provided) return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_provide_mo_basis_mo_value", NULL);
  if (mo_value == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_mo_basis_mo_value", "NULL pointer");
  // force the recomputation, and leave the cached array stale afterwards
  // (org/qmckl_mo.org:1066-1074)
  ctx->mo_basis.mo_value_date = ctx->point.date - 1;
  qmckl_exit_code rc = dev_provide_mo_value(context, mo_value);
  ctx->mo_basis.mo_value_date = ctx->point.date - 1;
  return rc;
}

qmckl_exit_code qmckl_get_mo_basis_mo_vgl(qmckl_context context, double* const mo_vgl, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_NULL_CONTEXT;
  Context* ctx = ctx_of(context);
  if (!ctx->mo_basis.provided) return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_provide_mo_basis_mo_vgl", NULL);
  const int64_t sze = ctx->point.num * 5 * ctx->mo_basis.mo_num;
  if (size_max < sze) return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_get_mo_basis_mo_vgl", "input array too small");
  if (mo_vgl == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_mo_basis_mo_vgl", "NULL pointer");
  return dev_provide_mo_vgl(context, mo_vgl);
}

qmckl_exit_code qmckl_get_mo_basis_mo_vgl_inplace(qmckl_context context, double* const mo_vgl, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT)
    return qmckl_failwith(context, QMCKL_INVALID_CONTEXT, "qmckl_get_mo_basis_mo_vgl", NULL);
  Context* ctx = ctx_of(context);
  const int64_t sze = ctx->mo_basis.mo_num * 5 * ctx->point.num;
  if (size_max < sze) return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_get_mo_basis_mo_vgl", "input array too small");
  if (!ctx->mo_basis.provided) return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_provide_mo_basis_mo_vgl", NULL);
  if (mo_vgl == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_mo_basis_mo_vgl", "NULL pointer");
  ctx->mo_basis.mo_vgl_date = ctx->point.date - 1;
  qmckl_exit_code rc = dev_provide_mo_vgl(context, mo_vgl);
  ctx->mo_basis.mo_vgl_date = ctx->point.date - 1;
  return rc;
}

}  // extern "C"
