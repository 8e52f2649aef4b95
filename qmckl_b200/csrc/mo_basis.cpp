// MO basis: setters, getters, finalization, MO selection, rescaling, the cusp
// adjustment and the MO array getters.
//
// Follows org/qmckl_mo.org: setters 192-290 (mo_num once, coefficient may be
// replaced), finalize 316-373 (coefficient_t = transpose, cached MO arrays
// dropped, context touched), cusp radii 479-700, getters 483-560, select_mo
// 874-966 (re-fits the cusp parameters of the kept MOs), rescale 3479-3529,
// mo_value get/inplace 988-1112, mo_vgl get/inplace 1626-1747, mo_hessian
// 2362-2400.
#include <cmath>
#include <cstdio>

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
  ctx->mo_basis.mo_hessian_date = 0;
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
  qmckl_exit_code rc = finalize_mo_basis(context);
  // the cusp parameters of the kept MOs are fitted again (org/qmckl_mo.org:955-962)
  if (rc == QMCKL_SUCCESS && !ctx->mo_basis.r_cusp.empty()) {
    const std::vector<double> r = ctx->mo_basis.r_cusp;
    rc = qmckl_set_mo_basis_r_cusp(context, r.data(), (int64_t)r.size());
  }
  return rc;
}

qmckl_exit_code qmckl_set_mo_basis_r_cusp(qmckl_context context, const double* r_cusp, const int64_t size_max) {
  // org/qmckl_mo.org:479-700.  The fit needs the MOs at the nuclei without
  // the s AOs that the adjustment leaves out there (the cusp-adjusted MO
  // values with zero parameters) and the s-AO part of each MO at distance
  // r_cusp from its nucleus; both come from this context's own getters on
  // temporary points, and the caller's points are restored afterwards.
  const char* fn = "qmckl_set_mo_basis_r_cusp";
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_NULL_CONTEXT;
  Context* ctx = ctx_of(context);
  if (r_cusp == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, fn, "r_cusp: Null pointer");
  const int64_t N = ctx->nucleus.num;
  if (size_max < N) return qmckl_failwith(context, QMCKL_INVALID_ARG_3, fn, "Array too small");
  if (!ctx->mo_basis.provided || !ctx->ao_basis.provided || !ctx->nucleus.provided)
    return qmckl_failwith(context, QMCKL_NOT_PROVIDED, fn, "nuclei, AO basis and MO basis must be set first");
  // the cubic's denominators vanish for these radii (the reference asserts,
  // org/qmckl_mo.org:662-668); nuclei with charge < 0.1 are not fitted
  for (int64_t n = 0; n < N; ++n) {
    const double Z = ctx->nucleus.charge[n], R = r_cusp[n];
    if (Z < 0.1) continue;
    if (!(R != 0.) || !(std::fabs(2. * R * Z - 6.) > 1.e-6) || !(std::fabs(R * R * Z - 3. * R) > 1.e-6) ||
        !(std::fabs(R * R * R * Z - 3. * R * R) > 1.e-6)) {
      char msg[QMCKL_MAX_MSG_LEN];
      std::snprintf(msg, sizeof msg, "r_cusp[%lld] = %g makes the cusp fit singular for charge %g", (long long)n, R, Z);
      return qmckl_failwith(context, QMCKL_INVALID_ARG_2, fn, msg);
    }
  }
  if (alloc_should_fail()) return qmckl_failwith(context, QMCKL_ALLOCATION_FAILED, fn, NULL);
  const int64_t A = ctx->ao_basis.ao_num, M = ctx->mo_basis.mo_num;
  const int64_t old_num = ctx->point.num;
  const std::vector<double> old_coord = ctx->point.coord;   // [3][old_num]
  MoBasisRec& mo = ctx->mo_basis;
  mo.r_cusp.assign(r_cusp, r_cusp + N);
  mo.cusp_param.assign((size_t)(N * 4 * M), 0.0);
  mo.cusp_version += 1;
  mo.mo_vgl_date = mo.mo_value_date = mo.mo_hessian_date = 0;
  auto fail = [&](qmckl_exit_code rc, const char* what) {
    mo.r_cusp.clear();
    mo.cusp_param.clear();
    mo.cusp_version += 1;
    mo.mo_vgl_date = mo.mo_value_date = mo.mo_hessian_date = 0;
    return qmckl_failwith(context, rc == QMCKL_SUCCESS ? QMCKL_FAILURE : rc, fn, what);
  };
  // MO values at the nuclei, without the s AOs left out there
  std::vector<double> coord(ctx->nucleus.coord);   // [3][N]
  qmckl_exit_code rc = qmckl_set_point(context, 'T', N, coord.data(), 3 * N);
  if (rc != QMCKL_SUCCESS) return fail(rc, "Unable to set coordinates at the nuclei");
  std::vector<double> eta((size_t)(N * M));
  rc = qmckl_get_mo_basis_mo_value(context, eta.data(), N * M);
  if (rc != QMCKL_SUCCESS) return fail(rc, "Unable to compute the MOs at the nuclei");
  // AO VGL at distance r_cusp from each nucleus along z
  for (int64_t n = 0; n < N; ++n) coord[2 * N + n] += r_cusp[n];
  rc = qmckl_set_point(context, 'T', N, coord.data(), 3 * N);
  if (rc != QMCKL_SUCCESS) return fail(rc, "Unable to set coordinates at r_cusp");
  std::vector<double> av((size_t)(N * 5 * A));
  rc = qmckl_get_ao_basis_ao_vgl(context, av.data(), N * 5 * A);
  if (rc != QMCKL_SUCCESS) return fail(rc, "Unable to compute the AOs at r_cusp");
  const std::vector<int64_t>& ao_nucl = ctx->ao_basis.d.ao_nucl;
  const std::vector<int32_t>& ao_l = ctx->ao_basis.d.ao_ang_mom;
  for (int64_t n = 0; n < N; ++n) {
    const double Z = ctx->nucleus.charge[n];
    if (Z < 0.1) continue;   // dummy atoms
    const double R = r_cusp[n];
    const double* a = &av[(size_t)n * 5 * A];
    for (int64_t i = 0; i < M; ++i) {
      // the nucleus's own s-AO part of MO i: value, z derivative, Laplacian
      double phi = 0., grad_phi = 0., lap_phi = 0.;
      for (int64_t k = 0; k < A; ++k)
        if (ao_nucl[k] == n && ao_l[k] == 0) {
          const double ck = mo.coefficient[i * A + k];
          phi += ck * a[k];
          grad_phi += ck * a[3 * A + k];
          lap_phi += ck * a[4 * A + k];
        }
      const double eta_i = eta[n * M + i];
      double* c = &mo.cusp_param[(size_t)n * 4 * M];
      c[i] = -(R * (2. * eta_i * Z - 6. * grad_phi) + lap_phi * R * R + 6. * phi) / (2. * R * Z - 6.);
      c[M + i] = (lap_phi * R * R * Z - 6. * grad_phi * R * Z + 6. * phi * Z + 6. * eta_i * Z) / (2. * R * Z - 6.);
      c[2 * M + i] = -(R * (-5. * grad_phi * Z - 1.5 * lap_phi) + lap_phi * R * R * Z + 3. * phi * Z + 3. * eta_i * Z +
                       6. * grad_phi) / (R * R * Z - 3. * R);
      c[3 * M + i] = (R * (-2. * grad_phi * Z - lap_phi) + 0.5 * lap_phi * R * R * Z + phi * Z + eta_i * Z +
                      3. * grad_phi) / (R * R * R * Z - 3. * R * R);
    }
  }
  mo.cusp_version += 1;
  mo.mo_vgl_date = mo.mo_value_date = mo.mo_hessian_date = 0;
  // the caller's points back (none set: the last temporary points stay, as in
  // the reference)
  if (old_num > 0) {
    rc = qmckl_set_point(context, 'T', old_num, old_coord.data(), 3 * old_num);
    if (rc != QMCKL_SUCCESS) return qmckl_failwith(context, QMCKL_FAILURE, fn, "Unable to set old coordinates");
  }
  return QMCKL_SUCCESS;
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

qmckl_exit_code qmckl_get_mo_basis_mo_hessian(qmckl_context context, double* const mo_hessian, const int64_t size_max) {
  // org/qmckl_mo.org:2368-2400 (layout [3][point][3][mo])
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_NULL_CONTEXT;
  Context* ctx = ctx_of(context);
  if (!ctx->mo_basis.provided) return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_provide_mo_basis_mo_hessian", NULL);
  const int64_t sze = ctx->point.num * 3 * 3 * ctx->mo_basis.mo_num;
  if (size_max < sze) return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_get_mo_basis_mo_hessian", "input array too small");
  if (mo_hessian == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_mo_basis_mo_hessian", "NULL pointer");
  return dev_provide_mo_hessian(context, mo_hessian);
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
