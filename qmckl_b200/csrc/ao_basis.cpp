// AO basis: setters, getters, finalization and the AO array getters.
//
// Setters/getters follow org/qmckl_ao.org:388-2266 (bit masks of the
// `uninitialized` word, exit codes, size_max checks, automatic finalization
// when the 14th field is set).  Finalization restates qmckl_finalize_basis
// (org/qmckl_ao.org:2965-3226) and the HPC tables of qmckl_finalize_basis_hpc
// (3280-3410): per-nucleus exponents sorted ascending and de-duplicated, with a
// sparse (primitive, coefficient) list per shell, which is the form the GPU
// kernels consume.  The array getters (3415-3798) compute on the device and
// copy into the caller's buffer.
#include <algorithm>
#include <numeric>

#include "internal.h"

using namespace qb;

namespace {

constexpr int kMaxAngMom = 7;

inline int64_t lstart(int l) { return (int64_t)l * (l + 1) * (l + 2) / 6; }

qmckl_exit_code pre(qmckl_context context, int32_t mask) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT)
    return qmckl_failwith(context, QMCKL_NULL_CONTEXT, "qmckl_set_ao_*", NULL);
  Context* ctx = ctx_of(context);
  if (mask != 0 && !(ctx->ao_basis.uninitialized & mask))
    return qmckl_failwith(context, QMCKL_ALREADY_SET, "qmckl_set_ao_*", NULL);
  return QMCKL_SUCCESS;
}

qmckl_exit_code post(qmckl_context context, int32_t mask) {
  Context* ctx = ctx_of(context);
  ctx->ao_basis.uninitialized &= ~mask;
  ctx->ao_basis.provided = (ctx->ao_basis.uninitialized == 0);
  if (ctx->ao_basis.provided) return finalize_basis(context);
  return QMCKL_SUCCESS;
}

template <typename T>
qmckl_exit_code set_array(qmckl_context context, int32_t mask, const char* fname,
                          int64_t needed, const char* needed_what, const T* src,
                          int64_t size_max, std::vector<T>& dst,
                          qmckl_exit_code not_set_code = QMCKL_FAILURE,
                          qmckl_exit_code small_code = QMCKL_INVALID_ARG_3) {
  qmckl_exit_code rc = pre(context, mask);
  if (rc != QMCKL_SUCCESS) return rc;
  if (needed <= 0) return qmckl_failwith(context, not_set_code, fname, needed_what);
  if (size_max < needed) return qmckl_failwith(context, small_code, fname, "input array too small");
  if (src == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, fname, "NULL pointer");
  if (alloc_should_fail()) return qmckl_failwith(context, QMCKL_ALLOCATION_FAILED, fname, NULL);
  dst.assign(src, src + needed);
  return post(context, mask);
}

template <typename T>
qmckl_exit_code get_array(qmckl_context context, int32_t mask, const char* fname,
                          T* dst, int64_t size_max, int64_t n, const std::vector<T>& src,
                          const char* small_msg) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT)
    return qmckl_failwith(context, QMCKL_INVALID_CONTEXT, fname, NULL);
  Context* ctx = ctx_of(context);
  if ((ctx->ao_basis.uninitialized & mask) != 0) return qmckl_failwith(context, QMCKL_NOT_PROVIDED, fname, NULL);
  if (dst == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, fname, "NULL pointer");
  if (size_max < n) return qmckl_failwith(context, QMCKL_INVALID_ARG_3, fname, small_msg);
  std::copy(src.begin(), src.begin() + n, dst);
  return QMCKL_SUCCESS;
}

}  // namespace

namespace qb {

qmckl_exit_code finalize_basis(qmckl_context context) {
  Context* ctx = ctx_of(context);
  AoBasisRec& B = ctx->ao_basis;
  int64_t nucl_num = 0;
  qmckl_exit_code rc = qmckl_get_nucleus_num(context, &nucl_num);
  if (rc != QMCKL_SUCCESS) return rc;
  const int64_t S = B.shell_num, P = B.prim_num, A = B.ao_num, N = nucl_num;
  if ((int64_t)B.nucleus_index.size() < N || (int64_t)B.nucleus_shell_num.size() < N)
    return qmckl_failwith(context, QMCKL_FAILURE, "qmckl_finalize_basis", "nucleus tables shorter than nucl_num");
  // consistency of the shell/primitive tables (the reference asserts these)
  for (int64_t s = 0; s < S; ++s) {
    if (B.shell_ang_mom[s] < 0 || B.shell_ang_mom[s] > kMaxAngMom)
      return qmckl_failwith(context, QMCKL_FAILURE, "qmckl_finalize_basis", "shell angular momentum out of the supported range 0..7");
    if (B.shell_prim_index[s] < 0 || B.shell_prim_num[s] < 0 || B.shell_prim_index[s] + B.shell_prim_num[s] > P)
      return qmckl_failwith(context, QMCKL_FAILURE, "qmckl_finalize_basis", "shell primitive range outside prim_num");
  }
  for (int64_t n = 0; n < N; ++n)
    if (B.nucleus_index[n] < 0 || B.nucleus_shell_num[n] < 0 || B.nucleus_index[n] + B.nucleus_shell_num[n] > S)
      return qmckl_failwith(context, QMCKL_FAILURE, "qmckl_finalize_basis", "nucleus shell range outside shell_num");
  if (!B.r_power_set) { B.r_power.assign((size_t)S, 0); B.r_power_set = true; }
  if (alloc_should_fail()) return qmckl_failwith(context, QMCKL_ALLOCATION_FAILED, "qmckl_finalize_basis", NULL);

  AoDerived d;
  d.nucleus_prim_index.resize(N + 1);
  for (int64_t n = 0; n < N; ++n) d.nucleus_prim_index[n] = B.shell_prim_index[B.nucleus_index[n]];
  d.nucleus_prim_index[N] = P;

  d.ao_ang_mom.assign(A, 0);
  d.ao_nucl.assign(A, 0);
  d.ao_index.assign(S + 1, 0);
  int64_t k = 0;
  for (int64_t n = 0; n < N; ++n)
    for (int64_t s = B.nucleus_index[n]; s < B.nucleus_index[n] + B.nucleus_shell_num[n]; ++s) {
      const int l = B.shell_ang_mom[s];
      d.ao_index[s] = k;
      for (int64_t m = lstart(l); m < lstart(l + 1); ++m) {
        if (k < A) { d.ao_ang_mom[k] = l; d.ao_nucl[k] = n; }
        ++k;
      }
    }
  d.ao_index[S] = A + 1;
  if (k != A)
    return qmckl_failwith(context, QMCKL_FAILURE, "qmckl_finalize_basis",
                          "ao_num does not match the cartesian functions of the shells");

  d.coefficient_normalized.assign(P, 0.0);
  for (int64_t s = 0; s < S; ++s)
    for (int64_t p = B.shell_prim_index[s]; p < B.shell_prim_index[s] + B.shell_prim_num[s]; ++p)
      d.coefficient_normalized[p] = B.coefficient[p] * B.prim_factor[p] * B.shell_factor[s];

  d.nucleus_max_ang_mom.assign(N, 0);
  d.nucleus_range.assign(N, 0.0);
  for (int64_t n = 0; n < N; ++n)
    for (int64_t s = B.nucleus_index[n]; s < B.nucleus_index[n] + B.nucleus_shell_num[n]; ++s) {
      d.nucleus_max_ang_mom[n] = std::max(d.nucleus_max_ang_mom[n], B.shell_ang_mom[s]);
      for (int64_t p = B.shell_prim_index[s]; p < B.shell_prim_index[s] + B.shell_prim_num[s]; ++p) {
        const double range = (double)(B.r_power[s] + 1) / B.exponent[p];
        d.nucleus_range[n] = std::max(d.nucleus_range[n], range);
      }
    }

  // Sorted, de-duplicated exponents per nucleus and the sparse per-shell
  // coefficient lists over them (the qmckl_finalize_basis_hpc tables).
  d.prim_num_per_nucleus.assign(N, 0);
  d.nuc_prim_start.assign(N + 1, 0);
  d.shell_coef_start.assign(S + 1, 0);
  std::vector<std::vector<std::pair<int32_t, double>>> shell_list(S);
  for (int64_t n = 0; n < N; ++n) {
    const int64_t s0 = B.nucleus_index[n], ns = B.nucleus_shell_num[n];
    std::vector<std::pair<double, int64_t>> ex;   // (exponent, position in nucleus order)
    std::vector<int64_t> owner;                   // shell of each position
    std::vector<double> cn;
    for (int64_t s = s0; s < s0 + ns; ++s)
      for (int64_t p = B.shell_prim_index[s]; p < B.shell_prim_index[s] + B.shell_prim_num[s]; ++p) {
        ex.emplace_back(B.exponent[p], (int64_t)ex.size());
        owner.push_back(s);
        cn.push_back(d.coefficient_normalized[p]);
      }
    std::stable_sort(ex.begin(), ex.end(),
                     [](const std::pair<double, int64_t>& a, const std::pair<double, int64_t>& b) { return a.first < b.first; });
    std::vector<int32_t> uniq(ex.size());
    int32_t nu = 0;
    for (size_t i = 0; i < ex.size(); ++i) {
      if (i > 0 && ex[i].first != ex[i - 1].first) ++nu;
      uniq[i] = nu;
    }
    if (!ex.empty()) ++nu;
    d.nuc_prim_start[n] = (int32_t)d.expo_sorted.size();
    std::vector<double> uexp(nu);
    for (size_t i = 0; i < ex.size(); ++i) uexp[uniq[i]] = ex[i].first;
    d.expo_sorted.insert(d.expo_sorted.end(), uexp.begin(), uexp.end());
    d.prim_num_per_nucleus[n] = nu;
    for (int64_t s = s0; s < s0 + ns; ++s) {
      std::vector<double> merged(nu, 0.0);
      for (size_t i = 0; i < ex.size(); ++i) {
        const int64_t pos = ex[i].second;
        merged[uniq[i]] += (owner[pos] == s) ? cn[pos] : 0.0;
      }
      for (int32_t u = 0; u < nu; ++u)
        if (merged[u] != 0.0) shell_list[s].emplace_back(u, merged[u]);
    }
  }
  d.nuc_prim_start[N] = (int32_t)d.expo_sorted.size();
  for (int64_t s = 0; s < S; ++s) {
    d.shell_coef_start[s] = (int32_t)d.coef_prim.size();
    for (auto& pc : shell_list[s]) { d.coef_prim.push_back(pc.first); d.coef_val.push_back(pc.second); }
  }
  d.shell_coef_start[S] = (int32_t)d.coef_prim.size();

  B.d = std::move(d);
  B.basis_version += 1;
  return qmckl_context_touch(context);
}

}  // namespace qb

extern "C" {

qmckl_exit_code qmckl_set_ao_basis_type(qmckl_context context, const char basis_type) {
  const int32_t mask = 1;
  qmckl_exit_code rc = pre(context, mask);
  if (rc != QMCKL_SUCCESS) return rc;
  if (basis_type != 'G' && basis_type != 'S')
    return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_set_ao_basis_type", NULL);
  ctx_of(context)->ao_basis.type = basis_type;
  return post(context, mask);
}

qmckl_exit_code qmckl_set_ao_basis_shell_num(qmckl_context context, const int64_t shell_num) {
  const int32_t mask = 1 << 1;
  qmckl_exit_code rc = pre(context, mask);
  if (rc != QMCKL_SUCCESS) return rc;
  if (shell_num <= 0) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_set_ao_basis_shell_num", "shell_num <= 0");
  const int64_t prim_num = ctx_of(context)->ao_basis.prim_num;
  if (0 < prim_num && prim_num < shell_num)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_set_ao_basis_shell_num", "shell_num > prim_num");
  ctx_of(context)->ao_basis.shell_num = shell_num;
  return post(context, mask);
}

qmckl_exit_code qmckl_set_ao_basis_prim_num(qmckl_context context, const int64_t prim_num) {
  const int32_t mask = 1 << 2;
  qmckl_exit_code rc = pre(context, mask);
  if (rc != QMCKL_SUCCESS) return rc;
  if (prim_num <= 0) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_set_ao_basis_shell_num", "prim_num must be positive");
  const int64_t shell_num = ctx_of(context)->ao_basis.shell_num;
  if (shell_num <= 0) return qmckl_failwith(context, QMCKL_FAILURE, "qmckl_set_ao_basis_shell_num", "shell_num is not set");
  if (prim_num < shell_num) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_set_ao_basis_shell_num", "prim_num < shell_num");
  ctx_of(context)->ao_basis.prim_num = prim_num;
  return post(context, mask);
}

qmckl_exit_code qmckl_set_ao_basis_nucleus_shell_num(qmckl_context context, const int64_t* nucleus_shell_num, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return qmckl_failwith(context, QMCKL_NULL_CONTEXT, "qmckl_set_ao_*", NULL);
  return set_array(context, 1 << 3, "qmckl_set_ao_basis_nucleus_shell_num", ctx_of(context)->nucleus.num,
                   "shell_num is not set", nucleus_shell_num, size_max, ctx_of(context)->ao_basis.nucleus_shell_num);
}

qmckl_exit_code qmckl_set_ao_basis_nucleus_index(qmckl_context context, const int64_t* nucleus_index, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return qmckl_failwith(context, QMCKL_NULL_CONTEXT, "qmckl_set_ao_*", NULL);
  return set_array(context, 1 << 4, "qmckl_set_ao_basis_nucleus_index", ctx_of(context)->nucleus.num,
                   "nucl_num is not set", nucleus_index, size_max, ctx_of(context)->ao_basis.nucleus_index,
                   QMCKL_FAILURE, QMCKL_FAILURE);
}

qmckl_exit_code qmckl_set_ao_basis_shell_ang_mom(qmckl_context context, const int32_t* shell_ang_mom, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return qmckl_failwith(context, QMCKL_NULL_CONTEXT, "qmckl_set_ao_*", NULL);
  return set_array(context, 1 << 5, "qmckl_set_ao_basis_shell_ang_mom", ctx_of(context)->ao_basis.shell_num,
                   "shell_num is not set", shell_ang_mom, size_max, ctx_of(context)->ao_basis.shell_ang_mom);
}

qmckl_exit_code qmckl_set_ao_basis_shell_prim_num(qmckl_context context, const int64_t* shell_prim_num, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return qmckl_failwith(context, QMCKL_NULL_CONTEXT, "qmckl_set_ao_*", NULL);
  return set_array(context, 1 << 6, "qmckl_set_ao_basis_shell_prim_num", ctx_of(context)->ao_basis.shell_num,
                   "shell_num is not set", shell_prim_num, size_max, ctx_of(context)->ao_basis.shell_prim_num);
}

qmckl_exit_code qmckl_set_ao_basis_shell_prim_index(qmckl_context context, const int64_t* shell_prim_index, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return qmckl_failwith(context, QMCKL_NULL_CONTEXT, "qmckl_set_ao_*", NULL);
  return set_array(context, 1 << 7, "qmckl_set_ao_basis_shell_prim_index", ctx_of(context)->ao_basis.shell_num,
                   "shell_num is not set", shell_prim_index, size_max, ctx_of(context)->ao_basis.shell_prim_index);
}

qmckl_exit_code qmckl_set_ao_basis_shell_factor(qmckl_context context, const double* shell_factor, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return qmckl_failwith(context, QMCKL_NULL_CONTEXT, "qmckl_set_ao_*", NULL);
  return set_array(context, 1 << 8, "qmckl_set_ao_basis_shell_factor", ctx_of(context)->ao_basis.shell_num,
                   "shell_num is not set", shell_factor, size_max, ctx_of(context)->ao_basis.shell_factor);
}

qmckl_exit_code qmckl_set_ao_basis_exponent(qmckl_context context, const double* exponent, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return qmckl_failwith(context, QMCKL_NULL_CONTEXT, "qmckl_set_ao_*", NULL);
  return set_array(context, 1 << 9, "qmckl_set_ao_basis_exponent", ctx_of(context)->ao_basis.prim_num,
                   "prim_num is not set", exponent, size_max, ctx_of(context)->ao_basis.exponent);
}

qmckl_exit_code qmckl_set_ao_basis_coefficient(qmckl_context context, const double* coefficient, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return qmckl_failwith(context, QMCKL_NULL_CONTEXT, "qmckl_set_ao_*", NULL);
  return set_array(context, 1 << 10, "qmckl_set_ao_basis_coefficient", ctx_of(context)->ao_basis.prim_num,
                   "prim_num is not set", coefficient, size_max, ctx_of(context)->ao_basis.coefficient);
}

qmckl_exit_code qmckl_set_ao_basis_prim_factor(qmckl_context context, const double* prim_factor, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return qmckl_failwith(context, QMCKL_NULL_CONTEXT, "qmckl_set_ao_*", NULL);
  return set_array(context, 1 << 11, "qmckl_set_ao_basis_prim_factor", ctx_of(context)->ao_basis.prim_num,
                   "prim_num is not set", prim_factor, size_max, ctx_of(context)->ao_basis.prim_factor);
}

qmckl_exit_code qmckl_set_ao_basis_ao_num(qmckl_context context, const int64_t ao_num) {
  const int32_t mask = 1 << 12;
  qmckl_exit_code rc = pre(context, mask);
  if (rc != QMCKL_SUCCESS) return rc;
  if (ao_num <= 0) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_set_ao_basis_shell_num", "ao_num must be positive");
  const int64_t shell_num = ctx_of(context)->ao_basis.shell_num;
  if (shell_num <= 0) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_set_ao_basis_shell_num", "shell_num is not set");
  if (ao_num < shell_num) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_set_ao_basis_shell_num", "ao_num < shell_num");
  ctx_of(context)->ao_basis.ao_num = ao_num;
  return post(context, mask);
}

qmckl_exit_code qmckl_set_ao_basis_ao_factor(qmckl_context context, const double* ao_factor, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return qmckl_failwith(context, QMCKL_NULL_CONTEXT, "qmckl_set_ao_*", NULL);
  return set_array(context, 1 << 13, "qmckl_set_ao_basis_ao_factor", ctx_of(context)->ao_basis.ao_num,
                   "ao_num is not set", ao_factor, size_max, ctx_of(context)->ao_basis.ao_factor);
}

qmckl_exit_code qmckl_set_ao_basis_r_power(qmckl_context context, const int32_t* r_power, const int64_t size_max) {
  // optional field: no mask (org/qmckl_ao.org:1199-1262)
  qmckl_exit_code rc = pre(context, 0);
  if (rc != QMCKL_SUCCESS) return rc;
  Context* ctx = ctx_of(context);
  const int64_t shell_num = ctx->ao_basis.shell_num;
  if (shell_num == 0) return qmckl_failwith(context, QMCKL_FAILURE, "qmckl_set_ao_basis_r_power", "shell_num is not set");
  if (size_max < shell_num) return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_set_ao_basis_r_power", "input array too small");
  if (r_power == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_set_ao_basis_r_power", "NULL pointer");
  ctx->ao_basis.r_power.assign(r_power, r_power + shell_num);
  ctx->ao_basis.r_power_set = true;
  return post(context, 0);
}

qmckl_exit_code qmckl_set_ao_basis_cartesian(qmckl_context context, const bool cartesian) {
  // The reference reuses mask bit 1 here (org/qmckl_ao.org:1275), so calling it
  // after qmckl_set_ao_basis_type returns QMCKL_ALREADY_SET; kept as is.
  const int32_t mask = 1;
  qmckl_exit_code rc = pre(context, mask);
  if (rc != QMCKL_SUCCESS) return rc;
  ctx_of(context)->ao_basis.ao_cartesian = cartesian;
  return post(context, mask);
}

/* ----------------------------------------------------------------- getters */

qmckl_exit_code qmckl_get_ao_basis_type(const qmckl_context context, char* const basis_type) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT)
    return qmckl_failwith(context, QMCKL_INVALID_CONTEXT, "qmckl_get_ao_basis_type", NULL);
  Context* ctx = ctx_of(context);
  if (ctx->ao_basis.uninitialized & 1) return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_get_ao_basis_type", NULL);
  if (basis_type == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_ao_basis_type", "NULL pointer");
  *basis_type = ctx->ao_basis.type;
  return QMCKL_SUCCESS;
}

#define QB_SCALAR_GETTER(NAME, FIELD, MASK)                                                        \
  qmckl_exit_code qmckl_get_ao_basis_##NAME(const qmckl_context context, int64_t* const out) {     \
    if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT)                                        \
      return qmckl_failwith(context, QMCKL_INVALID_CONTEXT, "qmckl_get_ao_basis_" #NAME, NULL);    \
    Context* ctx = ctx_of(context);                                                                \
    if (ctx->ao_basis.uninitialized & (MASK))                                                      \
      return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_get_ao_basis_" #NAME, NULL);       \
    if (out == nullptr)                                                                            \
      return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_ao_basis_" #NAME, "NULL pointer"); \
    *out = ctx->ao_basis.FIELD;                                                                    \
    return QMCKL_SUCCESS;                                                                          \
  }
QB_SCALAR_GETTER(shell_num, shell_num, 1 << 1)
QB_SCALAR_GETTER(prim_num, prim_num, 1 << 2)
QB_SCALAR_GETTER(ao_num, ao_num, 1 << 12)
#undef QB_SCALAR_GETTER

qmckl_exit_code qmckl_get_ao_basis_nucleus_shell_num(const qmckl_context context, int64_t* const v, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  Context* c = ctx_of(context);
  return get_array(context, 1 << 3, "qmckl_get_ao_basis_nucleus_shell_num", v, size_max, c->nucleus.num,
                   c->ao_basis.nucleus_shell_num, "Array too small. Expected nucl_num");
}
qmckl_exit_code qmckl_get_ao_basis_nucleus_index(const qmckl_context context, int64_t* const v, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  Context* c = ctx_of(context);
  return get_array(context, 1 << 4, "qmckl_get_ao_basis_nucleus_index", v, size_max, c->nucleus.num,
                   c->ao_basis.nucleus_index, "Array too small. Expected nucl_num");
}
qmckl_exit_code qmckl_get_ao_basis_r_power(const qmckl_context context, int32_t* const v, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  Context* c = ctx_of(context);
  // The reference requires the whole basis to be set (org/qmckl_ao.org:1734-1740).
  if (c->ao_basis.uninitialized != 0) return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_get_ao_basis_r_power", NULL);
  return get_array(context, 0, "qmckl_get_ao_basis_r_power", v, size_max, c->ao_basis.shell_num,
                   c->ao_basis.r_power, "Array too small. Expected shell_num");
}
qmckl_exit_code qmckl_get_ao_basis_shell_ang_mom(const qmckl_context context, int32_t* const v, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  Context* c = ctx_of(context);
  return get_array(context, 1 << 5, "qmckl_get_ao_basis_shell_ang_mom", v, size_max, c->ao_basis.shell_num,
                   c->ao_basis.shell_ang_mom, "Array too small. Expected shell_num");
}
qmckl_exit_code qmckl_get_ao_basis_shell_prim_num(const qmckl_context context, int64_t* const v, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  Context* c = ctx_of(context);
  return get_array(context, 1 << 6, "qmckl_get_ao_basis_shell_prim_num", v, size_max, c->ao_basis.shell_num,
                   c->ao_basis.shell_prim_num, "Array too small. Expected shell_num");
}
qmckl_exit_code qmckl_get_ao_basis_shell_prim_index(const qmckl_context context, int64_t* const v, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  Context* c = ctx_of(context);
  return get_array(context, 1 << 7, "qmckl_get_ao_basis_shell_prim_index", v, size_max, c->ao_basis.shell_num,
                   c->ao_basis.shell_prim_index, "Array too small. Expected shell_num");
}
qmckl_exit_code qmckl_get_ao_basis_shell_factor(const qmckl_context context, double* const v, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  Context* c = ctx_of(context);
  return get_array(context, 1 << 8, "qmckl_get_ao_basis_shell_factor", v, size_max, c->ao_basis.shell_num,
                   c->ao_basis.shell_factor, "Array too small. Expected shell_num");
}
qmckl_exit_code qmckl_get_ao_basis_exponent(const qmckl_context context, double* const v, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  Context* c = ctx_of(context);
  return get_array(context, 1 << 9, "qmckl_get_ao_basis_exponent", v, size_max, c->ao_basis.prim_num,
                   c->ao_basis.exponent, "Array too small. Expected prim_num");
}
qmckl_exit_code qmckl_get_ao_basis_coefficient(const qmckl_context context, double* const v, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  Context* c = ctx_of(context);
  return get_array(context, 1 << 10, "qmckl_get_ao_basis_coefficient", v, size_max, c->ao_basis.prim_num,
                   c->ao_basis.coefficient, "Array too small. Expected prim_num");
}
qmckl_exit_code qmckl_get_ao_basis_prim_factor(const qmckl_context context, double* const v, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  Context* c = ctx_of(context);
  return get_array(context, 1 << 11, "qmckl_get_ao_basis_prim_factor", v, size_max, c->ao_basis.prim_num,
                   c->ao_basis.prim_factor, "Array too small. Expected prim_num");
}
qmckl_exit_code qmckl_get_ao_basis_ao_factor(const qmckl_context context, double* const v, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  Context* c = ctx_of(context);
  return get_array(context, 1 << 13, "qmckl_get_ao_basis_ao_factor", v, size_max, c->ao_basis.ao_num,
                   c->ao_basis.ao_factor, "Array too small. Expected ao_num");
}
qmckl_exit_code qmckl_get_ao_basis_cartesian(const qmckl_context context, bool* const cartesian) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  if (cartesian == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_ao_basis_cartesian", "NULL pointer");
  *cartesian = ctx_of(context)->ao_basis.ao_cartesian;
  return QMCKL_SUCCESS;
}

bool qmckl_ao_basis_provided(const qmckl_context context) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return false;
  return ctx_of(context)->ao_basis.provided;
}

/* ------------------------------------------------- computed array getters */

qmckl_exit_code qmckl_get_ao_basis_primitive_vgl(qmckl_context context, double* const primitive_vgl, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT)
    return qmckl_failwith(context, QMCKL_INVALID_CONTEXT, "qmckl_get_ao_basis_primitive_vgl", NULL);
  if (size_max <= 0) return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_get_ao_basis_primitive_vgl", "size_max <= 0");
  Context* ctx = ctx_of(context);
  if (!ctx->ao_basis.provided) return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_provide_ao_basis_primitive_vgl", NULL);
  const int64_t sze = ctx->ao_basis.prim_num * 5 * ctx->point.num;
  if (size_max < sze) return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_get_ao_basis_primitive_vgl", "input array too small");
  if (primitive_vgl == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_ao_basis_primitive_vgl", "NULL pointer");
  return dev_provide_primitive_vgl(context, primitive_vgl);
}

qmckl_exit_code qmckl_get_ao_basis_shell_vgl(qmckl_context context, double* const shell_vgl, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT)
    return qmckl_failwith(context, QMCKL_INVALID_CONTEXT, "qmckl_get_ao_basis_shell_vgl", NULL);
  Context* ctx = ctx_of(context);
  if (!ctx->ao_basis.provided) return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_provide_ao_basis_shell_vgl", NULL);
  const int64_t sze = ctx->ao_basis.shell_num * 5 * ctx->point.num;
  if (size_max < sze) return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_get_ao_basis_shell_vgl", "input array too small");
  if (shell_vgl == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_ao_basis_shell_vgl", "NULL pointer");
  return dev_provide_shell_vgl(context, shell_vgl);
}

qmckl_exit_code qmckl_get_ao_basis_ao_vgl(qmckl_context context, double* const ao_vgl, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT)
    return qmckl_failwith(context, QMCKL_INVALID_CONTEXT, "qmckl_get_ao_basis_ao_vgl", NULL);
  Context* ctx = ctx_of(context);
  if (!ctx->ao_basis.provided) return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_provide_ao_basis_ao_vgl", NULL);
  const int64_t sze = ctx->ao_basis.ao_num * 5 * ctx->point.num;
  if (size_max < sze) return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_get_ao_basis_ao_vgl", "input array too small");
  if (ao_vgl == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_ao_basis_ao_vgl", "NULL pointer");
  return dev_provide_ao_vgl(context, ao_vgl);
}

qmckl_exit_code qmckl_get_ao_basis_ao_vgl_inplace(qmckl_context context, double* const ao_vgl, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT)
    return qmckl_failwith(context, QMCKL_INVALID_CONTEXT, "qmckl_get_ao_basis_ao_vgl", NULL);
  Context* ctx = ctx_of(context);
  const int64_t sze = ctx->ao_basis.ao_num * 5 * ctx->point.num;
  if (size_max < sze) return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_get_ao_basis_ao_vgl", "input array too small");
  // The reference touches the context and computes straight into the caller's
  // array (org/qmckl_ao.org:3631-3655); the touch forces the recomputation.
  qmckl_exit_code rc = qmckl_context_touch(context);
  if (rc != QMCKL_SUCCESS) return rc;
  if (!ctx->ao_basis.provided) return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_provide_ao_basis_ao_vgl", NULL);
  if (ao_vgl == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_ao_basis_ao_vgl", "NULL pointer");
  return dev_provide_ao_vgl(context, ao_vgl);
}

qmckl_exit_code qmckl_get_ao_basis_ao_hessian(qmckl_context context, double* const ao_hessian, const int64_t size_max) {
  // org/qmckl_ao.org:9400-9440
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_NULL_CONTEXT;
  Context* ctx = ctx_of(context);
  if (!ctx->ao_basis.provided) return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_provide_ao_basis_ao_hessian", NULL);
  const int64_t sze = ctx->ao_basis.ao_num * 4 * 3 * ctx->point.num;
  if (size_max < sze) return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_get_ao_basis_ao_hessian", "input array too small");
  if (ao_hessian == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_ao_basis_ao_hessian", "NULL pointer");
  return dev_provide_ao_hessian(context, ao_hessian);
}

qmckl_exit_code qmckl_get_ao_basis_ao_value(qmckl_context context, double* const ao_value, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT)
    return qmckl_failwith(context, QMCKL_INVALID_CONTEXT, "qmckl_get_ao_basis_ao_value", NULL);
  Context* ctx = ctx_of(context);
  if (!ctx->ao_basis.provided) return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_provide_ao_basis_ao_value", NULL);
  const int64_t sze = ctx->ao_basis.ao_num * ctx->point.num;
  if (size_max < sze) return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_get_ao_basis_ao_value", "input array too small");
  if (ao_value == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_ao_basis_ao_value", "NULL pointer");
  return dev_provide_ao_value(context, ao_value);
}

qmckl_exit_code qmckl_get_ao_basis_ao_value_inplace(qmckl_context context, double* const ao_value, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT)
    return qmckl_failwith(context, QMCKL_INVALID_CONTEXT, "qmckl_get_ao_basis_ao_value", NULL);
  Context* ctx = ctx_of(context);
  const int64_t sze = ctx->ao_basis.ao_num * ctx->point.num;
  if (size_max < sze) return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_get_ao_basis_ao_value", "input array too small");
  qmckl_exit_code rc = qmckl_context_touch(context);
  if (rc != QMCKL_SUCCESS) return rc;
  if (!ctx->ao_basis.provided) return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_provide_ao_basis_ao_value", NULL);
  if (ao_value == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_ao_basis_ao_value", "NULL pointer");
  return dev_provide_ao_value(context, ao_value);
}

}  // extern "C"
