// The reference's standalone AO helper functions: powers of a coordinate,
// cartesian monomials with their gradients and Laplacians, and Gaussians with
// theirs, for one point.  They take no basis from the context (a null context
// is the only context error, as in the reference) and run on the host: a
// single point's monomials are a few hundred flops, below any launch cost.
// The GPU path computes the same monomials inside the AO kernels.
//
//   qmckl_ao_power                          org/qmckl_ao.org:5937-6026
//   qmckl_ao_gaussian_vgl                   org/qmckl_ao.org:3804-3910
//   qmckl_ao_polynomial_vgl[_doc]           org/qmckl_ao.org:6210-6364
//   qmckl_ao_polynomial_transp_vgl[_doc]    org/qmckl_ao.org:6467-6619
//   qmckl_ao_polynomial_transp_vgl_hpc      org/qmckl_ao.org:6624-6914
//
// Monomial order (all forms): degree d ascending; within a degree the power
// of x descending, then the power of y descending.  Derivative factors are
// carried as doubles (da, db, dc) and each product is formed in the order the
// reference forms it, so that values agree to the last bit with a build that
// does not contract a*b+c into fused multiply-adds.
#include <cmath>
#include <cstdint>
#include <vector>

#include "qmckl.h"

namespace {

constexpr double kShift = 1.e-20;
constexpr int32_t kMaxL = 1000;

inline int64_t npoly(int32_t lmax) { return (int64_t)(lmax + 1) * (lmax + 2) * (lmax + 3) / 6; }

// Where the three forms differ:
//  * displacement_shift: 1e-20 added to X - R before the powers (non-transposed doc form);
//  * value_shift: 1e-20 added to every value of degree >= 1 after the products (HPC form);
//  * layout: component c of monomial m at VGL[c * cs + m * ms].
struct Form {
  bool displacement_shift;
  bool value_shift;
  int64_t cs, ms;
};

void monomials(const Form& f, const double* X, const double* R, int32_t lmax, int64_t* n, int32_t* L,
               int64_t ldl, double* VGL) {
  auto V = [&](int c, int64_t m) -> double& { return VGL[c * f.cs + m * f.ms]; };
  auto set_l = [&](int64_t m, int32_t a, int32_t b, int32_t c) {
    L[m * ldl + 0] = a;
    L[m * ldl + 1] = b;
    L[m * ldl + 2] = c;
  };
  const double vs = f.value_shift ? kShift : 0.0;

  set_l(0, 0, 0, 0);
  V(0, 0) = 1.0;
  for (int c = 1; c < 5; ++c) V(c, 0) = 0.0;
  if (lmax == 0) {
    *n = 1;
    return;
  }

  double Y[3];
  for (int i = 0; i < 3; ++i) Y[i] = f.displacement_shift ? (X[i] - R[i]) + kShift : X[i] - R[i];

  // pw[d][i + 2] = Y[d]^i for i = -2 .. lmax, with the negative powers set
  // to 1 (they only ever multiply a zero derivative factor).
  std::vector<double> pw_store(3 * (size_t)(lmax + 3));
  double* pw[3];
  for (int d = 0; d < 3; ++d) {
    pw[d] = pw_store.data() + d * (size_t)(lmax + 3);
    pw[d][0] = pw[d][1] = pw[d][2] = 1.0;
    for (int32_t i = 1; i <= lmax; ++i) pw[d][i + 2] = pw[d][i + 1] * Y[d];
  }

  for (int m = 1; m <= 3; ++m) {
    set_l(m, m == 1, m == 2, m == 3);
    V(0, m) = pw[m - 1][3] + vs;
    for (int c = 1; c < 5; ++c) V(c, m) = (c == m) ? 1.0 : 0.0;
  }

  int64_t m = 4;
  double dd = 2.0;
  for (int32_t d = 2; d <= lmax; ++d) {
    double da = dd;
    for (int32_t a = d; a >= 0; --a) {
      double db = dd - da;
      for (int32_t b = d - a; b >= 0; --b) {
        const int32_t c = d - a - b;
        const double dc = dd - da - db;
        set_l(m, a, b, c);
        double xy = pw[0][a + 2] * pw[1][b + 2];
        double yz = pw[1][b + 2] * pw[2][c + 2];
        double xz = pw[0][a + 2] * pw[2][c + 2];
        V(0, m) = xy * pw[2][c + 2] + vs;
        xy = dc * xy;
        xz = db * xz;
        yz = da * yz;
        V(1, m) = pw[0][a + 1] * yz;
        V(2, m) = pw[1][b + 1] * xz;
        V(3, m) = pw[2][c + 1] * xy;
        V(4, m) = (da - 1.) * pw[0][a] * yz + (db - 1.) * pw[1][b] * xz + (dc - 1.) * pw[2][c] * xy;
        db -= 1.0;
        ++m;
      }
      da -= 1.0;
    }
    dd += 1.0;
  }
  *n = m;
}

// Argument checks shared by the three monomial forms, in the reference's
// order; pointer checks (which the reference leaves to an assert or to the
// caller) come last and name the argument's position.
qmckl_exit_code check_poly(qmckl_context context, const double* X, const double* R, int32_t lmax, int64_t* n,
                           int32_t* L, int64_t ldl, double* VGL, int64_t ldv, int64_t ldv_min) {
  if (context == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  // lmax above kMaxL (1.7e8 monomials) is refused rather than left to an
  // allocation or, near 2e6, an overflowing count; the reference's own
  // transposed doc form holds powers up to 21 only
  if (lmax < 0 || lmax > kMaxL) return QMCKL_INVALID_ARG_4;
  if (ldl < 3) return QMCKL_INVALID_ARG_7;
  if (ldv < ldv_min) return QMCKL_INVALID_ARG_9;
  if (X == nullptr) return QMCKL_INVALID_ARG_2;
  if (R == nullptr) return QMCKL_INVALID_ARG_3;
  if (n == nullptr) return QMCKL_INVALID_ARG_5;
  if (L == nullptr) return QMCKL_INVALID_ARG_6;
  if (VGL == nullptr) return QMCKL_INVALID_ARG_8;
  return QMCKL_SUCCESS;
}

}  // namespace

extern "C" {

qmckl_exit_code qmckl_ao_power(const qmckl_context context, const int64_t n, const double* X, const int32_t* LMAX,
                               double* const P, const int64_t ldp) {
  if (context == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  // The reference rejects n <= ldp (not n <= 0) with argument 2; kept as is.
  if (n <= ldp) return QMCKL_INVALID_ARG_2;
  if (X == nullptr) return QMCKL_INVALID_ARG_3;
  if (LMAX == nullptr) return QMCKL_INVALID_ARG_4;
  int32_t kmax = INT32_MIN;
  for (int64_t i = 0; i < n; ++i) kmax = LMAX[i] > kmax ? LMAX[i] : kmax;
  if (ldp < kmax) return QMCKL_INVALID_ARG_6;
  if (kmax <= 0) return QMCKL_INVALID_ARG_4;
  if (P == nullptr) return QMCKL_INVALID_ARG_5;
  for (int64_t i = 0; i < n; ++i) {
    double* p = P + i * ldp;
    p[0] = X[i];
    for (int32_t k = 1; k < LMAX[i]; ++k) p[k] = p[k - 1] * X[i];
  }
  return QMCKL_SUCCESS;
}

// The C prototype the reference's header generates for this function reads
// n, A and VGL as pointers; the function itself (Fortran, bind(C)) takes n by
// value, A as the exponents and VGL as the output, which is what a working
// caller passes and what is implemented here.
qmckl_exit_code qmckl_ao_gaussian_vgl(const qmckl_context context, const double* X, const double* R, const int64_t n,
                                      const double* A, double* const VGL, const int64_t ldv) {
  if (context == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  if (n <= 0) return QMCKL_INVALID_ARG_4;
  if (ldv < n) return QMCKL_INVALID_ARG_7;
  if (X == nullptr) return QMCKL_INVALID_ARG_2;
  if (R == nullptr) return QMCKL_INVALID_ARG_3;
  if (A == nullptr) return QMCKL_INVALID_ARG_5;
  if (VGL == nullptr) return QMCKL_INVALID_ARG_6;
  const double y0 = X[0] - R[0], y1 = X[1] - R[1], y2 = X[2] - R[2];
  const double r2 = y0 * y0 + y1 * y1 + y2 * y2;
  const double t = -2.0 * y0, u = -2.0 * y1, v = -2.0 * y2, r4 = 4.0 * r2;
  for (int64_t i = 0; i < n; ++i) {
    const double g = std::exp(-A[i] * r2);
    const double ag = A[i] * g;
    VGL[i] = g;
    VGL[ldv + i] = t * ag;
    VGL[2 * ldv + i] = u * ag;
    VGL[3 * ldv + i] = v * ag;
    VGL[4 * ldv + i] = (r4 * A[i] - 6.0) * ag;
  }
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_ao_polynomial_vgl_doc(const qmckl_context context, const double* X, const double* R,
                                            const int32_t lmax, int64_t* n, int32_t* const L, const int64_t ldl,
                                            double* const VGL, const int64_t ldv) {
  const qmckl_exit_code rc = check_poly(context, X, R, lmax, n, L, ldl, VGL, ldv, 5);
  if (rc != QMCKL_SUCCESS) return rc;
  monomials(Form{true, false, 1, ldv}, X, R, lmax, n, L, ldl, VGL);
  return QMCKL_SUCCESS;
}

// The reference routes the non-transposed form to its doc version in every
// build (org/qmckl_ao.org:6211-6228).
qmckl_exit_code qmckl_ao_polynomial_vgl(const qmckl_context context, const double* X, const double* R,
                                        const int32_t lmax, int64_t* n, int32_t* const L, const int64_t ldl,
                                        double* const VGL, const int64_t ldv) {
  return qmckl_ao_polynomial_vgl_doc(context, X, R, lmax, n, L, ldl, VGL, ldv);
}

qmckl_exit_code qmckl_ao_polynomial_transp_vgl_doc(const qmckl_context context, const double* X, const double* R,
                                                   const int32_t lmax, int64_t* n, int32_t* const L,
                                                   const int64_t ldl, double* const VGL, const int64_t ldv) {
  const qmckl_exit_code rc =
      check_poly(context, X, R, lmax, n, L, ldl, VGL, ldv, lmax < 0 || lmax > kMaxL ? 0 : npoly(lmax));
  if (rc != QMCKL_SUCCESS) return rc;
  monomials(Form{false, false, ldv, 1}, X, R, lmax, n, L, ldl, VGL);
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_ao_polynomial_transp_vgl_hpc(const qmckl_context context, const double* X, const double* R,
                                                   const int32_t lmax, int64_t* n, int32_t* const L,
                                                   const int64_t ldl, double* const VGL, const int64_t ldv) {
  const qmckl_exit_code rc =
      check_poly(context, X, R, lmax, n, L, ldl, VGL, ldv, lmax < 0 || lmax > kMaxL ? 0 : npoly(lmax));
  if (rc != QMCKL_SUCCESS) return rc;
  monomials(Form{false, true, ldv, 1}, X, R, lmax, n, L, ldl, VGL);
  return QMCKL_SUCCESS;
}

// The reference's production build (HAVE_HPC) routes the transposed form to
// the HPC version (org/qmckl_ao.org:6468-6484); so does this library.
qmckl_exit_code qmckl_ao_polynomial_transp_vgl(const qmckl_context context, const double* X, const double* R,
                                               const int32_t lmax, int64_t* n, int32_t* const L, const int64_t ldl,
                                               double* const VGL, const int64_t ldv) {
  return qmckl_ao_polynomial_transp_vgl_hpc(context, X, R, lmax, n, L, ldl, VGL, ldv);
}

}  // extern "C"
