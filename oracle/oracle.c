/*
 * CPU oracle for the orbital-evaluation path -- TEST INFRASTRUCTURE ONLY.
 * See oracle.h for what it restates and how it is pinned.  Every function
 * cites the reference file:line whose algorithm it follows.  Nothing in the
 * product library links this file.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

struct oracle_basis {
  int64_t nucl_num, shell_num, prim_num, ao_num;
  int64_t* nucleus_index;
  int64_t* nucleus_shell_num;
  int32_t* shell_ang_mom;
  int64_t* shell_prim_num;
  int64_t* shell_prim_index;
  double*  exponent;
  double*  coef_norm;         /* coefficient * prim_factor * shell_factor */
  double*  ao_factor;
  double*  nucleus_range;     /* max over primitives of 1/a  (r_power = 0) */
  int32_t* nucleus_max_l;
  int64_t* ao_index;          /* first AO of each shell */
  /* per-nucleus sorted, de-duplicated exponent tables */
  int64_t  prim_max, shell_max;
  int64_t* nprim;             /* [nucl] unique exponents per nucleus */
  double*  expo_nuc;          /* [nucl][prim_max] */
  double*  coef_nuc;          /* [nucl][shell_max][prim_max] */
};

static int64_t lstart(int l) { return (int64_t)l * (l + 1) * (l + 2) / 6; }

/* Monomial tables hold every cartesian power of degree <= ORACLE_MAX_L
 * (120 monomials at l = 7); power tables pw[.][i + 2] = Y^i for
 * i = -2 .. ORACLE_MAX_L + 1 (the Hessian reads one power past lmax). */
#define ORACLE_NPOLY 120
#define ORACLE_NPW (ORACLE_MAX_L + 4)

double oracle_cutoff(int32_t precision) {
  /* org/qmckl_ao.org:7814: cutoff = log(2^(precision-1)) */
  return log((double)(((uint64_t)1) << (precision - 1)));
}

typedef struct { double expo; int64_t index; } expo_idx;

static int cmp_expo(const void* l, const void* r) {
  const expo_idx* a = (const expo_idx*)l;
  const expo_idx* b = (const expo_idx*)r;
  if (a->expo > b->expo) return 1;
  if (a->expo < b->expo) return -1;
  return 0;
}

/* qmckl_finalize_basis (org/qmckl_ao.org:2965-3226) and
 * qmckl_finalize_basis_hpc (org/qmckl_ao.org:3280-3410). */
oracle_basis* oracle_basis_create(const oracle_basis_in* in) {
  for (int64_t s = 0; s < in->shell_num; ++s)
    if (in->shell_ang_mom[s] < 0 || in->shell_ang_mom[s] > ORACLE_MAX_L) return NULL;
  oracle_basis* b = (oracle_basis*)calloc(1, sizeof(oracle_basis));
  const int64_t N = in->nucl_num, S = in->shell_num, Pn = in->prim_num, A = in->ao_num;
  b->nucl_num = N; b->shell_num = S; b->prim_num = Pn; b->ao_num = A;
#define DUP(dst, src, n, T) do { dst = (T*)malloc(sizeof(T) * (size_t)(n)); memcpy(dst, src, sizeof(T) * (size_t)(n)); } while (0)
  DUP(b->nucleus_index, in->nucleus_index, N, int64_t);
  DUP(b->nucleus_shell_num, in->nucleus_shell_num, N, int64_t);
  DUP(b->shell_ang_mom, in->shell_ang_mom, S, int32_t);
  DUP(b->shell_prim_num, in->shell_prim_num, S, int64_t);
  DUP(b->shell_prim_index, in->shell_prim_index, S, int64_t);
  DUP(b->exponent, in->exponent, Pn, double);
  DUP(b->ao_factor, in->ao_factor, A, double);
#undef DUP
  b->coef_norm = (double*)malloc(sizeof(double) * Pn);
  for (int64_t s = 0; s < S; ++s)
    for (int64_t p = in->shell_prim_index[s]; p < in->shell_prim_index[s] + in->shell_prim_num[s]; ++p)
      b->coef_norm[p] = in->coefficient[p] * in->prim_factor[p] * in->shell_factor[s];

  b->nucleus_max_l = (int32_t*)calloc(N, sizeof(int32_t));
  b->nucleus_range = (double*)calloc(N, sizeof(double));
  for (int64_t n = 0; n < N; ++n) {
    for (int64_t s = in->nucleus_index[n]; s < in->nucleus_index[n] + in->nucleus_shell_num[n]; ++s) {
      if (in->shell_ang_mom[s] > b->nucleus_max_l[n]) b->nucleus_max_l[n] = in->shell_ang_mom[s];
      for (int64_t p = in->shell_prim_index[s]; p < in->shell_prim_index[s] + in->shell_prim_num[s]; ++p) {
        const double range = 1.0 / in->exponent[p];  /* (r_power+1)/a with r_power = 0 (3203-3208) */
        if (range > b->nucleus_range[n]) b->nucleus_range[n] = range;
      }
    }
  }

  /* ao_index: org/qmckl_ao.org:7787-7805 */
  b->ao_index = (int64_t*)malloc(sizeof(int64_t) * (S + 1));
  {
    int64_t k = 0;
    for (int64_t n = 0; n < N; ++n)
      for (int64_t s = in->nucleus_index[n]; s < in->nucleus_index[n] + in->nucleus_shell_num[n]; ++s) {
        b->ao_index[s] = k;
        k += lstart(in->shell_ang_mom[s] + 1) - lstart(in->shell_ang_mom[s]);
      }
    b->ao_index[S] = A + 1;
  }

  /* HPC per-nucleus tables: sort exponents ascending, merge duplicates */
  int64_t prim_max = 0, shell_max = 0;
  for (int64_t n = 0; n < N; ++n) {
    int64_t np = 0;
    if (in->nucleus_shell_num[n] > shell_max) shell_max = in->nucleus_shell_num[n];
    for (int64_t s = in->nucleus_index[n]; s < in->nucleus_index[n] + in->nucleus_shell_num[n]; ++s)
      np += in->shell_prim_num[s];
    if (np > prim_max) prim_max = np;
  }
  if (prim_max < 1) prim_max = 1;
  if (shell_max < 1) shell_max = 1;
  b->prim_max = prim_max; b->shell_max = shell_max;
  b->nprim = (int64_t*)calloc(N, sizeof(int64_t));
  b->expo_nuc = (double*)calloc((size_t)N * prim_max, sizeof(double));
  b->coef_nuc = (double*)calloc((size_t)N * shell_max * prim_max, sizeof(double));
  expo_idx* ex = (expo_idx*)malloc(sizeof(expo_idx) * prim_max);
  double* orig = (double*)malloc(sizeof(double) * prim_max);
  double* row = (double*)malloc(sizeof(double) * prim_max);
  double* merged = (double*)malloc(sizeof(double) * prim_max);
  int64_t* uniq = (int64_t*)malloc(sizeof(int64_t) * prim_max);
  for (int64_t n = 0; n < N; ++n) {
    const int64_t s0 = in->nucleus_index[n], ns = in->nucleus_shell_num[n];
    int64_t np = 0;
    for (int64_t s = s0; s < s0 + ns; ++s)
      for (int64_t p = in->shell_prim_index[s]; p < in->shell_prim_index[s] + in->shell_prim_num[s]; ++p) {
        ex[np].expo = in->exponent[p];
        ex[np].index = np;
        ++np;
      }
    qsort(ex, (size_t)np, sizeof(expo_idx), cmp_expo);
    int64_t nu = 0;
    for (int64_t i = 0; i < np; ++i) {
      if (i > 0 && ex[i].expo != ex[i - 1].expo) ++nu;
      uniq[i] = nu;
    }
    if (np > 0) ++nu;
    int64_t pos = 0;
    for (int64_t j = 0; j < ns; ++j) {
      const int64_t s = s0 + j;
      for (int64_t i = 0; i < np; ++i) orig[i] = 0.0;
      for (int64_t p = in->shell_prim_index[s]; p < in->shell_prim_index[s] + in->shell_prim_num[s]; ++p)
        orig[pos++] = b->coef_norm[p];
      for (int64_t i = 0; i < np; ++i) row[i] = orig[ex[i].index];
      for (int64_t i = 0; i < np; ++i) merged[i] = 0.0;
      for (int64_t i = 0; i < np; ++i) merged[uniq[i]] += row[i];
      for (int64_t i = 0; i < nu; ++i) b->coef_nuc[(n * shell_max + j) * prim_max + i] = merged[i];
    }
    for (int64_t i = 0; i < np; ++i) b->expo_nuc[n * prim_max + uniq[i]] = ex[i].expo;
    b->nprim[n] = nu;
  }
  free(ex); free(orig); free(row); free(merged); free(uniq);
  return b;
}

void oracle_basis_destroy(oracle_basis* b) {
  if (!b) return;
  free(b->nucleus_index); free(b->nucleus_shell_num); free(b->shell_ang_mom);
  free(b->shell_prim_num); free(b->shell_prim_index); free(b->exponent);
  free(b->coef_norm); free(b->ao_factor); free(b->nucleus_range); free(b->nucleus_max_l);
  free(b->ao_index); free(b->nprim); free(b->expo_nuc); free(b->coef_nuc);
  free(b);
}

double oracle_nucleus_range(const oracle_basis* b, int64_t n) { return b->nucleus_range[n]; }
int64_t oracle_prim_per_nucleus(const oracle_basis* b, int64_t n) { return b->nprim[n]; }

/* Cartesian monomials of degree <= lmax with value/gradient/Laplacian, HPC
 * ordering and arithmetic (org/qmckl_ao.org:6624-6914 generic branch;
 * 8700-8760 for the l=1 and l=2 tables).  vgl[c][m], c = 0..4. */
static void poly_vgl_hpc(int lmax, double x, double y, double z, double vgl[5][ORACLE_NPOLY]) {
  const double shift = 1.e-20;
  for (int c = 0; c < 5; ++c)
    for (int m = 0; m < ORACLE_NPOLY; ++m) vgl[c][m] = 0.0;
  vgl[0][0] = 1.0;
  if (lmax == 0) return;
  vgl[0][1] = x + shift; vgl[0][2] = y + shift; vgl[0][3] = z + shift;
  vgl[1][1] = 1.0; vgl[2][2] = 1.0; vgl[3][3] = 1.0;
  if (lmax == 1) return;
  if (lmax == 2) {
    vgl[0][4] = x * x + shift; vgl[0][5] = x * y + shift; vgl[0][6] = x * z + shift;
    vgl[0][7] = y * y + shift; vgl[0][8] = y * z + shift; vgl[0][9] = z * z + shift;
    vgl[1][4] = x + x; vgl[1][5] = y; vgl[1][6] = z;
    vgl[2][5] = x; vgl[2][7] = y + y; vgl[2][8] = z;
    vgl[3][6] = x; vgl[3][8] = y; vgl[3][9] = z + z;
    vgl[4][4] = 2.0; vgl[4][7] = 2.0; vgl[4][9] = 2.0;
    return;
  }
  double pw[3][ORACLE_NPW];  /* pw[.][i+2] = coordinate^i, pw[.][0..2] = 1 */
  const double Y[3] = {x, y, z};
  for (int d = 0; d < 3; ++d) {
    pw[d][0] = pw[d][1] = pw[d][2] = 1.0;
    for (int i = 3; i <= lmax + 2; ++i) pw[d][i] = pw[d][i - 1] * Y[d];
  }
  int m = 4;
  double dd = 2.0;
  for (int d = 2; d <= lmax; ++d) {
    double da = dd;
    for (int a = d; a >= 0; --a) {
      double db = dd - da;
      for (int bb = d - a; bb >= 0; --bb) {
        const int c = d - a - bb;
        const double dc = dd - da - db;
        double xy = pw[0][a + 2] * pw[1][bb + 2];
        double yz = pw[1][bb + 2] * pw[2][c + 2];
        double xz = pw[0][a + 2] * pw[2][c + 2];
        vgl[0][m] = xy * pw[2][c + 2] + shift;
        xy *= dc; xz *= db; yz *= da;
        vgl[1][m] = pw[0][a + 1] * yz;
        vgl[2][m] = pw[1][bb + 1] * xz;
        vgl[3][m] = pw[2][c + 1] * xy;
        vgl[4][m] = (da - 1.) * pw[0][a] * yz + (db - 1.) * pw[1][bb] * xz + (dc - 1.) * pw[2][c] * xy;
        db -= 1.0;
        ++m;
      }
      da -= 1.0;
    }
    dd += 1.0;
  }
}

/* qmckl_compute_ao_vgl_hpc_gaussian (org/qmckl_ao.org:8601-8973). */
int oracle_ao_vgl_hpc(const oracle_basis* b, int32_t precision, int64_t point_num,
                      const double* coord, const double* nucl_coord,
                      double* ao_vgl, int32_t nthreads) {
  const double cutoff = oracle_cutoff(precision);
  const int double_precision = precision > 23;
  const int64_t N = b->nucl_num, A = b->ao_num, PM = b->prim_max, SM = b->shell_max;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
#endif
  {
    double* ar2 = (double*)malloc(sizeof(double) * PM);
    double (*em)[5] = (double (*)[5])malloc(sizeof(double) * 5 * PM);
    double (*ce)[5] = (double (*)[5])malloc(sizeof(double) * 5 * SM);
    double poly[5][ORACLE_NPOLY];
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 16)
#endif
    for (int64_t ip = 0; ip < point_num; ++ip) {
      double* out = ao_vgl + ip * 5 * A;
      memset(out, 0, sizeof(double) * 5 * A);
      const double ex = coord[ip], ey = coord[ip + point_num], ez = coord[ip + 2 * point_num];
      for (int64_t n = 0; n < N; ++n) {
        const double x = ex - nucl_coord[n];
        const double y = ey - nucl_coord[n + N];
        const double z = ez - nucl_coord[n + 2 * N];
        const double r2 = x * x + y * y + z * z;
        if (r2 > cutoff * b->nucleus_range[n]) continue;
        const int lmax = b->nucleus_max_l[n];
        poly_vgl_hpc(lmax, x, y, z, poly);
        int64_t nidx = 0;
        for (int64_t i = 0; i < b->nprim[n]; ++i) {
          const double v = b->expo_nuc[n * PM + i] * r2;
          if (v <= cutoff) { ar2[i] = v; ++nidx; } else break;
        }
        for (int64_t i = 0; i < nidx; ++i)
          em[i][0] = double_precision ? exp(-ar2[i]) : (double)expf(-(float)ar2[i]);
        for (int64_t i = 0; i < nidx; ++i) {
          double f = b->expo_nuc[n * PM + i] * em[i][0];
          f = -f - f;
          em[i][1] = f * x; em[i][2] = f * y; em[i][3] = f * z;
          em[i][4] = f * (3.0 - 2.0 * ar2[i]);
        }
        const int64_t s0 = b->nucleus_index[n], ns = b->nucleus_shell_num[n];
        for (int64_t j = 0; j < ns; ++j) {
          double acc[5] = {0., 0., 0., 0., 0.};
          const double* cj = b->coef_nuc + (n * SM + j) * PM;
          for (int64_t i = 0; i < b->nprim[n]; ++i) {
            if (cj[i] == 0.) continue;          /* sparse list of non-zero coefficients */
            if (i >= nidx) break;
            for (int c = 0; c < 5; ++c) acc[c] += cj[i] * em[i][c];
          }
          for (int c = 0; c < 5; ++c) ce[j][c] = acc[c];
        }
        for (int64_t s = s0; s < s0 + ns; ++s) {
          const double s1 = ce[s - s0][0];
          if (s1 == 0.0 || nidx == 0) continue;
          const double s2 = ce[s - s0][1], s3 = ce[s - s0][2], s4 = ce[s - s0][3], s5 = ce[s - s0][4];
          const int l = b->shell_ang_mom[s];
          const int64_t k = b->ao_index[s];
          const int64_t nm = lstart(l + 1) - lstart(l);
          const double* f = b->ao_factor + k;
          if (nm == 1) {
            out[k] = s1 * f[0]; out[A + k] = s2 * f[0]; out[2 * A + k] = s3 * f[0];
            out[3 * A + k] = s4 * f[0]; out[4 * A + k] = s5 * f[0];
            continue;
          }
          const int64_t i0 = lstart(l);
          for (int64_t il = 0; il < nm; ++il) {
            const double p1 = poly[0][i0 + il], p2 = poly[1][i0 + il], p3 = poly[2][i0 + il];
            const double p4 = poly[3][i0 + il], p5 = poly[4][i0 + il];
            out[k + il] = p1 * s1 * f[il];
            out[A + k + il] = (p2 * s1 + p1 * s2) * f[il];
            out[2 * A + k + il] = (p3 * s1 + p1 * s3) * f[il];
            out[3 * A + k + il] = (p4 * s1 + p1 * s4) * f[il];
            if (nm == 3)
              out[4 * A + k + il] = (p1 * s5 + 2.0 * (p2 * s2 + p3 * s3 + p4 * s4)) * f[il];
            else
              out[4 * A + k + il] = (p5 * s1 + p1 * s5 + 2.0 * (p2 * s2 + p3 * s3 + p4 * s4)) * f[il];
          }
        }
      }
    }
    free(ar2); free(em); free(ce);
  }
  return 0;
}

/* qmckl_compute_ao_value_hpc_gaussian (org/qmckl_ao.org:7822-8080).  The
 * value-only kernel uses the same radial contraction with the value column only. */
int oracle_ao_value_hpc(const oracle_basis* b, int32_t precision, int64_t point_num,
                        const double* coord, const double* nucl_coord,
                        double* ao_value, int32_t nthreads) {
  const double cutoff = oracle_cutoff(precision);
  const int double_precision = precision > 23;
  const int64_t N = b->nucl_num, A = b->ao_num, PM = b->prim_max, SM = b->shell_max;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
#endif
  {
    double* ar2 = (double*)malloc(sizeof(double) * PM);
    double* em = (double*)malloc(sizeof(double) * PM);
    double* ce = (double*)malloc(sizeof(double) * SM);
    double poly[5][ORACLE_NPOLY];
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 16)
#endif
    for (int64_t ip = 0; ip < point_num; ++ip) {
      double* out = ao_value + ip * A;
      memset(out, 0, sizeof(double) * A);
      const double ex = coord[ip], ey = coord[ip + point_num], ez = coord[ip + 2 * point_num];
      for (int64_t n = 0; n < N; ++n) {
        const double x = ex - nucl_coord[n];
        const double y = ey - nucl_coord[n + N];
        const double z = ez - nucl_coord[n + 2 * N];
        const double r2 = x * x + y * y + z * z;
        if (r2 > cutoff * b->nucleus_range[n]) continue;
        const int lmax = b->nucleus_max_l[n];
        poly_vgl_hpc(lmax, x, y, z, poly);
        int64_t nidx = 0;
        for (int64_t i = 0; i < b->nprim[n]; ++i) {
          const double v = b->expo_nuc[n * PM + i] * r2;
          if (v <= cutoff) { ar2[i] = v; ++nidx; } else break;
        }
        for (int64_t i = 0; i < nidx; ++i)
          em[i] = double_precision ? exp(-ar2[i]) : (double)expf(-(float)ar2[i]);
        const int64_t s0 = b->nucleus_index[n], ns = b->nucleus_shell_num[n];
        for (int64_t j = 0; j < ns; ++j) {
          double acc = 0.;
          const double* cj = b->coef_nuc + (n * SM + j) * PM;
          for (int64_t i = 0; i < b->nprim[n]; ++i) {
            if (cj[i] == 0.) continue;
            if (i >= nidx) break;
            acc += cj[i] * em[i];
          }
          ce[j] = acc;
        }
        for (int64_t s = s0; s < s0 + ns; ++s) {
          const double s1 = ce[s - s0];
          if (s1 == 0.0 || nidx == 0) continue;
          const int l = b->shell_ang_mom[s];
          const int64_t k = b->ao_index[s];
          const int64_t nm = lstart(l + 1) - lstart(l);
          const double* f = b->ao_factor + k;
          if (nm == 1) { out[k] = s1 * f[0]; continue; }
          for (int64_t il = 0; il < nm; ++il) out[k + il] = poly[0][lstart(l) + il] * s1 * f[il];
        }
      }
    }
    free(ar2); free(em); free(ce);
  }
  return 0;
}

/* qmckl_compute_ao_basis_primitive_gaussian_vgl (org/qmckl_ao.org:4468-4520).
 * prim_vgl[point][5][prim]; primitives beyond the cutoff are left at zero. */
int oracle_primitive_vgl(const oracle_basis* b, int32_t precision, int64_t point_num,
                         const double* coord, const double* nucl_coord, double* prim_vgl) {
  const double cutoff = oracle_cutoff(precision);
  const int64_t N = b->nucl_num, Pn = b->prim_num;
  memset(prim_vgl, 0, sizeof(double) * 5 * Pn * point_num);
  for (int64_t n = 0; n < N; ++n) {
    const int64_t s0 = b->nucleus_index[n];
    const int64_t p0 = b->shell_prim_index[s0];
    const int64_t p1 = (n + 1 < N) ? b->shell_prim_index[b->nucleus_index[n + 1]] : Pn;
    for (int64_t p = p0; p < p1; ++p)
      for (int64_t ip = 0; ip < point_num; ++ip) {
        const double x = coord[ip] - nucl_coord[n];
        const double y = coord[ip + point_num] - nucl_coord[n + N];
        const double z = coord[ip + 2 * point_num] - nucl_coord[n + 2 * N];
        const double r2 = x * x + y * y + z * z;
        const double ar2 = b->exponent[p] * r2;
        if (ar2 > cutoff) continue;
        const double v = exp(-ar2);
        const double two_a = -2.0 * b->exponent[p] * v;
        double* o = prim_vgl + ip * 5 * Pn;
        o[p] = v; o[Pn + p] = two_a * x; o[2 * Pn + p] = two_a * y; o[3 * Pn + p] = two_a * z;
        o[4 * Pn + p] = two_a * (3.0 - 2.0 * ar2);
      }
  }
  return 0;
}

/* qmckl_compute_ao_basis_shell_gaussian_vgl (org/qmckl_ao.org:4769-4868).
 * shell_vgl[point][5][shell]; shells of out-of-range nuclei are left at zero. */
int oracle_shell_vgl_doc(const oracle_basis* b, int32_t precision, int64_t point_num,
                         const double* coord, const double* nucl_coord, double* shell_vgl) {
  const double cutoff = oracle_cutoff(precision);
  const int64_t N = b->nucl_num, S = b->shell_num;
  memset(shell_vgl, 0, sizeof(double) * 5 * S * point_num);
  for (int64_t ip = 0; ip < point_num; ++ip) {
    for (int64_t n = 0; n < N; ++n) {
      const double x = coord[ip] - nucl_coord[n];
      const double y = coord[ip + point_num] - nucl_coord[n + N];
      const double z = coord[ip + 2 * point_num] - nucl_coord[n + 2 * N];
      const double r2 = x * x + y * y + z * z;
      if (r2 > cutoff * b->nucleus_range[n]) continue;
      for (int64_t s = b->nucleus_index[n]; s < b->nucleus_index[n] + b->nucleus_shell_num[n]; ++s) {
        double acc[5] = {0., 0., 0., 0., 0.};
        for (int64_t p = b->shell_prim_index[s]; p < b->shell_prim_index[s] + b->shell_prim_num[s]; ++p) {
          const double ar2 = b->exponent[p] * r2;
          if (ar2 > cutoff) continue;
          const double v = b->coef_norm[p] * exp(-ar2);
          const double two_a = -2.0 * b->exponent[p] * v;
          acc[0] += v; acc[1] += two_a * x; acc[2] += two_a * y; acc[3] += two_a * z;
          acc[4] += two_a * (3.0 - 2.0 * ar2);
        }
        double* o = shell_vgl + ip * 5 * S;
        for (int c = 0; c < 5; ++c) o[c * S + s] = acc[c];
      }
    }
  }
  return 0;
}

/* qmckl_ao_polynomial_vgl_doc (org/qmckl_ao.org:6233-6364): the 1e-20 shift is
 * added to the displacement before the powers are formed. vgl[c][m]. */
static void poly_vgl_doc(int lmax, const double X[3], const double R[3], double vgl[5][ORACLE_NPOLY]) {
  double Y[3], pw[3][ORACLE_NPW];  /* pw[.][i+2] = Y^i, i >= -2 */
  for (int i = 0; i < 3; ++i) Y[i] = (X[i] - R[i]) + 1.e-20;
  for (int c = 0; c < 5; ++c)
    for (int m = 0; m < ORACLE_NPOLY; ++m) vgl[c][m] = 0.0;
  vgl[0][0] = 1.0;
  if (lmax == 0) return;
  for (int d = 0; d < 3; ++d) {
    pw[d][0] = pw[d][1] = pw[d][2] = 1.0;
    for (int i = 1; i <= lmax; ++i) pw[d][i + 2] = pw[d][i + 1] * Y[d];
  }
  vgl[0][1] = pw[0][3]; vgl[1][1] = 1.0;
  vgl[0][2] = pw[1][3]; vgl[2][2] = 1.0;
  vgl[0][3] = pw[2][3]; vgl[3][3] = 1.0;
  int m = 4;
  double dd = 2.0;
  for (int d = 2; d <= lmax; ++d) {
    double da = dd;
    for (int a = d; a >= 0; --a) {
      double db = dd - da;
      for (int bb = d - a; bb >= 0; --bb) {
        const int c = d - a - bb;
        const double dc = dd - da - db;
        double xy = pw[0][a + 2] * pw[1][bb + 2];
        double yz = pw[1][bb + 2] * pw[2][c + 2];
        double xz = pw[0][a + 2] * pw[2][c + 2];
        vgl[0][m] = xy * pw[2][c + 2];
        xy = dc * xy; xz = db * xz; yz = da * yz;
        vgl[1][m] = pw[0][a + 1] * yz;
        vgl[2][m] = pw[1][bb + 1] * xz;
        vgl[3][m] = pw[2][c + 1] * xy;
        vgl[4][m] = (da - 1.) * pw[0][a] * yz + (db - 1.) * pw[1][bb] * xz + (dc - 1.) * pw[2][c] * xy;
        db -= 1.0;
        ++m;
      }
      da -= 1.0;
    }
    dd += 1.0;
  }
}

int oracle_poly_vgl(int32_t which, int32_t lmax, const double* X, const double* R, double* vgl) {
  if (lmax < 0 || lmax > ORACLE_MAX_L) return -1;
  double (*v)[ORACLE_NPOLY] = (double (*)[ORACLE_NPOLY])vgl;
  if (which == 1)
    poly_vgl_hpc(lmax, X[0] - R[0], X[1] - R[1], X[2] - R[2], v);
  else
    poly_vgl_doc(lmax, X, R, v);
  return (int)lstart(lmax + 1);
}

/* qmckl_compute_ao_vgl_doc (org/qmckl_ao.org:8438-8570) on top of the doc shell
 * VGL and doc polynomials. */
int oracle_ao_vgl_doc(const oracle_basis* b, int32_t precision, int64_t point_num,
                      const double* coord, const double* nucl_coord, double* ao_vgl) {
  const double cutoff = oracle_cutoff(precision);
  const int64_t N = b->nucl_num, S = b->shell_num, A = b->ao_num;
  double* sv = (double*)malloc(sizeof(double) * 5 * S * point_num);
  oracle_shell_vgl_doc(b, precision, point_num, coord, nucl_coord, sv);
  double poly[5][ORACLE_NPOLY];
  for (int64_t ip = 0; ip < point_num; ++ip) {
    double* out = ao_vgl + ip * 5 * A;
    memset(out, 0, sizeof(double) * 5 * A);
    const double X[3] = {coord[ip], coord[ip + point_num], coord[ip + 2 * point_num]};
    const double* s = sv + ip * 5 * S;
    for (int64_t n = 0; n < N; ++n) {
      const double R[3] = {nucl_coord[n], nucl_coord[n + N], nucl_coord[n + 2 * N]};
      const double x = X[0] - R[0], y = X[1] - R[1], z = X[2] - R[2];
      const double r2 = x * x + y * y + z * z;
      if (r2 > cutoff * b->nucleus_range[n]) continue;
      poly_vgl_doc(b->nucleus_max_l[n], X, R, poly);
      for (int64_t sh = b->nucleus_index[n]; sh < b->nucleus_index[n] + b->nucleus_shell_num[n]; ++sh) {
        const int l = b->shell_ang_mom[sh];
        int64_t k = b->ao_index[sh];
        for (int64_t il = lstart(l); il < lstart(l + 1); ++il, ++k) {
          const double f = b->ao_factor[k];
          out[k] = poly[0][il] * s[sh] * f;
          out[A + k] = (poly[1][il] * s[sh] + poly[0][il] * s[S + sh]) * f;
          out[2 * A + k] = (poly[2][il] * s[sh] + poly[0][il] * s[2 * S + sh]) * f;
          out[3 * A + k] = (poly[3][il] * s[sh] + poly[0][il] * s[3 * S + sh]) * f;
          out[4 * A + k] = (poly[4][il] * s[sh] + poly[0][il] * s[4 * S + sh] +
                            2.0 * (poly[1][il] * s[S + sh] + poly[2][il] * s[2 * S + sh] +
                                   poly[3][il] * s[3 * S + sh])) * f;
        }
      }
    }
  }
  free(sv);
  return 0;
}

/* qmckl_compute_mo_basis_mo_vgl_hpc (org/qmckl_mo.org:2015-2163): gather the
 * AOs with non-zero value, then 4-way unrolled axpy over the MOs. */
int oracle_mo_vgl(int64_t ao_num, int64_t mo_num, int64_t point_num,
                  const double* coefficient_t, const double* ao_vgl,
                  double* mo_vgl, int32_t nthreads) {
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
#endif
  {
    int64_t* idx = (int64_t*)malloc(sizeof(int64_t) * (ao_num + 1));
    double* av = (double*)malloc(sizeof(double) * 5 * (ao_num + 1));
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
    for (int64_t ip = 0; ip < point_num; ++ip) {
      double* v[5];
      const double* a[5];
      for (int c = 0; c < 5; ++c) {
        v[c] = mo_vgl + ip * 5 * mo_num + c * mo_num;
        a[c] = ao_vgl + ip * 5 * ao_num + c * ao_num;
      }
      memset(v[0], 0, sizeof(double) * 5 * mo_num);
      int64_t nidx = 0;
      for (int64_t k = 0; k < ao_num; ++k)
        if (a[0][k] != 0.) {
          idx[nidx] = k;
          for (int c = 0; c < 5; ++c) av[c * ao_num + nidx] = a[c][k];
          ++nidx;
        }
      int64_t n = 0;
      for (n = 0; n < nidx - 4; n += 4) {
        const double* c1 = coefficient_t + idx[n] * mo_num;
        const double* c2 = coefficient_t + idx[n + 1] * mo_num;
        const double* c3 = coefficient_t + idx[n + 2] * mo_num;
        const double* c4 = coefficient_t + idx[n + 3] * mo_num;
        for (int c = 0; c < 5; ++c) {
          const double a1 = av[c * ao_num + n], a2 = av[c * ao_num + n + 1];
          const double a3 = av[c * ao_num + n + 2], a4 = av[c * ao_num + n + 3];
          double* vc = v[c];
          for (int64_t i = 0; i < mo_num; ++i)
            vc[i] = vc[i] + c1[i] * a1 + c2[i] * a2 + c3[i] * a3 + c4[i] * a4;
        }
      }
      for (int64_t m = n; m < nidx; ++m) {
        const double* ck = coefficient_t + idx[m] * mo_num;
        for (int c = 0; c < 5; ++c) {
          const double a1 = av[c * ao_num + m];
          double* vc = v[c];
          for (int64_t i = 0; i < mo_num; ++i) vc[i] = vc[i] + ck[i] * a1;
        }
      }
    }
    free(idx); free(av);
  }
  return 0;
}

/* qmckl_compute_mo_basis_mo_value_hpc (org/qmckl_mo.org:1517-1620). */
int oracle_mo_value(int64_t ao_num, int64_t mo_num, int64_t point_num,
                    const double* coefficient_t, const double* ao_value,
                    double* mo_value, int32_t nthreads) {
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
#endif
  {
    int64_t* idx = (int64_t*)malloc(sizeof(int64_t) * (ao_num + 1));
    double* av = (double*)malloc(sizeof(double) * (ao_num + 1));
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
    for (int64_t ip = 0; ip < point_num; ++ip) {
      double* v = mo_value + ip * mo_num;
      const double* a = ao_value + ip * ao_num;
      memset(v, 0, sizeof(double) * mo_num);
      int64_t nidx = 0;
      for (int64_t k = 0; k < ao_num; ++k)
        if (a[k] != 0.) { idx[nidx] = k; av[nidx] = a[k]; ++nidx; }
      int64_t n = 0;
      for (n = 0; n < nidx - 8; n += 8) {
        const double* c[8];
        for (int j = 0; j < 8; ++j) c[j] = coefficient_t + idx[n + j] * mo_num;
        for (int64_t i = 0; i < mo_num; ++i)
          v[i] = v[i] + c[0][i] * av[n] + c[1][i] * av[n + 1] + c[2][i] * av[n + 2] +
                 c[3][i] * av[n + 3] + c[4][i] * av[n + 4] + c[5][i] * av[n + 5] +
                 c[6][i] * av[n + 6] + c[7][i] * av[n + 7];
      }
      for (int64_t m = n; m < nidx; ++m) {
        const double* ck = coefficient_t + idx[m] * mo_num;
        for (int64_t i = 0; i < mo_num; ++i) v[i] = v[i] + ck[i] * av[m];
      }
    }
    free(idx); free(av);
  }
  return 0;
}

/* ------------------------------------------------------------------ derivatives
 *
 * Second and third derivatives used by the nuclear-derivative checks.  The
 * reference builds them from the doc (Fortran) routines: shell Hessian
 * qmckl_compute_ao_basis_shell_gaussian_hessian (org/qmckl_ao.org:5480-5580),
 * polynomial Hessian qmckl_compute_ao_polynomial_hessian_doc (7113-7236), AO
 * Hessian qmckl_compute_ao_hessian_doc (9590-9720), and the orbital forces
 * qmckl_compute_forces_mo_value_doc / _mo_g / _mo_l
 * (org/qmckl_forces.org:5688-5800, 6132-6337, 6648-6772). */

/* shell_hessian[point][3][4][shell]: [d][m] = d_d d_m R for m < 3 and
 * [d][3] = d_d lap R (org/qmckl_ao.org:5530-5578).  Primitives with a r^2 >
 * cutoff are skipped one by one (no sort), as the reference does. */
int oracle_shell_hessian_doc(const oracle_basis* b, int32_t precision, int64_t point_num,
                             const double* coord, const double* nucl_coord, double* shell_hessian) {
  const double cutoff = oracle_cutoff(precision);
  const int64_t N = b->nucl_num, S = b->shell_num;
  memset(shell_hessian, 0, sizeof(double) * 12 * S * point_num);
  for (int64_t ip = 0; ip < point_num; ++ip) {
    double* o = shell_hessian + ip * 12 * S;
    for (int64_t n = 0; n < N; ++n) {
      const double xyz[3] = {coord[ip] - nucl_coord[n], coord[ip + point_num] - nucl_coord[n + N],
                             coord[ip + 2 * point_num] - nucl_coord[n + 2 * N]};
      const double r2 = xyz[0] * xyz[0] + xyz[1] * xyz[1] + xyz[2] * xyz[2];
      if (r2 > cutoff * b->nucleus_range[n]) continue;
      for (int64_t s = b->nucleus_index[n]; s < b->nucleus_index[n] + b->nucleus_shell_num[n]; ++s) {
        for (int64_t p = b->shell_prim_index[s]; p < b->shell_prim_index[s] + b->shell_prim_num[s]; ++p) {
          const double ar2 = b->exponent[p] * r2;
          if (ar2 > cutoff) continue;
          const double v = b->coef_norm[p] * exp(-ar2);
          const double two_a = 2.0 * b->exponent[p];
          for (int i = 0; i < 3; ++i) {
            for (int j = 0; j < 3; ++j) {
              double* h = &o[(j * 4 + i) * S + s];
              if (i == j) *h -= two_a * v;
              *h += two_a * two_a * xyz[i] * xyz[j] * v;
            }
            o[(i * 4 + 3) * S + s] += (5.0 * two_a * two_a * xyz[i] - two_a * two_a * two_a * r2 * xyz[i]) * v;
          }
        }
      }
    }
  }
  return 0;
}

/* hess[n][m][k] = d_k d_m P_n (m < 3), hess[n][3][k] = d_k lap P_n, with the
 * 1e-20 shift on the displacement (org/qmckl_ao.org:7113-7236). */
static void poly_hessian_doc(int lmax, const double X[3], const double R[3], double hess[ORACLE_NPOLY][4][3]) {
  double Y[3], pw[3][ORACLE_NPW];  /* pw[.][i+2] = Y^i for i >= -2 */
  for (int i = 0; i < 3; ++i) Y[i] = (X[i] - R[i]) + 1.e-20;
  memset(hess, 0, sizeof(double) * ORACLE_NPOLY * 4 * 3);
  if (lmax < 2) return;
  for (int d = 0; d < 3; ++d) {
    pw[d][0] = pw[d][1] = pw[d][2] = 1.0;
    for (int i = 1; i <= lmax; ++i) pw[d][i + 2] = pw[d][i + 1] * Y[d];
  }
#define PW(d, e) pw[d][(e) + 2]
  int n = 4;
  double dd = 2.0;
  for (int d = 2; d <= lmax; ++d) {
    double da = dd;
    for (int a = d; a >= 0; --a) {
      double db = dd - da;
      for (int bb = d - a; bb >= 0; --bb) {
        const int c = d - a - bb;
        const double dc = dd - da - db;
        double (*h)[3] = hess[n];
        h[0][0] = da * (da - 1.) * PW(0, a - 2) * PW(1, bb) * PW(2, c);
        h[1][1] = db * (db - 1.) * PW(0, a) * PW(1, bb - 2) * PW(2, c);
        h[2][2] = dc * (dc - 1.) * PW(0, a) * PW(1, bb) * PW(2, c - 2);
        h[1][0] = h[0][1] = da * db * PW(0, a - 1) * PW(1, bb - 1) * PW(2, c);
        h[2][0] = h[0][2] = da * dc * PW(0, a - 1) * PW(1, bb) * PW(2, c - 1);
        h[2][1] = h[1][2] = db * dc * PW(0, a) * PW(1, bb - 1) * PW(2, c - 1);
        h[3][0] = da * db * (db - 1.) * PW(0, a - 1) * PW(1, bb - 2) * PW(2, c) +
                  da * dc * (dc - 1.) * PW(0, a - 1) * PW(1, bb) * PW(2, c - 2);
        h[3][1] = db * da * (da - 1.) * PW(0, a - 2) * PW(1, bb - 1) * PW(2, c) +
                  db * dc * (dc - 1.) * PW(0, a) * PW(1, bb - 1) * PW(2, c - 2);
        h[3][2] = dc * da * (da - 1.) * PW(0, a - 2) * PW(1, bb) * PW(2, c - 1) +
                  dc * db * (db - 1.) * PW(0, a) * PW(1, bb - 2) * PW(2, c - 1);
        if (da > 2) h[3][0] += da * (da - 1.) * (da - 2.) * PW(0, a - 3) * PW(1, bb) * PW(2, c);
        if (db > 2) h[3][1] += db * (db - 1.) * (db - 2.) * PW(0, a) * PW(1, bb - 3) * PW(2, c);
        if (dc > 2) h[3][2] += dc * (dc - 1.) * (dc - 2.) * PW(0, a) * PW(1, bb) * PW(2, c - 3);
        db -= 1.0;
        ++n;
      }
      da -= 1.0;
    }
    dd += 1.0;
  }
#undef PW
}

/* ao_hessian[3][point][4][ao]: [i][p][j][k] = d_i d_j chi_k (j < 3) and
 * [i][p][3][k] = d_i lap chi_k, derivatives with respect to the electron
 * coordinates (org/qmckl_ao.org:9590-9720). */
int oracle_ao_hessian_doc(const oracle_basis* b, int32_t precision, int64_t point_num,
                          const double* coord, const double* nucl_coord, double* ao_hessian) {
  const double cutoff = oracle_cutoff(precision);
  const int64_t N = b->nucl_num, S = b->shell_num, A = b->ao_num;
  double* sv = (double*)malloc(sizeof(double) * 5 * S * point_num);
  double* sh = (double*)malloc(sizeof(double) * 12 * S * point_num);
  oracle_shell_vgl_doc(b, precision, point_num, coord, nucl_coord, sv);
  oracle_shell_hessian_doc(b, precision, point_num, coord, nucl_coord, sh);
  double poly[5][ORACLE_NPOLY], ph[ORACLE_NPOLY][4][3];
  for (int64_t ip = 0; ip < point_num; ++ip) {
    for (int i = 0; i < 3; ++i) memset(ao_hessian + (i * point_num + ip) * 4 * A, 0, sizeof(double) * 4 * A);
    const double X[3] = {coord[ip], coord[ip + point_num], coord[ip + 2 * point_num]};
    const double* s = sv + ip * 5 * S;
    const double* H = sh + ip * 12 * S;
    for (int64_t n = 0; n < N; ++n) {
      const double R[3] = {nucl_coord[n], nucl_coord[n + N], nucl_coord[n + 2 * N]};
      const double x = X[0] - R[0], y = X[1] - R[1], z = X[2] - R[2];
      const double r2 = x * x + y * y + z * z;
      if (r2 > cutoff * b->nucleus_range[n]) continue;
      poly_hessian_doc(b->nucleus_max_l[n], X, R, ph);
      poly_vgl_doc(b->nucleus_max_l[n], X, R, poly);
      for (int64_t shl = b->nucleus_index[n]; shl < b->nucleus_index[n] + b->nucleus_shell_num[n]; ++shl) {
        const int l = b->shell_ang_mom[shl];
        int64_t k = b->ao_index[shl];
        for (int64_t il = lstart(l); il < lstart(l + 1); ++il, ++k) {
          const double f = b->ao_factor[k];
          for (int i = 0; i < 3; ++i) {
            double* o = ao_hessian + (i * point_num + ip) * 4 * A;
            for (int j = 0; j < 3; ++j)
              o[j * A + k] = (ph[il][i][j] * s[shl] + poly[0][il] * H[(i * 4 + j) * S + shl] +
                              poly[j + 1][il] * s[(i + 1) * S + shl] + poly[i + 1][il] * s[(j + 1) * S + shl]) * f;
            double t = 0.0;
            for (int m = 0; m < 3; ++m)
              t += ph[il][i][m] * s[(m + 1) * S + shl] + poly[m + 1][il] * H[(i * 4 + m) * S + shl];
            o[3 * A + k] = (ph[il][3][i] * s[shl] + poly[0][il] * H[(i * 4 + 3) * S + shl] +
                            poly[4][il] * s[(i + 1) * S + shl] + poly[i + 1][il] * s[4 * S + shl] + 2.0 * t) * f;
          }
        }
      }
    }
  }
  free(sv); free(sh);
  return 0;
}

/* Gradient of L = sum_{p,c,i} W[p][c][i] mo_vgl[p][c][i] (W in the mo_vgl
 * layout [point][5][mo]).
 *   grad_nucl[a][n]  through the orbital forces of the reference:
 *       forces_mo_value[a][p][n][i] = -sum_{k on a} Ct(i,k) ao_vgl[p][1+n][k]
 *       forces_mo_g[a][n][p][m][i]  = -sum_{k on a} Ct(i,k) ao_hessian[n][p][m][k]
 *       forces_mo_l[a][n][p][i]     = -sum_{k on a} Ct(i,k) ao_hessian[n][p][3][k]
 *     (org/qmckl_forces.org:5688-5800, 6132-6337, 6648-6772), then contracted
 *     with W over (p, i) and the component;
 *   grad_coef[i][k]  = sum_{p,c} W[p][c][i] ao_vgl[p][c][k]  ([mo][ao], the
 *     qmckl_set_mo_basis_coefficient layout);
 *   grad_coord[n][p] = derivative with respect to the point coordinates
 *     (the same sums over all nuclei, opposite sign).
 * Any output pointer may be NULL. */
int oracle_mo_vgl_adjoint(const oracle_basis* b, int32_t precision, int64_t point_num, const double* coord,
                          const double* nucl_coord, int64_t mo_num, const double* coefficient,
                          const double* weight, double* grad_coef, double* grad_nucl, double* grad_coord) {
  const int64_t N = b->nucl_num, A = b->ao_num, M = mo_num, P = point_num;
  double* av = (double*)malloc(sizeof(double) * 5 * A * P);
  double* ah = (double*)malloc(sizeof(double) * 12 * A * P);
  oracle_ao_vgl_doc(b, precision, P, coord, nucl_coord, av);
  oracle_ao_hessian_doc(b, precision, P, coord, nucl_coord, ah);
  if (grad_coef) {
    memset(grad_coef, 0, sizeof(double) * M * A);
    for (int64_t p = 0; p < P; ++p)
      for (int c = 0; c < 5; ++c) {
        const double* w = weight + (p * 5 + c) * M;
        const double* a = av + (p * 5 + c) * A;
        for (int64_t i = 0; i < M; ++i) {
          const double wi = w[i];
          if (wi == 0.0) continue;
          double* g = grad_coef + i * A;
          for (int64_t k = 0; k < A; ++k) g[k] += wi * a[k];
        }
      }
  }
  if (grad_nucl) memset(grad_nucl, 0, sizeof(double) * 3 * N);
  if (grad_coord) memset(grad_coord, 0, sizeof(double) * 3 * P);
  double* fv = (double*)malloc(sizeof(double) * 3 * M);     /* forces_mo_value[a][p][.][.] */
  double* fg = (double*)malloc(sizeof(double) * 9 * M);     /* forces_mo_g[a][.][p][.][.]  */
  double* fl = (double*)malloc(sizeof(double) * 3 * M);     /* forces_mo_l[a][.][p][.]     */
  for (int64_t a = 0; a < N; ++a) {
    const int64_t s0 = b->nucleus_index[a], s1 = s0 + b->nucleus_shell_num[a];
    const int64_t k0 = s1 > s0 ? b->ao_index[s0] : 0;
    const int64_t k1 = s1 > s0 ? b->ao_index[s1 - 1] + (lstart(b->shell_ang_mom[s1 - 1] + 1) -
                                                         lstart(b->shell_ang_mom[s1 - 1])) : 0;
    for (int64_t p = 0; p < P; ++p) {
      memset(fv, 0, sizeof(double) * 3 * M);
      memset(fg, 0, sizeof(double) * 9 * M);
      memset(fl, 0, sizeof(double) * 3 * M);
      for (int64_t k = k0; k < k1; ++k) {
        const double* ck = coefficient;   /* Ct(i,k) = coefficient[i][k] */
        for (int n = 0; n < 3; ++n) {
          const double c1 = av[(p * 5 + 1 + n) * A + k];
          for (int64_t i = 0; i < M; ++i) fv[n * M + i] -= c1 * ck[i * A + k];
          const double* h = ah + (n * P + p) * 4 * A;
          for (int m = 0; m < 3; ++m) {
            const double hm = h[m * A + k];
            if (hm != 0.0)
              for (int64_t i = 0; i < M; ++i) fg[(n * 3 + m) * M + i] -= ck[i * A + k] * hm;
          }
          const double hl = h[3 * A + k];
          for (int64_t i = 0; i < M; ++i) fl[n * M + i] -= ck[i * A + k] * hl;
        }
      }
      for (int n = 0; n < 3; ++n) {
        double acc = 0.0;
        for (int64_t i = 0; i < M; ++i) {
          acc += weight[(p * 5 + 0) * M + i] * fv[n * M + i];
          for (int m = 0; m < 3; ++m) acc += weight[(p * 5 + 1 + m) * M + i] * fg[(n * 3 + m) * M + i];
          acc += weight[(p * 5 + 4) * M + i] * fl[n * M + i];
        }
        if (grad_nucl) grad_nucl[a * 3 + n] += acc;
        if (grad_coord) grad_coord[n * P + p] -= acc;
      }
    }
  }
  free(fv); free(fg); free(fl); free(av); free(ah);
  return 0;
}

/* Orbital forces as full tensors (derivatives with respect to the nuclear
 * coordinates), the reference's getters qmckl_get_forces_ao_value /
 * _mo_value / _mo_g / _mo_l (org/qmckl_forces.org:5129-5160, 5300-5345,
 * 5688-5800, 6132-6337, 6648-6772):
 *   forces_ao_value[a][p][n][k] = -ao_vgl[p][1+n][k]    (k on nucleus a, else 0)
 *   forces_mo_value[a][p][n][i] = -sum_{k on a} C[i][k] ao_vgl[p][1+n][k]
 *   forces_mo_g[a][n][p][m][i]  = -sum_{k on a} C[i][k] ao_hessian[n][p][m][k]
 *   forces_mo_l[a][n][p][i]     = -sum_{k on a} C[i][k] ao_hessian[n][p][3][k]
 * coefficient [mo][ao]; any output may be NULL. */
int oracle_forces(const oracle_basis* b, int32_t precision, int64_t point_num, const double* coord,
                  const double* nucl_coord, int64_t mo_num, const double* coefficient, double* fao,
                  double* fmv, double* fmg, double* fml) {
  const int64_t N = b->nucl_num, A = b->ao_num, M = mo_num, P = point_num;
  double* av = (double*)malloc(sizeof(double) * 5 * A * P);
  double* ah = (double*)malloc(sizeof(double) * 12 * A * P);
  oracle_ao_vgl_doc(b, precision, P, coord, nucl_coord, av);
  oracle_ao_hessian_doc(b, precision, P, coord, nucl_coord, ah);
  if (fao) memset(fao, 0, sizeof(double) * N * P * 3 * A);
  if (fmv) memset(fmv, 0, sizeof(double) * N * P * 3 * M);
  if (fmg) memset(fmg, 0, sizeof(double) * N * 3 * P * 3 * M);
  if (fml) memset(fml, 0, sizeof(double) * N * 3 * P * M);
  for (int64_t a = 0; a < N; ++a) {
    const int64_t s0 = b->nucleus_index[a], s1 = s0 + b->nucleus_shell_num[a];
    if (s1 <= s0) continue;
    const int64_t k0 = b->ao_index[s0];
    const int64_t k1 = b->ao_index[s1 - 1] + (lstart(b->shell_ang_mom[s1 - 1] + 1) - lstart(b->shell_ang_mom[s1 - 1]));
    for (int64_t p = 0; p < P; ++p)
      for (int n = 0; n < 3; ++n) {
        const double* g = av + (p * 5 + 1 + n) * A;
        const double* h = ah + (n * P + p) * 4 * A;
        for (int64_t k = k0; k < k1; ++k) {
          if (fao) fao[((a * P + p) * 3 + n) * A + k] = -g[k];
          for (int64_t i = 0; i < M; ++i) {
            const double c = coefficient[i * A + k];
            if (fmv) fmv[((a * P + p) * 3 + n) * M + i] -= c * g[k];
            if (fmg)
              for (int m = 0; m < 3; ++m) fmg[(((a * 3 + n) * P + p) * 3 + m) * M + i] -= c * h[m * A + k];
            if (fml) fml[((a * 3 + n) * P + p) * M + i] -= c * h[3 * A + k];
          }
        }
      }
  }
  free(av);
  free(ah);
  return 0;
}
