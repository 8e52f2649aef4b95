/*
 * CPU oracle for the orbital-evaluation path (TEST INFRASTRUCTURE ONLY).
 *
 * This is a plain-C restatement of the reference's CPU algorithms for
 * AO VGL / AO value / MO VGL / MO value.  Only the tests, the smoke check and
 * the CPU-baseline leg of bench.py may load it, and only as the checker: the
 * product path (libqmckl_b200.so) never links, loads or calls it.
 *
 * Pinning: the restatement is checked against the golden vectors the reference
 * ships in its own unit tests for the CHBrClF fixture (primitive_vgl,
 * shell_vgl, ao_vgl, ao_value at 1e-14 absolute; org/qmckl_ao.org:4697-4712,
 * 5236-5252, 9355-9384, 8399-8405) and, where it was compiled here, against the
 * reference's own C HPC kernels built into oracle/_ref (oracle/build_ref.py).
 *
 * Arrays follow the reference's layouts:
 *   coord       double[3][point_num]   (x block, y block, z block; org/qmckl_point.org:105-112)
 *   nucl_coord  double[3][nucl_num]    (org/qmckl_nucleus.org:109-122)
 *   ao_vgl      double[point_num][5][ao_num]  (org/qmckl_ao.org:2944)
 *   mo_vgl      double[point_num][5][mo_num]  (org/qmckl_mo.org:132)
 */
#ifndef QMCKL_B200_ORACLE_H
#define QMCKL_B200_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Raw basis, exactly the arrays handed to the qmckl_set_ao_basis_* setters. */
typedef struct oracle_basis_in {
  int64_t nucl_num, shell_num, prim_num, ao_num;
  const int64_t* nucleus_index;      /* [nucl_num]  */
  const int64_t* nucleus_shell_num;  /* [nucl_num]  */
  const int32_t* shell_ang_mom;      /* [shell_num] */
  const int64_t* shell_prim_num;     /* [shell_num] */
  const int64_t* shell_prim_index;   /* [shell_num] */
  const double*  shell_factor;       /* [shell_num] */
  const double*  exponent;           /* [prim_num]  */
  const double*  coefficient;        /* [prim_num]  */
  const double*  prim_factor;        /* [prim_num]  */
  const double*  ao_factor;          /* [ao_num]    */
} oracle_basis_in;

typedef struct oracle_basis oracle_basis;  /* finalized tables (opaque) */

/* Largest shell angular momentum the oracle evaluates (k shells, l = 7,
 * the largest the reference's own polynomial tests exercise,
 * org/qmckl_ao.org:7042-7076). */
#define ORACLE_MAX_L 7

/* NULL when a shell has l < 0 or l > ORACLE_MAX_L. */
oracle_basis* oracle_basis_create(const oracle_basis_in* in);
void          oracle_basis_destroy(oracle_basis* b);
double        oracle_nucleus_range(const oracle_basis* b, int64_t inucl);
int64_t       oracle_prim_per_nucleus(const oracle_basis* b, int64_t inucl);

/* Screening threshold ln(2^(precision-1)) (org/qmckl_ao.org:7779-7816). */
double oracle_cutoff(int32_t precision);

/* Production (HAVE_HPC) path restatements. nthreads <= 0 uses OpenMP's default. */
int oracle_ao_vgl_hpc(const oracle_basis* b, int32_t precision, int64_t point_num,
                      const double* coord, const double* nucl_coord,
                      double* ao_vgl, int32_t nthreads);
int oracle_ao_value_hpc(const oracle_basis* b, int32_t precision, int64_t point_num,
                        const double* coord, const double* nucl_coord,
                        double* ao_value, int32_t nthreads);

/* Reference ("doc", Fortran) path restatements. */
int oracle_primitive_vgl(const oracle_basis* b, int32_t precision, int64_t point_num,
                         const double* coord, const double* nucl_coord, double* prim_vgl);
int oracle_shell_vgl_doc(const oracle_basis* b, int32_t precision, int64_t point_num,
                         const double* coord, const double* nucl_coord, double* shell_vgl);
int oracle_ao_vgl_doc(const oracle_basis* b, int32_t precision, int64_t point_num,
                      const double* coord, const double* nucl_coord, double* ao_vgl);

/* Cartesian monomials of degree <= lmax at X - R with their gradient and
 * Laplacian, vgl[c * 120 + m] (c = 0..4, m in the canonical order of
 * org/qmckl_ao.org:5928-5933), by the HPC arithmetic (which = 1; shift added
 * after the products, org/qmckl_ao.org:6624-6914) or the doc arithmetic
 * (which = 0; shift added to the displacement, 6233-6364).  Returns the
 * number of monomials, -1 for lmax outside 0..ORACLE_MAX_L. */
int oracle_poly_vgl(int32_t which, int32_t lmax, const double* X, const double* R, double* vgl);

/* MO contraction, skipping AOs whose value is zero (org/qmckl_mo.org:2015-2163). */
int oracle_mo_vgl(int64_t ao_num, int64_t mo_num, int64_t point_num,
                  const double* coefficient_t, const double* ao_vgl,
                  double* mo_vgl, int32_t nthreads);
int oracle_mo_value(int64_t ao_num, int64_t mo_num, int64_t point_num,
                    const double* coefficient_t, const double* ao_value,
                    double* mo_value, int32_t nthreads);

/* Derivatives (nuclear-derivative checks).
 *   shell_hessian[point][3][4][shell], ao_hessian[3][point][4][ao]: second
 *   derivatives and derivatives of the Laplacian with respect to the point
 *   coordinates (the reference's qmckl_get_ao_basis_ao_hessian layout). */
int oracle_shell_hessian_doc(const oracle_basis* b, int32_t precision, int64_t point_num,
                             const double* coord, const double* nucl_coord, double* shell_hessian);
int oracle_ao_hessian_doc(const oracle_basis* b, int32_t precision, int64_t point_num,
                          const double* coord, const double* nucl_coord, double* ao_hessian);
/* Gradient of L = sum W * mo_vgl (W: [point][5][mo]) with respect to the MO
 * coefficients ([mo][ao]), the nuclear coordinates ([nucl][3]) and the point
 * coordinates ([3][point]), through the reference's orbital forces.  Outputs
 * may be NULL. */
int oracle_mo_vgl_adjoint(const oracle_basis* b, int32_t precision, int64_t point_num, const double* coord,
                          const double* nucl_coord, int64_t mo_num, const double* coefficient,
                          const double* weight, double* grad_coef, double* grad_nucl, double* grad_coord);

/* Orbital forces, full tensors (the reference's forces getters):
 *   fao [nucl][point][3][ao], fmv [nucl][point][3][mo],
 *   fmg [nucl][3][point][3][mo], fml [nucl][3][point][mo]; NULL to skip. */
int oracle_forces(const oracle_basis* b, int32_t precision, int64_t point_num, const double* coord,
                  const double* nucl_coord, int64_t mo_num, const double* coefficient, double* fao,
                  double* fmv, double* fmg, double* fml);

#ifdef __cplusplus
}
#endif
#endif
