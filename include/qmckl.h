/*
 * qmckl.h -- the subset of the QMCkl public C API served by qmckl_b200.
 *
 * Prototypes, exit codes and conventions are those of the reference library
 * (its qmckl.h is generated from the org sources; each block below cites the
 * org file:line of the declaration it reproduces).  A program written against
 * the reference's orbital-evaluation API compiles unchanged against this header
 * and links against libqmckl_b200.so.
 */
#ifndef QMCKL_H
#define QMCKL_H

#include <stdbool.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* org/qmckl_context.org:104-105 */
typedef int64_t qmckl_context;
#define QMCKL_NULL_CONTEXT (qmckl_context)0

/* org/qmckl_error.org:67-120 */
typedef int32_t qmckl_exit_code;
#define QMCKL_SUCCESS               ((qmckl_exit_code) 0)
#define QMCKL_INVALID_ARG_1         ((qmckl_exit_code) 1)
#define QMCKL_INVALID_ARG_2         ((qmckl_exit_code) 2)
#define QMCKL_INVALID_ARG_3         ((qmckl_exit_code) 3)
#define QMCKL_INVALID_ARG_4         ((qmckl_exit_code) 4)
#define QMCKL_INVALID_ARG_5         ((qmckl_exit_code) 5)
#define QMCKL_INVALID_ARG_6         ((qmckl_exit_code) 6)
#define QMCKL_INVALID_ARG_7         ((qmckl_exit_code) 7)
#define QMCKL_INVALID_ARG_8         ((qmckl_exit_code) 8)
#define QMCKL_INVALID_ARG_9         ((qmckl_exit_code) 9)
#define QMCKL_INVALID_ARG_10        ((qmckl_exit_code) 10)
#define QMCKL_INVALID_ARG_11        ((qmckl_exit_code) 11)
#define QMCKL_INVALID_ARG_12        ((qmckl_exit_code) 12)
#define QMCKL_INVALID_ARG_13        ((qmckl_exit_code) 13)
#define QMCKL_INVALID_ARG_14        ((qmckl_exit_code) 14)
#define QMCKL_INVALID_ARG_15        ((qmckl_exit_code) 15)
#define QMCKL_INVALID_ARG_16        ((qmckl_exit_code) 16)
#define QMCKL_INVALID_ARG_17        ((qmckl_exit_code) 17)
#define QMCKL_INVALID_ARG_18        ((qmckl_exit_code) 18)
#define QMCKL_INVALID_ARG_19        ((qmckl_exit_code) 19)
#define QMCKL_INVALID_ARG_20        ((qmckl_exit_code) 20)
#define QMCKL_FAILURE               ((qmckl_exit_code) 101)
#define QMCKL_ERRNO                 ((qmckl_exit_code) 102)
#define QMCKL_INVALID_CONTEXT       ((qmckl_exit_code) 103)
#define QMCKL_ALLOCATION_FAILED     ((qmckl_exit_code) 104)
#define QMCKL_DEALLOCATION_FAILED   ((qmckl_exit_code) 105)
#define QMCKL_NOT_PROVIDED          ((qmckl_exit_code) 106)
#define QMCKL_OUT_OF_BOUNDS         ((qmckl_exit_code) 107)
#define QMCKL_ALREADY_SET           ((qmckl_exit_code) 108)
#define QMCKL_INVALID_EXIT_CODE     ((qmckl_exit_code) 109)

/* org/qmckl_error.org:402-403 */
#define QMCKL_MAX_FUN_LEN 256
#define QMCKL_MAX_MSG_LEN 1024

/* org/qmckl_numprec.org:100-107 */
#define QMCKL_DEFAULT_PRECISION 53
#define QMCKL_DEFAULT_RANGE 11

/* ---- context: org/qmckl_context.org:222-843 ---- */
qmckl_context   qmckl_context_check(const qmckl_context context);
qmckl_exit_code qmckl_context_touch(const qmckl_context context);
qmckl_context   qmckl_context_create(void);
qmckl_context   qmckl_context_copy(const qmckl_context context);
qmckl_exit_code qmckl_context_destroy(const qmckl_context context);
void            qmckl_lock(qmckl_context context);
void            qmckl_unlock(qmckl_context context);
qmckl_exit_code qmckl_context_set_num_threads(qmckl_context context, const int32_t num_threads);
qmckl_exit_code qmckl_context_get_num_threads(const qmckl_context context, int32_t* const num_threads);

/* ---- errors: org/qmckl_error.org:218-700 ---- */
const char*     qmckl_string_of_error(const qmckl_exit_code error);
qmckl_exit_code qmckl_set_error(qmckl_context context, const qmckl_exit_code exit_code,
                                const char* function_name, const char* message);
qmckl_exit_code qmckl_get_error(qmckl_context context, qmckl_exit_code* exit_code,
                                char* function_name, char* message);
qmckl_exit_code qmckl_failwith(qmckl_context context, const qmckl_exit_code exit_code,
                               const char* function, const char* message);
qmckl_exit_code qmckl_last_error(qmckl_context context, char* buffer);
qmckl_exit_code qmckl_check(qmckl_context context, qmckl_exit_code rc);

/* ---- numerical precision: org/qmckl_numprec.org:170-435 ---- */
qmckl_exit_code qmckl_set_numprec_precision(const qmckl_context context, const int precision);
int32_t         qmckl_get_numprec_precision(const qmckl_context context);
qmckl_exit_code qmckl_set_numprec_range(const qmckl_context context, const int range);
int32_t         qmckl_get_numprec_range(const qmckl_context context);
double          qmckl_get_numprec_epsilon(const qmckl_context context);
int32_t         qmckl_test_precision_64(double a, double b);
int32_t         qmckl_test_precision_32(float a, float b);

/* ---- points: org/qmckl_point.org:141-392 ---- */
qmckl_exit_code qmckl_get_point_num(const qmckl_context context, int64_t* const num);
qmckl_exit_code qmckl_get_point(const qmckl_context context, const char transp,
                                double* const coord, const int64_t size_max);
qmckl_exit_code qmckl_set_point(qmckl_context context, const char transp, const int64_t num,
                                const double* coord, const int64_t size_max);

/* ---- nuclei: org/qmckl_nucleus.org:159-612 ---- */
bool            qmckl_nucleus_provided(const qmckl_context context);
qmckl_exit_code qmckl_get_nucleus_num(const qmckl_context context, int64_t* const num);
qmckl_exit_code qmckl_get_nucleus_charge(const qmckl_context context, double* const charge,
                                         const int64_t size_max);
qmckl_exit_code qmckl_get_nucleus_coord(const qmckl_context context, const char transp,
                                        double* const coord, const int64_t size_max);
qmckl_exit_code qmckl_set_nucleus_num(qmckl_context context, const int64_t num);
qmckl_exit_code qmckl_set_nucleus_charge(qmckl_context context, const double* charge,
                                         const int64_t size_max);
qmckl_exit_code qmckl_set_nucleus_coord(qmckl_context context, const char transp,
                                        const double* coord, const int64_t size_max);

/* ---- electrons: org/qmckl_electron.org:223-618 ---- */
bool            qmckl_electron_provided(const qmckl_context context);
qmckl_exit_code qmckl_set_electron_num(qmckl_context context, const int64_t up_num,
                                       const int64_t down_num);
qmckl_exit_code qmckl_set_electron_coord(qmckl_context context, const char transp,
                                         const int64_t walk_num, const double* coord,
                                         const int64_t size_max);
qmckl_exit_code qmckl_get_electron_num(const qmckl_context context, int64_t* const num);
qmckl_exit_code qmckl_get_electron_up_num(const qmckl_context context, int64_t* const up_num);
qmckl_exit_code qmckl_get_electron_down_num(const qmckl_context context, int64_t* const down_num);
qmckl_exit_code qmckl_get_electron_walk_num(const qmckl_context context, int64_t* const walk_num);
qmckl_exit_code qmckl_get_electron_coord(const qmckl_context context, const char transp,
                                         double* const coord, const int64_t size_max);
/* TREXIO input (org/qmckl_trexio.org:1106-1190): electrons, nuclei, AO basis
 * and MO coefficients of a TREXIO file in the text backend (a directory of
 * <group>.txt files), set through the context's setters as the reference's
 * readers do.  Anything else (an HDF5 file) is QMCKL_INVALID_ARG_2, as the
 * reference reports a file none of its backends opens. */
qmckl_exit_code qmckl_trexio_read(const qmckl_context context, const char* file_name, const int64_t size_max);
/* point-nucleus distances [point][nucl] (org/qmckl_electron.org:1205-1262) */
qmckl_exit_code qmckl_get_electron_en_distance(qmckl_context context, double* const distance,
                                               const int64_t size_max);

/* ---- AO basis: org/qmckl_ao.org:419-2266 (setters/getters), 3415-3798 (arrays) ---- */
qmckl_exit_code qmckl_set_ao_basis_type(qmckl_context context, const char basis_type);
qmckl_exit_code qmckl_set_ao_basis_shell_num(qmckl_context context, const int64_t shell_num);
qmckl_exit_code qmckl_set_ao_basis_prim_num(qmckl_context context, const int64_t prim_num);
qmckl_exit_code qmckl_set_ao_basis_nucleus_shell_num(qmckl_context context, const int64_t* nucleus_shell_num, const int64_t size_max);
qmckl_exit_code qmckl_set_ao_basis_nucleus_index(qmckl_context context, const int64_t* nucleus_index, const int64_t size_max);
qmckl_exit_code qmckl_set_ao_basis_shell_ang_mom(qmckl_context context, const int32_t* shell_ang_mom, const int64_t size_max);
qmckl_exit_code qmckl_set_ao_basis_shell_prim_num(qmckl_context context, const int64_t* shell_prim_num, const int64_t size_max);
qmckl_exit_code qmckl_set_ao_basis_shell_prim_index(qmckl_context context, const int64_t* shell_prim_index, const int64_t size_max);
qmckl_exit_code qmckl_set_ao_basis_shell_factor(qmckl_context context, const double* shell_factor, const int64_t size_max);
qmckl_exit_code qmckl_set_ao_basis_exponent(qmckl_context context, const double* exponent, const int64_t size_max);
qmckl_exit_code qmckl_set_ao_basis_coefficient(qmckl_context context, const double* coefficient, const int64_t size_max);
qmckl_exit_code qmckl_set_ao_basis_prim_factor(qmckl_context context, const double* prim_factor, const int64_t size_max);
qmckl_exit_code qmckl_set_ao_basis_ao_num(qmckl_context context, const int64_t ao_num);
qmckl_exit_code qmckl_set_ao_basis_ao_factor(qmckl_context context, const double* ao_factor, const int64_t size_max);
qmckl_exit_code qmckl_set_ao_basis_r_power(qmckl_context context, const int32_t* r_power, const int64_t size_max);
qmckl_exit_code qmckl_set_ao_basis_cartesian(qmckl_context context, const bool cartesian);

qmckl_exit_code qmckl_get_ao_basis_type(const qmckl_context context, char* const basis_type);
qmckl_exit_code qmckl_get_ao_basis_shell_num(const qmckl_context context, int64_t* const shell_num);
qmckl_exit_code qmckl_get_ao_basis_prim_num(const qmckl_context context, int64_t* const prim_num);
qmckl_exit_code qmckl_get_ao_basis_nucleus_shell_num(const qmckl_context context, int64_t* const nucleus_shell_num, const int64_t size_max);
qmckl_exit_code qmckl_get_ao_basis_nucleus_index(const qmckl_context context, int64_t* const nucleus_index, const int64_t size_max);
qmckl_exit_code qmckl_get_ao_basis_r_power(const qmckl_context context, int32_t* const r_power, const int64_t size_max);
qmckl_exit_code qmckl_get_ao_basis_shell_ang_mom(const qmckl_context context, int32_t* const shell_ang_mom, const int64_t size_max);
qmckl_exit_code qmckl_get_ao_basis_shell_prim_num(const qmckl_context context, int64_t* const shell_prim_num, const int64_t size_max);
qmckl_exit_code qmckl_get_ao_basis_shell_prim_index(const qmckl_context context, int64_t* const shell_prim_index, const int64_t size_max);
qmckl_exit_code qmckl_get_ao_basis_shell_factor(const qmckl_context context, double* const shell_factor, const int64_t size_max);
qmckl_exit_code qmckl_get_ao_basis_exponent(const qmckl_context context, double* const exponent, const int64_t size_max);
qmckl_exit_code qmckl_get_ao_basis_coefficient(const qmckl_context context, double* const coefficient, const int64_t size_max);
qmckl_exit_code qmckl_get_ao_basis_prim_factor(const qmckl_context context, double* const prim_factor, const int64_t size_max);
qmckl_exit_code qmckl_get_ao_basis_ao_num(const qmckl_context context, int64_t* const ao_num);
qmckl_exit_code qmckl_get_ao_basis_cartesian(const qmckl_context context, bool* const cartesian);
qmckl_exit_code qmckl_get_ao_basis_ao_factor(const qmckl_context context, double* const ao_factor, const int64_t size_max);
bool            qmckl_ao_basis_provided(const qmckl_context context);

qmckl_exit_code qmckl_get_ao_basis_primitive_vgl(qmckl_context context, double* const primitive_vgl, const int64_t size_max);
qmckl_exit_code qmckl_get_ao_basis_shell_vgl(qmckl_context context, double* const shell_vgl, const int64_t size_max);
qmckl_exit_code qmckl_get_ao_basis_ao_vgl(qmckl_context context, double* const ao_vgl, const int64_t size_max);
qmckl_exit_code qmckl_get_ao_basis_ao_vgl_inplace(qmckl_context context, double* const ao_vgl, const int64_t size_max);
qmckl_exit_code qmckl_get_ao_basis_ao_value(qmckl_context context, double* const ao_value, const int64_t size_max);
qmckl_exit_code qmckl_get_ao_basis_ao_value_inplace(qmckl_context context, double* const ao_value, const int64_t size_max);
/* ao_hessian[3][point_num][4][ao_num]: [i][p][j][k] = d_i d_j AO_k (j < 3) and
 * d_i (Laplacian of AO_k) (j = 3), derivatives with respect to the point
 * coordinates (org/qmckl_ao.org:9400-9404, 9590-9720). */
qmckl_exit_code qmckl_get_ao_basis_ao_hessian(qmckl_context context, double* const ao_hessian, const int64_t size_max);

/* Orbital forces: derivatives with respect to the nuclear coordinates
 * (org/qmckl_forces.org).  Layouts:
 *   forces_ao_value [nucl][point][3][ao]    (5129-5160; 0 for AOs of other nuclei)
 *   forces_mo_value [nucl][point][3][mo]    (5475-5575)
 *   forces_mo_g     [nucl][3][point][3][mo] (5919-6000): d/dR_{a,n} of the MO gradient
 *   forces_mo_l     [nucl][3][point][mo]    (6499-6530): d/dR_{a,n} of the MO Laplacian */
qmckl_exit_code qmckl_get_forces_ao_value(qmckl_context context, double* const forces_ao_value, const int64_t size_max);
qmckl_exit_code qmckl_get_forces_mo_value(qmckl_context context, double* const forces_mo_value, const int64_t size_max);
qmckl_exit_code qmckl_get_forces_mo_value_inplace(qmckl_context context, double* const forces_mo_value,
                                                  const int64_t size_max);
qmckl_exit_code qmckl_get_forces_mo_g(qmckl_context context, double* const forces_mo_g, const int64_t size_max);
qmckl_exit_code qmckl_get_forces_mo_g_inplace(qmckl_context context, double* const forces_mo_g, const int64_t size_max);
qmckl_exit_code qmckl_get_forces_mo_l(qmckl_context context, double* const forces_mo_l, const int64_t size_max);

/* ---- standalone AO helpers, one point, computed on the host ---- */
/* P[i*ldp + k-1] = X[i]^k, k = 1..LMAX[i] (org/qmckl_ao.org:5971-6026; as there,
 * n <= ldp is rejected with QMCKL_INVALID_ARG_2). */
qmckl_exit_code qmckl_ao_power(const qmckl_context context, const int64_t n, const double* X, const int32_t* LMAX,
                               double* const P, const int64_t ldp);
/* VGL[c*ldv + i], c = value, d/dx, d/dy, d/dz, Laplacian of exp(-A[i] |X-R|^2)
 * (org/qmckl_ao.org:3839-3910).  The reference's generated C prototype reads
 * n, A and VGL as pointers; its bind(C) function takes n by value, A as input
 * and VGL as output, which is the ABI declared here. */
qmckl_exit_code qmckl_ao_gaussian_vgl(const qmckl_context context, const double* X, const double* R, const int64_t n,
                                      const double* A, double* const VGL, const int64_t ldv);
/* Cartesian monomials of X - R of degree <= lmax, L[m*ldl + {0,1,2}] their
 * powers, *n their number (org/qmckl_ao.org:6195-6619, 6624-6914); lmax
 * outside 0..1000 gives QMCKL_INVALID_ARG_4.
 * Non-transposed forms: VGL[m*ldv + c]; transposed forms: VGL[c*ldv + m]. */
qmckl_exit_code qmckl_ao_polynomial_vgl(const qmckl_context context, const double* X, const double* R,
                                        const int32_t lmax, int64_t* n, int32_t* const L, const int64_t ldl,
                                        double* const VGL, const int64_t ldv);
qmckl_exit_code qmckl_ao_polynomial_vgl_doc(const qmckl_context context, const double* X, const double* R,
                                            const int32_t lmax, int64_t* n, int32_t* const L, const int64_t ldl,
                                            double* const VGL, const int64_t ldv);
qmckl_exit_code qmckl_ao_polynomial_transp_vgl(const qmckl_context context, const double* X, const double* R,
                                               const int32_t lmax, int64_t* n, int32_t* const L, const int64_t ldl,
                                               double* const VGL, const int64_t ldv);
qmckl_exit_code qmckl_ao_polynomial_transp_vgl_doc(const qmckl_context context, const double* X, const double* R,
                                                   const int32_t lmax, int64_t* n, int32_t* const L,
                                                   const int64_t ldl, double* const VGL, const int64_t ldv);
qmckl_exit_code qmckl_ao_polynomial_transp_vgl_hpc(const qmckl_context context, const double* X, const double* R,
                                                   const int32_t lmax, int64_t* n, int32_t* const L,
                                                   const int64_t ldl, double* const VGL, const int64_t ldv);

/* ---- MO basis: org/qmckl_mo.org:192-1747, 2362-2400, 3479 ---- */
qmckl_exit_code qmckl_set_mo_basis_mo_num(qmckl_context context, const int64_t mo_num);
qmckl_exit_code qmckl_set_mo_basis_coefficient(qmckl_context context, const double* coefficient, const int64_t size_max);
/* cusp adjustment radius per nucleus (org/qmckl_mo.org:479-700) */
qmckl_exit_code qmckl_set_mo_basis_r_cusp(qmckl_context context, const double* r_cusp, const int64_t size_max);
qmckl_exit_code qmckl_get_mo_basis_mo_num(const qmckl_context context, int64_t* mo_num);
qmckl_exit_code qmckl_get_mo_basis_coefficient(const qmckl_context context, double* const coefficient, const int64_t size_max);
bool            qmckl_mo_basis_provided(const qmckl_context context);
qmckl_exit_code qmckl_mo_basis_select_mo(const qmckl_context context, const int32_t* keep, const int64_t size_max);
qmckl_exit_code qmckl_mo_basis_rescale(qmckl_context context, const double scaling_factor);
qmckl_exit_code qmckl_get_mo_basis_mo_value(qmckl_context context, double* const mo_value, const int64_t size_max);
qmckl_exit_code qmckl_get_mo_basis_mo_value_inplace(qmckl_context context, double* const mo_value, const int64_t size_max);
qmckl_exit_code qmckl_get_mo_basis_mo_vgl(qmckl_context context, double* const mo_vgl, const int64_t size_max);
qmckl_exit_code qmckl_get_mo_basis_mo_vgl_inplace(qmckl_context context, double* const mo_vgl, const int64_t size_max);
/* [3][point][3][mo] */
qmckl_exit_code qmckl_get_mo_basis_mo_hessian(qmckl_context context, double* const mo_hessian, const int64_t size_max);

#ifdef __cplusplus
}
#endif
#endif /* QMCKL_H */
