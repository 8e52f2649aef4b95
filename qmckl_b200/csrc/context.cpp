// Context, error, numerical-precision and lock management.
//
// Behaviour follows org/qmckl_context.org (create 308-411, check 227-240,
// touch 262-279, copy 468-597, threads 599-760, destroy 777-843),
// org/qmckl_error.org (string_of_error 218-380, set/get_error 402-520,
// failwith 539-598, last_error 601-640, check 660-700) and
// org/qmckl_numprec.org (170-435).
#include <cassert>
#include <cstdio>
#include <cstdlib>
#include <new>
#include <string>
#include <thread>

#include "internal.h"
#include "qmckl_b200.h"

namespace qb {
int64_t g_alloc_fail_countdown = -1;
bool alloc_should_fail() {
  if (g_alloc_fail_countdown < 0) return false;
  if (g_alloc_fail_countdown == 0) { g_alloc_fail_countdown = -1; return true; }
  --g_alloc_fail_countdown;
  return false;
}
}  // namespace qb

using namespace qb;

extern "C" {

void qmckl_b200_inject_alloc_failure(const int64_t n) { g_alloc_fail_countdown = n; }

qmckl_context qmckl_context_check(const qmckl_context context) {
  if (context == QMCKL_NULL_CONTEXT) return QMCKL_NULL_CONTEXT;
  const Context* ctx = ctx_of(context);
  if (ctx->tag != VALID_TAG) return QMCKL_NULL_CONTEXT;
  return context;
}

qmckl_exit_code qmckl_context_touch(const qmckl_context context) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT)
    return qmckl_failwith(context, QMCKL_INVALID_CONTEXT, "qmckl_context_touch", NULL);
  Context* ctx = ctx_of(context);
  ctx->date += 1;
  ctx->point.date = ctx->date;
  ctx->electron.walker.point.date = ctx->date;
  return QMCKL_SUCCESS;
}

qmckl_context qmckl_context_create(void) {
  if (alloc_should_fail()) return QMCKL_NULL_CONTEXT;
  Context* ctx = new (std::nothrow) Context();
  if (ctx == nullptr) return QMCKL_NULL_CONTEXT;
  ctx->tag = VALID_TAG;
  unsigned hc = std::thread::hardware_concurrency();
  ctx->num_threads = hc > 0 ? (int32_t)hc : 1;
  // org/qmckl_ao.org:398-414: the AO basis starts with 14 unset fields, cartesian by default
  ctx->ao_basis.uninitialized = (1 << 14) - 1;
  ctx->ao_basis.ao_cartesian = true;
  ctx->mo_basis.uninitialized = (1 << 2) - 1;
  ctx->nucleus.uninitialized = (1 << 3) - 1;
  ctx->electron.uninitialized = (1 << 1) - 1;
  return (qmckl_context)ctx;
}

qmckl_context qmckl_context_copy(const qmckl_context context) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_NULL_CONTEXT;
  const Context* src = ctx_of(context);
  if (alloc_should_fail()) return QMCKL_NULL_CONTEXT;
  Context* dst = new (std::nothrow) Context();
  if (dst == nullptr) return QMCKL_NULL_CONTEXT;
  dst->tag = VALID_TAG;
  dst->precision = src->precision;
  dst->range = src->range;
  dst->num_threads = src->num_threads;
  dst->error = src->error;
  dst->date = src->date;
  dst->point = src->point;
  dst->nucleus = src->nucleus;
  dst->electron = src->electron;
  dst->ao_basis = src->ao_basis;
  dst->mo_basis = src->mo_basis;
  dst->form = src->form;
  // Computed arrays are not copied (as in org/qmckl_mo.org:448-455): the new
  // context gets its own device state and recomputes on first use.
  dst->ao_basis.primitive_vgl_date = dst->ao_basis.shell_vgl_date = 0;
  dst->ao_basis.ao_vgl_date = dst->ao_basis.ao_value_date = dst->ao_basis.ao_hessian_date = 0;
  dst->mo_basis.mo_vgl_date = dst->mo_basis.mo_value_date = dst->mo_basis.mo_hessian_date = 0;
  dst->extra = nullptr;
  return (qmckl_context)dst;
}

qmckl_exit_code qmckl_context_destroy(const qmckl_context context) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  Context* ctx = ctx_of(context);
  dev_detach(ctx);
  ctx->tag = INVALID_TAG;
  delete ctx;
  return QMCKL_SUCCESS;
}

void qmckl_lock(qmckl_context context) {
  if (context == QMCKL_NULL_CONTEXT) return;
  Context* ctx = ctx_of(context);
  ctx->mutex.lock();
  ctx->lock_count += 1;
}

void qmckl_unlock(qmckl_context context) {
  if (context == QMCKL_NULL_CONTEXT) return;
  Context* ctx = ctx_of(context);
  ctx->lock_count -= 1;
  ctx->mutex.unlock();
}

qmckl_exit_code qmckl_context_set_num_threads(qmckl_context context, const int32_t num_threads) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  if (num_threads <= 0)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_context_set_num_threads",
                          "num_threads must be positive");
  qmckl_lock(context);
  ctx_of(context)->num_threads = num_threads;
  qmckl_unlock(context);
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_context_get_num_threads(const qmckl_context context, int32_t* const num_threads) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  if (num_threads == NULL)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_context_get_num_threads",
                          "num_threads is a null pointer");
  *num_threads = ctx_of(context)->num_threads;
  return QMCKL_SUCCESS;
}

/* ---------------------------------------------------------------- errors */

const char* qmckl_string_of_error(const qmckl_exit_code error) {
  switch (error) {
    case QMCKL_SUCCESS: return "Success";
    case QMCKL_INVALID_ARG_1: return "Invalid argument 1";
    case QMCKL_INVALID_ARG_2: return "Invalid argument 2";
    case QMCKL_INVALID_ARG_3: return "Invalid argument 3";
    case QMCKL_INVALID_ARG_4: return "Invalid argument 4";
    case QMCKL_INVALID_ARG_5: return "Invalid argument 5";
    case QMCKL_INVALID_ARG_6: return "Invalid argument 6";
    case QMCKL_INVALID_ARG_7: return "Invalid argument 7";
    case QMCKL_INVALID_ARG_8: return "Invalid argument 8";
    case QMCKL_INVALID_ARG_9: return "Invalid argument 9";
    case QMCKL_INVALID_ARG_10: return "Invalid argument 10";
    case QMCKL_INVALID_ARG_11: return "Invalid argument 11";
    case QMCKL_INVALID_ARG_12: return "Invalid argument 12";
    case QMCKL_INVALID_ARG_13: return "Invalid argument 13";
    case QMCKL_INVALID_ARG_14: return "Invalid argument 14";
    case QMCKL_INVALID_ARG_15: return "Invalid argument 15";
    case QMCKL_INVALID_ARG_16: return "Invalid argument 16";
    case QMCKL_INVALID_ARG_17: return "Invalid argument 17";
    case QMCKL_INVALID_ARG_18: return "Invalid argument 18";
    case QMCKL_INVALID_ARG_19: return "Invalid argument 19";
    case QMCKL_INVALID_ARG_20: return "Invalid argument 20";
    case QMCKL_FAILURE: return "Failure";
    case QMCKL_ERRNO: return "Errno";
    case QMCKL_INVALID_CONTEXT: return "Invalid context";
    case QMCKL_ALLOCATION_FAILED: return "Allocation failed";
    case QMCKL_DEALLOCATION_FAILED: return "De-allocation failed";
    case QMCKL_NOT_PROVIDED: return "Not provided";
    case QMCKL_OUT_OF_BOUNDS: return "Index out of bounds";
    case QMCKL_ALREADY_SET: return "Already set";
    default: return "Invalid exit code";
  }
}

qmckl_exit_code qmckl_set_error(qmckl_context context, const qmckl_exit_code exit_code,
                                const char* function_name, const char* message) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  if (function_name == NULL || message == NULL) return QMCKL_INVALID_ARG_3;
  if (exit_code <= QMCKL_SUCCESS || exit_code >= QMCKL_INVALID_EXIT_CODE) return QMCKL_INVALID_ARG_2;
  qmckl_lock(context);
  Context* ctx = ctx_of(context);
  ctx->error.exit_code = exit_code;
  std::strncpy(ctx->error.function, function_name, QMCKL_MAX_FUN_LEN - 1);
  ctx->error.function[QMCKL_MAX_FUN_LEN - 1] = 0;
  std::strncpy(ctx->error.message, message, QMCKL_MAX_MSG_LEN - 1);
  ctx->error.message[QMCKL_MAX_MSG_LEN - 1] = 0;
  qmckl_unlock(context);
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_get_error(qmckl_context context, qmckl_exit_code* exit_code,
                                char* function_name, char* message) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  if (exit_code == NULL || function_name == NULL || message == NULL) return QMCKL_INVALID_ARG_2;
  qmckl_lock(context);
  Context* ctx = ctx_of(context);
  std::strncpy(function_name, ctx->error.function, QMCKL_MAX_FUN_LEN);
  std::strncpy(message, ctx->error.message, QMCKL_MAX_MSG_LEN);
  *exit_code = ctx->error.exit_code;
  qmckl_unlock(context);
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_failwith(qmckl_context context, const qmckl_exit_code exit_code,
                               const char* function, const char* message) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  if (function == NULL) function = "(unknown)";
  qmckl_set_error(context, exit_code, function,
                  message == NULL ? qmckl_string_of_error(exit_code) : message);
  return exit_code;
}

qmckl_exit_code qmckl_last_error(qmckl_context context, char* buffer) {
  if (buffer == NULL) return QMCKL_INVALID_ARG_2;
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) {
    std::strncpy(buffer, "Null context", 13);
    return QMCKL_FAILURE;
  }
  char fname[QMCKL_MAX_FUN_LEN];
  char msg[QMCKL_MAX_MSG_LEN];
  qmckl_exit_code last;
  qmckl_exit_code rc = qmckl_get_error(context, &last, fname, msg);
  if (rc != QMCKL_SUCCESS) return rc;
  std::string text = std::string("Error -- ") + qmckl_string_of_error(last) + " -- in " + fname + "\n" + msg;
  std::strncpy(buffer, text.c_str(), QMCKL_MAX_MSG_LEN - 1);
  buffer[QMCKL_MAX_MSG_LEN - 1] = 0;
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_check(qmckl_context context, qmckl_exit_code rc) {
  if (rc != QMCKL_SUCCESS) {
    char fname[QMCKL_MAX_FUN_LEN] = {0};
    char msg[QMCKL_MAX_MSG_LEN] = {0};
    std::fprintf(stderr, "===========\nQMCKL ERROR\n%s\n", qmckl_string_of_error(rc));
    qmckl_exit_code last;
    if (qmckl_get_error(context, &last, fname, msg) == QMCKL_SUCCESS)
      std::fprintf(stderr, "Function: %s\nMessage: %s\n===========\n", fname, msg);
  }
  return rc;
}

/* ------------------------------------------------------ numerical precision */

qmckl_exit_code qmckl_set_numprec_precision(const qmckl_context context, const int precision) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  if (precision < 2)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_update_numprec_precision", "precision < 2");
  if (precision > 53)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_update_numprec_precision", "precision > 53");
  qmckl_lock(context);
  ctx_of(context)->precision = (uint32_t)precision;
  qmckl_unlock(context);
  return QMCKL_SUCCESS;
}

int32_t qmckl_get_numprec_precision(const qmckl_context context) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT)
    return qmckl_failwith(context, QMCKL_INVALID_CONTEXT, "qmckl_get_numprec_precision", "");
  return (int32_t)ctx_of(context)->precision;
}

qmckl_exit_code qmckl_set_numprec_range(const qmckl_context context, const int range) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  if (range < 2) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_set_numprec_range", "range < 2");
  if (range > 11) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_set_numprec_range", "range > 11");
  qmckl_lock(context);
  ctx_of(context)->range = (uint32_t)range;
  qmckl_unlock(context);
  return QMCKL_SUCCESS;
}

int32_t qmckl_get_numprec_range(const qmckl_context context) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT)
    return qmckl_failwith(context, QMCKL_INVALID_CONTEXT, "qmckl_get_numprec_range", "");
  return (int32_t)ctx_of(context)->range;
}

double qmckl_get_numprec_epsilon(const qmckl_context context) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  const int precision = (int)ctx_of(context)->precision;
  return 1. / (double)(((uint64_t)1) << (precision - 1));
}

static int64_t count_ulp_difference_64(double a, double b) {
  int64_t x, y;
  std::memcpy(&x, &a, 8);
  std::memcpy(&y, &b, 8);
  if ((x < 0) != (y < 0) && a != 0.0 && b != 0.0) {
    const int64_t dx = x < 0 ? INT64_MAX + x : INT64_MAX - x;
    const int64_t dy = y < 0 ? INT64_MAX + y : INT64_MAX - y;
    return dx + dy;
  }
  int64_t r = x - y;
  return r > 0 ? r : -r;
}

int32_t qmckl_test_precision_64(double a, double b) {
  int64_t diff = count_ulp_difference_64(a, b);
  if (diff == 0) return 53;
  int32_t result = 53;
  for (int i = 0; i < 53 && diff != 0; ++i) {
    diff >>= 1;
    result--;
  }
  return result;
}

int32_t qmckl_test_precision_32(float a, float b) { return qmckl_test_precision_64((double)a, (double)b); }

/* ------------------------------------------------------------ B200 knobs */

qmckl_exit_code qmckl_b200_set_form(qmckl_context context, const int32_t form) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  if (form < QMCKL_B200_FORM_AUTO || form > QMCKL_B200_FORM_MIXED)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_b200_set_form", "unknown form");
  Context* ctx = ctx_of(context);
  if (ctx->form != form) {
    ctx->form = form;
    qmckl_context_touch(context);   // cached arrays were computed in the other form
  }
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_b200_get_form(const qmckl_context context, int32_t* const form) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  if (form == NULL) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_b200_get_form", "NULL pointer");
  *form = ctx_of(context)->form;
  return QMCKL_SUCCESS;
}

}  // extern "C"
