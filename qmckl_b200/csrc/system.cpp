// Points, nuclei and electrons: the inputs of the orbital-evaluation path.
//
// Follows org/qmckl_point.org (get 141-265, set 277-392),
// org/qmckl_nucleus.org (getters 159-330, setters 380-612) and
// org/qmckl_electron.org (num/coord setters 223-392, getters 400-618):
// same argument checks, exit codes and date updates.  Coordinates are stored
// as the reference's column-major num x 3 matrices ([3][num] in C order).
#include "internal.h"

using namespace qb;

namespace {

qmckl_exit_code store_points(qmckl_context context, PointRec& pt, const char transp,
                             const int64_t num, const double* coord) {
  if (num != pt.num) {
    if (alloc_should_fail())
      return qmckl_failwith(context, QMCKL_ALLOCATION_FAILED, "qmckl_set_point", NULL);
    pt.coord.assign((size_t)(3 * num), 0.0);
  }
  pt.num = num;
  double* a = pt.coord.data();
  if (transp == 'T') {
    std::memcpy(a, coord, sizeof(double) * 3 * num);
  } else {
    for (int64_t i = 0; i < num; ++i) {
      a[i] = coord[3 * i];
      a[i + num] = coord[3 * i + 1];
      a[i + 2 * num] = coord[3 * i + 2];
    }
  }
  return QMCKL_SUCCESS;
}

}  // namespace

extern "C" {

/* ------------------------------------------------------------------ points */

qmckl_exit_code qmckl_get_point_num(const qmckl_context context, int64_t* const num) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  if (num == NULL)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_point_num", "num is a null pointer");
  *num = ctx_of(context)->point.num;
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_get_point(const qmckl_context context, const char transp,
                                double* const coord, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  if (coord == NULL)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_point_coord", "coord is a null pointer");
  Context* ctx = ctx_of(context);
  const int64_t n = ctx->point.num;
  if (n == 0) return QMCKL_NOT_PROVIDED;
  if (size_max < 3 * n)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_get_point_coord", "size_max too small");
  const double* a = ctx->point.coord.data();
  if (transp == 'N') {
    for (int64_t i = 0; i < n; ++i) {
      coord[3 * i] = a[i];
      coord[3 * i + 1] = a[i + n];
      coord[3 * i + 2] = a[i + 2 * n];
    }
  } else {
    std::memcpy(coord, a, sizeof(double) * 3 * n);
  }
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_set_point(qmckl_context context, const char transp, const int64_t num,
                                const double* coord, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  if (num <= 0)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_set_point", "Number of points should be >0.");
  if (size_max < 3 * num)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_4, "qmckl_set_point", "Array too small");
  if (transp != 'N' && transp != 'T')
    return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_set_point", "transp should be 'N' or 'T'");
  if (coord == NULL)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_set_point", "coord is a NULL pointer");
  Context* ctx = ctx_of(context);
  qmckl_exit_code rc = store_points(context, ctx->point, transp, num, coord);
  if (rc != QMCKL_SUCCESS) return rc;
  return qmckl_context_touch(context);
}

/* ------------------------------------------------------------------ nuclei */

bool qmckl_nucleus_provided(const qmckl_context context) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return false;
  return ctx_of(context)->nucleus.provided;
}

qmckl_exit_code qmckl_get_nucleus_num(const qmckl_context context, int64_t* const num) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  if (num == NULL)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_nucleus_num", "num is a null pointer");
  Context* ctx = ctx_of(context);
  if (ctx->nucleus.uninitialized & 1) {
    *num = 0;
    return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_get_nucleus_num", "nucleus data is not provided");
  }
  *num = ctx->nucleus.num;
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_get_nucleus_charge(const qmckl_context context, double* const charge,
                                         const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  if (charge == NULL)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_nucleus_charge", "charge is a null pointer");
  Context* ctx = ctx_of(context);
  if (ctx->nucleus.uninitialized & (1 << 1))
    return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_get_nucleus_charge", "nucleus data is not provided");
  if (ctx->nucleus.num > size_max)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_get_nucleus_charge", "Array too small");
  std::memcpy(charge, ctx->nucleus.charge.data(), sizeof(double) * ctx->nucleus.num);
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_get_nucleus_coord(const qmckl_context context, const char transp,
                                        double* const coord, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  if (transp != 'N' && transp != 'T')
    return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_nucleus_coord", "transp should be 'N' or 'T'");
  if (coord == NULL)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_get_nucleus_coord", "coord is a null pointer");
  Context* ctx = ctx_of(context);
  if (ctx->nucleus.uninitialized & (1 << 2))
    return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_get_nucleus_coord", "nucleus data is not provided");
  const int64_t n = ctx->nucleus.num;
  if (size_max < 3 * n)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_4, "qmckl_get_nucleus_coord", "Array too small");
  const double* a = ctx->nucleus.coord.data();
  if (transp == 'N') {
    for (int64_t i = 0; i < n; ++i) {
      coord[3 * i] = a[i];
      coord[3 * i + 1] = a[i + n];
      coord[3 * i + 2] = a[i + 2 * n];
    }
  } else {
    std::memcpy(coord, a, sizeof(double) * 3 * n);
  }
  return QMCKL_SUCCESS;
}

static qmckl_exit_code nucleus_pre(qmckl_context context, int32_t mask) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  Context* ctx = ctx_of(context);
  if (mask != 0 && !(ctx->nucleus.uninitialized & mask))
    return qmckl_failwith(context, QMCKL_ALREADY_SET, "qmckl_set_nucleus_*", NULL);
  return QMCKL_SUCCESS;
}

static qmckl_exit_code nucleus_post(qmckl_context context, int32_t mask) {
  Context* ctx = ctx_of(context);
  ctx->nucleus.uninitialized &= ~mask;
  ctx->nucleus.provided = (ctx->nucleus.uninitialized == 0);
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_set_nucleus_num(qmckl_context context, const int64_t num) {
  const int32_t mask = 1 << 0;
  qmckl_exit_code rc = nucleus_pre(context, mask);
  if (rc != QMCKL_SUCCESS) return rc;
  if (num <= 0) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_set_nucleus_num", "num <= 0");
  ctx_of(context)->nucleus.num = num;
  return nucleus_post(context, mask);
}

qmckl_exit_code qmckl_set_nucleus_charge(qmckl_context context, const double* charge,
                                         const int64_t size_max) {
  const int32_t mask = 1 << 1;
  qmckl_exit_code rc = nucleus_pre(context, mask);
  if (rc != QMCKL_SUCCESS) return rc;
  if (charge == NULL)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_set_nucleus_charge", "charge is a null pointer");
  int64_t num = 0;
  rc = qmckl_get_nucleus_num(context, &num);
  if (rc != QMCKL_SUCCESS) return rc;
  if (num > size_max)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_set_nucleus_charge", "Array too small");
  if (alloc_should_fail())
    return qmckl_failwith(context, QMCKL_ALLOCATION_FAILED, "qmckl_set_nucleus_charge", NULL);
  ctx_of(context)->nucleus.charge.assign(charge, charge + num);
  return nucleus_post(context, mask);
}

qmckl_exit_code qmckl_set_nucleus_coord(qmckl_context context, const char transp,
                                        const double* coord, const int64_t size_max) {
  const int32_t mask = 1 << 2;
  // Nuclear coordinates may be reset (no already-set check), and, as in the
  // reference, setting them does not touch the context (org/qmckl_nucleus.org:541-610).
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  Context* ctx = ctx_of(context);
  const int64_t n = ctx->nucleus.num;
  if (size_max < 3 * n)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_4, "qmckl_set_nucleus_coord", "Array too small");
  if (coord == NULL)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_set_nucleus_coord", "coord is a null pointer");
  if (alloc_should_fail())
    return qmckl_failwith(context, QMCKL_ALLOCATION_FAILED, "qmckl_set_nucleus_coord", NULL);
  ctx->nucleus.coord.assign((size_t)(3 * n), 0.0);
  double* a = ctx->nucleus.coord.data();
  if (transp == 'N') {
    for (int64_t i = 0; i < n; ++i) {
      a[i] = coord[3 * i];
      a[i + n] = coord[3 * i + 1];
      a[i + 2 * n] = coord[3 * i + 2];
    }
  } else {
    std::memcpy(a, coord, sizeof(double) * 3 * n);
  }
  ctx->nucleus.coord_version += 1;
  return nucleus_post(context, mask);
}

/* --------------------------------------------------------------- electrons */

bool qmckl_electron_provided(const qmckl_context context) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return false;
  return ctx_of(context)->electron.provided;
}

qmckl_exit_code qmckl_set_electron_num(qmckl_context context, const int64_t up_num,
                                       const int64_t down_num) {
  const int32_t mask = 1 << 0;
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  Context* ctx = ctx_of(context);
  if (!(ctx->electron.uninitialized & mask))
    return qmckl_failwith(context, QMCKL_ALREADY_SET, "qmckl_set_electron_*", NULL);
  if (up_num <= 0) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_set_electron_num", "up_num <= 0");
  if (down_num < 0) return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_set_electron_num", "down_num < 0");
  ctx->electron.up_num = up_num;
  ctx->electron.down_num = down_num;
  ctx->electron.num = up_num + down_num;
  ctx->electron.uninitialized &= ~mask;
  ctx->electron.provided = (ctx->electron.uninitialized == 0);
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_set_electron_coord(qmckl_context context, const char transp,
                                         const int64_t walk_num, const double* coord,
                                         const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  Context* ctx = ctx_of(context);
  if (transp != 'N' && transp != 'T')
    return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_set_electron_coord", "transp should be 'N' or 'T'");
  if (walk_num <= 0)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_set_electron_coord", "walk_num <= 0");
  if (coord == NULL)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_4, "qmckl_set_electron_coord", "coord is a null pointer");
  const int64_t elec_num = ctx->electron.num;
  if (elec_num == 0)
    return qmckl_failwith(context, QMCKL_FAILURE, "qmckl_set_electron_coord", "elec_num is not set");
  // Swap the current and previous walker sets (org/qmckl_electron.org:356-366).
  // The reference then copies the new current set's point record into the
  // context's (sharing its coordinate array) and overwrites the coordinates;
  // here the record's count and date are taken over and its buffer swapped
  // in, so that the coordinates are copied once, not three times.
  std::swap(ctx->electron.walker, ctx->electron.walker_old);
  PointRec& wp = ctx->electron.walker.point;
  std::swap(ctx->point.coord, wp.coord);
  ctx->point.num = wp.num;
  ctx->point.date = wp.date;
  qmckl_exit_code rc = qmckl_set_point(context, transp, walk_num * elec_num, coord, size_max);
  if (rc != QMCKL_SUCCESS) {
    wp.coord = ctx->point.coord;   // the record keeps its coordinates, as in the reference
    return rc;
  }
  ctx->electron.walker.num = walk_num;
  wp.num = ctx->point.num;
  wp.date = ctx->point.date;
  wp.coord.assign(ctx->point.coord.begin(), ctx->point.coord.end());
  if (ctx->electron.walker_old.num == 0)
    return qmckl_set_electron_coord(context, transp, walk_num, coord, size_max);
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_get_electron_num(const qmckl_context context, int64_t* const num) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  if (num == NULL) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_electron_num", "num is a null pointer");
  Context* ctx = ctx_of(context);
  if (ctx->electron.uninitialized & 1) return QMCKL_NOT_PROVIDED;
  *num = ctx->electron.num;
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_get_electron_up_num(const qmckl_context context, int64_t* const up_num) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  if (up_num == NULL) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_electron_up_num", "up_num is a null pointer");
  Context* ctx = ctx_of(context);
  if (ctx->electron.uninitialized & 1) return QMCKL_NOT_PROVIDED;
  *up_num = ctx->electron.up_num;
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_get_electron_down_num(const qmckl_context context, int64_t* const down_num) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  if (down_num == NULL) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_electron_down_num", "down_num is a null pointer");
  Context* ctx = ctx_of(context);
  if (ctx->electron.uninitialized & 1) return QMCKL_NOT_PROVIDED;
  *down_num = ctx->electron.down_num;
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_get_electron_walk_num(const qmckl_context context, int64_t* const walk_num) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  if (walk_num == NULL) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_electron_walk_num", "walk_num is a null pointer");
  *walk_num = ctx_of(context)->electron.walker.num;
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_get_electron_coord(const qmckl_context context, const char transp,
                                         double* const coord, const int64_t size_max) {
  if (transp != 'N' && transp != 'T')
    return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_electron_coord", "transp should be 'N' or 'T'");
  if (coord == NULL)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_get_electron_coord", "coord is a null pointer");
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  Context* ctx = ctx_of(context);
  if (!ctx->electron.provided)
    return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_get_electron_coord", NULL);
  return qmckl_get_point(context, transp, coord, size_max);
}

qmckl_exit_code qmckl_get_electron_en_distance(qmckl_context context, double* const distance, const int64_t size_max) {
  // org/qmckl_electron.org:1226-1262, 1270-1340: distances between the
  // context's points and the nuclei, [point][nucl], computed on the GPU
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_NULL_CONTEXT;
  Context* ctx = ctx_of(context);
  if (!ctx->nucleus.provided) return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_provide_en_distance", NULL);
  if (distance == NULL)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_get_electron_en_distance", "distance is a null pointer");
  if (size_max < ctx->point.num * ctx->nucleus.num)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_get_electron_en_distance", "size_max < num*nucl_num");
  return dev_en_distance(context, distance);
}

}  // extern "C"
