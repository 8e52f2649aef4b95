// Mixed-form MO VGL with all scratch in a fixed, library-owned device array.
//
// Some callers cannot allocate device memory at the moment they need MO
// values: a QMC code whose device memory is owned by a pool allocator that
// reserved the free memory up front (a new cudaMalloc would fail, and
// cudaFree would hand memory back behind the pool's back).  For them,
// qmckl_b200_mo_vgl_device_noalloc evaluates the mixed form exactly like
// qmckl_b200_mo_vgl_device with the unfused kernels, but its scratch (the
// bfloat16 pieces of the AO matrix) lives in g_scratch below instead of
// device memory allocated by the library.  The caller still passes the
// coordinates and the output buffer.
#include <cstdio>

#include "internal.h"
#include "mo_tc.cuh"
#include "qmckl_b200.h"

namespace qb {
namespace {

// Fixed scratch: 32 MiB of AO pieces.  Every GPU that loads the library holds
// this array until the process exits.
constexpr size_t kScratchBytes = size_t(32) << 20;
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Device address of g_scratch on the current device.  In host code the
// symbol g_scratch is only a host-side stand-in, never a device address.  The
// lookup is repeated on every call (it costs nothing once the module is
// loaded), so a recreated primary context never leaves a stale address.
cudaError_t scratch_address(void** ptr) { return cudaGetSymbolAddress(ptr, g_scratch); }

}  // namespace

// Called by every context's first regular mixed-form evaluation: the first
// lookup loads this file's module and with it the 32 MiB array, at a time
// when the library is allowed to allocate.
cudaError_t noalloc_prime() {
  void* p = nullptr;
  return scratch_address(&p);
}

}  // namespace qb

using namespace qb;

extern "C" qmckl_exit_code qmckl_b200_mo_vgl_device_noalloc(qmckl_context context, const int64_t point_num,
                                                            const double* d_coord, double* d_mo_vgl) {
  const char* fname = "qmckl_b200_mo_vgl_device_noalloc";
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  Context* ctx = ctx_of(context);
  if (!ctx->ao_basis.provided || !ctx->mo_basis.provided)
    return qmckl_failwith(context, QMCKL_NOT_PROVIDED, fname, "AO or MO basis not provided");
  if (point_num < 0) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, fname, "point_num < 0");
  if (point_num > 0 && d_coord == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_3, fname, "NULL pointer");
  if (point_num > 0 && d_mo_vgl == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_4, fname, "NULL pointer");
  PreparedMixed pm;
  qmckl_exit_code rc = dev_prepared_mixed(context, &pm);
  if (rc != QMCKL_SUCCESS) return rc;
  // the largest point count first, so that no product below can overflow
  const int64_t max_points = (int64_t)(kScratchBytes / tc_a_bytes(pm.plan, 5));
  if (point_num > max_points) {
    char msg[QMCKL_MAX_MSG_LEN];
    std::snprintf(msg, sizeof msg,
                  "point_num %lld exceeds the fixed 32 MiB scratch: at most %lld points per call for this basis",
                  (long long)point_num, (long long)max_points);
    return qmckl_failwith(context, QMCKL_INVALID_ARG_2, fname, msg);
  }
  if (point_num == 0) return QMCKL_SUCCESS;
  void* base = nullptr;
  cudaError_t e = scratch_address(&base);
  if (e != cudaSuccess) {
    char msg[QMCKL_MAX_MSG_LEN];
    std::snprintf(msg, sizeof msg, "cudaGetSymbolAddress of the fixed scratch failed: %s", cudaGetErrorString(e));
    return qmckl_failwith(context, QMCKL_FAILURE, fname, msg);
  }
  e = tc_run_scratch(pm.T, pm.plan, point_num, 5, d_coord, pm.cutoff, pm.coef, base, pm.err, d_mo_vgl, pm.stream,
                     pm.cusp_r);
  if (e == cudaSuccess && pm.cusp_r != nullptr)
    e = launch_cusp_mo(point_num, 5, d_coord, point_num, pm.T.nucl_num, pm.T.nucl_coord, pm.cusp_r, pm.cusp_prm,
                       (int)pm.plan.mo_num, d_mo_vgl, pm.stream);
  if (e != cudaSuccess) {
    char msg[QMCKL_MAX_MSG_LEN];
    std::snprintf(msg, sizeof msg, "CUDA error: %s", cudaGetErrorString(e));
    return qmckl_failwith(context, QMCKL_FAILURE, fname, msg);
  }
  return QMCKL_SUCCESS;
}
