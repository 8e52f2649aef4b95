// Internal state of a qmckl_b200 context (host side).
//
// The field set mirrors the reference's qmckl_context_struct
// (org/qmckl_context.org:141-188) restricted to what the orbital-evaluation
// path needs: numerical precision, error record, memory registry, the date
// clock, points, nuclei, electrons, the AO basis and the MO basis.  Computed
// arrays (ao_vgl, mo_vgl, ...) live on the GPU in the DeviceState hung off
// `extra` (the reference's `qmckl_extra` hook, org/qmckl_context.org:183-198);
// only their dates live here.
#pragma once

#include <cstdint>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "qmckl.h"

namespace qb {

constexpr uint64_t VALID_TAG = 0xBEEFFACEull;    // org/qmckl_context.org:210-211
constexpr uint64_t INVALID_TAG = 0xDEADBEEFull;

struct ErrorRec {
  qmckl_exit_code exit_code = QMCKL_SUCCESS;
  char function[QMCKL_MAX_FUN_LEN] = {0};
  char message[QMCKL_MAX_MSG_LEN] = {0};
};

struct PointRec {                 // org/qmckl_point.org:105-112
  int64_t num = 0;
  uint64_t date = 0;
  std::vector<double> coord;      // [3][num]: x block, y block, z block
};

struct NucleusRec {               // org/qmckl_nucleus.org:109-122
  int64_t num = 0;
  std::vector<double> charge;
  std::vector<double> coord;      // [3][num]
  uint64_t coord_version = 0;     // bumped by every qmckl_set_nucleus_coord
  int32_t uninitialized = (1 << 3) - 1;
  bool provided = false;
};

struct WalkerRec {
  int64_t num = 0;
  PointRec point;
};

struct ElectronRec {              // org/qmckl_electron.org:144-170
  int64_t num = 0, up_num = 0, down_num = 0;
  WalkerRec walker, walker_old;
  int32_t uninitialized = (1 << 1) - 1;
  bool provided = false;
};

// Per-nucleus tables derived at finalization (org/qmckl_ao.org:2965-3410).
struct AoDerived {
  std::vector<int64_t> nucleus_prim_index;   // [nucl+1]
  std::vector<double> coefficient_normalized; // [prim]
  std::vector<int32_t> nucleus_max_ang_mom;  // [nucl]
  std::vector<double> nucleus_range;         // [nucl]
  std::vector<int32_t> ao_ang_mom;           // [ao]
  std::vector<int64_t> ao_nucl;              // [ao]
  std::vector<int64_t> ao_index;             // [shell+1] first AO of a shell
  // sorted / de-duplicated exponents per nucleus (HPC tables)
  std::vector<int32_t> prim_num_per_nucleus; // [nucl]
  std::vector<int32_t> nuc_prim_start;       // [nucl+1] into expo_sorted
  std::vector<double> expo_sorted;           // concatenated
  // sparse (prim, coef) list per shell over the sorted primitives of its nucleus
  std::vector<int32_t> shell_coef_start;     // [shell+1]
  std::vector<int32_t> coef_prim;            // local index in the nucleus table
  std::vector<double> coef_val;
};

struct AoBasisRec {               // org/qmckl_ao.org:148-206
  int64_t shell_num = 0, prim_num = 0, ao_num = 0;
  std::vector<int64_t> nucleus_index, nucleus_shell_num;
  std::vector<int32_t> r_power, shell_ang_mom;
  std::vector<int64_t> shell_prim_num, shell_prim_index;
  std::vector<double> shell_factor, exponent, coefficient, prim_factor, ao_factor;
  bool r_power_set = false;
  AoDerived d;
  uint64_t basis_version = 0;     // bumped by each finalization
  uint64_t primitive_vgl_date = 0, shell_vgl_date = 0, ao_vgl_date = 0, ao_value_date = 0, ao_hessian_date = 0;
  int32_t uninitialized = (1 << 14) - 1;
  bool provided = false;
  bool ao_cartesian = true;
  char type = 0;
};

struct MoBasisRec {               // org/qmckl_mo.org:127-145
  int64_t mo_num = 0;
  std::vector<double> coefficient;    // [mo][ao]
  std::vector<double> coefficient_t;  // [ao][mo]
  uint64_t coef_version = 0;
  uint64_t mo_vgl_date = 0, mo_value_date = 0, mo_hessian_date = 0;
  // cusp adjustment (org/qmckl_mo.org:479-700): radius per nucleus (empty:
  // none) and the cubic's parameters [nucl][4][mo]
  std::vector<double> r_cusp;
  std::vector<double> cusp_param;
  uint64_t cusp_version = 0;          // bumped whenever either changes
  int32_t uninitialized = (1 << 2) - 1;
  bool provided = false;
};

struct DeviceState;   // device.cu

struct Context {
  uint64_t tag = VALID_TAG;
  uint32_t precision = QMCKL_DEFAULT_PRECISION, range = QMCKL_DEFAULT_RANGE;
  std::recursive_mutex mutex;
  int lock_count = 0;
  int32_t num_threads = 1;
  ErrorRec error;
  std::unordered_map<void*, size_t> memory;   // qmckl_malloc registry
  uint64_t date = 0;
  PointRec point;
  NucleusRec nucleus;
  ElectronRec electron;
  AoBasisRec ao_basis;
  MoBasisRec mo_basis;
  int32_t form = 0;                 // QMCKL_B200_FORM_*
  DeviceState* extra = nullptr;     // the reference's qmckl_extra hook
};

inline Context* ctx_of(qmckl_context c) { return reinterpret_cast<Context*>(c); }

// Device side (device.cu).  All return QMCKL_SUCCESS or an exit code after
// recording the error in the context.
qmckl_exit_code dev_attach(qmckl_context context);
void dev_detach(Context* ctx);
qmckl_exit_code dev_copy(qmckl_context dst, const Context* src);
qmckl_exit_code dev_provide_primitive_vgl(qmckl_context context, double* host_out);
qmckl_exit_code dev_provide_shell_vgl(qmckl_context context, double* host_out);
qmckl_exit_code dev_provide_ao_vgl(qmckl_context context, double* host_out);
qmckl_exit_code dev_provide_ao_value(qmckl_context context, double* host_out);
qmckl_exit_code dev_provide_ao_hessian(qmckl_context context, double* host_out);
qmckl_exit_code dev_provide_forces(qmckl_context context, int which, double* host_out);
qmckl_exit_code dev_provide_mo_vgl(qmckl_context context, double* host_out);
qmckl_exit_code dev_provide_mo_value(qmckl_context context, double* host_out);
qmckl_exit_code dev_provide_mo_hessian(qmckl_context context, double* host_out);
qmckl_exit_code dev_en_distance(qmckl_context context, double* host_out);
qmckl_exit_code dev_invalidate_mo(qmckl_context context);
struct PreparedMixed;
qmckl_exit_code dev_prepared_mixed(qmckl_context context, PreparedMixed* out);
// K-block records of the fused kernels for the basis and nuclei of a context (device.cu)
bool build_krec_records(const Context* ctx, std::vector<uint8_t>& records, int& rec_bytes);
// The same records in the fused kernels' own K order, with the K blocks'
// tile-skipping tables and the AO at each K position (device.cu); the basis
// order when the reordered records would exceed max_rec_bytes.
bool build_fused_records(const Context* ctx, double cutoff, size_t max_rec_bytes, std::vector<uint8_t>& recs,
                         int& rec_bytes, std::vector<uint8_t>& kskip, std::vector<int64_t>& ao_perm);
// Row-bound envelopes of the mixed form's 2-piece float16 operands (device.cu)
void build_envelopes(const Context* ctx, std::vector<float>& env, float& r0, float& inv_log2q);

// AO finalization helpers (ao_basis.cpp)
qmckl_exit_code finalize_basis(qmckl_context context);
qmckl_exit_code finalize_mo_basis(qmckl_context context);

// test hook: number of successful qmckl_malloc / device allocations before an
// injected failure (-1 = never).  Exposed through qmckl_b200_inject_alloc_failure.
extern int64_t g_alloc_fail_countdown;
bool alloc_should_fail();

}  // namespace qb
