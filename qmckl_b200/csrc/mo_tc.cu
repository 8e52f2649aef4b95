// Mixed-precision MO contraction (placeholder until the tcgen05 kernel lands).
#include "mo_tc.cuh"

namespace qb {

TcPlan tc_plan(int64_t ao_num, int64_t mo_num, int pieces) {
  TcPlan p;
  p.ao_num = ao_num; p.mo_num = mo_num; p.pieces = pieces;
  p.k_pad = (ao_num + 63) / 64 * 64;
  p.n_pad = (mo_num + 15) / 16 * 16;
  p.coef_bytes = (size_t)pieces * p.n_pad * p.k_pad * 2;
  return p;
}
size_t tc_a_bytes(const TcPlan& plan, int64_t rows) { return (size_t)plan.pieces * rows * plan.k_pad * 2; }
cudaError_t tc_prepare_coef(const TcPlan&, const double*, void*, cudaStream_t) { return cudaErrorNotSupported; }
cudaError_t tc_run(const DevTables&, const TcPlan&, int64_t, int, const double*, double, const void*, void*, double*,
                   cudaStream_t) {
  return cudaErrorNotSupported;
}

}  // namespace qb
