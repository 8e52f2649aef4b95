// Device state of a context and the providers of the computed arrays.
//
// The DeviceState hangs off the context's extension pointer (the reference's
// qmckl_extra hook, org/qmckl_context.org:183-198).  Providers mirror the
// reference's date-stamped lazy caches (org/qmckl_ao.org:9035-9225,
// org/qmckl_mo.org:1762-1877): an array is recomputed only when
// ctx->point.date is newer than its date, and its date is then set to
// ctx->date.  Inputs are uploaded when their host version changed: points on
// every new point date, nuclear coordinates on every qmckl_set_nucleus_coord,
// basis tables on every finalization, MO coefficients on every
// finalize_mo_basis / rescale.  The host getters copy the device result into
// the caller's buffer; the qmckl_b200_*_device entry points leave it on the GPU.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "internal.h"
#include "ao_tile.cuh"
#include "kernels.cuh"
#include "mo_tc.cuh"
#include "qmckl_b200.h"

namespace qb {

// Squared radius beyond which every AO of shell s (on nucleus n) vanishes in
// the fused producers: the nucleus is screened out (r^2 > cutoff * range) or
// the shell's smallest exponent a_min, its first primitive, already breaks
// the primitive loop (a_min r^2 > cutoff).  Widened by 1e-12 so that the
// comparison in the kernel is conservative against rounding; -1 for a shell
// without primitives.
double shell_r2max(const Context* ctx, int s, int n, double cutoff) {
  const AoDerived& d = ctx->ao_basis.d;
  if (d.shell_coef_start[s] >= d.shell_coef_start[s + 1]) return -1.0;
  const double a_min = d.expo_sorted[d.nuc_prim_start[n] + d.coef_prim[d.shell_coef_start[s]]];
  const double r2 = std::min(cutoff * d.nucleus_range[n], a_min > 0.0 ? cutoff / a_min : 1e300);
  return r2 * (1.0 + 1e-12);
}

// Records of the fused kernels: one per 64-AO K block, everything its AO
// producers read (layout in fused_common.cuh), from the finalized basis and
// the nuclear coordinates of a context.  rec_bytes is the common record size
// (a multiple of 128).  Returns false when the AOs are not numbered shell by
// shell in increasing order.
//
// `order` (optional) is the sequence of shells along the K dimension (the
// identity when null); then *ao_perm[k] is the AO at K position k, and, for
// the tile skipping of the fused kernel, *kb_sh[kb] the range of positions
// in `order` of block kb's shells and *sph[q] the screening sphere of shell
// order[q]: its nucleus and the squared radius beyond which all its AOs
// vanish (shell_r2max).
bool build_krec_records(const Context* ctx, std::vector<uint8_t>& h, int& rec_bytes,
                        const std::vector<int32_t>* order, std::vector<int64_t>* ao_perm, std::vector<int2>* kb_sh,
                        std::vector<double4>* sph, double cutoff, std::vector<int2>* kpos = nullptr) {
  const AoBasisRec& B = ctx->ao_basis;
  const AoDerived& d = B.d;
  const int64_t A = B.ao_num, N = ctx->nucleus.num, S = B.shell_num;
  if (A <= 0 || (int64_t)ctx->nucleus.coord.size() < 3 * N) return false;
  std::vector<int32_t> aosh(A, -1), code(A, 0), shell_nuc(S, 0);
  for (int64_t m = 0; m < N; ++m)
    for (int64_t s = B.nucleus_index[m]; s < B.nucleus_index[m] + B.nucleus_shell_num[m]; ++s) shell_nuc[s] = (int32_t)m;
  for (int64_t s = 0; s < S; ++s) {
    const int l = B.shell_ang_mom[s];
    int64_t k = d.ao_index[s];
    for (int a = l; a >= 0; --a)
      for (int b = l - a; b >= 0; --b) {
        if (k < A) {
          aosh[k] = (int32_t)s;
          code[k] = a | (b << 4) | ((l - a - b) << 8) | (l << 12);
        }
        ++k;
      }
  }
  for (int64_t k = 0; k < A; ++k)
    if (aosh[k] < 0 || (k > 0 && aosh[k] < aosh[k - 1])) return false;
  // K positions: kq[k] = position in the shell sequence, korig[k] = AO
  std::vector<int32_t> seq(S);
  if (order) {
    if ((int64_t)order->size() != S) return false;
    seq = *order;
  } else {
    for (int64_t q = 0; q < S; ++q) seq[q] = (int32_t)q;
  }
  std::vector<int32_t> kq(A);
  std::vector<int64_t> korig(A);
  if (kpos) kpos->assign(S, make_int2(0, 0));
  {
    int64_t k = 0;
    for (int64_t q = 0; q < S; ++q) {
      const int s = seq[q];
      const int64_t nk = (int64_t)(B.shell_ang_mom[s] + 1) * (B.shell_ang_mom[s] + 2) / 2;
      if (kpos) (*kpos)[q] = make_int2((int)k, (int)nk);
      for (int64_t t = 0; t < nk; ++t, ++k) {
        if (k >= A) return false;
        kq[k] = (int32_t)q;
        korig[k] = d.ao_index[s] + t;
      }
    }
    if (k != A) return false;
  }
  const int64_t nkb = (A + 63) / 64;
  struct KRecShell { double x, y, z, range; int32_t pb, pe; float cusp_r2; int32_t pad; };
  const std::vector<double>& rc = ctx->mo_basis.r_cusp;   // empty: no cusp adjustment
  size_t rec = 0;
  for (int64_t kb = 0; kb < nkb; ++kb) {
    const int64_t k0 = kb * 64, k1 = std::min<int64_t>(k0 + 64, A);
    const int q0 = kq[k0], q1 = kq[k1 - 1];
    size_t np = 0;
    for (int q = q0; q <= q1; ++q) np += d.shell_coef_start[seq[q] + 1] - d.shell_coef_start[seq[q]];
    rec = std::max(rec, 16 + 64 * 8 + (size_t)(q1 - q0 + 1) * sizeof(KRecShell) + np * 16);
  }
  rec = (rec + 127) / 128 * 128;
  h.assign(rec * nkb, 0);
  if (kb_sh) kb_sh->assign(nkb, make_int2(0, 0));
  for (int64_t kb = 0; kb < nkb; ++kb) {
    uint8_t* r = h.data() + kb * rec;
    const int64_t k0 = kb * 64, k1 = std::min<int64_t>(k0 + 64, A);
    const int q0 = kq[k0], q1 = kq[k1 - 1];
    if (kb_sh) (*kb_sh)[kb] = make_int2(q0, q1 + 1);
    int32_t* hdr = (int32_t*)r;
    int32_t* ao = (int32_t*)(r + 16);
    KRecShell* sh = (KRecShell*)(r + 16 + 64 * 8);
    double* prm = (double*)(r + 16 + 64 * 8 + (size_t)(q1 - q0 + 1) * sizeof(KRecShell));
    hdr[0] = q1 - q0 + 1;
    for (int64_t t = 0; t < 64; ++t) {
      const int64_t k = k0 + t;
      if (k < k1) {
        const float f = (float)B.ao_factor[korig[k]];
        ao[2 * t] = code[korig[k]] | ((kq[k] - q0) << 16);
        std::memcpy(&ao[2 * t + 1], &f, 4);
      } else {
        ao[2 * t] = -1;
        ao[2 * t + 1] = 0;
      }
    }
    int np = 0;
    for (int q = q0; q <= q1; ++q) {
      const int sq = seq[q];
      const int n = shell_nuc[sq];
      KRecShell& e = sh[q - q0];
      e.x = ctx->nucleus.coord[n];
      e.y = ctx->nucleus.coord[n + N];
      e.z = ctx->nucleus.coord[n + 2 * N];
      e.range = d.nucleus_range[n];
      e.cusp_r2 = (!rc.empty() && B.shell_ang_mom[sq] == 0) ? (float)(rc[n] * rc[n]) : -1.f;
      e.pad = 0;
      e.pb = np;
      for (int j = d.shell_coef_start[sq]; j < d.shell_coef_start[sq + 1]; ++j) {
        prm[2 * np] = d.expo_sorted[d.nuc_prim_start[n] + d.coef_prim[j]];
        prm[2 * np + 1] = d.coef_val[j];
        ++np;
      }
      e.pe = np;
    }
    hdr[1] = np;
  }
  if (ao_perm) *ao_perm = korig;
  if (sph) {
    sph->resize(S);
    for (int64_t q = 0; q < S; ++q) {
      const int sq = seq[q];
      const int n = shell_nuc[sq];
      (*sph)[q] = make_double4(ctx->nucleus.coord[n], ctx->nucleus.coord[n + N], ctx->nucleus.coord[n + 2 * N],
                               shell_r2max(ctx, sq, n, cutoff));
    }
  }
  rec_bytes = (int)rec;
  return true;
}

bool build_krec_records(const Context* ctx, std::vector<uint8_t>& h, int& rec_bytes) {
  return build_krec_records(ctx, h, rec_bytes, nullptr, nullptr, nullptr, nullptr, 0.0);
}

// Shell order of the fused kernel's K dimension: the shells in three classes
// of their screening radius (the largest third first), each class in Morton
// order (5 bits per axis) of its nucleus over the nuclei's bounding box, ties
// in shell order.  The 64-AO K blocks of the compact classes then hold shells
// of nearby nuclei, which vanish together over a tile of spatially close
// points; on the config-1 molecule 48% of (tile, K block) pairs are then
// entirely zero and skipped, against 5% in the basis order.
std::vector<int32_t> fused_shell_order(const Context* ctx, double cutoff) {
  const AoBasisRec& B = ctx->ao_basis;
  const int64_t S = B.shell_num, N = ctx->nucleus.num;
  std::vector<int32_t> shell_nuc(S, 0);
  for (int64_t m = 0; m < N; ++m)
    for (int64_t s = B.nucleus_index[m]; s < B.nucleus_index[m] + B.nucleus_shell_num[m]; ++s) shell_nuc[s] = (int32_t)m;
  std::vector<double> r2(S);
  for (int64_t s = 0; s < S; ++s) r2[s] = shell_r2max(ctx, (int)s, shell_nuc[s], cutoff);
  std::vector<double> sorted_r2 = r2;
  std::sort(sorted_r2.begin(), sorted_r2.end());
  const double t1 = sorted_r2[S / 3], t2 = sorted_r2[(2 * S) / 3];
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int64_t n = 0; n < N; ++n)
    for (int c = 0; c < 3; ++c) {
      lo[c] = std::min(lo[c], ctx->nucleus.coord[n + c * N]);
      hi[c] = std::max(hi[c], ctx->nucleus.coord[n + c * N]);
    }
  auto morton = [&](int n) {
    uint32_t key = 0;
    for (int c = 0; c < 3; ++c) {
      const double w = hi[c] - lo[c];
      int cell = w > 0.0 ? (int)std::floor((ctx->nucleus.coord[n + c * N] - lo[c]) / w * 32.0) : 0;
      cell = std::min(31, std::max(0, cell));
      for (int b = 0; b < 5; ++b) key |= (uint32_t)((cell >> b) & 1) << (3 * b + c);
    }
    return key;
  };
  std::vector<int64_t> key(S);
  for (int64_t s = 0; s < S; ++s) {
    const int cls = r2[s] >= t2 ? 0 : (r2[s] >= t1 ? 1 : 2);
    key[s] = ((int64_t)cls << 40) | ((int64_t)morton(shell_nuc[s]) << 20) | s;
  }
  std::vector<int32_t> order(S);
  for (int64_t s = 0; s < S; ++s) order[s] = (int32_t)s;
  std::sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return key[a] < key[b]; });
  return order;
}

// Records and tile-skipping tables of the fused kernels in the K order of
// fused_shell_order, or in the basis order when the reordered records would
// exceed max_rec_bytes (the shared memory they get); kskip is laid out as
// the kernels read it (int2 per K block, double4 per shell from
// kskip_sph_offset, int2 K position and AO count per shell from
// kskip_kpos_offset) and ao_perm[k] is the AO at K position k.  False when
// the AO numbering allows no records.
bool build_fused_records(const Context* ctx, double cutoff, size_t max_rec_bytes, std::vector<uint8_t>& recs,
                         int& rec_bytes, std::vector<uint8_t>& kskip, std::vector<int64_t>& ao_perm) {
  const int64_t A = ctx->ao_basis.ao_num, S = ctx->ao_basis.shell_num;
  std::vector<int2> kb_sh, kpos;
  std::vector<double4> sph;
  const std::vector<int32_t> order = fused_shell_order(ctx, cutoff);
  bool ok = build_krec_records(ctx, recs, rec_bytes, &order, &ao_perm, &kb_sh, &sph, cutoff, &kpos) &&
            (size_t)rec_bytes <= max_rec_bytes;
  if (!ok && !build_krec_records(ctx, recs, rec_bytes, nullptr, &ao_perm, &kb_sh, &sph, cutoff, &kpos)) return false;
  const int kblocks = (int)((A + 63) / 64);
  if (kb_sh.empty() || kb_sh.back().y != (int)S) return false;   // the kernels read shell_num there
  kskip.assign(tc_kskip_bytes(A, S), 0);
  std::memcpy(kskip.data(), kb_sh.data(), sizeof(int2) * kb_sh.size());
  std::memcpy(kskip.data() + fz::kskip_sph_offset(kblocks), sph.data(), sizeof(double4) * sph.size());
  std::memcpy(kskip.data() + fz::kskip_kpos_offset(kblocks, (int)S), kpos.data(), sizeof(int2) * kpos.size());
  return true;
}

// Row-bound envelopes of the 2-piece float16 operands (fused_common.cuh
// RowBound) for the basis of a context: env[nucl][3][kEnvCells], and the
// radial cells (r0, 1 / log2 of the cell ratio) shared by all nuclei.
void build_envelopes(const Context* ctx, std::vector<float>& env, float& r0, float& inv_log2q) {
  using fz::kEnvCells;
  const AoBasisRec& B = ctx->ao_basis;
  const AoDerived& d = B.d;
  const int64_t N = ctx->nucleus.num, A = B.ao_num;
  const double cutoff = std::log((double)(((uint64_t)1) << (ctx->precision - 1)));
  double r_far = 1e-2;
  std::vector<double> r_max((size_t)N);
  for (int64_t n = 0; n < N; ++n) {
    r_max[n] = std::sqrt(std::max(0.0, cutoff * d.nucleus_range[n]));
    r_far = std::max(r_far, r_max[n]);
  }
  r0 = 1.0e-3f;
  inv_log2q = (float)((kEnvCells - 2) / std::log2(r_far / r0));
  env.assign((size_t)N * 3 * kEnvCells, 0.f);
  std::vector<double> ex, cf;
  std::vector<ShellBound> sb;
  for (int64_t n = 0; n < N; ++n) {
    ex.clear();
    cf.clear();
    sb.clear();
    std::vector<std::pair<size_t, size_t>> span;
    for (int64_t s = B.nucleus_index[n]; s < B.nucleus_index[n] + B.nucleus_shell_num[n]; ++s) {
      const size_t b0 = ex.size();
      for (int j = d.shell_coef_start[s]; j < d.shell_coef_start[s + 1]; ++j) {
        ex.push_back(d.expo_sorted[d.nuc_prim_start[n] + d.coef_prim[j]]);
        cf.push_back(d.coef_val[j]);
      }
      span.push_back({b0, ex.size()});
      const int l = B.shell_ang_mom[s];
      double f = 0.0;
      for (int64_t k = d.ao_index[s]; k < d.ao_index[s] + (l + 1) * (l + 2) / 2 && k < A; ++k)
        f = std::max(f, std::fabs(B.ao_factor[k]));
      sb.push_back(ShellBound{l, f, nullptr, nullptr, 0});
    }
    for (size_t q = 0; q < sb.size(); ++q) {
      sb[q].expo = ex.data() + span[q].first;
      sb[q].coef = cf.data() + span[q].first;
      sb[q].nprim = (int)(span[q].second - span[q].first);
    }
    tc_envelope(sb.data(), (int)sb.size(), r_max[n], r0, inv_log2q, env.data() + (size_t)n * 3 * kEnvCells);
  }
}

static std::atomic<int64_t> g_launches{0};
constexpr int kSlices = 8;                 // slices of a host-getter evaluation (copy overlap)
constexpr int64_t kSliceMinPoints = 2048;  // slicing only above 8 x this many points
void count_launch(int n) { g_launches += n; }

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
};

struct DeviceState {
  int device = -1;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  bool stream_given = false;     // set by qmckl_b200_set_stream (0 = the legacy default stream)
  // basis tables
  uint64_t basis_version = 0;
  DevBuf tables;
  DevTables T{};
  AoTiles tiles{};
  std::vector<char> host_tables;
  uint64_t nucl_version = ~0ull;
  DevBuf nucl;
  // points
  uint64_t coord_date = ~0ull;
  int64_t coord_num = -1;
  DevBuf coord;
  // outputs
  DevBuf prim_vgl, shell_vgl, ao_vgl, ao_value, mo_vgl, mo_value;
  // MO coefficients (FP64 transpose [ao][mo])
  uint64_t coef_version = ~0ull;
  DevBuf coef_t;
  // mixed form: split-bf16 coefficient pieces and the A-matrix scratch
  TcPlan tc;                       // fused kernel (split_pieces)
  uint64_t tc_coef_version = ~0ull;
  int tc_pieces = 0;
  DevBuf tc_coef, tc_a;
  TcPlan tc3;                      // unfused kernels and the fixed-scratch entry: 3 bfloat16 pieces
  uint64_t tc3_coef_version = ~0ull;
  DevBuf tc3_coef;
  // row-bound envelopes of the float16 operands (per basis)
  DevBuf env;
  // orbital forces: AO range of each nucleus and the output buffer
  DevBuf nuc_ao, forces;
  uint64_t nuc_ao_version = ~0ull;
  // host getters: slices of the evaluation copied out on a second stream
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t slice_ev[8] = {};
  uint64_t env_basis_version = ~0ull;
  float env_r0 = 0.f, env_inv_log2q = 0.f;
  int32_t split_pieces = 3;   // bfloat16 x 3; 2 = float16 x 2 with row / MO scales (split.cuh)
  // mixed form: fused AO -> MO kernel (default) instead of AO pieces in device memory + GEMM
  bool fused = true;
  // per-K-block records of the fused kernel (rebuilt on basis or nuclear moves)
  DevBuf krec;
  DevBuf order;      // point order of the fused kernel: keys[P], perm[P], cell counts
  int rec_bytes = 0;
  uint64_t krec_basis_version = ~0ull, krec_nucl_version = ~0ull;
  // derivatives: AO Hessian and the MO VGL adjoint (FP64 coefficient [mo][ao],
  // per-chunk coordinates, AO / pulled-back weight buffer, split-K partials)
  DevBuf ao_hessian;
  uint64_t coef_rows_version = ~0ull;
  DevBuf coef_rows, adj_coord, adj_buf, adj_part, adj_nucl;
  // mixed-form adjoint: bfloat16 pieces of the weights and of coefficient_t
  uint64_t adj_ct_version = ~0ull;
  DevBuf adj_wp, adj_ct;
  // cusp adjustment: radii [nucl] followed by the cubics' parameters
  // [nucl][4][mo]; AO arrays with the left-out AOs zeroed, which feed only the
  // MO step; point-nucleus distances; MO Hessian
  uint64_t cusp_version = ~0ull, krec_cusp_version = ~0ull;
  DevBuf cusp, ao_masked, en_dist, mo_hessian;
  // fused kernel: K order (AO at each K position; the coefficient pieces of
  // the fused plan follow it), tile-skipping tables, cutoff they were built for
  std::vector<int64_t> fused_perm;
  DevBuf kskip, kstat;   // kstat: 16-AO k-steps issued / dense, summed over the fused launches
  double krec_cutoff = -1.0;
  // error word of the mixed form's tensor-core kernels: a bounded barrier
  // wait that gives up writes its code here; it is read (and cleared) at the
  // context's next synchronization point, never by the evaluation itself
  DevBuf tc_err;
  // tile-sparse FP64 contraction: screening spheres and AO ranges of the
  // shells (basis order), coefficient_t with an even row length when the MO
  // count is odd
  uint64_t f64_sph_basis = ~0ull, f64_sph_nucl = ~0ull;
  double f64_sph_cutoff = -1.0;
  uint64_t coef_f_version = ~0ull;
  DevBuf f64_sph, coef_f;
};

namespace {

qmckl_exit_code cuda_fail(qmckl_context context, cudaError_t e, const char* where) {
  char msg[QMCKL_MAX_MSG_LEN];
  std::snprintf(msg, sizeof msg, "CUDA error: %s", cudaGetErrorString(e));
  return qmckl_failwith(context, QMCKL_FAILURE, where, msg);
}

#define QB_CUDA(expr, where)                                  \
  do {                                                        \
    cudaError_t e_ = (expr);                                  \
    if (e_ != cudaSuccess) return cuda_fail(context, e_, where); \
  } while (0)

qmckl_exit_code ensure(qmckl_context context, DevBuf& b, size_t bytes, const char* where) {
  if (b.cap >= bytes && b.p != nullptr) return QMCKL_SUCCESS;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
  if (alloc_should_fail()) return qmckl_failwith(context, QMCKL_ALLOCATION_FAILED, where, "device allocation");
  cudaError_t e = cudaMalloc(&b.p, std::max<size_t>(bytes, 256));
  if (e != cudaSuccess) {
    cudaGetLastError();
    b.p = nullptr;
    char msg[QMCKL_MAX_MSG_LEN];
    std::snprintf(msg, sizeof msg, "device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    return qmckl_failwith(context, QMCKL_ALLOCATION_FAILED, where, msg);
  }
  b.cap = std::max<size_t>(bytes, 256);
  return QMCKL_SUCCESS;
}

void release(DevBuf& b) {
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
}

double cutoff_of(const Context* ctx) {
  // org/qmckl_ao.org:7814
  return std::log((double)(((uint64_t)1) << (ctx->precision - 1)));
}

bool use_mixed(const Context* ctx) {
  if (ctx->form == QMCKL_B200_FORM_MIXED) return true;
  if (ctx->form == QMCKL_B200_FORM_FP64) return false;
  return ctx->precision <= 26;
}

// Pack the finalized basis into one device allocation.
qmckl_exit_code upload_tables(qmckl_context context, DeviceState* ds) {
  Context* ctx = ctx_of(context);
  const AoBasisRec& B = ctx->ao_basis;
  const AoDerived& d = B.d;
  const int64_t N = ctx->nucleus.num, S = B.shell_num, Pn = B.prim_num, A = B.ao_num;

  // nucleus blocks
  std::vector<int4> blocks;
  std::vector<int2> block_slots;
  std::vector<int32_t> slot_nuc;
  std::vector<int2> slot_coef;
  std::vector<int32_t> ao_code(A, 0);
  for (int64_t n = 0; n < N; ++n) {
    if (B.nucleus_shell_num[n] > kBlockSlots)
      return qmckl_failwith(context, QMCKL_FAILURE, "qmckl_b200_upload_basis",
                            "more than 64 shells on one nucleus is not supported");
  }
  // The lanes of a warp stage a block's shells 32 at a time, each pass
  // lasting as long as its longest primitive list; slots are therefore
  // numbered by descending primitive count (ties in shell order), so that
  // the long contracted shells share a pass (config-1 molecule: 89 instead
  // of 131 primitive steps per point).  Results do not depend on the order.
  std::vector<std::pair<int64_t, int64_t>> blk_shells;   // (shell, nucleus)
  int64_t n = 0;
  while (n < N) {
    const int nb = (int)n;
    const int slot_begin = (int)slot_nuc.size();
    int64_t ao_begin = -1, ao_end = -1;
    blk_shells.clear();
    while (n < N && (n - nb) < kBlockNuc && (int64_t)blk_shells.size() + B.nucleus_shell_num[n] <= kBlockSlots) {
      for (int64_t s = B.nucleus_index[n]; s < B.nucleus_index[n] + B.nucleus_shell_num[n]; ++s)
        blk_shells.emplace_back(s, n);
      ++n;
    }
    std::stable_sort(blk_shells.begin(), blk_shells.end(), [&](const auto& u, const auto& v) {
      return d.shell_coef_start[u.first + 1] - d.shell_coef_start[u.first] >
             d.shell_coef_start[v.first + 1] - d.shell_coef_start[v.first];
    });
    for (size_t i = 0; i < blk_shells.size(); ++i) {
      const int64_t s = blk_shells[i].first, sn = blk_shells[i].second;
      const int slot = (int)i;
      slot_nuc.push_back((int32_t)sn);
      slot_coef.push_back(make_int2(d.shell_coef_start[s], d.shell_coef_start[s + 1]));
      const int l = B.shell_ang_mom[s];
      const int64_t k0 = d.ao_index[s];
      int64_t k = k0;
      for (int a = l; a >= 0; --a)
        for (int b = l - a; b >= 0; --b) {
          const int c = l - a - b;
          ao_code[k] = a | (b << 4) | (c << 8) | (l << 12) | (slot << 16) | ((int)(sn - nb) << 24);
          ++k;
        }
      if (ao_begin < 0 || k0 < ao_begin) ao_begin = k0;
      if (k > ao_end) ao_end = k;
    }
    if (ao_begin < 0) { ao_begin = 0; ao_end = 0; }
    blocks.push_back(make_int4(nb, (int)n, (int)ao_begin, (int)ao_end));
    block_slots.push_back(make_int2(slot_begin, (int)slot_nuc.size()));
  }
  // AO ranges of consecutive blocks must tile [0, A): true when the shells of
  // each nucleus are numbered consecutively, which the AO numbering implies.
  {
    int64_t expect = 0;
    for (auto& b4 : blocks) {
      if (b4.z != expect && b4.w > b4.z)
        return qmckl_failwith(context, QMCKL_FAILURE, "qmckl_b200_upload_basis", "AOs are not ordered by nucleus");
      if (b4.w > b4.z) expect = b4.w;
    }
  }
  std::vector<int32_t> prim_nuc(Pn, 0);
  for (int64_t m = 0; m < N; ++m)
    for (int64_t q = d.nucleus_prim_index[m]; q < d.nucleus_prim_index[m + 1] && q < Pn; ++q) prim_nuc[q] = (int32_t)m;
  std::vector<int32_t> shell_nuc(S, 0);
  std::vector<int2> shell_prims(S);
  for (int64_t m = 0; m < N; ++m)
    for (int64_t s = B.nucleus_index[m]; s < B.nucleus_index[m] + B.nucleus_shell_num[m]; ++s) shell_nuc[s] = (int32_t)m;
  for (int64_t s = 0; s < S; ++s)
    shell_prims[s] = make_int2((int)B.shell_prim_index[s], (int)(B.shell_prim_index[s] + B.shell_prim_num[s]));
  // prim_nuc for primitives via their shells (covers any ordering)
  for (int64_t s = 0; s < S; ++s)
    for (int64_t q = B.shell_prim_index[s]; q < B.shell_prim_index[s] + B.shell_prim_num[s]; ++q) prim_nuc[q] = shell_nuc[s];

  // layout: [offset of each array, 256-byte aligned]
  std::vector<char>& H = ds->host_tables;
  H.clear();
  auto put = [&](const void* src, size_t bytes) -> size_t {
    size_t off = (H.size() + 255) & ~size_t(255);
    H.resize(off + std::max<size_t>(bytes, 1));
    if (bytes) std::memcpy(H.data() + off, src, bytes);
    return off;
  };
  const size_t o_range = put(d.nucleus_range.data(), sizeof(double) * N);
  const size_t o_nps = put(d.nuc_prim_start.data(), sizeof(int32_t) * (N + 1));
  const size_t o_expo = put(d.expo_sorted.data(), sizeof(double) * d.expo_sorted.size());
  const size_t o_block = put(blocks.data(), sizeof(int4) * blocks.size());
  const size_t o_bslot = put(block_slots.data(), sizeof(int2) * block_slots.size());
  const size_t o_snuc = put(slot_nuc.data(), sizeof(int32_t) * slot_nuc.size());
  const size_t o_scoef = put(slot_coef.data(), sizeof(int2) * slot_coef.size());
  const size_t o_cprim = put(d.coef_prim.data(), sizeof(int32_t) * d.coef_prim.size());
  const size_t o_cval = put(d.coef_val.data(), sizeof(double) * d.coef_val.size());
  const size_t o_code = put(ao_code.data(), sizeof(int32_t) * A);
  const size_t o_fac = put(B.ao_factor.data(), sizeof(double) * A);
  const size_t o_pnuc = put(prim_nuc.data(), sizeof(int32_t) * Pn);
  const size_t o_pexp = put(B.exponent.data(), sizeof(double) * Pn);
  const size_t o_pcoef = put(d.coefficient_normalized.data(), sizeof(double) * Pn);
  const size_t o_shnuc = put(shell_nuc.data(), sizeof(int32_t) * S);
  const size_t o_shpr = put(shell_prims.data(), sizeof(int2) * S);
  std::vector<int32_t> ao_shell(A, 0);
  std::vector<int2> shell_coef(S);
  for (int64_t s = 0; s < S; ++s) {
    shell_coef[s] = make_int2(d.shell_coef_start[s], d.shell_coef_start[s + 1]);
    const int l = B.shell_ang_mom[s];
    for (int64_t k = d.ao_index[s]; k < d.ao_index[s] + (l + 1) * (l + 2) / 2 && k < A; ++k) ao_shell[k] = (int32_t)s;
  }
  const size_t o_aosh = put(ao_shell.data(), sizeof(int32_t) * A);
  const size_t o_shco = put(shell_coef.data(), sizeof(int2) * S);
  // (exponent, coefficient) of every coefficient entry, for one load per primitive
  std::vector<double2> coef_ac(d.coef_val.size());
  for (int64_t sh = 0; sh < S; ++sh)
    for (int j = d.shell_coef_start[sh]; j < d.shell_coef_start[sh + 1]; ++j)
      coef_ac[j] = make_double2(d.expo_sorted[d.nuc_prim_start[shell_nuc[sh]] + d.coef_prim[j]], d.coef_val[j]);
  const size_t o_cac = put(coef_ac.data(), sizeof(double2) * coef_ac.size());
  // AO tiles of the tiled kernels (ao_tile.cu)
  std::vector<int4> tiles;
  std::vector<int2> tile_nuc;
  std::vector<int32_t> ao_tcode(A, 0);
  {
    bool ordered = true;
    for (int64_t k = 1; k < A; ++k) ordered = ordered && ao_shell[k] >= ao_shell[k - 1];
    for (int64_t s = 1; s < S; ++s) ordered = ordered && shell_nuc[s] >= shell_nuc[s - 1];
    int64_t k = 0;
    while (ordered && k < A) {
      int64_t width = 64;
      for (;;) {
        const int64_t ke = std::min<int64_t>(k + width, A);
        const int s0 = ao_shell[k], s1 = ao_shell[ke - 1];
        const int n0 = shell_nuc[s0], n1 = shell_nuc[s1];
        if ((s1 - s0 + 1 <= kTileShells && n1 - n0 + 1 <= kTileNuc) || width == 8) {
          if (s1 - s0 + 1 > kTileShells || n1 - n0 + 1 > kTileNuc) { ordered = false; break; }
          tiles.push_back(make_int4((int)k, (int)ke, s0, s1 + 1));
          tile_nuc.push_back(make_int2(n0, n1 + 1));
          for (int64_t q = k; q < ke; ++q)
            ao_tcode[q] = (ao_code[q] & 0xFFFF) | ((ao_shell[q] - s0) << 16) | ((shell_nuc[ao_shell[q]] - n0) << 21);
          k = ke;
          break;
        }
        width /= 2;
      }
    }
    if (!ordered || tiles.size() > 65535) { tiles.clear(); tile_nuc.clear(); }
  }
  const size_t o_tile = put(tiles.data(), sizeof(int4) * tiles.size());
  const size_t o_tnuc = put(tile_nuc.data(), sizeof(int2) * tile_nuc.size());
  const size_t o_tcode = put(ao_tcode.data(), sizeof(int32_t) * A);
  qmckl_exit_code rc = ensure(context, ds->tables, H.size(), "qmckl_b200_upload_basis");
  if (rc != QMCKL_SUCCESS) return rc;
  QB_CUDA(cudaMemcpyAsync(ds->tables.p, H.data(), H.size(), cudaMemcpyHostToDevice, ds->stream), "qmckl_b200_upload_basis");
  char* base = (char*)ds->tables.p;
  DevTables& T = ds->T;
  T.nucl_num = (int32_t)N;
  T.shell_num = (int32_t)S;
  T.prim_num = (int32_t)Pn;
  T.ao_num = (int32_t)A;
  T.nblock = (int32_t)blocks.size();
  T.nslot = (int32_t)slot_nuc.size();
  T.nucleus_range = (const double*)(base + o_range);
  T.nuc_prim_start = (const int32_t*)(base + o_nps);
  T.expo = (const double*)(base + o_expo);
  T.block = (const int4*)(base + o_block);
  T.block_slots = (const int2*)(base + o_bslot);
  T.slot_nuc = (const int32_t*)(base + o_snuc);
  T.slot_coef = (const int2*)(base + o_scoef);
  T.coef_prim = (const int32_t*)(base + o_cprim);
  T.coef_val = (const double*)(base + o_cval);
  T.ao_code = (const int32_t*)(base + o_code);
  T.ao_factor = (const double*)(base + o_fac);
  T.prim_nuc = (const int32_t*)(base + o_pnuc);
  T.prim_expo = (const double*)(base + o_pexp);
  T.prim_coef = (const double*)(base + o_pcoef);
  T.shell_nuc = (const int32_t*)(base + o_shnuc);
  T.shell_prims = (const int2*)(base + o_shpr);
  T.ao_shell = (const int32_t*)(base + o_aosh);
  T.shell_coef = (const int2*)(base + o_shco);
  T.coef_ac = (const double2*)(base + o_cac);
  ds->tiles.ntiles = (int32_t)tiles.size();
  ds->tiles.tile = (const int4*)(base + o_tile);
  ds->tiles.tile_nuc = (const int2*)(base + o_tnuc);
  ds->tiles.ao_tcode = (const int32_t*)(base + o_tcode);
  ds->basis_version = B.basis_version;
  ds->nucl_version = ~0ull;   // re-point the nuclear coordinates below
  return QMCKL_SUCCESS;
}

qmckl_exit_code sync_inputs(qmckl_context context, DeviceState* ds, bool need_points, bool need_tables = true) {
  Context* ctx = ctx_of(context);
  if (need_tables && (ds->basis_version != ctx->ao_basis.basis_version || ds->tables.p == nullptr)) {
    qmckl_exit_code rc = upload_tables(context, ds);
    if (rc != QMCKL_SUCCESS) return rc;
  }
  if (ds->nucl_version != ctx->nucleus.coord_version) {
    const int64_t N = ctx->nucleus.num;
    if ((int64_t)ctx->nucleus.coord.size() < 3 * N)
      return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_b200_upload_nucleus", "nuclear coordinates are not set");
    qmckl_exit_code rc = ensure(context, ds->nucl, sizeof(double) * 3 * N, "qmckl_b200_upload_nucleus");
    if (rc != QMCKL_SUCCESS) return rc;
    QB_CUDA(cudaMemcpyAsync(ds->nucl.p, ctx->nucleus.coord.data(), sizeof(double) * 3 * N,
                            cudaMemcpyHostToDevice, ds->stream), "qmckl_b200_upload_nucleus");
    ds->nucl_version = ctx->nucleus.coord_version;
  }
  ds->T.nucl_coord = (const double*)ds->nucl.p;
  if (need_points && (ds->coord_date != ctx->point.date || ds->coord_num != ctx->point.num)) {
    const int64_t P = ctx->point.num;
    qmckl_exit_code rc = ensure(context, ds->coord, sizeof(double) * 3 * std::max<int64_t>(P, 1), "qmckl_b200_upload_points");
    if (rc != QMCKL_SUCCESS) return rc;
    if (P > 0)
      QB_CUDA(cudaMemcpyAsync(ds->coord.p, ctx->point.coord.data(), sizeof(double) * 3 * P,
                              cudaMemcpyHostToDevice, ds->stream), "qmckl_b200_upload_points");
    ds->coord_date = ctx->point.date;
    ds->coord_num = P;
  }
  return QMCKL_SUCCESS;
}

qmckl_exit_code sync_coef(qmckl_context context, DeviceState* ds) {
  Context* ctx = ctx_of(context);
  if (ds->coef_version == ctx->mo_basis.coef_version && ds->coef_t.p) return QMCKL_SUCCESS;
  const int64_t A = ctx->ao_basis.ao_num, M = ctx->mo_basis.mo_num;
  qmckl_exit_code rc = ensure(context, ds->coef_t, sizeof(double) * A * M, "qmckl_b200_upload_mo");
  if (rc != QMCKL_SUCCESS) return rc;
  QB_CUDA(cudaMemcpyAsync(ds->coef_t.p, ctx->mo_basis.coefficient_t.data(), sizeof(double) * A * M,
                          cudaMemcpyHostToDevice, ds->stream), "qmckl_b200_upload_mo");
  ds->coef_version = ctx->mo_basis.coef_version;
  return QMCKL_SUCCESS;
}

// Radii and cubic parameters of the cusp adjustment on the device (*r, *prm);
// both null when the context has none.
qmckl_exit_code sync_cusp(qmckl_context context, DeviceState* ds, const double** r, const double** prm) {
  Context* ctx = ctx_of(context);
  *r = *prm = nullptr;
  if (ctx->mo_basis.r_cusp.empty()) return QMCKL_SUCCESS;
  const int64_t N = ctx->nucleus.num, M = ctx->mo_basis.mo_num;
  const size_t nb = sizeof(double) * (size_t)N, pb = sizeof(double) * (size_t)(N * 4 * M);
  if (ds->cusp_version != ctx->mo_basis.cusp_version || !ds->cusp.p || ds->cusp.cap < nb + pb) {
    qmckl_exit_code rc = ensure(context, ds->cusp, nb + pb, "qmckl_b200_upload_cusp");
    if (rc != QMCKL_SUCCESS) return rc;
    QB_CUDA(cudaMemcpyAsync(ds->cusp.p, ctx->mo_basis.r_cusp.data(), nb, cudaMemcpyHostToDevice, ds->stream),
            "qmckl_b200_upload_cusp");
    QB_CUDA(cudaMemcpyAsync((char*)ds->cusp.p + nb, ctx->mo_basis.cusp_param.data(), pb, cudaMemcpyHostToDevice,
                            ds->stream),
            "qmckl_b200_upload_cusp");
    ds->cusp_version = ctx->mo_basis.cusp_version;
  }
  *r = (const double*)ds->cusp.p;
  *prm = (const double*)((const char*)ds->cusp.p + nb);
  return QMCKL_SUCCESS;
}

// Wait for the context's stream, then report (and clear) a bounded barrier
// wait that gave up in a tensor-core kernel since the last check.
qmckl_exit_code sync_and_check(qmckl_context context, DeviceState* ds, const char* where) {
  int h = 0;
  if (ds->tc_err.p != nullptr)
    QB_CUDA(cudaMemcpyAsync(&h, ds->tc_err.p, sizeof(int), cudaMemcpyDeviceToHost, ds->stream), where);
  QB_CUDA(cudaStreamSynchronize(ds->stream), where);
  if (h != 0) {
    QB_CUDA(cudaMemsetAsync(ds->tc_err.p, 0, sizeof(int), ds->stream), where);
    QB_CUDA(cudaStreamSynchronize(ds->stream), where);
    char msg[QMCKL_MAX_MSG_LEN];
    std::snprintf(msg, sizeof msg,
                  "a bounded barrier wait of a tensor-core kernel gave up (code %d): the mixed-form results "
                  "enqueued since the last synchronization are not valid",
                  h);
    return qmckl_failwith(context, QMCKL_FAILURE, where, msg);
  }
  return QMCKL_SUCCESS;
}

qmckl_exit_code copy_out(qmckl_context context, DeviceState* ds, double* host, const void* dev, size_t bytes,
                         const char* where) {
  if (host != nullptr && bytes > 0)
    QB_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, ds->stream), where);
  return sync_and_check(context, ds, where);
}

DeviceState* state(qmckl_context context) { return ctx_of(context)->extra; }

// ---- compute steps on the device (no date logic) ----

// cusp_r (optional): zero the AOs that the cusp adjustment leaves out of the
// MOs (the array then only feeds the MO step).
qmckl_exit_code run_ao_vgl(qmckl_context context, DeviceState* ds, int64_t P, const double* coord, double* out,
                           const double* cusp_r = nullptr) {
  Context* ctx = ctx_of(context);
  QB_CUDA(launch_ao_vgl_f64(ds->T, P, coord, cutoff_of(ctx), ctx->precision > 23, out, ds->stream, cusp_r),
          "qmckl_b200_ao_vgl");
  return QMCKL_SUCCESS;
}

qmckl_exit_code run_ao_value(qmckl_context context, DeviceState* ds, int64_t P, const double* coord, double* out,
                             const double* cusp_r = nullptr) {
  Context* ctx = ctx_of(context);
  QB_CUDA(launch_ao_value_f64(ds->T, P, coord, cutoff_of(ctx), ctx->precision > 23, out, ds->stream, cusp_r),
          "qmckl_b200_ao_value");
  return QMCKL_SUCCESS;
}

// The fused kernel's device tables: K-block records in the shell order of
// fused_shell_order (or the basis order when the reordered records do not fit
// the kernel's shared memory), the tile-skipping tables, and the coefficient
// pieces of the fused plan in the same K order.  *usable = false when the AO
// numbering allows no records or the kernel does not fit (the unfused kernels
// are used then).
// The fused K order: K-block records, tile-skipping tables and fused_perm
// (rebuilt on basis, nuclear, cusp or precision changes).  *ok = false when
// the AO numbering allows no records.
qmckl_exit_code prepare_korder(qmckl_context context, DeviceState* ds, bool* ok) {
  const char* fname = "qmckl_b200_mo_korder";
  Context* ctx = ctx_of(context);
  *ok = false;
  const int64_t A = ctx->ao_basis.ao_num, M = ctx->mo_basis.mo_num;
  const double cutoff = cutoff_of(ctx);
  const TcPlan plan = tc_plan_fused(A, M, ds->split_pieces);
  // the VGL kernel decides the order; the value kernel (128-point tiles) may
  // still not fit, which run_mo_mixed checks per call
  auto fits = [&](int rec) { return tc_fused_smem(plan, 5, rec) <= 232448; };
  const bool fresh = ds->krec.p != nullptr && ds->kskip.p != nullptr &&
                     ds->krec_basis_version == ctx->ao_basis.basis_version &&
                     ds->krec_nucl_version == ctx->nucleus.coord_version &&
                     ds->krec_cusp_version == ctx->mo_basis.cusp_version && ds->krec_cutoff == cutoff;
  if (!fresh) {
    std::vector<uint8_t> h, ks;
    std::vector<int64_t> perm;
    int rec = 0;
    // the largest record that keeps the VGL kernel within its shared memory
    size_t max_rec = 128;
    while (fits((int)(max_rec + 128))) max_rec += 128;
    if (!build_fused_records(ctx, cutoff, max_rec, h, rec, ks, perm)) return QMCKL_SUCCESS;
    qmckl_exit_code rc = ensure(context, ds->krec, h.size(), fname);
    if (rc != QMCKL_SUCCESS) return rc;
    const size_t kbytes = ks.size();
    rc = ensure(context, ds->kskip, kbytes, fname);
    if (rc != QMCKL_SUCCESS) return rc;
    QB_CUDA(cudaMemcpy(ds->krec.p, h.data(), h.size(), cudaMemcpyHostToDevice), fname);
    QB_CUDA(cudaMemcpy(ds->kskip.p, ks.data(), kbytes, cudaMemcpyHostToDevice), fname);
    ds->rec_bytes = rec;
    ds->krec_basis_version = ctx->ao_basis.basis_version;
    ds->krec_nucl_version = ctx->nucleus.coord_version;
    ds->krec_cusp_version = ctx->mo_basis.cusp_version;
    ds->krec_cutoff = cutoff;
    if (perm != ds->fused_perm) {
      ds->fused_perm = std::move(perm);
      ds->tc_coef_version = ~0ull;   // the coefficient pieces follow the K order
    }
  }
  *ok = true;
  return QMCKL_SUCCESS;
}

// The fused kernel's device tables: the K order above, and the coefficient
// pieces of the fused plan in the same K order.  *usable = false when the AO
// numbering allows no records or the kernel does not fit (the unfused
// kernels are used then).
qmckl_exit_code prepare_fused(qmckl_context context, DeviceState* ds, bool* usable) {
  const char* fname = "qmckl_b200_mo_mixed";
  Context* ctx = ctx_of(context);
  *usable = false;
  const int64_t A = ctx->ao_basis.ao_num, M = ctx->mo_basis.mo_num;
  const int pieces = ds->split_pieces;
  const TcPlan plan = tc_plan_fused(A, M, pieces);
  bool ok = false;
  qmckl_exit_code rc0 = prepare_korder(context, ds, &ok);
  if (rc0 != QMCKL_SUCCESS || !ok) return rc0;
  if (tc_fused_smem(plan, 5, ds->rec_bytes) > 232448) return QMCKL_SUCCESS;
  if (ds->kstat.p == nullptr) {
    qmckl_exit_code rc = ensure(context, ds->kstat, 2 * sizeof(unsigned long long), fname);
    if (rc != QMCKL_SUCCESS) return rc;
    QB_CUDA(cudaMemsetAsync(ds->kstat.p, 0, 2 * sizeof(unsigned long long), ds->stream), fname);
  }
  if (ds->tc_coef_version != ctx->mo_basis.coef_version || ds->tc_pieces != pieces || !ds->tc_coef.p ||
      ds->tc.n_tile != plan.n_tile || ds->tc.nacc != plan.nacc) {
    // coefficient columns in the K order of the records
    std::vector<double> cp((size_t)(M * A));
    const std::vector<double>& c = ctx->mo_basis.coefficient;
    for (int64_t i = 0; i < M; ++i)
      for (int64_t k = 0; k < A; ++k) cp[i * A + k] = c[i * A + ds->fused_perm[k]];
    qmckl_exit_code rc = ensure(context, ds->tc_coef, plan.coef_bytes, fname);
    if (rc != QMCKL_SUCCESS) return rc;
    QB_CUDA(tc_prepare_coef(plan, cp.data(), ds->tc_coef.p, ds->stream), fname);
    ds->tc = plan;
    ds->tc_coef_version = ctx->mo_basis.coef_version;
    ds->tc_pieces = pieces;
  }
  *usable = true;
  return QMCKL_SUCCESS;
}

// Coefficient pieces of the unfused plan (3 bfloat16 pieces) and the
// row-bound envelopes on the device.
qmckl_exit_code prepare_mixed(qmckl_context context, DeviceState* ds) {
  Context* ctx = ctx_of(context);
  const int64_t A = ctx->ao_basis.ao_num, M = ctx->mo_basis.mo_num;
  if (ds->tc_err.p == nullptr) {
    qmckl_exit_code rc = ensure(context, ds->tc_err, sizeof(int), "qmckl_b200_mo_mixed");
    if (rc != QMCKL_SUCCESS) return rc;
    QB_CUDA(cudaMemsetAsync(ds->tc_err.p, 0, sizeof(int), ds->stream), "qmckl_b200_mo_mixed");
    // the allocation-free entry point's code and fixed scratch are loaded
    // now, with this allocating call (a failure here only matters to it, and
    // it reports its own)
    if (tc_prime_unfused() != cudaSuccess || noalloc_prime() != cudaSuccess) cudaGetLastError();
  }
  if (ds->tc3_coef_version != ctx->mo_basis.coef_version || !ds->tc3_coef.p) {
    TcPlan plan = tc_plan(A, M, 3);
    qmckl_exit_code rc = ensure(context, ds->tc3_coef, plan.coef_bytes, "qmckl_b200_mo_mixed");
    if (rc != QMCKL_SUCCESS) return rc;
    QB_CUDA(tc_prepare_coef(plan, ctx->mo_basis.coefficient.data(), ds->tc3_coef.p, ds->stream), "qmckl_b200_mo_mixed");
    ds->tc3 = plan;
    ds->tc3_coef_version = ctx->mo_basis.coef_version;
  }
  if (ds->env_basis_version != ctx->ao_basis.basis_version || !ds->env.p) {
    std::vector<float> env;
    float r0 = 0.f, il = 0.f;
    build_envelopes(ctx, env, r0, il);
    qmckl_exit_code rc = ensure(context, ds->env, sizeof(float) * std::max<size_t>(env.size(), 1), "qmckl_b200_mo_mixed");
    if (rc != QMCKL_SUCCESS) return rc;
    if (!env.empty())
      QB_CUDA(cudaMemcpy(ds->env.p, env.data(), sizeof(float) * env.size(), cudaMemcpyHostToDevice), "qmckl_b200_mo_mixed");
    ds->env_r0 = r0;
    ds->env_inv_log2q = il;
    ds->env_basis_version = ctx->ao_basis.basis_version;
  }
  return QMCKL_SUCCESS;
}

// Box of the nuclei, widened by 4 bohr: the grid of the spatial point order.
void nucleus_box(const Context* ctx, double* lo, double* hi) {
  const int64_t N = ctx->nucleus.num;
  for (int d = 0; d < 3; ++d) {
    lo[d] = 1e300;
    hi[d] = -1e300;
  }
  for (int64_t n = 0; n < N; ++n)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], ctx->nucleus.coord[n + d * N] - 4.0);
      hi[d] = std::max(hi[d], ctx->nucleus.coord[n + d * N] + 4.0);
    }
}

// FP64 MO contraction out[p][c][mo] = sum_k ao[p][c][k] coefficient_t[k][mo]
// of P points (coordinates coord with stride cstride), tile-sparse: points
// in spatial tiles, and for each tile only the AOs of the shells that reach
// one of its points (the others are exact zeros there), summed in the basis
// order.
qmckl_exit_code contract_f64(qmckl_context context, DeviceState* ds, int64_t P, int comps, const double* coord,
                             int64_t cstride, const double* ao, double* out) {
  const char* fname = "qmckl_b200_mo_fp64";
  Context* ctx = ctx_of(context);
  const AoBasisRec& B = ctx->ao_basis;
  const int64_t A = B.ao_num, M = ctx->mo_basis.mo_num, S = B.shell_num, N = ctx->nucleus.num;
  if (P <= 0) return QMCKL_SUCCESS;
  qmckl_exit_code rc;
  const double cutoff = cutoff_of(ctx);
  // shell screening spheres in the basis order
  if (!ds->f64_sph.p || ds->f64_sph_basis != B.basis_version || ds->f64_sph_nucl != ctx->nucleus.coord_version ||
      ds->f64_sph_cutoff != cutoff) {
    std::vector<double4> sph((size_t)S);
    std::vector<int2> sao((size_t)S);
    for (int64_t m = 0; m < N; ++m)
      for (int64_t sh = B.nucleus_index[m]; sh < B.nucleus_index[m] + B.nucleus_shell_num[m]; ++sh) {
        const int l = B.shell_ang_mom[sh];
        const int64_t a0 = B.d.ao_index[sh];
        const int64_t na = std::max<int64_t>(0, std::min<int64_t>((int64_t)(l + 1) * (l + 2) / 2, A - a0));
        sph[(size_t)sh] = make_double4(ctx->nucleus.coord[m], ctx->nucleus.coord[m + N], ctx->nucleus.coord[m + 2 * N],
                                       shell_r2max(ctx, (int)sh, (int)m, cutoff));
        sao[(size_t)sh] = make_int2((int)a0, (int)na);
      }
    const size_t sb = (sizeof(double4) * (size_t)S + 255) / 256 * 256;
    rc = ensure(context, ds->f64_sph, sb + sizeof(int2) * (size_t)S, fname);
    if (rc != QMCKL_SUCCESS) return rc;
    QB_CUDA(cudaMemcpy(ds->f64_sph.p, sph.data(), sizeof(double4) * (size_t)S, cudaMemcpyHostToDevice), fname);
    QB_CUDA(cudaMemcpy((uint8_t*)ds->f64_sph.p + sb, sao.data(), sizeof(int2) * (size_t)S, cudaMemcpyHostToDevice),
            fname);
    ds->f64_sph_basis = B.basis_version;
    ds->f64_sph_nucl = ctx->nucleus.coord_version;
    ds->f64_sph_cutoff = cutoff;
  }
  const size_t sb = (sizeof(double4) * (size_t)S + 255) / 256 * 256;
  // coefficient_t with 16-byte aligned rows (a padded copy for an odd MO count)
  const double* Bt = (const double*)ds->coef_t.p;
  int64_t ldb = M;
  if (M & 1) {
    ldb = M + 1;
    if (ds->coef_f_version != ctx->mo_basis.coef_version || !ds->coef_f.p) {
      std::vector<double> cf((size_t)(A * ldb), 0.0);
      const std::vector<double>& c = ctx->mo_basis.coefficient;
      for (int64_t k = 0; k < A; ++k)
        for (int64_t i = 0; i < M; ++i) cf[(size_t)(k * ldb + i)] = c[(size_t)(i * A + k)];
      rc = ensure(context, ds->coef_f, sizeof(double) * cf.size(), fname);
      if (rc != QMCKL_SUCCESS) return rc;
      QB_CUDA(cudaMemcpy(ds->coef_f.p, cf.data(), sizeof(double) * cf.size(), cudaMemcpyHostToDevice), fname);
      ds->coef_f_version = ctx->mo_basis.coef_version;
    }
    Bt = (const double*)ds->coef_f.p;
  }
  // scratch: keys[P], perm[P], cell counts, then the tiles' AO lists (256-byte aligned)
  const size_t sort_bytes = (sizeof(int) * 2 * (size_t)P + sizeof(unsigned int) * (kSortCells + 1) + 255) / 256 * 256;
  rc = ensure(context, ds->order, sort_bytes + f64_plan_bytes(P, comps, A), fname);
  if (rc != QMCKL_SUCCESS) return rc;
  int* keys = (int*)ds->order.p;
  int* perm = keys + P;
  unsigned int* counts = (unsigned int*)(perm + P);
  void* plan = (uint8_t*)ds->order.p + sort_bytes;
  double lo[3], hi[3];
  nucleus_box(ctx, lo, hi);
  QB_CUDA(point_order(coord, P, lo, hi, keys, counts, perm, ds->stream, cstride), fname);
  QB_CUDA(launch_f64_plan(P, comps, coord, cstride, perm, (int)S, ds->f64_sph.p, (uint8_t*)ds->f64_sph.p + sb, A, plan,
                          ds->stream),
          fname);
  QB_CUDA(launch_gemm_f64_sparse(P, comps, M, ao, A, perm, plan, A, Bt, ldb, out, M, ds->stream), fname);
  return QMCKL_SUCCESS;
}

// Mixed-form MO VGL / value of P points into `out` (device).  With host_out
// (the host getters), the fused path evaluates the points in slices and
// copies each slice to the host on a second stream while the next slice is
// computed; *copied then reports that host_out holds the result.
qmckl_exit_code run_mo_mixed(qmckl_context context, DeviceState* ds, int64_t P, const double* coord,
                             double* out, int comps, double* host_out = nullptr, bool* copied = nullptr) {
  Context* ctx = ctx_of(context);
  if (copied) *copied = false;
  qmckl_exit_code rc0 = prepare_mixed(context, ds);
  if (rc0 != QMCKL_SUCCESS) return rc0;
  const double *cr = nullptr, *cprm = nullptr;   // cusp adjustment (none: null)
  rc0 = sync_cusp(context, ds, &cr, &cprm);
  if (rc0 != QMCKL_SUCCESS) return rc0;
  const int NN = (int)ctx->nucleus.num, MM = (int)ctx->mo_basis.mo_num;
  if (ds->fused) {
    bool ok = false;
    rc0 = prepare_fused(context, ds, &ok);
    if (rc0 != QMCKL_SUCCESS) return rc0;
    if (ok && tc_fused_smem(ds->tc, comps, ds->rec_bytes) <= 232448) {
      // spatial order of the points, then the fused AO -> MO kernel (the AO
      // pieces never leave shared memory)
      // scratch: keys[P], perm[P], cell counts, then the tile plan (256-byte aligned)
      const size_t sort_bytes = (sizeof(int) * 2 * (size_t)P + sizeof(unsigned int) * (kSortCells + 1) + 255) / 256 * 256;
      const size_t obytes = sort_bytes + tc_tile_plan_bytes(ds->tc, P, comps);
      qmckl_exit_code rc = ensure(context, ds->order, obytes, "qmckl_b200_mo_mixed");
      if (rc != QMCKL_SUCCESS) return rc;
      int* keys = (int*)ds->order.p;
      int* perm = keys + P;
      unsigned int* counts = (unsigned int*)(perm + P);
      void* tplan = (uint8_t*)ds->order.p + sort_bytes;
      double lo[3], hi[3];
      nucleus_box(ctx, lo, hi);
      const int64_t N = ctx->nucleus.num;
      fz::RowBound rb{(const double*)ds->nucl.p, (const float*)ds->env.p, (int)N, ds->env_r0, ds->env_inv_log2q};
      const int64_t M = ctx->mo_basis.mo_num;
      const bool slices = host_out != nullptr && P >= 8 * kSliceMinPoints;
      if (slices && ds->copy_stream == nullptr) {
        QB_CUDA(cudaStreamCreateWithFlags(&ds->copy_stream, cudaStreamNonBlocking), "qmckl_b200_mo_mixed");
        for (cudaEvent_t& ev : ds->slice_ev) QB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "qmckl_b200_mo_mixed");
      }
      const int64_t step = slices ? ((P + kSlices - 1) / kSlices + 24) / 25 * 25 : P;
      int slice = 0;
      for (int64_t a = 0; a < P; a += step, ++slice) {
        const int64_t n = std::min(step, P - a);
        double* o = out + a * comps * M;
        QB_CUDA(point_order(coord + a, n, lo, hi, keys, counts, perm, ds->stream, P), "qmckl_b200_mo_mixed");
        QB_CUDA(tc_run_fused(ds->T, ds->tc, n, comps, coord + a, cutoff_of(ctx), ds->tc_coef.p, ds->krec.p,
                             ds->rec_bytes, perm, rb, o, (int*)ds->tc_err.p, ds->stream, P, ds->kskip.p,
                             (unsigned long long*)ds->kstat.p, tplan),
                "qmckl_b200_mo_mixed");
        if (cr != nullptr)
          QB_CUDA(launch_cusp_mo(n, comps, coord + a, P, NN, (const double*)ds->nucl.p, cr, cprm, MM, o, ds->stream),
                  "qmckl_b200_mo_mixed");
        if (slices) {
          cudaEvent_t ev = ds->slice_ev[slice % kSlices];
          QB_CUDA(cudaEventRecord(ev, ds->stream), "qmckl_b200_mo_mixed");
          QB_CUDA(cudaStreamWaitEvent(ds->copy_stream, ev, 0), "qmckl_b200_mo_mixed");
          QB_CUDA(cudaMemcpyAsync(host_out + a * comps * M, o, sizeof(double) * n * comps * M, cudaMemcpyDeviceToHost,
                                  ds->copy_stream),
                  "qmckl_get_mo_basis_mo_vgl");
        }
      }
      if (slices) {
        QB_CUDA(cudaStreamSynchronize(ds->copy_stream), "qmckl_get_mo_basis_mo_vgl");
        if (copied) *copied = true;
      }
      return QMCKL_SUCCESS;
    }
  }
  const int64_t rows = (int64_t)comps * P;
  const size_t abytes = tc_a_bytes(ds->tc3, rows);
  qmckl_exit_code rc = ensure(context, ds->tc_a, abytes, "qmckl_b200_mo_mixed");
  if (rc != QMCKL_SUCCESS) return rc;
  QB_CUDA(tc_run(ds->T, ds->tc3, P, comps, coord, cutoff_of(ctx), ds->tc3_coef.p, ds->tc_a.p, out,
                 (int*)ds->tc_err.p, ds->stream,
                 ds->tiles.ntiles > 0 ? &ds->tiles : nullptr, cr),
          "qmckl_b200_mo_mixed");
  if (cr != nullptr)
    QB_CUDA(launch_cusp_mo(P, comps, coord, P, NN, (const double*)ds->nucl.p, cr, cprm, MM, out, ds->stream),
            "qmckl_b200_mo_mixed");
  return QMCKL_SUCCESS;
}

qmckl_exit_code run_mo(qmckl_context context, DeviceState* ds, int64_t P, const double* coord,
                       double* ao_scratch, double* out, int comps) {
  Context* ctx = ctx_of(context);
  const int64_t M = ctx->mo_basis.mo_num;
  if (use_mixed(ctx)) return run_mo_mixed(context, ds, P, coord, out, comps);
  qmckl_exit_code rc = sync_coef(context, ds);
  if (rc != QMCKL_SUCCESS) return rc;
  const double *cr = nullptr, *cprm = nullptr;
  rc = sync_cusp(context, ds, &cr, &cprm);
  if (rc != QMCKL_SUCCESS) return rc;
  rc = comps == 5 ? run_ao_vgl(context, ds, P, coord, ao_scratch, cr)
                  : run_ao_value(context, ds, P, coord, ao_scratch, cr);
  if (rc != QMCKL_SUCCESS) return rc;
  rc = contract_f64(context, ds, P, comps, coord, P, ao_scratch, out);
  if (rc != QMCKL_SUCCESS) return rc;
  if (cr != nullptr)
    QB_CUDA(launch_cusp_mo(P, comps, coord, P, (int)ctx->nucleus.num, (const double*)ds->nucl.p, cr, cprm, (int)M, out,
                           ds->stream),
            "qmckl_b200_mo");
  return QMCKL_SUCCESS;
}

}  // namespace

qmckl_exit_code dev_attach(qmckl_context context) {
  Context* ctx = ctx_of(context);
  if (ctx->extra) {
    if (ctx->extra->device >= 0) QB_CUDA(cudaSetDevice(ctx->extra->device), "qmckl_b200_attach");
    return QMCKL_SUCCESS;
  }
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return qmckl_failwith(context, QMCKL_FAILURE, "qmckl_b200_attach",
                          "no CUDA device: qmckl_b200 computes on the GPU only");
  }
  DeviceState* ds = new DeviceState();
  QB_CUDA(cudaGetDevice(&ds->device), "qmckl_b200_attach");
  ctx->extra = ds;
  return QMCKL_SUCCESS;
}

static qmckl_exit_code ensure_stream(qmckl_context context, DeviceState* ds) {
  if (ds->stream != nullptr || ds->stream_given) return QMCKL_SUCCESS;
  QB_CUDA(cudaStreamCreateWithFlags(&ds->stream, cudaStreamNonBlocking), "qmckl_b200_attach");
  ds->own_stream = true;
  return QMCKL_SUCCESS;
}

static qmckl_exit_code attach_all(qmckl_context context) {
  qmckl_exit_code rc = dev_attach(context);
  if (rc != QMCKL_SUCCESS) return rc;
  return ensure_stream(context, state(context));
}

void dev_detach(Context* ctx) {
  DeviceState* ds = ctx->extra;
  if (!ds) return;
  if (ds->device >= 0) cudaSetDevice(ds->device);
  if (ds->stream) cudaStreamSynchronize(ds->stream);
  for (DevBuf* b : {&ds->tables, &ds->nucl, &ds->coord, &ds->prim_vgl, &ds->shell_vgl, &ds->ao_vgl, &ds->ao_value,
                    &ds->mo_vgl, &ds->mo_value, &ds->coef_t, &ds->tc_coef, &ds->tc_a, &ds->krec, &ds->order,
                    &ds->ao_hessian, &ds->coef_rows, &ds->adj_coord, &ds->adj_buf, &ds->adj_part, &ds->adj_nucl,
                    &ds->tc3_coef, &ds->env, &ds->nuc_ao, &ds->forces, &ds->adj_wp, &ds->adj_ct,
                    &ds->cusp, &ds->ao_masked, &ds->en_dist, &ds->mo_hessian, &ds->kskip, &ds->kstat,
                    &ds->tc_err, &ds->f64_sph, &ds->coef_f})
    release(*b);
  if (ds->copy_stream) {
    cudaStreamSynchronize(ds->copy_stream);
    cudaStreamDestroy(ds->copy_stream);
    for (cudaEvent_t ev : ds->slice_ev)
      if (ev) cudaEventDestroy(ev);
  }
  if (ds->own_stream && ds->stream) cudaStreamDestroy(ds->stream);
  delete ds;
  ctx->extra = nullptr;
}

// The device data a fixed-scratch evaluation needs, without allocating: the
// basis tables and split coefficients must already be on the device (any
// regular mixed evaluation of the context puts them there); nuclear
// coordinates moved since then are copied into their existing buffer.
qmckl_exit_code dev_prepared_mixed(qmckl_context context, PreparedMixed* out) {
  Context* ctx = ctx_of(context);
  DeviceState* ds = ctx->extra;
  const char* fname = "qmckl_b200_mo_vgl_device_noalloc";
  if (ds == nullptr || ds->tables.p == nullptr || ds->basis_version != ctx->ao_basis.basis_version ||
      ds->tc3_coef.p == nullptr || ds->tc3_coef_version != ctx->mo_basis.coef_version || ds->tc_err.p == nullptr ||
      (ds->stream == nullptr && !ds->stream_given))
    return qmckl_failwith(context, QMCKL_NOT_PROVIDED, fname,
                          "basis or MO coefficients not on the device yet: run one regular mixed-form "
                          "evaluation of this context first");
  if (ds->device >= 0) QB_CUDA(cudaSetDevice(ds->device), fname);
  if (ds->nucl_version != ctx->nucleus.coord_version) {
    const size_t bytes = sizeof(double) * 3 * ctx->nucleus.num;
    if (ds->nucl.p == nullptr || ds->nucl.cap < bytes)
      return qmckl_failwith(context, QMCKL_NOT_PROVIDED, fname, "nuclear coordinates not on the device yet");
    QB_CUDA(cudaMemcpyAsync(ds->nucl.p, ctx->nucleus.coord.data(), bytes, cudaMemcpyHostToDevice, ds->stream), fname);
    ds->nucl_version = ctx->nucleus.coord_version;
  }
  out->T = ds->T;
  out->T.nucl_coord = (const double*)ds->nucl.p;
  out->plan = ds->tc3;
  out->coef = ds->tc3_coef.p;
  out->stream = ds->stream;
  out->cutoff = cutoff_of(ctx);
  out->err = (int*)ds->tc_err.p;
  if (!ctx->mo_basis.r_cusp.empty()) {
    if (ds->cusp.p == nullptr || ds->cusp_version != ctx->mo_basis.cusp_version)
      return qmckl_failwith(context, QMCKL_NOT_PROVIDED, fname,
                            "cusp parameters not on the device yet: run one regular mixed-form evaluation of this "
                            "context first");
    out->cusp_r = (const double*)ds->cusp.p;
    out->cusp_prm = out->cusp_r + ctx->nucleus.num;
  }
  return QMCKL_SUCCESS;
}

qmckl_exit_code dev_invalidate_mo(qmckl_context context) {
  DeviceState* ds = state(context);
  if (ds) {
    ds->coef_version = ~0ull;
    ds->tc_coef_version = ~0ull;
    ds->tc3_coef_version = ~0ull;
    ds->coef_f_version = ~0ull;
  }
  return QMCKL_SUCCESS;
}

qmckl_exit_code dev_provide_primitive_vgl(qmckl_context context, double* host_out) {
  qmckl_exit_code rc = attach_all(context);
  if (rc != QMCKL_SUCCESS) return rc;
  Context* ctx = ctx_of(context);
  DeviceState* ds = state(context);
  rc = sync_inputs(context, ds, true);
  if (rc != QMCKL_SUCCESS) return rc;
  const int64_t P = ctx->point.num, n = ctx->ao_basis.prim_num;
  const size_t bytes = sizeof(double) * 5 * n * P;
  // The reference recomputes this array on every call (its provider stamps
  // shell_vgl_date instead, org/qmckl_ao.org:4606-4616); recomputed here too.
  rc = ensure(context, ds->prim_vgl, bytes, "qmckl_provide_ao_basis_primitive_vgl");
  if (rc != QMCKL_SUCCESS) return rc;
  QB_CUDA(launch_primitive_vgl(ds->T, P, (const double*)ds->coord.p, cutoff_of(ctx), (double*)ds->prim_vgl.p, ds->stream),
          "qmckl_provide_ao_basis_primitive_vgl");
  ctx->ao_basis.primitive_vgl_date = ctx->date;
  return copy_out(context, ds, host_out, ds->prim_vgl.p, bytes, "qmckl_get_ao_basis_primitive_vgl");
}

qmckl_exit_code dev_provide_shell_vgl(qmckl_context context, double* host_out) {
  qmckl_exit_code rc = attach_all(context);
  if (rc != QMCKL_SUCCESS) return rc;
  Context* ctx = ctx_of(context);
  DeviceState* ds = state(context);
  const int64_t P = ctx->point.num, n = ctx->ao_basis.shell_num;
  const size_t bytes = sizeof(double) * 5 * n * P;
  if (ctx->point.date > ctx->ao_basis.shell_vgl_date || ds->shell_vgl.cap < bytes) {
    rc = sync_inputs(context, ds, true);
    if (rc != QMCKL_SUCCESS) return rc;
    rc = ensure(context, ds->shell_vgl, bytes, "qmckl_provide_ao_basis_shell_vgl");
    if (rc != QMCKL_SUCCESS) return rc;
    QB_CUDA(launch_shell_vgl(ds->T, P, (const double*)ds->coord.p, cutoff_of(ctx), (double*)ds->shell_vgl.p, ds->stream),
            "qmckl_provide_ao_basis_shell_vgl");
    ctx->ao_basis.shell_vgl_date = ctx->date;
  }
  return copy_out(context, ds, host_out, ds->shell_vgl.p, bytes, "qmckl_get_ao_basis_shell_vgl");
}

qmckl_exit_code dev_provide_ao_vgl(qmckl_context context, double* host_out) {
  qmckl_exit_code rc = attach_all(context);
  if (rc != QMCKL_SUCCESS) return rc;
  Context* ctx = ctx_of(context);
  DeviceState* ds = state(context);
  if (ctx->ao_basis.type != 'G')
    return qmckl_failwith(context, QMCKL_FAILURE, "qmckl_provide_ao_basis_ao_vgl", "only Gaussian basis sets are implemented");
  const int64_t P = ctx->point.num, A = ctx->ao_basis.ao_num;
  const size_t bytes = sizeof(double) * 5 * A * P;
  if (ctx->point.date > ctx->ao_basis.ao_vgl_date || ds->ao_vgl.cap < bytes) {
    rc = sync_inputs(context, ds, true);
    if (rc != QMCKL_SUCCESS) return rc;
    rc = ensure(context, ds->ao_vgl, bytes, "qmckl_provide_ao_basis_ao_vgl");
    if (rc != QMCKL_SUCCESS) return rc;
    rc = run_ao_vgl(context, ds, P, (const double*)ds->coord.p, (double*)ds->ao_vgl.p);
    if (rc != QMCKL_SUCCESS) return rc;
    ctx->ao_basis.ao_vgl_date = ctx->date;
  }
  return copy_out(context, ds, host_out, ds->ao_vgl.p, bytes, "qmckl_get_ao_basis_ao_vgl");
}

qmckl_exit_code dev_provide_ao_value(qmckl_context context, double* host_out) {
  qmckl_exit_code rc = attach_all(context);
  if (rc != QMCKL_SUCCESS) return rc;
  Context* ctx = ctx_of(context);
  DeviceState* ds = state(context);
  if (ctx->ao_basis.type != 'G')
    return qmckl_failwith(context, QMCKL_FAILURE, "qmckl_provide_ao_basis_ao_value", "only Gaussian basis sets are implemented");
  const int64_t P = ctx->point.num, A = ctx->ao_basis.ao_num;
  const size_t bytes = sizeof(double) * A * P;
  if (ctx->point.date > ctx->ao_basis.ao_value_date || ds->ao_value.cap < bytes) {
    rc = sync_inputs(context, ds, true);
    if (rc != QMCKL_SUCCESS) return rc;
    rc = ensure(context, ds->ao_value, bytes, "qmckl_provide_ao_basis_ao_value");
    if (rc != QMCKL_SUCCESS) return rc;
    rc = run_ao_value(context, ds, P, (const double*)ds->coord.p, (double*)ds->ao_value.p);
    if (rc != QMCKL_SUCCESS) return rc;
    ctx->ao_basis.ao_value_date = ctx->date;
  }
  return copy_out(context, ds, host_out, ds->ao_value.p, bytes, "qmckl_get_ao_basis_ao_value");
}

// qmckl_provide_ao_basis_ao_hessian (org/qmckl_ao.org:9470-9540): recomputed
// when the points are newer than the array.
qmckl_exit_code dev_provide_ao_hessian(qmckl_context context, double* host_out) {
  qmckl_exit_code rc = attach_all(context);
  if (rc != QMCKL_SUCCESS) return rc;
  Context* ctx = ctx_of(context);
  DeviceState* ds = state(context);
  if (ctx->ao_basis.type != 'G')
    return qmckl_failwith(context, QMCKL_FAILURE, "qmckl_provide_ao_basis_ao_hessian", "only Gaussian basis sets are implemented");
  const int64_t P = ctx->point.num, A = ctx->ao_basis.ao_num;
  const size_t bytes = sizeof(double) * 12 * A * P;
  if (ctx->point.date > ctx->ao_basis.ao_hessian_date || ds->ao_hessian.cap < bytes) {
    rc = sync_inputs(context, ds, true);
    if (rc != QMCKL_SUCCESS) return rc;
    rc = ensure(context, ds->ao_hessian, bytes, "qmckl_provide_ao_basis_ao_hessian");
    if (rc != QMCKL_SUCCESS) return rc;
    QB_CUDA(launch_ao_hessian(ds->T, P, (const double*)ds->coord.p, cutoff_of(ctx), ctx->precision <= 23,
                              (double*)ds->ao_hessian.p, ds->stream),
            "qmckl_provide_ao_basis_ao_hessian");
    ctx->ao_basis.ao_hessian_date = ctx->date;
  }
  return copy_out(context, ds, host_out, ds->ao_hessian.p, bytes, "qmckl_get_ao_basis_ao_hessian");
}

// Orbital forces (org/qmckl_forces.org:5129-6880): which = 0 forces_mo_value,
// 1 forces_mo_g, 2 forces_mo_l, 3 forces_ao_value, recomputed on every call
// from the current ao_vgl / ao_hessian of the context's points.
qmckl_exit_code dev_provide_forces(qmckl_context context, int which, double* host_out) {
  static const char* const names[4] = {"qmckl_get_forces_mo_value", "qmckl_get_forces_mo_g",
                                       "qmckl_get_forces_mo_l", "qmckl_get_forces_ao_value"};
  const char* fname = names[which];
  qmckl_exit_code rc = attach_all(context);
  if (rc != QMCKL_SUCCESS) return rc;
  Context* ctx = ctx_of(context);
  DeviceState* ds = state(context);
  const int64_t P = ctx->point.num, A = ctx->ao_basis.ao_num, N = ctx->nucleus.num;
  const int64_t M = which == 3 ? 0 : ctx->mo_basis.mo_num;
  rc = (which == 1 || which == 2) ? dev_provide_ao_hessian(context, nullptr) : dev_provide_ao_vgl(context, nullptr);
  if (rc != QMCKL_SUCCESS) return rc;
  if (which != 3) {
    rc = sync_coef(context, ds);
    if (rc != QMCKL_SUCCESS) return rc;
  }
  if (ds->nuc_ao_version != ctx->ao_basis.basis_version || !ds->nuc_ao.p) {
    const AoBasisRec& B = ctx->ao_basis;
    std::vector<int2> r((size_t)std::max<int64_t>(N, 1), make_int2(0, 0));
    for (int64_t n = 0; n < N; ++n) {
      const int64_t s0 = B.nucleus_index[n], s1 = s0 + B.nucleus_shell_num[n];
      if (s1 > s0) {
        const int l = B.shell_ang_mom[s1 - 1];
        r[n] = make_int2((int)B.d.ao_index[s0], (int)(B.d.ao_index[s1 - 1] + (l + 1) * (l + 2) / 2));
      }
    }
    rc = ensure(context, ds->nuc_ao, sizeof(int2) * r.size(), fname);
    if (rc != QMCKL_SUCCESS) return rc;
    QB_CUDA(cudaMemcpyAsync(ds->nuc_ao.p, r.data(), sizeof(int2) * r.size(), cudaMemcpyHostToDevice, ds->stream), fname);
    QB_CUDA(cudaStreamSynchronize(ds->stream), fname);
    ds->nuc_ao_version = ctx->ao_basis.basis_version;
  }
  const int64_t count = which == 3 ? N * P * 3 * A : N * (which == 1 ? 9 : 3) * P * M;
  const size_t bytes = sizeof(double) * (size_t)count;
  rc = ensure(context, ds->forces, bytes, fname);
  if (rc != QMCKL_SUCCESS) return rc;
  const double* X = (which == 1 || which == 2) ? (const double*)ds->ao_hessian.p : (const double*)ds->ao_vgl.p;
  QB_CUDA(launch_forces(which, P, A, M, (int)N, (const int2*)ds->nuc_ao.p, X, (const double*)ds->coef_t.p,
                        (double*)ds->forces.p, ds->stream),
          fname);
  return copy_out(context, ds, host_out, ds->forces.p, bytes, fname);
}

qmckl_exit_code dev_provide_mo_vgl(qmckl_context context, double* host_out) {
  qmckl_exit_code rc = attach_all(context);
  if (rc != QMCKL_SUCCESS) return rc;
  Context* ctx = ctx_of(context);
  DeviceState* ds = state(context);
  if (ctx->ao_basis.type != 'G')
    return qmckl_failwith(context, QMCKL_FAILURE, "qmckl_provide_mo_basis_mo_vgl", "only Gaussian basis sets are implemented");
  if (!ctx->ao_basis.provided)
    return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_ao_basis", NULL);
  const int64_t P = ctx->point.num, A = ctx->ao_basis.ao_num, M = ctx->mo_basis.mo_num;
  const size_t bytes = sizeof(double) * 5 * M * P;
  bool copied = false;   // set when the evaluation already copied the slices to host_out
  if (ctx->point.date > ctx->mo_basis.mo_vgl_date || ds->mo_vgl.cap < bytes) {
    rc = sync_inputs(context, ds, true);
    if (rc != QMCKL_SUCCESS) return rc;
    rc = ensure(context, ds->mo_vgl, bytes, "qmckl_provide_mo_basis_mo_vgl");
    if (rc != QMCKL_SUCCESS) return rc;
    if (use_mixed(ctx)) {
      rc = run_mo_mixed(context, ds, P, (const double*)ds->coord.p, (double*)ds->mo_vgl.p, 5, host_out, &copied);
    } else if (!ctx->mo_basis.r_cusp.empty()) {
      // FP64 form with the cusp adjustment: the AOs that it leaves out are
      // zeroed in a separate AO array (the cached ao_vgl stays the plain one)
      rc = ensure(context, ds->ao_masked, sizeof(double) * 5 * A * P, "qmckl_provide_mo_basis_mo_vgl");
      if (rc != QMCKL_SUCCESS) return rc;
      rc = run_mo(context, ds, P, (const double*)ds->coord.p, (double*)ds->ao_masked.p, (double*)ds->mo_vgl.p, 5);
    } else {
      // FP64 form: the AO array is materialised (and cached) as in the reference
      rc = sync_coef(context, ds);
      if (rc != QMCKL_SUCCESS) return rc;
      const size_t abytes = sizeof(double) * 5 * A * P;
      if (ctx->point.date > ctx->ao_basis.ao_vgl_date || ds->ao_vgl.cap < abytes) {
        rc = ensure(context, ds->ao_vgl, abytes, "qmckl_provide_ao_basis_ao_vgl");
        if (rc != QMCKL_SUCCESS) return rc;
        rc = run_ao_vgl(context, ds, P, (const double*)ds->coord.p, (double*)ds->ao_vgl.p);
        if (rc != QMCKL_SUCCESS) return rc;
        ctx->ao_basis.ao_vgl_date = ctx->date;
      }
      rc = contract_f64(context, ds, P, 5, (const double*)ds->coord.p, P, (const double*)ds->ao_vgl.p,
                        (double*)ds->mo_vgl.p);
    }
    if (rc != QMCKL_SUCCESS) return rc;
    ctx->mo_basis.mo_vgl_date = ctx->date;
  }
  return copy_out(context, ds, copied ? nullptr : host_out, ds->mo_vgl.p, bytes, "qmckl_get_mo_basis_mo_vgl");
}

qmckl_exit_code dev_provide_mo_value(qmckl_context context, double* host_out) {
  qmckl_exit_code rc = attach_all(context);
  if (rc != QMCKL_SUCCESS) return rc;
  Context* ctx = ctx_of(context);
  DeviceState* ds = state(context);
  if (ctx->ao_basis.type != 'G')
    return qmckl_failwith(context, QMCKL_FAILURE, "qmckl_provide_mo_basis_mo_value", "only Gaussian basis sets are implemented");
  const int64_t P = ctx->point.num, A = ctx->ao_basis.ao_num, M = ctx->mo_basis.mo_num;
  const size_t bytes = sizeof(double) * M * P;
  if (ctx->point.date > ctx->mo_basis.mo_value_date || ds->mo_value.cap < bytes) {
    rc = ensure(context, ds->mo_value, bytes, "qmckl_provide_mo_basis_mo_value");
    if (rc != QMCKL_SUCCESS) return rc;
    if (ctx->mo_basis.mo_vgl_date == ctx->point.date && ds->mo_vgl.p != nullptr &&
        ds->mo_vgl.cap >= sizeof(double) * 5 * M * P) {
      // mo_vgl is current: take its value rows (org/qmckl_mo.org:1186-1198)
      QB_CUDA(cudaMemcpy2DAsync(ds->mo_value.p, sizeof(double) * M, ds->mo_vgl.p, sizeof(double) * 5 * M,
                                sizeof(double) * M, P, cudaMemcpyDeviceToDevice, ds->stream),
              "qmckl_provide_mo_basis_mo_value");
    } else {
      rc = sync_inputs(context, ds, true);
      if (rc != QMCKL_SUCCESS) return rc;
      if (use_mixed(ctx)) {
        rc = run_mo_mixed(context, ds, P, (const double*)ds->coord.p, (double*)ds->mo_value.p, 1);
      } else if (!ctx->mo_basis.r_cusp.empty()) {
        rc = ensure(context, ds->ao_masked, sizeof(double) * A * P, "qmckl_provide_mo_basis_mo_value");
        if (rc != QMCKL_SUCCESS) return rc;
        rc = run_mo(context, ds, P, (const double*)ds->coord.p, (double*)ds->ao_masked.p, (double*)ds->mo_value.p, 1);
      } else {
        rc = sync_coef(context, ds);
        if (rc != QMCKL_SUCCESS) return rc;
        const size_t abytes = sizeof(double) * A * P;
        if (ctx->point.date > ctx->ao_basis.ao_value_date || ds->ao_value.cap < abytes) {
          rc = ensure(context, ds->ao_value, abytes, "qmckl_provide_ao_basis_ao_value");
          if (rc != QMCKL_SUCCESS) return rc;
          rc = run_ao_value(context, ds, P, (const double*)ds->coord.p, (double*)ds->ao_value.p);
          if (rc != QMCKL_SUCCESS) return rc;
          ctx->ao_basis.ao_value_date = ctx->date;
        }
        rc = contract_f64(context, ds, P, 1, (const double*)ds->coord.p, P, (const double*)ds->ao_value.p,
                          (double*)ds->mo_value.p);
      }
      if (rc != QMCKL_SUCCESS) return rc;
    }
    ctx->mo_basis.mo_value_date = ctx->date;
  }
  return copy_out(context, ds, host_out, ds->mo_value.p, bytes, "qmckl_get_mo_basis_mo_value");
}

// MO Hessian (org/qmckl_mo.org:2428-2600, FP64 in both forms, as the AO
// Hessian): mo_hessian[jj][p][kk][i] = sum_k ao_hessian[jj][p][kk][k] *
// coefficient_t[k][i], kk < 3, as three GEMMs (one per kk: rows (jj, p) of
// stride 4 ao_num); with the cusp adjustment from an AO Hessian whose
// left-out AOs are zeroed, plus the cubics' Hessians.
qmckl_exit_code dev_provide_mo_hessian(qmckl_context context, double* host_out) {
  const char* fname = "qmckl_provide_mo_basis_mo_hessian";
  qmckl_exit_code rc = attach_all(context);
  if (rc != QMCKL_SUCCESS) return rc;
  Context* ctx = ctx_of(context);
  DeviceState* ds = state(context);
  if (ctx->ao_basis.type != 'G') return qmckl_failwith(context, QMCKL_FAILURE, fname, "only Gaussian basis sets are implemented");
  if (!ctx->ao_basis.provided) return qmckl_failwith(context, QMCKL_NOT_PROVIDED, "qmckl_ao_basis", NULL);
  const int64_t P = ctx->point.num, A = ctx->ao_basis.ao_num, M = ctx->mo_basis.mo_num;
  const size_t bytes = sizeof(double) * 9 * M * P;
  if (ctx->point.date > ctx->mo_basis.mo_hessian_date || ds->mo_hessian.cap < bytes) {
    rc = sync_inputs(context, ds, true);
    if (rc == QMCKL_SUCCESS) rc = sync_coef(context, ds);
    const double *cr = nullptr, *cprm = nullptr;
    if (rc == QMCKL_SUCCESS) rc = sync_cusp(context, ds, &cr, &cprm);
    if (rc == QMCKL_SUCCESS) rc = ensure(context, ds->mo_hessian, bytes, fname);
    if (rc != QMCKL_SUCCESS) return rc;
    const double* H = nullptr;
    if (cr != nullptr) {
      rc = ensure(context, ds->ao_masked, sizeof(double) * 12 * A * P, fname);
      if (rc != QMCKL_SUCCESS) return rc;
      QB_CUDA(launch_ao_hessian(ds->T, P, (const double*)ds->coord.p, cutoff_of(ctx), ctx->precision <= 23,
                                (double*)ds->ao_masked.p, ds->stream, cr),
              fname);
      H = (const double*)ds->ao_masked.p;
    } else {
      rc = dev_provide_ao_hessian(context, nullptr);
      if (rc != QMCKL_SUCCESS) return rc;
      H = (const double*)ds->ao_hessian.p;
    }
    double* out = (double*)ds->mo_hessian.p;
    for (int kk = 0; kk < 3; ++kk)
      QB_CUDA(launch_gemm_f64(3 * P, M, A, H + kk * A, 4 * A, (const double*)ds->coef_t.p, M, out + kk * M, 3 * M,
                              ds->stream),
              fname);
    if (cr != nullptr)
      QB_CUDA(launch_cusp_hessian(P, (const double*)ds->coord.p, (int)ctx->nucleus.num, (const double*)ds->nucl.p, cr,
                                  cprm, (int)M, out, ds->stream),
              fname);
    ctx->mo_basis.mo_hessian_date = ctx->date;
  }
  return copy_out(context, ds, host_out, ds->mo_hessian.p, bytes, "qmckl_get_mo_basis_mo_hessian");
}

// en_distance[point][nucl] (org/qmckl_electron.org:1270-1393), recomputed on
// every call.
qmckl_exit_code dev_en_distance(qmckl_context context, double* host_out) {
  qmckl_exit_code rc = attach_all(context);
  if (rc != QMCKL_SUCCESS) return rc;
  Context* ctx = ctx_of(context);
  DeviceState* ds = state(context);
  const int64_t P = ctx->point.num, N = ctx->nucleus.num;
  rc = sync_inputs(context, ds, true, false);
  if (rc != QMCKL_SUCCESS) return rc;
  const size_t bytes = sizeof(double) * P * N;
  rc = ensure(context, ds->en_dist, std::max<size_t>(bytes, 8), "qmckl_provide_en_distance");
  if (rc != QMCKL_SUCCESS) return rc;
  QB_CUDA(launch_en_distance(P, (const double*)ds->coord.p, (int)N, (const double*)ds->nucl.p, (double*)ds->en_dist.p,
                             ds->stream),
          "qmckl_provide_en_distance");
  return copy_out(context, ds, host_out, ds->en_dist.p, bytes, "qmckl_get_electron_en_distance");
}

}  // namespace qb

using namespace qb;

extern "C" {

int64_t qmckl_b200_kernel_launch_count(void) { return g_launches.load(); }

qmckl_exit_code qmckl_b200_get_kblock_stats(qmckl_context context, int64_t* evaluated, int64_t* total,
                                           const int32_t reset) {
  const char* fname = "qmckl_b200_get_kblock_stats";
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  if (evaluated == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, fname, "NULL pointer");
  if (total == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_3, fname, "NULL pointer");
  *evaluated = *total = 0;
  DeviceState* ds = state(context);
  if (ds == nullptr || ds->kstat.p == nullptr) return QMCKL_SUCCESS;
  if (ds->device >= 0) QB_CUDA(cudaSetDevice(ds->device), fname);
  unsigned long long h[2] = {0, 0};
  QB_CUDA(cudaMemcpyAsync(h, ds->kstat.p, sizeof h, cudaMemcpyDeviceToHost, ds->stream), fname);
  if (reset) QB_CUDA(cudaMemsetAsync(ds->kstat.p, 0, sizeof h, ds->stream), fname);
  QB_CUDA(cudaStreamSynchronize(ds->stream), fname);
  *evaluated = (int64_t)h[0];
  *total = (int64_t)h[1];
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_b200_set_split_terms(qmckl_context context, const int32_t pieces) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  if (pieces != 2 && pieces != 3)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_b200_set_split_terms", "pieces must be 2 or 3");
  qmckl_exit_code rc = dev_attach(context);
  if (rc != QMCKL_SUCCESS) return rc;
  if (state(context)->split_pieces != pieces) {
    state(context)->split_pieces = pieces;
    qmckl_context_touch(context);
  }
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_b200_set_mixed_kernel(qmckl_context context, const int32_t fused) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  qmckl_exit_code rc = dev_attach(context);
  if (rc != QMCKL_SUCCESS) return rc;
  state(context)->fused = fused != 0;
  return qmckl_context_touch(context);
}

qmckl_exit_code qmckl_b200_set_device(qmckl_context context, const int32_t device) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  Context* ctx = ctx_of(context);
  if (ctx->extra && (ctx->extra->tables.p || ctx->extra->stream || ctx->extra->stream_given))
    return qmckl_failwith(context, QMCKL_ALREADY_SET, "qmckl_b200_set_device", "set the device before the first evaluation");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_b200_set_device", "no such device");
  }
  qmckl_exit_code rc = dev_attach(context);
  if (rc != QMCKL_SUCCESS) return rc;
  ctx->extra->device = device;
  QB_CUDA(cudaSetDevice(device), "qmckl_b200_set_device");
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_b200_set_stream(qmckl_context context, void* stream) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  qmckl_exit_code rc = dev_attach(context);
  if (rc != QMCKL_SUCCESS) return rc;
  DeviceState* ds = state(context);
  if (ds->own_stream && ds->stream) {
    cudaStreamSynchronize(ds->stream);
    cudaStreamDestroy(ds->stream);
  }
  ds->stream = (cudaStream_t)stream;
  ds->own_stream = false;
  ds->stream_given = true;
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_b200_synchronize(qmckl_context context) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  DeviceState* ds = state(context);
  if (!ds || (!ds->stream && !ds->stream_given)) return QMCKL_SUCCESS;
  if (ds->device >= 0) QB_CUDA(cudaSetDevice(ds->device), "qmckl_b200_synchronize");
  return sync_and_check(context, ds, "qmckl_b200_synchronize");
}

qmckl_exit_code qmckl_b200_inject_wait_failure(qmckl_context context, const int32_t code) {
  const char* fname = "qmckl_b200_inject_wait_failure";
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  DeviceState* ds = state(context);
  if (ds == nullptr || ds->tc_err.p == nullptr)
    return qmckl_failwith(context, QMCKL_NOT_PROVIDED, fname, "no mixed-form evaluation on this context yet");
  if (ds->device >= 0) QB_CUDA(cudaSetDevice(ds->device), fname);
  QB_CUDA(cudaMemcpyAsync(ds->tc_err.p, &code, sizeof(int), cudaMemcpyHostToDevice, ds->stream), fname);
  QB_CUDA(cudaStreamSynchronize(ds->stream), fname);
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_b200_get_fused_plan(const int64_t ao_num, const int64_t mo_num, const int32_t pieces,
                                          int32_t* n_tile, int32_t* n_tiles, int32_t* accumulators,
                                          int32_t* stages) {
  if (ao_num <= 0) return QMCKL_INVALID_ARG_1;
  if (mo_num <= 0) return QMCKL_INVALID_ARG_2;
  if (pieces != 2 && pieces != 3) return QMCKL_INVALID_ARG_3;
  if (!n_tile || !n_tiles || !accumulators || !stages) return QMCKL_INVALID_ARG_4;
  const TcPlan p = tc_plan_fused(ao_num, mo_num, pieces);
  *n_tile = p.n_tile;
  *n_tiles = p.n_tiles;
  *accumulators = p.nacc;
  *stages = p.nst;
  return QMCKL_SUCCESS;
}

qmckl_exit_code qmckl_b200_inject_late_warps(const int64_t ns) {
  if (ns < 0 || ns > 10000000) return QMCKL_INVALID_ARG_1;
  return tc_set_late_warps((unsigned int)ns) == cudaSuccess ? QMCKL_SUCCESS : QMCKL_FAILURE;
}

static qmckl_exit_code device_entry(qmckl_context context, const char* fname, int64_t point_num,
                                    const double* d_coord, void* d_out, bool need_mo) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  Context* ctx = ctx_of(context);
  if (!ctx->ao_basis.provided) return qmckl_failwith(context, QMCKL_NOT_PROVIDED, fname, "AO basis not provided");
  if (need_mo && !ctx->mo_basis.provided) return qmckl_failwith(context, QMCKL_NOT_PROVIDED, fname, "MO basis not provided");
  if (ctx->ao_basis.type != 'G') return qmckl_failwith(context, QMCKL_FAILURE, fname, "only Gaussian basis sets are implemented");
  if (point_num < 0) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, fname, "point_num < 0");
  if (point_num > 0 && d_coord == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_3, fname, "NULL pointer");
  if (point_num > 0 && d_out == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_4, fname, "NULL pointer");
  qmckl_exit_code rc = attach_all(context);
  if (rc != QMCKL_SUCCESS) return rc;
  return sync_inputs(context, state(context), false);
}

qmckl_exit_code qmckl_b200_ao_vgl_device(qmckl_context context, const int64_t point_num, const double* d_coord,
                                         double* d_ao_vgl) {
  qmckl_exit_code rc = device_entry(context, "qmckl_b200_ao_vgl_device", point_num, d_coord, d_ao_vgl, false);
  if (rc != QMCKL_SUCCESS) return rc;
  return run_ao_vgl(context, state(context), point_num, d_coord, d_ao_vgl);
}

qmckl_exit_code qmckl_b200_ao_value_device(qmckl_context context, const int64_t point_num, const double* d_coord,
                                           double* d_ao_value) {
  qmckl_exit_code rc = device_entry(context, "qmckl_b200_ao_value_device", point_num, d_coord, d_ao_value, false);
  if (rc != QMCKL_SUCCESS) return rc;
  return run_ao_value(context, state(context), point_num, d_coord, d_ao_value);
}

static qmckl_exit_code mo_device(qmckl_context context, const char* fname, int64_t point_num, const double* d_coord,
                                 double* d_out, int comps) {
  qmckl_exit_code rc = device_entry(context, fname, point_num, d_coord, d_out, true);
  if (rc != QMCKL_SUCCESS) return rc;
  Context* ctx = ctx_of(context);
  DeviceState* ds = state(context);
  if (use_mixed(ctx)) return run_mo_mixed(context, ds, point_num, d_coord, d_out, comps);
  const size_t abytes = sizeof(double) * comps * ctx->ao_basis.ao_num * point_num;
  DevBuf& scratch = comps == 5 ? ds->ao_vgl : ds->ao_value;
  rc = ensure(context, scratch, abytes, fname);
  if (rc != QMCKL_SUCCESS) return rc;
  // the AO scratch no longer holds the context's cached points
  if (comps == 5) ctx->ao_basis.ao_vgl_date = 0; else ctx->ao_basis.ao_value_date = 0;
  return run_mo(context, ds, point_num, d_coord, (double*)scratch.p, d_out, comps);
}

qmckl_exit_code qmckl_b200_mo_vgl_device(qmckl_context context, const int64_t point_num, const double* d_coord,
                                         double* d_mo_vgl) {
  return mo_device(context, "qmckl_b200_mo_vgl_device", point_num, d_coord, d_mo_vgl, 5);
}

qmckl_exit_code qmckl_b200_mo_value_device(qmckl_context context, const int64_t point_num, const double* d_coord,
                                           double* d_mo_value) {
  return mo_device(context, "qmckl_b200_mo_value_device", point_num, d_coord, d_mo_value, 1);
}

// ---- orbital forces (org/qmckl_forces.org:5129-5160, 5475-5575, 5919-6000, 6499-6530)

static qmckl_exit_code forces_getter(qmckl_context context, int which, double* out, int64_t size_max, bool need_mo,
                                     int64_t per_point_nucl) {
  static const char* const names[4] = {"qmckl_get_forces_mo_value", "qmckl_get_forces_mo_g",
                                       "qmckl_get_forces_mo_l", "qmckl_get_forces_ao_value"};
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_NULL_CONTEXT;
  Context* ctx = ctx_of(context);
  if (!ctx->ao_basis.provided) return qmckl_failwith(context, QMCKL_NOT_PROVIDED, names[which], "AO basis not provided");
  if (need_mo && !ctx->mo_basis.provided)
    return qmckl_failwith(context, QMCKL_NOT_PROVIDED, names[which], "MO basis not provided");
  const int64_t sze = per_point_nucl * ctx->point.num * ctx->nucleus.num;
  if (size_max < sze)
    return qmckl_failwith(context, QMCKL_INVALID_ARG_3, names[which],
                          which == 3 ? "Array too small. Expected walk_num*nucl_num*point_num*3" : "input array too small");
  if (out == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, names[which], "NULL pointer");
  return dev_provide_forces(context, which, out);
}

qmckl_exit_code qmckl_get_forces_ao_value(qmckl_context context, double* const forces_ao_value,
                                          const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_NULL_CONTEXT;
  return forces_getter(context, 3, forces_ao_value, size_max, false, 3 * ctx_of(context)->ao_basis.ao_num);
}

qmckl_exit_code qmckl_get_forces_mo_value(qmckl_context context, double* const forces_mo_value,
                                          const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_NULL_CONTEXT;
  return forces_getter(context, 0, forces_mo_value, size_max, true, 3 * ctx_of(context)->mo_basis.mo_num);
}

qmckl_exit_code qmckl_get_forces_mo_value_inplace(qmckl_context context, double* const forces_mo_value,
                                                  const int64_t size_max) {
  return qmckl_get_forces_mo_value(context, forces_mo_value, size_max);
}

qmckl_exit_code qmckl_get_forces_mo_g(qmckl_context context, double* const forces_mo_g, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_NULL_CONTEXT;
  return forces_getter(context, 1, forces_mo_g, size_max, true, 9 * ctx_of(context)->mo_basis.mo_num);
}

qmckl_exit_code qmckl_get_forces_mo_g_inplace(qmckl_context context, double* const forces_mo_g,
                                              const int64_t size_max) {
  return qmckl_get_forces_mo_g(context, forces_mo_g, size_max);
}

qmckl_exit_code qmckl_get_forces_mo_l(qmckl_context context, double* const forces_mo_l, const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_NULL_CONTEXT;
  return forces_getter(context, 2, forces_mo_l, size_max, true, 3 * ctx_of(context)->mo_basis.mo_num);
}

qmckl_exit_code qmckl_b200_ao_hessian_device(qmckl_context context, const int64_t point_num, const double* d_coord,
                                             double* d_ao_hessian) {
  qmckl_exit_code rc =
      device_entry(context, "qmckl_b200_ao_hessian_device", point_num, d_coord, d_ao_hessian, false);
  if (rc != QMCKL_SUCCESS) return rc;
  Context* ctx = ctx_of(context);
  QB_CUDA(launch_ao_hessian(state(context)->T, point_num, d_coord, cutoff_of(ctx), ctx->precision <= 23, d_ao_hessian,
                            state(context)->stream),
          "qmckl_b200_ao_hessian_device");
  return QMCKL_SUCCESS;
}

// Adjoint of MO VGL.  With L = sum_{p,c,i} W[p][c][i] mo_vgl[p][c][i]:
//   grad_coef[i][k]  = sum_{p,c} W[p][c][i] ao_vgl[p][c][k]
//   grad_nucl[a][d]  = dL/dR_a,  grad_coord[d][p] = dL/dr_p
// Points are processed in chunks that bound the scratch to about 2 GiB.  Per
// chunk: the AO matrix is recomputed (nothing of the forward pass is kept),
// grad_coef accumulates AO^T W (split-K FP64 GEMM, partials summed in a fixed
// order), the AO buffer is then overwritten with G = W C ([point][5][ao]) and
// the derivative kernel contracts G with the AO Hessian and Laplacian
// gradient into grad_nucl / grad_coord.
}  // extern "C"

namespace qb {
namespace {

// Rows of W and of the AO matrix per K slice of the coefficient-gradient
// contraction: each slice accumulates in FP32 in one CTA, the slices are
// summed in FP64.  On the adjoint workload (40,704 points, 2000 AOs, 160 MOs)
// the largest error of dL/dC against the FP64 form is 4.0e-7 of the largest
// entry with 2048 rows, 7.0e-7 with 4096 and 1.7e-6 with 16384.
constexpr int kAdjointSliceRows = 2048;

// Mixed-form adjoint: the two contractions on the tensor cores.  Per chunk
// of points: the weights W[(p,c)][mo] as 3 bfloat16 pieces; the AOs in FP64
// arithmetic (FP32 exponentials where a r^2 <= 30, as in the derivative
// kernel) stored as 3 bfloat16 pieces of rows p*5 + c; dC += AO^T W by the
// split-K TN kernel, the partials summed in a fixed order into the [mo][ao]
// layout; G = W C^T (FP32) from the pieces of coefficient_t; then the
// derivative kernel in its mixed form.  Synchronizes once at the end to read
// the kernels' error word.
qmckl_exit_code adjoint_mixed(qmckl_context context, DeviceState* ds, int64_t P, const double* d_coord,
                              const double* d_weight, double* d_grad_coef, double* d_grad_nucl, double* d_grad_coord) {
  const char* fname = "qmckl_b200_mo_vgl_adjoint_device";
  Context* ctx = ctx_of(context);
  const int64_t A = ctx->ao_basis.ao_num, M = ctx->mo_basis.mo_num, N = ctx->nucleus.num;
  const double cutoff = cutoff_of(ctx);
  cudaStream_t s = ds->stream;
  const int64_t ldw = (M + 7) / 8 * 8, lda = (A + 7) / 8 * 8;
  const int kps = kAdjointSliceRows / 32;
  qmckl_exit_code rc = sync_coef(context, ds);
  if (rc != QMCKL_SUCCESS) return rc;
  if (ds->adj_ct_version != ctx->mo_basis.coef_version || !ds->adj_ct.p) {
    rc = ensure(context, ds->adj_ct, sizeof(uint16_t) * 3 * A * ldw, fname);
    if (rc != QMCKL_SUCCESS) return rc;
    QB_CUDA(tc_split_rows((const double*)ds->coef_t.p, A, (int)M, M, ds->adj_ct.p, (int)ldw, A * ldw, s), fname);
    ds->adj_ct_version = ctx->mo_basis.coef_version;
  }
  const int64_t budget = (int64_t)2 << 30;
  const int64_t row_bytes = std::max<int64_t>(20 * A, 30 * lda);   // G (FP32) or the AO pieces, per point
  const int64_t max_chunk = std::min<int64_t>(P, std::max<int64_t>(64, budget / row_bytes));
  const int64_t nchunks = (P + max_chunk - 1) / max_chunk;
  const int64_t chunk = (P + nchunks - 1) / nchunks;   // equal chunks keep every launch full
  const int splits = tc_tn_splits(5 * chunk, kps);
  rc = ensure(context, ds->adj_coord, sizeof(double) * 3 * chunk, fname);
  if (rc == QMCKL_SUCCESS) rc = ensure(context, ds->adj_buf, (size_t)row_bytes * chunk, fname);
  if (rc == QMCKL_SUCCESS) rc = ensure(context, ds->adj_wp, sizeof(uint16_t) * 3 * 5 * chunk * ldw, fname);
  if (rc == QMCKL_SUCCESS && ds->tc_err.p == nullptr) {
    rc = ensure(context, ds->tc_err, sizeof(int), fname);
    if (rc == QMCKL_SUCCESS) QB_CUDA(cudaMemsetAsync(ds->tc_err.p, 0, sizeof(int), s), fname);
  }
  if (rc == QMCKL_SUCCESS && d_grad_coef) rc = ensure(context, ds->adj_part, sizeof(double) * splits * A * M, fname);
  if (rc == QMCKL_SUCCESS && !d_grad_nucl) rc = ensure(context, ds->adj_nucl, sizeof(double) * 3 * N, fname);
  if (rc != QMCKL_SUCCESS) return rc;
  double* gnucl = d_grad_nucl ? d_grad_nucl : (double*)ds->adj_nucl.p;
  void* buf = ds->adj_buf.p;
  double* cc = (double*)ds->adj_coord.p;
  // a bounded wait that gives up is left in the context's error word for its
  // next synchronization point (qmckl_b200_synchronize, a host getter)
  int* err = (int*)ds->tc_err.p;
  for (int64_t p0 = 0; p0 < P; p0 += chunk) {
    const int64_t n = std::min<int64_t>(chunk, P - p0), rows = 5 * n;
    const double* w = d_weight + p0 * 5 * M;
    QB_CUDA(cudaMemcpy2DAsync(cc, sizeof(double) * n, d_coord + p0, sizeof(double) * P, sizeof(double) * n, 3,
                              cudaMemcpyDeviceToDevice, s), fname);
    QB_CUDA(tc_split_rows(w, rows, (int)M, M, ds->adj_wp.p, (int)ldw, rows * ldw, s), fname);
    if (d_grad_coef) {
      QB_CUDA(launch_ao_vgl_pieces(ds->T, n, cc, cutoff, false, buf, lda, rows * lda, s), fname);
      QB_CUDA(tc_gemm_tn_split(buf, lda, rows * lda, A, ds->adj_wp.p, ldw, rows * ldw, (int)M, rows, kps,
                               (double*)ds->adj_part.p, err, s),
              fname);
      QB_CUDA(launch_add_transposed((const double*)ds->adj_part.p, tc_tn_splits(rows, kps), A, M, d_grad_coef, true,
                                    s),
              fname);
    }
    if (d_grad_nucl || d_grad_coord) {
      QB_CUDA(tc_gemm_nt(ds->adj_wp.p, ldw, rows * ldw, rows, M, ds->adj_ct.p, ldw, A * ldw, A, (float*)buf, A, err,
                         s),
              fname);
      QB_CUDA(launch_mo_adjoint_nuclear(ds->T, n, cc, n, cutoff, true, buf, gnucl,
                                        d_grad_coord ? d_grad_coord + p0 : nullptr, P, s),
              fname);
    }
  }
  return QMCKL_SUCCESS;
}

}  // namespace
}  // namespace qb

extern "C" {

qmckl_exit_code qmckl_b200_mo_vgl_adjoint_device(qmckl_context context, const int64_t point_num,
                                                 const double* d_coord, const double* d_weight, double* d_grad_coef,
                                                 double* d_grad_nucl, double* d_grad_coord) {
  const char* fname = "qmckl_b200_mo_vgl_adjoint_device";
  qmckl_exit_code rc = device_entry(context, fname, point_num, d_coord, (void*)d_weight, true);
  if (rc != QMCKL_SUCCESS) return rc;
  if (!ctx_of(context)->mo_basis.r_cusp.empty())
    return qmckl_failwith(context, QMCKL_FAILURE, fname,
                          "the adjoint is that of the MOs without the cusp adjustment, and r_cusp is set");
  Context* ctx = ctx_of(context);
  DeviceState* ds = state(context);
  const int64_t P = point_num, A = ctx->ao_basis.ao_num, M = ctx->mo_basis.mo_num, N = ctx->nucleus.num;
  const bool mixed = use_mixed(ctx) || ctx->precision <= 23;
  const double cutoff = cutoff_of(ctx);
  cudaStream_t s = ds->stream;
  if (d_grad_coef) QB_CUDA(cudaMemsetAsync(d_grad_coef, 0, sizeof(double) * M * A, s), fname);
  if (d_grad_nucl) QB_CUDA(cudaMemsetAsync(d_grad_nucl, 0, sizeof(double) * 3 * N, s), fname);
  if (d_grad_coord) QB_CUDA(cudaMemsetAsync(d_grad_coord, 0, sizeof(double) * 3 * P, s), fname);
  if (P == 0 || (!d_grad_coef && !d_grad_nucl && !d_grad_coord)) return QMCKL_SUCCESS;
  if (mixed) return adjoint_mixed(context, ds, P, d_coord, d_weight, d_grad_coef, d_grad_nucl, d_grad_coord);
  // FP64 coefficient rows [mo][ao] for G = W C
  if (ds->coef_rows_version != ctx->mo_basis.coef_version || !ds->coef_rows.p) {
    rc = ensure(context, ds->coef_rows, sizeof(double) * M * A, fname);
    if (rc != QMCKL_SUCCESS) return rc;
    QB_CUDA(cudaMemcpyAsync(ds->coef_rows.p, ctx->mo_basis.coefficient.data(), sizeof(double) * M * A,
                            cudaMemcpyHostToDevice, s), fname);
    ds->coef_rows_version = ctx->mo_basis.coef_version;
  }
  const int64_t budget = (int64_t)2 << 30;
  const int64_t chunk = std::min<int64_t>(P, std::max<int64_t>(64, budget / (int64_t)(40 * A)));
  // split-K count: about two CTAs per SM for the (ao x mo) output tiles
  const int64_t tiles = ((A + 127) / 128) * ((M + 79) / 80);
  const int splits = (int)std::max<int64_t>(1, std::min<int64_t>(32, (2 * 148 + tiles - 1) / tiles));
  rc = ensure(context, ds->adj_coord, sizeof(double) * 3 * chunk, fname);
  if (rc == QMCKL_SUCCESS) rc = ensure(context, ds->adj_buf, sizeof(double) * 5 * chunk * A, fname);
  if (rc == QMCKL_SUCCESS && d_grad_coef) rc = ensure(context, ds->adj_part, sizeof(double) * splits * A * M, fname);
  if (rc == QMCKL_SUCCESS && !d_grad_nucl) rc = ensure(context, ds->adj_nucl, sizeof(double) * 3 * N, fname);
  if (rc != QMCKL_SUCCESS) return rc;
  double* gnucl = d_grad_nucl ? d_grad_nucl : (double*)ds->adj_nucl.p;
  double* buf = (double*)ds->adj_buf.p;
  double* cc = (double*)ds->adj_coord.p;
  for (int64_t p0 = 0; p0 < P; p0 += chunk) {
    const int64_t n = std::min<int64_t>(chunk, P - p0);
    const double* w = d_weight + p0 * 5 * M;
    QB_CUDA(cudaMemcpy2DAsync(cc, sizeof(double) * n, d_coord + p0, sizeof(double) * P, sizeof(double) * n, 3,
                              cudaMemcpyDeviceToDevice, s), fname);
    if (d_grad_coef) {
      QB_CUDA(launch_ao_vgl_f64(ds->T, n, cc, cutoff, !mixed, buf, s), fname);
      QB_CUDA(launch_gemm_f64_tn_split(A, M, 5 * n, buf, A, w, M, (double*)ds->adj_part.p, splits, s), fname);
      QB_CUDA(launch_add_transposed((const double*)ds->adj_part.p, splits, A, M, d_grad_coef, true, s), fname);
    }
    if (d_grad_nucl || d_grad_coord) {
      QB_CUDA(launch_gemm_f64(5 * n, A, M, w, M, (const double*)ds->coef_rows.p, A, buf, A, s), fname);
      QB_CUDA(launch_mo_adjoint_nuclear(ds->T, n, cc, n, cutoff, mixed, buf, gnucl,
                                        d_grad_coord ? d_grad_coord + p0 : nullptr, P, s),
              fname);
    }
  }
  // the AO scratch of the FP64 form was not touched; cached arrays stay valid
  return QMCKL_SUCCESS;
}

}  // extern "C"
