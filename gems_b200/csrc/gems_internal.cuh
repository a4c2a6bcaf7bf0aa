// gems_internal.cuh -- device-session state shared by the CUDA translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/gems_b200.h"
#include "plan.h"

namespace gems {

// 2^-256 underflow threshold and its log (tree/phylotree.h:61-80)
constexpr double kScaleThr = 8.636168555094444625386e-78;
constexpr int kScaleExp = 256;
constexpr double kLogScaleThr = -177.4456782233459932741;
// mixed precision (FP32 real-space partials): rescale by 2^64 below 2^-64
constexpr float kScaleThrF = 5.421010862427522e-20f;  // 2^-64
constexpr int kScaleExpF = 64;
constexpr double kLogScaleThrF = -44.361419555836498;  // 64 * log(2) negated

constexpr int kMaxStates = 64;
constexpr int kMaxCat = 16;

// device copy of gems_op (same layout)
struct DevOp {
  int dst_slot;
  int l_kind, l_id;
  int r_kind, r_id;
  int pad_;
  double l_len, r_len;
};
static_assert(sizeof(DevOp) == sizeof(gems_op), "op layout");

// per-launch view of a session, passed by value to kernels
struct DevCtx {
  int P;         // padded pattern count (multiple of 32)
  int nptn;      // real pattern count
  int n, C, block, G;  // states, categories, C*n, lanes per pattern (pow2 >= C)
  int unknown;   // STATE_UNKNOWN
  int safe;
  const uint8_t *tips;   // [ntaxa][P]
  const double *freq;    // [P]
  const double *invar;   // [P]
  void *partials;        // [nslots][P][block] (double, or float in mixed; see mix_off)
  uint16_t *scale;       // [nslots][P * (safe ? C : 1)]
  const double *inv_evec;  // [n][n]
  const double *evec;      // [n][n]
  const double *eval;      // [n]
  const double *rates;     // [C]
  const double *props;     // [C]
  const double *tip;       // [(unknown+1)][n] eigen-space tip vectors
  const double *tip_real;  // [(unknown+1)][n] indicator vectors (mixed path)
  double *theta;           // [P][block]
  double *scale_all;       // [P]
  double *pattern_lh;      // [P]
  double *df_frac;         // [P]
  double *ddf_term;        // [P] ddf_frac - df_frac^2 (reweighted derivatives)
  double *red;             // reduction partials
  size_t slot_elems;       // P * block (tiled: P rounded up to 128, times block)
  size_t slot_scale;       // P * (safe ? C : 1)
};

// Layout of FP32 partials.  The 4-, 20- and 61-state mixed forms store each slot tile-major:
//   [tile of 128 patterns][chunk = category * K + state / 4][128 rows][4 states]
// with K = 1 (4 states), 5 (20 states) or 16 (61 states padded to 64, the pad stored as zeros).  This is
// the tensor-core operand layout: one contiguous block per (tile, slot) -- or per (tile, slot,
// category) for 61 states -- so a tile moves with one bulk copy, and a warp's 32 rows of one
// chunk are 512 contiguous bytes; for 4 states a thread that holds a pattern's C categories
// stores C float4s, each instruction of a warp a contiguous 512-byte run.
// mix_off<N>: offset of state 0 of category cc of pattern p within a slot; mix_cs<N>: floats
// between consecutive 4-state chunks of that row; mix_k<N>: chunks per category (0: not tiled).
constexpr int kMixTile = 128;
template <int N>
__host__ __device__ constexpr int mix_k() {
  return N == 20 ? 5 : (N == 61 ? 16 : (N == 4 ? 1 : 0));
}
template <int N>
__host__ __device__ inline size_t mix_off(const DevCtx &c, long p, int cc) {
  if constexpr (mix_k<N>() > 0) {
    constexpr int K = mix_k<N>();
    return (size_t)(p / kMixTile) * ((size_t)c.C * K * kMixTile * 4) +
           (size_t)cc * K * kMixTile * 4 + (size_t)(p % kMixTile) * 4;
  } else {
    return (size_t)p * c.block + (size_t)cc * N;
  }
}
template <int N>
__host__ __device__ constexpr int mix_cs() {
  return mix_k<N>() > 0 ? kMixTile * 4 : 4;
}

// Layout of FP64 partials: pattern-major [P][C][n], except 4 states, tile-major like the mixed
// forms so that stores coalesce:
//   [tile of 128 patterns][category][half h: states 2h, 2h + 1][128 rows][2 doubles]
// (a lane's or thread's 16-byte store of one half, and a warp's store of a category half is one
// contiguous run).  f64_off: offset of a (pattern, category) row's states x, x + 1 (x even).
constexpr int kF64Half = kMixTile * 2;  // doubles between the two halves of a row
template <int N>
__host__ __device__ inline size_t f64_off(const DevCtx &c, long p, int cc, int x = 0) {
  if constexpr (N == 4) {
    return (size_t)(p / kMixTile) * ((size_t)c.C * 2 * kF64Half) +
           (size_t)(2 * cc + (x >> 1)) * kF64Half + (size_t)(p % kMixTile) * 2 + (x & 1);
  } else {
    return (size_t)p * c.block + (size_t)cc * N + x;
  }
}

#ifdef __CUDACC__
// a (pattern, category) row of an FP64 partial slot, in 16-byte pieces (N even) or doubles
template <int N>
__device__ __forceinline__ void load_row(const double *__restrict__ slot, const DevCtx &c, long p,
                                         int cc, double (&v)[N]) {
  if constexpr (N % 2 == 0) {
#pragma unroll
    for (int i = 0; i < N; i += 2) {
      const double2 t = __ldcg(reinterpret_cast<const double2 *>(slot + f64_off<N>(c, p, cc, i)));
      v[i] = t.x, v[i + 1] = t.y;
    }
  } else {
    const double *src = slot + f64_off<N>(c, p, cc);
#pragma unroll
    for (int i = 0; i < N; i++) v[i] = __ldcg(src + i);
  }
}
template <int N>
__device__ __forceinline__ void store_row(double *__restrict__ slot, const DevCtx &c, long p,
                                          int cc, const double (&v)[N]) {
  if constexpr (N % 2 == 0) {
#pragma unroll
    for (int i = 0; i < N; i += 2)
      *reinterpret_cast<double2 *>(slot + f64_off<N>(c, p, cc, i)) = make_double2(v[i], v[i + 1]);
  } else {
    double *dst = slot + f64_off<N>(c, p, cc);
#pragma unroll
    for (int i = 0; i < N; i++) dst[i] = v[i];
  }
}
#endif

// one session of a batched tensor-core launch (sessions that share the op list: the same tree
// and lengths, e.g. candidate models on one alignment)
struct TcJob {
  DevCtx c;
  const DevOp *ops;
  const float *tab;
};

struct Session {
  gems_session_desc desc;
  int P = 0;
  int unknown = 0;
  int block = 0;
  int G = 1;
  int nops_max = 0;
  int plan_depth = 0;    // stack positions the uploaded op list's plan uses
  size_t op_stride = 0;  // doubles per op in opmats
  cudaStream_t stream = nullptr;
  bool model_set = false;
  bool tips_ok = true;  // false after a rejected tip upload
  bool theta_valid = false;
  gems_branch theta_branch{};
  long long launches = 0;
  // device buffers
  uint8_t *d_tips = nullptr;
  double *d_freq = nullptr, *d_invar = nullptr;
  void *d_partials = nullptr;
  uint16_t *d_scale = nullptr;
  double *d_theta = nullptr, *d_scale_all = nullptr, *d_pattern_lh = nullptr, *d_df_frac = nullptr;
  double *d_ddf_term = nullptr;
  // bootstrap reweightings (RELL): R rows of P pattern counts
  float *d_rell_w = nullptr;       // [R][P] counts, then the partial-sum scratch
  double *d_rell_part = nullptr;
  int rell_R = 0;
  size_t rell_ld = 0;
  double *d_model = nullptr;  // eval | evec | inv_evec | rates | props | tip | tip_real
  DevOp *d_ops = nullptr;
  double *d_opmats = nullptr;
  double *d_branch = nullptr;  // per-branch tables: val0,val1,val2 [block] + tip table
  double *d_red = nullptr;     // reduction partials
  double *d_result = nullptr;  // final scalars
  int *d_flag = nullptr;       // device status flags (barrier timeouts)
  unsigned int *d_bar = nullptr;  // grid barrier counters
  // batched launches led by this session: job table (device and pinned host copies)
  static constexpr int kMaxBatch = 128;
  TcJob *d_jobs = nullptr;
  TcJob *h_jobs = nullptr;
  // streamed evaluation from host data (gems_branch_lnl_from_host): a copy stream, one event
  // per pattern chunk and a pinned word for the tip check, created on first use
  static constexpr int kMaxChunks = 64;
  cudaStream_t copy_stream = nullptr;
  cudaStream_t check_stream = nullptr;  // tip-byte checks of the chunks the copy stream brought
  cudaEvent_t start_ev = nullptr;
  cudaEvent_t chunk_ev[kMaxChunks] = {};
  unsigned int *h_tipmax = nullptr;
  // pinned host staging
  DevOp *h_ops = nullptr;
  double *h_result = nullptr;
  int nred = 0;  // size of d_red in doubles
  std::vector<double> h_evec, h_inv;  // host copy of the eigenvectors in use
  // tensor-core path (20 states, mixed): per-op table stride in floats
  bool tc_enabled = true;
  // FP64 61-state traversal as register-tiled GEMMs (else the per-row kernel)
  bool g61_enabled = true;
  // 4-state traversal: launch shape chosen by timing the variants on the first large traversal
  bool autotune = true;
  int force_shape = -1;  // >= 0: that launch shape, no tuning (comparisons)
  int newton_share = 1;  // the Newton kernel takes at most 1/newton_share of the GPU
  bool tc20_halves = false;  // 20-state tcgen05 traversal at two CTAs per SM, in half-steps
  bool tc61_roles = true;    // 61-state tcgen05 traversal with split / MMA / epilogue warp roles
  size_t op_stride_tc = 0;
  // FP32 partials stored tile-major (20- and 61-state mixed forms); elements per slot
  bool tiled = false;
  size_t slot_elems = 0;
  // kernel timing (gems_profile_*): event pairs recorded around launches
  static constexpr int kProfKernels = 8;
  bool prof_on = false;
  struct ProfPair {
    cudaEvent_t a, b;
    int kernel;
  };
  std::vector<ProfPair> prof_pending;
  std::vector<cudaEvent_t> prof_free;
  double prof_ms[kProfKernels] = {};
  long long prof_n[kProfKernels] = {};
  DevCtx ctx() const;
};

// tip bytes into a session (host or device source), checked on the device (session.cu)
int load_tips(Session *s, const uint8_t *src, size_t src_pitch, cudaMemcpyKind kind);

// brackets a launch with timing events when profiling is on
int prof_begin(Session *s, int kernel, cudaEvent_t *a);
int prof_end(Session *s, int kernel, cudaEvent_t a);
void prof_collect(Session *s);

// error handling
void set_error(const std::string &msg);
int cuda_status(cudaError_t e, const char *what);

#define GEMS_CUDA(call)                                   \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return cuda_status(e_, #call); \
  } while (0)

// launch helpers implemented in kernels.cu
int launch_prep_ops(Session *s, int nops);
// patterns [p0, p1) of the traversal, p1 <= P (every launch_traverse* below alike)
int launch_traverse(Session *s, int nops, int p0, int p1);
int launch_branch_lnl(Session *s, const gems_branch *br, double *lnl);
int launch_theta(Session *s, const gems_branch *br);
int launch_derv(Session *s, double length, double *df, double *ddf);
int launch_from_buffer(Session *s, double length, double *lnl);
int launch_newton(Session *s, double length0, double min_len, double max_len, double xacc,
                  int max_steps, double *opt_len, int *nevals);
// the same in two halves: enqueue (result copied to pinned host memory), then wait and read
int launch_newton_async(Session *s, double guess, double min_len, double max_len, double xacc,
                        int max_steps);
int newton_result(Session *s, double *opt_len, int *nevals);
int launch_eigen(Session *s, const double *exch_upper, const double *freq);
// the same for nsess sessions of one state count in one launch (inputs stacked per session)
int launch_eigen_batch(Session *const *ss, int nsess, const double *exch_upper,
                       const double *freq);
// mixed precision (kernels_mixed.cu)
int launch_prep_ops_mixed(Session *s, int nops);
int launch_traverse_mixed(Session *s, int nops, int p0, int p1);
// the same without waiting: with want_lnl the result is copied to s->h_result, read by
// theta_mixed_lnl once the session's stream has completed
int enqueue_theta_mixed(Session *s, const gems_branch *br, bool want_lnl, bool store_theta);
double theta_mixed_lnl(const Session *s);
int launch_theta_mixed(Session *s, const gems_branch *br, bool want_lnl, bool store_theta,
                       double *lnl);
// factored whole-traversal kernels for 4 and 20 states (kernels_traverse.cu)
bool traverse_v2_supported(const Session *s);
int launch_prep_ops_v2(Session *s, int nops);
// patterns [p0, p1) of the traversal (p1 <= P); tip state bytes are clamped to STATE_UNKNOWN
int launch_traverse_v2(Session *s, int nops, int p0, int p1);
// patterns that one wave of resident blocks of the traversal kernel covers (0 if unknown)
int traverse_v2_wave_patterns(const Session *s);
// launch shape of the 4-state traversal in use for this session's class (patterns per lane
// group, blocks per SM); returns 1 while the tuner has not chosen yet, else 0
int traverse_v2_shape(const Session *s, int *patterns_per_group, int *blocks_per_sm);
// tcgen05 split-TF32 traversal for 20 states (kernels_tc.cu)
size_t tc20_op_floats(int ncat, int unknown);
bool tc20_supported(const Session *s);
int launch_prep_ops_tc20(Session *s, int nops);
// p0 a multiple of 128, p1 a multiple of 128 or P
int launch_traverse_tc20(Session *s, int nops, int p0, int p1);
// tcgen05 split-TF32 traversal for 61 states, SAFE (kernels_tc61.cu)
size_t tc61_op_floats(int ncat);
bool tc61_supported(const Session *s);
int launch_prep_ops_tc61(Session *s, int nops);
// p0 a multiple of 128, p1 a multiple of 128 or P
int launch_traverse_tc61(Session *s, int nops, int p0, int p1);
int launch_traverse_tc61_batch(Session *const *ss, int nsess, int nops, int p0, int p1,
                               bool with_tables);
// FP64 61-state traversal as register-tiled GEMMs, C in {1, 2, 4, 8} (kernels_g61.cu)
size_t g61_op_doubles(int ncat, int unknown);
bool g61_supported(const Session *s);
int launch_prep_ops_g61(Session *s, int nops);
// p0 and p1 multiples of g61_pattern_granule (p1 may be P)
int g61_pattern_granule(const Session *s);
int launch_traverse_g61(Session *s, int nops, int p0, int p1);
// the grid barrier's time-out path, run on purpose (kernels_fp64.cu)
int check_barrier_timeout(int device, int *status);
// bootstrap reweighting (kernels_rell.cu)
// scratch of the tiled reductions (per replicate row and pattern chunk), in doubles
size_t rell_scratch_doubles(int R, int P);
int launch_rell_lnl(Session *s, double *d_out);
int launch_rell_derv(Session *s, double *d_out);

}  // namespace gems

struct gems_session : public gems::Session {};
