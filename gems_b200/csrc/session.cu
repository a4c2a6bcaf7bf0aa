// session.cu -- C-ABI of the kernel set: device sessions, uploads, model, kernel calls.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "gems_internal.cuh"

namespace gems {

static thread_local std::string g_err;

void set_error(const std::string &msg) { g_err = msg; }

int cuda_status(cudaError_t e, const char *what) {
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) return GEMS_ERR_OOM;
  return GEMS_ERR_CUDA;
}

DevCtx Session::ctx() const {
  DevCtx c{};
  c.P = P;
  c.nptn = desc.nptn;
  c.n = desc.nstates;
  c.C = desc.ncat;
  c.block = block;
  c.G = G;
  c.unknown = unknown;
  c.safe = desc.scaling == GEMS_SCALE_SAFE;
  c.tips = d_tips;
  c.freq = d_freq;
  c.invar = d_invar;
  c.partials = d_partials;
  c.scale = d_scale;
  const int n = desc.nstates;
  c.eval = d_model;
  c.evec = d_model + n;
  c.inv_evec = d_model + n + n * n;
  c.rates = d_model + n + 2 * n * n;
  c.props = c.rates + desc.ncat;
  c.tip = c.props + desc.ncat;
  c.tip_real = c.tip + (size_t)(unknown + 1) * n;
  c.theta = d_theta;
  c.scale_all = d_scale_all;
  c.pattern_lh = d_pattern_lh;
  c.df_frac = d_df_frac;
  c.ddf_term = d_ddf_term;
  c.red = d_red;
  c.slot_elems = slot_elems;
  c.slot_scale = (size_t)P * (desc.scaling == GEMS_SCALE_SAFE ? desc.ncat : 1);
  return c;
}

static cudaEvent_t prof_event(Session *s) {
  cudaEvent_t e = nullptr;
  if (!s->prof_free.empty()) {
    e = s->prof_free.back();
    s->prof_free.pop_back();
  } else if (cudaEventCreate(&e) != cudaSuccess) {
    e = nullptr;
  }
  return e;
}

int prof_begin(Session *s, int kernel, cudaEvent_t *a) {
  (void)kernel;
  *a = nullptr;
  if (!s->prof_on) return GEMS_OK;
  *a = prof_event(s);
  if (*a) GEMS_CUDA(cudaEventRecord(*a, s->stream));
  return GEMS_OK;
}

int prof_end(Session *s, int kernel, cudaEvent_t a) {
  if (!a) return GEMS_OK;
  cudaEvent_t b = prof_event(s);
  if (!b) return GEMS_OK;
  GEMS_CUDA(cudaEventRecord(b, s->stream));
  s->prof_pending.push_back({a, b, kernel});
  return GEMS_OK;
}

void prof_collect(Session *s) {
  for (auto &pp : s->prof_pending) {
    float ms = 0.f;
    if (cudaEventSynchronize(pp.b) == cudaSuccess &&
        cudaEventElapsedTime(&ms, pp.a, pp.b) == cudaSuccess && pp.kernel >= 0 &&
        pp.kernel < Session::kProfKernels) {
      s->prof_ms[pp.kernel] += ms;
      s->prof_n[pp.kernel] += 1;
    }
    s->prof_free.push_back(pp.a);
    s->prof_free.push_back(pp.b);
  }
  s->prof_pending.clear();
}

static int state_unknown(int n) { return n == 4 ? 18 : (n == 20 ? 23 : n); }
static int pad_patterns(int nptn) { return ((nptn + 63) / 64) * 64; }
static int pow2_at_least(int x) {
  int g = 1;
  while (g < x) g <<= 1;
  return g;
}

struct Sizes {
  bool tiled;
  size_t slot_elems;
  size_t partial_bytes, scale_bytes, theta_bytes, opmats_bytes, branch_bytes, red_doubles,
      model_doubles, total;
  int nops_max;
  size_t op_stride;
};

static Sizes compute_sizes(const gems_session_desc &d) {
  Sizes z{};
  const size_t P = pad_patterns(d.nptn);
  const size_t blk = (size_t)d.nstates * d.ncat;
  const int unk = state_unknown(d.nstates);
  const size_t elem = d.precision == GEMS_PREC_MIXED ? sizeof(float) : sizeof(double);
  // 20- and 61-state mixed partials are tile-major in 128-pattern tiles (the tensor-core
  // layout; 61 states padded to 64)
  z.tiled = (d.nstates == 4 || d.nstates == 20 || d.nstates == 61) &&
            d.precision == GEMS_PREC_MIXED;
  z.slot_elems = z.tiled ? (P + kMixTile - 1) / kMixTile * kMixTile * d.ncat *
                               (d.nstates == 61 ? 64 : d.nstates)
                         : d.nstates == 4 ? (P + kMixTile - 1) / kMixTile * kMixTile * blk
                                          : P * blk;  // FP64 4 states: tile-major (f64_off)
  z.partial_bytes = (size_t)d.nslots * z.slot_elems * elem;
  z.scale_bytes = (size_t)d.nslots * P * (d.scaling == GEMS_SCALE_SAFE ? d.ncat : 1) * 2;
  // theta + scale_all, pattern_lh, df_frac, ddf_term
  z.theta_bytes = P * blk * sizeof(double) + 4 * P * sizeof(double);
  z.nops_max = d.ntaxa + 8;
  z.op_stride = 2 * (size_t)d.ncat * d.nstates * d.nstates + 2 * (size_t)(unk + 1) * blk;
  if (d.nstates == 20 && d.precision == GEMS_PREC_MIXED && d.ncat <= 4) {
    // the tensor-core tables (floats) share the buffer
    const size_t need = (tc20_op_floats(d.ncat, unk) + 1) / 2;
    if (z.op_stride < need) z.op_stride = need;
  }
  if (d.nstates == 61 && d.precision == GEMS_PREC_MIXED && d.scaling == GEMS_SCALE_SAFE) {
    const size_t need = (tc61_op_floats(d.ncat) + 1) / 2;
    if (z.op_stride < need) z.op_stride = need;
  }
  if (d.nstates == 61 && d.precision == GEMS_PREC_FP64) {
    const size_t need = g61_op_doubles(d.ncat, unk);
    if (z.op_stride < need) z.op_stride = need;
  }
  z.op_stride = (z.op_stride + 7) & ~(size_t)7;  // 64-byte aligned op tables
  z.opmats_bytes = (size_t)z.nops_max * z.op_stride * sizeof(double);
  z.branch_bytes = (3 * blk + (size_t)(unk + 1) * blk) * sizeof(double);
  z.red_doubles = 4 * (P * 16 / 256 + 1024);
  z.model_doubles = d.nstates + 2 * (size_t)d.nstates * d.nstates + 2 * d.ncat +
                    2 * (size_t)(unk + 1) * d.nstates;
  z.total = z.partial_bytes + z.scale_bytes + z.theta_bytes + z.opmats_bytes + z.branch_bytes +
            z.red_doubles * 8 + z.model_doubles * 8 + (size_t)d.ntaxa * P + 2 * P * 8 +
            (size_t)z.nops_max * sizeof(DevOp);
  return z;
}

static int validate(const gems_session_desc *d) {
  if (!d) return GEMS_ERR_BAD_ARG;
  if (d->ntaxa < 3 || d->nptn < 1 || d->nstates < 2 || d->nstates > kMaxStates || d->ncat < 1 ||
      d->ncat > kMaxCat || d->nslots < 1 ||
      (d->precision != GEMS_PREC_FP64 && d->precision != GEMS_PREC_MIXED) ||
      (d->scaling != GEMS_SCALE_NORM && d->scaling != GEMS_SCALE_SAFE)) {
    set_error("invalid session descriptor");
    return GEMS_ERR_BAD_ARG;
  }
  if (d->nstates != 4 && d->nstates != 20 && d->nstates != 61) {
    set_error("state count must be 4, 20 or 61");
    return GEMS_ERR_BAD_ARG;
  }
  return GEMS_OK;
}

static void free_session(Session *s) {
  cudaFree(s->d_tips);
  cudaFree(s->d_freq);
  cudaFree(s->d_invar);
  cudaFree(s->d_partials);
  cudaFree(s->d_scale);
  cudaFree(s->d_theta);
  cudaFree(s->d_rell_w);
  cudaFree(s->d_model);
  cudaFree(s->d_ops);
  cudaFree(s->d_opmats);
  cudaFree(s->d_branch);
  cudaFree(s->d_red);
  cudaFree(s->d_result);
  cudaFree(s->d_flag);
  cudaFree(s->d_bar);
  cudaFreeHost(s->h_ops);
  cudaFree(s->d_jobs);
  cudaFreeHost(s->h_jobs);
  cudaFreeHost(s->h_result);
  if (s->copy_stream) {
    cudaStreamSynchronize(s->copy_stream);
    cudaStreamDestroy(s->copy_stream);
  }
  if (s->check_stream) {
    cudaStreamSynchronize(s->check_stream);
    cudaStreamDestroy(s->check_stream);
  }
  if (s->start_ev) cudaEventDestroy(s->start_ev);
  for (cudaEvent_t e : s->chunk_ev)
    if (e) cudaEventDestroy(e);
  cudaFreeHost(s->h_tipmax);
  if (s->stream) {
    cudaStreamSynchronize(s->stream);
    prof_collect(s);
    for (cudaEvent_t e : s->prof_free) cudaEventDestroy(e);
    s->prof_free.clear();
    cudaStreamDestroy(s->stream);
  }
}

static int upload_ops(Session *s, const gems_op *ops, int nops) {
  if (nops < 0 || nops > s->nops_max) {
    set_error("too many traversal ops");
    return GEMS_ERR_BAD_ARG;
  }
  if (nops == 0) return GEMS_OK;
  for (int k = 0; k < nops; k++) {
    const gems_op &o = ops[k];
    auto bad_child = [&](int kind, int id) {
      if (kind == GEMS_CHILD_TIP) return id < 0 || id >= s->desc.ntaxa;
      if (kind == GEMS_CHILD_PARTIAL) return id < 0 || id >= s->desc.nslots || id == o.dst_slot;
      return true;
    };
    if (o.dst_slot < 0 || o.dst_slot >= s->desc.nslots || bad_child(o.left_kind, o.left_id) ||
        bad_child(o.right_kind, o.right_id) || !(o.left_len >= 0) || !(o.right_len >= 0)) {
      set_error("invalid traversal op");
      return GEMS_ERR_BAD_ARG;
    }
  }
  // host staging: wait for any kernel still reading the previous op table
  GEMS_CUDA(cudaStreamSynchronize(s->stream));
  s->plan_depth = plan_ops(ops, nops, s->desc.nslots, reinterpret_cast<gems_op *>(s->h_ops));
  GEMS_CUDA(cudaMemcpyAsync(s->d_ops, s->h_ops, sizeof(DevOp) * nops, cudaMemcpyHostToDevice,
                            s->stream));
  return GEMS_OK;
}

static int check_branch(Session *s, const gems_branch *br) {
  if (!br || br->dad_slot < 0 || br->dad_slot >= s->desc.nslots || !(br->length >= 0)) {
    set_error("invalid branch");
    return GEMS_ERR_BAD_ARG;
  }
  if (br->node_kind == GEMS_CHILD_TIP) {
    if (br->node_id < 0 || br->node_id >= s->desc.ntaxa) return GEMS_ERR_BAD_ARG;
  } else if (br->node_kind == GEMS_CHILD_PARTIAL) {
    if (br->node_id < 0 || br->node_id >= s->desc.nslots || br->node_id == br->dad_slot)
      return GEMS_ERR_BAD_ARG;
  } else {
    return GEMS_ERR_BAD_ARG;
  }
  return GEMS_OK;
}

static void invalidate_theta(Session *s, const gems_op *ops, int nops) {
  for (int k = 0; k < nops; k++)
    if (s->theta_valid &&
        (ops[k].dst_slot == s->theta_branch.dad_slot ||
         (s->theta_branch.node_kind == GEMS_CHILD_PARTIAL &&
          ops[k].dst_slot == s->theta_branch.node_id)))
      s->theta_valid = false;
}

// The traversal kernel family a session uses, and the pattern granule a pattern range of it
// must respect (lower bound a multiple of it; upper bound a multiple of it or the end).
enum class Form { kTc20, kTc61, kV2, kG61, kMixed, kFp64 };

static Form traversal_form(const Session *s) {
  if (tc20_supported(s)) return Form::kTc20;
  if (tc61_supported(s)) return Form::kTc61;
  if (traverse_v2_supported(s)) return Form::kV2;
  if (g61_supported(s)) return Form::kG61;
  return s->desc.precision == GEMS_PREC_MIXED ? Form::kMixed : Form::kFp64;
}

static int pattern_granule(const Session *s) {
  switch (traversal_form(s)) {
    case Form::kTc20:
    case Form::kTc61: return 128;
    case Form::kG61: return g61_pattern_granule(s);
    default: return 1;
  }
}

// the op tables of `nops` uploaded ops, then their traversal over patterns [p0, p1)
static int run_ops_range(Session *s, const gems_op *ops, int nops, int p0, int p1) {
  if (!s->model_set) {
    set_error("model not set");
    return GEMS_ERR_STATE;
  }
  if (!s->tips_ok) {
    set_error("tip states invalid (last upload was rejected)");
    return GEMS_ERR_STATE;
  }
  int st = upload_ops(s, ops, nops);
  if (st) return st;
  switch (traversal_form(s)) {
    case Form::kTc20:
      if ((st = launch_prep_ops_tc20(s, nops))) return st;
      if ((st = launch_traverse_tc20(s, nops, p0, p1))) return st;
      break;
    case Form::kTc61:
      if ((st = launch_prep_ops_tc61(s, nops))) return st;
      if ((st = launch_traverse_tc61(s, nops, p0, p1))) return st;
      break;
    case Form::kV2:
      if ((st = launch_prep_ops_v2(s, nops))) return st;
      if ((st = launch_traverse_v2(s, nops, p0, p1))) return st;
      break;
    case Form::kG61:
      if ((st = launch_prep_ops_g61(s, nops))) return st;
      if ((st = launch_traverse_g61(s, nops, p0, p1))) return st;
      break;
    case Form::kMixed:
      if ((st = launch_prep_ops_mixed(s, nops))) return st;
      if ((st = launch_traverse_mixed(s, nops, p0, p1))) return st;
      break;
    case Form::kFp64:
      if ((st = launch_prep_ops(s, nops))) return st;
      if ((st = launch_traverse(s, nops, p0, p1))) return st;
      break;
  }
  invalidate_theta(s, ops, nops);
  return GEMS_OK;
}

static int run_ops(Session *s, const gems_op *ops, int nops) {
  return run_ops_range(s, ops, nops, 0, s->P);
}

static void copy_pattern_lh(Session *s, double *pattern_lh, double lnl_raw_finite) {
  (void)lnl_raw_finite;
  if (!pattern_lh) return;
  cudaMemcpyAsync(pattern_lh, s->d_pattern_lh, sizeof(double) * s->desc.nptn,
                  cudaMemcpyDeviceToHost, s->stream);
  cudaStreamSynchronize(s->stream);
  for (int p = 0; p < s->desc.nptn; p++)
    if (!std::isfinite(pattern_lh[p])) pattern_lh[p] = 4.0 * kLogScaleThr;
}

// largest state byte of the uploaded tips in columns [c0, c1) (rows of P bytes, P a multiple of
// 64, the first nptn of each row valid; c0 and c1 multiples of 16): a grid-stride loop over
// 16-byte words, per-byte maxima with __vmaxu4
__global__ void k_tips_max(const uint8_t *__restrict__ tips, int P, int nptn, int ntaxa, int c0,
                           int c1, unsigned int *out) {
  const long long words_per_row = (c1 - c0) / 16, total = words_per_row * ntaxa;
  unsigned int m4 = 0;
  for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < total;
       w += (long long)gridDim.x * blockDim.x) {
    const long long row = w / words_per_row;
    const int col = c0 + (int)(w - row * words_per_row) * 16;
    uint4 v = *reinterpret_cast<const uint4 *>(tips + row * P + col);
    if (col + 16 > nptn) {  // the row's padding bytes do not count
      unsigned int b[4] = {v.x, v.y, v.z, v.w};
      for (int j = 0; j < 16; j++)
        if (col + j >= nptn) b[j / 4] &= ~(0xFFu << (8 * (j % 4)));
      v = make_uint4(b[0], b[1], b[2], b[3]);
    }
    m4 = __vmaxu4(m4, __vmaxu4(__vmaxu4(v.x, v.y), __vmaxu4(v.z, v.w)));
  }
  unsigned int m = max(max(m4 & 0xFFu, (m4 >> 8) & 0xFFu), max((m4 >> 16) & 0xFFu, m4 >> 24));
  m = __reduce_max_sync(0xffffffffu, m);
  if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

// copies rows of nptn tip bytes (host or device, row stride src_pitch) into the session and
// checks them on the device: on a bad byte the tips of the session are invalid (traversals are
// refused) until the next successful load
int load_tips(Session *s, const uint8_t *src, size_t src_pitch, cudaMemcpyKind kind) {
  unsigned int *d_max = reinterpret_cast<unsigned int *>(s->d_flag) + 8;
  GEMS_CUDA(cudaMemsetAsync(d_max, 0, sizeof(unsigned int), s->stream));
  GEMS_CUDA(cudaMemcpy2DAsync(s->d_tips, s->P, src, src_pitch, s->desc.nptn, s->desc.ntaxa, kind,
                              s->stream));
  k_tips_max<<<148 * 8, 256, 0, s->stream>>>(s->d_tips, s->P, s->desc.nptn, s->desc.ntaxa, 0,
                                             s->P, d_max);
  s->launches++;
  GEMS_CUDA(cudaGetLastError());
  unsigned int mx = 0;
  GEMS_CUDA(cudaMemcpyAsync(&mx, d_max, sizeof(mx), cudaMemcpyDeviceToHost, s->stream));
  GEMS_CUDA(cudaStreamSynchronize(s->stream));
  s->theta_valid = false;
  if ((int)mx > s->unknown) {
    s->tips_ok = false;
    set_error("tip state byte out of range");
    return GEMS_ERR_BAD_ARG;
  }
  s->tips_ok = true;
  return GEMS_OK;
}

}  // namespace gems

using namespace gems;

extern "C" {

const char *gems_version(void) { return "gems_b200 0.1 (sm_100a)"; }
const char *gems_last_error(void) { return gems::g_err.c_str(); }

int gems_device_count(int *count) {
  if (!count) return GEMS_ERR_BAD_ARG;
  cudaError_t e = cudaGetDeviceCount(count);
  if (e != cudaSuccess) {
    *count = 0;
    cudaGetLastError();
    set_error(cudaGetErrorString(e));
    return GEMS_ERR_NO_DEVICE;
  }
  return GEMS_OK;
}

int gems_session_footprint(const gems_session_desc *desc, size_t *bytes) {
  int st = validate(desc);
  if (st) return st;
  if (!bytes) return GEMS_ERR_BAD_ARG;
  *bytes = compute_sizes(*desc).total;
  return GEMS_OK;
}

int gems_session_create(const gems_session_desc *desc, gems_session **out) {
  int st = validate(desc);
  if (st) return st;
  if (!out) return GEMS_ERR_BAD_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("no CUDA device");
    return GEMS_ERR_NO_DEVICE;
  }
  if (desc->device < 0 || desc->device >= ndev) return GEMS_ERR_BAD_ARG;
  GEMS_CUDA(cudaSetDevice(desc->device));
  Sizes z = compute_sizes(*desc);
  size_t free_b = 0, total_b = 0;
  GEMS_CUDA(cudaMemGetInfo(&free_b, &total_b));
  if (z.total > free_b) {
    set_error("session footprint exceeds free device memory");
    return GEMS_ERR_ADMISSION;
  }
  gems_session *s = new gems_session();
  s->desc = *desc;
  s->P = pad_patterns(desc->nptn);
  s->unknown = state_unknown(desc->nstates);
  s->block = desc->nstates * desc->ncat;
  s->G = pow2_at_least(desc->ncat);
  s->nops_max = z.nops_max;
  s->op_stride = z.op_stride;
  s->op_stride_tc = 2 * z.op_stride;  // same buffer viewed as floats
  s->nred = (int)z.red_doubles;
  s->tiled = z.tiled;
  s->slot_elems = z.slot_elems;
  auto fail = [&](cudaError_t e, const char *what) {
    int code = cuda_status(e, what);
    free_session(s);
    delete s;
    return code;
  };
  cudaError_t e;
#define ALLOC(ptr, bytes)                                           \
  if ((e = cudaMalloc((void **)&(ptr), (bytes))) != cudaSuccess) \
    return fail(e, "cudaMalloc " #ptr);
  const size_t P = s->P;
  ALLOC(s->d_tips, (size_t)desc->ntaxa * P);
  ALLOC(s->d_freq, P * sizeof(double));
  ALLOC(s->d_invar, P * sizeof(double));
  ALLOC(s->d_partials, z.partial_bytes);
  ALLOC(s->d_scale, z.scale_bytes);
  ALLOC(s->d_theta, z.theta_bytes);
  s->d_scale_all = s->d_theta + P * s->block;
  s->d_pattern_lh = s->d_scale_all + P;
  s->d_df_frac = s->d_pattern_lh + P;
  s->d_ddf_term = s->d_df_frac + P;
  ALLOC(s->d_model, z.model_doubles * sizeof(double));
  ALLOC(s->d_ops, (size_t)z.nops_max * sizeof(DevOp));
  ALLOC(s->d_opmats, z.opmats_bytes);
  ALLOC(s->d_branch, z.branch_bytes);
  ALLOC(s->d_red, z.red_doubles * sizeof(double));
  ALLOC(s->d_result, 16 * sizeof(double));
  ALLOC(s->d_flag, 16 * sizeof(int));
  ALLOC(s->d_bar, 16 * sizeof(unsigned int));
#undef ALLOC
  if ((e = cudaHostAlloc((void **)&s->h_ops, (size_t)z.nops_max * sizeof(DevOp), 0)) !=
      cudaSuccess)
    return fail(e, "cudaHostAlloc ops");
  if ((e = cudaMalloc((void **)&s->d_jobs, sizeof(TcJob) * Session::kMaxBatch)) != cudaSuccess)
    return fail(e, "cudaMalloc jobs");
  if ((e = cudaHostAlloc((void **)&s->h_jobs, sizeof(TcJob) * Session::kMaxBatch, 0)) !=
      cudaSuccess)
    return fail(e, "cudaHostAlloc jobs");
  if ((e = cudaHostAlloc((void **)&s->h_result, 16 * sizeof(double), 0)) != cudaSuccess)
    return fail(e, "cudaHostAlloc result");
  if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess)
    return fail(e, "cudaStreamCreate");
  // padded patterns: unknown state, weight 0, zero scale counters
  if ((e = cudaMemsetAsync(s->d_tips, s->unknown, (size_t)desc->ntaxa * P, s->stream)) ||
      (e = cudaMemsetAsync(s->d_freq, 0, P * sizeof(double), s->stream)) ||
      (e = cudaMemsetAsync(s->d_invar, 0, P * sizeof(double), s->stream)) ||
      (e = cudaMemsetAsync(s->d_scale, 0, z.scale_bytes, s->stream)) ||
      (e = cudaStreamSynchronize(s->stream)))
    return fail(e, "initialise session");
  *out = s;
  return GEMS_OK;
}

int gems_session_destroy(gems_session *s) {
  if (!s) return GEMS_ERR_BAD_ARG;
  cudaSetDevice(s->desc.device);
  cudaStreamSynchronize(s->stream);
  free_session(s);
  delete s;
  return GEMS_OK;
}

int gems_session_traversal_shape(gems_session *s, int *patterns_per_group, int *blocks_per_sm,
                                 int *tuned) {
  if (!s || !patterns_per_group || !blocks_per_sm || !tuned) return GEMS_ERR_BAD_ARG;
  *tuned = traverse_v2_shape(s, patterns_per_group, blocks_per_sm) == 0 && s->desc.nstates == 4;
  return GEMS_OK;
}

int gems_check_barrier_timeout(int device, int *status) {
  if (!status) return GEMS_ERR_BAD_ARG;
  return check_barrier_timeout(device, status);
}

int gems_session_sync(gems_session *s) {
  if (!s) return GEMS_ERR_BAD_ARG;
  GEMS_CUDA(cudaStreamSynchronize(s->stream));
  return GEMS_OK;
}

int gems_session_info(gems_session *s, gems_session_desc *desc) {
  if (!s || !desc) return GEMS_ERR_BAD_ARG;
  *desc = s->desc;
  return GEMS_OK;
}

int gems_session_set_option(gems_session *s, int option, int value) {
  if (!s) return GEMS_ERR_BAD_ARG;
  switch (option) {
    case GEMS_OPT_TENSOR_CORES:
      s->tc_enabled = value != 0;
      return GEMS_OK;
    case GEMS_OPT_TILED_FP64:
      s->g61_enabled = value != 0;
      return GEMS_OK;
    case GEMS_OPT_NEWTON_SHARE:
      if (value < 1 || value > 64) return GEMS_ERR_BAD_ARG;
      s->newton_share = value;
      return GEMS_OK;
    case GEMS_OPT_TC20_HALVES:
      s->tc20_halves = value != 0;
      return GEMS_OK;
    case GEMS_OPT_TC61_ROLES:
      s->tc61_roles = value != 0;
      return GEMS_OK;
    case GEMS_OPT_AUTOTUNE:
      if (value < 0) return GEMS_ERR_BAD_ARG;
      s->autotune = value == 1;
      s->force_shape = value >= 2 ? value - 2 : -1;
      return GEMS_OK;
    default:
      return GEMS_ERR_BAD_ARG;
  }
}

int gems_session_stream(gems_session *s, void **stream) {
  if (!s || !stream) return GEMS_ERR_BAD_ARG;
  *stream = (void *)s->stream;
  return GEMS_OK;
}

int gems_upload_tips(gems_session *s, const uint8_t *states) {
  if (!s || !states) return GEMS_ERR_BAD_ARG;
  GEMS_CUDA(cudaSetDevice(s->desc.device));
  return load_tips(s, states, s->desc.nptn, cudaMemcpyHostToDevice);
}

int gems_upload_patterns(gems_session *s, const double *ptn_freq, const double *ptn_invar) {
  if (!s || !ptn_freq) return GEMS_ERR_BAD_ARG;
  GEMS_CUDA(cudaSetDevice(s->desc.device));
  const int n = s->desc.nptn;
  GEMS_CUDA(cudaMemcpyAsync(s->d_freq, ptn_freq, n * sizeof(double), cudaMemcpyHostToDevice,
                            s->stream));
  if (ptn_invar) {
    GEMS_CUDA(cudaMemcpyAsync(s->d_invar, ptn_invar, n * sizeof(double), cudaMemcpyHostToDevice,
                              s->stream));
  } else {
    GEMS_CUDA(cudaMemsetAsync(s->d_invar, 0, n * sizeof(double), s->stream));
  }
  GEMS_CUDA(cudaStreamSynchronize(s->stream));
  s->theta_valid = false;
  return GEMS_OK;
}

// tip vectors for every state code: real-space indicator and eigen-space inv_evec . indicator
// (phylotreesse.cpp:361-371, modelsubst.cpp:183-208, modeldna.cpp:462-474,
//  modelprotein.cpp:1240-1255)
static void build_tip_tables(int n, int unk, const double *inv_evec, std::vector<double> &tip,
                             std::vector<double> &tip_real) {
  tip.assign((size_t)(unk + 1) * n, 0.0);
  tip_real.assign((size_t)(unk + 1) * n, 0.0);
  static const int amb_aa[3][2] = {{2, 3}, {5, 6}, {9, 10}};
  for (int s = 0; s <= unk; s++) {
    double *ind = &tip_real[(size_t)s * n];
    if (s < n) {
      ind[s] = 1.0;
    } else if (n == 4 && s < 18) {
      const int cs = s - n + 1;
      for (int j = 0; j < 4; j++)
        if (cs & (1 << j)) ind[j] = 1.0;
    } else if (n == 20 && s < 23) {
      ind[amb_aa[s - 20][0]] = 1.0;
      ind[amb_aa[s - 20][1]] = 1.0;
    } else {
      for (int j = 0; j < n; j++) ind[j] = 1.0;
    }
    for (int i = 0; i < n; i++) {
      double acc = 0.0;
      for (int j = 0; j < n; j++) acc += inv_evec[i * n + j] * ind[j];
      tip[(size_t)s * n + i] = acc;
    }
  }
}

static int upload_model(gems_session *s, const double *eval, const double *evec,
                        const double *inv_evec, const double *rates, const double *props) {
  const int n = s->desc.nstates, C = s->desc.ncat;
  std::vector<double> tip, tip_real;
  build_tip_tables(n, s->unknown, inv_evec, tip, tip_real);
  std::vector<double> m;
  m.insert(m.end(), eval, eval + n);
  m.insert(m.end(), evec, evec + n * n);
  m.insert(m.end(), inv_evec, inv_evec + n * n);
  m.insert(m.end(), rates, rates + C);
  m.insert(m.end(), props, props + C);
  m.insert(m.end(), tip.begin(), tip.end());
  m.insert(m.end(), tip_real.begin(), tip_real.end());
  GEMS_CUDA(cudaMemcpyAsync(s->d_model, m.data(), m.size() * sizeof(double),
                            cudaMemcpyHostToDevice, s->stream));
  GEMS_CUDA(cudaStreamSynchronize(s->stream));
  s->h_evec.assign(evec, evec + n * n);
  s->h_inv.assign(inv_evec, inv_evec + n * n);
  s->model_set = true;
  s->theta_valid = false;
  return GEMS_OK;
}

int gems_set_model(gems_session *s, const double *eval, const double *evec,
                   const double *inv_evec, const double *rates, const double *props) {
  if (!s || !eval || !evec || !inv_evec || !rates || !props) return GEMS_ERR_BAD_ARG;
  GEMS_CUDA(cudaSetDevice(s->desc.device));
  for (int c = 0; c < s->desc.ncat; c++)
    if (!(rates[c] >= 0) || !(props[c] >= 0)) return GEMS_ERR_BAD_ARG;
  return upload_model(s, eval, evec, inv_evec, rates, props);
}

int gems_set_rates(gems_session *s, const double *rates, const double *props) {
  if (!s || !rates || !props) return GEMS_ERR_BAD_ARG;
  if (!s->model_set) {
    set_error("model not set");
    return GEMS_ERR_STATE;
  }
  const int n = s->desc.nstates, C = s->desc.ncat;
  for (int c = 0; c < C; c++)
    if (!(rates[c] >= 0) || !(props[c] >= 0)) return GEMS_ERR_BAD_ARG;
  GEMS_CUDA(cudaSetDevice(s->desc.device));
  // the model block is [eval n][evec n*n][inv_evec n*n][rates C][props C][tip tables]: only the
  // rates and proportions change (the tip tables depend on inv_evec alone)
  std::vector<double> rp(rates, rates + C);
  rp.insert(rp.end(), props, props + C);
  GEMS_CUDA(cudaMemcpyAsync(s->d_model + n + 2 * (size_t)n * n, rp.data(), rp.size() * sizeof(double),
                            cudaMemcpyHostToDevice, s->stream));
  GEMS_CUDA(cudaStreamSynchronize(s->stream));
  s->theta_valid = false;
  return GEMS_OK;
}

int gems_set_model_from_rates(gems_session *s, const double *exch_upper, const double *freq,
                              const double *rates, const double *props) {
  if (!s || !exch_upper || !freq || !rates || !props) return GEMS_ERR_BAD_ARG;
  GEMS_CUDA(cudaSetDevice(s->desc.device));
  const int n = s->desc.nstates, C = s->desc.ncat;
  int st = launch_eigen(s, exch_upper, freq);
  if (st) return st;
  std::vector<double> es((size_t)n + 2 * n * n);
  GEMS_CUDA(cudaMemcpyAsync(es.data(), s->d_model, es.size() * sizeof(double),
                            cudaMemcpyDeviceToHost, s->stream));
  GEMS_CUDA(cudaStreamSynchronize(s->stream));
  (void)C;
  return upload_model(s, es.data(), es.data() + n, es.data() + n + n * n, rates, props);
}

int gems_set_model_from_rates_batch(gems_session *const *ss, int nsess, const double *exch_upper,
                                    const double *freq, const double *rates,
                                    const double *props) {
  if (!ss || nsess < 1 || nsess > Session::kMaxBatch || !exch_upper || !freq || !rates || !props)
    return GEMS_ERR_BAD_ARG;
  for (int i = 0; i < nsess; i++) {
    if (!ss[i] || ss[i]->desc.device != ss[0]->desc.device ||
        ss[i]->desc.nstates != ss[0]->desc.nstates || ss[i]->desc.ncat != ss[0]->desc.ncat) {
      set_error("batched models: sessions must share device, state and category counts");
      return GEMS_ERR_BAD_ARG;
    }
    for (int j = 0; j < i; j++)
      if (ss[j] == ss[i]) return GEMS_ERR_BAD_ARG;
  }
  const int n = ss[0]->desc.nstates, C = ss[0]->desc.ncat;
  for (int i = 0; i < nsess * C; i++)
    if (!(rates[i] >= 0) || !(props[i] >= 0)) return GEMS_ERR_BAD_ARG;
  GEMS_CUDA(cudaSetDevice(ss[0]->desc.device));
  std::vector<Session *> v(ss, ss + nsess);
  if (int st = launch_eigen_batch(v.data(), nsess, exch_upper, freq)) return st;
  std::vector<double> es((size_t)n + 2 * n * n);
  for (int i = 0; i < nsess; i++) {
    GEMS_CUDA(cudaMemcpy(es.data(), ss[i]->d_model, es.size() * sizeof(double),
                         cudaMemcpyDeviceToHost));
    if (int st = upload_model(ss[i], es.data(), es.data() + n, es.data() + n + n * n,
                              rates + (size_t)i * C, props + (size_t)i * C))
      return st;
  }
  return GEMS_OK;
}

int gems_get_eigensystem(gems_session *s, double *eval, double *evec, double *inv_evec) {
  if (!s || !s->model_set) return GEMS_ERR_STATE;
  const int n = s->desc.nstates;
  std::vector<double> es((size_t)n + 2 * n * n);
  GEMS_CUDA(cudaMemcpyAsync(es.data(), s->d_model, es.size() * sizeof(double),
                            cudaMemcpyDeviceToHost, s->stream));
  GEMS_CUDA(cudaStreamSynchronize(s->stream));
  if (eval) std::memcpy(eval, es.data(), n * sizeof(double));
  if (evec) std::memcpy(evec, es.data() + n, n * n * sizeof(double));
  if (inv_evec) std::memcpy(inv_evec, es.data() + n + n * n, n * n * sizeof(double));
  return GEMS_OK;
}

int gems_traverse(gems_session *s, const gems_op *ops, int nops) {
  if (!s || (nops > 0 && !ops)) return GEMS_ERR_BAD_ARG;
  GEMS_CUDA(cudaSetDevice(s->desc.device));
  int st = run_ops(s, ops, nops);
  if (st) return st;
  GEMS_CUDA(cudaStreamSynchronize(s->stream));
  return GEMS_OK;
}

int gems_session_pattern_granule(gems_session *s, int *granule) {
  if (!s || !granule) return GEMS_ERR_BAD_ARG;
  *granule = pattern_granule(s);
  return GEMS_OK;
}

int gems_compute_partial(gems_session *s, const gems_op *op, int ptn_lower, int ptn_upper) {
  if (!s || !op) return GEMS_ERR_BAD_ARG;
  const int n = s->desc.nptn, g = pattern_granule(s);
  if (ptn_lower < 0 || ptn_upper > n || ptn_lower >= ptn_upper || ptn_lower % g != 0 ||
      (ptn_upper % g != 0 && ptn_upper != n)) {
    set_error("gems_compute_partial: pattern range out of bounds or not aligned to the "
              "session's pattern granule (gems_session_pattern_granule)");
    return GEMS_ERR_BAD_ARG;
  }
  GEMS_CUDA(cudaSetDevice(s->desc.device));
  // the last range of a traversal also covers the padding patterns, as a whole-list traversal
  // does, so that the slot holds the same bytes either way
  const int p1 = ptn_upper == n ? s->P : ptn_upper;
  int st = run_ops_range(s, op, 1, ptn_lower, p1);
  if (st) return st;
  GEMS_CUDA(cudaStreamSynchronize(s->stream));
  return GEMS_OK;
}

// every session's own op list (ops[i], nops[i]); sessions must share device, pattern count,
// states, categories and slots.  All tcgen05 61-state sessions with lists of one length: one
// launch for every session's op tables and one traversal launch over every (session, tile);
// otherwise one traversal per session, each on its own stream (their work overlaps).
static int traverse_batch_lists(gems_session *const *ss, int nsess, const gems_op *const *ops,
                                const int *nops) {
  if (!ss || !ops || !nops || nsess <= 0 || nsess > Session::kMaxBatch) return GEMS_ERR_BAD_ARG;
  Session *s0 = ss[0];
  if (!s0) return GEMS_ERR_BAD_ARG;
  bool tc = true;
  for (int i = 0; i < nsess; i++) {
    Session *s = ss[i];
    if (!s || s->desc.device != s0->desc.device || s->desc.nptn != s0->desc.nptn ||
        s->desc.nstates != s0->desc.nstates || s->desc.ncat != s0->desc.ncat ||
        s->desc.nslots != s0->desc.nslots) {
      set_error("batched sessions must share device, patterns, states, categories and slots");
      return GEMS_ERR_BAD_ARG;
    }
    if (nops[i] < 0 || (nops[i] > 0 && !ops[i])) return GEMS_ERR_BAD_ARG;
    if (!s->model_set || !s->tips_ok) {
      set_error(!s->model_set ? "model not set" : "tip states invalid (last upload was rejected)");
      return GEMS_ERR_STATE;
    }
    for (int j = 0; j < i; j++)
      if (ss[j] == s) {
        set_error("a session appears twice in the batch");
        return GEMS_ERR_BAD_ARG;
      }
    tc = tc && tc61_supported(s) && nops[i] == nops[0];
  }
  GEMS_CUDA(cudaSetDevice(s0->desc.device));
  if (!tc || nops[0] == 0) {
    for (int i = 0; i < nsess; i++)
      if (int st = run_ops(ss[i], ops[i], nops[i])) return st;
    for (int i = 0; i < nsess; i++) GEMS_CUDA(cudaStreamSynchronize(ss[i]->stream));
    return GEMS_OK;
  }
  // one op list shared by every session (candidate models on one tree): validated and planned
  // once, the plan copied to each session
  bool shared = true;
  for (int i = 1; i < nsess; i++)
    shared = shared && ops[i] == ops[0] && ss[i]->desc.ntaxa == s0->desc.ntaxa &&
             ss[i]->nops_max == s0->nops_max;
  if (int st = upload_ops(s0, ops[0], nops[0])) return st;
  for (int i = 1; i < nsess; i++) {
    Session *s = ss[i];
    if (!shared) {
      if (int st = upload_ops(s, ops[i], nops[i])) return st;
      continue;
    }
    GEMS_CUDA(cudaStreamSynchronize(s->stream));  // no kernel still reads its op table
    std::memcpy(s->h_ops, s0->h_ops, sizeof(DevOp) * nops[0]);
    s->plan_depth = s0->plan_depth;
    GEMS_CUDA(cudaMemcpyAsync(s->d_ops, s->h_ops, sizeof(DevOp) * nops[0], cudaMemcpyHostToDevice,
                              s->stream));
  }
  // the batched launches (every session's op tables, then the traversal) run on the first
  // session's stream after every session's op list is on the device
  for (int i = 1; i < nsess; i++) GEMS_CUDA(cudaStreamSynchronize(ss[i]->stream));
  std::vector<Session *> v(ss, ss + nsess);
  if (int st = launch_traverse_tc61_batch(v.data(), nsess, nops[0], 0, s0->P, true)) return st;
  for (int i = 0; i < nsess; i++) invalidate_theta(ss[i], ops[i], nops[i]);
  return GEMS_OK;
}

int gems_traverse_batch(gems_session *const *ss, int nsess, const gems_op *ops, int nops) {
  if (!ss || nsess <= 0 || nsess > Session::kMaxBatch || (nops > 0 && !ops))
    return GEMS_ERR_BAD_ARG;
  std::vector<const gems_op *> o(nsess, ops);
  std::vector<int> n(nsess, nops);
  return traverse_batch_lists(ss, nsess, o.data(), n.data());
}

int gems_branch_lnl_batch_ops(gems_session *const *ss, int nsess, const gems_op *const *ops,
                              const int *nops, const gems_branch *br, double *lnl) {
  if (!lnl || !br) return GEMS_ERR_BAD_ARG;
  for (int i = 0; i < nsess && ss; i++)
    if (ss[i])
      if (int st = check_branch(ss[i], &br[i])) return st;
  if (int st = traverse_batch_lists(ss, nsess, ops, nops)) return st;
  bool mixed = true;
  for (int i = 0; i < nsess; i++) mixed = mixed && ss[i]->desc.precision == GEMS_PREC_MIXED;
  if (!mixed) {
    for (int i = 0; i < nsess; i++)
      if (int st = gems_branch_lnl(ss[i], nullptr, 0, &br[i], &lnl[i], nullptr)) return st;
    return GEMS_OK;
  }
  // every session's branch terms enqueued on its own stream first, then the results read
  for (int i = 0; i < nsess; i++)
    if (int st = enqueue_theta_mixed(ss[i], &br[i], true, false)) return st;
  for (int i = 0; i < nsess; i++) {
    GEMS_CUDA(cudaStreamSynchronize(ss[i]->stream));
    lnl[i] = theta_mixed_lnl(ss[i]);
  }
  return GEMS_OK;
}

int gems_branch_lnl_batch(gems_session *const *ss, int nsess, const gems_op *ops, int nops,
                          const gems_branch *br, double *lnl) {
  if (!ss || !lnl || !br || nsess <= 0 || nsess > Session::kMaxBatch) return GEMS_ERR_BAD_ARG;
  std::vector<const gems_op *> o(nsess, ops);
  std::vector<int> n(nsess, nops);
  std::vector<gems_branch> b(nsess, *br);
  return gems_branch_lnl_batch_ops(ss, nsess, o.data(), n.data(), b.data(), lnl);
}

int gems_branch_lnl(gems_session *s, const gems_op *ops, int nops, const gems_branch *br,
                    double *lnl, double *pattern_lh) {
  if (!s || !lnl || (nops > 0 && !ops)) return GEMS_ERR_BAD_ARG;
  GEMS_CUDA(cudaSetDevice(s->desc.device));
  int st = check_branch(s, br);
  if (st) return st;
  if ((st = run_ops(s, ops, nops))) return st;
  if (s->desc.precision == GEMS_PREC_MIXED)
    st = launch_theta_mixed(s, br, true, false, lnl);
  else
    st = launch_branch_lnl(s, br, lnl);
  if (st) return st;
  copy_pattern_lh(s, pattern_lh, *lnl);
  return GEMS_OK;
}

// New tips, pattern weights and +I terms from the host, then the lnL of one branch, with the
// upload overlapped with the traversal: the tip rows go up in `nchunks` pattern chunks on a
// copy stream, each checked there (k_tips_max over its columns), and the traversal of a chunk
// starts on the session stream as soon as its copy is done.  The check is read on the host once
// the last copy is done, while the traversal still runs; the traversal clamps state bytes, so a
// bad byte makes the call fail and the tips invalid, as gems_upload_tips does.  Sessions whose
// traversal kernel does not take a pattern range (tcgen05, 61 states, generic n) load first and
// evaluate after.
int gems_branch_lnl_from_host(gems_session *s, const uint8_t *states, const double *ptn_freq,
                              const double *ptn_invar, const gems_op *ops, int nops,
                              const gems_branch *br, int nchunks, double *lnl,
                              double *pattern_lh) {
  if (!s || !states || !ptn_freq || !lnl || (nops > 0 && !ops) || nchunks < 1 ||
      nchunks > Session::kMaxChunks)
    return GEMS_ERR_BAD_ARG;
  GEMS_CUDA(cudaSetDevice(s->desc.device));
  int st = check_branch(s, br);
  if (st) return st;
  if (!s->model_set) {
    set_error("model not set");
    return GEMS_ERR_STATE;
  }
  const bool ranged = traverse_v2_supported(s) && !tc20_supported(s) && !tc61_supported(s);
  if (!ranged || nchunks == 1 || nops == 0) {
    if ((st = gems_upload_tips(s, states))) return st;
    if ((st = gems_upload_patterns(s, ptn_freq, ptn_invar))) return st;
    return gems_branch_lnl(s, ops, nops, br, lnl, pattern_lh);
  }
  if (!s->copy_stream)
    GEMS_CUDA(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking));
  if (!s->check_stream)
    GEMS_CUDA(cudaStreamCreateWithFlags(&s->check_stream, cudaStreamNonBlocking));
  if (!s->start_ev) GEMS_CUDA(cudaEventCreateWithFlags(&s->start_ev, cudaEventDisableTiming));
  for (cudaEvent_t &e : s->chunk_ev)
    if (!e) GEMS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  if (!s->h_tipmax) GEMS_CUDA(cudaHostAlloc((void **)&s->h_tipmax, sizeof(unsigned int), 0));
  const int n = s->desc.nptn, ntaxa = s->desc.ntaxa;
  unsigned int *d_max = reinterpret_cast<unsigned int *>(s->d_flag) + 8;
  // the copy stream carries only the copies, back to back; each chunk's tip-byte check runs on
  // the check stream once the chunk has arrived, beside the next copy
  cudaStream_t cs = s->copy_stream, ks = s->check_stream;
  // nothing queued on the session stream may still read the old tips, weights or +I terms
  GEMS_CUDA(cudaEventRecord(s->start_ev, s->stream));
  GEMS_CUDA(cudaStreamWaitEvent(cs, s->start_ev, 0));
  GEMS_CUDA(cudaStreamWaitEvent(ks, s->start_ev, 0));
  GEMS_CUDA(cudaMemsetAsync(d_max, 0, sizeof(unsigned int), ks));
  // +I terms first (the traversal's scaling rule reads them); the weights, which only the branch
  // terms read, go up after the last tip chunk
  if (ptn_invar)
    GEMS_CUDA(
        cudaMemcpyAsync(s->d_invar, ptn_invar, n * sizeof(double), cudaMemcpyHostToDevice, cs));
  else
    GEMS_CUDA(cudaMemsetAsync(s->d_invar, 0, n * sizeof(double), cs));
  s->theta_valid = false;
  // the op tables do not depend on the data: prepared while the first chunk goes up
  if ((st = upload_ops(s, ops, nops))) return st;
  if ((st = launch_prep_ops_v2(s, nops))) return st;
  // chunks of whole waves of resident blocks, so that no chunk's launch ends on a partly filled
  // wave, rounded to 128 patterns (P is a multiple of 64: every bound is a multiple of 16)
  const int wave = std::max(128, traverse_v2_wave_patterns(s));
  const int waves = (s->P + wave - 1) / wave;
  const long long per = (long long)((waves + nchunks - 1) / nchunks) * wave;
  const int chunk = (int)std::min<long long>((per + 127) / 128 * 128, (s->P + 127) / 128 * 128);
  for (int c = 0, p0 = 0; p0 < s->P; c++, p0 += chunk) {
    const int p1 = std::min(s->P, p0 + chunk);
    const int w = std::min(p1, n) - p0;
    if (w > 0)
      GEMS_CUDA(cudaMemcpy2DAsync(s->d_tips + p0, s->P, states + p0, n, w, ntaxa,
                                  cudaMemcpyHostToDevice, cs));
    GEMS_CUDA(cudaEventRecord(s->chunk_ev[c], cs));
    GEMS_CUDA(cudaStreamWaitEvent(ks, s->chunk_ev[c], 0));
    const long long words = (long long)(p1 - p0) / 16 * ntaxa;
    const int grid = (int)std::min<long long>(148 * 8, (words + 255) / 256);
    k_tips_max<<<grid, 256, 0, ks>>>(s->d_tips, s->P, n, ntaxa, p0, p1, d_max);
    s->launches++;
    GEMS_CUDA(cudaGetLastError());
    GEMS_CUDA(cudaStreamWaitEvent(s->stream, s->chunk_ev[c], 0));
    if ((st = launch_traverse_v2(s, nops, p0, p1))) return st;
  }
  GEMS_CUDA(cudaMemcpyAsync(s->d_freq, ptn_freq, n * sizeof(double), cudaMemcpyHostToDevice, cs));
  GEMS_CUDA(cudaMemcpyAsync(s->h_tipmax, d_max, sizeof(unsigned int), cudaMemcpyDeviceToHost, ks));
  GEMS_CUDA(cudaStreamSynchronize(cs));
  GEMS_CUDA(cudaStreamSynchronize(ks));
  if ((int)*s->h_tipmax > s->unknown) {
    s->tips_ok = false;
    GEMS_CUDA(cudaStreamSynchronize(s->stream));
    set_error("tip state byte out of range");
    return GEMS_ERR_BAD_ARG;
  }
  s->tips_ok = true;
  invalidate_theta(s, ops, nops);
  st = s->desc.precision == GEMS_PREC_MIXED ? launch_theta_mixed(s, br, true, false, lnl)
                                            : launch_branch_lnl(s, br, lnl);
  if (st) return st;
  copy_pattern_lh(s, pattern_lh, *lnl);
  return GEMS_OK;
}

int gems_branch_derv(gems_session *s, const gems_op *ops, int nops, const gems_branch *br,
                     int compute_theta, double *df, double *ddf, double *df_frac) {
  if (!s || !df || !ddf || (nops > 0 && !ops)) return GEMS_ERR_BAD_ARG;
  GEMS_CUDA(cudaSetDevice(s->desc.device));
  int st = check_branch(s, br);
  if (st) return st;
  if (compute_theta) {
    if ((st = run_ops(s, ops, nops))) return st;
    st = s->desc.precision == GEMS_PREC_MIXED ? launch_theta_mixed(s, br, false, true, nullptr)
                                              : launch_theta(s, br);
    if (st) return st;
    s->theta_valid = true;
    s->theta_branch = *br;
  } else if (!s->theta_valid) {
    set_error("theta not computed");
    return GEMS_ERR_STATE;
  }
  if ((st = launch_derv(s, br->length, df, ddf))) return st;
  if (df_frac) {
    GEMS_CUDA(cudaMemcpyAsync(df_frac, s->d_df_frac, sizeof(double) * s->desc.nptn,
                              cudaMemcpyDeviceToHost, s->stream));
    GEMS_CUDA(cudaStreamSynchronize(s->stream));
  }
  return GEMS_OK;
}

int gems_lnl_from_buffer(gems_session *s, double length, double *lnl, double *pattern_lh) {
  if (!s || !lnl || !(length >= 0)) return GEMS_ERR_BAD_ARG;
  if (!s->theta_valid) {
    set_error("theta not computed");
    return GEMS_ERR_STATE;
  }
  GEMS_CUDA(cudaSetDevice(s->desc.device));
  int st = launch_from_buffer(s, length, lnl);
  if (st) return st;
  copy_pattern_lh(s, pattern_lh, *lnl);
  return GEMS_OK;
}

int gems_newton_branch_async(gems_session *s, const gems_op *ops, int nops,
                             const gems_branch *br, int compute_theta, double min_len,
                             double max_len, double xacc, int max_steps) {
  if (!s || (nops > 0 && !ops) || !(min_len >= 0) || !(max_len >= min_len) || max_steps < 1)
    return GEMS_ERR_BAD_ARG;
  GEMS_CUDA(cudaSetDevice(s->desc.device));
  int st = check_branch(s, br);
  if (st) return st;
  if (compute_theta) {
    if ((st = run_ops(s, ops, nops))) return st;
    st = s->desc.precision == GEMS_PREC_MIXED ? launch_theta_mixed(s, br, false, true, nullptr)
                                              : launch_theta(s, br);
    if (st) return st;
    s->theta_valid = true;
    s->theta_branch = *br;
  } else if (!s->theta_valid) {
    set_error("theta not computed");
    return GEMS_ERR_STATE;
  }
  return launch_newton_async(s, br->length, min_len, max_len, xacc, max_steps);
}

int gems_newton_branch_wait(gems_session *s, double *opt_len, int *nevals) {
  if (!s || !opt_len) return GEMS_ERR_BAD_ARG;
  GEMS_CUDA(cudaSetDevice(s->desc.device));
  int ne = 0;
  const int st = newton_result(s, opt_len, &ne);
  if (nevals) *nevals = ne;
  return st;
}

int gems_newton_branch(gems_session *s, const gems_op *ops, int nops, const gems_branch *br,
                       int compute_theta, double min_len, double max_len, double xacc,
                       int max_steps, double *opt_len, int *nevals) {
  if (!opt_len) return GEMS_ERR_BAD_ARG;
  int st = gems_newton_branch_async(s, ops, nops, br, compute_theta, min_len, max_len, xacc,
                                    max_steps);
  if (st) return st;
  return gems_newton_branch_wait(s, opt_len, nevals);
}

int gems_get_partial(gems_session *s, int slot, double *partial, uint16_t *scale) {
  if (!s || slot < 0 || slot >= s->desc.nslots) return GEMS_ERR_BAD_ARG;
  GEMS_CUDA(cudaSetDevice(s->desc.device));
  const size_t blk = s->block, n = (size_t)s->desc.nptn * blk;
  if (partial) {
    if (s->desc.precision == GEMS_PREC_FP64 && s->desc.nstates != 4) {
      const double *src = static_cast<const double *>(s->d_partials) + (size_t)slot * s->slot_elems;
      GEMS_CUDA(cudaMemcpyAsync(partial, src, n * sizeof(double), cudaMemcpyDeviceToHost,
                                s->stream));
    } else if (s->desc.precision == GEMS_PREC_FP64) {  // 4 states: tile-major rows
      std::vector<double> tmp(s->slot_elems);
      const double *src = static_cast<const double *>(s->d_partials) + (size_t)slot * s->slot_elems;
      GEMS_CUDA(cudaMemcpyAsync(tmp.data(), src, s->slot_elems * sizeof(double),
                                cudaMemcpyDeviceToHost, s->stream));
      GEMS_CUDA(cudaStreamSynchronize(s->stream));
      const DevCtx c = s->ctx();
      for (long p = 0; p < s->desc.nptn; p++)
        for (int cc = 0; cc < s->desc.ncat; cc++)
          for (int x = 0; x < 4; x++)
            partial[(size_t)p * blk + (size_t)cc * 4 + x] = tmp[f64_off<4>(c, p, cc, x)];
    } else {
      std::vector<float> tmp(s->slot_elems);
      const float *src = static_cast<const float *>(s->d_partials) + (size_t)slot * s->slot_elems;
      GEMS_CUDA(cudaMemcpyAsync(tmp.data(), src, s->slot_elems * sizeof(float),
                                cudaMemcpyDeviceToHost, s->stream));
      GEMS_CUDA(cudaStreamSynchronize(s->stream));
      const DevCtx c = s->ctx();
      const int nst = s->desc.nstates;
      for (long p = 0; p < s->desc.nptn; p++)
        for (int cc = 0; cc < s->desc.ncat; cc++) {
          for (int x = 0; x < nst; x++) {
            const size_t o =
                !s->tiled   ? (size_t)p * blk + (size_t)cc * nst + x
                : nst == 4  ? mix_off<4>(c, p, cc) + x
                : nst == 20 ? mix_off<20>(c, p, cc) + (size_t)(x / 4) * mix_cs<20>() + x % 4
                            : mix_off<61>(c, p, cc) + (size_t)(x / 4) * mix_cs<61>() + x % 4;
            partial[(size_t)p * blk + (size_t)cc * nst + x] = tmp[o];
          }
        }
    }
  }
  if (scale) {
    const size_t per = s->desc.scaling == GEMS_SCALE_SAFE ? s->desc.ncat : 1;
    GEMS_CUDA(cudaMemcpyAsync(scale, s->d_scale + (size_t)slot * s->P * per,
                              (size_t)s->desc.nptn * per * 2, cudaMemcpyDeviceToHost, s->stream));
  }
  GEMS_CUDA(cudaStreamSynchronize(s->stream));
  return GEMS_OK;
}

int gems_get_theta(gems_session *s, double *theta, double *scale_all) {
  if (!s) return GEMS_ERR_BAD_ARG;
  if (!s->theta_valid) return GEMS_ERR_STATE;
  if (theta)
    GEMS_CUDA(cudaMemcpyAsync(theta, s->d_theta, sizeof(double) * s->desc.nptn * s->block,
                              cudaMemcpyDeviceToHost, s->stream));
  if (scale_all)
    GEMS_CUDA(cudaMemcpyAsync(scale_all, s->d_scale_all, sizeof(double) * s->desc.nptn,
                              cudaMemcpyDeviceToHost, s->stream));
  GEMS_CUDA(cudaStreamSynchronize(s->stream));
  return GEMS_OK;
}

int gems_upload_reweightings(gems_session *s, const float *weights, int R) {
  if (!s || !weights || R < 1 || 2 * R > s->nred) return GEMS_ERR_BAD_ARG;
  GEMS_CUDA(cudaSetDevice(s->desc.device));
  if (s->d_rell_w && s->rell_R != R) {
    cudaFree(s->d_rell_w);
    s->d_rell_w = nullptr;
    s->d_rell_part = nullptr;
    s->rell_R = 0;
  }
  const size_t ld = (size_t)s->P;
  if (!s->d_rell_w) {
    // the counts (rows of P floats, P a multiple of 64: every row 256-byte aligned), then the
    // scratch of the tiled reductions
    const size_t wbytes = (size_t)R * ld * sizeof(float);
    const size_t bytes = wbytes + rell_scratch_doubles(R, s->P) * sizeof(double);
    size_t free_b = 0, total_b = 0;
    GEMS_CUDA(cudaMemGetInfo(&free_b, &total_b));
    if (bytes > free_b) {
      set_error("reweightings exceed free device memory");
      return GEMS_ERR_ADMISSION;
    }
    GEMS_CUDA(cudaMalloc((void **)&s->d_rell_w, bytes));
    GEMS_CUDA(cudaMemsetAsync(s->d_rell_w, 0, wbytes, s->stream));
    s->d_rell_part = reinterpret_cast<double *>(reinterpret_cast<char *>(s->d_rell_w) + wbytes);
  }
  s->rell_R = R;
  s->rell_ld = ld;
  GEMS_CUDA(cudaMemcpy2DAsync(s->d_rell_w, ld * sizeof(float), weights,
                              (size_t)s->desc.nptn * sizeof(float),
                              (size_t)s->desc.nptn * sizeof(float), R, cudaMemcpyHostToDevice,
                              s->stream));
  GEMS_CUDA(cudaStreamSynchronize(s->stream));
  return GEMS_OK;
}

int gems_reweighted_lnl(gems_session *s, double *lnl) {
  if (!s || !lnl) return GEMS_ERR_BAD_ARG;
  GEMS_CUDA(cudaSetDevice(s->desc.device));
  int st = launch_rell_lnl(s, s->d_red);
  if (st) return st;
  GEMS_CUDA(cudaMemcpyAsync(lnl, s->d_red, sizeof(double) * s->rell_R, cudaMemcpyDeviceToHost,
                            s->stream));
  GEMS_CUDA(cudaStreamSynchronize(s->stream));
  return GEMS_OK;
}

int gems_reweighted_derv(gems_session *s, double *df, double *ddf) {
  if (!s || !df || !ddf) return GEMS_ERR_BAD_ARG;
  GEMS_CUDA(cudaSetDevice(s->desc.device));
  int st = launch_rell_derv(s, s->d_red);
  if (st) return st;
  std::vector<double> tmp(2 * (size_t)s->rell_R);
  GEMS_CUDA(cudaMemcpyAsync(tmp.data(), s->d_red, sizeof(double) * tmp.size(),
                            cudaMemcpyDeviceToHost, s->stream));
  GEMS_CUDA(cudaStreamSynchronize(s->stream));
  for (int r = 0; r < s->rell_R; r++) {
    df[r] = tmp[2 * r];
    ddf[r] = tmp[2 * r + 1];
  }
  return GEMS_OK;
}

int gems_launch_count(gems_session *s, long long *count) {
  if (!s || !count) return GEMS_ERR_BAD_ARG;
  *count = s->launches;
  return GEMS_OK;
}

int gems_profile_enable(gems_session *s, int on) {
  if (!s) return GEMS_ERR_BAD_ARG;
  s->prof_on = on != 0;
  return GEMS_OK;
}

int gems_profile_read(gems_session *s, int kernel_id, double *total_ms, long long *launches) {
  if (!s || kernel_id < 0 || kernel_id >= Session::kProfKernels) return GEMS_ERR_BAD_ARG;
  GEMS_CUDA(cudaStreamSynchronize(s->stream));
  prof_collect(s);
  if (total_ms) *total_ms = s->prof_ms[kernel_id];
  if (launches) *launches = s->prof_n[kernel_id];
  s->prof_ms[kernel_id] = 0.0;
  s->prof_n[kernel_id] = 0;
  return GEMS_OK;
}

}  // extern "C"
