// kernels_mixed.cu -- mixed-precision form: FP32 real-space partials, FP64 everywhere else.
//
// Partials are stored as non-negative real-space vectors (FP32), pattern-major like the FP64
// form.  One node update per category c is
//      out[c] = (P_c(t_L) . L[c]) (*) (P_c(t_R) . R[c]),   P_c(t) = evec diag(exp(eval r_c t)) inv_evec
// with P built in FP64 and rounded once to FP32 (4n^2 flops instead of the eigen-space 6n^2;
// no cancellation since every term is >= 0).  Underflow is handled per pattern (NORM) or per
// (pattern, category) (SAFE): below 2^-64 the values are multiplied by 2^64 and a uint16
// counter is incremented; each count is worth 64*log(2) in the log-likelihood.
// The branch terms are FP64: both partials are lifted to the eigen basis in FP64
// (inv_evec . real), and theta / the log-likelihood reduction / the derivative sums / Newton
// reuse the FP64 kernels, so every accepted length is re-evaluated in FP64.
#include <climits>
#include <cmath>
#include <string>

#include "gems_internal.cuh"

namespace gems {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ float group_maxf(float v, int G) {
  for (int o = 1; o < G; o <<= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double group_sum(double v, int G) {
  for (int o = 1; o < G; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ int group_min(int v, int G) {
  for (int o = 1; o < G; o <<= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double (*sh)[32]) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < K; k++) {
    double x = v[k];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sh[k][w] = x;
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int k = 0; k < K; k++) {
      double x = lane < nw ? sh[k][lane] : 0.0;
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      v[k] = x;
    }
  }
  __syncthreads();
}

// P_c(t) for both children of every op (FP64 -> FP32), and tip tables P_c . indicator.
// opmats (as float): [op][side][C][n][n] then [op][side][unknown+1][C][n]; grid (nops, 2).
__global__ void k_prep_ops_mixed(DevCtx c, const DevOp *ops, float *opm, size_t stride_f) {
  extern __shared__ double ex[];  // [C][n] exp terms
  const int k = blockIdx.x, side = blockIdx.y;
  const DevOp op = ops[k];
  const int kind = side ? op.r_kind : op.l_kind;
  const double len = side ? op.r_len : op.l_len;
  const int n = c.n, C = c.C, nn = n * n;
  for (int idx = threadIdx.x; idx < C * n; idx += blockDim.x) {
    const int cc = idx / n, i = idx - cc * n;
    ex[idx] = exp(c.eval[i] * (c.rates[cc] * len));
  }
  __syncthreads();
  float *Pm = opm + (size_t)k * stride_f + (size_t)side * C * nn;
  for (int idx = threadIdx.x; idx < C * nn; idx += blockDim.x) {
    const int cc = idx / nn, r = idx - cc * nn, x = r / n, y = r - x * n;
    double acc = 0.0;
    for (int i = 0; i < n; i++) acc = fma(c.evec[x * n + i] * ex[cc * n + i], c.inv_evec[i * n + y], acc);
    Pm[idx] = (float)fmax(acc, 0.0);
  }
  if (kind != GEMS_CHILD_TIP) return;
  __syncthreads();
  float *leaf = opm + (size_t)k * stride_f + (size_t)2 * C * nn + (size_t)side * (c.unknown + 1) * c.block;
  const int rows = (c.unknown + 1) * c.block;
  for (int idx = threadIdx.x; idx < rows; idx += blockDim.x) {
    const int s = idx / c.block, r = idx - s * c.block, cc = r / n, x = r - cc * n;
    const double *ind = c.tip_real + (size_t)s * n;
    const float *prow = Pm + (size_t)cc * nn + (size_t)x * n;
    float acc = 0.f;
    for (int y = 0; y < n; y++) acc = fmaf(prow[y], (float)ind[y], acc);
    leaf[idx] = acc;
  }
}

// N states of one (pattern, category) row; cs = floats between 4-state chunks (mix_cs)
template <int N>
__device__ __forceinline__ void load_vecf(const float *__restrict__ src, float (&v)[N], int cs) {
  if constexpr (N % 4 == 0) {
#pragma unroll
    for (int i = 0; i < N / 4; i++) {
      float4 t = __ldcg(reinterpret_cast<const float4 *>(src + (size_t)i * cs));
      v[4 * i] = t.x;
      v[4 * i + 1] = t.y;
      v[4 * i + 2] = t.z;
      v[4 * i + 3] = t.w;
    }
  } else {
#pragma unroll
    for (int i = 0; i < N; i++) v[i] = __ldcg(src + (size_t)(i / 4) * cs + i % 4);
  }
}

template <int N>
__device__ __forceinline__ void store_vecf(float *__restrict__ dst, const float (&v)[N], int cs) {
  if constexpr (N % 4 == 0) {
#pragma unroll
    for (int i = 0; i < N / 4; i++)
      *reinterpret_cast<float4 *>(dst + (size_t)i * cs) =
          make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
  } else {
    // whole 4-state chunks; in the tile-major form the padding states are stored as zeros
    // (they meet zero rows of P in the tensor-core products)
#pragma unroll
    for (int i = 0; i < (N + 3) / 4; i++) {
      float4 w;
      w.x = v[4 * i];
      w.y = 4 * i + 1 < N ? v[4 * i + 1] : 0.f;
      w.z = 4 * i + 2 < N ? v[4 * i + 2] : 0.f;
      w.w = 4 * i + 3 < N ? v[4 * i + 3] : 0.f;
      if (mix_k<N>() > 0) {
        *reinterpret_cast<float4 *>(dst + (size_t)i * cs) = w;
      } else {
        dst[4 * i] = w.x;
        if (4 * i + 1 < N) dst[4 * i + 1] = w.y;
        if (4 * i + 2 < N) dst[4 * i + 2] = w.z;
        if (4 * i + 3 < N) dst[4 * i + 3] = w.w;
      }
    }
  }
}

template <int N, bool SAFE>
__device__ __forceinline__ void child_msg_f(const DevCtx &c, int kind, int id, const float *Pm,
                                            const float *leaf, long p, int gl, float (&v)[N],
                                            int &s) {
  if (kind == GEMS_CHILD_TIP) {
    const int st = c.tips[(size_t)id * c.P + p];
    const float *lt = leaf + (size_t)st * c.block + gl * N;
#pragma unroll
    for (int x = 0; x < N; x++) v[x] = __ldg(lt + x);
    s = 0;
  } else {
    const float *src = static_cast<const float *>(c.partials) + (size_t)id * c.slot_elems +
                       mix_off<N>(c, p, gl);
    float L[N];
    load_vecf<N>(src, L, mix_cs<N>());
    const float *pm = Pm + (size_t)gl * N * N;
#pragma unroll
    for (int x = 0; x < N; x++) {
      float acc = 0.f;
#pragma unroll
      for (int y = 0; y < N; y++) acc = fmaf(__ldg(pm + x * N + y), L[y], acc);
      v[x] = acc;
    }
    const uint16_t *sc = c.scale + (size_t)id * c.slot_scale;
    s = SAFE ? sc[(size_t)p * c.C + gl] : sc[p];
  }
}

template <int N, bool SAFE>
__global__ void __launch_bounds__(kThreads) k_traverse_mixed(DevCtx c, const DevOp *__restrict__ ops,
                                                             int nops, const float *__restrict__ opm,
                                                             size_t stride_f, int p0, int p1) {
  const int G = c.G;
  const int gl = threadIdx.x & (G - 1);
  const long p = p0 + ((long)blockIdx.x * blockDim.x + threadIdx.x) / G;
  const bool act = p < p1 && gl < c.C;
  const int C = c.C;
  const size_t nnC = (size_t)C * N * N;
  float *part = static_cast<float *>(c.partials);
  for (int k = 0; k < nops; k++) {
    const DevOp op = ops[k];
    const float *mats = opm + (size_t)k * stride_f;
    const bool tiptip = op.l_kind == GEMS_CHILD_TIP && op.r_kind == GEMS_CHILD_TIP;
    float out[N];
    float lh_max = 0.f;
    int sl = 0, sr = 0;
    if (act) {
      float vl[N], vr[N];
      child_msg_f<N, SAFE>(c, op.l_kind, op.l_id, mats, mats + 2 * nnC, p, gl, vl, sl);
      child_msg_f<N, SAFE>(c, op.r_kind, op.r_id, mats + nnC,
                           mats + 2 * nnC + (size_t)(c.unknown + 1) * c.block, p, gl, vr, sr);
#pragma unroll
      for (int x = 0; x < N; x++) {
        out[x] = vl[x] * vr[x];
        lh_max = fmaxf(lh_max, out[x]);
      }
    }
    if (!SAFE) lh_max = group_maxf(lh_max, G);
    int s_out = sl + sr;
    if (act) {
      if (!tiptip && lh_max < kScaleThrF && c.invar[p] == 0.0) {
#pragma unroll
        for (int x = 0; x < N; x++) out[x] *= 18446744073709551616.0f;  // 2^64
        s_out += 1;
      }
      store_vecf<N>(part + (size_t)op.dst_slot * c.slot_elems + mix_off<N>(c, p, gl), out, mix_cs<N>());
      uint16_t *sc = c.scale + (size_t)op.dst_slot * c.slot_scale;
      if (SAFE)
        sc[(size_t)p * C + gl] = (uint16_t)s_out;
      else if (gl == 0)
        sc[p] = (uint16_t)s_out;
    }
    __syncwarp();
  }
}

// eigen-basis FP64 lift of one category of a real FP32 partial (or of a tip indicator)
template <int N>
__device__ __forceinline__ void lift(const DevCtx &c, const float (&a)[N], double (&e)[N]) {
#pragma unroll 4
  for (int i = 0; i < N; i++) {
    double acc = 0.0;
#pragma unroll
    for (int x = 0; x < N; x++) acc = fma(__ldg(c.inv_evec + i * N + x), (double)a[x], acc);
    e[i] = acc;
  }
}

// theta (FP64, eigen basis) from FP32 real partials; also the branch lnL when want_lnl.
template <int N, bool SAFE>
__global__ void __launch_bounds__(kThreads) k_theta_mixed(DevCtx c, gems_branch br, int want_lnl,
                                                          int store_theta,
                                                          const double *__restrict__ val) {
  __shared__ double sh[2][32];
  const int G = c.G;
  const int gl = threadIdx.x & (G - 1);
  const long p = ((long)blockIdx.x * blockDim.x + threadIdx.x) / G;
  const bool act = p < c.P && gl < c.C;
  const float *part = static_cast<const float *>(c.partials);
  int ssum = 0;
  double th[N];
  if (act) {
    float a[N];
    load_vecf<N>(part + (size_t)br.dad_slot * c.slot_elems + mix_off<N>(c, p, gl), a, mix_cs<N>());
    double de[N];
    lift<N>(c, a, de);
    const uint16_t *sd = c.scale + (size_t)br.dad_slot * c.slot_scale;
    ssum = SAFE ? sd[(size_t)p * c.C + gl] : sd[p];
    if (br.node_kind == GEMS_CHILD_TIP) {
      const int st = c.tips[(size_t)br.node_id * c.P + p];
      const double *tp = c.tip + (size_t)st * N;
#pragma unroll
      for (int i = 0; i < N; i++) th[i] = __ldg(tp + i) * de[i];
    } else {
      float b[N];
      load_vecf<N>(part + (size_t)br.node_id * c.slot_elems + mix_off<N>(c, p, gl), b, mix_cs<N>());
      double ne[N];
      lift<N>(c, b, ne);
#pragma unroll
      for (int i = 0; i < N; i++) th[i] = ne[i] * de[i];
      const uint16_t *sn = c.scale + (size_t)br.node_id * c.slot_scale;
      ssum += SAFE ? sn[(size_t)p * c.C + gl] : sn[p];
    }
  }
  int ms = ssum;
  if (SAFE) {
    ms = group_min(act ? ssum : INT_MAX, G);
    if (act) {
      // a category one count above the minimum is 2^-64 smaller; two or more: negligible
      if (ssum == ms + 1) {
#pragma unroll
        for (int i = 0; i < N; i++) th[i] *= 5.421010862427522e-20;  // 2^-64
      } else if (ssum > ms + 1) {
#pragma unroll
        for (int i = 0; i < N; i++) th[i] = 0.0;
      }
    }
  }
  if (act && store_theta) {
    double *dst = c.theta + (size_t)p * c.block + gl * N;
#pragma unroll
    for (int i = 0; i < N; i++) dst[i] = th[i];
    if (gl == 0) c.scale_all[p] = (double)ms * kLogScaleThrF;
  }
  if (!want_lnl) return;
  double lh_cat = 0.0;
  if (act) {
#pragma unroll
    for (int i = 0; i < N; i++) lh_cat = fma(__ldg(val + gl * N + i), th[i], lh_cat);
  }
  const double lh_sum = group_sum(lh_cat, G);
  double v[2] = {0.0, 0.0};
  if (act && gl == 0) {
    const double lh = fabs(lh_sum) + c.invar[p];
    const double plh = log(lh) + ms * kLogScaleThrF;
    c.pattern_lh[p] = plh;
    if (p < c.nptn) {
      const double f = c.freq[p];
      v[0] = plh * f;
      v[1] = (isfinite(plh) ? plh : 4.0 * kLogScaleThr) * f;
    }
  }
  block_sum<2>(v, sh);
  if (threadIdx.x == 0) {
    c.red[2 * blockIdx.x] = v[0];
    c.red[2 * blockIdx.x + 1] = v[1];
  }
}

__global__ void k_val_table(DevCtx c, double len, double *val) {
  for (int idx = threadIdx.x; idx < c.block; idx += blockDim.x) {
    const int cc = idx / c.n, i = idx - cc * c.n;
    val[idx] = exp(c.eval[i] * (c.rates[cc] * len)) * c.props[cc];
  }
}

template <int K>
__global__ void k_reduce_final_m(const double *red, int nblk, double *out) {
  __shared__ double sh[K][32];
  double v[K];
#pragma unroll
  for (int k = 0; k < K; k++) v[k] = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < K; k++) v[k] += red[(size_t)K * b + k];
  block_sum<K>(v, sh);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < K; k++) out[k] = v[k];
}

inline int grid_for(const Session *s) {
  const long threads = (long)s->P * s->G;
  return (int)((threads + kThreads - 1) / kThreads);
}

}  // namespace

#define GEMS_DISPATCH_NM(n, NAME, ...)                                  \
  switch (n) {                                                          \
    case 4: { constexpr int NS = 4; __VA_ARGS__; } break;               \
    case 20: { constexpr int NS = 20; __VA_ARGS__; } break;             \
    case 61: { constexpr int NS = 61; __VA_ARGS__; } break;             \
    default: set_error(std::string(NAME) + ": unsupported state count"); \
      return GEMS_ERR_BAD_ARG;                                          \
  }

int launch_prep_ops_mixed(Session *s, int nops) {
  if (nops <= 0) return GEMS_OK;
  DevCtx c = s->ctx();
  const size_t smem = sizeof(double) * s->desc.ncat * s->desc.nstates;
  k_prep_ops_mixed<<<dim3(nops, 2), 256, smem, s->stream>>>(
      c, s->d_ops, reinterpret_cast<float *>(s->d_opmats), s->op_stride);
  s->launches++;
  GEMS_CUDA(cudaGetLastError());
  return GEMS_OK;
}

int launch_traverse_mixed(Session *s, int nops, int p0, int p1) {
  if (nops <= 0 || p1 <= p0) return GEMS_OK;
  DevCtx c = s->ctx();
  const int grid = (int)(((long)(p1 - p0) * s->G + kThreads - 1) / kThreads);
  const bool safe = s->desc.scaling == GEMS_SCALE_SAFE;
  const float *opm = reinterpret_cast<const float *>(s->d_opmats);
  cudaEvent_t ev0;
  if (int st = prof_begin(s, 0, &ev0)) return st;
  GEMS_DISPATCH_NM(s->desc.nstates, "traverse_mixed",
    if (safe) k_traverse_mixed<NS, true><<<grid, kThreads, 0, s->stream>>>(c, s->d_ops, nops, opm, s->op_stride, p0, p1);
    else k_traverse_mixed<NS, false><<<grid, kThreads, 0, s->stream>>>(c, s->d_ops, nops, opm, s->op_stride, p0, p1));
  s->launches++;
  GEMS_CUDA(cudaGetLastError());
  return prof_end(s, 0, ev0);
}

// theta (and optionally the branch lnL) from the two FP32 partials of br
int enqueue_theta_mixed(Session *s, const gems_branch *br, bool want_lnl, bool store_theta) {
  DevCtx c = s->ctx();
  const int grid = grid_for(s);
  const bool safe = s->desc.scaling == GEMS_SCALE_SAFE;
  double *val = s->d_branch;
  if (want_lnl) {
    k_val_table<<<1, 256, 0, s->stream>>>(c, br->length, val);
    s->launches++;
  }
  cudaEvent_t ev0;
  if (int st = prof_begin(s, want_lnl ? 1 : 2, &ev0)) return st;
  const int wl = want_lnl ? 1 : 0, stt = store_theta ? 1 : 0;
  GEMS_DISPATCH_NM(s->desc.nstates, "theta_mixed",
    if (safe) k_theta_mixed<NS, true><<<grid, kThreads, 0, s->stream>>>(c, *br, wl, stt, val);
    else k_theta_mixed<NS, false><<<grid, kThreads, 0, s->stream>>>(c, *br, wl, stt, val));
  s->launches++;
  GEMS_CUDA(cudaGetLastError());
  if (int st = prof_end(s, want_lnl ? 1 : 2, ev0)) return st;
  if (!want_lnl) return GEMS_OK;
  k_reduce_final_m<2><<<1, 256, 0, s->stream>>>(s->d_red, grid, s->d_result);
  s->launches++;
  GEMS_CUDA(cudaGetLastError());
  GEMS_CUDA(cudaMemcpyAsync(s->h_result, s->d_result, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                            s->stream));
  return GEMS_OK;
}

double theta_mixed_lnl(const Session *s) {
  return std::isfinite(s->h_result[0]) ? s->h_result[0] : s->h_result[1];
}

int launch_theta_mixed(Session *s, const gems_branch *br, bool want_lnl, bool store_theta,
                       double *lnl) {
  if (int st = enqueue_theta_mixed(s, br, want_lnl, store_theta)) return st;
  if (!want_lnl) return GEMS_OK;
  GEMS_CUDA(cudaStreamSynchronize(s->stream));
  *lnl = theta_mixed_lnl(s);
  return GEMS_OK;
}

}  // namespace gems
