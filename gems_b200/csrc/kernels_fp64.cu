// kernels_fp64.cu -- FP64 eigen-space likelihood kernels for sm_100a.
//
// Layout in HBM (per partial slot): pattern-major, then category, then state:
//   partial[p][c][x] at ((p * C) + c) * n + x, doubles.  One pattern's block of C*n values is
//   contiguous, so a group of G (= next pow2 >= C) adjacent lanes handles one pattern, lane c
//   owning category c: a warp covers 32/G consecutive patterns and reads/writes one
//   contiguous span (coalesced), and the per-pattern max / min / sums are warp shuffles.
//
// Arithmetic follows tree/phylokernelnew.h (reversible, non-site-specific kernel):
//   E_c(t)[x][i]   = evec[x][i] * exp(eval[i] * r_c * t)                          (:1043-1062)
//   tip table      = sum_i E_c[x][i] * tip[state][i], unknown row = 1                (:1064-1088)
//   partial        = inv_evec . ((E_L . L) * (E_R . R)) per category               (:1911-2035)
//   NORM scaling   : max |partial| over the pattern's block < 2^-256 and ptn_invar == 0
//                    -> ldexp(.,256), scale_num[p] += 1; tip-tip never scaled     (:2019-2034)
//   SAFE scaling   : the same per (pattern, category)                             (:1997-2013)
//   branch lnL     : sum_c sum_i val*node*dad, |.| + invar, log + scale*log(2^-256) (:2658-3275)
//   theta, derivatives and lnL-from-buffer                                         (:2053-2650,
//                                                                                    :3285-3495)
// Reductions over patterns are deterministic: per-CTA sums in a fixed tree, then one CTA sums
// the per-CTA values in index order.
#include <cooperative_groups.h>

#include <climits>
#include <algorithm>
#include <cmath>
#include <string>

#include "gems_internal.cuh"

namespace gems {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double group_max(double v, int G) {
  for (int o = 1; o < G; o <<= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
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

// Sum `v` over the CTA (fixed tree order); result valid in thread 0.
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

// ----------------------------------------------------------------------------------------
// Per-op transition tables (computePartialInfo): E_L, E_R and tip tables for tip children.
// grid = (nops, 2 sides)
// ----------------------------------------------------------------------------------------
__global__ void k_prep_ops(DevCtx c, const DevOp *ops, double *opmats, size_t stride) {
  const int k = blockIdx.x, side = blockIdx.y;
  const DevOp op = ops[k];
  const int kind = side ? op.r_kind : op.l_kind;
  const double len = side ? op.r_len : op.l_len;
  const int n = c.n, C = c.C, nn = n * n;
  double *E = opmats + (size_t)k * stride + (size_t)side * C * nn;
  for (int idx = threadIdx.x; idx < C * nn; idx += blockDim.x) {
    const int cc = idx / nn, r = idx - cc * nn, x = r / n, i = r - x * n;
    E[idx] = c.evec[x * n + i] * exp(c.eval[i] * (c.rates[cc] * len));
  }
  if (kind != GEMS_CHILD_TIP) return;
  __syncthreads();
  double *leaf = opmats + (size_t)k * stride + (size_t)2 * C * nn +
                 (size_t)side * (c.unknown + 1) * c.block;
  const int nrow = c.unknown * c.block;
  for (int idx = threadIdx.x; idx < nrow; idx += blockDim.x) {
    const int s = idx / c.block, r = idx - s * c.block;
    const double *e = E + (size_t)r * n;
    const double *t = c.tip + (size_t)s * n;
    double acc = 0.0;
    for (int i = 0; i < n; i++) acc = fma(e[i], t[i], acc);
    leaf[idx] = acc;
  }
  for (int idx = threadIdx.x; idx < c.block; idx += blockDim.x) leaf[nrow + idx] = 1.0;
}

template <int N>
__device__ __forceinline__ void load_vec(const double *__restrict__ src, double (&v)[N]) {
  if constexpr (N % 2 == 0) {
    const double2 *s2 = reinterpret_cast<const double2 *>(src);
#pragma unroll
    for (int i = 0; i < N / 2; i++) {
      double2 t = __ldcg(s2 + i);
      v[2 * i] = t.x;
      v[2 * i + 1] = t.y;
    }
  } else {
#pragma unroll
    for (int i = 0; i < N; i++) v[i] = __ldcg(src + i);
  }
}

template <int N>
__device__ __forceinline__ void store_vec(double *__restrict__ dst, const double (&v)[N]) {
  if constexpr (N % 2 == 0) {
    double2 *d2 = reinterpret_cast<double2 *>(dst);
#pragma unroll
    for (int i = 0; i < N / 2; i++) d2[i] = make_double2(v[2 * i], v[2 * i + 1]);
  } else {
#pragma unroll
    for (int i = 0; i < N; i++) dst[i] = v[i];
  }
}

// Real-space message from one child for category gl: E_c . child (internal) or the tip row.
template <int N, bool SAFE>
__device__ __forceinline__ void child_msg(const DevCtx &c, int kind, int id, const double *E,
                                          const double *leaf, long p, int gl, double (&v)[N],
                                          int &s) {
  if (kind == GEMS_CHILD_TIP) {
    const int st = c.tips[(size_t)id * c.P + p];
    const double *lt = leaf + (size_t)st * c.block + gl * N;
#pragma unroll
    for (int x = 0; x < N; x++) v[x] = __ldg(lt + x);
    s = 0;
  } else {
    const double *slot = static_cast<const double *>(c.partials) + (size_t)id * c.slot_elems;
    double L[N];
    load_row<N>(slot, c, p, gl, L);
    const double *e = E + (size_t)gl * N * N;
#pragma unroll
    for (int x = 0; x < N; x++) {
      double acc = 0.0;
#pragma unroll
      for (int i = 0; i < N; i++) acc = fma(__ldg(e + x * N + i), L[i], acc);
      v[x] = acc;
    }
    const uint16_t *sc = c.scale + (size_t)id * c.slot_scale;
    s = SAFE ? sc[(size_t)p * c.C + gl] : sc[p];
  }
}

// Whole traversal for the patterns [p0, p1) of this launch, p1 <= P: every op in postorder.
// A pattern is always handled by the same lane group, so children written by an earlier op are
// read back by the same warp (ordered by __syncwarp); no inter-CTA dependency exists.
template <int N, bool SAFE>
__global__ void __launch_bounds__(kThreads) k_traverse(DevCtx c, const DevOp *__restrict__ ops,
                                                       int nops, const double *__restrict__ opmats,
                                                       size_t stride, int p0, int p1) {
  const int G = c.G;
  const int gl = threadIdx.x & (G - 1);
  const long p = p0 + ((long)blockIdx.x * blockDim.x + threadIdx.x) / G;
  const bool act = p < p1 && gl < c.C;
  const int C = c.C;
  const size_t nnC = (size_t)C * N * N;
  double *part = static_cast<double *>(c.partials);
  for (int k = 0; k < nops; k++) {
    const DevOp op = ops[k];
    const double *mats = opmats + (size_t)k * stride;
    const bool tiptip = op.l_kind == GEMS_CHILD_TIP && op.r_kind == GEMS_CHILD_TIP;
    double out[N];
    double lh_max = 0.0;
    int sl = 0, sr = 0;
    if (act) {
      double tmp[N];
      {
        double vl[N];
        child_msg<N, SAFE>(c, op.l_kind, op.l_id, mats, mats + 2 * nnC, p, gl, vl, sl);
        double vr[N];
        child_msg<N, SAFE>(c, op.r_kind, op.r_id, mats + nnC,
                           mats + 2 * nnC + (size_t)(c.unknown + 1) * c.block, p, gl, vr, sr);
#pragma unroll
        for (int x = 0; x < N; x++) tmp[x] = vl[x] * vr[x];
      }
#pragma unroll
      for (int j = 0; j < N; j++) {
        double acc = 0.0;
#pragma unroll
        for (int x = 0; x < N; x++) acc = fma(__ldg(c.inv_evec + j * N + x), tmp[x], acc);
        out[j] = acc;
        lh_max = fmax(lh_max, fabs(acc));
      }
    }
    if (!SAFE) lh_max = group_max(lh_max, G);
    int s_out = sl + sr;
    if (act) {
      if (!tiptip && lh_max < kScaleThr && c.invar[p] == 0.0) {
#pragma unroll
        for (int j = 0; j < N; j++) out[j] = ldexp(out[j], kScaleExp);
        s_out += 1;
      }
      store_row<N>(part + (size_t)op.dst_slot * c.slot_elems, c, p, gl, out);
      uint16_t *sc = c.scale + (size_t)op.dst_slot * c.slot_scale;
      if (SAFE)
        sc[(size_t)p * C + gl] = (uint16_t)s_out;
      else if (gl == 0)
        sc[p] = (uint16_t)s_out;
    }
    __syncwarp();
  }
}

// ----------------------------------------------------------------------------------------
// Branch tables: val[c][i] = exp(eval_i * r_c * t) * prop_c, and for a tip node the table
// val (x) tip[state] (phylokernelnew.h:2731-2766, :2785-2818).
// ----------------------------------------------------------------------------------------
__global__ void k_prep_branch(DevCtx c, double len, int tip_node, double *bt) {
  const int n = c.n, blk = c.block;
  for (int idx = threadIdx.x; idx < blk; idx += blockDim.x) {
    const int cc = idx / n, i = idx - cc * n;
    bt[idx] = exp(c.eval[i] * (c.rates[cc] * len)) * c.props[cc];
  }
  if (!tip_node) return;
  __syncthreads();
  const int rows = (c.unknown + 1) * blk;
  for (int idx = threadIdx.x; idx < rows; idx += blockDim.x) {
    const int s = idx / blk, r = idx - s * blk, i = r % n;
    bt[blk + idx] = bt[r] * c.tip[(size_t)s * n + i];
  }
}

template <int N, bool SAFE>
__global__ void __launch_bounds__(kThreads) k_branch_lnl(DevCtx c, gems_branch br,
                                                         const double *__restrict__ bt) {
  __shared__ double sh[2][32];
  const int G = c.G;
  const int gl = threadIdx.x & (G - 1);
  const long p = ((long)blockIdx.x * blockDim.x + threadIdx.x) / G;
  const bool act = p < c.P && gl < c.C;
  const double *part = static_cast<const double *>(c.partials);
  double lh_cat = 0.0;
  int ssum = 0;
  if (act) {
    double dad[N];
    load_row<N>(part + (size_t)br.dad_slot * c.slot_elems, c, p, gl, dad);
    const uint16_t *sd = c.scale + (size_t)br.dad_slot * c.slot_scale;
    ssum = SAFE ? sd[(size_t)p * c.C + gl] : sd[p];
    if (br.node_kind == GEMS_CHILD_TIP) {
      const int st = c.tips[(size_t)br.node_id * c.P + p];
      const double *nt = bt + c.block + (size_t)st * c.block + gl * N;
#pragma unroll
      for (int i = 0; i < N; i++) lh_cat = fma(__ldg(nt + i), dad[i], lh_cat);
    } else {
      double nd[N];
      load_row<N>(part + (size_t)br.node_id * c.slot_elems, c, p, gl, nd);
      const double *val = bt + gl * N;
#pragma unroll
      for (int i = 0; i < N; i++) lh_cat = fma(__ldg(val + i) * nd[i], dad[i], lh_cat);
      const uint16_t *sn = c.scale + (size_t)br.node_id * c.slot_scale;
      ssum += SAFE ? sn[(size_t)p * c.C + gl] : sn[p];
    }
  }
  double min_scale = ssum;
  if (SAFE) {
    const int ms = group_min(act ? ssum : INT_MAX, G);
    if (act) {
      if (ssum == ms + 1)
        lh_cat *= kScaleThr;
      else if (ssum > ms + 1)
        lh_cat = 0.0;
    }
    min_scale = ms;
  }
  const double lh_sum = group_sum(lh_cat, G);
  double v[2] = {0.0, 0.0};
  if (act && gl == 0) {
    const double lh = fabs(lh_sum) + c.invar[p];
    const double plh = log(lh) + min_scale * kLogScaleThr;
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

// Sums K interleaved per-CTA values in index order (deterministic), one CTA.
template <int K>
__global__ void k_reduce_final(const double *red, int nblk, double *out) {
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

// theta = node (.) dad (or tip (.) dad), SAFE per-category pre-scaling, buffer_scale_all
template <int N, bool SAFE>
__global__ void __launch_bounds__(kThreads) k_theta(DevCtx c, gems_branch br) {
  const int G = c.G;
  const int gl = threadIdx.x & (G - 1);
  const long p = ((long)blockIdx.x * blockDim.x + threadIdx.x) / G;
  const bool act = p < c.P && gl < c.C;
  const double *part = static_cast<const double *>(c.partials);
  double th[N];
  int ssum = 0;
  if (act) {
    double dad[N];
    load_row<N>(part + (size_t)br.dad_slot * c.slot_elems, c, p, gl, dad);
    const uint16_t *sd = c.scale + (size_t)br.dad_slot * c.slot_scale;
    ssum = SAFE ? sd[(size_t)p * c.C + gl] : sd[p];
    if (br.node_kind == GEMS_CHILD_TIP) {
      const int st = c.tips[(size_t)br.node_id * c.P + p];
      const double *tp = c.tip + (size_t)st * N;
#pragma unroll
      for (int i = 0; i < N; i++) th[i] = __ldg(tp + i) * dad[i];
    } else {
      double nd[N];
      load_row<N>(part + (size_t)br.node_id * c.slot_elems, c, p, gl, nd);
#pragma unroll
      for (int i = 0; i < N; i++) th[i] = nd[i] * dad[i];
      const uint16_t *sn = c.scale + (size_t)br.node_id * c.slot_scale;
      ssum += SAFE ? sn[(size_t)p * c.C + gl] : sn[p];
    }
  }
  int ms = ssum;
  if (SAFE) {
    ms = group_min(act ? ssum : INT_MAX, G);
    if (act) {
      if (ssum == ms + 1) {
#pragma unroll
        for (int i = 0; i < N; i++) th[i] *= kScaleThr;
      } else if (ssum > ms + 1) {
#pragma unroll
        for (int i = 0; i < N; i++) th[i] = 0.0;
      }
    }
  }
  if (act) {
    store_vec<N>(c.theta + (size_t)p * c.block + gl * N, th);
    if (gl == 0) c.scale_all[p] = (double)ms * kLogScaleThr;
  }
}

// val0/val1/val2 tables for length t into shared memory
__device__ __forceinline__ void derv_tables(const DevCtx &c, double t, double *v0, double *v1,
                                            double *v2) {
  for (int idx = threadIdx.x; idx < c.block; idx += blockDim.x) {
    const int cc = idx / c.n, i = idx - cc * c.n;
    const double cof = c.eval[i] * c.rates[cc];
    const double val = exp(cof * t) * c.props[cc];
    const double val1 = cof * val;
    v0[idx] = val;
    v1[idx] = val1;
    v2[idx] = cof * val1;
  }
}

// Per-pattern derivative terms over patterns [p0, ...) with stride; returns this thread's
// contributions (nonzero on group leaders only).
template <int N>
__device__ __forceinline__ void derv_pattern(const DevCtx &c, long p, int gl, bool act,
                                             const double *v0, const double *v1,
                                             const double *v2, double &a, double &b,
                                             bool store_g) {
  double lh = 0.0, d1 = 0.0, d2 = 0.0;
  if (act) {
    double th[N];
    load_vec<N>(c.theta + (size_t)p * c.block + gl * N, th);
    const int o = gl * N;
#pragma unroll
    for (int i = 0; i < N; i++) {
      lh = fma(v0[o + i], th[i], lh);
      d1 = fma(v1[o + i], th[i], d1);
      d2 = fma(v2[o + i], th[i], d2);
    }
  }
  lh = group_sum(lh, c.G);
  d1 = group_sum(d1, c.G);
  d2 = group_sum(d2, c.G);
  if (act && gl == 0 && p < c.nptn) {
    const double l = fabs(lh) + c.invar[p];
    const double inv = 1.0 / l;
    const double dff = d1 * inv, ddff = d2 * inv;
    const double f = c.freq[p];
    const double t1 = dff * f, t2 = ddff * f;
    a += t1;
    b += fma(-t1, dff, t2);
    if (store_g) {
      c.df_frac[p] = dff;
      c.ddf_term[p] = fma(-dff, dff, ddff);
    }
  }
}

template <int N>
__global__ void __launch_bounds__(kThreads) k_derv(DevCtx c, double t) {
  extern __shared__ double dyn[];
  __shared__ double sh[2][32];
  double *v0 = dyn, *v1 = dyn + c.block, *v2 = dyn + 2 * c.block;
  derv_tables(c, t, v0, v1, v2);
  __syncthreads();
  const int G = c.G;
  const int gl = threadIdx.x & (G - 1);
  const long p = ((long)blockIdx.x * blockDim.x + threadIdx.x) / G;
  const bool act = p < c.P && gl < c.C;
  double v[2] = {0.0, 0.0};
  derv_pattern<N>(c, p, gl, act, v0, v1, v2, v[0], v[1], true);
  block_sum<2>(v, sh);
  if (threadIdx.x == 0) {
    c.red[2 * blockIdx.x] = v[0];
    c.red[2 * blockIdx.x + 1] = v[1];
  }
}

template <int N>
__global__ void __launch_bounds__(kThreads) k_from_buffer(DevCtx c, double t) {
  extern __shared__ double dyn[];
  __shared__ double sh[2][32];
  double *v0 = dyn;
  for (int idx = threadIdx.x; idx < c.block; idx += blockDim.x) {
    const int cc = idx / c.n, i = idx - cc * c.n;
    v0[idx] = exp(c.eval[i] * c.rates[cc] * t) * c.props[cc];
  }
  __syncthreads();
  const int G = c.G;
  const int gl = threadIdx.x & (G - 1);
  const long p = ((long)blockIdx.x * blockDim.x + threadIdx.x) / G;
  const bool act = p < c.P && gl < c.C;
  double lh = 0.0;
  if (act) {
    double th[N];
    load_vec<N>(c.theta + (size_t)p * c.block + gl * N, th);
#pragma unroll
    for (int i = 0; i < N; i++) lh = fma(v0[gl * N + i], th[i], lh);
  }
  lh = group_sum(lh, G);
  double v[2] = {0.0, 0.0};
  if (act && gl == 0) {
    const double l = fabs(lh) + c.invar[p];
    const double plh = log(fabs(l)) + c.scale_all[p];
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

// ----------------------------------------------------------------------------------------
// Device-side Newton (Optimization::minimizeNewton, utils/optimization.cpp:422-499) as one
// cooperative kernel: each evaluation is a grid-wide reduction of (df, ddf) over theta,
// separated by a bounded grid barrier; every CTA then sums the per-CTA values in the same
// order and runs the same scalar update, so all CTAs follow one iterate sequence.
// ----------------------------------------------------------------------------------------
constexpr unsigned long long kBarrierSpins = 1ull << 24;

__device__ bool grid_barrier(unsigned int *bar, unsigned int nblk, int *flag) {
  __shared__ int ok_sh;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    volatile unsigned int *vgen = bar + 1;
    const unsigned int gen = *vgen;
    __threadfence();
    const unsigned int arrived = atomicAdd(bar, 1u);
    if (arrived == nblk - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      unsigned long long spins = 0;
      while (*vgen == gen) {
        if (++spins > kBarrierSpins) {
          ok = 0;
          atomicExch(flag, GEMS_ERR_TIMEOUT);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    ok_sh = ok;
  }
  __syncthreads();
  return ok_sh != 0;
}

// The barrier's time-out path on purpose: the grid waits for one more block than it has, so
// every block gives up after kBarrierSpins (about a second) and the flag reads GEMS_ERR_TIMEOUT.
__global__ void k_barrier_probe(unsigned int *bar, int *flag) {
  if (grid_barrier(bar, gridDim.x + 1, flag) && threadIdx.x == 0) atomicExch(flag, GEMS_OK);
}

template <int N>
__global__ void __launch_bounds__(kThreads) k_newton(DevCtx c, double guess, double x1, double x2,
                                                     double xacc, int maxstep,
                                                     unsigned int *bar, int *flag,
                                                     double *result) {
  extern __shared__ double dyn[];
  __shared__ double sh[2][32];
  __shared__ double tot[2];
  double *v0 = dyn, *v1 = dyn + c.block, *v2 = dyn + 2 * c.block;
  const int G = c.G;
  const int gl = threadIdx.x & (G - 1);
  const long groups_per_grid = (long)gridDim.x * blockDim.x / G;
  const long p0 = ((long)blockIdx.x * blockDim.x + threadIdx.x) / G;
  const unsigned int nblk = gridDim.x;
  int nevals = 0, parity = 0;

  // evaluates f = -dlnL/dt and df = -d2lnL/dt2 at t (computeFuncDerv, phylotree.cpp:2555)
  auto eval = [&](double t, double &f, double &df) -> bool {
    __syncthreads();
    derv_tables(c, t, v0, v1, v2);
    __syncthreads();
    double v[2] = {0.0, 0.0};
    for (long p = p0; p < c.P; p += groups_per_grid) {
      const bool act = gl < c.C;
      derv_pattern<N>(c, p, gl, act, v0, v1, v2, v[0], v[1], false);
    }
    block_sum<2>(v, sh);
    double *red = c.red + (size_t)parity * 2 * nblk;
    if (threadIdx.x == 0) {
      red[2 * blockIdx.x] = v[0];
      red[2 * blockIdx.x + 1] = v[1];
    }
    if (!grid_barrier(bar, nblk, flag)) return false;
    double s[2] = {0.0, 0.0};
    for (unsigned int b = threadIdx.x; b < nblk; b += blockDim.x) {
      s[0] += __ldcg(red + 2 * b);
      s[1] += __ldcg(red + 2 * b + 1);
    }
    block_sum<2>(s, sh);
    if (threadIdx.x == 0) {
      tot[0] = s[0];
      tot[1] = s[1];
    }
    __syncthreads();
    double all_df = tot[0], all_ddf = tot[1];
    if (!isfinite(all_df)) all_df = all_ddf = 0.0;
    f = -all_df;
    df = -all_ddf;
    parity ^= 1;
    nevals++;
    return true;
  };

  double f, df, dx, temp, xh, xl, rts, rts_old;
  double ret = 0.0;
  int status = GEMS_OK;
  rts = guess;
  if (rts < x1) rts = x1;
  if (rts > x2) rts = x2;
  do {
    if (!eval(rts, f, df)) { status = GEMS_ERR_TIMEOUT; ret = rts; break; }
    if (!isfinite(f) || !isfinite(df)) { status = GEMS_ERR_NUMERIC_UNDERFLOW; ret = rts; break; }
    if (df >= 0.0 && fabs(f) < xacc) { ret = rts; break; }
    if (f < 0.0) { xl = rts; xh = x2; } else { xh = rts; xl = x1; }
    dx = fabs(xh - xl);
    bool done = false;
    for (int j = 1; j <= maxstep && !done; j++) {
      rts_old = rts;
      if ((df <= 0.0) || (((rts - xh) * df - f) * ((rts - xl) * df - f) >= 0.0)) {
        dx = 0.5 * (xh - xl);
        rts = xl + dx;
        if (xl == rts) { ret = rts; done = true; break; }
      } else {
        dx = f / df;
        temp = rts;
        rts -= dx;
        if (temp == rts) { ret = rts; done = true; break; }
      }
      if (fabs(dx) < xacc || (j == maxstep)) { ret = rts_old; done = true; break; }
      if (!eval(rts, f, df)) { status = GEMS_ERR_TIMEOUT; ret = rts; done = true; break; }
      if (!isfinite(f) || !isfinite(df)) {
        status = GEMS_ERR_NUMERIC_UNDERFLOW; ret = rts; done = true; break;
      }
      if (df > 0.0 && fabs(f) < xacc) { ret = rts; done = true; break; }
      if (f < 0.0) xl = rts;
      else if (f > 0.0) xh = rts;
    }
    if (!done) ret = 0.0;
  } while (false);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    result[0] = ret;
    result[1] = (double)nevals;
    result[2] = (double)status;
  }
}

// unpack a FP64 slot (identity copy; layout is already pattern-major)

inline int grid_for(const Session *s) {
  const long groups = s->P;
  const long threads = groups * s->G;
  return (int)((threads + kThreads - 1) / kThreads);
}

}  // namespace

// ---- dispatch helpers over the state count -----------------------------------------------
#define GEMS_DISPATCH_N(n, NAME, ...)                                  \
  switch (n) {                                                         \
    case 4: { constexpr int NS = 4; __VA_ARGS__; } break;              \
    case 20: { constexpr int NS = 20; __VA_ARGS__; } break;            \
    case 61: { constexpr int NS = 61; __VA_ARGS__; } break;            \
    default: set_error(std::string(NAME) + ": unsupported state count"); \
      return GEMS_ERR_BAD_ARG;                                         \
  }

int launch_prep_ops(Session *s, int nops) {
  if (nops <= 0) return GEMS_OK;
  DevCtx c = s->ctx();
  k_prep_ops<<<dim3(nops, 2), 256, 0, s->stream>>>(c, s->d_ops, s->d_opmats, s->op_stride);
  s->launches++;
  GEMS_CUDA(cudaGetLastError());
  return GEMS_OK;
}

int launch_traverse(Session *s, int nops, int p0, int p1) {
  if (nops <= 0 || p1 <= p0) return GEMS_OK;
  DevCtx c = s->ctx();
  const int grid = (int)(((long)(p1 - p0) * s->G + kThreads - 1) / kThreads);
  const bool safe = s->desc.scaling == GEMS_SCALE_SAFE;
  cudaEvent_t ev0;
  if (int st = prof_begin(s, 0, &ev0)) return st;
  GEMS_DISPATCH_N(s->desc.nstates, "traverse",
    if (safe) k_traverse<NS, true><<<grid, kThreads, 0, s->stream>>>(c, s->d_ops, nops, s->d_opmats, s->op_stride, p0, p1);
    else k_traverse<NS, false><<<grid, kThreads, 0, s->stream>>>(c, s->d_ops, nops, s->d_opmats, s->op_stride, p0, p1));
  s->launches++;
  GEMS_CUDA(cudaGetLastError());
  return prof_end(s, 0, ev0);
}

static int finish_pair(Session *s, int nblk, double *out_main, bool fixup_lnl) {
  k_reduce_final<2><<<1, 256, 0, s->stream>>>(s->d_red, nblk, s->d_result);
  s->launches++;
  GEMS_CUDA(cudaGetLastError());
  GEMS_CUDA(cudaMemcpyAsync(s->h_result, s->d_result, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                            s->stream));
  GEMS_CUDA(cudaStreamSynchronize(s->stream));
  if (fixup_lnl) {
    // non-finite total: clamp non-finite pattern values to 4*log(2^-256)
    // (phylokernelnew.h:3168-3184)
    out_main[0] = std::isfinite(s->h_result[0]) ? s->h_result[0] : s->h_result[1];
  } else {
    out_main[0] = s->h_result[0];
    out_main[1] = s->h_result[1];
  }
  return GEMS_OK;
}

int launch_branch_lnl(Session *s, const gems_branch *br, double *lnl) {
  DevCtx c = s->ctx();
  const int tip = br->node_kind == GEMS_CHILD_TIP;
  k_prep_branch<<<1, 256, 0, s->stream>>>(c, br->length, tip, s->d_branch);
  s->launches++;
  const int grid = grid_for(s);
  const bool safe = s->desc.scaling == GEMS_SCALE_SAFE;
  cudaEvent_t ev0;
  if (int st = prof_begin(s, 1, &ev0)) return st;
  GEMS_DISPATCH_N(s->desc.nstates, "branch_lnl",
    if (safe) k_branch_lnl<NS, true><<<grid, kThreads, 0, s->stream>>>(c, *br, s->d_branch);
    else k_branch_lnl<NS, false><<<grid, kThreads, 0, s->stream>>>(c, *br, s->d_branch));
  s->launches++;
  GEMS_CUDA(cudaGetLastError());
  if (int st = prof_end(s, 1, ev0)) return st;
  return finish_pair(s, grid, lnl, true);
}

int launch_theta(Session *s, const gems_branch *br) {
  DevCtx c = s->ctx();
  const int grid = grid_for(s);
  const bool safe = s->desc.scaling == GEMS_SCALE_SAFE;
  cudaEvent_t ev0;
  if (int st = prof_begin(s, 2, &ev0)) return st;
  GEMS_DISPATCH_N(s->desc.nstates, "theta",
    if (safe) k_theta<NS, true><<<grid, kThreads, 0, s->stream>>>(c, *br);
    else k_theta<NS, false><<<grid, kThreads, 0, s->stream>>>(c, *br));
  s->launches++;
  GEMS_CUDA(cudaGetLastError());
  return prof_end(s, 2, ev0);
}

int launch_derv(Session *s, double length, double *df, double *ddf) {
  DevCtx c = s->ctx();
  const int grid = grid_for(s);
  const size_t smem = 3 * sizeof(double) * s->block;
  cudaEvent_t ev0;
  if (int st = prof_begin(s, 3, &ev0)) return st;
  GEMS_DISPATCH_N(s->desc.nstates, "derv",
    k_derv<NS><<<grid, kThreads, smem, s->stream>>>(c, length));
  s->launches++;
  GEMS_CUDA(cudaGetLastError());
  if (int st = prof_end(s, 3, ev0)) return st;
  double out[2];
  int st = finish_pair(s, grid, out, false);
  if (st) return st;
  *df = out[0];
  *ddf = out[1];
  if (!std::isfinite(*df)) *df = *ddf = 0.0;  // phylokernelnew.h:2646-2649
  return GEMS_OK;
}

int launch_from_buffer(Session *s, double length, double *lnl) {
  DevCtx c = s->ctx();
  const int grid = grid_for(s);
  const size_t smem = sizeof(double) * s->block;
  cudaEvent_t ev0;
  if (int st = prof_begin(s, 4, &ev0)) return st;
  GEMS_DISPATCH_N(s->desc.nstates, "from_buffer",
    k_from_buffer<NS><<<grid, kThreads, smem, s->stream>>>(c, length));
  s->launches++;
  GEMS_CUDA(cudaGetLastError());
  if (int st = prof_end(s, 4, ev0)) return st;
  return finish_pair(s, grid, lnl, true);
}

int launch_newton(Session *s, double guess, double min_len, double max_len, double xacc,
                  int max_steps, double *opt_len, int *nevals) {
  if (int st = launch_newton_async(s, guess, min_len, max_len, xacc, max_steps)) return st;
  return newton_result(s, opt_len, nevals);
}

int newton_result(Session *s, double *opt_len, int *nevals) {
  GEMS_CUDA(cudaStreamSynchronize(s->stream));
  *opt_len = s->h_result[0];
  *nevals = (int)s->h_result[1];
  return (int)s->h_result[2];
}

int launch_newton_async(Session *s, double guess, double min_len, double max_len, double xacc,
                        int max_steps) {
  DevCtx c = s->ctx();
  const size_t smem = 3 * sizeof(double) * s->block;
  int dev = s->desc.device, nsm = 0, per_sm = 0;
  GEMS_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  void *fn = nullptr;
  GEMS_DISPATCH_N(s->desc.nstates, "newton", fn = (void *)k_newton<NS>);
  GEMS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kThreads, smem));
  if (per_sm < 1) {
    set_error("newton: kernel does not fit on an SM");
    return GEMS_ERR_CUDA;
  }
  long want = grid_for(s);
  long maxg = std::max(1L, (long)nsm * per_sm / s->newton_share);
  int grid = (int)(want < maxg ? want : maxg);
  if (grid < 1) grid = 1;
  if (2 * 2 * grid > s->nred) {
    set_error("newton: reduction buffer too small");
    return GEMS_ERR_STATE;
  }
  GEMS_CUDA(cudaMemsetAsync(s->d_bar, 0, 2 * sizeof(unsigned int), s->stream));
  GEMS_CUDA(cudaMemsetAsync(s->d_flag, 0, sizeof(int), s->stream));
  unsigned int *bar = s->d_bar;
  int *flag = s->d_flag;
  double *res = s->d_result;
  void *args[] = {&c, &guess, &min_len, &max_len, &xacc, &max_steps, &bar, &flag, &res};
  cudaEvent_t ev0;
  if (int st = prof_begin(s, 5, &ev0)) return st;
  GEMS_CUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kThreads), args, smem, s->stream));
  s->launches++;
  if (int st = prof_end(s, 5, ev0)) return st;
  GEMS_CUDA(cudaMemcpyAsync(s->h_result, s->d_result, 3 * sizeof(double), cudaMemcpyDeviceToHost,
                            s->stream));
  return GEMS_OK;
}

int check_barrier_timeout(int device, int *status) {
  GEMS_CUDA(cudaSetDevice(device));
  unsigned int *bar = nullptr;
  int *flag = nullptr;
  GEMS_CUDA(cudaMalloc((void **)&bar, 2 * sizeof(unsigned int)));
  cudaError_t e = cudaMalloc((void **)&flag, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(bar, 0, 2 * sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMemset(flag, 0, sizeof(int));
  if (e == cudaSuccess) {
    void *args[] = {&bar, &flag};
    e = cudaLaunchCooperativeKernel((void *)k_barrier_probe, dim3(2), dim3(32), args, 0, nullptr);
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  int h = -1;
  if (e == cudaSuccess) e = cudaMemcpy(&h, flag, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(bar);
  cudaFree(flag);
  if (e != cudaSuccess) return cuda_status(e, "barrier probe");
  *status = h;
  return GEMS_OK;
}


}  // namespace gems
