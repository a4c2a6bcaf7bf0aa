// kernels_traverse.cu -- whole-traversal kernels for 4- and 20-state models (FP64 and mixed).
//
// One CTA owns a tile of patterns and runs every node update of the traversal over it, in
// postorder; a pattern stays with one lane group for all ops, so a child written by an earlier
// op is read back by the same warp (L2-resident in practice: the DRAM traffic of a traversal is
// dominated by the partial writes).  Lane c of a group owns rate category c.
//
// FP64 form.  The reference precomputes E_c = evec . diag(exp(eval r_c t)) per child
// (phylokernelnew.h:1043-1062) and applies it with a dense n x n product per category.  Here
// the product is factored as
//      E_c . L = evec . (d_c (*) L),        d_c[i] = exp(eval_i r_c t)
// evec and inv_evec do not depend on the category or the op: they travel as kernel parameters,
// so every lane of a warp reads the same element (uniform operand, no per-lane load), and an
// op only loads its 2 x n exponential factors, stored category-fastest so the lanes of a
// group read one 32-byte sector.  Tip children use the table sum_i E_c[x][i] tip[s][i]
// (stored [s][x][c]).  The FP64 values agree with the reference form to rounding.
//
// Mixed form (FP32 real space): the transition matrices P_c(t) are op-dependent; they are
// stored [x][c][y], so lane c reads its row x of P_c as contiguous float4s.
#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <mutex>
#include <string>

#include "gems_internal.cuh"

namespace gems {

namespace {

constexpr int kThreads = 256;
constexpr int kOpChunk = 256;  // op descriptors staged in shared memory per pass
static_assert((kOpChunk & (kOpChunk - 1)) == 0, "kOpChunk is a power of two");

template <int N>
struct EigPack {
  double evec[N * N];
  double inv[N * N];
};

__device__ __forceinline__ double group_max(double v, int G) {
  for (int o = 1; o < G; o <<= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float group_maxf(float v, int G) {
  for (int o = 1; o < G; o <<= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Op descriptors of a traversal loop, staged kOpChunk at a time in shared memory as
// {dst, l_id, r_id, l_kind | r_kind << 8}: each op starts with a shared-memory read instead of a
// dependent global load (measured on the 512-taxon DNA traversal: 10% faster mixed, 5% FP64).
// Every thread of the block calls stage_ops at the same op index.
struct OpIds {
  int dst_slot, l_kind, l_id, r_kind, r_id;
};
__device__ __forceinline__ void stage_ops(const DevOp *ops, int k0, int nops, int4 *s_ops) {
  const int nk = min(kOpChunk, nops - k0);
  __syncthreads();  // the previous chunk is no longer read
  for (int i = threadIdx.x; i < nk; i += blockDim.x) {
    const DevOp o = ops[k0 + i];
    s_ops[i] = make_int4(o.dst_slot, o.l_id, o.r_id, o.l_kind | (o.r_kind << 8));
  }
  __syncthreads();
}
__device__ __forceinline__ OpIds staged_op(const int4 *s_ops, int j) {
  const int4 v = s_ops[j];
  return {v.x, v.w & 0xff, v.y, v.w >> 8, v.z};
}

// ---------------------------------------------------------------------------------------
// FP64 op tables: d[side][i][c] = exp(eval_i r_c t_side); tip tables leaf[side][s][x][c]
// table layout per op (doubles): [2][N][C] then [2][U1][N][C]
// ---------------------------------------------------------------------------------------
__global__ void k_prep_ops_f64(DevCtx c, const DevOp *ops, double *tab, size_t stride) {
  extern __shared__ double dsh[];  // [N][C]
  const int k = blockIdx.x, side = blockIdx.y;
  const DevOp op = ops[k];
  const int kind = side ? op.r_kind : op.l_kind;
  const double len = side ? op.r_len : op.l_len;
  const int n = c.n, C = c.C, blk = c.block;
  double *d = tab + (size_t)k * stride + (size_t)side * blk;
  for (int idx = threadIdx.x; idx < blk; idx += blockDim.x) {
    const int i = idx / C, cc = idx - i * C;
    const double v = exp(c.eval[i] * (c.rates[cc] * len));
    d[idx] = v;
    dsh[idx] = v;
  }
  if (kind != GEMS_CHILD_TIP) return;
  __syncthreads();
  double *leaf = tab + (size_t)k * stride + (size_t)2 * blk + (size_t)side * (c.unknown + 1) * blk;
  const int rows = c.unknown * blk;
  for (int idx = threadIdx.x; idx < rows; idx += blockDim.x) {
    const int s = idx / blk, r = idx - s * blk, x = r / C, cc = r - x * C;
    const double *t = c.tip + (size_t)s * n;
    double acc = 0.0;
    for (int i = 0; i < n; i++) acc = fma(c.evec[x * n + i] * dsh[i * C + cc], t[i], acc);
    leaf[idx] = acc;
  }
  for (int idx = threadIdx.x; idx < blk; idx += blockDim.x) leaf[rows + idx] = 1.0;
}

template <int N, bool SAFE>
__device__ __forceinline__ void msg_f64(const DevCtx &c, const EigPack<N> &E, int kind, int id,
                                        const double *__restrict__ d,
                                        const double *__restrict__ leaf, long p, int gl,
                                        double (&v)[N], int &s) {
  const int C = c.C;
  if (kind == GEMS_CHILD_TIP) {
    const int st = min((int)c.tips[(size_t)id * c.P + p], c.unknown);
    const double *lt = leaf + (size_t)st * c.block + gl;
#pragma unroll
    for (int x = 0; x < N; x++) v[x] = __ldg(lt + x * C);
    s = 0;
  } else {
    double L[N];
    load_row<N>(static_cast<const double *>(c.partials) + (size_t)id * c.slot_elems, c, p, gl, L);
#pragma unroll
    for (int i = 0; i < N; i++) L[i] *= __ldg(d + i * C + gl);
#pragma unroll
    for (int x = 0; x < N; x++) {
      double acc = 0.0;
#pragma unroll
      for (int i = 0; i < N; i++) acc = fma(E.evec[x * N + i], L[i], acc);
      v[x] = acc;
    }
    const uint16_t *sc = c.scale + (size_t)id * c.slot_scale;
    s = SAFE ? sc[(size_t)p * C + gl] : sc[p];
  }
}

template <int N, bool SAFE>
__global__ void __launch_bounds__(kThreads) k_traverse_f64(DevCtx c, const DevOp *__restrict__ ops,
                                                           int nops,
                                                           const double *__restrict__ tab,
                                                           size_t stride, const EigPack<N> E,
                                                           int p0, int p1) {
  const int G = c.G;
  const int gl = threadIdx.x & (G - 1);
  const long p = p0 + ((long)blockIdx.x * blockDim.x + threadIdx.x) / G;
  const bool act = p < p1 && gl < c.C;
  const int C = c.C, blk = c.block;
  double *part = static_cast<double *>(c.partials);
  __shared__ int4 s_ops[kOpChunk];
  for (int k = 0; k < nops; k++) {
    if ((k & (kOpChunk - 1)) == 0) stage_ops(ops, k, nops, s_ops);
    const OpIds op = staged_op(s_ops, k & (kOpChunk - 1));
    const double *tk = tab + (size_t)k * stride;
    const bool tiptip = op.l_kind == GEMS_CHILD_TIP && op.r_kind == GEMS_CHILD_TIP;
    double out[N];
    double lh_max = 0.0;
    int sl = 0, sr = 0;
    if (act) {
      double tmp[N];
      {
        double vl[N], vr[N];
        msg_f64<N, SAFE>(c, E, op.l_kind, op.l_id, tk, tk + 2 * blk, p, gl, vl, sl);
        msg_f64<N, SAFE>(c, E, op.r_kind, op.r_id, tk + blk,
                         tk + 2 * blk + (size_t)(c.unknown + 1) * blk, p, gl, vr, sr);
#pragma unroll
        for (int x = 0; x < N; x++) tmp[x] = vl[x] * vr[x];
      }
#pragma unroll
      for (int j = 0; j < N; j++) {
        double acc = 0.0;
#pragma unroll
        for (int x = 0; x < N; x++) acc = fma(E.inv[j * N + x], tmp[x], acc);
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

// FP64, 4 states: PP patterns per lane group at B blocks per SM (as k_traverse_mix4), same
// arithmetic in the same order as msg_f64 / k_traverse_f64, so every (PP, B) gives the same
// values.  Measured on the 512-taxon, 1M-pattern case: one pattern per group (40 registers)
// 23.6 ms; two at 4 blocks per SM 22.5 ms, at 3 or 5 blocks 23.7 / 24.5 ms; three at 3 blocks
// 22.4 ms; four at 2 blocks 24.7 ms.  The variant in use is picked by the tuner below.
template <bool SAFE, int PP>
__device__ __forceinline__ void msg_f64_4(const DevCtx &c, const EigPack<4> &E, int kind, int id,
                                          const double *__restrict__ d,
                                          const double *__restrict__ leaf,
                                          const long (&p)[PP], int gq,
                                          double (&v)[PP][4], int (&s)[PP]) {
  const int C = c.C;
  if (kind == GEMS_CHILD_TIP) {
    int st[PP];
#pragma unroll
    for (int u = 0; u < PP; u++) st[u] = min((int)c.tips[(size_t)id * c.P + p[u]], c.unknown);
#pragma unroll
    for (int u = 0; u < PP; u++) {
      const double *lt = leaf + (size_t)st[u] * c.block + gq;
#pragma unroll
      for (int x = 0; x < 4; x++) v[u][x] = __ldg(lt + x * C);
      s[u] = 0;
    }
  } else {
    const double *base = static_cast<const double *>(c.partials) + (size_t)id * c.slot_elems;
    double L[PP][4];
#pragma unroll
    for (int u = 0; u < PP; u++) load_row<4>(base, c, p[u], gq, L[u]);
    const uint16_t *sc = c.scale + (size_t)id * c.slot_scale;
#pragma unroll
    for (int u = 0; u < PP; u++) s[u] = SAFE ? sc[(size_t)p[u] * C + gq] : sc[p[u]];
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const double di = __ldg(d + i * C + gq);
#pragma unroll
      for (int u = 0; u < PP; u++) L[u][i] *= di;
    }
#pragma unroll
    for (int u = 0; u < PP; u++)
#pragma unroll
      for (int x = 0; x < 4; x++) {
        double acc = 0.0;
#pragma unroll
        for (int i = 0; i < 4; i++) acc = fma(E.evec[x * 4 + i], L[u][i], acc);
        v[u][x] = acc;
      }
  }
}

template <bool SAFE, int PP, int B>
__global__ void __launch_bounds__(kThreads, B)
    k_traverse_f64x(DevCtx c, const DevOp *__restrict__ ops, int nops,
                    const double *__restrict__ tab, size_t stride, const EigPack<4> E, int p0,
                    int p1) {
  const int G = c.G, C = c.C, blk = c.block;
  const int gl = threadIdx.x & (G - 1);
  const int gq = gl < C ? gl : 0;  // loads of idle lanes stay inside the tables
  const int per = kThreads / G;
  const long pb = p0 + (long)blockIdx.x * per * PP + threadIdx.x / G;
  long p[PP];
  bool act[PP];
#pragma unroll
  for (int u = 0; u < PP; u++) {
    const long q = pb + (long)u * per;
    act[u] = q < p1 && gl < C;
    p[u] = q < p1 ? q : p0;
  }
  double *part = static_cast<double *>(c.partials);
  __shared__ int4 s_ops[kOpChunk];
  for (int k = 0; k < nops; k++) {
    if ((k & (kOpChunk - 1)) == 0) stage_ops(ops, k, nops, s_ops);
    const OpIds op = staged_op(s_ops, k & (kOpChunk - 1));
    const double *tk = tab + (size_t)k * stride;
    const bool tiptip = op.l_kind == GEMS_CHILD_TIP && op.r_kind == GEMS_CHILD_TIP;
    double vl[PP][4], vr[PP][4];
    int sl[PP], sr[PP];
    msg_f64_4<SAFE, PP>(c, E, op.l_kind, op.l_id, tk, tk + 2 * blk, p, gq, vl, sl);
    msg_f64_4<SAFE, PP>(c, E, op.r_kind, op.r_id, tk + blk, tk + 2 * blk + (size_t)(c.unknown + 1) * blk,
                    p, gq, vr, sr);
#pragma unroll
    for (int u = 0; u < PP; u++) {
      double tmp[4], out[4];
#pragma unroll
      for (int x = 0; x < 4; x++) tmp[x] = vl[u][x] * vr[u][x];
      double lh_max = 0.0;
#pragma unroll
      for (int j = 0; j < 4; j++) {
        double acc = 0.0;
#pragma unroll
        for (int x = 0; x < 4; x++) acc = fma(E.inv[j * 4 + x], tmp[x], acc);
        out[j] = acc;
        lh_max = fmax(lh_max, fabs(acc));
      }
      if (!act[u]) lh_max = 0.0;
      if (!SAFE) lh_max = group_max(lh_max, G);
      if (act[u]) {
        int s_out = sl[u] + sr[u];
        if (!tiptip && lh_max < kScaleThr && c.invar[p[u]] == 0.0) {
#pragma unroll
          for (int j = 0; j < 4; j++) out[j] = ldexp(out[j], kScaleExp);
          s_out += 1;
        }
        store_row<4>(part + (size_t)op.dst_slot * c.slot_elems, c, p[u], gl, out);
        uint16_t *sc = c.scale + (size_t)op.dst_slot * c.slot_scale;
        if (SAFE)
          sc[(size_t)p[u] * C + gl] = (uint16_t)s_out;
        else if (gl == 0)
          sc[p[u]] = (uint16_t)s_out;
      }
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------------------
// Mixed: P_c(t) = evec diag(exp(eval r_c t)) inv_evec in FP64, rounded to FP32, stored
// [side][x][y][c]; tip tables [side][s][x][c] = P_c . indicator(s).
// ---------------------------------------------------------------------------------------
__global__ void k_prep_ops_mix(DevCtx c, const DevOp *ops, float *tab, size_t stride_f) {
  extern __shared__ double ex[];  // [C][n]
  const int k = blockIdx.x, side = blockIdx.y;
  const DevOp op = ops[k];
  const int kind = side ? op.r_kind : op.l_kind;
  const double len = side ? op.r_len : op.l_len;
  const int n = c.n, C = c.C, nnC = n * n * C;
  for (int idx = threadIdx.x; idx < C * n; idx += blockDim.x) {
    const int cc = idx / n, i = idx - cc * n;
    ex[idx] = exp(c.eval[i] * (c.rates[cc] * len));
  }
  __syncthreads();
  float *Pm = tab + (size_t)k * stride_f + (size_t)side * nnC;
  for (int idx = threadIdx.x; idx < nnC; idx += blockDim.x) {
    // stored [x][c][y]: lane c of a group reads its row x as n contiguous floats
    const int x = idx / (C * n), r = idx - x * C * n, cc = r / n, y = r - cc * n;
    double acc = 0.0;
    for (int i = 0; i < n; i++) acc = fma(c.evec[x * n + i] * ex[cc * n + i], c.inv_evec[i * n + y], acc);
    Pm[idx] = (float)fmax(acc, 0.0);
  }
  if (kind != GEMS_CHILD_TIP) return;
  __syncthreads();
  float *leaf = tab + (size_t)k * stride_f + (size_t)2 * nnC + (size_t)side * (c.unknown + 1) * c.block;
  const int rows = (c.unknown + 1) * c.block;
  // stored [s][c][x]: a category's message for state s is n contiguous floats
  for (int idx = threadIdx.x; idx < rows; idx += blockDim.x) {
    const int s = idx / c.block, r = idx - s * c.block, cc = r / n, x = r - cc * n;
    const double *ind = c.tip_real + (size_t)s * n;
    float acc = 0.f;
    for (int y = 0; y < n; y++) acc = fmaf(Pm[(x * C + cc) * n + y], (float)ind[y], acc);
    leaf[idx] = acc;
  }
}

template <int N, bool SAFE>
__device__ __forceinline__ void msg_mix(const DevCtx &c, int kind, int id,
                                        const float *__restrict__ Pm,
                                        const float *__restrict__ leaf, long p, int gl,
                                        float (&v)[N], int &s) {
  const int C = c.C;
  if (kind == GEMS_CHILD_TIP) {
    const int st = min((int)c.tips[(size_t)id * c.P + p], c.unknown);
    const float *lt = leaf + (size_t)st * c.block + gl * N;
#pragma unroll
    for (int x = 0; x < N; x++) v[x] = __ldg(lt + x);
    s = 0;
  } else {
    const float *src = static_cast<const float *>(c.partials) + (size_t)id * c.slot_elems +
                       mix_off<N>(c, p, gl);
    const int cs = mix_cs<N>();
    float L[N];
    if constexpr (N % 4 == 0) {
#pragma unroll
      for (int i = 0; i < N / 4; i++) {
        const float4 t = __ldcg(reinterpret_cast<const float4 *>(src + (size_t)i * cs));
        L[4 * i] = t.x;
        L[4 * i + 1] = t.y;
        L[4 * i + 2] = t.z;
        L[4 * i + 3] = t.w;
      }
    } else {
#pragma unroll
      for (int i = 0; i < N; i++) L[i] = __ldcg(src + i);
    }
#pragma unroll
    for (int x = 0; x < N; x++) {
      const float *row = Pm + ((size_t)x * C + gl) * N;
      float pr[N];
      if constexpr (N % 4 == 0) {
#pragma unroll
        for (int i = 0; i < N / 4; i++) {
          const float4 t = __ldg(reinterpret_cast<const float4 *>(row) + i);
          pr[4 * i] = t.x;
          pr[4 * i + 1] = t.y;
          pr[4 * i + 2] = t.z;
          pr[4 * i + 3] = t.w;
        }
      } else {
#pragma unroll
        for (int y = 0; y < N; y++) pr[y] = __ldg(row + y);
      }
      float acc = 0.f;
#pragma unroll
      for (int y = 0; y < N; y++) acc = fmaf(pr[y], L[y], acc);
      v[x] = acc;
    }
    const uint16_t *sc = c.scale + (size_t)id * c.slot_scale;
    s = SAFE ? sc[(size_t)p * C + gl] : sc[p];
  }
}

// 20 states on CUDA cores (4 states run k_traverse_mix4)
template <int N, bool SAFE>
__global__ void __launch_bounds__(kThreads, 1) k_traverse_mix(DevCtx c, const DevOp *__restrict__ ops,
                                                           int nops, const float *__restrict__ tab,
                                                           size_t stride_f, int p0, int p1) {
  const int G = c.G;
  const int gl = threadIdx.x & (G - 1);
  const long p = p0 + ((long)blockIdx.x * blockDim.x + threadIdx.x) / G;
  const bool act = p < p1 && gl < c.C;
  const int C = c.C;
  const size_t nnC = (size_t)N * N * C;
  float *part = static_cast<float *>(c.partials);
  __shared__ int4 s_ops[kOpChunk];
  for (int k = 0; k < nops; k++) {
    if ((k & (kOpChunk - 1)) == 0) stage_ops(ops, k, nops, s_ops);
    const OpIds op = staged_op(s_ops, k & (kOpChunk - 1));
    const float *tk = tab + (size_t)k * stride_f;
    const bool tiptip = op.l_kind == GEMS_CHILD_TIP && op.r_kind == GEMS_CHILD_TIP;
    float out[N];
    float lh_max = 0.f;
    int sl = 0, sr = 0;
    if (act) {
      float vl[N], vr[N];
      msg_mix<N, SAFE>(c, op.l_kind, op.l_id, tk, tk + 2 * nnC, p, gl, vl, sl);
      msg_mix<N, SAFE>(c, op.r_kind, op.r_id, tk + nnC,
                       tk + 2 * nnC + (size_t)(c.unknown + 1) * c.block, p, gl, vr, sr);
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
      float *dst = part + (size_t)op.dst_slot * c.slot_elems + mix_off<N>(c, p, gl);
      if constexpr (N % 4 == 0) {
        const int cs = mix_cs<N>();
#pragma unroll
        for (int i = 0; i < N / 4; i++)
          *reinterpret_cast<float4 *>(dst + (size_t)i * cs) =
              make_float4(out[4 * i], out[4 * i + 1], out[4 * i + 2], out[4 * i + 3]);
      } else {
#pragma unroll
        for (int i = 0; i < N; i++) dst[i] = out[i];
      }
      uint16_t *sc = c.scale + (size_t)op.dst_slot * c.slot_scale;
      if (SAFE)
        sc[(size_t)p * C + gl] = (uint16_t)s_out;
      else if (gl == 0)
        sc[p] = (uint16_t)s_out;
    }
    __syncwarp();
  }
}

// 4 states: the kernel is latency-bound on its child loads.  Each lane group handles PP
// patterns (at B blocks per SM), kThreads / G apart, so that a warp has the child loads of all of them in flight at
// once and loads each P row once for all of them; same arithmetic, in the same order, as
// msg_mix / k_traverse_mix.  Measured on the 512-taxon, 1M-pattern case: one pattern per group
// at 8 blocks per SM (32 registers) 14.8 ms; two at 5 blocks (48 registers) 12.6 ms; two at 4
// or 6 blocks 14.8 / 12.7 ms; four at 3 blocks 12.8 ms.  The variant in use is picked by the
// tuner below; every (PP, B) gives the same values.
template <bool SAFE, int PP>
__device__ __forceinline__ void msg_mix4(const DevCtx &c, int kind, int id,
                                         const float *__restrict__ Pm,
                                         const float *__restrict__ leaf,
                                         const long (&p)[PP], int gq,
                                         float (&v)[PP][4], int (&s)[PP]) {
  const int C = c.C;
  if (kind == GEMS_CHILD_TIP) {
    int st[PP];
#pragma unroll
    for (int u = 0; u < PP; u++) st[u] = min((int)c.tips[(size_t)id * c.P + p[u]], c.unknown);
#pragma unroll
    for (int u = 0; u < PP; u++) {
      const float4 t = __ldg(reinterpret_cast<const float4 *>(leaf + (size_t)st[u] * c.block) + gq);
      v[u][0] = t.x, v[u][1] = t.y, v[u][2] = t.z, v[u][3] = t.w;
      s[u] = 0;
    }
  } else {
    const float *base = static_cast<const float *>(c.partials) + (size_t)id * c.slot_elems;
    float4 L[PP];
#pragma unroll
    for (int u = 0; u < PP; u++)
      L[u] = __ldcg(reinterpret_cast<const float4 *>(base + mix_off<4>(c, p[u], gq)));
    const uint16_t *sc = c.scale + (size_t)id * c.slot_scale;
#pragma unroll
    for (int u = 0; u < PP; u++) s[u] = SAFE ? sc[(size_t)p[u] * C + gq] : sc[p[u]];
#pragma unroll
    for (int x = 0; x < 4; x++) {
      const float4 r = __ldg(reinterpret_cast<const float4 *>(Pm + ((size_t)x * C + gq) * 4));
#pragma unroll
      for (int u = 0; u < PP; u++)
        v[u][x] = fmaf(r.w, L[u].w, fmaf(r.z, L[u].z, fmaf(r.y, L[u].y, fmaf(r.x, L[u].x, 0.f))));
    }
  }
}

template <bool SAFE, int PP, int B>
__global__ void __launch_bounds__(kThreads, B)
    k_traverse_mix4(DevCtx c, const DevOp *__restrict__ ops, int nops,
                    const float *__restrict__ tab, size_t stride_f, int p0, int p1) {
  const int G = c.G, C = c.C;
  const int gl = threadIdx.x & (G - 1);
  const int gq = gl < C ? gl : 0;  // loads of idle lanes stay inside the tables
  const int per = kThreads / G;
  const long pb = p0 + (long)blockIdx.x * per * PP + threadIdx.x / G;
  long p[PP];
  bool act[PP];
#pragma unroll
  for (int u = 0; u < PP; u++) {
    const long q = pb + (long)u * per;
    act[u] = q < p1 && gl < C;
    p[u] = q < p1 ? q : p0;
  }
  const size_t nnC = (size_t)16 * C;
  float *part = static_cast<float *>(c.partials);
  __shared__ int4 s_ops[kOpChunk];
  for (int k = 0; k < nops; k++) {
    if ((k & (kOpChunk - 1)) == 0) stage_ops(ops, k, nops, s_ops);
    const OpIds op = staged_op(s_ops, k & (kOpChunk - 1));
    const float *tk = tab + (size_t)k * stride_f;
    const bool tiptip = op.l_kind == GEMS_CHILD_TIP && op.r_kind == GEMS_CHILD_TIP;
    float vl[PP][4], vr[PP][4];
    int sl[PP], sr[PP];
    msg_mix4<SAFE, PP>(c, op.l_kind, op.l_id, tk, tk + 2 * nnC, p, gq, vl, sl);
    msg_mix4<SAFE, PP>(c, op.r_kind, op.r_id, tk + nnC, tk + 2 * nnC + (size_t)(c.unknown + 1) * c.block,
                   p, gq, vr, sr);
#pragma unroll
    for (int u = 0; u < PP; u++) {
      float lh_max = 0.f;
#pragma unroll
      for (int x = 0; x < 4; x++) {
        vl[u][x] *= vr[u][x];
        lh_max = fmaxf(lh_max, vl[u][x]);
      }
      if (!act[u]) lh_max = 0.f;
      if (!SAFE) lh_max = group_maxf(lh_max, G);
      if (act[u]) {
        int s_out = sl[u] + sr[u];
        if (!tiptip && lh_max < kScaleThrF && c.invar[p[u]] == 0.0) {
#pragma unroll
          for (int x = 0; x < 4; x++) vl[u][x] *= 18446744073709551616.0f;  // 2^64
          s_out += 1;
        }
        *reinterpret_cast<float4 *>(part + (size_t)op.dst_slot * c.slot_elems + mix_off<4>(c, p[u], gl)) =
            make_float4(vl[u][0], vl[u][1], vl[u][2], vl[u][3]);
        uint16_t *sc = c.scale + (size_t)op.dst_slot * c.slot_scale;
        if (SAFE)
          sc[(size_t)p[u] * C + gl] = (uint16_t)s_out;
        else if (gl == 0)
          sc[p[u]] = (uint16_t)s_out;
      }
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------------------
// 4 states with the traversal plan (plan.h): a child produced earlier in the same launch comes
// from registers (forwarded: its consumer is the next op) or from a per-thread stack in shared
// memory, not from a dependent global load; every output is still stored to its slot, with a
// streaming store.  DRAM then carries what a traversal must move: the partial writes, the tip
// bytes, children computed before the launch.  Same arithmetic in the same order as
// msg_mix4 / k_traverse_mix4 (R = float) and msg_f64_4 / k_traverse_f64x (R = double), so the
// values are bit-identical to theirs.  Shared memory: depth positions x PP patterns x
// kThreads threads of 4 values (FP32 as one float4, FP64 as two double2 planes) and a uint16
// scale counter.
// ---------------------------------------------------------------------------------------
template <typename R, int PP>
struct Stack4 {
  unsigned char *base;
  int depth;
  static constexpr size_t kVal = 4 * sizeof(R);  // bytes of one thread's entry
  __device__ __forceinline__ size_t vidx(int pos, int u) const {
    return ((size_t)pos * PP + u) * kThreads + threadIdx.x;
  }
  __device__ __forceinline__ void put(int pos, int u, const R (&v)[4], int sc) const {
    if constexpr (sizeof(R) == 4) {
      reinterpret_cast<float4 *>(base)[vidx(pos, u)] = make_float4(v[0], v[1], v[2], v[3]);
    } else {
      double2 *d = reinterpret_cast<double2 *>(base);
      const size_t plane = (size_t)depth * PP * kThreads;
      d[vidx(pos, u)] = make_double2(v[0], v[1]);
      d[plane + vidx(pos, u)] = make_double2(v[2], v[3]);
    }
    scales()[vidx(pos, u)] = (uint16_t)sc;
  }
  __device__ __forceinline__ void get(int pos, int u, R (&v)[4], int &sc) const {
    if constexpr (sizeof(R) == 4) {
      const float4 t = reinterpret_cast<const float4 *>(base)[vidx(pos, u)];
      v[0] = t.x, v[1] = t.y, v[2] = t.z, v[3] = t.w;
    } else {
      const double2 *d = reinterpret_cast<const double2 *>(base);
      const size_t plane = (size_t)depth * PP * kThreads;
      const double2 a = d[vidx(pos, u)], b = d[plane + vidx(pos, u)];
      v[0] = a.x, v[1] = a.y, v[2] = b.x, v[3] = b.y;
    }
    sc = scales()[vidx(pos, u)];
  }
  __device__ __forceinline__ uint16_t *scales() const {
    return reinterpret_cast<uint16_t *>(base + (size_t)depth * PP * kThreads * kVal);
  }
  static size_t bytes(int depth) { return (size_t)depth * PP * kThreads * (kVal + 2); }
};

// ---------------------------------------------------------------------------------------
// 4 states, one thread per pattern (all C categories in registers), with the traversal plan.
// Every per-op input a thread needs sits in shared memory before the op starts: the op
// descriptors, the op tables and the tip bytes of the CTA's 128 patterns are copied with
// cp.async one chunk of ops ahead (double-buffered; chunk_p<R>() ops), and children produced in
// the launch come from registers (forwarded) or the per-thread stack.  Per op a warp then does
// shared-memory reads, FMAs and one coalesced 32 x (C*4 values) store: no load on its critical
// path.  Mixed form: the tip messages are taken from the staged P_c(t) (a tip's value for
// state set S is the sum of the P columns in S, added in state order as the table of
// k_prep_ops_mix forms it, so the bits are the same).  FP64 form: the staged tables hold the
// exp factors and the leaf rows of the four bases and of the unknown state; ambiguity codes
// read their row from global memory.  Values are bit-identical to k_traverse_mix4 /
// k_traverse_f64x.
// ---------------------------------------------------------------------------------------
constexpr int kThreadsP = 128;  // patterns per CTA
constexpr int kChunkP = 8;      // ops staged together (lane-per-category kernel)
// ops staged together by the one-thread-per-pattern kernel: 8 for FP32; 4 for FP64, whose
// tables are twice the size and whose stack lives in shared memory, so that three CTAs fit an
// SM (the plan depth of a 512-taxon tree is 3: 68 KB a CTA)
template <typename R>
__host__ __device__ constexpr int chunk_p() { return sizeof(R) == 4 ? 8 : 4; }

// staged op table: the head (mixed: P_c(t) as [side][x][c][y] floats; FP64: the exp factors as
// [side][i][c] doubles), then per side the leaf rows of the bases A, C, G, T and of the unknown
// state; the global table holds the head, then a row per state and side (mixed [c][x], FP64
// [x][c])
template <typename R, int C>
struct Tab4P {
  static constexpr int kH = sizeof(R) == 4 ? 2 * 16 * C : 2 * 4 * C;  // head elements
  // a staged leaf row: 4C values padded by 16 bytes (4 floats, 2 doubles) so that the rows of
  // different states start in different bank groups (lanes of a warp read the rows of their
  // own states; unpadded rows are a multiple of 128 bytes apart and collide)
  static constexpr int kRow = sizeof(R) == 4 ? 4 * C + 4 : 4 * C + 2;
  static constexpr int kLeaf = 5 * kRow;  // leaf elements per side
  static constexpr int kBytes = (kH + 2 * kLeaf) * (int)sizeof(R);
};

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                   static_cast<uint32_t>(__cvta_generic_to_shared(smem))),
               "l"(gmem)
               : "memory");
}
// 8-byte copy (the op descriptors are 40 bytes, 8-byte aligned)
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(
                   static_cast<uint32_t>(__cvta_generic_to_shared(smem))),
               "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait1() {
  asm volatile("cp.async.wait_group 1;" ::: "memory");
}

template <typename R, int C>
struct StageP {
  DevOp desc[2][chunk_p<R>()];
  alignas(16) unsigned char tab[2][chunk_p<R>()][Tab4P<R, C>::kBytes];
  alignas(16) uint8_t tips[2][chunk_p<R>()][2][kThreadsP];
};
// every 16-byte copy target inside StageP, and the stack placed after it, stay 16-byte aligned
static_assert(Tab4P<float, 1>::kBytes % 16 == 0 && Tab4P<double, 1>::kBytes % 16 == 0 &&
                  sizeof(StageP<float, 1>) % 16 == 0 && sizeof(StageP<double, 8>) % 16 == 0,
              "16-byte pieces");

// copies the descriptors, tables and tip bytes of ops [k0, k0 + nk) into buffer b (every thread
// takes a share of the 16-byte pieces); tip bytes of a side are copied only for a tip child, and
// only when the CTA's first pattern is 16-byte aligned (tips_async), else read directly
template <typename R, int C>
__device__ __forceinline__ void stage4p(StageP<R, C> &st, int b, const DevCtx &c,
                                        const DevOp *__restrict__ ops, const R *__restrict__ tab,
                                        size_t stride, int k0, int nk, long pbase,
                                        bool tips_async) {
  using T = Tab4P<R, C>;
  const int tid = threadIdx.x;
  // descriptors: sizeof(DevOp) / 8 pieces of 8 bytes each
  constexpr int kDescPieces = sizeof(DevOp) / 8;
  static_assert(sizeof(DevOp) % 8 == 0 && alignof(DevOp) >= 8, "8-byte pieces of a DevOp");
  for (int q = tid; q < kDescPieces * nk; q += kThreadsP) {
    const int i = q / kDescPieces, r = q - i * kDescPieces;
    cp_async8(reinterpret_cast<char *>(&st.desc[b][i]) + 8 * r,
              reinterpret_cast<const char *>(ops + k0 + i) + 8 * r);
  }
  constexpr int kPieces = (T::kH + 10 * 4 * C) * (int)sizeof(R) / 16;  // pieces copied
  for (int q = tid; q < nk * kPieces; q += kThreadsP) {
    const int i = q / kPieces, r = q - i * kPieces;
    const R *tk = tab + (size_t)(k0 + i) * stride;
    const int blk = 4 * C, u1 = c.unknown + 1;
    constexpr int hP = T::kH * (int)sizeof(R) / 16, rowP = 4 * C * (int)sizeof(R) / 16;
    const char *src;
    int dst;  // byte offset inside the staged table
    if (r < hP) {
      src = reinterpret_cast<const char *>(tk) + 16 * r;
      dst = 16 * r;
    } else {
      const int o = r - hP, side = o / (5 * rowP), rr = o - side * 5 * rowP, row = rr / rowP,
                pc = rr - row * rowP;
      const R *leaf = tk + T::kH + (size_t)side * u1 * blk;
      src = reinterpret_cast<const char *>(leaf + (size_t)(row < 4 ? row : c.unknown) * blk) + 16 * pc;
      dst = (T::kH + side * T::kLeaf + row * T::kRow) * (int)sizeof(R) + 16 * pc;
    }
    cp_async16(st.tab[b][i] + dst, src);
  }
  if (tips_async) {
    // 8 pieces per tip side; pieces past the padded pattern count are not copied (never read)
    for (int q = tid; q < nk * 2 * 8; q += kThreadsP) {
      const int i = q >> 4, sd = (q >> 3) & 1, r = q & 7;
      const DevOp &o = ops[k0 + i];
      const int kind = sd ? o.r_kind : o.l_kind, id = sd ? o.r_id : o.l_id;
      if (kind != GEMS_CHILD_TIP || pbase + 16 * r >= c.P) continue;
      cp_async16(&st.tips[b][i][sd][16 * r], c.tips + (size_t)id * c.P + pbase + 16 * r);
    }
  }
}

// a pattern's category 0 within a slot: FP32 tile-major (mix_off<4>), FP64 pattern-major
template <typename R>
__device__ __forceinline__ size_t pat_off(const DevCtx &c, long p) {
  if constexpr (sizeof(R) == 4) return mix_off<4>(c, p, 0);
  else return f64_off<4>(c, p, 0, 0);
}

// 16-byte moves of a thread's C x 4 values (FP32: one float4 per category; FP64: two double2)
// src points at category 0 of the pattern in the tile-major slot: FP32 categories mix_cs<4>()
// floats apart; FP64 (f64_off) in halves kF64Half doubles apart, a category two halves
template <int C>
__device__ __forceinline__ void ld_cg(const float *src, float (&v)[C][4]) {
#pragma unroll
  for (int q = 0; q < C; q++) {
    const float4 t = __ldcg(reinterpret_cast<const float4 *>(src + (size_t)q * mix_cs<4>()));
    v[q][0] = t.x, v[q][1] = t.y, v[q][2] = t.z, v[q][3] = t.w;
  }
}
template <int C>
__device__ __forceinline__ void ld_cg(const double *src, double (&v)[C][4]) {
#pragma unroll
  for (int q = 0; q < 2 * C; q++) {  // piece q: category q / 2, half q % 2 (f64_off)
    const double2 t = __ldcg(reinterpret_cast<const double2 *>(src + (size_t)q * kF64Half));
    v[q >> 1][2 * (q & 1)] = t.x, v[q >> 1][2 * (q & 1) + 1] = t.y;
  }
}
template <int C>
__device__ __forceinline__ void st_cs(float *dst, const float (&v)[C][4]) {
#pragma unroll
  for (int q = 0; q < C; q++)
    __stcs(reinterpret_cast<float4 *>(dst + (size_t)q * mix_cs<4>()),
           make_float4(v[q][0], v[q][1], v[q][2], v[q][3]));
}
template <int C>
__device__ __forceinline__ void st_cs(double *dst, const double (&v)[C][4]) {
#pragma unroll
  for (int q = 0; q < 2 * C; q++)
    __stcs(reinterpret_cast<double2 *>(dst + (size_t)q * kF64Half),
           make_double2(v[q >> 1][2 * (q & 1)], v[q >> 1][2 * (q & 1) + 1]));
}
// shared memory, [piece][thread] (a warp's accesses are 512 contiguous bytes)
template <int C>
__device__ __forceinline__ void sm_put(unsigned char *base, const float (&v)[C][4]) {
#pragma unroll
  for (int q = 0; q < C; q++)
    reinterpret_cast<float4 *>(base)[q * kThreadsP + threadIdx.x] =
        make_float4(v[q][0], v[q][1], v[q][2], v[q][3]);
}
template <int C>
__device__ __forceinline__ void sm_put(unsigned char *base, const double (&v)[C][4]) {
#pragma unroll
  for (int q = 0; q < 2 * C; q++)
    reinterpret_cast<double2 *>(base)[q * kThreadsP + threadIdx.x] =
        make_double2(v[q >> 1][2 * (q & 1)], v[q >> 1][2 * (q & 1) + 1]);
}
template <int C>
__device__ __forceinline__ void sm_get(const unsigned char *base, float (&v)[C][4]) {
#pragma unroll
  for (int q = 0; q < C; q++) {
    const float4 t = reinterpret_cast<const float4 *>(base)[q * kThreadsP + threadIdx.x];
    v[q][0] = t.x, v[q][1] = t.y, v[q][2] = t.z, v[q][3] = t.w;
  }
}
template <int C>
__device__ __forceinline__ void sm_get(const unsigned char *base, double (&v)[C][4]) {
#pragma unroll
  for (int q = 0; q < 2 * C; q++) {
    const double2 t = reinterpret_cast<const double2 *>(base)[q * kThreadsP + threadIdx.x];
    v[q >> 1][2 * (q & 1)] = t.x, v[q >> 1][2 * (q & 1) + 1] = t.y;
  }
}

// the fields of an op a thread uses, and its tip bytes (0 for a partial child)
struct OpFetch {
  int w, l_id, r_id, dst, tb[2];
};
__device__ __forceinline__ OpFetch fetch4p(const DevOp &o, const uint8_t (&tips)[2][kThreadsP],
                                           bool tips_async, const DevCtx &c, long p) {
  OpFetch f;
  f.w = o.pad_;
  f.l_id = o.l_id;
  f.r_id = o.r_id;
  f.dst = o.dst_slot;
  f.tb[0] = f.tb[1] = 0;
  if (plan_lkind(f.w) == GEMS_CHILD_TIP)
    f.tb[0] = tips_async ? tips[0][threadIdx.x] : c.tips[(size_t)f.l_id * c.P + p];
  if (plan_rkind(f.w) == GEMS_CHILD_TIP)
    f.tb[1] = tips_async ? tips[1][threadIdx.x] : c.tips[(size_t)f.r_id * c.P + p];
  return f;
}

// the plan's stack of one thread: FP32 positions 0 and 1 in registers (the common ones:
// positions are handed out lowest first), deeper ones in shared memory; FP64 all in shared
// memory (its registers already limit the resident blocks)
template <typename R>
__host__ __device__ constexpr int reg_pos() {
  return sizeof(R) == 4 ? 2 : 0;
}
template <typename R, int C>
struct StackP {
  unsigned char *base;
  int depth;  // positions held in shared memory (plan depth - reg_pos<R>())
  static constexpr int kEntry = 4 * C * (int)sizeof(R);  // value bytes of one thread's entry
  __device__ __forceinline__ uint16_t *scs() const {
    return reinterpret_cast<uint16_t *>(base + (size_t)depth * kEntry * kThreadsP);
  }
  static size_t bytes(int plan_depth) {
    return (size_t)std::max(plan_depth - reg_pos<R>(), 0) * kThreadsP * (kEntry + 2 * C);
  }
  // counters: C per entry under SAFE scaling, the first one only under NORM (all are equal)
  template <bool SAFE>
  __device__ __forceinline__ void put(int pos, const R (&v)[C][4], const int (&sc)[C]) const {
    sm_put<C>(base + (size_t)pos * kEntry * kThreadsP, v);
#pragma unroll
    for (int cc = 0; cc < (SAFE ? C : 1); cc++)
      scs()[((size_t)pos * C + cc) * kThreadsP + threadIdx.x] = (uint16_t)sc[cc];
  }
  template <bool SAFE>
  __device__ __forceinline__ void get(int pos, R (&v)[C][4], int (&sc)[C]) const {
    sm_get<C>(base + (size_t)pos * kEntry * kThreadsP, v);
#pragma unroll
    for (int cc = 0; cc < (SAFE ? C : 1); cc++)
      sc[cc] = scs()[((size_t)pos * C + cc) * kThreadsP + threadIdx.x];
    if (!SAFE) {
#pragma unroll
      for (int cc = 1; cc < C; cc++) sc[cc] = sc[0];
    }
  }
};

// one child's message for all categories: L from the plan's source, the op's transition applied
template <typename R, bool SAFE, int C>
__device__ __forceinline__ void msg4p(const DevCtx &c, const EigPack<4> &E, int kind, int id,
                                      int src, int pos, const StackP<R, C> &stk,
                                      const R (&fwd)[C][4], const int (&fwd_s)[C],
                                      const R (&r0)[C][4], const int (&r0s)[C],
                                      const R (&r1)[C][4], const int (&r1s)[C],
                                      const unsigned char *__restrict__ tabS,
                                      const R *__restrict__ tk, int side, int tipbyte, long p,
                                      R (&v)[C][4], int (&s)[C]) {
  using T = Tab4P<R, C>;
  if (kind == GEMS_CHILD_TIP) {
    const int st = min(tipbyte, c.unknown);
#pragma unroll
    for (int cc = 0; cc < C; cc++) s[cc] = 0;
    if constexpr (sizeof(R) == 4) {
      if (st < 4 || st == c.unknown) {
        const float4 *row = reinterpret_cast<const float4 *>(tabS) +
                            (T::kH + side * T::kLeaf + (st < 4 ? st : 4) * T::kRow) / 4;
#pragma unroll
        for (int cc = 0; cc < C; cc++) {
          const float4 t = row[cc];
          v[cc][0] = t.x, v[cc][1] = t.y, v[cc][2] = t.z, v[cc][3] = t.w;
        }
      } else {
        // an ambiguity code: the sum of the P columns of its states, in state order
        const int mask = st - 3;
        const float4 *P4 = reinterpret_cast<const float4 *>(tabS) + side * 4 * C;
#pragma unroll
        for (int x = 0; x < 4; x++)
#pragma unroll
          for (int cc = 0; cc < C; cc++) {
            const float4 r = P4[x * C + cc];
            float acc = 0.f;
            if (mask & 1) acc = acc + r.x;
            if (mask & 2) acc = acc + r.y;
            if (mask & 4) acc = acc + r.z;
            if (mask & 8) acc = acc + r.w;
            v[cc][x] = acc;
          }
      }
    } else {
      const int blk = 4 * C;
      const double *row;
      if (st < 4 || st == c.unknown) {
        row = reinterpret_cast<const double *>(tabS) + T::kH + side * T::kLeaf +
              (st < 4 ? st : 4) * T::kRow;
#pragma unroll
        for (int x = 0; x < 4; x++)
#pragma unroll
          for (int cc = 0; cc < C; cc++) v[cc][x] = row[x * C + cc];
      } else {
        row = tk + 2 * blk + (size_t)side * (c.unknown + 1) * blk + (size_t)st * blk;
#pragma unroll
        for (int x = 0; x < 4; x++)
#pragma unroll
          for (int cc = 0; cc < C; cc++) v[cc][x] = __ldg(row + x * C + cc);
      }
    }
    return;
  }
  R L[C][4];
  if (src == kSrcFwd) {
#pragma unroll
    for (int cc = 0; cc < C; cc++) {
#pragma unroll
      for (int x = 0; x < 4; x++) L[cc][x] = fwd[cc][x];
      s[cc] = fwd_s[cc];
    }
  } else if (src == kSrcStack && pos < reg_pos<R>()) {
    const R(&rv)[C][4] = pos == 0 ? r0 : r1;
    const int(&rs)[C] = pos == 0 ? r0s : r1s;
#pragma unroll
    for (int cc = 0; cc < C; cc++) {
#pragma unroll
      for (int x = 0; x < 4; x++) L[cc][x] = rv[cc][x];
      s[cc] = rs[cc];
    }
  } else if (src == kSrcStack) {
    stk.template get<SAFE>(min(pos - reg_pos<R>(), stk.depth - 1), L, s);
  } else {
    ld_cg<C>(static_cast<const R *>(c.partials) + (size_t)id * c.slot_elems + pat_off<R>(c, p),
             L);
    const uint16_t *sc = c.scale + (size_t)id * c.slot_scale;
    if (SAFE) {
#pragma unroll
      for (int cc = 0; cc < C; cc++) s[cc] = sc[(size_t)p * C + cc];
    } else {
      const int v0 = sc[p];
#pragma unroll
      for (int cc = 0; cc < C; cc++) s[cc] = v0;
    }
  }
  if constexpr (sizeof(R) == 4) {
    const float4 *P4 = reinterpret_cast<const float4 *>(tabS) + side * 4 * C;
#pragma unroll
    for (int x = 0; x < 4; x++)
#pragma unroll
      for (int cc = 0; cc < C; cc++) {
        const float4 r = P4[x * C + cc];
        v[cc][x] = fmaf(r.w, L[cc][3], fmaf(r.z, L[cc][2], fmaf(r.y, L[cc][1], fmaf(r.x, L[cc][0], 0.f))));
      }
  } else {
    const double *d = reinterpret_cast<const double *>(tabS) + side * 4 * C;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int cc = 0; cc < C; cc++) L[cc][i] *= d[i * C + cc];
#pragma unroll
    for (int cc = 0; cc < C; cc++)
#pragma unroll
      for (int x = 0; x < 4; x++) {
        double acc = 0.0;
#pragma unroll
        for (int i = 0; i < 4; i++) acc = fma(E.evec[x * 4 + i], L[cc][i], acc);
        v[cc][x] = acc;
      }
  }
}

template <typename R, bool SAFE, int C>
__global__ void __launch_bounds__(kThreadsP, sizeof(R) == 4 ? 4 : 3)
    k_traverse4p(DevCtx c, const DevOp *__restrict__ ops, int nops, const R *__restrict__ tab,
                 size_t stride, const EigPack<4> E, int p0, int p1, int depth) {
  extern __shared__ __align__(16) unsigned char smem_p[];
  StageP<R, C> &st = *reinterpret_cast<StageP<R, C> *>(smem_p);
  const StackP<R, C> stk{smem_p + sizeof(StageP<R, C>), max(depth - reg_pos<R>(), 0)};
  R r0[C][4], r1[C][4];
  int r0s[C], r1s[C];
#pragma unroll
  for (int cc = 0; cc < C; cc++) {
    r0s[cc] = r1s[cc] = 0;
#pragma unroll
    for (int x = 0; x < 4; x++) r0[cc][x] = r1[cc][x] = R(0);
  }
  const long pbase = p0 + (long)blockIdx.x * kThreadsP;
  const long pq = pbase + threadIdx.x;
  const bool act = pq < p1;
  const long p = act ? pq : p0;
  const bool tips_async = (pbase & 15) == 0;
  R fwd[C][4];
  int fwd_s[C];
#pragma unroll
  for (int cc = 0; cc < C; cc++) {
    fwd_s[cc] = 0;
#pragma unroll
    for (int x = 0; x < 4; x++) fwd[cc][x] = R(0);
  }
  R *part = static_cast<R *>(c.partials);
  constexpr int kCh = chunk_p<R>();
  stage4p<R, C>(st, 0, c, ops, tab, stride, 0, min(kCh, nops), pbase, tips_async);
  cp_async_commit();
  for (int k0 = 0; k0 < nops; k0 += kCh) {
    const int b = (k0 / kCh) & 1, nk = min(kCh, nops - k0);
    if (k0 + kCh < nops)
      stage4p<R, C>(st, b ^ 1, c, ops, tab, stride, k0 + kCh, min(kCh, nops - k0 - kCh), pbase,
                    tips_async);
    cp_async_commit();
    cp_async_wait1();  // this chunk's copies are done (the next chunk's may still fly)
    __syncthreads();
    // an op's descriptor fields and tip bytes are fetched while the previous op computes, so
    // that the chain descriptor -> tip byte -> leaf row is off each op's critical path
    OpFetch cur = fetch4p(st.desc[b][0], st.tips[b][0], tips_async, c, p), nxt{};
    for (int i = 0; i < nk; i++) {
      if (i + 1 < nk) nxt = fetch4p(st.desc[b][i + 1], st.tips[b][i + 1], tips_async, c, p);
      const int w = cur.w;
      const int lkind = plan_lkind(w), rkind = plan_rkind(w);
      const bool tiptip = lkind == GEMS_CHILD_TIP && rkind == GEMS_CHILD_TIP;
      const R *tk = tab + (size_t)(k0 + i) * stride;
      R vl[C][4], vr[C][4];
      int sl[C], sr[C];
      msg4p<R, SAFE, C>(c, E, lkind, cur.l_id, plan_lsrc(w), plan_lpos(w), stk, fwd, fwd_s, r0,
                        r0s, r1, r1s, st.tab[b][i], tk, 0, cur.tb[0], p, vl, sl);
      msg4p<R, SAFE, C>(c, E, rkind, cur.r_id, plan_rsrc(w), plan_rpos(w), stk, fwd, fwd_s, r0,
                        r0s, r1, r1s, st.tab[b][i], tk, 1, cur.tb[1], p, vr, sr);
      R out[C][4];
      R mx[C];
#pragma unroll
      for (int cc = 0; cc < C; cc++) {
        mx[cc] = R(0);
        if constexpr (sizeof(R) == 4) {
#pragma unroll
          for (int x = 0; x < 4; x++) {
            out[cc][x] = vl[cc][x] * vr[cc][x];
            mx[cc] = fmaxf(mx[cc], out[cc][x]);
          }
        } else {
          double tmp[4];
#pragma unroll
          for (int x = 0; x < 4; x++) tmp[x] = vl[cc][x] * vr[cc][x];
#pragma unroll
          for (int j = 0; j < 4; j++) {
            double acc = 0.0;
#pragma unroll
            for (int x = 0; x < 4; x++) acc = fma(E.inv[j * 4 + x], tmp[x], acc);
            out[cc][j] = acc;
            mx[cc] = fmax(mx[cc], fabs(acc));
          }
        }
      }
      int so[C];
      if constexpr (SAFE) {
#pragma unroll
        for (int cc = 0; cc < C; cc++) {
          so[cc] = sl[cc] + sr[cc];
          bool thr;
          if constexpr (sizeof(R) == 4) thr = mx[cc] < kScaleThrF;
          else thr = mx[cc] < kScaleThr;
          if (!tiptip && thr && c.invar[p] == 0.0) {
#pragma unroll
            for (int x = 0; x < 4; x++) {
              if constexpr (sizeof(R) == 4) out[cc][x] *= 18446744073709551616.0f;  // 2^64
              else out[cc][x] = ldexp(out[cc][x], kScaleExp);
            }
            so[cc] += 1;
          }
        }
      } else {
        R m = mx[0];
#pragma unroll
        for (int cc = 1; cc < C; cc++) m = sizeof(R) == 4 ? fmaxf(m, mx[cc]) : fmax(m, mx[cc]);
        int s0 = sl[0] + sr[0];
        bool thr;
        if constexpr (sizeof(R) == 4) thr = m < kScaleThrF;
        else thr = m < kScaleThr;
        if (!tiptip && thr && c.invar[p] == 0.0) {
#pragma unroll
          for (int cc = 0; cc < C; cc++)
#pragma unroll
            for (int x = 0; x < 4; x++) {
              if constexpr (sizeof(R) == 4) out[cc][x] *= 18446744073709551616.0f;  // 2^64
              else out[cc][x] = ldexp(out[cc][x], kScaleExp);
            }
          s0 += 1;
        }
#pragma unroll
        for (int cc = 0; cc < C; cc++) so[cc] = s0;
      }
      if (act) {
        st_cs<C>(part + (size_t)cur.dst * c.slot_elems + pat_off<R>(c, p), out);
        uint16_t *sc = c.scale + (size_t)cur.dst * c.slot_scale;
        if (SAFE) {
#pragma unroll
          for (int cc = 0; cc < C; cc++) sc[(size_t)p * C + cc] = (uint16_t)so[cc];
        } else {
          sc[p] = (uint16_t)so[0];
        }
      }
      if (plan_out(w) == kSrcStack) {
        const int op_pos = plan_opos(w);
        if (op_pos < reg_pos<R>()) {
#pragma unroll
          for (int cc = 0; cc < C; cc++) {
#pragma unroll
            for (int x = 0; x < 4; x++) {
              if (op_pos == 0) r0[cc][x] = out[cc][x];
              else r1[cc][x] = out[cc][x];
            }
            if (op_pos == 0) r0s[cc] = so[cc];
            else r1s[cc] = so[cc];
          }
        } else {
          stk.template put<SAFE>(min(op_pos - reg_pos<R>(), max(stk.depth - 1, 0)), out, so);
        }
      }
#pragma unroll
      for (int cc = 0; cc < C; cc++) {
#pragma unroll
        for (int x = 0; x < 4; x++) fwd[cc][x] = out[cc][x];
        fwd_s[cc] = so[cc];
      }
      cur = nxt;
    }
    __syncthreads();  // buffer b is refilled two chunks on
  }
}

// ---------------------------------------------------------------------------------------
// 4 states, a lane per category (G lanes a pattern, PP patterns a lane group), with the
// traversal plan and every per-op input staged in shared memory one chunk of kChunkP ops ahead
// (as k_traverse4p): op descriptors, op tables (head and the leaf rows of A, C, G, T and the
// unknown state) and the tip bytes of the CTA's patterns.  Lane c applies its category's
// transition: FP64 d_c (*) L then evec, FP32 the rows of P_c; the tip message is the lane's part
// of the staged leaf row (ambiguity codes read the global table).  Same arithmetic and order as
// k_traverse_f64x / k_traverse_mix4: bit-identical values.
// ---------------------------------------------------------------------------------------
struct StageQ {  // byte offsets of the regions of the dynamic shared memory
  int tab_bytes, npb;  // bytes of one staged op table; patterns of the CTA
  size_t desc, tab, tips, stack;
  __host__ __device__ static size_t up16(size_t x) { return (x + 15) & ~(size_t)15; }
  __host__ __device__ StageQ(bool fp64, int C, int npb_) : npb(npb_) {
    const int kH = fp64 ? 8 * C : 32 * C, kLeaf = 20 * C;
    tab_bytes = (kH + 2 * kLeaf) * (fp64 ? 8 : 4);
    desc = 0;
    tab = up16(desc + 2 * kChunkP * sizeof(DevOp));
    tips = up16(tab + (size_t)2 * kChunkP * tab_bytes);
    stack = up16(tips + (size_t)2 * kChunkP * 2 * npb);
  }
};

template <typename R>
__device__ __forceinline__ void stage4q(unsigned char *sm, const StageQ &L, int b,
                                        const DevCtx &c, const DevOp *__restrict__ ops,
                                        const R *__restrict__ tab, size_t stride, int k0, int nk,
                                        long pbase, bool tips_async) {
  const int tid = threadIdx.x, nt = blockDim.x, C = c.C, blk = 4 * C, u1 = c.unknown + 1;
  constexpr int kDescPieces = sizeof(DevOp) / 8;
  DevOp *desc = reinterpret_cast<DevOp *>(sm + L.desc) + b * kChunkP;
  for (int q = tid; q < kDescPieces * nk; q += nt) {
    const int i = q / kDescPieces, r = q - i * kDescPieces;
    cp_async8(reinterpret_cast<char *>(desc + i) + 8 * r,
              reinterpret_cast<const char *>(ops + k0 + i) + 8 * r);
  }
  const int pieces = L.tab_bytes / 16;
  const int hB = (sizeof(R) == 4 ? 32 * C : 8 * C) * (int)sizeof(R);
  const int rowsB = 16 * C * (int)sizeof(R), rowB = 4 * C * (int)sizeof(R);
  unsigned char *tb = sm + L.tab + (size_t)b * kChunkP * L.tab_bytes;
  for (int q = tid; q < nk * pieces; q += nt) {
    const int i = q / pieces, r = q - i * pieces, off = 16 * r;
    const R *tk = tab + (size_t)(k0 + i) * stride;
    const char *src;
    if (off < hB) {
      src = reinterpret_cast<const char *>(tk) + off;
    } else {
      const int o = off - hB, side = o / (rowsB + rowB), w = o - side * (rowsB + rowB);
      const R *leaf = tk + hB / (int)sizeof(R) + (size_t)side * u1 * blk;
      src = w < rowsB ? reinterpret_cast<const char *>(leaf) + w
                      : reinterpret_cast<const char *>(leaf + (size_t)c.unknown * blk) + (w - rowsB);
    }
    cp_async16(tb + (size_t)i * L.tab_bytes + off, src);
  }
  if (tips_async) {
    const int per_side = L.npb / 16;
    uint8_t *tp = sm + L.tips + (size_t)b * kChunkP * 2 * L.npb;
    for (int q = tid; q < nk * 2 * per_side; q += nt) {
      const int i = q / (2 * per_side), rem = q - i * 2 * per_side, sd = rem / per_side,
                r = rem - sd * per_side;
      const DevOp &o = ops[k0 + i];
      const int kind = sd ? o.r_kind : o.l_kind, id = sd ? o.r_id : o.l_id;
      if (kind != GEMS_CHILD_TIP || pbase + 16 * r >= c.P) continue;
      cp_async16(tp + ((size_t)i * 2 + sd) * L.npb + 16 * r,
                 c.tips + (size_t)id * c.P + pbase + 16 * r);
    }
  }
}

// a lane's message for one child: L from the plan's source, its category's transition applied
template <typename R, bool SAFE, int PP>
__device__ __forceinline__ void msg4q(const DevCtx &c, const EigPack<4> &E, int kind, int id,
                                      int src, int pos, const Stack4<R, PP> &stk,
                                      const R (&fwd)[PP][4], const int (&fwd_s)[PP],
                                      const unsigned char *__restrict__ tabS,
                                      const R *__restrict__ tk, int side, const int (&tb)[PP],
                                      const long (&p)[PP], int gq, R (&v)[PP][4], int (&s)[PP]) {
  const int C = c.C, blk = 4 * C;
  const int kH = sizeof(R) == 4 ? 32 * C : 8 * C, kLeaf = 20 * C;
  if (kind == GEMS_CHILD_TIP) {
#pragma unroll
    for (int u = 0; u < PP; u++) {
      const int st = min(tb[u], c.unknown);
      s[u] = 0;
      if (st < 4 || st == c.unknown) {
        const R *row = reinterpret_cast<const R *>(tabS) + kH + side * kLeaf +
                       (st < 4 ? st : 4) * blk;
        if constexpr (sizeof(R) == 4) {  // [c][x]
          const float4 t = reinterpret_cast<const float4 *>(row)[gq];
          v[u][0] = t.x, v[u][1] = t.y, v[u][2] = t.z, v[u][3] = t.w;
        } else {  // [x][c]
#pragma unroll
          for (int x = 0; x < 4; x++) v[u][x] = row[x * C + gq];
        }
      } else {
        const R *leaf = tk + kH + (size_t)side * (c.unknown + 1) * blk + (size_t)st * blk;
        if constexpr (sizeof(R) == 4) {
          const float4 t = __ldg(reinterpret_cast<const float4 *>(leaf) + gq);
          v[u][0] = t.x, v[u][1] = t.y, v[u][2] = t.z, v[u][3] = t.w;
        } else {
#pragma unroll
          for (int x = 0; x < 4; x++) v[u][x] = __ldg(leaf + x * C + gq);
        }
      }
    }
    return;
  }
  R L[PP][4];
  if (src == kSrcFwd) {
#pragma unroll
    for (int u = 0; u < PP; u++) {
#pragma unroll
      for (int x = 0; x < 4; x++) L[u][x] = fwd[u][x];
      s[u] = fwd_s[u];
    }
  } else if (src == kSrcStack) {
#pragma unroll
    for (int u = 0; u < PP; u++) stk.get(min(pos, stk.depth - 1), u, L[u], s[u]);
  } else {
    const R *base = static_cast<const R *>(c.partials) + (size_t)id * c.slot_elems;
    const uint16_t *sc = c.scale + (size_t)id * c.slot_scale;
#pragma unroll
    for (int u = 0; u < PP; u++) {
      if constexpr (sizeof(R) == 4) {
        const float4 t = __ldcg(reinterpret_cast<const float4 *>(base + mix_off<4>(c, p[u], gq)));
        L[u][0] = t.x, L[u][1] = t.y, L[u][2] = t.z, L[u][3] = t.w;
      } else {
        load_row<4>(base, c, p[u], gq, L[u]);
      }
      s[u] = SAFE ? sc[(size_t)p[u] * C + gq] : sc[p[u]];
    }
  }
  if constexpr (sizeof(R) == 4) {
    const float4 *P4 = reinterpret_cast<const float4 *>(tabS) + side * 4 * C;
#pragma unroll
    for (int x = 0; x < 4; x++) {
      const float4 r = P4[x * C + gq];
#pragma unroll
      for (int u = 0; u < PP; u++)
        v[u][x] = fmaf(r.w, L[u][3], fmaf(r.z, L[u][2], fmaf(r.y, L[u][1], fmaf(r.x, L[u][0], 0.f))));
    }
  } else {
    const double *d = reinterpret_cast<const double *>(tabS) + side * 4 * C;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const double di = d[i * C + gq];
#pragma unroll
      for (int u = 0; u < PP; u++) L[u][i] *= di;
    }
#pragma unroll
    for (int u = 0; u < PP; u++)
#pragma unroll
      for (int x = 0; x < 4; x++) {
        double acc = 0.0;
#pragma unroll
        for (int i = 0; i < 4; i++) acc = fma(E.evec[x * 4 + i], L[u][i], acc);
        v[u][x] = acc;
      }
  }
}

template <typename R, bool SAFE, int PP, int B>
__global__ void __launch_bounds__(kThreads, B)
    k_traverse4q(DevCtx c, const DevOp *__restrict__ ops, int nops, const R *__restrict__ tab,
                 size_t stride, const EigPack<4> E, int p0, int p1, int depth) {
  extern __shared__ __align__(16) unsigned char smem_q[];
  const int G = c.G, C = c.C;
  const int gl = threadIdx.x & (G - 1);
  const int gq = gl < C ? gl : 0;  // loads of idle lanes stay inside the tables
  const int per = kThreads / G;
  const StageQ L(sizeof(R) == 8, C, per * PP);
  const long pbase = p0 + (long)blockIdx.x * per * PP;
  const bool tips_async = (pbase & 15) == 0;
  long p[PP];
  bool act[PP];
  int toff[PP];  // the pattern's byte in the staged tip rows
#pragma unroll
  for (int u = 0; u < PP; u++) {
    toff[u] = u * per + threadIdx.x / G;
    const long q = pbase + toff[u];
    act[u] = q < p1 && gl < C;
    p[u] = q < p1 ? q : p0;
  }
  const Stack4<R, PP> stk{smem_q + L.stack, depth};
  R fwd[PP][4];
  int fwd_s[PP];
#pragma unroll
  for (int u = 0; u < PP; u++) {
    fwd_s[u] = 0;
#pragma unroll
    for (int x = 0; x < 4; x++) fwd[u][x] = R(0);
  }
  R *part = static_cast<R *>(c.partials);
  stage4q<R>(smem_q, L, 0, c, ops, tab, stride, 0, min(kChunkP, nops), pbase, tips_async);
  cp_async_commit();
  for (int k0 = 0; k0 < nops; k0 += kChunkP) {
    const int b = (k0 / kChunkP) & 1, nk = min(kChunkP, nops - k0);
    if (k0 + kChunkP < nops)
      stage4q<R>(smem_q, L, b ^ 1, c, ops, tab, stride, k0 + kChunkP,
                 min(kChunkP, nops - k0 - kChunkP), pbase, tips_async);
    cp_async_commit();
    cp_async_wait1();
    __syncthreads();
    const DevOp *desc = reinterpret_cast<const DevOp *>(smem_q + L.desc) + b * kChunkP;
    const unsigned char *tabs = smem_q + L.tab + (size_t)b * kChunkP * L.tab_bytes;
    const uint8_t *tips = smem_q + L.tips + (size_t)b * kChunkP * 2 * L.npb;
    for (int i = 0; i < nk; i++) {
      const DevOp &o = desc[i];
      const int w = o.pad_;
      const int lkind = plan_lkind(w), rkind = plan_rkind(w);
      const bool tiptip = lkind == GEMS_CHILD_TIP && rkind == GEMS_CHILD_TIP;
      const R *tk = tab + (size_t)(k0 + i) * stride;
      const unsigned char *tabS = tabs + (size_t)i * L.tab_bytes;
      int tbl[PP], tbr[PP];
#pragma unroll
      for (int u = 0; u < PP; u++) {
        tbl[u] = tbr[u] = 0;
        if (lkind == GEMS_CHILD_TIP)
          tbl[u] = tips_async ? tips[(size_t)(2 * i) * L.npb + toff[u]]
                              : c.tips[(size_t)o.l_id * c.P + p[u]];
        if (rkind == GEMS_CHILD_TIP)
          tbr[u] = tips_async ? tips[(size_t)(2 * i + 1) * L.npb + toff[u]]
                              : c.tips[(size_t)o.r_id * c.P + p[u]];
      }
      R vl[PP][4], vr[PP][4];
      int sl[PP], sr[PP];
      msg4q<R, SAFE, PP>(c, E, lkind, o.l_id, plan_lsrc(w), plan_lpos(w), stk, fwd, fwd_s, tabS,
                         tk, 0, tbl, p, gq, vl, sl);
      msg4q<R, SAFE, PP>(c, E, rkind, o.r_id, plan_rsrc(w), plan_rpos(w), stk, fwd, fwd_s, tabS,
                         tk, 1, tbr, p, gq, vr, sr);
      const int outk = plan_out(w), opos = min(plan_opos(w), max(depth - 1, 0));
#pragma unroll
      for (int u = 0; u < PP; u++) {
        R out[4];
        R lh_max = R(0);
        if constexpr (sizeof(R) == 4) {
#pragma unroll
          for (int x = 0; x < 4; x++) {
            out[x] = vl[u][x] * vr[u][x];
            lh_max = fmaxf(lh_max, out[x]);
          }
        } else {
          double tmp[4];
#pragma unroll
          for (int x = 0; x < 4; x++) tmp[x] = vl[u][x] * vr[u][x];
#pragma unroll
          for (int j = 0; j < 4; j++) {
            double acc = 0.0;
#pragma unroll
            for (int x = 0; x < 4; x++) acc = fma(E.inv[j * 4 + x], tmp[x], acc);
            out[j] = acc;
            lh_max = fmax(lh_max, fabs(acc));
          }
        }
        if (!act[u]) lh_max = R(0);
        if constexpr (!SAFE) {
          if constexpr (sizeof(R) == 4) lh_max = group_maxf(lh_max, G);
          else lh_max = group_max(lh_max, G);
        }
        int s_out = sl[u] + sr[u];
        bool thr;
        if constexpr (sizeof(R) == 4) thr = lh_max < kScaleThrF;
        else thr = lh_max < kScaleThr;
        if (act[u] && !tiptip && thr && c.invar[p[u]] == 0.0) {
#pragma unroll
          for (int x = 0; x < 4; x++) {
            if constexpr (sizeof(R) == 4) out[x] *= 18446744073709551616.0f;  // 2^64
            else out[x] = ldexp(out[x], kScaleExp);
          }
          s_out += 1;
        }
        if (act[u]) {
          if constexpr (sizeof(R) == 4) {
            __stcs(reinterpret_cast<float4 *>(part + (size_t)o.dst_slot * c.slot_elems +
                                              mix_off<4>(c, p[u], gl)),
                   make_float4(out[0], out[1], out[2], out[3]));
          } else {
            double *slot = part + (size_t)o.dst_slot * c.slot_elems;
            __stcs(reinterpret_cast<double2 *>(slot + f64_off<4>(c, p[u], gl, 0)),
                   make_double2(out[0], out[1]));
            __stcs(reinterpret_cast<double2 *>(slot + f64_off<4>(c, p[u], gl, 2)),
                   make_double2(out[2], out[3]));
          }
          uint16_t *sc = c.scale + (size_t)o.dst_slot * c.slot_scale;
          if (SAFE)
            sc[(size_t)p[u] * C + gl] = (uint16_t)s_out;
          else if (gl == 0)
            sc[p[u]] = (uint16_t)s_out;
        }
        if (outk == kSrcStack) stk.put(opos, u, out, s_out);
#pragma unroll
        for (int x = 0; x < 4; x++) fwd[u][x] = out[x];
        fwd_s[u] = s_out;
      }
    }
    __syncthreads();  // buffer b is refilled two chunks on
  }
}

inline int grid_for(const Session *s, int p0, int p1) {
  const long threads = (long)(p1 - p0) * s->G;
  return (int)((threads + kThreads - 1) / kThreads);
}

// ---------------------------------------------------------------------------------------
// Launch shapes of the 4-state kernels and their tuner.  A variant is (patterns per lane
// group, blocks per SM); all give the same values, so the choice only moves the time.  The
// first full traversal of a session class (precision, scaling, categories, pattern count to
// the power of two) with enough work times every variant once on its own op list and keeps
// the fastest for the process; smaller traversals and pattern ranges use the cached choice or
// the first variant (the measured best on the 512-taxon case).
// ---------------------------------------------------------------------------------------
struct Variant4 {
  int pp, blocks;
  const void *fn[2];  // [safe]
  bool stack;         // plan-driven kernel: takes the plan depth, dynamic smem
  size_t (*smem)(int depth, int C, int G);
  // one thread per pattern (k_traverse4p): kernels and shared memory by category count
  bool per_pattern = false;
  const void *fnC[2][4] = {};       // [safe][C = 1, 2, 4, 8]
  size_t (*smemC[4])(int depth) = {};
};
template <int PP, int B>
Variant4 mix_variant() {
  return {PP, B, {(const void *)k_traverse_mix4<false, PP, B>, (const void *)k_traverse_mix4<true, PP, B>},
          false, nullptr};
}
template <int PP, int B>
Variant4 f64_variant() {
  return {PP, B, {(const void *)k_traverse_f64x<false, PP, B>, (const void *)k_traverse_f64x<true, PP, B>},
          false, nullptr};
}
template <typename R, int PP>
size_t smem4q(int depth, int C, int G) {
  return StageQ(sizeof(R) == 8, C, kThreads / G * PP).stack + Stack4<R, PP>::bytes(depth);
}
template <typename R, int PP, int B>
Variant4 staged_variant() {
  return {PP, B,
          {(const void *)k_traverse4q<R, false, PP, B>, (const void *)k_traverse4q<R, true, PP, B>},
          true, &smem4q<R, PP>};
}
template <typename R, int C>
size_t smem4p(int depth) {
  return sizeof(StageP<R, C>) + StackP<R, C>::bytes(depth);
}
template <typename R>
Variant4 pattern_variant() {
  Variant4 v{1, 0, {nullptr, nullptr}, true, nullptr};
  v.per_pattern = true;
  const void *f[2][4] = {{(const void *)k_traverse4p<R, false, 1>, (const void *)k_traverse4p<R, false, 2>,
                          (const void *)k_traverse4p<R, false, 4>, (const void *)k_traverse4p<R, false, 8>},
                         {(const void *)k_traverse4p<R, true, 1>, (const void *)k_traverse4p<R, true, 2>,
                          (const void *)k_traverse4p<R, true, 4>, (const void *)k_traverse4p<R, true, 8>}};
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 4; b++) v.fnC[a][b] = f[a][b];
  v.smemC[0] = &smem4p<R, 1>;
  v.smemC[1] = &smem4p<R, 2>;
  v.smemC[2] = &smem4p<R, 4>;
  v.smemC[3] = &smem4p<R, 8>;
  return v;
}
int cat_index(int C) { return C == 1 ? 0 : C == 2 ? 1 : C == 4 ? 2 : C == 8 ? 3 : -1; }
const Variant4 *variants4(bool mixed, int *n) {
  static const Variant4 mix[] = {pattern_variant<float>(),        staged_variant<float, 2, 4>(),
                                 staged_variant<float, 1, 6>(),   mix_variant<2, 5>(),
                                 mix_variant<2, 6>(),             mix_variant<4, 3>(),
                                 mix_variant<1, 8>()};
  static const Variant4 f64[] = {pattern_variant<double>(),       staged_variant<double, 1, 4>(),
                                 staged_variant<double, 2, 3>(),  f64_variant<2, 4>(),
                                 f64_variant<3, 3>(),             f64_variant<1, 6>()};
  *n = mixed ? 7 : 6;
  return mixed ? mix : f64;
}
constexpr long long kTuneMinWork = 1ll << 22;  // patterns x ops below which no tuning is done
// the tuner times the plan-driven variants only (the first kTuned of each list); the kernels
// that read every child and table from global memory stay available by forcing their shape
constexpr int kTuned = 3;

std::mutex g_tune_mu;
std::map<std::array<int, 4>, int> g_tune;

std::array<int, 4> tune_key(const Session *s, bool mixed) {
  int b = 0;
  while (b < 30 && (1 << (b + 1)) <= s->P) b++;
  return {mixed ? 1 : 0, s->desc.scaling == GEMS_SCALE_SAFE ? 1 : 0, s->desc.ncat, b};
}
int tuned4(const Session *s, bool mixed) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  auto it = g_tune.find(tune_key(s, mixed));
  return it == g_tune.end() ? -1 : it->second;
}

// dynamic shared memory a kernel may take on a device: the opt-in maximum per block less the
// kernel's static shared memory.  Looked up once per (kernel, device), when the kernel's limit
// attribute is also raised to it (an attribute of the kernel, shared by every host thread), so
// that launches make no attribute calls.
std::mutex g_smem_mu;
std::map<std::pair<const void *, int>, size_t> g_smem;
size_t max_dyn_smem(const void *fn, int device, size_t want) {
  std::lock_guard<std::mutex> g(g_smem_mu);
  auto key = std::make_pair(fn, device);
  auto it = g_smem.find(key);
  if (it != g_smem.end()) return it->second;
  int optin = 0;
  cudaFuncAttributes fa{};
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) !=
          cudaSuccess ||
      cudaFuncGetAttributes(&fa, fn) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  const size_t lim = optin > (int)fa.sharedSizeBytes ? (size_t)optin - fa.sharedSizeBytes : 0;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)std::min(want, lim)) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  g_smem[key] = std::min(want, lim);
  return g_smem[key];
}

int launch4(Session *s, bool mixed, int v, int nops, int p0, int p1, const EigPack<4> *E) {
  int nv = 0;
  const Variant4 *all = variants4(mixed, &nv);
  const bool safe = s->desc.scaling == GEMS_SCALE_SAFE;
  const int ci = cat_index(s->desc.ncat);
  auto kernel = [&](const Variant4 &x) -> const void * {
    return x.per_pattern ? (ci >= 0 ? x.fnC[safe][ci] : nullptr) : x.fn[safe];
  };
  auto smem_of = [&](const Variant4 &x, int depth) -> size_t {
    return x.per_pattern ? x.smemC[ci](depth) : x.smem(depth, s->desc.ncat, s->G);
  };
  // a variant that cannot run this session (categories without an instance, a plan deeper than
  // its shared memory) hands over to the first variant that reads children from global memory
  auto usable = [&](const Variant4 &x) {
    if (!x.stack) return true;
    const void *f = kernel(x);
    return f && smem_of(x, s->plan_depth) <=
                    max_dyn_smem(f, s->desc.device, smem_of(x, kPlanMaxPos));
  };
  if (!usable(all[v])) {
    v = 0;
    while (v < nv && all[v].stack) v++;
  }
  const Variant4 &var = all[v];
  const void *fn = kernel(var);
  const int threads = var.per_pattern ? kThreadsP : kThreads;
  const long per = var.per_pattern ? kThreadsP : (long)(kThreads / s->G) * var.pp;
  const int grid = (int)((p1 - p0 + per - 1) / per);
  DevCtx c = s->ctx();
  const DevOp *ops = s->d_ops;
  size_t stride = s->op_stride;
  if (var.stack) {
    int depth = s->plan_depth;
    const size_t smem = smem_of(var, depth);
    EigPack<4> e{};
    if (E) e = *E;
    void *args[] = {&c, &ops, &nops, (void *)&s->d_opmats, &stride, &e, &p0, &p1, &depth};
    GEMS_CUDA(cudaLaunchKernel(fn, dim3(grid), dim3(threads), args, smem, s->stream));
  } else if (mixed) {
    const float *tab = reinterpret_cast<const float *>(s->d_opmats);
    void *args[] = {&c, &ops, &nops, &tab, &stride, &p0, &p1};
    GEMS_CUDA(cudaLaunchKernel(fn, dim3(grid), dim3(threads), args, 0, s->stream));
  } else {
    const double *tab = s->d_opmats;
    EigPack<4> e = *E;
    void *args[] = {&c, &ops, &nops, &tab, &stride, &e, &p0, &p1};
    GEMS_CUDA(cudaLaunchKernel(fn, dim3(grid), dim3(threads), args, 0, s->stream));
  }
  s->launches++;
  return GEMS_OK;
}

int shape4(const Session *s, bool mixed) {  // forced, tuned (-1: not yet), for this session
  int nv = 0;
  variants4(mixed, &nv);
  return s->force_shape >= 0 ? (s->force_shape < nv ? s->force_shape : nv - 1) : tuned4(s, mixed);
}

int traverse4(Session *s, bool mixed, int nops, int p0, int p1, const EigPack<4> *E) {
  int nv = 0;
  variants4(mixed, &nv);
  const int v = shape4(s, mixed);
  const bool tune = v < 0 && s->autotune && p0 == 0 && p1 == s->P &&
                    (long long)s->P * nops >= kTuneMinWork;
  if (!tune) return launch4(s, mixed, v < 0 ? 0 : v, nops, p0, p1, E);
  cudaEvent_t ev[2];
  GEMS_CUDA(cudaEventCreate(&ev[0]));
  if (cudaEventCreate(&ev[1]) != cudaSuccess) {
    cudaEventDestroy(ev[0]);
    return cuda_status(cudaErrorUnknown, "tuner events");
  }
  int best = 0, st = GEMS_OK;
  float best_ms = 0.f;
  for (int i = 0; i < std::min(nv, kTuned) && st == GEMS_OK; i++) {  // all write the same partials
    cudaEventRecord(ev[0], s->stream);
    st = launch4(s, mixed, i, nops, p0, p1, E);
    cudaEventRecord(ev[1], s->stream);
    float ms = 0.f;
    // another shape replaces the first (default) one only when it is more than 2% faster, so
    // that timing noise does not move the choice
    if (st == GEMS_OK && cudaEventSynchronize(ev[1]) == cudaSuccess &&
        cudaEventElapsedTime(&ms, ev[0], ev[1]) == cudaSuccess &&
        (i == 0 || ms < best_ms * (best == 0 ? 0.98f : 1.0f))) {
      best = i;
      best_ms = ms;
    }
  }
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  if (st) return st;
  std::lock_guard<std::mutex> g(g_tune_mu);
  g_tune[tune_key(s, mixed)] = best;
  return GEMS_OK;
}

template <int N>
int launch_f64(Session *s, int nops, int p0, int p1) {
  DevCtx c = s->ctx();
  EigPack<N> E;
  if (s->h_evec.size() != (size_t)N * N || s->h_inv.size() != (size_t)N * N) {
    set_error("eigensystem not set");
    return GEMS_ERR_STATE;
  }
  for (int i = 0; i < N * N; i++) {
    E.evec[i] = s->h_evec[i];
    E.inv[i] = s->h_inv[i];
  }
  const bool safe = s->desc.scaling == GEMS_SCALE_SAFE;
  if constexpr (N == 4) {
    return traverse4(s, false, nops, p0, p1, &E);
  } else {
    const int grid = grid_for(s, p0, p1);
    if (safe)
      k_traverse_f64<N, true><<<grid, kThreads, 0, s->stream>>>(c, s->d_ops, nops, s->d_opmats,
                                                                 s->op_stride, E, p0, p1);
    else
      k_traverse_f64<N, false><<<grid, kThreads, 0, s->stream>>>(c, s->d_ops, nops, s->d_opmats,
                                                                  s->op_stride, E, p0, p1);
  }
  s->launches++;
  GEMS_CUDA(cudaGetLastError());
  return GEMS_OK;
}

}  // namespace

bool traverse_v2_supported(const Session *s) {
  return s->desc.nstates == 4 || s->desc.nstates == 20;
}

int launch_prep_ops_v2(Session *s, int nops) {
  if (nops <= 0) return GEMS_OK;
  DevCtx c = s->ctx();
  if (s->desc.precision == GEMS_PREC_MIXED) {
    const size_t smem = sizeof(double) * s->block;
    k_prep_ops_mix<<<dim3(nops, 2), 256, smem, s->stream>>>(
        c, s->d_ops, reinterpret_cast<float *>(s->d_opmats), s->op_stride);
  } else {
    const size_t smem = sizeof(double) * s->block;
    k_prep_ops_f64<<<dim3(nops, 2), 256, smem, s->stream>>>(c, s->d_ops, s->d_opmats,
                                                             s->op_stride);
  }
  s->launches++;
  GEMS_CUDA(cudaGetLastError());
  return GEMS_OK;
}

int traverse_v2_wave_patterns(const Session *s) {
  const bool mixed = s->desc.precision == GEMS_PREC_MIXED;
  const bool safe = s->desc.scaling == GEMS_SCALE_SAFE;
  const bool four = s->desc.nstates == 4;
  int per_block = kThreads / s->G, threads = kThreads;
  size_t smem = 0;
  const void *fn = nullptr;
  if (four) {
    int nv = 0, v = shape4(s, mixed);
    const Variant4 &var = variants4(mixed, &nv)[v < 0 ? 0 : v];
    const int ci = cat_index(s->desc.ncat);
    if (var.per_pattern && ci >= 0) {
      fn = var.fnC[safe][ci];
      smem = var.smemC[ci](s->plan_depth);
      per_block = threads = kThreadsP;
    } else if (!var.per_pattern) {
      fn = var.fn[safe];
      per_block *= var.pp;
      if (var.stack) smem = var.smem(s->plan_depth, s->desc.ncat, s->G);
    } else {
      return 0;
    }
  } else {
    fn = mixed ? (safe ? (const void *)k_traverse_mix<20, true> : (const void *)k_traverse_mix<20, false>)
               : (safe ? (const void *)k_traverse_f64<20, true> : (const void *)k_traverse_f64<20, false>);
  }
  int nsm = 0, per_sm = 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, s->desc.device) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return per_sm * nsm * per_block;
}

int traverse_v2_shape(const Session *s, int *patterns_per_group, int *blocks_per_sm) {
  *patterns_per_group = 1;
  *blocks_per_sm = 0;
  if (s->desc.nstates != 4) return GEMS_OK;
  const bool mixed = s->desc.precision == GEMS_PREC_MIXED;
  int nv = 0, v = shape4(s, mixed);
  const Variant4 &var = variants4(mixed, &nv)[v < 0 ? 0 : v];
  *patterns_per_group = var.pp;
  *blocks_per_sm = var.blocks;
  const int ci = cat_index(s->desc.ncat);
  if (var.per_pattern && ci >= 0) {
    // one thread per pattern: the resident blocks follow from the plan's shared memory
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, var.fnC[s->desc.scaling == GEMS_SCALE_SAFE][ci], kThreadsP,
            var.smemC[ci](s->plan_depth)) == cudaSuccess)
      *blocks_per_sm = per_sm;
    else
      cudaGetLastError();
  }
  return v < 0 ? 1 : GEMS_OK;
}

int launch_traverse_v2(Session *s, int nops, int p0, int p1) {
  if (nops <= 0 || p1 <= p0) return GEMS_OK;
  cudaEvent_t ev0;
  if (int st = prof_begin(s, 0, &ev0)) return st;
  int st = GEMS_OK;
  if (s->desc.precision == GEMS_PREC_MIXED) {
    DevCtx c = s->ctx();
    const int grid = grid_for(s, p0, p1);
    const bool safe = s->desc.scaling == GEMS_SCALE_SAFE;
    const float *tab = reinterpret_cast<const float *>(s->d_opmats);
    if (s->desc.nstates == 4) {
      st = traverse4(s, true, nops, p0, p1, nullptr);
    } else {
      if (safe) k_traverse_mix<20, true><<<grid, kThreads, 0, s->stream>>>(c, s->d_ops, nops, tab, s->op_stride, p0, p1);
      else k_traverse_mix<20, false><<<grid, kThreads, 0, s->stream>>>(c, s->d_ops, nops, tab, s->op_stride, p0, p1);
      s->launches++;
      GEMS_CUDA(cudaGetLastError());
    }
  } else {
    st = s->desc.nstates == 4 ? launch_f64<4>(s, nops, p0, p1) : launch_f64<20>(s, nops, p0, p1);
  }
  if (st) return st;
  return prof_end(s, 0, ev0);
}

}  // namespace gems
