// kernels_rell.cu -- bootstrap reweighting (RELL) of resident per-pattern terms.
//
// UFBoot evaluates each bootstrap replicate r as a dot product of the per-pattern
// log-likelihoods with the replicate's pattern counts (tree/iqtree.cpp:3870-3916 with
// PhyloTree::dotProductSIMD, tree/phylokernel.h:65; the reference casts pattern_lh to float).
// Here the R x P count matrix is resident in HBM and one launch evaluates every replicate as a
// tiled GEMV: CTA (chunk, group) stages its chunk of the pattern terms in shared memory once
// (as float for the lnL, as the reference's BootValType) and applies it to a group of replicate
// rows, one warp per row streaming float4 counts; each (row, chunk) partial sum lands in a
// scratch row, and a second kernel adds a row's partials in chunk order (deterministic).  The
// same tiling gives reweighted first and second derivatives from the terms the derivative
// kernel leaves behind (df_frac_p and ddf_frac_p - df_frac_p^2): one [R x P] . [P x 2] product.
// Algorithmic bytes: the R x P FP32 counts once, the pattern terms once per row group.
#include <cmath>

#include "gems_internal.cuh"

namespace gems {

namespace {

constexpr int kRellChunkLnl = 4096;   // patterns per CTA, lnL (16 KB of float terms)
constexpr int kRellChunkDerv = 2048;  // patterns per CTA, derivatives (32 KB of double terms)

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

constexpr int kRellThreads = 256;  // 8 warps
constexpr int kRellRows = 32;      // replicate rows per CTA (4 per warp)

__device__ __forceinline__ double warp_sum(double x) {
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  return x;
}

// part[r * nchunk + chunk] = sum over the chunk's patterns of w[r][p] * (float)plh[p]
__global__ void __launch_bounds__(kRellThreads) k_rell_lnl(const float *__restrict__ w,
                                                           const double *__restrict__ plh,
                                                           int nptn, size_t ld, int R,
                                                           double *__restrict__ part,
                                                           int nchunk) {
  __shared__ __align__(16) float sp[kRellChunkLnl];
  const long base = (long)blockIdx.x * kRellChunkLnl;
  const int n = (int)min((long)kRellChunkLnl, nptn - base);
  for (int i = threadIdx.x; i < kRellChunkLnl; i += blockDim.x)
    sp[i] = i < n ? (float)plh[base + i] : 0.f;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n4 = (n + 3) / 4;  // rows are zero past nptn up to ld (a multiple of 64)
  const float4 *s4 = reinterpret_cast<const float4 *>(sp);
  for (int rr = warp; rr < kRellRows; rr += kRellThreads / 32) {
    const int r = blockIdx.y * kRellRows + rr;
    if (r >= R) break;
    const float4 *row = reinterpret_cast<const float4 *>(w + (size_t)r * ld + base);
    double acc = 0.0;
#pragma unroll 8
    for (int i = lane; i < n4; i += 32) {
      const float4 a = __ldcs(row + i), b = s4[i];
      acc = fma((double)a.x, (double)b.x, acc);
      acc = fma((double)a.y, (double)b.y, acc);
      acc = fma((double)a.z, (double)b.z, acc);
      acc = fma((double)a.w, (double)b.w, acc);
    }
    acc = warp_sum(acc);
    if (lane == 0) part[(size_t)r * nchunk + blockIdx.x] = acc;
  }
}

// part[(2 r) * nchunk + chunk] = sum w[r][p] df_frac[p], part[(2 r + 1) * nchunk + chunk] =
// sum w[r][p] ddf_term[p] over the chunk's patterns
__global__ void __launch_bounds__(kRellThreads) k_rell_derv(const float *__restrict__ w,
                                                            const double *__restrict__ dfr,
                                                            const double *__restrict__ ddt,
                                                            int nptn, size_t ld, int R,
                                                            double *__restrict__ part,
                                                            int nchunk) {
  __shared__ __align__(16) double sd[2][kRellChunkDerv];
  const long base = (long)blockIdx.x * kRellChunkDerv;
  const int n = (int)min((long)kRellChunkDerv, nptn - base);
  for (int i = threadIdx.x; i < kRellChunkDerv; i += blockDim.x) {
    sd[0][i] = i < n ? dfr[base + i] : 0.0;
    sd[1][i] = i < n ? ddt[base + i] : 0.0;
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n4 = (n + 3) / 4;
  for (int rr = warp; rr < kRellRows; rr += kRellThreads / 32) {
    const int r = blockIdx.y * kRellRows + rr;
    if (r >= R) break;
    const float4 *row = reinterpret_cast<const float4 *>(w + (size_t)r * ld + base);
    double a0 = 0.0, a1 = 0.0;
#pragma unroll 4
    for (int i = lane; i < n4; i += 32) {
      const float4 a = __ldcs(row + i);
      const int q = 4 * i;
      a0 = fma((double)a.x, sd[0][q], a0);
      a1 = fma((double)a.x, sd[1][q], a1);
      a0 = fma((double)a.y, sd[0][q + 1], a0);
      a1 = fma((double)a.y, sd[1][q + 1], a1);
      a0 = fma((double)a.z, sd[0][q + 2], a0);
      a1 = fma((double)a.z, sd[1][q + 2], a1);
      a0 = fma((double)a.w, sd[0][q + 3], a0);
      a1 = fma((double)a.w, sd[1][q + 3], a1);
    }
    a0 = warp_sum(a0);
    a1 = warp_sum(a1);
    if (lane == 0) {
      part[(size_t)(2 * r) * nchunk + blockIdx.x] = a0;
      part[(size_t)(2 * r + 1) * nchunk + blockIdx.x] = a1;
    }
  }
}

// out[k] = sum over chunks of part[k * nchunk + chunk], one CTA per output, fixed order
__global__ void k_rell_final(const double *__restrict__ part, int nchunk, double *out) {
  __shared__ double sh[1][32];
  double v[1] = {0.0};
  const double *row = part + (size_t)blockIdx.x * nchunk;
  for (int i = threadIdx.x; i < nchunk; i += blockDim.x) v[0] += row[i];
  block_sum<1>(v, sh);
  if (threadIdx.x == 0) out[blockIdx.x] = v[0];
}

}  // namespace

size_t rell_scratch_doubles(int R, int P) {
  return (size_t)2 * R * ((P + kRellChunkDerv - 1) / kRellChunkDerv);
}

int launch_rell_lnl(Session *s, double *d_out) {
  if (!s->d_rell_w || s->rell_R <= 0) {
    set_error("no reweightings uploaded");
    return GEMS_ERR_STATE;
  }
  const int nptn = s->desc.nptn, R = s->rell_R;
  const int nchunk = (nptn + kRellChunkLnl - 1) / kRellChunkLnl;
  cudaEvent_t ev0;
  if (int st = prof_begin(s, 6, &ev0)) return st;
  k_rell_lnl<<<dim3(nchunk, (R + kRellRows - 1) / kRellRows), kRellThreads, 0, s->stream>>>(
      s->d_rell_w, s->d_pattern_lh, nptn, s->rell_ld, R, s->d_rell_part, nchunk);
  s->launches++;
  GEMS_CUDA(cudaGetLastError());
  k_rell_final<<<R, 128, 0, s->stream>>>(s->d_rell_part, nchunk, d_out);
  s->launches++;
  GEMS_CUDA(cudaGetLastError());
  return prof_end(s, 6, ev0);
}

int launch_rell_derv(Session *s, double *d_out) {
  if (!s->d_rell_w || s->rell_R <= 0) {
    set_error("no reweightings uploaded");
    return GEMS_ERR_STATE;
  }
  const int nptn = s->desc.nptn, R = s->rell_R;
  const int nchunk = (nptn + kRellChunkDerv - 1) / kRellChunkDerv;
  k_rell_derv<<<dim3(nchunk, (R + kRellRows - 1) / kRellRows), kRellThreads, 0, s->stream>>>(
      s->d_rell_w, s->d_df_frac, s->d_ddf_term, nptn, s->rell_ld, R, s->d_rell_part, nchunk);
  s->launches++;
  GEMS_CUDA(cudaGetLastError());
  // outputs 2r (df) and 2r + 1 (ddf), as the host reads them
  k_rell_final<<<2 * R, 128, 0, s->stream>>>(s->d_rell_part, nchunk, d_out);
  s->launches++;
  GEMS_CUDA(cudaGetLastError());
  return GEMS_OK;
}

}  // namespace gems
