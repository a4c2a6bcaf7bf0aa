// kernels_rell.cu -- bootstrap reweighting (RELL) of resident per-pattern terms.
//
// UFBoot evaluates each bootstrap replicate r as a dot product of the per-pattern
// log-likelihoods with the replicate's pattern counts (tree/iqtree.cpp:3870-3916 with
// PhyloTree::dotProductSIMD, tree/phylokernel.h:65; the reference casts pattern_lh to float
// and accumulates in float).  Here the R x P count matrix is resident in HBM and one launch
// evaluates every replicate: CTA r streams row r (FP32 counts) against the resident pattern
// terms and reduces in a fixed order (deterministic).  The same machinery gives reweighted
// first and second derivatives from the terms the derivative kernel leaves behind
// (df_frac_p and ddf_frac_p - df_frac_p^2), i.e. one [R x P] . [P x 2] product.
#include <cmath>

#include "gems_internal.cuh"

namespace gems {

namespace {

constexpr int kThreads = 512;

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

// lnl[r] = sum_p w[r][p] * (float)pattern_lh[p]
__global__ void __launch_bounds__(kThreads) k_rell_lnl(const float *__restrict__ w,
                                                       const double *__restrict__ plh, int nptn,
                                                       size_t ld, double *out) {
  __shared__ double sh[1][32];
  const float *row = w + (size_t)blockIdx.x * ld;
  double v[1] = {0.0};
  const int n4 = nptn / 4;
  const float4 *r4 = reinterpret_cast<const float4 *>(row);
  for (int i = threadIdx.x; i < n4; i += blockDim.x) {
    const float4 a = __ldcs(r4 + i);
    const int p = 4 * i;
    v[0] += (double)a.x * (double)(float)plh[p] + (double)a.y * (double)(float)plh[p + 1] +
            (double)a.z * (double)(float)plh[p + 2] + (double)a.w * (double)(float)plh[p + 3];
  }
  for (int p = 4 * n4 + threadIdx.x; p < nptn; p += blockDim.x)
    v[0] += (double)row[p] * (double)(float)plh[p];
  block_sum<1>(v, sh);
  if (threadIdx.x == 0) out[blockIdx.x] = v[0];
}

// df[r] = sum_p w[r][p] df_frac[p],  ddf[r] = sum_p w[r][p] ddf_term[p]
__global__ void __launch_bounds__(kThreads) k_rell_derv(const float *__restrict__ w,
                                                        const double *__restrict__ dfr,
                                                        const double *__restrict__ ddt, int nptn,
                                                        size_t ld, double *out) {
  __shared__ double sh[2][32];
  const float *row = w + (size_t)blockIdx.x * ld;
  double v[2] = {0.0, 0.0};
  for (int p = threadIdx.x; p < nptn; p += blockDim.x) {
    const double wp = (double)__ldcs(row + p);
    v[0] = fma(wp, dfr[p], v[0]);
    v[1] = fma(wp, ddt[p], v[1]);
  }
  block_sum<2>(v, sh);
  if (threadIdx.x == 0) {
    out[2 * blockIdx.x] = v[0];
    out[2 * blockIdx.x + 1] = v[1];
  }
}

}  // namespace

int launch_rell_lnl(Session *s, double *d_out) {
  if (!s->d_rell_w || s->rell_R <= 0) {
    set_error("no reweightings uploaded");
    return GEMS_ERR_STATE;
  }
  cudaEvent_t ev0;
  if (int st = prof_begin(s, 6, &ev0)) return st;
  k_rell_lnl<<<s->rell_R, kThreads, 0, s->stream>>>(s->d_rell_w, s->d_pattern_lh, s->desc.nptn,
                                                     s->rell_ld, d_out);
  s->launches++;
  GEMS_CUDA(cudaGetLastError());
  return prof_end(s, 6, ev0);
}

int launch_rell_derv(Session *s, double *d_out) {
  if (!s->d_rell_w || s->rell_R <= 0) {
    set_error("no reweightings uploaded");
    return GEMS_ERR_STATE;
  }
  k_rell_derv<<<s->rell_R, kThreads, 0, s->stream>>>(s->d_rell_w, s->d_df_frac, s->d_ddf_term,
                                                      s->desc.nptn, s->rell_ld, d_out);
  s->launches++;
  GEMS_CUDA(cudaGetLastError());
  return GEMS_OK;
}

}  // namespace gems
