// noalloc.cu -- log-likelihood from a caller-owned theta buffer, without any allocation.
//
// Some callers cannot allocate device memory at the point they need a likelihood:
//  * a host application whose own memory pool has reserved (nearly) all of the device, so a
//    library cudaMalloc either fails or steals from the pool's budget behind its back;
//  * an embedding that accounts every device byte itself (a serving process with a fixed
//    per-tenant budget) and forbids libraries from allocating outside that accounting;
//  * a tight evaluation loop that must not touch the allocator, because cudaMalloc and
//    cudaFree synchronise the device and would stall the other streams on every evaluation.
// gems_lnl_from_theta_noalloc serves them: it evaluates the same sum as gems_lnl_from_buffer
// (theta . exp(eval r_c t) prop_c per pattern, |.| + invar, log, + scale, weighted by the
// pattern counts) over buffers the caller already owns, and keeps its only scratch -- the
// per-CTA partial sums of the deterministic two-level reduction -- in a fixed file-scope device
// array instead of allocating it.  The call is synchronous: it waits for its stream and returns
// the lnL on the host.
//
// The scratch array holds kNoAllocMaxBlocks pairs of doubles plus the two final sums
// (256 KiB + 16 B).  Every GPU that loads this library holds it until the process exits.  A
// call needs one pair per CTA of 256 threads, and a CTA covers 256 / G patterns
// (G = the smallest power of two >= ncat), so nptn is limited to kNoAllocMaxBlocks * 256 / G
// (4,194,304 patterns for 1 category, 1,048,576 for 4, 524,288 for 8); larger calls are
// rejected with GEMS_ERR_BAD_ARG before anything is launched.
//
// Every call shares the one array and it keeps the last call's contents.  Each call writes
// every slot it reads before reading it (one pair per CTA of this call, then the final pair),
// so nothing has to start at zero.  Calls whose kernels overlap on the GPU (different streams,
// or different host threads on one device) race on the array and must be serialised by the
// caller.
//
// Host code does not use the array's name as a device address: on the first call on a device
// (with that device current) the address is looked up once with cudaGetSymbolAddress and cached
// per device.  That first call should therefore come before any stream capture on that device.
// The cached address belongs to the device's primary context: after cudaDeviceReset the
// library's device state (sessions and this address alike) is gone and the library must not be
// used again in that process.
#include <cmath>
#include <mutex>

#include "gems_internal.cuh"

namespace gems {

namespace {

constexpr int kThreadsNa = 256;
constexpr int kNoAllocMaxBlocks = 16384;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[2 * kNoAllocMaxBlocks + 2];

struct ModelPack {
  double eval[kMaxStates];
  double rates[kMaxCat];
  double props[kMaxCat];
};

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

// per-CTA sums of freq * pattern lnL (raw, and with non-finite values clamped to
// 4 log(2^-256)) into scratch[2 * blockIdx.x .. +1]
__global__ void __launch_bounds__(kThreadsNa) k_lnl_theta_na(
    const double *__restrict__ theta, const double *__restrict__ scale_all,
    const double *__restrict__ freq, const double *__restrict__ invar, int nptn, int n, int C,
    int G, double t, const ModelPack m, double *scratch) {
  __shared__ double val[kMaxStates * kMaxCat];
  __shared__ double sh[2][32];
  const int blk = n * C;
  for (int idx = threadIdx.x; idx < blk; idx += blockDim.x) {
    const int cc = idx / n, i = idx - cc * n;
    val[idx] = exp(m.eval[i] * m.rates[cc] * t) * m.props[cc];
  }
  __syncthreads();
  const int gl = threadIdx.x & (G - 1);
  const long p = ((long)blockIdx.x * blockDim.x + threadIdx.x) / G;
  const bool act = p < nptn && gl < C;
  double lh = 0.0;
  if (act) {
    const double *th = theta + (size_t)p * blk + (size_t)gl * n;
    for (int i = 0; i < n; i++) lh = fma(val[gl * n + i], th[i], lh);
  }
  for (int o = 1; o < G; o <<= 1) lh += __shfl_xor_sync(0xffffffffu, lh, o);
  double v[2] = {0.0, 0.0};
  if (act && gl == 0) {
    const double l = fabs(lh) + (invar ? invar[p] : 0.0);
    const double plh = log(fabs(l)) + scale_all[p];
    const double f = freq[p];
    v[0] = plh * f;
    v[1] = (isfinite(plh) ? plh : 4.0 * kLogScaleThr) * f;
  }
  block_sum<2>(v, sh);
  if (threadIdx.x == 0) {
    scratch[2 * blockIdx.x] = v[0];
    scratch[2 * blockIdx.x + 1] = v[1];
  }
}

// sums the per-CTA pairs in index order into scratch[2 * nblk .. +1]
__global__ void k_lnl_theta_na_final(double *scratch, int nblk) {
  __shared__ double sh[2][32];
  double v[2] = {0.0, 0.0};
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
    v[0] += scratch[2 * b];
    v[1] += scratch[2 * b + 1];
  }
  block_sum<2>(v, sh);
  if (threadIdx.x == 0) {
    scratch[2 * nblk] = v[0];
    scratch[2 * nblk + 1] = v[1];
  }
}

std::mutex g_na_mutex;
double *g_na_ptr[kMaxDevices] = {};

// device address of the scratch array on the current device (looked up once per device)
int noalloc_scratch(double **out) {
  int dev = -1;
  GEMS_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("device ordinal out of range for the allocation-free entry point");
    return GEMS_ERR_BAD_ARG;
  }
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if (!g_na_ptr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    g_na_ptr[dev] = static_cast<double *>(p);
  }
  *out = g_na_ptr[dev];
  return GEMS_OK;
}

}  // namespace

}  // namespace gems

using namespace gems;

extern "C" int gems_lnl_from_theta_noalloc(const double *theta, const double *scale_all,
                                           const double *freq, const double *invar, int nptn,
                                           int nstates, int ncat, const double *eval,
                                           const double *rates, const double *props,
                                           double length, void *stream, double *lnl) {
  if (!theta || !scale_all || !freq || !eval || !rates || !props || !lnl || nptn < 1 ||
      nstates < 2 || nstates > kMaxStates || ncat < 1 || ncat > kMaxCat || !(length >= 0)) {
    set_error("gems_lnl_from_theta_noalloc: invalid argument");
    return GEMS_ERR_BAD_ARG;
  }
  int G = 1;
  while (G < ncat) G <<= 1;
  const long long threads = (long long)nptn * G;
  const long long nblk = (threads + kThreadsNa - 1) / kThreadsNa;
  if (nblk > kNoAllocMaxBlocks) {
    set_error("gems_lnl_from_theta_noalloc: nptn exceeds the fixed scratch (at most 16384 "
              "CTAs of 256 threads, i.e. 4194304 / G patterns)");
    return GEMS_ERR_BAD_ARG;
  }
  double *scratch = nullptr;
  int st = noalloc_scratch(&scratch);
  if (st) return st;
  ModelPack m{};
  for (int i = 0; i < nstates; i++) m.eval[i] = eval[i];
  for (int c = 0; c < ncat; c++) {
    m.rates[c] = rates[c];
    m.props[c] = props[c];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_lnl_theta_na<<<(unsigned)nblk, kThreadsNa, 0, s>>>(theta, scale_all, freq, invar, nptn,
                                                       nstates, ncat, G, length, m, scratch);
  GEMS_CUDA(cudaGetLastError());
  k_lnl_theta_na_final<<<1, 256, 0, s>>>(scratch, (int)nblk);
  GEMS_CUDA(cudaGetLastError());
  double out[2];
  GEMS_CUDA(cudaMemcpyAsync(out, scratch + 2 * nblk, sizeof(out), cudaMemcpyDeviceToHost, s));
  GEMS_CUDA(cudaStreamSynchronize(s));
  // non-finite total: clamp non-finite pattern values (tree/phylokernelnew.h:3441-3450)
  *lnl = std::isfinite(out[0]) ? out[0] : out[1];
  return GEMS_OK;
}
