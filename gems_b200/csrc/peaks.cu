// peaks.cu -- compute peaks of the GPU the session runs on, measured (not spec-sheet numbers):
// FP64 and FP32 FMA throughput of the CUDA cores, and the dense TF32 rate of the tcgen05 tensor
// cores (kind::tf32, M = 128, N = 256, K = 8, one CTA per SM).  These are the denominators of
// the compute rooflines of the 20- and 61-state kernels (the HBM denominator is a measured copy).
//
// Every loop is bounded, every shared-memory and TMEM access is inside the CTA's allocation,
// and the MMA completion wait gives up after a clock budget (reported as GEMS_ERR_TIMEOUT).
#include <cstdint>
#include <functional>
#include <string>

#include "gems_internal.cuh"

namespace gems {
namespace {

constexpr int kFmaChains = 8;

template <typename T>
__global__ void __launch_bounds__(256) k_fma_loop(int iters, T seed, T *out) {
  T a[kFmaChains];
#pragma unroll
  for (int j = 0; j < kFmaChains; j++) a[j] = seed + (T)(threadIdx.x + j);
  const T m = (T)0.999999, c = (T)1e-7;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int j = 0; j < kFmaChains; j++) a[j] = fma(a[j], m, c);
  }
  T s = 0;
#pragma unroll
  for (int j = 0; j < kFmaChains; j++) s += a[j];
  if (s == (T)-1) out[0] = s;  // never true; keeps the chains live
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// one CTA per SM: 12 MMAs of 128 x 256 x 8 per round, A and B zero tiles in shared memory
__global__ void __launch_bounds__(128, 1) k_tf32_loop(int rounds, long long *cycles, int *flag) {
  extern __shared__ __align__(1024) unsigned char sm[];
  constexpr int kA = 6 * 128 * 16, kB = 6 * 256 * 16;  // 3 K steps of 8 (2 chunks of 4)
  __shared__ uint64_t bar;
  __shared__ uint32_t tbase;
  const int t = threadIdx.x;
  for (int i = t; i < (kA + kB) / 16; i += blockDim.x)
    reinterpret_cast<float4 *>(sm)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (t < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(
                     smem_u32(&tbase))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tm = tbase;
  auto desc = [](uint32_t a, uint32_t lbo) {
    return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)(128 >> 4) << 32) | ((uint64_t)1 << 46);
  };
  const uint64_t da = desc(smem_u32(sm), 128 * 16), db = desc(smem_u32(sm + kA), 256 * 16);
  constexpr uint32_t idesc =
      (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(256 >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
  uint32_t ph = 0;
  bool ok = true;
  const long long t0 = clock64();
  for (int r = 0; r < rounds && ok; r++) {
    if (t < 32) {
      uint32_t pred = 0;
      asm volatile(
          "{\n\t.reg .pred P;\n\telect.sync _|P, 0xffffffff;\n\tselp.u32 %0, 1, 0, P;\n\t}\n"
          : "=r"(pred));
      if (pred) {
#pragma unroll
        for (int tile = 0; tile < 2; tile++)
#pragma unroll
          for (int ks = 0; ks < 3; ks++)
#pragma unroll
            for (int pr = 0; pr < 2; pr++) {
              const uint64_t ko = (uint64_t)((2 * ks * 128 * 16) >> 4);
              const uint64_t kb = (uint64_t)((2 * ks * 256 * 16) >> 4);
              asm volatile(
                  "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                  "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(
                      tm + tile * 256),
                  "l"(da + ko), "l"(db + kb), "r"(idesc), "r"((ks | pr) ? 1u : 0u)
                  : "memory");
            }
        asm volatile(
            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                smem_u32(&bar))
            : "memory");
      }
      __syncwarp();
    }
    const long long w0 = clock64();
    for (;;) {
      uint32_t done;
      asm volatile(
          "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
          "selp.u32 %0, 1, 0, p;\n\t}\n"
          : "=r"(done)
          : "r"(smem_u32(&bar)), "r"(ph)
          : "memory");
      if (done) break;
      if (clock64() - w0 > 2000000000LL) {
        ok = false;
        break;
      }
    }
    ph ^= 1;
    __syncthreads();
  }
  const long long t1 = clock64();
  if (!ok && t == 0) atomicExch(flag, 1);
  if (t == 0) cycles[blockIdx.x] = t1 - t0;
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (t < 32)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tm) : "memory");
}

int time_kernel_ms(cudaStream_t st, float *ms, const std::function<void()> &launch) {
  cudaEvent_t a, b;
  GEMS_CUDA(cudaEventCreate(&a));
  GEMS_CUDA(cudaEventCreate(&b));
  launch();  // warm-up
  GEMS_CUDA(cudaEventRecord(a, st));
  launch();
  GEMS_CUDA(cudaEventRecord(b, st));
  GEMS_CUDA(cudaEventSynchronize(b));
  GEMS_CUDA(cudaEventElapsedTime(ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return GEMS_OK;
}

}  // namespace
}  // namespace gems

using namespace gems;

extern "C" int gems_measure_peaks(int device, double *fp64_tflops, double *fp32_tflops,
                                  double *tf32_tflops) {
  if (!fp64_tflops || !fp32_tflops || !tf32_tflops) return GEMS_ERR_BAD_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    set_error("no CUDA device");
    return GEMS_ERR_NO_DEVICE;
  }
  GEMS_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  GEMS_CUDA(cudaGetDeviceProperties(&prop, device));
  const int sms = prop.multiProcessorCount;
  cudaStream_t st;
  GEMS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  double *d64 = nullptr;
  float *d32 = nullptr;
  long long *dcyc = nullptr;
  int *dflag = nullptr;
  int rc = GEMS_OK;
  auto cleanup = [&]() {
    cudaFree(d64);
    cudaFree(d32);
    cudaFree(dcyc);
    cudaFree(dflag);
    cudaStreamDestroy(st);
  };
  if (cudaMalloc(&d64, 8) != cudaSuccess || cudaMalloc(&d32, 8) != cudaSuccess ||
      cudaMalloc(&dcyc, sizeof(long long) * sms) != cudaSuccess ||
      cudaMalloc(&dflag, sizeof(int)) != cudaSuccess) {
    cleanup();
    set_error("peak measurement: out of device memory");
    return GEMS_ERR_OOM;
  }
  cudaMemsetAsync(dflag, 0, sizeof(int), st);
  const int blocks = sms * 8, threads = 256;
  const int it64 = 4096, it32 = 16384;
  float ms64 = 0, ms32 = 0, mstc = 0;
  rc = time_kernel_ms(st, &ms64, [&]() { k_fma_loop<double><<<blocks, threads, 0, st>>>(it64, 1.0, d64); });
  if (!rc)
    rc = time_kernel_ms(st, &ms32, [&]() { k_fma_loop<float><<<blocks, threads, 0, st>>>(it32, 1.f, d32); });
  const int smem = 200 * 1024;  // one CTA per SM (the kernel uses the first 36 KB)
  const int rounds = 400;
  if (!rc && cudaFuncSetAttribute(k_tf32_loop, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
                 cudaSuccess)
    rc = cuda_status(cudaGetLastError(), "cudaFuncSetAttribute");
  if (!rc)
    rc = time_kernel_ms(st, &mstc, [&]() { k_tf32_loop<<<sms, 128, smem, st>>>(rounds, dcyc, dflag); });
  int flag = 0;
  if (!rc) {
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, dflag, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = cuda_status(e, "peak measurement");
  }
  cleanup();
  if (rc) return rc;
  if (flag) {
    set_error("peak measurement: MMA wait expired");
    return GEMS_ERR_TIMEOUT;
  }
  *fp64_tflops = 2.0 * kFmaChains * (double)blocks * threads * it64 / (ms64 * 1e-3) / 1e12;
  *fp32_tflops = 2.0 * kFmaChains * (double)blocks * threads * it32 / (ms32 * 1e-3) / 1e12;
  *tf32_tflops = 2.0 * 12.0 * 128 * 256 * 8 * (double)rounds * sms / (mstc * 1e-3) / 1e12;
  return GEMS_OK;
}
