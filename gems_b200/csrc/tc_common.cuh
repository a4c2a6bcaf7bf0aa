// tc_common.cuh -- PTX wrappers shared by the tcgen05 traversal kernels (20 and 61 states):
// mbarriers with bounded waits, bulk copies, UMMA shared-memory descriptors, tcgen05.mma
// kind::tf32 (A in shared or tensor memory), commit, fences, lane election, TMEM stores, and
// the TF32 hi/lo split.
#pragma once

#include <cstdint>

namespace gems {
namespace tc {

constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at 1.9 GHz: every wait gives up after it

__device__ __forceinline__ uint32_t sptr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t cnt) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(cnt) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
// false when the phase did not complete within the clock budget
__device__ inline bool mbar_wait(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > kWaitCycles) return false;
  return true;
}
// a bounded wait that also gives up once another part of the CTA has failed (*err set)
__device__ __forceinline__ bool ws_wait(uint32_t bar, uint32_t parity, const int *err) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (*(const volatile int *)err) return false;
    if (clock64() - t0 > kWaitCycles) return false;
  }
  return true;
}
// a counter in shared memory published by one thread (release) and polled by others (acquire)
__device__ __forceinline__ int ld_acquire_s(const int *p) {
  int v;
  asm volatile("ld.acquire.cta.shared::cta.u32 %0, [%1];" : "=r"(v) : "r"(sptr(p)) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_s(int *p, int v) {
  asm volatile("st.release.cta.shared::cta.u32 [%0], %1;" ::"r"(sptr(p)), "r"(v) : "memory");
}
// bounded wait until the counter reaches `need` (false on expiry or once *err is set)
__device__ __forceinline__ bool wait_count(const int *cnt, int need, const int *err) {
  const long long t0 = clock64();
  while (ld_acquire_s(cnt) < need)
    if (*(const volatile int *)err || clock64() - t0 > kWaitCycles) return false;
  return true;
}
// OR of `pred` over the NT threads that use named barrier BAR (all of them wait for all)
template <int BAR, int NT>
__device__ __forceinline__ bool bar_or(bool pred) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)pred), "n"(BAR), "n"(NT)
      : "memory");
  return r != 0;
}
template <int BAR, int NT>
__device__ __forceinline__ void bar_sync() {
  asm volatile("bar.sync %0, %1;" ::"n"(BAR), "n"(NT) : "memory");
}
// contiguous global -> shared copy completing on an mbarrier (16-byte aligned, size % 16 == 0)
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes,
                                         uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}
// contiguous shared -> global copy in a bulk async-group (16-byte aligned, size % 16 == 0);
// bulk_commit closes the group, bulk_wait<N> waits until at most N groups are incomplete
// (writes performed), bulk_wait_read<N> until at most N groups still read shared memory
__device__ __forceinline__ void bulk_s2g(void *dst, uint32_t src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(src),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void bulk_wait() {
  asm volatile("cp.async.bulk.wait_group %0;" ::"n"(N) : "memory");
}
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
// UMMA shared-memory descriptor, K-major, no swizzle (Blackwell version field = 1)
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}
// instruction descriptor: D f32, A/B tf32, both K-major, M = 128, N given
__host__ __device__ constexpr uint32_t idesc_tf32(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(128 >> 4) << 24);
}
// D (TMEM) (+)= A (shared, descriptor) . B (shared, descriptor)
__device__ __forceinline__ void mma_ss(uint32_t dtm, uint64_t a, uint64_t b, uint32_t idesc,
                                       uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtm),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
// same, A read from tensor memory (lane = row, one column per K element)
__device__ __forceinline__ void mma_ts(uint32_t dtm, uint32_t atm, uint64_t b, uint32_t idesc,
                                       uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(dtm),
      "r"(atm), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   bar)
               : "memory");
}
// one lane of a converged warp (the MMA and copy instructions are issued by a single thread;
// issuing them from a warp-uniform branch keeps their operands in uniform registers)
__device__ __forceinline__ bool elect_one() {
  uint32_t pred = 0;
  asm volatile(
      "{\n\t.reg .pred P;\n\telect.sync _|P, 0xffffffff;\n\tselp.u32 %0, 1, 0, P;\n\t}\n"
      : "=r"(pred));
  return pred != 0;
}
__device__ __forceinline__ void fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_st_wait() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem),
               "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t tmem, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols)
               : "memory");
}
// Round a finite FP32 value to TF32 (10 fraction bits), to nearest with ties away from zero:
// adding half a TF32 ulp (bit 12) to the sign-magnitude bits and clearing the 13 low bits
// rounds the magnitude up exactly when the dropped bits are at least half an ulp (a carry
// into the exponent gives the next binade correctly).  Two integer operations.
__device__ __forceinline__ float tf32_rna(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}
__device__ __forceinline__ void split4(float4 v, float4 &h, float4 &l) {
  h = make_float4(tf32_rna(v.x), tf32_rna(v.y), tf32_rna(v.z), tf32_rna(v.w));
  l = make_float4(tf32_rna(v.x - h.x), tf32_rna(v.y - h.y), tf32_rna(v.z - h.z),
                  tf32_rna(v.w - h.w));
}

}  // namespace tc
}  // namespace gems
