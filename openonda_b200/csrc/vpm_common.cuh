// vpm_common.cuh -- shared device helpers for the VPM pair-sum kernels (sm_100a).
//
// * Packed particle record: {x, y, z, sigma | ax, ay, az, nu} in the compute precision
//   (64 B).  A tile of consecutive records is one contiguous byte range, so it moves into
//   shared memory with a single bulk-async (TMA) copy.
// * Bulk-async copy global -> shared completing on an mbarrier (cp.async.bulk, no
//   multicast: every load reads this GPU's own memory).
// * mbarrier waits are bounded by %globaltimer: after VPM_WAIT_LIMIT_NS the wait gives up,
//   records VPM_DEVERR_WAIT_TIMEOUT in the device error word and the caller unwinds.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace vpm {

constexpr double kPi = 3.14159265358979323846;
constexpr double kOneOver4Pi = 1.0 / (4.0 * kPi);
constexpr double kRefEps = 1e-8;  // ParticlesPhysicsCuda.py:6

// Device-side error bits (read by vpm_device_errors()).
constexpr int VPM_DEVERR_WAIT_TIMEOUT = 1;
constexpr int VPM_DEVERR_NONUNIFORM_CORE = 2;

constexpr unsigned long long VPM_WAIT_LIMIT_NS = 1000000000ull;  // 1 s

// Packed particle record.  E = double (FP64 path) or float2 (FP32 path, every value stored
// twice as {v, v} so a 16-byte shared-memory load yields two broadcast operand pairs for the
// paired FP32 instructions).  Both forms are 64 bytes.
template <class E>
struct alignas(16) Rec {
  E x, y, z, s;
  E ax, ay, az, nu;
};
static_assert(sizeof(Rec<double>) == 64, "FP64 record is 64 B");
static_assert(sizeof(Rec<float2>) == 64, "FP32 record is 64 B");

// Device error word.  The library is compiled as one translation unit (vpm_abi.cu
// includes every kernel header), so this is the only instance.
__device__ int g_device_errors = 0;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Wait for phase `parity` of `bar`; false (and the device error bit set) after the limit.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_timer_ns();
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_timer_ns() - t0 > VPM_WAIT_LIMIT_NS) {
      atomicOr(&g_device_errors, VPM_DEVERR_WAIT_TIMEOUT);
      return false;
    }
  }
}

// Bulk-async copy of `bytes` (multiple of 16, both addresses 16-byte aligned) from global
// memory of this GPU into this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_load_g2s(void* smem_dst, const void* gmem_src,
                                              uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_addr(smem_dst)), "l"(gmem_src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

}  // namespace vpm
