// Bulk asynchronous copies (TMA engine, untiled cp.async.bulk, no multicast)
// completing on shared-memory mbarriers, and bounded waits.
//
// Every wait here gives up after a clock budget and reports failure instead
// of spinning forever; callers record an error word for the host and drain
// their own copies (again bounded) before returning.
#pragma once
#include <stdint.h>

#include "pf_common.cuh"

namespace pf {

// ~1 s at 1.9 GHz
constexpr long long kWaitCycles = 2000000000LL;

enum DeviceError { kErrNone = 0, kErrWaitP2 = 2, kErrWaitP3 = 3 };

PF_D uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

PF_D void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

// make mbarrier initialisation visible to the async proxy
PF_D void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// order earlier generic-proxy accesses of shared memory before later
// async-proxy (bulk copy) writes to it
PF_D void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

PF_D void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// global -> shared bulk copy; dst, src 16-byte aligned, bytes a multiple of 16
PF_D void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

PF_D bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// true when the phase with this parity completed within the budget
PF_D bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > kWaitCycles) return false;
  }
  return true;
}

}  // namespace pf
