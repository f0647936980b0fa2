// Device primitives of the streamed persistent kernels: shared-memory
// mbarriers, bulk asynchronous global -> shared copies (cp.async.bulk, the
// non-tensor TMA path, no multicast), a nanosecond clock for bounded waits,
// and a grid-wide barrier for cooperative launches.
//
// Every wait here is bounded (HOEFEM_WAIT_NS): a wait that runs out reports
// failure to its caller, which records HOEFEM_ERR_DEVICE_TIMEOUT and winds the
// kernel down (copies in flight are waited for, again with a bound) instead of
// spinning forever.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace hoefem {
namespace pipe {

constexpr uint64_t HOEFEM_WAIT_NS = 2000000000ull;  // 2 s

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t clock_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Makes the initialised barriers visible to the async (bulk copy) proxy.
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// True once the phase with the given parity has completed.
__device__ __forceinline__ bool mbar_test(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for a phase; false if it did not complete within the bound or
// *stop became non-zero first (stop may be null).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, const volatile int* stop = nullptr) {
  if (mbar_test(bar, parity)) return true;
  const uint64_t t0 = clock_ns();
  for (;;) {
    if (mbar_test(bar, parity)) return true;
    if (stop && *stop) return false;
    if (clock_ns() - t0 > HOEFEM_WAIT_NS) return false;
  }
}

// Bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned) from
// this GPU's global memory into this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

// The same with an L2 eviction-priority policy (createpolicy value).
__device__ __forceinline__ void bulk_g2s_hint(void* dst, const void* src, unsigned bytes, uint64_t* bar,
                                              uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
      : "memory");
}

// L2 policies: keep the lines (evict last) or stream them (evict first).
__device__ __forceinline__ uint64_t policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}

// Named barrier over `nthreads` threads (a multiple of 32) of the CTA.
__device__ __forceinline__ void named_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Grid barrier of a cooperative launch (one leader thread per CTA, after the
// CTA's participating threads have synchronised): the leader adds to a
// counter whose top bit flips once every CTA has arrived (block 0 adds
// 2^31 - (G - 1), the others 1), then waits for the flip.  The add is a
// release at GPU scope (it orders the CTA's writes before the barrier, which
// the CTA barrier has ordered before the leader's add) and an acquire fence
// follows the flip, instead of two sequentially consistent fences.  Returns
// false if the flip did not come within the bound or *abort was raised (in
// which case it raises *abort itself so that every CTA winds down).
__device__ __forceinline__ bool grid_barrier_leader(unsigned* counter, int* abort_flag) {
  const unsigned inc = blockIdx.x == 0 ? (0x80000000u - (gridDim.x - 1u)) : 1u;
  unsigned old;
  asm volatile("atom.add.release.gpu.u32 %0, [%1], %2;" : "=r"(old) : "l"(counter), "r"(inc) : "memory");
  const uint64_t t0 = clock_ns();
  bool ok = true;
  for (;;) {
    const unsigned cur = *(volatile unsigned*)counter;
    if (((old ^ cur) & 0x80000000u) != 0u) break;
    if (*(volatile int*)abort_flag) {
      ok = false;
      break;
    }
    if (clock_ns() - t0 > HOEFEM_WAIT_NS) {
      atomicExch(abort_flag, 1);
      ok = false;
      break;
    }
  }
  asm volatile("fence.acq_rel.gpu;" ::: "memory");
  return ok;
}

}  // namespace pipe
}  // namespace hoefem
