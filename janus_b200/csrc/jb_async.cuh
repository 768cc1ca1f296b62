// Asynchronous bulk copies between global and shared memory (the TMA engine's
// non-tensor form, cp.async.bulk) completed on an mbarrier, for sm_100a.
//
// Every copy lands in the issuing CTA's own shared memory (no copy is shared
// across the CTAs of a cluster).  Every wait is bounded: after
// c_jb_wait_first polls (kWaitLimit by default) the kernel records a timeout
// in g_jb_fault (read by the solvers at each host synchronisation and by
// jb_device_status), waits once more, at most kWaitLimit polls, for its own
// copies, and the caller returns without touching the tile.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace jb {

// set by kernels whose bounded wait ran out (bit 0); read and cleared on the
// host by jb_device_status.  Defined here: include this header from exactly
// one translation unit (jb_kernels.cu).
__device__ unsigned int g_jb_fault = 0;

constexpr unsigned kWaitLimit = 1u << 24;

// polls of the first bounded wait (kWaitLimit unless lowered through
// jb_set_wait_limit to exercise the failure path in tests, 0: give up at
// once; the drain wait after a timeout always keeps kWaitLimit)
__constant__ unsigned c_jb_wait_first = kWaitLimit;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

// make the barrier initialisation visible to the async (TMA) proxy
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
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

// bounded wait for phase `parity` of the barrier; false on timeout (and the
// fault bit is set)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const unsigned first = c_jb_wait_first;
  for (unsigned i = 0; i < first; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  atomicOr(&g_jb_fault, 1u);
  for (unsigned i = 0; i < kWaitLimit; ++i)
    if (mbar_try_wait(bar, parity)) break;
  return false;
}

// global -> shared, `bytes` a multiple of 16, both addresses 16-byte aligned
// hint: bring the 128-byte line holding p into L1 (no effect on results)
__device__ __forceinline__ void prefetch_l1(const void* p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

__device__ __forceinline__ void bulk_load(void* sdst, const void* gsrc, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_u32(sdst)), "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// shared -> global, same alignment rules; completes in the thread's bulk group
__device__ __forceinline__ void bulk_store(void* gdst, const void* ssrc, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst),
               "r"(smem_u32(ssrc)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// wait until the shared-memory sources of this thread's bulk stores are read
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// the same, for all but the most recently committed group
__device__ __forceinline__ void bulk_wait_read_1() {
  asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
}

// order this thread's generic-proxy shared-memory writes before later
// async-proxy (bulk copy) accesses
__device__ __forceinline__ void fence_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// tiled tensor copies (TMA) through a CUtensorMap kernel parameter, into or
// out of this CTA's shared memory only.  The box's innermost coordinate x
// times the element size is a multiple of 16 bytes at every call site.
__device__ __forceinline__ void tma_load_3d(void* sdst, const CUtensorMap* map, int x, int y,
                                            int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(smem_u32(sdst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z),
      "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, int x, int y, int z,
                                             const void* ssrc) {
  asm volatile(
      "cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];"
      ::"l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(ssrc))
      : "memory");
}

__device__ __forceinline__ bool aligned16(const void* p) {
  return (reinterpret_cast<uintptr_t>(p) & 15u) == 0;
}

}  // namespace jb
