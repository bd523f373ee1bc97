// Bulk asynchronous global -> shared copies (the TMA unit's 1D "cp.async.bulk" path) completed
// through shared-memory mbarriers, for sm_100a.  No cluster multicast is used anywhere.
//
// Every wait is bounded: after kWaitLimit polls (each may suspend the thread for up to
// kWaitHintNs while the phase is incomplete) the waiting thread records a timeout in the kernel's
// error word and the kernel skips the rest of its work, so a wrong transaction count can never
// hang the GPU (worst case about kWaitLimit * kWaitHintNs = 2 s); the host turns the error word
// into DCAACC_DEVICE_INDEX_ERR.  The suspend hint keeps waiting warps from spending issue slots on
// polling.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace dcaacc {

constexpr uint32_t kWaitLimit = 1u << 20;  // reached only on a bug
constexpr uint32_t kWaitHintNs = 2000;     // suspend-time hint of one poll

// Error word bits written by kernels (read back by the host after the launch).
constexpr int kErrBarrierTimeout = 1;
constexpr int kErrIndex = 2;

__device__ inline uint32_t smemAddr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ inline void mbarInit(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(bar)), "r"(count) : "memory");
}

// Makes initialised barriers visible to the async proxy (the bulk-copy engine).
__device__ inline void fenceBarrierInit() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier generic-proxy shared-memory accesses before later async-proxy ones.
__device__ inline void fenceProxyAsync() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ inline void mbarArriveExpectTx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddr(bar)), "r"(bytes)
               : "memory");
}

// bytes must be a multiple of 16 and both addresses 16-byte aligned.
__device__ inline void bulkCopyG2S(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smemAddr(dst)),
      "l"(src), "r"(bytes), "r"(smemAddr(bar))
      : "memory");
}

__device__ inline void mbarArrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smemAddr(bar)) : "memory");
}

__device__ inline bool mbarTryWait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smemAddr(bar)), "r"(parity), "r"(kWaitHintNs)
      : "memory");
  return ok != 0;
}

// Bounded wait for the barrier phase with the given parity.  Returns false on timeout after
// recording it in *err.  limit: polls before giving up (kernels that take a runtime limit pass it;
// 0 is not a valid limit).
__device__ inline bool mbarWait(uint64_t* bar, uint32_t parity, int* err, uint32_t limit = kWaitLimit) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbarTryWait(bar, parity))
      return true;
  atomicOr(err, kErrBarrierTimeout);
  return false;
}

}  // namespace dcaacc
