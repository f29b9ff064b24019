// Tensor-memory-accelerator (TMA) tile loads with an mbarrier, as inline PTX for sm_100a.
//
// Every wait is bounded: after the iteration budget the caller records an error flag and
// returns instead of spinning forever.
#pragma once
#include <cuda.h>
#include <cstdint>

namespace dgb {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// orders this thread's earlier generic-proxy shared-memory accesses before later async-proxy ones
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// 3D tiled bulk tensor load global -> shared completing on `bar` (coordinates innermost first;
// the innermost coordinate times the element size must be a multiple of 16 bytes).
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// Prefetch of a 3D tile into L2 (no shared-memory destination, no completion to wait for); same
// coordinate rules as tma_load_3d.
__device__ __forceinline__ void tma_prefetch_3d(const CUtensorMap* map, int x, int y, int z) {
  asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y), "r"(z)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Default poll budget of a bounded wait (about 4 M polls: far beyond any copy's latency).
constexpr long long kDefaultPolls = 1ll << 22;

// Bounded wait for phase `parity` of `bar`; false when the budget ran out.  A caller whose first
// wait gave up waits again with the default budget before it leaves, so that no copy still lands
// in the shared memory of a finished CTA.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long max_polls = kDefaultPolls) {
  for (long long k = 0; k < max_polls; ++k)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

}  // namespace dgb
