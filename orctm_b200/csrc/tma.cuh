// Tensor-memory-accelerator (TMA) staging for sm_100a: mbarrier helpers,
// tiled bulk-tensor loads into shared memory, and the host-side encoding of
// a tensor map over a field of the padded device layout (common.cuh).
//
// Only plain loads from this GPU's own memory are issued (no cluster
// multicast).  Every wait on an mbarrier is bounded by a clock budget, so a
// copy that never lands makes the waiting thread give up and report it
// instead of spinning forever.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace orctm {

// about one second at the B200's clock: far beyond any legitimate wait
constexpr long long kWaitCycles = 2000000000LL;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

// makes initialised barriers visible to the async (TMA) proxy
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for the phase of the given parity to complete; false when the clock
// budget ran out first.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > kWaitCycles) return false;
  return true;
}

// 3D tiled load of the box at (x, y, z) into shared memory, completing
// transaction bytes on the barrier.  x must be a multiple of 16 bytes' worth
// of elements (checked by the callers' tile origins).
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// Host: a tensor map over levels 0..nlev-1 of a padded-layout field
// (pitch P elements, JN rows per level) of FP64 or FP32 elements, read in
// boxes of bx x by x 1.  Returns a CUDA driver status (0 = success).
int encode_field_map(CUtensorMap* map, const void* base, int elem_bytes, int P, int JN, int nlev,
                     int bx, int by);

}  // namespace orctm
