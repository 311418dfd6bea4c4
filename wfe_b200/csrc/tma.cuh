// Tensor-memory-accelerator (TMA) helpers for sm_100a: mbarrier set-up, a
// bounded wait on its phase, and 3D tiled bulk-tensor loads from global into
// shared memory (no cluster multicast).  Inline PTX; the tensor maps are
// encoded on the host (model.cu) and passed as __grid_constant__ parameters.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace wfe {
namespace tma {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// makes the initialised barrier visible to the async (TMA) proxy
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// plain arrive (count 1) on the barrier's current phase
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// named barrier `id` over the first `n` threads of the CTA (n a multiple of 32)
__device__ __forceinline__ void named_sync(int id, int n) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

// named barrier that also returns whether any participating thread passed v
__device__ __forceinline__ bool named_or(int id, int n, bool v) {
  int r;
  asm volatile(
      "{\n"
      ".reg .pred p, q;\n"
      "setp.ne.s32 p, %1, 0;\n"
      "bar.red.or.pred q, %2, %3, p;\n"
      "selp.s32 %0, 1, 0, q;\n"
      "}\n"
      : "=r"(r)
      : "r"((int)v), "r"(id), "r"(n)
      : "memory");
  return r != 0;
}

// one non-blocking probe of the barrier's phase `parity`
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// one probe that may suspend the thread for at most about `hint_ns`
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity, uint32_t hint_ns) {
  uint32_t done;
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
      "selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity), "r"(hint_ns)
      : "memory");
  return done != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// waits for phase `parity` for at most `max_ns` nanoseconds of wall time;
// false when it gave up
__device__ __forceinline__ bool mbar_wait_for(uint64_t* bar, uint32_t parity, uint64_t max_ns) {
  if (mbar_try(bar, parity, 1000)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_try(bar, parity, 1000))
    if (global_ns() - t0 > max_ns) return false;
  return true;
}

// waits for phase `parity` with at most `limit` probes; false when it gave up
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
  for (uint32_t n = 0; n < limit; ++n)
    if (mbar_test(bar, parity)) return true;
  return false;
}

// 3D tile load: box of the tensor map at element coordinates (x, y, z), x
// innermost, into shared memory at dst; completion counted on bar
__device__ __forceinline__ void load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                        uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}

}  // namespace tma
}  // namespace wfe
