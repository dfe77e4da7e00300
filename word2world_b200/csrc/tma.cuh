// Shared-memory barriers (mbarrier) and TMA row gathers for sm_100a, as
// inline PTX.
//
// Row gather: cp.async.bulk.tensor.2d with the tile::gather4 load mode copies
// four rows of a 2-D tensor, picked by their row indices, into consecutive
// shared memory (row i at dst + i * row bytes) and signals completion on an
// mbarrier with its byte count.  The tensor map is 2-D: the innermost
// dimension is one row's elements, the box one row high and one row wide, so
// every gather starts at column 0 (16-byte aligned).  The destination is the
// executing CTA's own shared memory (128-byte aligned); no load here reads
// from or writes to another CTA or another GPU.
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace w2w {
namespace tma {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void bar_init(unsigned long long* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Makes initialised barriers visible to the asynchronous (TMA) proxy; follow
// with a CTA barrier before any use.
__device__ __forceinline__ void bar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void bar_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// One arrival that also announces `bytes` of asynchronous copies this phase.
__device__ __forceinline__ void bar_arrive_expect(unsigned long long* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// True once the phase with parity `parity` has completed (acquire).  Never
// blocks: callers poll it a bounded number of times.
__device__ __forceinline__ bool bar_test(unsigned long long* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0u;
}

// Waits (suspended in hardware, woken when the phase completes) at most about
// `hint_ns` nanoseconds for the phase with parity `parity`; true once it has
// completed (acquire).
__device__ __forceinline__ bool bar_try_wait(unsigned long long* bar, uint32_t parity, uint32_t hint_ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0u;
}

// Four rows (r0..r3) of `map` into dst (4 * row bytes, 128-byte aligned),
// completing on `bar`.
__device__ __forceinline__ void gather4(void* dst, const CUtensorMap* map, unsigned long long* bar, int r0, int r1,
                                        int r2, int r3) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5, %6, %7}], [%2];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_addr(bar)), "r"(0), "r"(r0), "r"(r1), "r"(r2), "r"(r3)
      : "memory");
}

__device__ __forceinline__ void prefetch_map(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

}  // namespace tma
}  // namespace w2w
