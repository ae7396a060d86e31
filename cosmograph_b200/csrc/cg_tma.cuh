// cg_tma.cuh -- tile copies by the tensor memory accelerator (TMA) with an
// mbarrier, for bricks whose halo tile lies inside the box (no periodic
// wrap).  One thread issues the copy of a whole field tile; the CTA waits on
// the barrier's phase.  Loads only, never multicast.
//
// Rules the callers keep (they are checked on the host, cg_mixed_inst.cu):
//   * the tensor map is 4-D {nz, ny, nx, field} with byte strides that are
//     multiples of 16, so nz * sizeof(T) is a multiple of 16;
//   * the innermost start coordinate (z) times sizeof(T) is a multiple of 16;
//   * the shared-memory destination is 128-byte aligned.
#pragma once

#include <cuda.h>

#include <cstdint>

namespace cg {
namespace tma {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void bar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// order this thread's earlier generic-proxy accesses to shared memory before
// later async-proxy (TMA) writes to it
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// make a tensor map that the host copied into global memory visible to the
// tensor-map proxy before this thread's copies use it
__device__ __forceinline__ void acquire_map(const void* map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.sys [%0], 128;" ::"l"(reinterpret_cast<uint64_t>(map))
               : "memory");
}

__device__ __forceinline__ void arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// a 4-D tile of `map` at {c0, c1, c2, c3} into shared memory at dst
__device__ __forceinline__ void load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                        uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
      : "memory");
}

// prefetch a 4-D tile of `map` at {c0, c1, c2, c3} into L2 (no completion to wait for)
__device__ __forceinline__ void prefetch_4d(const CUtensorMap* map, int c0, int c1, int c2, int c3) {
  asm volatile("cp.async.bulk.prefetch.tensor.4d.L2.global.tile [%0, {%1, %2, %3, %4}];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(c0), "r"(c1), "r"(c2), "r"(c3)
               : "memory");
}

// Wait until the barrier completes the phase with parity `phase`; gives up
// after `limit` clock cycles and returns false.  Each round tests the phase
// without blocking, then checks the limit, then waits with try_wait (which
// may suspend the thread for a while), so that a small limit is honoured.
__device__ __forceinline__ bool wait(uint64_t* bar, unsigned phase, long long limit) {
  const long long t0 = clock64();
  while (true) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(phase)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > limit) return false;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(phase)
        : "memory");
    if (done) return true;
  }
}

// A bounded wait that lets a late copy land: after the first `limit` cycles
// the wait goes on for up to kDrainCycles more, so that a copy that is only
// slow completes before its buffer is reused or the CTA exits.  Returns 0
// (in time), 1 (late: landed during the drain) or 2 (lost: never landed).
constexpr long long kDrainCycles = 2000000000LL;  // about a second
__device__ __forceinline__ int wait_drain(uint64_t* bar, unsigned phase, long long limit) {
  if (wait(bar, phase, limit)) return 0;
  return wait(bar, phase, kDrainCycles) ? 1 : 2;
}

}  // namespace tma
}  // namespace cg
