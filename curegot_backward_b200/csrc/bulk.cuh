// Bulk asynchronous copies global -> shared with mbarrier completion, and a
// per-warp ring of staging buffers built on them (sm_90+ PTX, used on sm_100a).
//
// A ring has kRingStages buffers of kRingBytes each and one mbarrier per
// buffer.  Chunk g of a warp's stream goes to stage g % kRingStages and is
// complete when that stage's barrier finishes phase (g / kRingStages) & 1.
// Lane 0 issues the copies (arrive.expect_tx + cp.async.bulk); all lanes wait.
// Every wait is bounded: after kRingSpin polls it gives up and reports it.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace cg {

constexpr int kRingStages = 3;
constexpr int kRingBytes = 2048;
constexpr long kRingSpin = 1L << 24;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init1(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Generic-proxy accesses to shared memory before this point are ordered
// before later async-proxy (bulk copy) accesses.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// bytes: a multiple of 16; src and dst: 16-byte aligned.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// Hint: bring [src, src + bytes) into L2 (no completion, no shared memory).
// bytes: a multiple of 16; src: 16-byte aligned.
__device__ __forceinline__ void prefetch_l2_bulk(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
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

// Bounded wait for the given phase parity; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (long it = 0; it < kRingSpin; ++it)
    if (mbar_test(bar, parity)) return true;
  return false;
}

// One warp's ring: buffers (kRingStages x kRingBytes, 128-byte aligned) and
// barriers in shared memory, plus the warp-uniform chunk counters.
struct WarpRing {
  unsigned char* buf;
  uint64_t* bar;
  uint32_t issued;    // chunks issued so far (global sequence number)
  uint32_t consumed;  // chunks waited for and read
  bool failed;        // a wait gave up

  __device__ __forceinline__ unsigned char* stage(uint32_t g) const {
    return buf + (size_t)(g % kRingStages) * kRingBytes;
  }
  __device__ __forceinline__ uint64_t* barrier(uint32_t g) const {
    return bar + (g % kRingStages);
  }
  // Wait for chunk `consumed`; on success the caller reads stage(consumed).
  __device__ __forceinline__ bool wait_next() {
    const uint32_t g = consumed;
    const bool ok = mbar_wait_bounded(barrier(g), (g / kRingStages) & 1u);
    return __all_sync(0xffffffffu, ok);
  }
  // After a failed wait: wait (bounded) for every copy still in flight, so
  // none lands in shared memory after the block has moved on.
  __device__ __forceinline__ void drain() {
    for (uint32_t g = consumed; g < issued; ++g)
      mbar_wait_bounded(barrier(g), (g / kRingStages) & 1u);
    consumed = issued;
    failed = true;
  }
};

// Initialise the rings of every warp of the block (call from all threads;
// ends with a block barrier).
__device__ __forceinline__ void rings_init(unsigned char* dyn, uint64_t* bars, int warps,
                                           WarpRing& ring) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
    for (int s = 0; s < kRingStages; ++s) mbar_init1(bars + warp * kRingStages + s);
  if (threadIdx.x == 0) fence_mbar_init();
  __syncthreads();
  ring.buf = dyn + (size_t)warp * kRingStages * kRingBytes;
  ring.bar = bars + warp * kRingStages;
  ring.issued = ring.consumed = 0;
  ring.failed = false;
  (void)warps;
}

}  // namespace cg
