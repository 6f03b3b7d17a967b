// Bulk (TMA) row copies from global into shared memory, completed on mbarriers.
//
// A warp streams rows through a ring of shared-memory slots: one lane issues
// `cp.async.bulk` copies of whole row segments (no multicast, this GPU's
// memory or the caller's buffers only) and arms the slot's mbarrier with the
// byte count; every lane waits on the barrier's phase before reading the slot.
// A copy moves up to a few KB with one instruction, where per-thread cp.async
// needs one instruction per 16 bytes and per lane; at the occupancy of the
// streaming kernels (4-5 CTAs of 128 threads per SM) bulk copies keep HBM
// near its copy bandwidth, per-thread copies reach about three quarters of it.
//
// Requirements of the instruction: source and destination 16-byte aligned, a
// size that is a multiple of 16 bytes.  Waits are bounded: a phase that does
// not complete in time sets the plan's error word, so a lost copy becomes an
// error the host reports instead of a hang.
#pragma once

#include <cstdint>

namespace gd {
namespace bulk {

constexpr int kWaitTries = 1 << 22;     // try_wait attempts before a wait is given up
constexpr unsigned kErrWait = 1u;       // error word bit: a bulk-copy wait timed out

__device__ __forceinline__ unsigned saddr(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared.b64 [%0], %1;\n" ::"r"(saddr(bar)), "r"(count) : "memory");
}

// Make the initialised barriers visible to the bulk-copy (async) proxy.
__device__ __forceinline__ void init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// Order this thread's earlier shared-memory reads before a bulk copy that
// overwrites the same bytes.
__device__ __forceinline__ void proxy_fence() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// Arrive on `bar` and announce `bytes` of bulk copies for its current phase
// (zero completes the phase at once).
__device__ __forceinline__ void arrive_expect(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared.b64 _, [%0], %1;\n" ::"r"(saddr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void copy(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          saddr(dst)),
      "l"(src), "r"(bytes), "r"(saddr(bar))
      : "memory");
}

__device__ __forceinline__ bool try_wait(uint64_t *bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(saddr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Wait (bounded: `tries` attempts) for phase `parity` of `bar`, called by a
// whole warp.  On a timeout the error word is set and the wait is retried
// once, bounded again, so that copies still in flight land before the caller
// moves on.  Returns whether the phase completed.
__device__ __forceinline__ bool wait(uint64_t *bar, unsigned parity, unsigned *err,
                                     int tries = kWaitTries) {
  bool done = false;
  for (int k = 0; k < tries && !done; ++k) done = try_wait(bar, parity);
  if (__all_sync(0xffffffffu, done)) return true;
  if ((threadIdx.x & 31) == 0) atomicOr(err, kErrWait);
  for (int k = 0; k < tries && !done; ++k) done = try_wait(bar, parity);
  return __all_sync(0xffffffffu, done);
}

}  // namespace bulk
}  // namespace gd
