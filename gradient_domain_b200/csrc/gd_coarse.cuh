// The coarse part of the V-cycle in one persistent launch.
//
// Below the last level that runs on the register-streaming strips, every
// remaining step of a V-cycle - the shared-memory tile levels on the way down,
// the one-CTA bottom of every instance, the tile levels on the way up - is a
// phase whose work items (tiles of every instance at that level, or
// instances) are independent of each other but depend on the previous phase.
// One cooperative launch of one CTA per SM walks the phases (every tile level
// here has the small tile shape): each CTA takes
// the phase's items round-robin, then all CTAs meet at a grid barrier before
// the next phase.  This replaces one launch per phase (2 x tile levels + 1) and
// its launch gap and tail; the work of every item is the same device function
// the per-level kernels run, so the result is bitwise the same.
//
// The barrier is a counter and a generation word in the plan's counter array.
// Its wait is bounded: a CTA that has waited kBarrierTries rounds sets
// kErrBarrier in the plan's error word and goes on (the solve then fails
// instead of hanging; with a cooperative launch every CTA is resident, so the
// limit is never reached in a correct run).
#pragma once

#include "gd_tile.cuh"

namespace gd {
namespace coarse {

constexpr int kMaxPhases = 40;
constexpr int kCounter = 8, kGeneration = 9;  // slots of the plan's counter array
constexpr unsigned kErrBarrier = 4u;          // error word bit: a grid barrier gave up
constexpr int kBarrierTries = 1 << 24;        // polls (tens of ns each) before giving up

enum : int { kPhaseDown = 0, kPhaseBottom = 1, kPhaseUp = 2 };

struct Phases {
  int count;
  int kind[kMaxPhases];
  int base[kMaxPhases];   // first tile of the phase (tile phases)
  int items[kMaxPhases];  // tiles, or instances for the bottom
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Every CTA of the grid arrives once; the last to arrive resets the counter and
// advances the generation, the others wait for the generation to move.
__device__ __forceinline__ void grid_barrier(unsigned *counter) {
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned *count = counter + kCounter, *gen = counter + kGeneration;
    const unsigned g = ld_acquire(gen);
    __threadfence();  // this CTA's writes of the phase before it counts as arrived
    if (atomicAdd(count, 1u) == gridDim.x - 1) {
      *count = 0u;
      __threadfence();
      atomicAdd(gen, 1u);
    } else {
      int tries = 0;
      while (ld_acquire(gen) == g) {
        if (++tries > kBarrierTries) {
          atomicOr(counter + kErrWord, kErrBarrier);
          break;
        }
      }
    }
    __threadfence();
  }
  __syncthreads();
}

template <typename T, int S>
__global__ void __launch_bounds__(kBThreads, 1) k_coarse(Args<T> a, Phases ph) {
  extern __shared__ __align__(16) unsigned char smem[];
  for (int q = 0; q < ph.count; ++q) {
    if (q > 0) grid_barrier(a.counter);
    const int kind = ph.kind[q];
    for (int k = blockIdx.x; k < ph.items[q]; k += gridDim.x) {
      __syncthreads();  // the previous item's readers of shared memory are done
      if (kind == kPhaseBottom) {
        if (a.st[k].status == GD_ACTIVE) bottom_instance<T, S, S>(a, k, smem);
      } else {
        const Tile tl = a.tiles[ph.base[q] + k];
        const LevelInfo L = a.lv[tl.level];
        const LevelInfo Lc = a.lv[tl.level + 1];
        if (a.st[tl.inst].status != GD_ACTIVE) continue;
        if (kind == kPhaseDown)
          tile::down_tile<T, S, kBThreads, tile::kTYs, tile::kTXs>(a, tl, L, Lc, smem);
        else
          tile::up_tile<T, S, kBThreads, tile::kTYs, tile::kTXs>(a, tl, L, Lc, smem);
      }
    }
  }
}

}  // namespace coarse
}  // namespace gd
