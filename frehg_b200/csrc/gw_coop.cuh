// Device helpers shared by the cooperative solver kernels: the bounded grid
// barrier and the fixed-order (deterministic) block and grid reductions.
#pragma once

#include "gw_internal.h"

namespace fgw {
namespace coop {

constexpr int kCgBlock = 256;
constexpr long long kSpinLimit = 20000000LL;  // ~2-4 s of polling

__device__ inline unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ inline int ld_relaxed_int(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier for a cooperative (co-resident) launch.  Returns false
// when the barrier gave up; the caller then leaves the kernel.
__device__ inline bool grid_sync(CgState* st, unsigned nblocks) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int good = 1;
    if (ld_relaxed_int(&st->err) != 0) {
      good = 0;
    } else {
      const unsigned my = ld_acquire(&st->bar_gen);
      __threadfence();
      const unsigned arrived = atomicAdd(&st->bar_count, 1u) + 1u;
      if (arrived == nblocks) {
        atomicExch(&st->bar_count, 0u);
        __threadfence();
        atomicAdd(&st->bar_gen, 1u);
      } else {
        long long spins = 0;
        while (ld_acquire(&st->bar_gen) == my) {
          if (++spins > kSpinLimit || ld_relaxed_int(&st->err) != 0) {
            atomicExch(&st->err, 1);
            good = 0;
            break;
          }
          __nanosleep(64);
        }
      }
      __threadfence();
    }
    ok = good;
  }
  __syncthreads();
  return ok != 0;
}

__device__ inline double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Fixed-order block sum; result broadcast to every thread.
__device__ inline double block_sum_all(double v) {
  __shared__ double sh[32];
  __shared__ double res;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  if (wid == 0) {
    v = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0.0;
    v = warp_sum(v);
    if (lane == 0) res = v;
  }
  __syncthreads();
  const double out = res;
  __syncthreads();
  return out;
}

// Sum of the G per-block partials, identical in every block.
__device__ inline double reduce_partials(const double* part, int G) {
  double v = 0.0;
  for (int b = threadIdx.x; b < G; b += blockDim.x) v += part[b];
  return block_sum_all(v);
}

// The member of a batched launch whose block range [first[i], first[i+1])
// holds block b (first has n + 1 ascending entries).
__device__ inline int instance_of(const int* first, int n, int b) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (first[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

}  // namespace coop
}  // namespace fgw
