// Kernels of the served (continuously batched) engine: moving a newly seeded
// group of references into the shared arena and tracking which in-flight
// references still have unsorted rows.
#pragma once

#include "common.cuh"
#include "doubling.cuh"

namespace sufgpu {

// SA and ranks of a freshly seeded group were written relative to its arena
// offset; make them absolute (positions and rows are arena coordinates).
static __global__ void __launch_bounds__(256)
relocate_kernel(u32* __restrict__ sa, u32* __restrict__ rank, u64 m, u32 bias) {
  const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
  for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += stride) {
    sa[i] += bias;
    rank[i] += bias;
  }
}

// dst[i] = src[i] + bias (append a group's active list to the shared list,
// or rebase a finished reference's SA/ranks to its own coordinates).
static __global__ void __launch_bounds__(256)
shift_kernel(const u32* __restrict__ src, u64 count, long long bias, u32* __restrict__ dst) {
  const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
  for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += stride) {
    dst[i] = static_cast<u32>(static_cast<long long>(src[i]) + bias);
  }
}

// alive[j] = 1 for every in-flight reference j with a row in the active list.
static __global__ void __launch_bounds__(256)
alive_kernel(const u32* __restrict__ active, u64 count, Segments segs, u8* __restrict__ alive) {
  const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
  for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += stride) {
    const u32 j = segs.count == 1 ? 0 : find_segment(segs.begin, segs.count, active[i]);
    alive[j] = 1;
  }
}

}  // namespace sufgpu
