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

namespace sufgpu {

// Compacts finished references into one contiguous batch for the output
// phase: row r of the batch belongs to reference j (batch offset dst[j],
// arena position src[j]); text, LCP are copied, SA values and ranks are
// rebased from arena to batch coordinates.
static __global__ void __launch_bounds__(256)
gather_finished_kernel(const u8* __restrict__ text, const u32* __restrict__ sa,
                       const u32* __restrict__ rank, const u32* __restrict__ lcp,
                       const u64* __restrict__ dst, const u64* __restrict__ src, u32 count,
                       u64 m, u8* __restrict__ text_out, u32* __restrict__ sa_out,
                       u32* __restrict__ rank_out, u32* __restrict__ lcp_out) {
  const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
  SegCursor cur;
  for (u64 r = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; r < m; r += stride) {
    cur.locate(dst, count, r);
    const u64 from = src[cur.j] + (r - cur.lo);
    const long long shift = static_cast<long long>(cur.lo) - static_cast<long long>(src[cur.j]);
    text_out[r] = text[from];
    sa_out[r] = static_cast<u32>(static_cast<long long>(sa[from]) + shift);
    rank_out[r] = static_cast<u32>(static_cast<long long>(rank[from]) + shift);
    lcp_out[r] = lcp[from];
  }
}

}  // namespace sufgpu
