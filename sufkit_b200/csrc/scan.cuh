// Block-wide scans used by the single-pass (decoupled look-back) tile kernels.
#pragma once

#include "common.cuh"

namespace sufgpu {

// Exclusive block scan of one value per thread.  warp_smem needs BLOCK/32
// entries.  Returns the thread's exclusive prefix; *total receives the block
// aggregate (identical in every thread).  Contains __syncthreads().
template <int BLOCK, class Op>
__device__ __forceinline__ u64 block_exclusive_scan(u64 value, Op op,
                                                    u64* warp_smem,
                                                    u64* total) {
  constexpr int kWarps = BLOCK / 32;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  u64 inclusive = value;
#pragma unroll
  for (int offset = 1; offset < 32; offset <<= 1) {
    const u64 y = __shfl_up_sync(0xffffffffu, inclusive, offset);
    if (lane >= offset) inclusive = op(inclusive, y);
  }
  if (lane == 31) warp_smem[warp] = inclusive;
  __syncthreads();
  if (warp == 0) {
    u64 w = lane < kWarps ? warp_smem[lane] : Op::identity;
#pragma unroll
    for (int offset = 1; offset < 32; offset <<= 1) {
      const u64 y = __shfl_up_sync(0xffffffffu, w, offset);
      if (lane >= offset) w = op(w, y);
    }
    if (lane < kWarps) warp_smem[lane] = w;
  }
  __syncthreads();
  const u64 warp_prefix = warp ? warp_smem[warp - 1] : Op::identity;
  u64 before = __shfl_up_sync(0xffffffffu, inclusive, 1);
  if (lane == 0) before = Op::identity;
  *total = warp_smem[kWarps - 1];
  __syncthreads();
  return op(warp_prefix, before);
}

// Claims the next tile index of a single-pass kernel (tiles are claimed in the
// order blocks start running, which the look-back relies on).
__device__ __forceinline__ u32 claim_tile(u32* counter, u32* smem_slot) {
  if (threadIdx.x == 0) *smem_slot = atomicAdd(counter, 1u);
  __syncthreads();
  const u32 tile = *smem_slot;
  return tile;
}

}  // namespace sufgpu
