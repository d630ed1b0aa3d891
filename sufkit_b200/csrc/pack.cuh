// Coordinate packing (native32 / split40 / split48 / native64) and the
// permutation check that precedes it.
#pragma once

#include "common.cuh"
#include "doubling.cuh"

namespace sufgpu {

// Writes value - segment start (so batched instances get local coordinates)
// into the low plane, and the high plane when the width has one.  Device
// coordinates are 32-bit, so high planes of split40/48 receive zeros and the
// native64 plane the zero-extended value.
static __global__ void __launch_bounds__(256)
pack_kernel(const u32* __restrict__ values, u64 n, Segments segs, u32 bits,
            void* __restrict__ low, void* __restrict__ high) {
  const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
  SegCursor cur;
  for (u64 r = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += stride) {
    u64 v = values[r];
    if (segs.count > 1) {
      cur.locate(segs.begin, segs.count, r);
      v -= cur.lo;
    }
    if (bits == 64) {
      static_cast<u64*>(low)[r] = v;
    } else {
      static_cast<u32*>(low)[r] = static_cast<u32>(v);
      if (bits == 40) static_cast<u8*>(high)[r] = static_cast<u8>(v >> 32);
      if (bits == 48) static_cast<u16*>(high)[r] = static_cast<u16>(v >> 32);
    }
  }
}

// SA validation (the check RepackSuffixArray performs on the host): every row
// holds a position of its own instance, and ISA[SA[r]] == r, which together
// make SA a permutation.
static __global__ void __launch_bounds__(256)
validate_kernel(const u32* __restrict__ sa, const u32* __restrict__ isa, u64 n,
                Segments segs, DeviceFlags* flags) {
  const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
  for (u64 r = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += stride) {
    const u32 p = sa[r];
    bool ok = p < n;
    if (ok && segs.count > 1) {
      const u32 seg = find_segment(segs.begin, segs.count, r);
      ok = p >= segs.begin[seg] && p < segs.begin[seg + 1];
    }
    if (ok) ok = isa[p] == r;
    if (!ok) flag_error(flags, kErrNotPermutation);
  }
}

}  // namespace sufgpu
