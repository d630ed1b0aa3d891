// Exact k-mer prefix directory of a Fast index (the reference's
// FastPrefixIndex, src/fast_prefix_index.cpp:131-205,322-376): for every k-mer
// over A, C, G, T (text bytes 2..5), the SA rows [begin, end) of the suffixes
// that start with it, packed as begin | end << 32; empty k-mers hold
// (n, n).  The reference walks text positions and widens each k-mer's
// interval with the row from the ISA; here each SA row computes its own
// suffix's k-mer, and the rows where the k-mer changes write the interval
// ends.  A k-mer's rows are contiguous in the SA, so every half of an entry
// is written exactly once.
#pragma once

#include "common.cuh"

namespace sufgpu {

constexpr u32 kDirTile = 1024;

static __global__ void __launch_bounds__(256)
prefix_fill_kernel(u64* __restrict__ intervals, u64 entries, u64 empty) {
  for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < entries;
       i += static_cast<u64>(gridDim.x) * blockDim.x) {
    intervals[i] = empty;
  }
}

// counts[0] += rows with a canonical k-mer (the reference's IndexedKmers),
// counts[1] += distinct k-mers present (NonemptyEntries).
static __global__ void __launch_bounds__(kDirTile)
prefix_directory_kernel(const u8* __restrict__ text, const u32* __restrict__ sa, u64 n, u32 k,
                        u64* __restrict__ intervals, unsigned long long* counts,
                        DeviceFlags* flags) {
  __shared__ u32 keys[kDirTile + 2];  // rows r0-1 .. r0+kDirTile; kNone = no canonical k-mer
  const u64 r0 = static_cast<u64>(blockIdx.x) * kDirTile;
  for (u32 i = threadIdx.x; i < kDirTile + 2; i += blockDim.x) {
    const long long r = static_cast<long long>(r0) - 1 + i;
    u32 key = kNone;
    if (r >= 0 && static_cast<u64>(r) < n) {
      const u64 p = sa[r];
      if (p >= n) {
        flag_error(flags, kErrBounds);
      } else if (p + k <= n) {
        u32 kk = 0;
        bool canonical = true;
        for (u32 j = 0; j < k; ++j) {
          const u32 c = text[p + j];
          canonical &= c >= 2 && c <= 5;
          kk = (kk << 2) | ((c - 2) & 3);
        }
        if (canonical) key = kk;
      }
    }
    keys[i] = key;
  }
  __syncthreads();
  const u64 r = r0 + threadIdx.x;
  const u32 key = r < n ? keys[threadIdx.x + 1] : kNone;
  const bool begins = key != kNone && keys[threadIdx.x] != key;
  if (key != kNone) {
    u32* entry = reinterpret_cast<u32*>(intervals + key);
    if (begins) entry[0] = static_cast<u32>(r);
    if (keys[threadIdx.x + 2] != key) entry[1] = static_cast<u32>(r + 1);
  }
  const u32 lane = threadIdx.x & 31;
  const u32 valid = __popc(__ballot_sync(0xffffffffu, key != kNone));
  const u32 firsts = __popc(__ballot_sync(0xffffffffu, begins));
  if (lane == 0 && (valid || firsts)) {
    atomicAdd(&counts[0], static_cast<unsigned long long>(valid));
    atomicAdd(&counts[1], static_cast<unsigned long long>(firsts));
  }
}

}  // namespace sufgpu
