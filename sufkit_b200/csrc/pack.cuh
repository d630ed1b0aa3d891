// Coordinate packing (native32 / split40 / split48 / native64) and the
// permutation check that precedes it.
#pragma once

#include "common.cuh"
#include "doubling.cuh"
#include "scan.cuh"

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

// Suffix-array sampling at rate K > 1 (the reference's BuildDivsufsort with
// sampling_rate K, src/divsufsort_backend.cpp:62-73,81-150): keep the rows
// whose instance-local position is a multiple of K, in row order; sampled
// ISA[local / K] = sampled row; sampled LCP[j] = lcp of sampled rows j-1 and j,
// which is the minimum of the complete row LCPs after row j-1 up to row j.
// Rows are scanned in 2048-row tiles (decoupled look-back over the kept
// counts).  Every instance keeps exactly ceil(n_i / K) rows, so its sampled
// rows start at out_begin[i] (host-computed).  Sampled positions and rows are
// instance-local; lcp_k must start as all ones (the minima are atomic).
static __global__ void __launch_bounds__(kScanBlock)
sample_kernel(const u32* __restrict__ sa, const u32* __restrict__ lcp, u64 n, Segments segs,
              u32 rate, const u64* __restrict__ out_begin, u64 kept_total,
              u32* __restrict__ sa_k, u32* __restrict__ isa_k, u32* __restrict__ lcp_k,
              u64* status_sum, u32* tile_counter, DeviceFlags* flags) {
  __shared__ u64 warp_smem[kScanBlock / 32];
  __shared__ u64 tile_prefix;
  __shared__ u32 tile_slot;
  const u32 tile = claim_tile(tile_counter, &tile_slot);
  const u64 row0 = static_cast<u64>(tile) * kScanTile + threadIdx.x * kScanItems;
  SegCursor cur;
  u32 local[kScanItems];
  u32 kept = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const u64 r = row0 + i;
    local[i] = 1;  // not kept
    if (r < n) {
      cur.locate(segs.begin, segs.count, r);
      const u64 p = sa[r];
      if (p < cur.lo || p >= cur.hi) {
        flag_error(flags, kErrBounds);
        continue;
      }
      local[i] = static_cast<u32>(p - cur.lo);
      kept += local[i] % rate == 0;
    }
  }
  u64 agg;
  const u64 excl = block_exclusive_scan<kScanBlock>(kept, SumOp{}, warp_smem, &agg);
  if ((threadIdx.x >> 5) == 0) {
    const u64 pre = warp_lookback(status_sum, tile, agg, SumOp{}, flags, 8);
    if ((threadIdx.x & 31) == 0) tile_prefix = pre;
  }
  __syncthreads();
  u64 j = tile_prefix + excl;  // sampled rows before this thread's first row
  u64 run_seg = ~0ull;
  u32 run_min = 0xffffffffu;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const u64 r = row0 + i;
    if (r >= n) break;
    const bool keep = local[i] % rate == 0;
    // Row r closes the LCP segment of sampled row j (kept or not).
    if (lcp && j < kept_total) {
      if (j != run_seg) {
        if (run_seg != ~0ull) atomicMin(&lcp_k[run_seg], run_min);
        run_seg = j;
        run_min = 0xffffffffu;
      }
      const u32 v = lcp[r];
      run_min = v < run_min ? v : run_min;
    }
    if (keep) {
      if (j >= kept_total) {
        flag_error(flags, kErrBounds);
        break;
      }
      cur.locate(segs.begin, segs.count, r);
      const u32 inst = segs.count == 1 ? 0 : find_segment(segs.begin, segs.count, r);
      const u64 off = out_begin[inst];
      const u64 slot = off + local[i] / rate;
      if (slot >= kept_total || j < off) {
        flag_error(flags, kErrBounds);
        break;
      }
      sa_k[j] = local[i];
      isa_k[slot] = static_cast<u32>(j - off);
      ++j;
    }
  }
  if (run_seg != ~0ull) atomicMin(&lcp_k[run_seg], run_min);
}

}  // namespace sufgpu
