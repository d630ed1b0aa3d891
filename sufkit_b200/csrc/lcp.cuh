// LCP kernels: PHI, irreducible PLCP, propagation, row-order gather, byte
// coding (primary bytes + text-ordered overflow anchors).
//
// PLCP[i] = lcp(i, phi[i]) where phi[i] is the suffix just before i in SA
// order.  A position is reducible when text[i-1] == text[phi[i]-1]; then
// phi[i-1] = phi[i] - 1 and PLCP[i] = PLCP[i-1] - 1 exactly.  Only irreducible
// positions compare text (their total is O(n log n) and close to n on genomic
// text); every reducible PLCP follows from the nearest irreducible position r
// before it as PLCP[r] - (i - r).  This gives the same values as the
// reference's sequential Kasai loop without its carry chain.
#pragma once

#include "common.cuh"
#include "doubling.cuh"
#include "scan.cuh"

namespace sufgpu {

// Eight text bytes starting at an arbitrary position (little-endian, first
// byte lowest).  The text buffer carries >= 16 readable bytes past its end.
__device__ __forceinline__ u64 load8(const u8* __restrict__ text, u64 pos) {
  const u64 base = pos & ~7ull;
  const u32 s = static_cast<u32>(pos & 7) * 8;
  const u64 lo = __ldg(reinterpret_cast<const unsigned long long*>(text + base));
  if (s == 0) return lo;
  const u64 hi = __ldg(reinterpret_cast<const unsigned long long*>(text + base + 8));
  return (lo >> s) | (hi << (64 - s));
}

__global__ void __launch_bounds__(256)
phi_kernel(const u32* __restrict__ sa, u64 n, Segments segs,
           u32* __restrict__ phi) {
  const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
  for (u64 r = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += stride) {
    const u32 p = sa[r];
    phi[p] = is_segment_start(segs, r) ? kNone : sa[r - 1];
  }
}

// Thread-level compare budget before a position is handed to a warp.
constexpr u32 kThreadLcpBytes = 64;

struct LongLcpItem {
  u32 i, j;
  u64 done;  // bytes already known equal
};

__global__ void __launch_bounds__(256)
plcp_irreducible_kernel(const u8* __restrict__ text, const u32* __restrict__ phi,
                        u64 n, Segments segs, u32* __restrict__ plcp,
                        u8* __restrict__ irreducible, LongLcpItem* queue,
                        u64 queue_cap, u64* queue_count, DeviceFlags* flags) {
  const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
  for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    const u32 j = phi[i];
    if (j == kNone) {
      plcp[i] = 0;
      irreducible[i] = 1;
      continue;
    }
    const u64 seg_first = segs.count == 1 ? 0 : segs.begin[find_segment(segs.begin, segs.count, i)];
    const bool irr = i == seg_first || j == seg_first || text[i - 1] != text[j - 1];
    irreducible[i] = irr;
    if (!irr) continue;
    const u64 end = segment_end(segs, i);
    const u64 far = i > j ? i : j;
    const u64 limit = end - far;
    const u64 budget = limit < kThreadLcpBytes ? limit : kThreadLcpBytes;
    u64 l = 0;
    bool mismatch = false;
    while (l < budget) {
      const u64 x = load8(text, i + l) ^ load8(text, j + l);
      if (x) {
        l += static_cast<u64>(__ffsll(static_cast<long long>(x)) - 1) >> 3;
        mismatch = true;
        break;
      }
      l += 8;
    }
    if (l > limit) l = limit;
    if (!mismatch && l < limit) {
      const u64 slot = atomicAdd(reinterpret_cast<unsigned long long*>(queue_count), 1ull);
      if (slot < queue_cap) {
        queue[slot] = LongLcpItem{static_cast<u32>(i), j, l};
      } else {
        flag_error(flags, kErrQueueOverflow);
      }
    }
    plcp[i] = static_cast<u32>(l);
  }
}

// One warp per long item: 32 lanes x 16 bytes per step.
__global__ void __launch_bounds__(256)
long_lcp_kernel(const u8* __restrict__ text, const LongLcpItem* __restrict__ queue,
                const u64* queue_count, u64 queue_cap, Segments segs,
                u32* __restrict__ plcp) {
  const u32 lane = threadIdx.x & 31;
  const u64 warps = static_cast<u64>(gridDim.x) * (blockDim.x / 32);
  u64 count = *queue_count;
  if (count > queue_cap) count = queue_cap;
  for (u64 w = (static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x) / 32; w < count; w += warps) {
    const LongLcpItem item = queue[w];
    const u64 end = segment_end(segs, item.i);
    const u64 far = item.i > item.j ? item.i : item.j;
    const u64 limit = end - far;
    u64 l = item.done;
    while (l < limit) {
      const u64 off = l + lane * 16;
      // Lanes at or past the limit load nothing and report a stop at off;
      // loads therefore never reach beyond limit + 16 <= the padded end.
      u64 local = 0;
      if (off < limit) {
        const u64 x0 = load8(text, item.i + off) ^ load8(text, item.j + off);
        const u64 x1 = load8(text, item.i + off + 8) ^ load8(text, item.j + off + 8);
        local = 16;
        if (x0) local = static_cast<u64>(__ffsll(static_cast<long long>(x0)) - 1) >> 3;
        else if (x1) local = 8 + (static_cast<u64>(__ffsll(static_cast<long long>(x1)) - 1) >> 3);
      }
      const u32 hit = __ballot_sync(0xffffffffu, local < 16);
      if (hit) {
        const u32 first = __ffs(hit) - 1;
        const u64 found = __shfl_sync(0xffffffffu, off + local, first);
        l = found;
        break;
      }
      l += 512;
    }
    if (l > limit) l = limit;
    if (lane == 0) plcp[item.i] = static_cast<u32>(l);
  }
}

// Reducible positions: PLCP[i] = PLCP[r] - (i - r), r = last irreducible <= i.
__global__ void __launch_bounds__(kScanBlock)
plcp_propagate_kernel(const u8* __restrict__ irreducible, u64 n,
                      u32* __restrict__ plcp, u64* status_max,
                      u32* tile_counter, DeviceFlags* flags) {
  __shared__ u64 warp_smem[kScanBlock / 32];
  __shared__ u64 tile_prefix;
  __shared__ u32 tile_slot;
  const u32 tile = claim_tile(tile_counter, &tile_slot);
  const u64 i0 = static_cast<u64>(tile) * kScanTile + threadIdx.x * kScanItems;
  bool irr[kScanItems];
  u64 last = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const u64 i = i0 + k;
    irr[k] = i < n && irreducible[i];
    if (irr[k]) last = i;
  }
  u64 agg;
  const u64 excl = block_exclusive_scan<kScanBlock>(last, MaxOp{}, warp_smem, &agg);
  if ((threadIdx.x >> 5) == 0) {
    const u64 p = warp_lookback(status_max, tile, agg, MaxOp{}, flags, 7);
    if ((threadIdx.x & 31) == 0) tile_prefix = p;
  }
  __syncthreads();
  u64 r = tile_prefix > excl ? tile_prefix : excl;
  u32 base = 0;
  bool have = false;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const u64 i = i0 + k;
    if (i >= n) break;
    if (irr[k]) {
      r = i;
      have = false;
      continue;
    }
    if (!have) {
      base = plcp[r];
      have = true;
    }
    plcp[i] = base - static_cast<u32>(i - r);
  }
}

// Row order: LCP[r] = PLCP[SA[r]].
template <class Out>
__global__ void __launch_bounds__(256)
lcp_gather_kernel(const u32* __restrict__ sa, const u32* __restrict__ plcp,
                  u64 n, Out* __restrict__ lcp) {
  const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
  for (u64 r = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += stride) {
    lcp[r] = static_cast<Out>(plcp[sa[r]]);
  }
}

__global__ void __launch_bounds__(256)
lcp_primary_kernel(const u32* __restrict__ sa, const u32* __restrict__ plcp,
                   u64 n, u8* __restrict__ primary) {
  const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
  for (u64 r = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += stride) {
    const u32 v = plcp[sa[r]];
    primary[r] = static_cast<u8>(v < 255 ? v : 255);
  }
}

// Overflow anchors in text order: p opens an anchor when PLCP[p] >= 255 and p
// does not continue the run of p-1 (PLCP[p-1] == PLCP[p] + 1, same instance).
// Positions are written as global (concatenated-text) positions; the host
// splits them per instance and subtracts the instance start.
template <class Coord>
__global__ void __launch_bounds__(kScanBlock)
anchor_kernel(const u32* __restrict__ plcp, u64 n, Segments segs,
              Coord* __restrict__ anchor_pos, Coord* __restrict__ anchor_val,
              u64 anchor_cap, u64* status_sum, u32* tile_counter,
              u64* anchor_count, DeviceFlags* flags) {
  __shared__ u64 warp_smem[kScanBlock / 32];
  __shared__ u64 tile_prefix;
  __shared__ u32 tile_slot;
  const u32 tile = claim_tile(tile_counter, &tile_slot);
  const u64 i0 = static_cast<u64>(tile) * kScanTile + threadIdx.x * kScanItems;
  u32 v[kScanItems + 1];
#pragma unroll
  for (int k = 0; k < kScanItems + 1; ++k) {
    const long long i = static_cast<long long>(i0) - 1 + k;
    v[k] = (i >= 0 && static_cast<u64>(i) < n) ? plcp[i] : 0;
  }
  bool open[kScanItems];
  u32 opens = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const u64 i = i0 + k;
    open[k] = false;
    if (i < n && v[k + 1] >= 255) {
      const bool continues = !is_segment_start(segs, i) && v[k] == v[k + 1] + 1;
      open[k] = !continues;
      opens += open[k];
    }
  }
  u64 agg;
  const u64 excl = block_exclusive_scan<kScanBlock>(opens, SumOp{}, warp_smem, &agg);
  if ((threadIdx.x >> 5) == 0) {
    const u64 p = warp_lookback(status_sum, tile, agg, SumOp{}, flags, 8);
    if ((threadIdx.x & 31) == 0) tile_prefix = p;
  }
  __syncthreads();
  u64 out = tile_prefix + excl;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (!open[k]) continue;
    const u64 i = i0 + k;
    if (out < anchor_cap) {
      anchor_pos[out] = static_cast<Coord>(i);
      anchor_val[out] = static_cast<Coord>(v[k + 1]);
    } else {
      flag_error(flags, kErrQueueOverflow);
    }
    ++out;
  }
  const u64 tiles = (n + kScanTile - 1) / kScanTile;
  if (tile == tiles - 1 && threadIdx.x == 0) *anchor_count = tile_prefix + agg;
}

}  // namespace sufgpu
