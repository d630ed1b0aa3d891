// Segmented sort of a doubling round's composite keys inside shared memory.
//
// Rows arrive grouped (each group is a contiguous run of the active list), so
// a tile whose groups are all small (at most small_group rows) needs no
// passes at all: each row's place in its group is the number of rows of the
// group with a smaller second key (ties by position), O(group size) shared
// memory reads per row.  Tiles with a larger group take the radix passes.
//
// A round sorts the active rows by (dense group id, second key), but rows only
// move inside their own group, and groups are small (copies of a repeat).  So
// instead of LSD passes over all id and key bits through HBM, each block takes
// the groups that start inside one 2048-row window of the active list (at most
// 4096 rows in all), replaces the global group id by a tile-local one, and
// sorts the tile in shared memory with 8-bit LSD passes over
// (local id, second key): one read and one write of HBM per row, no look-back.
// A window whose groups exceed the tile (a group of more than 2048 rows
// starting in it) is counted in *big; the host then sorts that round with the
// global passes instead, so results never depend on group sizes.
#pragma once

#include "common.cuh"
#include "radix.cuh"
#include "scan.cuh"

namespace sufgpu {

constexpr int kSegBlock = 256;
constexpr int kSegItems = 16;
constexpr int kSegCap = kSegBlock * kSegItems;  // rows one block sorts
constexpr int kSegWindow = kSegCap / 2;          // group starts per block
// Default for small_group: tiles whose groups all have at most this many
// rows rank each row by counting inside its group instead of running the
// radix passes.
constexpr u32 kSegSmallGroup = 96;

struct SegSortSmem {
  u64 keys[kSegCap];
  u32 vals[2][kSegCap];
  u32 warp_hist[kSegBlock / 32][kRadixDigits];
  u32 digit_excl[kRadixDigits];
  u64 warp_scan[kSegBlock / 32];
  u32 range[4];  // lo, hi, first group, groups
  u32 largest;   // rows of the tile's largest group
};

// First index in gstart[0, groups) with gstart[i] >= x (groups if none).
__device__ __forceinline__ u64 first_group_at(const u32* gstart, u64 groups, u64 x) {
  u64 lo = 0, hi = groups;
  while (lo < hi) {
    const u64 mid = (lo + hi) >> 1;
    if (gstart[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// ckey = (dense id << second_bits) | second for rows [0, count); gstart[g] is
// the first row of group g and *group_count the number of groups.  Writes the
// sorted keys and values of every window that fits (all of them unless
// *big > 0 afterwards).
// count_ptr: the round's active rows (the grid covers an upper bound).  With
// abort set, a window too large for a block also writes abort_tag there so
// that the rest of a host-free round sequence stands still.
static __global__ void __launch_bounds__(kSegBlock, 2)
seg_sort_kernel(const u64* __restrict__ ckey, const u32* __restrict__ cval,
                const u64* __restrict__ count_ptr,
                const u32* __restrict__ gstart, const u64* __restrict__ group_count,
                u32 second_bits, u64* __restrict__ out_keys, u32* __restrict__ out_vals,
                u32* big, u64* abort, u64 abort_tag, DeviceFlags* flags, u32 small_group) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SegSortSmem& sm = *reinterpret_cast<SegSortSmem*>(smem_raw);
  constexpr int kWarps = kSegBlock / 32;
  const u32 lane = threadIdx.x & 31;
  const u32 warp = threadIdx.x >> 5;
  if (abort && *abort) return;
  const u64 count = *count_ptr;
  if (static_cast<u64>(blockIdx.x) * kSegWindow >= count) return;
  if (threadIdx.x == 0) {
    const u64 groups = *group_count;
    const u64 w0 = static_cast<u64>(blockIdx.x) * kSegWindow;
    const u64 g_lo = w0 == 0 ? 0 : first_group_at(gstart, groups, w0);
    const u64 g_hi = first_group_at(gstart, groups, w0 + kSegWindow);
    u64 lo = g_lo < groups ? gstart[g_lo] : count;
    u64 hi = g_hi < groups ? gstart[g_hi] : count;
    if (lo > hi || hi > count) {  // inconsistent group table: write nothing
      flag_error(flags, kErrBounds);
      lo = hi = 0;
    }
    sm.range[0] = static_cast<u32>(lo);
    sm.range[1] = static_cast<u32>(hi);
    sm.range[2] = static_cast<u32>(g_lo);
    sm.range[3] = static_cast<u32>(g_hi - g_lo);
  }
  __syncthreads();
  const u32 lo = sm.range[0];
  const u32 n_rows = sm.range[1] - lo;
  const u32 g_first = sm.range[2];
  const u32 n_groups = sm.range[3];
  if (n_rows == 0) return;
  if (n_rows > static_cast<u32>(kSegCap)) {
    if (threadIdx.x == 0) {
      atomicAdd(big, 1u);
      if (abort) *abort = abort_tag;
    }
    return;
  }
  // Tile-local composite keys: (local group << second_bits) | second.
  const u64 second_mask = (1ull << second_bits) - 1;
  if (threadIdx.x == 0) sm.largest = 0;
  for (u32 s = threadIdx.x; s < n_rows; s += kSegBlock) {
    const u64 k = ckey[lo + s];
    sm.keys[s] = (((k >> second_bits) - g_first) << second_bits) | (k & second_mask);
    sm.vals[0][s] = cval[lo + s];
  }
  // The tile's largest group.
  u32 largest = 0;
  for (u32 g = threadIdx.x; g < n_groups; g += kSegBlock) {
    const u32 gs = gstart[g_first + g];
    const u32 ge = g + 1 < n_groups ? gstart[g_first + g + 1] : lo + n_rows;
    largest = max(largest, ge - gs);
  }
  for (int offset = 16; offset > 0; offset >>= 1) {
    largest = max(largest, __shfl_xor_sync(0xffffffffu, largest, offset));
  }
  __syncthreads();  // sm.largest = 0 is visible
  if (lane == 0 && largest) atomicMax(&sm.largest, largest);
  __syncthreads();
  if (sm.largest <= small_group) {
    // Rank by counting inside the group; positions are tile-local.
    for (u32 s = threadIdx.x; s < n_rows; s += kSegBlock) {
      const u64 k = sm.keys[s];
      const u32 g = static_cast<u32>(k >> second_bits);
      const u32 gs = gstart[g_first + g] - lo;
      const u32 ge = g + 1 < n_groups ? gstart[g_first + g + 1] - lo : n_rows;
      if (gs > s || ge <= s || ge > n_rows) {  // inconsistent group table
        flag_error(flags, kErrBounds);
        continue;
      }
      const u64 mine = k & second_mask;
      u32 below = 0;
      for (u32 j = gs; j < ge; ++j) {
        const u64 other = sm.keys[j] & second_mask;
        below += (other < mine) || (other == mine && j < s);
      }
      out_keys[lo + gs + below] = (static_cast<u64>(g + g_first) << second_bits) | mine;
      out_vals[lo + gs + below] = sm.vals[0][s];
    }
    return;
  }
  const u32 total_bits = second_bits + max(1u, bits_for(n_groups > 0 ? n_groups - 1 : 0));
  const u32 passes = (total_bits + kRadixBits - 1) / kRadixBits;
  // Each warp ranks a contiguous run of `items` x 32 slots (contiguous per
  // warp keeps the ranking stable); only as many items as the tile needs.
  const u32 items = (n_rows + kSegBlock - 1) / kSegBlock;
  const u32 warp_base = warp * 32 * items;
  const u32 lanemask_lt = (1u << lane) - 1;
  u32 cur = 0;
  __syncthreads();
  for (u32 p = 0; p < passes; ++p) {
    const u32 shift = p * kRadixBits;
    for (int d = lane; d < kRadixDigits; d += 32) sm.warp_hist[warp][d] = 0;
    u64 key[kSegItems];
    u32 rank[kSegItems];
#pragma unroll
    for (int i = 0; i < kSegItems; ++i) {
      const u32 slot = warp_base + i * 32 + lane;
      key[i] = (i < items && slot < n_rows) ? sm.keys[slot] : ~0ull;
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < kSegItems; ++i) {
      if (i >= items) break;  // uniform across the block
      const u32 slot = warp_base + i * 32 + lane;
      const bool valid = slot < n_rows;
      const u32 digit = valid ? static_cast<u32>((key[i] >> shift) & 0xff) : 0x100u;
      u32 peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
      for (int b = 0; b < kRadixBits; ++b) {
        const bool bit = (digit >> b) & 1;
        const u32 vote = __ballot_sync(0xffffffffu, bit);
        peers &= bit ? vote : ~vote;
      }
      if (!valid) peers = 1u << lane;
      const u32 leader = __ffs(peers) - 1;
      u32 base = 0;
      if (valid && lane == leader) {
        base = sm.warp_hist[warp][digit];
        sm.warp_hist[warp][digit] = base + __popc(peers);
      }
      base = __shfl_sync(0xffffffffu, base, leader);
      rank[i] = base + __popc(peers & lanemask_lt);
      __syncwarp();
    }
    __syncthreads();
    const u32 d = threadIdx.x;
    u32 digit_count = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      const u32 c = sm.warp_hist[w][d];
      sm.warp_hist[w][d] = digit_count;
      digit_count += c;
    }
    u64 tile_total;
    sm.digit_excl[d] = static_cast<u32>(
        block_exclusive_scan<kSegBlock>(digit_count, SumOp{}, sm.warp_scan, &tile_total));
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kSegItems; ++i) {
      if (i >= items) break;
      const u32 slot = warp_base + i * 32 + lane;
      if (slot < n_rows) {
        const u32 digit = static_cast<u32>((key[i] >> shift) & 0xff);
        const u32 ls = sm.digit_excl[digit] + sm.warp_hist[warp][digit] + rank[i];
        sm.keys[ls] = key[i];
        sm.vals[cur ^ 1][ls] = sm.vals[cur][slot];
      }
    }
    cur ^= 1;
    __syncthreads();
  }
  for (u32 s = threadIdx.x; s < n_rows; s += kSegBlock) {
    const u64 k = sm.keys[s];
    out_keys[lo + s] = (((k >> second_bits) + g_first) << second_bits) | (k & second_mask);
    out_vals[lo + s] = sm.vals[cur][s];
  }
}

}  // namespace sufgpu
