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
#include "doubling.cuh"
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

// The radix passes of a tile whose rows hold tile-local composite keys in
// sm.keys and values in sm.vals[0]: 8-bit LSD passes over (local group,
// second key) in shared memory.  Returns the vals buffer holding the result
// (keys end in sm.keys).  Ends with __syncthreads().
__device__ __forceinline__ u32 segsort_radix_passes(SegSortSmem& sm, u32 n_rows, u32 n_groups,
                                                    u32 second_bits) {
  constexpr int kWarps = kSegBlock / 32;
  const u32 lane = threadIdx.x & 31;
  const u32 warp = threadIdx.x >> 5;
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
  return cur;
}

// ckey = (dense id << second_bits) | second for rows [0, count); gstart[g] is
// the first row of group g and *group_count the number of groups.  Writes the
// sorted keys and values of every window that fits (all of them unless
// *big > 0 afterwards).
// count_ptr: the round's active rows (the grid covers an upper bound).  With
// abort set, a window too large for a block also writes abort_tag there so
// that the rest of a host-free round sequence stands still.
// kMinBlocks: blocks per SM the register budget is capped for (the tile's
// 75 KB of shared memory fits three).
template <int kMinBlocks>
static __global__ void __launch_bounds__(kSegBlock, kMinBlocks)
seg_sort_kernel(const u64* __restrict__ ckey, const u32* __restrict__ cval,
                const u64* __restrict__ count_ptr,
                const u32* __restrict__ gstart, const u64* __restrict__ group_count,
                u32 second_bits, u64* __restrict__ out_keys, u32* __restrict__ out_vals,
                u32* big, u64* abort, u64 abort_tag, DeviceFlags* flags, u32 small_group) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SegSortSmem& sm = *reinterpret_cast<SegSortSmem*>(smem_raw);
  const u32 lane = threadIdx.x & 31;
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
  const u32 cur = segsort_radix_passes(sm, n_rows, n_groups, second_bits);
  for (u32 s = threadIdx.x; s < n_rows; s += kSegBlock) {
    const u64 k = sm.keys[s];
    out_keys[lo + s] = (((k >> second_bits) + g_first) << second_bits) | (k & second_mask);
    out_vals[lo + s] = sm.vals[cur][s];
  }
}

// ---- Round step 2 fused with the group sort.
//
// A window's groups are whole inside its block, and so is everything the
// round's second step derives from them: a row of the sorted tile heads a
// new sub-group when its (group, second key) differs from the row before,
// it stays active unless it is a sub-group of one, its SA row is the group's
// head row plus its offset in the group, and its new rank is the group's head
// row plus its sub-group's offset.  Only the next active list needs the rows
// of the windows before (a sum over windows, by decoupled look-back), so the
// block writes SA, ranks and its part of the next active list straight from
// the sorted tile: no sorted keys go back to memory and no second kernel
// reads them.  The second keys were all read by round_keys before this
// kernel starts, so writing ranks here races with nothing.
//
// A window too large for a block sets *big and the round's abort word (when
// given) and the host redoes the round from the untouched keys with the
// global passes and round_rank; the rows this kernel already wrote get the
// same values again (both sorts are stable, so the order is the same).
struct SegRankSmem {
  SegSortSmem sort;
  u32 perm[kSegCap];  // counting path: tile slot of each sorted row
  u64 prefix;         // the window's first slot in the next active list
  u32 tile;
  u32 counted;        // 1: sorted rows are perm[] indirect
};

static __global__ void __launch_bounds__(kSegBlock, 2)
seg_rank_kernel(const u64* __restrict__ ckey, const u32* __restrict__ cval, RoundState rs,
                const u32* __restrict__ gstart, const u32* __restrict__ ghead,
                const u64* __restrict__ group_count, u64 group_cap, u32 second_bits, u64 rows,
                u32* __restrict__ sa, u32* __restrict__ rank, u32* __restrict__ next_active,
                u64* status, u32* tile_counter, u32* big, u64* abort, u64 abort_tag,
                DeviceFlags* flags, u32 small_group) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SegRankSmem& sr = *reinterpret_cast<SegRankSmem*>(smem_raw);
  SegSortSmem& sm = sr.sort;
  const u32 lane = threadIdx.x & 31;
  const u32 warp = threadIdx.x >> 5;
  if (round_skipped(rs)) return;
  const u64 count = *rs.count;
  if (count == 0) {  // converged: the next round has nothing either
    if (blockIdx.x == 0 && threadIdx.x == 0) *rs.next_count = 0;
    return;
  }
  // Windows are claimed in order (the look-back needs it); every claimed
  // window below `windows` publishes its count, skipped or not.
  const u32 w = claim_tile(tile_counter, &sr.tile);
  const u64 windows = (count + kSegWindow - 1) / kSegWindow;
  if (w >= windows) return;
  if (threadIdx.x == 0) {
    const u64 groups = *group_count;
    const u64 w0 = static_cast<u64>(w) * kSegWindow;
    const u64 g_lo = w0 == 0 ? 0 : first_group_at(gstart, groups, w0);
    const u64 g_hi = first_group_at(gstart, groups, w0 + kSegWindow);
    u64 lo = g_lo < groups ? gstart[g_lo] : count;
    u64 hi = g_hi < groups ? gstart[g_hi] : count;
    if (lo > hi || hi > count) {  // inconsistent group table: write nothing
      flag_error(flags, kErrBounds);
      lo = hi = 0;
    }
    if (hi - lo > static_cast<u64>(kSegCap)) {  // the host redoes this round
      atomicAdd(big, 1u);
      if (abort) *abort = abort_tag;
      lo = hi = 0;
    }
    sm.range[0] = static_cast<u32>(lo);
    sm.range[1] = static_cast<u32>(hi);
    sm.range[2] = static_cast<u32>(g_lo);
    sm.range[3] = static_cast<u32>(g_hi - g_lo);
    sm.largest = 0;
  }
  __syncthreads();
  const u32 lo = sm.range[0];
  const u32 n_rows = sm.range[1] - lo;
  const u32 g_first = sm.range[2];
  const u32 n_groups = sm.range[3];
  const u64 second_mask = (1ull << second_bits) - 1;
  // Sort the window's rows (uniform branches: n_rows is the block's).
  u32 cur = 0;
  if (n_rows > 0) {
    for (u32 s = threadIdx.x; s < n_rows; s += kSegBlock) {
      const u64 k = ckey[lo + s];
      sm.keys[s] = (((k >> second_bits) - g_first) << second_bits) | (k & second_mask);
      sm.vals[0][s] = cval[lo + s];
    }
    u32 largest = 0;
    for (u32 g = threadIdx.x; g < n_groups; g += kSegBlock) {
      const u32 gs = gstart[g_first + g];
      const u32 ge = g + 1 < n_groups ? gstart[g_first + g + 1] : lo + n_rows;
      largest = max(largest, ge - gs);
    }
    for (int offset = 16; offset > 0; offset >>= 1) {
      largest = max(largest, __shfl_xor_sync(0xffffffffu, largest, offset));
    }
    if (lane == 0 && largest) atomicMax(&sm.largest, largest);
    __syncthreads();
    if (sm.largest <= small_group) {
      // Counting: sorted slot gs + below of each row; perm holds the rows.
      for (u32 s = threadIdx.x; s < n_rows; s += kSegBlock) sr.perm[s] = s;
      __syncthreads();
      for (u32 s = threadIdx.x; s < n_rows; s += kSegBlock) {
        const u64 k = sm.keys[s];
        const u32 g = static_cast<u32>(k >> second_bits);
        const u32 gs = g < n_groups ? gstart[g_first + g] - lo : n_rows;
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
        sr.perm[gs + below] = s;
      }
      if (threadIdx.x == 0) sr.counted = 1;
    } else {
      cur = segsort_radix_passes(sm, n_rows, n_groups, second_bits);
      if (threadIdx.x == 0) sr.counted = 0;
    }
    __syncthreads();
  }
  const bool counted = n_rows > 0 && sr.counted;
  // Sorted row t of the tile: its slot in sm.keys / sm.vals[...].
  auto slot_of = [&](u32 t) -> u32 { return counted ? min(sr.perm[t], n_rows - 1) : t; };
  const u32* vals = counted ? sm.vals[0] : sm.vals[cur];

  // Sub-group heads: bit i of `heads` for sorted row base + i (i <= 16; rows
  // past the tile count as heads, so the last row of the window closes its
  // sub-group).
  const u32 base = threadIdx.x * kSegItems;
  u32 heads = 0;
  u64 prev = base > 0 && base - 1 < n_rows ? sm.keys[slot_of(base - 1)] : ~0ull;
#pragma unroll
  for (int i = 0; i <= kSegItems; ++i) {
    const u32 t = base + i;
    bool h = true;
    if (t < n_rows) {
      const u64 k = sm.keys[slot_of(t)];
      h = t == 0 || k != prev;
      prev = k;
    }
    heads |= static_cast<u32>(h) << i;
  }
  u64 head_max = 0;
  u32 keep = 0;
#pragma unroll
  for (int i = 0; i < kSegItems; ++i) {
    const u32 t = base + i;
    if (t < n_rows) {
      if ((heads >> i) & 1) head_max = t;
      keep += ((heads >> i) & (heads >> (i + 1)) & 1) ? 0u : 1u;
    }
  }
  u64 agg_max, agg_keep;
  const u64 excl_max = block_exclusive_scan<kSegBlock>(head_max, MaxOp{}, sm.warp_scan, &agg_max);
  const u64 excl_keep = block_exclusive_scan<kSegBlock>(keep, SumOp{}, sm.warp_scan, &agg_keep);
  if (warp == 0) {
    const u64 p = warp_lookback(status, w, agg_keep, SumOp{}, flags, 23);
    if (lane == 0) sr.prefix = p;
  }
  __syncthreads();
  const u64 out_base = sr.prefix;
  u64 sub = excl_max;  // tile-local head of the current sub-group
  u64 out = out_base + excl_keep;
#pragma unroll
  for (int i = 0; i < kSegItems; ++i) {
    const u32 t = base + i;
    if (t >= n_rows) break;
    const bool h = (heads >> i) & 1;
    if (h) sub = t;
    const bool kept = !(h && ((heads >> (i + 1)) & 1));
    const u32 slot = slot_of(t);
    const u32 g = static_cast<u32>(sm.keys[slot] >> second_bits);
    const u32 p = vals[slot];
    const u64 dense = static_cast<u64>(g_first) + g;
    u32 gf = 0, gh = 0;
    bool bad = g >= n_groups || dense >= group_cap;
    if (!bad) {
      gf = gstart[dense];
      gh = ghead[dense];
    }
    const u64 a = static_cast<u64>(lo) + t;
    const u64 row = static_cast<u64>(gh) + (a - gf);
    bad = bad || a < gf || row >= rows || p >= rows;
    if (bad) {
      flag_error(flags, kErrBounds);
      if (kept) ++out;
      continue;
    }
    sa[row] = p;
    rank[p] = static_cast<u32>(gh + (lo + sub - gf));
    if (kept) next_active[out++] = p;
  }
  if (w == windows - 1 && threadIdx.x == 0) *rs.next_count = out_base + agg_keep;
}

// After seg_rank_kernel: the round's bookkeeping, unless the round (or an
// earlier one of the graph) was aborted, in which case the host redoes it.
static __global__ void round_close_kernel(RoundState rs) {
  if (round_skipped(rs)) return;
  if (rs.double_h) *rs.h *= 2;
  if (rs.totals) {
    rs.totals[0] += *rs.count;
    rs.totals[1] += 1;
  }
}

}  // namespace sufgpu
