// Prefix-doubling suffix sort kernels.
//
// Seed: every position gets a 64-bit key packing its first s symbols (symbols
// remapped to 1..sigma, 0 = past the end of the instance; or, for a DNA text,
// 2 bits per A/C/G/T plus a tag, see TwoBitSeed), and (key, position) pairs
// are radix sorted.  Groups of equal keys then get their head row as rank;
// rows in groups of two or more go to the active list.
//
// Round (prefix length h -> 2h): each active position p gets the composite key
// (dense group id, rank[p+h] + 1 or 0 past the end); a radix sort of the
// active list orders every group by its second key; new heads, SA rows and
// ranks are written, and positions that became singletons retire.  Only the
// still-unsorted positions are ever touched after the seed.
#pragma once

#include <cooperative_groups.h>

#include "common.cuh"
#include "scan.cuh"

namespace sufgpu {

constexpr int kScanBlock = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanBlock * kScanItems;

// Segment bounds for one instance-aware kernel.  count == 1 with begin = {0, n}
// for a single reference.
// When `end` is set the segments need not be contiguous (the served engine's
// arena): segment j is [begin[j], end[j]) and begin has count entries.
struct Segments {
  const u64* begin;  // count+1 offsets into the concatenated text
  u32 count;
  const u64* end = nullptr;
};

__device__ __forceinline__ u64 segment_end(const Segments& s, u64 x) {
  if (s.end) return s.end[s.count == 1 ? 0 : find_segment(s.begin, s.count, x)];
  if (s.count == 1) return s.begin[1];
  return s.begin[find_segment(s.begin, s.count, x) + 1];
}

__device__ __forceinline__ bool is_segment_start(const Segments& s, u64 x) {
  if (x == 0) return true;
  if (s.count == 1) return false;
  return s.begin[find_segment(s.begin, s.count, x)] == x;
}

// Byte histogram of the text (for the symbol remap).  Runs of one byte value
// are counted in registers first so long N runs do not serialise on one
// shared-memory counter.
static __global__ void __launch_bounds__(256)
alphabet_histogram_kernel(const u8* __restrict__ text, u64 n,
                          u32* __restrict__ hist) {
  __shared__ u32 local[256];
  local[threadIdx.x] = 0;
  __syncthreads();
  const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x * 16;
  for (u64 base = (static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x) * 16;
       base < n; base += stride) {
    u8 bytes[16];
    if (base + 16 <= n) {
      const uint4 v = *reinterpret_cast<const uint4*>(text + base);
      const u32 w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int i = 0; i < 16; ++i) bytes[i] = static_cast<u8>(w[i >> 2] >> ((i & 3) * 8));
    } else {
      for (int i = 0; i < 16; ++i) bytes[i] = base + i < n ? text[base + i] : 0;
    }
    const int valid = base + 16 <= n ? 16 : static_cast<int>(n - base);
    u32 run_value = bytes[0];
    u32 run_len = 0;
    for (int i = 0; i < valid; ++i) {
      if (bytes[i] == run_value) {
        ++run_len;
      } else {
        atomicAdd(&local[run_value], run_len);
        run_value = bytes[i];
        run_len = 1;
      }
    }
    if (run_len) atomicAdd(&local[run_value], run_len);
  }
  __syncthreads();
  if (local[threadIdx.x]) atomicAdd(&hist[threadIdx.x], local[threadIdx.x]);
}

// Seed keys.  Each thread computes kSeedRun consecutive keys by sliding a
// window over text staged in shared memory (tile + halo).  code[] maps bytes
// to 1..sigma (sigma <= 256, so 16-bit codes); symbols at or beyond the
// instance end contribute 0.  The tile's keys are staged in shared memory and
// written out coalesced, and the digit histograms of every radix pass over
// bits [0, passes*8) are accumulated on the way (per instance segment), so
// the seed sort needs no separate histogram read of the keys.
constexpr int kSeedBlock = 256;
constexpr int kSeedRun = 16;
constexpr int kSeedTile = kSeedBlock * kSeedRun;
constexpr int kSeedHalo = 64;
constexpr int kMaxSeedPasses = 8;  // 64-bit keys, 8-bit digits
// Keys per thread when the kernel only counts (the fused first pass writes
// the keys): no key buffer in shared memory, so each thread can slide its
// window over four times as many positions, and the window it builds from
// scratch at its first position (s symbols) is paid once per 64 keys.
constexpr int kSeedCountRun = 64;

// kRun keys per thread; the key buffer exists for the position-order write
// (kRun == kSeedRun) only.
template <int kRun>
struct SeedSmemT {
  u64 keys[kRun == kSeedRun ? kSeedBlock * kRun : 1];
  u32 hist[8][256];
  u16 code[256];
  __align__(16) u8 window[kSeedBlock * kRun + kSeedHalo];
};
using SeedSmem = SeedSmemT<kSeedRun>;

// Two-bit seed for texts of four consecutive regular symbols (A, C, G, T in
// the logical text) and few others.  A window's key is the 2-bit codes of its
// regular symbols followed by a 2-bit tag t:
//   t = 1  every symbol regular: the codes of the whole window;
//   t = 0  its first irregular symbol (at offset j) is below the regular ones
//          or past the end: the codes of offsets [0, j), then all A;
//   t = 2  that symbol is above them: the codes of [0, j), then all T;
//   t = 3  every symbol is the largest symbol `hi` (inside a run of N).
// The map is monotone in the windows' order, one-to-one on the t = 1 and
// t = 3 windows, and strict between a t = 1 / t = 3 window and any other, so
// after the sort every group of t = 1 or t = 3 keys is exact and only rows of
// the same t = 0 / t = 2 key ("rare rows") may hold different windows in the
// wrong order.  Their exact keys (the code-table key) go to a side list that
// is sorted on its own; seed ranks place them from it.
struct TwoBitSeed {
  u32 lo = 0;         // code of the first regular symbol (regular: lo..lo+3)
  u32 hi = 0;         // code of the largest symbol when above the regular ones
  u64 all_hi = 0;     // exact key of a window of s x hi
  u64* rare_key = nullptr;  // exact keys of rare rows (unordered)
  u32* rare_pos = nullptr;
  u64 rare_cap = 0;
  u64* rare_count = nullptr;  // may exceed rare_cap: the host then falls back
  // Batches: a rare row's listed key carries its instance above the exact
  // key's bits (instance << inst_shift | exact), so the list sorts by
  // instance, then key.  0 for one instance.
  u32 inst_shift = 0;
};

// Two-bit key from the window's exact key, its regular codes k2 (2 bits per
// symbol, 0 for irregular ones) and its irregular mask (bit s-1-k set when
// offset k is irregular).
__host__ __device__ __forceinline__ u64 two_bit_key(u64 exact, u64 k2, u32 irregular, u32 s,
                                                    u32 bits, const TwoBitSeed& tb) {
  if (irregular == 0) return (k2 << 2) | 1;
#ifdef __CUDA_ARCH__
  const u32 top = 31 - __clz(irregular);
#else
  u32 top = 31;
  while (!((irregular >> top) & 1u)) --top;
#endif
  const u32 j = s - 1 - top;  // first irregular offset
  const u32 cj = static_cast<u32>(exact >> (bits * (s - 1 - j))) & ((1u << bits) - 1);
  const u32 tail = 2 * (s - j);
  const u64 head = (k2 >> tail) << tail;
  if (cj < tb.lo) return head << 2;
  const u64 fill = (1ull << tail) - 1;
  if (j == 0 && tb.hi && exact == tb.all_hi) return ((head | fill) << 2) | 3;
  return ((head | fill) << 2) | 2;
}

// The same from the exact key alone (s symbols of `bits`).
__host__ __device__ __forceinline__ u64 two_bit_of_exact(u64 exact, u32 s, u32 bits,
                                                         const TwoBitSeed& tb) {
  u64 k2 = 0;
  u32 irregular = 0;
  for (u32 k = 0; k < s; ++k) {
    const u32 c = static_cast<u32>(exact >> (bits * (s - 1 - k))) & ((1u << bits) - 1);
    const bool reg = c >= tb.lo && c < tb.lo + 4;
    k2 = (k2 << 2) | (reg ? c - tb.lo : 0u);
    irregular = (irregular << 1) | (reg ? 0u : 1u);
  }
  return two_bit_key(exact, k2, irregular, s, bits, tb);
}

// packed_shift > 0 selects the packed seed: key = (prefix << packed_shift) |
// instance-local index (no value array); histograms then cover the passes
// over bits [packed_shift, packed_shift + 8*passes).
// kTwoBit: sort keys are two-bit keys (one instance); rare rows also append
// (exact key, position) to tb's list.
// kRun = kSeedCountRun: histograms and rare list only (keys must be null).
template <bool kTwoBit, int kRun = kSeedRun>
static __global__ void __launch_bounds__(kSeedBlock)
seed_keys_kernel(const u8* __restrict__ text, u64 n, Segments segs,
                 const u16* __restrict__ code_table, u32 bits, u32 symbols,
                 u32 passes, u32* __restrict__ hist_out, u32 packed_shift,
                 u64* __restrict__ keys, u32* __restrict__ vals, TwoBitSeed tb) {
  constexpr int kTile = kSeedBlock * kRun;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SeedSmemT<kRun>& sm = *reinterpret_cast<SeedSmemT<kRun>*>(smem_raw);
  sm.code[threadIdx.x] = code_table[threadIdx.x];
  for (int i = threadIdx.x; i < 8 * 256; i += kSeedBlock) (&sm.hist[0][0])[i] = 0;
  const u64 tile_first = static_cast<u64>(blockIdx.x) * kTile;
  // Stage tile + halo as 16-byte vectors (the text buffer is padded).
  for (int i = threadIdx.x; i < (kTile + kSeedHalo) / 16; i += kSeedBlock) {
    const u64 at = tile_first + static_cast<u64>(i) * 16;
    uint4 v = make_uint4(0, 0, 0, 0);
    if (at < n) v = *reinterpret_cast<const uint4*>(text + at);
    *reinterpret_cast<uint4*>(sm.window + i * 16) = v;
  }
  __syncthreads();
  const u32 block_seg = segs.count == 1 ? 0 : find_segment(segs.begin, segs.count, tile_first);
  const u64 mask = symbols * bits >= 64 ? ~0ull : ((1ull << (symbols * bits)) - 1);
  const u64 mask2 = 2 * symbols >= 64 ? ~0ull : ((1ull << (2 * symbols)) - 1);
  const u32 smask = symbols >= 32 ? ~0u : ((1u << symbols) - 1);
  const u32 local0 = threadIdx.x * kRun;
  u64 pos = tile_first + local0;
  u32 seg = segs.count == 1 ? 0 : (pos < n ? find_segment(segs.begin, segs.count, pos) : block_seg);
  u64 end = pos < n ? segs.begin[seg + 1] : n;
  u64 seg_lo = pos < n ? segs.begin[seg] : 0;
  u64 key = 0, k2 = 0;
  u32 irregular = 0;
  bool fresh = true;
  // Pushes the code of one more symbol into the window state.
  auto push = [&](u32 c) {
    key = ((key << bits) | c) & mask;
    if (kTwoBit) {
      const bool reg = c >= tb.lo && c < tb.lo + 4;
      k2 = ((k2 << 2) | (reg ? c - tb.lo : 0u)) & mask2;
      irregular = ((irregular << 1) | (reg ? 0u : 1u)) & smask;
    }
  };
  u32 run_digit[kMaxSeedPasses], run_len[kMaxSeedPasses];
#pragma unroll
  for (int p = 0; p < kMaxSeedPasses; ++p) run_digit[p] = run_len[p] = 0;
#pragma unroll 1
  for (int r = 0; r < kRun; ++r, ++pos) {
    const bool valid = pos < n;
    if (valid && pos >= end) {  // crossed into the next instance
      seg = find_segment(segs.begin, segs.count, pos);
      end = segs.begin[seg + 1];
      seg_lo = segs.begin[seg];
      fresh = true;
    }
    const u32 local = local0 + r;
    u64 sort_key = 0;
    bool rare = false;
    if (valid) {
      if (fresh) {
        key = k2 = 0;
        irregular = 0;
        for (u32 t = 0; t < symbols; ++t) push(pos + t < end ? sm.code[sm.window[local + t]] : 0u);
        fresh = false;
      } else {
        const u64 q = pos + symbols - 1;
        push(q < end ? sm.code[sm.window[local + symbols - 1]] : 0u);
      }
      sort_key = key;
      if (kTwoBit) {
        sort_key = two_bit_key(key, k2, irregular, symbols, bits, tb);
        rare = (sort_key & 1) == 0;
      }
      if constexpr (kRun == kSeedRun) {
        sm.keys[local] = packed_shift ? (sort_key << packed_shift) | (pos - seg_lo) : sort_key;
      }
    }
    if (kTwoBit) {
      const u64 slot = warp_append(tb.rare_count, rare);
      if (rare && slot < tb.rare_cap) {
        tb.rare_key[slot] = tb.inst_shift ? key | (static_cast<u64>(seg) << tb.inst_shift) : key;
        tb.rare_pos[slot] = static_cast<u32>(pos);
      }
    }
    // Histogram of every pass.  The thread's keys are consecutive
    // positions, so equal digits come in runs (long runs of one symbol give
    // whole runs of equal keys): count each run in registers and add it with
    // one shared-memory atomic when the digit changes.
    const bool mine = valid && seg == block_seg;
#pragma unroll
    for (int p = 0; p < kMaxSeedPasses; ++p) {
      if (p >= static_cast<int>(passes)) break;
      const u32 digit = static_cast<u32>((sort_key >> (p * 8)) & 0xff);
      if (mine) {
        if (run_len[p] && digit == run_digit[p]) {
          ++run_len[p];
        } else {
          if (run_len[p]) atomicAdd(&sm.hist[p][run_digit[p]], run_len[p]);
          run_digit[p] = digit;
          run_len[p] = 1;
        }
      } else if (valid) {
        atomicAdd(&hist_out[(static_cast<u64>(seg) * passes + p) * 256 + digit], 1u);
      }
    }
  }
#pragma unroll
  for (int p = 0; p < kMaxSeedPasses; ++p) {
    if (p < static_cast<int>(passes) && run_len[p]) {
      atomicAdd(&sm.hist[p][run_digit[p]], run_len[p]);
    }
  }
  __syncthreads();
  // keys == null: histograms (and the rare list) only; seed_sorted_kernel
  // generates the keys again and writes them partitioned by the first digit.
  if constexpr (kRun == kSeedRun) {
    for (u32 i = threadIdx.x; keys && i < kTile; i += kSeedBlock) {
      const u64 at = tile_first + i;
      if (at < n) {
        keys[at] = sm.keys[i];
        if (!packed_shift) vals[at] = static_cast<u32>(at);
      }
    }
  }
  for (u32 i = threadIdx.x; i < passes * 256; i += kSeedBlock) {
    const u32 c = (&sm.hist[0][0])[i];
    if (c) atomicAdd(&hist_out[static_cast<u64>(block_seg) * passes * 256 + i], c);
  }
}

// After the seed sort: head flags, head-row ranks (rank[SA[r]] = head row of
// r; the one full random scatter of the build, at the device's scattered-store
// rate) and the initial active list.  Two scans share the tile: a max-scan of
// head rows and a sum-scan of active flags (the compaction).
// Also writes the LCP of every seed-group head row straight from the keys: two
// different seed keys share exactly (leading zeros of their XOR - unused top
// bits) / bits symbols.  Rows inside a seed group get kLcpUnknown and are
// resolved from the text later (their LCP is at least the seed length).
constexpr u32 kLcpUnknown = 0xffffffffu;

// Rare rows of a two-bit seed (one instance), sorted by their exact keys:
// positions and, in the same order (so ascending too), their two-bit keys.
struct RareRows {
  const u64* key = nullptr;
  const u32* pos = nullptr;
  const u64* k2 = nullptr;
  u64 count = 0;
  const u8* text = nullptr;
};

// First index in v[lo, hi) with v[i] >= x (hi if none).
__device__ __forceinline__ u64 lower_bound_u64(const u64* v, u64 lo, u64 hi, u64 x) {
  while (lo < hi) {
    const u64 mid = (lo + hi) >> 1;
    if (v[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Common prefix of the s-symbol windows at p != q of a text of n symbols.
__device__ __forceinline__ u32 window_lcp(const u8* text, u64 n, u64 p, u64 q, u32 s) {
  u32 l = 0;
  while (l < s && p + l < n && q + l < n && text[p + l] == text[q + l]) ++l;
  return l;
}

// Ranks leave as (position << 32 | head row) words in row order (pairs), so
// the write is coalesced; the window scatter below turns them into rank[].
// kTwoBit: keys are two-bit keys (one instance).  Groups of t = 1 / t = 3
// keys are exact and handled here; rows of t = 0 / t = 2 keys (rare rows) get
// placeholder pairs and SA entries, no LCP (nor the row after them), and stay
// off the active list: rare_place_kernel and rare_active_kernel finish them.
// Registers capped for five blocks per SM (measured: 43.6 against 46.2 ms at
// 3.1 Gbp; 19.1 against 19.9 ms for 256 bacterial references).
template <bool kTwoBit>
static __global__ void __launch_bounds__(kScanBlock, 5)
seed_rank_kernel(const u64* __restrict__ keys, u32* __restrict__ sa,
                 u64 n, Segments segs, u32 packed_shift, u32 bits, u32 symbols,
                 u64* __restrict__ pairs, u32* __restrict__ lcp,
                 u32* __restrict__ active, u64* status_max, u64* status_sum,
                 u32* tile_counter, u64* active_count, DeviceFlags* flags,
                 u32 run_keys = 0, u32 local_pairs = 0) {
  __shared__ u64 warp_smem[kScanBlock / 32];
  __shared__ u64 tile_prefix[2];
  __shared__ u32 tile_slot;
  const u32 tile = claim_tile(tile_counter, &tile_slot);
  const u64 row0 = static_cast<u64>(tile) * kScanTile + threadIdx.x * kScanItems;

  // Compare only the prefix part of packed keys.
  u64 k[kScanItems + 2];  // rows row0-1 .. row0+kScanItems
#pragma unroll
  for (int i = 0; i < kScanItems + 2; ++i) {
    const long long r = static_cast<long long>(row0) - 1 + i;
    k[i] = (r >= 0 && static_cast<u64>(r) < n) ? keys[r] >> packed_shift : 0;
  }
  SegCursor cur;
  bool head[kScanItems + 1];
  const u32 unused_top = kTwoBit ? 64 - (2 * symbols + 2) : 64 - bits * symbols;
#pragma unroll
  for (int i = 0; i < kScanItems + 1; ++i) {
    const u64 r = row0 + i;
    bool start = r >= n;
    if (!start) {
      cur.locate(segs.begin, segs.count, r);
      start = r == cur.lo;
    }
    head[i] = start || k[i + 1] != k[i];
    if (i < kScanItems && r < n) {
      u32 v = kLcpUnknown;
      bool write = true;
      const u32 x = static_cast<u32>(__clzll(static_cast<long long>(k[i + 1] ^ k[i])));
      if (start) {
        v = 0;
      } else if (kTwoBit) {
        const u32 t = static_cast<u32>(k[i + 1] & 3), tp = static_cast<u32>(k[i] & 3);
        if (!(t & 1) || (head[i] && !(tp & 1))) write = false;  // a rare row involved
        else if (head[i]) v = t != tp ? 0 : (x - unused_top) / 2;
      } else if (head[i]) {
        v = (x - unused_top) / bits;
      }
      if (write) lcp[r] = v;
    }
  }
  // With run_keys set, rows whose seed key is one symbol repeated s times
  // (members of long runs) stay off the active list: the run split places
  // them (runs.cuh).
  const u32 sym_bits = kTwoBit ? 2 : bits;
  const u64 run_low = symbols > 1 ? (1ull << (sym_bits * (symbols - 1))) - 1 : 0;
  bool active_row[kScanItems];
  u64 head_max = 0;  // inclusive running max within the thread
  u32 act = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const u64 r = row0 + i;
    active_row[i] = false;
    if (r < n) {
      if (head[i]) head_max = r;
      const u64 prefix = kTwoBit ? k[i + 1] >> 2 : k[i + 1];
      const bool rare_row = kTwoBit && !(k[i + 1] & 1);
      const bool run_member = run_keys && !rare_row && (prefix >> sym_bits) == (prefix & run_low);
      active_row[i] = !(head[i] && head[i + 1]) && !run_member && !rare_row;
      act += active_row[i];
    }
  }
  // Positions of this thread's rows, loaded before the scans so that their
  // latency overlaps the look-back (packed keys carry them in the low bits).
  const u64 local_mask = packed_shift ? (1ull << packed_shift) - 1 : 0;
  u32 pos[kScanItems];
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const u64 r = row0 + i;
    pos[i] = 0;
    if (r < n) pos[i] = packed_shift ? static_cast<u32>(keys[r] & local_mask) : sa[r];
  }
  u64 agg_max, agg_sum;
  const u64 excl_max = block_exclusive_scan<kScanBlock>(head_max, MaxOp{}, warp_smem, &agg_max);
  const u64 excl_sum = block_exclusive_scan<kScanBlock>(act, SumOp{}, warp_smem, &agg_sum);
  const u32 warp = threadIdx.x >> 5;
  if (warp == 0) {
    const u64 p = warp_lookback(status_max, tile, agg_max, MaxOp{}, flags, 2);
    if ((threadIdx.x & 31) == 0) tile_prefix[0] = p;
  } else if (warp == 1) {
    const u64 p = warp_lookback(status_sum, tile, agg_sum, SumOp{}, flags, 3);
    if ((threadIdx.x & 31) == 0) tile_prefix[1] = p;
  }
  __syncthreads();
  u64 running_max = tile_prefix[0] > excl_max ? tile_prefix[0] : excl_max;
  u64 out = tile_prefix[1] + excl_sum;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const u64 r = row0 + i;
    if (r < n) {
      if (head[i]) running_max = r;
      u32 p;
      if (packed_shift) {
        cur.locate(segs.begin, segs.count, r);
        p = static_cast<u32>(cur.lo + pos[i]);
        sa[r] = p;
      } else {
        p = pos[i];
      }
      const u64 head_row = running_max;
      if (p >= n) {
        flag_error(flags, kErrBounds);
        continue;
      }
      // With local_pairs the pair carries the instance-local position (the
      // batched rank write groups by windows of each instance).
      u64 pair_pos = p;
      if (local_pairs) {
        cur.locate(segs.begin, segs.count, r);
        pair_pos = p - cur.lo;
      }
      pairs[r] = (pair_pos << 32) | static_cast<u32>(head_row);
      if (active_row[i]) active[out++] = p;
    }
  }
  const u64 tiles = (n + kScanTile - 1) / kScanTile;
  if (tile == tiles - 1 && threadIdx.x == 0) *active_count = tile_prefix[1] + agg_sum;
}

// Rare rows of a two-bit seed: entry idx of the sorted list is row g + (idx -
// i0) of the rows sharing its two-bit key k (g = first row of k in the sorted
// keys, i0 = first entry of k).  Writes its SA entry, its pair (position,
// exact head row), its LCP and, for the last entry of k, the LCP of the row
// after it.  keys: the sorted seed keys (two-bit key << packed_shift, with the
// instance-local index below when packed).
static __global__ void __launch_bounds__(256)
rare_place_kernel(const u64* __restrict__ keys, u64 n, u32 packed_shift, RareRows rare,
                  u32 bits, u32 symbols, Segments segs, u32* __restrict__ sa,
                  u64* __restrict__ pairs, u32* __restrict__ lcp, DeviceFlags* flags) {
  const u64 local_mask = packed_shift ? (1ull << packed_shift) - 1 : 0;
  const u32 unused = 64 - bits * symbols;
  const bool batch = segs.count > 1;
  // Two-bit keys of a batch's rare list carry the instance above their bits.
  const u32 k2_bits = 2 * symbols + 2;
  const u64 k2_mask = k2_bits >= 64 ? ~0ull : (1ull << k2_bits) - 1;
  for (u64 idx = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; idx < rare.count;
       idx += static_cast<u64>(gridDim.x) * blockDim.x) {
    const u64 k = rare.k2[idx];
    const u64 inst = batch ? k >> k2_bits : 0;
    if (inst >= segs.count) {
      flag_error(flags, kErrBounds);
      continue;
    }
    const u64 lo = segs.begin[inst], hi = segs.begin[inst + 1];  // the instance's rows
    const u64 kk = batch ? k & k2_mask : k;
    auto row_pos = [&](u64 r) -> u32 {  // a non-rare row's (global) position
      return packed_shift ? static_cast<u32>(lo + (keys[r] & local_mask)) : sa[r];
    };
    auto rare_row = [&](u64 r) { return ((keys[r] >> packed_shift) & 1) == 0; };
    const u64 i0 = lower_bound_u64(rare.k2, 0, idx, k);
    const u64 g = lower_bound_u64(keys, lo, hi, kk << packed_shift);
    const u64 row = g + (idx - i0);
    if (row >= hi || (keys[row] >> packed_shift) != kk) {
      flag_error(flags, kErrBounds);
      continue;
    }
    const u32 p = rare.pos[idx];
    const u64 ek = rare.key[idx];
    const u64 e0 = lower_bound_u64(rare.key, i0, idx, ek);
    if (p < lo || p >= hi) {
      flag_error(flags, kErrBounds);
      continue;
    }
    sa[row] = p;
    // Batches pair the instance-local position with the head row (the rank
    // write groups by windows of each instance).
    const u64 pair_pos = batch ? p - lo : p;
    pairs[row] = (pair_pos << 32) | static_cast<u32>(g + (e0 - i0));
    u32 v;
    if (row == lo) {
      v = 0;
    } else if (e0 < idx) {
      v = kLcpUnknown;  // the same window as the row before
    } else if (idx > i0 || rare_row(row - 1)) {  // the row before is entry idx - 1
      if (idx == 0) {
        flag_error(flags, kErrBounds);
        continue;
      }
      const u32 x = static_cast<u32>(__clzll(static_cast<long long>(ek ^ rare.key[idx - 1])));
      v = (x - unused) / bits;
    } else {
      v = window_lcp(rare.text, hi, p, row_pos(row - 1), symbols);
    }
    lcp[row] = v;
    const bool last = idx + 1 == rare.count || rare.k2[idx + 1] != k;
    if (last && row + 1 < hi && !rare_row(row + 1)) {
      lcp[row + 1] = window_lcp(rare.text, hi, row_pos(row + 1), p, symbols);
    }
  }
}

// Two-bit keys of the sorted rare rows.
static __global__ void __launch_bounds__(256)
rare_two_bit_kernel(const u64* __restrict__ key, u64 count, u32 symbols, u32 bits,
                    TwoBitSeed tb, u64* __restrict__ k2) {
  for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
       i += static_cast<u64>(gridDim.x) * blockDim.x) {
    if (tb.inst_shift) {
      const u64 inst = key[i] >> tb.inst_shift;
      const u64 exact = key[i] & ((1ull << tb.inst_shift) - 1);
      k2[i] = two_bit_of_exact(exact, symbols, bits, tb) | (inst << (2 * symbols + 2));
    } else {
      k2[i] = two_bit_of_exact(key[i], symbols, bits, tb);
    }
  }
}

// Rare rows whose exact window is shared (groups of two or more, contiguous in
// the sorted list) join the active list after the *base rows seed_rank put
// there; *total receives their number.
static __global__ void __launch_bounds__(kScanBlock)
rare_active_kernel(const u64* __restrict__ key, const u32* __restrict__ pos, u64 count,
                   u32* __restrict__ active, const u64* base, u64* total, u64* status,
                   u32* tile_counter, DeviceFlags* flags) {
  __shared__ u64 warp_smem[kScanBlock / 32];
  __shared__ u64 tile_prefix;
  __shared__ u32 tile_slot;
  const u32 tile = claim_tile(tile_counter, &tile_slot);
  const u64 e0 = static_cast<u64>(tile) * kScanTile + threadIdx.x * kScanItems;
  bool take[kScanItems];
  u32 act = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const u64 e = e0 + i;
    take[i] = false;
    if (e < count) {
      const u64 v = key[e];
      take[i] = (e > 0 && key[e - 1] == v) || (e + 1 < count && key[e + 1] == v);
      act += take[i];
    }
  }
  u64 agg;
  const u64 excl = block_exclusive_scan<kScanBlock>(act, SumOp{}, warp_smem, &agg);
  if ((threadIdx.x >> 5) == 0) {
    const u64 p = warp_lookback(status, tile, agg, SumOp{}, flags, 7);
    if ((threadIdx.x & 31) == 0) tile_prefix = p;
  }
  __syncthreads();
  u64 out = *base + tile_prefix + excl;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (take[i]) active[out++] = pos[e0 + i];
  }
  const u64 tiles = (count + kScanTile - 1) / kScanTile;
  if (tile == tiles - 1 && threadIdx.x == 0) *total = tile_prefix + agg;
}

// rank[pos] = head for (pos << 32 | head) pairs grouped by 2048-position
// windows (pairs [w*2048, (w+1)*2048) hold exactly window w's positions: SA
// is a permutation).  Each block stages one window in shared memory and writes
// it out coalesced.
constexpr u32 kWindowBits = 11;
constexpr u32 kWindow = 1u << kWindowBits;

static __global__ void __launch_bounds__(256)
window_scatter_kernel(const u64* __restrict__ pairs, u64 n, u32* __restrict__ rank,
                      DeviceFlags* flags) {
  __shared__ u32 window[kWindow];
  const u64 first = static_cast<u64>(blockIdx.x) * kWindow;
  const u32 count = static_cast<u32>(n - first < kWindow ? n - first : kWindow);
  for (u32 i = threadIdx.x; i < count; i += 256) {
    const u64 v = pairs[first + i];
    const u64 pos = v >> 32;
    if ((pos >> kWindowBits) != blockIdx.x || (pos & (kWindow - 1)) >= count) {
      flag_error(flags, kErrBounds);  // not a permutation
      continue;
    }
    window[pos & (kWindow - 1)] = static_cast<u32>(v);
  }
  __syncthreads();
  for (u32 i = threadIdx.x; i < count; i += 256) rank[first + i] = window[i];
}

// rank[pos] = head for pairs grouped by windows of 2^16 positions (one
// grouping pass fewer than 2048-position windows for texts of 2^28 to 2^32
// symbols, and of 2^17 to 2^24), written through a cluster of kCtas blocks:
// each block holds its share of the window (2^16 / kCtas words: 128 KB for
// two blocks, 64 KB for four, so that two clusters share an SM), reads its
// share of the window's pairs and stores each head into the owning block's
// shared memory (distributed shared memory), then writes its share out
// coalesced.
constexpr u32 kClusterWindowBits = 16;

template <int kCtas>
struct ClusterWindow {
  static constexpr u32 kSliceBits = kClusterWindowBits - (kCtas == 4 ? 2 : 1);
  static constexpr u32 kSlice = 1u << kSliceBits;
  static constexpr u32 kBlock = kCtas == 4 ? 512 : 1024;
};

template <int kCtas>
__device__ __forceinline__ void cluster_window_scatter(const u64* __restrict__ pairs, u64 n,
                                                       u32* __restrict__ rank,
                                                       DeviceFlags* flags, u32* slice) {
  using W = ClusterWindow<kCtas>;
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  const u32 me = cluster.block_rank();
  const u64 w = blockIdx.x / kCtas;
  const u64 first = w << kClusterWindowBits;
  const u64 count = n - first < (1ull << kClusterWindowBits) ? n - first
                                                               : (1ull << kClusterWindowBits);
  cluster.sync();  // every block's shared memory is live before remote stores
  const u64 lo = static_cast<u64>(me) * W::kSlice;
  const u64 hi = lo + W::kSlice < count ? lo + W::kSlice : count;
  for (u64 i = lo + threadIdx.x; i < hi; i += W::kBlock) {
    const u64 v = pairs[first + i];
    const u64 pos = v >> 32;
    const u64 local = pos - first;
    if ((pos >> kClusterWindowBits) != w || local >= count) {
      flag_error(flags, kErrBounds);  // not a permutation
      continue;
    }
    u32* const owner = cluster.map_shared_rank(slice, static_cast<u32>(local >> W::kSliceBits));
    owner[local & (W::kSlice - 1)] = static_cast<u32>(v);
  }
  cluster.sync();
  for (u64 i = lo + threadIdx.x; i < hi; i += W::kBlock) rank[first + i] = slice[i - lo];
}

static __global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(1024, 1)
cluster_window_scatter_kernel(const u64* __restrict__ pairs, u64 n, u32* __restrict__ rank,
                              DeviceFlags* flags) {
  extern __shared__ u32 slice[];
  cluster_window_scatter<2>(pairs, n, rank, flags, slice);
}

static __global__ void __cluster_dims__(4, 1, 1) __launch_bounds__(512, 2)
cluster4_window_scatter_kernel(const u64* __restrict__ pairs, u64 n, u32* __restrict__ rank,
                               DeviceFlags* flags) {
  extern __shared__ u32 slice[];
  cluster_window_scatter<4>(pairs, n, rank, flags, slice);
}

// The same per instance of a batch: pairs carry instance-local positions
// and are grouped by 2^16-position window inside each instance's rows, so
// instance j's window w is rows begin[j] + [w << 16, min((w + 1) << 16, n_j)).
// wbegin[j] = windows of the instances before j (count + 1 entries).  Both
// blocks of a cluster serve the same window.
static __global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(1024, 1)
cluster_segment_window_scatter_kernel(const u64* __restrict__ pairs, Segments segs,
                                      const u64* __restrict__ wbegin, u32* __restrict__ rank,
                                      DeviceFlags* flags) {
  using W = ClusterWindow<2>;
  extern __shared__ u32 slice[];
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  const u32 me = cluster.block_rank();
  const u64 window = blockIdx.x >> 1;
  u32 lo_j = 0, hi_j = segs.count;  // instance j with wbegin[j] <= window < wbegin[j + 1]
  while (hi_j - lo_j > 1) {
    const u32 mid = (lo_j + hi_j) >> 1;
    if (wbegin[mid] <= window) lo_j = mid;
    else hi_j = mid;
  }
  const u64 w = window - wbegin[lo_j];
  const u64 base = segs.begin[lo_j];
  const u64 len = segs.begin[lo_j + 1] - base;
  const u64 first = w << kClusterWindowBits;
  const u64 count = first >= len ? 0
                    : (len - first < (1ull << kClusterWindowBits) ? len - first
                                                                  : (1ull << kClusterWindowBits));
  if (count == 0 && threadIdx.x == 0 && me == 0) flag_error(flags, kErrBounds);
  cluster.sync();  // every block's shared memory is live before remote stores
  const u64 lo = static_cast<u64>(me) * W::kSlice;
  const u64 hi = lo + W::kSlice < count ? lo + W::kSlice : count;
  for (u64 i = lo + threadIdx.x; i < hi; i += W::kBlock) {
    const u64 v = pairs[base + first + i];
    const u64 pos = v >> 32;
    const u64 local = pos - first;
    if ((pos >> kClusterWindowBits) != w || local >= count) {
      flag_error(flags, kErrBounds);  // not a permutation of the instance
      continue;
    }
    u32* const owner = cluster.map_shared_rank(slice, static_cast<u32>(local >> W::kSliceBits));
    owner[local & (W::kSlice - 1)] = static_cast<u32>(v);
  }
  cluster.sync();
  for (u64 i = lo + threadIdx.x; i < hi; i += W::kBlock) rank[base + first + i] = slice[i - lo];
}

// Rank write by window slots (one instance).  Each (position << 32 | head)
// pair takes the next slot of its window of 2^kSlotBits positions with one
// atomic and is stored there; a window's pairs are then staged in shared
// memory and its ranks written out whole.  Windows fill front to back, so
// the partially written sectors of all windows (32 bytes each) stay in L2 and
// leave it whole: one pass over the pairs instead of the keys-only radix
// passes that group them by window.
constexpr u32 kSlotBits = 13;
constexpr u32 kSlotWindow = 1u << kSlotBits;

static __global__ void __launch_bounds__(256)
rank_slot_kernel(const u64* __restrict__ pairs, u64 n, u32* __restrict__ fill,
                 u64* __restrict__ slotted, DeviceFlags* flags) {
  const u64 windows = (n + kSlotWindow - 1) >> kSlotBits;
  const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
  for (u64 r = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += stride) {
    const u64 v = pairs[r];
    const u64 w = (v >> 32) >> kSlotBits;
    if (w >= windows) {
      flag_error(flags, kErrBounds);  // not a permutation
      continue;
    }
    const u32 slot = atomicAdd(fill + w, 1u);
    const u64 at = (w << kSlotBits) + slot;
    if (slot >= kSlotWindow || at >= n) {  // more pairs than positions: not a permutation
      flag_error(flags, kErrBounds);
      continue;
    }
    slotted[at] = v;
  }
}

// One block per slot window; dynamic shared memory of kSlotWindow words.
static __global__ void __launch_bounds__(256)
slot_window_scatter_kernel(const u64* __restrict__ slotted, u64 n, u32* __restrict__ rank,
                           DeviceFlags* flags) {
  extern __shared__ u32 window_smem[];
  const u64 first = static_cast<u64>(blockIdx.x) << kSlotBits;
  const u32 count = static_cast<u32>(n - first < kSlotWindow ? n - first : kSlotWindow);
  for (u32 i = threadIdx.x; i < count; i += 256) {
    const u64 v = slotted[first + i];
    const u64 pos = v >> 32;
    if ((pos >> kSlotBits) != blockIdx.x || (pos & (kSlotWindow - 1)) >= count) {
      flag_error(flags, kErrBounds);  // not a permutation
      continue;
    }
    window_smem[pos & (kSlotWindow - 1)] = static_cast<u32>(v);
  }
  __syncthreads();
  for (u32 i = threadIdx.x; i < count; i += 256) rank[first + i] = window_smem[i];
}

// The same for a batch: windows of 2^kSlotBits instance-local positions,
// numbered per instance from wbegin (wbegin[j] = the first window of
// instance j); pairs carry instance-local positions.  The slots of window w
// of instance j are rows begin_j + w * 2^kSlotBits onward.
static __global__ void __launch_bounds__(256)
rank_slot_segments_kernel(const u64* __restrict__ pairs, Segments segs,
                          const u64* __restrict__ wbegin, u32* __restrict__ fill,
                          u64* __restrict__ slotted, DeviceFlags* flags) {
  const u64 n = segs.begin[segs.count];
  const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
  SegCursor cur;
  for (u64 r = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += stride) {
    cur.locate(segs.begin, segs.count, r);
    const u64 v = pairs[r];
    const u64 local = v >> 32;
    const u64 len = cur.hi - cur.lo;
    if (local >= len) {
      flag_error(flags, kErrBounds);  // not a permutation
      continue;
    }
    const u64 w = local >> kSlotBits;
    const u32 slot = atomicAdd(fill + wbegin[cur.j] + w, 1u);
    const u64 at = cur.lo + (w << kSlotBits) + slot;
    if (slot >= kSlotWindow || at >= cur.hi) {
      flag_error(flags, kErrBounds);
      continue;
    }
    slotted[at] = v;
  }
}

// One block per window of the batch; dynamic shared memory of kSlotWindow words.
static __global__ void __launch_bounds__(256)
slot_segment_window_scatter_kernel(const u64* __restrict__ slotted, Segments segs,
                                   const u64* __restrict__ wbegin, u32* __restrict__ rank,
                                   DeviceFlags* flags) {
  extern __shared__ u32 window_smem[];
  u32 lo = 0, hi = segs.count;  // instance j with wbegin[j] <= blockIdx.x < wbegin[j + 1]
  while (hi - lo > 1) {
    const u32 mid = (lo + hi) >> 1;
    if (wbegin[mid] <= blockIdx.x) lo = mid;
    else hi = mid;
  }
  const u64 w = blockIdx.x - wbegin[lo];
  const u64 base = segs.begin[lo];
  const u64 len = segs.begin[lo + 1] - base;
  const u64 first = w << kSlotBits;
  if (first >= len) {
    flag_error(flags, kErrBounds);
    return;
  }
  const u32 count = static_cast<u32>(len - first < kSlotWindow ? len - first : kSlotWindow);
  for (u32 i = threadIdx.x; i < count; i += 256) {
    const u64 v = slotted[base + first + i];
    const u64 local = v >> 32;
    if ((local >> kSlotBits) != w || (local & (kSlotWindow - 1)) >= count) {
      flag_error(flags, kErrBounds);  // not a permutation
      continue;
    }
    window_smem[local & (kSlotWindow - 1)] = static_cast<u32>(v);
  }
  __syncthreads();
  for (u32 i = threadIdx.x; i < count; i += 256) rank[base + first + i] = window_smem[i];
}

// Long-run lookup for the rounds (runs.cuh builds it): sorted run starts and
// ends plus a bitmap of the 2^kRunBlockBits-position blocks that hold run
// members.  count == 0 disables it.
constexpr u32 kRunBlockBits = 12;

struct RunIndex {
  const u32* a = nullptr;     // sorted starts
  const u32* e = nullptr;     // matching ends
  const u32* bitmap = nullptr;
  u32 count = 0;
};

// The run end e if p is a member with at least h symbols of run ahead, else 0.
__device__ __forceinline__ u64 run_jump(const RunIndex& ri, u64 p, u64 h) {
  if (ri.count == 0) return 0;
  const u64 blk = p >> kRunBlockBits;
  if (!((ri.bitmap[blk >> 5] >> (blk & 31)) & 1u)) return 0;
  u32 lo = 0, hi = ri.count;  // last run with a <= p
  if (ri.a[0] > p) return 0;
  while (hi - lo > 1) {
    const u32 mid = (lo + hi) >> 1;
    if (ri.a[mid] <= p) lo = mid;
    else hi = mid;
  }
  const u64 e = ri.e[lo];
  return (p < e && e - p >= h) ? e : 0;
}

// Device-side round state, so that a sequence of rounds can run without the
// host (and be captured in a CUDA graph): the active count of the round (read
// by its kernels, which are launched for an upper bound and skip the rest),
// the prefix length h, and an abort word that a round sets when its groups
// need the host (the kernels after it then do nothing).
struct RoundState {
  const u64* count;  // active rows of this round
  u64* next_count;   // written by round_rank
  u64* h;            // prefix length; doubled by round_rank when double_h
  const u64* abort;  // nonzero: skip (null: never)
  u64* totals;       // [0] += active rows, [1] += rounds (null: not kept)
  u32 double_h;
};

__device__ __forceinline__ bool round_skipped(const RoundState& rs) {
  return rs.abort && *rs.abort;
}

// The same window write per instance: pairs carry instance-local positions
// and are grouped by 2048-position window inside each instance's rows, so
// instance j's window w is rows begin[j] + [w * 2048, min((w + 1) * 2048, n_j)).
// wbegin[j] = windows of the instances before j (count + 1 entries).
static __global__ void __launch_bounds__(256)
segment_window_scatter_kernel(const u64* __restrict__ pairs, Segments segs,
                              const u64* __restrict__ wbegin, u32* __restrict__ rank,
                              DeviceFlags* flags) {
  __shared__ u32 window[kWindow];
  u32 lo = 0, hi = segs.count;  // instance j with wbegin[j] <= blockIdx.x < wbegin[j + 1]
  while (hi - lo > 1) {
    const u32 mid = (lo + hi) >> 1;
    if (wbegin[mid] <= blockIdx.x) lo = mid;
    else hi = mid;
  }
  const u64 w = blockIdx.x - wbegin[lo];
  const u64 base = segs.begin[lo];
  const u64 len = segs.begin[lo + 1] - base;
  const u64 first = w * kWindow;
  if (first >= len) {
    flag_error(flags, kErrBounds);
    return;
  }
  const u32 count = static_cast<u32>(len - first < kWindow ? len - first : kWindow);
  for (u32 i = threadIdx.x; i < count; i += 256) {
    const u64 v = pairs[base + first + i];
    const u64 local = v >> 32;
    if ((local >> kWindowBits) != w || (local & (kWindow - 1)) >= count) {
      flag_error(flags, kErrBounds);  // not a permutation
      continue;
    }
    window[local & (kWindow - 1)] = static_cast<u32>(v);
  }
  __syncthreads();
  for (u32 i = threadIdx.x; i < count; i += 256) rank[base + first + i] = window[i];
}

// Round step 1: composite keys for the active list.  counters: *group_count
// receives the number of groups G.  ghead/gstart are indexed by dense id.
// inst_h, when set, holds each segment's own prefix length h (the served
// engine advances references admitted at different times side by side);
// otherwise *rs.h is the round's prefix length.
static __global__ void __launch_bounds__(kScanBlock)
round_keys_kernel(const u32* __restrict__ active, RoundState rs,
                  const u32* __restrict__ rank, const u64* __restrict__ inst_h,
                  Segments segs,
                  u32 second_bits, u64* __restrict__ ckey,
                  u32* __restrict__ cval, u32* __restrict__ ghead,
                  u32* __restrict__ gstart, u64 group_cap, u64* status_sum,
                  u32* tile_counter, u64* group_count, DeviceFlags* flags,
                  RunIndex runs) {
  __shared__ u64 warp_smem[kScanBlock / 32];
  __shared__ u64 tile_prefix;
  __shared__ u32 tile_slot;
  if (round_skipped(rs)) return;
  const u64 count = *rs.count;
  const u64 h = inst_h ? 0 : *rs.h;
  const u32 tile = claim_tile(tile_counter, &tile_slot);
  // Launched for an upper bound: tiles past the count (after every real
  // tile, so no look-back waits on them) leave at once.
  if (static_cast<u64>(tile) * kScanTile >= count) return;
  const u64 a0 = static_cast<u64>(tile) * kScanTile + threadIdx.x * kScanItems;

  u32 pos[kScanItems];
  u32 grp[kScanItems];
  bool start[kScanItems];
  u32 prev_group = 0xffffffffu;
  if (a0 > 0 && a0 <= count) prev_group = rank[active[a0 - 1]];
  u32 starts = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const u64 a = a0 + i;
    if (a < count) {
      pos[i] = active[a];
      grp[i] = rank[pos[i]];
      start[i] = a == 0 || grp[i] != prev_group;
      prev_group = grp[i];
      starts += start[i];
    } else {
      start[i] = false;
    }
  }
  u64 agg;
  const u64 excl = block_exclusive_scan<kScanBlock>(starts, SumOp{}, warp_smem, &agg);
  if ((threadIdx.x >> 5) == 0) {
    const u64 p = warp_lookback(status_sum, tile, agg, SumOp{}, flags, 4);
    if ((threadIdx.x & 31) == 0) tile_prefix = p;
  }
  __syncthreads();
  u64 dense = tile_prefix + excl;  // number of group starts before this item
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const u64 a = a0 + i;
    if (a < count) {
      if (start[i]) {
        if (dense < group_cap) {
          ghead[dense] = grp[i];
          gstart[dense] = static_cast<u32>(a);
        } else {
          flag_error(flags, kErrBounds);
        }
        ++dense;
      }
      const u64 p = pos[i];
      u64 end, q;
      if (inst_h) {
        const u32 j = segs.count == 1 ? 0 : find_segment(segs.begin, segs.count, p);
        end = segs.end ? segs.end[j] : segs.begin[j + 1];
        q = p + inst_h[j];
      } else {
        end = segment_end(segs, p);
        const u64 jump = run_jump(runs, p, h);  // a long-run member: its run end
        q = jump ? jump : p + h;
      }
      const u64 second = q < end ? static_cast<u64>(rank[q]) + 1 : 0;
      ckey[a] = ((dense - 1) << second_bits) | second;
      cval[a] = static_cast<u32>(p);
    }
  }
  const u64 tiles = (count + kScanTile - 1) / kScanTile;
  if (tile == tiles - 1 && threadIdx.x == 0) *group_count = tile_prefix + agg;
}

// Round step 2 (after sorting the composite keys): new heads, SA rows, ranks,
// and the next active list.
static __global__ void __launch_bounds__(kScanBlock)
round_rank_kernel(const u64* __restrict__ ckey, const u32* __restrict__ cval,
                  RoundState rs, u32 second_bits, const u32* __restrict__ ghead,
                  const u32* __restrict__ gstart, u64 group_cap, u64 rows,
                  u32* __restrict__ sa,
                  u32* __restrict__ rank, u32* __restrict__ next_active,
                  u64* status_max, u64* status_sum, u32* tile_counter,
                  DeviceFlags* flags) {
  __shared__ u64 warp_smem[kScanBlock / 32];
  __shared__ u64 tile_prefix[2];
  __shared__ u32 tile_slot;
  if (round_skipped(rs)) return;
  const u64 count = *rs.count;
  if (count == 0) {  // converged: the next round has nothing either
    if (blockIdx.x == 0 && threadIdx.x == 0) *rs.next_count = 0;
    return;
  }
  const u32 tile = claim_tile(tile_counter, &tile_slot);
  if (static_cast<u64>(tile) * kScanTile >= count) return;
  const u64 a0 = static_cast<u64>(tile) * kScanTile + threadIdx.x * kScanItems;

  u64 k[kScanItems + 2];
#pragma unroll
  for (int i = 0; i < kScanItems + 2; ++i) {
    const long long a = static_cast<long long>(a0) - 1 + i;
    k[i] = (a >= 0 && static_cast<u64>(a) < count) ? ckey[a] : ~0ull;
  }
  bool head[kScanItems + 1];
#pragma unroll
  for (int i = 0; i < kScanItems + 1; ++i) {
    const u64 a = a0 + i;
    head[i] = a >= count || a == 0 || k[i + 1] != k[i];
  }
  u64 head_max = 0;
  u32 keep = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const u64 a = a0 + i;
    if (a < count) {
      if (head[i]) head_max = a;
      if (!(head[i] && head[i + 1])) ++keep;
    }
  }
  // Values and group tables of this thread's rows, loaded before the scans
  // so that their latency overlaps the look-back.
  u32 val[kScanItems], g_head[kScanItems], g_first[kScanItems];
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const u64 a = a0 + i;
    const u64 dense = k[i + 1] >> second_bits;
    val[i] = 0;
    g_head[i] = 0;
    g_first[i] = 0;
    if (a < count && dense < group_cap) {
      val[i] = cval[a];
      g_head[i] = ghead[dense];
      g_first[i] = gstart[dense];
    }
  }
  u64 agg_max, agg_sum;
  const u64 excl_max = block_exclusive_scan<kScanBlock>(head_max, MaxOp{}, warp_smem, &agg_max);
  const u64 excl_sum = block_exclusive_scan<kScanBlock>(keep, SumOp{}, warp_smem, &agg_sum);
  const u32 warp = threadIdx.x >> 5;
  if (warp == 0) {
    const u64 p = warp_lookback(status_max, tile, agg_max, MaxOp{}, flags, 5);
    if ((threadIdx.x & 31) == 0) tile_prefix[0] = p;
  } else if (warp == 1) {
    const u64 p = warp_lookback(status_sum, tile, agg_sum, SumOp{}, flags, 6);
    if ((threadIdx.x & 31) == 0) tile_prefix[1] = p;
  }
  __syncthreads();
  u64 sub_start = tile_prefix[0] > excl_max ? tile_prefix[0] : excl_max;
  u64 out = tile_prefix[1] + excl_sum;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const u64 a = a0 + i;
    if (a < count) {
      if (head[i]) sub_start = a;
      const u64 dense = k[i + 1] >> second_bits;
      if (dense >= group_cap) {
        flag_error(flags, kErrBounds);
        continue;
      }
      const u32 group_head = g_head[i];
      const u32 group_first = g_first[i];
      const u32 p = val[i];
      const u64 row = group_head + (a - group_first);
      if (row >= rows || p >= rows || a < group_first) {
        flag_error(flags, kErrBounds);
        continue;
      }
      sa[row] = p;
      rank[p] = static_cast<u32>(group_head + (sub_start - group_first));
      if (!(head[i] && head[i + 1])) next_active[out++] = p;
    }
  }
  const u64 tiles = (count + kScanTile - 1) / kScanTile;
  if (tile == tiles - 1 && threadIdx.x == 0) {
    *rs.next_count = tile_prefix[1] + agg_sum;
    if (rs.double_h) *rs.h *= 2;
    if (rs.totals) {
      rs.totals[0] += count;
      rs.totals[1] += 1;
    }
  }
}

}  // namespace sufgpu
