// Seed keys fused with the first pass of the segmented seed sort.
//
// The seed sort is an LSD radix sort of the seed keys over 8-bit digits.  Its
// first pass needs no stability: the order it preserves is the order of the
// keys it is given, and nothing downstream depends on the order of rows that
// share a whole seed key (the doubling rounds reorder every seed group, and
// two-bit rare rows are placed from their own sorted list).  So the kernel
// that generates a tile's keys from the text also ranks them by their lowest
// digit with shared-memory atomics, takes each digit's global offset from a
// decoupled look-back, and writes the tile out partitioned by that digit:
// the keys never make the round trip through memory in position order, which
// saves one full read and write of (key, position) per symbol.  The digit
// offsets come from histograms that seed_keys_kernel computes in a pass over
// the text that writes no keys.
#pragma once

#include "common.cuh"
#include "doubling.cuh"
#include "radix.cuh"
#include "scan.cuh"

namespace sufgpu {

struct SeedSortSmem {
  u64 keys[kSortTile];  // the tile in digit order
  u32 vals[kSortTile];
  u32 hist[kRadixDigits];
  u32 digit_excl[kRadixDigits];
  long long digit_gbase[kRadixDigits];
  u64 warp_scan[kSortBlock / 32];
  u16 code[256];
  // Text of the tile and its halo, staged from the 16-byte boundary at or
  // below the tile's first position (an instance may start anywhere).
  __align__(16) u8 window[kSortTile + kSeedHalo + 16];
  u32 tile;
};

// One tile of the segmented seed sort per block (kSortBlock threads x
// kSortItems consecutive positions each; tiles never cross an instance, as in
// radix_onesweep_kernel).  shift = the first sorted bit (packed_shift or 0);
// digit_start = [segment][pass][digit] absolute output offsets, of which pass
// 0 is used.  kTwoBit keys as in seed_keys_kernel (rare rows were already
// listed by the histogram pass).
template <bool kTwoBit>
static __global__ void __launch_bounds__(kSortBlock, 3)
seed_sorted_kernel(const u8* __restrict__ text, SortSegments ss,
                   const u16* __restrict__ code_table, u32 bits, u32 symbols, u32 packed_shift,
                   u32 passes, const u64* __restrict__ digit_start, u64* __restrict__ keys_out,
                   u32* __restrict__ vals_out, u64* status, u32* tile_counter, DeviceFlags* flags,
                   TwoBitSeed tb) {
  static_assert(kSortTile == kSortBlock * kSortItems, "tile shape");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SeedSortSmem& sm = *reinterpret_cast<SeedSortSmem*>(smem_raw);
  sm.code[threadIdx.x] = code_table[threadIdx.x];
  sm.hist[threadIdx.x] = 0;
  const u32 tile = claim_tile(tile_counter, &sm.tile);
  u32 seg;
  u64 first, last;
  segment_of_tile(ss, tile, &seg, &first, &last);
  const u64 seg_lo = ss.begin[seg];
  const u64 seg_end = ss.begin[seg + 1];
  const bool first_tile_of_segment = tile == ss.tile_begin[seg];
  const u64 base = first & ~static_cast<u64>(15);
  const u32 off = static_cast<u32>(first - base);
  const u64 text_end = ss.begin[ss.count];  // the text buffer is padded past it
  for (int i = threadIdx.x; i < (kSortTile + kSeedHalo + 16) / 16; i += kSortBlock) {
    const u64 at = base + static_cast<u64>(i) * 16;
    uint4 v = make_uint4(0, 0, 0, 0);
    if (at < text_end) v = *reinterpret_cast<const uint4*>(text + at);
    *reinterpret_cast<uint4*>(sm.window + i * 16) = v;
  }
  __syncthreads();
  const u64 count = last - first;
  const u64 mask = symbols * bits >= 64 ? ~0ull : ((1ull << (symbols * bits)) - 1);
  const u64 mask2 = 2 * symbols >= 64 ? ~0ull : ((1ull << (2 * symbols)) - 1);
  const u32 smask = symbols >= 32 ? ~0u : ((1u << symbols) - 1);
  const u32 local0 = threadIdx.x * kSortItems;
  u64 key = 0, k2 = 0;
  u32 irregular = 0;
  auto push = [&](u32 c) {
    key = ((key << bits) | c) & mask;
    if (kTwoBit) {
      const bool reg = c >= tb.lo && c < tb.lo + 4;
      k2 = ((k2 << 2) | (reg ? c - tb.lo : 0u)) & mask2;
      irregular = ((irregular << 1) | (reg ? 0u : 1u)) & smask;
    }
  };
  u64 out_key[kSortItems];
  u32 rank[kSortItems];
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    const u32 local = local0 + r;
    const u64 pos = first + local;
    out_key[r] = 0;
    rank[r] = 0;
    if (local >= count) continue;
    if (r == 0) {
      for (u32 t = 0; t < symbols; ++t) {
        push(pos + t < seg_end ? sm.code[sm.window[off + local + t]] : 0u);
      }
    } else {
      const u64 q = pos + symbols - 1;
      push(q < seg_end ? sm.code[sm.window[off + local + symbols - 1]] : 0u);
    }
    u64 sort_key = key;
    if (kTwoBit) sort_key = two_bit_key(key, k2, irregular, symbols, bits, tb);
    out_key[r] = packed_shift ? (sort_key << packed_shift) | (pos - seg_lo) : sort_key;
    const u32 digit = static_cast<u32>((out_key[r] >> packed_shift) & 0xff);
    rank[r] = atomicAdd(&sm.hist[digit], 1u);  // unstable: see the file comment
  }
  __syncthreads();
  // Per digit: the tile-local start, then the global start by look-back
  // (a segment's first tile seeds it from digit_start).
  const u32 d = threadIdx.x;
  const u32 digit_count = sm.hist[d];
  u64 tile_total;
  const u64 local_start =
      block_exclusive_scan<kSortBlock>(digit_count, SumOp{}, sm.warp_scan, &tile_total);
  sm.digit_excl[d] = static_cast<u32>(local_start);
  u64* my_status = status + static_cast<u64>(tile) * kRadixDigits + d;
  u64 global_start;
  if (first_tile_of_segment) {
    global_start = digit_start[(static_cast<u64>(seg) * passes) * kRadixDigits + d];
    store_status(my_status, kFlagPrefix | ((global_start + digit_count) & kValueMask));
  } else {
    store_status(my_status, kFlagAggregate | digit_count);
    u64 exclusive = 0;
    long long t = static_cast<long long>(tile) - 1;
    while (true) {
      const u64 v = wait_status(status + static_cast<u64>(t) * kRadixDigits + d, flags, 22);
      exclusive += v & kValueMask;
      if ((v >> 62) == 2) break;
      --t;
    }
    global_start = exclusive;
    store_status(my_status, kFlagPrefix | ((global_start + digit_count) & kValueMask));
  }
  sm.digit_gbase[d] = static_cast<long long>(global_start) - static_cast<long long>(local_start);
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    const u32 local = local0 + r;
    if (local >= count) continue;
    const u32 digit = static_cast<u32>((out_key[r] >> packed_shift) & 0xff);
    const u32 slot = sm.digit_excl[digit] + rank[r];
    sm.keys[slot] = out_key[r];
    sm.vals[slot] = static_cast<u32>(first + local);
  }
  __syncthreads();
  for (u32 s = threadIdx.x; s < count; s += kSortBlock) {
    const u64 k = sm.keys[s];
    const u32 digit = static_cast<u32>((k >> packed_shift) & 0xff);
    const u64 out = static_cast<u64>(sm.digit_gbase[digit] + static_cast<long long>(s));
    if (out < seg_lo || out >= seg_end) {  // only after a failed look-back
      flag_error(flags, kErrBounds);
      continue;
    }
    keys_out[out] = k;
    if (!packed_shift) vals_out[out] = sm.vals[s];
  }
}

}  // namespace sufgpu
