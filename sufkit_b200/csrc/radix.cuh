// Segmented LSD radix sort of (u64 key, u32 value) pairs, onesweep style.
//
// Many independent segments (one per reference instance in a batch) are sorted
// by the same launches: tiles never cross a segment, digit offsets are kept
// per segment, and the decoupled look-back of a tile stops at its segment's
// first tile.  One histogram launch counts every digit of every pass at once;
// each pass is then one launch that ranks a 4096-key tile in shared memory
// (warp match-any ranking, stable), looks back for its global digit offsets,
// and scatters through shared memory so that runs of equal digits are written
// contiguously.
#pragma once

#include "common.cuh"
#include "scan.cuh"

namespace sufgpu {

constexpr int kRadixBits = 8;
constexpr int kRadixDigits = 1 << kRadixBits;
constexpr int kSortBlock = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortBlock * kSortItems;
constexpr int kMaxPasses = 8;

struct SortSegments {
  const u64* begin;       // count+1 element offsets
  const u32* tile_begin;  // count+1 tile offsets
  u32 count;
  u32 total_tiles;
  u32 tile_size = kSortTile;  // keys per tile (the onesweep variant's tile)
};

__device__ __forceinline__ void segment_of_tile(const SortSegments& s, u32 tile,
                                                u32* seg, u64* first,
                                                u64* last) {
  u32 lo = 0, hi = s.count;
  while (hi - lo > 1) {
    const u32 mid = (lo + hi) >> 1;
    if (s.tile_begin[mid] <= tile) lo = mid;
    else hi = mid;
  }
  // Skip empty segments that share the tile offset.
  while (lo + 1 < s.count && s.tile_begin[lo + 1] <= tile) ++lo;
  *seg = lo;
  const u64 start = s.begin[lo] + static_cast<u64>(tile - s.tile_begin[lo]) * s.tile_size;
  const u64 end_seg = s.begin[lo + 1];
  *first = start;
  *last = start + s.tile_size < end_seg ? start + s.tile_size : end_seg;
}

// hist layout: [segment][pass][digit], u32 counts.  Per item and pass a warp
// whose lanes share one digit adds once (long runs of equal keys); otherwise
// each lane adds to the block's shared histogram.
static __global__ void __launch_bounds__(kSortBlock)
radix_histogram_kernel(const u64* __restrict__ keys, SortSegments segs,
                       u32 begin_bit, u32 passes, u32* __restrict__ hist) {
  __shared__ u32 local[kMaxPasses][kRadixDigits];
  for (int i = threadIdx.x; i < kMaxPasses * kRadixDigits; i += kSortBlock) {
    (&local[0][0])[i] = 0;
  }
  __syncthreads();
  u32 seg;
  u64 first, last;
  segment_of_tile(segs, blockIdx.x, &seg, &first, &last);
  const u32 lane = threadIdx.x & 31;
  const int items = static_cast<int>(segs.tile_size / kSortBlock);
#pragma unroll 4
  for (int item = 0; item < items; ++item) {
    const u64 idx = first + static_cast<u64>(item) * kSortBlock + threadIdx.x;
    const bool valid = idx < last;
    const u64 key = valid ? keys[idx] : 0;
    const bool full = __all_sync(0xffffffffu, valid);
    for (u32 p = 0; p < passes; ++p) {
      const u32 digit = static_cast<u32>((key >> (begin_bit + p * kRadixBits)) & 0xff);
      const u32 d0 = __shfl_sync(0xffffffffu, digit, 0);
      if (full && __all_sync(0xffffffffu, digit == d0)) {
        if (lane == 0) atomicAdd(&local[p][d0], 32u);
      } else if (valid) {
        atomicAdd(&local[p][digit], 1u);
      }
    }
  }
  __syncthreads();
  u32* out = hist + static_cast<u64>(seg) * passes * kRadixDigits;
  for (u32 i = threadIdx.x; i < passes * kRadixDigits; i += kSortBlock) {
    const u32 c = (&local[0][0])[i];
    if (c) atomicAdd(&out[i], c);
  }
}

// digit_start layout: [segment][pass][digit], absolute u64 element offsets.
// needed[p] is set when some segment has more than one non-empty digit in
// pass p (otherwise the pass is the identity and is skipped).
static __global__ void __launch_bounds__(kRadixDigits)
radix_offsets_kernel(const u32* __restrict__ hist, const u64* __restrict__ begin,
                     u32 passes, u64* __restrict__ digit_start,
                     u32* __restrict__ needed) {
  __shared__ u64 warp_smem[kRadixDigits / 32];
  __shared__ u32 nonzero;
  const u32 seg = blockIdx.x;
  const u32 d = threadIdx.x;
  for (u32 p = 0; p < passes; ++p) {
    if (d == 0) nonzero = 0;
    __syncthreads();
    const u64 base = (static_cast<u64>(seg) * passes + p) * kRadixDigits;
    const u32 c = hist[base + d];
    if (c) atomicAdd(&nonzero, 1u);
    u64 total;
    const u64 excl = block_exclusive_scan<kRadixDigits>(c, SumOp{}, warp_smem, &total);
    digit_start[base + d] = begin[seg] + excl;
    if (d == 0 && nonzero > 1) atomicOr(&needed[p], 1u);
    __syncthreads();
  }
}

// One LSD pass over bits [shift, shift+8), for a tile of kSortTile pairs
// handled by kBlock threads x kItems items.  Shared memory holds the tile's
// keys and values (kVals) in sorted-slot order and per-warp digit counters.
// The counters are 16-bit (a warp ranks at most 32 x kItems <= 512 keys, and
// a tile-local slot is below 4096), which keeps a 4096-pair tile at 56 KB: four
// blocks per SM instead of two.
template <int kBlock, int kTile = kSortTile, bool kVals = true>
struct OnesweepSmem {
  u64 keys[kTile];
  u32 vals[kVals ? kTile : 1];
  unsigned short warp_hist[kBlock / 32][kRadixDigits];
  long long digit_gbase[kRadixDigits];
  u64 warp_scan[kBlock / 32];
  u64 mbar;  // completion barrier of the bulk tile load (kTma)
  u32 tile;
};
static_assert(kSortTile <= 65535, "16-bit tile-local slots");

// Bulk (TMA engine) copy of `bytes` contiguous bytes from this GPU's global
// memory into the CTA's shared memory, completing on an mbarrier: one
// cp.async.bulk, no multicast.  dst, src 16-byte aligned; bytes a multiple
// of 16.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, u32 bytes, u64* mbar) {
  const u32 d = static_cast<u32>(__cvta_generic_to_shared(dst));
  const u32 m = static_cast<u32>(__cvta_generic_to_shared(mbar));
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      :: "r"(d), "l"(src), "r"(bytes), "r"(m) : "memory");
}

__device__ __forceinline__ void mbar_init(u64* mbar, u32 count) {
  const u32 m = static_cast<u32>(__cvta_generic_to_shared(mbar));
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(m), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(u64* mbar, u32 bytes) {
  const u32 m = static_cast<u32>(__cvta_generic_to_shared(mbar));
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
               :: "r"(m), "r"(bytes) : "memory");
}

// Waits for phase 0 of the barrier; false after the spin limit (the caller
// flags an error instead of hanging).
__device__ __forceinline__ bool mbar_wait0(u64* mbar) {
  const u32 m = static_cast<u32>(__cvta_generic_to_shared(mbar));
  for (u32 spins = 0; spins < kSpinLimit; ++spins) {
    u32 done = 0;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done) : "r"(m), "r"(0u) : "memory");
    if (done) return true;
  }
  return false;
}

// kVals = false sorts keys only (vals_in/vals_out unused): the packed seed
// carries each suffix's instance-local index in the low key bits.
// Blocks per SM: four 256x16 (a 56 KB pair tile: four fit the SM's shared
// memory; 64 registers, measured faster than three blocks at 80 despite a
// few spilled words), four 256x8, two 512x8 (three without values).
// Registers are capped so that occupancy, not the allocator, decides.
// kTma: the tile's keys arrive by one bulk copy into shared memory (single-
// segment sorts, whose tiles start on 4096-key boundaries) instead of
// per-thread loads; the rest is the same.
template <bool kBallot, int kBlock, int kItems, bool kVals = true, bool kTma = false>
static __global__ void __launch_bounds__(kBlock, kBlock == 512 ? (kVals ? 2 : 3) : 4)
radix_onesweep_kernel(const u64* __restrict__ keys_in,
                      const u32* __restrict__ vals_in,
                      u64* __restrict__ keys_out, u32* __restrict__ vals_out,
                      SortSegments segs, u32 shift, u32 pass, u32 passes,
                      const u64* __restrict__ digit_start, u64* status,
                      u32* tile_counter, DeviceFlags* flags) {
  static_assert(kBlock >= kRadixDigits, "one thread per digit");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  OnesweepSmem<kBlock, kBlock * kItems, kVals>& sm =
      *reinterpret_cast<OnesweepSmem<kBlock, kBlock * kItems, kVals>*>(smem_raw);
  constexpr int kWarps = kBlock / 32;
  const u32 lane = threadIdx.x & 31;
  const u32 warp = threadIdx.x >> 5;

  for (int i = threadIdx.x; i < kWarps * kRadixDigits; i += kBlock) {
    (&sm.warp_hist[0][0])[i] = 0;
  }
  const u32 tile = claim_tile(tile_counter, &sm.tile);
  u32 seg;
  u64 first, last;
  segment_of_tile(segs, tile, &seg, &first, &last);
  const u32 count = static_cast<u32>(last - first);
  const bool first_tile_of_segment = tile == segs.tile_begin[seg];

  // Warp-striped load: warp w owns tile slots [w*32*kItems, (w+1)*32*kItems).
  u64 key[kItems];
  u32 rank[kItems];
  const u32 warp_base = warp * 32 * kItems;
  u32 bulk = 0;  // keys that arrived by the bulk copy (an even count: 16-byte multiple)
  if (kTma) {
    // The bulk copy needs a 16-byte aligned source; some callers sort
    // buffers at 8-byte offsets (a second ping-pong half), which take the
    // per-thread loads instead (bulk = 0: the barrier completes at once).
    const bool aligned = (reinterpret_cast<uintptr_t>(keys_in + first) & 15) == 0;
    bulk = aligned ? count & ~1u : 0;
    if (threadIdx.x == 0) mbar_init(&sm.mbar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
      mbar_expect_tx(&sm.mbar, bulk * 8);
      if (bulk) bulk_load(sm.keys, keys_in + first, bulk * 8, &sm.mbar);
    }
    if (!mbar_wait0(&sm.mbar)) {
      flag_error(flags, kErrLookbackTimeout, 30);
      bulk = 0;  // fall back to global loads (the build already failed)
    }
  }
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    const u32 slot = warp_base + i * 32 + lane;
    key[i] = slot < count ? (slot < bulk ? sm.keys[slot] : keys_in[first + slot]) : ~0ull;
  }
  if (kTma) __syncthreads();  // sm.keys is the scatter buffer below
  // Stable warp-level ranking by digit; invalid slots never update counters.
  // kBallot selects peers with eight ballots over the digit bits instead of
  // one match-any.
  const u32 lanemask_lt = (1u << lane) - 1;
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    const u32 slot = warp_base + i * 32 + lane;
    const bool valid = slot < count;
    const u32 digit = valid ? static_cast<u32>((key[i] >> shift) & 0xff) : 0x100u;
    u32 peers;
    if (kBallot) {
      peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
      for (int b = 0; b < kRadixBits; ++b) {
        const bool bit = (digit >> b) & 1;
        const u32 vote = __ballot_sync(0xffffffffu, bit);
        peers &= bit ? vote : ~vote;
      }
      if (!valid) peers = 1u << lane;
    } else {
      peers = __match_any_sync(0xffffffffu, digit);
    }
    const u32 leader = __ffs(peers) - 1;
    u32 base = 0;
    if (valid && lane == leader) {
      base = sm.warp_hist[warp][digit];
      sm.warp_hist[warp][digit] = static_cast<unsigned short>(base + __popc(peers));
    }
    base = __shfl_sync(0xffffffffu, base, leader);
    rank[i] = base + __popc(peers & lanemask_lt);
    __syncwarp();
  }
  __syncthreads();

  // Per digit: tile count and tile-local start; then warp_hist[w][d] becomes
  // the first sorted slot of warp w's keys of digit d.
  const u32 d = threadIdx.x;
  u32 digit_count = 0;
  if (d < kRadixDigits) {
#pragma unroll
    for (int w = 0; w < kWarps; ++w) digit_count += sm.warp_hist[w][d];
  }
  u64 tile_total;
  const u64 local_start =
      block_exclusive_scan<kBlock>(digit_count, SumOp{}, sm.warp_scan, &tile_total);
  if (d < kRadixDigits) {
    u32 running = static_cast<u32>(local_start);
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      const u32 c = sm.warp_hist[w][d];
      sm.warp_hist[w][d] = static_cast<unsigned short>(running);
      running += c;
    }
  }

  // Decoupled look-back, one digit per thread.  Prefix values are absolute
  // output positions; a segment's first tile seeds them from digit_start.
  if (d < kRadixDigits) {
    u64* my_status = status + static_cast<u64>(tile) * kRadixDigits + d;
    u64 global_start;
    if (first_tile_of_segment) {
      global_start =
          digit_start[(static_cast<u64>(seg) * passes + pass) * kRadixDigits + d];
      store_status(my_status, kFlagPrefix | ((global_start + digit_count) & kValueMask));
    } else {
      store_status(my_status, kFlagAggregate | digit_count);
      u64 exclusive = 0;
      long long t = static_cast<long long>(tile) - 1;
      while (true) {
        const u64 v = wait_status(status + static_cast<u64>(t) * kRadixDigits + d,
                                  flags, 1);
        exclusive += v & kValueMask;
        if ((v >> 62) == 2) break;
        --t;
      }
      global_start = exclusive;
      store_status(my_status, kFlagPrefix | ((global_start + digit_count) & kValueMask));
    }
    sm.digit_gbase[d] = static_cast<long long>(global_start) - static_cast<long long>(local_start);
  }
  __syncthreads();

  // Keys and values to their tile-local sorted slot, then runs out.
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    const u32 slot = warp_base + i * 32 + lane;
    if (slot < count) {
      const u32 digit = static_cast<u32>((key[i] >> shift) & 0xff);
      const u32 local_slot = sm.warp_hist[warp][digit] + rank[i];
      sm.keys[local_slot] = key[i];
      if (kVals) sm.vals[local_slot] = vals_in[first + slot];
    }
  }
  __syncthreads();
  const u64 seg_first = segs.begin[seg];
  const u64 seg_end = segs.begin[seg + 1];
  for (u32 s = threadIdx.x; s < count; s += kBlock) {
    const u64 k = sm.keys[s];
    const u32 digit = static_cast<u32>((k >> shift) & 0xff);
    const u64 out = static_cast<u64>(sm.digit_gbase[digit] + static_cast<long long>(s));
    if (out < seg_first || out >= seg_end) {  // only after a failed look-back
      flag_error(flags, kErrBounds);
      continue;
    }
    keys_out[out] = k;
    if (kVals) vals_out[out] = sm.vals[s];
  }
}

}  // namespace sufgpu
