// LCP kernels (row order), byte coding and overflow anchors.
//
// LCP[r] = lcp(SA[r-1], SA[r]).  Rows at seed-group boundaries already carry
// their LCP (from the seed keys).  Every other row compares up to 64 bytes
// past the seed length directly (on genomic text almost every row ends
// there).  A row whose next 64 bytes also match is "long":
//   * if its suffix b = SA[r] is irreducible (text[b-1] != text[a-1] for
//     a = SA[r-1], or b or a starts its instance), a warp finishes the compare;
//   * otherwise b is reducible: PLCP[b] = PLCP[b-1] - 1, and by induction
//     PLCP[b] = PLCP[p] - (b - p) for the nearest irreducible text position
//     p < b.  That p has PLCP[p] >= PLCP[b] + (b - p) > 64, so it is one of the
//     long irreducible rows; after those are sorted by position a binary search
//     finds it.
// This reaches the values of the reference's Kasai loop (src/divsufsort_
// backend.cpp:121-150) without a text-order carry chain, without the PHI
// scatter and without a row-order gather; only long rows touch a queue.
//
// Byte-coded overflow anchors (src/lcp_storage.cpp:394-412) open at text
// positions p with PLCP[p] >= 255 that do not continue the run of p-1.  A
// reducible p always continues, so anchors are a filter of the sorted long
// irreducible rows: p opens unless PLCP[p-1] == PLCP[p] + 1.
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

constexpr u32 kDirectLcpBytes = 64;

struct LongRow {
  u32 row;   // SA row
  u32 pos;   // suffix position b = SA[row]
  u32 prev;  // a = SA[row - 1]
  u32 done;  // bytes known equal
};

// Row pass.  lcp receives final values for short rows; long rows go to the
// irreducible queue or the pending (reducible) list.
// With known_prefix > 0, rows whose lcp[] is already set (seed-group heads,
// resolved from the seed keys) are skipped and the others start comparing at
// known_prefix, the seed length they are known to share.
// Each warp inspects kLcpChunk consecutive rows at a time, lists the ones that
// still need a compare in shared memory and then gives one listed row to each
// lane: the compare loop runs with full warps instead of idling the lanes of
// the (usually most) rows that are already resolved.
constexpr int kLcpChunk = 128;
constexpr int kLcpRowsBlock = 256;

// Number of leading equal bytes of text[b + m, ...) and text[a + m, ...)
// from m up to budget (at least budget once reached; the caller clamps).
// Reads aligned 8-byte words and carries each one into the next step, so a
// step costs one load per side; the last word read ends at most 15 bytes
// past position b + m (resp. a + m) < the instance end.  Sets *mismatch when
// a differing byte was found before budget.
__device__ __forceinline__ u32 match_length(const u8* __restrict__ text, u32 b, u32 a, u32 m,
                                            u32 budget, bool* mismatch) {
  *mismatch = false;
  if (m >= budget) return m;
  const u64 pb = static_cast<u64>(b) + m, pa = static_cast<u64>(a) + m;
  const u32 sb = static_cast<u32>(pb & 7) * 8, sa = static_cast<u32>(pa & 7) * 8;
  const unsigned long long* wb = reinterpret_cast<const unsigned long long*>(text + (pb & ~7ull));
  const unsigned long long* wa = reinterpret_cast<const unsigned long long*>(text + (pa & ~7ull));
  u64 lob = __ldg(wb), loa = __ldg(wa);
  while (true) {
    const u64 hib = __ldg(++wb), hia = __ldg(++wa);
    const u64 xb = sb ? (lob >> sb) | (hib << (64 - sb)) : lob;
    const u64 xa = sa ? (loa >> sa) | (hia << (64 - sa)) : loa;
    const u64 x = xb ^ xa;
    if (x) {
      *mismatch = true;
      return m + (static_cast<u32>(__ffsll(static_cast<long long>(x)) - 1) >> 3);
    }
    m += 8;
    if (m >= budget) return m;
    lob = hib;
    loa = hia;
  }
}

static __global__ void __launch_bounds__(kLcpRowsBlock)
lcp_rows_kernel(const u8* __restrict__ text, const u32* __restrict__ sa, u64 n,
                Segments segs, u32 known_prefix, u32* __restrict__ lcp,
                LongRow* __restrict__ longs, u64 long_cap, u64* long_count,
                u32* __restrict__ pending, u64 pending_cap, u64* pending_count,
                DeviceFlags* flags) {
  constexpr int kWarps = kLcpRowsBlock / 32;
  __shared__ u32 listed[kWarps][kLcpChunk];
  const u32 lane = threadIdx.x & 31;
  const u32 warp = threadIdx.x >> 5;
  const u32 lanemask_lt = (1u << lane) - 1;
  const u64 chunks = (n + kLcpChunk - 1) / kLcpChunk;
  const u64 warps_total = static_cast<u64>(gridDim.x) * kWarps;
  SegCursor cur;
  for (u64 ch = static_cast<u64>(blockIdx.x) * kWarps + warp; ch < chunks; ch += warps_total) {
    const u64 r0 = ch * kLcpChunk;
    u32 count = 0;
#pragma unroll
    for (int k = 0; k < kLcpChunk / 32; ++k) {
      const u64 r = r0 + k * 32 + lane;
      const bool need = r < n && (known_prefix == 0 || lcp[r] == kLcpUnknown);
      const u32 mask = __ballot_sync(0xffffffffu, need);
      if (need) listed[warp][count + __popc(mask & lanemask_lt)] = k * 32 + lane;
      count += __popc(mask);
    }
    __syncwarp();
    for (u32 base = 0; base < count; base += 32) {
      bool is_long = false, irreducible = false;
      u32 b = 0, a = 0, l = 0;
      u64 r = 0;
      if (base + lane < count) {
        r = r0 + listed[warp][base + lane];
        b = sa[r];
        cur.locate(segs.begin, segs.count, r);
        const u64 seg_first = cur.lo;
        // A caller-supplied SA (sufgpu_lcp_noalloc) may hold entries outside
        // the row's instance: flag them and skip the row instead of reading
        // text past the instance end.
        const bool b_bad = b < seg_first || b >= cur.hi;
        const bool a_bad = r != seg_first && (sa[r - 1] < seg_first || sa[r - 1] >= cur.hi);
        if (b_bad || a_bad) {
          flag_error(flags, kErrBounds);
          lcp[r] = 0;
        } else if (r == seg_first) {
          lcp[r] = 0;
        } else {
          a = sa[r - 1];
          const u32 far = a > b ? a : b;
          const u32 limit = static_cast<u32>(cur.hi - far);
          const u32 budget = min(limit, known_prefix + kDirectLcpBytes);
          bool mismatch;
          u32 m = match_length(text, b, a, min(known_prefix, limit), budget, &mismatch);
          if (m > limit) m = limit;
          if (mismatch || m >= limit) {
            lcp[r] = m;
          } else {
            is_long = true;
            l = m;
            irreducible = b == seg_first || a == seg_first || text[b - 1] != text[a - 1];
          }
        }
      }
      const u64 q = warp_append(long_count, is_long && irreducible);
      if (is_long && irreducible) {
        if (q < long_cap) longs[q] = LongRow{static_cast<u32>(r), b, a, l};
        else flag_error(flags, kErrQueueOverflow);
      }
      const u64 sidx = warp_append(pending_count, is_long && !irreducible);
      if (is_long && !irreducible) {
        if (sidx < pending_cap) pending[sidx] = static_cast<u32>(r);
        else flag_error(flags, kErrQueueOverflow);
      }
    }
    __syncwarp();  // the list is rewritten for the next chunk
  }
}

// One warp per long irreducible row: 32 lanes x 16 bytes per step.  Writes
// the final LCP and the (position, value) pair for the position sort.
static __global__ void __launch_bounds__(256)
long_rows_kernel(const u8* __restrict__ text, const LongRow* __restrict__ longs,
                 const u64* long_count, u64 long_cap, Segments segs,
                 u32* __restrict__ lcp, u64* __restrict__ sort_pos,
                 u32* __restrict__ sort_val) {
  const u32 lane = threadIdx.x & 31;
  const u64 warps = static_cast<u64>(gridDim.x) * (blockDim.x / 32);
  u64 count = *long_count;
  if (count > long_cap) count = long_cap;
  for (u64 w = (static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x) / 32; w < count; w += warps) {
    const LongRow item = longs[w];
    const u64 end = segment_end(segs, item.row);
    const u64 far = item.pos > item.prev ? item.pos : item.prev;
    const u64 limit = end - far;
    u64 l = item.done;
    while (l < limit) {
      const u64 off = l + lane * 16;
      // Lanes at or past the limit load nothing and report a stop at off, so
      // loads never reach beyond limit + 16 <= the padded end of the text.
      u64 local = 0;
      if (off < limit) {
        const u64 x0 = load8(text, item.pos + off) ^ load8(text, item.prev + off);
        const u64 x1 = load8(text, item.pos + off + 8) ^ load8(text, item.prev + off + 8);
        local = 16;
        if (x0) local = static_cast<u64>(__ffsll(static_cast<long long>(x0)) - 1) >> 3;
        else if (x1) local = 8 + (static_cast<u64>(__ffsll(static_cast<long long>(x1)) - 1) >> 3);
      }
      const u32 hit = __ballot_sync(0xffffffffu, local < 16);
      if (hit) {
        l = __shfl_sync(0xffffffffu, off + local, __ffs(hit) - 1);
        break;
      }
      l += 512;
    }
    if (l > limit) l = limit;
    if (lane == 0) {
      lcp[item.row] = static_cast<u32>(l);
      sort_pos[w] = item.pos;
      sort_val[w] = static_cast<u32>(l);
    }
  }
}

// Pending (reducible long) rows: PLCP[b] = PLCP[p] - (b - p) with p the last
// long irreducible position <= b (sorted_pos is ascending).
static __global__ void __launch_bounds__(256)
pending_rows_kernel(const u32* __restrict__ sa, const u32* __restrict__ pending,
                    const u64* pending_count, u64 pending_cap,
                    const u64* __restrict__ sorted_pos, const u32* __restrict__ sorted_val,
                    const u64* long_count, u64 long_cap, u32* __restrict__ lcp,
                    DeviceFlags* flags) {
  u64 count = *pending_count;
  if (count > pending_cap) count = pending_cap;
  u64 q = *long_count;
  if (q > long_cap) q = long_cap;
  const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
  for (u64 k = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; k < count; k += stride) {
    const u32 r = pending[k];
    const u64 b = sa[r];
    u64 lo = 0, hi = q;  // first index with sorted_pos > b
    while (lo < hi) {
      const u64 mid = (lo + hi) >> 1;
      if (sorted_pos[mid] <= b) lo = mid + 1;
      else hi = mid;
    }
    if (lo == 0) {
      flag_error(flags, kErrBounds);
      continue;
    }
    const u64 p = sorted_pos[lo - 1];
    lcp[r] = sorted_val[lo - 1] - static_cast<u32>(b - p);
  }
}

template <class Out>
static __global__ void __launch_bounds__(256)
widen_kernel(const u32* __restrict__ in, u64 n, Out* __restrict__ out) {
  const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
  for (u64 r = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += stride) {
    out[r] = static_cast<Out>(in[r]);
  }
}

static __global__ void __launch_bounds__(256)
lcp_primary_kernel(const u32* __restrict__ lcp, u64 n, u8* __restrict__ primary) {
  const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
  for (u64 r = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += stride) {
    const u32 v = lcp[r];
    primary[r] = static_cast<u8>(v < 255 ? v : 255);
  }
}

// Overflow anchors from the position-sorted long irreducible rows (global
// positions; the host splits them per instance).  Compaction keeps order.
template <class Coord>
static __global__ void __launch_bounds__(kScanBlock)
anchor_kernel(const u64* __restrict__ sorted_pos, const u32* __restrict__ sorted_val,
              const u64* long_count, u64 long_cap, Segments segs,
              const u32* __restrict__ rank, const u32* __restrict__ lcp,
              Coord* __restrict__ anchor_pos, Coord* __restrict__ anchor_val,
              u64 anchor_cap, u64* status_sum, u32* tile_counter,
              u64* anchor_count, DeviceFlags* flags) {
  __shared__ u64 warp_smem[kScanBlock / 32];
  __shared__ u64 tile_prefix;
  __shared__ u32 tile_slot;
  u64 q = *long_count;
  if (q > long_cap) q = long_cap;
  const u32 tile = claim_tile(tile_counter, &tile_slot);
  const u64 i0 = static_cast<u64>(tile) * kScanTile + threadIdx.x * kScanItems;
  bool open[kScanItems];
  u32 opens = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const u64 i = i0 + k;
    open[k] = false;
    if (i < q && sorted_val[i] >= 255) {
      const u64 p = sorted_pos[i];
      bool continues = false;
      if (!is_segment_start(segs, p)) continues = lcp[rank[p - 1]] == sorted_val[i] + 1;
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
      anchor_pos[out] = static_cast<Coord>(sorted_pos[i]);
      anchor_val[out] = static_cast<Coord>(sorted_val[i]);
    } else {
      flag_error(flags, kErrQueueOverflow);
    }
    ++out;
  }
  if (threadIdx.x == 0 && (tile + 1) * static_cast<u64>(kScanTile) >= q) {
    // The tile holding the last item writes the total (tile_prefix covers
    // every earlier tile).
    *anchor_count = tile_prefix + agg;
  }
}

// Byte-coded overflow anchors of a sampled build (rate K > 1), in sample
// order: sample t of instance i (s = t - off[i], text position s*K) has
// PLCP_K = lcp_k[off[i] + isa_k[t]]; it opens an anchor when PLCP_K >= 255
// unless sample s-1 of the same instance overflowed with a value v' >= K and
// v' - K == PLCP_K (src/lcp_storage.cpp:394-412 with sampling rate K).
// Anchors are instance-local positions; inst_count[i] counts instance i's.
template <class Coord>
static __global__ void __launch_bounds__(kScanBlock)
sampled_anchor_kernel(const u32* __restrict__ isa_k, const u32* __restrict__ lcp_k,
                      const u64* __restrict__ off, u32 count, u64 kept, u32 rate,
                      Coord* __restrict__ anchor_pos, Coord* __restrict__ anchor_val,
                      u64 anchor_cap, u64* __restrict__ inst_count, u64* status_sum,
                      u32* tile_counter, u64* anchor_count, DeviceFlags* flags) {
  __shared__ u64 warp_smem[kScanBlock / 32];
  __shared__ u64 tile_prefix;
  __shared__ u32 tile_slot;
  const u32 tile = claim_tile(tile_counter, &tile_slot);
  const u64 t0 = static_cast<u64>(tile) * kScanTile + threadIdx.x * kScanItems;
  bool open[kScanItems];
  u32 value[kScanItems];
  u32 inst_of[kScanItems];
  u32 opens = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const u64 t = t0 + k;
    open[k] = false;
    value[k] = 0;
    inst_of[k] = 0;
    if (t >= kept) continue;
    const u32 inst = count == 1 ? 0 : find_segment(off, count, t);
    const u64 base = off[inst];
    const u64 rows = off[inst + 1] - base;
    const u32 row = isa_k[t];
    if (row >= rows) {
      flag_error(flags, kErrBounds);
      continue;
    }
    const u32 v = lcp_k[base + row];
    if (v < 255) continue;
    bool continues = false;
    if (t > base) {
      const u32 prow = isa_k[t - 1];
      if (prow < rows) {
        const u32 pv = lcp_k[base + prow];
        continues = pv >= 255 && pv >= rate && pv - rate == v;
      }
    }
    open[k] = !continues;
    value[k] = v;
    inst_of[k] = inst;
    opens += open[k];
  }
  u64 agg;
  const u64 excl = block_exclusive_scan<kScanBlock>(opens, SumOp{}, warp_smem, &agg);
  if ((threadIdx.x >> 5) == 0) {
    const u64 p = warp_lookback(status_sum, tile, agg, SumOp{}, flags, 9);
    if ((threadIdx.x & 31) == 0) tile_prefix = p;
  }
  __syncthreads();
  u64 out = tile_prefix + excl;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (!open[k]) continue;
    const u64 t = t0 + k;
    if (out < anchor_cap) {
      anchor_pos[out] = static_cast<Coord>((t - off[inst_of[k]]) * rate);
      anchor_val[out] = static_cast<Coord>(value[k]);
      atomicAdd(reinterpret_cast<unsigned long long*>(inst_count + inst_of[k]), 1ull);
    } else {
      flag_error(flags, kErrQueueOverflow);
    }
    ++out;
  }
  if (threadIdx.x == 0 && (tile + 1) * static_cast<u64>(kScanTile) >= kept) {
    *anchor_count = tile_prefix + agg;
  }
}

}  // namespace sufgpu
