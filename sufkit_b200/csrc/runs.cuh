// Long single-symbol runs (N gaps, poly-A tracts): ordered directly instead of
// by prefix doubling.
//
// A position p inside a run of symbol c that still has d >= s symbols of the
// run ahead of it (s = seed length) has the seed key c^s, so all such
// "members" of one instance share one seed group.  With x the symbol after
// the run (or the instance end, which sorts first) and e = p + d the run end:
//   * members with x < c ("class 0") precede members with x > c ("class 1");
//   * class 0 is ordered by d ascending, class 1 by d descending;
//   * equal (class, d) are ordered by the suffix at e.
// So the seed group splits at once into sub-groups (class, d), laid out by
// counting: with the class's runs sorted by length L, sub-group d holds
// cnt(d) = #{L >= d} rows and starts after sum_{d' < d} cnt(d') rows (class 0)
// or sum_{d' > d} cnt(d') rows (class 1).  A doubling round with offset h then
// compares a member by the rank of its run end e whenever d >= h: the
// sub-group shares d symbols and e's group shares h, so equal keys still
// share >= 2h symbols and every round keeps the usual invariant.  Without
// this, a run of length L keeps ~L suffixes active for log2(L/s) rounds
// (2.1 G row-rounds for the 150 Mbp of N runs in a human-scale reference).
#pragma once

#include "common.cuh"
#include "doubling.cuh"

namespace sufgpu {

// Long-run boundary records, appended unordered (the host sorts them):
//   start: (a << 8) | c      a = first position, c = the run's byte
//   end:   (e << 1) | class  e = one past the last position
// Only runs of length >= s inside one instance are recorded.  counts[0] and
// counts[1] receive the number of starts and ends (beyond cap: counted, not
// written; the host then leaves the runs to the doubling rounds).
constexpr u32 kRunChunk = 16;

static __global__ void __launch_bounds__(256)
long_runs_kernel(const u8* __restrict__ text, u64 n, Segments segs, u32 s,
                 u64* __restrict__ starts, u64* __restrict__ ends, u64 cap,
                 u64* __restrict__ counts) {
  const u64 chunks = (n + kRunChunk - 1) / kRunChunk;
  for (u64 ch = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; ch < chunks;
       ch += static_cast<u64>(gridDim.x) * blockDim.x) {
    const u64 base = ch * kRunChunk;
    // The text buffer is padded past n, so the 16-byte load is in bounds.
    const uint4 v = *reinterpret_cast<const uint4*>(text + base);
    const u32 w[4] = {v.x, v.y, v.z, v.w};
    // A run of >= 16 identical bytes covers a whole aligned 8-byte word, so
    // with s >= 16 a chunk that starts or ends one sees a uniform word among
    // the chunk's two and its neighbours' (random sequence: almost never).
    // With 11 <= s < 16 a run covers two consecutive aligned 4-byte words
    // in [base - 8, base + 24); with 8 <= s < 11 one aligned 4-byte word in
    // [base - 4, base + 20).
    if (s >= 16) {
      const u64* w8 = reinterpret_cast<const u64*>(text + base);
      const u64 around[4] = {base >= 8 ? w8[-1] : 0x0102030405060708ull,
                             (static_cast<u64>(v.y) << 32) | v.x,
                             (static_cast<u64>(v.w) << 32) | v.z, w8[2]};
      bool any = false;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        any |= around[k] == (around[k] & 0xffull) * 0x0101010101010101ull;
      }
      if (!any) continue;
    } else if (s >= 11) {
      const u32* w4 = reinterpret_cast<const u32*>(text + base);
      const u32 around[8] = {base >= 8 ? w4[-2] : 0x01020304u, base >= 4 ? w4[-1] : 0x05060708u,
                             v.x, v.y, v.z, v.w, w4[4], w4[5]};
      bool any = false;
#pragma unroll
      for (int k = 0; k + 1 < 8; ++k) {
        any |= around[k] == around[k + 1] && around[k] == (around[k] & 0xffu) * 0x01010101u;
      }
      if (!any) continue;
    } else {
      const u32* w4 = reinterpret_cast<const u32*>(text + base);
      const u32 around[6] = {base >= 4 ? w4[-1] : 0x01020304u, v.x, v.y, v.z, v.w, w4[4]};
      bool any = false;
#pragma unroll
      for (int k = 0; k < 6; ++k) any |= around[k] == (around[k] & 0xffu) * 0x01010101u;
      if (!any) continue;
    }
    const u8 before = base > 0 ? text[base - 1] : 0;
    const u8 after = text[base + kRunChunk];
    SegCursor cur;
    for (u32 i = 0; i < kRunChunk; ++i) {
      const u64 p = base + i;
      if (p >= n) break;
      const u8 c = static_cast<u8>(w[i >> 2] >> ((i & 3) * 8));
      const u8 prev = i ? static_cast<u8>(w[(i - 1) >> 2] >> (((i - 1) & 3) * 8)) : before;
      const u8 next = i + 1 < kRunChunk ? static_cast<u8>(w[(i + 1) >> 2] >> (((i + 1) & 3) * 8))
                                        : after;
      // Cheap rejections first: a long run starts where the next byte repeats
      // c and ends where the previous byte does.
      const bool maybe_start = next == c;
      const bool maybe_end = prev == c;
      if (!maybe_start && !maybe_end) continue;
      cur.locate(segs.begin, segs.count, p);
      const u64 lo = cur.lo, hi = segs.end ? segs.end[cur.j] : cur.hi;
      if (maybe_start && (p == lo || prev != c) && p + s <= hi) {
        bool longrun = true;
        for (u32 k = 2; k < s; ++k) {
          if (text[p + k] != c) {
            longrun = false;
            break;
          }
        }
        if (longrun) {
          const u64 at = atomicAdd(reinterpret_cast<unsigned long long*>(&counts[0]), 1ull);
          if (at < cap) starts[at] = (p << 8) | c;
        }
      }
      if (maybe_end && (p + 1 == hi || next != c) && p + 1 >= lo + s) {
        bool longrun = true;
        for (u32 k = 2; k < s; ++k) {
          if (text[p - k] != c) {
            longrun = false;
            break;
          }
        }
        if (longrun) {
          const u64 e = p + 1;
          const u32 cls = (e == hi || text[e] < c) ? 0u : 1u;
          const u64 at = atomicAdd(reinterpret_cast<unsigned long long*>(&counts[1]), 1ull);
          if (at < cap) ends[at] = (e << 1) | cls;
        }
      }
    }
  }
}

// One run, in position order (run_a/run_e hold the same runs as plain arrays
// for the round lookup).
struct RunRecord {
  u64 first_member;  // members of runs before this one (prefix over runs)
  u32 a, e;          // run [a, e)
  u32 desc;          // its (instance, symbol, class) descriptor
  u32 slot;          // row offset inside every sub-group it belongs to
  u32 g0;            // head row of the seed group (gathered on the device)
  u32 pad;
};

// Runs of one (instance, symbol, class): sub-group layout inputs.
struct RunClass {
  u64 base_rel;       // first row of the class, relative to the seed group head
  u64 act_first_rel;  // first row (relative to the class) in a sub-group of >= 2
  u64 act_count;      // rows in sub-groups of >= 2
  u64 act_off;        // their offset in the appended active region
  u64 size;           // rows in the class
  u32 off;            // into sorted_len (m entries) and prefix (m + 1 entries)
  u32 poff;
  u32 m;
  u32 cls;
};

static __global__ void __launch_bounds__(256)
run_heads_kernel(RunRecord* __restrict__ runs, u32 count, const u32* __restrict__ rank) {
  const u32 r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < count) runs[r].g0 = rank[runs[r].a];
}

// Sub-group head of a member with d symbols of run ahead (see the header).
__device__ __forceinline__ u64 run_subgroup_head(const RunClass& k, const u32* sorted_len,
                                                 const u64* prefix, u32 s, u64 d) {
  const u32* L = sorted_len + k.off;
  const u64* P = prefix + k.poff;
  // lo = #{L < d} (class 0) or #{L <= d} (class 1).
  u32 lo = 0, hi = k.m;
  while (lo < hi) {
    const u32 mid = (lo + hi) >> 1;
    const bool left = k.cls == 0 ? L[mid] < d : L[mid] <= d;
    if (left) lo = mid + 1;
    else hi = mid;
  }
  if (k.cls == 0) return k.base_rel + P[lo] + static_cast<u64>(k.m - lo) * (d - s);
  return k.base_rel + (P[k.m] - P[lo]) - d * static_cast<u64>(k.m - lo);
}

// One thread per member: its SA row, its rank (sub-group head) and, for
// sub-groups of two or more, its slot in the appended active region.
static __global__ void __launch_bounds__(256)
run_split_kernel(const RunRecord* __restrict__ runs, u32 count,
                 const RunClass* __restrict__ classes, const u32* __restrict__ sorted_len,
                 const u64* __restrict__ prefix, u32 s, u64 members, u64 rows,
                 u32* __restrict__ sa, u32* __restrict__ rank, u32* __restrict__ active,
                 u64 active_base, DeviceFlags* flags) {
  for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < members;
       i += static_cast<u64>(gridDim.x) * blockDim.x) {
    u32 lo = 0, hi = count;  // the run r with first_member <= i
    while (hi - lo > 1) {
      const u32 mid = (lo + hi) >> 1;
      if (runs[mid].first_member <= i) lo = mid;
      else hi = mid;
    }
    const RunRecord run = runs[lo];
    const u64 p = run.a + (i - run.first_member);
    const u64 d = run.e - p;
    const RunClass k = classes[run.desc];
    const u64 head_rel = run_subgroup_head(k, sorted_len, prefix, s, d);
    const u64 row_rel = head_rel + run.slot;  // relative to the seed group head
    const u64 in_class = row_rel - k.base_rel;
    const u64 row = run.g0 + row_rel;
    if (d < s || p >= run.e || in_class >= k.size || row >= rows) {
      flag_error(flags, kErrBounds);
      continue;
    }
    rank[p] = static_cast<u32>(run.g0 + head_rel);
    // Rows of sub-groups of two or more get their SA entry from the round
    // that sorts them; singletons are final here.
    if (in_class >= k.act_first_rel && in_class < k.act_first_rel + k.act_count) {
      const u64 slot = active_base + k.act_off + (in_class - k.act_first_rel);
      if (slot >= rows) {
        flag_error(flags, kErrBounds);
        continue;
      }
      active[slot] = static_cast<u32>(p);
    } else {
      sa[row] = static_cast<u32>(p);
    }
  }
}

}  // namespace sufgpu
