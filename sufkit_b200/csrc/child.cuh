// Compact CHILD table (enhanced suffix array navigation) from the row LCP.
//
// sufkit builds it with two sequential monotone-stack passes
// (BuildChildFor, src/suffix_array.cpp:1438-1496): down and up links in the
// first, next-L links (overriding) in the second; n marks "no link".  The
// final entry of row x follows from three nearest-value arrays, which the GPU
// computes for every row independently:
//   NSE(x) = first i > x with LCP[i] <= LCP[x]   (n if none)
//   NS(x)  = first i > x with LCP[i] <  LCP[x]   (n if none)
//   PSE(x) = last  k < x with LCP[k] <= LCP[x]   (none if none)
// and
//   child[x] = NSE(x)                          if NSE(x) < n, LCP[NSE(x)] == LCP[x]
//            = max{m : PSE(m) = x}             elif NSE(x) > x + 1          (down)
//            = min{m : NS(m) = x + 1}          elif LCP[x+1] < LCP[x]        (up)
//            = n                               otherwise.
// (The down link is the leftmost minimum of LCP(x, NSE(x)), which is the
// largest row whose previous smaller-or-equal value is x; the up link is the
// last entry the stack pops at x + 1, the smallest row whose next strictly
// smaller value is x + 1.)  The searches run over a tree of minima with
// fan-out 32, so a row whose answer is far away (LCP rising through a long
// repeat) climbs O(log_32 n) levels instead of scanning.
#pragma once

#include "common.cuh"

namespace sufgpu {

constexpr int kChildFan = 32;
constexpr int kChildMaxLevels = 8;  // 32^7 > 2^32 rows

// The levels of minima: level 0 is the LCP itself; level k+1 holds the
// minimum of each 32 entries of level k.
struct MinTree {
  const u32* level[kChildMaxLevels];
  u64 size[kChildMaxLevels];
  int levels;  // including level 0
};

static __global__ void __launch_bounds__(256)
child_min_level_kernel(const u32* __restrict__ in, u64 count, u32* __restrict__ out,
                       u64 out_count) {
  const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
  for (u64 b = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; b < out_count;
       b += stride) {
    const u64 first = b * kChildFan;
    const u64 last = first + kChildFan < count ? first + kChildFan : count;
    u32 m = 0xffffffffu;
    for (u64 i = first; i < last; ++i) m = min(m, __ldg(in + i));
    out[b] = m;
  }
}

template <bool kStrict>
__device__ __forceinline__ bool child_hit(u32 value, u32 v) {
  return kStrict ? value < v : value <= v;
}

// First index > x whose value is <= v (< v when kStrict), or n.
template <bool kStrict>
__device__ u64 child_next(const MinTree& t, u64 x, u32 v) {
  const u64 n = t.size[0];
  // Rest of x's group of 32 at level 0, then siblings at higher levels.
  u64 idx = x;
  int lev = 0;
  u64 found = ~0ull;
  while (lev < t.levels) {
    const u64 end_group = (idx | (kChildFan - 1)) + 1;
    const u64 end = end_group < t.size[lev] ? end_group : t.size[lev];
    for (u64 j = idx + 1; j < end; ++j) {
      if (child_hit<kStrict>(__ldg(t.level[lev] + j), v)) {
        found = j;
        break;
      }
    }
    if (found != ~0ull) break;
    idx >>= 5;
    ++lev;
  }
  if (found == ~0ull) return n;
  // Descend to the first hit inside the found subtree.
  while (lev > 0) {
    --lev;
    const u64 first = found * kChildFan;
    const u64 last = first + kChildFan < t.size[lev] ? first + kChildFan : t.size[lev];
    u64 j = first;
    while (j < last && !child_hit<kStrict>(__ldg(t.level[lev] + j), v)) ++j;
    if (j >= last) return n;  // unreachable: the parent's minimum guarantees a hit
    found = j;
  }
  return found;
}

// Last index < x whose value is <= v, or ~0 (none).
__device__ u64 child_prev(const MinTree& t, u64 x, u32 v) {
  u64 idx = x;
  int lev = 0;
  u64 found = ~0ull;
  while (lev < t.levels) {
    const u64 begin = idx & ~static_cast<u64>(kChildFan - 1);
    for (u64 j = idx; j > begin;) {
      --j;
      if (__ldg(t.level[lev] + j) <= v) {
        found = j;
        break;
      }
    }
    if (found != ~0ull) break;
    idx >>= 5;
    ++lev;
  }
  if (found == ~0ull) return ~0ull;
  while (lev > 0) {
    --lev;
    const u64 first = found * kChildFan;
    const u64 last = first + kChildFan < t.size[lev] ? first + kChildFan : t.size[lev];
    u64 j = last;
    while (j > first && __ldg(t.level[lev] + j - 1) > v) --j;
    if (j == first) return ~0ull;  // unreachable, as above
    found = j - 1;
  }
  return found;
}

// Per row: NSE(x) into nse, and the scatters down[PSE(x)] = max(x),
// up[NS(x)] = min(x).  down starts at 0, up at n.
static __global__ void __launch_bounds__(256)
child_links_kernel(MinTree t, u32* __restrict__ nse, u32* __restrict__ down,
                   u32* __restrict__ up) {
  const u64 n = t.size[0];
  const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
  for (u64 x = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; x < n; x += stride) {
    const u32 v = __ldg(t.level[0] + x);
    const u64 next_le = child_next<false>(t, x, v);
    nse[x] = static_cast<u32>(next_le);
    // Rows between x and NSE(x) are > v, so NS(x) is NSE(x) or lies beyond it.
    u64 next_lt = n;
    if (next_le < n) {
      next_lt = __ldg(t.level[0] + next_le) < v ? next_le : child_next<true>(t, next_le, v);
    }
    if (next_lt < n) atomicMin(up + next_lt, static_cast<u32>(x));
    const u64 prev_le = child_prev(t, x, v);
    if (prev_le != ~0ull) atomicMax(down + prev_le, static_cast<u32>(x));
  }
}

static __global__ void __launch_bounds__(256)
child_final_kernel(const u32* __restrict__ lcp, u64 n, const u32* __restrict__ nse,
                   const u32* __restrict__ down, const u32* __restrict__ up,
                   u32* __restrict__ child) {
  const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
  for (u64 x = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; x < n; x += stride) {
    const u64 j = nse[x];
    const u32 v = lcp[x];
    u64 out = n;
    if (j < n && lcp[j] == v) {
      out = j;
    } else if (j > x + 1) {
      out = down[x];
    } else if (x + 1 < n && lcp[x + 1] < v) {
      out = up[x + 1];
    }
    child[x] = static_cast<u32>(out);
  }
}

}  // namespace sufgpu
