// Shared device helpers for the sufgpu construction engine (sm_100a).
//
// Everything here is integer work on HBM-resident arrays: 32-bit positions and
// ranks (a logical text of up to 2^32 - 1 symbols), 64-bit sort keys, and
// decoupled look-back status words for the single-pass scans and the onesweep
// radix passes.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sufgpu {

using u8 = std::uint8_t;
using u16 = std::uint16_t;
using u32 = std::uint32_t;
using u64 = std::uint64_t;

constexpr u32 kNone = 0xffffffffu;  // "no predecessor" in PHI

// Device error word bits (DeviceFlags::error).  The host reads them after every
// build and turns any set bit into a build failure.
enum : u32 {
  kErrLookbackTimeout = 1u << 0,  // a look-back wait hit its iteration limit
  kErrRoundLimit = 1u << 1,       // doubling did not converge
  kErrNotPermutation = 1u << 2,   // SA validation failed
  kErrLcpWidth = 1u << 3,         // LCP value exceeds the requested width
  kErrQueueOverflow = 1u << 4,    // long-LCP work queue overflowed
  kErrBounds = 1u << 5,           // an index check failed (debug builds)
};

struct DeviceFlags {
  u32 error;
  u32 timeout_site;  // first look-back site that timed out (debug aid)
};

// ---------------------------------------------------------------------------
// Decoupled look-back status words: [63:62] flag, [61:0] value.
//   flag 0 = not yet published, 1 = tile aggregate, 2 = inclusive prefix.
// The value and its flag share one 64-bit word, so relaxed GPU-scope loads and
// stores are enough: a reader that sees the flag sees the value with it.
// ---------------------------------------------------------------------------
constexpr u64 kFlagAggregate = 1ull << 62;
constexpr u64 kFlagPrefix = 2ull << 62;
constexpr u64 kValueMask = (1ull << 62) - 1;

__device__ __forceinline__ void store_status(u64* p, u64 v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v)
               : "memory");
}

__device__ __forceinline__ u64 load_status(const u64* p) {
  u64 v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p)
               : "memory");
  return v;
}

// Spin limit for one look-back wait.  Each failed poll sleeps ~100 ns, so the
// limit is ~0.4 s: far beyond any legitimate wait (a predecessor tile that has
// already started publishes within microseconds), short enough that a logic
// error returns an error instead of hanging the GPU.
constexpr u32 kSpinLimit = 1u << 22;

__device__ __forceinline__ void flag_error(DeviceFlags* flags, u32 bit,
                                           u32 site = 0) {
  const u32 old = atomicOr(&flags->error, bit);
  if (bit == kErrLookbackTimeout && (old & kErrLookbackTimeout) == 0) {
    flags->timeout_site = site;
  }
}

// Waits for the status word at p to be published; returns it.  On timeout the
// error flag is set and an inclusive prefix of 0 is returned so that the
// caller (and every tile behind it) finishes instead of waiting forever.
__device__ __forceinline__ u64 wait_status(const u64* p, DeviceFlags* flags,
                                           u32 site) {
  u64 v = load_status(p);
  u32 spins = 0;
  while ((v >> 62) == 0) {
    if (++spins > kSpinLimit) {
      flag_error(flags, kErrLookbackTimeout, site);
      return kFlagPrefix;
    }
    __nanosleep(100);
    v = load_status(p);
  }
  return v;
}

struct SumOp {
  __device__ __forceinline__ u64 operator()(u64 a, u64 b) const {
    return a + b;
  }
  static constexpr u64 identity = 0;
};
struct MaxOp {
  __device__ __forceinline__ u64 operator()(u64 a, u64 b) const {
    return a > b ? a : b;
  }
  static constexpr u64 identity = 0;
};

// Warp-cooperative look-back: warp 0 of a tile calls this with the tile's
// aggregate; every lane returns the exclusive prefix (op over all previous
// tiles).  Tile 0 publishes its aggregate as the inclusive prefix directly.
// Looks at 32 predecessors per step.
template <class Op>
__device__ __forceinline__ u64 warp_lookback(u64* status, u32 tile,
                                             u64 aggregate, Op op,
                                             DeviceFlags* flags, u32 site) {
  const u32 lane = threadIdx.x & 31;
  if (tile == 0) {
    if (lane == 0) store_status(&status[0], kFlagPrefix | (aggregate & kValueMask));
    return Op::identity;
  }
  if (lane == 0) store_status(&status[tile], kFlagAggregate | (aggregate & kValueMask));
  u64 exclusive = Op::identity;
  long long window_end = static_cast<long long>(tile) - 1;  // inclusive
  while (true) {
    const long long t = window_end - lane;
    u64 v = kFlagPrefix;  // beyond tile 0: acts as an identity prefix
    if (t >= 0) v = wait_status(&status[t], flags, site);
    const u32 prefix_mask = __ballot_sync(0xffffffffu, (v >> 62) == 2);
    // Lanes up to (and including) the nearest prefix contribute.
    const u32 stop = prefix_mask ? (__ffs(prefix_mask) - 1) : 32;
    u64 contrib = (lane <= stop && t >= 0) ? (v & kValueMask) : Op::identity;
    for (int offset = 16; offset > 0; offset >>= 1) {
      contrib = op(contrib, __shfl_down_sync(0xffffffffu, contrib, offset));
    }
    contrib = __shfl_sync(0xffffffffu, contrib, 0);
    exclusive = op(exclusive, contrib);
    if (prefix_mask) break;
    window_end -= 32;
  }
  if (lane == 0) {
    store_status(&status[tile], kFlagPrefix | (op(exclusive, aggregate) & kValueMask));
  }
  return exclusive;
}

// Warp-aggregated append of one item per participating lane (all 32 lanes
// call it): the lane's slot in the list whose length *counter holds.
__device__ __forceinline__ u64 warp_append(u64* counter, bool take) {
  const u32 mask = __ballot_sync(0xffffffffu, take);
  if (!mask) return 0;
  const u32 lane = threadIdx.x & 31;
  const u32 leader = __ffs(mask) - 1;
  u64 base = 0;
  if (lane == leader) base = atomicAdd(reinterpret_cast<unsigned long long*>(counter), __popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  return base + __popc(mask & ((1u << lane) - 1));
}

// Number of bits needed to represent values 0..v.
__host__ __device__ __forceinline__ u32 bits_for(u64 v) {
  u32 b = 0;
  while (b < 64 && (v >> b) != 0) ++b;
  return b;
}

// Segment (reference instance) lookup: the segment whose half-open element
// range [begin[j], begin[j+1]) contains x.  begin has count+1 entries.
__device__ __forceinline__ u32 find_segment(const u64* begin, u32 count,
                                            u64 x) {
  u32 lo = 0, hi = count;  // answer in [lo, hi)
  while (hi - lo > 1) {
    const u32 mid = (lo + hi) >> 1;
    if (begin[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Per-thread cache of the segment holding the last looked-up element; kernels
// whose threads walk increasing indices search only when they leave it.
struct SegCursor {
  u64 lo = 1, hi = 0;  // empty until the first lookup
  u32 j = 0;
  __device__ __forceinline__ void locate(const u64* begin, u32 count, u64 x) {
    if (x >= lo && x < hi) return;
    j = count == 1 ? 0 : find_segment(begin, count, x);
    lo = begin[j];
    hi = begin[j + 1];
  }
};

}  // namespace sufgpu
