// sufgpu_lcp_noalloc: the row-order LCP phase for callers that cannot
// allocate device memory.
//
// Some callers can't call cudaMalloc: code running inside another framework's
// allocator (its pool owns every byte of the device and a foreign cudaMalloc
// fails or fragments it), callbacks that run while an allocation lock is held,
// and real-time loops where an allocation may block for milliseconds.  This
// entry point computes LCP[r] = lcp(SA[r-1], SA[r]) for a device-resident
// text and suffix array into a caller-owned device array, and takes every
// byte of scratch (the text copy with its read-ahead padding, the long-row
// queue, the pending list, the position sort and its look-back words) from
// one fixed array compiled into this library.  It never calls cudaMalloc,
// cudaFree or any allocating library routine.
//
// Limits and sharing:
//   * n <= SUFGPU_NOALLOC_MAX_SYMBOLS (2^18); larger inputs are rejected.
//   * The scratch array (kScratchBytes = 11,952,896 bytes, 11.4 MiB; a
//     static_assert below keeps it under 12 MiB) exists on every GPU that
//     loads the library, from load until process exit.
//   * sa must be a permutation of [0, n).  An entry outside [0, n) is
//     flagged by the row kernel, which skips that row's text compare, and
//     the call returns SUFGPU_BUILD_FAILURE.
//   * All calls share it and it keeps the previous call's contents; each call
//     clears what must start at zero.  Calls that overlap on the GPU (two
//     streams, two host threads) race on it and must be serialized by the
//     caller.
//   * The first call on a device does the one-time set-up for that device:
//     with the device current it resolves the array's device address
//     (cudaGetSymbolAddress) and sets a kernel attribute.  Make that first
//     call on each device before any stream capture begins.

#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/sufgpu/sufgpu.h"
#include "common.cuh"
#include "lcp.cuh"
#include "radix.cuh"

using namespace sufgpu;

namespace {

constexpr u64 kMax = SUFGPU_NOALLOC_MAX_SYMBOLS;
constexpr u64 kTextPad = 64;
constexpr u64 kMaxTiles = (kMax + kSortTile - 1) / kSortTile;

constexpr u64 align256(u64 v) { return (v + 255) / 256 * 256; }

// Scratch layout (byte offsets).
constexpr u64 kOffText = 0;
constexpr u64 kOffLongs = kOffText + align256(kMax + kTextPad);
constexpr u64 kOffPending = kOffLongs + align256(kMax * sizeof(LongRow));
constexpr u64 kOffKeys = kOffPending + align256(kMax * 4);
constexpr u64 kOffKeysAlt = kOffKeys + align256(kMax * 8);
constexpr u64 kOffVals = kOffKeysAlt + align256(kMax * 8);
constexpr u64 kOffValsAlt = kOffVals + align256(kMax * 4);
constexpr u64 kOffStatus = kOffValsAlt + align256(kMax * 4);
constexpr u64 kOffHist = kOffStatus + align256(kMaxTiles * kRadixDigits * 8);
constexpr u64 kOffDigits = kOffHist + align256(kMaxPasses * kRadixDigits * 4);
constexpr u64 kOffSmall = kOffDigits + align256(kMaxPasses * kRadixDigits * 8);
// Small area: seg_begin[2] (u64), sort_begin[2] (u64), seg_tiles[2] (u32),
// counters[64] (u32), scalars[16] (u64), flags.
constexpr u64 kSmallBytes = 16 + 16 + 8 + 256 + 128 + sizeof(DeviceFlags);
constexpr u64 kScratchBytes = kOffSmall + align256(kSmallBytes);
static_assert(kScratchBytes <= (u64(12) << 20), "the documented scratch bound is 12 MiB");

static __device__ __align__(256) unsigned char g_lcp_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

// Once per device, with that device current: the device address of the
// scratch array (a host-side reference to g_lcp_scratch is only a stand-in).
cudaError_t scratch_for_current_device(unsigned char** out) {
  int device = 0;
  cudaError_t err = cudaGetDevice(&device);
  if (err != cudaSuccess) return err;
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[device]) {
    void* ptr = nullptr;
    err = cudaGetSymbolAddress(&ptr, g_lcp_scratch);
    if (err != cudaSuccess) return err;
    err = cudaFuncSetAttribute(radix_onesweep_kernel<true, kSortBlock, kSortItems>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(sizeof(OnesweepSmem<kSortBlock, kSortTile, true>)));
    if (err != cudaSuccess) return err;
    g_scratch_ptr[device] = static_cast<unsigned char*>(ptr);
  }
  *out = g_scratch_ptr[device];
  return cudaSuccess;
}

#define NA_CUDA(call)                        \
  do {                                       \
    if ((call) != cudaSuccess) {             \
      cudaGetLastError();                    \
      return SUFGPU_BUILD_FAILURE;           \
    }                                        \
  } while (0)

u64 blocks_for(u64 work) {
  const u64 want = (work + 255) / 256;
  return want < 1 ? 1 : (want > 148 * 16 ? 148 * 16 : want);
}

}  // namespace

extern "C" sufgpu_status sufgpu_lcp_noalloc(const uint8_t* text, const uint32_t* sa,
                                            uint64_t n, uint32_t* lcp, void* stream_handle) {
  if (n > kMax) return SUFGPU_INVALID_INPUT;  // beyond the fixed scratch size
  if (n == 0) return SUFGPU_OK;
  if (!text || !sa || !lcp) return SUFGPU_INVALID_INPUT;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_handle);
  unsigned char* base = nullptr;
  NA_CUDA(scratch_for_current_device(&base));

  u8* d_text = base + kOffText;
  LongRow* longs = reinterpret_cast<LongRow*>(base + kOffLongs);
  u32* pending = reinterpret_cast<u32*>(base + kOffPending);
  u64* keys = reinterpret_cast<u64*>(base + kOffKeys);
  u64* keys_alt = reinterpret_cast<u64*>(base + kOffKeysAlt);
  u32* vals = reinterpret_cast<u32*>(base + kOffVals);
  u32* vals_alt = reinterpret_cast<u32*>(base + kOffValsAlt);
  u64* status = reinterpret_cast<u64*>(base + kOffStatus);
  u32* hist = reinterpret_cast<u32*>(base + kOffHist);
  u64* digits = reinterpret_cast<u64*>(base + kOffDigits);
  unsigned char* small = base + kOffSmall;
  u64* seg_begin = reinterpret_cast<u64*>(small);
  u64* sort_begin = reinterpret_cast<u64*>(small + 16);
  u32* sort_tiles = reinterpret_cast<u32*>(small + 32);
  u32* counters = reinterpret_cast<u32*>(small + 40);
  u64* scalars = reinterpret_cast<u64*>(small + 40 + 256);
  DeviceFlags* flags = reinterpret_cast<DeviceFlags*>(small + 40 + 256 + 128);

  // The kernels read up to 16 bytes past a compared position, so the text is
  // copied into the padded scratch region.
  NA_CUDA(cudaMemcpyAsync(d_text, text, n, cudaMemcpyDeviceToDevice, stream));
  NA_CUDA(cudaMemsetAsync(d_text + n, 0, kTextPad, stream));
  // Everything that must start at zero: the small area (segment table,
  // counters, queue counts, error flags).
  NA_CUDA(cudaMemsetAsync(small, 0, kSmallBytes, stream));
  const u64 seg_host[2] = {0, n};
  NA_CUDA(cudaMemcpyAsync(seg_begin, seg_host, sizeof(seg_host), cudaMemcpyHostToDevice, stream));
  NA_CUDA(cudaStreamSynchronize(stream));  // seg_host lives on this stack frame

  const Segments segs{seg_begin, 1};
  lcp_rows_kernel<<<static_cast<unsigned>(blocks_for((n + kLcpChunk / 32 - 1) / (kLcpChunk / 32))),
                    kLcpRowsBlock, 0,
                    stream>>>(
      d_text, sa, n, segs, 0, lcp, longs, kMax, scalars + 0, pending, kMax, scalars + 1, flags);
  NA_CUDA(cudaGetLastError());
  u64 counts[2] = {0, 0};
  NA_CUDA(cudaMemcpyAsync(counts, scalars, sizeof(counts), cudaMemcpyDeviceToHost, stream));
  NA_CUDA(cudaStreamSynchronize(stream));
  const u64 q = counts[0], pend = counts[1];
  if (q > kMax || pend > kMax) return SUFGPU_BUILD_FAILURE;

  const u64* sorted_pos = keys;
  const u32* sorted_val = vals;
  if (q > 0) {
    long_rows_kernel<<<148 * 8, 256, 0, stream>>>(d_text, longs, scalars + 0, kMax, segs, lcp,
                                                   keys, vals);
    NA_CUDA(cudaGetLastError());
    // Sort the long rows by position: one segment [0, q).
    const u32 tiles = static_cast<u32>((q + kSortTile - 1) / kSortTile);
    const u64 sb[2] = {0, q};
    const u32 st[2] = {0, tiles};
    NA_CUDA(cudaMemcpyAsync(sort_begin, sb, sizeof(sb), cudaMemcpyHostToDevice, stream));
    NA_CUDA(cudaMemcpyAsync(sort_tiles, st, sizeof(st), cudaMemcpyHostToDevice, stream));
    NA_CUDA(cudaStreamSynchronize(stream));
    const SortSegments ss{sort_begin, sort_tiles, 1, tiles};
    const u32 bits = bits_for(n);
    const u32 passes = (bits + kRadixBits - 1) / kRadixBits;
    NA_CUDA(cudaMemsetAsync(hist, 0, u64(passes) * kRadixDigits * 4, stream));
    radix_histogram_kernel<<<tiles, kSortBlock, 0, stream>>>(keys, ss, 0, passes, hist);
    NA_CUDA(cudaGetLastError());
    radix_offsets_kernel<<<1, kRadixDigits, 0, stream>>>(hist, sort_begin, passes, digits,
                                                          counters + 32);
    NA_CUDA(cudaGetLastError());
    u64* kin = keys;
    u32* vin = vals;
    u64* kout = keys_alt;
    u32* vout = vals_alt;
    for (u32 p = 0; p < passes; ++p) {
      NA_CUDA(cudaMemsetAsync(status, 0, u64(tiles) * kRadixDigits * 8, stream));
      NA_CUDA(cudaMemsetAsync(counters, 0, 4, stream));
      radix_onesweep_kernel<true, kSortBlock, kSortItems>
          <<<tiles, kSortBlock, sizeof(OnesweepSmem<kSortBlock, kSortTile, true>), stream>>>(
          kin, vin, kout, vout, ss, p * kRadixBits, p, passes, digits, status, counters, flags);
      NA_CUDA(cudaGetLastError());
      u64* tk = kin; kin = kout; kout = tk;
      u32* tv = vin; vin = vout; vout = tv;
    }
    sorted_pos = kin;
    sorted_val = vin;
  }
  if (pend > 0) {
    if (q == 0) return SUFGPU_BUILD_FAILURE;
    pending_rows_kernel<<<static_cast<unsigned>(blocks_for(pend)), 256, 0, stream>>>(
        sa, pending, scalars + 1, kMax, sorted_pos, sorted_val, scalars + 0, kMax, lcp, flags);
    NA_CUDA(cudaGetLastError());
  }
  DeviceFlags host_flags{};
  NA_CUDA(cudaMemcpyAsync(&host_flags, flags, sizeof(host_flags), cudaMemcpyDeviceToHost, stream));
  NA_CUDA(cudaStreamSynchronize(stream));
  return host_flags.error ? SUFGPU_BUILD_FAILURE : SUFGPU_OK;
}
