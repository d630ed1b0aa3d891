// Drop-in construction backend for sufkit, at the link level.
//
// sufkit's SuffixArray::Build (src/suffix_array.cpp:4211-4232 in sufkit) gets
// its suffix array, ISA and Kasai LCP from two functions declared in
// src/divsufsort_backend.hpp:28-34:
//
//   DivSufsortBuildResult<int32_t> BuildDivsufsort32(text, sampling_rate,
//                                                    retain_lcp, retain_isa, threads);
//   DivSufsortBuildResult<int64_t> BuildDivsufsort64(...);
//
// This file defines both on top of the sufgpu C ABI (include/sufgpu/sufgpu.h).
// Linked into libsufkit in place of src/divsufsort_backend.cpp, every caller
// of those functions -- Build's Fast and Low-memory profiles, storage
// repacking, ISA and LCP finalisation, Save and the .sufidx 1.4 writer --
// runs unchanged on a suffix array built by the GPU.  The results equal
// divsufsort's word for word, so the saved index is byte-identical to a
// divsufsort build's and carries the same provenance.
//
// Semantics follow the replaced functions:
//   * text is the logical text with its sentinel; sampling_rate K >= 1 keeps
//     the rows of positions that are multiples of K;
//   * isa[p / K] = row when retain_isa; lcp[row] (row order) when retain_lcp,
//     the LCP of consecutive kept rows; otherwise both vectors are empty;
//   * threads only has to be non-zero (the device does the work);
//   * errors become sufkit::Error with the matching ErrorCode (the sufgpu
//     status is ErrorCode + 1): size limits kInvalidInput, CUDA failures
//     kBuildFailure.
// The 64-bit SA is written straight into the DivSufsort64Buffer that sufkit
// later hands to CoordinateStorage::FromDivSufsort64, with no host copy.
//
// Compile against sufkit's headers: -I<sufkit>/include -I<sufkit>/src, plus
// this repository's include/, and link libsufgpu.so.

#include <chrono>
#include <cstdint>
#include <limits>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include <sufkit/types.hpp>

#include "divsufsort_backend.hpp"
#include "sufgpu/sufgpu.h"

namespace sufkit::detail {
namespace {

// One device context per process, created on first use; builds on it are
// serialised, as the replaced constructor runs synchronously on the caller.
std::mutex g_mutex;
sufgpu_ctx* g_ctx = nullptr;

[[noreturn]] void Raise(sufgpu_status status, const std::string& message) {
  const auto code = status == SUFGPU_OK
                        ? ErrorCode::kBuildFailure
                        : static_cast<ErrorCode>(static_cast<int>(status) - 1);
  throw Error(code, message);
}

sufgpu_ctx* ContextLocked() {
  if (g_ctx == nullptr) {
    const sufgpu_status status = sufgpu_create(&g_ctx, 0);
    if (status != SUFGPU_OK) {
      g_ctx = nullptr;
      Raise(status, std::string("CUDA constructor unavailable: ") + sufgpu_last_error(nullptr));
    }
  }
  return g_ctx;
}

template <class Index>
DivSufsortBuildResult<Index> BuildOnDevice(const std::vector<std::uint8_t>& text,
                                           std::uint32_t sampling_rate, bool retain_lcp,
                                           bool retain_isa, std::uint32_t threads) {
  const auto begin = std::chrono::steady_clock::now();
  if (threads == 0) throw Error(ErrorCode::kInvalidInput, "thread count must be greater than zero");
  if (sampling_rate == 0) throw Error(ErrorCode::kInvalidInput, "sampling rate must be at least 1");
  const std::uint64_t index_limit = static_cast<std::uint64_t>(std::numeric_limits<Index>::max());
  if (text.size() > index_limit) {
    throw Error(ErrorCode::kInvalidInput,
                std::is_same_v<Index, std::int32_t> ? "reference is too large for the 32-bit constructor"
                                                    : "reference is too large for the 64-bit constructor");
  }
  if (text.size() > sufgpu_max_symbols()) {
    throw Error(ErrorCode::kInvalidInput, "reference exceeds the device limit of 2^32-1 symbols");
  }
  DivSufsortBuildResult<Index> result;
  const std::uint64_t n = text.size();
  const std::uint64_t rows = (n + sampling_rate - 1) / sampling_rate;
  result.suffix_array.resize(rows);
  const bool isa_out = retain_isa || retain_lcp;
  if (isa_out) result.isa.resize(rows);
  if (retain_lcp) result.lcp.resize(rows);

  sufgpu_build_desc desc{};
  desc.sa_storage_bits = sizeof(Index) * 8;
  desc.isa_storage_bits = isa_out ? 64 : 0;
  desc.lcp_encoding = retain_lcp ? SUFGPU_LCP_RAW64 : SUFGPU_LCP_NONE;
  desc.flags = SUFGPU_FLAG_VALIDATE;
  desc.sampling_rate = sampling_rate;
  sufgpu_outputs out{};
  out.sa_low = result.suffix_array.data();
  out.isa_low = isa_out ? result.isa.data() : nullptr;
  out.lcp = retain_lcp ? result.lcp.data() : nullptr;
  sufgpu_build_stats stats{};
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    sufgpu_ctx* ctx = ContextLocked();
    const sufgpu_status status = sufgpu_build(ctx, text.data(), n, &desc, &out, nullptr, &stats);
    if (status != SUFGPU_OK) Raise(status, sufgpu_last_error(ctx));
  }
  // The replaced constructor reports SA time including its host work; here
  // the SA phase is everything up to the ISA and LCP phases the device timed.
  const double total =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - begin).count();
  result.isa_seconds = stats.isa_seconds;
  result.lcp_seconds = stats.lcp_seconds;
  result.sa_seconds = total - stats.isa_seconds - stats.lcp_seconds;
  if (!retain_isa) result.isa.clear();
  return result;
}

}  // namespace

DivSufsortBuildResult<std::int32_t> BuildDivsufsort32(const std::vector<std::uint8_t>& text,
                                                      std::uint32_t sampling_rate,
                                                      bool retain_lcp, bool retain_isa,
                                                      std::uint32_t threads) {
  return BuildOnDevice<std::int32_t>(text, sampling_rate, retain_lcp, retain_isa, threads);
}

DivSufsortBuildResult<std::int64_t> BuildDivsufsort64(const std::vector<std::uint8_t>& text,
                                                      std::uint32_t sampling_rate,
                                                      bool retain_lcp, bool retain_isa,
                                                      std::uint32_t threads) {
  return BuildOnDevice<std::int64_t>(text, sampling_rate, retain_lcp, retain_isa, threads);
}

}  // namespace sufkit::detail
