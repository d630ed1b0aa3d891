// C++ face of sufgpu for sufkit's constructor slot.
//
// BuildCuda32 / BuildCuda64 have the signature and result shape of
// sufkit::detail::BuildDivsufsort32 / BuildDivsufsort64
// (src/divsufsort_backend.hpp:13-33): the complete SA in Index, and, when
// retained, the ISA and the Kasai LCP as uint64 rows, plus per-phase seconds.
// Errors are thrown as sufgpu::Error whose ErrorCode values equal
// sufkit::ErrorCode (include/sufkit/types.hpp:708-721), so the sufkit-side
// wrapper rethrows them as sufkit::Error one to one.
//
// BuildCudaStorage goes one step further for the Low-memory profile: it
// returns the stored planes (split40/48 or native SA, byte-coded or raw LCP)
// directly, which is what RepackSuffixArray + BuildByteCodedLcpDirect
// (src/suffix_array.cpp:852-910, 1103-1115) would produce on the host.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "sufgpu.h"

namespace sufgpu {

enum class ErrorCode : std::uint8_t {
  kInvalidInput,
  kIoError,
  kUnsupportedBackend,
  kCorruptIndex,
  kVersionMismatch,
  kBuildFailure
};

class SUFGPU_API Error : public std::runtime_error {
 public:
  Error(ErrorCode code, const std::string& message)
      : std::runtime_error(message), code_(code) {}
  ErrorCode Code() const noexcept { return code_; }

 private:
  ErrorCode code_;
};

template <class Index>
struct CudaBuildResult {
  std::vector<Index> suffix_array;
  std::vector<std::uint64_t> isa;  // only if retain_isa
  std::vector<std::uint64_t> lcp;  // only if retain_lcp (row order)
  double sa_seconds = 0.0;
  double isa_seconds = 0.0;
  double lcp_seconds = 0.0;
};

SUFGPU_API CudaBuildResult<std::int32_t> BuildCuda32(const std::vector<std::uint8_t>& text,
                                                     std::uint32_t sampling_rate,
                                                     bool retain_lcp, bool retain_isa,
                                                     std::uint32_t threads);

SUFGPU_API CudaBuildResult<std::int64_t> BuildCuda64(const std::vector<std::uint8_t>& text,
                                                     std::uint32_t sampling_rate,
                                                     bool retain_lcp, bool retain_isa,
                                                     std::uint32_t threads);

// Stored planes for a profile: SA in storage_bits (32/40/48/64), optional ISA,
// LCP raw or byte-coded (anchors in 32 or 64 bits per the encoding).
struct StoredBuild {
  std::uint32_t sa_bits = 32;
  std::vector<std::uint32_t> sa_low32;
  std::vector<std::uint64_t> sa_native64;
  std::vector<std::uint8_t> sa_high8;
  std::vector<std::uint16_t> sa_high16;
  std::uint32_t isa_bits = 0;
  std::vector<std::uint32_t> isa_low32;
  std::vector<std::uint64_t> isa_native64;
  std::vector<std::uint8_t> isa_high8;
  std::vector<std::uint16_t> isa_high16;
  std::uint32_t lcp_encoding = SUFGPU_LCP_NONE;
  std::vector<std::uint32_t> lcp_raw32;
  std::vector<std::uint64_t> lcp_raw64;
  std::vector<std::uint8_t> lcp_primary;
  std::vector<std::uint64_t> anchor_positions;
  std::vector<std::uint64_t> anchor_values;
  sufgpu_build_stats stats{};
};

SUFGPU_API StoredBuild BuildCudaStorage(const std::vector<std::uint8_t>& text,
                                        std::uint32_t sa_bits, std::uint32_t isa_bits,
                                        std::uint32_t lcp_encoding);

}  // namespace sufgpu
