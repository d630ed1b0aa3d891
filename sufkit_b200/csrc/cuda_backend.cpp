// C++ adapter over the C ABI (include/sufgpu/cuda_backend.hpp).
#include "../../include/sufgpu/cuda_backend.hpp"

#include <limits>
#include <mutex>

namespace sufgpu {
namespace {

// One context per process for the adapter (builds on it are serialized,
// matching the reference's synchronous constructor call).
struct Shared {
  std::mutex mutex;
  sufgpu_ctx* ctx = nullptr;
  ~Shared() {
    if (ctx) sufgpu_destroy(ctx);
  }
};

Shared& shared() {
  static Shared s;
  return s;
}

[[noreturn]] void Throw(sufgpu_status status, const std::string& message) {
  const auto code = status == SUFGPU_OK ? ErrorCode::kBuildFailure
                                        : static_cast<ErrorCode>(static_cast<int>(status) - 1);
  throw Error(code, message);
}

sufgpu_ctx* context_locked() {
  Shared& s = shared();
  if (!s.ctx) {
    const auto status = sufgpu_create(&s.ctx, 0);
    if (status != SUFGPU_OK) {
      s.ctx = nullptr;
      Throw(status, std::string("cannot create the CUDA context: ") + sufgpu_last_error(nullptr));
    }
  }
  return s.ctx;
}

template <class Index>
CudaBuildResult<Index> BuildCuda(const std::vector<std::uint8_t>& text,
                                 std::uint32_t sampling_rate, bool retain_lcp,
                                 bool retain_isa, std::uint32_t threads) {
  // Same argument checks as BuildDivsufsort (src/divsufsort_backend.cpp:29-42).
  if (threads == 0) throw Error(ErrorCode::kInvalidInput, "thread count must be greater than zero");
  if (sampling_rate == 0) throw Error(ErrorCode::kInvalidInput, "sampling rate must be at least 1");
  const std::uint64_t limit = std::is_same_v<Index, std::int32_t>
                                  ? std::uint64_t(std::numeric_limits<std::int32_t>::max())
                                  : std::uint64_t(std::numeric_limits<std::int64_t>::max());
  if (text.size() > limit) {
    throw Error(ErrorCode::kInvalidInput, std::is_same_v<Index, std::int32_t>
                                              ? "reference is too large for the 32-bit constructor"
                                              : "reference is too large for the 64-bit constructor");
  }
  if (text.size() > sufgpu_max_symbols()) {
    throw Error(ErrorCode::kInvalidInput, "reference exceeds the device build limit of 2^32-1 symbols");
  }
  CudaBuildResult<Index> result;
  const std::uint64_t n = text.size();
  // Sampled rows: the suffixes at multiples of the rate (divsufsort_backend.cpp:62-73).
  const std::uint64_t rows = (n + sampling_rate - 1) / sampling_rate;
  result.suffix_array.resize(rows);
  if (retain_isa || retain_lcp) result.isa.resize(rows);
  if (retain_lcp) result.lcp.resize(rows);
  sufgpu_build_desc desc{};
  desc.sa_storage_bits = sizeof(Index) * 8;
  desc.isa_storage_bits = (retain_isa || retain_lcp) ? 64 : 0;
  desc.lcp_encoding = retain_lcp ? SUFGPU_LCP_RAW64 : SUFGPU_LCP_NONE;
  desc.flags = SUFGPU_FLAG_VALIDATE;
  desc.sampling_rate = sampling_rate;
  sufgpu_outputs out{};
  out.sa_low = result.suffix_array.data();
  out.isa_low = result.isa.empty() ? nullptr : result.isa.data();
  out.lcp = result.lcp.empty() ? nullptr : result.lcp.data();
  sufgpu_build_stats stats{};
  std::lock_guard<std::mutex> lock(shared().mutex);
  sufgpu_ctx* ctx = context_locked();
  const auto status = sufgpu_build(ctx, text.data(), n, &desc, &out, nullptr, &stats);
  if (status != SUFGPU_OK) Throw(status, sufgpu_last_error(ctx));
  result.sa_seconds = stats.sa_seconds;
  result.isa_seconds = stats.isa_seconds;
  result.lcp_seconds = stats.lcp_seconds;
  if (!retain_isa) result.isa.clear();
  return result;
}

}  // namespace

CudaBuildResult<std::int32_t> BuildCuda32(const std::vector<std::uint8_t>& text,
                                          std::uint32_t sampling_rate, bool retain_lcp,
                                          bool retain_isa, std::uint32_t threads) {
  return BuildCuda<std::int32_t>(text, sampling_rate, retain_lcp, retain_isa, threads);
}

CudaBuildResult<std::int64_t> BuildCuda64(const std::vector<std::uint8_t>& text,
                                          std::uint32_t sampling_rate, bool retain_lcp,
                                          bool retain_isa, std::uint32_t threads) {
  return BuildCuda<std::int64_t>(text, sampling_rate, retain_lcp, retain_isa, threads);
}

StoredBuild BuildCudaStorage(const std::vector<std::uint8_t>& text, std::uint32_t sa_bits,
                             std::uint32_t isa_bits, std::uint32_t lcp_encoding) {
  StoredBuild b;
  const std::uint64_t n = text.size();
  b.sa_bits = sa_bits;
  b.isa_bits = isa_bits;
  b.lcp_encoding = lcp_encoding;
  sufgpu_outputs out{};
  auto planes = [&](std::uint32_t bits, std::vector<std::uint32_t>& low32,
                    std::vector<std::uint64_t>& native, std::vector<std::uint8_t>& h8,
                    std::vector<std::uint16_t>& h16, void** low, void** high) {
    if (bits == 0) return;
    if (bits == 64) {
      native.resize(n);
      *low = native.data();
    } else {
      low32.resize(n);
      *low = low32.data();
    }
    if (bits == 40) {
      h8.resize(n);
      *high = h8.data();
    } else if (bits == 48) {
      h16.resize(n);
      *high = h16.data();
    }
  };
  planes(sa_bits, b.sa_low32, b.sa_native64, b.sa_high8, b.sa_high16, &out.sa_low, &out.sa_high);
  planes(isa_bits, b.isa_low32, b.isa_native64, b.isa_high8, b.isa_high16, &out.isa_low,
         &out.isa_high);
  if (lcp_encoding == SUFGPU_LCP_RAW32) {
    b.lcp_raw32.resize(n);
    out.lcp = b.lcp_raw32.data();
  } else if (lcp_encoding == SUFGPU_LCP_RAW64) {
    b.lcp_raw64.resize(n);
    out.lcp = b.lcp_raw64.data();
  } else if (lcp_encoding != SUFGPU_LCP_NONE) {
    b.lcp_primary.resize(n);
    out.lcp = b.lcp_primary.data();
  }
  sufgpu_build_desc desc{sa_bits, isa_bits, lcp_encoding, SUFGPU_FLAG_VALIDATE};
  sufgpu_anchors anchors{};
  std::lock_guard<std::mutex> lock(shared().mutex);
  sufgpu_ctx* ctx = context_locked();
  const auto status = sufgpu_build(ctx, text.data(), n, &desc, &out, &anchors, &b.stats);
  if (status != SUFGPU_OK) Throw(status, sufgpu_last_error(ctx));
  if (anchors.count) {
    b.anchor_positions.resize(anchors.count);
    b.anchor_values.resize(anchors.count);
    for (std::uint64_t i = 0; i < anchors.count; ++i) {
      if (anchors.coordinate_bits == 32) {
        b.anchor_positions[i] = static_cast<const std::uint32_t*>(anchors.positions)[i];
        b.anchor_values[i] = static_cast<const std::uint32_t*>(anchors.values)[i];
      } else {
        b.anchor_positions[i] = static_cast<const std::uint64_t*>(anchors.positions)[i];
        b.anchor_values[i] = static_cast<const std::uint64_t*>(anchors.values)[i];
      }
    }
  }
  return b;
}

}  // namespace sufgpu
