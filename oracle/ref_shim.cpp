// Test infrastructure only (see oracle/Makefile).  A flat C interface over the
// reference's own construction code so that Python tests and the CPU-baseline
// leg of bench.py can call it through ctypes.  Every function forwards to the
// reference function it names; nothing here re-implements the algorithm.
//
// Reference entry points wrapped (paths inside the sufkit project):
//   divsufsort / divsufsort64      third_party/libdivsufsort/lib/divsufsort.c:331-358
//   detail::BuildDivsufsort32/64   src/divsufsort_backend.cpp:24-171
//   CoordinateStorage::From*       src/coordinate_storage.cpp:439-602
//   LcpStorage::BuildByteCoded*    src/lcp_storage.cpp:217-420, 532-563
//   GenomeReference::FromFasta     src/genome_reference.cpp:222-268
//   SuffixArray::Build / Save      src/suffix_array.cpp:4086-4390, 4853-4916
//   detail::BuildCaps32/64         src/caps_backend.cpp (CaPS-SA, third_party/caps-sa)

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <filesystem>
#include <limits>
#include <memory>
#include <string>
#include <variant>
#include <vector>

// GenomeReference keeps its encoded bytes behind a private pointer; the oracle
// needs them to pin our FASTA encoder, so open the class for this one file.
#define private public
#include <sufkit/genome_reference.hpp>
#undef private

#include <sufkit/sufkit.hpp>

#include "caps_backend.hpp"
#include "coordinate_storage.hpp"
#include "divsufsort_backend.hpp"
#include "fast_prefix_index.hpp"
#include "genome_reference_internal.hpp"
#include "lcp_storage.hpp"

extern "C" {
#include "divsufsort.h"
#include "divsufsort64.h"
}

namespace {

thread_local std::string g_last_error;

int Fail(const std::exception& error) {
  g_last_error = error.what();
  if (const auto* sufkit_error = dynamic_cast<const sufkit::Error*>(&error)) {
    return 1 + static_cast<int>(sufkit_error->Code());
  }
  return 100;
}

using sufkit::CoordinateStorageWidth;
using sufkit::ErrorCode;
using sufkit::detail::CoordinateStorage;
using sufkit::detail::IntegerArrayView;
using sufkit::detail::LcpStorage;

CoordinateStorageWidth WidthFromBits(int bits) {
  switch (bits) {
    case 0:
      return CoordinateStorageWidth::kAutoSelect;
    case 32:
      return CoordinateStorageWidth::kBits32;
    case 40:
      return CoordinateStorageWidth::kBits40;
    case 48:
      return CoordinateStorageWidth::kBits48;
    case 64:
      return CoordinateStorageWidth::kBits64;
  }
  throw sufkit::Error(ErrorCode::kInvalidInput, "bad storage width");
}

// Copies a packed CoordinateStorage into caller planes.
void ExportCoordinates(const CoordinateStorage& storage, uint32_t* low32,
                       void* high, uint64_t* native64, int* width_out) {
  *width_out = static_cast<int>(storage.Width());
  storage.Visit([&](const auto& values) {
    using Values = std::decay_t<decltype(values)>;
    if constexpr (std::is_same_v<Values, std::vector<std::uint32_t>>) {
      std::copy(values.begin(), values.end(), low32);
    } else if constexpr (std::is_same_v<Values, std::vector<std::uint64_t>>) {
      std::copy(values.begin(), values.end(), native64);
    } else if constexpr (std::is_same_v<Values,
                                        sufkit::detail::Coordinate40Storage>) {
      std::copy(values.low.begin(), values.low.end(), low32);
      std::copy(values.high.begin(), values.high.end(),
                static_cast<uint8_t*>(high));
    } else {
      std::copy(values.low.begin(), values.low.end(), low32);
      std::copy(values.high.begin(), values.high.end(),
                static_cast<uint16_t*>(high));
    }
  });
}

template <class Coordinate>
void ExportAnchors(const std::vector<Coordinate>* positions,
                   const std::vector<Coordinate>* values, uint64_t* pos_out,
                   uint64_t* val_out, uint64_t cap, uint64_t* count) {
  *count = positions->size();
  if (positions->size() > cap) {
    throw sufkit::Error(ErrorCode::kInvalidInput, "anchor capacity too small");
  }
  for (std::size_t i = 0; i < positions->size(); ++i) {
    pos_out[i] = (*positions)[i];
    val_out[i] = (*values)[i];
  }
}

void ExportByteCoded(const LcpStorage& storage, uint8_t* primary,
                     uint64_t* anchor_pos, uint64_t* anchor_val,
                     uint64_t anchor_cap, uint64_t* anchor_count) {
  const auto* bytes = storage.BytePrimary();
  if (bytes == nullptr) {
    *anchor_count = 0;
    return;
  }
  std::copy(bytes->begin(), bytes->end(), primary);
  if (storage.AnchorPositions32() != nullptr) {
    ExportAnchors(storage.AnchorPositions32(), storage.AnchorValues32(),
                  anchor_pos, anchor_val, anchor_cap, anchor_count);
  } else {
    ExportAnchors(storage.AnchorPositions64(), storage.AnchorValues64(),
                  anchor_pos, anchor_val, anchor_cap, anchor_count);
  }
}

}  // namespace

extern "C" {

const char* sufref_last_error(void) { return g_last_error.c_str(); }

int sufref_divsufsort32(const uint8_t* text, int32_t* sa, int32_t n) {
  return divsufsort(text, sa, n);
}

int sufref_divsufsort64(const uint8_t* text, int64_t* sa, int64_t n) {
  return divsufsort64(text, sa, n);
}

// detail::BuildDivsufsort32/64 with sampling rate 1, exactly as
// SuffixArray::Build calls it.  sa_out/isa_out/lcp_out receive n values each
// (isa_out/lcp_out only when retained).  seconds[0..2] = sa/isa/lcp seconds.
int sufref_adapter_build(int width, const uint8_t* text, uint64_t n,
                         int retain_lcp, int retain_isa, uint32_t threads,
                         uint64_t* sa_out, uint64_t* isa_out,
                         uint64_t* lcp_out, double* seconds) {
  try {
    std::vector<std::uint8_t> input(text, text + n);
    auto run = [&](auto built) {
      for (std::size_t i = 0; i < built.suffix_array.size(); ++i) {
        sa_out[i] = static_cast<uint64_t>(built.suffix_array[i]);
      }
      if (isa_out != nullptr && !built.isa.empty()) {
        std::copy(built.isa.begin(), built.isa.end(), isa_out);
      }
      if (lcp_out != nullptr && !built.lcp.empty()) {
        std::copy(built.lcp.begin(), built.lcp.end(), lcp_out);
      }
      if (seconds != nullptr) {
        seconds[0] = built.sa_seconds;
        seconds[1] = built.isa_seconds;
        seconds[2] = built.lcp_seconds;
      }
    };
    if (width == 32) {
      run(sufkit::detail::BuildDivsufsort32(input, 1, retain_lcp != 0,
                                            retain_isa != 0, threads));
    } else {
      run(sufkit::detail::BuildDivsufsort64(input, 1, retain_lcp != 0,
                                            retain_isa != 0, threads));
    }
    return 0;
  } catch (const std::exception& error) {
    return Fail(error);
  }
}

// detail::BuildDivsufsort32/64 with sampling rate K: *rows_out receives the
// number of sampled rows written to sa_out/isa_out/lcp_out (ceil(n / K)).
int sufref_adapter_build_sampled(int width, const uint8_t* text, uint64_t n, uint32_t rate,
                                 int retain_lcp, int retain_isa, uint32_t threads,
                                 uint64_t* sa_out, uint64_t* isa_out, uint64_t* lcp_out,
                                 uint64_t* rows_out) {
  try {
    std::vector<std::uint8_t> input(text, text + n);
    auto run = [&](auto built) {
      *rows_out = built.suffix_array.size();
      for (std::size_t i = 0; i < built.suffix_array.size(); ++i) {
        sa_out[i] = static_cast<uint64_t>(built.suffix_array[i]);
      }
      if (isa_out != nullptr && !built.isa.empty()) {
        std::copy(built.isa.begin(), built.isa.end(), isa_out);
      }
      if (lcp_out != nullptr && !built.lcp.empty()) {
        std::copy(built.lcp.begin(), built.lcp.end(), lcp_out);
      }
    };
    if (width == 32) {
      run(sufkit::detail::BuildDivsufsort32(input, rate, retain_lcp != 0, retain_isa != 0,
                                            threads));
    } else {
      run(sufkit::detail::BuildDivsufsort64(input, rate, retain_lcp != 0, retain_isa != 0,
                                            threads));
    }
    return 0;
  } catch (const std::exception& error) {
    return Fail(error);
  }
}

// FastPrefixIndex::Build (default options) over the reference's own
// divsufsort64 SA/ISA of a logical text (contigs split at separators, one
// final sentinel).  *k_out receives the selected k (0 = no directory) and
// intervals_out (4^k entries) begin | end << 32 per k-mer from Lookup, with
// (n, n) for k-mers that do not occur.
int sufref_prefix_directory(const uint8_t* text, uint64_t n, uint64_t resident_core_bytes,
                            uint32_t* k_out, uint64_t* intervals_out, uint64_t* kmers_out,
                            uint64_t* entries_out) {
  try {
    std::vector<std::uint8_t> input(text, text + n);
    std::vector<int64_t> sa(n);
    if (divsufsort64(text, reinterpret_cast<saidx64_t*>(sa.data()), static_cast<saidx64_t>(n)) != 0) {
      throw std::runtime_error("divsufsort64 failed");
    }
    std::vector<std::uint64_t> sa64(n), isa64(n);
    for (uint64_t r = 0; r < n; ++r) {
      sa64[r] = static_cast<std::uint64_t>(sa[r]);
      isa64[sa64[r]] = r;
    }
    auto sa_s = CoordinateStorage::FromUInt64(std::move(sa64), WidthFromBits(64), n,
                                              ErrorCode::kBuildFailure, "suffix array");
    auto isa_s = CoordinateStorage::FromUInt64(std::move(isa64), WidthFromBits(64), n,
                                               ErrorCode::kBuildFailure, "inverse suffix array");
    std::vector<sufkit::Position> starts, lengths;
    sufkit::Position start = 0;
    for (uint64_t i = 0; i + 1 < n; ++i) {
      if (text[i] == 1) {
        starts.push_back(start);
        lengths.push_back(i - start);
        start = i + 1;
      }
    }
    auto index = sufkit::detail::FastPrefixIndex::Build(input, sa_s, isa_s, starts, lengths,
                                                resident_core_bytes);
    *k_out = index.K();
    *kmers_out = index.IndexedKmers();
    *entries_out = index.NonemptyEntries();
    const uint32_t k = index.K();
    if (k == 0) return 0;
    std::vector<std::uint8_t> pattern(k);
    for (uint64_t key = 0; key < (uint64_t{1} << (2 * k)); ++key) {
      for (uint32_t j = 0; j < k; ++j) {
        pattern[j] = static_cast<std::uint8_t>(2 + ((key >> (2 * (k - 1 - j))) & 3));
      }
      const auto interval = index.Lookup(pattern);
      if (!interval || interval->Empty()) {
        intervals_out[key] = n | (n << 32);
      } else {
        intervals_out[key] = interval->begin | (interval->end << 32);
      }
    }
    return 0;
  } catch (const std::exception& error) {
    return Fail(error);
  }
}

// CoordinateStorage::FromUInt64 (the validating packer used by
// RepackSuffixArray and BuildIsa).  Writes the planes of the resolved width;
// *width_out receives that width in bits.
int sufref_pack(const uint64_t* values, uint64_t count, uint64_t symbol_count,
                int storage_bits, uint32_t* low32, void* high,
                uint64_t* native64, int* width_out) {
  try {
    std::vector<std::uint64_t> input(values, values + count);
    auto storage = CoordinateStorage::FromUInt64(
        std::move(input), WidthFromBits(storage_bits), symbol_count,
        ErrorCode::kBuildFailure, "suffix array");
    ExportCoordinates(storage, low32, high, native64, width_out);
    return 0;
  } catch (const std::exception& error) {
    return Fail(error);
  }
}

// detail::BuildCaps32/64: the CaPS-SA parallel constructor sufkit vendors,
// SA (and its construction LCP when lcp_out is not null) as uint64 rows;
// seconds[0] = wall time of the call.
int sufref_caps_build(int width, const uint8_t* text, uint64_t n, uint32_t threads,
                      uint64_t* sa_out, uint64_t* lcp_out, double* seconds) {
  try {
    std::vector<uint8_t> t(text, text + n);
    const auto begin = std::chrono::steady_clock::now();
    auto copy = [&](const auto& built) {
      if (seconds) {
        seconds[0] = std::chrono::duration<double>(std::chrono::steady_clock::now() - begin)
                         .count();
      }
      for (uint64_t i = 0; i < built.suffix_array.size(); ++i) sa_out[i] = built.suffix_array[i];
      if (lcp_out) {
        for (uint64_t i = 0; i < built.lcp.size(); ++i) lcp_out[i] = built.lcp[i];
      }
    };
    if (width == 32) copy(sufkit::detail::BuildCaps32(t, threads, lcp_out != nullptr));
    else copy(sufkit::detail::BuildCaps64(t, threads, lcp_out != nullptr));
    return 0;
  } catch (const std::exception& error) {
    return Fail(error);
  }
}

// LcpStorage::BuildByteCodedDirect: generalized Kasai written straight into
// the byte-coded layout (src/lcp_storage.cpp:304-420).
int sufref_bytecoded_direct(const uint8_t* text, uint64_t n,
                            const uint64_t* sa, const uint64_t* isa,
                            int coordinate_width, uint8_t* primary,
                            uint64_t* anchor_pos, uint64_t* anchor_val,
                            uint64_t anchor_cap, uint64_t* anchor_count) {
  try {
    auto storage = LcpStorage::BuildByteCodedDirect(
        text, n, IntegerArrayView(sa, n), IntegerArrayView(isa, n), 1,
        static_cast<std::uint8_t>(coordinate_width), ErrorCode::kBuildFailure);
    storage.Validate(IntegerArrayView(sa, n), n, ErrorCode::kCorruptIndex);
    ExportByteCoded(storage, primary, anchor_pos, anchor_val, anchor_cap,
                    anchor_count);
    return 0;
  } catch (const std::exception& error) {
    return Fail(error);
  }
}

// The same for a sampled suffix array (rate K > 1): rows = ceil(n / K)
// sampled SA rows and the dense sampled ISA (src/lcp_storage.cpp:304-420).
int sufref_bytecoded_direct_sampled(const uint8_t* text, uint64_t n, const uint64_t* sa,
                                    const uint64_t* isa, uint64_t rows, uint32_t rate,
                                    int coordinate_width, uint8_t* primary,
                                    uint64_t* anchor_pos, uint64_t* anchor_val,
                                    uint64_t anchor_cap, uint64_t* anchor_count) {
  try {
    auto storage = LcpStorage::BuildByteCodedDirect(
        text, n, IntegerArrayView(sa, rows), IntegerArrayView(isa, rows), rate,
        static_cast<std::uint8_t>(coordinate_width), ErrorCode::kBuildFailure);
    ExportByteCoded(storage, primary, anchor_pos, anchor_val, anchor_cap,
                    anchor_count);
    return 0;
  } catch (const std::exception& error) {
    return Fail(error);
  }
}

// LcpStorage::BuildByteCoded from a raw row-order LCP and the ISA.
int sufref_bytecoded_from_raw(const uint64_t* lcp, const uint64_t* isa,
                              uint64_t n, int coordinate_width,
                              uint8_t* primary, uint64_t* anchor_pos,
                              uint64_t* anchor_val, uint64_t anchor_cap,
                              uint64_t* anchor_count) {
  try {
    auto storage = LcpStorage::BuildByteCoded(
        IntegerArrayView(lcp, n), IntegerArrayView(isa, n), 1,
        static_cast<std::uint8_t>(coordinate_width), n,
        ErrorCode::kBuildFailure);
    ExportByteCoded(storage, primary, anchor_pos, anchor_val, anchor_cap,
                    anchor_count);
    return 0;
  } catch (const std::exception& error) {
    return Fail(error);
  }
}

// Decodes one byte-coded LCP row through LcpStorage::Exact (queries use this).
int sufref_bytecoded_exact(const uint8_t* primary, uint64_t n,
                           const uint64_t* anchor_pos,
                           const uint64_t* anchor_val, uint64_t anchors,
                           const uint64_t* rows, const uint64_t* suffixes,
                           uint64_t queries, uint64_t* out) {
  try {
    std::vector<std::uint8_t> p(primary, primary + n);
    std::vector<std::uint64_t> ap(anchor_pos, anchor_pos + anchors);
    std::vector<std::uint64_t> av(anchor_val, anchor_val + anchors);
    auto storage = LcpStorage::FromByteCoded64(
        std::move(p), std::move(ap), std::move(av), 1, n,
        ErrorCode::kCorruptIndex);
    for (uint64_t q = 0; q < queries; ++q) {
      out[q] = storage.Exact(rows[q], suffixes[q]);
    }
    return 0;
  } catch (const std::exception& error) {
    return Fail(error);
  }
}

// GenomeReference::FromFasta; copies the normalized bytes (contig separators
// included, no sentinel).  Returns the byte count, or -1 on error (message in
// sufref_last_error), or -2 when cap is too small (required size in *needed).
int64_t sufref_encode_fasta(const char* path, uint8_t* out, uint64_t cap,
                            uint64_t* needed, uint64_t* fingerprint) {
  try {
    auto reference = sufkit::GenomeReference::FromFasta(path);
    const auto& encoded = reference.impl_->data.encoded;
    *needed = encoded.size();
    if (fingerprint != nullptr) {
      *fingerprint = reference.Fingerprint();
    }
    if (encoded.size() > cap) {
      return -2;
    }
    std::copy(encoded.begin(), encoded.end(), out);
    return static_cast<int64_t>(encoded.size());
  } catch (const std::exception& error) {
    Fail(error);
    return -1;
  }
}

// SuffixArray::Build through the public API with the divsufsort backend.
//   profile 0 = FastSuffixArrayBuildOptions, 1 = LowMemorySuffixArrayBuildOptions
//   coordinate_width 32/64, storage_width 0/32/40/48/64, acceleration per
//   sufkit::SaAcceleration (ignored by Low-memory), threads >= 1.
// stats[0..11] = sa, storage_compaction, isa, lcp, child, learned,
// caps_construct, caps_output_allocation, text_prepare, lcp_finalize,
// prefix_directory, total seconds.  info[0..5] = text_symbols,
// stored_coordinate_width, lcp_encoding, lcp_overflow_anchors, sa_bytes,
// lcp_bytes.  When save_path is not null the index is saved there.
int sufref_suffix_array_build(const char* fasta_path, int profile,
                              int coordinate_width, int storage_width,
                              int acceleration, uint32_t threads,
                              const char* save_path, double* stats,
                              uint64_t* info) {
  try {
    auto reference = sufkit::GenomeReference::FromFasta(fasta_path);
    auto options = profile == 0 ? sufkit::FastSuffixArrayBuildOptions()
                                : sufkit::LowMemorySuffixArrayBuildOptions();
    options.backend = sufkit::SaBackend::kDivsufsort;
    options.coordinate_width = coordinate_width == 32
                                   ? sufkit::CoordinateWidth::kBits32
                                   : sufkit::CoordinateWidth::kBits64;
    options.storage_width = WidthFromBits(storage_width);
    if (acceleration >= 0) {
      options.acceleration = static_cast<sufkit::SaAcceleration>(acceleration);
    }
    options.threads = threads;
    sufkit::SuffixArrayBuildStatistics statistics;
    options.statistics = &statistics;
    auto index = sufkit::SuffixArray::Build(reference, options);
    if (stats != nullptr) {
      const double values[12] = {statistics.sa_seconds,
                                 statistics.storage_compaction_seconds,
                                 statistics.isa_seconds,
                                 statistics.lcp_seconds,
                                 statistics.child_seconds,
                                 statistics.learned_index_seconds,
                                 statistics.caps_construct_seconds,
                                 statistics.caps_output_allocation_seconds,
                                 statistics.text_prepare_seconds,
                                 statistics.lcp_finalize_seconds,
                                 statistics.prefix_directory_seconds,
                                 statistics.total_seconds};
      std::copy(values, values + 12, stats);
    }
    const auto index_info = index.GetInfo();
    if (info != nullptr) {
      info[0] = index_info.text_symbols;
      info[1] = index_info.stored_coordinate_width;
      info[2] = static_cast<uint64_t>(index_info.lcp_encoding);
      info[3] = index_info.lcp_overflow_anchors;
      info[4] = index_info.sa_bytes;
      info[5] = index_info.lcp_bytes;
    }
    if (save_path != nullptr) {
      index.Save(save_path);
    }
    return 0;
  } catch (const std::exception& error) {
    return Fail(error);
  }
}

// SuffixAt(row) for rows [0, count) of an index built as above; lets tests
// compare the public build's rows with ours.
int sufref_suffix_array_rows(const char* fasta_path, int profile,
                             int coordinate_width, int storage_width,
                             uint64_t* rows_out, uint64_t count) {
  try {
    auto reference = sufkit::GenomeReference::FromFasta(fasta_path);
    auto options = profile == 0 ? sufkit::FastSuffixArrayBuildOptions()
                                : sufkit::LowMemorySuffixArrayBuildOptions();
    options.backend = sufkit::SaBackend::kDivsufsort;
    options.coordinate_width = coordinate_width == 32
                                   ? sufkit::CoordinateWidth::kBits32
                                   : sufkit::CoordinateWidth::kBits64;
    options.storage_width = WidthFromBits(storage_width);
    auto index = sufkit::SuffixArray::Build(reference, options);
    const auto symbols = index.GetInfo().text_symbols;
    for (uint64_t row = 0; row < count && row < symbols; ++row) {
      rows_out[row] = index.SuffixAt(row);
    }
    return 0;
  } catch (const std::exception& error) {
    return Fail(error);
  }
}

// SuffixArray::Load of a saved .sufidx (src/suffix_array.cpp, which fully
// validates containers, CRCs and semantics), then Count(pattern) and
// SuffixAt(row) for rows [0, count).  info[0..2] = text_symbols,
// stored_coordinate_width, lcp_encoding of the loaded index.
int sufref_load_query(const char* path, const char* pattern, uint64_t* occurrences,
                      uint64_t* rows_out, uint64_t count, uint64_t* info) {
  try {
    auto index = sufkit::SuffixArray::Load(path);
    const auto index_info = index.GetInfo();
    if (info != nullptr) {
      info[0] = index_info.text_symbols;
      info[1] = index_info.stored_coordinate_width;
      info[2] = static_cast<uint64_t>(index_info.lcp_encoding);
    }
    if (occurrences != nullptr && pattern != nullptr) *occurrences = index.Count(pattern);
    for (uint64_t row = 0; row < count && row < index_info.text_symbols; ++row) {
      rows_out[row] = index.SuffixAt(row);
    }
    return 0;
  } catch (const std::exception& error) {
    return Fail(error);
  }
}

}  // extern "C"
