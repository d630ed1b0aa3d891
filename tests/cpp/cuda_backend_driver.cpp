// Test driver for the C++ adapter (include/sufgpu/cuda_backend.hpp): reads a
// logical text, runs BuildCuda32/64 and BuildCudaStorage, and writes the rows
// as little-endian uint64 files for tests/test_cpp_adapter.py to compare with
// the reference.  Error paths are exercised too (exit code 0 on success).
#include <cstdio>
#include <fstream>
#include <iostream>
#include <iterator>
#include <string>
#include <vector>

#include "../../include/sufgpu/cuda_backend.hpp"

template <class V>
void dump(const std::string& path, const V& values) {
  std::ofstream out(path, std::ios::binary);
  for (auto v : values) {
    const std::uint64_t x = static_cast<std::uint64_t>(v);
    out.write(reinterpret_cast<const char*>(&x), 8);
  }
}

int main(int argc, char** argv) {
  if (argc != 3) {
    std::cerr << "usage: driver <text.bin> <out-prefix>\n";
    return 2;
  }
  std::ifstream in(argv[1], std::ios::binary);
  std::vector<std::uint8_t> text((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
  const std::string prefix = argv[2];
  auto r64 = sufgpu::BuildCuda64(text, 1, true, true, 4);
  dump(prefix + ".sa64", r64.suffix_array);
  dump(prefix + ".isa64", r64.isa);
  dump(prefix + ".lcp64", r64.lcp);
  auto r32 = sufgpu::BuildCuda32(text, 1, true, false, 1);
  dump(prefix + ".sa32", r32.suffix_array);
  dump(prefix + ".lcp32", r32.lcp);
  if (!r32.isa.empty()) return 3;
  auto lowmem = sufgpu::BuildCudaStorage(text, 40, 0, SUFGPU_LCP_BYTE32);
  dump(prefix + ".sa40low", lowmem.sa_low32);
  dump(prefix + ".sa40high", lowmem.sa_high8);
  dump(prefix + ".primary", lowmem.lcp_primary);
  dump(prefix + ".anchor_pos", lowmem.anchor_positions);
  dump(prefix + ".anchor_val", lowmem.anchor_values);
  // Sampling rate 4: the suffixes at multiples of 4 (ISA and LCP retained).
  auto sampled = sufgpu::BuildCuda64(text, 4, true, true, 1);
  dump(prefix + ".sa_k4", sampled.suffix_array);
  dump(prefix + ".isa_k4", sampled.isa);
  dump(prefix + ".lcp_k4", sampled.lcp);
  // Error categories match sufkit::ErrorCode.
  int checks = 0;
  try {
    sufgpu::BuildCuda32(text, 0, true, false, 1);
  } catch (const sufgpu::Error& e) {
    checks += e.Code() == sufgpu::ErrorCode::kInvalidInput;
  }
  try {
    sufgpu::BuildCuda64(text, 1, true, false, 0);
  } catch (const sufgpu::Error& e) {
    checks += e.Code() == sufgpu::ErrorCode::kInvalidInput;
  }
  if (checks != 2) return 4;
  std::printf("ok %zu\n", text.size());
  return 0;
}
