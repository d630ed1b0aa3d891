// FASTA normalisation and the reference fingerprint on the GPU.
//
// GenomeReference::FromFasta (src/genome_reference.cpp:131-156, 222-268, fed
// by kseq) turns FASTA into the logical text: every sequence byte through the
// encoding table (A/C/G/T in any case -> 2..5, anything else -> 6), a 1 after
// every record, and the FNV-1a 64 hash of those bytes as the fingerprint.
//
// Normalisation is one single-pass tile kernel over the raw bytes.  Each
// byte needs the start of its line (is it a header line?), which is the last
// newline before it: a max-scan with decoupled look-back; the kept bytes
// then get their output positions from a sum-scan, also with look-back.
// Records start at the first '>' of the input (bytes before it are skipped)
// and at every later line that starts with '>'; the 1 closing a record is
// written at the position of the next record's '>' (and after the last byte
// for the last record, by the host).  Newlines are dropped, and so is a '\r'
// that ends a line.  Inputs this path does not take are flagged, for the
// host reader to handle: FASTQ (lines starting with '@' or '+'), and a lone
// "\r" line right after a header, which kseq keeps as a base.
//
// FNV-1a (h = (h ^ b) * P mod 2^64) is sequential, so it is restated
// chunk-parallel:
//   * the low byte x of h evolves on its own, x' = ((x ^ b) * P) mod 256, and
//     bit j of x' depends only on bits 0..j of x and b (multiplication by the
//     odd P carries upward only).  With bits 0..j-1 of a chunk's start known,
//     bit j at its end is (simulated end bit with start bit j = 0) XOR (the
//     true start bit j), so 8 passes, each an exclusive XOR-scan over chunks,
//     give the low byte at every chunk start;
//   * with the start byte known, a chunk is an affine map of the full state:
//     h_end = h_start * P^L + C, where C = sum_i d_i P^(L-i) and d_i =
//     (x_i ^ b_i) - x_i is the low-byte change of step i (Horner order).
//     The host folds the chunks' maps in order.
#pragma once

#include "common.cuh"
#include "scan.cuh"

namespace sufgpu {

constexpr int kFastaBlock = 256;
constexpr int kFastaItems = 16;
constexpr int kFastaTile = kFastaBlock * kFastaItems;
constexpr u64 kFastaWalkLimit = 1u << 16;  // bounded walks back over a line

// Unsupported-input bits (host falls back to its reader, documented).
constexpr u32 kFastaFastq = 1u << 0;
constexpr u32 kFastaLoneCr = 1u << 1;
constexpr u32 kFastaWalk = 1u << 2;

__device__ __forceinline__ u8 fasta_code(u8 c) {
  switch (c) {
    case 'A': case 'a': return 2;
    case 'C': case 'c': return 3;
    case 'G': case 'g': return 4;
    case 'T': case 't': return 5;
    default: return 6;
  }
}

struct FastaHeader {
  u64 raw;  // position of the record's '>'
  u64 out;  // output position of the 1 closing the previous record
};

// raw has n bytes plus >= 16 readable padding bytes.  first = position of the
// first '>' (the host checked the first '>'/'@' is a '>').
static __global__ void __launch_bounds__(kFastaBlock)
fasta_normalize_kernel(const u8* __restrict__ raw, u64 n, u64 first, u8* __restrict__ out,
                       u64 out_cap, u64* status_nl, u64* status_out, u32* tile_counter,
                       FastaHeader* __restrict__ headers, u64 header_cap, u64* header_count,
                       u32* unsupported, u64* out_total, DeviceFlags* flags) {
  __shared__ u64 warp_smem[kFastaBlock / 32];
  __shared__ u64 tile_prefix[2];
  __shared__ u32 tile_slot;
  const u32 tile = claim_tile(tile_counter, &tile_slot);
  const u64 p0 = static_cast<u64>(tile) * kFastaTile + threadIdx.x * kFastaItems;
  u8 b[kFastaItems + 1];
  {
    uint4 v = make_uint4(0, 0, 0, 0);
    if (p0 < n) v = *reinterpret_cast<const uint4*>(raw + p0);
    const u32 w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int i = 0; i < kFastaItems; ++i) b[i] = static_cast<u8>(w[i >> 2] >> ((i & 3) * 8));
    b[kFastaItems] = p0 + kFastaItems < n ? raw[p0 + kFastaItems] : 0;
  }
  // Newlines: last position + 1 in this thread (0 = none).
  u64 last_nl = 0;
#pragma unroll
  for (int i = 0; i < kFastaItems; ++i) {
    if (p0 + i < n && b[i] == '\n') last_nl = p0 + i + 1;
  }
  u64 agg_nl;
  const u64 excl_nl = block_exclusive_scan<kFastaBlock>(last_nl, MaxOp{}, warp_smem, &agg_nl);
  if ((threadIdx.x >> 5) == 0) {
    const u64 p = warp_lookback(status_nl, tile, agg_nl, MaxOp{}, flags, 20);
    if ((threadIdx.x & 31) == 0) tile_prefix[0] = p;
  }
  __syncthreads();
  u64 line = excl_nl > tile_prefix[0] ? excl_nl : tile_prefix[0];  // start of the current line
  if (line < first) line = first;
  bool header = line < n && raw[line] == '>';
  u32 bad = 0;
  u8 value[kFastaItems];
  bool emit[kFastaItems];
  u32 count = 0;
#pragma unroll
  for (int i = 0; i < kFastaItems; ++i) {
    const u64 p = p0 + i;
    emit[i] = false;
    value[i] = 0;
    if (p >= n || p < first) continue;
    const u8 c = b[i];
    if (p == line && p > first) {  // a line start (the first record's is `first`)
      header = c == '>';
      if (c == '@' || c == '+') bad |= kFastaFastq;
    }
    if (c == '\n') {
      line = p + 1;
      continue;
    }
    if (header) {
      if (p == line && p > first) {  // a record's '>': the 1 closing the previous one
        emit[i] = true;
        value[i] = 1;
        ++count;
      }
      continue;
    }
    const bool line_end = p + 1 == n || (i + 1 < kFastaItems ? b[i + 1] : b[kFastaItems]) == '\n';
    if (c == '\r' && line_end) {
      if (p == line) {
        // A lone "\r" line: kseq keeps it when it is the record's first
        // sequence byte, i.e. when only empty lines separate it from the header.
        u64 q = p;
        u64 steps = 0;
        while (q > first && raw[q - 1] == '\n' && steps < kFastaWalkLimit) {
          --q;
          ++steps;
        }
        // q-1 is the last byte of the previous non-empty line; find its start.
        u64 s = q - 1;
        while (s > first && raw[s - 1] != '\n' && steps < kFastaWalkLimit) {
          --s;
          ++steps;
        }
        if (steps >= kFastaWalkLimit) bad |= kFastaWalk;
        else if (raw[s] == '>') bad |= kFastaLoneCr;
      }
      continue;
    }
    emit[i] = true;
    value[i] = fasta_code(c);
    ++count;
  }
  if (bad) atomicOr(unsupported, bad);
  u64 agg_out;
  const u64 excl_out = block_exclusive_scan<kFastaBlock>(count, SumOp{}, warp_smem, &agg_out);
  if ((threadIdx.x >> 5) == 1) {
    const u64 p = warp_lookback(status_out, tile, agg_out, SumOp{}, flags, 21);
    if ((threadIdx.x & 31) == 0) tile_prefix[1] = p;
  }
  __syncthreads();
  u64 o = tile_prefix[1] + excl_out;
#pragma unroll
  for (int i = 0; i < kFastaItems; ++i) {
    if (!emit[i]) continue;
    if (o < out_cap) out[o] = value[i];
    else flag_error(flags, kErrQueueOverflow);
    if (value[i] == 1) {
      const u64 h = atomicAdd(reinterpret_cast<unsigned long long*>(header_count), 1ull);
      if (h < header_cap) headers[h] = FastaHeader{p0 + i, o};
      else flag_error(flags, kErrQueueOverflow);
    }
    ++o;
  }
  const u64 tiles = (n + kFastaTile - 1) / kFastaTile;
  if (tile == tiles - 1 && threadIdx.x == 0) *out_total = tile_prefix[1] + agg_out;
}

// FNV-1a low-byte pass j: chunk c (bytes [c*L, min(n, (c+1)*L))) starts from
// start[c] (its known low bits; bits >= j are 0 except in chunk 0, whose
// start is exact) and reports bit j of its end state.
static __global__ void __launch_bounds__(256)
fnv_level_kernel(const u8* __restrict__ data, u64 n, u64 chunk, u64 chunks,
                 const u8* __restrict__ start, u32 j, u8* __restrict__ end_bit) {
  const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
  constexpr u32 kMul = static_cast<u32>(1099511628211ull & 0xff);
  for (u64 c = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; c < chunks; c += stride) {
    const u64 lo = c * chunk;
    const u64 hi = lo + chunk < n ? lo + chunk : n;
    u32 x = start[c];
    u64 p = lo;
    for (; p + 16 <= hi; p += 16) {  // chunk starts are 16-byte aligned
      const uint4 v = *reinterpret_cast<const uint4*>(data + p);
      const u32 w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int i = 0; i < 16; ++i) x = ((x ^ ((w[i >> 2] >> ((i & 3) * 8)) & 0xff)) * kMul) & 0xff;
    }
    for (; p < hi; ++p) x = ((x ^ data[p]) * kMul) & 0xff;
    end_bit[c] = static_cast<u8>((x >> j) & 1);
  }
}

// Affine map of chunk c given its exact start byte: mult[c] = P^L and
// add[c] = C with h_end = h_start * P^L + C (mod 2^64).
static __global__ void __launch_bounds__(256)
fnv_affine_kernel(const u8* __restrict__ data, u64 n, u64 chunk, u64 chunks,
                  const u8* __restrict__ start, u64* __restrict__ mult, u64* __restrict__ add) {
  const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
  constexpr u64 kPrime = 1099511628211ull;
  for (u64 c = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; c < chunks; c += stride) {
    const u64 lo = c * chunk;
    const u64 hi = lo + chunk < n ? lo + chunk : n;
    u64 x = start[c];
    u64 acc = 0, pw = 1;
    for (u64 p = lo; p < hi; ++p) {
      const u64 y = x ^ data[p];
      acc = (acc + (y - x)) * kPrime;  // y - x wraps mod 2^64 like the hash
      pw *= kPrime;
      x = (y * kPrime) & 0xff;
    }
    mult[c] = pw;
    add[c] = acc;
  }
}

}  // namespace sufgpu
