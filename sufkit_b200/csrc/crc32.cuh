// CRC-32 (the zlib / gzip checksum the reference's container writer keeps per
// .sufidx section, src/serialization.cpp:47-56) of device-resident planes.
//
// Arithmetic over GF(2): in zlib's bit order (reflected), bit 31 of a word is
// the coefficient of x^0 and bit 0 that of x^31; P is the generator
// x^32 + x^26 + x^23 + x^22 + x^16 + x^12 + x^11 + x^10 + x^8 + x^7 + x^5 +
// x^4 + x^2 + x + 1, whose low 32 coefficients read 0xEDB88320 in this order.
// The raw remainder R(data) (state 0 before the first byte, nothing XORed at
// the end) is linear, and appending B to A maps the remainders as
//     R(A B) = R(A) * x^(8|B|) mod P  xor  R(B),
// which is how independent pieces combine.  zlib's crc32(c, data) runs R from
// state c ^ 0xFFFFFFFF and XORs the result with 0xFFFFFFFF.
#pragma once

#include "common.cuh"

namespace sufgpu {

constexpr u32 kCrcPoly = 0xEDB88320u;
constexpr u32 kCrcPiece = 64;                   // bytes per thread
constexpr u32 kCrcBlock = 256;                  // threads per block
constexpr u32 kCrcChunk = kCrcPiece * kCrcBlock;  // 16 KiB per block

// a(x) * b(x) mod P.
__host__ __device__ inline u32 crc_mulmod(u32 a, u32 b) {
  u32 product = 0;
  for (int i = 0; i < 32; ++i) {  // b = b_in * x^i as i advances
    if ((a >> (31 - i)) & 1u) product ^= b;
    b = (b & 1u) ? (b >> 1) ^ kCrcPoly : b >> 1;
  }
  return product;
}

// x^(8 * bytes) mod P by binary powering of x^8 (bit 23 in this order).
__host__ __device__ inline u32 crc_shift_factor(u64 bytes) {
  u32 result = 0x80000000u;  // x^0
  u32 base = 0x00800000u;    // x^8
  while (bytes) {
    if (bytes & 1u) result = crc_mulmod(result, base);
    base = crc_mulmod(base, base);
    bytes >>= 1;
  }
  return result;
}

// Byte table of the remainder step: t[i] = R of the single byte i.
__host__ __device__ inline u32 crc_table_entry(u32 i) {
  u32 c = i;
  for (int k = 0; k < 8; ++k) c = (c & 1u) ? (c >> 1) ^ kCrcPoly : c >> 1;
  return c;
}

// Raw remainders of the full 16 KiB chunks of data[0, chunks * kCrcChunk):
// each thread takes one 64-byte piece, then the block folds its 256 pieces
// in a tree (each level's right-hand neighbour is 64 * 2^level bytes long).
static __global__ void __launch_bounds__(kCrcBlock)
crc_chunks_kernel(const u8* __restrict__ data, u64 chunks, u32* __restrict__ raw) {
  __shared__ u32 table[256];
  __shared__ u32 level_factor[8];
  __shared__ u32 part[kCrcBlock];
  table[threadIdx.x] = crc_table_entry(threadIdx.x);
  if (threadIdx.x < 8) level_factor[threadIdx.x] = crc_shift_factor(u64(kCrcPiece) << threadIdx.x);
  __syncthreads();
  for (u64 chunk = blockIdx.x; chunk < chunks; chunk += gridDim.x) {
    const u8* piece = data + chunk * kCrcChunk + threadIdx.x * kCrcPiece;
    u32 c = 0;
#pragma unroll
    for (u32 w = 0; w < kCrcPiece / 16; ++w) {
      const uint4 v = reinterpret_cast<const uint4*>(piece)[w];
      const u32 words[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int q = 0; q < 4; ++q) {
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          c = table[(c ^ (words[q] >> (8 * b))) & 0xffu] ^ (c >> 8);
        }
      }
    }
    part[threadIdx.x] = c;
    __syncthreads();
    for (u32 level = 0, span = 1; span < kCrcBlock; ++level, span <<= 1) {
      if ((threadIdx.x & (2 * span - 1)) == 0) {
        part[threadIdx.x] =
            crc_mulmod(part[threadIdx.x], level_factor[level]) ^ part[threadIdx.x + span];
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) raw[chunk] = part[0];
    __syncthreads();
  }
}

// One fold level over node remainders: node j covers `width` bytes except
// possibly the last, which covers last_width.  out[j] = in[2j] shifted by the
// length of in[2j+1], xor in[2j+1] (or in[2j] when it has no partner).
static __global__ void __launch_bounds__(256)
crc_fold_kernel(const u32* __restrict__ in, u64 count, u64 width, u64 last_width,
                u32 full_factor, u32* __restrict__ out) {
  for (u64 j = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; 2 * j < count;
       j += static_cast<u64>(gridDim.x) * blockDim.x) {
    const u64 left = 2 * j, right = left + 1;
    if (right >= count) {
      out[j] = in[left];
      continue;
    }
    const u32 factor = right == count - 1 && last_width != width ? crc_shift_factor(last_width)
                                                                 : full_factor;
    out[j] = crc_mulmod(in[left], factor) ^ in[right];
  }
}

}  // namespace sufgpu
