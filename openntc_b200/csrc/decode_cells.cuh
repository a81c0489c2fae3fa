// Packed latent cells of the .ntc pyramids, read the way ntc_decode.hlsli:135-140 / 239-254
// extracts them: shared by the int8 and the float-model decoders.
#pragma once
#include <cstdint>

namespace ontc {

// The BITS bits of packed cell `cell` (bits [cell * BITS, (cell + 1) * BITS) of the level
// starting at word `word_off`) as a little-endian stream of 32-bit words.  A code never
// spans two words, so code c is (s[c*B / 32] >> (c*B % 32)) & mask.
template <int BITS>
__device__ __forceinline__ void cell_stream(const uint32_t* __restrict__ buf, uint32_t words, uint32_t word_off,
                                            uint32_t cell, uint32_t (&s)[(BITS + 31) / 32])
{
  constexpr int NW = (BITS + 31) / 32;
  const uint64_t bitpos = (uint64_t)cell * (uint64_t)BITS;
  const uint64_t w = (uint64_t)word_off + (bitpos >> 5);  // 64-bit: never wraps past the bound check
  if constexpr (BITS % 32 == 0) {
#pragma unroll
    for (int j = 0; j < NW; j++) s[j] = w + j < words ? __ldg(buf + w + j) : 0u;
  } else {
    uint32_t raw[NW + 1];
#pragma unroll
    for (int j = 0; j <= NW; j++) raw[j] = w + j < words ? __ldg(buf + w + j) : 0u;
    const uint32_t off = (uint32_t)bitpos & 31u;
#pragma unroll
    for (int j = 0; j < NW; j++) s[j] = __funnelshift_r(raw[j], raw[j + 1], off);
  }
}

template <int B>
__device__ __forceinline__ uint32_t code_of(const uint32_t* s, int c)
{
  return (s[(c * B) >> 5] >> ((c * B) & 31)) & ((1u << B) - 1u);
}

}  // namespace ontc
