// dd_device.cuh — device building blocks shared by the histogram kernels:
// codeword generators, Philox4x32-10, and the warp-private shared-memory bins.
#pragma once
#include <cstdint>

namespace dd {

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), written from the
// published round function: two 32x32->64 products with 0xD2511F53 and
// 0xCD9E8D57 per round, key schedule bumped by 0x9E3779B9 / 0xBB67AE85.
// ---------------------------------------------------------------------------
struct Philox4 { uint32_t x, y, z, w; };

__host__ __device__ __forceinline__ Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                          uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
#if defined(__CUDA_ARCH__)
    // separate low and high multiplies: measured faster on sm_100a than one
    // 32x32->64 multiply, whose wide result occupies the FMA-heavy pipe longer
    const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
    const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
#else
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t lo0 = (uint32_t)p0, hi0 = (uint32_t)(p0 >> 32);
    const uint32_t lo1 = (uint32_t)p1, hi1 = (uint32_t)(p1 >> 32);
#endif
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
  }
  return Philox4{c0, c1, c2, c3};
}

// ---------------------------------------------------------------------------
// Ext-Hamming codewords.  Two definitions exist in the reference:
//  - hamming_cw_gpu: parity bits WITHOUT the overall parity bit, placed in the
//    low bits (computeHamming<N>, src/hamming.cu:39-59; the grid/MC copies in
//    hamming_grid.cu:32-48 and hamming_mc.cu lack the N<8 branch);
//  - hamming_cw_ext: the extended codeword WITH the overall parity bit
//    (computeHamming08/16/24/32, src/hamming.h:22-64), used by the brute force.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ unsigned popc64(uint64_t v) {
#if defined(__CUDA_ARCH__)
  return __popcll(v);
#else
  return (unsigned)__builtin_popcountll(v);
#endif
}

__host__ __device__ __forceinline__ uint64_t hamming_cw_gpu(uint64_t v, unsigned N, bool n4_branch) {
  uint64_t hm = 0;
  hm |= (uint64_t)(popc64(v & 0x56AAAD5Bull) & 1);
  hm |= (uint64_t)(popc64(v & 0x9B33366Dull) & 1) << 1;
  hm |= (uint64_t)(popc64(v & 0xE3C3C78Eull) & 1) << 2;
  if (n4_branch && N < 8) return (v << 3) | hm;
  hm |= (uint64_t)(popc64(v & 0x03FC07F0ull) & 1) << 3;
  if (N < 16) return (v << 4) | hm;
  hm |= (uint64_t)(popc64(v & 0x03FFF800ull) & 1) << 4;
  if (N < 32) return (v << 5) | hm;
  hm |= (uint64_t)(popc64(v & 0xFC000000ull) & 1) << 5;
  return (v << 6) | hm;
}

// Parity masks of the extended codes, bit 1.. of the parity field; bit 0 is
// the overall parity.  Shift of the message = number of parity bits.
__host__ __device__ __forceinline__ uint64_t hamming_cw_ext(uint64_t v, unsigned n) {
  uint64_t hm = 0;
  unsigned shift;
  if (n == 8) {
    hm |= (uint64_t)(popc64(v & 0x5Bull) & 1) << 1;
    hm |= (uint64_t)(popc64(v & 0x6Dull) & 1) << 2;
    hm |= (uint64_t)(popc64(v & 0x8Eull) & 1) << 3;
    hm |= (uint64_t)(popc64(v & 0xF0ull) & 1) << 4;
    hm |= (popc64(v & 0xFFull) + popc64(hm)) & 1;
    shift = 5;
  } else if (n == 16) {
    hm |= (uint64_t)(popc64(v & 0xAD5Bull) & 1) << 1;
    hm |= (uint64_t)(popc64(v & 0x366Dull) & 1) << 2;
    hm |= (uint64_t)(popc64(v & 0xC78Eull) & 1) << 3;
    hm |= (uint64_t)(popc64(v & 0x07F0ull) & 1) << 4;
    hm |= (uint64_t)(popc64(v & 0xF800ull) & 1) << 5;
    hm |= (popc64(v & 0xFFFFull) + popc64(hm)) & 1;
    shift = 6;
  } else if (n == 24) {
    hm |= (uint64_t)(popc64(v & 0xAAAD5Bull) & 1) << 1;
    hm |= (uint64_t)(popc64(v & 0x33366Dull) & 1) << 2;
    hm |= (uint64_t)(popc64(v & 0xC3C78Eull) & 1) << 3;
    hm |= (uint64_t)(popc64(v & 0xFC07F0ull) & 1) << 4;
    hm |= (uint64_t)(popc64(v & 0xFFF800ull) & 1) << 5;
    hm |= (popc64(v & 0xFFFFFFull) + popc64(hm)) & 1;
    shift = 6;
  } else {  // 32
    hm |= (uint64_t)(popc64(v & 0x56AAAD5Bull) & 1) << 1;
    hm |= (uint64_t)(popc64(v & 0x9B33366Dull) & 1) << 2;
    hm |= (uint64_t)(popc64(v & 0xE3C3C78Eull) & 1) << 3;
    hm |= (uint64_t)(popc64(v & 0x03FC07F0ull) & 1) << 4;
    hm |= (uint64_t)(popc64(v & 0x03FFF800ull) & 1) << 5;
    hm |= (uint64_t)(popc64(v & 0xFC000000ull) & 1) << 6;
    hm |= (popc64(v & 0xFFFFFFFFull) + popc64(hm)) & 1;
    shift = 7;
  }
  return (v << shift) | hm;
}

// Monte Carlo index draw: sample t of stream idx -> uniform index in [0, 2^n).
// n <= 32: four samples per Philox block (counter = (t>>2, idx)); n > 32: two
// 64-bit samples per block (counter = (t>>1, idx)).  The index is the top n
// bits of the sample word.  Host and device share this definition.
__host__ __device__ __forceinline__ uint64_t mc_index(uint64_t seed, uint64_t idx, uint64_t t, unsigned n) {
  if (n <= 32) {
    const uint64_t blk = t >> 2;
    Philox4 o = philox4x32_10((uint32_t)blk, (uint32_t)(blk >> 32), (uint32_t)idx, (uint32_t)(idx >> 32),
                              (uint32_t)seed, (uint32_t)(seed >> 32));
    const unsigned q = (unsigned)(t & 3);
    const uint32_t r = q == 0 ? o.x : q == 1 ? o.y : q == 2 ? o.z : o.w;
    return n == 32 ? (uint64_t)r : (uint64_t)(r >> (32 - n));
  }
  const uint64_t blk = t >> 1;
  Philox4 o = philox4x32_10((uint32_t)blk, (uint32_t)(blk >> 32), (uint32_t)idx, (uint32_t)(idx >> 32),
                            (uint32_t)seed, (uint32_t)(seed >> 32));
  const uint64_t r = (t & 1) ? (((uint64_t)o.z << 32) | o.w) : (((uint64_t)o.x << 32) | o.y);
  return n == 64 ? r : (r >> (64 - n));
}

// Grid lattice codeword: v = A * (T)(k * stepsize), T = uint32 or uint64 as the
// reference's Caller picks it (src/an_coding_grid.cu:83-106).
__host__ __device__ __forceinline__ uint64_t lattice_value(uint64_t A, uint64_t k, double step, uint32_t t32) {
  if (t32) return (uint64_t)(uint32_t)(A * (uint64_t)(uint32_t)((double)k * step));
  return A * (uint64_t)((double)k * step);
}

// Upper-triangle decode (both kernels' super-tile order): s in [0, M(M+1)/2)
// -> (r, c), r <= c, column by column: column c holds rows 0..c, and
// T(c) = c(c+1)/2 entries precede it.  Consecutive super tiles share their
// columns, so the tcgen05 kernel keeps one column operand for a run of them.
// The square root only seeds the column; the two loops correct it exactly
// against the integer column starts.
__device__ __forceinline__ void tri_decode(uint64_t s, uint64_t M, uint64_t& r, uint64_t& c) {
  double x = (sqrt(8.0 * (double)s + 1.0) - 1.0) * 0.5;
  int64_t cc = (int64_t)x;
  if (cc < 0) cc = 0;
  if ((uint64_t)cc >= M) cc = (int64_t)M - 1;
  auto T = [](uint64_t c_) { return c_ * (c_ + 1) / 2; };
  while ((uint64_t)cc + 1 < M && T((uint64_t)cc + 1) <= s) ++cc;
  while (cc > 0 && T((uint64_t)cc) > s) --cc;
  c = (uint64_t)cc;
  r = s - T(c);
}

// Tile lt of a grid (rectangle) job: 128 rows x 1024 columns, column tile by
// column tile (both kernels), so consecutive tiles share their columns.
// row_tiles = ceil(rows / 128).
__host__ __device__ __forceinline__ void rect_decode(uint64_t lt, uint64_t row_tiles, uint64_t& r0, uint64_t& c0) {
  r0 = (lt % row_tiles) * 128;
  c0 = (lt / row_tiles) * 1024;
}

}  // namespace dd
