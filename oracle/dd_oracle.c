/*
 * dd_oracle.c — CPU restatement of the reference's distance-distribution
 * algorithms.  TEST INFRASTRUCTURE ONLY: the parity tests, smoke() and the
 * bench's cpu_baseline leg use it as the checker.  Nothing in the product
 * links, loads or calls it.
 *
 * Pinned against: the golden tables in distance_distribution/src/solutions.h,
 * the archived result files under distance_distribution/results/, and the
 * reference's own `codrel` binary built from its sources (oracle/ref.mk),
 * see tests/test_oracle_pins.py.
 *
 * Every function returns the RAW device histogram that the corresponding
 * reference driver sums on the host (hcounts[0][] in the .cu drivers), plus
 * the driver's post-processing into uint128 counts (dd_oracle_post_*).
 *
 * Build: gcc -O3 -fopenmp -shared -fPIC -o oracle/_build/libdd_oracle.so oracle/dd_oracle.c -lm
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;

#define MAXB 64

static inline unsigned popc64(uint64_t v) { return (unsigned)__builtin_popcountll(v); }

/* ------------------------------------------------------------------ */
/* shapes                                                               */
/* ------------------------------------------------------------------ */

/* h as the GPU drivers compute it: ceil(log(A)/log(2.0)), src/an_coding.cu:280,
 * src/an_coding.cpp:111, src/globals.cpp:274. */
unsigned dd_oracle_h_ceil(uint64_t A) { return (unsigned)ceil(log((double)A) / log(2.0)); }
/* h as the super-A sweeps compute it: floor(log(A)/log(2.0))+1,
 * distance_distribution_super_a/src/main.cpp:209,261. */
unsigned dd_oracle_h_floor1(uint64_t A) { return (unsigned)(floor(log((double)A) / log(2.0)) + 1); }
/* Ext-Hamming check bits as run_hamming: src/hamming.cu:133. */
unsigned dd_oracle_hamming_h(unsigned n) { return n == 4 ? 4 : (n == 8 ? 5 : (n < 32 ? 6 : 7)); }

/* ------------------------------------------------------------------ */
/* AN exhaustive                                                        */
/* ------------------------------------------------------------------ */

/* Unordered pairs i<j of [0,2^n): raw[popc(A*i ^ A*j)]++.  Same quantity as
 * dancoding_shared (src/an_coding.cu:50-105; bin 0 never counted) and, after
 * doubling, as countANCodingUndetectableErrors<64> (src/an_coding.cpp:50-102),
 * whose 64x64 shard loop is kept here. */
void dd_oracle_an_exhaustive(uint64_t A, unsigned n, uint64_t* raw, unsigned nbins)
{
  const uint64_t N = 1ull << n;
  const uint64_t S = 64;
  memset(raw, 0, nbins * sizeof(uint64_t));
#pragma omp parallel
  {
    uint64_t loc[MAXB + 1] = {0};
#pragma omp for schedule(dynamic, 1)
    for (long long sx = 0; sx < (long long)N; sx += (long long)S) {
      uint64_t xe = (uint64_t)sx + S < N ? (uint64_t)sx + S : N;
      for (uint64_t x = (uint64_t)sx; x < xe; ++x) {          /* triangle of the diagonal shard */
        uint64_t m1 = x * A;
        for (uint64_t y = x + 1; y < xe; ++y) ++loc[popc64(m1 ^ (y * A))];
      }
      for (uint64_t sy = (uint64_t)sx + S; sy < N; sy += S) { /* rest of the slice */
        uint64_t ye = sy + S < N ? sy + S : N;
        for (uint64_t x = (uint64_t)sx; x < xe; ++x) {
          uint64_t m1 = x * A;
          for (uint64_t y = sy; y < ye; ++y) ++loc[popc64(m1 ^ (y * A))];
        }
      }
    }
#pragma omp critical
    for (unsigned b = 0; b < nbins; ++b) raw[b] += loc[b];
  }
}

/* Restricted to rows [r0,r1) x all j>i: used to check one row band of a big
 * instance (k=24) without enumerating all pairs. */
void dd_oracle_an_rows(uint64_t A, unsigned n, uint64_t r0, uint64_t r1, uint64_t* raw, unsigned nbins)
{
  const uint64_t N = 1ull << n;
  memset(raw, 0, nbins * sizeof(uint64_t));
#pragma omp parallel
  {
    uint64_t loc[MAXB + 1] = {0};
#pragma omp for schedule(dynamic, 1)
    for (long long i = (long long)r0; i < (long long)r1; ++i) {
      uint64_t w = (uint64_t)i * A;
      for (uint64_t j = (uint64_t)i + 1; j < N; ++j) ++loc[popc64(w ^ (j * A))];
    }
#pragma omp critical
    for (unsigned b = 0; b < nbins; ++b) raw[b] += loc[b];
  }
}

/* Unordered pairs at distance 1 and 2, found by flipping one or two of the
 * `bits` low bits of every codeword and testing the result for membership
 * (a multiple of A below A*2^n).  Independent of any pair enumeration; used
 * to arbitrate archived results that fail the conservation law. */
void dd_oracle_an_low_distance(uint64_t A, unsigned n, unsigned bits, uint64_t* d1, uint64_t* d2)
{
  const uint64_t N = 1ull << n, lim = A * N;
  uint64_t c1 = 0, c2 = 0;
#pragma omp parallel for reduction(+ : c1, c2) schedule(static)
  for (long long i = 0; i < (long long)N; ++i) {
    const uint64_t c = A * (uint64_t)i;
    for (unsigned a = 0; a < bits; ++a) {
      const uint64_t x1 = c ^ (1ull << a);
      if (x1 > c && x1 < lim && x1 % A == 0) ++c1;
      for (unsigned b = a + 1; b < bits; ++b) {
        const uint64_t x = x1 ^ (1ull << b);
        if (x > c && x < lim && x % A == 0) ++c2;
      }
    }
  }
  *d1 = c1;
  *d2 = c2;
}

/* ------------------------------------------------------------------ */
/* AN grid                                                              */
/* ------------------------------------------------------------------ */

/* Number of lattice points k with v_k = A*(T)(k*stepsize) < A<<n, k = 0,1,..
 * as dancoding_grid_1d_shared walks them (src/an_coding_grid.cu:78-107): the
 * unrolled blocks and the remainder loop together visit k = 0..K-1 where K is
 * the first k with (T)(k*stepsize) >= 2^n.  T is uint32 when n+h+1 <= 32
 * (Caller, an_coding_grid.cu:159-185).  The walk is restated literally,
 * including the Aend_p early-exit, so the count cannot drift from it. */
static uint64_t grid_lattice_count(uint64_t A, unsigned n, double stepsize, int t32, uint64_t unroll)
{
  const uint64_t Aend = A << n;
  uint64_t v = 0, k = 0;
#define CAST_T(x) (t32 ? (uint64_t)(uint32_t)(x) : (uint64_t)(x))
  uint64_t Aend_p = t32 ? (uint32_t)(Aend - A * CAST_T((double)unroll * stepsize))
                        : Aend - A * CAST_T((double)unroll * stepsize);
  for (v = 0, k = 0; v < Aend_p; k += unroll) {
    for (uint64_t u = 0; u < unroll; ++u) {
      /* body visits v_{k+u}; then v := A*(T)((k+u+1)*stepsize) */
      v = A * CAST_T((double)(k + u + 1) * stepsize);
      if (t32) v = (uint32_t)v;
    }
  }
  /* remainder loop: `++k, v = A * (T)(k * stepsize)` uses the incremented k */
  for (; v < Aend; ++k, v = t32 ? (uint32_t)(A * CAST_T((double)k * stepsize))
                                : A * CAST_T((double)k * stepsize)) {
  }
#undef CAST_T
  return k;
}

/* Lattice points the 1-D grid kernel visits for (A, n, h, m). */
uint64_t dd_oracle_grid1d_points(uint64_t A, unsigned n, unsigned h, uint64_t m)
{
  const uint64_t N = 1ull << n;
  if (m > N) m = N;
  const double step = 1.0 * (double)N / (double)m;
  return grid_lattice_count(A, n, step, (n + h + 1) <= 32, m <= 16 ? 3 : 16);
}

/* Lattice points of dancoding_grid_2d's column walk (an_coding_grid.cu:133). */
uint64_t dd_oracle_grid2d_points(uint64_t A, unsigned n, uint64_t m)
{
  const uint64_t N = 1ull << n;
  if (m > N) m = N;
  const double step = 1.0 * (double)N / (double)m;
  const uint64_t Aend = A << n;
  const int t32 = Aend < (1ull << 32);
  uint64_t v = 0, k = 0;
  while (v < Aend) {
    ++k;
    uint64_t tv = (uint64_t)((double)k * step);
    if (t32) tv = (uint32_t)tv;
    v = A * tv;
  }
  return k;
}

/* 1-D grid: every codeword w=A*i, i in [0,2^n) (iterations2 = 2^n,
 * an_coding_grid.cu:258) against the lattice v_k = A*(T)(k*stepsize),
 * stepsize = 1.0*2^n/m (an_coding_grid.cu:296); bin 0 counted.
 * Returns the lattice size K in *kcount. */
void dd_oracle_an_grid1d(uint64_t A, unsigned n, unsigned h, uint64_t m, uint64_t* raw, unsigned nbins,
                         uint64_t* kcount)
{
  const uint64_t N = 1ull << n;
  if (m > N) m = N;
  const double step = 1.0 * (double)N / (double)m;
  const int t32 = (n + h + 1) <= 32;
  const uint64_t unroll = m <= 16 ? 3 : 16;
  const uint64_t K = grid_lattice_count(A, n, step, t32, unroll);
  if (kcount) *kcount = K;
  memset(raw, 0, nbins * sizeof(uint64_t));
  const uint64_t KB = 4096; /* lattice points per block, so few-point lattices still spread over threads */
  uint64_t vbuf[4096];
  for (uint64_t kb = 0; kb < K; kb += KB) {
    const uint64_t ke = kb + KB < K ? kb + KB : K;
    for (uint64_t k = kb; k < ke; ++k) {
      uint64_t t = (uint64_t)((double)k * step);
      if (t32) t = (uint32_t)t;
      vbuf[k - kb] = A * t;
    }
#pragma omp parallel
    {
      uint64_t loc[MAXB + 1] = {0};
#pragma omp for schedule(static)
      for (long long i = 0; i < (long long)N; ++i) {
        const uint64_t w = A * (uint64_t)i;
        for (uint64_t k = 0; k < ke - kb; ++k) ++loc[popc64(w ^ vbuf[k])];
      }
#pragma omp critical
      for (unsigned b = 0; b < nbins; ++b) raw[b] += loc[b];
    }
  }
}

/* 2-D grid (dancoding_grid_2d, an_coding_grid.cu:121-140): w_i = A*(T)(i*stepsize2)
 * for i in [0, m2), v_k = A*(T)(k*stepsize) while v_k < A<<n; bin 0 NOT
 * counted.  T is uint32 iff A<<n < 2^32 (an_coding_grid.cu:188).  Returns the
 * number of coincident lattice points (the distance-0 pairs the reference's
 * kernel leaves out of bin 0). */
uint64_t dd_oracle_an_grid2d(uint64_t A, unsigned n, uint64_t m, uint64_t m2, uint64_t* raw, unsigned nbins)
{
  uint64_t zero = 0;
  const uint64_t N = 1ull << n;
  if (m > N) m = N;
  if (m2 > N) m2 = N;
  const double step = 1.0 * (double)N / (double)m;
  const double step2 = 1.0 * (double)N / (double)m2;
  const uint64_t Aend = A << n;
  const int t32 = Aend < (1ull << 32);
  memset(raw, 0, nbins * sizeof(uint64_t));
#pragma omp parallel
  {
    uint64_t loc[MAXB + 1] = {0};
#pragma omp for schedule(dynamic, 64)
    for (long long i = 0; i < (long long)m2; ++i) {
      uint64_t tw = (uint64_t)((double)(uint64_t)i * step2);
      if (t32) tw = (uint32_t)tw;
      uint64_t w = A * tw;
      uint64_t v = 0, k = 0;
      while (v < Aend) {
        ++loc[popc64(w ^ v)];
        ++k;
        uint64_t tv = (uint64_t)((double)k * step);
        if (t32) tv = (uint32_t)tv;
        v = A * tv;
      }
    }
#pragma omp critical
    {
      for (unsigned b = 1; b < nbins; ++b) raw[b] += loc[b];
      zero += loc[0];
    }
  }
  return zero;
}

/* ------------------------------------------------------------------ */
/* Philox4x32-10 and Monte Carlo                                        */
/* ------------------------------------------------------------------ */

/* Philox4x32 with 10 rounds, from Salmon, Moraes, Dror, Shaw, "Parallel Random
 * Numbers: As Easy as 1, 2, 3" (SC'11): round multipliers 0xD2511F53 and
 * 0xCD9E8D57, key schedule increments 0x9E3779B9 and 0xBB67AE85. */
void dd_oracle_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Sample t of stream `idx`: a uniform index in [0, 2^n).  n<=32: four samples
 * per Philox block, counter (t>>2, idx); n>32: two 64-bit samples per block,
 * counter (t>>1, idx); the index is the top n bits of the sample word. */
uint64_t dd_oracle_mc_index(uint64_t seed, uint64_t idx, uint64_t t, unsigned n)
{
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t out[4];
  if (n <= 32) {
    uint64_t blk = t >> 2;
    uint32_t ctr[4] = {(uint32_t)blk, (uint32_t)(blk >> 32), (uint32_t)idx, (uint32_t)(idx >> 32)};
    dd_oracle_philox(ctr, key, out);
    uint32_t r = out[t & 3];
    return n == 32 ? (uint64_t)r : (uint64_t)(r >> (32 - n));
  } else {
    uint64_t blk = t >> 1;
    uint32_t ctr[4] = {(uint32_t)blk, (uint32_t)(blk >> 32), (uint32_t)idx, (uint32_t)(idx >> 32)};
    dd_oracle_philox(ctr, key, out);
    unsigned q = (unsigned)(t & 1) * 2;
    uint64_t r = ((uint64_t)out[q] << 32) | out[q + 1];
    return n == 64 ? r : (r >> (64 - n));
  }
}

/* AN Monte Carlo (dancoding_mc_shared, src/an_coding_mc.cu:94-158, with the
 * cuRAND Sobol draw replaced by dd_oracle_mc_index): for every codeword
 * w = A*i, `it` samples v = A*j; bin 0 counted.  it is capped at 2^n
 * (an_coding_mc.cu:242). */
void dd_oracle_an_mc(uint64_t A, unsigned n, uint64_t it, uint64_t seed, uint64_t* raw, unsigned nbins)
{
  const uint64_t N = 1ull << n;
  if (it > N) it = N;
  memset(raw, 0, nbins * sizeof(uint64_t));
#pragma omp parallel
  {
    uint64_t loc[MAXB + 1] = {0};
#pragma omp for schedule(dynamic, 256)
    for (long long i = 0; i < (long long)N; ++i) {
      uint64_t w = A * (uint64_t)i;
      for (uint64_t t = 0; t < it; ++t) ++loc[popc64(w ^ (A * dd_oracle_mc_index(seed, (uint64_t)i, t, n)))];
    }
#pragma omp critical
    for (unsigned b = 0; b < nbins; ++b) raw[b] += loc[b];
  }
}

/* ------------------------------------------------------------------ */
/* Ext-Hamming                                                          */
/* ------------------------------------------------------------------ */

/* Codeword WITHOUT the overall parity bit, as the GPU drivers build it
 * (computeHamming<N>, src/hamming.cu:39-59; hamming_grid.cu:32-48 and
 * hamming_mc.cu use the variant without the N<8 branch).  N is the template
 * bucket: 8 for n in {4,8}. */
uint64_t dd_oracle_hamming_cw_gpu(uint64_t v, unsigned N, int with_n4_branch)
{
  uint64_t hm = 0;
  hm |= (uint64_t)(popc64(v & 0x56AAAD5Bull) & 1);
  hm |= (uint64_t)(popc64(v & 0x9B33366Dull) & 1) << 1;
  hm |= (uint64_t)(popc64(v & 0xE3C3C78Eull) & 1) << 2;
  if (with_n4_branch && N < 8) return (v << 3) | hm;
  hm |= (uint64_t)(popc64(v & 0x03FC07F0ull) & 1) << 3;
  if (N < 16) return (v << 4) | hm;
  hm |= (uint64_t)(popc64(v & 0x03FFF800ull) & 1) << 4;
  if (N < 32) return (v << 5) | hm;
  hm |= (uint64_t)(popc64(v & 0xFC000000ull) & 1) << 5;
  return (v << 6) | hm;
}

/* Extended Hamming codeword WITH the overall parity bit, as the brute-force
 * CPU paths build it: computeHamming08/16/24/32, src/hamming.h:22-64. */
uint64_t dd_oracle_hamming_cw_ext(uint64_t v, unsigned n)
{
  uint64_t hm = 0;
  switch (n) {
  case 8:
    hm |= (uint64_t)(popc64(v & 0x5B) & 1) << 1;
    hm |= (uint64_t)(popc64(v & 0x6D) & 1) << 2;
    hm |= (uint64_t)(popc64(v & 0x8E) & 1) << 3;
    hm |= (uint64_t)(popc64(v & 0xF0) & 1) << 4;
    hm |= (popc64(v & 0xFF) + popc64(hm)) & 1;
    return (v << 5) | hm;
  case 16:
    hm |= (uint64_t)(popc64(v & 0xAD5B) & 1) << 1;
    hm |= (uint64_t)(popc64(v & 0x366D) & 1) << 2;
    hm |= (uint64_t)(popc64(v & 0xC78E) & 1) << 3;
    hm |= (uint64_t)(popc64(v & 0x07F0) & 1) << 4;
    hm |= (uint64_t)(popc64(v & 0xF800) & 1) << 5;
    hm |= (popc64(v & 0xFFFF) + popc64(hm)) & 1;
    return (v << 6) | hm;
  case 24:
    hm |= (uint64_t)(popc64(v & 0xAAAD5B) & 1) << 1;
    hm |= (uint64_t)(popc64(v & 0x33366D) & 1) << 2;
    hm |= (uint64_t)(popc64(v & 0xC3C78E) & 1) << 3;
    hm |= (uint64_t)(popc64(v & 0xFC07F0) & 1) << 4;
    hm |= (uint64_t)(popc64(v & 0xFFF800) & 1) << 5;
    hm |= (popc64(v & 0xFFFFFF) + popc64(hm)) & 1;
    return (v << 6) | hm;
  default: /* 32 */
    hm |= (uint64_t)(popc64(v & 0x56AAAD5B) & 1) << 1;
    hm |= (uint64_t)(popc64(v & 0x9B33366D) & 1) << 2;
    hm |= (uint64_t)(popc64(v & 0xE3C3C78E) & 1) << 3;
    hm |= (uint64_t)(popc64(v & 0x03FC07F0) & 1) << 4;
    hm |= (uint64_t)(popc64(v & 0x03FFF800) & 1) << 5;
    hm |= (uint64_t)(popc64(v & 0xFC000000) & 1) << 6;
    hm |= (popc64(v & 0xFFFFFFFF) + popc64(hm)) & 1;
    return (v << 7) | hm;
  }
}

static unsigned hamming_bucket(unsigned n) { return n <= 8 ? 8 : n; }

/* Weight enumerator of dhamming (src/hamming.cu:64-81): raw[popc(cw(x))]++ for
 * every message x in [0, 2^n). */
void dd_oracle_hamming_weights(unsigned n, uint64_t* raw, unsigned nbins)
{
  const uint64_t N = 1ull << n;
  const unsigned B = hamming_bucket(n);
  memset(raw, 0, nbins * sizeof(uint64_t));
#pragma omp parallel
  {
    uint64_t loc[MAXB + 8] = {0};
#pragma omp for schedule(static)
    for (long long x = 0; x < (long long)N; ++x) ++loc[popc64(dd_oracle_hamming_cw_gpu((uint64_t)x, B, 1))];
#pragma omp critical
    for (unsigned b = 0; b < nbins; ++b) raw[b] += loc[b];
  }
}

/* Brute force of hamming_native_short.cpp:29-84: every ordered pair (a,b) of
 * extended codewords, and with 1-bit spheres every one of the n+h flips of b.
 * Literal loop (the flips are enumerated, not derived). */
void dd_oracle_hamming_pairs(unsigned n, int with_1bit, uint64_t* raw, unsigned nbins)
{
  const uint64_t N = 1ull << n;
  const unsigned L = n + dd_oracle_hamming_h(n);
  memset(raw, 0, nbins * sizeof(uint64_t));
#pragma omp parallel
  {
    uint64_t loc[MAXB + 1] = {0};
#pragma omp for schedule(dynamic, 1)
    for (long long a = 0; a < (long long)N; ++a) {
      uint64_t x = dd_oracle_hamming_cw_ext((uint64_t)a, n);
      for (uint64_t b = 0; b < N; ++b) {
        uint64_t y = dd_oracle_hamming_cw_ext(b, n);
        ++loc[popc64(x ^ y)];
        if (with_1bit)
          for (unsigned p = 0; p < L; ++p) ++loc[popc64(x ^ (y ^ (1ull << p)))];
      }
    }
#pragma omp critical
    for (unsigned b = 0; b < nbins; ++b) raw[b] += loc[b];
  }
}

/* `-e 3` (hamming_native_short_ordering.cpp:39-84): pairs a<b only, the flips
 * of b, and every count doubled at the end. */
void dd_oracle_hamming_pairs_distinct(unsigned n, int with_1bit, uint64_t* raw, unsigned nbins)
{
  const uint64_t N = 1ull << n;
  const unsigned L = n + dd_oracle_hamming_h(n);
  memset(raw, 0, nbins * sizeof(uint64_t));
#pragma omp parallel
  {
    uint64_t loc[MAXB + 1] = {0};
#pragma omp for schedule(dynamic, 1)
    for (long long a = 0; a < (long long)N; ++a) {
      uint64_t x = dd_oracle_hamming_cw_ext((uint64_t)a, n);
      for (uint64_t b = (uint64_t)a + 1; b < N; ++b) {
        uint64_t y = dd_oracle_hamming_cw_ext(b, n);
        ++loc[popc64(x ^ y)];
        if (with_1bit)
          for (unsigned p = 0; p < L; ++p) ++loc[popc64(x ^ (y ^ (1ull << p)))];
      }
    }
#pragma omp critical
    for (unsigned b = 0; b < nbins; ++b) raw[b] += loc[b];
  }
  for (unsigned b = 0; b < nbins; ++b) raw[b] <<= 1;
}

/* Ext-Hamming 1-D grid (dhamming_grid_1d, src/hamming_grid.cu:53-74):
 * shards of ShardSize messages, count_shards = iterations / ShardSize
 * (hamming_grid.cu:126), x = (u64)(w + k*stepsize) with w = shard*ShardSize*(u64)stepsize
 * and stepsize = (double)(1.0L*2^n/iterations) (hamming_grid.cu:163).  nvcc
 * contracts `w + k*stepsize` into one fused multiply-add, so fma() is used. */
static uint64_t hamming_shard_size(unsigned n)
{
  switch (n <= 8 ? 8 : n) { /* Hamming::traits::Shards, src/hamming.h:74-82 */
  case 8: return 1;
  case 16: return 16;
  case 24: return 128;
  case 32: return 256;
  case 40: return 512;
  default: return 1024;
  }
}
void dd_oracle_hamming_grid(unsigned n, uint64_t iterations, uint64_t* raw, unsigned nbins, uint64_t* samples)
{
  const uint64_t N = 1ull << n;
  if (iterations > N) iterations = N;
  const uint64_t SS = hamming_shard_size(n);
  const uint64_t shards = iterations / SS;
  const double step = (double)(1.0L * (long double)N / (long double)iterations);
  const unsigned B = hamming_bucket(n);
  if (samples) *samples = shards * SS;
  memset(raw, 0, nbins * sizeof(uint64_t));
#pragma omp parallel
  {
    uint64_t loc[MAXB + 8] = {0};
#pragma omp for schedule(static)
    for (long long s = 0; s < (long long)shards; ++s) {
      uint64_t w = (uint64_t)s * SS * (uint64_t)step;
      for (uint64_t k = 0; k < SS; ++k) {
        uint64_t x = (uint64_t)fma((double)k, step, (double)w);
        ++loc[popc64(dd_oracle_hamming_cw_gpu(x, B, 0))];
      }
    }
#pragma omp critical
    for (unsigned b = 0; b < nbins; ++b) raw[b] += loc[b];
  }
}

/* Ext-Hamming Monte Carlo (dhamming_mc, src/hamming_mc.cu:57-81) with the
 * cuRAND draw replaced by dd_oracle_mc_index(seed, 0, s, N): s in
 * [0, (it/ShardSize)*ShardSize). */
void dd_oracle_hamming_mc(unsigned n, uint64_t iterations, uint64_t seed, uint64_t* raw, unsigned nbins,
                          uint64_t* samples)
{
  const uint64_t N = 1ull << n;
  if (iterations > N) iterations = N;
  const uint64_t SS = hamming_shard_size(n);
  const uint64_t S = (iterations / SS) * SS;
  const unsigned B = hamming_bucket(n);
  if (samples) *samples = S;
  memset(raw, 0, nbins * sizeof(uint64_t));
#pragma omp parallel
  {
    uint64_t loc[MAXB + 8] = {0};
#pragma omp for schedule(static)
    for (long long s = 0; s < (long long)S; ++s)
      ++loc[popc64(dd_oracle_hamming_cw_gpu(dd_oracle_mc_index(seed, 0, (uint64_t)s, B), B, 0))];
#pragma omp critical
    for (unsigned b = 0; b < nbins; ++b) raw[b] += loc[b];
  }
}

/* ------------------------------------------------------------------ */
/* post-processing (host tails of the drivers)                          */
/* ------------------------------------------------------------------ */

static void put128(u128 v, uint64_t* lo, uint64_t* hi) { *lo = (uint64_t)v; *hi = (uint64_t)(v >> 64); }

/* run_ancoding, src/an_coding.cu:382-387: counts[0]=2^n, counts[i]=raw[i]<<1. */
void dd_oracle_post_an_exhaustive(unsigned n, const uint64_t* raw, unsigned nbins, uint64_t* lo, uint64_t* hi)
{
  put128((u128)1 << n, &lo[0], &hi[0]);
  for (unsigned i = 1; i < nbins; ++i) put128(((u128)raw[i]) << 1, &lo[i], &hi[i]);
}

/* run_ancoding_grid, an_coding_grid.cu:316-322 (all bins, incl. 0, scaled by a
 * long double factor and truncated). */
void dd_oracle_post_an_grid(int gdim, unsigned n, uint64_t m, uint64_t m2, const uint64_t* raw, unsigned nbins,
                            uint64_t* lo, uint64_t* hi)
{
  long double factor = gdim == 1 ? powl(2.0L, (long double)n) / m
                                 : powl(4.0L, (long double)n) / (m * m2);
  for (unsigned i = 0; i < nbins; ++i) put128((u128)(factor * raw[i]), &lo[i], &hi[i]);
}

/* run_ancoding_mc, an_coding_mc.cu:300-304. */
void dd_oracle_post_an_mc(unsigned n, uint64_t it, const uint64_t* raw, unsigned nbins, uint64_t* lo, uint64_t* hi)
{
  for (unsigned i = 0; i < nbins; ++i)
    put128((u128)((long double)(powl(2.0L, (long double)n) / it * raw[i])), &lo[i], &hi[i]);
}

/* run_hamming, src/hamming.cu:183-208. */
void dd_oracle_post_hamming_weights(unsigned n, int with_1bit, const uint64_t* raw, unsigned nbins,
                                    uint64_t* lo, uint64_t* hi)
{
  u128 c[MAXB + 2] = {0};
  const unsigned L = nbins - 1;
  c[0] = (u128)1 << n;
  c[1] = with_1bit ? ((u128)1 << n) * L : 0;
  c[2] = 0;
  for (unsigned i = 4; i < nbins; i += 2) { c[i] = (u128)raw[i] + raw[i - 1]; c[i - 1] = 0; }
  if (with_1bit)
    for (unsigned i = 3; i < nbins; i += 2)
      c[i] = (i + 1 < nbins) ? (u128)(i + 1) * c[i + 1] + (u128)(L - i + 1) * c[i - 1]
                             : (u128)(L - i + 1) * c[i - 1];
  for (unsigned i = 3; i < nbins; ++i) c[i] <<= n;
  for (unsigned i = 0; i < nbins; ++i) put128(c[i], &lo[i], &hi[i]);
}

/* run_hamming_grid (hamming_grid.cu:183-202) and run_hamming_mc
 * (hamming_mc.cu:195-214): scale, odd->even merge from i=2, sphere from i=1. */
void dd_oracle_post_hamming_sampled(int is_mc, unsigned n, int with_1bit, uint64_t iterations,
                                    const uint64_t* raw, unsigned nbins, uint64_t* lo, uint64_t* hi)
{
  u128 c[MAXB + 2] = {0};
  const unsigned L = nbins - 1;
  long double factor = is_mc ? powl(2.0L, (long double)(2 * n)) / iterations : powl(2.0L, (long double)n);
  c[0] = (u128)(factor * raw[0]);
  for (unsigned i = 2; i < nbins; i += 2) c[i] = (u128)(factor * (raw[i] + raw[i - 1]));
  if (with_1bit)
    for (unsigned i = 1; i < nbins; i += 2)
      c[i] = (i + 1 < nbins) ? (u128)(i + 1) * c[i + 1] + (u128)(L - i + 1) * c[i - 1]
                             : (u128)(L - i + 1) * c[i - 1];
  for (unsigned i = 0; i < nbins; ++i) put128(c[i], &lo[i], &hi[i]);
}

int dd_oracle_num_threads(void)
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ------------------------------------------------------------------ */
/* super-A candidates (ANcandidates)                                    */
/* ------------------------------------------------------------------ */

/* Smallest signed-digit weight popcount(c ^ 3c) over the codewords c = A*x,
 * x in [1, 2^k), as worker() scans them (ANcandidates/ANcandidates.cpp:120-138):
 * the scan stops once the running minimum is below `floor_`, and then returns
 * that running minimum. */
unsigned dd_oracle_naf_min(uint64_t A, unsigned k, unsigned floor_)
{
  const uint64_t xmax = (1ull << k) - 1ull;
  unsigned m = 0xffffffffu;
  uint64_t c = A;
  for (uint64_t x = 1; x <= xmax && m >= floor_; ++x, c += A) {
    const unsigned w = popc64(c ^ (3ull * c));
    if (w < m) m = w;
  }
  return m;
}

/* One (k, a) cell of ANcandidates' main loop (:256-298): every odd A in
 * [2^(a-1)+1, 2^a-1], the largest minimum weight among them (|SDR|) and the A
 * values reaching it, written ascending to out (at most cap).  Returns the
 * number of candidates.  Workers share the best completed minimum as the
 * early-exit floor, as the reference's do (:124, :140-152). */
uint64_t dd_oracle_an_candidates(unsigned k, unsigned a, uint64_t* out, uint64_t cap, unsigned* sdr)
{
  *sdr = 0;
  if (a < 2) return 0;
  const uint64_t minA = (1ull << (a - 1)) + 1ull, numA = 1ull << (a - 2);
  unsigned char* mins = (unsigned char*)malloc(numA);
  unsigned best = 0;
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t i = 0; i < (int64_t)numA; ++i) {
    unsigned floor_;
#pragma omp atomic read
    floor_ = best;
    const unsigned m = dd_oracle_naf_min(minA + 2ull * (uint64_t)i, k, floor_);
    mins[i] = (unsigned char)m;
    if (m >= floor_) {
#pragma omp critical(dd_oracle_naf_best)
      if (m > best) best = m;
    }
  }
  uint64_t count = 0;
  for (uint64_t i = 0; i < numA; ++i)
    if (mins[i] == best) {
      if (count < cap) out[count] = minA + 2ull * i;
      ++count;
    }
  free(mins);
  *sdr = best;
  return count;
}
