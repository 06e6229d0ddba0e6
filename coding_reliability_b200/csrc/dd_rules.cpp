// dd_rules.cpp — host rules of the reference's drivers: shape derivation,
// planning of device jobs, post-processing of raw histograms, the golden-table
// error estimates and the results-file text layout.  No CUDA calls here, so
// all of it is testable without a GPU.
#include <cmath>
#include <cstring>
#include <iomanip>
#include <sstream>

#include "dd_host.h"

namespace dd {

uint32_t h_ceil_log2(uint64_t A) { return (uint32_t)std::ceil(std::log((double)A) / std::log(2.0)); }
uint32_t h_floor_log2_p1(uint64_t A) { return (uint32_t)(std::floor(std::log((double)A) / std::log(2.0)) + 1); }
uint32_t hamming_h(uint32_t n) { return n == 4 ? 4 : (n == 8 ? 5 : (n < 32 ? 6 : 7)); }

static bool is_pow2(uint64_t A) { return (A & (A - 1)) == 0; }

static uint32_t bit_length(u128 v) {
  uint32_t b = 0;
  while (v) { ++b; v >>= 1; }
  return b;
}

// Ext-Hamming traits, src/hamming.h:74-82.
static uint32_t hamming_shard(uint32_t n) {
  switch (n <= 8 ? 8 : n) {
    case 8: return 1;
    case 16: return 16;
    case 24: return 128;
    case 32: return 256;
    case 40: return 512;
    default: return 1024;
  }
}

// Lattice value index (T)(k*step) as the grid kernels compute it.  The
// searches below only compare it against limits <= 2^n, and for every k
// whose product is below 2^32 the uint32 and uint64 casts agree; above that
// the uint32 cast wraps, which would make the sequence non-monotone, so the
// comparison uses the exact (non-wrapping) truncation.
static uint64_t lattice_index(uint64_t k, double step, bool t32) {
  (void)t32;
  const double x = (double)k * step;
  return x >= 18446744073709551615.0 ? ~0ull : (uint64_t)x;
}

// First k >= lo with (T)(k*step) >= limit (the index sequence is non-decreasing).
static uint64_t first_at_or_above(uint64_t lo, uint64_t hi, double step, bool t32, uint64_t limit) {
  while (lo < hi) {
    const uint64_t mid = lo + (hi - lo) / 2;
    if (lattice_index(mid, step, t32) >= limit) hi = mid; else lo = mid + 1;
  }
  return lo;
}

// Points dancoding_grid_1d_shared visits (an_coding_grid.cu:78-107): blocks of
// `unroll` lattice points while the block's first point is below Aend_p, then
// single points while below Aend.  v_k < Aend <=> (T)(k*step) < 2^n.
static uint64_t grid1d_points(uint32_t n, double step, bool t32, uint64_t unroll) {
  const uint64_t N = 1ull << n;
  const uint64_t kmax = N + 2;
  const uint64_t exact = first_at_or_above(0, kmax, step, t32, N);
  // Aend_p = Aend - A*(T)(unroll*step)  <=>  index limit N - (T)(unroll*step)
  const uint64_t ustep = lattice_index(unroll, step, t32);
  uint64_t blocks_end = 0;
  if (ustep < N) {
    const uint64_t limit = N - ustep;
    // block starts k0 = b*unroll with index(k0) < limit: count of such b
    uint64_t lo = 0, hi = kmax / unroll + 2;
    while (lo < hi) {
      const uint64_t mid = lo + (hi - lo) / 2;
      if (lattice_index(mid * unroll, step, t32) >= limit) hi = mid; else lo = mid + 1;
    }
    blocks_end = lo * unroll;
  }
  return blocks_end > exact ? blocks_end : exact;
}

int derive_shape(const dd_request& req, Shape& s, std::string& err) {
  s = Shape();
  s.code = req.code;
  s.mode = req.mode;
  s.n = req.n;
  if (req.code == DD_CODE_AN) {
    if (req.n < 1 || req.n > 48) { err = "AN: n must be in [1, 48]"; return DD_ERR_UNSUPPORTED; }
    if (req.mode > DD_MODE_MONTE_CARLO) { err = "unknown mode"; return DD_ERR_INVALID_ARGUMENT; }
    if (req.convention > DD_CONV_SUPER_A) { err = "unknown convention"; return DD_ERR_INVALID_ARGUMENT; }
    uint64_t A = req.A == 0 ? 1 : req.A;  // src/main.cpp:79
    if (A >> 32) { err = "AN: A must be below 2^32"; return DD_ERR_UNSUPPORTED; }
    uint32_t h;
    if (req.convention == DD_CONV_SUPER_A) {
      h = req.h ? req.h : h_floor_log2_p1(A);  // computed from A before normalisation
      if (is_pow2(A)) A = 1;
    } else if (req.convention == DD_CONV_CPU) {
      if (req.mode != DD_MODE_EXHAUSTIVE) { err = "CPU convention exists for exhaustive mode only"; return DD_ERR_INVALID_ARGUMENT; }
      h = req.h ? req.h : h_ceil_log2(A);
    } else {
      if (is_pow2(A)) A = 1;  // src/an_coding.cu:278-279
      h = req.h ? req.h : h_ceil_log2(A);
    }
    s.A = A;
    s.h = h;
    s.nbins = req.n + h + 1;
    if (s.nbins > kMaxBins) { err = "CountCounts not supported (n+h+1 > 64)"; return DD_ERR_UNSUPPORTED; }
    const uint64_t N = 1ull << req.n;
    const u128 maxcw = (u128)A * (N - 1);
    const uint32_t bits = bit_length(maxcw);
    if (bits > req.n + h) { err = "h too small for A: codewords exceed n+h bits"; return DD_ERR_INVALID_ARGUMENT; }
    s.wide = bits > 32;
    if (req.mode == DD_MODE_EXHAUSTIVE) {
      if (req.n > 40) { err = "AN exhaustive: n > 40 not supported"; return DD_ERR_UNSUPPORTED; }
    } else if (req.mode == DD_MODE_GRID_1D || req.mode == DD_MODE_GRID_2D) {
      if (req.m == 0) { err = "grid: m must be > 0"; return DD_ERR_INVALID_ARGUMENT; }
      s.m = req.m > N ? N : req.m;  // an_coding_grid.cu:257
      s.step = 1.0 * (double)N / (double)s.m;
      if (req.mode == DD_MODE_GRID_1D) {
        if (s.m < 3) { err = "1-D grid needs m >= 3 (an_coding_grid.cu:155)"; return DD_ERR_INVALID_ARGUMENT; }
        s.m2 = N;
        s.t32 = s.nbins <= 32;
        s.lattice = grid1d_points(req.n, s.step, s.t32, s.m <= 16 ? 3 : 16);
        // The unrolled walk could in principle run past the last in-range point
        // (v_k >= A<<n); that never happens for stepsize >= 1, and a point past
        // the range could have n+h+1 set bits, so refuse rather than overflow.
        if (s.lattice > first_at_or_above(0, N + 2, s.step, s.t32, N) ||
            (s.lattice && lattice_index(s.lattice - 1, s.step, s.t32) >= N)) {
          err = "1-D grid: lattice walk leaves the codeword range";
          return DD_ERR_UNSUPPORTED;
        }
      } else {
        const uint64_t m2 = req.m2 ? req.m2 : req.m;  // src/main.cpp:127-128
        s.m2 = m2 > N ? N : m2;
        s.step2 = 1.0 * (double)N / (double)s.m2;
        s.t32 = (A << req.n) < (1ull << 32);     // an_coding_grid.cu:188
        s.lattice = first_at_or_above(0, N + 2, s.step, s.t32, N);
        if (lattice_index(s.m2 - 1, s.step2, s.t32) >= N) {
          err = "2-D grid: row lattice leaves the codeword range";
          return DD_ERR_UNSUPPORTED;
        }
      }
    } else {
      if (req.m == 0) { err = "Monte Carlo: m must be > 0"; return DD_ERR_INVALID_ARGUMENT; }
      s.m = req.m > N ? N : req.m;  // an_coding_mc.cu:242
    }
    return DD_OK;
  }
  if (req.code == DD_CODE_EXT_HAMMING) {
    const uint32_t n = req.n;
    if (n != 4 && n != 8 && n != 16 && n != 24 && n != 32 && n != 40 && n != 48) {
      err = "Unsupported n.";
      return DD_ERR_UNSUPPORTED;
    }
    s.h = hamming_h(n);
    s.nbins = n + s.h + 1;
    s.A = 1;
    s.bucket = n <= 8 ? 8 : n;
    s.shard = hamming_shard(n);
    const uint64_t N = 1ull << n;
    if (req.mode == DD_MODE_EXHAUSTIVE) {
      if (req.hamming_method == DD_HAMMING_ALL_PAIRS || req.hamming_method == DD_HAMMING_ALL_PAIRS_DISTINCT) {
        if (n != 8 && n != 16 && n != 24) { err = "all-pairs Ext-Hamming: n in {8,16,24}"; return DD_ERR_UNSUPPORTED; }
        s.wide = n + s.h > 32;
      } else if (req.hamming_method != DD_HAMMING_WEIGHTS) {
        err = "unknown hamming_method";
        return DD_ERR_INVALID_ARGUMENT;
      }
      s.samples = N;
    } else if (req.mode == DD_MODE_GRID_1D || req.mode == DD_MODE_MONTE_CARLO) {
      if (n == 4) { err = "Ext-Hamming grid/MC: n=4 not supported"; return DD_ERR_UNSUPPORTED; }
      if (req.m == 0) { err = "m must be > 0"; return DD_ERR_INVALID_ARGUMENT; }
      s.m = req.m > N ? N : req.m;
      s.samples = (s.m / s.shard) * s.shard;  // hamming_grid.cu:126, hamming_mc.cu:132
      if (req.mode == DD_MODE_GRID_1D) s.step = (double)(1.0L * (long double)N / (long double)s.m);
    } else {
      err = "Ext-Hamming has no 2-D grid";
      return DD_ERR_INVALID_ARGUMENT;
    }
    return DD_OK;
  }
  err = "unknown code";
  return DD_ERR_INVALID_ARGUMENT;
}

uint64_t job_tiles(const Job& j) {
  switch (j.kind) {
    case JOB_PAIRS:
      if (j.shape == SHAPE_TRIANGLE) return j.col_tiles * (j.col_tiles + 1) / 2 * kStrips;
      return ((j.rows + kWarpRows - 1) / kWarpRows) * j.col_tiles;
    case JOB_MC:
    {
      const uint64_t spl = j.iters - j.sample_begin, per_tile = 32 * mc_rows_per_lane(spl);
      return spl ? ((j.rows + per_tile - 1) / per_tile) * mc_chunks(spl) : 0;
    }
    default:
      return (j.iters + 32 * 256 - 1) / (32 * 256);
  }
}

void plan_jobs(const Shape& s, const dd_request& req, std::vector<Job>& jobs) {
  Job j;
  std::memset(&j, 0, sizeof(j));
  j.A = s.A;
  j.n = s.n;
  j.nbins = s.nbins;
  j.wide = s.wide;
  j.t32 = s.t32;
  j.bucket = s.bucket;
  j.shard = s.shard;
  j.seed = req.seed;
  const uint64_t N = 1ull << s.n;
  if (s.code == DD_CODE_AN) {
    if (s.mode == DD_MODE_EXHAUSTIVE) {
      j.kind = JOB_PAIRS; j.shape = SHAPE_TRIANGLE;
      j.row_kind = ROW_PROGRESSION; j.col_kind = COL_PROGRESSION;
      j.rows = j.cols = N;
      j.col_tiles = (N + kSuper - 1) / kSuper;
    } else if (s.mode == DD_MODE_GRID_1D) {
      // rows: the lattice (few), columns: every codeword (an arithmetic progression)
      j.kind = JOB_PAIRS; j.shape = SHAPE_RECT;
      j.row_kind = ROW_LATTICE; j.col_kind = COL_PROGRESSION;
      j.rows = s.lattice; j.cols = N; j.row_step = s.step;
      j.col_tiles = (N + kTileCols - 1) / kTileCols;
    } else if (s.mode == DD_MODE_GRID_2D) {
      j.kind = JOB_PAIRS; j.shape = SHAPE_RECT;
      j.row_kind = ROW_LATTICE; j.col_kind = COL_LATTICE;
      j.rows = s.m2; j.cols = s.lattice; j.row_step = s.step2; j.col_step = s.step;
      j.col_tiles = (s.lattice + kTileCols - 1) / kTileCols;
    } else {
      j.kind = JOB_MC;
      j.rows = N; j.iters = s.m;
    }
  } else {
    if (s.mode == DD_MODE_EXHAUSTIVE && req.hamming_method != DD_HAMMING_WEIGHTS) {
      j.kind = JOB_PAIRS; j.shape = SHAPE_TRIANGLE;
      j.row_kind = ROW_HAMMING_EXT; j.col_kind = COL_HAMMING_EXT;
      j.rows = j.cols = N;
      j.col_tiles = (N + kSuper - 1) / kSuper;
    } else {
      j.kind = JOB_WEIGHTS;
      j.iters = s.samples;
      j.wgen = s.mode == DD_MODE_EXHAUSTIVE ? WGEN_ALL : (s.mode == DD_MODE_GRID_1D ? WGEN_GRID : WGEN_MC);
      j.row_step = s.step;
    }
  }
  j.tiles = job_tiles(j);
  jobs.push_back(j);
}

u128 planned_pairs(const Shape& s, const dd_request& req) {
  const u128 N = (u128)1 << s.n;
  if (s.code == DD_CODE_AN) {
    switch (s.mode) {
      case DD_MODE_EXHAUSTIVE: return N * (N - 1) / 2;
      case DD_MODE_GRID_1D: return N * s.lattice;
      case DD_MODE_GRID_2D: return (u128)s.m2 * s.lattice;
      default: return N * s.m;
    }
  }
  if (s.mode == DD_MODE_EXHAUSTIVE && req.hamming_method != DD_HAMMING_WEIGHTS) return N * (N - 1) / 2;
  return s.samples;
}

// ---------------------------------------------------------------------------
// post-processing
// ---------------------------------------------------------------------------
static void store128(u128 v, uint64_t& lo, uint64_t& hi) { lo = (uint64_t)v; hi = (uint64_t)(v >> 64); }

// res.raw receives raw_in unchanged: the device bins of every evaluated pair,
// whatever the entry point (dd_histogram, the sum of dd_histogram_part calls,
// a query server slot).  Conventions that drop bins apply to counts only.
void postprocess(const dd_request& req, const Shape& s, const uint64_t* raw_in, dd_result& res) {
  uint64_t raw[kMaxBins + 1] = {0};
  for (uint32_t i = 0; i < s.nbins; ++i) raw[i] = raw_in[i];
  u128 c[kMaxBins + 2];
  for (auto& x : c) x = 0;
  const uint32_t nb = s.nbins, n = s.n;
  res.max_rel_error = -1.0;
  if (s.code == DD_CODE_AN) {
    if (s.mode == DD_MODE_EXHAUSTIVE) {
      // src/an_coding.cu:382-387 (and an_coding.cpp's diagonal ++ / off-diagonal +=2)
      c[0] = (u128)1 << n;
      for (uint32_t i = 1; i < nb; ++i) c[i] = (u128)raw[i] << 1;
    } else if (s.mode == DD_MODE_GRID_1D || s.mode == DD_MODE_GRID_2D) {
      // dancoding_grid_2d never flushes bin 0 (an_coding_grid.cu:121-140): the
      // coincident lattice points the device counted there are left out of counts
      if (s.mode == DD_MODE_GRID_2D) raw[0] = 0;
      // an_coding_grid.cu:316-322
      const long double factor = s.mode == DD_MODE_GRID_1D
                                     ? powl(2.0L, (long double)n) / s.m
                                     : powl(4.0L, (long double)n) / (s.m * s.m2);
      for (uint32_t i = 0; i < nb; ++i) c[i] = (u128)(factor * raw[i]);
      res.max_rel_error = rel_error_an(s.A, n, c, 0, nullptr);
    } else {
      // an_coding_mc.cu:300-304
      for (uint32_t i = 0; i < nb; ++i)
        c[i] = (u128)((long double)(powl(2.0L, (long double)n) / s.m * raw[i]));
      res.max_rel_error = rel_error_an(s.A, n, c, 0, nullptr);
    }
    // minimum distance: src/an_coding.cu:390-403, an_coding.cpp:121-134,
    // super_a/src/main.cpp:157-170 (range (nbins+1)/2).
    const uint32_t lim = req.convention == DD_CONV_SUPER_A ? (nb + 1) / 2 : nb / 2;
    u128 mincb = req.convention == DD_CONV_CPU ? (u128)0xFFFFFFFFull : ~(u128)0;
    uint64_t minb = 0xFFFF;
    for (uint32_t i = 1; i < lim; ++i)
      if (c[i] != 0 && c[i] < mincb) { minb = i; mincb = c[i]; break; }
    res.minb = minb;
    store128(mincb, res.mincb_lo, res.mincb_hi);
  } else {
    const uint32_t L = nb - 1;
    const bool w1 = req.with_1bit != 0;
    if (s.mode == DD_MODE_EXHAUSTIVE && req.hamming_method != DD_HAMMING_WEIGHTS) {
      // raw = unordered pairs i<j.  `-e 2/4` count ordered pairs incl. the
      // diagonal (hamming_native_short.cpp:52-71), `-e 3` only a<b doubled
      // (hamming_native_short_ordering.cpp:52-81); with spheres every pair at
      // distance d adds d flips at d-1 and L-d flips at d+1.
      u128 P[kMaxBins + 2];
      for (auto& x : P) x = 0;
      P[0] = (req.hamming_method == DD_HAMMING_ALL_PAIRS ? ((u128)1 << n) : 0) + ((u128)raw[0] << 1);
      for (uint32_t i = 1; i < nb; ++i) P[i] = (u128)raw[i] << 1;
      for (uint32_t d = 0; d < nb; ++d) {
        c[d] += P[d];
        if (w1) {
          if (d > 0) c[d - 1] += (u128)d * P[d];
          if (d + 1 < nb) c[d + 1] += (u128)(L - d) * P[d];
        }
      }
    } else if (s.mode == DD_MODE_EXHAUSTIVE) {
      // src/hamming.cu:183-208
      c[0] = (u128)1 << n;
      c[1] = w1 ? ((u128)1 << n) * L : 0;
      c[2] = 0;
      for (uint32_t i = 4; i < nb; i += 2) { c[i] = (u128)raw[i] + raw[i - 1]; c[i - 1] = 0; }
      if (w1)
        for (uint32_t i = 3; i < nb; i += 2)
          c[i] = (i + 1 < nb) ? (u128)(i + 1) * c[i + 1] + (u128)(L - i + 1) * c[i - 1]
                              : (u128)(L - i + 1) * c[i - 1];
      for (uint32_t i = 3; i < nb; ++i) c[i] <<= n;
    } else {
      // hamming_grid.cu:183-202, hamming_mc.cu:195-214
      const long double factor = s.mode == DD_MODE_MONTE_CARLO ? powl(2.0L, (long double)(2 * n)) / s.m
                                                               : powl(2.0L, (long double)n);
      c[0] = (u128)(factor * raw[0]);
      for (uint32_t i = 2; i < nb; i += 2) c[i] = (u128)(factor * (raw[i] + raw[i - 1]));
      if (w1)
        for (uint32_t i = 1; i < nb; i += 2)
          c[i] = (i + 1 < nb) ? (u128)(i + 1) * c[i + 1] + (u128)(L - i + 1) * c[i - 1]
                              : (u128)(L - i + 1) * c[i - 1];
      res.max_rel_error = abs_error_hamming(n, c, 0, w1, nullptr);
    }
    res.minb = 0xFFFF;
    store128(~(u128)0, res.mincb_lo, res.mincb_hi);
  }
  res.nbins = nb;
  res.h = s.h;
  res.A = s.A;
  res.iterations = s.m;
  res.iterations2 = s.mode == DD_MODE_GRID_2D ? s.m2 : 0;
  for (uint32_t i = 0; i < kMaxBins; ++i) {
    res.raw[i] = i < nb ? raw_in[i] : 0;
    store128(i < nb ? c[i] : 0, res.counts_lo[i], res.counts_hi[i]);
  }
}

// ---------------------------------------------------------------------------
// Golden tables of the reference (distance_distribution/src/solutions.h:18-114):
// Ext-Hamming weight distributions and exact AN histograms for A in {61, 641},
// n in {8, 16, 24}.  They are data the error estimates compare against, so
// they are the same numbers.
// ---------------------------------------------------------------------------
static const uint64_t kSolHam8[] = {0, 0, 0, 0, 55, 0, 96, 0, 87, 0, 16, 0, 1, 0};
static const uint64_t kSolHam16[] = {0, 0, 0, 0, 263, 0, 2224, 0, 10202, 0, 19952, 0,
                                     20414, 0, 9872, 0, 2389, 0, 208, 0, 11, 0, 0};
static const uint64_t kSolHam24[] = {0, 0, 0, 0, 945, 0, 18200, 0, 183885, 0, 936936, 0,
                                     2705885, 0, 4541040, 0, 4547475, 0, 2700880, 0, 939939, 0,
                                     182520, 0, 18655, 0, 840, 0, 15, 0, 0};
static const uint64_t kSolHam32[] = {0, 0, 0, 0, 1583, 0, 51744, 0, 965668, 0, 9908896, 0,
                                     61116300, 0, 235727520, 0, 589304574, 0, 974127392, 0,
                                     1077087634, 0, 797231712, 0, 392806740, 0, 126854112, 0,
                                     26224444, 0, 3311840, 0, 238729, 0, 8288, 0, 119, 0, 0, 0};
static const uint64_t kAn8A61[] = {256, 0, 0, 1362, 4106, 8358, 12092, 13468, 11884, 8176, 4134, 1262, 304, 134, 0};
static const uint64_t kAn16A61[] = {65536, 0, 0, 1606966, 8059514, 27430662, 76516894, 175266760,
                                    328771580, 510287490, 662075682, 721640166, 661335744, 508583906,
                                    326705966, 174110768, 76242514, 26993534, 7476282, 1531440, 234736,
                                    31156, 0, 0};
static const uint64_t kAn24A61[] = {16777216ull, 0ull, 0ull, 1149033026ull, 7730342814ull, 37886151670ull,
                                    157227382818ull, 540172017744ull, 1548938717128ull, 3775178858076ull,
                                    7912978808738ull, 14366801387648ull, 22718650779984ull, 31423264112014ull,
                                    38125165878518ull, 40640411783310ull, 38080772766468ull, 31348111833932ull,
                                    22633509878072ull, 14291703266250ull, 7859208391852ull, 3742071413564ull,
                                    1530719780276ull, 532399828822ull, 155292628118ull, 37269877988ull,
                                    7160570684ull, 1060815102ull, 115652770ull, 7976054ull, 0ull, 0ull};
static const uint64_t kAn24A641[] = {16777216, 0, 10076802, 153434946, 1150452598, 6049205330,
                                     28899516102, 115368656122, 378189081646, 1058452761638,
                                     2573467489292, 5466591303774, 10201679305232, 16811402697690,
                                     24559836981782, 31900986742874, 36914263923702, 38095535515896,
                                     35074592513254, 28799084410110, 21063110529820, 13694798923552,
                                     7892709334408, 4016481691866, 1795726693726, 700858354732,
                                     236678653462, 68351026422, 16618883926, 3276574070, 529150272,
                                     92569066, 10129120, 3350208, 0};
static const uint64_t kAn16A641[] = {65536, 0, 0, 262054, 1471362, 5233458, 18030526, 51777972, 119084336,
                                     228590406, 374383580, 526096540, 636024742, 662561746, 594903286,
                                     460477338, 306623886, 174747162, 84584460, 34452696, 11614808,
                                     3148728, 651320, 135498, 45856, 0};
static const uint64_t kAn8A641[] = {256, 0, 0, 596, 1302, 2316, 4624, 8218, 11060, 12318, 11024, 7378,
                                    3958, 1792, 552, 118, 24, 0, 0};

template <typename T>
static T binomial(T n, T k) {  // binomialCoeff, src/globals.h:85-102 (same operation order)
  T res = 1;
  if (k > n - k) k = n - k;
  for (T i = 0; i < k; ++i) {
    res *= (n - i);
    res /= (i + 1);
  }
  return res;
}

static const uint64_t* an_solution(uint64_t A, uint32_t n, uint32_t* h) {
  if (A != 641 && A != 61) return nullptr;
  *h = A == 641 ? 10 : 6;
  if (n == 24) return A == 641 ? kAn24A641 : kAn24A61;
  if (n == 16) return A == 641 ? kAn16A641 : kAn16A61;
  if (n == 8) return A == 641 ? kAn8A641 : kAn8A61;
  return nullptr;
}

double rel_error_an(uint64_t A, uint32_t n, const u128* tgt, int offset, double* errors) {
  uint32_t h = 0;
  const uint64_t* sol = an_solution(A, n, &h);
  if (!sol) return -1.0;
  double mx = 0;
  if (errors) std::memset(errors, 0, (n + h + 1) * sizeof(double));
  for (uint32_t k = offset; k < n + h; ++k) {  // src/globals.cpp:117-152
    const double p = (double)sol[k];
    double err;
    if (p > 0.) err = std::fabs((double)tgt[k] / p - 1.0);
    else if (tgt[k] > 0) err = 1.0;
    else err = 0.0;
    if (errors) errors[k] = err;
    if (err > mx) mx = err;
  }
  return mx;
}

double abs_error_an(uint64_t A, uint32_t n, const u128* tgt, int offset, double* errors) {
  uint32_t h = 0;
  const uint64_t* sol = an_solution(A, n, &h);
  if (!sol) return -1.0;
  double mx = 0;
  if (errors) std::memset(errors, 0, (n + h + 1) * sizeof(double));
  for (uint32_t k = offset; k < n + h; ++k) {  // src/globals.cpp:153-183
    const u128 s = sol[k];
    const double p = (double)(s > tgt[k] ? s - tgt[k] : tgt[k] - s);
    const double err = p / (std::pow(2.0, n) * binomial<double>((double)n + h, (double)k));
    if (errors) errors[k] = err;
    if (err > mx) mx = err;
  }
  return mx;
}

// get_sol_hamming, src/globals.cpp:30-63.
static bool sol_hamming(u128* sol, uint32_t n, uint32_t* h_out) {
  const uint64_t* base;
  *h_out = n == 8 ? 5 : (n == 16 || n == 24) ? 6 : 7;
  const uint32_t h = *h_out;
  switch (n) {
    case 8: base = kSolHam8; break;
    case 16: base = kSolHam16; break;
    case 24: base = kSolHam24; break;
    case 32: base = kSolHam32; break;
    default: return false;
  }
  sol[0] = (u128)1 << n;
  sol[1] = (u128)(n + h) * sol[0];
  for (uint32_t i = 3; i < n + h + 1; i += 2) {
    if (i + 1 < n + h + 1) {
      sol[i + 1] = (u128)base[i + 1] << n;
      sol[i] = (u128)(i + 1) * sol[i + 1] + (u128)(n + h - i + 1) * sol[i - 1];
    } else {
      sol[i] = (u128)(n + h - i + 1) * sol[i - 1];
    }
  }
  return true;
}

double rel_error_hamming(uint32_t n, const u128* tgt, int offset, int w1bit, double* errors) {
  u128 sol[kMaxBins + 2];
  for (auto& x : sol) x = 0;
  uint32_t h = 0;
  if (errors) std::memset(errors, 0, (n + h + 1) * sizeof(double));  // h still 0, as the reference
  if (!sol_hamming(sol, n, &h)) return -1.0;
  double mx = 0;
  if (w1bit == 0 && (offset & 1) == 1) offset += 1;
  for (uint32_t k = offset; k < n + h + 1; k += w1bit ? 1 : 2) {
    const double p = (double)sol[k];
    double err;
    if (p > 0.) err = std::fabs((double)tgt[k] / p - 1.0);
    else if (tgt[k] > 0) err = 1.0;
    else err = 0.0;
    if (errors) errors[k] = err;
    if (err > mx) mx = err;
  }
  return mx;
}

double abs_error_hamming(uint32_t n, const u128* tgt, int offset, int w1bit, double* errors) {
  u128 sol[kMaxBins + 2];
  for (auto& x : sol) x = 0;
  uint32_t h = 0;
  if (errors) std::memset(errors, 0, (n + h + 1) * sizeof(double));
  if (!sol_hamming(sol, n, &h)) return -1.0;
  double mx = 0;
  if (w1bit == 0 && (offset & 1) == 1) offset += 1;
  for (uint32_t k = offset; k < n + h + 1; k += w1bit ? 1 : 2) {
    const double p = (double)(sol[k] > tgt[k] ? sol[k] - tgt[k] : tgt[k] - sol[k]);
    const double err = p / (std::pow(2.0, n) * binomial<double>((double)n + h, (double)k));
    if (errors) errors[k] = err;
    if (err > mx) mx = err;
  }
  return mx;
}

// ---------------------------------------------------------------------------
// results-file layout
// ---------------------------------------------------------------------------
std::string bits_string(uint64_t v, uint64_t n) {
  std::string out;
  const uint64_t mask = n >= 64 ? ~0ull : (1ull << n) - 1;
  uint64_t p = n;
  v &= mask;
  for (; v & mask; v <<= 1, --p) out.push_back((char)('0' + ((v & mask) >> (n - 1))));
  for (; p; --p) out.push_back('0');
  return out;
}

static std::ostream& put_u128(std::ostream& os, u128 v) {
  char buf[64];
  char* d = buf + sizeof(buf);
  do { *--d = "0123456789"[(int)(v % 10)]; v /= 10; } while (v);
  os.write(d, buf + sizeof(buf) - d);
  return os;
}

// The stream sequence of process_result (src/globals.cpp:185-231), including
// its sticky precision: setprecision(7) for the error columns (and 12 for huge
// counts) stays in force for every later value in the same stream.
std::string format_table(const u128* counts, const std::vector<StatRow>& stats, uint32_t n, uint32_t h,
                         const double* errors_abs, const double* errors_rel, const std::string& app,
                         long double* total_out) {
  using namespace std;
  stringstream ss;
  const char sep = ',';
  long double total = 0;
  for (uint32_t i = 0; i < n + h + 1; ++i) total += (long double)counts[i];
  long double prob, base1 = pow(2.0, n), base2, base;
  double mxabs = 0, mxrel = 0;
  for (uint32_t i = 0; i < n + h + 1; ++i) {
    base2 = binomial<long double>((long double)(n + h), (long double)i);
    base = base1 * base2;
    prob = counts[i] / base;
    if (n >= 32 && counts[i] > ((u128)1 << 64))
      ss << setw(4) << i << sep << setw(12) << setprecision(12) << (long double)counts[i];
    else
      ss << setw(4) << i << sep << setw(14) << (unsigned long long)counts[i];
    ss << sep << setw(14) << prob << sep << setw(14) << base;
    if (errors_abs) {
      ss << sep << setw(13) << setprecision(7) << errors_abs[i];
      if (errors_abs[i] > mxabs) mxabs = errors_abs[i];
    }
    if (errors_rel) {
      ss << sep << setw(13) << setprecision(7) << errors_rel[i];
      if (errors_rel[i] > mxrel) mxrel = errors_rel[i];
    }
    ss << endl;
  }
  ss << endl << endl;
  for (size_t i = 0; i < stats.size(); ++i)
    ss << i << sep << '"' << stats[i].label << '"' << sep << stats[i].value << sep << stats[i].unit << endl;
  ss << endl << "\"Total\"" << sep << total << endl;
  if (errors_abs) ss << "\"MaxAbsErr\"" << sep << mxabs << endl;
  if (errors_rel) ss << "\"MaxRelErr\"" << sep << mxrel << endl;
  ss << endl;
  ss << app;
  if (total_out) *total_out = total;
  (void)put_u128;
  return ss.str();
}

}  // namespace dd
