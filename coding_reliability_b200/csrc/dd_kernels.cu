// dd_kernels.cu — the popc-path histogram kernels (sm_100a).
//
// One persistent kernel serves every job kind.  Each warp is an independent
// worker: it claims a tile from a global counter, accumulates distances into
// its own shared-memory bins (one uint32 column per lane, so increments never
// collide), and flushes those bins warp-aggregated into the job's uint64
// global bins when it moves to another job, every kFlushEvery tiles, and at
// exit.  Codewords are generated in registers (A*x, lattice points, Hamming
// parity), never read from HBM.
//
// Reference kernels this replaces (all plain SIMT, written for sm_35):
//   dancoding_shared        distance_distribution/src/an_coding.cu:50-105
//   dancoding_grid_1d_shared                       src/an_coding_grid.cu:60-114
//   dancoding_grid_2d                              src/an_coding_grid.cu:121-140
//   dancoding_mc_shared                            src/an_coding_mc.cu:94-158
//   dhamming / dhamming_grid_1d / dhamming_mc      src/hamming.cu:64-81, hamming_grid.cu:53-74,
//                                                  hamming_mc.cu:57-81
//   super-A dancoding_shared / dancoding           distance_distribution_super_a/src/an_coding.cu:32-99
#include <cuda_runtime.h>
#include <cstdint>

#include "dd_device.cuh"
#include "dd_jobs.h"
#include "dd_kernels.h"

namespace dd {

// ---------------------------------------------------------------------------
// shared-memory bin increments
// ---------------------------------------------------------------------------
#ifdef DD_SELF_CHECK
// Self-checking build (libcodrel_b200_checked.so): every bin access is range
// checked against the calling warp's shared-memory region; a violation is
// recorded (first one wins) and the access is skipped.
struct CheckState {
  uint32_t lo, hi;            // this warp's bin region [lo, hi) in the shared window
  unsigned* status;
  unsigned long long* record;  // [0] flag, [1] offset, [2] lo, [3] hi, [4] tile
  unsigned long long tile;
};
__device__ __forceinline__ CheckState& check_state() {
  __shared__ CheckState st[kWarpsPerCta];
  return st[threadIdx.x >> 5];
}
#endif

template <int kMode>
__device__ __forceinline__ void bump(uint32_t saddr) {
#ifdef DD_SELF_CHECK
  {
    CheckState& cs = check_state();
    if (saddr < cs.lo || saddr + 4 > cs.hi || (saddr & 3)) {
      atomicOr(cs.status, 8u);
      if (atomicCAS(cs.record, 0ull, 1ull) == 0ull) {
        cs.record[1] = saddr; cs.record[2] = cs.lo; cs.record[3] = cs.hi; cs.record[4] = cs.tile;
      }
      return;
    }
  }
#endif
  if constexpr (kMode == HIST_RED) {
    asm volatile("red.shared.add.u32 [%0], 1;" ::"r"(saddr) : "memory");
  } else {
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(saddr) : "memory");
    asm volatile("st.shared.u32 [%0], %1;" ::"r"(saddr), "r"(v + 1) : "memory");
  }
}

// Bump for the generic paths: the bin index is checked against the job's bin
// count; an out-of-range distance is dropped and reported in the status word.
template <int kMode>
__device__ __forceinline__ void bump_checked(uint32_t lane_base, uint32_t d, uint32_t nbins, unsigned* status) {
  if (d < nbins) bump<kMode>(lane_base + (d << 7));
  else atomicOr(status, KSTATUS_BAD_DISTANCE);
}

// Warp-aggregated flush: lane l sums bin rows l and l+32 over the 32 lane
// columns (rotated so the 32 lanes hit 32 different banks), zeroes them and
// adds the 64-bit sums to the global bins.
__device__ __forceinline__ void flush_bins(uint32_t* wbins, unsigned long long* gbins, uint32_t nbins, int lane) {
  __syncwarp();
  for (uint32_t b = lane; b < nbins; b += 32) {
    unsigned long long s = 0;
#pragma unroll 8
    for (int k = 0; k < 32; ++k) {
      const int kk = (k + lane) & 31;
      s += wbins[b * 32 + kk];
      wbins[b * 32 + kk] = 0;
    }
    if (s) atomicAdd(gbins + b, s);
  }
  __syncwarp();
}

// ---------------------------------------------------------------------------
// generators
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t row_value(const Job& J, uint64_t i) {
  switch (J.row_kind) {
    case ROW_LATTICE: return lattice_value(J.A, i, J.row_step, J.t32);
    case ROW_HAMMING_EXT: return hamming_cw_ext(i, J.n);
    default: return J.A * i;
  }
}

__device__ __forceinline__ uint64_t col_value(const Job& J, uint64_t j) {
  switch (J.col_kind) {
    case COL_LATTICE: return lattice_value(J.A, j, J.col_step, J.t32);
    case COL_HAMMING_EXT: return hamming_cw_ext(j, J.n);
    default: return J.A * j;
  }
}

// ---------------------------------------------------------------------------
// pair tiles
// ---------------------------------------------------------------------------

// Fast path: 32 lanes x kRowsPerLane valid rows, columns [c, ce) an arithmetic
// progression v = A*j with warp-uniform v; `off[q]` is the shared address of
// lane's bin 0 for row q, already shifted by the high-word distance.
template <int kMode>
__device__ __forceinline__ void run_progression(const uint32_t (&w)[kRowsPerLane], const uint32_t (&off)[kRowsPerLane],
                                                uint32_t v, uint32_t a, uint32_t count) {
  uint32_t j = 0;
  for (; j + 8 <= count; j += 8) {
#pragma unroll
    for (int u = 0; u < 8; ++u) {
#pragma unroll
      for (int q = 0; q < kRowsPerLane; ++q) bump<kMode>(off[q] + (__popc(w[q] ^ v) << 7));
      v += a;
    }
  }
  for (; j < count; ++j) {
#pragma unroll
    for (int q = 0; q < kRowsPerLane; ++q) bump<kMode>(off[q] + (__popc(w[q] ^ v) << 7));
    v += a;
  }
}

// Columns read from a per-warp table in shared memory (Ext-Hamming codewords).
template <int kMode>
__device__ __forceinline__ void run_table(const uint32_t (&w)[kRowsPerLane], const uint32_t (&off)[kRowsPerLane],
                                          const uint32_t* table, uint32_t count) {
  uint32_t j = 0;
  for (; j + 4 <= count; j += 4) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint32_t v = table[j + u];
#pragma unroll
      for (int q = 0; q < kRowsPerLane; ++q) bump<kMode>(off[q] + (__popc(w[q] ^ v) << 7));
    }
  }
  for (; j < count; ++j) {
    const uint32_t v = table[j];
#pragma unroll
    for (int q = 0; q < kRowsPerLane; ++q) bump<kMode>(off[q] + (__popc(w[q] ^ v) << 7));
  }
}

// Slow path for diagonal and partial tiles and for generic 64-bit columns:
// every pair checked, 64-bit popcount.
template <int kMode>
__device__ __forceinline__ void run_generic(const Job& J, const uint64_t (&w)[kRowsPerLane],
                                            const uint64_t (&ri)[kRowsPerLane], const bool (&rv)[kRowsPerLane],
                                            uint32_t lane_base, uint64_t c0, uint64_t c1, bool diag,
                                            unsigned* status) {
  for (uint64_t j = c0; j < c1; ++j) {
    const uint64_t v = col_value(J, j);
#pragma unroll
    for (int q = 0; q < kRowsPerLane; ++q)
      if (rv[q] && (!diag || j > ri[q])) bump_checked<kMode>(lane_base, popc64(w[q] ^ v), J.nbins, status);
  }
}

template <int kMode>
__device__ void pairs_tile(const Job& J, uint64_t lt, uint32_t* wbins, uint32_t* table, int lane, unsigned* status) {
  uint64_t r0, c0, c1;
  bool diag = false;
  if (J.shape == SHAPE_TRIANGLE) {
    const uint64_t s = lt / kStrips;
    const uint32_t strip = (uint32_t)(lt % kStrips);
    uint64_t sr, sc;
    tri_decode(s, J.col_tiles, sr, sc);
    r0 = sr * kSuper + (uint64_t)strip * kWarpRows;
    c0 = sc * kSuper;
    c1 = c0 + kSuper < J.cols ? c0 + kSuper : J.cols;
    diag = (sr == sc);
  } else {
    static_assert(kWarpRows == 128 && kTileCols == 1024, "rect_decode's tile shape");
    rect_decode(lt, (J.rows + kWarpRows - 1) / kWarpRows, r0, c0);
    c1 = c0 + kTileCols < J.cols ? c0 + kTileCols : J.cols;
  }
  if (r0 >= J.rows) return;

  uint64_t w[kRowsPerLane], ri[kRowsPerLane];
  bool rv[kRowsPerLane];
  bool all_valid = true;
#pragma unroll
  for (int q = 0; q < kRowsPerLane; ++q) {
    ri[q] = r0 + (uint64_t)q * 32 + lane;
    rv[q] = ri[q] < J.rows;
    all_valid &= rv[q];
    w[q] = rv[q] ? row_value(J, ri[q]) : 0;
  }
  all_valid = __all_sync(0xffffffffu, all_valid);
  const uint32_t lane_base = (uint32_t)__cvta_generic_to_shared(wbins) + (uint32_t)lane * 4u;

  // Diagonal tile: columns <= r0 pair with no row; (r0, r0+kWarpRows) need the
  // j > i mask; the rest is a full rectangle.
  uint64_t cf = c0;
  if (diag) {
    const uint64_t mlo = r0 + 1 > c0 ? r0 + 1 : c0;
    const uint64_t mhi = r0 + kWarpRows < c1 ? r0 + kWarpRows : c1;
    if (mlo < mhi) run_generic<kMode>(J, w, ri, rv, lane_base, mlo, mhi, true, status);
    cf = mhi > mlo ? mhi : mlo;
    if (cf < c0) cf = c0;
  }
  if (cf >= c1) return;

  // The unchecked fast paths need every distance of the tile below nbins: the
  // widest row or column codeword of the tile must have at most nbins-1 bits.
  uint32_t wbits = 0;
#pragma unroll
  for (int q = 0; q < kRowsPerLane; ++q) wbits = max(wbits, 64u - (uint32_t)__clzll((long long)w[q]));
  wbits = __reduce_max_sync(0xffffffffu, wbits);
  if (J.col_kind == COL_PROGRESSION) wbits = max(wbits, 64u - (uint32_t)__clzll((long long)(J.A * (c1 - 1))));
  const bool fits = wbits < J.nbins;

  if (!all_valid || !fits || J.col_kind == COL_LATTICE || (J.wide && J.col_kind != COL_PROGRESSION) ||
      (J.col_kind == COL_PROGRESSION && J.wide && (J.A >> 32))) {
    run_generic<kMode>(J, w, ri, rv, lane_base, cf, c1, false, status);
    return;
  }

  uint32_t wl[kRowsPerLane], off[kRowsPerLane];
#pragma unroll
  for (int q = 0; q < kRowsPerLane; ++q) wl[q] = (uint32_t)w[q];

  if (J.col_kind == COL_HAMMING_EXT) {
    const uint32_t cnt = (uint32_t)(c1 - cf);
    for (uint32_t jj = lane; jj < cnt; jj += 32) table[jj] = (uint32_t)hamming_cw_ext(cf + jj, J.n);
    __syncwarp();
#pragma unroll
    for (int q = 0; q < kRowsPerLane; ++q) off[q] = lane_base;
    run_table<kMode>(wl, off, table, cnt);
    __syncwarp();
    return;
  }

  const uint32_t a = (uint32_t)J.A;
  if (!J.wide) {
#pragma unroll
    for (int q = 0; q < kRowsPerLane; ++q) off[q] = lane_base;
    run_progression<kMode>(wl, off, (uint32_t)(J.A * cf), a, (uint32_t)(c1 - cf));
    return;
  }
  // Wide codewords: split the columns where the high word of A*j changes, so
  // that each segment needs one 32-bit popcount per pair; the high-word
  // distance of row q is folded into its bin offset.
  uint32_t wh[kRowsPerLane];
#pragma unroll
  for (int q = 0; q < kRowsPerLane; ++q) wh[q] = (uint32_t)(w[q] >> 32);
  uint64_t j = cf;
  uint64_t v = J.A * j;
  while (j < c1) {
    const uint32_t vl = (uint32_t)v, vh = (uint32_t)(v >> 32);
    const uint64_t to_wrap = ((1ull << 32) - vl + a - 1) / a;
    const uint64_t je = j + to_wrap < c1 ? j + to_wrap : c1;
#pragma unroll
    for (int q = 0; q < kRowsPerLane; ++q) off[q] = lane_base + (__popc(wh[q] ^ vh) << 7);
    run_progression<kMode>(wl, off, vl, a, (uint32_t)(je - j));
    v += J.A * (je - j);
    j = je;
  }
}

// ---------------------------------------------------------------------------
// Monte Carlo tiles (shape: mc_rows_per_lane / mc_chunks in dd_jobs.h).
//
// The samples of a lane are independent, so the fast loops draw several Philox
// blocks before they bin anything: the bins are bumped by volatile asm, which
// the compiler does not move computations across, and one block at a time
// would leave the ten-round multiply chain of each block exposed.
// ---------------------------------------------------------------------------
constexpr int kMcBlocksPerStep = 4;

// Many samples per codeword: one codeword per lane, up to kMcSamplesPerTile of
// its samples, drawn kMcBlocksPerStep Philox blocks at a time.
template <int kMode>
__device__ __forceinline__ void mc_many(const Job& J, uint64_t i, uint64_t t, uint64_t t1, uint32_t lane_base,
                                        unsigned* status) {
  const uint64_t w = J.A * i;
  const uint32_t k0 = (uint32_t)J.seed, k1 = (uint32_t)(J.seed >> 32);
  const uint32_t i0 = (uint32_t)i, i1 = (uint32_t)(i >> 32);
  if (J.n <= 32) {
    // four 32-bit samples per block (counter (t >> 2, i)); index = top n bits
    const unsigned sh = 32 - J.n;
    const uint32_t wl = (uint32_t)w;
    const uint32_t a = (uint32_t)J.A;  // A < 2^32
    const bool wide = J.wide != 0;
    // up to the next block boundary (a continued run may start inside a block)
    for (; t < t1 && (t & 3); ++t) {
      const uint64_t v = J.A * mc_index(J.seed, i, t, J.n);
      bump_checked<kMode>(lane_base, popc64(w ^ v), J.nbins, status);
    }
    constexpr int kS = 4 * kMcBlocksPerStep;
    for (; t + kS <= t1; t += kS) {
      uint32_t r[kS], d[kS];
#pragma unroll
      for (int b = 0; b < kMcBlocksPerStep; ++b) {
        const uint64_t blk = (t >> 2) + b;
        const Philox4 o = philox4x32_10((uint32_t)blk, (uint32_t)(blk >> 32), i0, i1, k0, k1);
        r[4 * b] = o.x; r[4 * b + 1] = o.y; r[4 * b + 2] = o.z; r[4 * b + 3] = o.w;
      }
      if (wide) {
#pragma unroll
        for (int u = 0; u < kS; ++u) d[u] = popc64(w ^ ((uint64_t)a * (r[u] >> sh)));
      } else {
#pragma unroll
        for (int u = 0; u < kS; ++u) d[u] = __popc(wl ^ (a * (r[u] >> sh)));
      }
#pragma unroll
      for (int u = 0; u < kS; ++u) bump_checked<kMode>(lane_base, d[u], J.nbins, status);
    }
  } else {
    // two 64-bit samples per block (counter (t >> 1, i)); index = top n bits
    const unsigned sh = 64 - J.n;
    if (t < t1 && (t & 1)) {
      const uint64_t v = J.A * mc_index(J.seed, i, t, J.n);
      bump_checked<kMode>(lane_base, popc64(w ^ v), J.nbins, status);
      ++t;
    }
    constexpr int kS = 2 * kMcBlocksPerStep;
    for (; t + kS <= t1; t += kS) {
      uint64_t r[kS];
      uint32_t d[kS];
#pragma unroll
      for (int b = 0; b < kMcBlocksPerStep; ++b) {
        const uint64_t blk = (t >> 1) + b;
        const Philox4 o = philox4x32_10((uint32_t)blk, (uint32_t)(blk >> 32), i0, i1, k0, k1);
        r[2 * b] = ((uint64_t)o.x << 32) | o.y;
        r[2 * b + 1] = ((uint64_t)o.z << 32) | o.w;
      }
#pragma unroll
      for (int u = 0; u < kS; ++u) d[u] = popc64(w ^ ((uint64_t)(uint32_t)J.A * (r[u] >> sh)));
#pragma unroll
      for (int u = 0; u < kS; ++u) bump_checked<kMode>(lane_base, d[u], J.nbins, status);
    }
  }
  for (; t < t1; ++t) {
    const uint64_t v = J.A * mc_index(J.seed, i, t, J.n);
    bump_checked<kMode>(lane_base, popc64(w ^ v), J.nbins, status);
  }
}

// Few samples per codeword (fewer than kMcSamplesPerTile): each lane takes
// several codewords with all of their samples, one Philox block at a time.
template <int kMode>
__device__ __noinline__ void mc_few(uint64_t A, uint64_t seed, uint32_t n, uint32_t nbins, uint64_t i, uint64_t t,
                                    uint64_t t1, uint32_t lane_base, unsigned* status) {
  const uint64_t w = A * i;
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  const uint32_t i0 = (uint32_t)i, i1 = (uint32_t)(i >> 32);
  const uint64_t a = (uint32_t)A;  // A < 2^32
  const unsigned per_block = n <= 32 ? 4u : 2u;
  for (; t < t1 && (t & (per_block - 1)); ++t)
    bump_checked<kMode>(lane_base, popc64(w ^ (A * mc_index(seed, i, t, n))), nbins, status);
  for (; t + per_block <= t1; t += per_block) {
    const uint64_t blk = t / per_block;
    const Philox4 o = philox4x32_10((uint32_t)blk, (uint32_t)(blk >> 32), i0, i1, k0, k1);
    if (per_block == 4) {
      const unsigned sh = 32 - n;
      const uint32_t d0 = popc64(w ^ (a * (o.x >> sh))), d1 = popc64(w ^ (a * (o.y >> sh)));
      const uint32_t d2 = popc64(w ^ (a * (o.z >> sh))), d3 = popc64(w ^ (a * (o.w >> sh)));
      bump_checked<kMode>(lane_base, d0, nbins, status);
      bump_checked<kMode>(lane_base, d1, nbins, status);
      bump_checked<kMode>(lane_base, d2, nbins, status);
      bump_checked<kMode>(lane_base, d3, nbins, status);
    } else {
      const unsigned sh = 64 - n;
      const uint32_t d0 = popc64(w ^ (a * ((((uint64_t)o.x << 32) | o.y) >> sh)));
      const uint32_t d1 = popc64(w ^ (a * ((((uint64_t)o.z << 32) | o.w) >> sh)));
      bump_checked<kMode>(lane_base, d0, nbins, status);
      bump_checked<kMode>(lane_base, d1, nbins, status);
    }
  }
  for (; t < t1; ++t) bump_checked<kMode>(lane_base, popc64(w ^ (A * mc_index(seed, i, t, n))), nbins, status);
}

template <int kMode>
__device__ void mc_tile(const Job& J, uint64_t lt, uint32_t* wbins, int lane, unsigned* status) {
  const uint64_t spl = J.iters - J.sample_begin;
  const uint64_t rpl = mc_rows_per_lane(spl), chunks = mc_chunks(spl);
  const uint64_t rt = lt / chunks, ch = lt % chunks;
  const uint64_t t0 = J.sample_begin + ch * kMcSamplesPerTile;
  const uint64_t t1 = t0 + kMcSamplesPerTile < J.iters ? t0 + kMcSamplesPerTile : J.iters;
  const uint32_t lane_base = (uint32_t)__cvta_generic_to_shared(wbins) + (uint32_t)lane * 4u;
  if (rpl == 1) {
    const uint64_t i = rt * 32 + lane;
    if (i < J.rows) mc_many<kMode>(J, i, t0, t1, lane_base, status);
    return;
  }
  for (uint64_t r = 0; r < rpl; ++r) {
    const uint64_t i = (rt * rpl + r) * 32 + lane;
    if (i >= J.rows) return;
    mc_few<kMode>(J.A, J.seed, J.n, J.nbins, i, t0, t1, lane_base, status);
  }
}

// ---------------------------------------------------------------------------
// Ext-Hamming weight tiles: 32 lanes x 256 generated messages.
// ---------------------------------------------------------------------------
template <int kMode>
__device__ void weights_tile(const Job& J, uint64_t lt, uint32_t* wbins, int lane, unsigned* status) {
  const uint32_t lane_base = (uint32_t)__cvta_generic_to_shared(wbins) + (uint32_t)lane * 4u;
  const uint64_t g0 = lt * (32ull * 256ull);
#pragma unroll 4
  for (uint32_t k = 0; k < 256; ++k) {
    const uint64_t g = g0 + (uint64_t)k * 32 + lane;
    if (g >= J.iters) break;
    uint64_t x;
    bool n4 = false;
    if (J.wgen == WGEN_GRID) {
      const uint64_t sh = g / J.shard, kk = g % J.shard;
      const uint64_t wsh = sh * J.shard * (uint64_t)J.row_step;
      x = (uint64_t)fma((double)kk, J.row_step, (double)wsh);
    } else if (J.wgen == WGEN_MC) {
      x = mc_index(J.seed, 0, g, J.bucket);
    } else {
      x = g;
      n4 = true;
    }
    bump_checked<kMode>(lane_base, popc64(hamming_cw_gpu(x, J.bucket, n4)), J.nbins, status);
  }
}

// ---------------------------------------------------------------------------
// the persistent kernel
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t find_job(const Job* jobs, uint32_t njobs, uint64_t t) {
  uint32_t lo = 0, hi = njobs - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (__ldg(&jobs[mid].tile_begin) <= t) lo = mid; else hi = mid - 1;
  }
  return lo;
}

template <int kMode>
__global__ void __launch_bounds__(kWarpsPerCta * 32) hist_kernel(LaunchArgs args) {
  extern __shared__ __align__(16) uint32_t smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t per_warp = args.smem_bins * 32 + (args.use_col_table ? kTileCols : 0);
  uint32_t* wbins = smem + warp * per_warp;
  uint32_t* table = wbins + args.smem_bins * 32;
  for (uint32_t k = lane; k < args.smem_bins * 32; k += 32) wbins[k] = 0;
#ifdef DD_SELF_CHECK
  if (lane == 0) {
    CheckState& cs = check_state();
    cs.lo = (uint32_t)__cvta_generic_to_shared(wbins);
    cs.hi = cs.lo + args.smem_bins * 32 * 4;
    cs.status = args.status;
    cs.record = reinterpret_cast<unsigned long long*>(args.status) + 1;
    cs.tile = 0;
  }
#endif
  __syncwarp();

  uint32_t cur = 0xffffffffu;
  uint32_t since_flush = 0;
  Job J;
  for (;;) {
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(args.counter, 1ull);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= args.total_tiles) break;
    const uint32_t jn = find_job(args.jobs, args.njobs, t);
    if (jn >= args.njobs || t < args.jobs[jn].tile_begin ||
        t - args.jobs[jn].tile_begin >= args.jobs[jn].tiles || args.jobs[jn].nbins > args.smem_bins) {
      if (lane == 0) atomicOr(args.status, KSTATUS_BAD_JOB);
      continue;
    }
    if (jn != cur) {
      if (cur != 0xffffffffu && since_flush) flush_bins(wbins, J.bins, J.nbins, lane);
      since_flush = 0;
      J = args.jobs[jn];
      cur = jn;
    }
    const uint64_t lt = t - J.tile_begin + J.tile_offset;
#ifdef DD_SELF_CHECK
    if (lane == 0) check_state().tile = t;
    __syncwarp();
#endif
    if (J.kind == JOB_PAIRS) pairs_tile<kMode>(J, lt, wbins, table, lane, args.status);
    else if (J.kind == JOB_MC) mc_tile<kMode>(J, lt, wbins, lane, args.status);
    else weights_tile<kMode>(J, lt, wbins, lane, args.status);
    if (++since_flush >= kFlushEvery) { flush_bins(wbins, J.bins, J.nbins, lane); since_flush = 0; }
  }
  if (cur != 0xffffffffu && since_flush) flush_bins(wbins, J.bins, J.nbins, lane);
}

// ---------------------------------------------------------------------------
// The plain baseline: one launch per instance, one codeword row per thread in
// a grid-stride loop, every j > i in an inner loop, a per-thread column of
// shared-memory bins bumped by load/add/store, and one 64-bit atomic per bin
// and thread at the end.  This is the straightforward SIMT design the
// reference uses (dancoding_shared, src/an_coding.cu:50-105), kept as the
// comparison point for the persistent and batched paths.
// ---------------------------------------------------------------------------
constexpr int kPlainThreads = 128;

__global__ void __launch_bounds__(kPlainThreads) plain_an_kernel(uint64_t A, uint64_t N, uint32_t nbins,
                                                                 unsigned long long* bins) {
  extern __shared__ uint32_t cnt[];  // nbins x kPlainThreads
  for (uint32_t k = threadIdx.x; k < nbins * kPlainThreads; k += kPlainThreads) cnt[k] = 0;
  __syncthreads();
  uint32_t* mine = cnt + threadIdx.x;
  for (uint64_t i = (uint64_t)blockIdx.x * kPlainThreads + threadIdx.x; i < N;
       i += (uint64_t)gridDim.x * kPlainThreads) {
    const uint64_t w = A * i;
    for (uint64_t j = i + 1, v = w + A; j < N; ++j, v += A) {
      const uint32_t d = popc64(w ^ v);
      if (d < nbins) mine[d * kPlainThreads] += 1;
    }
  }
  __syncthreads();
  for (uint32_t b = 0; b < nbins; ++b)
    if (mine[b * kPlainThreads]) atomicAdd(bins + b, (unsigned long long)mine[b * kPlainThreads]);
}

cudaError_t launch_plain(uint64_t A, uint64_t N, uint32_t nbins, unsigned long long* bins, int grid,
                         cudaStream_t stream) {
  plain_an_kernel<<<grid, kPlainThreads, (size_t)nbins * kPlainThreads * sizeof(uint32_t), stream>>>(A, N, nbins,
                                                                                                   bins);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// POPC issue-rate probe: 8 independent popc chains per thread.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) popc_rate_kernel(uint32_t iters, uint32_t seed, uint32_t* sink) {
  uint32_t x0 = seed ^ threadIdx.x, x1 = x0 * 3u + 1, x2 = x0 * 5u + 2, x3 = x0 * 7u + 3;
  uint32_t x4 = x0 * 9u + 4, x5 = x0 * 11u + 5, x6 = x0 * 13u + 6, x7 = x0 * 15u + 7;
  for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      x0 += __popc(x0); x1 += __popc(x1); x2 += __popc(x2); x3 += __popc(x3);
      x4 += __popc(x4); x5 += __popc(x5); x6 += __popc(x6); x7 += __popc(x7);
    }
  }
  const uint32_t r = x0 ^ x1 ^ x2 ^ x3 ^ x4 ^ x5 ^ x6 ^ x7;
  if (r == 0x12345678u) sink[blockIdx.x] = r;
}

// Shared-memory atomic rate, measured the way the tcgen05 kernel's epilogues
// use the pipe: one CTA per SM of blockDim.x threads, every thread adding 1 in
// a 128 KB table, 32 independent adds per loop iteration to addresses held in
// registers (so no address arithmetic limits the rate), conflict-free within
// each warp (the 32 lanes always hit 32 banks).
//   kRedPerThread: every thread its own column of 32 rows (row stride
//                  blockDim.x words), a different row for each of its 32 adds
//                  (the single epilogue's per-thread bins);
//   kRedLaneShared: one column per lane shared by every warp of the CTA, 1024
//                  cells, 32 cells per thread spread like distances around the
//                  middle of the table and differing between warps (the paired
//                  epilogue's joint table).
constexpr int kRedRows = 32;
constexpr uint32_t kRedCells = 1024;
enum RedPattern : int { kRedPerThread = 0, kRedLaneShared = 1 };

template <int kPattern>
__global__ void __launch_bounds__(1024, 1) red_rate_kernel(uint32_t iters, uint32_t* sink) {
  extern __shared__ uint32_t tab[];
  const uint32_t nthr = blockDim.x, tid = threadIdx.x, lane = tid & 31;
  const uint32_t words = kPattern == kRedPerThread ? kRedRows * nthr : kRedCells * 32u;
  for (uint32_t k = tid; k < words; k += nthr) tab[k] = 0;
  __syncthreads();
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(tab);
  uint32_t a[32];
#pragma unroll
  for (uint32_t u = 0; u < 32; ++u) {
    if constexpr (kPattern == kRedPerThread) {
      a[u] = sbase + tid * 4u + ((u * 7u) & (kRedRows - 1)) * nthr * 4u;
    } else {
      // two 16-bit popcounts of a hash: a binomial-like cell around 512
      uint32_t h = (tid * 32u + u) * 0x9E3779B1u;
      h ^= h >> 15;
      h *= 0x85EBCA77u;
      h ^= h >> 13;
      const uint32_t cell = (__popc(h & 0xFFFFu) + __popc(h >> 16)) * 31u;  // [0, 32 * 31] < kRedCells
      a[u] = sbase + lane * 4u + cell * 128u;
    }
  }
  for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
    for (uint32_t u = 0; u < 32; ++u) asm volatile("red.shared.add.u32 [%0], 1;" ::"r"(a[u]) : "memory");
  }
  __syncthreads();
  uint32_t s = 0;
  for (uint32_t k = tid; k < words; k += nthr) s += tab[k];
  if (s == 0x9E3779B9u) sink[blockIdx.x] = s;  // keeps the adds alive (the value is irrelevant)
}

// ---------------------------------------------------------------------------
// host-callable launchers
// ---------------------------------------------------------------------------
size_t hist_smem_bytes(uint32_t smem_bins, bool col_table) {
  return (size_t)kWarpsPerCta * ((size_t)smem_bins * 32 + (col_table ? kTileCols : 0)) * sizeof(uint32_t);
}

static const void* kernel_ptr(int mode) {
  return mode == HIST_RED ? (const void*)hist_kernel<HIST_RED> : (const void*)hist_kernel<HIST_LDST>;
}

// The dynamic shared-memory limit of hist_kernel is a per-function attribute
// shared by every host thread, so every caller sets the same value: the largest
// any plan asks for (kMaxBins bin rows and the column table).  A per-launch
// value could be lowered by one thread between another's set and launch.
static cudaError_t hist_smem_limit(int mode, size_t smem) {
  const size_t limit = hist_smem_bytes(kMaxBins, true);
  if (smem > limit) return cudaErrorInvalidValue;
  return cudaFuncSetAttribute(kernel_ptr(mode), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)limit);
}

cudaError_t hist_occupancy(int mode, size_t smem, int* ctas_per_sm) {
  cudaError_t e = hist_smem_limit(mode, smem);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, kernel_ptr(mode), kWarpsPerCta * 32, smem);
}

cudaError_t launch_hist(int mode, const LaunchArgs& args, int grid, size_t smem, cudaStream_t stream) {
  cudaError_t e = hist_smem_limit(mode, smem);
  if (e != cudaSuccess) return e;
  if (mode == HIST_RED)
    hist_kernel<HIST_RED><<<grid, kWarpsPerCta * 32, smem, stream>>>(args);
  else
    hist_kernel<HIST_LDST><<<grid, kWarpsPerCta * 32, smem, stream>>>(args);
  return cudaGetLastError();
}

cudaError_t launch_popc_rate(uint32_t iters, int grid, uint32_t* sink, cudaStream_t stream) {
  popc_rate_kernel<<<grid, 256, 0, stream>>>(iters, 0x9e3779b9u, sink);
  return cudaGetLastError();
}

// One CTA per SM: the tables need 128 KB, the launch asks for more than half an SM.
cudaError_t launch_red_rate(uint32_t iters, int grid, int threads, int pattern, uint32_t* sink, cudaStream_t stream) {
  const int smem = 132 * 1024;
  if (threads < 32 || threads > 1024 || threads % 32) return cudaErrorInvalidValue;
  const void* fn = pattern == kRedLaneShared ? (const void*)red_rate_kernel<kRedLaneShared>
                                             : (const void*)red_rate_kernel<kRedPerThread>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  if (pattern == kRedLaneShared)
    red_rate_kernel<kRedLaneShared><<<grid, threads, smem, stream>>>(iters, sink);
  else
    red_rate_kernel<kRedPerThread><<<grid, threads, smem, stream>>>(iters, sink);
  return cudaGetLastError();
}
uint64_t red_rate_adds(uint32_t iters, int grid, int threads) { return (uint64_t)grid * threads * iters * 32u; }

}  // namespace dd
