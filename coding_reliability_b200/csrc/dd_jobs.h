// dd_jobs.h — the device-side description of histogram work, shared by the
// host planner (dd_host.cu) and the kernels (dd_kernels.cu).
//
// A launch processes a list of Jobs.  Each Job owns a contiguous range of the
// launch's global tile index space [tile_begin, tile_begin + tiles); a warp
// claims one tile at a time from a global counter and accumulates into its own
// shared-memory bins, which it flushes into the Job's 64-bit global bins.
#pragma once
#include <cstdint>

namespace dd {

constexpr int kMaxBins = 64;        // COUNTS_MAX_WIDTH (super_a/src/globals.h:44)
constexpr int kWarpsPerCta = 8;     // 256 threads per CTA; warps work independently
constexpr int kRowsPerLane = 4;     // codewords held in registers per lane
constexpr int kWarpRows = 32 * kRowsPerLane;   // 128 rows per warp tile
constexpr int kTileCols = 1024;     // columns per warp tile
constexpr int kSuper = 1024;        // triangle super-tile side
constexpr int kStrips = kSuper / kWarpRows;    // warp tiles per super tile (8)
constexpr int kMcSamplesPerTile = 256;         // Monte Carlo: samples per lane per tile
constexpr uint64_t kMcMaxRowsPerLane = 64;     // Monte Carlo: codewords per lane per tile (few samples each)

#if defined(__CUDACC__)
#define DD_HOST_DEVICE __host__ __device__
#else
#define DD_HOST_DEVICE
#endif

// Monte Carlo tile shape, shared by the host (tile counts) and the kernel: with
// `spl` samples per codeword to draw, a lane takes one codeword and up to
// kMcSamplesPerTile of its samples, or, when spl is smaller than that, several
// codewords with all their samples, so that every tile holds about
// 32 x kMcSamplesPerTile samples.
DD_HOST_DEVICE inline uint64_t mc_rows_per_lane(uint64_t spl) {
  if (spl >= (uint64_t)kMcSamplesPerTile) return 1;
  const uint64_t r = (uint64_t)kMcSamplesPerTile / (spl ? spl : 1);
  return r < kMcMaxRowsPerLane ? r : kMcMaxRowsPerLane;
}
DD_HOST_DEVICE inline uint64_t mc_chunks(uint64_t spl) {
  return spl >= (uint64_t)kMcSamplesPerTile ? (spl + kMcSamplesPerTile - 1) / kMcSamplesPerTile : 1;
}
constexpr uint32_t kFlushEvery = 1u << 16;     // warp tiles between flushes (uint32 counter bound)

enum JobKind : uint32_t {
  JOB_PAIRS = 0,     // rows x columns distance histogram (exhaustive, grid, Hamming all-pairs)
  JOB_MC = 1,        // AN Monte Carlo: every codeword row x `it` Philox-drawn columns
  JOB_WEIGHTS = 2    // Ext-Hamming weight histogram of generated messages (exhaustive, grid, MC)
};
enum TileShape : uint32_t { SHAPE_TRIANGLE = 0, SHAPE_RECT = 1 };
enum RowKind : uint32_t { ROW_PROGRESSION = 0, ROW_LATTICE = 1, ROW_HAMMING_EXT = 2 };
enum ColKind : uint32_t { COL_PROGRESSION = 0, COL_LATTICE = 1, COL_HAMMING_EXT = 2 };
enum WeightGen : uint32_t { WGEN_ALL = 0, WGEN_GRID = 1, WGEN_MC = 2 };

struct Job {
  unsigned long long* bins;  // global uint64[kMaxBins] (device)
  uint64_t A;                // AN multiplier
  uint64_t rows;             // row items (TRIANGLE: N codewords)
  uint64_t cols;             // column items
  uint64_t tile_begin;       // first global tile index of this job
  uint64_t tiles;            // tiles of this job
  uint64_t col_tiles;        // RECT: column tiles per row tile; TRIANGLE: super tiles per side
  uint64_t seed;             // MC Philox key
  uint64_t iters;            // MC: samples per codeword; WEIGHTS: samples
  double row_step;           // ROW_LATTICE stepsize
  double col_step;           // COL_LATTICE stepsize
  uint32_t n;                // data bits
  uint32_t nbins;            // bins of this job (<= kMaxBins)
  uint32_t kind;             // JobKind
  uint32_t shape;            // TileShape
  uint32_t row_kind;         // RowKind
  uint32_t col_kind;         // ColKind
  uint32_t t32;              // lattice casts go through uint32 (the reference's T)
  uint32_t wide;             // codewords exceed 32 bits
  uint32_t wgen;             // WeightGen
  uint32_t bucket;           // Ext-Hamming template bucket N (8 for n in {4,8})
  uint32_t shard;            // Ext-Hamming grid: Shards<N>
  uint32_t pk_s;             // tcgen05 pair-packed epilogue: S = largest distance + 1, the packed
                             // value of a distance pair (d1, d2) is d1 + S * (d2 - pk_lo)
  uint64_t tile_offset;      // first tile of the instance this job covers (a launch may run a
                             // sub-range [tile_offset, tile_offset + tiles) of the instance)
  uint64_t sample_begin;     // MC: every codeword draws its samples [sample_begin, iters) only
  int32_t pk_lo;             // tcgen05 pair-packed epilogue: first d2 of the joint-bin window
  uint32_t pk_limit;         // tcgen05 pair-packed epilogue: packed values below it are table cells
};

// Status bits a kernel reports back (the word is zeroed before each launch).
enum : uint32_t {
  KSTATUS_TIMEOUT = 1u,       // a bounded wait ran out
  KSTATUS_BAD_DISTANCE = 2u,  // a distance outside the job's bins was produced (and dropped)
  KSTATUS_BAD_JOB = 4u        // a tile mapped outside the job table
};

// One launch: the job table and the shared work counter.
struct LaunchArgs {
  const Job* jobs;
  uint32_t njobs;
  uint32_t smem_bins;        // bin rows reserved per warp in shared memory
  uint64_t total_tiles;
  unsigned long long* counter;  // global work counter (zeroed before launch)
  unsigned* status;          // KSTATUS_* bits
  uint32_t use_col_table;    // reserve a per-warp column table
  uint32_t pad;
};

}  // namespace dd
