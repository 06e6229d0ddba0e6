// dd_mma.cu — tcgen05 kind::i8 bit-plane MMA kernel: AN exhaustive, 1-D / 2-D
// grid and Ext-Hamming all-pairs jobs.
//
// The Hamming distance of two codewords x, y (bit planes b_x, b_y in {0,1}^L)
// is d = popc(x) + popc(y) - 2<b_x, b_y>.  The operands put that whole
// expression into one int8 GEMM with K = 64.  Two epilogue variants:
//
// Single (one distance per MMA column):
//   A row i    (codeword x_i): bytes k<L: -2*b_ik;  byte L: popc(x_i);  byte L+1: 1
//   B column j (codeword y_j): bytes k<L:    b_jk;  byte L: 1;          byte L+1: popc(y_j)
// so the INT32 accumulator D[i][j] is exactly d(i, j); the epilogue bumps one
// shared-memory bin per pair (per-thread bin columns).
//
// Pair-packed (two distances per MMA column): column p carries two codewords y
// and y' (the adjacent columns 2p and 2p + 1 of the strip), with S = largest
// distance + 1:
//   A row i:    bytes k<L: -2*b_ik;            byte L: popc(x_i); byte L+1: S;              byte L+2: 1
//   B column p: bytes k<L: b_yk + S*b_y'k;     byte L: 1 + S;     byte L+1: popc(y') - lo;  byte L+2: popc(y)
// so D[i][p] = d(x_i, y) + S*(d(x_i, y') - lo), every byte within int8.  That
// value is directly the cell of a joint (d1, d2) table whenever d2 lies in the
// job's window [lo, lo + rows): the table holds as many whole rows of S cells as
// fit in shared memory (mma_pk_layout), and the host places the window on the
// job's distance distribution (mma_pack_setup).  One shared-memory atomic then
// counts two pairs.  The unsigned maximum of 32 values against S * rows shows
// at once whether any lies outside the window (a d2 below it gives a negative,
// i.e. huge, value); only then are the values checked one by one and the
// outliers counted as two single distances in a fallback row.  A job whose
// window holds every d2 (lo = 0, rows = S) skips the test.  The table has one
// column per lane, shared by all epilogue warps, and is folded into the job's
// bins (row sums for d2, column sums for d1) when the job changes, every
// kPkFlushTiles tiles and at exit, between two bounded epilogue-wide barriers.
// It also halves the MMAs, tensor-memory loads and column-operand bytes per
// pair.
//
// Work unit: the popc kernel's tile space (1024x1024 super tiles of the i<j
// triangle, column by column, split into 8 strips of 128 rows; for grid jobs,
// 128 lattice rows x 1024 columns, column tile by column tile; tri_decode and
// rect_decode in dd_device.cuh).  A strip is 128 rows (UMMA M) x
// 1024 columns = 4 MMA tiles of N = 256 (single) or 2 tiles of N = 256 packed
// columns, accumulated in two TMEM buffers of 256 columns: the MMA of tile t+1
// runs while the epilogue bins tile t.  (Four buffers of N = 128 measured 17 %
// slower for the single epilogue: every tile costs each epilogue warp a barrier
// poll and an arrive through the shared-memory pipe that its atomics saturate,
// so fewer, wider tiles win over deeper buffering.)  Generator warps claim 32
// strips at a time (four super tiles when the job's tile range is aligned,
// which in the column-by-column order mostly share one column) and write the
// column operand only when the column super tile changes, into the second of
// two buffers when both fit beside the bins, so the next operand is written
// while the current one's MMAs run; the row operand is double-buffered by
// strip.  One CTA per SM (16 epilogue warps, 1 issuer warp, 3 generator
// warps, 512 TMEM columns).
//
// The single epilogue is bound by the shared-memory atomic rate (one
// red.shared per pair; about 31 per clock per SM measured on B200), twice the
// POPC issue rate (16 per clock per SM) that bounds the popc kernel; the
// pair-packed epilogue needs one atomic per two pairs.  A waiting epilogue warp
// pauses between its barrier polls, which share that pipe with the atomics.
//
// Every mbarrier wait is bounded (MmaArgs::timeout_ns); on expiry the CTA
// records KSTATUS_TIMEOUT, every other wait gives up, the last MMA drains
// (bounded) and the TMEM is released.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdint>

#include "dd_device.cuh"
#include "dd_jobs.h"
#include "dd_mma.h"

namespace dd {

namespace {

constexpr int kEpiWarps = 16;                          // epilogue warps
constexpr int kEpiThreads = kEpiWarps * 32;            // 512: bin columns per bin row
constexpr int kIssuerWarp = kEpiWarps;                 // warp 16: its lane 0 issues every MMA
constexpr int kGenWarps = 3;                           // warps 17..19: claim, decode, write operands
constexpr int kGenThreads = kGenWarps * 32;
constexpr int kThreads = kEpiThreads + 32 + kGenThreads;
constexpr int kM = 128;                 // rows per strip (UMMA M)
constexpr int kN = 256;                 // columns per MMA tile (UMMA N)
constexpr int kTilesPerStrip = kSuper / kN;  // 4
constexpr int kK = 64;                  // bytes of K per row/column
constexpr int kLBO = 128;               // bytes between K-adjacent 8x16B core matrices
constexpr int kSBO = 512;               // bytes between M/N-adjacent 8-row groups (4 core matrices)
constexpr int kABytes = kM * kK;        // 8 KB
constexpr int kBTileBytes = kN * kK;    // 16 KB
constexpr int kBBytes = kTilesPerStrip * kBTileBytes;  // 64 KB
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kMinSmem = 120 * 1024;  // more than half an SM: one CTA (and one TMEM owner) per SM
// Bound of the wait for in-flight MMAs before an aborted CTA releases its TMEM;
// fixed, independent of MmaArgs::timeout_ns (which a caller may set very short).
constexpr unsigned long long kDrainTimeoutNs = 2000000000ull;
constexpr int kBufs = kTmemCols / kN;   // accumulator buffers
// Pauses (ns) between the polls of a waiting epilogue warp (for its next tile),
// of the issuer (for a free accumulator buffer or the next strip's operands) and
// of the generators (for a free operand slot).  A poll is a shared-memory pipe
// operation, as is every binning atomic, and an issue slot taken from the
// epilogue warps of the same scheduler.  Single epilogue, k=22: 5.96e12 pairs/s
// without an epilogue pause, 6.09e12 at 120 ns, 6.14e12 at 400 ns, 6.03e12 at
// 1000 ns.  Paired epilogue, whose binning is issue-bound, k=22: issuer 8.77e12
// without a pause, 9.06-9.08e12 at 64-500 ns; then epilogue 8.95e12 at 100 ns,
// 9.02e12 at 400 ns, 9.11e12 at 800 ns, 9.02e12 at 1600 ns; generators 200 ns: -1 %.
constexpr unsigned kEpiPollNs = 800;
constexpr unsigned kIssuerPollNs = 200;
constexpr unsigned kGenPollNs = 0;
constexpr int kColsPerWarp = kN / (kEpiWarps / 4);  // columns of a tile each epilogue warp reads
constexpr int kLoads = kColsPerWarp / 32;           // 32-column TMEM loads per warp and tile
static_assert(kEpiWarps % 4 == 0 && kColsPerWarp % 32 == 0, "whole 32-column TMEM loads per warp and tile");
// Strips a generator claim takes: 4 super tiles, which in the column-by-column
// tile order share their column operand (written once per claim and column).
constexpr int kClaimStrips = 4 * kStrips;
// pair-packed epilogue
constexpr int kPkHalf = kSuper / 2;                 // packed columns of a strip: p holds columns 2p, 2p + 1
constexpr int kPkTilesPerStrip = kPkHalf / kN;      // 2 MMA tiles of 256 packed columns per strip
constexpr int kPkBBytes = kPkTilesPerStrip * kBTileBytes;  // 32 KB column operand per super tile
constexpr uint32_t kPkFb = 64;                      // fallback row after the joint cells: single distances 0..63
// Tiles between table flushes: a tile adds at most 16 warps x 64 values x 2
// (an outlier counts twice in the fallback row) to a lane's column, so a
// uint32 cell stays below 2^31 within 2^20 tiles.  (The 32 lane columns of a
// cell can hold more than 2^32 together: the flush sums them in 64 bits.)
constexpr uint32_t kPkFlushTiles = 1u << 20;
template <bool kPk>
__host__ __device__ constexpr int tiles_per_strip() { return kPk ? kPkTilesPerStrip : kTilesPerStrip; }
__host__ __device__ constexpr uint32_t buf_of(uint64_t g) { return (uint32_t)(g % kBufs); }
__host__ __device__ constexpr uint32_t parity_of(uint64_t g) { return (uint32_t)(g / kBufs) & 1u; }

// ---------------------------------------------------------------- PTX wrappers
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint32_t addr, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(addr), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t addr, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(addr), "r"(phase)
      : "memory");
  return ok != 0;
}

// Bounded wait: true when the phase completed, false after timeout_ns.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t addr, uint32_t phase, unsigned long long timeout_ns) {
  if (mbar_try_wait(addr, phase)) return true;
  const uint64_t t0 = globaltimer();
  while (true) {
    if (mbar_try_wait(addr, phase)) return true;
    if (globaltimer() - t0 > timeout_ns) return false;
  }
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// Shared-memory matrix descriptor, no swizzle, K-major (version field = 1).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr & 0x3FFFF) >> 4);
  d |= (uint64_t)(kLBO >> 4) << 16;
  d |= (uint64_t)(kSBO >> 4) << 32;
  d |= (uint64_t)1 << 46;
  return d;  // base offset 0, absolute-LBO mode off, layout type 0 (SWIZZLE_NONE)
}

// Instruction descriptor: D = S32, A = B = signed 8-bit, both K-major, M=128, N=kN.
constexpr uint32_t kIdesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kN >> 3) << 17) |
                            ((uint32_t)(kM >> 4) << 24);

__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(kIdesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

// 32 consecutive TMEM columns of this warp's 32 lanes; tmem_wait_ld completes it.
__device__ __forceinline__ void tmem_ld32_nowait(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
        "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
        "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void red_shared(uint32_t addr) {
  asm volatile("red.shared.add.u32 [%0], 1;" ::"r"(addr) : "memory");
}

// ---------------------------------------------------------------- operands
// 4 bits -> 4 bytes of 0/1 (bit q of the nibble to byte q).
__device__ __forceinline__ uint32_t spread_nibble(uint64_t x, int q) {
  const uint32_t nib = (uint32_t)(x >> (4 * q)) & 0xFu;
  return (nib * 0x00204081u) & 0x01010101u;
}

// Writes 16-byte chunk c (bytes 16c..16c+15) of row/column `r` of a K-major
// no-swizzle operand whose 8-row groups are kSBO apart.
__device__ __forceinline__ void put_chunk(uint8_t* base, int r, int c, uint4 v) {
  *reinterpret_cast<uint4*>(base + (r >> 3) * kSBO + c * kLBO + (r & 7) * 16) = v;
}

// Row (pair-packed epilogue) of codeword x with L bit planes: bytes -2*bit, then popc(x), S, 1.
__device__ __forceinline__ void write_row_pk(uint8_t* base, int r, uint64_t x, int L, uint32_t S) {
  uint32_t w[16];
  const uint32_t pc = (uint32_t)popc64(x);
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    if (4 * q < L) w[q] = spread_nibble(x, q) * 0xFEu;
    else if (4 * q == L) w[q] = pc | (S << 8) | (1u << 16);
    else w[q] = 0;
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) put_chunk(base, r, c, make_uint4(w[4 * c], w[4 * c + 1], w[4 * c + 2], w[4 * c + 3]));
}

// Packed column of codewords y, y2 (pair-packed epilogue): bytes bit(y) + S*bit(y2)
// (each <= S + 1 <= 127, no carries between bytes), then 1 + S, popc(y2) - lo, popc(y).
__device__ __forceinline__ void write_col_pk(uint8_t* base, int r, uint64_t y, uint64_t y2, int L, uint32_t S,
                                             int32_t lo) {
  uint32_t w[16];
  const uint32_t c1 = (uint32_t)popc64(y), c2 = (uint32_t)((int32_t)popc64(y2) - lo) & 0xFFu;
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    if (4 * q < L) w[q] = spread_nibble(y, q) + S * spread_nibble(y2, q);
    else if (4 * q == L) w[q] = (1u + S) | (c2 << 8) | (c1 << 16);
    else w[q] = 0;
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) put_chunk(base, r, c, make_uint4(w[4 * c], w[4 * c + 1], w[4 * c + 2], w[4 * c + 3]));
}

// Row/column operand of codeword x with L bit planes (L multiple of 4, L <= 60).
// is_a: bytes -2*bit, then popc(x), 1;  else: bit, then 1, popc(x).
__device__ __forceinline__ void write_operand(uint8_t* base, int r, uint64_t x, int L, bool is_a) {
  uint32_t w[16];
  const uint32_t pc = (uint32_t)popc64(x);
  const uint32_t mul = is_a ? 0xFEu : 1u;  // 0x01 * 0xFE = 0xFE = -2 as int8, no carries between bytes
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    if (4 * q < L) w[q] = spread_nibble(x, q) * mul;
    else if (4 * q == L) w[q] = is_a ? (pc | (1u << 8)) : (1u | (pc << 8));
    else w[q] = 0;
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) put_chunk(base, r, c, make_uint4(w[4 * c], w[4 * c + 1], w[4 * c + 2], w[4 * c + 3]));
}

// ---------------------------------------------------------------- decode
__device__ __forceinline__ uint32_t find_job(const Job* jobs, uint32_t njobs, uint64_t t) {
  uint32_t lo = 0, hi = njobs - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (__ldg(&jobs[mid].tile_begin) <= t) lo = mid; else hi = mid - 1;
  }
  return lo;
}

constexpr uint32_t kInfoDone = 1u, kInfoFull = 2u, kInfoRect = 4u;

// One strip (128 rows x one super tile of columns) as the generators publish it.
struct StripInfo {
  unsigned long long r0, c0;
  unsigned long long n;     // rows (codewords of a triangle job, lattice points of a grid job)
  unsigned long long cols;  // columns
  uint32_t job, flags;      // kInfoDone | kInfoFull | kInfoRect
  uint32_t bbuf, pad;       // column-operand buffer the strip reads
};

// Codeword of row i / column j of job J: A*i for the codeword progression, the
// lattice codeword for grid rows and (2-D) columns, the extended Hamming
// codeword for the all-pairs Hamming jobs.
__device__ __forceinline__ uint64_t mma_row_value(const Job* J, uint64_t i) {
  switch (__ldg(&J->row_kind)) {
    case ROW_LATTICE: return lattice_value(__ldg(&J->A), i, __ldg(&J->row_step), __ldg(&J->t32));
    case ROW_HAMMING_EXT: return hamming_cw_ext(i, __ldg(&J->n));
    default: return __ldg(&J->A) * i;
  }
}
__device__ __forceinline__ uint64_t mma_col_value(const Job* J, uint64_t j) {
  switch (__ldg(&J->col_kind)) {
    case COL_LATTICE: return lattice_value(__ldg(&J->A), j, __ldg(&J->col_step), __ldg(&J->t32));
    case COL_HAMMING_EXT: return hamming_cw_ext(j, __ldg(&J->n));
    default: return __ldg(&J->A) * j;
  }
}

struct Shared {
  uint64_t full[kBufs];   // tile in TMEM buffer b ready: tcgen05.commit + the issuer's arrive (count 2)
  uint64_t empty[kBufs];  // TMEM buffer b read: one arrive per epilogue warp (count kEpiWarps)
  // strip info for the epilogue, by issued strip (tile g belongs to strip g / tiles
  // per strip), a ring of 4: read once per strip, so the epilogue's per-tile
  // shared-memory traffic is the barrier poll and arrive only (its loads would
  // queue behind the atomics)
  StripInfo estrip[4];
  // strip queue, generators -> issuer (slot = strip & 1, with that slot's row operand)
  StripInfo strip[2];
  uint64_t slot_full[2];  // strip ready: the generators' thread 0 arrives (count 1)
  uint64_t slot_free[2];  // every MMA of the strip done: tcgen05.commit after its last tile (count 1)
  uint64_t epi_bar;       // pair-packed: epilogue-wide barrier around table flushes (count kEpiWarps)
  unsigned long long sbins[kMaxBins];  // pair-packed: per-distance sums of one table flush
  uint32_t tmem_base;
  uint32_t abort;         // set by whichever wait ran out; every other wait then gives up too
  uint32_t gflag;         // generators: result of their thread 0's wait
  uint32_t pad;
  // generators: first strip of claim c in gclaim[c & 1].  Thread 0 rewrites an entry
  // two claims later, past the barrier of the claim in between, which every thread
  // reaches only after reading the entry (a single word could be overwritten first
  // when every strip of a claim is skipped)
  unsigned long long gclaim[2];
};

// Barrier 1 over the generator warps only (barrier 0 is __syncthreads).
__device__ __forceinline__ void gen_bar() { asm volatile("bar.sync 1, %0;" ::"n"(kGenThreads) : "memory"); }

__device__ __forceinline__ void mbar_arrive(uint32_t addr) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(addr) : "memory");
}

// Bounded wait (single thread): true when the phase completed; false after
// timeout_ns or once another thread has aborted (then this one aborts too).
// The abort flag (shared memory) and the timer are checked every 32 polls.  The
// polls go through the shared-memory pipe that the epilogue's atomics load, so a
// waiter may pause kSleepNs between polls to leave that pipe to the binning warps.
template <unsigned kSleepNs = 0>
__device__ __forceinline__ bool wait_or_abort(uint32_t addr, uint32_t parity, unsigned long long timeout_ns,
                                              volatile uint32_t* abort) {
  if (mbar_try_wait(addr, parity)) return true;
  const uint64_t t0 = globaltimer();
  for (uint32_t spin = 1;; ++spin) {
    if constexpr (kSleepNs > 0) __nanosleep(kSleepNs);
    if (mbar_try_wait(addr, parity)) return true;
    if ((spin & 31) == 0) {
      if (*abort) return false;
      if (globaltimer() - t0 > timeout_ns) {
        *abort = 1u;
        return false;
      }
    }
  }
}

}  // namespace

// ---------------------------------------------------------------- kernel
// Epilogue-wide barrier of the pair-packed epilogue (every epilogue warp, one
// arrive each), bounded like every other wait; false once the CTA aborts.
__device__ __forceinline__ bool epi_sync(Shared* sh, uint32_t& phase, int lane, unsigned long long timeout_ns,
                                         volatile uint32_t* abort) {
  __syncwarp();
  bool r = true;
  if (lane == 0) {
    mbar_arrive(smem_u32(&sh->epi_bar));
    r = wait_or_abort<kEpiPollNs>(smem_u32(&sh->epi_bar), phase, timeout_ns, abort);
  }
  phase ^= 1u;
  const bool ok = __shfl_sync(0xffffffffu, r ? 1 : 0, 0) != 0;
  __syncwarp();
  return ok;
}

// Two single distances of a packed value (fallback row), for the outliers of
// full tiles and the checked pairs of partial tiles: Q = P + S*lo = d1 + S*d2.
// False for a value no operands can produce (d2 >= kPkFb).  Q < 64 * S <= 3904
// is exact in float, and (Q + 1/2) / S lies at least 1/(2S) from an integer,
// far above the error of the rounded reciprocal.
__device__ __forceinline__ bool pk_decode(uint32_t P, uint32_t S, float inv_s, int32_t lo, uint32_t& d1,
                                          uint32_t& d2) {
  const uint32_t Q = P + S * (uint32_t)lo;
  if (Q >= S * kPkFb) return false;
  d2 = (uint32_t)(((float)Q + 0.5f) * inv_s);
  d1 = Q - d2 * S;
  return true;
}

// A packed value counted as two single distances in the fallback row (lane
// column base fb), for the outliers of full tiles and the checked pairs of
// partial tiles; which of the two pairs count: bit 0 (d1), bit 1 (d2).  Not
// inlined: one copy instead of one per value of the unrolled binning loops,
// which keeps the rarely run code out of the hot loop's instruction stream.
__device__ __noinline__ void pk_fallback(uint32_t P, uint32_t S, float inv_s, int32_t lo, uint32_t fb,
                                         uint32_t which, unsigned* status) {
  uint32_t d1, d2;
  if (!pk_decode(P, S, inv_s, lo, d1, d2)) {  // not a value the operands can produce
    atomicOr(status, KSTATUS_BAD_DISTANCE);
    return;
  }
  if (which & 1u) red_shared(fb + (d1 << 7));
  if (which & 2u) red_shared(fb + (d2 << 7));
}

// Warp roles: warps 0..15 bin (epilogue), warp 16 issues the MMAs (lane 0),
// warps 17..19 claim strips and write their operands.  Hand-offs go through
// mbarriers only: slot_full/slot_free (a strip's operands written / its MMAs
// done), full[b] (the MMA result in TMEM buffer b is ready, and for a strip's
// first tile the strip's StripInfo),
// empty[b] (all 16 epilogue warps have read buffer b), and for the
// pair-packed epilogue epi_bar around each table flush.  No CTA-wide barrier
// runs between set-up and exit.
//
// Epilogue warp w reads TMEM lanes 32*(w%4).. (its rows) and 64 columns
// 64*(w/4).. of each 256-column tile.  Single epilogue: it bumps one
// shared-memory counter per pair in its own bin columns (row stride
// kEpiThreads words), so warps never share a counter and each warp flushes its
// own columns.  A distance is at most L (both operands have L bit planes,
// popc(x) <= L), and there are at least L + 1 bin rows (mma_hist_rows), so it
// indexes the rows unchecked; rows at or above the job's bin count are flagged
// at the flush.  Pair-packed epilogue: one counter per packed value in the
// joint table's column of its lane (see the file comment).
template <bool kPk>
__global__ void __launch_bounds__(kThreads, 1) mma_hist_kernel(MmaArgs args) {
  constexpr int kTps = tiles_per_strip<kPk>();
  constexpr int kColBytes = kPk ? kPkBBytes : kBBytes;  // column operand of one super tile
  extern __shared__ __align__(1024) uint8_t smem[];
  // b_bufs column operands of a super tile, double-buffered when they fit, so the
  // next super tile's operand is written while the current one's MMAs run
  uint8_t* sB = smem;
  uint8_t* sA = smem + (size_t)args.b_bufs * kColBytes;       // 2 x 8 KB: row operand, double-buffered by strip
  uint32_t* hist = reinterpret_cast<uint32_t*>(sA + 2 * kABytes);  // bins (single) or the joint table (packed)
  // packed: pk_cells joint cells then the kPkFb fallback cells, one column per lane
  const size_t hist_words = kPk ? (size_t)(args.pk_cells + kPkFb) * 32 : (size_t)args.hist_rows * kEpiThreads;
  Shared* sh = reinterpret_cast<Shared*>(sA + 2 * kABytes + hist_words * 4);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  volatile uint32_t* abort = &sh->abort;

  for (uint32_t k = tid; k < hist_words; k += kThreads) hist[k] = 0;
  if (tid < kMaxBins) sh->sbins[tid] = 0;
  if (tid == 0) {
    for (int b = 0; b < kBufs; ++b) {
      mbar_init(smem_u32(&sh->full[b]), 2);
      mbar_init(smem_u32(&sh->empty[b]), kEpiWarps);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&sh->slot_full[b]), 1);
      mbar_init(smem_u32(&sh->slot_free[b]), 1);
    }
    mbar_init(smem_u32(&sh->epi_bar), kEpiWarps);
    sh->abort = 0;
    fence_mbar_init();
  }
  if (warp == kIssuerWarp) tmem_alloc(smem_u32(&sh->tmem_base), kTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sh->tmem_base;

  if (warp > kIssuerWarp) {
    // ------------------------------------------------------------ generators
    // All kGenThreads threads walk the same strips (uniform control flow
    // between the named barriers); their thread 0 claims work and waits.
    const int gtid = tid - (kEpiThreads + 32);
    uint64_t s = 0;  // strips published
    uint32_t bjob = 0xffffffffu;
    uint64_t bsc = ~0ull;  // column super tile whose operand is in buffer bcur
    uint32_t bfill = 0, bcur = 0;  // column operands written so far, the buffer of the latest
    uint32_t nclaim = 0;           // claims taken
    unsigned long long t = 0, end = 0;
    bool normal = false;
    for (;;) {
      if (t >= end) {
        if (gtid == 0) sh->gclaim[nclaim & 1] = atomicAdd(args.counter, (unsigned long long)kClaimStrips);
        gen_bar();
        const unsigned long long base = sh->gclaim[nclaim & 1];
        ++nclaim;
        if (base >= args.total_tiles) { normal = true; break; }
        t = base;
        end = base + kClaimStrips < args.total_tiles ? base + (unsigned long long)kClaimStrips
                                                     : (unsigned long long)args.total_tiles;
      }
      const unsigned long long tt = t++;
      const uint32_t jn = find_job(args.jobs, args.njobs, tt);
      if (jn >= args.njobs) {
        if (gtid == 0) atomicOr(args.status, KSTATUS_BAD_JOB);
        continue;
      }
      const Job* jp = args.jobs + jn;
      const uint64_t tb = __ldg(&jp->tile_begin), tiles = __ldg(&jp->tiles);
      if (tt < tb || tt - tb >= tiles) {
        if (gtid == 0) atomicOr(args.status, KSTATUS_BAD_JOB);
        continue;
      }
      const uint64_t A = __ldg(&jp->A), N = __ldg(&jp->rows), NC = __ldg(&jp->cols);
      const uint64_t lt = tt - tb + __ldg(&jp->tile_offset);
      const bool rect = __ldg(&jp->shape) == SHAPE_RECT;
      uint64_t r0, c0, sc;
      bool full;
      if (rect) {
        // grid job: 128 rows x 1024 columns per tile, column tile by column tile,
        // so that consecutive tiles share the column operand
        static_assert(kM == 128 && kSuper == 1024, "rect_decode's tile shape");
        rect_decode(lt, (N + kM - 1) / kM, r0, c0);
        sc = c0 / kSuper;
        full = (r0 + kM <= N) && (c0 + kSuper <= NC);
      } else {
        uint64_t sr;
        tri_decode(lt / kStrips, __ldg(&jp->col_tiles), sr, sc);
        r0 = sr * kSuper + (lt % kStrips) * kM;
        c0 = sc * kSuper;
        full = (r0 + kM <= N) && (c0 + kSuper <= N) && sr != sc;
      }
      if (r0 >= N) continue;  // uniform over the group
      // every AN codeword of the job lies below A * 2^n (lattice points are indices
      // < 2^n); an extended Hamming codeword has nbins - 1 bits
      int L;
      if (__ldg(&jp->row_kind) == ROW_HAMMING_EXT) {
        L = (int)__ldg(&jp->nbins) - 1;
      } else {
        const uint64_t maxcw = A * ((1ull << __ldg(&jp->n)) - 1ull);
        L = 64 - __clzll((long long)(maxcw | 1));
      }
      L = (L + 3) & ~3;
      const uint32_t S = __ldg(&jp->pk_s);
      const int32_t lo = __ldg(&jp->pk_lo);
      const uint32_t slot = (uint32_t)(s & 1);
      const bool need_b = jn != bjob || sc != bsc;
      // this slot's row operand may be rewritten once every MMA of strip s-2 is
      // done; a single column-operand buffer once every MMA of strip s-1 is done.
      // With two buffers, the one rewritten was last read by strips up to s-2 (the
      // other buffer serves at least strip s-1), so the s-2 wait covers it too.
      if (gtid == 0) {
        bool ok = true;
        if (need_b && args.b_bufs == 1 && s >= 1)
          ok = wait_or_abort<kGenPollNs>(smem_u32(&sh->slot_free[(s - 1) & 1]), (uint32_t)((s - 1) >> 1) & 1u,
                                         args.timeout_ns, abort);
        else if (s >= 2)
          ok = wait_or_abort<kGenPollNs>(smem_u32(&sh->slot_free[slot]), (uint32_t)((s - 2) >> 1) & 1u,
                                         args.timeout_ns, abort);
        sh->gflag = ok ? 1u : 0u;
      }
      gen_bar();
      if (!sh->gflag) break;
      if (need_b) {
        bcur = args.b_bufs == 2 ? (bfill & 1u) : 0u;
        ++bfill;
        uint8_t* bb = sB + (size_t)bcur * kColBytes;
        const uint64_t ncols = rect ? NC : N;
        if constexpr (kPk) {
          // packed column p: the adjacent columns c0 + 2p and c0 + 2p + 1, so a
          // diagonal or edge strip has few packed values with just one valid pair
#pragma unroll 1
          for (int cc = gtid; cc < kPkHalf; cc += kGenThreads) {
            const uint64_t j = c0 + 2 * (uint64_t)cc, j2 = j + 1;
            write_col_pk(bb + (cc / kN) * kBTileBytes, cc % kN, j < ncols ? mma_col_value(jp, j) : 0,
                         j2 < ncols ? mma_col_value(jp, j2) : 0, L, S, lo);
          }
        } else {
#pragma unroll 1
          for (int cc = gtid; cc < kSuper; cc += kGenThreads) {
            const uint64_t j = c0 + cc;
            write_operand(bb + (cc / kN) * kBTileBytes, cc % kN, j < ncols ? mma_col_value(jp, j) : 0, L, false);
          }
        }
        bjob = jn;
        bsc = sc;
      }
      uint8_t* a = sA + slot * kABytes;
#pragma unroll 1
      for (int rr = gtid; rr < kM; rr += kGenThreads) {
        const uint64_t i = r0 + rr;
        const uint64_t x = i < N ? mma_row_value(jp, i) : 0;
        if constexpr (kPk) write_row_pk(a, rr, x, L, S);
        else write_operand(a, rr, x, L, true);
      }
      fence_proxy_async();
      gen_bar();  // both operands complete
      if (gtid == 0) {
        StripInfo& si = sh->strip[slot];
        si.r0 = r0;
        si.c0 = c0;
        si.n = N;
        si.cols = rect ? NC : N;
        si.job = jn;
        si.flags = (full ? kInfoFull : 0u) | (rect ? kInfoRect : 0u);
        si.bbuf = bcur;
        mbar_arrive(smem_u32(&sh->slot_full[slot]));
      }
      ++s;
    }
    if (gtid == 0 && normal) {
      // the issuer has finished with strip s-2 (this slot) once that strip's MMAs are done
      if (s < 2 || wait_or_abort(smem_u32(&sh->slot_free[s & 1]), (uint32_t)((s - 2) >> 1) & 1u, args.timeout_ns,
                                 abort)) {
        sh->strip[s & 1].flags = kInfoDone;
        mbar_arrive(smem_u32(&sh->slot_full[s & 1]));
      }
    }
  } else if (warp == kIssuerWarp) {
    // ------------------------------------------------------------ issuer (lane 0)
    if (lane == 0) {
      uint64_t g = 0;  // tiles issued
      bool normal = false;
      // until the epilogue has read tile gg-kBufs, the previous tile of gg's buffer
      auto wait_empty = [&](uint64_t gg) -> bool {
        return gg < kBufs ||
               wait_or_abort<kIssuerPollNs>(smem_u32(&sh->empty[buf_of(gg)]), parity_of(gg - kBufs), args.timeout_ns,
                                            abort);
      };
      for (uint64_t s = 0;; ++s) {
        const uint32_t slot = (uint32_t)(s & 1);
        if (!wait_or_abort<kIssuerPollNs>(smem_u32(&sh->slot_full[slot]), (uint32_t)(s >> 1) & 1u, args.timeout_ns, abort))
          break;
        const StripInfo si = sh->strip[slot];
        if (si.flags & kInfoDone) { normal = true; break; }
        const uint32_t a0 = smem_u32(sA + slot * kABytes);
        bool ok = true;
        for (int tile = 0; tile < kTps; ++tile, ++g) {
          if (!wait_empty(g)) { ok = false; break; }
          const uint32_t b = buf_of(g);
          if (tile == 0) {
            // the entry of strip s-4: every warp read it at tile g-4*kTps, long
            // before tile g-kBufs, which wait_empty has seen released
            StripInfo& es = sh->estrip[(g / kTps) & 3];
            es = si;
            es.flags = si.flags & (kInfoFull | kInfoRect);
          }
          tc_fence_after();
          const uint32_t d = tmem + b * (uint32_t)kN;
          const uint32_t b0 = smem_u32(sB + (size_t)si.bbuf * kColBytes + tile * kBTileBytes);
#pragma unroll
          for (int ks = 0; ks < kK / 32; ++ks)  // K = 32 bytes per instruction = 2 core matrices
            mma_i8(d, smem_desc(a0 + ks * 2 * kLBO), smem_desc(b0 + ks * 2 * kLBO), ks > 0 ? 1u : 0u);
          mma_commit(smem_u32(&sh->full[b]));
          mbar_arrive(smem_u32(&sh->full[b]));
        }
        if (!ok) break;
        mma_commit(smem_u32(&sh->slot_free[slot]));  // the strip's operands are free once its MMAs are done
      }
      if (normal && wait_empty(g)) {
        // end of work: a strip marked done wakes the epilogue warps (g is a strip's first tile)
        sh->estrip[(g / kTps) & 3].flags = kInfoDone;
        mbar_arrive(smem_u32(&sh->full[buf_of(g)]));
        mbar_arrive(smem_u32(&sh->full[buf_of(g)]));
      } else {
        *abort = 1u;
        atomicOr(args.status, KSTATUS_TIMEOUT);
        // let the last MMA drain (bounded, in-order completion) before TMEM is released
        if (g > 0) mbar_wait_bounded(smem_u32(&sh->full[buf_of(g - 1)]), parity_of(g - 1), kDrainTimeoutNs);
      }
    }
    __syncwarp();
  } else {
    // ------------------------------------------------------------ epilogue
    const int q = warp & 3, sub = warp >> 2;
    uint32_t cur = 0xffffffffu, nbins = 0, since_flush = 0;
    unsigned long long* bins = nullptr;
    bool ok = true;
    // pair-packed state: the table's column of this lane, the current job's S and window
    const uint32_t pk_lane = smem_u32(hist) + (uint32_t)lane * 4u;
    const uint32_t pk_fb = pk_lane + (args.pk_cells << 7);
    uint32_t pkS = 1, pklimit = 0, epi_phase = 0;
    int32_t pklo = 0;
    float pkinv = 1.0f;
    bool pkall = false;  // the window holds every (d1, d2): no value can fall outside it
    // single: this warp's bin columns -> the job's global bins
    auto flush = [&]() {
      for (uint32_t b = 0; b < args.hist_rows; ++b) {
        const uint32_t x = hist[b * kEpiThreads + tid];
        hist[b * kEpiThreads + tid] = 0;
        const uint32_t s = __reduce_add_sync(0xffffffffu, x);
        if (lane == 0 && s) {
          if (b < nbins) atomicAdd(bins + b, (unsigned long long)s);
          else atomicOr(args.status, KSTATUS_BAD_DISTANCE);
        }
      }
    };
    // pair-packed: every epilogue warp folds a share of the table's cells into the
    // flush sums (a joint cell adds to d1 and to d2), then warp 0 adds the sums to
    // the job's bins.  False once the CTA aborted.
    auto flush_pk = [&]() -> bool {
      if (!epi_sync(sh, epi_phase, lane, args.timeout_ns, abort)) return false;
      for (uint32_t c = (uint32_t)warp; c < args.pk_cells + kPkFb; c += kEpiWarps) {
        const uint32_t x = hist[c * 32 + lane];
        hist[c * 32 + lane] = 0;
        // 32 cells of up to 2^31 each: reduce the 16-bit halves, sum in 64 bits
        const unsigned long long s = (unsigned long long)__reduce_add_sync(0xffffffffu, x & 0xFFFFu) +
                                     ((unsigned long long)__reduce_add_sync(0xffffffffu, x >> 16) << 16);
        if (lane == 0 && s) {
          if (c < args.pk_cells) {
            const uint32_t d1 = c % pkS, d2 = c / pkS + (uint32_t)pklo;
            atomicAdd(&sh->sbins[d1], s);
            if (d2 < (uint32_t)kMaxBins) atomicAdd(&sh->sbins[d2], s);
            else atomicOr(args.status, KSTATUS_BAD_DISTANCE);
          } else {
            atomicAdd(&sh->sbins[c - args.pk_cells], s);
          }
        }
      }
      if (!epi_sync(sh, epi_phase, lane, args.timeout_ns, abort)) return false;
      if (warp == 0) {
        for (uint32_t d = (uint32_t)lane; d < (uint32_t)kMaxBins; d += 32) {
          const unsigned long long v = sh->sbins[d];
          sh->sbins[d] = 0;
          if (v) {
            if (d < nbins) atomicAdd(bins + d, v);
            else atomicOr(args.status, KSTATUS_BAD_DISTANCE);
          }
        }
      }
      return true;
    };
    // pair-packed: one packed value counted as two single distances (fallback row)
    auto pk_single = [&](uint32_t P, bool v1, bool v2) {
      pk_fallback(P, pkS, pkinv, pklo, pk_fb, (v1 ? 1u : 0u) | (v2 ? 2u : 0u), args.status);
    };
    unsigned long long r0 = 0, cs = 0, n = 0, nc = 0;  // the current strip: first row and column, rows, columns
    uint32_t flags = 0, job = 0;
    // lane 0 waits (bounded) for tile g; the warp learns the result
    auto wait_full = [&](uint64_t g) -> bool {
      bool r = true;
      if (lane == 0) r = wait_or_abort<kEpiPollNs>(smem_u32(&sh->full[buf_of(g)]), parity_of(g), args.timeout_ns, abort);
      const bool ok_ = __shfl_sync(0xffffffffu, r ? 1 : 0, 0) != 0;
      __syncwarp();  // lane 0's wait acquired the MMA result (and StripInfo); this orders it for the warp
      return ok_;
    };
    // the strip that tile g (a strip's first tile) starts; false at the end marker
    auto read_strip = [&](uint64_t g) -> bool {
      const StripInfo& es = sh->estrip[(g / kTps) & 3];
      flags = es.flags;
      if (flags & kInfoDone) return false;
      job = es.job;
      if constexpr (!kPk) {  // the paired epilogue reads them from es where it needs them
        r0 = es.r0;
        cs = es.c0;
        n = es.n;
        nc = es.cols;
      }
      return true;
    };
    // 32 TMEM columns (half h of this warp's 64) of tile g: issued, completed by tmem_wait_ld
    auto ld_half = [&](uint64_t g, int h, uint32_t (&dst)[32]) {
      tmem_ld32_nowait(tmem + ((uint32_t)(q * 32) << 16) + buf_of(g) * (uint32_t)kN +
                           (uint32_t)(sub * kColsPerWarp + 32 * h),
                       dst);
    };
    if constexpr (kPk) {
      auto set_job = [&](uint32_t jb) {
        cur = jb;
        bins = args.jobs[jb].bins;
        nbins = args.jobs[jb].nbins;
        pkS = args.jobs[jb].pk_s;
        pklo = args.jobs[jb].pk_lo;
        pklimit = args.jobs[jb].pk_limit;  // <= pk_cells (host)
        pkinv = 1.0f / (float)pkS;
        // lo = 0 and S rows: every value d1 + S*d2 < S*S = limit, the test is void
        pkall = pklo == 0 && pklimit == pkS * pkS;
      };
      // bins 32 packed values, half h of tile g of the current strip
      auto bin_half = [&](const uint32_t (&x)[32], uint64_t g, int h) {
        if ((flags & kInfoFull) && pkall) {
#pragma unroll
          for (int u = 0; u < 32; ++u) red_shared(pk_lane + (x[u] << 7));
        } else if (flags & kInfoFull) {
          // one unsigned max over the values tests every d2 against the window
          // at once (a d2 below it gives a negative value, i.e. a huge one);
          // a tree of depth 5, not a chain of dependent maxima
          uint32_t m[16];
#pragma unroll
          for (int u = 0; u < 16; ++u) m[u] = max(x[2 * u], x[2 * u + 1]);
#pragma unroll
          for (int w = 8; w >= 1; w >>= 1)
#pragma unroll
            for (int u = 0; u < w; ++u) m[u] = max(m[u], m[u + w]);
          if (__any_sync(0xffffffffu, m[0] >= pklimit)) {
            // some d2 outside the window: those values count as two single distances
#pragma unroll
            for (int u = 0; u < 32; ++u) {
              if (x[u] < pklimit) red_shared(pk_lane + (x[u] << 7));
              else pk_single(x[u], true, true);
            }
          } else {
#pragma unroll
            for (int u = 0; u < 32; ++u) red_shared(pk_lane + (x[u] << 7));
          }
        } else {
          // partial strip: every pair checked; a value whose two pairs both count
          // and whose d2 lies in the window still takes one joint cell.  Value u
          // holds columns cbase + 2u and cbase + 2u + 1: a pair counts when its
          // row is a row of the job and its column offset o in [0, 64) satisfies
          // lo_o < o < hi_o (triangle: the column lies above the row's diagonal
          // and inside the job; grid: inside the job), bounds clamped to 32 bits.
          // The strip's entry stays valid while its tiles are binned: the issuer
          // rewrites it for strip s+4 only after every warp has released the
          // tiles of strip s+3.  (Kept inline: a non-inlined copy of this loop,
          // fed through a local array, measured slower.)
          const StripInfo& es = sh->estrip[(g / kTps) & 3];
          const uint64_t i = es.r0 + (uint64_t)(q * 32 + lane);
          const uint64_t cbase = es.c0 + 2 * ((g % kTps) * (uint64_t)kN + (uint64_t)(sub * kColsPerWarp + 32 * h));
          const bool rect = (flags & kInfoRect) != 0;
          const int64_t dlo = rect ? -1 : (int64_t)i - (int64_t)cbase;            // o > dlo
          const int64_t dhi = (int64_t)(rect ? es.cols : es.n) - (int64_t)cbase;  // o < dhi
          const int32_t lo_o = i < es.n ? (int32_t)(dlo < -1 ? -1 : (dlo > 64 ? 64 : dlo)) : 64;
          const int32_t hi_o = (int32_t)(dhi < 0 ? 0 : (dhi > 64 ? 64 : dhi));
#pragma unroll
          for (int u = 0; u < 32; ++u) {
            const bool v1 = 2 * u > lo_o && 2 * u < hi_o;
            const bool v2 = 2 * u + 1 > lo_o && 2 * u + 1 < hi_o;
            if (v1 && v2 && x[u] < pklimit) red_shared(pk_lane + (x[u] << 7));
            else if (v1 || v2) pk_single(x[u], v1, v2);
          }
        }
      };
      for (uint64_t g = 0;; ++g) {
        if (!wait_full(g)) { ok = false; break; }
        if (g % kTps == 0) {
          if (!read_strip(g)) break;  // the end marker
          // a new job: the table must hold one job's counts, so every warp folds
          // it first (all warps see the same strips, so they flush at the same tile)
          if (job != cur) {
            if (cur != 0xffffffffu && !flush_pk()) { ok = false; break; }
            since_flush = 0;
            set_job(job);
          }
        }
        tc_fence_after();
        uint32_t v[kLoads][32];
#pragma unroll
        for (int h = 0; h < kLoads; ++h) ld_half(g, h, v[h]);
        tmem_wait_ld();
        // the buffer may be refilled as soon as every warp has its values in registers
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&sh->empty[buf_of(g)]));
#pragma unroll
        for (int h = 0; h < kLoads; ++h) bin_half(v[h], g, h);
        if (++since_flush >= kPkFlushTiles) {
          if (!flush_pk()) { ok = false; break; }
          since_flush = 0;
        }
      }
      if (ok && cur != 0xffffffffu) flush_pk();
    } else {
      for (uint64_t g = 0;; ++g) {
        const uint32_t b = buf_of(g);
        if (!wait_full(g)) { ok = false; break; }
        const uint32_t tile = (uint32_t)(g % kTps);
        if (tile == 0 && !read_strip(g)) break;
        tc_fence_after();
        uint32_t v[kLoads][32];
#pragma unroll
        for (int h = 0; h < kLoads; ++h) ld_half(g, h, v[h]);
        tmem_wait_ld();
        // the buffer may be refilled as soon as every warp has its values in registers
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&sh->empty[b]));
        if (job != cur) {
          if (cur != 0xffffffffu && since_flush) flush();
          since_flush = 0;
          cur = job;
          bins = args.jobs[job].bins;
          nbins = args.jobs[job].nbins;
        }
        const uint32_t hist_lane = smem_u32(hist) + (uint32_t)tid * 4u;
        if (flags & kInfoFull) {
#pragma unroll
          for (int h = 0; h < kLoads; ++h)
#pragma unroll
            for (int u = 0; u < 32; ++u) red_shared(hist_lane + (v[h][u] << 11));
        } else {
          const unsigned long long c0 = cs + (unsigned long long)tile * kN;
          const uint64_t i = r0 + (uint64_t)(q * 32 + lane);
          const uint64_t j0 = c0 + (uint64_t)(sub * kColsPerWarp);
#pragma unroll
          for (int h = 0; h < kLoads; ++h)
#pragma unroll
            for (int u = 0; u < 32; ++u) {
              const uint64_t j = j0 + 32 * h + u;
              const bool in = (flags & kInfoRect) ? (i < n && j < nc) : (i < n && j < n && j > i);
              if (in) red_shared(hist_lane + (v[h][u] << 11));
            }
        }
        if (++since_flush >= kFlushEvery) { flush(); since_flush = 0; }
      }
      if (ok && cur != 0xffffffffu && since_flush) flush();
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kIssuerWarp) {
    tc_fence_after();
    tmem_dealloc(tmem, kTmemCols);
  }
}

// ---------------------------------------------------------------- host side
int mma_max_distance(const Job& j) {
  if (j.row_kind == ROW_HAMMING_EXT) return (int)j.nbins - 1;  // extended Hamming codeword: n data + h check bits
  const unsigned __int128 maxcw = (unsigned __int128)j.A * ((1ull << j.n) - 1ull);
  int bits = 0;
  for (unsigned __int128 v = maxcw; v; v >>= 1) ++bits;
  return bits ? bits : 1;
}

// Bit planes of the operands of job j: the bits of A * (2^n - 1), which bounds
// every codeword of the job, rounded up to 4 (the kernel computes the same).
int mma_operand_bits(const Job& j) { return (mma_max_distance(j) + 3) & ~3; }

static uint64_t host_row_value(const Job& j, uint64_t i) {
  switch (j.row_kind) {
    case ROW_LATTICE: return lattice_value(j.A, i, j.row_step, j.t32);
    case ROW_HAMMING_EXT: return hamming_cw_ext(i, j.n);
    default: return j.A * i;
  }
}
static uint64_t host_col_value(const Job& j, uint64_t c) {
  switch (j.col_kind) {
    case COL_LATTICE: return lattice_value(j.A, c, j.col_step, j.t32);
    case COL_HAMMING_EXT: return hamming_cw_ext(c, j.n);
    default: return j.A * c;
  }
}

// Shared memory beside the joint table: the row operand (two strips), the
// column operand buffers, the Shared block and alignment slack.
static size_t pk_fixed_bytes(uint32_t b_bufs) {
  return (size_t)2 * kABytes + (size_t)b_bufs * kPkBBytes + sizeof(Shared) + 64;
}

static size_t smem_optin() {
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return 227 * 1024;
  return (size_t)optin;
}

void mma_pk_layout(uint32_t smax, uint32_t* cells, uint32_t* b_bufs) {
  const size_t optin = smem_optin();
  const size_t want = (size_t)smax * smax;
  auto fit = [&](uint32_t bufs) -> size_t {  // joint cells that fit beside `bufs` column buffers
    const size_t fixed = pk_fixed_bytes(bufs) + (size_t)kPkFb * 128;
    return optin > fixed ? (optin - fixed) / 128 : 0;
  };
  if (want <= fit(2)) {
    *cells = (uint32_t)want;
    *b_bufs = 2;
  } else {
    *cells = (uint32_t)std::min(want, fit(1));
    *b_bufs = 1;
  }
}

void mma_pack_setup(Job& j, uint32_t cells) {
  const uint32_t S = (uint32_t)mma_max_distance(j) + 1u;
  uint32_t rows = cells / S;  // whole rows of S cells: d2 - lo in [0, rows)
  if (rows > S) rows = S;
  int32_t lo = 0;
  if (rows < S && j.rows && j.cols) {
    // mean distance of 512 pairs drawn by a fixed generator (the same job always
    // gets the same window, so a cached launch graph stays valid)
    uint64_t st = 0x9E3779B97F4A7C15ull ^ (j.A * 0xBF58476D1CE4E5B9ull) ^ ((uint64_t)j.n << 56) ^ j.rows;
    auto next = [&st]() {
      st ^= st << 13; st ^= st >> 7; st ^= st << 17;
      return st;
    };
    double sum = 0;
    const int kSamples = 512;
    for (int k = 0; k < kSamples; ++k) {
      const uint64_t i = next() % j.rows, c = next() % j.cols;
      sum += (double)popc64(host_row_value(j, i) ^ host_col_value(j, c));
    }
    lo = (int32_t)std::lround(sum / kSamples - (double)(rows - 1) / 2.0);
    if (lo > (int32_t)(S - rows)) lo = (int32_t)(S - rows);
    if (lo < 0) lo = 0;
  }
  j.pk_s = S;
  j.pk_lo = lo;
  j.pk_limit = S * rows;
}

bool mma_eligible(const Job& j) {
  if (j.kind != JOB_PAIRS || j.n > 48) return false;
  const bool tri = j.shape == SHAPE_TRIANGLE && ((j.row_kind == ROW_PROGRESSION && j.col_kind == COL_PROGRESSION) ||
                                                 (j.row_kind == ROW_HAMMING_EXT && j.col_kind == COL_HAMMING_EXT));
  const bool rect = j.shape == SHAPE_RECT && (j.row_kind == ROW_PROGRESSION || j.row_kind == ROW_LATTICE) &&
                    (j.col_kind == COL_PROGRESSION || j.col_kind == COL_LATTICE) && j.col_tiles * kSuper >= j.cols;
  return (tri || rect) && mma_operand_bits(j) <= 60;
}

size_t mma_smem_bytes(uint32_t hist_rows, uint32_t b_bufs, bool packed, uint32_t pk_cells) {
  size_t s;
  if (packed) {
    s = pk_fixed_bytes(b_bufs) + ((size_t)pk_cells + kPkFb) * 128;
  } else {
    s = (size_t)2 * kABytes + (size_t)b_bufs * kBBytes + (size_t)hist_rows * kEpiThreads * 4 + sizeof(Shared) + 64;
  }
  return s < kMinSmem ? kMinSmem : s;
}

uint32_t mma_b_bufs(uint32_t hist_rows) {
  return mma_smem_bytes(hist_rows, 2, false, 0) <= smem_optin() ? 2u : 1u;
}

cudaError_t launch_mma(const MmaArgs& args, int grid, size_t smem, cudaStream_t stream) {
  // the per-function limit is process-wide: every caller sets the same value
  // (the device's opt-in maximum), so host threads launching plans of different
  // sizes cannot lower it under one another
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  if (smem > (size_t)optin) return cudaErrorInvalidValue;
  if (args.packed) {
    e = cudaFuncSetAttribute(mma_hist_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
    if (e != cudaSuccess) return e;
    mma_hist_kernel<true><<<grid, kThreads, smem, stream>>>(args);
  } else {
    e = cudaFuncSetAttribute(mma_hist_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
    if (e != cudaSuccess) return e;
    mma_hist_kernel<false><<<grid, kThreads, smem, stream>>>(args);
  }
  return cudaGetLastError();
}

}  // namespace dd
