// dd_mma.cu — tcgen05 kind::i8 bit-plane MMA kernel: AN exhaustive, 1-D / 2-D
// grid and Ext-Hamming all-pairs jobs.
//
// The Hamming distance of two codewords x, y (bit planes b_x, b_y in {0,1}^L)
// is d = popc(x) + popc(y) - 2<b_x, b_y>.  The operands put that whole
// expression into one int8 GEMM with K = 64:
//   A row i    (codeword x_i): bytes k<L: -2*b_ik;  byte L: popc(x_i);  byte L+1: 1
//   B column j (codeword y_j): bytes k<L:    b_jk;  byte L: 1;          byte L+1: popc(y_j)
// so the INT32 accumulator D[i][j] = Σ_k A[i][k]·B[k][j] is exactly d(i, j).
// The epilogue reads D from TMEM (tcgen05.ld) and bumps one shared-memory bin
// per pair; no other per-pair arithmetic is left.
//
// Work unit: the popc kernel's tile space (1024x1024 super tiles of the i<j
// triangle, split into 8 strips of 128 rows; for grid jobs, 128 lattice rows x
// 1024 columns, taken column-major).  A strip is 128 rows (UMMA M) x
// 1024 columns = 4 MMA tiles of N = 256, accumulated in two TMEM buffers of 256
// columns: the MMA of tile t+1 runs while the epilogue bins tile t.  (Four
// buffers of N = 128 measured 17 % slower: every tile costs each epilogue warp
// a barrier poll and an arrive through the shared-memory pipe that its atomics
// saturate, so fewer, wider tiles win over deeper buffering.)  Generator warps
// claim 8 strips at a time (one super tile when the job's tile range is
// aligned) and write the column operand once per super tile, into the second
// of two buffers when both fit beside the bins, so the next super tile's
// operand is written while the current one's MMAs run; the row operand is
// double-buffered by strip.
// One CTA per SM (16 epilogue warps, 1 issuer warp, 3 generator warps, 512 TMEM
// columns).
//
// The epilogue is bound by the shared-memory atomic rate (one red.shared per
// pair; about 31 per clock per SM measured on B200), twice the POPC issue rate
// (16 per clock per SM) that bounds the popc kernel.  A waiting epilogue warp
// pauses between its barrier polls, which share that pipe with the atomics.
//
// Every mbarrier wait is bounded (MmaArgs::timeout_ns); on expiry the CTA
// records KSTATUS_TIMEOUT, every other wait gives up, the last MMA drains
// (bounded) and the TMEM is released.
#include <cuda_runtime.h>
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
// of the issuer (for a free accumulator buffer) and of the generators (for a free
// operand slot).  A poll is a shared-memory pipe operation, as is every binning
// atomic: 400 ns for the epilogue measured best (k=22: 5.96e12 pairs/s without a
// pause, 6.09e12 at 120 ns, 6.14e12 at 400 ns, 6.03e12 at 1000 ns); a pause for
// the issuer changed nothing.
constexpr unsigned kEpiPollNs = 400;
constexpr unsigned kIssuerPollNs = 0;
constexpr unsigned kGenPollNs = 0;
constexpr int kColsPerWarp = kN / (kEpiWarps / 4);  // columns of a tile each epilogue warp reads
constexpr int kLoads = kColsPerWarp / 32;           // 32-column TMEM loads per warp and tile
static_assert(kEpiWarps % 4 == 0 && kColsPerWarp % 32 == 0, "whole 32-column TMEM loads per warp and tile");
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
  // strip info for the epilogue, by issued strip (tile g belongs to strip g / kTilesPerStrip):
  // read once per strip, so the epilogue's per-tile shared-memory traffic is the
  // barrier poll and arrive only (its loads would queue behind the atomics)
  StripInfo estrip[2];
  // strip queue, generators -> issuer (slot = strip & 1, with that slot's row operand)
  StripInfo strip[2];
  uint64_t slot_full[2];  // strip ready: the generators' thread 0 arrives (count 1)
  uint64_t slot_free[2];  // every MMA of the strip done: tcgen05.commit after its last tile (count 1)
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
// Warp roles: warps 0..15 bin (epilogue), warp 16 issues the MMAs (lane 0),
// warps 17..19 claim strips and write their operands.  Hand-offs go through
// mbarriers only: slot_full/slot_free (a strip's operands written / its MMAs
// done), full[b] (the MMA result in TMEM buffer b is ready, and for a strip's
// first tile the strip's StripInfo),
// empty[b] (all 16 epilogue warps have read buffer b).  No CTA-wide barrier
// runs between set-up and exit.
//
// Epilogue warp w reads TMEM lanes 32*(w%4).. (its rows) and 64 columns
// 64*(w/4).. of each 256-column tile, and bumps one shared-memory counter per
// pair in its own bin columns (row stride kEpiThreads words), so warps never
// share a counter and each warp flushes its own columns.  A distance is at
// most L (both operands have L bit planes, popc(x) <= L), and there are at
// least L + 1 bin rows (mma_hist_rows), so it indexes the rows unchecked;
// rows at or above the job's bin count are flagged at the flush.
__global__ void __launch_bounds__(kThreads, 1) mma_hist_kernel(MmaArgs args) {
  extern __shared__ __align__(1024) uint8_t smem[];
  // b_bufs x 64 KB: the column operand of a super tile (4 tiles of 256 columns), double-buffered
  // when it fits, so the next super tile's operand is written while the current one's MMAs run
  uint8_t* sB = smem;
  uint8_t* sA = smem + (size_t)args.b_bufs * kBBytes;        // 2 x 8 KB: row operand, double-buffered by strip
  uint32_t* hist = reinterpret_cast<uint32_t*>(sA + 2 * kABytes);  // hist_rows x kEpiThreads
  Shared* sh = reinterpret_cast<Shared*>(sA + 2 * kABytes + (size_t)args.hist_rows * kEpiThreads * 4);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  volatile uint32_t* abort = &sh->abort;

  for (uint32_t k = tid; k < args.hist_rows * kEpiThreads; k += kThreads) hist[k] = 0;
  if (tid == 0) {
    for (int b = 0; b < kBufs; ++b) {
      mbar_init(smem_u32(&sh->full[b]), 2);
      mbar_init(smem_u32(&sh->empty[b]), kEpiWarps);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&sh->slot_full[b]), 1);
      mbar_init(smem_u32(&sh->slot_free[b]), 1);
    }
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
        if (gtid == 0) sh->gclaim[nclaim & 1] = atomicAdd(args.counter, (unsigned long long)kStrips);
        gen_bar();
        const unsigned long long base = sh->gclaim[nclaim & 1];
        ++nclaim;
        if (base >= args.total_tiles) { normal = true; break; }
        t = base;
        end = base + kStrips < args.total_tiles ? base + (unsigned long long)kStrips
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
        // grid job: 128 rows x 1024 columns per tile, column-major here so that
        // consecutive tiles share the column operand
        const uint64_t row_tiles = (N + kM - 1) / kM;
        sc = lt / row_tiles;
        r0 = (lt % row_tiles) * kM;
        c0 = sc * kSuper;
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
        uint8_t* bb = sB + (size_t)bcur * kBBytes;
#pragma unroll 1
        for (int cc = gtid; cc < kSuper; cc += kGenThreads) {
          const uint64_t j = c0 + cc;
          write_operand(bb + (cc / kN) * kBTileBytes, cc % kN, j < (rect ? NC : N) ? mma_col_value(jp, j) : 0, L,
                        false);
        }
        bjob = jn;
        bsc = sc;
      }
      uint8_t* a = sA + slot * kABytes;
#pragma unroll 1
      for (int rr = gtid; rr < kM; rr += kGenThreads) {
        const uint64_t i = r0 + rr;
        write_operand(a, rr, i < N ? mma_row_value(jp, i) : 0, L, true);
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
      // until the epilogue has read tile gg-4, the previous tile of gg's buffer
      auto wait_empty = [&](uint64_t gg) -> bool {
        return gg < kBufs ||
               wait_or_abort<kIssuerPollNs>(smem_u32(&sh->empty[buf_of(gg)]), parity_of(gg - kBufs), args.timeout_ns,
                                            abort);
      };
      for (uint64_t s = 0;; ++s) {
        const uint32_t slot = (uint32_t)(s & 1);
        if (!wait_or_abort(smem_u32(&sh->slot_full[slot]), (uint32_t)(s >> 1) & 1u, args.timeout_ns, abort)) break;
        const StripInfo si = sh->strip[slot];
        if (si.flags & kInfoDone) { normal = true; break; }
        const uint32_t a0 = smem_u32(sA + slot * kABytes);
        bool ok = true;
        for (int tile = 0; tile < kTilesPerStrip; ++tile, ++g) {
          if (!wait_empty(g)) { ok = false; break; }
          const uint32_t b = buf_of(g);
          if (tile == 0) {
            // the entry of strip s-2: every warp read it at tile g-16 < g-4
            StripInfo& es = sh->estrip[(g / kTilesPerStrip) & 1];
            es = si;
            es.flags = si.flags & (kInfoFull | kInfoRect);
          }
          tc_fence_after();
          const uint32_t d = tmem + b * (uint32_t)kN;
          const uint32_t b0 = smem_u32(sB + (size_t)si.bbuf * kBBytes + tile * kBTileBytes);
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
        sh->estrip[(g / kTilesPerStrip) & 1].flags = kInfoDone;
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
    const uint32_t hist_lane = smem_u32(hist) + (uint32_t)tid * 4u;
    uint32_t cur = 0xffffffffu, nbins = 0, since_flush = 0;
    unsigned long long* bins = nullptr;
    bool ok = true;
    // this warp's bin columns -> the job's global bins
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
    unsigned long long r0 = 0, cs = 0, n = 0, nc = 0;  // the current strip: first row and column, rows, columns
    uint32_t flags = 0, job = 0;
    for (uint64_t g = 0;; ++g) {
      const uint32_t b = buf_of(g);
      bool r = true;
      if (lane == 0) r = wait_or_abort<kEpiPollNs>(smem_u32(&sh->full[b]), parity_of(g), args.timeout_ns, abort);
      if (!__shfl_sync(0xffffffffu, r ? 1 : 0, 0)) { ok = false; break; }
      __syncwarp();  // lane 0's wait acquired the MMA result (and StripInfo); this orders it for the warp
      const uint32_t tile = (uint32_t)(g % kTilesPerStrip);
      if (tile == 0) {
        const StripInfo& es = sh->estrip[(g / kTilesPerStrip) & 1];
        flags = es.flags;
        if (flags & kInfoDone) break;
        job = es.job;
        r0 = es.r0;
        cs = es.c0;
        n = es.n;
        nc = es.cols;
      }
      tc_fence_after();
      uint32_t v[kLoads][32];
#pragma unroll
      for (int h = 0; h < kLoads; ++h)
        tmem_ld32_nowait(tmem + ((uint32_t)(q * 32) << 16) + b * (uint32_t)kN + (uint32_t)(sub * kColsPerWarp + 32 * h),
                         v[h]);
      const unsigned long long c0 = cs + (unsigned long long)tile * kN;
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
      if (flags & kInfoFull) {
#pragma unroll
        for (int h = 0; h < kLoads; ++h)
#pragma unroll
          for (int u = 0; u < 32; ++u) red_shared(hist_lane + (v[h][u] << 11));
      } else {
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
  tc_fence_before();
  __syncthreads();
  if (warp == kIssuerWarp) {
    tc_fence_after();
    tmem_dealloc(tmem, kTmemCols);
  }
}

// ---------------------------------------------------------------- host side
// Bit planes of the operands of job j: the bits of A * (2^n - 1), which bounds
// every codeword of the job, rounded up to 4 (the kernel computes the same).
int mma_operand_bits(const Job& j) {
  int bits = 0;
  if (j.row_kind == ROW_HAMMING_EXT) {
    bits = (int)j.nbins - 1;  // extended Hamming codeword: n data + h check bits
  } else {
    const unsigned __int128 maxcw = (unsigned __int128)j.A * ((1ull << j.n) - 1ull);
    for (unsigned __int128 v = maxcw; v; v >>= 1) ++bits;
    if (bits == 0) bits = 1;
  }
  return (bits + 3) & ~3;
}

bool mma_eligible(const Job& j) {
  if (j.kind != JOB_PAIRS || j.n > 48) return false;
  const bool tri = j.shape == SHAPE_TRIANGLE && ((j.row_kind == ROW_PROGRESSION && j.col_kind == COL_PROGRESSION) ||
                                                 (j.row_kind == ROW_HAMMING_EXT && j.col_kind == COL_HAMMING_EXT));
  const bool rect = j.shape == SHAPE_RECT && (j.row_kind == ROW_PROGRESSION || j.row_kind == ROW_LATTICE) &&
                    (j.col_kind == COL_PROGRESSION || j.col_kind == COL_LATTICE) && j.col_tiles * kSuper >= j.cols;
  return (tri || rect) && mma_operand_bits(j) <= 60;
}

size_t mma_smem_bytes(uint32_t hist_rows, uint32_t b_bufs) {
  size_t s = (size_t)2 * kABytes + (size_t)b_bufs * kBBytes + (size_t)hist_rows * kEpiThreads * 4 + sizeof(Shared) + 64;
  return s < kMinSmem ? kMinSmem : s;
}

uint32_t mma_b_bufs(uint32_t hist_rows) {
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return 1;
  return mma_smem_bytes(hist_rows, 2) <= (size_t)optin ? 2u : 1u;
}

cudaError_t launch_mma(const MmaArgs& args, int grid, size_t smem, cudaStream_t stream) {
  cudaError_t e = cudaFuncSetAttribute(mma_hist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  mma_hist_kernel<<<grid, kThreads, smem, stream>>>(args);
  return cudaGetLastError();
}

}  // namespace dd
