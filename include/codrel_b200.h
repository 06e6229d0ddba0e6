/*
 * codrel_b200.h — C-ABI of the B200-native distance-distribution library.
 *
 * The library computes Hamming-distance histograms over the codewords of
 *   - AN codes:      cw(x) = A * x,            x in [0, 2^n)
 *   - Ext. Hamming:  cw(x) = x | parity bits,  x in [0, 2^n)
 * in exhaustive, 1-D/2-D grid and Monte Carlo modes, on one GPU.
 *
 * The reference tool (brics-db/coding_reliability, `distance_distribution`) has
 * no plugin/FFI layer: its boundary is the set of C++ driver functions declared
 * in distance_distribution/src/algorithms.h:20-34 and
 * distance_distribution_super_a/src/algorithms.h:20-21.  Every such driver does
 * (1) cudaMalloc + cudaMemset of <=64 uint64 bins, (2) one kernel launch per
 * device, (3) a D2H copy and host sum, (4) a host post-processing step.  The
 * entry points below replace steps (1)-(4) for one instance (dd_histogram), for
 * a batch of instances in one persistent launch (dd_batch_run), and for a
 * stream of queries (dd_server_*).  The C++ shims with the reference's own
 * names and signatures (codrel_dropin.h) sit on top of these.
 *
 * Conventions (all functions):
 *   - plain C types, caller-owned host buffers, no exit(): every call returns
 *     a dd_status; dd_last_error() gives a one-line message for the calling
 *     thread's last failure.  (The reference prints and exit()s through
 *     CHECK_ERROR, distance_distribution/lib/helper/inc/globals_cuda.h:42-74,
 *     and throws std::runtime_error for an unsupported n or bin count,
 *     src/an_coding.h:56, src/an_coding.cu:165.)
 *   - a dd_context owns one device, one CUDA stream and its device state; one
 *     context must not be used by two host threads at the same time, distinct
 *     contexts may.
 *   - uint128 counts are returned as (lo, hi) uint64 pairs.
 */
#ifndef CODREL_B200_H_
#define CODREL_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DD_MAX_BINS 64   /* COUNTS_MAX_WIDTH, distance_distribution_super_a/src/globals.h:44 */
#define DD_ABI_VERSION 1

typedef enum dd_status {
  DD_OK = 0,
  DD_ERR_INVALID_ARGUMENT = 1, /* malformed request (reference: assert / runtime_error) */
  DD_ERR_UNSUPPORTED = 2,      /* n or bin count outside what the kernels handle */
  DD_ERR_CUDA = 3,             /* a CUDA runtime call failed (reference: CHECK_ERROR -> exit) */
  DD_ERR_NO_DEVICE = 4,        /* no CUDA device / CUDA library not usable */
  DD_ERR_OUT_OF_MEMORY = 5,    /* device allocation failed or memory budget exceeded */
  DD_ERR_BUSY = 6,             /* server: admission refused (queue full) */
  DD_ERR_TIMEOUT = 7,          /* a bounded device-side wait ran out */
  DD_ERR_NOT_FOUND = 8,        /* server: unknown ticket */
  DD_ERR_CANCELLED = 9         /* server shut down before the query ran */
} dd_status;

typedef enum dd_code { DD_CODE_AN = 0, DD_CODE_EXT_HAMMING = 1 } dd_code;

typedef enum dd_mode {
  DD_MODE_EXHAUSTIVE = 0,  /* all pairs */
  DD_MODE_GRID_1D = 1,     /* codewords x lattice of m points (an_coding_grid.cu:60-114) */
  DD_MODE_GRID_2D = 2,     /* lattice of m2 points x lattice of m points (an_coding_grid.cu:121-140) */
  DD_MODE_MONTE_CARLO = 3  /* Philox4x32-10 sampled pairs (replaces cuRAND Sobol32) */
} dd_mode;

/* Which kernel family computes an AN exhaustive or grid histogram or an
 * Ext-Hamming all-pairs brute force (Monte Carlo, the Ext-Hamming weight
 * enumerator and anything wider than 60-bit operands use the popc kernel). */
typedef enum dd_kernel {
  DD_KERNEL_AUTO = 0,  /* autotuner's choice for the shape; jobs below 2^30 pairs stay on the popc
                          kernel, whose launch costs less than the tcgen05 kernel's fixed set-up */
  DD_KERNEL_POPC = 1,  /* XOR + POPC, warp-private shared-memory bins */
  DD_KERNEL_MMA = 2    /* tcgen05 kind::i8 bit-plane MMA, histogram epilogue from TMEM */
} dd_kernel;

/* Histogram epilogue of the tcgen05 kernel (dd_set_mma_epilogue). */
typedef enum dd_mma_epilogue {
  DD_MMA_EPILOGUE_AUTO = 0,    /* the autotuner's choice (paired until it has run) */
  DD_MMA_EPILOGUE_PAIRED = 1,  /* two codewords per MMA column: the accumulator is a packed distance
                                  pair, one shared-memory atomic per two pairs into a joint-bin table */
  DD_MMA_EPILOGUE_SINGLE = 2   /* one codeword per MMA column: one atomic per pair, per-thread bins */
} dd_mma_epilogue;

/* Ext-Hamming exhaustive algorithm (reference `-e` switch, src/main.cpp:245-268). */
typedef enum dd_hamming_method {
  DD_HAMMING_WEIGHTS = 0,   /* `-e 1`: weight enumerator x 2^n (src/hamming.cu:64-224) */
  DD_HAMMING_ALL_PAIRS = 1,  /* `-e 2` / `-e 4`: every ordered codeword pair incl. a==b
                                (+ the 1-bit spheres of the second codeword),
                                src/hamming_native_short.cpp:29-84, src/hamming_native.cpp:39-113 */
  DD_HAMMING_ALL_PAIRS_DISTINCT = 2  /* `-e 3`: pairs a<b (+ spheres of b), doubled; no a==b term,
                                        src/hamming_native_short_ordering.cpp:39-84 */
} dd_hamming_method;

/* Which reference driver's host conventions a request follows. */
typedef enum dd_convention {
  DD_CONV_GPU = 0,     /* run_ancoding & co (src/an_coding.cu:276-280): power-of-two A -> 1,
                          h = ceil(log(A)/log(2)), minb searched in [1, nbins/2) */
  DD_CONV_CPU = 1,     /* run_ancoding_cpu (src/an_coding.cpp:104-142): A kept as given */
  DD_CONV_SUPER_A = 2  /* super-A fork (super_a/src/an_coding.cu:135-244): h given by the caller
                          (floor(log(A)/log(2))+1), minb searched in [1, (nbins+1)/2) */
} dd_convention;

typedef struct dd_request {
  uint32_t code;            /* dd_code */
  uint32_t mode;            /* dd_mode */
  uint64_t A;               /* AN multiplier (ignored for Hamming); 0 is read as 1 (src/main.cpp:79) */
  uint32_t n;               /* data bits k */
  uint32_t h;               /* 0: derive as `convention` says; else the check-bit count to use */
  uint64_t m;               /* grid points (1st dim) / Monte Carlo iterations */
  uint64_t m2;              /* 2-D grid: points of the 2nd dim (0 -> m, src/main.cpp:127-128) */
  uint64_t seed;            /* Monte Carlo: Philox key */
  uint32_t with_1bit;       /* Ext-Hamming: add the 1-bit spheres (`-b`) */
  uint32_t hamming_method;  /* dd_hamming_method */
  uint32_t kernel;          /* dd_kernel */
  uint32_t convention;      /* dd_convention */
  uint64_t user_tag;        /* opaque, copied to the result */
} dd_request;

typedef struct dd_result {
  uint32_t status;          /* dd_status of this instance */
  uint32_t nbins;           /* n + h + 1 */
  uint32_t h;               /* check bits used */
  uint32_t kernel_used;     /* dd_kernel that ran */
  uint64_t A;               /* A after the convention's normalisation */
  uint64_t iterations;      /* m after capping at 2^n (grid / MC), else 0 */
  uint64_t iterations2;     /* m2 after capping (2-D grid), else 0 */
  uint64_t pairs_lo, pairs_hi;  /* distance evaluations the device performed (uint128) */
  uint64_t raw[DD_MAX_BINS];    /* device histogram of every evaluated pair (the reference's host-summed
                                   hcounts[0][]); 2-D grids: bin 0 holds the coincident lattice points,
                                   which dancoding_grid_2d never flushes and counts[0] leaves out */
  uint64_t counts_lo[DD_MAX_BINS];  /* post-processed uint128 counts[] (lo 64 bits) */
  uint64_t counts_hi[DD_MAX_BINS];  /*                                  (hi 64 bits) */
  uint64_t minb;            /* first non-zero bin in the convention's range, 0xFFFF if none */
  uint64_t mincb_lo, mincb_hi;
  double max_rel_error;     /* get_rel_error_AN / get_abs_error_hamming as the driver returns it,
                               -1 when the reference has no golden table for (A, n) */
  double kernel_ms;         /* device time of the histogram kernel(s), CUDA events */
  double total_ms;          /* host wall time of the whole call */
  uint64_t user_tag;
  uint32_t mma_epilogue;    /* dd_mma_epilogue that ran when kernel_used is DD_KERNEL_MMA, else 0 */
  uint32_t reserved;
} dd_result;

typedef struct dd_context dd_context;

/* --- library ---------------------------------------------------------- */
const char* dd_version(void);
const char* dd_status_string(int status);
/* Message of the calling thread's last failed call ("" if none). */
const char* dd_last_error(void);
/* Number of CUDA devices (0 when none / no driver). Never fails. */
int dd_device_count(void);

/* --- contexts ----------------------------------------------------------- */
/* device: CUDA ordinal.  stream: a cudaStream_t to issue all work on, or NULL
 * for a stream the context creates and owns. */
int dd_context_create(int device, void* stream, dd_context** out);
int dd_context_destroy(dd_context* ctx);

/* --- one instance ------------------------------------------------------- */
/* Computes one histogram synchronously: launch on the context's stream,
 * D2H of the raw bins, host post-processing.  Replaces run_ancoding,
 * run_ancoding_grid, run_ancoding_mc (src/an_coding*.cu), run_hamming,
 * run_hamming_grid, run_hamming_mc (src/hamming*.cu), run_ancoding_cpu
 * (src/an_coding.cpp:104), run_hamming_cpu* (src/hamming*.cpp) and the
 * super-A run_ancoding (super_a/src/an_coding.cu:135). */
int dd_histogram(dd_context* ctx, const dd_request* req, dd_result* res);

/* One part of a request's work: the tiles [tile_begin, tile_begin + tile_count)
 * of its tile space (dd_request_plan's `tiles`), computed on the context's GPU
 * and ADDED to raw[0 .. n+h+1) (nraw >= n+h+1).  Disjoint parts that cover the
 * tile space sum to the raw histogram of dd_histogram, bit for bit, whatever
 * their sizes, order, kernels or GPUs; dd_postprocess turns the sum into the
 * result.  So a long run can stop between parts and resume from (next tile,
 * raw) - the state the reference keeps in one kernel launch of up to hours
 * (src/an_coding.cu:243-282) - and one instance can be split over GPUs with
 * a host-side sum.  kernel_ms (may be NULL): device time of the part. */
int dd_histogram_part(dd_context* ctx, const dd_request* req, uint64_t tile_begin, uint64_t tile_count,
                      uint64_t* raw, uint32_t nraw, double* kernel_ms);

/* The plain one-launch-per-instance baseline for AN exhaustive requests: the
 * reference's design on this GPU (src/an_coding.cu:50-105 + :276-421): bins
 * allocated and freed per call, a grid-stride kernel of 128 CTAs per SM with
 * per-thread shared-memory bins, one launch, a D2H copy.  It is what the
 * persistent and batched paths are measured against; results are identical. */
int dd_histogram_plain(dd_context* ctx, const dd_request* req, dd_result* res);

/* --- no device allocation ------------------------------------------------ */
/* Has no counterpart in the reference.  For callers that cannot allocate
 * device memory (a host application that owns every device allocation through
 * its own pool, a plugin inside such a host, a device whose memory is fully
 * reserved): computes up to 32 histograms in one popc-path launch on `device`
 * and `stream` (NULL: the default stream) without calling cudaMalloc, cudaFree
 * or any allocating routine.  The kernel's scratch (bins, job table, work
 * counter, status word) is one fixed 21 KB __device__ array that every GPU
 * loading the library holds until exit; more than 32 requests per call are
 * refused with DD_ERR_INVALID_ARGUMENT.  Every call looks up the array's
 * device address on `device`; the first call on a device also loads the
 * module there and should come before any stream capture on that device.  The
 * caller's current device is restored before the call returns.  All calls
 * share the array: calls that overlap on the GPU race and must be serialised
 * by the caller.  Results equal dd_histogram's; kernel_ms is 0 (no events are
 * created). */
int dd_histogram_noalloc(int device, void* stream, const dd_request* reqs, uint32_t count, dd_result* results);

/* Monte Carlo continued (AN codes): the result of `req` (req->m samples per
 * codeword) computed from the first it_done samples, whose device histogram
 * the caller passes in raw_done (dd_result.raw of the earlier run with
 * m = it_done, same A, n and seed), plus only the samples [it_done, req->m).
 * A codeword's t-th sample depends on (seed, codeword, t) alone, so the result
 * is bit-identical to dd_histogram(req).  This lets an error-bound search
 * (the reference's ancoding_mc_search, src/main.cpp:179-202, which restarts
 * with 3x the iterations) grow the sample count without redrawing. */
int dd_mc_extend(dd_context* ctx, const dd_request* req, uint64_t it_done, const uint64_t* raw_done, dd_result* res);

/* --- batch -------------------------------------------------------------- */
typedef struct dd_batch_options {
  uint32_t use_graph;       /* capture the launch in a CUDA graph and replay it */
  uint32_t kernel;          /* dd_kernel for every AN exhaustive / grid instance (AUTO: autotuner) */
  uint32_t ctas_per_sm;     /* 0: autotuner */
  uint32_t reserved;
} dd_batch_options;

/* Runs `count` AN exhaustive instances (any mix of A and n) in ONE persistent
 * launch.  Replaces the super-A sweeps' sequential run_ancoding calls
 * (src/main.cpp:131-177, super_a/src/main.cpp:194-297).  Non-exhaustive or
 * Hamming requests in the batch are run one after the other on the stream. */
int dd_batch_run(dd_context* ctx, const dd_request* reqs, uint32_t count,
                 dd_result* results, const dd_batch_options* opts);

/* --- query server (continuous batching) --------------------------------- */
/* A server admits distance-distribution queries as they arrive.  Each admitted
 * query holds a resident slot (its uint64 bins and its pair-space cursor) on
 * the device; a scheduler thread runs rounds, each ONE persistent launch over a
 * fair share of every active query's remaining tiles, so queries that arrive
 * while others run join the next round and their work overlaps on the GPU.
 * Queries beyond the slots wait in a bounded queue; beyond the queue,
 * dd_server_submit returns DD_ERR_BUSY.  Results are identical to dd_histogram's.
 * dd_server_create runs the autotuner on the server's own context (about a
 * second), so KERNEL_AUTO queries run on the kernel measured fastest there.
 * No counterpart in the reference (its drivers run one query per process). */
typedef struct dd_server dd_server;

typedef struct dd_server_options {
  uint64_t memory_budget_bytes; /* device bytes for resident query state; 0 = 64 MiB */
  uint32_t max_queue;           /* queries waiting for a slot before submit refuses; 0 = 1024 */
  uint32_t round_ms;            /* target device time of one round; 0 = 20 ms */
  uint32_t dry_run;             /* 1: schedule without a device (rounds advance cursors only,
                                   results carry zero bins) - for tests of the host logic */
  uint32_t inject_alloc_failure;/* test hook: 1 = the slot allocation fails */
} dd_server_options;

typedef struct dd_server_stats {
  uint64_t submitted, admitted, completed, rejected, cancelled, rounds;
  uint32_t active, queued, slots, slots_free;
  double p50_ms, p99_ms;        /* latency from submit to result, the last 65536 completed queries */
  double pairs_per_s;           /* distance evaluations of completed queries / busy device time */
  double busy_ms;               /* device time of all rounds */
  uint64_t pairs_lo, pairs_hi;  /* distance evaluations of completed queries (uint128) */
} dd_server_stats;

int dd_server_create(int device, const dd_server_options* opts, dd_server** out);
/* Validates and enqueues; *ticket identifies the query. */
int dd_server_submit(dd_server* s, const dd_request* req, uint64_t* ticket);
/* *done = 1 and *res filled once the query finished (res->status tells how). */
int dd_server_poll(dd_server* s, uint64_t ticket, dd_result* res, int* done);
/* Blocks up to timeout_s seconds (< 0: no limit); DD_ERR_TIMEOUT if still running. */
int dd_server_wait(dd_server* s, uint64_t ticket, double timeout_s, dd_result* res);
/* Result retention: a finished query's result is kept until it has been delivered
 * (dd_server_wait returned it, dd_server_poll reported it done with a result
 * buffer, or its client cancelled it); the 4096 most recently delivered results
 * stay answerable, older ones are dropped (never while a thread waits on them)
 * and their tickets then give DD_ERR_NOT_FOUND.  dd_server_release drops a
 * finished query's result at once (DD_ERR_BUSY while it runs or is waited on). */
int dd_server_release(dd_server* s, uint64_t ticket);
/* A client that goes away: a queued query is dropped, an active one stops after
 * the current round and frees its slot; its result status is DD_ERR_CANCELLED. */
int dd_server_cancel(dd_server* s, uint64_t ticket);
int dd_server_get_stats(dd_server* s, dd_server_stats* out);
/* Stops the scheduler: unfinished queries end with DD_ERR_CANCELLED, which
 * wakes every thread blocked in dd_server_wait; later submits are refused.  The
 * handle stays valid (wait / poll / stats still answer) until dd_server_destroy. */
int dd_server_shutdown(dd_server* s);
/* dd_server_shutdown, then frees the server once every call still inside it
 * (a waiter it woke) has returned.  No call may start after this one. */
int dd_server_destroy(dd_server* s);

/* --- host-only helpers (no device needed) ------------------------------- */
/* Derives nbins/h/A for a request exactly as the reference's drivers do. */
int dd_request_shape(const dd_request* req, uint32_t* nbins, uint32_t* h, uint64_t* A_eff);
/* The device work a request plans: lattice points the grid modes visit (the
 * reference's walk, src/an_coding_grid.cu:78-107), work tiles of the popc
 * kernel, and distance evaluations (uint128 as lo/hi).  Any pointer may be NULL. */
int dd_request_plan(const dd_request* req, uint64_t* lattice, uint64_t* tiles, uint64_t* pairs_lo,
                    uint64_t* pairs_hi);
/* The reference's post-processing of a raw device histogram into counts[],
 * minb/mincb and the error estimate (the host tail of every run_* driver). */
int dd_postprocess(const dd_request* req, const uint64_t* raw, uint32_t nraw, dd_result* res);
/* Renders a result in the reference's results-file layout
 * (process_result, src/globals.cpp:185-305): writes at most cap bytes
 * (NUL-terminated) and stores the full length in *len.  `device_line` is
 * appended as the reference appends its "Device" lines (may be NULL). */
int dd_format_result(const dd_request* req, const dd_result* res, const char* device_line,
                     char* buf, size_t cap, size_t* len);
/* Philox4x32-10 (Salmon et al., SC'11), the counter-based generator behind
 * Monte Carlo mode: out = philox(ctr, key). */
void dd_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* --- autotuning --------------------------------------------------------- */
typedef struct dd_tuning {
  uint32_t kernel;            /* dd_kernel chosen for AN exhaustive requests with kernel = AUTO */
  uint32_t hist_mode;         /* popc path bin increment: 0 = red.shared.add, 1 = load/add/store */
  double popc_red_pairs_per_s;
  double popc_ldst_pairs_per_s;
  double mma_pairs_per_s;     /* tcgen05, single epilogue */
  uint64_t probe_pairs;       /* pairs of the probe instance each variant ran */
  double mma_paired_pairs_per_s;  /* tcgen05, paired epilogue */
  uint32_t mma_epilogue;      /* dd_mma_epilogue chosen for the tcgen05 kernel */
  uint32_t reserved;
} dd_tuning;

/* Times every kernel variant (popc with either bin increment, tcgen05 with
 * either epilogue) on a probe instance (A = 65521, k = 20: 36-bit codewords,
 * 5.5e11 pairs, about a second in all) on this context's GPU and keeps the
 * fastest for kernel = AUTO, and the faster tcgen05 epilogue for the
 * tcgen05 kernel.  Runs by itself before the first large AUTO request. */
int dd_autotune(dd_context* ctx, dd_tuning* out);

/* Epilogue of this context's tcgen05 launches (dd_mma_epilogue): AUTO follows
 * the autotuner; PAIRED and SINGLE fix it (for measurements and tests).  Both
 * give the identical histogram. */
int dd_set_mma_epilogue(dd_context* ctx, uint32_t epilogue);

/* --- measurement -------------------------------------------------------- */
/* Measures the device's POPC issue rate (popc/s) with a dependency-free POPC
 * loop on the context's stream. */
int dd_measure_popc_peak(dd_context* ctx, double* popc_per_s);
/* One point of the shared-memory atomic sweep: red.shared.add.u32 per second
 * on every SM, one CTA of warps_per_sm warps each, 32 independent adds per
 * loop iteration, conflict-free within each warp.  pattern 0: every thread
 * its own column of 32 rows (the single tcgen05 epilogue's bins); pattern 1:
 * one column per lane shared by every warp of the CTA, 1024 cells (the paired
 * epilogue's joint table). */
typedef struct dd_red_probe {
  uint32_t warps_per_sm;
  uint32_t pattern;
  double adds_per_s;
} dd_red_probe;

/* Runs the sweep (warps per SM 8, 12, ..., 32 for each pattern, best of three
 * launches each) and writes up to cap points; *count = points written. */
int dd_measure_red_sweep(dd_context* ctx, dd_red_probe* out, uint32_t cap, uint32_t* count);
/* The maximum of that sweep: the device's shared-memory atomic rate, the
 * bound of the tcgen05 path's histogram epilogue. */
int dd_measure_red_peak(dd_context* ctx, double* adds_per_s);

/* --- failure detection -------------------------------------------------- */
/* Bound (ns) of every device-side wait of this context's tcgen05 launches;
 * 0 restores the default of 2 s.  A wait that runs out makes the kernel stop,
 * release its tensor memory and report DD_ERR_TIMEOUT; the context stays
 * usable.  A very short bound makes the first wait run out, which is how the
 * timeout path is tested without a fault or a hang. */
int dd_set_wait_timeout(dd_context* ctx, uint64_t ns);

/* --- super-A candidates --------------------------------------------------- */
/* Replaces the worker loop of ANcandidates (ANcandidates/ANcandidates.cpp:35-163,
 * main :236-301): for every odd A with exactly a_bits bits the smallest
 * signed-digit weight popcount(A·x XOR 3·A·x) over x in [1, 2^k), and the A
 * values whose weight is the largest of the range (the candidates). */
typedef struct dd_candidates_result {
  int32_t status;
  uint32_t k;               /* data bits */
  uint32_t a_bits;          /* bit width of A */
  uint32_t sdr;             /* the candidates' weight (the reference's |SDR|) */
  uint64_t num_A;           /* odd A values scanned */
  uint64_t num_candidates;  /* all candidates, also when more than fit the list */
  uint64_t evaluations;     /* codewords weighed (the early exit skips the rest) */
  double kernel_ms;
  double total_ms;
} dd_candidates_result;

/* Writes min(num_candidates, capacity) candidates to out_A in ascending order
 * (the smallest ones when the list is too short).  1 <= k <= 48,
 * 1 <= a_bits <= 32, k + a_bits <= 61; a_bits = 1 has no odd A (sdr 0, no
 * candidates), as in the reference. */
int dd_an_candidates(dd_context* ctx, uint32_t k, uint32_t a_bits, uint64_t* out_A, uint64_t capacity,
                     dd_candidates_result* res);

#ifdef __cplusplus
}
#endif
#endif /* CODREL_B200_H_ */
