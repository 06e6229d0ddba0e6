// dd_host.cu — C-ABI implementation: contexts, launches, batches, graphs.
//
// The reference crosses the host/device boundary once per driver call:
// cudaMalloc + cudaMemset of the bins, one launch per device, a D2H copy and a
// host sum, then cudaDeviceReset (src/an_coding.cu:320-421).  Here a context
// keeps its device buffers resident across calls, one launch serves any number
// of instances, and the only per-call traffic is the job table (H2D) and the
// raw bins (D2H), both through pinned host buffers on the context's stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/codrel_b200.h"
#include "dd_device.cuh"
#include "dd_host.h"
#include "dd_kernels.h"
#include "dd_mma.h"

struct dd_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int num_sms = 0;
  // device state
  unsigned long long* d_bins = nullptr;  // bin_slots x kMaxBins
  uint32_t bin_slots = 0;
  unsigned long long* d_ctl = nullptr;   // [0] popc work counter, [1] MMA work counter, [2] status, [3..15] diagnostics
  dd::Job* d_jobs = nullptr;
  uint32_t job_cap = 0;
  // pinned host mirrors
  unsigned long long* h_bins = nullptr;
  unsigned long long* h_ctl = nullptr;
  dd::Job* h_jobs = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // tuning
  int hist_mode = dd::HIST_RED;
  int tuned = 0;
  uint32_t mma_epilogue = DD_MMA_EPILOGUE_AUTO;         // requested (dd_set_mma_epilogue)
  uint32_t mma_tuned_epilogue = DD_MMA_EPILOGUE_PAIRED;  // the autotuner's verdict for AUTO
  unsigned long long mma_timeout_ns = 2000000000ull;  // bound of every device-side wait
  // batch graph cache
  cudaGraphExec_t gexec = nullptr;
  std::vector<dd::Job> gjobs;  // job table the cached graph was built for
  int ggrid[2] = {0, 0};
  size_t gsmem[2] = {0, 0};
  int ghist_mode = 0;                  // popc bin-increment form the graph launches
  unsigned long long gtimeout_ns = 0;  // device-side wait bound baked into the graph
};

namespace dd {

constexpr int kCtlWords = 16;
static thread_local std::string t_last_error;
void set_error(const std::string& msg) { t_last_error = msg; }

static int cuda_fail(cudaError_t e, const char* what) {
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return DD_ERR_CUDA;
}

#define DD_CUDA(call)                                   \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

// The cached launch graph's copy nodes and kernel arguments point at these
// buffers, so it is dropped whenever one of them is reallocated (no graph is in
// flight here: every launch is synchronised before its call returns).
static void drop_graph(dd_context* ctx) {
  if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
  ctx->gexec = nullptr;
  ctx->gjobs.clear();
}

static int ensure_capacity(dd_context* ctx, uint32_t slots, uint32_t njobs) {
  DD_CUDA(cudaSetDevice(ctx->device));
  if (slots > ctx->bin_slots || njobs > ctx->job_cap) drop_graph(ctx);
  if (slots > ctx->bin_slots) {
    if (ctx->d_bins) cudaFree(ctx->d_bins);
    if (ctx->h_bins) cudaFreeHost(ctx->h_bins);
    ctx->d_bins = nullptr;
    ctx->h_bins = nullptr;
    ctx->bin_slots = 0;
    const uint32_t cap = std::max<uint32_t>(slots, 64);
    cudaError_t e = cudaMalloc(&ctx->d_bins, (size_t)cap * kMaxBins * sizeof(unsigned long long));
    if (e != cudaSuccess) { set_error("bins: cudaMalloc failed"); return DD_ERR_OUT_OF_MEMORY; }
    DD_CUDA(cudaMallocHost(&ctx->h_bins, (size_t)cap * kMaxBins * sizeof(unsigned long long)));
    ctx->bin_slots = cap;
  }
  if (njobs > ctx->job_cap) {
    if (ctx->d_jobs) cudaFree(ctx->d_jobs);
    if (ctx->h_jobs) cudaFreeHost(ctx->h_jobs);
    ctx->d_jobs = nullptr;
    ctx->h_jobs = nullptr;
    ctx->job_cap = 0;
    const uint32_t cap = std::max<uint32_t>(njobs, 64);
    cudaError_t e = cudaMalloc(&ctx->d_jobs, (size_t)cap * sizeof(Job));
    if (e != cudaSuccess) { set_error("jobs: cudaMalloc failed"); return DD_ERR_OUT_OF_MEMORY; }
    DD_CUDA(cudaMallocHost(&ctx->h_jobs, (size_t)cap * sizeof(Job)));
    ctx->job_cap = cap;
  }
  return DD_OK;
}

struct LaunchPlan {
  LaunchArgs pargs;          // popc kernel: table entries [0, npopc)
  int pgrid = 0;
  size_t psmem = 0;
  uint32_t npopc = 0;
  MmaArgs margs;             // MMA kernel: table entries [npopc, npopc + nmma)
  int mgrid = 0;
  size_t msmem = 0;
  uint32_t nmma = 0;
  uint32_t nslots = 0;       // bin slots (one per request, in request order)
};

// Epilogue of the context's tcgen05 launches.
static uint32_t mma_epilogue_of(const dd_context* ctx) {
  return ctx->mma_epilogue == DD_MMA_EPILOGUE_AUTO ? ctx->mma_tuned_epilogue : ctx->mma_epilogue;
}

// Jobs below this many distance evaluations stay on the popc kernel under
// AUTO: the tcgen05 kernel's fixed cost per launch (TMEM allocation, clearing
// its ~180 KB of shared-memory table, barrier set-up) outweighs its rate there
// (A = 641, k = 12, 8.4e6 pairs: popc 0.09 ms, tcgen05 0.44 ms; k = 16, 2.1e9
// pairs, one launch each: tcgen05 0.41 ms, popc 0.57 ms).
constexpr double kMmaMinPairs = 1073741824.0;  // 2^30

// Which kernel runs a job: explicit MMA or POPC requests are honoured where
// the job allows them; AUTO uses the context's measured preference for jobs
// large enough to amortise the tcgen05 kernel's launch.
static bool want_mma(const dd_context* ctx, const Job& j, uint32_t kernel) {
  if (!mma_eligible(j)) return false;
  if (kernel == DD_KERNEL_MMA) return true;
  if (kernel == DD_KERNEL_POPC) return false;
  const double pairs = j.shape == SHAPE_TRIANGLE ? 0.5 * (double)j.rows * (double)j.rows
                                                 : (double)j.rows * (double)j.cols;
  return ctx->tuned == 2 && pairs >= kMmaMinPairs;  // autotuner's verdict for AN exhaustive shapes
}

// Orders the job table (popc jobs first, then MMA jobs), assigns tile ranges
// and bin slots (slot = request index), and sizes both persistent grids.
static int plan_launch(dd_context* ctx, std::vector<Job>& jobs, const std::vector<uint32_t>& kernels,
                       LaunchPlan& lp, bool own_bins = true) {
  std::vector<Job> table;
  table.reserve(jobs.size());
  for (int pass = 0; pass < 2; ++pass)
    for (size_t i = 0; i < jobs.size(); ++i) {
      const bool m = want_mma(ctx, jobs[i], kernels[i]);
      if ((pass == 1) != m) continue;
      Job j = jobs[i];
      if (own_bins) j.bins = ctx->d_bins + i * kMaxBins;
      table.push_back(j);
    }
  lp.nslots = (uint32_t)jobs.size();
  uint64_t tp = 0, tm = 0;
  uint32_t maxb = 1, maxbm = 1;
  bool col_table = false;
  lp.npopc = 0;
  for (size_t i = 0; i < jobs.size(); ++i) lp.npopc += want_mma(ctx, jobs[i], kernels[i]) ? 0 : 1;
  lp.nmma = (uint32_t)table.size() - lp.npopc;
  for (uint32_t k = 0; k < lp.npopc; ++k) {
    Job& j = table[k];
    j.tile_begin = tp;
    tp += j.tiles;
    maxb = std::max(maxb, j.nbins);
    col_table |= (j.kind == JOB_PAIRS && j.col_kind == COL_HAMMING_EXT && !j.wide);
  }
  for (uint32_t k = lp.npopc; k < table.size(); ++k) {
    Job& j = table[k];
    j.tile_begin = tm;
    tm += j.tiles;
    maxbm = std::max(maxbm, j.nbins);
  }
  unsigned* status = reinterpret_cast<unsigned*>(ctx->d_ctl + 2);
  lp.pargs.jobs = ctx->d_jobs;
  lp.pargs.njobs = lp.npopc;
  lp.pargs.smem_bins = maxb;
  lp.pargs.total_tiles = tp;
  lp.pargs.counter = ctx->d_ctl;
  lp.pargs.status = status;
  lp.pargs.use_col_table = col_table ? 1u : 0u;
  lp.pargs.pad = 0;
  if (lp.npopc && tp) {
    lp.psmem = hist_smem_bytes(maxb, col_table);
    int occ = 0;
    DD_CUDA(hist_occupancy(ctx->hist_mode, lp.psmem, &occ));
    if (occ < 1) { set_error("kernel does not fit on an SM"); return DD_ERR_UNSUPPORTED; }
    const uint64_t want = (tp + kWarpsPerCta - 1) / kWarpsPerCta;
    lp.pgrid = (int)std::min<uint64_t>((uint64_t)ctx->num_sms * occ, std::max<uint64_t>(want, 1));
  }
  lp.margs.jobs = ctx->d_jobs + lp.npopc;
  lp.margs.njobs = lp.nmma;
  // rows for every distance an operand can produce (<= L), flagged at flush when >= nbins
  uint32_t maxl = 0;
  for (uint32_t k = lp.npopc; k < table.size(); ++k) maxl = std::max(maxl, (uint32_t)mma_operand_bits(table[k]));
  lp.margs.hist_rows = std::max(maxbm, maxl + 1);
  lp.margs.total_tiles = tm;
  lp.margs.counter = ctx->d_ctl + 1;
  lp.margs.status = status;
  lp.margs.timeout_ns = ctx->mma_timeout_ns;
  lp.margs.packed = mma_epilogue_of(ctx) == DD_MMA_EPILOGUE_PAIRED ? 1u : 0u;
  lp.margs.pk_cells = 0;
  lp.margs.pad = 0;
  if (lp.nmma && tm) {
    if (lp.margs.packed) {
      // one joint table for the launch, sized for its largest S; each job's
      // window of d2 rows and its packing parameters follow from it
      uint32_t smax = 1;
      for (uint32_t k = lp.npopc; k < table.size(); ++k)
        smax = std::max(smax, (uint32_t)mma_max_distance(table[k]) + 1u);
      mma_pk_layout(smax, &lp.margs.pk_cells, &lp.margs.b_bufs);
      for (uint32_t k = lp.npopc; k < table.size(); ++k) mma_pack_setup(table[k], lp.margs.pk_cells);
    } else {
      lp.margs.b_bufs = mma_b_bufs(lp.margs.hist_rows);
    }
    lp.msmem = mma_smem_bytes(lp.margs.hist_rows, lp.margs.b_bufs, lp.margs.packed != 0, lp.margs.pk_cells);
    lp.mgrid = (int)std::min<uint64_t>((uint64_t)ctx->num_sms, tm);  // one CTA (one TMEM owner) per SM
  }
  std::memcpy(ctx->h_jobs, table.data(), table.size() * sizeof(Job));
  return DD_OK;
}

// Enqueues: job table H2D, bins / counters / status reset, kernels (bracketed
// by events), bins + status D2H.
static int enqueue_launch(dd_context* ctx, const LaunchPlan& lp, bool capturing) {
  cudaStream_t s = ctx->stream;
  const uint32_t njobs = lp.npopc + lp.nmma;
  DD_CUDA(cudaMemcpyAsync(ctx->d_jobs, ctx->h_jobs, njobs * sizeof(Job), cudaMemcpyHostToDevice, s));
  DD_CUDA(cudaMemsetAsync(ctx->d_bins, 0, (size_t)lp.nslots * kMaxBins * sizeof(unsigned long long), s));
  DD_CUDA(cudaMemsetAsync(ctx->d_ctl, 0, kCtlWords * sizeof(unsigned long long), s));
  // Inside a stream capture the records must be external so that they become
  // event-record nodes of the graph (the kernel time is then measurable on
  // every replay); outside a capture the flag is not accepted.
  const unsigned evflags = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
  DD_CUDA(cudaEventRecordWithFlags(ctx->ev0, s, evflags));
  if (lp.pgrid) DD_CUDA(launch_hist(ctx->hist_mode, lp.pargs, lp.pgrid, lp.psmem, s));
  if (lp.mgrid) DD_CUDA(launch_mma(lp.margs, lp.mgrid, lp.msmem, s));
  DD_CUDA(cudaEventRecordWithFlags(ctx->ev1, s, evflags));
  DD_CUDA(cudaMemcpyAsync(ctx->h_bins, ctx->d_bins, (size_t)lp.nslots * kMaxBins * sizeof(unsigned long long),
                          cudaMemcpyDeviceToHost, s));
  DD_CUDA(cudaMemcpyAsync(ctx->h_ctl, ctx->d_ctl, kCtlWords * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  return DD_OK;
}

// Status word of the last launch (after the stream synchronised).
static int check_status(dd_context* ctx) {
  const unsigned st = (unsigned)ctx->h_ctl[2];
  if (st & 8u) {
    char buf[256];
    std::snprintf(buf, sizeof(buf), "self-check: shared access at %llu outside [%llu, %llu), tile %llu",
                  ctx->h_ctl[4], ctx->h_ctl[5], ctx->h_ctl[6], ctx->h_ctl[7]);
    set_error(buf);
    return DD_ERR_CUDA;
  }
  if (st & KSTATUS_TIMEOUT) { set_error("a device-side wait timed out"); return DD_ERR_TIMEOUT; }
  if (st & KSTATUS_BAD_DISTANCE) { set_error("kernel produced a distance outside the bins"); return DD_ERR_CUDA; }
  if (st & KSTATUS_BAD_JOB) { set_error("kernel saw a tile outside the job table"); return DD_ERR_CUDA; }
  return DD_OK;
}

// One launch over job sub-ranges whose bins live in caller-owned device
// memory (the server's resident slots): the bins are NOT reset, so successive
// rounds accumulate; only the control block is reset and read back.
int launch_round(dd_context* ctx, std::vector<Job>& jobs, const std::vector<uint32_t>& kernels, float* kernel_ms) {
  int st = ensure_capacity(ctx, 1, (uint32_t)jobs.size());
  if (st != DD_OK) return st;
  LaunchPlan lp;
  st = plan_launch(ctx, jobs, kernels, lp, false);
  if (st != DD_OK) return st;
  cudaStream_t s = ctx->stream;
  const uint32_t njobs = lp.npopc + lp.nmma;
  DD_CUDA(cudaMemcpyAsync(ctx->d_jobs, ctx->h_jobs, njobs * sizeof(Job), cudaMemcpyHostToDevice, s));
  DD_CUDA(cudaMemsetAsync(ctx->d_ctl, 0, kCtlWords * sizeof(unsigned long long), s));
  DD_CUDA(cudaEventRecord(ctx->ev0, s));
  if (lp.pgrid) DD_CUDA(launch_hist(ctx->hist_mode, lp.pargs, lp.pgrid, lp.psmem, s));
  if (lp.mgrid) DD_CUDA(launch_mma(lp.margs, lp.mgrid, lp.msmem, s));
  DD_CUDA(cudaEventRecord(ctx->ev1, s));
  DD_CUDA(cudaMemcpyAsync(ctx->h_ctl, ctx->d_ctl, kCtlWords * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  DD_CUDA(cudaStreamSynchronize(s));
  st = check_status(ctx);
  if (st != DD_OK) return st;
  if (kernel_ms) DD_CUDA(cudaEventElapsedTime(kernel_ms, ctx->ev0, ctx->ev1));
  return DD_OK;
}

bool uses_mma(const dd_context* ctx, const Job& j, uint32_t kernel) { return want_mma(ctx, j, kernel); }
uint32_t mma_epilogue_used(const dd_context* ctx) { return mma_epilogue_of(ctx); }
void* context_stream(const dd_context* ctx) { return (void*)ctx->stream; }
int context_device(const dd_context* ctx) { return ctx->device; }

static double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

static void fill_pairs(dd_result& r, u128 p) {
  r.pairs_lo = (uint64_t)p;
  r.pairs_hi = (uint64_t)(p >> 64);
}

}  // namespace dd

using namespace dd;

extern "C" {

const char* dd_version(void) { return "coding_reliability_b200 0.1 (sm_100a)"; }

const char* dd_status_string(int status) {
  switch (status) {
    case DD_OK: return "ok";
    case DD_ERR_INVALID_ARGUMENT: return "invalid argument";
    case DD_ERR_UNSUPPORTED: return "unsupported";
    case DD_ERR_CUDA: return "cuda error";
    case DD_ERR_NO_DEVICE: return "no device";
    case DD_ERR_OUT_OF_MEMORY: return "out of memory";
    case DD_ERR_BUSY: return "busy";
    case DD_ERR_TIMEOUT: return "timeout";
    case DD_ERR_NOT_FOUND: return "not found";
    case DD_ERR_CANCELLED: return "cancelled";
    default: return "unknown status";
  }
}

const char* dd_last_error(void) { return t_last_error.c_str(); }

int dd_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int dd_context_create(int device, void* stream, dd_context** out) {
  if (!out) { set_error("out is NULL"); return DD_ERR_INVALID_ARGUMENT; }
  *out = nullptr;
  int ndev = dd_device_count();
  if (ndev == 0) { set_error("no CUDA device"); return DD_ERR_NO_DEVICE; }
  if (device < 0 || device >= ndev) { set_error("device ordinal out of range"); return DD_ERR_INVALID_ARGUMENT; }
  dd_context* ctx = new dd_context();
  ctx->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) {
    // sm_100a code is arch-specific: it runs on compute capability 10.0 only
    int major = 0, minor = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
    cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device);
    if (major != 10 || minor != 0) {
      delete ctx;
      set_error("this library is built for sm_100a (B200) only");
      return DD_ERR_NO_DEVICE;
    }
  }
  if (e == cudaSuccess) {
    if (stream) ctx->stream = (cudaStream_t)stream;
    else { e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking); ctx->own_stream = true; }
  }
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_ctl, kCtlWords * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMallocHost(&ctx->h_ctl, kCtlWords * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev1);
  if (e != cudaSuccess) {
    set_error(std::string("context setup: ") + cudaGetErrorString(e));
    dd_context_destroy(ctx);
    return DD_ERR_CUDA;
  }
  int st = ensure_capacity(ctx, 64, 64);
  if (st != DD_OK) { dd_context_destroy(ctx); return st; }
  // Tuning override for measurements: CODREL_B200_HIST_MODE=red|ldst picks how
  // a lane bumps its shared-memory bin (default: red.shared.add).
  if (const char* m = std::getenv("CODREL_B200_HIST_MODE")) {
    if (std::strcmp(m, "ldst") == 0) ctx->hist_mode = HIST_LDST;
    else if (std::strcmp(m, "red") == 0) ctx->hist_mode = HIST_RED;
  }
  *out = ctx;
  return DD_OK;
}

int dd_context_destroy(dd_context* ctx) {
  if (!ctx) return DD_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
  if (ctx->d_bins) cudaFree(ctx->d_bins);
  if (ctx->d_ctl) cudaFree(ctx->d_ctl);
  if (ctx->h_ctl) cudaFreeHost(ctx->h_ctl);
  if (ctx->d_jobs) cudaFree(ctx->d_jobs);
  if (ctx->h_bins) cudaFreeHost(ctx->h_bins);
  if (ctx->h_jobs) cudaFreeHost(ctx->h_jobs);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return DD_OK;
}

int dd_request_shape(const dd_request* req, uint32_t* nbins, uint32_t* h, uint64_t* A_eff) {
  if (!req) { set_error("req is NULL"); return DD_ERR_INVALID_ARGUMENT; }
  Shape s;
  std::string err;
  int st = derive_shape(*req, s, err);
  if (st != DD_OK) { set_error(err); return st; }
  if (nbins) *nbins = s.nbins;
  if (h) *h = s.h;
  if (A_eff) *A_eff = s.A;
  return DD_OK;
}

int dd_request_plan(const dd_request* req, uint64_t* lattice, uint64_t* tiles, uint64_t* pairs_lo,
                    uint64_t* pairs_hi) {
  if (!req) { set_error("req is NULL"); return DD_ERR_INVALID_ARGUMENT; }
  Shape s;
  std::string err;
  int st = derive_shape(*req, s, err);
  if (st != DD_OK) { set_error(err); return st; }
  std::vector<Job> jobs;
  plan_jobs(s, *req, jobs);
  const u128 p = planned_pairs(s, *req);
  if (lattice) *lattice = s.lattice;
  if (tiles) *tiles = jobs[0].tiles;
  if (pairs_lo) *pairs_lo = (uint64_t)p;
  if (pairs_hi) *pairs_hi = (uint64_t)(p >> 64);
  return DD_OK;
}

int dd_postprocess(const dd_request* req, const uint64_t* raw, uint32_t nraw, dd_result* res) {
  if (!req || !raw || !res) { set_error("NULL argument"); return DD_ERR_INVALID_ARGUMENT; }
  Shape s;
  std::string err;
  int st = derive_shape(*req, s, err);
  if (st != DD_OK) { set_error(err); return st; }
  if (nraw < s.nbins) { set_error("raw histogram shorter than n+h+1"); return DD_ERR_INVALID_ARGUMENT; }
  std::memset(res, 0, sizeof(*res));
  postprocess(*req, s, raw, *res);
  res->user_tag = req->user_tag;
  res->status = DD_OK;
  return DD_OK;
}

void dd_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  Philox4 o = philox4x32_10(ctr[0], ctr[1], ctr[2], ctr[3], key[0], key[1]);
  out[0] = o.x; out[1] = o.y; out[2] = o.z; out[3] = o.w;
}

}  // extern "C"

namespace dd {

// One launch for `count` requests: plan, (graph-)enqueue, synchronise, check
// the kernels' status word, post-process every request.
// `continued` (Monte Carlo continuation, one request): draw only the samples
// [continued->it_done, m) and add continued->raw_done to the device bins.
struct McContinuation {
  uint64_t it_done;
  const uint64_t* raw_done;
};

static int run_requests(dd_context* ctx, const dd_request* reqs, uint32_t count, dd_result* results,
                        bool use_graph, const McContinuation* continued = nullptr) {
  const double t0 = now_ms();
  std::vector<Shape> shapes(count);
  std::vector<Job> jobs;
  std::vector<uint32_t> kernels(count);
  jobs.reserve(count);
  for (uint32_t i = 0; i < count; ++i) {
    std::string err;
    int st = derive_shape(reqs[i], shapes[i], err);
    if (st != DD_OK) {
      set_error(count > 1 ? "request " + std::to_string(i) + ": " + err : err);
      return st;
    }
    plan_jobs(shapes[i], reqs[i], jobs);
    kernels[i] = reqs[i].kernel;
  }
  if (continued) {
    Job& j = jobs[0];
    j.sample_begin = continued->it_done;
    j.tiles = job_tiles(j);
  }
  int st = ensure_capacity(ctx, count, count);
  if (st != DD_OK) return st;
  LaunchPlan lp;
  st = plan_launch(ctx, jobs, kernels, lp);
  if (st != DD_OK) return st;
  cudaStream_t s = ctx->stream;
  if (use_graph) {
    const size_t nj = lp.npopc + lp.nmma;
    const bool same = ctx->gexec && ctx->gjobs.size() == nj && ctx->ggrid[0] == lp.pgrid &&
                      ctx->ggrid[1] == lp.mgrid && ctx->gsmem[0] == lp.psmem && ctx->gsmem[1] == lp.msmem &&
                      ctx->ghist_mode == ctx->hist_mode && ctx->gtimeout_ns == lp.margs.timeout_ns &&
                      std::memcmp(ctx->gjobs.data(), ctx->h_jobs, nj * sizeof(Job)) == 0;
    if (!same) {
      drop_graph(ctx);
      cudaGraph_t g = nullptr;
      DD_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      st = enqueue_launch(ctx, lp, true);
      cudaError_t ce = cudaStreamEndCapture(s, &g);
      if (st != DD_OK) { if (g) cudaGraphDestroy(g); return st; }
      if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
      ce = cudaGraphInstantiate(&ctx->gexec, g, 0);
      cudaGraphDestroy(g);
      if (ce != cudaSuccess) { ctx->gexec = nullptr; return cuda_fail(ce, "cudaGraphInstantiate"); }
      ctx->gjobs.assign(ctx->h_jobs, ctx->h_jobs + nj);
      ctx->ggrid[0] = lp.pgrid; ctx->ggrid[1] = lp.mgrid;
      ctx->gsmem[0] = lp.psmem; ctx->gsmem[1] = lp.msmem;
      ctx->ghist_mode = ctx->hist_mode;
      ctx->gtimeout_ns = lp.margs.timeout_ns;
    }
    DD_CUDA(cudaGraphLaunch(ctx->gexec, s));
  } else {
    st = enqueue_launch(ctx, lp, false);
    if (st != DD_OK) return st;
  }
  DD_CUDA(cudaStreamSynchronize(s));
  st = check_status(ctx);
  if (st != DD_OK) return st;
  float ms = 0;
  DD_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  const double total = now_ms() - t0;
  for (uint32_t i = 0; i < count; ++i) {
    dd_result& r = results[i];
    std::memset(&r, 0, sizeof(r));
    uint64_t raw[kMaxBins];
    for (int b = 0; b < kMaxBins; ++b) raw[b] = ctx->h_bins[(size_t)i * kMaxBins + b];
    u128 pairs = planned_pairs(shapes[i], reqs[i]);
    if (continued) {
      for (uint32_t b = 0; b < shapes[i].nbins; ++b) raw[b] += continued->raw_done[b];
      pairs = (u128)(1ull << shapes[i].n) * (shapes[i].m - continued->it_done);
    }
    postprocess(reqs[i], shapes[i], raw, r);
    fill_pairs(r, pairs);
    r.kernel_used = want_mma(ctx, jobs[i], kernels[i]) ? DD_KERNEL_MMA : DD_KERNEL_POPC;
    r.mma_epilogue = r.kernel_used == DD_KERNEL_MMA ? mma_epilogue_of(ctx) : 0u;
    r.kernel_ms = ms;  // one launch: the whole batch's device time
    r.total_ms = total;
    r.user_tag = reqs[i].user_tag;
    r.status = DD_OK;
  }
  return DD_OK;
}

}  // namespace dd

extern "C" {

int dd_autotune(dd_context* ctx, dd_tuning* out) {
  if (!ctx) { set_error("NULL argument"); return DD_ERR_INVALID_ARGUMENT; }
  dd_request q;
  std::memset(&q, 0, sizeof(q));
  q.code = DD_CODE_AN;
  q.mode = DD_MODE_EXHAUSTIVE;
  q.A = 65521;
  q.n = 20;  // large enough that every kernel reaches its steady state (0.1 s per run)
  const uint64_t pairs = (1ull << 20) * ((1ull << 20) - 1) / 2;
  auto best_ms = [&](uint32_t kernel, int mode, uint32_t epilogue, double* ms_out) -> int {
    const int saved_mode = ctx->hist_mode, saved_tuned = ctx->tuned;
    const uint32_t saved_epi = ctx->mma_epilogue;
    ctx->hist_mode = mode;
    ctx->tuned = 1;  // keep AUTO out of the way while probing
    ctx->mma_epilogue = epilogue;
    q.kernel = kernel;
    double best = 1e30;
    int st = DD_OK;
    for (int rep = 0; rep < 3 && st == DD_OK; ++rep) {
      dd_result r;
      st = run_requests(ctx, &q, 1, &r, false);
      if (st == DD_OK && rep > 0 && r.kernel_ms < best) best = r.kernel_ms;
    }
    ctx->hist_mode = saved_mode;
    ctx->tuned = saved_tuned;
    ctx->mma_epilogue = saved_epi;
    *ms_out = best;
    return st;
  };
  double red = 0, ldst = 0, mma = 0, paired = 0;
  int st = best_ms(DD_KERNEL_POPC, HIST_RED, DD_MMA_EPILOGUE_AUTO, &red);
  if (st == DD_OK) st = best_ms(DD_KERNEL_POPC, HIST_LDST, DD_MMA_EPILOGUE_AUTO, &ldst);
  if (st == DD_OK) st = best_ms(DD_KERNEL_MMA, ctx->hist_mode, DD_MMA_EPILOGUE_SINGLE, &mma);
  if (st == DD_OK) st = best_ms(DD_KERNEL_MMA, ctx->hist_mode, DD_MMA_EPILOGUE_PAIRED, &paired);
  if (st != DD_OK) return st;
  ctx->hist_mode = red <= ldst ? HIST_RED : HIST_LDST;
  ctx->mma_tuned_epilogue = paired <= mma ? DD_MMA_EPILOGUE_PAIRED : DD_MMA_EPILOGUE_SINGLE;
  ctx->tuned = std::min(mma, paired) < std::min(red, ldst) ? 2 : 1;
  if (out) {
    std::memset(out, 0, sizeof(*out));
    out->kernel = ctx->tuned == 2 ? DD_KERNEL_MMA : DD_KERNEL_POPC;
    out->hist_mode = (uint32_t)ctx->hist_mode;
    out->popc_red_pairs_per_s = pairs / (red * 1e-3);
    out->popc_ldst_pairs_per_s = pairs / (ldst * 1e-3);
    out->mma_pairs_per_s = pairs / (mma * 1e-3);
    out->mma_paired_pairs_per_s = pairs / (paired * 1e-3);
    out->mma_epilogue = ctx->mma_tuned_epilogue;
    out->probe_pairs = pairs;
  }
  return DD_OK;
}

int dd_histogram(dd_context* ctx, const dd_request* req, dd_result* res) {
  if (!ctx || !req || !res) { set_error("NULL argument"); return DD_ERR_INVALID_ARGUMENT; }
  // First large AUTO exhaustive request: let the autotuner pick the kernel.
  if (!ctx->tuned && req->kernel == DD_KERNEL_AUTO && req->code == DD_CODE_AN &&
      req->mode == DD_MODE_EXHAUSTIVE && req->n >= 20) {
    const int st = dd_autotune(ctx, nullptr);
    if (st != DD_OK) return st;
  }
  return run_requests(ctx, req, 1, res, false);
}

int dd_batch_run(dd_context* ctx, const dd_request* reqs, uint32_t count, dd_result* results,
                 const dd_batch_options* opts) {
  if (!ctx || (!reqs && count) || (!results && count)) { set_error("NULL argument"); return DD_ERR_INVALID_ARGUMENT; }
  if (count == 0) return DD_OK;
  if (!ctx->tuned && count >= 16 && (!opts || opts->kernel == DD_KERNEL_AUTO)) {
    const int st = dd_autotune(ctx, nullptr);
    if (st != DD_OK) return st;
  }
  if (opts && opts->kernel != DD_KERNEL_AUTO) {
    std::vector<dd_request> r(reqs, reqs + count);
    for (auto& q : r) q.kernel = opts->kernel;
    return run_requests(ctx, r.data(), count, results, opts->use_graph != 0);
  }
  return run_requests(ctx, reqs, count, results, opts && opts->use_graph);
}

int dd_mc_extend(dd_context* ctx, const dd_request* req, uint64_t it_done, const uint64_t* raw_done, dd_result* res) {
  if (!ctx || !req || !res || (it_done && !raw_done)) { set_error("NULL argument"); return DD_ERR_INVALID_ARGUMENT; }
  if (req->code != DD_CODE_AN || req->mode != DD_MODE_MONTE_CARLO) {
    set_error("dd_mc_extend: AN Monte Carlo requests only");
    return DD_ERR_UNSUPPORTED;
  }
  Shape s;
  std::string err;
  int st = derive_shape(*req, s, err);
  if (st != DD_OK) { set_error(err); return st; }
  if (it_done > s.m) {
    set_error("dd_mc_extend: more samples done than requested (after capping at 2^n)");
    return DD_ERR_INVALID_ARGUMENT;
  }
  if (it_done == s.m) {  // nothing left to draw: post-process what the caller has
    uint64_t raw[kMaxBins] = {0};
    for (uint32_t b = 0; b < s.nbins; ++b) raw[b] = raw_done[b];
    std::memset(res, 0, sizeof(*res));
    postprocess(*req, s, raw, *res);
    res->user_tag = req->user_tag;
    return DD_OK;
  }
  const McContinuation c{it_done, raw_done};
  return run_requests(ctx, req, 1, res, false, &c);
}

int dd_histogram_part(dd_context* ctx, const dd_request* req, uint64_t tile_begin, uint64_t tile_count,
                      uint64_t* raw, uint32_t nraw, double* kernel_ms) {
  if (!ctx || !req || !raw) { set_error("NULL argument"); return DD_ERR_INVALID_ARGUMENT; }
  if (kernel_ms) *kernel_ms = 0.0;
  Shape s;
  std::string err;
  int st = derive_shape(*req, s, err);
  if (st != DD_OK) { set_error(err); return st; }
  if (nraw < s.nbins) { set_error("raw histogram shorter than n+h+1"); return DD_ERR_INVALID_ARGUMENT; }
  std::vector<Job> jobs;
  plan_jobs(s, *req, jobs);
  Job& j = jobs[0];
  if (tile_begin > j.tiles || tile_count > j.tiles - tile_begin) {
    set_error("tile range outside the request's tile space (dd_request_plan gives its size)");
    return DD_ERR_INVALID_ARGUMENT;
  }
  if (tile_count == 0) return DD_OK;
  // the kernel choice follows dd_histogram's (the autotuner's verdict for AUTO)
  if (!ctx->tuned && req->kernel == DD_KERNEL_AUTO && req->code == DD_CODE_AN && req->mode == DD_MODE_EXHAUSTIVE &&
      req->n >= 20) {
    st = dd_autotune(ctx, nullptr);
    if (st != DD_OK) return st;
  }
  st = ensure_capacity(ctx, 1, 1);
  if (st != DD_OK) return st;
  // the sub-range runs exactly as a query server round runs a query's share
  j.tile_offset = tile_begin;
  j.tiles = tile_count;
  j.bins = ctx->d_bins;
  DD_CUDA(cudaMemsetAsync(ctx->d_bins, 0, kMaxBins * sizeof(unsigned long long), ctx->stream));
  const std::vector<uint32_t> kernels{req->kernel};
  float ms = 0.0f;
  st = launch_round(ctx, jobs, kernels, &ms);
  if (st != DD_OK) return st;
  DD_CUDA(cudaMemcpyAsync(ctx->h_bins, ctx->d_bins, kMaxBins * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                          ctx->stream));
  DD_CUDA(cudaStreamSynchronize(ctx->stream));
  for (uint32_t b = 0; b < s.nbins; ++b) raw[b] += ctx->h_bins[b];
  if (kernel_ms) *kernel_ms = ms;
  return DD_OK;
}

int dd_histogram_plain(dd_context* ctx, const dd_request* req, dd_result* res) {
  if (!ctx || !req || !res) { set_error("NULL argument"); return DD_ERR_INVALID_ARGUMENT; }
  if (req->code != DD_CODE_AN || req->mode != DD_MODE_EXHAUSTIVE) {
    set_error("the plain baseline covers AN exhaustive requests only");
    return DD_ERR_UNSUPPORTED;
  }
  const double t0 = now_ms();
  Shape s;
  std::string err;
  int st = derive_shape(*req, s, err);
  if (st != DD_OK) { set_error(err); return st; }
  DD_CUDA(cudaSetDevice(ctx->device));
  // per call, as the reference's driver: allocate and clear the bins, launch
  // 128 CTAs per SM, copy the bins back, free them
  unsigned long long* bins = nullptr;
  DD_CUDA(cudaMalloc(&bins, s.nbins * sizeof(unsigned long long)));
  cudaError_t e = cudaMemsetAsync(bins, 0, s.nbins * sizeof(unsigned long long), ctx->stream);
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev0, ctx->stream);
  if (e == cudaSuccess) e = launch_plain(s.A, 1ull << s.n, s.nbins, bins, 128 * ctx->num_sms, ctx->stream);
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev1, ctx->stream);
  uint64_t raw[kMaxBins] = {0};
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(raw, bins, s.nbins * sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  float ms = 0;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  cudaFree(bins);
  if (e != cudaSuccess) return cuda_fail(e, "plain baseline");
  std::memset(res, 0, sizeof(*res));
  postprocess(*req, s, raw, *res);
  fill_pairs(*res, planned_pairs(s, *req));
  res->kernel_used = DD_KERNEL_POPC;
  res->kernel_ms = ms;
  res->user_tag = req->user_tag;
  res->total_ms = now_ms() - t0;
  return DD_OK;
}

int dd_measure_popc_peak(dd_context* ctx, double* popc_per_s) {
  if (!ctx || !popc_per_s) { set_error("NULL argument"); return DD_ERR_INVALID_ARGUMENT; }
  DD_CUDA(cudaSetDevice(ctx->device));
  uint32_t* sink = nullptr;
  const int grid = ctx->num_sms * 8;
  DD_CUDA(cudaMalloc(&sink, grid * sizeof(uint32_t)));
  const uint32_t iters = 4096;
  cudaError_t e = launch_popc_rate(iters / 8, grid, sink, ctx->stream);  // warm-up
  float best = 1e30f;
  for (int rep = 0; rep < 3 && e == cudaSuccess; ++rep) {
    e = cudaEventRecord(ctx->ev0, ctx->stream);
    if (e == cudaSuccess) e = launch_popc_rate(iters, grid, sink, ctx->stream);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev1, ctx->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(ctx->ev1);
    float ms = 0;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    if (e == cudaSuccess && ms < best) best = ms;
  }
  cudaFree(sink);
  if (e != cudaSuccess) return cuda_fail(e, "popc probe");
  const double popcs = (double)grid * 256.0 * iters * 16.0 * 8.0;
  *popc_per_s = popcs / (best * 1e-3);
  return DD_OK;
}

int dd_set_mma_epilogue(dd_context* ctx, uint32_t epilogue) {
  if (!ctx) { set_error("NULL argument"); return DD_ERR_INVALID_ARGUMENT; }
  if (epilogue > DD_MMA_EPILOGUE_SINGLE) { set_error("unknown tcgen05 epilogue"); return DD_ERR_INVALID_ARGUMENT; }
  ctx->mma_epilogue = epilogue;
  return DD_OK;
}

int dd_set_wait_timeout(dd_context* ctx, uint64_t ns) {
  if (!ctx) { set_error("NULL argument"); return DD_ERR_INVALID_ARGUMENT; }
  ctx->mma_timeout_ns = ns ? ns : 2000000000ull;
  return DD_OK;
}

int dd_measure_red_sweep(dd_context* ctx, dd_red_probe* out, uint32_t cap, uint32_t* count) {
  if (!ctx || !out || !count) { set_error("NULL argument"); return DD_ERR_INVALID_ARGUMENT; }
  *count = 0;
  DD_CUDA(cudaSetDevice(ctx->device));
  uint32_t* sink = nullptr;
  const int grid = ctx->num_sms;
  DD_CUDA(cudaMalloc(&sink, grid * sizeof(uint32_t)));
  const uint32_t iters = 20000;
  cudaError_t e = cudaSuccess;
  for (int pattern = 0; pattern < 2 && e == cudaSuccess; ++pattern)
    for (int warps = 8; warps <= 32 && e == cudaSuccess; warps += 4) {
      const int threads = warps * 32;
      e = launch_red_rate(iters / 10, grid, threads, pattern, sink, ctx->stream);  // warm-up
      float best = 1e30f;
      for (int rep = 0; rep < 3 && e == cudaSuccess; ++rep) {
        e = cudaEventRecord(ctx->ev0, ctx->stream);
        if (e == cudaSuccess) e = launch_red_rate(iters, grid, threads, pattern, sink, ctx->stream);
        if (e == cudaSuccess) e = cudaEventRecord(ctx->ev1, ctx->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(ctx->ev1);
        float ms = 0;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        if (e == cudaSuccess && ms < best) best = ms;
      }
      if (e == cudaSuccess && *count < cap) {
        dd_red_probe& r = out[(*count)++];
        r.warps_per_sm = (uint32_t)warps;
        r.pattern = (uint32_t)pattern;
        r.adds_per_s = (double)red_rate_adds(iters, grid, threads) / (best * 1e-3);
      }
    }
  cudaFree(sink);
  if (e != cudaSuccess) return cuda_fail(e, "shared-atomic probe");
  return DD_OK;
}

int dd_measure_red_peak(dd_context* ctx, double* adds_per_s) {
  if (!ctx || !adds_per_s) { set_error("NULL argument"); return DD_ERR_INVALID_ARGUMENT; }
  dd_red_probe rows[64];
  uint32_t n = 0;
  const int st = dd_measure_red_sweep(ctx, rows, 64, &n);
  if (st != DD_OK) return st;
  double best = 0;
  for (uint32_t i = 0; i < n; ++i) best = std::max(best, rows[i].adds_per_s);
  *adds_per_s = best;
  return DD_OK;
}

}  // extern "C"
