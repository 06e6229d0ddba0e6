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

struct dd_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int num_sms = 0;
  // device state
  unsigned long long* d_bins = nullptr;  // bin_slots x kMaxBins
  uint32_t bin_slots = 0;
  unsigned long long* d_counter = nullptr;
  dd::Job* d_jobs = nullptr;
  uint32_t job_cap = 0;
  // pinned host mirrors
  unsigned long long* h_bins = nullptr;
  dd::Job* h_jobs = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // tuning
  int hist_mode = dd::HIST_RED;
  int tuned = 0;
  // batch graph cache
  cudaGraphExec_t gexec = nullptr;
  std::vector<dd::Job> gjobs;  // job table the cached graph was built for
  int ggrid = 0;
  size_t gsmem = 0;
};

namespace dd {

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

static int ensure_capacity(dd_context* ctx, uint32_t slots, uint32_t njobs) {
  DD_CUDA(cudaSetDevice(ctx->device));
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
  LaunchArgs args;
  int grid = 0;
  size_t smem = 0;
};

// Fills the pinned job table, assigns tile ranges and bin slots, and sizes
// the persistent grid (one wave: SMs x resident CTAs).
static int plan_launch(dd_context* ctx, std::vector<Job>& jobs, LaunchPlan& lp) {
  uint64_t t = 0;
  uint32_t maxb = 1;
  bool table = false;
  for (size_t i = 0; i < jobs.size(); ++i) {
    jobs[i].tile_begin = t;
    t += jobs[i].tiles;
    jobs[i].bins = ctx->d_bins + i * kMaxBins;
    maxb = std::max(maxb, jobs[i].nbins);
    table |= (jobs[i].kind == JOB_PAIRS && jobs[i].col_kind == COL_HAMMING_EXT && !jobs[i].wide);
  }
  lp.args.jobs = ctx->d_jobs;
  lp.args.njobs = (uint32_t)jobs.size();
  lp.args.smem_bins = maxb;
  lp.args.total_tiles = t;
  lp.args.counter = ctx->d_counter;
  lp.args.use_col_table = table ? 1u : 0u;
  lp.smem = hist_smem_bytes(maxb, table);
  int occ = 0;
  DD_CUDA(hist_occupancy(ctx->hist_mode, lp.smem, &occ));
  if (occ < 1) { set_error("kernel does not fit on an SM"); return DD_ERR_UNSUPPORTED; }
  // never more warps than tiles
  const uint64_t want = (t + kWarpsPerCta - 1) / kWarpsPerCta;
  lp.grid = (int)std::min<uint64_t>((uint64_t)ctx->num_sms * occ, std::max<uint64_t>(want, 1));
  std::memcpy(ctx->h_jobs, jobs.data(), jobs.size() * sizeof(Job));
  return DD_OK;
}

// Enqueues: job table H2D, bins + counter reset, kernel (bracketed by events), bins D2H.
static int enqueue_launch(dd_context* ctx, const LaunchPlan& lp, uint32_t njobs, bool events) {
  cudaStream_t s = ctx->stream;
  DD_CUDA(cudaMemcpyAsync(ctx->d_jobs, ctx->h_jobs, njobs * sizeof(Job), cudaMemcpyHostToDevice, s));
  DD_CUDA(cudaMemsetAsync(ctx->d_bins, 0, (size_t)njobs * kMaxBins * sizeof(unsigned long long), s));
  DD_CUDA(cudaMemsetAsync(ctx->d_counter, 0, sizeof(unsigned long long), s));
  if (events) DD_CUDA(cudaEventRecord(ctx->ev0, s));
  if (lp.args.total_tiles) DD_CUDA(launch_hist(ctx->hist_mode, lp.args, lp.grid, lp.smem, s));
  if (events) DD_CUDA(cudaEventRecord(ctx->ev1, s));
  DD_CUDA(cudaMemcpyAsync(ctx->h_bins, ctx->d_bins, (size_t)njobs * kMaxBins * sizeof(unsigned long long),
                          cudaMemcpyDeviceToHost, s));
  return DD_OK;
}

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
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
    if (major != 10) {
      delete ctx;
      set_error("this library is built for sm_100a (B200) only");
      return DD_ERR_NO_DEVICE;
    }
  }
  if (e == cudaSuccess) {
    if (stream) ctx->stream = (cudaStream_t)stream;
    else { e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking); ctx->own_stream = true; }
  }
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_counter, sizeof(unsigned long long));
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
  if (ctx->d_counter) cudaFree(ctx->d_counter);
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

int dd_histogram(dd_context* ctx, const dd_request* req, dd_result* res) {
  if (!ctx || !req || !res) { set_error("NULL argument"); return DD_ERR_INVALID_ARGUMENT; }
  const double t0 = now_ms();
  Shape s;
  std::string err;
  int st = derive_shape(*req, s, err);
  if (st != DD_OK) { set_error(err); return st; }
  std::vector<Job> jobs;
  plan_jobs(s, *req, jobs);
  st = ensure_capacity(ctx, 1, 1);
  if (st != DD_OK) return st;
  LaunchPlan lp;
  st = plan_launch(ctx, jobs, lp);
  if (st != DD_OK) return st;
  st = enqueue_launch(ctx, lp, 1, true);
  if (st != DD_OK) return st;
  DD_CUDA(cudaStreamSynchronize(ctx->stream));
  float ms = 0;
  DD_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  std::memset(res, 0, sizeof(*res));
  uint64_t raw[kMaxBins];
  for (int i = 0; i < kMaxBins; ++i) raw[i] = ctx->h_bins[i];
  postprocess(*req, s, raw, *res);
  fill_pairs(*res, planned_pairs(s, *req));
  res->kernel_used = DD_KERNEL_POPC;
  res->kernel_ms = ms;
  res->user_tag = req->user_tag;
  res->status = DD_OK;
  res->total_ms = now_ms() - t0;
  return DD_OK;
}

int dd_batch_run(dd_context* ctx, const dd_request* reqs, uint32_t count, dd_result* results,
                 const dd_batch_options* opts) {
  if (!ctx || (!reqs && count) || (!results && count)) { set_error("NULL argument"); return DD_ERR_INVALID_ARGUMENT; }
  if (count == 0) return DD_OK;
  const double t0 = now_ms();
  const bool use_graph = opts && opts->use_graph;
  std::vector<Shape> shapes(count);
  std::vector<Job> jobs;
  jobs.reserve(count);
  for (uint32_t i = 0; i < count; ++i) {
    std::string err;
    int st = derive_shape(reqs[i], shapes[i], err);
    if (st != DD_OK) { set_error("request " + std::to_string(i) + ": " + err); return st; }
    plan_jobs(shapes[i], reqs[i], jobs);
  }
  int st = ensure_capacity(ctx, count, count);
  if (st != DD_OK) return st;
  LaunchPlan lp;
  st = plan_launch(ctx, jobs, lp);
  if (st != DD_OK) return st;
  cudaStream_t s = ctx->stream;
  if (use_graph) {
    bool same = ctx->gexec && ctx->gjobs.size() == jobs.size() && ctx->ggrid == lp.grid && ctx->gsmem == lp.smem &&
                std::memcmp(ctx->gjobs.data(), jobs.data(), jobs.size() * sizeof(Job)) == 0;
    if (!same) {
      if (ctx->gexec) { cudaGraphExecDestroy(ctx->gexec); ctx->gexec = nullptr; }
      cudaGraph_t g = nullptr;
      DD_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      st = enqueue_launch(ctx, lp, count, true);
      cudaError_t ce = cudaStreamEndCapture(s, &g);
      if (st != DD_OK) { if (g) cudaGraphDestroy(g); return st; }
      if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
      ce = cudaGraphInstantiate(&ctx->gexec, g, 0);
      cudaGraphDestroy(g);
      if (ce != cudaSuccess) { ctx->gexec = nullptr; return cuda_fail(ce, "cudaGraphInstantiate"); }
      ctx->gjobs = jobs;
      ctx->ggrid = lp.grid;
      ctx->gsmem = lp.smem;
    }
    DD_CUDA(cudaGraphLaunch(ctx->gexec, s));
  } else {
    st = enqueue_launch(ctx, lp, count, true);
    if (st != DD_OK) return st;
  }
  DD_CUDA(cudaStreamSynchronize(s));
  float ms = 0;
  DD_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  const double total = now_ms() - t0;
  for (uint32_t i = 0; i < count; ++i) {
    dd_result& r = results[i];
    std::memset(&r, 0, sizeof(r));
    uint64_t raw[kMaxBins];
    for (int b = 0; b < kMaxBins; ++b) raw[b] = ctx->h_bins[(size_t)i * kMaxBins + b];
    postprocess(reqs[i], shapes[i], raw, r);
    fill_pairs(r, planned_pairs(shapes[i], reqs[i]));
    r.kernel_used = DD_KERNEL_POPC;
    r.kernel_ms = ms;  // one launch: the whole batch's device time
    r.total_ms = total;
    r.user_tag = reqs[i].user_tag;
    r.status = DD_OK;
  }
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

}  // extern "C"
