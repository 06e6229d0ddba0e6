// dd_noalloc.cu — dd_histogram_noalloc: the popc-path histogram for callers
// that cannot allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is not allowed or not wanted —
// a host application that owns all device memory through its own pool and
// forbids foreign allocations, a plugin loaded into such a host, or a caller
// that must not perturb a device whose memory is fully reserved.  Every other
// entry point of this library keeps a dd_context whose creation allocates the
// bins, work counter, status word and job table with cudaMalloc.
//
// Here that scratch lives in one file-scope __device__ array of fixed size,
// present on every GPU that loads the library until the process exits.  The
// host code below never names the array as a device address: on every call,
// with the caller's device current, it asks the runtime for the array's address
// on that device (cudaGetSymbolAddress) and passes that pointer to the kernel.
// The lookup is not cached, so a context that was reset and re-created between
// calls gets the address of its own copy of the array.  The first call on a
// device also loads the module there, so it should come before any stream
// capture on that device.  The caller's current device is restored on return.
//
// Limits and sharing:
//   - at most kNoAllocMaxRequests requests per call (bins, job table and
//     counters of that many instances fit the array); larger calls are refused;
//   - every call uses the same array, which keeps the last call's contents;
//     each call clears the bins and counters it needs before its launch;
//   - calls whose work overlaps on the GPU (two host threads, or two streams,
//     on the same device) race on the array: serialise them.
// No cudaMalloc, cudaFree or other allocating routine is called; the caller's
// requests and results stay in host memory.
#include <cuda_runtime.h>

#include <chrono>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/codrel_b200.h"
#include "dd_host.h"
#include "dd_kernels.h"

namespace dd {
namespace {

constexpr uint32_t kNoAllocMaxRequests = 32;
constexpr uint32_t kCtl = 16;  // [0] work counter, [2] status word

struct NoAllocScratch {
  unsigned long long bins[kNoAllocMaxRequests][kMaxBins];  // 16 KB
  unsigned long long ctl[kCtl];
  Job jobs[kNoAllocMaxRequests];
};

// The scratch of dd_histogram_noalloc (about 21 KB per GPU).
static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

constexpr int kMaxDevices = 64;

// Device address of the scratch array on the current device.
int scratch_here(NoAllocScratch** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) {
    set_error(std::string("dd_histogram_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    return DD_ERR_CUDA;
  }
  *out = static_cast<NoAllocScratch*>(p);
  return DD_OK;
}

// Makes `device` current for the call and gives the caller's device back on
// every return path.
struct DeviceGuard {
  int saved = -1;
  cudaError_t enter(int device) {
    cudaError_t e = cudaGetDevice(&saved);
    if (e != cudaSuccess) { saved = -1; return e; }
    return saved == device ? cudaSuccess : cudaSetDevice(device);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (saved >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != saved) cudaSetDevice(saved);
  }
};

}  // namespace
}  // namespace dd

using namespace dd;

extern "C" int dd_histogram_noalloc(int device, void* stream, const dd_request* reqs, uint32_t count,
                                    dd_result* results) {
  if (!reqs || !results || count == 0) {
    set_error("dd_histogram_noalloc: reqs and results are required and count must be > 0");
    return DD_ERR_INVALID_ARGUMENT;
  }
  if (count > kNoAllocMaxRequests) {
    set_error("dd_histogram_noalloc: at most 32 requests per call (the fixed scratch holds 32 instances)");
    return DD_ERR_INVALID_ARGUMENT;
  }
  if (device < 0 || device >= kMaxDevices) {
    set_error("dd_histogram_noalloc: device ordinal out of range");
    return DD_ERR_INVALID_ARGUMENT;
  }
  const auto t0 = std::chrono::steady_clock::now();
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  DeviceGuard guard;
  cudaError_t e = guard.enter(device);
  if (e != cudaSuccess) {
    set_error(std::string("dd_histogram_noalloc: cudaSetDevice: ") + cudaGetErrorString(e));
    return DD_ERR_NO_DEVICE;
  }
  NoAllocScratch* scratch = nullptr;
  int st = scratch_here(&scratch);
  if (st != DD_OK) return st;

  // plan: one popc-path job per request, bins slot = request index
  Shape shapes[kNoAllocMaxRequests];
  Job table[kNoAllocMaxRequests];
  uint64_t tiles = 0;
  uint32_t maxb = 1;
  bool col_table = false;
  for (uint32_t i = 0; i < count; ++i) {
    std::string err;
    st = derive_shape(reqs[i], shapes[i], err);
    if (st != DD_OK) {
      set_error("dd_histogram_noalloc: request " + std::to_string(i) + ": " + err);
      return st;
    }
    std::vector<Job> one;
    plan_jobs(shapes[i], reqs[i], one);
    table[i] = one[0];
    table[i].bins = scratch->bins[i];
    table[i].tile_begin = tiles;
    tiles += table[i].tiles;
    if (table[i].nbins > maxb) maxb = table[i].nbins;
    col_table |= (table[i].kind == JOB_PAIRS && table[i].col_kind == COL_HAMMING_EXT && !table[i].wide);
  }
  LaunchArgs args;
  std::memset(&args, 0, sizeof(args));
  args.jobs = scratch->jobs;
  args.njobs = count;
  args.smem_bins = maxb;
  args.total_tiles = tiles;
  args.counter = &scratch->ctl[0];
  args.status = reinterpret_cast<unsigned*>(&scratch->ctl[2]);
  args.use_col_table = col_table ? 1u : 0u;
  const size_t smem = hist_smem_bytes(maxb, col_table);
  int occ = 0, sms = 0;
  e = hist_occupancy(HIST_RED, smem, &occ);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess || occ < 1) {
    set_error(std::string("dd_histogram_noalloc: launch set-up: ") + cudaGetErrorString(e));
    return DD_ERR_CUDA;
  }
  const uint64_t want = (tiles + kWarpsPerCta - 1) / kWarpsPerCta;
  const int grid = (int)(want < (uint64_t)sms * occ ? (want ? want : 1) : (uint64_t)sms * occ);

  // clear what must start at zero, upload the jobs, launch, read back
  unsigned long long raw[kNoAllocMaxRequests][kMaxBins];
  unsigned long long ctl[kCtl];
  e = cudaMemcpyAsync(scratch->jobs, table, count * sizeof(Job), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(scratch->bins, 0, count * sizeof(scratch->bins[0]), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(scratch->ctl, 0, sizeof(scratch->ctl), s);
  if (e == cudaSuccess && tiles) e = launch_hist(HIST_RED, args, grid, smem, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(raw, scratch->bins, count * sizeof(raw[0]), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ctl, scratch->ctl, sizeof(ctl), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    set_error(std::string("dd_histogram_noalloc: ") + cudaGetErrorString(e));
    return DD_ERR_CUDA;
  }
  const unsigned status = (unsigned)ctl[2];
  if (status) {
    set_error("dd_histogram_noalloc: the kernel reported status " + std::to_string(status));
    return (status & KSTATUS_TIMEOUT) ? DD_ERR_TIMEOUT : DD_ERR_CUDA;
  }
  const double total_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  for (uint32_t i = 0; i < count; ++i) {
    dd_result& r = results[i];
    std::memset(&r, 0, sizeof(r));
    uint64_t rb[kMaxBins];
    for (int b = 0; b < kMaxBins; ++b) rb[b] = raw[i][b];
    postprocess(reqs[i], shapes[i], rb, r);
    const u128 p = planned_pairs(shapes[i], reqs[i]);
    r.pairs_lo = (uint64_t)p;
    r.pairs_hi = (uint64_t)(p >> 64);
    r.kernel_used = DD_KERNEL_POPC;
    r.kernel_ms = 0;  // no CUDA events are created here
    r.total_ms = total_ms;
    r.user_tag = reqs[i].user_tag;
    r.status = DD_OK;
  }
  return DD_OK;
}
