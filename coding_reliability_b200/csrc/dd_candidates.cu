// dd_candidates.cu — super-A candidate pre-filter on the GPU (dd_an_candidates).
//
// The reference's ANcandidates tool (ANcandidates/ANcandidates.cpp:35-163,
// main :236-301) ranks every odd A of a bit width a by the smallest
// non-adjacent-form (symmetric signed-digit) weight over its non-zero
// codewords,
//     w(A) = min over x in [1, 2^k) of popcount(A·x XOR 3·A·x),
// and keeps the A values whose w(A) is the largest of the range: a codeword of
// small signed-digit weight is reachable from 0 by few arithmetic +-2^i errors,
// so these A are the candidates worth an exact distance distribution.  Its
// worker stops scanning an A as soon as the running minimum falls below the
// best minimum found so far (:122-138); that only skips A values that cannot
// be in the result, so the result is a pure function of (k, a).
//
// Here persistent warps claim (A, x segment) work items from a counter, A-major;
// in a segment lane l takes x = x0 + l + 32 t, carrying A·x by one add per
// step.  Every 32·kChunk values the warp takes its minimum and leaves when it,
// or the A's minimum so far, is below the best completed minimum (the same
// early exit, checked less often).  The warp that finishes an A's last segment
// raises the best with atomicMax.  A second kernel collects every A whose
// minimum equals the final best.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/codrel_b200.h"
#include "dd_host.h"

namespace dd {
namespace {

constexpr int kNafThreads = 256;
constexpr int kChunk = 64;  // values per lane between early-exit checks

// Control block, cleared before each call.
struct NafCtl {
  unsigned int best;         // largest minimum of a completed A
  unsigned int pad;
  unsigned long long next;   // (A, segment) claim counter
  unsigned long long found;  // candidates (may exceed the list's capacity)
  unsigned long long evals;  // codewords weighed, over all A
};

struct NafArgs {
  unsigned long long minA;  // first (odd) A
  unsigned long long numA;  // odd A values minA, minA+2, ...
  unsigned long long xmax;  // 2^k - 1
  unsigned int seg_shift;   // x segments per A = 2^seg_shift, each of seg_len values
  unsigned int pad;
  unsigned long long seg_len;
  NafCtl* ctl;
  unsigned int* amin;       // per A: minimum over its segments (or a running minimum below the best)
  unsigned int* done;       // per A: segments finished
  unsigned long long* out;  // candidates (unordered), capacity `cap`
  unsigned long long cap;
};

// Signed-digit weight of c: popcount(c XOR 3c) (ANcandidates.cpp:124-135).
__device__ __forceinline__ unsigned int naf_weight(unsigned long long c) {
  return (unsigned int)__popcll(c ^ (3ull * c));
}
__device__ __forceinline__ unsigned int naf_weight(unsigned int c) { return (unsigned int)__popc(c ^ (3u * c)); }

// True when the A's minimum so far, or the warp's running minimum m, is below
// the best completed minimum.  Lane 0 reads both words and broadcasts the
// decision: the values change under the warp's feet, and a decision taken per
// lane would split the warp before its next __reduce_min_sync.
__device__ __forceinline__ bool below_best(const NafArgs& a, unsigned long long i, unsigned int m) {
  unsigned int below = 0;
  if ((threadIdx.x & 31) == 0) {
    const unsigned int best = *(const volatile unsigned int*)&a.ctl->best;
    below = (m < best || *(const volatile unsigned int*)&a.amin[i] < best) ? 1u : 0u;
  }
  return __shfl_sync(0xffffffffu, below, 0) != 0;
}

// T: the codeword type, 32-bit when 3·A·x stays below 2^32.  Work item: one
// segment of one A's x range, A-major, so that the warps of the grid share the
// segments of the same few A values.  A segment is dropped (or left) as soon as
// its warp's running minimum or the A's minimum so far is below the best
// completed minimum: such an A cannot be a candidate.  The warp that finishes
// an A's last segment publishes the A's minimum into the best (a minimum that
// is below the best because a segment was left early does not change it).
template <typename T>
__global__ void __launch_bounds__(kNafThreads) naf_min_kernel(NafArgs a) {
  const unsigned int lane = threadIdx.x & 31;
  const unsigned long long chunk_span = 32ull * kChunk;
  const unsigned long long segs = 1ull << a.seg_shift;
  const unsigned long long items = a.numA << a.seg_shift;
  for (;;) {
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(&a.ctl->next, 1ull);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= items) return;
    const unsigned long long i = t >> a.seg_shift;
    const unsigned long long A = a.minA + 2ull * i;
    const unsigned long long x0 = 1ull + (t & (segs - 1)) * a.seg_len;
    const unsigned long long x1 = min(a.xmax, x0 + a.seg_len - 1);
    unsigned int rm = 0xffu;
    unsigned long long scanned = 0;
    if (x0 <= x1 && !below_best(a, i, 0xffu)) {
      const T step = (T)(32ull * A);
      T c = (T)(A * (x0 + lane));
      for (unsigned long long base = x0; base <= x1; base += chunk_span) {
        if (base + chunk_span - 1 <= x1) {  // warp-uniform: the whole chunk is in range
#pragma unroll 8
          for (int j = 0; j < kChunk; ++j) {
            rm = min(rm, naf_weight(c));
            c += step;
          }
        } else {
          unsigned long long x = base + lane;
          for (int j = 0; j < kChunk; ++j) {
            if (x <= x1) rm = min(rm, naf_weight(c));
            c += step;
            x += 32;
          }
        }
        scanned += min(x1, base + chunk_span - 1) - base + 1;
        if (below_best(a, i, __reduce_min_sync(0xffffffffu, rm))) break;
      }
    }
    const unsigned int m = __reduce_min_sync(0xffffffffu, rm);
    if (lane == 0) {
      if (m != 0xffu) atomicMin(&a.amin[i], m);
      __threadfence();
      if (atomicAdd(&a.done[i], 1u) + 1u == (unsigned int)segs) {
        __threadfence();
        atomicMax(&a.ctl->best, atomicAdd(&a.amin[i], 0u));
      }
      if (scanned) atomicAdd(&a.ctl->evals, scanned);
    }
  }
}

__global__ void naf_collect_kernel(NafArgs a) {
  const unsigned int best = a.ctl->best;
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < a.numA;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    if (a.amin[i] == best) {
      const unsigned long long slot = atomicAdd(&a.ctl->found, 1ull);
      if (slot < a.cap) a.out[slot] = a.minA + 2ull * i;
    }
  }
}

}  // namespace
}  // namespace dd

using namespace dd;

extern "C" int dd_an_candidates(dd_context* ctx, uint32_t k, uint32_t a_bits, uint64_t* out_A, uint64_t capacity,
                                dd_candidates_result* res) {
  if (!ctx || !res || (capacity && !out_A)) {
    set_error("dd_an_candidates: NULL argument");
    return DD_ERR_INVALID_ARGUMENT;
  }
  std::memset(res, 0, sizeof(*res));
  res->k = k;
  res->a_bits = a_bits;
  if (k < 1 || k > 48 || a_bits < 1 || a_bits > 32 || k + a_bits > 61) {
    set_error("dd_an_candidates: need 1 <= k <= 48, 1 <= a_bits <= 32, k + a_bits <= 61");
    return res->status = DD_ERR_INVALID_ARGUMENT;
  }
  const auto t0 = std::chrono::steady_clock::now();
  // odd A in [2^(a-1)+1, 2^a-1]; none for a = 1 (the reference's loop is empty there)
  const unsigned long long minA = (1ull << (a_bits - 1)) + 1ull;
  const unsigned long long maxA = (1ull << a_bits) - 1ull;
  const unsigned long long numA = maxA >= minA ? (maxA - minA) / 2ull + 1ull : 0ull;
  res->num_A = numA;
  if (numA == 0) {
    res->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return DD_OK;
  }
  const int device = context_device(ctx);
  cudaStream_t stream = (cudaStream_t)context_stream(ctx);
  cudaError_t e = cudaSetDevice(device);
  int sms = 0, per_sm = 0;
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const bool wide = k + a_bits + 2 > 32;
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, wide ? (const void*)naf_min_kernel<unsigned long long> : (const void*)naf_min_kernel<unsigned int>, kNafThreads, 0);
  const unsigned long long cap = std::max<unsigned long long>(capacity, 1);
  NafArgs a{};
  a.minA = minA;
  a.numA = numA;
  a.xmax = (1ull << k) - 1ull;
  a.cap = cap;
  // segments of 2^max(15, k-24) x values: at most 2^24 per A, each a whole
  // number of 32 x kChunk chunks
  const unsigned int seg_bits = std::max(15u, k > 24 ? k - 24 : 0u);
  a.seg_len = 1ull << seg_bits;
  a.seg_shift = k > seg_bits ? k - seg_bits : 0u;
  void* mem = nullptr;
  const size_t ctl_bytes = 256, arr_bytes = (numA * sizeof(unsigned int) + 255) / 256 * 256;
  if (e == cudaSuccess) e = cudaMalloc(&mem, ctl_bytes + 2 * arr_bytes + cap * sizeof(unsigned long long));
  if (e != cudaSuccess) {
    set_error(std::string("dd_an_candidates: ") + cudaGetErrorString(e));
    return res->status = (e == cudaErrorMemoryAllocation ? DD_ERR_OUT_OF_MEMORY : DD_ERR_CUDA);
  }
  a.ctl = (NafCtl*)mem;
  a.amin = (unsigned int*)((unsigned char*)mem + ctl_bytes);
  a.done = (unsigned int*)((unsigned char*)mem + ctl_bytes + arr_bytes);
  a.out = (unsigned long long*)((unsigned char*)mem + ctl_bytes + 2 * arr_bytes);
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  NafCtl h_ctl{};
  std::vector<unsigned long long> found;
  float ms = 0;
  e = cudaEventCreate(&ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&ev1);
  if (e == cudaSuccess) e = cudaMemsetAsync(a.ctl, 0, ctl_bytes, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(a.amin, 0xff, arr_bytes, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(a.done, 0, arr_bytes, stream);
  if (e == cudaSuccess) e = cudaEventRecord(ev0, stream);
  if (e == cudaSuccess) {
    const unsigned long long warps = (unsigned long long)sms * per_sm * (kNafThreads / 32);
    const unsigned long long want = std::min<unsigned long long>(numA << a.seg_shift, warps);
    const int grid = (int)std::max<unsigned long long>(1, (want + kNafThreads / 32 - 1) / (kNafThreads / 32));
    if (wide)
      naf_min_kernel<unsigned long long><<<grid, kNafThreads, 0, stream>>>(a);
    else
      naf_min_kernel<unsigned int><<<grid, kNafThreads, 0, stream>>>(a);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    const int grid = (int)std::min<unsigned long long>((numA + 255) / 256, (unsigned long long)sms * 8);
    naf_collect_kernel<<<grid, 256, 0, stream>>>(a);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaEventRecord(ev1, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_ctl, a.ctl, sizeof(h_ctl), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e == cudaSuccess && h_ctl.found <= cap) {
    found.resize(h_ctl.found);
    if (!found.empty())
      e = cudaMemcpyAsync(found.data(), a.out, found.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                          stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  } else if (e == cudaSuccess) {
    // more candidates than the list holds: return the smallest `capacity` A values
    std::vector<unsigned int> amin(numA);
    e = cudaMemcpyAsync(amin.data(), a.amin, numA * sizeof(unsigned int), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    for (unsigned long long i = 0; e == cudaSuccess && i < numA && found.size() < capacity; ++i)
      if (amin[i] == h_ctl.best) found.push_back(minA + 2ull * i);
  }
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev0, ev1);
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  const cudaError_t ef = cudaFree(mem);
  if (e == cudaSuccess) e = ef;
  if (e != cudaSuccess) {
    set_error(std::string("dd_an_candidates: ") + cudaGetErrorString(e));
    return res->status = DD_ERR_CUDA;
  }
  std::sort(found.begin(), found.end());
  if (capacity) std::copy(found.begin(), found.begin() + std::min<size_t>(found.size(), capacity), out_A);
  res->sdr = h_ctl.best;
  res->num_candidates = h_ctl.found;
  res->kernel_ms = ms;
  res->evaluations = h_ctl.evals;
  res->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return DD_OK;
}
