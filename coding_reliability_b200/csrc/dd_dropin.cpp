// dd_dropin.cpp — the reference's driver functions (same names and
// signatures, distance_distribution/src/algorithms.h:20-34 and
// distance_distribution_super_a/src/algorithms.h:20-21) on top of the C-ABI,
// with the reference's stdout/results-file output, and dd_format_result.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/codrel_b200.h"
#include "../../include/codrel_dropin.h"
#include "dd_host.h"

using dd::u128;

namespace {

constexpr int kOffset = 2;  // OFFSET, src/globals.cpp:24

// Monte Carlo seeds of the drop-in drivers: the constants the reference adds
// to its cuRAND offsets (an_coding_mc.cu:274, hamming_mc.cu:169).
constexpr uint64_t kSeedAnMc = 16384;
constexpr uint64_t kSeedHammingMc = 1337;

// The drivers share one context on device 0.  A dd_context serves one host
// thread at a time, so every call on it holds g_mu: drivers called from several
// threads of a host application run one after the other.
std::mutex g_mu;
dd_context* g_ctx = nullptr;

template <class F>
int on_shared_context(F&& f) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_ctx) {
    int st = dd_context_create(0, nullptr, &g_ctx);
    if (st != DD_OK) throw std::runtime_error(std::string("codrel_b200: ") + dd_last_error());
  }
  return f(g_ctx);
}

dd_result run_request(const dd_request& req) {
  dd_result res;
  int st = on_shared_context([&](dd_context* c) { return dd_histogram(c, &req, &res); });
  if (st != DD_OK) throw std::runtime_error(std::string("codrel_b200: ") + dd_last_error());
  return res;
}

dd_request make_request(uint32_t code, uint32_t mode, uint64_t A, uint32_t n) {
  dd_request r;
  std::memset(&r, 0, sizeof(r));
  r.code = code;
  r.mode = mode;
  r.A = A;
  r.n = n;
  return r;
}

void counts_of(const dd_result& r, u128* c) {
  for (int i = 0; i < DD_MAX_BINS; ++i) c[i] = ((u128)r.counts_hi[i] << 64) | r.counts_lo[i];
}

std::string device_lines() {
  std::stringstream ss;
  int dev = 0, mem = 0, clk = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&mem, cudaDevAttrMemoryClockRate, dev);
  cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, dev);
  ss << "\"Device\", " << dev << ", \"MemClock [MHz]\", " << mem / 1000 << ", \"GPUClock [MHz]\", " << clk / 1000
     << std::endl;
  return ss.str();
}

std::vector<dd::StatRow> gpu_stats(const dd_result& r) {
  return {{"Kernel Runtime", r.kernel_ms * 0.001, "s"}, {"Total Runtime", r.total_ms * 0.001, "s"}};
}
std::vector<dd::StatRow> cpu_stats(const dd_result& r) { return {{"Total Runtime", r.total_ms * 0.001, "s"}}; }

// process_result (src/globals.cpp:185-244): table to stdout, optional file.
long double process_result(const u128* counts, const std::vector<dd::StatRow>& stats, uint32_t n, uint32_t h,
                           const char* file_prefix, const double* ea, const double* er, const std::string& app) {
  long double total = 0;
  const std::string text = dd::format_table(counts, stats, n, h, ea, er, app, &total);
  std::cout << text;
  if (file_prefix) {
    char fname[256];
    std::snprintf(fname, sizeof(fname), "%s_n%u_h%u.csv", file_prefix, n, h);
    std::ofstream fp(fname);
    fp << text;
    fp.close();
    std::cout << "File " << fname << " written." << std::endl << std::endl;
  }
  return total;
}

void print_A_line(uint64_t A, uint32_t n) {
  std::cout << " A = ";
  std::cout << dd::bits_string(A, n);
  std::cout << " = " << (unsigned)A << std::endl;
}

void process_result_ancoding(const u128* counts, const std::vector<dd::StatRow>& stats, uint32_t n, uint32_t A,
                             const char* prefix, const std::string& app) {
  char tmp[192];
  const uint32_t h = (uint32_t)std::ceil(std::log(A) / std::log(2.0));
  long double total;
  if (prefix) {
    std::snprintf(tmp, sizeof(tmp), "%s_A%u", prefix, A);
    total = process_result(counts, stats, n, h, tmp, nullptr, nullptr, app);
  } else {
    total = process_result(counts, stats, n, h, nullptr, nullptr, nullptr, app);
  }
  std::cout << std::endl << "Sum counts = " << std::setw(12) << std::setprecision(12) << total << std::endl;
  print_A_line(A, n);
}

void process_result_ancoding_mc(const u128* counts, const std::vector<dd::StatRow>& stats, uint32_t n, uint32_t A,
                                uint32_t iterations, const char* prefix, const std::string& app) {
  char tmp[192];
  double ea[64], er[64];
  dd::abs_error_an(A, n, counts, kOffset, ea);
  dd::rel_error_an(A, n, counts, kOffset, er);
  const uint32_t h = (uint32_t)std::ceil(std::log2(A));
  long double total;
  if (prefix) {
    std::snprintf(tmp, sizeof(tmp), "%s_m%u_A%u", prefix, iterations, A);
    total = process_result(counts, stats, n, h, tmp, ea, er, app);
  } else {
    total = process_result(counts, stats, n, h, nullptr, ea, er, app);
  }
  std::cout << std::endl << "Sum counts = " << std::setw(12) << std::setprecision(12) << total
            << " (with estimation factor 2^n*counts[d]/iterations)" << std::endl;
  print_A_line(A, n);
}

void process_result_hamming(const u128* counts, const std::vector<dd::StatRow>& stats, uint32_t n, uint32_t h,
                            const char* prefix) {
  long double total = process_result(counts, stats, n, h, prefix, nullptr, nullptr, "");
  std::cout << std::endl << "Sum counts = " << std::setw(12) << std::setprecision(12) << total << std::endl;
}

void process_result_hamming_mc(const u128* counts, const std::vector<dd::StatRow>& stats, uint32_t n, uint32_t h,
                               int with_1bit, uint32_t iterations, const char* prefix) {
  char tmp[192];
  double ea[64], er[64];
  dd::abs_error_hamming(n, counts, kOffset, with_1bit, ea);
  dd::rel_error_hamming(n, counts, kOffset, with_1bit, er);
  long double total;
  if (prefix) {
    std::snprintf(tmp, sizeof(tmp), "%s_m%u", prefix, iterations);
    total = process_result(counts, stats, n, h, tmp, ea, er, "");
  } else {
    total = process_result(counts, stats, n, h, nullptr, ea, er, "");
  }
  std::cout << std::endl << "Sum counts = " << std::setw(12) << std::setprecision(12) << total
            << " (with estimation factor 2^n*counts[d]/iterations)" << std::endl;
}

void fill_min(const dd_result& r, uintll_t* minb, uint128_t* mincb) {
  if (minb && mincb) {
    *minb = r.minb;
    *mincb = ((u128)r.mincb_hi << 64) | r.mincb_lo;
  }
}

void fill_times(const dd_result& r, double* times) {
  if (times) {
    times[0] = r.total_ms * 0.001;
    times[1] = r.kernel_ms * 0.001;
  }
}

void hamming_common(uintll_t n, int with_1bit, int file_output, uint32_t method, const char* prefix, bool gpu_stats_rows,
                    bool print_banner, const char* banner) {
  if (print_banner) std::printf("%s", banner);
  dd_request q = make_request(DD_CODE_EXT_HAMMING, DD_MODE_EXHAUSTIVE, 1, (uint32_t)n);
  q.with_1bit = (uint32_t)with_1bit;
  q.hamming_method = method;
  dd_result r = run_request(q);
  u128 c[DD_MAX_BINS];
  counts_of(r, c);
  process_result_hamming(c, gpu_stats_rows ? gpu_stats(r) : cpu_stats(r), (uint32_t)n, r.h,
                         file_output ? prefix : nullptr);
}

}  // namespace

// ---------------------------------------------------------------------------
// main tool drivers
// ---------------------------------------------------------------------------
void run_ancoding(uintll_t n, uintll_t A, int verbose, double* times, uintll_t* minb, uint128_t* mincb, int file_output,
                  int nr_dev) {
  (void)nr_dev;  // one GPU
  dd_request q = make_request(DD_CODE_AN, DD_MODE_EXHAUSTIVE, A, (uint32_t)n);
  q.convention = DD_CONV_GPU;
  dd_result r = run_request(q);
  fill_min(r, minb, mincb);
  fill_times(r, times);
  if (verbose || file_output) {
    u128 c[DD_MAX_BINS];
    counts_of(r, c);
    process_result_ancoding(c, gpu_stats(r), (uint32_t)n, (uint32_t)r.A, file_output ? "ancoding_gpu" : nullptr,
                            device_lines());
  }
}

void run_ancoding_cpu(uintll_t n, uintll_t A, int verbose, double* times, uintll_t* minb, uint128_t* mincb,
                      int file_output) {
  dd_request q = make_request(DD_CODE_AN, DD_MODE_EXHAUSTIVE, A, (uint32_t)n);
  q.convention = DD_CONV_CPU;
  dd_result r = run_request(q);
  if (verbose || file_output) {
    u128 c[DD_MAX_BINS];
    counts_of(r, c);
    process_result_ancoding(c, cpu_stats(r), (uint32_t)n, (uint32_t)r.A, file_output ? "ancoding_cpu" : nullptr, "");
  }
  fill_min(r, minb, mincb);
  if (times) {  // an_coding.cpp:135-139 reads indices 0 and 1 of a one-row Statistics
    times[0] = r.total_ms * 0.001;
    times[1] = 0;
  }
}

double run_ancoding_grid(int gdim, uintll_t n, uintll_t iterations, uintll_t iterations2, uintll_t A, int verbose,
                         double* times, uintll_t* minb, uint128_t* mincb, int file_output, int nr_dev) {
  (void)nr_dev;
  dd_request q = make_request(DD_CODE_AN, gdim == 2 ? DD_MODE_GRID_2D : DD_MODE_GRID_1D, A, (uint32_t)n);
  q.m = iterations;
  q.m2 = iterations2;
  dd_result r = run_request(q);
  fill_min(r, minb, mincb);
  if (verbose || file_output) {
    char fname[256];
    std::snprintf(fname, sizeof(fname), "ancoding_grid%dd_%s", gdim, "gpu");
    u128 c[DD_MAX_BINS];
    counts_of(r, c);
    process_result_ancoding_mc(c, gpu_stats(r), (uint32_t)n, (uint32_t)r.A, (uint32_t)r.iterations,
                               file_output ? fname : nullptr, device_lines());
  }
  fill_times(r, times);
  return r.max_rel_error;
}

double run_ancoding_mc(uintll_t n, uintll_t iterations, uintll_t A, int verbose, double* times, uintll_t* minb,
                       uint128_t* mincb, int file_output, int nr_dev) {
  (void)nr_dev;
  dd_request q = make_request(DD_CODE_AN, DD_MODE_MONTE_CARLO, A, (uint32_t)n);
  q.m = iterations;
  q.seed = kSeedAnMc;
  dd_result r = run_request(q);
  fill_min(r, minb, mincb);
  if (verbose || file_output) {
    u128 c[DD_MAX_BINS];
    counts_of(r, c);
    process_result_ancoding_mc(c, gpu_stats(r), (uint32_t)n, (uint32_t)r.A, (uint32_t)r.iterations,
                               file_output ? "ancoding_mc_gpu" : nullptr, "");
  }
  fill_times(r, times);
  return r.max_rel_error;
}

double run_ancoding_mc_continue(uintll_t n, uintll_t iterations, uintll_t A, double* times, McSearchState& state) {
  dd_request q = make_request(DD_CODE_AN, DD_MODE_MONTE_CARLO, A, (uint32_t)n);
  q.m = iterations;
  q.seed = kSeedAnMc;
  dd_result r;
  int st = on_shared_context([&](dd_context* c) { return dd_mc_extend(c, &q, state.it_done, state.raw, &r); });
  if (st != DD_OK) throw std::runtime_error(std::string("codrel_b200: ") + dd_last_error());
  state.it_done = r.iterations;
  for (int b = 0; b < DD_MAX_BINS; ++b) state.raw[b] = r.raw[b];
  fill_times(r, times);
  return r.max_rel_error;
}

void run_hamming(uintll_t n, int with_1bit, int file_output, int nr_dev) {
  (void)nr_dev;
  hamming_common(n, with_1bit, file_output, DD_HAMMING_WEIGHTS, "hamming_gpu", true, false, "");
}

void run_hamming_cpu(uintll_t n, int with_1bit, int file_output) {
  hamming_common(n, with_1bit, file_output, DD_HAMMING_WEIGHTS, "hamming_cpu", false, true,
                 "Start Hamming Coding Algorithm (CPU)\n");
}

void run_hamming_cpu_native(uintll_t n, int with_1bit, int file_output) {
  hamming_common(n, with_1bit, file_output, DD_HAMMING_ALL_PAIRS, "hamming_cpu_native", false, true,
                 "Start Hamming Coding Algorithm - Native Approach (CPU)\n");
}

void run_hamming_cpu_native_short(uintll_t n, int with_1bit, int file_output) {
  hamming_common(n, with_1bit, file_output, DD_HAMMING_ALL_PAIRS, "hamming_cpu_native_short", false, true,
                 "Start Hamming Coding Algorithm - Native Short Approach (CPU)\n");
}

void run_hamming_cpu_native_short_ordering(uintll_t n, int with_1bit, int file_output) {
  hamming_common(n, with_1bit, file_output, DD_HAMMING_ALL_PAIRS_DISTINCT, "hamming_cpu_native_short_ordering", false, true,
                 "Start Hamming Coding Algorithm - Native Short Approach with Ordering (CPU)\n");
}

static double hamming_sampled(uint32_t mode, uintll_t n, int with_1bit, uintll_t iterations, int file_output) {
  dd_request q = make_request(DD_CODE_EXT_HAMMING, mode, 1, (uint32_t)n);
  q.with_1bit = (uint32_t)with_1bit;
  q.m = iterations;
  q.seed = kSeedHammingMc;
  int ndev = dd_device_count();
  cudaDeviceProp prop;
  std::memset(&prop, 0, sizeof(prop));
  cudaGetDeviceProperties(&prop, 0);
  std::printf("%s with %llu iterations\n",
              mode == DD_MODE_GRID_1D ? "Start 1D Hamming-Coding Algorithm - 1D Grid"
                                      : "Start Hamming-Coding Algorithm - Monte Carlo",
              (unsigned long long)(iterations > (1ull << n) ? (1ull << n) : iterations));
  std::printf("Found %d CUDA devices (%s).\n", ndev > 1 ? 1 : ndev, prop.name);
  dd_result r = run_request(q);
  u128 c[DD_MAX_BINS];
  counts_of(r, c);
  process_result_hamming_mc(c, gpu_stats(r), (uint32_t)n, r.h, with_1bit, (uint32_t)r.iterations,
                            file_output ? "hamming_mc" : nullptr);
  return r.max_rel_error;
}

double run_hamming_grid(uintll_t n, int with_1bit, uintll_t iterations, int file_output, int nr_dev) {
  (void)nr_dev;
  return hamming_sampled(DD_MODE_GRID_1D, n, with_1bit, iterations, file_output);
}

double run_hamming_mc(uintll_t n, int with_1bit, uintll_t iterations, int file_output, int nr_dev) {
  (void)nr_dev;
  return hamming_sampled(DD_MODE_MONTE_CARLO, n, with_1bit, iterations, file_output);
}

// operator<< for uint128 (src/globals.cpp:320-341 behaviour: plain decimal digits).
std::ostream& operator<<(std::ostream& dest, uint128_t value) {
  std::ostream::sentry s(dest);
  if (s) {
    char buf[64];
    char* d = buf + sizeof(buf);
    do { *--d = "0123456789"[(int)(value % 10)]; value /= 10; } while (value != 0);
    const std::streamsize len = (buf + sizeof(buf)) - d;
    if (dest.rdbuf()->sputn(d, len) != len) dest.setstate(std::ios_base::badbit);
  }
  return dest;
}

// ---------------------------------------------------------------------------
// super-A fork
// ---------------------------------------------------------------------------
namespace supera {

static void fill_counts(const dd_result& r, uint128_t* counts) {
  for (int i = 0; i < DD_MAX_BINS; ++i) counts[i] = 0;
  for (uint32_t i = 0; i < r.nbins; ++i) counts[i] = ((u128)r.counts_hi[i] << 64) | r.counts_lo[i];
}

void run_ancoding(uintll_t A, uint_t h, Flags& flags, double* times, uint128_t* counts) {
  dd_request q = make_request(DD_CODE_AN, DD_MODE_EXHAUSTIVE, A, (uint32_t)flags.n);
  q.h = h;
  q.convention = DD_CONV_SUPER_A;
  dd_result r = run_request(q);
  fill_counts(r, counts);
  if (times) {  // super_a/src/an_coding.cu:233-237: {kernel, total}
    times[0] = r.kernel_ms * 0.001;
    times[1] = r.total_ms * 0.001;
  }
}

void run_ancoding_grid(uintll_t A, uint_t h, Flags& flags, double* times, uint128_t* counts) {
  dd_request q = make_request(DD_CODE_AN, flags.with_grid == 2 ? DD_MODE_GRID_2D : DD_MODE_GRID_1D, A,
                              (uint32_t)flags.n);
  q.h = h;
  q.m = (uint64_t)flags.mc_iterations;
  q.m2 = (uint64_t)flags.mc_iterations_2;
  q.convention = DD_CONV_SUPER_A;
  dd_result r = run_request(q);
  fill_counts(r, counts);
  if (times) {
    times[0] = r.kernel_ms * 0.001;
    times[1] = r.total_ms * 0.001;
  }
}

void run_ancoding_batch(const uintll_t* As, const uint_t* hs, size_t count, Flags& flags, double* times,
                        uint128_t* counts) {
  std::vector<dd_request> reqs(count);
  for (size_t i = 0; i < count; ++i) {
    reqs[i] = make_request(DD_CODE_AN, DD_MODE_EXHAUSTIVE, As[i], (uint32_t)flags.n);
    reqs[i].h = hs[i];
    reqs[i].convention = DD_CONV_SUPER_A;
  }
  std::vector<dd_result> res(count);
  dd_batch_options opt;
  std::memset(&opt, 0, sizeof(opt));
  opt.use_graph = 1;
  int st = on_shared_context(
      [&](dd_context* c) { return dd_batch_run(c, reqs.data(), (uint32_t)count, res.data(), &opt); });
  if (st != DD_OK) throw std::runtime_error(std::string("codrel_b200: ") + dd_last_error());
  for (size_t i = 0; i < count; ++i) {
    fill_counts(res[i], counts + i * DD_MAX_BINS);
    if (times) {  // one launch for all: its time is shared evenly between the rows
      times[2 * i] = res[i].kernel_ms * 0.001 / count;
      times[2 * i + 1] = res[i].total_ms * 0.001 / count;
    }
  }
}

// super_a/src/globals.cpp:39-116: header once (static id), then one row per A.
void process_result(std::stringstream& ss, uintll_t A, uint_t h, const Flags& flags, double* times,
                    uint128_t* counts) {
  static unsigned int id = 0;
  const char sep = ',';
  long double total = 0;
  const uint_t n = (uint_t)flags.n;
  for (uint_t i = 0; i < n + h + 1; ++i) total += (long double)counts[i];
  long double prob, base1 = std::pow(2.0, n), base2, base;
  const int cnts = (int)(flags.n + h + 1);
  if (id == 0) {
    ss << "id, k, A, h, A_2, m_1, m_2, hlen";
    for (int i = 1; i <= cnts; ++i) ss << ", p_" << i;
    for (int i = 1; i <= cnts; ++i) ss << ", hist_" << i;
    ss << ", t_kernel, t, sum, minb, mincb, superA, minb2, mincb2, superA2\n";
  }
  ss << id++ << sep << flags.n << sep << A << sep << h << sep << dd::bits_string(A, n) << sep << flags.mc_iterations
     << sep << flags.mc_iterations_2 << sep << cnts;
  for (uint_t i = 1; i <= (uint_t)cnts; ++i) {
    long double res = 1, nn = (long double)(n + h), kk = (long double)i;
    if (kk > nn - kk) kk = nn - kk;  // binomialCoeff<long double>, super_a/src/globals.h:88-105
    for (long double j = 0; j < kk; ++j) { res *= (nn - j); res /= (j + 1); }
    base2 = res;
    base = base1 * base2;
    prob = counts[i] / base;
    ss << sep << prob;
  }
  for (uint_t i = 1; i <= (uint_t)cnts; ++i) {
    if (n >= 32 && counts[i] > ((uint128_t)1 << 64))
      ss << sep << std::setprecision(12) << (long double)counts[i];
    else
      ss << sep << (uintll_t)counts[i];
  }
  for (int i = 0; i < 2; ++i) ss << sep << times[i];
  ss << sep << total;
  if (flags.verbose == 1) {
    std::cout << "Kernel: " << times[0] << " s\n"
              << "Runtime: " << times[1] << " s\n"
              << flags.n << sep << A << sep << h << sep << flags.mc_iterations << sep << flags.mc_iterations_2
              << "\n";
  }
}

}  // namespace supera

// ---------------------------------------------------------------------------
// C-ABI: results-file text
// ---------------------------------------------------------------------------
extern "C" int dd_format_result(const dd_request* req, const dd_result* res, const char* device_line, char* buf,
                                size_t cap, size_t* len) {
  if (!req || !res) { dd::set_error("NULL argument"); return DD_ERR_INVALID_ARGUMENT; }
  dd::Shape s;
  std::string err;
  int st = dd::derive_shape(*req, s, err);
  if (st != DD_OK) { dd::set_error(err); return st; }
  u128 c[DD_MAX_BINS];
  counts_of(*res, c);
  const std::string app = device_line ? device_line : "";
  std::string text;
  const bool cpu = req->convention == DD_CONV_CPU ||
                   (req->code == DD_CODE_EXT_HAMMING && req->mode == DD_MODE_EXHAUSTIVE &&
                    req->hamming_method != DD_HAMMING_WEIGHTS);
  const auto stats = cpu ? cpu_stats(*res) : gpu_stats(*res);
  if (req->code == DD_CODE_AN) {
    if (req->mode == DD_MODE_EXHAUSTIVE) {
      const uint32_t h = (uint32_t)std::ceil(std::log((uint32_t)res->A) / std::log(2.0));
      text = dd::format_table(c, stats, s.n, h, nullptr, nullptr, app, nullptr);
    } else {
      double ea[64], er[64];
      dd::abs_error_an(res->A, s.n, c, kOffset, ea);
      dd::rel_error_an(res->A, s.n, c, kOffset, er);
      const uint32_t h = (uint32_t)std::ceil(std::log2((uint32_t)res->A));
      text = dd::format_table(c, stats, s.n, h, ea, er, app, nullptr);
    }
  } else if (req->mode == DD_MODE_EXHAUSTIVE) {
    text = dd::format_table(c, stats, s.n, s.h, nullptr, nullptr, app, nullptr);
  } else {
    double ea[64], er[64];
    dd::abs_error_hamming(s.n, c, kOffset, req->with_1bit, ea);
    dd::rel_error_hamming(s.n, c, kOffset, req->with_1bit, er);
    text = dd::format_table(c, stats, s.n, s.h, ea, er, app, nullptr);
  }
  if (len) *len = text.size();
  if (buf && cap) {
    const size_t k = text.size() < cap - 1 ? text.size() : cap - 1;
    std::memcpy(buf, text.data(), k);
    buf[k] = 0;
  }
  return DD_OK;
}
