// codrel_supera_main.cpp — the super-A fork's command line
// (distance_distribution_super_a/src/main.cpp:31-387) on the B200 library.
// Exact sweeps run every A of the range (or of the candidates file) in one
// persistent, graph-captured launch instead of one launch + reset per A.
//
//   -a NUM  A;  -s NUM / -S NUM  sweep start / end;  -c FILE  candidates file
//   -m NUM  1-D grid points;  -M NUM  2-D grid;  -k NUM  data bits
//   -f STR  output prefix;  -d NUM  GPUs (one is used);  -i NUM  device;  -v NUM
#include <cuda_runtime.h>

#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/codrel_b200.h"
#include "../../include/codrel_dropin.h"

using supera::Flags;
static Flags g_flags;

static void print_help() {
  std::printf(
      "\nUSAGE:\n\n\t-h\tprint help\n"
      "\t-a NUM\t AN-coding algorithm with A=<NUM>\n"
      "\t-s NUM\t ... search super A beginning with NUM\n"
      "\t-S NUM\t ... search super A ending with NUM\n"
      "\t-c NUM\t ... search super A by file which contains the candidates\n"
      "\t-m NUM\t 1-D grid approximation with NUM iterations\n"
      "\t-M NUM\t 2-D grid approximation with NUM iterations in second dimension\n"
      "\t-k NUM\t number of bits as input size\n"
      "\t-f STR\t prefix of output file (parameters are added).\n"
      "\t-d NUM\t Number of GPUs to be used (0=max).\n"
      "\t-i NUM\t GPU device index.\n"
      "\t-v NUM\t Verbosity level (0,1,2).\n"
      "\n");
}

static void parse_cmdline(int argc, char** argv) {
  auto arg = [&](int i) { return i + 1 < argc ? argv[i + 1] : "0"; };
  for (int i = 0; i < argc; ++i) {
    if (std::strcmp(argv[i], "-h") == 0) { print_help(); std::exit(0); }
    if (std::strcmp(argv[i], "-v") == 0) {
      g_flags.verbose = std::atoi(arg(i));
    } else if (std::strcmp(argv[i], "-a") == 0) {
      g_flags.A = std::atoi(arg(i));
      if (g_flags.A == 0) g_flags.A = 1;
    } else if (std::strcmp(argv[i], "-s") == 0) {
      g_flags.search_super_A = 1;
      g_flags.search_start = std::atoi(arg(i));
    } else if (std::strcmp(argv[i], "-S") == 0) {
      g_flags.search_super_A = 1;
      g_flags.search_end = std::atoi(arg(i));
    } else if (std::strcmp(argv[i], "-c") == 0) {
      g_flags.search_super_A = 2;
      g_flags.search_file = argv[i + 1];
    } else if (std::strcmp(argv[i], "-m") == 0) {
      g_flags.with_grid = 1;
      g_flags.mc_iterations = std::atoi(arg(i));
    } else if (std::strcmp(argv[i], "-M") == 0) {
      g_flags.with_grid = 2;
      g_flags.mc_iterations_2 = std::atoi(arg(i));
    }
    if (std::strcmp(argv[i], "-f") == 0) g_flags.file_prefix = argv[i + 1];
    if (std::strcmp(argv[i], "-k") == 0) g_flags.n = std::atoi(arg(i));
    if (std::strcmp(argv[i], "-d") == 0) g_flags.nr_dev = std::atoi(arg(i));
    if (std::strcmp(argv[i], "-i") == 0) {
      g_flags.dev = std::atoi(arg(i));
      g_flags.nr_dev = 1;
    }
  }
  if (g_flags.with_grid == 2 && g_flags.mc_iterations_2 == 0) g_flags.mc_iterations_2 = g_flags.mc_iterations;
  if (g_flags.search_start > g_flags.search_end) g_flags.search_end = g_flags.search_start;
  if (g_flags.search_start == 0 && g_flags.search_end > 0) g_flags.search_start = g_flags.search_end;
  if (!g_flags.file_prefix) g_flags.file_prefix = "result";
  if (g_flags.search_super_A == 2) {
    std::ifstream f(g_flags.search_file);
    if (!f.good()) throw std::runtime_error("Candidates file does not exist.");
  }
}

static void device_info(std::ostream& info, int dev) {
  cudaDeviceProp prop;
  int rt = 0, mem = 0, clk = 0;
  size_t f = 0, t = 0;
  cudaRuntimeGetVersion(&rt);
  cudaGetDeviceProperties(&prop, dev);
  cudaSetDevice(dev);
  cudaMemGetInfo(&f, &t);
  cudaDeviceGetAttribute(&mem, cudaDevAttrMemoryClockRate, dev);
  cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, dev);
  info << '"' << prop.name << '"' << ", \"CC\", " << prop.major << '.' << prop.minor << ", \"PCI Bus ID\", "
       << prop.pciBusID << ", \"PCI Device ID\", " << prop.pciDeviceID << ", \"Multiprocessors\", "
       << prop.multiProcessorCount << ", \"Memory [MiB]\", " << t / 1048576 << ", \"MemoryFree [MiB]\", "
       << f / 1048576 << ", \"ECC enabled\", " << prop.ECCEnabled << ", \"MemClock [MHz]\", " << mem / 1000
       << ", \"GPUClock [MHz]\", " << clk / 1000 << ", \"CUDA Runtime\", " << rt;
}

// get_lowest_prob, super_a/src/main.cpp:157-170.
static void get_lowest_prob(const uint128_t* counts, size_t count_counts, uint128_t& mincb, uintll_t& minb) {
  minb = 0xFFFF;
  mincb = (uint128_t)-1;
  for (uint_t i = 1; i < (count_counts + 1) / 2; ++i) {
    if (counts[i] != 0 && counts[i] < mincb) {
      minb = i;
      mincb = counts[i];
      break;
    }
  }
}

static std::vector<uintll_t> parse_candidates_file(const char* fname) {
  std::vector<uintll_t> out;
  std::ifstream fp(fname);
  std::string line, token;
  while (std::getline(fp, line)) {
    std::stringstream ss(line);
    while (std::getline(ss, token, ',')) {
      if (token.empty()) continue;
      const uintll_t v = std::stoll(token);
      if (v == 0) std::cerr << "Read A has value 0 [ignored].\n";
      else out.push_back(v);
    }
  }
  return out;
}

// The sweep loop of super_a/src/main.cpp:194-297 over a list of A values.
static double sweep(std::stringstream& ss, const std::vector<uintll_t>& As) {
  uint128_t mincb = 0, mxmincb = (uint128_t)-1, mxmincb2 = (uint128_t)-1;
  uintll_t minb = 0, mxminb = 0, mxminb2 = 0, superA = 0, superA2 = 0;
  const uintll_t n = g_flags.n;
  double ttimes = 0;
  const char sep = ',';
  std::vector<uint_t> hs(As.size());
  for (size_t i = 0; i < As.size(); ++i) hs[i] = (uint_t)(std::floor(std::log(As[i]) / std::log(2.0)) + 1);
  std::vector<uint128_t> counts(std::max<size_t>(As.size(), 1) * DD_MAX_BINS);
  std::vector<double> times(2 * std::max<size_t>(As.size(), 1));
  if (g_flags.with_grid == 0) {
    const size_t chunk = 4096;
    for (size_t b = 0; b < As.size(); b += chunk) {
      const size_t cnt = std::min(chunk, As.size() - b);
      supera::run_ancoding_batch(As.data() + b, hs.data() + b, cnt, g_flags, times.data() + 2 * b,
                                 counts.data() + b * DD_MAX_BINS);
    }
  } else {
    for (size_t i = 0; i < As.size(); ++i)
      supera::run_ancoding_grid(As[i], hs[i], g_flags, times.data() + 2 * i, counts.data() + i * DD_MAX_BINS);
  }
  for (size_t i = 0; i < As.size(); ++i) {
    const uintll_t A = As[i];
    const uint_t h = hs[i];
    uint128_t* c = counts.data() + i * DD_MAX_BINS;
    get_lowest_prob(c, n + h + 1, mincb, minb);
    if (mxminb < minb || (mxminb == minb && mxmincb > mincb)) {
      mxminb = minb;
      mxmincb = mincb;
      superA = A;
    }
    if (mxminb2 < minb || (mxminb2 == minb && mxmincb2 > mincb)) {
      mxminb2 = minb;
      mxmincb2 = mincb;
      superA2 = A;
    }
    ttimes += times[2 * i + 1];
    supera::process_result(ss, A, h, g_flags, times.data() + 2 * i, c);
    ss << sep << mxminb << sep << mxmincb << sep << superA << sep << mxminb2 << sep << mxmincb2 << sep << superA2;
    ss << "\n";
    if (((A + 1) & ~A) == (A + 1)) {  // A+1 a power of two: the next A starts a new class
      mxmincb2 = (uint128_t)-1;
      mxminb2 = 0;
      superA2 = 0;
    }
  }
  return ttimes;
}

int main(int argc, char** argv) {
  std::stringstream ss;
  char fname[512];
  double ttimes = 0;
  int ndevs = 0;
  if (cudaGetDeviceCount(&ndevs) != cudaSuccess || ndevs == 0) {
    std::fprintf(stderr, "No CUDA capable device found\n");
    return 2;
  }
  for (int i = 0; i < ndevs; ++i) {
    device_info(std::cout, i);
    std::cout << std::endl;
  }
  if (argc < 2) {
    print_help();
    return 0;
  }
  try {
    parse_cmdline(argc, argv);
    device_info(ss, g_flags.dev >= 0 ? g_flags.dev : 0);
    ss << "\n";
    if (g_flags.search_super_A == 1) {
      std::snprintf(fname, sizeof(fname), "%s_k%u_a%u-%u.csv", g_flags.file_prefix, (unsigned)g_flags.n,
                    (unsigned)g_flags.search_start, (unsigned)g_flags.search_end);
      std::vector<uintll_t> As;
      for (uintll_t A = g_flags.search_start; A <= g_flags.search_end; A += 2) As.push_back(A);
      ttimes = sweep(ss, As);
    } else if (g_flags.search_super_A == 2) {
      std::string tmp(g_flags.search_file);
      std::replace(tmp.begin(), tmp.end(), '/', '_');
      std::snprintf(fname, sizeof(fname), "%s_k%u_c_%s.csv", g_flags.file_prefix, (unsigned)g_flags.n, tmp.c_str());
      ttimes = sweep(ss, parse_candidates_file(g_flags.search_file));
    } else {
      uint128_t counts[DD_MAX_BINS] = {0};
      double times[2] = {0};
      const uint_t h = (uint_t)std::ceil(std::log(g_flags.A) / std::log(2.0));
      if (g_flags.with_grid) {
        std::snprintf(fname, sizeof(fname), "%s_k%u_h%u_a%u_g%u.csv", g_flags.file_prefix, (unsigned)g_flags.n, h,
                      (unsigned)g_flags.A, (unsigned)g_flags.with_grid);
        supera::run_ancoding_grid(g_flags.A, h, g_flags, times, counts);
      } else {
        std::snprintf(fname, sizeof(fname), "%s_k%u_h%u_a%u.csv", g_flags.file_prefix, (unsigned)g_flags.n, h,
                      (unsigned)g_flags.A);
        supera::run_ancoding(g_flags.A, h, g_flags, times, counts);
      }
      supera::process_result(ss, g_flags.A, h, g_flags, times, counts);
      ttimes = times[1];
    }
  } catch (const std::exception& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 2;
  }
  std::ofstream fp(fname);
  fp << "\"Total Time [s]\"," << ttimes << "\n";
  fp << ss.str();
  fp.close();
  return 0;
}
