// codrel_main.cpp — the reference tool's command line (flags, defaults and
// dispatch of distance_distribution/src/main.cpp:22-270) on the B200 library.
//
//   -e NUM  Ext-Hamming (1 = weight enumerator, 2/4 = all ordered pairs, 3 = pairs a<b)
//   -b      ... with 1-bit spheres
//   -a NUM  AN code with A=NUM
//   -g NUM  1 = 1-D grid, 2 = 2-D grid, with -m NUM points (-M for the 2nd dim)
//   -s DEC  AN Monte Carlo: triple the iterations until max. rel. error <= DEC
//   -S NUM  super-A search for 2^(NUM-1) < A < 2^NUM
//   -m NUM  Monte Carlo iterations / grid points;  -M NUM  2nd grid dimension
//   -n NUM  data bits;  -c  CPU-path conventions (the histogram still runs on the GPU)
//   -f      results file;  -d NUM  GPUs (one is used);  -v NUM  verbosity
//   -t NUM  cuRAND generator test: not provided (cuRAND is not used)
#include <cassert>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <stdexcept>
#include <vector>

#include "../../include/codrel_b200.h"
#include "../../include/codrel_dropin.h"

struct Flags {
  int an_coding;
  uintll_t A;
  int h_coding;
  int with_1bit;
  int with_mc;
  int with_grid;
  int mc_iterations;
  int mc_iterations_2;
  uintll_t n;
  int use_cpu;
  int rand_gen;
  double mc_search_bound;
  int search_super_A;
  int file_output;
  int nr_dev;
  int verbose;
} g_flags = {0, 61, 0, 0, 0, 0, 100, 0, 8, 0, 0, -1.0, 0, 0, 0, 1};  // src/main.cpp:39

static void print_help() {
  std::printf(
      "\nUSAGE:\n\n\t-h\tprint help\n"
      "\t-e NUM\t Extended Hamming-coding algorithm (1=optimized, 2=naive, 3=naive+ordering, 4=as [2]+more optimizations)\n"
      "\t-b    \t ... with 1-bit spheres\n"
      "\t-a NUM\t AN-coding algorithm with A=<NUM>\n"
      "\t-g NUM\t 1=1D-Grid 2=2D-Grid approximation with -m NUM points per dim. (Better than MonteCarlo)\n"
      "\t-s DEC\t ... AN-coding search optimal number of monte carlo iterations for given error bound <1.0.\n"
      "\t      \t -m or -M gives start value of number of iterations.\n"
      "\t-S NUM\t ... search super A within 2^NUM<A<2^(NUM+1)\n"
      "\t-m NUM\t Monte-Carlo with number of iterations, GPU, for -e 2 and -a\n"
      "\t-M NUM\t ... number of iterations in second dimension for 2D grid\n"
      "\t-n NUM\t number of bits as input size\n"
      "\t-c    \t use CPU implementation (has effect on -e 1 and -a)\n"
      "\t-t NUM\t test curand generator with number of iterations\n"
      "\t-f    \t with file output (file name is generated).\n"
      "\t-d NUM\t Number of GPUs to be used (0=max).\n"
      "\t-v NUM\t Verbosity level (0,1,2).\n"
      "\n");
}

static void parse_cmdline(int argc, char** argv) {
  g_flags.h_coding = 1;
  g_flags.file_output = 0;
  auto arg = [&](int i) { return i + 1 < argc ? argv[i + 1] : "0"; };
  for (int i = 0; i < argc; ++i) {
    if (std::strcmp(argv[i], "-h") == 0) { print_help(); std::exit(0); }
    if (std::strcmp(argv[i], "-v") == 0) {
      g_flags.verbose = std::atoi(arg(i));
    } else if (std::strcmp(argv[i], "-a") == 0) {
      g_flags.an_coding = 1;
      g_flags.h_coding = 0;
      g_flags.A = std::atoi(arg(i));
      if (g_flags.A == 0) g_flags.A = 1;
    } else if (std::strcmp(argv[i], "-e") == 0) {
      g_flags.h_coding = std::atoi(arg(i));
      g_flags.an_coding = 0;
    } else if (std::strcmp(argv[i], "-c") == 0) {
      g_flags.use_cpu = 1;
    } else if (std::strcmp(argv[i], "-s") == 0) {
      g_flags.mc_search_bound = std::atof(arg(i));
    } else if (std::strcmp(argv[i], "-S") == 0) {
      g_flags.search_super_A = std::atoi(arg(i));
    } else if (std::strcmp(argv[i], "-t") == 0) {
      g_flags.rand_gen = 1;
      g_flags.mc_iterations = std::atoi(arg(i));
    } else if (std::strcmp(argv[i], "-m") == 0) {
      g_flags.with_mc = 1;
      g_flags.mc_iterations = std::atoi(arg(i));
    } else if (std::strcmp(argv[i], "-M") == 0) {
      g_flags.with_mc = 1;
      g_flags.with_grid = 2;
      g_flags.mc_iterations_2 = std::atoi(arg(i));
    } else if (std::strcmp(argv[i], "-g") == 0) {
      g_flags.with_grid = std::atoi(arg(i));
    }
    if (std::strcmp(argv[i], "-f") == 0) g_flags.file_output = 1;
    if (std::strcmp(argv[i], "-b") == 0) g_flags.with_1bit = 1;
    if (std::strcmp(argv[i], "-n") == 0) g_flags.n = std::atoi(arg(i));
    if (std::strcmp(argv[i], "-d") == 0) g_flags.nr_dev = std::atoi(arg(i));
  }
  if (g_flags.h_coding && g_flags.n != 4 && g_flags.n != 8 && g_flags.n != 16 && g_flags.n != 24 && g_flags.n != 32 &&
      g_flags.n != 40 && g_flags.n != 48) {
    g_flags.n = 8;
    std::printf("Wrong input size, so set n to 8.\n");
  }
  if (g_flags.with_grid == 2 && g_flags.mc_iterations_2 == 0) g_flags.mc_iterations_2 = g_flags.mc_iterations;
}

// src/main.cpp:131-177, the sweep run as one batched launch for exact k<=16.
static void ancoding_search_super_A() {
  uint128_t mincb = 0, mxmincb = (uint128_t)-1, mxmincb2 = (uint128_t)-1;
  uintll_t minb = 0, mxminb = 0, mxminb2 = 0, A2 = 0;
  const uintll_t n = g_flags.n;
  uintll_t A = (1 << (g_flags.search_super_A - 1)) + 1;
  const uintll_t A_end = (1 << (g_flags.search_super_A)) - 1;
  uintll_t superA = 0;
  double times[2] = {0};
  double ttimes = 0;
  // Exact sweeps (n <= 16) run all A values in one persistent launch; the
  // per-A results are then walked in the reference's order.
  std::vector<dd_result> batch;
  if (n <= 16 && A <= A_end) {
    std::vector<dd_request> reqs;
    for (uintll_t a = A; a <= A_end; a += 2) {
      dd_request q;
      std::memset(&q, 0, sizeof(q));
      q.code = DD_CODE_AN;
      q.mode = DD_MODE_EXHAUSTIVE;
      q.A = a;
      q.n = (uint32_t)n;
      q.convention = DD_CONV_GPU;
      reqs.push_back(q);
    }
    batch.resize(reqs.size());
    dd_context* ctx = nullptr;
    if (dd_context_create(0, nullptr, &ctx) != DD_OK) throw std::runtime_error(dd_last_error());
    dd_batch_options opt;
    std::memset(&opt, 0, sizeof(opt));
    opt.use_graph = 1;
    int st = dd_batch_run(ctx, reqs.data(), (uint32_t)reqs.size(), batch.data(), &opt);
    dd_context_destroy(ctx);
    if (st != DD_OK) throw std::runtime_error(dd_last_error());
  }
  for (size_t idx = 0; A <= A_end; A += 2, ++idx) {
    if (n <= 16) {
      const dd_result& r = batch[idx];
      minb = r.minb;
      mincb = ((uint128_t)r.mincb_hi << 64) | r.mincb_lo;
      times[0] = r.total_ms * 0.001 / batch.size();
      times[1] = r.kernel_ms * 0.001 / batch.size();
    } else {
      run_ancoding_grid(g_flags.with_grid, g_flags.n, g_flags.mc_iterations, g_flags.mc_iterations_2, A, 0, times,
                        &minb, &mincb, 0, g_flags.nr_dev);
    }
    if (mxminb < minb || (mxminb == minb && mxmincb > mincb)) {
      if (mxminb != minb) {
        mxminb2 = mxminb;
        mxmincb2 = mxmincb;
        A2 = superA;
      }
      mxminb = minb;
      mxmincb = mincb;
      superA = A;
      std::cout << A << ": c[" << minb << "] = " << mincb << std::endl;
    }
    ttimes += times[1];
  }
  std::cout << "n," << n << ",h," << g_flags.search_super_A << ",superA," << superA << ",prevA," << A2 << ",c["
            << mxminb << "]," << mxmincb << ",c[" << mxminb2 << "]," << mxmincb2 << ",time[s]," << ttimes
            << (n <= 16 ? ",exact" : ",grid") << std::endl;
}

// src/main.cpp:179-202, with one difference: each step continues from the
// previous step's samples (run_ancoding_mc_continue draws only the new ones;
// the histogram equals a fresh run with the step's iterations), so a step's
// times are those of its new samples.
static void ancoding_mc_search() {
  int step = 0;
  double cur_err = 1.0;
  uintll_t nr_iterations = g_flags.mc_iterations;
  if (nr_iterations < 1) nr_iterations = 1;
  std::printf("AN-Coding MonteCarlo starting with %llu iterations\n", nr_iterations);
  FILE* f = std::fopen("ancoding_mc_search.csv", "w");
  double times[2];
  McSearchState state;
  while (true) {
    cur_err = run_ancoding_mc_continue(g_flags.n, nr_iterations, g_flags.A, times, state);
    std::printf("%llu iterations - max. rel. error %lf\n", nr_iterations, cur_err);
    if (f)
      std::fprintf(f, "%d,%llu,%lf,%llu,%lf,%lf,%lf\n", step, g_flags.n, g_flags.mc_search_bound, nr_iterations,
                   cur_err, times[0], times[1]);
    if (cur_err <= g_flags.mc_search_bound) break;
    if (cur_err < 0) {
      std::printf("No golden table for A=%llu, n=%llu: the error bound cannot be checked.\n", g_flags.A, g_flags.n);
      break;
    }
    if (nr_iterations >= (1ull << g_flags.n)) break;  // capped at 2^n: more iterations change nothing
    nr_iterations *= 3;
    ++step;
  }
  if (f) std::fclose(f);
  std::printf("Achieved error of %lf after %llu iterations\n", cur_err, nr_iterations);
}

int main(int argc, char** argv) {
  if (argc < 2) {
    print_help();
    return 0;
  }
  parse_cmdline(argc, argv);
  try {
    if (g_flags.rand_gen) {
      std::printf("-t: the cuRAND generator test is not part of this build (Monte Carlo uses Philox4x32-10).\n");
      return 1;
    } else if (g_flags.an_coding || g_flags.search_super_A) {
      if (g_flags.mc_search_bound > 0.0)
        ancoding_mc_search();
      else if (g_flags.search_super_A)
        ancoding_search_super_A();
      else if (g_flags.with_mc) {
        if (g_flags.with_grid)
          run_ancoding_grid(g_flags.with_grid, g_flags.n, g_flags.mc_iterations, g_flags.mc_iterations_2, g_flags.A,
                            g_flags.verbose, nullptr, nullptr, nullptr, g_flags.file_output, g_flags.nr_dev);
        else
          run_ancoding_mc(g_flags.n, g_flags.mc_iterations, g_flags.A, g_flags.verbose, nullptr, nullptr, nullptr,
                          g_flags.file_output, g_flags.nr_dev);
      } else if (g_flags.use_cpu)
        run_ancoding_cpu(g_flags.n, g_flags.A, g_flags.verbose, nullptr, nullptr, nullptr, g_flags.file_output);
      else
        run_ancoding(g_flags.n, g_flags.A, g_flags.verbose, nullptr, nullptr, nullptr, g_flags.file_output,
                     g_flags.nr_dev);
    } else if (g_flags.h_coding == 1) {
      if (g_flags.use_cpu)
        run_hamming_cpu(g_flags.n, g_flags.with_1bit, g_flags.file_output);
      else if (g_flags.with_grid)
        run_hamming_grid(g_flags.n, g_flags.with_1bit, g_flags.mc_iterations, g_flags.file_output, g_flags.nr_dev);
      else if (g_flags.with_mc)
        run_hamming_mc(g_flags.n, g_flags.with_1bit, g_flags.mc_iterations, g_flags.file_output, g_flags.nr_dev);
      else
        run_hamming(g_flags.n, g_flags.with_1bit, g_flags.file_output, g_flags.nr_dev);
    } else if (g_flags.h_coding == 2) {
      run_hamming_cpu_native_short(g_flags.n, g_flags.with_1bit, g_flags.file_output);
    } else if (g_flags.h_coding == 3) {
      run_hamming_cpu_native_short_ordering(g_flags.n, g_flags.with_1bit, g_flags.file_output);
    } else if (g_flags.h_coding == 4) {
      run_hamming_cpu_native(g_flags.n, g_flags.with_1bit, g_flags.file_output);
    }
  } catch (const std::exception& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 2;
  }
  return 0;
}
