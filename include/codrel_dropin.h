/*
 * codrel_dropin.h — C++ drop-in replacements for the reference's driver
 * functions, same names, signatures and output behaviour (stdout table,
 * optional results file), implemented on top of the C-ABI in codrel_b200.h.
 *
 *   distance_distribution/src/algorithms.h:20-34   (main tool)
 *   distance_distribution_super_a/src/algorithms.h:20-21 (super-A fork)
 *
 * Differences a caller can observe: every histogram is computed on one GPU
 * (the `_cpu*` entry points keep their file prefixes and conventions but do
 * not run on the CPU), errors are reported by exception instead of exit(), and
 * Monte Carlo draws come from Philox4x32-10.
 */
#ifndef CODREL_DROPIN_H_
#define CODREL_DROPIN_H_

#include <string>

typedef unsigned uint_t;
typedef unsigned long long uintll_t;
typedef unsigned __int128 uint128_t;

/* main tool, src/algorithms.h:20-30 */
void run_hamming(uintll_t n, int with_1bit, int file_output, int nr_dev);
void run_hamming_cpu(uintll_t n, int with_1bit, int file_output);
void run_hamming_cpu_native(uintll_t n, int with_1bit, int file_output);
void run_hamming_cpu_native_short(uintll_t n, int with_1bit, int file_output);
void run_hamming_cpu_native_short_ordering(uintll_t n, int with_1bit, int file_output);
void run_ancoding(uintll_t n, uintll_t A, int verbose, double* times, uintll_t* minb, uint128_t* mincb,
                  int file_output, int nr_dev);
void run_ancoding_cpu(uintll_t n, uintll_t A, int verbose, double* times, uintll_t* minb, uint128_t* mincb,
                      int file_output);
double run_hamming_mc(uintll_t n, int with_1bit, uintll_t iterations, int file_output, int nr_dev);
double run_ancoding_mc(uintll_t n, uintll_t iterations, uintll_t A, int verbose, double* times, uintll_t* minb,
                       uint128_t* mincb, int file_output, int nr_dev);
/* Addition without a counterpart in the reference: the Monte Carlo step of the
 * error-bound search (src/main.cpp:179-202) that continues from the previous
 * step's samples instead of redrawing them (dd_mc_extend).  `state` starts
 * zeroed; each call grows it to `iterations` samples per codeword.  Returns the
 * same max. rel. error as run_ancoding_mc(n, iterations, A, ...) would. */
struct McSearchState {
  uintll_t it_done = 0;
  uint64_t raw[DD_MAX_BINS] = {0};
};
double run_ancoding_mc_continue(uintll_t n, uintll_t iterations, uintll_t A, double* times, McSearchState& state);
double run_ancoding_grid(int gdim, uintll_t n, uintll_t iterations, uintll_t iterations2, uintll_t A, int verbose,
                         double* times, uintll_t* minb, uint128_t* mincb, int file_output, int nr_dev);
double run_hamming_grid(uintll_t n, int with_1bit, uintll_t iterations, int file_output, int nr_dev);

std::ostream& operator<<(std::ostream& dest, uint128_t value);

namespace supera {
/* Flags of the super-A fork, distance_distribution_super_a/src/globals.h:51-65. */
struct Flags {
  uintll_t A = 61;
  int with_grid = 0;
  int mc_iterations = 0;
  int mc_iterations_2 = 0;
  uintll_t n = 16;
  int search_super_A = 0;
  uintll_t search_start = 0;
  uintll_t search_end = 0;
  int nr_dev = 0;
  int dev = -1;
  int verbose = 0;
  const char* search_file = nullptr;
  const char* file_prefix = nullptr;
};
/* super_a/src/algorithms.h:20-21: counts[] must hold COUNTS_MAX_WIDTH (64) entries;
 * times = {kernel, total} seconds. */
void run_ancoding(uintll_t A, uint_t h, Flags& flags, double* times, uint128_t* counts);
void run_ancoding_grid(uintll_t A, uint_t h, Flags& flags, double* times, uint128_t* counts);
/* Many A values in one persistent launch (the batched form of the sweeps in
 * super_a/src/main.cpp:194-297).  counts: count x 64 entries; times[2*i..]. */
void run_ancoding_batch(const uintll_t* As, const uint_t* hs, size_t count, Flags& flags, double* times,
                        uint128_t* counts);
/* One CSV row per A, super_a/src/globals.cpp:39-116 (static row id). */
void process_result(std::stringstream& ss, uintll_t A, uint_t h, const Flags& flags, double* times,
                    uint128_t* counts);
}  // namespace supera

#endif /* CODREL_DROPIN_H_ */
