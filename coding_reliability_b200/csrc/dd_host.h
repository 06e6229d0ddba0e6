// dd_host.h — internal C++ interface of the host layer (shape rules, planning,
// post-processing, result formatting).  Used by the C-ABI (dd_host.cu) and by
// the drop-in shims with the reference's signatures (dd_dropin.cpp).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/codrel_b200.h"
#include "dd_jobs.h"

namespace dd {

typedef unsigned __int128 u128;

// Everything the drivers derive from a request before launching.
struct Shape {
  uint32_t code = 0, mode = 0, n = 0, h = 0, nbins = 0;
  uint64_t A = 1;            // after the convention's normalisation
  uint64_t m = 0, m2 = 0;    // capped iterations
  uint64_t lattice = 0;      // grid: lattice points K actually visited
  uint64_t samples = 0;      // Ext-Hamming grid / MC: generated messages
  bool wide = false;         // codewords need more than 32 bits
  bool t32 = false;          // the reference's T is uint32 for lattice casts
  double step = 0, step2 = 0;
  uint32_t bucket = 0, shard = 0;
};

// The reference's h rules.
uint32_t h_ceil_log2(uint64_t A);      // ceil(log(A)/log(2.0)), src/an_coding.cu:280
uint32_t h_floor_log2_p1(uint64_t A);  // floor(log(A)/log(2.0))+1, super_a/src/main.cpp:261
uint32_t hamming_h(uint32_t n);        // src/hamming.cu:133

// Fills `s` or returns a dd_status with a message in `err`.
int derive_shape(const dd_request& req, Shape& s, std::string& err);
// Appends the device job(s) for one request; bins pointer is filled by the caller.
void plan_jobs(const Shape& s, const dd_request& req, std::vector<Job>& jobs);
uint64_t job_tiles(const Job& j);
// Distance evaluations one request's jobs perform.
u128 planned_pairs(const Shape& s, const dd_request& req);

// Post-processing of the raw histogram into res (counts, minb, error).
void postprocess(const dd_request& req, const Shape& s, const uint64_t* raw, dd_result& res);

// Reference golden tables (src/solutions.h) and error estimates (src/globals.cpp:65-183).
double rel_error_an(uint64_t A, uint32_t n, const u128* tgt, int offset, double* errors);
double abs_error_an(uint64_t A, uint32_t n, const u128* tgt, int offset, double* errors);
double rel_error_hamming(uint32_t n, const u128* tgt, int offset, int w1bit, double* errors);
double abs_error_hamming(uint32_t n, const u128* tgt, int offset, int w1bit, double* errors);

// Text of one results file as process_result (src/globals.cpp:185-244) builds
// it.  `stats` holds (label, value) rows in the Statistics order.
struct StatRow { std::string label; double value; std::string unit; };
std::string format_table(const u128* counts, const std::vector<StatRow>& stats, uint32_t n, uint32_t h,
                         const double* errors_abs, const double* errors_rel, const std::string& app,
                         long double* total_out);
std::string bits_string(uint64_t v, uint64_t n);  // printbits, src/globals.cpp:306-315

void set_error(const std::string& msg);

// Round launcher of the query server: one launch over job sub-ranges
// (Job::tile_offset/tiles) whose bins point into caller-owned device memory,
// accumulated across rounds (the bins are not reset).
int launch_round(dd_context* ctx, std::vector<Job>& jobs, const std::vector<uint32_t>& kernels, float* kernel_ms);
bool uses_mma(const dd_context* ctx, const Job& j, uint32_t kernel);
uint32_t mma_epilogue_used(const dd_context* ctx);  // dd_mma_epilogue of the context's tcgen05 launches
void* context_stream(const dd_context* ctx);
int context_device(const dd_context* ctx);

}  // namespace dd
