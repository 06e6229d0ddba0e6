// codrel_ancandidates_main.cpp — drop-in for the reference's ANcandidates tool
// (ANcandidates/ANcandidates.cpp:150-301): same flags (-a/--Amin, -A/--Amax,
// -d/--Dmin, -D/--Dmax, -h/--help/-?), same return codes for bad command lines,
// same stdout (two range comments, a header, one tab-separated row per
// (A width, data width) cell, A width in the outer loop), computed on the GPU
// by dd_an_candidates.
//
// Differences: each row lists its candidates in ascending order (the
// reference's OpenMP workers append them in completion order); a missing flag
// value is reported instead of read past argv.  Additions:
//   --csv PREFIX   also write each cell's candidates, comma-separated on one
//                  line, to PREFIX_k<k>_a<a>.csv: the candidates-file format
//                  that codrel_supera -c reads (super_a/src/main.cpp:172-192)
//   --device N     GPU to use (default 0)
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/codrel_b200.h"

struct Config {
  size_t minD = 0, maxD = 0, minA = 0, maxA = 0;
  std::string csv;
  int device = 0;
};

static void help(const char* argv0) {
  std::string base(argv0);
  const size_t pos = base.find_last_of('/');
  std::cout << "USAGE: " << base.substr(pos == std::string::npos ? 0 : pos)
            << " -a|--Amin -A|--Amax -d|--dMin -D|--dMax\n"
               "\n\t-? -h --help               Print this message."
               "\n\t-a --Amin                  Minimum width of A [bits]."
               "\n\t-A --Amax                  Maximum width of A [bits]."
               "\n\t-d --Dmin                  Minimum data width [bits]."
               "\n\t-D --Dmax                  Maximum data width [bits]."
               "\n\t--csv PREFIX               Also write PREFIX_k<k>_a<a>.csv candidate files."
               "\n\t--device N                 GPU to use."
            << std::endl;
}

// Mirrors parseCmdArgs (ANcandidates.cpp:185-233): 255 for help, 1..4 for a
// value flag without a value, 100 when a width is missing or zero.
static int parse(int argc, char** argv, Config& c) {
  struct Flag {
    const char *s, *l;
    size_t* dst;
    int code;
  } flags[] = {{"-a", "--Amin", &c.minA, 1}, {"-A", "--Amax", &c.maxA, 2}, {"-d", "--Dmin", &c.minD, 3},
               {"-D", "--Dmax", &c.maxD, 4}};
  for (int i = 1; i < argc; ++i) {
    if (!std::strcmp(argv[i], "-h") || !std::strcmp(argv[i], "--help") || !std::strcmp(argv[i], "-?")) {
      help(argv[0]);
      return 255;
    }
    bool matched = false;
    for (const Flag& f : flags) {
      if (!std::strcmp(argv[i], f.s) || !std::strcmp(argv[i], f.l)) {
        matched = true;
        if (i + 1 >= argc) {
          std::cerr << "argument '" << argv[i] << "' requires an additional number!" << std::endl;
          return f.code;
        }
        *f.dst = std::strtoull(argv[++i], nullptr, 0);
      }
    }
    if (matched) continue;
    if (!std::strcmp(argv[i], "--csv") && i + 1 < argc) {
      c.csv = argv[++i];
    } else if (!std::strcmp(argv[i], "--device") && i + 1 < argc) {
      c.device = std::atoi(argv[++i]);
    }
  }
  if (c.minA == 0 || c.maxA == 0 || c.minD == 0 || c.maxD == 0) {
    help(argv[0]);
    return 100;
  }
  return 0;
}

int main(int argc, char** argv) {
  Config conf;
  if (int ret = parse(argc, argv, conf)) return ret;
  if (conf.maxD < conf.minD || conf.maxA < conf.minA) {
    std::cerr << "empty range of widths" << std::endl;
    return 5;
  }
  dd_context* ctx = nullptr;
  if (int st = dd_context_create(conf.device, nullptr, &ctx)) {
    std::cerr << "dd_context_create: " << dd_status_string(st) << ": " << dd_last_error() << std::endl;
    return 6;
  }
  const size_t numD = conf.maxD - conf.minD + 1, numAw = conf.maxA - conf.minA + 1;
  std::cout << "# bit width data = [" << conf.minD << ',' << conf.maxD << "]\n";
  std::cout << "# bit width A = [" << conf.minA << ',' << conf.maxA << "]\n";
  std::cout << "# n=|C|\tk=|D|\t|A|\t|SDR|\t|candidates|\tcandidates\n";
  int rc = 0;
  std::vector<uint64_t> list;
  for (size_t cell = 0; cell < numD * numAw; ++cell) {
    const uint32_t k = (uint32_t)(conf.minD + cell % numD);
    const uint32_t a = (uint32_t)(conf.minA + cell / numD);
    const uint64_t numA = a >= 2 ? (1ull << (a - 2)) : 0;
    list.resize((size_t)std::min<uint64_t>(std::max<uint64_t>(numA, 1), 1ull << 24));
    dd_candidates_result r;
    if (int st = dd_an_candidates(ctx, k, a, list.data(), list.size(), &r)) {
      std::cerr << "dd_an_candidates(k=" << k << ", a=" << a << "): " << dd_status_string(st) << ": "
                << dd_last_error() << std::endl;
      rc = 7;
      break;
    }
    const size_t shown = (size_t)std::min<uint64_t>(r.num_candidates, list.size());
    std::stringstream ss;
    ss << (k + a) << '\t' << k << '\t' << a << '\t' << r.sdr << '\t' << r.num_candidates << '\t';
    for (size_t i = 0; i < shown; ++i) ss << (i ? "," : "") << list[i];
    ss << '\n';
    std::cout << ss.str() << std::flush;
    if (!conf.csv.empty()) {
      std::ofstream f(conf.csv + "_k" + std::to_string(k) + "_a" + std::to_string(a) + ".csv");
      for (size_t i = 0; i < shown; ++i) f << (i ? "," : "") << list[i];
      f << '\n';
    }
  }
  dd_context_destroy(ctx);
  return rc;
}
