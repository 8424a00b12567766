// `spgemm` -- drop-in replacement for the reference's two executables.
//
// Same flags as optixSpMSpM (optixSpMSpM/src/optixSpMSpM/optixSpMSpM.cpp:
// 513-562) and cuSparse (cuSparse/src/main.cpp:601-645):
//   -m1/--mat1 A.mtx  -m2/--mat2 B.mtx  -o/--output C.mtx  -l/--log log.txt
//   -h/--help
// and the same contract: the log file receives one number, the milliseconds
// of the timed region (reference Timing::flushTimer, sutil/Timing.h:92-100),
// which -- like the reference's "computation time no io" region
// (optixSpMSpM.cpp:585-611, main.cpp:383-547) -- starts after the inputs are
// parsed and ends when C is complete on the device.  Exit code 0 on success,
// 1 on any failure (optixSpMSpM.cpp:654-659).
// Extra flags: --algo plain|learned|cusparse, --json report.json,
// --tune-cache tune.json, --drop-zeros (skip exact zeros like the
// ray-tracing writer), --device N, --mlp weights.bin, --transpose-m2 (C =
// A * B^T for rectangular inputs; the reference harness leaves these as a
// TODO, scripts/AE_test.py:165-171), --check (after the timed region, C is
// recomputed in FP64 on the GPU and its errors are printed and added to the
// --json report).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/rtspmspm.h"

namespace {

void usage(const char* argv0) {
  std::fprintf(stderr,
               "Usage  : %s [options]\n"
               "Options: --output | -o <filename>    Specify file for the result matrix\n"
               "         --mat1 | -m1 <filename>     Specify file for matrix 1\n"
               "         --mat2 | -m2 <filename>     Specify file for matrix 2\n"
               "         --log  | -l  <filename>     Specify file for log\n"
               "         --algo plain|learned|cusparse\n"
               "         --json <filename>           Per-stage report\n"
               "         --tune-cache <filename>     Autotune (cached per shape class and GPU)\n"
               "         --mlp <filename>            Predictor weights for --algo learned\n"
               "         --drop-zeros                Skip entries whose value is exactly 0\n"
               "         --transpose-m2              Multiply by the transpose of matrix 2\n"
               "         --check                     Report C's error against an FP64 recomputation\n"
               "         --device <n>\n"
               "         --help | -h                 Print this usage message\n",
               argv0);
  std::exit(1);
}

int die(spg_ctx* ctx, const char* what, spg_status st) {
  std::fprintf(stderr, "spgemm: %s failed: %s (%s)\n", what, spg_status_string(st), ctx ? spg_last_error(ctx) : "");
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  std::string m1, m2, out, log, json, tune_cache, mlp;
  int algo = SPG_ALGO_LEARNED, device = 0, drop_zeros = 0, transpose_b = 0, check = 0;
  for (int i = 1; i < argc; ++i) {
    const std::string a(argv[i]);
    auto next = [&]() -> std::string {
      if (i + 1 >= argc) usage(argv[0]);
      return std::string(argv[++i]);
    };
    if (a == "-h" || a == "--help") usage(argv[0]);
    else if (a == "-m1" || a == "--mat1") m1 = next();
    else if (a == "-m2" || a == "--mat2") m2 = next();
    else if (a == "-o" || a == "--output") out = next();
    else if (a == "-l" || a == "--log") log = next();
    else if (a == "--json") json = next();
    else if (a == "--tune-cache") tune_cache = next();
    else if (a == "--mlp") mlp = next();
    else if (a == "--drop-zeros") drop_zeros = 1;
    else if (a == "--transpose-m2") transpose_b = 1;
    else if (a == "--check") check = 1;
    else if (a == "--device") device = std::atoi(next().c_str());
    else if (a == "--algo") {
      const std::string v = next();
      if (v == "plain") algo = SPG_ALGO_PLAIN;
      else if (v == "learned") algo = SPG_ALGO_LEARNED;
      else if (v == "cusparse") algo = SPG_ALGO_CUSPARSE;
      else usage(argv[0]);
    } else {
      std::fprintf(stderr, "Unknown option %s\n", a.c_str());
      usage(argv[0]);
    }
  }
  if (m1.empty()) usage(argv[0]);
  if (m2.empty()) m2 = m1;
  spg_csr A{}, B{};
  spg_status st = spg_mtx_read(m1.c_str(), &A);
  if (st != SPG_OK) return die(nullptr, ("reading " + m1).c_str(), st);
  st = spg_mtx_read(m2.c_str(), &B);
  if (st != SPG_OK) return die(nullptr, ("reading " + m2).c_str(), st);
  if (transpose_b) {
    spg_csr T{};
    if ((st = spg_csr_transpose(&B, &T)) != SPG_OK) return die(nullptr, "transposing -m2", st);
    spg_csr_free(nullptr, &B);
    B = T;
  }
  if (A.cols != B.rows) {
    std::fprintf(stderr, "spgemm: inner dimensions differ (%lld vs %lld)\n", (long long)A.cols, (long long)B.rows);
    return 1;
  }
  spg_ctx* ctx = nullptr;
  st = spg_create(&ctx, device);
  if (st != SPG_OK) return die(nullptr, "spg_create", st);
  if (!mlp.empty() && (st = spg_mlp_load(ctx, mlp.c_str())) != SPG_OK) return die(ctx, "spg_mlp_load", st);
  spg_opts o{};
  o.algo = algo;
  o.stage_timing = json.empty() ? 0 : 1;
  if (!tune_cache.empty() && algo != SPG_ALGO_CUSPARSE) {
    // tuning runs on device copies so the timed region below stays comparable
    spg_csr dA{}, dB{};
    if ((st = spg_csr_copy(ctx, &A, SPG_DEVICE, &dA)) != SPG_OK) return die(ctx, "copy", st);
    if ((st = spg_csr_copy(ctx, &B, SPG_DEVICE, &dB)) != SPG_OK) return die(ctx, "copy", st);
    spg_tuning t{};
    if ((st = spg_tune(ctx, 1, &dA, &dB, tune_cache.c_str(), &t)) != SPG_OK) return die(ctx, "spg_tune", st);
    spg_csr_free(ctx, &dA);
    spg_csr_free(ctx, &dB);
    o.use_tuning = 1;
  }
  // timed region: upload, product, C complete on the device
  spg_csr C{};
  spg_report rep{};
  const auto t0 = std::chrono::high_resolution_clock::now();
  st = spg_multiply(ctx, &A, &B, &C, &o, &rep);
  const auto t1 = std::chrono::high_resolution_clock::now();
  if (st != SPG_OK) return die(ctx, "spg_multiply", st);
  const double ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  spg_check_report chk{};
  if (check) {
    if ((st = spg_check(ctx, &A, &B, &C, &chk)) != SPG_OK) return die(ctx, "spg_check", st);
    std::fprintf(stderr,
                 "spgemm: check vs FP64: max |err| %.3e, mean |err| %.3e, max |err|/sum|a*b| %.3e, "
                 "%lld entries, %lld missing, %lld extra\n",
                 chk.max_abs_err_fp64, chk.mean_abs_err_fp64, chk.max_rel_err, (long long)chk.entries,
                 (long long)chk.missing, (long long)chk.extra);
  }
  if (!out.empty() && (st = spg_mtx_write(ctx, out.c_str(), &C, drop_zeros)) != SPG_OK)
    return die(ctx, ("writing " + out).c_str(), st);
  if (!log.empty()) {
    FILE* f = std::fopen(log.c_str(), "w");
    if (!f) {
      std::fprintf(stderr, "spgemm: cannot write %s\n", log.c_str());
      return 1;
    }
    std::fprintf(f, "%.6f\n", ms);
    std::fclose(f);
  }
  if (!json.empty()) {
    FILE* f = std::fopen(json.c_str(), "w");
    if (!f) return 1;
    static const char* names[SPG_STAGE_COUNT] = {"upload", "products", "binning", "symbolic", "scan",     "numeric",
                                                 "features", "mlp",    "fixup",   "compact",  "download", "other"};
    std::fprintf(f, "{\"ms_wall\": %.6f, \"ms_device\": %.6f, \"products\": %lld, \"gflops\": %.3f, "
                    "\"nnz_c\": %lld, \"rows_predicted\": %lld, \"rows_overflow\": %lld, \"rows_heavy\": %lld, "
                    "\"stages_ms\": {",
                 ms, rep.ms_total, (long long)rep.products,
                 rep.ms_total > 0 ? 2.0 * (double)rep.products / (rep.ms_total * 1e6) : 0.0, (long long)rep.nnz_c,
                 (long long)rep.rows_predicted, (long long)rep.rows_overflow, (long long)rep.rows_heavy);
    for (int s = 0; s < SPG_STAGE_COUNT; ++s)
      std::fprintf(f, "%s\"%s\": %.6f", s ? ", " : "", names[s], rep.ms_stage[s]);
    std::fprintf(f, "}");
    if (check)
      std::fprintf(f, ", \"check\": {\"max_abs_err_fp64\": %.6e, \"mean_abs_err_fp64\": %.6e, "
                      "\"max_rel_err\": %.6e, \"entries\": %lld, \"missing\": %lld, \"extra\": %lld}",
                   chk.max_abs_err_fp64, chk.mean_abs_err_fp64, chk.max_rel_err, (long long)chk.entries,
                   (long long)chk.missing, (long long)chk.extra);
    std::fprintf(f, "}\n");
    std::fclose(f);
  }
  spg_csr_free(ctx, &C);
  spg_csr_free(ctx, &A);
  spg_csr_free(ctx, &B);
  spg_destroy(ctx);
  return 0;
}
