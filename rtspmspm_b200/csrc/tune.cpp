// Autotuner: grid search over bin thresholds (largest warp table, its load
// factor, and the entries above which rows take a CTA-wide table), hash-table
// sizes and block shapes (warps per CTA), timed with CUDA events on the
// caller's products; a batch (n > 1) searches the load factor of its queue
// tables only, the one setting its persistent launches take.  No reference
// counterpart (the reference has fixed launch parameters: optixLaunch(nnzA,
// 1, 1), optixSpMSpM.cpp:607-608).
//
// The best setting is kept in the context and, with a cache path, stored in
// a small JSON file keyed by (shape class, GPU name):
//   {"entries": [{"gpu": "...", "shape": "...", "ms": t,
//                 "warp_table_max": .., "max_load": .., "warps_per_block": ..,
//                 "block_table_max": .., "block_min_nnz": .., "esc_min_prod": ..}, ...]}
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "context.hpp"

using namespace spg;

namespace {

// Shape class: log2 buckets of rows, nnz per row of A and B, and batch size.
std::string shape_class(int32_t n, const spg_csr* A, const spg_csr* B) {
  double rows = 0, annz = 0, bnnz = 0, brows = 0;
  for (int32_t m = 0; m < n; ++m) {
    rows += (double)A[m].rows;
    annz += (double)A[m].nnz;
    bnnz += (double)B[m].nnz;
    brows += (double)B[m].rows;
  }
  auto lb = [](double v) { return v <= 1 ? 0 : (int)std::lround(std::log2(v)); };
  char buf[96];
  std::snprintf(buf, sizeof buf, "n%d-r%d-a%d-b%d", lb((double)n), lb(rows / n), lb(annz / std::max(1.0, rows)),
                lb(bnnz / std::max(1.0, brows)));
  return buf;
}

std::string json_escape(const std::string& s) {
  std::string o;
  for (char c : s) {
    if (c == '"' || c == '\\') o.push_back('\\');
    o.push_back(c);
  }
  return o;
}

struct Entry {
  std::string gpu, shape;
  double ms = 0;
  spg_tuning t{};
};

// Minimal reader for the cache format written below (one entry per line).
std::vector<Entry> read_cache(const char* path) {
  std::vector<Entry> out;
  std::ifstream f(path);
  if (!f) return out;
  std::string line;
  while (std::getline(f, line)) {
    if (line.find("\"gpu\"") == std::string::npos) continue;
    Entry e;
    e.t = default_tuning();
    auto str = [&](const char* key) {
      const std::string k = std::string("\"") + key + "\": \"";
      size_t p = line.find(k);
      if (p == std::string::npos) return std::string();
      p += k.size();
      size_t q = line.find('"', p);
      return line.substr(p, q - p);
    };
    auto num = [&](const char* key, double dflt) {
      const std::string k = std::string("\"") + key + "\": ";
      size_t p = line.find(k);
      if (p == std::string::npos) return dflt;
      return std::atof(line.c_str() + p + k.size());
    };
    e.gpu = str("gpu");
    e.shape = str("shape");
    e.ms = num("ms", 0);
    e.t.warp_table_max = (int32_t)num("warp_table_max", e.t.warp_table_max);
    e.t.max_load = (float)num("max_load", e.t.max_load);
    e.t.warps_per_block = (int32_t)num("warps_per_block", e.t.warps_per_block);
    e.t.block_table_max = (int32_t)num("block_table_max", e.t.block_table_max);
    e.t.block_min_nnz = (int32_t)num("block_min_nnz", e.t.block_min_nnz);
    e.t.esc_min_prod = (int32_t)num("esc_min_prod", e.t.esc_min_prod);
    out.push_back(e);
  }
  return out;
}

bool write_cache(const char* path, const std::vector<Entry>& es) {
  std::ofstream f(path);
  if (!f) return false;
  f << "{\"entries\": [\n";
  for (size_t i = 0; i < es.size(); ++i) {
    const Entry& e = es[i];
    f << "  {\"gpu\": \"" << json_escape(e.gpu) << "\", \"shape\": \"" << json_escape(e.shape) << "\", \"ms\": " << e.ms
      << ", \"warp_table_max\": " << e.t.warp_table_max << ", \"max_load\": " << e.t.max_load
      << ", \"warps_per_block\": " << e.t.warps_per_block << ", \"block_table_max\": " << e.t.block_table_max
      << ", \"block_min_nnz\": " << e.t.block_min_nnz << ", \"esc_min_prod\": " << e.t.esc_min_prod << "}"
      << (i + 1 < es.size() ? ",\n" : "\n");
  }
  f << "]}\n";
  return (bool)f;
}

}  // namespace

extern "C" {

spg_status spg_get_tuning(spg_ctx* ctx, spg_tuning* out) {
  if (!ctx || !out) return SPG_ERR_INVALID_ARG;
  *out = ctx->tuning;
  return SPG_OK;
}

spg_status spg_set_tuning(spg_ctx* ctx, const spg_tuning* in) {
  if (!ctx || !in) return SPG_ERR_INVALID_ARG;
  spg_tuning t = *in;
  const spg_tuning d = default_tuning();
  if (t.warp_table_max < 32 || t.warp_table_max > 4096 || (t.warp_table_max & (t.warp_table_max - 1)))
    return fail(ctx, SPG_ERR_INVALID_ARG, "warp_table_max must be a power of two in [32, 4096]");
  if (!(t.max_load > 0.05f && t.max_load < 0.95f)) return fail(ctx, SPG_ERR_INVALID_ARG, "max_load out of range");
  if (t.warps_per_block < 0 || t.warps_per_block > 16)
    return fail(ctx, SPG_ERR_INVALID_ARG, "warps_per_block 0 (per kernel) or 1..16");
  if (t.block_table_max < 1024 || t.block_table_max > 32768 || (t.block_table_max & (t.block_table_max - 1)))
    return fail(ctx, SPG_ERR_INVALID_ARG, "block_table_max must be a power of two in [1024, 32768]");
  if (t.tile_cols == 0) t.tile_cols = d.tile_cols;
  if (t.predict_margin <= 0.f) t.predict_margin = d.predict_margin;
  if (t.predict_slack < 0) t.predict_slack = d.predict_slack;
  if (!(t.learned_load > 0.05f && t.learned_load < 0.95f)) t.learned_load = d.learned_load;
  if (t.heavy_path < 0 || t.heavy_path > 2) return fail(ctx, SPG_ERR_INVALID_ARG, "heavy_path must be 0, 1 or 2");
  if (t.block_min_nnz > (1 << kBlkLogLargeT) / 2)
    return fail(ctx, SPG_ERR_INVALID_ARG, "block_min_nnz above the largest CTA table (use -1 to turn the CTA bins off)");
  if (t.esc_min_prod < -1 || t.esc_min_prod > 1024)
    return fail(ctx, SPG_ERR_INVALID_ARG, "esc_min_prod must be -1 (off), 0 (default) or 1..1024");
  if (t.small_rows < -1 || t.small_rows > kSmallMaxRows)
    return fail(ctx, SPG_ERR_INVALID_ARG, "small_rows must be -1 (off), 0 (default) or 1..65536");
  ctx->tuning = t;
  return SPG_OK;
}

spg_status spg_tune(spg_ctx* ctx, int32_t n, const spg_csr* A, const spg_csr* B, const char* cache_path,
                    spg_tuning* best) {
  if (!ctx || n <= 0 || !A || !B) return SPG_ERR_INVALID_ARG;
  const std::string shape = shape_class(n, A, B);
  std::vector<Entry> cache = cache_path ? read_cache(cache_path) : std::vector<Entry>{};
  for (const Entry& e : cache) {
    if (e.gpu == ctx->gpu_name && e.shape == shape) {
      SPG_TRY(spg_set_tuning(ctx, &e.t));
      if (best) *best = ctx->tuning;
      return SPG_OK;
    }
  }
  const spg_tuning saved = ctx->tuning;
  spg_tuning win = saved;
  double win_ms = 1e30;
  // a batch's queue launches take the load factor only (their table sizes
  // and CTA shapes are fixed); a single product searches the whole grid
  const bool batch = n > 1;
  const std::vector<int> tables = batch ? std::vector<int>{4096} : std::vector<int>{1024, 2048, 4096};
  const std::vector<float> loads = batch ? std::vector<float>{0.5f, 0.65f, 0.8f}
                                         : std::vector<float>{0.35f, 0.5f, 0.65f};
  const std::vector<int> wpbs = batch ? std::vector<int>{0} : std::vector<int>{0, 4, 8, 16};
  const std::vector<int> block_mins = batch ? std::vector<int>{0} : std::vector<int>{0, 512};
  for (int wt : tables)
    for (float ld : loads)
      for (int wp : wpbs)
        for (int bm : block_mins) {
          spg_tuning t = default_tuning();
          t.warp_table_max = wt;
          t.max_load = ld;
          t.warps_per_block = wp;
          t.block_min_nnz = bm;
          t.predict_margin = saved.predict_margin;
          t.predict_slack = saved.predict_slack;
          t.learned_load = saved.learned_load;
          ctx->tuning = t;
          spg_opts o{};
          o.algo = SPG_ALGO_PLAIN;
          o.use_tuning = 1;
          o.use_graph = 1;
          o.skip_validation = 1;
          double trial[3];
          for (int rep = 0; rep < 3; ++rep) {
            spg_report r{};
            double ms = 0;
            if (n == 1) {
              spg_csr C{};
              spg_status st = spg_multiply(ctx, A, B, &C, &o, &r);
              spg_csr_free(ctx, &C);
              if (st != SPG_OK) {
                ctx->tuning = saved;
                return st;
              }
              ms = r.ms_total;
            } else {
              std::vector<spg_csr> C((size_t)n);
              spg_status st = spg_multiply_batched(ctx, n, A, B, C.data(), &o, &r);
              for (auto& c : C) spg_csr_free(ctx, &c);
              if (st != SPG_OK) {
                ctx->tuning = saved;
                return st;
              }
              ms = r.ms_total;
            }
            trial[rep] = ms;
          }
          std::sort(trial, trial + 3);
          if (trial[1] < win_ms) {
            win_ms = trial[1];
            win = t;
          }
        }
  ctx->tuning = win;
  if (best) *best = win;
  if (cache_path) {
    Entry e;
    e.gpu = ctx->gpu_name;
    e.shape = shape;
    e.ms = win_ms;
    e.t = win;
    cache.push_back(e);
    if (!write_cache(cache_path, cache)) return fail(ctx, SPG_ERR_IO, "cannot write %s", cache_path);
  }
  return SPG_OK;
}

}  // extern "C"
