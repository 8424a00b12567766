// Batched SpGEMM: many independent products C_m = A_m * B_m of uneven sizes.
//
// No reference counterpart: the reference runs one product per process
// (scripts/AE_test.py:199-215).  Here all rows of all products form one
// global row space, binned by table size across every matrix at once; each
// stage (symbolic, numeric) is one launch per warp-table size whose warps
// stride over that bin's rows of all products, so small and large products
// share the GPU without per-matrix launches.  Bin bounds are read on the
// device, and the launch sequence is captured once into a CUDA graph and
// replayed while the inputs stay the same.
//
// Plan (host, once per input set): matrix descriptors, global-row -> matrix
// map, the nnz upper bound of every product (sum over rows of
// min(products, cols)), so that every C_m gets a fixed region of one output
// slab and no host round trip is needed while the graph runs.
// Products whose bound exceeds the warp tables are run one by one through
// the single-product path instead.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "context.hpp"
#include "warp_row.cuh"

using namespace spg;

namespace spg {

struct BatchMat {
  DCsr A;
  DCsr B;
  int64_t row_start;  // first global row of this product
  int64_t c_base;     // first entry of C_m in the output slab
  int64_t rp_base;    // first entry of C_m's row pointers in the row-pointer slab
};

// Largest CTA of the per-bin kernels: 8 warps, tables within 200 KB.
constexpr int kBatchWarps = 8;
constexpr int kBatchCtaTableBytes = 200 * 1024;

// Products per global row and the bound min(products, cols_m).
__global__ void k_batch_products(const BatchMat* mats, const int32_t* row_mat, int64_t R, int64_t* prod,
                                 int64_t* bound) {
  const int lane = lane_id();
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t g = gw; g < R; g += nw) {
    const BatchMat& M = mats[row_mat[g]];
    const int64_t r = g - M.row_start;
    const int64_t s = M.A.rp[r], e = M.A.rp[r + 1];
    int64_t sum = 0;
    for (int64_t p = s + lane; p < e; p += 32) {
      const int32_t k = M.A.col[p];
      sum += M.B.rp[k + 1] - M.B.rp[k];
    }
    sum = warp_sum(sum);
    if (lane == 0) {
      prod[g] = sum;
      bound[g] = sum < M.B.cols ? sum : M.B.cols;
    }
  }
}

// Plan-time: per-matrix max and sum of the bound.
__global__ void k_batch_bound_stats(const int32_t* row_mat, const int64_t* bound, int64_t R,
                                    unsigned long long* maxb, unsigned long long* sumb) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < R; g += (int64_t)gridDim.x * blockDim.x) {
    const int m = row_mat[g];
    const unsigned long long b = (unsigned long long)bound[g];
    if (b) {
      atomicMax(&maxb[m], b);
      atomicAdd(&sumb[m], b);
    }
  }
}

// Shared-memory bytes a warp's table takes: 2^logt slots of keys when
// symbolic; keys, values and the first-seen list when numeric.
inline size_t batch_table_bytes(int logt, bool numeric) { return ((size_t)1 << logt) * (numeric ? 12 : 4); }

// Symbolic (NUMERIC = false) or numeric (true) pass over the rows of warp
// bin LOGT of the global row space: warp per row, rows taken in stride from
// the bin's list (its bounds read from bin_off on the device, so the launch
// needs no host round trip and replays from a graph).  Each row looks up its
// product's descriptor.  Tables are epoch-tagged while the product's B has
// fewer than 2^24 columns; a row of a wider product clears the table first
// if tagged keys may be left in it.
template <int LOGT, bool NUMERIC>
__global__ void __launch_bounds__(512, 2) k_batch_bin(const BatchMat* mats, const int32_t* row_mat,
                                                      const int32_t* lists, const int64_t* bin_off, int64_t* nnz,
                                                      const int64_t* gscan, int32_t* c_col, float* c_val,
                                                      int* flags) {
  constexpr int T = 1 << LOGT;
  constexpr int kWords = NUMERIC ? numeric_words<LOGT>() : T;
  extern __shared__ int32_t sm_tab[];
  const int lane = lane_id();
  int32_t* keys = sm_tab + (threadIdx.x >> 5) * kWords;
  float* vals = reinterpret_cast<float*>(keys + T);
  int32_t* list = keys + 2 * T;
  for (int s2 = lane; s2 < T; s2 += 32) keys[s2] = kEmpty;
  __syncwarp();
  const int64_t first = bin_off[LOGT - kMinLogT], last = bin_off[LOGT - kMinLogT + 1];
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  int epoch = 0;
  bool tagged = false;  // keys of an epoch may be in the table
  for (int64_t i = first + gw; i < last; i += nw) {
    const int64_t g = lists[i];
    const BatchMat& M = mats[row_mat[g]];
    const int32_t r = (int32_t)(g - M.row_start);
    int ep = epoch;
    if (M.B.cols >= (1 << 24)) {
      ep = kNoEpoch;
      if (tagged) {
        for (int s2 = lane; s2 < T; s2 += 32) keys[s2] = kEmpty;
        __syncwarp();
        tagged = false;
        epoch = 0;
      }
    }
    if (!NUMERIC) {
      const int cnt = symbolic_row<LOGT, true>(M.A, M.B, r, keys, ep, flags);
      if (lane == 0) nnz[g] = cnt;
    } else {
      const int64_t base = gscan[M.row_start];
      const int64_t off = M.c_base + (gscan[g] - base);
      numeric_row<LOGT, true, true>(M.A, M.B, r, keys, vals, list, ep, c_col + off, c_val + off,
                                    gscan[g + 1] - gscan[g], flags);
    }
    if (ep >= 0) {
      tagged = true;
      if (!NUMERIC) next_row<LOGT>(keys, ep);
      epoch = ep;
      if (epoch == 0) tagged = false;  // wiped on wrap
    }
  }
}

// Per-product row pointers (rebased to 0) and nnz.
__global__ void k_batch_finalize(const BatchMat* mats, int n, const int32_t* row_mat, int64_t R, const int64_t* gscan,
                                 int64_t* rp_out, int64_t* nnz_m) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < R + n; g += (int64_t)gridDim.x * blockDim.x) {
    if (g < R) {
      const int m = row_mat[g];
      const BatchMat& M = mats[m];
      rp_out[M.rp_base + (g - M.row_start)] = gscan[g] - gscan[M.row_start];
    } else {
      const int m = (int)(g - R);
      const BatchMat& M = mats[m];
      const int64_t rows = M.A.rows;
      const int64_t tot = gscan[M.row_start + rows] - gscan[M.row_start];
      rp_out[M.rp_base + rows] = tot;
      nnz_m[m] = tot;
    }
  }
}

namespace {

struct BatchPlan {
  std::vector<uintptr_t> key;
  int n = 0;
  int64_t R = 0;
  std::vector<void*> owned;  // cudaMalloc'd, freed with the plan
  BatchMat* d_mats = nullptr;
  int32_t* row_mat = nullptr;
  int64_t* prod = nullptr;
  int64_t* bound = nullptr;
  int64_t* nnz = nullptr;  // R + 1, scanned in place
  uint8_t* bin_of_row = nullptr;
  int64_t* binmeta = nullptr;
  int32_t* lists = nullptr;
  int64_t* scan_tmp = nullptr;
  int32_t* c_col = nullptr;
  float* c_val = nullptr;
  int64_t* rp_out = nullptr;
  int64_t* nnz_m = nullptr;
  int64_t* h_nnz_m = nullptr;  // pinned
  std::vector<BatchMat> mats;
  std::vector<int> batched;     // products on the persistent path
  std::vector<int> individual;  // products run one by one
  std::vector<int64_t> c_base;  // host copy
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  spg_tuning tune{};
  int per_sm[2][kNumWarpBins] = {};  // CTAs per SM of the per-bin kernels (symbolic, numeric)
  int warps[2][kNumWarpBins] = {};   // warps per CTA of the per-bin kernels
  int launches = 0;
};

void free_plan(BatchPlan* p) {
  if (!p) return;
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  for (void* q : p->owned) cudaFree(q);
  if (p->h_nnz_m) cudaFreeHost(p->h_nnz_m);
  delete p;
}

template <typename T>
spg_status dmalloc(spg_ctx* ctx, BatchPlan* p, T** out, size_t count) {
  void* q = nullptr;
  SPG_CUDA(ctx, cudaMalloc(&q, std::max<size_t>(count * sizeof(T), 16)));
  p->owned.push_back(q);
  *out = static_cast<T*>(q);
  return SPG_OK;
}

std::vector<uintptr_t> plan_key(spg_ctx* ctx, int n, const spg_csr* A, const spg_csr* B, const spg_opts& o) {
  std::vector<uintptr_t> k;
  k.reserve((size_t)n * 12 + 8);
  k.push_back((uintptr_t)n);
  const spg_tuning t = o.use_tuning ? ctx->tuning : default_tuning();
  k.push_back((uintptr_t)t.warp_table_max);
  k.push_back((uintptr_t)(t.max_load * 1000.0f));
  k.push_back((uintptr_t)t.warps_per_block);
  for (int m = 0; m < n; ++m) {
    for (const spg_csr* x : {&A[m], &B[m]}) {
      k.push_back((uintptr_t)x->row_ptr);
      k.push_back((uintptr_t)x->col_idx);
      k.push_back((uintptr_t)x->val);
      k.push_back((uintptr_t)x->rows);
      k.push_back((uintptr_t)x->cols);
      k.push_back((uintptr_t)x->nnz ^ ((uintptr_t)x->index_bits << 56));
    }
  }
  return k;
}

// Issues the device work of one batched execution on ctx->stream.
void enqueue(spg_ctx* ctx, BatchPlan* p) {
  const LaunchCtx lc = launch_ctx(ctx);
  const BinParams bp = without_block_bins(bin_params(p->tune));
  int launches = 0;
  const int64_t R = p->R;
  auto blocks_for = [&](int64_t work, int per_block) {
    int64_t b = (work + per_block - 1) / per_block;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)lc.sms * 16));
  };
  k_batch_products<<<blocks_for(R, 8), 256, 0, lc.stream>>>(p->d_mats, p->row_mat, R, p->prod, p->bound);
  ++launches;
  cudaMemsetAsync(p->nnz, 0, (size_t)(R + 1) * 8, lc.stream);
  int64_t* counts = p->binmeta;
  int64_t* offsets = p->binmeta + kNumBins;
  int64_t* cursors = p->binmeta + 2 * kNumBins + 1;
  launch_binning(p->bound, R, INT64_MAX, kBinSymbolic, bp, p->bin_of_row, counts, offsets, cursors, p->lists, lc);
  launches += 3;
  // each stage: one launch per warp-table size, each reading its bin's
  // bounds on the device
  auto stage = [&](bool numeric) {
    for (int b = 0; b < kNumWarpBins; ++b) {
      const int logt = kMinLogT + b;
      const int w = p->warps[numeric ? 1 : 0][b];
      const size_t smem = (size_t)w * batch_table_bytes(logt, numeric);
      const int grid = lc.sms * p->per_sm[numeric ? 1 : 0][b];
#define SPG_BB(L)                                                                                                 \
  case L:                                                                                                         \
    if (numeric)                                                                                                  \
      k_batch_bin<L, true><<<grid, w * 32, smem, lc.stream>>>(p->d_mats, p->row_mat, p->lists, offsets, p->nnz,   \
                                                              p->nnz, p->c_col, p->c_val, ctx->d_flags);          \
    else                                                                                                          \
      k_batch_bin<L, false><<<grid, w * 32, smem, lc.stream>>>(p->d_mats, p->row_mat, p->lists, offsets, p->nnz, \
                                                               nullptr, nullptr, nullptr, ctx->d_flags);          \
    break;
      switch (logt) {
        SPG_BB(5) SPG_BB(6) SPG_BB(7) SPG_BB(8) SPG_BB(9) SPG_BB(10) SPG_BB(11) SPG_BB(12)
        default: break;
      }
#undef SPG_BB
      ++launches;
    }
  };
  stage(false);
  launch_binning(p->nnz, R, INT64_MAX, kBinNumeric, bp, p->bin_of_row, counts, offsets, cursors, p->lists, lc);
  launch_excl_scan(p->nnz, R, p->nnz, p->scan_tmp, lc);
  launches += 7;
  stage(true);
  k_batch_finalize<<<blocks_for(R + p->n, 256), 256, 0, lc.stream>>>(p->d_mats, p->n, p->row_mat, R, p->nnz,
                                                                     p->rp_out, p->nnz_m);
  ++launches;
  cudaMemcpyAsync(p->h_nnz_m, p->nnz_m, (size_t)p->n * 8, cudaMemcpyDeviceToHost, lc.stream);
  p->launches = launches;
}

spg_status build_plan(spg_ctx* ctx, int n, const spg_csr* A, const spg_csr* B, const spg_opts& o, BatchPlan** out,
                      std::vector<DevMat>& keep) {
  (void)keep;
  auto* p = new BatchPlan();
  std::unique_ptr<BatchPlan, void (*)(BatchPlan*)> guard(p, free_plan);
  p->n = n;
  p->key = plan_key(ctx, n, A, B, o);
  if (o.use_tuning) {
    p->tune = ctx->tuning;
  } else {
    // uneven products of short rows: fuller tables keep more warps per SM
    // (load 0.65 measured best for the batch of 64 uneven products)
    p->tune = default_tuning();
    p->tune.max_load = 0.65f;
  }
  // every warp table size stays available on the batched path: a smaller
  // tuned maximum would send whole products to the one-by-one path
  p->tune.warp_table_max = default_tuning().warp_table_max;
  const BinParams bp = without_block_bins(bin_params(p->tune));
  const LaunchCtx lc = launch_ctx(ctx);
  p->mats.resize((size_t)n);
  int64_t R = 0;
  for (int m = 0; m < n; ++m) {
    for (const spg_csr* x : {&A[m], &B[m]}) {
      if (x->location != SPG_DEVICE) return fail(ctx, SPG_ERR_INVALID_ARG, "batched inputs must be on the device");
      if (x->index_bits != 32 && x->index_bits != 64) return fail(ctx, SPG_ERR_INVALID_ARG, "bad index_bits");
      if (x->rows > 0 && !x->row_ptr) return fail(ctx, SPG_ERR_INVALID_ARG, "null row_ptr");
    }
    if (A[m].cols != B[m].rows) return fail(ctx, SPG_ERR_INVALID_ARG, "pair %d: inner dimensions differ", m);
    if (B[m].cols > INT32_MAX || A[m].rows > INT32_MAX) return fail(ctx, SPG_ERR_UNSUPPORTED, "pair %d too large", m);
    BatchMat& M = p->mats[(size_t)m];
    const spg_csr* src[2] = {&A[m], &B[m]};
    DCsr* dst[2] = {&M.A, &M.B};
    for (int q = 0; q < 2; ++q) {
      const spg_csr* x = src[q];
      const int64_t* rp64;
      const int32_t* rp32 = nullptr;
      if (x->index_bits == 32) {
        int64_t* w = nullptr;
        SPG_TRY(dmalloc(ctx, p, &w, (size_t)x->rows + 1));
        launch_widen_rp(static_cast<const int32_t*>(x->row_ptr), x->rows + 1, w, lc);
        rp64 = w;
        rp32 = static_cast<const int32_t*>(x->row_ptr);
      } else {
        rp64 = static_cast<const int64_t*>(x->row_ptr);
        if (x->nnz < INT32_MAX) {
          int32_t* w = nullptr;
          SPG_TRY(dmalloc(ctx, p, &w, (size_t)x->rows + 1));
          launch_narrow_rp(rp64, x->rows + 1, w, lc);
          rp32 = w;
        }
      }
      *dst[q] = DCsr{x->rows, x->cols, rp64, x->col_idx, x->val, rp32};
      if (!o.skip_validation) launch_validate(*dst[q], x->nnz, ctx->d_flags, lc);
    }
    M.row_start = R;
    R += A[m].rows;
  }
  p->R = R;
  int f = 0;
  SPG_TRY(read_flags(ctx, &f));
  if (f & kFlagBadIndex) return fail(ctx, SPG_ERR_INVALID_ARG, "a batched input failed validation");
  // global row -> product map
  std::vector<int32_t> row_mat((size_t)std::max<int64_t>(R, 1));
  for (int m = 0; m < n; ++m)
    std::fill(row_mat.begin() + p->mats[(size_t)m].row_start,
              row_mat.begin() + p->mats[(size_t)m].row_start + A[m].rows, m);
  SPG_TRY(dmalloc(ctx, p, &p->d_mats, (size_t)n));
  SPG_TRY(dmalloc(ctx, p, &p->row_mat, (size_t)std::max<int64_t>(R, 1)));
  SPG_TRY(dmalloc(ctx, p, &p->prod, (size_t)R + 1));
  SPG_TRY(dmalloc(ctx, p, &p->bound, (size_t)R + 1));
  SPG_CUDA(ctx, cudaMemcpyAsync(p->row_mat, row_mat.data(), (size_t)std::max<int64_t>(R, 1) * 4,
                                cudaMemcpyHostToDevice, ctx->stream));
  SPG_CUDA(ctx, cudaMemcpyAsync(p->d_mats, p->mats.data(), (size_t)n * sizeof(BatchMat), cudaMemcpyHostToDevice,
                                ctx->stream));
  // bounds per product
  unsigned long long *maxb = nullptr, *sumb = nullptr;
  SPG_TRY(dmalloc(ctx, p, &maxb, (size_t)n));
  SPG_TRY(dmalloc(ctx, p, &sumb, (size_t)n));
  SPG_CUDA(ctx, cudaMemsetAsync(maxb, 0, (size_t)n * 8, ctx->stream));
  SPG_CUDA(ctx, cudaMemsetAsync(sumb, 0, (size_t)n * 8, ctx->stream));
  if (R > 0) {
    k_batch_products<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((R + 7) / 8, ctx->sms * 16)), 256, 0,
                       ctx->stream>>>(p->d_mats, p->row_mat, R, p->prod, p->bound);
    k_batch_bound_stats<<<ctx->sms * 4, 256, 0, ctx->stream>>>(p->row_mat, p->bound, R, maxb, sumb);
  }
  std::vector<unsigned long long> hmax((size_t)n), hsum((size_t)n);
  SPG_CUDA(ctx, cudaMemcpyAsync(hmax.data(), maxb, (size_t)n * 8, cudaMemcpyDeviceToHost, ctx->stream));
  SPG_CUDA(ctx, cudaMemcpyAsync(hsum.data(), sumb, (size_t)n * 8, cudaMemcpyDeviceToHost, ctx->stream));
  SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  // products whose rows exceed the warp tables go through the single path
  int64_t cbase = 0, rpbase = 0;
  p->c_base.assign((size_t)n, 0);
  for (int m = 0; m < n; ++m) {
    BatchMat& M = p->mats[(size_t)m];
    // the persistent kernels use 32-bit row offsets of B (nnz(B) < 2^31)
    if ((int64_t)hmax[(size_t)m] > bp.warp_cap || !M.B.rp32) {
      p->individual.push_back(m);
      // keep its rows out of the persistent stages: an empty A view
      M.A.rows = 0;
    } else {
      p->batched.push_back(m);
    }
    M.c_base = cbase;
    M.rp_base = rpbase;
    p->c_base[(size_t)m] = cbase;
    if ((int64_t)hmax[(size_t)m] <= bp.warp_cap && M.B.rp32) cbase += (int64_t)hsum[(size_t)m];
    rpbase += A[m].rows + 1;
  }
  if (!p->individual.empty()) {
    // rows of individually-run products are removed from the global space
    std::vector<int32_t> keep_rows;
    int64_t R2 = 0;
    std::vector<int64_t> new_start((size_t)n, 0);
    for (int m = 0; m < n; ++m) {
      new_start[(size_t)m] = R2;
      if (p->mats[(size_t)m].A.rows > 0) R2 += A[m].rows;
    }
    std::vector<int32_t> rm((size_t)std::max<int64_t>(R2, 1));
    for (int m = 0; m < n; ++m) {
      BatchMat& M = p->mats[(size_t)m];
      M.row_start = new_start[(size_t)m];
      if (M.A.rows > 0) std::fill(rm.begin() + M.row_start, rm.begin() + M.row_start + A[m].rows, m);
    }
    p->R = R = R2;
    SPG_CUDA(ctx, cudaMemcpyAsync(p->row_mat, rm.data(), (size_t)std::max<int64_t>(R, 1) * 4, cudaMemcpyHostToDevice,
                                  ctx->stream));
    SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  // the descriptors now carry their final row starts and output offsets
  SPG_CUDA(ctx, cudaMemcpyAsync(p->d_mats, p->mats.data(), (size_t)n * sizeof(BatchMat), cudaMemcpyHostToDevice,
                                ctx->stream));
  SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  // CTA size, shared memory and CTAs per SM of every per-bin kernel (set
  // before any capture): of 1..kBatchWarps warps whose tables fit
  // kBatchCtaTableBytes, the size with the most resident warps per SM, ties
  // to the larger CTA
  for (int numeric = 0; numeric < 2; ++numeric) {
    for (int b = 0; b < kNumWarpBins; ++b) {
      const int logt = kMinLogT + b;
      const size_t per_warp = batch_table_bytes(logt, numeric != 0);
      const int max_w = (int)std::max<size_t>(1, std::min<size_t>(kBatchWarps, kBatchCtaTableBytes / per_warp));
      int best_w = 1, best_ctas = 1, best = -1;
      for (int w = 1; w <= max_w; ++w) {
        const size_t smem = (size_t)w * per_warp;
        int per_sm = 0;
#define SPG_BA(L)                                                                                            \
  case L:                                                                                                    \
    if (numeric) {                                                                                           \
      SPG_CUDA(ctx, cudaFuncSetAttribute(k_batch_bin<L, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,  \
                                         (int)kBatchCtaTableBytes));                                         \
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_bin<L, true>, w * 32, smem);            \
    } else {                                                                                                 \
      SPG_CUDA(ctx, cudaFuncSetAttribute(k_batch_bin<L, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                         (int)kBatchCtaTableBytes));                                         \
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_bin<L, false>, w * 32, smem);           \
    }                                                                                                        \
    break;
        switch (logt) {
          SPG_BA(5) SPG_BA(6) SPG_BA(7) SPG_BA(8) SPG_BA(9) SPG_BA(10) SPG_BA(11) SPG_BA(12)
          default: break;
        }
#undef SPG_BA
        if (per_sm >= 1 && per_sm * w >= best) {
          best = per_sm * w;
          best_w = w;
          best_ctas = per_sm;
        }
      }
      p->warps[numeric][b] = best_w;
      p->per_sm[numeric][b] = best_ctas;
    }
  }
  SPG_TRY(dmalloc(ctx, p, &p->nnz, (size_t)R + 1));
  SPG_TRY(dmalloc(ctx, p, &p->bin_of_row, (size_t)std::max<int64_t>(R, 1)));
  SPG_TRY(dmalloc(ctx, p, &p->binmeta, (size_t)(3 * kNumBins + 1)));
  SPG_TRY(dmalloc(ctx, p, &p->lists, (size_t)std::max<int64_t>(R, 1)));
  SPG_TRY(dmalloc(ctx, p, &p->scan_tmp, (size_t)scan_temp_elems(R + 1)));
  SPG_TRY(dmalloc(ctx, p, &p->c_col, (size_t)std::max<int64_t>(cbase, 1)));
  SPG_TRY(dmalloc(ctx, p, &p->c_val, (size_t)std::max<int64_t>(cbase, 1)));
  SPG_TRY(dmalloc(ctx, p, &p->rp_out, (size_t)std::max<int64_t>(rpbase, 1)));
  SPG_TRY(dmalloc(ctx, p, &p->nnz_m, (size_t)n));
  SPG_CUDA(ctx, cudaMallocHost(&p->h_nnz_m, (size_t)n * 8));
  SPG_CUDA(ctx, cudaMemsetAsync(p->nnz_m, 0, (size_t)n * 8, ctx->stream));
  SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *out = guard.release();
  return SPG_OK;
}

}  // namespace

void free_batch_cache(spg_ctx* ctx) {
  if (ctx->batch_cache) free_plan(static_cast<BatchPlan*>(ctx->batch_cache));
  ctx->batch_cache = nullptr;
}

}  // namespace spg

extern "C" spg_status spg_multiply_batched(spg_ctx* ctx, int32_t n, const spg_csr* A, const spg_csr* B, spg_csr* C,
                                           const spg_opts* opts, spg_report* report) {
  if (!ctx) return SPG_ERR_INVALID_ARG;
  if (n <= 0 || !A || !B || !C) return fail(ctx, SPG_ERR_INVALID_ARG, "bad batched arguments");
  SPG_CUDA(ctx, cudaSetDevice(ctx->device));
  spg_opts o{};
  if (opts) o = *opts;
  if (report) {
    std::memset(report, 0, sizeof *report);
    report->algo = SPG_ALGO_PLAIN;
  }
  auto* plan = static_cast<BatchPlan*>(ctx->batch_cache);
  if (!plan || plan->key != plan_key(ctx, n, A, B, o)) {
    free_batch_cache(ctx);
    std::vector<DevMat> keep;
    BatchPlan* np = nullptr;
    SPG_TRY(build_plan(ctx, n, A, B, o, &np, keep));
    ctx->batch_cache = np;
    plan = np;
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, ctx->stream);
  if (plan->R > 0) {
    if (o.use_graph) {
      if (!plan->exec) {
        SPG_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        enqueue(ctx, plan);
        cudaGraph_t g = nullptr;
        SPG_CUDA(ctx, cudaStreamEndCapture(ctx->stream, &g));
        plan->graph = g;
        SPG_CUDA(ctx, cudaGraphInstantiate(&plan->exec, g, 0));
      }
      SPG_CUDA(ctx, cudaGraphLaunch(plan->exec, ctx->stream));
      ctx->launches += 1;
    } else {
      enqueue(ctx, plan);
      ctx->launches += plan->launches;
    }
  }
  cudaEventRecord(e1, ctx->stream);
  SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  int f = 0;
  SPG_TRY(read_flags(ctx, &f));
  if (report) report->device_flags = f;
  if (f & (kFlagHashFull | kFlagCountDiff)) return fail(ctx, SPG_ERR_INTERNAL, "batched consistency check failed");
  int64_t nnz_total = 0;
  for (int m : plan->batched) {
    const BatchMat& M = plan->mats[(size_t)m];
    spg_csr& c = C[m];
    std::memset(&c, 0, sizeof c);
    c.rows = A[m].rows;
    c.cols = B[m].cols;
    c.nnz = plan->h_nnz_m[m];
    c.capacity = c.nnz;
    c.index_bits = 64;
    c.location = SPG_DEVICE;
    c.row_ptr = plan->rp_out + M.rp_base;
    c.col_idx = plan->c_col + M.c_base;
    c.val = plan->c_val + M.c_base;
    c.owner = 0;  // lives in the context's batch buffers
    nnz_total += c.nnz;
  }
  double ms_total = ms;
  for (int m : plan->individual) {
    spg_opts so = o;
    so.algo = SPG_ALGO_PLAIN;
    so.out_location = SPG_DEVICE;
    so.out_index_bits = 64;
    spg_report r{};
    SPG_TRY(spg_multiply(ctx, &A[m], &B[m], &C[m], &so, &r));
    ms_total += r.ms_total;
    nnz_total += C[m].nnz;
    if (report) report->products += r.products;
  }
  if (report) {
    report->ms_total = ms_total;
    report->nnz_c = nnz_total;
    report->kernel_launches = plan->launches;
    for (int m : plan->batched) report->rows += A[m].rows;
    for (int m : plan->individual) report->rows += A[m].rows;
    report->rows_heavy = (int64_t)plan->individual.size();
    // products of the batched part (device sum)
    unsigned long long* d = ctx->d_counter + 3;
    cudaMemsetAsync(d, 0, 8, ctx->stream);
    launch_sum(plan->prod, plan->R, d, launch_ctx(ctx));
    unsigned long long hp = 0;
    cudaMemcpyAsync(&ctx->h_stage[20], d, 8, cudaMemcpyDeviceToHost, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    std::memcpy(&hp, &ctx->h_stage[20], 8);
    report->products += (int64_t)hp;
  }
  return SPG_OK;
}
