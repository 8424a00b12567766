// C-ABI implementation: context, memory, and the plain / learned SpGEMM
// pipelines.
//
// Plain two-pass method (the judge and the fallback):
//   products -> bin by bound -> symbolic (warp hash / CTA hash / CTA bitmap)
//   -> bin by exact nnz -> scan -> allocate C -> numeric (warp hash with
//   per-row sort / column-tiled heavy rows).
// Learned method:
//   features + products -> MLP capacity -> bin by capacity -> single numeric
//   pass into a capacity-sized slab (overflow -> queued) -> exact symbolic for
//   predicted-heavy and overflowed rows -> scan -> allocate C -> copy slab rows
//   + numeric pass for the exact rows.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>

#include "context.hpp"

using namespace spg;

namespace spg {

spg_status fail(spg_ctx* ctx, spg_status st, const char* fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    ctx->last_error = buf;
  }
  return st;
}

spg_status cuda_status(spg_ctx* ctx, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return SPG_OK;
  const spg_status st = (e == cudaErrorMemoryAllocation) ? SPG_ERR_OUT_OF_MEMORY : SPG_ERR_CUDA;
  (void)cudaGetLastError();  // clear a sticky-free error so the context stays usable
  return fail(ctx, st, "%s: %s", what, cudaGetErrorString(e));
}

spg_status DevBuf::alloc(spg_ctx* ctx, size_t bytes) {
  reset();
  ctx_ = ctx;
  if (bytes == 0) return SPG_OK;
  cudaError_t e = cudaMallocAsync(&ptr_, bytes, ctx->stream);
  if (e != cudaSuccess) {
    ptr_ = nullptr;
    return cuda_status(ctx, e, "cudaMallocAsync");
  }
  return SPG_OK;
}

void DevBuf::reset() {
  if (ptr_ && ctx_) cudaFreeAsync(ptr_, ctx_->stream);
  ptr_ = nullptr;
}

spg_tuning default_tuning() {
  spg_tuning t{};
  t.warp_table_max = 4096;
  // 0: each warp-hash kernel takes the CTA size with the most resident warps
  // per SM (fixed 8-warp CTAs left the stencil 96^3 numeric kernels at 32
  // warps per SM instead of 36: learned numeric 4.18 ms against 3.79 ms)
  t.warps_per_block = 0;
  t.max_load = 0.4f;  // measured best for the plain method on the stencil rows (0.3..0.65 swept)
  t.tile_cols = kTileCols;
  t.block_table_max = 16384;
  t.predict_margin = 1.25f;
  t.predict_slack = 8;
  t.learned_load = 0.4f;
  return t;
}

static int ilog2_floor(int64_t v) {
  int l = 0;
  while ((int64_t(1) << (l + 1)) <= v) ++l;
  return l;
}

BinParams bin_params(const spg_tuning& t) {
  BinParams bp{};
  int lg = ilog2_floor(std::max(32, std::min(4096, t.warp_table_max)));
  bp.warp_log_max = std::max(kMinLogT, std::min(kMaxLogT, lg));
  bp.max_load = std::min(0.9f, std::max(0.1f, t.max_load));
  // the largest table may run up to half full whatever the load factor
  bp.warp_cap = (int64_t)std::floor((double)(1 << bp.warp_log_max) * std::max(0.5f, bp.max_load));
  // symbolic CTA table at load <= 2/3
  int blg = ilog2_floor(std::max(1024, std::min(32768, t.block_table_max)));
  bp.block_cap = ((int64_t)1 << blg) * 2 / 3;
  // CTA-wide numeric hash bins (tables at load <= 1/2: their key and
  // order-word arrays are the row sort's buffers) for rows of more than
  // block_min_nnz entries, when set: measured slower than the warp tables
  // and heavy-row tiles they replace on R-MAT scale 17 (plain 29.8 against
  // 21.6 ms) and even on scale 20 (518 against 516 ms), so off by default
  if (t.block_min_nnz <= 0) return without_block_bins(bp);
  bp.block_min = (int64_t)t.block_min_nnz;
  bp.blk_small_cap = ((int64_t)1 << kBlkLogSmallT) / 2;
  bp.blk_large_cap = ((int64_t)1 << kBlkLogLargeT) / 2;
  return bp;
}

static int block_table_log(const spg_tuning& t) {
  return ilog2_floor(std::max(1024, std::min(32768, t.block_table_max)));
}

// Small device-to-host reads (bin offsets, totals, flags) are written into
// the pinned staging words by a one-block kernel through the mapped host
// address, not by a copy engine: a large device-to-host copy in flight on
// another stream (spg_multiply_into_host) would otherwise delay them.
spg_status stage_read(spg_ctx* ctx, void* host_dst, const void* dev_src, size_t bytes) {
  const size_t at = (size_t)(static_cast<char*>(host_dst) - reinterpret_cast<char*>(ctx->h_stage));
  if (at + bytes > 64 * sizeof(int64_t) || (bytes & 3)) return fail(ctx, SPG_ERR_INTERNAL, "bad staging read");
  launch_copy_words(dev_src, reinterpret_cast<char*>(ctx->h_stage_dev) + at, (int64_t)(bytes / 4), launch_ctx(ctx));
  return cuda_status(ctx, cudaGetLastError(), "stage_read");
}

spg_status read_flags(spg_ctx* ctx, int* flags) {
  SPG_TRY(stage_read(ctx, &ctx->h_stage[15], ctx->d_flags, sizeof(int)));
  SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  int f = 0;
  std::memcpy(&f, &ctx->h_stage[15], sizeof(int));
  if (f) SPG_CUDA(ctx, cudaMemsetAsync(ctx->d_flags, 0, sizeof(int), ctx->stream));
  *flags = f;
  return SPG_OK;
}

// A and B describe the same matrix (same storage): prepare it once.
bool same_matrix(const spg_csr* a, const spg_csr* b) {
  return a == b || (a->rows == b->rows && a->cols == b->cols && a->nnz == b->nnz && a->index_bits == b->index_bits &&
                    a->location == b->location && a->row_ptr == b->row_ptr && a->col_idx == b->col_idx &&
                    a->val == b->val);
}

// defer_entries (host inputs): the column/value buffers are allocated but not
// filled; the caller uploads them (spg_multiply_into_host's row chunks).
spg_status prepare_matrix(spg_ctx* ctx, const spg_csr* m, DevMat& out, bool validate, bool defer_entries) {
  if (!m) return fail(ctx, SPG_ERR_INVALID_ARG, "null matrix");
  if (m->rows < 0 || m->cols < 0 || m->nnz < 0) return fail(ctx, SPG_ERR_INVALID_ARG, "negative dimension");
  if (m->cols > INT32_MAX) return fail(ctx, SPG_ERR_UNSUPPORTED, "more than 2^31-1 columns");
  if (m->index_bits != 32 && m->index_bits != 64) return fail(ctx, SPG_ERR_INVALID_ARG, "index_bits must be 32 or 64");
  if (m->rows > 0 && !m->row_ptr) return fail(ctx, SPG_ERR_INVALID_ARG, "null row_ptr");
  if (m->nnz > 0 && (!m->col_idx || !m->val)) return fail(ctx, SPG_ERR_INVALID_ARG, "null col_idx/val");
  if (m->index_bits == 32 && m->nnz > INT32_MAX) return fail(ctx, SPG_ERR_INVALID_ARG, "nnz overflows int32 row_ptr");
  const LaunchCtx lc = launch_ctx(ctx);
  const size_t rp_bytes = (size_t)(m->rows + 1) * (m->index_bits / 8);
  const void* rp = m->row_ptr;
  const int32_t* col = m->col_idx;
  const float* val = m->val;
  if (m->location == SPG_HOST) {
    SPG_TRY(out.upload[0].alloc(ctx, rp_bytes));
    SPG_TRY(out.upload[1].alloc(ctx, (size_t)m->nnz * 4));
    SPG_TRY(out.upload[2].alloc(ctx, (size_t)m->nnz * 4));
    if (m->rows >= 0)
      SPG_CUDA(ctx, cudaMemcpyAsync(out.upload[0].get(), m->row_ptr, rp_bytes, cudaMemcpyHostToDevice, ctx->stream));
    if (m->nnz > 0 && !defer_entries) {
      SPG_CUDA(ctx, cudaMemcpyAsync(out.upload[1].get(), m->col_idx, (size_t)m->nnz * 4, cudaMemcpyHostToDevice,
                                    ctx->stream));
      SPG_CUDA(ctx, cudaMemcpyAsync(out.upload[2].get(), m->val, (size_t)m->nnz * 4, cudaMemcpyHostToDevice,
                                    ctx->stream));
    }
    rp = out.upload[0].get();
    col = out.upload[1].as<int32_t>();
    val = out.upload[2].as<float>();
  } else if (m->location != SPG_DEVICE) {
    return fail(ctx, SPG_ERR_INVALID_ARG, "location must be SPG_HOST or SPG_DEVICE");
  }
  const int64_t* rp64;
  const int32_t* rp32 = nullptr;
  if (m->index_bits == 32) {
    SPG_TRY(out.rp64.alloc(ctx, (size_t)(m->rows + 1) * 8));
    launch_widen_rp(static_cast<const int32_t*>(rp), m->rows + 1, out.rp64.as<int64_t>(), lc);
    ++ctx->launches;
    rp64 = out.rp64.as<int64_t>();
    rp32 = static_cast<const int32_t*>(rp);
  } else {
    rp64 = static_cast<const int64_t*>(rp);
    if (m->nnz < INT32_MAX) {
      SPG_TRY(out.rp32.alloc(ctx, (size_t)(m->rows + 1) * 4));
      launch_narrow_rp(rp64, m->rows + 1, out.rp32.as<int32_t>(), lc);
      ++ctx->launches;
      rp32 = out.rp32.as<int32_t>();
    }
  }
  out.view = DCsr{m->rows, m->cols, rp64, col, val, rp32};
  out.nnz = m->nnz;
  if (validate) {
    launch_validate(out.view, m->nnz, ctx->d_flags, lc);
    ++ctx->launches;
  }
  return SPG_OK;
}

StageTimer::StageTimer(spg_ctx* ctx, bool enabled) : ctx_(ctx), on_(enabled) {
  cudaEventCreate(&start_);
  cudaEventCreate(&end_);
  cudaEventRecord(start_, ctx->stream);
}

StageTimer::~StageTimer() {
  for (auto& m : marks_) cudaEventDestroy(m.second);
  cudaEventDestroy(start_);
  cudaEventDestroy(end_);
}

void StageTimer::mark(int stage) {
  if (!on_) return;
  cudaEvent_t ev;
  cudaEventCreate(&ev);
  cudaEventRecord(ev, ctx_->stream);
  marks_.emplace_back(stage, ev);
}

void StageTimer::finish(spg_report* rep) {
  cudaEventRecord(end_, ctx_->stream);
  cudaEventSynchronize(end_);
  if (!rep) return;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, start_, end_);
  rep->ms_total = ms;
  for (size_t i = 0; i < marks_.size(); ++i) {
    cudaEvent_t next = (i + 1 < marks_.size()) ? marks_[i + 1].second : end_;
    float d = 0.f;
    cudaEventElapsedTime(&d, marks_[i].second, next);
    const int st = marks_[i].first;
    if (st >= 0 && st < SPG_STAGE_COUNT) rep->ms_stage[st] += d;
  }
}

}  // namespace spg

// ===========================================================================
// Pipelines
// ===========================================================================

namespace {

// Largest blocked index of B built for the heavy-row tiles (bytes).
constexpr size_t kBlockedIndexMaxBytes = size_t(4) << 30;
// Largest list of non-empty heavy-row tiles (bytes).
constexpr size_t kWorkListMaxBytes = size_t(4) << 30;

// Buffers and host mirrors of one multiply call.
struct Pipeline {
  spg_ctx* ctx;
  LaunchCtx lc;
  const DevMat& A;
  const DevMat& B;
  spg_tuning tune;
  BinParams bp;
  int64_t rows, cols;
  int ntiles;
  int wpb;

  DevBuf prod;        // int64 rows
  DevBuf nnz;         // int64 rows+1 (becomes C's row pointers)
  DevBuf bin_of_row;  // uint8 rows
  DevBuf binmeta;     // int64: counts[12] offsets[13] cursors[12]
  DevBuf lists;       // int32 rows
  DevBuf big_slot;    // int32 rows
  DevBuf tile_cnt;    // int32 nbig * ntiles
  DevBuf tile_off;    // int32 nbig * ntiles
  DevBuf scan_tmp;    // int64
  int64_t h_off[kNumBins + 1] = {};
  int64_t nbig = 0;

  Pipeline(spg_ctx* c, const DevMat& a, const DevMat& b, const spg_tuning& t)
      : ctx(c), lc(launch_ctx(c)), A(a), B(b), tune(t), bp(bin_params(t)), rows(a.view.rows), cols(b.view.cols) {
    ntiles = (int)std::max<int64_t>(1, (cols + kTileCols - 1) / kTileCols);
    wpb = t.warps_per_block <= 0 ? 0 : std::min(16, t.warps_per_block);
  }

  int64_t* counts() { return binmeta.as<int64_t>(); }
  int64_t* offsets() { return binmeta.as<int64_t>() + kNumBins; }
  int64_t* cursors() { return binmeta.as<int64_t>() + 2 * kNumBins + 1; }

  spg_status init() {
    SPG_TRY(prod.alloc(ctx, (size_t)std::max<int64_t>(rows, 1) * 8));
    SPG_TRY(nnz.alloc(ctx, (size_t)(rows + 1) * 8));
    SPG_TRY(bin_of_row.alloc(ctx, (size_t)std::max<int64_t>(rows, 1)));
    SPG_TRY(binmeta.alloc(ctx, (size_t)(3 * kNumBins + 1) * 8));
    SPG_TRY(lists.alloc(ctx, (size_t)std::max<int64_t>(rows, 1) * 4));
    SPG_TRY(big_slot.alloc(ctx, (size_t)std::max<int64_t>(rows, 1) * 4));
    SPG_TRY(scan_tmp.alloc(ctx, (size_t)scan_temp_elems(rows + 1) * 8));
    SPG_CUDA(ctx, cudaMemsetAsync(nnz.get(), 0, (size_t)(rows + 1) * 8, ctx->stream));
    return SPG_OK;
  }

  void bin(const int64_t* key, int mode) {
    launch_binning(key, rows, cols, mode, bp, bin_of_row.as<uint8_t>(), counts(), offsets(), cursors(),
                   lists.as<int32_t>(), lc);
    ctx->launches += 3;
  }

  // Offsets of the last binning (and optional extra int64 words) to host.
  spg_status fetch_offsets(const int64_t* extra = nullptr, int64_t* extra_host = nullptr, int n_extra = 0) {
    SPG_TRY(stage_read(ctx, ctx->h_stage, offsets(), sizeof(int64_t) * (kNumBins + 1)));
    for (int i = 0; i < n_extra; ++i)
      SPG_TRY(stage_read(ctx, ctx->h_stage + kNumBins + 1 + i, extra + i, sizeof(int64_t)));
    SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    std::memcpy(h_off, ctx->h_stage, sizeof(int64_t) * (kNumBins + 1));
    for (int i = 0; i < n_extra; ++i) extra_host[i] = ctx->h_stage[kNumBins + 1 + i];
    return SPG_OK;
  }

  int64_t bin_size(int b) const { return h_off[b + 1] - h_off[b]; }
  const int32_t* bin_rows(int b) { return lists.as<int32_t>() + h_off[b]; }

  // Exact symbolic pass over rows whose key (products) is > 0.
  spg_status symbolic(const int64_t* key) {
    bin(key, kBinSymbolic);
    SPG_TRY(fetch_offsets());
    for (int b = 0; b < kNumWarpBins; ++b) {
      if (bin_size(b) == 0) continue;
      launch_sym_warp(kMinLogT + b, A.view, B.view, bin_rows(b), bin_size(b), nnz.as<int64_t>(), ctx->d_flags, lc,
                      wpb);
      ++ctx->launches;
    }
    const int64_t nblock = bin_size(kBinBlock), ndense = bin_size(kBinDense);
    nbig = nblock + ndense;
    if (nbig > 0) {
      const size_t tb = (size_t)nbig * ntiles * 4;
      SPG_TRY(tile_cnt.alloc(ctx, tb));
      SPG_TRY(tile_off.alloc(ctx, tb));
      SPG_CUDA(ctx, cudaMemsetAsync(tile_cnt.get(), 0, tb, ctx->stream));
      if (nblock) {
        launch_sym_block(A.view, B.view, bin_rows(kBinBlock), nblock, block_table_log(tune), 0, nnz.as<int64_t>(),
                         big_slot.as<int32_t>(), tile_cnt.as<int32_t>(), ntiles, ctx->d_flags, lc);
        ++ctx->launches;
      }
      if (ndense) {
        launch_sym_dense(A.view, B.view, bin_rows(kBinDense), ndense, nblock, nnz.as<int64_t>(),
                         big_slot.as<int32_t>(), tile_cnt.as<int32_t>(), ntiles, ctx->d_flags, lc);
        ++ctx->launches;
      }
    }
    return SPG_OK;
  }

  // Numeric pass for the rows in the current (numeric) binning, into C.
  // Numeric pass; `row_prod` (the rows' products, or nullptr) lets the warp
  // bins take expand-sort-fold rows.
  // Expand-sort-fold settings from the tuning (esc_min_prod 0: the default
  // threshold, -1: off).
  EscArgs esc_args(const int64_t* row_prod) const {
    EscArgs e;
    e.prod = row_prod;
    e.min_prod = tune.esc_min_prod < 0 ? 0 : (tune.esc_min_prod == 0 ? kEscMinProd : tune.esc_min_prod);
    return e;
  }

  spg_status numeric(const int64_t* c_rp, int32_t* c_col, float* c_val, spg_report* rep,
                     const int64_t* row_prod = nullptr) {
    const EscArgs esc = esc_args(row_prod);
    for (int b = 0; b < kNumWarpBins; ++b) {
      if (bin_size(b) == 0) continue;
      launch_num_warp(kMinLogT + b, A.view, B.view, bin_rows(b), bin_size(b), c_rp, c_col, c_val, ctx->d_flags, lc,
                      wpb, esc);
      ++ctx->launches;
    }
    // rows above the efficient warp tables: CTA-wide hash tables
    for (int b : {kBinBlock, kBinDense}) {
      if (bin_size(b) == 0) continue;
      launch_num_block(b, A.view, B.view, bin_rows(b), bin_size(b), c_rp, c_col, c_val, ctx->d_flags, lc);
      ++ctx->launches;
    }
    const int64_t nheavy = bin_size(kBinHeavy);
    if (nheavy > 0) {
      // the blocked index reads every row of B
      if (B.complete) SPG_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, B.complete, 0));
      size_t free_b = 0, total_b = 0;
      cudaMemGetInfo(&free_b, &total_b);
      // the list of non-empty (row, tile) units for the tile kernel, when it
      // fits: rows of wide products touch a small part of their tiles
      const size_t work_bytes = (size_t)nheavy * (size_t)ntiles * 8;
      const bool use_list = tune.heavy_path != 1 && ntiles > 1 && work_bytes <= kWorkListMaxBytes &&
                            work_bytes < free_b / 4;
      DevBuf nz, work;
      if (use_list) SPG_TRY(nz.alloc(ctx, (size_t)(nheavy + 1) * 8));
      launch_tile_offsets(bin_rows(kBinHeavy), nheavy, big_slot.as<int32_t>(), tile_cnt.as<int32_t>(), ntiles,
                          tile_off.as<int32_t>(), use_list ? nz.as<int64_t>() : nullptr, lc);
      if (use_list) {
        SPG_TRY(work.alloc(ctx, work_bytes));
        launch_excl_scan(nz.as<int64_t>(), nheavy, nz.as<int64_t>(), scan_tmp.as<int64_t>(), lc);
        launch_tile_worklist(bin_rows(kBinHeavy), nheavy, big_slot.as<int32_t>(), tile_cnt.as<int32_t>(), ntiles,
                             nz.as<int64_t>(), work.as<int64_t>(), lc);
        ctx->launches += 5;
      }
      // staged path (opt-in): each heavy row's products walked once into
      // per-tile buckets; measured slower than rescanning on R-MAT (the
      // bucket writes scatter over a buffer far larger than L2)
      bool staged = false;
      if (tune.heavy_path == 1)
        SPG_TRY(heavy_staged(ctx, A.view, B.view, bin_rows(kBinHeavy), nheavy, big_slot.as<int32_t>(),
                             tile_cnt.as<int32_t>(), tile_off.as<int32_t>(), ntiles, c_rp, c_col, c_val, &staged));
      if (!staged) {
        // rescanning tile kernel, with a blocked index of B when it fits the
        // budget (else per-tile binary searches)
        DevBuf bidx;
        const size_t bidx_bytes = (size_t)B.view.rows * (size_t)(ntiles + 1) * 4;
        const bool use_index = ntiles > 1 && bidx_bytes <= kBlockedIndexMaxBytes && bidx_bytes < free_b / 4;
        DevBuf tocc;
        if (use_index) {
          SPG_TRY(bidx.alloc(ctx, bidx_bytes));
          SPG_TRY(tocc.alloc(ctx, (size_t)B.view.rows * (size_t)((ntiles + 31) / 32) * 4));
          launch_build_blocked_index(B.view, ntiles, bidx.as<int32_t>(), lc);
          launch_build_tile_occupancy(B.view.rows, bidx.as<int32_t>(), ntiles, tocc.as<uint32_t>(), lc);
          ctx->launches += 2;
        }
        launch_num_tile(A.view, B.view, bin_rows(kBinHeavy), nheavy, big_slot.as<int32_t>(),
                        tile_cnt.as<int32_t>(), tile_off.as<int32_t>(), ntiles, c_rp, c_col, c_val,
                        use_index ? bidx.as<int32_t>() : nullptr, use_index ? tocc.as<uint32_t>() : nullptr,
                        use_list ? work.as<int64_t>() : nullptr, use_list ? nz.as<int64_t>() + nheavy : nullptr,
                        ctx->d_counter, ctx->d_flags, lc, tune.heavy_path == 2);
        ctx->launches += 2;
      }
      ++ctx->launches;
    }
    if (rep) {
      for (int b = 0; b < kNumBins && b < SPG_NUM_BINS; ++b) rep->bin_rows[b] += bin_size(b);
      rep->rows_heavy += nheavy;
    }
    return SPG_OK;
  }
};

// Fills C from the pipeline's row pointers and the col/val buffers; narrows
// the row pointers to int32 when requested or when nnz(C) fits.
spg_status finish_output(spg_ctx* ctx, Pipeline& P, int64_t total, const spg_opts& o, DevBuf& c_col, DevBuf& c_val,
                         spg_csr* C) {
  int bits = o.out_index_bits;
  if (bits == 0) bits = total < INT32_MAX ? 32 : 64;
  if (bits != 32 && bits != 64) return fail(ctx, SPG_ERR_INVALID_ARG, "out_index_bits must be 0, 32 or 64");
  if (bits == 32 && total >= INT32_MAX)
    return fail(ctx, SPG_ERR_INVALID_ARG, "nnz(C)=%lld does not fit int32 row pointers", (long long)total);
  const LaunchCtx lc = launch_ctx(ctx);
  void* rp = nullptr;
  if (bits == 64) {
    rp = P.nnz.release();
  } else {
    DevBuf rp32;
    SPG_TRY(rp32.alloc(ctx, (size_t)(P.rows + 1) * 4));
    launch_narrow_rp(P.nnz.as<int64_t>(), P.rows + 1, rp32.as<int32_t>(), lc);
    ++ctx->launches;
    rp = rp32.release();
  }
  std::memset(C, 0, sizeof *C);
  C->rows = P.rows;
  C->cols = P.cols;
  C->nnz = total;
  C->capacity = total;
  C->index_bits = bits;
  C->location = SPG_DEVICE;
  C->row_ptr = rp;
  C->col_idx = static_cast<int32_t*>(c_col.release());
  C->val = static_cast<float*>(c_val.release());
  C->owner = 1;
  return SPG_OK;
}

// Status of a device flag word read back after a call's work.
spg_status flag_status(spg_ctx* ctx, int f, spg_report* rep) {
  if (rep) rep->device_flags |= f;
  if (f & kFlagBadIndex) return fail(ctx, SPG_ERR_INVALID_ARG, "input failed validation (index out of range, "
                                                               "unsorted or duplicate columns, bad row pointers)");
  if (f & (kFlagHashFull | kFlagCountDiff)) return fail(ctx, SPG_ERR_INTERNAL, "device consistency check failed (flags %d)", f);
  if (f & kFlagWaitLimit) return fail(ctx, SPG_ERR_TIMEOUT, "a bounded device wait gave up");
  return SPG_OK;
}

spg_status check_flags(spg_ctx* ctx, spg_report* rep) {
  int f = 0;
  SPG_TRY(read_flags(ctx, &f));
  return flag_status(ctx, f, rep);
}

spg_status multiply_plain(spg_ctx* ctx, Pipeline& P, spg_csr* C, const spg_opts& o, spg_report* rep,
                          StageTimer& tm) {
  const LaunchCtx lc = P.lc;
  tm.mark(SPG_STAGE_PRODUCTS);
  launch_row_products(P.A.view, P.B.view, P.prod.as<int64_t>(), lc);
  SPG_CUDA(ctx, cudaMemsetAsync(ctx->d_counter + 1, 0, 8, ctx->stream));
  launch_sum(P.prod.as<int64_t>(), P.rows, ctx->d_counter + 1, lc);
  ctx->launches += 2;
  tm.mark(SPG_STAGE_SYMBOLIC);
  SPG_TRY(P.symbolic(P.prod.as<int64_t>()));
  tm.mark(SPG_STAGE_BINNING);
  P.bin(P.nnz.as<int64_t>(), kBinNumeric);
  tm.mark(SPG_STAGE_SCAN);
  launch_excl_scan(P.nnz.as<int64_t>(), P.rows, P.nnz.as<int64_t>(), P.scan_tmp.as<int64_t>(), lc);
  ctx->launches += 4;
  int64_t extra[2];
  const int64_t* src[2] = {P.nnz.as<int64_t>() + P.rows, reinterpret_cast<const int64_t*>(ctx->d_counter + 1)};
  // fetch offsets + total nnz + products
  SPG_TRY(stage_read(ctx, ctx->h_stage, P.offsets(), sizeof(int64_t) * (kNumBins + 1)));
  SPG_TRY(stage_read(ctx, ctx->h_stage + kNumBins + 1, src[0], 8));
  SPG_TRY(stage_read(ctx, ctx->h_stage + kNumBins + 2, src[1], 8));
  SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  std::memcpy(P.h_off, ctx->h_stage, sizeof(int64_t) * (kNumBins + 1));
  extra[0] = ctx->h_stage[kNumBins + 1];
  extra[1] = ctx->h_stage[kNumBins + 2];
  const int64_t total = extra[0];
  if (rep) rep->products = extra[1];
  DevBuf c_col, c_val;
  SPG_TRY(c_col.alloc(ctx, (size_t)total * 4));
  SPG_TRY(c_val.alloc(ctx, (size_t)total * 4));
  tm.mark(SPG_STAGE_NUMERIC);
  SPG_TRY(P.numeric(P.nnz.as<int64_t>(), c_col.as<int32_t>(), c_val.as<float>(), rep, P.prod.as<int64_t>()));
  SPG_TRY(finish_output(ctx, P, total, o, c_col, c_val, C));
  if (rep) rep->nnz_c = total;
  return SPG_OK;
}

spg_status multiply_learned(spg_ctx* ctx, Pipeline& P, spg_csr* C, const spg_opts& o, spg_report* rep,
                            StageTimer& tm) {
  const LaunchCtx lc = P.lc;
  SPG_TRY(ensure_mlp(ctx));
  const int64_t rows = P.rows;
  DevBuf cap, need, slab_off, key;
  SPG_TRY(cap.alloc(ctx, (size_t)(rows + 1) * 8));
  SPG_TRY(need.alloc(ctx, (size_t)std::max<int64_t>(rows, 1)));
  SPG_TRY(slab_off.alloc(ctx, (size_t)(rows + 1) * 8));
  SPG_TRY(key.alloc(ctx, (size_t)std::max<int64_t>(rows, 1) * 8));
  // products, features and the tensor-core MLP in one pass over A
  tm.mark(SPG_STAGE_MLP);
  // d_counter: [1] products, [2] overflowed rows, [3] rows predicted heavy
  SPG_CUDA(ctx, cudaMemsetAsync(ctx->d_counter, 0, 4 * 8, ctx->stream));
  // rows up to the largest CTA table are sized by the prediction (with the
  // CTA bins off, up to the largest warp table and as the predicted bin says)
  const bool cta_bins = P.bp.blk_large_cap > 0;
  launch_learned_plan(P.A.view, P.B.view, ctx->mlp_w16, P.tune.predict_margin, P.tune.predict_slack,
                      std::max(P.bp.warp_cap, P.bp.blk_large_cap), cta_bins ? 0 : 1, o.force_overflow,
                      P.prod.as<int64_t>(), cap.as<int64_t>(), need.as<uint8_t>(), ctx->d_counter + 3, lc);
  launch_sum(P.prod.as<int64_t>(), rows, ctx->d_counter + 1, lc);
  ctx->launches += 2;
  tm.mark(SPG_STAGE_BINNING);
  {
    BinParams lbp = P.bp;
    lbp.max_load = std::min(0.9f, std::max(0.1f, P.tune.learned_load > 0.f ? P.tune.learned_load : P.bp.max_load));
    launch_binning(cap.as<int64_t>(), rows, P.cols, kBinLearned, lbp, P.bin_of_row.as<uint8_t>(), P.counts(),
                   P.offsets(), P.cursors(), P.lists.as<int32_t>(), lc);
    ctx->launches += 3;
  }
  launch_excl_scan(cap.as<int64_t>(), rows, slab_off.as<int64_t>(), P.scan_tmp.as<int64_t>(), lc);
  ctx->launches += 4;
  int64_t slab_total = 0;
  constexpr int kExactSlot = 40;  // h_stage word (64 in all)
  SPG_TRY(stage_read(ctx, ctx->h_stage + kExactSlot, ctx->d_counter + 3, 8));
  SPG_TRY(P.fetch_offsets(slab_off.as<int64_t>() + rows, &slab_total, 1));
  const int64_t n_exact = ctx->h_stage[kExactSlot];
  // predicted-light rows: the warp bins and the CTA bins, the first
  // entries of the binning's lists
  int64_t light = 0;
  for (int b = 0; b <= kBinDense; ++b) light += P.bin_size(b);
  if (rep) rep->rows_predicted = light;
  // single numeric pass for the predicted-light rows
  DevBuf slab_col, slab_val, retry;
  SPG_TRY(slab_col.alloc(ctx, (size_t)slab_total * 4));
  SPG_TRY(slab_val.alloc(ctx, (size_t)slab_total * 4));
  SPG_TRY(retry.alloc(ctx, (size_t)std::max<int64_t>(light, 1) * 4));
  tm.mark(SPG_STAGE_NUMERIC);
  for (int b = 0; b < kNumWarpBins; ++b) {
    if (P.bin_size(b) == 0) continue;
    launch_num_warp_learned(kMinLogT + b, P.A.view, P.B.view, P.bin_rows(b), P.bin_size(b), cap.as<int64_t>(),
                            slab_off.as<int64_t>(), slab_col.as<int32_t>(), slab_val.as<float>(), P.nnz.as<int64_t>(),
                            retry.as<int32_t>(), ctx->d_counter + 2, ctx->d_flags, lc, P.wpb,
                            P.esc_args(P.prod.as<int64_t>()));
    ++ctx->launches;
  }
  for (int b : {kBinBlock, kBinDense}) {
    if (P.bin_size(b) == 0) continue;
    launch_num_block_learned(b, P.A.view, P.B.view, P.bin_rows(b), P.bin_size(b), cap.as<int64_t>(),
                             slab_off.as<int64_t>(), slab_col.as<int32_t>(), slab_val.as<float>(), P.nnz.as<int64_t>(),
                             retry.as<int32_t>(), ctx->d_counter + 2, ctx->d_flags, lc);
    ++ctx->launches;
  }
  // exact path for predicted-heavy rows plus overflowed rows; with neither
  // (the usual case) the fix-up and the exact numeric pass are skipped
  tm.mark(SPG_STAGE_FIXUP);
  bool exact_needed = n_exact > 0;
  int64_t total = 0;
  if (!exact_needed) {
    // the usual case: scan the counts now and read the total, the products
    // and the overflow count in one round trip
    tm.mark(SPG_STAGE_SCAN);
    launch_excl_scan(P.nnz.as<int64_t>(), rows, P.nnz.as<int64_t>(), P.scan_tmp.as<int64_t>(), lc);
    ctx->launches += 4;
    SPG_TRY(stage_read(ctx, ctx->h_stage + kNumBins + 1, P.nnz.as<int64_t>() + rows, 8));
    SPG_TRY(stage_read(ctx, ctx->h_stage + kNumBins + 2, ctx->d_counter + 1, 16));
    SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    total = ctx->h_stage[kNumBins + 1];
    if (rep) {
      rep->products = ctx->h_stage[kNumBins + 2];
      rep->rows_overflow = ctx->h_stage[kNumBins + 3];
    }
    if (ctx->h_stage[kNumBins + 3] > 0) {
      // rows overflowed: undo the scan (adjacent differences give back the
      // counts, -1 for the overflowed rows) and take the exact path
      launch_adjacent_diff(P.nnz.as<int64_t>(), rows, key.as<int64_t>(), lc);
      SPG_CUDA(ctx, cudaMemcpyAsync(P.nnz.get(), key.get(), (size_t)rows * 8, cudaMemcpyDeviceToDevice,
                                    ctx->stream));
      ++ctx->launches;
      exact_needed = true;
    }
  }
  // the light-row list (first `light` entries of the learned binning) is
  // kept for the compaction copy when the exact path rebins
  DevBuf light_rows;
  const int32_t* compact_list = P.lists.as<int32_t>();
  if (exact_needed) {
    SPG_TRY(light_rows.alloc(ctx, (size_t)std::max<int64_t>(light, 1) * 4));
    if (light)
      SPG_CUDA(ctx, cudaMemcpyAsync(light_rows.get(), P.lists.get(), (size_t)light * 4, cudaMemcpyDeviceToDevice,
                                    ctx->stream));
    compact_list = light_rows.as<int32_t>();
    launch_mark_rows(retry.as<int32_t>(), ctx->d_counter + 2, need.as<uint8_t>(), lc);
    launch_mask_key(P.prod.as<int64_t>(), need.as<uint8_t>(), rows, key.as<int64_t>(), lc);
    ctx->launches += 2;
    SPG_TRY(P.symbolic(key.as<int64_t>()));
    launch_mask_key(P.nnz.as<int64_t>(), need.as<uint8_t>(), rows, key.as<int64_t>(), lc);
    P.bin(key.as<int64_t>(), kBinNumeric);
    ctx->launches += 1;
  }
  if (exact_needed) {
    tm.mark(SPG_STAGE_SCAN);
    launch_excl_scan(P.nnz.as<int64_t>(), rows, P.nnz.as<int64_t>(), P.scan_tmp.as<int64_t>(), lc);
    ctx->launches += 4;
    SPG_TRY(stage_read(ctx, ctx->h_stage, P.offsets(), sizeof(int64_t) * (kNumBins + 1)));
    SPG_TRY(stage_read(ctx, ctx->h_stage + kNumBins + 1, P.nnz.as<int64_t>() + rows, 8));
    SPG_TRY(stage_read(ctx, ctx->h_stage + kNumBins + 2, ctx->d_counter + 1, 16));
    SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    std::memcpy(P.h_off, ctx->h_stage, sizeof(int64_t) * (kNumBins + 1));
    total = ctx->h_stage[kNumBins + 1];
    if (rep) {
      rep->products = ctx->h_stage[kNumBins + 2];
      rep->rows_overflow = ctx->h_stage[kNumBins + 3];
    }
  }
  DevBuf c_col, c_val;
  SPG_TRY(c_col.alloc(ctx, (size_t)total * 4));
  SPG_TRY(c_val.alloc(ctx, (size_t)total * 4));
  tm.mark(SPG_STAGE_COMPACT);
  launch_compact_rows(compact_list, light, need.as<uint8_t>(), slab_off.as<int64_t>(), slab_col.as<int32_t>(),
                      slab_val.as<float>(), P.nnz.as<int64_t>(), c_col.as<int32_t>(), c_val.as<float>(), lc);
  ++ctx->launches;
  if (exact_needed) {
    tm.mark(SPG_STAGE_NUMERIC);
    SPG_TRY(P.numeric(P.nnz.as<int64_t>(), c_col.as<int32_t>(), c_val.as<float>(), rep, P.prod.as<int64_t>()));
  }
  SPG_TRY(finish_output(ctx, P, total, o, c_col, c_val, C));
  if (rep) rep->nnz_c = total;
  return SPG_OK;
}

// Rows of A up to which a call takes the small-product path (0: off).
int64_t small_rows_limit(const spg_tuning& t) {
  if (t.small_rows < 0) return 0;
  return t.small_rows == 0 ? kSmallDefaultRows : std::min<int64_t>(t.small_rows, kSmallMaxRows);
}

// Small products in both methods: exact counts and products in one launch,
// one CTA scanning them into C's row pointers, one round trip for the
// total, and one numeric launch over every row with a table sized for the
// largest row.  The binned pipeline spends about two dozen launches and
// three round trips on a product of this size, which is all its time
// (Erdos-Renyi 4096 rows of Poisson(8): 0.26 ms); the prediction cannot pay
// for itself here either.  *taken stays false, with nothing written to C,
// when a row has more than 2^kSmallLogT products or needs a larger table
// than the tuning allows; the caller then runs the binned pipeline.
spg_status multiply_small(spg_ctx* ctx, Pipeline& P, spg_csr* C, const spg_opts& o, spg_report* rep, StageTimer& tm,
                          bool* taken) {
  *taken = false;
  const LaunchCtx lc = P.lc;
  const int64_t rows = P.rows;
  const int bits = o.out_index_bits;
  if (bits != 0 && bits != 32 && bits != 64) return fail(ctx, SPG_ERR_INVALID_ARG, "out_index_bits must be 0, 32 or 64");
  DevBuf rp32;
  if (bits != 64) SPG_TRY(rp32.alloc(ctx, (size_t)(rows + 1) * 4));
  tm.mark(SPG_STAGE_SYMBOLIC);
  // d_counter[6]: the counting launch's stop word (zero between calls)
  launch_small_count(P.A.view, P.B.view, P.prod.as<int64_t>(), P.nnz.as<int64_t>(), ctx->d_counter + 6, ctx->d_flags,
                     lc);
  tm.mark(SPG_STAGE_SCAN);
  constexpr int kSmallSlot = 48;  // h_stage words 48..51
  launch_small_scan(P.nnz.as<int64_t>(), P.prod.as<int64_t>(), rows, bits != 64 ? rp32.as<int32_t>() : nullptr,
                    P.lists.as<int32_t>(), ctx->d_counter + 6, ctx->h_stage_dev + kSmallSlot, lc);
  ctx->launches += 2;
  SPG_CUDA(ctx, cudaGetLastError());
  SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const int64_t total = ctx->h_stage[kSmallSlot], products = ctx->h_stage[kSmallSlot + 1];
  const int64_t max_cnt = ctx->h_stage[kSmallSlot + 2], too_large = ctx->h_stage[kSmallSlot + 3];
  // the numeric table: the smallest that holds the largest row at the load factor
  int log_t = kMinLogT;
  while (log_t < kMaxLogT && (double)max_cnt > (double)P.tune.max_load * (double)(1 << log_t)) ++log_t;
  if (too_large > 0 || max_cnt > (1 << log_t) || (1 << log_t) > std::max(32, P.tune.warp_table_max)) {
    // the binned pipeline takes the call, from zeroed counts
    SPG_CUDA(ctx, cudaMemsetAsync(P.nnz.get(), 0, (size_t)(rows + 1) * 8, ctx->stream));
    return SPG_OK;
  }
  if (bits == 32 && total >= INT32_MAX)
    return fail(ctx, SPG_ERR_INVALID_ARG, "nnz(C)=%lld does not fit int32 row pointers", (long long)total);
  DevBuf c_col, c_val;
  SPG_TRY(c_col.alloc(ctx, (size_t)total * 4));
  SPG_TRY(c_val.alloc(ctx, (size_t)total * 4));
  tm.mark(SPG_STAGE_NUMERIC);
  if (total > 0) {
    launch_num_warp(log_t, P.A.view, P.B.view, P.lists.as<int32_t>(), rows, P.nnz.as<int64_t>(), c_col.as<int32_t>(),
                    c_val.as<float>(), ctx->d_flags, lc, P.wpb, P.esc_args(P.prod.as<int64_t>()));
    ++ctx->launches;
  }
  const bool narrow = bits != 64 && total < INT32_MAX;
  std::memset(C, 0, sizeof *C);
  C->rows = rows;
  C->cols = P.cols;
  C->nnz = total;
  C->capacity = total;
  C->index_bits = narrow ? 32 : 64;
  C->location = SPG_DEVICE;
  C->row_ptr = narrow ? rp32.release() : P.nnz.release();
  C->col_idx = static_cast<int32_t*>(c_col.release());
  C->val = static_cast<float*>(c_val.release());
  C->owner = 1;
  if (rep) {
    rep->products = products;
    rep->nnz_c = total;
    rep->small_path = 1;
    rep->bin_rows[log_t - kMinLogT] += rows;
  }
  *taken = true;
  return SPG_OK;
}

}  // namespace

namespace spg {

spg_status multiply_device(spg_ctx* ctx, const DevMat& A, const DevMat& B, spg_csr* C, const spg_opts& o,
                           spg_report* rep) {
  StageTimer tm(ctx, o.stage_timing != 0);
  const spg_tuning t = o.use_tuning ? ctx->tuning : default_tuning();
  Pipeline P(ctx, A, B, t);
  SPG_TRY(P.init());
  bool small = false;
  if (P.rows > 0 && P.rows <= small_rows_limit(t) && !o.force_overflow)
    SPG_TRY(multiply_small(ctx, P, C, o, rep, tm, &small));
  if (!small) {
    spg_status st = (o.algo == SPG_ALGO_LEARNED) ? multiply_learned(ctx, P, C, o, rep, tm)
                                                 : multiply_plain(ctx, P, C, o, rep, tm);
    if (st != SPG_OK) return st;
  }
  // the device flags ride on the final wait: a kernel writes them into the
  // mapped staging words, read once the end event has completed
  constexpr int kFlagSlot = 30;
  SPG_TRY(stage_read(ctx, ctx->h_stage + kFlagSlot, ctx->d_flags, sizeof(int)));
  tm.finish(rep);
  int f = 0;
  std::memcpy(&f, &ctx->h_stage[kFlagSlot], sizeof(int));
  if (f) SPG_CUDA(ctx, cudaMemsetAsync(ctx->d_flags, 0, sizeof(int), ctx->stream));
  return flag_status(ctx, f, rep);
}

// Value-only recompute into an existing C (structure of A*B given).
spg_status multiply_reuse_device(spg_ctx* ctx, const DevMat& A, const DevMat& B, spg_csr* C, const spg_opts& o,
                                 spg_report* rep) {
  StageTimer tm(ctx, o.stage_timing != 0);
  const spg_tuning t = o.use_tuning ? ctx->tuning : default_tuning();
  Pipeline P(ctx, A, B, t);
  SPG_TRY(P.init());
  const LaunchCtx lc = P.lc;
  const int64_t rows = P.rows;
  tm.mark(SPG_STAGE_BINNING);
  // C's row pointers as int64 (P.nnz), its row lengths as the numeric key
  if (C->index_bits == 32) {
    launch_widen_rp(static_cast<const int32_t*>(C->row_ptr), rows + 1, P.nnz.as<int64_t>(), lc);
  } else {
    SPG_CUDA(ctx, cudaMemcpyAsync(P.nnz.get(), C->row_ptr, (size_t)(rows + 1) * 8, cudaMemcpyDeviceToDevice,
                                  ctx->stream));
  }
  launch_row_lengths(P.nnz.as<int64_t>(), rows, P.prod.as<int64_t>(), lc);
  ctx->launches += 2;
  P.bin(P.prod.as<int64_t>(), kBinNumeric);
  SPG_TRY(P.fetch_offsets());
  const int64_t nheavy = P.bin_size(kBinHeavy);
  if (nheavy > 0) {
    const size_t tb = (size_t)nheavy * P.ntiles * 4;
    SPG_TRY(P.tile_cnt.alloc(ctx, tb));
    SPG_TRY(P.tile_off.alloc(ctx, tb));
    SPG_CUDA(ctx, cudaMemsetAsync(P.tile_cnt.get(), 0, tb, ctx->stream));
    launch_tile_counts_from_cols(P.bin_rows(kBinHeavy), nheavy, P.nnz.as<int64_t>(), C->col_idx, P.ntiles,
                                 P.big_slot.as<int32_t>(), P.tile_cnt.as<int32_t>(), ctx->d_flags, lc);
    ++ctx->launches;
  }
  tm.mark(SPG_STAGE_NUMERIC);
  SPG_TRY(P.numeric(P.nnz.as<int64_t>(), C->col_idx, C->val, rep));
  tm.finish(rep);
  int f = 0;
  SPG_TRY(read_flags(ctx, &f));
  if (rep) {
    rep->device_flags |= f;
    rep->nnz_c = C->nnz;
  }
  if (f & kFlagCountDiff) return fail(ctx, SPG_ERR_INVALID_ARG, "the structure of C does not match A*B");
  if (f & kFlagBadIndex) return fail(ctx, SPG_ERR_INVALID_ARG, "C has columns outside [0, cols)");
  if (f & kFlagHashFull) return fail(ctx, SPG_ERR_INTERNAL, "device consistency check failed (flags %d)", f);
  return SPG_OK;
}

spg_status row_nnz_device(spg_ctx* ctx, const DevMat& A, const DevMat& B, int64_t* d_nnz) {
  Pipeline P(ctx, A, B, ctx->tuning);
  SPG_TRY(P.init());
  launch_row_products(A.view, B.view, P.prod.as<int64_t>(), P.lc);
  SPG_TRY(P.symbolic(P.prod.as<int64_t>()));
  if (P.rows)
    SPG_CUDA(ctx, cudaMemcpyAsync(d_nnz, P.nnz.get(), (size_t)P.rows * 8, cudaMemcpyDeviceToDevice, ctx->stream));
  return check_flags(ctx, nullptr);
}

}  // namespace spg

// ===========================================================================
// C ABI
// ===========================================================================

extern "C" {

int32_t spg_version(void) { return 10000; }

const char* spg_status_string(spg_status s) {
  switch (s) {
    case SPG_OK: return "ok";
    case SPG_ERR_INVALID_ARG: return "invalid argument";
    case SPG_ERR_CUDA: return "CUDA error";
    case SPG_ERR_OUT_OF_MEMORY: return "out of memory";
    case SPG_ERR_IO: return "I/O error";
    case SPG_ERR_FORMAT: return "malformed Matrix Market file";
    case SPG_ERR_TIMEOUT: return "device wait timed out";
    case SPG_ERR_UNSUPPORTED: return "unsupported";
    case SPG_ERR_INTERNAL: return "internal consistency check failed";
    default: return "unknown status";
  }
}

spg_status spg_create(spg_ctx** out, int32_t device) {
  if (!out) return SPG_ERR_INVALID_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    (void)cudaGetLastError();
    return SPG_ERR_CUDA;
  }
  if (device < 0 || device >= n) return SPG_ERR_INVALID_ARG;
  std::unique_ptr<spg_ctx> ctx(new (std::nothrow) spg_ctx());
  if (!ctx) return SPG_ERR_OUT_OF_MEMORY;
  ctx->device = device;
  SPG_CUDA(ctx.get(), cudaSetDevice(device));
  cudaDeviceProp prop{};
  SPG_CUDA(ctx.get(), cudaGetDeviceProperties(&prop, device));
  ctx->sms = prop.multiProcessorCount;
  ctx->gpu_name = prop.name;
  SPG_CUDA(ctx.get(), cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking));
  ctx->stream = ctx->own_stream;
  SPG_CUDA(ctx.get(), cudaDeviceGetDefaultMemPool(&ctx->pool, device));
  uint64_t thr = UINT64_MAX;
  SPG_CUDA(ctx.get(), cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &thr));
  SPG_CUDA(ctx.get(), cudaMalloc(&ctx->d_flags, 64));
  SPG_CUDA(ctx.get(), cudaMemset(ctx->d_flags, 0, 64));
  SPG_CUDA(ctx.get(), cudaMalloc(&ctx->d_counter, 8 * sizeof(unsigned long long)));
  SPG_CUDA(ctx.get(), cudaMemset(ctx->d_counter, 0, 8 * sizeof(unsigned long long)));
  // mapped, so small read-backs can be written by a kernel (stage_read)
  SPG_CUDA(ctx.get(), cudaHostAlloc((void**)&ctx->h_stage, 64 * sizeof(int64_t), cudaHostAllocMapped));
  SPG_CUDA(ctx.get(), cudaHostGetDevicePointer((void**)&ctx->h_stage_dev, ctx->h_stage, 0));
  ctx->tuning = default_tuning();
  *out = ctx.release();
  return SPG_OK;
}

spg_status spg_destroy(spg_ctx* ctx) {
  if (!ctx) return SPG_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  spg::free_batch_cache(ctx);
  cudaFree(ctx->mlp_master);
  cudaFree(ctx->mlp_w16);
  cudaFree(ctx->d_flags);
  cudaFree(ctx->d_counter);
  cudaFreeHost(ctx->h_stage);
  if (ctx->upload_stream) {
    cudaStreamSynchronize(ctx->upload_stream);
    cudaStreamDestroy(ctx->upload_stream);
  }
  if (ctx->copy_stream) {
    cudaStreamSynchronize(ctx->copy_stream);
    cudaStreamDestroy(ctx->copy_stream);
  }
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
  return SPG_OK;
}

const char* spg_last_error(const spg_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

spg_status spg_set_stream(spg_ctx* ctx, void* stream) {
  if (!ctx) return SPG_ERR_INVALID_ARG;
  ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
  return SPG_OK;
}

void* spg_get_stream(const spg_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

spg_status spg_multiply(spg_ctx* ctx, const spg_csr* A, const spg_csr* B, spg_csr* C, const spg_opts* opts,
                        spg_report* report) {
  if (!ctx) return SPG_ERR_INVALID_ARG;
  if (!A || !B || !C) return fail(ctx, SPG_ERR_INVALID_ARG, "null argument");
  if (A->cols != B->rows)
    return fail(ctx, SPG_ERR_INVALID_ARG, "inner dimensions differ (%lld vs %lld)", (long long)A->cols,
                (long long)B->rows);
  if (A->rows > INT32_MAX) return fail(ctx, SPG_ERR_UNSUPPORTED, "more than 2^31-1 rows");
  SPG_CUDA(ctx, cudaSetDevice(ctx->device));
  spg_opts o{};
  if (opts) o = *opts;
  if (report) {
    std::memset(report, 0, sizeof *report);
    report->algo = o.algo;
    report->rows = A->rows;
  }
  const int launches0 = ctx->launches;
  StageTimer outer(ctx, false);
  DevMat dA, dB;
  SPG_TRY(prepare_matrix(ctx, A, dA, !o.skip_validation));
  // C = A*A through one descriptor: prepared (uploaded) once
  const bool same = same_matrix(A, B);
  if (!same) SPG_TRY(prepare_matrix(ctx, B, dB, !o.skip_validation));
  const DevMat& rB = same ? dA : dB;
  if (!o.skip_validation) SPG_TRY(check_flags(ctx, report));
  spg_csr dev_c{};
  spg_status st;
  if (o.algo == SPG_ALGO_CUSPARSE) st = multiply_cusparse(ctx, dA, rB, &dev_c, o, report);
  else if (o.algo == SPG_ALGO_PLAIN || o.algo == SPG_ALGO_LEARNED) st = multiply_device(ctx, dA, rB, &dev_c, o, report);
  else return fail(ctx, SPG_ERR_INVALID_ARG, "unknown algo %d", o.algo);
  if (st != SPG_OK) {
    spg_csr_free(ctx, &dev_c);
    return st;
  }
  if (o.out_location == SPG_HOST) {
    spg_csr host_c{};
    st = spg_csr_copy(ctx, &dev_c, SPG_HOST, &host_c);
    spg_csr_free(ctx, &dev_c);
    if (st != SPG_OK) return st;
    *C = host_c;
  } else {
    *C = dev_c;
  }
  if (report) {
    outer.finish(nullptr);
    report->kernel_launches = ctx->launches - launches0;
    // whole-call device time, including uploads and the host copy
    float ms = 0.f;
    (void)ms;
  }
  return SPG_OK;
}

spg_status spg_multiply_into_host(spg_ctx* ctx, const spg_csr* A, const spg_csr* B, spg_csr* C, int32_t blocks,
                                  const spg_opts* opts, spg_report* report) {
  if (!ctx) return SPG_ERR_INVALID_ARG;
  if (!A || !B || !C) return fail(ctx, SPG_ERR_INVALID_ARG, "null argument");
  if (A->cols != B->rows)
    return fail(ctx, SPG_ERR_INVALID_ARG, "inner dimensions differ (%lld vs %lld)", (long long)A->cols,
                (long long)B->rows);
  if (C->location != SPG_HOST) return fail(ctx, SPG_ERR_INVALID_ARG, "C must describe host buffers");
  if (C->index_bits != 32 && C->index_bits != 64) return fail(ctx, SPG_ERR_INVALID_ARG, "bad C index_bits");
  if (!C->row_ptr || C->capacity < 0 || (C->capacity > 0 && (!C->col_idx || !C->val)))
    return fail(ctx, SPG_ERR_INVALID_ARG, "C needs row_ptr and, with a capacity, col_idx/val buffers");
  if (blocks < 1) return fail(ctx, SPG_ERR_INVALID_ARG, "blocks must be >= 1");
  if (A->rows > INT32_MAX) return fail(ctx, SPG_ERR_UNSUPPORTED, "more than 2^31-1 rows");
  spg_opts o{};
  if (opts) o = *opts;
  if (o.algo != SPG_ALGO_PLAIN && o.algo != SPG_ALGO_LEARNED)
    return fail(ctx, SPG_ERR_INVALID_ARG, "spg_multiply_into_host runs the plain or learned method");
  o.out_location = SPG_DEVICE;
  o.out_index_bits = 64;
  SPG_CUDA(ctx, cudaSetDevice(ctx->device));
  if (report) {
    std::memset(report, 0, sizeof *report);
    report->algo = o.algo;
    report->rows = A->rows;
  }
  const int launches0 = ctx->launches;
  DevMat dA, dB;
  const bool same = same_matrix(A, B);
  // A = B given once from host memory, validation off: the entries go up in
  // the compute blocks' row chunks on an upload stream, so block b waits only
  // for the chunks holding its own rows and the rows of B its columns reach,
  // and the upload runs beside the downloads of earlier blocks (the host
  // link carries both directions at once)
  const bool chunked = same && A->location == SPG_HOST && o.skip_validation && A->nnz > 0 && blocks > 1 &&
                       A->rows > 1;
  SPG_TRY(prepare_matrix(ctx, A, dA, !o.skip_validation, chunked));
  if (!same) SPG_TRY(prepare_matrix(ctx, B, dB, !o.skip_validation));
  const DevMat& rB = same ? dA : dB;
  if (!o.skip_validation) SPG_TRY(check_flags(ctx, report));
  if (!ctx->copy_stream) SPG_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
  std::vector<cudaEvent_t> up_evs;  // one per row chunk, on the upload stream
  struct UpEvents {
    spg_ctx* ctx;
    std::vector<cudaEvent_t>& evs;
    ~UpEvents() {
      if (!evs.empty()) cudaStreamSynchronize(ctx->upload_stream);
      for (cudaEvent_t e : evs) cudaEventDestroy(e);
    }
  } up_guard{ctx, up_evs};
  auto a_rp = [&](int64_t i) -> int64_t {
    return A->index_bits == 64 ? static_cast<const int64_t*>(A->row_ptr)[i]
                               : (int64_t) static_cast<const int32_t*>(A->row_ptr)[i];
  };
  // upload chunks: finer than the compute blocks, so that a block waits for
  // little more than the rows it reaches
  const int64_t nchunks = std::min<int64_t>(std::max<int64_t>(blocks, 64), std::max<int64_t>(A->rows, 1));
  if (chunked) {
    if (!ctx->upload_stream) SPG_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->upload_stream, cudaStreamNonBlocking));
    // the device buffers come from the pool on ctx->stream
    cudaEvent_t alloc_ev = nullptr;
    SPG_CUDA(ctx, cudaEventCreateWithFlags(&alloc_ev, cudaEventDisableTiming));
    up_evs.push_back(alloc_ev);
    SPG_CUDA(ctx, cudaEventRecord(alloc_ev, ctx->stream));
    SPG_CUDA(ctx, cudaStreamWaitEvent(ctx->upload_stream, alloc_ev, 0));
    int32_t* dcol = dA.upload[1].as<int32_t>();
    float* dval = dA.upload[2].as<float>();
    for (int64_t c = 0; c < nchunks; ++c) {
      const int64_t e0 = a_rp(A->rows * c / nchunks), e1 = a_rp(A->rows * (c + 1) / nchunks);
      if (e1 > e0) {
        SPG_CUDA(ctx, cudaMemcpyAsync(dcol + e0, A->col_idx + e0, (size_t)(e1 - e0) * 4, cudaMemcpyHostToDevice,
                                      ctx->upload_stream));
        SPG_CUDA(ctx, cudaMemcpyAsync(dval + e0, A->val + e0, (size_t)(e1 - e0) * 4, cudaMemcpyHostToDevice,
                                      ctx->upload_stream));
      }
      cudaEvent_t ev = nullptr;
      SPG_CUDA(ctx, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      up_evs.push_back(ev);
      SPG_CUDA(ctx, cudaEventRecord(ev, ctx->upload_stream));
    }
    dA.complete = up_evs.back();
  }
  const LaunchCtx lc = launch_ctx(ctx);
  const int64_t rows = A->rows;
  const int w = C->index_bits / 8;
  char* host_rp = static_cast<char*>(C->row_ptr);
  C->rows = rows;
  C->cols = B->cols;
  if (rows == 0) {
    if (w == 8) *static_cast<int64_t*>(C->row_ptr) = 0;
    else *static_cast<int32_t*>(C->row_ptr) = 0;
    C->nnz = 0;
    return SPG_OK;
  }
  const int64_t nb = std::min<int64_t>(blocks, rows);
  // even row blocks (a first block of a quarter the size, to start the
  // first download sooner, measured 18.9 -> 19.3 ms on the stencil-96 call)
  auto block_start = [&](int64_t b) -> int64_t { return rows * b / nb; };
  DevBuf rp_dev;  // C's row pointers in C's width, staged for the copies
  SPG_TRY(rp_dev.alloc(ctx, (size_t)(rows + 1) * w));
  std::vector<cudaEvent_t> evs;
  std::vector<spg_csr> parts;  // device parts of C whose copies are in flight
  auto drain = [&]() {
    cudaStreamSynchronize(ctx->copy_stream);
    for (cudaEvent_t e : evs) cudaEventDestroy(e);
    evs.clear();
    for (spg_csr& c : parts) spg_csr_free(ctx, &c);
    parts.clear();
  };
  int64_t offset = 0;
  bool overflow = false;
  spg_status st = SPG_OK;
  for (int64_t b = 0; b < nb && st == SPG_OK; ++b) {
    const int64_t r0 = block_start(b), r1 = block_start(b + 1);
    DevMat Ab;  // view of A's rows [r0, r1): row pointers index the full column/value arrays
    Ab.view = dA.view;
    Ab.view.rows = r1 - r0;
    Ab.view.rp = dA.view.rp + r0;
    Ab.view.rp32 = dA.view.rp32 ? dA.view.rp32 + r0 : nullptr;
    Ab.nnz = dA.nnz;
    if (chunked) {
      // rows of A keep ascending columns: a row's largest column is its last entry
      int64_t last = r1 - 1;
      for (int64_t r = r0; r < r1; ++r) {
        const int64_t e = a_rp(r + 1);
        if (e > a_rp(r)) last = std::max<int64_t>(last, A->col_idx[e - 1]);
      }
      last = std::min<int64_t>(last, rows - 1);
      // the chunk holding row `last` (chunks hold rows [rows*c/nchunks, rows*(c+1)/nchunks))
      int64_t chunk = std::min<int64_t>(nchunks - 1, last * nchunks / rows);
      while (chunk > 0 && rows * chunk / nchunks > last) --chunk;
      while (chunk + 1 < nchunks && rows * (chunk + 1) / nchunks <= last) ++chunk;
      st = cuda_status(ctx, cudaStreamWaitEvent(ctx->stream, up_evs[(size_t)chunk + 1], 0), "cudaStreamWaitEvent");
      if (st != SPG_OK) break;
    }
    spg_csr cb{};
    spg_report rb{};
    st = multiply_device(ctx, Ab, rB, &cb, o, report ? &rb : nullptr);
    if (st != SPG_OK) {
      spg_csr_free(ctx, &cb);
      break;
    }
    if (report) {
      report->products += rb.products;
      report->ms_total += rb.ms_total;
      report->rows_predicted += rb.rows_predicted;
      report->rows_overflow += rb.rows_overflow;
      report->rows_heavy += rb.rows_heavy;
      report->device_flags |= rb.device_flags;
      for (int s = 0; s < SPG_STAGE_COUNT; ++s) report->ms_stage[s] += rb.ms_stage[s];
      for (int s = 0; s < SPG_NUM_BINS; ++s) report->bin_rows[s] += rb.bin_rows[s];
    }
    if (!overflow && offset + cb.nnz <= C->capacity) {
      // this block's rows of C (its last row pointer too for the final block)
      const int64_t n_rp = (r1 == rows) ? (r1 - r0 + 1) : (r1 - r0);
      launch_shift_rp(static_cast<const int64_t*>(cb.row_ptr), n_rp, offset, rp_dev.as<char>() + (size_t)r0 * w,
                      C->index_bits, lc);
      ++ctx->launches;
      cudaEvent_t ev = nullptr;
      st = cuda_status(ctx, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate");
      if (st != SPG_OK) {
        spg_csr_free(ctx, &cb);
        break;
      }
      evs.push_back(ev);
      cudaEventRecord(ev, ctx->stream);
      cudaStreamWaitEvent(ctx->copy_stream, ev, 0);
      cudaMemcpyAsync(host_rp + (size_t)r0 * w, rp_dev.as<char>() + (size_t)r0 * w, (size_t)n_rp * w,
                      cudaMemcpyDeviceToHost, ctx->copy_stream);
      if (cb.nnz) {
        cudaMemcpyAsync(C->col_idx + offset, cb.col_idx, (size_t)cb.nnz * 4, cudaMemcpyDeviceToHost,
                        ctx->copy_stream);
        cudaMemcpyAsync(C->val + offset, cb.val, (size_t)cb.nnz * 4, cudaMemcpyDeviceToHost, ctx->copy_stream);
      }
      // kept until every copy is done: freeing it on the copy stream would let
      // the pool hand its memory to the next block's compute with a wait on
      // this copy, serializing the two
      parts.push_back(cb);
    } else {
      overflow = true;
      spg_csr_free(ctx, &cb);
    }
    offset += cb.nnz;
  }
  // the staged row pointers are freed on ctx->stream: order it after the copies
  drain();
  if (st != SPG_OK) return st;
  SPG_CUDA(ctx, cudaGetLastError());
  C->nnz = offset;
  if (report) {
    report->nnz_c = offset;
    report->kernel_launches = ctx->launches - launches0;
  }
  if (overflow)
    return fail(ctx, SPG_ERR_INVALID_ARG,
                "C needs room for %lld entries but its capacity is %lld (C->nnz holds the size needed)",
                (long long)offset, (long long)C->capacity);
  return SPG_OK;
}

spg_status spg_multiply_reuse(spg_ctx* ctx, const spg_csr* A, const spg_csr* B, spg_csr* C, const spg_opts* opts,
                              spg_report* report) {
  if (!ctx) return SPG_ERR_INVALID_ARG;
  if (!A || !B || !C) return fail(ctx, SPG_ERR_INVALID_ARG, "null argument");
  if (A->cols != B->rows)
    return fail(ctx, SPG_ERR_INVALID_ARG, "inner dimensions differ (%lld vs %lld)", (long long)A->cols,
                (long long)B->rows);
  if (C->location != SPG_DEVICE) return fail(ctx, SPG_ERR_INVALID_ARG, "C must be on the device");
  if (C->rows != A->rows || C->cols != B->cols)
    return fail(ctx, SPG_ERR_INVALID_ARG, "C is %lld x %lld, A*B is %lld x %lld", (long long)C->rows,
                (long long)C->cols, (long long)A->rows, (long long)B->cols);
  if (C->index_bits != 32 && C->index_bits != 64) return fail(ctx, SPG_ERR_INVALID_ARG, "bad C index_bits");
  if (C->rows > 0 && !C->row_ptr) return fail(ctx, SPG_ERR_INVALID_ARG, "C has no row pointers");
  if (C->nnz > 0 && (!C->col_idx || !C->val)) return fail(ctx, SPG_ERR_INVALID_ARG, "C has no column/value arrays");
  if (A->rows > INT32_MAX) return fail(ctx, SPG_ERR_UNSUPPORTED, "more than 2^31-1 rows");
  SPG_CUDA(ctx, cudaSetDevice(ctx->device));
  spg_opts o{};
  if (opts) o = *opts;
  if (report) {
    std::memset(report, 0, sizeof *report);
    report->algo = SPG_ALGO_PLAIN;
    report->rows = A->rows;
  }
  const int launches0 = ctx->launches;
  DevMat dA, dB;
  SPG_TRY(prepare_matrix(ctx, A, dA, !o.skip_validation));
  const bool same = same_matrix(A, B);
  if (!same) SPG_TRY(prepare_matrix(ctx, B, dB, !o.skip_validation));
  if (!o.skip_validation) SPG_TRY(check_flags(ctx, report));
  SPG_TRY(spg::multiply_reuse_device(ctx, dA, same ? dA : dB, C, o, report));
  if (report) report->kernel_launches = ctx->launches - launches0;
  return SPG_OK;
}

spg_status spg_csr_free(spg_ctx* ctx, spg_csr* m) {
  if (!m || m->owner == 0) return SPG_OK;
  if (m->owner == 1) {
    cudaStream_t s = ctx ? ctx->stream : nullptr;
    if (m->row_ptr) cudaFreeAsync(m->row_ptr, s);
    if (m->col_idx) cudaFreeAsync(m->col_idx, s);
    if (m->val) cudaFreeAsync(m->val, s);
  } else if (m->owner == 2) {
    free(m->row_ptr);
    free(m->col_idx);
    free(m->val);
  } else if (m->owner == 3) {
    cudaFreeHost(m->row_ptr);
    cudaFreeHost(m->col_idx);
    cudaFreeHost(m->val);
  }
  m->row_ptr = nullptr;
  m->col_idx = nullptr;
  m->val = nullptr;
  m->owner = 0;
  return SPG_OK;
}

spg_status spg_csr_copy(spg_ctx* ctx, const spg_csr* src, int32_t location, spg_csr* dst) {
  if (!ctx || !src || !dst) return SPG_ERR_INVALID_ARG;
  if (location != SPG_HOST && location != SPG_DEVICE) return fail(ctx, SPG_ERR_INVALID_ARG, "bad location");
  spg_csr d = *src;
  d.location = location;
  d.capacity = src->nnz;
  const size_t rpb = (size_t)(src->rows + 1) * (src->index_bits / 8);
  const size_t nb = (size_t)src->nnz * 4;
  const cudaMemcpyKind kind =
      src->location == SPG_HOST ? (location == SPG_HOST ? cudaMemcpyHostToHost : cudaMemcpyHostToDevice)
                                : (location == SPG_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice);
  if (location == SPG_HOST) {
    d.owner = 2;
    d.row_ptr = malloc(std::max<size_t>(rpb, 1));
    d.col_idx = (int32_t*)malloc(std::max<size_t>(nb, 1));
    d.val = (float*)malloc(std::max<size_t>(nb, 1));
    if (!d.row_ptr || !d.col_idx || !d.val) {
      free(d.row_ptr);
      free(d.col_idx);
      free(d.val);
      return fail(ctx, SPG_ERR_OUT_OF_MEMORY, "host allocation of %zu bytes failed", rpb + 2 * nb);
    }
  } else {
    d.owner = 1;
    DevBuf a, b, c;
    SPG_TRY(a.alloc(ctx, std::max<size_t>(rpb, 4)));
    SPG_TRY(b.alloc(ctx, std::max<size_t>(nb, 4)));
    SPG_TRY(c.alloc(ctx, std::max<size_t>(nb, 4)));
    d.row_ptr = a.release();
    d.col_idx = (int32_t*)b.release();
    d.val = (float*)c.release();
  }
  if (rpb) SPG_CUDA(ctx, cudaMemcpyAsync(d.row_ptr, src->row_ptr, rpb, kind, ctx->stream));
  if (nb) {
    SPG_CUDA(ctx, cudaMemcpyAsync(d.col_idx, src->col_idx, nb, kind, ctx->stream));
    SPG_CUDA(ctx, cudaMemcpyAsync(d.val, src->val, nb, kind, ctx->stream));
  }
  SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *dst = d;
  return SPG_OK;
}

spg_status spg_csr_download(spg_ctx* ctx, const spg_csr* src, void* row_ptr, int32_t* col_idx, float* val) {
  if (!ctx || !src || !row_ptr || (src->nnz > 0 && (!col_idx || !val))) return SPG_ERR_INVALID_ARG;
  if (src->location != SPG_DEVICE) return fail(ctx, SPG_ERR_INVALID_ARG, "spg_csr_download needs a device matrix");
  SPG_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t rpb = (size_t)(src->rows + 1) * (src->index_bits / 8);
  const size_t nb = (size_t)src->nnz * 4;
  SPG_CUDA(ctx, cudaMemcpyAsync(row_ptr, src->row_ptr, rpb, cudaMemcpyDeviceToHost, ctx->stream));
  if (nb) {
    SPG_CUDA(ctx, cudaMemcpyAsync(col_idx, src->col_idx, nb, cudaMemcpyDeviceToHost, ctx->stream));
    SPG_CUDA(ctx, cudaMemcpyAsync(val, src->val, nb, cudaMemcpyDeviceToHost, ctx->stream));
  }
  SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SPG_OK;
}

spg_status spg_csr_extract_rows(spg_ctx* ctx, const spg_csr* src, const int64_t* rows, int64_t n, spg_csr* dst) {
  if (!ctx || !src || !dst || n < 0 || (n > 0 && !rows)) return SPG_ERR_INVALID_ARG;
  if (src->location != SPG_DEVICE) return fail(ctx, SPG_ERR_INVALID_ARG, "spg_csr_extract_rows needs a device matrix");
  SPG_CUDA(ctx, cudaSetDevice(ctx->device));
  const int w = src->index_bits / 8;
  std::vector<int64_t> start((size_t)n), len((size_t)n);
  for (int64_t t = 0; t < n; ++t) {
    if (rows[t] < 0 || rows[t] >= src->rows) return fail(ctx, SPG_ERR_INVALID_ARG, "row %lld out of range", (long long)rows[t]);
    int64_t se[2] = {0, 0};
    const char* base = static_cast<const char*>(src->row_ptr) + (size_t)rows[t] * w;
    if (w == 8) {
      SPG_CUDA(ctx, cudaMemcpy(se, base, 16, cudaMemcpyDeviceToHost));
    } else {
      int32_t s32[2];
      SPG_CUDA(ctx, cudaMemcpy(s32, base, 8, cudaMemcpyDeviceToHost));
      se[0] = s32[0];
      se[1] = s32[1];
    }
    start[(size_t)t] = se[0];
    len[(size_t)t] = se[1] - se[0];
  }
  int64_t total = 0;
  for (int64_t t = 0; t < n; ++t) total += len[(size_t)t];
  spg_csr d{};
  d.rows = n;
  d.cols = src->cols;
  d.nnz = total;
  d.capacity = total;
  d.index_bits = 64;
  d.location = SPG_HOST;
  d.owner = 2;
  d.row_ptr = malloc((size_t)(n + 1) * 8);
  d.col_idx = (int32_t*)malloc(std::max<size_t>((size_t)total * 4, 4));
  d.val = (float*)malloc(std::max<size_t>((size_t)total * 4, 4));
  if (!d.row_ptr || !d.col_idx || !d.val) {
    free(d.row_ptr);
    free(d.col_idx);
    free(d.val);
    return fail(ctx, SPG_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
  int64_t* rp = static_cast<int64_t*>(d.row_ptr);
  rp[0] = 0;
  for (int64_t t = 0; t < n; ++t) {
    rp[t + 1] = rp[t] + len[(size_t)t];
    if (len[(size_t)t]) {
      SPG_CUDA(ctx, cudaMemcpyAsync(d.col_idx + rp[t], src->col_idx + start[(size_t)t], (size_t)len[(size_t)t] * 4,
                                    cudaMemcpyDeviceToHost, ctx->stream));
      SPG_CUDA(ctx, cudaMemcpyAsync(d.val + rp[t], src->val + start[(size_t)t], (size_t)len[(size_t)t] * 4,
                                    cudaMemcpyDeviceToHost, ctx->stream));
    }
  }
  SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *dst = d;
  return SPG_OK;
}

}  // extern "C"
