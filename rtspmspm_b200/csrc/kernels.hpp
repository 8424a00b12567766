// Host-side declarations of the SpGEMM kernel launchers.
#pragma once

#include <algorithm>
#include <cstdint>
#include <cuda_runtime.h>

#ifndef SPG_TILE_SHIFT
#define SPG_TILE_SHIFT 11
#endif

namespace spg {

struct DCsr;

// Bin ids.  Warp-hash bins 0..7 hold tables of 2^(5+bin) slots.
constexpr int kMinLogT = 5;
constexpr int kMaxLogT = 12;
constexpr int kNumWarpBins = kMaxLogT - kMinLogT + 1;  // 8
constexpr int kBinBlock = 8;   // symbolic: CTA hash table; numeric: CTA hash of 2^12 slots
constexpr int kBinDense = 9;   // symbolic: CTA bitmap over the column span; numeric: CTA hash of 2^14 slots
constexpr int kBinHeavy = 10;  // numeric: column-tiled heavy rows
constexpr int kBinEmpty = 11;  // no products
constexpr int kNumBins = 12;

// Log2 of the CTA-wide numeric hash tables of kBinBlock / kBinDense.
constexpr int kBlkLogSmallT = 12;
constexpr int kBlkLogLargeT = 14;

constexpr int kBinSymbolic = 0;
constexpr int kBinNumeric = 1;
constexpr int kBinLearned = 2;

// Warps per CTA of the heavy tile kernel: up to 8 per-warp tiles (floats,
// bitmap, 32-float stage) within 227 KB of shared memory; the grid holds as
// many CTAs per SM as fit.
constexpr int kTileWarpBytes = ((1 << SPG_TILE_SHIFT) + (1 << SPG_TILE_SHIFT) / 32 + 32) * 4;
constexpr int kTileWarps = (227 * 1024) / kTileWarpBytes > 8 ? 8 : (227 * 1024) / kTileWarpBytes;
constexpr int kDenseWindowWords = 40960;   // 1,310,720 columns of bitmap per window

struct BinParams {
  int64_t warp_cap;    // largest bound (symbolic) / nnz (numeric) on a warp table
  int64_t block_cap;   // largest bound on the symbolic CTA table
  int warp_log_max;    // log2 of the largest warp table
  float max_load;      // numeric table load factor
  // numeric / learned binning: rows with more than block_min entries go to
  // the CTA-wide hash bins (kBinBlock up to blk_small_cap entries, kBinDense
  // up to blk_large_cap); block_min = INT64_MAX and the caps 0 turn them off
  int64_t block_min;
  int64_t blk_small_cap;
  int64_t blk_large_cap;
};

// BinParams with the CTA-wide numeric bins turned off (paths that only
// launch the warp bins and the heavy tiles).
inline BinParams without_block_bins(BinParams bp) {
  bp.block_min = INT64_MAX;
  bp.blk_small_cap = 0;
  bp.blk_large_cap = 0;
  return bp;
}

struct LaunchCtx {
  cudaStream_t stream;
  int sms;
};

void launch_widen_rp(const int32_t* in, int64_t n, int64_t* out, const LaunchCtx& lc);
void launch_narrow_rp(const int64_t* in, int64_t n, int32_t* out, const LaunchCtx& lc);
void launch_validate(const DCsr& M, int64_t nnz, int* flags, const LaunchCtx& lc);
void launch_row_products(const DCsr& A, const DCsr& B, int64_t* prod, const LaunchCtx& lc);

// Small products (at most kSmallMaxRows rows of A, every row of at most
// 2^kSmallLogT products): products and exact counts per row in one launch
// (nnz[row] = -1 for a row of more products), then one CTA scans the counts
// into C's row pointers (int64 in place, int32 into rp32 when given and the
// total fits), writes the identity row list and puts the total, the
// products, the largest count and the too-large rows into out[0..3]
// (mapped host words).
constexpr int kSmallLogT = 11;
constexpr int kSmallCountWarps = 4;
constexpr int kSmallScanThreads = 1024;
constexpr int64_t kSmallMaxRows = 65536;
constexpr int kSmallDefaultRows = 8192;
// `stop` (one device word, zero between calls): set by the counting launch
// at its first too-large row so that the remaining rows skip their counts;
// the scan clears it.
void launch_small_count(const DCsr& A, const DCsr& B, int64_t* prod, int64_t* nnz, unsigned long long* stop,
                        int* flags, const LaunchCtx& lc);
void launch_small_scan(int64_t* nnz, const int64_t* prod, int64_t rows, int32_t* rp32, int32_t* row_list,
                       unsigned long long* stop, int64_t* out, const LaunchCtx& lc);
void launch_sum(const int64_t* v, int64_t n, unsigned long long* out, const LaunchCtx& lc);
void launch_binning(const int64_t* key, int64_t rows, int64_t cols, int mode, const BinParams& bp,
                    uint8_t* bin_of_row, int64_t* counts, int64_t* offsets, int64_t* cursors, int32_t* lists,
                    const LaunchCtx& lc);
int64_t scan_temp_elems(int64_t n);
void launch_excl_scan(const int64_t* in, int64_t n, int64_t* out, int64_t* tmp, const LaunchCtx& lc);

void launch_sym_warp(int log_t, const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows, int64_t* nnz,
                     int* flags, const LaunchCtx& lc, int wpb);
void launch_sym_block(const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows, int log_table,
                      int64_t slot_base, int64_t* nnz, int32_t* big_slot, int32_t* tile_cnt, int ntiles, int* flags,
                      const LaunchCtx& lc);
void launch_sym_dense(const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows, int64_t slot_base,
                      int64_t* nnz, int32_t* big_slot, int32_t* tile_cnt, int ntiles, int* flags,
                      const LaunchCtx& lc);
// Default smallest product count of an expand-sort-fold row.
constexpr int kEscMinProd = 128;
// Expand-sort-fold rows in the warp numeric kernels: the row products
// (nullptr: off) and the smallest product count that takes the path
// (0: off).
struct EscArgs {
  const int64_t* prod = nullptr;
  int min_prod = 0;
};
void launch_num_warp(int log_t, const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows,
                     const int64_t* c_rp, int32_t* c_col, float* c_val, int* flags, const LaunchCtx& lc, int wpb,
                     const EscArgs& esc = EscArgs{});
void launch_num_warp_learned(int log_t, const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows,
                             const int64_t* cap, const int64_t* slab_off, int32_t* slab_col, float* slab_val,
                             int64_t* nnz_out, int32_t* retry_rows, unsigned long long* retry_count, int* flags,
                             const LaunchCtx& lc, int wpb, const EscArgs& esc = EscArgs{});
// CTA-wide hash numeric pass over the rows of bin kBinBlock (2^12-slot
// tables) or kBinDense (2^14) of a numeric / learned binning.
void launch_num_block(int bin, const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows, const int64_t* c_rp,
                      int32_t* c_col, float* c_val, int* flags, const LaunchCtx& lc);
void launch_num_block_learned(int bin, const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows,
                              const int64_t* cap, const int64_t* slab_off, int32_t* slab_col, float* slab_val,
                              int64_t* nnz_out, int32_t* retry_rows, unsigned long long* retry_count, int* flags,
                              const LaunchCtx& lc);
// Copies n 32-bit words with one small kernel (dst may be mapped pinned host
// memory: the read-back then needs no copy engine).
void launch_copy_words(const void* src, void* dst, int64_t n, const LaunchCtx& lc);
// Row pointers shifted by `off` into an int32 (out_bits 32) or int64 array.
void launch_shift_rp(const int64_t* in, int64_t n, int64_t off, void* out, int out_bits, const LaunchCtx& lc);
// Value-only recompute: row lengths of C, and heavy-row slots and per-tile
// counts from C's sorted columns (tile_cnt zeroed by the caller).
void launch_row_lengths(const int64_t* rp, int64_t rows, int64_t* len, const LaunchCtx& lc);
void launch_tile_counts_from_cols(const int32_t* heavy_rows, int64_t nheavy, const int64_t* c_rp,
                                  const int32_t* c_col, int ntiles, int32_t* big_slot, int32_t* tile_cnt, int* flags,
                                  const LaunchCtx& lc);
// Per heavy row: tile offsets (scan of the tile counts) and, when nz_cnt is
// given, its number of non-empty tiles.
void launch_tile_offsets(const int32_t* heavy_rows, int64_t nheavy, const int32_t* big_slot, const int32_t* tile_cnt,
                         int ntiles, int32_t* tile_off, int64_t* nz_cnt, const LaunchCtx& lc);
// The non-empty (heavy row, tile) units, h * ntiles + tile, at nz_off[h].
void launch_tile_worklist(const int32_t* heavy_rows, int64_t nheavy, const int32_t* big_slot, const int32_t* tile_cnt,
                          int ntiles, const int64_t* nz_off, int64_t* work, const LaunchCtx& lc);
void launch_build_blocked_index(const DCsr& B, int ntiles, int32_t* bidx, const LaunchCtx& lc);
// Tile occupancy bits of B from its blocked index (ceil(ntiles / 32) words per row).
void launch_build_tile_occupancy(int64_t rows, const int32_t* bidx, int ntiles, uint32_t* tocc, const LaunchCtx& lc);
// bidx: blocked index of B (launch_build_blocked_index) or null (binary
// searches); tocc: its occupancy bits or null; work/nwork: the list of
// non-empty tiles (launch_tile_worklist) and its length on the device, or
// null (every tile is visited); bulk: segments of 64+ entries staged into
// shared memory by bulk copies (when B's arrays are 16-byte aligned)
void launch_num_tile(const DCsr& A, const DCsr& B, const int32_t* heavy_rows, int64_t nheavy, const int32_t* big_slot,
                     const int32_t* tile_cnt, const int32_t* tile_off, int ntiles, const int64_t* c_rp,
                     int32_t* c_col, float* c_val, const int32_t* bidx, const uint32_t* tocc, const int64_t* work,
                     const int64_t* nwork, unsigned long long* tile_counter, int* flags, const LaunchCtx& lc,
                     bool bulk = false);
void launch_compact_rows(const int32_t* rows, int64_t nrows, const uint8_t* need_exact, const int64_t* slab_off,
                         const int32_t* slab_col, const float* slab_val, const int64_t* c_rp, int32_t* c_col,
                         float* c_val, const LaunchCtx& lc);
void launch_mark_rows(const int32_t* retry, const unsigned long long* count, uint8_t* need_exact, const LaunchCtx& lc);
// out[r] = scan[r + 1] - scan[r] (undoes an exclusive scan of rows counts).
void launch_adjacent_diff(const int64_t* scan, int64_t rows, int64_t* out, const LaunchCtx& lc);
void launch_mask_key(const int64_t* src, const uint8_t* mask, int64_t rows, int64_t* dst, const LaunchCtx& lc);

}  // namespace spg
