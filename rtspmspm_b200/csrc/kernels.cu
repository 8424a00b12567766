// Row-wise Gustavson SpGEMM kernels for sm_100a.
//
// Stage map (reference counterparts):
//   k_validate / k_row_products  -- the reference has no index build: B's
//       "row index" is the sphere BVH (optixSpMSpM.cpp:189-260); here it is
//       B's CSR row pointer, and the per-row intermediate-product count
//       replaces the ray count (one ray per A nonzero, optixSpMSpM.cu:113-201).
//   k_bin_*       -- groups rows by intermediate products (no counterpart).
//   k_sym_*       -- exact nnz per output row (inside cuSPARSE's
//       workEstimation, cuSparse/src/main.cpp:464-478).
//   k_num_*       -- the multiply-accumulate of the any-hit program
//       (optixSpMSpM.cu:234-260) into per-row shared-memory accumulators
//       instead of a dense rows x cols buffer (optixSpMSpM.cpp:164-171).
//   compaction + per-row sort -- the dense-to-COO scan of printResult
//       (optixSpMSpM.cpp:452-494), done per row on the device.
#include "common.cuh"
#include "kernels.hpp"
#include "warp_row.cuh"

namespace spg {

// --------------------------------------------------------------------------
// Input preparation
// --------------------------------------------------------------------------

__global__ void k_widen_rp(const int32_t* in, int64_t n, int64_t* out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (int64_t)in[i];
}

__global__ void k_narrow_rp(const int64_t* in, int64_t n, int32_t* out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (int32_t)in[i];
}

// Checks row pointers are monotone, columns are in [0, cols) and strictly
// increasing within each row (sorted, no duplicates).  One warp per row.
__global__ void k_validate(DCsr M, int64_t nnz, int* flags) {
  const int lane = lane_id();
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  bool bad = false;
  for (int64_t r = gw; r < M.rows; r += nw) {
    const int64_t s = M.rp[r], e = M.rp[r + 1];
    if (s > e || s < 0 || e > nnz) {
      bad = true;
      continue;
    }
    for (int64_t p = s + lane; p < e; p += 32) {
      int32_t c = M.col[p];
      if (c < 0 || c >= M.cols) bad = true;
      if (p > s && M.col[p - 1] >= c) bad = true;
    }
  }
  if (__any_sync(kFull, bad) && lane == 0) raise_flag(flags, kFlagBadIndex);
}

// Intermediate products per row (sum of |B_k| over k in A_i) and the upper
// bound min(products, cols of B) of its output nnz.  One warp per row.
__global__ void k_row_products(DCsr A, DCsr B, int64_t* prod) {
  const int lane = lane_id();
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = gw; r < A.rows; r += nw) {
    const int64_t s = A.rp[r], e = A.rp[r + 1];
    int64_t sum = 0;
    for (int64_t p = s + lane; p < e; p += 32) {
      int32_t k = A.col[p];
      sum += B.rp[k + 1] - B.rp[k];
    }
    sum = warp_sum(sum);
    if (lane == 0) prod[r] = sum;
  }
}

__global__ void k_sum_i64(const int64_t* v, int64_t n, unsigned long long* out) {
  unsigned long long s = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    s += (unsigned long long)v[i];
  s = warp_sum(s);
  if (lane_id() == 0 && s) atomicAdd(out, s);
}

// --------------------------------------------------------------------------
// Binning
// --------------------------------------------------------------------------

__device__ __forceinline__ int ceil_log2_i64(int64_t v) {
  // smallest L with 2^L >= v (v >= 1)
  return v <= 1 ? 0 : 64 - __clzll((unsigned long long)(v - 1));
}

// Bin of a row given its size key.
//  mode kBinSymbolic: key = products; bound u = min(key, cols).
//  mode kBinNumeric:  key = exact nnz.
//  mode kBinLearned:  key = predicted capacity (already capped by the bound).
__device__ __forceinline__ int bin_of(int64_t key, int64_t cols, int mode, const BinParams& bp) {
  if (mode == kBinSymbolic) {
    int64_t u = key < cols ? key : cols;
    if (u <= 0) return kBinEmpty;
    if (u <= bp.warp_cap) {
      int64_t need = u + (u >> 1) + 1;  // table load <= 2/3
      int lg = ceil_log2_i64(need);
      if (lg < kMinLogT) lg = kMinLogT;
      if (lg > bp.warp_log_max) lg = bp.warp_log_max;
      return lg - kMinLogT;
    }
    if (u <= bp.block_cap) return kBinBlock;
    return kBinDense;
  }
  if (key <= 0) return kBinEmpty;
  if (key <= bp.warp_cap) {
    int64_t need = (int64_t)ceilf((float)key / bp.max_load);
    int lg = ceil_log2_i64(need);
    if (lg < kMinLogT) lg = kMinLogT;
    if (lg > bp.warp_log_max) lg = bp.warp_log_max;
    return lg - kMinLogT;
  }
  return kBinHeavy;
}

// Histogram of bins (warp-aggregated atomics).
__global__ void k_bin_count(const int64_t* key, int64_t rows, int64_t cols, int mode, BinParams bp,
                            uint8_t* bin_of_row, int64_t* counts) {
  for (int64_t r0 = blockIdx.x * (int64_t)blockDim.x; r0 < rows; r0 += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = r0 + threadIdx.x;
    int b = -1;
    if (r < rows) {
      b = bin_of(key[r], cols, mode, bp);
      bin_of_row[r] = (uint8_t)b;
    }
    unsigned active = __ballot_sync(kFull, r < rows);
    if (r < rows) {
      unsigned grp = __match_any_sync(active, b);
      if (lane_id() == __ffs(grp) - 1) atomicAdd((unsigned long long*)&counts[b], (unsigned long long)__popc(grp));
    }
  }
}

// counts -> offsets[kNumBins+1]; cursors = offsets.
__global__ void k_bin_offsets(const int64_t* counts, int64_t* offsets, int64_t* cursors) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    int64_t s = 0;
    for (int b = 0; b < kNumBins; ++b) {
      offsets[b] = s;
      cursors[b] = s;
      s += counts[b];
    }
    offsets[kNumBins] = s;
  }
}

// Scatter row ids into per-bin lists (order within a bin follows warp
// arrival; it only affects scheduling, never results).
__global__ void k_bin_scatter(const uint8_t* bin_of_row, int64_t rows, int64_t* cursors, int32_t* lists) {
  for (int64_t r0 = blockIdx.x * (int64_t)blockDim.x; r0 < rows; r0 += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = r0 + threadIdx.x;
    unsigned active = __ballot_sync(kFull, r < rows);
    if (r < rows) {
      int b = bin_of_row[r];
      unsigned grp = __match_any_sync(active, b);
      int leader = __ffs(grp) - 1;
      unsigned long long base = 0;
      if (lane_id() == leader) base = atomicAdd((unsigned long long*)&cursors[b], (unsigned long long)__popc(grp));
      base = __shfl_sync(grp, base, leader);
      int rank = __popc(grp & ((1u << lane_id()) - 1u));
      lists[base + rank] = (int32_t)r;
    }
  }
}

// --------------------------------------------------------------------------
// Exclusive scan of int64 (three-phase, recursive over block sums)
// --------------------------------------------------------------------------

constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int64_t block_excl_scan(int64_t v, int64_t* sh_warp, int64_t& total) {
  const int lane = lane_id(), w = threadIdx.x >> 5;
  int64_t inc = warp_incl_scan(v);
  if (lane == 31) sh_warp[w] = inc;
  __syncthreads();
  if (w == 0) {
    int64_t x = lane < (kScanThreads / 32) ? sh_warp[lane] : 0;
    int64_t xi = warp_incl_scan(x);
    if (lane < (kScanThreads / 32)) sh_warp[lane] = xi - x;
    if (lane == 31) sh_warp[32] = xi;
  }
  __syncthreads();
  int64_t r = inc - v + sh_warp[w];
  total = sh_warp[32];
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const int64_t* in, int64_t n, int64_t* sums) {
  __shared__ int64_t sh[33];
  int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int64_t s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i)
    if (base + i < n) s += in[base + i];
  int64_t tot;
  block_excl_scan(s, sh, tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// out[i] = offset[block] + exclusive prefix within block; out may alias in.
__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const int64_t* in, int64_t n, const int64_t* block_off,
                                                               int64_t* out) {
  __shared__ int64_t sh[33];
  int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int64_t v[kScanItems];
  int64_t s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    v[i] = (base + i < n) ? in[base + i] : 0;
    s += v[i];
  }
  int64_t tot;
  int64_t pre = block_excl_scan(s, sh, tot) + (block_off ? block_off[blockIdx.x] : 0);
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (base + i < n) out[base + i] = pre;
    pre += v[i];
  }
}

__global__ void k_store_total(const int64_t* excl_last, const int64_t* in_last, int64_t* dst) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *dst = *excl_last + *in_last;
}

// --------------------------------------------------------------------------
// Symbolic pass
// --------------------------------------------------------------------------

// Warp per row; per-warp key table of 2^LOGT slots in shared memory.
template <int LOGT, bool R32>
__global__ void __launch_bounds__(512, 2) k_sym_warp(DCsr A, DCsr B, const int32_t* rows, int64_t nrows, int64_t* nnz_out, int* flags) {
  constexpr int T = 1 << LOGT;
  extern __shared__ int32_t sm_keys[];
  const int lane = lane_id();
  int32_t* keys = sm_keys + (threadIdx.x >> 5) * T;
  for (int s = lane; s < T; s += 32) keys[s] = kEmpty;
  __syncwarp();
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  // epoch-tagged keys need no per-row clearing (columns < 2^24)
  int epoch = B.cols < (1 << 24) ? 0 : kNoEpoch;
  for (int64_t idx = gw; idx < nrows; idx += nw) {
    const int32_t row = rows[idx];
    const int cnt = symbolic_row<LOGT, R32>(A, B, row, keys, epoch, flags);
    if (lane == 0) nnz_out[row] = cnt;
    if (epoch >= 0) next_row<LOGT>(keys, epoch);
  }
}

// One CTA per row; CTA-wide key table of `table` slots (power of two).
// Rows of this bin may become heavy in the numeric pass, so the per-tile
// counts of their output columns are recorded too.
__global__ void k_sym_block(DCsr A, DCsr B, const int32_t* rows, int64_t nrows, int log_table, int64_t slot_base,
                            int64_t* nnz_out, int32_t* big_slot, int32_t* tile_cnt, int ntiles, int* flags) {
  extern __shared__ int32_t sm_keys[];
  __shared__ int sh_cnt;
  const int table = 1 << log_table;
  const int lane = lane_id(), w = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int s = threadIdx.x; s < table; s += blockDim.x) sm_keys[s] = kEmpty;
  for (int64_t idx = blockIdx.x; idx < nrows; idx += gridDim.x) {
    const int32_t row = rows[idx];
    if (threadIdx.x == 0) sh_cnt = 0;
    __syncthreads();
    const int64_t s = A.rp[row], e = A.rp[row + 1];
    int cnt = 0;
    for (int64_t p = s + w; p < e; p += nwarps) {
      const int32_t k = A.col[p];
      const int64_t bs = B.rp[k], be = B.rp[k + 1];
      for (int64_t q = bs + lane; q < be; q += 32) {
        bool fresh;
        hash_insert(sm_keys, log_table, B.col[q], fresh, flags);
        cnt += fresh;
      }
    }
    cnt = warp_sum(cnt);
    if (lane == 0 && cnt) atomicAdd(&sh_cnt, cnt);
    __syncthreads();
    const int64_t slot = slot_base + idx;
    if (threadIdx.x == 0) {
      nnz_out[row] = sh_cnt;
      big_slot[row] = (int32_t)slot;
    }
    for (int t = threadIdx.x; t < table; t += blockDim.x) {
      int32_t key = sm_keys[t];
      if (key != kEmpty) {
        atomicAdd(&tile_cnt[slot * ntiles + (key >> kTileShift)], 1);
        sm_keys[t] = kEmpty;
      }
    }
    __syncthreads();
  }
}

// One CTA per row; a bitmap over the row's column span in shared memory
// (windows of `max_words` 32-bit words, a multiple of one tile).  Records
// the per-tile counts for the heavy numeric pass.
__global__ void k_sym_dense(DCsr A, DCsr B, const int32_t* rows, int64_t nrows, int max_words, int64_t slot_base,
                            int64_t* nnz_out, int32_t* big_slot, int32_t* tile_cnt, int ntiles, int* flags) {
  extern __shared__ uint32_t sm_bits[];
  __shared__ int sh_lo, sh_hi;
  __shared__ unsigned long long sh_total;
  const int lane = lane_id(), w = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int64_t idx = blockIdx.x; idx < nrows; idx += gridDim.x) {
    const int32_t row = rows[idx];
    const int64_t s = A.rp[row], e = A.rp[row + 1];
    if (threadIdx.x == 0) {
      sh_lo = 0x7fffffff;
      sh_hi = -1;
      sh_total = 0;
    }
    __syncthreads();
    // column span of the row's products
    int lo = 0x7fffffff, hi = -1;
    for (int64_t p = s + threadIdx.x; p < e; p += blockDim.x) {
      const int32_t k = A.col[p];
      const int64_t bs = B.rp[k], be = B.rp[k + 1];
      if (be > bs) {
        lo = min(lo, B.col[bs]);
        hi = max(hi, B.col[be - 1]);
      }
    }
    lo = warp_min(lo);
    hi = warp_max(hi);
    if (lane == 0) {
      atomicMin(&sh_lo, lo);
      atomicMax(&sh_hi, hi);
    }
    __syncthreads();
    const int span_lo = sh_lo & ~(kTileCols - 1), span_hi = sh_hi;
    const int64_t wcols = (int64_t)max_words * 32;
    for (int64_t w0 = span_lo; w0 <= span_hi; w0 += wcols) {
      const int64_t w1 = min(w0 + wcols, (int64_t)span_hi + 1);
      const int nwords = (int)((w1 - w0 + 31) >> 5);
      const int nwords_tiles = ((nwords + kTileWords - 1) / kTileWords) * kTileWords;
      for (int t = threadIdx.x; t < nwords_tiles; t += blockDim.x) sm_bits[t] = 0u;
      __syncthreads();
      for (int64_t p = s + w; p < e; p += nwarps) {
        const int32_t k = A.col[p];
        const int64_t bs = B.rp[k], be = B.rp[k + 1];
        for (int64_t q = bs + lane; q < be; q += 32) {
          const int32_t c = B.col[q];
          if (c >= w0 && c < w1) {
            const int off = (int)(c - w0);
            atomicOr(&sm_bits[off >> 5], 1u << (off & 31));
          }
        }
      }
      __syncthreads();
      // per-tile popcounts: one warp per tile
      const int ntile_w = nwords_tiles / kTileWords;
      for (int tw = w; tw < ntile_w; tw += nwarps) {
        int c = 0;
        for (int x = lane; x < kTileWords; x += 32) c += __popc(sm_bits[tw * kTileWords + x]);
        c = warp_sum(c);
        if (lane == 0) {
          const int64_t tile = (w0 >> kTileShift) + tw;
          if (c) {
            if (tile < ntiles) tile_cnt[(slot_base + idx) * ntiles + tile] = c;
            else raise_flag(flags, kFlagBadIndex);
            atomicAdd(&sh_total, (unsigned long long)c);
          }
        }
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      nnz_out[row] = (int64_t)sh_total;
      big_slot[row] = (int32_t)(slot_base + idx);
    }
    __syncthreads();
  }
}

// --------------------------------------------------------------------------
// Numeric pass: warp-level hash accumulator
// --------------------------------------------------------------------------

// Plain numeric pass: exact nnz known, writes straight into C.
template <int LOGT, bool R32>
__global__ void __launch_bounds__(512, 2) k_num_warp(DCsr A, DCsr B, const int32_t* rows, int64_t nrows,
                                                     const int64_t* c_rp, int32_t* c_col, float* c_val, int* flags) {
  constexpr int T = 1 << LOGT;
  extern __shared__ int32_t sm_tab[];
  const int lane = lane_id();
  int32_t* keys = sm_tab + (threadIdx.x >> 5) * numeric_words<LOGT>();
  float* vals = reinterpret_cast<float*>(keys + T);
  int32_t* list = keys + 2 * T;
  for (int s = lane; s < T; s += 32) keys[s] = kEmpty;
  __syncwarp();
  int epoch = B.cols < (1 << 24) ? 0 : kNoEpoch;
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t idx = gw; idx < nrows; idx += nw) {
    const int32_t row = rows[idx];
    const int64_t off = c_rp[row];
    numeric_row<LOGT, R32>(A, B, row, keys, vals, list, epoch, c_col + off, c_val + off, c_rp[row + 1] - off, flags);
  }
}

// Learned single-pass numeric: table sized by the predicted capacity; the
// row is written sorted into its slab slot.  Rows whose distinct count
// exceeds their capacity are queued for the exact re-run (nnz_out = -1).
template <int LOGT, bool R32>
__global__ void __launch_bounds__(512, 2) k_num_warp_learned(DCsr A, DCsr B, const int32_t* rows, int64_t nrows,
                                                             const int64_t* cap, const int64_t* slab_off,
                                                             int32_t* slab_col, float* slab_val, int64_t* nnz_out,
                                                             int32_t* retry_rows, unsigned long long* retry_count,
                                                             int* flags) {
  constexpr int T = 1 << LOGT;
  extern __shared__ int32_t sm_tab[];
  const int lane = lane_id();
  int32_t* keys = sm_tab + (threadIdx.x >> 5) * numeric_words<LOGT>();
  float* vals = reinterpret_cast<float*>(keys + T);
  int32_t* list = keys + 2 * T;
  for (int s = lane; s < T; s += 32) keys[s] = kEmpty;
  __syncwarp();
  int epoch = B.cols < (1 << 24) ? 0 : kNoEpoch;
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t idx = gw; idx < nrows; idx += nw) {
    const int32_t row = rows[idx];
    const int c = (int)cap[row];
    const int n = accumulate_row<LOGT, R32, true>(A, B, row, keys, vals, list, epoch, c, flags);
    if (n < 0) {
      // overflow: queue the row for the exact path
      if (lane == 0) {
        nnz_out[row] = -1;
        const unsigned long long pos = atomicAdd(retry_count, 1ull);
        retry_rows[pos] = row;
      }
    } else {
      const int64_t off = slab_off[row];
      emit_row<LOGT>(keys, vals, list, n, epoch, n, slab_col + off, slab_val + off);
      if (lane == 0) nnz_out[row] = n;
    }
    next_row<LOGT>(keys, epoch);
  }
}

// --------------------------------------------------------------------------
// Numeric pass: heavy rows, one warp per (row, column tile)
// --------------------------------------------------------------------------

// First position in B row [bs, be) whose column is >= c.
__device__ __forceinline__ int64_t lower_bound_col(const int32_t* col, int64_t bs, int64_t be, int64_t c) {
  while (bs < be) {
    const int64_t m = (bs + be) >> 1;
    if (col[m] < c) bs = m + 1;
    else be = m;
  }
  return bs;
}

// Blocked index of B: for every row k of B and every column tile t,
// bidx[k * (ntiles + 1) + t] = offset (from the row start) of the first
// entry whose column is >= t * kTileCols.  One warp per row; every slot is
// written exactly once.  Lets a heavy row's tile find the part of each B row
// it needs with two loads instead of two binary searches.
__global__ void k_build_blocked_index(DCsr B, int ntiles, int32_t* bidx) {
  const int lane = lane_id();
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t k = gw; k < B.rows; k += nw) {
    const int64_t s = B.rp[k], e = B.rp[k + 1];
    int32_t* out = bidx + k * (int64_t)(ntiles + 1);
    for (int64_t p = s + lane; p < e; p += 32) {
      const int tcur = B.col[p] >> kTileShift;
      const int tprev = p == s ? -1 : (B.col[p - 1] >> kTileShift);
      for (int t = tprev + 1; t <= tcur; ++t) out[t] = (int32_t)(p - s);
    }
    const int tlast = e > s ? (B.col[e - 1] >> kTileShift) : -1;
    for (int t = tlast + 1 + lane; t <= ntiles; t += 32) out[t] = (int32_t)(e - s);
  }
}

// Per heavy row: exclusive scan of its tile counts (warp per row slot).
__global__ void k_tile_offsets(const int32_t* heavy_rows, int64_t nheavy, const int32_t* big_slot,
                               const int32_t* tile_cnt, int ntiles, int32_t* tile_off) {
  const int lane = lane_id();
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t h = gw; h < nheavy; h += nw) {
    const int64_t slot = big_slot[heavy_rows[h]];
    int carry = 0;
    for (int t0 = 0; t0 < ntiles; t0 += 32) {
      const int t = t0 + lane;
      const int v = t < ntiles ? tile_cnt[slot * ntiles + t] : 0;
      const int inc = warp_incl_scan(v);
      if (t < ntiles) tile_off[slot * ntiles + t] = carry + inc - v;
      carry += __shfl_sync(kFull, inc, 31);
    }
  }
}

// One warp per (heavy row, 8192-column tile).  The tile's products are taken
// as one flattened stream in canonical order (k-major, then column), 32 per
// step; products of different k that hit the same column inside a step are
// grouped with __match_any_sync and added by the group's lowest lane in
// lane order, so every output entry sees its products in canonical order.
// Accumulator: dense tile of floats plus an occupancy bitmap.
__global__ void __launch_bounds__(kTileWarps * 32) k_num_tile(DCsr A, DCsr B, const int32_t* heavy_rows, int64_t nheavy,
                                                        const int32_t* big_slot, const int32_t* tile_cnt,
                                                        const int32_t* tile_off, int ntiles, const int64_t* c_rp,
                                                        int32_t* c_col, float* c_val, const int32_t* bidx,
                                                        unsigned long long* tile_counter, int* flags) {
  extern __shared__ uint32_t sm_tile[];
  const int lane = lane_id(), wib = threadIdx.x >> 5;
  float* acc = reinterpret_cast<float*>(sm_tile) + (size_t)wib * (kTileCols + kTileWords + 32);
  uint32_t* bits = reinterpret_cast<uint32_t*>(acc + kTileCols);
  float* stage = reinterpret_cast<float*>(bits + kTileWords);
  for (int s = lane; s < kTileCols; s += 32) acc[s] = 0.f;
  for (int s = lane; s < kTileWords; s += 32) bits[s] = 0u;
  __syncwarp();
  const int64_t total_tiles = nheavy * (int64_t)ntiles;
  for (;;) {
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(tile_counter, 1ull);
    t = __shfl_sync(kFull, t, 0);
    if ((int64_t)t >= total_tiles) break;
    const int64_t h = (int64_t)t / ntiles;
    const int tile = (int)((int64_t)t % ntiles);
    const int32_t row = heavy_rows[h];
    const int64_t slot = big_slot[row];
    const int want = tile_cnt[slot * ntiles + tile];
    if (want == 0) continue;
    const int64_t out = c_rp[row] + tile_off[slot * ntiles + tile];
    const int64_t c0 = (int64_t)tile << kTileShift;
    const int64_t c1 = c0 + kTileCols;
    const int64_t s = A.rp[row], e = A.rp[row + 1];
    for (int64_t base = s; base < e; base += 32) {
      const int64_t p = base + lane;
      int64_t bs = 0;
      int len = 0;
      float a = 0.f;
      if (p < e) {
        const int32_t k = A.col[p];
        a = A.val[p];
        int64_t rs = B.rp[k], re = B.rp[k + 1];
        if (ntiles > 1 && re > rs) {
          // narrow to the tile's columns
          if (bidx) {
            const int32_t* bi = bidx + (int64_t)k * (ntiles + 1) + tile;
            re = rs + bi[1];
            rs = rs + bi[0];
          } else {
            if (B.col[rs] < c0) rs = lower_bound_col(B.col, rs, re, c0);
            if (re > rs && B.col[re - 1] >= c1) re = lower_bound_col(B.col, rs, re, c1);
          }
        }
        bs = rs;
        len = (int)(re - rs);
      }
      const int incl = warp_incl_scan(len);
      const int total = __shfl_sync(kFull, incl, 31);
      const int excl = incl - len;
      for (int b0 = 0; b0 < total; b0 += 32) {
        const int tt = b0 + lane;
        const bool act = tt < total;
        const int src = warp_upper_bound(incl, act ? tt : total - 1);
        const int64_t sbs = __shfl_sync(kFull, bs, src);
        const int sex = __shfl_sync(kFull, excl, src);
        const float sa = __shfl_sync(kFull, a, src);
        int32_t j = -1 - lane;  // unique dummy for idle lanes
        float pr = 0.f;
        if (act) {
          const int64_t q = sbs + (tt - sex);
          j = B.col[q];
          pr = prod_rn(sa, B.val[q]);
        }
        stage[lane] = pr;
        const unsigned grp = __match_any_sync(kFull, j);
        __syncwarp();
        if (act && lane == __ffs(grp) - 1) {
          const int off = (int)(j - c0);
          if (off >= 0 && off < kTileCols) {
            float v = acc[off];
            unsigned g = grp;
            while (g) {
              const int m = __ffs(g) - 1;
              g &= g - 1;
              v = add_rn(v, stage[m]);
            }
            acc[off] = v;
            atomicOr(&bits[off >> 5], 1u << (off & 31));
          } else {
            raise_flag(flags, kFlagBadIndex);
          }
        }
        __syncwarp();
      }
    }
    // extract in column order: lane owns words [lane*8, lane*8+8)
    constexpr int kWPL = kTileWords / 32;
    int cnt = 0;
#pragma unroll
    for (int x = 0; x < kWPL; ++x) cnt += __popc(bits[lane * kWPL + x]);
    const int inc = warp_incl_scan(cnt);
    const int tot = __shfl_sync(kFull, inc, 31);
    if (tot != want && lane == 0) raise_flag(flags, kFlagCountDiff);
    int64_t pos = out + (inc - cnt);
    const int64_t lim = out + want;
#pragma unroll 1
    for (int x = 0; x < kWPL; ++x) {
      const int wi = lane * kWPL + x;
      uint32_t m = bits[wi];
      bits[wi] = 0u;
      while (m) {
        const int bi = __ffs(m) - 1;
        m &= m - 1;
        const int off = wi * 32 + bi;
        if (pos < lim) {
          c_col[pos] = (int32_t)(c0 + off);
          c_val[pos] = acc[off];
        }
        acc[off] = 0.f;
        ++pos;
      }
    }
    __syncwarp();
  }
}

// --------------------------------------------------------------------------
// Learned path helpers
// --------------------------------------------------------------------------

// Copies each light row that did not overflow (need_exact == 0) from the
// slab to its place in C; the row's length comes from C's row pointers.
__global__ void k_compact_rows(const int32_t* rows, int64_t nrows, const uint8_t* need_exact, const int64_t* slab_off,
                               const int32_t* slab_col, const float* slab_val, const int64_t* c_rp, int32_t* c_col,
                               float* c_val) {
  const int lane = lane_id();
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t idx = gw; idx < nrows; idx += nw) {
    const int32_t row = rows[idx];
    if (need_exact[row]) continue;
    const int64_t co = c_rp[row];
    const int64_t n = c_rp[row + 1] - co;
    const int64_t so = slab_off[row];
    for (int64_t t = lane; t < n; t += 32) {
      c_col[co + t] = slab_col[so + t];
      c_val[co + t] = slab_val[so + t];
    }
  }
}

// need_exact[retry[i]] = 1 for the rows queued by the learned pass.
__global__ void k_mark_rows(const int32_t* retry, const unsigned long long* count, uint8_t* need_exact) {
  const int64_t n = (int64_t)*count;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    need_exact[retry[i]] = 1;
}

// dst[r] = mask[r] ? src[r] : 0
__global__ void k_mask_key(const int64_t* src, const uint8_t* mask, int64_t rows, int64_t* dst) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x)
    dst[r] = mask[r] ? src[r] : 0;
}

// --------------------------------------------------------------------------
// Host launchers
// --------------------------------------------------------------------------

static int grid_for(int64_t work, int threads, int per_thread, int max_blocks) {
  int64_t b = (work * per_thread + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > max_blocks) b = max_blocks;
  return (int)b;
}

void launch_widen_rp(const int32_t* in, int64_t n, int64_t* out, const LaunchCtx& lc) {
  k_widen_rp<<<grid_for(n, 256, 1, lc.sms * 8), 256, 0, lc.stream>>>(in, n, out);
}

void launch_narrow_rp(const int64_t* in, int64_t n, int32_t* out, const LaunchCtx& lc) {
  k_narrow_rp<<<grid_for(n, 256, 1, lc.sms * 8), 256, 0, lc.stream>>>(in, n, out);
}

void launch_validate(const DCsr& M, int64_t nnz, int* flags, const LaunchCtx& lc) {
  if (M.rows == 0) return;
  k_validate<<<grid_for(M.rows, 256, 32, lc.sms * 16), 256, 0, lc.stream>>>(M, nnz, flags);
}

void launch_row_products(const DCsr& A, const DCsr& B, int64_t* prod, const LaunchCtx& lc) {
  if (A.rows == 0) return;
  k_row_products<<<grid_for(A.rows, 256, 32, lc.sms * 16), 256, 0, lc.stream>>>(A, B, prod);
}

void launch_sum(const int64_t* v, int64_t n, unsigned long long* out, const LaunchCtx& lc) {
  if (n == 0) return;
  k_sum_i64<<<grid_for(n, 256, 1, lc.sms * 4), 256, 0, lc.stream>>>(v, n, out);
}

void launch_binning(const int64_t* key, int64_t rows, int64_t cols, int mode, const BinParams& bp, uint8_t* bin_of_row,
                    int64_t* counts, int64_t* offsets, int64_t* cursors, int32_t* lists, const LaunchCtx& lc) {
  cudaMemsetAsync(counts, 0, sizeof(int64_t) * kNumBins, lc.stream);
  if (rows > 0)
    k_bin_count<<<grid_for(rows, 256, 1, lc.sms * 8), 256, 0, lc.stream>>>(key, rows, cols, mode, bp, bin_of_row,
                                                                              counts);
  k_bin_offsets<<<1, 32, 0, lc.stream>>>(counts, offsets, cursors);
  if (rows > 0)
    k_bin_scatter<<<grid_for(rows, 256, 1, lc.sms * 8), 256, 0, lc.stream>>>(bin_of_row, rows, cursors, lists);
}

int64_t scan_temp_elems(int64_t n) {
  int64_t total = 0;
  while (n > 1) {
    n = (n + kScanTile - 1) / kScanTile;
    total += n + 1;
  }
  return total + 1;
}

// Exclusive scan of in[0..n) into out[0..n) and total into out[n]
// (out has n+1 entries; may alias in).  tmp: scan_temp_elems(n) entries.
void launch_excl_scan(const int64_t* in, int64_t n, int64_t* out, int64_t* tmp, const LaunchCtx& lc) {
  if (n == 0) {
    cudaMemsetAsync(out, 0, sizeof(int64_t), lc.stream);
    return;
  }
  const int64_t nb = (n + kScanTile - 1) / kScanTile;
  // keep the last input element so out may alias in
  int64_t* last = tmp;
  cudaMemcpyAsync(last, in + n - 1, sizeof(int64_t), cudaMemcpyDeviceToDevice, lc.stream);
  if (nb == 1) {
    k_scan_apply<<<1, kScanThreads, 0, lc.stream>>>(in, n, nullptr, out);
  } else {
    int64_t* sums = tmp + 1;
    k_scan_reduce<<<(unsigned)nb, kScanThreads, 0, lc.stream>>>(in, n, sums);
    launch_excl_scan(sums, nb, sums, tmp + 1 + nb + 1, lc);
    k_scan_apply<<<(unsigned)nb, kScanThreads, 0, lc.stream>>>(in, n, sums, out);
  }
  k_store_total<<<1, 32, 0, lc.stream>>>(out + n - 1, last, out + n);
}

template <int LOGT, bool R32>
static void sym_warp_one(const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows, int64_t* nnz, int* flags,
                         const LaunchCtx& lc, int wpb) {
  const size_t smem = (size_t)wpb * (1 << LOGT) * sizeof(int32_t);
  cudaFuncSetAttribute(k_sym_warp<LOGT, R32>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sym_warp<LOGT, R32>, wpb * 32, smem);
  if (per_sm < 1) per_sm = 1;
  const int blocks = grid_for(nrows, wpb, 1, lc.sms * per_sm);
  k_sym_warp<LOGT, R32><<<blocks, wpb * 32, smem, lc.stream>>>(A, B, rows, nrows, nnz, flags);
}

void launch_sym_warp(int log_t, const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows, int64_t* nnz,
                     int* flags, const LaunchCtx& lc, int wpb) {
  if (nrows == 0) return;
  const int w = log_t >= 11 ? std::min(wpb, 8) : wpb;
#define SPG_SW(L)                                                                   \
  case L:                                                                           \
    if (B.rp32) sym_warp_one<L, true>(A, B, rows, nrows, nnz, flags, lc, w);        \
    else sym_warp_one<L, false>(A, B, rows, nrows, nnz, flags, lc, w);              \
    break;
  switch (log_t) {
    SPG_SW(5) SPG_SW(6) SPG_SW(7) SPG_SW(8) SPG_SW(9) SPG_SW(10) SPG_SW(11) SPG_SW(12)
    default: break;
  }
#undef SPG_SW
}

void launch_sym_block(const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows, int log_table,
                      int64_t slot_base, int64_t* nnz, int32_t* big_slot, int32_t* tile_cnt, int ntiles, int* flags,
                      const LaunchCtx& lc) {
  if (nrows == 0) return;
  const size_t smem = ((size_t)1 << log_table) * sizeof(int32_t);
  cudaFuncSetAttribute(k_sym_block, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sym_block, 512, smem);
  if (per_sm < 1) per_sm = 1;
  const int blocks = (int)std::min<int64_t>(nrows, (int64_t)lc.sms * per_sm);
  k_sym_block<<<blocks, 512, smem, lc.stream>>>(A, B, rows, nrows, log_table, slot_base, nnz, big_slot, tile_cnt,
                                                ntiles, flags);
}

void launch_sym_dense(const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows, int64_t slot_base,
                      int64_t* nnz, int32_t* big_slot, int32_t* tile_cnt, int ntiles, int* flags,
                      const LaunchCtx& lc) {
  if (nrows == 0) return;
  const int max_words = kDenseWindowWords;
  const size_t smem = (size_t)max_words * sizeof(uint32_t);
  cudaFuncSetAttribute(k_sym_dense, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int blocks = (int)std::min<int64_t>(nrows, (int64_t)lc.sms);
  k_sym_dense<<<blocks, 1024, smem, lc.stream>>>(A, B, rows, nrows, max_words, slot_base, nnz, big_slot, tile_cnt,
                                                 ntiles, flags);
}

template <int LOGT, bool R32>
static void num_warp_one(const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows, const int64_t* c_rp,
                         int32_t* c_col, float* c_val, int* flags, const LaunchCtx& lc, int wpb) {
  const size_t smem = (size_t)wpb * numeric_words<LOGT>() * 4;
  cudaFuncSetAttribute(k_num_warp<LOGT, R32>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_num_warp<LOGT, R32>, wpb * 32, smem);
  if (per_sm < 1) per_sm = 1;
  const int blocks = grid_for(nrows, wpb, 1, lc.sms * per_sm);
  k_num_warp<LOGT, R32><<<blocks, wpb * 32, smem, lc.stream>>>(A, B, rows, nrows, c_rp, c_col, c_val, flags);
}

static int wpb_for(int log_t, int wpb) {
  // keep a CTA's tables within 96 KB
  const int per_warp = (1 << log_t) * 12;
  int lim = (96 * 1024) / per_warp;
  if (lim < 1) lim = 1;
  return std::max(1, std::min(wpb, lim));
}

void launch_num_warp(int log_t, const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows,
                     const int64_t* c_rp, int32_t* c_col, float* c_val, int* flags, const LaunchCtx& lc, int wpb) {
  if (nrows == 0) return;
  const int w = wpb_for(log_t, wpb);
#define SPG_NW(L)                                                                          \
  case L:                                                                                  \
    if (B.rp32) num_warp_one<L, true>(A, B, rows, nrows, c_rp, c_col, c_val, flags, lc, w); \
    else num_warp_one<L, false>(A, B, rows, nrows, c_rp, c_col, c_val, flags, lc, w);       \
    break;
  switch (log_t) {
    SPG_NW(5) SPG_NW(6) SPG_NW(7) SPG_NW(8) SPG_NW(9) SPG_NW(10) SPG_NW(11) SPG_NW(12)
    default: break;
  }
#undef SPG_NW
}

template <int LOGT, bool R32>
static void num_warp_learned_one(const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows,
                                 const int64_t* cap, const int64_t* slab_off, int32_t* slab_col, float* slab_val,
                                 int64_t* nnz_out, int32_t* retry_rows, unsigned long long* retry_count, int* flags,
                                 const LaunchCtx& lc, int wpb) {
  const size_t smem = (size_t)wpb * numeric_words<LOGT>() * 4;
  cudaFuncSetAttribute(k_num_warp_learned<LOGT, R32>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_num_warp_learned<LOGT, R32>, wpb * 32, smem);
  if (per_sm < 1) per_sm = 1;
  const int blocks = grid_for(nrows, wpb, 1, lc.sms * per_sm);
  k_num_warp_learned<LOGT, R32><<<blocks, wpb * 32, smem, lc.stream>>>(A, B, rows, nrows, cap, slab_off, slab_col,
                                                                        slab_val, nnz_out, retry_rows, retry_count,
                                                                        flags);
}

void launch_num_warp_learned(int log_t, const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows,
                             const int64_t* cap, const int64_t* slab_off, int32_t* slab_col, float* slab_val,
                             int64_t* nnz_out, int32_t* retry_rows, unsigned long long* retry_count, int* flags,
                             const LaunchCtx& lc, int wpb) {
  if (nrows == 0) return;
  const int w = wpb_for(log_t, wpb);
#define SPG_NWL(L)                                                                                             \
  case L:                                                                                                      \
    if (B.rp32)                                                                                                \
      num_warp_learned_one<L, true>(A, B, rows, nrows, cap, slab_off, slab_col, slab_val, nnz_out, retry_rows, \
                                    retry_count, flags, lc, w);                                                \
    else                                                                                                       \
      num_warp_learned_one<L, false>(A, B, rows, nrows, cap, slab_off, slab_col, slab_val, nnz_out,            \
                                     retry_rows, retry_count, flags, lc, w);                                   \
    break;
  switch (log_t) {
    SPG_NWL(5) SPG_NWL(6) SPG_NWL(7) SPG_NWL(8) SPG_NWL(9) SPG_NWL(10) SPG_NWL(11) SPG_NWL(12)
    default: break;
  }
#undef SPG_NWL
}

void launch_tile_offsets(const int32_t* heavy_rows, int64_t nheavy, const int32_t* big_slot, const int32_t* tile_cnt,
                         int ntiles, int32_t* tile_off, const LaunchCtx& lc) {
  if (nheavy == 0) return;
  k_tile_offsets<<<grid_for(nheavy, 256, 32, lc.sms * 8), 256, 0, lc.stream>>>(heavy_rows, nheavy, big_slot, tile_cnt,
                                                                                ntiles, tile_off);
}

void launch_build_blocked_index(const DCsr& B, int ntiles, int32_t* bidx, const LaunchCtx& lc) {
  if (B.rows == 0) return;
  k_build_blocked_index<<<grid_for(B.rows, 256, 32, lc.sms * 16), 256, 0, lc.stream>>>(B, ntiles, bidx);
}

void launch_num_tile(const DCsr& A, const DCsr& B, const int32_t* heavy_rows, int64_t nheavy, const int32_t* big_slot,
                     const int32_t* tile_cnt, const int32_t* tile_off, int ntiles, const int64_t* c_rp,
                     int32_t* c_col, float* c_val, const int32_t* bidx, unsigned long long* tile_counter, int* flags,
                     const LaunchCtx& lc) {
  if (nheavy == 0) return;
  const size_t smem = (size_t)kTileWarps * (kTileCols + kTileWords + 32) * 4;
  cudaFuncSetAttribute(k_num_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_num_tile, kTileWarps * 32, smem);
  if (per_sm < 1) per_sm = 1;
  const int64_t tiles = nheavy * (int64_t)ntiles;
  const int blocks = (int)std::min<int64_t>((tiles + kTileWarps - 1) / kTileWarps, (int64_t)lc.sms * per_sm);
  cudaMemsetAsync(tile_counter, 0, sizeof(unsigned long long), lc.stream);
  k_num_tile<<<blocks, kTileWarps * 32, smem, lc.stream>>>(A, B, heavy_rows, nheavy, big_slot, tile_cnt, tile_off,
                                                           ntiles, c_rp, c_col, c_val, bidx, tile_counter, flags);
}

void launch_compact_rows(const int32_t* rows, int64_t nrows, const uint8_t* need_exact, const int64_t* slab_off,
                         const int32_t* slab_col, const float* slab_val, const int64_t* c_rp, int32_t* c_col,
                         float* c_val, const LaunchCtx& lc) {
  if (nrows == 0) return;
  k_compact_rows<<<grid_for(nrows, 256, 32, lc.sms * 16), 256, 0, lc.stream>>>(rows, nrows, need_exact, slab_off,
                                                                                slab_col, slab_val, c_rp, c_col, c_val);
}

void launch_mark_rows(const int32_t* retry, const unsigned long long* count, uint8_t* need_exact, const LaunchCtx& lc) {
  k_mark_rows<<<lc.sms, 256, 0, lc.stream>>>(retry, count, need_exact);
}

void launch_mask_key(const int64_t* src, const uint8_t* mask, int64_t rows, int64_t* dst, const LaunchCtx& lc) {
  if (rows == 0) return;
  k_mask_key<<<grid_for(rows, 256, 1, lc.sms * 8), 256, 0, lc.stream>>>(src, mask, rows, dst);
}

}  // namespace spg
