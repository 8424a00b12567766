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
#include <atomic>

#include "common.cuh"
#include "kernels.hpp"
#include "block_row.cuh"
#include "tile.cuh"
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
      // a row has at most u distinct columns, so a table of 1.25 u slots
      // stays at most 4/5 full, and usually far below (125 columns from
      // 729 products on the stencil: 2^10 slots instead of 2^11 at 2/3)
      int64_t need = u + (u >> 2) + 1;
      int lg = ceil_log2_i64(need);
      if (lg < kMinLogT) lg = kMinLogT;
      if (lg > bp.warp_log_max) lg = bp.warp_log_max;
      return lg - kMinLogT;
    }
    if (u <= bp.block_cap) return kBinBlock;
    return kBinDense;
  }
  if (key <= 0) return kBinEmpty;
  const bool warp_ok = key <= bp.warp_cap;
  if (!(warp_ok && key <= bp.block_min)) {
    // the CTA-wide hash bins
    if (key <= bp.blk_small_cap) return kBinBlock;
    if (key <= bp.blk_large_cap) return kBinDense;
  }
  if (warp_ok) {
    int64_t need = (int64_t)ceilf((float)key / bp.max_load);
    int lg = ceil_log2_i64(need);
    if (lg < kMinLogT) lg = kMinLogT;
    if (lg > bp.warp_log_max) lg = bp.warp_log_max;
    return lg - kMinLogT;
  }
  return kBinHeavy;
}

// Histogram of bins (warp-aggregated atomics).
// Histogram of bins: counts per block in shared memory, then one global
// atomic per (block, bin) -- rows of one matrix mostly share a bin, so
// per-warp global atomics would queue on one address.
__global__ void k_bin_count(const int64_t* key, int64_t rows, int64_t cols, int mode, BinParams bp,
                            uint8_t* bin_of_row, int64_t* counts) {
  __shared__ unsigned sh_cnt[kNumBins];
  if (threadIdx.x < kNumBins) sh_cnt[threadIdx.x] = 0;
  __syncthreads();
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
    const int b = bin_of(key[r], cols, mode, bp);
    bin_of_row[r] = (uint8_t)b;
    atomicAdd(&sh_cnt[b], 1u);
  }
  __syncthreads();
  if (threadIdx.x < kNumBins && sh_cnt[threadIdx.x])
    atomicAdd((unsigned long long*)&counts[threadIdx.x], (unsigned long long)sh_cnt[threadIdx.x]);
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

// Scatter row ids into per-bin lists: per tile of blockDim.x rows, ranks
// inside the block from shared-memory counters, one global atomic per (tile,
// bin) for the block's range.  Order within a bin only affects scheduling,
// never results.
__global__ void k_bin_scatter(const uint8_t* bin_of_row, int64_t rows, int64_t* cursors, int32_t* lists) {
  __shared__ unsigned sh_cnt[kNumBins];
  __shared__ unsigned long long sh_base[kNumBins];
  for (int64_t r0 = blockIdx.x * (int64_t)blockDim.x; r0 < rows; r0 += (int64_t)gridDim.x * blockDim.x) {
    if (threadIdx.x < kNumBins) sh_cnt[threadIdx.x] = 0;
    __syncthreads();
    const int64_t r = r0 + threadIdx.x;
    int b = -1;
    unsigned local = 0;
    if (r < rows) {
      b = bin_of_row[r];
      local = atomicAdd(&sh_cnt[b], 1u);
    }
    __syncthreads();
    if (threadIdx.x < kNumBins && sh_cnt[threadIdx.x])
      sh_base[threadIdx.x] = atomicAdd((unsigned long long*)&cursors[threadIdx.x],
                                       (unsigned long long)sh_cnt[threadIdx.x]);
    __syncthreads();
    if (b >= 0) lists[sh_base[b] + local] = (int32_t)r;
    __syncthreads();
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

// Second pass of the two-kernel scan (at most kScanTile blocks): each block
// sums the block totals before it, scans its tile on top, and the last block
// also writes the grand total to out[n].  out may alias in.
__global__ void __launch_bounds__(kScanThreads) k_scan_apply_sums(const int64_t* in, int64_t n, const int64_t* sums,
                                                                    int64_t* out) {
  __shared__ int64_t sh[33];
  // prefix of the block sums before this block
  int64_t ps = 0;
  for (int64_t i = threadIdx.x; i < blockIdx.x; i += blockDim.x) ps += sums[i];
  int64_t tot_before;
  block_excl_scan(ps, sh, tot_before);
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int64_t v[kScanItems];
  int64_t s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    v[i] = (base + i < n) ? in[base + i] : 0;
    s += v[i];
  }
  int64_t tot;
  int64_t pre = block_excl_scan(s, sh, tot) + tot_before;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (base + i < n) out[base + i] = pre;
    pre += v[i];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = tot_before + tot;
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

// Visits every product column of `row` with the whole CTA (NTHR threads), in
// no particular order: f(c).  A's row is taken NTHR entries at a time; a
// CTA-wide exclusive scan of their B-row lengths goes to shared memory
// (sh_excl[NTHR + 1], sh_bs[NTHR]) and the chunk's product stream is split
// evenly among the warps.  A warp walks its share 32 products per step: a
// window of the next 32 segment starts (one shared load per lane) and a
// shuffle search give each lane its segment, so hub rows of B are spread
// over every warp and short rows leave no lane idle.
template <int NTHR, bool R32, typename F>
__device__ __forceinline__ void cta_for_each_product(const DCsr& A, const DCsr& B, int32_t row,
                                                     typename RowOff<R32>::T* sh_excl,
                                                     typename RowOff<R32>::T* sh_bs,
                                                     typename RowOff<R32>::T* sh_wsum, F&& f) {
  using Off = typename RowOff<R32>::T;
  constexpr int NW = NTHR / 32;
  const int tid = threadIdx.x, lane = lane_id(), w = tid >> 5;
  const int64_t s = A.rp[row], e = A.rp[row + 1];
  for (int64_t c0 = s; c0 < e; c0 += NTHR) {
    const int64_t p = c0 + tid;
    Off bs = 0, len = 0;
    if (p < e) {
      const int32_t k = A.col[p];
      bs = RowOff<R32>::at(B, k);
      len = RowOff<R32>::at(B, k + 1) - bs;
    }
    const Off incl = warp_incl_scan(len);
    if (lane == 31) sh_wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
      const Off v = lane < NW ? sh_wsum[lane] : 0;
      const Off iv = warp_incl_scan(v);
      if (lane < NW) sh_wsum[lane] = iv - v;
      if (lane == NW - 1) sh_wsum[NW] = iv;
    }
    __syncthreads();
    sh_excl[tid] = incl - len + sh_wsum[w];
    sh_bs[tid] = bs;
    const int cnt = (int)min((int64_t)NTHR, e - c0);
    const Off total = sh_wsum[NW];
    if (tid == 0) sh_excl[cnt] = total;  // sentinel after the last entry
    __syncthreads();
    const Off lo = (Off)((int64_t)total * w / NW), hi = (Off)((int64_t)total * (w + 1) / NW);
    if (lo < hi) {
      // segment holding `lo`: sh_excl[i0] <= lo < sh_excl[i0 + 1]
      int i0 = 0, i1 = cnt;
      while (i1 - i0 > 1) {
        const int mid = (i0 + i1) >> 1;
        if (sh_excl[mid] <= lo) i0 = mid;
        else i1 = mid;
      }
      int kc = i0;
      for (Off pos = lo; pos < hi;) {
        // starts of the segments after kc, kc + 1, ..., kc + 31
        const int wi = kc + 1 + lane;
        const Off nxt = wi <= cnt ? sh_excl[wi] : (Off)(R32 ? 0x7fffffff : INT64_MAX);
        // the next 32 products all inside segment kc (long rows of B): no search
        const Off seg_end = __shfl_sync(kFull, nxt, 0);
        if (pos >= sh_excl[kc] && pos + 32 <= seg_end && pos + 32 <= hi) {
          f(B.col[sh_bs[kc] + (pos - sh_excl[kc]) + (Off)lane]);
          pos += 32;
          continue;
        }
        const Off wend = __shfl_sync(kFull, nxt, 31);
        if (wend <= pos) {
          // more than 31 empty segments in a row: slide the window on
          kc += 31;
          continue;
        }
        const Off lim = wend < hi ? wend : hi;
        const Off x = pos + (Off)lane;
        const bool act = x < lim;
        const int l = warp_upper_bound_t<Off>(nxt, act ? x : pos);
        const int i = kc + l;
        if (act) f(B.col[sh_bs[i] + (x - sh_excl[i])]);
        const int adv = (int)min((Off)32, lim - pos);
        kc = __shfl_sync(kFull, i, adv - 1);
        pos += adv;
      }
    }
    __syncthreads();
  }
}

// One CTA per row; CTA-wide key table of `table` slots (power of two).
// Rows of this bin may become heavy in the numeric pass, so the per-tile
// counts of their output columns are recorded too.
constexpr int kSymBlockThreads = 512;
template <bool R32>
__global__ void __launch_bounds__(kSymBlockThreads) k_sym_block(DCsr A, DCsr B, const int32_t* rows, int64_t nrows,
                                                                int log_table, int64_t slot_base, int64_t* nnz_out,
                                                                int32_t* big_slot, int32_t* tile_cnt, int ntiles,
                                                                int* flags) {
  using Off = typename RowOff<R32>::T;
  extern __shared__ int32_t sm_keys[];
  __shared__ Off sh_excl[kSymBlockThreads + 1], sh_bs[kSymBlockThreads], sh_wsum[kSymBlockThreads / 32 + 1];
  __shared__ int sh_cnt;
  const int table = 1 << log_table;
  const int lane = lane_id();
  for (int s = threadIdx.x; s < table; s += blockDim.x) sm_keys[s] = kEmpty;
  for (int64_t idx = blockIdx.x; idx < nrows; idx += gridDim.x) {
    const int32_t row = rows[idx];
    if (threadIdx.x == 0) sh_cnt = 0;
    __syncthreads();
    int cnt = 0;
    cta_for_each_product<kSymBlockThreads, R32>(A, B, row, sh_excl, sh_bs, sh_wsum, [&](int32_t c) {
      bool fresh;
      hash_insert(sm_keys, log_table, c, fresh, flags);
      cnt += fresh;
    });
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
constexpr int kSymDenseThreads = 1024;
template <bool R32>
__global__ void __launch_bounds__(kSymDenseThreads) k_sym_dense(DCsr A, DCsr B, const int32_t* rows, int64_t nrows,
                                                                int max_words, int64_t slot_base, int64_t* nnz_out,
                                                                int32_t* big_slot, int32_t* tile_cnt, int ntiles,
                                                                int* flags) {
  using Off = typename RowOff<R32>::T;
  extern __shared__ uint32_t sm_bits[];
  __shared__ Off sh_excl[kSymDenseThreads + 1], sh_bs[kSymDenseThreads], sh_wsum[kSymDenseThreads / 32 + 1];
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
      const Off bs = RowOff<R32>::at(B, k), be = RowOff<R32>::at(B, k + 1);
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
      cta_for_each_product<kSymDenseThreads, R32>(A, B, row, sh_excl, sh_bs, sh_wsum, [&](int32_t c) {
        if (c >= w0 && c < w1) {
          const int off = (int)(c - w0);
          atomicOr(&sm_bits[off >> 5], 1u << (off & 31));
        }
      });
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

// Plain numeric pass: exact nnz known, writes straight into C.  With the
// row products `prod` given, rows that esc_wanted() take esc_row.  56
// registers (36 resident warps per SM at 2^9-slot tables) also with the
// expand-sort-fold code inlined, which would take 64 unbounded.
template <int LOGT, bool R32>
__global__ void __maxnreg__(56) k_num_warp(DCsr A, DCsr B, const int32_t* rows, int64_t nrows,
                                                     const int64_t* c_rp, int32_t* c_col, float* c_val,
                                                     const int64_t* prod, int esc_min, int* flags) {
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
  const int ecap = esc_capacity(numeric_words<LOGT>());
  for (int64_t idx = gw; idx < nrows; idx += nw) {
    const int32_t row = rows[idx];
    const int64_t off = c_rp[row];
    const int64_t want = c_rp[row + 1] - off;
    if (prod) {
      const int64_t p = prod[row];
      if (esc_wanted(p, want, esc_min, ecap)) {
        const int n = esc_row<R32>(A, B, row, (int)p, keys, want, c_col + off, c_val + off);
        esc_wipe(keys, T);
        if (n >= 0) {
          if (n != want && lane == 0) raise_flag(flags, kFlagCountDiff);
          continue;
        }
      }
    }
    numeric_row<LOGT, R32>(A, B, row, keys, vals, list, epoch, c_col + off, c_val + off, want, flags);
  }
}

// Learned single-pass numeric: table sized by the predicted capacity; the
// row is written sorted into its slab slot.  Rows whose distinct count
// exceeds their capacity are queued for the exact re-run (nnz_out = -1).
// Rows that esc_wanted() (at their capacity) take esc_row.
template <int LOGT, bool R32>
__global__ void __maxnreg__(56) k_num_warp_learned(DCsr A, DCsr B, const int32_t* rows, int64_t nrows,
                                                             const int64_t* cap, const int64_t* slab_off,
                                                             int32_t* slab_col, float* slab_val, int64_t* nnz_out,
                                                             int32_t* retry_rows, unsigned long long* retry_count,
                                                             const int64_t* prod, int esc_min, int* flags) {
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
  const int ecap = esc_capacity(numeric_words<LOGT>());
  for (int64_t idx = gw; idx < nrows; idx += nw) {
    const int32_t row = rows[idx];
    const int c = (int)cap[row];
    if (prod) {
      const int64_t p = prod[row];
      if (esc_wanted(p, c, esc_min, ecap)) {
        const int64_t off = slab_off[row];
        const int n = esc_row<R32>(A, B, row, (int)p, keys, c, slab_col + off, slab_val + off);
        esc_wipe(keys, T);
        if (n >= 0) {
          if (lane == 0) {
            if (n > c) {
              nnz_out[row] = -1;
              retry_rows[atomicAdd(retry_count, 1ull)] = row;
            } else {
              nnz_out[row] = n;
            }
          }
          continue;
        }
      }
    }
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
      emit_row<LOGT>(keys, vals, list, n, epoch, n, slab_col + off, slab_val + off, false);
      if (lane == 0) nnz_out[row] = n;
    }
    next_row<LOGT>(keys, epoch);
  }
}

// --------------------------------------------------------------------------
// Numeric pass: CTA-wide hash accumulator (block_row.cuh)
// --------------------------------------------------------------------------

// Plain numeric pass, one CTA per row of the bin: exact nnz known, written
// straight into C.
template <int LOGT, bool R32>
__global__ void __launch_bounds__(kBlkThreads) k_num_block(DCsr A, DCsr B, const int32_t* rows, int64_t nrows,
                                                           const int64_t* c_rp, int32_t* c_col, float* c_val,
                                                           int* flags) {
  constexpr int T = 1 << LOGT;
  extern __shared__ int32_t sm_blk[];
  __shared__ BlockScratch sc;
  int32_t* keys = sm_blk;
  float* vals = reinterpret_cast<float*>(sm_blk + T);
  uint32_t* own = reinterpret_cast<uint32_t*>(sm_blk + 2 * T);
  for (int64_t idx = blockIdx.x; idx < nrows; idx += gridDim.x) {
    const int32_t row = rows[idx];
    const int64_t off = c_rp[row];
    const int64_t want = c_rp[row + 1] - off;
    const int lg = cta_table_log(want, LOGT);
    const int n = cta_accumulate_row<LOGT, R32, false>(A, B, row, keys, vals, own, sc, 0, flags, lg);
    if (n != want && threadIdx.x == 0) raise_flag(flags, kFlagCountDiff);
    cta_emit_row<LOGT>(keys, vals, own, sc, n, want, c_col + off, c_val + off, lg);
  }
}

// Learned single pass, one CTA per row: the row is written sorted into its
// slab slot; a row with more distinct columns than its capacity is queued
// for the exact re-run (nnz_out = -1).
template <int LOGT, bool R32>
__global__ void __launch_bounds__(kBlkThreads) k_num_block_learned(DCsr A, DCsr B, const int32_t* rows,
                                                                   int64_t nrows, const int64_t* cap,
                                                                   const int64_t* slab_off, int32_t* slab_col,
                                                                   float* slab_val, int64_t* nnz_out,
                                                                   int32_t* retry_rows,
                                                                   unsigned long long* retry_count, int* flags) {
  constexpr int T = 1 << LOGT;
  extern __shared__ int32_t sm_blk[];
  __shared__ BlockScratch sc;
  int32_t* keys = sm_blk;
  float* vals = reinterpret_cast<float*>(sm_blk + T);
  uint32_t* own = reinterpret_cast<uint32_t*>(sm_blk + 2 * T);
  for (int64_t idx = blockIdx.x; idx < nrows; idx += gridDim.x) {
    const int32_t row = rows[idx];
    const int64_t c = cap[row];
    const int lg = cta_table_log(c, LOGT);
    const int n = cta_accumulate_row<LOGT, R32, true>(A, B, row, keys, vals, own, sc, c, flags, lg);
    if (n < 0) {
      if (threadIdx.x == 0) {
        nnz_out[row] = -1;
        const unsigned long long pos = atomicAdd(retry_count, 1ull);
        retry_rows[pos] = row;
      }
      continue;
    }
    const int64_t off = slab_off[row];
    cta_emit_row<LOGT>(keys, vals, own, sc, n, n, slab_col + off, slab_val + off, lg);
    if (threadIdx.x == 0) nnz_out[row] = n;
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

// Tile occupancy of B from its blocked index: bit t of tocc[k * words + t /
// 32] is set when B row k has an entry in column tile t.  One warp per row,
// every word written.  ceil(tiles / 32) words per row (64 MB for 2^20 rows and
// 512 tiles, small enough to stay in L2), so a heavy row's tile rejects the
// rows of B that miss it with one cached load instead of four.
__global__ void k_build_tile_occupancy(int64_t rows, const int32_t* bidx, int ntiles, int words, uint32_t* tocc) {
  const int lane = lane_id();
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t k = gw; k < rows; k += nw) {
    const int32_t* bi = bidx + k * (int64_t)(ntiles + 1);
    for (int w = 0; w < words; ++w) {
      const int t = w * 32 + lane;
      const bool has = t < ntiles && bi[t + 1] > bi[t];
      const unsigned m = __ballot_sync(kFull, has);
      if (lane == 0) tocc[k * (int64_t)words + w] = m;
    }
  }
}

// Value-only recompute (structure of C given): per-row lengths of C and,
// for the rows of the heavy bin, their slot and per-tile entry counts taken
// from C's sorted columns.

// len[r] = rp[r + 1] - rp[r]
__global__ void k_row_lengths(const int64_t* rp, int64_t rows, int64_t* len) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x)
    len[r] = rp[r + 1] - rp[r];
}

// big_slot[heavy_rows[h]] = h; one warp per heavy row then counts the row's
// entries per column tile (tile_cnt[h * ntiles + t], zeroed beforehand) from
// the run starts of its sorted columns: a tile's count is the distance from
// its first entry to the next tile's first entry (or the row end).
__global__ void k_tile_counts_from_cols(const int32_t* heavy_rows, int64_t nheavy, const int64_t* c_rp,
                                        const int32_t* c_col, int ntiles, int32_t* big_slot, int32_t* tile_cnt,
                                        int* flags) {
  const int lane = lane_id();
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t h = gw; h < nheavy; h += nw) {
    const int32_t row = heavy_rows[h];
    if (lane == 0) big_slot[row] = (int32_t)h;
    int32_t* cnt = tile_cnt + h * ntiles;
    const int64_t s = c_rp[row], e = c_rp[row + 1];
    int pend_t = -1;     // tile whose run is still open (uniform)
    int64_t pend_p = 0;  // its first entry
    for (int64_t base = s; base < e; base += 32) {
      const int64_t p = base + lane;
      int t = -1;
      bool first = false;
      if (p < e) {
        t = c_col[p] >> kTileShift;
        first = p == s || (c_col[p - 1] >> kTileShift) != t;
        if ((unsigned)t >= (unsigned)ntiles) {
          raise_flag(flags, kFlagBadIndex);
          first = false;
        }
      }
      const unsigned fm = __ballot_sync(kFull, first);
      if (fm) {
        const int lead = __ffs(fm) - 1;
        if (pend_t >= 0 && lane == 0) cnt[pend_t] = (int32_t)(base + lead - pend_p);
        if (first) {
          const unsigned later = fm & ~((2u << lane) - 1u);
          if (later) cnt[t] = (int32_t)(__ffs(later) - 1 - lane);
        }
        const int last = 31 - __clz(fm);
        pend_t = __shfl_sync(kFull, t, last);
        pend_p = base + last;
      }
    }
    if (pend_t >= 0 && lane == 0) cnt[pend_t] = (int32_t)(e - pend_p);
  }
}

// Per heavy row: exclusive scan of its tile counts (warp per row slot) and,
// when nz_cnt is given, the number of its tiles with output entries.
__global__ void k_tile_offsets(const int32_t* heavy_rows, int64_t nheavy, const int32_t* big_slot,
                               const int32_t* tile_cnt, int ntiles, int32_t* tile_off, int64_t* nz_cnt) {
  const int lane = lane_id();
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t h = gw; h < nheavy; h += nw) {
    const int64_t slot = big_slot[heavy_rows[h]];
    int carry = 0, nz = 0;
    for (int t0 = 0; t0 < ntiles; t0 += 32) {
      const int t = t0 + lane;
      const int v = t < ntiles ? tile_cnt[slot * ntiles + t] : 0;
      const int inc = warp_incl_scan(v);
      if (t < ntiles) tile_off[slot * ntiles + t] = carry + inc - v;
      carry += __shfl_sync(kFull, inc, 31);
      nz += __popc(__ballot_sync(kFull, v > 0));
    }
    if (nz_cnt && lane == 0) nz_cnt[h] = nz;
  }
}

// The (heavy row, tile) units with output entries, as h * ntiles + tile,
// row after row from the exclusive scan nz_off of the per-row counts.
__global__ void k_tile_worklist(const int32_t* heavy_rows, int64_t nheavy, const int32_t* big_slot,
                                const int32_t* tile_cnt, int ntiles, const int64_t* nz_off, int64_t* work) {
  const int lane = lane_id();
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t h = gw; h < nheavy; h += nw) {
    const int64_t slot = big_slot[heavy_rows[h]];
    int64_t pos = nz_off[h];
    for (int t0 = 0; t0 < ntiles; t0 += 32) {
      const int t = t0 + lane;
      const bool nz = t < ntiles && tile_cnt[slot * ntiles + t] > 0;
      const unsigned m = __ballot_sync(kFull, nz);
      if (nz) work[pos + __popc(m & ((1u << lane) - 1u))] = h * (int64_t)ntiles + t;
      pos += __popc(m);
    }
  }
}

// Segments of at least this many entries are accumulated by the whole warp
// without collision checks; shorter ones are packed.
#ifndef SPG_TILE_LONG_SEG
#define SPG_TILE_LONG_SEG 16
#endif
constexpr int kTileLongSeg = SPG_TILE_LONG_SEG;

// One segment (the part of B row k inside the tile, scaled by a).  Its
// columns are distinct, so its products need no ordering among themselves:
// lanes take 128 entries per round, issue all loads, then all accumulator
// reads, then all writes.  `c0` is the tile's first column.
template <typename Off>
__device__ __forceinline__ void tile_segment(const DCsr& B, Off bs, int len, float a, int32_t c0, float* acc,
                                             uint32_t* bits, int* flags) {
  const int lane = lane_id();
  if (len <= 32) {
    // one round: a single load per lane
    if (lane < len) {
      const int32_t off = B.col[bs + lane] - c0;
      const float pr = prod_rn(a, B.val[bs + lane]);
      if ((uint32_t)off < (uint32_t)kTileCols) {
        acc[off] = add_rn(acc[off], pr);
        atomicOr(&bits[off >> 5], 1u << (off & 31));
      } else {
        raise_flag(flags, kFlagBadIndex);
      }
    }
    return;
  }
  for (int q0 = 0; q0 < len; q0 += 4 * 32) {
    int32_t off[4];
    float pr[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int q = q0 + u * 32 + lane;
      off[u] = -1;
      pr[u] = 0.f;
      if (q < len) {
        off[u] = B.col[bs + q] - c0;
        pr[u] = prod_rn(a, B.val[bs + q]);
      }
    }
    float cur[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) cur[u] = (uint32_t)off[u] < (uint32_t)kTileCols ? acc[off[u]] : 0.f;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if ((uint32_t)off[u] < (uint32_t)kTileCols) {
        acc[off[u]] = add_rn(cur[u], pr[u]);
        atomicOr(&bits[off[u] >> 5], 1u << (off[u] & 31));
      } else if (q0 + u * 32 + lane < len) {
        raise_flag(flags, kFlagBadIndex);
      }
    }
  }
}

// Segments of lanes [lo, hi) (all shorter than kTileLongSeg) taken as one
// stream in canonical order (segment-major), 32 products per step, two steps
// loaded at a time.  Products of one step that hit the same column (from
// different segments) are grouped with __match_any_sync and added by the
// group's lowest lane in lane order; steps without such a collision commit
// directly.
template <typename Off>
__device__ __forceinline__ void tile_packed(const DCsr& B, Off bs, int len, float a, int lo, int hi, int32_t c0,
                                            float* acc, uint32_t* bits, float* stage, int* flags) {
  const int lane = lane_id();
  const int lr = (lane >= lo && lane < hi) ? len : 0;
  const int incl = warp_incl_scan(lr);
  const int total = __shfl_sync(kFull, incl, 31);
  const int excl = incl - lr;
  for (int b0 = 0; b0 < total; b0 += 64) {
    int32_t off[2];
    float pr[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      off[h] = -1 - lane;  // unique dummy for idle lanes
      pr[h] = 0.f;
      if (b0 + h * 32 >= total) break;  // a run of at most 32 products: one step
      const int tt = b0 + h * 32 + lane;
      const bool act = tt < total;
      const int src = warp_upper_bound(incl, act ? tt : total - 1);
      const Off sbs = __shfl_sync(kFull, bs, src);
      const int sex = __shfl_sync(kFull, excl, src);
      const float sa = __shfl_sync(kFull, a, src);
      if (act) {
        const Off q = sbs + (Off)(tt - sex);
        off[h] = B.col[q] - c0;
        pr[h] = prod_rn(sa, B.val[q]);
      }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (b0 + h * 32 >= total) break;
      const bool act = b0 + h * 32 + lane < total;
      const unsigned grp = __match_any_sync(kFull, off[h]);
      const bool inb = (uint32_t)off[h] < (uint32_t)kTileCols;
      if (act && !inb) raise_flag(flags, kFlagBadIndex);
      if (__all_sync(kFull, grp == (1u << lane))) {
        if (act && inb) {
          acc[off[h]] = add_rn(acc[off[h]], pr[h]);
          atomicOr(&bits[off[h] >> 5], 1u << (off[h] & 31));
        }
      } else {
        stage[lane] = pr[h];
        __syncwarp();
        if (act && inb && lane == __ffs(grp) - 1) {
          float v = acc[off[h]];
          for (unsigned g = grp; g; g &= g - 1) v = add_rn(v, stage[__ffs(g) - 1]);
          acc[off[h]] = v;
          atomicOr(&bits[off[h] >> 5], 1u << (off[h] & 31));
        }
      }
      __syncwarp();
    }
  }
}

// Units of the tile kernel handed out per atomic ticket.
constexpr int kTicketTiles = 4;

// ---- bulk-staged long segments (tuning heavy_path 2) ----------------------
// A segment of at least kBulkMin entries inside the tile has its 16-byte
// aligned interior copied into the warp's staging area of shared memory by
// the bulk-copy engine (cp.async.bulk global -> shared, completion on an
// mbarrier), kBulkPiece entries of columns and values at a time; lanes then
// read the piece from shared memory.  The unaligned head and tail (at most
// three entries each) take plain loads.  Entries of one B row are distinct
// columns, so their order inside the segment does not matter.
constexpr int kBulkPiece = 64;
constexpr int kBulkMin = 64;
// 32-bit words per warp: columns, values, and the mbarrier (8 bytes).
constexpr int kBulkWarpWords = 2 * kBulkPiece + 4;
// Iterations of a bounded mbarrier wait before the kernel gives up.
constexpr uint32_t kBulkWaitLimit = 1u << 24;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t mbar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mbar));
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase) {
  for (uint32_t it = 0; it < kBulkWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(mbar), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Accumulates the segment [bs, bs + len) like tile_segment, through the
// staging area.  Returns false (kFlagWaitLimit raised) when a copy did not
// complete within the wait limit.
template <typename Off>
__device__ __forceinline__ bool tile_segment_bulk(const DCsr& B, Off bs, int len, float a, int32_t c0, float* acc,
                                                  uint32_t* bits, int32_t* st_col, float* st_val, uint32_t mbar,
                                                  uint32_t& phase, int* flags) {
  const int lane = lane_id();
  const Off end = bs + (Off)len;
  const Off h = min(end, (Off)((bs + 3) & ~(Off)3));  // first 16-byte aligned entry
  const Off t = max(h, (Off)(end & ~(Off)3));          // end of the aligned interior
  auto one = [&](Off q) {
    const int32_t off = B.col[q] - c0;
    const float pr = prod_rn(a, B.val[q]);
    if ((uint32_t)off < (uint32_t)kTileCols) {
      acc[off] = add_rn(acc[off], pr);
      atomicOr(&bits[off >> 5], 1u << (off & 31));
    } else {
      raise_flag(flags, kFlagBadIndex);
    }
  };
  // ragged head and tail: plain loads
  if (lane < (int)(h - bs)) one(bs + (Off)lane);
  if (lane < (int)(end - t)) one(t + (Off)lane);
  for (Off p0 = h; p0 < t; p0 += kBulkPiece) {
    const int n = (int)min((Off)kBulkPiece, t - p0);  // a multiple of 4 entries
    const uint32_t bytes = (uint32_t)n * 4u;
    __syncwarp();  // the previous piece has been read
    if (lane == 0) {
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(mbar), "r"(2u * bytes)
                   : "memory");
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
              smem_u32(st_col)),
          "l"(B.col + p0), "r"(bytes), "r"(mbar)
          : "memory");
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
              smem_u32(st_val)),
          "l"(B.val + p0), "r"(bytes), "r"(mbar)
          : "memory");
    }
    const bool ok = mbar_wait(mbar, phase);
    phase ^= 1u;
    if (!__all_sync(kFull, ok)) {
      if (lane == 0) raise_flag(flags, kFlagWaitLimit);
      mbar_wait(mbar, phase ^ 1u);  // once more for the copies in flight, also bounded
      return false;
    }
    for (int i = lane; i < n; i += 32) {
      const int32_t off = st_col[i] - c0;
      const float pr = prod_rn(a, st_val[i]);
      if ((uint32_t)off < (uint32_t)kTileCols) {
        acc[off] = add_rn(acc[off], pr);
        atomicOr(&bits[off >> 5], 1u << (off & 31));
      } else {
        raise_flag(flags, kFlagBadIndex);
      }
    }
  }
  __syncwarp();
  return true;
}

// One warp per (heavy row, 2^kTileShift-column tile), kTicketTiles tiles
// handed out per atomic ticket (from the list of non-empty tiles when given).  A's row is read 32 entries at a time (the next 32 loaded while the
// current ones are processed); each entry's B row is narrowed to the tile
// (blocked index, else binary search) and the segments are accumulated in
// canonical order (k ascending, then column): long segments by the whole
// warp, runs of short ones packed.  Accumulator: a dense tile of floats plus
// an occupancy bitmap, emitted in column order with coalesced stores and
// cleared as it is read.
// BULK: long segments through tile_segment_bulk (kBulkWarpWords more words
// of shared memory per warp, after the tile accumulators).
template <bool R32, bool BULK>
__global__ void __launch_bounds__(kTileWarps * 32) k_num_tile(DCsr A, DCsr B, const int32_t* heavy_rows, int64_t nheavy,
                                                        const int32_t* big_slot, const int32_t* tile_cnt,
                                                        const int32_t* tile_off, int ntiles, const int64_t* c_rp,
                                                        int32_t* c_col, float* c_val, const int32_t* bidx,
                                                        const uint32_t* tocc, int twords, const int64_t* work,
                                                        const int64_t* nwork, unsigned long long* tile_counter,
                                                        int* flags) {
  using Off = typename RowOff<R32>::T;
  extern __shared__ uint32_t sm_tile[];
  const int lane = lane_id(), wib = threadIdx.x >> 5;
  float* acc = reinterpret_cast<float*>(sm_tile) + (size_t)wib * kTileWarpWords;
  uint32_t* bits = reinterpret_cast<uint32_t*>(acc + kTileCols);
  float* stage = reinterpret_cast<float*>(bits + kTileWords);
  int32_t* st_col = reinterpret_cast<int32_t*>(sm_tile) + (size_t)kTileWarps * kTileWarpWords +
                    (size_t)wib * kBulkWarpWords;
  float* st_val = reinterpret_cast<float*>(st_col + kBulkPiece);
  const uint32_t mbar = smem_u32(st_col + 2 * kBulkPiece);
  uint32_t phase = 0;
  if (BULK && lane == 0) mbar_init(mbar);
  for (int s = lane; s < kTileCols; s += 32) acc[s] = 0.f;
  for (int s = lane; s < kTileWords; s += 32) bits[s] = 0u;
  __syncwarp();
  // units: the listed non-empty tiles, else every (row, tile)
  const int64_t units = work ? *nwork : nheavy * (int64_t)ntiles;
  for (int64_t u = kTicketTiles, u_end = 0;; ++u) {
    if (u >= u_end) {
      // the next kTicketTiles units for one atomic
      unsigned long long t = 0;
      if (lane == 0) t = atomicAdd(tile_counter, 1ull);
      u = (int64_t)__shfl_sync(kFull, t, 0) * kTicketTiles;
      if (u >= units) break;
      u_end = min(units, u + kTicketTiles);
    }
    const int64_t id = work ? work[u] : u;
    const int64_t h = id / ntiles;
    const int tile = (int)(id % ntiles);
    const int32_t row = heavy_rows[h];
    const int64_t slot = big_slot[row];
    const int want = tile_cnt[slot * ntiles + tile];
    if (want == 0) continue;
    const int64_t out = c_rp[row] + tile_off[slot * ntiles + tile];
    const int32_t c0 = tile << kTileShift;
    const int64_t c1 = (int64_t)c0 + kTileCols;
    const int64_t s = A.rp[row], e = A.rp[row + 1];
    int32_t k_nx = 0;
    float a_nx = 0.f;
    if (s + lane < e) {
      k_nx = A.col[s + lane];
      a_nx = A.val[s + lane];
    }
    for (int64_t base = s; base < e; base += 32) {
      const bool have = base + lane < e;
      const int32_t k = k_nx;
      const float a = a_nx;
      if (base + 32 + lane < e) {
        k_nx = A.col[base + 32 + lane];
        a_nx = A.val[base + 32 + lane];
      }
      Off bs = 0;
      int len = 0;
      // B rows without an entry in this tile are rejected by the occupancy bit
      if (have && (!tocc || ((tocc[(int64_t)k * twords + (tile >> 5)] >> (tile & 31)) & 1u))) {
        Off rs = RowOff<R32>::at(B, k), re = RowOff<R32>::at(B, k + 1);
        if (ntiles > 1 && re > rs) {
          // narrow to the tile's columns
          if (bidx) {
            const int32_t* bi = bidx + (int64_t)k * (ntiles + 1) + tile;
            re = rs + (Off)bi[1];
            rs = rs + (Off)bi[0];
          } else {
            if (B.col[rs] < c0) rs = (Off)lower_bound_col(B.col, rs, re, c0);
            if (re > rs && B.col[re - 1] >= c1) re = (Off)lower_bound_col(B.col, rs, re, c1);
          }
        }
        bs = rs;
        len = (int)(re - rs);
      }
      const int n = (int)min((int64_t)32, e - base);
      // none of these B rows reaches into the tile: next chunk
      if (!__any_sync(kFull, len > 0)) continue;
      const unsigned long_mask = __ballot_sync(kFull, len >= kTileLongSeg);
      int idx = 0;
      while (idx < n) {
        if ((long_mask >> idx) & 1u) {
          const Off sbs = __shfl_sync(kFull, bs, idx);
          const int sl = __shfl_sync(kFull, len, idx);
          const float sa = __shfl_sync(kFull, a, idx);
          if (BULK && sl >= kBulkMin) {
            if (!tile_segment_bulk(B, sbs, sl, sa, c0, acc, bits, st_col, st_val, mbar, phase, flags)) return;
          } else {
            tile_segment(B, sbs, sl, sa, c0, acc, bits, flags);
          }
          __syncwarp();
          ++idx;
        } else {
          const unsigned later = long_mask & (~0u << idx);
          const int hi = later ? min(n, __ffs(later) - 1) : n;
          tile_packed(B, bs, len, a, idx, hi, c0, acc, bits, stage, flags);
          idx = hi;
        }
      }
    }
    tile_emit(acc, bits, c0, out, want, c_col, c_val, flags);
  }
}

// --------------------------------------------------------------------------
// Learned path helpers
// --------------------------------------------------------------------------

// Copies each light row that did not overflow (need_exact == 0) from the
// slab to its place in C; the row's length comes from C's row pointers.
// Lanes move 128 entries per round, all loads issued before the stores.
__global__ void k_compact_rows(const int32_t* __restrict__ rows, int64_t nrows, const uint8_t* __restrict__ need_exact,
                               const int64_t* __restrict__ slab_off, const int32_t* __restrict__ slab_col,
                               const float* __restrict__ slab_val, const int64_t* __restrict__ c_rp,
                               int32_t* __restrict__ c_col, float* __restrict__ c_val) {
  const int lane = lane_id();
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t idx = gw; idx < nrows; idx += nw) {
    const int32_t row = rows[idx];
    if (need_exact[row]) continue;
    const int64_t co = c_rp[row];
    const int n = (int)(c_rp[row + 1] - co);
    const int64_t so = slab_off[row];
    for (int t0 = 0; t0 < n; t0 += 4 * 32) {
      int32_t cc[4];
      float vv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int t = t0 + u * 32 + lane;
        if (t < n) {
          cc[u] = slab_col[so + t];
          vv[u] = slab_val[so + t];
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int t = t0 + u * 32 + lane;
        if (t < n) {
          c_col[co + t] = cc[u];
          c_val[co + t] = vv[u];
        }
      }
    }
  }
}

// need_exact[retry[i]] = 1 for the rows queued by the learned pass.
__global__ void k_mark_rows(const int32_t* retry, const unsigned long long* count, uint8_t* need_exact) {
  const int64_t n = (int64_t)*count;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    need_exact[retry[i]] = 1;
}

// out[r] = scan[r + 1] - scan[r]: the counts back from their exclusive scan.
__global__ void k_adjacent_diff(const int64_t* scan, int64_t rows, int64_t* out) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x)
    out[r] = scan[r + 1] - scan[r];
}

// dst[r] = mask[r] ? src[r] : 0
__global__ void k_mask_key(const int64_t* src, const uint8_t* mask, int64_t rows, int64_t* dst) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x)
    dst[r] = mask[r] ? src[r] : 0;
}

// --------------------------------------------------------------------------
// Small products: a counting launch, a one-CTA scan and one numeric launch
// --------------------------------------------------------------------------

// Warp per row of a small product: the row's products (prod[row]) and, for
// rows of at most 2^kSmallLogT products, its exact output count from an
// epoch-tagged key table of 2^kSmallLogT slots (nnz[row]).  A row with more
// products gets nnz[row] = -1, which sends the call to the binned pipeline,
// and sets *stop, after which rows not yet counted are marked -1 too (the
// counts are of no use then); k_small_scan clears *stop.
template <bool R32>
__global__ void __launch_bounds__(kSmallCountWarps * 32) k_small_count(DCsr A, DCsr B, int64_t* prod, int64_t* nnz,
                                                                       unsigned long long* stop, int* flags) {
  using Off = typename RowOff<R32>::T;
  constexpr int T = 1 << kSmallLogT;
  extern __shared__ int32_t sm_keys[];
  const int lane = lane_id();
  int32_t* keys = sm_keys + (threadIdx.x >> 5) * T;
  for (int s = lane; s < T; s += 32) keys[s] = kEmpty;
  __syncwarp();
  int epoch = B.cols < (1 << 24) ? 0 : kNoEpoch;
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t row = gw; row < A.rows; row += nw) {
    const unsigned long long stopped = *reinterpret_cast<volatile unsigned long long*>(stop);
    const int64_t s = A.rp[row], e = A.rp[row + 1];
    int64_t p = 0;
    for (int64_t q = s + lane; q < e; q += 32) {
      const int32_t k = A.col[q];
      p += (int64_t)(RowOff<R32>::at(B, k + 1) - RowOff<R32>::at(B, k));
    }
    p = warp_sum(p);
    int64_t cnt = -1;
    if (p == 0) {
      cnt = 0;
    } else if (p <= T && !stopped) {
      cnt = symbolic_row<kSmallLogT, R32>(A, B, (int32_t)row, keys, epoch, flags);
      if (epoch >= 0) next_row<kSmallLogT>(keys, epoch);
    } else if (p > T && lane == 0) {
      *reinterpret_cast<volatile unsigned long long*>(stop) = 1ull;
    }
    if (lane == 0) {
      prod[row] = p;
      nnz[row] = cnt;
    }
  }
}

// One CTA over the counts of a small product (rows <= kSmallMaxRows): the
// exclusive scan into C's int64 row pointers in place (nnz[rows] = the
// total) and, when rp32 is given and the total fits, into int32 row
// pointers; the identity row list of the numeric launch; and, into the
// mapped host words out[0..3], the total, the products, the largest count
// and the number of rows too large to count (any of them sends the call to
// the binned pipeline).  Thread t owns rows [t * per, (t + 1) * per).
__global__ void __launch_bounds__(kSmallScanThreads) k_small_scan(int64_t* nnz, const int64_t* prod, int64_t rows,
                                                                  int32_t* rp32, int32_t* row_list,
                                                                  unsigned long long* stop, volatile int64_t* out) {
  constexpr int kW = kSmallScanThreads / 32;
  __shared__ int64_t wsum[kW], wprod[kW], wmax[kW], wbig[kW];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int64_t per = (rows + kSmallScanThreads - 1) / kSmallScanThreads;
  const int64_t r0 = min(rows, (int64_t)t * per), r1 = min(rows, r0 + per);
  int64_t sum = 0, psum = 0, mx = 0, big = 0;
  for (int64_t r = r0; r < r1; ++r) {
    const int64_t c = nnz[r];
    if (c < 0) {
      ++big;
    } else {
      sum += c;
      mx = max(mx, c);
    }
    psum += prod[r];
    row_list[r] = (int32_t)r;
  }
  const int64_t incl = warp_incl_scan(sum);
  const int64_t ps = warp_sum(psum), mm = warp_max(mx), bb = warp_sum(big);
  if (lane == 31) wsum[w] = incl;
  if (lane == 0) {
    wprod[w] = ps;
    wmax[w] = mm;
    wbig[w] = bb;
  }
  __syncthreads();
  int64_t wexcl = 0, total = 0;
  {
    const int64_t v = lane < kW ? wsum[lane] : 0;
    const int64_t vi = warp_incl_scan(v);
    wexcl = __shfl_sync(kFull, vi - v, w);
    total = __shfl_sync(kFull, vi, 31);
  }
  int64_t run = wexcl + incl - sum;
  const bool narrow = rp32 != nullptr && total < INT32_MAX;
  for (int64_t r = r0; r < r1; ++r) {
    const int64_t c = nnz[r];
    nnz[r] = run;
    if (narrow) rp32[r] = (int32_t)run;
    run += c < 0 ? 0 : c;
  }
  if (t == 0) {
    nnz[rows] = total;
    if (narrow) rp32[rows] = (int32_t)total;
    int64_t p = 0, m = 0, b = 0;
    for (int i = 0; i < kW; ++i) {
      p += wprod[i];
      m = max(m, wmax[i]);
      b += wbig[i];
    }
    out[0] = total;
    out[1] = p;
    out[2] = m;
    out[3] = b;
    *stop = 0ull;
  }
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

void launch_small_count(const DCsr& A, const DCsr& B, int64_t* prod, int64_t* nnz, unsigned long long* stop,
                        int* flags, const LaunchCtx& lc) {
  if (A.rows == 0) return;
  const size_t smem = (size_t)kSmallCountWarps * (1u << kSmallLogT) * 4;
  int per_sm = 0;
  if (B.rp32) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_small_count<true>, kSmallCountWarps * 32, smem);
  else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_small_count<false>, kSmallCountWarps * 32, smem);
  const int blocks = grid_for(A.rows, kSmallCountWarps, 1, lc.sms * (per_sm < 1 ? 1 : per_sm));
  if (B.rp32) k_small_count<true><<<blocks, kSmallCountWarps * 32, smem, lc.stream>>>(A, B, prod, nnz, stop, flags);
  else k_small_count<false><<<blocks, kSmallCountWarps * 32, smem, lc.stream>>>(A, B, prod, nnz, stop, flags);
}

void launch_small_scan(int64_t* nnz, const int64_t* prod, int64_t rows, int32_t* rp32, int32_t* row_list,
                       unsigned long long* stop, int64_t* out, const LaunchCtx& lc) {
  k_small_scan<<<1, kSmallScanThreads, 0, lc.stream>>>(nnz, prod, rows, rp32, row_list, stop, out);
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
  if (nb <= kScanTile) {
    // two kernels: block totals, then each block adds the totals before it
    int64_t* sums = tmp + 1;
    k_scan_reduce<<<(unsigned)nb, kScanThreads, 0, lc.stream>>>(in, n, sums);
    k_scan_apply_sums<<<(unsigned)nb, kScanThreads, 0, lc.stream>>>(in, n, sums, out);
    return;
  }
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

static int wpb_for(int log_t, int wpb) {
  // keep a CTA's tables within 96 KB
  const int per_warp = (1 << log_t) * 12;
  int lim = (96 * 1024) / per_warp;
  if (lim < 1) lim = 1;
  return std::max(1, std::min(wpb, lim));
}

// CTA size (warps, 1..max_w) giving a kernel the most resident warps per SM
// for `smem_per_warp` bytes of dynamic shared memory per warp; ties go to
// the larger CTA.  Register and shared-memory granularity make this differ
// by table size: 2^9-slot numeric tables (6 KB a warp) reach 36 warps with
// 6-warp CTAs but 32 with 8-warp ones; 2^11-slot symbolic tables (8 KB) fit
// 28 warps with 7-warp CTAs and 24 with 8-warp ones.
template <typename Kernel>
static int auto_wpb(Kernel kernel, size_t smem_per_warp, int max_w) {
  int best_w = 1, best = -1;
  for (int w = 1; w <= max_w; ++w) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, w * 32, (size_t)w * smem_per_warp) !=
        cudaSuccess)
      continue;
    if (per_sm * w >= best) {
      best = per_sm * w;
      best_w = w;
    }
  }
  return best_w;
}

// wpb <= 0 selects auto_wpb, computed once per kernel instantiation (the
// first device that launches it decides; all devices here are alike).
template <typename Kernel>
static int resolve_wpb(int wpb, std::atomic<int>& cache, Kernel kernel, size_t smem_per_warp, int max_w) {
  if (wpb > 0) return wpb;
  int w = cache.load(std::memory_order_relaxed);
  if (w <= 0) {
    w = auto_wpb(kernel, smem_per_warp, max_w);
    cache.store(w, std::memory_order_relaxed);
  }
  return w;
}

template <int LOGT, bool R32>
static void sym_warp_one(const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows, int64_t* nnz, int* flags,
                         const LaunchCtx& lc, int wpb) {
  cudaFuncSetAttribute(k_sym_warp<LOGT, R32>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  static std::atomic<int> auto_w{0};
  wpb = resolve_wpb(wpb, auto_w, k_sym_warp<LOGT, R32>, (size_t)(1 << LOGT) * sizeof(int32_t), 8);
  const size_t smem = (size_t)wpb * (1 << LOGT) * sizeof(int32_t);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sym_warp<LOGT, R32>, wpb * 32, smem);
  if (per_sm < 1) per_sm = 1;
  const int blocks = grid_for(nrows, wpb, 1, lc.sms * per_sm);
  k_sym_warp<LOGT, R32><<<blocks, wpb * 32, smem, lc.stream>>>(A, B, rows, nrows, nnz, flags);
}

void launch_sym_warp(int log_t, const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows, int64_t* nnz,
                     int* flags, const LaunchCtx& lc, int wpb) {
  if (nrows == 0) return;
  const int w = wpb <= 0 ? 0 : log_t >= 11 ? std::min(wpb, 8) : wpb;
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

template <bool R32>
static void sym_block_one(const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows, int log_table,
                          int64_t slot_base, int64_t* nnz, int32_t* big_slot, int32_t* tile_cnt, int ntiles,
                          int* flags, const LaunchCtx& lc) {
  const size_t smem = ((size_t)1 << log_table) * sizeof(int32_t);
  cudaFuncSetAttribute(k_sym_block<R32>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sym_block<R32>, kSymBlockThreads, smem);
  if (per_sm < 1) per_sm = 1;
  const int blocks = (int)std::min<int64_t>(nrows, (int64_t)lc.sms * per_sm);
  k_sym_block<R32><<<blocks, kSymBlockThreads, smem, lc.stream>>>(A, B, rows, nrows, log_table, slot_base, nnz, big_slot,
                                                     tile_cnt, ntiles, flags);
}

void launch_sym_block(const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows, int log_table,
                      int64_t slot_base, int64_t* nnz, int32_t* big_slot, int32_t* tile_cnt, int ntiles, int* flags,
                      const LaunchCtx& lc) {
  if (nrows == 0) return;
  if (B.rp32) sym_block_one<true>(A, B, rows, nrows, log_table, slot_base, nnz, big_slot, tile_cnt, ntiles, flags, lc);
  else sym_block_one<false>(A, B, rows, nrows, log_table, slot_base, nnz, big_slot, tile_cnt, ntiles, flags, lc);
}

template <bool R32>
static void sym_dense_one(const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows, int64_t slot_base,
                          int64_t* nnz, int32_t* big_slot, int32_t* tile_cnt, int ntiles, int* flags,
                          const LaunchCtx& lc) {
  const int max_words = kDenseWindowWords;
  const size_t smem = (size_t)max_words * sizeof(uint32_t);
  cudaFuncSetAttribute(k_sym_dense<R32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int blocks = (int)std::min<int64_t>(nrows, (int64_t)lc.sms);
  k_sym_dense<R32><<<blocks, kSymDenseThreads, smem, lc.stream>>>(A, B, rows, nrows, max_words, slot_base, nnz, big_slot,
                                                      tile_cnt, ntiles, flags);
}

void launch_sym_dense(const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows, int64_t slot_base,
                      int64_t* nnz, int32_t* big_slot, int32_t* tile_cnt, int ntiles, int* flags,
                      const LaunchCtx& lc) {
  if (nrows == 0) return;
  if (B.rp32) sym_dense_one<true>(A, B, rows, nrows, slot_base, nnz, big_slot, tile_cnt, ntiles, flags, lc);
  else sym_dense_one<false>(A, B, rows, nrows, slot_base, nnz, big_slot, tile_cnt, ntiles, flags, lc);
}

template <int LOGT, bool R32>
static void num_warp_one(const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows, const int64_t* c_rp,
                         int32_t* c_col, float* c_val, int* flags, const LaunchCtx& lc, int wpb, const EscArgs& esc) {
  cudaFuncSetAttribute(k_num_warp<LOGT, R32>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  static std::atomic<int> auto_w{0};
  wpb = resolve_wpb(wpb, auto_w, k_num_warp<LOGT, R32>, (size_t)numeric_words<LOGT>() * 4, wpb_for(LOGT, 8));
  const size_t smem = (size_t)wpb * numeric_words<LOGT>() * 4;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_num_warp<LOGT, R32>, wpb * 32, smem);
  if (per_sm < 1) per_sm = 1;
  const int blocks = grid_for(nrows, wpb, 1, lc.sms * per_sm);
  k_num_warp<LOGT, R32><<<blocks, wpb * 32, smem, lc.stream>>>(A, B, rows, nrows, c_rp, c_col, c_val, esc.prod,
                                                                esc.min_prod, flags);
}

void launch_num_warp(int log_t, const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows,
                     const int64_t* c_rp, int32_t* c_col, float* c_val, int* flags, const LaunchCtx& lc, int wpb,
                     const EscArgs& esc) {
  if (nrows == 0) return;
  const int w = wpb <= 0 ? 0 : wpb_for(log_t, wpb);
#define SPG_NW(L)                                                                          \
  case L:                                                                                  \
    if (B.rp32) num_warp_one<L, true>(A, B, rows, nrows, c_rp, c_col, c_val, flags, lc, w, esc); \
    else num_warp_one<L, false>(A, B, rows, nrows, c_rp, c_col, c_val, flags, lc, w, esc);       \
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
                                 const LaunchCtx& lc, int wpb, const EscArgs& esc) {
  cudaFuncSetAttribute(k_num_warp_learned<LOGT, R32>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  static std::atomic<int> auto_w{0};
  wpb = resolve_wpb(wpb, auto_w, k_num_warp_learned<LOGT, R32>, (size_t)numeric_words<LOGT>() * 4,
                    wpb_for(LOGT, 8));
  const size_t smem = (size_t)wpb * numeric_words<LOGT>() * 4;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_num_warp_learned<LOGT, R32>, wpb * 32, smem);
  if (per_sm < 1) per_sm = 1;
  const int blocks = grid_for(nrows, wpb, 1, lc.sms * per_sm);
  k_num_warp_learned<LOGT, R32><<<blocks, wpb * 32, smem, lc.stream>>>(A, B, rows, nrows, cap, slab_off, slab_col,
                                                                        slab_val, nnz_out, retry_rows, retry_count,
                                                                        esc.prod, esc.min_prod, flags);
}

void launch_num_warp_learned(int log_t, const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows,
                             const int64_t* cap, const int64_t* slab_off, int32_t* slab_col, float* slab_val,
                             int64_t* nnz_out, int32_t* retry_rows, unsigned long long* retry_count, int* flags,
                             const LaunchCtx& lc, int wpb, const EscArgs& esc) {
  if (nrows == 0) return;
  const int w = wpb <= 0 ? 0 : wpb_for(log_t, wpb);
#define SPG_NWL(L)                                                                                             \
  case L:                                                                                                      \
    if (B.rp32)                                                                                                \
      num_warp_learned_one<L, true>(A, B, rows, nrows, cap, slab_off, slab_col, slab_val, nnz_out, retry_rows, \
                                    retry_count, flags, lc, w, esc);                                                \
    else                                                                                                       \
      num_warp_learned_one<L, false>(A, B, rows, nrows, cap, slab_off, slab_col, slab_val, nnz_out,            \
                                     retry_rows, retry_count, flags, lc, w, esc);                                   \
    break;
  switch (log_t) {
    SPG_NWL(5) SPG_NWL(6) SPG_NWL(7) SPG_NWL(8) SPG_NWL(9) SPG_NWL(10) SPG_NWL(11) SPG_NWL(12)
    default: break;
  }
#undef SPG_NWL
}

template <int LOGT, bool R32>
static int block_grid(const void* kernel, int64_t nrows, const LaunchCtx& lc) {
  const size_t smem = (size_t)block_words<LOGT>() * 4;
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBlkThreads, smem);
  if (per_sm < 1) per_sm = 1;
  return (int)std::min<int64_t>(nrows, (int64_t)lc.sms * per_sm);
}

template <int LOGT, bool R32>
static void num_block_one(const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows, const int64_t* c_rp,
                          int32_t* c_col, float* c_val, int* flags, const LaunchCtx& lc) {
  const size_t smem = (size_t)block_words<LOGT>() * 4;
  const int blocks = block_grid<LOGT, R32>((const void*)k_num_block<LOGT, R32>, nrows, lc);
  k_num_block<LOGT, R32><<<blocks, kBlkThreads, smem, lc.stream>>>(A, B, rows, nrows, c_rp, c_col, c_val, flags);
}

template <int LOGT, bool R32>
static void num_block_learned_one(const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows,
                                  const int64_t* cap, const int64_t* slab_off, int32_t* slab_col, float* slab_val,
                                  int64_t* nnz_out, int32_t* retry_rows, unsigned long long* retry_count, int* flags,
                                  const LaunchCtx& lc) {
  const size_t smem = (size_t)block_words<LOGT>() * 4;
  const int blocks = block_grid<LOGT, R32>((const void*)k_num_block_learned<LOGT, R32>, nrows, lc);
  k_num_block_learned<LOGT, R32><<<blocks, kBlkThreads, smem, lc.stream>>>(A, B, rows, nrows, cap, slab_off,
                                                                           slab_col, slab_val, nnz_out, retry_rows,
                                                                           retry_count, flags);
}

void launch_num_block(int bin, const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows, const int64_t* c_rp,
                      int32_t* c_col, float* c_val, int* flags, const LaunchCtx& lc) {
  if (nrows == 0) return;
  if (bin == kBinBlock) {
    if (B.rp32) num_block_one<kBlkLogSmallT, true>(A, B, rows, nrows, c_rp, c_col, c_val, flags, lc);
    else num_block_one<kBlkLogSmallT, false>(A, B, rows, nrows, c_rp, c_col, c_val, flags, lc);
  } else {
    if (B.rp32) num_block_one<kBlkLogLargeT, true>(A, B, rows, nrows, c_rp, c_col, c_val, flags, lc);
    else num_block_one<kBlkLogLargeT, false>(A, B, rows, nrows, c_rp, c_col, c_val, flags, lc);
  }
}

void launch_num_block_learned(int bin, const DCsr& A, const DCsr& B, const int32_t* rows, int64_t nrows,
                              const int64_t* cap, const int64_t* slab_off, int32_t* slab_col, float* slab_val,
                              int64_t* nnz_out, int32_t* retry_rows, unsigned long long* retry_count, int* flags,
                              const LaunchCtx& lc) {
  if (nrows == 0) return;
#define SPG_NBL(L, R)                                                                                            \
  num_block_learned_one<L, R>(A, B, rows, nrows, cap, slab_off, slab_col, slab_val, nnz_out, retry_rows,       \
                              retry_count, flags, lc)
  if (bin == kBinBlock) {
    if (B.rp32) SPG_NBL(kBlkLogSmallT, true);
    else SPG_NBL(kBlkLogSmallT, false);
  } else {
    if (B.rp32) SPG_NBL(kBlkLogLargeT, true);
    else SPG_NBL(kBlkLogLargeT, false);
  }
#undef SPG_NBL
}

// dst[i] = src[i] for n 32-bit words; dst may be mapped pinned host memory.
__global__ void k_copy_words(const uint32_t* src, uint32_t* dst, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

void launch_copy_words(const void* src, void* dst, int64_t n, const LaunchCtx& lc) {
  if (n == 0) return;
  k_copy_words<<<1, 128, 0, lc.stream>>>(static_cast<const uint32_t*>(src), static_cast<uint32_t*>(dst), n);
}

// out[i] = in[i] + off as int32 (out_bits 32) or int64.
__global__ void k_shift_rp(const int64_t* in, int64_t n, int64_t off, void* out, int out_bits) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = in[i] + off;
    if (out_bits == 32) static_cast<int32_t*>(out)[i] = (int32_t)v;
    else static_cast<int64_t*>(out)[i] = v;
  }
}

void launch_shift_rp(const int64_t* in, int64_t n, int64_t off, void* out, int out_bits, const LaunchCtx& lc) {
  if (n == 0) return;
  k_shift_rp<<<grid_for(n, 256, 1, lc.sms * 8), 256, 0, lc.stream>>>(in, n, off, out, out_bits);
}

void launch_row_lengths(const int64_t* rp, int64_t rows, int64_t* len, const LaunchCtx& lc) {
  if (rows == 0) return;
  k_row_lengths<<<grid_for(rows, 256, 1, lc.sms * 8), 256, 0, lc.stream>>>(rp, rows, len);
}

void launch_tile_counts_from_cols(const int32_t* heavy_rows, int64_t nheavy, const int64_t* c_rp,
                                  const int32_t* c_col, int ntiles, int32_t* big_slot, int32_t* tile_cnt, int* flags,
                                  const LaunchCtx& lc) {
  if (nheavy == 0) return;
  k_tile_counts_from_cols<<<grid_for(nheavy, 256, 32, lc.sms * 8), 256, 0, lc.stream>>>(
      heavy_rows, nheavy, c_rp, c_col, ntiles, big_slot, tile_cnt, flags);
}

void launch_tile_offsets(const int32_t* heavy_rows, int64_t nheavy, const int32_t* big_slot, const int32_t* tile_cnt,
                         int ntiles, int32_t* tile_off, int64_t* nz_cnt, const LaunchCtx& lc) {
  if (nheavy == 0) return;
  k_tile_offsets<<<grid_for(nheavy, 256, 32, lc.sms * 8), 256, 0, lc.stream>>>(heavy_rows, nheavy, big_slot, tile_cnt,
                                                                                ntiles, tile_off, nz_cnt);
}

void launch_tile_worklist(const int32_t* heavy_rows, int64_t nheavy, const int32_t* big_slot, const int32_t* tile_cnt,
                          int ntiles, const int64_t* nz_off, int64_t* work, const LaunchCtx& lc) {
  if (nheavy == 0) return;
  k_tile_worklist<<<grid_for(nheavy, 256, 32, lc.sms * 8), 256, 0, lc.stream>>>(heavy_rows, nheavy, big_slot,
                                                                                 tile_cnt, ntiles, nz_off, work);
}

void launch_build_blocked_index(const DCsr& B, int ntiles, int32_t* bidx, const LaunchCtx& lc) {
  if (B.rows == 0) return;
  k_build_blocked_index<<<grid_for(B.rows, 256, 32, lc.sms * 16), 256, 0, lc.stream>>>(B, ntiles, bidx);
}

template <bool R32, bool BULK>
static void num_tile_one(const DCsr& A, const DCsr& B, const int32_t* heavy_rows, int64_t nheavy,
                         const int32_t* big_slot, const int32_t* tile_cnt, const int32_t* tile_off, int ntiles,
                         const int64_t* c_rp, int32_t* c_col, float* c_val, const int32_t* bidx,
                         const uint32_t* tocc, const int64_t* work, const int64_t* nwork,
                         unsigned long long* tile_counter, int* flags, const LaunchCtx& lc) {
  const size_t smem = (size_t)kTileWarps * (kTileWarpWords + (BULK ? kBulkWarpWords : 0)) * 4;
  const int twords = (ntiles + 31) / 32;
  cudaFuncSetAttribute(k_num_tile<R32, BULK>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_num_tile<R32, BULK>, kTileWarps * 32, smem);
  if (per_sm < 1) per_sm = 1;
  const int64_t tiles = nheavy * (int64_t)ntiles;
  const int blocks = (int)std::min<int64_t>((tiles + kTileWarps - 1) / kTileWarps, (int64_t)lc.sms * per_sm);
  cudaMemsetAsync(tile_counter, 0, sizeof(unsigned long long), lc.stream);
  k_num_tile<R32, BULK><<<blocks, kTileWarps * 32, smem, lc.stream>>>(A, B, heavy_rows, nheavy, big_slot, tile_cnt,
                                                                      tile_off, ntiles, c_rp, c_col, c_val, bidx,
                                                                      tocc, twords, work, nwork, tile_counter,
                                                                      flags);
}

void launch_num_tile(const DCsr& A, const DCsr& B, const int32_t* heavy_rows, int64_t nheavy, const int32_t* big_slot,
                     const int32_t* tile_cnt, const int32_t* tile_off, int ntiles, const int64_t* c_rp,
                     int32_t* c_col, float* c_val, const int32_t* bidx, const uint32_t* tocc, const int64_t* work,
                     const int64_t* nwork, unsigned long long* tile_counter, int* flags, const LaunchCtx& lc,
                     bool bulk) {
  if (nheavy == 0) return;
  // the bulk copies need 16-byte aligned column and value arrays
  bulk = bulk && ((reinterpret_cast<uintptr_t>(B.col) | reinterpret_cast<uintptr_t>(B.val)) & 15u) == 0;
#define SPG_NT(R, K)                                                                                          \
  num_tile_one<R, K>(A, B, heavy_rows, nheavy, big_slot, tile_cnt, tile_off, ntiles, c_rp, c_col, c_val, bidx, \
                     tocc, work, nwork, tile_counter, flags, lc)
  if (B.rp32) {
    if (bulk) SPG_NT(true, true);
    else SPG_NT(true, false);
  } else {
    if (bulk) SPG_NT(false, true);
    else SPG_NT(false, false);
  }
#undef SPG_NT
}

void launch_build_tile_occupancy(int64_t rows, const int32_t* bidx, int ntiles, uint32_t* tocc, const LaunchCtx& lc) {
  if (rows == 0) return;
  k_build_tile_occupancy<<<grid_for(rows, 256, 32, lc.sms * 16), 256, 0, lc.stream>>>(rows, bidx, ntiles,
                                                                                    (ntiles + 31) / 32, tocc);
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

void launch_adjacent_diff(const int64_t* scan, int64_t rows, int64_t* out, const LaunchCtx& lc) {
  if (rows == 0) return;
  k_adjacent_diff<<<grid_for(rows, 256, 1, lc.sms * 8), 256, 0, lc.stream>>>(scan, rows, out);
}

void launch_mask_key(const int64_t* src, const uint8_t* mask, int64_t rows, int64_t* dst, const LaunchCtx& lc) {
  if (rows == 0) return;
  k_mask_key<<<grid_for(rows, 256, 1, lc.sms * 8), 256, 0, lc.stream>>>(src, mask, rows, dst);
}

}  // namespace spg
