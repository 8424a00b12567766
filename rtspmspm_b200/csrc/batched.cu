// Batched SpGEMM: many independent products C_m = A_m * B_m of uneven sizes.
//
// No reference counterpart: the reference runs one product per process
// (scripts/AE_test.py:199-215).  Here all rows of all products form one
// global row space, binned by table size across every matrix at once; each
// stage (symbolic, numeric) is two persistent launches that drain a queue of
// (bin, row range) tiles of all products -- one queue of small warp tables,
// whose CTAs stay small so that many share an SM, and one of large warp
// tables plus a CTA-wide table for the largest rows -- so small and large
// products share the GPU without per-matrix or per-bin launches.  Bin bounds
// and tile counts are derived on the device, and the launch sequence is
// captured once into a CUDA graph and replayed while the inputs stay the
// same.
//
// Plan (host, once per input set): matrix descriptors, global-row -> matrix
// map, the nnz upper bound of every product (sum over rows of
// min(products, cols)), so that every C_m gets a fixed region of one output
// slab and no host round trip is needed while the graph runs.
// Products with a row of more than kBatchMaxBound products (capped at the
// columns) are run one by one through the single-product path instead.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "block_row.cuh"
#include "context.hpp"
#include "warp_row.cuh"

using namespace spg;

namespace spg {

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

// One persistent launch drains a queue of tiles -- runs of rows of one bin,
// all products mixed -- in the order the queue lists its bins (largest rows
// first).  A queue holds either warp bins only (each warp of the CTA takes
// rows of the tile with its own table of 2^L slots) or also the CTA bin
// (kBinBlock: the CTA takes the tile's rows one at a time with one CTA-wide
// table of 2^CTA_LOGT slots, block_row.cuh).  The tile count of every bin is
// derived on the device from the binning's offsets (k_queue_prefix), so the
// launch needs no host round trip and replays from a CUDA graph.
constexpr int kQueueMax = 8;

struct BatchQueue {
  int nq;                          // bins in this queue
  int bins[kQueueMax];             // bin per queue slot
  int rows_per_tile[kQueueMax];
};

// tile_pref[i] = tiles of queue slots before i (tile_pref[nq] = all).
__global__ void k_queue_prefix(const int64_t* bin_off, BatchQueue q, int64_t* tile_pref) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    int64_t t = 0;
    for (int i = 0; i < q.nq; ++i) {
      tile_pref[i] = t;
      const int64_t rows = bin_off[q.bins[i] + 1] - bin_off[q.bins[i]];
      t += (rows + q.rows_per_tile[i] - 1) / q.rows_per_tile[i];
    }
    tile_pref[q.nq] = t;
  }
}

// Outputs of the learned numeric pass: each predicted row is written sorted
// into its slab slot (slab_off[g], capacity cap[g]); a row with more columns
// than its capacity is queued in retry for the exact re-run (nnz[g] = -1).
struct LearnedOut {
  const int64_t* cap;
  const int64_t* slab_off;
  int32_t* slab_col;
  float* slab_val;
  int32_t* retry;
  unsigned long long* retry_count;
};

// One warp over rows [first, last) of a warp bin of table 2^LOGT (its slot
// `sm`, of the size of the queue's largest table).  Tables are epoch-tagged
// while the product's B has fewer than 2^24 columns; a row of a wider product
// clears the table first if tagged keys may be left in it.
template <int LOGT, bool NUMERIC, bool LEARNED>
__device__ __forceinline__ void warp_tile(const BatchMat* mats, const int32_t* row_mat, const int32_t* lists,
                                          int64_t first, int64_t last, int32_t* sm, int64_t* nnz,
                                          const int64_t* gscan, int32_t* c_col, float* c_val, const LearnedOut& lo,
                                          const int64_t* prod, int esc_min, int ecap, int* flags) {
  constexpr int T = 1 << LOGT;
  const int lane = lane_id();
  int32_t* keys = sm;
  float* vals = reinterpret_cast<float*>(keys + T);
  int32_t* list = keys + 2 * T;
  for (int s2 = lane; s2 < T; s2 += 32) keys[s2] = kEmpty;
  __syncwarp();
  int epoch = 0;
  bool tagged = false;  // keys of an epoch may be in the table
  for (int64_t i = first; i < last; ++i) {
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
    } else if (LEARNED) {
      const int c = (int)lo.cap[g];
      if (esc_wanted(prod[g], c, esc_min, ecap)) {
        // expand-sort-fold row in the warp's slot (its table wiped after)
        const int64_t off = lo.slab_off[g];
        const int n = esc_row<true>(M.A, M.B, r, (int)prod[g], keys, c, lo.slab_col + off, lo.slab_val + off);
        esc_wipe(keys, T);
        if (n >= 0) {
          if (lane == 0) {
            if (n > c) {
              nnz[g] = -1;
              lo.retry[atomicAdd(lo.retry_count, 1ull)] = (int32_t)g;
            } else {
              nnz[g] = n;
            }
          }
          continue;
        }
      }
      const int n = accumulate_row<LOGT, true, true>(M.A, M.B, r, keys, vals, list, ep, c, flags);
      if (n < 0) {
        if (lane == 0) {
          nnz[g] = -1;
          lo.retry[atomicAdd(lo.retry_count, 1ull)] = (int32_t)g;
        }
      } else {
        const int64_t off = lo.slab_off[g];
        emit_row<LOGT>(keys, vals, list, n, ep, n, lo.slab_col + off, lo.slab_val + off, false);
        if (lane == 0) nnz[g] = n;
      }
    } else {
      const int64_t off = M.c_base + (gscan[g] - gscan[M.row_start]);
      const int64_t want = gscan[g + 1] - gscan[g];
      if (esc_wanted(prod[g], want, esc_min, ecap)) {
        const int n = esc_row<true>(M.A, M.B, r, (int)prod[g], keys, want, c_col + off, c_val + off);
        esc_wipe(keys, T);
        if (n >= 0) {
          if (n != want && lane == 0) raise_flag(flags, kFlagCountDiff);
          continue;
        }
      }
      numeric_row<LOGT, true, true>(M.A, M.B, r, keys, vals, list, ep, c_col + off, c_val + off, want, flags);
    }
    if (LEARNED && ep < 0) next_row<LOGT>(keys, ep);  // plain keys: cleared after every row
    if (ep >= 0) {
      tagged = true;
      if (!NUMERIC || LEARNED) next_row<LOGT>(keys, ep);
      epoch = ep;
      if (epoch == 0) tagged = false;  // wiped on wrap
    }
  }
}

// Tile t of queue q: its bin and rows [first, last) of the bin's list.
__device__ __forceinline__ int decode_tile(const BatchQueue& q, const int64_t* tile_pref, const int64_t* bin_off,
                                           int64_t t, int64_t& first, int64_t& last) {
  int qi = 0;
  while (qi + 1 < q.nq && tile_pref[qi + 1] <= t) ++qi;
  const int b = q.bins[qi];
  first = bin_off[b] + (t - tile_pref[qi]) * q.rows_per_tile[qi];
  last = min(bin_off[b + 1], first + q.rows_per_tile[qi]);
  return b;
}

// Persistent symbolic (NUMERIC = false: exact nnz per row into nnz) or
// numeric (rows written into the output slab at gscan) pass over the queue
// q: warp bins of tables 2^LMIN..2^LMAX and, when CTA_LOGT > 0, the CTA bin,
// which the queue lists first.  CTA-bin tiles are taken by whole CTAs (one
// ticket per CTA); the first warp-bin tile a CTA draws goes to its warp 0
// and from then on every warp takes its own tickets, so warps working on
// rows of different sizes never wait for one another.  (MINB: CTAs per SM
// the registers must allow.)
template <bool NUMERIC, bool LEARNED, int LMIN, int LMAX, int CTA_LOGT, int MINB>
__global__ void __launch_bounds__(kBlkThreads, MINB) k_batch_queue(const BatchMat* mats, const int32_t* row_mat,
                                                                   const int32_t* lists, const int64_t* bin_off,
                                                                   BatchQueue q, const int64_t* tile_pref,
                                                                   const int64_t* bound, int64_t* nnz,
                                                                   const int64_t* gscan, int32_t* c_col,
                                                                   float* c_val, LearnedOut lo,
                                                                   const int64_t* prod, int esc_min,
                                                                   unsigned long long* counter, int* flags) {
  extern __shared__ int32_t sm_q[];
  __shared__ unsigned long long sh_tile;
  const int tid = threadIdx.x, lane = lane_id(), wib = tid >> 5;
  const int64_t ntiles = tile_pref[q.nq];
  int64_t handed = -1;  // a warp-bin tile drawn in CTA mode, for warp 0
  if (CTA_LOGT > 0) {
    constexpr int CL = CTA_LOGT > 0 ? CTA_LOGT : 1;
    constexpr int TC = 1 << CL;
    int32_t* keys = sm_q;
    float* vals = reinterpret_cast<float*>(sm_q + TC);
    uint32_t* own = reinterpret_cast<uint32_t*>(sm_q + 2 * TC);
    BlockScratch& sc = *reinterpret_cast<BlockScratch*>(sm_q + (NUMERIC ? 3 * TC : TC));
    for (;;) {
      if (tid == 0) sh_tile = atomicAdd(counter, 1ull);
      __syncthreads();
      const int64_t t = (int64_t)sh_tile;
      __syncthreads();  // read by every thread before the next ticket
      if (t >= ntiles) return;
      int64_t first, last;
      const int b = decode_tile(q, tile_pref, bin_off, t, first, last);
      if (b != kBinBlock) {
        handed = t;
        break;
      }
      for (int64_t i = first; i < last; ++i) {
        const int64_t g = lists[i];
        const BatchMat& M = mats[row_mat[g]];
        const int32_t r = (int32_t)(g - M.row_start);
        if (LEARNED) {
          const int64_t c = lo.cap[g];
          const int lg = cta_table_log(c, CL);
          const int n = cta_accumulate_row<CL, true, true>(M.A, M.B, r, keys, vals, own, sc, c, flags, lg);
          if (n < 0) {
            if (tid == 0) {
              nnz[g] = -1;
              lo.retry[atomicAdd(lo.retry_count, 1ull)] = (int32_t)g;
            }
          } else {
            const int64_t off = lo.slab_off[g];
            cta_emit_row<CL>(keys, vals, own, sc, n, n, lo.slab_col + off, lo.slab_val + off, lg);
            if (tid == 0) nnz[g] = n;
          }
        } else if (NUMERIC) {
          const int64_t off = M.c_base + (gscan[g] - gscan[M.row_start]);
          const int64_t want = gscan[g + 1] - gscan[g];
          const int lg = cta_table_log(want, CL);
          const int n = cta_accumulate_row<CL, true, false>(M.A, M.B, r, keys, vals, own, sc, 0, flags, lg);
          if (n != want && tid == 0) raise_flag(flags, kFlagCountDiff);
          cta_emit_row<CL>(keys, vals, own, sc, n, want, c_col + off, c_val + off, lg);
        } else {
          // symbolic: the table sized from the row's bound (products capped at the columns)
          const int lg = cta_table_log(bound[g], CL);
          const int n = cta_accumulate_row<CL, true, false, false>(M.A, M.B, r, keys, vals, own, sc, 0, flags, lg);
          if (tid == 0) nnz[g] = n;
        }
      }
    }
    __syncthreads();  // the CTA table's memory becomes the warps' tables
  }
  // warp mode: each warp its own tickets and table slot (whose words an
  // expand-sort-fold row may use whole)
  int32_t* slot = sm_q + (size_t)wib * (NUMERIC ? numeric_words<LMAX>() : (1 << LMAX));
  const int ecap = NUMERIC ? esc_capacity(numeric_words<LMAX>()) : 0;
  for (;;) {
    int64_t t;
    if (wib == 0 && handed >= 0) {
      t = handed;
      handed = -1;
    } else {
      unsigned long long x = 0;
      if (lane == 0) x = atomicAdd(counter, 1ull);
      t = (int64_t)__shfl_sync(kFull, x, 0);
    }
    if (t >= ntiles) break;
    int64_t first, last;
    const int b = decode_tile(q, tile_pref, bin_off, t, first, last);
    if (b == kBinBlock) {  // cannot happen: the CTA bin comes first in the queue
      if (lane == 0) raise_flag(flags, kFlagHashFull);
      continue;
    }
    const int L = kMinLogT + b;
#define SPG_WT(LL)                                                                                          \
  if (L == LL && LL >= LMIN && LL <= LMAX)                                                                  \
    warp_tile<(LL >= LMIN && LL <= LMAX) ? LL : LMIN, NUMERIC, LEARNED>(mats, row_mat, lists, first, last, slot, \
                                                                        nnz, gscan, c_col, c_val, lo, prod,       \
                                                                        NUMERIC ? esc_min : 0, ecap, flags);
    SPG_WT(5) SPG_WT(6) SPG_WT(7) SPG_WT(8) SPG_WT(9) SPG_WT(10) SPG_WT(11)
#undef SPG_WT
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

// Learned batch: copies every predicted row that did not overflow
// (need[g] == 0) from its slab slot to its place in C (warp per row).
// Lanes move 128 entries per round with all loads issued before the stores
// (one entry per lane per round moved 17.5 GB for the 512 uneven products
// in 11.8 ms).
__global__ void k_batch_compact(const BatchMat* __restrict__ mats, const int32_t* __restrict__ row_mat, int64_t R,
                                const uint8_t* __restrict__ need, const int64_t* __restrict__ slab_off,
                                const int32_t* __restrict__ slab_col, const float* __restrict__ slab_val,
                                const int64_t* __restrict__ gscan, int32_t* __restrict__ c_col,
                                float* __restrict__ c_val) {
  const int lane = lane_id();
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t g = gw; g < R; g += nw) {
    if (need[g]) continue;
    const BatchMat& M = mats[row_mat[g]];
    const int64_t n = gscan[g + 1] - gscan[g];
    const int64_t src = slab_off[g];
    const int64_t dst = M.c_base + (gscan[g] - gscan[M.row_start]);
    for (int64_t t0 = 0; t0 < n; t0 += 4 * 32) {
      int32_t cc[4];
      float vv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int64_t t = t0 + u * 32 + lane;
        if (t < n) {
          cc[u] = slab_col[src + t];
          vv[u] = slab_val[src + t];
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int64_t t = t0 + u * 32 + lane;
        if (t < n) {
          c_col[dst + t] = cc[u];
          c_val[dst + t] = vv[u];
        }
      }
    }
  }
}

namespace {

// The queue launches: symbolic small / large tables, numeric small / mid /
// large tables (the numeric ones also in a learned form).  Warp-only queues
// size their CTAs for their largest warp table, so small tables keep many
// warps per SM; the large queues hold the CTA bin.
constexpr int kQueues = 5;
constexpr int kQSymSmall = 0, kQSymLarge = 1, kQNumSmall = 2, kQNumMid = 3, kQNumLarge = 4;
// Rows of more than kBatchMaxBound products (capped at the columns) are
// beyond the queue's tables: their products run one by one instead.
constexpr int64_t kBatchMaxBound = 4096;
constexpr int kBatchCtaLogT = 13;  // CTA tables: 2^13 slots at load <= 1/2

BatchQueue queue_of(int which) {
  BatchQueue q{};
  auto add = [&](int bin, int rpt) {
    q.bins[q.nq] = bin;
    q.rows_per_tile[q.nq] = rpt;
    ++q.nq;
  };
  switch (which) {
    case kQSymSmall:
      for (int l = 10; l >= 5; --l) add(l - kMinLogT, l >= 9 ? 2 : 8);
      break;
    case kQSymLarge:
      add(kBinBlock, 1);
      add(11 - kMinLogT, 1);
      break;
    case kQNumSmall:
      for (int l = 9; l >= 5; --l) add(l - kMinLogT, l >= 8 ? 2 : 8);
      break;
    case kQNumMid:
      add(10 - kMinLogT, 1);
      break;
    default:
      add(kBinBlock, 1);
      break;
  }
  return q;
}

// Dynamic shared memory of a queue launch: one table slot of the queue's
// largest warp table per warp, or the CTA table and its scratch.
size_t queue_smem(int which) {
  const size_t sc = sizeof(BlockScratch);
  switch (which) {
    case kQSymSmall: return (size_t)kBlkWarps * 4 * (1 << 10);
    case kQSymLarge: return std::max((size_t)kBlkWarps * 4 * (1 << 11), (size_t)4 * (1 << kBatchCtaLogT) + sc);
    case kQNumSmall: return (size_t)kBlkWarps * 12 * (1 << 9);
    case kQNumMid: return (size_t)kBlkWarps * 12 * (1 << 10);
    default: return (size_t)12 * (1 << kBatchCtaLogT) + sc;
  }
}

// The kernel of queue `which` (the learned form of a numeric queue when
// `learned`) and, with `args`, its launch.
struct QueueArgs {
  const BatchMat* mats;
  const int32_t* row_mat;
  const int32_t* lists;
  const int64_t* bin_off;
  BatchQueue q;
  const int64_t* tile_pref;
  const int64_t* bound;
  int64_t* nnz;
  const int64_t* gscan;
  int32_t* c_col;
  float* c_val;
  LearnedOut lo;
  const int64_t* prod;
  int esc_min;
  unsigned long long* counter;
  int* flags;
};

template <bool NUMERIC, bool LEARNED, int LMIN, int LMAX, int CTA, int MINB>
const void* queue_launch(const QueueArgs* a, int grid, size_t smem, cudaStream_t st) {
  auto k = k_batch_queue<NUMERIC, LEARNED, LMIN, LMAX, CTA, MINB>;
  if (a)
    k<<<grid, kBlkThreads, smem, st>>>(a->mats, a->row_mat, a->lists, a->bin_off, a->q, a->tile_pref, a->bound,
                                       a->nnz, a->gscan, a->c_col, a->c_val, a->lo, a->prod, a->esc_min, a->counter,
                                       a->flags);
  return (const void*)k;
}

const void* queue_dispatch(int which, bool learned, const QueueArgs* a, int grid, size_t smem, cudaStream_t st) {
  switch (which) {
    case kQSymSmall: return queue_launch<false, false, 5, 10, 0, 4>(a, grid, smem, st);
    case kQSymLarge: return queue_launch<false, false, 11, 11, kBatchCtaLogT, 2>(a, grid, smem, st);
    case kQNumSmall:
      return learned ? queue_launch<true, true, 5, 9, 0, 4>(a, grid, smem, st)
                     : queue_launch<true, false, 5, 9, 0, 4>(a, grid, smem, st);
    case kQNumMid:
      return learned ? queue_launch<true, true, 10, 10, 0, 2>(a, grid, smem, st)
                     : queue_launch<true, false, 10, 10, 0, 2>(a, grid, smem, st);
    default:
      return learned ? queue_launch<true, true, 10, 10, kBatchCtaLogT, 2>(a, grid, smem, st)
                     : queue_launch<true, false, 10, 10, kBatchCtaLogT, 2>(a, grid, smem, st);
  }
}

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
  BinParams bp_sym{}, bp_num{}, bp_lrn{};  // binnings: symbolic, numeric, learned
  int grid[2][kQueues] = {};               // CTAs of each queue launch (plain, learned form)
  int64_t* tile_pref = nullptr;            // kQueues x (kQueueMax + 1)
  unsigned long long* qcount = nullptr;    // tile tickets, kQueues
  // learned method
  bool learned = false;
  int force_overflow = 0;
  int64_t* cap = nullptr;        // R + 1 predicted capacities
  int64_t* slab_off = nullptr;   // R + 1
  uint8_t* need = nullptr;       // rows on the exact path
  int64_t* mkey = nullptr;       // R masked sizes
  int32_t* retry = nullptr;      // overflowed rows
  int32_t* slab_col = nullptr;
  float* slab_val = nullptr;
  unsigned long long* lcount = nullptr;  // [0] rows predicted heavy, [1] overflowed rows
  unsigned long long* h_lcount = nullptr;  // pinned copy
  int launches = 0;
};

void free_plan(BatchPlan* p) {
  if (!p) return;
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  for (void* q : p->owned) cudaFree(q);
  if (p->h_nnz_m) cudaFreeHost(p->h_nnz_m);
  if (p->h_lcount) cudaFreeHost(p->h_lcount);
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
  k.push_back((uintptr_t)(t.learned_load * 1000.0f));
  k.push_back((uintptr_t)(o.algo == SPG_ALGO_LEARNED ? 1 + (o.force_overflow ? 1 : 0) : 0));
  k.push_back((uintptr_t)(intptr_t)t.esc_min_prod);
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
// Plain: bounds, symbolic binning, the symbolic queues, numeric binning and
// scan, the numeric queues, per-product row pointers.  Learned: the batched
// plan (products, features, tensor-core MLP capacity), learned binning, the
// learned numeric queues into a capacity-sized slab; rows predicted beyond
// the tables or overflowed go through the symbolic and numeric queues
// exactly (empty queues when there are none, so no host round trip is
// needed), the scan of the final sizes, the slab rows copied into C.
void enqueue(spg_ctx* ctx, BatchPlan* p) {
  const LaunchCtx lc = launch_ctx(ctx);
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
  const LearnedOut lo{p->cap, p->slab_off, p->slab_col, p->slab_val, p->retry, p->lcount ? p->lcount + 1 : nullptr};
  auto run_queue = [&](int which, bool learned) {
    QueueArgs a{};
    a.mats = p->d_mats;
    a.row_mat = p->row_mat;
    a.lists = p->lists;
    a.bin_off = offsets;
    a.q = queue_of(which);
    a.tile_pref = p->tile_pref + which * (kQueueMax + 1);
    a.bound = p->bound;
    a.nnz = p->nnz;
    a.gscan = p->nnz;
    a.c_col = p->c_col;
    a.c_val = p->c_val;
    a.lo = lo;
    a.prod = p->prod;
    a.esc_min = p->tune.esc_min_prod < 0 ? 0 : (p->tune.esc_min_prod == 0 ? kEscMinProd : p->tune.esc_min_prod);
    a.counter = p->qcount + which;
    a.flags = ctx->d_flags;
    cudaMemsetAsync(a.counter, 0, sizeof(unsigned long long), lc.stream);
    k_queue_prefix<<<1, 32, 0, lc.stream>>>(offsets, a.q, const_cast<int64_t*>(a.tile_pref));
    queue_dispatch(which, learned, &a, p->grid[learned ? 1 : 0][which], queue_smem(which), lc.stream);
    launches += 2;
  };
  auto exact_stages = [&](const int64_t* sym_key) {
    launch_binning(sym_key, R, INT64_MAX, kBinSymbolic, p->bp_sym, p->bin_of_row, counts, offsets, cursors,
                   p->lists, lc);
    launches += 3;
    run_queue(kQSymLarge, false);
    run_queue(kQSymSmall, false);
  };
  if (!p->learned) {
    exact_stages(p->bound);
    launch_binning(p->nnz, R, INT64_MAX, kBinNumeric, p->bp_num, p->bin_of_row, counts, offsets, cursors, p->lists,
                   lc);
    launch_excl_scan(p->nnz, R, p->nnz, p->scan_tmp, lc);
    launches += 7;
    run_queue(kQNumLarge, false);
    run_queue(kQNumMid, false);
    run_queue(kQNumSmall, false);
  } else {
    cudaMemsetAsync(p->lcount, 0, 2 * sizeof(unsigned long long), lc.stream);
    cudaMemsetAsync(p->need, 0, (size_t)std::max<int64_t>(R, 1), lc.stream);
    launch_learned_plan_batch(p->d_mats, p->row_mat, R, ctx->mlp_w16, p->tune.predict_margin, p->tune.predict_slack,
                              kBatchMaxBound, p->force_overflow, p->prod, p->cap, p->need, p->lcount, lc);
    launch_binning(p->cap, R, INT64_MAX, kBinLearned, p->bp_lrn, p->bin_of_row, counts, offsets, cursors, p->lists,
                   lc);
    launch_excl_scan(p->cap, R, p->slab_off, p->scan_tmp, lc);
    launches += 8;
    run_queue(kQNumLarge, true);
    run_queue(kQNumMid, true);
    run_queue(kQNumSmall, true);
    // the exact path for rows predicted beyond the tables and overflowed rows
    launch_mark_rows(p->retry, p->lcount + 1, p->need, lc);
    launch_mask_key(p->bound, p->need, R, p->mkey, lc);
    launches += 2;
    exact_stages(p->mkey);
    launch_mask_key(p->nnz, p->need, R, p->mkey, lc);
    launch_binning(p->mkey, R, INT64_MAX, kBinNumeric, p->bp_num, p->bin_of_row, counts, offsets, cursors, p->lists,
                   lc);
    launch_excl_scan(p->nnz, R, p->nnz, p->scan_tmp, lc);
    launches += 8;
    run_queue(kQNumLarge, false);
    run_queue(kQNumMid, false);
    run_queue(kQNumSmall, false);
    k_batch_compact<<<blocks_for(R, 8), 256, 0, lc.stream>>>(p->d_mats, p->row_mat, R, p->need, p->slab_off,
                                                            p->slab_col, p->slab_val, p->nnz, p->c_col, p->c_val);
    ++launches;
    cudaMemcpyAsync(p->h_lcount, p->lcount, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, lc.stream);
  }
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
    p->tune = default_tuning();
    // fuller queue tables keep more warps per SM (the autotuner's choice on
    // the 512 uneven products: 0.8, 129.9 ms against 138.4 ms at 0.65)
    p->tune.max_load = 0.8f;
    // the learned capacity already carries a margin over the prediction:
    // fuller tables at it match the plain tables' size
    p->tune.learned_load = 0.8f;
  }
  // every warp table size stays available on the batched path: a smaller
  // tuned maximum would send whole products to the one-by-one path
  p->tune.warp_table_max = default_tuning().warp_table_max;
  // symbolic binning: warp tables up to 2^11 slots at load <= 2/3, the CTA
  // table beyond; numeric: warp tables up to 2^10 slots at max_load, the CTA
  // table beyond (both CTA tables 2^13 slots at load <= 1/2)
  BinParams bs = without_block_bins(bin_params(p->tune));
  bs.warp_log_max = 11;
  bs.warp_cap = ((int64_t)1 << 11) * 2 / 3;
  bs.block_cap = kBatchMaxBound;
  p->bp_sym = bs;
  BinParams bn = without_block_bins(bin_params(p->tune));
  bn.warp_log_max = 10;
  bn.warp_cap = (int64_t)std::floor(1024.0 * bn.max_load);
  bn.block_min = bn.warp_cap;
  bn.blk_small_cap = kBatchMaxBound;
  bn.blk_large_cap = 0;
  p->bp_num = bn;
  // learned binning: as numeric, at the learned load factor
  BinParams bl = bn;
  bl.max_load = std::min(0.9f, std::max(0.1f, p->tune.learned_load > 0.f ? p->tune.learned_load : bn.max_load));
  bl.warp_cap = (int64_t)std::floor(1024.0 * bl.max_load);
  bl.block_min = bl.warp_cap;
  p->bp_lrn = bl;
  p->learned = o.algo == SPG_ALGO_LEARNED;
  p->force_overflow = o.force_overflow;
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
  // products with rows beyond the queue's tables go through the single path
  int64_t cbase = 0, rpbase = 0;
  p->c_base.assign((size_t)n, 0);
  for (int m = 0; m < n; ++m) {
    BatchMat& M = p->mats[(size_t)m];
    // the persistent kernels use 32-bit row offsets of B (nnz(B) < 2^31)
    if ((int64_t)hmax[(size_t)m] > kBatchMaxBound || !M.B.rp32) {
      p->individual.push_back(m);
      // keep its rows out of the persistent stages: an empty A view
      M.A.rows = 0;
    } else {
      p->batched.push_back(m);
    }
    M.c_base = cbase;
    M.rp_base = rpbase;
    p->c_base[(size_t)m] = cbase;
    if ((int64_t)hmax[(size_t)m] <= kBatchMaxBound && M.B.rp32) cbase += (int64_t)hsum[(size_t)m];
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
  // CTAs of every queue launch: as many as fit the SMs at once (set before
  // any capture)
  for (int form = 0; form < 2; ++form) {
    for (int w = 0; w < kQueues; ++w) {
      const size_t smem = queue_smem(w);
      const void* k = queue_dispatch(w, form == 1, nullptr, 0, 0, nullptr);
      SPG_CUDA(ctx, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      int per_sm = 0;
      SPG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kBlkThreads, smem));
      p->grid[form][w] = ctx->sms * std::max(1, per_sm);
    }
  }
  if (p->learned) {
    // capacities, slab offsets and a slab of the bound sum (the largest
    // capacity total), the exact-path marks and the retry list
    SPG_TRY(dmalloc(ctx, p, &p->cap, (size_t)R + 1));
    SPG_TRY(dmalloc(ctx, p, &p->slab_off, (size_t)R + 1));
    SPG_TRY(dmalloc(ctx, p, &p->need, (size_t)std::max<int64_t>(R, 1)));
    SPG_TRY(dmalloc(ctx, p, &p->mkey, (size_t)std::max<int64_t>(R, 1)));
    SPG_TRY(dmalloc(ctx, p, &p->retry, (size_t)std::max<int64_t>(R, 1)));
    SPG_TRY(dmalloc(ctx, p, &p->slab_col, (size_t)std::max<int64_t>(cbase, 1)));
    SPG_TRY(dmalloc(ctx, p, &p->slab_val, (size_t)std::max<int64_t>(cbase, 1)));
    SPG_TRY(dmalloc(ctx, p, &p->lcount, 2));
    SPG_CUDA(ctx, cudaMallocHost(&p->h_lcount, 2 * sizeof(unsigned long long)));
  }
  SPG_TRY(dmalloc(ctx, p, &p->tile_pref, (size_t)kQueues * (kQueueMax + 1)));
  SPG_TRY(dmalloc(ctx, p, &p->qcount, (size_t)kQueues));
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
  if (o.algo != SPG_ALGO_PLAIN && o.algo != SPG_ALGO_LEARNED)
    return fail(ctx, SPG_ERR_INVALID_ARG, "spg_multiply_batched runs the plain or learned method");
  if (report) {
    std::memset(report, 0, sizeof *report);
    report->algo = o.algo;
  }
  if (o.algo == SPG_ALGO_LEARNED) SPG_TRY(ensure_mlp(ctx));
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
    if (plan->learned && plan->R > 0) {
      // rows sized by the predictor, and those that overflowed their capacity
      report->rows_predicted = plan->R - (int64_t)plan->h_lcount[0];
      report->rows_overflow = (int64_t)plan->h_lcount[1];
    }
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
