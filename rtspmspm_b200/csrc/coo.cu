// COO -> CSR on the GPU: entries in any order become CSR with sorted
// columns, duplicate (i, j) pairs summed in FP32 in the order given.
//
// Replaces the reference's conversion step: it uploads the parsed COO and
// calls cusparseXcoo2csr (cuSparse/src/main.cpp:439-442), which needs
// row-sorted input and keeps duplicates; the reference's files come
// column-major (the reader sorts them on the host first).  Here the entries
// are ordered by a stable LSD radix sort on the key (row << 32) | column,
// 8 bits per pass over the bits the shape needs, so equal keys keep their
// input order; each run of equal keys is then folded left to right (the
// first value, plus the second, ...) exactly as the host reader folds
// duplicates, and row pointers come from the sorted rows.
#include <algorithm>
#include <cstring>
#include <vector>

#include "context.hpp"

namespace spg {
namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 8;                        // per lane
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 entries per CTA
constexpr int kDigits = 256;
constexpr int kScatterSmem = kSortTile * (8 + 4);  // the tile's keys and values in digit order

__global__ void k_coo_keys(const int32_t* ri, const int32_t* ci, int64_t n, int64_t rows, int64_t cols, uint64_t* key,
                           int* flags) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t r = ri[i], c = ci[i];
    if (r < 0 || r >= rows || c < 0 || c >= cols) {
      atomicOr(flags, kFlagBadIndex);
      key[i] = 0;
    } else {
      key[i] = ((uint64_t)(uint32_t)r << 32) | (uint32_t)c;
    }
  }
}

// Digit counts of each tile: hist[d * ntiles + tile].
__global__ void __launch_bounds__(kSortThreads) k_radix_hist(const uint64_t* key, int64_t n, int shift, int64_t ntiles,
                                                             int64_t* hist) {
  __shared__ int cnt[kDigits];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  const int64_t t0 = blockIdx.x * (int64_t)kSortTile;
  for (int q = threadIdx.x; q < kSortTile; q += kSortThreads) {
    const int64_t i = t0 + q;
    if (i < n) atomicAdd(&cnt[(int)((key[i] >> shift) & 0xffu)], 1);
  }
  __syncthreads();
  hist[(int64_t)threadIdx.x * ntiles + blockIdx.x] = cnt[threadIdx.x];
}

// Stable scatter of one tile: warp w owns entries [w * 32 * kSortItems, (w + 1) * 32 * kSortItems)
// of the tile, taken 32 consecutive at a time, so an entry's rank among the
// tile's entries of its digit follows (warp, step, lane) = input order.  The
// tile is first ordered by digit in shared memory (entry at tile position
// lp = the digit's first position in the tile + the counts of earlier warps
// + the entry's rank), then written out by consecutive threads, so each
// digit's run of the tile goes to consecutive global positions (coalesced
// stores; scattering straight from registers ran at 1.1 TB/s).  off:
// exclusive scan of hist (digit-major), the first output position of each
// (digit, tile).  Dynamic shared memory: kSortTile keys and values.
__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(const uint64_t* kin, const float* vin, int64_t n,
                                                                int shift, int64_t ntiles, const int64_t* off,
                                                                uint64_t* kout, float* vout) {
  __shared__ int base[kSortWarps][kDigits];
  __shared__ int first[kDigits];  // the digit's first position in the tile's digit order
  extern __shared__ uint64_t sm_sort[];
  uint64_t* sk = sm_sort;
  float* sv = reinterpret_cast<float*>(sm_sort + kSortTile);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  for (int d = lane; d < kDigits; d += 32) base[w][d] = 0;
  __syncwarp();
  const int64_t t0 = blockIdx.x * (int64_t)kSortTile;
  const int64_t w0 = t0 + (int64_t)w * (kSortItems * 32);
  uint64_t k[kSortItems];
  float v[kSortItems];
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    const int64_t i = w0 + j * 32 + lane;
    k[j] = i < n ? kin[i] : 0;
    v[j] = i < n ? vin[i] : 0.f;
  }
  // the warp's count per digit
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    const bool act = w0 + j * 32 + lane < n;
    const int d = act ? (int)((k[j] >> shift) & 0xffu) : kDigits + lane;
    const unsigned grp = __match_any_sync(kFull, d);
    if (act && (grp & lt) == 0u) base[w][d] += __popc(grp);
    __syncwarp();
  }
  __syncthreads();
  // per digit: its total in the tile and, per warp, the start of the warp's entries
  {
    const int d = threadIdx.x;
    int run = 0;
#pragma unroll
    for (int x = 0; x < kSortWarps; ++x) {
      const int c = base[x][d];
      base[x][d] = run;
      run += c;
    }
    // exclusive scan of the digit totals across the CTA (digit d = thread d)
    const int incl = warp_incl_scan(run);
    __shared__ int wtot[kSortWarps];
    if (lane == 31) wtot[w] = incl;
    __syncthreads();
    int pre = 0;
#pragma unroll
    for (int x = 0; x < kSortWarps; ++x) pre += x < w ? wtot[x] : 0;
    first[d] = pre + incl - run;
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kDigits; d += kSortThreads)
    for (int x = 0; x < kSortWarps; ++x) base[x][d] += first[d];
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    const bool act = w0 + j * 32 + lane < n;
    const int d = act ? (int)((k[j] >> shift) & 0xffu) : kDigits + lane;
    const unsigned grp = __match_any_sync(kFull, d);
    int lp = 0;
    if (act) lp = base[w][d] + __popc(grp & lt);
    __syncwarp();
    if (act) {
      sk[lp] = k[j];
      sv[lp] = v[j];
      if ((grp & lt) == 0u) base[w][d] += __popc(grp);
    }
    __syncwarp();
  }
  __syncthreads();
  // the tile in digit order, written by consecutive threads
  const int cnt = (int)min((int64_t)kSortTile, n - t0);
  for (int q = threadIdx.x; q < cnt; q += kSortThreads) {
    const uint64_t key = sk[q];
    const int d = (int)((key >> shift) & 0xffu);
    const int64_t pos = off[(int64_t)d * ntiles + blockIdx.x] + (q - first[d]);
    kout[pos] = key;
    vout[pos] = sv[q];
  }
}

// head[i] = 1 where entry i starts a run of equal keys.
__global__ void k_run_heads(const uint64_t* key, int64_t n, int64_t* head) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    head[i] = (i == 0 || key[i] != key[i - 1]) ? 1 : 0;
}

// One thread per run: its column and the left fold of its values into
// output entry pos[i]; the entry's row into urow.
__global__ void k_fold_runs(const uint64_t* key, const float* val, int64_t n, const int64_t* pos, int32_t* col,
                            float* out_val, int32_t* urow) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = key[i];
    if (i > 0 && key[i - 1] == k) continue;
    float s = val[i];
    for (int64_t q = i + 1; q < n && key[q] == k; ++q) s = __fadd_rn(s, val[q]);
    const int64_t u = pos[i];
    col[u] = (int32_t)(uint32_t)(k & 0xffffffffu);
    out_val[u] = s;
    urow[u] = (int32_t)(k >> 32);
  }
}

// Row pointers from the rows of the m sorted unique entries: entry u opens
// rows (urow[u - 1], urow[u]]; the rows after the last entry end at m.
__global__ void k_rp_from_rows(const int32_t* urow, int64_t m, int64_t rows, int64_t* rp) {
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u <= m; u += (int64_t)gridDim.x * blockDim.x) {
    const int64_t prev = u == 0 ? -1 : (int64_t)urow[u - 1];
    const int64_t cur = u == m ? rows : (int64_t)urow[u];
    for (int64_t r = prev + 1; r <= cur; ++r) rp[r] = u;
  }
}

int bits_for(int64_t n) {
  int b = 0;
  while (b < 62 && ((int64_t)1 << b) < n) ++b;
  return b;
}

int blocks_for(int64_t n, int sms) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sms * 8)); }

}  // namespace

// COO (device arrays) -> device CSR; see the file comment.
spg_status coo_to_csr_device(spg_ctx* ctx, int64_t rows, int64_t cols, int64_t n, const int32_t* ri, const int32_t* ci,
                             const float* vi, spg_csr* out) {
  const LaunchCtx lc = launch_ctx(ctx);
  DevBuf k0, k1, v0, v1;
  SPG_TRY(k0.alloc(ctx, (size_t)std::max<int64_t>(n, 1) * 8));
  SPG_TRY(k1.alloc(ctx, (size_t)std::max<int64_t>(n, 1) * 8));
  SPG_TRY(v0.alloc(ctx, (size_t)std::max<int64_t>(n, 1) * 4));
  SPG_TRY(v1.alloc(ctx, (size_t)std::max<int64_t>(n, 1) * 4));
  if (n > 0) {
    k_coo_keys<<<blocks_for(n, lc.sms), 256, 0, lc.stream>>>(ri, ci, n, rows, cols, k0.as<uint64_t>(), ctx->d_flags);
    SPG_CUDA(ctx, cudaMemcpyAsync(v0.get(), vi, (size_t)n * 4, cudaMemcpyDeviceToDevice, ctx->stream));
  }
  // LSD passes over the column bits, then over the row bits
  const int cbits = bits_for(cols), rbits = bits_for(rows);
  const int64_t ntiles = (n + kSortTile - 1) / kSortTile;
  DevBuf hist, tmp;
  SPG_TRY(hist.alloc(ctx, (size_t)std::max<int64_t>(kDigits * ntiles + 1, 1) * 8));
  SPG_TRY(tmp.alloc(ctx, (size_t)scan_temp_elems(std::max<int64_t>(kDigits * ntiles, n) + 1) * 8));
  uint64_t* kin = k0.as<uint64_t>();
  uint64_t* kout = k1.as<uint64_t>();
  float* vin = v0.as<float>();
  float* vout = v1.as<float>();
  std::vector<int> shifts;
  for (int s = 0; s < cbits; s += 8) shifts.push_back(s);
  for (int s = 0; s < rbits; s += 8) shifts.push_back(32 + s);
  if (n > 1) {
    SPG_CUDA(ctx, cudaFuncSetAttribute(k_radix_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, kScatterSmem));
    for (int shift : shifts) {
      k_radix_hist<<<(unsigned)ntiles, kSortThreads, 0, lc.stream>>>(kin, n, shift, ntiles, hist.as<int64_t>());
      launch_excl_scan(hist.as<int64_t>(), kDigits * ntiles, hist.as<int64_t>(), tmp.as<int64_t>(), lc);
      k_radix_scatter<<<(unsigned)ntiles, kSortThreads, kScatterSmem, lc.stream>>>(kin, vin, n, shift, ntiles,
                                                                        hist.as<int64_t>(), kout, vout);
      std::swap(kin, kout);
      std::swap(vin, vout);
    }
  }
  // runs of equal keys -> unique entries
  DevBuf pos;
  SPG_TRY(pos.alloc(ctx, (size_t)(n + 1) * 8));
  if (n > 0) k_run_heads<<<blocks_for(n, lc.sms), 256, 0, lc.stream>>>(kin, n, pos.as<int64_t>());
  launch_excl_scan(pos.as<int64_t>(), n, pos.as<int64_t>(), tmp.as<int64_t>(), lc);
  int64_t m = 0;
  SPG_TRY(stage_read(ctx, ctx->h_stage + 52, pos.as<int64_t>() + n, 8));
  int f = 0;
  SPG_TRY(stage_read(ctx, ctx->h_stage + 53, ctx->d_flags, 4));
  SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  m = ctx->h_stage[52];
  std::memcpy(&f, &ctx->h_stage[53], sizeof f);
  if (f) {
    SPG_CUDA(ctx, cudaMemsetAsync(ctx->d_flags, 0, sizeof(int), ctx->stream));
    if (f & kFlagBadIndex) return fail(ctx, SPG_ERR_INVALID_ARG, "COO entry outside [0, rows) x [0, cols)");
  }
  DevBuf col, val, urow, rp;
  SPG_TRY(col.alloc(ctx, (size_t)m * 4));
  SPG_TRY(val.alloc(ctx, (size_t)m * 4));
  SPG_TRY(urow.alloc(ctx, (size_t)std::max<int64_t>(m, 1) * 4));
  SPG_TRY(rp.alloc(ctx, (size_t)(rows + 1) * 8));
  if (n > 0)
    k_fold_runs<<<blocks_for(n, lc.sms), 256, 0, lc.stream>>>(kin, vin, n, pos.as<int64_t>(), col.as<int32_t>(),
                                                               val.as<float>(), urow.as<int32_t>());
  k_rp_from_rows<<<blocks_for(m + 1, lc.sms), 256, 0, lc.stream>>>(urow.as<int32_t>(), m, rows, rp.as<int64_t>());
  SPG_CUDA(ctx, cudaGetLastError());
  SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  std::memset(out, 0, sizeof *out);
  out->rows = rows;
  out->cols = cols;
  out->nnz = m;
  out->capacity = m;
  out->index_bits = 64;
  out->location = SPG_DEVICE;
  out->row_ptr = rp.release();
  out->col_idx = static_cast<int32_t*>(col.release());
  out->val = static_cast<float*>(val.release());
  out->owner = 1;
  return SPG_OK;
}

}  // namespace spg

extern "C" spg_status spg_coo_to_csr(spg_ctx* ctx, int64_t rows, int64_t cols, int64_t n, const int32_t* row_idx,
                                     const int32_t* col_idx, const float* val, int32_t location, spg_csr* out) {
  using namespace spg;
  if (!ctx || !out) return SPG_ERR_INVALID_ARG;
  std::memset(out, 0, sizeof *out);
  if (rows < 0 || cols < 0 || n < 0) return fail(ctx, SPG_ERR_INVALID_ARG, "negative dimension");
  if (rows > INT32_MAX || cols > INT32_MAX) return fail(ctx, SPG_ERR_UNSUPPORTED, "more than 2^31-1 rows or columns");
  if (n > 0 && (!row_idx || !col_idx || !val)) return fail(ctx, SPG_ERR_INVALID_ARG, "null COO array");
  if (location != SPG_HOST && location != SPG_DEVICE) return fail(ctx, SPG_ERR_INVALID_ARG, "bad location");
  SPG_CUDA(ctx, cudaSetDevice(ctx->device));
  if (location == SPG_DEVICE) return coo_to_csr_device(ctx, rows, cols, n, row_idx, col_idx, val, out);
  DevBuf ri, ci, vi;
  SPG_TRY(ri.alloc(ctx, (size_t)n * 4));
  SPG_TRY(ci.alloc(ctx, (size_t)n * 4));
  SPG_TRY(vi.alloc(ctx, (size_t)n * 4));
  if (n > 0) {
    SPG_CUDA(ctx, cudaMemcpyAsync(ri.get(), row_idx, (size_t)n * 4, cudaMemcpyHostToDevice, ctx->stream));
    SPG_CUDA(ctx, cudaMemcpyAsync(ci.get(), col_idx, (size_t)n * 4, cudaMemcpyHostToDevice, ctx->stream));
    SPG_CUDA(ctx, cudaMemcpyAsync(vi.get(), val, (size_t)n * 4, cudaMemcpyHostToDevice, ctx->stream));
  }
  return coo_to_csr_device(ctx, rows, cols, n, ri.as<int32_t>(), ci.as<int32_t>(), vi.as<float>(), out);
}
