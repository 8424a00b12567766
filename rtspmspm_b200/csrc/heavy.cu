// Heavy-row numeric pass through an HBM staging buffer.
//
// Rows whose output exceeds the warp tables are accumulated in dense column
// tiles (2^kTileShift columns, one warp per tile).  Instead of every tile
// rescanning its row of A (cost ~ nnz(A_i) x tiles), each heavy row's
// product stream is walked ONCE in canonical order (k ascending through A's
// row, then column ascending through B's row k) and every product (column,
// a*b) is written into its tile's bucket of the staging buffer, so a bucket
// holds its tile's products in canonical order.  A warp per (row, tile)
// then reads its bucket with coalesced loads and accumulates it exactly as
// the rescanning kernel would -- the same adds in the same order, so the
// result is bit-identical.
//
// Stages, per batch of heavy rows whose products fit the staging buffer:
//   count   (warp per chunk of kStageChunk A entries): products per tile;
//   offsets (CTA per row): bucket starts, and per chunk the first free
//           position of each bucket (chunks in order inside a bucket);
//   scatter (warp per chunk): the canonical walk, writing into the buckets;
//   accumulate (warp per (row, tile)): dense tile + bitmap, emitted sorted.
// Opt-in (spg_tuning.heavy_path = 1).  Measured on one B200 it is slower than
// the rescanning tile kernel on R-MAT (scale 17: 50.8 vs 13.2 ms, scale 20:
// 2.2 vs 0.45 s for the numeric stage): each scatter step writes its 32
// products into up to 32 different buckets of a buffer much larger than L2,
// so the writes reach DRAM as partial sectors.
// No reference counterpart beyond the any-hit multiply-accumulate
// (optixSpMSpM/src/optixSpMSpM/optixSpMSpM.cu:234-260).
#include <algorithm>
#include <vector>

#include "context.hpp"
#include "tile.cuh"

namespace spg {

constexpr int kStageChunk = 256;        // A entries per count/scatter chunk
constexpr int kStageWarps = 8;          // warps per CTA of the count/scatter kernels
constexpr int kStageMaxTiles = 4096;    // per-warp shared counters of the count/scatter kernels
constexpr int64_t kStageMaxProducts = int64_t(1) << 28;  // staging entries per batch (2 GB)

// Per heavy row: intermediate products and the number of chunks of A's row.
template <bool R32>
__global__ void k_heavy_prep(DCsr A, DCsr B, const int32_t* heavy_rows, int64_t nheavy, int64_t* prod_h,
                             int64_t* nch_h) {
  const int lane = lane_id();
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t h = gw; h < nheavy; h += nw) {
    const int32_t row = heavy_rows[h];
    const int64_t s = A.rp[row], e = A.rp[row + 1];
    int64_t sum = 0;
    for (int64_t p = s + lane; p < e; p += 32) {
      const int32_t k = A.col[p];
      sum += (int64_t)(RowOff<R32>::at(B, k + 1) - RowOff<R32>::at(B, k));
    }
    sum = warp_sum(sum);
    if (lane == 0) {
      prod_h[h] = sum;
      nch_h[h] = max((int64_t)1, (e - s + kStageChunk - 1) / kStageChunk);
    }
  }
}

// Heavy row of a chunk: the last h in [h0, h1) with chunk_base[h] <= gc.
__device__ __forceinline__ int64_t row_of_chunk(const int64_t* chunk_base, int64_t h0, int64_t h1, int64_t gc) {
  int64_t lo = h0, hi = h1;  // chunk_base[lo] <= gc < chunk_base[hi]
  while (hi - lo > 1) {
    const int64_t mid = (lo + hi) >> 1;
    if (chunk_base[mid] <= gc) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Count stage: products per tile of every chunk of the batch, counts[chunk *
// ntiles + t] (chunk relative to the batch).  Warp per chunk; per-warp shared
// counters.
template <bool R32>
__global__ void __launch_bounds__(kStageWarps * 32) k_heavy_count(DCsr A, DCsr B, const int32_t* heavy_rows,
                                                                 const int64_t* chunk_base, int64_t h0, int64_t h1,
                                                                 int ntiles, int32_t* counts, int* flags) {
  using Off = typename RowOff<R32>::T;
  extern __shared__ int32_t sm_cnt[];
  const int lane = lane_id();
  int32_t* cnt = sm_cnt + (threadIdx.x >> 5) * ntiles;
  for (int t = lane; t < ntiles; t += 32) cnt[t] = 0;
  __syncwarp();
  const int64_t c_first = chunk_base[h0], c_last = chunk_base[h1];
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t gc = c_first + gw; gc < c_last; gc += nw) {
    const int64_t h = row_of_chunk(chunk_base, h0, h1, gc);
    const int32_t row = heavy_rows[h];
    const int64_t s = A.rp[row], e = A.rp[row + 1];
    const int64_t cs = s + (gc - chunk_base[h]) * kStageChunk;
    const int64_t ce = min(e, cs + kStageChunk);
    for (int64_t base = cs; base < ce; base += 32) {
      const int64_t p = base + lane;
      Off bs = 0;
      int len = 0;
      if (p < ce) {
        const int32_t k = A.col[p];
        bs = RowOff<R32>::at(B, k);
        len = (int)(RowOff<R32>::at(B, k + 1) - bs);
      }
      for_each_col(B.col, bs, len, [&](int32_t c) {
        const int t = c >> kTileShift;
        if ((unsigned)t < (unsigned)ntiles) atomicAdd(&cnt[t], 1);
        else raise_flag(flags, kFlagBadIndex);
      });
    }
    __syncwarp();
    int32_t* out = counts + (gc - c_first) * ntiles;
    for (int t = lane; t < ntiles; t += 32) {
      out[t] = cnt[t];
      cnt[t] = 0;
    }
    __syncwarp();
  }
}

// Offsets stage: CTA per heavy row of the batch.  bucket[(h - h0) * (ntiles
// + 1) + t] = first staging position of tile t's bucket (the last entry is
// the row's end); counts[c][t] becomes the first position chunk c writes in
// bucket t.  Positions are relative to the batch's first product.
__global__ void k_heavy_offsets(const int64_t* chunk_base, const int64_t* prod_base, int64_t h0, int64_t h1,
                                int ntiles, int32_t* counts, int32_t* bucket) {
  extern __shared__ int32_t sm_tot[];
  __shared__ int32_t sh_part[1024 / 32 + 1];
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int64_t c_first = chunk_base[h0];
  for (int64_t h = h0 + blockIdx.x; h < h1; h += gridDim.x) {
    const int64_t cb = chunk_base[h] - c_first, ce = chunk_base[h + 1] - c_first;
    const int32_t row_base = (int32_t)(prod_base[h] - prod_base[h0]);
    for (int t = tid; t < ntiles; t += nthr) {
      int32_t sum = 0;
      for (int64_t c = cb; c < ce; ++c) sum += counts[c * ntiles + t];
      sm_tot[t] = sum;
    }
    __syncthreads();
    // exclusive scan of sm_tot over tiles: thread tid owns a contiguous run
    const int per = (ntiles + nthr - 1) / nthr;
    const int t0 = min(ntiles, tid * per), t1 = min(ntiles, t0 + per);
    int32_t run = 0;
    for (int t = t0; t < t1; ++t) run += sm_tot[t];
    int32_t incl = warp_incl_scan(run);
    if (lane_id() == 31) sh_part[tid >> 5] = incl;
    __syncthreads();
    if (tid < 32) {
      const int nwp = nthr >> 5;
      const int32_t v = tid < nwp ? sh_part[tid] : 0;
      const int32_t iv = warp_incl_scan(v);
      if (tid < nwp) sh_part[tid] = iv - v;
    }
    __syncthreads();
    int32_t pre = incl - run + sh_part[tid >> 5];
    int32_t* brow = bucket + (h - h0) * (int64_t)(ntiles + 1);
    for (int t = t0; t < t1; ++t) {
      const int32_t v = sm_tot[t];
      brow[t] = row_base + pre;
      // per-chunk first positions inside this bucket
      int32_t r = row_base + pre;
      for (int64_t c = cb; c < ce; ++c) {
        const int32_t x = counts[c * ntiles + t];
        counts[c * ntiles + t] = r;
        r += x;
      }
      pre += v;
    }
    if (tid == nthr - 1) brow[ntiles] = row_base + pre;
    __syncthreads();
  }
}

// Scatter stage: warp per chunk; the chunk's products in canonical order, 32
// consecutive ones per step (a flattened walk over 32 A entries at a time),
// each written at its tile's cursor.  Lanes sharing a tile take consecutive
// positions in lane order (= stream order).
template <bool R32>
__global__ void __launch_bounds__(kStageWarps * 32) k_heavy_scatter(DCsr A, DCsr B, const int32_t* heavy_rows,
                                                                   const int64_t* chunk_base, int64_t h0, int64_t h1,
                                                                   int ntiles, const int32_t* counts,
                                                                   int32_t* st_col, float* st_val) {
  using Off = typename RowOff<R32>::T;
  extern __shared__ int32_t sm_cur[];
  const int lane = lane_id();
  const unsigned lt = (1u << lane) - 1u;
  int32_t* cur = sm_cur + (threadIdx.x >> 5) * ntiles;
  const int64_t c_first = chunk_base[h0], c_last = chunk_base[h1];
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t gc = c_first + gw; gc < c_last; gc += nw) {
    const int32_t* first = counts + (gc - c_first) * ntiles;
    for (int t = lane; t < ntiles; t += 32) cur[t] = first[t];
    __syncwarp();
    const int64_t h = row_of_chunk(chunk_base, h0, h1, gc);
    const int32_t row = heavy_rows[h];
    const int64_t s = A.rp[row], e = A.rp[row + 1];
    const int64_t cs = s + (gc - chunk_base[h]) * kStageChunk;
    const int64_t ce = min(e, cs + kStageChunk);
    for (int64_t base = cs; base < ce; base += 32) {
      const int64_t p = base + lane;
      Off bs = 0;
      int len = 0;
      float a = 0.f;
      if (p < ce) {
        const int32_t k = A.col[p];
        a = A.val[p];
        bs = RowOff<R32>::at(B, k);
        len = (int)(RowOff<R32>::at(B, k + 1) - bs);
      }
      const int incl = warp_incl_scan(len);
      const int total = __shfl_sync(kFull, incl, 31);
      const int excl = incl - len;
      for (int b0 = 0; b0 < total; b0 += 32) {
        const int tt = b0 + lane;
        const bool act = tt < total;
        const int src = warp_upper_bound(incl, act ? tt : total - 1);
        const Off sbs = __shfl_sync(kFull, bs, src);
        const int sex = __shfl_sync(kFull, excl, src);
        const float sa = __shfl_sync(kFull, a, src);
        int32_t c = 0;
        float pr = 0.f;
        int t = -1 - lane;  // unique dummy for idle lanes
        if (act) {
          const Off q = sbs + (Off)(tt - sex);
          c = B.col[q];
          pr = prod_rn(sa, B.val[q]);
          t = c >> kTileShift;
          if ((unsigned)t >= (unsigned)ntiles) t = -1 - lane;  // flagged by the count stage
        }
        const unsigned grp = __match_any_sync(kFull, t);
        const int leader = __ffs(grp) - 1;
        const bool ok = act && t >= 0;
        int pos = 0;
        if (ok && lane == leader) {
          pos = cur[t];
          cur[t] = pos + __popc(grp);
        }
        pos = __shfl_sync(kFull, pos, leader) + __popc(grp & lt);
        if (ok) {
          st_col[pos] = c;
          st_val[pos] = pr;
        }
        __syncwarp();
      }
    }
  }
}

// Accumulate stage: one warp per (heavy row of the batch, tile) ticket; the
// bucket's products are read 64 at a time (coalesced) and added into the
// dense tile in order -- products of one step that hit the same column are
// grouped with __match_any_sync and added in lane order by the group's
// lowest lane -- then the tile is emitted into C.
__global__ void __launch_bounds__(kTileWarps * 32) k_heavy_accumulate(
    const int32_t* heavy_rows, int64_t h0, int64_t h1, const int32_t* big_slot, const int32_t* tile_cnt,
    const int32_t* tile_off, int ntiles, const int32_t* bucket, const int32_t* st_col, const float* st_val,
    const int64_t* c_rp, int32_t* c_col, float* c_val, unsigned long long* ticket, int* flags) {
  extern __shared__ uint32_t sm_tile[];
  const int lane = lane_id(), wib = threadIdx.x >> 5;
  float* acc = reinterpret_cast<float*>(sm_tile) + (size_t)wib * kTileWarpWords;
  uint32_t* bits = reinterpret_cast<uint32_t*>(acc + kTileCols);
  for (int s = lane; s < kTileCols; s += 32) acc[s] = 0.f;
  for (int s = lane; s < kTileWords; s += 32) bits[s] = 0u;
  __syncwarp();
  const int64_t total = (h1 - h0) * (int64_t)ntiles;
  for (;;) {
    unsigned long long tk = 0;
    if (lane == 0) tk = atomicAdd(ticket, 1ull);
    tk = __shfl_sync(kFull, tk, 0);
    if ((int64_t)tk >= total) break;
    const int64_t hl = (int64_t)tk / ntiles;
    const int tile = (int)((int64_t)tk % ntiles);
    const int32_t row = heavy_rows[h0 + hl];
    const int64_t slot = big_slot[row];
    const int want = tile_cnt[slot * ntiles + tile];
    const int32_t* brow = bucket + hl * (int64_t)(ntiles + 1);
    const int32_t b0 = brow[tile], b1 = brow[tile + 1];
    if (want == 0) {
      if (b1 > b0 && lane == 0) raise_flag(flags, kFlagCountDiff);
      continue;
    }
    const int32_t c0 = tile << kTileShift;
    for (int32_t q0 = b0; q0 < b1; q0 += 64) {
      int32_t off[2];
      float pr[2];
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int32_t q = q0 + u * 32 + lane;
        off[u] = -1 - lane;  // unique dummy for idle lanes
        pr[u] = 0.f;
        if (q < b1) {
          off[u] = st_col[q] - c0;
          pr[u] = st_val[q];
        }
      }
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        if (q0 + u * 32 >= b1) break;
        const bool act = q0 + u * 32 + lane < b1;
        const bool inb = (uint32_t)off[u] < (uint32_t)kTileCols;
        if (act && !inb) raise_flag(flags, kFlagBadIndex);
        const unsigned grp = __match_any_sync(kFull, off[u]);
        const bool lead = act && inb && (grp & ((1u << lane) - 1u)) == 0u;
        float v = lead ? acc[off[u]] : 0.f;
        v = group_sum_in_lane_order(grp, pr[u], v, lead);
        if (lead) {
          acc[off[u]] = v;
          atomicOr(&bits[off[u] >> 5], 1u << (off[u] & 31));
        }
        __syncwarp();
      }
    }
    tile_emit(acc, bits, c0, c_rp[row] + tile_off[slot * ntiles + tile], want, c_col, c_val, flags);
  }
}

// Host driver: returns with *done = false, having launched nothing, when the
// staged path does not apply (too many tiles for the shared counters, a row
// above the staging capacity, or too little free memory); the caller then
// runs the rescanning tile kernel.
spg_status heavy_staged(spg_ctx* ctx, const DCsr& A, const DCsr& B, const int32_t* heavy_rows, int64_t nheavy,
                        const int32_t* big_slot, const int32_t* tile_cnt, const int32_t* tile_off, int ntiles,
                        const int64_t* c_rp, int32_t* c_col, float* c_val, bool* done) {
  *done = false;
  if (nheavy == 0) {
    *done = true;
    return SPG_OK;
  }
  if (ntiles > kStageMaxTiles) return SPG_OK;
  const LaunchCtx lc = launch_ctx(ctx);
  DevBuf prod_h, nch_h, scan_tmp;
  SPG_TRY(prod_h.alloc(ctx, (size_t)(nheavy + 1) * 8));
  SPG_TRY(nch_h.alloc(ctx, (size_t)(nheavy + 1) * 8));
  SPG_TRY(scan_tmp.alloc(ctx, (size_t)scan_temp_elems(nheavy + 1) * 8));
  {
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((nheavy + 7) / 8, (int64_t)lc.sms * 16));
    if (B.rp32)
      k_heavy_prep<true><<<blocks, 256, 0, lc.stream>>>(A, B, heavy_rows, nheavy, prod_h.as<int64_t>(),
                                                         nch_h.as<int64_t>());
    else
      k_heavy_prep<false><<<blocks, 256, 0, lc.stream>>>(A, B, heavy_rows, nheavy, prod_h.as<int64_t>(),
                                                          nch_h.as<int64_t>());
  }
  launch_excl_scan(prod_h.as<int64_t>(), nheavy, prod_h.as<int64_t>(), scan_tmp.as<int64_t>(), lc);
  launch_excl_scan(nch_h.as<int64_t>(), nheavy, nch_h.as<int64_t>(), scan_tmp.as<int64_t>(), lc);
  ctx->launches += 9;
  std::vector<int64_t> pb((size_t)nheavy + 1), cb((size_t)nheavy + 1);
  SPG_CUDA(ctx, cudaMemcpyAsync(pb.data(), prod_h.get(), pb.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
  SPG_CUDA(ctx, cudaMemcpyAsync(cb.data(), nch_h.get(), cb.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
  SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  // batches of consecutive heavy rows within the staging capacity
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  const int64_t cap = std::min<int64_t>(kStageMaxProducts, (int64_t)(free_b / 4) / 8);
  if (cap < 1) return SPG_OK;
  std::vector<int64_t> cuts{0};
  int64_t max_chunks = 0, max_rows = 0;
  for (int64_t h = 0; h < nheavy;) {
    if (pb[(size_t)h + 1] - pb[(size_t)h] > cap) return SPG_OK;  // a row above the capacity
    int64_t e = std::upper_bound(pb.begin() + h + 1, pb.end(), pb[(size_t)h] + cap) - pb.begin() - 1;
    e = std::max<int64_t>(e, h + 1);
    max_chunks = std::max<int64_t>(max_chunks, cb[(size_t)e] - cb[(size_t)h]);
    max_rows = std::max<int64_t>(max_rows, e - h);
    cuts.push_back(e);
    h = e;
  }
  int64_t max_prod = 0;
  for (size_t i = 0; i + 1 < cuts.size(); ++i)
    max_prod = std::max<int64_t>(max_prod, pb[(size_t)cuts[i + 1]] - pb[(size_t)cuts[i]]);
  DevBuf st_col, st_val, counts, bucket;
  SPG_TRY(st_col.alloc(ctx, (size_t)std::max<int64_t>(max_prod, 1) * 4));
  SPG_TRY(st_val.alloc(ctx, (size_t)std::max<int64_t>(max_prod, 1) * 4));
  SPG_TRY(counts.alloc(ctx, (size_t)std::max<int64_t>(max_chunks, 1) * ntiles * 4));
  SPG_TRY(bucket.alloc(ctx, (size_t)std::max<int64_t>(max_rows, 1) * (ntiles + 1) * 4));
  const size_t cnt_smem = (size_t)kStageWarps * ntiles * 4;
  const size_t tile_smem = (size_t)kTileWarps * kTileWarpWords * 4;
  const size_t off_smem = (size_t)ntiles * 4;
  if (B.rp32) {
    cudaFuncSetAttribute(k_heavy_count<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cnt_smem);
    cudaFuncSetAttribute(k_heavy_scatter<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cnt_smem);
  } else {
    cudaFuncSetAttribute(k_heavy_count<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cnt_smem);
    cudaFuncSetAttribute(k_heavy_scatter<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cnt_smem);
  }
  cudaFuncSetAttribute(k_heavy_accumulate, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tile_smem);
  int acc_per_sm = 0, cs_per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&acc_per_sm, k_heavy_accumulate, kTileWarps * 32, tile_smem);
  if (B.rp32)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cs_per_sm, k_heavy_scatter<true>, kStageWarps * 32, cnt_smem);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cs_per_sm, k_heavy_scatter<false>, kStageWarps * 32, cnt_smem);
  acc_per_sm = std::max(1, acc_per_sm);
  cs_per_sm = std::max(1, cs_per_sm);
  const int64_t* chunk_base = nch_h.as<int64_t>();
  const int64_t* prod_base = prod_h.as<int64_t>();
  for (size_t i = 0; i + 1 < cuts.size(); ++i) {
    const int64_t h0 = cuts[i], h1 = cuts[i + 1];
    const int64_t nchunks = cb[(size_t)h1] - cb[(size_t)h0];
    const int cs_blocks =
        (int)std::max<int64_t>(1, std::min<int64_t>((nchunks + kStageWarps - 1) / kStageWarps, (int64_t)lc.sms * cs_per_sm));
    if (B.rp32) {
      k_heavy_count<true><<<cs_blocks, kStageWarps * 32, cnt_smem, lc.stream>>>(
          A, B, heavy_rows, chunk_base, h0, h1, ntiles, counts.as<int32_t>(), ctx->d_flags);
    } else {
      k_heavy_count<false><<<cs_blocks, kStageWarps * 32, cnt_smem, lc.stream>>>(
          A, B, heavy_rows, chunk_base, h0, h1, ntiles, counts.as<int32_t>(), ctx->d_flags);
    }
    const int off_blocks = (int)std::max<int64_t>(1, std::min<int64_t>(h1 - h0, (int64_t)lc.sms * 4));
    k_heavy_offsets<<<off_blocks, 256, off_smem, lc.stream>>>(chunk_base, prod_base, h0, h1, ntiles,
                                                               counts.as<int32_t>(), bucket.as<int32_t>());
    if (B.rp32) {
      k_heavy_scatter<true><<<cs_blocks, kStageWarps * 32, cnt_smem, lc.stream>>>(
          A, B, heavy_rows, chunk_base, h0, h1, ntiles, counts.as<int32_t>(), st_col.as<int32_t>(),
          st_val.as<float>());
    } else {
      k_heavy_scatter<false><<<cs_blocks, kStageWarps * 32, cnt_smem, lc.stream>>>(
          A, B, heavy_rows, chunk_base, h0, h1, ntiles, counts.as<int32_t>(), st_col.as<int32_t>(),
          st_val.as<float>());
    }
    SPG_CUDA(ctx, cudaMemsetAsync(ctx->d_counter, 0, 8, lc.stream));
    const int64_t tickets = (h1 - h0) * (int64_t)ntiles;
    const int acc_blocks = (int)std::max<int64_t>(
        1, std::min<int64_t>((tickets + kTileWarps - 1) / kTileWarps, (int64_t)lc.sms * acc_per_sm));
    k_heavy_accumulate<<<acc_blocks, kTileWarps * 32, tile_smem, lc.stream>>>(
        heavy_rows, h0, h1, big_slot, tile_cnt, tile_off, ntiles, bucket.as<int32_t>(), st_col.as<int32_t>(),
        st_val.as<float>(), c_rp, c_col, c_val, ctx->d_counter, ctx->d_flags);
    ctx->launches += 4;
  }
  SPG_CUDA(ctx, cudaGetLastError());
  *done = true;
  return SPG_OK;
}

}  // namespace spg
