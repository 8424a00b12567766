// Dense column-tile accumulator shared by the heavy-row numeric kernels: a
// warp owns 2^kTileShift floats, their occupancy bitmap and a 32-float
// stage in shared memory.
#pragma once

#include "common.cuh"

namespace spg {

// 32-bit words of shared memory per warp: floats, bitmap, stage.
constexpr int kTileWarpWords = kTileCols + kTileWords + 32;

// Position of the r-th (0-based) set bit of w; requires r < popc(w).
__device__ __forceinline__ int nth_set_bit(uint32_t w, int r) {
  int pos = 0;
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    const int c = __popc(w & ((1u << s) - 1u));
    if (r >= c) {
      r -= c;
      w >>= s;
      pos += s;
    }
  }
  return pos;
}

// Writes the tile's marked columns (c0 + offset) and values to
// out_col/out_val[out, out + want) in column order, 32 bitmap words (1024
// columns) per round with lanes on consecutive entries (coalesced stores),
// and clears the floats and the bitmap as they are read.  A count other
// than `want` raises kFlagCountDiff (nothing is written past want).
__device__ __forceinline__ void tile_emit(float* acc, uint32_t* bits, int32_t c0, int64_t out, int want,
                                          int32_t* out_col, float* out_val, int* flags) {
  const int lane = lane_id();
  int64_t pos = out;
  const int64_t lim = out + want;
  int found = 0;
#pragma unroll 1
  for (int g = 0; g < kTileWords; g += 32) {
    const uint32_t wd = bits[g + lane];
    const int c = __popc(wd);
    const int inc = warp_incl_scan(c);
    const int tot = __shfl_sync(kFull, inc, 31);
    const int exc = inc - c;
    for (int e0 = 0; e0 < tot; e0 += 32) {
      const int ei = e0 + lane;
      const bool act = ei < tot;
      const int src = warp_upper_bound(inc, act ? ei : tot - 1);
      const uint32_t sw = __shfl_sync(kFull, wd, src);
      const int sex = __shfl_sync(kFull, exc, src);
      if (act) {
        const int off = ((g + src) << 5) + nth_set_bit(sw, ei - sex);
        if (pos + ei < lim) {
          out_col[pos + ei] = c0 + off;
          out_val[pos + ei] = acc[off];
        }
        acc[off] = 0.f;
      }
    }
    bits[g + lane] = 0u;
    pos += tot;
    found += tot;
  }
  if (found != want && lane == 0) raise_flag(flags, kFlagCountDiff);
  __syncwarp();
}

}  // namespace spg
