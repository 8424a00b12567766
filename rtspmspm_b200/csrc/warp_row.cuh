// Per-row warp accumulators shared by the single-product kernels and the
// batched persistent kernels.  One warp owns one output row and a hash table
// of 2^LOGT slots in shared memory.
#pragma once

#include "common.cuh"

namespace spg {

// Prefetch depth: B-row steps whose first 32 entries are loaded before any
// of them is inserted, so a warp keeps kPrefetch independent loads in flight
// instead of one dependent load per step.
constexpr int kPrefetch = 8;

// Exact number of distinct output columns of `row` (keys-only table).
// epoch >= 0: epoch-tagged table (no clearing; caller advances the epoch and
// clears the table when it wraps).  epoch < 0: plain keys, cleared here.
template <int LOGT>
__device__ __forceinline__ int symbolic_row(const DCsr& A, const DCsr& B, int32_t row, int32_t* keys, int epoch,
                                            int* flags) {
  constexpr int T = 1 << LOGT;
  const int lane = lane_id();
  const int64_t s = A.rp[row], e = A.rp[row + 1];
  int cnt = 0;
  auto insert = [&](int32_t j) {
    if (epoch >= 0) {
      cnt += tagged_insert(keys, LOGT, j, (uint32_t)epoch, flags);
    } else {
      bool fresh;
      hash_insert(keys, LOGT, j, fresh, flags);
      cnt += fresh;
    }
  };
  for (int64_t base = s; base < e; base += 32) {
    const int64_t p = base + lane;
    int64_t bs = 0, be = 0;
    if (p < e) {
      const int32_t k = A.col[p];
      bs = B.rp[k];
      be = B.rp[k + 1];
    }
    const int n = (int)min((int64_t)32, e - base);
    for (int t0 = 0; t0 < n; t0 += 2 * kPrefetch) {
      int32_t c[2 * kPrefetch];
#pragma unroll
      for (int d = 0; d < 2 * kPrefetch; ++d) {
        const int t = t0 + d;
        const int64_t bst = __shfl_sync(kFull, bs, t & 31), ben = __shfl_sync(kFull, be, t & 31);
        const int64_t q = bst + lane;
        c[d] = (t < n && q < ben) ? B.col[q] : -1;
      }
#pragma unroll
      for (int d = 0; d < 2 * kPrefetch; ++d)
        if (c[d] >= 0) insert(c[d]);
      // entries beyond the first 32 of long B rows (symbolic order is free)
      for (int d = 0; d < 2 * kPrefetch && t0 + d < n; ++d) {
        const int t = t0 + d;
        const int64_t bst = __shfl_sync(kFull, bs, t), ben = __shfl_sync(kFull, be, t);
        for (int64_t q = bst + 32 + lane; q < ben; q += 32) insert(B.col[q]);
      }
    }
  }
  __syncwarp();
  cnt = warp_sum(cnt);
  if (epoch < 0) {
    for (int s2 = lane; s2 < T; s2 += 32) keys[s2] = kEmpty;
    __syncwarp();
  }
  return cnt;
}

// Accumulates row `row` into the warp's table in canonical order: k-serial
// (one B row at a time), lanes parallel over the columns of B_k.  Within
// one B row all columns are distinct, so each slot receives at most one
// product per step; __syncwarp orders the steps.  The first 32 entries of
// kPrefetch consecutive B rows are loaded before the group is inserted.
// With cap >= 0 the row aborts (returns false) as soon as more than `cap`
// distinct columns appear or the table fills: the learned path's overflow.
template <int LOGT>
__device__ __forceinline__ bool accumulate_row(const DCsr& A, const DCsr& B, int32_t row, int32_t* keys, float* vals,
                                               int64_t cap, int* flags, int& distinct) {
  const int lane = lane_id();
  const int64_t s = A.rp[row], e = A.rp[row + 1];
  int count = 0;
  for (int64_t base = s; base < e; base += 32) {
    const int64_t p = base + lane;
    int64_t bs = 0, be = 0;
    float a = 0.f;
    if (p < e) {
      const int32_t k = A.col[p];
      a = A.val[p];
      bs = B.rp[k];
      be = B.rp[k + 1];
    }
    const int n = (int)min((int64_t)32, e - base);
    for (int t0 = 0; t0 < n; t0 += kPrefetch) {
      int32_t c[kPrefetch];
      float v[kPrefetch];
#pragma unroll
      for (int d = 0; d < kPrefetch; ++d) {
        const int t = t0 + d;
        const int64_t bst = __shfl_sync(kFull, bs, t & 31), ben = __shfl_sync(kFull, be, t & 31);
        const int64_t q = bst + lane;
        const bool ok = t < n && q < ben;
        c[d] = ok ? B.col[q] : -1;
        v[d] = ok ? B.val[q] : 0.f;
      }
#pragma unroll
      for (int d = 0; d < kPrefetch; ++d) {
        const int t = t0 + d;
        if (t >= n) break;  // warp-uniform
        const float at = __shfl_sync(kFull, a, t);
        const int64_t bst = __shfl_sync(kFull, bs, t), ben = __shfl_sync(kFull, be, t);
        // first chunk (prefetched), then the rest of B_k, all before B_{k+1}
        for (int64_t q0 = bst; q0 < ben; q0 += 32) {
          const int64_t q = q0 + lane;
          int32_t j = -1;
          float bv = 0.f;
          if (q0 == bst) {
            j = c[d];
            bv = v[d];
          } else if (q < ben) {
            j = B.col[q];
            bv = B.val[q];
          }
          bool fresh = false, failed = false;
          if (j >= 0) {
            const float pr = prod_rn(at, bv);
            const int slot = hash_insert(keys, LOGT, j, fresh, cap >= 0 ? nullptr : flags);
            if (slot >= 0) vals[slot] = add_rn(vals[slot], pr);
            else failed = true;
          }
          count += __popc(__ballot_sync(kFull, fresh));
          if (cap >= 0 && (__any_sync(kFull, failed) || count > cap)) {
            __syncwarp();
            distinct = count;
            return false;
          }
        }
        __syncwarp();
      }
    }
  }
  distinct = count;
  return true;
}

// Moves the occupied slots to the front of the table (clearing the rest)
// and returns how many there are.
template <int LOGT>
__device__ __forceinline__ int compact_table(int32_t* keys, float* vals) {
  constexpr int T = 1 << LOGT;
  const int lane = lane_id();
  int n = 0;
  for (int base = 0; base < T; base += 32) {
    const int s = base + lane;
    const int32_t k = keys[s];
    const float v = vals[s];
    keys[s] = kEmpty;
    vals[s] = 0.f;
    const bool occ = k != kEmpty;
    const unsigned m = __ballot_sync(kFull, occ);
    __syncwarp();
    if (occ) {
      const int pos = n + __popc(m & ((1u << lane) - 1u));
      keys[pos] = k;
      vals[pos] = v;
    }
    n += __popc(m);
    __syncwarp();
  }
  return n;
}

template <int LOGT>
__device__ __forceinline__ void reset_front(int32_t* keys, float* vals, int n) {
  constexpr int T = 1 << LOGT;
  int np2 = 1;
  while (np2 < n) np2 <<= 1;
  if (np2 > T) np2 = T;
  for (int s = lane_id(); s < np2; s += 32) {
    keys[s] = kEmpty;
    vals[s] = 0.f;
  }
  __syncwarp();
}

// Numeric row with exact output size `want`: canonical accumulation, sort,
// write `want` entries to (out_col, out_val).  Leaves the table cleared.
template <int LOGT>
__device__ __forceinline__ void numeric_row(const DCsr& A, const DCsr& B, int32_t row, int32_t* keys, float* vals,
                                            int32_t* out_col, float* out_val, int64_t want, int* flags) {
  constexpr int T = 1 << LOGT;
  const int lane = lane_id();
  int distinct;
  accumulate_row<LOGT>(A, B, row, keys, vals, -1, flags, distinct);
  const int n = compact_table<LOGT>(keys, vals);
  if (n != want && lane == 0) raise_flag(flags, kFlagCountDiff);
  warp_sort_pairs(keys, vals, n, T);
  const int nw_out = (int)min((int64_t)n, want);
  for (int t = lane; t < nw_out; t += 32) {
    out_col[t] = keys[t];
    out_val[t] = vals[t];
  }
  __syncwarp();
  reset_front<LOGT>(keys, vals, n);
}

}  // namespace spg
