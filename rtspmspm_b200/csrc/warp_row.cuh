// Per-row warp accumulators shared by the single-product kernels and the
// batched persistent kernels.  One warp owns one output row and, in shared
// memory, a hash table of 2^LOGT (key, value) slots plus a list of the
// row's distinct columns in first-seen order.
//
// Keys are epoch-tagged when the columns fit in 24 bits: a slot holds
// (epoch << 24) | column and a slot of another epoch counts as empty, so
// tables are never cleared between rows (the caller advances the epoch and
// wipes the keys once every 255 rows).  A fresh claim *sets* the value
// (0 + product, as the canonical sum starts from 0), so values need no
// clearing either.  R32 selects 32-bit row offsets of B (nnz(B) < 2^31).
#pragma once

#include "common.cuh"

namespace spg {

constexpr int kNoEpoch = -1;  // plain keys (columns >= 2^24): cleared per row

// Insert into a numeric table; returns the slot (or -1 if the table is full)
// and whether the key was claimed by this call.
__device__ __forceinline__ int table_insert(int32_t* keys, int log_t, int32_t j, int epoch, bool& fresh) {
  const uint32_t mask = (1u << log_t) - 1u;
  const int32_t want = epoch >= 0 ? (int32_t)(((uint32_t)epoch << 24) | (uint32_t)j) : j;
  uint32_t s = hash_slot(j, log_t);
  fresh = false;
  for (uint32_t probe = 0; probe <= mask;) {
    const int32_t k = keys[s];
    if (k == want) return (int)s;
    const bool free_slot = epoch >= 0 ? (((uint32_t)k >> 24) != (uint32_t)epoch) : (k == kEmpty);
    if (free_slot) {
      const int32_t old = atomicCAS(&keys[s], k, want);
      if (old == k) {
        fresh = true;
        return (int)s;
      }
      continue;  // the slot changed under us: look at it again
    }
    s = (s + 1u) & mask;
    ++probe;
  }
  return -1;
}

__device__ __forceinline__ int table_find(const int32_t* keys, int log_t, int32_t j, int epoch) {
  const uint32_t mask = (1u << log_t) - 1u;
  const int32_t want = epoch >= 0 ? (int32_t)(((uint32_t)epoch << 24) | (uint32_t)j) : j;
  uint32_t s = hash_slot(j, log_t);
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    const int32_t k = keys[s];
    if (k == want) return (int)s;
    s = (s + 1u) & mask;
  }
  return -1;
}

// Exact number of distinct output columns of `row` (keys-only table).
// epoch >= 0: epoch-tagged table; kNoEpoch: plain keys, cleared here.
template <int LOGT, bool R32>
__device__ __forceinline__ int symbolic_row(const DCsr& A, const DCsr& B, int32_t row, int32_t* keys, int epoch,
                                            int* flags) {
  using Off = typename RowOff<R32>::T;
  constexpr int T = 1 << LOGT;
  const int lane = lane_id();
  const int64_t s = A.rp[row], e = A.rp[row + 1];
  int cnt = 0;
  for (int64_t base = s; base < e; base += 32) {
    const int64_t p = base + lane;
    Off bs = 0;
    int len = 0;
    if (p < e) {
      const int32_t k = A.col[p];
      bs = RowOff<R32>::at(B, k);
      len = (int)(RowOff<R32>::at(B, k + 1) - bs);
    }
    const int n = (int)min((int64_t)32, e - base);
    for (int t = 0; t < n; ++t) {
      const Off bst = __shfl_sync(kFull, bs, t);
      const int l = __shfl_sync(kFull, len, t);
      for (int q = lane; q < l; q += 32) {
        bool fresh;
        if (table_insert(keys, LOGT, B.col[bst + q], epoch, fresh) < 0) raise_flag(flags, kFlagHashFull);
        cnt += fresh;
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

// Accumulates row `row` in canonical order: k-serial (one B row at a time),
// lanes parallel over the columns of B_k.  Within one B row all columns are
// distinct, so each slot receives at most one product per step and
// __syncwarp orders the steps.  New columns are appended to `list` in the
// order they are first seen; returns their number, or -1 when LEARNED and
// more than `cap` distinct columns appear or the table fills (the learned
// path's overflow).
template <int LOGT, bool R32, bool LEARNED>
__device__ __forceinline__ int accumulate_row(const DCsr& A, const DCsr& B, int32_t row, int32_t* keys, float* vals,
                                              int32_t* list, int epoch, int cap, int* flags) {
  using Off = typename RowOff<R32>::T;
  const int lane = lane_id();
  const unsigned lt = (1u << lane) - 1u;
  const int64_t s = A.rp[row], e = A.rp[row + 1];
  int count = 0;
  for (int64_t base = s; base < e; base += 32) {
    const int64_t p = base + lane;
    Off bs = 0;
    int len = 0;
    float a = 0.f;
    if (p < e) {
      const int32_t k = A.col[p];
      a = A.val[p];
      bs = RowOff<R32>::at(B, k);
      len = (int)(RowOff<R32>::at(B, k + 1) - bs);
    }
    const int n = (int)min((int64_t)32, e - base);
    for (int t = 0; t < n; ++t) {
      const Off bst = __shfl_sync(kFull, bs, t);
      const int l = __shfl_sync(kFull, len, t);
      const float at = __shfl_sync(kFull, a, t);
      for (int q0 = 0; q0 < l; q0 += 32) {
        const int q = q0 + lane;
        bool fresh = false, failed = false;
        int32_t j = 0;
        if (q < l) {
          j = B.col[bst + q];
          const float pr = prod_rn(at, B.val[bst + q]);
          const int slot = table_insert(keys, LOGT, j, epoch, fresh);
          if (slot < 0) failed = true;
          else vals[slot] = add_rn(fresh ? 0.f : vals[slot], pr);
        }
        const unsigned m = __ballot_sync(kFull, fresh);
        if (LEARNED) {
          if (__any_sync(kFull, failed) || count + __popc(m) > cap) {
            __syncwarp();
            return -1;
          }
        } else if (failed) {
          raise_flag(flags, kFlagHashFull);
        }
        if (fresh) list[count + __popc(m & lt)] = j;
        count += __popc(m);
        __syncwarp();
      }
    }
  }
  return count;
}

// Sorts the n listed columns (keys only, E per lane in registers), looks up
// each value in the still-intact table and writes the first `limit` entries.
template <int E, int LOGT>
__device__ __forceinline__ void sort_lookup_write(const int32_t* keys, const float* vals, const int32_t* list, int n,
                                                  int epoch, int64_t limit, int32_t* out_col, float* out_val) {
  const int lane = lane_id();
  int32_t k[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int idx = lane * E + e;
    k[e] = idx < n ? list[idx] : 0x7fffffff;
  }
  warp_sort_keys_regs<E>(k);
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int idx = lane * E + e;
    if (idx < n && idx < limit) {
      const int slot = table_find(keys, LOGT, k[e], epoch);
      out_col[idx] = k[e];
      out_val[idx] = slot >= 0 ? vals[slot] : 0.f;
    }
  }
}

// Writes the row's n entries in column order (register sort up to 512
// entries, shared-memory bitonic sort of the list beyond that).
template <int LOGT>
__device__ __forceinline__ void emit_row(const int32_t* keys, const float* vals, int32_t* list, int n, int epoch,
                                         int64_t limit, int32_t* out_col, float* out_val) {
  constexpr int T = 1 << LOGT;
  if (n <= 32) {
    sort_lookup_write<1, LOGT>(keys, vals, list, n, epoch, limit, out_col, out_val);
  } else if (n <= 64) {
    sort_lookup_write<2, LOGT>(keys, vals, list, n, epoch, limit, out_col, out_val);
  } else if (n <= 128) {
    sort_lookup_write<4, LOGT>(keys, vals, list, n, epoch, limit, out_col, out_val);
  } else if (n <= 256) {
    sort_lookup_write<8, LOGT>(keys, vals, list, n, epoch, limit, out_col, out_val);
  } else if (T >= 1024 && n <= 512) {
    sort_lookup_write<16, LOGT>(keys, vals, list, n, epoch, limit, out_col, out_val);
  } else {
    const int lane = lane_id();
    warp_sort_keys(list, n, T);
    const int m = (int)min((int64_t)n, limit);
    for (int t = lane; t < m; t += 32) {
      const int slot = table_find(keys, LOGT, list[t], epoch);
      out_col[t] = list[t];
      out_val[t] = slot >= 0 ? vals[slot] : 0.f;
    }
  }
  __syncwarp();
}

// Ends a row: advances the epoch (wiping the keys when it wraps) or, with
// plain keys, clears the table.
template <int LOGT>
__device__ __forceinline__ void next_row(int32_t* keys, int& epoch) {
  constexpr int T = 1 << LOGT;
  const int lane = lane_id();
  if (epoch >= 0 && ++epoch < 255) return;
  for (int s = lane; s < T; s += 32) keys[s] = kEmpty;
  __syncwarp();
  if (epoch >= 0) epoch = 0;
}

// Numeric row with exact output size `want`: canonical accumulation, then
// the row in column order.
template <int LOGT, bool R32>
__device__ __forceinline__ void numeric_row(const DCsr& A, const DCsr& B, int32_t row, int32_t* keys, float* vals,
                                            int32_t* list, int& epoch, int32_t* out_col, float* out_val, int64_t want,
                                            int* flags) {
  const int n = accumulate_row<LOGT, R32, false>(A, B, row, keys, vals, list, epoch, 0, flags);
  if (n != want && lane_id() == 0) raise_flag(flags, kFlagCountDiff);
  emit_row<LOGT>(keys, vals, list, n, epoch, want, out_col, out_val);
  next_row<LOGT>(keys, epoch);
}

// 32-bit words of shared memory for one warp's numeric table: keys, values
// and the column list.
template <int LOGT>
constexpr int numeric_words() {
  return 3 * (1 << LOGT);
}

}  // namespace spg
