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
// A's row is taken 32 entries at a time; long B rows are read by the whole
// warp, short ones packed (for_each_col).
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
    for_each_col(B.col, bs, len, [&](int32_t c) {
      bool fresh;
      if (table_insert(keys, LOGT, c, epoch, fresh) < 0) raise_flag(flags, kFlagHashFull);
      cnt += fresh;
    });
  }
  __syncwarp();
  cnt = warp_sum(cnt);
  if (epoch < 0) {
    for (int s2 = lane; s2 < T; s2 += 32) keys[s2] = kEmpty;
    __syncwarp();
  }
  return cnt;
}

// Ends a step: a full table marks the lane `bad` when LEARNED (the learned
// path's overflow, judged once at the end of the row) and raises
// kFlagHashFull otherwise; __syncwarp orders the steps.
template <bool LEARNED>
__device__ __forceinline__ void end_step(bool failed, bool& bad, int* flags) {
  if (LEARNED) bad |= failed;
  else if (failed) raise_flag(flags, kFlagHashFull);
  __syncwarp();
}

// True when a list word can carry (column << LOGT) | slot: epoch-tagged
// tables and fewer than 2^(31 - LOGT) columns (words stay below the sorts'
// 0x7fffffff padding).  Such words sort like their columns, and the value's
// slot travels with them, so no table lookups follow the sort.
template <int LOGT>
__device__ __forceinline__ bool slot_packed(int64_t bcols, int epoch) {
  return epoch >= 0 && bcols < ((int64_t)1 << (31 - LOGT));
}

// Gathers the row's columns from its table into `list` (slot order; the
// emitters sort them) and returns their number: plain columns, or
// (column << LOGT) | slot words when `pack` (slot_packed).  A slot is live
// when its key carries the row's epoch (epoch-tagged tables) or is not empty
// (plain keys).  One pass of T / 32 reads per lane replaces a per-step
// record of new columns; the table holds at most T keys, so the list does
// too.
template <int LOGT>
__device__ __forceinline__ int gather_columns(const int32_t* keys, int32_t* list, int epoch, bool pack) {
  constexpr int T = 1 << LOGT;
  const int lane = lane_id();
  const unsigned lt = (1u << lane) - 1u;
  int count = 0;
#pragma unroll 4
  for (int s0 = 0; s0 < T; s0 += 32) {
    const int32_t k = keys[s0 + lane];
    const bool live = epoch >= 0 ? ((uint32_t)k >> 24) == (uint32_t)epoch : k != kEmpty;
    const unsigned m = __ballot_sync(kFull, live);
    if (live) {
      const int32_t j = epoch >= 0 ? (int32_t)((uint32_t)k & 0xFFFFFFu) : k;
      list[count + __popc(m & lt)] = pack ? (int32_t)(((uint32_t)j << LOGT) | (uint32_t)(s0 + lane)) : j;
    }
    count += __popc(m);
  }
  __syncwarp();
  return count;
}

// One segment (B row k scaled by a), k-serial: lanes over its columns, 32 per
// step.  Its columns are distinct, so each slot gets at most one product per
// step and __syncwarp orders the steps.
template <int LOGT, bool LEARNED, typename Off>
__device__ __forceinline__ void acc_segment(const DCsr& B, Off bs, int len, float a, int32_t* keys, float* vals,
                                            int epoch, bool& bad, int* flags) {
  const int lane = lane_id();
  for (int q0 = 0; q0 < len; q0 += 32) {
    const int q = q0 + lane;
    bool failed = false;
    if (q < len) {
      bool fresh;
      const int32_t j = B.col[bs + q];
      const float pr = prod_rn(a, B.val[bs + q]);
      const int slot = table_insert(keys, LOGT, j, epoch, fresh);
      if (slot < 0) failed = true;
      else vals[slot] = add_rn(fresh ? 0.f : vals[slot], pr);
    }
    end_step<LEARNED>(failed, bad, flags);
  }
}

// The chunk's n segments when each is one k-serial step (kPackBelow <= len
// <= 32): step idx's B loads are issued before step idx - 1's table work, so
// their latency overlaps it (stencil 96^3 plain numeric 3.90 -> 3.47 ms);
// a step's length comes from the shuffle that fetched its loads (three
// shuffles a step instead of four: learned numeric 3.34 -> 3.33 ms).
template <int LOGT, bool LEARNED, typename Off>
__device__ __forceinline__ void acc_single_steps(const DCsr& B, Off bs, int len, float a, int n, int32_t* keys,
                                                 float* vals, int epoch, bool& bad, int* flags) {
  const int lane = lane_id();
  int32_t jn = -1;
  float bn = 0.f;
  int nl = __shfl_sync(kFull, len, 0);  // the next step's length, carried over
  {
    const Off sbs = __shfl_sync(kFull, bs, 0);
    if (lane < nl) {
      jn = B.col[sbs + lane];
      bn = B.val[sbs + lane];
    }
  }
  for (int idx = 0; idx < n; ++idx) {
    const int32_t j = jn;
    const float bv = bn;
    const float sa = __shfl_sync(kFull, a, idx);
    const int sl = nl;
    if (idx + 1 < n) {
      const Off nbs = __shfl_sync(kFull, bs, idx + 1);
      nl = __shfl_sync(kFull, len, idx + 1);
      if (lane < nl) {
        jn = B.col[nbs + lane];
        bn = B.val[nbs + lane];
      }
    }
    bool failed = false;
    if (lane < sl) {
      bool fresh;
      const float pr = prod_rn(sa, bv);
      const int slot = table_insert(keys, LOGT, j, epoch, fresh);
      if (slot < 0) failed = true;
      else vals[slot] = add_rn(fresh ? 0.f : vals[slot], pr);
    }
    end_step<LEARNED>(failed, bad, flags);
  }
}

// Segments of lanes [lo, hi) (all shorter than kPackBelow) taken as one
// stream in canonical order (segment-major), 32 products per step.  Products
// of one step that hit the same column (from different segments) are grouped
// with __match_any_sync; the group's lowest lane inserts the column and adds
// the group's products in lane order, so every entry still sees its products
// in canonical order.
template <int LOGT, bool LEARNED, typename Off>
__device__ __forceinline__ void acc_packed(const DCsr& B, Off bs, int len, float a, int lo, int hi, int32_t* keys,
                                           float* vals, int epoch, bool& bad, int* flags) {
  const int lane = lane_id();
  const int lr = (lane >= lo && lane < hi) ? len : 0;
  const int incl = warp_incl_scan(lr);
  const int total = __shfl_sync(kFull, incl, 31);
  const int excl = incl - lr;
  for (int b0 = 0; b0 < total; b0 += 32) {
    const int tt = b0 + lane;
    const bool act = tt < total;
    const int src = warp_upper_bound(incl, act ? tt : total - 1);
    const Off sbs = __shfl_sync(kFull, bs, src);
    const int sex = __shfl_sync(kFull, excl, src);
    const float sa = __shfl_sync(kFull, a, src);
    int32_t j = -1 - lane;  // unique dummy for idle lanes
    float pr = 0.f;
    if (act) {
      const Off q = sbs + (Off)(tt - sex);
      j = B.col[q];
      pr = prod_rn(sa, B.val[q]);
    }
    const unsigned grp = __match_any_sync(kFull, j);
    const bool leader = act && (grp & ((1u << lane) - 1u)) == 0u;
    bool fresh = false;
    int slot = -1;
    if (leader) slot = table_insert(keys, LOGT, j, epoch, fresh);
    const bool ok = leader && slot >= 0;
    float v = (ok && !fresh) ? vals[slot] : 0.f;
    v = group_sum_in_lane_order(grp, pr, v, ok);
    if (ok) vals[slot] = v;
    end_step<LEARNED>(leader && slot < 0, bad, flags);
  }
}

// Accumulates row `row` in canonical order (k ascending through A's row,
// then column ascending through B's row k).  A's row is taken 32 entries at
// a time: B rows of kPackBelow or more entries go k-serially
// (acc_segment; acc_single_steps when every B row of the chunk is one
// step), runs of shorter ones are packed (acc_packed).  At the end
// the row's columns are gathered from the table into `list`
// (gather_columns); returns their number, or -1 when LEARNED and the row
// filled the table or has more than `cap` distinct columns (the learned
// path's overflow, checked once at the end of the row).
template <int LOGT, bool R32, bool LEARNED, bool PACK_OK = false>
__device__ __forceinline__ int accumulate_row(const DCsr& A, const DCsr& B, int32_t row, int32_t* keys, float* vals,
                                              int32_t* list, int epoch, int cap, int* flags) {
  using Off = typename RowOff<R32>::T;
  const int lane = lane_id();
  const int64_t s = A.rp[row], e = A.rp[row + 1];
  bool bad = false;
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
    if (__all_sync(kFull, p >= e || (len >= kPackBelow && len <= 32))) {
      acc_single_steps<LOGT, LEARNED>(B, bs, len, a, n, keys, vals, epoch, bad, flags);
      continue;
    }
    const unsigned long_mask = __ballot_sync(kFull, len >= kPackBelow);
    int idx = 0;
    while (idx < n) {
      if ((long_mask >> idx) & 1u) {
        const Off sbs = __shfl_sync(kFull, bs, idx);
        const int sl = __shfl_sync(kFull, len, idx);
        const float sa = __shfl_sync(kFull, a, idx);
        acc_segment<LOGT, LEARNED>(B, sbs, sl, sa, keys, vals, epoch, bad, flags);
        ++idx;
      } else {
        const unsigned later = long_mask & (~0u << idx);
        const int hi = later ? min(n, __ffs(later) - 1) : n;
        acc_packed<LOGT, LEARNED>(B, bs, len, a, idx, hi, keys, vals, epoch, bad, flags);
        idx = hi;
      }
    }
  }
  // the learned capacity is judged once per row: its overflow is rare
  if (LEARNED && __any_sync(kFull, bad)) return -1;
  const int count = gather_columns<LOGT>(keys, list, epoch, PACK_OK && slot_packed<LOGT>(B.cols, epoch));
  if (LEARNED && count > cap) return -1;
  return count;
}

// Sorts the n listed words (E per lane in registers, entry e * 32 + lane in
// register e of that lane), finds each value's
// slot (carried by the word when `pack`, else looked up in the still-intact
// table) and writes the first `limit` entries.
template <int E, int LOGT>
__device__ __forceinline__ void sort_lookup_write(const int32_t* keys, const float* vals, const int32_t* list, int n,
                                                  int epoch, int64_t limit, int32_t* out_col, float* out_val,
                                                  bool pack) {
  const int lane = lane_id();
  int32_t k[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int idx = e * 32 + lane;
    k[e] = idx < n ? list[idx] : 0x7fffffff;
  }
  warp_sort_keys_regs<E>(k);
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int idx = e * 32 + lane;
    if (idx < n && idx < limit) {
      if (pack) {
        out_col[idx] = (int32_t)((uint32_t)k[e] >> LOGT);
        out_val[idx] = vals[(uint32_t)k[e] & (uint32_t)((1 << LOGT) - 1)];
      } else {
        const int slot = table_find(keys, LOGT, k[e], epoch);
        out_col[idx] = k[e];
        out_val[idx] = slot >= 0 ? vals[slot] : 0.f;
      }
    }
  }
}

// Writes the row's n entries in column order with a warp LSD radix sort.
// Each listed column c becomes the word ((c - lo) << LOGT) | slot (lo = the
// row's smallest column, slot = its table slot), so the sort carries the
// value's location with it and no lookups follow.  Passes of `d`-bit digits
// (d <= 8) cover the bits of the column span; each pass is a histogram, an
// exclusive scan of the buckets and a stable scatter (32 words per step in
// list order, ranks within a bucket from __match_any_sync).  Buffers: the
// list and the key array take turns; the bucket counts live past the n
// words of the source.  Returns false, touching nothing, when the packed
// words do not fit 32 bits or the buffers are too small; on success the key
// array is wiped (the caller's table is empty afterwards).
template <int LOGT>
__device__ __forceinline__ bool radix_emit(int32_t* keys, const float* vals, int32_t* list, int n, int epoch,
                                           int64_t limit, int32_t* out_col, float* out_val, bool pack) {
  constexpr int T = 1 << LOGT;
  const int lane = lane_id();
  const unsigned lt = (1u << lane) - 1u;
  int lo = 0x7fffffff, hi = 0;
  for (int i = lane; i < n; i += 32) {
    const int c = pack ? (int)((uint32_t)list[i] >> LOGT) : list[i];
    lo = min(lo, c);
    hi = max(hi, c);
  }
  lo = (int)__reduce_min_sync(kFull, (unsigned)lo);
  hi = (int)__reduce_max_sync(kFull, (unsigned)hi);
  const uint32_t span = (uint32_t)(hi - lo);
  const int span_bits = span ? 32 - __clz(span) : 0;
  if (span_bits > 32 - LOGT) return false;
  int d = 8;
  while (d > 5 && n + (1 << d) > T) --d;
  if (n + (1 << d) > T) return false;
  // pack (the slot comes with a packed word, else from the intact table)
  for (int i = lane; i < n; i += 32) {
    const uint32_t w = (uint32_t)list[i];
    const int c = pack ? (int)(w >> LOGT) : (int)w;
    const int slot = pack ? (int)(w & (uint32_t)(T - 1)) : table_find(keys, LOGT, c, epoch);
    list[i] = (int32_t)(((uint32_t)(c - lo) << LOGT) | (uint32_t)(slot & (T - 1)));
  }
  __syncwarp();
  uint32_t* srcb = reinterpret_cast<uint32_t*>(list);
  uint32_t* dstb = reinterpret_cast<uint32_t*>(keys);
  const int nb = 1 << d;
  const uint32_t dm = (uint32_t)nb - 1u;
  for (int shift = LOGT; shift < LOGT + span_bits; shift += d) {
    int* hist = reinterpret_cast<int*>(srcb + n);
    for (int b = lane; b < nb; b += 32) hist[b] = 0;
    __syncwarp();
    for (int i = lane; i < n; i += 32) atomicAdd(&hist[(srcb[i] >> shift) & dm], 1);
    __syncwarp();
    // exclusive scan of the buckets, nb / 32 (<= 8) consecutive per lane
    const int per = (nb + 31) >> 5;
    int loc[8];
    int sum = 0;
#pragma unroll
    for (int x = 0; x < 8; ++x) {
      const int b = lane * per + x;
      loc[x] = (x < per && b < nb) ? hist[b] : 0;
      sum += loc[x];
    }
    int run = warp_incl_scan(sum) - sum;
#pragma unroll
    for (int x = 0; x < 8; ++x) {
      const int b = lane * per + x;
      if (x < per && b < nb) hist[b] = run;
      run += loc[x];
    }
    __syncwarp();
    // stable scatter
    for (int i0 = 0; i0 < n; i0 += 32) {
      const int i = i0 + lane;
      const bool act = i < n;
      const uint32_t v = act ? srcb[i] : 0u;
      const int dig = act ? (int)((v >> shift) & dm) : -1 - lane;
      const unsigned grp = __match_any_sync(kFull, dig);
      const int leader = __ffs(grp) - 1;
      int base = 0;
      if (act && lane == leader) base = atomicAdd(&hist[dig], __popc(grp));
      base = __shfl_sync(kFull, base, leader);
      if (act) dstb[base + __popc(grp & lt)] = v;
    }
    __syncwarp();
    uint32_t* t = srcb;
    srcb = dstb;
    dstb = t;
  }
  const int m = (int)min((int64_t)n, limit);
  for (int i = lane; i < m; i += 32) {
    const uint32_t v = srcb[i];
    out_col[i] = lo + (int32_t)(v >> LOGT);
    out_val[i] = vals[v & (uint32_t)(T - 1)];
  }
  __syncwarp();
  for (int s = lane; s < T; s += 32) keys[s] = kEmpty;
  __syncwarp();
  return true;
}

// Writes the row's n entries in column order: register bitonic sorts up to
// 128 entries, the radix sort above that, and (when the radix sort does not
// apply) a register sort up to 256 entries or a shared-memory bitonic sort.
template <int LOGT>
__device__ __forceinline__ void emit_row(int32_t* keys, const float* vals, int32_t* list, int n, int epoch,
                                         int64_t limit, int32_t* out_col, float* out_val, bool pack) {
  constexpr int T = 1 << LOGT;
  if (n <= 32) {
    sort_lookup_write<1, LOGT>(keys, vals, list, n, epoch, limit, out_col, out_val, pack);
  } else if (n <= 64) {
    sort_lookup_write<2, LOGT>(keys, vals, list, n, epoch, limit, out_col, out_val, pack);
  } else if (n <= 128) {
    sort_lookup_write<4, LOGT>(keys, vals, list, n, epoch, limit, out_col, out_val, pack);
  } else if (radix_emit<LOGT>(keys, vals, list, n, epoch, limit, out_col, out_val, pack)) {
    return;
  } else if (n <= 256) {
    sort_lookup_write<8, LOGT>(keys, vals, list, n, epoch, limit, out_col, out_val, pack);
  } else {
    const int lane = lane_id();
    warp_sort_keys(list, n, T);
    const int m = (int)min((int64_t)n, limit);
    for (int t = lane; t < m; t += 32) {
      const uint32_t w = (uint32_t)list[t];
      const int slot = pack ? (int)(w & (uint32_t)(T - 1)) : table_find(keys, LOGT, (int32_t)w, epoch);
      out_col[t] = pack ? (int32_t)(w >> LOGT) : (int32_t)w;
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

// ---- expand-sort-fold rows ------------------------------------------------
// For rows whose products mostly land on distinct columns the hash table
// costs more than it saves: the row's P products are written in canonical
// order (columns and values), turned into words ((column - lo) << b) |
// position (b = the bits of P - 1), radix sorted (stable, LSD) on the column
// bits, and folded left
// to right, each column's sum starting from 0 and adding its products in
// canonical order, as the hash accumulators do (the same bits).  Measured on
// Erdos-Renyi 2^18 rows of 17 entries (289 products, 286 outputs per row):
// numeric 3.85 -> 2.31 ms; rows of 64 products stay hashed (0.55 against
// 0.81 ms).
// Largest P that `words` 32-bit words of a warp's shared memory hold: two
// word buffers, the values and 256 bucket counts.
__host__ __device__ __forceinline__ int esc_capacity(int words) { return (words - 256) / 3; }

// True when a row of `prod` products and at least `out` output entries
// (its exact count, or the learned capacity) takes the expand-sort-fold
// path: esc_min > 0 (0 turns it off), prod in [esc_min, cap] and at least
// half of the products distinct.
__device__ __forceinline__ bool esc_wanted(int64_t prod, int64_t out, int esc_min, int cap) {
  return esc_min > 0 && prod >= esc_min && prod <= cap && 2 * out >= prod;
}

// Writes the row (P >= 1 products) sorted into out_col/out_val (its first
// `limit` entries) and returns its entry count, or -1, having written
// nothing, when its column span and positions need more than 31 bits (the
// caller hashes the row then).  `buf` holds esc_capacity(words) >= P; its
// contents are scratch afterwards.
template <bool R32>
__device__ __forceinline__ int esc_row(const DCsr& A, const DCsr& B, int32_t row, int P, int32_t* buf, int64_t limit,
                                       int32_t* out_col, float* out_val) {
  using Off = typename RowOff<R32>::T;
  const int lane = lane_id();
  const unsigned lt = (1u << lane) - 1u;
  uint32_t* wa = reinterpret_cast<uint32_t*>(buf);
  uint32_t* wb = wa + P;
  float* vals = reinterpret_cast<float*>(wb + P);
  int* hist = reinterpret_cast<int*>(vals + P);
  // expand in canonical order: columns into wa, products into vals
  const int64_t s = A.rp[row], e = A.rp[row + 1];
  int base = 0;
  int lo = 0x7fffffff, hi = -1;
  for (int64_t c0 = s; c0 < e; c0 += 32) {
    const int64_t q = c0 + lane;
    Off bs = 0;
    int len = 0;
    float a = 0.f;
    if (q < e) {
      const int32_t k = A.col[q];
      a = A.val[q];
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
      if (act && base + tt < P) {
        const Off qq = sbs + (Off)(tt - sex);
        const int32_t c = B.col[qq];
        lo = min(lo, c);
        hi = max(hi, c);
        wa[base + tt] = (uint32_t)c;
        vals[base + tt] = prod_rn(sa, B.val[qq]);
      }
    }
    base += total;
  }
  lo = (int)__reduce_min_sync(kFull, (unsigned)lo);
  hi = (int)__reduce_max_sync(kFull, (unsigned)hi);
  const uint32_t span = P > 0 ? (uint32_t)(hi - lo) : 0u;
  const int span_bits = span ? 32 - __clz(span) : 0;
  const int ib = P > 1 ? 32 - __clz((uint32_t)(P - 1)) : 1;  // position bits
  const uint32_t im = (1u << ib) - 1u;
  if (base != P || span_bits + ib > 31) {
    __syncwarp();
    return -1;
  }
  __syncwarp();
  for (int i = lane; i < P; i += 32) wa[i] = ((wa[i] - (uint32_t)lo) << ib) | (uint32_t)i;
  __syncwarp();
  // stable LSD radix sort on the column bits, 8-bit digits
  uint32_t* src = wa;
  uint32_t* dst = wb;
  for (int shift = ib; shift < ib + span_bits; shift += 8) {
    for (int b = lane; b < 256; b += 32) hist[b] = 0;
    __syncwarp();
    for (int i = lane; i < P; i += 32) atomicAdd(&hist[(src[i] >> shift) & 255u], 1);
    __syncwarp();
    int loc[8];
    int sum = 0;
#pragma unroll
    for (int x = 0; x < 8; ++x) {
      loc[x] = hist[lane * 8 + x];
      sum += loc[x];
    }
    int run = warp_incl_scan(sum) - sum;
#pragma unroll
    for (int x = 0; x < 8; ++x) {
      hist[lane * 8 + x] = run;
      run += loc[x];
    }
    __syncwarp();
    for (int i0 = 0; i0 < P; i0 += 32) {
      const int i = i0 + lane;
      const bool act = i < P;
      const uint32_t v = act ? src[i] : 0u;
      const int dig = act ? (int)((v >> shift) & 255u) : -1 - lane;
      const unsigned grp = __match_any_sync(kFull, dig);
      const int leader = __ffs(grp) - 1;
      int at = 0;
      if (act && lane == leader) at = atomicAdd(&hist[dig], __popc(grp));
      at = __shfl_sync(kFull, at, leader);
      if (act) dst[at + __popc(grp & lt)] = v;
    }
    __syncwarp();
    uint32_t* t = src;
    src = dst;
    dst = t;
  }
  // fold runs of equal columns left to right; run heads write the entries
  int count = 0;
  for (int i0 = 0; i0 < P; i0 += 32) {
    const int i = i0 + lane;
    const bool act = i < P;
    const uint32_t w = act ? src[i] : 0u;
    const uint32_t c = w >> ib;
    const bool head = act && (i == 0 || (src[i - 1] >> ib) != c);
    const unsigned hm = __ballot_sync(kFull, head);
    if (head) {
      float v = add_rn(0.f, vals[w & im]);
      for (int j = i + 1; j < P; ++j) {
        const uint32_t wj = src[j];
        if ((wj >> ib) != c) break;
        v = add_rn(v, vals[wj & im]);
      }
      const int o = count + __popc(hm & lt);
      if (o < limit) {
        out_col[o] = lo + (int32_t)c;
        out_val[o] = v;
      }
    }
    count += __popc(hm);
  }
  __syncwarp();
  return count;
}

// Wipes the first `words` words of a warp table's key array after an
// expand-sort-fold row used its memory.
__device__ __forceinline__ void esc_wipe(int32_t* keys, int words) {
  for (int s = lane_id(); s < words; s += 32) keys[s] = kEmpty;
  __syncwarp();
}

// Numeric row with exact output size `want`: canonical accumulation, then
// the row in column order.  PACK_OK lets list words carry their slots
// (slot_packed): measured faster for the batched kernels (batch-512
// 128.7 -> 125.5 ms) and slower for the single-product ones (stencil 96^3
// numeric 3.91 -> 3.94 ms), which keep plain column lists.
template <int LOGT, bool R32, bool PACK_OK = false>
__device__ __forceinline__ void numeric_row(const DCsr& A, const DCsr& B, int32_t row, int32_t* keys, float* vals,
                                            int32_t* list, int& epoch, int32_t* out_col, float* out_val, int64_t want,
                                            int* flags) {
  const bool pack = PACK_OK && slot_packed<LOGT>(B.cols, epoch);
  const int n = accumulate_row<LOGT, R32, false, PACK_OK>(A, B, row, keys, vals, list, epoch, 0, flags);
  if (n != want && lane_id() == 0) raise_flag(flags, kFlagCountDiff);
  emit_row<LOGT>(keys, vals, list, n, epoch, want, out_col, out_val, pack);
  next_row<LOGT>(keys, epoch);
}

// 32-bit words of shared memory for one warp's numeric table: keys, values
// and the column list.
template <int LOGT>
constexpr int numeric_words() {
  return 3 * (1 << LOGT);
}

}  // namespace spg
