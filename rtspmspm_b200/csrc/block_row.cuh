// CTA-wide numeric accumulator: one CTA (kBlkThreads threads) owns one output
// row and one shared hash table of 2^LOGT (key, value, order-word) slots, for
// rows too large for a warp's table but far from the heavy-row tiles.
//
// Canonical order with the whole CTA at work.  The row's product stream (k
// ascending through A's row, then column ascending through B's row k) is cut
// into steps of kBlkThreads consecutive products, thread t taking product
// step_base + t.  Columns are claimed in the table order-free (CAS); the adds
// of one step then run in rounds: every thread with a pending product
// offers its tag to its slot's order word with atomicMin, and the thread
// whose tag is smallest -- the earliest product of that column in the step --
// adds; the others try again in the next round.  Tags decrease with the step
// and the round, so a new round always wins over the words left by earlier
// ones, and rounds end once no product is pending (at most kBlkThreads
// rounds, one add per contested slot each).  Every entry therefore sees its
// products in canonical order, as in the warp accumulators.
//
// The row is written in column order by a CTA-wide LSD radix sort (8-bit
// digits of column - row minimum): each warp owns a contiguous part of the
// list, so a histogram per warp and offsets in (digit, warp) order make the
// scatter stable.  The key and order-word arrays are the sort's buffers, so
// the table must hold at least twice the row's entries (load <= 0.5).
#pragma once

#include "common.cuh"
#include "warp_row.cuh"

namespace spg {

constexpr int kBlkThreads = 256;
constexpr int kBlkWarps = kBlkThreads / 32;
// Shared scratch of the CTA accumulator besides its table: the staged chunk
// of A's row while accumulating, the radix histograms while sorting.
struct BlockScratch {
  union {
    struct {
      int64_t excl[kBlkThreads + 1];  // first product of each staged (non-empty) entry
      int64_t bs[kBlkThreads];        // its B row start
      float a[kBlkThreads];
    } st;
    int hist[kBlkWarps][256];
  } u;
  int64_t wsum[kBlkWarps + 1];
  int cnt;    // staged entries / gathered columns
  int fresh;  // distinct columns claimed
  int fail;   // an insert found the table full
  int lo, hi;  // column range of the row
};

// Exclusive prefix over the CTA's threads (kBlkThreads); *total gets the sum.
template <typename V>
__device__ __forceinline__ V cta_excl_scan(V v, int64_t* wsum, V& total) {
  const int lane = lane_id(), w = threadIdx.x >> 5;
  const V inc = warp_incl_scan(v);
  if (lane == 31) wsum[w] = (int64_t)inc;
  __syncthreads();
  if (w == 0) {
    const int64_t x = lane < kBlkWarps ? wsum[lane] : 0;
    const int64_t xi = warp_incl_scan(x);
    if (lane < kBlkWarps) wsum[lane] = xi - x;
    if (lane == kBlkWarps - 1) wsum[kBlkWarps] = xi;
  }
  __syncthreads();
  const V r = inc - v + (V)wsum[w];
  total = (V)wsum[kBlkWarps];
  __syncthreads();
  return r;
}

// Log2 of the CTA table a row of `entries` output entries uses: at load
// <= 1/2, at least 2^8 slots (one per thread), at most 2^logt_max.
__device__ __forceinline__ int cta_table_log(int64_t entries, int logt_max) {
  int l = 8;
  while (l < logt_max && ((int64_t)1 << l) < 2 * entries) ++l;
  return l;
}

// Accumulates `row` in canonical order into the CTA table (its first 2^logt
// slots, logt <= LOGT) and returns its number of distinct columns; LEARNED:
// -1 when the table filled or the row has more than `cap` columns (the
// learned path's overflow).  VALUES = false only counts the columns
// (symbolic pass: keys only, vals and own unused).  Uniform over the CTA.
// The table is cleared here, so rows need no clean-up between them.
template <int LOGT, bool R32, bool LEARNED, bool VALUES = true>
__device__ __forceinline__ int cta_accumulate_row(const DCsr& A, const DCsr& B, int32_t row, int32_t* keys,
                                                  float* vals, uint32_t* own, BlockScratch& sc, int64_t cap,
                                                  int* flags, int logt = LOGT) {
  const int T = 1 << logt;
  const int tid = threadIdx.x, lane = lane_id(), w = tid >> 5;
  for (int s = tid; s < T; s += kBlkThreads) {
    keys[s] = kEmpty;
    if (VALUES) {
      vals[s] = 0.f;
      own[s] = 0xffffffffu;
    }
  }
  if (tid == 0) {
    sc.fresh = 0;
    sc.fail = 0;
  }
  __syncthreads();
  const int64_t s0 = A.rp[row], e0 = A.rp[row + 1];
  uint32_t step = 0;
  int my_fresh = 0;
  for (int64_t cb = s0; cb < e0; cb += kBlkThreads) {
    // stage the chunk's non-empty entries: one scan of (length << 9 | non-empty)
    const int64_t p = cb + tid;
    int64_t bs = 0, len = 0;
    float a = 0.f;
    if (p < e0) {
      const int32_t k = A.col[p];
      a = A.val[p];
      bs = (int64_t)RowOff<R32>::at(B, k);
      len = (int64_t)RowOff<R32>::at(B, k + 1) - bs;
    }
    int64_t tot;
    const int64_t ex = cta_excl_scan<int64_t>((len << 9) | (len > 0 ? 1 : 0), sc.wsum, tot);
    const int ci = (int)(ex & 511);
    if (len > 0) {
      sc.u.st.excl[ci] = ex >> 9;
      sc.u.st.bs[ci] = bs;
      sc.u.st.a[ci] = a;
    }
    const int cnt = (int)(tot & 511);
    const int64_t total = tot >> 9;
    if (tid == 0) sc.u.st.excl[cnt] = total;
    __syncthreads();
    for (int64_t x0 = 0; x0 < total; x0 += kBlkThreads) {
      if (VALUES && step != 0 && (step & 0x7fffu) == 0) {
        // the step field of the tags wrapped: reset the order words
        for (int s = tid; s < T; s += kBlkThreads) own[s] = 0xffffffffu;
        __syncthreads();
      }
      const uint32_t stepcode = 0x7fffu - (step & 0x7fffu);
      const int64_t p0 = x0 + 32 * w;
      const int64_t pos = p0 + lane;
      const bool act = pos < total;
      int32_t col = 0;
      float pr = 0.f;
      if (p0 < total) {
        // the staged entry holding p0: excl[lo] <= p0 < excl[lo + 1]
        int lo = 0, hi = cnt;
        while (hi - lo > 1) {
          const int mid = (lo + hi) >> 1;
          if (sc.u.st.excl[mid] <= p0) lo = mid;
          else hi = mid;
        }
        // each staged entry holds a product, so the next 32 starts cover the
        // warp's 32 positions
        const int wi = lo + 1 + lane;
        const int64_t nxt = wi <= cnt ? sc.u.st.excl[wi] : INT64_MAX;
        const int ent = lo + warp_upper_bound_t<int64_t>(nxt, act ? pos : p0);
        if (act) {
          const int64_t q = sc.u.st.bs[ent] + (pos - sc.u.st.excl[ent]);
          col = B.col[q];
          if (VALUES) pr = prod_rn(sc.u.st.a[ent], B.val[q]);
        }
      }
      int slot = -1;
      bool pending = false;
      if (act) {
        bool fresh;
        slot = table_insert(keys, logt, col, kNoEpoch, fresh);
        if (slot < 0) {
          sc.fail = 1;
          if (!LEARNED) raise_flag(flags, kFlagHashFull);
        } else {
          pending = true;
          my_fresh += fresh ? 1 : 0;
        }
      }
      for (uint32_t round = 0; VALUES; ++round) {
        const uint32_t tag = (stepcode << 17) | ((0x1ffu - round) << 8) | (uint32_t)tid;
        if (pending) atomicMin(&own[slot], tag);
        __syncthreads();
        if (pending && own[slot] == tag) {
          vals[slot] = add_rn(vals[slot], pr);
          pending = false;
        }
        if (!__syncthreads_or(pending)) break;
        if (round >= (uint32_t)kBlkThreads) {  // cannot happen: a round settles every contested slot once
          raise_flag(flags, kFlagHashFull);
          break;
        }
      }
      ++step;
    }
    __syncthreads();  // the staging is rewritten by the next chunk
  }
  my_fresh = warp_sum(my_fresh);
  if (lane == 0 && my_fresh) atomicAdd(&sc.fresh, my_fresh);
  __syncthreads();
  const int n = sc.fresh;
  const bool failed = sc.fail != 0;
  __syncthreads();  // every thread has read the counters before they are reset
  if (LEARNED && (failed || n > cap)) return -1;
  return n;
}

// Writes the row's n entries (n <= 2^logt / 2, the table of
// cta_accumulate_row) in column order -- the first `limit` of them -- with a
// CTA-wide LSD radix sort; the table is consumed.
template <int LOGT>
__device__ __forceinline__ void cta_emit_row(int32_t* keys, const float* vals, uint32_t* own, BlockScratch& sc,
                                             int n, int64_t limit, int32_t* out_col, float* out_val,
                                             int logt = LOGT) {
  const int T = 1 << logt;
  const int tid = threadIdx.x, lane = lane_id(), w = tid >> 5;
  const unsigned lt = (1u << lane) - 1u;
  int32_t* col_a = reinterpret_cast<int32_t*>(own);
  int32_t* slot_a = reinterpret_cast<int32_t*>(own) + T / 2;
  int32_t* col_b = keys;
  int32_t* slot_b = keys + T / 2;
  if (tid == 0) {
    sc.cnt = 0;
    sc.lo = 0x7fffffff;
    sc.hi = -1;
  }
  __syncthreads();
  // gather the live slots (any order) and the row's column range
  int lo = 0x7fffffff, hi = -1;
  for (int s0 = 0; s0 < T; s0 += kBlkThreads) {
    const int s = s0 + tid;
    const int32_t k = keys[s];
    const bool live = k != kEmpty;
    const unsigned m = __ballot_sync(kFull, live);
    int base = 0;
    if (lane == 0 && m) base = atomicAdd(&sc.cnt, __popc(m));
    base = __shfl_sync(kFull, base, 0);
    if (live) {
      const int d = base + __popc(m & lt);
      if (d < T / 2) {
        col_a[d] = k;
        slot_a[d] = s;
      }
      lo = min(lo, k);
      hi = max(hi, k);
    }
  }
  lo = warp_min(lo);
  hi = warp_max(hi);
  if (lane == 0) {
    atomicMin(&sc.lo, lo);
    atomicMax(&sc.hi, hi);
  }
  __syncthreads();
  n = min(n, min(sc.cnt, T / 2));
  lo = sc.lo;
  const uint32_t span = n > 0 ? (uint32_t)(sc.hi - lo) : 0u;
  const int span_bits = span ? 32 - __clz(span) : 0;
  int32_t *cs = col_a, *ss = slot_a, *cd = col_b, *sd = slot_b;
  const int seg = (n + kBlkWarps - 1) / kBlkWarps;
  const int wbeg = min(n, w * seg), wend = min(n, wbeg + seg);
  for (int shift = 0; shift < span_bits; shift += 8) {
    int* hist = &sc.u.hist[0][0];
    for (int i = tid; i < kBlkWarps * 256; i += kBlkThreads) hist[i] = 0;
    __syncthreads();
    for (int i = wbeg + lane; i < wend; i += 32)
      atomicAdd(&sc.u.hist[w][((uint32_t)(cs[i] - lo) >> shift) & 255u], 1);
    __syncthreads();
    // offsets in (digit, warp) order; thread d takes digit d
    {
      const int d = tid;
      int h[kBlkWarps];
      int tot_d = 0;
#pragma unroll
      for (int x = 0; x < kBlkWarps; ++x) {
        h[x] = sc.u.hist[x][d];
        tot_d += h[x];
      }
      int all;
      int base = cta_excl_scan<int>(tot_d, sc.wsum, all);
#pragma unroll
      for (int x = 0; x < kBlkWarps; ++x) {
        sc.u.hist[x][d] = base;
        base += h[x];
      }
    }
    __syncthreads();
    // stable scatter, each warp over its part in order
    for (int i0 = wbeg; i0 < wend; i0 += 32) {
      const int i = i0 + lane;
      const bool act = i < wend;
      const int32_t c = act ? cs[i] : 0;
      const int dig = act ? (int)(((uint32_t)(c - lo) >> shift) & 255u) : -1 - lane;
      const unsigned grp = __match_any_sync(kFull, dig);
      const int leader = __ffs(grp) - 1;
      int b = 0;
      if (act && lane == leader) {
        b = sc.u.hist[w][dig];
        sc.u.hist[w][dig] = b + __popc(grp);
      }
      b = __shfl_sync(kFull, b, leader);
      if (act) {
        const int dst = b + __popc(grp & lt);
        cd[dst] = c;
        sd[dst] = ss[i];
      }
    }
    __syncthreads();
    int32_t* t = cs;
    cs = cd;
    cd = t;
    t = ss;
    ss = sd;
    sd = t;
  }
  const int m = (int)min((int64_t)n, limit);
  for (int i = tid; i < m; i += kBlkThreads) {
    out_col[i] = cs[i];
    out_val[i] = vals[ss[i]];
  }
  __syncthreads();  // the next row clears the table
}

// 32-bit words of dynamic shared memory of a CTA table: keys, values, order words.
template <int LOGT>
constexpr int block_words() {
  return 3 * (1 << LOGT);
}

}  // namespace spg
