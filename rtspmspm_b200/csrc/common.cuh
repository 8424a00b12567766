// Device-side building blocks shared by every SpGEMM kernel of the engine.
//
// Arithmetic contract (restated from the reference's any-hit accumulate,
// optixSpMSpM/src/optixSpMSpM/optixSpMSpM.cu:246-258): each intermediate
// product is rounded to FP32 (__fmul_rn) and then added in FP32 (__fadd_rn);
// no fused multiply-add.  Every accumulator adds the products of one output
// entry in canonical order: k ascending through A's row, then j ascending
// through B's row k.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace spg {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;
constexpr int32_t kEmpty = -1;        // empty hash-table key
#ifndef SPG_TILE_SHIFT
#define SPG_TILE_SHIFT 11
#endif
constexpr int kTileShift = SPG_TILE_SHIFT;  // heavy-row column tile: 2^11 = 2048 columns
constexpr int kTileCols = 1 << kTileShift;
constexpr int kTileWords = kTileCols / 32;

// Device error flags (mirrors SPG_FLAG_* of the public header).
constexpr int kFlagHashFull = 1;
constexpr int kFlagWaitLimit = 2;
constexpr int kFlagBadIndex = 4;
constexpr int kFlagCountDiff = 8;

// Read-only device view of a CSR matrix.  `rp` always holds 64-bit row
// pointers; `rp32` holds the same offsets as int32 when nnz < 2^31 (else
// null), so the hot loops can move half the bytes and shuffle one register.
struct DCsr {
  int64_t rows;
  int64_t cols;
  const int64_t* rp;
  const int32_t* col;
  const float* val;
  const int32_t* rp32;
};

// One product of a batch: its operands and where its rows and output live.
struct BatchMat {
  DCsr A;
  DCsr B;
  int64_t row_start;  // first global row of this product
  int64_t c_base;     // first entry of C_m in the output slab
  int64_t rp_base;    // first entry of C_m's row pointers in the row-pointer slab
};

// Row offset type of the hot loops: int32 when R32, else int64.
template <bool R32>
struct RowOff {
  using T = int64_t;
  static __device__ __forceinline__ int64_t at(const DCsr& M, int64_t i) { return M.rp[i]; }
};
template <>
struct RowOff<true> {
  using T = int32_t;
  static __device__ __forceinline__ int32_t at(const DCsr& M, int64_t i) { return M.rp32[i]; }
};

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

__device__ __forceinline__ void raise_flag(int* flags, int f) {
  if (flags) atomicOr(flags, f);
}

// Multiplicative (Fibonacci) hash of a column index into 2^log_t slots.
__device__ __forceinline__ uint32_t hash_slot(int32_t j, int log_t) {
  return ((uint32_t)j * 2654435761u) >> (32 - log_t);
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    T w = __shfl_xor_sync(kFull, v, o);
    v = w > v ? w : v;
  }
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_min(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    T w = __shfl_xor_sync(kFull, v, o);
    v = w < v ? w : v;
  }
  return v;
}

// Inclusive prefix sum across the warp.
template <typename T>
__device__ __forceinline__ T warp_incl_scan(T v) {
  const int lane = lane_id();
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T w = __shfl_up_sync(kFull, v, o);
    if (lane >= o) v += w;
  }
  return v;
}

// First lane l whose (nondecreasing) inclusive prefix incl[l] exceeds t.
// Requires t < incl[31].
__device__ __forceinline__ int warp_upper_bound(int incl, int t) {
  int lo = 0;
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    int v = __shfl_sync(kFull, incl, lo + s - 1);
    if (v <= t) lo += s;
  }
  return lo;
}

// First lane l whose (nondecreasing) value v[l] exceeds t, for any integer
// type; requires t < v[31].
template <typename T>
__device__ __forceinline__ int warp_upper_bound_t(T v, T t) {
  int lo = 0;
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    const T x = __shfl_sync(kFull, v, lo + s - 1);
    if (x <= t) lo += s;
  }
  return lo;
}

// Product in the reference's arithmetic: rounded to FP32, no contraction.
__device__ __forceinline__ float prod_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }

// Inserts key j into an open-addressing table of 2^log_t slots (linear
// probing).  Returns the slot and sets `fresh` when the key was new.
// Gives up after 2^log_t probes (table full): returns -1 and raises a flag.
__device__ __forceinline__ int hash_insert(int32_t* keys, int log_t, int32_t j, bool& fresh,
                                           int* flags) {
  const uint32_t mask = (1u << log_t) - 1u;
  uint32_t s = hash_slot(j, log_t);
  fresh = false;
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    int32_t k = keys[s];
    if (k == j) return (int)s;
    if (k == kEmpty) {
      int32_t old = atomicCAS(&keys[s], kEmpty, j);
      if (old == kEmpty) {
        fresh = true;
        return (int)s;
      }
      if (old == j) return (int)s;
    }
    s = (s + 1u) & mask;
  }
  raise_flag(flags, kFlagHashFull);
  return -1;
}

// Epoch-tagged keys-only table for counting: a slot holds (epoch << 24) | j,
// and a slot whose epoch differs from the current one counts as empty, so
// the table needs no clearing between rows (columns must be < 2^24).
// Returns true when j was new for this epoch.
__device__ __forceinline__ bool tagged_insert(int32_t* keys, int log_t, int32_t j, uint32_t epoch, int* flags) {
  const uint32_t mask = (1u << log_t) - 1u;
  const int32_t want = (int32_t)((epoch << 24) | (uint32_t)j);
  uint32_t s = hash_slot(j, log_t);
  for (uint32_t probe = 0; probe <= mask;) {
    const int32_t k = keys[s];
    if (k == want) return false;
    if (((uint32_t)k >> 24) != epoch) {
      const int32_t old = atomicCAS(&keys[s], k, want);
      if (old == k) return true;
      continue;  // the slot changed under us: look at it again
    }
    s = (s + 1u) & mask;
    ++probe;
  }
  raise_flag(flags, kFlagHashFull);
  return false;
}

// Looks up key j; returns its slot or -1.
__device__ __forceinline__ int hash_find(const int32_t* keys, int log_t, int32_t j) {
  const uint32_t mask = (1u << log_t) - 1u;
  uint32_t s = hash_slot(j, log_t);
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    int32_t k = keys[s];
    if (k == j) return (int)s;
    if (k == kEmpty) return -1;
    s = (s + 1u) & mask;
  }
  return -1;
}

// B-row segments shorter than this are packed several to a warp step; longer
// ones are read by the whole warp, one segment at a time.
constexpr int kPackBelow = 16;

// Visits every column c of the warp's 32 B-row segments [bs, bs + len) (one
// per lane) in no particular order: f(c).  Segments of kPackBelow or more
// entries are read by the whole warp, one at a time; shorter ones are packed
// into steps of 32 consecutive entries, so short rows of B do not leave
// lanes idle.
template <typename Off, typename F>
__device__ __forceinline__ void for_each_col(const int32_t* bcol, Off bs, int len, F&& f) {
  const int lane = lane_id();
  const bool is_long = len >= kPackBelow;
  const unsigned long_mask = __ballot_sync(kFull, is_long);
  for (unsigned m = long_mask; m; m &= m - 1) {
    const int l = __ffs(m) - 1;
    const Off sb = __shfl_sync(kFull, bs, l);
    const int sl = __shfl_sync(kFull, len, l);
    for (int q = lane; q < sl; q += 32) f(bcol[sb + q]);
  }
  const int sl = is_long ? 0 : len;
  const int incl = warp_incl_scan(sl);
  const int total = __shfl_sync(kFull, incl, 31);
  const int excl = incl - sl;
  for (int b0 = 0; b0 < total; b0 += 32) {
    const int tt = b0 + lane;
    const bool act = tt < total;
    const int src = warp_upper_bound(incl, act ? tt : total - 1);
    const Off sbs = __shfl_sync(kFull, bs, src);
    const int sex = __shfl_sync(kFull, excl, src);
    if (act) f(bcol[sbs + (Off)(tt - sex)]);
  }
}

// Sum, in lane order, of the values `pr` of the lanes in `grp` (a group of
// lanes sharing one output column, as found by __match_any_sync), started
// from v.  Every lane of the warp must call it; lanes whose group is
// theirs alone add just their own value.  Rounds = the largest group.
__device__ __forceinline__ float group_sum_in_lane_order(unsigned grp, float pr, float v, bool use) {
  const int rounds = (int)__reduce_max_sync(kFull, (unsigned)__popc(grp));
  unsigned rest = grp;
  for (int r = 0; r < rounds; ++r) {
    const bool has = rest != 0u;
    const int from = has ? __ffs(rest) - 1 : lane_id();
    rest &= rest - 1u;
    const float x = __shfl_sync(kFull, pr, from);
    if (use && has) v = add_rn(v, x);
  }
  return v;
}

// Bitonic sort of 32*E keys held in registers in striped order: element
// index = e * 32 + lane, ascending after the call.  Strides below 32 pair
// lanes (shuffles), larger ones pair registers of one lane.  The striped
// order makes the loads of the keys from shared memory and the stores of the
// sorted row contiguous across lanes (stencil 96^3 learned numeric 3.54 ->
// 3.31 ms against element index = lane * E + e).
template <int E>
__device__ __forceinline__ void warp_sort_keys_regs(int32_t (&key)[E]) {
  const int lane = lane_id();
  constexpr int N = 32 * E;
#pragma unroll
  for (int k = 2; k <= N; k <<= 1) {
#pragma unroll
    for (int s = k >> 1; s > 0; s >>= 1) {
      if (s < 32) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const int idx = e * 32 + lane;
          const int32_t pk = __shfl_xor_sync(kFull, key[e], s);
          const bool keep_small = ((idx & s) == 0) == ((idx & k) == 0);
          key[e] = keep_small ? min(pk, key[e]) : max(pk, key[e]);
        }
      } else {
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const int f = e ^ (s >> 5);
          if (f > e) {
            const int idx = e * 32 + lane;
            const bool asc = (idx & k) == 0;
            const int32_t x = key[e], y = key[f];
            key[e] = asc ? min(x, y) : max(x, y);
            key[f] = asc ? max(x, y) : min(x, y);
          }
        }
      }
    }
  }
}

// Sorts n distinct keys held in shared memory with one warp (bitonic network
// over next_pow2(n) <= cap slots; slots [n, np2) are padded with +inf).
static __device__ __noinline__ void warp_sort_keys(int32_t* keys, int n, int cap) {
  const int lane = lane_id();
  int np2 = 1;
  while (np2 < n) np2 <<= 1;
  if (np2 > cap) np2 = cap;
  for (int s = n + lane; s < np2; s += 32) keys[s] = 0x7fffffff;
  __syncwarp();
  for (int size = 2; size <= np2; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = lane; i < (np2 >> 1); i += 32) {
        int lo = ((i & ~(stride - 1)) << 1) | (i & (stride - 1));
        int hi = lo | stride;
        bool up = (lo & size) == 0;
        int32_t a = keys[lo], b = keys[hi];
        if ((a > b) == up) {
          keys[lo] = b;
          keys[hi] = a;
        }
      }
      __syncwarp();
    }
  }
}

}  // namespace spg
