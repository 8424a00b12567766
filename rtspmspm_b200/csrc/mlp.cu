// Learned row-size predictor: feature kernel, inference kernel and the
// training kernels (forward + backward + Adam) of an 8 -> 64 -> 64 -> 2 MLP
// with BF16 weights and FP32 accumulation.
//
// No reference counterpart: the reference sizes its output as a dense
// rows x cols buffer (optixSpMSpM/src/optixSpMSpM/optixSpMSpM.cpp:164-171)
// and never predicts row sizes.  The predictor replaces the symbolic pass
// for rows whose predicted size is trusted; overflowing rows are re-run by
// the exact path, so results never depend on the network.
#include <cuda_bf16.h>

#include <algorithm>

#include "common.cuh"
#include "mlp.hpp"

namespace spg {

// Feature scaling: every feature is a log2 quantity divided by 16.
constexpr float kFeatScale = 1.0f / 16.0f;

// Integer statistics of row r of A*B, computed by one warp (valid in every
// lane): |A_r|, products, max / min touched |B_k|, the output column span
// [lo, hi] and a 32-product sample's distinct count.  The sample takes, per
// lane l, A entry s + l (rows of at most 32 entries, folded into the main
// pass) or s + l*len/32, and a hashed position of that entry's B row.
struct RowStats {
  int64_t len, sum, mx, mn;
  int lo, hi;
  int distinct, nsample;
};

template <bool R32>
__device__ __forceinline__ RowStats row_stats(const DCsr& A, const DCsr& B, int64_t r) {
  using Off = typename RowOff<R32>::T;
  const int lane = lane_id();
  const int64_t s = A.rp[r], e = A.rp[r + 1];
  const int64_t len = e - s;
  const uint32_t hsh = (uint32_t)r * 2654435761u + (uint32_t)lane * 40503u;
  Off sum = 0, mx = 0;
  Off mn = R32 ? (Off)0x7fffffff : (Off)INT64_MAX;
  int lo = 0x7fffffff, hi = -1;
  int32_t j = -1 - lane;
  bool valid = false;
  for (int64_t p = s + lane; p < e; p += 32) {
    const int32_t k = A.col[p];
    const Off bs = RowOff<R32>::at(B, k), be = RowOff<R32>::at(B, k + 1);
    const Off l = be - bs;
    sum += l;
    mx = l > mx ? l : mx;
    mn = l < mn ? l : mn;
    if (l > 0) {
      lo = min(lo, B.col[bs]);
      hi = max(hi, B.col[be - 1]);
      if (len <= 32) {
        j = B.col[bs + (Off)(hsh % (uint32_t)l)];
        valid = true;
      }
    }
  }
  if (len > 32) {
    const int64_t p = s + (int64_t)lane * len / 32;
    const int32_t k = A.col[p];
    const Off bs = RowOff<R32>::at(B, k), be = RowOff<R32>::at(B, k + 1);
    if (be > bs) {
      j = B.col[bs + (Off)(hsh % (uint32_t)(be - bs))];
      valid = true;
    }
  }
  RowStats st;
  if (R32) {
    // a row's products are at most nnz(B) < 2^31
    st.sum = (int64_t)__reduce_add_sync(kFull, (unsigned)sum);
    st.mx = __reduce_max_sync(kFull, (int)mx);
    st.mn = __reduce_min_sync(kFull, (int)mn);
    if (st.mn == 0x7fffffff) st.mn = 0;
  } else {
    st.sum = warp_sum((int64_t)sum);
    st.mx = warp_max((int64_t)mx);
    st.mn = warp_min((int64_t)mn);
    if (st.mn == INT64_MAX) st.mn = 0;
  }
  st.lo = __reduce_min_sync(kFull, lo);
  st.hi = __reduce_max_sync(kFull, hi);
  const unsigned vm = __ballot_sync(kFull, valid);
  const unsigned grp = __match_any_sync(kFull, j);
  const bool leader = valid && lane == __ffs(grp & vm) - 1;
  st.distinct = __popc(__ballot_sync(kFull, leader));
  st.nsample = __popc(vm);
  st.len = len;
  return st;
}

// Feature i of a row (i < 8); every log2 feature is scaled by 1/16:
//  0 log2(1 + |A_r|)               4 log2(1 + cols of B)
//  1 log2(1 + products)            5 log2(1 + output column span)
//  2 log2(1 + max touched |B_k|)   6 distinct fraction of a 32-product sample
//  3 log2(1 + min touched |B_k|)   7 log2(1 + cols (1 - exp(-products/cols)))
__device__ __forceinline__ float feature_of(const RowStats& st, int64_t bcols, int i) {
  const float cols = (float)bcols;
  const float fsum = (float)st.sum;
  if (i == 6) return st.nsample ? (float)st.distinct / (float)st.nsample : 0.f;
  float x;
  if (i == 7) {
    x = cols > 0.f ? -cols * expm1f(-fsum / cols) : 0.f;
  } else {
    x = i == 0 ? (float)st.len
      : i == 1 ? fsum
      : i == 2 ? (float)st.mx
      : i == 3 ? (float)st.mn
      : i == 4 ? cols
      : (st.hi >= st.lo ? (float)(st.hi - st.lo + 1) : 0.f);
  }
  return log2f(1.f + x) * kFeatScale;
}

// Features of every row of A*B (warp per row, lane i < 8 writes feature i),
// plus the products per row when `prod` is set.
template <bool R32>
__global__ void k_features(DCsr A, DCsr B, float* feats, int64_t* prod) {
  const int lane = lane_id();
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = gw; r < A.rows; r += nw) {
    const RowStats st = row_stats<R32>(A, B, r);
    if (lane < kMlpIn) feats[r * kMlpIn + lane] = feature_of(st, B.cols, lane);
    if (prod && lane == 0) prod[r] = st.sum;
  }
}

// Parameter offsets inside the flat parameter vector.
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpIn * kMlpHidden;
constexpr int kOffW2 = kOffB1 + kMlpHidden;
constexpr int kOffB2 = kOffW2 + kMlpHidden * kMlpHidden;
constexpr int kOffW3 = kOffB2 + kMlpHidden;
constexpr int kOffB3 = kOffW3 + kMlpHidden * kMlpOut;
static_assert(kOffB3 + kMlpOut == kMlpParams, "parameter layout");

// Loads the BF16 parameters (weights and biases) into shared memory as FP32.
__device__ __forceinline__ void load_params(const __nv_bfloat16* w, float* sw) {
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) sw[i] = __bfloat162float(w[i]);
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Tensor-core inference: the MLP on 16-row tiles with mma.sync m16n8k16
// (BF16 operands, FP32 accumulation).  Weights live in shared memory
// transposed (n-major, k contiguous) so each B fragment is one 32-bit load.
// ---------------------------------------------------------------------------

struct MlpSmem {
  uint32_t w1t[kMlpHidden * 8];        // [n][k/2], k padded 8 -> 16
  uint32_t w2t[kMlpHidden * 32];       // [n][k/2]
  uint32_t w3t[8 * 32];                // [n][k/2], n padded 2 -> 8
  float b1[kMlpHidden], b2[kMlpHidden], b3[kMlpOut];
};

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ uint32_t pack_raw(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  const uint32_t l = *reinterpret_cast<const uint16_t*>(&lo);
  const uint32_t h = *reinterpret_cast<const uint16_t*>(&hi);
  return l | (h << 16);
}

__device__ __forceinline__ void load_mlp_smem(const __nv_bfloat16* w, MlpSmem& sm) {
  const __nv_bfloat16 z = __float2bfloat16_rn(0.f);
  for (int i = threadIdx.x; i < kMlpHidden * 8; i += blockDim.x) {
    const int n = i / 8, kp = i % 8;
    const int k0 = 2 * kp, k1 = 2 * kp + 1;
    const __nv_bfloat16 lo = k0 < kMlpIn ? w[kOffW1 + k0 * kMlpHidden + n] : z;
    const __nv_bfloat16 hi = k1 < kMlpIn ? w[kOffW1 + k1 * kMlpHidden + n] : z;
    sm.w1t[i] = pack_raw(lo, hi);
  }
  for (int i = threadIdx.x; i < kMlpHidden * 32; i += blockDim.x) {
    const int n = i / 32, kp = i % 32;
    sm.w2t[i] = pack_raw(w[kOffW2 + (2 * kp) * kMlpHidden + n], w[kOffW2 + (2 * kp + 1) * kMlpHidden + n]);
  }
  for (int i = threadIdx.x; i < 8 * 32; i += blockDim.x) {
    const int n = i / 32, kp = i % 32;
    sm.w3t[i] = n < kMlpOut ? pack_raw(w[kOffW3 + (2 * kp) * kMlpOut + n], w[kOffW3 + (2 * kp + 1) * kMlpOut + n]) : 0u;
  }
  for (int i = threadIdx.x; i < kMlpHidden; i += blockDim.x) {
    sm.b1[i] = __bfloat162float(w[kOffB1 + i]);
    sm.b2[i] = __bfloat162float(w[kOffB2 + i]);
  }
  if (threadIdx.x < kMlpOut) sm.b3[threadIdx.x] = __bfloat162float(w[kOffB3 + threadIdx.x]);
  __syncthreads();
}

__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// MLP forward of a 16-row tile whose features sit in x (16 x 8, FP32).
// On return, lanes with (lane & 3) == 0 hold: out[0..1] = (o0, o1) of row
// lane/4 and out[2..3] = (o0, o1) of row lane/4 + 8.
__device__ __forceinline__ void mlp_tile(const MlpSmem& sm, const float* x, float (&out)[4]) {
  const int lane = lane_id();
  const int g = lane >> 2, q = lane & 3;
  uint32_t a[4];
  a[0] = pack_bf16(x[g * kMlpIn + 2 * q], x[g * kMlpIn + 2 * q + 1]);
  a[1] = pack_bf16(x[(g + 8) * kMlpIn + 2 * q], x[(g + 8) * kMlpIn + 2 * q + 1]);
  a[2] = 0u;
  a[3] = 0u;
  float h[8][4];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    float d[4] = {0.f, 0.f, 0.f, 0.f};
    mma16816(d, a, sm.w1t[(nt * 8 + g) * 8 + q], 0u);
    const int c = nt * 8 + 2 * q;
    h[nt][0] = fmaxf(d[0] + sm.b1[c], 0.f);
    h[nt][1] = fmaxf(d[1] + sm.b1[c + 1], 0.f);
    h[nt][2] = fmaxf(d[2] + sm.b1[c], 0.f);
    h[nt][3] = fmaxf(d[3] + sm.b1[c + 1], 0.f);
  }
  float h2[8][4];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) h2[nt][0] = h2[nt][1] = h2[nt][2] = h2[nt][3] = 0.f;
#pragma unroll
  for (int kb = 0; kb < 4; ++kb) {
    const uint32_t ak[4] = {pack_bf16(h[2 * kb][0], h[2 * kb][1]), pack_bf16(h[2 * kb][2], h[2 * kb][3]),
                            pack_bf16(h[2 * kb + 1][0], h[2 * kb + 1][1]),
                            pack_bf16(h[2 * kb + 1][2], h[2 * kb + 1][3])};
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
      mma16816(h2[nt], ak, sm.w2t[(nt * 8 + g) * 32 + kb * 8 + q], sm.w2t[(nt * 8 + g) * 32 + kb * 8 + 4 + q]);
  }
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const int c = nt * 8 + 2 * q;
    h2[nt][0] = fmaxf(h2[nt][0] + sm.b2[c], 0.f);
    h2[nt][1] = fmaxf(h2[nt][1] + sm.b2[c + 1], 0.f);
    h2[nt][2] = fmaxf(h2[nt][2] + sm.b2[c], 0.f);
    h2[nt][3] = fmaxf(h2[nt][3] + sm.b2[c + 1], 0.f);
  }
  float d3[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
  for (int kb = 0; kb < 4; ++kb) {
    const uint32_t ak[4] = {pack_bf16(h2[2 * kb][0], h2[2 * kb][1]), pack_bf16(h2[2 * kb][2], h2[2 * kb][3]),
                            pack_bf16(h2[2 * kb + 1][0], h2[2 * kb + 1][1]),
                            pack_bf16(h2[2 * kb + 1][2], h2[2 * kb + 1][3])};
    mma16816(d3, ak, sm.w3t[g * 32 + kb * 8 + q], sm.w3t[g * 32 + kb * 8 + 4 + q]);
  }
  out[0] = d3[0] + sm.b3[0];
  out[1] = d3[1] + sm.b3[1];
  out[2] = d3[2] + sm.b3[0];
  out[3] = d3[3] + sm.b3[1];
}

constexpr int kPlanWarps = 8;

// Inference on precomputed features: (log2(1+nnz), bin) per row.
__global__ void __launch_bounds__(kPlanWarps * 32) k_mlp_predict(const __nv_bfloat16* w, const float* feats,
                                                                 int64_t rows, float* out) {
  __shared__ MlpSmem sm;
  __shared__ float tile[kPlanWarps][16 * kMlpIn];
  load_mlp_smem(w, sm);
  const int lane = lane_id(), wib = threadIdx.x >> 5;
  const int64_t ntiles = (rows + 15) / 16;
  for (int64_t t = blockIdx.x * (int64_t)kPlanWarps + wib; t < ntiles; t += (int64_t)gridDim.x * kPlanWarps) {
    const int64_t r0 = t * 16;
    for (int i = lane; i < 16 * kMlpIn; i += 32) {
      const int64_t r = r0 + i / kMlpIn;
      tile[wib][i] = r < rows ? feats[r * kMlpIn + (i % kMlpIn)] : 0.f;
    }
    __syncwarp();
    float o[4];
    mlp_tile(sm, tile[wib], o);
    if ((lane & 3) == 0) {
      const int64_t ra = r0 + (lane >> 2), rb = ra + 8;
      if (ra < rows) {
        out[ra * kMlpOut + 0] = o[0];
        out[ra * kMlpOut + 1] = o[1];
      }
      if (rb < rows) {
        out[rb * kMlpOut + 0] = o[2];
        out[rb * kMlpOut + 1] = o[3];
      }
    }
    __syncwarp();
  }
}

// Capacity from a prediction: cap = min(bound, ceil(margin * (2^o0 - 1)) +
// slack); a row goes to the exact path (need_exact = 1, cap = 0) when its
// cap exceeds the largest table of the learned pass (learn_cap) or, with
// bin_gate, its predicted bin says beyond the warp tables; force_overflow
// sets cap = 1 (every row then overflows and is re-run).
__device__ __forceinline__ void capacity_of(int64_t p, int64_t cols, float o0, float o1, float margin, int slack,
                                            int64_t learn_cap, int bin_gate, int force_overflow, int64_t& cap,
                                            uint8_t& ex) {
  const int64_t u = p < cols ? p : cols;
  cap = 0;
  ex = 0;
  if (u <= 0) return;
  const float lg = fminf(fmaxf(o0, 0.f), 40.f);
  const double pred = exp2((double)lg) - 1.0;
  const double cd = ceil(pred * (double)margin) + (double)slack;
  int64_t c = cd >= (double)u ? u : (int64_t)cd;
  if (c < 1) c = 1;
  if (force_overflow) c = 1;
  if (c > learn_cap || (bin_gate && o1 > (float)kMaxLogT + 0.5f)) {
    ex = 1;
    c = 0;
  }
  cap = c;
}

// Learned plan: per 16-row tile, the warp gathers each row's statistics
// (row by row, the whole warp on a row), computes the tile's 128 features
// four per lane, runs the MLP on the tile with tensor cores, and writes the
// products, capacity and exact-path mark of every row; n_exact counts the
// rows marked for the exact path.  BATCH: rows are the global rows of a
// batch (each row's operands from its product's descriptor, rows = R),
// else the rows of A * B.
template <bool R32, bool BATCH>
__global__ void __launch_bounds__(kPlanWarps * 32) k_learned_plan(DCsr A, DCsr B, const BatchMat* mats,
                                                                  const int32_t* row_mat, int64_t rows,
                                                                  const __nv_bfloat16* w, float margin, int slack,
                                                                  int64_t learn_cap, int bin_gate,
                                                                  int force_overflow, int64_t* prod, int64_t* cap,
                                                                  uint8_t* need_exact,
                                                                  unsigned long long* n_exact) {
  __shared__ MlpSmem sm;
  __shared__ float tile[kPlanWarps][16 * kMlpIn];
  __shared__ int64_t tprod[kPlanWarps][16];
  __shared__ int64_t tcols[kPlanWarps][16];
  __shared__ RowStats tstat[kPlanWarps][16];
  load_mlp_smem(w, sm);
  const int lane = lane_id(), wib = threadIdx.x >> 5;
  const int64_t ntiles = (rows + 15) / 16;
  for (int64_t t = blockIdx.x * (int64_t)kPlanWarps + wib; t < ntiles; t += (int64_t)gridDim.x * kPlanWarps) {
    const int64_t r0 = t * 16;
    const int nr = rows - r0 < 16 ? (int)(rows - r0) : 16;
    for (int i = 0; i < nr; ++i) {
      RowStats st;
      int64_t bcols = B.cols;
      if (BATCH) {
        const BatchMat& M = mats[row_mat[r0 + i]];
        st = row_stats<R32>(M.A, M.B, r0 + i - M.row_start);
        bcols = M.B.cols;
      } else {
        st = row_stats<R32>(A, B, r0 + i);
      }
      if (lane == 0) {
        tstat[wib][i] = st;
        tprod[wib][i] = st.sum;
        tcols[wib][i] = bcols;
      }
    }
    if (lane >= nr && lane < 16) {
      tprod[wib][lane] = 0;
      tcols[wib][lane] = 0;
    }
    __syncwarp();
    // the tile's 128 features, four per lane
    for (int idx = lane; idx < 16 * kMlpIn; idx += 32) {
      const int i = idx / kMlpIn;
      tile[wib][idx] = i < nr ? feature_of(tstat[wib][i], tcols[wib][i], idx % kMlpIn) : 0.f;
    }
    __syncwarp();
    float o[4];
    mlp_tile(sm, tile[wib], o);
    if ((lane & 3) == 0) {
      const int ia = lane >> 2, ib = ia + 8;
      const int64_t ra = r0 + ia, rb = r0 + ib;
      if (ra < rows) {
        int64_t c;
        uint8_t ex;
        capacity_of(tprod[wib][ia], tcols[wib][ia], o[0], o[1], margin, slack, learn_cap, bin_gate, force_overflow,
                    c, ex);
        prod[ra] = tprod[wib][ia];
        cap[ra] = c;
        need_exact[ra] = ex;
        if (ex) atomicAdd(n_exact, 1ull);
      }
      if (rb < rows) {
        int64_t c;
        uint8_t ex;
        capacity_of(tprod[wib][ib], tcols[wib][ib], o[2], o[3], margin, slack, learn_cap, bin_gate, force_overflow,
                    c, ex);
        prod[rb] = tprod[wib][ib];
        cap[rb] = c;
        need_exact[rb] = ex;
        if (ex) atomicAdd(n_exact, 1ull);
      }
    }
    __syncwarp();
  }
}

// Training, step 1 of 3 (one thread per row of the minibatch): forward
// with BF16 weights; keeps h1, z2 and dL/do for the backward kernels.
// Loss = 0.5 * mean over rows of sum_o w_o (y_o - t_o)^2 with w = (1, 1/4).
constexpr int kTrainThreads = 128;
constexpr float kLossW0 = 1.0f;
constexpr float kLossW1 = 0.25f;

__global__ void __launch_bounds__(kTrainThreads) k_mlp_fwd(const __nv_bfloat16* w, const float* feats,
                                                             const float* targets, int64_t n, float inv_n,
                                                             float* h1_out, float* z2_out, float* do_out,
                                                             float* loss_rows) {
  extern __shared__ float sw[];
  load_params(w, sw);
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    const volatile float* vw = sw;
    float x[kMlpIn], h1[kMlpHidden];
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) x[i] = feats[r * kMlpIn + i];
#pragma unroll
    for (int j = 0; j < kMlpHidden; ++j) {
      float a = vw[kOffB1 + j];
#pragma unroll
      for (int i = 0; i < kMlpIn; ++i) a += x[i] * vw[kOffW1 + i * kMlpHidden + j];
      h1[j] = a > 0.f ? a : 0.f;
      h1_out[r * kMlpHidden + j] = h1[j];
    }
    float o0 = vw[kOffB3], o1 = vw[kOffB3 + 1];
#pragma unroll 1
    for (int j = 0; j < kMlpHidden; ++j) {
      float a = vw[kOffB2 + j];
#pragma unroll
      for (int i = 0; i < kMlpHidden; ++i) a += h1[i] * vw[kOffW2 + i * kMlpHidden + j];
      z2_out[r * kMlpHidden + j] = a;
      const float h = a > 0.f ? a : 0.f;
      o0 += h * vw[kOffW3 + j * kMlpOut + 0];
      o1 += h * vw[kOffW3 + j * kMlpOut + 1];
    }
    const float e0 = o0 - targets[r * kMlpOut + 0];
    const float e1 = o1 - targets[r * kMlpOut + 1];
    do_out[r * kMlpOut + 0] = kLossW0 * e0 * inv_n;
    do_out[r * kMlpOut + 1] = kLossW1 * e1 * inv_n;
    loss_rows[r] = 0.5f * (kLossW0 * e0 * e0 + kLossW1 * e1 * e1);
  }
}

// Training, step 2 of 3 (one thread per row): back-propagates dL/do into
// dL/dz2 and dL/dz1 (pre-activation gradients of both hidden layers).
__global__ void __launch_bounds__(kTrainThreads) k_mlp_bwd_rows(const __nv_bfloat16* w, int64_t n, const float* h1_in,
                                                                  const float* z2_in, const float* do_in,
                                                                  float* dz1_out, float* dz2_out) {
  extern __shared__ float sw[];
  load_params(w, sw);
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    const volatile float* vw = sw;
    const float d0 = do_in[r * kMlpOut + 0], d1 = do_in[r * kMlpOut + 1];
    float dh1[kMlpHidden];
#pragma unroll
    for (int i = 0; i < kMlpHidden; ++i) dh1[i] = 0.f;
#pragma unroll 1
    for (int j = 0; j < kMlpHidden; ++j) {
      const float z = z2_in[r * kMlpHidden + j];
      const float dz = z > 0.f ? d0 * vw[kOffW3 + j * kMlpOut + 0] + d1 * vw[kOffW3 + j * kMlpOut + 1] : 0.f;
      dz2_out[r * kMlpHidden + j] = dz;
#pragma unroll
      for (int i = 0; i < kMlpHidden; ++i) dh1[i] += dz * vw[kOffW2 + i * kMlpHidden + j];
    }
#pragma unroll
    for (int i = 0; i < kMlpHidden; ++i)
      dz1_out[r * kMlpHidden + i] = h1_in[r * kMlpHidden + i] > 0.f ? dh1[i] : 0.f;
  }
}

// Training, step 3 of 3 (one thread per parameter): each gradient is a sum
// over the minibatch rows in row order -- deterministic, no atomics.
__global__ void k_mlp_grad_reduce(const float* feats, int64_t n, const float* h1, const float* z2, const float* d_o,
                                  const float* dz1, const float* dz2, float* grad) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kMlpParams) return;
  float g = 0.f;
  if (p < kOffB1) {  // W1[f][i]
    const int f = (p - kOffW1) / kMlpHidden, i = (p - kOffW1) % kMlpHidden;
    for (int64_t r = 0; r < n; ++r) g += feats[r * kMlpIn + f] * dz1[r * kMlpHidden + i];
  } else if (p < kOffW2) {  // b1[i]
    const int i = p - kOffB1;
    for (int64_t r = 0; r < n; ++r) g += dz1[r * kMlpHidden + i];
  } else if (p < kOffB2) {  // W2[i][j]
    const int i = (p - kOffW2) / kMlpHidden, j = (p - kOffW2) % kMlpHidden;
    for (int64_t r = 0; r < n; ++r) g += h1[r * kMlpHidden + i] * dz2[r * kMlpHidden + j];
  } else if (p < kOffW3) {  // b2[j]
    const int j = p - kOffB2;
    for (int64_t r = 0; r < n; ++r) g += dz2[r * kMlpHidden + j];
  } else if (p < kOffB3) {  // W3[j][k]
    const int j = (p - kOffW3) / kMlpOut, k = (p - kOffW3) % kMlpOut;
    for (int64_t r = 0; r < n; ++r) {
      const float z = z2[r * kMlpHidden + j];
      g += (z > 0.f ? z : 0.f) * d_o[r * kMlpOut + k];
    }
  } else {  // b3[k]
    const int k = p - kOffB3;
    for (int64_t r = 0; r < n; ++r) g += d_o[r * kMlpOut + k];
  }
  grad[p] = g;
}

// Sum of per-row losses divided by n (single CTA, fixed order per thread).
__global__ void k_loss_mean(const float* loss_rows, int64_t n, float inv_n, float* out) {
  __shared__ float sh[32];
  float s = 0.f;
  for (int64_t r = threadIdx.x; r < n; r += blockDim.x) s += loss_rows[r];
  s = warp_sum(s);
  if (lane_id() == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    float v = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.f;
    v = warp_sum(v);
    if (threadIdx.x == 0) *out = v * inv_n;
  }
}

// Adam with decoupled weight decay on the FP32 master weights; refreshes
// the BF16 copy used by the forward kernels.
__global__ void k_adam(float* master, __nv_bfloat16* w16, float* grad, float* m, float* v, int n, float lr,
                       float beta1, float beta2, float eps, float wd, float bc1, float bc2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float g = grad[i];
    const float mi = beta1 * m[i] + (1.f - beta1) * g;
    const float vi = beta2 * v[i] + (1.f - beta2) * g * g;
    m[i] = mi;
    v[i] = vi;
    float p = master[i];
    p -= lr * ((mi / bc1) / (sqrtf(vi / bc2) + eps) + wd * p);
    master[i] = p;
    w16[i] = __float2bfloat16_rn(p);
  }
}

__global__ void k_to_bf16(const float* src, __nv_bfloat16* dst, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    dst[i] = __float2bfloat16_rn(src[i]);
}

// Training targets from exact nnz: t0 = log2(1 + nnz), t1 = numeric bin as
// log2 of the warp table size (kMaxLogT + 1 for heavy rows).
__global__ void k_make_targets(const int64_t* nnz, const int32_t* idx, int64_t n, float max_load, int64_t warp_cap,
                               float* targets) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = nnz[idx ? idx[t] : t];
    float b;
    if (v <= 0) b = (float)kMinLogT;
    else if (v > warp_cap) b = (float)(kMaxLogT + 1);
    else {
      int64_t need = (int64_t)ceilf((float)v / max_load);
      int lg = need <= 1 ? 0 : 64 - __clzll((unsigned long long)(need - 1));
      if (lg < kMinLogT) lg = kMinLogT;
      if (lg > kMaxLogT) lg = kMaxLogT;
      b = (float)lg;
    }
    targets[t * 2 + 0] = (float)log2(1.0 + (double)v);
    targets[t * 2 + 1] = b;
  }
}

// Gathers rows idx[0..n) of a rows x width float matrix.
__global__ void k_gather_rows(const float* src, const int32_t* idx, int64_t n, int width, float* dst) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n * width; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = t / width;
    dst[t] = src[(int64_t)idx[r] * width + (t % width)];
  }
}

// --------------------------------------------------------------------------

void launch_features(const DCsr& A, const DCsr& B, float* feats, int64_t* prod, const LaunchCtx& lc) {
  if (A.rows == 0) return;
  int64_t blocks = (A.rows * 32 + 255) / 256;
  if (blocks > lc.sms * 16) blocks = lc.sms * 16;
  if (B.rp32) k_features<true><<<(unsigned)blocks, 256, 0, lc.stream>>>(A, B, feats, prod);
  else k_features<false><<<(unsigned)blocks, 256, 0, lc.stream>>>(A, B, feats, prod);
}

static int mlp_blocks(int64_t rows, int threads, int sms) {
  int64_t b = (rows + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > sms * 8) b = sms * 8;
  return (int)b;
}

void launch_mlp_predict(const void* w16, const float* feats, int64_t rows, float* out, const LaunchCtx& lc) {
  if (rows == 0) return;
  const int64_t tiles = (rows + 15) / 16;
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((tiles + kPlanWarps - 1) / kPlanWarps, lc.sms * 8));
  k_mlp_predict<<<blocks, kPlanWarps * 32, 0, lc.stream>>>((const __nv_bfloat16*)w16, feats, rows, out);
}

void launch_learned_plan(const DCsr& A, const DCsr& B, const void* w16, float margin, int slack, int64_t learn_cap,
                         int bin_gate, int force_overflow, int64_t* prod, int64_t* cap, uint8_t* need_exact,
                         unsigned long long* n_exact, const LaunchCtx& lc) {
  if (A.rows == 0) return;
  const int64_t tiles = (A.rows + 15) / 16;
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((tiles + kPlanWarps - 1) / kPlanWarps, lc.sms * 8));
  if (B.rp32)
    k_learned_plan<true, false><<<blocks, kPlanWarps * 32, 0, lc.stream>>>(
        A, B, nullptr, nullptr, A.rows, (const __nv_bfloat16*)w16, margin, slack, learn_cap, bin_gate, force_overflow,
        prod, cap, need_exact, n_exact);
  else
    k_learned_plan<false, false><<<blocks, kPlanWarps * 32, 0, lc.stream>>>(
        A, B, nullptr, nullptr, A.rows, (const __nv_bfloat16*)w16, margin, slack, learn_cap, bin_gate, force_overflow,
        prod, cap, need_exact, n_exact);
}

void launch_learned_plan_batch(const BatchMat* mats, const int32_t* row_mat, int64_t R, const void* w16, float margin,
                               int slack, int64_t learn_cap, int force_overflow, int64_t* prod, int64_t* cap,
                               uint8_t* need_exact, unsigned long long* n_exact, const LaunchCtx& lc) {
  if (R == 0) return;
  const int64_t tiles = (R + 15) / 16;
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((tiles + kPlanWarps - 1) / kPlanWarps, lc.sms * 8));
  const DCsr none{};
  // every product of the batch's queue has 32-bit row offsets of B
  k_learned_plan<true, true><<<blocks, kPlanWarps * 32, 0, lc.stream>>>(
      none, none, mats, row_mat, R, (const __nv_bfloat16*)w16, margin, slack, learn_cap, 0, force_overflow, prod,
      cap, need_exact, n_exact);
}

void launch_mlp_fwd_bwd(const void* w16, const float* feats, const float* targets, int64_t n, float* work,
                        float* grad, float* loss, const LaunchCtx& lc) {
  if (n == 0) return;
  float* h1 = work;
  float* z2 = h1 + n * kMlpHidden;
  float* dz1 = z2 + n * kMlpHidden;
  float* dz2 = dz1 + n * kMlpHidden;
  float* d_o = dz2 + n * kMlpHidden;
  float* lrows = d_o + n * kMlpOut;
  const int blocks = mlp_blocks(n, kTrainThreads, lc.sms);
  const size_t smem = kMlpParams * sizeof(float);
  const float inv_n = 1.0f / (float)n;
  k_mlp_fwd<<<blocks, kTrainThreads, smem, lc.stream>>>((const __nv_bfloat16*)w16, feats, targets, n, inv_n, h1, z2,
                                                        d_o, lrows);
  k_mlp_bwd_rows<<<blocks, kTrainThreads, smem, lc.stream>>>((const __nv_bfloat16*)w16, n, h1, z2, d_o, dz1, dz2);
  k_mlp_grad_reduce<<<(kMlpParams + 127) / 128, 128, 0, lc.stream>>>(feats, n, h1, z2, d_o, dz1, dz2, grad);
  if (loss) k_loss_mean<<<1, 1024, 0, lc.stream>>>(lrows, n, inv_n, loss);
}

int64_t mlp_work_floats(int64_t n) { return n * (4 * kMlpHidden + kMlpOut + 1); }

void launch_adam(float* master, void* w16, float* grad, float* m, float* v, float lr, float beta1, float beta2,
                 float eps, float wd, int step, const LaunchCtx& lc) {
  const float bc1 = 1.f - powf(beta1, (float)step);
  const float bc2 = 1.f - powf(beta2, (float)step);
  k_adam<<<(kMlpParams + 255) / 256, 256, 0, lc.stream>>>(master, (__nv_bfloat16*)w16, grad, m, v, kMlpParams, lr,
                                                          beta1, beta2, eps, wd, bc1, bc2);
}

void launch_to_bf16(const float* src, void* dst, int n, const LaunchCtx& lc) {
  k_to_bf16<<<(n + 255) / 256, 256, 0, lc.stream>>>(src, (__nv_bfloat16*)dst, n);
}

void launch_make_targets(const int64_t* nnz, const int32_t* idx, int64_t n, float max_load, int64_t warp_cap,
                         float* targets, const LaunchCtx& lc) {
  if (n == 0) return;
  k_make_targets<<<mlp_blocks(n, 256, lc.sms), 256, 0, lc.stream>>>(nnz, idx, n, max_load, warp_cap, targets);
}

void launch_gather_rows(const float* src, const int32_t* idx, int64_t n, int width, float* dst, const LaunchCtx& lc) {
  if (n == 0) return;
  k_gather_rows<<<mlp_blocks(n * width, 256, lc.sms), 256, 0, lc.stream>>>(src, idx, n, width, dst);
}

}  // namespace spg
