// FP64 check of a delivered product: every entry of C is recomputed from A
// and B in FP64 on the GPU and compared with the FP32 value C holds.
//
// The reference writes C without checking it (printResult,
// optixSpMSpM/src/optixSpMSpM/optixSpMSpM.cpp:452-494); the contract here
// asks for the error against FP64 per result.  The recomputation is
// independent of the engine's accumulators: one warp per row of C walks
// the row's products, finds each product's column in C's sorted row by
// binary search and adds a * b (exact in FP64: two FP32 factors) and
// |a * b| into FP64 sums.  Their order does not matter at FP64 precision
// for an error report of FP32 results.  Products whose column is missing
// from C's row, and entries of C that no product reaches, are counted.
// Rows are checked in blocks that fit a fixed scratch budget.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "context.hpp"

using namespace spg;

namespace {

constexpr int64_t kCheckMaxEntries = int64_t(1) << 26;  // entries of C per block (1.1 GB of scratch)

// Sums of the entries of C's rows [r0, r1): v[e] += a*b, s[e] += |a*b| for
// the entry e of C holding the product's column (e relative to c_rp[r0]).
__global__ void k_check_sums(DCsr A, DCsr B, const int64_t* c_rp, const int32_t* c_col, int64_t r0, int64_t r1,
                             double* v, double* s, uint8_t* hit, unsigned long long* missing) {
  const int lane = lane_id();
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t base = c_rp[r0];
  unsigned long long miss = 0;
  for (int64_t r = r0 + gw; r < r1; r += nw) {
    const int64_t cs = c_rp[r], ce = c_rp[r + 1];
    for (int64_t p = A.rp[r]; p < A.rp[r + 1]; ++p) {
      const int32_t k = A.col[p];
      const double a = (double)A.val[p];
      for (int64_t q = B.rp[k] + lane; q < B.rp[k + 1]; q += 32) {
        const int32_t j = B.col[q];
        int64_t lo = cs, hi = ce;
        while (lo < hi) {
          const int64_t m = (lo + hi) >> 1;
          if (c_col[m] < j) lo = m + 1;
          else hi = m;
        }
        if (lo < ce && c_col[lo] == j) {
          const double pr = a * (double)B.val[q];
          atomicAdd(&v[lo - base], pr);
          atomicAdd(&s[lo - base], fabs(pr));
          hit[lo - base] = 1;
        } else {
          ++miss;
        }
      }
    }
  }
  miss = warp_sum(miss);
  if (lane == 0 && miss) atomicAdd(missing, miss);
}

// Errors of the block's n entries: [0] max |c - v| (bits), [1] sum |c - v|
// (double bits, atomics), [2] max |c - v| / s (bits), [3] entries no product
// reaches.
__global__ void k_check_errors(const float* c_val, const double* v, const double* s, const uint8_t* hit, int64_t n,
                               unsigned long long* out) {
  double mx = 0.0, sum = 0.0, rel = 0.0;
  unsigned long long extra = 0;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    if (!hit[e]) {
      ++extra;
      continue;
    }
    const double err = fabs((double)c_val[e] - v[e]);
    mx = fmax(mx, err);
    sum += err;
    if (s[e] > 0.0) rel = fmax(rel, err / s[e]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmax(mx, __shfl_xor_sync(kFull, mx, o));
    rel = fmax(rel, __shfl_xor_sync(kFull, rel, o));
    sum += __shfl_xor_sync(kFull, sum, o);
    extra += __shfl_xor_sync(kFull, extra, o);
  }
  if (lane_id() == 0) {
    // non-negative doubles order like their bit patterns
    atomicMax(&out[0], (unsigned long long)__double_as_longlong(mx));
    atomicAdd(reinterpret_cast<double*>(&out[1]), sum);
    atomicMax(&out[2], (unsigned long long)__double_as_longlong(rel));
    atomicAdd(&out[3], extra);
  }
}

}  // namespace

extern "C" spg_status spg_check(spg_ctx* ctx, const spg_csr* A, const spg_csr* B, const spg_csr* C,
                                spg_check_report* out) {
  if (!ctx) return SPG_ERR_INVALID_ARG;
  if (!A || !B || !C || !out) return fail(ctx, SPG_ERR_INVALID_ARG, "null argument");
  if (A->cols != B->rows || C->rows != A->rows || C->cols != B->cols)
    return fail(ctx, SPG_ERR_INVALID_ARG, "C is not shaped like A * B");
  if (C->index_bits != 32 && C->index_bits != 64) return fail(ctx, SPG_ERR_INVALID_ARG, "bad C index_bits");
  SPG_CUDA(ctx, cudaSetDevice(ctx->device));
  std::memset(out, 0, sizeof *out);
  DevMat dA, dB, dC;
  SPG_TRY(prepare_matrix(ctx, A, dA, false));
  const bool same = same_matrix(A, B);
  if (!same) SPG_TRY(prepare_matrix(ctx, B, dB, false));
  SPG_TRY(prepare_matrix(ctx, C, dC, false));
  const DevMat& rB = same ? dA : dB;
  const LaunchCtx lc = launch_ctx(ctx);
  const int64_t rows = C->rows;
  // C's row pointers on the host, to cut the rows into blocks
  std::vector<int64_t> rp((size_t)rows + 1);
  SPG_CUDA(ctx, cudaMemcpyAsync(rp.data(), dC.view.rp, (size_t)(rows + 1) * 8, cudaMemcpyDeviceToHost, ctx->stream));
  SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const int64_t nnz = rp[(size_t)rows];
  const int64_t cap = std::min<int64_t>(std::max<int64_t>(nnz, 1), kCheckMaxEntries);
  DevBuf v, s, hit, acc;
  SPG_TRY(v.alloc(ctx, (size_t)cap * 8));
  SPG_TRY(s.alloc(ctx, (size_t)cap * 8));
  SPG_TRY(hit.alloc(ctx, (size_t)cap));
  SPG_TRY(acc.alloc(ctx, 5 * 8));
  SPG_CUDA(ctx, cudaMemsetAsync(acc.get(), 0, 5 * 8, ctx->stream));
  unsigned long long* d_acc = acc.as<unsigned long long>();
  double mx = 0.0, sum = 0.0, rel = 0.0;
  int64_t extra = 0;
  int64_t r0 = 0;
  while (r0 < rows) {
    // rows while their entries fit the scratch (a single row may exceed it:
    // such a row is rejected)
    int64_t r1 = r0 + 1;
    while (r1 < rows && rp[(size_t)r1 + 1] - rp[(size_t)r0] <= cap) ++r1;
    const int64_t n = rp[(size_t)r1] - rp[(size_t)r0];
    if (n > cap) return fail(ctx, SPG_ERR_UNSUPPORTED, "row %lld of C exceeds the check's scratch", (long long)r0);
    SPG_CUDA(ctx, cudaMemsetAsync(v.get(), 0, (size_t)n * 8, ctx->stream));
    SPG_CUDA(ctx, cudaMemsetAsync(s.get(), 0, (size_t)n * 8, ctx->stream));
    SPG_CUDA(ctx, cudaMemsetAsync(hit.get(), 0, (size_t)n, ctx->stream));
    SPG_CUDA(ctx, cudaMemsetAsync(d_acc, 0, 4 * 8, ctx->stream));
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((r1 - r0 + 7) / 8, (int64_t)ctx->sms * 16));
    k_check_sums<<<blocks, 256, 0, lc.stream>>>(dA.view, rB.view, dC.view.rp, dC.view.col, r0, r1, v.as<double>(),
                                                s.as<double>(), hit.as<uint8_t>(), d_acc + 4);
    const int eb = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)ctx->sms * 8));
    if (n > 0)
      k_check_errors<<<eb, 256, 0, lc.stream>>>(dC.view.val + rp[(size_t)r0], v.as<double>(), s.as<double>(),
                                                hit.as<uint8_t>(), n, d_acc);
    unsigned long long h[4];
    SPG_CUDA(ctx, cudaMemcpyAsync(h, d_acc, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    double bmx, bsum, brel;
    std::memcpy(&bmx, &h[0], 8);
    std::memcpy(&bsum, &h[1], 8);
    std::memcpy(&brel, &h[2], 8);
    mx = std::max(mx, bmx);
    sum += bsum;
    rel = std::max(rel, brel);
    extra += (int64_t)h[3];
    r0 = r1;
  }
  unsigned long long miss = 0;
  SPG_CUDA(ctx, cudaMemcpyAsync(&miss, d_acc + 4, 8, cudaMemcpyDeviceToHost, ctx->stream));
  SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  SPG_CUDA(ctx, cudaGetLastError());
  out->entries = nnz;
  out->max_abs_err_fp64 = mx;
  out->mean_abs_err_fp64 = nnz > extra ? sum / (double)(nnz - extra) : 0.0;
  out->max_rel_err = rel;
  out->missing = (int64_t)miss;
  out->extra = extra;
  return SPG_OK;
}
