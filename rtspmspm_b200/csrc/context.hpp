// Engine context and host-side helpers shared by the C-ABI implementation.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/rtspmspm.h"
#include "common.cuh"
#include "kernels.hpp"
#include "mlp.hpp"

struct spg_ctx {
  int device = 0;
  int sms = 148;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;  // device-to-host copies overlapped with compute (created on first use)
  cudaStream_t upload_stream = nullptr;  // host-to-device copies of input row chunks (created on first use)
  cudaMemPool_t pool = nullptr;
  std::string last_error;
  std::string gpu_name;
  spg_tuning tuning{};
  // predictor state (device)
  float* mlp_master = nullptr;  // FP32 master weights
  void* mlp_w16 = nullptr;      // BF16 copy used by the kernels
  bool mlp_loaded = false;
  // small device scratch
  int* d_flags = nullptr;
  unsigned long long* d_counter = nullptr;  // tile queue / retry counters (4 entries)
  // pinned host staging for small device->host reads
  int64_t* h_stage = nullptr;      // 64 words, mapped
  int64_t* h_stage_dev = nullptr;  // the same words seen from the device
  int launches = 0;
  // batched-launch graph cache
  void* batch_cache = nullptr;
};

namespace spg {

// Records a message on the context and returns `st`.
spg_status fail(spg_ctx* ctx, spg_status st, const char* fmt, ...);

// Converts a CUDA error into a status (and message); SPG_OK on success.
spg_status cuda_status(spg_ctx* ctx, cudaError_t e, const char* what);

#define SPG_CUDA(ctx, call)                                              \
  do {                                                                   \
    cudaError_t _e = (call);                                             \
    if (_e != cudaSuccess) return ::spg::cuda_status((ctx), _e, #call);  \
  } while (0)

#define SPG_TRY(call)                   \
  do {                                  \
    spg_status _s = (call);             \
    if (_s != SPG_OK) return _s;        \
  } while (0)

// Stream-ordered device allocation from the context's pool; released at
// scope exit (stream-ordered free) unless release() is called.
class DevBuf {
 public:
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { reset(); }
  spg_status alloc(spg_ctx* ctx, size_t bytes);
  void reset();
  void* release() {
    void* p = ptr_;
    ptr_ = nullptr;
    return p;
  }
  template <typename T>
  T* as() const {
    return static_cast<T*>(ptr_);
  }
  void* get() const { return ptr_; }

 private:
  spg_ctx* ctx_ = nullptr;
  void* ptr_ = nullptr;
};

inline LaunchCtx launch_ctx(const spg_ctx* ctx) { return LaunchCtx{ctx->stream, ctx->sms}; }

// Enqueues a copy of `bytes` (a multiple of 4) device bytes into the mapped
// staging words at host_dst (inside ctx->h_stage); valid after the next
// stream synchronisation.
spg_status stage_read(spg_ctx* ctx, void* host_dst, const void* dev_src, size_t bytes);

// Device view of an spg_csr already on the device with int64 row pointers.
struct DevMat {
  DCsr view{};
  int64_t nnz = 0;
  DevBuf rp64;      // widened row pointers when the input had int32 ones
  DevBuf rp32;      // narrowed row pointers when the input had int64 ones and nnz < 2^31
  DevBuf upload[3]; // copies of host inputs
  // set while the entries are still being uploaded in row chunks: kernels
  // that read every row (the heavy-row blocked index) wait for it
  cudaEvent_t complete = nullptr;
};

// Prepares `m` for the kernels: uploads host data and widens int32 row
// pointers.  `validate` runs the structure check kernel (flags raised on the
// context's device flag word).
spg_status prepare_matrix(spg_ctx* ctx, const spg_csr* m, DevMat& out, bool validate, bool defer_entries = false);

// A and B describe the same matrix (same storage): prepare it once.
bool same_matrix(const spg_csr* a, const spg_csr* b);

// Reads and clears the device flag word.
spg_status read_flags(spg_ctx* ctx, int* flags);

spg_tuning default_tuning();
BinParams bin_params(const spg_tuning& t);

// Pipelines (api.cu / batched.cu / cusparse_ref.cu).
spg_status multiply_device(spg_ctx* ctx, const DevMat& A, const DevMat& B, spg_csr* C, const spg_opts& o,
                           spg_report* rep);
spg_status multiply_cusparse(spg_ctx* ctx, const DevMat& A, const DevMat& B, spg_csr* C, const spg_opts& o,
                             spg_report* rep);
// Exact per-row nnz of A*B (int64, rows entries) with the plain symbolic pass.
spg_status row_nnz_device(spg_ctx* ctx, const DevMat& A, const DevMat& B, int64_t* d_nnz);
// Heavy-row numeric pass through per-tile staging buckets (heavy.cu);
// *done = false (nothing launched) when it does not apply.
spg_status heavy_staged(spg_ctx* ctx, const DCsr& A, const DCsr& B, const int32_t* heavy_rows, int64_t nheavy,
                        const int32_t* big_slot, const int32_t* tile_cnt, const int32_t* tile_off, int ntiles,
                        const int64_t* c_rp, int32_t* c_col, float* c_val, bool* done);

// Value-only recompute of C's values (C holds the structure of A*B).
spg_status multiply_reuse_device(spg_ctx* ctx, const DevMat& A, const DevMat& B, spg_csr* C, const spg_opts& o,
                                 spg_report* rep);
spg_status ensure_mlp(spg_ctx* ctx);
void free_batch_cache(spg_ctx* ctx);

// Stage timer on the context stream (CUDA events).
class StageTimer {
 public:
  StageTimer(spg_ctx* ctx, bool enabled);
  ~StageTimer();
  void mark(int stage);  // closes the previous stage, opens `stage`
  void finish(spg_report* rep);

 private:
  spg_ctx* ctx_;
  bool on_;
  cudaEvent_t start_ = nullptr;
  cudaEvent_t end_ = nullptr;
  std::vector<std::pair<int, cudaEvent_t>> marks_;
};

}  // namespace spg
