// Host-side declarations of the predictor kernels.
#pragma once

#include <cstdint>

#include "kernels.hpp"

namespace spg {

constexpr int kMlpIn = 8;
constexpr int kMlpHidden = 64;
constexpr int kMlpOut = 2;
constexpr int kMlpParams = kMlpIn * kMlpHidden + kMlpHidden + kMlpHidden * kMlpHidden + kMlpHidden +
                           kMlpHidden * kMlpOut + kMlpOut;

void launch_features(const DCsr& A, const DCsr& B, float* feats, int64_t* prod, const LaunchCtx& lc);
void launch_mlp_predict(const void* w16, const float* feats, int64_t rows, float* out, const LaunchCtx& lc);
// Fused learned plan: per row products, MLP capacity and exact-path mark
// (capacity above learn_cap, or with bin_gate a predicted bin beyond the
// warp tables).
void launch_learned_plan(const DCsr& A, const DCsr& B, const void* w16, float margin, int slack, int64_t learn_cap,
                         int bin_gate, int force_overflow, int64_t* prod, int64_t* cap, uint8_t* need_exact,
                         unsigned long long* n_exact, const LaunchCtx& lc);
// The same over the R global rows of a batch (products with int32 row
// offsets of B); no bin gate.
struct BatchMat;
void launch_learned_plan_batch(const BatchMat* mats, const int32_t* row_mat, int64_t R, const void* w16, float margin,
                               int slack, int64_t learn_cap, int force_overflow, int64_t* prod, int64_t* cap,
                               uint8_t* need_exact, unsigned long long* n_exact, const LaunchCtx& lc);
// Forward + backward over n rows; `work` holds mlp_work_floats(n) floats;
// grad gets the full gradient (overwritten); loss (device) the mean loss.
void launch_mlp_fwd_bwd(const void* w16, const float* feats, const float* targets, int64_t n, float* work,
                        float* grad, float* loss, const LaunchCtx& lc);
int64_t mlp_work_floats(int64_t n);
void launch_adam(float* master, void* w16, float* grad, float* m, float* v, float lr, float beta1, float beta2,
                 float eps, float wd, int step, const LaunchCtx& lc);
void launch_to_bf16(const float* src, void* dst, int n, const LaunchCtx& lc);
void launch_make_targets(const int64_t* nnz, const int32_t* idx, int64_t n, float max_load, int64_t warp_cap,
                         float* targets, const LaunchCtx& lc);
void launch_gather_rows(const float* src, const int32_t* idx, int64_t n, int width, float* dst, const LaunchCtx& lc);

}  // namespace spg
