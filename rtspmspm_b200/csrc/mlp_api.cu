// C-ABI of the learned row-size predictor: weights, training loop, and the
// hooks the tests use (features, exact nnz, inference, one gradient).
//
// Weight file (little endian): "SPGMLP\0\1", int32 version (1), int32 count
// (4866), count FP32 parameters in the layout of spg_mlp_get_params, then a
// uint32 FNV-1a checksum of the parameter bytes.
#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "context.hpp"

using namespace spg;

namespace {

constexpr char kMagic[8] = {'S', 'P', 'G', 'M', 'L', 'P', 0, 1};
constexpr int32_t kVersion = 1;

uint32_t fnv1a(const void* data, size_t n) {
  const unsigned char* p = static_cast<const unsigned char*>(data);
  uint32_t h = 2166136261u;
  for (size_t i = 0; i < n; ++i) {
    h ^= p[i];
    h *= 16777619u;
  }
  return h;
}

uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

std::vector<float> init_params(uint64_t seed) {
  std::vector<float> p(kMlpParams, 0.f);
  uint64_t s = seed;
  auto uni = [&](float a) {
    const double u = (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0);
    return (float)((2.0 * u - 1.0) * a);
  };
  int off = 0;
  const int fan_in[3] = {kMlpIn, kMlpHidden, kMlpHidden};
  const int fan_out[3] = {kMlpHidden, kMlpHidden, kMlpOut};
  for (int l = 0; l < 3; ++l) {
    const float a = l < 2 ? std::sqrt(6.0f / (float)fan_in[l]) : std::sqrt(1.0f / (float)fan_in[l]);
    for (int i = 0; i < fan_in[l] * fan_out[l]; ++i) p[off++] = uni(a);
    off += fan_out[l];  // biases stay 0
  }
  // start the size output near the ER prior (feature 7 is log2 of the
  // expected distinct count / 16): o0 ~ 16 * f7
  return p;
}

spg_status alloc_mlp(spg_ctx* ctx) {
  if (!ctx->mlp_master) SPG_CUDA(ctx, cudaMalloc(&ctx->mlp_master, kMlpParams * sizeof(float)));
  if (!ctx->mlp_w16) SPG_CUDA(ctx, cudaMalloc(&ctx->mlp_w16, kMlpParams * 2));
  return SPG_OK;
}

spg_status upload_params(spg_ctx* ctx, const float* host) {
  SPG_TRY(alloc_mlp(ctx));
  SPG_CUDA(ctx, cudaMemcpyAsync(ctx->mlp_master, host, kMlpParams * sizeof(float), cudaMemcpyHostToDevice,
                                ctx->stream));
  launch_to_bf16(ctx->mlp_master, ctx->mlp_w16, kMlpParams, launch_ctx(ctx));
  SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->mlp_loaded = true;
  return SPG_OK;
}

spg_status load_file(spg_ctx* ctx, const char* path) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(ctx, SPG_ERR_IO, "cannot open %s", path);
  char magic[8];
  int32_t ver = 0, count = 0;
  std::vector<float> p(kMlpParams);
  uint32_t sum = 0;
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kMagic, 8) == 0 &&
            std::fread(&ver, 4, 1, f) == 1 && ver == kVersion && std::fread(&count, 4, 1, f) == 1 &&
            count == kMlpParams && std::fread(p.data(), 4, kMlpParams, f) == (size_t)kMlpParams &&
            std::fread(&sum, 4, 1, f) == 1 && sum == fnv1a(p.data(), p.size() * 4);
  std::fclose(f);
  if (!ok) return fail(ctx, SPG_ERR_FORMAT, "%s is not a version-%d predictor file", path, kVersion);
  return upload_params(ctx, p.data());
}

std::string default_weights_path() {
  Dl_info info{};
  if (dladdr((void*)&spg_version, &info) && info.dli_fname) {
    std::string so(info.dli_fname);
    const size_t slash = so.rfind('/');
    const std::string dir = slash == std::string::npos ? "." : so.substr(0, slash);
    return dir + "/data/mlp_default.bin";
  }
  return "data/mlp_default.bin";
}

}  // namespace

namespace spg {

// Loads the shipped default weights, or a fixed random initialisation when
// no weight file is present (the learned path stays exact either way).
spg_status ensure_mlp(spg_ctx* ctx) {
  if (ctx->mlp_loaded) return SPG_OK;
  const std::string path = default_weights_path();
  FILE* f = std::fopen(path.c_str(), "rb");
  if (f) {
    std::fclose(f);
    if (load_file(ctx, path.c_str()) == SPG_OK) return SPG_OK;
  }
  std::vector<float> p = init_params(0);
  return upload_params(ctx, p.data());
}

}  // namespace spg

extern "C" {

spg_status spg_mlp_init(spg_ctx* ctx, uint64_t seed) {
  if (!ctx) return SPG_ERR_INVALID_ARG;
  SPG_CUDA(ctx, cudaSetDevice(ctx->device));
  std::vector<float> p = init_params(seed);
  return upload_params(ctx, p.data());
}

spg_status spg_mlp_load(spg_ctx* ctx, const char* path) {
  if (!ctx || !path) return SPG_ERR_INVALID_ARG;
  SPG_CUDA(ctx, cudaSetDevice(ctx->device));
  return load_file(ctx, path);
}

spg_status spg_mlp_get_params(spg_ctx* ctx, float* out, int64_t count) {
  if (!ctx || !out || count != kMlpParams) return SPG_ERR_INVALID_ARG;
  SPG_CUDA(ctx, cudaSetDevice(ctx->device));
  SPG_TRY(ensure_mlp(ctx));
  SPG_CUDA(ctx, cudaMemcpyAsync(out, ctx->mlp_master, kMlpParams * 4, cudaMemcpyDeviceToHost, ctx->stream));
  SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SPG_OK;
}

spg_status spg_mlp_set_params(spg_ctx* ctx, const float* in, int64_t count) {
  if (!ctx || !in || count != kMlpParams) return SPG_ERR_INVALID_ARG;
  SPG_CUDA(ctx, cudaSetDevice(ctx->device));
  return upload_params(ctx, in);
}

spg_status spg_mlp_save(spg_ctx* ctx, const char* path) {
  if (!ctx || !path) return SPG_ERR_INVALID_ARG;
  std::vector<float> p(kMlpParams);
  SPG_TRY(spg_mlp_get_params(ctx, p.data(), kMlpParams));
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(ctx, SPG_ERR_IO, "cannot write %s", path);
  const int32_t ver = kVersion, count = kMlpParams;
  const uint32_t sum = fnv1a(p.data(), p.size() * 4);
  bool ok = std::fwrite(kMagic, 1, 8, f) == 8 && std::fwrite(&ver, 4, 1, f) == 1 && std::fwrite(&count, 4, 1, f) == 1 &&
            std::fwrite(p.data(), 4, p.size(), f) == p.size() && std::fwrite(&sum, 4, 1, f) == 1;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? SPG_OK : fail(ctx, SPG_ERR_IO, "short write to %s", path);
}

spg_status spg_features(spg_ctx* ctx, const spg_csr* A, const spg_csr* B, float* d_out) {
  if (!ctx || !A || !B || !d_out) return SPG_ERR_INVALID_ARG;
  if (A->cols != B->rows) return fail(ctx, SPG_ERR_INVALID_ARG, "inner dimensions differ");
  SPG_CUDA(ctx, cudaSetDevice(ctx->device));
  DevMat dA, dB;
  SPG_TRY(prepare_matrix(ctx, A, dA, false));
  SPG_TRY(prepare_matrix(ctx, B, dB, false));
  launch_features(dA.view, dB.view, d_out, nullptr, launch_ctx(ctx));
  SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SPG_OK;
}

spg_status spg_row_nnz(spg_ctx* ctx, const spg_csr* A, const spg_csr* B, int64_t* d_out) {
  if (!ctx || !A || !B || !d_out) return SPG_ERR_INVALID_ARG;
  if (A->cols != B->rows) return fail(ctx, SPG_ERR_INVALID_ARG, "inner dimensions differ");
  SPG_CUDA(ctx, cudaSetDevice(ctx->device));
  DevMat dA, dB;
  SPG_TRY(prepare_matrix(ctx, A, dA, true));
  SPG_TRY(prepare_matrix(ctx, B, dB, true));
  int f = 0;
  SPG_TRY(read_flags(ctx, &f));
  if (f & kFlagBadIndex) return fail(ctx, SPG_ERR_INVALID_ARG, "input failed validation");
  SPG_TRY(row_nnz_device(ctx, dA, dB, d_out));
  SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SPG_OK;
}

spg_status spg_mlp_predict(spg_ctx* ctx, const float* d_features, int64_t rows, float* d_out) {
  if (!ctx || rows < 0 || (rows > 0 && (!d_features || !d_out))) return SPG_ERR_INVALID_ARG;
  SPG_CUDA(ctx, cudaSetDevice(ctx->device));
  SPG_TRY(ensure_mlp(ctx));
  launch_mlp_predict(ctx->mlp_w16, d_features, rows, d_out, launch_ctx(ctx));
  SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SPG_OK;
}

spg_status spg_mlp_grad(spg_ctx* ctx, const float* d_features, const float* d_targets, int64_t rows, float* loss,
                        float* grads) {
  if (!ctx || rows <= 0 || !d_features || !d_targets || !grads) return SPG_ERR_INVALID_ARG;
  SPG_CUDA(ctx, cudaSetDevice(ctx->device));
  SPG_TRY(ensure_mlp(ctx));
  DevBuf work, g, l;
  SPG_TRY(work.alloc(ctx, (size_t)mlp_work_floats(rows) * 4));
  SPG_TRY(g.alloc(ctx, kMlpParams * 4));
  SPG_TRY(l.alloc(ctx, 4));
  launch_mlp_fwd_bwd(ctx->mlp_w16, d_features, d_targets, rows, work.as<float>(), g.as<float>(), l.as<float>(),
                     launch_ctx(ctx));
  SPG_CUDA(ctx, cudaMemcpyAsync(grads, g.get(), kMlpParams * 4, cudaMemcpyDeviceToHost, ctx->stream));
  float lh = 0.f;
  SPG_CUDA(ctx, cudaMemcpyAsync(&lh, l.get(), 4, cudaMemcpyDeviceToHost, ctx->stream));
  SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (loss) *loss = lh;
  return SPG_OK;
}

spg_status spg_mlp_train(spg_ctx* ctx, int32_t n, const spg_csr* A, const spg_csr* B, const spg_train_opts* opts,
                         spg_train_report* report) {
  if (!ctx || n <= 0 || !A || !B) return SPG_ERR_INVALID_ARG;
  SPG_CUDA(ctx, cudaSetDevice(ctx->device));
  SPG_TRY(ensure_mlp(ctx));
  spg_train_opts o{};
  o.epochs = 20;
  o.batch = 4096;
  o.lr = 2e-3f;
  o.weight_decay = 1e-5f;
  o.max_rows_per_matrix = 20000;
  o.seed = 1;
  if (opts) {
    if (opts->epochs > 0) o.epochs = opts->epochs;
    if (opts->batch > 0) o.batch = opts->batch;
    if (opts->lr > 0) o.lr = opts->lr;
    if (opts->weight_decay >= 0) o.weight_decay = opts->weight_decay;
    if (opts->max_rows_per_matrix > 0) o.max_rows_per_matrix = opts->max_rows_per_matrix;
    o.seed = opts->seed;
  }
  const LaunchCtx lc = launch_ctx(ctx);
  const BinParams bp = bin_params(ctx->tuning);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, ctx->stream);
  std::mt19937_64 rng(o.seed);
  // 1) training set: features and exact-count targets of sampled rows
  std::vector<float> h_feats, h_tgts;
  for (int32_t m = 0; m < n; ++m) {
    if (A[m].cols != B[m].rows) return fail(ctx, SPG_ERR_INVALID_ARG, "pair %d: inner dimensions differ", m);
    DevMat dA, dB;
    SPG_TRY(prepare_matrix(ctx, &A[m], dA, true));
    SPG_TRY(prepare_matrix(ctx, &B[m], dB, true));
    int f = 0;
    SPG_TRY(read_flags(ctx, &f));
    if (f & kFlagBadIndex) return fail(ctx, SPG_ERR_INVALID_ARG, "pair %d failed validation", m);
    const int64_t rows = dA.view.rows;
    if (rows == 0) continue;
    DevBuf feats, prod, nnz, idx, gf, tg;
    SPG_TRY(feats.alloc(ctx, (size_t)rows * kMlpIn * 4));
    SPG_TRY(prod.alloc(ctx, (size_t)rows * 8));
    SPG_TRY(nnz.alloc(ctx, (size_t)rows * 8));
    launch_features(dA.view, dB.view, feats.as<float>(), prod.as<int64_t>(), lc);
    SPG_TRY(row_nnz_device(ctx, dA, dB, nnz.as<int64_t>()));
    std::vector<int64_t> hprod((size_t)rows);
    SPG_CUDA(ctx, cudaMemcpyAsync(hprod.data(), prod.get(), (size_t)rows * 8, cudaMemcpyDeviceToHost, ctx->stream));
    SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    std::vector<int32_t> cand;
    cand.reserve((size_t)rows);
    for (int64_t r = 0; r < rows; ++r)
      if (hprod[(size_t)r] > 0) cand.push_back((int32_t)r);
    if (cand.empty()) continue;
    std::shuffle(cand.begin(), cand.end(), rng);
    if ((int64_t)cand.size() > o.max_rows_per_matrix) cand.resize((size_t)o.max_rows_per_matrix);
    const int64_t k = (int64_t)cand.size();
    SPG_TRY(idx.alloc(ctx, (size_t)k * 4));
    SPG_TRY(gf.alloc(ctx, (size_t)k * kMlpIn * 4));
    SPG_TRY(tg.alloc(ctx, (size_t)k * kMlpOut * 4));
    SPG_CUDA(ctx, cudaMemcpyAsync(idx.get(), cand.data(), (size_t)k * 4, cudaMemcpyHostToDevice, ctx->stream));
    launch_gather_rows(feats.as<float>(), idx.as<int32_t>(), k, kMlpIn, gf.as<float>(), lc);
    launch_make_targets(nnz.as<int64_t>(), idx.as<int32_t>(), k, bp.max_load, bp.warp_cap, tg.as<float>(), lc);
    const size_t f0 = h_feats.size(), t0 = h_tgts.size();
    h_feats.resize(f0 + (size_t)k * kMlpIn);
    h_tgts.resize(t0 + (size_t)k * kMlpOut);
    SPG_CUDA(ctx, cudaMemcpyAsync(h_feats.data() + f0, gf.get(), (size_t)k * kMlpIn * 4, cudaMemcpyDeviceToHost,
                                  ctx->stream));
    SPG_CUDA(ctx, cudaMemcpyAsync(h_tgts.data() + t0, tg.get(), (size_t)k * kMlpOut * 4, cudaMemcpyDeviceToHost,
                                  ctx->stream));
    SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  const int64_t R = (int64_t)(h_tgts.size() / kMlpOut);
  if (R == 0) return fail(ctx, SPG_ERR_INVALID_ARG, "no rows with products in the training set");
  DevBuf dfeat, dtgt, perm, bfeat, btgt, work, grad, m1, m2, losses;
  SPG_TRY(dfeat.alloc(ctx, (size_t)R * kMlpIn * 4));
  SPG_TRY(dtgt.alloc(ctx, (size_t)R * kMlpOut * 4));
  SPG_CUDA(ctx, cudaMemcpyAsync(dfeat.get(), h_feats.data(), (size_t)R * kMlpIn * 4, cudaMemcpyHostToDevice,
                                ctx->stream));
  SPG_CUDA(ctx, cudaMemcpyAsync(dtgt.get(), h_tgts.data(), (size_t)R * kMlpOut * 4, cudaMemcpyHostToDevice,
                                ctx->stream));
  const int64_t bs = std::min<int64_t>(o.batch, R);
  const int64_t steps_per_epoch = (R + bs - 1) / bs;
  const int64_t total_steps = steps_per_epoch * o.epochs;
  SPG_TRY(perm.alloc(ctx, (size_t)R * 4));
  SPG_TRY(bfeat.alloc(ctx, (size_t)bs * kMlpIn * 4));
  SPG_TRY(btgt.alloc(ctx, (size_t)bs * kMlpOut * 4));
  SPG_TRY(work.alloc(ctx, (size_t)mlp_work_floats(bs) * 4));
  SPG_TRY(grad.alloc(ctx, kMlpParams * 4));
  SPG_TRY(m1.alloc(ctx, kMlpParams * 4));
  SPG_TRY(m2.alloc(ctx, kMlpParams * 4));
  SPG_TRY(losses.alloc(ctx, (size_t)total_steps * 4));
  SPG_CUDA(ctx, cudaMemsetAsync(m1.get(), 0, kMlpParams * 4, ctx->stream));
  SPG_CUDA(ctx, cudaMemsetAsync(m2.get(), 0, kMlpParams * 4, ctx->stream));
  std::vector<int32_t> order((size_t)R);
  std::iota(order.begin(), order.end(), 0);
  int step = 0;
  for (int ep = 0; ep < o.epochs; ++ep) {
    std::shuffle(order.begin(), order.end(), rng);
    SPG_CUDA(ctx, cudaMemcpyAsync(perm.get(), order.data(), (size_t)R * 4, cudaMemcpyHostToDevice, ctx->stream));
    // the host order buffer is reused next epoch: wait for the copy
    SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (int64_t b = 0; b < steps_per_epoch; ++b) {
      const int64_t s0 = b * bs;
      const int64_t cnt = std::min<int64_t>(bs, R - s0);
      launch_gather_rows(dfeat.as<float>(), perm.as<int32_t>() + s0, cnt, kMlpIn, bfeat.as<float>(), lc);
      launch_gather_rows(dtgt.as<float>(), perm.as<int32_t>() + s0, cnt, kMlpOut, btgt.as<float>(), lc);
      launch_mlp_fwd_bwd(ctx->mlp_w16, bfeat.as<float>(), btgt.as<float>(), cnt, work.as<float>(), grad.as<float>(),
                         losses.as<float>() + step, lc);
      ++step;
      const float lr = o.lr * 0.5f * (1.0f + std::cos(3.14159265f * (float)step / (float)total_steps));
      launch_adam(ctx->mlp_master, ctx->mlp_w16, grad.as<float>(), m1.as<float>(), m2.as<float>(), lr, 0.9f, 0.999f,
                  1e-8f, o.weight_decay, step, lc);
    }
  }
  std::vector<float> hl((size_t)total_steps);
  SPG_CUDA(ctx, cudaMemcpyAsync(hl.data(), losses.get(), (size_t)total_steps * 4, cudaMemcpyDeviceToHost,
                                ctx->stream));
  cudaEventRecord(e1, ctx->stream);
  SPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ctx->mlp_loaded = true;
  if (report) {
    double last = 0.0;
    for (int64_t b = total_steps - steps_per_epoch; b < total_steps; ++b) last += hl[(size_t)b];
    report->final_loss = last / (double)steps_per_epoch;
    report->ms_train = ms;
    report->rows_used = R;
    report->steps = (int32_t)total_steps;
  }
  return SPG_OK;
}

}  // extern "C"
