// cuSPARSE SpGEMM on the same GPU: a reported reference point, never the
// product path.  Mirrors the reference's second executable
// (cuSparse/src/main.cpp:365-591): CSR with 32-bit indices and FP32 values,
// workEstimation -> getNumProducts -> estimateMemory (chunk_fraction 0.01) ->
// compute -> copy with CUSPARSE_SPGEMM_ALG3 (main.cpp:430-539).
// opts.reserved[0] selects the algorithm: 0 = ALG3 (the reference's
// default), 1 = ALG1, 2 = ALG2.
#include <cusparse.h>

#include <cstring>

#include "context.hpp"

using namespace spg;

namespace {

struct SpHandle {
  cusparseHandle_t h = nullptr;
  cusparseSpMatDescr_t a = nullptr, b = nullptr, c = nullptr;
  cusparseSpGEMMDescr_t g = nullptr;
  ~SpHandle() {
    if (g) cusparseSpGEMM_destroyDescr(g);
    if (a) cusparseDestroySpMat(a);
    if (b) cusparseDestroySpMat(b);
    if (c) cusparseDestroySpMat(c);
    if (h) cusparseDestroy(h);
  }
};

}  // namespace

#define SPG_SPARSE(ctx, call)                                                                    \
  do {                                                                                           \
    cusparseStatus_t _s = (call);                                                                \
    if (_s != CUSPARSE_STATUS_SUCCESS)                                                           \
      return fail((ctx), _s == CUSPARSE_STATUS_ALLOC_FAILED || _s == CUSPARSE_STATUS_INSUFFICIENT_RESOURCES \
                             ? SPG_ERR_OUT_OF_MEMORY                                             \
                             : SPG_ERR_CUDA,                                                     \
                  "%s: %s", #call, cusparseGetErrorString(_s));                                  \
  } while (0)

namespace spg {

spg_status multiply_cusparse(spg_ctx* ctx, const DevMat& A, const DevMat& B, spg_csr* C, const spg_opts& o,
                             spg_report* rep) {
  if (A.nnz > INT32_MAX || B.nnz > INT32_MAX) return fail(ctx, SPG_ERR_UNSUPPORTED, "cuSPARSE path needs nnz < 2^31");
  const LaunchCtx lc = launch_ctx(ctx);
  StageTimer tm(ctx, false);
  DevBuf arp, brp, crp;
  SPG_TRY(arp.alloc(ctx, (size_t)(A.view.rows + 1) * 4));
  SPG_TRY(brp.alloc(ctx, (size_t)(B.view.rows + 1) * 4));
  SPG_TRY(crp.alloc(ctx, (size_t)(A.view.rows + 1) * 4));
  launch_narrow_rp(A.view.rp, A.view.rows + 1, arp.as<int32_t>(), lc);
  launch_narrow_rp(B.view.rp, B.view.rows + 1, brp.as<int32_t>(), lc);
  SpHandle H;
  SPG_SPARSE(ctx, cusparseCreate(&H.h));
  SPG_SPARSE(ctx, cusparseSetStream(H.h, ctx->stream));
  SPG_SPARSE(ctx, cusparseCreateCsr(&H.a, A.view.rows, A.view.cols, A.nnz, arp.get(), (void*)A.view.col,
                                    (void*)A.view.val, CUSPARSE_INDEX_32I, CUSPARSE_INDEX_32I,
                                    CUSPARSE_INDEX_BASE_ZERO, CUDA_R_32F));
  SPG_SPARSE(ctx, cusparseCreateCsr(&H.b, B.view.rows, B.view.cols, B.nnz, brp.get(), (void*)B.view.col,
                                    (void*)B.view.val, CUSPARSE_INDEX_32I, CUSPARSE_INDEX_32I,
                                    CUSPARSE_INDEX_BASE_ZERO, CUDA_R_32F));
  SPG_SPARSE(ctx, cusparseCreateCsr(&H.c, A.view.rows, B.view.cols, 0, crp.get(), nullptr, nullptr,
                                    CUSPARSE_INDEX_32I, CUSPARSE_INDEX_32I, CUSPARSE_INDEX_BASE_ZERO, CUDA_R_32F));
  SPG_SPARSE(ctx, cusparseSpGEMM_createDescr(&H.g));
  const float alpha = 1.0f, beta = 0.0f;
  const cusparseOperation_t op = CUSPARSE_OPERATION_NON_TRANSPOSE;
  const cusparseSpGEMMAlg_t alg = o.reserved[0] == 1 ? CUSPARSE_SPGEMM_ALG1
                                  : o.reserved[0] == 2 ? CUSPARSE_SPGEMM_ALG2
                                                       : CUSPARSE_SPGEMM_ALG3;
  size_t s1 = 0, s2 = 0, s3 = 0;
  DevBuf b1, b2, b3;
  SPG_SPARSE(ctx, cusparseSpGEMM_workEstimation(H.h, op, op, &alpha, H.a, H.b, &beta, H.c, CUDA_R_32F, alg, H.g,
                                                &s1, nullptr));
  SPG_TRY(b1.alloc(ctx, s1));
  SPG_SPARSE(ctx, cusparseSpGEMM_workEstimation(H.h, op, op, &alpha, H.a, H.b, &beta, H.c, CUDA_R_32F, alg, H.g,
                                                &s1, b1.get()));
  if (alg == CUSPARSE_SPGEMM_ALG3 || alg == CUSPARSE_SPGEMM_ALG2) {
    int64_t nprod = 0;
    SPG_SPARSE(ctx, cusparseSpGEMM_getNumProducts(H.g, &nprod));
    if (rep) rep->products = nprod;
    const float chunk = 0.01f;
    SPG_SPARSE(ctx, cusparseSpGEMM_estimateMemory(H.h, op, op, &alpha, H.a, H.b, &beta, H.c, CUDA_R_32F, alg, H.g,
                                                  chunk, &s3, nullptr, nullptr));
    SPG_TRY(b3.alloc(ctx, s3));
    SPG_SPARSE(ctx, cusparseSpGEMM_estimateMemory(H.h, op, op, &alpha, H.a, H.b, &beta, H.c, CUDA_R_32F, alg, H.g,
                                                  chunk, &s3, b3.get(), &s2));
    b3.reset();
    SPG_TRY(b2.alloc(ctx, s2));
    SPG_SPARSE(ctx, cusparseSpGEMM_compute(H.h, op, op, &alpha, H.a, H.b, &beta, H.c, CUDA_R_32F, alg, H.g, &s2,
                                           b2.get()));
  } else {
    SPG_SPARSE(ctx, cusparseSpGEMM_compute(H.h, op, op, &alpha, H.a, H.b, &beta, H.c, CUDA_R_32F, alg, H.g, &s2,
                                           nullptr));
    SPG_TRY(b2.alloc(ctx, s2));
    SPG_SPARSE(ctx, cusparseSpGEMM_compute(H.h, op, op, &alpha, H.a, H.b, &beta, H.c, CUDA_R_32F, alg, H.g, &s2,
                                           b2.get()));
  }
  int64_t cr = 0, cc = 0, cn = 0;
  SPG_SPARSE(ctx, cusparseSpMatGetSize(H.c, &cr, &cc, &cn));
  DevBuf ccol, cval;
  SPG_TRY(ccol.alloc(ctx, (size_t)cn * 4));
  SPG_TRY(cval.alloc(ctx, (size_t)cn * 4));
  SPG_SPARSE(ctx, cusparseCsrSetPointers(H.c, crp.get(), ccol.get(), cval.get()));
  SPG_SPARSE(ctx, cusparseSpGEMM_copy(H.h, op, op, &alpha, H.a, H.b, &beta, H.c, CUDA_R_32F, alg, H.g));
  std::memset(C, 0, sizeof *C);
  C->rows = A.view.rows;
  C->cols = B.view.cols;
  C->nnz = cn;
  C->capacity = cn;
  C->index_bits = 32;
  C->location = SPG_DEVICE;
  C->row_ptr = crp.release();
  C->col_idx = static_cast<int32_t*>(ccol.release());
  C->val = static_cast<float*>(cval.release());
  C->owner = 1;
  tm.finish(rep);
  if (rep) rep->nnz_c = cn;
  return SPG_OK;
}

}  // namespace spg
