/*
 * rtspmspm.h -- C ABI of the B200 SpGEMM engine (C = A * B, CSR x CSR -> CSR).
 *
 * The reference has no library boundary: its hot path is reached through a
 * process CLI, `<bin> -m1 A.mtx -m2 B.mtx -o C.mtx -l log.txt`
 * (optixSpMSpM/src/optixSpMSpM/optixSpMSpM.cpp:513-562,
 * cuSparse/src/main.cpp:601-645), called by scripts/AE_test.py:207-215.
 * This header is the library slot under that CLI: the `spgemm` executable of
 * this project keeps the same four flags and calls only these entry points.
 *
 * Conventions
 *  - Every call returns an spg_status; no C++ exception crosses the ABI.
 *    spg_last_error(ctx) gives a message for the last failing call on ctx.
 *  - Indices are 0-based inside the library (the .mtx files are 1-based).
 *  - Column indices are int32, values FP32, row pointers int32 or int64
 *    (spg_csr.index_bits).  Input rows must be sorted by column with no
 *    duplicates (spg_mtx_read produces that form from any .mtx file).
 *  - One context per host thread; calls on a context are ordered on its
 *    CUDA stream.  All memory the library allocates belongs to the context.
 *  - Values are accumulated in FP32 in the canonical per-row order (k
 *    ascending through A's row, then j ascending through B's row k; the
 *    product is rounded to FP32 before the add), so results are identical
 *    run to run and across the plain, learned and batched methods.
 */
#ifndef RTSPMSPM_H
#define RTSPMSPM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t spg_status;
#define SPG_OK                 0
#define SPG_ERR_INVALID_ARG    1  /* bad pointer, shape mismatch, unsorted input */
#define SPG_ERR_CUDA           2  /* a CUDA runtime call failed */
#define SPG_ERR_OUT_OF_MEMORY  3  /* device or host allocation failed */
#define SPG_ERR_IO             4  /* file could not be opened / written */
#define SPG_ERR_FORMAT         5  /* malformed Matrix Market file */
#define SPG_ERR_TIMEOUT        6  /* a bounded device wait gave up */
#define SPG_ERR_UNSUPPORTED    7  /* feature not available in this build */
#define SPG_ERR_INTERNAL       8  /* device-side consistency check failed */

#define SPG_HOST    0
#define SPG_DEVICE  1

typedef struct spg_ctx spg_ctx;

/*
 * CSR matrix.  `row_ptr` has rows+1 entries of `index_bits` width.
 * Replaces the reference's two input layouts: the float3 (i, k, a) ray array
 * of matrix 1 (optixSpMSpM.cpp:73-131) and the sphere centre / colour arrays
 * of matrix 2 (Sphere.cpp:26-78, optixSpMSpM.cpp:136-162), and the
 * COO->CSR arrays of the cuSPARSE driver (cuSparse/src/main.cpp:439-456).
 */
typedef struct spg_csr {
    int64_t  rows;
    int64_t  cols;
    int64_t  nnz;
    int32_t  index_bits;  /* 32 or 64 */
    int32_t  location;    /* SPG_HOST or SPG_DEVICE */
    void*    row_ptr;
    int32_t* col_idx;
    float*   val;
    int64_t  capacity;    /* entries allocated behind col_idx/val (>= nnz) */
    int32_t  owner;       /* 0: caller memory; else allocated here, release with spg_csr_free */
    int32_t  reserved;
} spg_csr;

#define SPG_ALGO_PLAIN     0  /* symbolic pass + numeric pass (exact sizes; the fallback) */
#define SPG_ALGO_LEARNED   1  /* MLP-sized single numeric pass, overflow -> exact re-run */
#define SPG_ALGO_CUSPARSE  2  /* cusparseSpGEMM ALG3, reported reference point only */

typedef struct spg_opts {
    int32_t algo;            /* SPG_ALGO_* */
    int32_t out_location;    /* where C is returned: SPG_DEVICE (default) or SPG_HOST */
    int32_t out_index_bits;  /* 0: 32 if nnz(C) < 2^31 else 64; or force 32 / 64 */
    int32_t stage_timing;    /* 1: record CUDA events per stage into the report */
    int32_t force_overflow;  /* test hook: learned path predicts one entry per row */
    int32_t use_tuning;      /* 1: use the context's tuned parameters (spg_tune) */
    int32_t use_graph;       /* batched: capture/replay the launch sequence as a CUDA graph */
    int32_t skip_validation; /* 1: trust that inputs are sorted, in range and duplicate-free */
    int32_t reserved[4];
} spg_opts;

/* Stage indices of spg_report.ms_stage. */
#define SPG_STAGE_UPLOAD    0
#define SPG_STAGE_PRODUCTS  1
#define SPG_STAGE_BINNING   2
#define SPG_STAGE_SYMBOLIC  3
#define SPG_STAGE_SCAN      4
#define SPG_STAGE_NUMERIC   5
#define SPG_STAGE_FEATURES  6
#define SPG_STAGE_MLP       7
#define SPG_STAGE_FIXUP     8
#define SPG_STAGE_COMPACT   9
#define SPG_STAGE_DOWNLOAD  10
#define SPG_STAGE_COUNT     12

#define SPG_NUM_BINS 16

/*
 * Per-call report.  Replaces the reference's one-number timer
 * (optixSpMSpM/src/sutil/Timing.h:55-100) with per-stage device times.
 */
typedef struct spg_report {
    double  ms_total;                   /* device time of the whole call (events) */
    double  ms_stage[SPG_STAGE_COUNT];  /* filled when opts.stage_timing = 1 */
    int64_t products;                   /* intermediate products (flops = 2x) */
    int64_t nnz_c;
    int64_t rows;
    int64_t rows_predicted;             /* learned: rows sized by the MLP */
    int64_t rows_overflow;              /* learned: rows re-run by the exact fallback */
    int64_t rows_heavy;                 /* rows on the column-tiled heavy path */
    int64_t bin_rows[SPG_NUM_BINS];     /* numeric rows per accumulator bin */
    int32_t algo;
    int32_t device_flags;               /* bit set of SPG_FLAG_* raised by kernels */
    int32_t kernel_launches;            /* launches issued by this call */
    int32_t small_path;                 /* 1: the call took the small-product path */
} spg_report;

#define SPG_FLAG_HASH_FULL   1  /* a hash table filled up (kernel bug guard) */
#define SPG_FLAG_WAIT_LIMIT  2  /* a bounded wait gave up */
#define SPG_FLAG_BAD_INDEX   4  /* an index failed its bounds check */
#define SPG_FLAG_COUNT_DIFF  8  /* numeric count differs from symbolic count */

/* ---- context -------------------------------------------------------------- */

/* Creates a context on `device` with its own stream and memory pool.
 * Replaces the per-process set-up of the reference (OptiX context
 * optixSpMSpM.cpp:174-187; cusparseCreate cuSparse/src/main.cpp:437). */
spg_status spg_create(spg_ctx** ctx, int32_t device);
spg_status spg_destroy(spg_ctx* ctx);
const char* spg_last_error(const spg_ctx* ctx);
const char* spg_status_string(spg_status status);
/* Use a caller stream (cudaStream_t passed as void*); NULL restores the
 * context's own stream. */
spg_status spg_set_stream(spg_ctx* ctx, void* stream);
void* spg_get_stream(const spg_ctx* ctx);
int32_t spg_version(void);

/* ---- the product ---------------------------------------------------------- */

/*
 * C = A * B.  A and B may live on the host or on the device (host inputs are
 * uploaded inside the call).  C is allocated by the library at
 * opts->out_location and released with spg_csr_free.  `opts` and `report`
 * may be NULL.
 * Replaces: the ray-tracing launch and its set-up
 * (optixSpMSpM.cpp:585-611, any-hit accumulate optixSpMSpM.cu:220-261) and
 * the cuSPARSE sequence workEstimation -> estimateMemory -> compute -> copy
 * (cuSparse/src/main.cpp:430-539).
 */
spg_status spg_multiply(spg_ctx* ctx, const spg_csr* A, const spg_csr* B, spg_csr* C,
                        const spg_opts* opts, spg_report* report);

/*
 * C = A * B delivered into caller-owned host buffers, with the device-to-host
 * copy of C overlapped with the product: A's rows are taken in `blocks`
 * row blocks, and each block's part of C is copied on a second stream while
 * the next block is computed.  C->row_ptr (rows+1 entries of C->index_bits
 * width), C->col_idx and C->val (C->capacity entries) are host memory
 * (pinned memory gives the full host-link bandwidth); on success C->rows,
 * C->cols and C->nnz are set.  With too small a capacity the call fails
 * with SPG_ERR_INVALID_ARG and C->nnz holds the size needed.  A and B given
 * by the same descriptor are uploaded once.  Plain or learned method.
 * Replaces the reference's compute-then-copy sequence (optixSpMSpM.cpp:
 * 585-611 then printResult's device-to-host copy :462-463).
 */
spg_status spg_multiply_into_host(spg_ctx* ctx, const spg_csr* A, const spg_csr* B, spg_csr* C,
                                  int32_t blocks, const spg_opts* opts, spg_report* report);

/*
 * Value-only recompute: C already holds the structure of A * B (the result
 * of an earlier spg_multiply on matrices with the same structure as A and
 * B, on the device, either index width).  Recomputes C->val in place from
 * the current values of A and B; the products pass, the symbolic pass and
 * the scan are skipped (rows are binned by C's row lengths, heavy-row tiles
 * are counted from C's sorted columns).  C->col_idx is rewritten with the
 * same columns.  As with cuSPARSE's reuse, the caller guarantees that A and
 * B keep the structure C was computed from; a differing count of distinct
 * columns in a row (in a column tile holding entries of C, for rows beyond
 * the warp tables) fails the call with SPG_ERR_INVALID_ARG.
 * report->products is not computed (0).
 * Replaces: cusparseSpGEMMreuse_compute after the structure phase
 * (cuSparse/src/main.cpp:98-296, second compute with new values :286-296).
 */
spg_status spg_multiply_reuse(spg_ctx* ctx, const spg_csr* A, const spg_csr* B, spg_csr* C,
                              const spg_opts* opts, spg_report* report);

/*
 * n independent products C[i] = A[i] * B[i] of uneven sizes: all rows of all
 * products are binned together by table size and each stage runs one launch
 * per table size over every product's rows of that bin (bin bounds read on
 * the device); with opts->use_graph the launch sequence is captured once
 * into a CUDA graph and replayed on later calls with the same inputs.
 * Inputs must be on the device.  No reference counterpart (the reference
 * runs one product per process, scripts/AE_test.py:199-215).
 */
spg_status spg_multiply_batched(spg_ctx* ctx, int32_t n, const spg_csr* A, const spg_csr* B,
                                spg_csr* C, const spg_opts* opts, spg_report* report);

/*
 * Allocation-free C = A * B, for callers that cannot let a library call
 * cudaMalloc: processes whose device memory belongs to their own arena or
 * budget, and hot paths that must not risk an allocation's latency or an
 * out-of-memory failure mid-call.  No counterpart in the reference.
 * A and B are device matrices with at most 262,144 rows each, and every
 * output row must fit the warp hash tables (at most 2,048 intermediate
 * products per row, capped at the column count); larger inputs are
 * rejected with an error and a message in errbuf.  C carries caller-owned
 * device buffers: row_ptr (rows+1 entries of C->index_bits width) and
 * col_idx/val with C->capacity entries; on success C->nnz is set, and when
 * the capacity is too small the call fails with C->nnz holding the size
 * needed.  Runs on `stream` on the calling thread's current device.
 * All scratch lives in one file-scope device array of about 9.3 MB that
 * every GPU loading the library keeps until the process exits; the first
 * call on a device looks up that array's address (make that first call
 * before any stream capture).  The address is kept for the life of the
 * process: do not use this entry point across a cudaDeviceReset.  Every
 * call shares the array, so calls whose work overlaps on the GPU (other
 * streams, other threads) race and must be serialized by the caller.  On
 * an error return the contents of C's buffers are unspecified; a CUDA
 * error already pending when the call begins is reported, not cleared.
 */
spg_status spg_multiply_noalloc(void* stream, const spg_csr* A, const spg_csr* B, spg_csr* C,
                                char* errbuf, int32_t errlen);

/*
 * FP64 check of a product C = A * B (C from any method, on the host or the
 * device): every entry of C is recomputed from A and B in FP64 on the GPU
 * (the product of two FP32 factors is exact in FP64) and compared with C's
 * FP32 value.  Reports the max and mean |c - c64|, the max of
 * |c - c64| / sum|a*b| (the contract's bound is 1e-5), products whose
 * column is missing from C's row and entries of C that no product reaches.
 * Costs a binary search in C's row per intermediate product; rows are taken
 * in blocks of at most 2^26 entries of scratch.  The reference writes C
 * unchecked (printResult, optixSpMSpM.cpp:452-494); no counterpart.
 */
typedef struct spg_check_report {
    int64_t entries;
    int64_t missing;            /* products whose column is absent from C's row */
    int64_t extra;              /* entries of C that no product reaches */
    double  max_abs_err_fp64;   /* max |c - c64| */
    double  mean_abs_err_fp64;  /* mean |c - c64| over the reached entries */
    double  max_rel_err;        /* max |c - c64| / sum |a*b| */
    int32_t reserved[4];
} spg_check_report;

spg_status spg_check(spg_ctx* ctx, const spg_csr* A, const spg_csr* B, const spg_csr* C,
                     spg_check_report* out);

/* Releases a matrix allocated by the library (owner != 0); no-op otherwise. */
spg_status spg_csr_free(spg_ctx* ctx, spg_csr* m);

/* Copies a matrix to SPG_HOST or SPG_DEVICE (library-owned result). */
spg_status spg_csr_copy(spg_ctx* ctx, const spg_csr* src, int32_t location, spg_csr* dst);

/*
 * Copies a device matrix into caller-provided host buffers (rows+1 row
 * pointers of src->index_bits width, nnz columns, nnz values; pinned memory
 * gives full PCIe/C2C bandwidth) and waits for the copy.  Replaces the
 * reference's device-to-host result copies (optixSpMSpM.cpp:462-463,
 * cuSparse/src/main.cpp:555-558).
 */
spg_status spg_csr_download(spg_ctx* ctx, const spg_csr* src, void* row_ptr, int32_t* col_idx, float* val);

/*
 * Copies rows rows[0..n) of a device matrix into a new host matrix (n rows,
 * int64 row pointers, library-owned; release with spg_csr_free).  For
 * inspecting parts of a product too large to copy whole.  No reference
 * counterpart.
 */
spg_status spg_csr_extract_rows(spg_ctx* ctx, const spg_csr* src, const int64_t* rows, int64_t n, spg_csr* dst);

/*
 * Transpose of a host matrix into a new host matrix (int64 row pointers,
 * library-owned; release with spg_csr_free): a counting sort by column that
 * visits rows in order, so every row of the transpose keeps ascending
 * columns.  For C = A * B^T inputs, which the reference harness leaves as a
 * TODO (scripts/AE_test.py:165-171, 216-217).
 */
spg_status spg_csr_transpose(const spg_csr* src, spg_csr* dst);

/* ---- Matrix Market IO (host) --------------------------------------------- */

/*
 * Reads a `coordinate real|integer|pattern general|symmetric` .mtx into a
 * host CSR (int64 row_ptr, sorted columns, duplicates summed).
 * Replaces cooFromFile (cuSparse/src/util.cpp:9-44), mat1ToGPU's parser
 * (optixSpMSpM.cpp:73-131) and Sphere::Sphere (Sphere.cpp:26-78).
 */
spg_status spg_mtx_read(const char* path, spg_csr* out);

/*
 * COO -> CSR on the GPU.  n entries (0-based row_idx / col_idx, val) in any
 * order, in host (location = SPG_HOST) or device (SPG_DEVICE) memory,
 * become a device CSR of the context (int64 row_ptr, sorted columns) whose
 * duplicate (i, j) pairs are summed in FP32 in the order given, the first
 * value plus the second plus ... (as spg_mtx_read sums duplicates).
 * Entries outside rows x cols fail with SPG_ERR_INVALID_ARG.  Replaces the
 * reference's upload + cusparseXcoo2csr (cuSparse/src/main.cpp:408-442),
 * which needs row-sorted input and keeps duplicates.  Free with
 * spg_csr_free.
 */
spg_status spg_coo_to_csr(spg_ctx* ctx, int64_t rows, int64_t cols, int64_t n, const int32_t* row_idx,
                          const int32_t* col_idx, const float* val, int32_t location, spg_csr* out);

/*
 * spg_mtx_read's parse (all host threads) followed by spg_coo_to_csr: the
 * file's entries go to the GPU as COO and the CSR is built there, with the
 * same result as spg_mtx_read uploaded (bit for bit).  Replaces the
 * reference's reader + host-to-device copy + cusparseXcoo2csr
 * (cuSparse/src/util.cpp:9-44, cuSparse/src/main.cpp:408-442).
 */
spg_status spg_mtx_read_device(spg_ctx* ctx, const char* path, spg_csr* out);

/*
 * Writes `%%MatrixMarket matrix coordinate real general`, `rows cols nnz`,
 * then 1-based `i j v` lines in row-major order with sorted columns.
 * drop_zeros = 1 skips entries whose value is exactly 0, as the ray-tracing
 * writer does (optixSpMSpM.cpp:452-494); 0 writes every structural entry as
 * printCooToFile does (cuSparse/src/util.cpp:49-69).  Accepts host or device C.
 */
spg_status spg_mtx_write(spg_ctx* ctx, const char* path, const spg_csr* m, int32_t drop_zeros);

/* ---- learned row-size predictor ------------------------------------------- */

#define SPG_MLP_FEATURES 8
#define SPG_MLP_HIDDEN   64
#define SPG_MLP_OUTPUTS  2

/* Loads / saves the predictor weights (versioned binary file). */
spg_status spg_mlp_load(spg_ctx* ctx, const char* path);
spg_status spg_mlp_save(spg_ctx* ctx, const char* path);
/* Re-initialises the weights from `seed` (Kaiming-uniform). */
spg_status spg_mlp_init(spg_ctx* ctx, uint64_t seed);
/* Host copy of the FP32 master weights, layout W1[8x64] b1[64] W2[64x64]
 * b2[64] W3[64x2] b3[2] (row-major, in x out). */
#define SPG_MLP_PARAMS (8 * 64 + 64 + 64 * 64 + 64 + 64 * 2 + 2)
spg_status spg_mlp_get_params(spg_ctx* ctx, float* out, int64_t count);
spg_status spg_mlp_set_params(spg_ctx* ctx, const float* in, int64_t count);

typedef struct spg_train_opts {
    int32_t epochs;
    int32_t batch;            /* rows per minibatch */
    float   lr;               /* Adam learning rate */
    float   weight_decay;
    int64_t max_rows_per_matrix;  /* sampled rows per training matrix */
    uint64_t seed;
    int32_t reserved[4];
} spg_train_opts;

typedef struct spg_train_report {
    double  final_loss;
    double  ms_train;
    int64_t rows_used;
    int32_t steps;
    int32_t reserved;
} spg_train_report;

/*
 * Trains the predictor on the GPU with the engine's own forward and backward
 * kernels.  Labels are the exact per-row nnz from the symbolic pass of each
 * (A[i], B[i]) pair; features come from the feature kernel.
 */
spg_status spg_mlp_train(spg_ctx* ctx, int32_t n, const spg_csr* A, const spg_csr* B,
                         const spg_train_opts* opts, spg_train_report* report);

/* Features of every row of A*B into a device buffer rows x 8 (FP32). */
spg_status spg_features(spg_ctx* ctx, const spg_csr* A, const spg_csr* B, float* d_out);
/* Exact per-row nnz of A*B (plain symbolic pass) into a device int64 buffer. */
spg_status spg_row_nnz(spg_ctx* ctx, const spg_csr* A, const spg_csr* B, int64_t* d_out);
/* Predicted log2(1 + nnz) and bin per row into a device buffer rows x 2. */
spg_status spg_mlp_predict(spg_ctx* ctx, const float* d_features, int64_t rows, float* d_out);
/*
 * One forward + backward pass over a device batch (features rows x 8,
 * targets rows x 2); writes the mean loss and the gradient of every
 * parameter (SPG_MLP_PARAMS floats, host buffer).  Used to check the
 * backward kernels against an FP64 CPU reference.
 */
spg_status spg_mlp_grad(spg_ctx* ctx, const float* d_features, const float* d_targets,
                        int64_t rows, float* loss, float* grads);

/* ---- autotuner ------------------------------------------------------------ */

typedef struct spg_tuning {
    int32_t warp_table_max;    /* largest per-warp hash table (entries) */
    int32_t warps_per_block;   /* warps per CTA for the warp-hash bins; 0 (default):
                                  per kernel, the size with the most resident warps */
    float   max_load;          /* hash-table load factor used for sizing */
    int32_t tile_cols;         /* column width of a heavy-row tile (power of two) */
    int32_t block_table_max;   /* CTA hash table for the symbolic mid bin */
    float   predict_margin;    /* learned: capacity = margin * predicted + slack */
    int32_t predict_slack;
    float   learned_load;      /* learned: table load factor at the predicted capacity */
    int32_t heavy_path;        /* rows beyond the warp tables: 0 = every column tile rescans
                                  its row of A; 1 = products staged once per tile in HBM
                                  buckets when they fit (else as 0); 2 = as 0, with B-row
                                  segments of 64+ entries in a tile copied into shared
                                  memory by bulk copies (cp.async.bulk, mbarrier) */
    int32_t block_min_nnz;     /* > 0: rows with more output entries than this (and at most
                                  8192) use a CTA-wide hash table; 0 or -1 (default): off,
                                  warp tables and heavy-row tiles only */
    int32_t esc_min_prod;      /* rows of at least this many products (0: default 128) whose
                                  output keeps half of them or more, and that fit the warp's
                                  table memory, are expanded, radix sorted on their columns and
                                  folded instead of hashed; -1: off */
    int32_t small_rows;        /* products whose A has at most this many rows (0: default 8192;
                                  at most 65536), every row of at most 2048 products, take the
                                  small-product path in both methods (three launches, one host
                                  round trip); -1: off */
} spg_tuning;

spg_status spg_get_tuning(spg_ctx* ctx, spg_tuning* out);
spg_status spg_set_tuning(spg_ctx* ctx, const spg_tuning* in);
/*
 * Grid search over bin thresholds, hash sizes and block shapes on the given
 * products; the best setting is stored in the context and, when cache_path
 * is not NULL, in a JSON cache keyed by (shape class, GPU name).
 */
spg_status spg_tune(spg_ctx* ctx, int32_t n, const spg_csr* A, const spg_csr* B,
                    const char* cache_path, spg_tuning* best);

#ifdef __cplusplus
}
#endif

#endif /* RTSPMSPM_H */
