/*
 * CPU oracle for C = A*B on CSR matrices -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker for the CUDA engine: only tests/, the smoke()
 * entry and bench.py's CPU-baseline leg may load it.  The product path never
 * links it.
 *
 * What it restates.  The reference computes every intermediate product
 * a_ik * b_kj once per (ray, sphere) hit and adds it into a dense FP32 C:
 *   ray per A nonzero (i,k,a):          optixSpMSpM/src/optixSpMSpM/optixSpMSpM.cu:143-150
 *   hit set = the spheres of B row k:   optixSpMSpM/src/optixSpMSpM/Sphere.cpp:64-75
 *   C[i][j] += a * b  (product rounded
 *   to FP32 first, then an FP32 add):   optixSpMSpM/src/optixSpMSpM/optixSpMSpM.cu:246-258
 *   output row-major, 1-based:          optixSpMSpM/src/optixSpMSpM/optixSpMSpM.cpp:475-486
 * The reference's summation order is whatever order the atomics land in.
 * Here the order is fixed to the canonical Gustavson order -- for each row i,
 * k ascending through A's row, then j ascending through B's row k -- with
 * the product rounded to FP32 and then added in FP32 (no fused multiply-add;
 * this file must be compiled with -ffp-contract=off).  The CUDA engine uses
 * the same order, so its values are expected to match bit for bit.
 *
 * The FP64 twin accumulates the FP64 products in the same order, and the
 * bound array holds sum |a_ik * b_kj| per output entry (FP64), the scale the
 * 1e-5 relative tolerance is measured against.
 *
 * The structure of C is symbolic: an entry exists iff at least one product
 * lands on it, even if the values cancel to zero (cuSPARSE SpGEMM, the
 * reference's second executable, keeps the same structure:
 * cuSparse/src/main.cpp:504-539).  The dense writer of the ray-tracing path
 * drops exact zeros instead (optixSpMSpM.cpp:479); the engine's .mtx writer
 * can do either.
 *
 * Parity pin: no golden outputs ship with the reference.  The oracle is
 * checked against outputs of the reference's own cuSPARSE driver
 * (cuSparse/src/main.cpp, built by oracle/Makefile into oracle/_ref/) on
 * small seeded inputs, committed under tests/golden/.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#if defined(__FP_FAST_FMAF) && !defined(ORACLE_ALLOW_FMA)
#error "oracle must be built without FMA contraction (-ffp-contract=off, no -mfma)"
#endif

typedef struct {
    int64_t rows, cols;
    const int64_t *row_ptr;
    const int32_t *col_idx;
    const float *val;
} orc_csr;

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* Intermediate products per row: sum over k in A_i of |B_k|. */
void orc_row_products(const orc_csr *A, const orc_csr *B, int64_t *out) {
    int64_t r;
#pragma omp parallel for schedule(dynamic, 1024)
    for (r = 0; r < A->rows; ++r) {
        int64_t s = 0;
        for (int64_t p = A->row_ptr[r]; p < A->row_ptr[r + 1]; ++p) {
            int32_t k = A->col_idx[p];
            s += B->row_ptr[k + 1] - B->row_ptr[k];
        }
        out[r] = s;
    }
}

static int cmp_i32(const void *a, const void *b) {
    int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    return (x > y) - (x < y);
}

/* Per-thread sparse accumulator (dense over the columns of B). */
typedef struct {
    int64_t tag;     /* incremented per row; mark[j] == tag <=> j seen */
    int64_t *mark;   /* tag of the last row that touched column j */
    float *acc;
    double *acc64;
    double *bound;
    int32_t *list;
} spa_t;

static int spa_init(spa_t *s, int64_t cols, int want_values) {
    s->tag = 0;
    s->mark = (int64_t *)calloc((size_t)(cols ? cols : 1), sizeof(int64_t));
    s->list = (int32_t *)malloc((size_t)(cols ? cols : 1) * sizeof(int32_t));
    s->acc = NULL; s->acc64 = NULL; s->bound = NULL;
    if (want_values) {
        s->acc = (float *)malloc((size_t)(cols ? cols : 1) * sizeof(float));
        s->acc64 = (double *)malloc((size_t)(cols ? cols : 1) * sizeof(double));
        s->bound = (double *)malloc((size_t)(cols ? cols : 1) * sizeof(double));
    }
    return s->mark && s->list && (!want_values || (s->acc && s->acc64 && s->bound));
}

static void spa_free(spa_t *s) {
    free(s->mark); free(s->list); free(s->acc); free(s->acc64); free(s->bound);
}

/* Number of distinct output columns of row r; list left in s->list. */
static int64_t row_symbolic(const orc_csr *A, const orc_csr *B, int64_t r, spa_t *s) {
    int64_t n = 0;
    const int64_t tag = ++s->tag;
    for (int64_t p = A->row_ptr[r]; p < A->row_ptr[r + 1]; ++p) {
        int32_t k = A->col_idx[p];
        for (int64_t q = B->row_ptr[k]; q < B->row_ptr[k + 1]; ++q) {
            int32_t j = B->col_idx[q];
            if (s->mark[j] != tag) {
                s->mark[j] = tag;
                s->list[n++] = j;
            }
        }
    }
    return n;
}

/*
 * Canonical-order numeric row: k ascending, then j ascending in B_k.
 * ``twin`` also fills the FP64 twin and the |a*b| bound.
 */
static int64_t row_numeric(const orc_csr *A, const orc_csr *B, int64_t r, spa_t *s,
                           int twin) {
    int64_t n = 0;
    const int64_t tag = ++s->tag;
    for (int64_t p = A->row_ptr[r]; p < A->row_ptr[r + 1]; ++p) {
        int32_t k = A->col_idx[p];
        float a = A->val[p];
        double a64 = (double)a;
        for (int64_t q = B->row_ptr[k]; q < B->row_ptr[k + 1]; ++q) {
            int32_t j = B->col_idx[q];
            float b = B->val[q];
            float prod = a * b;                 /* rounded to FP32 */
            if (s->mark[j] != tag) {
                s->mark[j] = tag;
                s->list[n++] = j;
                s->acc[j] = 0.0f;
                if (twin) {
                    s->acc64[j] = 0.0;
                    s->bound[j] = 0.0;
                }
            }
            s->acc[j] = s->acc[j] + prod;       /* FP32 add, no contraction */
            if (twin) {
                double prod64 = a64 * (double)b;    /* exact in FP64 */
                s->acc64[j] += prod64;
                s->bound[j] += fabs(prod64);
            }
        }
    }
    qsort(s->list, (size_t)n, sizeof(int32_t), cmp_i32);
    return n;
}

/* nnz of every row of C (exact symbolic count). Returns 0 on success. */
int orc_row_nnz(const orc_csr *A, const orc_csr *B, int64_t *out) {
    int err = 0;
#pragma omp parallel
    {
        spa_t s;
        int ok = spa_init(&s, B->cols, 0);
        if (!ok) {
#pragma omp atomic write
            err = 1;
        }
        int64_t r;
#pragma omp for schedule(dynamic, 256)
        for (r = 0; r < A->rows; ++r) {
            if (ok) out[r] = row_symbolic(A, B, r, &s);
        }
        spa_free(&s);
    }
    return err;
}

/*
 * Full product.  C_row_ptr must hold the exclusive scan of orc_row_nnz
 * (rows+1 entries); col/val/val64/bound are nnz(C) long.  val64 and bound
 * may be NULL.  Returns 0 on success.
 */
int orc_spgemm(const orc_csr *A, const orc_csr *B, const int64_t *C_row_ptr,
               int32_t *C_col, float *C_val, double *C_val64, double *C_bound) {
    int err = 0;
#pragma omp parallel
    {
        spa_t s;
        int ok = spa_init(&s, B->cols, 1);
        if (!ok) {
#pragma omp atomic write
            err = 1;
        }
        int64_t r;
#pragma omp for schedule(dynamic, 256)
        for (r = 0; r < A->rows; ++r) {
            if (!ok) continue;
            int64_t n = row_numeric(A, B, r, &s, 1);
            int64_t base = C_row_ptr[r];
            if (n != C_row_ptr[r + 1] - base) {
#pragma omp atomic write
                err = 2;
                continue;
            }
            for (int64_t t = 0; t < n; ++t) {
                int32_t j = s.list[t];
                C_col[base + t] = j;
                C_val[base + t] = s.acc[j];
                if (C_val64) C_val64[base + t] = s.acc64[j];
                if (C_bound) C_bound[base + t] = s.bound[j];
            }
        }
        spa_free(&s);
    }
    return err;
}

/*
 * Rows ``sel[0..nsel)`` only, packed one after another: out_ptr gets nsel+1
 * offsets (caller sizes col/val with orc_rows_nnz).  Used to check sampled
 * rows of products whose full C does not fit in host memory.
 */
int orc_rows_nnz(const orc_csr *A, const orc_csr *B, const int64_t *sel, int64_t nsel,
                 int64_t *out) {
    int err = 0;
#pragma omp parallel
    {
        spa_t s;
        int ok = spa_init(&s, B->cols, 0);
        if (!ok) {
#pragma omp atomic write
            err = 1;
        }
        int64_t t;
#pragma omp for schedule(dynamic, 16)
        for (t = 0; t < nsel; ++t) {
            if (ok) {
                out[t] = row_symbolic(A, B, sel[t], &s);
            }
        }
        spa_free(&s);
    }
    return err;
}

int orc_rows(const orc_csr *A, const orc_csr *B, const int64_t *sel, int64_t nsel,
             const int64_t *out_ptr, int32_t *C_col, float *C_val, double *C_val64,
             double *C_bound) {
    int err = 0;
#pragma omp parallel
    {
        spa_t s;
        int ok = spa_init(&s, B->cols, 1);
        if (!ok) {
#pragma omp atomic write
            err = 1;
        }
        int64_t t;
#pragma omp for schedule(dynamic, 16)
        for (t = 0; t < nsel; ++t) {
            if (!ok) continue;
            int64_t n = row_numeric(A, B, sel[t], &s, 1);
            int64_t base = out_ptr[t];
            if (n != out_ptr[t + 1] - base) {
#pragma omp atomic write
                err = 2;
                continue;
            }
            for (int64_t u = 0; u < n; ++u) {
                int32_t j = s.list[u];
                C_col[base + u] = j;
                C_val[base + u] = s.acc[j];
                if (C_val64) C_val64[base + u] = s.acc64[j];
                if (C_bound) C_bound[base + u] = s.bound[j];
            }
        }
        spa_free(&s);
    }
    return err;
}

/*
 * Timed CPU baseline: the FP32 canonical product of rows [r0, r1) with a
 * per-thread accumulator, counting and filling in one sweep (no output kept
 * beyond a per-thread checksum, so the sample size is not bounded by host
 * memory).  Returns the sum of per-row nnz; *checksum gets a value checksum.
 */
int64_t orc_baseline_rows(const orc_csr *A, const orc_csr *B, int64_t r0, int64_t r1,
                          double *checksum) {
    int64_t total = 0;
    double cs = 0.0;
#pragma omp parallel reduction(+ : total, cs)
    {
        spa_t s;
        int ok = spa_init(&s, B->cols, 1);
        int64_t r;
#pragma omp for schedule(dynamic, 64)
        for (r = r0; r < r1; ++r) {
            if (!ok) continue;
            int64_t n = row_numeric(A, B, r, &s, 0);
            total += n;
            for (int64_t t = 0; t < n; ++t) cs += (double)s.acc[s.list[t]];
        }
        spa_free(&s);
    }
    if (checksum) *checksum = cs;
    return total;
}
