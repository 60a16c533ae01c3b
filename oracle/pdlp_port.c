/*
 * pdlp_port.c -- CPU restatement of the reference PDLP engine, in plain C.
 *
 * TEST INFRASTRUCTURE ONLY. This is the oracle the GPU engine is checked
 * against when the reference library itself (oracle/_ref) is not available;
 * it is pinned against that library by tests/test_oracle_pin.py, bit for bit
 * on the serial path when both are built with oracle/Makefile's parity flags.
 * Nothing in the product links, loads or calls it.
 *
 * Every routine follows the serial path (threadCount = 1) of the reference at
 * Aryan-Kumar06/optimisation_solver, pdlp_engine/, and cites the file:line it
 * restates. The arithmetic is performed in the same order as the reference so
 * that results agree exactly; the structure (flat arrays, one solver context
 * struct) is this file's own.
 */
#define _POSIX_C_SOURCE 199309L
#include "oracle_abi.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define ORC_INF (1.0 / 0.0)

/* ------------------------------------------------------------------ */
/* Small helpers                                                        */
/* ------------------------------------------------------------------ */

static double dmin(double a, double b) { return b < a ? b : a; }   /* std::min */
static double dmax(double a, double b) { return a < b ? b : a; }   /* std::max */
static double clip(double v, double lo, double hi) { return dmax(lo, dmin(v, hi)); }
/* std::clamp: differs from clip() only for NaN, which clamp passes through. */
static double clampd(double v, double lo, double hi) { return v < lo ? lo : (hi < v ? hi : v); }
static int is_finite(double v) { return isfinite(v) ? 1 : 0; }

static double now_seconds(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static void* xmalloc(size_t bytes) {
    void* p = malloc(bytes ? bytes : 1);
    if (!p) {
        fprintf(stderr, "pdlp_port: out of memory\n");
        abort();
    }
    return p;
}

static double* dvec(int64_t n) { return (double*)xmalloc((size_t)n * sizeof(double)); }
static double* dzeros(int64_t n) { return (double*)calloc((size_t)(n ? n : 1), sizeof(double)); }
static double* dcopy(const double* src, int64_t n) {
    double* d = dvec(n);
    if (n) memcpy(d, src, (size_t)n * sizeof(double));
    return d;
}

/* ------------------------------------------------------------------ */
/* Sparse matrix: CSR plus its transpose (CSC of A)                     */
/* sparse_matrix.h:52-135                                               */
/* ------------------------------------------------------------------ */

typedef struct Matrix {
    int32_t rows, cols;
    int64_t nnz;
    int64_t* row_start;   /* [rows+1] */
    int32_t* col_index;   /* [nnz] */
    double* values;       /* [nnz] */
    int64_t* col_start;   /* [cols+1] */
    int32_t* row_index;   /* [nnz] */
    double* cvalues;      /* [nnz] */
} Matrix;

static void matrix_free(Matrix* m) {
    free(m->row_start); free(m->col_index); free(m->values);
    free(m->col_start); free(m->row_index); free(m->cvalues);
    memset(m, 0, sizeof(*m));
}

/* CSC from CSR by counting sort over CSR in row order, which leaves each
 * column sorted by row (sparse_matrix.cpp:171-198). */
static void matrix_build_transpose(Matrix* m) {
    m->col_start = (int64_t*)calloc((size_t)m->cols + 1, sizeof(int64_t));
    for (int64_t k = 0; k < m->nnz; ++k) m->col_start[m->col_index[k] + 1]++;
    for (int32_t j = 0; j < m->cols; ++j) m->col_start[j + 1] += m->col_start[j];
    m->row_index = (int32_t*)xmalloc((size_t)m->nnz * sizeof(int32_t));
    m->cvalues = dvec(m->nnz);
    int64_t* cursor = (int64_t*)xmalloc(((size_t)m->cols + 1) * sizeof(int64_t));
    memcpy(cursor, m->col_start, ((size_t)m->cols + 1) * sizeof(int64_t));
    for (int32_t i = 0; i < m->rows; ++i) {
        for (int64_t k = m->row_start[i]; k < m->row_start[i + 1]; ++k) {
            const int64_t pos = cursor[m->col_index[k]]++;
            m->row_index[pos] = i;
            m->cvalues[pos] = m->values[k];
        }
    }
    free(cursor);
}

typedef struct Entry { int32_t col; int32_t order; double value; } Entry;

static int entry_cmp(const void* a, const void* b) {
    const Entry* x = (const Entry*)a;
    const Entry* y = (const Entry*)b;
    if (x->col != y->col) return x->col < y->col ? -1 : 1;
    return x->order < y->order ? -1 : (x->order > y->order);
}

/* SparseMatrix::fromTriplets (sparse_matrix.cpp:76-201): counting sort by row,
 * per-row sort by column, duplicates summed, exact zeros dropped. Duplicates
 * are summed in input order; the reference's unstable per-row sort can only
 * give a different result when three or more entries share one position. */
static int matrix_from_triplets(int32_t rows, int32_t cols, int64_t count,
                                const int32_t* ti, const int32_t* tj, const double* tv,
                                Matrix* out) {
    memset(out, 0, sizeof(*out));
    if (rows < 0 || cols < 0) return -1;
    for (int64_t k = 0; k < count; ++k) {
        if (ti[k] < 0 || ti[k] >= rows || tj[k] < 0 || tj[k] >= cols) return -1;
        if (!is_finite(tv[k])) return -1;
    }
    out->rows = rows;
    out->cols = cols;
    int64_t* start = (int64_t*)calloc((size_t)rows + 1, sizeof(int64_t));
    for (int64_t k = 0; k < count; ++k) start[ti[k] + 1]++;
    for (int32_t i = 0; i < rows; ++i) start[i + 1] += start[i];
    Entry* scattered = (Entry*)xmalloc((size_t)(count ? count : 1) * sizeof(Entry));
    int64_t* cursor = (int64_t*)xmalloc(((size_t)rows + 1) * sizeof(int64_t));
    memcpy(cursor, start, ((size_t)rows + 1) * sizeof(int64_t));
    for (int64_t k = 0; k < count; ++k) {
        const int64_t pos = cursor[ti[k]]++;
        scattered[pos].col = tj[k];
        scattered[pos].order = (int32_t)(pos - start[ti[k]]);
        scattered[pos].value = tv[k];
    }
    free(cursor);

    out->row_start = (int64_t*)calloc((size_t)rows + 1, sizeof(int64_t));
    out->col_index = (int32_t*)xmalloc((size_t)(count ? count : 1) * sizeof(int32_t));
    out->values = dvec(count ? count : 1);
    int64_t written = 0;
    for (int32_t i = 0; i < rows; ++i) {
        Entry* row = scattered + start[i];
        const int64_t len = start[i + 1] - start[i];
        qsort(row, (size_t)len, sizeof(Entry), entry_cmp);
        for (int64_t k = 0; k < len;) {
            const int32_t col = row[k].col;
            double acc = row[k].value;
            ++k;
            while (k < len && row[k].col == col) {
                acc += row[k].value;
                ++k;
            }
            if (acc != 0.0) {
                out->col_index[written] = col;
                out->values[written] = acc;
                ++written;
            }
        }
        out->row_start[i + 1] = written;
    }
    out->nnz = written;
    free(scattered);
    free(start);
    matrix_build_transpose(out);
    return 0;
}

/* The caller's CSR, canonicalised through matrix_from_triplets exactly as the
 * reference builds every CompiledLp (src/adapter/pdlp_adapter.cpp:124-167).
 * Returns NULL or the reference's exception message. */
static const char* matrix_from_lp(const orc_lp* lp, Matrix* m) {
    const int64_t count = lp->nnz;
    int32_t* ti = (int32_t*)xmalloc((size_t)(count ? count : 1) * sizeof(int32_t));
    for (int32_t i = 0; i < lp->rows; ++i)
        for (int64_t k = lp->row_start[i]; k < lp->row_start[i + 1]; ++k) ti[k] = i;
    const char* error = NULL;
    for (int64_t k = 0; k < count; ++k) {
        if (lp->col_index[k] < 0 || lp->col_index[k] >= lp->cols) {
            error = "Sparse matrix triplet index is out of range";
            break;
        }
        if (!is_finite(lp->values[k])) {
            error = "Sparse matrix coefficient must be finite";
            break;
        }
    }
    if (!error && matrix_from_triplets(lp->rows, lp->cols, count, ti, lp->col_index,
                                       lp->values, m) != 0) {
        error = "Sparse matrix dimensions must be nonnegative";
    }
    free(ti);
    return error;
}

/* SparseMatrix::validate (sparse_matrix.cpp:203-241). */
static int matrix_valid(const Matrix* m) {
    if (m->rows < 0 || m->cols < 0) return 0;
    if (m->row_start[0] != 0 || m->col_start[0] != 0) return 0;
    if (m->row_start[m->rows] != m->nnz || m->col_start[m->cols] != m->nnz) return 0;
    for (int32_t i = 0; i < m->rows; ++i)
        if (m->row_start[i + 1] < m->row_start[i]) return 0;
    for (int32_t j = 0; j < m->cols; ++j)
        if (m->col_start[j + 1] < m->col_start[j]) return 0;
    for (int64_t k = 0; k < m->nnz; ++k) {
        if (m->col_index[k] < 0 || m->col_index[k] >= m->cols || !is_finite(m->values[k])) return 0;
        if (m->row_index[k] < 0 || m->row_index[k] >= m->rows || !is_finite(m->cvalues[k])) return 0;
    }
    return 1;
}

/* Four interleaved accumulators combined as (a0+a1)+(a2+a3), the reduction
 * order of multiplyRange / transposeMultiplyRange (sparse_matrix.cpp:276-341)
 * and of every fused pass in the engine. */
static double sparse_dot(const int64_t* start, const int32_t* index, const double* values,
                         int32_t line, const double* v) {
    int64_t k = start[line];
    const int64_t last = start[line + 1];
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    for (; k + 4 <= last; k += 4) {
        a0 += values[k] * v[index[k]];
        a1 += values[k + 1] * v[index[k + 1]];
        a2 += values[k + 2] * v[index[k + 2]];
        a3 += values[k + 3] * v[index[k + 3]];
    }
    for (; k < last; ++k) a0 += values[k] * v[index[k]];
    return (a0 + a1) + (a2 + a3);
}

static void matrix_multiply(const Matrix* m, const double* x, double* out) {
    for (int32_t i = 0; i < m->rows; ++i)
        out[i] = sparse_dot(m->row_start, m->col_index, m->values, i, x);
}

static void matrix_transpose_multiply(const Matrix* m, const double* y, double* out) {
    for (int32_t j = 0; j < m->cols; ++j)
        out[j] = sparse_dot(m->col_start, m->row_index, m->cvalues, j, y);
}

/* ------------------------------------------------------------------ */
/* The LP                                                               */
/* compiled_lp.h:17-63                                                  */
/* ------------------------------------------------------------------ */

typedef struct Lp {
    Matrix a;
    double* c;
    double offset;
    double* rl;
    double* ru;
    double* xl;
    double* xu;
} Lp;

static void lp_free(Lp* p) {
    matrix_free(&p->a);
    free(p->c); free(p->rl); free(p->ru); free(p->xl); free(p->xu);
    memset(p, 0, sizeof(*p));
}

static const char* lp_from_abi(const orc_lp* in, Lp* p) {
    memset(p, 0, sizeof(*p));
    const char* error = matrix_from_lp(in, &p->a);
    if (error) return error;
    p->c = dcopy(in->objective, in->cols);
    p->offset = in->objective_offset;
    p->rl = dcopy(in->row_lower, in->rows);
    p->ru = dcopy(in->row_upper, in->rows);
    p->xl = dcopy(in->var_lower, in->cols);
    p->xu = dcopy(in->var_upper, in->cols);
    return NULL;
}

/* CompiledLp::validate (compiled_lp.h:32-62). Returns NULL or the message. */
static const char* lp_invalid(const Lp* p) {
    if (!matrix_valid(&p->a)) return "CompiledLp contains an invalid sparse matrix";
    if (!is_finite(p->offset)) return "Objective offset must be finite";
    for (int32_t j = 0; j < p->a.cols; ++j) {
        if (!is_finite(p->c[j]) || isnan(p->xl[j]) || isnan(p->xu[j]) || p->xl[j] > p->xu[j])
            return "Invalid objective coefficient or variable bounds";
    }
    for (int32_t i = 0; i < p->a.rows; ++i) {
        if (isnan(p->rl[i]) || isnan(p->ru[i]) || p->rl[i] > p->ru[i]) return "Invalid row bounds";
    }
    return NULL;
}

/* ------------------------------------------------------------------ */
/* Ruiz equilibration (scaling.cpp:14-136)                              */
/* ------------------------------------------------------------------ */

static double scale_bound(double bound, double factor) {   /* scaling.cpp:14-19 */
    return is_finite(bound) ? bound * factor : bound;
}

/* Fills row_scale/col_scale and, when `scaled` is given, the scaled copy of
 * the LP: A-hat = diag(r) A diag(c), c-hat = c*col, bounds as in :109-135. */
static void ruiz(const Lp* p, int iterations, double* row_scale, double* col_scale, Lp* scaled) {
    const Matrix* m = &p->a;
    for (int32_t i = 0; i < m->rows; ++i) row_scale[i] = 1.0;
    for (int32_t j = 0; j < m->cols; ++j) col_scale[j] = 1.0;
    double* row_max = dzeros(m->rows);
    double* col_max = dzeros(m->cols);
    const int passes = iterations > 0 ? iterations : 0;
    for (int pass = 0; pass < passes; ++pass) {
        for (int32_t i = 0; i < m->rows; ++i) row_max[i] = 0.0;
        for (int32_t j = 0; j < m->cols; ++j) col_max[j] = 0.0;
        for (int32_t i = 0; i < m->rows; ++i) {
            const double rf = row_scale[i];
            double local = 0.0;
            for (int64_t k = m->row_start[i]; k < m->row_start[i + 1]; ++k) {
                const int32_t j = m->col_index[k];
                const double mag = fabs(m->values[k]) * rf * col_scale[j];
                local = dmax(local, mag);
                col_max[j] = dmax(col_max[j], mag);
            }
            row_max[i] = local;
        }
        for (int32_t i = 0; i < m->rows; ++i)
            if (row_max[i] > 1e-30) row_scale[i] /= sqrt(row_max[i]);
        for (int32_t j = 0; j < m->cols; ++j)
            if (col_max[j] > 1e-30) col_scale[j] /= sqrt(col_max[j]);
    }
    free(row_max);
    free(col_max);
    if (!scaled) return;

    /* SparseMatrix::scaled (sparse_matrix.cpp:243-274). */
    memset(scaled, 0, sizeof(*scaled));
    Matrix* s = &scaled->a;
    s->rows = m->rows; s->cols = m->cols; s->nnz = m->nnz;
    s->row_start = (int64_t*)xmalloc(((size_t)m->rows + 1) * sizeof(int64_t));
    memcpy(s->row_start, m->row_start, ((size_t)m->rows + 1) * sizeof(int64_t));
    s->col_index = (int32_t*)xmalloc((size_t)(m->nnz ? m->nnz : 1) * sizeof(int32_t));
    if (m->nnz) memcpy(s->col_index, m->col_index, (size_t)m->nnz * sizeof(int32_t));
    s->col_start = (int64_t*)xmalloc(((size_t)m->cols + 1) * sizeof(int64_t));
    memcpy(s->col_start, m->col_start, ((size_t)m->cols + 1) * sizeof(int64_t));
    s->row_index = (int32_t*)xmalloc((size_t)(m->nnz ? m->nnz : 1) * sizeof(int32_t));
    if (m->nnz) memcpy(s->row_index, m->row_index, (size_t)m->nnz * sizeof(int32_t));
    s->values = dcopy(m->values, m->nnz);
    s->cvalues = dcopy(m->cvalues, m->nnz);
    for (int32_t i = 0; i < m->rows; ++i) {
        const double f = row_scale[i];
        for (int64_t k = m->row_start[i]; k < m->row_start[i + 1]; ++k)
            s->values[k] *= f * col_scale[m->col_index[k]];
    }
    for (int32_t j = 0; j < m->cols; ++j) {
        const double f = col_scale[j];
        for (int64_t k = m->col_start[j]; k < m->col_start[j + 1]; ++k)
            s->cvalues[k] *= f * row_scale[m->row_index[k]];
    }
    scaled->offset = p->offset;
    scaled->c = dvec(m->cols);
    scaled->xl = dvec(m->cols);
    scaled->xu = dvec(m->cols);
    for (int32_t j = 0; j < m->cols; ++j) {
        const double f = col_scale[j];
        scaled->c[j] = p->c[j] * f;
        scaled->xl[j] = scale_bound(p->xl[j], 1.0 / f);
        scaled->xu[j] = scale_bound(p->xu[j], 1.0 / f);
    }
    scaled->rl = dvec(m->rows);
    scaled->ru = dvec(m->rows);
    for (int32_t i = 0; i < m->rows; ++i) {
        scaled->rl[i] = scale_bound(p->rl[i], row_scale[i]);
        scaled->ru[i] = scale_bound(p->ru[i], row_scale[i]);
    }
}

/* RuizScaler::conditionSpread (scaling.cpp:138-160). */
static double condition_spread(const Matrix* m) {
    double smallest = ORC_INF, largest = 0.0;
    for (int32_t i = 0; i < m->rows; ++i) {
        double local = 0.0;
        for (int64_t k = m->row_start[i]; k < m->row_start[i + 1]; ++k)
            local = dmax(local, fabs(m->values[k]));
        if (local > 0.0) {
            smallest = dmin(smallest, local);
            largest = dmax(largest, local);
        }
    }
    if (!is_finite(smallest) || smallest <= 0.0) return 1.0;
    return largest / smallest;
}

/* ------------------------------------------------------------------ */
/* Pock-Chambolle preconditioner and power iteration                    */
/* preconditioner.cpp:31-140                                            */
/* ------------------------------------------------------------------ */

typedef struct Precond { double *tau, *tau_inv, *sigma, *sigma_inv; } Precond;

static void precond_free(Precond* d) {
    free(d->tau); free(d->tau_inv); free(d->sigma); free(d->sigma_inv);
}

static void precondition(const Lp* p, int enabled, Precond* d) {
    const Matrix* m = &p->a;
    d->tau = dvec(m->cols); d->tau_inv = dvec(m->cols);
    d->sigma = dvec(m->rows); d->sigma_inv = dvec(m->rows);
    for (int32_t j = 0; j < m->cols; ++j) d->tau[j] = d->tau_inv[j] = 1.0;
    for (int32_t i = 0; i < m->rows; ++i) d->sigma[i] = d->sigma_inv[i] = 1.0;
    if (!enabled) return;
    double* col_sum = dzeros(m->cols);
    double* row_sum = dzeros(m->rows);
    for (int32_t i = 0; i < m->rows; ++i) {
        double acc = 0.0;
        for (int64_t k = m->row_start[i]; k < m->row_start[i + 1]; ++k) {
            const double mag = fabs(m->values[k]);
            acc += mag;
            col_sum[m->col_index[k]] += mag;
        }
        row_sum[i] = acc;
    }
    for (int32_t j = 0; j < m->cols; ++j) {
        const double s = col_sum[j] > 1e-12 ? 1.0 / col_sum[j] : 1.0;
        d->tau[j] = s;
        d->tau_inv[j] = 1.0 / s;
    }
    for (int32_t i = 0; i < m->rows; ++i) {
        const double s = row_sum[i] > 1e-12 ? 1.0 / row_sum[i] : 1.0;
        d->sigma[i] = s;
        d->sigma_inv[i] = 1.0 / s;
    }
    free(col_sum);
    free(row_sum);
}

/* MT19937 (Matsumoto and Nishimura, 1998) and the libstdc++ mapping of two
 * 32-bit draws onto a double in [0, 1), which std::uniform_real_distribution
 * then maps onto [a, b). Used only by the power iteration. */
typedef struct Mt { uint32_t s[624]; int i; } Mt;

static void mt_seed(Mt* g, uint32_t seed) {
    g->s[0] = seed;
    for (int k = 1; k < 624; ++k)
        g->s[k] = 1812433253u * (g->s[k - 1] ^ (g->s[k - 1] >> 30)) + (uint32_t)k;
    g->i = 624;
}

static uint32_t mt_next(Mt* g) {
    if (g->i >= 624) {
        for (int k = 0; k < 624; ++k) {
            const uint32_t y = (g->s[k] & 0x80000000u) | (g->s[(k + 1) % 624] & 0x7fffffffu);
            g->s[k] = g->s[(k + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        g->i = 0;
    }
    uint32_t y = g->s[g->i++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

static double mt_uniform(Mt* g, double a, double b) {
    double sum = 0.0, scale = 1.0;
    for (int k = 0; k < 2; ++k) {
        sum += (double)mt_next(g) * scale;
        scale *= 4294967296.0;
    }
    double r = sum / scale;
    if (r >= 1.0) r = nextafter(1.0, 0.0);
    return r * (b - a) + a;
}

static double normalize_in_place(double* v, int64_t n) {   /* preconditioner.cpp:14-27 */
    double sq = 0.0;
    for (int64_t k = 0; k < n; ++k) sq += v[k] * v[k];
    const double norm = sqrt(sq);
    if (norm > 0.0) {
        const double inv = 1.0 / norm;
        for (int64_t k = 0; k < n; ++k) v[k] *= inv;
    }
    return norm;
}

static double spectral_norm(const Matrix* m, int iterations, int* converged) {
    if (converged) *converged = 1;
    if (m->rows == 0 || m->cols == 0 || m->nnz == 0) return 0.0;
    Mt g;
    mt_seed(&g, 1u);
    double* x = dvec(m->cols);
    double* y = dvec(m->rows);
    double* z = dvec(m->cols);
    for (int32_t j = 0; j < m->cols; ++j) x[j] = mt_uniform(&g, -1.0, 1.0);
    if (normalize_in_place(x, m->cols) == 0.0) {
        for (int32_t j = 0; j < m->cols; ++j) x[j] = 1.0 / sqrt((double)m->cols);
    }
    const int budget = iterations > 1 ? iterations : 1;
    double previous = 0.0, estimate = 0.0;
    int reached = 0;
    for (int it = 0; it < budget; ++it) {
        matrix_multiply(m, x, y);
        matrix_transpose_multiply(m, y, z);
        double rayleigh = 0.0;
        for (int32_t j = 0; j < m->cols; ++j) rayleigh += x[j] * z[j];
        estimate = sqrt(dmax(rayleigh, 0.0));
        if (normalize_in_place(z, m->cols) == 0.0) {
            free(x); free(y); free(z);
            return estimate;
        }
        double* t = x; x = z; z = t;
        if (it > 0 && estimate > 0.0 && fabs(estimate - previous) <= 1e-8 * estimate) {
            reached = 1;
            break;
        }
        previous = estimate;
    }
    if (converged) *converged = reached;
    free(x); free(y); free(z);
    return estimate;
}

/* ------------------------------------------------------------------ */
/* Fused PDHG trial (pdhg_kernel.cpp:47-187, serial path of :189-277)    */
/* ------------------------------------------------------------------ */

typedef struct Trial { double primal, dual, interaction; int finite; } Trial;

static Trial pdhg_trial(const Lp* w, const Precond* d, const double* x, const double* y,
                        const double* ax, double step, double weight,
                        double* x_out, double* y_out, double* ax_out) {
    const Matrix* m = &w->a;
    Trial t = {0.0, 0.0, 0.0, 1};
    /* primalHalf over the columns (:47-104) */
    const double pm = step / weight;
    double moved = 0.0;
    for (int32_t j = 0; j < m->cols; ++j) {
        const double gradient = w->c[j] + sparse_dot(m->col_start, m->row_index, m->cvalues, j, y);
        const double prev = x[j];
        const double upd = clip(prev - pm * d->tau[j] * gradient, w->xl[j], w->xu[j]);
        const double delta = upd - prev;
        x_out[j] = upd;
        moved += delta * delta * d->tau_inv[j];
    }
    t.primal = moved;
    /* dualHalf over the rows (:109-187) */
    const double dm = step * weight;
    double dmoved = 0.0, product = 0.0;
    for (int32_t i = 0; i < m->rows; ++i) {
        const double next = sparse_dot(m->row_start, m->col_index, m->values, i, x_out);
        const double dact = next - ax[i];
        const double ext = next + dact;
        const double s = dmax(dm * d->sigma[i], 1e-300);
        const double prev = y[i];
        const double v = prev + s * ext;
        const double upd = dmax(v - s * w->ru[i], 0.0) + dmin(v - s * w->rl[i], 0.0);
        const double delta = upd - prev;
        y_out[i] = upd;
        ax_out[i] = next;
        dmoved += delta * delta * d->sigma_inv[i];
        product += delta * dact;
    }
    t.dual = dmoved;
    t.interaction = product;
    t.finite = is_finite(t.primal) && is_finite(t.dual) && is_finite(t.interaction);
    return t;
}

/* ------------------------------------------------------------------ */
/* Step size and primal weight (step_controller.cpp:17-98)              */
/* ------------------------------------------------------------------ */

typedef struct Steps {
    double eta;        /* globalStep */
    double omega;      /* primalWeight */
    double eta_max;    /* maximumSafeGlobalStep */
    double min_scale, w_min, w_max, smoothing;
} Steps;

static void steps_init(Steps* s, const orc_options* o, double safe) {
    s->eta_max = safe;
    s->eta = clampd(o->initial_step_safety * safe, o->minimum_step_scale * safe, safe);
    s->omega = 1.0;
    s->min_scale = o->minimum_step_scale;
    s->w_min = o->minimum_primal_weight;
    s->w_max = o->maximum_primal_weight;
    s->smoothing = o->primal_weight_smoothing;
}

static void steps_set_weight(Steps* s, double w) {
    if (w > 0.0 && is_finite(w)) s->omega = clampd(w, s->w_min, s->w_max);
}

static int steps_evaluate(Steps* s, double pmove, double dmove, double inter, int64_t iteration) {
    const double movement = s->omega * pmove + dmove / s->omega;
    const double coupling = fabs(inter);
    double limit = ORC_INF;
    if (coupling > 0.0 && movement > 0.0) limit = movement / (2.0 * coupling);
    const double index = (double)iteration + 2.0;
    const double shrink = 1.0 - pow(index, -0.3);
    const double grow = 1.0 + pow(index, -0.6);
    const int accepted = s->eta <= limit;
    double next = dmin(shrink * limit, grow * s->eta);
    next = clampd(next, s->min_scale * s->eta_max, 1e12);
    if (!is_finite(next) || next <= 0.0) next = s->eta;
    s->eta = next;
    return accepted;
}

static void steps_update_weight(Steps* s, double pdist, double ddist) {
    if (pdist <= 1e-16 || ddist <= 1e-16 || !is_finite(pdist) || !is_finite(ddist)) return;
    const double target = clampd(ddist / pdist, 1e-12, 1e12);
    const double sm = clampd(s->smoothing, 0.0, 1.0);
    steps_set_weight(s, exp(sm * log(target) + (1.0 - sm) * log(s->omega)));
}

/* ------------------------------------------------------------------ */
/* Termination (termination.cpp:14-333)                                 */
/* ------------------------------------------------------------------ */

typedef struct Metrics {
    double pobj, dobj, pres, dres, gap, kkt;
    int dual_valid, finite;
} Metrics;

static Metrics metrics_empty(void) {
    Metrics m = {NAN, -ORC_INF, ORC_INF, ORC_INF, ORC_INF, ORC_INF, 0, 0};
    return m;
}

typedef struct Checker { const Lp* p; double pnorm, dnorm; } Checker;

static void checker_init(Checker* k, const Lp* p) {
    k->p = p;
    double sum = 0.0;
    for (int32_t i = 0; i < p->a.rows; ++i) {
        if (is_finite(p->rl[i])) sum += p->rl[i] * p->rl[i];
        if (is_finite(p->ru[i]) && p->ru[i] != p->rl[i]) sum += p->ru[i] * p->ru[i];
    }
    k->pnorm = 1.0 + sqrt(sum);
    double cs = 0.0;
    for (int32_t j = 0; j < p->a.cols; ++j) cs += p->c[j] * p->c[j];
    k->dnorm = 1.0 + sqrt(cs);
}

static Metrics checker_evaluate(const Checker* k, const double* x, const double* y) {
    const Lp* p = k->p;
    const Matrix* m = &p->a;
    Metrics out = metrics_empty();
    /* rowPass (:66-135) */
    double viol = 0.0, support = 0.0, rinf = 0.0;
    for (int32_t i = 0; i < m->rows; ++i) {
        const double act = sparse_dot(m->row_start, m->col_index, m->values, i, x);
        const double lo = p->rl[i], hi = p->ru[i];
        const double excess = act - clip(act, lo, hi);
        viol += excess * excess;
        double proj = y[i];
        if (!is_finite(hi)) proj = dmin(proj, 0.0);
        if (!is_finite(lo)) proj = dmax(proj, 0.0);
        const double drift = y[i] - proj;
        rinf += drift * drift;
        if (proj > 0.0) support += proj * hi;
        else if (proj < 0.0) support += proj * lo;
    }
    /* columnPass (:140-209) */
    double obj = 0.0, inf = 0.0, cinf = 0.0;
    for (int32_t j = 0; j < m->cols; ++j) {
        const double reduced = p->c[j] + sparse_dot(m->col_start, m->row_index, m->cvalues, j, y);
        const double lo = p->xl[j], hi = p->xu[j];
        obj += p->c[j] * x[j];
        double proj = reduced;
        if (!is_finite(lo)) proj = dmin(proj, 0.0);
        if (!is_finite(hi)) proj = dmax(proj, 0.0);
        const double drift = reduced - proj;
        cinf += drift * drift;
        if (proj > 0.0) inf += proj * lo;
        else if (proj < 0.0) inf += proj * hi;
    }
    /* evaluate (:296-324) */
    out.pres = sqrt(viol) / k->pnorm;
    out.dres = sqrt(cinf + rinf) / k->dnorm;
    out.pobj = p->offset + obj;
    out.dobj = p->offset + inf - support;
    out.finite = is_finite(out.pobj) && is_finite(out.dobj) && is_finite(out.pres) && is_finite(out.dres);
    if (!out.finite) {
        out.dual_valid = 0;
        out.kkt = ORC_INF;
        return out;
    }
    out.dual_valid = 1;
    out.gap = fabs(out.pobj - out.dobj) / (1.0 + fabs(out.pobj) + fabs(out.dobj));
    out.kkt = dmax(dmax(out.pres, out.dres), out.gap);
    return out;
}

static int checker_optimal(const Metrics* m, const orc_options* o) {   /* :327-333 */
    return m->finite && m->dual_valid && m->pres <= o->primal_tolerance &&
           m->dres <= o->dual_tolerance && m->gap <= o->gap_tolerance;
}

/* ------------------------------------------------------------------ */
/* Infeasibility certificates (infeasibility.cpp:40-192)                */
/* ------------------------------------------------------------------ */

typedef struct Verdict { int proves; double value, rel; } Verdict;

static int normalize_into(const double* src, int64_t n, double* dst) {   /* :17-33 */
    double sq = 0.0;
    for (int64_t k = 0; k < n; ++k) sq += src[k] * src[k];
    const double norm = sqrt(sq);
    if (!(norm > 1e-300) || !is_finite(norm)) return 0;
    const double inv = 1.0 / norm;
    for (int64_t k = 0; k < n; ++k) dst[k] = src[k] * inv;
    return 1;
}

static Verdict test_dual_ray(const Lp* p, double tol, const double* dir) {
    const Matrix* m = &p->a;
    Verdict v = {0, 0.0, 1.0};
    double* nd = dvec(m->rows);
    if (!normalize_into(dir, m->rows, nd)) {
        free(nd);
        return v;
    }
    double* aty = dvec(m->cols);
    matrix_transpose_multiply(m, nd, aty);
    double box = 0.0, viol = 0.0;
    for (int32_t j = 0; j < m->cols; ++j) {
        const double r = aty[j];
        double proj = r;
        if (!is_finite(p->xl[j])) proj = dmin(proj, 0.0);
        if (!is_finite(p->xu[j])) proj = dmax(proj, 0.0);
        const double drift = r - proj;
        viol += drift * drift;
        if (proj > 0.0) box += proj * p->xl[j];
        else if (proj < 0.0) box += proj * p->xu[j];
    }
    double support = 0.0;
    for (int32_t i = 0; i < m->rows; ++i) {
        const double val = nd[i];
        double proj = val;
        if (!is_finite(p->ru[i])) proj = dmin(proj, 0.0);
        if (!is_finite(p->rl[i])) proj = dmax(proj, 0.0);
        const double drift = val - proj;
        viol += drift * drift;
        if (proj > 0.0) support += proj * p->ru[i];
        else if (proj < 0.0) support += proj * p->rl[i];
    }
    free(aty);
    free(nd);
    v.value = box - support;
    if (!is_finite(v.value)) return v;
    const double violation = sqrt(viol);
    if (v.value > 0.0) {
        v.rel = violation / v.value;
        v.proves = v.rel <= tol;
    }
    return v;
}

static Verdict test_primal_ray(const Lp* p, double tol, const double* dir) {
    const Matrix* m = &p->a;
    Verdict v = {0, 0.0, 1.0};
    double* nd = dvec(m->cols);
    if (!normalize_into(dir, m->cols, nd)) {
        free(nd);
        return v;
    }
    double* proj = dvec(m->cols);
    double viol = 0.0, rate = 0.0;
    for (int32_t j = 0; j < m->cols; ++j) {
        const double val = nd[j];
        double q = val;
        if (is_finite(p->xu[j])) q = dmin(q, 0.0);
        if (is_finite(p->xl[j])) q = dmax(q, 0.0);
        const double drift = val - q;
        viol += drift * drift;
        proj[j] = q;
        rate += p->c[j] * q;
    }
    double* act = dvec(m->rows);
    matrix_multiply(m, proj, act);
    for (int32_t i = 0; i < m->rows; ++i) {
        const double a = act[i];
        double q = a;
        if (is_finite(p->ru[i])) q = dmin(q, 0.0);
        if (is_finite(p->rl[i])) q = dmax(q, 0.0);
        const double drift = a - q;
        viol += drift * drift;
    }
    free(act);
    free(proj);
    free(nd);
    v.value = rate;
    if (!is_finite(rate)) return v;
    const double violation = sqrt(viol);
    if (rate < 0.0) {
        v.rel = violation / (-rate);
        v.proves = v.rel <= tol;
    }
    return v;
}

/* ------------------------------------------------------------------ */
/* Iterate average (iterate_average.cpp:40-95)                          */
/* ------------------------------------------------------------------ */

typedef struct Average { double *x, *y; double total; int32_t n, m; } Average;

static void average_add(Average* a, const double* x, const double* y, double w) {
    if (!(w > 0.0)) return;
    const double total = a->total + w;
    const double f = w / total;
    for (int32_t j = 0; j < a->n; ++j) a->x[j] += f * (x[j] - a->x[j]);
    for (int32_t i = 0; i < a->m; ++i) a->y[i] += f * (y[i] - a->y[i]);
    a->total = total;
}

static void average_reset(Average* a) {
    for (int32_t j = 0; j < a->n; ++j) a->x[j] = 0.0;
    for (int32_t i = 0; i < a->m; ++i) a->y[i] = 0.0;
    a->total = 0.0;
}

/* ------------------------------------------------------------------ */
/* Restart policy (restart_controller.cpp:8-63)                         */
/* ------------------------------------------------------------------ */

enum { CHOICE_NONE = 0, CHOICE_CURRENT = 1, CHOICE_AVERAGE = 2 };

static int restart_choose(const orc_options* o, double* previous_score, const Metrics* cur,
                          const Metrics* avg, double baseline, int64_t since, int64_t total,
                          double* candidate_score) {
    *candidate_score = ORC_INF;
    if (!o->use_restarts || since < o->minimum_restart_iterations) return CHOICE_NONE;
    const int af = is_finite(avg->kkt), cf = is_finite(cur->kkt);
    if (!af && !cf) return CHOICE_NONE;
    int cand = CHOICE_AVERAGE;
    double score = avg->kkt;
    if (!af || (cf && cur->kkt < avg->kkt)) {
        cand = CHOICE_CURRENT;
        score = cur->kkt;
    }
    *candidate_score = score;
    const double prev = *previous_score;
    *previous_score = score;
    const int bf = is_finite(baseline);
    if (bf && score <= o->restart_sufficient_decay * baseline) return cand;
    if (bf && score <= o->restart_necessary_decay * baseline && is_finite(prev) && score > prev)
        return cand;
    int64_t art = (int64_t)(o->restart_artificial_fraction * (double)total);
    if (art < 1) art = 1;
    if (since >= art || since >= o->maximum_restart_iterations) return cand;
    return CHOICE_NONE;
}

/* ------------------------------------------------------------------ */
/* Solver (pdlp_solver.cpp:116-548, feasibility_polishing.cpp:13-145)   */
/* ------------------------------------------------------------------ */

static double initial_value(double lo, double hi) {   /* pdlp_solver.cpp:30-41 */
    if (lo <= 0.0 && 0.0 <= hi) return 0.0;
    if (is_finite(lo)) return lo;
    if (is_finite(hi)) return hi;
    return 0.0;
}

typedef struct Solve {
    const orc_options* o;
    const Lp* orig;
    const Lp* work;
    int scaled;
    const double* rs;
    const double* cs;
    Checker checker;
    double* ox;   /* original-coordinate scratch of the last score */
    double* oy;
} Solve;

/* The `score` lambda (pdlp_solver.cpp:226-237): map to original coordinates
 * when scaled and evaluate there. Leaves the scored point in ox/oy, or points
 * at the inputs when unscaled. */
static Metrics score_point(Solve* s, const double* x, const double* y,
                           const double** sx, const double** sy) {
    if (s->scaled) {
        for (int32_t j = 0; j < s->orig->a.cols; ++j) s->ox[j] = s->cs[j] * x[j];
        for (int32_t i = 0; i < s->orig->a.rows; ++i) s->oy[i] = s->rs[i] * y[i];
        *sx = s->ox;
        *sy = s->oy;
    } else {
        *sx = x;
        *sy = y;
    }
    return checker_evaluate(&s->checker, *sx, *sy);
}

static void fill_result(orc_result* out, int status, const char* msg, const Metrics* m,
                        int64_t iterations, int64_t trials, int restarts, double t0) {
    out->status = status;
    snprintf(out->message, sizeof(out->message), "%s", msg);
    out->primal_objective = m->pobj;
    out->dual_objective = m->dobj;
    out->primal_residual = m->pres;
    out->dual_residual = m->dres;
    out->relative_gap = m->gap;
    out->iterations = iterations;
    out->step_trials = trials;
    out->restart_count = restarts;
    out->solve_time_seconds = now_seconds() - t0;
}

enum {
    ST_OPTIMAL = 0, ST_INFEASIBLE, ST_UNBOUNDED, ST_ITERATION_LIMIT, ST_TIME_LIMIT,
    ST_NUMERICAL_FAILURE, ST_INVALID_PROBLEM
};

void orc_default_options(orc_options* o) {   /* pdlp_options.h:7-75 */
    memset(o, 0, sizeof(*o));
    o->iteration_limit = 200000;
    o->time_limit_seconds = 0.0;
    o->primal_tolerance = 1e-6;
    o->dual_tolerance = 1e-6;
    o->gap_tolerance = 1e-6;
    o->termination_check_frequency = 100;
    o->power_iteration_count = 100;
    o->thread_count = 0;
    o->parallel_nonzero_threshold = 20000;
    o->initial_step_safety = 0.90;
    o->minimum_step_scale = 1e-6;
    o->maximum_primal_weight = 1e6;
    o->minimum_primal_weight = 1e-6;
    o->use_ruiz_scaling = 1;
    o->ruiz_iterations = 10;
    o->detect_infeasibility = 1;
    o->infeasibility_tolerance = 1e-8;
    o->use_diagonal_preconditioning = 1;
    o->use_adaptive_linesearch = 1;
    o->maximum_step_trials = 60;
    o->use_averaging = 1;
    o->use_restarts = 1;
    o->use_feasibility_polishing = 1;
    o->minimum_restart_iterations = 64;
    o->maximum_restart_iterations = 100000;
    o->restart_sufficient_decay = 0.20;
    o->restart_necessary_decay = 0.80;
    o->restart_artificial_fraction = 0.36;
    o->initial_primal_weight = 1.0;
    o->primal_weight_smoothing = 0.50;
    o->polishing_iterations = 5000;
}

/* FeasibilityPolisher::polish (feasibility_polishing.cpp:13-145). Updates
 * best/best_metrics in place when it finds a better point; returns the
 * iterations and trials it spent through the out-parameters. */
static void polish(Solve* s, const Precond* d, const Steps* in_steps, double* best_x,
                   double* best_y, Metrics* best_m, double remaining, int* iters_out,
                   int64_t* trials_out) {
    const orc_options* o = s->o;
    const Lp* w = s->work;
    const int32_t n = w->a.cols, m = w->a.rows;
    *iters_out = 0;
    *trials_out = 0;
    if (!o->use_feasibility_polishing || o->polishing_iterations <= 0) return;

    double* x = dvec(n);
    double* y = dvec(m);
    if (s->scaled) {   /* toScaled (scaling.cpp:39-53) */
        for (int32_t j = 0; j < n; ++j) x[j] = best_x[j] / s->cs[j];
        for (int32_t i = 0; i < m; ++i) y[i] = best_y[i] / s->rs[i];
    } else {
        memcpy(x, best_x, (size_t)n * sizeof(double));
        memcpy(y, best_y, (size_t)m * sizeof(double));
    }
    double* ax = dvec(m);
    matrix_multiply(&w->a, x, ax);
    double* tx = dvec(n);
    double* ty = dvec(m);
    double* tax = dvec(m);

    /* The polisher steps with its own copy of the parameters at half the step;
     * its controller starts from the static bound and shares only omega. */
    double step = in_steps->eta * 0.5;
    const double weight = in_steps->omega;
    Steps ctl;
    steps_init(&ctl, o, in_steps->eta_max);
    steps_set_weight(&ctl, in_steps->omega);
    Average avg = {dzeros(n), dzeros(m), 0.0, n, m};
    int64_t iteration = 0;   /* the polisher's own state.iteration */
    const double t0 = now_seconds();
    const int freq = o->termination_check_frequency > 1 ? o->termination_check_frequency : 1;
    const int max_trials = o->maximum_step_trials > 1 ? o->maximum_step_trials : 1;

    for (int it = 0; it < o->polishing_iterations; ++it) {
        int committed = 0, broken = 0;
        for (int attempt = 0; attempt < max_trials; ++attempt) {
            const Trial t = pdhg_trial(w, d, x, y, ax, step, weight, tx, ty, tax);
            ++*trials_out;
            if (!t.finite) {
                broken = 1;
                break;
            }
            if (!o->use_adaptive_linesearch) {
                committed = 1;
            } else {
                const int ok = steps_evaluate(&ctl, t.primal, t.dual, t.interaction, iteration);
                step = ctl.eta;
                committed = ok;
            }
            if (committed) {
                double* q;
                q = x; x = tx; tx = q;
                q = y; y = ty; ty = q;
                q = ax; ax = tax; tax = q;
                ++iteration;
                break;
            }
        }
        if (broken || !committed) break;
        if (o->use_averaging) average_add(&avg, x, y, step);
        ++*iters_out;
        const int last = it + 1 == o->polishing_iterations;
        if ((it + 1) % freq != 0 && !last) continue;
        if (remaining > 0.0 && now_seconds() - t0 >= remaining) break;
        const double *sx, *sy;
        Metrics cm = score_point(s, x, y, &sx, &sy);
        if (cm.kkt < best_m->kkt) {
            memcpy(best_x, sx, (size_t)n * sizeof(double));
            memcpy(best_y, sy, (size_t)m * sizeof(double));
            *best_m = cm;
        }
        if (o->use_averaging && avg.total != 0.0) {
            Metrics am = score_point(s, avg.x, avg.y, &sx, &sy);
            if (am.kkt < best_m->kkt) {
                memcpy(best_x, sx, (size_t)n * sizeof(double));
                memcpy(best_y, sy, (size_t)m * sizeof(double));
                *best_m = am;
            }
        }
        if (checker_optimal(best_m, o)) break;
    }
    free(x); free(y); free(ax); free(tx); free(ty); free(tax);
    free(avg.x); free(avg.y);
}

int orc_solve(const orc_lp* in, const orc_options* o, double* primal_out, double* dual_out,
              double* dual_ray_out, double* primal_ray_out, orc_result* out) {
    const double t0 = now_seconds();
    memset(out, 0, sizeof(*out));
    Metrics none = metrics_empty();

    Lp orig;
    const char* bad = lp_from_abi(in, &orig);
    if (!bad) bad = lp_invalid(&orig);
    if (bad) {
        fill_result(out, ST_INVALID_PROBLEM, bad, &none, 0, 0, 0, t0);
        out->final_primal_weight = 1.0;
        lp_free(&orig);
        return out->status;
    }
    if (o->iteration_limit < 0 || o->termination_check_frequency <= 0 ||
        o->primal_tolerance < 0.0 || o->dual_tolerance < 0.0 || o->gap_tolerance < 0.0 ||
        o->initial_step_safety <= 0.0 || o->minimum_primal_weight <= 0.0 ||
        o->maximum_primal_weight < o->minimum_primal_weight) {
        fill_result(out, ST_INVALID_PROBLEM, "Invalid PDLP options", &none, 0, 0, 0, t0);
        out->final_primal_weight = 1.0;
        lp_free(&orig);
        return out->status;
    }
    const int32_t n = orig.a.cols, m = orig.a.rows;

    /* Equilibrate (pdlp_solver.cpp:160-166). */
    Lp scaled_lp;
    memset(&scaled_lp, 0, sizeof(scaled_lp));
    double* rs = NULL;
    double* cs = NULL;
    const int scaled = o->use_ruiz_scaling && o->ruiz_iterations > 0 && orig.a.nnz > 0;
    if (scaled) {
        rs = dvec(m);
        cs = dvec(n);
        ruiz(&orig, o->ruiz_iterations, rs, cs, &scaled_lp);
    }
    const Lp* w = scaled ? &scaled_lp : &orig;

    double* x = dvec(n);
    double* y = dzeros(m);
    for (int32_t j = 0; j < n; ++j) x[j] = initial_value(w->xl[j], w->xu[j]);

    Precond d;
    precondition(w, o->use_diagonal_preconditioning, &d);
    double safe = 0.99;
    if (!o->use_diagonal_preconditioning) {   /* :189-202 */
        int conv = 0;
        const double norm = spectral_norm(&w->a, o->power_iteration_count, &conv);
        safe = norm > 0.0 ? 0.99 / (norm * (conv ? 1.02 : 1.25)) : 1.0;
    }
    Steps st;
    steps_init(&st, o, safe);
    steps_set_weight(&st, o->initial_primal_weight);

    double* ax = dvec(m);
    matrix_multiply(&w->a, x, ax);
    double* tx = dvec(n);
    double* ty = dvec(m);
    double* tax = dvec(m);
    Average avg = {dzeros(n), dzeros(m), 0.0, n, m};

    Solve s;
    s.o = o; s.orig = &orig; s.work = w; s.scaled = scaled; s.rs = rs; s.cs = cs;
    checker_init(&s.checker, &orig);
    s.ox = dvec(n);
    s.oy = dvec(m);

    const double *sx, *sy;
    Metrics cur = score_point(&s, x, y, &sx, &sy);
    double* best_x = dcopy(sx, n);
    double* best_y = dcopy(sy, m);
    Metrics best = cur;
    double baseline = cur.kkt;
    int64_t since = 0;
    int restarts = 0;
    double prev_candidate = ORC_INF;
    double* rx = dcopy(x, n);
    double* ry = dcopy(y, m);
    int64_t trials = 0;
    int64_t iteration = 0;
    double* pdir = dvec(n);
    double* ddir = dvec(m);
    double* col_ray = dvec(n);
    double* row_ray = dvec(m);
    int status = -1;
    const char* message = "";
    int ray_kind = 0;   /* 1 dual ray, 2 primal ray */

    if (checker_optimal(&cur, o)) {
        fill_result(out, ST_OPTIMAL, "Initial point satisfies the requested tolerances", &cur, 0,
                    0, 0, t0);
        out->final_primal_weight = 1.0;
        status = ST_OPTIMAL;
        goto finish_no_diag;
    }

    int limit_status = ST_ITERATION_LIMIT;
    const char* limit_message = "Iteration limit reached";
    const int max_trials = o->maximum_step_trials > 1 ? o->maximum_step_trials : 1;

    for (int64_t loop = 0; loop < o->iteration_limit; ++loop) {
        if (o->time_limit_seconds > 0.0 && now_seconds() - t0 >= o->time_limit_seconds) {
            limit_status = ST_TIME_LIMIT;
            limit_message = "Time limit reached";
            break;
        }
        int committed = 0;
        for (int attempt = 0; attempt < max_trials; ++attempt) {
            const Trial t = pdhg_trial(w, &d, x, y, ax, st.eta, st.omega, tx, ty, tax);
            ++trials;
            if (!t.finite) {
                status = ST_NUMERICAL_FAILURE;
                message = "PDHG generated a non-finite iterate";
                goto finish;
            }
            const int accept = !o->use_adaptive_linesearch ||
                               steps_evaluate(&st, t.primal, t.dual, t.interaction, iteration);
            if (accept) {
                double* q;
                q = x; x = tx; tx = q;
                q = y; y = ty; ty = q;
                q = ax; ax = tax; tax = q;
                ++iteration;
                committed = 1;
                break;
            }
        }
        if (!committed) {
            status = ST_NUMERICAL_FAILURE;
            message = "Adaptive linesearch failed to accept a step";
            goto finish;
        }
        ++since;
        if (o->use_averaging) average_add(&avg, x, y, st.eta);
        if (iteration % o->termination_check_frequency != 0) continue;

        cur = score_point(&s, x, y, &sx, &sy);
        if (cur.kkt < best.kkt) {
            memcpy(best_x, sx, (size_t)n * sizeof(double));
            memcpy(best_y, sy, (size_t)m * sizeof(double));
            best = cur;
        }
        Metrics am = cur;
        const int have_avg = o->use_averaging && avg.total != 0.0;
        if (have_avg) {
            am = score_point(&s, avg.x, avg.y, &sx, &sy);
            if (am.kkt < best.kkt) {
                memcpy(best_x, sx, (size_t)n * sizeof(double));
                memcpy(best_y, sy, (size_t)m * sizeof(double));
                best = am;
            }
        }
        if (o->detect_infeasibility) {   /* :377-422 */
            for (int32_t j = 0; j < n; ++j) pdir[j] = x[j] - rx[j];
            for (int32_t i = 0; i < m; ++i) ddir[i] = y[i] - ry[i];
            for (int32_t j = 0; j < n; ++j) col_ray[j] = scaled ? cs[j] * pdir[j] : pdir[j];
            for (int32_t i = 0; i < m; ++i) row_ray[i] = scaled ? rs[i] * ddir[i] : ddir[i];
            const Verdict dv = test_dual_ray(&orig, o->infeasibility_tolerance, row_ray);
            if (dv.proves) {
                status = ST_INFEASIBLE;
                message = "Primal infeasible: Farkas ray found";
                ray_kind = 1;
                goto finish;
            }
            const Verdict pv = test_primal_ray(&orig, o->infeasibility_tolerance, col_ray);
            if (pv.proves) {
                status = ST_UNBOUNDED;
                message = "Unbounded: improving ray found";
                ray_kind = 2;
                goto finish;
            }
        }
        if (checker_optimal(&best, o)) {
            status = ST_OPTIMAL;
            message = "Primal, dual, and gap tolerances satisfied";
            goto finish;
        }
        double cand_score;
        const int choice = restart_choose(o, &prev_candidate, &cur, &am, baseline, since,
                                          iteration, &cand_score);
        if (choice != CHOICE_NONE) {   /* :444-476 */
            const int from_avg = choice == CHOICE_AVERAGE && have_avg;
            const double* sel_x = from_avg ? avg.x : x;
            const double* sel_y = from_avg ? avg.y : y;
            double pd = 0.0, dd = 0.0;
            for (int32_t j = 0; j < n; ++j) { const double t = sel_x[j] - rx[j]; pd += t * t; }
            for (int32_t i = 0; i < m; ++i) { const double t = sel_y[i] - ry[i]; dd += t * t; }
            steps_update_weight(&st, sqrt(pd), sqrt(dd));
            if (from_avg) {
                memcpy(x, avg.x, (size_t)n * sizeof(double));
                memcpy(y, avg.y, (size_t)m * sizeof(double));
                matrix_multiply(&w->a, x, ax);
            }
            memcpy(rx, x, (size_t)n * sizeof(double));
            memcpy(ry, y, (size_t)m * sizeof(double));
            baseline = cand_score;
            average_reset(&avg);
            prev_candidate = ORC_INF;
            since = 0;
            ++restarts;
        }
    }

    {   /* Loop exhausted: polishing, then the limit status (:479-547). */
        int64_t total_iterations = iteration;
        int64_t total_trials = trials;
        status = limit_status;
        message = limit_message;
        if (o->use_feasibility_polishing && n > 0) {
            double remaining = 0.0;
            int go = 1;
            if (o->time_limit_seconds > 0.0) {
                remaining = o->time_limit_seconds - (now_seconds() - t0);
                if (remaining <= 0.0) go = 0;
            }
            if (go) {
                int pit = 0;
                int64_t ptr = 0;
                polish(&s, &d, &st, best_x, best_y, &best, remaining, &pit, &ptr);
                if (checker_optimal(&best, o)) {
                    status = ST_OPTIMAL;
                    message = "Tolerances satisfied after refinement polishing";
                    total_iterations += pit;
                    total_trials += ptr;
                }
            }
        }
        fill_result(out, status, message, &best, total_iterations, total_trials, restarts, t0);
        goto diagnostics;
    }

finish:
    fill_result(out, status, message, &best, iteration, trials, restarts, t0);
diagnostics:
    out->final_step_size = st.eta;
    out->static_step_bound = st.eta_max;
    out->final_primal_weight = st.omega;
finish_no_diag:
    out->primal_size = n;
    out->dual_size = m;
    if (primal_out) memcpy(primal_out, best_x, (size_t)n * sizeof(double));
    if (dual_out) memcpy(dual_out, best_y, (size_t)m * sizeof(double));
    if (ray_kind == 1) {
        out->has_dual_ray = 1;
        if (dual_ray_out) memcpy(dual_ray_out, row_ray, (size_t)m * sizeof(double));
    } else if (ray_kind == 2) {
        out->has_primal_ray = 1;
        if (primal_ray_out) memcpy(primal_ray_out, col_ray, (size_t)n * sizeof(double));
    }

    free(x); free(y); free(ax); free(tx); free(ty); free(tax);
    free(avg.x); free(avg.y); free(s.ox); free(s.oy);
    free(best_x); free(best_y); free(rx); free(ry);
    free(pdir); free(ddir); free(col_ray); free(row_ray);
    precond_free(&d);
    free(rs); free(cs);
    if (scaled) lp_free(&scaled_lp);
    lp_free(&orig);
    return out->status;
}

/* ------------------------------------------------------------------ */
/* Component entry points (oracle_abi.h)                                */
/* ------------------------------------------------------------------ */

int orc_from_triplets(int32_t rows, int32_t cols, int64_t count, const int32_t* row,
                      const int32_t* col, const double* value, int64_t* row_start,
                      int32_t* col_index, double* values, int64_t* col_start,
                      int32_t* row_index, double* csc_values, int64_t* nnz_out) {
    Matrix mtx;
    if (matrix_from_triplets(rows, cols, count, row, col, value, &mtx) != 0) return -1;
    memcpy(row_start, mtx.row_start, ((size_t)rows + 1) * sizeof(int64_t));
    memcpy(col_start, mtx.col_start, ((size_t)cols + 1) * sizeof(int64_t));
    if (mtx.nnz) {
        memcpy(col_index, mtx.col_index, (size_t)mtx.nnz * sizeof(int32_t));
        memcpy(values, mtx.values, (size_t)mtx.nnz * sizeof(double));
        memcpy(row_index, mtx.row_index, (size_t)mtx.nnz * sizeof(int32_t));
        memcpy(csc_values, mtx.cvalues, (size_t)mtx.nnz * sizeof(double));
    }
    *nnz_out = mtx.nnz;
    matrix_free(&mtx);
    return 0;
}

void orc_multiply(const orc_lp* lp, const double* x, double* ax) {
    Matrix mtx;
    matrix_from_lp(lp, &mtx);
    matrix_multiply(&mtx, x, ax);
    matrix_free(&mtx);
}

void orc_transpose_multiply(const orc_lp* lp, const double* y, double* aty) {
    Matrix mtx;
    matrix_from_lp(lp, &mtx);
    matrix_transpose_multiply(&mtx, y, aty);
    matrix_free(&mtx);
}

void orc_ruiz(const orc_lp* lp, int32_t iterations, double* row_scale, double* col_scale,
              double* scaled_values, double* scaled_objective, double* scaled_row_lower,
              double* scaled_row_upper, double* scaled_var_lower, double* scaled_var_upper) {
    Lp p, s;
    lp_from_abi(lp, &p);
    double* r = dvec(lp->rows);
    double* c = dvec(lp->cols);
    ruiz(&p, iterations, r, c, &s);
    if (row_scale) memcpy(row_scale, r, (size_t)lp->rows * sizeof(double));
    if (col_scale) memcpy(col_scale, c, (size_t)lp->cols * sizeof(double));
    if (scaled_values && lp->nnz) memcpy(scaled_values, s.a.values, (size_t)lp->nnz * sizeof(double));
    if (scaled_objective) memcpy(scaled_objective, s.c, (size_t)lp->cols * sizeof(double));
    if (scaled_row_lower) memcpy(scaled_row_lower, s.rl, (size_t)lp->rows * sizeof(double));
    if (scaled_row_upper) memcpy(scaled_row_upper, s.ru, (size_t)lp->rows * sizeof(double));
    if (scaled_var_lower) memcpy(scaled_var_lower, s.xl, (size_t)lp->cols * sizeof(double));
    if (scaled_var_upper) memcpy(scaled_var_upper, s.xu, (size_t)lp->cols * sizeof(double));
    free(r);
    free(c);
    lp_free(&s);
    lp_free(&p);
}

double orc_condition_spread(const orc_lp* lp) {
    Matrix mtx;
    matrix_from_lp(lp, &mtx);
    const double v = condition_spread(&mtx);
    matrix_free(&mtx);
    return v;
}

void orc_precondition(const orc_lp* lp, int32_t enabled, double* tau, double* tau_inverse,
                      double* sigma, double* sigma_inverse) {
    Lp p;
    lp_from_abi(lp, &p);
    Precond d;
    precondition(&p, enabled, &d);
    memcpy(tau, d.tau, (size_t)lp->cols * sizeof(double));
    memcpy(tau_inverse, d.tau_inv, (size_t)lp->cols * sizeof(double));
    memcpy(sigma, d.sigma, (size_t)lp->rows * sizeof(double));
    memcpy(sigma_inverse, d.sigma_inv, (size_t)lp->rows * sizeof(double));
    precond_free(&d);
    lp_free(&p);
}

double orc_spectral_norm(const orc_lp* lp, int32_t iterations, int32_t* converged) {
    Matrix mtx;
    matrix_from_lp(lp, &mtx);
    int conv = 0;
    const double v = spectral_norm(&mtx, iterations, &conv);
    if (converged) *converged = conv;
    matrix_free(&mtx);
    return v;
}

int orc_trial(const orc_lp* working, const double* tau, const double* tau_inverse,
              const double* sigma, const double* sigma_inverse, const double* x,
              const double* y, const double* ax, double step, double weight, double* x_out,
              double* y_out, double* ax_out, double* reductions) {
    Lp p;
    lp_from_abi(working, &p);
    Precond d = {(double*)tau, (double*)tau_inverse, (double*)sigma, (double*)sigma_inverse};
    const Trial t = pdhg_trial(&p, &d, x, y, ax, step, weight, x_out, y_out, ax_out);
    reductions[0] = t.primal;
    reductions[1] = t.dual;
    reductions[2] = t.interaction;
    lp_free(&p);
    return t.finite;
}

void orc_evaluate(const orc_lp* lp, const double* x, const double* y, double* metrics) {
    Lp p;
    lp_from_abi(lp, &p);
    Checker k;
    checker_init(&k, &p);
    const Metrics mt = checker_evaluate(&k, x, y);
    metrics[0] = mt.pobj; metrics[1] = mt.dobj; metrics[2] = mt.pres; metrics[3] = mt.dres;
    metrics[4] = mt.gap; metrics[5] = mt.kkt;
    metrics[6] = mt.finite ? 1.0 : 0.0;
    metrics[7] = mt.dual_valid ? 1.0 : 0.0;
    lp_free(&p);
}

void orc_test_dual_ray(const orc_lp* lp, double tolerance, const double* direction,
                       double* verdict) {
    Lp p;
    lp_from_abi(lp, &p);
    const Verdict v = test_dual_ray(&p, tolerance, direction);
    verdict[0] = v.proves; verdict[1] = v.value; verdict[2] = v.rel;
    lp_free(&p);
}

void orc_test_primal_ray(const orc_lp* lp, double tolerance, const double* direction,
                         double* verdict) {
    Lp p;
    lp_from_abi(lp, &p);
    const Verdict v = test_primal_ray(&p, tolerance, direction);
    verdict[0] = v.proves; verdict[1] = v.value; verdict[2] = v.rel;
    lp_free(&p);
}
