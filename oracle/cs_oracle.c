/*
 * TEST ORACLE ONLY -- CPU restatement of the reference's hot-path algorithms
 * (see cs_oracle.h).  Plain C, serial unless a thread count is passed.  Used
 * as the checker by tests/, __graft_entry__.smoke() and the CPU baseline leg
 * of bench.py; libcellshard_b200 never calls it.
 */
#include "cs_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define INVALID_COL 0xffffffffu

/* IEEE binary16 -> binary32, exact. */
float cso_h2f(uint16_t h) {
    const uint32_t sign = (uint32_t) (h & 0x8000u) << 16;
    uint32_t exp = (h >> 10) & 0x1fu;
    uint32_t man = h & 0x3ffu;
    uint32_t bits;
    if (exp == 0u) {
        if (man == 0u) {
            bits = sign;
        } else { /* subnormal: normalise */
            int e = -1;
            do {
                ++e;
                man <<= 1;
            } while ((man & 0x400u) == 0u);
            bits = sign | ((uint32_t) (127 - 15 - e) << 23) | ((man & 0x3ffu) << 13);
        }
    } else if (exp == 31u) {
        bits = sign | 0x7f800000u | (man << 13);
    } else {
        bits = sign | ((exp - 15u + 127u) << 23) | (man << 13);
    }
    float f;
    memcpy(&f, &bits, sizeof(f));
    return f;
}

static int half_nonzero(uint16_t h) { return (h & 0x7fffu) != 0u; }

/* ------------------------------------------------------------------------ */
/* mask_groups per-row reduce: for each participating row, values with        */
/* column < cols, nonzero, feature kept (mask_groups.cu:155,255,338); group   */
/* sums over the bits of each column's mask (:158-163); keep filter and      */
/* percentages (:177-194); masked-out rows are zeroed (:81-105).             */
/* Sums are accumulated in double and rounded once.                          */
/* ------------------------------------------------------------------------ */
typedef struct {
    double sum;
    float vmax;
    uint32_t det;
    double g[32];
} row_state;

static void rs_init(row_state *s) { memset(s, 0, sizeof(*s)); }

static void rs_add(row_state *s, float v, uint32_t gene, const uint32_t *masks, uint32_t G) {
    s->sum += v;
    if (v > s->vmax) s->vmax = v;
    s->det += 1u;
    if (masks != NULL && G != 0u) {
        uint32_t m = masks[gene];
        for (uint32_t g = 0; g < 32u; ++g)
            if (((m >> g) & 1u) && g < G) s->g[g] += v;
    }
}

static void rs_emit(const row_state *s, uint32_t row, uint32_t G, float min_total, uint32_t min_det, float max_frac,
                    uint32_t frac_idx, cso_reduce_out *o) {
    const float total = (float) s->sum;
    o->row_totals[row] = total;
    o->max_values[row] = s->vmax;
    o->detected[row] = s->det;
    const float num = frac_idx < G ? (float) s->g[frac_idx] : 0.0f;
    const float frac = total > 0.0f ? num / total : 0.0f;
    o->row_keep[row] = (uint8_t) (total >= min_total && s->det >= min_det && frac <= max_frac);
    if (o->group_counts != NULL && o->group_percentages != NULL) {
        for (uint32_t g = 0; g < G; ++g) {
            const float gs = (float) s->g[g];
            o->group_counts[(size_t) row * G + g] = gs;
            o->group_percentages[(size_t) row * G + g] = total > 0.0f ? (100.0f * gs) / total : 0.0f;
        }
    }
}

static void rs_empty(uint32_t row, uint32_t G, cso_reduce_out *o) {
    o->row_totals[row] = 0.0f;
    o->max_values[row] = 0.0f;
    o->detected[row] = 0u;
    o->row_keep[row] = 0u;
    if (o->group_counts != NULL && o->group_percentages != NULL) {
        for (uint32_t g = 0; g < G; ++g) {
            o->group_counts[(size_t) row * G + g] = 0.0f;
            o->group_percentages[(size_t) row * G + g] = 0.0f;
        }
    }
}

static int kept_feature(const uint8_t *fk, uint32_t c) { return fk == NULL || fk[c] != 0u; }

int cso_group_reduce_csr(uint32_t rows, uint32_t cols, const uint32_t *ptr, const uint32_t *idx, const uint16_t *val,
                         const uint32_t *masks, uint32_t G, const uint8_t *row_keep, const uint8_t *fk,
                         float min_total, uint32_t min_det, float max_frac, uint32_t frac_idx, cso_reduce_out *o) {
    if (G > 32u) return 0;
    for (uint32_t r = 0; r < rows; ++r) {
        if (row_keep != NULL && row_keep[r] == 0u) {
            rs_empty(r, G, o);
            continue;
        }
        row_state s;
        rs_init(&s);
        for (uint32_t i = ptr[r]; i < ptr[r + 1u]; ++i) {
            const uint32_t c = idx[i];
            if (c < cols && half_nonzero(val[i]) && kept_feature(fk, c)) rs_add(&s, cso_h2f(val[i]), c, masks, G);
        }
        rs_emit(&s, r, G, min_total, min_det, max_frac, frac_idx, o);
    }
    return 1;
}

int cso_group_reduce_bell(uint32_t rows, uint32_t cols, uint32_t B, uint32_t ell_cols, const uint32_t *bci,
                          const uint16_t *val, const uint32_t *masks, uint32_t G, const uint8_t *row_keep,
                          const uint8_t *fk, float min_total, uint32_t min_det, float max_frac, uint32_t frac_idx,
                          cso_reduce_out *o) {
    if (G > 32u) return 0;
    const uint32_t W = B != 0u ? ell_cols / B : 0u;
    for (uint32_t r = 0; r < rows; ++r) {
        if (row_keep != NULL && row_keep[r] == 0u) {
            rs_empty(r, G, o);
            continue;
        }
        row_state s;
        rs_init(&s);
        const uint32_t rb = B != 0u ? r / B : 0u;
        for (uint32_t e = 0; e < ell_cols; ++e) {
            const uint32_t slot = e / B;
            const uint32_t bc = W != 0u ? bci[(size_t) rb * W + slot] : INVALID_COL;
            const uint32_t gene = bc != INVALID_COL ? bc * B + e % B : cols;
            const uint16_t h = val[(size_t) r * ell_cols + e];
            if (gene < cols && half_nonzero(h) && kept_feature(fk, gene)) rs_add(&s, cso_h2f(h), gene, masks, G);
        }
        rs_emit(&s, r, G, min_total, min_det, max_frac, frac_idx, o);
    }
    return 1;
}

int cso_group_reduce_sell(uint32_t rows, uint32_t cols, uint32_t slice_count, uint32_t slice_rows,
                          const uint32_t *offsets, const uint32_t *widths, const uint32_t *slot_offsets,
                          const uint32_t *col_idx, const uint16_t *val, const uint32_t *masks, uint32_t G,
                          const uint8_t *row_keep, const uint8_t *fk, float min_total, uint32_t min_det,
                          float max_frac, uint32_t frac_idx, cso_reduce_out *o) {
    if (G > 32u) return 0;
    for (uint32_t r = 0; r < rows; ++r) {
        if (row_keep != NULL && row_keep[r] == 0u) {
            rs_empty(r, G, o);
            continue;
        }
        row_state s;
        rs_init(&s);
        if (slice_count != 0u) {
            uint32_t slice = 0u;
            if (slice_rows != 0u) {
                slice = r / slice_rows;
                if (slice >= slice_count) slice = slice_count - 1u;
            } else {
                while (slice + 1u < slice_count && r >= offsets[slice + 1u]) ++slice; /* mask_groups.cu:243 */
            }
            const uint32_t w = widths[slice];
            const size_t base = (size_t) slot_offsets[slice] + (size_t) (r - offsets[slice]) * w;
            for (uint32_t k = 0; k < w; ++k) {
                const uint32_t c = col_idx[base + k];
                const uint16_t h = val[base + k];
                if (c < cols && half_nonzero(h) && kept_feature(fk, c)) rs_add(&s, cso_h2f(h), c, masks, G);
            }
        }
        rs_emit(&s, r, G, min_total, min_det, max_frac, frac_idx, o);
    }
    return 1;
}

long long cso_reoptimize_bell(uint32_t rows, uint32_t cols, uint32_t B, uint32_t ell_cols, const uint32_t *bci,
                              const uint16_t *val, const uint8_t *row_keep, const uint8_t *fk,
                              const uint32_t *row_remap, const uint32_t *feature_remap, uint32_t out_rows,
                              uint32_t out_cols, uint32_t *major_ptr, uint32_t *minor_idx, uint16_t *out_val) {
    const uint32_t W = B != 0u ? ell_cols / B : 0u;
    int32_t *src_of = (int32_t *) malloc(((size_t) out_rows + 1u) * sizeof(int32_t));
    if (src_of == NULL) return -2;
    for (uint32_t i = 0; i < out_rows; ++i) src_of[i] = -1;
    for (uint32_t r = 0; r < rows; ++r) {
        if (row_keep != NULL && row_keep[r] == 0u) continue;
        const uint32_t orow = row_remap != NULL ? row_remap[r] : r;
        if (orow >= out_rows) continue;
        if (src_of[orow] >= 0) {
            free(src_of);
            return -1;
        }
        src_of[orow] = (int32_t) r;
    }
    size_t nnz = 0;
    for (uint32_t orow = 0; orow < out_rows; ++orow) {
        major_ptr[orow] = (uint32_t) nnz;
        const int32_t r = src_of[orow];
        if (r < 0) continue;
        const uint32_t rb = B != 0u ? (uint32_t) r / B : 0u;
        for (uint32_t e = 0; e < ell_cols; ++e) {
            const uint32_t slot = e / B;
            const uint32_t bc = bci[(size_t) rb * W + slot];
            if (bc == INVALID_COL) continue;
            const uint32_t gene = bc * B + e % B;
            const uint16_t h = val[(size_t) r * ell_cols + e];
            if (!(gene < cols && half_nonzero(h) && kept_feature(fk, gene))) continue;
            const uint32_t oc = feature_remap != NULL ? feature_remap[gene] : gene;
            if (oc >= out_cols) continue;
            minor_idx[nnz] = oc;
            out_val[nnz] = h;
            ++nnz;
        }
    }
    major_ptr[out_rows] = (uint32_t) nnz;
    free(src_of);
    return (long long) nnz;
}

/* ------------------------------------------------------------------------ */
/* Grouped moments in FP64, feature-partitioned over threads: each thread     */
/* owns a column range and walks every kept row in ascending order, so every  */
/* (group, feature) sum is taken in row order -- the result does not depend   */
/* on the thread count, and no thread holds a private G x C copy.  Rows whose */
/* columns are ascending are entered by binary search; others are filtered.   */
/* ------------------------------------------------------------------------ */
typedef struct {
    int kind; /* 0 = bell, 1 = csr */
    uint32_t rows, cols, B, ell_cols;
    const uint32_t *bci, *ptr, *idx;
    const uint16_t *val;
    const uint8_t *row_keep;
    const uint32_t *labels;
    const uint8_t *sorted; /* per row (csr) or row block (bell): columns ascending */
    uint32_t G, ddof;
    const uint8_t *fk;
    const uint32_t *group_rows;
    uint32_t f0, f1; /* owned features; multiples of B (bell) except at cols */
    double *sum, *sumsq, *mean, *var;
} mom_task;

static uint32_t lower_bound_u32(const uint32_t *a, uint32_t n, uint32_t x) {
    uint32_t lo = 0u, hi = n;
    while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2u;
        if (a[mid] < x)
            lo = mid + 1u;
        else
            hi = mid;
    }
    return lo;
}

static void *mom_worker(void *arg) {
    mom_task *t = (mom_task *) arg;
    const uint32_t W = t->B != 0u ? t->ell_cols / t->B : 0u;
    for (uint32_t g = 0; g < t->G; ++g)
        for (uint32_t f = t->f0; f < t->f1; ++f) {
            t->sum[(size_t) g * t->cols + f] = 0.0;
            t->sumsq[(size_t) g * t->cols + f] = 0.0;
        }
    for (uint32_t r = 0; r < t->rows; ++r) {
        if (t->row_keep != NULL && t->row_keep[r] == 0u) continue;
        const uint32_t g = t->labels != NULL ? t->labels[r] : 0u;
        if (g >= t->G) continue;
        double *s = t->sum + (size_t) g * t->cols;
        double *q = t->sumsq + (size_t) g * t->cols;
        if (t->kind == 0) {
            const uint32_t rb = r / t->B;
            const uint32_t *brow = t->bci + (size_t) rb * W;
            const uint16_t *vrow = t->val + (size_t) r * t->ell_cols;
            uint32_t slot = t->sorted[rb] ? lower_bound_u32(brow, W, t->f0 / t->B) : 0u;
            for (; slot < W; ++slot) {
                const uint32_t bc = brow[slot];
                if (bc == INVALID_COL) {
                    if (t->sorted[rb]) break;
                    continue;
                }
                if ((uint64_t) bc * t->B >= t->f1) {
                    if (t->sorted[rb]) break;
                    continue;
                }
                for (uint32_t l = 0; l < t->B; ++l) {
                    const uint32_t f = bc * t->B + l;
                    if (f >= t->cols || f < t->f0 || f >= t->f1) continue;
                    const double x = cso_h2f(vrow[(size_t) slot * t->B + l]);
                    s[f] += x;
                    q[f] += x * x;
                }
            }
        } else {
            const uint32_t a = t->ptr[r], e = t->ptr[r + 1u];
            uint32_t i = t->sorted[r] ? a + lower_bound_u32(t->idx + a, e - a, t->f0) : a;
            for (; i < e; ++i) {
                const uint32_t f = t->idx[i];
                if (f < t->f0 || f >= t->f1) {
                    if (t->sorted[r] && f >= t->f1) break;
                    continue;
                }
                const double x = cso_h2f(t->val[i]);
                s[f] += x;
                q[f] += x * x;
            }
        }
    }
    for (uint32_t g = 0; g < t->G; ++g) {
        const uint32_t n = t->group_rows[g];
        for (uint32_t f = t->f0; f < t->f1; ++f) {
            const size_t k = (size_t) g * t->cols + f;
            double sv = t->sum[k], qv = t->sumsq[k];
            if (t->fk != NULL && t->fk[f] == 0u) sv = qv = 0.0;
            double m = 0.0, v = 0.0;
            if (n > 0u && (t->fk == NULL || t->fk[f] != 0u)) {
                m = sv / (double) n;
                if (n > t->ddof) {
                    double m2 = qv - sv * m;
                    if (m2 < 0.0) m2 = 0.0;
                    v = m2 / (double) (n - t->ddof);
                }
            }
            t->sum[k] = sv;
            t->sumsq[k] = qv;
            if (t->mean != NULL) t->mean[k] = m;
            if (t->var != NULL) t->var[k] = v;
        }
    }
    return NULL;
}

static int moments_run(mom_task proto, const uint8_t *fk, uint32_t ddof, double *sum, double *sumsq, double *mean,
                       double *var, uint32_t *group_rows, int nthreads) {
    const uint32_t unit = proto.kind == 0 ? proto.B : 1u;
    const uint32_t units = (proto.cols + unit - 1u) / unit;
    if (nthreads < 1) nthreads = 1;
    if ((uint32_t) nthreads > units && units > 0u) nthreads = (int) units;
    if (nthreads < 1) nthreads = 1;
    uint32_t *n = (uint32_t *) calloc((size_t) proto.G + 1u, sizeof(uint32_t));
    const size_t nsorted = proto.kind == 0 ? ((size_t) proto.rows + proto.B - 1u) / proto.B : proto.rows;
    uint8_t *sorted = (uint8_t *) malloc(nsorted + 1u);
    mom_task *tasks = (mom_task *) calloc((size_t) nthreads, sizeof(mom_task));
    pthread_t *th = (pthread_t *) calloc((size_t) nthreads, sizeof(pthread_t));
    if (n == NULL || sorted == NULL || tasks == NULL || th == NULL) {
        free(n);
        free(sorted);
        free(tasks);
        free(th);
        return 0;
    }
    for (uint32_t r = 0; r < proto.rows; ++r) {
        if (proto.row_keep != NULL && proto.row_keep[r] == 0u) continue;
        const uint32_t g = proto.labels != NULL ? proto.labels[r] : 0u;
        if (g < proto.G) n[g] += 1u;
    }
    const uint32_t W = proto.kind == 0 ? proto.ell_cols / proto.B : 0u;
    for (size_t u = 0; u < nsorted; ++u) {
        const uint32_t *a = proto.kind == 0 ? proto.bci + u * W : proto.idx + proto.ptr[u];
        const uint32_t len = proto.kind == 0 ? W : proto.ptr[u + 1u] - proto.ptr[u];
        uint8_t ok = 1u;
        for (uint32_t j = 1; j < len && ok; ++j) ok = a[j - 1u] <= a[j];
        sorted[u] = ok;
    }
    for (int t = 0; t < nthreads; ++t) {
        tasks[t] = proto;
        tasks[t].sorted = sorted;
        tasks[t].fk = fk;
        tasks[t].ddof = ddof;
        tasks[t].group_rows = n;
        const uint64_t u0 = (uint64_t) units * (uint64_t) t / (uint64_t) nthreads;
        const uint64_t u1 = (uint64_t) units * (uint64_t) (t + 1) / (uint64_t) nthreads;
        tasks[t].f0 = (uint32_t) (u0 * unit < proto.cols ? u0 * unit : proto.cols);
        tasks[t].f1 = (uint32_t) (u1 * unit < proto.cols ? u1 * unit : proto.cols);
        tasks[t].sum = sum;
        tasks[t].sumsq = sumsq;
        tasks[t].mean = mean;
        tasks[t].var = var;
    }
    for (int t = 1; t < nthreads; ++t) pthread_create(&th[t], NULL, mom_worker, &tasks[t]);
    mom_worker(&tasks[0]);
    for (int t = 1; t < nthreads; ++t) pthread_join(th[t], NULL);
    if (group_rows != NULL)
        for (uint32_t g = 0; g < proto.G; ++g) group_rows[g] = n[g];
    free(n);
    free(sorted);
    free(tasks);
    free(th);
    return 1;
}

int cso_group_moments_bell(uint32_t rows, uint32_t cols, uint32_t B, uint32_t ell_cols, const uint32_t *bci,
                           const uint16_t *val, const uint8_t *row_keep, const uint8_t *fk, const uint32_t *labels,
                           uint32_t G, uint32_t ddof, double *sum, double *sumsq, double *mean, double *var,
                           uint32_t *group_rows, int nthreads) {
    if (B == 0u || G == 0u) return 0;
    mom_task p;
    memset(&p, 0, sizeof(p));
    p.kind = 0;
    p.rows = rows;
    p.cols = cols;
    p.B = B;
    p.ell_cols = ell_cols;
    p.bci = bci;
    p.val = val;
    p.row_keep = row_keep;
    p.labels = labels;
    p.G = G;
    return moments_run(p, fk, ddof, sum, sumsq, mean, var, group_rows, nthreads);
}

int cso_group_moments_csr(uint32_t rows, uint32_t cols, const uint32_t *ptr, const uint32_t *idx,
                          const uint16_t *val, const uint8_t *row_keep, const uint8_t *fk, const uint32_t *labels,
                          uint32_t G, uint32_t ddof, double *sum, double *sumsq, double *mean, double *var,
                          uint32_t *group_rows, int nthreads) {
    if (G == 0u) return 0;
    mom_task p;
    memset(&p, 0, sizeof(p));
    p.kind = 1;
    p.rows = rows;
    p.cols = cols;
    p.B = 1u;
    p.ptr = ptr;
    p.idx = idx;
    p.val = val;
    p.row_keep = row_keep;
    p.labels = labels;
    p.G = G;
    return moments_run(p, fk, ddof, sum, sumsq, mean, var, group_rows, nthreads);
}

int cso_group_moments_bell_f32(uint32_t rows, uint32_t cols, uint32_t B, uint32_t ell_cols, const uint32_t *bci,
                               const uint16_t *val, const uint8_t *row_keep, const uint32_t *labels, uint32_t G,
                               float *sum, float *sumsq) {
    if (B == 0u) return 0;
    const uint32_t W = ell_cols / B;
    memset(sum, 0, (size_t) G * cols * sizeof(float));
    memset(sumsq, 0, (size_t) G * cols * sizeof(float));
    for (uint32_t r = 0; r < rows; ++r) {
        if (row_keep != NULL && row_keep[r] == 0u) continue;
        const uint32_t g = labels != NULL ? labels[r] : 0u;
        if (g >= G) continue;
        const uint32_t rb = r / B;
        for (uint32_t slot = 0; slot < W; ++slot) {
            const uint32_t bc = bci[(size_t) rb * W + slot];
            if (bc == INVALID_COL) continue;
            for (uint32_t l = 0; l < B; ++l) {
                const uint32_t f = bc * B + l;
                if (f >= cols) continue;
                const float x = cso_h2f(val[(size_t) r * ell_cols + (size_t) slot * B + l]);
                sum[(size_t) g * cols + f] += x;
                sumsq[(size_t) g * cols + f] += x * x;
            }
        }
    }
    return 1;
}

/* ------------------------------------------------------------------------ */
/* CSR -> Blocked-ELL (blocked_ell_from_compressed.cuh:33-91 shape with epoch */
/* marks; :294-342 sorted unique block cols per row block, value scatter in  */
/* CSR order, nnz = count of nonzero written values, :332-344).             */
/* ------------------------------------------------------------------------ */
static int cmp_u32(const void *a, const void *b) {
    const uint32_t x = *(const uint32_t *) a, y = *(const uint32_t *) b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

int cso_blocked_ell_shape(uint32_t rows, uint32_t cols, const uint32_t *ptr, const uint32_t *idx, uint32_t B,
                          uint32_t *ell_width, uint64_t *total_blocks) {
    *ell_width = 0u;
    *total_blocks = 0u;
    if (rows == 0u || cols == 0u || B == 0u) return 1;
    const uint32_t col_blocks = (cols + B - 1u) / B;
    const uint32_t row_blocks = (rows + B - 1u) / B;
    uint32_t *marks = (uint32_t *) calloc(col_blocks, sizeof(uint32_t));
    if (marks == NULL) return 0;
    uint32_t epoch = 1u;
    for (uint32_t rb = 0; rb < row_blocks; ++rb) {
        uint32_t unique = 0u;
        const uint32_t r1 = rb * B + B < rows ? rb * B + B : rows;
        for (uint32_t r = rb * B; r < r1; ++r)
            for (uint32_t i = ptr[r]; i < ptr[r + 1u]; ++i) {
                const uint32_t bc = idx[i] / B;
                if (marks[bc] != epoch) {
                    marks[bc] = epoch;
                    ++unique;
                }
            }
        *total_blocks += unique;
        if (unique > *ell_width) *ell_width = unique;
        ++epoch;
    }
    free(marks);
    return 1;
}

uint32_t cso_blocked_ell_from_csr(uint32_t rows, uint32_t cols, const uint32_t *ptr, const uint32_t *idx,
                                  const uint16_t *val, uint32_t B, uint32_t W, uint32_t *bci, uint16_t *out_val) {
    const uint32_t row_blocks = (rows + B - 1u) / B;
    const uint32_t col_blocks = (cols + B - 1u) / B;
    const uint32_t ell_cols = W * B;
    for (size_t i = 0; i < (size_t) row_blocks * W; ++i) bci[i] = INVALID_COL;
    memset(out_val, 0, (size_t) rows * ell_cols * sizeof(uint16_t));
    uint32_t *marks = (uint32_t *) calloc(col_blocks + 1u, sizeof(uint32_t));
    uint32_t *slot_of = (uint32_t *) calloc(col_blocks + 1u, sizeof(uint32_t));
    uint32_t *list = (uint32_t *) calloc(W + 1u, sizeof(uint32_t));
    uint32_t epoch = 1u;
    for (uint32_t rb = 0; rb < row_blocks; ++rb) {
        uint32_t unique = 0u;
        ++epoch;
        const uint32_t r1 = rb * B + B < rows ? rb * B + B : rows;
        for (uint32_t r = rb * B; r < r1; ++r)
            for (uint32_t i = ptr[r]; i < ptr[r + 1u]; ++i) {
                const uint32_t bc = idx[i] / B;
                if (marks[bc] != epoch) {
                    marks[bc] = epoch;
                    list[unique++] = bc;
                }
            }
        qsort(list, unique, sizeof(uint32_t), cmp_u32);
        for (uint32_t s = 0; s < unique; ++s) {
            bci[(size_t) rb * W + s] = list[s];
            slot_of[list[s]] = s;
        }
        for (uint32_t r = rb * B; r < r1; ++r)
            for (uint32_t i = ptr[r]; i < ptr[r + 1u]; ++i) {
                const uint32_t c = idx[i];
                out_val[(size_t) r * ell_cols + (size_t) slot_of[c / B] * B + c % B] = val[i];
            }
    }
    uint32_t nnz = 0u;
    for (size_t i = 0; i < (size_t) rows * ell_cols; ++i) nnz += half_nonzero(out_val[i]);
    free(marks);
    free(slot_of);
    free(list);
    return nnz;
}

/* ------------------------------------------------------------------------ */
/* CSR -> Sliced-ELL: uniform slices of clamp(slice_rows, 1, rows) rows,      */
/* width = max row nnz in the slice (build_uniform_sliced_layout_,           */
/* sliced_ell_from_blocked_ell.cuh:111-142), slot offsets = u32 running sum  */
/* (sharded_device.cuh:716-723), entries copied into each row's first slots, */
/* padding col 0xffffffff val 0 (sliced_ell.cuh:218-221, sliced_ell_from_   */
/* compressed.cuh:125-140).                                                  */
/* ------------------------------------------------------------------------ */
static uint32_t clamp_slice(uint32_t rows, uint32_t h) {
    if (rows == 0u) return 0u;
    if (h < 1u) h = 1u;
    return h < rows ? h : rows;
}

uint32_t cso_sliced_slice_count(uint32_t rows, uint32_t slice_rows) {
    const uint32_t h = clamp_slice(rows, slice_rows);
    return rows == 0u ? 0u : (rows + h - 1u) / h;
}

uint64_t cso_sliced_ell_layout(uint32_t rows, const uint32_t *ptr, uint32_t slice_rows, uint32_t *offsets,
                               uint32_t *widths, uint32_t *slot_offsets) {
    const uint32_t h = clamp_slice(rows, slice_rows);
    const uint32_t S = cso_sliced_slice_count(rows, slice_rows);
    offsets[0] = 0u;
    uint32_t run = 0u;
    uint64_t total = 0u;
    for (uint32_t s = 0; s < S; ++s) {
        const uint32_t r0 = s * h, r1 = r0 + h < rows ? r0 + h : rows;
        uint32_t w = 0u;
        for (uint32_t r = r0; r < r1; ++r) {
            const uint32_t n = ptr[r + 1u] - ptr[r];
            if (n > w) w = n;
        }
        offsets[s + 1u] = r1;
        widths[s] = w;
        slot_offsets[s] = run;
        run += (r1 - r0) * w;
        total += (uint64_t) (r1 - r0) * w;
    }
    return total;
}

void cso_sliced_ell_fill(uint32_t rows, const uint32_t *ptr, const uint32_t *idx, const uint16_t *val,
                         uint32_t slice_rows, const uint32_t *offsets, const uint32_t *widths,
                         const uint32_t *slot_offsets, uint32_t *col_idx, uint16_t *out_val) {
    const uint32_t S = cso_sliced_slice_count(rows, slice_rows);
    for (uint32_t s = 0; s < S; ++s) {
        const uint32_t w = widths[s];
        for (uint32_t r = offsets[s]; r < offsets[s + 1u]; ++r) {
            const size_t base = (size_t) slot_offsets[s] + (size_t) (r - offsets[s]) * w;
            uint32_t k = 0u;
            for (uint32_t i = ptr[r]; i < ptr[r + 1u]; ++i, ++k) {
                col_idx[base + k] = idx[i];
                out_val[base + k] = val[i];
            }
            for (; k < w; ++k) {
                col_idx[base + k] = INVALID_COL;
                out_val[base + k] = 0u;
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Blocked-ELL -> its live entries as CSR, the input of the Sliced-ELL layout  */
/* and fill above: per row, slots in order, lanes in order, an entry when the  */
/* slot's block column is valid, the column is < cols and the value is nonzero */
/* as a float (count_blocked_ell_row_nnz_ and the emit loop,                  */
/* sliced_ell_from_blocked_ell.cuh:36-62,146-190).  With ptr == NULL only the  */
/* row counts are written (into row_nnz) and the total returned.              */
/* ------------------------------------------------------------------------ */
uint64_t cso_bell_live_csr(uint32_t rows, uint32_t cols, uint32_t B, uint32_t ell_cols, const uint32_t *bci,
                           const uint16_t *val, uint32_t *ptr, uint32_t *idx, uint16_t *out_val) {
    const uint32_t W = B != 0u ? ell_cols / B : 0u;
    uint64_t n = 0u;
    if (ptr != NULL) ptr[0] = 0u;
    for (uint32_t r = 0; r < rows; ++r) {
        const uint32_t rb = B != 0u ? r / B : 0u;
        for (uint32_t s = 0; s < W; ++s) {
            const uint32_t bc = bci[(size_t) rb * W + s];
            if (bc == INVALID_COL) continue;
            for (uint32_t l = 0; l < B; ++l) {
                const uint32_t c = bc * B + l;
                const uint16_t h = val[(size_t) r * ell_cols + (size_t) s * B + l];
                if (c >= cols || cso_h2f(h) == 0.0f) continue;
                if (idx != NULL) {
                    idx[n] = c;
                    out_val[n] = h;
                }
                ++n;
            }
        }
        if (ptr != NULL) ptr[r + 1u] = (uint32_t) n;
    }
    return n;
}

uint64_t cso_sliced_padded_slots(uint32_t rows, const uint32_t *ptr, uint32_t candidate) {
    const uint32_t h = clamp_slice(rows, candidate);
    uint64_t padded = 0u;
    for (uint32_t r0 = 0; r0 < rows; r0 += h) {
        const uint32_t r1 = r0 + h < rows ? r0 + h : rows;
        uint32_t w = 0u;
        for (uint32_t r = r0; r < r1; ++r) {
            const uint32_t n = ptr[r + 1u] - ptr[r];
            if (n > w) w = n;
        }
        padded += (uint64_t) (r1 - r0) * w;
    }
    return padded;
}

/* ------------------------------------------------------------------------ */
/* Transpose: stable counting sort by column (rows ascending per column).    */
/* ------------------------------------------------------------------------ */
void cso_csr_transpose(uint32_t cDim, uint32_t uDim, const uint32_t *ptr, const uint32_t *idx, const uint16_t *val,
                       uint32_t *out_ptr, uint32_t *out_idx, uint16_t *out_val) {
    memset(out_ptr, 0, ((size_t) uDim + 1u) * sizeof(uint32_t));
    const uint32_t nnz = cDim ? ptr[cDim] : 0u;
    for (uint32_t i = 0; i < nnz; ++i) out_ptr[idx[i] + 1u] += 1u;
    for (uint32_t c = 0; c < uDim; ++c) out_ptr[c + 1u] += out_ptr[c];
    uint32_t *head = (uint32_t *) malloc(((size_t) uDim + 1u) * sizeof(uint32_t));
    memcpy(head, out_ptr, ((size_t) uDim + 1u) * sizeof(uint32_t));
    for (uint32_t r = 0; r < cDim; ++r)
        for (uint32_t i = ptr[r]; i < ptr[r + 1u]; ++i) {
            const uint32_t d = head[idx[i]]++;
            out_idx[d] = r;
            out_val[d] = val[i];
        }
    free(head);
}

/* ------------------------------------------------------------------------ */
/* nnz bucketing: counts (count_major_nnz.cuh), stable ascending sort by     */
/* count with row ids as values (CUB SortPairs over all 32 key bits,         */
/* major_nnz_raw.cuh:96-108), equal-count offsets where the first n % B      */
/* buckets take one extra row (fill_equal_count_bucket_offsets.cuh:13-25).   */
/* ------------------------------------------------------------------------ */
static const uint32_t *g_sort_keys;
static int cmp_by_key_then_id(const void *a, const void *b) {
    const uint32_t x = *(const uint32_t *) a, y = *(const uint32_t *) b;
    const uint32_t kx = g_sort_keys[x], ky = g_sort_keys[y];
    if (kx != ky) return kx < ky ? -1 : 1;
    return x < y ? -1 : (x > y ? 1 : 0);
}

void cso_major_nnz_plan(const uint32_t *major_ptr, uint32_t n, uint32_t requested, uint32_t *major_nnz,
                        uint32_t *sorted, uint32_t *order, uint32_t *bucket_offsets) {
    if (n == 0u) {
        if (bucket_offsets != NULL) bucket_offsets[0] = 0u;
        return;
    }
    for (uint32_t i = 0; i < n; ++i) {
        major_nnz[i] = major_ptr[i + 1u] - major_ptr[i];
        order[i] = i;
    }
    g_sort_keys = major_nnz;
    qsort(order, n, sizeof(uint32_t), cmp_by_key_then_id);
    for (uint32_t i = 0; i < n; ++i) sorted[i] = major_nnz[order[i]];
    if (bucket_offsets != NULL) {
        uint32_t B = requested < 1u ? 1u : requested;
        if (B > n) B = n;
        const uint32_t size = n / B, rem = n % B;
        uint32_t off = 0u;
        for (uint32_t b = 0; b < B; ++b) {
            bucket_offsets[b] = off;
            off += size + (b < rem ? 1u : 0u);
        }
        bucket_offsets[B] = n;
    }
}

void cso_pow2_bins(const uint32_t *sorted, uint32_t n, uint32_t *bins) {
    bins[0] = 0u;
    for (uint32_t k = 1; k <= 32u; ++k) {
        const uint64_t bound = (uint64_t) 1u << k;
        uint32_t lo = 0u, hi = n;
        while (lo < hi) {
            const uint32_t mid = lo + (hi - lo) / 2u;
            if ((uint64_t) sorted[mid] < bound)
                lo = mid + 1u;
            else
                hi = mid;
        }
        bins[k] = lo;
    }
    bins[33] = n;
}

void cso_rebuild(const uint32_t *ptr, const uint32_t *idx, const uint16_t *val, uint32_t n, const uint32_t *order,
                 uint32_t *dst_ptr, uint32_t *dst_idx, uint16_t *dst_val, uint32_t *inverse) {
    uint32_t run = 0u;
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t src = order[i];
        const uint32_t len = ptr[src + 1u] - ptr[src];
        dst_ptr[i] = run;
        memcpy(dst_idx + run, idx + ptr[src], (size_t) len * sizeof(uint32_t));
        memcpy(dst_val + run, val + ptr[src], (size_t) len * sizeof(uint16_t));
        run += len;
        if (inverse != NULL) inverse[src] = i;
    }
    dst_ptr[n] = run;
}

/* ------------------------------------------------------------------------ */
/* Execution bucketing of one Blocked-ELL part                               */
/* (src/io/csh5/execution_builders_part.hh:1018-1272).  Row blocks are       */
/* ordered by their count of valid block columns (a stable ascending sort    */
/* that leaves a partial last row block in place), cut into equal row-block  */
/* ranges whose width is their widest member, and copied with the valid      */
/* slots compacted to the front of each row block.                           */
/* ------------------------------------------------------------------------ */
#define CSO_INVALID 0xffffffffu

static uint32_t bell_rb_rows(uint32_t rows, uint32_t B, uint32_t rb) {
    const uint64_t begin = (uint64_t) rb * B;
    if (begin >= rows) return 0u;
    return rows - begin < B ? (uint32_t) (rows - begin) : B;
}

uint64_t cso_packed_blocked_ell_bytes(uint32_t rows, uint32_t ell_cols, uint32_t B) {
    /* io/pack/packfile.cuh:110-116: 16-byte disk header, two u32 words, the
     * block column indices and the fp16 values */
    const uint64_t rb = B == 0u ? 0u : ((uint64_t) rows + B - 1u) / B;
    const uint64_t w = B == 0u ? 0u : ell_cols / B;
    return 16u + 8u + rb * w * 4u + (uint64_t) rows * ell_cols * 2u;
}

uint32_t cso_bell_exec_layout(uint32_t rows, uint32_t B, uint32_t W, const uint32_t *bci, uint32_t requested,
                              uint32_t *order, uint32_t *widths, uint32_t *seg_rb, uint32_t *seg_w) {
    const uint32_t RB = B == 0u ? 0u : (uint32_t) (((uint64_t) rows + B - 1u) / B);
    seg_rb[0] = 0u;
    if (RB == 0u) return 0u;
    for (uint32_t rb = 0; rb < RB; ++rb) {
        uint32_t n = 0u;
        for (uint32_t s = 0; s < W; ++s) n += bci[(size_t) rb * W + s] != CSO_INVALID;
        order[rb] = rb;
        widths[rb] = n;
    }
    const uint32_t sortable = bell_rb_rows(rows, B, RB - 1u) != B ? RB - 1u : RB;
    g_sort_keys = widths;
    qsort(order, sortable, sizeof(uint32_t), cmp_by_key_then_id);
    const uint32_t nb = requested < 1u ? 1u : (requested > RB ? RB : requested);
    for (uint32_t b = 0; b < nb; ++b) {
        /* u32 products, as written in the reference */
        const uint32_t lo = (b * RB) / nb, hi = ((b + 1u) * RB) / nb;
        uint32_t w = 0u;
        for (uint32_t p = lo; p < hi; ++p)
            if (widths[order[p]] > w) w = widths[order[p]];
        seg_w[b] = w;
        seg_rb[b + 1u] = hi;
    }
    if (nb > 1u) {
        uint32_t same = 1u;
        for (uint32_t b = 1; b < nb; ++b) same &= seg_w[b] == seg_w[0];
        if (same) {
            seg_rb[1] = RB;
            return 1u;
        }
    }
    return nb;
}

static uint32_t bell_seg_rows(uint32_t rows, uint32_t B, const uint32_t *order, uint32_t lo, uint32_t hi) {
    uint32_t n = 0u;
    for (uint32_t p = lo; p < hi; ++p) n += bell_rb_rows(rows, B, order[p]);
    return n;
}

uint32_t cso_bell_exec_build_layout(uint32_t rows, uint32_t B, uint32_t W, const uint32_t *bci, uint32_t requested,
                                    uint32_t *order, uint32_t *widths, uint32_t *seg_rb, uint32_t *seg_w,
                                    uint64_t *bytes) {
    uint32_t S = cso_bell_exec_layout(rows, B, W, bci, requested, order, widths, seg_rb, seg_w);
    uint64_t cand = 0u;
    for (uint32_t s = 0; s < S; ++s)
        cand += cso_packed_blocked_ell_bytes(bell_seg_rows(rows, B, order, seg_rb[s], seg_rb[s + 1u]), seg_w[s] * B, B);
    const uint64_t orig = cso_packed_blocked_ell_bytes(rows, W * B, B);
    if (S > 1u && cand >= orig) {
        S = cso_bell_exec_layout(rows, B, W, bci, 1u, order, widths, seg_rb, seg_w);
        cand = orig;
    }
    if (bytes != NULL) *bytes = cand;
    return S;
}

void cso_bell_exec_fill(uint32_t rows, uint32_t B, uint32_t W, const uint32_t *bci, const uint16_t *val,
                        const uint32_t *order, uint32_t S, const uint32_t *seg_rb, const uint32_t *seg_w,
                        uint32_t *seg_bci, uint16_t *seg_val, uint32_t *exec_to_canonical,
                        uint32_t *canonical_to_exec) {
    const size_t src_ell = (size_t) W * B;
    size_t bci_off = 0u, val_off = 0u;
    uint32_t exec_row = 0u;
    for (uint32_t s = 0; s < S; ++s) {
        const uint32_t lo = seg_rb[s], hi = seg_rb[s + 1u], dw = seg_w[s];
        const size_t dst_ell = (size_t) dw * B;
        const uint32_t seg_rows = bell_seg_rows(rows, B, order, lo, hi);
        for (size_t i = 0; i < (size_t) (hi - lo) * dw; ++i) seg_bci[bci_off + i] = CSO_INVALID;
        memset(seg_val + val_off, 0, (size_t) seg_rows * dst_ell * sizeof(uint16_t));
        for (uint32_t p = lo; p < hi; ++p) {
            const uint32_t dst_rb = p - lo, src_rb = order[p], n = bell_rb_rows(rows, B, src_rb);
            for (uint32_t r = 0; r < n; ++r) {
                exec_to_canonical[exec_row + r] = src_rb * B + r;
                canonical_to_exec[src_rb * B + r] = exec_row + r;
            }
            uint32_t slot = 0u;
            for (uint32_t k = 0; k < W; ++k) {
                const uint32_t c = bci[(size_t) src_rb * W + k];
                if (c == CSO_INVALID) continue;
                seg_bci[bci_off + (size_t) dst_rb * dw + slot] = c;
                for (uint32_t r = 0; r < n; ++r)
                    memcpy(seg_val + val_off + ((size_t) dst_rb * B + r) * dst_ell + (size_t) slot * B,
                           val + ((size_t) src_rb * B + r) * src_ell + (size_t) k * B, (size_t) B * sizeof(uint16_t));
                ++slot;
            }
            exec_row += n;
        }
        bci_off += (size_t) (hi - lo) * dw;
        val_off += (size_t) seg_rows * dst_ell;
    }
}

int cso_bell_choose_bucket_count(uint32_t rows, uint32_t B, uint32_t W, const uint32_t *bci, uint32_t *count,
                                 uint64_t *bytes) {
    const uint32_t RB = B == 0u ? 0u : (uint32_t) (((uint64_t) rows + B - 1u) / B);
    const uint32_t top = RB < 8u ? (RB < 1u ? 1u : RB) : 8u;
    uint32_t *order = (uint32_t *) malloc(((size_t) RB + 1u) * 2u * sizeof(uint32_t));
    uint32_t seg_rb[9], seg_w[8];
    uint32_t best = 1u;
    uint64_t best_bytes = UINT64_MAX;
    if (order == NULL) return 0;
    for (uint32_t b = 1; b <= top; ++b) {
        uint64_t x = 0u;
        cso_bell_exec_build_layout(rows, B, W, bci, b, order, order + RB + 1u, seg_rb, seg_w, &x);
        if (x < best_bytes) {
            best_bytes = x;
            best = b;
        }
    }
    free(order);
    *count = best;
    *bytes = best_bytes;
    return 1;
}

/* ------------------------------------------------------------------------ */
/* Execution bucketing of one Sliced-ELL part                                */
/* (src/io/csh5/execution_builders_part.hh:1274-1596).  Rows are ordered by  */
/* their live slot count (stable, ascending) and split into at most the      */
/* requested number of single-slice segments by a dynamic programme that     */
/* minimises packed bytes (fixed segment bytes + 6 bytes per slot, a segment  */
/* as wide as its last row), solved with a monotone convex-hull of lines;    */
/* neighbouring segments of equal width are merged.                          */
/* ------------------------------------------------------------------------ */
uint64_t cso_packed_sliced_ell_bytes(uint32_t slice_count, uint64_t total_slots) {
    /* io/pack/packfile.cu:179-188: 13-byte header, one u32, slice offsets,
     * slice widths, column indices and fp16 values */
    return 13u + 4u + ((uint64_t) slice_count + 1u) * 4u + (uint64_t) slice_count * 4u + total_slots * 6u;
}

static uint32_t sell_find_slice(uint32_t rows, uint32_t S, const uint32_t *offsets, uint32_t row) {
    if (row >= rows) return S;
    for (uint32_t s = 0; s < S; ++s)
        if (row < offsets[s + 1u]) return s;
    return S;
}

typedef struct {
    int64_t slope, intercept;
    uint32_t cut;
} cso_line;

static int64_t line_at(const cso_line *l, uint32_t x) { return l->intercept + l->slope * (int64_t) x; }

static int line_redundant(const cso_line *a, const cso_line *m, const cso_line *b) {
    const __int128 left = (__int128) (b->intercept - a->intercept) * (__int128) (a->slope - m->slope);
    const __int128 right = (__int128) (m->intercept - a->intercept) * (__int128) (a->slope - b->slope);
    return left <= right;
}

/* sorted_widths[rows] (ascending); seg_row[S+1], seg_w[S] sized for
 * min(requested, rows) segments.  Returns S, or -1 when no split exists. */
int cso_sell_exec_dp(uint32_t rows, const uint32_t *sorted_widths, uint32_t requested, uint32_t *seg_row,
                     uint32_t *seg_w) {
    const uint32_t K = requested < 1u ? 1u : (requested > rows ? (rows < 1u ? 1u : rows) : requested);
    const uint64_t fixed = cso_packed_sliced_ell_bytes(1u, 0u), slot = 6u, inf = UINT64_MAX / 4u;
    seg_row[0] = 0u;
    if (rows == 0u) return 0;
    uint64_t *prev = (uint64_t *) malloc(((size_t) rows + 1u) * sizeof(uint64_t));
    uint64_t *curr = (uint64_t *) malloc(((size_t) rows + 1u) * sizeof(uint64_t));
    uint32_t *cuts = (uint32_t *) calloc(((size_t) K + 1u) * ((size_t) rows + 1u), sizeof(uint32_t));
    cso_line *hull = (cso_line *) malloc(((size_t) rows + 1u) * sizeof(cso_line));
    uint32_t *raw_off = (uint32_t *) malloc(((size_t) K + 1u) * sizeof(uint32_t));
    uint32_t *raw_w = (uint32_t *) malloc(((size_t) K + 1u) * sizeof(uint32_t));
    int out = -1;
    if (!prev || !curr || !cuts || !hull || !raw_off || !raw_w) goto done;
    for (uint32_t i = 0; i <= rows; ++i) prev[i] = inf;
    prev[0] = 0u;
    for (uint32_t k = 1; k <= K; ++k) {
        size_t n = 0u, head = 0u;
        for (uint32_t i = 0; i <= rows; ++i) curr[i] = inf;
        if (prev[k - 1u] != inf) {
            hull[n].slope = -(int64_t) slot * (int64_t) (k - 1u);
            hull[n].intercept = (int64_t) prev[k - 1u];
            hull[n].cut = k - 1u;
            ++n;
        }
        for (uint32_t r = k; r <= rows; ++r) {
            const uint32_t w = sorted_widths[r - 1u];
            while (head + 1u < n && line_at(&hull[head + 1u], w) < line_at(&hull[head], w)) ++head;
            if (head < n) {
                curr[r] = fixed + slot * (uint64_t) w * (uint64_t) r + (uint64_t) line_at(&hull[head], w);
                cuts[(size_t) k * (rows + 1u) + r] = hull[head].cut;
            }
            if (prev[r] != inf) {
                const cso_line l = {-(int64_t) slot * (int64_t) r, (int64_t) prev[r], r};
                while (n >= head + 2u && line_redundant(&hull[n - 2u], &hull[n - 1u], &l)) --n;
                hull[n++] = l;
            }
        }
        uint64_t *t = prev;
        prev = curr;
        curr = t;
    }
    if (prev[rows] == inf) goto done;
    {
        uint32_t r = rows;
        raw_off[K] = rows;
        for (uint32_t k = K; k != 0u; --k) {
            const uint32_t begin = cuts[(size_t) k * (rows + 1u) + r];
            raw_off[k - 1u] = begin;
            raw_w[k - 1u] = sorted_widths[r - 1u];
            r = begin;
        }
        uint32_t S = 0u;
        for (uint32_t k = 0; k < K; ++k) {
            if (S != 0u && seg_w[S - 1u] == raw_w[k]) {
                seg_row[S] = raw_off[k + 1u];
            } else {
                seg_w[S] = raw_w[k];
                seg_row[S + 1u] = raw_off[k + 1u];
                ++S;
            }
        }
        out = (int) S;
    }
done:
    free(prev);
    free(curr);
    free(cuts);
    free(hull);
    free(raw_off);
    free(raw_w);
    return out;
}

/* order[rows], row_widths[rows] (canonical row index) and the DP split;
 * *bytes = bucketed bytes after the fallback to one segment
 * (build_bucketed_sliced_execution_partition:1547-1570).  Returns S or -1. */
int cso_sell_exec_build_layout(uint32_t rows, uint32_t S_src, const uint32_t *offsets, const uint32_t *widths,
                               const uint32_t *col_idx, uint32_t requested, uint32_t *order, uint32_t *row_widths,
                               uint32_t *sorted_widths, uint32_t *seg_row, uint32_t *seg_w, uint64_t *bytes) {
    uint64_t total = 0u;
    for (uint32_t s = 0; s < S_src; ++s) total += (uint64_t) (offsets[s + 1u] - offsets[s]) * widths[s];
    for (uint32_t r = 0; r < rows; ++r) {
        const uint32_t s = sell_find_slice(rows, S_src, offsets, r);
        uint32_t n = 0u;
        if (s < S_src) {
            uint64_t base = 0u;
            for (uint32_t t = 0; t < s; ++t) base += (uint64_t) (offsets[t + 1u] - offsets[t]) * widths[t];
            base += (uint64_t) (r - offsets[s]) * widths[s];
            for (uint32_t k = 0; k < widths[s]; ++k) n += col_idx[base + k] != CSO_INVALID;
        }
        order[r] = r;
        row_widths[r] = n;
    }
    g_sort_keys = row_widths;
    qsort(order, rows, sizeof(uint32_t), cmp_by_key_then_id);
    for (uint32_t r = 0; r < rows; ++r) sorted_widths[r] = row_widths[order[r]];
    int S = cso_sell_exec_dp(rows, sorted_widths, requested, seg_row, seg_w);
    if (S < 0) return -1;
    uint64_t cand = 0u;
    for (int s = 0; s < S; ++s) {
        const uint32_t n = seg_row[s + 1] - seg_row[s];
        cand += cso_packed_sliced_ell_bytes(n != 0u ? 1u : 0u, (uint64_t) n * seg_w[s]);
    }
    const uint64_t orig = cso_packed_sliced_ell_bytes(S_src, total);
    if (S > 1 && cand >= orig) {
        S = cso_sell_exec_dp(rows, sorted_widths, 1u, seg_row, seg_w);
        cand = orig;
    }
    if (bytes != NULL) *bytes = cand;
    return S;
}

void cso_sell_exec_fill(uint32_t rows, uint32_t S_src, const uint32_t *offsets, const uint32_t *widths,
                        const uint32_t *col_idx, const uint16_t *val, const uint32_t *order, uint32_t S,
                        const uint32_t *seg_row, const uint32_t *seg_w, uint32_t *seg_col, uint16_t *seg_val,
                        uint32_t *exec_to_canonical, uint32_t *canonical_to_exec) {
    size_t off = 0u;
    for (uint32_t s = 0; s < S; ++s) {
        const uint32_t w = seg_w[s];
        for (uint32_t p = seg_row[s]; p < seg_row[s + 1u]; ++p) {
            const uint32_t row = order[p], src = sell_find_slice(rows, S_src, offsets, row);
            uint32_t *dc = seg_col + off + (size_t) (p - seg_row[s]) * w;
            uint16_t *dv = seg_val + off + (size_t) (p - seg_row[s]) * w;
            for (uint32_t k = 0; k < w; ++k) {
                dc[k] = CSO_INVALID;
                dv[k] = 0u;
            }
            if (src < S_src) {
                uint64_t base = 0u;
                for (uint32_t t = 0; t < src; ++t) base += (uint64_t) (offsets[t + 1u] - offsets[t]) * widths[t];
                base += (uint64_t) (row - offsets[src]) * widths[src];
                uint32_t d = 0u;
                for (uint32_t k = 0; k < widths[src]; ++k) {
                    if (col_idx[base + k] == CSO_INVALID) continue;
                    dc[d] = col_idx[base + k];
                    dv[d] = val[base + k];
                    ++d;
                }
            }
            exec_to_canonical[p] = row;
            canonical_to_exec[row] = p;
        }
        off += (size_t) (seg_row[s + 1u] - seg_row[s]) * w;
    }
}

int cso_sell_choose_bucket_count(uint32_t rows, uint32_t S_src, const uint32_t *offsets, const uint32_t *widths,
                                 const uint32_t *col_idx, uint32_t *count, uint64_t *bytes) {
    const uint32_t top = rows < 8u ? (rows < 1u ? 1u : rows) : 8u;
    uint32_t *buf = (uint32_t *) malloc(((size_t) rows + 1u) * 3u * sizeof(uint32_t));
    uint32_t seg_row[9], seg_w[8];
    uint32_t best = 1u;
    uint64_t best_bytes = UINT64_MAX;
    if (buf == NULL) return 0;
    for (uint32_t b = 1; b <= top; ++b) {
        uint64_t x = 0u;
        if (cso_sell_exec_build_layout(rows, S_src, offsets, widths, col_idx, b, buf, buf + rows + 1u,
                                       buf + 2u * ((size_t) rows + 1u), seg_row, seg_w, &x) < 0) {
            free(buf);
            return 0;
        }
        if (x < best_bytes) {
            best_bytes = x;
            best = b;
        }
    }
    free(buf);
    *count = best;
    *bytes = best_bytes;
    return 1;
}

/* ------------------------------------------------------------------------ */
/* Ingest-time bucket-count choice (bucket::build_plan,                      */
/* src/bucket/operators/blocked_ell_bucket.cuh:70-95,149-210, and            */
/* estimate_bucketed_bytes_from_gpu_plan / choose_bucket_count_for_part,     */
/* include/CellShard/ingest/internal/dataset/internal/                       */
/* convert_layout_support_part.hh:116-181).  Row blocks are ordered by the   */
/* 64-bit key (valid width << 32 | hash of the valid block columns), stably. */
/* ------------------------------------------------------------------------ */
static const uint64_t *g_sort_keys64;
static int cmp_by_key64_then_id(const void *a, const void *b) {
    const uint32_t x = *(const uint32_t *) a, y = *(const uint32_t *) b;
    const uint64_t kx = g_sort_keys64[x], ky = g_sort_keys64[y];
    if (kx != ky) return kx < ky ? -1 : 1;
    return x < y ? -1 : (x > y ? 1 : 0);
}

void cso_bell_bucket_plan(uint32_t rows, uint32_t B, uint32_t W, const uint32_t *bci, uint32_t *order,
                          uint32_t *width_sorted) {
    const uint32_t RB = B == 0u ? 0u : (uint32_t) (((uint64_t) rows + B - 1u) / B);
    uint64_t *keys = (uint64_t *) malloc(((size_t) RB + 1u) * sizeof(uint64_t));
    if (keys == NULL) return;
    for (uint32_t rb = 0; rb < RB; ++rb) {
        uint32_t width = 0u, hash = 2166136261u;
        for (uint32_t s = 0; s < W; ++s) {
            const uint32_t c = bci[(size_t) rb * W + s];
            if (c == CSO_INVALID) continue;
            ++width;
            hash ^= c + 0x9e3779b9u + (hash << 6) + (hash >> 2);
            hash *= 16777619u;
        }
        keys[rb] = ((uint64_t) width << 32) | hash;
        order[rb] = rb;
    }
    g_sort_keys64 = keys;
    qsort(order, RB, sizeof(uint32_t), cmp_by_key64_then_id);
    for (uint32_t i = 0; i < RB; ++i) width_sorted[i] = (uint32_t) (keys[order[i]] >> 32);
    free(keys);
}

uint64_t cso_bell_estimate_bucketed_bytes(uint32_t rows, uint32_t B, const uint32_t *order,
                                          const uint32_t *width_sorted, uint32_t RB, uint32_t buckets) {
    uint64_t bytes = 0u;
    if (RB == 0u || buckets == 0u) return 0u;
    for (uint32_t b = 0; b < buckets; ++b) {
        const uint32_t lo = (b * RB) / buckets, hi = ((b + 1u) * RB) / buckets;
        if (hi <= lo) continue;
        const uint32_t w = width_sorted[hi - 1u];
        uint32_t seg_rows = 0u;
        for (uint32_t p = lo; p < hi; ++p) seg_rows += bell_rb_rows(rows, B, order[p]);
        bytes += (uint64_t) (hi - lo) * w * 4u;
        bytes += (uint64_t) seg_rows * w * B * 2u;
    }
    bytes += (uint64_t) rows * 4u * 2u;
    bytes += ((uint64_t) buckets + 1u) * 4u;
    return bytes;
}

uint32_t cso_bell_choose_ingest_bucket_count(uint32_t rows, uint32_t B, uint32_t W, const uint32_t *bci) {
    const uint32_t RB = B == 0u ? 0u : (uint32_t) (((uint64_t) rows + B - 1u) / B);
    const uint32_t top = RB < 8u ? RB : 8u;
    uint64_t best = cso_packed_blocked_ell_bytes(rows, W * B, B);
    uint32_t best_b = 1u;
    if (RB <= 1u) return 1u;
    uint32_t *order = (uint32_t *) malloc((size_t) RB * 2u * sizeof(uint32_t));
    if (order == NULL) return 0u;
    cso_bell_bucket_plan(rows, B, W, bci, order, order + RB);
    for (uint32_t b = 1; b <= (top < 1u ? 1u : top); ++b) {
        const uint64_t x = cso_bell_estimate_bucketed_bytes(rows, B, order, order + RB, RB, b);
        if (x < best || (x == best && b < best_b)) {
            best = x;
            best_b = b;
        }
    }
    free(order);
    return best_b;
}

/* ------------------------------------------------------------------------ */
/* COO -> Blocked-ELL (convert::blocked_ell_from_coo and                     */
/* choose_blocked_ell_block_size_from_coo, src/convert/                      */
/* blocked_ell_from_compressed.cuh:105-257,349-437): row blocks' distinct    */
/* block columns ascending, width = the largest count; values placed in      */
/* COO order (a repeated (row, col) keeps the last); nnz[0] = stored values  */
/* that are nonzero as floats (the host routine's count), nnz[1] = those     */
/* also in a valid slot with column < cols (the CUDA routine's count,        */
/* blocked_ell_from_coo_cuda.cuh:179-198).  Returns the width, or -1 when a  */
/* row index is out of range.                                                */
/* ------------------------------------------------------------------------ */
static uint32_t coo_col(const uint32_t *col, const uint32_t *map, uint64_t i) {
    return map != NULL ? map[col[i]] : col[i];
}

/* per row block: distinct block columns, ascending, into bc (offsets off[RB+1]) */
static int coo_block_cols(uint32_t rows, uint32_t nnz, const uint32_t *row, const uint32_t *col, const uint32_t *map,
                          uint32_t B, uint32_t *off, uint32_t *bc, uint32_t *width, uint64_t *total) {
    const uint32_t RB = (uint32_t) (((uint64_t) rows + B - 1u) / B);
    uint32_t *cur = (uint32_t *) calloc((size_t) RB + 1u, sizeof(uint32_t));
    if (cur == NULL) return 0;
    memset(off, 0, ((size_t) RB + 1u) * sizeof(uint32_t));
    for (uint32_t i = 0; i < nnz; ++i) ++off[row[i] / B + 1u];
    for (uint32_t rb = 0; rb < RB; ++rb) {
        off[rb + 1u] += off[rb];
        cur[rb] = off[rb];
    }
    for (uint32_t i = 0; i < nnz; ++i) bc[cur[row[i] / B]++] = coo_col(col, map, i) / B;
    *width = 0u;
    *total = 0u;
    for (uint32_t rb = 0; rb < RB; ++rb) {
        uint32_t n = off[rb + 1u] - off[rb], u = 0u;
        qsort(bc + off[rb], n, sizeof(uint32_t), cmp_u32);
        for (uint32_t j = 0; j < n; ++j)
            if (j == 0u || bc[off[rb] + j] != bc[off[rb] + j - 1u]) bc[off[rb] + u++] = bc[off[rb] + j];
        cur[rb] = u; /* distinct count, compacted to the front */
        if (u > *width) *width = u;
        *total += u;
    }
    for (uint32_t rb = 0; rb < RB; ++rb) off[rb] = cur[rb]; /* reuse: distinct count per row block */
    free(cur);
    return 1;
}

long long cso_blocked_ell_from_coo(uint32_t rows, uint32_t cols, uint32_t nnz, const uint32_t *row,
                                   const uint32_t *col, const uint16_t *val, const uint32_t *map, uint32_t B,
                                   uint32_t *bci, uint16_t *out_val, uint64_t *nnz_out, uint64_t *total_blocks) {
    const uint32_t RB = (uint32_t) (((uint64_t) rows + B - 1u) / B);
    for (uint32_t i = 0; i < nnz; ++i)
        if (row[i] >= rows) return -1;
    uint32_t *off = (uint32_t *) malloc(((size_t) RB + 1u) * sizeof(uint32_t));
    uint32_t *start = (uint32_t *) malloc(((size_t) RB + 1u) * sizeof(uint32_t));
    uint32_t *bc = (uint32_t *) malloc(((size_t) nnz + 1u) * sizeof(uint32_t));
    uint32_t W = 0u;
    uint64_t tot = 0u;
    if (!off || !start || !bc || !coo_block_cols(rows, nnz, row, col, map, B, off, bc, &W, &tot)) {
        free(off);
        free(start);
        free(bc);
        return -1;
    }
    /* recover each row block's start in bc: the counting pass order */
    {
        uint32_t *cnt = (uint32_t *) calloc((size_t) RB + 1u, sizeof(uint32_t));
        for (uint32_t i = 0; i < nnz; ++i) ++cnt[row[i] / B + 1u];
        for (uint32_t rb = 0; rb < RB; ++rb) cnt[rb + 1u] += cnt[rb];
        memcpy(start, cnt, ((size_t) RB + 1u) * sizeof(uint32_t));
        free(cnt);
    }
    const size_t ell = (size_t) W * B;
    if (bci != NULL)
        for (size_t i = 0; i < (size_t) RB * W; ++i) bci[i] = CSO_INVALID;
    if (out_val != NULL) memset(out_val, 0, (size_t) rows * ell * sizeof(uint16_t));
    for (uint32_t rb = 0; rb < RB && bci != NULL; ++rb)
        for (uint32_t s = 0; s < off[rb]; ++s) bci[(size_t) rb * W + s] = bc[start[rb] + s];
    uint64_t nz_all = 0u, nz_in = 0u;
    for (uint32_t i = 0; i < nnz && out_val != NULL; ++i) {
        const uint32_t c = coo_col(col, map, i), rb = row[i] / B, b = c / B;
        /* binary search of the block column among the row block's slots */
        uint32_t lo = 0u, hi = off[rb], slot = 0u;
        while (lo < hi) {
            const uint32_t mid = lo + (hi - lo) / 2u;
            if (bc[start[rb] + mid] < b)
                lo = mid + 1u;
            else
                hi = mid;
        }
        slot = lo;
        uint16_t *dst = out_val + (size_t) row[i] * ell + (size_t) slot * B + c % B;
        const int prev = half_nonzero(*dst), next = half_nonzero(val[i]);
        const int in = c < cols;
        nz_all += (uint64_t) (next - prev);
        if (in) nz_in += (uint64_t) (next - prev);
        *dst = val[i];
    }
    if (nnz_out != NULL) {
        nnz_out[0] = nz_all;
        nnz_out[1] = nz_in;
    }
    if (total_blocks != NULL) *total_blocks = tot;
    free(off);
    free(start);
    free(bc);
    return W;
}

/* width and total blocks for one candidate (the chooser's inputs) */
int cso_coo_block_shape(uint32_t rows, uint32_t nnz, const uint32_t *row, const uint32_t *col, const uint32_t *map,
                        uint32_t B, uint32_t *width, uint64_t *total_blocks) {
    const uint32_t RB = (uint32_t) (((uint64_t) rows + B - 1u) / B);
    uint32_t *off = (uint32_t *) malloc(((size_t) RB + 1u) * sizeof(uint32_t));
    uint32_t *bc = (uint32_t *) malloc(((size_t) nnz + 1u) * sizeof(uint32_t));
    int ok = off && bc && coo_block_cols(rows, nnz, row, col, map, B, off, bc, width, total_blocks);
    free(off);
    free(bc);
    return ok;
}
