/*
 * oracle.c -- CPU restatement of ThermoFEM's sparse solve path.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle the CUDA path is tested against; see oracle.h).
 * Reference citations are paths inside the Mgepahmge/ThermoFEM project.
 */
#include "oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

void or_free(void *p) { free(p); }

void or_csr_free(or_csr *a) {
    if (!a) return;
    free(a->offsets);
    free(a->indices);
    free(a->values);
    a->offsets = NULL;
    a->indices = NULL;
    a->values = NULL;
}

int or_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* Coordinate compression: stable sort by (row, column) and a left-to-right  */
/* reduction of equal coordinates.  Restates the host oracle's compress()    */
/* (test/support/NativeAggregationOracle.cu:52-86): std::stable_sort by      */
/* (row, column), then sum or max in sorted order, keeping explicit zeros.   */
/* Two stable counting sorts (by column, then by row) give the same order.   */
/* ------------------------------------------------------------------------ */
static int compress(int n, int64_t m, const int *row, const int *col, const double *val, int maximum, or_csr *out) {
    memset(out, 0, sizeof(*out));
    out->rows = out->cols = n;
    int64_t *count = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
    int64_t *perm1 = (int64_t *)malloc(sizeof(int64_t) * (size_t)(m ? m : 1));
    int64_t *perm2 = (int64_t *)malloc(sizeof(int64_t) * (size_t)(m ? m : 1));
    out->offsets = (int *)calloc((size_t)n + 1, sizeof(int));
    if (!count || !perm1 || !perm2 || !out->offsets) {
        free(count); free(perm1); free(perm2); or_csr_free(out);
        return OR_LENGTH;
    }
    /* pass 1: stable by column */
    for (int64_t e = 0; e < m; ++e) count[col[e] + 1]++;
    for (int c = 0; c < n; ++c) count[c + 1] += count[c];
    for (int64_t e = 0; e < m; ++e) perm1[count[col[e]]++] = e;
    /* pass 2: stable by row */
    memset(count, 0, sizeof(int64_t) * ((size_t)n + 1));
    for (int64_t e = 0; e < m; ++e) count[row[e] + 1]++;
    for (int r = 0; r < n; ++r) count[r + 1] += count[r];
    for (int64_t k = 0; k < m; ++k) {
        int64_t e = perm1[k];
        perm2[count[row[e]]++] = e;
    }
    free(perm1);
    free(count);
    /* reduce */
    out->indices = (int *)malloc(sizeof(int) * (size_t)(m ? m : 1));
    out->values = (double *)malloc(sizeof(double) * (size_t)(m ? m : 1));
    if (!out->indices || !out->values) {
        free(perm2); or_csr_free(out);
        return OR_LENGTH;
    }
    int64_t u = 0;
    int prevRow = -1, prevCol = -1;
    int status = OR_OK;
    for (int64_t k = 0; k < m; ++k) {
        int64_t e = perm2[k];
        if (row[e] == prevRow && col[e] == prevCol) {
            double *v = &out->values[u - 1];
            *v = maximum ? (*v > val[e] ? *v : val[e]) : *v + val[e];
            if (!isfinite(*v)) status = OR_NONFINITE;
        } else {
            out->indices[u] = col[e];
            out->values[u] = val[e];
            out->offsets[row[e] + 1]++;
            ++u;
            prevRow = row[e];
            prevCol = col[e];
        }
    }
    free(perm2);
    for (int r = 0; r < n; ++r) out->offsets[r + 1] += out->offsets[r];
    out->nnz = u;
    if (status != OR_OK) or_csr_free(out);
    return status;
}

/* Structural validation of a host CSR (NativeAggregationOracle.cu:27-46). */
static int validate_csr(int n, const int *rp, const int *ci, const double *v, int64_t nnz) {
    if (n < 1 || !rp || rp[0] != 0 || rp[n] != nnz) return OR_INVALID;
    for (int r = 0; r < n; ++r)
        if (rp[r] < 0 || rp[r] > rp[r + 1]) return OR_INVALID;
    for (int64_t j = 0; j < nnz; ++j)
        if (ci[j] < 0 || ci[j] >= n || !isfinite(v[j])) return OR_INVALID;
    return OR_OK;
}

static int entries_of(const or_csr *a, const int *map, int **row, int **col, double **val, int64_t *m,
                      int skip_intra_nonpositive) {
    int64_t cap = a->nnz ? a->nnz : 1;
    *row = (int *)malloc(sizeof(int) * (size_t)cap);
    *col = (int *)malloc(sizeof(int) * (size_t)cap);
    *val = (double *)malloc(sizeof(double) * (size_t)cap);
    if (!*row || !*col || !*val) return OR_LENGTH;
    int64_t k = 0;
    for (int r = 0; r < a->rows; ++r) {
        for (int j = a->offsets[r]; j < a->offsets[r + 1]; ++j) {
            int rr = map ? map[r] : r, cc = map ? map[a->indices[j]] : a->indices[j];
            if (skip_intra_nonpositive && (rr == cc || !(a->values[j] > 0))) continue;
            (*row)[k] = rr;
            (*col)[k] = cc;
            (*val)[k] = a->values[j];
            ++k;
        }
    }
    *m = k;
    return OR_OK;
}

/* Canonical CSR: sort and sum duplicates, keep explicit zeros
 * (GpuAggregation.cu:991-1007 -> galerkin with a null map; oracle :119-129). */
int or_canonical(int n, const int *rp, const int *ci, const double *v, int64_t nnz, or_csr *out) {
    int s = validate_csr(n, rp, ci, v, nnz);
    if (s) return s;
    or_csr in = {n, n, nnz, (int *)rp, (int *)ci, (double *)v};
    int *row, *col;
    double *val;
    int64_t m;
    s = entries_of(&in, NULL, &row, &col, &val, &m, 0);
    if (!s) s = compress(n, m, row, col, val, 0, out);
    free(row); free(col); free(val);
    return s;
}

/* Row validation and row max |offdiag| (GpuAggregation.cu:247-271):
 * nonfinite entries, zero diagonal or nonfinite reciprocal fail. */
int or_validate(const or_csr *a, double *row_max) {
    int bad = 0;
    for (int i = 0; i < a->rows; ++i) {
        double diag = 0, mx = 0;
        for (int j = a->offsets[i]; j < a->offsets[i + 1]; ++j) {
            if (!isfinite(a->values[j])) bad = 1;
            if (a->indices[j] == i) diag = a->values[j];
            else mx = fmax(mx, fabs(a->values[j]));
        }
        if (diag == 0 || !isfinite(diag) || !isfinite(1.0 / diag)) bad = 1;
        if (row_max) row_max[i] = mx;
    }
    return bad ? OR_INVALID : OR_OK;
}

/* Symmetric strength graph, max-merged (GpuAggregation.cu:339-390;
 * oracle :130-159).  Edge weight |a_ij|/max_k|a_ik| kept when > 0 and >= theta. */
int or_strength(const or_csr *a, double theta, or_csr *graph) {
    if (!isfinite(theta) || theta < 0 || theta > 1) return OR_INVALID;
    int s = validate_csr(a->rows, a->offsets, a->indices, a->values, a->nnz);
    if (s) return s;
    int64_t cap = 2 * (a->nnz ? a->nnz : 1);
    int *row = (int *)malloc(sizeof(int) * (size_t)cap), *col = (int *)malloc(sizeof(int) * (size_t)cap);
    double *val = (double *)malloc(sizeof(double) * (size_t)cap);
    int64_t m = 0;
    for (int r = 0; r < a->rows; ++r) {
        double mx = 0;
        for (int j = a->offsets[r]; j < a->offsets[r + 1]; ++j)
            if (a->indices[j] != r) mx = fmax(mx, fabs(a->values[j]));
        if (mx == 0) continue;
        for (int j = a->offsets[r]; j < a->offsets[r + 1]; ++j) {
            int c = a->indices[j];
            double w = fabs(a->values[j]) / mx;
            if (c != r && w > 0 && w >= theta) {
                row[m] = r; col[m] = c; val[m] = w; ++m;
                row[m] = c; col[m] = r; val[m] = w; ++m;
            }
        }
    }
    s = compress(a->rows, m, row, col, val, 1, graph);
    free(row); free(col); free(val);
    return s;
}

/* Symmetric edge priority used to break equal weights
 * (GpuAggregation.cu:49-54; oracle :107-113): splitmix64 finaliser of
 * (min << 32 | max). */
static uint64_t edge_priority(int i, int j) {
    uint64_t lo = (uint64_t)(unsigned)(i < j ? i : j), hi = (uint64_t)(unsigned)(i < j ? j : i);
    uint64_t h = (lo << 32) | hi;
    h = (h ^ (h >> 30)) * 0xbf58476d1ce4e5b9ULL;
    h = (h ^ (h >> 27)) * 0x94d049bb133111ebULL;
    return h ^ (h >> 31);
}

/* Synchronous handshake matching (GpuAggregation.cu:402-505; oracle :160-205).
 * Each round: every unmatched vertex proposes to its unmatched neighbour of
 * largest weight (ties: larger edge priority, then smaller id) from one
 * snapshot; mutual proposals become pairs.  Roots (unmatched or smaller end)
 * get consecutive ids by an exclusive prefix sum. */
int or_match_pairs(const or_csr *g, int rounds, int *map, int *count) {
    if (rounds < 1 || rounds > 8) return OR_INVALID;
    int n = g->rows;
    int *mate = (int *)malloc(sizeof(int) * (size_t)n), *proposal = (int *)malloc(sizeof(int) * (size_t)n);
    int *prefix = (int *)malloc(sizeof(int) * ((size_t)n + 1));
    for (int i = 0; i < n; ++i) mate[i] = proposal[i] = -1;
    for (int round = 0; round < rounds; ++round) {
        for (int i = 0; i < n; ++i) {
            int best = -1;
            double score = 0;
            uint64_t priority = 0;
            if (mate[i] < 0) {
                for (int j = g->offsets[i]; j < g->offsets[i + 1]; ++j) {
                    int c = g->indices[j];
                    double w = g->values[j];
                    if (c == i || mate[c] >= 0 || w <= 0 || w < score) continue;
                    uint64_t cand = edge_priority(i, c);
                    if (w > score || (w == score && (best < 0 || cand > priority || (cand == priority && c < best)))) {
                        best = c;
                        score = w;
                        priority = cand;
                    }
                }
            }
            proposal[i] = best;
        }
        for (int i = 0; i < n; ++i)
            if (proposal[i] >= 0 && proposal[proposal[i]] == i) mate[i] = proposal[i];
    }
    prefix[0] = 0;
    for (int i = 0; i < n; ++i) prefix[i + 1] = prefix[i] + ((mate[i] < 0 || i < mate[i]) ? 1 : 0);
    for (int i = 0; i < n; ++i) map[i] = prefix[mate[i] < 0 ? i : (i < mate[i] ? i : mate[i])];
    *count = prefix[n];
    free(mate); free(proposal); free(prefix);
    return OR_OK;
}

/* Graph quotient by map, intra-aggregate edges dropped, parallel edges
 * max-merged (GpuAggregation.cu:534-576; oracle :206-219). */
int or_contract(const or_csr *g, const int *map, int count, or_csr *out) {
    int *row, *col;
    double *val;
    int64_t m;
    int s = entries_of(g, map, &row, &col, &val, &m, 1);
    if (!s) s = compress(count, m, row, col, val, 1, out);
    free(row); free(col); free(val);
    return s;
}

/* Two-stage matching, composition and two rounds of singleton absorption
 * (GpuAggregation.cu:766-818; oracle :220-298). */
int or_aggregate(const or_csr *g, int rounds, int absorb, int *map, int *offsets, int *members, int *coarse,
                 int64_t hist[4]) {
    int n = g->rows, first = 0, second_count = 0;
    int s = or_match_pairs(g, rounds, map, &first);
    if (s) return s;
    or_csr contracted;
    s = or_contract(g, map, first, &contracted);
    if (s) return s;
    int *second = (int *)malloc(sizeof(int) * (size_t)(first ? first : 1));
    s = or_match_pairs(&contracted, rounds, second, &second_count);
    or_csr_free(&contracted);
    if (s) { free(second); return s; }
    for (int i = 0; i < n; ++i) map[i] = second[map[i]];
    free(second);
    int count = second_count;
    int *sizes = (int *)calloc((size_t)count + 1, sizeof(int));
    int *slots = (int *)malloc(sizeof(int) * 4 * (size_t)(count ? count : 1));
    int *proposal = (int *)malloc(sizeof(int) * (size_t)n);
    double *scores = (double *)malloc(sizeof(double) * (size_t)n);
    int *next = (int *)malloc(sizeof(int) * (size_t)n);
#define REBUILD_MEMBERS()                                                        \
    do {                                                                         \
        memset(sizes, 0, sizeof(int) * ((size_t)count + 1));                     \
        for (int i_ = 0; i_ < n; ++i_) {                                         \
            int c_ = map[i_];                                                    \
            if (sizes[c_] >= 4) { s = OR_LENGTH; break; }                        \
            slots[(size_t)c_ * 4 + sizes[c_]++] = i_;                            \
        }                                                                        \
    } while (0)
    REBUILD_MEMBERS(); /* ascending member order by construction */
    if (absorb && !s) {
        for (int round = 0; round < 2 && !s; ++round) {
            /* proposals from the pre-round snapshot */
            for (int i = 0; i < n; ++i) {
                proposal[i] = -1;
                scores[i] = 0;
                if (sizes[map[i]] != 1) continue;
                for (int j = g->offsets[i]; j < g->offsets[i + 1]; ++j) {
                    int c = map[g->indices[j]];
                    double w = g->values[j];
                    if (sizes[c] < 2 || sizes[c] >= 4 || w <= 0) continue;
                    if (w > scores[i] || (w == scores[i] && (proposal[i] < 0 || c < proposal[i]))) {
                        proposal[i] = c;
                        scores[i] = w;
                    }
                }
            }
            memcpy(next, map, sizeof(int) * (size_t)n);
            /* each target keeps its best (weight desc, id asc) distinct proposers
             * up to its remaining capacity */
            for (int c = 0; c < count; ++c) {
                if (sizes[c] < 2 || sizes[c] >= 4) continue;
                int cap = 4 - sizes[c];
                int sel[2] = {-1, -1};
                double sw[2] = {-1, -1};
                for (int k = 0; k < sizes[c]; ++k) {
                    int r = slots[(size_t)c * 4 + k];
                    for (int j = g->offsets[r]; j < g->offsets[r + 1]; ++j) {
                        int i = g->indices[j];
                        if (proposal[i] != c || i == sel[0] || i == sel[1]) continue;
                        double w = scores[i];
                        for (int q = 0; q < cap; ++q) {
                            if (w > sw[q] || (w == sw[q] && i < sel[q])) {
                                for (int t = cap - 1; t > q; --t) { sel[t] = sel[t - 1]; sw[t] = sw[t - 1]; }
                                sel[q] = i;
                                sw[q] = w;
                                break;
                            }
                        }
                    }
                }
                for (int q = 0; q < cap; ++q)
                    if (sel[q] >= 0) next[sel[q]] = c;
            }
            memcpy(map, next, sizeof(int) * (size_t)n);
            REBUILD_MEMBERS();
        }
    }
    if (!s) {
        /* compact empty ids; member CSR in ascending fine order; histogram */
        int *compact = (int *)malloc(sizeof(int) * (size_t)(count ? count : 1));
        int used = 0;
        for (int c = 0; c < count; ++c) compact[c] = sizes[c] ? used++ : -1;
        for (int i = 0; i < n; ++i) map[i] = compact[map[i]];
        hist[0] = hist[1] = hist[2] = hist[3] = 0;
        offsets[0] = 0;
        int pos = 0;
        for (int c = 0; c < count; ++c) {
            if (!sizes[c]) continue;
            hist[sizes[c] - 1]++;
            for (int k = 0; k < sizes[c]; ++k) members[pos++] = slots[(size_t)c * 4 + k];
            offsets[compact[c] + 1] = pos;
        }
        *coarse = used;
        free(compact);
    }
#undef REBUILD_MEMBERS
    free(sizes); free(slots); free(proposal); free(scores); free(next);
    return s;
}

/* Ac = P^T A P by coordinate mapping and sum (GpuAggregation.cu:136-234;
 * oracle :299-317); nnz(Ac) <= nnz(A), merged zeros kept. */
int or_galerkin(const or_csr *a, const int *map, int coarse, or_csr *out) {
    int *row, *col;
    double *val;
    int64_t m;
    int s = entries_of(a, map, &row, &col, &val, &m, 0);
    if (!s) s = compress(coarse, m, row, col, val, 0, out);
    free(row); free(col); free(val);
    return s;
}

/* Dense partial-pivot LU (GpuAggregation.cu:827-893): full-row swaps,
 * pivot = first largest |m[i][k]|, singular when the pivot is nonfinite or
 * <= 64 * DBL_EPSILON * max|A|. */
int or_lu_factor(const or_csr *a, double *m, int *pivots) {
    int n = a->rows;
    double scale = 0;
    memset(m, 0, sizeof(double) * (size_t)n * (size_t)n);
    for (int r = 0; r < n; ++r)
        for (int j = a->offsets[r]; j < a->offsets[r + 1]; ++j) {
            m[(size_t)r * n + a->indices[j]] = a->values[j];
            scale = fmax(scale, fabs(a->values[j]));
        }
    for (int k = 0; k < n; ++k) {
        int p = k;
        for (int i = k + 1; i < n; ++i)
            if (fabs(m[(size_t)i * n + k]) > fabs(m[(size_t)p * n + k])) p = i;
        double piv = m[(size_t)p * n + k];
        if (!isfinite(piv) || fabs(piv) <= 64 * DBL_EPSILON * scale) return 0;
        pivots[k] = p;
        if (p != k)
            for (int j = 0; j < n; ++j) {
                double t = m[(size_t)p * n + j];
                m[(size_t)p * n + j] = m[(size_t)k * n + j];
                m[(size_t)k * n + j] = t;
            }
        for (int r = k + 1; r < n; ++r) {
            m[(size_t)r * n + k] /= m[(size_t)k * n + k];
            for (int j = k + 1; j < n; ++j) m[(size_t)r * n + j] -= m[(size_t)r * n + k] * m[(size_t)k * n + j];
        }
    }
    for (size_t i = 0; i < (size_t)n * n; ++i)
        if (!isfinite(m[i])) return 0;
    return 1;
}

/* Pivot permutation, then column-oriented forward and back substitution
 * (GpuAggregation.cu:904-939); b and x may alias. */
void or_lu_solve(int n, const double *lu, const int *pivots, const double *b, double *x) {
    double *v = (double *)malloc(sizeof(double) * (size_t)n);
    memcpy(v, b, sizeof(double) * (size_t)n);
    for (int k = 0; k < n; ++k) {
        double t = v[k];
        v[k] = v[pivots[k]];
        v[pivots[k]] = t;
    }
    for (int k = 0; k < n; ++k)
        for (int r = k + 1; r < n; ++r) v[r] -= lu[(size_t)r * n + k] * v[k];
    for (int k = n - 1; k >= 0; --k) {
        v[k] /= lu[(size_t)k * n + k];
        for (int r = 0; r < k; ++r) v[r] -= lu[(size_t)r * n + k] * v[k];
    }
    memcpy(x, v, sizeof(double) * (size_t)n);
    free(v);
}

/* ------------------------------------------------------------------------ */
/* Iteration kernels (IterationContext.cu:140-269), OpenMP over rows.        */
/* ------------------------------------------------------------------------ */
void or_spmv(const or_csr *a, const double *x, double *y) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < a->rows; ++i) {
        double s = 0;
        for (int j = a->offsets[i]; j < a->offsets[i + 1]; ++j) s += a->values[j] * x[a->indices[j]];
        y[i] = s;
    }
}

/* Fixed partition: chunks of 4096 entries summed left to right, then the
 * chunk sums left to right, so the value does not depend on the number of
 * threads (an OpenMP reduction clause would make it depend on the host). */
#define OR_DOT_CHUNK 4096
double or_dot(int64_t n, const double *x, const double *y) {
    const int64_t chunks = (n + OR_DOT_CHUNK - 1) / OR_DOT_CHUNK;
    double local[64];
    double *part = chunks <= 64 ? local : (double *)malloc(sizeof(double) * (size_t)chunks);
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < chunks; ++c) {
        const int64_t e = (c + 1) * OR_DOT_CHUNK < n ? (c + 1) * OR_DOT_CHUNK : n;
        double s = 0;
        for (int64_t i = c * OR_DOT_CHUNK; i < e; ++i) s += x[i] * y[i];
        part[c] = s;
    }
    double s = 0;
    for (int64_t c = 0; c < chunks; ++c) s += part[c];
    if (part != local) free(part);
    return s;
}

double or_norm(int64_t n, const double *x) { return sqrt(or_dot(n, x, x)); }

static void residual(const or_csr *a, const double *b, const double *x, double *r) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < a->rows; ++i) {
        double s = 0;
        for (int j = a->offsets[i]; j < a->offsets[i + 1]; ++j) s += a->values[j] * x[a->indices[j]];
        r[i] = b[i] - s;
    }
}

/* Jacobi sweeps x += w * Dinv * (b - A x) (Jacobi.cuh:60-74,
 * IterationContext.cu:26-32); Dinv from the summed diagonal (Diagonal.cuh). */
static void jacobi_sweeps(const or_csr *a, const double *inv, int sweeps, double w, const double *b, double *x,
                          double *tmp) {
    for (int s = 0; s < sweeps; ++s) {
        or_spmv(a, x, tmp);
#pragma omp parallel for schedule(static)
        for (int i = 0; i < a->rows; ++i) x[i] += w * inv[i] * (b[i] - tmp[i]);
    }
}

static int inverse_diagonal(const or_csr *a, double *inv) {
    for (int i = 0; i < a->rows; ++i) {
        double d = 0;
        for (int j = a->offsets[i]; j < a->offsets[i + 1]; ++j)
            if (a->indices[j] == i) d += a->values[j];
        if (!isfinite(d) || d == 0 || !isfinite(1.0 / d)) return OR_INVALID;
        inv[i] = 1.0 / d;
    }
    return OR_OK;
}

int or_jacobi(const or_csr *a, int sweeps, double weight, const double *b, double *x) {
    double *inv = (double *)malloc(sizeof(double) * (size_t)a->rows);
    double *tmp = (double *)malloc(sizeof(double) * (size_t)a->rows);
    double *rhs = (double *)malloc(sizeof(double) * (size_t)a->rows);
    memcpy(rhs, b, sizeof(double) * (size_t)a->rows);
    int s = inverse_diagonal(a, inv);
    if (!s) jacobi_sweeps(a, inv, sweeps, weight, rhs, x, tmp);
    free(inv); free(tmp); free(rhs);
    return s;
}

/* ------------------------------------------------------------------------ */
/* AMG hierarchy (Amg.cuh:81-143) and cycle (Cycle.cuh:35-63,               */
/* Amg.cuh:197-257).                                                        */
/* ------------------------------------------------------------------------ */
typedef struct {
    or_csr a;
    double *inv;
    double *rhs, *x, *r, *tmp;
    int *map, *offsets, *members; /* transfer to the next level (NULL on the last) */
    int coarse;
    int64_t hist[4];
} or_level;

struct or_amg {
    or_amg_options opt;
    int nlev;
    or_level *lev;
    double *lu;
    int *pivots;
    int factored;
    const char *stop, *coarse_solver;
    int64_t *visits;
};

static void level_free(or_level *l) {
    or_csr_free(&l->a);
    free(l->inv); free(l->rhs); free(l->x); free(l->r); free(l->tmp);
    free(l->map); free(l->offsets); free(l->members);
}

void or_amg_free(or_amg *m) {
    if (!m) return;
    for (int d = 0; d < m->nlev; ++d) level_free(&m->lev[d]);
    free(m->lev); free(m->lu); free(m->pivots); free(m->visits);
    free(m);
}

or_amg *or_amg_setup(const or_csr *input, const or_amg_options *opt, int *status) {
    *status = OR_OK;
    if (opt->max_levels < 1 || opt->max_levels > 20 || opt->coarse_rows < 1 || opt->matching_rounds < 1 ||
        opt->matching_rounds > 8 || opt->pre_sweeps < 0 || opt->post_sweeps < 0 || opt->coarse_sweeps < 1 ||
        !(opt->jacobi_weight > 0 && opt->jacobi_weight < 2) ||
        !(opt->strength_threshold >= 0 && opt->strength_threshold <= 1) || opt->cycle < 0 || opt->cycle > 2) {
        *status = OR_INVALID;
        return NULL;
    }
    or_amg *m = (or_amg *)calloc(1, sizeof(or_amg));
    m->opt = *opt;
    m->lev = (or_level *)calloc(21, sizeof(or_level));
    or_csr native;
    int s = or_canonical(input->rows, input->offsets, input->indices, input->values, input->nnz, &native);
    if (s) { *status = s; or_amg_free(m); return NULL; }
    for (int depth = 0;; ++depth) {
        or_level *l = &m->lev[m->nlev++];
        l->a = native;
        int n = native.rows;
        s = or_validate(&native, NULL);
        l->inv = (double *)malloc(sizeof(double) * (size_t)n);
        if (!s) s = inverse_diagonal(&native, l->inv);
        if (s) { *status = s; or_amg_free(m); return NULL; }
        l->rhs = (double *)calloc((size_t)n, sizeof(double));
        l->x = (double *)calloc((size_t)n, sizeof(double));
        l->r = (double *)calloc((size_t)n, sizeof(double));
        l->tmp = (double *)calloc((size_t)n, sizeof(double));
        if (n <= opt->coarse_rows) { m->stop = "coarse size"; break; }
        if (depth + 1 == opt->max_levels) { m->stop = "level limit"; break; }
        or_csr g;
        s = or_strength(&native, opt->strength_threshold, &g);
        if (s) { *status = s; or_amg_free(m); return NULL; }
        if (g.nnz == 0) { or_csr_free(&g); m->stop = "empty strength graph"; break; }
        l->map = (int *)malloc(sizeof(int) * (size_t)n);
        l->offsets = (int *)malloc(sizeof(int) * ((size_t)n + 1));
        l->members = (int *)malloc(sizeof(int) * (size_t)n);
        s = or_aggregate(&g, opt->matching_rounds, opt->absorb_singletons, l->map, l->offsets, l->members, &l->coarse,
                         l->hist);
        or_csr_free(&g);
        if (s) { *status = s; or_amg_free(m); return NULL; }
        if (l->coarse >= n) {
            free(l->map); free(l->offsets); free(l->members);
            l->map = l->offsets = l->members = NULL;
            memset(l->hist, 0, sizeof(l->hist));
            m->stop = "no contraction";
            break;
        }
        or_csr coarse;
        s = or_galerkin(&native, l->map, l->coarse, &coarse);
        if (s) { *status = s; or_amg_free(m); return NULL; }
        native = coarse;
    }
    or_level *last = &m->lev[m->nlev - 1];
    int lu_rows = opt->coarse_lu_rows > 0 ? opt->coarse_lu_rows : 64;
    int singular = 0;
    if (last->a.rows <= lu_rows) {
        m->lu = (double *)malloc(sizeof(double) * (size_t)last->a.rows * (size_t)last->a.rows);
        m->pivots = (int *)malloc(sizeof(int) * (size_t)last->a.rows);
        m->factored = or_lu_factor(&last->a, m->lu, m->pivots);
        singular = !m->factored;
    }
    m->coarse_solver = m->factored ? "pivoted GPU LU" : (singular ? "Jacobi (singular LU)" : "Jacobi (coarsening stopped)");
    m->visits = (int64_t *)calloc((size_t)m->nlev, sizeof(int64_t));
    return m;
}

int or_amg_levels(const or_amg *m) { return m->nlev; }
void or_amg_level_info(const or_amg *m, int d, int64_t *rows, int64_t *nnz, int64_t hist[4]) {
    *rows = m->lev[d].a.rows;
    *nnz = m->lev[d].a.nnz;
    for (int k = 0; k < 4; ++k) hist[k] = m->lev[d].hist[k];
}
const char *or_amg_stop_reason(const or_amg *m) { return m->stop; }
const char *or_amg_coarse_solver(const or_amg *m) { return m->coarse_solver; }
const int *or_amg_map(const or_amg *m, int d) { return m->lev[d].map; }
const or_csr *or_amg_matrix(const or_amg *m, int d) { return &m->lev[d].a; }

static void restrict_sum(const or_level *l, const double *fine, double *coarse) {
#pragma omp parallel for schedule(static)
    for (int c = 0; c < l->coarse; ++c) {
        double s = 0;
        for (int j = l->offsets[c]; j < l->offsets[c + 1]; ++j) s += fine[l->members[j]];
        coarse[c] = s;
    }
}

static void cycle(or_amg *m, int kind, int d, int zero) {
    or_level *l = &m->lev[d];
    int n = l->a.rows;
    m->visits[d]++;
    if (zero || kind == 2) memset(l->x, 0, sizeof(double) * (size_t)n);
    if (d + 1 == m->nlev) {
        if (m->factored) or_lu_solve(n, m->lu, m->pivots, l->rhs, l->x);
        else jacobi_sweeps(&l->a, l->inv, m->opt.coarse_sweeps, m->opt.jacobi_weight, l->rhs, l->x, l->tmp);
        return;
    }
    or_level *c = &m->lev[d + 1];
    if (kind == 2) {
        restrict_sum(l, l->rhs, c->rhs);
        cycle(m, 2, d + 1, 1);
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) l->x[i] += c->x[l->map[i]];
        cycle(m, 0, d, 0);
        return;
    }
    jacobi_sweeps(&l->a, l->inv, m->opt.pre_sweeps, m->opt.jacobi_weight, l->rhs, l->x, l->tmp);
    residual(&l->a, l->rhs, l->x, l->r);
    restrict_sum(l, l->r, c->rhs);
    cycle(m, kind, d + 1, 1);
    if (kind == 1) cycle(m, kind, d + 1, 0);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) l->x[i] += c->x[l->map[i]];
    jacobi_sweeps(&l->a, l->inv, m->opt.post_sweeps, m->opt.jacobi_weight, l->rhs, l->x, l->tmp);
}

void or_amg_apply(or_amg *m, const double *rhs, double *x, int64_t *visits) {
    memcpy(m->lev[0].rhs, rhs, sizeof(double) * (size_t)m->lev[0].a.rows);
    memset(m->visits, 0, sizeof(int64_t) * (size_t)m->nlev);
    cycle(m, m->opt.cycle, 0, 1);
    memcpy(x, m->lev[0].x, sizeof(double) * (size_t)m->lev[0].a.rows);
    if (visits) memcpy(visits, m->visits, sizeof(int64_t) * (size_t)m->nlev);
}

/* ------------------------------------------------------------------------ */
/* Krylov solvers.                                                           */
/* ------------------------------------------------------------------------ */
static void precond(or_amg *m, int64_t n, const double *r, double *z) {
    if (m) or_amg_apply(m, r, z, NULL);
    else memcpy(z, r, sizeof(double) * (size_t)n);
}

static void axpy(int64_t n, double a, const double *x, double *y) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) y[i] += a * x[i];
}

static void scale(int64_t n, double a, double *x) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) x[i] *= a;
}

/* Final report from the true residual (Cg.cuh:105-121, BiCgStab.cuh:122-136). */
static or_solve_result finish(const or_csr *a, const double *b, const double *x, double *r, int status, int it,
                              double normB, double tol) {
    residual(a, b, x, r);
    double res = or_norm(a->rows, r);
    if (!isfinite(res) || !isfinite(normB)) status = 3;
    else if (res <= tol) status = 0;
    else if (status == 0) status = 1;
    or_solve_result out = {status, it, res, normB > 0 ? res / normB : res};
    return out;
}

or_solve_result or_cg(const or_csr *a, or_amg *M, const double *b, double *x, const or_solver_options *o) {
    int64_t n = a->rows;
    double *r = (double *)malloc(sizeof(double) * (size_t)n), *z = (double *)malloc(sizeof(double) * (size_t)n);
    double *p = (double *)malloc(sizeof(double) * (size_t)n), *ap = (double *)malloc(sizeof(double) * (size_t)n);
    double normB = or_norm(n, b);
    double tol = fmax(o->absolute_tolerance, o->relative_tolerance * normB);
    or_solve_result out;
    residual(a, b, x, r);
    double res = or_norm(n, r);
    if (!isfinite(normB) || !isfinite(res)) { out = finish(a, b, x, r, 3, 0, normB, tol); goto done; }
    if (res <= tol) { out = finish(a, b, x, r, 0, 0, normB, tol); goto done; }
    double prevRho = 0;
    int fresh = 1;
    for (int k = 0; k < o->max_iterations; ++k) {
        int it = k + 1;
        precond(M, n, r, z);
        double rho = or_dot(n, r, z);
        if (!isfinite(rho)) { out = finish(a, b, x, r, 3, it, normB, tol); goto done; }
        if (rho <= 0) { out = finish(a, b, x, r, 2, it, normB, tol); goto done; }
        if (fresh) {
            memcpy(p, z, sizeof(double) * (size_t)n);
            fresh = 0;
        } else {
            double beta = rho / prevRho;
            if (!isfinite(beta)) { out = finish(a, b, x, r, 3, it, normB, tol); goto done; }
            scale(n, beta, p);
            axpy(n, 1.0, z, p);
        }
        or_spmv(a, p, ap);
        double curv = or_dot(n, p, ap);
        if (!isfinite(curv)) { out = finish(a, b, x, r, 3, it, normB, tol); goto done; }
        if (curv <= 0) { out = finish(a, b, x, r, 2, it, normB, tol); goto done; }
        double alpha = rho / curv;
        if (!isfinite(alpha)) { out = finish(a, b, x, r, 3, it, normB, tol); goto done; }
        axpy(n, alpha, p, x);
        axpy(n, -alpha, ap, r);
        res = or_norm(n, r);
        if (!isfinite(res)) { out = finish(a, b, x, r, 3, it, normB, tol); goto done; }
        if (res <= tol || it % o->refresh_interval == 0) {
            residual(a, b, x, r);
            res = or_norm(n, r);
            if (!isfinite(res) || res <= tol) { out = finish(a, b, x, r, 1, it, normB, tol); goto done; }
            fresh = 1;
        }
        prevRho = rho;
    }
    out = finish(a, b, x, r, 1, o->max_iterations, normB, tol);
done:
    free(r); free(z); free(p); free(ap);
    return out;
}

or_solve_result or_bicgstab(const or_csr *a, or_amg *M, const double *b, double *x, const or_solver_options *o) {
    int64_t n = a->rows;
    size_t bytes = sizeof(double) * (size_t)n;
    double *r = (double *)malloc(bytes), *sh = (double *)malloc(bytes), *p = (double *)malloc(bytes);
    double *v = (double *)malloc(bytes), *s = (double *)malloc(bytes), *t = (double *)malloc(bytes);
    double *ph = (double *)malloc(bytes), *shat = (double *)malloc(bytes);
    double normB = or_norm(n, b);
    double tol = fmax(o->absolute_tolerance, o->relative_tolerance * normB);
    or_solve_result out;
    residual(a, b, x, r);
    double res = or_norm(n, r);
    if (!isfinite(normB) || !isfinite(res)) { out = finish(a, b, x, r, 3, 0, normB, tol); goto done; }
    if (res <= tol) { out = finish(a, b, x, r, 0, 0, normB, tol); goto done; }
    memcpy(sh, r, bytes);
    double rhoPrev = 1, alpha = 1, omega = 1;
    int fresh = 1;
    for (int k = 0; k < o->max_iterations; ++k) {
        int it = k + 1;
        double rho = or_dot(n, sh, r);
        if (!isfinite(rho)) { out = finish(a, b, x, r, 3, it, normB, tol); goto done; }
        if (rho == 0) { out = finish(a, b, x, r, 2, it, normB, tol); goto done; }
        if (fresh) {
            memcpy(p, r, bytes);
            fresh = 0;
        } else {
            double beta = (rho / rhoPrev) * (alpha / omega);
            if (!isfinite(beta)) { out = finish(a, b, x, r, 3, it, normB, tol); goto done; }
            axpy(n, -omega, v, p);
            scale(n, beta, p);
            axpy(n, 1.0, r, p);
        }
        precond(M, n, p, ph);
        or_spmv(a, ph, v);
        double den = or_dot(n, sh, v);
        if (!isfinite(den)) { out = finish(a, b, x, r, 3, it, normB, tol); goto done; }
        if (den == 0) { out = finish(a, b, x, r, 2, it, normB, tol); goto done; }
        alpha = rho / den;
        if (!isfinite(alpha)) { out = finish(a, b, x, r, 3, it, normB, tol); goto done; }
        memcpy(s, r, bytes);
        axpy(n, -alpha, v, s);
        axpy(n, alpha, ph, x);
        double normS = or_norm(n, s);
        if (!isfinite(normS)) { out = finish(a, b, x, r, 3, it, normB, tol); goto done; }
        if (normS <= tol) {
            residual(a, b, x, r);
            res = or_norm(n, r);
            if (res <= tol || !isfinite(res)) { out = finish(a, b, x, r, 1, it, normB, tol); goto done; }
            memcpy(sh, r, bytes);
            fresh = 1;
            continue;
        }
        precond(M, n, s, shat);
        or_spmv(a, shat, t);
        double tt = or_dot(n, t, t), ts = or_dot(n, t, s);
        if (!isfinite(tt) || !isfinite(ts)) { out = finish(a, b, x, r, 3, it, normB, tol); goto done; }
        if (tt == 0) { out = finish(a, b, x, r, 2, it, normB, tol); goto done; }
        omega = ts / tt;
        if (!isfinite(omega)) { out = finish(a, b, x, r, 3, it, normB, tol); goto done; }
        if (omega == 0) { out = finish(a, b, x, r, 2, it, normB, tol); goto done; }
        axpy(n, omega, shat, x);
        memcpy(r, s, bytes);
        axpy(n, -omega, t, r);
        res = or_norm(n, r);
        if (!isfinite(res)) { out = finish(a, b, x, r, 3, it, normB, tol); goto done; }
        if (res <= tol || it % o->refresh_interval == 0) {
            residual(a, b, x, r);
            res = or_norm(n, r);
            if (res <= tol || !isfinite(res)) { out = finish(a, b, x, r, 1, it, normB, tol); goto done; }
            memcpy(sh, r, bytes);
            fresh = 1;
        }
        rhoPrev = rho;
    }
    out = finish(a, b, x, r, 1, o->max_iterations, normB, tol);
done:
    free(r); free(sh); free(p); free(v); free(s); free(t); free(ph); free(shat);
    return out;
}

/* ------------------------------------------------------------------------ */
/* Generators.                                                               */
/* ------------------------------------------------------------------------ */
/* MT19937 (Matsumoto & Nishimura 1998), the generator behind the reference's
 * std::mt19937 test inputs. */
typedef struct {
    uint32_t mt[624];
    int idx;
} mt_state;

static void mt_seed(mt_state *s, uint32_t seed) {
    s->mt[0] = seed;
    for (int i = 1; i < 624; ++i) s->mt[i] = 1812433253u * (s->mt[i - 1] ^ (s->mt[i - 1] >> 30)) + (uint32_t)i;
    s->idx = 624;
}

static uint32_t mt_next(mt_state *s) {
    if (s->idx >= 624) {
        for (int i = 0; i < 624; ++i) {
            uint32_t y = (s->mt[i] & 0x80000000u) | (s->mt[(i + 1) % 624] & 0x7fffffffu);
            s->mt[i] = s->mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        s->idx = 0;
    }
    uint32_t y = s->mt[s->idx++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

void or_mt19937(uint32_t seed, int count, uint32_t *out) {
    mt_state s;
    mt_seed(&s, seed);
    for (int i = 0; i < count; ++i) out[i] = mt_next(&s);
}

/* sample(n) of test/amg_native_test.cpp:28-52: random -1..-4 off-diagonals
 * (about 1 in 11 plus the two neighbours), every 13th row/column isolated,
 * diagonal 2 + sum |offdiag|; columns ascending. */
int or_sample_matrix(int n, or_csr *out) {
    mt_state s;
    mt_seed(&s, (uint32_t)(173 + n));
    int64_t cap = (int64_t)n * n + n;
    out->rows = out->cols = n;
    out->offsets = (int *)malloc(sizeof(int) * ((size_t)n + 1));
    out->indices = (int *)malloc(sizeof(int) * (size_t)cap);
    out->values = (double *)malloc(sizeof(double) * (size_t)cap);
    int64_t k = 0;
    out->offsets[0] = 0;
    for (int i = 0; i < n; ++i) {
        double diagonal = 2;
        int64_t start = k;
        int diag_pos = -1;
        for (int j = 0; j < n; ++j) {
            if (i != j && i % 13 != 0 && j % 13 != 0) {
                int take = (mt_next(&s) % 11 == 0) || abs(i - j) == 1;
                if (take) {
                    double value = -(double)(1 + mt_next(&s) % 4);
                    if (j > i && diag_pos < 0) diag_pos = (int)(k++ - start);
                    out->indices[k] = j;
                    out->values[k] = value;
                    ++k;
                    diagonal -= value;
                }
            }
        }
        if (diag_pos < 0) diag_pos = (int)(k++ - start);
        out->indices[start + diag_pos] = i;
        out->values[start + diag_pos] = diagonal;
        out->offsets[i + 1] = (int)k;
    }
    out->nnz = k;
    return OR_OK;
}
