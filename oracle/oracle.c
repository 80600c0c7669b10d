/*
 * CPU oracle for the pressure-correction hot path (TEST INFRASTRUCTURE ONLY).
 * Serial C restatement of the reference algorithms; every function cites the reference
 * file:line it follows (paths relative to the Yipexnn/CFD project root). Build with
 * -ffp-contract=off: no fused multiply-add, matching the reference's x86-64 host rounding.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------------------------ */
/* small utilities                                                                             */
/* ------------------------------------------------------------------------------------------ */

typedef struct {
    int n_rows, n_cols, nnz;
    int* rp;
    int* ci;
    double* va;
} csr_t;

static void csr_free(csr_t* m) {
    free(m->rp);
    free(m->ci);
    free(m->va);
    memset(m, 0, sizeof(*m));
}

static void sort_int_asc(int* a, int n) {
    for (int i = 1; i < n; ++i) {
        int v = a[i];
        int j = i;
        for (; j > 0 && a[j - 1] > v; --j) a[j] = a[j - 1];
        a[j] = v;
    }
}

/* ------------------------------------------------------------------------------------------ */
/* LDU matrix                                                                                  */
/* ------------------------------------------------------------------------------------------ */

/* ldu_matrix.cpp:572-612: triplets (c,c), (own,nei), (nei,own) -> setFromTriplets (sorted,
 * duplicates merged) -> linear search of each position. */
int orc_build_pattern(int n, int nf, const int* own, const int* nei, int* row_ptr, int* col,
                      int* diag_pos, int* upper_pos, int* lower_pos) {
    if (n < 0 || nf < 0) return -1;
    for (int f = 0; f < nf; ++f) {
        if (own[f] < 0 || own[f] >= n || nei[f] < 0 || nei[f] >= n) return -1;
    }
    int* cnt = (int*)calloc((size_t)n + 1, sizeof(int));
    for (int c = 0; c < n; ++c) cnt[c + 1] += 1;
    for (int f = 0; f < nf; ++f) {
        cnt[own[f] + 1] += 1;
        cnt[nei[f] + 1] += 1;
    }
    for (int c = 0; c < n; ++c) cnt[c + 1] += cnt[c];
    int total = cnt[n];
    int* tmp = (int*)malloc(sizeof(int) * (size_t)(total > 0 ? total : 1));
    int* fill = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int c = 0; c < n; ++c) fill[c] = cnt[c];
    for (int c = 0; c < n; ++c) tmp[fill[c]++] = c;
    for (int f = 0; f < nf; ++f) {
        tmp[fill[own[f]]++] = nei[f];
        tmp[fill[nei[f]]++] = own[f];
    }
    int nnz = 0;
    row_ptr[0] = 0;
    for (int c = 0; c < n; ++c) {
        int b = cnt[c], e = cnt[c + 1];
        sort_int_asc(tmp + b, e - b);
        for (int k = b; k < e; ++k) {
            if (k > b && tmp[k] == tmp[k - 1]) continue;
            col[nnz++] = tmp[k];
        }
        row_ptr[c + 1] = nnz;
    }
    free(tmp);
    free(fill);
    free(cnt);
    for (int c = 0; c < n; ++c) {
        diag_pos[c] = -1;
        for (int k = row_ptr[c]; k < row_ptr[c + 1]; ++k)
            if (col[k] == c) { diag_pos[c] = k; break; }
    }
    for (int f = 0; f < nf; ++f) {
        upper_pos[f] = lower_pos[f] = -1;
        for (int k = row_ptr[own[f]]; k < row_ptr[own[f] + 1]; ++k)
            if (col[k] == nei[f]) { upper_pos[f] = k; break; }
        for (int k = row_ptr[nei[f]]; k < row_ptr[nei[f] + 1]; ++k)
            if (col[k] == own[f]) { lower_pos[f] = k; break; }
    }
    return nnz;
}

/* krylov_openmp.cpp:289-300 (serial host loop). */
void orc_assemble(int n_cells, int n_faces, const int* own, const int* nei, const double* flux,
                  const double* gamma, const double* delta, double convection, double* upper,
                  double* lower, double* diag, double* div) {
    (void)n_cells;
    for (int f = 0; f < n_faces; ++f) {
        const double fl = flux[f];
        const double g = gamma[f] * delta[f];
        const double pos = fl > 0.0 ? convection * fl : 0.0;
        const double neg = fl < 0.0 ? convection * fl : 0.0;
        upper[f] = neg - g;
        lower[f] = -pos - g;
        diag[own[f]] += pos + g;
        diag[nei[f]] += -neg + g;
        div[own[f]] += fl;
        div[nei[f]] -= fl;
    }
}

/* ldu_matrix.cpp:39-56 */
void orc_ldu_multiply(int n, int nf, const int* own, const int* nei, const double* diag,
                      const double* upper, const double* lower, const double* x, double* y) {
    for (int c = 0; c < n; ++c) y[c] = 0.0;
    for (int f = 0; f < nf; ++f) {
        y[own[f]] += upper[f] * x[nei[f]];
        y[nei[f]] += lower[f] * x[own[f]];
    }
    for (int c = 0; c < n; ++c) y[c] += diag[c] * x[c];
}

/* ldu_matrix.cpp:69-103 (one process). */
void orc_ldu_residual_norms(int n, int nf, const int* own, const int* nei, const double* diag,
                            const double* upper, const double* lower, const double* source,
                            const double* x, double* out) {
    out[0] = out[1] = 0.0;
    if (n == 0) return;
    double* ax = (double*)malloc(sizeof(double) * (size_t)n);
    double* rs = (double*)malloc(sizeof(double) * (size_t)n);
    orc_ldu_multiply(n, nf, own, nei, diag, upper, lower, x, ax);
    double sum = 0.0;
    for (int c = 0; c < n; ++c) sum += x[c];
    const double x_ref = sum / (double)n;
    for (int c = 0; c < n; ++c) rs[c] = diag[c];
    for (int f = 0; f < nf; ++f) {
        rs[own[f]] += upper[f];
        rs[nei[f]] += lower[f];
    }
    double res = 0.0, norm = 0.0;
    for (int c = 0; c < n; ++c) {
        const double ax_ref = rs[c] * x_ref;
        res += fabs(source[c] - ax[c]);
        norm += fabs(ax[c] - ax_ref) + fabs(source[c] - ax_ref);
    }
    out[0] = res;
    out[1] = norm;
    free(ax);
    free(rs);
}

/* ldu_matrix.cpp:105-109 */
void orc_set_reference(double* diag, double* source, int cell, double value) {
    source[cell] += diag[cell] * value;
    diag[cell] += diag[cell];
}

/* device_solver.cpp:127-134 */
void orc_ldu_to_csr(int n, int nf, const int* diag_pos, const int* upper_pos,
                    const int* lower_pos, const double* diag, const double* upper,
                    const double* lower, double* val) {
    for (int i = 0; i < n; ++i) val[diag_pos[i]] = diag[i];
    for (int f = 0; f < nf; ++f) {
        val[upper_pos[f]] = upper[f];
        val[lower_pos[f]] = lower[f];
    }
}

/* krylov_kernels.inc:12-24 */
void orc_csr_spmv(int n, const int* rp, const int* ci, const double* va, const double* x,
                  double* y) {
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) s += va[k] * x[ci[k]];
        y[i] = s;
    }
}

/* ------------------------------------------------------------------------------------------ */
/* Aggregation and smoothed-aggregation setup (amg.cpp)                                        */
/* ------------------------------------------------------------------------------------------ */

static int strong(int i, int j, double v, const double* d, double theta) {
    return i != j && fabs(v) > theta * sqrt(fabs(d[i] * d[j]));
}

/* amg.cpp:12-78 */
int orc_aggregate(int n, const int* rp, const int* ci, const double* va, const double* diag,
                  double theta, int* agg) {
    for (int i = 0; i < n; ++i) agg[i] = -1;
    int n_agg = 0;
    /* pass 1: seeds whose strong neighbourhood is still free */
    for (int i = 0; i < n; ++i) {
        if (agg[i] >= 0) continue;
        int is_free = 1, has_strong = 0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            if (strong(i, ci[k], va[k], diag, theta)) {
                has_strong = 1;
                if (agg[ci[k]] >= 0) { is_free = 0; break; }
            }
        }
        if (!is_free || !has_strong) continue;
        agg[i] = n_agg;
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (strong(i, ci[k], va[k], diag, theta)) agg[ci[k]] = n_agg;
        ++n_agg;
    }
    /* pass 2: attach to the strongest pass-1 neighbour (strict >, first wins) */
    int* pass1 = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    memcpy(pass1, agg, sizeof(int) * (size_t)n);
    for (int i = 0; i < n; ++i) {
        if (agg[i] >= 0) continue;
        double best = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            const int j = ci[k];
            if (strong(i, j, va[k], diag, theta) && pass1[j] >= 0 && fabs(va[k]) > best) {
                best = fabs(va[k]);
                agg[i] = pass1[j];
            }
        }
    }
    free(pass1);
    /* pass 3: leftovers with their free strong neighbours */
    for (int i = 0; i < n; ++i) {
        if (agg[i] < 0) {
            agg[i] = n_agg;
            for (int k = rp[i]; k < rp[i + 1]; ++k)
                if (strong(i, ci[k], va[k], diag, theta) && agg[ci[k]] < 0) agg[ci[k]] = n_agg;
            ++n_agg;
        }
    }
    return n_agg;
}

/* Gustavson product C = A * B with the accumulation order of Eigen's conservative sparse
 * product: for row i, for k ascending in A(i,:), for j ascending in B(k,:): first touch
 * assigns a_ik*b_kj, later touches add. Columns of each result row sorted ascending. */
static void spgemm(const csr_t* a, const csr_t* b, csr_t* c) {
    const int n = a->n_rows, m = b->n_cols;
    int* mark = (int*)malloc(sizeof(int) * (size_t)(m > 0 ? m : 1));
    double* acc = (double*)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
    int* list = (int*)malloc(sizeof(int) * (size_t)(m > 0 ? m : 1));
    for (int j = 0; j < m; ++j) mark[j] = -1;
    int cap = a->nnz + 16;
    c->n_rows = n;
    c->n_cols = m;
    c->rp = (int*)malloc(sizeof(int) * (size_t)(n + 1));
    c->ci = (int*)malloc(sizeof(int) * (size_t)cap);
    c->va = (double*)malloc(sizeof(double) * (size_t)cap);
    int nnz = 0;
    c->rp[0] = 0;
    for (int i = 0; i < n; ++i) {
        int cnt = 0;
        for (int ka = a->rp[i]; ka < a->rp[i + 1]; ++ka) {
            const int k = a->ci[ka];
            const double x = a->va[ka];
            for (int kb = b->rp[k]; kb < b->rp[k + 1]; ++kb) {
                const int j = b->ci[kb];
                if (mark[j] != i) {
                    mark[j] = i;
                    acc[j] = x * b->va[kb];
                    list[cnt++] = j;
                } else {
                    acc[j] += x * b->va[kb];
                }
            }
        }
        sort_int_asc(list, cnt);
        if (nnz + cnt > cap) {
            while (nnz + cnt > cap) cap *= 2;
            c->ci = (int*)realloc(c->ci, sizeof(int) * (size_t)cap);
            c->va = (double*)realloc(c->va, sizeof(double) * (size_t)cap);
        }
        for (int t = 0; t < cnt; ++t) {
            c->ci[nnz] = list[t];
            c->va[nnz] = acc[list[t]];
            ++nnz;
        }
        c->rp[i + 1] = nnz;
    }
    c->nnz = nnz;
    free(mark);
    free(acc);
    free(list);
}

/* prune(0.0): drop entries whose value is exactly zero (either sign). */
static void prune_zeros(csr_t* m) {
    int nnz = 0;
    int start = 0;
    for (int i = 0; i < m->n_rows; ++i) {
        const int end = m->rp[i + 1];
        for (int k = start; k < end; ++k) {
            if (m->va[k] != 0.0) {
                m->ci[nnz] = m->ci[k];
                m->va[nnz] = m->va[k];
                ++nnz;
            }
        }
        start = end;
        m->rp[i + 1] = nnz;
    }
    m->nnz = nnz;
}

static void transpose(const csr_t* a, csr_t* t) {
    t->n_rows = a->n_cols;
    t->n_cols = a->n_rows;
    t->nnz = a->nnz;
    t->rp = (int*)calloc((size_t)t->n_rows + 1, sizeof(int));
    t->ci = (int*)malloc(sizeof(int) * (size_t)(a->nnz > 0 ? a->nnz : 1));
    t->va = (double*)malloc(sizeof(double) * (size_t)(a->nnz > 0 ? a->nnz : 1));
    for (int k = 0; k < a->nnz; ++k) t->rp[a->ci[k] + 1] += 1;
    for (int j = 0; j < t->n_rows; ++j) t->rp[j + 1] += t->rp[j];
    int* fill = (int*)malloc(sizeof(int) * (size_t)(t->n_rows > 0 ? t->n_rows : 1));
    for (int j = 0; j < t->n_rows; ++j) fill[j] = t->rp[j];
    for (int i = 0; i < a->n_rows; ++i) {
        for (int k = a->rp[i]; k < a->rp[i + 1]; ++k) {
            const int j = a->ci[k];
            t->ci[fill[j]] = i;
            t->va[fill[j]] = a->va[k];
            ++fill[j];
        }
    }
    free(fill);
}

static void csr_copy(const csr_t* a, csr_t* c) {
    c->n_rows = a->n_rows;
    c->n_cols = a->n_cols;
    c->nnz = a->nnz;
    c->rp = (int*)malloc(sizeof(int) * (size_t)(a->n_rows + 1));
    c->ci = (int*)malloc(sizeof(int) * (size_t)(a->nnz > 0 ? a->nnz : 1));
    c->va = (double*)malloc(sizeof(double) * (size_t)(a->nnz > 0 ? a->nnz : 1));
    memcpy(c->rp, a->rp, sizeof(int) * (size_t)(a->n_rows + 1));
    memcpy(c->ci, a->ci, sizeof(int) * (size_t)a->nnz);
    memcpy(c->va, a->va, sizeof(double) * (size_t)a->nnz);
}

/* amg.cpp:82-92: last diagonal entry of each row (0 if none). */
static void diagonal_of(const csr_t* a, double* d) {
    for (int i = 0; i < a->n_rows; ++i) {
        d[i] = 0.0;
        for (int k = a->rp[i]; k < a->rp[i + 1]; ++k)
            if (a->ci[k] == i) d[i] = a->va[k];
    }
}

#define ORC_MAX_LEVELS 64

struct orc_amg {
    int n_levels;
    csr_t a[ORC_MAX_LEVELS], p[ORC_MAX_LEVELS], r[ORC_MAX_LEVELS];
    double* inv_diag[ORC_MAX_LEVELS];
    int* agg[ORC_MAX_LEVELS];
    int n_agg[ORC_MAX_LEVELS];
    int n_c;
    double* ldl; /* dense LDL^T factor of the coarsest operator (L below, D on the diagonal) */
    int ldl_ok;
    double* coarse_inv; /* row-major inverse */
};

/* Dense LDL^T without pivoting, in natural order; fails if a pivot is exactly zero (the
 * failure mode of SimplicialLDLT, amg.cpp:185-189). */
static int ldlt_factor(int n, const double* a, double* f) {
    memcpy(f, a, sizeof(double) * (size_t)n * (size_t)n);
    for (int j = 0; j < n; ++j) {
        double d = f[(size_t)j * n + j];
        for (int k = 0; k < j; ++k) {
            const double l = f[(size_t)j * n + k];
            d -= l * l * f[(size_t)k * n + k];
        }
        if (d == 0.0 || !isfinite(d)) return 0;
        f[(size_t)j * n + j] = d;
        for (int i = j + 1; i < n; ++i) {
            double s = f[(size_t)i * n + j];
            for (int k = 0; k < j; ++k)
                s -= f[(size_t)i * n + k] * f[(size_t)j * n + k] * f[(size_t)k * n + k];
            f[(size_t)i * n + j] = s / d;
        }
    }
    return 1;
}

static void ldlt_solve(int n, const double* f, const double* b, double* x) {
    for (int i = 0; i < n; ++i) {
        double s = b[i];
        for (int k = 0; k < i; ++k) s -= f[(size_t)i * n + k] * x[k];
        x[i] = s;
    }
    for (int i = 0; i < n; ++i) x[i] /= f[(size_t)i * n + i];
    for (int i = n - 1; i >= 0; --i) {
        double s = x[i];
        for (int k = i + 1; k < n; ++k) s -= f[(size_t)k * n + i] * x[k];
        x[i] = s;
    }
}

/* Moore-Penrose pseudo-inverse of a symmetric matrix by cyclic Jacobi eigen-decomposition
 * (stand-in for the CompleteOrthogonalDecomposition fallback, amg.cpp:239). */
static void sym_pinv(int n, const double* a, double* out) {
    double* m = (double*)malloc(sizeof(double) * (size_t)n * n);
    double* v = (double*)calloc((size_t)n * n, sizeof(double));
    memcpy(m, a, sizeof(double) * (size_t)n * n);
    for (int i = 0; i < n; ++i) v[(size_t)i * n + i] = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) off += m[(size_t)p * n + q] * m[(size_t)p * n + q];
        if (off < 1e-30) break;
        for (int p = 0; p < n; ++p) {
            for (int q = p + 1; q < n; ++q) {
                const double apq = m[(size_t)p * n + q];
                if (fabs(apq) < 1e-300) continue;
                const double app = m[(size_t)p * n + p], aqq = m[(size_t)q * n + q];
                const double theta = (aqq - app) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; ++k) {
                    const double mkp = m[(size_t)k * n + p], mkq = m[(size_t)k * n + q];
                    m[(size_t)k * n + p] = c * mkp - s * mkq;
                    m[(size_t)k * n + q] = s * mkp + c * mkq;
                }
                for (int k = 0; k < n; ++k) {
                    const double mpk = m[(size_t)p * n + k], mqk = m[(size_t)q * n + k];
                    m[(size_t)p * n + k] = c * mpk - s * mqk;
                    m[(size_t)q * n + k] = s * mpk + c * mqk;
                }
                for (int k = 0; k < n; ++k) {
                    const double vkp = v[(size_t)k * n + p], vkq = v[(size_t)k * n + q];
                    v[(size_t)k * n + p] = c * vkp - s * vkq;
                    v[(size_t)k * n + q] = s * vkp + c * vkq;
                }
            }
        }
    }
    double lmax = 0.0;
    for (int i = 0; i < n; ++i) lmax = fmax(lmax, fabs(m[(size_t)i * n + i]));
    const double tol = lmax * 2.220446049250313e-16 * (double)n;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            double s = 0.0;
            for (int k = 0; k < n; ++k) {
                const double l = m[(size_t)k * n + k];
                if (fabs(l) > tol) s += v[(size_t)i * n + k] * v[(size_t)j * n + k] / l;
            }
            out[(size_t)i * n + j] = s;
        }
    free(m);
    free(v);
}

/* amg.cpp:122-190 */
orc_amg* orc_amg_setup(int n, const int* rp, const int* ci, const double* va, double theta,
                       int max_levels, int coarse_size) {
    if (n <= 0 || max_levels < 1) return NULL;
    if (max_levels > ORC_MAX_LEVELS) max_levels = ORC_MAX_LEVELS;
    orc_amg* h = (orc_amg*)calloc(1, sizeof(orc_amg));
    csr_t cur;
    cur.n_rows = cur.n_cols = n;
    cur.nnz = rp[n];
    cur.rp = (int*)malloc(sizeof(int) * (size_t)(n + 1));
    cur.ci = (int*)malloc(sizeof(int) * (size_t)(cur.nnz > 0 ? cur.nnz : 1));
    cur.va = (double*)malloc(sizeof(double) * (size_t)(cur.nnz > 0 ? cur.nnz : 1));
    memcpy(cur.rp, rp, sizeof(int) * (size_t)(n + 1));
    memcpy(cur.ci, ci, sizeof(int) * (size_t)cur.nnz);
    memcpy(cur.va, va, sizeof(double) * (size_t)cur.nnz);
    for (int l = 0; l < max_levels; ++l) {
        const int nl = cur.n_rows;
        double* d = (double*)malloc(sizeof(double) * (size_t)nl);
        diagonal_of(&cur, d);
        double* inv = (double*)malloc(sizeof(double) * (size_t)nl);
        for (int i = 0; i < nl; ++i) inv[i] = d[i] != 0.0 ? 1.0 / d[i] : 0.0;
        h->a[l] = cur;
        h->inv_diag[l] = inv;
        h->n_levels = l + 1;
        const int last = nl <= coarse_size || l + 1 == max_levels;
        if (last) { free(d); break; }
        int* agg = (int*)malloc(sizeof(int) * (size_t)nl);
        const int n_agg = orc_aggregate(nl, cur.rp, cur.ci, cur.va, d, theta, agg);
        free(d);
        if (n_agg >= nl || n_agg == 0) { free(agg); break; }
        h->agg[l] = agg;
        h->n_agg[l] = n_agg;
        /* Gershgorin bound and damping (amg.cpp:160-167) */
        double rho = 0.0;
        for (int i = 0; i < nl; ++i) {
            double row = 0.0;
            for (int k = cur.rp[i]; k < cur.rp[i + 1]; ++k) row += fabs(cur.va[k]);
            rho = fmax(rho, row * fabs(inv[i]));
        }
        const double omega = rho > 0.0 ? 4.0 / (3.0 * rho) : 0.0;
        /* dinv_a = D^-1 A; smoothed = dinv_a * P_tent (amg.cpp:168-169) */
        csr_t dinv_a;
        csr_copy(&cur, &dinv_a);
        for (int i = 0; i < nl; ++i)
            for (int k = dinv_a.rp[i]; k < dinv_a.rp[i + 1]; ++k)
                dinv_a.va[k] = inv[i] * cur.va[k];
        csr_t pt;
        pt.n_rows = nl;
        pt.n_cols = n_agg;
        pt.nnz = nl;
        pt.rp = (int*)malloc(sizeof(int) * (size_t)(nl + 1));
        pt.ci = (int*)malloc(sizeof(int) * (size_t)nl);
        pt.va = (double*)malloc(sizeof(double) * (size_t)nl);
        for (int i = 0; i <= nl; ++i) pt.rp[i] = i;
        for (int i = 0; i < nl; ++i) { pt.ci[i] = agg[i]; pt.va[i] = 1.0; }
        csr_t sm;
        spgemm(&dinv_a, &pt, &sm);
        csr_free(&dinv_a);
        /* P = P_tent - omega * smoothed over the union pattern, then prune(0) (amg.cpp:170-172) */
        csr_t p;
        p.n_rows = nl;
        p.n_cols = n_agg;
        p.rp = (int*)malloc(sizeof(int) * (size_t)(nl + 1));
        p.ci = (int*)malloc(sizeof(int) * (size_t)(sm.nnz + nl));
        p.va = (double*)malloc(sizeof(double) * (size_t)(sm.nnz + nl));
        int nnz = 0;
        p.rp[0] = 0;
        for (int i = 0; i < nl; ++i) {
            const int tj = agg[i];
            int used_t = 0;
            for (int k = sm.rp[i]; k < sm.rp[i + 1]; ++k) {
                const int j = sm.ci[k];
                const double ws = omega * sm.va[k];
                if (!used_t && tj < j) {
                    p.ci[nnz] = tj;
                    p.va[nnz] = 1.0 - 0.0;
                    ++nnz;
                    used_t = 1;
                }
                if (j == tj) {
                    p.ci[nnz] = j;
                    p.va[nnz] = 1.0 - ws;
                    used_t = 1;
                } else {
                    p.ci[nnz] = j;
                    p.va[nnz] = 0.0 - ws;
                }
                ++nnz;
            }
            if (!used_t) {
                p.ci[nnz] = tj;
                p.va[nnz] = 1.0 - 0.0;
                ++nnz;
            }
            p.rp[i + 1] = nnz;
        }
        p.nnz = nnz;
        csr_free(&sm);
        csr_free(&pt);
        prune_zeros(&p);
        csr_t r;
        transpose(&p, &r);
        csr_t ap, coarse;
        spgemm(&cur, &p, &ap);
        spgemm(&r, &ap, &coarse);
        csr_free(&ap);
        prune_zeros(&coarse);
        h->p[l] = p;
        h->r[l] = r;
        csr_copy(&coarse, &cur);
        csr_free(&coarse);
        if (l + 1 == max_levels) break; /* unreachable: last level handled above */
    }
    /* if the loop ended by "no coarsening", cur is owned by h->a[n_levels-1] already */
    const int lc = h->n_levels - 1;
    const int nc = h->a[lc].n_rows;
    h->n_c = nc;
    double* dense = (double*)calloc((size_t)nc * nc, sizeof(double));
    for (int i = 0; i < nc; ++i)
        for (int k = h->a[lc].rp[i]; k < h->a[lc].rp[i + 1]; ++k)
            dense[(size_t)i * nc + h->a[lc].ci[k]] += h->a[lc].va[k];
    h->ldl = (double*)malloc(sizeof(double) * (size_t)nc * nc);
    h->ldl_ok = ldlt_factor(nc, dense, h->ldl);
    h->coarse_inv = (double*)malloc(sizeof(double) * (size_t)nc * nc);
    if (h->ldl_ok) {
        double* e = (double*)calloc((size_t)nc, sizeof(double));
        double* col = (double*)malloc(sizeof(double) * (size_t)nc);
        for (int j = 0; j < nc; ++j) {
            e[j] = 1.0;
            ldlt_solve(nc, h->ldl, e, col);
            e[j] = 0.0;
            for (int i = 0; i < nc; ++i) h->coarse_inv[(size_t)i * nc + j] = col[i];
        }
        free(e);
        free(col);
    } else {
        sym_pinv(nc, dense, h->coarse_inv);
    }
    free(dense);
    return h;
}

void orc_amg_free(orc_amg* h) {
    if (!h) return;
    for (int l = 0; l < h->n_levels; ++l) {
        csr_free(&h->a[l]);
        csr_free(&h->p[l]);
        csr_free(&h->r[l]);
        free(h->inv_diag[l]);
        free(h->agg[l]);
    }
    free(h->ldl);
    free(h->coarse_inv);
    free(h);
}

int orc_amg_levels(const orc_amg* h) { return h->n_levels; }

int orc_amg_level_csr(const orc_amg* h, int level, int which, int* n_rows, int* n_cols,
                      int* nnz, const int** rp, const int** ci, const double** va) {
    if (level < 0 || level >= h->n_levels) return 0;
    const csr_t* m = which == 0 ? &h->a[level] : which == 1 ? &h->p[level] : &h->r[level];
    if (m->rp == NULL) return 0;
    *n_rows = m->n_rows;
    *n_cols = m->n_cols;
    *nnz = m->nnz;
    *rp = m->rp;
    *ci = m->ci;
    *va = m->va;
    return 1;
}

const int* orc_amg_aggregates(const orc_amg* h, int level, int* n_agg) {
    if (level < 0 || level >= h->n_levels) return NULL;
    *n_agg = h->n_agg[level];
    return h->agg[level];
}

const double* orc_amg_coarse_inverse(const orc_amg* h, int* n_c, int* ok) {
    *n_c = h->n_c;
    *ok = h->ldl_ok;
    return h->coarse_inv;
}

/* amg.cpp:242-251 */
double orc_amg_operator_complexity(const orc_amg* h) {
    double total = 0.0;
    for (int l = 0; l < h->n_levels; ++l) total += (double)h->a[l].nnz;
    return total / (double)h->a[0].nnz;
}

/* ---- CPU AmgCg: Gauss-Seidel V-cycle + pcg ---- */

/* amg.cpp:94-118 */
static void gauss_seidel(const csr_t* a, const double* inv_diag, const double* b, double* x,
                         int forward) {
    const int n = a->n_rows;
    for (int s = 0; s < n; ++s) {
        const int i = forward ? s : n - 1 - s;
        double sum = b[i];
        double d = 0.0;
        for (int k = a->rp[i]; k < a->rp[i + 1]; ++k) {
            if (a->ci[k] == i) d = a->va[k];
            else sum -= a->va[k] * x[a->ci[k]];
        }
        x[i] = d != 0.0 ? sum * inv_diag[i] : x[i];
    }
}

static void csr_mv(const csr_t* a, const double* x, double* y) {
    orc_csr_spmv(a->n_rows, a->rp, a->ci, a->va, x, y);
}

/* amg.cpp:192-216 (pre_smooth = post_smooth = 1) */
static void gs_cycle(const orc_amg* h, int l, const double* b, double* x) {
    const csr_t* a = &h->a[l];
    const int n = a->n_rows;
    if (l + 1 == h->n_levels) {
        if (h->ldl_ok) {
            ldlt_solve(n, h->ldl, b, x);
        } else {
            for (int s = 0; s < 20; ++s) {
                gauss_seidel(a, h->inv_diag[l], b, x, 1);
                gauss_seidel(a, h->inv_diag[l], b, x, 0);
            }
        }
        return;
    }
    gauss_seidel(a, h->inv_diag[l], b, x, 1);
    double* res = (double*)malloc(sizeof(double) * (size_t)n);
    csr_mv(a, x, res);
    for (int i = 0; i < n; ++i) res[i] = b[i] - res[i];
    const int nc = h->r[l].n_rows;
    double* rc = (double*)malloc(sizeof(double) * (size_t)nc);
    double* ec = (double*)calloc((size_t)nc, sizeof(double));
    csr_mv(&h->r[l], res, rc);
    gs_cycle(h, l + 1, rc, ec);
    csr_mv(&h->p[l], ec, res);
    for (int i = 0; i < n; ++i) x[i] += res[i];
    gauss_seidel(a, h->inv_diag[l], b, x, 0);
    free(res);
    free(rc);
    free(ec);
}

static double dotv(int n, const double* x, const double* y) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += x[i] * y[i];
    return s;
}

/* amg.cpp:253-285 */
int orc_pcg_gs(const orc_amg* h, const double* b, double* x, double tolerance,
               int max_iterations, double* res_out) {
    const csr_t* a = &h->a[0];
    const int n = a->n_rows;
    double* r = (double*)malloc(sizeof(double) * (size_t)n);
    double* z = (double*)calloc((size_t)n, sizeof(double));
    double* p = (double*)malloc(sizeof(double) * (size_t)n);
    double* ap = (double*)malloc(sizeof(double) * (size_t)n);
    int iterations = 0;
    csr_mv(a, x, r);
    for (int i = 0; i < n; ++i) r[i] = b[i] - r[i];
    double res = sqrt(dotv(n, r, r));
    if (res > tolerance) {
        memset(z, 0, sizeof(double) * (size_t)n);
        gs_cycle(h, 0, r, z);
        memcpy(p, z, sizeof(double) * (size_t)n);
        double rz = dotv(n, r, z);
        for (int it = 1; it <= max_iterations; ++it) {
            csr_mv(a, p, ap);
            const double pap = dotv(n, p, ap);
            if (pap <= 0.0) break;
            const double alpha = rz / pap;
            for (int i = 0; i < n; ++i) x[i] += alpha * p[i];
            for (int i = 0; i < n; ++i) r[i] -= alpha * ap[i];
            iterations = it;
            res = sqrt(dotv(n, r, r));
            if (res <= tolerance) break;
            memset(z, 0, sizeof(double) * (size_t)n);
            gs_cycle(h, 0, r, z);
            const double rz_new = dotv(n, r, z);
            const double beta = rz_new / rz;
            for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
            rz = rz_new;
        }
    }
    *res_out = res;
    free(r);
    free(z);
    free(p);
    free(ap);
    return iterations;
}

/* ------------------------------------------------------------------------------------------ */
/* Accelerator-path algorithm (krylov_kernels.inc + krylov_openmp.cpp)                          */
/* ------------------------------------------------------------------------------------------ */

static void view_spmv(const orc_csr_view* a, const double* x, double* y) {
    orc_csr_spmv(a->n, a->rp, a->ci, a->va, x, y);
}

/* krylov_openmp.cpp:147-157: last nonzero diagonal entry, default 1. */
static void inverse_diagonal(const orc_csr_view* a, double* d) {
    for (int i = 0; i < a->n; ++i) {
        d[i] = 1.0;
        for (int k = a->rp[i]; k < a->rp[i + 1]; ++k)
            if (a->ci[k] == i && a->va[k] != 0.0) d[i] = 1.0 / a->va[k];
    }
}

typedef struct {
    const orc_csr_view* a;
    const orc_csr_view* p;
    const orc_csr_view* r;
    double** dinv;
    double** x;
    double** b;
    double** t;
    int n_levels;
    const double* coarse_inverse;
    int sweeps;
    double w;
} vc_ctx;

/* krylov_kernels.inc:182-194 */
static void amg_jacobi(const vc_ctx* c, int l) {
    const int n = c->a[l].n;
    double* x = c->x[l];
    const double* b = c->b[l];
    double* t = c->t[l];
    const double* d = c->dinv[l];
    for (int s = 0; s < c->sweeps; ++s) {
        view_spmv(&c->a[l], x, t);
        for (int i = 0; i < n; ++i) x[i] += c->w * d[i] * (b[i] - t[i]);
    }
}

/* krylov_kernels.inc:197-238 */
static void vcycle(const vc_ctx* c, int l) {
    const int n = c->a[l].n;
    if (l == c->n_levels - 1) {
        for (int i = 0; i < n; ++i) {
            double s = 0.0;
            for (int j = 0; j < n; ++j) s += c->coarse_inverse[(size_t)i * n + j] * c->b[l][j];
            c->x[l][i] = s;
        }
        return;
    }
    double* x = c->x[l];
    double* t = c->t[l];
    const double* b = c->b[l];
    for (int i = 0; i < n; ++i) x[i] = 0.0;
    amg_jacobi(c, l);
    view_spmv(&c->a[l], x, t);
    for (int i = 0; i < n; ++i) t[i] = b[i] - t[i];
    view_spmv(&c->r[l], t, c->b[l + 1]);
    vcycle(c, l + 1);
    view_spmv(&c->p[l], c->x[l + 1], t);
    for (int i = 0; i < n; ++i) x[i] += t[i];
    amg_jacobi(c, l);
}

static void vc_alloc(vc_ctx* c, int n_levels, const orc_csr_view* a, const orc_csr_view* p,
                     const orc_csr_view* r, const double* ci, int sweeps, double w) {
    c->a = a;
    c->p = p;
    c->r = r;
    c->n_levels = n_levels;
    c->coarse_inverse = ci;
    c->sweeps = sweeps;
    c->w = w;
    c->dinv = (double**)malloc(sizeof(double*) * (size_t)n_levels);
    c->x = (double**)malloc(sizeof(double*) * (size_t)n_levels);
    c->b = (double**)malloc(sizeof(double*) * (size_t)n_levels);
    c->t = (double**)malloc(sizeof(double*) * (size_t)n_levels);
    for (int l = 0; l < n_levels; ++l) {
        const size_t n = (size_t)(a[l].n > 0 ? a[l].n : 1);
        c->dinv[l] = (double*)malloc(sizeof(double) * n);
        inverse_diagonal(&a[l], c->dinv[l]);
        c->x[l] = (double*)calloc(n, sizeof(double));
        c->b[l] = (double*)calloc(n, sizeof(double));
        c->t[l] = (double*)calloc(n, sizeof(double));
    }
}

static void vc_free(vc_ctx* c) {
    for (int l = 0; l < c->n_levels; ++l) {
        free(c->dinv[l]);
        free(c->x[l]);
        free(c->b[l]);
        free(c->t[l]);
    }
    free(c->dinv);
    free(c->x);
    free(c->b);
    free(c->t);
}

void orc_vcycle_apply(int n_levels, const orc_csr_view* a, const orc_csr_view* p,
                      const orc_csr_view* r, const double* coarse_inverse, int sweeps,
                      double weight, const double* rhs, double* z) {
    vc_ctx c;
    vc_alloc(&c, n_levels, a, p, r, coarse_inverse, sweeps, weight);
    memcpy(c.b[0], rhs, sizeof(double) * (size_t)a[0].n);
    vcycle(&c, 0);
    memcpy(z, c.x[0], sizeof(double) * (size_t)a[0].n);
    vc_free(&c);
}

/* krylov_kernels.inc:240-301 */
orc_stats orc_amg_cg(int n_levels, const orc_csr_view* a, const orc_csr_view* p,
                     const orc_csr_view* r, const double* coarse_inverse, int sweeps,
                     double weight, const double* b, double* x, double abs_tol, int max_iter) {
    orc_stats st = {0, 0.0, 0};
    vc_ctx c;
    vc_alloc(&c, n_levels, a, p, r, coarse_inverse, sweeps, weight);
    const int n = a[0].n;
    double* rv = (double*)calloc((size_t)n, sizeof(double));
    double* pv = (double*)calloc((size_t)n, sizeof(double));
    double* q = (double*)calloc((size_t)n, sizeof(double));
    view_spmv(&a[0], x, q);
    for (int i = 0; i < n; ++i) rv[i] = b[i] - q[i];
    double res = sqrt(dotv(n, rv, rv));
    if (res <= abs_tol) {
        st.residual = res;
        st.converged = 1;
        goto done;
    }
    double* zb = c.b[0];
    double* z = c.x[0];
    memcpy(zb, rv, sizeof(double) * (size_t)n);
    vcycle(&c, 0);
    memcpy(pv, z, sizeof(double) * (size_t)n);
    double rz = dotv(n, rv, z);
    for (st.iterations = 1; st.iterations <= max_iter; ++st.iterations) {
        view_spmv(&a[0], pv, q);
        const double pq = dotv(n, pv, q);
        if (pq == 0.0) break;
        const double alpha = rz / pq;
        for (int i = 0; i < n; ++i) {
            x[i] += alpha * pv[i];
            rv[i] -= alpha * q[i];
        }
        res = sqrt(dotv(n, rv, rv));
        if (res <= abs_tol) {
            st.converged = 1;
            break;
        }
        memcpy(zb, rv, sizeof(double) * (size_t)n);
        vcycle(&c, 0);
        const double rz_new = dotv(n, rv, z);
        const double beta = rz_new / rz;
        rz = rz_new;
        for (int i = 0; i < n; ++i) pv[i] = z[i] + beta * pv[i];
    }
    if (st.iterations > max_iter) st.iterations = max_iter;
    st.residual = res;
done:
    free(rv);
    free(pv);
    free(q);
    vc_free(&c);
    return st;
}

/* krylov_kernels.inc:44-169 with the diagonal of solve_openmp (krylov_openmp.cpp:99-106). */
orc_stats orc_krylov(const orc_csr_view* a, const double* b, double* x, int method,
                     double abs_tol, int max_iter) {
    orc_stats st = {0, 0.0, 0};
    const int n = a->n;
    const size_t sz = (size_t)(n > 0 ? n : 1);
    double* dinv = (double*)malloc(sizeof(double) * sz);
    inverse_diagonal(a, dinv);
    double* w = (double*)calloc(sz * 8, sizeof(double));
    double *r = w, *z = w + sz, *p = w + 2 * sz, *q = w + 3 * sz;
    if (method == 0) {
        view_spmv(a, x, q);
        for (int i = 0; i < n; ++i) r[i] = b[i] - q[i];
        double res = sqrt(dotv(n, r, r));
        if (res <= abs_tol) {
            st.residual = res;
            st.converged = 1;
            goto out;
        }
        for (int i = 0; i < n; ++i) z[i] = r[i] * dinv[i];
        for (int i = 0; i < n; ++i) p[i] = z[i];
        double rz = dotv(n, r, z);
        for (st.iterations = 1; st.iterations <= max_iter; ++st.iterations) {
            view_spmv(a, p, q);
            const double pq = dotv(n, p, q);
            if (pq == 0.0) break;
            const double alpha = rz / pq;
            for (int i = 0; i < n; ++i) {
                x[i] += alpha * p[i];
                r[i] -= alpha * q[i];
            }
            res = sqrt(dotv(n, r, r));
            if (res <= abs_tol) {
                st.converged = 1;
                break;
            }
            for (int i = 0; i < n; ++i) z[i] = r[i] * dinv[i];
            const double rz_new = dotv(n, r, z);
            const double beta = rz_new / rz;
            rz = rz_new;
            for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
        }
        if (st.iterations > max_iter) st.iterations = max_iter;
        st.residual = res;
    } else {
        double *r0 = w + sz, *pp = w + 2 * sz, *v = w + 3 * sz, *s = w + 4 * sz,
               *t = w + 5 * sz, *ph = w + 6 * sz, *sh = w + 7 * sz;
        view_spmv(a, x, v);
        for (int i = 0; i < n; ++i) {
            r[i] = b[i] - v[i];
            r0[i] = r[i];
            pp[i] = 0.0;
            v[i] = 0.0;
        }
        double res = sqrt(dotv(n, r, r));
        if (res <= abs_tol) {
            st.residual = res;
            st.converged = 1;
            goto out;
        }
        double rho = 1.0, alpha = 1.0, omega = 1.0;
        for (st.iterations = 1; st.iterations <= max_iter; ++st.iterations) {
            const double rho_new = dotv(n, r0, r);
            if (rho_new == 0.0 || omega == 0.0) break;
            const double beta = (rho_new / rho) * (alpha / omega);
            rho = rho_new;
            for (int i = 0; i < n; ++i) pp[i] = r[i] + beta * (pp[i] - omega * v[i]);
            for (int i = 0; i < n; ++i) ph[i] = pp[i] * dinv[i];
            view_spmv(a, ph, v);
            const double r0v = dotv(n, r0, v);
            if (r0v == 0.0) break;
            alpha = rho / r0v;
            for (int i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
            const double s_norm = sqrt(dotv(n, s, s));
            if (s_norm <= abs_tol) {
                for (int i = 0; i < n; ++i) x[i] += alpha * ph[i];
                res = s_norm;
                st.converged = 1;
                break;
            }
            for (int i = 0; i < n; ++i) sh[i] = s[i] * dinv[i];
            view_spmv(a, sh, t);
            const double tt = dotv(n, t, t);
            omega = tt > 0.0 ? dotv(n, t, s) / tt : 0.0;
            for (int i = 0; i < n; ++i) {
                x[i] += alpha * ph[i] + omega * sh[i];
                r[i] = s[i] - omega * t[i];
            }
            res = sqrt(dotv(n, r, r));
            if (res <= abs_tol) {
                st.converged = 1;
                break;
            }
        }
        if (st.iterations > max_iter) st.iterations = max_iter;
        st.residual = res;
    }
out:
    free(dinv);
    free(w);
    return st;
}
