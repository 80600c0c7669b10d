#include "host_algos.hpp"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>

#include <omp.h>

namespace cfdb {

LduPatternHost build_pattern(int n, int nf, const int* owner, const int* neighbour) {
    if (n < 0 || nf < 0) fail(1, "build_pattern: negative size");
    for (int f = 0; f < nf; ++f) {
        if (owner[f] < 0 || owner[f] >= n || neighbour[f] < 0 || neighbour[f] >= n) {
            fail(1, "build_pattern: face " + std::to_string(f) + " addresses a cell out of range");
        }
    }
    LduPatternHost p;
    p.n = n;
    p.n_faces = nf;
    std::vector<int> cnt(static_cast<size_t>(n) + 1, 0);
    for (int c = 0; c < n; ++c) cnt[c + 1] = 1;
    for (int f = 0; f < nf; ++f) {
        ++cnt[owner[f] + 1];
        ++cnt[neighbour[f] + 1];
    }
    for (int c = 0; c < n; ++c) cnt[c + 1] += cnt[c];
    std::vector<int> tmp(static_cast<size_t>(cnt[n]));
    std::vector<int> fill(cnt.begin(), cnt.end() - 1);
    for (int c = 0; c < n; ++c) tmp[fill[c]++] = c;
    for (int f = 0; f < nf; ++f) {
        tmp[fill[owner[f]]++] = neighbour[f];
        tmp[fill[neighbour[f]]++] = owner[f];
    }
    p.row_ptr.assign(static_cast<size_t>(n) + 1, 0);
    // sort + unique each row (rows are short)
    std::vector<int> row_len(static_cast<size_t>(n));
#pragma omp parallel for schedule(static) if (n > 100000)
    for (int c = 0; c < n; ++c) {
        int* b = tmp.data() + cnt[c];
        int* e = tmp.data() + cnt[c + 1];
        std::sort(b, e);
        row_len[c] = static_cast<int>(std::unique(b, e) - b);
    }
    for (int c = 0; c < n; ++c) p.row_ptr[c + 1] = p.row_ptr[c] + row_len[c];
    p.col.resize(static_cast<size_t>(p.row_ptr[n]));
    p.diag_pos.resize(static_cast<size_t>(n));
#pragma omp parallel for schedule(static) if (n > 100000)
    for (int c = 0; c < n; ++c) {
        std::memcpy(p.col.data() + p.row_ptr[c], tmp.data() + cnt[c], sizeof(int) * row_len[c]);
        const int* b = p.col.data() + p.row_ptr[c];
        p.diag_pos[c] = p.row_ptr[c] + static_cast<int>(std::lower_bound(b, b + row_len[c], c) - b);
    }
    p.upper_pos.resize(static_cast<size_t>(nf));
    p.lower_pos.resize(static_cast<size_t>(nf));
#pragma omp parallel for schedule(static) if (nf > 100000)
    for (int f = 0; f < nf; ++f) {
        const int o = owner[f], nb = neighbour[f];
        const int* cols = p.col.data();
        const int* bo = cols + p.row_ptr[o];
        const int* bn = cols + p.row_ptr[nb];
        p.upper_pos[f] = p.row_ptr[o] + static_cast<int>(std::lower_bound(bo, cols + p.row_ptr[o + 1], nb) - bo);
        p.lower_pos[f] = p.row_ptr[nb] + static_cast<int>(std::lower_bound(bn, cols + p.row_ptr[nb + 1], o) - bn);
    }
    return p;
}

namespace {

bool strong(int i, int j, double v, const std::vector<double>& d, double theta) {
    return i != j && std::fabs(v) > theta * std::sqrt(std::fabs(d[i] * d[j]));
}

// Gustavson C = A * B (see header for the accumulation order); row-parallel, two passes.
HostCsr spgemm(const HostCsr& a, const HostCsr& b) {
    HostCsr c;
    c.n_rows = a.n_rows;
    c.n_cols = b.n_cols;
    const int n = a.n_rows, m = b.n_cols;
    c.rp.assign(static_cast<size_t>(n) + 1, 0);
    std::vector<int> len(static_cast<size_t>(n), 0);
#pragma omp parallel if (n > 256)
    {
        std::vector<int> mark(static_cast<size_t>(std::max(m, 1)), -1);
#pragma omp for schedule(dynamic, 64)
        for (int i = 0; i < n; ++i) {
            int cnt = 0;
            for (int ka = a.rp[i]; ka < a.rp[i + 1]; ++ka) {
                const int k = a.ci[ka];
                for (int kb = b.rp[k]; kb < b.rp[k + 1]; ++kb) {
                    const int j = b.ci[kb];
                    if (mark[j] != i) {
                        mark[j] = i;
                        ++cnt;
                    }
                }
            }
            len[i] = cnt;
        }
    }
    long long total = 0;
    for (int i = 0; i < n; ++i) total += len[i];
    if (total > 0x7fffffffLL) {
        fail(1, "amg setup: a Galerkin product exceeds 2^31 nonzeros (coarse operators densify; "
                "lower strength_threshold)");
    }
    for (int i = 0; i < n; ++i) c.rp[i + 1] = c.rp[i] + len[i];
    c.ci.resize(static_cast<size_t>(c.rp[n]));
    c.va.resize(static_cast<size_t>(c.rp[n]));
#pragma omp parallel if (n > 256)
    {
        std::vector<int> mark(static_cast<size_t>(std::max(m, 1)), -1);
        std::vector<double> acc(static_cast<size_t>(std::max(m, 1)));
        std::vector<int> list;
#pragma omp for schedule(dynamic, 64)
        for (int i = 0; i < n; ++i) {
            list.clear();
            for (int ka = a.rp[i]; ka < a.rp[i + 1]; ++ka) {
                const int k = a.ci[ka];
                const double x = a.va[ka];
                for (int kb = b.rp[k]; kb < b.rp[k + 1]; ++kb) {
                    const int j = b.ci[kb];
                    if (mark[j] != i) {
                        mark[j] = i;
                        acc[j] = x * b.va[kb];
                        list.push_back(j);
                    } else {
                        acc[j] += x * b.va[kb];
                    }
                }
            }
            std::sort(list.begin(), list.end());
            int o = c.rp[i];
            for (const int j : list) {
                c.ci[o] = j;
                c.va[o] = acc[j];
                ++o;
            }
        }
    }
    return c;
}

void prune_zeros(HostCsr& m) {
    int nnz = 0;
    int start = 0;
    for (int i = 0; i < m.n_rows; ++i) {
        const int end = m.rp[i + 1];
        for (int k = start; k < end; ++k) {
            if (m.va[k] != 0.0) {
                m.ci[nnz] = m.ci[k];
                m.va[nnz] = m.va[k];
                ++nnz;
            }
        }
        start = end;
        m.rp[i + 1] = nnz;
    }
    m.ci.resize(static_cast<size_t>(nnz));
    m.va.resize(static_cast<size_t>(nnz));
}

// Rows of the transpose list their columns in ascending order (the order of the serial
// fill), built in parallel: each thread takes a contiguous block of rows of `a`, and the
// entries of its block follow those of the blocks before it in every output row.
HostCsr transpose(const HostCsr& a) {
    HostCsr t;
    t.n_rows = a.n_cols;
    t.n_cols = a.n_rows;
    const int m = a.n_cols;
    t.rp.assign(static_cast<size_t>(m) + 1, 0);
    t.ci.resize(static_cast<size_t>(a.nnz()));
    t.va.resize(static_cast<size_t>(a.nnz()));
    const int nt = a.n_rows > 4096 ? omp_get_max_threads() : 1;
    // The rows are split over the threads the team actually has: inside another parallel
    // region (a batch of systems set up in parallel) a nested team has one thread.
    std::vector<std::vector<int>> cnt;
    int team = 1;
#pragma omp parallel num_threads(nt) if (nt > 1)
    {
#pragma omp single
        {
            team = omp_get_num_threads();
            cnt.resize(static_cast<size_t>(team));
        }
        const int tid = omp_get_thread_num();
        const long long n_rows = a.n_rows;
        const int r0 = static_cast<int>(n_rows * tid / team);
        const int r1 = static_cast<int>(n_rows * (tid + 1) / team);
        std::vector<int>& c = cnt[static_cast<size_t>(tid)];
        c.assign(static_cast<size_t>(m), 0);
        for (int i = r0; i < r1; ++i)
            for (int k = a.rp[i]; k < a.rp[i + 1]; ++k) ++c[a.ci[k]];
#pragma omp barrier
#pragma omp single
        {
            // row lengths, then each thread's starting offset within every row
            for (int j = 0; j < m; ++j) {
                int len = 0;
                for (int q = 0; q < team; ++q) {
                    const int v = cnt[static_cast<size_t>(q)][j];
                    cnt[static_cast<size_t>(q)][j] = len;
                    len += v;
                }
                t.rp[j + 1] = len;
            }
            for (int j = 0; j < m; ++j) t.rp[j + 1] += t.rp[j];
        }
        for (int i = r0; i < r1; ++i) {
            for (int k = a.rp[i]; k < a.rp[i + 1]; ++k) {
                const int j = a.ci[k];
                const int o = t.rp[j] + c[j]++;
                t.ci[o] = i;
                t.va[o] = a.va[k];
            }
        }
    }
    return t;
}

std::vector<double> last_diagonal(const HostCsr& a) {
    std::vector<double> d(static_cast<size_t>(a.n_rows), 0.0);
#pragma omp parallel for schedule(static) if (a.n_rows > 100000)
    for (int i = 0; i < a.n_rows; ++i) {
        for (int k = a.rp[i]; k < a.rp[i + 1]; ++k) {
            if (a.ci[k] == i) d[i] = a.va[k];
        }
    }
    return d;
}

bool ldlt_factor(int n, const std::vector<double>& a, std::vector<double>& f) {
    f = a;
    for (int j = 0; j < n; ++j) {
        double d = f[static_cast<size_t>(j) * n + j];
        for (int k = 0; k < j; ++k) {
            const double l = f[static_cast<size_t>(j) * n + k];
            d -= l * l * f[static_cast<size_t>(k) * n + k];
        }
        if (d == 0.0 || !std::isfinite(d)) return false;
        f[static_cast<size_t>(j) * n + j] = d;
        // rows below the pivot are independent
#pragma omp parallel for schedule(static) if (n - j > 128)
        for (int i = j + 1; i < n; ++i) {
            double s = f[static_cast<size_t>(i) * n + j];
            for (int k = 0; k < j; ++k) {
                s -= f[static_cast<size_t>(i) * n + k] * f[static_cast<size_t>(j) * n + k] *
                     f[static_cast<size_t>(k) * n + k];
            }
            f[static_cast<size_t>(i) * n + j] = s / d;
        }
    }
    return true;
}

void ldlt_solve(int n, const std::vector<double>& f, const double* b, double* x) {
    for (int i = 0; i < n; ++i) {
        double s = b[i];
        for (int k = 0; k < i; ++k) s -= f[static_cast<size_t>(i) * n + k] * x[k];
        x[i] = s;
    }
    for (int i = 0; i < n; ++i) x[i] /= f[static_cast<size_t>(i) * n + i];
    for (int i = n - 1; i >= 0; --i) {
        double s = x[i];
        for (int k = i + 1; k < n; ++k) s -= f[static_cast<size_t>(k) * n + i] * x[k];
        x[i] = s;
    }
}

// Pseudo-inverse of a symmetric matrix through cyclic Jacobi eigen-decomposition.
void sym_pinv(int n, const std::vector<double>& a, std::vector<double>& out) {
    std::vector<double> m = a;
    std::vector<double> v(static_cast<size_t>(n) * n, 0.0);
    auto M = [&](int i, int j) -> double& { return m[static_cast<size_t>(i) * n + j]; };
    auto V = [&](int i, int j) -> double& { return v[static_cast<size_t>(i) * n + j]; };
    for (int i = 0; i < n; ++i) V(i, i) = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) off += M(p, q) * M(p, q);
        if (off < 1e-30) break;
        for (int p = 0; p < n; ++p) {
            for (int q = p + 1; q < n; ++q) {
                const double apq = M(p, q);
                if (std::fabs(apq) < 1e-300) continue;
                const double theta = (M(q, q) - M(p, p)) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; ++k) {
                    const double mkp = M(k, p), mkq = M(k, q);
                    M(k, p) = c * mkp - s * mkq;
                    M(k, q) = s * mkp + c * mkq;
                }
                for (int k = 0; k < n; ++k) {
                    const double mpk = M(p, k), mqk = M(q, k);
                    M(p, k) = c * mpk - s * mqk;
                    M(q, k) = s * mpk + c * mqk;
                }
                for (int k = 0; k < n; ++k) {
                    const double vkp = V(k, p), vkq = V(k, q);
                    V(k, p) = c * vkp - s * vkq;
                    V(k, q) = s * vkp + c * vkq;
                }
            }
        }
    }
    double lmax = 0.0;
    for (int i = 0; i < n; ++i) lmax = std::max(lmax, std::fabs(M(i, i)));
    const double tol = lmax * 2.220446049250313e-16 * n;
    out.assign(static_cast<size_t>(n) * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            double s = 0.0;
            for (int k = 0; k < n; ++k) {
                const double l = M(k, k);
                if (std::fabs(l) > tol) s += V(i, k) * V(j, k) / l;
            }
            out[static_cast<size_t>(i) * n + j] = s;
        }
}

} // namespace

double Hierarchy::operator_complexity() const {
    if (a.empty()) return 0.0;
    double t = 0.0;
    for (const auto& m : a) t += static_cast<double>(m.nnz());
    return t / static_cast<double>(a.front().nnz());
}

int aggregate(const HostCsr& a, const std::vector<double>& d, double theta, std::vector<int>& agg) {
    const int n = a.n_rows;
    agg.assign(static_cast<size_t>(n), -1);
    int n_agg = 0;
    for (int i = 0; i < n; ++i) {
        if (agg[i] >= 0) continue;
        bool is_free = true, has_strong = false;
        for (int k = a.rp[i]; k < a.rp[i + 1]; ++k) {
            if (strong(i, a.ci[k], a.va[k], d, theta)) {
                has_strong = true;
                if (agg[a.ci[k]] >= 0) {
                    is_free = false;
                    break;
                }
            }
        }
        if (!is_free || !has_strong) continue;
        agg[i] = n_agg;
        for (int k = a.rp[i]; k < a.rp[i + 1]; ++k) {
            if (strong(i, a.ci[k], a.va[k], d, theta)) agg[a.ci[k]] = n_agg;
        }
        ++n_agg;
    }
    const std::vector<int> pass1 = agg;
    for (int i = 0; i < n; ++i) {
        if (agg[i] >= 0) continue;
        double best = 0.0;
        for (int k = a.rp[i]; k < a.rp[i + 1]; ++k) {
            const int j = a.ci[k];
            if (strong(i, j, a.va[k], d, theta) && pass1[j] >= 0 && std::fabs(a.va[k]) > best) {
                best = std::fabs(a.va[k]);
                agg[i] = pass1[j];
            }
        }
    }
    for (int i = 0; i < n; ++i) {
        if (agg[i] < 0) {
            agg[i] = n_agg;
            for (int k = a.rp[i]; k < a.rp[i + 1]; ++k) {
                if (strong(i, a.ci[k], a.va[k], d, theta) && agg[a.ci[k]] < 0) agg[a.ci[k]] = n_agg;
            }
            ++n_agg;
        }
    }
    return n_agg;
}

int aggregate_strong(int n, const int* srp, const int* sci, const double* sav, std::vector<int>& agg) {
    agg.assign(static_cast<size_t>(n), -1);
    int n_agg = 0;
    // pass 1: seeds whose strong neighbourhood is non-empty and entirely unaggregated
    for (int i = 0; i < n; ++i) {
        if (agg[i] >= 0 || srp[i] == srp[i + 1]) continue;
        bool is_free = true;
        for (int k = srp[i]; k < srp[i + 1]; ++k) {
            if (agg[sci[k]] >= 0) {
                is_free = false;
                break;
            }
        }
        if (!is_free) continue;
        agg[i] = n_agg;
        for (int k = srp[i]; k < srp[i + 1]; ++k) agg[sci[k]] = n_agg;
        ++n_agg;
    }
    // pass 2: join the pass-1 aggregate of the strongest strong neighbour (strictly larger wins)
    const std::vector<int> pass1 = agg;
#pragma omp parallel for schedule(static) if (n > 65536)
    for (int i = 0; i < n; ++i) {
        if (agg[i] >= 0) continue;
        double best = 0.0;
        for (int k = srp[i]; k < srp[i + 1]; ++k) {
            const int j = sci[k];
            if (pass1[j] >= 0 && sav[k] > best) {
                best = sav[k];
                agg[i] = pass1[j];
            }
        }
    }
    // pass 3: leftovers seed new aggregates with their unaggregated strong neighbours
    for (int i = 0; i < n; ++i) {
        if (agg[i] < 0) {
            agg[i] = n_agg;
            for (int k = srp[i]; k < srp[i + 1]; ++k)
                if (agg[sci[k]] < 0) agg[sci[k]] = n_agg;
            ++n_agg;
        }
    }
    return n_agg;
}

int aggregate_strong_ranked(int n, const int* srp, const int* sci, const uint16_t* rank, std::vector<int>& agg) {
    agg.assign(static_cast<size_t>(n), -1);
    int n_agg = 0;
    for (int i = 0; i < n; ++i) {
        if (agg[i] >= 0 || srp[i] == srp[i + 1]) continue;
        bool is_free = true;
        for (int k = srp[i]; k < srp[i + 1]; ++k) {
            if (agg[sci[k]] >= 0) {
                is_free = false;
                break;
            }
        }
        if (!is_free) continue;
        agg[i] = n_agg;
        for (int k = srp[i]; k < srp[i + 1]; ++k) agg[sci[k]] = n_agg;
        ++n_agg;
    }
    const std::vector<int> pass1 = agg;
    // pass 2 reads only pass 1's result: rows are independent
#pragma omp parallel for schedule(static) if (n > 65536)
    for (int i = 0; i < n; ++i) {
        if (agg[i] >= 0) continue;
        int best = INT_MAX;
        for (int k = srp[i]; k < srp[i + 1]; ++k) {
            const int j = sci[k];
            if (pass1[j] >= 0 && rank[k] < best) {
                best = rank[k];
                agg[i] = pass1[j];
            }
        }
    }
    for (int i = 0; i < n; ++i) {
        if (agg[i] < 0) {
            agg[i] = n_agg;
            for (int k = srp[i]; k < srp[i + 1]; ++k)
                if (agg[sci[k]] < 0) agg[sci[k]] = n_agg;
            ++n_agg;
        }
    }
    return n_agg;
}

bool dense_inverse(int n, const std::vector<double>& a, std::vector<double>& inv) {
    std::vector<double> f;
    if (!ldlt_factor(n, a, f)) {
        sym_pinv(n, a, inv);
        return false;
    }
    inv.assign(static_cast<size_t>(n) * n, 0.0);
    // one independent solve per column
#pragma omp parallel if (n > 64)
    {
        std::vector<double> e(static_cast<size_t>(n), 0.0), col(static_cast<size_t>(n));
#pragma omp for schedule(static)
        for (int j = 0; j < n; ++j) {
            e[j] = 1.0;
            ldlt_solve(n, f, e.data(), col.data());
            e[j] = 0.0;
            for (int i = 0; i < n; ++i) inv[static_cast<size_t>(i) * n + j] = col[i];
        }
    }
    return true;
}

Hierarchy amg_setup(const HostCsr& a0, const AmgSettings& s) {
    if (a0.n_rows != a0.n_cols) fail(1, "AmgPreconditioner: matrix must be square");
    if (a0.n_rows <= 0) fail(1, "amg_setup: empty matrix");
    Hierarchy h;
    HostCsr cur = a0;
    for (int l = 0; l < s.max_levels; ++l) {
        const int nl = cur.n_rows;
        const std::vector<double> d = last_diagonal(cur);
        const bool last = nl <= s.coarse_size || l + 1 == s.max_levels;
        if (last) {
            h.a.push_back(std::move(cur));
            break;
        }
        std::vector<int> agg;
        const int n_agg = aggregate(cur, d, s.theta, agg);
        if (n_agg >= nl || n_agg == 0) {
            h.a.push_back(std::move(cur));
            break;
        }
        std::vector<double> inv(static_cast<size_t>(nl));
        for (int i = 0; i < nl; ++i) inv[i] = d[i] != 0.0 ? 1.0 / d[i] : 0.0;
        double rho = 0.0;
#pragma omp parallel for reduction(max : rho) schedule(static) if (nl > 2048)
        for (int i = 0; i < nl; ++i) {
            double row = 0.0;
            for (int k = cur.rp[i]; k < cur.rp[i + 1]; ++k) row += std::fabs(cur.va[k]);
            rho = std::max(rho, row * std::fabs(inv[i]));
        }
        const double omega = rho > 0.0 ? 4.0 / (3.0 * rho) : 0.0;
        // P = P_tent - omega * (D^-1 A) P_tent over the union pattern, pruned (amg.cpp:168-172).
        // Row i of (D^-1 A) P_tent accumulates (inv_i * a_ik) * 1.0 into column agg[k], k ascending.
        HostCsr p;
        p.n_rows = nl;
        p.n_cols = n_agg;
        p.rp.assign(static_cast<size_t>(nl) + 1, 0);
        std::vector<int> plen(static_cast<size_t>(nl));
        std::vector<std::vector<int>> pc_t;
        std::vector<std::vector<double>> pv_t;
        const int nthreads = omp_get_max_threads();
        pc_t.resize(static_cast<size_t>(nthreads));
        pv_t.resize(static_cast<size_t>(nthreads));
        std::vector<int> row_start(static_cast<size_t>(nl));
        std::vector<int> row_tid(static_cast<size_t>(nl));
#pragma omp parallel if (nl > 2048)
        {
            const int tid = omp_get_thread_num();
            std::vector<int> mark(static_cast<size_t>(n_agg), -1);
            std::vector<double> acc(static_cast<size_t>(n_agg));
            std::vector<int> list;
            auto& oc = pc_t[tid];
            auto& ov = pv_t[tid];
#pragma omp for schedule(static)
            for (int i = 0; i < nl; ++i) {
                list.clear();
                for (int k = cur.rp[i]; k < cur.rp[i + 1]; ++k) {
                    const int j = agg[cur.ci[k]];
                    const double v = (inv[i] * cur.va[k]) * 1.0;
                    if (mark[j] != i) {
                        mark[j] = i;
                        acc[j] = v;
                        list.push_back(j);
                    } else {
                        acc[j] += v;
                    }
                }
                std::sort(list.begin(), list.end());
                row_start[i] = static_cast<int>(oc.size());
                row_tid[i] = tid;
                const int tj = agg[i];
                bool used = false;
                int cnt = 0;
                auto emit = [&](int j, double v) {
                    if (v != 0.0) {
                        oc.push_back(j);
                        ov.push_back(v);
                        ++cnt;
                    }
                };
                for (const int j : list) {
                    const double ws = omega * acc[j];
                    if (!used && tj < j) {
                        emit(tj, 1.0 - 0.0);
                        used = true;
                    }
                    if (j == tj) {
                        emit(j, 1.0 - ws);
                        used = true;
                    } else {
                        emit(j, 0.0 - ws);
                    }
                }
                if (!used) emit(tj, 1.0 - 0.0);
                plen[i] = cnt;
            }
        }
        for (int i = 0; i < nl; ++i) p.rp[i + 1] = p.rp[i] + plen[i];
        p.ci.resize(static_cast<size_t>(p.rp[nl]));
        p.va.resize(static_cast<size_t>(p.rp[nl]));
        // gather the per-thread row buffers back in row order
#pragma omp parallel for schedule(static) if (nl > 2048)
        for (int i = 0; i < nl; ++i) {
            const int src = row_start[i];
            const int t = row_tid[i];
            std::memcpy(p.ci.data() + p.rp[i], pc_t[t].data() + src, sizeof(int) * plen[i]);
            std::memcpy(p.va.data() + p.rp[i], pv_t[t].data() + src, sizeof(double) * plen[i]);
        }
        HostCsr r = transpose(p);
        HostCsr ap = spgemm(cur, p);
        HostCsr coarse = spgemm(r, ap);
        prune_zeros(coarse);
        h.a.push_back(std::move(cur));
        h.p.push_back(std::move(p));
        h.r.push_back(std::move(r));
        h.agg.push_back(std::move(agg));
        h.n_agg.push_back(n_agg);
        cur = std::move(coarse);
    }
    const HostCsr& c = h.a.back();
    h.n_c = c.n_rows;
    std::vector<double> dense(static_cast<size_t>(h.n_c) * h.n_c, 0.0);
    for (int i = 0; i < h.n_c; ++i)
        for (int k = c.rp[i]; k < c.rp[i + 1]; ++k) dense[static_cast<size_t>(i) * h.n_c + c.ci[k]] += c.va[k];
    h.ldlt_ok = dense_inverse(h.n_c, dense, h.coarse_inverse);
    return h;
}

} // namespace cfdb
