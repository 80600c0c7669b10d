// C++ driver of the cfd::gpu front end (include/cfd_gpu_krylov.hpp), written the way the
// reference's own accelerator tests use that surface (test_gpu.cpp): a manufactured 2-D
// five-point problem, the converged-input rule, the persistent LDU solver with an AMG
// hierarchy, the assembly formulas and the error types. Exit status 0 when every check passes.
//
//   test_cfd_gpu_api            checks on the GPU
//   test_cfd_gpu_api --no-device  checks the no-device behaviour (no host fallback)
#include <cfd_gpu_fv.hpp>
#include <cfd_gpu_krylov.hpp>
#include <cfdb.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <vector>

namespace g = cfd::gpu;

static int failures = 0;
#define CHECK(cond)                                                                    \
    do {                                                                               \
        if (!(cond)) {                                                                 \
            std::fprintf(stderr, "%s:%d: check failed: %s\n", __FILE__, __LINE__, #cond); \
            ++failures;                                                                \
        }                                                                              \
    } while (0)

template <class E, class F> static bool throws(F&& f) {
    try {
        f();
    } catch (const E&) {
        return true;
    } catch (...) {
        return false;
    }
    return false;
}

// 2-D five-point Laplacian (Dirichlet) on an m x m grid, CSR with sorted columns.
struct Csr {
    int n = 0;
    std::vector<int> rp, ci;
    std::vector<double> va;
    g::CsrView view() const { return g::CsrView{n, static_cast<int>(va.size()), rp.data(), ci.data(), va.data()}; }
};

static Csr five_point(int m) {
    Csr a;
    a.n = m * m;
    a.rp.push_back(0);
    for (int j = 0; j < m; ++j)
        for (int i = 0; i < m; ++i) {
            const int r = j * m + i;
            if (j > 0) a.ci.push_back(r - m), a.va.push_back(-1.0);
            if (i > 0) a.ci.push_back(r - 1), a.va.push_back(-1.0);
            a.ci.push_back(r), a.va.push_back(4.0);
            if (i + 1 < m) a.ci.push_back(r + 1), a.va.push_back(-1.0);
            if (j + 1 < m) a.ci.push_back(r + m), a.va.push_back(-1.0);
            a.rp.push_back(static_cast<int>(a.ci.size()));
        }
    return a;
}

static std::vector<double> matvec(const Csr& a, const std::vector<double>& x) {
    std::vector<double> y(a.n, 0.0);
    for (int r = 0; r < a.n; ++r)
        for (int k = a.rp[r]; k < a.rp[r + 1]; ++k) y[r] += a.va[k] * x[a.ci[k]];
    return y;
}

static double norm(const std::vector<double>& v) {
    double s = 0.0;
    for (double e : v) s += e * e;
    return std::sqrt(s);
}

static double residual(const Csr& a, const std::vector<double>& b, const std::vector<double>& x) {
    std::vector<double> ax = matvec(a, x);
    for (int i = 0; i < a.n; ++i) ax[i] = b[i] - ax[i];
    return norm(ax);
}

// Box mesh n x n x n: internal faces ordered by (owner, neighbour), owner < neighbour.
struct Box {
    int n_cells = 0;
    std::vector<int> owner, neighbour;
};

static Box box(int m) {
    Box b;
    b.n_cells = m * m * m;
    auto id = [m](int i, int j, int k) { return (k * m + j) * m + i; };
    for (int k = 0; k < m; ++k)
        for (int j = 0; j < m; ++j)
            for (int i = 0; i < m; ++i) {
                const int c = id(i, j, k);
                if (i + 1 < m) b.owner.push_back(c), b.neighbour.push_back(id(i + 1, j, k));
                if (j + 1 < m) b.owner.push_back(c), b.neighbour.push_back(id(i, j + 1, k));
                if (k + 1 < m) b.owner.push_back(c), b.neighbour.push_back(id(i, j, k + 1));
            }
    return b;
}

// A row of n unit cubes along x (cell c centred at (c + 0.5, 0.5, 0.5)) as an FvMeshView: the
// n - 1 internal faces first, then per cell its boundary faces. Least-squares matrices are
// inverted by cofactors.
struct FvRow {
    int n, nif, nf;
    std::vector<int> own, nei, off, faces;
    std::vector<double> w, sf, cf, cc, vol, kv, lsq_d, lsq;
    explicit FvRow(int cells) : n(cells), nif(cells - 1) {
        for (int c = 0; c + 1 < n; ++c) face(c, c + 1, {1, 0, 0}, {c + 1.0, 0.5, 0.5});
        for (int c = 0; c < n; ++c) {
            if (c == 0) face(c, -1, {-1, 0, 0}, {0.0, 0.5, 0.5});
            if (c == n - 1) face(c, -1, {1, 0, 0}, {double(n), 0.5, 0.5});
            face(c, -1, {0, -1, 0}, {c + 0.5, 0.0, 0.5});
            face(c, -1, {0, 1, 0}, {c + 0.5, 1.0, 0.5});
            face(c, -1, {0, 0, -1}, {c + 0.5, 0.5, 0.0});
            face(c, -1, {0, 0, 1}, {c + 0.5, 0.5, 1.0});
        }
        nf = static_cast<int>(own.size());
        for (int c = 0; c < n; ++c) {
            cc.insert(cc.end(), {c + 0.5, 0.5, 0.5});
            vol.push_back(1.0);
        }
        std::vector<std::vector<int>> lists(n);
        std::vector<double> m(9 * n, 0.0);
        for (int f = 0; f < nf; ++f) {
            const int p = own[f];
            double d[3];
            for (int i = 0; i < 3; ++i) d[i] = (f < nif ? cc[3 * nei[f] + i] : cf[3 * f + i]) - cc[3 * p + i];
            const double dd = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            for (int i = 0; i < 3; ++i) {
                lsq_d.push_back(d[i] / dd);
                kv.push_back(0.0); // orthogonal: S = d delta
            }
            for (int c : {p, f < nif ? nei[f] : -1}) {
                if (c < 0) continue;
                lists[c].push_back(f);
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) m[9 * c + 3 * j + i] += d[i] * d[j] / dd;
            }
        }
        off.push_back(0);
        for (int c = 0; c < n; ++c) {
            faces.insert(faces.end(), lists[c].begin(), lists[c].end());
            off.push_back(static_cast<int>(faces.size()));
            const double* a = &m[9 * c];
            auto at = [&](int r, int k) { return a[3 * k + r]; };
            double inv[9];
            const double det = at(0, 0) * (at(1, 1) * at(2, 2) - at(1, 2) * at(2, 1)) -
                               at(0, 1) * (at(1, 0) * at(2, 2) - at(1, 2) * at(2, 0)) +
                               at(0, 2) * (at(1, 0) * at(2, 1) - at(1, 1) * at(2, 0));
            for (int r = 0; r < 3; ++r)
                for (int k = 0; k < 3; ++k) {
                    const int r1 = (k + 1) % 3, r2 = (k + 2) % 3, k1 = (r + 1) % 3, k2 = (r + 2) % 3;
                    inv[3 * k + r] = (at(r1, k1) * at(r2, k2) - at(r1, k2) * at(r2, k1)) / det;
                }
            lsq.insert(lsq.end(), inv, inv + 9);
        }
    }
    void face(int p, int q, std::initializer_list<double> s, std::initializer_list<double> x) {
        own.push_back(p);
        if (q >= 0) {
            nei.push_back(q);
            w.push_back(0.5);
        }
        sf.insert(sf.end(), s);
        cf.insert(cf.end(), x);
    }
    g::FvMeshView view() const {
        g::FvMeshView v;
        v.n_cells = n;
        v.n_internal_faces = nif;
        v.n_faces = nf;
        v.owner = own.data();
        v.neighbour = nei.data();
        v.cell_offsets = off.data();
        v.cell_faces = faces.data();
        v.weight = w.data();
        v.sf = sf.data();
        v.face_centre = cf.data();
        v.cell_centre = cc.data();
        v.volume = vol.data();
        v.correction = kv.data();
        v.lsq_d = lsq_d.data();
        v.lsq_inverse = lsq.data();
        return v;
    }
};

// DeviceFv (fv_device.hpp): linear fields have exact gradients with every scheme on this
// orthogonal row; errors are the reference's exception types.
static void check_device_fv() {
    const FvRow row(5);
    g::DeviceFv fv(row.view());
    CHECK(fv.on_device());
    const double a[3] = {2.0, 3.0, -1.0};
    auto lin = [&](const double* x) { return a[0] * x[0] + a[1] * x[1] + a[2] * x[2] + 0.5; };
    std::vector<double> phi(row.n), bv(row.nf - row.nif), u(3 * row.n), ub(3 * (row.nf - row.nif));
    for (int c = 0; c < row.n; ++c) {
        phi[c] = lin(&row.cc[3 * c]);
        for (int i = 0; i < 3; ++i) u[3 * c + i] = (i + 1) * phi[c];
    }
    for (int f = row.nif; f < row.nf; ++f) {
        bv[f - row.nif] = lin(&row.cf[3 * f]);
        for (int i = 0; i < 3; ++i) ub[3 * (f - row.nif) + i] = (i + 1) * bv[f - row.nif];
    }
    std::vector<double> nu(row.nif, 0.1), flux(row.nif, 1.0);
    std::vector<double> src(3 * row.n, 0.0);
    CHECK(throws<std::logic_error>([&] {
        fv.momentum_corrections(flux.data(), nu.data(), true, false, false, nullptr, 0.0, false, src.data());
    }));
    for (int scheme = 0; scheme < 3; ++scheme) {
        std::vector<double> grad(3 * row.n), vg(9 * row.n);
        fv.gradient(phi.data(), bv.data(), scheme, grad.data());
        fv.vector_gradient(u.data(), ub.data(), scheme, vg.data());
        double err = 0.0;
        for (int c = 0; c < row.n; ++c)
            for (int j = 0; j < 3; ++j) {
                err = std::fmax(err, std::fabs(grad[3 * c + j] - a[j]));
                for (int i = 0; i < 3; ++i) err = std::fmax(err, std::fabs(vg[9 * c + 3 * i + j] - (i + 1) * a[j]));
            }
        CHECK(err < 1e-12);
    }
    // uniform flux through orthogonal faces with a linear field: the linear-upwind corrections
    // telescope to F (phi_f - phi_up) differences; the interior cells receive the same source
    std::vector<double> s(row.n, 0.0);
    fv.scalar_corrections(phi.data(), bv.data(), 1, flux.data(), nu.data(), true, s.data());
    CHECK(std::fabs(s[0] + 1.0) < 1e-12 && std::fabs(s[row.n - 1] - 1.0) < 1e-12);
    for (int c = 1; c + 1 < row.n; ++c) CHECK(std::fabs(s[c]) < 1e-12);
    fv.momentum_corrections(flux.data(), nu.data(), true, true, false, nullptr, 0.0, true, src.data());
    CHECK(std::isfinite(src[0]));
    CHECK(throws<std::invalid_argument>([&] { fv.gradient(phi.data(), bv.data(), 7, phi.data()); }));
    g::FvMeshView bad = row.view();
    bad.n_faces = bad.n_internal_faces - 1;
    CHECK(throws<std::invalid_argument>([&] { g::DeviceFv x(bad); }));
}

static void check_no_device() {
    CHECK(g::backend_name() == "cuda");
    CHECK(!g::device_available());
    Csr a = five_point(4);
    std::vector<double> b(a.n, 1.0), x(a.n, 0.0);
    CHECK(throws<std::runtime_error>([&] { g::solve(a.view(), b.data(), x.data(), g::Method::Cg, {}); }));
    const FvRow row(3);
    CHECK(throws<std::runtime_error>([&] { g::DeviceFv fv(row.view()); }));
}

static void check_device() {
    CHECK(g::backend_name() == "cuda");
    CHECK(g::device_available());
    CHECK(!g::device_description().empty());

    // manufactured 2-D problem, Jacobi CG
    Csr a = five_point(48);
    std::vector<double> xs(a.n), x(a.n, 0.0);
    for (int i = 0; i < a.n; ++i) xs[i] = std::sin(0.3 * i) + 1.0;
    const std::vector<double> b = matvec(a, xs);
    g::SolveControl ctl;
    ctl.abs_tolerance = 1e-10 * norm(b);
    ctl.max_iterations = 2000;
    const g::SolveStats st = g::solve(a.view(), b.data(), x.data(), g::Method::Cg, ctl);
    CHECK(st.converged && st.on_device);
    CHECK(residual(a, b, x) <= 1.01 * ctl.abs_tolerance);
    // an already converged input returns at once
    const g::SolveStats st0 = g::solve(a.view(), b.data(), xs.data(), g::Method::Cg, ctl);
    CHECK(st0.converged && st0.iterations == 0);
    // Jacobi-preconditioned BiCGStab (the momentum solver) on the same problem
    std::vector<double> xb(a.n, 0.0);
    const g::SolveStats sb = g::solve(a.view(), b.data(), xb.data(), g::Method::BiCgStab, ctl);
    CHECK(sb.converged && sb.on_device && sb.iterations > 0);
    CHECK(residual(a, b, xb) <= 1.01 * ctl.abs_tolerance);

    // assembly formulas (pure diffusion: upper = lower = -gamma * delta)
    const Box m = box(12);
    const int nf = static_cast<int>(m.owner.size());
    std::vector<double> flux(nf), gamma(nf), delta(nf), up(nf), lo(nf), dg(m.n_cells, 0.0), dv(m.n_cells, 0.0);
    for (int f = 0; f < nf; ++f) {
        flux[f] = std::sin(0.7 * f);
        gamma[f] = 1.0 + 0.5 * std::cos(0.1 * f);
        delta[f] = 2.0 + 0.25 * std::sin(0.05 * f);
    }
    g::assemble_convection_diffusion(m.n_cells, nf, m.owner.data(), m.neighbour.data(), flux.data(), gamma.data(),
                                     delta.data(), 0.0, up.data(), lo.data(), dg.data(), dv.data());
    bool exact = true;
    for (int f = 0; f < nf; ++f) exact = exact && up[f] == -(gamma[f] * delta[f]) && lo[f] == up[f];
    CHECK(exact);
    double dsum = 0.0, osum = 0.0, divsum = 0.0;
    for (int c = 0; c < m.n_cells; ++c) dsum += dg[c], divsum += dv[c];
    for (int f = 0; f < nf; ++f) osum += up[f] + lo[f];
    CHECK(std::fabs(dsum + osum) <= 1e-9 * dsum && std::fabs(divsum) <= 1e-9);

    // persistent LDU solver with an AMG hierarchy (pressure system with a reference cell)
    std::vector<int> rp(m.n_cells + 1), col(m.n_cells + 2 * nf), dpos(m.n_cells), upos(nf), lpos(nf);
    int nnz = 0;
    if (cfdb_build_pattern(m.n_cells, nf, m.owner.data(), m.neighbour.data(), rp.data(), col.data(), dpos.data(),
                           upos.data(), lpos.data(), &nnz) != CFDB_OK) {
        CHECK(false);
        return;
    }
    dg[0] += dg[0];
    std::vector<double> vals(nnz, 0.0);
    for (int c = 0; c < m.n_cells; ++c) vals[dpos[c]] = dg[c];
    for (int f = 0; f < nf; ++f) vals[upos[f]] = up[f], vals[lpos[f]] = lo[f];
    const cfdb_csr ac{m.n_cells, nnz, rp.data(), col.data(), vals.data()};
    cfdb_amg_settings set;
    cfdb_default_amg_settings(&set);
    set.strength_threshold = 0.04;
    cfdb_hierarchy* h = nullptr;
    CHECK(cfdb_amg_setup(&ac, &set, &h) == CFDB_OK);
    cfdb_amg_view cv{};
    CHECK(cfdb_hierarchy_view(h, 2, 0.7, &cv) == CFDB_OK);
    CHECK(cv.n_levels >= 2);
    g::AmgView amg;
    auto cpp = [](const cfdb_csr& c) { return g::CsrView{c.n, c.nnz, c.row_ptr, c.col, c.val}; };
    for (int l = 0; l < cv.n_levels; ++l) amg.levels.push_back({cpp(cv.levels[l].a), cpp(cv.levels[l].p), cpp(cv.levels[l].r)});
    amg.coarse_inverse = cv.coarse_inverse;

    const g::LduPattern pat{m.n_cells, nf, nnz, rp.data(), col.data(), dpos.data(), upos.data(), lpos.data()};
    g::DeviceSolver ds(pat);
    CHECK(ds.on_device() == (g::device_available() && g::backend_name() == "cuda"));
    CHECK(throws<std::invalid_argument>([&] { ds.set_amg(g::AmgView{}); }));
    ds.set_amg(amg);
    Csr A;
    A.n = m.n_cells;
    A.rp = rp;
    A.ci.assign(col.begin(), col.begin() + nnz);
    A.va = vals;
    std::vector<double> rhs(m.n_cells);
    double mean = 0.0;
    for (int c = 0; c < m.n_cells; ++c) mean += (rhs[c] = std::cos(0.37 * c));
    for (double& v : rhs) v -= mean / m.n_cells;
    for (int mixed = 0; mixed < 2; ++mixed) {
        ds.set_mixed_precision(mixed != 0);
        std::vector<double> xp(m.n_cells, 0.0);
        g::SolveControl c2;
        c2.abs_tolerance = 1e-8 * norm(rhs);
        c2.max_iterations = 200;
        const g::SolveStats s2 = ds.solve(dg.data(), up.data(), lo.data(), rhs.data(), xp.data(), g::Method::Cg, true, c2);
        CHECK(s2.converged && s2.on_device && s2.iterations < 60);
        CHECK(residual(A, rhs, xp) <= 1.01 * c2.abs_tolerance);
        // Jacobi CG through the same persistent solver
        std::vector<double> xj(m.n_cells, 0.0);
        c2.max_iterations = 2000;
        const g::SolveStats s3 = ds.solve(dg.data(), up.data(), lo.data(), rhs.data(), xj.data(), g::Method::Cg, false, c2);
        CHECK(s3.converged && s3.iterations > s2.iterations);
    }
    // extensions: hierarchy built on the device, and LduMatrix::solve with its AmgCache
    {
        g::DeviceSolver dd(pat);
        g::AmgSetupSettings as;
        as.strength_threshold = 0.04;
        dd.setup_amg(dg.data(), up.data(), lo.data(), as);
        std::vector<double> xd(m.n_cells, 0.0);
        g::SolveControl c4;
        c4.abs_tolerance = 1e-8 * norm(rhs);
        c4.max_iterations = 200;
        const g::SolveStats s4 = dd.solve(dg.data(), up.data(), lo.data(), rhs.data(), xd.data(), g::Method::Cg, true, c4);
        CHECK(s4.converged && s4.iterations < 60);
        g::LduSolveSettings ls;
        ls.tolerance = 1e-14;
        ls.rel_tolerance = 1e-8;
        ls.max_age = 2;
        bool pattern_ok = true;
        for (int call = 0; call < 3; ++call) {
            std::vector<double> xl(m.n_cells, 0.0);
            const g::LduSolveResult r = dd.solve_ldu(dg.data(), up.data(), lo.data(), rhs.data(), xl.data(), ls, as);
            pattern_ok = pattern_ok && r.amg_rebuilt == (call != 1) && r.iterations > 0;
            CHECK(r.initial_residual > 0.0 && r.final_residual < 1e-6 * r.initial_residual);
            CHECK(residual(A, rhs, xl) <= 1.01e-8 * norm(rhs));
        }
        CHECK(pattern_ok);
    }
    cfdb_hierarchy_destroy(h);
}

int main(int argc, char** argv) {
    const bool no_device = argc > 1 && std::strcmp(argv[1], "--no-device") == 0;
    try {
        if (no_device) check_no_device();
        else {
            check_device();
            check_device_fv();
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "unexpected exception: %s\n", e.what());
        return 2;
    }
    if (failures == 0) std::printf("all checks passed\n");
    return failures == 0 ? 0 : 1;
}
