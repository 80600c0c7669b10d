// C-ABI shim over the reference's Eigen-dependent host sources (TEST INFRASTRUCTURE ONLY).
//
// oracle/build.py compiles the reference's unchanged
//   src/mesh/src/{mesh.cpp, mesh_builder.cpp, box_mesher.cpp}   (mesh, face ordering, geometry)
//   src/fv/src/fv_geometry.cpp                                  (delta coefficients, weights)
//   src/fv/src/ldu_matrix.cpp                                   (LduMatrix, build_csr_pattern,
//                                                                solve / solve_persistent)
//   src/fv/src/amg.cpp, parallel_amg.cpp, src/parallel/src/comm.cpp
// against the header-only Eigen stand-in in oracle/eigen_standin (Eigen is not in the image),
// together with this shim and the accelerator host path (ref_shim.cpp), into
// oracle/_ref/libcfdref.so. Integer results (face ordering, CSR pattern, aggregates) are the
// reference's own; floating-point results follow Eigen as far as the stand-in does (its header
// states where it does and where it does not).
//
// The two generators at the end (jittered lattice points, pressure inputs) are NOT reference
// code: they restate this project's synthetic workload definitions so that the reference arm of
// the benchmark can build its inputs without the product library.
#include <cfd/fv/amg.hpp>
#include <cfd/fv/fv_geometry.hpp>
#include <cfd/fv/ldu_matrix.hpp>
#include <cfd/mesh/box_mesher.hpp>
#include <cfd/mesh/mesh_builder.hpp>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <exception>
#include <memory>
#include <random>
#include <span>
#include <string>
#include <vector>

namespace {

using cfd::core::Label;
using cfd::core::Scalar;
using cfd::core::Vec3;
using cfd::fv::CsrMatrix;

struct LduHandle {
    std::unique_ptr<cfd::mesh::Mesh> mesh_copy; // when built from arrays
    const cfd::mesh::Mesh* mesh = nullptr;
    cfd::fv::CsrPattern pattern;
    std::unique_ptr<cfd::fv::LduMatrix> ldu;
    cfd::fv::AmgCache cache;
};

CsrMatrix csr_from(int n_rows, int n_cols, const int* rp, const int* ci, const double* va) {
    CsrMatrix m(n_rows, n_cols);
    m.outer_.assign(rp, rp + n_rows + 1);
    m.inner_.assign(ci, ci + rp[n_rows]);
    m.val_.assign(va, va + rp[n_rows]);
    return m;
}

template <typename F> int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

} // namespace

extern "C" {

// ---- mesh (mesh_builder.cpp, mesh.cpp, box_mesher.cpp) ---------------------------------------

// cfd::mesh::make_box_mesh on the unit cube with per-direction grading (box_mesher.cpp:30-143).
void* refx_box_mesh(int nx, int ny, int nz, double gx, double gy, double gz) {
    try {
        cfd::mesh::BoxSpec spec;
        spec.nx = nx;
        spec.ny = ny;
        spec.nz = nz;
        spec.grading = Vec3(gx, gy, gz);
        return new cfd::mesh::Mesh(cfd::mesh::make_box_mesh(spec));
    } catch (const std::exception&) {
        return nullptr;
    }
}

// cfd::mesh::MeshBuilder (mesh_builder.cpp:51-233): cells of one shape (4 nodes: tets, 8 nodes:
// hexes), boundary faces tagged with patches "p0".."p{n_patches-1}" declared in order (3 or 4
// nodes each; tag_nodes padded with -1 to 4 per face).
void* refx_mesh_build(int n_points, const double* points, int n_cells, int nodes_per_cell,
                      const int* cells, int n_tags, const int* tag_nodes, const int* tag_patch,
                      int n_patches) {
    try {
        std::vector<Vec3> pts(static_cast<std::size_t>(n_points));
        for (int i = 0; i < n_points; ++i) {
            pts[static_cast<std::size_t>(i)] = Vec3(points[3 * i], points[3 * i + 1], points[3 * i + 2]);
        }
        cfd::mesh::MeshBuilder b(std::move(pts));
        const auto shape = nodes_per_cell == 4 ? cfd::mesh::CellShape::Tet : cfd::mesh::CellShape::Hex;
        for (int c = 0; c < n_cells; ++c) {
            b.add_cell(shape, std::span<const Label>(cells + static_cast<std::ptrdiff_t>(c) * nodes_per_cell,
                                                     static_cast<std::size_t>(nodes_per_cell)));
        }
        std::vector<std::string> names;
        for (int p = 0; p < n_patches; ++p) {
            names.push_back("p" + std::to_string(p));
            b.add_patch(names.back(), cfd::mesh::PatchType::Wall);
        }
        for (int t = 0; t < n_tags; ++t) {
            const int* q = tag_nodes + 4 * t;
            const int nn = q[3] < 0 ? 3 : 4;
            b.add_boundary_face(std::span<const Label>(q, static_cast<std::size_t>(nn)),
                                names[static_cast<std::size_t>(tag_patch[t])]);
        }
        return new cfd::mesh::Mesh(b.build());
    } catch (const std::exception&) {
        return nullptr;
    }
}

void refx_mesh_destroy(void* h) { delete static_cast<cfd::mesh::Mesh*>(h); }

void refx_mesh_sizes(const void* h, int* n_cells, int* n_faces, int* n_internal, int* n_points,
                     int* n_face_nodes) {
    const auto* m = static_cast<const cfd::mesh::Mesh*>(h);
    *n_cells = m->n_cells();
    *n_faces = m->n_faces();
    *n_internal = m->n_internal_faces();
    *n_points = m->n_points();
    int total = 0;
    for (Label f = 0; f < m->n_faces(); ++f) total += static_cast<int>(m->face(f).size());
    *n_face_nodes = total;
}

// owner[n_faces], neighbour[n_internal], face offsets[n_faces + 1] and nodes, patch ranges.
void refx_mesh_topology(const void* h, int* owner, int* neighbour, int* face_offsets, int* face_nodes) {
    const auto* m = static_cast<const cfd::mesh::Mesh*>(h);
    std::copy(m->owner().begin(), m->owner().end(), owner);
    std::copy(m->neighbour().begin(), m->neighbour().end(), neighbour);
    int k = 0;
    face_offsets[0] = 0;
    for (Label f = 0; f < m->n_faces(); ++f) {
        for (const Label v : m->face(f)) face_nodes[k++] = v;
        face_offsets[f + 1] = k;
    }
}

// face centres and area vectors [3 n_faces], cell centres [3 n_cells], volumes [n_cells].
void refx_mesh_geometry(const void* h, double* face_centres, double* face_areas, double* cell_centres,
                        double* volumes) {
    const auto* m = static_cast<const cfd::mesh::Mesh*>(h);
    for (Label f = 0; f < m->n_faces(); ++f) {
        for (int a = 0; a < 3; ++a) {
            face_centres[3 * f + a] = m->face_centres()[static_cast<std::size_t>(f)][a];
            face_areas[3 * f + a] = m->face_area_vectors()[static_cast<std::size_t>(f)][a];
        }
    }
    for (Label c = 0; c < m->n_cells(); ++c) {
        for (int a = 0; a < 3; ++a) cell_centres[3 * c + a] = m->cell_centres()[static_cast<std::size_t>(c)][a];
        volumes[c] = m->cell_volumes()[static_cast<std::size_t>(c)];
    }
}

// cfd::fv::FvGeometry (fv_geometry.cpp:17-69): delta coefficients [n_faces], weights
// [n_internal]; and its CSR pattern (build_csr_pattern, ldu_matrix.cpp:572-612).
int refx_fv_geometry(const void* h, double* delta, double* weights, int* row_ptr, int* col, int* diag_pos,
                     int* upper_pos, int* lower_pos) {
    return guarded([&] {
        const auto* m = static_cast<const cfd::mesh::Mesh*>(h);
        const cfd::fv::FvGeometry g(*m);
        std::copy(g.delta_coeffs().begin(), g.delta_coeffs().end(), delta);
        std::copy(g.weights().begin(), g.weights().end(), weights);
        const auto& p = g.csr_pattern();
        const auto n = static_cast<std::size_t>(m->n_cells());
        std::copy(p.structure.outerIndexPtr(), p.structure.outerIndexPtr() + n + 1, row_ptr);
        std::copy(p.structure.innerIndexPtr(), p.structure.innerIndexPtr() + p.structure.nonZeros(), col);
        std::copy(p.diag_pos.begin(), p.diag_pos.end(), diag_pos);
        std::copy(p.upper_pos.begin(), p.upper_pos.end(), upper_pos);
        std::copy(p.lower_pos.begin(), p.lower_pos.end(), lower_pos);
    });
}

int refx_pattern_nnz(const void* h) {
    const auto* m = static_cast<const cfd::mesh::Mesh*>(h);
    return m->n_cells() + 2 * m->n_internal_faces();
}

// ---- AMG (amg.cpp) ----------------------------------------------------------------------------

void* refx_amg_setup(int n, const int* rp, const int* ci, const double* va, double theta, int max_levels,
                     int coarse_size) {
    try {
        cfd::fv::AmgSettings s;
        s.strength_threshold = theta;
        s.max_levels = max_levels;
        s.coarse_size = coarse_size;
        auto amg = std::make_unique<cfd::fv::AmgPreconditioner>(s);
        amg->setup(csr_from(n, n, rp, ci, va));
        return amg.release();
    } catch (const std::exception&) {
        return nullptr;
    }
}

void refx_amg_destroy(void* h) { delete static_cast<cfd::fv::AmgPreconditioner*>(h); }

int refx_amg_levels(const void* h) { return static_cast<const cfd::fv::AmgPreconditioner*>(h)->levels(); }

double refx_amg_operator_complexity(const void* h) {
    return static_cast<const cfd::fv::AmgPreconditioner*>(h)->operator_complexity();
}

// which: 0 = A, 1 = P, 2 = R of a level. Pointers stay valid while the hierarchy lives.
int refx_amg_level(const void* h, int level, int which, int* rows, int* cols, int* nnz, const int** rp,
                   const int** ci, const double** va) {
    const auto* amg = static_cast<const cfd::fv::AmgPreconditioner*>(h);
    if (level < 0 || level >= amg->levels() || (which > 0 && level + 1 >= amg->levels())) return 1;
    const CsrMatrix& m = which == 0   ? amg->level_matrix(level)
                         : which == 1 ? amg->level_prolongation(level)
                                      : amg->level_restriction(level);
    *rows = static_cast<int>(m.rows());
    *cols = static_cast<int>(m.cols());
    *nnz = static_cast<int>(m.nonZeros());
    *rp = m.outerIndexPtr();
    *ci = m.innerIndexPtr();
    *va = m.valuePtr();
    return 0;
}

// AmgPreconditioner::coarse_inverse (amg.cpp:227-240), written row-major.
int refx_amg_coarse_inverse(const void* h, double* out) {
    return guarded([&] {
        const auto inv = static_cast<const cfd::fv::AmgPreconditioner*>(h)->coarse_inverse();
        for (Eigen::Index i = 0; i < inv.rows(); ++i)
            for (Eigen::Index j = 0; j < inv.cols(); ++j) out[i * inv.cols() + j] = inv(i, j);
    });
}

// AmgPreconditioner::apply (amg.cpp:192-225): one Gauss-Seidel V-cycle.
int refx_amg_apply(const void* h, int n, const double* r, double* z) {
    return guarded([&] {
        const cfd::fv::DenseVector rv = Eigen::Map<const cfd::fv::DenseVector>(r, n);
        cfd::fv::DenseVector zv;
        static_cast<const cfd::fv::AmgPreconditioner*>(h)->apply(rv, zv);
        std::copy(zv.data(), zv.data() + n, z);
    });
}

// cfd::fv::amg_aggregate (amg.cpp:12-78) on a CSR matrix with the given diagonal.
int refx_amg_aggregate(int n, const int* rp, const int* ci, const double* va, const double* diag,
                       double theta, int* agg) {
    try {
        const CsrMatrix a = csr_from(n, n, rp, ci, va);
        const cfd::fv::DenseVector d = Eigen::Map<const cfd::fv::DenseVector>(diag, n);
        int n_agg = 0;
        const std::vector<int> out = cfd::fv::amg_aggregate(a, d, theta, n_agg);
        std::copy(out.begin(), out.end(), agg);
        return n_agg;
    } catch (const std::exception&) {
        return -1;
    }
}

// cfd::fv::pcg (amg.cpp:253-285): the CPU AmgCg, x in/out.
int refx_pcg(const void* h, int n, const int* rp, const int* ci, const double* va, const double* b, double* x,
             double tol, int max_iterations, int* iterations, double* residual) {
    return guarded([&] {
        const CsrMatrix a = csr_from(n, n, rp, ci, va);
        const cfd::fv::DenseVector bv = Eigen::Map<const cfd::fv::DenseVector>(b, n);
        cfd::fv::DenseVector xv = Eigen::Map<const cfd::fv::DenseVector>(x, n);
        const auto r = cfd::fv::pcg(a, bv, xv, *static_cast<const cfd::fv::AmgPreconditioner*>(h), tol,
                                    max_iterations);
        std::copy(xv.data(), xv.data() + n, x);
        *iterations = r.iterations;
        *residual = r.residual_norm;
    });
}

// ---- LduMatrix (ldu_matrix.cpp) on a mesh -------------------------------------------------------

// An LduMatrix over the mesh (borrowed; it must outlive the handle), with the mesh's CSR
// pattern attached (as FvGeometry does) and a persistent AmgCache.
void* refx_ldu_create(const void* mesh) {
    try {
        auto h = std::make_unique<LduHandle>();
        h->mesh = static_cast<const cfd::mesh::Mesh*>(mesh);
        h->pattern = cfd::fv::build_csr_pattern(*h->mesh);
        h->ldu = std::make_unique<cfd::fv::LduMatrix>(*h->mesh);
        h->ldu->pattern = &h->pattern;
        return h.release();
    } catch (const std::exception&) {
        return nullptr;
    }
}

void refx_ldu_destroy(void* h) { delete static_cast<LduHandle*>(h); }

void refx_ldu_set(void* h, const double* diag, const double* upper, const double* lower, const double* source) {
    auto& l = *static_cast<LduHandle*>(h)->ldu;
    std::copy(diag, diag + l.diag.size(), l.diag.begin());
    std::copy(upper, upper + l.upper.size(), l.upper.begin());
    std::copy(lower, lower + l.lower.size(), l.lower.begin());
    std::copy(source, source + l.source.size(), l.source.begin());
}

void refx_ldu_get(const void* h, double* diag, double* source) {
    const auto& l = *static_cast<const LduHandle*>(h)->ldu;
    std::copy(l.diag.begin(), l.diag.end(), diag);
    std::copy(l.source.begin(), l.source.end(), source);
}

// LduMatrix::set_reference (ldu_matrix.cpp:105-109).
void refx_ldu_set_reference(void* h, int cell, double value) {
    static_cast<LduHandle*>(h)->ldu->set_reference(cell, value);
}

// LduMatrix::multiply (ldu_matrix.cpp:39-56).
void refx_ldu_multiply(const void* h, const double* x, double* y) {
    const auto& l = *static_cast<const LduHandle*>(h)->ldu;
    const std::vector<Scalar> xv(x, x + l.diag.size());
    std::vector<Scalar> yv;
    l.multiply(xv, yv);
    std::copy(yv.begin(), yv.end(), y);
}

// LduMatrix::residual_norms (ldu_matrix.cpp:69-103).
void refx_ldu_residual_norms(const void* h, const double* x, double* res, double* norm) {
    const auto& l = *static_cast<const LduHandle*>(h)->ldu;
    const std::vector<Scalar> xv(x, x + l.diag.size());
    const auto [r, nrm] = l.residual_norms(xv);
    *res = r;
    *norm = nrm;
}

// LduMatrix::build_csr_pattern of the handle's mesh (ldu_matrix.cpp:572-612).
void refx_ldu_pattern(const void* h, int* row_ptr, int* col, int* diag_pos, int* upper_pos, int* lower_pos) {
    const auto& p = static_cast<const LduHandle*>(h)->pattern;
    const auto n = static_cast<std::size_t>(p.structure.rows());
    std::copy(p.structure.outerIndexPtr(), p.structure.outerIndexPtr() + n + 1, row_ptr);
    std::copy(p.structure.innerIndexPtr(), p.structure.innerIndexPtr() + p.structure.nonZeros(), col);
    std::copy(p.diag_pos.begin(), p.diag_pos.end(), diag_pos);
    std::copy(p.upper_pos.begin(), p.upper_pos.end(), upper_pos);
    std::copy(p.lower_pos.begin(), p.lower_pos.end(), lower_pos);
}

// LduMatrix::solve (ldu_matrix.cpp:111-282) with the handle's AmgCache (with_cache = 0: none,
// as solve_scalar calls it); type is LinearSolverType (0 ConjugateGradient, 1 BiCgStab,
// 2 AmgCg, 3 GpuCg, 4 GpuBiCgStab). with_pattern = 0 detaches the CSR pattern (the
// non-persistent branches).
int refx_ldu_solve(void* h, int type, double tolerance, double rel_tolerance, int max_iterations, int max_age,
                   int with_pattern, int with_cache, double* x, double* initial, double* final_residual,
                   int* iterations, int* amg_age, int* amg_levels) {
    return guarded([&] {
        auto* hh = static_cast<LduHandle*>(h);
        hh->ldu->pattern = with_pattern ? &hh->pattern : nullptr;
        hh->cache.max_age = max_age;
        cfd::fv::LinearSolverSettings s;
        s.type = static_cast<cfd::fv::LinearSolverType>(type);
        s.tolerance = tolerance;
        s.rel_tolerance = rel_tolerance;
        s.max_iterations = max_iterations;
        std::vector<Scalar> xv(x, x + hh->ldu->diag.size());
        const auto r = hh->ldu->solve(xv, s, with_cache ? &hh->cache : nullptr);
        std::copy(xv.begin(), xv.end(), x);
        *initial = r.initial_residual;
        *final_residual = r.final_residual;
        *iterations = r.iterations;
        *amg_age = hh->cache.age;
        *amg_levels = hh->cache.amg ? hh->cache.amg->levels() : 0;
    });
}

// ---- restated workload generators (this project's definitions, not reference code) -------------

// Lattice nodes (k outer, then j, then i) on the given coordinates, interior coordinates moved
// by jitter * h * U(-1, 1) with h the smaller adjacent spacing; one U(-1, 1) draw per
// coordinate of every node, boundary coordinates drawn and left in place.
void refx_jittered_lattice(int nx, int ny, int nz, const double* xs, const double* ys, const double* zs,
                           double jitter, std::uint64_t seed, double* points) {
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    const double* ax[3] = {xs, ys, zs};
    const int n[3] = {nx, ny, nz};
    std::size_t t = 0;
    for (int k = 0; k <= nz; ++k)
        for (int j = 0; j <= ny; ++j)
            for (int i = 0; i <= nx; ++i) {
                const int c[3] = {i, j, k};
                double* p = points + 3 * t;
                for (int a = 0; a < 3; ++a) {
                    p[a] = ax[a][c[a]];
                    const double r = u(rng);
                    if (c[a] == 0 || c[a] == n[a]) continue;
                    const double h = std::min(ax[a][c[a] + 1] - ax[a][c[a]], ax[a][c[a]] - ax[a][c[a] - 1]);
                    p[a] += jitter * h * r;
                }
                ++t;
            }
}

// Pressure inputs of the synthetic configurations: cell factor X = exp(sigma N(0,1)) (1 when
// sigma = 0), rAU = X (unit_rau) or V X, face rAU = w rAU_P + (1 - w) rAU_N; face flux u . S
// with u ~ U(-1, 1)^3 per face (flux_kind 0) or 0; source N(0, 1) minus its mean (rhs_kind 1)
// or 0.
void refx_pressure_inputs(int n_cells, int n_internal, const int* owner, const int* neighbour,
                          const double* weights, const double* volumes, const double* face_areas, double sigma,
                          int unit_rau, int flux_kind, int rhs_kind, std::uint64_t seed, double* gamma,
                          double* flux, double* source) {
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> g01(0.0, 1.0);
    std::uniform_real_distribution<double> u11(-1.0, 1.0);
    std::vector<double> rau(static_cast<std::size_t>(n_cells));
    for (int c = 0; c < n_cells; ++c) {
        const double x = sigma > 0.0 ? std::exp(sigma * g01(rng)) : 1.0;
        rau[static_cast<std::size_t>(c)] = unit_rau ? x : volumes[c] * x;
    }
    for (int f = 0; f < n_internal; ++f) {
        const double w = weights[f];
        gamma[f] = w * rau[static_cast<std::size_t>(owner[f])] + (1.0 - w) * rau[static_cast<std::size_t>(neighbour[f])];
    }
    for (int f = 0; f < n_internal; ++f) {
        if (flux_kind == 0) {
            const double ux = u11(rng), uy = u11(rng), uz = u11(rng);
            const double* s = face_areas + 3 * f;
            flux[f] = ux * s[0] + uy * s[1] + uz * s[2];
        } else {
            flux[f] = 0.0;
        }
    }
    if (rhs_kind == 1) {
        double mean = 0.0;
        for (int c = 0; c < n_cells; ++c) {
            source[c] = g01(rng);
            mean += source[c];
        }
        mean /= static_cast<double>(n_cells);
        for (int c = 0; c < n_cells; ++c) source[c] -= mean;
    } else {
        for (int c = 0; c < n_cells; ++c) source[c] = 0.0;
    }
}

} // extern "C"
