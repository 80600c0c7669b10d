// Drop-in check: the reference's own callers of the accelerator layer, compiled unchanged
// against this project's C++ front end and linked with libcfdb.so.
//
// oracle/build.py (build_dropin) compiles this file together with the reference's unchanged
// src/fv/src/{ldu_matrix.cpp, amg.cpp, parallel_amg.cpp, fv_geometry.cpp},
// src/mesh/src/{mesh.cpp, mesh_builder.cpp, box_mesher.cpp}, src/parallel/src/comm.cpp and its
// host path src/gpu/src/krylov_openmp.cpp, with <cfd/gpu/krylov.hpp> and
// <cfd/gpu/fv_device.hpp> resolving to include/cfd_gpu_krylov.hpp and include/cfd_gpu_fv.hpp
// (Eigen: the oracle's stand-in). So LduMatrix::solve with LinearSolverType::GpuCg takes the
// reference's own route -- solve_persistent (ldu_matrix.cpp:287-366) with its AmgCache and the
// reference's AmgPreconditioner::setup -- into cfd::gpu::DeviceSolver of libcfdb.so, and the
// CPU solver types reach gpu::solve_host of the reference's krylov_openmp.cpp.
//
// Usage: test_dropin_ldu <n>   (an n^3 box from make_box_mesh). Prints one JSON object per
// solve: the path, iterations, normalised residuals and the true relative 2-norm residual.
#include <cfd/fv/fv_geometry.hpp>
#include <cfd/fv/ldu_matrix.hpp>
#include <cfd/gpu/krylov.hpp>
#include <cfd/mesh/box_mesher.hpp>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <vector>

namespace {

double true_rel_residual(const cfd::fv::LduMatrix& eq, const std::vector<double>& x) {
    std::vector<double> r;
    eq.residual(x, r);
    double rr = 0.0, bb = 0.0;
    for (std::size_t i = 0; i < r.size(); ++i) {
        rr += r[i] * r[i];
        bb += eq.source[i] * eq.source[i];
    }
    return std::sqrt(rr / bb);
}

void report(const char* path, const cfd::fv::LinearSolveResult& r, const cfd::fv::LduMatrix& eq,
            const std::vector<double>& x, int amg_age) {
    double sum = 0.0;
    for (const double v : x) sum += v;
    std::printf("{\"path\": \"%s\", \"iterations\": %d, \"initial\": %.17g, \"final\": %.17g, "
                "\"true_rel_residual\": %.17g, \"amg_age\": %d, \"x_sum\": %.17g}\n",
                path, r.iterations, r.initial_residual, r.final_residual, true_rel_residual(eq, x), amg_age, sum);
}

} // namespace

int main(int argc, char** argv) {
    try {
        const int n = argc > 1 ? std::atoi(argv[1]) : 16;
        cfd::mesh::BoxSpec spec;
        spec.nx = spec.ny = spec.nz = n;
        const cfd::mesh::Mesh mesh = cfd::mesh::make_box_mesh(spec);
        const cfd::fv::FvGeometry geo(mesh);
        const int nc = mesh.n_cells(), nif = mesh.n_internal_faces();
        // a pressure equation as FlowSolver::pressure_correction assembles it
        // (flow_solver.cpp:757-796): exact, platform-independent face data
        std::vector<double> flux(static_cast<std::size_t>(nif)), gamma(static_cast<std::size_t>(nif));
        for (int f = 0; f < nif; ++f) {
            flux[static_cast<std::size_t>(f)] = static_cast<double>((static_cast<long long>(f) * 7919) % 1000) / 500.0 - 1.0;
            gamma[static_cast<std::size_t>(f)] = 1.0 + 0.125 * static_cast<double>(f % 7);
        }
        cfd::fv::LduMatrix eq(mesh);
        eq.pattern = &geo.csr_pattern();
        std::vector<double> div(static_cast<std::size_t>(nc), 0.0);
        cfd::gpu::assemble_convection_diffusion(nc, nif, mesh.owner().data(), mesh.neighbour().data(), flux.data(),
                                                gamma.data(), geo.delta_coeffs().data(), 0.0, eq.upper.data(),
                                                eq.lower.data(), eq.diag.data(), div.data());
        for (int c = 0; c < nc; ++c) eq.source[static_cast<std::size_t>(c)] -= div[static_cast<std::size_t>(c)];
        eq.set_reference(0, 0.0);
        std::printf("{\"backend\": \"%s\", \"device_available\": %s, \"cells\": %d}\n",
                    cfd::gpu::backend_name().c_str(), cfd::gpu::device_available() ? "true" : "false", nc);

        cfd::fv::LinearSolverSettings s;
        s.tolerance = 0.0;
        s.rel_tolerance = 1e-8;
        s.max_iterations = 500;
        // GPU path: solve_persistent with the AmgCache (hierarchy rebuilt every max_age solves)
        cfd::fv::AmgCache cache;
        cache.max_age = 2;
        s.type = cfd::fv::LinearSolverType::GpuCg;
        for (int k = 0; k < 3; ++k) {
            std::vector<double> x(static_cast<std::size_t>(nc), 0.0);
            const auto r = eq.solve(x, s, &cache);
            report("GpuCg", r, eq, x, cache.age);
        }
        // GPU path without a pattern: the one-shot AMG-CG branch (ldu_matrix.cpp:173-216)
        {
            cfd::fv::LduMatrix eq2 = eq;
            eq2.pattern = nullptr;
            cfd::fv::AmgCache c2;
            std::vector<double> x(static_cast<std::size_t>(nc), 0.0);
            const auto r = eq2.solve(x, s, &c2);
            report("GpuCg_one_shot", r, eq2, x, c2.age);
        }
        // persistent BiCGStab on the GPU
        {
            cfd::fv::AmgCache c3;
            s.type = cfd::fv::LinearSolverType::GpuBiCgStab;
            std::vector<double> x(static_cast<std::size_t>(nc), 0.0);
            const auto r = eq.solve(x, s, &c3);
            report("GpuBiCgStab", r, eq, x, c3.age);
        }
        // the CPU path of the same call surface: gpu::solve_host of the reference's krylov_openmp.cpp
        {
            s.type = cfd::fv::LinearSolverType::BiCgStab;
            std::vector<double> x(static_cast<std::size_t>(nc), 0.0);
            const auto r = eq.solve(x, s, nullptr);
            report("BiCgStab_host", r, eq, x, 0);
        }
        return 0;
    } catch (const std::exception& e) {
        std::printf("{\"error\": \"%s\"}\n", e.what());
        return 2;
    }
}
