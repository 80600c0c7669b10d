// Drop-in check at the solver level: the reference's own FlowSolver (src/fv/src/flow_solver.cpp),
// compiled unchanged against this project's C++ front end and linked with libcfdb.so, runs
// SIMPLE iterations with the pressure solved by "solver": {"device": "gpu"}
// (LinearSolverType::GpuCg). Every accelerator call it makes lands in the product: the face
// assembly of the pressure and momentum equations (cfd::gpu::assemble_convection_diffusion,
// flow_solver.cpp:761-770), the persistent pressure solves and the momentum BiCGStab solves
// (cfd::gpu::DeviceSolver through LduMatrix::solve_persistent), and, since GpuCg selects
// FlowSolver::device_fv, the gradients, limiter and face corrections (cfd::gpu::DeviceFv
// through FvGeometry::device).
//
// oracle/build.py (build_dropin) compiles it with the reference's unchanged flow_solver.cpp and
// the sources of the LDU drop-in (test_dropin_ldu.cpp).
//
// Usage: test_dropin_flow <nx> <ny> <nz> <grading_x> <iterations> <fields_out>
// The box is make_box_mesh's unit cube (patches xmin, xmax, ymin, ymax, zmin, zmax): inlet at
// xmin (u = 1), outlet at xmax (p = 0.25), a moving wall at ymax (u = 0.3), symmetry at zmin,
// walls elsewhere; nu = 0.01, p and u solved to a normalised residual of 1e-12. Prints one JSON
// object per SIMPLE iteration (its initial residuals) and writes u (n x 3), p, phi as float64
// to fields_out.
#include <cfd/fv/flow_solver.hpp>
#include <cfd/gpu/krylov.hpp>
#include <cfd/mesh/box_mesher.hpp>

#include <cstdio>
#include <cstdlib>
#include <exception>
#include <map>
#include <string>
#include <vector>

int main(int argc, char** argv) {
    try {
        if (argc < 7) {
            std::printf("{\"error\": \"usage: test_dropin_flow nx ny nz grading_x iterations fields_out\"}\n");
            return 1;
        }
        cfd::mesh::BoxSpec spec;
        spec.nx = std::atoi(argv[1]);
        spec.ny = std::atoi(argv[2]);
        spec.nz = std::atoi(argv[3]);
        spec.grading = cfd::core::Vec3(std::atof(argv[4]), 1.0, 1.0);
        const int iterations = std::atoi(argv[5]);
        const cfd::mesh::Mesh mesh = cfd::mesh::make_box_mesh(spec);
        using cfd::fv::BoundaryCondition;
        using cfd::fv::FlowBoundary;
        std::map<std::string, BoundaryCondition> bc;
        bc["xmin"] = BoundaryCondition{FlowBoundary::VelocityInlet, cfd::core::Vec3(1.0, 0.0, 0.0), 0.0};
        bc["xmax"] = BoundaryCondition{FlowBoundary::PressureOutlet, cfd::core::Vec3::Zero(), 0.25};
        bc["ymax"] = BoundaryCondition{FlowBoundary::Wall, cfd::core::Vec3(0.3, 0.0, 0.0), 0.0};
        bc["zmin"] = BoundaryCondition{FlowBoundary::Symmetry, cfd::core::Vec3::Zero(), 0.0};
        cfd::fv::FlowSettings s;
        s.nu = 0.01;
        s.p_solver = {cfd::fv::LinearSolverType::GpuCg, 1e-12, 0.0, 2000};
        s.u_solver = {cfd::fv::LinearSolverType::GpuBiCgStab, 1e-12, 0.0, 2000};
        cfd::fv::FlowSolver flow(mesh, bc, s);
        std::printf("{\"backend\": \"%s\", \"device_available\": %s, \"cells\": %d}\n",
                    cfd::gpu::backend_name().c_str(), cfd::gpu::device_available() ? "true" : "false",
                    mesh.n_cells());
        for (int it = 0; it < iterations; ++it) {
            const cfd::fv::Residuals r = flow.simple_iteration();
            std::printf("{\"iteration\": %d, \"u\": [%.17g, %.17g, %.17g], \"p\": %.17g, \"continuity\": %.17g}\n", it,
                        r.u[0], r.u[1], r.u[2], r.p, r.continuity);
        }
        std::FILE* f = std::fopen(argv[6], "wb");
        if (f == nullptr) throw std::runtime_error("cannot write the fields");
        for (const auto& v : flow.velocity()) std::fwrite(v.data(), sizeof(double), 3, f);
        std::fwrite(flow.pressure().data(), sizeof(double), flow.pressure().size(), f);
        std::fwrite(flow.face_flux().data(), sizeof(double), flow.face_flux().size(), f);
        std::fclose(f);
        return 0;
    } catch (const std::exception& e) {
        std::printf("{\"error\": \"%s\"}\n", e.what());
        return 2;
    }
}
