// C-ABI shim over the reference's FlowSolver (src/fv/src/flow_solver.cpp), compiled unchanged
// against the Eigen stand-in into oracle/_ref/libcfdref.so (TEST INFRASTRUCTURE ONLY).
//
// It drives one SIMPLE iteration step by step, as FlowSolver::simple_iteration
// (flow_solver.cpp:849-860) does: the momentum system (assemble_momentum), the momentum
// predictor (solve_momentum) and the pressure correction (pressure_correction,
// flow_solver.cpp:673-847), so that each step's inputs and outputs can be compared with the
// oracle's restatement and, through it, with the device step. Those three members are private;
// their addresses are taken in explicit instantiations of a class template, where the language
// does not check access (C++20 [temp.spec.general]/6), so the reference's sources stay as they
// are. It also runs the reference's solve_scalar (src/fv/src/scalar_transport.cpp) on a mesh.
#include <cfd/fv/flow_solver.hpp>
#include <cfd/fv/scalar_transport.hpp>
#include <cfd/mesh/mesh.hpp>

#include <algorithm>
#include <exception>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

namespace {

using cfd::core::Scalar;
using cfd::core::Vec3;
using cfd::fv::FlowSolver;

template <class Tag, auto Member> struct Expose {
    friend constexpr auto member_of(Tag) { return Member; }
};
struct AssembleMomentum {
    friend constexpr auto member_of(AssembleMomentum);
};
struct SolveMomentum {
    friend constexpr auto member_of(SolveMomentum);
};
struct PressureCorrection {
    friend constexpr auto member_of(PressureCorrection);
};
template struct Expose<AssembleMomentum, &FlowSolver::assemble_momentum>;
template struct Expose<SolveMomentum, &FlowSolver::solve_momentum>;
template struct Expose<PressureCorrection, &FlowSolver::pressure_correction>;

template <class T> struct FirstArgument;
template <class R, class C, class A, class... Rest> struct FirstArgument<R (C::*)(A, Rest...)> {
    using type = std::remove_cvref_t<A>;
};
template <class R, class C, class A, class... Rest> struct FirstArgument<R (C::*)(A, Rest...) const> {
    using type = std::remove_cvref_t<A>;
};
// FlowSolver::MomentumSystem: shared off-diagonal coefficients (base), per-component diagonal
// and source
using MomentumSystem = FirstArgument<decltype(member_of(PressureCorrection{}))>::type;

struct FlowHandle {
    std::unique_ptr<FlowSolver> solver;
    std::unique_ptr<MomentumSystem> sys;
    std::size_t n_cells = 0, n_faces = 0, n_internal = 0;
};

template <typename F> int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

std::vector<Vec3> vec3s(const double* a, std::size_t n) {
    std::vector<Vec3> v(n);
    for (std::size_t i = 0; i < n; ++i) v[i] = Vec3(a[3 * i], a[3 * i + 1], a[3 * i + 2]);
    return v;
}

void put_vec3s(const std::vector<Vec3>& v, double* out) {
    for (std::size_t i = 0; i < v.size(); ++i)
        for (int k = 0; k < 3; ++k) out[3 * i + static_cast<std::size_t>(k)] = v[i][k];
}

} // namespace

extern "C" {

// FlowSolver(mesh, conditions, settings) (flow_solver.cpp:35-67), one condition per mesh patch
// in the mesh's patch order (n_patches of them). Per patch: kind (FlowBoundary: 0 inlet,
// 1 wall, 2 outlet, 3 symmetry, 4 empty), velocity (3), pressure. real = {nu, alpha_u, alpha_p,
// p tolerance, p rel_tolerance, u tolerance, u rel_tolerance}; ints = {n_non_orth_correctors,
// p solver type, p max_iterations, u solver type, u max_iterations, convection scheme,
// gradient scheme} (LinearSolverType, ConvectionScheme, GradientScheme as numbered there).
void* refx_flow_create(const void* mesh, int n_patches, const int* kind, const double* velocity,
                       const double* pressure, const double* real, const int* ints) {
    try {
        const auto& m = *static_cast<const cfd::mesh::Mesh*>(mesh);
        if (n_patches != static_cast<int>(m.patches().size())) throw std::invalid_argument("one condition per patch");
        std::map<std::string, cfd::fv::BoundaryCondition> conditions;
        for (int p = 0; p < n_patches; ++p) {
            cfd::fv::BoundaryCondition c;
            c.kind = static_cast<cfd::fv::FlowBoundary>(kind[p]);
            c.velocity = Vec3(velocity[3 * p], velocity[3 * p + 1], velocity[3 * p + 2]);
            c.pressure = pressure[p];
            conditions[m.patches()[static_cast<std::size_t>(p)].name] = c;
        }
        cfd::fv::FlowSettings s;
        s.nu = real[0];
        s.alpha_u = real[1];
        s.alpha_p = real[2];
        s.p_solver.tolerance = real[3];
        s.p_solver.rel_tolerance = real[4];
        s.u_solver.tolerance = real[5];
        s.u_solver.rel_tolerance = real[6];
        s.n_non_orth_correctors = ints[0];
        s.p_solver.type = static_cast<cfd::fv::LinearSolverType>(ints[1]);
        s.p_solver.max_iterations = ints[2];
        s.u_solver.type = static_cast<cfd::fv::LinearSolverType>(ints[3]);
        s.u_solver.max_iterations = ints[4];
        s.convection = static_cast<cfd::fv::ConvectionScheme>(ints[5]);
        s.gradient = static_cast<cfd::fv::GradientScheme>(ints[6]);
        auto h = std::make_unique<FlowHandle>();
        h->solver = std::make_unique<FlowSolver>(m, std::move(conditions), s);
        h->n_cells = static_cast<std::size_t>(m.n_cells());
        h->n_faces = static_cast<std::size_t>(m.n_faces());
        h->n_internal = static_cast<std::size_t>(m.n_internal_faces());
        return h.release();
    } catch (const std::exception&) {
        return nullptr;
    }
}

void refx_flow_destroy(void* h) { delete static_cast<FlowHandle*>(h); }

// FlowSolver::set_state (u: n_cells x 3, p: n_cells, phi: n_faces or null to recompute).
int refx_flow_set_state(void* h, const double* u, const double* p, const double* phi) {
    return guarded([&] {
        auto& f = *static_cast<FlowHandle*>(h);
        std::vector<Scalar> pv(p, p + f.n_cells);
        if (phi != nullptr) {
            f.solver->set_state(vec3s(u, f.n_cells), std::move(pv), std::vector<Scalar>(phi, phi + f.n_faces));
        } else {
            f.solver->set_state(vec3s(u, f.n_cells), std::move(pv));
        }
    });
}

int refx_flow_get_state(const void* h, double* u, double* p, double* phi) {
    return guarded([&] {
        const auto& f = *static_cast<const FlowHandle*>(h);
        put_vec3s(f.solver->velocity(), u);
        std::copy(f.solver->pressure().begin(), f.solver->pressure().end(), p);
        std::copy(f.solver->face_flux().begin(), f.solver->face_flux().end(), phi);
    });
}

// Per boundary face (f - n_internal_faces): FlowBoundary kind, outlet pressure, fixed velocity.
int refx_flow_boundary(const void* h, int* kind, double* pressure, double* velocity) {
    return guarded([&] {
        const auto& f = *static_cast<const FlowHandle*>(h);
        for (std::size_t b = 0; b < f.n_faces - f.n_internal; ++b) {
            const auto& c = f.solver->boundary_condition(static_cast<cfd::core::Label>(b));
            kind[b] = static_cast<int>(c.kind);
            pressure[b] = c.pressure;
            for (int k = 0; k < 3; ++k) velocity[3 * b + static_cast<std::size_t>(k)] = c.velocity[k];
        }
    });
}

// FlowSolver::assemble_momentum(sys, dt, relax) into the handle's momentum system, as
// simple_iteration sets it up (flow_solver.cpp:850-853).
int refx_flow_momentum(void* h, double dt, int relax) {
    return guarded([&] {
        auto& f = *static_cast<FlowHandle*>(h);
        const auto& geo = f.solver->geometry();
        f.sys.reset(new MomentumSystem{cfd::fv::LduMatrix(geo.mesh()), {}, {}});
        f.sys->base.pattern = &geo.csr_pattern();
        f.sys->base.halo = geo.halo();
        ((*f.solver).*member_of(AssembleMomentum{}))(*f.sys, dt, relax != 0);
    });
}

// The handle's momentum system: diag and source per component (n_cells x 3), the shared
// upper / lower coefficients (n_internal_faces).
int refx_flow_momentum_arrays(const void* h, double* diag, double* upper, double* lower, double* source) {
    return guarded([&] {
        const auto& f = *static_cast<const FlowHandle*>(h);
        if (!f.sys) throw std::logic_error("no momentum system");
        put_vec3s(f.sys->diag, diag);
        put_vec3s(f.sys->source, source);
        std::copy(f.sys->base.upper.begin(), f.sys->base.upper.end(), upper);
        std::copy(f.sys->base.lower.begin(), f.sys->base.lower.end(), lower);
    });
}

// FlowSolver::solve_momentum(sys): the momentum predictor; residual gets the initial
// normalised residual per component.
int refx_flow_solve_momentum(void* h, double* residual) {
    return guarded([&] {
        auto& f = *static_cast<FlowHandle*>(h);
        if (!f.sys) throw std::logic_error("no momentum system");
        const Vec3 r = ((*f.solver).*member_of(SolveMomentum{}))(*f.sys);
        for (int k = 0; k < 3; ++k) residual[k] = r[k];
    });
}

// FlowSolver::pressure_correction(sys, relax_p, u_prev, phi_prev) (flow_solver.cpp:673-847);
// u_prev (n_cells x 3) and phi_prev (n_faces) may be null.
int refx_flow_pressure_correction(void* h, int relax_p, const double* u_prev, const double* phi_prev,
                                  double* initial_residual) {
    return guarded([&] {
        auto& f = *static_cast<FlowHandle*>(h);
        if (!f.sys) throw std::logic_error("no momentum system");
        std::vector<Vec3> up;
        std::vector<Scalar> pp;
        if (u_prev != nullptr) up = vec3s(u_prev, f.n_cells);
        if (phi_prev != nullptr) pp.assign(phi_prev, phi_prev + f.n_faces);
        *initial_residual = ((*f.solver).*member_of(PressureCorrection{}))(
            *f.sys, relax_p != 0, u_prev != nullptr ? &up : nullptr, phi_prev != nullptr ? &pp : nullptr);
    });
}

// FlowSolver::simple_iteration (flow_solver.cpp:849-866): residuals = {u (3), p, continuity}.
int refx_flow_simple_iteration(void* h, double* residuals) {
    return guarded([&] {
        auto& f = *static_cast<FlowHandle*>(h);
        const cfd::fv::Residuals r = f.solver->simple_iteration();
        for (int k = 0; k < 3; ++k) residuals[k] = r.u[k];
        residuals[3] = r.p;
        residuals[4] = r.continuity;
    });
}

// solve_scalar (scalar_transport.cpp:49-183) on a mesh with its own FvGeometry: the equation
// given per face (gamma_face, n_faces), per cell (su, sp) and per boundary face (kind:
// ScalarBoundary::Kind 0 fixed value, 1 zero gradient, 2 fixed gradient, 3 mixed; value;
// coefficient); fixed_cell / fixed_value, old_value and capacity may be null. flags = {solver type
// (LinearSolverType), max_iterations, linear_upwind, gradient scheme}; real = {relaxation, dt,
// tolerance, rel_tolerance}. field is solved in place; result = {initial, final, iterations}.
int refx_scalar_solve(const void* mesh, const double* face_flux, const double* gamma_face, const double* su,
                      const double* sp, const int* bc_kind, const double* bc_value, const double* bc_coefficient,
                      const unsigned char* fixed_cell, const double* fixed_value, const double* old_value,
                      const double* capacity, const int* flags, const double* real, double* field, double* result) {
    return guarded([&] {
        const auto& m = *static_cast<const cfd::mesh::Mesh*>(mesh);
        const auto nc = static_cast<std::size_t>(m.n_cells());
        const auto nf = static_cast<std::size_t>(m.n_faces());
        const auto nb = nf - static_cast<std::size_t>(m.n_internal_faces());
        const cfd::fv::FvGeometry geo(m);
        cfd::fv::ScalarEquation eq;
        eq.gamma_face.assign(gamma_face, gamma_face + nf);
        eq.su.assign(su, su + nc);
        eq.sp.assign(sp, sp + nc);
        eq.boundary.resize(nb);
        for (std::size_t b = 0; b < nb; ++b) {
            eq.boundary[b].kind = static_cast<cfd::fv::ScalarBoundary::Kind>(bc_kind[b]);
            eq.boundary[b].value = bc_value[b];
            eq.boundary[b].coefficient = bc_coefficient[b];
        }
        if (fixed_cell != nullptr) {
            eq.fixed_cell.assign(fixed_cell, fixed_cell + nc);
            eq.fixed_value.assign(fixed_value, fixed_value + nc);
        }
        std::vector<Scalar> old, cap;
        if (old_value != nullptr) {
            old.assign(old_value, old_value + nc);
            eq.old_value = &old;
        }
        if (capacity != nullptr) {
            cap.assign(capacity, capacity + nc);
            eq.capacity = &cap;
        }
        eq.linear_upwind = flags[2] != 0;
        eq.gradient = static_cast<cfd::fv::GradientScheme>(flags[3]);
        eq.relaxation = real[0];
        eq.dt = real[1];
        cfd::fv::LinearSolverSettings s;
        s.type = static_cast<cfd::fv::LinearSolverType>(flags[0]);
        s.max_iterations = flags[1];
        s.tolerance = real[2];
        s.rel_tolerance = real[3];
        std::vector<Scalar> flux(face_flux, face_flux + nf);
        std::vector<Scalar> x(field, field + nc);
        const auto r = cfd::fv::solve_scalar(geo, flux, eq, x, s);
        std::copy(x.begin(), x.end(), field);
        result[0] = r.initial_residual;
        result[1] = r.final_residual;
        result[2] = static_cast<double>(r.iterations);
    });
}

} // extern "C"
