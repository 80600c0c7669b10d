// cfd::gpu C++ front end over the C ABI (declared in include/cfd_gpu_krylov.hpp).
#include "../../include/cfd_gpu_krylov.hpp"

#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/cfdb.h"

namespace cfd::gpu {

namespace {

[[noreturn]] void raise(int rc) {
    char buf[1024];
    cfdb_last_error(buf, sizeof(buf));
    const std::string msg(buf);
    if (rc == CFDB_ERR_BAD_ARG) throw std::invalid_argument(msg);
    if (rc == CFDB_ERR_CUDA || rc == CFDB_ERR_OOM || rc == CFDB_ERR_NO_DEVICE) {
        throw std::runtime_error(msg.rfind("CUDA", 0) == 0 ? msg : "CUDA " + msg);
    }
    throw std::runtime_error(msg);
}

void check(int rc) {
    if (rc != CFDB_OK) raise(rc);
}

cfdb_csr to_c(const CsrView& v) { return cfdb_csr{v.n, v.nnz, v.row_ptr, v.col, v.val}; }

cfdb_control to_c(const SolveControl& c) { return cfdb_control{c.abs_tolerance, c.max_iterations}; }

SolveStats from_c(const cfdb_stats& s) {
    SolveStats o;
    o.iterations = s.iterations;
    o.residual = s.residual;
    o.converged = s.converged != 0;
    o.on_device = s.on_device != 0;
    return o;
}

int method_c(Method m) { return m == Method::Cg ? CFDB_METHOD_CG : CFDB_METHOD_BICGSTAB; }

// AmgView -> cfdb_amg_view; the level array lives in `levels`.
cfdb_amg_view view_c(const AmgView& amg, std::vector<cfdb_amg_level>& levels) {
    levels.clear();
    for (const AmgLevelView& l : amg.levels) levels.push_back(cfdb_amg_level{to_c(l.a), to_c(l.p), to_c(l.r)});
    cfdb_amg_view v{};
    v.n_levels = static_cast<int>(levels.size());
    v.levels = levels.data();
    v.coarse_inverse = amg.coarse_inverse;
    v.smooth_sweeps = amg.smooth_sweeps;
    v.jacobi_weight = amg.jacobi_weight;
    return v;
}

} // namespace

SolveStats solve(const CsrView& a, const double* b, double* x, Method method, const SolveControl& control) {
    const cfdb_csr ac = to_c(a);
    const cfdb_control cc = to_c(control);
    cfdb_stats st{};
    check(cfdb_solve(&ac, b, x, method_c(method), &cc, &st));
    return from_c(st);
}

SolveStats solve_amg_cg(const AmgView& amg, const double* b, double* x, const SolveControl& control) {
    if (amg.levels.empty()) throw std::invalid_argument("solve_amg_cg: empty AMG hierarchy");
    std::vector<cfdb_amg_level> lv;
    const cfdb_amg_view v = view_c(amg, lv);
    const cfdb_control cc = to_c(control);
    cfdb_stats st{};
    check(cfdb_solve_amg_cg(&v, b, x, &cc, &st));
    return from_c(st);
}

struct DeviceSolver::Impl {
    cfdb_system* sys = nullptr;
};

DeviceSolver::DeviceSolver(const LduPattern& p) : impl_(std::make_unique<Impl>()) {
    const cfdb_ldu_pattern pc{p.n, p.n_faces, p.nnz, p.row_ptr, p.col, p.diag_pos, p.upper_pos, p.lower_pos};
    check(cfdb_system_create(&pc, &impl_->sys));
}

DeviceSolver::~DeviceSolver() {
    if (impl_ && impl_->sys != nullptr) cfdb_system_destroy(impl_->sys);
}

void DeviceSolver::set_amg(const AmgView& amg) {
    if (amg.levels.empty()) throw std::invalid_argument("DeviceSolver::set_amg: empty AMG hierarchy");
    std::vector<cfdb_amg_level> lv;
    const cfdb_amg_view v = view_c(amg, lv);
    check(cfdb_system_set_amg(impl_->sys, &v));
}

SolveStats DeviceSolver::solve(const double* diag, const double* upper, const double* lower, const double* b,
                               double* x, Method method, bool use_amg, const SolveControl& control) {
    const cfdb_control cc = to_c(control);
    cfdb_stats st{};
    check(cfdb_system_solve(impl_->sys, diag, upper, lower, b, x, method_c(method), use_amg ? 1 : 0, &cc, &st));
    return from_c(st);
}

bool DeviceSolver::on_device() const { return cfdb_system_on_device(impl_->sys) != 0; }

void DeviceSolver::set_mixed_precision(bool mixed) {
    check(cfdb_system_set_precision(impl_->sys, mixed ? CFDB_PRECISION_MIXED : CFDB_PRECISION_FP64));
}

void* DeviceSolver::handle() const { return impl_->sys; }

namespace {
cfdb_amg_settings amg_c(const AmgSetupSettings& a) {
    cfdb_amg_settings s{};
    cfdb_default_amg_settings(&s);
    s.strength_threshold = a.strength_threshold;
    s.max_levels = a.max_levels;
    s.coarse_size = a.coarse_size;
    return s;
}
} // namespace

void DeviceSolver::setup_amg(const double* diag, const double* upper, const double* lower,
                             const AmgSetupSettings& settings) {
    const cfdb_amg_settings s = amg_c(settings);
    check(cfdb_system_setup_amg_device(impl_->sys, diag, upper, lower, &s, 0));
}

LduSolveResult DeviceSolver::solve_ldu(const double* diag, const double* upper, const double* lower,
                                       const double* source, double* x, const LduSolveSettings& settings,
                                       const AmgSetupSettings& amg) {
    cfdb_ldu_settings ls{};
    ls.method = method_c(settings.method);
    ls.tolerance = settings.tolerance;
    ls.rel_tolerance = settings.rel_tolerance;
    ls.max_iterations = settings.max_iterations;
    ls.max_age = settings.max_age;
    const cfdb_amg_settings as = amg_c(amg);
    cfdb_ldu_result r{};
    check(cfdb_system_solve_ldu(impl_->sys, diag, upper, lower, source, x, &ls, &as, 0, &r));
    LduSolveResult o;
    o.initial_residual = r.initial_residual;
    o.final_residual = r.final_residual;
    o.iterations = r.iterations;
    o.amg_rebuilt = r.amg_rebuilt != 0;
    return o;
}

void assemble_convection_diffusion(int n_cells, int n_faces, const int* owner, const int* neighbour,
                                   const double* flux, const double* gamma, const double* delta_coeff,
                                   double convection, double* upper, double* lower, double* diag,
                                   double* divergence) {
    check(cfdb_assemble(n_cells, n_faces, owner, neighbour, flux, gamma, delta_coeff, convection, upper, lower,
                        diag, divergence));
}

std::string backend_name() {
    char buf[64];
    check(cfdb_backend_name(buf, sizeof(buf)));
    return buf;
}

bool device_available() { return cfdb_device_available() != 0; }

std::string device_description() {
    char buf[256];
    check(cfdb_device_description(buf, sizeof(buf)));
    return buf;
}

} // namespace cfd::gpu
