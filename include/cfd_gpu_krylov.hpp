// C++ front end of cfdb with the call surface of the reference's accelerator layer
// (namespace cfd::gpu, src/gpu/include/cfd/gpu/krylov.hpp): the same type names, members,
// defaults and signatures, so the reference's callers (LduMatrix::solve_persistent,
// ldu_matrix.cpp:287-366; FlowSolver::pressure_correction, flow_solver.cpp:757-796; the tests
// of test_gpu.cpp) compile against it unchanged. Every call goes through the C ABI of
// include/cfdb.h (implemented in libcfdb.so) and runs on the GPU; there is no host fallback.
//
// Errors are thrown as the reference throws them: std::invalid_argument for bad arguments
// (krylov.hpp callers rely on it for an empty hierarchy, device_solver.cpp:89) and
// std::runtime_error("CUDA ...") for device failures (krylov_cuda.cu:18-22).
//
// The reference's host-thread path (solve_host, solve_amg_cg_host and the detail:: host
// functions, krylov.hpp:41-42, 63-64, 125-136) is the reference's CPU code, not a GPU fallback:
// libcfdb.so does not implement it. A drop-in build links the reference's own
// src/gpu/src/krylov_openmp.cpp object beside libcfdb.so; it defines solve_host and the
// detail:: functions, and solve_amg_cg_host below forwards to it as dispatch.cpp:25-28 does.
#pragma once

#include <memory>
#include <string>
#include <vector>

namespace cfd::gpu {

// krylov.hpp:10-16
struct CsrView {
    int n = 0;
    int nnz = 0;
    const int* row_ptr = nullptr;
    const int* col = nullptr;
    const double* val = nullptr;
};

// krylov.hpp:19
enum class Method { Cg, BiCgStab };

// krylov.hpp:21-24
struct SolveControl {
    double abs_tolerance = 1e-10;
    int max_iterations = 1000;
};

// krylov.hpp:26-31
struct SolveStats {
    int iterations = 0;
    double residual = 0.0;
    bool converged = false;
    bool on_device = false;
};

// krylov.hpp:37-38: Jacobi-preconditioned CG or BiCGStab on a host CSR matrix, on the GPU.
SolveStats solve(const CsrView& a, const double* b, double* x, Method method,
                 const SolveControl& control);

// krylov.hpp:41-42: the same algorithms on host threads -- defined by the reference's
// krylov_openmp.cpp (linked beside libcfdb.so), not by libcfdb.so.
SolveStats solve_host(const CsrView& a, const double* b, double* x, Method method,
                      const SolveControl& control);

// krylov.hpp:48-58
struct AmgLevelView {
    CsrView a;
    CsrView p;
    CsrView r;
};
struct AmgView {
    std::vector<AmgLevelView> levels;
    const double* coarse_inverse = nullptr;
    int smooth_sweeps = 2;
    double jacobi_weight = 0.7;
};

// krylov.hpp:61-62
SolveStats solve_amg_cg(const AmgView& amg, const double* b, double* x,
                        const SolveControl& control);

// krylov.hpp:125-136: the reference's host implementation, defined by its krylov_openmp.cpp.
namespace detail {
SolveStats solve_openmp(const CsrView& a, const double* b, double* x, Method method,
                        const SolveControl& control);
SolveStats solve_openmp(const CsrView& a, const double* b, double* x, Method method,
                        const SolveControl& control, bool allow_device);
bool openmp_device_available();
SolveStats solve_amg_openmp(const AmgView& amg, const double* b, double* x,
                            const SolveControl& control, bool allow_device);
void assemble_openmp(int n_cells, int n_faces, const int* owner, const int* neighbour,
                     const double* flux, const double* gamma, const double* delta_coeff,
                     double convection, double* upper, double* lower, double* diag,
                     double* divergence);
} // namespace detail

// krylov.hpp:63-64: AMG-PCG on host threads, through the reference's krylov_openmp.cpp (the
// one-line forwarder of dispatch.cpp:25-28).
inline SolveStats solve_amg_cg_host(const AmgView& amg, const double* b, double* x,
                                    const SolveControl& control) {
    return detail::solve_amg_openmp(amg, b, x, control, false);
}

// krylov.hpp:68-77
struct LduPattern {
    int n = 0;
    int n_faces = 0;
    int nnz = 0;
    const int* row_ptr = nullptr;
    const int* col = nullptr;
    const int* diag_pos = nullptr;
    const int* upper_pos = nullptr;
    const int* lower_pos = nullptr;
};

// Extensions (no reference counterpart) used by DeviceSolver::setup_amg / solve_ldu below.
// amg.hpp:17-23 AmgSettings.
struct AmgSetupSettings {
    double strength_threshold = 0.08;
    int max_levels = 25;
    int coarse_size = 400;
};
// ldu_matrix.hpp:23-28 LinearSolverSettings of the GPU path, with AmgCache::max_age.
struct LduSolveSettings {
    Method method = Method::Cg;  // LinearSolverType::GpuCg (AMG-CG) or GpuBiCgStab
    double tolerance = 1e-10;    // absolute, on the normalised residual
    double rel_tolerance = 0.01; // relative to the initial normalised residual
    int max_iterations = 1000;
    int max_age = 20;            // hierarchy rebuilt after this many CG solves
};
// ldu_matrix.hpp:30-34 LinearSolveResult.
struct LduSolveResult {
    double initial_residual = 0.0;
    double final_residual = 0.0;
    int iterations = 0;
    bool amg_rebuilt = false;
};

// krylov.hpp:83-103: persistent solver on one pattern; the device matrix is assembled from
// LDU coefficients on every solve and the AMG hierarchy stays resident between set_amg calls.
class DeviceSolver {
public:
    explicit DeviceSolver(const LduPattern& pattern);
    ~DeviceSolver();
    DeviceSolver(const DeviceSolver&) = delete;
    DeviceSolver& operator=(const DeviceSolver&) = delete;
    DeviceSolver(DeviceSolver&&) = delete;
    DeviceSolver& operator=(DeviceSolver&&) = delete;

    void set_amg(const AmgView& amg);
    SolveStats solve(const double* diag, const double* upper, const double* lower,
                     const double* b, double* x, Method method, bool use_amg,
                     const SolveControl& control);
    [[nodiscard]] bool on_device() const;

    // Extensions (no reference counterpart): the arithmetic of the V-cycle (false: FP64, the
    // reference algorithm; true: FP32 V-cycle inside FP64 flexible CG) and the C handle.
    void set_mixed_precision(bool mixed);
    [[nodiscard]] void* handle() const;
    // AmgPreconditioner::setup of the LDU matrix on the GPU and installation of the hierarchy
    // (replaces the host setup + set_amg of LduMatrix::solve_persistent, ldu_matrix.cpp:314-353).
    void setup_amg(const double* diag, const double* upper, const double* lower,
                   const AmgSetupSettings& settings = {});
    // LduMatrix::solve with the GPU path and its AmgCache (ldu_matrix.cpp:111-131, 287-366):
    // normalised residuals on the device, hierarchy (re)built on the device every max_age CG
    // solves. Host arrays; x is the initial guess in and the solution out.
    LduSolveResult solve_ldu(const double* diag, const double* upper, const double* lower,
                             const double* source, double* x, const LduSolveSettings& settings,
                             const AmgSetupSettings& amg = {});

private:
    struct Impl;
    std::unique_ptr<Impl> impl_;
};

// krylov.hpp:105-116 (pressure equation: convection = 0). diag and divergence accumulate.
void assemble_convection_diffusion(int n_cells, int n_faces, const int* owner,
                                   const int* neighbour, const double* flux, const double* gamma,
                                   const double* delta_coeff, double convection, double* upper,
                                   double* lower, double* diag, double* divergence);

// krylov.hpp:118-123
[[nodiscard]] std::string backend_name();
[[nodiscard]] bool device_available();
[[nodiscard]] std::string device_description();

} // namespace cfd::gpu
