// C++ front end of the finite-volume cell kernels with the call surface of the reference's
// cfd::gpu::DeviceFv (src/gpu/include/cfd/gpu/fv_device.hpp:15-72): the same FvMeshView members
// and DeviceFv signatures, so FvGeometry::device() (fv_geometry.cpp:209-260) and its callers
// (FlowSolver::velocity_gradient / momentum corrections, flow_solver.cpp:225-241, 530-537;
// scalar_transport.cpp:83) compile against it unchanged. Every call goes through the C ABI of
// include/cfdb.h (libcfdb.so) and runs on the GPU; there is no host-thread fallback, so
// on_device() is always true.
//
// Errors: std::invalid_argument for a bad mesh view or argument (fv_device.cpp:17-27),
// std::logic_error for momentum_corrections before vector_gradient (fv_openmp.cpp:205-207),
// std::runtime_error("CUDA ...") for device failures.
#pragma once

#include <memory>

namespace cfd::gpu {

// fv_device.hpp:15-31. Faces [0, n_internal_faces) are internal; vectors are 3 doubles per entry.
struct FvMeshView {
    int n_cells = 0;
    int n_internal_faces = 0;
    int n_faces = 0;
    const int* owner = nullptr;          // n_faces
    const int* neighbour = nullptr;      // n_internal_faces
    const int* cell_offsets = nullptr;   // n_cells + 1: faces of each cell (CSR) ...
    const int* cell_faces = nullptr;     // ... in ascending face order
    const double* weight = nullptr;      // n_internal_faces
    const double* sf = nullptr;          // 3 n_faces
    const double* face_centre = nullptr; // 3 n_faces
    const double* cell_centre = nullptr; // 3 n_cells
    const double* volume = nullptr;      // n_cells
    const double* correction = nullptr;  // 3 n_faces
    const double* lsq_d = nullptr;       // 3 n_faces
    const double* lsq_inverse = nullptr; // 9 n_cells, column-major
};

// fv_device.hpp:33-72. scheme: 0 Green-Gauss, 1 least squares, 2 skewness-corrected Gauss.
class DeviceFv {
public:
    explicit DeviceFv(const FvMeshView& mesh);
    ~DeviceFv();
    DeviceFv(const DeviceFv&) = delete;
    DeviceFv& operator=(const DeviceFv&) = delete;

    void gradient(const double* phi, const double* bv, int scheme, double* grad);
    void vector_gradient(const double* u, const double* ub, int scheme, double* grad);
    void scalar_corrections(const double* phi, const double* bv, int scheme, const double* flux,
                            const double* gamma, bool linear_upwind, double* source);
    void momentum_corrections(const double* flux, const double* nu_face, bool linear_upwind,
                              bool limited, bool venkat, const double* eps2, double central,
                              bool transpose_term, double* source);
    [[nodiscard]] bool on_device() const;

    // Extension (no reference counterpart): the C handle, for the *_device entry points of
    // include/cfdb.h that take device arrays.
    [[nodiscard]] void* handle() const;

    struct Impl;

private:
    std::unique_ptr<Impl> impl_;
};

} // namespace cfd::gpu
