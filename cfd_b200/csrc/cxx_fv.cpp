// cfd::gpu::DeviceFv front end over the C ABI (declared in include/cfd_gpu_fv.hpp).
#include "../../include/cfd_gpu_fv.hpp"

#include <stdexcept>
#include <string>

#include "../../include/cfdb.h"

namespace cfd::gpu {

namespace {

void check(int rc) {
    if (rc == CFDB_OK) return;
    char buf[1024];
    cfdb_last_error(buf, sizeof(buf));
    const std::string msg(buf);
    if (rc == CFDB_ERR_BAD_ARG) throw std::invalid_argument(msg);
    if (rc == CFDB_ERR_NOT_READY) throw std::logic_error(msg);
    if (rc == CFDB_ERR_CUDA || rc == CFDB_ERR_OOM || rc == CFDB_ERR_NO_DEVICE) {
        throw std::runtime_error(msg.rfind("CUDA", 0) == 0 ? msg : "CUDA " + msg);
    }
    throw std::runtime_error(msg);
}

} // namespace

struct DeviceFv::Impl {
    cfdb_device_fv* fv = nullptr;
};

DeviceFv::DeviceFv(const FvMeshView& m) : impl_(std::make_unique<Impl>()) {
    const cfdb_fv_mesh_view v{m.n_cells, m.n_internal_faces, m.n_faces, m.owner, m.neighbour, m.cell_offsets,
                              m.cell_faces, m.weight, m.sf, m.face_centre, m.cell_centre, m.volume,
                              m.correction, m.lsq_d, m.lsq_inverse};
    check(cfdb_device_fv_create(&v, &impl_->fv));
}

DeviceFv::~DeviceFv() {
    if (impl_ && impl_->fv != nullptr) cfdb_device_fv_destroy(impl_->fv);
}

void DeviceFv::gradient(const double* phi, const double* bv, int scheme, double* grad) {
    check(cfdb_device_fv_gradient(impl_->fv, phi, bv, scheme, grad));
}

void DeviceFv::vector_gradient(const double* u, const double* ub, int scheme, double* grad) {
    check(cfdb_device_fv_vector_gradient(impl_->fv, u, ub, scheme, grad));
}

void DeviceFv::scalar_corrections(const double* phi, const double* bv, int scheme, const double* flux,
                                  const double* gamma, bool linear_upwind, double* source) {
    check(cfdb_device_fv_scalar_corrections(impl_->fv, phi, bv, scheme, flux, gamma, linear_upwind ? 1 : 0,
                                            source));
}

void DeviceFv::momentum_corrections(const double* flux, const double* nu_face, bool linear_upwind, bool limited,
                                    bool venkat, const double* eps2, double central, bool transpose_term,
                                    double* source) {
    check(cfdb_device_fv_momentum_corrections(impl_->fv, flux, nu_face, linear_upwind ? 1 : 0, limited ? 1 : 0,
                                              venkat ? 1 : 0, eps2, central, transpose_term ? 1 : 0, source));
}

bool DeviceFv::on_device() const { return cfdb_device_fv_on_device(impl_->fv) != 0; }

void* DeviceFv::handle() const { return impl_->fv; }

} // namespace cfd::gpu
