// Pressure gradient and velocity correction of FlowSolver::pressure_correction on the device
// (the Gauss branch of FlowSolver::pressure_gradient, flow_solver.cpp:339-372, and the velocity
// correction, flow_solver.cpp:843-846).
//
// The reference accumulates face by face: each internal face adds S_f p_f to its owner and
// subtracts it from its neighbour, then each boundary face adds S_f p_b to its owner. Here
// one thread per cell walks its internal faces in ascending face order and then its boundary
// faces in ascending order, so every cell receives the same contributions in the same order;
// every product and sum is rounded separately (no FMA). Vectors are xyz-interleaved.
#include "../../include/cfdb.h"

#include <algorithm>
#include <string>
#include <vector>

#include "common.hpp"

namespace cfdb {
void set_thread_error(const std::string& msg);
} // namespace cfdb

using namespace cfdb;

struct cfdb_fv {
    int device = 0;
    int n = 0, nf = 0, ni = 0;
    cudaStream_t st = nullptr;
    DeviceArena mem;
    int* owner = nullptr;     // n_faces
    int* neighbour = nullptr; // internal faces
    double* w = nullptr;      // internal faces
    double* sf = nullptr;     // 3 n_faces
    double* cf = nullptr;     // 3 n_faces
    double* cc = nullptr;     // 3 n_cells
    double* vol = nullptr;    // n_cells
    int* kind = nullptr;      // boundary faces: cfdb_boundary_kind
    double* pout = nullptr;   // boundary faces: outlet pressure
    int* iptr = nullptr;      // cell -> internal faces (ascending)
    int* iface = nullptr;
    int* bptr = nullptr;      // cell -> boundary faces (ascending)
    int* bface = nullptr;
    double* internal = nullptr; // 3 n_cells: internal-face part of the gradient sum
    double* prev = nullptr;     // 3 n_cells: first-pass gradient
    ~cfdb_fv() {
        if (st != nullptr) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
    }
};

namespace {

// sum over the cell's internal faces, in face order, of +-S_f (w p_P + (1 - w) p_N)
__global__ void k_grad_internal(int n, const int* __restrict__ iptr, const int* __restrict__ iface,
                                const int* __restrict__ owner, const int* __restrict__ neighbour,
                                const double* __restrict__ w, const double* __restrict__ sf,
                                const double* __restrict__ p, double* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    double g0 = 0.0, g1 = 0.0, g2 = 0.0;
    for (int k = iptr[c]; k < iptr[c + 1]; ++k) {
        const int f = iface[k];
        const int o = owner[f];
        const double wf = w[f];
        const double s = __dadd_rn(__dmul_rn(wf, p[o]), __dmul_rn(__dsub_rn(1.0, wf), p[neighbour[f]]));
        const double f0 = __dmul_rn(sf[3 * f], s), f1 = __dmul_rn(sf[3 * f + 1], s), f2 = __dmul_rn(sf[3 * f + 2], s);
        if (o == c) {
            g0 = __dadd_rn(g0, f0);
            g1 = __dadd_rn(g1, f1);
            g2 = __dadd_rn(g2, f2);
        } else {
            g0 = __dsub_rn(g0, f0);
            g1 = __dsub_rn(g1, f1);
            g2 = __dsub_rn(g2, f2);
        }
    }
    out[3 * c] = g0;
    out[3 * c + 1] = g1;
    out[3 * c + 2] = g2;
}

// grad = (internal + sum over the cell's boundary faces of S_f p_b) / V. Pass 2 (prev != null)
// extrapolates p_b of every boundary face but pressure outlets tangentially with the first-pass
// gradient: p_b = p_P + prev_P . (d - (d . n) n), d = face centre - cell centre, n = S / |S|.
__global__ void k_grad_boundary(int n, int ni, const int* __restrict__ bptr, const int* __restrict__ bface,
                                const int* __restrict__ kind, const double* __restrict__ pout,
                                const double* __restrict__ sf, const double* __restrict__ cf,
                                const double* __restrict__ cc, const double* __restrict__ vol,
                                const double* __restrict__ p, const double* __restrict__ internal,
                                const double* __restrict__ prev, double* __restrict__ grad) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    double g0 = internal[3 * c], g1 = internal[3 * c + 1], g2 = internal[3 * c + 2];
    for (int k = bptr[c]; k < bptr[c + 1]; ++k) {
        const int f = bface[k];
        const int b = f - ni;
        const bool outlet = kind[b] == CFDB_BC_PRESSURE_OUTLET;
        double pb = outlet ? pout[b] : p[c];
        const double s0 = sf[3 * f], s1 = sf[3 * f + 1], s2 = sf[3 * f + 2];
        if (prev != nullptr && !outlet) {
            const double area = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(s0, s0), __dmul_rn(s1, s1)), __dmul_rn(s2, s2)));
            const double n0 = __ddiv_rn(s0, area), n1 = __ddiv_rn(s1, area), n2 = __ddiv_rn(s2, area);
            const double d0 = __dsub_rn(cf[3 * f], cc[3 * c]);
            const double d1 = __dsub_rn(cf[3 * f + 1], cc[3 * c + 1]);
            const double d2 = __dsub_rn(cf[3 * f + 2], cc[3 * c + 2]);
            const double dn = __dadd_rn(__dadd_rn(__dmul_rn(d0, n0), __dmul_rn(d1, n1)), __dmul_rn(d2, n2));
            const double t0 = __dsub_rn(d0, __dmul_rn(dn, n0));
            const double t1 = __dsub_rn(d1, __dmul_rn(dn, n1));
            const double t2 = __dsub_rn(d2, __dmul_rn(dn, n2));
            const double e = __dadd_rn(__dadd_rn(__dmul_rn(prev[3 * c], t0), __dmul_rn(prev[3 * c + 1], t1)),
                                       __dmul_rn(prev[3 * c + 2], t2));
            pb = __dadd_rn(pb, e);
        }
        g0 = __dadd_rn(g0, __dmul_rn(s0, pb));
        g1 = __dadd_rn(g1, __dmul_rn(s1, pb));
        g2 = __dadd_rn(g2, __dmul_rn(s2, pb));
    }
    const double v = vol[c];
    grad[3 * c] = __ddiv_rn(g0, v);
    grad[3 * c + 1] = __ddiv_rn(g1, v);
    grad[3 * c + 2] = __ddiv_rn(g2, v);
}

// u = HbyA - rAU grad p
__global__ void k_correct_velocity(int n, const double* __restrict__ hbya, const double* __restrict__ rau,
                                   const double* __restrict__ grad, double* __restrict__ u) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const double r = rau[c];
    for (int i = 0; i < 3; ++i) u[3 * c + i] = __dsub_rn(hbya[3 * c + i], __dmul_rn(r, grad[3 * c + i]));
}

int grid(int n) { return std::max(1, (n + 255) / 256); }

template <class F> int guarded_fv(F&& f) {
    try {
        f();
        return CFDB_OK;
    } catch (const Error& e) {
        set_thread_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        set_thread_error(e.what());
        return CFDB_ERR_INTERNAL;
    }
}

} // namespace

extern "C" {

int cfdb_fv_create(int n_cells, int n_faces, int n_internal_faces, const int* owner, const int* neighbour,
                   const double* face_areas, const double* face_centres, const double* cell_centres,
                   const double* cell_volumes, const double* weights, const int* boundary_kind,
                   const double* boundary_pressure, cfdb_fv** out) {
    return guarded_fv([&] {
        if (out == nullptr || n_cells <= 0 || n_internal_faces < 0 || n_faces < n_internal_faces)
            fail(CFDB_ERR_BAD_ARG, "cfdb_fv_create: bad sizes");
        const int nb = n_faces - n_internal_faces;
        if (!owner || (n_internal_faces > 0 && (!neighbour || !weights)) || !face_areas || !face_centres ||
            !cell_centres || !cell_volumes || (nb > 0 && (!boundary_kind || !boundary_pressure)))
            fail(CFDB_ERR_BAD_ARG, "cfdb_fv_create: null array");
        for (int f = 0; f < n_faces; ++f) {
            if (owner[f] < 0 || owner[f] >= n_cells || (f < n_internal_faces && (neighbour[f] < 0 || neighbour[f] >= n_cells)))
                fail(CFDB_ERR_BAD_ARG, "cfdb_fv_create: face " + std::to_string(f) + " addresses a cell out of range");
        }
        for (int b = 0; b < nb; ++b)
            if (boundary_kind[b] < CFDB_BC_VELOCITY_INLET || boundary_kind[b] > CFDB_BC_EMPTY)
                fail(CFDB_ERR_BAD_ARG, "cfdb_fv_create: unknown boundary kind");
        auto* fv = new cfdb_fv;
        try {
            CFDB_CUDA(cudaGetDevice(&fv->device));
            CFDB_CUDA(cudaStreamCreateWithFlags(&fv->st, cudaStreamNonBlocking));
            fv->n = n_cells;
            fv->nf = n_faces;
            fv->ni = n_internal_faces;
            // cell -> face lists in ascending face order
            std::vector<int> iptr(n_cells + 1, 0), bptr(n_cells + 1, 0);
            for (int f = 0; f < n_internal_faces; ++f) {
                ++iptr[owner[f] + 1];
                ++iptr[neighbour[f] + 1];
            }
            for (int f = n_internal_faces; f < n_faces; ++f) ++bptr[owner[f] + 1];
            for (int c = 0; c < n_cells; ++c) {
                iptr[c + 1] += iptr[c];
                bptr[c + 1] += bptr[c];
            }
            std::vector<int> iface(iptr[n_cells]), bface(bptr[n_cells]);
            std::vector<int> fi(iptr.begin(), iptr.end() - 1), fb(bptr.begin(), bptr.end() - 1);
            for (int f = 0; f < n_internal_faces; ++f) {
                iface[fi[owner[f]]++] = f;
                iface[fi[neighbour[f]]++] = f;
            }
            for (int f = n_internal_faces; f < n_faces; ++f) bface[fb[owner[f]]++] = f;
            auto up = [&](const auto* src, size_t cnt) {
                using T = std::remove_const_t<std::remove_pointer_t<decltype(src)>>;
                std::vector<T> h(src, src + cnt);
                return fv->mem.upload(h, fv->st);
            };
            fv->owner = up(owner, n_faces);
            fv->neighbour = up(neighbour, n_internal_faces);
            fv->w = up(weights, n_internal_faces);
            fv->sf = up(face_areas, 3 * static_cast<size_t>(n_faces));
            fv->cf = up(face_centres, 3 * static_cast<size_t>(n_faces));
            fv->cc = up(cell_centres, 3 * static_cast<size_t>(n_cells));
            fv->vol = up(cell_volumes, n_cells);
            fv->kind = up(boundary_kind, nb);
            fv->pout = up(boundary_pressure, nb);
            fv->iptr = fv->mem.upload(iptr, fv->st);
            fv->iface = fv->mem.upload(iface, fv->st);
            fv->bptr = fv->mem.upload(bptr, fv->st);
            fv->bface = fv->mem.upload(bface, fv->st);
            fv->internal = fv->mem.alloc<double>(3 * static_cast<size_t>(n_cells));
            fv->prev = fv->mem.alloc<double>(3 * static_cast<size_t>(n_cells));
            CFDB_CUDA(cudaStreamSynchronize(fv->st));
        } catch (...) {
            delete fv;
            throw;
        }
        *out = fv;
    });
}

int cfdb_fv_destroy(cfdb_fv* fv) {
    if (fv != nullptr) {
        cudaSetDevice(fv->device);
        delete fv;
    }
    return CFDB_OK;
}

int cfdb_fv_pressure_gradient_device(cfdb_fv* fv, const double* p, double* grad) {
    return guarded_fv([&] {
        if (fv == nullptr || p == nullptr || grad == nullptr) fail(CFDB_ERR_BAD_ARG, "null argument");
        CFDB_CUDA(cudaSetDevice(fv->device));
        const int n = fv->n;
        k_grad_internal<<<grid(n), 256, 0, fv->st>>>(n, fv->iptr, fv->iface, fv->owner, fv->neighbour, fv->w, fv->sf, p,
                                                     fv->internal);
        // two passes (flow_solver.cpp:348-370): the second extrapolates with the first's result
        k_grad_boundary<<<grid(n), 256, 0, fv->st>>>(n, fv->ni, fv->bptr, fv->bface, fv->kind, fv->pout, fv->sf, fv->cf,
                                                     fv->cc, fv->vol, p, fv->internal, nullptr, fv->prev);
        k_grad_boundary<<<grid(n), 256, 0, fv->st>>>(n, fv->ni, fv->bptr, fv->bface, fv->kind, fv->pout, fv->sf, fv->cf,
                                                     fv->cc, fv->vol, p, fv->internal, fv->prev, grad);
        CFDB_CUDA(cudaGetLastError());
        CFDB_CUDA(cudaStreamSynchronize(fv->st));
    });
}

int cfdb_fv_correct_velocity_device(cfdb_fv* fv, const double* hbya, const double* rau, const double* grad,
                                    double* u) {
    return guarded_fv([&] {
        if (fv == nullptr || hbya == nullptr || rau == nullptr || grad == nullptr || u == nullptr)
            fail(CFDB_ERR_BAD_ARG, "null argument");
        CFDB_CUDA(cudaSetDevice(fv->device));
        k_correct_velocity<<<grid(fv->n), 256, 0, fv->st>>>(fv->n, hbya, rau, grad, u);
        CFDB_CUDA(cudaGetLastError());
        CFDB_CUDA(cudaStreamSynchronize(fv->st));
    });
}

} // extern "C"
