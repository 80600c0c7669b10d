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
#include <cmath>
#include <string>
#include <vector>

#include "common.hpp"

static_assert(CFDB_ERR_NO_DEVICE == 4, "require_cuda_device (common.hpp) reports status 4");

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
    double* delta = nullptr;  // n_faces: delta coefficients (fv_geometry.cpp:43-50)
    double* corr = nullptr;   // 3 internal faces: non-orthogonal corrections S - d delta
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

// HbyA = (source - offdiag(U) U) / diag and rAU = V / mean(diag) (flow_solver.cpp:688-707),
// per component; the off-diagonal product gathers the cell's faces in ascending order
// (ldu_matrix.cpp:39-49: upper * x[N] for owned faces, lower * x[P] otherwise).
__global__ void k_hbya_rau(int n, const int* __restrict__ iptr, const int* __restrict__ iface,
                           const int* __restrict__ owner, const int* __restrict__ neighbour,
                           const double* __restrict__ upper, const double* __restrict__ lower,
                           const double* __restrict__ diag, const double* __restrict__ source,
                           const double* __restrict__ u, const double* __restrict__ vol,
                           double* __restrict__ hbya, double* __restrict__ rau) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    for (int i = 0; i < 3; ++i) {
        double off = 0.0;
        for (int k = iptr[c]; k < iptr[c + 1]; ++k) {
            const int f = iface[k];
            const int o = owner[f];
            off = o == c ? __dadd_rn(off, __dmul_rn(upper[f], u[3 * neighbour[f] + i]))
                         : __dadd_rn(off, __dmul_rn(lower[f], u[3 * o + i]));
        }
        hbya[3 * c + i] = __ddiv_rn(__dsub_rn(source[3 * c + i], off), diag[3 * c + i]);
    }
    const double mean = __ddiv_rn(__dadd_rn(__dadd_rn(diag[3 * c], diag[3 * c + 1]), diag[3 * c + 2]), 3.0);
    rau[c] = __ddiv_rn(vol[c], mean);
}

__device__ __forceinline__ double dot3(const double* a, const double* b) {
    return __dadd_rn(__dadd_rn(__dmul_rn(a[0], b[0]), __dmul_rn(a[1], b[1])), __dmul_rn(a[2], b[2]));
}

// predicted face flux and face rAU (flow_solver.cpp:709-733), with the relaxation-independent
// correction when u_prev / phi_prev are given (flow_solver.cpp:735-752)
__global__ void k_face_flux(int nf, int ni, const int* __restrict__ owner, const int* __restrict__ neighbour,
                            const double* __restrict__ w, const double* __restrict__ sf,
                            const int* __restrict__ kind, const double* __restrict__ hbya,
                            const double* __restrict__ rau, const double* __restrict__ ufix,
                            const double* __restrict__ u_prev, const double* __restrict__ phi_prev, double beta,
                            double* __restrict__ phi, double* __restrict__ rau_f) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const int o = owner[f];
    const double* s = sf + 3 * f;
    double ph, rf;
    if (f < ni) {
        const int nb = neighbour[f];
        const double wf = w[f], wn = __dsub_rn(1.0, wf);
        double v[3];
        for (int i = 0; i < 3; ++i) v[i] = __dadd_rn(__dmul_rn(wf, hbya[3 * o + i]), __dmul_rn(wn, hbya[3 * nb + i]));
        ph = dot3(v, s);
        rf = __dadd_rn(__dmul_rn(wf, rau[o]), __dmul_rn(wn, rau[nb]));
        if (u_prev != nullptr) {
            double uf[3];
            for (int i = 0; i < 3; ++i) uf[i] = __dadd_rn(__dmul_rn(wf, u_prev[3 * o + i]), __dmul_rn(wn, u_prev[3 * nb + i]));
            ph = __dadd_rn(ph, __dmul_rn(beta, __dsub_rn(phi_prev[f], dot3(uf, s))));
        }
    } else {
        const int b = f - ni;
        rf = rau[o];
        const int k = kind[b];
        if (k == CFDB_BC_VELOCITY_INLET || k == CFDB_BC_WALL) {
            ph = dot3(ufix + 3 * b, s);
        } else if (k == CFDB_BC_PRESSURE_OUTLET) {
            ph = dot3(hbya + 3 * o, s);
            if (u_prev != nullptr) ph = __dadd_rn(ph, __dmul_rn(beta, __dsub_rn(phi_prev[f], dot3(u_prev + 3 * o, s))));
        } else {
            ph = 0.0;
        }
    }
    phi[f] = ph;
    rau_f[f] = rf;
}

// boundary terms of the pressure equation (flow_solver.cpp:784-796): source -= phi_HbyA for
// every boundary face, and for outlets diag += rAU_f delta, source += rAU_f delta p_out; then
// set_reference(ref_cell, ref_value) (ldu_matrix.cpp:105-109) unless ref_cell < 0
__global__ void k_pressure_boundary(int n, int ni, const int* __restrict__ bptr, const int* __restrict__ bface,
                                    const int* __restrict__ kind, const double* __restrict__ pout,
                                    const double* __restrict__ phi, const double* __restrict__ rau_f,
                                    const double* __restrict__ delta, int ref_cell, double ref_value,
                                    double* __restrict__ diag, double* __restrict__ source) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    double d = diag[c], s = source[c];
    for (int k = bptr[c]; k < bptr[c + 1]; ++k) {
        const int f = bface[k];
        const int b = f - ni;
        s = __dsub_rn(s, phi[f]);
        if (kind[b] == CFDB_BC_PRESSURE_OUTLET) {
            const double coeff = __dmul_rn(rau_f[f], delta[f]);
            d = __dadd_rn(d, coeff);
            s = __dadd_rn(s, __dmul_rn(coeff, pout[b]));
        }
    }
    if (c == ref_cell) {
        s = __dadd_rn(s, __dmul_rn(d, ref_value));
        d = __dadd_rn(d, d);
    }
    diag[c] = d;
    source[c] = s;
}

// non-orthogonal correction fluxes rAU_f k . (w gp_P + (1 - w) gp_N) (flow_solver.cpp:808-815)
__global__ void k_non_orth_faces(int ni, const int* __restrict__ owner, const int* __restrict__ neighbour,
                                 const double* __restrict__ w, const double* __restrict__ corr,
                                 const double* __restrict__ rau_f, const double* __restrict__ grad,
                                 double* __restrict__ non_orth) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= ni) return;
    const int o = owner[f], nb = neighbour[f];
    const double wf = w[f], wn = __dsub_rn(1.0, wf);
    double v[3];
    for (int i = 0; i < 3; ++i) v[i] = __dadd_rn(__dmul_rn(wf, grad[3 * o + i]), __dmul_rn(wn, grad[3 * nb + i]));
    non_orth[f] = __dmul_rn(rau_f[f], dot3(corr + 3 * f, v));
}

// source = base + (owned faces) non_orth - (neighbour faces) non_orth, faces in ascending order
__global__ void k_non_orth_source(int n, const int* __restrict__ iptr, const int* __restrict__ iface,
                                  const int* __restrict__ owner, const double* __restrict__ non_orth,
                                  const double* __restrict__ base, double* __restrict__ source) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    double s = base[c];
    for (int k = iptr[c]; k < iptr[c + 1]; ++k) {
        const int f = iface[k];
        s = owner[f] == c ? __dadd_rn(s, non_orth[f]) : __dsub_rn(s, non_orth[f]);
    }
    source[c] = s;
}

// conservative face flux on every face (flow_solver.cpp:818-833)
__global__ void k_fv_correct_flux(int nf, int ni, const int* __restrict__ owner, const int* __restrict__ neighbour,
                                  const int* __restrict__ kind, const double* __restrict__ pout,
                                  const double* __restrict__ phi_hbya, const double* __restrict__ rau_f,
                                  const double* __restrict__ delta, const double* __restrict__ non_orth,
                                  const double* __restrict__ p, double* __restrict__ phi) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const int o = owner[f];
    const double coeff = __dmul_rn(rau_f[f], delta[f]);
    if (f < ni) {
        const double v = __dsub_rn(phi_hbya[f], __dmul_rn(coeff, __dsub_rn(p[neighbour[f]], p[o])));
        phi[f] = __dsub_rn(v, non_orth != nullptr ? non_orth[f] : 0.0);
    } else {
        const int b = f - ni;
        double v = phi_hbya[f];
        if (kind[b] == CFDB_BC_PRESSURE_OUTLET) v = __dsub_rn(v, __dmul_rn(coeff, __dsub_rn(pout[b], p[o])));
        phi[f] = v;
    }
}

// p = p_prev + alpha (p_new - p_prev) (flow_solver.cpp:837-840)
__global__ void k_fv_relax(int n, const double* __restrict__ p_prev, const double* __restrict__ p_new,
                           double alpha, double* __restrict__ p) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    p[c] = __dadd_rn(p_prev[c], __dmul_rn(alpha, __dsub_rn(p_new[c], p_prev[c])));
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
        require_cuda_device();
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
            // delta coefficients of every face and non-orthogonal corrections of the internal ones
            // (fv_geometry.cpp:34-50): delta = |S|^2 / max(S.d, 0.05 |S||d|), k = S - d delta,
            // d = centre of the neighbour (or of the boundary face) minus centre of the owner
            std::vector<double> delta(n_faces), corr(3 * static_cast<size_t>(n_internal_faces));
            auto dot = [](const double* a, const double* b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; };
            for (int f = 0; f < n_faces; ++f) {
                const double* s = face_areas + 3 * static_cast<size_t>(f);
                const double* cp = cell_centres + 3 * static_cast<size_t>(owner[f]);
                const double* to = f < n_internal_faces ? cell_centres + 3 * static_cast<size_t>(neighbour[f])
                                                        : face_centres + 3 * static_cast<size_t>(f);
                const double d[3] = {to[0] - cp[0], to[1] - cp[1], to[2] - cp[2]};
                const double area = std::sqrt(dot(s, s));
                const double s_dot_d = std::max(dot(s, d), 0.05 * area * std::sqrt(dot(d, d)));
                if (!(area > 0.0) || !(s_dot_d > 0.0)) fail(CFDB_ERR_BAD_ARG, "cfdb_fv_create: degenerate face " + std::to_string(f));
                delta[f] = area * area / s_dot_d;
                if (f < n_internal_faces)
                    for (int i = 0; i < 3; ++i) corr[3 * static_cast<size_t>(f) + i] = s[i] - d[i] * delta[f];
            }
            fv->delta = fv->mem.upload(delta, fv->st);
            fv->corr = fv->mem.upload(corr, fv->st);
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

int cfdb_fv_sizes(const cfdb_fv* fv, int* n_cells, int* n_faces, int* n_internal_faces) {
    if (fv == nullptr) return CFDB_ERR_BAD_ARG;
    if (n_cells) *n_cells = fv->n;
    if (n_faces) *n_faces = fv->nf;
    if (n_internal_faces) *n_internal_faces = fv->ni;
    return CFDB_OK;
}

int cfdb_fv_delta_device(const cfdb_fv* fv, const double** delta) {
    if (fv == nullptr || delta == nullptr) return CFDB_ERR_BAD_ARG;
    *delta = fv->delta;
    return CFDB_OK;
}

int cfdb_fv_hbya_rau_device(cfdb_fv* fv, const double* mom_diag, const double* mom_upper, const double* mom_lower,
                            const double* mom_source, const double* u, double* hbya, double* rau) {
    return guarded_fv([&] {
        if (fv == nullptr || !mom_diag || !mom_source || !u || !hbya || !rau ||
            (fv->ni > 0 && (!mom_upper || !mom_lower)))
            fail(CFDB_ERR_BAD_ARG, "null argument");
        CFDB_CUDA(cudaSetDevice(fv->device));
        k_hbya_rau<<<grid(fv->n), 256, 0, fv->st>>>(fv->n, fv->iptr, fv->iface, fv->owner, fv->neighbour, mom_upper,
                                                    mom_lower, mom_diag, mom_source, u, fv->vol, hbya, rau);
        CFDB_CUDA(cudaGetLastError());
        CFDB_CUDA(cudaStreamSynchronize(fv->st));
    });
}

int cfdb_fv_face_flux_device(cfdb_fv* fv, const double* hbya, const double* rau, const double* fixed_velocity,
                             const double* u_prev, const double* phi_prev, double beta, double* phi_hbya,
                             double* rau_f) {
    return guarded_fv([&] {
        if (fv == nullptr || !hbya || !rau || !phi_hbya || !rau_f || (fv->nf > fv->ni && !fixed_velocity) ||
            ((u_prev == nullptr) != (phi_prev == nullptr)))
            fail(CFDB_ERR_BAD_ARG, "null argument (u_prev and phi_prev go together)");
        CFDB_CUDA(cudaSetDevice(fv->device));
        k_face_flux<<<grid(fv->nf), 256, 0, fv->st>>>(fv->nf, fv->ni, fv->owner, fv->neighbour, fv->w, fv->sf, fv->kind,
                                                      hbya, rau, fixed_velocity, u_prev, phi_prev, beta, phi_hbya,
                                                      rau_f);
        CFDB_CUDA(cudaGetLastError());
        CFDB_CUDA(cudaStreamSynchronize(fv->st));
    });
}

int cfdb_fv_pressure_boundary_device(cfdb_fv* fv, const double* phi_hbya, const double* rau_f, int ref_cell,
                                     double ref_value, double* diag, double* source) {
    return guarded_fv([&] {
        if (fv == nullptr || !phi_hbya || !rau_f || !diag || !source) fail(CFDB_ERR_BAD_ARG, "null argument");
        if (ref_cell >= fv->n) fail(CFDB_ERR_BAD_ARG, "reference cell out of range");
        CFDB_CUDA(cudaSetDevice(fv->device));
        k_pressure_boundary<<<grid(fv->n), 256, 0, fv->st>>>(fv->n, fv->ni, fv->bptr, fv->bface, fv->kind, fv->pout,
                                                             phi_hbya, rau_f, fv->delta, ref_cell, ref_value, diag,
                                                             source);
        CFDB_CUDA(cudaGetLastError());
        CFDB_CUDA(cudaStreamSynchronize(fv->st));
    });
}

int cfdb_fv_non_orth_device(cfdb_fv* fv, const double* grad, const double* rau_f, const double* base_source,
                            double* non_orth, double* source) {
    return guarded_fv([&] {
        if (fv == nullptr || !grad || !rau_f || !base_source || !non_orth || !source)
            fail(CFDB_ERR_BAD_ARG, "null argument");
        CFDB_CUDA(cudaSetDevice(fv->device));
        if (fv->ni > 0)
            k_non_orth_faces<<<grid(fv->ni), 256, 0, fv->st>>>(fv->ni, fv->owner, fv->neighbour, fv->w, fv->corr, rau_f,
                                                               grad, non_orth);
        k_non_orth_source<<<grid(fv->n), 256, 0, fv->st>>>(fv->n, fv->iptr, fv->iface, fv->owner, non_orth, base_source,
                                                           source);
        CFDB_CUDA(cudaGetLastError());
        CFDB_CUDA(cudaStreamSynchronize(fv->st));
    });
}

int cfdb_fv_correct_flux_device(cfdb_fv* fv, const double* phi_hbya, const double* rau_f, const double* non_orth,
                                const double* p_new, double* phi) {
    return guarded_fv([&] {
        if (fv == nullptr || !phi_hbya || !rau_f || !p_new || !phi) fail(CFDB_ERR_BAD_ARG, "null argument");
        CFDB_CUDA(cudaSetDevice(fv->device));
        k_fv_correct_flux<<<grid(fv->nf), 256, 0, fv->st>>>(fv->nf, fv->ni, fv->owner, fv->neighbour, fv->kind,
                                                            fv->pout, phi_hbya, rau_f, fv->delta, non_orth, p_new,
                                                            phi);
        CFDB_CUDA(cudaGetLastError());
        CFDB_CUDA(cudaStreamSynchronize(fv->st));
    });
}

int cfdb_fv_relax_device(cfdb_fv* fv, const double* p_prev, const double* p_new, double alpha, double* p) {
    return guarded_fv([&] {
        if (fv == nullptr || !p_prev || !p_new || !p) fail(CFDB_ERR_BAD_ARG, "null argument");
        CFDB_CUDA(cudaSetDevice(fv->device));
        k_fv_relax<<<grid(fv->n), 256, 0, fv->st>>>(fv->n, p_prev, p_new, alpha, p);
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
