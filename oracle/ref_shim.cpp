// C-ABI shim over the reference's own host implementation of the accelerator path
// (TEST INFRASTRUCTURE ONLY). It is compiled together with the reference's unchanged sources
// src/gpu/src/{krylov_openmp.cpp, device_solver.cpp, dispatch.cpp} (which include
// krylov_kernels.inc) and src/gpu/src/{fv_openmp.cpp, fv_device.cpp} (which include
// fv_cell.inc) into oracle/_ref/libcfdref.so by oracle/build.py. Without CFD_GPU_CUDA
// those sources run the accelerator algorithm on host threads, exactly as the reference's CI
// does (.github/workflows/ci.yml:157-169). Used to pin the C oracle and as the timed
// reference CPU baseline.
#include <cfd/gpu/fv_device.hpp>
#include <cfd/gpu/krylov.hpp>

#include <exception>
#include <vector>

namespace {

struct RefCsr {
    int n;
    int nnz;
    const int* rp;
    const int* ci;
    const double* va;
};

cfd::gpu::CsrView view(const RefCsr& m) {
    if (m.rp == nullptr) {
        return {};
    }
    return {m.n, m.nnz, m.rp, m.ci, m.va};
}

void put(const cfd::gpu::SolveStats& st, int* iters, double* res, int* conv) {
    *iters = st.iterations;
    *res = st.residual;
    *conv = st.converged ? 1 : 0;
}

} // namespace

extern "C" {

// cfd::gpu::assemble_convection_diffusion (krylov.hpp:105-116) -> host serial loop.
int ref_assemble(int nc, int nf, const int* own, const int* nei, const double* flux,
                 const double* gamma, const double* delta, double conv, double* upper,
                 double* lower, double* diag, double* div) {
    try {
        cfd::gpu::assemble_convection_diffusion(nc, nf, own, nei, flux, gamma, delta, conv, upper,
                                                lower, diag, div);
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

// cfd::gpu::solve_host (krylov.hpp:41-42): Jacobi CG (method 0) / BiCGStab (method 1).
int ref_solve_host(const RefCsr* a, const double* b, double* x, int method, double tol,
                   int max_iter, int* iters, double* res, int* conv) {
    try {
        const auto st = cfd::gpu::solve_host(
            view(*a), b, x, method == 0 ? cfd::gpu::Method::Cg : cfd::gpu::Method::BiCgStab,
            {tol, max_iter});
        put(st, iters, res, conv);
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

// cfd::gpu::solve_amg_cg_host (krylov.hpp:63-64) on an explicit hierarchy.
int ref_solve_amg_cg_host(int n_levels, const RefCsr* a, const RefCsr* p, const RefCsr* r,
                          const double* coarse_inverse, int sweeps, double weight,
                          const double* b, double* x, double tol, int max_iter, int* iters,
                          double* res, int* conv) {
    try {
        cfd::gpu::AmgView h;
        for (int l = 0; l < n_levels; ++l) {
            cfd::gpu::AmgLevelView lv;
            lv.a = view(a[l]);
            if (l + 1 < n_levels) {
                lv.p = view(p[l]);
                lv.r = view(r[l]);
            }
            h.levels.push_back(lv);
        }
        h.coarse_inverse = coarse_inverse;
        h.smooth_sweeps = sweeps;
        h.jacobi_weight = weight;
        put(cfd::gpu::solve_amg_cg_host(h, b, x, {tol, max_iter}), iters, res, conv);
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

// cfd::gpu::DeviceSolver (krylov.hpp:83-103) without a device: host CSR scatter of the LDU
// coefficients, then the host AMG-PCG (use_amg) or Jacobi Krylov method.
int ref_device_solver_solve(int n, int nf, int nnz, const int* row_ptr, const int* col,
                            const int* diag_pos, const int* upper_pos, const int* lower_pos,
                            int n_levels, const RefCsr* a, const RefCsr* p, const RefCsr* r,
                            const double* coarse_inverse, const double* diag,
                            const double* upper, const double* lower, const double* b,
                            double* x, int method, int use_amg, double tol, int max_iter,
                            int* iters, double* res, int* conv) {
    try {
        const cfd::gpu::LduPattern pt{n, nf, nnz, row_ptr, col, diag_pos, upper_pos, lower_pos};
        cfd::gpu::DeviceSolver solver(pt);
        if (n_levels > 0) {
            cfd::gpu::AmgView h;
            for (int l = 0; l < n_levels; ++l) {
                cfd::gpu::AmgLevelView lv;
                lv.a = l == 0 ? cfd::gpu::CsrView{} : view(a[l]);
                if (l + 1 < n_levels) {
                    lv.p = view(p[l]);
                    lv.r = view(r[l]);
                }
                h.levels.push_back(lv);
            }
            h.coarse_inverse = coarse_inverse;
            solver.set_amg(h);
        }
        const auto st = solver.solve(
            diag, upper, lower, b, x,
            method == 0 ? cfd::gpu::Method::Cg : cfd::gpu::Method::BiCgStab, use_amg != 0,
            {tol, max_iter});
        put(st, iters, res, conv);
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

// Persistent cfd::gpu::DeviceSolver, as LduMatrix::solve_persistent keeps it in its AmgCache
// (ldu_matrix.cpp:302-312): created once per pattern, hierarchy installed on (re)build, then
// solve() per pressure solve.
void* ref_ds_create(int n, int nf, int nnz, const int* row_ptr, const int* col, const int* diag_pos,
                    const int* upper_pos, const int* lower_pos) {
    try {
        const cfd::gpu::LduPattern pt{n, nf, nnz, row_ptr, col, diag_pos, upper_pos, lower_pos};
        return new cfd::gpu::DeviceSolver(pt);
    } catch (const std::exception&) {
        return nullptr;
    }
}

int ref_ds_set_amg(void* h, int n_levels, const RefCsr* a, const RefCsr* p, const RefCsr* r,
                   const double* coarse_inverse, int sweeps, double weight) {
    try {
        cfd::gpu::AmgView v;
        for (int l = 0; l < n_levels; ++l) {
            cfd::gpu::AmgLevelView lv;
            lv.a = l == 0 ? cfd::gpu::CsrView{} : view(a[l]);
            if (l + 1 < n_levels) {
                lv.p = view(p[l]);
                lv.r = view(r[l]);
            }
            v.levels.push_back(lv);
        }
        v.coarse_inverse = coarse_inverse;
        v.smooth_sweeps = sweeps;
        v.jacobi_weight = weight;
        static_cast<cfd::gpu::DeviceSolver*>(h)->set_amg(v);
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

int ref_ds_solve(void* h, const double* diag, const double* upper, const double* lower,
                 const double* b, double* x, int method, int use_amg, double tol, int max_iter,
                 int* iters, double* res, int* conv) {
    try {
        const auto st = static_cast<cfd::gpu::DeviceSolver*>(h)->solve(
            diag, upper, lower, b, x,
            method == 0 ? cfd::gpu::Method::Cg : cfd::gpu::Method::BiCgStab, use_amg != 0,
            {tol, max_iter});
        put(st, iters, res, conv);
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

void ref_ds_destroy(void* h) {
    delete static_cast<cfd::gpu::DeviceSolver*>(h);
}

int ref_backend_is_host() {
    return cfd::gpu::backend_name() == "host" ? 1 : 0;
}

// cfd::gpu::DeviceFv (fv_device.hpp:33-72) over an FvMeshView of host arrays. Without an
// accelerator the reference runs the per-cell kernels of fv_cell.inc on host threads.
void* ref_fv_create(int n_cells, int n_internal_faces, int n_faces, const int* owner,
                    const int* neighbour, const int* cell_offsets, const int* cell_faces,
                    const double* weight, const double* sf, const double* face_centre,
                    const double* cell_centre, const double* volume, const double* correction,
                    const double* lsq_d, const double* lsq_inverse) {
    try {
        cfd::gpu::FvMeshView v;
        v.n_cells = n_cells;
        v.n_internal_faces = n_internal_faces;
        v.n_faces = n_faces;
        v.owner = owner;
        v.neighbour = neighbour;
        v.cell_offsets = cell_offsets;
        v.cell_faces = cell_faces;
        v.weight = weight;
        v.sf = sf;
        v.face_centre = face_centre;
        v.cell_centre = cell_centre;
        v.volume = volume;
        v.correction = correction;
        v.lsq_d = lsq_d;
        v.lsq_inverse = lsq_inverse;
        return new cfd::gpu::DeviceFv(v);
    } catch (const std::exception&) {
        return nullptr;
    }
}

void ref_fv_destroy(void* h) {
    delete static_cast<cfd::gpu::DeviceFv*>(h);
}

int ref_fv_gradient(void* h, const double* phi, const double* bv, int scheme, double* grad) {
    try {
        static_cast<cfd::gpu::DeviceFv*>(h)->gradient(phi, bv, scheme, grad);
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

int ref_fv_vector_gradient(void* h, const double* u, const double* ub, int scheme,
                           double* grad) {
    try {
        static_cast<cfd::gpu::DeviceFv*>(h)->vector_gradient(u, ub, scheme, grad);
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

int ref_fv_scalar_corrections(void* h, const double* phi, const double* bv, int scheme,
                              const double* flux, const double* gamma, int linear_upwind,
                              double* source) {
    try {
        static_cast<cfd::gpu::DeviceFv*>(h)->scalar_corrections(phi, bv, scheme, flux, gamma,
                                                               linear_upwind != 0, source);
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

int ref_fv_momentum_corrections(void* h, const double* flux, const double* nu_face,
                                int linear_upwind, int limited, int venkat, const double* eps2,
                                double central, int transpose_term, double* source) {
    try {
        static_cast<cfd::gpu::DeviceFv*>(h)->momentum_corrections(
            flux, nu_face, linear_upwind != 0, limited != 0, venkat != 0, eps2, central,
            transpose_term != 0, source);
        return 0;
    } catch (const std::exception&) {
        return 2;
    }
}

} // extern "C"
