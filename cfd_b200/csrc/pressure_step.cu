// FlowSolver::pressure_correction (flow_solver.cpp:673-847) as one C-ABI call, composed in C++
// from the library's device entry points in the reference's order, every array in device
// memory: HbyA and rAU from the momentum system (flow_solver.cpp:688-708), the predicted face
// flux and face rAU with the relaxation-independent term (:710-755), the pressure equation
// with its boundary terms and reference cell (:757-796), the non-orthogonal correctors around
// the persistent LDU solve with its AmgCache (:798-822), the conservative flux, pressure
// relaxation and velocity correction (:824-846). Each step is the device kernel that is
// bit-identical to the reference's face or cell loop; the solve is cfdb_system_solve_ldu.
#include "../../include/cfdb.h"

#include <string>

#include "common.hpp"

namespace cfdb {
void set_thread_error(const std::string& msg); // capi.cu
}

namespace {

void ok(int rc, const char* what) {
    if (rc != CFDB_OK) {
        char msg[512];
        cfdb_last_error(msg, sizeof msg);
        cfdb::fail(rc, std::string(what) + ": " + msg);
    }
}

struct Stream {
    cudaStream_t s = nullptr;
    Stream() { CFDB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
    ~Stream() {
        if (s != nullptr) cudaStreamDestroy(s);
    }
};

} // namespace

extern "C" int cfdb_pressure_correction_device(cfdb_system* sys, cfdb_fv* fv, const double* mom_diag,
                                               const double* mom_upper, const double* mom_lower,
                                               const double* mom_source, double* u, double* p,
                                               const double* fixed_velocity, const double* u_prev,
                                               const double* phi_prev, const cfdb_pressure_settings* s,
                                               const cfdb_pressure_workspace* w, cfdb_ldu_result* results,
                                               double* initial_residual) {
    try {
        if (sys == nullptr || fv == nullptr || s == nullptr || w == nullptr || u == nullptr || p == nullptr)
            cfdb::fail(CFDB_ERR_BAD_ARG, "cfdb_pressure_correction_device: null argument");
        int n = 0, nf = 0, ni = 0;
        ok(cfdb_fv_sizes(fv, &n, &nf, &ni), "fv sizes");
        int sys_n = 0, sys_nf = 0;
        ok(cfdb_system_sizes(sys, &sys_n, &sys_nf), "system sizes");
        if (sys_n != n || sys_nf != ni)
            cfdb::fail(CFDB_ERR_BAD_ARG, "cfdb_pressure_correction_device: the system and the geometry differ in size");
        if (s->n_non_orth_correctors < 0) cfdb::fail(CFDB_ERR_BAD_ARG, "negative non-orthogonal correctors");
        if (!w->hbya || !w->rau || !w->phi_hbya || !w->rau_f || !w->diag || !w->source || !w->base_source ||
            !w->p_prev || !w->p_new || !w->non_orth || !w->grad || !w->phi || (ni > 0 && (!w->upper || !w->lower)))
            cfdb::fail(CFDB_ERR_BAD_ARG, "cfdb_pressure_correction_device: workspace array missing");
        const size_t bn = sizeof(double) * static_cast<size_t>(n);
        Stream st;
        auto fill0 = [&](double* a, size_t count) {
            if (count > 0) CFDB_CUDA(cudaMemsetAsync(a, 0, sizeof(double) * count, st.s));
        };
        auto copy = [&](double* dst, const double* src) { CFDB_CUDA(cudaMemcpyAsync(dst, src, bn, cudaMemcpyDeviceToDevice, st.s)); };
        auto done = [&]() { CFDB_CUDA(cudaStreamSynchronize(st.s)); };

        // HbyA, rAU; predicted face flux and face rAU (relaxation-independent term when the
        // previous velocity and flux are given and alpha_u < 1)
        ok(cfdb_fv_hbya_rau_device(fv, mom_diag, mom_upper, mom_lower, mom_source, u, w->hbya, w->rau), "HbyA");
        const bool majumdar = u_prev != nullptr && phi_prev != nullptr && s->alpha_u < 1.0;
        ok(cfdb_fv_face_flux_device(fv, w->hbya, w->rau, fixed_velocity, majumdar ? u_prev : nullptr,
                                    majumdar ? phi_prev : nullptr, majumdar ? 1.0 - s->alpha_u : 0.0, w->phi_hbya,
                                    w->rau_f),
           "face flux");
        // pressure equation: internal faces (zero source0: base_source serves as it), then the
        // boundary faces and the reference cell
        fill0(w->upper, static_cast<size_t>(ni));
        fill0(w->lower, static_cast<size_t>(ni));
        fill0(w->diag, static_cast<size_t>(n));
        fill0(w->source, static_cast<size_t>(n));
        fill0(w->base_source, static_cast<size_t>(n));
        done();
        const double* delta = nullptr;
        ok(cfdb_fv_delta_device(fv, &delta), "delta");
        ok(cfdb_system_assemble_pressure_device(sys, w->phi_hbya, w->rau_f, delta, nullptr, w->base_source, -1, 0.0,
                                                w->upper, w->lower, w->diag, w->source),
           "pressure assembly");
        // the assembly is enqueued on the system's stream and returns at once: it must be done
        // before the geometry's stream adds the boundary terms to the same diag and source
        void* sys_stream = nullptr;
        ok(cfdb_system_stream(sys, &sys_stream), "system stream");
        CFDB_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(sys_stream)));
        ok(cfdb_fv_pressure_boundary_device(fv, w->phi_hbya, w->rau_f, s->ref_cell, s->ref_value, w->diag, w->source),
           "pressure boundary");
        copy(w->base_source, w->source);
        copy(w->p_prev, p);
        copy(w->p_new, p);
        fill0(w->non_orth, static_cast<size_t>(ni > 0 ? ni : 1));
        fill0(w->grad, 3 * static_cast<size_t>(n));
        done();
        // non-orthogonal correctors around the persistent solve
        const int n_solves = s->n_non_orth_correctors + 1;
        for (int corr = 0; corr < n_solves; ++corr) {
            fill0(w->non_orth, static_cast<size_t>(ni > 0 ? ni : 1));
            copy(w->source, w->base_source);
            done();
            if (corr > 0 || s->n_non_orth_correctors > 0) {
                ok(cfdb_fv_pressure_gradient_device(fv, w->p_new, w->grad), "pressure gradient");
                ok(cfdb_fv_non_orth_device(fv, w->grad, w->rau_f, w->base_source, w->non_orth, w->source),
                   "non-orthogonal source");
            }
            cfdb_ldu_result r{};
            ok(cfdb_system_solve_ldu(sys, w->diag, w->upper, w->lower, w->source, w->p_new, &s->p_solver, &s->amg,
                                     1, &r),
               "pressure solve");
            if (corr == 0 && initial_residual != nullptr) *initial_residual = r.initial_residual;
            if (results != nullptr) results[corr] = r;
            if (w->solve_p != nullptr) copy(w->solve_p + static_cast<size_t>(corr) * n, w->p_new);
            if (w->solve_source != nullptr) copy(w->solve_source + static_cast<size_t>(corr) * n, w->source);
            done();
        }
        // conservative flux, relaxed pressure, velocity correction
        ok(cfdb_fv_correct_flux_device(fv, w->phi_hbya, w->rau_f, w->non_orth, w->p_new, w->phi), "flux correction");
        if (s->relax_p) {
            ok(cfdb_fv_relax_device(fv, w->p_prev, w->p_new, s->alpha_p, p), "pressure relaxation");
        } else {
            copy(p, w->p_new);
            done();
        }
        ok(cfdb_fv_pressure_gradient_device(fv, p, w->grad), "pressure gradient");
        ok(cfdb_fv_correct_velocity_device(fv, w->hbya, w->rau, w->grad, u), "velocity correction");
        return CFDB_OK;
    } catch (const cfdb::Error& e) {
        cfdb::set_thread_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        cfdb::set_thread_error(e.what());
        return CFDB_ERR_INTERNAL;
    }
}
