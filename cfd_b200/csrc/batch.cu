// Batches of independent pressure systems in one device plan (declared in include/cfdb.h).
#include "../../include/cfdb.h"

#include <algorithm>
#include <chrono>
#include <climits>
#include <cstring>
#include <memory>
#include <string>

#include "dsetup.hpp"
#include "engine.hpp"
#include "host_algos.hpp"

namespace cfdb {
void set_thread_error(const std::string& msg); // capi.cu
Tuning tuning_from(const cfdb_tuning* t);     // capi.cu
}

using namespace cfdb;

struct cfdb_batch {
    int device = 0;
    int n_sys = 0;
    std::vector<int> nc, nf;
    std::vector<long long> coff, foff; // first cell / face of each system
    long long tc = 0, tf = 0;
    std::vector<LduPatternHost> pats;
    std::vector<std::vector<int>> src, dsrc;
    std::vector<std::shared_ptr<const Hierarchy>> hs;
    std::unique_ptr<Engine> eng;
    int precision = CFDB_PRECISION_FP64;
    Tuning tuning{};
    int sweeps = 2;
    double weight = 0.7;
    bool dirty = true;
    // fused assembly: global owner per face, cell -> face lists (global indices), reference mask
    DeviceArena arena;
    int* d_owner = nullptr;
    int* d_cf_ptr = nullptr;
    int* d_cf_face = nullptr;
    int* d_ref = nullptr;
    std::vector<int> ref_cached;
    unsigned long long launches = 0;
    double setup_hierarchies_s = 0.0; // last setup: the per-system hierarchies
    double setup_plan_s = 0.0;        // last setup: the batch plan built from them
};

namespace {

template <class F> int guarded_b(F&& f) {
    try {
        f();
        return CFDB_OK;
    } catch (const Error& e) {
        set_thread_error(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        set_thread_error("host allocation failed");
        return CFDB_ERR_OOM;
    } catch (const std::exception& e) {
        set_thread_error(e.what());
        return CFDB_ERR_INTERNAL;
    }
}

void ensure_batch_engine(cfdb_batch* b) {
    if (!b->dirty && b->eng) return;
    CFDB_CUDA(cudaSetDevice(b->device));
    if (!b->eng) b->eng = std::make_unique<Engine>(b->device);
    b->eng->set_tuning(b->tuning);
    std::vector<SystemSpec> specs(b->n_sys);
    bool all_h = true;
    for (int s = 0; s < b->n_sys; ++s) all_h = all_h && static_cast<bool>(b->hs[s]);
    for (int s = 0; s < b->n_sys; ++s) {
        SystemSpec& sp = specs[s];
        sp.n = b->nc[s];
        sp.rp = b->pats[s].row_ptr.data();
        sp.ci = b->pats[s].col.data();
        sp.src = b->src[s];
        sp.diag_src = b->dsrc[s];
        sp.vs_len = 0;
        sp.absolute_src = true;
        if (all_h) sp.h = b->hs[s];
    }
    const bool mixed = b->precision == CFDB_PRECISION_MIXED;
    b->eng->build(std::move(specs), b->sweeps, b->weight, !mixed, mixed);
    b->dirty = false;
}

} // namespace

extern "C" {

int cfdb_batch_create(int n_systems, const int* n_cells, const int* n_faces, const int* owner,
                      const int* neighbour, cfdb_batch** out) {
    return guarded_b([&] {
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
            (void)cudaGetLastError();
            fail(CFDB_ERR_NO_DEVICE, "no CUDA device: this library has no host fallback");
        }
        if (out == nullptr || n_systems <= 0 || n_cells == nullptr || n_faces == nullptr)
            fail(CFDB_ERR_BAD_ARG, "cfdb_batch_create: bad arguments");
        auto b = std::make_unique<cfdb_batch>();
        CFDB_CUDA(cudaGetDevice(&b->device));
        b->n_sys = n_systems;
        b->nc.assign(n_cells, n_cells + n_systems);
        b->nf.assign(n_faces, n_faces + n_systems);
        b->coff.resize(n_systems);
        b->foff.resize(n_systems);
        for (int s = 0; s < n_systems; ++s) {
            if (b->nc[s] <= 0 || b->nf[s] < 0) fail(CFDB_ERR_BAD_ARG, "cfdb_batch_create: empty system");
            b->coff[s] = b->tc;
            b->foff[s] = b->tf;
            b->tc += b->nc[s];
            b->tf += b->nf[s];
        }
        if (b->tf > 0 && (owner == nullptr || neighbour == nullptr)) fail(CFDB_ERR_BAD_ARG, "null face addressing");
        if (b->tc + 2 * b->tf >= INT_MAX) fail(CFDB_ERR_BAD_ARG, "batch too large for 32-bit indexing");
        b->pats.resize(n_systems);
        b->src.resize(n_systems);
        b->dsrc.resize(n_systems);
        b->hs.resize(n_systems);
        std::vector<int> errs(n_systems, 0);
#pragma omp parallel for schedule(dynamic, 1)
        for (int s = 0; s < n_systems; ++s) {
            try {
                const int* own = owner + b->foff[s];
                const int* nei = neighbour + b->foff[s];
                b->pats[s] = build_pattern(b->nc[s], b->nf[s], own, nei);
                const LduPatternHost& p = b->pats[s];
                auto& sr = b->src[s];
                sr.assign(static_cast<size_t>(p.nnz()), -1);
                const int c0 = static_cast<int>(b->coff[s]);
                const int u0 = static_cast<int>(b->tc + b->foff[s]);
                const int l0 = static_cast<int>(b->tc + b->tf + b->foff[s]);
                for (int i = 0; i < p.n; ++i) sr[p.diag_pos[i]] = c0 + i;
                for (int f = 0; f < p.n_faces; ++f) {
                    sr[p.upper_pos[f]] = u0 + f;
                    sr[p.lower_pos[f]] = l0 + f;
                }
                b->dsrc[s].resize(p.n);
                for (int i = 0; i < p.n; ++i) b->dsrc[s][i] = c0 + i;
            } catch (...) {
                errs[s] = 1;
            }
        }
        for (int s = 0; s < n_systems; ++s)
            if (errs[s]) fail(CFDB_ERR_BAD_ARG, "cfdb_batch_create: system " + std::to_string(s) + " has invalid addressing");
        // global addressing for the fused assembly
        std::vector<int> gown(static_cast<size_t>(b->tf)), ptr(static_cast<size_t>(b->tc) + 1, 0), face;
        for (int s = 0; s < n_systems; ++s)
            for (int f = 0; f < b->nf[s]; ++f) {
                const long long g = b->foff[s] + f;
                gown[g] = static_cast<int>(b->coff[s]) + owner[g];
                ++ptr[b->coff[s] + owner[g] + 1];
                ++ptr[b->coff[s] + neighbour[g] + 1];
            }
        for (long long c = 0; c < b->tc; ++c) ptr[c + 1] += ptr[c];
        face.resize(static_cast<size_t>(ptr[b->tc]));
        std::vector<int> fill(ptr.begin(), ptr.end() - 1);
        for (int s = 0; s < n_systems; ++s)
            for (int f = 0; f < b->nf[s]; ++f) {
                const long long g = b->foff[s] + f;
                face[fill[b->coff[s] + owner[g]]++] = static_cast<int>(g);
                face[fill[b->coff[s] + neighbour[g]]++] = static_cast<int>(g);
            }
        CFDB_CUDA(cudaSetDevice(b->device));
        b->d_owner = b->arena.upload(gown, nullptr);
        b->d_cf_ptr = b->arena.upload(ptr, nullptr);
        b->d_cf_face = b->arena.upload(face, nullptr);
        b->d_ref = b->arena.alloc<int>(static_cast<size_t>(b->tc));
        CFDB_CUDA(cudaMemset(b->d_ref, 0, sizeof(int) * static_cast<size_t>(b->tc)));
        CFDB_CUDA(cudaDeviceSynchronize());
        ensure_batch_engine(b.get());
        *out = b.release();
    });
}

int cfdb_batch_destroy(cfdb_batch* b) {
    if (b != nullptr) {
        cudaSetDevice(b->device);
        // device buffers go back to the pool at once: let the work that uses them finish
        if (b->eng) cudaStreamSynchronize(b->eng->stream());
        delete b;
    }
    return CFDB_OK;
}

int cfdb_batch_sizes(const cfdb_batch* b, long long* total_cells, long long* total_faces) {
    if (b == nullptr) return CFDB_ERR_BAD_ARG;
    if (total_cells) *total_cells = b->tc;
    if (total_faces) *total_faces = b->tf;
    return CFDB_OK;
}

int cfdb_batch_setup_amg(cfdb_batch* b, const double* diag, const double* upper, const double* lower,
                         const cfdb_amg_settings* settings) {
    return guarded_b([&] {
        if (b == nullptr || diag == nullptr || (b->tf > 0 && (upper == nullptr || lower == nullptr)))
            fail(CFDB_ERR_BAD_ARG, "cfdb_batch_setup_amg: null argument");
        AmgSettings st;
        if (settings != nullptr) {
            st.theta = settings->strength_threshold;
            st.max_levels = settings->max_levels;
            st.coarse_size = settings->coarse_size;
            st.sweeps = settings->smooth_sweeps;
            st.weight = settings->jacobi_weight;
        }
        std::vector<std::string> errs(b->n_sys);
        const auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic, 1)
        for (int s = 0; s < b->n_sys; ++s) {
            try {
                const LduPatternHost& p = b->pats[s];
                HostCsr a;
                a.n_rows = a.n_cols = p.n;
                a.rp = p.row_ptr;
                a.ci = p.col;
                a.va.assign(static_cast<size_t>(p.nnz()), 0.0);
                for (int i = 0; i < p.n; ++i) a.va[p.diag_pos[i]] = diag[b->coff[s] + i];
                for (int f = 0; f < p.n_faces; ++f) {
                    a.va[p.upper_pos[f]] = upper[b->foff[s] + f];
                    a.va[p.lower_pos[f]] = lower[b->foff[s] + f];
                }
                b->hs[s] = std::make_shared<Hierarchy>(amg_setup(a, st));
            } catch (const std::exception& e) {
                errs[s] = e.what();
            }
        }
        for (int s = 0; s < b->n_sys; ++s)
            if (!errs[s].empty()) fail(CFDB_ERR_BAD_ARG, "system " + std::to_string(s) + ": " + errs[s]);
        b->sweeps = st.sweeps;
        b->weight = st.weight;
        b->dirty = true;
        const auto t1 = std::chrono::steady_clock::now();
        ensure_batch_engine(b);
        b->setup_hierarchies_s = std::chrono::duration<double>(t1 - t0).count();
        b->setup_plan_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
    });
}

// The hierarchies of every system built on the device (amg_setup_device per system: strength
// graph, smoothed prolongation, transpose and Galerkin products in CUDA kernels, aggregation on
// the host), several systems at a time on their own streams and host threads, then copied into
// the plan as the host build's are. Bit-identical to cfdb_batch_setup_amg. diag / upper / lower
// are device arrays, concatenated in system order.
int cfdb_batch_setup_amg_device(cfdb_batch* b, const double* diag, const double* upper, const double* lower,
                                const cfdb_amg_settings* settings, int concurrency) {
    return guarded_b([&] {
        if (b == nullptr || diag == nullptr || (b->tf > 0 && (upper == nullptr || lower == nullptr)))
            fail(CFDB_ERR_BAD_ARG, "cfdb_batch_setup_amg_device: null argument");
        CFDB_CUDA(cudaSetDevice(b->device));
        AmgSettings st;
        if (settings != nullptr) {
            st.theta = settings->strength_threshold;
            st.max_levels = settings->max_levels;
            st.coarse_size = settings->coarse_size;
            st.sweeps = settings->smooth_sweeps;
            st.weight = settings->jacobi_weight;
            st.table_limit = settings->device_table_limit;
        }
        if (st.max_levels < 1) fail(CFDB_ERR_BAD_ARG, "max_levels must be >= 1");
        const int workers = std::max(1, std::min(concurrency > 0 ? concurrency : 8, b->n_sys));
        std::vector<std::string> errs(b->n_sys);
        const auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic, 1) num_threads(workers)
        for (int s = 0; s < b->n_sys; ++s) {
            cudaStream_t cs = nullptr;
            try {
                CFDB_CUDA(cudaSetDevice(b->device));
                CFDB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
                const LduPatternHost& p = b->pats[s];
                DeviceHierarchy dh;
                DevCsr a0;
                a0.n_rows = a0.n_cols = p.n;
                a0.nnz = p.nnz();
                a0.rp = dh.mem.alloc<int>(p.row_ptr.size());
                a0.ci = dh.mem.alloc<int>(std::max<size_t>(p.col.size(), 1));
                a0.va = dh.mem.alloc<double>(std::max<size_t>(p.col.size(), 1));
                int* pos = dh.mem.alloc<int>(static_cast<size_t>(p.n + 2 * p.n_faces) + 1);
                CFDB_CUDA(cudaMemcpyAsync(a0.rp, p.row_ptr.data(), sizeof(int) * p.row_ptr.size(), cudaMemcpyHostToDevice, cs));
                if (a0.nnz > 0)
                    CFDB_CUDA(cudaMemcpyAsync(a0.ci, p.col.data(), sizeof(int) * p.col.size(), cudaMemcpyHostToDevice, cs));
                CFDB_CUDA(cudaMemcpyAsync(pos, p.diag_pos.data(), sizeof(int) * p.n, cudaMemcpyHostToDevice, cs));
                if (p.n_faces > 0) {
                    CFDB_CUDA(cudaMemcpyAsync(pos + p.n, p.upper_pos.data(), sizeof(int) * p.n_faces, cudaMemcpyHostToDevice, cs));
                    CFDB_CUDA(cudaMemcpyAsync(pos + p.n + p.n_faces, p.lower_pos.data(), sizeof(int) * p.n_faces,
                                              cudaMemcpyHostToDevice, cs));
                }
                ldu_to_csr_values(p.n, p.n_faces, pos, pos + p.n, pos + p.n + p.n_faces, diag + b->coff[s],
                                  p.n_faces > 0 ? upper + b->foff[s] : nullptr, p.n_faces > 0 ? lower + b->foff[s] : nullptr,
                                  a0.va, cs);
                amg_setup_device(a0, st, cs, dh);
                b->hs[s] = std::make_shared<Hierarchy>(download_hierarchy(dh, /*with_a0=*/true, cs));
                CFDB_CUDA(cudaStreamSynchronize(cs));
            } catch (const std::exception& e) {
                errs[s] = e.what();
            }
            if (cs != nullptr) cudaStreamDestroy(cs);
        }
        for (int s = 0; s < b->n_sys; ++s)
            if (!errs[s].empty()) fail(CFDB_ERR_BAD_ARG, "system " + std::to_string(s) + ": " + errs[s]);
        b->sweeps = st.sweeps;
        b->weight = st.weight;
        b->dirty = true;
        const auto t1 = std::chrono::steady_clock::now();
        ensure_batch_engine(b);
        b->setup_hierarchies_s = std::chrono::duration<double>(t1 - t0).count();
        b->setup_plan_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
    });
}

int cfdb_batch_set_precision(cfdb_batch* b, int precision) {
    return guarded_b([&] {
        if (b == nullptr) fail(CFDB_ERR_BAD_ARG, "null batch");
        if (precision != CFDB_PRECISION_FP64 && precision != CFDB_PRECISION_MIXED)
            fail(CFDB_ERR_BAD_ARG, "unknown precision");
        if (b->precision != precision) {
            b->precision = precision;
            b->dirty = true;
            ensure_batch_engine(b);
        }
    });
}

int cfdb_batch_set_tuning(cfdb_batch* b, const cfdb_tuning* t) {
    return guarded_b([&] {
        if (b == nullptr || t == nullptr) fail(CFDB_ERR_BAD_ARG, "null argument");
        b->tuning = tuning_from(t);
        b->dirty = true;
        ensure_batch_engine(b);
    });
}

int cfdb_batch_assemble_pressure_device(cfdb_batch* b, const double* flux, const double* gamma, const double* delta,
                                        const double* source0, const int* ref_cell, double ref_value, double* upper,
                                        double* lower, double* diag, double* source) {
    return guarded_b([&] {
        if (b == nullptr || !flux || !gamma || !delta || !source0 || !upper || !lower || !diag || !source)
            fail(CFDB_ERR_BAD_ARG, "cfdb_batch_assemble_pressure_device: null argument");
        CFDB_CUDA(cudaSetDevice(b->device));
        ensure_batch_engine(b);
        cudaStream_t st = b->eng->stream();
        std::vector<int> refs(b->n_sys, -1);
        if (ref_cell != nullptr) refs.assign(ref_cell, ref_cell + b->n_sys);
        if (refs != b->ref_cached) {
            std::vector<int> mask(static_cast<size_t>(b->tc), 0);
            for (int s = 0; s < b->n_sys; ++s) {
                if (refs[s] >= b->nc[s]) fail(CFDB_ERR_BAD_ARG, "reference cell out of range");
                if (refs[s] >= 0) mask[b->coff[s] + refs[s]] = 1;
            }
            CFDB_CUDA(cudaMemcpyAsync(b->d_ref, mask.data(), sizeof(int) * mask.size(), cudaMemcpyHostToDevice, st));
            CFDB_CUDA(cudaStreamSynchronize(st));
            b->ref_cached = refs;
        }
        const long long tf = b->tf, tc = b->tc;
        if (tf > 0) {
            k_assemble_faces<<<static_cast<int>((tf + 255) / 256), 256, 0, st>>>(static_cast<int>(tf), flux, gamma,
                                                                                 delta, 0.0, upper, lower);
            ++b->launches;
        }
        k_assemble_pressure_cells<<<static_cast<int>((tc + 255) / 256), 256, 0, st>>>(
            static_cast<int>(tc), b->d_cf_ptr, b->d_cf_face, flux, gamma, delta, b->d_owner, nullptr, source0, -1,
            b->d_ref, ref_value, diag, source);
        ++b->launches;
        CFDB_CUDA(cudaGetLastError());
    });
}

int cfdb_batch_solve_device(cfdb_batch* b, const double* diag, const double* upper, const double* lower,
                            const double* rhs, double* x, int use_amg, const cfdb_control* controls,
                            cfdb_stats* stats) {
    return guarded_b([&] {
        if (b == nullptr || !diag || !rhs || !x || !controls || (b->tf > 0 && (!upper || !lower)))
            fail(CFDB_ERR_BAD_ARG, "cfdb_batch_solve_device: null argument");
        CFDB_CUDA(cudaSetDevice(b->device));
        ensure_batch_engine(b);
        Engine& e = *b->eng;
        Mode mode = Mode::Jacobi;
        if (use_amg) {
            if (!e.has_amg()) fail(CFDB_ERR_NOT_READY, "cfdb_batch_solve_device: no hierarchy set (cfdb_batch_setup_amg)");
            mode = b->precision == CFDB_PRECISION_MIXED ? Mode::AmgMixed : Mode::AmgFp64;
        }
        e.set_values_device(diag, upper, lower, static_cast<int>(b->tc), static_cast<int>(b->tc + b->tf));
        e.set_rhs_guess_concat(rhs, x);
        std::vector<SolveRequest> req(b->n_sys);
        for (int s = 0; s < b->n_sys; ++s) req[s] = SolveRequest{controls[s].abs_tolerance, controls[s].max_iterations};
        const auto res = e.solve(mode, req);
        e.get_solution_concat(x);
        if (stats != nullptr) {
            for (int s = 0; s < b->n_sys; ++s)
                stats[s] = cfdb_stats{res[s].iterations, res[s].residual, res[s].converged ? 1 : 0, 1,
                                      res[s].true_residual};
        }
    });
}

int cfdb_batch_profile(cfdb_batch* b, int reps, cfdb_kernel_record* records, int max_records, int* n_records) {
    return guarded_b([&] {
        if (b == nullptr || records == nullptr || n_records == nullptr) fail(CFDB_ERR_BAD_ARG, "null argument");
        CFDB_CUDA(cudaSetDevice(b->device));
        ensure_batch_engine(b);
        const Mode mode = !b->eng->has_amg() ? Mode::Jacobi
                          : b->precision == CFDB_PRECISION_MIXED ? Mode::AmgMixed
                                                                 : Mode::AmgFp64;
        const auto recs = b->eng->profile(mode, reps);
        const int n = std::min<int>(static_cast<int>(recs.size()), max_records);
        for (int i = 0; i < n; ++i) {
            std::memcpy(records[i].name, recs[i].name, sizeof(records[i].name));
            records[i].level = recs[i].level;
            records[i].ms = recs[i].ms;
            records[i].bytes = recs[i].bytes;
        }
        *n_records = n;
    });
}

int cfdb_batch_stream(const cfdb_batch* b, void** stream) {
    if (b == nullptr || stream == nullptr || !b->eng) return CFDB_ERR_BAD_ARG;
    *stream = b->eng->stream();
    return CFDB_OK;
}

int cfdb_batch_setup_profile(const cfdb_batch* b, char* buf, size_t len) {
    if (b == nullptr || buf == nullptr || len == 0) return CFDB_ERR_BAD_ARG;
    const std::string t = b->eng ? b->eng->build_times().text() : std::string();
    const size_t n = std::min(len - 1, t.size());
    std::memcpy(buf, t.data(), n);
    buf[n] = '\0';
    return CFDB_OK;
}

int cfdb_batch_setup_times(const cfdb_batch* b, double* hierarchies_s, double* plan_s) {
    if (b == nullptr) return CFDB_ERR_BAD_ARG;
    if (hierarchies_s != nullptr) *hierarchies_s = b->setup_hierarchies_s;
    if (plan_s != nullptr) *plan_s = b->setup_plan_s;
    return CFDB_OK;
}

int cfdb_batch_device_bytes(const cfdb_batch* b, size_t* bytes) {
    if (b == nullptr || bytes == nullptr) return CFDB_ERR_BAD_ARG;
    *bytes = (b->eng ? b->eng->device_bytes() : 0) + b->arena.bytes();
    return CFDB_OK;
}

int cfdb_batch_kernel_launches(const cfdb_batch* b, unsigned long long* count) {
    if (b == nullptr || count == nullptr) return CFDB_ERR_BAD_ARG;
    *count = b->launches + (b->eng ? b->eng->kernel_launches() : 0);
    return CFDB_OK;
}

} // extern "C"
