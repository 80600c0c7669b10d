// C ABI of the cfdb library (declared in include/cfdb.h).
#include "../../include/cfdb.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <climits>
#include <cstring>
#include <memory>
#include <new>
#include <string>

#include "dsetup.hpp"
#include "engine.hpp"
#include "ldu_solve.hpp"
#include "host_algos.hpp"

using namespace cfdb;

namespace {

thread_local std::string g_last_error;

int set_error(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

template <class F> int guarded(F&& f) {
    try {
        f();
        return CFDB_OK;
    } catch (const Error& e) {
        return set_error(e.code, e.what());
    } catch (const std::bad_alloc&) {
        return set_error(CFDB_ERR_OOM, "host allocation failed");
    } catch (const std::exception& e) {
        return set_error(CFDB_ERR_INTERNAL, e.what());
    }
}

int copy_str(const std::string& s, char* buf, size_t len) {
    if (buf == nullptr || len == 0) return set_error(CFDB_ERR_BAD_ARG, "null buffer");
    const size_t n = std::min(len - 1, s.size());
    std::memcpy(buf, s.data(), n);
    buf[n] = '\0';
    return CFDB_OK;
}

void require_device() {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        (void)cudaGetLastError();
        fail(CFDB_ERR_NO_DEVICE, "no CUDA device: this library has no host fallback");
    }
}

HostCsr csr_from(const cfdb_csr& v, int n_cols) {
    HostCsr m;
    m.n_rows = v.n;
    m.n_cols = n_cols;
    if (v.n < 0 || v.nnz < 0) fail(CFDB_ERR_BAD_ARG, "negative CSR size");
    if (v.n > 0 && (v.row_ptr == nullptr || (v.nnz > 0 && (v.col == nullptr || v.val == nullptr)))) {
        fail(CFDB_ERR_BAD_ARG, "CSR view with null arrays");
    }
    m.rp.assign(v.row_ptr, v.row_ptr + v.n + 1);
    if (m.rp[0] != 0 || m.rp[v.n] != v.nnz) fail(CFDB_ERR_BAD_ARG, "CSR row_ptr inconsistent with nnz");
    for (int i = 0; i < v.n; ++i)
        if (m.rp[i + 1] < m.rp[i]) fail(CFDB_ERR_BAD_ARG, "CSR row_ptr not monotone");
    m.ci.assign(v.col, v.col + v.nnz);
    m.va.assign(v.val, v.val + v.nnz);
    for (int c : m.ci)
        if (c < 0 || c >= n_cols) fail(CFDB_ERR_BAD_ARG, "CSR column index out of range");
    return m;
}

// Copies an AmgView into a host hierarchy; level 0's operator is optional (skip_a0).
std::shared_ptr<Hierarchy> hierarchy_from(const cfdb_amg_view& v, int n0, bool skip_a0) {
    if (v.n_levels <= 0 || v.levels == nullptr) fail(CFDB_ERR_BAD_ARG, "empty hierarchy");
    auto h = std::make_shared<Hierarchy>();
    const int L = v.n_levels;
    std::vector<int> n(L);
    n[0] = n0;
    for (int l = 1; l < L; ++l) n[l] = v.levels[l].a.n;
    for (int l = 0; l < L; ++l) {
        if (l == 0 && skip_a0) {
            h->a.emplace_back();
            h->a.back().n_rows = h->a.back().n_cols = n0;
        } else {
            h->a.push_back(csr_from(v.levels[l].a, n[l]));
        }
        if (l + 1 < L) {
            h->p.push_back(csr_from(v.levels[l].p, n[l + 1]));
            h->r.push_back(csr_from(v.levels[l].r, n[l]));
        }
    }
    h->n_c = n[L - 1];
    if (v.coarse_inverse == nullptr) fail(CFDB_ERR_BAD_ARG, "hierarchy without coarse inverse");
    h->coarse_inverse.assign(v.coarse_inverse, v.coarse_inverse + static_cast<size_t>(h->n_c) * h->n_c);
    h->ldlt_ok = true;
    return h;
}

AmgSettings settings_from(const cfdb_amg_settings* settings) {
    AmgSettings s;
    if (settings != nullptr) {
        s.theta = settings->strength_threshold;
        s.max_levels = settings->max_levels;
        s.coarse_size = settings->coarse_size;
        s.sweeps = settings->smooth_sweeps;
        s.weight = settings->jacobi_weight;
        s.table_limit = settings->device_table_limit;
    }
    if (s.max_levels < 1) fail(CFDB_ERR_BAD_ARG, "max_levels must be >= 1");
    if (s.table_limit < 0) fail(CFDB_ERR_BAD_ARG, "device_table_limit must be >= 0");
    return s;
}

// A non-blocking stream for the duration of one call.
struct CallStream {
    cudaStream_t s = nullptr;
    CallStream() { CFDB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
    ~CallStream() {
        if (s != nullptr) cudaStreamDestroy(s);
    }
    CallStream(const CallStream&) = delete;
    CallStream& operator=(const CallStream&) = delete;
};

// A second stream with one event per slice, kept for an object's life: the read-backs of a
// pipelined host-array call run on it while the next slice's uploads and kernels run on the
// engine's stream.
struct SliceStream {
    cudaStream_t s = nullptr;
    std::vector<cudaEvent_t> ev;
    void ensure(size_t n_events) {
        if (s == nullptr) CFDB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        while (ev.size() < n_events) {
            cudaEvent_t e = nullptr;
            CFDB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            ev.push_back(e);
        }
    }
    SliceStream() = default;
    ~SliceStream() {
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
        if (s != nullptr) cudaStreamDestroy(s);
    }
    SliceStream(const SliceStream&) = delete;
    SliceStream& operator=(const SliceStream&) = delete;
};

} // namespace

namespace cfdb {
// Records the calling thread's last error message (used by entry points in other files).
void set_thread_error(const std::string& msg) { g_last_error = msg; }

// Validated engine tuning from the C struct (shared with the batch API).
Tuning tuning_from(const cfdb_tuning* t) {
    if (t == nullptr) fail(CFDB_ERR_BAD_ARG, "null tuning");
    if (t->target_tiles < 0 || t->wide_row < 0 || t->lanes_div < 1)
        fail(CFDB_ERR_BAD_ARG, "tuning values out of range");
    if (t->sell_rows < kSellRows || t->sell_rows % kSellRows != 0 || t->sell_rows > 16 * kSellRows)
        fail(CFDB_ERR_BAD_ARG, "tuning: sell_rows must be a multiple of 256 in 256..4096");
    return Tuning{t->target_tiles, t->wide_row, t->lanes_div, t->fuse_first != 0 ? 1 : 0, t->sell_rows,
                  t->krylov_pair != 0 ? 1 : 0, t->col16 != 0 ? 1 : 0, std::max(t->tail_rows, 0), t->pdl != 0 ? 1 : 0,
                  t->wait_polls == 0 ? Tuning{}.wait_polls : t->wait_polls, std::max(t->mixed_sweeps, 0),
                  t->mixed_weight > 0.0 ? t->mixed_weight : 0.0,
                  t->tail_cluster > 0 ? std::min(std::max(t->tail_cluster, 2), 16) : 0, t->vcycle_pair != 0 ? 1 : 0,
                  t->krylov_stage > 0 ? std::min(std::max(t->krylov_stage, 2), 4) : 0};
}

} // namespace cfdb

// ------------------------------------------------------------------------------------------------
// system object
// ------------------------------------------------------------------------------------------------

namespace {
long long next_layout_id() {
    static std::atomic<long long> next{1};
    return next++;
}
} // namespace

struct cfdb_system {
    int device = 0;
    LduPatternHost pat;
    std::vector<int> owner, neighbour; // kept when created from mesh addressing
    long long layout_id = next_layout_id(); // the pattern and value maps never change
    std::unique_ptr<Engine> eng;
    std::shared_ptr<const Hierarchy> h;
    std::shared_ptr<const DeviceLevels> dl; // device-resident levels of a device setup
    bool h_shapes_only = false;             // h came from a device setup (matrices on the device)
    bool keep_levels = true;                // keep dl after a device setup (plan rebuilds)
    int sweeps = 2;
    double weight = 0.7;
    int precision = CFDB_PRECISION_FP64;
    bool dirty = true;
    // value map of the level-0 CSR entries into [diag | upper | lower]
    std::vector<int> src;
    std::vector<int> diag_src;
    // device copies for the fused face assembly
    DeviceArena asm_arena;
    int* d_owner = nullptr;
    int* d_neighbour = nullptr; // uploaded on first use (flux correction)
    int* d_cf_ptr = nullptr;
    int* d_cf_face = nullptr;
    double* h_asm = nullptr; // device staging of cfdb_system_assemble (host-array variant)
    // slices of cfdb_system_assemble: cells [asm_cells[j], asm_cells[j+1]) need the faces
    // [0, asm_faces[j+1]), so slice j's read-back overlaps slice j+1's upload
    std::vector<int> asm_cells, asm_faces;
    SliceStream asm_d2h;
    unsigned long long launches = 0;
    // device copy of the pattern for the device AMG setup (uploaded on first use)
    DeviceArena pat_arena;
    int* d_rp = nullptr;
    int* d_ci = nullptr;
    int* d_dpos = nullptr;
    int* d_upos = nullptr;
    int* d_lpos = nullptr;
    std::string setup_profile; // phase times of the last hierarchy setup
    PinnedBuffer stage;        // page-locked staging of the device setup's read-backs
    // persistent LDU solve (cfdb_system_solve_ldu): AmgCache state and device staging
    int age = 0;               // CG solves since the last hierarchy setup
    bool amg_built = false;    // a setup has run (its hierarchy may have one level)
    int* d_src = nullptr;      // value map of the pattern entries (pat_arena)
    DeviceArena ldu_arena;
    double* ldu_stage = nullptr; // diag | upper | lower | source | x (host-array calls)
    double* norm_part = nullptr;
};

namespace {

void build_value_map(cfdb_system* s) {
    const LduPatternHost& p = s->pat;
    s->src.assign(static_cast<size_t>(p.nnz()), -1);
    for (int i = 0; i < p.n; ++i) s->src[p.diag_pos[i]] = i;
    for (int f = 0; f < p.n_faces; ++f) {
        s->src[p.upper_pos[f]] = p.n + f;
        s->src[p.lower_pos[f]] = p.n + p.n_faces + f;
    }
    s->diag_src.resize(static_cast<size_t>(p.n));
    for (int i = 0; i < p.n; ++i) s->diag_src[i] = i;
}

// Cell slices of the host-array assembly and, per slice, the face prefix its cells need: the
// largest face index of any cell up to the slice's end, plus one. With faces ordered by owner
// (owner < neighbour) the prefixes grow evenly; any other order stays correct, with fewer
// copies overlapped.
void plan_assembly_slices(cfdb_system* s) {
    constexpr int kSliceCells = 1 << 18;
    constexpr int kMaxSlices = 8;
    const int n = s->pat.n, nf = s->pat.n_faces;
    const int k = std::max(1, std::min(kMaxSlices, n / kSliceCells));
    std::vector<int> last(static_cast<size_t>(n), -1); // largest face index of each cell
    for (int f = 0; f < nf; ++f) {
        last[s->owner[f]] = std::max(last[s->owner[f]], f);
        last[s->neighbour[f]] = std::max(last[s->neighbour[f]], f);
    }
    s->asm_cells.assign(1, 0);
    s->asm_faces.assign(1, 0);
    int upto = -1, c = 0;
    for (int j = 0; j < k; ++j) {
        const int c1 = j + 1 == k ? n : static_cast<int>(static_cast<long long>(n) * (j + 1) / k);
        for (; c < c1; ++c) upto = std::max(upto, last[c]);
        s->asm_cells.push_back(c1);
        s->asm_faces.push_back(j + 1 == k ? nf : upto + 1);
    }
}

void ensure_engine(cfdb_system* s) {
    if (!s->dirty && s->eng) return;
    if (s->h && s->h_shapes_only && !s->dl)
        fail(CFDB_ERR_NOT_READY, "the hierarchy was built on the device without keeping its levels "
                                 "(cfdb_system_set_keep_levels): set it up again before changing the plan");
    CFDB_CUDA(cudaSetDevice(s->device));
    if (!s->eng) s->eng = std::make_unique<Engine>(s->device);
    SystemSpec sp;
    sp.n = s->pat.n;
    sp.rp = s->pat.row_ptr.data();
    sp.ci = s->pat.col.data();
    sp.src_ref = &s->src;
    sp.diag_src_ref = &s->diag_src;
    sp.layout_id = s->layout_id;
    sp.vs_len = s->pat.n + 2 * s->pat.n_faces;
    sp.h = s->h;
    sp.dl = s->h ? s->dl : nullptr;
    const bool mixed = s->precision == CFDB_PRECISION_MIXED;
    std::vector<SystemSpec> v;
    v.push_back(std::move(sp));
    s->eng->build(std::move(v), s->sweeps, s->weight, /*need64=*/!mixed, /*need32=*/mixed);
    s->dirty = false;
}

// Device copy of the system's pattern (uploaded once).
void pattern_on_device(cfdb_system* sys, cudaStream_t st) {
    if (sys->d_rp != nullptr) return;
    const LduPatternHost& p = sys->pat;
    sys->d_rp = sys->pat_arena.upload(p.row_ptr, st);
    sys->d_ci = sys->pat_arena.upload(p.col, st);
    sys->d_dpos = sys->pat_arena.upload(p.diag_pos, st);
    sys->d_upos = sys->pat_arena.upload(p.upper_pos, st);
    sys->d_lpos = sys->pat_arena.upload(p.lower_pos, st);
    sys->d_src = sys->pat_arena.upload(sys->src, st);
    CFDB_CUDA(cudaStreamSynchronize(st));
}

void validate_pattern(const cfdb_ldu_pattern& p) {
    if (p.n <= 0 || p.n_faces < 0 || p.nnz < p.n) fail(CFDB_ERR_BAD_ARG, "invalid pattern sizes");
    if (p.row_ptr == nullptr || p.col == nullptr || p.diag_pos == nullptr ||
        (p.n_faces > 0 && (p.upper_pos == nullptr || p.lower_pos == nullptr))) {
        fail(CFDB_ERR_BAD_ARG, "pattern with null arrays");
    }
    if (p.row_ptr[0] != 0 || p.row_ptr[p.n] != p.nnz) fail(CFDB_ERR_BAD_ARG, "pattern row_ptr inconsistent");
    for (int i = 0; i < p.n; ++i) {
        if (p.row_ptr[i + 1] < p.row_ptr[i]) fail(CFDB_ERR_BAD_ARG, "pattern row_ptr not monotone");
        if (p.diag_pos[i] < p.row_ptr[i] || p.diag_pos[i] >= p.row_ptr[i + 1])
            fail(CFDB_ERR_BAD_ARG, "diag_pos outside its row");
    }
    for (int k = 0; k < p.nnz; ++k)
        if (p.col[k] < 0 || p.col[k] >= p.n) fail(CFDB_ERR_BAD_ARG, "pattern column out of range");
    for (int f = 0; f < p.n_faces; ++f) {
        if (p.upper_pos[f] < 0 || p.upper_pos[f] >= p.nnz || p.lower_pos[f] < 0 || p.lower_pos[f] >= p.nnz)
            fail(CFDB_ERR_BAD_ARG, "face position out of range");
    }
}

// Cell -> face lists in ascending face order (owner and neighbour faces merged).
void cell_faces(int n, int nf, const int* own, const int* nei, std::vector<int>& ptr, std::vector<int>& face) {
    ptr.assign(static_cast<size_t>(n) + 1, 0);
    for (int f = 0; f < nf; ++f) {
        ++ptr[own[f] + 1];
        ++ptr[nei[f] + 1];
    }
    for (int c = 0; c < n; ++c) ptr[c + 1] += ptr[c];
    face.resize(static_cast<size_t>(ptr[n]));
    std::vector<int> fill(ptr.begin(), ptr.end() - 1);
    for (int f = 0; f < nf; ++f) {
        face[fill[own[f]]++] = f;
        face[fill[nei[f]]++] = f;
    }
}

SolveResult run_single(cfdb_system* s, const double* diag, const double* upper, const double* lower,
                       const double* b, double* x, int method, int use_amg, const cfdb_control* c, bool dev) {
    if (c == nullptr) fail(CFDB_ERR_BAD_ARG, "null control");
    if (method != CFDB_METHOD_CG && method != CFDB_METHOD_BICGSTAB) fail(CFDB_ERR_BAD_ARG, "unknown method");
    if (diag == nullptr || b == nullptr || x == nullptr || (s->pat.n_faces > 0 && (upper == nullptr || lower == nullptr)))
        fail(CFDB_ERR_BAD_ARG, "null array");
    ensure_engine(s);
    Engine& e = *s->eng;
    const int n = s->pat.n, nf = s->pat.n_faces;
    if (dev) {
        e.set_values_device(diag, upper, lower, n, n + nf);
    } else {
        // the caller's arrays are read by the copies before this call returns
        e.upload_values_ldu(diag, upper, lower, n, nf);
    }
    e.set_rhs(0, b, dev);
    e.set_guess(0, x, dev);
    // krylov_cuda.cu:659-669: with a hierarchy and use_amg the solve is AMG-CG whatever the
    // method; otherwise Jacobi-preconditioned CG or BiCGStab on the FP64 level-0 operator
    Mode mode = Mode::Jacobi;
    if (use_amg && s->h) mode = s->precision == CFDB_PRECISION_MIXED ? Mode::AmgMixed : Mode::AmgFp64;
    SolveRequest rq;
    rq.tol = c->abs_tolerance;
    rq.max_it = c->max_iterations;
    const auto res = (mode == Mode::Jacobi && method == CFDB_METHOD_BICGSTAB) ? std::vector<SolveResult>{e.solve_bicgstab(rq)}
                                                                              : e.solve(mode, {rq});
    e.get_solution(0, x, dev);
    CFDB_CUDA(cudaStreamSynchronize(e.stream()));
    return res[0];
}

void put_stats(cfdb_stats* st, const SolveResult& r) {
    if (st == nullptr) return;
    st->iterations = r.iterations;
    st->residual = r.residual;
    st->converged = r.converged ? 1 : 0;
    st->on_device = 1;
    st->true_residual = r.true_residual;
}

} // namespace

extern "C" {

int cfdb_backend_name(char* buf, size_t len) { return copy_str("cuda", buf, len); }

int cfdb_device_available(void) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        (void)cudaGetLastError();
        return 0;
    }
    return count > 0 ? 1 : 0;
}

int cfdb_device_description(char* buf, size_t len) {
    std::string s = "cuda";
    int dev = 0;
    cudaDeviceProp prop{};
    if (cfdb_device_available() && cudaGetDevice(&dev) == cudaSuccess &&
        cudaGetDeviceProperties(&prop, dev) == cudaSuccess) {
        s += std::string(" (device: ") + prop.name + ", sm_" + std::to_string(prop.major) +
             std::to_string(prop.minor) + ")";
    } else {
        (void)cudaGetLastError();
        s += " (no CUDA device)";
    }
    return copy_str(s, buf, len);
}

int cfdb_last_error(char* buf, size_t len) { return copy_str(g_last_error, buf, len); }

int cfdb_release_cached_memory(void) {
    return guarded([&] {
        require_device();
        int dev = 0;
        CFDB_CUDA(cudaGetDevice(&dev));
        trim_device_pools(dev);
    });
}

void cfdb_default_amg_settings(cfdb_amg_settings* s) {
    if (s == nullptr) return;
    s->strength_threshold = 0.08;
    s->max_levels = 25;
    s->coarse_size = 400;
    s->smooth_sweeps = 2;
    s->jacobi_weight = 0.7;
    s->device_table_limit = 0;
}

int cfdb_build_pattern(int n, int n_faces, const int* owner, const int* neighbour, int* row_ptr, int* col,
                       int* diag_pos, int* upper_pos, int* lower_pos, int* nnz) {
    return guarded([&] {
        if (n <= 0 || n_faces < 0 || (n_faces > 0 && (owner == nullptr || neighbour == nullptr)) ||
            row_ptr == nullptr || col == nullptr || diag_pos == nullptr || nnz == nullptr)
            fail(CFDB_ERR_BAD_ARG, "cfdb_build_pattern: bad arguments");
        const LduPatternHost p = build_pattern(n, n_faces, owner, neighbour);
        std::memcpy(row_ptr, p.row_ptr.data(), sizeof(int) * (n + 1));
        std::memcpy(col, p.col.data(), sizeof(int) * p.col.size());
        std::memcpy(diag_pos, p.diag_pos.data(), sizeof(int) * n);
        if (n_faces > 0) {
            std::memcpy(upper_pos, p.upper_pos.data(), sizeof(int) * n_faces);
            std::memcpy(lower_pos, p.lower_pos.data(), sizeof(int) * n_faces);
        }
        *nnz = p.nnz();
    });
}

// ---- assembly ----

static int assemble_impl(int n_cells, int n_faces, const int* owner, const int* neighbour, const double* flux,
                         const double* gamma, const double* delta, double convection, double* upper,
                         double* lower, double* diag, double* div, bool dev) {
    return guarded([&] {
        require_device();
        if (n_cells < 0 || n_faces < 0) fail(CFDB_ERR_BAD_ARG, "negative size");
        if (n_faces == 0) return; // reference: nothing to do (krylov_cuda.cu:705-707)
        if (!owner || !neighbour || !flux || !gamma || !delta || !upper || !lower || !diag || !div)
            fail(CFDB_ERR_BAD_ARG, "null array");
        std::vector<int> h_own, h_nei;
        const int* own_h = owner;
        const int* nei_h = neighbour;
        if (dev) {
            h_own.resize(n_faces);
            h_nei.resize(n_faces);
            CFDB_CUDA(cudaMemcpy(h_own.data(), owner, sizeof(int) * n_faces, cudaMemcpyDeviceToHost));
            CFDB_CUDA(cudaMemcpy(h_nei.data(), neighbour, sizeof(int) * n_faces, cudaMemcpyDeviceToHost));
            own_h = h_own.data();
            nei_h = h_nei.data();
        }
        for (int f = 0; f < n_faces; ++f) {
            if (own_h[f] < 0 || own_h[f] >= n_cells || nei_h[f] < 0 || nei_h[f] >= n_cells)
                fail(CFDB_ERR_BAD_ARG, "face addresses a cell out of range");
        }
        std::vector<int> ptr, face;
        cell_faces(n_cells, n_faces, own_h, nei_h, ptr, face);
        DeviceArena ar; // released after the guard has drained the stream
        cudaStream_t st = nullptr;
        CFDB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        struct StreamGuard {
            cudaStream_t s;
            ~StreamGuard() { cudaStreamSynchronize(s); cudaStreamDestroy(s); }
        } guard{st};
        const int* d_ptr = ar.upload(ptr, st);
        const int* d_face = ar.upload(face, st);
        const int* d_own;
        const double *d_flux, *d_gamma, *d_delta;
        double *d_up, *d_lo, *d_diag, *d_div;
        if (dev) {
            d_own = owner;
            d_flux = flux;
            d_gamma = gamma;
            d_delta = delta;
            d_up = upper;
            d_lo = lower;
            d_diag = diag;
            d_div = div;
        } else {
            int* o = ar.alloc<int>(n_faces);
            double* buf = ar.alloc<double>(5 * static_cast<size_t>(n_faces) + 2 * static_cast<size_t>(n_cells));
            CFDB_CUDA(cudaMemcpyAsync(o, owner, sizeof(int) * n_faces, cudaMemcpyHostToDevice, st));
            double* fl = buf;
            double* ga = fl + n_faces;
            double* de = ga + n_faces;
            d_up = de + n_faces;
            d_lo = d_up + n_faces;
            d_diag = d_lo + n_faces;
            d_div = d_diag + n_cells;
            CFDB_CUDA(cudaMemcpyAsync(fl, flux, sizeof(double) * n_faces, cudaMemcpyHostToDevice, st));
            CFDB_CUDA(cudaMemcpyAsync(ga, gamma, sizeof(double) * n_faces, cudaMemcpyHostToDevice, st));
            CFDB_CUDA(cudaMemcpyAsync(de, delta, sizeof(double) * n_faces, cudaMemcpyHostToDevice, st));
            CFDB_CUDA(cudaMemcpyAsync(d_diag, diag, sizeof(double) * n_cells, cudaMemcpyHostToDevice, st));
            CFDB_CUDA(cudaMemcpyAsync(d_div, div, sizeof(double) * n_cells, cudaMemcpyHostToDevice, st));
            d_own = o;
            d_flux = fl;
            d_gamma = ga;
            d_delta = de;
        }
        k_assemble_faces<<<(n_faces + 255) / 256, 256, 0, st>>>(n_faces, d_flux, d_gamma, d_delta, convection, d_up,
                                                               d_lo);
        k_assemble_cells<<<(n_cells + 255) / 256, 256, 0, st>>>(n_cells, d_ptr, d_face, d_flux, d_gamma, d_delta, d_own,
                                                               convection, d_diag, d_div);
        CFDB_CUDA(cudaGetLastError());
        if (!dev) {
            CFDB_CUDA(cudaMemcpyAsync(upper, d_up, sizeof(double) * n_faces, cudaMemcpyDeviceToHost, st));
            CFDB_CUDA(cudaMemcpyAsync(lower, d_lo, sizeof(double) * n_faces, cudaMemcpyDeviceToHost, st));
            CFDB_CUDA(cudaMemcpyAsync(diag, d_diag, sizeof(double) * n_cells, cudaMemcpyDeviceToHost, st));
            CFDB_CUDA(cudaMemcpyAsync(div, d_div, sizeof(double) * n_cells, cudaMemcpyDeviceToHost, st));
        }
        CFDB_CUDA(cudaStreamSynchronize(st));
    });
}

int cfdb_assemble(int n_cells, int n_faces, const int* owner, const int* neighbour, const double* flux,
                  const double* gamma, const double* delta_coeff, double convection, double* upper, double* lower,
                  double* diag, double* divergence) {
    return assemble_impl(n_cells, n_faces, owner, neighbour, flux, gamma, delta_coeff, convection, upper, lower,
                         diag, divergence, false);
}

int cfdb_assemble_device(int n_cells, int n_faces, const int* owner, const int* neighbour, const double* flux,
                         const double* gamma, const double* delta_coeff, double convection, double* upper,
                         double* lower, double* diag, double* divergence) {
    return assemble_impl(n_cells, n_faces, owner, neighbour, flux, gamma, delta_coeff, convection, upper, lower,
                         diag, divergence, true);
}

// ---- one-shot solves ----

int cfdb_solve(const cfdb_csr* a, const double* b, double* x, int method, const cfdb_control* control,
               cfdb_stats* stats) {
    return guarded([&] {
        require_device();
        if (a == nullptr || b == nullptr || x == nullptr || control == nullptr) fail(CFDB_ERR_BAD_ARG, "null argument");
        if (method != CFDB_METHOD_CG && method != CFDB_METHOD_BICGSTAB) fail(CFDB_ERR_BAD_ARG, "unknown method");
        if (a->n == 0) {
            put_stats(stats, SolveResult{0, 0.0, true, 0.0});
            return;
        }
        const HostCsr m = csr_from(*a, a->n);
        int dev = 0;
        CFDB_CUDA(cudaGetDevice(&dev));
        Engine e(dev);
        SystemSpec sp;
        sp.n = m.n_rows;
        sp.rp = m.rp.data();
        sp.ci = m.ci.data();
        sp.src.resize(m.nnz());
        for (int k = 0; k < m.nnz(); ++k) sp.src[k] = k;
        sp.diag_src.assign(m.n_rows, -1);
        for (int i = 0; i < m.n_rows; ++i)
            for (int k = m.rp[i]; k < m.rp[i + 1]; ++k)
                if (m.ci[k] == i && m.va[k] != 0.0) sp.diag_src[i] = k;
        sp.vs_len = m.nnz();
        std::vector<SystemSpec> v;
        v.push_back(std::move(sp));
        e.build(std::move(v), 2, 0.7, true, false);
        e.upload_values({m.va.data()});
        e.set_rhs(0, b, false);
        e.set_guess(0, x, false);
        const SolveRequest rq{control->abs_tolerance, control->max_iterations};
        const SolveResult r = method == CFDB_METHOD_BICGSTAB ? e.solve_bicgstab(rq) : e.solve(Mode::Jacobi, {rq})[0];
        e.get_solution(0, x, false);
        put_stats(stats, r);
    });
}

int cfdb_solve_amg_cg(const cfdb_amg_view* amg, const double* b, double* x, const cfdb_control* control,
                      cfdb_stats* stats) {
    return guarded([&] {
        require_device();
        if (amg == nullptr || amg->n_levels <= 0 || amg->levels == nullptr)
            fail(CFDB_ERR_BAD_ARG, "solve_amg_cg: empty hierarchy");
        if (b == nullptr || x == nullptr || control == nullptr) fail(CFDB_ERR_BAD_ARG, "null argument");
        const int n0 = amg->levels[0].a.n;
        auto h = hierarchy_from(*amg, n0, false);
        const HostCsr& m = h->a[0];
        int dev = 0;
        CFDB_CUDA(cudaGetDevice(&dev));
        Engine e(dev);
        SystemSpec sp;
        sp.n = m.n_rows;
        sp.rp = m.rp.data();
        sp.ci = m.ci.data();
        sp.src.resize(m.nnz());
        for (int k = 0; k < m.nnz(); ++k) sp.src[k] = k;
        sp.diag_src.assign(m.n_rows, -1);
        for (int i = 0; i < m.n_rows; ++i)
            for (int k = m.rp[i]; k < m.rp[i + 1]; ++k)
                if (m.ci[k] == i && m.va[k] != 0.0) sp.diag_src[i] = k;
        sp.vs_len = m.nnz();
        sp.h = h;
        std::vector<SystemSpec> v;
        v.push_back(std::move(sp));
        e.build(std::move(v), amg->smooth_sweeps, amg->jacobi_weight, true, false);
        e.upload_values({m.va.data()});
        e.set_rhs(0, b, false);
        e.set_guess(0, x, false);
        const auto r = e.solve(Mode::AmgFp64, {SolveRequest{control->abs_tolerance, control->max_iterations}});
        e.get_solution(0, x, false);
        put_stats(stats, r[0]);
    });
}

// ---- hierarchy ----

struct cfdb_hierarchy {
    Hierarchy h;
    std::vector<cfdb_amg_level> view_levels;
};

int cfdb_amg_setup(const cfdb_csr* a, const cfdb_amg_settings* settings, cfdb_hierarchy** out) {
    return guarded([&] {
        if (a == nullptr || out == nullptr) fail(CFDB_ERR_BAD_ARG, "null argument");
        AmgSettings s;
        if (settings != nullptr) {
            s.theta = settings->strength_threshold;
            s.max_levels = settings->max_levels;
            s.coarse_size = settings->coarse_size;
            s.sweeps = settings->smooth_sweeps;
            s.weight = settings->jacobi_weight;
        }
        if (s.max_levels < 1) fail(CFDB_ERR_BAD_ARG, "max_levels must be >= 1");
        const HostCsr m = csr_from(*a, a->n);
        auto* h = new cfdb_hierarchy;
        try {
            h->h = amg_setup(m, s);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int cfdb_amg_setup_device(const cfdb_csr* a, const cfdb_amg_settings* settings, cfdb_hierarchy** out) {
    return guarded([&] {
        require_device();
        if (a == nullptr || out == nullptr) fail(CFDB_ERR_BAD_ARG, "null argument");
        const AmgSettings s = settings_from(settings);
        const HostCsr m = csr_from(*a, a->n);
        CallStream cs;
        DeviceHierarchy dh;
        DevCsr a0;
        a0.n_rows = a0.n_cols = m.n_rows;
        a0.nnz = m.nnz();
        a0.rp = dh.mem.alloc<int>(m.rp.size());
        a0.ci = dh.mem.alloc<int>(m.ci.size());
        a0.va = dh.mem.alloc<double>(m.va.size());
        CFDB_CUDA(cudaMemcpyAsync(a0.rp, m.rp.data(), sizeof(int) * m.rp.size(), cudaMemcpyHostToDevice, cs.s));
        if (a0.nnz > 0) {
            CFDB_CUDA(cudaMemcpyAsync(a0.ci, m.ci.data(), sizeof(int) * m.ci.size(), cudaMemcpyHostToDevice, cs.s));
            CFDB_CUDA(cudaMemcpyAsync(a0.va, m.va.data(), sizeof(double) * m.va.size(), cudaMemcpyHostToDevice, cs.s));
        }
        amg_setup_device(a0, s, cs.s, dh);
        auto* h = new cfdb_hierarchy;
        try {
            h->h = download_hierarchy(dh, /*with_a0=*/true, cs.s);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int cfdb_hierarchy_destroy(cfdb_hierarchy* h) {
    delete h;
    return CFDB_OK;
}

int cfdb_hierarchy_levels(const cfdb_hierarchy* h, int* n_levels) {
    if (h == nullptr || n_levels == nullptr) return set_error(CFDB_ERR_BAD_ARG, "null argument");
    *n_levels = h->h.levels();
    return CFDB_OK;
}

static cfdb_csr view_of(const HostCsr& m) {
    return cfdb_csr{m.n_rows, m.nnz(), m.rp.data(), m.ci.data(), m.va.data()};
}

int cfdb_hierarchy_level(const cfdb_hierarchy* h, int level, int which, int* n_rows, int* n_cols, cfdb_csr* m) {
    if (h == nullptr || m == nullptr) return set_error(CFDB_ERR_BAD_ARG, "null argument");
    if (level < 0 || level >= h->h.levels()) return set_error(CFDB_ERR_BAD_ARG, "level out of range");
    const HostCsr* src = nullptr;
    if (which == 0) src = &h->h.a[level];
    else if (level + 1 < h->h.levels()) src = which == 1 ? &h->h.p[level] : &h->h.r[level];
    if (src == nullptr) return set_error(CFDB_ERR_BAD_ARG, "no such operator on this level");
    *m = view_of(*src);
    if (n_rows) *n_rows = src->n_rows;
    if (n_cols) *n_cols = src->n_cols;
    return CFDB_OK;
}

int cfdb_hierarchy_aggregates(const cfdb_hierarchy* h, int level, const int** agg, int* n_aggregates) {
    if (h == nullptr || agg == nullptr) return set_error(CFDB_ERR_BAD_ARG, "null argument");
    if (level < 0 || level + 1 >= h->h.levels()) return set_error(CFDB_ERR_BAD_ARG, "level has no aggregates");
    *agg = h->h.agg[level].data();
    if (n_aggregates) *n_aggregates = h->h.n_agg[level];
    return CFDB_OK;
}

int cfdb_hierarchy_coarse_inverse(const cfdb_hierarchy* h, const double** inv, int* n_c) {
    if (h == nullptr || inv == nullptr) return set_error(CFDB_ERR_BAD_ARG, "null argument");
    *inv = h->h.coarse_inverse.data();
    if (n_c) *n_c = h->h.n_c;
    return CFDB_OK;
}

int cfdb_hierarchy_view(cfdb_hierarchy* h, int smooth_sweeps, double jacobi_weight, cfdb_amg_view* view) {
    if (h == nullptr || view == nullptr) return set_error(CFDB_ERR_BAD_ARG, "null argument");
    const int L = h->h.levels();
    h->view_levels.assign(L, cfdb_amg_level{});
    for (int l = 0; l < L; ++l) {
        h->view_levels[l].a = view_of(h->h.a[l]);
        if (l + 1 < L) {
            h->view_levels[l].p = view_of(h->h.p[l]);
            h->view_levels[l].r = view_of(h->h.r[l]);
        }
    }
    view->n_levels = L;
    view->levels = h->view_levels.data();
    view->coarse_inverse = h->h.coarse_inverse.data();
    view->smooth_sweeps = smooth_sweeps;
    view->jacobi_weight = jacobi_weight;
    return CFDB_OK;
}

int cfdb_hierarchy_operator_complexity(const cfdb_hierarchy* h, double* oc) {
    if (h == nullptr || oc == nullptr) return set_error(CFDB_ERR_BAD_ARG, "null argument");
    *oc = h->h.operator_complexity();
    return CFDB_OK;
}

// ---- persistent system ----

int cfdb_system_create(const cfdb_ldu_pattern* pattern, cfdb_system** out) {
    return guarded([&] {
        require_device();
        if (pattern == nullptr || out == nullptr) fail(CFDB_ERR_BAD_ARG, "null argument");
        validate_pattern(*pattern);
        auto s = std::make_unique<cfdb_system>();
        CFDB_CUDA(cudaGetDevice(&s->device));
        LduPatternHost& p = s->pat;
        p.n = pattern->n;
        p.n_faces = pattern->n_faces;
        p.row_ptr.assign(pattern->row_ptr, pattern->row_ptr + pattern->n + 1);
        p.col.assign(pattern->col, pattern->col + pattern->nnz);
        p.diag_pos.assign(pattern->diag_pos, pattern->diag_pos + pattern->n);
        if (pattern->n_faces > 0) {
            p.upper_pos.assign(pattern->upper_pos, pattern->upper_pos + pattern->n_faces);
            p.lower_pos.assign(pattern->lower_pos, pattern->lower_pos + pattern->n_faces);
        }
        build_value_map(s.get());
        ensure_engine(s.get());
        *out = s.release();
    });
}

int cfdb_system_create_mesh(int n_cells, int n_faces, const int* owner, const int* neighbour, cfdb_system** out) {
    return guarded([&] {
        require_device();
        if (out == nullptr || n_cells <= 0 || n_faces < 0 || (n_faces > 0 && (!owner || !neighbour)))
            fail(CFDB_ERR_BAD_ARG, "bad arguments");
        auto s = std::make_unique<cfdb_system>();
        CFDB_CUDA(cudaGetDevice(&s->device));
        s->pat = build_pattern(n_cells, n_faces, owner, neighbour);
        s->owner.assign(owner, owner + n_faces);
        s->neighbour.assign(neighbour, neighbour + n_faces);
        build_value_map(s.get());
        std::vector<int> ptr, face;
        cell_faces(n_cells, n_faces, owner, neighbour, ptr, face);
        CFDB_CUDA(cudaSetDevice(s->device));
        s->d_owner = s->asm_arena.upload(s->owner, nullptr);
        s->d_cf_ptr = s->asm_arena.upload(ptr, nullptr);
        s->d_cf_face = s->asm_arena.upload(face, nullptr);
        CFDB_CUDA(cudaDeviceSynchronize());
        ensure_engine(s.get());
        *out = s.release();
    });
}

int cfdb_system_destroy(cfdb_system* sys) {
    return guarded([&] {
        if (sys == nullptr) return;
        cudaSetDevice(sys->device);
        // device buffers go back to the pool at once: let the work that uses them finish
        if (sys->eng) cudaStreamSynchronize(sys->eng->stream());
        delete sys;
    });
}

int cfdb_system_on_device(const cfdb_system* sys) { return sys != nullptr && sys->eng ? 1 : 0; }

int cfdb_system_set_amg(cfdb_system* sys, const cfdb_amg_view* amg) {
    return guarded([&] {
        if (sys == nullptr || amg == nullptr) fail(CFDB_ERR_BAD_ARG, "null argument");
        if (amg->n_levels <= 0 || amg->levels == nullptr)
            fail(CFDB_ERR_BAD_ARG, "DeviceSolver::set_amg: empty hierarchy");
        sys->h = hierarchy_from(*amg, sys->pat.n, /*skip_a0=*/true);
        sys->dl.reset();
        sys->h_shapes_only = false;
        sys->sweeps = amg->smooth_sweeps;
        sys->weight = amg->jacobi_weight;
        sys->dirty = true;
        ensure_engine(sys);
    });
}

int cfdb_system_setup_amg(cfdb_system* sys, const double* diag, const double* upper, const double* lower,
                          const cfdb_amg_settings* settings) {
    return guarded([&] {
        if (sys == nullptr || diag == nullptr) fail(CFDB_ERR_BAD_ARG, "null argument");
        const LduPatternHost& p = sys->pat;
        HostCsr a;
        a.n_rows = a.n_cols = p.n;
        a.rp = p.row_ptr;
        a.ci = p.col;
        a.va.assign(static_cast<size_t>(p.nnz()), 0.0);
        for (int i = 0; i < p.n; ++i) a.va[p.diag_pos[i]] = diag[i];
        for (int f = 0; f < p.n_faces; ++f) {
            a.va[p.upper_pos[f]] = upper[f];
            a.va[p.lower_pos[f]] = lower[f];
        }
        AmgSettings s;
        if (settings != nullptr) {
            s.theta = settings->strength_threshold;
            s.max_levels = settings->max_levels;
            s.coarse_size = settings->coarse_size;
            s.sweeps = settings->smooth_sweeps;
            s.weight = settings->jacobi_weight;
        }
        const double t0 = PhaseTimes::now();
        auto h = std::make_shared<Hierarchy>(amg_setup(a, s));
        const double t1 = PhaseTimes::now();
        sys->dl.reset();
        sys->h_shapes_only = false;
        if (h->levels() <= 1) {
            // ldu_matrix.cpp:358: a single-level hierarchy runs Jacobi CG instead of AMG
            sys->h.reset();
        } else {
            sys->h = h;
        }
        sys->sweeps = s.sweeps;
        sys->weight = s.weight;
        sys->dirty = true;
        ensure_engine(sys);
        PhaseTimes pt;
        pt.add("hierarchy", t1 - t0);
        pt.add("plan", PhaseTimes::now() - t1);
        sys->setup_profile = pt.text();
    });
}

int cfdb_system_setup_amg_device(cfdb_system* sys, const double* diag, const double* upper, const double* lower,
                                 const cfdb_amg_settings* settings, int device_arrays) {
    return guarded([&] {
        if (sys == nullptr || diag == nullptr || (sys->pat.n_faces > 0 && (upper == nullptr || lower == nullptr)))
            fail(CFDB_ERR_BAD_ARG, "null argument");
        const double t_in = PhaseTimes::now();
        const AmgSettings s = settings_from(settings);
        const LduPatternHost& p = sys->pat;
        CFDB_CUDA(cudaSetDevice(sys->device));
        CallStream cs;
        pattern_on_device(sys, cs.s);
        // The previous hierarchy's device levels serve only plan rebuilds (the plan holds its
        // own copies), and this call replaces the plan: free them first, so that the new
        // hierarchy takes over their blocks instead of growing the memory pool by a second
        // hierarchy. Until the new one is installed the system has none.
        if (sys->dl) {
            CFDB_CUDA(cudaStreamSynchronize(sys->eng ? sys->eng->stream() : cs.s));
            sys->dl.reset();
            if (sys->h_shapes_only) {
                sys->h.reset();
                sys->h_shapes_only = false;
                sys->dirty = true;
            }
        }
        const double t_wait = PhaseTimes::now();
        DeviceHierarchy dh;
        const double *dd = diag, *du = upper, *dl = lower;
        if (!device_arrays) {
            double* ldu = dh.mem.alloc<double>(static_cast<size_t>(p.n) + 2 * static_cast<size_t>(p.n_faces));
            CFDB_CUDA(cudaMemcpyAsync(ldu, diag, sizeof(double) * p.n, cudaMemcpyHostToDevice, cs.s));
            if (p.n_faces > 0) {
                CFDB_CUDA(cudaMemcpyAsync(ldu + p.n, upper, sizeof(double) * p.n_faces, cudaMemcpyHostToDevice, cs.s));
                CFDB_CUDA(cudaMemcpyAsync(ldu + p.n + p.n_faces, lower, sizeof(double) * p.n_faces,
                                          cudaMemcpyHostToDevice, cs.s));
            }
            dd = ldu;
            du = ldu + p.n;
            dl = ldu + p.n + p.n_faces;
        }
        DevCsr a0;
        a0.n_rows = a0.n_cols = p.n;
        a0.nnz = p.nnz();
        a0.rp = sys->d_rp;
        a0.ci = sys->d_ci;
        a0.va = dh.mem.alloc<double>(static_cast<size_t>(p.nnz()));
        CFDB_CUDA(cudaMemsetAsync(a0.va, 0, sizeof(double) * p.nnz(), cs.s));
        ldu_to_csr_values(p.n, p.n_faces, sys->d_dpos, sys->d_upos, sys->d_lpos, dd, du, dl, a0.va, cs.s);
        const double t0 = PhaseTimes::now();
        // the hierarchy's own arrays go to an arena the system keeps: the plan is laid out on
        // the device from them, and plan rebuilds need no host copy
        auto kept = std::make_shared<DeviceLevels>();
        amg_setup_device(a0, s, cs.s, dh, &sys->stage, &kept->mem);
        const double t1 = PhaseTimes::now();
        // input_wait: the system's stream drained (its queued work) before the old levels go
        dh.times.add("input_wait", t_wait - t_in);
        dh.times.add("input", t0 - t_wait);
        adopt_levels(dh, *kept);
        auto h = std::make_shared<Hierarchy>(hierarchy_shape(dh));
        const double t2 = PhaseTimes::now();
        dh.times.add("keep", t2 - t1);
        if (h->levels() <= 1) {
            sys->h.reset(); // ldu_matrix.cpp:358: one level runs Jacobi CG
            sys->dl.reset();
            sys->h_shapes_only = false;
        } else {
            sys->h = h;
            sys->dl = kept;
            sys->h_shapes_only = true;
        }
        sys->sweeps = s.sweeps;
        sys->weight = s.weight;
        sys->dirty = true;
        ensure_engine(sys);
        if (!sys->keep_levels) sys->dl.reset();
        dh.times.add("plan", PhaseTimes::now() - t2);
        for (const auto& pt : sys->eng->build_times().t) dh.times.add(pt.first, pt.second);
        sys->setup_profile = dh.times.text();
    });
}

int cfdb_system_time_sweep(cfdb_system* sys, int level, int reps, double* ms, double* bytes) {
    return guarded([&] {
        if (sys == nullptr || ms == nullptr) fail(CFDB_ERR_BAD_ARG, "null argument");
        CFDB_CUDA(cudaSetDevice(sys->device));
        ensure_engine(sys);
        *ms = sys->eng->time_sweep(level, reps, bytes);
    });
}

int cfdb_system_set_keep_levels(cfdb_system* sys, int keep) {
    if (sys == nullptr) return set_error(CFDB_ERR_BAD_ARG, "null system");
    sys->keep_levels = keep != 0;
    return CFDB_OK;
}

int cfdb_system_setup_profile(const cfdb_system* sys, char* buf, size_t len) {
    if (sys == nullptr) return set_error(CFDB_ERR_BAD_ARG, "null system");
    return copy_str(sys->setup_profile, buf, len);
}

int cfdb_system_set_precision(cfdb_system* sys, int precision) {
    return guarded([&] {
        if (sys == nullptr) fail(CFDB_ERR_BAD_ARG, "null system");
        if (precision != CFDB_PRECISION_FP64 && precision != CFDB_PRECISION_MIXED)
            fail(CFDB_ERR_BAD_ARG, "unknown precision");
        if (sys->precision != precision) {
            sys->precision = precision;
            sys->dirty = true;
            ensure_engine(sys);
        }
    });
}

int cfdb_system_solve(cfdb_system* sys, const double* diag, const double* upper, const double* lower, const double* b,
                      double* x, int method, int use_amg, const cfdb_control* control, cfdb_stats* stats) {
    return guarded([&] {
        if (sys == nullptr) fail(CFDB_ERR_BAD_ARG, "null system");
        CFDB_CUDA(cudaSetDevice(sys->device));
        put_stats(stats, run_single(sys, diag, upper, lower, b, x, method, use_amg, control, false));
    });
}

int cfdb_system_solve_device(cfdb_system* sys, const double* diag, const double* upper, const double* lower,
                             const double* b, double* x, int method, int use_amg, const cfdb_control* control,
                             cfdb_stats* stats) {
    return guarded([&] {
        if (sys == nullptr) fail(CFDB_ERR_BAD_ARG, "null system");
        CFDB_CUDA(cudaSetDevice(sys->device));
        put_stats(stats, run_single(sys, diag, upper, lower, b, x, method, use_amg, control, true));
    });
}

void cfdb_default_ldu_settings(cfdb_ldu_settings* s) {
    if (s == nullptr) return;
    s->method = CFDB_METHOD_CG;
    s->tolerance = 1e-10;
    s->rel_tolerance = 0.01;
    s->max_iterations = 1000;
    s->max_age = 20;
}

int cfdb_system_solve_ldu(cfdb_system* sys, const double* diag, const double* upper, const double* lower,
                          const double* source, double* x, const cfdb_ldu_settings* settings,
                          const cfdb_amg_settings* amg, int device_arrays, cfdb_ldu_result* result) {
    return guarded([&] {
        if (sys == nullptr || settings == nullptr || result == nullptr) fail(CFDB_ERR_BAD_ARG, "null argument");
        const LduPatternHost& p = sys->pat;
        const int n = p.n, nf = p.n_faces;
        if (diag == nullptr || source == nullptr || x == nullptr || (nf > 0 && (upper == nullptr || lower == nullptr)))
            fail(CFDB_ERR_BAD_ARG, "null array");
        if (settings->method != CFDB_METHOD_CG && settings->method != CFDB_METHOD_BICGSTAB)
            fail(CFDB_ERR_BAD_ARG, "unknown method");
        CFDB_CUDA(cudaSetDevice(sys->device));
        ensure_engine(sys);
        cudaStream_t st = sys->eng->stream();
        pattern_on_device(sys, st);
        if (sys->norm_part == nullptr) sys->norm_part = sys->ldu_arena.alloc<double>(3 * static_cast<size_t>(kLduNormBlocks));
        const double *dd = diag, *du = upper, *dl = lower, *db = source;
        double* dx = x;
        if (!device_arrays) {
            if (sys->ldu_stage == nullptr)
                sys->ldu_stage = sys->ldu_arena.alloc<double>(4 * static_cast<size_t>(n) + 2 * static_cast<size_t>(nf));
            double* s = sys->ldu_stage;
            auto put = [&](double* dst, const double* src, int cnt) {
                if (cnt > 0) sys->eng->copier().to_device(dst, src, sizeof(double) * cnt, st);
            };
            put(s, diag, n);
            put(s + n, upper, nf);
            put(s + n + nf, lower, nf);
            put(s + n + 2 * nf, source, n);
            put(s + 2 * n + 2 * nf, x, n);
            dd = s;
            du = s + n;
            dl = s + n + nf;
            db = s + n + 2 * nf;
            dx = s + 2 * n + 2 * nf;
        }
        const LduDevice m{n, nf, sys->d_rp, sys->d_ci, sys->d_src};
        // ldu_matrix.cpp:118-125: initial normalised residual; nothing to do below the tolerance
        const LduNorms n0 = ldu_residual_norms(m, dd, du, dl, db, dx, sys->norm_part, st);
        constexpr double kSmall = 1e-20; // ldu_matrix.cpp:22
        *result = cfdb_ldu_result{};
        result->initial_residual = n0.res / (n0.norm + kSmall);
        result->final_residual = result->initial_residual;
        if (result->initial_residual < settings->tolerance) return;
        // ldu_matrix.cpp:293-301: absolute CG target from the relative and absolute tolerances
        const double target = std::max(settings->rel_tolerance,
                                       settings->tolerance / std::max(result->initial_residual, kSmall)) *
                              std::sqrt(n0.r2);
        const bool cg = settings->method == CFDB_METHOD_CG;
        // ldu_matrix.cpp:314-353: (re)build the hierarchy at the first CG solve and after
        // max_age solves, here on the device from this matrix
        if (cg && (!sys->amg_built || sys->age >= settings->max_age)) {
            const int rc = cfdb_system_setup_amg_device(sys, dd, du, dl, amg, 1);
            if (rc != CFDB_OK) fail(rc, g_last_error);
            sys->age = 0;
            sys->amg_built = true;
            result->amg_rebuilt = 1;
        }
        if (cg) ++sys->age;
        const bool use_amg = cg && sys->h != nullptr;
        const cfdb_control ctl{std::max(target, 1e-300), settings->max_iterations};
        const SolveResult r = run_single(sys, dd, du, dl, db, dx, settings->method, use_amg ? 1 : 0, &ctl, true);
        result->iterations = r.iterations;
        const LduNorms n1 = ldu_residual_norms(m, dd, du, dl, db, dx, sys->norm_part, st);
        result->final_residual = n1.res / (n1.norm + kSmall);
        if (!device_arrays) sys->eng->copier().to_host(x, dx, sizeof(double) * n, st);
    });
}

int cfdb_system_assemble_device(cfdb_system* sys, const double* flux, const double* gamma, const double* delta,
                                double convection, double* upper, double* lower, double* diag, double* div) {
    return guarded([&] {
        if (sys == nullptr) fail(CFDB_ERR_BAD_ARG, "null system");
        if (sys->d_cf_ptr == nullptr) fail(CFDB_ERR_BAD_ARG, "system was not created from mesh addressing");
        if (!flux || !gamma || !delta || !upper || !lower || !diag || !div) fail(CFDB_ERR_BAD_ARG, "null array");
        CFDB_CUDA(cudaSetDevice(sys->device));
        ensure_engine(sys);
        cudaStream_t st = sys->eng->stream();
        const int n = sys->pat.n, nf = sys->pat.n_faces;
        if (nf > 0) {
            k_assemble_faces<<<(nf + 255) / 256, 256, 0, st>>>(nf, flux, gamma, delta, convection, upper, lower);
            ++sys->launches;
        }
        k_assemble_cells<<<(n + 255) / 256, 256, 0, st>>>(n, sys->d_cf_ptr, sys->d_cf_face, flux, gamma, delta,
                                                          sys->d_owner, convection, diag, div);
        ++sys->launches;
        CFDB_CUDA(cudaGetLastError());
        CFDB_CUDA(cudaStreamSynchronize(st));
    });
}

int cfdb_system_apply_amg(cfdb_system* sys, const double* r, double* z) {
    return guarded([&] {
        if (sys == nullptr || r == nullptr || z == nullptr) fail(CFDB_ERR_BAD_ARG, "null argument");
        if (!sys->h) fail(CFDB_ERR_NOT_READY, "apply_amg: no hierarchy installed");
        CFDB_CUDA(cudaSetDevice(sys->device));
        ensure_engine(sys);
        const Mode mode = sys->precision == CFDB_PRECISION_MIXED ? Mode::AmgMixed : Mode::AmgFp64;
        sys->eng->set_residual(0, r, false);
        sys->eng->apply_vcycle(mode, {0});
        sys->eng->get_precond(0, z, false, mode);
    });
}

int cfdb_system_set_ordered(cfdb_system* sys, int ordered) {
    return guarded([&] {
        if (sys == nullptr) fail(CFDB_ERR_BAD_ARG, "null system");
        CFDB_CUDA(cudaSetDevice(sys->device));
        ensure_engine(sys);
        if (sys->eng->ordered() != (ordered != 0)) {
            sys->eng->set_ordered(ordered != 0);
            sys->dirty = true;
            ensure_engine(sys);
        }
    });
}

int cfdb_system_profile(cfdb_system* sys, int use_amg, int reps, cfdb_kernel_record* records, int max_records,
                        int* n_records) {
    return guarded([&] {
        if (sys == nullptr || records == nullptr || n_records == nullptr) fail(CFDB_ERR_BAD_ARG, "null argument");
        CFDB_CUDA(cudaSetDevice(sys->device));
        ensure_engine(sys);
        Mode mode = Mode::Jacobi;
        if (use_amg && sys->h) mode = sys->precision == CFDB_PRECISION_MIXED ? Mode::AmgMixed : Mode::AmgFp64;
        const auto recs = sys->eng->profile(mode, reps);
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

int cfdb_system_assemble(cfdb_system* sys, const double* flux, const double* gamma, const double* delta,
                         double convection, double* upper, double* lower, double* diag, double* div) {
    return guarded([&] {
        if (sys == nullptr) fail(CFDB_ERR_BAD_ARG, "null system");
        if (sys->d_cf_ptr == nullptr) fail(CFDB_ERR_BAD_ARG, "system was not created from mesh addressing");
        if (!flux || !gamma || !delta || !upper || !lower || !diag || !div) fail(CFDB_ERR_BAD_ARG, "null array");
        CFDB_CUDA(cudaSetDevice(sys->device));
        ensure_engine(sys);
        cudaStream_t st = sys->eng->stream();
        const int n = sys->pat.n, nf = sys->pat.n_faces;
        if (sys->h_asm == nullptr) {
            sys->h_asm = sys->asm_arena.alloc<double>(5 * static_cast<size_t>(nf) + 2 * static_cast<size_t>(n));
        }
        double* d_fl = sys->h_asm;
        double* d_ga = d_fl + nf;
        double* d_de = d_ga + nf;
        double* d_up = d_de + nf;
        double* d_lo = d_up + nf;
        double* d_dg = d_lo + nf;
        double* d_dv = d_dg + n;
        if (sys->asm_cells.empty()) plan_assembly_slices(sys);
        const int n_slices = static_cast<int>(sys->asm_cells.size()) - 1;
        sys->asm_d2h.ensure(static_cast<size_t>(n_slices) + 1);
        cudaStream_t rb = sys->asm_d2h.s;
        // Slice j: upload the faces it adds to the prefix and its cells' diag / div, compute
        // those faces' coefficients and those cells' sums, then read them back on the second
        // stream while slice j+1 uploads (the copy engines run both directions at once).
        auto h2d = [&](double* dst, const double* src, int off, int cnt) {
            if (cnt > 0)
                CFDB_CUDA(cudaMemcpyAsync(dst + off, src + off, sizeof(double) * cnt, cudaMemcpyHostToDevice, st));
        };
        auto d2h = [&](double* dst, const double* src, int off, int cnt) {
            if (cnt > 0)
                CFDB_CUDA(cudaMemcpyAsync(dst + off, src + off, sizeof(double) * cnt, cudaMemcpyDeviceToHost, rb));
        };
        for (int j = 0; j < n_slices; ++j) {
            const int f0 = sys->asm_faces[j], f1 = sys->asm_faces[j + 1];
            const int c0 = sys->asm_cells[j], c1 = sys->asm_cells[j + 1];
            h2d(d_fl, flux, f0, f1 - f0);
            h2d(d_ga, gamma, f0, f1 - f0);
            h2d(d_de, delta, f0, f1 - f0);
            h2d(d_dg, diag, c0, c1 - c0);
            h2d(d_dv, div, c0, c1 - c0);
            if (f1 > f0) {
                k_assemble_faces<<<(f1 - f0 + 255) / 256, 256, 0, st>>>(f1 - f0, d_fl + f0, d_ga + f0, d_de + f0,
                                                                        convection, d_up + f0, d_lo + f0);
                ++sys->launches;
            }
            if (c1 > c0) {
                k_assemble_cell_range<<<(c1 - c0 + 255) / 256, 256, 0, st>>>(
                    c0, c1, sys->d_cf_ptr, sys->d_cf_face, d_fl, d_ga, d_de, sys->d_owner, convection, d_dg, d_dv);
                ++sys->launches;
            }
            CFDB_CUDA(cudaGetLastError());
            CFDB_CUDA(cudaEventRecord(sys->asm_d2h.ev[j], st));
            CFDB_CUDA(cudaStreamWaitEvent(rb, sys->asm_d2h.ev[j], 0));
            d2h(upper, d_up, f0, f1 - f0);
            d2h(lower, d_lo, f0, f1 - f0);
            d2h(diag, d_dg, c0, c1 - c0);
            d2h(div, d_dv, c0, c1 - c0);
        }
        // the engine's stream resumes only after the last read-back
        CFDB_CUDA(cudaEventRecord(sys->asm_d2h.ev[n_slices], rb));
        CFDB_CUDA(cudaStreamWaitEvent(st, sys->asm_d2h.ev[n_slices], 0));
        CFDB_CUDA(cudaStreamSynchronize(st));
    });
}

int cfdb_system_assemble_pressure_device(cfdb_system* sys, const double* flux, const double* gamma,
                                         const double* delta, const double* diag0, const double* source0,
                                         int ref_cell, double ref_value, double* upper, double* lower,
                                         double* diag, double* source) {
    return guarded([&] {
        if (sys == nullptr) fail(CFDB_ERR_BAD_ARG, "null system");
        if (sys->d_cf_ptr == nullptr) fail(CFDB_ERR_BAD_ARG, "system was not created from mesh addressing");
        if (!flux || !gamma || !delta || !source0 || !upper || !lower || !diag || !source)
            fail(CFDB_ERR_BAD_ARG, "null array");
        if (ref_cell >= sys->pat.n) fail(CFDB_ERR_BAD_ARG, "reference cell out of range");
        CFDB_CUDA(cudaSetDevice(sys->device));
        ensure_engine(sys);
        cudaStream_t st = sys->eng->stream();
        const int n = sys->pat.n, nf = sys->pat.n_faces;
        if (nf > 0) {
            k_assemble_faces<<<(nf + 255) / 256, 256, 0, st>>>(nf, flux, gamma, delta, 0.0, upper, lower);
            ++sys->launches;
        }
        k_assemble_pressure_cells<<<(n + 255) / 256, 256, 0, st>>>(n, sys->d_cf_ptr, sys->d_cf_face, flux, gamma,
                                                                   delta, sys->d_owner, diag0, source0, ref_cell,
                                                                   nullptr, ref_value, diag, source);
        ++sys->launches;
        CFDB_CUDA(cudaGetLastError());
    });
}

int cfdb_system_correct_pressure_device(cfdb_system* sys, const double* flux, const double* gamma,
                                        const double* delta, const double* non_orth, const double* p_new,
                                        const double* p_prev, double alpha, double* phi, double* p) {
    return guarded([&] {
        if (sys == nullptr) fail(CFDB_ERR_BAD_ARG, "null system");
        if (sys->d_cf_ptr == nullptr) fail(CFDB_ERR_BAD_ARG, "system was not created from mesh addressing");
        const int n = sys->pat.n, nf = sys->pat.n_faces;
        if (p_new == nullptr || p == nullptr || (nf > 0 && (!flux || !gamma || !delta || !phi)))
            fail(CFDB_ERR_BAD_ARG, "null array");
        CFDB_CUDA(cudaSetDevice(sys->device));
        ensure_engine(sys);
        cudaStream_t st = sys->eng->stream();
        if (nf > 0) {
            if (sys->d_neighbour == nullptr) {
                sys->d_neighbour = sys->asm_arena.upload(sys->neighbour, st);
            }
            k_correct_flux<<<(nf + 255) / 256, 256, 0, st>>>(nf, sys->d_owner, sys->d_neighbour, flux, gamma, delta,
                                                             non_orth, p_new, phi);
            ++sys->launches;
        }
        k_relax<<<(n + 255) / 256, 256, 0, st>>>(n, p_prev, p_new, alpha, p);
        ++sys->launches;
        CFDB_CUDA(cudaGetLastError());
    });
}

int cfdb_system_kernel_launches(const cfdb_system* sys, unsigned long long* count) {
    if (sys == nullptr || count == nullptr) return set_error(CFDB_ERR_BAD_ARG, "null argument");
    *count = sys->launches + (sys->eng ? sys->eng->kernel_launches() : 0);
    return CFDB_OK;
}

void cfdb_default_tuning(cfdb_tuning* t) {
    if (t == nullptr) return;
    const Tuning d{};
    t->target_tiles = d.target_tiles;
    t->wide_row = d.wide_row;
    t->lanes_div = d.lanes_div;
    t->fuse_first = d.fuse_first;
    t->sell_rows = d.sell_rows;
    t->krylov_pair = d.krylov_pair;
    t->tail_rows = d.tail_rows;
    t->col16 = d.col16;
    t->pdl = d.pdl;
    t->wait_polls = d.wait_polls;
    t->mixed_sweeps = d.mixed_sweeps;
    t->mixed_weight = d.mixed_weight;
    t->tail_cluster = d.tail_cluster;
    t->vcycle_pair = d.vcycle_pair;
    t->krylov_stage = d.krylov_stage;
}

int cfdb_system_set_tuning(cfdb_system* sys, const cfdb_tuning* t) {
    return guarded([&] {
        if (sys == nullptr) fail(CFDB_ERR_BAD_ARG, "null system");
        const Tuning tu = tuning_from(t);
        CFDB_CUDA(cudaSetDevice(sys->device));
        ensure_engine(sys);
        sys->eng->set_tuning(tu);
        sys->dirty = true;
        ensure_engine(sys);
    });
}

int cfdb_system_sizes(const cfdb_system* sys, int* n_cells, int* n_faces) {
    if (sys == nullptr) return set_error(CFDB_ERR_BAD_ARG, "null system");
    if (n_cells) *n_cells = sys->pat.n;
    if (n_faces) *n_faces = sys->pat.n_faces;
    return CFDB_OK;
}

int cfdb_system_stream(const cfdb_system* sys, void** stream) {
    if (sys == nullptr || stream == nullptr || !sys->eng) return set_error(CFDB_ERR_BAD_ARG, "null argument");
    *stream = sys->eng->stream();
    return CFDB_OK;
}

int cfdb_system_device_bytes(const cfdb_system* sys, size_t* bytes) {
    if (sys == nullptr || bytes == nullptr) return set_error(CFDB_ERR_BAD_ARG, "null argument");
    *bytes = (sys->eng ? sys->eng->device_bytes() : 0) + sys->asm_arena.bytes() + sys->pat_arena.bytes() +
             (sys->dl ? sys->dl->bytes() : 0);
    return CFDB_OK;
}

} // extern "C"
