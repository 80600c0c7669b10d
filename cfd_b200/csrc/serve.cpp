// Serving loop for pressure solves (declared in include/cfdb_serve.h).
//
// Requests (a registered mesh, LDU coefficients, right-hand side) are queued at submit time and
// taken by worker slots as soon as a slot is free: continuous batching at the request level.
// Every mesh owns one resident persistent system (pattern, hierarchy, device copies of the last
// matrix / right-hand side / solution, its own CUDA stream), so requests on different meshes run
// concurrently and overlap on the GPU; requests on one mesh are serialised on its system.
// Residency is bounded by an HBM budget: a system is admitted only when its (estimated, then
// measured) device footprint fits next to the resident ones, evicting idle systems in
// least-recently-used order; requests that do not fit wait in the queue until memory frees up.
// Hierarchies age as the reference's AmgCache does (rebuilt after max_age solves); with
// background_rebuild a rebuild thread builds the new one on a spare system from a copy of the
// triggering request's matrix while the mesh keeps serving with the old one.
#include "../../include/cfdb_serve.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "common.hpp"

namespace cfdb {
void set_thread_error(const std::string& msg); // capi.cu
}

using cfdb::fail;

namespace {

using Clock = std::chrono::steady_clock;

struct Mesh {
    int n = 0, nf = 0;
    std::vector<int> owner, neighbour;
};

// State of a mesh's background hierarchy rebuild (cfg.background_rebuild), guarded by the
// server lock: queued for the rebuild thread, being built on the spare system, or ready to be
// swapped in by the next request on the mesh.
enum class Rebuild { Idle, Queued, Building, Ready };

struct Resident {
    cfdb_system* sys = nullptr;
    size_t bytes = 0;
    double *d_diag = nullptr, *d_upper = nullptr, *d_lower = nullptr, *d_rhs = nullptr, *d_x = nullptr;
    long long matrix_key = -1;   // key of the LDU values on the device
    long long solution_key = -1; // key of the matrix the device solution belongs to
    long long hier_key = -1;     // key of the matrix the hierarchy was built from
    int age = 0;                 // solves since the hierarchy was built
    bool busy = false;
    Clock::time_point last_use{};
    // background rebuild: a second system on the same mesh builds the new hierarchy from device
    // copies of the triggering request's matrix while `sys` keeps serving; the two are swapped
    // by the next request on the mesh once the build is done
    cfdb_system* spare = nullptr;
    double *s_diag = nullptr, *s_upper = nullptr, *s_lower = nullptr;
    cudaEvent_t copied = nullptr; // the copies of the matrix are complete
    long long spare_key = -1;     // key of the matrix the spare's hierarchy is built from
    Rebuild rebuild = Rebuild::Idle;
    bool background_failed = false; // a background build failed: rebuild on the request path
};

struct Request {
    long long ticket = 0;
    int mesh = 0;
    long long key = 0;
    bool warm = false;
    double rel_tol = 1e-8;
    int max_iter = 500;
    // borrowed from the caller until the ticket is waited for
    const double *diag = nullptr, *upper = nullptr, *lower = nullptr, *rhs = nullptr;
    double* x = nullptr;
    Clock::time_point submitted{}, started{}, finished{};
    cfdb_stats stats{};
    int status = CFDB_OK;
    std::string error;
    bool done = false;
};

} // namespace

struct cfdb_server {
    cfdb_server_config cfg{};
    int device = 0;
    Clock::time_point t0{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stopping = false;
    std::deque<Mesh> meshes; // stable element addresses while meshes are added
    std::unordered_map<int, std::unique_ptr<Resident>> resident;
    size_t resident_bytes = 0;
    std::deque<std::shared_ptr<Request>> queue;
    std::map<long long, std::shared_ptr<Request>> tickets;
    long long next_ticket = 1;
    std::vector<std::thread> workers;
    long long completed = 0;
    long long evictions = 0;
    long long rebuilds = 0;            // hierarchy rebuilds on the request path
    long long background_rebuilds = 0; // hierarchies built by the rebuild thread and swapped in
    std::deque<int> rebuild_queue;     // meshes whose spare system is to be rebuilt
    std::condition_variable cv_rebuild;
    std::thread rebuilder;
};

namespace {

size_t estimate_bytes(const cfdb_server& s, const Mesh& m) {
    // measured footprint of the persistent systems: about 800 bytes per cell (hierarchy, SELL
    // copies, Krylov vectors) plus the server's device copies of one matrix and three vectors;
    // with background rebuilds, a spare system and a second copy of the matrix
    const size_t per_cell = s.cfg.precision == CFDB_PRECISION_MIXED ? 700 : 800;
    const size_t matrix = sizeof(double) * (static_cast<size_t>(m.n) + 2 * static_cast<size_t>(m.nf));
    const size_t one = per_cell * static_cast<size_t>(m.n) + matrix + sizeof(double) * 3 * static_cast<size_t>(m.n);
    return s.cfg.background_rebuild ? one + per_cell * static_cast<size_t>(m.n) + matrix : one;
}

void release(cfdb_server& s, Resident& r) {
    if (r.sys != nullptr) cfdb_system_destroy(r.sys);
    if (r.spare != nullptr) cfdb_system_destroy(r.spare);
    for (double* p : {r.d_diag, r.d_upper, r.d_lower, r.d_rhs, r.d_x, r.s_diag, r.s_upper, r.s_lower})
        if (p != nullptr) cudaFree(p);
    if (r.copied != nullptr) cudaEventDestroy(r.copied);
    s.resident_bytes -= std::min(s.resident_bytes, r.bytes);
    r = Resident{};
}

// Frees idle resident systems (least recently used first) until `need` more bytes fit.
// Called with the lock held. Returns whether the request fits now.
bool make_room(cfdb_server& s, size_t need, int keep_mesh) {
    const size_t budget = static_cast<size_t>(s.cfg.hbm_budget_bytes);
    while (s.resident_bytes + need > budget) {
        int victim = -1;
        Clock::time_point oldest = Clock::time_point::max();
        for (auto& kv : s.resident) {
            const Resident& c = *kv.second;
            const bool rebuilding = c.rebuild == Rebuild::Queued || c.rebuild == Rebuild::Building;
            if (kv.first == keep_mesh || c.busy || rebuilding || c.sys == nullptr) continue;
            if (kv.second->last_use < oldest) {
                oldest = kv.second->last_use;
                victim = kv.first;
            }
        }
        if (victim < 0) return false;
        release(s, *s.resident[victim]);
        s.resident.erase(victim);
        ++s.evictions;
        cfdb_release_cached_memory(); // the evicted system's blocks go back to the driver
    }
    return true;
}

void check(int rc) {
    if (rc != CFDB_OK) {
        char buf[1024];
        cfdb_last_error(buf, sizeof(buf));
        throw cfdb::Error(rc, buf);
    }
}

void dmalloc(double** p, size_t n) {
    const cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), sizeof(double) * std::max<size_t>(n, 1));
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        fail(CFDB_ERR_OOM, std::string("server: device allocation failed: ") + cudaGetErrorString(e));
    }
}

// A persistent system on the mesh with the server's precision, plan and tuning.
cfdb_system* new_system(const cfdb_server& s, const Mesh& m) {
    cfdb_system* sys = nullptr;
    check(cfdb_system_create_mesh(m.n, m.nf, m.owner.data(), m.neighbour.data(), &sys));
    try {
        check(cfdb_system_set_precision(sys, s.cfg.precision));
        check(cfdb_system_set_keep_levels(sys, 0)); // the plan of a resident system never changes
        cfdb_tuning tun;
        cfdb_default_tuning(&tun);
        tun.pdl = s.cfg.pdl;
        tun.mixed_sweeps = s.cfg.mixed_sweeps;
        tun.mixed_weight = s.cfg.mixed_weight;
        check(cfdb_system_set_tuning(sys, &tun));
    } catch (...) {
        cfdb_system_destroy(sys);
        throw;
    }
    return sys;
}

enum ExecuteOutcome { kRebuiltInline = 1, kQueueRebuild = 2 };

// Runs one request on its (locked) resident system. No server lock held. may_queue: the
// resident has no background rebuild in progress or waiting. Returns ExecuteOutcome bits.
int execute(cfdb_server& s, Resident& r, const Mesh& m, Request& q, bool created, bool may_queue) {
    cudaSetDevice(s.device);
    int outcome = 0;
    if (created) {
        r.sys = new_system(s, m);
        dmalloc(&r.d_diag, m.n);
        dmalloc(&r.d_upper, m.nf);
        dmalloc(&r.d_lower, m.nf);
        dmalloc(&r.d_rhs, m.n);
        dmalloc(&r.d_x, m.n);
    }
    void* stream_v = nullptr;
    check(cfdb_system_stream(r.sys, &stream_v));
    cudaStream_t st = static_cast<cudaStream_t>(stream_v);
    const bool new_matrix = r.matrix_key != q.key || q.key < 0;
    if (new_matrix) {
        CFDB_CUDA(cudaMemcpyAsync(r.d_diag, q.diag, sizeof(double) * m.n, cudaMemcpyHostToDevice, st));
        if (m.nf > 0) {
            CFDB_CUDA(cudaMemcpyAsync(r.d_upper, q.upper, sizeof(double) * m.nf, cudaMemcpyHostToDevice, st));
            CFDB_CUDA(cudaMemcpyAsync(r.d_lower, q.lower, sizeof(double) * m.nf, cudaMemcpyHostToDevice, st));
        }
        r.matrix_key = q.key;
    }
    // hierarchy (re)build from this request's matrix (already on the device), as the
    // reference's AmgCache does after max_age solves, with the sparse algebra on the GPU; when the
    // request's matrix is the one the hierarchy was built from, the rebuild would reproduce it bit
    // for bit, so it waits for the next new matrix
    const bool same_as_hierarchy = q.key >= 0 && r.hier_key == q.key;
    const bool aged = s.cfg.max_age > 0 && r.age >= s.cfg.max_age && !same_as_hierarchy;
    const bool background = s.cfg.background_rebuild != 0 && !r.background_failed;
    if (created || (aged && !background)) {
        CFDB_CUDA(cudaStreamSynchronize(st));
        check(cfdb_system_setup_amg_device(r.sys, r.d_diag, r.d_upper, r.d_lower, &s.cfg.settings, 1));
        r.age = 0;
        r.hier_key = q.key;
        if (!created) outcome |= kRebuiltInline;
    } else if (aged && may_queue) {
        // the rebuild thread builds the spare system's hierarchy from copies of this matrix
        // (the next request on the mesh may overwrite d_diag / d_upper / d_lower); this
        // request and the ones after it solve with the current hierarchy until the swap
        if (r.s_diag == nullptr) {
            dmalloc(&r.s_diag, m.n);
            dmalloc(&r.s_upper, m.nf);
            dmalloc(&r.s_lower, m.nf);
            CFDB_CUDA(cudaEventCreateWithFlags(&r.copied, cudaEventDisableTiming));
        }
        CFDB_CUDA(cudaMemcpyAsync(r.s_diag, r.d_diag, sizeof(double) * m.n, cudaMemcpyDeviceToDevice, st));
        if (m.nf > 0) {
            CFDB_CUDA(cudaMemcpyAsync(r.s_upper, r.d_upper, sizeof(double) * m.nf, cudaMemcpyDeviceToDevice, st));
            CFDB_CUDA(cudaMemcpyAsync(r.s_lower, r.d_lower, sizeof(double) * m.nf, cudaMemcpyDeviceToDevice, st));
        }
        CFDB_CUDA(cudaEventRecord(r.copied, st));
        r.spare_key = q.key;
        outcome |= kQueueRebuild;
    }
    CFDB_CUDA(cudaMemcpyAsync(r.d_rhs, q.rhs, sizeof(double) * m.n, cudaMemcpyHostToDevice, st));
    if (!(q.warm && r.solution_key == q.key && q.key >= 0)) {
        CFDB_CUDA(cudaMemsetAsync(r.d_x, 0, sizeof(double) * m.n, st));
    }
    double bn = 0.0;
    for (int i = 0; i < m.n; ++i) bn += q.rhs[i] * q.rhs[i];
    const cfdb_control ctl{q.rel_tol * std::sqrt(bn), q.max_iter};
    check(cfdb_system_solve_device(r.sys, r.d_diag, r.d_upper, r.d_lower, r.d_rhs, r.d_x, CFDB_METHOD_CG, 1, &ctl,
                                   &q.stats));
    r.solution_key = q.key;
    ++r.age;
    if (q.x != nullptr) CFDB_CUDA(cudaMemcpyAsync(q.x, r.d_x, sizeof(double) * m.n, cudaMemcpyDeviceToHost, st));
    CFDB_CUDA(cudaStreamSynchronize(st));
    return outcome;
}

// The background rebuild thread: builds queued meshes' spare hierarchies one at a time on the
// spare system's own stream, while the workers keep solving with the current ones.
void rebuild_loop(cfdb_server* sp) {
    cfdb_server& s = *sp;
    cudaSetDevice(s.device);
    std::unique_lock<std::mutex> lk(s.mu);
    for (;;) {
        s.cv_rebuild.wait(lk, [&] { return s.stopping || !s.rebuild_queue.empty(); });
        if (s.stopping) {
            for (int id : s.rebuild_queue) {
                auto it = s.resident.find(id);
                if (it != s.resident.end()) it->second->rebuild = Rebuild::Idle;
            }
            s.rebuild_queue.clear();
            return;
        }
        const int mesh = s.rebuild_queue.front();
        s.rebuild_queue.pop_front();
        auto it = s.resident.find(mesh);
        if (it == s.resident.end()) continue; // queued residents are never evicted; defensive
        Resident& r = *it->second;
        r.rebuild = Rebuild::Building;
        const Mesh& m = s.meshes[mesh];
        const bool first = r.spare == nullptr;
        lk.unlock();
        bool ok = true;
        size_t spare_bytes = 0;
        try {
            // while Building, only this thread touches the spare system and its matrix copies
            if (first) r.spare = new_system(s, m);
            CFDB_CUDA(cudaEventSynchronize(r.copied));
            check(cfdb_system_setup_amg_device(r.spare, r.s_diag, r.s_upper, r.s_lower, &s.cfg.settings, 1));
            if (first) {
                cfdb_system_device_bytes(r.spare, &spare_bytes);
                spare_bytes += sizeof(double) * (static_cast<size_t>(m.n) + 2 * static_cast<size_t>(m.nf));
            }
        } catch (const std::exception&) {
            ok = false;
        }
        lk.lock();
        r.bytes += spare_bytes;
        s.resident_bytes += spare_bytes;
        r.rebuild = ok ? Rebuild::Ready : Rebuild::Idle;
        if (!ok) r.background_failed = true;
        s.cv_work.notify_all();
    }
}

void worker_loop(cfdb_server* sp) {
    cfdb_server& s = *sp;
    cudaSetDevice(s.device);
    std::unique_lock<std::mutex> lk(s.mu);
    for (;;) {
        // the first queued request whose mesh is idle and whose system is resident or fits;
        // with the most-work-first policy, the meshes' first queued requests are tried in
        // order of the cells queued on each mesh (ties: queue order), so that at saturation
        // the long per-mesh chains start first and the run does not end on one of them
        std::shared_ptr<Request> q;
        Resident* r = nullptr;
        bool created = false;
        using QueueIt = std::deque<std::shared_ptr<Request>>::iterator;
        std::vector<QueueIt> order;
        for (;;) {
            if (s.stopping && s.queue.empty()) return;
            order.clear();
            if (s.cfg.schedule == CFDB_SCHEDULE_MOST_WORK) {
                std::unordered_map<int, std::pair<double, QueueIt>> per_mesh;
                for (auto it = s.queue.begin(); it != s.queue.end(); ++it) {
                    auto ins = per_mesh.try_emplace((*it)->mesh, 0.0, it);
                    ins.first->second.first += static_cast<double>(s.meshes[(*it)->mesh].n);
                }
                std::vector<std::pair<double, QueueIt>> by_work;
                by_work.reserve(per_mesh.size());
                for (auto& kv : per_mesh) by_work.push_back(kv.second);
                std::sort(by_work.begin(), by_work.end(), [](const auto& a, const auto& b) {
                    return a.first != b.first ? a.first > b.first : (*a.second)->ticket < (*b.second)->ticket;
                });
                for (auto& w : by_work) order.push_back(w.second);
            } else {
                for (auto it = s.queue.begin(); it != s.queue.end(); ++it) order.push_back(it);
            }
            for (QueueIt it : order) {
                auto& cand = *it;
                auto rit = s.resident.find(cand->mesh);
                if (rit != s.resident.end()) {
                    if (rit->second->busy) continue;
                    r = rit->second.get();
                    created = r->sys == nullptr;
                } else {
                    const size_t need = estimate_bytes(s, s.meshes[cand->mesh]);
                    if (!make_room(s, need, cand->mesh)) continue;
                    auto res = std::make_unique<Resident>();
                    res->bytes = need;
                    s.resident_bytes += need;
                    r = res.get();
                    s.resident[cand->mesh] = std::move(res);
                    created = true;
                }
                q = cand;
                s.queue.erase(it);
                break;
            }
            if (q) break;
            s.cv_work.wait(lk);
        }
        r->busy = true;
        if (r->rebuild == Rebuild::Ready) {
            // the background build is done: its hierarchy serves from this request on
            std::swap(r->sys, r->spare);
            r->hier_key = r->spare_key;
            r->age = 0;
            r->rebuild = Rebuild::Idle;
            ++s.background_rebuilds;
        }
        const bool may_queue = r->rebuild == Rebuild::Idle;
        q->started = Clock::now();
        lk.unlock();
        int outcome = 0;
        try {
            outcome = execute(s, *r, s.meshes[q->mesh], *q, created, may_queue);
        } catch (const cfdb::Error& e) {
            q->status = e.code;
            q->error = e.what();
        } catch (const std::exception& e) {
            q->status = CFDB_ERR_INTERNAL;
            q->error = e.what();
        }
        q->finished = Clock::now();
        lk.lock();
        if (outcome & kRebuiltInline) ++s.rebuilds;
        if ((outcome & kQueueRebuild) && q->status == CFDB_OK) {
            r->rebuild = Rebuild::Queued;
            s.rebuild_queue.push_back(q->mesh);
            s.cv_rebuild.notify_one();
        }
        if (created && r->sys != nullptr) {
            size_t b = 0;
            cfdb_system_device_bytes(r->sys, &b);
            const size_t actual = b + sizeof(double) * (3 * static_cast<size_t>(s.meshes[q->mesh].n) +
                                                        2 * static_cast<size_t>(s.meshes[q->mesh].nf));
            s.resident_bytes = s.resident_bytes - std::min(s.resident_bytes, r->bytes) + actual;
            r->bytes = actual;
        }
        if (q->status != CFDB_OK && r->sys == nullptr) {
            s.resident_bytes -= std::min(s.resident_bytes, r->bytes);
            s.resident.erase(q->mesh);
        } else {
            r->busy = false;
            r->last_use = Clock::now();
        }
        q->done = true;
        ++s.completed;
        s.cv_done.notify_all();
        s.cv_work.notify_all();
    }
}

template <class F> int guarded_s(F&& f) {
    try {
        f();
        return CFDB_OK;
    } catch (const cfdb::Error& e) {
        cfdb::set_thread_error(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        cfdb::set_thread_error("host allocation failed");
        return CFDB_ERR_OOM;
    } catch (const std::exception& e) {
        cfdb::set_thread_error(e.what());
        return CFDB_ERR_INTERNAL;
    }
}

double seconds(const cfdb_server& s, Clock::time_point t) {
    return std::chrono::duration<double>(t - s.t0).count();
}

} // namespace

extern "C" {

void cfdb_default_server_config(cfdb_server_config* c) {
    if (c == nullptr) return;
    c->slots = 4;
    c->hbm_budget_bytes = 150e9;
    c->precision = CFDB_PRECISION_MIXED;
    cfdb_default_amg_settings(&c->settings);
    c->max_age = 0;
    c->pdl = 0;
    c->mixed_sweeps = 0;
    c->mixed_weight = 0.0;
    c->background_rebuild = 0;
    c->schedule = CFDB_SCHEDULE_FIFO;
}

int cfdb_server_create(const cfdb_server_config* cfg, cfdb_server** out) {
    return guarded_s([&] {
        if (cfg == nullptr || out == nullptr) fail(CFDB_ERR_BAD_ARG, "null argument");
        if (cfg->slots < 1 || cfg->slots > 64) fail(CFDB_ERR_BAD_ARG, "slots must be in 1..64");
        if (cfg->schedule != CFDB_SCHEDULE_FIFO && cfg->schedule != CFDB_SCHEDULE_MOST_WORK)
            fail(CFDB_ERR_BAD_ARG, "unknown schedule");
        if (!(cfg->hbm_budget_bytes > 0)) fail(CFDB_ERR_BAD_ARG, "HBM budget must be positive");
        if (!cfdb_device_available()) fail(CFDB_ERR_NO_DEVICE, "no CUDA device: this library has no host fallback");
        auto s = std::make_unique<cfdb_server>();
        s->cfg = *cfg;
        CFDB_CUDA(cudaGetDevice(&s->device));
        s->t0 = Clock::now();
        for (int i = 0; i < cfg->slots; ++i) s->workers.emplace_back(worker_loop, s.get());
        if (cfg->background_rebuild) s->rebuilder = std::thread(rebuild_loop, s.get());
        *out = s.release();
    });
}

int cfdb_server_destroy(cfdb_server* s) {
    if (s == nullptr) return CFDB_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
    }
    s->cv_work.notify_all();
    for (auto& t : s->workers) t.join();
    s->cv_rebuild.notify_all();
    if (s->rebuilder.joinable()) s->rebuilder.join();
    cudaSetDevice(s->device);
    for (auto& kv : s->resident) release(*s, *kv.second);
    delete s;
    return CFDB_OK;
}

int cfdb_server_add_mesh(cfdb_server* s, int n_cells, int n_faces, const int* owner, const int* neighbour, int* mesh_id) {
    return guarded_s([&] {
        if (s == nullptr || mesh_id == nullptr || n_cells <= 0 || n_faces < 0 || (n_faces > 0 && (!owner || !neighbour)))
            fail(CFDB_ERR_BAD_ARG, "cfdb_server_add_mesh: bad arguments");
        for (int f = 0; f < n_faces; ++f)
            if (owner[f] < 0 || owner[f] >= n_cells || neighbour[f] < 0 || neighbour[f] >= n_cells)
                fail(CFDB_ERR_BAD_ARG, "cfdb_server_add_mesh: face addresses a cell out of range");
        Mesh m;
        m.n = n_cells;
        m.nf = n_faces;
        m.owner.assign(owner, owner + n_faces);
        m.neighbour.assign(neighbour, neighbour + n_faces);
        std::lock_guard<std::mutex> lk(s->mu);
        s->meshes.push_back(std::move(m));
        *mesh_id = static_cast<int>(s->meshes.size()) - 1;
    });
}

int cfdb_server_submit(cfdb_server* s, int mesh_id, long long matrix_key, const double* diag, const double* upper,
                       const double* lower, const double* rhs, double* x, int warm_start, double rel_tol,
                       int max_iterations, long long* ticket) {
    return guarded_s([&] {
        if (s == nullptr || ticket == nullptr || !diag || !rhs) fail(CFDB_ERR_BAD_ARG, "cfdb_server_submit: null argument");
        auto q = std::make_shared<Request>();
        q->submitted = Clock::now();
        const Mesh* mp = nullptr;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (mesh_id < 0 || mesh_id >= static_cast<int>(s->meshes.size())) fail(CFDB_ERR_BAD_ARG, "unknown mesh");
            mp = &s->meshes[mesh_id];
        }
        const Mesh& m = *mp;
        if (m.nf > 0 && (!upper || !lower)) fail(CFDB_ERR_BAD_ARG, "cfdb_server_submit: null face coefficients");
        if (!(rel_tol > 0.0) || max_iterations < 0) fail(CFDB_ERR_BAD_ARG, "cfdb_server_submit: bad tolerance");
        q->mesh = mesh_id;
        q->key = matrix_key;
        q->warm = warm_start != 0;
        q->rel_tol = rel_tol;
        q->max_iter = max_iterations;
        q->diag = diag;
        q->upper = upper;
        q->lower = lower;
        q->rhs = rhs;
        q->x = x;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (s->stopping) fail(CFDB_ERR_BAD_ARG, "server is stopping");
            if (estimate_bytes(*s, m) > static_cast<size_t>(s->cfg.hbm_budget_bytes))
                fail(CFDB_ERR_OOM, "request can never fit the server's HBM budget");
            q->ticket = s->next_ticket++;
            s->tickets[q->ticket] = q;
            s->queue.push_back(q);
            *ticket = q->ticket;
        }
        s->cv_work.notify_one();
    });
}

int cfdb_server_wait(cfdb_server* s, long long ticket, cfdb_stats* stats, double* times) {
    return guarded_s([&] {
        if (s == nullptr) fail(CFDB_ERR_BAD_ARG, "null server");
        std::shared_ptr<Request> q;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            auto it = s->tickets.find(ticket);
            if (it == s->tickets.end()) fail(CFDB_ERR_BAD_ARG, "unknown ticket");
            q = it->second;
            s->cv_done.wait(lk, [&] { return q->done; });
            s->tickets.erase(it);
        }
        if (times != nullptr) {
            times[0] = seconds(*s, q->submitted);
            times[1] = seconds(*s, q->started);
            times[2] = seconds(*s, q->finished);
        }
        if (q->status != CFDB_OK) fail(q->status, q->error);
        if (stats != nullptr) *stats = q->stats;
    });
}

int cfdb_server_info(cfdb_server* s, cfdb_server_info_t* info) {
    if (s == nullptr || info == nullptr) return CFDB_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    info->resident_systems = static_cast<int>(s->resident.size());
    info->resident_bytes = static_cast<double>(s->resident_bytes);
    info->queued = static_cast<int>(s->queue.size());
    info->completed = s->completed;
    info->evictions = s->evictions;
    info->rebuilds = s->rebuilds;
    info->background_rebuilds = s->background_rebuilds;
    return CFDB_OK;
}

} // extern "C"
