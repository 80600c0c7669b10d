// Smoothed-aggregation AMG setup on the device (fv::AmgPreconditioner::setup, amg.cpp:122-190).
//
// The sparse algebra of every level (strength graph, tentative and smoothed prolongation,
// restriction, Galerkin products, zero pruning) runs in device kernels. The aggregation
// (amg.cpp:12-78) is a sequence of greedy passes whose result depends on the visiting order:
// passes 1 and 2 run on the device with the sequential result (pass 1 as the lexicographically
// first independent set it is, resolved by sweeps); a level that leaves rows for pass 3 is
// aggregated on the host from its strength graph. Every product and
// sum is rounded in the order the host build (amg_setup, host_algos.cpp) uses, so the device
// hierarchy is bit-identical to it: aggregates, P, R, coarse operators and coarse inverse.
#pragma once

#include <chrono>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "common.hpp"
#include "host_algos.hpp"

namespace cfdb {

// Bump allocator over device chunks that grow geometrically; everything is released at once.
class Scratch {
public:
    template <class T> T* alloc(size_t count) {
        return static_cast<T*>(raw(sizeof(T) * (count > 0 ? count : 1)));
    }
    [[nodiscard]] size_t bytes() const { return total_; }

private:
    void* raw(size_t bytes);
    struct Chunk {
        DeviceBuffer buf;
        size_t used = 0;
    };
    std::vector<Chunk> chunks_;
    size_t total_ = 0;
};

// Wall-clock seconds of named setup phases, accumulated over levels, in first-use order.
struct PhaseTimes {
    std::vector<std::pair<std::string, double>> t;
    void add(const std::string& name, double seconds) {
        for (auto& p : t) {
            if (p.first == name) {
                p.second += seconds;
                return;
            }
        }
        t.emplace_back(name, seconds);
    }
    // "name=seconds;name=seconds"
    [[nodiscard]] std::string text() const {
        std::string s;
        for (const auto& p : t) {
            if (!s.empty()) s += ';';
            s += p.first + '=' + std::to_string(p.second);
        }
        return s;
    }
    static double now() {
        return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
    }
};

// CSR matrix in device memory (sorted, unique columns per row).
struct DevCsr {
    int n_rows = 0;
    int n_cols = 0;
    int nnz = 0;
    int* rp = nullptr;
    int* ci = nullptr;
    double* va = nullptr;
};

// Hierarchy with device-resident levels. a[0] is the input; the arrays live in `mem`.
struct DeviceHierarchy {
    Scratch mem;
    std::vector<DevCsr> a, p, r;
    // aggregates of each non-coarsest level on the device (in mem); the host copy `agg` is kept
    // where the host aggregated, and made by download_hierarchy elsewhere
    std::vector<const int*> dagg;
    std::vector<std::vector<int>> agg;
    std::vector<int> n_agg;
    int n_c = 0;
    bool ldlt_ok = false;
    std::vector<double> coarse_inverse;
    PhaseTimes times;
    [[nodiscard]] int levels() const { return static_cast<int>(a.size()); }
};

// Builds the hierarchy of a0 (device CSR, already in h.mem or caller-owned and alive for the
// call) with settings s on stream st. Synchronises st. stage: page-locked staging of the
// strength graphs read back for aggregation (null: a temporary one).
// keep: where the hierarchy's own arrays (P_l, R_l, A_l for l >= 1) are allocated, so that a
// caller can hold them after h's scratch is released (null: in h.mem).
void amg_setup_device(const DevCsr& a0, const AmgSettings& s, cudaStream_t st, DeviceHierarchy& h,
                      PinnedBuffer* stage = nullptr, DeviceArena* keep = nullptr);

// Host copy of a device hierarchy; level 0's matrix is copied only when with_a0.
Hierarchy download_hierarchy(const DeviceHierarchy& d, bool with_a0, cudaStream_t st);

// The levels a device plan is built from (A_l for l >= 1, P_l, R_l), allocated by the setup
// in their own arena (amg_setup_device's `keep`) and kept with the system, so that the plan can
// be rebuilt (precision or tuning changes) without the host.
struct DeviceLevels {
    DeviceArena mem;
    std::vector<DevCsr> a, p, r; // a[0] is empty (level 0 comes from the system's pattern)
    [[nodiscard]] size_t bytes() const { return mem.bytes(); }
};
// Points k's level views at the arrays of d (which the setup allocated in k.mem).
void adopt_levels(const DeviceHierarchy& d, DeviceLevels& k);

// Shape-only host copy of a device hierarchy (sizes, coarse inverse, and the aggregates of the
// levels the host aggregated; matrix arrays and the device-aggregated levels' aggregates empty)
// for plan construction from the device levels.
Hierarchy hierarchy_shape(const DeviceHierarchy& d);

// ---- engine operator layouts built from a device CSR block (one system, column offset 0) ----
// out[0..n_pad] = rp, then the padding rows' (empty) offsets.
void csr_rows_padded(const DevCsr& m, int n_pad, int* out, cudaStream_t st);
// col / values copied with four zero slack entries after the last (nnz + 4 each); v64 / v32
// optional.
void csr_copy_values(const DevCsr& m, int* col, double* v64, float* v32, cudaStream_t st);
// SELL-32 shape: rows reordered by length (stable, longest first) within aligned windows of
// `window` positions; perm (n_pad) = row at each position; slice (n_pad / 32 + 1) = slot
// offsets. Returns the slot count.
long long sell_shape(const DevCsr& m, int n_pad, int window, int* perm, int* slice, cudaStream_t st);
// SELL-32 fill: slot slice[s] + k*32 + lane holds entry k of the row at position 32 s + lane;
// other slots read column pad_col with value 0. v64 / v32 optional.
void sell_fill(const DevCsr& m, int n_pad, const int* perm, const int* slice, int pad_col, int* col, double* v64,
               float* v32, cudaStream_t st);
// wd[i] = weight * (1 / last nonzero diagonal entry of row i, or 1 if none) for rows below
// m.n_rows, weight on the padding rows up to n_pad; wd32 = (float) wd. Either output optional.
void weighted_inverse_diagonal(const DevCsr& m, int n_pad, double weight, double* wd64, float* wd32, cudaStream_t st);

// Level-0 CSR values from LDU coefficients (device arrays): va[diag_pos[i]] = diag[i],
// va[upper_pos[f]] = upper[f], va[lower_pos[f]] = lower[f].
void ldu_to_csr_values(int n, int nf, const int* diag_pos, const int* upper_pos, const int* lower_pos,
                       const double* diag, const double* upper, const double* lower, double* va,
                       cudaStream_t st);

} // namespace cfdb
