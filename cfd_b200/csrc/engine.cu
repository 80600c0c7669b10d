#include "engine.hpp"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <cstdio>
#include <numeric>

namespace cfdb {

namespace {


// SELL-32 under construction on the host.
struct SellBuild {
    std::vector<int> slice{0};
    std::vector<int> col;
    std::vector<double> val;
    std::vector<int> src;
    bool with_src = false;
    bool sort = false;      // reorder rows by length within aligned windows of kSellRows
    std::vector<int> perm;  // row at each position (when sort)
    std::vector<char> pad;  // 1 for padding slots
};

// 16-bit column offsets of the groups [ptr[g], ptr[g+1]) of `col` (SELL slices or CSR rows):
// base[g] = smallest real column of the group, c16[k] = col[k] - base[g]; padding entries
// (pad[k] != 0) and entries outside every group get offset 0. False when some group spans
// 65536 columns or more (the operator then keeps int32 columns).
bool compress_cols(const std::vector<int>& ptr, const std::vector<int>& col, const std::vector<char>* pad,
                   std::vector<uint16_t>& c16, std::vector<int>& base) {
    const long long ng = static_cast<long long>(ptr.size()) - 1;
    c16.assign(col.size(), 0);
    base.assign(static_cast<size_t>(std::max(ng, 1LL)), 0);
    int ok = 1;
#pragma omp parallel for schedule(static) reduction(&& : ok)
    for (long long g = 0; g < ng; ++g) {
        int lo = INT_MAX, hi = INT_MIN;
        for (int k = ptr[g]; k < ptr[g + 1]; ++k) {
            if (pad != nullptr && (*pad)[k]) continue;
            lo = std::min(lo, col[k]);
            hi = std::max(hi, col[k]);
        }
        if (lo > hi) continue;  // padding only
        if (static_cast<long long>(hi) - lo > 65535) {
            ok = 0;
            continue;
        }
        base[g] = lo;
        for (int k = ptr[g]; k < ptr[g + 1]; ++k) {
            if (pad != nullptr && (*pad)[k]) continue;
            c16[k] = static_cast<uint16_t>(col[k] - lo);
        }
    }
    return ok != 0;
}

// Appends rows [0, n_rows) of a CSR block (n_pad >= n_rows, multiple of 32) whose first row has
// global index row0. Column indices are shifted by col_off; padding slots read column pad_col
// with value 0. src_of (optional): value-source index per CSR entry (shifted by src_off).
// Slices are laid out serially (a prefix sum of their widths) and filled in parallel.
void sell_append(SellBuild& sb, int n_rows, int n_pad, const int* rp, const int* ci,
                 const double* va, const int* src_of, int col_off, int src_off, int pad_col) {
    // order[q]: block row at block position q (identity unless sorting)
    std::vector<int> order(static_cast<size_t>(n_pad));
    std::iota(order.begin(), order.end(), 0);
    auto len_of = [&](int i) { return i < n_rows ? rp[i + 1] - rp[i] : -1; };
    if (sb.sort) {
#pragma omp parallel for schedule(dynamic, 16) if (n_pad > 65536)
        for (int w0 = 0; w0 < n_pad; w0 += kSellRows) {
            const int w1 = std::min(n_pad, w0 + kSellRows);
            std::stable_sort(order.begin() + w0, order.begin() + w1,
                             [&](int a, int b) { return len_of(a) > len_of(b); });
        }
        const int row0 = static_cast<int>(sb.perm.size());
        sb.perm.resize(static_cast<size_t>(row0) + n_pad);
        for (int q = 0; q < n_pad; ++q) sb.perm[static_cast<size_t>(row0) + q] = row0 + order[q];
    }
    const int n_sl = n_pad / 32;
    std::vector<long long> start(static_cast<size_t>(n_sl) + 1, 0);
    const long long base0 = sb.slice.back();
    start[0] = base0;
    {
        std::vector<int> width(static_cast<size_t>(n_sl), 0);
#pragma omp parallel for schedule(static) if (n_sl > 4096)
        for (int sl = 0; sl < n_sl; ++sl) {
            int w = 0;
            for (int q = sl * 32; q < sl * 32 + 32; ++q) w = std::max(w, len_of(order[q]));
            width[sl] = w;
        }
        for (int sl = 0; sl < n_sl; ++sl) start[sl + 1] = start[sl] + 32LL * width[sl];
    }
    const long long total = start[n_sl];
    if (total > INT_MAX) fail(1, "operator too large for 32-bit slot offsets");
    sb.col.resize(static_cast<size_t>(total), pad_col);
    sb.val.resize(static_cast<size_t>(total), 0.0);
    sb.pad.resize(static_cast<size_t>(total), 1);
    if (sb.with_src) sb.src.resize(static_cast<size_t>(total), -1);
#pragma omp parallel for schedule(static) if (n_sl > 4096)
    for (int sl = 0; sl < n_sl; ++sl) {
        const long long base = start[sl];
        for (int lane = 0; lane < 32; ++lane) {
            const int i = order[sl * 32 + lane];
            if (i >= n_rows) continue;
            const int len = rp[i + 1] - rp[i];
            for (int k = 0; k < len; ++k) {
                const size_t slot = static_cast<size_t>(base + static_cast<long long>(k) * 32 + lane);
                const int e = rp[i] + k;
                sb.pad[slot] = 0;
                sb.col[slot] = ci[e] + col_off;
                sb.val[slot] = va != nullptr ? va[e] : 0.0;
                if (sb.with_src) sb.src[slot] = src_of != nullptr ? src_of[e] + src_off : -1;
            }
        }
    }
    const size_t s0 = sb.slice.size();
    sb.slice.resize(s0 + n_sl);
    for (int sl = 0; sl < n_sl; ++sl) sb.slice[s0 + sl] = static_cast<int>(start[sl + 1]);
}

// One CSR block of a multi-system operator (the arguments of sell_append / csr_append).
struct BlockSpec {
    int n_rows = 0, n_pad = 0;
    const int* rp = nullptr;
    const int* ci = nullptr;
    const double* va = nullptr;
    const int* src_of = nullptr;
    int col_off = 0, src_off = 0, pad_col = 0;
};

// sell_append over many blocks in order, with the same result as appending them one after
// another: the blocks' row orders and slice widths are worked out in parallel (one block per
// thread), the slot offsets follow from a prefix sum over the blocks, and the blocks are then
// filled in parallel. A single block goes through sell_append and its own inner parallelism.
void sell_append_blocks(SellBuild& sb, const std::vector<BlockSpec>& blocks) {
    const int nb = static_cast<int>(blocks.size());
    if (nb == 1) {
        const BlockSpec& b = blocks[0];
        sell_append(sb, b.n_rows, b.n_pad, b.rp, b.ci, b.va, b.src_of, b.col_off, b.src_off, b.pad_col);
        return;
    }
    std::vector<std::vector<int>> order(static_cast<size_t>(nb)), width(static_cast<size_t>(nb));
    std::vector<long long> slots(static_cast<size_t>(nb) + 1, 0), rows(static_cast<size_t>(nb) + 1, 0),
        slices(static_cast<size_t>(nb) + 1, 0);
#pragma omp parallel for schedule(dynamic, 1)
    for (int bi = 0; bi < nb; ++bi) {
        const BlockSpec& b = blocks[static_cast<size_t>(bi)];
        auto len_of = [&](int i) { return i < b.n_rows ? b.rp[i + 1] - b.rp[i] : -1; };
        std::vector<int>& o = order[static_cast<size_t>(bi)];
        o.resize(static_cast<size_t>(b.n_pad));
        std::iota(o.begin(), o.end(), 0);
        if (sb.sort) {
            for (int w0 = 0; w0 < b.n_pad; w0 += kSellRows) {
                const int w1 = std::min(b.n_pad, w0 + kSellRows);
                std::stable_sort(o.begin() + w0, o.begin() + w1, [&](int a, int c) { return len_of(a) > len_of(c); });
            }
        }
        const int n_sl = b.n_pad / 32;
        std::vector<int>& w = width[static_cast<size_t>(bi)];
        w.assign(static_cast<size_t>(n_sl), 0);
        long long total = 0;
        for (int sl = 0; sl < n_sl; ++sl) {
            int m = 0;
            for (int q = sl * 32; q < sl * 32 + 32; ++q) m = std::max(m, len_of(o[q]));
            w[static_cast<size_t>(sl)] = m;
            total += 32LL * m;
        }
        slots[static_cast<size_t>(bi) + 1] = total;
        rows[static_cast<size_t>(bi) + 1] = b.n_pad;
        slices[static_cast<size_t>(bi) + 1] = n_sl;
    }
    const long long slot0 = sb.slice.back(), row0 = static_cast<long long>(sb.perm.size());
    const long long slice0 = static_cast<long long>(sb.slice.size()) - 1;
    for (int bi = 0; bi < nb; ++bi) {
        slots[static_cast<size_t>(bi) + 1] += slots[static_cast<size_t>(bi)];
        rows[static_cast<size_t>(bi) + 1] += rows[static_cast<size_t>(bi)];
        slices[static_cast<size_t>(bi) + 1] += slices[static_cast<size_t>(bi)];
    }
    const long long total = slot0 + slots[static_cast<size_t>(nb)];
    if (total > INT_MAX) fail(1, "operator too large for 32-bit slot offsets");
    sb.col.resize(static_cast<size_t>(total), 0);
    sb.val.resize(static_cast<size_t>(total), 0.0);
    sb.pad.resize(static_cast<size_t>(total), 1);
    if (sb.with_src) sb.src.resize(static_cast<size_t>(total), -1);
    if (sb.sort) sb.perm.resize(static_cast<size_t>(row0 + rows[static_cast<size_t>(nb)]));
    sb.slice.resize(static_cast<size_t>(slice0 + slices[static_cast<size_t>(nb)] + 1));
#pragma omp parallel for schedule(dynamic, 1)
    for (int bi = 0; bi < nb; ++bi) {
        const BlockSpec& b = blocks[static_cast<size_t>(bi)];
        const std::vector<int>& o = order[static_cast<size_t>(bi)];
        const std::vector<int>& w = width[static_cast<size_t>(bi)];
        const long long r0 = row0 + rows[static_cast<size_t>(bi)];
        if (sb.sort)
            for (int q = 0; q < b.n_pad; ++q) sb.perm[static_cast<size_t>(r0 + q)] = static_cast<int>(r0 + o[q]);
        long long base = slot0 + slots[static_cast<size_t>(bi)];
        const long long s0 = slice0 + slices[static_cast<size_t>(bi)];
        for (int sl = 0; sl < b.n_pad / 32; ++sl) {
            for (int lane = 0; lane < 32; ++lane) {
                const int i = o[static_cast<size_t>(sl) * 32 + lane];
                const int len = i < b.n_rows ? b.rp[i + 1] - b.rp[i] : 0;
                for (int k = 0; k < w[static_cast<size_t>(sl)]; ++k) {
                    const size_t slot = static_cast<size_t>(base + static_cast<long long>(k) * 32 + lane);
                    if (k < len) {
                        const int e = b.rp[i] + k;
                        sb.pad[slot] = 0;
                        sb.col[slot] = b.ci[e] + b.col_off;
                        sb.val[slot] = b.va != nullptr ? b.va[e] : 0.0;
                        if (sb.with_src) sb.src[slot] = b.src_of != nullptr ? b.src_of[e] + b.src_off : -1;
                    } else {
                        sb.col[slot] = b.pad_col;
                    }
                }
            }
            base += 32LL * w[static_cast<size_t>(sl)];
            sb.slice[static_cast<size_t>(s0 + sl + 1)] = static_cast<int>(base);
        }
    }
}

// CSR under construction on the host (global rows of a level; padding rows are empty).
struct CsrBuild {
    std::vector<int> rp{0};
    std::vector<int> col;
    std::vector<double> val;
};

void csr_append(CsrBuild& cb, int n_rows, int n_pad, const int* rp, const int* ci, const double* va, int col_off) {
    const long long base = static_cast<long long>(cb.col.size());
    const long long nnz = n_rows > 0 ? rp[n_rows] - rp[0] : 0;
    if (base + nnz > INT_MAX) fail(1, "operator too large for 32-bit offsets");
    cb.col.resize(static_cast<size_t>(base + nnz));
    cb.val.resize(static_cast<size_t>(base + nnz));
    const size_t r0 = cb.rp.size();
    cb.rp.resize(r0 + n_pad);
#pragma omp parallel for schedule(static) if (n_rows > 16384)
    for (int i = 0; i < n_pad; ++i) {
        if (i < n_rows) {
            const long long o = base + rp[i] - rp[0];
            for (int k = rp[i]; k < rp[i + 1]; ++k) {
                cb.col[static_cast<size_t>(o + k - rp[i])] = ci[k] + col_off;
                cb.val[static_cast<size_t>(o + k - rp[i])] = va[k];
            }
        }
        cb.rp[r0 + i] = static_cast<int>(base + (i < n_rows ? rp[i + 1] - rp[0] : nnz));
    }
}

// csr_append over many blocks in order (one block per thread after a prefix sum of their
// entries); a single block goes through csr_append.
void csr_append_blocks(CsrBuild& cb, const std::vector<BlockSpec>& blocks) {
    const int nb = static_cast<int>(blocks.size());
    if (nb == 1) {
        const BlockSpec& b = blocks[0];
        csr_append(cb, b.n_rows, b.n_pad, b.rp, b.ci, b.va, b.col_off);
        return;
    }
    std::vector<long long> ent(static_cast<size_t>(nb) + 1, 0), rows(static_cast<size_t>(nb) + 1, 0);
    for (int bi = 0; bi < nb; ++bi) {
        const BlockSpec& b = blocks[static_cast<size_t>(bi)];
        ent[static_cast<size_t>(bi) + 1] = ent[static_cast<size_t>(bi)] + (b.n_rows > 0 ? b.rp[b.n_rows] - b.rp[0] : 0);
        rows[static_cast<size_t>(bi) + 1] = rows[static_cast<size_t>(bi)] + b.n_pad;
    }
    const long long base0 = static_cast<long long>(cb.col.size());
    if (base0 + ent[static_cast<size_t>(nb)] > INT_MAX) fail(1, "operator too large for 32-bit offsets");
    const size_t r00 = cb.rp.size();
    cb.col.resize(static_cast<size_t>(base0 + ent[static_cast<size_t>(nb)]));
    cb.val.resize(static_cast<size_t>(base0 + ent[static_cast<size_t>(nb)]));
    cb.rp.resize(r00 + static_cast<size_t>(rows[static_cast<size_t>(nb)]));
#pragma omp parallel for schedule(dynamic, 1)
    for (int bi = 0; bi < nb; ++bi) {
        const BlockSpec& b = blocks[static_cast<size_t>(bi)];
        const long long base = base0 + ent[static_cast<size_t>(bi)];
        const long long nnz = ent[static_cast<size_t>(bi) + 1] - ent[static_cast<size_t>(bi)];
        const size_t r0 = r00 + static_cast<size_t>(rows[static_cast<size_t>(bi)]);
        for (int i = 0; i < b.n_pad; ++i) {
            if (i < b.n_rows) {
                const long long o = base + b.rp[i] - b.rp[0];
                for (int k = b.rp[i]; k < b.rp[i + 1]; ++k) {
                    cb.col[static_cast<size_t>(o + k - b.rp[i])] = b.ci[k] + b.col_off;
                    cb.val[static_cast<size_t>(o + k - b.rp[i])] = b.va[k];
                }
            }
            cb.rp[r0 + static_cast<size_t>(i)] = static_cast<int>(base + (i < b.n_rows ? b.rp[i + 1] - b.rp[0] : nnz));
        }
    }
}

std::vector<float> to_float(const std::vector<double>& v) {
    std::vector<float> f(v.size());
#pragma omp parallel for schedule(static) if (v.size() > (1u << 20))
    for (long long i = 0; i < static_cast<long long>(v.size()); ++i) f[i] = static_cast<float>(v[i]);
    return f;
}

// krylov_openmp.cpp:147-157 / krylov_cuda.cu:345-352: last nonzero diagonal entry, default 1.
std::vector<double> inverse_diagonal(const HostCsr& a) {
    std::vector<double> d(static_cast<size_t>(a.n_rows), 1.0);
#pragma omp parallel for schedule(static) if (a.n_rows > 65536)
    for (int i = 0; i < a.n_rows; ++i)
        for (int k = a.rp[i]; k < a.rp[i + 1]; ++k)
            if (a.ci[k] == i && a.va[k] != 0.0) d[i] = 1.0 / a.va[k];
    return d;
}

int grid_of(long long n) { return static_cast<int>(std::max<long long>(1, (n + 255) / 256)); }

// Kernel launch, with programmatic dependent launch when pdl: the kernel may be scheduled while
// its predecessor in the stream finishes (every kernel of kernels.cuh starts with pdl_entry(),
// which lets its own successor be scheduled and then waits for its predecessor's completion).
template <class... P, class... A>
void launch_k(bool pdl, void (*kernel)(P...), int grid, int block, size_t smem, cudaStream_t s, A&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(static_cast<unsigned>(grid));
    cfg.blockDim = dim3(static_cast<unsigned>(block));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    CFDB_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...));
}

} // namespace

Engine::Engine(int device) : device_(device) {
    CFDB_CUDA(cudaSetDevice(device));
    CFDB_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    CFDB_CUDA(cudaMallocHost(&h_pinned_, 4 * sizeof(int)));
}

Engine::~Engine() {
    cudaSetDevice(device_);
    release_graphs();
    if (stream_ != nullptr) {
        cudaStreamSynchronize(stream_);
        cudaStreamDestroy(stream_);
    }
    if (h_pinned_ != nullptr) cudaFreeHost(h_pinned_);
    arena_.clear();
}

void Engine::release_graphs() {
    for (auto& g : graphs_)
        for (auto& e : g)
            if (e != nullptr) {
                cudaGraphExecDestroy(e);
                e = nullptr;
            }
}

int Engine::level_rows(int l) const { return l < n_levels_ ? lv_[l].n_rows : 0; }

long long Engine::level_slots(int l) const { return l < n_levels_ ? lv_[l].a.slots : 0; }

void Engine::build(std::vector<SystemSpec> systems, int sweeps, double weight, bool need64,
                   bool need32) {
    build_times_ = PhaseTimes{};
    double t_mark = PhaseTimes::now();
    auto phase = [&](const char* name) {
        CFDB_CUDA(cudaStreamSynchronize(stream_));
        const double t = PhaseTimes::now();
        build_times_.add(name, t - t_mark);
        t_mark = t;
    };
    CFDB_CUDA(cudaSetDevice(device_));
    CFDB_CUDA(cudaStreamSynchronize(stream_));
    release_graphs();
    arena_.clear();
    phase("plan_release");
    lv_.clear();
    tail32_ = nullptr;
    tail64_ = nullptr;
    tail_n32_ = tail_n64_ = tail_grid32_ = tail_grid64_ = 0;
    tail_bar_ = nullptr;
    bcg_ = nullptr;
    n_sys_ = static_cast<int>(systems.size());
    if (n_sys_ == 0) fail(1, "engine: no systems");
    if (sweeps < 0) fail(1, "engine: negative smoothing sweeps");
    sweeps_ = sweeps;
    weight_ = weight;
    // mixed precision (the FP32 V-cycle alone): its smoother schedule may differ from the
    // hierarchy's (Tuning.mixed_sweeps / mixed_weight, picked by the autotuner); the FP64 path
    // keeps the reference's schedule
    if (need32 && !need64) {
        if (tuning_.mixed_sweeps > 0) sweeps_ = tuning_.mixed_sweeps;
        if (tuning_.mixed_weight > 0.0) weight_ = tuning_.mixed_weight;
    }
    need64_ = need64;
    need32_ = need32;
    has_amg_ = true;
    for (const auto& s : systems) {
        if (!s.h) has_amg_ = false;
        if (s.n <= 0) fail(1, "engine: empty system");
        if (s.dl && (n_sys_ != 1 || !s.h)) fail(1, "engine: device-resident levels need a single-system plan");
    }
    if (!has_amg_) {
        for (auto& s : systems) s.h.reset();
    }
    std::vector<int> L(n_sys_);
    for (int s = 0; s < n_sys_; ++s) L[s] = systems[s].h ? systems[s].h->levels() : 1;
    perm_.resize(n_sys_);
    std::iota(perm_.begin(), perm_.end(), 0);
    std::stable_sort(perm_.begin(), perm_.end(), [&](int a, int b) { return L[a] > L[b]; });
    rank_.assign(n_sys_, 0);
    for (int k = 0; k < n_sys_; ++k) rank_[perm_[k]] = k;
    n_levels_ = L[perm_[0]];
    n_of_.resize(n_sys_);
    for (int s = 0; s < n_sys_; ++s) n_of_[s] = systems[s].n;
    auto rows_at = [&](int s, int l) { return l == 0 ? systems[s].n : systems[s].h->a[l].n_rows; };
    for (int s = 0; s < n_sys_; ++s) {
        if (systems[s].h && systems[s].h->a.size() > 0 && !systems[s].h->a[0].empty() &&
            systems[s].h->a[0].n_rows != systems[s].n) {
            fail(1, "engine: hierarchy level 0 does not match the system size");
        }
        if (systems[s].h) {
            const auto& h = *systems[s].h;
            for (int l = 0; l + 1 < h.levels(); ++l) {
                const int nl = rows_at(s, l), nc = h.a[l + 1].n_rows;
                if (h.p[l].n_rows != nl || h.p[l].n_cols != nc || h.r[l].n_rows != nc ||
                    h.r[l].n_cols != nl) {
                    fail(1, "engine: transfer operator sizes do not match level " + std::to_string(l));
                }
            }
            if (h.n_c != rows_at(s, h.levels() - 1) ||
                h.coarse_inverse.size() != static_cast<size_t>(h.n_c) * h.n_c) {
                fail(1, "engine: coarse inverse size does not match the coarsest level");
            }
        }
    }
    // value-source offsets in batch order
    vs_off_.assign(n_sys_, 0);
    vs_total_ = 0;
    for (int k = 0; k < n_sys_; ++k) {
        vs_off_[perm_[k]] = vs_total_;
        vs_total_ += systems[perm_[k]].vs_len;
    }
    // per-level offsets
    std::vector<std::vector<int>> off(n_levels_, std::vector<int>(n_sys_, -1));
    lv_.resize(n_levels_);
    for (int l = 0; l < n_levels_; ++l) {
        DevLevel& d = lv_[l];
        int cursor = 0;
        d.n_rows_nc = -1;
        for (int k = 0; k < n_sys_; ++k) {
            const int s = perm_[k];
            if (L[s] <= l) continue;
            if (L[s] - 1 == l && d.n_rows_nc < 0) d.n_rows_nc = cursor;
            off[l][s] = cursor;
            cursor += round_up(rows_at(s, l), 32);
        }
        d.n_rows = cursor;
        if (d.n_rows_nc < 0) d.n_rows_nc = cursor;
    }
    off0_.resize(n_sys_);
    for (int s = 0; s < n_sys_; ++s) off0_[s] = off[0][s];
    cudaStream_t st = stream_;
    // Krylov tiles of level 0 (the reductions): kSellRows rows, or a fixed tile count when
    // target_tiles > 0; coarser levels use their operators' own tiles
    std::vector<int> sys_tile0(n_sys_ + 1, 0);
    for (int l = 0; l < 1; ++l) {
        DevLevel& d = lv_[l];
        const int base = tuning_.target_tiles > 0
                             ? std::max(kSellRows, round_up(ceil_div(std::max(d.n_rows, 1), tuning_.target_tiles), kSellRows))
                             : kSellRows;
        std::vector<int> trow, tsys;
        int nc_tiles = -1;
        for (int k = 0; k < n_sys_; ++k) {
            const int s = perm_[k];
            if (L[s] <= l) continue;
            if (L[s] - 1 == l && nc_tiles < 0) nc_tiles = static_cast<int>(tsys.size());
            if (l == 0) sys_tile0[k] = static_cast<int>(tsys.size());
            const int pad = round_up(rows_at(s, l), 32);
            for (int r = 0; r < pad; r += base) {
                trow.push_back(off[l][s] + r);
                tsys.push_back(k);
            }
        }
        if (l == 0) sys_tile0[n_sys_] = static_cast<int>(tsys.size());
        trow.push_back(d.n_rows);
        d.n_tiles = static_cast<int>(tsys.size());
        d.n_tiles_nc = nc_tiles < 0 ? d.n_tiles : nc_tiles;
        d.tiles.row = arena_.upload(trow, st);
        d.tiles.sys = n_sys_ > 1 ? arena_.upload(tsys, st) : nullptr;
    }
    // Launch tiles of one operator over the rows of `row_level` of the systems `include`
    // selects (a prefix in batch order); `nc` marks the systems that continue past that level.
    auto op_tiles = [&](DevSell64_32& m, int fmt, int row_level, auto include, auto nc) {
        const int rpt = fmt == kFmtSell ? std::max(kSellRows, tuning_.sell_rows / kSellRows * kSellRows)
                                        : (fmt <= 32 ? kFineRows : kBlock / fmt);
        m.block = fmt == kFmtSell ? kBlock : (fmt <= 32 ? kFineRows * fmt : kBlock);
        std::vector<int> trow, tsys;
        int n_nc = -1, end = 0;
        for (int k = 0; k < n_sys_; ++k) {
            const int s = perm_[k];
            if (!include(s)) continue;
            if (!nc(s) && n_nc < 0) n_nc = static_cast<int>(tsys.size());
            const int pad = round_up(rows_at(s, row_level), 32);
            for (int r = 0; r < pad; r += rpt) {
                trow.push_back(off[row_level][s] + r);
                tsys.push_back(k);
            }
            end = off[row_level][s] + pad;
        }
        trow.push_back(end);
        m.n_tiles = static_cast<int>(tsys.size());
        m.n_tiles_nc = n_nc < 0 ? m.n_tiles : n_nc;
        m.tiles.row = arena_.upload(trow, st);
        m.tiles.sys = n_sys_ > 1 ? arena_.upload(tsys, st) : nullptr;
    };
    // level-0 operator (values filled per solve) + value maps. Its layout depends only on the
    // systems' patterns, so a single-system plan rebuilt over the same pattern (a new
    // hierarchy, precision or tuning) reuses it from the previous build.
    L0Key key;
    key.n_sys = n_sys_;
    if (n_sys_ == 1) {
        const SystemSpec& sp = systems[0];
        key.rp = sp.rp;
        key.ci = sp.ci;
        key.n = sp.n;
        key.nnz = sp.rp[sp.n];
        key.vs_len = sp.vs_len;
        key.absolute_src = sp.absolute_src;
        if (sp.layout_id != 0) {
            key.map_hash = sp.layout_id;
        } else {
            const std::vector<int>& sv = sp.src_ref ? *sp.src_ref : sp.src;
            const std::vector<int>& dv = sp.diag_src_ref ? *sp.diag_src_ref : sp.diag_src;
            long long h = 0;
            for (size_t k = 0; k < sv.size(); ++k) h = h * 1000003 + sv[k];
            for (size_t k = 0; k < dv.size(); ++k) h = h * 1000003 + dv[k];
            key.map_hash = h;
        }
    }
    key.need32 = need32_;
    key.col16 = tuning_.col16 != 0;
    if (n_sys_ == 1 && l0_valid_ && key == l0_key_) {
        DevLevel& d = lv_[0];
        d.a = l0_.a;
        d.wd64 = l0_.wd64;
        d.wd32 = l0_.wd32;
        src0_ = l0_.src0;
        diag_src0_ = l0_.diag_src0;
        row_map_ = l0_.row_map;
        dinv0_ = l0_.dinv0;
        user_rows_ = l0_.user_rows;
        op_tiles(d.a, kFmtSell, 0, [](int) { return true; }, [&](int s) { return L[s] > 1; });
    } else {
        l0_valid_ = false;
        arena0_.clear();
        SellBuild sb;
        sb.with_src = true;
        std::vector<int> dsrc(static_cast<size_t>(lv_[0].n_rows), -1);
        std::vector<BlockSpec> blocks;
        blocks.reserve(static_cast<size_t>(n_sys_));
        for (int k = 0; k < n_sys_; ++k) {
            const int s = perm_[k];
            const SystemSpec& sp = systems[s];
            const std::vector<int>& sv = sp.src_ref ? *sp.src_ref : sp.src;
            const std::vector<int>& dv = sp.diag_src_ref ? *sp.diag_src_ref : sp.diag_src;
            if (static_cast<int>(sv.size()) != sp.rp[sp.n] || static_cast<int>(dv.size()) != sp.n) {
                fail(1, "engine: level-0 value map size mismatch");
            }
            const int so = sp.absolute_src ? 0 : vs_off_[s];
            blocks.push_back(BlockSpec{sp.n, round_up(sp.n, 32), sp.rp, sp.ci, nullptr, sv.data(), off[0][s], so,
                                       off[0][s]});
        }
        sell_append_blocks(sb, blocks);
#pragma omp parallel for schedule(dynamic, 1) if (n_sys_ > 1)
        for (int k = 0; k < n_sys_; ++k) {
            const int s = perm_[k];
            const SystemSpec& sp = systems[s];
            const std::vector<int>& dv = sp.diag_src_ref ? *sp.diag_src_ref : sp.diag_src;
            const int so = sp.absolute_src ? 0 : vs_off_[s];
            for (int i = 0; i < sp.n; ++i) dsrc[off[0][s] + i] = dv[i] >= 0 ? dv[i] + so : -1;
        }
        DevLevel& d = lv_[0];
        d.a.n_slices = static_cast<int>(sb.slice.size()) - 1;
        d.a.slots = sb.slice.back();
        for (int sl = 0; sl < d.a.n_slices; ++sl) {
            const int e = sb.slice[static_cast<size_t>(std::min(sl + 8, d.a.n_slices))];
            d.a.max8_slots = std::max(d.a.max8_slots, e - sb.slice[static_cast<size_t>(sl)]);
        }
        const int* dslice = arena0_.upload(sb.slice, st);
        const int* dcol = arena0_.upload(sb.col, st);
        d.a.s64 = {dslice, dcol, arena0_.alloc<double>(d.a.slots), kFmtSell};
        if (need32_) {
            d.a.s32 = {dslice, dcol, arena0_.alloc<float>(d.a.slots), kFmtSell};
            std::vector<uint16_t> c16;
            std::vector<int> cbase;
            if (tuning_.col16 && compress_cols(sb.slice, sb.col, &sb.pad, c16, cbase)) {
                d.a.s32.c16 = arena0_.upload(c16, st);
                d.a.s32.cbase = arena0_.upload(cbase, st);
            }
        }
        long long nnz0 = 0;
        for (int s = 0; s < n_sys_; ++s) nnz0 += systems[s].rp[systems[s].n];
        d.a.nnz = nnz0;
        src0_ = arena0_.upload(sb.src, st);
        diag_src0_ = arena0_.upload(dsrc, st);
        std::vector<int> rmap(static_cast<size_t>(lv_[0].n_rows), -1);
        long long uo = 0;
        for (int s = 0; s < n_sys_; ++s) {
            for (int i = 0; i < systems[s].n; ++i) rmap[off[0][s] + i] = static_cast<int>(uo + i);
            uo += systems[s].n;
        }
        user_rows_ = uo;
        row_map_ = arena0_.upload(rmap, st);
        d.wd64 = arena0_.alloc<double>(d.n_rows);
        if (need32_) d.wd32 = arena0_.alloc<float>(d.n_rows);
        dinv0_ = arena0_.alloc<double>(d.n_rows);
        op_tiles(d.a, kFmtSell, 0, [](int) { return true; }, [&](int s) { return L[s] > 1; });
        if (n_sys_ == 1) {
            l0_key_ = key;
            l0_ = L0Cache{d.a, d.wd64, d.wd32, src0_, diag_src0_, row_map_, dinv0_, user_rows_};
            l0_valid_ = true;
        }
    }
    phase("plan_level0");
    // coarser levels, transfers
    for (int l = 0; l < n_levels_; ++l) {
        DevLevel& d = lv_[l];
        // One operator over the systems that continue past level l: rows of each block from
        // `pick(s)`, columns shifted into the target level's concatenated index space. Wide
        // operators (more than kWideRow entries per row on average) are stored as CSR for the
        // warp-per-row kernels unless the engine is in ordered (bit-reproducible) mode.
        // dsrc: the operator as a device CSR (single-system plans with device-resident levels)
        auto build_op = [&](auto pick, const DevCsr* dsrc, int col_level, int row_level, DevSell64_32& m) {
            long long nnz = 0, rows = 0;
            for (int k = 0; k < n_sys_; ++k) {
                const int s = perm_[k];
                if (L[s] - 1 <= l) continue;
                nnz += dsrc != nullptr ? dsrc->nnz : pick(s).nnz();
                rows += pick(s).n_rows;
            }
            // lanes per row: about lanes_div entries per lane, and enough lanes in all to keep
            // ~150K threads busy on operators with few, long rows; never more than the row length
            const double avg = rows > 0 ? static_cast<double>(nnz) / static_cast<double>(rows) : 0.0;
            constexpr double kFillThreads = 148.0 * 1024.0;
            int lanes = 4;
            while (lanes < 256 && 2.0 * lanes <= std::max(avg, 4.0) &&
                   (lanes * std::max(tuning_.lanes_div, 1) < avg ||
                    static_cast<double>(lanes) * static_cast<double>(rows) < kFillThreads)) {
                lanes *= 2;
            }
            // CSR lane groups for long rows, and for operators too short to fill the GPU with one
            // thread per row; SELL (rows sorted by length within 256-row windows) otherwise
            const bool wide = !ordered_ && rows > 0 &&
                              (avg > tuning_.wide_row || static_cast<double>(rows) < kFillThreads);
            if (dsrc != nullptr) {
                // the same layouts built on the device (columns offset 0: one system)
                const DevCsr& a = *dsrc;
                const int n_pad = round_up(a.n_rows, 32);
                if (wide) {
                    int* dp = arena_.alloc<int>(static_cast<size_t>(n_pad) + 1);
                    csr_rows_padded(a, n_pad, dp, st);
                    int* dc = arena_.alloc<int>(static_cast<size_t>(a.nnz) + 4);
                    double* v64 = need64_ ? arena_.alloc<double>(static_cast<size_t>(a.nnz) + 4) : nullptr;
                    float* v32 = need32_ ? arena_.alloc<float>(static_cast<size_t>(a.nnz) + 4) : nullptr;
                    csr_copy_values(a, dc, v64, v32, st);
                    m.n_slices = n_pad;
                    m.slots = a.nnz;
                    if (need64_) m.s64 = {dp, dc, v64, lanes};
                    if (need32_) m.s32 = {dp, dc, v32, lanes};
                    op_tiles(m, lanes, row_level, [&](int s) { return L[s] - 1 > l; }, [](int) { return true; });
                } else {
                    int* dperm = arena_.alloc<int>(std::max(n_pad, 1));
                    int* dp = arena_.alloc<int>(static_cast<size_t>(n_pad / 32) + 1);
                    const long long slots = sell_shape(a, n_pad, kSellRows, dperm, dp, st);
                    int* dc = arena_.alloc<int>(static_cast<size_t>(slots));
                    double* v64 = need64_ ? arena_.alloc<double>(static_cast<size_t>(slots)) : nullptr;
                    float* v32 = need32_ ? arena_.alloc<float>(static_cast<size_t>(slots)) : nullptr;
                    sell_fill(a, n_pad, dperm, dp, 0, dc, v64, v32, st);
                    m.n_slices = n_pad / 32;
                    m.slots = slots;
                    if (need64_) m.s64 = {dp, dc, v64, kFmtSell, dperm};
                    if (need32_) m.s32 = {dp, dc, v32, kFmtSell, dperm};
                    op_tiles(m, kFmtSell, row_level, [&](int s) { return L[s] - 1 > l; }, [](int) { return true; });
                }
                m.nnz = nnz;
                return;
            }
            if (wide) {
                CsrBuild cbd;
                std::vector<BlockSpec> blocks;
                for (int k = 0; k < n_sys_; ++k) {
                    const int s = perm_[k];
                    if (L[s] - 1 <= l) continue;
                    const HostCsr& a = pick(s);
                    blocks.push_back(BlockSpec{a.n_rows, round_up(a.n_rows, 32), a.rp.data(), a.ci.data(), a.va.data(),
                                               nullptr, off[col_level][s], 0, 0});
                }
                csr_append_blocks(cbd, blocks);
                m.n_slices = static_cast<int>(cbd.rp.size()) - 1;
                m.slots = cbd.rp.back();
                // slack for the aligned quad loads of the last row
                cbd.col.insert(cbd.col.end(), 4, 0);
                cbd.val.insert(cbd.val.end(), 4, 0.0);
                std::vector<uint16_t> c16;
                std::vector<int> cbase;
                const bool packed = need32_ && tuning_.col16 && compress_cols(cbd.rp, cbd.col, nullptr, c16, cbase);
                const int* dp = arena_.upload(cbd.rp, st);
                const int* dc = (need64_ || !packed) ? arena_.upload(cbd.col, st) : nullptr;
                if (need64_) m.s64 = {dp, dc, arena_.upload(cbd.val, st), lanes};
                if (need32_) {
                    m.s32 = {dp, dc, arena_.upload(to_float(cbd.val), st), lanes};
                    if (packed) {
                        m.s32.c16 = arena_.upload(c16, st);
                        m.s32.cbase = arena_.upload(cbase, st);
                    }
                }
                op_tiles(m, lanes, row_level, [&](int s) { return L[s] - 1 > l; }, [](int) { return true; });
            } else {
                SellBuild sb;
                sb.sort = true;
                std::vector<BlockSpec> blocks;
                int next_row = 0;
                for (int k = 0; k < n_sys_; ++k) {
                    const int s = perm_[k];
                    if (L[s] - 1 <= l) continue;
                    const HostCsr& a = pick(s);
                    if (next_row != off[row_level][s]) fail(1, "engine: operator rows out of order");
                    next_row += round_up(a.n_rows, 32);
                    blocks.push_back(BlockSpec{a.n_rows, round_up(a.n_rows, 32), a.rp.data(), a.ci.data(), a.va.data(),
                                               nullptr, off[col_level][s], 0, off[col_level][s]});
                }
                sell_append_blocks(sb, blocks);
                m.n_slices = static_cast<int>(sb.slice.size()) - 1;
                m.slots = sb.slice.back();
                std::vector<uint16_t> c16;
                std::vector<int> cbase;
                const bool packed = need32_ && tuning_.col16 && compress_cols(sb.slice, sb.col, &sb.pad, c16, cbase);
                const int* dp = arena_.upload(sb.slice, st);
                const int* dc = (need64_ || !packed) ? arena_.upload(sb.col, st) : nullptr;
                const int* dperm = arena_.upload(sb.perm, st);
                if (need64_) m.s64 = {dp, dc, arena_.upload(sb.val, st), kFmtSell, dperm};
                if (need32_) {
                    m.s32 = {dp, dc, arena_.upload(to_float(sb.val), st), kFmtSell, dperm};
                    if (packed) {
                        m.s32.c16 = arena_.upload(c16, st);
                        m.s32.cbase = arena_.upload(cbase, st);
                    }
                }
                op_tiles(m, kFmtSell, row_level, [&](int s) { return L[s] - 1 > l; }, [](int) { return true; });
            }
            m.nnz = nnz;
        };
        const DeviceLevels* dl = systems[perm_[0]].dl.get();
        const bool dev_l = dl != nullptr && L[perm_[0]] - 1 > l;
        if (l > 0) {
            if (dev_l) {
                // weight / diagonal on the device from A_l (rows padded to the level's block)
                if (need64_) d.wd64 = arena_.alloc<double>(std::max(d.n_rows_nc, 1));
                if (need32_) d.wd32 = arena_.alloc<float>(std::max(d.n_rows_nc, 1));
                weighted_inverse_diagonal(dl->a[l], d.n_rows_nc, weight_, d.wd64, d.wd32, st);
            } else {
                std::vector<double> wd(static_cast<size_t>(d.n_rows_nc), weight_);
#pragma omp parallel for schedule(dynamic, 1) if (n_sys_ > 1)
                for (int k = 0; k < n_sys_; ++k) {
                    const int s = perm_[k];
                    if (L[s] - 1 <= l) continue; // only systems with a coarser level need A_l here
                    const HostCsr& a = systems[s].h->a[l];
                    const std::vector<double> dinv = inverse_diagonal(a);
                    for (int i = 0; i < a.n_rows; ++i) wd[off[l][s] + i] = weight_ * dinv[i];
                }
                if (need64_) d.wd64 = arena_.upload(wd, st);
                if (need32_) d.wd32 = arena_.upload(to_float(wd), st);
            }
            build_op([&](int s) -> const HostCsr& { return systems[s].h->a[l]; }, dev_l ? &dl->a[l] : nullptr, l, l,
                     d.a);
        }
        if (l + 1 < n_levels_) {
            build_op([&](int s) -> const HostCsr& { return systems[s].h->p[l]; }, dev_l ? &dl->p[l] : nullptr, l + 1,
                     l, d.p);
            build_op([&](int s) -> const HostCsr& { return systems[s].h->r[l]; }, dev_l ? &dl->r[l] : nullptr, l,
                     l + 1, d.r);
        }
        // vectors (zero-initialised)
        auto vec64 = [&](int n) {
            double* p = arena_.alloc<double>(n);
            CFDB_CUDA(cudaMemsetAsync(p, 0, sizeof(double) * std::max(n, 1), st));
            return p;
        };
        auto vec32 = [&](int n) {
            float* p = arena_.alloc<float>(n);
            CFDB_CUDA(cudaMemsetAsync(p, 0, sizeof(float) * std::max(n, 1), st));
            return p;
        };
        if (need64_ || l == 0) {
            d.x64 = vec64(d.n_rows);
            d.y64 = vec64(d.n_rows);
            d.t64 = vec64(d.n_rows);
            if (l > 0) d.b64 = vec64(d.n_rows);
        }
        if (need32_) {
            d.x32 = vec32(d.n_rows);
            d.y32 = vec32(d.n_rows);
            d.t32 = vec32(d.n_rows);
            if (l > 0) d.b32 = vec32(d.n_rows);
        }
    }
    phase("plan_levels");
    // Krylov vectors and state
    {
        const int n0 = lv_[0].n_rows;
        auto vec64 = [&](int n) {
            double* p = arena_.alloc<double>(n);
            CFDB_CUDA(cudaMemsetAsync(p, 0, sizeof(double) * std::max(n, 1), st));
            return p;
        };
        b_ = vec64(n0);
        x_ = vec64(n0);
        r_ = vec64(n0);
        p_ = vec64(n0);
        q_ = vec64(n0);
        vs_ = arena_.alloc<double>(std::max(vs_total_, 1));
        st_ = arena_.alloc<SysState>(n_sys_);
        CFDB_CUDA(cudaMemsetAsync(st_, 0, sizeof(SysState) * n_sys_, st));
        // two-level reduction: groups of kGroupTiles tiles within each system
        std::vector<int> grp0(n_sys_ + 1, 0);
        for (int k = 0; k < n_sys_; ++k) grp0[k + 1] = grp0[k] + ceil_div(sys_tile0[k + 1] - sys_tile0[k], kGroupTiles);
        const int n_groups = std::max(grp0[n_sys_], 1);
        red_.partials = arena_.alloc<double>(2 * static_cast<size_t>(std::max(lv_[0].n_tiles, 1)));
        red_.gpartials = arena_.alloc<double>(2 * static_cast<size_t>(n_groups));
        int* cnt = arena_.alloc<int>(n_sys_ + n_groups);
        CFDB_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * (n_sys_ + n_groups), st));
        red_.counters = cnt;
        red_.gcounters = cnt + n_sys_;
        red_.sys_tile0 = arena_.upload(sys_tile0, st);
        red_.grp0 = arena_.upload(grp0, st);
        n_active_ = arena_.alloc<int>(1);
        tail_bar_ = arena_.alloc<unsigned>(2);
        CFDB_CUDA(cudaMemsetAsync(tail_bar_, 0, 2 * sizeof(unsigned), st));
        error_ = arena_.alloc<int>(1);
        CFDB_CUDA(cudaMemsetAsync(error_, 0, sizeof(int), st));
    }
    // coarse blocks (one per system with two or more levels; single-level systems are
    // Jacobi-preconditioned and have none)
    n_blocks_ = 0;
    fused_final_ = has_amg_ && sweeps_ > 0;
    if (has_amg_) {
        std::vector<int> bsys, brow, bn, blevel;
        std::vector<long long> moff;
        std::vector<double> mt, mr;
        std::vector<int> tblk, trow;
        size_t max_n = 0;
        for (int k = 0; k < n_sys_; ++k) {
            const int s = perm_[k];
            const Hierarchy& h = *systems[s].h;
            const int c = h.levels() - 1;
            if (c == 0) {
                fused_final_ = false; // their r.z comes from k_cg_rz
                continue;
            }
            const int n = h.n_c;
            bsys.push_back(k);
            brow.push_back(off[c][s]);
            bn.push_back(n);
            blevel.push_back(c);
            moff.push_back(static_cast<long long>(mt.size()));
            const size_t o = mt.size();
            mt.resize(o + static_cast<size_t>(n) * n);
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < n; ++j)
                    mt[o + static_cast<size_t>(j) * n + i] = h.coarse_inverse[static_cast<size_t>(i) * n + j];
            mr.insert(mr.end(), h.coarse_inverse.begin(), h.coarse_inverse.end());
            for (int i = 0; i < n; i += kCoarseRows) {
                tblk.push_back(static_cast<int>(bsys.size()) - 1);
                trow.push_back(i);
            }
            max_n = std::max(max_n, static_cast<size_t>(round_up(n, 32)));
        }
        n_blocks_ = static_cast<int>(bsys.size());
        coarse_bytes_ = 0.0;
        coarse_rows_ = 0.0;
        for (int b = 0; b < n_blocks_; ++b) {
            coarse_bytes_ += 8.0 * bn[b] * static_cast<double>(bn[b]);
            coarse_rows_ += bn[b];
        }
        n_single_ = 0;
        for (int k = 0; k < n_sys_; ++k)
            if (systems[perm_[k]].h->levels() == 1) ++n_single_;
        single_.assign(n_sys_, 0);
        for (int s = 0; s < n_sys_; ++s) single_[s] = systems[s].h->levels() == 1 ? 1 : 0;
        cb_.sys = arena_.upload(bsys, st);
        cb_.row = arena_.upload(brow, st);
        cb_.n = arena_.upload(bn, st);
        cb_.m_off = arena_.upload(moff, st);
        cb_.mt = arena_.upload(mt, st);
        cb_.mr = arena_.upload(mr, st);
        cb_.tile_blk = arena_.upload(tblk, st);
        cb_.tile_row = arena_.upload(trow, st);
        n_ctiles_ = static_cast<int>(tblk.size());
        block_level_ = arena_.upload(blevel, st);
        coarse_smem64_ = max_n * sizeof(double);
        coarse_smem32_ = max_n * sizeof(float);
        if (coarse_smem64_ > 200 * 1024) fail(1, "coarsest level too large for the dense solve (> 25600 rows)");
        std::vector<double*> bl64(n_levels_), xl64(n_levels_);
        std::vector<float*> bl32(n_levels_), xl32(n_levels_);
        for (int l = 0; l < n_levels_; ++l) {
            bl64[l] = l == 0 ? r_ : lv_[l].b64;
            xl64[l] = lv_[l].x64;
            bl32[l] = lv_[l].b32; // level 0 (single-level systems) handled by the FP64 kernel
            xl32[l] = lv_[l].x32;
        }
        b_level64_ = arena_.upload(bl64, st);
        x_level64_ = arena_.upload(xl64, st);
        b_level32_ = arena_.upload(bl32, st);
        x_level32_ = arena_.upload(xl32, st);
        if (coarse_smem64_ > 48 * 1024) {
            CFDB_CUDA(cudaFuncSetAttribute(k_vc_coarse<double, double>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(coarse_smem64_)));
            CFDB_CUDA(cudaFuncSetAttribute(k_vc_coarse<double, float>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(coarse_smem64_)));
            CFDB_CUDA(cudaFuncSetAttribute(k_vc_coarse<float, float>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(coarse_smem32_)));
        }
    }
    phase("plan_rest");
}

void Engine::set_values_device(const double* p0, const double* p1, const double* p2, int n1, int n2) {
    const DevLevel& d = lv_[0];
    ValueSource vs{p0, p1, p2, n1, n2};
    const long long n = std::max<long long>(d.a.slots, d.n_rows);
    launch_k(tuning_.pdl != 0, k_fill_level0, grid_of(n), 256, 0, stream_, static_cast<int>(d.a.slots), d.n_rows, src0_, diag_src0_, vs,
                                                   weight_, d.a.s64.val ? const_cast<double*>(d.a.s64.val) : nullptr,
                                                   d.a.s32.val ? const_cast<float*>(d.a.s32.val) : nullptr, d.wd64,
                                                   d.wd32);
    // plain inverse diagonal for Jacobi preconditioning: weight 1
    launch_k(tuning_.pdl != 0, k_fill_level0, grid_of(d.n_rows), 256, 0, stream_, 0, d.n_rows, src0_, diag_src0_, vs, 1.0, nullptr,
                                                          nullptr, dinv0_, nullptr);
    launches_ += 2;
    CFDB_CUDA(cudaGetLastError());
}

void Engine::upload_values(const std::vector<const double*>& host_src) {
    // host_src[s]: the value source of original system s
    std::vector<int> lens(n_sys_);
    for (int k = 0; k < n_sys_; ++k) {
        const int s = perm_[k];
        const int next = k + 1 < n_sys_ ? vs_off_[perm_[k + 1]] : vs_total_;
        lens[s] = next - vs_off_[s];
    }
    for (int s = 0; s < n_sys_; ++s) {
        if (lens[s] > 0) copier_.to_device(vs_ + vs_off_[s], host_src[s], sizeof(double) * lens[s], stream_);
    }
    set_values_device(vs_, vs_, vs_, INT_MAX, INT_MAX);
}

void Engine::upload_values_ldu(const double* diag, const double* upper, const double* lower, int n, int nf) {
    if (n_sys_ != 1 || vs_total_ != static_cast<long long>(n) + 2LL * nf) fail(1, "upload_values_ldu: layout mismatch");
    copier_.to_device(vs_, diag, sizeof(double) * n, stream_);
    if (nf > 0) {
        copier_.to_device(vs_ + n, upper, sizeof(double) * nf, stream_);
        copier_.to_device(vs_ + n + nf, lower, sizeof(double) * nf, stream_);
    }
    set_values_device(vs_, vs_, vs_, INT_MAX, INT_MAX);
}

void Engine::upload_values_device_concat(const std::vector<const double*>& dev_src) {
    std::vector<int> lens(n_sys_);
    for (int k = 0; k < n_sys_; ++k) {
        const int s = perm_[k];
        const int next = k + 1 < n_sys_ ? vs_off_[perm_[k + 1]] : vs_total_;
        lens[s] = next - vs_off_[s];
    }
    for (int s = 0; s < n_sys_; ++s) {
        if (lens[s] > 0) {
            CFDB_CUDA(cudaMemcpyAsync(vs_ + vs_off_[s], dev_src[s], sizeof(double) * lens[s],
                                      cudaMemcpyDeviceToDevice, stream_));
        }
    }
    set_values_device(vs_, vs_, vs_, INT_MAX, INT_MAX);
}

void Engine::set_rhs_guess_concat(const double* b, const double* x0) {
    const int n = lv_[0].n_rows;
    launch_k(tuning_.pdl != 0, k_gather_rows, grid_of(n), 256, 0, stream_, n, row_map_, b, b_);
    launch_k(tuning_.pdl != 0, k_gather_rows, grid_of(n), 256, 0, stream_, n, row_map_, x0, x_);
    launches_ += 2;
    CFDB_CUDA(cudaGetLastError());
}

void Engine::get_solution_concat(double* x) {
    const int n = lv_[0].n_rows;
    launch_k(tuning_.pdl != 0, k_scatter_rows, grid_of(n), 256, 0, stream_, n, row_map_, x_, x);
    ++launches_;
    CFDB_CUDA(cudaGetLastError());
    CFDB_CUDA(cudaStreamSynchronize(stream_));
}

void Engine::set_rhs(int s, const double* b, bool dev) {
    if (dev)
        CFDB_CUDA(cudaMemcpyAsync(b_ + off0_[s], b, sizeof(double) * n_of_[s], cudaMemcpyDeviceToDevice, stream_));
    else
        copier_.to_device(b_ + off0_[s], b, sizeof(double) * n_of_[s], stream_);
}

void Engine::set_guess(int s, const double* x, bool dev) {
    if (dev)
        CFDB_CUDA(cudaMemcpyAsync(x_ + off0_[s], x, sizeof(double) * n_of_[s], cudaMemcpyDeviceToDevice, stream_));
    else
        copier_.to_device(x_ + off0_[s], x, sizeof(double) * n_of_[s], stream_);
}

void Engine::get_solution(int s, double* x, bool dev) {
    if (dev)
        CFDB_CUDA(cudaMemcpyAsync(x, x_ + off0_[s], sizeof(double) * n_of_[s], cudaMemcpyDeviceToDevice, stream_));
    else
        copier_.to_host(x, x_ + off0_[s], sizeof(double) * n_of_[s], stream_);
}

void Engine::set_residual(int s, const double* r, bool dev) {
    CFDB_CUDA(cudaMemcpyAsync(r_ + off0_[s], r, sizeof(double) * n_of_[s],
                              dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, stream_));
}

void Engine::get_precond(int s, double* z, bool dev, Mode mode) {
    CFDB_CUDA(cudaStreamSynchronize(stream_));
    const int n = n_of_[s];
    if (mode == Mode::AmgMixed) {
        std::vector<float> tmp(n);
        CFDB_CUDA(cudaMemcpy(tmp.data(), lv_[0].x32 + off0_[s], sizeof(float) * n, cudaMemcpyDeviceToHost));
        if (dev) fail(1, "get_precond: device output not supported for FP32");
        for (int i = 0; i < n; ++i) z[i] = tmp[i];
    } else {
        CFDB_CUDA(cudaMemcpy(z, lv_[0].x64 + off0_[s], sizeof(double) * n,
                             dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost));
    }
}

// ---------------------------------------------------------------------------------------------
// V-cycle enqueue
// ---------------------------------------------------------------------------------------------

namespace {
template <class T> T* vx(double* a, float* b);
template <> double* vx<double>(double* a, float*) { return a; }
template <> float* vx<float>(double*, float* b) { return b; }
template <class T> Sell<T> vs_sel(const Sell<double>& a, const Sell<float>& b);
template <> Sell<double> vs_sel<double>(const Sell<double>& a, const Sell<float>&) { return a; }
template <> Sell<float> vs_sel<float>(const Sell<double>&, const Sell<float>& b) { return b; }

// Calls fn with the visiting strategy v as a compile-time constant.
template <class Fn> void with_visit(int v, Fn&& fn) {
    if (v == kVisitSell2) fn(std::integral_constant<int, kVisitSell2>{});
    else if (v == kVisitSell1) fn(std::integral_constant<int, kVisitSell1>{});
    else if (v == kVisitWarp) fn(std::integral_constant<int, kVisitWarp>{});
    else fn(std::integral_constant<int, kVisitBlock>{});
}
} // namespace

// Buffer holding the first pre-smoothing iterate of level l, chosen so that after the
// remaining pre sweeps and the post sweeps the iterate lands in x.
template <class T> T* Engine::start_buffer(int l) const {
    T* x = vx<T>(lv_[l].x64, lv_[l].x32);
    T* y = vx<T>(lv_[l].y64, lv_[l].y32);
    const bool fuse = sweeps_ >= 2 && tuning_.fuse_first != 0;
    const int writes_pre = fuse ? sweeps_ - 1 : sweeps_;
    T* target = (sweeps_ % 2 == 0) ? x : y;
    return (writes_pre % 2 == 1) ? target : (target == x ? y : x);
}

X1Out Engine::x1_out(Mode mode) const {
    X1Out o{};
    const bool fuse = sweeps_ >= 2 && tuning_.fuse_first != 0;
    if (mode == Mode::Jacobi || !has_amg_ || sweeps_ == 0 || fuse || n_levels_ < 2) return o;
    const DevLevel& d = lv_[0];
    o.n = d.n_rows_nc;
    if (mode == Mode::AmgMixed) {
        o.wd32 = d.wd32;
        o.x32 = start_buffer<float>(0);
    } else {
        o.wd64 = d.wd64;
        o.x64 = start_buffer<double>(0);
    }
    return o;
}

// First level of the persistent tail, or n_levels_ when the tail is not used: the levels from
// there down must all be small (<= tail_rows rows) lane-group CSR operators, the schedule the
// unfused one (first sweeps written by the restrictions), and the engine not in ordered mode.
int Engine::tail_level() const {
    const bool fuse = sweeps_ >= 2 && tuning_.fuse_first != 0;
    if (!has_amg_ || ordered_ || fuse || sweeps_ == 0 || tuning_.tail_rows <= 0 || n_levels_ < 3) return n_levels_;
    int lt = n_levels_ - 1;
    while (lt - 1 >= 1) {
        const int l = lt - 1;
        const DevLevel& d = lv_[l];
        if (d.n_rows > tuning_.tail_rows) break;
        auto csr = [](const DevSell64_32& m) { return m.s64.val != nullptr ? m.s64.fmt != kFmtSell : m.s32.fmt != kFmtSell; };
        if (d.a.n_tiles > 0 && !csr(d.a)) break;
        if (d.p.n_tiles > 0 && !csr(d.p)) break;
        if (d.r.n_tiles > 0 && !csr(d.r)) break;
        lt = l;
    }
    return lt <= n_levels_ - 2 ? lt : n_levels_;
}

// Phase list of the tail for precision T (uploaded before any graph capture that uses it).
template <class T> void Engine::prepare_tail() {
    TailPhase<T>*& dev = sizeof(T) == 8 ? reinterpret_cast<TailPhase<T>*&>(tail64_) : reinterpret_cast<TailPhase<T>*&>(tail32_);
    int& count = sizeof(T) == 8 ? tail_n64_ : tail_n32_;
    int& grid = sizeof(T) == 8 ? tail_grid64_ : tail_grid32_;
    double& bytes = sizeof(T) == 8 ? tail_bytes64_ : tail_bytes32_;
    if (dev != nullptr) return;
    const int L = n_levels_;
    const int lt = tail_level();
    count = 0;
    if (lt >= L) return;
    auto X = [&](int l) { return vx<T>(lv_[l].x64, lv_[l].x32); };
    auto Y = [&](int l) { return vx<T>(lv_[l].y64, lv_[l].y32); };
    auto Tv = [&](int l) { return vx<T>(lv_[l].t64, lv_[l].t32); };
    auto Bv = [&](int l) { return vx<T>(lv_[l].b64, lv_[l].b32); };
    auto WD = [&](int l) -> const T* {
        if constexpr (sizeof(T) == 8) return lv_[l].wd64;
        else return lv_[l].wd32;
    };
    auto OP = [&](const DevSell64_32& m) { return vs_sel<T>(m.s64, m.s32); };
    const double sv = sizeof(T);
    auto csr_b = [&](const DevSell64_32& m, double rows, double cols) {
        const double cb = sizeof(T) == 4 && m.s32.c16 != nullptr ? 2.0 : 4.0;
        return static_cast<double>(m.nnz) * (sv + cb) + 4.0 * (rows + 1.0) + sv * cols + sv * rows;
    };
    std::vector<TailPhase<T>> ph;
    bytes = 0.0;
    int max_blocks = 1;
    auto add = [&](int kind, const DevSell64_32& m, int n, const T* x, const T* b, const T* wd, T* y, T* x1, int n1,
                   double by) {
        TailPhase<T> p{};
        p.kind = kind;
        p.n = n;
        p.m = OP(m);
        p.x = x;
        p.b = b;
        p.wd = wd;
        p.y = y;
        p.x1 = x1;
        p.n1 = n1;
        ph.push_back(p);
        bytes += by;
        if (kind != kTailCoarse) max_blocks = std::max(max_blocks, ceil_div(n, kBlock / p.m.fmt));
    };
    std::vector<T*> cur(L, nullptr);
    for (int l = lt; l + 1 < L; ++l) {
        const DevLevel& d = lv_[l];
        const double n = d.n_rows_nc;
        T* x = X(l);
        T* y = Y(l);
        T* c = start_buffer<T>(l);
        for (int k = 1; k < sweeps_; ++k) {
            T* o = c == x ? y : x;
            add(kTailJacobi, d.a, d.a.n_slices, c, Bv(l), WD(l), o, nullptr, 0, csr_b(d.a, n, n) + 3.0 * sv * n);
            c = o;
        }
        cur[l] = c;
        add(kTailResidual, d.a, d.a.n_slices, c, Bv(l), nullptr, Tv(l), nullptr, 0, csr_b(d.a, n, n) + sv * n);
        const DevLevel& nx = lv_[l + 1];
        const bool next_x1 = l + 2 < L && nx.n_rows_nc > 0;
        add(kTailRestrict, d.r, d.r.n_slices, Tv(l), nullptr, next_x1 ? WD(l + 1) : nullptr, Bv(l + 1),
            next_x1 ? start_buffer<T>(l + 1) : nullptr, next_x1 ? nx.n_rows_nc : 0,
            csr_b(d.r, nx.n_rows, n) + (next_x1 ? 2.0 * sv * nx.n_rows_nc : 0.0));
    }
    {
        TailPhase<T> p{};
        p.kind = kTailCoarse;
        ph.push_back(p);
        bytes += coarse_bytes_ + 2.0 * sv * coarse_rows_;
        max_blocks = std::max(max_blocks, n_ctiles_);
    }
    for (int l = L - 2; l >= lt; --l) {
        const DevLevel& d = lv_[l];
        const double n = d.n_rows_nc;
        T* x = X(l);
        T* y = Y(l);
        T* c = cur[l];
        add(kTailProlong, d.p, d.p.n_slices, X(l + 1), nullptr, nullptr, c, nullptr, 0,
            csr_b(d.p, n, lv_[l + 1].n_rows) + sv * n);
        for (int k = 0; k < sweeps_; ++k) {
            T* o = c == x ? y : x;
            add(kTailJacobi, d.a, d.a.n_slices, c, Bv(l), WD(l), o, nullptr, 0, csr_b(d.a, n, n) + 3.0 * sv * n);
            c = o;
        }
    }
    const size_t smem = sizeof(T) == 8 ? coarse_smem64_ : coarse_smem32_;
    if (tuning_.tail_cluster > 0) {
        // one cluster of tail_cluster CTAs; kept only if such a cluster can be resident
        const int cs = std::min(std::max(tuning_.tail_cluster, 2), 16);
        CFDB_CUDA(cudaFuncSetAttribute(k_vc_tail<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem)));
        CFDB_CUDA(cudaFuncSetAttribute(k_vc_tail<T, true>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        cudaLaunchConfig_t q{};
        q.gridDim = dim3(static_cast<unsigned>(cs));
        q.blockDim = dim3(kBlock);
        q.dynamicSmemBytes = smem;
        cudaLaunchAttribute a[1];
        a[0].id = cudaLaunchAttributeClusterDimension;
        a[0].val.clusterDim.x = static_cast<unsigned>(cs);
        a[0].val.clusterDim.y = 1;
        a[0].val.clusterDim.z = 1;
        q.attrs = a;
        q.numAttrs = 1;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, k_vc_tail<T, true>, &q) != cudaSuccess || clusters <= 0) {
            (void)cudaGetLastError();
            return; // no such cluster fits: keep the separate kernels
        }
        grid = cs;
    } else {
        // grid: co-resident CTAs (cooperative launch), no more than the largest phase can use
        CFDB_CUDA(cudaFuncSetAttribute(k_vc_tail<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem)));
        int per_sm = 0, sms = 0;
        CFDB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_vc_tail<T, false>, kBlock, smem));
        CFDB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_));
        if (per_sm <= 0) return;  // cannot be co-resident: keep the separate kernels
        grid = std::max(1, std::min(per_sm * sms, max_blocks));
    }
    TailPhase<T>* d = arena_.alloc<TailPhase<T>>(ph.size());
    CFDB_CUDA(cudaMemcpyAsync(d, ph.data(), sizeof(TailPhase<T>) * ph.size(), cudaMemcpyHostToDevice, stream_));
    CFDB_CUDA(cudaStreamSynchronize(stream_));
    dev = d;
    count = static_cast<int>(ph.size());
}

template <class T> void Engine::launch_tail(cudaStream_t s) {
    const TailPhase<T>* ph = sizeof(T) == 8 ? reinterpret_cast<const TailPhase<T>*>(tail64_)
                                            : reinterpret_cast<const TailPhase<T>*>(tail32_);
    const int count = sizeof(T) == 8 ? tail_n64_ : tail_n32_;
    const int grid = sizeof(T) == 8 ? tail_grid64_ : tail_grid32_;
    T* const* b_lv;
    T* const* x_lv;
    if constexpr (sizeof(T) == 8) {
        b_lv = b_level64_;
        x_lv = x_level64_;
    } else {
        b_lv = b_level32_;
        x_lv = x_level32_;
    }
    const size_t smem = sizeof(T) == 8 ? coarse_smem64_ : coarse_smem32_;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(static_cast<unsigned>(grid));
    cfg.blockDim = dim3(kBlock);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (tuning_.tail_cluster > 0) {
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = static_cast<unsigned>(grid);
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        CFDB_CUDA(cudaLaunchKernelEx(&cfg, k_vc_tail<T, true>, ph, count, cb_, n_ctiles_, b_lv, x_lv,
                                     static_cast<const int*>(block_level_), tail_bar_, error_, tuning_.wait_polls));
    } else {
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        CFDB_CUDA(cudaLaunchKernelEx(&cfg, k_vc_tail<T, false>, ph, count, cb_, n_ctiles_, b_lv, x_lv,
                                     static_cast<const int*>(block_level_), tail_bar_, error_, tuning_.wait_polls));
    }
}

template <class T>
void Engine::enqueue_vcycle_t(bool fused_final, int flexible, bool x1_ready0) {
    cudaStream_t s = stream_;
    const SysState* stv = st_;
    const int L = n_levels_;
    // final pre-smoothing buffer so that after `sweeps_` post sweeps the iterate lands in x
    const bool fuse = sweeps_ >= 2 && tuning_.fuse_first != 0;
    // unfused schedule: each restriction also writes the coarser level's first sweep
    const bool x1_by_restrict = !fuse && sweeps_ > 0;
    auto X = [&](int l) { return vx<T>(lv_[l].x64, lv_[l].x32); };
    auto Y = [&](int l) { return vx<T>(lv_[l].y64, lv_[l].y32); };
    auto Tv = [&](int l) { return vx<T>(lv_[l].t64, lv_[l].t32); };
    auto Bv = [&](int l) { return vx<T>(lv_[l].b64, lv_[l].b32); };
    auto WD = [&](int l) -> const T* {
        if constexpr (sizeof(T) == 8) return lv_[l].wd64;
        else return lv_[l].wd32;
    };
    auto A = [&](int l) { return vs_sel<T>(lv_[l].a.s64, lv_[l].a.s32); };
    auto P = [&](int l) { return vs_sel<T>(lv_[l].p.s64, lv_[l].p.s32); };
    auto R = [&](int l) { return vs_sel<T>(lv_[l].r.s64, lv_[l].r.s32); };

    const double sv = sizeof(T);
    const double sb0 = 8.0; // level-0 right-hand side: the FP64 Krylov residual
    auto spmv_b = [&](const DevSell64_32& m, double rows, double cols) {
        const double cb = sizeof(T) == 4 && m.s32.c16 != nullptr ? 2.0 : 4.0;
        return static_cast<double>(m.nnz) * (sv + cb) + 4.0 * (rows + 1.0) + sv * cols + sv * rows;
    };
    // tiles of an operator: one row per warp for CSR operators, slice runs for SELL ones
    struct Launch {
        Tiles first;
        int second; // grid
        int block;
        int visit;  // row-visiting strategy of the operator's kernels
    };
    auto TL = [&](int, const DevSell64_32& m, bool nc) -> Launch {
        return {m.tiles, nc ? m.n_tiles_nc : m.n_tiles, m.block, vcycle_visit(m)};
    };
    std::vector<T*> cur(L, nullptr);
    // levels lt and below run in the persistent tail kernel when its phases are prepared
    const int tail_count = sizeof(T) == 8 ? tail_n64_ : tail_n32_;
    const int lt = tail_count > 0 ? tail_level() : L;
    // ---- down ----
    for (int l = 0; l + 1 < L && l < lt; ++l) {
        const DevLevel& d = lv_[l];
        if (d.a.n_tiles_nc == 0) continue;  // no system continues past this level
        const double n = d.n_rows_nc;
        const double sb = l == 0 ? sb0 : sv;
        T* x = X(l);
        T* y = Y(l);
        T* start = start_buffer<T>(l);
        const bool x1_ready = l == 0 ? x1_ready0 : x1_by_restrict;
        if (sweeps_ == 0) {
            CFDB_CUDA(cudaMemsetAsync(x, 0, sizeof(T) * d.n_rows_nc, s));
            cur[l] = x;
        } else if (x1_ready) {
            // first sweep already in `start` (written with the right-hand side)
            const auto ta = TL(l, d.a, true);
            T* c = start;
            for (int k = 1; k < sweeps_; ++k) {
                T* o = c == x ? y : x;
                if (l == 0) with_visit(ta.visit, [&](auto V) { launch_k(tuning_.pdl != 0, k_vc_jacobi<T, double, decltype(V)::value>, ta.second, ta.block, 0, s, A(l), ta.first, stv, WD(l), r_, c, o); });
                else with_visit(ta.visit, [&](auto V) { launch_k(tuning_.pdl != 0, k_vc_jacobi<T, T, decltype(V)::value>, ta.second, ta.block, 0, s, A(l), ta.first, stv, WD(l), Bv(l), c, o); });
                mark("smooth", l, spmv_b(d.a, n, n) + sv * n + sb * n);
                c = o;
            }
            cur[l] = c;
        } else {
            const auto ta = TL(l, d.a, true);
            if (l == 0) {
                with_visit(ta.visit, [&](auto V) { launch_k(tuning_.pdl != 0, k_vc_first<T, double, decltype(V)::value>, ta.second, ta.block, 0, s, A(l), ta.first, stv, WD(l), r_, start, fuse); });
            } else {
                with_visit(ta.visit, [&](auto V) { launch_k(tuning_.pdl != 0, k_vc_first<T, T, decltype(V)::value>, ta.second, ta.block, 0, s, A(l), ta.first, stv, WD(l), Bv(l), start, fuse); });
            }
            mark("smooth_first", l, fuse ? spmv_b(d.a, n, n) - sv * n + sv * n + sb * n : 2.0 * sv * n + sb * n);
            T* c = start;
            for (int k = fuse ? 2 : 1; k < sweeps_; ++k) {
                T* o = c == x ? y : x;
                if (l == 0) with_visit(ta.visit, [&](auto V) { launch_k(tuning_.pdl != 0, k_vc_jacobi<T, double, decltype(V)::value>, ta.second, ta.block, 0, s, A(l), ta.first, stv, WD(l), r_, c, o); });
                else with_visit(ta.visit, [&](auto V) { launch_k(tuning_.pdl != 0, k_vc_jacobi<T, T, decltype(V)::value>, ta.second, ta.block, 0, s, A(l), ta.first, stv, WD(l), Bv(l), c, o); });
                mark("smooth", l, spmv_b(d.a, n, n) + sv * n + sb * n);
                c = o;
            }
            cur[l] = c;
        }
        const auto tr = TL(l, d.a, true);
        if (l == 0) with_visit(tr.visit, [&](auto V) { launch_k(tuning_.pdl != 0, k_vc_residual<T, double, decltype(V)::value>, tr.second, tr.block, 0, s, A(l), tr.first, stv, r_, cur[l], Tv(l)); });
        else with_visit(tr.visit, [&](auto V) { launch_k(tuning_.pdl != 0, k_vc_residual<T, T, decltype(V)::value>, tr.second, tr.block, 0, s, A(l), tr.first, stv, Bv(l), cur[l], Tv(l)); });
        mark("residual", l, spmv_b(d.a, n, n) + sb * n);
        const DevLevel& nx = lv_[l + 1];
        const auto tq = TL(l + 1, d.r, false);
        const bool next_x1 = x1_by_restrict && l + 2 < L && nx.n_rows_nc > 0;
        with_visit(tq.visit, [&](auto V) {
            launch_k(tuning_.pdl != 0, k_vc_spmv<T, decltype(V)::value>, tq.second, tq.block, 0, s, 
                R(l), tq.first, stv, Tv(l), Bv(l + 1), next_x1 ? WD(l + 1) : nullptr,
                next_x1 ? start_buffer<T>(l + 1) : nullptr, next_x1 ? nx.n_rows_nc : 0);
        });
        mark("restrict", l, spmv_b(d.r, nx.n_rows, n) + (next_x1 ? 2.0 * sv * nx.n_rows_nc : 0.0));
    }
    // ---- coarsest blocks (dense inverse of each multi-level system's coarsest operator) ----
    const Control ctl{n_active_, error_, tuning_.wait_polls};
    const int ord = ordered_ ? 1 : 0;
    if (lt < L) {
        launch_tail<T>(s);
        mark("tail", lt, sizeof(T) == 8 ? tail_bytes64_ : tail_bytes32_);
    } else if (n_ctiles_ > 0) {
        if constexpr (sizeof(T) == 8) {
            launch_k(tuning_.pdl != 0, k_vc_coarse<double, double>, n_ctiles_, kBlock, coarse_smem64_, s, cb_, stv, b_level64_, x_level64_,
                                                                                  block_level_, ctl, ord);
        } else {
            launch_k(tuning_.pdl != 0, k_vc_coarse<float, float>, n_ctiles_, kBlock, coarse_smem32_, s, cb_, stv, b_level32_, x_level32_,
                                                                                block_level_, ctl, ord);
        }
        mark("coarse", L - 1, coarse_bytes_ + 2.0 * sv * coarse_rows_);
    }
    // ---- up ----
    for (int l = std::min(L - 2, lt - 1); l >= 0; --l) {
        const DevLevel& d = lv_[l];
        if (d.a.n_tiles_nc == 0) continue;  // no system continues past this level
        const double n = d.n_rows_nc;
        const double sb = l == 0 ? sb0 : sv;
        T* x = X(l);
        T* y = Y(l);
        T* c = cur[l];
        const auto tp = TL(l, d.p, true);
        with_visit(tp.visit, [&](auto V) {
            launch_k(tuning_.pdl != 0, k_vc_prolong<T, decltype(V)::value>, tp.second, tp.block, 0, s, P(l), tp.first, stv, X(l + 1), c);
        });
        const auto ta = TL(l, d.a, true);
        mark("prolong", l, spmv_b(d.p, n, lv_[l + 1].n_rows) + sv * n);
        for (int k = 0; k < sweeps_; ++k) {
            T* o = c == x ? y : x;
            const bool last = k + 1 == sweeps_;
            if (l == 0 && last && fused_final) {
                with_visit(krylov_visit(), [&](auto V) {
                    launch_k(tuning_.pdl != 0, k_vc_jacobi_final<T, decltype(V)::value>, d.n_tiles_nc, kBlock, 0, s, 
                        A(0), d.tiles, st_, WD(0), r_, c, o, q_, red_, Control{n_active_, error_, tuning_.wait_polls}, flexible);
                });
                mark("smooth_dot", l, spmv_b(d.a, n, n) + sv * n + sb * n + (flexible ? 8.0 * n : 0.0));
            } else if (l == 0) {
                with_visit(ta.visit, [&](auto V) { launch_k(tuning_.pdl != 0, k_vc_jacobi<T, double, decltype(V)::value>, ta.second, ta.block, 0, s, A(l), ta.first, stv, WD(l), r_, c, o); });
                mark("smooth", l, spmv_b(d.a, n, n) + sv * n + sb * n);
            } else {
                with_visit(ta.visit, [&](auto V) { launch_k(tuning_.pdl != 0, k_vc_jacobi<T, T, decltype(V)::value>, ta.second, ta.block, 0, s, A(l), ta.first, stv, WD(l), Bv(l), c, o); });
                mark("smooth", l, spmv_b(d.a, n, n) + sv * n + sb * n);
            }
            c = o;
        }
    }
}

void Engine::enqueue_vcycle(Mode mode, bool fused_final, int flexible, bool x1_ready0) {
    if (mode == Mode::AmgMixed) enqueue_vcycle_t<float>(fused_final, flexible, x1_ready0);
    else enqueue_vcycle_t<double>(fused_final, flexible, x1_ready0);
}

// Preconditioner output z (level-0 iterate) in the precision of the mode.
void Engine::enqueue_init(Mode mode) {
    const DevLevel& d = lv_[0];
    const Control ctl{n_active_, error_, tuning_.wait_polls};
    const double n = d.n_rows;
    const double a0 = static_cast<double>(d.a.nnz) * 12.0 + 4.0 * (n + 1.0) + 16.0 * n;
    const X1Out x1o = x1_out(mode);
    const double x1b = (mode == Mode::AmgMixed ? 8.0 : 16.0) * x1o.n;
    with_visit(krylov_visit(), [&](auto V) {
        launch_k(tuning_.pdl != 0, k_cg_init<decltype(V)::value>, d.n_tiles, kBlock, 0, stream_, d.a.s64, d.tiles, st_, b_, x_, r_, red_, ctl, x1o);
    });
    mark("cg_init", 0, a0 + 16.0 * n + x1b);
    const int flexible = mode == Mode::AmgMixed ? 1 : 0;
    if (mode == Mode::Jacobi) {
        launch_k(tuning_.pdl != 0, k_cg_rz<double>, d.n_tiles, kBlock, 0, stream_, d.tiles, st_, r_, d.x64, dinv0_, nullptr, q_, red_, ctl, 0);
        mark("cg_rz", 0, 24.0 * n);
        return;
    }
    enqueue_vcycle(mode, fused_final_, flexible, x1o.n > 0);
    if (!fused_final_) enqueue_rz(mode, flexible);
}

void Engine::enqueue_rz(Mode mode, int flexible) {
    const DevLevel& d = lv_[0];
    const Control ctl{n_active_, error_, tuning_.wait_polls};
    const double n = d.n_rows;
    if (mode == Mode::AmgMixed) {
        launch_k(tuning_.pdl != 0, k_cg_rz<float>, d.n_tiles, kBlock, 0, stream_, d.tiles, st_, r_, d.x32, nullptr, dinv0_, q_, red_, ctl, flexible);
        mark("cg_rz", 0, 12.0 * n + (flexible ? 8.0 * n : 0.0));
    } else {
        launch_k(tuning_.pdl != 0, k_cg_rz<double>, d.n_tiles, kBlock, 0, stream_, d.tiles, st_, r_, d.x64, nullptr, dinv0_, q_, red_, ctl, flexible);
        mark("cg_rz", 0, 16.0 * n + (flexible ? 8.0 * n : 0.0));
    }
}

// Shared-memory budget of the staged SpMV's buffers: two CTAs per SM whatever the buffer count.
constexpr int kStageBytes = 96 * 1024;

template <int S> constexpr int stage_limit() { return kStageBytes / (S * 12) / 32 * 32; }

// The staged level-0 Krylov SpMV runs when Tuning.krylov_stage asks for it and the operator
// allows it: SELL, values and columns 16-byte aligned (bulk copies). Its buffers hold the
// widest 8-slice chunk up to the budget (wider chunks are summed from global memory). The
// kernels' shared-memory limit is always set to the budget, so that engines sharing them in one
// process never lower it for one another.
void Engine::prepare_stage() {
    stage_cap_ = 0;
    const int S = tuning_.krylov_stage;
    const DevSell64_32& a = lv_[0].a;
    if (S < 2 || S > 4 || a.s64.fmt != kFmtSell || a.max8_slots <= 0) return;
    if ((reinterpret_cast<uintptr_t>(a.s64.val) | reinterpret_cast<uintptr_t>(a.s64.col)) % 16 != 0) return;
    int limit = 0;
    if (S == 2) {
        limit = stage_limit<2>();
        CFDB_CUDA(cudaFuncSetAttribute(k_cg_spmv_pq_staged<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * limit * 12));
    } else if (S == 3) {
        limit = stage_limit<3>();
        CFDB_CUDA(cudaFuncSetAttribute(k_cg_spmv_pq_staged<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, 3 * limit * 12));
    } else {
        limit = stage_limit<4>();
        CFDB_CUDA(cudaFuncSetAttribute(k_cg_spmv_pq_staged<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, 4 * limit * 12));
    }
    stage_cap_ = std::min(round_up(a.max8_slots, 32), limit);
}

void Engine::enqueue_iteration(Mode mode) {
    const DevLevel& d = lv_[0];
    const Control ctl{n_active_, error_, tuning_.wait_polls};
    const double n = d.n_rows;
    const double a0 = static_cast<double>(d.a.nnz) * 12.0 + 4.0 * (n + 1.0) + 16.0 * n;
    if (mode == Mode::AmgMixed) {
        launch_k(tuning_.pdl != 0, k_cg_pupdate<float>, d.n_tiles, kBlock, 0, stream_, d.tiles, st_, d.x32, r_, dinv0_, p_);
        mark("cg_p_update", 0, 20.0 * n);
    } else {
        launch_k(tuning_.pdl != 0, k_cg_pupdate<double>, d.n_tiles, kBlock, 0, stream_, d.tiles, st_, d.x64, r_, dinv0_, p_);
        mark("cg_p_update", 0, 24.0 * n);
    }
    if (stage_cap_ > 0) {
        const size_t smem = static_cast<size_t>(tuning_.krylov_stage) * stage_cap_ * 12;
        auto staged = [&](auto kernel) {
            launch_k(tuning_.pdl != 0, kernel, d.n_tiles, kBlock, smem, stream_, d.a.s64, d.tiles, st_, p_, q_, red_, ctl,
                     stage_cap_);
        };
        if (tuning_.krylov_stage == 2) staged(k_cg_spmv_pq_staged<2>);
        else if (tuning_.krylov_stage == 3) staged(k_cg_spmv_pq_staged<3>);
        else staged(k_cg_spmv_pq_staged<4>);
    } else {
        with_visit(krylov_visit(), [&](auto V) {
            launch_k(tuning_.pdl != 0, k_cg_spmv_pq<decltype(V)::value>, d.n_tiles, kBlock, 0, stream_, d.a.s64, d.tiles, st_, p_, q_, red_, ctl);
        });
    }
    mark("cg_spmv_pq", 0, a0);
    const X1Out x1o = x1_out(mode);
    const double x1b = (mode == Mode::AmgMixed ? 8.0 : 16.0) * x1o.n;
    {
        const int vt = mode == Mode::AmgMixed ? 1 : 0;
        if (x1o.n > 0 && x1o.x32 != nullptr)
            launch_k(tuning_.pdl != 0, k_cg_xr<1>, d.n_tiles, kBlock, 0, stream_, d.tiles, st_, x_, r_, p_, q_, red_, ctl, vt, x1o);
        else if (x1o.n > 0 && x1o.x64 != nullptr)
            launch_k(tuning_.pdl != 0, k_cg_xr<2>, d.n_tiles, kBlock, 0, stream_, d.tiles, st_, x_, r_, p_, q_, red_, ctl, vt, x1o);
        else
            launch_k(tuning_.pdl != 0, k_cg_xr<0>, d.n_tiles, kBlock, 0, stream_, d.tiles, st_, x_, r_, p_, q_, red_, ctl, vt, x1o);
    }
    mark("cg_xr", 0, 48.0 * n + x1b);
    if (mode == Mode::AmgMixed) {
        with_visit(krylov_visit(), [&](auto V) {
            launch_k(tuning_.pdl != 0, k_cg_true_check<decltype(V)::value>, d.n_tiles, kBlock, 0, stream_, d.a.s64, d.tiles, st_, b_, x_, r_,
                                                                               red_, ctl, x1o);
        });
        mark("cg_true_check", 0, 0.0);
    }
    const int flexible = mode == Mode::AmgMixed ? 1 : 0;
    if (mode == Mode::Jacobi) {
        launch_k(tuning_.pdl != 0, k_cg_rz<double>, d.n_tiles, kBlock, 0, stream_, d.tiles, st_, r_, d.x64, dinv0_, nullptr, q_, red_, ctl, 0);
        mark("cg_rz", 0, 24.0 * n);
        return;
    }
    enqueue_vcycle(mode, fused_final_, flexible, x1o.n > 0);
    if (!fused_final_) enqueue_rz(mode, flexible);
}

void Engine::mark(const char* name, int level, double bytes) {
    if (prof_ == nullptr) return;
    cudaEvent_t e = nullptr;
    CFDB_CUDA(cudaEventCreate(&e));
    CFDB_CUDA(cudaEventRecord(e, stream_));
    ProfRecord r{};
    std::snprintf(r.name, sizeof(r.name), "%s", name);
    r.level = level;
    r.bytes = bytes;
    prof_->push_back({r, e});
}

std::vector<ProfRecord> Engine::profile(Mode mode, int reps) {
    CFDB_CUDA(cudaSetDevice(device_));
    if (mode != Mode::Jacobi && !has_amg_) fail(5, "profile: no AMG hierarchy set");
    if (mode == Mode::AmgMixed) prepare_tail<float>();
    else if (mode == Mode::AmgFp64) prepare_tail<double>();
    prepare_stage();
    std::vector<ProfRecord> out;
    std::vector<int> count;
    // b = 1 on every real row, x = 0: a nonzero residual whatever the engine held before (the
    // right-hand side and the guess are overwritten by the next solve anyway)
    {
        const int n = lv_[0].n_rows;
        launch_k(tuning_.pdl != 0, k_fill_rows, grid_of(n), 256, 0, stream_, n, row_map_, 1.0, b_);
        CFDB_CUDA(cudaMemsetAsync(x_, 0, sizeof(double) * n, stream_));
        launches_ += 1;
    }
    for (int rep = 0; rep < std::max(reps, 1); ++rep) {
        // every system active, never converging: the profiled kernels do all their work
        std::vector<SysState> hs(n_sys_);
        for (int s = 0; s < n_sys_; ++s) {
            SysState& t = hs[rank_[s]];
            std::memset(&t, 0, sizeof(t));
            t.tol = -1.0;
            t.max_it = 1 << 30;
            t.active = 1;
            t.first = 1;
            t.jacobi = mode != Mode::Jacobi && !single_.empty() && single_[s] ? 1 : 0;
        }
        CFDB_CUDA(cudaMemcpyAsync(st_, hs.data(), sizeof(SysState) * n_sys_, cudaMemcpyHostToDevice, stream_));
        const int n_act = n_sys_;
        CFDB_CUDA(cudaMemcpyAsync(n_active_, &n_act, sizeof(int), cudaMemcpyHostToDevice, stream_));
        std::vector<std::pair<ProfRecord, cudaEvent_t>> ev;
        prof_ = &ev;
        try {
            mark("start", 0, 0.0);
            enqueue_init(mode);
            mark("iteration_start", 0, 0.0);
            enqueue_iteration(mode);
        } catch (...) {
            prof_ = nullptr;
            for (auto& e : ev) cudaEventDestroy(e.second);
            throw;
        }
        prof_ = nullptr;
        CFDB_CUDA(cudaStreamSynchronize(stream_));
        if (rep == 0) {
            for (size_t i = 1; i < ev.size(); ++i) out.push_back(ev[i].first);
            count.assign(out.size(), 0);
        }
        for (size_t i = 1; i < ev.size() && i - 1 < out.size(); ++i) {
            float ms = 0.f;
            CFDB_CUDA(cudaEventElapsedTime(&ms, ev[i - 1].second, ev[i].second));
            if (rep > 0 || reps == 1) {
                out[i - 1].ms += ms;
                ++count[i - 1];
            }
        }
        for (auto& e : ev) cudaEventDestroy(e.second);
    }
    for (size_t i = 0; i < out.size(); ++i)
        if (count[i] > 0) out[i].ms /= count[i];
    return out;
}

void Engine::capture_graphs(Mode mode) {
    const int m = static_cast<int>(mode);
    if (graphs_[m][0] != nullptr) return;
    if (mode == Mode::AmgMixed) prepare_tail<float>();
    else if (mode == Mode::AmgFp64) prepare_tail<double>();
    prepare_stage();
    for (int which = 0; which < 2; ++which) {
        cudaGraph_t g = nullptr;
        CFDB_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        try {
            if (which == 0) enqueue_init(mode);
            else enqueue_iteration(mode);
        } catch (...) {
            cudaStreamEndCapture(stream_, &g);
            if (g != nullptr) cudaGraphDestroy(g);
            throw;
        }
        CFDB_CUDA(cudaStreamEndCapture(stream_, &g));
        size_t n_nodes = 0;
        CFDB_CUDA(cudaGraphGetNodes(g, nullptr, &n_nodes));
        std::vector<cudaGraphNode_t> nodes(n_nodes);
        CFDB_CUDA(cudaGraphGetNodes(g, nodes.data(), &n_nodes));
        int kernels = 0;
        for (auto nd : nodes) {
            cudaGraphNodeType t;
            CFDB_CUDA(cudaGraphNodeGetType(nd, &t));
            if (t == cudaGraphNodeTypeKernel) ++kernels;
        }
        graph_kernels_[m][which] = kernels;
        cudaGraphExec_t e = nullptr;
        const cudaError_t err = cudaGraphInstantiate(&e, g, 0);
        cudaGraphDestroy(g);
        CFDB_CUDA(err);
        graphs_[m][which] = e;
    }
}

std::vector<SolveResult> Engine::solve(Mode mode, const std::vector<SolveRequest>& req) {
    CFDB_CUDA(cudaSetDevice(device_));
    if (static_cast<int>(req.size()) != n_sys_) fail(1, "solve: one request per system expected");
    if (mode != Mode::Jacobi && !has_amg_) fail(5, "solve: no AMG hierarchy set");
    if (mode == Mode::AmgMixed && !need32_) fail(5, "solve: mixed precision needs the FP32 hierarchy");
    if (mode == Mode::AmgFp64 && !need64_) fail(5, "solve: FP64 AMG needs the FP64 hierarchy");
    std::vector<SysState> hs(n_sys_);
    int max_it = 0;
    for (int s = 0; s < n_sys_; ++s) {
        SysState& t = hs[rank_[s]];
        std::memset(&t, 0, sizeof(t));
        t.tol = req[s].tol;
        t.max_it = req[s].max_it;
        t.active = 1;
        t.first = 1;
        t.jacobi = mode != Mode::Jacobi && !single_.empty() && single_[s] ? 1 : 0;
        max_it = std::max(max_it, req[s].max_it);
    }
    capture_graphs(mode);
    CFDB_CUDA(cudaMemcpyAsync(st_, hs.data(), sizeof(SysState) * n_sys_, cudaMemcpyHostToDevice, stream_));
    const int n_act = n_sys_;
    CFDB_CUDA(cudaMemcpyAsync(n_active_, &n_act, sizeof(int), cudaMemcpyHostToDevice, stream_));
    CFDB_CUDA(cudaGraphLaunch(graphs_[static_cast<int>(mode)][0], stream_));
    launches_ += graph_kernels_[static_cast<int>(mode)][0];
    // Iterations: keep one graph launch in flight ahead of the convergence readback.
    cudaEvent_t ev[2];
    CFDB_CUDA(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
    CFDB_CUDA(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
    volatile int* flag = h_pinned_;
    int launched = 0;
    bool done = false;
    const int cap = max_it + 2;
    while (!done && launched < cap) {
        CFDB_CUDA(cudaGraphLaunch(graphs_[static_cast<int>(mode)][1], stream_));
        launches_ += graph_kernels_[static_cast<int>(mode)][1];
        CFDB_CUDA(cudaMemcpyAsync(h_pinned_ + 2 * (launched & 1), n_active_, sizeof(int), cudaMemcpyDeviceToHost,
                                  stream_));
        CFDB_CUDA(cudaMemcpyAsync(h_pinned_ + 2 * (launched & 1) + 1, error_, sizeof(int), cudaMemcpyDeviceToHost,
                                  stream_));
        CFDB_CUDA(cudaEventRecord(ev[launched & 1], stream_));
        ++launched;
        if (launched >= 2) {
            const int prev = (launched - 2) & 1;
            CFDB_CUDA(cudaEventSynchronize(ev[prev]));
            if (flag[2 * prev] <= 0 || flag[2 * prev + 1] != 0) done = true;
        }
    }
    CFDB_CUDA(cudaStreamSynchronize(stream_));
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    int err = 0;
    CFDB_CUDA(cudaMemcpy(&err, error_, sizeof(int), cudaMemcpyDeviceToHost));
    if (err != 0) {
        // an expired grid barrier leaves stale arrival counts: reset them with the flag, so
        // the next solve starts from a clean state
        CFDB_CUDA(cudaMemset(error_, 0, sizeof(int)));
        if (tail_bar_ != nullptr) CFDB_CUDA(cudaMemset(tail_bar_, 0, 2 * sizeof(unsigned)));
        fail(6, err == 2 ? "solve: a bounded device wait expired (persistent-tail grid barrier)"
                         : "solve: a bounded device wait expired (coarse-level staging)");
    }
    // true residual for reporting
    const DevLevel& d = lv_[0];
    with_visit(krylov_visit(), [&](auto V) {
        launch_k(tuning_.pdl != 0, k_true_residual<decltype(V)::value>, d.n_tiles, kBlock, 0, stream_, d.a.s64, d.tiles, st_, b_, x_, red_);
    });
    ++launches_;
    CFDB_CUDA(cudaGetLastError());
    CFDB_CUDA(cudaMemcpyAsync(hs.data(), st_, sizeof(SysState) * n_sys_, cudaMemcpyDeviceToHost, stream_));
    CFDB_CUDA(cudaStreamSynchronize(stream_));
    std::vector<SolveResult> out(n_sys_);
    for (int s = 0; s < n_sys_; ++s) {
        const SysState& t = hs[rank_[s]];
        SolveResult& o = out[s];
        o.iterations = t.active ? t.max_it : t.iters_out;
        o.residual = t.res;
        o.converged = t.converged != 0;
        o.true_residual = t.true_res;
    }
    return out;
}

void Engine::apply_vcycle(Mode mode, const std::vector<int>&) {
    if (!has_amg_) fail(5, "apply_vcycle: no hierarchy");
    if (mode == Mode::AmgMixed) prepare_tail<float>();
    else prepare_tail<double>();
    // run with all systems treated as active (state pointer null) and no Krylov bookkeeping
    SysState* keep = st_;
    st_ = nullptr;
    try {
        if (mode == Mode::AmgMixed) enqueue_vcycle_t<float>(false, 0, false);
        else enqueue_vcycle_t<double>(false, 0, false);
    } catch (...) {
        st_ = keep;
        throw;
    }
    st_ = keep;
    CFDB_CUDA(cudaGetLastError());
    CFDB_CUDA(cudaStreamSynchronize(stream_));
}

double Engine::time_sweep(int level, int reps, double* bytes) {
    if (level < 0 || level >= n_levels_ || reps < 1) fail(1, "time_sweep: bad level or reps");
    const DevLevel& d = lv_[level];
    const bool fp32 = need32_;
    const DevSell64_32& m = d.a;
    const bool nc = level + 1 < n_levels_;
    const Tiles tiles = m.tiles;
    const int grid = nc ? m.n_tiles_nc : m.n_tiles;
    if (grid == 0) fail(1, "time_sweep: level has no operator tiles");
    const int visit = vcycle_visit(m);
    const double sv = fp32 ? 4.0 : 8.0;
    const double sb = level == 0 ? 8.0 : sv;
    const double n = d.n_rows_nc;
    const double cb = fp32 && m.s32.c16 != nullptr ? 2.0 : 4.0;
    if (bytes != nullptr) *bytes = static_cast<double>(m.nnz) * (sv + cb) + 4.0 * (n + 1.0) + 3.0 * sv * n + sb * n;
    cudaEvent_t a, b;
    CFDB_CUDA(cudaEventCreate(&a));
    CFDB_CUDA(cudaEventCreate(&b));
    auto launch = [&](auto tag) {
        using T = decltype(tag);
        const Sell<T> op = vs_sel<T>(m.s64, m.s32);
        const T* wd = nullptr;
        T *x, *y;
        if constexpr (sizeof(T) == 8) {
            wd = d.wd64;
            x = d.x64;
            y = d.y64;
        } else {
            wd = d.wd32;
            x = d.x32;
            y = d.y32;
        }
        with_visit(visit, [&](auto V) {
            if (level == 0) {
                launch_k(tuning_.pdl != 0, k_vc_jacobi<T, double, decltype(V)::value>, grid, m.block, 0, stream_, op, tiles, nullptr, wd, r_, x, y);
            } else {
                const T* bv;
                if constexpr (sizeof(T) == 8) bv = d.b64;
                else bv = d.b32;
                launch_k(tuning_.pdl != 0, k_vc_jacobi<T, T, decltype(V)::value>, grid, m.block, 0, stream_, op, tiles, nullptr, wd, bv, x, y);
            }
        });
    };
    for (int w = 0; w < 2; ++w) fp32 ? launch(0.0f) : launch(0.0); // warm-up
    CFDB_CUDA(cudaEventRecord(a, stream_));
    for (int i = 0; i < reps; ++i) fp32 ? launch(0.0f) : launch(0.0);
    CFDB_CUDA(cudaEventRecord(b, stream_));
    CFDB_CUDA(cudaEventSynchronize(b));
    CFDB_CUDA(cudaGetLastError());
    float ms = 0.f;
    CFDB_CUDA(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms / reps;
}

double Engine::time_level0_sweep(bool fp32, int reps) {
    const DevLevel& d = lv_[0];
    cudaEvent_t a, b;
    CFDB_CUDA(cudaEventCreate(&a));
    CFDB_CUDA(cudaEventCreate(&b));
    CFDB_CUDA(cudaEventRecord(a, stream_));
    for (int i = 0; i < reps; ++i) {
        if (fp32) {
            launch_k(tuning_.pdl != 0, k_vc_jacobi<float, double, kVisitSell2>, d.n_tiles, kBlock, 0, stream_, d.a.s32, d.tiles, nullptr, d.wd32, r_,
                                                                         d.x32, d.y32);
        } else {
            launch_k(tuning_.pdl != 0, k_vc_jacobi<double, double, kVisitSell2>, d.n_tiles, kBlock, 0, stream_, d.a.s64, d.tiles, nullptr, d.wd64, r_,
                                                                          d.x64, d.y64);
        }
    }
    CFDB_CUDA(cudaEventRecord(b, stream_));
    CFDB_CUDA(cudaEventSynchronize(b));
    float ms = 0.f;
    CFDB_CUDA(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms / reps;
}

} // namespace cfdb
