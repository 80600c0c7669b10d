// Smoothed-aggregation AMG setup on the device (see dsetup.hpp).
//
// Per level (amg.cpp:122-190, in the host build's rounding order):
//   d      last diagonal entry of each row (amg.cpp:82-92)
//   S      strength graph: i != j and |a_ij| > theta sqrt|d_i d_j| (amg.cpp:22-27)
//   agg    aggregation passes 1-2 on the device (k_seed_sweep, k_pass2); a level with rows left
//          for pass 3 is read back and aggregated on the host (amg.cpp:12-78)
//   inv    1/d or 0; rho = max_i |inv_i| sum_j |a_ij|; omega = 4 / (3 rho) (amg.cpp:150-166)
//   C      (D^-1 A) P_tent: row i accumulates inv_i a_ik into column agg(k), k ascending
//   P      P_tent - omega C over the union pattern, exact zeros dropped (amg.cpp:168-172)
//   R      P^T, each row's columns ascending (amg.cpp:175)
//   A_c    R (A P), exact zeros dropped (amg.cpp:176-178)
//
// Sparse products are Gustavson row products. The host sums row i's contributions in the order
// (k ascending over A(i,:), then B(k,:) in column order), the first one assigning. Here a group
// of threads (a warp, or a CTA for long rows) owns one row and walks A(i,:) one k at a time:
// within one k the columns of B(k,:) are distinct, so the group's threads update distinct
// accumulators, and the group synchronises between k. Every accumulator therefore sees its
// contributions in exactly the host order. Accumulators live in an open-addressing table
// (shared memory, or device memory for the rare rows too long for it), sized from a symbolic
// pass; a bitonic sort of the table then yields the row's columns in ascending order.
#include "dsetup.hpp"

#include <algorithm>
#include <climits>
#include <cstring>

namespace cfdb {

void* Scratch::raw(size_t bytes) {
    bytes = (bytes + 255) & ~static_cast<size_t>(255);
    if (chunks_.empty() || chunks_.back().used + bytes > chunks_.back().buf.bytes()) {
        const size_t last = chunks_.empty() ? 0 : chunks_.back().buf.bytes();
        const size_t sz = std::max({bytes, 2 * last, static_cast<size_t>(4) << 20});
        chunks_.emplace_back();
        chunks_.back().buf.allocate(sz, /*transient=*/true);
        total_ += sz;
    }
    Chunk& c = chunks_.back();
    void* p = static_cast<char*>(c.buf.get()) + c.used;
    c.used += bytes;
    return p;
}

namespace {

constexpr int kEmpty = INT_MAX; // free table slot; sorts after every column index
constexpr int kErrInternal = 7; // CFDB_ERR_INTERNAL
constexpr int kThreads = 256;

template <int G> __device__ __forceinline__ void group_sync() {
    if constexpr (G == 32) {
        __syncwarp();
    } else {
        __syncthreads();
    }
}

__device__ __forceinline__ unsigned slot_of(int key, int cap) {
    return (static_cast<unsigned>(key) * 0x9E3779B1u) & static_cast<unsigned>(cap - 1);
}

int grid_for(long long n, int threads = kThreads) {
    return static_cast<int>(std::max<long long>(1, (n + threads - 1) / threads));
}

size_t aligned(size_t bytes) { return (bytes + 255) & ~static_cast<size_t>(255); }

int next_pow2(long long v) {
    long long p = 1;
    while (p < v) p <<= 1;
    if (p > (1LL << 30)) fail(1, "device AMG setup: row too long for a hash table");
    return static_cast<int>(p);
}

// ---------------------------------------------------------------------------------------------
// exclusive scan of int counts (n + 1 outputs, the last = total), 64-bit internally
// ---------------------------------------------------------------------------------------------

constexpr int kScanThreads = 1024;
constexpr int kScanChunk = 2 * kScanThreads;

__device__ long long block_exclusive_scan(long long v, long long* sh, long long* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    long long x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[w] = x;
    __syncthreads();
    if (w == 0) {
        long long s = lane < nw ? sh[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const long long y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) sh[lane] = s;
    }
    __syncthreads();
    const long long before = w > 0 ? sh[w - 1] : 0;
    if (total != nullptr) *total = sh[nw - 1];
    __syncthreads();
    return before + x - v;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_sums(const int* __restrict__ in, int n, long long* bsum) {
    __shared__ long long sh[32];
    const long long i0 = static_cast<long long>(blockIdx.x) * kScanChunk + 2 * threadIdx.x;
    const long long v = (i0 < n ? in[i0] : 0) + (i0 + 1 < n ? in[i0 + 1] : 0);
    long long total = 0;
    block_exclusive_scan(v, sh, &total);
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// Single CTA: block sums -> exclusive block offsets (in place); total and out[n].
__global__ void __launch_bounds__(kScanThreads) k_scan_top(long long* bsum, int nb, long long* total_out, int* out_n) {
    __shared__ long long sh[32];
    const int per = (nb + kScanThreads - 1) / kScanThreads;
    const int b0 = min(nb, static_cast<int>(threadIdx.x) * per), b1 = min(nb, b0 + per);
    long long s = 0;
    for (int b = b0; b < b1; ++b) s += bsum[b];
    long long total = 0;
    long long run = block_exclusive_scan(s, sh, &total);
    for (int b = b0; b < b1; ++b) {
        const long long v = bsum[b];
        bsum[b] = run;
        run += v;
    }
    if (threadIdx.x == 0) {
        *total_out = total;
        *out_n = static_cast<int>(total > INT_MAX ? INT_MAX : total);
    }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const int* __restrict__ in, int n,
                                                             const long long* __restrict__ boff, int* out) {
    __shared__ long long sh[32];
    const long long i0 = static_cast<long long>(blockIdx.x) * kScanChunk + 2 * threadIdx.x;
    const long long v0 = i0 < n ? in[i0] : 0, v1 = i0 + 1 < n ? in[i0 + 1] : 0;
    const long long base = boff[blockIdx.x] + block_exclusive_scan(v0 + v1, sh, nullptr);
    if (i0 < n) out[i0] = static_cast<int>(base);
    if (i0 + 1 < n) out[i0 + 1] = static_cast<int>(base + v0);
}

// ---------------------------------------------------------------------------------------------
// level kernels
// ---------------------------------------------------------------------------------------------

__global__ void k_ldu_values(int n, int nf, const int* __restrict__ dpos, const int* __restrict__ upos,
                             const int* __restrict__ lpos, const double* __restrict__ d,
                             const double* __restrict__ u, const double* __restrict__ l, double* va) {
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < n) va[dpos[t]] = d[t];
    if (t < nf) {
        va[upos[t]] = u[t];
        va[lpos[t]] = l[t];
    }
}

// last diagonal entry of each row (any value), 0 if none
__global__ void k_last_diag(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                            const double* __restrict__ va, double* d) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k)
        if (ci[k] == i) v = va[k];
    d[i] = v;
}

__device__ __forceinline__ bool strong_entry(int i, int j, double v, double di, const double* d, double theta) {
    return i != j && fabs(v) > __dmul_rn(theta, __dsqrt_rn(fabs(__dmul_rn(di, d[j]))));
}

// FILL = false: number of strong entries per row; true: their columns and |a_ij|
template <bool FILL>
__global__ void k_strong(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                         const double* __restrict__ va, const double* __restrict__ d, double theta, int* cnt,
                         const int* __restrict__ srp, int* sci, double* sav) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double di = d[i];
    int c = 0;
    const int o = FILL ? srp[i] : 0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
        const int j = ci[k];
        if (strong_entry(i, j, va[k], di, d, theta)) {
            if (FILL) {
                sci[o + c] = j;
                sav[o + c] = fabs(va[k]);
            }
            ++c;
        }
    }
    if (!FILL) cnt[i] = c;
}

// rank of each strong entry within its row by (|a| descending, position ascending); rows have
// at most 4096 strong entries (checked by the host)
__global__ void k_strong_rank(int n, const int* __restrict__ srp, const double* __restrict__ sav, uint16_t* rank) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int b = srp[i], e = srp[i + 1];
    for (int k = b; k < e; ++k) {
        const double v = sav[k];
        int r = 0;
        for (int q = b; q < e; ++q) {
            const double w = sav[q];
            r += (w > v) || (w == v && q < k);
        }
        rank[k] = static_cast<uint16_t>(r);
    }
}

__global__ void k_max_degree(int n, const int* __restrict__ srp, int* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) atomicMax(out, srp[i + 1] - srp[i]);
}

// ---- aggregation passes 1 and 2 (amg.cpp:20-64) on the device ----
// Pass 1 visits the rows in order and makes row i a seed when it has a strong connection and
// neither i nor any strong neighbour is aggregated yet; a seed aggregates itself and its strong
// neighbours. With N[i] = {i} u S(i) (S: the strong connections of row i), row i is therefore a
// seed exactly when it has a strong connection and no earlier seed s has N[s] meeting N[i]: the
// seeds are the lexicographically first maximal independent set of that conflict relation over
// the rows with strong connections. Sweeps resolve it in parallel: row i becomes a seed once
// every earlier row s whose N[s] meets N[i] is known not to be one, and not a seed as soon as
// one of them is. Both outcomes are final and follow from final states only, so a sweep may
// read states written during the same sweep (Gauss-Seidel order across CTAs helps, nothing
// relies on it); the smallest undecided row always decides, so the sweeps end, with the
// sequential result. The rows s whose N[s] contains j are j itself and the transpose of S at j.
// Decisions happen only near the smallest undecided row `lo` (a seed needs every earlier
// conflict decided), so a sweep visits the window [lo, lo + kSeedWindow) and records the next
// lo; sweeps run in batches on the device, the host reading lo once per batch.
enum : int { kUndecided = 0, kSeed = 1, kNotSeed = 2 };

__global__ void k_seed_init(int n, const int* __restrict__ srp, int* state) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) state[i] = srp[i + 1] > srp[i] ? kUndecided : kNotSeed;
}

constexpr int kSeedWindow = 1 << 18;
constexpr int kSeedBatch = 32;  // sweeps per host check

// One sweep over the rows [lo, lo + kSeedWindow), lo = *lo_in (every row below it is decided);
// *lo_out receives the smallest row still undecided, or lo + kSeedWindow when the window
// settled (*lo_out preset to INT_MAX). trp / tci: the transpose of S, rows ascending. For each
// j in N[i] the earlier rows s with j in N[s] are scanned in ascending order up to the first one
// not known to be a non-seed: a seed decides row i at once; an undecided one makes row i wait,
// and the scan moves on to the next j, where a seed may still decide it.
__global__ void k_seed_sweep(int n, const int* __restrict__ lo_in, int* lo_out, const int* __restrict__ srp,
                             const int* __restrict__ sci, const int* __restrict__ trp, const int* __restrict__ tci,
                             int* state_) {
    const int lo = *lo_in;
    if (blockIdx.x == 0 && threadIdx.x == 0)
        atomicMin(lo_out, static_cast<int>(min(static_cast<long long>(lo) + kSeedWindow, static_cast<long long>(n))));
    const long long ii = static_cast<long long>(lo) + static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (ii >= n) return;
    const int i = static_cast<int>(ii);
    volatile int* state = state_;
    if (state[i] != kUndecided) return;
    bool waiting = false;
    for (int k = srp[i] - 1; k < srp[i + 1]; ++k) {
        const int j = k < srp[i] ? i : sci[k];
        if (j < i) {  // s = j itself
            const int v = state[j];
            if (v == kSeed) {
                state[i] = kNotSeed;
                return;
            }
            if (v == kUndecided) {
                waiting = true;
                continue;
            }
        }
        for (int q = trp[j]; q < trp[j + 1]; ++q) {
            const int s = tci[q];
            if (s >= i) break;
            const int v = state[s];
            if (v == kSeed) {
                state[i] = kNotSeed;
                return;
            }
            if (v == kUndecided) {
                waiting = true;
                break;
            }
        }
    }
    if (waiting) atomicMin(lo_out, i);
    else state[i] = kSeed;
}

__global__ void k_seed_flags(int n, const int* __restrict__ state, int* flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flag[i] = state[i] == kSeed ? 1 : 0;
}

// Aggregate of every row after pass 1: that of the one seed s with the row in N[s], else -1.
// Seeds are numbered in row order (id: exclusive scan of the seed flags).
__global__ void k_pass1_cover(int n, const int* __restrict__ trp, const int* __restrict__ tci,
                              const int* __restrict__ state, const int* __restrict__ id, int* agg1) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int a = state[i] == kSeed ? id[i] : -1;
    for (int q = trp[i]; q < trp[i + 1] && a < 0; ++q) {
        const int s = tci[q];
        if (state[s] == kSeed) a = id[s];
    }
    agg1[i] = a;
}

// Pass 2 (amg.cpp:49-63): a row without aggregate joins that of its strongest strong neighbour
// aggregated in pass 1 (the first in row order among equal |a_ij|; sav holds |a_ij|). Rows
// still without one are left for pass 3 and counted.
__global__ void k_pass2(int n, const int* __restrict__ srp, const int* __restrict__ sci,
                        const double* __restrict__ sav, const int* __restrict__ agg1, int* agg, int* left) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int a = agg1[i];
    if (a < 0) {
        double best = 0.0;
        for (int k = srp[i]; k < srp[i + 1]; ++k) {
            const int g = agg1[sci[k]];
            if (g >= 0 && sav[k] > best) {
                best = sav[k];
                a = g;
            }
        }
        if (a < 0) atomicAdd(left, 1);
    }
    agg[i] = a;
}

__global__ void k_left_flags(int n, const int* __restrict__ agg, int* flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flag[i] = agg[i] < 0 ? 1 : 0;
}

__global__ void k_left_list(int n, const int* __restrict__ agg, const int* __restrict__ pos, int* list) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && agg[i] < 0) list[pos[i]] = i;
}

// Pass 3 (amg.cpp:66-76) when few rows are left: one thread walks them in row order; a row still
// without an aggregate opens the next one and takes its strong neighbours still without one.
__global__ void k_pass3(int n_left, const int* __restrict__ list, const int* __restrict__ srp,
                        const int* __restrict__ sci, int* agg, int* n_agg) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int a = *n_agg;
    for (int t = 0; t < n_left; ++t) {
        const int i = list[t];
        if (agg[i] >= 0) continue;
        agg[i] = a;
        for (int k = srp[i]; k < srp[i + 1]; ++k)
            if (agg[sci[k]] < 0) agg[sci[k]] = a;
        ++a;
    }
    *n_agg = a;
}

// inv = 1/d (0 where d == 0); rho = max_i |inv_i| sum_j |a_ij| (bits of a non-negative double)
__global__ void k_inv_rho(int n, const int* __restrict__ rp, const double* __restrict__ va,
                          const double* __restrict__ d, double* inv, unsigned long long* rho_bits) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double di = d[i];
    const double iv = di != 0.0 ? __ddiv_rn(1.0, di) : 0.0;
    inv[i] = iv;
    double row = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) row = __dadd_rn(row, fabs(va[k]));
    const double v = __dmul_rn(row, fabs(iv));
    if (v > 0.0) atomicMax(rho_bits, static_cast<unsigned long long>(__double_as_longlong(v)));
}

// ---------------------------------------------------------------------------------------------
// Gustavson products
// ---------------------------------------------------------------------------------------------

struct GemmArgs {
    const int* arp;
    const int* aci;
    const double* ava;
    const double* ascale; // per row of A (null: 1)
    const int* brp;       // null: B is the tentative prolongator, row k = (tent[k], 1.0)
    const int* bci;
    const double* bva;
    const int* tent;
    const int* rows;      // the rows of this launch
    int n_list;
    int* cnt;             // symbolic: distinct columns per row
    int* over_rows;       // symbolic, table-limited launch: rows whose table filled
    int* n_over;
    int limit;            // symbolic: most distinct columns a table may take
    const int* crp;       // numeric output
    int* cci;
    double* cva;
    int* err;
    // device-memory tables, one row per CTA: offset and capacity per list position
    const long long* goff;
    const int* gcap;
    int* gkeys;
    double* gvals;
};

template <int G> __device__ void bitonic_sort(int* keys, double* vals, int cap, int t) {
    for (int k = 2; k <= cap; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int s = t; s < cap; s += G) {
                const int p = s ^ j;
                if (p > s) {
                    const int ks = keys[s], kp = keys[p];
                    const bool asc = (s & k) == 0;
                    if (ks != kp && (ks > kp) == asc) {
                        keys[s] = kp;
                        keys[p] = ks;
                        if (vals != nullptr) {
                            const double v = vals[s];
                            vals[s] = vals[p];
                            vals[p] = v;
                        }
                    }
                }
            }
            group_sync<G>();
        }
    }
}

// Moves the occupied slots (key != kEmpty) of a table to its front, keeping their order, and
// returns their number. wc: G / 32 ints of shared memory (G > 32).
template <int G> __device__ int compact_front(int* keys, double* vals, int cap, int t, int* wc) {
    int base = 0;
    const int lane = t & 31, w = t >> 5;
    const unsigned below = (1u << lane) - 1u;
    for (int s0 = 0; s0 < cap; s0 += G) {
        const int s = s0 + t;
        const int key = s < cap ? keys[s] : kEmpty;
        const bool occ = key != kEmpty;
        const double val = occ ? vals[s] : 0.0;
        const unsigned bal = __ballot_sync(0xffffffffu, occ);
        int pos, total;
        if constexpr (G == 32) {
            pos = base + __popc(bal & below);
            total = __popc(bal);
        } else {
            if (lane == 0) wc[w] = __popc(bal);
            __syncthreads();
            int before = 0;
            total = 0;
            for (int q = 0; q < G / 32; ++q) {
                const int c = wc[q];
                if (q < w) before += c;
                total += c;
            }
            pos = base + before + __popc(bal & below);
        }
        group_sync<G>(); // the chunk is read before any of it is overwritten (pos <= s)
        if (occ) {
            keys[pos] = key;
            vals[pos] = val;
        }
        base += total;
        group_sync<G>();
    }
    return base;
}

// One row per group of G threads, PER groups per CTA. CAP > 0: table of CAP slots in shared
// memory; CAP == 0: table in device memory (g.gkeys / g.gvals at g.goff, g.gcap slots).
// Symbolic (NUMERIC = false): counts distinct columns; with LIMIT, a row whose count passes
// 3/4 of the table is recorded in g.over_rows instead. Numeric: accumulates and writes the
// sorted row at g.crp[i].
template <bool NUMERIC, int G, int CAP, int PER>
__global__ void __launch_bounds__(G* PER) k_gemm_rows(GemmArgs g) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_count[PER];
    __shared__ int s_over[PER];
    __shared__ int s_wc[G > 32 ? G / 32 : 1];
    const int grp = threadIdx.x / G, t = threadIdx.x % G;
    const int pos = blockIdx.x * PER + grp;
    if (pos >= g.n_list) return; // whole groups only
    const int i = g.rows[pos];
    int cap = CAP;
    int* keys;
    double* vals = nullptr;
    double* sv = nullptr; // warp groups, numeric: the chunk's contributions, one per lane
    if constexpr (CAP > 0) {
        if constexpr (NUMERIC) {
            double* base = reinterpret_cast<double*>(smem);
            vals = base + static_cast<size_t>(grp) * CAP;
            if constexpr (G == 32) {
                sv = base + static_cast<size_t>(PER) * CAP + grp * 32;
                keys = reinterpret_cast<int*>(base + static_cast<size_t>(PER) * (CAP + 32)) + grp * CAP;
            } else {
                keys = reinterpret_cast<int*>(base + static_cast<size_t>(PER) * CAP) + grp * CAP;
            }
        } else {
            keys = reinterpret_cast<int*>(smem) + grp * CAP;
        }
    } else {
        cap = g.gcap[pos];
        keys = g.gkeys + g.goff[pos];
        if constexpr (NUMERIC) vals = g.gvals + g.goff[pos];
    }
    for (int s = t; s < cap; s += G) keys[s] = kEmpty;
    if (t == 0) {
        s_count[grp] = 0;
        s_over[grp] = 0;
    }
    group_sync<G>();
    const int limit = min(g.limit, cap - cap / 4);
    const int a0 = g.arp[i], a1 = g.arp[i + 1];
    // slot of key j (inserted when absent; fresh = inserted now), or -1 when the table is full
    auto find = [&](int j, bool& fresh) -> int {
        unsigned h = slot_of(j, cap);
        for (int probes = 0; probes < cap; ++probes) {
            const int prev = atomicCAS(&keys[h], kEmpty, j);
            if (prev == kEmpty || prev == j) {
                fresh = prev == kEmpty;
                return static_cast<int>(h);
            }
            h = (h + 1) & static_cast<unsigned>(cap - 1);
        }
        return -1;
    };
    if constexpr (G == 32 && CAP > 0) {
        // Warp groups take the row's contributions 32 at a time in their order (k ascending
        // over A(i,:), then B(k,:)), whatever k-groups a chunk spans. Within a chunk, the lanes
        // holding one column are matched; the lowest of them adds their values in lane order.
        const unsigned full = 0xffffffffu;
        const int lane = t;
        for (int w0 = a0; w0 < a1; w0 += 32) {
            const int q = w0 + lane;
            int len = 0, bstart = 0;
            double av = 0.0;
            if (q < a1) {
                const int kk = g.aci[q];
                if (g.brp != nullptr) {
                    bstart = g.brp[kk];
                    len = g.brp[kk + 1] - bstart;
                } else {
                    bstart = kk;
                    len = 1;
                }
                if constexpr (NUMERIC) {
                    av = g.ava[q];
                    if (g.ascale != nullptr) av = __dmul_rn(g.ascale[i], av);
                }
            }
            int inc = len;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(full, inc, o);
                if (lane >= o) inc += y;
            }
            const int total = __shfl_sync(full, inc, 31);
            const int exc = inc - len;
            bool stop = false;
            for (int f0 = 0; f0 < total && !stop; f0 += 32) {
                const int f = f0 + lane;
                const bool active = f < total;
                int src = 0; // first lane whose inclusive prefix exceeds f
                for (int step = 16; step > 0; step >>= 1) {
                    const int v = __shfl_sync(full, inc, src + step - 1);
                    if (v <= f) src += step;
                }
                const int off = f - __shfl_sync(full, exc, src);
                const int kb = __shfl_sync(full, bstart, src) + off;
                const double avs = __shfl_sync(full, av, src);
                const int j = active ? (g.brp != nullptr ? g.bci[kb] : g.tent[kb]) : -1 - lane;
                if constexpr (NUMERIC) {
                    sv[lane] = active ? __dmul_rn(avs, g.brp != nullptr ? g.bva[kb] : 1.0) : 0.0;
                    const unsigned same = __match_any_sync(full, j);
                    __syncwarp();
                    if (active && lane == __ffs(same) - 1) {
                        bool fresh = false;
                        const int h = find(j, fresh);
                        if (h < 0) {
                            s_over[grp] = 1;
                        } else {
                            unsigned m = same & (same - 1u); // the others, ascending
                            double acc = fresh ? sv[lane] : __dadd_rn(vals[h], sv[lane]);
                            while (m != 0u) {
                                const int b = __ffs(m) - 1;
                                m &= m - 1u;
                                acc = __dadd_rn(acc, sv[b]);
                            }
                            vals[h] = acc;
                        }
                    }
                } else {
                    if (active) {
                        bool fresh = false;
                        const int h = find(j, fresh);
                        if (h < 0) s_over[grp] = 1;
                        else if (fresh) atomicAdd(&s_count[grp], 1);
                    }
                }
                __syncwarp();
                stop = s_over[grp] || (!NUMERIC && s_count[grp] > limit);
                __syncwarp(); // every lane has read the flags before any lane updates them again
            }
            if (stop) break; // uniform within the warp
        }
    } else {
        for (int ka = a0; ka < a1; ++ka) {
            const int k = g.aci[ka];
            double av = 0.0;
            if constexpr (NUMERIC) {
                av = g.ava[ka];
                if (g.ascale != nullptr) av = __dmul_rn(g.ascale[i], av);
            }
            const int b0 = g.brp != nullptr ? g.brp[k] : k;
            const int b1 = g.brp != nullptr ? g.brp[k + 1] : k + 1;
            for (int kb = b0 + t; kb < b1; kb += G) {
                const int j = g.brp != nullptr ? g.bci[kb] : g.tent[kb];
                bool fresh = false;
                const int h = find(j, fresh);
                if (h < 0) { // full table: symbolic overflow, numeric error
                    s_over[grp] = 1;
                    continue;
                }
                if constexpr (NUMERIC) {
                    const double c = __dmul_rn(av, g.brp != nullptr ? g.bva[kb] : 1.0);
                    vals[h] = fresh ? c : __dadd_rn(vals[h], c);
                } else {
                    if (fresh) atomicAdd(&s_count[grp], 1);
                }
            }
            group_sync<G>();
            const bool stop = s_over[grp] || (!NUMERIC && s_count[grp] > limit);
            group_sync<G>(); // every thread has read the flags before any thread updates them again
            if (stop) break; // uniform within the group
        }
    }
    if constexpr (!NUMERIC) {
        if (t == 0) {
            if (s_over[grp] || s_count[grp] > limit) {
                g.cnt[i] = 0;
                if (g.over_rows != nullptr) {
                    g.over_rows[atomicAdd(g.n_over, 1)] = i;
                } else {
                    atomicExch(g.err, 1);
                }
            } else {
                g.cnt[i] = s_count[grp];
            }
        }
    } else {
        if (s_over[grp]) {
            if (t == 0) atomicExch(g.err, 2);
            return;
        }
        // sort only the occupied slots: compact them, pad to a power of two, bitonic sort
        const int used = compact_front<G>(keys, vals, cap, t, s_wc);
        int p2 = 1;
        while (p2 < used) p2 <<= 1;
        for (int s = used + t; s < p2; s += G) keys[s] = kEmpty;
        group_sync<G>();
        bitonic_sort<G>(keys, vals, p2, t);
        const int c0 = g.crp[i], len = g.crp[i + 1] - c0;
        if (len != used) {
            if (t == 0) atomicExch(g.err, 3);
            return;
        }
        for (int s = t; s < len; s += G) {
            g.cci[c0 + s] = keys[s];
            g.cva[c0 + s] = vals[s];
        }
    }
}

// upper bound of the distinct columns of row i of A B: min(sum_k |B(k,:)|, n_cols)
__global__ void k_gemm_bound(int n, const int* __restrict__ arp, const int* __restrict__ aci,
                             const int* __restrict__ brp, int n_cols, int* ub) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    long long u = 0;
    for (int ka = arp[i]; ka < arp[i + 1]; ++ka) {
        const int k = aci[ka];
        u += brp != nullptr ? brp[k + 1] - brp[k] : 1;
    }
    ub[i] = static_cast<int>(u < n_cols ? u : n_cols);
}

// Table-size classes of a row (distinct columns, or entries of a row to sort), smallest first:
// (threads per row, shared-memory slots, rows per CTA); the last class uses device memory.
constexpr int kClasses = 6;
struct Limits {
    int lim[kClasses - 1]; // class q holds measures <= lim[q] (and > lim[q - 1])
};

// rows into classes by measure (lists[c * n + ...]); counts[c] rows in class c
__global__ void k_classify(int n, const int* __restrict__ m, Limits L, int* lists, int* counts) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int v = m[i];
    int c = kClasses - 1;
    for (int q = kClasses - 2; q >= 0; --q)
        if (v <= L.lim[q]) c = q;
    // one atomic per class present in the warp
    const int lane = threadIdx.x & 31;
    const unsigned same = __match_any_sync(__activemask(), c);
    const int leader = __ffs(same) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(&counts[c], __popc(same));
    base = __shfl_sync(same, base, leader);
    lists[static_cast<size_t>(c) * n + base + __popc(same & ((1u << lane) - 1u))] = i;
}

// rows of a list whose count is at most `lim` (symbolic retry: rows a smaller table rejected)
// smoothed prolongator rows from C = (D^-1 A) P_tent (sorted): count (FILL = false) or write
template <bool FILL>
__global__ void k_p_emit(int n, const int* __restrict__ crp, const int* __restrict__ cci,
                         const double* __restrict__ cva, const int* __restrict__ agg, double omega, int* pcnt,
                         const int* __restrict__ prp, int* pci, double* pva) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int tj = agg[i];
    const int o = FILL ? prp[i] : 0;
    int c = 0;
    bool used = false;
    auto emit = [&](int j, double v) {
        if (v != 0.0) {
            if (FILL) {
                pci[o + c] = j;
                pva[o + c] = v;
            }
            ++c;
        }
    };
    for (int q = crp[i]; q < crp[i + 1]; ++q) {
        const int j = cci[q];
        const double ws = __dmul_rn(omega, cva[q]);
        if (!used && tj < j) {
            emit(tj, 1.0);
            used = true;
        }
        if (j == tj) {
            emit(j, __dsub_rn(1.0, ws));
            used = true;
        } else {
            emit(j, __dsub_rn(0.0, ws));
        }
    }
    if (!used) emit(tj, 1.0);
    if (!FILL) pcnt[i] = c;
}

// transpose: column counts, scatter, then each row sorted by its (distinct) column
__global__ void k_col_count(long long nnz, const int* __restrict__ ci, int* cnt) {
    const long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e < nnz) atomicAdd(&cnt[ci[e]], 1);
}

__global__ void k_t_fill(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ va,
                         const int* __restrict__ trp, int* cursor, int* tci, double* tva) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
        const int j = ci[k];
        const int o = trp[j] + atomicAdd(&cursor[j], 1);
        tci[o] = i;
        tva[o] = va[k];
    }
}

__global__ void k_row_len(int n, const int* __restrict__ rp, int* len) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) len[i] = rp[i + 1] - rp[i];
}

// sorts rows of (ci, va) by ci; CAP > 0: in shared memory, else in device tables (gkeys/gvals)
template <int G, int CAP, int PER>
__global__ void __launch_bounds__(G* PER) k_seg_sort(const int* __restrict__ rows, int n_list, const int* __restrict__ rp,
                                                      int* ci, double* va, const long long* goff, const int* gcap,
                                                      int* gkeys, double* gvals) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int grp = threadIdx.x / G, t = threadIdx.x % G;
    const int pos = blockIdx.x * PER + grp;
    if (pos >= n_list) return;
    const int i = rows[pos];
    int cap = CAP;
    int* keys;
    double* vals;
    if constexpr (CAP > 0) {
        vals = reinterpret_cast<double*>(smem) + static_cast<size_t>(grp) * CAP;
        keys = reinterpret_cast<int*>(reinterpret_cast<double*>(smem) + static_cast<size_t>(PER) * CAP) + grp * CAP;
    } else {
        cap = gcap[pos];
        keys = gkeys + goff[pos];
        vals = gvals + goff[pos];
    }
    const int r0 = rp[i], len = rp[i + 1] - r0;
    if (len > cap) return; // classified by length: cannot happen
    int p2 = 1;
    while (p2 < len) p2 <<= 1;
    for (int s = t; s < p2; s += G) {
        keys[s] = s < len ? ci[r0 + s] : kEmpty;
        vals[s] = s < len ? va[r0 + s] : 0.0;
    }
    group_sync<G>();
    bitonic_sort<G>(keys, vals, p2, t);
    for (int s = t; s < len; s += G) {
        ci[r0 + s] = keys[s];
        va[r0 + s] = vals[s];
    }
}

__global__ void k_nz_count(int n, const int* __restrict__ rp, const double* __restrict__ va, int* cnt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = 0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) c += va[k] != 0.0;
    cnt[i] = c;
}

__global__ void k_nz_compact(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ va,
                             const int* __restrict__ nrp, int* nci, double* nva) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int o = nrp[i];
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
        if (va[k] != 0.0) {
            nci[o] = ci[k];
            nva[o] = va[k];
            ++o;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// host drivers
// ---------------------------------------------------------------------------------------------

// Shared-memory table classes: slots per table, and the largest measure each takes (3/4 full)
constexpr int kCap[kClasses - 1] = {64, 128, 512, 2048, 8192};
constexpr int kFill[kClasses - 1] = {48, 96, 384, 1536, 6144};
// device-memory tables are processed in batches of at most this many slots
constexpr long long kGlobalSlots = 64LL << 20;

struct Ctx {
    cudaStream_t st;
    Scratch* mem;
    long long* d_total;
    int* d_counts; // class counters (kClasses) + one spare
    int* d_err;
    int lim;       // largest row (distinct columns / entries) given a shared-memory table
    DeviceArena* keep = nullptr; // where the hierarchy's own arrays go (null: mem)
    template <class T> T* out(size_t count) { return keep != nullptr ? keep->alloc<T>(count) : mem->alloc<T>(count); }
};

template <class T> void to_host(std::vector<T>& h, const T* d, size_t n, cudaStream_t st) {
    h.resize(n);
    if (n > 0) CFDB_CUDA(cudaMemcpyAsync(h.data(), d, sizeof(T) * n, cudaMemcpyDeviceToHost, st));
}

void sync(cudaStream_t st) { CFDB_CUDA(cudaStreamSynchronize(st)); }

// out[0..n] = exclusive scan of in[0..n), out[n] = total; returns the total.
long long scan(Ctx& cx, const int* in, int n, int* out) {
    const int nb = std::max(1, (n + kScanChunk - 1) / kScanChunk);
    long long* bsum = cx.mem->alloc<long long>(nb);
    k_scan_sums<<<nb, kScanThreads, 0, cx.st>>>(in, n, bsum);
    k_scan_top<<<1, kScanThreads, 0, cx.st>>>(bsum, nb, cx.d_total, out + n);
    k_scan_apply<<<nb, kScanThreads, 0, cx.st>>>(in, n, bsum, out);
    CFDB_CUDA(cudaGetLastError());
    long long total = 0;
    CFDB_CUDA(cudaMemcpyAsync(&total, cx.d_total, sizeof(total), cudaMemcpyDeviceToHost, cx.st));
    sync(cx.st);
    return total;
}

int checked_nnz(long long total, const char* what) {
    if (total > INT_MAX) {
        fail(1, std::string("device AMG setup: ") + what +
                    " exceeds 2^31 nonzeros (coarse operators densify; lower strength_threshold)");
    }
    return static_cast<int>(total);
}

// Rows of class lists: counts after k_classify (host copy).
struct Classes {
    int* lists = nullptr;
    int count[kClasses] = {};
};

// limits lim[q] = min(base[q], cx.lim); classes above the limit stay empty
Classes classify(Ctx& cx, int n, const int* measure, const int (&base)[kClasses - 1]) {
    Limits L;
    for (int q = 0; q < kClasses - 1; ++q) L.lim[q] = std::min(base[q], cx.lim);
    Classes c;
    c.lists = cx.mem->alloc<int>(kClasses * static_cast<size_t>(std::max(n, 1)));
    CFDB_CUDA(cudaMemsetAsync(cx.d_counts, 0, (kClasses + 1) * sizeof(int), cx.st));
    if (n > 0) k_classify<<<grid_for(n), kThreads, 0, cx.st>>>(n, measure, L, c.lists, cx.d_counts);
    CFDB_CUDA(cudaMemcpyAsync(c.count, cx.d_counts, kClasses * sizeof(int), cudaMemcpyDeviceToHost, cx.st));
    sync(cx.st);
    return c;
}

// Device-memory tables for the rows `rows` (host list) with `caps` slots each, run in batches.
template <class Launch>
void global_batches(Ctx& cx, const std::vector<int>& rows, const std::vector<int>& caps, bool with_vals,
                    Launch&& launch) {
    size_t b0 = 0;
    while (b0 < rows.size()) {
        size_t b1 = b0;
        long long slots = 0;
        std::vector<long long> off;
        std::vector<int> cap;
        while (b1 < rows.size() && (b1 == b0 || slots + caps[b1] <= kGlobalSlots)) {
            off.push_back(slots);
            cap.push_back(caps[b1]);
            slots += caps[b1];
            ++b1;
        }
        const int nb = static_cast<int>(b1 - b0);
        Scratch tmp;
        int* d_rows = tmp.alloc<int>(nb);
        long long* d_off = tmp.alloc<long long>(nb);
        int* d_cap = tmp.alloc<int>(nb);
        int* keys = tmp.alloc<int>(static_cast<size_t>(slots));
        double* vals = with_vals ? tmp.alloc<double>(static_cast<size_t>(slots)) : nullptr;
        CFDB_CUDA(cudaMemcpyAsync(d_rows, rows.data() + b0, sizeof(int) * nb, cudaMemcpyHostToDevice, cx.st));
        CFDB_CUDA(cudaMemcpyAsync(d_off, off.data(), sizeof(long long) * nb, cudaMemcpyHostToDevice, cx.st));
        CFDB_CUDA(cudaMemcpyAsync(d_cap, cap.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, cx.st));
        launch(d_rows, nb, d_off, d_cap, keys, vals);
        sync(cx.st); // tmp is released here
        b0 = b1;
    }
}

template <class K> void set_smem(K kernel, size_t bytes) {
    if (bytes > 48 * 1024) {
        CFDB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
    }
}

// One Gustavson kernel launch over the rows of a list, with the table class `cls` (0..4).
template <bool NUMERIC> void gemm_launch(Ctx& cx, GemmArgs g, int cls, const int* rows, int n_list) {
    if (n_list <= 0) return;
    g.rows = rows;
    g.n_list = n_list;
    const size_t b = NUMERIC ? 12 : 4;      // bytes per slot
    const size_t chunk = NUMERIC ? 32 * 8 : 0; // warp groups: one chunk of contributions
    cudaStream_t st = cx.st;
    switch (cls) {
    case 0:
        k_gemm_rows<NUMERIC, 32, 64, 8><<<(n_list + 7) / 8, 256, 8 * (64 * b + chunk), st>>>(g);
        break;
    case 1:
        k_gemm_rows<NUMERIC, 32, 128, 8><<<(n_list + 7) / 8, 256, 8 * (128 * b + chunk), st>>>(g);
        break;
    case 2:
        k_gemm_rows<NUMERIC, 32, 512, 4><<<(n_list + 3) / 4, 128, 4 * (512 * b + chunk), st>>>(g);
        break;
    case 3:
        k_gemm_rows<NUMERIC, kThreads, 2048, 1><<<n_list, kThreads, 2048 * b, st>>>(g);
        break;
    default:
        set_smem(k_gemm_rows<NUMERIC, kThreads, 8192, 1>, 8192 * b);
        k_gemm_rows<NUMERIC, kThreads, 8192, 1><<<n_list, kThreads, 8192 * b, st>>>(g);
        break;
    }
    CFDB_CUDA(cudaGetLastError());
}

// C = diag(ascale) A B (B explicit, or the tentative prolongator of `tent` when b == null).
DevCsr spgemm(Ctx& cx, const DevCsr& a, const double* ascale, const DevCsr* b, const int* tent, int n_cols) {
    const int n = a.n_rows;
    cudaStream_t st = cx.st;
    DevCsr c;
    c.n_rows = n;
    c.n_cols = n_cols;
    GemmArgs g{};
    g.arp = a.rp;
    g.aci = a.ci;
    g.ava = a.va;
    g.ascale = ascale;
    g.brp = b != nullptr ? b->rp : nullptr;
    g.bci = b != nullptr ? b->ci : nullptr;
    g.bva = b != nullptr ? b->va : nullptr;
    g.tent = tent;
    g.err = cx.d_err;
    // symbolic: rows whose bound min(sum_k |B(k,:)|, n_cols) fits the two smallest tables go
    // there; the others start in the 512-slot warp tables and move to larger tables when they
    // fill up (the bound is loose: most such rows have far fewer distinct columns)
    int* ub = cx.mem->alloc<int>(std::max(n, 1));
    if (n > 0) k_gemm_bound<<<grid_for(n), kThreads, 0, st>>>(n, a.rp, a.ci, g.brp, n_cols, ub);
    int* cnt = cx.mem->alloc<int>(static_cast<size_t>(n) + 1);
    g.cnt = cnt;
    const Classes sc = classify(cx, n, ub, kFill);
    g.limit = INT_MAX;
    gemm_launch<false>(cx, g, 0, sc.lists, sc.count[0]);
    gemm_launch<false>(cx, g, 1, sc.lists + n, sc.count[1]);
    int* over[2] = {cx.mem->alloc<int>(std::max(n, 1)), cx.mem->alloc<int>(std::max(n, 1))};
    int* n_over = cx.mem->alloc<int>(2);
    int pending = 0, cur = 0;
    for (int q = 2; q < kClasses; ++q) pending += sc.count[q];
    for (int cls = 2; cls < kClasses - 1 && pending > 0; ++cls) {
        CFDB_CUDA(cudaMemsetAsync(n_over + cur, 0, sizeof(int), st));
        GemmArgs h = g;
        h.limit = std::min(kFill[cls], cx.lim);
        h.over_rows = over[cur];
        h.n_over = n_over + cur;
        if (cls == 2) {
            for (int q = 2; q < kClasses; ++q) gemm_launch<false>(cx, h, 2, sc.lists + static_cast<size_t>(q) * n, sc.count[q]);
        } else {
            gemm_launch<false>(cx, h, cls, over[1 - cur], pending);
        }
        CFDB_CUDA(cudaMemcpyAsync(&pending, n_over + cur, sizeof(int), cudaMemcpyDeviceToHost, st));
        sync(st);
        cur = 1 - cur;
    }
    if (pending > 0) { // rows beyond every shared-memory table: device-memory tables
        std::vector<int> rows, ub_h;
        to_host(rows, over[1 - cur], static_cast<size_t>(pending), st);
        to_host(ub_h, ub, static_cast<size_t>(n), st);
        sync(st);
        std::vector<int> caps(rows.size());
        for (size_t q = 0; q < rows.size(); ++q) caps[q] = next_pow2(2LL * std::max(ub_h[rows[q]], 1));
        global_batches(cx, rows, caps, false, [&](int* d_rows, int nb, long long* d_off, int* d_cap, int* keys, double*) {
            GemmArgs h = g;
            h.rows = d_rows;
            h.n_list = nb;
            h.limit = INT_MAX;
            h.goff = d_off;
            h.gcap = d_cap;
            h.gkeys = keys;
            k_gemm_rows<false, kThreads, 0, 1><<<nb, kThreads, 0, st>>>(h);
            CFDB_CUDA(cudaGetLastError());
        });
    }
    c.rp = cx.mem->alloc<int>(static_cast<size_t>(n) + 1);
    c.nnz = checked_nnz(scan(cx, cnt, n, c.rp), "a sparse product");
    c.ci = cx.mem->alloc<int>(static_cast<size_t>(c.nnz) + 4);
    c.va = cx.mem->alloc<double>(static_cast<size_t>(c.nnz) + 4);
    // numeric: classes by the exact count
    const Classes nc = classify(cx, n, cnt, kFill);
    g.crp = c.rp;
    g.cci = c.ci;
    g.cva = c.va;
    for (int q = 0; q < kClasses - 1; ++q) gemm_launch<true>(cx, g, q, nc.lists + static_cast<size_t>(q) * n, nc.count[q]);
    if (nc.count[kClasses - 1] > 0) {
        std::vector<int> rows, rp_h;
        to_host(rows, nc.lists + static_cast<size_t>(kClasses - 1) * n, static_cast<size_t>(nc.count[kClasses - 1]), st);
        to_host(rp_h, c.rp, static_cast<size_t>(n) + 1, st);
        sync(st);
        std::vector<int> caps(rows.size());
        for (size_t q = 0; q < rows.size(); ++q) {
            const long long len = rp_h[rows[q] + 1] - rp_h[rows[q]];
            caps[q] = next_pow2((4 * len + 2) / 3 + 1);
        }
        global_batches(cx, rows, caps, true, [&](int* d_rows, int nb, long long* d_off, int* d_cap, int* keys, double* vals) {
            GemmArgs h = g;
            h.rows = d_rows;
            h.n_list = nb;
            h.goff = d_off;
            h.gcap = d_cap;
            h.gkeys = keys;
            h.gvals = vals;
            k_gemm_rows<true, kThreads, 0, 1><<<nb, kThreads, 0, st>>>(h);
            CFDB_CUDA(cudaGetLastError());
        });
    }
    return c;
}

// Sorts every row of t by column, with the table class of its length.
void sort_rows(Ctx& cx, DevCsr& t) {
    cudaStream_t st = cx.st;
    const int m = t.n_rows;
    int* len = cx.mem->alloc<int>(std::max(m, 1));
    if (m > 0) k_row_len<<<grid_for(m), kThreads, 0, st>>>(m, t.rp, len);
    const Classes c = classify(cx, m, len, kCap);
    auto lst = [&](int q) { return c.lists + static_cast<size_t>(q) * m; };
    const size_t b = 12;
    if (c.count[0] > 0)
        k_seg_sort<32, 64, 8><<<(c.count[0] + 7) / 8, 256, 8 * 64 * b, st>>>(lst(0), c.count[0], t.rp, t.ci, t.va, nullptr, nullptr, nullptr, nullptr);
    if (c.count[1] > 0)
        k_seg_sort<32, 128, 8><<<(c.count[1] + 7) / 8, 256, 8 * 128 * b, st>>>(lst(1), c.count[1], t.rp, t.ci, t.va, nullptr, nullptr, nullptr, nullptr);
    if (c.count[2] > 0)
        k_seg_sort<32, 512, 4><<<(c.count[2] + 3) / 4, 128, 4 * 512 * b, st>>>(lst(2), c.count[2], t.rp, t.ci, t.va, nullptr, nullptr, nullptr, nullptr);
    if (c.count[3] > 0)
        k_seg_sort<kThreads, 2048, 1><<<c.count[3], kThreads, 2048 * b, st>>>(lst(3), c.count[3], t.rp, t.ci, t.va, nullptr, nullptr, nullptr, nullptr);
    if (c.count[4] > 0) {
        set_smem(k_seg_sort<kThreads, 8192, 1>, 8192 * b);
        k_seg_sort<kThreads, 8192, 1><<<c.count[4], kThreads, 8192 * b, st>>>(lst(4), c.count[4], t.rp, t.ci, t.va, nullptr, nullptr, nullptr, nullptr);
    }
    CFDB_CUDA(cudaGetLastError());
    if (c.count[5] > 0) {
        std::vector<int> rows, len_h;
        to_host(rows, lst(5), static_cast<size_t>(c.count[5]), st);
        to_host(len_h, len, static_cast<size_t>(m), st);
        sync(st);
        std::vector<int> caps(rows.size());
        for (size_t q = 0; q < rows.size(); ++q) caps[q] = next_pow2(len_h[rows[q]]);
        global_batches(cx, rows, caps, true, [&](int* d_rows, int nb, long long* d_off, int* d_cap, int* keys, double* vals) {
            k_seg_sort<kThreads, 0, 1><<<nb, kThreads, 0, st>>>(d_rows, nb, t.rp, t.ci, t.va, d_off, d_cap, keys, vals);
            CFDB_CUDA(cudaGetLastError());
        });
    }
}

DevCsr transpose(Ctx& cx, const DevCsr& a) {
    cudaStream_t st = cx.st;
    DevCsr t;
    t.n_rows = a.n_cols;
    t.n_cols = a.n_rows;
    const int m = a.n_cols;
    int* cnt = cx.mem->alloc<int>(static_cast<size_t>(m) + 1);
    CFDB_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * (static_cast<size_t>(m) + 1), st));
    if (a.nnz > 0) k_col_count<<<grid_for(a.nnz), kThreads, 0, st>>>(a.nnz, a.ci, cnt);
    t.rp = cx.out<int>(static_cast<size_t>(m) + 1);
    t.nnz = checked_nnz(scan(cx, cnt, m, t.rp), "a transpose");
    t.ci = cx.out<int>(static_cast<size_t>(t.nnz) + 4);
    t.va = cx.out<double>(static_cast<size_t>(t.nnz) + 4);
    CFDB_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * (static_cast<size_t>(m) + 1), st));
    if (a.n_rows > 0) k_t_fill<<<grid_for(a.n_rows), kThreads, 0, st>>>(a.n_rows, a.rp, a.ci, a.va, t.rp, cnt, t.ci, t.va);
    sort_rows(cx, t);
    return t;
}

DevCsr prune_zeros(Ctx& cx, const DevCsr& a) {
    cudaStream_t st = cx.st;
    DevCsr o;
    o.n_rows = a.n_rows;
    o.n_cols = a.n_cols;
    int* cnt = cx.mem->alloc<int>(static_cast<size_t>(a.n_rows) + 1);
    if (a.n_rows > 0) k_nz_count<<<grid_for(a.n_rows), kThreads, 0, st>>>(a.n_rows, a.rp, a.va, cnt);
    o.rp = cx.out<int>(static_cast<size_t>(a.n_rows) + 1);
    o.nnz = checked_nnz(scan(cx, cnt, a.n_rows, o.rp), "a coarse operator");
    o.ci = cx.out<int>(static_cast<size_t>(o.nnz) + 4);
    o.va = cx.out<double>(static_cast<size_t>(o.nnz) + 4);
    if (a.n_rows > 0)
        k_nz_compact<<<grid_for(a.n_rows), kThreads, 0, st>>>(a.n_rows, a.rp, a.ci, a.va, o.rp, o.ci, o.va);
    CFDB_CUDA(cudaGetLastError());
    return o;
}

// Rows left by pass 2 that pass 3 runs on the device (one thread); more go to the host.
constexpr int kPass3Device = 1024;

// Levels aggregated on the device: large and sparse ones (the fine level of a mesh). Each
// pass-1 sweep costs microseconds and more with every strong entry per row, while the host's
// sequential pass costs nanoseconds per strong entry plus the strength graph's read-back.
// Measured on the jittered 6-tet box of 5.1M cells: the fine level (3.9 strong entries per row)
// 14 ms on the device (930 sweeps) against 21.5 ms on the host plus 3 ms of read-back; the first
// coarse level (861K rows, 8.7 per row) 16 ms against 11 ms.
bool device_aggregation(int n, long long ns) { return n >= (1 << 18) && ns <= 6LL * n; }

// The aggregation on the device from the strength graph (srp, sci, sav = |a_ij|): passes 1 and
// 2 in parallel, pass 3 by one thread when at most kPass3Device rows are left for it. agg
// receives every row's aggregate. Returns the number of aggregates, or -1 when more rows are
// left for pass 3 (isolated rows, or rows none of whose strong neighbours pass 1 aggregated):
// the caller then aggregates on the host.
int aggregate_device(Ctx& cx, int n, int ns, int* srp, int* sci, double* sav, int* agg) {
    cudaStream_t st = cx.st;
    Ctx tx = cx;
    tx.keep = nullptr; // the transpose is scratch
    DevCsr g;
    g.n_rows = g.n_cols = n;
    g.nnz = ns;
    g.rp = srp;
    g.ci = sci;
    g.va = sav;
    const DevCsr t = transpose(tx, g);
    int* state = cx.mem->alloc<int>(n);
    int* counter = cx.d_counts + kClasses; // the spare counter
    k_seed_init<<<grid_for(n), kThreads, 0, st>>>(n, srp, state);
    // lo of each sweep of a batch; lo[0] = 0, then the last lo of the previous batch
    int* lo = cx.mem->alloc<int>(kSeedBatch + 1);
    CFDB_CUDA(cudaMemsetAsync(lo, 0, sizeof(int), st));
    const int grid = grid_for(std::min(n, kSeedWindow));
    for (long long sweeps = 0;;) {
        // every sweep decides at least its smallest undecided row
        if (sweeps > n + kSeedBatch) fail(kErrInternal, "device aggregation did not settle");
        CFDB_CUDA(cudaMemsetAsync(lo + 1, 0x7f, sizeof(int) * kSeedBatch, st));
        for (int b = 0; b < kSeedBatch; ++b)
            k_seed_sweep<<<grid, kThreads, 0, st>>>(n, lo + b, lo + b + 1, srp, sci, t.rp, t.ci, state);
        CFDB_CUDA(cudaGetLastError());
        sweeps += kSeedBatch;
        int last = 0;
        CFDB_CUDA(cudaMemcpyAsync(&last, lo + kSeedBatch, sizeof(int), cudaMemcpyDeviceToHost, st));
        sync(st);
        if (last >= n) break;
        CFDB_CUDA(cudaMemcpyAsync(lo, lo + kSeedBatch, sizeof(int), cudaMemcpyDeviceToDevice, st));
    }
    int* flag = cx.mem->alloc<int>(static_cast<size_t>(n) + 1);
    int* id = cx.mem->alloc<int>(static_cast<size_t>(n) + 1);
    k_seed_flags<<<grid_for(n), kThreads, 0, st>>>(n, state, flag);
    const long long n_seeds = scan(cx, flag, n, id);
    int* agg1 = cx.mem->alloc<int>(n);
    k_pass1_cover<<<grid_for(n), kThreads, 0, st>>>(n, t.rp, t.ci, state, id, agg1);
    CFDB_CUDA(cudaMemsetAsync(counter, 0, sizeof(int), st));
    k_pass2<<<grid_for(n), kThreads, 0, st>>>(n, srp, sci, sav, agg1, agg, counter);
    CFDB_CUDA(cudaGetLastError());
    int left = 0;
    CFDB_CUDA(cudaMemcpyAsync(&left, counter, sizeof(int), cudaMemcpyDeviceToHost, st));
    sync(st);
    if (left > 0 && left <= kPass3Device) {
        int* pos = cx.mem->alloc<int>(static_cast<size_t>(n) + 1);
        int* list = cx.mem->alloc<int>(left);
        k_left_flags<<<grid_for(n), kThreads, 0, st>>>(n, agg, flag);
        scan(cx, flag, n, pos);
        k_left_list<<<grid_for(n), kThreads, 0, st>>>(n, agg, pos, list);
        int n_agg = static_cast<int>(n_seeds);
        CFDB_CUDA(cudaMemcpyAsync(counter, &n_agg, sizeof(int), cudaMemcpyHostToDevice, st));
        k_pass3<<<1, 32, 0, st>>>(left, list, srp, sci, agg, counter);
        CFDB_CUDA(cudaGetLastError());
        CFDB_CUDA(cudaMemcpyAsync(&n_agg, counter, sizeof(int), cudaMemcpyDeviceToHost, st));
        sync(st);
        return n_agg;
    }
    return left > 0 ? -1 : static_cast<int>(n_seeds);
}

HostCsr csr_to_host(const DevCsr& d, cudaStream_t st) {
    HostCsr h;
    h.n_rows = d.n_rows;
    h.n_cols = d.n_cols;
    to_host(h.rp, d.rp, static_cast<size_t>(d.n_rows) + 1, st);
    to_host(h.ci, d.ci, static_cast<size_t>(d.nnz), st);
    to_host(h.va, d.va, static_cast<size_t>(d.nnz), st);
    sync(st);
    return h;
}

void check_err(Ctx& cx) {
    int e = 0;
    CFDB_CUDA(cudaMemcpyAsync(&e, cx.d_err, sizeof(int), cudaMemcpyDeviceToHost, cx.st));
    sync(cx.st);
    if (e != 0) fail(kErrInternal, "device AMG setup: inconsistent sparse product (code " + std::to_string(e) + ")");
}

} // namespace

void ldu_to_csr_values(int n, int nf, const int* diag_pos, const int* upper_pos, const int* lower_pos,
                       const double* diag, const double* upper, const double* lower, double* va, cudaStream_t st) {
    const int m = std::max(n, nf);
    if (m > 0) k_ldu_values<<<grid_for(m), kThreads, 0, st>>>(n, nf, diag_pos, upper_pos, lower_pos, diag, upper, lower, va);
    CFDB_CUDA(cudaGetLastError());
}

void amg_setup_device(const DevCsr& a0, const AmgSettings& s, cudaStream_t st, DeviceHierarchy& h,
                      PinnedBuffer* stage, DeviceArena* keep) {
    PinnedBuffer own_stage;
    if (stage == nullptr) stage = &own_stage;
    if (a0.n_rows != a0.n_cols) fail(1, "AmgPreconditioner: matrix must be square");
    if (a0.n_rows <= 0) fail(1, "amg_setup: empty matrix");
    Ctx cx{st, &h.mem, nullptr, nullptr, nullptr, s.table_limit > 0 ? s.table_limit : INT_MAX, keep};
    cx.d_total = h.mem.alloc<long long>(1);
    cx.d_counts = h.mem.alloc<int>(kClasses + 1);
    cx.d_err = h.mem.alloc<int>(1);
    CFDB_CUDA(cudaMemsetAsync(cx.d_err, 0, sizeof(int), st));
    unsigned long long* rho_bits = h.mem.alloc<unsigned long long>(1);
    double t_mark = PhaseTimes::now();
    auto phase = [&](const char* name) { // closes the phase that ends here (stream drained)
        sync(st);
        const double t = PhaseTimes::now();
        h.times.add(name, t - t_mark);
        t_mark = t;
    };
    DevCsr cur = a0;
    for (int l = 0; l < s.max_levels; ++l) {
        const int nl = cur.n_rows;
        double* d = h.mem.alloc<double>(nl);
        k_last_diag<<<grid_for(nl), kThreads, 0, st>>>(nl, cur.rp, cur.ci, cur.va, d);
        const bool last = nl <= s.coarse_size || l + 1 == s.max_levels;
        if (last) {
            h.a.push_back(cur);
            break;
        }
        // strength graph
        int* scnt = h.mem.alloc<int>(static_cast<size_t>(nl) + 1);
        k_strong<false><<<grid_for(nl), kThreads, 0, st>>>(nl, cur.rp, cur.ci, cur.va, d, s.theta, scnt, nullptr,
                                                           nullptr, nullptr);
        int* srp = h.mem.alloc<int>(static_cast<size_t>(nl) + 1);
        const int ns = checked_nnz(scan(cx, scnt, nl, srp), "the strength graph");
        int* sci = h.mem.alloc<int>(ns);
        double* sav = h.mem.alloc<double>(ns);
        k_strong<true><<<grid_for(nl), kThreads, 0, st>>>(nl, cur.rp, cur.ci, cur.va, d, s.theta, nullptr, srp, sci,
                                                          sav);
        CFDB_CUDA(cudaGetLastError());
        phase("strength");
        // aggregation: passes 1 and 2 on the device; when rows are left for pass 3 the host runs
        // all three passes from the strength graph
        std::vector<int> agg;
        int* dagg = h.mem.alloc<int>(nl);
        int n_agg = device_aggregation(nl, ns) ? aggregate_device(cx, nl, ns, srp, sci, sav, dagg) : -1;
        if (n_agg < 0) {
            // read back: offsets, columns and, per entry, its strength rank within the row (2
            // bytes; the |a_ij| themselves when a row has more than 65536 strong entries)
            CFDB_CUDA(cudaMemsetAsync(cx.d_counts, 0, sizeof(int), st));
            k_max_degree<<<grid_for(nl), kThreads, 0, st>>>(nl, srp, cx.d_counts);
            int max_deg = 0;
            CFDB_CUDA(cudaMemcpyAsync(&max_deg, cx.d_counts, sizeof(int), cudaMemcpyDeviceToHost, st));
            sync(st);
            const bool ranked = max_deg <= std::min(4096, cx.lim); // ranks cost O(degree^2) per row
            const size_t b_rp = aligned(sizeof(int) * (static_cast<size_t>(nl) + 1));
            const size_t b_ci = aligned(sizeof(int) * static_cast<size_t>(ns));
            const size_t b_key = aligned((ranked ? sizeof(uint16_t) : sizeof(double)) * static_cast<size_t>(ns));
            char* host = static_cast<char*>(stage->get(b_rp + b_ci + b_key));
            const int* srp_h = reinterpret_cast<const int*>(host);
            const int* sci_h = reinterpret_cast<const int*>(host + b_rp);
            CFDB_CUDA(cudaMemcpyAsync(host, srp, sizeof(int) * (static_cast<size_t>(nl) + 1), cudaMemcpyDeviceToHost, st));
            if (ns > 0) CFDB_CUDA(cudaMemcpyAsync(host + b_rp, sci, sizeof(int) * ns, cudaMemcpyDeviceToHost, st));
            if (ranked) {
                uint16_t* rank = h.mem.alloc<uint16_t>(ns);
                k_strong_rank<<<grid_for(nl), kThreads, 0, st>>>(nl, srp, sav, rank);
                if (ns > 0)
                    CFDB_CUDA(cudaMemcpyAsync(host + b_rp + b_ci, rank, sizeof(uint16_t) * ns, cudaMemcpyDeviceToHost, st));
            } else if (ns > 0) {
                CFDB_CUDA(cudaMemcpyAsync(host + b_rp + b_ci, sav, sizeof(double) * ns, cudaMemcpyDeviceToHost, st));
            }
            CFDB_CUDA(cudaGetLastError());
            sync(st);
            n_agg = ranked ? aggregate_strong_ranked(nl, srp_h, sci_h, reinterpret_cast<const uint16_t*>(host + b_rp + b_ci), agg)
                           : aggregate_strong(nl, srp_h, sci_h, reinterpret_cast<const double*>(host + b_rp + b_ci), agg);
            CFDB_CUDA(cudaMemcpyAsync(dagg, agg.data(), sizeof(int) * nl, cudaMemcpyHostToDevice, st));
        }
        phase("aggregate");
        if (n_agg >= nl || n_agg == 0) {
            sync(st);
            h.a.push_back(cur);
            break;
        }
        // Jacobi-smoothing weight
        double* inv = h.mem.alloc<double>(nl);
        CFDB_CUDA(cudaMemsetAsync(rho_bits, 0, sizeof(unsigned long long), st));
        k_inv_rho<<<grid_for(nl), kThreads, 0, st>>>(nl, cur.rp, cur.va, d, inv, rho_bits);
        unsigned long long rb = 0;
        CFDB_CUDA(cudaMemcpyAsync(&rb, rho_bits, sizeof(rb), cudaMemcpyDeviceToHost, st));
        sync(st);
        double rho = 0.0;
        std::memcpy(&rho, &rb, sizeof(rho));
        const double omega = rho > 0.0 ? 4.0 / (3.0 * rho) : 0.0;
        // P = P_tent - omega (D^-1 A) P_tent, pruned
        const DevCsr c = spgemm(cx, cur, inv, nullptr, dagg, n_agg);
        DevCsr p;
        p.n_rows = nl;
        p.n_cols = n_agg;
        int* pcnt = h.mem.alloc<int>(static_cast<size_t>(nl) + 1);
        k_p_emit<false><<<grid_for(nl), kThreads, 0, st>>>(nl, c.rp, c.ci, c.va, dagg, omega, pcnt, nullptr, nullptr,
                                                           nullptr);
        p.rp = cx.out<int>(static_cast<size_t>(nl) + 1);
        p.nnz = checked_nnz(scan(cx, pcnt, nl, p.rp), "a prolongation");
        p.ci = cx.out<int>(static_cast<size_t>(p.nnz) + 4);
        p.va = cx.out<double>(static_cast<size_t>(p.nnz) + 4);
        k_p_emit<true><<<grid_for(nl), kThreads, 0, st>>>(nl, c.rp, c.ci, c.va, dagg, omega, nullptr, p.rp, p.ci, p.va);
        CFDB_CUDA(cudaGetLastError());
        phase("prolongation");
        const DevCsr r = transpose(cx, p);
        phase("transpose");
        const DevCsr ap = spgemm(cx, cur, nullptr, &p, nullptr, n_agg);
        phase("AP");
        const DevCsr rap = spgemm(cx, r, nullptr, &ap, nullptr, n_agg);
        const DevCsr coarse = prune_zeros(cx, rap);
        check_err(cx);
        phase("RAP");
        h.a.push_back(cur);
        h.p.push_back(p);
        h.r.push_back(r);
        h.agg.push_back(std::move(agg));
        h.dagg.push_back(dagg);
        h.n_agg.push_back(n_agg);
        cur = coarse;
    }
    // coarsest level: dense inverse on the host (amg.cpp:227-240)
    const HostCsr c = csr_to_host(h.a.back(), st);
    h.n_c = c.n_rows;
    std::vector<double> dense(static_cast<size_t>(h.n_c) * h.n_c, 0.0);
    for (int i = 0; i < h.n_c; ++i)
        for (int k = c.rp[i]; k < c.rp[i + 1]; ++k) dense[static_cast<size_t>(i) * h.n_c + c.ci[k]] += c.va[k];
    h.ldlt_ok = dense_inverse(h.n_c, dense, h.coarse_inverse);
    phase("coarse_inverse");
}

Hierarchy download_hierarchy(const DeviceHierarchy& d, bool with_a0, cudaStream_t st) {
    Hierarchy h;
    for (int l = 0; l < d.levels(); ++l) {
        if (l == 0 && !with_a0) {
            h.a.emplace_back();
            h.a.back().n_rows = h.a.back().n_cols = d.a[0].n_rows;
        } else {
            h.a.push_back(csr_to_host(d.a[l], st));
        }
    }
    for (size_t l = 0; l < d.p.size(); ++l) {
        h.p.push_back(csr_to_host(d.p[l], st));
        h.r.push_back(csr_to_host(d.r[l], st));
    }
    h.agg = d.agg;
    for (size_t l = 0; l < h.agg.size(); ++l)
        if (h.agg[l].empty() && d.a[l].n_rows > 0) to_host(h.agg[l], d.dagg[l], static_cast<size_t>(d.a[l].n_rows), st);
    sync(st);
    h.n_agg = d.n_agg;
    h.n_c = d.n_c;
    h.ldlt_ok = d.ldlt_ok;
    h.coarse_inverse = d.coarse_inverse;
    return h;
}

// ---------------------------------------------------------------------------------------------
// engine operator layouts from device CSR blocks
// ---------------------------------------------------------------------------------------------

namespace {

__global__ void k_rows_padded(int n, int n_pad, const int* __restrict__ rp, int* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= n_pad) out[i] = i <= n ? rp[i] : rp[n];
}

__global__ void k_copy_values(long long nnz, const int* __restrict__ ci, const double* __restrict__ va, int* col,
                              double* v64, float* v32) {
    const long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= nnz + 4) return;
    const bool real = e < nnz;
    const double v = real ? va[e] : 0.0;
    col[e] = real ? ci[e] : 0;
    if (v64 != nullptr) v64[e] = v;
    if (v32 != nullptr) v32[e] = __double2float_rn(v);
}

// One CTA per window of kSellWindow positions: stable order by row length, longest first
// (padding rows, length -1, last), and 32 x the widest row of each slice of the window.
constexpr int kSellWindow = 256;
__global__ void __launch_bounds__(kSellWindow) k_sell_order(int n, int n_pad, const int* __restrict__ rp, int* perm,
                                                           int* width32) {
    __shared__ int len_s[kSellWindow];
    __shared__ int sorted_len[kSellWindow];
    const int t = threadIdx.x;
    const int w0 = blockIdx.x * kSellWindow;
    const int wn = min(kSellWindow, n_pad - w0);
    int len = -2;
    if (t < wn) {
        const int row = w0 + t;
        len = row < n ? rp[row + 1] - rp[row] : -1;
    }
    len_s[t] = len;
    __syncthreads();
    if (t < wn) {
        int rank = 0;
        for (int j = 0; j < wn; ++j) {
            const int lj = len_s[j];
            rank += (lj > len) || (lj == len && j < t);
        }
        perm[w0 + rank] = w0 + t;
        sorted_len[rank] = len > 0 ? len : 0;
    }
    __syncthreads();
    const int w = t >> 5, lane = t & 31;
    if (w * 32 < wn) {
        int m = sorted_len[w * 32 + lane];
        for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0) width32[w0 / 32 + w] = 32 * m;
    }
}

__global__ void k_sell_fill(int n, int n_sl, const int* __restrict__ perm, const int* __restrict__ slice,
                            const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ va,
                            int pad_col, int* col, double* v64, float* v32) {
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const long long sl = t >> 5;
    const int lane = static_cast<int>(t & 31);
    if (sl >= n_sl) return;
    const int row = perm[sl * 32 + lane];
    const int s0 = slice[sl];
    const int w = (slice[sl + 1] - s0) / 32;
    const int b = row < n ? rp[row] : 0;
    const int len = row < n ? rp[row + 1] - b : 0;
    for (int k = 0; k < w; ++k) {
        const long long slot = s0 + static_cast<long long>(k) * 32 + lane;
        const bool real = k < len;
        const double v = real ? va[b + k] : 0.0;
        col[slot] = real ? ci[b + k] : pad_col;
        if (v64 != nullptr) v64[slot] = v;
        if (v32 != nullptr) v32[slot] = __double2float_rn(v);
    }
}

__global__ void k_weighted_inv_diag(int n, int n_pad, const int* __restrict__ rp, const int* __restrict__ ci,
                                    const double* __restrict__ va, double weight, double* wd64, float* wd32) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pad) return;
    double w = weight;
    if (i < n) {
        double dinv = 1.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] == i && va[k] != 0.0) dinv = __ddiv_rn(1.0, va[k]);
        w = __dmul_rn(weight, dinv);
    }
    if (wd64 != nullptr) wd64[i] = w;
    if (wd32 != nullptr) wd32[i] = __double2float_rn(w);
}

} // namespace

void adopt_levels(const DeviceHierarchy& d, DeviceLevels& k) {
    k.a.clear();
    k.p.clear();
    k.r.clear();
    for (int l = 0; l < d.levels(); ++l) {
        if (l == 0) {
            DevCsr e;
            e.n_rows = e.n_cols = d.a[0].n_rows;
            k.a.push_back(e);
        } else {
            k.a.push_back(d.a[l]);
        }
    }
    k.p = d.p;
    k.r = d.r;
}

Hierarchy hierarchy_shape(const DeviceHierarchy& d) {
    auto shape = [](const DevCsr& m) {
        HostCsr h;
        h.n_rows = m.n_rows;
        h.n_cols = m.n_cols;
        return h;
    };
    Hierarchy h;
    for (const DevCsr& m : d.a) h.a.push_back(shape(m));
    for (const DevCsr& m : d.p) h.p.push_back(shape(m));
    for (const DevCsr& m : d.r) h.r.push_back(shape(m));
    h.agg = d.agg;
    h.n_agg = d.n_agg;
    h.n_c = d.n_c;
    h.ldlt_ok = d.ldlt_ok;
    h.coarse_inverse = d.coarse_inverse;
    return h;
}

void csr_rows_padded(const DevCsr& m, int n_pad, int* out, cudaStream_t st) {
    k_rows_padded<<<grid_for(static_cast<long long>(n_pad) + 1), kThreads, 0, st>>>(m.n_rows, n_pad, m.rp, out);
    CFDB_CUDA(cudaGetLastError());
}

void csr_copy_values(const DevCsr& m, int* col, double* v64, float* v32, cudaStream_t st) {
    k_copy_values<<<grid_for(static_cast<long long>(m.nnz) + 4), kThreads, 0, st>>>(m.nnz, m.ci, m.va, col, v64, v32);
    CFDB_CUDA(cudaGetLastError());
}

long long sell_shape(const DevCsr& m, int n_pad, int window, int* perm, int* slice, cudaStream_t st) {
    if (window != kSellWindow) fail(1, "sell_shape: unsupported window");
    if (n_pad % 32 != 0 || n_pad < m.n_rows) fail(1, "sell_shape: bad padding");
    const int n_sl = n_pad / 32;
    Scratch tmp;
    Ctx cx{st, &tmp, tmp.alloc<long long>(1), tmp.alloc<int>(kClasses + 1), tmp.alloc<int>(1), INT_MAX};
    int* width32 = tmp.alloc<int>(std::max(n_sl, 1));
    if (n_pad > 0)
        k_sell_order<<<(n_pad + kSellWindow - 1) / kSellWindow, kSellWindow, 0, st>>>(m.n_rows, n_pad, m.rp, perm, width32);
    CFDB_CUDA(cudaGetLastError());
    const long long total = scan(cx, width32, n_sl, slice);
    if (total > INT_MAX) fail(1, "operator too large for 32-bit slot offsets");
    return total;
}

void sell_fill(const DevCsr& m, int n_pad, const int* perm, const int* slice, int pad_col, int* col, double* v64,
               float* v32, cudaStream_t st) {
    const int n_sl = n_pad / 32;
    if (n_sl > 0)
        k_sell_fill<<<grid_for(32LL * n_sl), kThreads, 0, st>>>(m.n_rows, n_sl, perm, slice, m.rp, m.ci, m.va, pad_col,
                                                                col, v64, v32);
    CFDB_CUDA(cudaGetLastError());
}

void weighted_inverse_diagonal(const DevCsr& m, int n_pad, double weight, double* wd64, float* wd32, cudaStream_t st) {
    if (n_pad > 0)
        k_weighted_inv_diag<<<grid_for(n_pad), kThreads, 0, st>>>(m.n_rows, n_pad, m.rp, m.ci, m.va, weight, wd64, wd32);
    CFDB_CUDA(cudaGetLastError());
}

} // namespace cfdb
