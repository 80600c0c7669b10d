// Device kernels of the pressure solve (sm_100a).
//
// Layout: every sparse operator (level operators A_l, prolongations P_l, restrictions R_l) is
// stored in SELL-32: rows in slices of 32, a slice's entries column-major (slot = base + k*32 +
// lane), so a warp reads 32 consecutive values and 32 consecutive column indices per step.
// Within a row, entries keep the CSR column order, so every row sum is accumulated in exactly
// the order of the reference's CSR SpMV (krylov_cuda.cu:24-34 / krylov_kernels.inc:12-24).
// The FP64 kernels are compiled without FMA contraction: every product and sum is rounded as
// in the reference's host path, so V-cycles are bit-reproducible against the CPU oracle.
//
// Work decomposition: each level's rows are concatenated over the systems of a batch (a single
// solve is a batch of one), each system's block padded to a multiple of 32 rows. A tile is a
// run of whole slices of ONE system; one CTA of 256 threads processes one tile. Tiles carry
// their system id so converged systems are skipped and reductions stay per system.
//
// Reductions (CG dot products) are deterministic: each tile writes its partial sums, the last
// CTA of a system to finish (atomic ticket) adds that system's partials in a fixed order and
// runs the scalar part of the Krylov step (alpha, beta, convergence tests) for that system.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace cfdb {

constexpr int kBlock = 256;
// Rows of a SELL tile of the V-cycle kernels (one row per thread); also the window within which
// a SELL operator's rows may be reordered by length.
constexpr int kSellRows = kBlock;

// Programmatic dependent launch (sm_90+): let the next kernel of the stream be scheduled once
// every CTA of this one has started, then wait until the previous kernel has completed and its
// writes are visible. Both are no-ops for a kernel launched without the attribute. Every kernel
// below except the persistent tail calls it first, before touching global memory.
__device__ __forceinline__ void pdl_entry() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Storage of one sparse operator of a level, selected by `fmt`:
//  0 (kFmtSell): SELL-32, one thread per row; `slice` = slice offsets. Row sums keep the CSR
//     order.
//  G in {4, 8, 16, 32, 64, 128, 256}: CSR with G lanes per row; `slice` = row offsets. Used
//     for wide coarse-level rows (tens to thousands of entries), where one thread per row would
//     serialise long load chains; lanes sum strided entries and combine them with a fixed
//     butterfly (and, above 32 lanes, a fixed-order sum over the row's warps): deterministic,
//     but not the sequential CSR order. Tiles of a CSR operator hold 8 rows (G <= 32, blockDim
//     8 G) or 256 / G rows (G > 32, blockDim 256).
enum : int { kFmtSell = 0 };

template <class T> struct Sell {
    const int* slice; // SELL: n_slices + 1 slot offsets; CSR: n_rows + 1 row offsets
    const int* col;
    const T* val;
    int fmt;
    // SELL only: row held at each position (rows sorted by length, longest first, within each
    // aligned window of kSellRows positions, which cuts slice padding); null = identity
    const int* perm = nullptr;
    // Compressed columns (FP32 copies whose every SELL slice / CSR row spans fewer than 65536
    // columns): column = cbase[slice or row] + c16[k]; `col` is then unused. Null = int32 `col`.
    const uint16_t* c16 = nullptr;
    const int* cbase = nullptr;
};

struct Tiles {
    const int* row; // n_tiles + 1 first rows
    const int* sys; // n_tiles system ids (null when the plan holds one system: all 0)
};

// Per-system Krylov state (device resident; host reads it only at the end of a solve).
struct SysState {
    double tol;       // absolute tolerance on |r|_2
    double res;       // last |r|_2
    double rz;        // r . z
    double pq;        // p . q
    double alpha;
    double beta;
    double true_res;  // |b - A x|_2 recomputed after the solve
    int it;           // current iteration number (1-based, as the reference loop counter)
    int max_it;
    int iters_out;    // reported iterations
    int active;
    int converged;
    int first;        // next p-update is p = z
    int phase;        // 0: initial preconditioning, 1: inside the loop
    int check;        // mixed precision: recursive residual met the target, verify in FP64
    int breakdown;    // p.q == 0 or rho == 0 style exits
    int jacobi;       // single-level hierarchy: Jacobi-preconditioned FP64 CG (z = r / diag), as
                      // ldu_matrix.cpp:357 solves a system whose hierarchy has one level
};

struct Control {
    int* n_active;   // number of active systems (device)
    int* error;      // device error flag (bounded waits)
    int wait_polls = 1 << 22; // poll limit of the bounded waits (< 0: give up at once)
};

// Polls allowed to drain a CTA's own bulk copy after its bounded wait expired: the CTA must
// not exit while the copy can still write its shared memory.
constexpr int kDrainPolls = 1 << 22;

// ---------------------------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------------------------

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of two values; result valid in thread 0. Fixed tree: deterministic.
__device__ __forceinline__ void block_sum2(double& a, double& b) {
    __shared__ double sa[kBlock / 32], sb[kBlock / 32];
    a = warp_sum(a);
    b = warp_sum(b);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        sa[w] = a;
        sb[w] = b;
    }
    __syncthreads();
    if (w == 0) {
        a = l < kBlock / 32 ? sa[l] : 0.0;
        b = l < kBlock / 32 ? sb[l] : 0.0;
        a = warp_sum(a);
        b = warp_sum(b);
    }
    __syncthreads();
}

// Per-tile partial sums and their tickets, reduced in two fixed-order levels: the last CTA of
// each group of kGroupTiles consecutive tiles of a system sums the group's partials, and the
// last group of the system sums the group totals. Deterministic, and no CTA sums more than
// kGroupTiles or (tiles / kGroupTiles) values.
constexpr int kGroupTiles = 64;
struct Reduce {
    double* partials;        // 2 per tile
    double* gpartials;       // 2 per group
    int* counters;           // per system: groups finished
    int* gcounters;          // per group: tiles finished
    const int* sys_tile0;    // n_systems + 1: first tile of each system
    const int* grp0;         // n_systems + 1: first group of each system
};

// Sum of the pairs src[first..last) in index order by the block; valid in thread 0.
__device__ __forceinline__ void sum_pairs(const double* src, int first, int last, double& a, double& b) {
    a = 0.0;
    b = 0.0;
    for (int t = first + threadIdx.x; t < last; t += blockDim.x) {
        a += __ldcg(&src[2 * t]);
        b += __ldcg(&src[2 * t + 1]);
    }
    block_sum2(a, b);
}

// Writes this tile's partials; returns true in every thread of the system's last CTA, whose
// thread 0 then holds the system totals in (a, b).
__device__ __forceinline__ bool reduce_system(double& a, double& b, int tile, int s, const Reduce& r) {
    __shared__ int last;
    block_sum2(a, b);
    const int t0 = r.sys_tile0[s], t1 = r.sys_tile0[s + 1];
    const int g = (tile - t0) / kGroupTiles;
    const int gi = r.grp0[s] + g;
    const int gf = t0 + g * kGroupTiles;
    const int gl = min(t1, gf + kGroupTiles);
    if (threadIdx.x == 0) {
        r.partials[2 * tile] = a;
        r.partials[2 * tile + 1] = b;
        __threadfence();
        const int ticket = atomicAdd(&r.gcounters[gi], 1);
        last = ticket == gl - gf - 1;
        if (last) r.gcounters[gi] = 0;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    sum_pairs(r.partials, gf, gl, a, b);
    if (threadIdx.x == 0) {
        r.gpartials[2 * gi] = a;
        r.gpartials[2 * gi + 1] = b;
        __threadfence();
        const int n_groups = r.grp0[s + 1] - r.grp0[s];
        const int ticket = atomicAdd(&r.counters[s], 1);
        last = ticket == n_groups - 1;
        if (last) r.counters[s] = 0;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    sum_pairs(r.gpartials, r.grp0[s], r.grp0[s + 1], a, b);
    return true;
}

__device__ __forceinline__ void deactivate(SysState& st, Control c) {
    st.active = 0;
    atomicSub(c.n_active, 1);
}

// s + a*b: FP64 rounds the product and the sum separately (reference rounding); FP32 fuses.
template <class T> __device__ __forceinline__ T madd(T s, T a, T b) {
    if constexpr (sizeof(T) == 8) return __dadd_rn(s, __dmul_rn(a, b));
    else return fmaf(a, b, s);
}

// Predicated batch of four SELL entries starting at k (column -1 beyond the row end e); C16:
// compressed columns (the caller has checked m.c16).
template <bool C16, class T>
__device__ __forceinline__ void sell_load4(const Sell<T>& m, int k, int e, int base, T (&v)[4], int (&c)[4]) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const bool ok = k + 32 * u < e;
        v[u] = ok ? __ldg(&m.val[k + 32 * u]) : T(0);
        if constexpr (C16) c[u] = ok ? base + static_cast<int>(__ldg(&m.c16[k + 32 * u])) : -1;
        else c[u] = ok ? __ldg(&m.col[k + 32 * u]) : -1;
    }
}

template <class T, class XA>
__device__ __forceinline__ void sell_acc4(T& s, const T (&v)[4], const int (&c)[4], XA xa) {
    T xv[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) xv[u] = c[u] >= 0 ? xa(c[u]) : T(0);
#pragma unroll
    for (int u = 0; u < 4; ++u)
        if (c[u] >= 0) s = madd<T>(s, v[u], xv[u]);
}

// Row sum of a SELL row: sum_k val[k] * xa(col[k]) in CSR order. Entries are taken in batches
// of four, software-pipelined: the column / value loads of the next batch are issued before the
// gathers of the current one, so a thread keeps two batches of the row in flight. Every row of
// a slice has the slice's width, so the batch predicates are warp-uniform.
template <bool C16, class T, class XA>
__device__ __forceinline__ T sell_row_sum_c(const Sell<T>& m, int row, XA xa) {
    const int slice = row >> 5;
    const int lane = row & 31;
    int k = __ldg(&m.slice[slice]) + lane;
    const int end = __ldg(&m.slice[slice + 1]);
    const int base = C16 ? __ldg(&m.cbase[slice]) : 0;
    T s = T(0);
    if (k >= end) return s;
    T v[4];
    int c[4];
    sell_load4<C16>(m, k, end, base, v, c);
    for (;;) {
        k += 128;
        T vn[4];
        int cn[4];
        sell_load4<C16>(m, k, end, base, vn, cn);
        sell_acc4(s, v, c, xa);
        if (k >= end) break;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            v[u] = vn[u];
            c[u] = cn[u];
        }
    }
    return s;
}

template <class T, class XA>
__device__ __forceinline__ T sell_row_sum(const Sell<T>& m, int row, XA xa) {
    if constexpr (sizeof(T) == 4) {
        if (m.c16 != nullptr) return sell_row_sum_c<true>(m, row, xa);
    }
    return sell_row_sum_c<false>(m, row, xa);
}

// Two SELL rows of one thread, both software-pipelined as in sell_row_sum (up to four batches
// in flight per thread); each row is still accumulated in its own CSR order.
template <bool C16, class T, class XA>
__device__ __forceinline__ void sell_row_sum2_c(const Sell<T>& m, int ra, int rb, XA xa, T& sa, T& sb) {
    int ka = __ldg(&m.slice[ra >> 5]) + (ra & 31);
    const int ea = __ldg(&m.slice[(ra >> 5) + 1]);
    int kb = __ldg(&m.slice[rb >> 5]) + (rb & 31);
    const int eb = __ldg(&m.slice[(rb >> 5) + 1]);
    const int ba = C16 ? __ldg(&m.cbase[ra >> 5]) : 0, bb = C16 ? __ldg(&m.cbase[rb >> 5]) : 0;
    sa = T(0);
    sb = T(0);
    T va[4], vb[4];
    int ca[4], cb[4];
    sell_load4<C16>(m, ka, ea, ba, va, ca);
    sell_load4<C16>(m, kb, eb, bb, vb, cb);
    for (;;) {
        ka += 128;
        kb += 128;
        T van[4], vbn[4];
        int can[4], cbn[4];
        sell_load4<C16>(m, ka, ea, ba, van, can);
        sell_load4<C16>(m, kb, eb, bb, vbn, cbn);
        sell_acc4(sa, va, ca, xa);
        sell_acc4(sb, vb, cb, xa);
        if (ka >= ea && kb >= eb) break;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            va[u] = van[u];
            ca[u] = can[u];
            vb[u] = vbn[u];
            cb[u] = cbn[u];
        }
    }
}

template <class T, class XA>
__device__ __forceinline__ void sell_row_sum2(const Sell<T>& m, int ra, int rb, XA xa, T& sa, T& sb) {
    if constexpr (sizeof(T) == 4) {
        if (m.c16 != nullptr) {
            sell_row_sum2_c<true>(m, ra, rb, xa, sa, sb);
            return;
        }
    }
    sell_row_sum2_c<false>(m, ra, rb, xa, sa, sb);
}

template <class T, class X>
__device__ __forceinline__ T sell_row(const Sell<T>& m, int row, const X* __restrict__ x) {
    return sell_row_sum(m, row, [x](int j) { return static_cast<T>(x[j]); });
}

// Four consecutive values from a 16-byte aligned address.
__device__ __forceinline__ void ld4(const float* p, float (&v)[4]) {
    const float4 q = __ldg(reinterpret_cast<const float4*>(p));
    v[0] = q.x;
    v[1] = q.y;
    v[2] = q.z;
    v[3] = q.w;
}
__device__ __forceinline__ void ld4(const double* p, double (&v)[4]) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    v[0] = a.x;
    v[1] = a.y;
    v[2] = b.x;
    v[3] = b.y;
}

// Four consecutive CSR columns at an aligned index k into c[o..o+3] (8-byte loads when
// compressed, 16-byte otherwise).
template <class T>
__device__ __forceinline__ void ld4col(const Sell<T>& m, int k, int base, int (&c)[8], int o) {
    if (sizeof(T) == 4 && m.c16 != nullptr) {
        const uint2 q = __ldg(reinterpret_cast<const uint2*>(m.c16 + k));
        c[o] = base + static_cast<int>(q.x & 0xffffu);
        c[o + 1] = base + static_cast<int>(q.x >> 16);
        c[o + 2] = base + static_cast<int>(q.y & 0xffffu);
        c[o + 3] = base + static_cast<int>(q.y >> 16);
    } else {
        const int4 q = __ldg(reinterpret_cast<const int4*>(m.col + k));
        c[o] = q.x;
        c[o + 1] = q.y;
        c[o + 2] = q.z;
        c[o + 3] = q.w;
    }
}

// Partial CSR row sum of one lane. The row is read in aligned quads (16-byte vector loads of
// columns and values): lane `sub` takes quads sub, sub + G, ... of the row's aligned span, two
// quads per pass, and masks the entries outside [row begin, row end). CSR arrays carry four
// entries of slack so the last quad never reads past them.
template <class T, class XA>
__device__ __forceinline__ T csr_lane_sum(const Sell<T>& m, int row, int sub, int G, XA xa) {
    const int b = __ldg(&m.slice[row]);
    const int e = __ldg(&m.slice[row + 1]);
    const int base = sizeof(T) == 4 && m.c16 != nullptr ? __ldg(&m.cbase[row]) : 0;
    T s = T(0);
    for (int k = (b & ~3) + 4 * sub; k < e; k += 8 * G) {
        const int k2 = k + 4 * G;
        const bool two = k2 < e;
        int c[8];
        T v[8], xv[8];
        {
            ld4col(m, k, base, c, 0);
            T t[4];
            ld4(m.val + k, t);
#pragma unroll
            for (int u = 0; u < 4; ++u) v[u] = t[u];
        }
        if (two) {
            ld4col(m, k2, base, c, 4);
            T t[4];
            ld4(m.val + k2, t);
#pragma unroll
            for (int u = 0; u < 4; ++u) v[4 + u] = t[u];
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int kk = (u < 4 ? k : k2) + (u & 3);
            const bool ok = (u < 4 || two) && kk >= b && kk < e;
            xv[u] = ok ? xa(c[u]) : T(0);
            if (!ok) v[u] = T(0);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) s = madd<T>(s, v[u], xv[u]);
    }
    return s;
}

// CSR row sum by a group of G lanes (G a power of two dividing 32); partial sums are combined
// with a fixed butterfly over the group. Every lane of the group returns the same total. All
// lanes of the warp must call it (the shuffles use the full mask).
template <class T, class XA>
__device__ __forceinline__ T csr_group_sum(const Sell<T>& m, int row, bool valid, int sub, int G, XA xa) {
    T s = valid ? csr_lane_sum(m, row, sub, G, xa) : T(0);
    for (int o = G >> 1; o > 0; o >>= 1) s = s + __shfl_xor_sync(0xffffffffu, s, o);
    return s;
}

// CSR row sum by G = 64..256 lanes (whole warps) of a 256-thread block holding 256 / G rows:
// butterfly within each warp, then the row's warps are added in warp order. Returns the
// total in the row's first lane. Every thread of the block must call it (__syncthreads).
template <class T, class XA>
__device__ __forceinline__ T csr_block_sum(const Sell<T>& m, int row, bool valid, int sub, int G, XA xa) {
    __shared__ T red[kBlock / 32];
    T s = valid ? csr_lane_sum(m, row, sub, G, xa) : T(0);
    for (int o = 16; o > 0; o >>= 1) s = s + __shfl_xor_sync(0xffffffffu, s, o);
    const int w = static_cast<int>(threadIdx.x) >> 5;
    if ((threadIdx.x & 31) == 0) red[w] = s;
    __syncthreads();
    T t = T(0);
    if (sub == 0) {
        const int w0 = w;  // the row's first warp
        for (int q = 0; q < G / 32; ++q) t = t + red[w0 + q];
    }
    __syncthreads();
    return t;
}

struct TileCtx;

// Rows of a fine tile (CSR operators with G <= 32): one group of G = fmt lanes per row,
// blockDim = 8 * G. Wider groups take 256 / G rows per tile with blockDim 256.
constexpr int kFineRows = 8;


// Row-visiting strategies of the tiled kernels, fixed at compile time so that each kernel
// instance holds the registers of one strategy only:
//  kVisitSell2  SELL, two rows per thread per pass (big tiles of the Krylov kernels, and the
//               V-cycle kernels with Tuning.vcycle_pair), rows optionally reordered;
//  kVisitSell1  SELL, one row per thread per pass, rows optionally reordered (V-cycle kernels);
//  kVisitWarp   CSR, G <= 32 lanes per row (8 rows per tile);
//  kVisitBlock  CSR, G = 64..256 lanes per row (256 / G rows per tile).
enum : int { kVisitSell2 = 0, kVisitSell1 = 1, kVisitWarp = 2, kVisitBlock = 3 };

// Calls f(row, sum_j a_row,j xa(j)) for every row of the tile.
template <int V, class T, class XA, class F>
__device__ __forceinline__ void visit_rows_v(const Sell<T>& m, int r0, int r1, XA xa, F f) {
    if constexpr (V == kVisitSell2) {
        int row = r0 + threadIdx.x;
        auto at = [&](int q) { return m.perm != nullptr ? __ldg(&m.perm[q]) : q; };
        for (; row + kBlock < r1; row += 2 * kBlock) {
            T s0, s1;
            sell_row_sum2(m, row, row + kBlock, xa, s0, s1);
            f(at(row), s0);
            f(at(row + kBlock), s1);
        }
        if (row < r1) f(at(row), sell_row_sum(m, row, xa));
    } else if constexpr (V == kVisitSell1) {
        // reordered operators: tiles are aligned windows of positions
        for (int row = r0 + threadIdx.x; row < r1; row += kBlock)
            f(m.perm != nullptr ? __ldg(&m.perm[row]) : row, sell_row_sum(m, row, xa));
    } else {
        const int G = m.fmt;
        const int row = r0 + static_cast<int>(threadIdx.x) / G;
        const int sub = static_cast<int>(threadIdx.x) & (G - 1);
        const bool valid = row < r1;
        if constexpr (V == kVisitWarp) {
            const T s = csr_group_sum(m, row, valid, sub, G, xa);
            if (valid && sub == 0) f(row, s);
        } else {
            const T s = csr_block_sum(m, row, valid, sub, G, xa);
            if (valid && sub == 0) f(row, s);
        }
    }
}

// As visit_rows_v, with each row's epilogue operands loaded ahead of its sum: e = pre(row) is
// issued before the row's column / value loads, so the loads of p[row], b[row], ... overlap the
// sum instead of following it; then f(row, sum, e). The arithmetic is unchanged. Measured on
// the jittered tet box (5.1M cells): the level-0 Krylov SpMV 104 -> 91 us and the level-0
// residual 73 -> 70 us gain from it; the one-row SELL sweeps, prolongations and restrictions
// (32 registers at full occupancy) lost 3-7 %, so they keep visit_rows_v.
template <int V, class T, class XA, class P, class F>
__device__ __forceinline__ void visit_rows_e(const Sell<T>& m, int r0, int r1, XA xa, P pre, F f) {
    if constexpr (V == kVisitSell2) {
        int row = r0 + threadIdx.x;
        auto at = [&](int q) { return m.perm != nullptr ? __ldg(&m.perm[q]) : q; };
        for (; row + kBlock < r1; row += 2 * kBlock) {
            const int ra = at(row), rb = at(row + kBlock);
            const auto e0 = pre(ra);
            const auto e1 = pre(rb);
            T s0, s1;
            sell_row_sum2(m, row, row + kBlock, xa, s0, s1);
            f(ra, s0, e0);
            f(rb, s1, e1);
        }
        if (row < r1) {
            const int ra = at(row);
            const auto e = pre(ra);
            f(ra, sell_row_sum(m, row, xa), e);
        }
    } else if constexpr (V == kVisitSell1) {
        for (int row = r0 + threadIdx.x; row < r1; row += kBlock) {
            const int rr = m.perm != nullptr ? __ldg(&m.perm[row]) : row;
            const auto e = pre(rr);
            f(rr, sell_row_sum(m, row, xa), e);
        }
    } else {
        const int G = m.fmt;
        const int row = r0 + static_cast<int>(threadIdx.x) / G;
        const int sub = static_cast<int>(threadIdx.x) & (G - 1);
        const bool valid = row < r1;
        decltype(pre(0)) e{};
        if (valid && sub == 0) e = pre(row);
        T s;
        if constexpr (V == kVisitWarp) s = csr_group_sum(m, row, valid, sub, G, xa);
        else s = csr_block_sum(m, row, valid, sub, G, xa);
        if (valid && sub == 0) f(row, s, e);
    }
}

// CTAs per SM the V-cycle kernels are compiled for: the one-row SELL sweeps fit in 32
// registers (full occupancy); the lane-group and two-row kernels hold more (FP64 most).
template <class T, int V>
constexpr int kMinBlocks = V == kVisitSell1 ? 8 : (sizeof(T) == 8 || V == kVisitSell2 ? 4 : 6);

// Strategy of an operator's V-cycle kernels.
__host__ __device__ inline int visit_of(int fmt) {
    return fmt == kFmtSell ? kVisitSell1 : (fmt <= 32 ? kVisitWarp : kVisitBlock);
}

// Tile bookkeeping shared by all tiled kernels.
struct TileCtx {
    int tile, s, r0, r1;
};

__device__ __forceinline__ bool tile_begin(const Tiles& t, const SysState* st, TileCtx& c) {
    c.tile = blockIdx.x;
    c.s = t.sys != nullptr ? __ldg(&t.sys[c.tile]) : 0;  // null: a single system
    c.r0 = __ldg(&t.row[c.tile]);
    c.r1 = __ldg(&t.row[c.tile + 1]);
    return st == nullptr || *((volatile const int*)&st[c.s].active) != 0;
}

// ---------------------------------------------------------------------------------------------
// level-0 values from the LDU (or CSR) source arrays
// ---------------------------------------------------------------------------------------------

// src indexes a virtual array [seg0 | seg1 | seg2]; -1 marks padding. For a single system the
// three segments are diag (n), upper (nf), lower (nf); for a batch all sources are one array.
struct ValueSource {
    const double* p0;
    const double* p1;
    const double* p2;
    int n1; // first index of seg1
    int n2; // first index of seg2
};

__device__ __forceinline__ double vs_load(const ValueSource& v, int i) {
    if (i < v.n1) return v.p0[i];
    if (i < v.n2) return v.p1[i - v.n1];
    return v.p2[i - v.n2];
}

// val[s] = source value of slot s; wd[i] = w * (diag_i != 0 ? 1/diag_i : 1)
// (krylov_cuda.cu:541-562: assemble_diag / assemble_faces / inv_diag kernels, fused).
static __global__ void k_fill_level0(int n_slots, int n_rows, const int* __restrict__ src,
                              const int* __restrict__ diag_src, ValueSource vs, double weight,
                              double* __restrict__ val64, float* __restrict__ val32,
                              double* __restrict__ wd64, float* __restrict__ wd32) {
    pdl_entry();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n_slots) {
        const int s = __ldg(&src[i]);
        const double v = s >= 0 ? vs_load(vs, s) : 0.0;
        if (val64 != nullptr) val64[i] = v;
        if (val32 != nullptr) val32[i] = static_cast<float>(v);
    }
    if (i < n_rows) {
        const int s = __ldg(&diag_src[i]);
        const double d = s >= 0 ? vs_load(vs, s) : 0.0;
        const double dinv = d != 0.0 ? 1.0 / d : 1.0;
        const double wd = weight * dinv;
        if (wd64 != nullptr) wd64[i] = wd;
        if (wd32 != nullptr) wd32[i] = static_cast<float>(wd);
    }
}

// Engine layout <-> caller's concatenated vectors (map[i] = caller index of engine row i, or -1).
static __global__ void k_gather_rows(int n, const int* __restrict__ map, const double* __restrict__ src,
                                     double* __restrict__ dst) {
    pdl_entry();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const int s = map[i];
        dst[i] = (s >= 0 && src != nullptr) ? src[s] : 0.0;
    }
}

// dst[i] = value on the caller's rows, 0 on padding rows.
static __global__ void k_fill_rows(int n, const int* __restrict__ map, double value, double* __restrict__ dst) {
    pdl_entry();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = map[i] >= 0 ? value : 0.0;
}

static __global__ void k_scatter_rows(int n, const int* __restrict__ map, const double* __restrict__ src,
                                      double* __restrict__ dst) {
    pdl_entry();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const int s = map[i];
        if (s >= 0) dst[s] = src[i];
    }
}

// ---------------------------------------------------------------------------------------------
// V-cycle kernels (krylov_kernels.inc:182-238, krylov_cuda.cu:392-408)
// T: arithmetic of the cycle (double: reference, float: mixed). B: type of the right-hand side
// (level 0 reads the FP64 Krylov residual directly in both modes).
// ---------------------------------------------------------------------------------------------

template <class T> __device__ __forceinline__ T jac_update(T x, T wd, T b, T ax) {
    if constexpr (sizeof(T) == 8) {
        return __dadd_rn(x, __dmul_rn(wd, __dsub_rn(b, ax)));
    } else {
        return fmaf(wd, b - ax, x);
    }
}

// First Jacobi sweep from x = 0 (A*0 = 0): x1 = 0 + wd * b, in the arithmetic of T.
template <class T, class B> __device__ __forceinline__ T first_sweep(T wd, B b) {
    if constexpr (sizeof(T) == 8) return __dadd_rn(0.0, __dmul_rn(wd, static_cast<double>(b)));
    else return wd * static_cast<T>(b);
}

// The first sweep of the next V-cycle's level-0 pre-smoothing, written by the kernels that
// produce the Krylov residual r (so no separate sweep kernel reads r again): rows below n
// (systems with a coarser level) get x1 = first_sweep(wd, r) in the V-cycle's precision.
struct X1Out {
    const float* wd32 = nullptr;
    float* x32 = nullptr;
    const double* wd64 = nullptr;
    double* x64 = nullptr;
    int n = 0;
    __device__ __forceinline__ void put(int row, double r) const {
        if (row < n) {
            if (x32 != nullptr) x32[row] = first_sweep<float>(wd32[row], r);
            if (x64 != nullptr) x64[row] = first_sweep<double>(wd64[row], r);
        }
    }
};

// First smoothing step from x = 0: x1 = 0 + wd * b (t = A*0 = 0), and when fused2 also the
// second sweep y = x1 + wd (b - A x1) with x1 of the neighbours recomputed on the fly.
template <class T, class B, int V>
static __global__ void __launch_bounds__(kBlock, (kMinBlocks<T, V>)) k_vc_first(Sell<T> a, Tiles tiles, const SysState* st,
                                                     const T* __restrict__ wd,
                                                     const B* __restrict__ b, T* __restrict__ y,
                                                     int fused2) {
    pdl_entry();
    TileCtx c;
    if (!tile_begin(tiles, st, c)) return;
    auto x1 = [&](int j) -> T {
        if constexpr (sizeof(T) == 8) return __dadd_rn(0.0, __dmul_rn(wd[j], static_cast<T>(b[j])));
        else return wd[j] * static_cast<T>(b[j]);
    };
    if (!fused2) {
        for (int row = c.r0 + threadIdx.x; row < c.r1; row += blockDim.x) y[row] = x1(row);
        return;
    }
    visit_rows_v<V>(a, c.r0, c.r1, x1, [&](int row, T s) {
        y[row] = jac_update<T>(x1(row), wd[row], static_cast<T>(b[row]), s);
    });
}

// y = x + wd (b - A x)
template <class T, class B, int V>
static __global__ void __launch_bounds__(kBlock, (kMinBlocks<T, V>)) k_vc_jacobi(Sell<T> a, Tiles tiles, const SysState* st,
                                                      const T* __restrict__ wd,
                                                      const B* __restrict__ b,
                                                      const T* __restrict__ x, T* __restrict__ y) {
    pdl_entry();
    TileCtx c;
    if (!tile_begin(tiles, st, c)) return;
    visit_rows_v<V>(a, c.r0, c.r1, [x](int j) { return x[j]; }, [&](int row, T s) {
        y[row] = jac_update<T>(x[row], wd[row], static_cast<T>(b[row]), s);
    });
}

// t = b - A x
template <class T, class B, int V>
static __global__ void __launch_bounds__(kBlock, (kMinBlocks<T, V>)) k_vc_residual(Sell<T> a, Tiles tiles, const SysState* st,
                                                        const B* __restrict__ b,
                                                        const T* __restrict__ x,
                                                        T* __restrict__ t) {
    pdl_entry();
    TileCtx c;
    if (!tile_begin(tiles, st, c)) return;
    visit_rows_e<V>(a, c.r0, c.r1, [x](int j) { return x[j]; }, [&](int row) { return b[row]; },
                    [&](int row, T s, B bi) {
                        if constexpr (sizeof(T) == 8) t[row] = __dsub_rn(static_cast<T>(bi), s);
                        else t[row] = static_cast<T>(bi) - s;
                    });
}

// y = M x (restriction into the next level's right-hand side)
template <class T, int V>
static __global__ void __launch_bounds__(kBlock, (kMinBlocks<T, V>)) k_vc_spmv(Sell<T> m, Tiles tiles, const SysState* st,
                                                    const T* __restrict__ x, T* __restrict__ y,
                                                    const T* __restrict__ wd1, T* __restrict__ x1,
                                                    int n1) {
    pdl_entry();
    TileCtx c;
    if (!tile_begin(tiles, st, c)) return;
    visit_rows_v<V>(m, c.r0, c.r1, [x](int j) { return x[j]; }, [&](int row, T s) {
        y[row] = s;
        // restriction: also the first pre-smoothing sweep of the coarser level
        if (x1 != nullptr && row < n1) x1[row] = first_sweep<T>(wd1[row], s);
    });
}

// x += P xc
template <class T, int V>
static __global__ void __launch_bounds__(kBlock, (kMinBlocks<T, V>)) k_vc_prolong(Sell<T> p, Tiles tiles, const SysState* st,
                                                       const T* __restrict__ xc,
                                                       T* __restrict__ x) {
    pdl_entry();
    TileCtx c;
    if (!tile_begin(tiles, st, c)) return;
    visit_rows_v<V>(p, c.r0, c.r1, [xc](int j) { return xc[j]; }, [&](int row, T s) {
        if constexpr (sizeof(T) == 8) x[row] = __dadd_rn(x[row], s);
        else x[row] = x[row] + s;
    });
}

// ---- coarsest level: x = M b with the dense FP64 inverse (krylov_cuda.cu:298-307) ----
// Work is split into tiles of kCoarseRows rows of one coarse block, one CTA each. Each CTA
// stages its block's right-hand side into shared memory with a TMA bulk copy (1-D
// cp.async.bulk, no multicast) and then
//  * ordered mode: one thread per row walks j = 0..n-1 in the reference order over the
//    column-major copy of the inverse (a warp's loads of one column are coalesced), eight
//    columns loaded ahead of the dependent sum;
//  * default: one warp per row over the row-major inverse (lanes stride the row, coalesced),
//    partial sums combined with a fixed butterfly.

constexpr int kCoarseRows = kBlock / 32;

struct CoarseBlocks {
    const int* sys;          // system of each block
    const int* row;          // first row of the block in its level's vectors
    const int* n;            // block size
    const long long* m_off;  // offset of the block's inverse in `mt` / `mr`
    const double* mt;        // column-major (transposed) inverses
    const double* mr;        // row-major inverses
    const int* tile_blk;     // block of each tile
    const int* tile_row;     // first row (within the block) of each tile
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

template <class TB, class TX>
static __global__ void __launch_bounds__(kBlock) k_vc_coarse(CoarseBlocks cb, const SysState* st,
                                                      const TB* const* __restrict__ b_level,
                                                      TX* const* __restrict__ x_level,
                                                      const int* __restrict__ block_level,
                                                      Control ctl, int ordered) {
    pdl_entry();
    using T = TB;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar;
    const int blk = cb.tile_blk[blockIdx.x];
    const int s = cb.sys[blk];
    if (st != nullptr && *((volatile const int*)&st[s].active) == 0) return;
    const int lvl = block_level[blk];
    const int r0 = cb.row[blk];
    const int n = cb.n[blk];
    const int i0 = cb.tile_row[blockIdx.x];
    const T* b = b_level[lvl] + r0;
    TX* x = x_level[lvl] + r0;
    T* bs = reinterpret_cast<T*>(smem_raw);
    // bytes: the block is padded to 32 rows, so this is a multiple of 128 and 16-aligned.
    const uint32_t bytes = static_cast<uint32_t>(((n + 31) / 32) * 32 * sizeof(T));
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&bar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&bar)),
                     "r"(bytes)
                     : "memory");
        uint32_t done = 0;
        while (done < bytes) {
            const uint32_t chunk = bytes - done < 32768u ? bytes - done : 32768u;
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    smem_u32(reinterpret_cast<unsigned char*>(bs) + done)),
                "l"(reinterpret_cast<const unsigned char*>(b) + done), "r"(chunk), "r"(smem_u32(&bar))
                : "memory");
            done += chunk;
        }
    }
    // bounded wait on phase 0
    auto wait_phase0 = [&](int polls) {
        uint32_t done = 0;
        for (int spin = 0; spin < polls && !done; ++spin) {
            asm volatile(
                "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                : "=r"(done)
                : "r"(smem_u32(&bar)), "r"(0)
                : "memory");
        }
        return done != 0;
    };
    if (!wait_phase0(ctl.wait_polls)) {
        if (threadIdx.x == 0) atomicExch(ctl.error, 1);
        // the expired wait must not leave the bulk copy writing this CTA's shared memory after
        // it exits: drain it (bounded too), then return
        (void)wait_phase0(kDrainPolls);
        return;
    }
    if (ordered) {
        const int i = i0 + threadIdx.x;
        if (threadIdx.x >= kCoarseRows || i >= n) return;
        const double* mt = cb.mt + cb.m_off[blk];
        double acc = 0.0;
        int j = 0;
        for (; j + 8 <= n; j += 8) {
            double m[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) m[u] = __ldg(&mt[static_cast<long long>(j + u) * n + i]);
#pragma unroll
            for (int u = 0; u < 8; ++u) acc = __dadd_rn(acc, __dmul_rn(m[u], static_cast<double>(bs[j + u])));
        }
        for (; j < n; ++j)
            acc = __dadd_rn(acc, __dmul_rn(__ldg(&mt[static_cast<long long>(j) * n + i]), static_cast<double>(bs[j])));
        x[i] = static_cast<TX>(acc);
    } else {
        const int i = i0 + (threadIdx.x >> 5);
        const int lane = threadIdx.x & 31;
        if (i >= n) return;
        const double* mr = cb.mr + cb.m_off[blk] + static_cast<long long>(i) * n;
        double acc = 0.0;
        for (int j = lane; j < n; j += 32) acc = __dadd_rn(acc, __dmul_rn(__ldg(&mr[j]), static_cast<double>(bs[j])));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc = __dadd_rn(acc, __shfl_xor_sync(0xffffffffu, acc, o));
        if (lane == 0) x[i] = static_cast<TX>(acc);
    }
}

// ---- staged SELL visit: the operator stream through shared memory ----
// The slots of a tile's rows are contiguous per chunk of kBlock positions (8 whole slices: the
// tiles start on slice boundaries), so one thread moves a chunk's values and columns into
// shared memory with two bulk copies (1-D cp.async.bulk, no multicast, mbarrier completion).
// Thread 0 keeps S - 1 chunks in flight while the block sums the current one from shared
// memory: a row's gathers then follow a shared-memory load of its columns instead of a DRAM
// load, and the bytes in flight cost no registers. Each thread takes position c0 + threadIdx.x
// of every chunk, the order in which kVisitSell1 and kVisitSell2 visit a tile, and sums each
// row in CSR order, so rows, sums and the per-thread epilogue order are theirs bit for bit. A
// chunk with more slots than a stage holds is summed from global memory as kVisitSell1 does.

__device__ __forceinline__ void mbar_init1(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(1) : "memory");
}

__device__ __forceinline__ void mbar_expect(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// 1-D bulk copy global -> this CTA's shared memory (both addresses 16-byte aligned, bytes a
// multiple of 16), completing `bytes` transactions on bar.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Bounded wait for the phase of the given parity: true once it has completed, false after
// `polls` unsuccessful tries (none when polls <= 0).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int polls) {
    uint32_t done = 0;
    for (int spin = 0; spin < polls && !done; ++spin) {
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
    }
    return done != 0;
}

// Sum of one row of a staged chunk: k = the row's first slot and e = its slice's end, both
// relative to the chunk's first slot. Eight entries per batch, their gathers in flight
// together; entries in CSR order, padding (column -1) skipped, as sell_row_sum.
template <class T, class XA>
__device__ __forceinline__ T staged_row_sum(const T* sv, const int* sc, int k, int e, XA xa) {
    T s = T(0);
    for (; k < e; k += 8 * 32) {
        int c[8];
        T xv[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) c[u] = k + 32 * u < e ? sc[k + 32 * u] : -1;
#pragma unroll
        for (int u = 0; u < 8; ++u) xv[u] = c[u] >= 0 ? xa(c[u]) : T(0);
#pragma unroll
        for (int u = 0; u < 8; ++u)
            if (c[u] >= 0) s = madd<T>(s, sv[k + 32 * u], xv[u]);
    }
    return s;
}

// As visit_rows_e over the SELL positions [r0, r1) (r0 a multiple of 32), with the operator
// staged in S buffers of `cap` slots each (dynamic shared memory: S * cap * (sizeof(T) + 4)
// bytes, cap a multiple of 32). Returns false when a bounded wait expired: ctl.error is set,
// the CTA's copies in flight have been waited out (bounded too) and the remaining rows are
// not visited; every thread returns together, so the caller's block reduction still runs.
template <int S, class T, class XA, class P, class F>
__device__ __forceinline__ bool visit_rows_staged(const Sell<T>& m, int r0, int r1, int cap, const Control& ctl,
                                                  XA xa, P pre, F f) {
    static_assert(S >= 2 && S <= 4, "stages");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar[S];
    T* sval = reinterpret_cast<T*>(smem_raw);
    int* scol = reinterpret_cast<int*>(smem_raw + static_cast<size_t>(S) * cap * sizeof(T));
    const int n_chunks = (r1 - r0 + kBlock - 1) / kBlock;
    // first slot and slot count of chunk j
    auto span = [&](int j, int& first, int& count) {
        const int c0 = r0 + j * kBlock;
        const int c1 = min(c0 + kBlock, r1);
        first = __ldg(&m.slice[c0 >> 5]);
        count = __ldg(&m.slice[(c1 + 31) >> 5]) - first;
    };
    auto fits = [cap](int count) { return count > 0 && count <= cap; };
    auto issue = [&](int j) {  // thread 0
        int first, count;
        span(j, first, count);
        if (!fits(count)) return;
        const int s = j % S;
        // the block's reads of this buffer (ordered before this thread by the block barrier)
        // precede the copy's writes
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect(&bar[s], static_cast<uint32_t>(count) * static_cast<uint32_t>(sizeof(T) + sizeof(int)));
        bulk_load(sval + static_cast<size_t>(s) * cap, m.val + first, static_cast<uint32_t>(count * sizeof(T)), &bar[s]);
        bulk_load(scol + static_cast<size_t>(s) * cap, m.col + first, static_cast<uint32_t>(count * sizeof(int)), &bar[s]);
    };
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) mbar_init1(&bar[s]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int j = 0; j < S - 1 && j < n_chunks; ++j) issue(j);
    uint32_t par = 0;  // bit s: parity of buffer s's next phase
    for (int j = 0; j < n_chunks; ++j) {
        int first, count;
        span(j, first, count);
        const bool staged = fits(count);
        const int s = j % S;
        const int pos = r0 + j * kBlock + static_cast<int>(threadIdx.x);
        const bool has = pos < r1;
        const int row = has ? (m.perm != nullptr ? __ldg(&m.perm[pos]) : pos) : 0;
        decltype(pre(0)) e{};
        if (has) e = pre(row);
        const bool late = staged && !mbar_wait(&bar[s], (par >> s) & 1u, ctl.wait_polls);
        if (__syncthreads_or(late)) {
            if (threadIdx.x == 0) {
                atomicExch(ctl.error, 1);
                // the copies of chunks j .. j + S - 2 are in flight: let them land first
                for (int q = j; q < min(j + S - 1, n_chunks); ++q) {
                    int fq, nq;
                    span(q, fq, nq);
                    if (fits(nq)) (void)mbar_wait(&bar[q % S], (par >> (q % S)) & 1u, kDrainPolls);
                }
            }
            __syncthreads();
            return false;
        }
        if (staged) par ^= 1u << s;
        if (threadIdx.x == 0 && j + S - 1 < n_chunks) issue(j + S - 1);
        if (has) {
            T sum;
            if (staged) {
                const int sl = pos >> 5;
                sum = staged_row_sum(sval + static_cast<size_t>(s) * cap, scol + static_cast<size_t>(s) * cap,
                                     __ldg(&m.slice[sl]) - first + (pos & 31), __ldg(&m.slice[sl + 1]) - first, xa);
            } else {
                sum = sell_row_sum(m, pos, xa);
            }
            f(row, sum, e);
        }
    }
    return true;
}

// ---------------------------------------------------------------------------------------------
// Krylov kernels (krylov_kernels.inc:240-301 / krylov_cuda.cu:462-507), level-0 FP64
// ---------------------------------------------------------------------------------------------

// r = b - A x ; |r|_2 ; stop if already converged (iterations = 0)
template <int V>
static __global__ void __launch_bounds__(kBlock) k_cg_init(Sell<double> a, Tiles tiles, SysState* st,
                                                    const double* __restrict__ b,
                                                    const double* __restrict__ x,
                                                    double* __restrict__ r, Reduce red,
                                                    Control ctl, X1Out x1o) {
    pdl_entry();
    TileCtx c;
    if (!tile_begin(tiles, st, c)) return;
    double rr = 0.0, unused = 0.0;
    visit_rows_e<V>(a, c.r0, c.r1, [x](int j) { return x[j]; }, [&](int row) { return b[row]; },
                    [&](int row, double ax, double bi) {
                        const double ri = __dsub_rn(bi, ax);
                        r[row] = ri;
                        x1o.put(row, ri);
                        rr = __dadd_rn(rr, __dmul_rn(ri, ri));
                    });
    if (reduce_system(rr, unused, c.tile, c.s, red) && threadIdx.x == 0) {
        SysState& s = st[c.s];
        s.res = sqrt(rr);
        s.phase = 0;
        s.first = 1;
        s.check = 0;
        s.it = 0;
        if (s.res <= s.tol) {
            s.converged = 1;
            s.iters_out = 0;
            deactivate(s, ctl);
        }
    }
}

// p = z (first) or p = z + beta p. Jacobi systems recompute z = r * jac0 (r has not changed
// since their r.z), which keeps their z in FP64 whatever the precision of `z`.
template <class Z>
static __global__ void __launch_bounds__(kBlock) k_cg_pupdate(Tiles tiles, const SysState* st,
                                                       const Z* __restrict__ z,
                                                       const double* __restrict__ r,
                                                       const double* __restrict__ jac0,
                                                       double* __restrict__ p) {
    pdl_entry();
    TileCtx c;
    if (!tile_begin(tiles, st, c)) return;
    const bool first = st[c.s].first != 0;
    const bool jsys = st[c.s].jacobi != 0;
    const double beta = st[c.s].beta;
    // four rows per thread per pass: all loads of the pass are issued before any store
    for (int r0 = c.r0 + threadIdx.x; r0 < c.r1; r0 += 4 * kBlock) {
        double zi[4], pi[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int row = r0 + u * kBlock;
            const bool ok = row < c.r1;
            zi[u] = !ok ? 0.0 : (jsys ? __dmul_rn(r[row], jac0[row]) : static_cast<double>(z[row]));
            pi[u] = ok && !first ? p[row] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int row = r0 + u * kBlock;
            if (row < c.r1) p[row] = first ? zi[u] : __dadd_rn(zi[u], __dmul_rn(beta, pi[u]));
        }
    }
}

// p.q of the tiles of one system ; alpha = rz / pq (break if pq == 0)
__device__ __forceinline__ void cg_finish_pq(double pq, const TileCtx& c, SysState* st, const Reduce& red,
                                             const Control& ctl) {
    double unused = 0.0;
    if (reduce_system(pq, unused, c.tile, c.s, red) && threadIdx.x == 0) {
        SysState& s = st[c.s];
        s.first = 0;
        s.pq = pq;
        if (pq == 0.0) {
            s.iters_out = s.it;
            s.breakdown = 1;
            deactivate(s, ctl);
        } else {
            s.alpha = s.rz / pq;
        }
    }
}

// k_cg_spmv_pq (below) with the operator staged through shared memory: S buffers of `cap`
// slots (visit_rows_staged). Same q and p.q bit for bit.
template <int S>
static __global__ void __launch_bounds__(kBlock) k_cg_spmv_pq_staged(Sell<double> a, Tiles tiles, SysState* st,
                                                              const double* __restrict__ p,
                                                              double* __restrict__ q, Reduce red,
                                                              Control ctl, int cap) {
    pdl_entry();
    TileCtx c;
    if (!tile_begin(tiles, st, c)) return;
    double pq = 0.0;
    visit_rows_staged<S>(a, c.r0, c.r1, cap, ctl, [p](int j) { return p[j]; }, [&](int row) { return p[row]; },
                         [&](int row, double qi, double pi) {
                             q[row] = qi;
                             pq = __dadd_rn(pq, __dmul_rn(pi, qi));
                         });
    cg_finish_pq(pq, c, st, red, ctl);
}

// q = A p ; p.q ; alpha = rz / pq (break if pq == 0)
template <int V>
static __global__ void __launch_bounds__(kBlock) k_cg_spmv_pq(Sell<double> a, Tiles tiles, SysState* st,
                                                       const double* __restrict__ p,
                                                       double* __restrict__ q, Reduce red,
                                                       Control ctl) {
    pdl_entry();
    TileCtx c;
    if (!tile_begin(tiles, st, c)) return;
    double pq = 0.0;
    visit_rows_e<V>(a, c.r0, c.r1, [p](int j) { return p[j]; }, [&](int row) { return p[row]; },
                    [&](int row, double qi, double pi) {
                        q[row] = qi;
                        pq = __dadd_rn(pq, __dmul_rn(pi, qi));
                    });
    cg_finish_pq(pq, c, st, red, ctl);
}

// x += alpha p ; r -= alpha q ; |r|_2 ; converged?
// verify_true: mixed mode marks the system for an FP64 true-residual check instead.
// X1: the V-cycle's first sweep written from the new r (x1o): 0 none, 1 FP32, 2 FP64; its
// weights are loaded with the pass's other operands (an instance per form, so the instance
// without it holds no registers for them).
template <int X1>
static __global__ void __launch_bounds__(kBlock, (X1 == 0 ? 5 : 4)) k_cg_xr(Tiles tiles, SysState* st,
                                                  double* __restrict__ x, double* __restrict__ r,
                                                  const double* __restrict__ p,
                                                  const double* __restrict__ q, Reduce red,
                                                  Control ctl, int verify_true, X1Out x1o) {
    pdl_entry();
    TileCtx c;
    if (!tile_begin(tiles, st, c)) return;
    const double alpha = st[c.s].alpha;
    double rr = 0.0, unused = 0.0;
    // four rows per thread per pass: all loads of the pass are issued before any store
    for (int r0 = c.r0 + threadIdx.x; r0 < c.r1; r0 += 4 * kBlock) {
        double xi[4], pi[4], ri[4], qi[4], w64[4];
        float w32[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int row = r0 + u * kBlock;
            const bool ok = row < c.r1;
            xi[u] = ok ? x[row] : 0.0;
            pi[u] = ok ? p[row] : 0.0;
            ri[u] = ok ? r[row] : 0.0;
            qi[u] = ok ? q[row] : 0.0;
            if constexpr (X1 == 1) w32[u] = ok && row < x1o.n ? x1o.wd32[row] : 0.0f;
            if constexpr (X1 == 2) w64[u] = ok && row < x1o.n ? x1o.wd64[row] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int row = r0 + u * kBlock;
            if (row >= c.r1) continue;
            x[row] = __dadd_rn(xi[u], __dmul_rn(alpha, pi[u]));
            const double rn = __dsub_rn(ri[u], __dmul_rn(alpha, qi[u]));
            r[row] = rn;
            if constexpr (X1 == 1) {
                if (row < x1o.n) x1o.x32[row] = first_sweep<float>(w32[u], rn);
            }
            if constexpr (X1 == 2) {
                if (row < x1o.n) x1o.x64[row] = first_sweep<double>(w64[u], rn);
            }
            rr = __dadd_rn(rr, __dmul_rn(rn, rn));
        }
    }
    if (reduce_system(rr, unused, c.tile, c.s, red) && threadIdx.x == 0) {
        SysState& s = st[c.s];
        s.res = sqrt(rr);
        if (s.res <= s.tol) {
            if (verify_true && !s.jacobi) {
                s.check = 1;
            } else {
                s.converged = 1;
                s.iters_out = s.it;
                deactivate(s, ctl);
            }
        }
    }
}

// Mixed precision: for systems whose recursive residual met the target, recompute
// r = b - A x in FP64; converged if |r| <= tol, else restart the search direction.
template <int V>
static __global__ void __launch_bounds__(kBlock) k_cg_true_check(Sell<double> a, Tiles tiles, SysState* st,
                                                          const double* __restrict__ b,
                                                          const double* __restrict__ x,
                                                          double* __restrict__ r, Reduce red,
                                                          Control ctl, X1Out x1o) {
    pdl_entry();
    TileCtx c;
    if (!tile_begin(tiles, st, c)) return;
    if (st[c.s].check == 0) return;
    double rr = 0.0, unused = 0.0;
    visit_rows_e<V>(a, c.r0, c.r1, [x](int j) { return x[j]; }, [&](int row) { return b[row]; },
                    [&](int row, double ax, double bi) {
                        const double ri = __dsub_rn(bi, ax);
                        r[row] = ri;
                        x1o.put(row, ri);
                        rr = __dadd_rn(rr, __dmul_rn(ri, ri));
                    });
    if (reduce_system(rr, unused, c.tile, c.s, red) && threadIdx.x == 0) {
        SysState& s = st[c.s];
        s.check = 0;
        s.res = sqrt(rr);
        if (s.res <= s.tol) {
            s.converged = 1;
            s.iters_out = s.it;
            deactivate(s, ctl);
        } else {
            s.first = 1;
        }
    }
}

// Scalar tail of the preconditioning step for one system (last CTA, thread 0):
// rz_new (and zq = z.q for the flexible variant) -> beta, iteration counter.
__device__ __forceinline__ void precond_tail(SysState& s, double rz_new, double zq, int flexible,
                                             Control ctl) {
    if (s.phase == 0) {
        s.phase = 1;
        s.rz = rz_new;
        s.it = 1;
    } else {
        if (!s.first) {
            // reference: beta = rz_new / rz; flexible CG (Notay): beta = -(z . q) / (p . q)
            s.beta = flexible ? -(zq / s.pq) : rz_new / s.rz;
        }
        s.rz = rz_new;
        s.it += 1;
    }
    if (s.it > s.max_it) {
        s.iters_out = s.max_it;
        deactivate(s, ctl);
    }
}

// Last post-smoothing sweep of level 0 fused with r.z (and z.q): z = x + wd (b - A x).
template <class T, int V>
static __global__ void __launch_bounds__(kBlock) k_vc_jacobi_final(Sell<T> a, Tiles tiles, SysState* st,
                                                            const T* __restrict__ wd,
                                                            const double* __restrict__ r,
                                                            const T* __restrict__ x,
                                                            T* __restrict__ z,
                                                            const double* __restrict__ q,
                                                            Reduce red, Control ctl,
                                                            int flexible) {
    pdl_entry();
    TileCtx c;
    if (!tile_begin(tiles, st, c)) return;
    double rz = 0.0, zq = 0.0;
    visit_rows_v<V>(a, c.r0, c.r1, [x](int j) { return x[j]; }, [&](int row, T s) {
        const double ri = r[row];
        const T zi = jac_update<T>(x[row], wd[row], static_cast<T>(ri), s);
        z[row] = zi;
        const double zd = static_cast<double>(zi);
        rz = __dadd_rn(rz, __dmul_rn(ri, zd));
        if (flexible) zq = __dadd_rn(zq, __dmul_rn(zd, q[row]));
    });
    if (reduce_system(rz, zq, c.tile, c.s, red) && threadIdx.x == 0) {
        precond_tail(st[c.s], rz, zq, flexible, ctl);
    }
}

// Unfused r.z (and z.q) when the preconditioner output is not produced by a smoothing sweep
// (no smoothing; Jacobi preconditioning z = dinv * r for every system when jac != null, or for
// the systems flagged `jacobi` (jac0, z not stored: k_cg_pupdate recomputes it)).
template <class Z>
static __global__ void __launch_bounds__(kBlock) k_cg_rz(Tiles tiles, SysState* st,
                                                  const double* __restrict__ r,
                                                  Z* __restrict__ z, const double* __restrict__ jac,
                                                  const double* __restrict__ jac0,
                                                  const double* __restrict__ q, Reduce red,
                                                  Control ctl, int flexible) {
    pdl_entry();
    TileCtx c;
    if (!tile_begin(tiles, st, c)) return;
    const bool jsys = st[c.s].jacobi != 0;
    const int flex = jsys ? 0 : flexible;
    double rz = 0.0, zq = 0.0;
    // four rows per thread per pass: all loads of the pass are issued before the sums
    for (int r0 = c.r0 + threadIdx.x; r0 < c.r1; r0 += 4 * kBlock) {
        double ri[4], zd[4], qi[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int row = r0 + u * kBlock;
            const bool ok = row < c.r1;
            ri[u] = ok ? r[row] : 0.0;
            if (!ok) {
                zd[u] = 0.0;
            } else if (jac != nullptr) {
                zd[u] = __dmul_rn(ri[u], jac[row]);
            } else if (jsys) {
                zd[u] = __dmul_rn(ri[u], jac0[row]);
            } else {
                zd[u] = static_cast<double>(z[row]);
            }
            qi[u] = ok && flex ? q[row] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int row = r0 + u * kBlock;
            if (row >= c.r1) continue;
            if (jac != nullptr) z[row] = static_cast<Z>(zd[u]);
            rz = __dadd_rn(rz, __dmul_rn(ri[u], zd[u]));
            if (flex) zq = __dadd_rn(zq, __dmul_rn(zd[u], qi[u]));
        }
    }
    if (reduce_system(rz, zq, c.tile, c.s, red) && threadIdx.x == 0) {
        precond_tail(st[c.s], rz, zq, flex, ctl);
    }
}

// |b - A x|_2 per system into st.true_res (reporting only; all systems).
template <int V>
static __global__ void __launch_bounds__(kBlock) k_true_residual(Sell<double> a, Tiles tiles, SysState* st,
                                                          const double* __restrict__ b,
                                                          const double* __restrict__ x,
                                                          Reduce red) {
    pdl_entry();
    TileCtx c;
    tile_begin(tiles, nullptr, c);
    double rr = 0.0, unused = 0.0;
    visit_rows_v<V>(a, c.r0, c.r1, [x](int j) { return x[j]; }, [&](int row, double ax) {
        const double ri = __dsub_rn(b[row], ax);
        rr = __dadd_rn(rr, __dmul_rn(ri, ri));
    });
    if (reduce_system(rr, unused, c.tile, c.s, red) && threadIdx.x == 0) {
        st[c.s].true_res = sqrt(rr);
    }
}

// ---------------------------------------------------------------------------------------------
// Face-loop assembly (krylov_cuda.cu:681-697 / krylov_openmp.cpp:289-300), atomic-free.
// Each cell gathers its faces in ascending face order, which reproduces the serial loop's
// accumulation order bit for bit. cf_face[k] holds the face, cf_sign[k] 0 when the cell owns it.
// ---------------------------------------------------------------------------------------------
static __global__ void k_assemble_faces(int nf, const double* __restrict__ flux,
                                 const double* __restrict__ gamma,
                                 const double* __restrict__ delta, double convection,
                                 double* __restrict__ upper, double* __restrict__ lower) {
    pdl_entry();
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const double fl = flux[f];
    const double g = __dmul_rn(gamma[f], delta[f]);
    const double pos = fl > 0.0 ? __dmul_rn(convection, fl) : 0.0;
    const double neg = fl < 0.0 ? __dmul_rn(convection, fl) : 0.0;
    upper[f] = __dsub_rn(neg, g);
    lower[f] = __dsub_rn(-pos, g);
}

// Conservative face flux from the pressure solution (flow_solver.cpp:821-826):
// phi = flux - (gamma * delta) * (p[N] - p[P]) - non_orth (non_orth may be null: zero),
// rounded in that order.
static __global__ void k_correct_flux(int nf, const int* __restrict__ owner, const int* __restrict__ neighbour,
                                      const double* __restrict__ flux, const double* __restrict__ gamma,
                                      const double* __restrict__ delta, const double* __restrict__ non_orth,
                                      const double* __restrict__ p, double* __restrict__ phi) {
    pdl_entry();
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const double dp = __dsub_rn(p[neighbour[f]], p[owner[f]]);
    const double v = __dsub_rn(flux[f], __dmul_rn(__dmul_rn(gamma[f], delta[f]), dp));
    phi[f] = __dsub_rn(v, non_orth != nullptr ? non_orth[f] : 0.0);
}

// Pressure under-relaxation (flow_solver.cpp:837-840): p = p_prev + alpha (p_new - p_prev), or
// p = p_new when p_prev is null.
static __global__ void k_relax(int n, const double* __restrict__ p_prev, const double* __restrict__ p_new,
                               double alpha, double* __restrict__ p) {
    pdl_entry();
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    p[c] = p_prev != nullptr ? __dadd_rn(p_prev[c], __dmul_rn(alpha, __dsub_rn(p_new[c], p_prev[c]))) : p_new[c];
}

// Pressure assembly epilogue fused into the cell gather (flow_solver.cpp:768-770 and 794-796):
// diag = diag0 + sum of face coefficients, source = source0 - div(flux), then
// set_reference(ref_cell, ref_value): source += diag * value, diag += diag (for the cell
// ref_cell, or every cell flagged in ref_mask when batches carry one reference per system).
static __global__ void k_assemble_pressure_cells(int n, const int* __restrict__ cf_ptr,
                                                 const int* __restrict__ cf_face,
                                                 const double* __restrict__ flux,
                                                 const double* __restrict__ gamma,
                                                 const double* __restrict__ delta,
                                                 const int* __restrict__ owner,
                                                 const double* __restrict__ diag0,
                                                 const double* __restrict__ source0, int ref_cell,
                                                 const int* __restrict__ ref_mask, double ref_value,
                                                 double* __restrict__ diag,
                                                 double* __restrict__ source) {
    pdl_entry();
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    double d = diag0 != nullptr ? diag0[c] : 0.0;
    double v = 0.0;
    const int end = cf_ptr[c + 1];
    for (int k = cf_ptr[c]; k < end; ++k) {
        const int f = cf_face[k];
        const double fl = flux[f];
        const double g = __dmul_rn(gamma[f], delta[f]);
        d = __dadd_rn(d, __dadd_rn(0.0, g));
        if (owner[f] == c) v = __dadd_rn(v, fl);
        else v = __dsub_rn(v, fl);
    }
    double src = __dsub_rn(source0[c], v);
    if (c == ref_cell || (ref_mask != nullptr && ref_mask[c] != 0)) {
        src = __dadd_rn(src, __dmul_rn(d, ref_value));
        d = __dadd_rn(d, d);
    }
    diag[c] = d;
    source[c] = src;
}

// Diagonal and divergence of cell c: its faces in ascending order, added to what diag and div
// hold (assemble_convection_diffusion accumulates).
static __device__ __forceinline__ void assemble_cell(int c, const int* __restrict__ cf_ptr,
                                                     const int* __restrict__ cf_face,
                                                     const double* __restrict__ flux,
                                                     const double* __restrict__ gamma,
                                                     const double* __restrict__ delta,
                                                     const int* __restrict__ owner, double convection,
                                                     double* __restrict__ diag, double* __restrict__ div);

static __global__ void k_assemble_cells(int n, const int* __restrict__ cf_ptr,
                                 const int* __restrict__ cf_face, const double* __restrict__ flux,
                                 const double* __restrict__ gamma,
                                 const double* __restrict__ delta, const int* __restrict__ owner,
                                 double convection, double* __restrict__ diag,
                                 double* __restrict__ div) {
    pdl_entry();
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    assemble_cell(c, cf_ptr, cf_face, flux, gamma, delta, owner, convection, diag, div);
}

// Cells [c0, c1) only: one slice of a host-array assembly whose copies are pipelined.
static __global__ void k_assemble_cell_range(int c0, int c1, const int* __restrict__ cf_ptr,
                                             const int* __restrict__ cf_face, const double* __restrict__ flux,
                                             const double* __restrict__ gamma, const double* __restrict__ delta,
                                             const int* __restrict__ owner, double convection,
                                             double* __restrict__ diag, double* __restrict__ div) {
    const int c = c0 + static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    if (c >= c1) return;
    assemble_cell(c, cf_ptr, cf_face, flux, gamma, delta, owner, convection, diag, div);
}

static __device__ __forceinline__ void assemble_cell(int c, const int* __restrict__ cf_ptr,
                                                     const int* __restrict__ cf_face,
                                                     const double* __restrict__ flux,
                                                     const double* __restrict__ gamma,
                                                     const double* __restrict__ delta,
                                                     const int* __restrict__ owner, double convection,
                                                     double* __restrict__ diag, double* __restrict__ div) {
    double d = diag[c];
    double v = div[c];
    const int end = cf_ptr[c + 1];
    for (int k = cf_ptr[c]; k < end; ++k) {
        const int f = cf_face[k];
        const double fl = flux[f];
        const double g = __dmul_rn(gamma[f], delta[f]);
        const double pos = fl > 0.0 ? __dmul_rn(convection, fl) : 0.0;
        const double neg = fl < 0.0 ? __dmul_rn(convection, fl) : 0.0;
        if (owner[f] == c) {
            d = __dadd_rn(d, __dadd_rn(pos, g));
            v = __dadd_rn(v, fl);
        } else {
            d = __dadd_rn(d, __dadd_rn(-neg, g));
            v = __dsub_rn(v, fl);
        }
    }
    diag[c] = d;
    div[c] = v;
}

// ---------------------------------------------------------------------------------------------
// V-cycle tail: the small coarse levels and the dense coarse solve in one persistent kernel.
// Each coarse level costs six small kernels whose run time is launch and ramp latency; here
// every phase is a grid-stride loop over the operator's rows, separated by a grid barrier.
// The kernel is launched cooperatively (all CTAs co-resident) and every barrier wait is
// bounded: on expiry the kernel sets the error flag and returns. It processes every system's
// rows (no per-system activity test: the rows of converged systems are only level vectors).
// Phase arithmetic is the same per row as the separate kernels (same lane sums and coarse
// row products), so the results do not depend on which path ran.
// ---------------------------------------------------------------------------------------------
enum : int { kTailJacobi = 0, kTailResidual = 1, kTailRestrict = 2, kTailProlong = 3, kTailCoarse = 4 };

template <class T> struct TailPhase {
    int kind;
    int n;          // rows of the operator
    Sell<T> m;      // CSR operator (lane groups); unused by kTailCoarse
    const T* x;     // gathered vector (A x, R t, P xc)
    const T* b;     // right-hand side (jacobi, residual)
    const T* wd;    // w/diag (jacobi), or of the coarser level (restriction's first sweep)
    T* y;           // output (jacobi / residual / restriction), iterate (prolongation, in place)
    T* x1;          // restriction: first sweep of the coarser level (rows < n1), or null
    int n1;
};

// Grid-wide barrier over `nblocks` co-resident CTAs: bar[0] counts arrivals, bar[1] is the
// generation. Bounded by `limit` polls (< 0: none): returns false (error flag set) if the
// generation does not move. After an expiry the counters are stale; the host resets them.
__device__ __forceinline__ bool tail_barrier(unsigned* bar, unsigned nblocks, int* error, int limit) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* gen = bar + 1;
        const unsigned g0 = *gen;
        __threadfence();
        int good = 1;
        if (atomicAdd(&bar[0], 1u) + 1u == nblocks) {
            atomicExch(&bar[0], 0u);
            __threadfence();
            atomicAdd(&bar[1], 1u);
        } else {
            for (int spin = 0; *gen == g0; ++spin) {
                if (spin >= limit) {
                    good = 0;
                    atomicExch(error, 2);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

// f(row, sum) for every row of a CSR lane-group operator, grid-stride over blocks of
// kBlock / G rows (every thread of a block runs the same number of passes).
template <class T, class XA, class F>
__device__ __forceinline__ void tail_rows(const Sell<T>& m, int n, XA xa, F f) {
    const int G = m.fmt;
    const int rpb = kBlock / G;
    const int sub = static_cast<int>(threadIdx.x) & (G - 1);
    for (int base = blockIdx.x * rpb; base < n; base += gridDim.x * rpb) {
        const int row = base + static_cast<int>(threadIdx.x) / G;
        const bool valid = row < n;
        T s;
        if (G <= 32) s = csr_group_sum(m, row, valid, sub, G, xa);
        else s = csr_block_sum(m, row, valid, sub, G, xa);
        if (valid && sub == 0) f(row, s);
    }
}

// Barrier over the CTAs of one thread-block cluster (all of them run every phase): the
// hardware cluster barrier with release / acquire semantics at cluster scope, so the global
// writes of one phase are visible to the loads of the next. No polling: it cannot time out.
__device__ __forceinline__ void tail_cluster_barrier() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// The phases of the small coarse levels and the coarse solve in one launch. kCluster = false:
// a cooperative grid of co-resident CTAs separated by the bounded grid barrier; kCluster =
// true: a single thread-block cluster (gridDim.x = cluster size) separated by the cluster
// barrier, for levels small enough that a few SMs keep up with them.
template <class T, bool kCluster>
static __global__ void __launch_bounds__(kBlock, 4) k_vc_tail(const TailPhase<T>* __restrict__ phases, int n_phases,
                                                    CoarseBlocks cb, int n_ctiles, T* const* __restrict__ b_level,
                                                    T* const* __restrict__ x_level,
                                                    const int* __restrict__ block_level, unsigned* bar,
                                                    int* error, int wait_polls) {
    extern __shared__ __align__(16) unsigned char tail_smem[];
    for (int ph = 0; ph < n_phases; ++ph) {
        const TailPhase<T> P = phases[ph];
        if (P.kind == kTailCoarse) {
            T* bs = reinterpret_cast<T*>(tail_smem);
            for (int t = blockIdx.x; t < n_ctiles; t += gridDim.x) {
                const int blk = cb.tile_blk[t];
                const int n = cb.n[blk];
                const int r0 = cb.row[blk];
                const int lvl = block_level[blk];
                const T* b = b_level[lvl] + r0;
                T* x = x_level[lvl] + r0;
                for (int j = threadIdx.x; j < n; j += kBlock) bs[j] = __ldcg(&b[j]);
                __syncthreads();
                const int i = cb.tile_row[t] + (threadIdx.x >> 5);
                const int lane = threadIdx.x & 31;
                if (i < n) {
                    const double* mr = cb.mr + cb.m_off[blk] + static_cast<long long>(i) * n;
                    double acc = 0.0;
                    for (int j = lane; j < n; j += 32) acc = __dadd_rn(acc, __dmul_rn(__ldg(&mr[j]), static_cast<double>(bs[j])));
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) acc = __dadd_rn(acc, __shfl_xor_sync(0xffffffffu, acc, o));
                    if (lane == 0) x[i] = static_cast<T>(acc);
                }
                __syncthreads();
            }
        } else {
            // vectors written by earlier phases of this kernel are read through L2 (ld.cg): the
            // grid barrier orders the writes, and L2 is coherent across SMs. One row-sum
            // instance serves every phase kind (the kind only selects the epilogue).
            const T* x = P.x;
            auto xa = [x](int j) { return __ldcg(&x[j]); };
            tail_rows(P.m, P.n, xa, [&](int row, T s) {
                if (P.kind == kTailJacobi) {
                    P.y[row] = jac_update<T>(__ldcg(&x[row]), P.wd[row], __ldcg(&P.b[row]), s);
                } else if (P.kind == kTailResidual) {
                    if constexpr (sizeof(T) == 8) P.y[row] = __dsub_rn(__ldcg(&P.b[row]), s);
                    else P.y[row] = __ldcg(&P.b[row]) - s;
                } else if (P.kind == kTailRestrict) {
                    P.y[row] = s;
                    if (P.x1 != nullptr && row < P.n1) P.x1[row] = first_sweep<T>(P.wd[row], s);
                } else {
                    if constexpr (sizeof(T) == 8) P.y[row] = __dadd_rn(__ldcg(&P.y[row]), s);
                    else P.y[row] = __ldcg(&P.y[row]) + s;
                }
            });
        }
        if (ph + 1 < n_phases) {
            if constexpr (kCluster) tail_cluster_barrier();
            else if (!tail_barrier(bar, gridDim.x, error, wait_polls)) return;
        }
    }
}

} // namespace cfdb
