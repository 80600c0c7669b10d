// Allocation-free variant of the Jacobi-preconditioned CG solve (declared in include/cfdb.h as
// cfdb_solve_device_noalloc).
//
// Why it exists: cudaMalloc synchronises the device and may block, and some callers cannot
// use it at all -- a host application that has already carved the GPU's memory into its own
// pool (a flow solver whose time loop owns every device buffer), a latency-critical loop that
// must never stall on the allocator, or code that runs while another component forbids new
// allocations. This entry point takes the caller's device arrays for the matrix, right-hand
// side and solution and keeps every work vector in one file-scope static device array, so the
// call itself never allocates device memory.
//
// Limits and caveats:
//  * at most kNaMaxRows (65,536) rows; larger systems are rejected with CFDB_ERR_BAD_ARG;
//  * the static array (about 2.6 MB) is held by every GPU that loads the library until exit;
//  * on each device, the first call looks up the array's device address with
//    cudaGetSymbolAddress (host code must not pass the symbol itself to a kernel); make that
//    first call before any stream capture;
//  * every call shares the array and leaves its last contents there; calls that overlap on the
//    GPU (for example from two host threads at once) race and must be serialised by the caller;
//  * it runs on the legacy default stream: a caller that wrote a, b or x on a non-blocking
//    stream must finish those writes (synchronise that stream) before the call;
//  * the arrays must be device memory of the current device (or managed memory), and the CSR
//    structure is checked on the device before use (row offsets, then column indices).
#include "../../include/cfdb.h"

#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>

#include "common.hpp"
#include "pointer_rule.hpp"

static_assert(static_cast<int>(cudaMemoryTypeUnregistered) == cfdb::kPtrUnregistered &&
                  static_cast<int>(cudaMemoryTypeHost) == cfdb::kPtrHost &&
                  static_cast<int>(cudaMemoryTypeDevice) == cfdb::kPtrDevice &&
                  static_cast<int>(cudaMemoryTypeManaged) == cfdb::kPtrManaged,
              "cudaMemoryType values");

namespace cfdb {
void set_thread_error(const std::string& msg); // capi.cu
}

namespace {

constexpr int kNaMaxRows = 65536;
constexpr int kNaBlock = 256;
constexpr int kNaMaxBlocks = kNaMaxRows / kNaBlock;
// Layout in doubles: dinv | r | z | p | q | partial sums (one per block) | scalars (32 slots:
// slot 0 the reduced scalar, slots 8.. the validation flags as ints).
constexpr size_t kNaVec = static_cast<size_t>(kNaMaxRows);
constexpr size_t kNaOffPart = 5 * kNaVec;
constexpr size_t kNaOffScalar = kNaOffPart + kNaMaxBlocks;
constexpr size_t kNaDoubles = kNaOffScalar + 32;
constexpr size_t kNaFlagSlot = 8;

static __device__ __align__(256) double g_na_scratch[kNaDoubles];

std::mutex g_na_mu;
constexpr int kNaMaxDevices = 64;
double* g_na_base[kNaMaxDevices] = {};

// Device address of the scratch array on the current device (looked up once per device).
double* scratch_base(int dev) {
    if (dev < 0 || dev >= kNaMaxDevices) cfdb::fail(CFDB_ERR_BAD_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_na_mu);
    if (g_na_base[dev] == nullptr) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_na_scratch);
        if (e != cudaSuccess) {
            (void)cudaGetLastError();
            cfdb::fail(CFDB_ERR_CUDA, std::string("CUDA cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        }
        g_na_base[dev] = static_cast<double*>(p);
    }
    return g_na_base[dev];
}

struct NaCsr {
    int n;
    const int* rp;
    const int* ci;
    const double* va;
};

__device__ __forceinline__ double na_row(const NaCsr& a, int i, const double* __restrict__ x) {
    double s = 0.0;
    for (int k = a.rp[i]; k < a.rp[i + 1]; ++k) s = __dadd_rn(s, __dmul_rn(a.va[k], x[a.ci[k]]));
    return s;
}

// Block sum of one value into part[blockIdx.x] (fixed tree: deterministic).
__device__ __forceinline__ void na_block_sum(double v, double* part) {
    __shared__ double sh[kNaBlock / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = threadIdx.x < kNaBlock / 32 ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) part[blockIdx.x] = v;
    }
}

// CSR structure checks before any kernel reads through the caller's indices. Rows: every
// row_ptr entry in [0, nnz], non-decreasing, row_ptr[0] = 0 and row_ptr[n] = nnz (flag bit 1).
__global__ void k_na_check_rows(int n, int nnz, const int* __restrict__ rp, int* flag) {
    const int i = blockIdx.x * kNaBlock + threadIdx.x;
    if (i > n) return;
    const int v = rp[i];
    bool bad = v < 0 || v > nnz || (i == 0 && v != 0) || (i == n && v != nnz);
    if (i < n) bad = bad || rp[i + 1] < v;
    if (bad) atomicOr(flag, 1);
}

// Columns (run only once the rows passed): every column index in [0, n) (flag bit 2).
__global__ void k_na_check_cols(int n, int nnz, const int* __restrict__ ci, int* flag) {
    for (int k = blockIdx.x * kNaBlock + threadIdx.x; k < nnz; k += gridDim.x * kNaBlock) {
        const int c = ci[k];
        if (c < 0 || c >= n) {
            atomicOr(flag, 2);
            return;
        }
    }
}

// dinv = 1 / (last nonzero diagonal entry), 1 if none (krylov_openmp.cpp:99-106);
// r = b - A x; partial r.r
__global__ void k_na_init(NaCsr a, const double* __restrict__ b, const double* __restrict__ x,
                          double* __restrict__ dinv, double* __restrict__ r, double* part) {
    const int i = blockIdx.x * kNaBlock + threadIdx.x;
    double rr = 0.0;
    if (i < a.n) {
        double d = 1.0;
        for (int k = a.rp[i]; k < a.rp[i + 1]; ++k)
            if (a.ci[k] == i && a.va[k] != 0.0) d = 1.0 / a.va[k];
        dinv[i] = d;
        const double ri = __dsub_rn(b[i], na_row(a, i, x));
        r[i] = ri;
        rr = __dmul_rn(ri, ri);
    }
    na_block_sum(rr, part);
}

// z = r * dinv; p = z when first; partial r.z
__global__ void k_na_precond(int n, const double* __restrict__ r, const double* __restrict__ dinv,
                             double* __restrict__ z, double* __restrict__ p, int first, double* part) {
    const int i = blockIdx.x * kNaBlock + threadIdx.x;
    double rz = 0.0;
    if (i < n) {
        const double zi = __dmul_rn(r[i], dinv[i]);
        z[i] = zi;
        if (first) p[i] = zi;
        rz = __dmul_rn(r[i], zi);
    }
    na_block_sum(rz, part);
}

// q = A p; partial p.q
__global__ void k_na_spmv(NaCsr a, const double* __restrict__ p, double* __restrict__ q, double* part) {
    const int i = blockIdx.x * kNaBlock + threadIdx.x;
    double pq = 0.0;
    if (i < a.n) {
        const double qi = na_row(a, i, p);
        q[i] = qi;
        pq = __dmul_rn(p[i], qi);
    }
    na_block_sum(pq, part);
}

// x += alpha p; r -= alpha q; partial r.r
__global__ void k_na_update(int n, double alpha, const double* __restrict__ p, const double* __restrict__ q,
                            double* __restrict__ x, double* __restrict__ r, double* part) {
    const int i = blockIdx.x * kNaBlock + threadIdx.x;
    double rr = 0.0;
    if (i < n) {
        x[i] = __dadd_rn(x[i], __dmul_rn(alpha, p[i]));
        const double ri = __dsub_rn(r[i], __dmul_rn(alpha, q[i]));
        r[i] = ri;
        rr = __dmul_rn(ri, ri);
    }
    na_block_sum(rr, part);
}

// p = z + beta p
__global__ void k_na_pupdate(int n, double beta, const double* __restrict__ z, double* __restrict__ p) {
    const int i = blockIdx.x * kNaBlock + threadIdx.x;
    if (i < n) p[i] = __dadd_rn(z[i], __dmul_rn(beta, p[i]));
}

// partial (b - A x)^2 for the reported true residual
__global__ void k_na_true(NaCsr a, const double* __restrict__ b, const double* __restrict__ x, double* part) {
    const int i = blockIdx.x * kNaBlock + threadIdx.x;
    double rr = 0.0;
    if (i < a.n) {
        const double ri = __dsub_rn(b[i], na_row(a, i, x));
        rr = __dmul_rn(ri, ri);
    }
    na_block_sum(rr, part);
}

// Sum of the block partials in a fixed order into *out (one warp).
__global__ void k_na_finish(int n_blocks, const double* __restrict__ part, double* out) {
    double s = 0.0;
    for (int t = threadIdx.x; t < n_blocks; t += 32) s += part[t];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) *out = s;
}

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        cfdb::fail(e == cudaErrorMemoryAllocation ? CFDB_ERR_OOM : CFDB_ERR_CUDA,
                   std::string("CUDA ") + what + ": " + cudaGetErrorString(e));
    }
}

// Device memory of the current device, or managed memory.
bool usable_here(const void* p, int dev) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return cfdb::pointer_usable_on(static_cast<int>(at.type), at.device, dev);
}

} // namespace

extern "C" int cfdb_solve_device_noalloc(const cfdb_csr* a, const double* b, double* x, int method,
                                         const cfdb_control* control, cfdb_stats* stats) {
    try {
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
            (void)cudaGetLastError();
            cfdb::fail(CFDB_ERR_NO_DEVICE, "no CUDA device: this library has no host fallback");
        }
        if (a == nullptr || b == nullptr || x == nullptr || control == nullptr)
            cfdb::fail(CFDB_ERR_BAD_ARG, "cfdb_solve_device_noalloc: null argument");
        if (method != CFDB_METHOD_CG)
            cfdb::fail(CFDB_ERR_BAD_ARG, "cfdb_solve_device_noalloc: only CG (Jacobi-preconditioned) is provided");
        if (a->n < 0 || a->nnz < 0) cfdb::fail(CFDB_ERR_BAD_ARG, "cfdb_solve_device_noalloc: negative size");
        if (a->n > kNaMaxRows) {
            cfdb::fail(CFDB_ERR_BAD_ARG, "cfdb_solve_device_noalloc: n = " + std::to_string(a->n) +
                                             " exceeds the maximum of " + std::to_string(kNaMaxRows) +
                                             " rows of its static scratch");
        }
        if (a->n == 0) {
            if (stats) *stats = cfdb_stats{0, 0.0, 1, 1, 0.0};
            return CFDB_OK;
        }
        int dev = 0;
        check(cudaGetDevice(&dev), "cudaGetDevice");
        if (!usable_here(a->row_ptr, dev) || !usable_here(a->col, dev) || !usable_here(a->val, dev) ||
            !usable_here(b, dev) || !usable_here(x, dev)) {
            cfdb::fail(CFDB_ERR_BAD_ARG, "cfdb_solve_device_noalloc: every array must be device memory of the "
                                         "current device (device " + std::to_string(dev) + ") or managed memory");
        }
        double* base = scratch_base(dev);
        const int n = a->n;
        double* dinv = base;
        double* r = base + kNaVec;
        double* z = base + 2 * kNaVec;
        double* p = base + 3 * kNaVec;
        double* q = base + 4 * kNaVec;
        double* part = base + kNaOffPart;
        double* scalar = base + kNaOffScalar;
        const NaCsr m{n, a->row_ptr, a->col, a->val};
        const int blocks = (n + kNaBlock - 1) / kNaBlock;
        cudaStream_t s = nullptr; // legacy default stream; the call is synchronous
        auto reduce = [&]() -> double {
            k_na_finish<<<1, 32, 0, s>>>(blocks, part, scalar);
            double h = 0.0;
            check(cudaMemcpyAsync(&h, scalar, sizeof(double), cudaMemcpyDeviceToHost, s), "copy scalar");
            check(cudaStreamSynchronize(s), "synchronize");
            return h;
        };
        // validate the CSR structure on the device (flags in the scratch; no allocation)
        int* flag = reinterpret_cast<int*>(scalar + kNaFlagSlot);
        check(cudaMemsetAsync(flag, 0, sizeof(int), s), "clear flag");
        k_na_check_rows<<<(n + kNaBlock) / kNaBlock, kNaBlock, 0, s>>>(n, a->nnz, a->row_ptr, flag);
        int hflag = 0;
        check(cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, s), "copy flag");
        check(cudaStreamSynchronize(s), "synchronize");
        if (hflag == 0 && a->nnz > 0) {
            const int cblocks = std::min((a->nnz + kNaBlock - 1) / kNaBlock, 1184);
            k_na_check_cols<<<cblocks, kNaBlock, 0, s>>>(n, a->nnz, a->col, flag);
            check(cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, s), "copy flag");
            check(cudaStreamSynchronize(s), "synchronize");
        }
        if (hflag & 1)
            cfdb::fail(CFDB_ERR_BAD_ARG, "cfdb_solve_device_noalloc: row_ptr is not a valid CSR row offset array "
                                         "(row_ptr[0] = 0, non-decreasing, row_ptr[n] = nnz)");
        if (hflag & 2) cfdb::fail(CFDB_ERR_BAD_ARG, "cfdb_solve_device_noalloc: a column index is outside [0, n)");
        cfdb_stats st{0, 0.0, 0, 1, 0.0};
        // krylov_kernels.inc:44-95
        k_na_init<<<blocks, kNaBlock, 0, s>>>(m, b, x, dinv, r, part);
        double res = std::sqrt(reduce());
        if (res <= control->abs_tolerance) {
            st.converged = 1;
        } else {
            k_na_precond<<<blocks, kNaBlock, 0, s>>>(n, r, dinv, z, p, 1, part);
            double rz = reduce();
            for (st.iterations = 1; st.iterations <= control->max_iterations; ++st.iterations) {
                k_na_spmv<<<blocks, kNaBlock, 0, s>>>(m, p, q, part);
                const double pq = reduce();
                if (pq == 0.0) break;
                const double alpha = rz / pq;
                k_na_update<<<blocks, kNaBlock, 0, s>>>(n, alpha, p, q, x, r, part);
                res = std::sqrt(reduce());
                if (res <= control->abs_tolerance) {
                    st.converged = 1;
                    break;
                }
                k_na_precond<<<blocks, kNaBlock, 0, s>>>(n, r, dinv, z, p, 0, part);
                const double rz_new = reduce();
                const double beta = rz_new / rz;
                rz = rz_new;
                k_na_pupdate<<<blocks, kNaBlock, 0, s>>>(n, beta, z, p);
            }
            if (st.iterations > control->max_iterations) st.iterations = control->max_iterations;
        }
        st.residual = res;
        k_na_true<<<blocks, kNaBlock, 0, s>>>(m, b, x, part);
        st.true_residual = std::sqrt(reduce());
        check(cudaGetLastError(), "kernel launch");
        if (stats) *stats = st;
        return CFDB_OK;
    } catch (const cfdb::Error& e) {
        cfdb::set_thread_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        cfdb::set_thread_error(e.what());
        return CFDB_ERR_INTERNAL;
    }
}
