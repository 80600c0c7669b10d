// Residual norms of an LDU system on the device, for the persistent LDU solve
// (LduMatrix::solve_persistent, ldu_matrix.cpp:287-366, and LduMatrix::residual_norms,
// ldu_matrix.cpp:69-103).
//
// Row i of A x is summed over the CSR pattern of the LDU matrix (columns ascending), its
// coefficients read from [diag | upper | lower] through the pattern's value map. Each block
// sums a fixed set of rows and the host adds the block sums in block order, so the norms are
// reproducible; they differ from the reference's face-loop sums only in summation order.
#include "ldu_solve.hpp"

#include <vector>

namespace cfdb {

namespace {

constexpr int kNormThreads = 256;

__device__ __forceinline__ double ldu_value(int s, int n, int nf, const double* __restrict__ diag,
                                            const double* __restrict__ upper, const double* __restrict__ lower) {
    return s < n ? diag[s] : s < n + nf ? upper[s - n] : lower[s - n - nf];
}

template <int K> __device__ void block_sums(double (&v)[K], double* part) {
    __shared__ double sh[K][kNormThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < K; ++q) {
        double s = v[q];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) sh[q][w] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < K; ++q) {
            double s = 0.0;
            for (int u = 0; u < kNormThreads / 32; ++u) s += sh[q][u];
            part[K * blockIdx.x + q] = s;
        }
    }
}

__global__ void __launch_bounds__(kNormThreads) k_sum(int n, const double* __restrict__ x, double* part) {
    double v[1] = {0.0};
    for (int i = blockIdx.x * kNormThreads + threadIdx.x; i < n; i += gridDim.x * kNormThreads) v[0] += x[i];
    block_sums<1>(v, part);
}

// per block: sum |b - Ax|, sum |Ax - rs x_ref| + |b - rs x_ref| (rs = row sum), sum (b - Ax)^2
__global__ void __launch_bounds__(kNormThreads) k_norms(int n, int nf, const int* __restrict__ rp,
                                                        const int* __restrict__ ci, const int* __restrict__ src,
                                                        const double* __restrict__ diag, const double* __restrict__ upper,
                                                        const double* __restrict__ lower, const double* __restrict__ b,
                                                        const double* __restrict__ x, double x_ref, double* part) {
    double v[3] = {0.0, 0.0, 0.0};
    for (int i = blockIdx.x * kNormThreads + threadIdx.x; i < n; i += gridDim.x * kNormThreads) {
        double ax = 0.0, rs = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            const double a = ldu_value(src[k], n, nf, diag, upper, lower);
            ax += a * x[ci[k]];
            rs += a;
        }
        const double ax_ref = rs * x_ref;
        const double r = b[i] - ax;
        v[0] += fabs(r);
        v[1] += fabs(ax - ax_ref) + fabs(b[i] - ax_ref);
        v[2] += r * r;
    }
    block_sums<3>(v, part);
}

} // namespace

LduNorms ldu_residual_norms(const LduDevice& m, const double* diag, const double* upper, const double* lower,
                            const double* b, const double* x, double* part, cudaStream_t st) {
    LduNorms out;
    if (m.n == 0) return out;
    std::vector<double> h(3 * static_cast<size_t>(kLduNormBlocks));
    k_sum<<<kLduNormBlocks, kNormThreads, 0, st>>>(m.n, x, part);
    CFDB_CUDA(cudaGetLastError());
    CFDB_CUDA(cudaMemcpyAsync(h.data(), part, sizeof(double) * kLduNormBlocks, cudaMemcpyDeviceToHost, st));
    CFDB_CUDA(cudaStreamSynchronize(st));
    double sum = 0.0;
    for (int q = 0; q < kLduNormBlocks; ++q) sum += h[q];
    const double x_ref = sum / static_cast<double>(m.n);
    k_norms<<<kLduNormBlocks, kNormThreads, 0, st>>>(m.n, m.nf, m.rp, m.ci, m.src, diag, upper, lower, b, x, x_ref,
                                                     part);
    CFDB_CUDA(cudaGetLastError());
    CFDB_CUDA(cudaMemcpyAsync(h.data(), part, sizeof(double) * 3 * kLduNormBlocks, cudaMemcpyDeviceToHost, st));
    CFDB_CUDA(cudaStreamSynchronize(st));
    for (int q = 0; q < kLduNormBlocks; ++q) {
        out.res += h[3 * q];
        out.norm += h[3 * q + 1];
        out.r2 += h[3 * q + 2];
    }
    return out;
}

} // namespace cfdb
