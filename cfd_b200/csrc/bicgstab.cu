// Jacobi-preconditioned BiCGStab on an engine's level-0 operator (the momentum solver of the
// reference's accelerator layer, krylov_kernels.inc:97-169, selected by Method::BiCgStab).
//
// The iteration follows the reference's recurrences and stopping rules step by step (rho from
// r0.r, the pp / ph / v / s / sh / t updates, omega = (t.s) / (t.t) or 0, the early exit on
// |s| and the exits on rho == 0, omega == 0 and r0.v == 0; iterations capped at the maximum).
// Every update rounds each product and sum separately in the reference's operand order. Dot
// products are summed per block in a fixed order and the block sums are added on the host in
// block order, so results are reproducible; they differ from the reference's sequential sums
// only in summation order. The host drives the loop (four scalar read-backs per iteration):
// BiCGStab is not on the pressure path.
#include <cmath>
#include <vector>

#include "engine.hpp"

namespace cfdb {

namespace {

constexpr int kBcgBlocks = 592;  // 148 SMs x 4

int bcg_grid(int n) { return n > 0 ? (n + 255) / 256 : 1; }

// part[2 b], part[2 b + 1]: block b's share of x.y and u.w (u may be null).
static __global__ void __launch_bounds__(kBlock) k_bcg_dot2(int n, const double* __restrict__ x,
                                                            const double* __restrict__ y,
                                                            const double* __restrict__ u,
                                                            const double* __restrict__ w, double* part) {
    double a = 0.0, b = 0.0;
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
        a = __dadd_rn(a, __dmul_rn(x[i], y[i]));
        if (u != nullptr) b = __dadd_rn(b, __dmul_rn(u[i], w[i]));
    }
    block_sum2(a, b);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = a;
        part[2 * blockIdx.x + 1] = b;
    }
}

// r = b - ax; r0 = r; pp = v = 0
static __global__ void k_bcg_init(int n, const double* __restrict__ b, double* __restrict__ ax,
                                  double* __restrict__ r, double* __restrict__ r0, double* __restrict__ pp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const double ri = __dsub_rn(b[i], ax[i]);
        r[i] = ri;
        r0[i] = ri;
        pp[i] = 0.0;
        ax[i] = 0.0;  // ax is v
    }
}

// pp = r + beta (pp - omega v); ph = pp * dinv
static __global__ void k_bcg_p(int n, const double* __restrict__ r, const double* __restrict__ v,
                               const double* __restrict__ dinv, double beta, double omega,
                               double* __restrict__ pp, double* __restrict__ ph) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const double p = __dadd_rn(r[i], __dmul_rn(beta, __dsub_rn(pp[i], __dmul_rn(omega, v[i]))));
        pp[i] = p;
        ph[i] = __dmul_rn(p, dinv[i]);
    }
}

// s = r - alpha v; sh = s * dinv
static __global__ void k_bcg_s(int n, const double* __restrict__ r, const double* __restrict__ v,
                               const double* __restrict__ dinv, double alpha, double* __restrict__ s,
                               double* __restrict__ sh) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const double si = __dsub_rn(r[i], __dmul_rn(alpha, v[i]));
        s[i] = si;
        sh[i] = __dmul_rn(si, dinv[i]);
    }
}

// x += alpha ph + omega sh; r = s - omega t   (omega_on = 0: x += alpha ph only)
static __global__ void k_bcg_xr(int n, double alpha, double omega, int omega_on, const double* __restrict__ ph,
                                const double* __restrict__ sh, const double* __restrict__ s,
                                const double* __restrict__ t, double* __restrict__ x, double* __restrict__ r) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        if (omega_on) {
            x[i] = __dadd_rn(x[i], __dadd_rn(__dmul_rn(alpha, ph[i]), __dmul_rn(omega, sh[i])));
            r[i] = __dsub_rn(s[i], __dmul_rn(omega, t[i]));
        } else {
            x[i] = __dadd_rn(x[i], __dmul_rn(alpha, ph[i]));
        }
    }
}

} // namespace

SolveResult Engine::solve_bicgstab(const SolveRequest& rq) {
    CFDB_CUDA(cudaSetDevice(device_));
    if (n_sys_ != 1) fail(1, "solve_bicgstab: single-system plans only");
    const DevLevel& d = lv_[0];
    const int n = d.n_rows;
    if (bcg_ == nullptr) bcg_ = arena_.alloc<double>(6 * static_cast<size_t>(n) + 2 * kBcgBlocks);
    double* r0 = bcg_;
    double* v = r0 + n;
    double* s = v + n;
    double* t = s + n;
    double* ph = t + n;
    double* sh = ph + n;
    double* part = sh + n;
    double* r = r_;
    double* pp = p_;
    cudaStream_t st = stream_;
    const int g = bcg_grid(n);
    auto spmv = [&](const double* in, double* out) {
        k_vc_spmv<double, kVisitSell2><<<d.n_tiles, kBlock, 0, st>>>(d.a.s64, d.tiles, nullptr, in, out, nullptr,
                                                                     nullptr, 0);
        ++launches_;
    };
    std::vector<double> hp(2 * kBcgBlocks);
    auto dot2 = [&](const double* x, const double* y, const double* u, const double* w, double& a, double& b) {
        k_bcg_dot2<<<kBcgBlocks, kBlock, 0, st>>>(n, x, y, u, w, part);
        ++launches_;
        CFDB_CUDA(cudaMemcpyAsync(hp.data(), part, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, st));
        CFDB_CUDA(cudaStreamSynchronize(st));
        a = 0.0;
        b = 0.0;
        for (int k = 0; k < kBcgBlocks; ++k) {
            a += hp[2 * k];
            b += hp[2 * k + 1];
        }
    };
    SolveResult out;
    spmv(x_, v);
    k_bcg_init<<<g, 256, 0, st>>>(n, b_, v, r, r0, pp);
    ++launches_;
    double rr = 0.0, unused = 0.0;
    dot2(r, r, nullptr, nullptr, rr, unused);
    double res = std::sqrt(rr);
    if (res <= rq.tol) {
        out.residual = res;
        out.converged = true;
        out.true_residual = res;
        return out;
    }
    double rho = 1.0, alpha = 1.0, omega = 1.0;
    int it = 1;
    for (; it <= rq.max_it; ++it) {
        double rho_new = 0.0;
        dot2(r0, r, nullptr, nullptr, rho_new, unused);
        if (rho_new == 0.0 || omega == 0.0) break;
        const double beta = (rho_new / rho) * (alpha / omega);
        rho = rho_new;
        k_bcg_p<<<g, 256, 0, st>>>(n, r, v, dinv0_, beta, omega, pp, ph);
        ++launches_;
        spmv(ph, v);
        double r0v = 0.0;
        dot2(r0, v, nullptr, nullptr, r0v, unused);
        if (r0v == 0.0) break;
        alpha = rho / r0v;
        k_bcg_s<<<g, 256, 0, st>>>(n, r, v, dinv0_, alpha, s, sh);
        ++launches_;
        double ss = 0.0;
        dot2(s, s, nullptr, nullptr, ss, unused);
        const double s_norm = std::sqrt(ss);
        if (s_norm <= rq.tol) {
            k_bcg_xr<<<g, 256, 0, st>>>(n, alpha, 0.0, 0, ph, sh, s, t, x_, r);
            ++launches_;
            res = s_norm;
            out.converged = true;
            break;
        }
        spmv(sh, t);
        double tt = 0.0, ts = 0.0;
        dot2(t, t, t, s, tt, ts);
        omega = tt > 0.0 ? ts / tt : 0.0;
        k_bcg_xr<<<g, 256, 0, st>>>(n, alpha, omega, 1, ph, sh, s, t, x_, r);
        ++launches_;
        dot2(r, r, nullptr, nullptr, rr, unused);
        res = std::sqrt(rr);
        if (res <= rq.tol) {
            out.converged = true;
            break;
        }
    }
    CFDB_CUDA(cudaGetLastError());
    out.iterations = it > rq.max_it ? rq.max_it : it;
    out.residual = res;
    // |b - A x| of the returned solution, as the CG paths report it
    spmv(x_, v);
    k_bcg_init<<<g, 256, 0, st>>>(n, b_, v, t, s, ph);  // t = b - Ax (s, ph are scratch here)
    ++launches_;
    double tr = 0.0;
    dot2(t, t, nullptr, nullptr, tr, unused);
    out.true_residual = std::sqrt(tr);
    return out;
}

} // namespace cfdb
