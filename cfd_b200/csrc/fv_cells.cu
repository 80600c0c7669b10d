// cfd::gpu::DeviceFv on the device: cell gradients (Green-Gauss, weighted least squares,
// skewness-corrected Gauss) and the explicit internal-face corrections of the scalar and
// momentum equations (linear upwind, LUST blending, Barth-Jespersen / Venkatakrishnan limiter,
// non-orthogonal correction, transpose viscous term). Interface: fv_device.hpp:33-72 (DeviceFv,
// FvMeshView); per-cell arithmetic: fv_cell.inc:24-261; call sequence: fv_openmp.cpp:158-305.
//
// Every cell sums the same terms in the same order as the reference's per-cell loops (its
// faces in ascending order, the cell_faces CSR of the mesh view), and every product and sum is
// rounded separately (no FMA contraction: this file is compiled with --fmad=false), so the
// results are bit-identical to the reference's host build. Gradients: one thread per (cell,
// component), all components of a vector field in one launch (the reference makes one pass
// per component). Explicit corrections: a face's flux does not depend on which of its cells
// sums it, so it is computed once per internal face (coalesced over faces) and then summed
// per cell in face order. Limiter: one thread per cell. Mesh arrays stay resident on the
// device for the life of the object; vectors are xyz-interleaved, gradients of vectors are 9
// values per cell with g[3 i + j] = du_i / dx_j.
#include "../../include/cfdb.h"

#include <algorithm>
#include <string>
#include <vector>

#include "common.hpp"

namespace cfdb {
void set_thread_error(const std::string& msg);
} // namespace cfdb

using namespace cfdb;

namespace {

// Device copy of an FvMeshView (fv_device.hpp:15-31).
struct FvMesh {
    int nc = 0, nif = 0, nf = 0;
    const int* own = nullptr;     // n_faces
    const int* nei = nullptr;     // n_internal_faces
    const int* start = nullptr;   // n_cells + 1
    const int* faces = nullptr;   // start[n_cells], ascending per cell
    // per slot of faces: the cell across an internal face, c' >= 0 when this cell owns it and
    // -2 - c' when this cell is its neighbour; -1 for a boundary face (built at create, so the
    // gathers need no owner / neighbour loads)
    const int* across = nullptr;
    const double* w = nullptr;    // n_internal_faces
    const double* sf = nullptr;   // 3 n_faces
    const double* cf = nullptr;   // 3 n_faces
    const double* cc = nullptr;   // 3 n_cells
    const double* vol = nullptr;  // n_cells
    const double* kv = nullptr;   // 3 n_faces: non-orthogonal correction vectors
    const double* lsq_d = nullptr; // 3 n_faces: d / |d|^2
    const double* lsq = nullptr;  // 9 n_cells: column-major inverse of sum d d^T / |d|^2
};

} // namespace

struct cfdb_device_fv {
    int device = 0;
    cudaStream_t st = nullptr;
    DeviceArena mem;
    FvMesh m;
    // resident fields of the host-array entry points (fv_openmp.cpp:326-337)
    double* phi = nullptr;   // n_cells
    double* bv = nullptr;    // boundary faces
    double* sgrad = nullptr; // 3 n_cells
    double* vphi = nullptr;  // 3 n_cells
    double* vbv = nullptr;   // 3 boundary faces
    double* vgrad = nullptr; // 9 n_cells
    double* lim = nullptr;   // 3 n_cells
    double* flux = nullptr;  // internal faces
    double* coef = nullptr;  // internal faces
    double* src = nullptr;   // 3 n_cells
    double* tmp = nullptr;   // 9 n_cells: least-squares gradient of the corrected scheme
    double* eface = nullptr; // 3 internal faces: explicit face fluxes before the cell sums
    int maxf = 0;            // 4, 6 or 8: no cell has more faces (batched face sums); 0: any
    bool have_vector = false;
    StagedCopier copier;     // host-array entry points
    // FvGeometry's face factors for the scalar equation (cfdb_device_fv_set_face_geometry)
    double* dc = nullptr;    // n_faces: delta coefficients
    double* un = nullptr;    // 3 n_faces: unit normals
    double* area = nullptr;  // n_faces: face areas
    ~cfdb_device_fv() {
        if (st != nullptr) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
    }
};

namespace {

constexpr int kThreads = 256;

int grid(int n) { return std::max(1, (n + kThreads - 1) / kThreads); }

// Gradient of component i of a field with NC values per cell / boundary face: Green-Gauss
// with linear face interpolation, or weighted least squares (fv_cell.inc:24-74). One thread
// per (cell, component), t = NC c + i, so a vector field's three components are three
// independent threads with the scalar kernel's register footprint; the components share
// their face-index and face-vector loads in L1. out[3 (NC c + i) + j] = d phi_i / dx_j.
template <int NC, bool LSQ>
__global__ void __launch_bounds__(kThreads, LSQ ? 8 : 6) k_cell_gradient(FvMesh m, const double* __restrict__ phi,
                                                            const double* __restrict__ bv,
                                                            double* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m.nc * NC) return;
    const int c = NC == 1 ? t : t / NC;
    const int i = NC == 1 ? 0 : t - c * NC;
    double g0 = 0.0, g1 = 0.0, g2 = 0.0;
    const double pc = phi[t];
    const int k1 = m.start[c + 1];
    for (int k = m.start[c]; k < k1; ++k) {
        const int f = m.faces[k];
        const int x = m.across[k];
        if (x != -1) {
            // phi_P and phi_N of the face: this cell's value and the one across
            const bool mine = x >= 0;
            const double pa = phi[(mine ? x : -2 - x) * NC + i];
            if (LSQ) {
                const double dv = mine ? pa - pc : pc - pa; // phi_N - phi_P
                g0 += m.lsq_d[3 * f] * dv;
                g1 += m.lsq_d[3 * f + 1] * dv;
                g2 += m.lsq_d[3 * f + 2] * dv;
            } else {
                const double wf = m.w[f];
                const double pf = mine ? wf * pc + (1.0 - wf) * pa : wf * pa + (1.0 - wf) * pc;
                if (mine) {
                    g0 += m.sf[3 * f] * pf;
                    g1 += m.sf[3 * f + 1] * pf;
                    g2 += m.sf[3 * f + 2] * pf;
                } else {
                    g0 -= m.sf[3 * f] * pf;
                    g1 -= m.sf[3 * f + 1] * pf;
                    g2 -= m.sf[3 * f + 2] * pf;
                }
            }
        } else {
            const double b = bv[(f - m.nif) * NC + i];
            if (LSQ) {
                const double dv = b - pc;
                g0 += m.lsq_d[3 * f] * dv;
                g1 += m.lsq_d[3 * f + 1] * dv;
                g2 += m.lsq_d[3 * f + 2] * dv;
            } else {
                g0 += m.sf[3 * f] * b;
                g1 += m.sf[3 * f + 1] * b;
                g2 += m.sf[3 * f + 2] * b;
            }
        }
    }
    double* o = out + 3 * static_cast<size_t>(t);
    if (LSQ) {
        const double* a = m.lsq + 9 * static_cast<size_t>(c); // column-major
        o[0] = a[0] * g0 + a[3] * g1 + a[6] * g2;
        o[1] = a[1] * g0 + a[4] * g1 + a[7] * g2;
        o[2] = a[2] * g0 + a[5] * g1 + a[8] * g2;
    } else {
        const double v = m.vol[c];
        o[0] = g0 / v;
        o[1] = g1 / v;
        o[2] = g2 / v;
    }
}

// Skewness-corrected Green-Gauss (fv_cell.inc:76-121) of component i, one thread per
// (cell, component): face values w phi_P + (1 - w) phi_N + (w g_P + (1 - w) g_N) . (x_f - x_ip)
// with the least-squares gradient g (layout of k_cell_gradient's output).
template <int NC>
__global__ void __launch_bounds__(kThreads) k_cell_gradient_corrected(FvMesh m, const double* __restrict__ phi,
                                                                      const double* __restrict__ bv,
                                                                      const double* __restrict__ g,
                                                                      double* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m.nc * NC) return;
    const int c = NC == 1 ? t : t / NC;
    const int i = NC == 1 ? 0 : t - c * NC;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    const int k1 = m.start[c + 1];
    for (int k = m.start[c]; k < k1; ++k) {
        const int f = m.faces[k];
        const int x = m.across[k];
        if (x != -1) {
            const int p = x >= 0 ? c : -2 - x, n = x >= 0 ? x : c;
            const double wf = m.w[f];
            double pf = wf * phi[p * NC + i] + (1.0 - wf) * phi[n * NC + i];
            const double* gp = g + 3 * (static_cast<size_t>(p) * NC + i);
            const double* gn = g + 3 * (static_cast<size_t>(n) * NC + i);
            double dot = 0.0;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const double xip = wf * m.cc[3 * p + j] + (1.0 - wf) * m.cc[3 * n + j];
                const double gf = wf * gp[j] + (1.0 - wf) * gn[j];
                dot = j == 0 ? gf * (m.cf[3 * f] - xip) : dot + gf * (m.cf[3 * f + j] - xip);
            }
            pf += dot;
            if (p == c) {
                a0 += m.sf[3 * f] * pf;
                a1 += m.sf[3 * f + 1] * pf;
                a2 += m.sf[3 * f + 2] * pf;
            } else {
                a0 -= m.sf[3 * f] * pf;
                a1 -= m.sf[3 * f + 1] * pf;
                a2 -= m.sf[3 * f + 2] * pf;
            }
        } else {
            const double b = bv[(f - m.nif) * NC + i];
            a0 += m.sf[3 * f] * b;
            a1 += m.sf[3 * f + 1] * b;
            a2 += m.sf[3 * f + 2] * b;
        }
    }
    double* o = out + 3 * static_cast<size_t>(t);
    const double v = m.vol[c];
    o[0] = a0 / v;
    o[1] = a1 / v;
    o[2] = a2 / v;
}

// Barth-Jespersen / Venkatakrishnan limiter per component of the vector field u with boundary
// values ub and gradient g (9 per cell) (fv_cell.inc:123-163), one thread per cell.
__global__ void __launch_bounds__(kThreads) k_cell_limiter(FvMesh m, const double* __restrict__ u,
                                                           const double* __restrict__ ub,
                                                           const double* __restrict__ g, int venkat,
                                                           double e0, double e1, double e2,
                                                           double* __restrict__ lim) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const double eps2[3] = {e0, e1, e2};
    double uc[3], lo[3], hi[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) uc[i] = lo[i] = hi[i] = u[3 * c + i];
    const int k0 = m.start[c], k1 = m.start[c + 1];
    for (int k = k0; k < k1; ++k) {
        const int x = m.across[k];
        const double* v = x != -1 ? u + 3 * (x >= 0 ? x : -2 - x) : ub + 3 * (m.faces[k] - m.nif);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double vi = v[i];
            lo[i] = vi < lo[i] ? vi : lo[i];
            hi[i] = vi > hi[i] ? vi : hi[i];
        }
    }
    double l[3] = {1.0, 1.0, 1.0};
    const double* gc = g + 9 * static_cast<size_t>(c);
    double gv[9];
#pragma unroll
    for (int j = 0; j < 9; ++j) gv[j] = gc[j];
    const double x0 = m.cc[3 * c], x1 = m.cc[3 * c + 1], x2 = m.cc[3 * c + 2];
    for (int k = k0; k < k1; ++k) {
        const int f = m.faces[k];
        const double r0 = m.cf[3 * f] - x0;
        const double r1 = m.cf[3 * f + 1] - x1;
        const double r2 = m.cf[3 * f + 2] - x2;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double d = gv[3 * i] * r0 + gv[3 * i + 1] * r1 + gv[3 * i + 2] * r2;
            if (d < 1e-300 && d > -1e-300) continue;
            const double bound = d > 0.0 ? hi[i] - uc[i] : lo[i] - uc[i];
            double q;
            if (venkat) {
                q = (bound * bound + eps2[i] + 2.0 * d * bound) / (bound * bound + 2.0 * d * d + d * bound + eps2[i]);
            } else {
                const double ratio = bound / d;
                q = ratio > 0.0 ? ratio : 0.0;
            }
            l[i] = q < l[i] ? q : l[i];
        }
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) lim[3 * c + i] = l[i];
}

// Explicit internal-face flux of a scalar equation with the cell gradient g (3 per cell)
// (fv_cell.inc:165-196). The flux e_f depends on the face alone, so it is computed once per
// internal face (one thread per face); k_cell_face_sums then adds +-e_f over each cell's faces
// in the reference's order. The two cells of a face receive the same rounded e_f as in the
// reference, which computes it once from each side.
__global__ void __launch_bounds__(kThreads) k_scalar_face_terms(FvMesh m, const double* __restrict__ g,
                                                                const double* __restrict__ flux,
                                                                const double* __restrict__ gamma,
                                                                int linear_upwind, double* __restrict__ e_out) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nif) return;
    const int p = m.own[f], n = m.nei[f];
    const double fl = flux[f];
    double e = 0.0;
    if (linear_upwind) {
        const int up = fl >= 0.0 ? p : n;
        const double r0 = m.cf[3 * f] - m.cc[3 * up];
        const double r1 = m.cf[3 * f + 1] - m.cc[3 * up + 1];
        const double r2 = m.cf[3 * f + 2] - m.cc[3 * up + 2];
        e -= fl * (g[3 * up] * r0 + g[3 * up + 1] * r1 + g[3 * up + 2] * r2);
    }
    const double wf = m.w[f];
    const double gf0 = wf * g[3 * p] + (1.0 - wf) * g[3 * n];
    const double gf1 = wf * g[3 * p + 1] + (1.0 - wf) * g[3 * n + 1];
    const double gf2 = wf * g[3 * p + 2] + (1.0 - wf) * g[3 * n + 2];
    e += gamma[f] * (m.kv[3 * f] * gf0 + m.kv[3 * f + 1] * gf1 + m.kv[3 * f + 2] * gf2);
    e_out[f] = e;
}

// Explicit internal-face flux of the momentum equation (fv_cell.inc:198-259), once per face.
__global__ void __launch_bounds__(kThreads) k_momentum_face_terms(
    FvMesh m, const double* __restrict__ g, const double* __restrict__ lim, int limited,
    const double* __restrict__ flux, const double* __restrict__ nu_face, int linear_upwind, double central,
    const double* __restrict__ u, int transpose_term, double* __restrict__ e_out) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nif) return;
    const int p = m.own[f], n = m.nei[f];
    const double fl = flux[f];
    const double wf = m.w[f];
    double e[3] = {0.0, 0.0, 0.0};
    if (linear_upwind) {
        const int up = fl >= 0.0 ? p : n;
        const double r0 = m.cf[3 * f] - m.cc[3 * up];
        const double r1 = m.cf[3 * f + 1] - m.cc[3 * up + 1];
        const double r2 = m.cf[3 * f + 2] - m.cc[3 * up + 2];
        const double* gu = g + 9 * static_cast<size_t>(up);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            double d = gu[3 * i] * r0 + gu[3 * i + 1] * r1 + gu[3 * i + 2] * r2;
            if (central > 0.0) {
                const double uf = wf * u[3 * p + i] + (1.0 - wf) * u[3 * n + i];
                d = (1.0 - central) * d + central * (uf - u[3 * up + i]);
            }
            if (limited) d = lim[3 * up + i] * d;
            e[i] -= fl * d;
        }
    }
    const double* gp = g + 9 * static_cast<size_t>(p);
    const double* gn = g + 9 * static_cast<size_t>(n);
    double gf[9];
#pragma unroll
    for (int j = 0; j < 9; ++j) gf[j] = wf * gp[j] + (1.0 - wf) * gn[j];
    const double nu = nu_face[f];
    const double k0 = m.kv[3 * f], k1 = m.kv[3 * f + 1], k2 = m.kv[3 * f + 2];
#pragma unroll
    for (int i = 0; i < 3; ++i) e[i] += nu * (gf[3 * i] * k0 + gf[3 * i + 1] * k1 + gf[3 * i + 2] * k2);
    if (transpose_term) {
        const double a0 = m.sf[3 * f], a1 = m.sf[3 * f + 1], a2 = m.sf[3 * f + 2];
#pragma unroll
        for (int i = 0; i < 3; ++i) e[i] += nu * (gf[i] * a0 + gf[i + 3] * a1 + gf[i + 6] * a2);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) e_out[3 * static_cast<size_t>(f) + i] = e[i];
}

// source[c] += sum over the cell's faces, in ascending order up to its first boundary face
// (fv_cell.inc:172-174, 210-212), of +e_f (owner) or -e_f (neighbour); NC values per face.
// MAXF > 0: every cell has at most MAXF faces; the indices, owners and face terms of all its
// faces are loaded before the (unchanged, ordered) sums.
template <int NC, int MAXF>
__global__ void __launch_bounds__(kThreads) k_cell_face_sums(FvMesh m, const double* __restrict__ e,
                                                             double* __restrict__ source) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    double s[NC];
#pragma unroll
    for (int i = 0; i < NC; ++i) s[i] = 0.0;
    const int k0 = m.start[c], k1 = m.start[c + 1];
    if (MAXF > 0) {
        constexpr int F = MAXF > 0 ? MAXF : 1;
        int f[F];
        bool mine[F];
        double ev[F][NC];
        bool live = true;
        int x[F];
#pragma unroll
        for (int j = 0; j < F; ++j) x[j] = k0 + j < k1 ? m.across[k0 + j] : -1; // past the end: a stop
#pragma unroll
        for (int j = 0; j < F; ++j) {
            live = live && x[j] != -1;
            f[j] = live ? m.faces[k0 + j] : -1;
        }
#pragma unroll
        for (int j = 0; j < F; ++j) {
            mine[j] = x[j] >= 0;
#pragma unroll
            for (int i = 0; i < NC; ++i) ev[j][i] = f[j] >= 0 ? e[static_cast<size_t>(f[j]) * NC + i] : 0.0;
        }
#pragma unroll
        for (int j = 0; j < F; ++j) {
            if (f[j] < 0) break;
#pragma unroll
            for (int i = 0; i < NC; ++i) s[i] = mine[j] ? s[i] + ev[j][i] : s[i] - ev[j][i];
        }
    } else {
        for (int k = k0; k < k1; ++k) {
            const int x = m.across[k];
            if (x == -1) break; // the first boundary face
            const int f = m.faces[k];
            const bool mine = x >= 0;
#pragma unroll
            for (int i = 0; i < NC; ++i) {
                const double ev = e[static_cast<size_t>(f) * NC + i];
                s[i] = mine ? s[i] + ev : s[i] - ev;
            }
        }
    }
#pragma unroll
    for (int i = 0; i < NC; ++i) source[static_cast<size_t>(c) * NC + i] += s[i];
}

// ---- the scalar equation of solve_scalar (scalar_transport.cpp:50-176, GPU path) ----------

// std::min / std::max of the reference: (b < a) ? b : a and (a < b) ? b : a (signed zeros kept)
__device__ __forceinline__ double ref_min(double a, double b) { return b < a ? b : a; }
__device__ __forceinline__ double ref_max(double a, double b) { return a < b ? b : a; }

// |(x_f - x_P) . n_f| (scalar_transport.cpp:27-28, 133, 140)
__device__ __forceinline__ double normal_distance(const FvMesh& m, const double* __restrict__ un, int f, int p) {
    const double d0 = m.cf[3 * f] - m.cc[3 * p];
    const double d1 = m.cf[3 * f + 1] - m.cc[3 * p + 1];
    const double d2 = m.cf[3 * f + 2] - m.cc[3 * p + 2];
    return fabs(d0 * un[3 * f] + d1 * un[3 * f + 1] + d2 * un[3 * f + 2]);
}

// boundary_values (scalar_transport.cpp:10-40), one thread per boundary face
__global__ void __launch_bounds__(kThreads) k_scalar_boundary_values(FvMesh m, const double* __restrict__ un,
                                                                     const int* __restrict__ kind,
                                                                     const double* __restrict__ value,
                                                                     const double* __restrict__ coef,
                                                                     const double* __restrict__ field,
                                                                     double* __restrict__ bv) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m.nf - m.nif) return;
    const int f = m.nif + b;
    const int p = m.own[f];
    switch (kind[b]) {
    case CFDB_SCALAR_FIXED_VALUE: bv[b] = value[b]; break;
    case CFDB_SCALAR_FIXED_GRADIENT: bv[b] = field[p] + value[b] * normal_distance(m, un, f, p); break;
    case CFDB_SCALAR_MIXED: {
        const double rd = coef[b] * normal_distance(m, un, f, p);
        bv[b] = (field[p] + rd * value[b]) / (1.0 + rd);
        break;
    }
    default: bv[b] = field[p]; break; // zero gradient
    }
}

// Internal-face coefficients of assemble_convection_diffusion with convection = 1
// (krylov.hpp:105-116) and the fixed-cell rule (scalar_transport.cpp:162-170).
__global__ void __launch_bounds__(kThreads) k_scalar_face_coeffs(FvMesh m, const double* __restrict__ flux,
                                                                 const double* __restrict__ gamma,
                                                                 const double* __restrict__ dc,
                                                                 const unsigned char* __restrict__ fixed,
                                                                 double* __restrict__ upper, double* __restrict__ lower) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nif) return;
    const double fl = flux[f];
    const double g = gamma[f] * dc[f];
    const double pos = fl > 0.0 ? 1.0 * fl : 0.0;
    const double neg = fl < 0.0 ? 1.0 * fl : 0.0;
    upper[f] = fixed != nullptr && fixed[m.own[f]] != 0 ? 0.0 : neg - g;
    lower[f] = fixed != nullptr && fixed[m.nei[f]] != 0 ? 0.0 : -pos - g;
}

struct ScalarCellTerms {
    const double* su;
    const double* sp;
    const double* old_value;
    const double* capacity;
    const unsigned char* fixed;
    const double* fixed_value;
    double relaxation;
    double dt;
};

// Per cell, in the reference's order: the internal faces' diagonal and divergence
// (assemble_convection_diffusion), the boundary faces (scalar_transport.cpp:127-148), then the
// cell terms (:150-161) and fixed cells (:171-177). source holds the explicit face corrections
// on entry. One thread per cell over its faces in ascending order (internal before boundary).
__global__ void __launch_bounds__(kThreads) k_scalar_cells(FvMesh m, const double* __restrict__ flux,
                                                           const double* __restrict__ gamma,
                                                           const double* __restrict__ dc,
                                                           const double* __restrict__ un,
                                                           const double* __restrict__ area,
                                                           const int* __restrict__ kind,
                                                           const double* __restrict__ value,
                                                           const double* __restrict__ coef, ScalarCellTerms t,
                                                           double* __restrict__ field, double* __restrict__ diag,
                                                           double* __restrict__ source) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    double d = 0.0, div = 0.0, src = source[c];
    const int k1 = m.start[c + 1];
    for (int k = m.start[c]; k < k1; ++k) {
        const int f = m.faces[k];
        const double fl = flux[f];
        const int x = m.across[k];
        if (x != -1) {
            const double g = gamma[f] * dc[f];
            if (x >= 0) { // this cell owns the face
                const double pos = fl > 0.0 ? 1.0 * fl : 0.0;
                d = d + (pos + g);
                div = div + fl;
            } else {
                const double neg = fl < 0.0 ? 1.0 * fl : 0.0;
                d = d + (-neg + g);
                div = div - fl;
            }
            continue;
        }
        const int b = f - m.nif;
        div += fl;
        const int kb = kind[b];
        if (kb == CFDB_SCALAR_FIXED_VALUE) {
            const double diff = gamma[f] * dc[f];
            d += diff + ref_max(fl, 0.0);
            src += (diff - ref_min(fl, 0.0)) * value[b];
        } else if (kb == CFDB_SCALAR_MIXED) {
            const double dn = normal_distance(m, un, f, c);
            const double rd = coef[b] * dn;
            const double cm = gamma[f] * dc[f] * rd / (1.0 + rd);
            d += cm + fl;
            src += cm * value[b];
        } else {
            d += fl;
            if (kb == CFDB_SCALAR_FIXED_GRADIENT) {
                const double dn = normal_distance(m, un, f, c);
                src += gamma[f] * value[b] * area[f] - fl * value[b] * dn;
            }
        }
    }
    const double vol = m.vol[c];
    const double phi = field[c];
    d -= div; // bounded convection form
    d -= ref_min(t.sp[c], 0.0) * vol;
    src += t.su[c] * vol + ref_max(t.sp[c], 0.0) * phi * vol;
    if (t.dt > 0.0) {
        const double ddt = vol / t.dt * (t.capacity != nullptr ? t.capacity[c] : 1.0);
        d += ddt;
        src += ddt * (t.old_value != nullptr ? t.old_value[c] : phi);
    }
    if (t.relaxation < 1.0) {
        const double d1 = d / t.relaxation;
        src += (d1 - d) * phi;
        d = d1;
    }
    if (t.fixed != nullptr && t.fixed[c] != 0) {
        d = 1.0;
        src = t.fixed_value[c];
        field[c] = t.fixed_value[c];
    }
    diag[c] = d;
    source[c] = src;
}

template <class F> int guarded(F&& f) {
    try {
        f();
        return CFDB_OK;
    } catch (const Error& e) {
        set_thread_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        set_thread_error(e.what());
        return CFDB_ERR_INTERNAL;
    }
}

void check_scheme(int scheme) {
    if (scheme < CFDB_GRAD_GAUSS || scheme > CFDB_GRAD_GAUSS_CORRECTED)
        fail(CFDB_ERR_BAD_ARG, "DeviceFv: unknown gradient scheme " + std::to_string(scheme));
}

// Launches K<..., MAXF> with the mesh's face-count class (0: any number of faces).
#define CFDB_FV_BY_MAXF(fv, LAUNCH)          \
    switch ((fv)->maxf) {                   \
    case 4: LAUNCH(4); break;               \
    case 6: LAUNCH(6); break;               \
    case 8: LAUNCH(8); break;               \
    default: LAUNCH(0); break;              \
    }

int grid_of(long long threads) { return static_cast<int>(std::max(1LL, (threads + kThreads - 1) / kThreads)); }

// gradient_loop of fv_openmp.cpp:250-297: all NC components in one launch
template <int NC>
void launch_gradient(cfdb_device_fv* fv, const double* phi, const double* bv, int scheme, double* out) {
    const FvMesh& m = fv->m;
    if (bv == nullptr) bv = fv->vbv; // no boundary faces: never read, but a valid address
    const int blocks = grid_of(static_cast<long long>(m.nc) * NC);
    if (scheme == CFDB_GRAD_GAUSS_CORRECTED) {
        k_cell_gradient<NC, true><<<blocks, kThreads, 0, fv->st>>>(m, phi, bv, fv->tmp);
        k_cell_gradient_corrected<NC><<<blocks, kThreads, 0, fv->st>>>(m, phi, bv, fv->tmp, out);
    } else if (scheme == CFDB_GRAD_LEAST_SQUARES) {
        k_cell_gradient<NC, true><<<blocks, kThreads, 0, fv->st>>>(m, phi, bv, out);
    } else {
        k_cell_gradient<NC, false><<<blocks, kThreads, 0, fv->st>>>(m, phi, bv, out);
    }
    CFDB_CUDA(cudaGetLastError());
}

template <int NC, int MAXF> void launch_face_sums(const cfdb_device_fv* fv, double* source) {
    k_cell_face_sums<NC, MAXF><<<grid(fv->m.nc), kThreads, 0, fv->st>>>(fv->m, fv->eface, source);
}

void launch_scalar_corrections(cfdb_device_fv* fv, const double* phi, const double* bv, int scheme,
                               const double* flux, const double* gamma, int linear_upwind, double* source) {
    launch_gradient<1>(fv, phi, bv, scheme, fv->sgrad);
    if (fv->m.nif > 0)
        k_scalar_face_terms<<<grid(fv->m.nif), kThreads, 0, fv->st>>>(fv->m, fv->sgrad, flux, gamma,
                                                                      linear_upwind != 0 ? 1 : 0, fv->eface);
#define L(F) launch_face_sums<1, F>(fv, source)
    CFDB_FV_BY_MAXF(fv, L)
#undef L
    CFDB_CUDA(cudaGetLastError());
}

void launch_momentum_corrections(cfdb_device_fv* fv, const double* u, const double* ub, const double* g,
                                 const double* flux, const double* nu_face, int linear_upwind, int limited,
                                 int venkat, const double* eps2, double central, int transpose_term,
                                 double* source) {
    // the limiter is used only with linear upwind (fv_openmp.cpp:216)
    const int use_lim = limited != 0 && linear_upwind != 0 ? 1 : 0;
    const double e0 = venkat ? eps2[0] : 0.0, e1 = venkat ? eps2[1] : 0.0, e2 = venkat ? eps2[2] : 0.0;
    const int vk = venkat != 0 ? 1 : 0;
    if (ub == nullptr) ub = fv->vbv; // no boundary faces: never read, but a valid address
    if (use_lim)
        k_cell_limiter<<<grid(fv->m.nc), kThreads, 0, fv->st>>>(fv->m, u, ub, g, vk, e0, e1, e2, fv->lim);
    if (fv->m.nif > 0)
        k_momentum_face_terms<<<grid(fv->m.nif), kThreads, 0, fv->st>>>(
            fv->m, g, fv->lim, use_lim, flux, nu_face, linear_upwind != 0 ? 1 : 0, central, u,
            transpose_term != 0 ? 1 : 0, fv->eface);
#define L(F) launch_face_sums<3, F>(fv, source)
    CFDB_FV_BY_MAXF(fv, L)
#undef L
    CFDB_CUDA(cudaGetLastError());
}

void h2d(cfdb_device_fv* fv, double* dst, const double* src, size_t n) {
    fv->copier.to_device(dst, src, n * sizeof(double), fv->st);
}

void d2h(cfdb_device_fv* fv, double* dst, const double* src, size_t n) {
    fv->copier.to_host(dst, src, n * sizeof(double), fv->st);
}

size_t ncells(const cfdb_device_fv* fv) { return static_cast<size_t>(fv->m.nc); }
size_t nbound(const cfdb_device_fv* fv) { return static_cast<size_t>(fv->m.nf - fv->m.nif); }
size_t ninternal(const cfdb_device_fv* fv) { return static_cast<size_t>(fv->m.nif); }

void need(bool ok, const char* what) {
    if (!ok) fail(CFDB_ERR_BAD_ARG, std::string("DeviceFv: null argument among ") + what);
}

} // namespace

extern "C" {

int cfdb_device_fv_create(const cfdb_fv_mesh_view* v, cfdb_device_fv** out) {
    return guarded([&] {
        if (v == nullptr || out == nullptr) fail(CFDB_ERR_BAD_ARG, "DeviceFv: null argument");
        *out = nullptr;
        const int nc = v->n_cells, nif = v->n_internal_faces, nf = v->n_faces;
        // FvHostMesh (fv_device.cpp:22-50): sizes, then every array present
        if (nc <= 0 || nif < 0 || nf < nif || v->cell_offsets == nullptr)
            fail(CFDB_ERR_BAD_ARG, "DeviceFv: invalid mesh sizes");
        const size_t c = static_cast<size_t>(nc), f = static_cast<size_t>(nf), fi = static_cast<size_t>(nif);
        const int n_slots = v->cell_offsets[nc];
        auto missing = [&](const void* p, size_t n, const char* what) {
            if (n > 0 && p == nullptr) fail(CFDB_ERR_BAD_ARG, std::string("DeviceFv: missing mesh array ") + what);
        };
        missing(v->owner, f, "owner");
        missing(v->neighbour, fi, "neighbour");
        missing(v->cell_faces, n_slots > 0 ? static_cast<size_t>(n_slots) : 0, "cell_faces");
        missing(v->weight, fi, "weight");
        missing(v->sf, f, "sf");
        missing(v->face_centre, f, "face_centre");
        missing(v->cell_centre, c, "cell_centre");
        missing(v->volume, c, "volume");
        missing(v->correction, f, "correction");
        missing(v->lsq_d, f, "lsq_d");
        missing(v->lsq_inverse, c, "lsq_inverse");
        // every index the kernels follow stays inside its array
        if (v->cell_offsets[0] != 0) fail(CFDB_ERR_BAD_ARG, "DeviceFv: cell_offsets[0] != 0");
        for (int i = 0; i < nc; ++i)
            if (v->cell_offsets[i + 1] < v->cell_offsets[i])
                fail(CFDB_ERR_BAD_ARG, "DeviceFv: cell_offsets decrease at cell " + std::to_string(i));
        for (int k = 0; k < n_slots; ++k)
            if (v->cell_faces[k] < 0 || v->cell_faces[k] >= nf)
                fail(CFDB_ERR_BAD_ARG, "DeviceFv: cell_faces[" + std::to_string(k) + "] out of range");
        for (int i = 0; i < nf; ++i)
            if (v->owner[i] < 0 || v->owner[i] >= nc || (i < nif && (v->neighbour[i] < 0 || v->neighbour[i] >= nc)))
                fail(CFDB_ERR_BAD_ARG, "DeviceFv: face " + std::to_string(i) + " addresses a cell out of range");
        require_cuda_device();
        auto* fv = new cfdb_device_fv;
        try {
            CFDB_CUDA(cudaGetDevice(&fv->device));
            CFDB_CUDA(cudaStreamCreateWithFlags(&fv->st, cudaStreamNonBlocking));
            auto up = [&](const auto* p, size_t n) {
                using T = std::remove_const_t<std::remove_pointer_t<decltype(p)>>;
                std::vector<T> h(p, p + n);
                return static_cast<const T*>(fv->mem.upload(h, fv->st));
            };
            FvMesh& m = fv->m;
            m.nc = nc;
            m.nif = nif;
            m.nf = nf;
            m.own = up(v->owner, f);
            m.nei = up(v->neighbour, fi);
            m.start = up(v->cell_offsets, c + 1);
            m.faces = up(v->cell_faces, static_cast<size_t>(n_slots));
            {
                std::vector<int> across(static_cast<size_t>(n_slots));
                for (int cc = 0; cc < nc; ++cc)
                    for (int k = v->cell_offsets[cc]; k < v->cell_offsets[cc + 1]; ++k) {
                        const int f = v->cell_faces[k];
                        across[k] = f >= nif ? -1 : v->owner[f] == cc ? v->neighbour[f] : -2 - v->owner[f];
                    }
                m.across = fv->mem.upload(across, fv->st);
            }
            m.w = up(v->weight, fi);
            m.sf = up(v->sf, 3 * f);
            m.cf = up(v->face_centre, 3 * f);
            m.cc = up(v->cell_centre, 3 * c);
            m.vol = up(v->volume, c);
            m.kv = up(v->correction, 3 * f);
            m.lsq_d = up(v->lsq_d, 3 * f);
            m.lsq = up(v->lsq_inverse, 9 * c);
            const size_t nb = f - fi;
            fv->phi = fv->mem.alloc<double>(c);
            fv->bv = fv->mem.alloc<double>(nb);
            fv->sgrad = fv->mem.alloc<double>(3 * c);
            fv->vphi = fv->mem.alloc<double>(3 * c);
            fv->vbv = fv->mem.alloc<double>(3 * nb);
            fv->vgrad = fv->mem.alloc<double>(9 * c);
            fv->lim = fv->mem.alloc<double>(3 * c);
            fv->flux = fv->mem.alloc<double>(fi);
            fv->coef = fv->mem.alloc<double>(fi);
            fv->src = fv->mem.alloc<double>(3 * c);
            fv->tmp = fv->mem.alloc<double>(9 * c);
            fv->eface = fv->mem.alloc<double>(3 * fi);
            int deg = 0;
            for (int i = 0; i < nc; ++i) deg = std::max(deg, v->cell_offsets[i + 1] - v->cell_offsets[i]);
            fv->maxf = deg <= 4 ? 4 : deg <= 6 ? 6 : deg <= 8 ? 8 : 0;
            CFDB_CUDA(cudaStreamSynchronize(fv->st));
        } catch (...) {
            delete fv;
            throw;
        }
        *out = fv;
    });
}

int cfdb_device_fv_destroy(cfdb_device_fv* fv) {
    if (fv != nullptr) {
        cudaSetDevice(fv->device);
        delete fv;
    }
    return CFDB_OK;
}

int cfdb_device_fv_on_device(const cfdb_device_fv* fv) { return fv != nullptr ? 1 : 0; }

int cfdb_device_fv_device_bytes(const cfdb_device_fv* fv, size_t* bytes) {
    if (fv == nullptr || bytes == nullptr) return CFDB_ERR_BAD_ARG;
    *bytes = fv->mem.bytes();
    return CFDB_OK;
}

int cfdb_device_fv_stream(const cfdb_device_fv* fv, void** stream) {
    if (fv == nullptr || stream == nullptr) return CFDB_ERR_BAD_ARG;
    *stream = fv->st;
    return CFDB_OK;
}

int cfdb_device_fv_gradient(cfdb_device_fv* fv, const double* phi, const double* bv, int scheme, double* grad) {
    return guarded([&] {
        need(fv != nullptr && phi != nullptr && grad != nullptr && (nbound(fv) == 0 || bv != nullptr), "phi, bv, grad");
        check_scheme(scheme);
        CFDB_CUDA(cudaSetDevice(fv->device));
        h2d(fv, fv->phi, phi, ncells(fv));
        h2d(fv, fv->bv, bv, nbound(fv));
        launch_gradient<1>(fv, fv->phi, fv->bv, scheme, fv->sgrad);
        d2h(fv, grad, fv->sgrad, 3 * ncells(fv));
        CFDB_CUDA(cudaStreamSynchronize(fv->st));
    });
}

int cfdb_device_fv_vector_gradient(cfdb_device_fv* fv, const double* u, const double* ub, int scheme, double* grad) {
    return guarded([&] {
        need(fv != nullptr && u != nullptr && grad != nullptr && (nbound(fv) == 0 || ub != nullptr), "u, ub, grad");
        check_scheme(scheme);
        CFDB_CUDA(cudaSetDevice(fv->device));
        fv->have_vector = false;
        h2d(fv, fv->vphi, u, 3 * ncells(fv));
        h2d(fv, fv->vbv, ub, 3 * nbound(fv));
        launch_gradient<3>(fv, fv->vphi, fv->vbv, scheme, fv->vgrad);
        d2h(fv, grad, fv->vgrad, 9 * ncells(fv));
        CFDB_CUDA(cudaStreamSynchronize(fv->st));
        fv->have_vector = true;
    });
}

int cfdb_device_fv_scalar_corrections(cfdb_device_fv* fv, const double* phi, const double* bv, int scheme,
                                      const double* flux, const double* gamma, int linear_upwind, double* source) {
    return guarded([&] {
        need(fv != nullptr && phi != nullptr && source != nullptr && (nbound(fv) == 0 || bv != nullptr) &&
                 (ninternal(fv) == 0 || (flux != nullptr && gamma != nullptr)), "phi, bv, flux, gamma, source");
        check_scheme(scheme);
        CFDB_CUDA(cudaSetDevice(fv->device));
        h2d(fv, fv->phi, phi, ncells(fv));
        h2d(fv, fv->bv, bv, nbound(fv));
        h2d(fv, fv->flux, flux, ninternal(fv));
        h2d(fv, fv->coef, gamma, ninternal(fv));
        h2d(fv, fv->src, source, ncells(fv));
        launch_scalar_corrections(fv, fv->phi, fv->bv, scheme, fv->flux, fv->coef, linear_upwind, fv->src);
        d2h(fv, source, fv->src, ncells(fv));
        CFDB_CUDA(cudaStreamSynchronize(fv->st));
    });
}

int cfdb_device_fv_momentum_corrections(cfdb_device_fv* fv, const double* flux, const double* nu_face,
                                        int linear_upwind, int limited, int venkat, const double* eps2,
                                        double central, int transpose_term, double* source) {
    return guarded([&] {
        need(fv != nullptr && source != nullptr && (ninternal(fv) == 0 || (flux != nullptr && nu_face != nullptr)) &&
                 (!venkat || eps2 != nullptr), "flux, nu_face, eps2, source");
        // fv_openmp.cpp:205-207
        if (!fv->have_vector) fail(CFDB_ERR_NOT_READY, "DeviceFv::momentum_corrections before vector_gradient");
        CFDB_CUDA(cudaSetDevice(fv->device));
        h2d(fv, fv->flux, flux, ninternal(fv));
        h2d(fv, fv->coef, nu_face, ninternal(fv));
        h2d(fv, fv->src, source, 3 * ncells(fv));
        launch_momentum_corrections(fv, fv->vphi, fv->vbv, fv->vgrad, fv->flux, fv->coef, linear_upwind, limited,
                                    venkat, eps2, central, transpose_term, fv->src);
        d2h(fv, source, fv->src, 3 * ncells(fv));
        CFDB_CUDA(cudaStreamSynchronize(fv->st));
    });
}

int cfdb_device_fv_gradient_device(cfdb_device_fv* fv, const double* phi, const double* bv, int scheme,
                                   double* grad) {
    return guarded([&] {
        need(fv != nullptr && phi != nullptr && grad != nullptr && (nbound(fv) == 0 || bv != nullptr), "phi, bv, grad");
        check_scheme(scheme);
        CFDB_CUDA(cudaSetDevice(fv->device));
        launch_gradient<1>(fv, phi, bv, scheme, grad);
        CFDB_CUDA(cudaStreamSynchronize(fv->st));
    });
}

int cfdb_device_fv_vector_gradient_device(cfdb_device_fv* fv, const double* u, const double* ub, int scheme,
                                          double* grad) {
    return guarded([&] {
        need(fv != nullptr && u != nullptr && grad != nullptr && (nbound(fv) == 0 || ub != nullptr), "u, ub, grad");
        check_scheme(scheme);
        CFDB_CUDA(cudaSetDevice(fv->device));
        launch_gradient<3>(fv, u, ub, scheme, grad);
        CFDB_CUDA(cudaStreamSynchronize(fv->st));
    });
}

int cfdb_device_fv_scalar_corrections_device(cfdb_device_fv* fv, const double* phi, const double* bv, int scheme,
                                             const double* flux, const double* gamma, int linear_upwind,
                                             double* source) {
    return guarded([&] {
        need(fv != nullptr && phi != nullptr && source != nullptr && (nbound(fv) == 0 || bv != nullptr) &&
                 (ninternal(fv) == 0 || (flux != nullptr && gamma != nullptr)), "phi, bv, flux, gamma, source");
        check_scheme(scheme);
        CFDB_CUDA(cudaSetDevice(fv->device));
        launch_scalar_corrections(fv, phi, bv, scheme, flux, gamma, linear_upwind, source);
        CFDB_CUDA(cudaStreamSynchronize(fv->st));
    });
}

int cfdb_device_fv_momentum_corrections_device(cfdb_device_fv* fv, const double* u, const double* ub,
                                               const double* grad, const double* flux, const double* nu_face,
                                               int linear_upwind, int limited, int venkat, const double* eps2,
                                               double central, int transpose_term, double* source) {
    return guarded([&] {
        need(fv != nullptr && u != nullptr && grad != nullptr && source != nullptr &&
                 (nbound(fv) == 0 || ub != nullptr) &&
                 (ninternal(fv) == 0 || (flux != nullptr && nu_face != nullptr)) && (!venkat || eps2 != nullptr), "u, ub, grad, flux, nu_face, eps2, source");
        CFDB_CUDA(cudaSetDevice(fv->device));
        launch_momentum_corrections(fv, u, ub, grad, flux, nu_face, linear_upwind, limited, venkat, eps2, central,
                                    transpose_term, source);
        CFDB_CUDA(cudaStreamSynchronize(fv->st));
    });
}

int cfdb_device_fv_set_face_geometry(cfdb_device_fv* fv, const double* delta_coeffs, const double* unit_normals,
                                     const double* face_areas) {
    return guarded([&] {
        if (fv == nullptr || (fv->m.nf > 0 && (!delta_coeffs || !unit_normals || !face_areas)))
            fail(CFDB_ERR_BAD_ARG, "DeviceFv: null face geometry");
        CFDB_CUDA(cudaSetDevice(fv->device));
        const size_t nf = static_cast<size_t>(fv->m.nf);
        if (fv->dc == nullptr) {
            fv->dc = fv->mem.alloc<double>(nf);
            fv->un = fv->mem.alloc<double>(3 * nf);
            fv->area = fv->mem.alloc<double>(nf);
        }
        if (nf > 0) {
            CFDB_CUDA(cudaMemcpyAsync(fv->dc, delta_coeffs, sizeof(double) * nf, cudaMemcpyHostToDevice, fv->st));
            CFDB_CUDA(cudaMemcpyAsync(fv->un, unit_normals, sizeof(double) * 3 * nf, cudaMemcpyHostToDevice, fv->st));
            CFDB_CUDA(cudaMemcpyAsync(fv->area, face_areas, sizeof(double) * nf, cudaMemcpyHostToDevice, fv->st));
        }
        CFDB_CUDA(cudaStreamSynchronize(fv->st));
    });
}

int cfdb_device_fv_scalar_system_device(cfdb_device_fv* fv, const cfdb_scalar_equation* eq, const double* face_flux,
                                        double* field, double* upper, double* lower, double* diag, double* source) {
    return guarded([&] {
        if (fv == nullptr || eq == nullptr || face_flux == nullptr || field == nullptr || diag == nullptr ||
            source == nullptr || eq->gamma_face == nullptr || eq->su == nullptr || eq->sp == nullptr)
            fail(CFDB_ERR_BAD_ARG, "scalar system: null argument");
        const FvMesh& m = fv->m;
        const int nb = m.nf - m.nif;
        if (m.nif > 0 && (upper == nullptr || lower == nullptr)) fail(CFDB_ERR_BAD_ARG, "scalar system: null upper/lower");
        if (nb > 0 && (!eq->bc_kind || !eq->bc_value || !eq->bc_coefficient))
            fail(CFDB_ERR_BAD_ARG, "scalar system: boundary conditions missing");
        if (eq->fixed_cell != nullptr && eq->fixed_value == nullptr)
            fail(CFDB_ERR_BAD_ARG, "scalar system: fixed cells without values");
        if (!(eq->relaxation > 0.0)) fail(CFDB_ERR_BAD_ARG, "scalar system: relaxation must be positive");
        if (fv->dc == nullptr) fail(CFDB_ERR_NOT_READY, "scalar system: cfdb_device_fv_set_face_geometry first");
        check_scheme(eq->gradient);
        CFDB_CUDA(cudaSetDevice(fv->device));
        // bv = boundary_values(field) (scalar_transport.cpp:80), into the resident buffer
        if (nb > 0)
            k_scalar_boundary_values<<<grid(nb), kThreads, 0, fv->st>>>(m, fv->un, eq->bc_kind, eq->bc_value,
                                                                        eq->bc_coefficient, field, fv->bv);
        // a.source = 0, then the explicit face corrections (scalar_transport.cpp:81-83)
        CFDB_CUDA(cudaMemsetAsync(source, 0, sizeof(double) * m.nc, fv->st));
        launch_scalar_corrections(fv, field, fv->bv, eq->gradient, face_flux, eq->gamma_face, eq->linear_upwind,
                                  source);
        if (m.nif > 0)
            k_scalar_face_coeffs<<<grid(m.nif), kThreads, 0, fv->st>>>(m, face_flux, eq->gamma_face, fv->dc,
                                                                       eq->fixed_cell, upper, lower);
        const ScalarCellTerms t{eq->su, eq->sp, eq->old_value, eq->capacity, eq->fixed_cell, eq->fixed_value,
                                eq->relaxation, eq->dt};
        k_scalar_cells<<<grid(m.nc), kThreads, 0, fv->st>>>(m, face_flux, eq->gamma_face, fv->dc, fv->un, fv->area,
                                                            eq->bc_kind, eq->bc_value, eq->bc_coefficient, t, field,
                                                            diag, source);
        CFDB_CUDA(cudaGetLastError());
        CFDB_CUDA(cudaStreamSynchronize(fv->st));
    });
}

} // extern "C"

