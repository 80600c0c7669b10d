// Device residual norms of an LDU system (LduMatrix::residual_norms, ldu_matrix.cpp:69-103),
// used by the persistent LDU solve of the C ABI (cfdb_system_solve_ldu).
#pragma once

#include "common.hpp"

namespace cfdb {

// The LDU matrix's CSR pattern on the device: row offsets, columns, and for each pattern entry
// the index of its coefficient in [diag (n) | upper (nf) | lower (nf)].
struct LduDevice {
    int n = 0;
    int nf = 0;
    const int* rp = nullptr;
    const int* ci = nullptr;
    const int* src = nullptr;
};

// res = sum |b - A x|, norm = sum (|A x - A x_ref| + |b - A x_ref|) with x_ref = mean(x) (the
// OpenFOAM normalisation; normalised residual = res / (norm + 1e-20)), r2 = sum (b - A x)^2.
struct LduNorms {
    double res = 0.0;
    double norm = 0.0;
    double r2 = 0.0;
};

constexpr int kLduNormBlocks = 592; // 148 SMs x 4; partial sums per block

// part: device scratch of 3 * kLduNormBlocks doubles. Synchronises st.
LduNorms ldu_residual_norms(const LduDevice& m, const double* diag, const double* upper, const double* lower,
                            const double* b, const double* x, double* part, cudaStream_t st);

} // namespace cfdb
