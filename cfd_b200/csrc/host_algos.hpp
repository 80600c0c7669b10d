// Host algorithms around the device solver: LDU pattern construction and the
// smoothed-aggregation AMG setup. These run on the CPU (as in the reference, where the
// hierarchy is built on the host and only the V-cycle / CG run on the accelerator).
#pragma once

#include "common.hpp"

namespace cfdb {

struct AmgSettings {
    double theta = 0.08;  // amg.hpp:18
    int max_levels = 25;  // amg.hpp:19
    int coarse_size = 400; // amg.hpp:20
    int sweeps = 2;       // krylov.hpp:56
    double weight = 0.7;  // krylov.hpp:57
    int table_limit = 0;  // device setup: largest row kept in shared-memory tables (0: default)
};

struct LduPatternHost {
    int n = 0;
    int n_faces = 0;
    std::vector<int> row_ptr, col, diag_pos, upper_pos, lower_pos;
    [[nodiscard]] int nnz() const { return row_ptr.empty() ? 0 : row_ptr.back(); }
};

// fv::build_csr_pattern (ldu_matrix.cpp:572-612): sorted unique columns per row.
LduPatternHost build_pattern(int n, int nf, const int* owner, const int* neighbour);

// Hierarchy as produced by fv::AmgPreconditioner::setup (amg.cpp:122-190).
struct Hierarchy {
    std::vector<HostCsr> a, p, r;          // a[0] = the input matrix
    std::vector<std::vector<int>> agg;     // aggregates of each non-coarsest level
    std::vector<int> n_agg;
    int n_c = 0;
    bool ldlt_ok = false;
    std::vector<double> coarse_inverse;    // dense row-major n_c x n_c
    [[nodiscard]] int levels() const { return static_cast<int>(a.size()); }
    [[nodiscard]] double operator_complexity() const;
};

// Aggregation of amg.cpp:12-78 (serial, order dependent by design).
int aggregate(const HostCsr& a, const std::vector<double>& diag, double theta, std::vector<int>& agg);

// The same aggregation from the strength graph alone: row i's strong connections (i != j and
// |a_ij| > theta sqrt|d_i d_j|) in CSR order, columns sci[srp[i]..srp[i+1]) with |a_ij| in sav.
// Every test of amg.cpp:12-78 reads only strong entries, so the result equals aggregate().
int aggregate_strong(int n, const int* srp, const int* sci, const double* sav, std::vector<int>& agg);
// The same with sav replaced by each strong entry's rank within its row by (|a_ij| descending,
// position ascending): the strict-maximum choice of pass 2 is then the smallest eligible rank.
int aggregate_strong_ranked(int n, const int* srp, const int* sci, const uint16_t* rank, std::vector<int>& agg);

// Full setup. Sparse products use Gustavson order (row i: k ascending in A(i,:), j ascending
// in B(k,:), first touch assigns), run row-parallel, so the result is independent of threads.
Hierarchy amg_setup(const HostCsr& a, const AmgSettings& s);

// Dense LDL^T inverse (natural order, no pivoting); returns false if a pivot is zero, in which
// case inv receives the Moore-Penrose pseudo-inverse.
bool dense_inverse(int n, const std::vector<double>& a, std::vector<double>& inv);

} // namespace cfdb
