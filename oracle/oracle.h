/*
 * CPU oracle for the pressure-correction hot path (TEST INFRASTRUCTURE ONLY).
 *
 * A plain-C, serial restatement of the reference algorithms (Yipexnn/CFD) that the CUDA
 * path replaces. Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference legs may load it, and only as the checker or the timed CPU baseline; the
 * product library never links or calls it.
 *
 * Pinning: the assembly, Jacobi-CG, BiCGStab and the Jacobi-smoothed AMG-PCG restated here
 * are checked bit-for-bit against the reference's own host sources compiled unchanged into
 * oracle/_ref (see oracle/ref_shim.cpp). The aggregation / smoothed-aggregation setup and the
 * Gauss-Seidel AmgCg follow src/fv/src/amg.cpp, whose Eigen products cannot be compiled here:
 * their Galerkin summation order is the documented Gustavson order below ("parity unpinned"
 * against Eigen for coarse-level values; level-0 aggregates depend only on assembled values).
 *
 * Floating point: compile without contraction (-ffp-contract=off) so every product and sum is
 * rounded exactly as the reference's x86-64 host build rounds it.
 */
#ifndef CFD_ORACLE_H
#define CFD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- LDU matrix (src/fv/src/ldu_matrix.cpp) ---- */

/* build_csr_pattern (ldu_matrix.cpp:572-612): CSR structure of diag + both face entries with
 * sorted unique columns; positions of diag / upper (own,nei) / lower (nei,own).
 * col must hold n + 2*nf entries; returns nnz (or -1 on an index error). */
int orc_build_pattern(int n, int nf, const int* own, const int* nei, int* row_ptr, int* col,
                      int* diag_pos, int* upper_pos, int* lower_pos);

/* Serial face loop of assemble_openmp (src/gpu/src/krylov_openmp.cpp:289-300);
 * diag and div are accumulated, not cleared. */
void orc_assemble(int n_cells, int n_faces, const int* own, const int* nei, const double* flux,
                  const double* gamma, const double* delta, double convection, double* upper,
                  double* lower, double* diag, double* div);

/* LduMatrix::multiply (ldu_matrix.cpp:39-56): face-loop scatter then diagonal. */
void orc_ldu_multiply(int n, int nf, const int* own, const int* nei, const double* diag,
                      const double* upper, const double* lower, const double* x, double* y);

/* LduMatrix::residual_norms (ldu_matrix.cpp:69-103), serial: out[0] = |b-Ax|_1,
 * out[1] = normFactor. */
void orc_ldu_residual_norms(int n, int nf, const int* own, const int* nei, const double* diag,
                            const double* upper, const double* lower, const double* source,
                            const double* x, double* out);

/* LduMatrix::set_reference (ldu_matrix.cpp:105-109). */
void orc_set_reference(double* diag, double* source, int cell, double value);

/* Scatter of LDU values into CSR positions (device_solver.cpp:127-134). */
void orc_ldu_to_csr(int n, int nf, const int* diag_pos, const int* upper_pos,
                    const int* lower_pos, const double* diag, const double* upper,
                    const double* lower, double* val);

/* ---- CSR helpers ---- */
void orc_csr_spmv(int n, const int* rp, const int* ci, const double* va, const double* x,
                  double* y);

/* ---- Smoothed-aggregation AMG setup (src/fv/src/amg.cpp) ---- */

/* amg_aggregate (amg.cpp:12-78): three-pass greedy aggregation on the strength graph.
 * Returns the number of aggregates; agg[n] receives the aggregate of each row. */
int orc_aggregate(int n, const int* rp, const int* ci, const double* va, const double* diag,
                  double theta, int* agg);

typedef struct orc_amg orc_amg;

/* AmgPreconditioner::setup (amg.cpp:122-190) with AmgSettings (theta, max_levels,
 * coarse_size). Returns NULL on a non-square / invalid input. */
orc_amg* orc_amg_setup(int n, const int* rp, const int* ci, const double* va, double theta,
                       int max_levels, int coarse_size);
void orc_amg_free(orc_amg* h);
int orc_amg_levels(const orc_amg* h);
/* which: 0 = A (operator), 1 = P (prolongation), 2 = R (restriction). Returns 0 if absent. */
int orc_amg_level_csr(const orc_amg* h, int level, int which, int* n_rows, int* n_cols,
                      int* nnz, const int** rp, const int** ci, const double** va);
/* Aggregates of level l (l < levels-1). */
const int* orc_amg_aggregates(const orc_amg* h, int level, int* n_agg);
/* Dense row-major inverse of the coarsest operator (AmgPreconditioner::coarse_inverse,
 * amg.cpp:227-240); *ok = 1 if the LDL^T factorisation succeeded (else pseudo-inverse). */
const double* orc_amg_coarse_inverse(const orc_amg* h, int* n_c, int* ok);
double orc_amg_operator_complexity(const orc_amg* h);

/* pcg with the Gauss-Seidel V-cycle (amg.cpp:192-216, 253-285): the CPU AmgCg path.
 * Returns iterations; *res_out = |r|_2 at exit. */
int orc_pcg_gs(const orc_amg* h, const double* b, double* x, double tolerance,
               int max_iterations, double* res_out);

/* ---- Accelerator-path algorithms (src/gpu/src/krylov_kernels.inc) ---- */

typedef struct {
    int n;
    const int* rp;
    const int* ci;
    const double* va;
} orc_csr_view;

typedef struct {
    int iterations;
    double residual;
    int converged;
} orc_stats;

/* amg_cg (krylov_kernels.inc:240-301) with the Jacobi V-cycle (:182-238) over an explicit
 * hierarchy: a[l] for all levels, p[l] / r[l] for l < n_levels-1, the dense row-major inverse
 * of the coarsest operator. */
orc_stats orc_amg_cg(int n_levels, const orc_csr_view* a, const orc_csr_view* p,
                     const orc_csr_view* r, const double* coarse_inverse, int sweeps,
                     double weight, const double* b, double* x, double abs_tol, int max_iter);

/* One V-cycle application z = M^-1 r (vcycle with zero initial guess, :209-238). */
void orc_vcycle_apply(int n_levels, const orc_csr_view* a, const orc_csr_view* p,
                      const orc_csr_view* r, const double* coarse_inverse, int sweeps,
                      double weight, const double* rhs, double* z);

/* Jacobi-preconditioned cg (:44-95) and bicgstab (:98-169); method 0 = CG, 1 = BiCGStab. */
orc_stats orc_krylov(const orc_csr_view* a, const double* b, double* x, int method,
                     double abs_tol, int max_iter);

#ifdef __cplusplus
}
#endif
#endif
