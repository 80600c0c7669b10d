/*
 * cfdb: B200-native (sm_100a) pressure-correction solver -- the C ABI.
 *
 * Drop-in for the accelerator call surface of Yipexnn/CFD (namespace cfd::gpu,
 * src/gpu/include/cfd/gpu/krylov.hpp), the path selected by "solver": {"device": "gpu"}.
 * Each entry point names the reference interface it replaces. Plain C types only: host
 * pointers unless the name ends in _device (then every array argument is a device pointer on
 * the system's GPU). All calls return a cfdb_status; on failure cfdb_last_error() gives the
 * message of the calling thread's last error. Non-convergence is not an error (stats).
 */
#ifndef CFDB_H
#define CFDB_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    CFDB_OK = 0,
    CFDB_ERR_BAD_ARG = 1,   /* reference: std::invalid_argument */
    CFDB_ERR_CUDA = 2,      /* reference: std::runtime_error("CUDA <what>: <msg>") */
    CFDB_ERR_OOM = 3,       /* device allocation failed / admission over budget */
    CFDB_ERR_NO_DEVICE = 4, /* no CUDA device: this library has no host fallback */
    CFDB_ERR_NOT_READY = 5, /* e.g. AMG solve requested before a hierarchy was set */
    CFDB_ERR_TIMEOUT = 6,   /* a bounded device wait expired */
    CFDB_ERR_INTERNAL = 7
} cfdb_status;

/* krylov.hpp:10-16 CsrView: square or rectangular CSR (0-based). */
typedef struct {
    int n;   /* rows */
    int nnz;
    const int* row_ptr; /* n + 1 */
    const int* col;     /* nnz */
    const double* val;  /* nnz */
} cfdb_csr;

/* krylov.hpp:48-52 AmgLevelView: a (n_l x n_l), p (n_l x n_{l+1}), r (n_{l+1} x n_l). */
typedef struct {
    cfdb_csr a;
    cfdb_csr p;
    cfdb_csr r;
} cfdb_amg_level;

/* krylov.hpp:53-58 AmgView. coarse_inverse: dense row-major inverse of the coarsest a. */
typedef struct {
    int n_levels;
    const cfdb_amg_level* levels;
    const double* coarse_inverse;
    int smooth_sweeps;    /* reference default 2 */
    double jacobi_weight; /* reference default 0.7 */
} cfdb_amg_view;

/* krylov.hpp:21-24 SolveControl. */
typedef struct {
    double abs_tolerance; /* stop when |r|_2 <= abs_tolerance */
    int max_iterations;
} cfdb_control;

/* krylov.hpp:26-31 SolveStats (+ the true residual recomputed in FP64 after the solve). */
typedef struct {
    int iterations;
    double residual; /* |r|_2 of the solver's residual at exit (reference semantics) */
    int converged;
    int on_device;
    double true_residual; /* |b - A x|_2 recomputed in FP64 from the returned x */
} cfdb_stats;

/* krylov.hpp:68-77 LduPattern: CSR pattern + positions of diag / upper / lower values. */
typedef struct {
    int n;
    int n_faces;
    int nnz;
    const int* row_ptr;
    const int* col;
    const int* diag_pos;
    const int* upper_pos;
    const int* lower_pos;
} cfdb_ldu_pattern;

typedef enum { CFDB_METHOD_CG = 0, CFDB_METHOD_BICGSTAB = 1 } cfdb_method;

/* Arithmetic of the AMG V-cycle. FP64: the reference algorithm. MIXED: hierarchy and V-cycle
 * in FP32 (FP32 accumulation) inside an FP64 flexible CG; the outer residual recompute, dots
 * and the coarsest-level inverse stay FP64. */
typedef enum { CFDB_PRECISION_FP64 = 0, CFDB_PRECISION_MIXED = 1 } cfdb_precision;

/* amg.hpp:17-23 AmgSettings (+ the AmgView smoother defaults). */
typedef struct {
    double strength_threshold; /* 0.08 */
    int max_levels;            /* 25 */
    int coarse_size;           /* 400 */
    int smooth_sweeps;         /* 2 */
    double jacobi_weight;      /* 0.7 */
    /* device setup only (no effect on results): rows of a sparse product or transpose with
     * more entries than this use device-memory tables instead of shared memory (0: 6144) */
    int device_table_limit;
} cfdb_amg_settings;

/* ---- backend queries: krylov.hpp:118-123 ---- */
int cfdb_backend_name(char* buf, size_t len);        /* backend_name(): "cuda" */
int cfdb_device_available(void);                    /* device_available() */
int cfdb_device_description(char* buf, size_t len); /* device_description() */
int cfdb_last_error(char* buf, size_t len);          /* message of the last failed call */
/* Device memory freed by destroyed systems, plans and setups stays cached in the library's
 * stream-ordered pools for reuse; this returns it to the driver (current device). */
int cfdb_release_cached_memory(void);
void cfdb_default_amg_settings(cfdb_amg_settings* s);

/* ---- one-shot calls ---- */

/* assemble_convection_diffusion (krylov.hpp:105-116; CUDA krylov_cuda.cu:701-741).
 * upper = min(cF,0) - G, lower = -max(cF,0) - G, diag[own] += max(cF,0) + G,
 * diag[nei] += -min(cF,0) + G, div[own] += F, div[nei] -= F, G = gamma*delta, c = convection.
 * diag and divergence are accumulated (not cleared). Atomic-free, bit-identical to the
 * reference's serial loop (each cell adds its faces in ascending face order). */
int cfdb_assemble(int n_cells, int n_faces, const int* owner, const int* neighbour,
                  const double* flux, const double* gamma, const double* delta_coeff,
                  double convection, double* upper, double* lower, double* diag,
                  double* divergence);
/* Same on device arrays (no host copies), on the calling thread's library stream. */
int cfdb_assemble_device(int n_cells, int n_faces, const int* owner, const int* neighbour,
                         const double* flux, const double* gamma, const double* delta_coeff,
                         double convection, double* upper, double* lower, double* diag,
                         double* divergence);

/* solve (krylov.hpp:37-38): Jacobi-preconditioned CG / BiCGStab on a host CSR matrix. */
int cfdb_solve(const cfdb_csr* a, const double* b, double* x, int method,
               const cfdb_control* control, cfdb_stats* stats);

/* solve_amg_cg (krylov.hpp:61-62): AMG-preconditioned CG, A = levels[0].a. */
int cfdb_solve_amg_cg(const cfdb_amg_view* amg, const double* b, double* x,
                      const cfdb_control* control, cfdb_stats* stats);

/* Allocation-free Jacobi-preconditioned CG (no counterpart in the reference). For callers that
 * cannot call cudaMalloc -- a host application that owns all device memory through its own
 * pool, or a latency-critical loop that must not stall on the allocator. The matrix (CSR),
 * b and x (initial guess in, solution out) are the caller's device arrays; the work vectors
 * live in one static device array of the library, so at most 65,536 rows (larger n is
 * rejected with CFDB_ERR_BAD_ARG). The first call on each device resolves that array's address
 * and should come before any stream capture. Calls share the array: calls that overlap on the
 * GPU race. Same iteration and stopping rule as cfdb_solve; runs on the legacy default
 * stream and returns when the solve is done, so a caller that wrote a, b or x on a
 * non-blocking stream must finish those writes first. Every array must be device memory of the
 * current device (or managed memory); the CSR structure (row offsets, column range) is checked
 * on the device before use, and a bad one is rejected with CFDB_ERR_BAD_ARG. */
int cfdb_solve_device_noalloc(const cfdb_csr* a, const double* b, double* x, int method,
                              const cfdb_control* control, cfdb_stats* stats);

/* ---- CSR pattern: fv::build_csr_pattern (src/fv/src/ldu_matrix.cpp:572-612) ----
 * col, upper_pos, lower_pos sized n + 2*n_faces / n_faces; returns nnz in *nnz. */
int cfdb_build_pattern(int n, int n_faces, const int* owner, const int* neighbour,
                       int* row_ptr, int* col, int* diag_pos, int* upper_pos, int* lower_pos,
                       int* nnz);

/* ---- host AMG setup: fv::AmgPreconditioner::setup (src/fv/src/amg.cpp:122-190) ---- */
typedef struct cfdb_hierarchy cfdb_hierarchy;
int cfdb_amg_setup(const cfdb_csr* a, const cfdb_amg_settings* settings,
                   cfdb_hierarchy** out);
/* The same hierarchy built on the device (sparse products, strength graph, transfers and
 * Galerkin operators in CUDA kernels; the sequential aggregation on the host), bit-identical
 * to cfdb_amg_setup. */
int cfdb_amg_setup_device(const cfdb_csr* a, const cfdb_amg_settings* settings,
                          cfdb_hierarchy** out);
int cfdb_hierarchy_destroy(cfdb_hierarchy* h);
/* levels() / level_matrix / level_prolongation / level_restriction (amg.hpp:37-54);
 * which: 0 = a, 1 = p, 2 = r. Pointers stay valid while h lives. */
int cfdb_hierarchy_levels(const cfdb_hierarchy* h, int* n_levels);
int cfdb_hierarchy_level(const cfdb_hierarchy* h, int level, int which, int* n_rows,
                         int* n_cols, cfdb_csr* m);
int cfdb_hierarchy_aggregates(const cfdb_hierarchy* h, int level, const int** agg,
                              int* n_aggregates);
/* coarse_inverse() (amg.cpp:227-240), dense row-major. */
int cfdb_hierarchy_coarse_inverse(const cfdb_hierarchy* h, const double** inv, int* n_c);
/* AmgView of the hierarchy with the given smoother; levels storage owned by h. */
int cfdb_hierarchy_view(cfdb_hierarchy* h, int smooth_sweeps, double jacobi_weight,
                        cfdb_amg_view* view);
int cfdb_hierarchy_operator_complexity(const cfdb_hierarchy* h, double* oc);

/* ---- persistent system: DeviceSolver (krylov.hpp:83-103; krylov_cuda.cu:566-677) ---- */
typedef struct cfdb_system cfdb_system;

/* DeviceSolver(const LduPattern&): the pattern is copied; the GPU is the current device. */
int cfdb_system_create(const cfdb_ldu_pattern* pattern, cfdb_system** out);
/* Same from mesh addressing (builds the pattern; keeps owner/neighbour for the fused
 * face-data assembly below). */
int cfdb_system_create_mesh(int n_cells, int n_faces, const int* owner, const int* neighbour,
                            cfdb_system** out);
int cfdb_system_destroy(cfdb_system* sys);                 /* ~DeviceSolver() */
int cfdb_system_on_device(const cfdb_system* sys);         /* on_device() */
/* set_amg(const AmgView&): levels[0].a is ignored (assembled on the device). */
int cfdb_system_set_amg(cfdb_system* sys, const cfdb_amg_view* amg);
/* Builds the hierarchy from LDU coefficients on the host (AmgPreconditioner::setup) and
 * installs it, as LduMatrix::solve_persistent does on an AMG rebuild (ldu_matrix.cpp:314-353).*/
int cfdb_system_setup_amg(cfdb_system* sys, const double* diag, const double* upper,
                          const double* lower, const cfdb_amg_settings* settings);
/* cfdb_system_setup_amg with the hierarchy built on the device (as cfdb_amg_setup_device);
 * device_arrays: diag/upper/lower are device pointers (ready when the call is made). */
int cfdb_system_setup_amg_device(cfdb_system* sys, const double* diag, const double* upper,
                                 const double* lower, const cfdb_amg_settings* settings,
                                 int device_arrays);
/* Kernel timing: average device time (ms) of `reps` back-to-back Jacobi sweeps of level
 * `level` in the installed plan (its precision and launch shape) and the algorithmic bytes of
 * one sweep. The sweep reads the level's current vectors; solve results are not affected. */
int cfdb_system_time_sweep(cfdb_system* sys, int level, int reps, double* ms, double* bytes);
/* Whether a device setup keeps its levels on the device (default 1). They let the plan be
 * rebuilt (set_precision, set_tuning, set_ordered) without a new setup; without them such a
 * change after a device setup fails with CFDB_ERR_NOT_READY until the next setup. */
int cfdb_system_set_keep_levels(cfdb_system* sys, int keep);
/* Wall-clock seconds of the phases of the last hierarchy setup of sys, as text
 * "phase=seconds;..." (host setup: hierarchy, plan; device setup: strength, aggregate,
 * prolongation, transpose, AP, RAP, coarse_inverse, input, keep, plan). */
int cfdb_system_setup_profile(const cfdb_system* sys, char* buf, size_t len);
int cfdb_system_set_precision(cfdb_system* sys, int precision);
/* solve(diag, upper, lower, b, x, method, use_amg, control): assembles A from LDU on the
 * device and solves A x = b; x is the initial guess in and the solution out. */
int cfdb_system_solve(cfdb_system* sys, const double* diag, const double* upper,
                      const double* lower, const double* b, double* x, int method, int use_amg,
                      const cfdb_control* control, cfdb_stats* stats);
/* Same with device-resident arrays (no host transfers): the HBM-resident hot path. */
int cfdb_system_solve_device(cfdb_system* sys, const double* diag, const double* upper,
                             const double* lower, const double* b, double* x, int method,
                             int use_amg, const cfdb_control* control, cfdb_stats* stats);
/* ---- pressure gradient and velocity correction (FlowSolver::pressure_correction after the
 * solve: pressure_gradient's Gauss branch, flow_solver.cpp:339-372, and u = HbyA - rAU grad p,
 * flow_solver.cpp:843-846) on device arrays ---- */
typedef enum { /* flow_solver.hpp:16 FlowBoundary */
    CFDB_BC_VELOCITY_INLET = 0,
    CFDB_BC_WALL = 1,
    CFDB_BC_PRESSURE_OUTLET = 2,
    CFDB_BC_SYMMETRY = 3,
    CFDB_BC_EMPTY = 4
} cfdb_boundary_kind;
typedef struct cfdb_fv cfdb_fv;
/* Mesh geometry in the reference's contract (host arrays, copied): owner (n_faces), neighbour
 * and interpolation weights (internal faces), face area vectors and face centres (3 n_faces,
 * xyz-interleaved), cell centres (3 n_cells), cell volumes; per boundary face (n_faces -
 * n_internal_faces, in face order) its cfdb_boundary_kind and, for pressure outlets, the
 * fixed pressure. */
int cfdb_fv_create(int n_cells, int n_faces, int n_internal_faces, const int* owner,
                   const int* neighbour, const double* face_areas, const double* face_centres,
                   const double* cell_centres, const double* cell_volumes, const double* weights,
                   const int* boundary_kind, const double* boundary_pressure, cfdb_fv** out);
/* Cells, faces and internal faces of the geometry (no reference counterpart). */
int cfdb_fv_sizes(const cfdb_fv* fv, int* n_cells, int* n_faces, int* n_internal_faces);
int cfdb_fv_destroy(cfdb_fv* fv);
/* grad (3 n_cells) of the cell pressure p (n_cells): Gauss sums with boundary values p_P, or
 * the outlet pressure, in two passes, the second extrapolating zero-gradient boundary values
 * tangentially with the first pass's gradient. Device arrays; returns when done. */
int cfdb_fv_pressure_gradient_device(cfdb_fv* fv, const double* p, double* grad);
/* u = hbya - rau * grad (u, hbya, grad: 3 n_cells; rau: n_cells). Device arrays. */
int cfdb_fv_correct_velocity_device(cfdb_fv* fv, const double* hbya, const double* rau,
                                    const double* grad, double* u);
/* The delta coefficients of all faces (device array of n_faces, owned by fv;
 * fv_geometry.cpp:43-50), e.g. the internal prefix for cfdb_system_assemble_pressure_device. */
int cfdb_fv_delta_device(const cfdb_fv* fv, const double** delta);
/* HbyA = (source - offdiag(U)) / diag per component and rAU = V / mean(diag)
 * (flow_solver.cpp:688-707) from the momentum system: diag, source 3 n_cells, shared
 * off-diagonal upper / lower (internal faces), velocity u 3 n_cells. */
int cfdb_fv_hbya_rau_device(cfdb_fv* fv, const double* mom_diag, const double* mom_upper,
                            const double* mom_lower, const double* mom_source, const double* u,
                            double* hbya, double* rau);
/* Predicted face flux phi_hbya and face rAU (n_faces each; flow_solver.cpp:709-733): linear
 * interpolation on internal faces; on boundary faces rAU_P and, by kind, the fixed velocity
 * (fixed_velocity: 3 per boundary face; inlets and walls), HbyA_P (outlets) or 0. With u_prev
 * and phi_prev (else both NULL) the relaxation-independent term beta (phi_prev - u_prev_f . S)
 * is added (flow_solver.cpp:735-752). */
int cfdb_fv_face_flux_device(cfdb_fv* fv, const double* hbya, const double* rau,
                             const double* fixed_velocity, const double* u_prev,
                             const double* phi_prev, double beta, double* phi_hbya, double* rau_f);
/* Boundary terms of the pressure equation after the internal assembly (flow_solver.cpp:
 * 784-796): source -= phi_hbya on every boundary face, outlets add rAU_f delta to diag and
 * rAU_f delta p_out to source; then set_reference(ref_cell, ref_value) unless ref_cell < 0. */
int cfdb_fv_pressure_boundary_device(cfdb_fv* fv, const double* phi_hbya, const double* rau_f,
                                     int ref_cell, double ref_value, double* diag, double* source);
/* Non-orthogonal corrector (flow_solver.cpp:805-816): non_orth = rAU_f k . (w grad_P +
 * (1 - w) grad_N) per internal face; source = base_source + sum of +-non_orth per cell. */
int cfdb_fv_non_orth_device(cfdb_fv* fv, const double* grad, const double* rau_f,
                            const double* base_source, double* non_orth, double* source);
/* Conservative flux on every face from the pressure solution (flow_solver.cpp:818-833);
 * non_orth may be NULL (zero). */
int cfdb_fv_correct_flux_device(cfdb_fv* fv, const double* phi_hbya, const double* rau_f,
                                const double* non_orth, const double* p_new, double* phi);
/* p = p_prev + alpha (p_new - p_prev) (flow_solver.cpp:837-840). */
int cfdb_fv_relax_device(cfdb_fv* fv, const double* p_prev, const double* p_new, double alpha,
                         double* p);

/* ---- persistent LDU solve: LduMatrix::solve with "solver": {"device": "gpu"}
 * (ldu_matrix.cpp:111-131 with solve_persistent, ldu_matrix.cpp:287-366) ---- */
typedef struct {
    int method;           /* CFDB_METHOD_CG (LinearSolverType::GpuCg: AMG-CG) or
                             CFDB_METHOD_BICGSTAB (GpuBiCgStab: Jacobi BiCGStab) */
    double tolerance;     /* absolute, on the normalised residual (1e-10) */
    double rel_tolerance; /* relative to the initial normalised residual (0.01) */
    int max_iterations;   /* 1000 */
    int max_age;          /* AmgCache::max_age: hierarchy rebuilt after this many CG solves (20) */
} cfdb_ldu_settings;
typedef struct {
    double initial_residual; /* LinearSolveResult: normalised residuals before and after */
    double final_residual;
    int iterations;
    int amg_rebuilt;         /* 1 when this call (re)built the hierarchy */
} cfdb_ldu_result;
void cfdb_default_ldu_settings(cfdb_ldu_settings* s);
/* Solves A x = source for the LDU matrix (x: initial guess in, solution out) with the
 * reference's stopping rule: returns at once when the normalised residual of x is below
 * `tolerance`; otherwise CG/BiCGStab runs to max(rel_tolerance, tolerance / initial) times the
 * initial residual 2-norm. With CG the hierarchy is built (on the device) at the first call and
 * again every max_age solves; a one-level hierarchy runs Jacobi CG (ldu_matrix.cpp:358).
 * device_arrays: all arrays are device pointers (else host arrays, copied once per call). */
int cfdb_system_solve_ldu(cfdb_system* sys, const double* diag, const double* upper,
                          const double* lower, const double* source, double* x,
                          const cfdb_ldu_settings* settings, const cfdb_amg_settings* amg,
                          int device_arrays, cfdb_ldu_result* result);

/* ---- the whole pressure correction: FlowSolver::pressure_correction
 * (src/fv/src/flow_solver.cpp:673-847) with every array in device memory ----
 * HbyA / rAU from the momentum system, the predicted face flux and face rAU (with the
 * relaxation-independent term when u_prev and phi_prev are given and alpha_u < 1), the pressure
 * equation with boundary terms and reference cell, n_non_orth_correctors + 1 persistent LDU
 * solves (cfdb_system_solve_ldu, AmgCache rule) with the non-orthogonal corrector sources, the
 * conservative face flux, pressure relaxation and the velocity correction, in the reference's
 * order, each step the device kernel bit-identical to the reference's loop. u (n x 3) and p (n)
 * are updated in place; ws->phi receives the conservative flux. sys and fv must describe the
 * same mesh (sys over its internal faces). The workspace is the caller's device memory, so the
 * call allocates none of its own. results (optional, n_non_orth_correctors + 1 entries, host)
 * and ws->solve_p / ws->solve_source (optional, (n_non_orth_correctors + 1) x n each) record
 * every solve. Returns when the step is done. */
typedef struct {
    double alpha_u;            /* momentum under-relaxation (for the relaxation-independent term) */
    double alpha_p;            /* pressure under-relaxation */
    int n_non_orth_correctors;
    int ref_cell;              /* -1: none (a case with a pressure outlet) */
    double ref_value;
    int relax_p;               /* 1: p = p_prev + alpha_p (p_new - p_prev); 0: p = p_new */
    cfdb_ldu_settings p_solver;
    cfdb_amg_settings amg;
} cfdb_pressure_settings;
typedef struct {
    double* hbya;         /* n x 3 */
    double* rau;          /* n */
    double* phi_hbya;     /* n_faces */
    double* rau_f;        /* n_faces */
    double* upper;        /* n_internal_faces */
    double* lower;        /* n_internal_faces */
    double* diag;         /* n */
    double* source;       /* n: right-hand side of the current solve */
    double* base_source;  /* n: right-hand side before the corrector terms */
    double* p_prev;       /* n */
    double* p_new;        /* n */
    double* non_orth;     /* max(n_internal_faces, 1) */
    double* grad;         /* n x 3 */
    double* phi;          /* n_faces: conservative face flux (output) */
    double* solve_p;      /* optional */
    double* solve_source; /* optional */
} cfdb_pressure_workspace;
int cfdb_pressure_correction_device(cfdb_system* sys, cfdb_fv* fv, const double* mom_diag,
                                    const double* mom_upper, const double* mom_lower,
                                    const double* mom_source, double* u, double* p,
                                    const double* fixed_velocity, const double* u_prev,
                                    const double* phi_prev, const cfdb_pressure_settings* settings,
                                    const cfdb_pressure_workspace* ws, cfdb_ldu_result* results,
                                    double* initial_residual);
/* Fused pressure assembly on device arrays (flow_solver.cpp:757-783 with the face loop of
 * krylov_cuda.cu:681-697): from face flux / gamma / delta (n_faces) builds the device matrix
 * directly and returns upper, lower (n_faces) and diag, divergence (n_cells, accumulated)
 * like cfdb_assemble. Requires cfdb_system_create_mesh. */
int cfdb_system_assemble_device(cfdb_system* sys, const double* flux, const double* gamma,
                                const double* delta_coeff, double convection, double* upper,
                                double* lower, double* diag, double* divergence);
/* AmgPreconditioner::apply (amg.hpp:33; accelerator V-cycle krylov_kernels.inc:209-238): one
 * V-cycle z = M^-1 r with zero initial guess on the installed hierarchy and the current
 * matrix (set by the last solve), in the system's precision. Host arrays. */
int cfdb_system_apply_amg(cfdb_system* sys, const double* r, double* z);
/* Ordered arithmetic: every level operator stored for thread-per-row sums in the CSR column
 * order, so FP64 V-cycles are bit-identical to the reference's sequential host arithmetic
 * (slower on wide coarse levels). Default off: wide coarse rows use warp-per-row sums. */
int cfdb_system_set_ordered(cfdb_system* sys, int ordered);

/* Per-kernel device time of the initial preconditioning plus one iteration (events around
 * every kernel, averaged over reps after one warm-up), with each kernel's algorithmic bytes. */
typedef struct {
    char name[32];
    int level;
    double ms;
    double bytes;
} cfdb_kernel_record;
int cfdb_system_profile(cfdb_system* sys, int use_amg, int reps, cfdb_kernel_record* records,
                        int max_records, int* n_records);

/* cfdb_system_assemble_device with host arrays (the reference's assemble call on a persistent
 * mesh: inputs copied to the device, results copied back). On meshes of 2^19 cells or more the
 * copies run in up to 8 cell slices, each slice's results copied back while the next slice
 * uploads; page-locked arrays let the two directions overlap. Returns when every result is in
 * the host arrays. */
int cfdb_system_assemble(cfdb_system* sys, const double* flux, const double* gamma,
                         const double* delta_coeff, double convection, double* upper,
                         double* lower, double* diag, double* divergence);
/* The whole pressure-equation assembly of FlowSolver::pressure_correction for internal faces
 * on device arrays (flow_solver.cpp:757-796, convection 0): upper = lower = -gamma*delta,
 * diag = diag0 + sum of gamma*delta (diag0 may be NULL: zero), source = source0 - div(flux),
 * then set_reference(ref_cell, ref_value) unless ref_cell < 0. Requires
 * cfdb_system_create_mesh. Enqueued on the system's stream (cfdb_system_stream) and returns at
 * once: work on other streams that reads or writes the outputs must wait for that stream. */
/* The steps of FlowSolver::pressure_correction after the pressure solve, for internal faces on
 * device arrays: the conservative face flux phi = flux - gamma*delta*(p_new[N] - p_new[P]) -
 * non_orth (flow_solver.cpp:821-826; non_orth may be NULL: zero) and the under-relaxed
 * pressure p = p_prev + alpha (p_new - p_prev) (flow_solver.cpp:837-840; p_prev NULL: p =
 * p_new). Enqueued on the system's stream. Requires cfdb_system_create_mesh. */
int cfdb_system_correct_pressure_device(cfdb_system* sys, const double* flux, const double* gamma,
                                        const double* delta, const double* non_orth,
                                        const double* p_new, const double* p_prev, double alpha,
                                        double* phi, double* p);
int cfdb_system_assemble_pressure_device(cfdb_system* sys, const double* flux,
                                         const double* gamma, const double* delta_coeff,
                                         const double* diag0, const double* source0,
                                         int ref_cell, double ref_value, double* upper,
                                         double* lower, double* diag, double* source);
/* Number of this library's kernels the system has launched so far (graph nodes included). */
int cfdb_system_kernel_launches(const cfdb_system* sys, unsigned long long* count);

/* Launch-shape / schedule knobs of the device plan (see cfd_b200/autotune.py). */
typedef struct {
    int target_tiles; /* level-0 Krylov tiles (reductions): about this many CTAs, default 1184 =
                         148 SMs x 8; 0 = 256 rows per CTA */
    int wide_row;     /* average row length above which CSR lane groups are used, default 48 */
    int lanes_div;    /* lanes per CSR row ~ average row length / lanes_div (4..256, and enough
                         lanes for ~150K threads per operator), default 16 */
    int fuse_first;   /* first two smoothing sweeps in one kernel, default 0 */
    int sell_rows;    /* rows per CTA of SELL operators (one row per thread per pass): a multiple
                         of 256, default 256 */
    int krylov_pair;  /* level-0 Krylov SpMV kernels take two rows per thread per pass (1) or one
                         (0), default 1 */
    int tail_rows;    /* coarse levels of at most this many rows, with all coarser ones, run as one
                         persistent kernel; 0 (default) disables it */
    int col16;        /* FP32 operators keep 16-bit column offsets from a per-slice / per-row base
                         where every slice / row spans fewer than 65536 columns, default 0 */
    int pdl;          /* programmatic dependent launch between consecutive kernels (a kernel is
                         scheduled while its predecessor drains), default 1 */
    int wait_polls;   /* poll limit of the bounded device waits (coarse-level staging barrier,
                         persistent-tail grid barrier), default 2^22 (0 = default); a negative value
                         makes every such wait give up at once, which the tests of the expiry path
                         (CFDB_ERR_TIMEOUT) use. An expired staging wait still drains its own
                         copy before the CTA exits. */
    int mixed_sweeps; /* mixed precision only: Jacobi sweeps before and after the coarse
                         correction on every level (0, default: the hierarchy's, 2 for the
                         reference's AmgView); the FP64 path always keeps the hierarchy's */
    double mixed_weight; /* mixed precision only: Jacobi weight (0, default: the hierarchy's,
                         0.7); flexible CG tolerates any fixed schedule, and the autotuner picks
                         the one with the shortest time to the tolerance */
    int tail_cluster; /* with tail_rows: run the tail as one thread-block cluster of this many CTAs
                         (2..16), its phases separated by the hardware cluster barrier; 0
                         (default): a cooperative grid with the bounded grid barrier */
    int vcycle_pair;  /* V-cycle kernels of SELL operators take two rows per thread per pass (1)
                         or one (0, default) */
    int krylov_stage; /* level-0 Krylov SpMV with the operator streamed through shared memory by
                         bulk copies, in this many buffers (2..4); 0 (default): loaded by the
                         threads (krylov_pair). Same results bit for bit. */
} cfdb_tuning;
void cfdb_default_tuning(cfdb_tuning* t);
int cfdb_system_set_tuning(cfdb_system* sys, const cfdb_tuning* t);

/* Stream of the system (cudaStream_t as void*), for callers that order their own work. */
int cfdb_system_stream(const cfdb_system* sys, void** stream);
/* Cells and internal faces of the system's pattern. */
int cfdb_system_sizes(const cfdb_system* sys, int* n_cells, int* n_faces);
/* Device bytes held by the system (pattern, hierarchy, work vectors). */
int cfdb_system_device_bytes(const cfdb_system* sys, size_t* bytes);

/* ---- batches: many independent pressure systems of uneven size in one device plan ----
 * (No counterpart in the reference, which solves systems one at a time through DeviceSolver.)
 * Every level of every system is concatenated into one set of arrays; each kernel launch of the
 * solve covers all systems (per-system convergence masks, per-system dot products), and the
 * whole iteration is one captured CUDA graph. Arrays are concatenated in system order: cells
 * of system 0, then system 1, ...; faces likewise; owner / neighbour hold LOCAL cell indices. */
typedef struct cfdb_batch cfdb_batch;
int cfdb_batch_create(int n_systems, const int* n_cells, const int* n_faces, const int* owner,
                      const int* neighbour, cfdb_batch** out);
int cfdb_batch_destroy(cfdb_batch* b);
int cfdb_batch_sizes(const cfdb_batch* b, long long* total_cells, long long* total_faces);
/* Hierarchies of all systems from host LDU arrays (AmgPreconditioner::setup per system,
 * systems in parallel on the host). */
int cfdb_batch_setup_amg(cfdb_batch* b, const double* diag, const double* upper,
                         const double* lower, const cfdb_amg_settings* settings);
/* The same hierarchies built on the device (the device setup of cfdb_amg_setup_device per
 * system, `concurrency` systems at a time on their own streams; 0: 8), bit-identical to
 * cfdb_batch_setup_amg. diag / upper / lower are device arrays. */
int cfdb_batch_setup_amg_device(cfdb_batch* b, const double* diag, const double* upper,
                                const double* lower, const cfdb_amg_settings* settings,
                                int concurrency);
int cfdb_batch_set_precision(cfdb_batch* b, int precision);
int cfdb_batch_set_tuning(cfdb_batch* b, const cfdb_tuning* t);
/* cfdb_system_assemble_pressure_device for every system (device arrays); ref_cell: host array
 * of per-system local reference cells (-1: none). */
int cfdb_batch_assemble_pressure_device(cfdb_batch* b, const double* flux, const double* gamma,
                                        const double* delta_coeff, const double* source0,
                                        const int* ref_cell, double ref_value, double* upper,
                                        double* lower, double* diag, double* source);
/* Solves every system (device arrays); x: initial guesses in, solutions out. controls and
 * stats: one per system (host arrays). use_amg = 0 runs Jacobi-preconditioned CG. */
int cfdb_batch_solve_device(cfdb_batch* b, const double* diag, const double* upper,
                            const double* lower, const double* rhs, double* x, int use_amg,
                            const cfdb_control* controls, cfdb_stats* stats);
int cfdb_batch_profile(cfdb_batch* b, int reps, cfdb_kernel_record* records, int max_records,
                       int* n_records);
int cfdb_batch_stream(const cfdb_batch* b, void** stream);
int cfdb_batch_device_bytes(const cfdb_batch* b, size_t* bytes);
/* Wall time of the last setup: the per-system hierarchies, then the batch plan built from them. */
int cfdb_batch_setup_times(const cfdb_batch* b, double* hierarchies_s, double* plan_s);
/* Phase times of the last plan build, "name=seconds;..." (as cfdb_system_setup_profile). */
int cfdb_batch_setup_profile(const cfdb_batch* b, char* buf, size_t len);
int cfdb_batch_kernel_launches(const cfdb_batch* b, unsigned long long* count);

/* ---- finite-volume cell kernels: cfd::gpu::DeviceFv (fv_device.hpp:33-72) ---- */
typedef enum { /* fv_geometry.hpp:31 GradientScheme */
    CFDB_GRAD_GAUSS = 0,
    CFDB_GRAD_LEAST_SQUARES = 1,
    CFDB_GRAD_GAUSS_CORRECTED = 2
} cfdb_gradient_scheme;
/* FvMeshView (fv_device.hpp:15-31): host arrays, copied to the device by cfdb_device_fv_create.
 * Faces [0, n_internal_faces) are internal; vectors are 3 doubles per entry (xyz). */
typedef struct {
    int n_cells;
    int n_internal_faces;
    int n_faces;
    const int* owner;          /* n_faces */
    const int* neighbour;      /* n_internal_faces */
    const int* cell_offsets;   /* n_cells + 1: faces of each cell (CSR) ... */
    const int* cell_faces;     /* ... in ascending face order */
    const double* weight;      /* n_internal_faces: phi_f = w phi_P + (1 - w) phi_N */
    const double* sf;          /* 3 n_faces: face area vectors */
    const double* face_centre; /* 3 n_faces */
    const double* cell_centre; /* 3 n_cells */
    const double* volume;      /* n_cells */
    const double* correction;  /* 3 n_faces: non-orthogonal correction vectors */
    const double* lsq_d;       /* 3 n_faces: d / |d|^2 (d = C_N - C_P or C_f - C_P) */
    const double* lsq_inverse; /* 9 n_cells: (sum d d^T / |d|^2)^-1, column-major */
} cfdb_fv_mesh_view;
typedef struct cfdb_device_fv cfdb_device_fv;
/* DeviceFv::DeviceFv: checks the sizes and that every array is present (fv_device.cpp:22-50)
 * and that every index stays in range, then keeps the mesh resident on the current device. */
int cfdb_device_fv_create(const cfdb_fv_mesh_view* view, cfdb_device_fv** out);
int cfdb_device_fv_destroy(cfdb_device_fv* fv);
int cfdb_device_fv_on_device(const cfdb_device_fv* fv); /* 1: there is no host path */
int cfdb_device_fv_device_bytes(const cfdb_device_fv* fv, size_t* bytes);
int cfdb_device_fv_stream(const cfdb_device_fv* fv, void** stream);
/* The four DeviceFv calls on HOST arrays, with the reference's semantics: grad (3 n_cells) of
 * phi (n_cells) with boundary face values bv (n_boundary); the vector gradient (9 n_cells,
 * grad[9 c + 3 i + j] = du_i / dx_j) of u (3 n_cells) with ub (3 n_boundary), kept on the
 * device for momentum_corrections; scalar and momentum explicit face corrections accumulated
 * into source (n_cells / 3 n_cells). momentum_corrections before a vector_gradient fails with
 * CFDB_ERR_NOT_READY; eps2 (3 values) is read only when venkat != 0. */
int cfdb_device_fv_gradient(cfdb_device_fv* fv, const double* phi, const double* bv, int scheme,
                            double* grad);
int cfdb_device_fv_vector_gradient(cfdb_device_fv* fv, const double* u, const double* ub,
                                   int scheme, double* grad);
int cfdb_device_fv_scalar_corrections(cfdb_device_fv* fv, const double* phi, const double* bv,
                                      int scheme, const double* flux, const double* gamma,
                                      int linear_upwind, double* source);
int cfdb_device_fv_momentum_corrections(cfdb_device_fv* fv, const double* flux,
                                        const double* nu_face, int linear_upwind, int limited,
                                        int venkat, const double* eps2, double central,
                                        int transpose_term, double* source);
/* The same on DEVICE arrays (no copies); momentum corrections take the field, its boundary
 * values and its vector gradient explicitly. Each returns when its kernels are done. */
int cfdb_device_fv_gradient_device(cfdb_device_fv* fv, const double* phi, const double* bv,
                                   int scheme, double* grad);
int cfdb_device_fv_vector_gradient_device(cfdb_device_fv* fv, const double* u, const double* ub,
                                          int scheme, double* grad);
int cfdb_device_fv_scalar_corrections_device(cfdb_device_fv* fv, const double* phi,
                                             const double* bv, int scheme, const double* flux,
                                             const double* gamma, int linear_upwind,
                                             double* source);
int cfdb_device_fv_momentum_corrections_device(cfdb_device_fv* fv, const double* u,
                                               const double* ub, const double* grad,
                                               const double* flux, const double* nu_face,
                                               int linear_upwind, int limited, int venkat,
                                               const double* eps2, double central,
                                               int transpose_term, double* source);

/* ---- the scalar transport equation on the device: solve_scalar's GPU path
 * (scalar_transport.cpp:50-176) up to a.solve, which is cfdb_system_solve_ldu ---- */
typedef enum { /* scalar_transport.hpp:14 ScalarBoundary::Kind */
    CFDB_SCALAR_FIXED_VALUE = 0,
    CFDB_SCALAR_ZERO_GRADIENT = 1,
    CFDB_SCALAR_FIXED_GRADIENT = 2,
    CFDB_SCALAR_MIXED = 3
} cfdb_scalar_bc_kind;
/* ScalarEquation (scalar_transport.hpp:24-37); every array on the device. */
typedef struct {
    const double* gamma_face;          /* n_faces: diffusivity */
    const double* su;                  /* n_cells: explicit source per unit volume */
    const double* sp;                  /* n_cells: implicit source coefficient */
    const int* bc_kind;                /* n_boundary: cfdb_scalar_bc_kind */
    const double* bc_value;            /* n_boundary */
    const double* bc_coefficient;      /* n_boundary: Mixed h / gamma */
    const unsigned char* fixed_cell;   /* optional n_cells: 1 = value fixed */
    const double* fixed_value;         /* with fixed_cell */
    double relaxation;                 /* implicit under-relaxation (1: none) */
    double dt;                         /* > 0: implicit Euler with old_value (else the field) */
    const double* old_value;           /* optional */
    const double* capacity;            /* optional factor of the time term */
    int linear_upwind;
    int gradient;                      /* cfdb_gradient_scheme of the explicit corrections */
} cfdb_scalar_equation;
/* FvGeometry's delta coefficients (n_faces), unit normals (3 n_faces) and face areas (n_faces)
 * (fv_geometry.cpp:33-50), host arrays copied to the device, for the scalar equation. */
int cfdb_device_fv_set_face_geometry(cfdb_device_fv* fv, const double* delta_coeffs,
                                     const double* unit_normals, const double* face_areas);
/* The LDU system of solve_scalar on device arrays: boundary values of field, the explicit
 * face corrections, the convection-diffusion coefficients (convection 1), boundary-face terms,
 * sources, time term, under-relaxation and fixed cells (field takes the fixed values). upper /
 * lower: internal faces; diag, source: cells. Bit-identical to the face-by-face host loops. */
int cfdb_device_fv_scalar_system_device(cfdb_device_fv* fv, const cfdb_scalar_equation* eq,
                                        const double* face_flux, double* field, double* upper,
                                        double* lower, double* diag, double* source);

#ifdef __cplusplus
}
#endif
#endif
