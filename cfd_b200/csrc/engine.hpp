// Solver engine: one plan over a batch of independent pressure systems (a single solve is a
// batch of one). Owns the device hierarchy in SELL-32, the Krylov vectors, per-system state
// and the captured CUDA graphs of the iteration.
#pragma once

#include <memory>
#include <vector>

#include "common.hpp"
#include "dsetup.hpp"
#include "host_algos.hpp"
#include "kernels.cuh"

namespace cfdb {

enum class Mode { AmgFp64 = 0, AmgMixed = 1, Jacobi = 2 };

struct SystemSpec {
    int n = 0;                        // level-0 rows
    const int* rp = nullptr;          // level-0 CSR pattern (host, sorted columns)
    const int* ci = nullptr;
    std::vector<int> src;             // per pattern entry: index into this system's value source
    std::vector<int> diag_src;        // per row: value-source index of the diagonal, or -1
    // the same maps owned by the caller (used instead of src / diag_src when set; no copy)
    const std::vector<int>* src_ref = nullptr;
    const std::vector<int>* diag_src_ref = nullptr;
    // identifies the pattern and value maps (0: unknown); equal ids mean equal level-0 layouts
    long long layout_id = 0;
    int vs_len = 0;                   // length of this system's value source
    bool absolute_src = false;        // src already indexes the batch-wide value source
    std::shared_ptr<const Hierarchy> h; // levels >= 1, transfers, coarse inverse (null: none)
    // Device-resident levels (single-system plans): when set, h holds only the shapes and the
    // coarse inverse, and the operators of levels >= 1 are laid out on the device from dl.
    std::shared_ptr<const DeviceLevels> dl;
};

// Launch-shape and schedule knobs (no effect on the arithmetic of a row sum except that wide
// operators switch between the ordered SELL sum and the lane-group CSR sum).
struct Tuning {
    int target_tiles = 148 * 8; // level-0 Krylov tiles: about this many (0: 256 rows each)
    int wide_row = 48;          // average row length above which CSR lane groups are used
    int lanes_div = 16;         // lanes per CSR row ~ average row length / lanes_div (4..256),
                                // and at least enough lanes to give ~150K threads per operator
    int fuse_first = 0;         // first two smoothing sweeps in one kernel (x1 recomputed)
    int sell_rows = kSellRows;  // rows per CTA of SELL operators (multiple of kSellRows)
    int krylov_pair = 1;        // level-0 Krylov SpMV kernels: two rows per thread per pass
    int col16 = 0;              // FP32 operators store 16-bit column offsets where they fit
    int tail_rows = 0;          // coarse levels of at most this many rows (and everything below
                                // them) run as one persistent tail kernel; 0 disables it
    int pdl = 1;                // programmatic dependent launch between consecutive kernels
    int wait_polls = 1 << 22;   // poll limit of the bounded device waits (< 0: give up at once)
    int mixed_sweeps = 0;       // mixed precision: Jacobi sweeps per level (0: the hierarchy's)
    double mixed_weight = 0.0;  // mixed precision: Jacobi weight (0: the hierarchy's)
    int tail_cluster = 0;       // the tail as one thread-block cluster of this many CTAs (2..16)
                                // separated by the cluster barrier; 0: a cooperative grid
    int vcycle_pair = 0;        // V-cycle kernels of SELL operators take two rows per thread per
                                // pass (as the level-0 Krylov kernels with krylov_pair), or one
    int krylov_stage = 0;       // level-0 Krylov SpMV with the operator staged through shared
                                // memory in this many buffers (2..4); 0: krylov_pair's kernels
};

struct SolveRequest {
    double tol = 1e-10;
    int max_it = 1000;
};

// One profiled kernel launch: algorithmic bytes and average device time.
struct ProfRecord {
    char name[32];
    int level;
    double ms;
    double bytes;
};

struct SolveResult {
    int iterations = 0;
    double residual = 0.0;
    bool converged = false;
    double true_residual = 0.0;
};

class Engine {
public:
    explicit Engine(int device);
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    // Builds the device plan. need64 / need32: keep FP64 / FP32 copies of the V-cycle levels.
    void build(std::vector<SystemSpec> systems, int sweeps, double weight, bool need64,
               bool need32);
    [[nodiscard]] bool built() const { return n_sys_ > 0; }
    [[nodiscard]] int n_systems() const { return n_sys_; }
    [[nodiscard]] bool has_amg() const { return has_amg_; }
    [[nodiscard]] bool has32() const { return need32_; }
    [[nodiscard]] bool has64() const { return need64_; }
    [[nodiscard]] size_t device_bytes() const { return arena_.bytes() + arena0_.bytes(); }
    [[nodiscard]] cudaStream_t stream() const { return stream_; }
    StagedCopier& copier() { return copier_; }
    [[nodiscard]] int device() const { return device_; }
    [[nodiscard]] int levels() const { return n_levels_; }
    [[nodiscard]] int level_rows(int l) const;
    [[nodiscard]] long long level_slots(int l) const;

    // Level-0 values from a value source. For one system: three device arrays (diag, upper,
    // lower) addressed by the source indices [0,n1) [n1,n2) [n2,..). upload_values copies a host
    // value source (concatenated per system in batch order) first.
    void set_values_device(const double* p0, const double* p1, const double* p2, int n1, int n2);
    void upload_values(const std::vector<const double*>& host_src);
    // Single system: LDU values straight from the caller's host arrays (no staging copy).
    void upload_values_ldu(const double* diag, const double* upper, const double* lower, int n, int nf);
    void upload_values_device_concat(const std::vector<const double*>& dev_src);

    // Right-hand side / initial guess of system s (original batch index), host or device.
    void set_rhs(int s, const double* b, bool device_ptr);
    void set_guess(int s, const double* x, bool device_ptr);
    void get_solution(int s, double* x, bool device_ptr);

    // Runs the solve for all systems on the engine stream; blocks until done.
    std::vector<SolveResult> solve(Mode mode, const std::vector<SolveRequest>& req);
    // Jacobi-preconditioned BiCGStab on the level-0 operator (single-system plans; bicgstab.cu).
    SolveResult solve_bicgstab(const SolveRequest& req);

    // Launch the pieces of one V-cycle application z = M^-1 r for system-batch inputs that are
    // already in the level-0 residual vector (used by the parity tests).
    void apply_vcycle(Mode mode, const std::vector<int>& sys_rhs_ready);
    void set_residual(int s, const double* r, bool device_ptr);
    void get_precond(int s, double* z, bool device_ptr, Mode mode);

    // Kernel timing probe: average device time (ms) of the level-0 FP64/FP32 smoother sweep.
    double time_level0_sweep(bool fp32, int reps);
    // Average device time (ms) of `reps` back-to-back Jacobi sweeps of level l in the plan's
    // precision and launch shape (level 0 reads the Krylov residual); *bytes = algorithmic bytes
    // of one sweep (operator, weights, right-hand side, iterate in and out).
    double time_sweep(int level, int reps, double* bytes);

    // Runs the initial preconditioning and one full iteration eagerly with CUDA events around
    // every kernel (all systems kept active); returns per-kernel device time averaged over reps
    // (the first repetition is a warm-up when reps > 1) with the algorithmic bytes of each.
    std::vector<ProfRecord> profile(Mode mode, int reps);

    // Ordered mode: every operator in SELL with thread-per-row sums in CSR order, so FP64
    // V-cycles are bit-identical to the reference's sequential host arithmetic. Takes effect
    // at the next build().
    void set_ordered(bool on) { ordered_ = on; }
    void set_tuning(const Tuning& t) { tuning_ = t; }
    [[nodiscard]] const Tuning& tuning() const { return tuning_; }

    // Batch vectors in the caller's order (systems concatenated, no padding), device arrays:
    // gathers b and the initial guess (x0 == nullptr: zero) into the engine layout, scatters
    // the solution back.
    void set_rhs_guess_concat(const double* b, const double* x0);
    void get_solution_concat(double* x);
    [[nodiscard]] long long user_rows() const { return user_rows_; }
    // Kernels launched by this engine so far (graph kernel nodes counted per graph launch).
    [[nodiscard]] unsigned long long kernel_launches() const { return launches_; }
    [[nodiscard]] bool ordered() const { return ordered_; }
    // wall-clock seconds of the phases of the last build()
    [[nodiscard]] const PhaseTimes& build_times() const { return build_times_; }

private:
    struct DevSell64_32 {
        Sell<double> s64{};
        Sell<float> s32{};
        int n_slices = 0;     // SELL slices, or CSR rows
        long long slots = 0;  // stored entries (SELL: with padding)
        long long nnz = 0;    // algorithmic nonzeros
        int max8_slots = 0;   // SELL: most slots of any 8 consecutive slices (a staged chunk)
        // launch tiles of the operator's own row space: kSellRows rows (SELL), 8 rows (CSR,
        // G <= 32) or 256 / G rows (CSR, G > 32); block = threads per CTA
        Tiles tiles{};
        int n_tiles = 0;
        int n_tiles_nc = 0;   // tiles of systems that continue to a coarser level
        int block = kBlock;
    };
    struct DevLevel {
        int n_rows = 0;     // all present systems (padded)
        int n_rows_nc = 0;  // prefix of systems that continue to a coarser level
        int n_tiles = 0;
        int n_tiles_nc = 0;
        Tiles tiles{};       // runs of whole slices (the reductions of the Krylov kernels)
        DevSell64_32 a, p, r;
        double* wd64 = nullptr;
        float* wd32 = nullptr;
        double *x64 = nullptr, *y64 = nullptr, *t64 = nullptr, *b64 = nullptr;
        float *x32 = nullptr, *y32 = nullptr, *t32 = nullptr, *b32 = nullptr;
        int final_in_y = 0; // after post-smoothing the iterate lives in y
    };

    void capture_graphs(Mode mode);
    // x1_ready0: the level-0 first pre-smoothing sweep was written by the residual producer
    void enqueue_vcycle(Mode mode, bool fused_final, int flexible, bool x1_ready0);
    template <class T> void enqueue_vcycle_t(bool fused_final, int flexible, bool x1_ready0);
    template <class T> T* start_buffer(int l) const;
    // V-cycle tail (small coarse levels in one persistent kernel): first level, phases
    int tail_level() const;
    // staged level-0 Krylov SpMV (Tuning.krylov_stage): buffer size in slots, 0 when off
    void prepare_stage();
    template <class T> void prepare_tail();
    template <class T> void launch_tail(cudaStream_t s);
    // rows per thread per pass of the level-0 Krylov SpMV kernels (two, or one)
    int krylov_visit() const { return tuning_.krylov_pair ? kVisitSell2 : kVisitSell1; }
    // row-visiting strategy of a V-cycle operator's kernels
    int vcycle_visit(const DevSell64_32& m) const {
        const int v = visit_of(m.s64.val != nullptr ? m.s64.fmt : m.s32.fmt);
        return v == kVisitSell1 && tuning_.vcycle_pair ? kVisitSell2 : v;
    }
    // where the residual producers of `mode` write the level-0 first sweep (n = 0: nowhere)
    X1Out x1_out(Mode mode) const;
    void enqueue_init(Mode mode);
    void enqueue_iteration(Mode mode);
    void enqueue_rz(Mode mode, int flexible);
    void mark(const char* name, int level, double bytes);
    void release_graphs();

    int device_;
    cudaStream_t stream_ = nullptr;
    StagedCopier copier_; // host-array uploads and downloads
    DeviceArena arena_;
    int n_sys_ = 0;
    int n_levels_ = 0;
    int sweeps_ = 2;
    double weight_ = 0.7;
    bool need64_ = true;
    bool need32_ = false;
    bool has_amg_ = false;
    bool fused_final_ = true;
    bool ordered_ = false;
    Tuning tuning_{};
    int* row_map_ = nullptr;       // per level-0 row: index in the caller's concatenated vectors, -1 padding
    long long user_rows_ = 0;
    std::vector<std::pair<ProfRecord, cudaEvent_t>>* prof_ = nullptr;
    double coarse_bytes_ = 0.0, coarse_rows_ = 0.0;

    // batch order: perm_[k] = original index of the k-th system (sorted by level count)
    std::vector<int> perm_, rank_;
    std::vector<int> n_of_;          // level-0 rows per original system
    std::vector<int> off0_;          // level-0 row offset per original system
    std::vector<int> vs_off_;        // value-source offset per original system (batch order)
    int vs_total_ = 0;
    std::vector<DevLevel> lv_;
    // level-0 value map
    int* src0_ = nullptr;
    int* diag_src0_ = nullptr;
    double* vs_ = nullptr;
    double* dinv0_ = nullptr;
    double* bcg_ = nullptr;  // BiCGStab work vectors (allocated on first use)
    // Krylov vectors (level 0)
    double *b_ = nullptr, *x_ = nullptr, *r_ = nullptr, *p_ = nullptr, *q_ = nullptr;
    // state
    SysState* st_ = nullptr;
    Reduce red_{};
    int* n_active_ = nullptr;
    int* error_ = nullptr;
    int* h_pinned_ = nullptr; // [0] n_active, [1] error
    // coarse blocks
    int n_blocks_ = 0;
    int n_single_ = 0;        // systems whose hierarchy has one level (Jacobi-preconditioned CG)
    std::vector<int> single_; // per original system: 1 if its hierarchy has one level
    int n_ctiles_ = 0;        // coarse-solve tiles
    // persistent tail: phase lists per precision (device), barrier words
    TailPhase<float>* tail32_ = nullptr;
    TailPhase<double>* tail64_ = nullptr;
    int tail_n32_ = 0, tail_n64_ = 0, tail_grid32_ = 0, tail_grid64_ = 0;
    int stage_cap_ = 0;
    double tail_bytes32_ = 0.0, tail_bytes64_ = 0.0;
    unsigned* tail_bar_ = nullptr;
    CoarseBlocks cb_{};
    int* block_level_ = nullptr;
    double** b_level64_ = nullptr;
    double** x_level64_ = nullptr;
    float** b_level32_ = nullptr;
    float** x_level32_ = nullptr;
    size_t coarse_smem64_ = 0, coarse_smem32_ = 0;
    // graphs per mode: [mode][0] init, [mode][1] iteration
    cudaGraphExec_t graphs_[3][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};
    int graph_kernels_[3][2] = {{0, 0}, {0, 0}, {0, 0}};
    unsigned long long launches_ = 0;
    PhaseTimes build_times_;
    // level-0 layout kept across builds of a single-system plan over the same pattern
    struct L0Key {
        int n_sys = 0;
        const int* rp = nullptr;
        const int* ci = nullptr;
        int n = 0, nnz = 0, vs_len = 0;
        bool absolute_src = false;
        long long map_hash = 0;
        bool need32 = false, col16 = false;
        bool operator==(const L0Key& o) const {
            return n_sys == o.n_sys && rp == o.rp && ci == o.ci && n == o.n && nnz == o.nnz && vs_len == o.vs_len &&
                   absolute_src == o.absolute_src && map_hash == o.map_hash && need32 == o.need32 && col16 == o.col16;
        }
    };
    struct L0Cache {
        DevSell64_32 a;
        double* wd64;
        float* wd32;
        int* src0;
        int* diag_src0;
        int* row_map;
        double* dinv0;
        long long user_rows;
    };
    DeviceArena arena0_;
    L0Key l0_key_{};
    L0Cache l0_{};
    bool l0_valid_ = false;
};

} // namespace cfdb
