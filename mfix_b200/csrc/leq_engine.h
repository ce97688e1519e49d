// leq_engine.h -- host-side solver engine: batches of MFIX 7-point systems,
// device-resident state, the BiCGSTAB iteration schedule (FP64 drop-in and the
// FP32-inner / FP64-refinement form) and the LINE-preconditioner sweep plan.
#pragma once
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "leq_common.cuh"
#include "leq_kernels.cuh"

namespace mfixgpu {

enum Precision : int { PREC_FP64 = 0, PREC_MIXED = 1 };

// One system to solve.  Pointers are host or device memory as the call says.
struct SystemSpec {
    int imax2 = 0, jmax2 = 0, kmax2 = 0, do_k = 1;
    int cyc = 0;          // cyclic axes: 1 I (CYCLIC_X), 2 J (CYCLIC_Y), 4 K (CYCLIC_Z)
    int64_t n = 0;
    double *a = nullptr;  // 7*n, A_M(DIMENSION_3,-3:3) layout
    double *b = nullptr;  // n
    double *x = nullptr;  // n, initial guess in / solution out
    double tol = 1e-8;
    int itmax = 500;
};

// The kernels read A_M, B_M and VAR two cells at a time (16-byte loads).
inline bool aligned16(const SystemSpec &s)
{
    return !(((uintptr_t)s.a | (uintptr_t)s.b | (uintptr_t)s.x) & 15);
}

struct SolveResult {
    int ier = 0;
    int iterations = 0;    // reference ITER counter (mixed: inner iterations)
    int iter_tot_add = 0;  // contribution to ITER_TOT(VNO)
    int exit_kind = 0;
    int line_skips = 0;
    int line_fallbacks = 0;
    int outer_steps = 0;
    int fp64_fallback = 0;     // mixed form handed the system to an FP64 re-solve
    int mixed_iterations = 0;  // FP32 iterations spent before that hand-over
    int deflated = 0;          // mixed form: the near-null mode was deflated (near-singular operator)
    double rnorm0 = 0.0, rnorm = 0.0;
};

struct SolveOptions {
    int method = 2;              // LEQ_METHOD: 2 BiCGSTAB (model/leq_bicgs.f), 3 GMRES (model/leq_gmres.f),
                                 // 4 BiCGSTAB then GMRES on breakdown, 5 CG (model/leq_cg.f); 3-5 in FP64
    int pc = PC_LINE;
    char sweep[4] = {'R', 'S', 'R', 'S'};
    int precision = PREC_FP64;
    bool on_device = false;      // a/b/x are device pointers (solved in place)
    bool write_back_ab = true;   // copy the unit-scaled A/B back to host arrays
    uint64_t seed = 0x5EEDULL;   // Rtilde stream
    double inner_tol = 1e-2;     // mixed form: residual drop between reliable updates
    double mixed_growth = 10.0;  // mixed form: true-residual growth over the best that hands over to FP64
    int mixed_stalls = 6;        // mixed form: reliable updates without a 10% gain that hand over
    double mixed_min_margin = 1e-4;  // mixed form: smaller diagonal-dominance margins are deflated (or go to FP64)
    bool deflate = true;         // mixed form: deflate the near-null mode of systems below mixed_min_margin
                                 // (false: they go straight to the FP64 drop-in)
    int replace_every = 20;      // mixed form, deflated systems: FP64 residual replacement interval (0: off)
    double restart_growth = 100.0;  // mixed form, deflated systems: Krylov restart on this true-residual growth (0: off)
    int minimize_dotproducts = 0;   // FP64 BiCGSTAB: MINIMIZE_DOTPRODUCTS (no Snorm exit, Rnorm every icheck_bicgs)
    int icheck_bicgs = 1;           // ICHECK_BICGS
    int staged_matvec = 2;       // mixed form: matvecs with operands staged by bulk copies (1: with x's
                                 // line / plane windows; 0: register loads)
    bool transposed = false;     // DO_TRANSPOSE (model/solve_lin_eq.f:139-150): LEQ_BICGSt's preconditioner
                                 // letters, and A is scaled in a copy (only B comes back scaled)
    int check_every = 4;         // iterations between host checks of the state
    bool use_graph = true;       // capture the iteration body in a CUDA graph
    bool time_kernels = false;   // record events around every J-line launch (no graph replay)
    bool skip_scale = false;     // the system is unit-scaled already (FP64 re-solve after a mixed attempt)
    bool autotune = true;        // pick lanes per J-line by measurement for unseen line lengths
    int force_lanes = 0;         // > 0: lanes per J-line for every system (experiments)
};

// Kernel classes timed one by one with option time_kernels.
enum KernelClass : int {
    KC_JLINE = 0,     // LINE preconditioner half-sweep (J-line solves)
    KC_P_UPDATE,      // P = R + beta (P - omega V)
    KC_MATVEC_ALPHA,  // V = A Phat, alpha
    KC_S_UPDATE,      // S = R - alpha V, Snorm
    KC_MATVEC_OMEGA,  // T = A Shat, omega
    KC_XR_UPDATE,     // X, R, Rnorm, rho
    KC_OUTER,         // mixed form: FP64 reliable update
    KC_OTHER,         // copies, DIAG, sequential line sweeps
    KC_COUNT
};

// Device-side timing of the last solve (CUDA events on the engine's stream).
struct SolveTiming {
    float device_ms = 0.f;    // setup + iterations, inputs already on the device
    float jline_ms = 0.f;     // sum over J-line launches (time_kernels only)
    int jline_launches = 0;
    long long kernel_launches = 0;  // kernels of this library launched by the solve
    float class_ms[KC_COUNT] = {};  // time_kernels only: summed launch durations per class
    int class_launches[KC_COUNT] = {};
};

// Host table -> device copy; the device array is reallocated (with headroom)
// only when it must grow.  cudaFree waits for the kernels still using it.
template <typename T>
inline cudaError_t upload(T **dptr, size_t *cap_elems, const T *src, size_t n, cudaStream_t s)
{
    if (n > *cap_elems || *dptr == nullptr) {
        if (*dptr) cudaFree(*dptr);
        *dptr = nullptr;
        const size_t want = std::max<size_t>(n + n / 2, 16);
        cudaError_t e = cudaMalloc((void **)dptr, want * sizeof(T));
        if (e != cudaSuccess) return e;
        *cap_elems = want;
    }
    if (n == 0) return cudaSuccess;
    return cudaMemcpyAsync(*dptr, src, n * sizeof(T), cudaMemcpyHostToDevice, s);
}

// A system joining a live batch: device arrays (a/b/x of `dev`) and a work
// block of live_work_bytes(); the caller keeps both until the system has left.
struct LiveSystem {
    SystemSpec dev;
    char *work = nullptr;
    bool scaled = false;      // A/B unit-scaled already: the setup starts after the scaling
    const double *x0 = nullptr;  // non-null: x = x0 before the setup (FP64 re-solve of a mixed attempt)
    cudaEvent_t after = nullptr; // non-null: the engine's stream waits for it before touching the system
    char *x0_slot = nullptr;     // mixed form: where the initial guess is kept (default: after the FP64 region)
};

struct LiveDone {
    int slot;
    SolveResult res;
};

struct DeviceArena {
    char *base = nullptr;
    size_t cap = 0, used = 0;
    void *take(size_t bytes);
    void reset() { used = 0; }
    cudaError_t reserve(size_t bytes);
    void release();
};

class Engine {
public:
    Engine();
    ~Engine();
    // Solve a batch.  Returns 0 or a negative error code; per-system IER in out.
    int solve(const std::vector<SystemSpec> &specs, const SolveOptions &opt, std::vector<SolveResult> &out);
    const std::string &last_error() const { return err_; }
    int device() const { return dev_; }
    int sm_count() const { return sms_; }
    cudaStream_t stream() const { return stream_; }
    size_t arena_bytes() const { return arena_.cap; }
    const SolveTiming &timing() const { return timing_; }

    // ---- live batch: a fixed table of slots whose systems join and leave
    // between iterations (continuous batching).  Every system follows the same
    // kernel sequence as when solved alone: setup, then one body per iteration.
    int live_open(int capacity, const SolveOptions &opt);
    int live_add(const LiveSystem &s);  // slot, or MFIXGPU_ERR_NOMEM-style -11 when full
    void live_remove(int slot);         // the slot's system takes no further part
    // Applies joins and leaves (tables, graph, setup of new systems), then runs
    // `iterations` bodies and records a snapshot of the states.
    int live_step(int iterations);
    // Systems found finished in the previous snapshot (latest: the newest one,
    // waited for); each is reported once.
    int live_collect(std::vector<LiveDone> &done, bool latest);
    // The oldest unread snapshot, if it is complete (never waits); *collected says
    // whether one was read.  Snapshots are read in order.
    int live_collect_ready(std::vector<LiveDone> &done, bool *collected);
    // snapshots recorded and not read yet (chunks whose results are pending)
    int live_inflight() const { return (int)(snap_count_ - 1 - collected_upto_); }
    int live_used() const { return live_used_; }
    int live_capacity() const { return (int)slot_used_.size(); }
    bool live_dirty() const { return live_dirty_; }
    // Recorded after the last commit: kernels enqueued before it may still read
    // the tables of systems removed by that commit, none after it.
    cudaEvent_t live_fence() const { return ev_fence_; }
    long long live_commits() const { return commits_; }
    long long live_bodies() const { return body_total_; }
    double live_busy_ms() const { return busy_ms_; }  // device time of the collected chunks (commits included)
    long long launches() const { return launches_; }

    // per-routine entry points on device pointers (parity tests of single kernels)
    int matvec(const SystemSpec &g, const double *a, const double *x, double *y);
    int msolve(const SystemSpec &g, const double *a, const double *b, double *var, int pc, const char sweep[4]);
    int dot(const double *x, const double *y, int64_t n, double *out_host);

private:
    int run_batch(const std::vector<SystemSpec> &specs, const SolveOptions &opt, std::vector<SolveResult> &out);
    int run_batch_live(const std::vector<SystemSpec> &specs, const SolveOptions &opt, std::vector<SolveResult> &out);
    int run_gmres(const SystemSpec &s, const SolveOptions &opt, SolveResult &out);
    std::vector<double *> x0_;  // per system of the last batch: the mixed form's copy of the initial guess
    int launch_setup(const SolveOptions &opt, bool scale);
    int launch_body(const SolveOptions &opt);
    int setup_batch(const std::vector<SystemSpec> &specs, const SolveOptions &opt);
    int plan_msolve(const SolveOptions &opt, int src, int dst, int gate, int elem);
    int run_msolve_plan(int which, int elem);
    int bind_lists();
    int configure_lines(int elem, int only_L = 0);
    std::vector<int> tune_lengths_;  // configure_lines(elem, -1): the line lengths being tuned
    void shape_for(int L, int elem, int forced, int *G, int *c, int *kind);
    int autotune_lines(const SolveOptions &opt, int elem);
    void save_tune_cache();

public:
    void load_tune_cache(const std::string &path);
    int tune_table(int *out, int max_entries) const;

private:
    int fail(const std::string &msg, int code);

    int dev_ = -1, sms_ = 0;
    CellOcc occ_[2] = {};  // resident blocks per SM of each cell kernel, [fp32]
    cudaStream_t stream_ = nullptr;
    // Copy-back of the unit-scaled A/B to host arrays: A and B are final once
    // the setup has scaled them, so the copies run on a side stream during the
    // iterations.
    struct Writeback {
        void *dst;
        const void *src;
        size_t bytes;
    };
    std::vector<Writeback> writeback_;
    cudaStream_t side_ = nullptr;
    cudaEvent_t ev_setup_ = nullptr;
    int issue_writeback();
    cudaEvent_t ev_a_ = nullptr, ev_b_ = nullptr, ev_t0_ = nullptr, ev_t1_ = nullptr;
    DeviceArena arena_;     // iteration vectors and other per-solve work memory
    DeviceArena in_arena_;  // device copies of host inputs (A_M, B_M, VAR)
    std::string err_;

    // Table uploads go through a ring of pinned staging buffers: a copy from
    // pageable memory would first wait for the stream to drain, which idles the
    // GPU while a live batch's host work runs.  A buffer is reused after the
    // event recorded behind its copies.
    static constexpr int STAGES = 4;
    char *stage_buf_[STAGES] = {};
    size_t stage_cap_[STAGES] = {}, stage_used_ = 0;
    cudaEvent_t stage_ev_[STAGES] = {};
    int stage_cur_ = 0;
    cudaError_t stage_open(size_t bytes);
    cudaError_t stage_close();
    template <typename T>
    cudaError_t stage_copy(T *dst, const T *src, size_t n)
    {
        if (n == 0) return cudaSuccess;
        const size_t off = (stage_used_ + 63) / 64 * 64, bytes = n * sizeof(T);
        if (off + bytes > stage_cap_[stage_cur_])  // not foreseen by stage_open: a plain copy
            return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream_);
        std::memcpy(stage_buf_[stage_cur_] + off, src, bytes);
        stage_used_ = off + bytes;
        return cudaMemcpyAsync(dst, stage_buf_[stage_cur_] + off, bytes, cudaMemcpyHostToDevice, stream_);
    }
    template <typename T>
    cudaError_t upload_staged(T **dptr, size_t *cap_elems, const T *src, size_t n)
    {
        if (n > *cap_elems || *dptr == nullptr) {
            if (*dptr) cudaFree(*dptr);
            *dptr = nullptr;
            const size_t want = std::max<size_t>(n + n / 2, 16);
            cudaError_t e = cudaMalloc((void **)dptr, want * sizeof(T));
            if (e != cudaSuccess) return e;
            *cap_elems = want;
        }
        return stage_copy(*dptr, src, n);
    }

    // batch tables (host mirrors + device copies)
    int nsys_ = 0;
    std::vector<SysDev> h_sys_;
    std::vector<SysState> h_st_;
    std::vector<Tile> h_tiles_;
    std::vector<int> h_prefix_;
    std::vector<int> h_allprefix_;  // all J-lines of each system (factorization kernel)
    SysDev *d_sys_ = nullptr;
    SysState *d_st_ = nullptr;
    Tile *d_tiles_ = nullptr;
    int *d_prefix_ = nullptr;
    int *d_line_sys_ = nullptr;  // system of each parity-wave work item
    std::vector<int> h_line_sys_;
    size_t line_sys_cap_ = 0;
    int *d_allprefix_ = nullptr;
    double *d_partials_ = nullptr;
    SysState *h_st_pinned_ = nullptr;  // state snapshots: pinned, mapped host memory
    SysState *d_st_mapped_ = nullptr;  // the same memory as the kernels address it
    size_t h_st_pinned_cap_ = 0;
    int reserve_snapshots(size_t entries);  // (re)allocates h_st_pinned_ for `entries` states
    BatchView view_{};
    LaunchCfg cfg_{};

    // sweep plans: [0] for P -> Phat, [1] for S -> Shat
    struct Step {
        int type;  // 0 J-line wave, 1 copy, 2 sequential line list
        WaveArgs w;
        SeqLineArgs s;
    };
    std::vector<Step> plan_[2];
    int2 *d_lines_ = nullptr;
    size_t d_lines_cap_ = 0;
    double *d_seq_scratch_ = nullptr;
    size_t d_seq_scratch_cap_ = 0;
    std::vector<int2> h_lines_;
    struct ListRef {
        int which;
        size_t index, offset;
    };
    std::vector<ListRef> list_refs_;

    // standalone kernels
    SysDev *d_one_sys_ = nullptr;
    double *d_dot_partials_ = nullptr;
    double *gm_basis_ = nullptr;  // GMRES Krylov basis, (ITMAX+1) x DIMENSION_3
    size_t gm_basis_bytes_ = 0;
    double *gm_scal_ = nullptr;   // GMRES: block partials, then the current Hessenberg column and y
    int gm_scal_cap_ = 0;
    unsigned long long *gm_max_ = nullptr;
    unsigned int *d_dot_counter_ = nullptr;
    double *d_dot_out_ = nullptr;
    size_t sys_cap_ = 0, st_cap_ = 0, tiles_cap_ = 0, prefix_cap_ = 0, part_cap_ = 0, allprefix_cap_ = 0;
    // time_kernels: an event pair around every launch of the iteration body
    bool ktime_ = false;
    static constexpr int KT_MAX = 1 << 16;
    std::vector<cudaEvent_t> kt_ev_;  // 2 per timed launch, created on first use
    std::vector<int> kt_class_;
    int kt_count_ = 0;
    void kt_begin();
    void kt_end(int kclass);
    void kt_harvest();
    long long launches_ = 0;
    SolveTiming timing_;

    // live batch
    int live_commit();
    int live_take(long long q, std::vector<LiveDone> &done);
    SolveOptions live_opt_{};
    std::vector<char> slot_used_, slot_fresh_, slot_reported_, slot_cleared_;
    std::vector<LiveSystem> slot_sys_;
    std::vector<long long> slot_join_snap_, slot_join_body_;
    int live_used_ = 0;
    bool live_dirty_ = false;
    bool live_tune_ = false;  // autotune new line lengths at the next commit
    cudaGraphExec_t live_exec_ = nullptr;
    // replaced body graphs, destroyed once a snapshot taken after their last launch has been read
    std::vector<std::pair<cudaGraphExec_t, long long>> retired_execs_;
    long long live_per_body_ = 0;
    long long snap_count_ = 0, body_total_ = 0, collected_upto_ = -1, commits_ = 0;
    long long snap_bodies_[2] = {0, 0};
    cudaEvent_t ev_c0_[2] = {}, ev_c1_[2] = {};  // around each chunk (commit + iterations)
    double busy_ms_ = 0.0;
    cudaEvent_t ev_fence_ = nullptr;
};

SolveResult result_of(const SysState &st, bool mixed);

// choice of lanes per J-line and rows per lane for a line of length L
void line_shape(int L, int *G, int *c);

// Work memory of one system with n cells and `lines` J-lines: the iteration
// vectors and factors of the given precision, plus the initial-guess copy of
// the mixed form (work_bytes); live_work_bytes also leaves room for an FP64
// re-solve of a mixed attempt in the same block.
size_t vec_region_bytes(int64_t n, int64_t lines, int precision);
// Line pitch and cells of the arrays in a form's precision (the mixed form pads
// each J-line of its FP32 arrays to a multiple of four cells).
int form_pitch(int jmax2, int precision);
int64_t form_cells(int64_t n, int64_t lines, int precision);
size_t work_bytes(int64_t n, int64_t lines, int precision);
size_t live_work_bytes(int64_t n, int64_t lines, int precision);
// Points d's work arrays into `work` (d.n and d.x64[0] set); x0: where the
// mixed form keeps the initial guess.
void carve_work(SysDev &d, char *work, int64_t lines, int precision, char *x0);

}  // namespace mfixgpu
