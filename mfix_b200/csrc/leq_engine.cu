// leq_engine.cu -- host engine of the B200 LEQ_BICGS path.
//
// One Engine per device: an arena of device memory grown on demand and reused
// across calls (the reference allocates and frees its eight work vectors inside
// every call, model/leq_bicgs.f:238-245, 499-506), one stream, batch tables.
// The iteration body is a fixed sequence of kernels that read every scalar from
// device memory, so it is captured once per solve into a CUDA graph and replayed;
// the host reads the per-system state back every few iterations, double
// buffered, to stop once every system is done.
#include "leq_engine.h"

#include <algorithm>
#include <cstring>
#include <cstdio>
#include <map>

namespace mfixgpu {

#define CK(call)                                                                  \
    do {                                                                          \
        cudaError_t e_ = (call);                                                  \
        if (e_ != cudaSuccess) return fail(std::string(#call) + ": " + cudaGetErrorString(e_), -13); \
    } while (0)

static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// The autotuner's choices are shared by every engine of the process (one-shot
// solves and live batches pick the same lanes per line for the same line length,
// so a system gives the same bits in either).
namespace {
struct TuneTable {
    std::mutex mu;
    std::map<std::pair<int, int>, int> lanes;  // (element bytes, line length) -> lanes per line
    std::string path;
};
TuneTable &tunes()
{
    static TuneTable t;
    return t;
}
}  // namespace

// Lanes per J-line: the smallest power of two that leaves at most 12 rows per
// lane (at most 32 lanes); rows per lane rounded up to odd so that lanes reading row t
// of their chunks hit distinct shared-memory banks.
void line_shape(int L, int *G, int *c)
{
    int g = 1;
    while (g < 32 && g * 12 < L) g *= 2;
    int cc = (L + g - 1) / g;
    if (cc < 1) cc = 1;
    if ((cc & 1) == 0) ++cc;
    *G = g;
    *c = g == 1 ? 1 : cc;  // one lane per line stages nothing
}

void *DeviceArena::take(size_t bytes)
{
    const size_t off = align_up(used, 256);
    if (off + bytes > cap) return nullptr;
    used = off + bytes;
    return base + off;
}

cudaError_t DeviceArena::reserve(size_t bytes)
{
    if (bytes <= cap) return cudaSuccess;
    if (base) cudaFree(base);
    base = nullptr;
    cap = 0;
    const size_t want = align_up(bytes + bytes / 8, 1 << 20);
    cudaError_t e = cudaMalloc((void **)&base, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        e = cudaMalloc((void **)&base, bytes);
        if (e != cudaSuccess) return e;
        cap = bytes;
        return cudaSuccess;
    }
    cap = want;
    return cudaSuccess;
}

void DeviceArena::release()
{
    if (base) cudaFree(base);
    base = nullptr;
    cap = used = 0;
}

Engine::Engine()
{
    cudaGetDevice(&dev_);
    cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, dev_);
    cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking);
    cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking);
    cudaEventCreateWithFlags(&ev_setup_, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev_a_, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev_b_, cudaEventDisableTiming);
    cudaEventCreate(&ev_t0_);
    cudaEventCreate(&ev_t1_);
    cell_occupancy(false, &occ_[0]);
    cell_occupancy(true, &occ_[1]);
}

Engine::~Engine()
{
    if (stream_) cudaStreamSynchronize(stream_);
    if (side_) cudaStreamSynchronize(side_);
    arena_.release();
    in_arena_.release();
    cudaFree(d_sys_);
    cudaFree(d_st_);
    cudaFree(d_tiles_);
    cudaFree(d_prefix_);
    cudaFree(d_line_sys_);
    cudaFree(d_allprefix_);
    cudaFree(d_partials_);
    cudaFree(d_lines_);
    cudaFree(d_seq_scratch_);
    cudaFree(d_one_sys_);
    cudaFree(d_dot_partials_);
    cudaFree(gm_basis_);
    cudaFree(gm_scal_);
    cudaFree(gm_max_);
    cudaFree(d_dot_counter_);
    cudaFree(d_dot_out_);
    if (h_st_pinned_) cudaFreeHost(h_st_pinned_);
    for (int q = 0; q < STAGES; ++q) {
        if (stage_buf_[q]) cudaFreeHost(stage_buf_[q]);
        if (stage_ev_[q]) cudaEventDestroy(stage_ev_[q]);
    }
    if (live_exec_) cudaGraphExecDestroy(live_exec_);
    for (auto &r : retired_execs_) cudaGraphExecDestroy(r.first);
    for (int q = 0; q < 2; ++q) {
        if (ev_c0_[q]) cudaEventDestroy(ev_c0_[q]);
        if (ev_c1_[q]) cudaEventDestroy(ev_c1_[q]);
    }
    if (ev_fence_) cudaEventDestroy(ev_fence_);
    if (ev_a_) cudaEventDestroy(ev_a_);
    if (ev_b_) cudaEventDestroy(ev_b_);
    if (ev_t0_) cudaEventDestroy(ev_t0_);
    if (ev_t1_) cudaEventDestroy(ev_t1_);
    for (auto &e : kt_ev_)
        if (e) cudaEventDestroy(e);
    if (ev_setup_) cudaEventDestroy(ev_setup_);
    if (side_) cudaStreamDestroy(side_);
    if (stream_) cudaStreamDestroy(stream_);
}

// The host buffers the state snapshots land in: pinned and mapped, written by
// k_state_snapshot through their device address.  The stream is drained before
// an old buffer is freed (a snapshot may still be writing into it).
int Engine::reserve_snapshots(size_t entries)
{
    if (entries <= h_st_pinned_cap_) return 0;
    if (h_st_pinned_) {
        CK(cudaStreamSynchronize(stream_));
        cudaFreeHost(h_st_pinned_);
    }
    h_st_pinned_ = nullptr;
    d_st_mapped_ = nullptr;
    h_st_pinned_cap_ = 0;
    CK(cudaHostAlloc((void **)&h_st_pinned_, sizeof(SysState) * entries, cudaHostAllocMapped));
    CK(cudaHostGetDevicePointer((void **)&d_st_mapped_, h_st_pinned_, 0));
    h_st_pinned_cap_ = entries;
    return 0;
}

int Engine::fail(const std::string &msg, int code)
{
    err_ = msg;
    return code;
}


// The result of one system from its final device state.
SolveResult result_of(const SysState &st, bool mixed)
{
    SolveResult r;
    r.ier = st.ier;
    r.iterations = mixed ? st.inner_total : st.iter;
    r.iter_tot_add = st.iter_tot_add;
    r.exit_kind = st.exit_kind;
    r.line_skips = st.line_skips;
    r.line_fallbacks = st.line_fallbacks;
    r.outer_steps = st.outer_steps;
    r.deflated = mixed ? st.defl : 0;
    r.rnorm0 = mixed ? st.outer_rnorm0 : st.rnorm0;
    r.rnorm = mixed ? st.outer_rnorm : st.rnorm;
    if (st.status != ST_DONE) {
        r.ier = -15;
        r.exit_kind = EX_ERROR;
    }
    if (st.err & 4) {
        r.ier = -15;  // a staged copy did not complete within its time limit
        r.exit_kind = EX_ERROR;
    }
    if (st.err & 2) {
        r.ier = -12;  // DGTSV INFO != 0 inside a JK/IJ sweep (the reference stops there)
        r.exit_kind = EX_ERROR;
    }
    return r;
}

// ------------------------------------------------------------------ staged uploads
cudaError_t Engine::stage_open(size_t bytes)
{
    stage_cur_ = (stage_cur_ + 1) % STAGES;
    stage_used_ = 0;
    if (stage_ev_[stage_cur_]) {
        cudaError_t e = cudaEventSynchronize(stage_ev_[stage_cur_]);  // its last copies are done
        if (e != cudaSuccess) return e;
    } else {
        cudaError_t e = cudaEventCreateWithFlags(&stage_ev_[stage_cur_], cudaEventDisableTiming);
        if (e != cudaSuccess) return e;
    }
    if (bytes > stage_cap_[stage_cur_]) {
        if (stage_buf_[stage_cur_]) cudaFreeHost(stage_buf_[stage_cur_]);
        stage_buf_[stage_cur_] = nullptr;
        stage_cap_[stage_cur_] = 0;
        const size_t want = std::max<size_t>(2 * bytes, 1 << 20);
        cudaError_t e = cudaMallocHost((void **)&stage_buf_[stage_cur_], want);
        if (e != cudaSuccess) return e;
        stage_cap_[stage_cur_] = want;
    }
    return cudaSuccess;
}

cudaError_t Engine::stage_close() { return cudaEventRecord(stage_ev_[stage_cur_], stream_); }

// ------------------------------------------------------------------ work memory
// One system's work memory: in the mixed form the FP32 diagonals first, then the
// nine iteration vectors and the three J-line factor arrays (elements of the
// form's precision), then the per-line flags; the mixed form's copy of the
// initial guess follows that region.
// Line pitch and cells of a system's arrays in the form's precision: the mixed
// form's FP32 arrays pad each J-line to a multiple of four cells.
int form_pitch(int jmax2, int precision) { return precision == PREC_MIXED ? (jmax2 + 3) / 4 * 4 : jmax2; }
int64_t form_cells(int64_t n, int64_t lines, int precision)
{
    if (precision != PREC_MIXED || lines <= 0) return n;
    return (int64_t)form_pitch((int)(n / lines), precision) * lines;
}

size_t vec_region_bytes(int64_t n, int64_t lines, int precision)
{
    const size_t ew = precision == PREC_MIXED ? 4 : 8;
    const size_t m = (size_t)form_cells(n, lines, precision);
    size_t b = 0;
    if (precision == PREC_MIXED)  // FP32 diagonals, row sums, deflation vector z and A z
        b += align_up(7 * m * 4, 256) + 2 * align_up(m * 4, 256) + align_up(m, 256);
    b += (NVEC + 3) * align_up(m * ew, 256) + align_up((size_t)lines * 4, 256);
    return b;
}

size_t work_bytes(int64_t n, int64_t lines, int precision)
{
    return vec_region_bytes(n, lines, precision) + (precision == PREC_MIXED ? align_up((size_t)n * 8, 256) : 0);
}

// A block that serves a mixed attempt and then, if it gives up, the FP64
// re-solve: the FP64 region (larger than the mixed one) followed by the initial guess.
size_t live_work_bytes(int64_t n, int64_t lines, int precision)
{
    if (precision != PREC_MIXED) return vec_region_bytes(n, lines, PREC_FP64);
    return std::max(vec_region_bytes(n, lines, PREC_FP64), vec_region_bytes(n, lines, PREC_MIXED)) +
           align_up((size_t)n * 8, 256);
}

void carve_work(SysDev &d, char *work, int64_t lines, int precision, char *x0)
{
    const size_t n = (size_t)form_cells(d.n, lines, precision);
    const size_t ew = precision == PREC_MIXED ? 4 : 8;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char *p = work + off;
        off += align_up(bytes, 256);
        return p;
    };
    d.a32 = nullptr;
    d.defect = nullptr;
    d.defl_z = nullptr;
    d.defl_az = nullptr;
    d.x64[1] = nullptr;
    if (precision == PREC_MIXED) {
        d.a32 = (float *)take(7 * n * 4);
        d.defect = (float *)take(n * 4);
        d.defl_az = (float *)take(n * 4);
        d.defl_z = (unsigned char *)take(n);
        d.x64[1] = (double *)x0;  // initial guess, kept for an FP64 re-solve
    }
    for (int v = 0; v < NVEC; ++v) d.vec[v] = take(n * ew);
    for (int f = 0; f < 3; ++f) d.fac[f] = take(n * ew);
    d.line_flag = (int *)take((size_t)lines * 4);
    if (precision != PREC_MIXED) d.vec[V_X] = d.x64[0];
}

// ------------------------------------------------------------------ batch setup
int Engine::setup_batch(const std::vector<SystemSpec> &specs, const SolveOptions &opt)
{
    nsys_ = (int)specs.size();
    const bool mixed = opt.precision == PREC_MIXED;

    // work memory: the iteration vectors, plus the FP32 diagonals and a copy of
    // the initial guess in the mixed form (inputs are device arrays by now)
    size_t bytes = 4096;
    for (const auto &s : specs) bytes += work_bytes(s.n, (int64_t)s.imax2 * s.kmax2, opt.precision) + 256;
    cudaError_t e = arena_.reserve(bytes);
    if (e != cudaSuccess) return fail(std::string("device memory for the batch: ") + cudaGetErrorString(e), -11);
    arena_.reset();

    h_sys_.assign(nsys_, SysDev{});
    h_st_.assign(nsys_, SysState{});
    h_tiles_.clear();
    h_prefix_.assign(nsys_ + 1, 0);
    h_allprefix_.assign(nsys_ + 1, 0);
    int tile_base = 0;
    for (int s = 0; s < nsys_; ++s) {
        const SystemSpec &sp = specs[s];
        SysDev &d = h_sys_[s];
        d.imax2 = sp.imax2;
        d.jmax2 = sp.jmax2;
        d.kmax2 = sp.kmax2;
        d.do_k = sp.do_k;
        d.cyc = sp.cyc;
        d.n = sp.n;
        d.div_j = make_fastdiv((uint32_t)sp.jmax2);
        d.div_i = make_fastdiv((uint32_t)sp.imax2);
        d.jp = form_pitch(sp.jmax2, opt.precision);
        d.np = (int64_t)d.jp * sp.imax2 * sp.kmax2;
        d.div_jp = make_fastdiv((uint32_t)d.jp);
        d.pc = opt.pc;
        d.ntiles = (int)((std::max(sp.n, d.np) + TILE_CELLS - 1) / TILE_CELLS);
        d.tile_base = tile_base;
        tile_base += d.ntiles;
        shape_for(sp.jmax2, mixed ? 4 : 8, opt.force_lanes, &d.lane_group, &d.rows_per_lane, &d.line_kind);
        d.half_lines = (sp.imax2 + 1) / 2;
        d.div_h = make_fastdiv((uint32_t)d.half_lines);
        d.a64 = sp.a;
        d.b64 = sp.b;
        d.x64[0] = sp.x;
        const int64_t lines = (int64_t)sp.imax2 * sp.kmax2;
        char *work = (char *)arena_.take(work_bytes(sp.n, lines, opt.precision));
        carve_work(d, work, lines, opt.precision, mixed ? work + vec_region_bytes(sp.n, lines, opt.precision) : nullptr);
        for (int t = 0; t < d.ntiles; ++t) h_tiles_.push_back(Tile{s, t});
        h_allprefix_[s + 1] = h_allprefix_[s] + sp.imax2 * sp.kmax2;

        SysState &st = h_st_[s];
        st.tol = sp.tol;
        st.itmax = sp.itmax;
        st.status = ST_RUNNING;
        st.phase = opt.skip_scale ? PH_INIT : PH_SETUP;
        st.mixed = mixed ? 1 : 0;
        st.method = opt.method;
        st.inner_tol = opt.inner_tol;
        st.growth_limit = opt.mixed_growth;
        st.stall_limit = opt.mixed_stalls;
        st.min_margin = opt.mixed_min_margin;
        st.defl_allow = opt.deflate ? 1 : 0;
        st.replace_every = opt.replace_every;
        st.icheck = (opt.minimize_dotproducts && !mixed) ? (opt.transposed ? 5 : std::max(1, opt.icheck_bicgs)) : 0;
        st.restart_growth = opt.restart_growth;
        st.margin_bits = 0x7f800000u;
        st.i = 1;
        st.iter = 1;
    }

    x0_.assign(nsys_, nullptr);
    if (mixed)
        for (int q = 0; q < nsys_; ++q) {
            x0_[q] = h_sys_[q].x64[1];
            CK(cudaMemcpyAsync(h_sys_[q].x64[1], h_sys_[q].x64[0], (size_t)h_sys_[q].n * 8, cudaMemcpyDeviceToDevice,
                               stream_));
        }

    // tables are small; their device copies are reallocated only when they grow
    CK(upload(&d_st_, &st_cap_, h_st_.data(), h_st_.size(), stream_));
    CK(upload(&d_tiles_, &tiles_cap_, h_tiles_.data(), h_tiles_.size(), stream_));
    CK(upload(&d_allprefix_, &allprefix_cap_, h_allprefix_.data(), h_allprefix_.size(), stream_));
    const size_t need_part = 2 * (size_t)std::max(tile_base, 1);
    if (need_part > part_cap_) {
        cudaFree(d_partials_);
        d_partials_ = nullptr;
        CK(cudaMalloc((void **)&d_partials_, need_part * sizeof(double)));
        part_cap_ = need_part;
    }
    if (const int rs = reserve_snapshots(2 * (size_t)nsys_)) return rs;

    view_.st = d_st_;
    view_.tiles = d_tiles_;
    view_.ntiles = (int)h_tiles_.size();
    view_.nsys = nsys_;
    view_.partials = d_partials_;

    cfg_.stream = stream_;

    // setup kernels: one block per tile; iteration kernels: persistent grids of
    // resident blocks that stride over the tiles
    cfg_.cell_grid = std::max(1, view_.ntiles);
    cfg_.stencil_grid = std::max(1, view_.ntiles);
    const CellOcc &oc = occ_[mixed ? 1 : 0];
    auto grid = [&](int bpsm) { return std::max(1, std::min(view_.ntiles, sms_ * bpsm)); };
    cfg_.g_p = grid(oc.p_update);
    cfg_.g_s = grid(oc.s_update);
    cfg_.g_xr = grid(oc.xr_update);
    cfg_.g_mv = grid(oc.matvec);
    cfg_.g_mv_pair = grid(oc.matvec_pair);
    cfg_.rows_pair = cfg_.rows_single = 0;
    for (int q = 0; q < nsys_; ++q)
        if (h_sys_[q].n > 0) ((h_sys_[q].jp & 1) ? cfg_.rows_single : cfg_.rows_pair) = 1;
    cfg_.mv_staged = 0;
    cfg_.g_mv_staged = 1;
    if (mixed && opt.staged_matvec >= 1 && opt.staged_matvec <= MV_SHAPES && oc.matvec_staged[opt.staged_matvec] > 0) {
        cfg_.mv_staged = opt.staged_matvec;
        cfg_.g_mv_staged = grid(oc.matvec_staged[opt.staged_matvec]);
    }
    cfg_.g_copy = grid(oc.copy);
    cfg_.g_outer = grid(oc.outer);
    return configure_lines(mixed ? 4 : 8);
    return 0;
}

// Work items of the J-line kernel (parity waves) and its launch shape, from each
// system's lanes per line; the system table goes to the device here.  only_L = -1
// keeps the line work of the systems whose line length is in tune_lengths_ only
// (autotuning); only_L > 0
// keeps the line work of the systems with that line length only (autotuning).
int Engine::configure_lines(int elem, int only_L)
{
    h_prefix_.assign(nsys_ + 1, 0);
    int cmax = 1;
    for (int s = 0; s < nsys_; ++s) {
        const SysDev &d = h_sys_[s];
        cmax = std::max(cmax, d.rows_per_lane);
        const int lpw = 32 / d.lane_group;
        const bool tuned = only_L < 0 && std::find(tune_lengths_.begin(), tune_lengths_.end(), d.jmax2) !=
                                                tune_lengths_.end();
        const bool keep = d.n > 0 && (only_L == 0 || d.jmax2 == only_L || tuned);  // n = 0: empty slot of a live batch
        const int64_t slots = keep ? (int64_t)d.half_lines * d.kmax2 : 0;
        h_prefix_[s + 1] = h_prefix_[s] + (int)((slots + lpw - 1) / lpw);
    }
    h_line_sys_.resize(std::max(h_prefix_[nsys_], 1));
    for (int s = 0; s < nsys_; ++s)
        std::fill(h_line_sys_.begin() + h_prefix_[s], h_line_sys_.begin() + h_prefix_[s + 1], s);
    CK(stage_open(sizeof(SysDev) * h_sys_.size() + sizeof(int) * (h_prefix_.size() + h_line_sys_.size()) + 256));
    CK(upload_staged(&d_sys_, &sys_cap_, h_sys_.data(), h_sys_.size()));
    CK(upload_staged(&d_prefix_, &prefix_cap_, h_prefix_.data(), h_prefix_.size()));
    CK(upload_staged(&d_line_sys_, &line_sys_cap_, h_line_sys_.data(), (size_t)h_prefix_[nsys_]));
    CK(stage_close());
    // the uploads may have (re)allocated the tables: the kernels' view follows them
    view_.sys = d_sys_;
    view_.line_prefix = d_prefix_;
    view_.line_sys = d_line_sys_;
    if (!view_.sys || !view_.st || !view_.tiles || !view_.line_prefix || !view_.line_sys || !view_.partials)
        return fail("internal: batch tables missing on the device", -13);
    cfg_.line_cmax = cmax;
    int wpb = 1;
    const int bpsm = elem == 4 ? prepare_line_kernel<float>(cmax, &wpb) : prepare_line_kernel<double>(cmax, &wpb);
    if (bpsm <= 0) return fail("J-lines too long for the shared-memory staging of the line kernel", -10);
    cfg_.line_warps = wpb;
    const int items = h_prefix_[nsys_];
    cfg_.line_grid = std::max(1, std::min((items + wpb - 1) / wpb, sms_ * bpsm));
    // which line kernels the batch needs (systems with no line work count for none)
    // rows per access of the warp kernel: four when every system's lines start on
    // 16-byte boundaries (the mixed form's padded FP32 arrays) and its lanes' spans
    // are multiples of four, two when they start on 8- or 16-byte boundaries
    cfg_.line_thread = cfg_.line_warp = cfg_.line_single = 0;
    cfg_.line_vw = elem == 4 ? 4 : 2;
    for (int s = 0; s < nsys_; ++s) {
        if (h_prefix_[s + 1] == h_prefix_[s]) continue;
        const SysDev &d = h_sys_[s];
        if (d.line_kind == LK_THREAD) {
            cfg_.line_thread = 1;
        } else {
            cfg_.line_warp = 1;
            if (d.jp & 1) cfg_.line_single = 1;
            if ((d.jp & 3) || d.lane_group < 4) cfg_.line_vw = std::min(cfg_.line_vw, 2);
        }
    }
    if (cfg_.line_single) cfg_.line_vw = 1;
    if (!cfg_.line_thread && !cfg_.line_warp) cfg_.line_warp = 1;  // empty batch: a no-op launch
    const int tocc = elem == 4 ? line_thread_occupancy<float>() : line_thread_occupancy<double>();
    cfg_.line_grid_thread = std::max(1, std::min((items + 3) / 4, sms_ * tocc));
    return 0;
}

static constexpr int MAX_TUNED_ROWS = 17;

// Rows per lane; one lane per line (G = 1) stages nothing, so it counts as one.
static int rows_for(int L, int G)
{
    if (G == 1) return 1;
    int c = (L + G - 1) / G;
    if (c < 1) c = 1;
    if ((c & 1) == 0) ++c;
    return c;
}

static void set_shape(int L, int lanes, int *G, int *c, int *kind)
{
    const int g = std::max(1, std::min(lanes, 32));
    *G = g;
    *c = rows_for(L, g);
    *kind = g == 1 ? LK_THREAD : LK_WARP;
}

// Lanes per J-line for a line of length L: a forced value, the autotuner's
// choice for (precision, L), or the default of line_shape().
void Engine::shape_for(int L, int elem, int forced, int *G, int *c, int *kind)
{
    if (forced > 0) {
        int g = 1;
        while (g * 2 <= std::min(forced, 32)) g *= 2;
        set_shape(L, g, G, c, kind);
        return;
    }
    {
        std::lock_guard<std::mutex> lk(tunes().mu);
        auto it = tunes().lanes.find(std::make_pair(elem, L));
        if (it != tunes().lanes.end()) {
            set_shape(L, it->second, G, c, kind);
            return;
        }
    }
    line_shape(L, G, c);
    *kind = *G == 1 ? LK_THREAD : LK_WARP;
}

// The autotuner: for the line lengths of the batch without a recorded choice, time
// a red/black pass of the J-line kernel over all their lines at once (the other
// systems' line work masked out) for each lanes-per-line value g, each length
// taking the smallest power of two at or above g that leaves it at most
// MAX_TUNED_ROWS rows per lane, and keep the fastest g for all of them.  Timing
// the whole mix at once ranks the shapes as the batch runs them: timing each
// length alone, on its few systems, left a 512-system FP64 batch 10% slower than
// one shape for every line.  The row bound keeps the kernel's shared-memory
// staging, sized by the batch's largest rows per lane, small enough for full
// occupancy.
int Engine::autotune_lines(const SolveOptions &opt, int elem)
{
    std::vector<int> todo;
    for (int s = 0; s < nsys_; ++s) {
        if (h_sys_[s].n == 0) continue;  // empty slot of a live batch
        const int L = h_sys_[s].jmax2;
        {
            std::lock_guard<std::mutex> lk(tunes().mu);
            if (tunes().lanes.count(std::make_pair(elem, L))) continue;
        }
        if (std::find(todo.begin(), todo.end(), L) == todo.end()) todo.push_back(L);
    }
    if (todo.empty()) return 0;
    WaveArgs w[2] = {};
    for (int q = 0; q < 2; ++q) {
        w[q].kind = 0;
        w[q].par = 1 - q;
        w[q].rhs = V_P;
        w[q].nbr = V_PH;
        w[q].old = V_P;
        w[q].dst = V_PH;
        w[q].write_old = 1;
        w[q].gate = G_ANY;
    }
    // lanes of length L under the candidate g: the smallest power of two at or
    // above g within the row bound; for a line too long for the bound at any
    // width, 32 while its staging stays within 48 KB per warp, else none (0:
    // the candidate is skipped; one lane per line always fits)
    auto lanes_for = [&](int L, int g) {
        for (int h = g; h <= 32; h *= 2) {
            int G = 1, c = 1, kind = LK_WARP;
            set_shape(L, h, &G, &c, &kind);
            if (kind != LK_WARP || (c <= MAX_TUNED_ROWS && (size_t)kernel_smem_line_bytes(c, elem) <= 48 * 1024))
                return h;
        }
        int G = 1, c = 1, kind = LK_WARP;
        set_shape(L, 32, &G, &c, &kind);
        return (size_t)kernel_smem_line_bytes(c, elem) <= 48 * 1024 ? 32 : 0;
    };
    // the timing events and the tuning mask are released on every way out
    struct TuneScope {
        std::vector<int> &mask;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        ~TuneScope()
        {
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
            mask.clear();
        }
    } scope{tune_lengths_};
    CK(cudaEventCreate(&scope.e0));
    CK(cudaEventCreate(&scope.e1));
    const cudaEvent_t e0 = scope.e0, e1 = scope.e1;
    tune_lengths_ = todo;
    int best_g = 0;
    float best_ms = 1e30f;
    for (int g = 1; g <= 32; g *= 2) {
        bool fits = true;
        for (int L : todo) fits = fits && lanes_for(L, g) > 0;
        if (!fits) continue;
        for (int s = 0; s < nsys_; ++s) {
            const int L = h_sys_[s].jmax2;
            if (h_sys_[s].n > 0 && std::find(todo.begin(), todo.end(), L) != todo.end())
                set_shape(L, lanes_for(L, g), &h_sys_[s].lane_group, &h_sys_[s].rows_per_lane, &h_sys_[s].line_kind);
        }
        int rc = configure_lines(elem, -1);
        if (rc) return rc;
        float tot = 0.f;
        for (int rep = 0; rep < 4; ++rep) {
            if (rep == 1) CK(cudaEventRecord(e0, stream_));
            for (int q = 0; q < 2; ++q) CK(elem == 4 ? launch_jline<float>(view_, cfg_, w[q]) : launch_jline<double>(view_, cfg_, w[q]));
        }
        CK(cudaEventRecord(e1, stream_));
        CK(cudaEventSynchronize(e1));
        cudaEventElapsedTime(&tot, e0, e1);
        if (tot < best_ms) {
            best_ms = tot;
            best_g = g;
        }
    }
    for (int L : todo) {
        int g = best_g > 0 ? lanes_for(L, best_g) : 0;
        if (g == 0) {  // no candidate timed
            int c_unused = 0;
            line_shape(L, &g, &c_unused);
        }
        {
            std::lock_guard<std::mutex> lk(tunes().mu);
            tunes().lanes[std::make_pair(elem, L)] = g;
        }
        for (int s = 0; s < nsys_; ++s)
            if (h_sys_[s].jmax2 == L && h_sys_[s].n > 0)
                set_shape(L, g, &h_sys_[s].lane_group, &h_sys_[s].rows_per_lane, &h_sys_[s].line_kind);
    }
    (void)opt;
    save_tune_cache();
    return configure_lines(elem);
}

void Engine::load_tune_cache(const std::string &path)
{
    std::lock_guard<std::mutex> lk(tunes().mu);
    tunes().path = path;
    FILE *f = path.empty() ? nullptr : std::fopen(path.c_str(), "r");
    if (!f) return;
    int elem, L, G;
    char buf[256];
    while (std::fgets(buf, sizeof buf, f))
        if (std::sscanf(buf, " {\"elem\": %d, \"L\": %d, \"lanes\": %d}", &elem, &L, &G) == 3 && G >= 1 &&
            G <= 32)
            tunes().lanes[std::make_pair(elem, L)] = G;
    std::fclose(f);
}

void Engine::save_tune_cache()
{
    std::lock_guard<std::mutex> lk(tunes().mu);
    const auto &line_tune_ = tunes().lanes;
    if (tunes().path.empty()) return;
    FILE *f = std::fopen(tunes().path.c_str(), "w");
    if (!f) return;
    std::fprintf(f, "[\n");
    size_t q = 0;
    for (const auto &kv : line_tune_)
        std::fprintf(f, "  {\"elem\": %d, \"L\": %d, \"lanes\": %d}%s\n", kv.first.first, kv.first.second, kv.second,
                     ++q < line_tune_.size() ? "," : "");
    std::fprintf(f, "]\n");
    std::fclose(f);
}

int Engine::tune_table(int *out, int max_entries) const
{
    std::lock_guard<std::mutex> lk(tunes().mu);
    int q = 0;
    for (const auto &kv : tunes().lanes) {
        if (q < max_entries) {
            out[3 * q] = kv.first.first;
            out[3 * q + 1] = kv.first.second;
            out[3 * q + 2] = kv.second;
        }
        ++q;
    }
    return q;
}

// ------------------------------------------------------------------ LINE preconditioner plan
// LEQ_MSOLVE (model/leqsol_mod.f:286-598) as a list of device steps.  Var = B
// (SETGUESS) is folded into the first red/black pass when the first active
// letter is 'R': its first wave reads neighbours and old values from B, its
// second wave reads its own old values from B.
int Engine::plan_msolve(const SolveOptions &opt, int src, int dst, int gate, int which)
{
    plan_[which].clear();
    if (opt.pc == PC_NONE) return 0;
    if (opt.pc == PC_DIAG) {
        Step st{};
        st.type = 3;
        st.w.rhs = src;
        st.w.dst = dst;
        st.w.gate = gate;
        plan_[which].push_back(st);
        return 0;
    }
    // the 2-D branch of LEQ_MSOLVE applies when no system of the batch is 3-D;
    // letters I/K/A (single systems only) read d0's geometry
    int any3d = -1;
    for (int s = 0; s < nsys_; ++s)
        if (h_sys_[s].n > 0) any3d = std::max(any3d, h_sys_[s].do_k ? 1 : 0);
    int s0 = 0;
    while (s0 + 1 < nsys_ && h_sys_[s0].n == 0) ++s0;
    SysDev d0 = h_sys_[s0];
    d0.do_k = any3d != 0;
    const bool single = nsys_ == 1;
    auto letter = [&](char ch) -> int {
        if (ch == 'R' || ch == 'r') return 'R';
        if (ch == 'I' || ch == 'i') return 'I';
        if (ch == 'K' || ch == 'k') return 'K';
        if (ch == 'A' || ch == 'a') return 'A';
        return 0;
    };
    // LEQ_MSOLVEt (DO_TRANSPOSE, model/leq_bicgst.f:978-1177) serves I in 2-D (its
    // red/black branch is 3-D only) and R, I, K in 3-D (no A); with an odd number of
    // I-lines its red/black loop wraps within a k row, so that lines of one pass
    // neighbour each other and their order matters: not served.
    auto noop = [&](int L) {
        if (!d0.do_k && (L == 'A' || L == 'K')) return true;  // no-ops in the 2-D branch
        if (opt.transposed && ((!d0.do_k && L == 'R') || L == 'A')) return true;
        return false;
    };
    if (opt.transposed && d0.do_k && (d0.imax2 & 1))
        for (int q = 0; q < 4; ++q)
            if (letter(opt.sweep[q]) == 'R')
                return fail("DO_TRANSPOSE red/black sweeps with an odd IMAX2 are not served", -10);
    int first = 0;
    for (int q = 0; q < 4 && !first; ++q) {
        const int L = letter(opt.sweep[q]);
        if (!L || noop(L)) continue;
        first = L;
    }
    if (!first) {
        Step cp{};
        cp.type = 1;
        cp.w.rhs = src;
        cp.w.dst = dst;
        cp.w.gate = gate;
        plan_[which].push_back(cp);
        return 0;
    }
    // red/black lines that wrap onto a line of their own colour (odd cyclic
    // periods) run in wrap levels, after a plain Var = B copy
    int wrap_levels = 1;
    for (int s = 0; s < nsys_; ++s) {
        const SysDev &d = h_sys_[s];
        if (d.n == 0) continue;
        wrap_levels = std::max(wrap_levels, 1 + wrap_level(d, d.imax2 - 1, d.kmax2 - 1));
    }
    bool fused_guess = (first == 'R') && wrap_levels == 1;
    if (!fused_guess) {
        Step cp{};
        cp.type = 1;
        cp.w.rhs = src;
        cp.w.dst = dst;
        cp.w.gate = gate;
        plan_[which].push_back(cp);
    }
    int waves_done = 0;
    auto wave = [&](int kind, int par, int count, const int2 *list, int nlines, int lvl = 0) {
        Step st{};
        st.type = 0;
        WaveArgs &w = st.w;
        w.kind = kind;
        w.par = par;
        w.lvl = lvl;
        w.rhs = src;
        w.dst = dst;
        w.gate = gate;
        w.count = count;
        w.list = list;
        w.nlines = nlines;
        if (fused_guess && waves_done == 0) {
            w.nbr = src;
            w.old = src;
            w.write_old = 1;
        } else if (fused_guess && waves_done == 1) {
            w.nbr = dst;
            w.old = src;
            w.write_old = 1;
        } else {
            w.nbr = dst;
            w.old = dst;
            w.write_old = 0;
        }
        ++waves_done;
        plan_[which].push_back(st);
    };
    auto red_black = [&]() {
        for (int par = 1; par >= 0; --par) {
            if (wrap_levels == 1) {
                wave(0, par, 0, nullptr, 0);
            } else {
                for (int l = 0; l < wrap_levels; ++l) wave(0, par, 0, nullptr, 0, l + 1);
            }
        }
    };
    std::vector<std::pair<size_t, size_t>> list_refs;  // (plan index, offset into h_lines_) for kind 2 / seq
    for (int q = 0; q < 4; ++q) {
        const int L = letter(opt.sweep[q]);
        if (!L || noop(L)) continue;
        if (!d0.do_k) {
            if (L == 'R') {  // :382-391, i odd then i even (the kernel flips the 3-D parity)
                red_black();
            } else if (L == 'I') {  // :374-379, i = 1..imax2 in order
                if (!single) return fail("sweep letter 'I' is served for single-system solves only", -10);
                for (int dgl = 2; dgl <= d0.imax2 + 1; ++dgl) wave(1, dgl, 1, nullptr, 0);
            }
            continue;
        }
        if (L == 'R') {  // :497-522, (i+k) odd first
            red_black();
        } else if (L == 'I' || L == 'K') {
            // :567-582: lexicographic line Gauss-Seidel; both orders give the same
            // result, and the lines of one anti-diagonal i+k = const are independent.
            if (!single) return fail("sweep letters 'I'/'K' are served for single-system solves only", -10);
            const int lpw = 32 / d0.lane_group;
            for (int dgl = 2; dgl <= d0.imax2 + d0.kmax2; ++dgl) {
                const int ilo = std::max(1, dgl - d0.kmax2), ihi = std::min(d0.imax2, dgl - 1);
                const int cnt = ihi - ilo + 1;
                wave(1, dgl, (cnt + lpw - 1) / lpw, nullptr, 0);
            }
        } else if (L == 'A') {
            if (!single) return fail("sweep letter 'A' is served for single-system solves only", -10);
            // :398-470: JK, IJ then IK loops, each sequential in the reference.  Lines are
            // grouped into levels so that every line sees exactly the neighbour values
            // it sees in the reference order.
            const int isize = d0.imax2, jsize = d0.jmax2, ksize = d0.kmax2;
            for (int part = 0; part < 3; ++part) {
                // part 0: I-lines at (j,k); part 1: K-lines at (i,j); part 2: J-lines at (i,k)
                const int n1 = part == 0 ? jsize : isize;   // fast coordinate of the line
                const int n2 = part == 1 ? jsize : ksize;   // slow coordinate
                std::vector<int2> order;
                for (int icase = 1; icase <= 2; ++icase)
                    for (int m = icase; m <= n1 * n2; m += 2) {
                        int b2 = (m % n1 != 0) ? m / n1 + 1 : m / n1;
                        int b1 = (m - 1 - (b2 - 1) * n1) + 1 + (b2 % 2);
                        if (b1 > n1) b1 = b1 - n1;
                        order.push_back(make_int2(b1, b2));
                    }
                std::vector<int> level((size_t)n1 * n2, 0);
                int maxlev = 0;
                std::vector<int> lev_of(order.size());
                // the line's neighbour lines along the two cross axes, wrapped along a
                // cyclic axis as the increments are (model/set_increments.f:73-113)
                const int cyc1 = part == 0 ? (d0.cyc & 2) : (d0.cyc & 1);
                const int cyc2 = part == 1 ? (d0.cyc & 2) : (d0.cyc & 4);
                auto step = [](int b, int s, int m, int cyc) {  // neighbour of 1-based b in direction s
                    if (cyc && b >= 2 && b <= m - 1) {
                        if (s < 0) return b == 2 ? m - 1 : b - 1;
                        return b == m - 1 ? 2 : b + 1;
                    }
                    return b + s;  // out of range: no neighbour line (clamped onto itself)
                };
                for (size_t t = 0; t < order.size(); ++t) {
                    const int b1 = order[t].x, b2 = order[t].y;
                    int lv = 0;
                    const int nb[4][2] = {{step(b1, -1, n1, cyc1), b2}, {step(b1, 1, n1, cyc1), b2},
                                          {b1, step(b2, -1, n2, cyc2)}, {b1, step(b2, 1, n2, cyc2)}};
                    for (auto &p : nb)
                        if (p[0] >= 1 && p[0] <= n1 && p[1] >= 1 && p[1] <= n2)
                            lv = std::max(lv, level[(size_t)(p[1] - 1) * n1 + (p[0] - 1)]);
                    level[(size_t)(b2 - 1) * n1 + (b1 - 1)] = lv + 1;
                    lev_of[t] = lv + 1;
                    maxlev = std::max(maxlev, lv + 1);
                }
                for (int lv = 1; lv <= maxlev; ++lv) {
                    const size_t off = h_lines_.size();
                    for (size_t t = 0; t < order.size(); ++t)
                        if (lev_of[t] == lv) h_lines_.push_back(order[t]);
                    const int cnt = (int)(h_lines_.size() - off);
                    if (part == 2) {
                        const int lpw = 32 / d0.lane_group;
                        wave(2, 0, (cnt + lpw - 1) / lpw, nullptr, cnt);
                    } else {
                        Step st{};
                        st.type = 2;
                        st.s.axis = part == 0 ? 0 : 2;
                        st.s.count = cnt;
                        st.s.rhs = src;
                        st.s.var = dst;
                        st.s.fatal_on_info = 1;
                        st.s.gate = gate;
                        st.s.lmax = std::max(d0.imax2, d0.kmax2);
                        if (!fused_guess || waves_done >= 2) {
                            plan_[which].push_back(st);
                        } else {
                            return fail("internal: ASAS after a fused first pass", -13);
                        }
                    }
                    list_refs.push_back({plan_[which].size() - 1, off});
                }
            }
        }
    }
    for (auto &r : list_refs) list_refs_.push_back({which, r.first, r.second});
    return 0;
}

// Line lists of both plans go to the device in one upload, after both plans exist.
int Engine::bind_lists()
{
    if (list_refs_.empty()) return 0;
    size_t cap = d_lines_cap_;
    cudaError_t e = upload(&d_lines_, &cap, h_lines_.data(), h_lines_.size(), stream_);
    if (e != cudaSuccess) return fail(cudaGetErrorString(e), -13);
    d_lines_cap_ = cap;
    size_t scratch_need = 0;
    for (auto &r : list_refs_) {
        Step &st = plan_[r.which][r.index];
        if (st.type == 0) st.w.list = d_lines_ + r.offset;
        if (st.type == 2) {
            st.s.lines = d_lines_ + r.offset;
            scratch_need = std::max(scratch_need, (size_t)4 * st.s.lmax * st.s.count);
        }
    }
    if (scratch_need > d_seq_scratch_cap_) {
        cudaFree(d_seq_scratch_);
        d_seq_scratch_ = nullptr;
        e = cudaMalloc((void **)&d_seq_scratch_, scratch_need * sizeof(double));
        if (e != cudaSuccess) return fail(cudaGetErrorString(e), -11);
        d_seq_scratch_cap_ = scratch_need;
    }
    for (auto &r : list_refs_) {
        Step &st = plan_[r.which][r.index];
        if (st.type == 2) st.s.scratch = d_seq_scratch_;
    }
    return 0;
}

// ---- time_kernels: events around each launch, summed per kernel class at the end
void Engine::kt_begin()
{
    if (!ktime_ || kt_count_ >= KT_MAX) return;
    if ((int)kt_ev_.size() < 2 * (kt_count_ + 1)) {
        const size_t old = kt_ev_.size();
        kt_ev_.resize(std::max<size_t>(2 * (kt_count_ + 1), old * 2), nullptr);
        for (size_t q = old; q < kt_ev_.size(); ++q) cudaEventCreate(&kt_ev_[q]);
    }
    cudaEventRecord(kt_ev_[2 * kt_count_], stream_);
}

void Engine::kt_end(int kclass)
{
    if (!ktime_ || kt_count_ >= KT_MAX) return;
    cudaEventRecord(kt_ev_[2 * kt_count_ + 1], stream_);
    if ((int)kt_class_.size() <= kt_count_) kt_class_.resize(kt_count_ + 1);
    kt_class_[kt_count_++] = kclass;
}

void Engine::kt_harvest()
{
    for (int q = 0; q < kt_count_; ++q) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, kt_ev_[2 * q], kt_ev_[2 * q + 1]);
        timing_.class_ms[kt_class_[q]] += ms;
        timing_.class_launches[kt_class_[q]] += 1;
    }
    timing_.jline_ms = timing_.class_ms[KC_JLINE];
    timing_.jline_launches = timing_.class_launches[KC_JLINE];
    kt_count_ = 0;
    ktime_ = false;
}

int Engine::run_msolve_plan(int which, int elem)
{
    for (const Step &st : plan_[which]) {
        cudaError_t e = cudaSuccess;
        kt_begin();
        if (st.type == 0) {
            e = (elem == 8) ? launch_jline<double>(view_, cfg_, st.w) : launch_jline<float>(view_, cfg_, st.w);
        } else if (st.type == 1) {
            e = (elem == 8) ? launch_copy<double>(view_, cfg_, st.w.rhs, st.w.dst, st.w.gate)
                            : launch_copy<float>(view_, cfg_, st.w.rhs, st.w.dst, st.w.gate);
        } else if (st.type == 2) {
            e = (elem == 8) ? launch_seq_lines<double>(view_, st.s, stream_) : launch_seq_lines<float>(view_, st.s, stream_);
        } else if (st.type == 3) {
            e = (elem == 8) ? launch_diag<double>(view_, cfg_, st.w.rhs, st.w.dst, st.w.gate)
                            : launch_diag<float>(view_, cfg_, st.w.rhs, st.w.dst, st.w.gate);
        }
        kt_end(st.type == 0 ? KC_JLINE : KC_OTHER);
        if (e != cudaSuccess) return fail(std::string("sweep launch: ") + cudaGetErrorString(e), -13);
        ++launches_;
    }
    return 0;
}

// ------------------------------------------------------------------ solve
int Engine::solve(const std::vector<SystemSpec> &specs, const SolveOptions &opt, std::vector<SolveResult> &out)
{
    err_.clear();
    out.assign(specs.size(), SolveResult{});
    if (specs.empty()) return 0;
    for (const auto &s : specs) {
        if (s.imax2 < 1 || s.jmax2 < 1 || s.kmax2 < 1) return fail("grid extents must be >= 1", -14);
        if (!s.do_k && s.kmax2 != 1) return fail("a 2-D system (do_k = 0) needs kmax2 = 1", -14);
        if ((int64_t)s.imax2 * s.jmax2 * s.kmax2 != s.n) return fail("DIMENSION_3 != IMAX2*JMAX2*KMAX2", -14);
        if (s.n > (int64_t)INT32_MAX - TILE_CELLS) return fail("system too large for 32-bit cell indexing", -14);
        if (!s.a || !s.b || !s.x) return fail("null array", -14);
        if (opt.on_device && !aligned16(s))
            return fail("device arrays must start on 16-byte boundaries (cudaMalloc gives 256)", -14);
    }
    if (opt.pc != PC_LINE && opt.pc != PC_DIAG && opt.pc != PC_NONE) return fail("unknown preconditioner", -10);

    // inputs on the device: the caller's arrays, or copies in the input arena.
    // DO_TRANSPOSE scales a transposed copy of A_M that SOLVE_LIN_EQ discards
    // (model/solve_lin_eq.f:139-150): A is scaled in a copy even when it is on the device.
    std::vector<SystemSpec> dev = specs;
    if (opt.transposed && opt.on_device) {
        size_t bytes = 4096;
        for (const auto &s : specs) bytes += align_up(7 * (size_t)s.n * 8, 256);
        cudaError_t e = in_arena_.reserve(bytes);
        if (e != cudaSuccess) return fail(std::string("device memory for the copy of A: ") + cudaGetErrorString(e), -11);
        in_arena_.reset();
        for (size_t q = 0; q < specs.size(); ++q) {
            dev[q].a = (double *)in_arena_.take(7 * (size_t)specs[q].n * 8);
            CK(cudaMemcpyAsync(dev[q].a, specs[q].a, 7 * (size_t)specs[q].n * 8, cudaMemcpyDeviceToDevice, stream_));
        }
    }
    if (!opt.on_device) {
        size_t bytes = 4096;
        for (const auto &s : specs) bytes += align_up(7 * (size_t)s.n * 8, 256) + 2 * align_up((size_t)s.n * 8, 256);
        cudaError_t e = in_arena_.reserve(bytes);
        if (e != cudaSuccess) return fail(std::string("device memory for the inputs: ") + cudaGetErrorString(e), -11);
        in_arena_.reset();
        for (size_t q = 0; q < specs.size(); ++q) {
            const size_t n = (size_t)specs[q].n;
            dev[q].a = (double *)in_arena_.take(7 * n * 8);
            dev[q].b = (double *)in_arena_.take(n * 8);
            dev[q].x = (double *)in_arena_.take(n * 8);
            CK(cudaMemcpyAsync(dev[q].a, specs[q].a, 7 * n * 8, cudaMemcpyHostToDevice, stream_));
            CK(cudaMemcpyAsync(dev[q].b, specs[q].b, n * 8, cudaMemcpyHostToDevice, stream_));
            CK(cudaMemcpyAsync(dev[q].x, specs[q].x, n * 8, cudaMemcpyHostToDevice, stream_));
        }
    }
    SolveOptions o = opt;
    o.on_device = true;
    if (opt.method < 1 || opt.method > 5) return fail("LEQ_METHOD not served (1 SOR, 2 BiCGSTAB, 3 GMRES, 4, 5 CG)", -10);
    if ((opt.method == 1 || opt.method == 3 || opt.method == 4) && specs.size() != 1)
        return fail("METHOD 1, 3 and 4 serve single systems", -10);
    if (opt.method == 5 || opt.method == 3) o.precision = PREC_FP64;  // CG and GMRES run their FP64 form only
    writeback_.clear();
    if (!opt.on_device && opt.write_back_ab && opt.method != 3)  // GMRES leaves A and B as they are
        for (size_t q = 0; q < specs.size(); ++q) {
            const size_t n = (size_t)specs[q].n;
            if (!opt.transposed) writeback_.push_back({specs[q].a, dev[q].a, 7 * n * 8});
            writeback_.push_back({specs[q].b, dev[q].b, n * 8});
        }
    // several systems with red/black sweeps: a live batch, which drops systems
    // as they finish; otherwise the fixed batch (also the timed-kernel path)
    bool rs_only = true;
    for (int q = 0; q < 4; ++q) {
        const char ch = opt.sweep[q];
        if (ch == 'I' || ch == 'i' || ch == 'K' || ch == 'k' || ch == 'A' || ch == 'a') rs_only = false;
    }
    if (opt.method == 1) {  // LEQ_SOR: the scaling and one point-Jacobi step (model/leq_sor.f)
        const int64_t n = dev[0].n;
        SysDev d{};
        d.imax2 = dev[0].imax2;
        d.jmax2 = dev[0].jmax2;
        d.kmax2 = dev[0].kmax2;
        d.do_k = dev[0].do_k;
        d.cyc = dev[0].cyc;
        d.n = n;
        d.div_j = make_fastdiv((uint32_t)d.jmax2);
        d.div_i = make_fastdiv((uint32_t)d.imax2);
        d.jp = d.jmax2;
        d.np = n;
        d.div_jp = d.div_j;
        if (!d_one_sys_) CK(cudaMalloc((void **)&d_one_sys_, sizeof(SysDev)));
        CK(cudaMemcpyAsync(d_one_sys_, &d, sizeof(SysDev), cudaMemcpyHostToDevice, stream_));
        if ((size_t)n * 8 > gm_basis_bytes_) {  // VAR_tmp in the GMRES scratch
            cudaFree(gm_basis_);
            gm_basis_bytes_ = 0;
            if (cudaMalloc((void **)&gm_basis_, (size_t)n * 8) != cudaSuccess) {
                gm_basis_ = nullptr;
                cudaGetLastError();
                return fail("device memory for VAR_tmp", -11);
            }
            gm_basis_bytes_ = (size_t)n * 8;
        }
        timing_ = SolveTiming{};
        CK(cudaEventRecord(ev_t0_, stream_));
        const int grid = std::max(1, std::min((int)((n + 255) / 256), sms_ * 8));
        CK(launch_sor(d_one_sys_, dev[0].a, dev[0].b, dev[0].x, gm_basis_, dev[0].itmax, n, grid, stream_));
        CK(cudaEventRecord(ev_t1_, stream_));
        CK(cudaEventSynchronize(ev_t1_));
        cudaEventElapsedTime(&timing_.device_ms, ev_t0_, ev_t1_);
        timing_.kernel_launches = dev[0].itmax >= 1 ? 2 : 1;
        out[0] = SolveResult{};
        out[0].iterations = std::max(dev[0].itmax, 0) + 1;
        out[0].iter_tot_add = out[0].iterations;  // the value ITER_TOT(VNO) is set to (:119)
        out[0].exit_kind = EX_ITMAX;
        int rc = issue_writeback();
        if (rc) return rc;
        if (!opt.on_device) {
            CK(cudaMemcpyAsync(specs[0].x, dev[0].x, (size_t)n * 8, cudaMemcpyDeviceToHost, stream_));
            CK(cudaStreamSynchronize(stream_));
            CK(cudaStreamSynchronize(side_));
        }
        return 0;
    }
    if (opt.method == 3) {  // LEQ_GMRES
        int rc = run_gmres(dev[0], o, out[0]);
        if (rc) return rc;
        if (!opt.on_device) {
            CK(cudaMemcpyAsync(specs[0].x, dev[0].x, (size_t)specs[0].n * 8, cudaMemcpyDeviceToHost, stream_));
            CK(cudaStreamSynchronize(stream_));
        }
        return 0;
    }
    if (opt.method == 4) o.method = 2;  // BiCGSTAB first (model/solve_lin_eq.f:161-171)
    int rc = (specs.size() > 1 && rs_only && !opt.time_kernels && o.method == 2) ? run_batch_live(dev, o, out)
                                                                                 : run_batch(dev, o, out);
    if (rc) return rc;
    SolveTiming total = timing_;

    // mixed form: systems whose FP32 iteration gave up are solved again by the
    // FP64 drop-in, from their initial guess
    if (o.precision == PREC_MIXED) {
        std::vector<SystemSpec> fb;
        std::vector<int> idx;
        for (size_t q = 0; q < out.size(); ++q)
            if (out[q].exit_kind == EX_FALLBACK) {
                CK(cudaMemcpyAsync(dev[q].x, x0_[q], (size_t)dev[q].n * 8, cudaMemcpyDeviceToDevice,
                                   stream_));
                fb.push_back(dev[q]);
                idx.push_back((int)q);
            }
        if (!fb.empty()) {
            SolveOptions f = o;
            f.precision = PREC_FP64;
            f.skip_scale = true;
            std::vector<SolveResult> fo;
            rc = run_batch(fb, f, fo);
            if (rc) return rc;
            for (size_t q = 0; q < idx.size(); ++q) {
                const int mixed_its = out[idx[q]].iterations;
                out[idx[q]] = fo[q];
                out[idx[q]].fp64_fallback = 1;
                out[idx[q]].mixed_iterations = mixed_its;
            }
            total.device_ms += timing_.device_ms;
            total.jline_ms += timing_.jline_ms;
            total.jline_launches += timing_.jline_launches;
            total.kernel_launches += timing_.kernel_launches;
            for (int k = 0; k < KC_COUNT; ++k) {
                total.class_ms[k] += timing_.class_ms[k];
                total.class_launches[k] += timing_.class_launches[k];
            }
        }
    }
    timing_ = total;

    // METHOD 4: a BiCGSTAB breakdown (IER -2) continues with GMRES on the scaled
    // system from BiCGSTAB's VAR, IER reset to 0 first (model/solve_lin_eq.f:161-171)
    if (opt.method == 4 && out[0].ier == -2) {
        SolveOptions g = o;
        g.method = 3;
        g.precision = PREC_FP64;
        SolveResult gr;
        if ((rc = run_gmres(dev[0], g, gr))) return rc;
        gr.iter_tot_add = out[0].iter_tot_add;  // LEQ_BICGS's ITER_TOT; GMRES adds none
        out[0] = gr;
        timing_.device_ms += total.device_ms;
    }

    // results back to the caller's host arrays (A/B went back during the iterations)
    if ((rc = issue_writeback())) return rc;  // a batch that ended before issuing them
    if (!opt.on_device) {
        for (size_t q = 0; q < specs.size(); ++q) {
            const size_t n = (size_t)specs[q].n;
            CK(cudaMemcpyAsync(specs[q].x, dev[q].x, n * 8, cudaMemcpyDeviceToHost, stream_));
        }
        CK(cudaStreamSynchronize(stream_));
        CK(cudaStreamSynchronize(side_));
    }
    return 0;
}

// Queues the pending copy-back of the scaled A/B on the side stream, behind
// everything enqueued so far on the engine stream (the scaling).
int Engine::issue_writeback()
{
    if (writeback_.empty()) return 0;
    CK(cudaEventRecord(ev_setup_, stream_));
    CK(cudaStreamWaitEvent(side_, ev_setup_, 0));
    for (const Writeback &w : writeback_) CK(cudaMemcpyAsync(w.dst, w.src, w.bytes, cudaMemcpyDeviceToHost, side_));
    writeback_.clear();
    return 0;
}

// The per-system setup, each step gated on the system's phase (so it is a no-op
// for systems past it): unit scaling, J-line factors, FP32 copy or initial
// residual and Rtilde, entry to the loop.
int Engine::launch_setup(const SolveOptions &opt, bool scale)
{
    const bool mixed = opt.precision == PREC_MIXED;
    const bool cg = opt.method == 5;
    if (scale) {
        CK(cg ? launch_scale_diag(view_, cfg_) : launch_scale(view_, cfg_));
        CK(launch_after_scale(view_, cfg_));
        launches_ += 2;
    }
    if (opt.pc == PC_LINE) {
        CK(mixed ? launch_line_factor<float>(view_, cfg_, d_allprefix_, h_allprefix_[nsys_])
                 : launch_line_factor<double>(view_, cfg_, d_allprefix_, h_allprefix_[nsys_]));
        launches_ += 1;
    }
    if (mixed) {
        CK(launch_to_f32(view_, cfg_));
        CK(launch_defl_setup(view_, cfg_));
        launches_ += 2;
    } else if (cg) {  // R = B - A Var and Rnorm0 (model/leq_cg.f:236-259)
        CK(launch_init_residual<double>(view_, cfg_));
        launches_ += 1;
    } else {
        CK(launch_init_residual<double>(view_, cfg_));
        CK(launch_init_rtilde<double>(view_, cfg_, opt.seed));
        launches_ += 2;
    }
    CK(launch_init_done(view_, cfg_));
    launches_ += 1;
    return 0;
}

// One BiCGSTAB iteration for every system of the batch (model/leq_bicgs.f:316-466).
int Engine::launch_body(const SolveOptions &opt)
{
    const bool mixed = opt.precision == PREC_MIXED;
    const int src_ph = opt.pc == PC_NONE ? V_P : V_PH;
    const int src_sh = opt.pc == PC_NONE ? V_S : V_SH;
    int r;
    launches_ += (mixed ? 6 : 5) + 2 * (cfg_.rows_pair + cfg_.rows_single - 1);
#define TK(kc, call)  \
    do {              \
        kt_begin();   \
        CK(call);     \
        kt_end(kc);   \
    } while (0)
    if (opt.method == 5) {  // LEQ_CG0, model/leq_cg.f:271-410
        const int z_id = opt.pc == PC_NONE ? V_R : V_PH;
        if ((r = run_msolve_plan(0, 8))) return r;
        launches_ += 4 - ((mixed ? 6 : 5) + 2 * (cfg_.rows_pair + cfg_.rows_single - 1));
        TK(KC_S_UPDATE, launch_cg_rho(view_, cfg_, z_id));
        TK(KC_P_UPDATE, launch_cg_p(view_, cfg_, z_id));
        TK(KC_MATVEC_ALPHA, launch_cg_matvec(view_, cfg_));
        TK(KC_XR_UPDATE, launch_cg_xr(view_, cfg_));
    } else if (mixed) {
        TK(KC_OUTER, launch_outer_step(view_, cfg_));
        TK(KC_P_UPDATE, (launch_p_update<float, true>(view_, cfg_)));
        if ((r = run_msolve_plan(0, 4))) return r;
        TK(KC_MATVEC_ALPHA, (launch_matvec_alpha<float, true>(view_, cfg_, src_ph)));
        TK(KC_S_UPDATE, (launch_s_update<float, true>(view_, cfg_)));
        if ((r = run_msolve_plan(1, 4))) return r;
        TK(KC_MATVEC_OMEGA, (launch_matvec_omega<float, true>(view_, cfg_, src_sh)));
        TK(KC_XR_UPDATE, (launch_xr_update<float, true>(view_, cfg_, src_ph, src_sh)));
    } else {
        TK(KC_P_UPDATE, (launch_p_update<double, false>(view_, cfg_)));
        if ((r = run_msolve_plan(0, 8))) return r;
        TK(KC_MATVEC_ALPHA, (launch_matvec_alpha<double, false>(view_, cfg_, src_ph)));
        TK(KC_S_UPDATE, (launch_s_update<double, false>(view_, cfg_)));
        if ((r = run_msolve_plan(1, 8))) return r;
        TK(KC_MATVEC_OMEGA, (launch_matvec_omega<double, false>(view_, cfg_, src_sh)));
        TK(KC_XR_UPDATE, (launch_xr_update<double, false>(view_, cfg_, src_ph, src_sh)));
    }
#undef TK
    return 0;
}

// One batch whose arrays are all on the device.
int Engine::run_batch(const std::vector<SystemSpec> &specs, const SolveOptions &opt, std::vector<SolveResult> &out)
{
    out.assign(specs.size(), SolveResult{});
    const bool mixed = opt.precision == PREC_MIXED;
    const int elem = mixed ? 4 : 8;

    int rc = setup_batch(specs, opt);
    if (rc) return rc;
    const int gate_p = G_INNER, gate_s = G_INNER_NOSNORM;
    h_lines_.clear();
    list_refs_.clear();
    auto plans = [&]() -> int {
        int r;
        if (opt.method == 5) return plan_msolve(opt, V_R, V_PH, gate_p, 0);  // Z = MSOLVE(R)
        if ((r = plan_msolve(opt, V_P, V_PH, gate_p, 0))) return r;
        return plan_msolve(opt, V_S, V_SH, gate_s, 1);
    };
    if ((rc = plans())) return rc;
    if ((rc = bind_lists())) return rc;

    ktime_ = opt.time_kernels;
    kt_count_ = 0;
    launches_ = 0;
    timing_ = SolveTiming{};
    CK(cudaEventRecord(ev_t0_, stream_));

    // ---- setup
    if ((rc = launch_setup(opt, !opt.skip_scale))) return rc;
    if ((rc = issue_writeback())) return rc;
    if (opt.pc == PC_LINE && opt.autotune && opt.force_lanes <= 0) {
        bool rs_only = true;
        for (int q = 0; q < 4; ++q) {
            const char ch = opt.sweep[q];
            if (ch == 'I' || ch == 'i' || ch == 'K' || ch == 'k' || ch == 'A' || ch == 'a') rs_only = false;
        }
        if (rs_only) {
            if ((rc = autotune_lines(opt, elem))) return rc;
            h_lines_.clear();
            list_refs_.clear();
            if ((rc = plans())) return rc;
            if ((rc = bind_lists())) return rc;
        }
    }

    auto body = [&]() -> int { return launch_body(opt); };

    int max_itmax = 0;
    for (const auto &s : specs) max_itmax = std::max(max_itmax, s.itmax);
    const int max_loops = std::max(1, max_itmax + 2);
    const bool graph = opt.use_graph && !ktime_;
    cudaGraphExec_t gexec = nullptr;
    long long per_body = 0;
    if (graph) {
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        const long long before = launches_;
        rc = body();
        per_body = launches_ - before;
        launches_ = before;
        cudaError_t ce = cudaStreamEndCapture(stream_, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ce != cudaSuccess) return fail(std::string("graph capture: ") + cudaGetErrorString(ce), -13);
        ce = cudaGraphInstantiate(&gexec, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) return fail(std::string("graph instantiate: ") + cudaGetErrorString(ce), -13);
    }
    auto run_once = [&]() -> int {
        if (graph) {
            CK(cudaGraphLaunch(gexec, stream_));
            launches_ += per_body;
            return 0;
        }
        return body();
    };

    // Timed kernels: the state is read after every iteration (still one
    // snapshot behind, so that the stream never drains and no host latency
    // enters the intervals): at most two iterations run after the last system
    // is done, and their launches return at once.
    const int K = ktime_ ? 1 : std::max(1, opt.check_every);
    int loops = 0, snap = 0;
    bool have_prev = false, finished = false;
    while (loops < max_loops && !finished) {
        for (int q = 0; q < K && loops < max_loops; ++q, ++loops)
            if ((rc = run_once())) {
                if (gexec) cudaGraphExecDestroy(gexec);
                return rc;
            }
        CK(launch_state_snapshot(d_st_, d_st_mapped_ + (size_t)(snap & 1) * nsys_, nsys_, stream_));
        ++launches_;
        CK(cudaEventRecord((snap & 1) ? ev_b_ : ev_a_, stream_));
        if (have_prev) {
            const int prev = (snap - 1) & 1;
            CK(cudaEventSynchronize(prev ? ev_b_ : ev_a_));
            const SysState *pb = h_st_pinned_ + (size_t)prev * nsys_;
            finished = true;
            for (int s = 0; s < nsys_; ++s)
                if (pb[s].status == ST_RUNNING) {
                    finished = false;
                    break;
                }
        }
        have_prev = true;
        ++snap;
    }
    if (gexec) cudaGraphExecDestroy(gexec);
    CK(cudaEventRecord(ev_t1_, stream_));
    CK(cudaStreamSynchronize(stream_));
    CK(cudaMemcpy(h_st_.data(), d_st_, sizeof(SysState) * nsys_, cudaMemcpyDeviceToHost));
    cudaEventElapsedTime(&timing_.device_ms, ev_t0_, ev_t1_);
    timing_.kernel_launches = launches_;

    // ---- results back
    for (int s = 0; s < nsys_; ++s) out[s] = result_of(h_st_[s], mixed);
    CK(cudaStreamSynchronize(stream_));
    if (ktime_) kt_harvest();
    return 0;
}

// ------------------------------------------------------------------ LEQ_GMRES
// GMRES(ITMAX) with one restart cycle (MAX_IT = 1, model/solve_lin_eq.f:86),
// left-preconditioned by LEQ_MSOLVE with the sweep letters; A and B are not
// scaled (model/leq_gmres.f:17-584).  The vector work runs on the device (matvec,
// the J-line sweeps, fused modified Gram-Schmidt passes with deterministic
// sums); the Hessenberg column comes to the host once per step, where the Givens
// rotations (ROTMAT, :593-628), the convergence test and the back substitution
// run in FP64 as in the reference.  IER 0, or 1 when not converged.
int Engine::run_gmres(const SystemSpec &s, const SolveOptions &opt, SolveResult &r)
{
    r = SolveResult{};
    SolveOptions o = opt;
    o.method = 3;
    o.precision = PREC_FP64;
    o.skip_scale = true;
    o.pc = PC_LINE;  // LEQ_GMRES always preconditions with LEQ_MSOLVE (model/leq_gmres.f:73-74)
    const int64_t n = s.n;
    const int M = std::max(0, s.itmax);
    const int grid = std::max(1, std::min((int)((n + 255) / 256), sms_ * 8));
    ktime_ = false;
    timing_ = SolveTiming{};
    cudaEvent_t t0, t1;
    CK(cudaEventCreate(&t0));
    CK(cudaEventCreate(&t1));
    CK(cudaEventRecord(t0, stream_));
    launches_ = 0;

    // B = 0: Var = 0 and nothing else (:64-70)
    if (!gm_max_) CK(cudaMalloc((void **)&gm_max_, sizeof(unsigned long long)));
    CK(cudaMemsetAsync(gm_max_, 0, sizeof(unsigned long long), stream_));
    CK(launch_gm_maxabs(s.b, n, gm_max_, grid, stream_));
    unsigned long long bmax = 0;
    CK(cudaMemcpyAsync(&bmax, gm_max_, sizeof bmax, cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    launches_ += 1;
    if (bmax == 0) {
        CK(cudaMemsetAsync(s.x, 0, (size_t)n * 8, stream_));
        r.exit_kind = EX_RHO0;
        CK(cudaEventRecord(t1, stream_));
        CK(cudaEventSynchronize(t1));
        cudaEventElapsedTime(&timing_.device_ms, t0, t1);
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        timing_.kernel_launches = launches_;
        return 0;
    }
    // the system's tables and work vectors, the J-line factors, the sweep plan
    int rc = setup_batch({s}, o);
    if (rc) return rc;
    h_lines_.clear();
    list_refs_.clear();
    if ((rc = plan_msolve(o, V_T, V_S, G_INNER, 0))) return rc;  // WW = MSOLVE(TEMP)
    if ((rc = bind_lists())) return rc;
    CK(launch_line_factor<double>(view_, cfg_, d_allprefix_, h_allprefix_[nsys_]));
    CK(launch_init_done(view_, cfg_));
    launches_ += 2;
    const SysDev &d = h_sys_[0];
    double *T = (double *)d.vec[V_T], *W = (double *)d.vec[V_S];
    const size_t basis = (size_t)(M + 1) * (size_t)n * 8;
    if (basis > gm_basis_bytes_) {
        cudaFree(gm_basis_);
        gm_basis_ = nullptr;
        gm_basis_bytes_ = 0;
        if (cudaMalloc((void **)&gm_basis_, basis) != cudaSuccess) {
            cudaGetLastError();
            return fail("device memory for the GMRES basis ((ITMAX+1) x DIMENSION_3 doubles)", -11);
        }
        gm_basis_bytes_ = basis;
    }
    const int need = grid + M + 2 + std::max(M, 1);
    if (need > gm_scal_cap_) {
        cudaFree(gm_scal_);
        CK(cudaMalloc((void **)&gm_scal_, sizeof(double) * (size_t)need));
        gm_scal_cap_ = need;
    }
    double *partials = gm_scal_, *dh = gm_scal_ + grid, *dy = dh + M + 2;
    double *V = gm_basis_;
    auto norm2 = [&](const double *x, const double *y, double *out) -> int {
        CK(launch_gm_mgs(const_cast<double *>(x), nullptr, nullptr, y, n, partials, grid, stream_));
        CK(launch_gm_sum(partials, grid, dh, stream_));
        CK(cudaMemcpyAsync(out, dh, sizeof(double), cudaMemcpyDeviceToHost, stream_));
        CK(cudaStreamSynchronize(stream_));
        launches_ += 2;
        return 0;
    };
    // R = MSOLVE(B - A Var) into W (:220-239)
    auto residual = [&]() -> int {
        CK(launch_matvec_plain<double>(view_.sys, d, s.a, s.x, T, stream_, grid));
        CK(launch_gm_sub(s.b, T, n, grid, stream_));
        launches_ += 2;
        return run_msolve_plan(0, 8);
    };
    // back substitution of H(1:m,1:m) y = SS(1:m) and Var += V(:,1:m) y (:361-426)
    std::vector<double> H((size_t)(M + 1) * std::max(M, 1), 0.0), cs(M + 1, 0.0), sn(M + 1, 0.0), ss(M + 2, 0.0);
    const int ldh = M + 1;
    auto update = [&](int m) -> int {
        std::vector<double> y(std::max(m, 1), 0.0);
        for (int i = 0; i < m; ++i) y[i] = ss[i];
        for (int i = m - 1; i >= 0; --i) {
            const double yi = y[i] / H[i + (size_t)i * ldh];
            y[i] = yi;
            for (int j = 0; j < i; ++j) y[j] = y[j] - H[j + (size_t)i * ldh] * yi;
        }
        if (m > 0) {
            CK(cudaMemcpyAsync(dy, y.data(), sizeof(double) * (size_t)m, cudaMemcpyHostToDevice, stream_));
            CK(launch_gm_update(s.x, V, dy, m, n, grid, stream_));
            launches_ += 1;
        }
        return 0;
    };

    double bb = 0.0;
    if ((rc = norm2(s.b, s.b, &bb))) return rc;
    double bnrm2 = std::sqrt(bb);
    if (bnrm2 == 0.0) bnrm2 = 1.0;
    if ((rc = residual())) return rc;
    double rr = 0.0;
    if ((rc = norm2(W, W, &rr))) return rc;
    double norm_r = std::sqrt(rr);
    double error = norm_r / bnrm2;
    const double error0 = error;
    const double rnorm0 = norm_r;
    // the single restart cycle (:255-540); its opening residual equals the one above
    CK(launch_gm_scale(W, 1.0 / norm_r, V, n, grid, stream_));
    launches_ += 1;
    ss[0] = norm_r;
    int steps = 0;
    bool converged = false;
    std::vector<double> h(M + 2, 0.0);
    for (int i = 0; i < M && !converged; ++i) {
        double *vi = V + (size_t)i * n;
        CK(launch_matvec_plain<double>(view_.sys, d, s.a, vi, T, stream_, grid));
        launches_ += 1;
        if ((rc = run_msolve_plan(0, 8))) return rc;  // WW = MSOLVE(A V(:,I)) (:297-298)
        // modified Gram-Schmidt, each axpy fused with the next dot (:299-322)
        for (int k = 0; k <= i; ++k) {
            CK(launch_gm_mgs(W, k ? V + (size_t)(k - 1) * n : nullptr, dh + k - 1, V + (size_t)k * n, n, partials, grid,
                             stream_));
            CK(launch_gm_sum(partials, grid, dh + k, stream_));
        }
        CK(launch_gm_mgs(W, vi, dh + i, W, n, partials, grid, stream_));
        CK(launch_gm_sum(partials, grid, dh + i + 1, stream_));
        launches_ += 2 * (i + 2);
        CK(cudaMemcpyAsync(h.data(), dh, sizeof(double) * (size_t)(i + 2), cudaMemcpyDeviceToHost, stream_));
        CK(cudaStreamSynchronize(stream_));
        double *col = H.data() + (size_t)i * ldh;
        for (int k = 0; k <= i; ++k) col[k] = h[k];
        col[i + 1] = std::sqrt(h[i + 1]);  // NORM_W
        CK(launch_gm_scale(W, 1.0 / col[i + 1], V + (size_t)(i + 1) * n, n, grid, stream_));
        launches_ += 1;
        for (int k = 0; k < i; ++k) {  // earlier rotations (:329-333)
            const double t = cs[k] * col[k] + sn[k] * col[k + 1];
            col[k + 1] = -sn[k] * col[k] + cs[k] * col[k + 1];
            col[k] = t;
        }
        // ROTMAT (:593-628)
        const double a = col[i], b = col[i + 1];
        if (b == 0.0) {
            cs[i] = 1.0;
            sn[i] = 0.0;
        } else if (std::fabs(b) > std::fabs(a)) {
            const double t = a / b;
            sn[i] = 1.0 / std::sqrt(1.0 + t * t);
            cs[i] = t * sn[i];
        } else {
            const double t = b / a;
            cs[i] = 1.0 / std::sqrt(1.0 + t * t);
            sn[i] = t * cs[i];
        }
        const double t = cs[i] * ss[i];
        ss[i + 1] = -sn[i] * ss[i];
        ss[i] = t;
        col[i] = cs[i] * col[i] + sn[i] * col[i + 1];
        col[i + 1] = 0.0;
        error = std::fabs(ss[i + 1]) / bnrm2;
        steps = i + 1;
        if (error <= s.tol * error0) {  // (:352-360)
            if ((rc = update(i + 1))) return rc;
            converged = true;
        }
    }
    if (!converged) {  // ITMAX steps: update with them all, then the new residual (:445-540)
        if ((rc = update(M))) return rc;
        if ((rc = residual())) return rc;
        if ((rc = norm2(W, W, &rr))) return rc;
        norm_r = std::sqrt(rr);
        error = norm_r / bnrm2;
    }
    CK(cudaEventRecord(t1, stream_));
    CK(cudaEventSynchronize(t1));
    cudaEventElapsedTime(&timing_.device_ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    timing_.kernel_launches = launches_;
    r.ier = error > s.tol * error0 ? 1 : 0;
    r.iterations = steps;
    r.exit_kind = r.ier ? EX_ITMAX : EX_RNORM;
    r.rnorm0 = rnorm0;
    r.rnorm = error * bnrm2;
    r.line_skips = 0;
    return 0;
}

// ------------------------------------------------------------------ per-routine entry points
int Engine::matvec(const SystemSpec &g, const double *a, const double *x, double *y)
{
    SysDev d{};
    d.imax2 = g.imax2;
    d.jmax2 = g.jmax2;
    d.kmax2 = g.kmax2;
    d.do_k = g.do_k;
    d.cyc = g.cyc;
    d.n = g.n;
    d.div_j = make_fastdiv((uint32_t)g.jmax2);
    d.div_i = make_fastdiv((uint32_t)g.imax2);
    d.jp = g.jmax2;
    d.np = g.n;
    d.div_jp = d.div_j;
    if (!d_one_sys_) CK(cudaMalloc((void **)&d_one_sys_, sizeof(SysDev)));
    CK(cudaMemcpyAsync(d_one_sys_, &d, sizeof(SysDev), cudaMemcpyHostToDevice, stream_));
    const int grid = std::max(1, std::min((int)((g.n + CELL_THREADS - 1) / CELL_THREADS), sms_ * 8));
    CK(launch_matvec_plain<double>(d_one_sys_, d, a, x, y, stream_, grid));
    CK(cudaStreamSynchronize(stream_));
    return 0;
}

int Engine::dot(const double *x, const double *y, int64_t n, double *out_host)
{
    const int grid = std::max(1, std::min((int)((n + 4095) / 4096), sms_ * 4));
    if (!d_dot_partials_) {
        CK(cudaMalloc((void **)&d_dot_partials_, sizeof(double) * (size_t)sms_ * 4));
        CK(cudaMalloc((void **)&d_dot_counter_, sizeof(unsigned int)));
        CK(cudaMalloc((void **)&d_dot_out_, sizeof(double)));
        CK(cudaMemsetAsync(d_dot_counter_, 0, sizeof(unsigned int), stream_));
    }
    CK(launch_dot(x, y, n, d_dot_partials_, d_dot_counter_, d_dot_out_, grid, stream_));
    CK(cudaMemcpyAsync(out_host, d_dot_out_, sizeof(double), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    return 0;
}

// One LEQ_MSOLVE on device arrays: var = M^{-1} b (the J-line kernels run over a
// one-system batch whose P / P_preconditioned slots point at b / var).
int Engine::msolve(const SystemSpec &g, const double *a, const double *b, double *var, int pc, const char sweep[4])
{
    SolveOptions opt;
    opt.pc = pc;
    std::memcpy(opt.sweep, sweep, 4);
    opt.on_device = true;
    SystemSpec s = g;
    s.a = const_cast<double *>(a);
    s.b = const_cast<double *>(b);
    s.x = var;
    if (!aligned16(s)) return fail("device arrays must start on 16-byte boundaries (cudaMalloc gives 256)", -14);
    std::vector<SystemSpec> one{s};
    int rc = setup_batch(one, opt);
    if (rc) return rc;
    h_sys_[0].vec[V_P] = const_cast<double *>(b);
    h_sys_[0].vec[V_PH] = var;
    CK(cudaMemcpyAsync(d_sys_, h_sys_.data(), sizeof(SysDev), cudaMemcpyHostToDevice, stream_));
    h_lines_.clear();
    list_refs_.clear();
    if ((rc = plan_msolve(opt, V_P, V_PH, G_ANY, 0))) return rc;
    if ((rc = bind_lists())) return rc;
    if (pc == PC_NONE) CK(cudaMemcpyAsync(var, b, (size_t)g.n * 8, cudaMemcpyDeviceToDevice, stream_));
    if (pc == PC_LINE) {
        h_st_[0].phase = PH_INIT;  // the factorization kernel serves systems in their setup
        CK(cudaMemcpyAsync(d_st_, h_st_.data(), sizeof(SysState), cudaMemcpyHostToDevice, stream_));
        CK(launch_line_factor<double>(view_, cfg_, d_allprefix_, h_allprefix_[nsys_]));
    }
    if ((rc = run_msolve_plan(0, 8))) return rc;
    CK(cudaStreamSynchronize(stream_));
    CK(cudaMemcpy(h_st_.data(), d_st_, sizeof(SysState), cudaMemcpyDeviceToHost));
    if (h_st_[0].err & 2) return fail("DGTSV reported INFO != 0 in a JK/IJ sweep", -12);
    return 0;
}

}  // namespace mfixgpu
