// leq_live.cu -- the engine's live batch: continuous batching of LEQ_BICGS solves.
//
// A live batch is a fixed table of slots.  Systems join and leave between
// iterations; each join or leave rebuilds the small batch tables (cell tiles,
// line-work prefixes, partial-sum slots), re-captures the iteration body as a
// CUDA graph and launches the gated setup kernels, which only touch systems
// still in their setup phases.  A system therefore runs exactly the kernel
// sequence it runs when solved alone (setup, then one body per iteration, its
// reductions over its own tiles in a fixed order), and its result is the same
// bits in a mix as alone.
#include "leq_engine.h"

#include <algorithm>
#include <cstring>

namespace mfixgpu {

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return fail(std::string(#call) + ": " + cudaGetErrorString(e_), -13); \
    } while (0)

// An empty slot: no cells, no tiles, no line work; its state is never running.
static SysDev idle_sys()
{
    SysDev d{};
    d.imax2 = d.jmax2 = d.kmax2 = 1;
    d.do_k = 1;
    d.n = 0;
    d.jp = 1;
    d.np = 0;
    d.div_j = d.div_i = d.div_h = d.div_jp = make_fastdiv(1);
    d.pc = PC_NONE;
    d.lane_group = 32;
    d.line_kind = LK_WARP;
    d.rows_per_lane = 1;
    d.half_lines = 1;
    return d;
}

static SysState idle_state()
{
    SysState s{};
    s.status = ST_DONE;
    s.exit_kind = EX_ERROR;
    return s;
}

int Engine::live_open(int capacity, const SolveOptions &opt)
{
    err_.clear();
    if (capacity < 1 || capacity > 65536) return fail("live batch capacity must be 1..65536", -14);
    if (opt.pc != PC_LINE && opt.pc != PC_DIAG && opt.pc != PC_NONE) return fail("unknown preconditioner", -10);
    for (int q = 0; q < 4; ++q) {
        const char ch = opt.sweep[q];
        if (ch == 'I' || ch == 'i' || ch == 'K' || ch == 'k' || ch == 'A' || ch == 'a')
            return fail("sweep letters I/K/A are served for single-system solves only", -10);
    }
    live_opt_ = opt;
    live_opt_.on_device = true;
    live_opt_.time_kernels = false;
    // graphs of an earlier live batch on this engine
    CK(cudaStreamSynchronize(stream_));
    for (auto &r : retired_execs_) cudaGraphExecDestroy(r.first);
    retired_execs_.clear();
    if (live_exec_) cudaGraphExecDestroy(live_exec_);
    live_exec_ = nullptr;
    const bool mixed = opt.precision == PREC_MIXED;

    nsys_ = capacity;
    h_sys_.assign(capacity, idle_sys());
    h_st_.assign(capacity, idle_state());
    slot_used_.assign(capacity, 0);
    slot_fresh_.assign(capacity, 0);
    slot_reported_.assign(capacity, 0);
    slot_cleared_.assign(capacity, 0);
    slot_sys_.assign(capacity, LiveSystem{});
    slot_join_snap_.assign(capacity, 0);
    slot_join_body_.assign(capacity, 0);
    live_used_ = 0;
    snap_count_ = body_total_ = commits_ = 0;
    collected_upto_ = -1;

    h_tiles_.clear();
    h_allprefix_.assign(capacity + 1, 0);
    if (upload(&d_st_, &st_cap_, h_st_.data(), h_st_.size(), stream_) != cudaSuccess ||
        upload(&d_tiles_, &tiles_cap_, h_tiles_.data(), 0, stream_) != cudaSuccess ||
        upload(&d_allprefix_, &allprefix_cap_, h_allprefix_.data(), h_allprefix_.size(), stream_) != cudaSuccess)
        return fail("device memory for the live batch tables", -11);
    if (!d_partials_) {
        CK(cudaMalloc((void **)&d_partials_, 2 * 1024 * sizeof(double)));
        part_cap_ = 2 * 1024;
    }
    {
        const int rs = reserve_snapshots(2 * (size_t)capacity);
        if (rs) return rs;
    }
    if (!ev_fence_) CK(cudaEventCreateWithFlags(&ev_fence_, cudaEventDisableTiming));
    for (int q = 0; q < 2; ++q) {
        if (!ev_c0_[q]) CK(cudaEventCreate(&ev_c0_[q]));
        if (!ev_c1_[q]) CK(cudaEventCreate(&ev_c1_[q]));
    }
    busy_ms_ = 0.0;
    view_.st = d_st_;
    view_.tiles = d_tiles_;
    view_.ntiles = 0;
    view_.nsys = capacity;
    view_.partials = d_partials_;
    cfg_.stream = stream_;
    int rc = configure_lines(mixed ? 4 : 8);
    if (rc) return rc;

    // the sweep plans of R/S sweeps depend on no system: built once
    h_lines_.clear();
    list_refs_.clear();
    if ((rc = plan_msolve(live_opt_, V_P, V_PH, G_INNER, 0))) return rc;
    if ((rc = plan_msolve(live_opt_, V_S, V_SH, G_INNER_NOSNORM, 1))) return rc;
    if ((rc = bind_lists())) return rc;
    live_dirty_ = false;
    CK(cudaEventRecord(ev_fence_, stream_));
    return 0;
}

int Engine::live_add(const LiveSystem &ls)
{
    const SystemSpec &sp = ls.dev;
    if (slot_used_.empty()) return fail("live batch not open", -14);
    if (sp.imax2 < 1 || sp.jmax2 < 1 || sp.kmax2 < 1) return fail("grid extents must be >= 1", -14);
    if (!sp.do_k && sp.kmax2 != 1) return fail("a 2-D system (do_k = 0) needs kmax2 = 1", -14);
    if ((int64_t)sp.imax2 * sp.jmax2 * sp.kmax2 != sp.n) return fail("DIMENSION_3 != IMAX2*JMAX2*KMAX2", -14);
    if (sp.n > (int64_t)INT32_MAX - TILE_CELLS) return fail("system too large for 32-bit cell indexing", -14);
    if (!sp.a || !sp.b || !sp.x || !ls.work) return fail("null array", -14);
    if (!aligned16(sp) || ((uintptr_t)ls.work & 255))
        return fail("device arrays must start on 16-byte boundaries (work blocks on 256)", -14);
    int slot = -1;
    for (int s = 0; s < (int)slot_used_.size() && slot < 0; ++s)
        if (!slot_used_[s]) slot = s;
    if (slot < 0) return fail("live batch full", -11);

    const int prec = live_opt_.precision;
    const bool mixed = prec == PREC_MIXED;
    SysDev d{};
    d.imax2 = sp.imax2;
    d.jmax2 = sp.jmax2;
    d.kmax2 = sp.kmax2;
    d.do_k = sp.do_k;
    d.cyc = sp.cyc;
    d.n = sp.n;
    d.div_j = make_fastdiv((uint32_t)sp.jmax2);
    d.div_i = make_fastdiv((uint32_t)sp.imax2);
    d.jp = form_pitch(sp.jmax2, prec);
    d.np = (int64_t)d.jp * sp.imax2 * sp.kmax2;
    d.div_jp = make_fastdiv((uint32_t)d.jp);
    d.pc = live_opt_.pc;
    d.ntiles = (int)((std::max(sp.n, d.np) + TILE_CELLS - 1) / TILE_CELLS);
    shape_for(sp.jmax2, mixed ? 4 : 8, live_opt_.force_lanes, &d.lane_group, &d.rows_per_lane, &d.line_kind);
    d.half_lines = (sp.imax2 + 1) / 2;
    d.div_h = make_fastdiv((uint32_t)d.half_lines);
    d.a64 = sp.a;
    d.b64 = sp.b;
    d.x64[0] = sp.x;
    const int64_t lines = (int64_t)sp.imax2 * sp.kmax2;
    char *x0 = !mixed      ? nullptr
               : ls.x0_slot ? ls.x0_slot
                            : ls.work + std::max(vec_region_bytes(sp.n, lines, PREC_FP64),
                                                 vec_region_bytes(sp.n, lines, PREC_MIXED));
    carve_work(d, ls.work, lines, prec, x0);

    SysState st{};
    st.tol = sp.tol;
    st.itmax = sp.itmax;
    st.status = ST_RUNNING;
    st.phase = ls.scaled ? PH_INIT : PH_SETUP;
    st.mixed = mixed ? 1 : 0;
    st.method = live_opt_.method;
    st.inner_tol = live_opt_.inner_tol;
    st.growth_limit = live_opt_.mixed_growth;
    st.stall_limit = live_opt_.mixed_stalls;
    st.min_margin = live_opt_.mixed_min_margin;
    st.defl_allow = live_opt_.deflate ? 1 : 0;
    st.replace_every = live_opt_.replace_every;
    st.icheck = (live_opt_.minimize_dotproducts && !st.mixed)
                    ? (live_opt_.transposed ? 5 : std::max(1, live_opt_.icheck_bicgs))
                    : 0;
    st.restart_growth = live_opt_.restart_growth;
    st.margin_bits = 0x7f800000u;
    st.i = 1;
    st.iter = 1;

    h_sys_[slot] = d;
    h_st_[slot] = st;
    slot_sys_[slot] = ls;
    slot_used_[slot] = 1;
    slot_fresh_[slot] = 1;
    slot_reported_[slot] = 0;
    slot_cleared_[slot] = 0;
    ++live_used_;
    live_dirty_ = true;
    return slot;
}

void Engine::live_remove(int slot)
{
    if (slot < 0 || slot >= (int)slot_used_.size() || !slot_used_[slot]) return;
    slot_used_[slot] = 0;
    slot_fresh_[slot] = 0;
    slot_cleared_[slot] = 1;
    h_sys_[slot] = idle_sys();
    h_st_[slot] = idle_state();
    slot_sys_[slot] = LiveSystem{};
    --live_used_;
    live_dirty_ = true;
}

int Engine::live_commit()
{
    const int cap = (int)slot_used_.size();
    const bool mixed = live_opt_.precision == PREC_MIXED;
    bool any_fresh = false;

    // states of the slots that changed hands; the copies are stream ordered
    // after every kernel already enqueued
    size_t ntiles = 0;
    for (int s = 0; s < cap; ++s)
        if (slot_used_[s]) ntiles += h_sys_[s].ntiles;
    CK(stage_open(sizeof(SysState) * cap + sizeof(Tile) * ntiles + sizeof(int) * (cap + 1) + 1024));
    for (int s = 0; s < cap; ++s) {
        if (slot_cleared_[s]) {
            CK(stage_copy(d_st_ + s, &h_st_[s], 1));
            slot_cleared_[s] = 0;
        }
        if (!slot_fresh_[s]) continue;
        any_fresh = true;
        const LiveSystem &ls = slot_sys_[s];
        const size_t n = (size_t)ls.dev.n;
        if (ls.after) CK(cudaStreamWaitEvent(stream_, ls.after, 0));
        if (ls.x0) CK(cudaMemcpyAsync(ls.dev.x, ls.x0, n * 8, cudaMemcpyDeviceToDevice, stream_));
        if (mixed) CK(cudaMemcpyAsync(h_sys_[s].x64[1], ls.dev.x, n * 8, cudaMemcpyDeviceToDevice, stream_));
        CK(stage_copy(d_st_ + s, &h_st_[s], 1));
    }

    // tables of the systems now in the batch
    h_tiles_.clear();
    h_allprefix_.assign(cap + 1, 0);
    int tile_base = 0;
    for (int s = 0; s < cap; ++s) {
        SysDev &d = h_sys_[s];
        d.tile_base = tile_base;
        if (slot_used_[s]) {
            for (int t = 0; t < d.ntiles; ++t) h_tiles_.push_back(Tile{s, t});
            tile_base += d.ntiles;
        }
        h_allprefix_[s + 1] = h_allprefix_[s] + (slot_used_[s] ? d.imax2 * d.kmax2 : 0);
    }
    CK(upload_staged(&d_tiles_, &tiles_cap_, h_tiles_.data(), h_tiles_.size()));
    CK(upload_staged(&d_allprefix_, &allprefix_cap_, h_allprefix_.data(), h_allprefix_.size()));
    CK(stage_close());
    const size_t need_part = 2 * (size_t)std::max(tile_base, 1);
    if (need_part > part_cap_) {
        cudaFree(d_partials_);  // waits for the kernels that still use it
        d_partials_ = nullptr;
        const size_t want = std::max(need_part, part_cap_ * 2);
        CK(cudaMalloc((void **)&d_partials_, want * sizeof(double)));
        part_cap_ = want;
    }
    view_.st = d_st_;
    view_.tiles = d_tiles_;
    view_.ntiles = (int)h_tiles_.size();
    view_.nsys = cap;
    view_.partials = d_partials_;
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
    if (mixed && live_opt_.staged_matvec >= 1 && live_opt_.staged_matvec <= MV_SHAPES && oc.matvec_staged[live_opt_.staged_matvec] > 0) {
        cfg_.mv_staged = live_opt_.staged_matvec;
        cfg_.g_mv_staged = grid(oc.matvec_staged[live_opt_.staged_matvec]);
    }
    cfg_.g_copy = grid(oc.copy);
    cfg_.g_outer = grid(oc.outer);
    int rc = configure_lines(mixed ? 4 : 8);
    if (rc) return rc;

    // setup of the systems that joined (gated: a no-op for the others)
    if (any_fresh && (rc = launch_setup(live_opt_, true))) return rc;
    // new line lengths: lanes per line picked by measurement (one-shot batches)
    if (any_fresh && live_tune_ && (rc = autotune_lines(live_opt_, mixed ? 4 : 8))) return rc;

    // the iteration body for this membership
    if (live_exec_) retired_execs_.push_back({live_exec_, snap_count_});  // its launches may still run
    live_exec_ = nullptr;
    if (live_used_ > 0 && live_opt_.use_graph) {
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        const long long before = launches_;
        rc = launch_body(live_opt_);
        live_per_body_ = launches_ - before;
        launches_ = before;
        cudaError_t ce = cudaStreamEndCapture(stream_, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ce != cudaSuccess) return fail(std::string("graph capture: ") + cudaGetErrorString(ce), -13);
        ce = cudaGraphInstantiate(&live_exec_, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) return fail(std::string("graph instantiate: ") + cudaGetErrorString(ce), -13);
    }

    for (int s = 0; s < cap; ++s)
        if (slot_fresh_[s]) {
            slot_fresh_[s] = 0;
            slot_join_snap_[s] = snap_count_;
            slot_join_body_[s] = body_total_;
        }
    CK(cudaEventRecord(ev_fence_, stream_));
    live_dirty_ = false;
    ++commits_;
    return 0;
}

int Engine::live_step(int iterations)
{
    if (slot_used_.empty()) return fail("live batch not open", -14);
    int rc;
    const int b = (int)(snap_count_ & 1);
    CK(cudaEventRecord(ev_c0_[b], stream_));
    if (live_dirty_ && (rc = live_commit())) return rc;
    if (live_used_ == 0 || iterations <= 0) return 0;
    for (int q = 0; q < iterations; ++q) {
        if (live_exec_) {
            CK(cudaGraphLaunch(live_exec_, stream_));
            launches_ += live_per_body_;
        } else if ((rc = launch_body(live_opt_))) {
            return rc;
        }
    }
    body_total_ += iterations;
    const int cap = (int)slot_used_.size();
    CK(cudaEventRecord(ev_c1_[b], stream_));
    CK(launch_state_snapshot(d_st_, d_st_mapped_ + (size_t)b * cap, cap, stream_));
    ++launches_;
    CK(cudaEventRecord(b ? ev_b_ : ev_a_, stream_));
    snap_bodies_[b] = body_total_;
    ++snap_count_;
    return 0;
}

int Engine::live_collect(std::vector<LiveDone> &done, bool latest)
{
    const long long q = latest ? snap_count_ - 1 : snap_count_ - 2;
    if (q < 0 || q <= collected_upto_) return 0;
    const int b = (int)(q & 1);
    CK(cudaEventSynchronize(b ? ev_b_ : ev_a_));
    return live_take(q, done);
}

int Engine::live_collect_ready(std::vector<LiveDone> &done, bool *collected)
{
    *collected = false;
    const long long q = collected_upto_ + 1;
    if (q >= snap_count_) return 0;
    const int b = (int)(q & 1);
    const cudaError_t e = cudaEventQuery(b ? ev_b_ : ev_a_);
    if (e == cudaErrorNotReady) return 0;
    if (e != cudaSuccess) return fail(std::string("state snapshot: ") + cudaGetErrorString(e), -13);
    *collected = true;
    return live_take(q, done);
}

// Reads snapshot q (complete): finished systems, busy time, retired graphs.
int Engine::live_take(long long q, std::vector<LiveDone> &done)
{
    const int b = (int)(q & 1);
    float chunk_ms = 0.f;
    if (cudaEventElapsedTime(&chunk_ms, ev_c0_[b], ev_c1_[b]) == cudaSuccess) busy_ms_ += chunk_ms;
    cudaGetLastError();
    // snapshot q follows every launch of the graphs retired before it was taken
    for (size_t r = 0; r < retired_execs_.size();)
        if (retired_execs_[r].second <= q) {
            cudaGraphExecDestroy(retired_execs_[r].first);
            retired_execs_[r] = retired_execs_.back();
            retired_execs_.pop_back();
        } else {
            ++r;
        }
    const int cap = (int)slot_used_.size();
    const bool mixed = live_opt_.precision == PREC_MIXED;
    const SysState *ps = h_st_pinned_ + (size_t)b * cap;
    for (int s = 0; s < cap; ++s) {
        if (!slot_used_[s] || slot_reported_[s] || slot_fresh_[s] || q < slot_join_snap_[s]) continue;
        const SysState &st = ps[s];
        // a system still running after ITMAX + 2 bodies is reported incomplete, as
        // the one-shot solve reports it
        if (st.status != ST_RUNNING || snap_bodies_[b] - slot_join_body_[s] >= (long long)st.itmax + 2) {
            done.push_back(LiveDone{s, result_of(st, mixed)});
            slot_reported_[s] = 1;
        }
    }
    collected_upto_ = q;
    return 0;
}

}  // namespace mfixgpu

namespace mfixgpu {

// A one-shot batch of several systems run as a live batch: all join at once,
// each leaves when it finishes, so the kernels stop visiting finished systems.
int Engine::run_batch_live(const std::vector<SystemSpec> &specs, const SolveOptions &opt,
                           std::vector<SolveResult> &out)
{
    const int ns = (int)specs.size();
    out.assign(ns, SolveResult{});
    size_t bytes = 4096;
    for (const auto &s : specs) bytes += work_bytes(s.n, (int64_t)s.imax2 * s.kmax2, opt.precision) + 512;
    cudaError_t e = arena_.reserve(bytes);
    if (e != cudaSuccess) return fail(std::string("device memory for the batch: ") + cudaGetErrorString(e), -11);
    arena_.reset();
    int rc = live_open(ns, opt);
    if (rc) return rc;
    launches_ = 0;
    timing_ = SolveTiming{};
    x0_.assign(ns, nullptr);
    int max_itmax = 0;
    for (int q = 0; q < ns; ++q) {
        const SystemSpec &sp = specs[q];
        const int64_t lines = (int64_t)sp.imax2 * sp.kmax2;
        LiveSystem ls;
        ls.dev = sp;
        ls.work = (char *)arena_.take(work_bytes(sp.n, lines, opt.precision));
        ls.scaled = opt.skip_scale;
        if (opt.precision == PREC_MIXED) ls.x0_slot = ls.work + vec_region_bytes(sp.n, lines, PREC_MIXED);
        const int slot = live_add(ls);
        if (slot != q) return slot < 0 ? slot : fail("internal: live slot order", -13);
        x0_[q] = h_sys_[q].x64[1];
        max_itmax = std::max(max_itmax, sp.itmax);
    }
    CK(cudaEventRecord(ev_t0_, stream_));
    // the first commit runs the setup; new line lengths are tuned right after it
    live_tune_ = opt.autotune && opt.force_lanes <= 0 && opt.pc == PC_LINE;
    const int K = std::max(1, opt.check_every);
    int remaining = ns;
    std::vector<LiveDone> done;
    while (remaining > 0) {
        if ((rc = live_step(K))) {
            live_tune_ = false;
            return rc;
        }
        if ((rc = issue_writeback())) return rc;  // A/B are scaled: copy them back meanwhile
        done.clear();
        if ((rc = live_collect(done, false))) return rc;
        for (const LiveDone &d : done) {
            out[d.slot] = d.res;
            live_remove(d.slot);
            --remaining;
        }
        if (body_total_ > (long long)max_itmax + 2 + 4LL * K + 8) break;  // every system reports by itmax + 2
    }
    live_tune_ = false;
    CK(cudaEventRecord(ev_t1_, stream_));
    CK(cudaStreamSynchronize(stream_));
    cudaEventElapsedTime(&timing_.device_ms, ev_t0_, ev_t1_);
    timing_.kernel_launches = launches_;
    if (remaining > 0)
        for (int q = 0; q < ns; ++q)
            if (slot_used_[q] && !slot_reported_[q]) {
                out[q] = SolveResult{};
                out[q].ier = -15;
                out[q].exit_kind = EX_ERROR;
            }
    return 0;
}

}  // namespace mfixgpu
