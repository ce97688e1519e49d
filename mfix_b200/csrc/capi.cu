// capi.cu -- the extern "C" boundary (include/mfixgpu.h).
//
// The Fortran SOLVE_LIN_EQ signature is kept: the drop-in receives the whole
// A_M / B_M arrays and the phase index M, decodes METHOD / PC / SWEEP the way
// model/solve_lin_eq.f:131-191 and model/leq_bicgs.f:74-87 do, and hands one
// system to the engine.  No C++ exception crosses the boundary; every failure
// is an IER code.
#include <chrono>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>

#include "../../include/mfixgpu.h"
#include "leq_engine.h"

using namespace mfixgpu;

namespace {

struct Geometry {
    bool set = false;
    int imax2 = 0, jmax2 = 0, kmax2 = 0, do_k = 1;
    int64_t n = 0;
    int dimension_m = 0;
    int cyc = 0;  // cyclic axes: 1 CYCLIC_X, 2 CYCLIC_Y, 4 CYCLIC_Z
};

struct Options {
    int precision = PREC_FP64;
    int write_back_ab = 1;
    uint64_t seed = 0x5EEDULL;
    double inner_tol = 1e-2;
    double mixed_growth = 10.0;
    int mixed_stalls = 6;
    double mixed_min_margin = 1e-4;
    int deflate = 1;
    int replace_every = 20;
    double restart_growth = 100.0;
    int minimize_dotproducts = 0;
    int icheck_bicgs = 1;
    int staged_matvec = 2;
    int do_transpose = 0;
    int check_every = 4;
    int use_graph = 1;
    int time_kernels = 0;
    int autotune = 1;
    int line_lanes = 0;
};

struct Global {
    std::mutex mu;
    std::unique_ptr<Engine> engine;
    Geometry geom;
    Options opt;
    int iter_tot[10] = {0};
    mfixgpu_stats last{};
    SolveTiming last_timing{};
    std::string err;
    // SOLVE_LIN_EQ calls queued by mfixgpu_solve_lin_eq_defer_ until the next flush;
    // each keeps the geometry registered when it was queued
    struct Deferred {
        int vno, m, itmax;
        double *var, *a_m, *b_m, tol;
        char sweep[4], pc[4];
        int *ier;
        Geometry geom;
    };
    std::vector<Deferred> deferred;
    DeviceArena pp;  // device copies of the pressure-correction fields and the assembled system
};

int flush_locked(Global &g);

// ---- the gas pressure-correction system on the device (pp_assembly.cu)
// The fields' device copies (or the caller's device pointers) and the system's
// device arrays, from the arena g.pp.  Returns 0 or an error code (g.err set).
struct PPDevice {
    PPFields f{};
    double *a = nullptr, *b = nullptr, *bmmax = nullptr, *x = nullptr, *part = nullptr;
    int grid = 0;
};

int pp_prepare(Global &g, Engine *e, const mfixgpu_pp_fields *hf, PPDevice &dv)
{
    if (!g.geom.set) {
        g.err = "mfixgpu_init_geometry has not been called";
        return MFIXGPU_ERR_NOGEOM;
    }
    if (!hf) {
        g.err = "null field record";
        return MFIXGPU_ERR_ARGS;
    }
    if (g.geom.cyc) {
        g.err = "the device assembly of the pressure correction serves non-cyclic boxes";
        return MFIXGPU_ERR_UNSUPPORTED;
    }
    if (!hf->ro_g0_defined) {
        g.err = "a compressible run (RO_G0 undefined, COMPRESSIBLE_PP_G) is not served by the device assembly";
        return MFIXGPU_ERR_UNSUPPORTED;
    }
    const int mmax = hf->mmax;
    if (mmax < 0 || mmax > g.geom.dimension_m || (mmax > 0 && !hf->close_packed)) {
        g.err = "MMAX outside 0:DIMENSION_M, or CLOSE_PACKED missing";
        return MFIXGPU_ERR_ARGS;
    }
    const bool do_k = g.geom.do_k != 0;
    bool solids = false;
    for (int m = 0; m < mmax; ++m) solids = solids || !hf->close_packed[m];
    const void *need[] = {hf->flag, hf->rop_ge, hf->rop_gn, hf->ayz, hf->axz, hf->u_g, hf->v_g, hf->rop_g,
                          hf->rop_go, hf->vol, hf->sum_r_g, hf->d_e, hf->d_n};
    for (const void *q : need)
        if (!q) {
            g.err = "null field array";
            return MFIXGPU_ERR_ARGS;
        }
    if (do_k && (!hf->rop_gt || !hf->axy || !hf->w_g || !hf->d_t)) {
        g.err = "null K-direction field array of a 3-D run";
        return MFIXGPU_ERR_ARGS;
    }
    if (solids && (!hf->rop_se || !hf->rop_sn || !hf->u_s || !hf->v_s || !hf->rop_s || !hf->rop_so ||
                   !hf->sum_r_s || (do_k && (!hf->rop_st || !hf->w_s)))) {
        g.err = "null solids field array";
        return MFIXGPU_ERR_ARGS;
    }
    const size_t n = (size_t)g.geom.n;
    const size_t cell = n * 8, dph = (size_t)(mmax + 1) * n * 8, sph = (size_t)mmax * n * 8;
    size_t bytes = 10 * cell + 3 * 256 + 4096 + 64 * 16;  // A (7n), B, B_MMAX, PP_G + partials
    if (!hf->on_device) bytes += n * 4 + 13 * cell + 3 * dph + 9 * sph + 64 * 256;
    bytes += (size_t)(mmax + 1) * 4 + 256;
    cudaError_t ce = g.pp.reserve(bytes);
    if (ce != cudaSuccess) {
        g.err = std::string("device memory for the pressure-correction system: ") + cudaGetErrorString(ce);
        return MFIXGPU_ERR_NOMEM;
    }
    g.pp.reset();
    cudaStream_t s = e->stream();
    auto put = [&](const void *src, size_t nbytes) -> const void * {
        if (!src) return nullptr;
        if (hf->on_device) return src;
        void *d = g.pp.take(nbytes);
        if (!d || cudaMemcpyAsync(d, src, nbytes, cudaMemcpyHostToDevice, s) != cudaSuccess) return nullptr;
        return d;
    };
    PPFields &f = dv.f;
    f.flag = (const int *)put(hf->flag, n * 4);
    f.rop_ge = (const double *)put(hf->rop_ge, cell);
    f.rop_gn = (const double *)put(hf->rop_gn, cell);
    f.rop_gt = (const double *)put(do_k ? hf->rop_gt : nullptr, cell);
    f.ayz = (const double *)put(hf->ayz, cell);
    f.axz = (const double *)put(hf->axz, cell);
    f.axy = (const double *)put(do_k ? hf->axy : nullptr, cell);
    f.u_g = (const double *)put(hf->u_g, cell);
    f.v_g = (const double *)put(hf->v_g, cell);
    f.w_g = (const double *)put(do_k ? hf->w_g : nullptr, cell);
    f.rop_g = (const double *)put(hf->rop_g, cell);
    f.rop_go = (const double *)put(hf->rop_go, cell);
    f.vol = (const double *)put(hf->vol, cell);
    f.sum_r_g = (const double *)put(hf->sum_r_g, cell);
    f.d_e = (const double *)put(hf->d_e, dph);
    f.d_n = (const double *)put(hf->d_n, dph);
    f.d_t = (const double *)put(do_k ? hf->d_t : nullptr, dph);
    f.mmax = mmax;
    if (solids) {
        f.rop_se = (const double *)put(hf->rop_se, sph);
        f.rop_sn = (const double *)put(hf->rop_sn, sph);
        f.rop_st = (const double *)put(do_k ? hf->rop_st : nullptr, sph);
        f.u_s = (const double *)put(hf->u_s, sph);
        f.v_s = (const double *)put(hf->v_s, sph);
        f.w_s = (const double *)put(do_k ? hf->w_s : nullptr, sph);
        f.rop_s = (const double *)put(hf->rop_s, sph);
        f.rop_so = (const double *)put(hf->rop_so, sph);
        f.sum_r_s = (const double *)put(hf->sum_r_s, sph);
    }
    // CLOSE_PACKED is host memory in every case; a close-packed phase is skipped
    std::vector<int> cp(mmax + 1, 1);
    for (int m = 0; m < mmax; ++m) cp[m] = hf->close_packed[m] ? 1 : 0;
    int *cpd = (int *)g.pp.take(cp.size() * 4);
    if (!cpd || cudaMemcpyAsync(cpd, cp.data(), cp.size() * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) {
        g.err = "copy of CLOSE_PACKED";
        return MFIXGPU_ERR_CUDA;
    }
    // pageable host sources: the copies must have read them before the call returns
    if (cudaStreamSynchronize(s) != cudaSuccess) {
        g.err = std::string("copy of the fields: ") + cudaGetErrorString(cudaGetLastError());
        return MFIXGPU_ERR_CUDA;
    }
    f.close_packed = cpd;
    f.odt = hf->odt;
    f.ijk_p_g = hf->ijk_p_g;
    if (!f.flag || !f.rop_ge || !f.rop_gn || !f.ayz || !f.axz || !f.u_g || !f.v_g || !f.rop_g || !f.rop_go ||
        !f.vol || !f.sum_r_g || !f.d_e || !f.d_n) {
        g.err = "copy of the fields to the device";
        return MFIXGPU_ERR_CUDA;
    }
    dv.a = (double *)g.pp.take(7 * cell);
    dv.b = (double *)g.pp.take(cell);
    dv.bmmax = (double *)g.pp.take(cell);
    dv.x = (double *)g.pp.take(cell);
    dv.grid = std::max(1, std::min((int)((n + 255) / 256), 64 * 16));
    dv.part = (double *)g.pp.take((size_t)dv.grid * 2 * 8);
    if (!dv.a || !dv.b || !dv.bmmax || !dv.x || !dv.part) {
        g.err = "internal: pressure-correction arena too small";
        return MFIXGPU_ERR_CUDA;
    }
    return 0;
}

int pp_assemble(Global &g, Engine *e, PPDevice &dv)
{
    PPGeom pg{g.geom.imax2, g.geom.jmax2, g.geom.kmax2, g.geom.do_k, g.geom.n};
    const int grid = std::max(1, std::min((int)((g.geom.n + 255) / 256), e->sm_count() * 8));
    cudaError_t ce = launch_conv_source_pp(dv.f, pg, dv.a, dv.b, dv.bmmax, grid, e->stream());
    if (ce != cudaSuccess) {
        g.err = std::string("pressure-correction assembly: ") + cudaGetErrorString(ce);
        return MFIXGPU_ERR_CUDA;
    }
    return 0;
}

Global &G()
{
    static Global g;
    return g;
}

Engine *engine_locked(Global &g)
{
    if (!g.engine) {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
            cudaGetLastError();
            g.err = "no CUDA device visible";
            return nullptr;
        }
        try {
            g.engine.reset(new Engine());
        } catch (...) {
            g.err = "engine construction failed";
            return nullptr;
        }
    }
    return g.engine.get();
}

// Fortran CHARACTER(LEN=4) value of a (pointer, length) pair: truncated or blank padded.
void fortran_char4(const char *s, size_t len, char out[4])
{
    for (int q = 0; q < 4; ++q) out[q] = (s && (size_t)q < len) ? s[q] : ' ';
}

// model/leq_bicgs.f:74-87 (exact, case-sensitive comparison as in Fortran)
int decode_pc(const char pc4[4])
{
    if (!std::memcmp(pc4, "LINE", 4)) return PC_LINE;
    if (!std::memcmp(pc4, "DIAG", 4)) return PC_DIAG;
    if (!std::memcmp(pc4, "NONE", 4)) return PC_NONE;
    return -1;
}

double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

SolveOptions make_opts(const Options &o, int pc, const char sweep4[4])
{
    SolveOptions so;
    so.pc = pc;
    std::memcpy(so.sweep, sweep4, 4);
    so.precision = o.precision;
    so.write_back_ab = o.write_back_ab != 0;
    so.seed = o.seed;
    so.inner_tol = o.inner_tol;
    so.mixed_growth = o.mixed_growth;
    so.mixed_stalls = o.mixed_stalls;
    so.mixed_min_margin = o.mixed_min_margin;
    so.deflate = o.deflate != 0;
    so.replace_every = o.replace_every;
    so.restart_growth = o.restart_growth;
    so.minimize_dotproducts = o.minimize_dotproducts;
    so.icheck_bicgs = o.icheck_bicgs;
    so.staged_matvec = o.staged_matvec;
    so.check_every = o.check_every;
    so.use_graph = o.use_graph != 0;
    so.time_kernels = o.time_kernels != 0;
    so.autotune = o.autotune != 0;
    so.force_lanes = o.line_lanes;
    return so;
}

void solve_impl(int vno, double *var, double *a_m, double *b_m, int m, int itmax, int method, const char sweep4[4],
                double tol, const char pc4[4], int *ier)
{
    Global &g = G();
    std::lock_guard<std::mutex> lk(g.mu);
    const double t0 = now_s();
    g.last = mfixgpu_stats{};
    auto finish = [&](int code) {
        if (ier) *ier = code;
        g.last.ier = code;
        g.last.seconds = now_s() - t0;
    };
    if (!ier) return;
    if (!g.geom.set) {
        g.err = "mfixgpu_init_geometry has not been called";
        return finish(MFIXGPU_ERR_NOGEOM);
    }
    if (!var || !a_m || !b_m) {
        g.err = "null array argument";
        return finish(MFIXGPU_ERR_ARGS);
    }
    if (m < 0 || m > g.geom.dimension_m) {
        g.err = "phase index M outside 0:DIMENSION_M";
        return finish(MFIXGPU_ERR_ARGS);
    }
    // model/solve_lin_eq.f:131-191: SOR (1), BiCGSTAB (2), GMRES (3), BiCGSTAB then GMRES (4), CG (5)
    if (method < 1 || method > 5) {
        g.err = "LEQ_METHOD " + std::to_string(method) + " is not served by the GPU path (1-5)";
        return finish(MFIXGPU_ERR_UNSUPPORTED);
    }
    // LEQ_GMRES and LEQ_SOR take no PC argument (:133-135, :156-158)
    const int pc = (method == 1 || method == 3) ? PC_LINE : decode_pc(pc4);
    if (pc < 0) {
        g.err = "preconditioner option not found";  // the reference's message, model/leq_bicgs.f:84-85
        return finish(MFIXGPU_ERR_UNSUPPORTED);
    }
    Engine *e = engine_locked(g);
    if (!e) return finish(MFIXGPU_ERR_CUDA);
    const int64_t n = g.geom.n;
    SystemSpec s;
    s.imax2 = g.geom.imax2;
    s.jmax2 = g.geom.jmax2;
    s.kmax2 = g.geom.kmax2;
    s.do_k = g.geom.do_k;
    s.cyc = g.geom.cyc;
    s.n = n;
    s.a = a_m + (size_t)m * 7 * (size_t)n;  // A_M(:,:,M)
    s.b = b_m + (size_t)m * (size_t)n;      // B_M(:,M)
    s.x = var;
    s.tol = tol;
    s.itmax = itmax;
    std::vector<SolveResult> out;
    SolveOptions so = make_opts(g.opt, pc, sweep4);
    so.method = method;
    so.transposed = g.opt.do_transpose && method == 2;  // DO_TRANSPOSE applies to CASE (2) only (:139-150)
    const int rc = e->solve({s}, so, out);
    if (rc) {
        g.err = e->last_error();
        return finish(rc);
    }
    const SolveResult &r = out[0];
    const int code = method == 1 ? *ier : r.ier;  // LEQ_SOR leaves IER alone
    if (vno >= 1 && vno <= 10) {
        if (method == 1)
            g.iter_tot[vno - 1] = r.iter_tot_add;  // ITER_TOT(VNO) = ITER (model/leq_sor.f:119)
        else
            g.iter_tot[vno - 1] += r.iter_tot_add;
    }
    g.last.iterations = r.iterations;
    g.last.iter_tot_add = r.iter_tot_add;
    g.last.exit_kind = r.exit_kind;
    g.last.line_skips = r.line_skips;
    g.last.line_fallbacks = r.line_fallbacks;
    g.last.outer_steps = r.outer_steps;
    g.last.rnorm0 = r.rnorm0;
    g.last.rnorm = r.rnorm;
    g.last.device_ms = e->timing().device_ms;
    g.last.jline_ms = e->timing().jline_ms;
    g.last.jline_launches = e->timing().jline_launches;
    g.last.kernel_launches = e->timing().kernel_launches;
    g.last.fp64_fallback = r.fp64_fallback;
    g.last.mixed_iterations = r.mixed_iterations;
    g.last.deflated = r.deflated;
    g.last_timing = e->timing();
    finish(code);
}

// A SOLVE_LIN_EQ call queued for the next flush when it can join a batch
// (METHOD 2 with red/black sweeps); any other call is solved at once.  The
// checks are solve_impl's, so a call that would fail fails here, at once.
void defer_impl(int vno, double *var, double *a_m, double *b_m, int m, int itmax, int method, const char sweep4[4],
                double tol, const char pc4[4], int *ier)
{
    if (!ier) return;
    bool batchable = method == 2;
    for (int q = 0; q < 4; ++q) {
        const char ch = sweep4[q];
        if (ch == 'I' || ch == 'i' || ch == 'K' || ch == 'k' || ch == 'A' || ch == 'a') batchable = false;
    }
    {
        Global &g = G();
        std::lock_guard<std::mutex> lk(g.mu);
        int code = 0;
        if (!g.geom.set) {
            g.err = "mfixgpu_init_geometry has not been called";
            code = MFIXGPU_ERR_NOGEOM;
        } else if (!var || !a_m || !b_m) {
            g.err = "null array argument";
            code = MFIXGPU_ERR_ARGS;
        } else if (m < 0 || m > g.geom.dimension_m) {
            g.err = "phase index M outside 0:DIMENSION_M";
            code = MFIXGPU_ERR_ARGS;
        } else if (batchable && decode_pc(pc4) < 0) {
            g.err = "preconditioner option not found";
            code = MFIXGPU_ERR_UNSUPPORTED;
        }
        if (code) {
            *ier = code;
            return;
        }
        if (batchable) {
            // a call that reads or writes the arrays of a queued call (the same VAR,
            // or the same A_M(:,:,M) slice) would be solved beside it; the queue is
            // solved first, so that the calls see each other in call order
            const double *slice = a_m + (size_t)m * 7 * (size_t)g.geom.n;
            for (const auto &q : g.deferred)
                if (q.var == var || q.a_m + (size_t)q.m * 7 * (size_t)q.geom.n == slice) {
                    flush_locked(g);
                    break;
                }
            Global::Deferred d{vno, m, itmax, var, a_m, b_m, tol, {}, {}, ier, g.geom};
            std::memcpy(d.sweep, sweep4, 4);
            std::memcpy(d.pc, pc4, 4);
            g.deferred.push_back(d);
            *ier = MFIXGPU_ERR_INCOMPLETE;  // until the flush
            return;
        }
    }
    solve_impl(vno, var, a_m, b_m, m, itmax, method, sweep4, tol, pc4, ier);
}

// Solves the queue, one batch per (PC, SWEEP, geometry), and writes the IERs in
// the order the calls were queued (calls that share one IER variable see the
// verdict of the last call, as the reference's back-to-back calls leave it).
int flush_locked(Global &g)
{
    std::vector<Global::Deferred> all;
    all.swap(g.deferred);
    if (all.empty()) return 0;
    Engine *e = engine_locked(g);
    if (!e) {
        for (auto &d : all) *d.ier = MFIXGPU_ERR_CUDA;
        return MFIXGPU_ERR_CUDA;
    }
    const double t0 = now_s();
    int first_rc = 0;
    std::vector<bool> done(all.size(), false);
    std::vector<int> code(all.size(), MFIXGPU_ERR_INCOMPLETE);
    mfixgpu_stats agg{};
    auto same_geom = [](const Geometry &a, const Geometry &b) {
        return a.imax2 == b.imax2 && a.jmax2 == b.jmax2 && a.kmax2 == b.kmax2 && a.do_k == b.do_k && a.n == b.n &&
               a.cyc == b.cyc;
    };
    for (size_t q0 = 0; q0 < all.size(); ++q0) {
        if (done[q0]) continue;
        // one batch per (PC, SWEEP, geometry): every call of the group shares the solver options
        std::vector<size_t> grp;
        for (size_t q = q0; q < all.size(); ++q)
            if (!done[q] && !std::memcmp(all[q].pc, all[q0].pc, 4) && !std::memcmp(all[q].sweep, all[q0].sweep, 4) &&
                same_geom(all[q].geom, all[q0].geom)) {
                grp.push_back(q);
                done[q] = true;
            }
        std::vector<SystemSpec> specs(grp.size());
        for (size_t k = 0; k < grp.size(); ++k) {
            const Global::Deferred &d = all[grp[k]];
            const int64_t n = d.geom.n;
            SystemSpec &s = specs[k];
            s.imax2 = d.geom.imax2;
            s.jmax2 = d.geom.jmax2;
            s.kmax2 = d.geom.kmax2;
            s.do_k = d.geom.do_k;
            s.cyc = d.geom.cyc;
            s.n = n;
            s.a = d.a_m + (size_t)d.m * 7 * (size_t)n;  // A_M(:,:,M)
            s.b = d.b_m + (size_t)d.m * (size_t)n;      // B_M(:,M)
            s.x = d.var;
            s.tol = d.tol;
            s.itmax = d.itmax;
        }
        std::vector<SolveResult> out;
        SolveOptions so = make_opts(g.opt, decode_pc(all[q0].pc), all[q0].sweep);
        so.transposed = g.opt.do_transpose != 0;  // queued calls are METHOD 2
        const int rc = e->solve(specs, so, out);
        if (rc) {
            g.err = e->last_error();
            for (size_t q : grp) code[q] = rc;
            if (!first_rc) first_rc = rc;
            continue;
        }
        for (size_t k = 0; k < grp.size(); ++k) {
            const Global::Deferred &d = all[grp[k]];
            code[grp[k]] = out[k].ier;
            if (d.vno >= 1 && d.vno <= 10) g.iter_tot[d.vno - 1] += out[k].iter_tot_add;
            agg.iterations = std::max(agg.iterations, out[k].iterations);
            agg.iter_tot_add += out[k].iter_tot_add;
        }
        agg.device_ms += e->timing().device_ms;
        agg.kernel_launches += e->timing().kernel_launches;
        g.last_timing = e->timing();
    }
    for (size_t q = 0; q < all.size(); ++q) *all[q].ier = code[q];
    agg.seconds = now_s() - t0;
    agg.ier = first_rc;
    g.last = agg;
    return first_rc;
}

}  // namespace

namespace mfixgpu {
void set_last_error(const std::string &msg)
{
    Global &g = G();
    std::lock_guard<std::mutex> lk(g.mu);
    g.err = msg;
}
}  // namespace mfixgpu

extern "C" {

int mfixgpu_init_geometry(const int *imax2, const int *jmax2, const int *kmax2, const int *do_k,
                          const int64_t *dimension_3, const int *dimension_m)
{
    Global &g = G();
    std::lock_guard<std::mutex> lk(g.mu);
    if (!imax2 || !jmax2 || !kmax2 || !do_k || !dimension_3 || !dimension_m) return MFIXGPU_ERR_ARGS;
    if (*imax2 < 1 || *jmax2 < 1 || *kmax2 < 1 || *dimension_m < 0) return MFIXGPU_ERR_ARGS;
    if (!*do_k && *kmax2 != 1) return MFIXGPU_ERR_ARGS;
    if ((int64_t)*imax2 * *jmax2 * *kmax2 != *dimension_3) return MFIXGPU_ERR_ARGS;
    g.geom.set = true;
    g.geom.imax2 = *imax2;
    g.geom.jmax2 = *jmax2;
    g.geom.kmax2 = *kmax2;
    g.geom.do_k = *do_k ? 1 : 0;
    g.geom.cyc = 0;  // set by mfixgpu_init_cyclic
    g.geom.n = *dimension_3;
    g.geom.dimension_m = *dimension_m;
    return 0;
}

int mfixgpu_init_cyclic(const int *cyclic_x, const int *cyclic_y, const int *cyclic_z)
{
    Global &g = G();
    std::lock_guard<std::mutex> lk(g.mu);
    if (!cyclic_x || !cyclic_y || !cyclic_z) return MFIXGPU_ERR_ARGS;
    if (!g.geom.set) return MFIXGPU_ERR_NOGEOM;
    int c = (*cyclic_x ? 1 : 0) | (*cyclic_y ? 2 : 0) | (*cyclic_z ? 4 : 0);
    if (!g.geom.do_k) c &= 3;  // no K direction in 2-D
    g.geom.cyc = c;
    return 0;
}

void mfixgpu_solve_lin_eq_(const char *vname, const int *vno, double *var, double *a_m, double *b_m, const int *m,
                           const int *itmax, const int *method, const char *sweep, const double *tol1,
                           const char *pc, int *ier, size_t vname_len, size_t sweep_len, size_t pc_len)
{
    (void)vname;
    (void)vname_len;
    if (!vno || !m || !itmax || !method || !tol1) {
        if (ier) *ier = MFIXGPU_ERR_ARGS;
        return;
    }
    char s4[4], p4[4];
    fortran_char4(sweep, sweep_len, s4);
    fortran_char4(pc, pc_len, p4);
    solve_impl(*vno, var, a_m, b_m, *m, *itmax, *method, s4, *tol1, p4, ier);
}

void mfixgpu_solve_lin_eq(const char *vname, int vname_len, int vno, double *var, double *a_m, double *b_m, int m,
                          int itmax, int method, const char *sweep, int sweep_len, double tol1, const char *pc,
                          int pc_len, int *ier)
{
    (void)vname;
    (void)vname_len;
    char s4[4], p4[4];
    fortran_char4(sweep, sweep_len < 0 ? 0 : (size_t)sweep_len, s4);
    fortran_char4(pc, pc_len < 0 ? 0 : (size_t)pc_len, p4);
    solve_impl(vno, var, a_m, b_m, m, itmax, method, s4, tol1, p4, ier);
}

void mfixgpu_solve_lin_eq_defer_(const char *vname, const int *vno, double *var, double *a_m, double *b_m,
                                 const int *m, const int *itmax, const int *method, const char *sweep,
                                 const double *tol1, const char *pc, int *ier, size_t vname_len, size_t sweep_len,
                                 size_t pc_len)
{
    (void)vname;
    (void)vname_len;
    if (!vno || !m || !itmax || !method || !tol1) {
        if (ier) *ier = MFIXGPU_ERR_ARGS;
        return;
    }
    char s4[4], p4[4];
    fortran_char4(sweep, sweep_len, s4);
    fortran_char4(pc, pc_len, p4);
    defer_impl(*vno, var, a_m, b_m, *m, *itmax, *method, s4, *tol1, p4, ier);
}

int mfixgpu_solve_lin_eq_pending(void)
{
    Global &g = G();
    std::lock_guard<std::mutex> lk(g.mu);
    return (int)g.deferred.size();
}

int mfixgpu_solve_lin_eq_flush(void)
{
    Global &g = G();
    std::lock_guard<std::mutex> lk(g.mu);
    return flush_locked(g);
}

int mfixgpu_iter_tot(int vno)
{
    Global &g = G();
    std::lock_guard<std::mutex> lk(g.mu);
    return (vno >= 1 && vno <= 10) ? g.iter_tot[vno - 1] : 0;
}

void mfixgpu_reset_iter_tot(void)
{
    Global &g = G();
    std::lock_guard<std::mutex> lk(g.mu);
    for (int &v : g.iter_tot) v = 0;
}

int mfixgpu_last_stats(mfixgpu_stats *out)
{
    if (!out) return MFIXGPU_ERR_ARGS;
    Global &g = G();
    std::lock_guard<std::mutex> lk(g.mu);
    *out = g.last;
    return 0;
}

const char *mfixgpu_last_error(void)
{
    Global &g = G();
    return g.err.c_str();
}

int mfixgpu_last_kernel_times(double *ms, long long *launches, int max_classes)
{
    Global &g = G();
    std::lock_guard<std::mutex> lk(g.mu);
    for (int k = 0; k < KC_COUNT && k < max_classes; ++k) {
        if (ms) ms[k] = g.last_timing.class_ms[k];
        if (launches) launches[k] = g.last_timing.class_launches[k];
    }
    return KC_COUNT;
}

int mfixgpu_set_option(const char *name, double value)
{
    if (!name) return MFIXGPU_ERR_ARGS;
    Global &g = G();
    std::lock_guard<std::mutex> lk(g.mu);
    const std::string k(name);
    if (k == "precision") {
        if (value != 0 && value != 1) return MFIXGPU_ERR_ARGS;
        g.opt.precision = (int)value;
    } else if (k == "write_back_ab") {
        g.opt.write_back_ab = value != 0;
    } else if (k == "rtilde_seed") {
        g.opt.seed = (uint64_t)value;
    } else if (k == "inner_tol") {
        if (!(value > 0 && value < 1)) return MFIXGPU_ERR_ARGS;
        g.opt.inner_tol = value;
    } else if (k == "mixed_growth") {
        if (!(value > 1)) return MFIXGPU_ERR_ARGS;
        g.opt.mixed_growth = value;
    } else if (k == "deflate") {
        g.opt.deflate = value != 0;
    } else if (k == "do_transpose") {
        g.opt.do_transpose = value != 0;
    } else if (k == "replace_every") {
        if (value < 0) return MFIXGPU_ERR_ARGS;
        g.opt.replace_every = (int)value;
    } else if (k == "minimize_dotproducts") {
        g.opt.minimize_dotproducts = value != 0;
    } else if (k == "icheck_bicgs") {
        if (value < 1) return MFIXGPU_ERR_ARGS;
        g.opt.icheck_bicgs = (int)value;
    } else if (k == "restart_growth") {
        if (!(value == 0 || value > 1)) return MFIXGPU_ERR_ARGS;
        g.opt.restart_growth = value;
    } else if (k == "staged_matvec") {
        if (!(value >= 0 && value <= MV_SHAPES)) return MFIXGPU_ERR_ARGS;
        g.opt.staged_matvec = (int)value;
    } else if (k == "mixed_min_margin") {
        if (!(value >= 0)) return MFIXGPU_ERR_ARGS;
        g.opt.mixed_min_margin = value;
    } else if (k == "mixed_stalls") {
        if (value < 1) return MFIXGPU_ERR_ARGS;
        g.opt.mixed_stalls = (int)value;
    } else if (k == "check_every") {
        if (value < 1) return MFIXGPU_ERR_ARGS;
        g.opt.check_every = (int)value;
    } else if (k == "use_graph") {
        g.opt.use_graph = value != 0;
    } else if (k == "time_kernels") {
        g.opt.time_kernels = value != 0;
    } else if (k == "autotune") {
        g.opt.autotune = value != 0;
    } else if (k == "line_lanes") {
        if (value < 0 || value > 32) return MFIXGPU_ERR_ARGS;
        g.opt.line_lanes = (int)value;
    } else {
        return MFIXGPU_ERR_ARGS;
    }
    return 0;
}

double mfixgpu_get_option(const char *name)
{
    if (!name) return 0.0;
    Global &g = G();
    std::lock_guard<std::mutex> lk(g.mu);
    const std::string k(name);
    if (k == "precision") return g.opt.precision;
    if (k == "write_back_ab") return g.opt.write_back_ab;
    if (k == "rtilde_seed") return (double)g.opt.seed;
    if (k == "inner_tol") return g.opt.inner_tol;
    if (k == "mixed_growth") return g.opt.mixed_growth;
    if (k == "mixed_stalls") return g.opt.mixed_stalls;
    if (k == "mixed_min_margin") return g.opt.mixed_min_margin;
    if (k == "deflate") return g.opt.deflate;
    if (k == "replace_every") return g.opt.replace_every;
    if (k == "staged_matvec") return g.opt.staged_matvec;
    if (k == "restart_growth") return g.opt.restart_growth;
    if (k == "minimize_dotproducts") return g.opt.minimize_dotproducts;
    if (k == "icheck_bicgs") return g.opt.icheck_bicgs;
    if (k == "do_transpose") return g.opt.do_transpose;
    if (k == "check_every") return g.opt.check_every;
    if (k == "use_graph") return g.opt.use_graph;
    if (k == "time_kernels") return g.opt.time_kernels;
    if (k == "autotune") return g.opt.autotune;
    if (k == "line_lanes") return g.opt.line_lanes;
    return 0.0;
}

int mfixgpu_autotune_cache(const char *path)
{
    Global &g = G();
    std::lock_guard<std::mutex> lk(g.mu);
    Engine *e = engine_locked(g);
    if (!e) return MFIXGPU_ERR_CUDA;
    e->load_tune_cache(path ? std::string(path) : std::string());
    return 0;
}

int mfixgpu_autotune_table(int *out, int max_entries)
{
    Global &g = G();
    std::lock_guard<std::mutex> lk(g.mu);
    if (!g.engine) return 0;
    return g.engine->tune_table(out, out ? max_entries : 0);
}

void mfixgpu_finalize(void)
{
    Global &g = G();
    std::lock_guard<std::mutex> lk(g.mu);
    // calls still queued are dropped unsolved: their IER keeps MFIXGPU_ERR_INCOMPLETE
    g.deferred.clear();
    g.pp.release();
    g.engine.reset();
}

int mfixgpu_conv_source_pp_g(const mfixgpu_pp_fields *f, double *a_m, double *b_m, double *b_mmax)
{
    Global &g = G();
    std::lock_guard<std::mutex> lk(g.mu);
    if (!f || !a_m || !b_m || !b_mmax) return MFIXGPU_ERR_ARGS;
    Engine *e = engine_locked(g);
    if (!e) return MFIXGPU_ERR_CUDA;
    PPDevice dv;
    int rc = pp_prepare(g, e, f, dv);
    if (rc) return rc;
    if (f->on_device) {  // assembled straight into the caller's device arrays
        dv.a = a_m;
        dv.b = b_m;
        dv.bmmax = b_mmax;
    }
    if ((rc = pp_assemble(g, e, dv))) return rc;
    const size_t cell = (size_t)g.geom.n * 8;
    cudaStream_t s = e->stream();
    cudaError_t ce = cudaSuccess;
    if (!f->on_device) {
        ce = cudaMemcpyAsync(a_m, dv.a, 7 * cell, cudaMemcpyDeviceToHost, s);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(b_m, dv.b, cell, cudaMemcpyDeviceToHost, s);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(b_mmax, dv.bmmax, cell, cudaMemcpyDeviceToHost, s);
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) {
        g.err = std::string("pressure-correction assembly: ") + cudaGetErrorString(ce);
        return MFIXGPU_ERR_CUDA;
    }
    return 0;
}

void mfixgpu_solve_pp_g_(const mfixgpu_pp_fields *f, const double *normg, double *pp_g, double *resg,
                         const int *itmax, const int *method, const char *sweep, const double *tol, const char *pc,
                         int *ier, size_t sweep_len, size_t pc_len)
{
    if (!ier) return;
    if (!normg || !pp_g || !resg || !itmax || !method || !tol || !f) {
        *ier = MFIXGPU_ERR_ARGS;
        return;
    }
    Global &g = G();
    std::unique_lock<std::mutex> lk(g.mu);
    const double t0 = now_s();
    g.last = mfixgpu_stats{};
    Engine *e = engine_locked(g);
    if (!e) {
        *ier = MFIXGPU_ERR_CUDA;
        return;
    }
    if (*method < 1 || *method > 5) {
        g.err = "LEQ_METHOD " + std::to_string(*method) + " is not served by the GPU path (1-5)";
        *ier = MFIXGPU_ERR_UNSUPPORTED;
        return;
    }
    char s4[4], p4[4];
    fortran_char4(sweep, sweep_len, s4);
    fortran_char4(pc, pc_len, p4);
    const int pcode = (*method == 1 || *method == 3) ? PC_LINE : decode_pc(p4);
    if (pcode < 0) {
        g.err = "preconditioner option not found";
        *ier = MFIXGPU_ERR_UNSUPPORTED;
        return;
    }
    PPDevice dv;
    int rc = pp_prepare(g, e, f, dv);
    if (!rc) rc = pp_assemble(g, e, dv);
    cudaStream_t s = e->stream();
    const int64_t n = g.geom.n;
    // PP_G(:) = ZERO (model/solve_pp_g.f:71)
    if (!rc && cudaMemsetAsync(dv.x, 0, (size_t)n * 8, s) != cudaSuccess) rc = MFIXGPU_ERR_CUDA;
    // NORMG = 0: normalization from the dominant terms (:94-101), then RESG (:102-104)
    double norm = *normg, r = 0.0;
    if (!rc && norm == 0.0) {
        if (resid_pp(dv.f.flag, dv.bmmax, n, 1.0, dv.part, dv.grid, s, &r) != cudaSuccess) rc = MFIXGPU_ERR_CUDA;
        norm = r / 10.0;  // DEN = 1.0D1
    }
    if (!rc && resid_pp(dv.f.flag, dv.b, n, norm, dv.part, dv.grid, s, resg) != cudaSuccess) rc = MFIXGPU_ERR_CUDA;
    if (rc) {
        if (rc == MFIXGPU_ERR_CUDA && g.err.empty()) g.err = "pressure-correction residual";
        *ier = rc;
        return;
    }
    // SOLVE_LIN_EQ('Pp_g', 1, PP_G, A_M, B_M, 0, LEQI, LEQM, ...) (:113-114) on the device arrays
    SystemSpec sp;
    sp.imax2 = g.geom.imax2;
    sp.jmax2 = g.geom.jmax2;
    sp.kmax2 = g.geom.kmax2;
    sp.do_k = g.geom.do_k;
    sp.n = n;
    sp.a = dv.a;
    sp.b = dv.b;
    sp.x = dv.x;
    sp.tol = *tol;
    sp.itmax = *itmax;
    SolveOptions so = make_opts(g.opt, pcode, s4);
    so.method = *method;
    so.on_device = true;
    so.transposed = g.opt.do_transpose && *method == 2;
    std::vector<SolveResult> out;
    rc = e->solve({sp}, so, out);
    if (rc) {
        g.err = e->last_error();
        *ier = rc;
        return;
    }
    if (cudaMemcpyAsync(pp_g, dv.x, (size_t)n * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        g.err = "copy of PP_G";
        *ier = MFIXGPU_ERR_CUDA;
        return;
    }
    const SolveResult &res = out[0];
    const int code = *method == 1 ? *ier : res.ier;
    if (*method == 1)
        g.iter_tot[0] = res.iter_tot_add;
    else
        g.iter_tot[0] += res.iter_tot_add;  // ITER_TOT(1), VNO = 1 for 'Pp_g'
    g.last.iterations = res.iterations;
    g.last.iter_tot_add = res.iter_tot_add;
    g.last.exit_kind = res.exit_kind;
    g.last.outer_steps = res.outer_steps;
    g.last.rnorm0 = res.rnorm0;
    g.last.rnorm = res.rnorm;
    g.last.fp64_fallback = res.fp64_fallback;
    g.last.mixed_iterations = res.mixed_iterations;
    g.last.deflated = res.deflated;
    g.last.device_ms = e->timing().device_ms;
    g.last.kernel_launches = e->timing().kernel_launches;
    g.last.ier = code;
    g.last.seconds = now_s() - t0;
    *ier = code;
}

int mfixgpu_leq_matvec(const mfixgpu_geom *gm, const double *a_dev, const double *var_dev, double *avar_dev)
{
    if (!gm || !a_dev || !var_dev || !avar_dev) return MFIXGPU_ERR_ARGS;
    if ((int64_t)gm->imax2 * gm->jmax2 * gm->kmax2 != gm->dimension_3 || gm->imax2 < 1 || gm->jmax2 < 1 ||
        gm->kmax2 < 1)
        return MFIXGPU_ERR_ARGS;
    Global &g = G();
    std::lock_guard<std::mutex> lk(g.mu);
    Engine *e = engine_locked(g);
    if (!e) return MFIXGPU_ERR_CUDA;
    SystemSpec s;
    s.imax2 = gm->imax2;
    s.jmax2 = gm->jmax2;
    s.kmax2 = gm->kmax2;
    s.do_k = gm->do_k ? 1 : 0;
    s.cyc = gm->cyclic & 7;
    s.n = gm->dimension_3;
    const int rc = e->matvec(s, a_dev, var_dev, avar_dev);
    if (rc) g.err = e->last_error();
    return rc;
}

int mfixgpu_leq_msolve(const mfixgpu_geom *gm, const double *b_dev, const double *a_dev, double *var_dev,
                       const char *sweep, const char *pc)
{
    if (!gm || !b_dev || !a_dev || !var_dev || !sweep || !pc) return MFIXGPU_ERR_ARGS;
    if ((int64_t)gm->imax2 * gm->jmax2 * gm->kmax2 != gm->dimension_3 || gm->imax2 < 1 || gm->jmax2 < 1 ||
        gm->kmax2 < 1 || (!gm->do_k && gm->kmax2 != 1))
        return MFIXGPU_ERR_ARGS;
    char s4[4], p4[4];
    fortran_char4(sweep, 4, s4);
    fortran_char4(pc, 4, p4);
    const int pcode = decode_pc(p4);
    if (pcode < 0) return MFIXGPU_ERR_UNSUPPORTED;
    Global &g = G();
    std::lock_guard<std::mutex> lk(g.mu);
    Engine *e = engine_locked(g);
    if (!e) return MFIXGPU_ERR_CUDA;
    SystemSpec s;
    s.imax2 = gm->imax2;
    s.jmax2 = gm->jmax2;
    s.kmax2 = gm->kmax2;
    s.do_k = gm->do_k ? 1 : 0;
    s.cyc = gm->cyclic & 7;
    s.n = gm->dimension_3;
    const int rc = e->msolve(s, a_dev, b_dev, var_dev, pcode, s4);
    if (rc) g.err = e->last_error();
    return rc;
}

int mfixgpu_dot_product_par(const double *r1_dev, const double *r2_dev, int64_t n, double *out)
{
    if (!r1_dev || !r2_dev || !out || n < 0) return MFIXGPU_ERR_ARGS;
    Global &g = G();
    std::lock_guard<std::mutex> lk(g.mu);
    Engine *e = engine_locked(g);
    if (!e) return MFIXGPU_ERR_CUDA;
    if (n == 0) {
        *out = 0.0;
        return 0;
    }
    const int rc = e->dot(r1_dev, r2_dev, n, out);
    if (rc) g.err = e->last_error();
    return rc;
}

int mfixgpu_batch_solve(mfixgpu_system *systems, int nsys, const char *sweep, const char *pc, int precision,
                        int on_device)
{
    if (!systems || nsys < 0 || !sweep || !pc) return MFIXGPU_ERR_ARGS;
    if (precision != 0 && precision != 1) return MFIXGPU_ERR_ARGS;
    char s4[4], p4[4];
    fortran_char4(sweep, 4, s4);
    fortran_char4(pc, 4, p4);
    const int pcode = decode_pc(p4);
    if (pcode < 0) return MFIXGPU_ERR_UNSUPPORTED;
    if (pcode == PC_LINE && nsys > 1)
        for (int q = 0; q < 4; ++q) {
            const char ch = s4[q];
            if (ch == 'I' || ch == 'i' || ch == 'K' || ch == 'k' || ch == 'A' || ch == 'a')
                return MFIXGPU_ERR_UNSUPPORTED;
        }
    Global &g = G();
    std::lock_guard<std::mutex> lk(g.mu);
    Engine *e = engine_locked(g);
    if (!e) return MFIXGPU_ERR_CUDA;
    std::vector<SystemSpec> specs(nsys);
    for (int q = 0; q < nsys; ++q) {
        const mfixgpu_system &m = systems[q];
        SystemSpec &s = specs[q];
        s.imax2 = m.imax2;
        s.jmax2 = m.jmax2;
        s.kmax2 = m.kmax2;
        s.do_k = m.do_k ? 1 : 0;
        s.n = m.dimension_3;
        s.a = m.a_m;
        s.b = m.b_m;
        s.x = m.var;
        s.tol = m.tol;
        s.itmax = m.itmax;
    }
    Options o = g.opt;
    o.precision = precision;
    SolveOptions so = make_opts(o, pcode, s4);
    so.on_device = on_device != 0;
    std::vector<SolveResult> out;
    const double t0 = now_s();
    const int rc = e->solve(specs, so, out);
    if (rc) {
        g.err = e->last_error();
        return rc;
    }
    g.last = mfixgpu_stats{};
    g.last.seconds = now_s() - t0;
    g.last.device_ms = e->timing().device_ms;
    g.last.jline_ms = e->timing().jline_ms;
    g.last.jline_launches = e->timing().jline_launches;
    g.last.kernel_launches = e->timing().kernel_launches;
    g.last_timing = e->timing();
    for (int q = 0; q < nsys; ++q) {
        systems[q].ier = out[q].ier;
        systems[q].iterations = out[q].iterations;
        systems[q].outer_steps = out[q].outer_steps;
        systems[q].exit_kind = out[q].exit_kind;
        systems[q].rnorm0 = out[q].rnorm0;
        systems[q].rnorm = out[q].rnorm;
        systems[q].fp64_fallback = out[q].fp64_fallback;
        g.last.deflated += out[q].deflated;
        g.last.fp64_fallback += out[q].fp64_fallback;
    }
    return 0;
}

}  // extern "C"
