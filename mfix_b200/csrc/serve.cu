// serve.cu -- the request server: continuous batching of LEQ_BICGS solves.
//
// One worker thread owns the device.  Requests wait in arrival order until
// their device block (A_M, B_M, VAR and work memory) fits the HBM budget and
// a slot of the live batch is free; their arrays are then copied in on a copy
// stream, and the system joins the live batch at the next iteration boundary.
// Finished systems leave at the next boundary, their VAR goes back on the copy
// stream, and their block returns to a stream-ordered memory pool once no
// kernel enqueued before their departure can still read the batch tables.
// In the mixed form a second, FP64 live batch takes the systems whose FP32
// iteration gave up: they re-solve from their initial guess in the same block.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/mfixgpu.h"
#include "leq_engine.h"

namespace mfixgpu {
void set_last_error(const std::string &msg);
}

using namespace mfixgpu;

namespace {

size_t al256(size_t v) { return (v + 255) / 256 * 256; }

enum Stage : int { S_QUEUED = 0, S_COPY_IN = 1, S_BATCH = 2, S_COPY_OUT = 3, S_DONE = 4 };

struct Req {
    long long id = 0;
    SystemSpec user;  // the caller's arrays
    int flags = 0;
    size_t bytes = 0;  // device block
    char *block = nullptr;
    SystemSpec dev;  // arrays the kernels use
    char *work = nullptr;
    cudaEvent_t ev = nullptr;
    int stage = S_QUEUED;
    Engine *eng = nullptr;
    int slot = -1;
    int fallback = 0, mixed_iterations = 0;
    long long handover_after = 0;  // the mixed batch's commit count after which it may join the FP64 batch
    SolveResult res;
    double t_submit = 0, t_admit = 0, t_start = 0, t_done = 0;
};

struct PendingFree {
    char *block;
    size_t bytes;
    Engine *eng;
    long long after;  // the engine's commit that removed the system
};

class Server {
public:
    ~Server() { shutdown(); }

    int start()
    {
        std::unique_lock<std::mutex> lk(mu_);
        thread_ = std::thread([this] { worker(); });
        cv_done_.wait(lk, [&] { return started_; });
        return setup_rc_;
    }

    long long submit(const mfixgpu_system &s, int flags)
    {
        if (s.imax2 < 1 || s.jmax2 < 1 || s.kmax2 < 1 || (int64_t)s.imax2 * s.jmax2 * s.kmax2 != s.dimension_3 ||
            (!s.do_k && s.kmax2 != 1) || s.dimension_3 > (int64_t)INT32_MAX - TILE_CELLS)
            return MFIXGPU_ERR_ARGS;
        if (!s.a_m || !s.b_m || !s.var || (flags & ~7)) return MFIXGPU_ERR_ARGS;
        if ((flags & MFIXGPU_REQ_ON_DEVICE) && (((uintptr_t)s.a_m | (uintptr_t)s.b_m | (uintptr_t)s.var) & 15))
            return MFIXGPU_ERR_ARGS;  // device arrays on 16-byte boundaries
        auto r = std::unique_ptr<Req>(new (std::nothrow) Req());
        if (!r) return MFIXGPU_ERR_NOMEM;
        r->user.imax2 = s.imax2;
        r->user.jmax2 = s.jmax2;
        r->user.kmax2 = s.kmax2;
        r->user.do_k = s.do_k ? 1 : 0;
        r->user.n = s.dimension_3;
        r->user.a = s.a_m;
        r->user.b = s.b_m;
        r->user.x = s.var;
        r->user.tol = s.tol;
        r->user.itmax = s.itmax;
        r->flags = flags;
        const size_t n = (size_t)s.dimension_3;
        r->bytes = live_work_bytes(s.dimension_3, (int64_t)s.imax2 * s.kmax2, cfg_.precision) + 256;
        if (!(flags & MFIXGPU_REQ_ON_DEVICE)) r->bytes += al256(7 * n * 8) + 2 * al256(n * 8);
        std::lock_guard<std::mutex> lk(mu_);
        if (fatal_) return fatal_;
        if (stop_) return MFIXGPU_ERR_ARGS;
        if ((double)r->bytes > budget_) return MFIXGPU_ERR_NOMEM;
        r->t_submit = now();
        r->id = next_id_++;
        const long long id = r->id;
        incoming_.push_back(r.get());
        all_[id] = std::move(r);
        ++submitted_;
        cv_work_.notify_one();
        return id;
    }

    int poll(long long t, mfixgpu_request *out)
    {
        std::lock_guard<std::mutex> lk(mu_);
        return take_locked(t, out);
    }

    int wait(long long t, double timeout, mfixgpu_request *out)
    {
        std::unique_lock<std::mutex> lk(mu_);
        auto ready = [&] {
            auto it = all_.find(t);
            return it == all_.end() || it->second->stage == S_DONE;
        };
        if (timeout < 0)
            cv_done_.wait(lk, ready);
        else
            cv_done_.wait_for(lk, std::chrono::duration<double>(timeout), ready);
        return take_locked(t, out);
    }

    int wait_any(double timeout, long long *t, mfixgpu_request *out)
    {
        std::unique_lock<std::mutex> lk(mu_);
        const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeout < 0 ? 1e9 : timeout);
        for (;;) {
            while (!finished_.empty()) {
                const long long id = finished_.front();
                finished_.pop_front();
                if (all_.count(id)) {
                    if (t) *t = id;
                    return take_locked(id, out);
                }
            }
            if (cv_done_.wait_until(lk, deadline) == std::cv_status::timeout && finished_.empty()) return 0;
        }
    }

    void counters(mfixgpu_server_counters *o)
    {
        std::lock_guard<std::mutex> lk(mu_);
        *o = mfixgpu_server_counters{};
        o->submitted = submitted_;
        o->completed = completed_;
        long long q = 0, c = 0, r = 0;
        for (auto &kv : all_) {
            const int st = kv.second->stage;
            if (st == S_QUEUED) ++q;
            if (st == S_COPY_IN) ++c;
            if (st == S_BATCH) ++r;
        }
        o->queued = q;
        o->copying = c;
        o->running = r;
        o->commits = commits_;
        o->iterations = bodies_;
        o->kernel_launches = launches_;
        o->fp64_fallbacks = fallbacks_;
        o->max_running = max_running_;
        o->reserved_bytes = (double)reserved_;
        o->peak_reserved_bytes = (double)peak_reserved_;
        o->budget_bytes = budget_;
        o->seconds = now();
        o->busy_ms[0] = busy_ms_[0];
        o->busy_ms[1] = busy_ms_[1];
    }

    void cancel_queued()
    {
        std::lock_guard<std::mutex> lk(mu_);
        cancel_ = true;
        cv_work_.notify_all();
    }

    void shutdown()
    {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
            cv_work_.notify_all();
        }
        if (thread_.joinable()) thread_.join();
    }

private:
    double now() const
    {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
    }

    int take_locked(long long t, mfixgpu_request *out)
    {
        auto it = all_.find(t);
        if (it == all_.end()) return MFIXGPU_ERR_ARGS;
        const Req &r = *it->second;
        if (out) {
            *out = mfixgpu_request{};
            out->status = r.stage;
            out->t_submit = r.t_submit;
            out->t_admit = r.t_admit;
            out->t_start = r.t_start;
            out->t_done = r.t_done;
            if (r.stage == S_DONE) {
                out->ier = r.res.ier;
                out->iterations = r.res.iterations;
                out->iter_tot_add = r.res.iter_tot_add;
                out->exit_kind = r.res.exit_kind;
                out->outer_steps = r.res.outer_steps;
                out->fp64_fallback = r.fallback;
                out->mixed_iterations = r.mixed_iterations;
                out->rnorm0 = r.res.rnorm0;
                out->rnorm = r.res.rnorm;
            }
        }
        if (r.stage != S_DONE) return 0;
        all_.erase(it);
        return 1;
    }

    void set_stage(Req *r, int stage, double *stamp)
    {
        std::lock_guard<std::mutex> lk(mu_);
        r->stage = stage;
        if (stamp) *stamp = now();
    }

    // ---- worker thread
    cudaEvent_t get_event()
    {
        if (!free_events_.empty()) {
            cudaEvent_t e = free_events_.back();
            free_events_.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return nullptr;
        return e;
    }

    void publish(Req *r, const SolveResult &res)
    {
        if (r->ev) free_events_.push_back(r->ev);
        r->ev = nullptr;
        std::lock_guard<std::mutex> lk(mu_);
        r->res = res;
        r->stage = S_DONE;
        r->t_done = now();
        ++completed_;
        finished_.push_back(r->id);
        cv_done_.notify_all();
    }

    void fail_request(Req *r, int code)
    {
        SolveResult res;
        res.ier = code;
        res.exit_kind = EX_ERROR;
        publish(r, res);
    }

    int setup()
    {
        if (cudaSetDevice(cfg_.device) != cudaSuccess) return fail_setup("cudaSetDevice failed");
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return fail_setup("cudaMemGetInfo failed");
        budget_ = cfg_.hbm_budget > 0 ? cfg_.hbm_budget : 0.85 * (double)free_b;
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = cfg_.device;
        if (cudaMemPoolCreate(&pool_, &props) != cudaSuccess) return fail_setup("cudaMemPoolCreate failed");
        uint64_t keep = UINT64_MAX;  // blocks stay with the pool between requests
        cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &keep);
        if (cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking) != cudaSuccess)
            return fail_setup("stream creation failed");
        SolveOptions o;
        o.pc = cfg_.pc_code;
        std::memcpy(o.sweep, cfg_.sweep, 4);
        o.inner_tol = cfg_.inner_tol > 0 ? cfg_.inner_tol : 1e-2;
        o.autotune = false;
        try {
            if (cfg_.precision == PREC_MIXED) {
                mix_.reset(new Engine());
                o.precision = PREC_MIXED;
                if (mix_->live_open(cfg_.max_systems, o)) return fail_setup(mix_->last_error());
            }
            f64_.reset(new Engine());
        } catch (...) {
            return fail_setup("engine construction failed");
        }
        o.precision = PREC_FP64;
        if (f64_->live_open(cfg_.max_systems, o)) return fail_setup(f64_->last_error());
        return 0;
    }

    int fail_setup(const std::string &msg)
    {
        set_last_error("server: " + msg);
        return MFIXGPU_ERR_CUDA;
    }

    void go_fatal(const std::string &msg)
    {
        set_last_error("server: " + msg);
        std::lock_guard<std::mutex> lk(mu_);
        fatal_ = MFIXGPU_ERR_CUDA;
    }

    Engine *first_engine() { return mix_ ? mix_.get() : f64_.get(); }

    void admit()
    {
        Engine *e = first_engine();
        while (!queue_.empty()) {
            Req *r = queue_.front();
            if (e->live_used() + (int)copying_.size() >= e->live_capacity()) break;
            if ((double)(reserved_.load() + r->bytes) > budget_) break;
            char *block = nullptr;
            cudaError_t ce = cudaMallocFromPoolAsync((void **)&block, r->bytes, pool_, copy_);
            if (ce != cudaSuccess) {
                cudaGetLastError();
                if (running_ == 0 && copying_.empty() && unloading_.empty() && frees_.empty()) {
                    queue_.pop_front();
                    fail_request(r, MFIXGPU_ERR_NOMEM);
                    continue;
                }
                break;  // retry once requests in flight give memory back
            }
            r->ev = get_event();
            if (!r->ev) {
                cudaFreeAsync(block, copy_);
                return go_fatal("event creation failed");
            }
            r->block = block;
            const size_t n = (size_t)r->user.n;
            r->dev = r->user;
            char *p = block;
            if (!(r->flags & MFIXGPU_REQ_ON_DEVICE)) {
                r->dev.a = (double *)p;
                p += al256(7 * n * 8);
                r->dev.b = (double *)p;
                p += al256(n * 8);
                r->dev.x = (double *)p;
                p += al256(n * 8);
                ce = cudaMemcpyAsync(r->dev.a, r->user.a, 7 * n * 8, cudaMemcpyHostToDevice, copy_);
                if (ce == cudaSuccess)
                    ce = cudaMemcpyAsync(r->dev.b, r->user.b, n * 8, cudaMemcpyHostToDevice, copy_);
                if (ce == cudaSuccess && !(r->flags & MFIXGPU_REQ_ZERO_GUESS))
                    ce = cudaMemcpyAsync(r->dev.x, r->user.x, n * 8, cudaMemcpyHostToDevice, copy_);
            }
            if (ce == cudaSuccess && (r->flags & MFIXGPU_REQ_ZERO_GUESS)) ce = cudaMemsetAsync(r->dev.x, 0, n * 8, copy_);
            r->work = p;
            if (ce == cudaSuccess) ce = cudaEventRecord(r->ev, copy_);
            if (ce != cudaSuccess) return go_fatal(std::string("copy in: ") + cudaGetErrorString(ce));
            reserved_ += r->bytes;
            peak_reserved_ = std::max(peak_reserved_.load(), reserved_.load());
            queue_.pop_front();
            copying_.push_back(r);
            set_stage(r, S_COPY_IN, &r->t_admit);
        }
    }

    void join()
    {
        Engine *e = first_engine();
        while (!copying_.empty()) {
            Req *r = copying_.front();
            const cudaError_t q = cudaEventQuery(r->ev);
            if (q == cudaErrorNotReady) break;  // copies complete in order on one stream
            if (q != cudaSuccess) return go_fatal(std::string("copy in: ") + cudaGetErrorString(q));
            LiveSystem ls;
            ls.dev = r->dev;
            ls.work = r->work;
            const int slot = e->live_add(ls);
            if (slot < 0) return go_fatal(e->last_error());
            r->eng = e;
            r->slot = slot;
            owner(e)[slot] = r;
            ++running_;
            copying_.pop_front();
            set_stage(r, S_BATCH, &r->t_start);
        }
        // mixed attempts that gave up: into the FP64 batch, after the mixed
        // batch's commit that removed them
        while (!handover_.empty() && f64_->live_used() < f64_->live_capacity()) {
            Req *r = handover_.front();
            if (mix_->live_commits() < r->handover_after) break;
            LiveSystem ls;
            ls.dev = r->dev;
            ls.work = r->work;
            ls.scaled = true;
            const int64_t lines = (int64_t)r->dev.imax2 * r->dev.kmax2;
            ls.x0 = (const double *)(r->work + std::max(vec_region_bytes(r->dev.n, lines, PREC_FP64),
                                                         vec_region_bytes(r->dev.n, lines, PREC_MIXED)));
            ls.after = mix_->live_fence();
            const int slot = f64_->live_add(ls);
            if (slot < 0) return go_fatal(f64_->last_error());
            r->eng = f64_.get();
            r->slot = slot;
            owner(f64_.get())[slot] = r;
            ++running_;
            handover_.pop_front();
        }
    }

    std::vector<Req *> &owner(Engine *e)
    {
        auto &v = (e == mix_.get()) ? own_mix_ : own_f64_;
        if ((int)v.size() < e->live_capacity()) v.resize(e->live_capacity(), nullptr);
        return v;
    }

    // Each live batch keeps up to two chunks of iterations queued and is stepped
    // on its own: a batch whose chunk finished never waits for the other's.
    bool step()
    {
        bool stepped = false;
        for (Engine *e : {mix_.get(), f64_.get()}) {
            if (!e || (e->live_used() == 0 && !e->live_dirty())) continue;
            if (e->live_inflight() >= 2) continue;
            const long long b0 = e->live_bodies(), l0 = e->launches(), c0 = e->live_commits();
            if (e->live_step(cfg_.check_every)) {
                go_fatal(e->last_error());
                return stepped;
            }
            stepped = true;
            std::lock_guard<std::mutex> lk(mu_);
            bodies_ += e->live_bodies() - b0;
            launches_ += e->launches() - l0;
            commits_ += e->live_commits() - c0;
            max_running_ = std::max(max_running_, (long long)running_);
        }
        return stepped;
    }

    bool collect()
    {
        bool any = false;
        for (Engine *e : {mix_.get(), f64_.get()}) {
            if (!e) continue;
            done_.clear();
            bool got = false;
            if (e->live_collect_ready(done_, &got)) {
                go_fatal(e->last_error());
                return any;
            }
            if (!got) continue;
            any = true;
            {
                std::lock_guard<std::mutex> lk(mu_);
                busy_ms_[(e == first_engine()) ? 0 : 1] = e->live_busy_ms();
            }
            for (const LiveDone &d : done_) {
                Req *r = owner(e)[d.slot];
                owner(e)[d.slot] = nullptr;
                e->live_remove(d.slot);
                --running_;
                if (!r) continue;
                if (e == mix_.get() && d.res.exit_kind == EX_FALLBACK) {
                    r->fallback = 1;
                    r->mixed_iterations = d.res.iterations;
                    {
                        std::lock_guard<std::mutex> lk(mu_);
                        ++fallbacks_;
                    }
                    r->handover_after = mix_->live_commits() + 1;  // the commit that removes it
                    handover_.push_back(r);
                    continue;
                }
                copy_out(r, e, d.res);
            }
        }
        return any;
    }

    void copy_out(Req *r, Engine *e, const SolveResult &res)
    {
        r->res = res;
        const size_t n = (size_t)r->user.n;
        cudaError_t ce = cudaSuccess;
        if (!(r->flags & MFIXGPU_REQ_ON_DEVICE)) {
            ce = cudaMemcpyAsync(r->user.x, r->dev.x, n * 8, cudaMemcpyDeviceToHost, copy_);
            if (ce == cudaSuccess && (r->flags & MFIXGPU_REQ_WRITE_AB)) {
                ce = cudaMemcpyAsync(r->user.a, r->dev.a, 7 * n * 8, cudaMemcpyDeviceToHost, copy_);
                if (ce == cudaSuccess) ce = cudaMemcpyAsync(r->user.b, r->dev.b, n * 8, cudaMemcpyDeviceToHost, copy_);
            }
        }
        if (ce == cudaSuccess) ce = cudaEventRecord(r->ev, copy_);
        if (ce != cudaSuccess) return go_fatal(std::string("copy out: ") + cudaGetErrorString(ce));
        frees_.push_back(PendingFree{r->block, r->bytes, e, e->live_commits() + 1});
        r->block = nullptr;
        unloading_.push_back(r);
        set_stage(r, S_COPY_OUT, nullptr);
    }

    void retire()
    {
        for (size_t q = 0; q < unloading_.size();) {
            Req *r = unloading_[q];
            const cudaError_t e = cudaEventQuery(r->ev);
            if (e == cudaErrorNotReady) {
                ++q;
                continue;
            }
            if (e != cudaSuccess) return go_fatal(std::string("copy out: ") + cudaGetErrorString(e));
            unloading_.erase(unloading_.begin() + q);
            const SolveResult res = r->res;
            publish(r, res);
        }
        for (size_t q = 0; q < frees_.size();) {
            const PendingFree &f = frees_[q];
            if (f.eng->live_commits() < f.after) {
                ++q;
                continue;
            }
            cudaStreamWaitEvent(copy_, f.eng->live_fence(), 0);
            cudaFreeAsync(f.block, copy_);
            reserved_ -= f.bytes;
            frees_.erase(frees_.begin() + q);
        }
    }

    // after a CUDA failure: every request not yet done ends with the error
    void drain_fatal()
    {
        std::vector<Req *> rs;
        for (Req *r : queue_) rs.push_back(r);
        for (Req *r : copying_) rs.push_back(r);
        for (Req *r : handover_) rs.push_back(r);
        for (Req *r : unloading_) rs.push_back(r);
        for (auto *v : {&own_mix_, &own_f64_})
            for (Req *&r : *v)
                if (r) {
                    rs.push_back(r);
                    r = nullptr;
                }
        queue_.clear();
        copying_.clear();
        handover_.clear();
        unloading_.clear();
        running_ = 0;
        for (Req *r : rs) fail_request(r, MFIXGPU_ERR_CUDA);
    }

    void worker()
    {
        const int rc = setup();
        {
            std::lock_guard<std::mutex> lk(mu_);
            setup_rc_ = rc;
            started_ = true;
            if (rc) fatal_ = rc;
            cv_done_.notify_all();
        }
        if (rc) {
            teardown();
            return;
        }
        for (;;) {
            bool fatal;
            {
                std::unique_lock<std::mutex> lk(mu_);
                while (!incoming_.empty()) {
                    queue_.push_back(incoming_.front());
                    incoming_.pop_front();
                }
                fatal = fatal_ != 0;
                if (cancel_) {
                    cancel_ = false;
                    lk.unlock();
                    for (Req *r : queue_) fail_request(r, MFIXGPU_ERR_CANCELLED);
                    queue_.clear();
                    lk.lock();
                }
                const bool busy = !queue_.empty() || !copying_.empty() || running_ > 0 || !handover_.empty() ||
                                  !unloading_.empty() || !frees_.empty() || (mix_ && mix_->live_dirty()) ||
                                  f64_->live_dirty();
                if (!busy || fatal) {
                    if (fatal) {
                        lk.unlock();
                        drain_fatal();
                        lk.lock();
                    }
                    if (stop_ && incoming_.empty()) break;
                    cv_work_.wait_for(lk, std::chrono::milliseconds(50),
                                      [&] { return !incoming_.empty() || stop_; });
                    continue;
                }
            }
            admit();
            join();
            const bool stepped = step();
            const bool collected = collect();
            retire();
            if (!stepped && !collected) {
                const bool chunks = (mix_ && mix_->live_inflight() > 0) || f64_->live_inflight() > 0;
                if (chunks)
                    std::this_thread::sleep_for(std::chrono::microseconds(50));  // chunks still running
                else if (!copying_.empty())
                    cudaEventSynchronize(copying_.front()->ev);  // nothing on the engines: wait for a copy
                else if (!unloading_.empty())
                    cudaEventSynchronize(unloading_.front()->ev);
            }
        }
        teardown();
    }

    void teardown()
    {
        if (copy_) cudaStreamSynchronize(copy_);
        for (const PendingFree &f : frees_) cudaFree(f.block);  // only after a failure
        frees_.clear();
        mix_.reset();
        f64_.reset();
        if (copy_) cudaStreamSynchronize(copy_);
        for (cudaEvent_t e : free_events_) cudaEventDestroy(e);
        free_events_.clear();
        if (pool_) cudaMemPoolDestroy(pool_);
        pool_ = nullptr;
        if (copy_) cudaStreamDestroy(copy_);
        copy_ = nullptr;
    }

public:
    struct Config {
        int precision = PREC_MIXED;
        int max_systems = 256;
        int check_every = 8;
        int device = 0;
        double hbm_budget = 0;
        double inner_tol = 1e-2;
        char sweep[4] = {'R', 'S', 'R', 'S'};
        int pc_code = PC_LINE;
    };

private:
    Config cfg_;
    std::chrono::steady_clock::time_point t0_;
    std::thread thread_;

    // shared with callers (mu_)
    std::mutex mu_;
    std::condition_variable cv_work_, cv_done_;
    bool started_ = false, stop_ = false, cancel_ = false;
    int setup_rc_ = 0, fatal_ = 0;
    double budget_ = 0;
    double busy_ms_[2] = {0.0, 0.0};
    long long next_id_ = 0, submitted_ = 0, completed_ = 0, commits_ = 0, bodies_ = 0, launches_ = 0,
              fallbacks_ = 0, max_running_ = 0;
    std::deque<Req *> incoming_;
    std::deque<long long> finished_;
    std::unordered_map<long long, std::unique_ptr<Req>> all_;

    // worker only
    std::unique_ptr<Engine> mix_, f64_;
    cudaStream_t copy_ = nullptr;
    cudaMemPool_t pool_ = nullptr;
    std::deque<Req *> queue_, copying_, handover_;
    std::vector<Req *> unloading_, own_mix_, own_f64_;
    std::vector<PendingFree> frees_;
    std::vector<LiveDone> done_;
    std::vector<cudaEvent_t> free_events_;
    int running_ = 0;
    std::atomic<size_t> reserved_{0}, peak_reserved_{0};  // read by counters()

public:
    Server(const Config &c) : cfg_(c), t0_(std::chrono::steady_clock::now()) {}
};

}  // namespace

extern "C" {

int mfixgpu_server_create(const mfixgpu_server_config *cfg, void **server)
{
    if (!server) return MFIXGPU_ERR_ARGS;
    *server = nullptr;
    Server::Config c;
    if (cfg) {
        if (cfg->precision != 0 && cfg->precision != 1) return MFIXGPU_ERR_ARGS;
        c.precision = cfg->precision == 1 ? PREC_MIXED : PREC_FP64;
        if (cfg->max_systems > 0) c.max_systems = cfg->max_systems;
        if (cfg->check_every > 0) c.check_every = cfg->check_every;
        c.device = cfg->device;
        c.hbm_budget = cfg->hbm_budget;
        if (cfg->inner_tol > 0) c.inner_tol = cfg->inner_tol;
        bool blank = true;
        for (int q = 0; q < 4; ++q) blank = blank && (cfg->sweep[q] == ' ' || cfg->sweep[q] == 0);
        if (!blank)
            for (int q = 0; q < 4; ++q) c.sweep[q] = cfg->sweep[q] ? cfg->sweep[q] : ' ';
        char p4[4];
        bool pblank = true;
        for (int q = 0; q < 4; ++q) {
            p4[q] = cfg->pc[q] ? cfg->pc[q] : ' ';
            pblank = pblank && p4[q] == ' ';
        }
        if (!pblank) {
            if (!std::memcmp(p4, "LINE", 4))
                c.pc_code = PC_LINE;
            else if (!std::memcmp(p4, "DIAG", 4))
                c.pc_code = PC_DIAG;
            else if (!std::memcmp(p4, "NONE", 4))
                c.pc_code = PC_NONE;
            else
                return MFIXGPU_ERR_UNSUPPORTED;
        }
    }
    if (c.max_systems > 65536) return MFIXGPU_ERR_ARGS;
    for (int q = 0; q < 4; ++q) {
        const char ch = c.sweep[q];
        if (ch == 'I' || ch == 'i' || ch == 'K' || ch == 'k' || ch == 'A' || ch == 'a') return MFIXGPU_ERR_UNSUPPORTED;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_last_error("no CUDA device visible");
        return MFIXGPU_ERR_CUDA;
    }
    if (c.device < 0 || c.device >= ndev) return MFIXGPU_ERR_ARGS;
    Server *s = new (std::nothrow) Server(c);
    if (!s) return MFIXGPU_ERR_NOMEM;
    const int rc = s->start();
    if (rc) {
        delete s;
        return rc;
    }
    *server = s;
    return 0;
}

long long mfixgpu_server_submit(void *server, const mfixgpu_system *sys, int flags)
{
    if (!server || !sys) return MFIXGPU_ERR_ARGS;
    return static_cast<Server *>(server)->submit(*sys, flags);
}

int mfixgpu_server_poll(void *server, long long ticket, mfixgpu_request *out)
{
    if (!server) return MFIXGPU_ERR_ARGS;
    return static_cast<Server *>(server)->poll(ticket, out);
}

int mfixgpu_server_wait(void *server, long long ticket, double timeout_s, mfixgpu_request *out)
{
    if (!server) return MFIXGPU_ERR_ARGS;
    return static_cast<Server *>(server)->wait(ticket, timeout_s, out);
}

int mfixgpu_server_wait_any(void *server, double timeout_s, long long *ticket, mfixgpu_request *out)
{
    if (!server) return MFIXGPU_ERR_ARGS;
    return static_cast<Server *>(server)->wait_any(timeout_s, ticket, out);
}

int mfixgpu_server_counters_get(void *server, mfixgpu_server_counters *out)
{
    if (!server || !out) return MFIXGPU_ERR_ARGS;
    static_cast<Server *>(server)->counters(out);
    return 0;
}

int mfixgpu_server_cancel_queued(void *server)
{
    if (!server) return MFIXGPU_ERR_ARGS;
    static_cast<Server *>(server)->cancel_queued();
    return 0;
}

int mfixgpu_server_destroy(void *server)
{
    if (!server) return MFIXGPU_ERR_ARGS;
    delete static_cast<Server *>(server);
    return 0;
}

}  // extern "C"
