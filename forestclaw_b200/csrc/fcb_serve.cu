// Ensemble serving loop (see fcb_serve.hpp).
#include "fcb_serve.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <tuple>

namespace fcb {

namespace {

// Options that must agree for two solves to share a step launch.
auto launch_key(const fcb_options_t& o) {
    return std::make_tuple(o.solver_kind, o.problem, o.mx, o.my, o.mbc, o.meqn, o.maux, o.mwaves, o.order[0],
                           o.order[1], std::vector<int>(o.mthlim, o.mthlim + 8), o.precision, o.claw_version,
                           o.grav, o.gamma, o.dry_tolerance, o.ax, o.bx, o.ay, o.by);
}

}  // namespace

Server::Server(size_t budget_bytes, cudaStream_t st) : budget_(budget_bytes), st_(st) {
    t0_ = std::chrono::steady_clock::now();
    try {
        check(cudaMalloc(&d_cfl_, kSlots * sizeof(unsigned long long)), "cfl slots");
        check(cudaHostAlloc(&h_cfl_, kSlots * sizeof(unsigned long long), cudaHostAllocDefault), "host cfl slots");
        for (int k = 0; k < kRing; ++k)
            check(cudaEventCreateWithFlags(&desc_ev_[k], cudaEventDisableTiming), "cudaEventCreate");
        check(cudaEventCreateWithFlags(&step_ev_, cudaEventDisableTiming), "cudaEventCreate");
    } catch (...) {
        cudaFree(d_cfl_);
        cudaFreeHost(h_cfl_);
        for (int k = 0; k < kRing; ++k)
            if (desc_ev_[k]) cudaEventDestroy(desc_ev_[k]);
        if (step_ev_) cudaEventDestroy(step_ev_);
        throw;
    }
    for (int k = kSlots - 1; k >= 0; --k) free_slots_.push_back(k);
}

Server::~Server() {
    cudaStreamSynchronize(st_);
    for (auto& kv : reqs_) {
        if (kv.second.st) cudaStreamSynchronize(kv.second.st);
        kv.second.ctx.reset();
        free_stream(kv.second);
    }
    reqs_.clear();
    cudaFree(d_cfl_);
    cudaFreeHost(h_cfl_);
    for (int k = 0; k < kRing; ++k) {
        cudaFreeHost(h_desc_pinned_[k]);
        cudaEventDestroy(desc_ev_[k]);
    }
    cudaEventDestroy(step_ev_);
}

void Server::check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Error(FCB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

void Server::free_stream(Request& r) noexcept {
    if (r.ev_ready) cudaEventDestroy(r.ev_ready);
    if (r.ev_done) cudaEventDestroy(r.ev_done);
    if (r.st) cudaStreamDestroy(r.st);
    r.ev_ready = r.ev_done = nullptr;
    r.st = nullptr;
}

double Server::now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
}

int Server::submit(const fcb_options_t& opt) {
    if (opt.step_variant == 2 || opt.step_variant >= 4)
        throw Error(FCB_ERR_INVALID, "served solves use the four-barrier or pipelined step form");
    if (opt.nout != 1) throw Error(FCB_ERR_INVALID, "served solves run to tfinal in one output interval (nout = 1)");
    if (opt.time_sync) throw Error(FCB_ERR_INVALID, "served solves do not run the time synchronisation");
    if (opt.src_term) throw Error(FCB_ERR_INVALID, "served solves have no source-term stage");
    Request r;
    r.id = next_id_++;
    r.opt = opt;
    r.t_submit = now();
    reqs_.emplace(r.id, std::move(r));
    queue_.push_back(r.id);
    return r.id;
}

const Request& Server::request(int id) const {
    auto it = reqs_.find(id);
    if (it == reqs_.end()) throw Error(FCB_ERR_INVALID, "unknown request");
    return it->second;
}

long long Server::active_cells() const {
    long long n = 0;
    for (int id : active_) {
        const Request& r = reqs_.at(id);
        n += (long long)r.ctx->num_patches() * r.opt.mx * r.opt.my;
    }
    return n;
}

// Admit queued requests in arrival order while their device memory fits the
// budget and their cells the work limit.  The head is initialised on first
// sight (its size is known only then); if it does not fit, it keeps its state
// and waits when only the work limit stops it, and is dropped and rebuilt
// later when its memory does not fit.
void Server::admit() {
    long long cells_now = max_cells_ > 0 ? active_cells() : 0;
    while (!queue_.empty()) {
        Request& r = reqs_.at(queue_.front());
        if (!active_.empty() && r.bytes > 0 && !r.ctx && used_ + r.bytes > budget_) return;  // known size, no room
        if (!active_.empty() && r.ctx && max_cells_ > 0 && cells_now + r.cells > max_cells_) return;
        if (free_slots_.empty()) return;  // kSlots requests admitted at once
        if (!r.ctx) {
            try {
                check(cudaStreamCreateWithFlags(&r.st, cudaStreamNonBlocking), "request stream");
                check(cudaEventCreateWithFlags(&r.ev_ready, cudaEventDisableTiming), "cudaEventCreate");
                check(cudaEventCreateWithFlags(&r.ev_done, cudaEventDisableTiming), "cudaEventCreate");
                r.ctx = std::make_unique<Context>(r.opt, r.st);
                r.ctx->initialize();
            } catch (const Error& e) {
                r.ctx.reset();
                free_stream(r);
                r.state = REQ_FAILED;
                r.error = e.what();
                r.t_finish = now();
                queue_.pop_front();
                continue;
            }
            r.bytes = r.ctx->device_bytes();
            r.cells = (long long)r.ctx->num_patches() * r.opt.mx * r.opt.my;
            if (!active_.empty() && used_ + r.bytes > budget_) {  // first sight of its size: wait for room
                r.ctx.reset();
                free_stream(r);
                return;
            }
            used_ += r.bytes;  // held from here on, also while it waits for the work limit
            if (!active_.empty() && max_cells_ > 0 && cells_now + r.cells > max_cells_) return;
        }
        r.cslot = free_slots_.back();
        free_slots_.pop_back();
        r.state = REQ_ACTIVE;
        r.ending = false;
        r.t_start = now();
        r.t = 0.0;
        r.dt_min = r.opt.initial_dt;
        r.n_inner = 0;
        begin_macro(r);
        active_.push_back(r.id);
        queue_.pop_front();
        cells_now += r.cells;
    }
}

// fclaw2d_run (src/fclaw2d_run.c, outstyle 1) up to the advance.
void Server::begin_macro(Request& r) {
    const fcb_options_t& o = r.opt;
    if (!o.use_fixed_dt) r.ctx->save_step();
    r.dt_step = r.dt_min;
    r.took_small = 0;
    if (!o.use_fixed_dt) {
        const double tol = 1e-2 * r.dt_step;
        const double small_step = o.tfinal - (r.t + r.dt_step);
        if (small_step < tol) {
            r.dt_step = o.tfinal - r.t;
            if (small_step < 0) r.took_small = 1;
        }
    }
    r.fine_total = r.fine_left = r.ctx->serve_begin(r.t, r.dt_step);
    r.macro_cfl = 0.0;
    // the macro step's CFL maximum accumulates in the request's slot
    check(cudaMemsetAsync(d_cfl_ + r.cslot, 0, sizeof(unsigned long long), r.st), "cfl slot");
}

// fclaw2d_run after the advance: CFL retry, dt update, regrid, end of run.  A
// NaN anywhere in the macro step wins the maximum (its bits are the largest).
void Server::end_macro(Request& r) {
    const fcb_options_t& o = r.opt;
    if (std::isnan(r.macro_cfl)) throw Error(FCB_ERR_NUMERIC, "NaN CFL");
    r.ctx->count_advance();
    if (r.macro_cfl > o.max_cfl && o.reduce_cfl && !o.use_fixed_dt) {
        r.ctx->restore_step();
        r.dt_min = r.dt_min * o.desired_cfl / r.macro_cfl;
        begin_macro(r);
        return;
    }
    ++r.n_inner;
    r.t += r.dt_step;
    if (!o.use_fixed_dt) {
        const double dt_new = r.dt_min * o.desired_cfl / r.macro_cfl;
        if (!r.took_small) r.dt_min = dt_new;
    }
    r.ctx->set_curr_time(r.t);
    if (o.regrid_interval > 0 && r.n_inner % o.regrid_interval == 0) r.ctx->regrid();
    if (r.t < o.tfinal) {
        begin_macro(r);
        return;
    }
    r.state = REQ_DONE;
}

void Server::retire(Request& r, bool slot_idle) {
    r.t_finish = now();
    used_ -= r.bytes;
    // a slot that a queued launch may still write is not handed out again
    if (r.cslot >= 0 && slot_idle) free_slots_.push_back(r.cslot);
    r.cslot = -1;
    r.ending = false;
    active_.erase(std::remove(active_.begin(), active_.end(), r.id), active_.end());
}

void Server::finish_macros(bool wait) {
    std::vector<int> ids;
    for (int id : active_)
        if (reqs_.at(id).ending) ids.push_back(id);
    // the requests whose stream has reached the end of their macro step
    std::vector<Request*> ready;
    bool first = true;
    for (int id : ids) {
        Request& r = reqs_.at(id);
        const cudaError_t q = (wait && first) ? cudaEventSynchronize(r.ev_done) : cudaEventQuery(r.ev_done);
        first = false;
        if (q == cudaErrorNotReady) continue;
        r.ending = false;
        if (q != cudaSuccess) {
            cudaGetLastError();
            r.state = REQ_FAILED;
            r.error = std::string("macro step: ") + cudaGetErrorString(q);
            continue;
        }
        std::memcpy(&r.macro_cfl, &h_cfl_[r.cslot], sizeof(double));
        ready.push_back(&r);
    }
    // fclaw2d_run's logic of each (CFL retry, dt, regrid) touches only that
    // request's context, stream and CFL slot, so the requests run it on
    // separate host threads (a regrid costs the host milliseconds)
    auto finish = [this](Request* r) {
        try {
            end_macro(*r);
        } catch (const Error& e) {
            r->state = REQ_FAILED;
            r->error = e.what();
        } catch (const std::exception& e) {
            r->state = REQ_FAILED;
            r->error = e.what();
        }
    };
    if (ready.size() == 1) {
        finish(ready[0]);
    } else if (ready.size() > 1) {
        std::vector<std::thread> th;
        th.reserve(ready.size() - 1);
        for (size_t k = 1; k < ready.size(); ++k) th.emplace_back(finish, ready[k]);
        finish(ready[0]);
        for (auto& t : th) t.join();
    }
    for (int id : ids) {
        Request& r = reqs_.at(id);
        if (!r.ending && r.state != REQ_ACTIVE) retire(r, true);
    }
}

int Server::round() {
    admit();
    std::vector<int> run;
    for (int id : active_)
        if (!reqs_.at(id).ending) run.push_back(id);
    if (run.empty()) {
        // nothing to launch: wait for the oldest macro step in flight
        if (!active_.empty()) finish_macros(true);
        return (int)active_.size();
    }
    // group the running requests by launch key, one launch per group
    std::vector<std::vector<int>> groups;
    {
        std::vector<decltype(launch_key(fcb_options_t{}))> keys;
        for (int id : run) {
            const auto k = launch_key(reqs_.at(id).opt);
            size_t g = 0;
            while (g < keys.size() && !(keys[g] == k)) ++g;
            if (g == keys.size()) {
                keys.push_back(k);
                groups.emplace_back();
            }
            groups[g].push_back(id);
        }
    }
    // descriptors of this fine step for every running request
    h_desc_.clear();
    std::vector<std::pair<size_t, size_t>> ranges;
    for (const auto& g : groups) {
        const size_t b = h_desc_.size();
        for (int id : g) {
            Request& r = reqs_.at(id);
            r.cell_updates += r.ctx->serve_step_descs(r.cslot, h_desc_);
        }
        ranges.emplace_back(b, h_desc_.size() - b);
    }
    // upload through the next pinned buffer of the ring, once the copy that
    // last read it has run
    const int k = ring_;
    ring_ = (ring_ + 1) % kRing;
    check(cudaEventSynchronize(desc_ev_[k]), "descriptor staging");
    if (h_desc_.size() > h_desc_cap_[k]) {
        cudaFreeHost(h_desc_pinned_[k]);
        h_desc_pinned_[k] = nullptr;
        h_desc_cap_[k] = std::max(h_desc_.size(), 2 * h_desc_cap_[k]);
        check(cudaHostAlloc(&h_desc_pinned_[k], h_desc_cap_[k] * sizeof(PatchDesc), cudaHostAllocDefault),
              "host desc");
    }
    std::memcpy(h_desc_pinned_[k], h_desc_.data(), h_desc_.size() * sizeof(PatchDesc));
    d_desc_.reserve(std::max<size_t>(1, h_desc_.size()));
    // the step reads what each request's stream has written so far
    for (int id : run) {
        Request& r = reqs_.at(id);
        check(cudaEventRecord(r.ev_ready, r.st), "cudaEventRecord");
        check(cudaStreamWaitEvent(st_, r.ev_ready, 0), "cudaStreamWaitEvent");
    }
    check(cudaMemcpyAsync(d_desc_.p, h_desc_pinned_[k], h_desc_.size() * sizeof(PatchDesc), cudaMemcpyHostToDevice,
                          st_),
          "descriptors");
    check(cudaEventRecord(desc_ev_[k], st_), "cudaEventRecord");
    for (size_t g = 0; g < groups.size(); ++g) {
        const Request& r0 = reqs_.at(groups[g][0]);
        check(launch_step_batch(r0.opt, r0.ctx->aux_kind(), d_desc_.p + ranges[g].first, (int)ranges[g].second,
                                d_cfl_, st_),
              "batched step");
        ++launches_;
    }
    check(cudaEventRecord(step_ev_, st_), "cudaEventRecord");
    // each request's time interpolations and ghost update after its fine step,
    // on its own stream; at the end of its macro step, its CFL comes back
    for (int id : run) {
        Request& r = reqs_.at(id);
        try {
            check(cudaStreamWaitEvent(r.st, step_ev_, 0), "cudaStreamWaitEvent");
            r.ctx->serve_after_step();
            if (--r.fine_left == 0) {
                check(cudaMemcpyAsync(&h_cfl_[r.cslot], d_cfl_ + r.cslot, sizeof(unsigned long long),
                                      cudaMemcpyDeviceToHost, r.st),
                      "cfl");
                check(cudaEventRecord(r.ev_done, r.st), "cudaEventRecord");
                r.ending = true;
            }
        } catch (const Error& e) {
            r.state = REQ_FAILED;
            r.error = e.what();
            retire(r, false);
        }
    }
    ++rounds_;
    // the macro-step ends (host logic, regrids) run while this round's work is
    // queued on the GPU
    finish_macros(false);
    return (int)active_.size();
}

void Server::get_q(int id, double* host, size_t n) {
    Request& r = reqs_.at(id);
    if (!r.ctx) throw Error(FCB_ERR_STATE, "request has no state (queued, failed or released)");
    r.ctx->get_q(host, n, false);
}

void Server::release(int id) {
    auto it = reqs_.find(id);
    if (it == reqs_.end()) return;
    Request& r = it->second;
    if (r.state == REQ_ACTIVE) throw Error(FCB_ERR_STATE, "request still running");
    if (r.state == REQ_QUEUED) {
        queue_.erase(std::remove(queue_.begin(), queue_.end(), id), queue_.end());
        if (r.ctx) used_ -= r.bytes;  // initialised while it waited for the work limit
    }
    if (r.st) cudaStreamSynchronize(r.st);
    r.ctx.reset();
    free_stream(r);
    reqs_.erase(it);
}

}  // namespace fcb
