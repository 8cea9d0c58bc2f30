// Ensemble serving: independent solves admitted as they arrive, resident on the
// device, advanced together with continuous batching.
//
// Each request is one solve (its own forest, arena and ghost plans, one
// fcb::Context on its own CUDA stream), subcycled or not as its options say.
// A round advances every running request by one fine step of its macro step
// (the level updates that fclaw2d_advance_all_levels makes between two ghost
// updates: with subcycling the finest level and the coarser levels whose step
// falls on it, each with its own dt): the patches of all requests that share a
// launch key (solver, patch shape, method, precision) go into ONE step launch
// on the server's stream, each patch carrying its own arrays, geometry, dt and
// CFL slot (PatchDesc); the launch waits for each request's stream, and each
// request's stream waits for the launch before its time interpolations and
// ghost update.  The CFL maximum of a macro step accumulates in the request's
// device slot and is read back, on the request's stream, only when the macro
// step ends; the round does not wait for the GPU.  A request whose macro step
// has ended sits out until its stream reaches that point, then the per-request
// macro-step logic of fclaw2d_run runs on the host (outstyle 1: small last
// step, CFL retry from the saved copy, dt = dt * desired_cfl / cfl, regrid
// every regrid_interval), synchronising only the request's own stream, while
// the rounds already queued keep the GPU busy.  Queued requests are admitted in
// arrival order while their device memory fits the budget (and their cells the
// work limit, if one is set).  Results are those of fcb_run on the same
// options, bit for bit: batching changes which launch a patch is in, never its
// arithmetic.
#pragma once
#include <cuda_runtime.h>

#include <chrono>
#include <deque>
#include <map>
#include <memory>
#include <vector>

#include "fcb_runtime.hpp"

namespace fcb {

enum RequestState : int { REQ_QUEUED = 0, REQ_ACTIVE = 1, REQ_DONE = 2, REQ_FAILED = 3 };

struct Request {
    int id = 0;
    fcb_options_t opt{};
    cudaStream_t st = nullptr;        // the request's own stream (non-blocking)
    cudaEvent_t ev_ready = nullptr;   // its stream's work before a step launch
    cudaEvent_t ev_done = nullptr;    // its stream's work up to the end of a macro step
    std::unique_ptr<Context> ctx;     // destroyed before st
    int state = REQ_QUEUED;
    bool ending = false;              // macro step enqueued to its end, CFL not yet read
    int cslot = -1;                   // its CFL slot on the device and in pinned memory
    // time stepping (fclaw2d_run, outstyle 1, nout = 1)
    double t = 0.0;           // start of the current macro step
    double dt_min = 0.0;      // dt of the minimum level (adapted)
    double dt_step = 0.0;     // dt of the current macro step
    int took_small = 0;
    int fine_left = 0;        // fine steps left in the current macro step
    int fine_total = 0;
    double macro_cfl = 0.0;
    int n_inner = 0;
    size_t bytes = 0;
    long long cells = 0;      // cells of its current mesh (patches x mx x my)
    double t_submit = 0.0, t_start = 0.0, t_finish = 0.0;  // seconds on the server clock
    long long cell_updates = 0;
    std::string error;
};

class Server {
  public:
    Server(size_t budget_bytes, cudaStream_t st);
    ~Server();
    int submit(const fcb_options_t& opt);
    // One round; returns the number of active requests after it.
    int round();
    const Request& request(int id) const;
    void get_q(int id, double* host, size_t n);
    void release(int id);
    // Cap on the cells of the admitted solves' meshes (0: none).  The queue head
    // waits, initialised, until the active solves' cells plus its own fit;
    // one solve is always admitted when none runs.
    void set_work_limit(long long max_cells) { max_cells_ = max_cells; }
    int queued() const { return (int)queue_.size(); }
    int active() const { return (int)active_.size(); }
    size_t used_bytes() const { return used_; }
    double now() const;
    long long rounds() const { return rounds_; }
    long long launches() const { return launches_; }

  private:
    void admit();
    void begin_macro(Request& r);
    void end_macro(Request& r);
    // ending requests whose stream has reached the end of their macro step:
    // read the CFL and run end_macro; with wait, block for the oldest one first
    void finish_macros(bool wait);
    // a finished or failed request leaves the active set; slot_idle: no launch
    // still in flight writes its CFL slot, which may then serve a new request
    void retire(Request& r, bool slot_idle);
    void free_stream(Request& r) noexcept;
    void check(cudaError_t e, const char* what);

    size_t budget_;
    size_t used_ = 0;
    long long max_cells_ = 0;
    long long active_cells() const;
    cudaStream_t st_;
    std::chrono::steady_clock::time_point t0_;
    int next_id_ = 0;
    std::map<int, Request> reqs_;
    std::deque<int> queue_;
    std::vector<int> active_;
    // round buffers: the descriptors of a round go through one of kRing pinned
    // buffers (reused once the copy that read it has run), so the host runs at
    // most kRing rounds ahead of the GPU
    static constexpr int kRing = 3;
    static constexpr int kSlots = 4096;  // CFL slots: requests admitted at once
    std::vector<PatchDesc> h_desc_;
    DevBuf<PatchDesc> d_desc_;
    unsigned long long* d_cfl_ = nullptr;  // kSlots, device
    unsigned long long* h_cfl_ = nullptr;  // kSlots, pinned
    std::vector<int> free_slots_;
    PatchDesc* h_desc_pinned_[kRing] = {};
    size_t h_desc_cap_[kRing] = {};
    cudaEvent_t desc_ev_[kRing] = {};
    int ring_ = 0;
    cudaEvent_t step_ev_ = nullptr;
    long long rounds_ = 0, launches_ = 0;
};

}  // namespace fcb
