// Ensemble serving: independent solves admitted as they arrive, resident on the
// device, advanced together with continuous batching.
//
// Each request is one solve (its own forest, arena and ghost plans, one
// fcb::Context), subcycled or not as its options say.  A round advances every
// active request by one fine step of its macro step (the level updates that
// fclaw2d_advance_all_levels makes between two ghost updates: with subcycling
// the finest level and the coarser levels whose step falls on it, each with
// its own dt): the patches of all requests that share a launch key (solver,
// patch shape, method, precision) go into ONE step launch, each patch carrying
// its own arrays, geometry and dt (PatchDesc); then each request's time
// interpolations and ghost update run and the per-request CFL numbers come
// back in one copy.  Between rounds the loop retires finished requests, admits
// queued ones in arrival order while their device memory fits the budget (and
// their cells the work limit, if one is set), and runs the per-request macro-
// step logic of fclaw2d_run (outstyle 1: small last step, CFL retry from the
// saved copy, dt = dt * desired_cfl / cfl, regrid every regrid_interval).
// Results are those of fcb_run on the same options, bit for bit: batching
// changes which launch a patch is in, never its arithmetic.
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
    std::unique_ptr<Context> ctx;
    int state = REQ_QUEUED;
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
    // round buffers
    std::vector<PatchDesc> h_desc_;
    DevBuf<PatchDesc> d_desc_;
    DevBuf<unsigned long long> d_cfl_;
    unsigned long long* h_cfl_ = nullptr;  // pinned
    size_t h_cfl_cap_ = 0;
    PatchDesc* h_desc_pinned_ = nullptr;
    size_t h_desc_cap_ = 0;
    long long rounds_ = 0, launches_ = 0;
};

}  // namespace fcb
