// Host runtime of one solve: options, forest, device arena, ghost-operation
// lists and the level schedule.  All device work is enqueued on one stream.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>
#include <thread>
#include <exception>
#include <memory>

#include "../../include/fclaw_b200.h"
#include "fcb_comm.hpp"
#include "fcb_device.h"
#include "fcb_forest.hpp"

namespace fcb {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// One step launch over patches of several solves (identical options apart from
// the initial data, t_final and refinement depth): the pipelined form, FP64 or mixed.
cudaError_t launch_step_batch(const fcb_options_t& opt, int aux_kind, const PatchDesc* d_desc, int n,
                              unsigned long long* d_cfl, cudaStream_t st);

// Kernel launchers (fcb_step.cu, fcb_ghost.cu, fcb_amr.cu)
cudaError_t launch_step(int solver, int aux_kind, int mwaves, int mx, int my, int mbc, const StepArgs& a,
                        cudaStream_t st, int claw_version = 4);
cudaError_t launch_step_warp_swirl(int mx, int mbc, const StepArgs& a, cudaStream_t st);
cudaError_t launch_step_pipe(int solver, int aux_kind, int mwaves, int mx, int my, int mbc, int claw_version,
                             const StepArgs& a, cudaStream_t st);
cudaError_t launch_step_pipe_mixed(int solver, int aux_kind, int mwaves, int mx, int my, int mbc,
                                   int claw_version, const StepArgs& a, cudaStream_t st);
// the ghost-exchange-fused pipelined forms (a.fuse, a.qsrc set; a mesh of one level)
cudaError_t launch_step_pipe_fused(int solver, int aux_kind, int mwaves, int mx, int my, int mbc, int claw_version,
                                   const StepArgs& a, cudaStream_t st);
cudaError_t launch_step_pipe_fused_mixed(int solver, int aux_kind, int mwaves, int mx, int my, int mbc,
                                         int claw_version, const StepArgs& a, cudaStream_t st);
// src2 after the step (fcb_src.cu): kind 1 = the axisymmetric Euler source
cudaError_t launch_src2(int kind, const StepArgs& a, int mx, int my, int mbc, int meqn, cudaStream_t st);
struct GhostArgs;
// Lane add/multiply operations per second of this GPU in FP64 (fp64) or FP32
// (fcb_probe.cu).
cudaError_t measure_fp_rate(bool fp64, cudaStream_t st, double* ops_per_second);
// Time synchronisation (fcb_timesync.cu).
cudaError_t launch_ts_store_flux(const StepArgs& a, int mx, int my, int mbc, int meqn, cudaStream_t st);
cudaError_t launch_ts_apply(const TsArgs& a, cudaStream_t st);
cudaError_t launch_zero_registers(double* treg, int64_t stride, const int32_t* slots, int n, cudaStream_t st);
cudaError_t launch_ghost_wave(const GhostArgs& a, cudaStream_t st, int unroll);
cudaError_t launch_timeinterp(double* q, const double* qlast, double* qti, int64_t stride,
                              const int32_t* slots, int n, int mx, int my, int mbc, int meqn,
                              double alpha, cudaStream_t st);
struct QinitArgs;
cudaError_t launch_qinit(const QinitArgs& a, cudaStream_t st);
cudaError_t launch_setaux(int problem, int maux, const double* params, double* aux, int64_t stride,
                          const int32_t* slots, const PatchMeta* meta, int n, int mx, int my, int mbc, cudaStream_t st);
struct TagArgs;
cudaError_t launch_tag(const TagArgs& a, cudaStream_t st);
cudaError_t launch_regrid(double* q, int64_t stride, const int32_t* ops, const int32_t* fine, int nops,
                          int mx, int my, int mbc, int meqn, cudaStream_t st);
// scatter == false: dst[p] = src[slots[p]]; scatter == true: src[slots[p]] = dst[p];
// meqn5 > 0: dst holds the patches in the clawpack 5 order q(m,i,j)
cudaError_t launch_gather(const double* src, int64_t stride, const int32_t* slots, int n, int64_t psize,
                          double* dst, bool scatter, int meqn5, cudaStream_t st);
cudaError_t launch_mass(const double* q, int64_t stride, const int32_t* slots, const PatchMeta* meta, int n,
                        int mx, int my, int mbc, int meqn, double* out, cudaStream_t st);

// A device buffer that only grows.
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t cap = 0;
    void reserve(size_t n);
    void release();
    ~DevBuf() { release(); }
};

// One exchange of whole patch arrays between the ranks of a partitioned solve
// (the ghost-patch exchange of fclaw2d_exchange.c): items slot * 2 + array
// (0 q, 1 the time-interpolated q), grouped by peer rank in rank order, in
// increasing leaf order within a peer on both sides.
struct XList {
    std::vector<int32_t> send, recv;
    std::vector<int> send_n, recv_n;        // items per peer rank
    size_t send_first = 0, recv_first = 0;  // offsets in the context's device item buffer
    bool any = false;                       // some rank sends something (the same on every rank)
};

struct GhostPlan {
    std::vector<int> wave_begin;   // op offsets of each wave, size nwaves+1
    size_t first = 0;              // first op of the plan in the context's op buffer
    std::vector<int> group_begin;  // per wave: first group, size nwaves+1
    size_t first_group = 0;        // first group of the plan in the context's group buffer
    // partitioned solves: waves [0, nA) are the averages, copies and coarse
    // physical boundaries, which read only the interiors of their sources (x1
    // brings those of other ranks' patches first); x2 then brings the other
    // ranks' coarse patches, ghost cells included, that the interpolations read
    int nA = 0;
    XList x1, x2;
};

// Host-only planning query of a partitioned solve (fcb_partition_plan).
struct PartitionPlan {
    int first = 0, count = 0, ghosts = 0, records = 0;
    std::vector<int> x1_send, x1_recv, x2_send, x2_recv;  // patches per peer rank
};

class Context {
  public:
    // comm: null for a solve on one rank; otherwise this context is rank
    // comm->rank() of a partitioned solve (leaves in contiguous Morton ranges)
    Context(const fcb_options_t& o, cudaStream_t st, std::shared_ptr<Comm> comm = nullptr);
    ~Context();

    void initialize();
    void run();
    double advance_all_levels(double t, double dt);
    // the same macro step without waiting for its CFL number, which goes into a
    // running maximum on the device; read_max_cfl waits, returns and resets it
    void advance_all_levels_async(double t, double dt);
    double read_max_cfl();
    double update_single_step(int level, double t, double dt);
    void update_single_step_async(int level, double t, double dt);
    double single_step_update(int patchno, double t, double dt, int iter, int total);
    void ghost_update(int minlevel, int maxlevel, double sync_time, int time_interp);
    void timeinterp(int level, double alpha);
    bool regrid();
    void physical_set_bc(int level, int time_interp);

    int num_patches() const { return (int)forest_.leaves.size(); }
    const Leaf& leaf(int p) const { return forest_.leaves[p]; }
    const Neighbors& nbrs(int p) const { return nbrs_[p]; }
    size_t patch_size() const { return (size_t)opt_.meqn * nx_ * ny_; }
    void get_q(double* host, size_t n, bool qinterp);
    void set_q(const double* host, size_t n);
    void conservation(double* sums);
    void synchronize();
    fcb_counters_t counters() const { return cnt_; }
    double curr_time() const { return curr_time_; }
    const fcb_options_t& options() const { return opt_; }
    int aux_kind() const { return aux_kind_; }

    // --- one macro step of fclaw2d_advance_all_levels (subcycled or not), one
    // fine step at a time, for launches that batch several solves (serving) ---
    // serve_begin: start the macro step at t_curr with coarse step dt; returns
    // its number of fine steps.
    int serve_begin(double t_curr, double dt);
    // the level updates of the next fine step (as run_schedule orders them):
    // one descriptor per patch with its level's t and dt and CFL slot req;
    // returns the cells it updates
    long long serve_step_descs(int req, std::vector<PatchDesc>& out);
    // after the batched step launch: that fine step's time interpolations and
    // the ghost update that follows it (the final one after the last fine step)
    void serve_after_step();
    // the CFL-retry copy of q
    void save_step();
    void restore_step();
    void set_curr_time(double t) { curr_time_ = t; }
    void count_advance() { ++cnt_.count_amr_advance; }
    size_t device_bytes() const;
    // fclaw2d_clawpatch_output_ascii: frame iframe into dir/fort.tNNNN, fort.qNNNN
    void output_ascii(int iframe, const std::string& dir);
    // the step kernel an advance would launch on the current mesh, timed on
    // scratch arrays (fused: the ghost-exchange-fused step); ms per launch
    double step_kernel_time(double t, double dt, int launches, bool* fused);
    // autotuner: the step form (1 four-barrier CTA, 2 warp, 3 pipelined) and the
    // ghost-fill unroll used by the last launches
    int step_form_used() const { return step_form_used_; }
    int ghost_unroll_used() const { return ghost_unroll_; }
    int fused_used() const { return fused_used_; }
    int bands_used() const { return bands_used_; }
    // --- partitioned solves (fclaw2d_partition.c, fclaw2d_exchange.c) ---
    bool partitioned() const { return comm_ != nullptr; }
    int rank() const { return rank_; }
    int nranks() const { return nranks_; }
    int own_first() const { return own_first_; }
    int own_count() const { return own_count_; }
    // fclaw2d_domain_global_maximum (forestclaw2d.c:51)
    double global_maximum(double v);
    // marks the communicator failed, so that the other ranks stop at their next collective
    void abort_comm(const std::string& why) noexcept;
    // rank `rank` of `nranks` over the given leaves (Morton order): owned range,
    // ghost layer size and the exchange counts of one ghost update; no device call
    static PartitionPlan partition_plan(const fcb_options_t& o, const std::vector<Leaf>& leaves, int rank,
                                        int nranks, int minlevel, int maxlevel, int time_interp);

  private:
    // --- setup ---
    void check(cudaError_t e, const char* what);
    void ensure_scalars();
    void ensure_capacity(int nslots);
    int alloc_slot();
    void mesh_changed();  // rebuild neighbour tables, level lists, metadata; drop ghost plans
    void compute_neighbors();
    PatchMeta meta_of(const Leaf& l) const;
    // --- ghost plans ---
    const GhostPlan& plan(int minlevel, int maxlevel, int time_interp);
    // records in the reference's order with LEAF indices in dst / src; *phase_b:
    // index of the first interpolation record
    void build_ops(int minlevel, int maxlevel, int time_interp, std::vector<GhostOp>& ops, size_t* phase_b) const;
    // A ghost plan before it is appended to the context's op buffer: records in
    // wave order, wave offsets, and the group starts of each wave (relative).
    struct PlanBuild {
        std::vector<GhostOp> ops;
        std::vector<int> wave_begin, group_begin;
        std::vector<int32_t> groups;
        int nA = 0;
        XList x1, x2;
    };
    PlanBuild build_plan(int minlevel, int maxlevel, int time_interp) const;
    PlanBuild make_waves(const std::vector<GhostOp>& ops) const;
    const GhostPlan& commit_plan(const std::tuple<int, int, int>& key, PlanBuild&& b);
    // Missing plans of a macro step are built on host threads while its first
    // level updates run on the GPU; plan() waits for them.  Every build ends
    // (finish_plans) before advance_all_levels returns, so no build outlives a
    // call that may change the forest.
    void start_plans(const std::vector<std::tuple<int, int, int>>& keys);
    void finish_plans();
    void join_plans() noexcept;
    void discard_plans() noexcept;
    void prefetch_plans();
    void upload_ops();
    // patch arenas and scratch come from a per-device stream-ordered pool that
    // keeps freed memory (solves created and destroyed by a serving loop reuse
    // each other's memory; a free never synchronises the device)
    template <class T>
    void arena_alloc(T*& p, size_t bytes);
    void arena_free(void* p);
    std::vector<std::tuple<int, int, int>> dry_plan_keys_;  // plans the dry pass met
    // time synchronisation: registers, and per minlevel the launches of one
    // fclaw2d_time_sync call (records grouped per patch, groups per launch)
    struct TsPlan {
        std::vector<size_t> first_group;  // per launch: first group in the group buffer
        std::vector<int> ngroups;         // per launch
    };
    void time_sync(int minlevel);
    const TsPlan& ts_plan(int minlevel);
    bool time_sync_ = false;
    double* d_treg_ = nullptr;
    int64_t treg_stride_ = 0;
    std::map<int, TsPlan> ts_plans_;
    std::vector<TsOp> h_ts_ops_;
    std::vector<int32_t> h_ts_groups_;
    DevBuf<TsOp> d_ts_ops_;
    DevBuf<int32_t> d_ts_groups_;
    TsOp* h_ts_ops_pinned_ = nullptr;
    size_t h_ts_ops_pinned_cap_ = 0;
    int32_t* h_ts_groups_pinned_ = nullptr;
    size_t h_ts_groups_pinned_cap_ = 0;
    std::vector<std::tuple<int, int, int>> plan_todo_;
    std::vector<PlanBuild> plan_built_;
    std::vector<std::exception_ptr> plan_err_;
    std::vector<std::thread> plan_threads_;
    // pinned staging of the op and group buffers, and the event of its last upload
    GhostOp* h_ops_pinned_ = nullptr;
    size_t h_ops_pinned_cap_ = 0;
    int32_t* h_groups_pinned_ = nullptr;
    size_t h_groups_pinned_cap_ = 0;
    cudaEvent_t upload_ev_ = nullptr;
    void run_plan(const GhostPlan& g);
    // --- regrid helpers ---
    void tag(bool domain_init, std::vector<int>& target);
    bool adapt(const std::vector<int>& target, std::vector<Leaf>& out);
    void repopulate(const std::vector<Leaf>& old_leaves, const std::vector<int>& old_slots,
                    bool domain_init);
    void qinit_slots(const std::vector<int32_t>& slots);
    // --- partitioned solves ---
    void partition_leaves();             // cut_, owner_, own range for forest_ (weighted Morton ranges)
    std::vector<char> local_set() const;  // per leaf: owned, or a face/corner neighbour of an owned leaf
    void exchange(const XList& x, const int32_t* d_items = nullptr);  // items: the plan item buffer
    // every rank receives the owned ranges of all ranks: d_own holds this rank's
    // own_count_ * per_leaf doubles, d_all receives num_patches() * per_leaf
    void allgather_owned(const double* d_own, int per_leaf, double* d_all);
    void repopulate_partitioned(const std::vector<Leaf>& old_leaves, const std::vector<int>& old_slots,
                                const std::vector<int>& old_owner, bool domain_init);
    bool owned(int p) const { return owner_.empty() || owner_[p] == rank_; }
    std::shared_ptr<Comm> comm_;
    int rank_ = 0, nranks_ = 1;
    std::vector<int> owner_;  // per leaf (partitioned solves)
    std::vector<int> cut_;    // rank r owns leaves [cut_[r], cut_[r+1])
    int own_first_ = 0, own_count_ = 0;
    std::vector<int32_t> h_xitems_;
    DevBuf<int32_t> d_xitems_;
    DevBuf<double> d_xsend_, d_xrecv_;
    double launch_level_step(int level, double t, double dt, unsigned long long* cfl_slot);
    // --- ghost-exchange fusion on a mesh of one level ---
    // The fused step reads arena d_q_ (ghost cells through the neighbour table
    // d_fuse_) and writes the interiors into d_qalt_; the two are then swapped.
    // The ghost update that would follow is recorded (ghosts_stale_) and run by
    // ensure_ghosts() before anything reads ghost cells.
    bool fusion_possible() const;             // mesh, options and step form allow it
    bool use_fusion(double t, double dt);     // possible and chosen (tuner or forced)
    void advance_fused(double t, double dt);
    void advance_enqueue(double t, double dt);  // a macro step, its CFL left in d_cfl_[0]
    void launch_fused_step(double t, double dt, const double* src, double* dst, unsigned long long* cfl_slot);
    // device time of `launches` step launches (fused: the fused step; with_fill:
    // the unfused step followed by the ghost fill) on scratch copies of q
    double time_steps(bool fused, bool with_fill, int launches, double t, double dt);
    void build_fuse_table();
    void fill_step_args(StepArgs& a, double t, double dt, unsigned long long* cfl_slot) const;
    void launch_step_form(const StepArgs& a, int n);
  public:
    void ensure_ghosts();  // run the deferred ghost update, if one is pending
  private:
    double* d_qalt_ = nullptr;
    DevBuf<FuseNbr> d_fuse_;
    bool fuse_ok_ = false;        // the table of the current mesh is complete
    bool ghosts_stale_ = false;
    int stale_min_ = 0, stale_max_ = 0;
    double stale_t_ = 0.0;
    bool saved_stale_ = false;    // ghosts_stale_ of the CFL-retry copy
    // the ghost cells are what a ghost update of every level gives (or such an
    // update is pending): a fused step reads exactly these values from the
    // neighbours.  False after initialize without init_ghostcell (qinit's own
    // ghost values), set_q and level updates, until the next full ghost update.
    bool ghosts_filled_ = false;
    bool saved_filled_ = false;
    int fused_used_ = 0;          // the last advance ran the fused step
    // --- macro step ---
    void run_schedule(double t, double dt);  // the level schedule of one advance_all_levels
    std::vector<uintptr_t> macro_fingerprint() const;
    void drop_macro_graph();
    void launch_level_step_slots(const int32_t* d_slots, int n, double t, double dt, unsigned long long* cfl_slot);
    void launch_levels_step_slots(const int32_t* d_slots, int n, int lvl0, int nlvl, const double* t,
                                  const double* dt, unsigned long long* cfl_slot);

    fcb_options_t opt_;
    cudaStream_t st_;
    int nx_, ny_;
    int64_t stride_;      // doubles per slot
    int aux_kind_;
    QuadForest forest_;
    std::vector<int> slot_of_;        // per leaf
    std::vector<Neighbors> nbrs_;     // per leaf
    std::vector<int> free_slots_;
    int nslots_used_ = 0;
    int capacity_ = 0;
    // device arena
    double* d_q_ = nullptr;
    double* d_qlast_ = nullptr;
    double* d_qti_ = nullptr;
    double* d_qsave_ = nullptr;
    double* d_aux_ = nullptr;         // stored aux (bathymetry), recomputed after every mesh change
    int64_t aux_stride_ = 0;
    PatchMeta* d_meta_ = nullptr;
    std::vector<PatchMeta> h_meta_;  // host copy of the slot metadata
    // level lists (device), grouped by level
    // serving: the schedule counters of the macro step in progress, and the
    // level updates and time interpolations of its current fine step
    struct SchedCounter { int last_step = 0, step_inc = 1, total_steps = 1; double current_time = 0.0, dt_step = 0.0; };
    std::vector<SchedCounter> sv_ts_;
    int sv_nf_ = 0;
    struct SvStep { int level; double t, dt; };
    std::vector<SvStep> sv_steps_;
    std::vector<std::pair<int, double>> sv_ti_;
    DevBuf<int32_t> d_xfer_, d_xfer_fine_;  // regrid transfer lists
    DevBuf<int32_t> d_level_slots_;
    std::vector<int> level_begin_;    // size maxlevel+2
    int gmin_ = 0, gmax_ = 0;         // coarsest and finest leaf level (set with the level lists)
    std::vector<int32_t> h_level_slots_;
    DevBuf<int32_t> d_ti_slots_;      // per level: slots with fine-grid neighbours
    std::vector<int> ti_begin_;
    DevBuf<int32_t> d_all_slots_;     // all leaves in Morton order
    // ghost plans
    std::map<std::tuple<int, int, int>, GhostPlan> plans_;
    std::vector<GhostOp> h_ops_;
    DevBuf<GhostOp> d_ops_;
    std::vector<int32_t> h_groups_;  // absolute op indices; one extra end marker per plan wave
    DevBuf<int32_t> d_groups_;
    bool ops_dirty_ = true;
    // scalars
    unsigned long long* d_cfl_ = nullptr;  // [0]: advance accumulator, [1]: level / batch
    unsigned long long* h_cfl_ = nullptr;  // pinned readback of one CFL word
    double read_cfl(const unsigned long long* d);  // copy one CFL word back and synchronize
    double* d_scratch_ = nullptr;          // tagging / mass output
    size_t scratch_cap_ = 0;
    // per-patch single_step_update batching
    std::vector<int32_t> pending_;
    DevBuf<int32_t> d_pending_;
    // contiguous staging buffer for host transfers
    double* d_stage_ = nullptr;
    size_t stage_cap_ = 0;
    // macro-step graph: per step launch {dt, vt} in a device table, so that one
    // captured graph replays every macro step of a mesh
    bool dry_ = false;               // schedule pass that only fills the table
    bool use_dyn_ = false;           // step launches read {dt, vt} from the table
    double* h_dyn_ = nullptr;        // pinned
    size_t dyn_cap_ = 0;             // entries
    int dyn_n_ = 0;
    DevBuf<double> d_dyn_;
    uint64_t mesh_version_ = 0;
    cudaGraphExec_t macro_exec_ = nullptr;
    cudaStream_t cap_st_ = nullptr;  // capture stream (the caller's stream may be the legacy one)
    // autotuner
    int tune_step_form(const StepArgs& a, int n);
    int tune_ghost_unroll(const GhostPlan& g);
    int step_form_used_ = 0;
    int bands_used_ = 1;             // row bands of the last four-barrier launch
    int ghost_unroll_ = 0;
    std::vector<uintptr_t> macro_key_, macro_seen_;
    fcb_counters_t macro_delta_{};
    // state
    bool initialized_ = false;
    double curr_time_ = 0.0;
    fcb_counters_t cnt_{};
};

}  // namespace fcb
