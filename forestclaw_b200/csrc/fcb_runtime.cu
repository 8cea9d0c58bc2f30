// Host runtime: forest management, slot arena, ghost plans and the level
// schedule of ForestClaw's time-stepping core on one GPU.
#include "fcb_runtime.hpp"
#include "fcb_output.hpp"

#include <algorithm>
#include <cmath>
#include <mutex>
#include <thread>
#include <exception>
#include <cstring>
#include <functional>
#include <unordered_map>

namespace fcb {

template <class T>
void DevBuf<T>::reserve(size_t n) {
    if (n <= cap) return;
    size_t nc = std::max(n, cap + cap / 2);
    T* np = nullptr;
    if (cudaMalloc(&np, nc * sizeof(T)) != cudaSuccess) throw Error(FCB_ERR_CUDA, "cudaMalloc failed (DevBuf)");
    if (p) {
        cudaDeviceSynchronize();
        cudaFree(p);
    }
    p = np;
    cap = nc;
}
template <class T>
void DevBuf<T>::release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
}
template struct DevBuf<int32_t>;
template struct DevBuf<GhostOp>;
template struct DevBuf<unsigned long long>;
template struct DevBuf<PatchDesc>;
template struct DevBuf<double>;
template struct DevBuf<TsOp>;

namespace {
cudaMemPool_t arena_pool() {
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) throw Error(FCB_ERR_CUDA, "cudaGetDevice failed");
    std::lock_guard<std::mutex> lk(mu);
    auto it = pools.find(dev);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) throw Error(FCB_ERR_CUDA, "cudaMemPoolCreate failed");
    uint64_t keep = UINT64_MAX;  // freed blocks stay in the pool for the next allocation
    if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess)
        throw Error(FCB_ERR_CUDA, "cudaMemPoolSetAttribute failed");
    pools[dev] = pool;
    return pool;
}
}  // namespace

template <class T>
void Context::arena_alloc(T*& p, size_t bytes) {
    void* q = nullptr;
    check(cudaMallocFromPoolAsync(&q, std::max<size_t>(bytes, 256), arena_pool(), st_), "arena allocation");
    p = static_cast<T*>(q);
}

void Context::arena_free(void* p) {
    if (p) cudaFreeAsync(p, st_);
}

void Context::check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Error(FCB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

static int solver_meqn(int kind) {
    switch (kind) {
        case FCB_SOLVER_ADVECTION: return 1;
        case FCB_SOLVER_ADVECTION_MANIFOLD: return 1;
        case FCB_SOLVER_SWE_ROE: return 3;
        case FCB_SOLVER_EULER4_ROE: return 4;
        case FCB_SOLVER_GEOCLAW_FWAVE: return 3;
        default: return -1;
    }
}

Context::Context(const fcb_options_t& o, cudaStream_t st, std::shared_ptr<Comm> comm)
    : opt_(o), st_(st), comm_(std::move(comm)) {
    auto bad = [](const std::string& m) { throw Error(FCB_ERR_INVALID, m); };
    if (comm_) {
        rank_ = comm_->rank();
        nranks_ = comm_->size();
        if (opt_.time_sync) bad("time-sync is not available in a partitioned solve");
        // the exchanges are host-driven collectives: every launch is issued from the host
        opt_.macro_graph = 0;
    }
    if (opt_.mx != opt_.my) bad("mx must equal my");
    if (opt_.mbc != 2) bad("mbc must be 2");
    if (opt_.mx != 8 && opt_.mx != 16 && opt_.mx != 32 && opt_.mx != 64) bad("mx must be 8, 16, 32 or 64");
    if (opt_.mcapa > 0 && opt_.solver_kind != FCB_SOLVER_ADVECTION_MANIFOLD)
        bad("capacity (mcapa > 0) is built for the manifold advection solver, which reads it in aux(1)");
    if (opt_.solver_kind == FCB_SOLVER_ADVECTION_MANIFOLD) {
        if (opt_.mcapa != 1 || opt_.maux < 3)
            bad("the manifold advection solver needs mcapa = 1 and maux >= 3 (capacity, then the edge velocities)");
        if (opt_.problem != FCB_PROBLEM_FILAMENT) bad("the manifold advection solver runs the filament problem");
        if (opt_.precision != 0 || (opt_.step_variant != 0 && opt_.step_variant != 1))
            bad("capacity is built in the four-barrier FP64 step form (step_variant 0 or 1)");
        if (opt_.time_sync) bad("time-sync is built for the shallow-water Roe solver");
        opt_.ghost_fusion = 1;  // the fused step is a pipelined form
    }
    if (opt_.problem == FCB_PROBLEM_FILAMENT && opt_.solver_kind != FCB_SOLVER_ADVECTION_MANIFOLD)
        bad("the filament problem stores capacity and edge velocities for the manifold advection solver");
    if (solver_meqn(opt_.solver_kind) < 0) bad("unknown solver kind");
    if (opt_.meqn != solver_meqn(opt_.solver_kind)) bad("meqn does not match the solver");
    if (opt_.mwaves != opt_.meqn) bad("mwaves must equal meqn for the configured solvers");
    for (int k = 0; k < 4; ++k)
        if (opt_.mthbc[k] != 1 && opt_.mthbc[k] != 3) bad("mthbc must be 1 (extrapolation) or 3 (wall)");
    if (opt_.minlevel < 0 || opt_.maxlevel < opt_.minlevel || opt_.maxlevel > 20) bad("bad minlevel/maxlevel");
    if (opt_.threshold_variable < 1 || opt_.threshold_variable > opt_.meqn) bad("bad threshold_variable");
    if (opt_.problem == FCB_PROBLEM_SWIRL && opt_.solver_kind != FCB_SOLVER_ADVECTION) bad("swirl needs advection");
    if (opt_.solver_kind == FCB_SOLVER_ADVECTION && opt_.problem != FCB_PROBLEM_SWIRL &&
        opt_.problem != FCB_PROBLEM_PERIODIC_DISC)
        bad("the advection solver takes its velocities from the swirl stream function or from stored aux");
    if (opt_.problem == FCB_PROBLEM_PERIODIC_DISC && (opt_.solver_kind != FCB_SOLVER_ADVECTION || opt_.maux < 2))
        bad("the periodic disc problem is advection with velocities in aux(1:2) (maux >= 2)");
    // a brick of b x b blocks is one tree with levels offset by log2(b)
    // (fclaw2d_map_brick.c: the brick's patch corners are that tree's corners)
    if (opt_.brick == 0) opt_.brick = 1;
    if (opt_.brick < 1 || opt_.brick > 1024 || (opt_.brick & (opt_.brick - 1)) != 0)
        bad("brick (mi = mj) must be a power of two");
    {
        int off = 0;
        while ((1 << off) < opt_.brick) ++off;
        opt_.minlevel += off;
        opt_.maxlevel += off;
        opt_.smooth_level += off;
    }
    if ((opt_.periodic_x || opt_.periodic_y) && (opt_.time_sync || comm_))
        bad("periodic domains run on one rank without time-sync");
    forest_.periodic_x = opt_.periodic_x != 0;
    forest_.periodic_y = opt_.periodic_y != 0;
    if ((opt_.problem == FCB_PROBLEM_RADIALDAM || opt_.problem == FCB_PROBLEM_RADIALDAM_CELLAVE ||
         opt_.problem == FCB_PROBLEM_HUMP) &&
        opt_.solver_kind != FCB_SOLVER_SWE_ROE)
        bad("radialdam and hump need SWE");
    if (opt_.problem < FCB_PROBLEM_SWIRL || opt_.problem > FCB_PROBLEM_FILAMENT) bad("unknown problem");
    if (opt_.ax == 0.0 && opt_.bx == 0.0 && opt_.ay == 0.0 && opt_.by == 0.0) {
        opt_.bx = 1.0;  // all four unset: the unit square
        opt_.by = 1.0;
    }
    if (!(opt_.bx > opt_.ax) || !(opt_.by > opt_.ay)) bad("the domain extent needs bx > ax and by > ay");
    if (opt_.problem == FCB_PROBLEM_QUADRANTS && opt_.solver_kind != FCB_SOLVER_EULER4_ROE) bad("quadrants needs Euler");
    if ((opt_.problem == FCB_PROBLEM_BATHY) != (opt_.solver_kind == FCB_SOLVER_GEOCLAW_FWAVE))
        bad("the bathymetry problem and the GeoClaw f-wave solver go together");
    aux_kind_ = (opt_.solver_kind == FCB_SOLVER_ADVECTION) ? (opt_.problem == FCB_PROBLEM_SWIRL ? AUX_SWIRL : AUX_STORED)
              : (opt_.solver_kind == FCB_SOLVER_GEOCLAW_FWAVE || opt_.solver_kind == FCB_SOLVER_ADVECTION_MANIFOLD)
                  ? AUX_STORED
                  : AUX_NONE;
    if (opt_.solver_kind == FCB_SOLVER_GEOCLAW_FWAVE) {
        if (opt_.maux != 1) bad("the GeoClaw solver reads aux(1) = b: maux must be 1");
        if (opt_.order[1] != 0) bad("rpt2_geoclaw stops in the reference: the GeoClaw solver needs order (., 0)");
        if (opt_.claw_version == 5) bad("the GeoClaw solver is on the clawpack 4.6 path");
        if (opt_.step_variant == 1 || opt_.step_variant == 2)
            bad("the GeoClaw solver exists in the pipelined step form only");
        if (!(opt_.dry_tolerance >= 0.0)) bad("dry_tolerance must be >= 0");
    }
    if (opt_.step_variant < 0 || opt_.step_variant > 5) bad("step_variant must be 0 to 5");
    if (opt_.precision != 0 && opt_.precision != 1) bad("precision must be 0 (FP64) or 1 (mixed)");
    const bool not_pipe = opt_.step_variant == 1 || opt_.step_variant == 2 || opt_.step_variant >= 4;
    if (opt_.precision == 1 && not_pipe) bad("the mixed-precision update exists in the pipelined step form only");
    if (opt_.step_variant >= 4 && opt_.solver_kind != FCB_SOLVER_SWE_ROE && opt_.solver_kind != FCB_SOLVER_EULER4_ROE)
        bad("row bands (step_variant 4, 5) are built for the Roe solvers' four-barrier form");
    if ((opt_.mx & (opt_.mx - 1)) != 0) bad("mx must be a power of two");
    if (opt_.macro_graph < 0 || opt_.macro_graph > 2) bad("macro_graph must be 0, 1 or 2");
    if (opt_.ghost_fusion < 0 || opt_.ghost_fusion > 2) bad("ghost_fusion must be 0, 1 or 2");
    if (opt_.src_term < 0 || opt_.src_term > 1) bad("src_term must be 0 (none) or 1 (axisymmetric Euler source)");
    if (opt_.src_term == 1 && opt_.solver_kind != FCB_SOLVER_EULER4_ROE)
        bad("the axisymmetric source (src_term 1) is the Euler equations' (shockbubble src2)");
    if (comm_) opt_.ghost_fusion = 1;  // a partitioned ghost update exchanges between ranks
    if (opt_.claw_version == 0) opt_.claw_version = 4;
    if (opt_.claw_version != 4 && opt_.claw_version != 5) bad("claw_version must be 4 (clawpack 4.6) or 5");
    if (opt_.claw_version == 5 && not_pipe && opt_.solver_kind != FCB_SOLVER_ADVECTION_MANIFOLD)
        bad("the clawpack 5 update exists in the pipelined step form only (and the four-barrier form with capacity)");
    if (opt_.time_sync) {
        if (opt_.solver_kind != FCB_SOLVER_SWE_ROE)
            bad("time-sync needs the conservative flux rpn2_cons, given here for the shallow-water Roe solver");
        if (opt_.precision != 0) bad("time-sync is FP64 only");
        if (opt_.step_variant != 0 && opt_.step_variant != 1 && opt_.step_variant != 3)
            bad("time-sync accumulates its registers in the four-barrier and pipelined step forms (step_variant 0, 1 "
                "or 3)");
        time_sync_ = true;
    }
    nx_ = opt_.mx + 2 * opt_.mbc;
    ny_ = opt_.my + 2 * opt_.mbc;
    const int64_t ps = (int64_t)opt_.meqn * nx_ * ny_;
    stride_ = (ps + 31) / 32 * 32;  // 256-byte aligned slots
    aux_stride_ = aux_kind_ == AUX_STORED ? ((int64_t)opt_.maux * nx_ * ny_ + 31) / 32 * 32 : 0;
    treg_stride_ = time_sync_ ? ((int64_t)RegLayout{opt_.mx, opt_.my, opt_.meqn}.size() + 31) / 32 * 32 : 0;
}

// The CFL words (first device use of a context: creation itself touches no device).
void Context::ensure_scalars() {
    if (d_cfl_) return;
    // [0] macro step, [1] level / batch, [2] global maximum, [3] autotuner,
    // [4] running maximum of the asynchronous macro steps
    check(cudaMalloc(&d_cfl_, 5 * sizeof(unsigned long long)), "cudaMalloc cfl");
    check(cudaMemsetAsync(d_cfl_, 0, 5 * sizeof(unsigned long long), st_), "memset cfl");
    check(cudaHostAlloc(&h_cfl_, sizeof(unsigned long long), cudaHostAllocDefault), "cudaHostAlloc cfl");
}

namespace {
// rank and size only: the host-only planning query makes no collective call
class PlanOnlyComm final : public Comm {
  public:
    PlanOnlyComm(int r, int n) : r_(r), n_(n) {}
    int rank() const override { return r_; }
    int size() const override { return n_; }
    void alltoallv(const void*, const size_t*, const size_t*, void*, const size_t*, const size_t*,
                   cudaStream_t) override {
        throw Error(FCB_ERR_INTERNAL, "planning query made a collective call");
    }
    void allreduce_max_u64(unsigned long long*, int, cudaStream_t) override {
        throw Error(FCB_ERR_INTERNAL, "planning query made a collective call");
    }
    void sync(cudaStream_t) override {}
    void abort(const std::string&) override {}

  private:
    int r_, n_;
};
}  // namespace

PartitionPlan Context::partition_plan(const fcb_options_t& o, const std::vector<Leaf>& leaves, int rank,
                                      int nranks, int minlevel, int maxlevel, int ti) {
    if (nranks < 1 || rank < 0 || rank >= nranks) throw Error(FCB_ERR_INVALID, "bad rank / number of ranks");
    Context c(o, nullptr, std::make_shared<PlanOnlyComm>(rank, nranks));
    c.forest_.leaves = leaves;
    const int n = (int)leaves.size();
    try {
        c.nbrs_.resize(n);
        for (int p = 0; p < n; ++p) c.nbrs_[p] = c.forest_.neighbors(p);
    } catch (const std::runtime_error& e) {
        throw Error(FCB_ERR_INVALID, std::string("leaves: ") + e.what());
    }
    c.partition_leaves();
    const std::vector<char> loc = c.local_set();
    c.slot_of_.assign(n, -1);
    int k = 0;
    for (int p = 0; p < n; ++p)
        if (loc[p]) c.slot_of_[p] = k++;
    c.capacity_ = std::max(1, k);
    PartitionPlan out;
    out.first = c.own_first_;
    out.count = c.own_count_;
    out.ghosts = k - c.own_count_;
    const PlanBuild b = c.build_plan(minlevel, maxlevel, ti);
    out.x1_send = b.x1.send_n;
    out.x1_recv = b.x1.recv_n;
    out.x2_send = b.x2.send_n;
    out.x2_recv = b.x2.recv_n;
    out.records = (int)b.ops.size();
    return out;
}

static double cfl_from_bits(unsigned long long b) {
    double v;
    std::memcpy(&v, &b, sizeof v);
    return v;
}

double Context::read_cfl(const unsigned long long* d) {
    check(cudaMemcpyAsync(h_cfl_, d, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st_), "cfl");
    synchronize();
    const double c = cfl_from_bits(*h_cfl_);
    if (std::isnan(c))
        throw Error(FCB_ERR_NUMERIC, "NaN CFL: non-finite state, or a Riemann problem the reference stops on "
                                     "(negative depth, sonic state in riemann_aug_JCP)");
    return c;
}

Context::~Context() {
    join_plans();
    cudaStreamSynchronize(st_);
    if (upload_ev_) cudaEventDestroy(upload_ev_);
    cudaFreeHost(h_ops_pinned_);
    cudaFreeHost(h_groups_pinned_);
    drop_macro_graph();
    if (cap_st_) cudaStreamDestroy(cap_st_);
    cudaFreeHost(h_dyn_);
    arena_free(d_q_);
    arena_free(d_qlast_);
    arena_free(d_qti_);
    arena_free(d_qsave_);
    arena_free(d_qalt_);
    arena_free(d_aux_);
    arena_free(d_meta_);
    arena_free(d_treg_);
    cudaStreamSynchronize(st_);
    cudaFree(d_cfl_);
    cudaFreeHost(h_cfl_);
    cudaFree(d_scratch_);
    cudaFree(d_stage_);
    cudaFreeHost(h_ts_ops_pinned_);
    cudaFreeHost(h_ts_groups_pinned_);
}

void Context::synchronize() { check(cudaStreamSynchronize(st_), "cudaStreamSynchronize"); }

void Context::ensure_capacity(int n) {
    if (n <= capacity_) return;
    const int nc = std::max({n, capacity_ + capacity_ / 2, 64});
    const size_t bytes = (size_t)nc * stride_ * sizeof(double);
    // stream-ordered: allocation, zeroing, copy of the old contents and the
    // free of the old arena are all queued on the context's stream
    auto grow = [&](double*& p) {
        double* np = nullptr;
        arena_alloc(np, bytes);
        check(cudaMemsetAsync(np, 0, bytes, st_), "cudaMemset arena");
        if (p) {
            check(cudaMemcpyAsync(np, p, (size_t)capacity_ * stride_ * sizeof(double), cudaMemcpyDeviceToDevice, st_),
                  "arena copy");
            arena_free(p);
        }
        p = np;
    };
    grow(d_q_);
    grow(d_qlast_);
    grow(d_qti_);
    if (time_sync_) {
        const size_t rb = (size_t)nc * treg_stride_ * sizeof(double);
        double* np = nullptr;
        arena_alloc(np, rb);
        check(cudaMemsetAsync(np, 0, rb, st_), "cudaMemset registers");
        if (d_treg_) {
            check(cudaMemcpyAsync(np, d_treg_, (size_t)capacity_ * treg_stride_ * sizeof(double),
                                  cudaMemcpyDeviceToDevice, st_),
                  "registers copy");
            arena_free(d_treg_);
        }
        d_treg_ = np;
    }
    if (!opt_.use_fixed_dt) grow(d_qsave_);
    arena_free(d_qalt_);  // the second arena of fused steps: reallocated at its next use
    d_qalt_ = nullptr;
    if (aux_kind_ == AUX_STORED) {  // recomputed for every patch by mesh_changed
        arena_free(d_aux_);
        d_aux_ = nullptr;
        arena_alloc(d_aux_, (size_t)nc * aux_stride_ * sizeof(double));
    }
    PatchMeta* nm = nullptr;
    arena_alloc(nm, (size_t)nc * sizeof(PatchMeta));
    if (d_meta_) {
        check(cudaMemcpyAsync(nm, d_meta_, (size_t)capacity_ * sizeof(PatchMeta), cudaMemcpyDeviceToDevice, st_), "meta");
        arena_free(d_meta_);
    }
    d_meta_ = nm;
    capacity_ = nc;
    // the arenas are used by synchronous copies on other streams too (uploads)
    check(cudaStreamSynchronize(st_), "sync");
}

int Context::alloc_slot() {
    if (!free_slots_.empty()) {
        const int s = free_slots_.back();
        free_slots_.pop_back();
        return s;
    }
    return nslots_used_++;
}

PatchMeta Context::meta_of(const Leaf& l) const {
    // fclaw2d_clawpatch.cpp clawpatch_define: xlower = ax + (bx-ax)*patch->xlower, dx = (xupper-xlower)/mx
    const double R = (double)QuadForest::kRoot;
    const double xl = (double)l.x / R, yl = (double)l.y / R;
    const double xu = (double)(l.x + QuadForest::width(l.level)) / R;
    const double yu = (double)(l.y + QuadForest::width(l.level)) / R;
    const double ax = opt_.ax, bx = opt_.bx, ay = opt_.ay, by = opt_.by;
    PatchMeta m;
    m.xlower = ax + (bx - ax) * xl;
    m.ylower = ay + (by - ay) * yl;
    m.dx = ((ax + (bx - ax) * xu) - m.xlower) / opt_.mx;
    m.dy = ((ay + (by - ay) * yu) - m.ylower) / opt_.my;
    m.level = l.level;
    m.flags = 0;
    return m;
}

// Neighbour relations of every leaf (point location in the Morton-sorted
// leaves), split over host threads for large forests.
void Context::compute_neighbors() {
    const int n = num_patches();
    nbrs_.resize(n);
    const int nt = (int)std::min<unsigned>({8u, std::max(1u, std::thread::hardware_concurrency()), (unsigned)(n / 512 + 1)});
    if (nt == 1) {
        for (int p = 0; p < n; ++p) nbrs_[p] = forest_.neighbors(p);
        return;
    }
    std::vector<std::thread> ts;
    std::vector<std::exception_ptr> err(nt);
    for (int k = 0; k < nt; ++k)
        ts.emplace_back([&, k] {
            try {
                for (int p = (int)((int64_t)n * k / nt); p < (int)((int64_t)n * (k + 1) / nt); ++p)
                    nbrs_[p] = forest_.neighbors(p);
            } catch (...) {
                err[k] = std::current_exception();
            }
        });
    for (auto& t : ts) t.join();
    for (auto& e : err)
        if (e) std::rethrow_exception(e);
}

void Context::mesh_changed() {
    discard_plans();
    ++mesh_version_;
    drop_macro_graph();
    const int n = num_patches();
    compute_neighbors();
    // slot metadata
    if (!partitioned()) {
        own_first_ = 0;
        own_count_ = n;
    }
    std::vector<PatchMeta> hm((size_t)capacity_);
    check(cudaStreamSynchronize(st_), "sync");
    for (int p = 0; p < n; ++p) {
        if (slot_of_[p] < 0) continue;  // neither owned nor in the ghost layer
        PatchMeta m = meta_of(forest_.leaves[p]);
        if (nbrs_[p].has_fine) m.flags |= PATCH_SAVE_LAST;
        hm[slot_of_[p]] = m;
    }
    check(cudaMemcpy(d_meta_, hm.data(), (size_t)capacity_ * sizeof(PatchMeta), cudaMemcpyHostToDevice), "meta upload");
    h_meta_ = hm;
    // level lists in Morton order
    const int L = QuadForest::kMaxLevel + 2;
    level_begin_.assign(L + 1, 0);
    ti_begin_.assign(L + 1, 0);
    std::vector<std::vector<int32_t>> by(L), tby(L);
    for (int p = own_first_; p < own_first_ + own_count_; ++p) {
        by[forest_.leaves[p].level].push_back(slot_of_[p]);
        if (nbrs_[p].has_fine) tby[forest_.leaves[p].level].push_back(slot_of_[p]);
    }
    h_level_slots_.clear();
    std::vector<int32_t> tis;
    for (int l = 0; l < L; ++l) {
        level_begin_[l] = (int)h_level_slots_.size();
        h_level_slots_.insert(h_level_slots_.end(), by[l].begin(), by[l].end());
        ti_begin_[l] = (int)tis.size();
        tis.insert(tis.end(), tby[l].begin(), tby[l].end());
    }
    level_begin_[L] = (int)h_level_slots_.size();
    ti_begin_[L] = (int)tis.size();
    gmin_ = forest_.min_level();
    gmax_ = forest_.max_level();
    d_level_slots_.reserve(std::max<size_t>(1, h_level_slots_.size()));
    d_ti_slots_.reserve(std::max<size_t>(1, tis.size()));
    d_all_slots_.reserve(std::max(1, own_count_));
    if (!h_level_slots_.empty())
        check(cudaMemcpy(d_level_slots_.p, h_level_slots_.data(), h_level_slots_.size() * 4, cudaMemcpyHostToDevice),
              "levels");
    if (!tis.empty()) check(cudaMemcpy(d_ti_slots_.p, tis.data(), tis.size() * 4, cudaMemcpyHostToDevice), "ti");
    // the owned leaves in Morton order (all leaves on one rank)
    std::vector<int32_t> all(slot_of_.begin() + own_first_, slot_of_.begin() + own_first_ + own_count_);
    if (!all.empty()) check(cudaMemcpy(d_all_slots_.p, all.data(), all.size() * 4, cudaMemcpyHostToDevice), "all slots");
    if ((opt_.problem == FCB_PROBLEM_BATHY || opt_.problem == FCB_PROBLEM_PERIODIC_DISC ||
         opt_.problem == FCB_PROBLEM_FILAMENT) &&
        own_count_ > 0) {
        // the stored aux depends on the cell centres only (bathymetry) or is
        // constant (the periodic problem's velocities): recomputed for every patch
        check(launch_setaux(opt_.problem, opt_.maux, opt_.problem_params, d_aux_, aux_stride_, d_all_slots_.p, d_meta_,
                            own_count_, opt_.mx, opt_.my, opt_.mbc, st_),
              "setaux");
        ++cnt_.count_kernel_launches;
    }
    plans_.clear();
    ts_plans_.clear();
    h_ts_ops_.clear();
    h_ts_groups_.clear();
    h_ops_.clear();
    h_groups_.clear();
    h_xitems_.clear();
    ops_dirty_ = true;
    build_fuse_table();
}

// ---------------------------------------------------------------------------
// Ghost plans
// ---------------------------------------------------------------------------
namespace {
struct Rect {
    int i0, i1, j0, j1;
    bool hits(const Rect& o) const { return i0 <= o.i1 && o.i0 <= i1 && j0 <= o.j1 && o.j0 <= j1; }
};
struct Touch {
    int64_t key;  // slot * 2 + time-interp array
    Rect r;
    bool write;
};
}  // namespace

// fclaw2d_ghost_update_async (src/fclaw2d_ghost_fill.c:611-831) on one rank:
// the records are emitted in the order the reference's callbacks run.
void Context::build_ops(int minlevel, int maxlevel, int ti, std::vector<GhostOp>& ops, size_t* phase_b) const {
    const int mx = opt_.mx, my = opt_.my;
    const int n = num_patches();
    std::vector<std::vector<int>> at((size_t)QuadForest::kMaxLevel + 1);
    for (int p = 0; p < n; ++p) at[forest_.leaves[p].level].push_back(p);
    auto level_list = [&](int l) -> const std::vector<int>& {
        static const std::vector<int> empty;
        return (l < 0 || l > QuadForest::kMaxLevel) ? empty : at[l];
    };
    auto xl = [&](int p) { return (double)forest_.leaves[p].x / (double)QuadForest::kRoot; };
    auto yl = [&](int p) { return (double)forest_.leaves[p].y / (double)QuadForest::kRoot; };
    auto base = [&](int type, int dst, int src, int face, int dti, int sti) {
        GhostOp o{};
        o.type = type; o.dst = dst; o.src = src; o.face = face; o.dst_ti = dti; o.src_ti = sti;
        for (int k = 0; k < 4; ++k) o.mthbc[k] = -1;
        return o;
    };
    // copy2ghost (fclaw2d_ghost_fill.c:145-168)
    auto copy2ghost = [&](int level, int t) {
        const double iw = (double)(1 << level);
        for (int p : level_list(level))
            for (int f = 0; f < 4; ++f) {
                if (nbrs_[p].face_rel[f] != REL_SAMESIZE) continue;
                const int q = nbrs_[p].face_nbr[f][0];
                const int* im = nbrs_[p].face_img[f];  // periodic image of q next to p
                GhostOp o = base(OP_COPY_FACE, p, q, f, t, t);
                o.dx = (int)((xl(p) - (xl(q) + im[0])) * iw * (double)mx);
                o.dy = (int)((yl(p) - (yl(q) + im[1])) * iw * (double)my);
                ops.push_back(o);
            }
        for (int p : level_list(level))
            for (int c = 0; c < 4; ++c) {
                if (nbrs_[p].corner_rel[c] != REL_SAMESIZE) continue;
                const int q = nbrs_[p].corner_nbr[c];
                const int* im = nbrs_[p].corner_img[c];
                GhostOp o = base(OP_COPY_CORNER, p, q, c, t, t);
                o.dx = (int)((xl(p) - (xl(q) + im[0]) + 0.) * (iw * (double)mx));
                o.dy = (int)((yl(p) - (yl(q) + im[1]) + 0.) * (iw * (double)my));
                ops.push_back(o);
            }
    };
    // half-size transform offset D: fine index = 2*coarse + D
    auto half = [&](int c, int f, const int* im, int& Dx, int& Dy) {
        const double ow = (double)(1 << forest_.leaves[f].level);
        Dx = (int)((xl(c) - (xl(f) + im[0])) * ow * (double)mx) - 1;
        Dy = (int)((yl(c) - (yl(f) + im[1])) * ow * (double)my) - 1;
    };
    // average2ghost (fclaw2d_ghost_fill.c:171-226), interpolate2ghost (:228-287)
    auto coarse_fine = [&](int level, int t, bool average) {
        for (int p : level_list(level)) {
            if (!nbrs_[p].on_cf) continue;
            for (int f = 0; f < 4; ++f) {
                if (nbrs_[p].face_rel[f] != REL_HALFSIZE) continue;
                for (int ig = 0; ig < 2; ++ig) {
                    const int q = nbrs_[p].face_nbr[f][ig];
                    GhostOp o = average ? base(OP_AVERAGE_FACE, p, q, f, t, 0) : base(OP_INTERP_FACE, q, p, f, 0, t);
                    half(p, q, nbrs_[p].face_img[f], o.dx, o.dy);
                    ops.push_back(o);
                }
            }
        }
        for (int p : level_list(level)) {
            if (!nbrs_[p].on_cf) continue;
            for (int c = 0; c < 4; ++c) {
                if (nbrs_[p].corner_rel[c] != REL_HALFSIZE) continue;
                const int q = nbrs_[p].corner_nbr[c];
                GhostOp o = average ? base(OP_AVERAGE_CORNER, p, q, c, t, 0) : base(OP_INTERP_CORNER, q, p, c, 0, t);
                half(p, q, nbrs_[p].corner_img[c], o.dx, o.dy);
                ops.push_back(o);
            }
        }
    };
    // setphysical (fclaw2d_ghost_fill.c:290-308) -> clawpack46_bc2
    auto setphysical = [&](int level, int t) {
        for (int p : level_list(level)) {
            GhostOp o = base(OP_PHYSBC, p, p, 0, t, t);
            bool any = false;
            for (int f = 0; f < 4; ++f)
                if (nbrs_[p].face_rel[f] == REL_BOUNDARY) { o.mthbc[f] = opt_.mthbc[f]; any = true; }
            if (any) ops.push_back(o);
        }
    };
    const int mincoarse = minlevel, maxcoarse = maxlevel - 1;
    for (int l = maxcoarse; l >= mincoarse; --l) coarse_fine(l, 0, true);
    if (ti) coarse_fine(mincoarse - 1, 1, true);
    for (int l = maxlevel; l >= minlevel; --l) copy2ghost(l, 0);
    if (ti) copy2ghost(minlevel - 1, 1);
    for (int l = maxcoarse; l >= mincoarse; --l) setphysical(l, 0);
    if (ti) setphysical(mincoarse - 1, 1);
    if (phase_b) *phase_b = ops.size();
    for (int l = maxcoarse; l >= mincoarse; --l) coarse_fine(l, 0, false);
    if (ti) coarse_fine(mincoarse - 1, 1, false);
    const int minfine = mincoarse + 1, maxfine = maxlevel;
    for (int l = maxfine; l >= minfine; --l) setphysical(l, 0);
    if (ti) setphysical(minfine - 1, 1);
    for (int l = maxlevel; l >= minlevel; --l) setphysical(l, 0);
    if (ti) setphysical(minlevel - 1, 1);
}

// A ghost plan.  One rank: every record, in waves.  Partitioned: the records
// whose destination this rank owns, in two wave sets (averages / copies /
// coarse physical boundaries, then interpolations / remaining physical
// boundaries), and the two exchanges before them.  No record writes a patch
// interior, and the interpolations from level l read coarse ghost cells before
// the interpolations into level l (which come later, l descending) write them,
// so the first set reads only source interiors as they were before the update,
// and the second reads sources as the first set left them: sending those two
// states of the other ranks' patches reproduces the one-rank order exactly.
Context::PlanBuild Context::build_plan(int minlevel, int maxlevel, int ti) const {
    std::vector<GhostOp> ops;
    size_t phase_b = 0;
    build_ops(minlevel, maxlevel, ti, ops, &phase_b);
    if (!partitioned()) {
        for (GhostOp& o : ops) {
            o.dst = slot_of_[o.dst];
            o.src = slot_of_[o.src];
        }
        PlanBuild b = make_waves(ops);
        b.nA = (int)b.wave_begin.size() - 1;
        return b;
    }
    // exchange items (leaf * 2 + array) this rank receives from / sends to each rank
    const int R = nranks_;
    std::vector<std::vector<int64_t>> recv[2], send[2];
    for (int x = 0; x < 2; ++x) {
        recv[x].resize(R);
        send[x].resize(R);
    }
    bool any[2] = {false, false};
    std::vector<GhostOp> mine[2];
    for (size_t k = 0; k < ops.size(); ++k) {
        GhostOp o = ops[k];
        const int x = k < phase_b ? 0 : 1;
        const int od = owner_[o.dst], os = owner_[o.src];
        if (od != os) {
            any[x] = true;
            const int64_t item = (int64_t)o.src * 2 + o.src_ti;
            if (od == rank_) recv[x][os].push_back(item);
            else if (os == rank_) send[x][od].push_back(item);
        }
        if (od != rank_) continue;
        o.dst = slot_of_[o.dst];
        o.src = slot_of_[o.src];
        if (o.dst < 0 || o.src < 0) throw Error(FCB_ERR_INTERNAL, "ghost record outside the local patches");
        mine[x].push_back(o);
    }
    PlanBuild b = make_waves(mine[0]);
    b.nA = (int)b.wave_begin.size() - 1;
    PlanBuild c = make_waves(mine[1]);
    const int nops = (int)b.ops.size(), ngroups = (int)b.groups.size();
    b.ops.insert(b.ops.end(), c.ops.begin(), c.ops.end());
    for (size_t w = 1; w < c.wave_begin.size(); ++w) b.wave_begin.push_back(c.wave_begin[w] + nops);
    b.group_begin.pop_back();
    for (int g : c.group_begin) b.group_begin.push_back(g + ngroups);
    for (int32_t g : c.groups) b.groups.push_back(g + nops);
    for (int x = 0; x < 2; ++x) {
        XList& xl = x == 0 ? b.x1 : b.x2;
        xl.any = any[x];
        xl.send_n.assign(R, 0);
        xl.recv_n.assign(R, 0);
        for (int r = 0; r < R; ++r) {
            for (auto* v : {&recv[x][r], &send[x][r]}) {
                std::sort(v->begin(), v->end());
                v->erase(std::unique(v->begin(), v->end()), v->end());
            }
            for (int64_t it : send[x][r]) xl.send.push_back(slot_of_[it >> 1] * 2 + (int32_t)(it & 1));
            for (int64_t it : recv[x][r]) {
                const int sl = slot_of_[it >> 1];
                if (sl < 0) throw Error(FCB_ERR_INTERNAL, "ghost-layer patch without a slot");
                xl.recv.push_back(sl * 2 + (int32_t)(it & 1));
            }
            xl.send_n[r] = (int)send[x][r].size();
            xl.recv_n[r] = (int)recv[x][r].size();
        }
    }
    return b;
}

// Records in waves: each record goes one wave after the latest earlier record
// it conflicts with (read-after-write, write-after-read, write-after-write on
// overlapping cells of the same array), so the records of a wave are
// independent and the waves keep the reference's order.
Context::PlanBuild Context::make_waves(const std::vector<GhostOp>& ops) const {
    const int mx = opt_.mx, my = opt_.my, mbc = opt_.mbc;
    const Rect whole{1 - mbc, mx + mbc, 1 - mbc, my + mbc};
    const Rect interior{1, mx, 1, my};
    std::vector<int> wave(ops.size(), 0);
    // writes and reads seen so far, per array (slot * 2 + time-interp flag):
    // a read conflicts only with writes, a write with both.  Each array's
    // touches form a list through flat arrays (newest first), no allocation
    // per array.
    const size_t narr = (size_t)2 * std::max(1, capacity_);
    struct Seen {
        Rect r;
        int wave;
        int next;
    };
    std::vector<Seen> seen;
    seen.reserve(2 * ops.size());
    std::vector<int> head_w(narr, -1), head_r(narr, -1);
    auto band = [&](int face) -> Rect {
        if (face == 0) return {1 - mbc, 0, 1, my};
        if (face == 1) return {mx + 1, mx + mbc, 1, my};
        if (face == 2) return {1, mx, 1 - mbc, 0};
        return {1, mx, my + 1, my + mbc};
    };
    auto corner = [&](int c) -> Rect {
        const int i0 = (c & 1) ? mx + 1 : 1 - mbc, j0 = (c & 2) ? my + 1 : 1 - mbc;
        return {i0, i0 + mbc - 1, j0, j0 + mbc - 1};
    };
    auto shift = [](Rect r, int dx, int dy) { return Rect{r.i0 + dx, r.i1 + dx, r.j0 + dy, r.j1 + dy}; };
    auto clip = [&](Rect r) {
        return Rect{std::max(r.i0, whole.i0), std::min(r.i1, whole.i1), std::max(r.j0, whole.j0), std::min(r.j1, whole.j1)};
    };
    for (size_t k = 0; k < ops.size(); ++k) {
        const GhostOp& o = ops[k];
        Touch t[2];
        const int64_t kd = (int64_t)o.dst * 2 + o.dst_ti, ks = (int64_t)o.src * 2 + o.src_ti;
        switch (o.type) {
            case OP_COPY_FACE:
                t[0] = {kd, band(o.face), true};
                t[1] = {ks, shift(band(o.face), o.dx, o.dy), false};
                break;
            case OP_COPY_CORNER:
                t[0] = {kd, corner(o.face), true};
                t[1] = {ks, shift(corner(o.face), o.dx, o.dy), false};
                break;
            case OP_AVERAGE_FACE:
            case OP_AVERAGE_CORNER:
                t[0] = {kd, o.type == OP_AVERAGE_FACE ? band(o.face) : corner(o.face), true};
                t[1] = {ks, interior, false};
                break;
            case OP_INTERP_FACE:
            case OP_INTERP_CORNER: {
                // coarse cells read: the coarse band (one cell deep) grown by one
                Rect cb;
                if (o.type == OP_INTERP_FACE) {
                    if (o.face == 0) cb = {1, mbc / 2, 1, mx};
                    else if (o.face == 1) cb = {mx - mbc / 2 + 1, mx, 1, mx};
                    else if (o.face == 2) cb = {1, mx, 1, mbc / 2};
                    else cb = {1, mx, my - mbc / 2 + 1, my};
                } else {
                    const int i0 = (o.face & 1) ? mx - mbc / 2 + 1 : 1, j0 = (o.face & 2) ? my - mbc / 2 + 1 : 1;
                    cb = {i0, i0 + mbc / 2 - 1, j0, j0 + mbc / 2 - 1};
                }
                t[0] = {ks, Rect{cb.i0 - 1, cb.i1 + 1, cb.j0 - 1, cb.j1 + 1}, false};
                t[1] = {kd, clip(Rect{2 * cb.i0 + o.dx, 2 * cb.i1 + o.dx + 1, 2 * cb.j0 + o.dy, 2 * cb.j1 + o.dy + 1}), true};
                break;
            }
            default:  // OP_PHYSBC: reads and writes the whole array
                t[0] = {kd, whole, true};
                t[1] = {kd, whole, false};
                break;
        }
        int w = 0;
        for (const Touch& a : t) {
            for (int i = head_w[(size_t)a.key]; i >= 0; i = seen[i].next)
                if (seen[i].wave >= w && a.r.hits(seen[i].r)) w = seen[i].wave + 1;
            if (a.write)
                for (int i = head_r[(size_t)a.key]; i >= 0; i = seen[i].next)
                    if (seen[i].wave >= w && a.r.hits(seen[i].r)) w = seen[i].wave + 1;
        }
        wave[k] = w;
        for (const Touch& a : t) {
            int& h = (a.write ? head_w : head_r)[(size_t)a.key];
            seen.push_back({a.r, w, h});
            h = (int)seen.size() - 1;
        }
    }
    const int nw = ops.empty() ? 0 : *std::max_element(wave.begin(), wave.end()) + 1;
    PlanBuild b;
    b.wave_begin.assign(nw + 1, 0);
    std::vector<int> count(nw, 0);
    for (int w : wave) ++count[w];
    for (int w = 0; w < nw; ++w) b.wave_begin[w + 1] = b.wave_begin[w] + count[w];
    // records ordered by (wave, destination), keeping the reference's order
    // among equal keys: a stable counting sort by destination slot, then a
    // stable counting sort by wave
    const size_t n = ops.size();
    std::vector<int> by_dst(n);
    {
        std::vector<int> start((size_t)std::max(1, capacity_) + 1, 0);
        for (const GhostOp& o : ops) {
            if (o.dst < 0 || o.dst >= std::max(1, capacity_)) throw Error(FCB_ERR_INTERNAL, "ghost record outside the arena");
            ++start[(size_t)o.dst + 1];
        }
        for (size_t d = 1; d < start.size(); ++d) start[d] += start[d - 1];
        for (size_t k = 0; k < n; ++k) by_dst[start[(size_t)ops[k].dst]++] = (int)k;
    }
    b.ops.resize(n);
    std::vector<int> pos(b.wave_begin.begin(), b.wave_begin.end() - (nw ? 1 : 0));
    for (int k : by_dst) b.ops[pos[wave[k]]++] = ops[k];
    // within a wave, records with the same destination patch form one group
    b.group_begin.assign(nw + 1, 0);
    for (int w = 0; w < nw; ++w) {
        b.group_begin[w] = (int)b.groups.size();
        for (int k = b.wave_begin[w]; k < b.wave_begin[w + 1]; ++k)
            if (k == b.wave_begin[w] || b.ops[k].dst != b.ops[k - 1].dst) b.groups.push_back(k);
        b.groups.push_back(b.wave_begin[w + 1]);  // end marker of the wave
    }
    b.group_begin[nw] = (int)b.groups.size();
    return b;
}

const GhostPlan& Context::commit_plan(const std::tuple<int, int, int>& key, PlanBuild&& b) {
    GhostPlan g;
    g.first = h_ops_.size();
    g.first_group = h_groups_.size();
    g.wave_begin = std::move(b.wave_begin);
    g.group_begin = std::move(b.group_begin);
    for (int32_t k : b.groups) h_groups_.push_back((int32_t)(g.first + k));
    h_ops_.insert(h_ops_.end(), b.ops.begin(), b.ops.end());
    g.nA = b.nA;
    g.x1 = std::move(b.x1);
    g.x2 = std::move(b.x2);
    for (XList* x : {&g.x1, &g.x2}) {
        for (const auto* v : {&x->send, &x->recv})
            for (int32_t it : *v)
                if (it < 0 || (it >> 1) >= capacity_) throw Error(FCB_ERR_INTERNAL, "exchange item outside the arena");
        x->send_first = h_xitems_.size();
        h_xitems_.insert(h_xitems_.end(), x->send.begin(), x->send.end());
        x->recv_first = h_xitems_.size();
        h_xitems_.insert(h_xitems_.end(), x->recv.begin(), x->recv.end());
    }
    ops_dirty_ = true;
    return plans_.emplace(key, std::move(g)).first->second;
}

const GhostPlan& Context::plan(int minlevel, int maxlevel, int ti) {
    const auto key = std::make_tuple(minlevel, maxlevel, ti);
    auto it = plans_.find(key);
    if (it != plans_.end()) return it->second;
    if (!plan_todo_.empty()) {
        finish_plans();
        it = plans_.find(key);
        if (it != plans_.end()) return it->second;
    }
    return commit_plan(key, build_plan(minlevel, maxlevel, ti));
}

void Context::start_plans(const std::vector<std::tuple<int, int, int>>& keys) {
    finish_plans();
    for (const auto& k : keys)
        if (!plans_.count(k) && std::find(plan_todo_.begin(), plan_todo_.end(), k) == plan_todo_.end())
            plan_todo_.push_back(k);
    if (plan_todo_.empty()) return;
    plan_built_.assign(plan_todo_.size(), PlanBuild{});
    plan_err_.assign(plan_todo_.size(), nullptr);
    // the builds only read the forest, neighbour tables, slot map and options
    for (size_t k = 0; k < plan_todo_.size(); ++k)
        plan_threads_.emplace_back([this, k] {
            try {
                const auto& t = plan_todo_[k];
                plan_built_[k] = build_plan(std::get<0>(t), std::get<1>(t), std::get<2>(t));
            } catch (...) {
                plan_err_[k] = std::current_exception();
            }
        });
}

// Starts the builds of the ghost plans that one macro step uses on the current
// mesh (the keys come from a dry run of the schedule, which launches nothing)
// and of the full ghost update.  The next plan() that needs any of them waits
// for all.
void Context::prefetch_plans() {
    const bool dyn0 = use_dyn_;
    const int n0 = dyn_n_;
    use_dyn_ = true;
    dry_ = true;
    dyn_n_ = 0;
    dry_plan_keys_.clear();
    try {
        run_schedule(curr_time_, 1.0);
    } catch (...) {
        dry_ = false;
        use_dyn_ = dyn0;
        dyn_n_ = n0;
        throw;
    }
    dry_ = false;
    use_dyn_ = dyn0;
    dyn_n_ = n0;
    dry_plan_keys_.emplace_back(gmin_, gmax_, 0);
    start_plans(dry_plan_keys_);
}

void Context::discard_plans() noexcept {
    join_plans();
    plan_todo_.clear();
    plan_built_.clear();
    plan_err_.clear();
}

void Context::join_plans() noexcept {
    for (auto& t : plan_threads_)
        if (t.joinable()) t.join();
    plan_threads_.clear();
}

void Context::finish_plans() {
    join_plans();
    if (plan_todo_.empty()) return;
    std::exception_ptr err;
    for (size_t k = 0; k < plan_todo_.size(); ++k) {
        if (plan_err_[k]) {
            if (!err) err = plan_err_[k];
            continue;
        }
        if (!plans_.count(plan_todo_[k])) commit_plan(plan_todo_[k], std::move(plan_built_[k]));
    }
    plan_todo_.clear();
    plan_built_.clear();
    plan_err_.clear();
    if (err) std::rethrow_exception(err);
}

// Copies the op and group buffers to the device through pinned staging, in
// stream order (ghost launches already queued read the old contents first).
void Context::upload_ops() {
    if (upload_ev_) check(cudaEventSynchronize(upload_ev_), "ops upload");  // staging free again
    else check(cudaEventCreateWithFlags(&upload_ev_, cudaEventDisableTiming), "cudaEventCreate");
    // staging grows geometrically from 64 Ki records (a pinned free synchronises the device)
    if (h_ops_.size() > h_ops_pinned_cap_) {
        cudaFreeHost(h_ops_pinned_);
        h_ops_pinned_ = nullptr;
        h_ops_pinned_cap_ = std::max({h_ops_.size(), 2 * h_ops_pinned_cap_, (size_t)1 << 16});
        check(cudaHostAlloc(&h_ops_pinned_, h_ops_pinned_cap_ * sizeof(GhostOp), cudaHostAllocDefault), "host ops");
    }
    if (h_groups_.size() > h_groups_pinned_cap_) {
        cudaFreeHost(h_groups_pinned_);
        h_groups_pinned_ = nullptr;
        h_groups_pinned_cap_ = std::max({h_groups_.size(), 2 * h_groups_pinned_cap_, (size_t)1 << 16});
        check(cudaHostAlloc(&h_groups_pinned_, h_groups_pinned_cap_ * sizeof(int32_t), cudaHostAllocDefault),
              "host groups");
    }
    d_ops_.reserve(std::max<size_t>(1, h_ops_.size()));
    d_groups_.reserve(std::max<size_t>(1, h_groups_.size()));
    if (!h_ops_.empty()) {
        std::memcpy(h_ops_pinned_, h_ops_.data(), h_ops_.size() * sizeof(GhostOp));
        check(cudaMemcpyAsync(d_ops_.p, h_ops_pinned_, h_ops_.size() * sizeof(GhostOp), cudaMemcpyHostToDevice, st_),
              "ops");
    }
    if (!h_ts_ops_.empty()) {
        if (h_ts_ops_.size() > h_ts_ops_pinned_cap_) {
            cudaFreeHost(h_ts_ops_pinned_);
            h_ts_ops_pinned_ = nullptr;
            h_ts_ops_pinned_cap_ = std::max(h_ts_ops_.size(), 2 * h_ts_ops_pinned_cap_);
            check(cudaHostAlloc(&h_ts_ops_pinned_, h_ts_ops_pinned_cap_ * sizeof(TsOp), cudaHostAllocDefault),
                  "host ts ops");
        }
        if (h_ts_groups_.size() > h_ts_groups_pinned_cap_) {
            cudaFreeHost(h_ts_groups_pinned_);
            h_ts_groups_pinned_ = nullptr;
            h_ts_groups_pinned_cap_ = std::max(h_ts_groups_.size(), 2 * h_ts_groups_pinned_cap_);
            check(cudaHostAlloc(&h_ts_groups_pinned_, h_ts_groups_pinned_cap_ * sizeof(int32_t), cudaHostAllocDefault),
                  "host ts groups");
        }
        d_ts_ops_.reserve(h_ts_ops_.size());
        d_ts_groups_.reserve(h_ts_groups_.size());
        std::memcpy(h_ts_ops_pinned_, h_ts_ops_.data(), h_ts_ops_.size() * sizeof(TsOp));
        std::memcpy(h_ts_groups_pinned_, h_ts_groups_.data(), h_ts_groups_.size() * sizeof(int32_t));
        check(cudaMemcpyAsync(d_ts_ops_.p, h_ts_ops_pinned_, h_ts_ops_.size() * sizeof(TsOp), cudaMemcpyHostToDevice,
                              st_),
              "ts ops");
        check(cudaMemcpyAsync(d_ts_groups_.p, h_ts_groups_pinned_, h_ts_groups_.size() * sizeof(int32_t),
                              cudaMemcpyHostToDevice, st_),
              "ts groups");
    }
    if (!h_groups_.empty()) {
        std::memcpy(h_groups_pinned_, h_groups_.data(), h_groups_.size() * sizeof(int32_t));
        check(cudaMemcpyAsync(d_groups_.p, h_groups_pinned_, h_groups_.size() * sizeof(int32_t),
                              cudaMemcpyHostToDevice, st_),
              "groups");
    }
    if (!h_xitems_.empty()) {
        // exchange items (partitioned solves): small, copied synchronously
        d_xitems_.reserve(h_xitems_.size());
        check(cudaMemcpyAsync(d_xitems_.p, h_xitems_.data(), h_xitems_.size() * sizeof(int32_t),
                              cudaMemcpyHostToDevice, st_),
              "exchange items");
        check(cudaStreamSynchronize(st_), "sync");
    }
    check(cudaEventRecord(upload_ev_, st_), "cudaEventRecord");
    ops_dirty_ = false;
}

// ---------------------------------------------------------------------------
// Time synchronisation (fclaw2d_time_sync.c:157-205, correct_coarse_cells
// :115-155).  Per level L from the finest option level down to minlevel the
// reference runs: A(L) same-size corrections of the level's patches, B(L) reset
// of their same-size registers, and below the finest level C(L)
// fine-to-coarse corrections at the level's coarse/fine faces and D(L) reset
// of those registers on levels L and L+1; finally E, the reset of the
// physical-boundary registers of every level.  Records are grouped per patch
// (one CTA each, the records of a patch in order); launches merge steps that
// touch disjoint data: B(L+1)+A(L) or D(L+1)+A(L) (registers of other levels
// vs q and same-size registers of L), B(L)+C(L) (same-size vs coarse/fine
// registers), and D(min)+E (different faces).
// ---------------------------------------------------------------------------
const Context::TsPlan& Context::ts_plan(int minlevel) {
    auto it = ts_plans_.find(minlevel);
    if (it != ts_plans_.end()) return it->second;
    const int n = num_patches();
    const int top = opt_.maxlevel;
    std::vector<std::vector<int>> at((size_t)QuadForest::kMaxLevel + 2);
    for (int p = 0; p < n; ++p) at[forest_.leaves[p].level].push_back(p);
    auto level_list = [&](int l) -> const std::vector<int>& {
        static const std::vector<int> empty;
        return (l < 0 || l > QuadForest::kMaxLevel) ? empty : at[l];
    };
    auto xl = [&](int p) { return (double)forest_.leaves[p].x / (double)QuadForest::kRoot; };
    auto yl = [&](int p) { return (double)forest_.leaves[p].y / (double)QuadForest::kRoot; };
    using Step = std::vector<std::pair<int, TsOp>>;  // (patch, record) in reference order
    auto same = [&](int L) {
        Step st;
        const double iw = (double)(1 << L);
        for (int p : level_list(L))
            for (int f = 0; f < 4; ++f) {
                if (nbrs_[p].face_rel[f] != REL_SAMESIZE) continue;
                const int q = nbrs_[p].face_nbr[f][0];
                TsOp o{TS_SAMESIZE, slot_of_[p], f, slot_of_[q], 0, 0};
                // fclaw2d_patch_transform_face, same block: i2 = i1 + shift
                o.dx = (int)((xl(p) - xl(q)) * iw * (double)opt_.mx);
                o.dy = (int)((yl(p) - yl(q)) * iw * (double)opt_.my);
                st.push_back({p, o});
            }
        return st;
    };
    auto reset = [&](const std::vector<int>& ps, auto pred) {
        Step st;
        for (int p : ps)
            for (int f = 0; f < 4; ++f)
                if (pred(p, f)) st.push_back({p, TsOp{TS_RESET, slot_of_[p], f, 0, 0, 0}});
        return st;
    };
    auto f2c = [&](int L) {
        Step st;
        for (int p : level_list(L))
            for (int f = 0; f < 4; ++f) {
                if (nbrs_[p].face_rel[f] != REL_HALFSIZE) continue;
                for (int ig = 0; ig < 2; ++ig) {
                    const int q = nbrs_[p].face_nbr[f][ig];
                    TsOp o{TS_F2C, slot_of_[p], f, slot_of_[q], 0, 0};
                    // fclaw2d_patch_transform_face2, same block: first fine index 1 + D + 2(c-1)
                    const double ow = (double)(1 << forest_.leaves[q].level);
                    o.dx = (int)((xl(p) - xl(q)) * ow * (double)opt_.mx);
                    o.dy = (int)((yl(p) - yl(q)) * ow * (double)opt_.my);
                    st.push_back({p, o});
                }
            }
        return st;
    };
    auto rel = [&](int p, int f) { return nbrs_[p].face_rel[f]; };
    auto lev = [&](int p) { return (int)forest_.leaves[p].level; };
    std::vector<Step> launches;
    auto cat = [](Step a, const Step& b) {
        a.insert(a.end(), b.begin(), b.end());
        return a;
    };
    Step pending;
    for (int L = top; L >= minlevel; --L) {
        const Step A = same(L);
        launches.push_back(cat(pending, A));
        const Step B = reset(level_list(L), [&](int p, int f) { return rel(p, f) == REL_SAMESIZE && lev(p) == L; });
        if (L < top) {
            launches.push_back(cat(B, f2c(L)));
            Step D = reset(level_list(L), [&](int p, int f) { return rel(p, f) == REL_HALFSIZE && lev(p) == L; });
            D = cat(D, reset(level_list(L + 1),
                             [&](int p, int f) { return rel(p, f) == REL_DOUBLESIZE && lev(p) == L + 1; }));
            pending = D;
        } else {
            pending = B;
        }
    }
    Step E;
    for (int L = top; L >= minlevel; --L)
        E = cat(E, reset(level_list(L), [&](int p, int f) { return rel(p, f) == REL_BOUNDARY; }));
    launches.push_back(cat(pending, E));
    // group each launch's records per patch, patches in order of first appearance
    TsPlan plan;
    for (const Step& st : launches) {
        std::vector<int> order;
        std::unordered_map<int, std::vector<TsOp>> by;
        for (const auto& pr : st) {
            auto f = by.find(pr.first);
            if (f == by.end()) {
                order.push_back(pr.first);
                by[pr.first] = {pr.second};
            } else {
                f->second.push_back(pr.second);
            }
        }
        if (order.empty()) continue;
        plan.first_group.push_back(h_ts_groups_.size());
        plan.ngroups.push_back((int)order.size());
        for (int p : order) {
            h_ts_groups_.push_back((int32_t)h_ts_ops_.size());
            for (const TsOp& o : by[p]) h_ts_ops_.push_back(o);
        }
        h_ts_groups_.push_back((int32_t)h_ts_ops_.size());  // end marker of the launch
    }
    ops_dirty_ = true;
    return ts_plans_.emplace(minlevel, std::move(plan)).first->second;
}

void Context::time_sync(int minlevel) {
    const TsPlan& plan = ts_plan(minlevel);
    if (dry_) return;
    if (ops_dirty_) upload_ops();
    for (size_t k = 0; k < plan.ngroups.size(); ++k) {
        TsArgs a;
        a.q = d_q_;
        a.treg = d_treg_;
        a.q_stride = stride_;
        a.treg_stride = treg_stride_;
        a.meta = d_meta_;
        a.mx = opt_.mx; a.my = opt_.my; a.mbc = opt_.mbc; a.meqn = opt_.meqn;
        a.ops = d_ts_ops_.p;
        a.groups = d_ts_groups_.p + plan.first_group[k];
        a.ngroups = plan.ngroups[k];
        check(launch_ts_apply(a, st_), "time sync");
        ++cnt_.count_kernel_launches;
    }
}

void Context::run_plan(const GhostPlan& g) {
    if (ops_dirty_) upload_ops();
    ghost_unroll_ = opt_.step_variant == 0 ? tune_ghost_unroll(g) : 4;
    const int nw = (int)g.wave_begin.size() - 1;
    exchange(g.x1);
    for (int w = 0; w < nw; ++w) {
        if (w == g.nA) exchange(g.x2);
        GhostArgs a;
        a.q = d_q_;
        a.qti = d_qti_;
        a.stride = stride_;
        a.mx = opt_.mx; a.my = opt_.my; a.mbc = opt_.mbc; a.meqn = opt_.meqn;
        a.ops = d_ops_.p;
        a.groups = d_groups_.p + g.first_group + g.group_begin[w];  // group starts, then an end marker
        a.ngroups = g.group_begin[w + 1] - g.group_begin[w] - 1;
        a.interp_fp32 = opt_.precision == 1;
        check(launch_ghost_wave(a, st_, ghost_unroll_), "ghost wave");
        ++cnt_.count_ghost_waves;
        ++cnt_.count_kernel_launches;
    }
    if (g.nA >= nw) exchange(g.x2);
}

// The ghost-patch exchange (fclaw2d_exchange_ghost_patches_begin/_end,
// fclaw2d_exchange.c:308-413): whole patch arrays packed by slot, one
// alltoallv, unpacked into the ghost-layer slots.  Every rank calls it for
// every exchange whose list is non-empty on some rank.
void Context::exchange(const XList& x, const int32_t* d_items) {
    if (!partitioned() || !x.any) return;
    if (!d_items) d_items = d_xitems_.p;
    const int64_t ps = (int64_t)patch_size();
    const size_t ns = x.send.size(), nr = x.recv.size();
    d_xsend_.reserve(std::max<size_t>(1, ns * ps));
    d_xrecv_.reserve(std::max<size_t>(1, nr * ps));
    check(launch_pack_patches(d_q_, d_qti_, stride_, d_items + x.send_first, (int)ns, ps, d_xsend_.p, true, st_),
          "pack");
    std::vector<size_t> so(nranks_), sb(nranks_), ro(nranks_), rb(nranks_);
    size_t a = 0, b = 0;
    for (int r = 0; r < nranks_; ++r) {
        so[r] = a;
        sb[r] = (size_t)x.send_n[r] * ps * sizeof(double);
        a += sb[r];
        ro[r] = b;
        rb[r] = (size_t)x.recv_n[r] * ps * sizeof(double);
        b += rb[r];
    }
    comm_->alltoallv(d_xsend_.p, so.data(), sb.data(), d_xrecv_.p, ro.data(), rb.data(), st_);
    check(launch_pack_patches(d_q_, d_qti_, stride_, d_items + x.recv_first, (int)nr, ps, d_xrecv_.p, false, st_),
          "unpack");
    cnt_.count_kernel_launches += (ns ? 1 : 0) + (nr ? 1 : 0);
}

void Context::allgather_owned(const double* d_own, int per_leaf, double* d_all) {
    std::vector<size_t> so(nranks_, 0), sb(nranks_, (size_t)own_count_ * per_leaf * sizeof(double)), ro(nranks_),
        rb(nranks_);
    for (int r = 0; r < nranks_; ++r) {
        ro[r] = (size_t)cut_[r] * per_leaf * sizeof(double);
        rb[r] = (size_t)(cut_[r + 1] - cut_[r]) * per_leaf * sizeof(double);
    }
    comm_->alltoallv(d_own, so.data(), sb.data(), d_all, ro.data(), rb.data(), st_);
}

double Context::global_maximum(double v) {
    if (!partitioned()) return v;
    ensure_scalars();
    unsigned long long bits;
    std::memcpy(&bits, &v, sizeof bits);
    if (std::signbit(v)) bits = 0;  // CFL numbers are >= 0
    check(cudaMemcpyAsync(d_cfl_ + 2, &bits, sizeof bits, cudaMemcpyHostToDevice, st_), "global max");
    comm_->allreduce_max_u64(d_cfl_ + 2, 1, st_);
    check(cudaMemcpyAsync(h_cfl_, d_cfl_ + 2, sizeof bits, cudaMemcpyDeviceToHost, st_), "global max");
    comm_->sync(st_);
    return cfl_from_bits(*h_cfl_);
}

void Context::abort_comm(const std::string& why) noexcept {
    if (comm_) comm_->abort(why);
}

// ---------------------------------------------------------------------------
// Partition (fclaw2d_partition_domain, fclaw2d_partition.c:113-197, over
// p4est_wrap_partition): rank r owns the Morton range [cut_[r], cut_[r+1]).
// Cut r is the first leaf at which the running weight reaches r/R of the total
// (weight 2^level with weighted_partition and subcycling, else 1), moved to the
// nearer end of a complete family it would split (p4est's partition for
// coarsening).  The solution never depends on the cuts: they only balance work.
// ---------------------------------------------------------------------------
void Context::partition_leaves() {
    const int n = num_patches();
    const int R = nranks_;
    const int e = (opt_.subcycle && opt_.weighted_partition) ? 1 : 0;
    std::vector<uint64_t> pre((size_t)n + 1, 0);
    for (int p = 0; p < n; ++p) pre[p + 1] = pre[p] + ((uint64_t)1 << (e * forest_.leaves[p].level));
    const unsigned __int128 W = pre[n];
    cut_.assign(R + 1, 0);
    cut_[R] = n;
    for (int r = 1; r < R; ++r) {
        const uint64_t target = (uint64_t)((W * (unsigned)r + (unsigned)R - 1) / (unsigned)R);
        int k = (int)(std::lower_bound(pre.begin(), pre.end(), target) - pre.begin());
        k = std::min(k, n);
        for (int a = std::max(0, k - 3); a < k; ++a)
            if (forest_.is_first_sibling(a) && a + 4 > k) {
                k = (k - a <= a + 4 - k) ? a : a + 4;
                break;
            }
        cut_[r] = std::min(n, std::max(k, cut_[r - 1]));
    }
    owner_.assign(n, 0);
    for (int r = 0; r < R; ++r)
        for (int p = cut_[r]; p < cut_[r + 1]; ++p) owner_[p] = r;
    own_first_ = cut_[rank_];
    own_count_ = cut_[rank_ + 1] - cut_[rank_];
}

std::vector<char> Context::local_set() const {
    const int n = num_patches();
    std::vector<char> loc(n, 0);
    for (int p = own_first_; p < own_first_ + own_count_; ++p) {
        loc[p] = 1;
        const Neighbors& nb = nbrs_[p];
        for (int f = 0; f < 4; ++f)
            for (int k = 0; k < 2; ++k)
                if (nb.face_nbr[f][k] >= 0) loc[nb.face_nbr[f][k]] = 1;
        for (int c = 0; c < 4; ++c)
            if (nb.corner_nbr[c] >= 0) loc[nb.corner_nbr[c]] = 1;
    }
    return loc;
}

void Context::ghost_update(int minlevel, int maxlevel, double, int time_interp) {
    if (!d_q_) throw Error(FCB_ERR_STATE, "ghost_update before initialize");
    ensure_ghosts();
    if (dry_) {
        dry_plan_keys_.emplace_back(minlevel, maxlevel, time_interp);
        return;
    }
    run_plan(plan(minlevel, maxlevel, time_interp));
    if (minlevel <= gmin_ && maxlevel >= gmax_) ghosts_filled_ = true;
}

void Context::physical_set_bc(int level, int time_interp) {
    ensure_ghosts();
    std::vector<GhostOp> ops;
    for (int p = own_first_; p < own_first_ + own_count_; ++p) {
        if (forest_.leaves[p].level != level) continue;
        GhostOp o{};
        o.type = OP_PHYSBC; o.dst = o.src = slot_of_[p]; o.dst_ti = o.src_ti = time_interp;
        bool any = false;
        for (int f = 0; f < 4; ++f) {
            o.mthbc[f] = -1;
            if (nbrs_[p].face_rel[f] == REL_BOUNDARY) { o.mthbc[f] = opt_.mthbc[f]; any = true; }
        }
        if (any) ops.push_back(o);
    }
    if (ops.empty()) return;
    GhostPlan g;
    g.first = h_ops_.size();
    g.wave_begin = {0, (int)ops.size()};
    g.first_group = h_groups_.size();
    for (size_t k = 0; k < ops.size(); ++k) h_groups_.push_back((int32_t)(g.first + k));
    h_groups_.push_back((int32_t)(g.first + ops.size()));
    g.group_begin = {0, (int)ops.size() + 1};
    h_ops_.insert(h_ops_.end(), ops.begin(), ops.end());
    ops_dirty_ = true;
    run_plan(g);
}

// ---------------------------------------------------------------------------
// Stepping
// ---------------------------------------------------------------------------
void Context::launch_level_step_slots(const int32_t* d_slots, int n, double t, double dt,
                                      unsigned long long* cfl_slot) {
    const double tl[1] = {t}, dl[1] = {dt};
    launch_levels_step_slots(d_slots, n, 0, 1, tl, dl, cfl_slot);
}

// The launch arguments every step form shares: arenas, method, time step,
// swirl velocity scale, physical parameters, CFL slot.
void Context::fill_step_args(StepArgs& a, double t, double dt, unsigned long long* cfl_slot) const {
    a.q = d_q_;
    a.qlast = d_qlast_;
    a.aux = aux_kind_ == AUX_STORED ? d_aux_ : nullptr;
    a.meta = d_meta_;
    a.q_stride = stride_;
    a.aux_stride = aux_stride_;
    a.maux = aux_kind_ == AUX_STORED ? opt_.maux : 0;
    a.order0 = opt_.order[0];
    a.order1 = opt_.order[1];
    for (int k = 0; k < 8; ++k) a.mthlim[k] = opt_.mthlim[k];
    a.dt = dt;
    if (aux_kind_ == AUX_SWIRL) {
        // swirl b4step2.f: vt = cos(pi2*(time+dt/2)/tperiod), pi2 = 2*(4*atan(1))
        const double pi = 4.0 * std::atan(1.0);
        const double pi2 = 2.0 * pi;
        const double tperiod = opt_.problem_params[0];
        a.vt = (tperiod == 0.0) ? 0.0 : std::cos(pi2 * (t + dt / 2.0) / tperiod);
    }
    a.grav = opt_.grav;
    a.gamma = opt_.gamma;
    a.gamma1 = opt_.gamma - 1.0;
    a.drytol = opt_.dry_tolerance;
    a.cfl_out = cfl_slot;
    a.treg = time_sync_ ? d_treg_ : nullptr;
    a.treg_stride = treg_stride_;
    a.lvl0 = 0;
    a.nlvl = 1;
}

// One step launch over patches of levels lvl0 .. lvl0 + nlvl - 1 (their slots
// contiguous in d_slots), level l at time t[l - lvl0] with step dt[l - lvl0].
// nlvl > 1 needs the macro-step table (use_dyn_): each level's {dt, vt} pair.
void Context::launch_levels_step_slots(const int32_t* d_slots, int n, int lvl0, int nlvl, const double* tl,
                                       const double* dtl, unsigned long long* cfl_slot) {
    if (n <= 0) return;
    if (nlvl > 1 && !use_dyn_) throw Error(FCB_ERR_INTERNAL, "merged level updates need the step-parameter table");
    const double t = tl[0], dt = dtl[0];
    StepArgs a{};
    fill_step_args(a, t, dt, cfl_slot);
    a.slots = d_slots;
    a.npatches = n;
    a.lvl0 = lvl0;
    a.nlvl = nlvl;
    if (use_dyn_) {
        // {dt, vt} of launch dyn_n_ of the macro step (one pair per level of a
        // merged launch): written to the table by the dry pass, read from the
        // device table by the launch itself
        if (dry_) {
            for (int k = 0; k < nlvl; ++k) {
            if (dyn_n_ >= (int)dyn_cap_) {
                const size_t nc = std::max<size_t>(64, 2 * dyn_cap_);
                double* np = nullptr;
                check(cudaHostAlloc(&np, nc * 2 * sizeof(double), cudaHostAllocDefault), "cudaHostAlloc dyn");
                if (h_dyn_) {
                    std::copy(h_dyn_, h_dyn_ + 2 * dyn_cap_, np);
                    cudaFreeHost(h_dyn_);
                }
                h_dyn_ = np;
                dyn_cap_ = nc;
            }
            double vk = 0.0;
            if (aux_kind_ == AUX_SWIRL) {
                const double pi2 = 2.0 * (4.0 * std::atan(1.0));
                const double tperiod = opt_.problem_params[0];
                vk = (tperiod == 0.0) ? 0.0 : std::cos(pi2 * (tl[k] + dtl[k] / 2.0) / tperiod);
            }
            h_dyn_[2 * dyn_n_] = dtl[k];
            h_dyn_[2 * dyn_n_ + 1] = vk;
            ++dyn_n_;
            }
            return;
        }
        if (!d_dyn_.p || 2 * (size_t)(dyn_n_ + nlvl) > d_dyn_.cap)
            throw Error(FCB_ERR_STATE, "step-parameter table not sized by the dry pass");
        a.dyn = d_dyn_.p + 2 * dyn_n_;
        dyn_n_ += nlvl;
    }
    launch_step_form(a, n);
    if (opt_.src_term > 0) {
        // clawpack46_update: src2 after step2 for every patch of the update
        check(launch_src2(opt_.src_term, a, opt_.mx, opt_.my, opt_.mbc, opt_.meqn, st_), "src2");
        ++cnt_.count_kernel_launches;
    }
}

// The step launch of a level update in the form chosen for it (the autotuner's,
// or step_variant), with the time-sync flux store before it when time-sync is on.
void Context::launch_step_form(const StepArgs& a, int n) {
    // The warp form computes each swirl velocity node once, which equals the
    // reference's per-cell evaluations because the unit-square mesh with mx a
    // power of two is dyadic (xll + dx == next xll exactly); checked at creation.
    cudaError_t e = cudaErrorNotSupported;
    if (time_sync_) {
        // clawpack46_time_sync_store_flux: f(q) at the patch faces before the update
        check(launch_ts_store_flux(a, opt_.mx, opt_.my, opt_.mbc, opt_.meqn, st_), "time-sync store flux");
        ++cnt_.count_kernel_launches;
    }
    // the tuner's choice is form + 8 * (row bands - 1): the four-barrier form
    // may split every patch's rows into bands of separate CTAs
    const int code = opt_.step_variant == 0      ? tune_step_form(a, n)
                     : opt_.step_variant >= 4      ? 1 + 8 * (opt_.step_variant - 3)
                                                   : opt_.step_variant;
    const int v = code % 8, nb = code / 8 + 1;
    step_form_used_ = v;
    bands_used_ = nb;
    if (nb > 1) {
        // the bands of a patch read rows beyond their own: they read a copy of
        // the arena taken before the launch and update q in place
        if (!d_qalt_) arena_alloc(d_qalt_, (size_t)capacity_ * stride_ * sizeof(double));
        check(cudaMemcpyAsync(d_qalt_, a.q, (size_t)capacity_ * stride_ * sizeof(double), cudaMemcpyDeviceToDevice,
                              st_),
              "band source copy");
        StepArgs b = a;
        b.qsrc = d_qalt_;
        b.nbands = nb;
        check(launch_step(opt_.solver_kind, aux_kind_, opt_.mwaves, opt_.mx, opt_.my, opt_.mbc, b, st_,
                          opt_.claw_version),
              "step");
        cnt_.count_single_step += n;
        ++cnt_.count_kernel_launches;
        return;
    }
    if (opt_.precision == 1) {
        e = launch_step_pipe_mixed(opt_.solver_kind, aux_kind_, opt_.mwaves, opt_.mx, opt_.my, opt_.mbc,
                                   opt_.claw_version, a, st_);
        if (e == cudaErrorNotSupported) throw Error(FCB_ERR_INVALID, "no mixed-precision step for this case");
    } else if (v == 2) {
        if (aux_kind_ == AUX_SWIRL) e = launch_step_warp_swirl(opt_.mx, opt_.mbc, a, st_);
        if (e == cudaErrorNotSupported) throw Error(FCB_ERR_INVALID, "no warp-synchronous step for this case");
    } else if (v == 3) {
        // default: the pipelined form for scalar advection; the Roe solvers keep
        // the four-barrier form, whose smaller register footprint suits them
        e = launch_step_pipe(opt_.solver_kind, aux_kind_, opt_.mwaves, opt_.mx, opt_.my, opt_.mbc, opt_.claw_version,
                             a, st_);
        if (e == cudaErrorNotSupported && v == 3) throw Error(FCB_ERR_INVALID, "no pipelined step for this case");
    }
    if (e == cudaErrorNotSupported) {
        StepArgs b = a;
        if ((opt_.solver_kind == FCB_SOLVER_SWE_ROE || opt_.solver_kind == FCB_SOLVER_EULER4_ROE) && !a.treg &&
            !a.desc) {
            // the launcher may split the last, partial wave into row bands,
            // reading those patches from a copy in the scratch arena
            if (!d_qalt_) arena_alloc(d_qalt_, (size_t)capacity_ * stride_ * sizeof(double));
            b.qtail = d_qalt_;
        }
        e = launch_step(opt_.solver_kind, aux_kind_, opt_.mwaves, opt_.mx, opt_.my, opt_.mbc, b, st_,
                        opt_.claw_version);
    }
    check(e, "step");
    cnt_.count_single_step += n;
    ++cnt_.count_kernel_launches;
}

double Context::launch_level_step(int level, double t, double dt, unsigned long long* cfl_slot) {
    if (level < 0 || level > QuadForest::kMaxLevel) return 0.0;
    const int b = level_begin_[level], e = level_begin_[level + 1];
    launch_level_step_slots(d_level_slots_.p + b, e - b, t, dt, cfl_slot);
    return 0.0;
}

double Context::update_single_step(int level, double t, double dt) {
    if (!initialized_) throw Error(FCB_ERR_STATE, "update_single_step before initialize");
    ensure_ghosts();
    ghosts_filled_ = false;  // the step updates ghost cells; no ghost update follows
    check(cudaMemsetAsync(d_cfl_ + 1, 0, sizeof(unsigned long long), st_), "memset");
    launch_level_step(level, t, dt, d_cfl_ + 1);
    return read_cfl(d_cfl_ + 1);
}

void Context::update_single_step_async(int level, double t, double dt) {
    if (!initialized_) throw Error(FCB_ERR_STATE, "update_single_step before initialize");
    ensure_ghosts();
    ghosts_filled_ = false;
    launch_level_step(level, t, dt, d_cfl_);
}

double Context::single_step_update(int patchno, double t, double dt, int iter, int total) {
    if (!initialized_) throw Error(FCB_ERR_STATE, "single_step_update before initialize");
    if (patchno < 0 || patchno >= num_patches()) throw Error(FCB_ERR_INVALID, "bad patch number");
    if (!owned(patchno)) throw Error(FCB_ERR_INVALID, "patch not owned by this rank");
    ensure_ghosts();
    ghosts_filled_ = false;
    if (iter == 0) pending_.clear();
    pending_.push_back(slot_of_[patchno]);
    if (iter + 1 < total) return 0.0;
    d_pending_.reserve(pending_.size());
    check(cudaMemcpyAsync(d_pending_.p, pending_.data(), pending_.size() * 4, cudaMemcpyHostToDevice, st_), "pending");
    check(cudaMemsetAsync(d_cfl_ + 1, 0, sizeof(unsigned long long), st_), "memset");
    launch_level_step_slots(d_pending_.p, (int)pending_.size(), t, dt, d_cfl_ + 1);
    pending_.clear();
    return read_cfl(d_cfl_ + 1);
}

void Context::timeinterp(int level, double alpha) {
    if (dry_ || level < 0 || level > QuadForest::kMaxLevel) return;
    ensure_ghosts();
    const int b = ti_begin_[level], e = ti_begin_[level + 1];
    if (e == b) return;
    check(launch_timeinterp(d_q_, d_qlast_, d_qti_, stride_, d_ti_slots_.p + b, e - b, opt_.mx, opt_.my, opt_.mbc,
                            opt_.meqn, alpha, st_),
          "timeinterp");
    ++cnt_.count_kernel_launches;
}

// fclaw2d_advance_all_levels (src/fclaw2d_advance.c:247-357)
void Context::run_schedule(double t_curr, double dt) {
    const int gmin = gmin_, gmax = gmax_;
    struct Counter { int last_step, step_inc, total_steps; double current_time, dt_step; };
    std::vector<Counter> ts(opt_.maxlevel + 1);
    for (int l = opt_.minlevel; l <= opt_.maxlevel; ++l) { ts[l].last_step = 0; ts[l].current_time = t_curr; }
    if (opt_.subcycle) {
        double dt_level = dt;
        int steps_inc = 1 << (gmax - opt_.minlevel);
        int total_steps = 1;
        for (int l = opt_.minlevel; l <= opt_.maxlevel; ++l) {
            ts[l].dt_step = dt_level; ts[l].total_steps = total_steps; ts[l].step_inc = steps_inc;
            dt_level /= 2; steps_inc /= 2; total_steps *= 2;
        }
    } else {
        const int rf = 1 << (opt_.maxlevel - opt_.minlevel);
        for (int l = opt_.minlevel; l <= opt_.maxlevel; ++l) {
            ts[l].step_inc = 1; ts[l].dt_step = dt / rf; ts[l].total_steps = rf;
        }
    }
    if (!dry_) check(cudaMemsetAsync(d_cfl_, 0, sizeof(unsigned long long), st_), "memset");
    // With the step-parameter table the level updates between two ghost
    // updates (levels gmax down to some l, contiguous in the level-sorted slot
    // list) go out as one launch: they touch disjoint patches, the CFL is a
    // max, and each patch reads its own level's {dt, vt}.  Time interpolation,
    // ghost updates and time-sync flush the queued levels first.
    const bool merge = use_dyn_ && !time_sync_;
    int q_lo = -1, q_hi = -1;
    std::vector<double> q_t((size_t)QuadForest::kMaxLevel + 2), q_dt((size_t)QuadForest::kMaxLevel + 2);
    auto flush = [&]() {
        if (q_hi < 0) return;
        const int b = level_begin_[q_lo], e = level_begin_[q_hi + 1];
        launch_levels_step_slots(d_level_slots_.p + b, e - b, q_lo, q_hi - q_lo + 1, q_t.data() + q_lo,
                                 q_dt.data() + q_lo, d_cfl_);
        q_lo = q_hi = -1;
    };
    auto step_level = [&](int level, double t, double dts) {
        if (!merge || level < 0 || level > QuadForest::kMaxLevel) {
            launch_level_step(level, t, dts, d_cfl_);
            return;
        }
        if (q_hi >= 0 && level != q_lo - 1) flush();  // keep the queued levels contiguous
        if (q_hi < 0) q_hi = level;
        q_lo = level;
        q_t[level] = t;
        q_dt[level] = dts;
    };
    std::function<void(int, int)> advance_level = [&](int level, int curr_fine_step) {
        step_level(level, ts[level].current_time, ts[level].dt_step);
        ts[level].last_step += ts[level].step_inc;
        ts[level].current_time += ts[level].dt_step;
        if (level > gmin) {
            const int last_coarse_step = ts[level - 1].last_step;
            if (last_coarse_step == curr_fine_step) {
                advance_level(level - 1, last_coarse_step);
                if (opt_.subcycle) {
                    const int coarse_inc = ts[level - 1].step_inc;
                    const double alpha = ((double)(ts[level].last_step % coarse_inc)) / coarse_inc;
                    flush();
                    timeinterp(level - 1, alpha);
                }
            }
        }
    };
    const int n_fine = ts[gmax].total_steps;
    for (int nf = 0; nf < n_fine; ++nf) {
        advance_level(gmax, nf);
        flush();
        const int last_step = ts[gmax].last_step;
        if (last_step < ts[gmax].total_steps) {
            const double sync_time = ts[gmax].current_time;
            if (opt_.subcycle) {
                int ti_level = gmax - 1;
                while (last_step % ts[ti_level].step_inc == 0) --ti_level;
                ghost_update(ti_level + 1, gmax, sync_time, 1);
                if (time_sync_) time_sync(ti_level + 1);  // fclaw2d_advance.c:298-303
            } else {
                ghost_update(gmin, gmax, sync_time, 0);
                if (time_sync_) time_sync(gmin);
            }
        }
    }
    ghost_update(gmin, gmax, ts[gmax].current_time, 0);
    if (time_sync_) time_sync(gmin);  // fclaw2d_advance.c:337-341
}

std::vector<uintptr_t> Context::macro_fingerprint() const {
    return {(uintptr_t)d_q_, (uintptr_t)d_qlast_, (uintptr_t)d_qti_, (uintptr_t)d_meta_,
            (uintptr_t)d_level_slots_.p, (uintptr_t)d_ti_slots_.p, (uintptr_t)d_ops_.p, (uintptr_t)d_groups_.p,
            (uintptr_t)d_dyn_.p, (uintptr_t)d_cfl_, (uintptr_t)mesh_version_, (uintptr_t)plans_.size(),
            (uintptr_t)dyn_n_, (uintptr_t)gmin_, (uintptr_t)gmax_, (uintptr_t)d_treg_,
            (uintptr_t)d_ts_ops_.p, (uintptr_t)d_ts_groups_.p, (uintptr_t)ts_plans_.size(), (uintptr_t)d_qalt_};
}

void Context::drop_macro_graph() {
    if (macro_exec_) cudaGraphExecDestroy(macro_exec_);
    macro_exec_ = nullptr;
    macro_key_.clear();
    macro_seen_.clear();
}

// fclaw2d_advance_all_levels (src/fclaw2d_advance.c:247-346).  With
// macro_graph on, the first call on a mesh runs eagerly (building and uploading
// the ghost plans), the second captures the schedule into a CUDA graph, and
// later calls replay it; every call first runs the schedule "dry" on the host
// to fill the {dt, vt} table that the step launches read.
double Context::advance_all_levels(double t_curr, double dt) {
    advance_enqueue(t_curr, dt);
    return read_cfl(d_cfl_);
}

namespace {
// acc = max(acc, v) on the bits of non-negative doubles (a NaN wins)
__global__ void cfl_merge_kernel(unsigned long long* acc, const unsigned long long* v) { atomicMax(acc, *v); }
}  // namespace

// The macro step without the wait for its CFL number: the number is folded
// into a running maximum on the device, which read_max_cfl returns.
void Context::advance_all_levels_async(double t_curr, double dt) {
    advance_enqueue(t_curr, dt);
    cfl_merge_kernel<<<1, 1, 0, st_>>>(d_cfl_ + 4, d_cfl_);
    check(cudaGetLastError(), "cfl merge");
    ++cnt_.count_kernel_launches;
}

double Context::read_max_cfl() {
    if (!d_cfl_) throw Error(FCB_ERR_STATE, "read_max_cfl before initialize");
    check(cudaMemcpyAsync(h_cfl_, d_cfl_ + 4, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st_), "cfl");
    check(cudaMemsetAsync(d_cfl_ + 4, 0, sizeof(unsigned long long), st_), "memset");
    synchronize();
    const double c = cfl_from_bits(*h_cfl_);
    if (std::isnan(c)) throw Error(FCB_ERR_NUMERIC, "NaN CFL in an asynchronous macro step");
    return c;
}

void Context::advance_enqueue(double t_curr, double dt) {
    if (!initialized_) throw Error(FCB_ERR_STATE, "advance before initialize");
    fused_used_ = 0;
    if (use_fusion(t_curr, dt)) {
        advance_fused(t_curr, dt);
        return;
    }
    ensure_ghosts();
    // on an error, plan builds still running are joined and dropped
    struct PlanGuard {
        Context* c;
        bool armed = true;
        ~PlanGuard() {
            if (armed) c->discard_plans();
        }
    } plans_guard{this};
    use_dyn_ = opt_.macro_graph != 0;
    if (use_dyn_) {
        dyn_n_ = 0;
        dry_ = true;
        dry_plan_keys_.clear();
        try {
            run_schedule(t_curr, dt);
        } catch (...) {
            dry_ = false;
            throw;
        }
        dry_ = false;
        // the ghost plans of this macro step that do not exist yet (after a
        // regrid, none) are built on host threads while the first level
        // updates run
        start_plans(dry_plan_keys_);
        // auto: the graph, whenever the macro step has a level update (a replay
        // beats host launches even for the three launches of one level)
        if (opt_.macro_graph == 2 && dyn_n_ < 1) use_dyn_ = false;
    }
    if (use_dyn_) {
        d_dyn_.reserve(std::max<size_t>(2, 2 * (size_t)dyn_n_));
        if (dyn_n_ > 0)
            check(cudaMemcpyAsync(d_dyn_.p, h_dyn_, 2 * (size_t)dyn_n_ * sizeof(double), cudaMemcpyHostToDevice, st_),
                  "step parameters");
        const int n_launch = dyn_n_;
        std::vector<uintptr_t> key = macro_fingerprint();
        if (macro_exec_ && key == macro_key_) {
            check(cudaGraphLaunch(macro_exec_, st_), "cudaGraphLaunch");
            ++cnt_.count_graph_replays;
            cnt_.count_single_step += macro_delta_.count_single_step;
            cnt_.count_kernel_launches += macro_delta_.count_kernel_launches;
            cnt_.count_ghost_waves += macro_delta_.count_ghost_waves;
        } else if (key == macro_seen_ && !ops_dirty_) {
            drop_macro_graph();
            const fcb_counters_t c0 = cnt_;
            dyn_n_ = 0;
            cudaGraph_t graph = nullptr;
            // capture on a private stream: the work is only recorded there, and the
            // graph is launched on the caller's stream (which may be the legacy
            // default stream, which cannot be captured)
            if (!cap_st_) check(cudaStreamCreateWithFlags(&cap_st_, cudaStreamNonBlocking), "cudaStreamCreate");
            const cudaStream_t user_st = st_;
            st_ = cap_st_;
            cudaError_t be = cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal);
            if (be != cudaSuccess) {
                st_ = user_st;
                check(be, "cudaStreamBeginCapture");
            }
            try {
                run_schedule(t_curr, dt);
            } catch (...) {
                cudaStreamEndCapture(st_, &graph);
                if (graph) cudaGraphDestroy(graph);
                st_ = user_st;
                use_dyn_ = false;
                throw;
            }
            cudaError_t ee = cudaStreamEndCapture(st_, &graph);
            st_ = user_st;
            check(ee, "cudaStreamEndCapture");
            cudaError_t e = cudaGraphInstantiate(&macro_exec_, graph, 0);
            cudaGraphDestroy(graph);
            check(e, "cudaGraphInstantiate");
            if (dyn_n_ != n_launch) throw Error(FCB_ERR_STATE, "macro-step schedule changed during capture");
            macro_key_ = key;
            macro_delta_.count_single_step = cnt_.count_single_step - c0.count_single_step;
            macro_delta_.count_kernel_launches = cnt_.count_kernel_launches - c0.count_kernel_launches;
            macro_delta_.count_ghost_waves = cnt_.count_ghost_waves - c0.count_ghost_waves;
            check(cudaGraphLaunch(macro_exec_, st_), "cudaGraphLaunch");
        } else {
            dyn_n_ = 0;
            run_schedule(t_curr, dt);
            macro_seen_ = macro_fingerprint();
        }
    } else {
        run_schedule(t_curr, dt);
    }
    use_dyn_ = false;
    finish_plans();
    plans_guard.armed = false;
    ++cnt_.count_amr_advance;
    ghosts_filled_ = true;  // the macro step ends with a ghost update of every level
}

// ---------------------------------------------------------------------------
// Autotuner.  For step_variant 0 the library times the step forms that exist
// for a (solver, aux, waves, mx, clawpack version, precision, limiter, size)
// key on the first level update of that key, and the ghost-fill unroll on the first
// ghost update of a patch shape, both on scratch copies of the arrays (the
// real state is not touched).  Choices are cached for the process.  Never runs while a
// macro-step graph is captured (the first call on a mesh is eager).
// ---------------------------------------------------------------------------
namespace {
std::mutex g_tune_mu;
std::map<std::vector<int>, int> g_step_form_cache, g_ghost_unroll_cache;

int default_step_form(const fcb_options_t& o) {
    if (o.solver_kind == SOLVER_ADVECTION_MANIFOLD) return 1;  // capacity: four-barrier form only
    return (o.solver_kind == SOLVER_ADVECTION || o.claw_version == 5 || o.solver_kind == SOLVER_GEOCLAW_FWAVE ||
            o.precision == 1)
               ? 3
               : 1;
}
}  // namespace

int Context::tune_step_form(const StepArgs& a, int n) {
    const bool fixed_lim = opt_.order[0] == 2 && opt_.order[1] == 2;
    int nb = 0;
    while ((1 << (nb + 1)) <= n) ++nb;
    const std::vector<int> key = {opt_.solver_kind, aux_kind_, opt_.mwaves, opt_.mx, opt_.claw_version, opt_.precision,
                                  fixed_lim ? opt_.mthlim[0] : -1, nb};
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_step_form_cache.find(key);
        if (it != g_step_form_cache.end()) return it->second;
    }
    // codes: form + 8 * (row bands - 1).  The four-barrier form with 2 or 3
    // row bands (step_variant 4, 5) is not a candidate: on B200 it measured
    // +1 % (shallow water) and -12 % (Euler) on the AMR configurations, whose
    // level updates are bound by the SMs' throughput at one 255-register CTA
    // each, not by the length of one CTA's row sweep.
    // The Roe systems of clawpack 4.6 in FP64 run the four-barrier form: since
    // it shares the per-cell quantities of the Riemann problems it measured
    // faster than the pipelined form at every size on B200 (shallow water
    // mx = 32 about 2x, Euler 1.01-1.9x), and a choice between the two made
    // per octave of the patch count could flip on a close race at one size and
    // cost 2x at another (a one-wave four-barrier launch against a two-wave
    // pipelined one), so the pipelined form is not tried for them.
    std::vector<int> cand;
    if (opt_.solver_kind == SOLVER_ADVECTION_MANIFOLD) cand = {1};  // capacity: four-barrier form only
    else if (opt_.precision == 1 || opt_.claw_version == 5 || opt_.solver_kind == SOLVER_GEOCLAW_FWAVE) cand = {3};
    else if (aux_kind_ == AUX_SWIRL) cand = {1, 2, 3};
    else if (opt_.solver_kind == SOLVER_SWE_ROE || opt_.solver_kind == SOLVER_EULER4_ROE ||
             opt_.solver_kind == SOLVER_ADVECTION_MANIFOLD)
        cand = {1};
    else cand = {1, 3};
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st_, &cs);
    if (cand.size() == 1 || cs != cudaStreamCaptureStatusNone || dry_) return cand.size() == 1 ? cand[0] : default_step_form(opt_);
    const size_t bytes = (size_t)capacity_ * stride_ * sizeof(double);
    double *tq = nullptr, *tl = nullptr, *ts = nullptr;
    try {
        arena_alloc(tq, bytes);
        arena_alloc(tl, bytes);
        arena_alloc(ts, bytes);
    } catch (const Error&) {
        cudaGetLastError();
        arena_free(tq);
        arena_free(tl);
        arena_free(ts);
        return default_step_form(opt_);  // no room for scratch copies: no tuning
    }
    check(cudaMemcpyAsync(tq, d_q_, bytes, cudaMemcpyDeviceToDevice, st_), "tune copy");
    StepArgs b = a;
    b.q = tq;
    b.qlast = tl;
    b.dyn = nullptr;
    b.cfl_out = d_cfl_ + 3;
    b.treg = nullptr;  // the trial steps leave the time-sync registers alone
    cudaEvent_t e0, e1;
    check(cudaEventCreate(&e0), "event");
    check(cudaEventCreate(&e1), "event");
    int best = default_step_form(opt_);
    float best_ms = 1e30f;
    // two rounds over the candidates, each candidate's best round counts: a
    // single timing per form was seen to pick a form ~7 % slower in steady state
    std::vector<float> best_of(cand.size(), 1e30f);
    std::vector<char> ok(cand.size(), 1);
    for (int round = 0; round < 2; ++round)
    for (size_t ci = 0; ci < cand.size(); ++ci) {
        if (!ok[ci]) continue;
        const int code = cand[ci];
        const int v = code % 8, nb = code / 8 + 1;
        auto launch = [&]() -> cudaError_t {
            if (v == 2) return launch_step_warp_swirl(opt_.mx, opt_.mbc, b, st_);
            if (v == 3)
                return launch_step_pipe(opt_.solver_kind, aux_kind_, opt_.mwaves, opt_.mx, opt_.my, opt_.mbc,
                                        opt_.claw_version, b, st_);
            if (nb > 1) {
                cudaError_t ce = cudaMemcpyAsync(ts, tq, bytes, cudaMemcpyDeviceToDevice, st_);
                if (ce != cudaSuccess) return ce;
                StepArgs bb = b;
                bb.qsrc = ts;
                bb.nbands = nb;
                return launch_step(opt_.solver_kind, aux_kind_, opt_.mwaves, opt_.mx, opt_.my, opt_.mbc, bb, st_,
                                   opt_.claw_version);
            }
            return launch_step(opt_.solver_kind, aux_kind_, opt_.mwaves, opt_.mx, opt_.my, opt_.mbc, b, st_,
                               opt_.claw_version);
        };
        if (launch() != cudaSuccess) {  // form not available for this case
            cudaGetLastError();
            ok[ci] = 0;
            continue;
        }
        check(cudaEventRecord(e0, st_), "event");
        for (int r = 0; r < 3; ++r) check(launch(), "tune launch");
        check(cudaEventRecord(e1, st_), "event");
        check(cudaEventSynchronize(e1), "event");
        float ms = 0;
        check(cudaEventElapsedTime(&ms, e0, e1), "event");
        best_of[ci] = std::min(best_of[ci], ms);
    }
    for (size_t ci = 0; ci < cand.size(); ++ci)
        if (ok[ci] && best_of[ci] < best_ms) { best_ms = best_of[ci]; best = cand[ci]; }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    arena_free(tq);
    arena_free(tl);
    arena_free(ts);
    check(cudaStreamSynchronize(st_), "sync");
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_step_form_cache[key] = best;
    return best;
}

int Context::tune_ghost_unroll(const GhostPlan& g) {
    const std::vector<int> key = {opt_.mx, opt_.meqn, opt_.precision};
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_ghost_unroll_cache.find(key);
        if (it != g_ghost_unroll_cache.end()) return it->second;
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st_, &cs);
    if (cs != cudaStreamCaptureStatusNone || g.wave_begin.size() < 2) return 4;
    // scratch copies of the arena and the time-interpolation arena, so the
    // timed passes leave the real state untouched
    const size_t bytes = (size_t)capacity_ * stride_ * sizeof(double);
    double *tq = nullptr, *tt = nullptr;
    try {
        arena_alloc(tq, bytes);
        arena_alloc(tt, bytes);
    } catch (const Error&) {
        cudaGetLastError();
        arena_free(tq);
        arena_free(tt);
        return 4;
    }
    check(cudaMemcpyAsync(tq, d_q_, bytes, cudaMemcpyDeviceToDevice, st_), "tune copy");
    if (d_qti_) check(cudaMemcpyAsync(tt, d_qti_, bytes, cudaMemcpyDeviceToDevice, st_), "tune copy");
    cudaEvent_t e0, e1;
    check(cudaEventCreate(&e0), "event");
    check(cudaEventCreate(&e1), "event");
    int best = 4;
    float best_ms = 1e30f;
    const int nw = (int)g.wave_begin.size() - 1;
    for (int u : {2, 4, 8}) {
        auto pass = [&]() {
            for (int w = 0; w < nw; ++w) {
                GhostArgs ga;
                ga.q = tq; ga.qti = tt; ga.stride = stride_;
                ga.mx = opt_.mx; ga.my = opt_.my; ga.mbc = opt_.mbc; ga.meqn = opt_.meqn;
                ga.ops = d_ops_.p;
                ga.groups = d_groups_.p + g.first_group + g.group_begin[w];
                ga.ngroups = g.group_begin[w + 1] - g.group_begin[w] - 1;
                ga.interp_fp32 = opt_.precision == 1;
                check(launch_ghost_wave(ga, st_, u), "tune ghost");
            }
        };
        pass();
        check(cudaEventRecord(e0, st_), "event");
        for (int r = 0; r < 3; ++r) pass();
        check(cudaEventRecord(e1, st_), "event");
        check(cudaEventSynchronize(e1), "event");
        float ms = 0;
        check(cudaEventElapsedTime(&ms, e0, e1), "event");
        if (ms < best_ms) { best_ms = ms; best = u; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    arena_free(tq);
    arena_free(tt);
    check(cudaStreamSynchronize(st_), "sync");
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_ghost_unroll_cache[key] = best;
    return best;
}

// ---------------------------------------------------------------------------
// Batched serving support
// ---------------------------------------------------------------------------
// Non-subcycled fclaw2d_advance_all_levels (src/fclaw2d_advance.c:300-324): each
// of the 2^(maxlevel-minlevel) fine steps updates every level with the fine dt
// and is followed by a ghost fill over all levels, so a fine step is one batch
// of all leaves.
// ---------------------------------------------------------------------------
// Ghost-exchange fusion on a mesh of one level.
//
// On such a mesh every macro step is n_fine level updates, each followed by a
// ghost update whose records are same-size copies and physical boundary
// conditions only (fclaw2d_advance.c:285-341 with one level).  The fused step
// reads each patch's ghost cells from its neighbours' interiors through a
// per-slot table (the values those records would write), reads from one arena
// and writes the updated interiors into the other, so no patch reads a
// neighbour that the same launch has already updated.  The ghost cells the
// reference's step would also update are dead: the following ghost update
// overwrites every one of them.  The last ghost update of the macro step is
// recorded and run by ensure_ghosts() before anything reads ghost cells, so
// every array a caller sees equals the unfused result bit for bit.
// ---------------------------------------------------------------------------
void Context::build_fuse_table() {
    fuse_ok_ = false;
    if (partitioned() || gmin_ != gmax_ || own_count_ <= 0 || capacity_ <= 0) return;
    std::vector<FuseNbr> t((size_t)capacity_);
    for (auto& f : t) {
        for (int k = 0; k < 4; ++k) f.face[k] = f.corner[k] = -1;
        for (int k = 0; k < 4; ++k) f.bc[k] = 0;
    }
    for (int p = 0; p < num_patches(); ++p) {
        const Neighbors& nb = nbrs_[p];
        FuseNbr f;
        for (int k = 0; k < 4; ++k) {
            f.bc[k] = 0;
            f.face[k] = f.corner[k] = -1;
            if (nb.face_rel[k] == REL_BOUNDARY) f.bc[k] = opt_.mthbc[k];
            else if (nb.face_rel[k] == REL_SAMESIZE) f.face[k] = slot_of_[nb.face_nbr[k][0]];
            else return;  // a coarse/fine face: not a mesh of one level
            if (nb.corner_rel[k] == REL_SAMESIZE) f.corner[k] = slot_of_[nb.corner_nbr[k]];
        }
        // a corner block is copied from the corner neighbour unless one of its
        // two faces is a physical boundary; that neighbour must exist
        for (int c = 0; c < 4; ++c) {
            const int fx = (c & 1) ? 1 : 0, fy = (c & 2) ? 3 : 2;
            if (f.bc[fx] == 0 && f.bc[fy] == 0 && f.corner[c] < 0) return;
        }
        t[slot_of_[p]] = f;
    }
    d_fuse_.reserve((size_t)capacity_);
    check(cudaMemcpy(d_fuse_.p, t.data(), t.size() * sizeof(FuseNbr), cudaMemcpyHostToDevice), "fuse table");
    fuse_ok_ = true;
}

bool Context::fusion_possible() const {
    // the fused step reads the neighbours' interiors where the unfused one
    // reads its own ghost cells: equal only when those hold a ghost update's values
    return opt_.ghost_fusion != 1 && fuse_ok_ && ghosts_filled_ && !partitioned() && !time_sync_ && !dry_ &&
           opt_.src_term == 0 &&
           gmin_ == gmax_ &&
           own_count_ > 0 && (opt_.step_variant == 0 || opt_.step_variant == 3) && opt_.mbc == 2 &&
           (opt_.mx == 8 || opt_.mx == 16 || opt_.mx == 32);
}

namespace {
std::map<std::vector<int>, int> g_fusion_cache;
}  // namespace

bool Context::use_fusion(double t, double dt) {
    if (!fusion_possible()) return false;
    if (opt_.ghost_fusion == 2) return true;
    // autotuner axis: the fused step against the best unfused form plus the
    // ghost fill, on scratch copies, once per key for the process
    const bool fixed_lim = opt_.order[0] == 2 && opt_.order[1] == 2;
    int nb = 0;
    while ((1 << (nb + 1)) <= own_count_) ++nb;
    const std::vector<int> key = {opt_.solver_kind, aux_kind_, opt_.mwaves, opt_.mx, opt_.claw_version, opt_.precision,
                                  fixed_lim ? opt_.mthlim[0] : -1, nb};
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_fusion_cache.find(key);
        if (it != g_fusion_cache.end()) return it->second != 0;
    }
    int choice = 1;
    try {
        const double tf = time_steps(true, false, 3, t, dt);
        const double tu = time_steps(false, true, 3, t, dt);
        choice = tf < tu ? 1 : 0;
    } catch (const Error&) {
        cudaGetLastError();
        choice = 1;  // no room for the scratch copies: fuse (no extra arena beyond the second one)
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_fusion_cache[key] = choice;
    return choice != 0;
}

void Context::launch_fused_step(double t, double dt, const double* src, double* dst, unsigned long long* cfl_slot) {
    const int b = level_begin_[gmax_], e = level_begin_[gmax_ + 1];
    StepArgs a{};
    fill_step_args(a, t, dt, cfl_slot);
    a.q = dst;
    a.qsrc = src;
    a.fuse = d_fuse_.p;
    a.slots = d_level_slots_.p + b;
    a.npatches = e - b;
    cudaError_t r = opt_.precision == 1
                        ? launch_step_pipe_fused_mixed(opt_.solver_kind, aux_kind_, opt_.mwaves, opt_.mx, opt_.my,
                                                       opt_.mbc, opt_.claw_version, a, st_)
                        : launch_step_pipe_fused(opt_.solver_kind, aux_kind_, opt_.mwaves, opt_.mx, opt_.my,
                                                 opt_.mbc, opt_.claw_version, a, st_);
    check(r, "fused step");
    cnt_.count_single_step += e - b;
    ++cnt_.count_kernel_launches;
}

// fclaw2d_advance_all_levels on a mesh of one level l: n_fine updates of l
// (subcycled: 2^(l - minlevel) steps of dt halved per level; otherwise
// 2^(maxlevel - minlevel) steps of dt/rf), each followed by a ghost update.
void Context::advance_fused(double t_curr, double dt) {
    int n_fine;
    double dt_fine = dt;
    if (opt_.subcycle) {
        for (int l = opt_.minlevel; l < gmax_; ++l) dt_fine /= 2;
        n_fine = 1 << (gmax_ - opt_.minlevel);
    } else {
        const int rf = 1 << (opt_.maxlevel - opt_.minlevel);
        n_fine = rf;
        dt_fine = dt / rf;
    }
    if (!d_qalt_) arena_alloc(d_qalt_, (size_t)capacity_ * stride_ * sizeof(double));
    check(cudaMemsetAsync(d_cfl_, 0, sizeof(unsigned long long), st_), "memset");
    double tk = t_curr;
    for (int k = 0; k < n_fine; ++k) {
        launch_fused_step(tk, dt_fine, d_q_, d_qalt_, d_cfl_);
        std::swap(d_q_, d_qalt_);
        tk += dt_fine;
    }
    ghosts_stale_ = true;
    stale_min_ = gmin_;
    stale_max_ = gmax_;
    stale_t_ = tk;
    fused_used_ = 1;
    step_form_used_ = 3;
    ++cnt_.count_amr_advance;
}

void Context::ensure_ghosts() {
    if (!ghosts_stale_ || dry_) return;
    ghosts_stale_ = false;
    run_plan(plan(stale_min_, stale_max_, 0));
}

double Context::time_steps(bool fused, bool with_fill, int launches, double t, double dt) {
    const size_t bytes = (size_t)capacity_ * stride_ * sizeof(double);
    double *s0 = nullptr, *s1 = nullptr;
    try {
        arena_alloc(s0, bytes);
        arena_alloc(s1, bytes);
    } catch (...) {
        arena_free(s0);
        arena_free(s1);
        throw;
    }
    const fcb_counters_t cnt0 = cnt_;
    const int form0 = step_form_used_;
    double* const q_real = d_q_;
    check(cudaMemcpyAsync(s0, d_q_, bytes, cudaMemcpyDeviceToDevice, st_), "timing copy");
    check(cudaMemcpyAsync(s1, d_q_, bytes, cudaMemcpyDeviceToDevice, st_), "timing copy");
    const int b = level_begin_[gmax_], e = level_begin_[gmax_ + 1];
    int parity = 0;
    auto one = [&]() {
        if (fused) {
            launch_fused_step(t, dt, parity ? s1 : s0, parity ? s0 : s1, d_cfl_ + 3);
            parity ^= 1;
        } else {
            StepArgs a{};
            fill_step_args(a, t, dt, d_cfl_ + 3);
            a.q = s0;
            a.qlast = s1;
            a.slots = d_level_slots_.p + b;
            a.npatches = e - b;
            launch_step_form(a, e - b);
            if (with_fill) {
                d_q_ = s0;  // the ghost fill of the scratch copy (run_plan reads d_q_)
                try {
                    run_plan(plan(gmax_, gmax_, 0));
                } catch (...) {
                    d_q_ = q_real;
                    throw;
                }
                d_q_ = q_real;
            }
        }
    };
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    double ms_per = 0.0;
    try {
        one();  // warm-up: plans, tuned forms, first-launch setup
        check(cudaEventCreate(&e0), "event");
        check(cudaEventCreate(&e1), "event");
        check(cudaEventRecord(e0, st_), "event");
        for (int k = 0; k < launches; ++k) one();
        check(cudaEventRecord(e1, st_), "event");
        check(cudaEventSynchronize(e1), "event");
        float ms = 0.0f;
        check(cudaEventElapsedTime(&ms, e0, e1), "event");
        ms_per = ms / launches;
    } catch (...) {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        arena_free(s0);
        arena_free(s1);
        cnt_ = cnt0;
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    arena_free(s0);
    arena_free(s1);
    check(cudaStreamSynchronize(st_), "sync");
    cnt_ = cnt0;  // timing launches are not the solve's
    step_form_used_ = form0;
    return ms_per;
}

double Context::step_kernel_time(double t, double dt, int launches, bool* fused) {
    if (!initialized_) throw Error(FCB_ERR_STATE, "step_kernel_time before initialize");
    if (launches < 1) throw Error(FCB_ERR_INVALID, "launches must be >= 1");
    ensure_ghosts();  // the unfused step reads the scratch copy's ghost cells
    const bool f = use_fusion(t, dt);
    *fused = f;
    return time_steps(f, false, launches, t, dt);
}

// The schedule of run_schedule (fclaw2d_advance.c:247-346) one fine step at a
// time: the same counters, the same recursion over coarser levels whose step
// falls on this fine step, the same time interpolations and ghost updates.
int Context::serve_begin(double t_curr, double dt) {
    if (!initialized_) throw Error(FCB_ERR_STATE, "step before initialize");
    if (partitioned()) throw Error(FCB_ERR_INVALID, "served solves are not partitioned");
    sv_ts_.assign(opt_.maxlevel + 1, SchedCounter{});
    for (int l = opt_.minlevel; l <= opt_.maxlevel; ++l) sv_ts_[l].current_time = t_curr;
    if (opt_.subcycle) {
        double dt_level = dt;
        int steps_inc = 1 << (gmax_ - opt_.minlevel);
        int total_steps = 1;
        for (int l = opt_.minlevel; l <= opt_.maxlevel; ++l) {
            sv_ts_[l].dt_step = dt_level; sv_ts_[l].total_steps = total_steps; sv_ts_[l].step_inc = steps_inc;
            dt_level /= 2; steps_inc /= 2; total_steps *= 2;
        }
    } else {
        const int rf = 1 << (opt_.maxlevel - opt_.minlevel);
        for (int l = opt_.minlevel; l <= opt_.maxlevel; ++l) {
            sv_ts_[l].step_inc = 1; sv_ts_[l].dt_step = dt / rf; sv_ts_[l].total_steps = rf;
        }
    }
    sv_nf_ = 0;
    sv_steps_.clear();
    sv_ti_.clear();
    return sv_ts_[gmax_].total_steps;
}

long long Context::serve_step_descs(int req, std::vector<PatchDesc>& out) {
    if (!initialized_) throw Error(FCB_ERR_STATE, "step before initialize");
    if (sv_ts_.empty() || sv_nf_ >= sv_ts_[gmax_].total_steps) throw Error(FCB_ERR_STATE, "no fine step left");
    ensure_ghosts();
    ghosts_filled_ = false;
    sv_steps_.clear();
    sv_ti_.clear();
    std::function<void(int, int)> advance_level = [&](int level, int curr_fine_step) {
        SchedCounter& c = sv_ts_[level];
        sv_steps_.push_back({level, c.current_time, c.dt_step});
        c.last_step += c.step_inc;
        c.current_time += c.dt_step;
        if (level > gmin_) {
            const int last_coarse_step = sv_ts_[level - 1].last_step;
            if (last_coarse_step == curr_fine_step) {
                advance_level(level - 1, last_coarse_step);
                if (opt_.subcycle) {
                    const int coarse_inc = sv_ts_[level - 1].step_inc;
                    sv_ti_.emplace_back(level - 1, ((double)(c.last_step % coarse_inc)) / coarse_inc);
                }
            }
        }
    };
    advance_level(gmax_, sv_nf_);
    long long cells = 0;
    const double pi = 4.0 * std::atan(1.0);
    for (const SvStep& u : sv_steps_) {
        double vt = 0.0;
        if (aux_kind_ == AUX_SWIRL) {
            const double tperiod = opt_.problem_params[0];
            vt = (tperiod == 0.0) ? 0.0 : std::cos(2.0 * pi * (u.t + u.dt / 2.0) / tperiod);
        }
        const int b = level_begin_[u.level], e = level_begin_[u.level + 1];
        for (int k = b; k < e; ++k) {
            const int slot = h_level_slots_[k];
            PatchDesc d{};
            d.q = d_q_ + (int64_t)slot * stride_;
            d.qlast = d_qlast_ + (int64_t)slot * stride_;
            d.aux = aux_kind_ == AUX_STORED ? d_aux_ + (int64_t)slot * aux_stride_ : nullptr;
            d.meta = h_meta_[slot];
            d.dt = u.dt;
            d.vt = vt;
            d.req = req;
            out.push_back(d);
        }
        cnt_.count_single_step += e - b;
        cells += (long long)(e - b) * opt_.mx * opt_.my;
    }
    return cells;
}

void Context::serve_after_step() {
    for (const auto& ti : sv_ti_) timeinterp(ti.first, ti.second);
    sv_ti_.clear();
    ++sv_nf_;
    const SchedCounter& top = sv_ts_[gmax_];
    if (top.last_step < top.total_steps) {
        if (opt_.subcycle) {
            int ti_level = gmax_ - 1;
            while (top.last_step % sv_ts_[ti_level].step_inc == 0) --ti_level;
            ghost_update(ti_level + 1, gmax_, top.current_time, 1);
        } else {
            ghost_update(gmin_, gmax_, top.current_time, 0);
        }
    } else {
        ghost_update(gmin_, gmax_, top.current_time, 0);
    }
}

// fclaw2d_clawpatch_save_step / restore_step: the CFL-retry copy
void Context::save_step() {
    if (!d_qsave_) return;
    check(cudaMemcpyAsync(d_qsave_, d_q_, (size_t)capacity_ * stride_ * sizeof(double), cudaMemcpyDeviceToDevice, st_),
          "save_time_step");
}
void Context::restore_step() {
    if (!d_qsave_) return;
    check(cudaMemcpyAsync(d_q_, d_qsave_, (size_t)capacity_ * stride_ * sizeof(double), cudaMemcpyDeviceToDevice, st_),
          "restore_time_step");
}

size_t Context::device_bytes() const {
    const int arenas = 3 + (d_qsave_ ? 1 : 0) + (d_qalt_ ? 1 : 0);
    return (size_t)capacity_ * ((size_t)stride_ * arenas + (size_t)aux_stride_ + (size_t)treg_stride_) * sizeof(double) +
           (size_t)capacity_ * sizeof(PatchMeta) + h_ops_.size() * sizeof(GhostOp);
}

cudaError_t launch_step_batch(const fcb_options_t& opt, int aux_kind, const PatchDesc* d_desc, int n,
                              unsigned long long* d_cfl, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    StepArgs a{};
    a.desc = d_desc;
    a.npatches = n;
    a.maux = aux_kind == AUX_STORED ? opt.maux : 0;
    a.order0 = opt.order[0];
    a.order1 = opt.order[1];
    for (int k = 0; k < 8; ++k) a.mthlim[k] = opt.mthlim[k];
    a.grav = opt.grav;
    a.gamma = opt.gamma;
    a.gamma1 = opt.gamma - 1.0;
    a.drytol = opt.dry_tolerance;
    a.cfl_out = d_cfl;
    // the Roe systems of clawpack 4.6 in FP64 run the four-barrier CTA form (on
    // B200 about twice the pipelined form's rate for shallow water at mx = 32)
    // (capacity exists in that form only, clawpack 4.6 and 5)
    if (opt.solver_kind == FCB_SOLVER_ADVECTION_MANIFOLD)
        return launch_step(opt.solver_kind, aux_kind, opt.mwaves, opt.mx, opt.my, opt.mbc, a, st, opt.claw_version);
    if (opt.precision != 1 && opt.claw_version != 5 &&
        (opt.solver_kind == FCB_SOLVER_SWE_ROE || opt.solver_kind == FCB_SOLVER_EULER4_ROE))
        return launch_step(opt.solver_kind, aux_kind, opt.mwaves, opt.mx, opt.my, opt.mbc, a, st);
    return opt.precision == 1
               ? launch_step_pipe_mixed(opt.solver_kind, aux_kind, opt.mwaves, opt.mx, opt.my, opt.mbc,
                                        opt.claw_version, a, st)
               : launch_step_pipe(opt.solver_kind, aux_kind, opt.mwaves, opt.mx, opt.my, opt.mbc, opt.claw_version,
                                  a, st);
}

// ---------------------------------------------------------------------------
// Regrid
// ---------------------------------------------------------------------------
// Partitioned solves tag their own leaves and gather every rank's values, so
// that every rank adapts the whole forest identically.
void Context::tag(bool domain_init, std::vector<int>& target) {
    const int n = num_patches();
    const size_t need = (size_t)4 * n + (partitioned() ? (size_t)4 * own_count_ : 0);
    if (need > scratch_cap_) {
        if (d_scratch_) {
            check(cudaStreamSynchronize(st_), "sync");
            cudaFree(d_scratch_);
        }
        check(cudaMalloc(&d_scratch_, need * sizeof(double)), "cudaMalloc scratch");
        scratch_cap_ = need;
    }
    double* own_out = partitioned() ? d_scratch_ + (size_t)4 * n : d_scratch_;
    if (own_count_ > 0) {
        TagArgs a{};
        a.q = d_q_; a.stride = stride_; a.slots = d_all_slots_.p; a.meta = d_meta_;
        a.n = own_count_; a.mx = opt_.mx; a.my = opt_.my; a.mbc = opt_.mbc; a.ivar = opt_.threshold_variable - 1;
        a.criteria = opt_.refinement_criteria;
        a.refine_th = opt_.refine_threshold; a.coarsen_th = opt_.coarsen_threshold;
        a.out = own_out;
        check(launch_tag(a, st_), "tag");
        ++cnt_.count_kernel_launches;
    }
    if (partitioned()) allgather_owned(own_out, 4, d_scratch_);
    std::vector<double> h((size_t)4 * n);
    check(cudaMemcpyAsync(h.data(), d_scratch_, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st_), "tags");
    if (partitioned()) comm_->sync(st_);
    else synchronize();
    target.resize(n);
    for (int p = 0; p < n; ++p) target[p] = forest_.leaves[p].level;
    const bool minmax = opt_.refinement_criteria == FCB_TAG_MINMAX;
    // cb_regrid_tag4coarsening over families (fclaw2d_regrid.c:70-97,
    // clawpatch_tag4coarsening fclaw2d_clawpatch.cpp:860-914)
    for (int p = 0; p < n; ++p) {
        if (!forest_.is_first_sibling(p)) continue;
        const int level = forest_.leaves[p].level;
        if (level > opt_.minlevel && opt_.coarsen_threshold > 0 && !domain_init) {
            bool keep;
            if (minmax) {
                double lo = h[4 * p], hi = h[4 * p + 1];
                for (int k = 1; k < 4; ++k) { lo = std::min(lo, h[4 * (p + k)]); hi = std::max(hi, h[4 * (p + k) + 1]); }
                keep = (hi - lo > opt_.coarsen_threshold);
            } else {
                keep = false;
                for (int k = 0; k < 4; ++k) keep = keep || h[4 * (p + k) + 3] != 0.0;
            }
            if (!keep)
                for (int k = 0; k < 4; ++k) target[p + k] = std::max(forest_.leaves[p + k].level - 1, 0);
        }
        p += 3;
    }
    // cb_fclaw2d_regrid_tag4refinement (fclaw2d_regrid.c:45-67)
    for (int p = 0; p < n; ++p) {
        const int level = forest_.leaves[p].level;
        if (level >= opt_.maxlevel) continue;
        bool refine;
        if (opt_.refine_threshold < 0) refine = true;
        else if (minmax) refine = (h[4 * p + 1] - h[4 * p] > opt_.refine_threshold);
        else refine = h[4 * p + 2] != 0.0;
        if (refine) target[p] = level + 1;
    }
}

// fclaw2d_domain_adapt (fclaw2d_convenience.c:498-680) + p4est_wrap_adapt:
// refine marked leaves once, coarsen complete marked families, balance.
bool Context::adapt(const std::vector<int>& target, std::vector<Leaf>& out) {
    const int n = num_patches();
    enum { REFINE = 1, COARSEN = 2 };
    std::vector<int> flag(n, 0);
    auto refine = [&](int p) { flag[p] = REFINE; };
    auto coarsen = [&](int p) { flag[p] = forest_.leaves[p].level > 0 ? COARSEN : 0; };
    for (int p = 0; p < n; ++p) {
        const int level = forest_.leaves[p].level;
        int t = target[p];
        if (opt_.smooth_refine) {
            const Neighbors& nb = nbrs_[p];
            auto consider = [&](int q) {
                if (forest_.leaves[q].level >= opt_.smooth_level) t = std::max(t, target[q]);
            };
            for (int f = 0; t <= level && f < 4; ++f) {
                if (nb.face_rel[f] == REL_SAMESIZE || nb.face_rel[f] == REL_DOUBLESIZE) consider(nb.face_nbr[f][0]);
                else if (nb.face_rel[f] == REL_HALFSIZE) { consider(nb.face_nbr[f][0]); consider(nb.face_nbr[f][1]); }
            }
            for (int c = 0; t <= level && c < 4; ++c)
                if (nb.corner_rel[c] != 0) consider(nb.corner_nbr[c]);
        }
        if (t > level) refine(p);
        else if (t < level) coarsen(p);
    }
    bool changed = false;
    std::vector<Leaf> r;
    std::vector<int> rf;
    r.reserve(n);
    for (int p = 0; p < n; ++p) {
        const Leaf& l = forest_.leaves[p];
        if (flag[p] == REFINE) {
            changed = true;
            const int32_t hh = QuadForest::width(l.level + 1);
            for (int k = 0; k < 4; ++k) {
                r.push_back(QuadForest::make(l.level + 1, l.x + (k & 1) * hh, l.y + (k >> 1) * hh));
                rf.push_back(0);
            }
        } else {
            r.push_back(l);
            rf.push_back(flag[p]);
        }
    }
    QuadForest tmp;
    tmp.leaves = r;
    std::vector<Leaf> c;
    c.reserve(r.size());
    for (size_t p = 0; p < r.size();) {
        if (tmp.is_first_sibling((int)p) && rf[p] == COARSEN && rf[p + 1] == COARSEN && rf[p + 2] == COARSEN &&
            rf[p + 3] == COARSEN) {
            c.push_back(QuadForest::make(r[p].level - 1, r[p].x, r[p].y));
            changed = true;
            p += 4;
        } else {
            c.push_back(r[p]);
            ++p;
        }
    }
    if (!changed) return false;
    QuadForest f;
    f.periodic_x = forest_.periodic_x;  // balance wraps across the periodic sides too
    f.periodic_y = forest_.periodic_y;
    f.leaves = c;
    f.balance();
    out = f.leaves;
    return true;
}

void Context::qinit_slots(const std::vector<int32_t>& slots) {
    if (slots.empty()) return;
    DevBuf<int32_t> d;
    d.reserve(slots.size());
    check(cudaMemcpy(d.p, slots.data(), slots.size() * 4, cudaMemcpyHostToDevice), "qinit slots");
    QinitArgs a{};
    a.q = d_q_; a.stride = stride_; a.slots = d.p; a.meta = d_meta_;
    a.n = (int)slots.size(); a.mx = opt_.mx; a.my = opt_.my; a.mbc = opt_.mbc; a.meqn = opt_.meqn;
    a.problem = opt_.problem; a.gamma1 = opt_.gamma - 1.0;
    for (int k = 0; k < 32; ++k) a.p[k] = opt_.problem_params[k];
    check(launch_qinit(a, st_), "qinit");
    ++cnt_.count_kernel_launches;
    synchronize();
}

// fclaw2d_domain_iterate_adapted + cb_fclaw2d_regrid_repopulate (fclaw2d_regrid.c:114-230)
void Context::repopulate(const std::vector<Leaf>& old_leaves, const std::vector<int>& old_slots,
                         bool domain_init) {
    const int nn = num_patches();
    std::vector<int> ns(nn, -1);
    std::vector<int32_t> transfer, fine, fresh, freed;
    int oj = 0, nj = 0;
    // pass 1: assign slots (new slots never reuse a slot freed in this regrid)
    std::vector<std::tuple<int, int, int>> events;  // kind, oj, nj
    while (oj < (int)old_leaves.size()) {
        const Leaf& o = old_leaves[oj];
        const Leaf& w = forest_.leaves[nj];
        if (o.level < w.level) { events.emplace_back(0, oj, nj); oj += 1; nj += 4; }
        else if (o.level > w.level) { events.emplace_back(1, oj, nj); oj += 4; nj += 1; }
        else { ns[nj] = old_slots[oj]; oj += 1; nj += 1; }
    }
    if (nj != nn) throw Error(FCB_ERR_INTERNAL, "iterate_adapted: leaf count mismatch");
    int need = nslots_used_;
    for (auto& e : events) need += (std::get<0>(e) == 0) ? 4 : 1;
    ensure_capacity(need);
    // new slots come from slots freed before this regrid or from the end of the
    // arena, never from the slots this regrid frees (its transfer reads them)
    for (auto& e : events) {
        const int kind = std::get<0>(e), o = std::get<1>(e), w = std::get<2>(e);
        if (kind == 0) {
            const int f0 = (int)fine.size();
            for (int k = 0; k < 4; ++k) { ns[w + k] = alloc_slot(); fine.push_back(ns[w + k]); fresh.push_back(ns[w + k]); }
            transfer.insert(transfer.end(), {0, old_slots[o], f0});
            freed.push_back(old_slots[o]);
        } else {
            ns[w] = alloc_slot();
            fresh.push_back(ns[w]);
            const int f0 = (int)fine.size();
            for (int k = 0; k < 4; ++k) { fine.push_back(old_slots[o + k]); freed.push_back(old_slots[o + k]); }
            transfer.insert(transfer.end(), {1, ns[w], f0});
        }
    }
    slot_of_ = ns;
    if (time_sync_ && !fresh.empty()) {
        // fclaw2d_clawpatch_time_sync_new: every new patch starts with zero registers
        DevBuf<int32_t> df;
        df.reserve(fresh.size());
        check(cudaMemcpy(df.p, fresh.data(), fresh.size() * 4, cudaMemcpyHostToDevice), "fresh slots");
        check(launch_zero_registers(d_treg_, treg_stride_, df.p, (int)fresh.size(), st_), "zero registers");
        check(cudaStreamSynchronize(st_), "sync");
    }
    // metadata of the new mesh is needed by qinit; transfers only need slots
    if (domain_init) {
        mesh_changed();
        qinit_slots(fresh);
    } else if (!transfer.empty()) {
        // the transfer lists live in buffers that only grow: a freed device
        // buffer would synchronise the whole device (every stream of a server);
        // the previous transfer finished before its regrid returned
        d_xfer_.reserve(transfer.size());
        d_xfer_fine_.reserve(fine.size());
        check(cudaMemcpy(d_xfer_.p, transfer.data(), transfer.size() * 4, cudaMemcpyHostToDevice), "transfer");
        check(cudaMemcpy(d_xfer_fine_.p, fine.data(), fine.size() * 4, cudaMemcpyHostToDevice), "fine");
        check(launch_regrid(d_q_, stride_, d_xfer_.p, d_xfer_fine_.p, (int)transfer.size() / 3, opt_.mx, opt_.my,
                            opt_.mbc, opt_.meqn, st_),
              "regrid transfer");
        ++cnt_.count_kernel_launches;
        synchronize();
    }
    free_slots_.insert(free_slots_.end(), freed.begin(), freed.end());
}

// fclaw2d_domain_iterate_adapted + cb_fclaw2d_regrid_repopulate
// (fclaw2d_regrid.c:114-230) followed by the patch transfer of
// fclaw2d_partition_domain (fclaw2d_partition.c:113-197), with one exchange:
// the owner of every new leaf receives the old patches its data comes from (the
// leaf itself, its parent, or its four children, ghost cells included) from
// their old owners, then runs the regrid transfer on its own slots.  Leaves of
// the new ghost layer get slots and receive data at the next ghost update.
void Context::repopulate_partitioned(const std::vector<Leaf>& old_leaves, const std::vector<int>& old_slots,
                                     const std::vector<int>& old_owner, bool domain_init) {
    const int nn = num_patches(), no = (int)old_leaves.size(), R = nranks_;
    partition_leaves();
    compute_neighbors();
    const std::vector<char> loc = local_set();
    // kind: 0 the same leaf, 1 a child of old leaf src, 2 the parent of old leaves src..src+3
    std::vector<int> kind(nn, 0), src(nn, -1);
    {
        int oj = 0, nj = 0;
        while (oj < no && nj < nn) {
            const Leaf& o = old_leaves[oj];
            const Leaf& w = forest_.leaves[nj];
            if (o.level < w.level) {
                for (int k = 0; k < 4; ++k) { kind[nj + k] = 1; src[nj + k] = oj; }
                oj += 1; nj += 4;
            } else if (o.level > w.level) {
                kind[nj] = 2; src[nj] = oj;
                oj += 4; nj += 1;
            } else {
                src[nj] = oj;
                ++oj; ++nj;
            }
        }
        if (nj != nn || oj != no) throw Error(FCB_ERR_INTERNAL, "iterate_adapted: leaf count mismatch");
    }
    // fresh leaves of the initial refinement are initialised, not transferred
    auto fresh = [&](int w) { return domain_init && kind[w] != 0; };
    std::vector<std::vector<int>> recv(R), send(R);
    bool any = false;
    for (int w = 0; w < nn; ++w) {
        if (fresh(w)) continue;
        const int ns = kind[w] == 2 ? 4 : 1;
        for (int k = 0; k < ns; ++k) {
            const int s = src[w] + k, os = old_owner[s], ow = owner_[w];
            if (os == ow) continue;
            any = true;
            if (ow == rank_) recv[os].push_back(s);
            else if (os == rank_) send[ow].push_back(s);
        }
    }
    for (int r = 0; r < R; ++r)
        for (auto* v : {&recv[r], &send[r]}) {
            std::sort(v->begin(), v->end());
            v->erase(std::unique(v->begin(), v->end()), v->end());
        }
    // slots: an upper bound of the new ones first (the arena may move)
    int need = nslots_used_;
    for (int r = 0; r < R; ++r) need += (int)recv[r].size();
    for (int w = 0; w < nn; ++w) need += loc[w] ? 1 : 0;
    for (int w = 0; w < nn; w += (kind[w] == 1 ? 4 : 1)) need += kind[w] == 1 ? 4 : 0;
    ensure_capacity(need);
    std::vector<int> ns(nn, -1), recv_slot(no, -1);
    std::vector<char> adopted_old(no, 0);
    std::vector<int32_t> temps;
    // leaves that stay the same and stay local keep their slot
    for (int w = 0; w < nn; ++w)
        if (kind[w] == 0 && loc[w] && old_slots[src[w]] >= 0) {
            ns[w] = old_slots[src[w]];
            adopted_old[src[w]] = 1;
        }
    // received patches land in their old ghost-layer slot, or a new slot
    for (int r = 0; r < R; ++r)
        for (int s : recv[r]) {
            if (old_slots[s] >= 0) {
                recv_slot[s] = old_slots[s];
            } else {
                recv_slot[s] = alloc_slot();
                temps.push_back(recv_slot[s]);
            }
        }
    for (int w = 0; w < nn; ++w) {
        if (!loc[w] || ns[w] >= 0) continue;
        if (kind[w] == 0 && owner_[w] == rank_) {  // moved here from another rank
            ns[w] = recv_slot[src[w]];
        } else {
            ns[w] = alloc_slot();
        }
    }
    // regrid transfer records on this rank: refined families with an owned child
    // (all four children are written), coarsened parents owned here
    auto src_slot = [&](int s) { return old_owner[s] == rank_ ? old_slots[s] : recv_slot[s]; };
    std::vector<int32_t> transfer, fine, fresh_slots;
    for (int w = 0; w < nn;) {
        if (kind[w] == 1) {
            bool mine = false;
            for (int k = 0; k < 4; ++k) mine = mine || owner_[w + k] == rank_;
            if (mine && !domain_init) {
                const int f0 = (int)fine.size();
                for (int k = 0; k < 4; ++k) {
                    int sl = ns[w + k];
                    if (sl < 0) {
                        sl = alloc_slot();
                        temps.push_back(sl);
                    }
                    fine.push_back(sl);
                }
                transfer.insert(transfer.end(), {0, src_slot(src[w]), f0});
            }
            for (int k = 0; k < 4; ++k)
                if (fresh(w + k) && owner_[w + k] == rank_) fresh_slots.push_back(ns[w + k]);
            w += 4;
            continue;
        }
        if (kind[w] == 2 && owner_[w] == rank_) {
            if (domain_init) {
                fresh_slots.push_back(ns[w]);
            } else {
                const int f0 = (int)fine.size();
                for (int k = 0; k < 4; ++k) fine.push_back(src_slot(src[w] + k));
                transfer.insert(transfer.end(), {1, ns[w], f0});
            }
        }
        ++w;
    }
    for (int w = 0; w < nn; ++w)
        if (owner_[w] == rank_ && ns[w] < 0) throw Error(FCB_ERR_INTERNAL, "owned leaf without a slot");
    for (size_t k = 0; k < transfer.size(); k += 3)
        if (transfer[k + 1] < 0 || transfer[k + 1] >= capacity_) throw Error(FCB_ERR_INTERNAL, "transfer slot");
    for (int32_t sl : fine)
        if (sl < 0 || sl >= capacity_) throw Error(FCB_ERR_INTERNAL, "transfer slot");
    for (int r = 0; r < R; ++r) {
        for (int s : send[r])
            if (old_slots[s] < 0 || old_slots[s] >= capacity_) throw Error(FCB_ERR_INTERNAL, "sent patch without a slot");
        for (int s : recv[r])
            if (recv_slot[s] < 0 || recv_slot[s] >= capacity_) throw Error(FCB_ERR_INTERNAL, "received patch slot");
    }
    // the exchange: old owners' patches (whole arrays) to the new owners
    if (any) {
        XList x;
        x.any = true;
        x.send_n.assign(R, 0);
        x.recv_n.assign(R, 0);
        for (int r = 0; r < R; ++r) {
            for (int s : send[r]) x.send.push_back(old_slots[s] * 2);
            for (int s : recv[r]) x.recv.push_back(recv_slot[s] * 2);
            x.send_n[r] = (int)send[r].size();
            x.recv_n[r] = (int)recv[r].size();
        }
        std::vector<int32_t> items(x.send);
        items.insert(items.end(), x.recv.begin(), x.recv.end());
        x.send_first = 0;
        x.recv_first = x.send.size();
        DevBuf<int32_t> d;
        d.reserve(std::max<size_t>(1, items.size()));
        if (!items.empty())
            check(cudaMemcpy(d.p, items.data(), items.size() * sizeof(int32_t), cudaMemcpyHostToDevice), "items");
        exchange(x, d.p);
        comm_->sync(st_);
    }
    if (!transfer.empty()) {
        DevBuf<int32_t> dt, df;
        dt.reserve(transfer.size());
        df.reserve(fine.size());
        check(cudaMemcpy(dt.p, transfer.data(), transfer.size() * 4, cudaMemcpyHostToDevice), "transfer");
        check(cudaMemcpy(df.p, fine.data(), fine.size() * 4, cudaMemcpyHostToDevice), "fine");
        check(launch_regrid(d_q_, stride_, dt.p, df.p, (int)transfer.size() / 3, opt_.mx, opt_.my, opt_.mbc,
                            opt_.meqn, st_),
              "regrid transfer");
        ++cnt_.count_kernel_launches;
        synchronize();
    }
    // slots no longer referenced return to the free list
    std::vector<char> live((size_t)capacity_, 0);
    for (int w = 0; w < nn; ++w)
        if (ns[w] >= 0) live[ns[w]] = 1;
    std::vector<char> seen((size_t)capacity_, 0);
    auto release = [&](int sl) {
        if (sl >= 0 && !live[sl] && !seen[sl]) {
            seen[sl] = 1;
            free_slots_.push_back(sl);
        }
    };
    for (int s = 0; s < no; ++s) release(old_slots[s]);
    for (int32_t sl : temps) release(sl);
    slot_of_ = ns;
    if (!fresh_slots.empty()) {
        mesh_changed();
        qinit_slots(fresh_slots);
    }
}

bool Context::regrid() {
    if (!initialized_) throw Error(FCB_ERR_STATE, "regrid before initialize");
    ensure_ghosts();  // tagging and the regrid transfer read ghost cells
    std::vector<int> target;
    tag(false, target);
    std::vector<Leaf> nl;
    const bool changed = adapt(target, nl);
    if (changed) {
        const std::vector<Leaf> old = forest_.leaves;
        const std::vector<int> old_slots = slot_of_;
        const std::vector<int> old_owner = owner_;
        forest_.leaves = nl;
        if (partitioned()) repopulate_partitioned(old, old_slots, old_owner, false);
        else repopulate(old, old_slots, false);
        mesh_changed();
        // this update's plan and the next macro step's, built together, for a
        // context that advances through fcb_advance_all_levels (a served solve
        // steps level by level and builds its one plan on demand)
        if (cnt_.count_amr_advance > 0) prefetch_plans();
        ghost_update(forest_.min_level(), forest_.max_level(), curr_time_, 0);
        ++cnt_.count_amr_new_domain;
    }
    ++cnt_.count_amr_regrid;
    return changed;
}

// fclaw2d_initialize (src/fclaw2d_initialize.c:75-248)
void Context::initialize() {
    ensure_scalars();
    ghosts_stale_ = false;
    ghosts_filled_ = false;  // qinit sets the ghost cells itself (unless init_ghostcell)
    forest_.uniform(opt_.minlevel);
    const int n = num_patches();
    free_slots_.clear();
    nslots_used_ = 0;
    if (partitioned()) {
        // fclaw2d_domain_new_unitsquare + the first partition: this rank's Morton
        // range and its ghost layer get slots
        partition_leaves();
        compute_neighbors();
        const std::vector<char> loc = local_set();
        ensure_capacity(std::max(1, (int)std::count(loc.begin(), loc.end(), 1)));
        slot_of_.assign(n, -1);
        for (int p = 0; p < n; ++p)
            if (loc[p]) slot_of_[p] = alloc_slot();
    } else {
        ensure_capacity(n);
        slot_of_.resize(n);
        for (int p = 0; p < n; ++p) slot_of_[p] = alloc_slot();
    }
    mesh_changed();
    qinit_slots(std::vector<int32_t>(slot_of_.begin() + own_first_, slot_of_.begin() + own_first_ + own_count_));
    initialized_ = true;
    if (opt_.init_ghostcell) ghost_update(forest_.min_level(), forest_.max_level(), 0.0, 0);
    if (opt_.minlevel < opt_.maxlevel) {
        for (int level = opt_.minlevel; level <= opt_.maxlevel; ++level) {
            std::vector<int> target;
            tag(true, target);
            std::vector<Leaf> nl;
            if (!adapt(target, nl)) break;
            const std::vector<Leaf> old = forest_.leaves;
            const std::vector<int> old_slots = slot_of_;
            const std::vector<int> old_owner = owner_;
            forest_.leaves = nl;
            if (partitioned()) repopulate_partitioned(old, old_slots, old_owner, true);
            else repopulate(old, old_slots, true);
            mesh_changed();
        }
    }
    if (opt_.init_ghostcell) ghost_update(forest_.min_level(), forest_.max_level(), 0.0, 0);
    synchronize();
}

// outstyle_1 (src/fclaw2d_run.c:120-290)
void Context::run() {
    if (!initialized_) throw Error(FCB_ERR_STATE, "run before initialize");
    const double final_time = opt_.tfinal;
    const int nout = opt_.nout;
    double dt_minlevel = opt_.initial_dt;
    const double t0 = 0;
    const double dt_outer = (final_time - t0) / ((double)nout);
    double t_curr = t0;
    int n_inner = 0;
    const size_t arena_bytes = (size_t)capacity_ * stride_ * sizeof(double);
    for (int n = 0; n < nout; ++n) {
        const double tstart = t_curr;
        curr_time_ = t_curr;
        const double tend = tstart + dt_outer;
        while (t_curr < tend) {
            const size_t bytes = (size_t)capacity_ * stride_ * sizeof(double);
            (void)arena_bytes;
            if (!opt_.use_fixed_dt) {
                check(cudaMemcpyAsync(d_qsave_, d_q_, bytes, cudaMemcpyDeviceToDevice, st_), "save_time_step");
                saved_stale_ = ghosts_stale_;  // the copy holds the ghost cells as they are now
                saved_filled_ = ghosts_filled_;
            }
            double dt_step = dt_minlevel;
            const double tol = 1e-2 * dt_step;
            int took_small_step = 0;
            if (!opt_.use_fixed_dt) {
                const double small_step = tend - (t_curr + dt_step);
                if (small_step < tol) {
                    dt_step = tend - t_curr;
                    if (small_step < 0) took_small_step = 1;
                }
            }
            // fclaw2d_run.c:206: the CFL maximum over all ranks
            const double maxcfl_step = global_maximum(advance_all_levels(t_curr, dt_step));
            if (std::isnan(maxcfl_step)) throw Error(FCB_ERR_NUMERIC, "NaN in the CFL number");
            if ((maxcfl_step > opt_.max_cfl) && opt_.reduce_cfl) {
                if (!opt_.use_fixed_dt) {
                    check(cudaMemcpyAsync(d_q_, d_qsave_, bytes, cudaMemcpyDeviceToDevice, st_), "restore_time_step");
                    ghosts_stale_ = saved_stale_;
                    ghosts_filled_ = saved_filled_;
                    dt_minlevel = dt_minlevel * opt_.desired_cfl / maxcfl_step;
                    continue;
                }
            }
            ++n_inner;
            t_curr += dt_step;
            if (!opt_.use_fixed_dt) {
                const double dt_new = dt_minlevel * opt_.desired_cfl / maxcfl_step;
                if (!took_small_step) dt_minlevel = dt_new;
            }
            curr_time_ = t_curr;
            if (opt_.regrid_interval > 0 && n_inner % opt_.regrid_interval == 0) regrid();
        }
        curr_time_ = t_curr;
    }
    synchronize();
}

// ---------------------------------------------------------------------------
// Data movement and diagnostics
// ---------------------------------------------------------------------------
// The owned patches (all patches on one rank) at their places in the
// all-leaves layout; the other entries of the host buffer are not touched.
void Context::get_q(double* host, size_t n, bool qinterp) {
    ensure_ghosts();
    const size_t ps = patch_size();
    const size_t total = ps * num_patches();
    if (n < total) throw Error(FCB_ERR_INVALID, "host buffer too small");
    const size_t mine = ps * own_count_;
    if (mine == 0) return;
    if (mine > stage_cap_) {
        cudaFree(d_stage_);
        check(cudaMalloc(&d_stage_, mine * sizeof(double)), "cudaMalloc stage");
        stage_cap_ = mine;
    }
    check(launch_gather(qinterp ? d_qti_ : d_q_, stride_, d_all_slots_.p, own_count_, (int64_t)ps, d_stage_,
                        false, opt_.claw_version == 5 ? opt_.meqn : 0, st_),
          "gather");
    ++cnt_.count_kernel_launches;
    check(cudaMemcpyAsync(host + ps * own_first_, d_stage_, mine * sizeof(double), cudaMemcpyDeviceToHost, st_),
          "get_q");
    synchronize();
}

// fclaw2d_clawpatch_output_ascii: rank 0 writes the header, then the ranks
// append their patches in rank order (fclaw2d_domain_serialization_enter/leave),
// each turn separated by a collective barrier.  One rank writes the whole frame.
void Context::output_ascii(int iframe, const std::string& dir) {
    if (!initialized_) throw Error(FCB_ERR_STATE, "output before initialize");
    if (iframe < 0 || iframe > 9999) throw Error(FCB_ERR_INVALID, "frame number must be in 0..9999");
    ensure_ghosts();
    const size_t ps = patch_size();
    const int n = own_count_;
    std::vector<double> host(ps * (size_t)n);
    if (n > 0) {
        if (ps * (size_t)n > stage_cap_) {
            cudaFree(d_stage_);
            check(cudaMalloc(&d_stage_, ps * (size_t)n * sizeof(double)), "cudaMalloc stage");
            stage_cap_ = ps * (size_t)n;
        }
        // the clawpack 4.6 layout for both versions: the values per cell are the same
        check(launch_gather(d_q_, stride_, d_all_slots_.p, n, (int64_t)ps, d_stage_, false, 0, st_), "gather");
        ++cnt_.count_kernel_launches;
        check(cudaMemcpyAsync(host.data(), d_stage_, host.size() * sizeof(double), cudaMemcpyDeviceToHost, st_),
              "output");
        synchronize();
    }
    std::vector<OutputPatch> ps_out((size_t)n);
    for (int k = 0; k < n; ++k) {
        const int p = own_first_ + k;
        const PatchMeta m = meta_of(forest_.leaves[p]);
        // a brick's patches report the block's level and the block number
        // (blocks in row-major order, block i + mi*j, as fclaw2d_map_brick)
        int off = 0;
        while ((1 << off) < opt_.brick) ++off;
        ps_out[k] = OutputPatch{p, (int)forest_.leaves[p].level - off, m.xlower, m.ylower, m.dx, m.dy};
        const int64_t bw = (int64_t)QuadForest::kRoot / opt_.brick;
        ps_out[k].block = (int)(forest_.leaves[p].x / bw + opt_.brick * (forest_.leaves[p].y / bw));
    }
    auto barrier = [&] {
        if (!partitioned()) return;
        check(cudaMemsetAsync(d_cfl_ + 2, 0, sizeof(unsigned long long), st_), "barrier");
        comm_->allreduce_max_u64(d_cfl_ + 2, 1, st_);
        comm_->sync(st_);
    };
    std::string err;
    for (int r = 0; r < nranks_; ++r) {
        if (r == rank_ && err.empty()) {
            try {
                if (r == 0)
                    write_ascii_header(dir, iframe, curr_time_, opt_.meqn, opt_.maux, (long)num_patches());
                append_ascii_patches(dir, iframe, opt_.meqn, opt_.mx, opt_.my, opt_.mbc, ps_out, host.data(), ps,
                                     rank_);
            } catch (const std::runtime_error& e) {
                err = e.what();  // reported after the turns, so every rank takes every barrier
            }
        }
        barrier();
    }
    if (!err.empty()) throw Error(FCB_ERR_INVALID, err);
}

void Context::set_q(const double* host, size_t n) {
    const size_t ps = patch_size();
    const size_t total = ps * num_patches();
    if (n < total) throw Error(FCB_ERR_INVALID, "host buffer too small");
    const size_t mine = ps * own_count_;
    if (mine == 0) return;
    if (mine > stage_cap_) {
        cudaFree(d_stage_);
        check(cudaMalloc(&d_stage_, mine * sizeof(double)), "cudaMalloc stage");
        stage_cap_ = mine;
    }
    check(cudaMemcpyAsync(d_stage_, host + ps * own_first_, mine * sizeof(double), cudaMemcpyHostToDevice, st_),
          "set_q");
    check(launch_gather(d_q_, stride_, d_all_slots_.p, own_count_, (int64_t)ps, d_stage_, true,
                        opt_.claw_version == 5 ? opt_.meqn : 0, st_),
          "scatter");
    ++cnt_.count_kernel_launches;
    ghosts_stale_ = false;  // every cell of every patch was just written
    ghosts_filled_ = false;
    synchronize();
}

// Per-patch sums on the owning ranks, gathered, then the same compensated sum
// over all patches in Morton order on every rank (identical to one rank).
void Context::conservation(double* sums) {
    const int n = num_patches();
    const size_t need = (size_t)n * opt_.meqn + (partitioned() ? (size_t)own_count_ * opt_.meqn : 0);
    if (need > scratch_cap_) {
        if (d_scratch_) {
            check(cudaStreamSynchronize(st_), "sync");
            cudaFree(d_scratch_);
        }
        check(cudaMalloc(&d_scratch_, need * sizeof(double)), "cudaMalloc scratch");
        scratch_cap_ = need;
    }
    double* own_out = partitioned() ? d_scratch_ + (size_t)n * opt_.meqn : d_scratch_;
    if (own_count_ > 0) {
        check(launch_mass(d_q_, stride_, d_all_slots_.p, d_meta_, own_count_, opt_.mx, opt_.my, opt_.mbc, opt_.meqn,
                          own_out, st_),
              "mass");
        ++cnt_.count_kernel_launches;
    }
    if (partitioned()) allgather_owned(own_out, opt_.meqn, d_scratch_);
    std::vector<double> h((size_t)n * opt_.meqn);
    check(cudaMemcpyAsync(h.data(), d_scratch_, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st_), "mass");
    if (partitioned()) comm_->sync(st_);
    else synchronize();
    for (int m = 0; m < opt_.meqn; ++m) {
        double s = 0.0, c = 0.0;
        for (int p = 0; p < n; ++p) {
            const double y = h[(size_t)p * opt_.meqn + m] - c;
            const double t = s + y;
            c = (t - s) - y;
            s = t;
        }
        sums[m] = s;
    }
}

}  // namespace fcb
