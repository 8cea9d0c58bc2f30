// extern "C" entry points declared in include/fclaw_b200.h.  Every call
// catches exceptions and CUDA errors and turns them into status codes; the
// library never terminates the process.
#include <cmath>
#include <memory>
#include <new>
#include <string>

#include "fcb_runtime.hpp"
#include "fcb_serve.hpp"

struct fcb_server {
    fcb::Server* impl;
};

struct fcb_context {
    fcb::Context* impl;
};

struct fcb_comm {
    std::shared_ptr<fcb::Comm> impl;
};

namespace {
thread_local std::string g_error;

template <class F>
int guard(F&& f) {
    try {
        f();
        return FCB_OK;
    } catch (const fcb::Error& e) {
        g_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_error = "out of host memory";
        return FCB_ERR_INTERNAL;
    } catch (const std::exception& e) {
        g_error = e.what();
        return FCB_ERR_INTERNAL;
    }
}

int need(const void* p, const char* what) {
    if (!p) throw fcb::Error(FCB_ERR_INVALID, std::string("null argument: ") + what);
    return 0;
}

// A collective call of a partitioned solve that fails on this rank marks the
// communicator failed, so the other ranks' next collective returns
// FCB_ERR_COMM instead of waiting out the time limit.
template <class F>
int collective(fcb_context_t* ctx, F&& f) {
    const int rc = guard(std::forward<F>(f));
    if (rc != FCB_OK && rc != FCB_ERR_COMM && ctx && ctx->impl && ctx->impl->partitioned())
        ctx->impl->abort_comm(g_error);
    return rc;
}
}  // namespace

namespace fcb {
__attribute__((visibility("hidden"))) void set_last_error(const std::string& msg) { g_error = msg; }
}  // namespace fcb

extern "C" {

const char* fcb_last_error(void) { return g_error.c_str(); }
int fcb_abi_version(void) { return FCB_ABI_VERSION; }

int fcb_context_create(const fcb_options_t* opt, void* cuda_stream, fcb_context_t** out) {
    return guard([&] {
        need(opt, "opt");
        need(out, "out");
        *out = nullptr;
        auto* c = new fcb_context{nullptr};
        try {
            c->impl = new fcb::Context(*opt, (cudaStream_t)cuda_stream);
        } catch (...) {
            delete c;
            throw;
        }
        *out = c;
    });
}

int fcb_context_destroy(fcb_context_t* ctx) {
    return guard([&] {
        if (!ctx) return;
        delete ctx->impl;
        delete ctx;
    });
}

#define CTX()                 \
    need(ctx, "ctx");         \
    fcb::Context& C = *ctx->impl

int fcb_initialize(fcb_context_t* ctx) { return collective(ctx, [&] { CTX(); C.initialize(); }); }
int fcb_run(fcb_context_t* ctx) { return collective(ctx, [&] { CTX(); C.run(); }); }

int fcb_advance_all_levels(fcb_context_t* ctx, double t, double dt, double* maxcfl) {
    return collective(ctx, [&] {
        CTX();
        need(maxcfl, "maxcfl");
        *maxcfl = C.advance_all_levels(t, dt);
        if (std::isnan(*maxcfl)) throw fcb::Error(FCB_ERR_NUMERIC, "NaN in the CFL number");
    });
}

int fcb_advance_all_levels_async(fcb_context_t* ctx, double t, double dt) {
    return collective(ctx, [&] {
        CTX();
        C.advance_all_levels_async(t, dt);
    });
}

int fcb_read_max_cfl(fcb_context_t* ctx, double* maxcfl) {
    return guard([&] {
        CTX();
        need(maxcfl, "maxcfl");
        *maxcfl = C.read_max_cfl();
    });
}

int fcb_update_single_step(fcb_context_t* ctx, int level, double t, double dt, double* maxcfl) {
    return guard([&] {
        CTX();
        need(maxcfl, "maxcfl");
        *maxcfl = C.update_single_step(level, t, dt);
        if (std::isnan(*maxcfl)) throw fcb::Error(FCB_ERR_NUMERIC, "NaN in the CFL number");
    });
}

int fcb_update_single_step_async(fcb_context_t* ctx, int level, double t, double dt) {
    return guard([&] { CTX(); C.update_single_step_async(level, t, dt); });
}

int fcb_single_step_update(fcb_context_t* ctx, int patchno, double t, double dt, int iter, int total_count,
                           double* cfl) {
    return guard([&] {
        CTX();
        need(cfl, "cfl");
        if (iter < 0 || total_count <= 0 || iter >= total_count) throw fcb::Error(FCB_ERR_INVALID, "bad iter/total_count");
        *cfl = C.single_step_update(patchno, t, dt, iter, total_count);
    });
}

int fcb_ghost_update(fcb_context_t* ctx, int minlevel, int maxlevel, double sync_time, int time_interp) {
    return collective(ctx, [&] {
        CTX();
        C.ghost_update(minlevel, maxlevel, sync_time, time_interp);
    });
}

int fcb_timeinterp(fcb_context_t* ctx, int level, double alpha) {
    return guard([&] { CTX(); C.timeinterp(level, alpha); });
}

int fcb_regrid(fcb_context_t* ctx, int* changed) {
    return collective(ctx, [&] {
        CTX();
        const bool ch = C.regrid();
        if (changed) *changed = ch ? 1 : 0;
    });
}

int fcb_physical_set_bc(fcb_context_t* ctx, int level, int time_interp) {
    return guard([&] { CTX(); C.physical_set_bc(level, time_interp); });
}

int fcb_num_patches(fcb_context_t* ctx, int* n) {
    return guard([&] {
        CTX();
        need(n, "n");
        *n = C.num_patches();
    });
}

int fcb_patch_info(fcb_context_t* ctx, int p, int* level, int* x, int* y) {
    return guard([&] {
        CTX();
        if (p < 0 || p >= C.num_patches()) throw fcb::Error(FCB_ERR_INVALID, "bad patch number");
        const fcb::Leaf& l = C.leaf(p);
        if (level) *level = l.level;
        if (x) *x = l.x;
        if (y) *y = l.y;
    });
}

int fcb_patch_neighbors(fcb_context_t* ctx, int p, int* out) {
    return guard([&] {
        CTX();
        need(out, "out");
        if (p < 0 || p >= C.num_patches()) throw fcb::Error(FCB_ERR_INVALID, "bad patch number");
        const fcb::Neighbors& n = C.nbrs(p);
        for (int f = 0; f < 4; ++f) {
            out[f] = n.face_rel[f];
            out[4 + 2 * f] = n.face_nbr[f][0];
            out[5 + 2 * f] = n.face_nbr[f][1];
            out[12 + f] = n.corner_rel[f];
            out[16 + f] = n.corner_nbr[f];
        }
        out[20] = n.has_fine;
        out[21] = n.on_cf;
    });
}

int fcb_patch_size(fcb_context_t* ctx, size_t* n) {
    return guard([&] {
        CTX();
        need(n, "n");
        *n = C.patch_size();
    });
}

int fcb_get_q(fcb_context_t* ctx, double* host, size_t n) {
    return guard([&] { CTX(); need(host, "host"); C.get_q(host, n, false); });
}
int fcb_set_q(fcb_context_t* ctx, const double* host, size_t n) {
    return guard([&] { CTX(); need(host, "host"); C.set_q(host, n); });
}
int fcb_get_qinterp(fcb_context_t* ctx, double* host, size_t n) {
    return guard([&] { CTX(); need(host, "host"); C.get_q(host, n, true); });
}

int fcb_counters(fcb_context_t* ctx, fcb_counters_t* out) {
    return guard([&] {
        CTX();
        need(out, "out");
        *out = C.counters();
    });
}

int fcb_conservation_check(fcb_context_t* ctx, double* sums) {
    return collective(ctx, [&] { CTX(); need(sums, "sums"); C.conservation(sums); });
}

int fcb_curr_time(fcb_context_t* ctx, double* t) {
    return guard([&] { CTX(); need(t, "t"); *t = C.curr_time(); });
}

int fcb_synchronize(fcb_context_t* ctx) { return guard([&] { CTX(); C.synchronize(); }); }

// ---- partitioned solves ------------------------------------------------------
int fcb_comm_create_local(int nranks, double timeout_s, fcb_comm_t** comms) {
    return guard([&] {
        need(comms, "comms");
        auto g = fcb::make_local_group(nranks, timeout_s);
        for (int r = 0; r < nranks; ++r) comms[r] = nullptr;
        for (int r = 0; r < nranks; ++r) comms[r] = new fcb_comm{g[r]};
    });
}

int fcb_comm_nccl_unique_id(const char* nccl_library, unsigned char id[128]) {
    return guard([&] {
        need(id, "id");
        fcb::nccl_unique_id(nccl_library, id);
    });
}

int fcb_comm_create_nccl(const char* nccl_library, const unsigned char id[128], int rank, int nranks,
                         double timeout_s, fcb_comm_t** out) {
    return guard([&] {
        need(id, "id");
        need(out, "out");
        *out = nullptr;
        auto c = fcb::make_nccl_comm(nccl_library, id, rank, nranks, timeout_s);
        *out = new fcb_comm{std::move(c)};
    });
}

int fcb_comm_destroy(fcb_comm_t* comm) {
    return guard([&] { delete comm; });
}

int fcb_context_create_partitioned(const fcb_options_t* opt, void* cuda_stream, fcb_comm_t* comm,
                                   fcb_context_t** out) {
    return guard([&] {
        need(opt, "opt");
        need(comm, "comm");
        need(out, "out");
        *out = nullptr;
        auto* c = new fcb_context{nullptr};
        try {
            c->impl = new fcb::Context(*opt, (cudaStream_t)cuda_stream, comm->impl);
        } catch (...) {
            delete c;
            throw;
        }
        *out = c;
    });
}

int fcb_partition_info(fcb_context_t* ctx, int* rank, int* nranks, int* first, int* count) {
    return guard([&] {
        CTX();
        need(rank, "rank");
        need(nranks, "nranks");
        need(first, "first");
        need(count, "count");
        *rank = C.rank();
        *nranks = C.nranks();
        *first = C.own_first();
        *count = C.own_count();
    });
}

int fcb_partition_plan(const fcb_options_t* opt, int nranks, int rank, int nleaves, const int* level, const int* x,
                       const int* y, int minlevel, int maxlevel, int time_interp, int* first, int* count,
                       int* ghosts, int* x1_send, int* x1_recv, int* x2_send, int* x2_recv) {
    return guard([&] {
        need(opt, "opt");
        for (const void* p : {(const void*)level, (const void*)x, (const void*)y, (const void*)first,
                              (const void*)count, (const void*)ghosts, (const void*)x1_send, (const void*)x1_recv,
                              (const void*)x2_send, (const void*)x2_recv})
            need(p, "array");
        if (nleaves < 1) throw fcb::Error(FCB_ERR_INVALID, "no leaves");
        std::vector<fcb::Leaf> leaves;
        leaves.reserve(nleaves);
        for (int k = 0; k < nleaves; ++k) {
            if (level[k] < 0 || level[k] > 20) throw fcb::Error(FCB_ERR_INVALID, "leaf level out of range");
            const int32_t w = fcb::QuadForest::width(level[k]);
            if (x[k] < 0 || y[k] < 0 || x[k] % w || y[k] % w || x[k] >= fcb::QuadForest::kRoot ||
                y[k] >= fcb::QuadForest::kRoot)
                throw fcb::Error(FCB_ERR_INVALID, "leaf corner not on its level's grid");
            leaves.push_back(fcb::QuadForest::make(level[k], x[k], y[k]));
            if (k && !(leaves[k - 1].key < leaves[k].key)) throw fcb::Error(FCB_ERR_INVALID, "leaves not in Morton order");
        }
        const fcb::PartitionPlan pp =
            fcb::Context::partition_plan(*opt, leaves, rank, nranks, minlevel, maxlevel, time_interp);
        *first = pp.first;
        *count = pp.count;
        *ghosts = pp.ghosts;
        for (int r = 0; r < nranks; ++r) {
            x1_send[r] = pp.x1_send[r];
            x1_recv[r] = pp.x1_recv[r];
            x2_send[r] = pp.x2_send[r];
            x2_recv[r] = pp.x2_recv[r];
        }
    });
}

int fcb_global_maximum(fcb_context_t* ctx, double value, double* out) {
    return collective(ctx, [&] {
        CTX();
        need(out, "out");
        *out = C.global_maximum(value);
    });
}

int fcb_output_ascii(fcb_context_t* ctx, int iframe, const char* dir) {
    return collective(ctx, [&] {
        CTX();
        C.output_ascii(iframe, dir ? std::string(dir) : std::string("."));
    });
}

int fcb_measure_fp_rate(int fp64, void* cuda_stream, double* ops_per_second) {
    return guard([&] {
        need(ops_per_second, "ops_per_second");
        const cudaError_t e = fcb::measure_fp_rate(fp64 != 0, (cudaStream_t)cuda_stream, ops_per_second);
        if (e != cudaSuccess) throw fcb::Error(FCB_ERR_CUDA, std::string("fp rate probe: ") + cudaGetErrorString(e));
    });
}

int fcb_step_kernel_time(fcb_context_t* ctx, double t, double dt, int launches, int* fused, double* ms_per_launch) {
    return guard([&] {
        CTX();
        need(fused, "fused");
        need(ms_per_launch, "ms_per_launch");
        bool f = false;
        *ms_per_launch = C.step_kernel_time(t, dt, launches, &f);
        *fused = f ? 1 : 0;
    });
}

int fcb_autotune_info(fcb_context_t* ctx, int* step_form, int* ghost_unroll) {
    return guard([&] {
        CTX();
        need(step_form, "step_form");
        need(ghost_unroll, "ghost_unroll");
        *step_form = C.step_form_used();
        *ghost_unroll = C.ghost_unroll_used();
    });
}

// ---- serving ----
int fcb_server_create(size_t budget_bytes, void* cuda_stream, fcb_server_t** out) {
    return guard([&] {
        need(out, "out");
        *out = nullptr;
        auto* sv = new fcb_server{nullptr};
        try {
            sv->impl = new fcb::Server(budget_bytes, (cudaStream_t)cuda_stream);
        } catch (...) {
            delete sv;
            throw;
        }
        *out = sv;
    });
}
int fcb_server_destroy(fcb_server_t* s) {
    return guard([&] {
        if (!s) return;
        delete s->impl;
        delete s;
    });
}
int fcb_server_submit(fcb_server_t* s, const fcb_options_t* opt, int* id) {
    return guard([&] {
        need(s, "server");
        need(opt, "opt");
        need(id, "id");
        *id = s->impl->submit(*opt);
    });
}
int fcb_server_round(fcb_server_t* s, int* active, int* queued) {
    return guard([&] {
        need(s, "server");
        const int a = s->impl->round();
        if (active) *active = a;
        if (queued) *queued = s->impl->queued();
    });
}
int fcb_server_status(fcb_server_t* s, int id, fcb_request_status_t* out) {
    return guard([&] {
        need(s, "server");
        need(out, "out");
        const fcb::Request& r = s->impl->request(id);
        out->state = r.state;
        out->num_patches = r.ctx ? r.ctx->num_patches() : 0;
        out->t = r.t;
        out->submit_s = r.t_submit;
        out->start_s = r.t_start;
        out->finish_s = r.t_finish;
        out->cell_updates = r.cell_updates;
        out->count_amr_advance = r.ctx ? r.ctx->counters().count_amr_advance : 0;
        if (r.state == FCB_REQ_FAILED) fcb::set_last_error(r.error);
    });
}
int fcb_server_get_q(fcb_server_t* s, int id, double* host, size_t n) {
    return guard([&] {
        need(s, "server");
        need(host, "host");
        s->impl->get_q(id, host, n);
    });
}
int fcb_server_release(fcb_server_t* s, int id) {
    return guard([&] {
        need(s, "server");
        s->impl->release(id);
    });
}
int fcb_server_set_work_limit(fcb_server_t* s, long long max_cells) {
    return guard([&] {
        need(s, "server");
        if (max_cells < 0) throw fcb::Error(FCB_ERR_INVALID, "max_cells must be >= 0");
        s->impl->set_work_limit(max_cells);
    });
}

int fcb_server_clock(fcb_server_t* s, double* now, long long* rounds, long long* launches) {
    return guard([&] {
        need(s, "server");
        if (now) *now = s->impl->now();
        if (rounds) *rounds = s->impl->rounds();
        if (launches) *launches = s->impl->launches();
    });
}

}  // extern "C"
