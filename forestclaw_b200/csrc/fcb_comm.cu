// Communicators of a partitioned solve (fcb_comm.hpp): the in-process group
// and NCCL, plus the two small kernels the exchanges use.
#include "fcb_comm.hpp"
#include "fcb_runtime.hpp"

#include <dlfcn.h>
#include <nccl.h>

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>

namespace fcb {

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
namespace {
__global__ void max_words_kernel(unsigned long long* v, const unsigned long long* words, int n, int nranks) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    unsigned long long m = 0;
    for (int r = 0; r < nranks; ++r) m = max(m, words[(size_t)r * n + k]);
    v[k] = m;
}

// one CTA per item; the patch's psize doubles in both directions
__global__ void pack_patches_kernel(double* q, double* qti, int64_t stride, const int32_t* items, int64_t psize,
                                    double* buf, int pack) {
    const int32_t it = items[blockIdx.x];
    double* a = ((it & 1) ? qti : q) + (int64_t)(it >> 1) * stride;
    double* b = buf + (int64_t)blockIdx.x * psize;
    if (pack)
        for (int64_t i = threadIdx.x; i < psize; i += blockDim.x) b[i] = a[i];
    else
        for (int64_t i = threadIdx.x; i < psize; i += blockDim.x) a[i] = b[i];
}
}  // namespace

cudaError_t launch_max_words(unsigned long long* v, const unsigned long long* words, int n, int nranks,
                             cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    max_words_kernel<<<(n + 127) / 128, 128, 0, st>>>(v, words, n, nranks);
    return cudaGetLastError();
}

cudaError_t launch_pack_patches(double* q, double* qti, int64_t stride, const int32_t* items, int n, int64_t psize,
                                double* buf, bool pack, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    pack_patches_kernel<<<n, 256, 0, st>>>(q, qti, stride, items, psize, buf, pack ? 1 : 0);
    return cudaGetLastError();
}

namespace {
[[noreturn]] void comm_fail(const std::string& m) { throw Error(FCB_ERR_COMM, m); }
void cuda_ok(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Error(FCB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------
// In-process group
// ---------------------------------------------------------------------------
struct Group {
    int n;
    std::chrono::duration<double> timeout;
    std::mutex mu;
    std::condition_variable cv;
    uint64_t gen = 0;
    int arrived = 0;
    bool failed = false;
    std::string why;
    // per rank: events (created by the rank's first collective, then fixed)
    std::vector<cudaEvent_t> ready, done;
    // per call parity and rank: the published send descriptor (a rank is at
    // most one call ahead of the slowest, so two buffers suffice)
    struct Post {
        const char* send = nullptr;
        std::vector<size_t> off, bytes;
    };
    std::vector<Post> post[2];

    void fail_locked(const std::string& m) {
        if (!failed) {
            failed = true;
            why = m;
        }
        cv.notify_all();
    }
    void barrier(int r) {
        std::unique_lock<std::mutex> lk(mu);
        if (failed) comm_fail("communicator failed: " + why);
        const uint64_t my = gen;
        if (++arrived == n) {
            arrived = 0;
            ++gen;
            cv.notify_all();
            return;
        }
        if (!cv.wait_for(lk, timeout, [&] { return gen != my || failed; }))
            fail_locked("rank " + std::to_string(r) + " waited " + std::to_string(timeout.count()) +
                        " s for the other ranks at a collective");
        if (failed) comm_fail("communicator failed: " + why);
    }
};

class LocalComm final : public Comm {
  public:
    LocalComm(std::shared_ptr<Group> g, int r) : g_(std::move(g)), r_(r) {}
    ~LocalComm() override {
        if (ready_) cudaEventDestroy(ready_);
        if (done_) cudaEventDestroy(done_);
        if (scratch_) cudaFree(scratch_);
    }
    int rank() const override { return r_; }
    int size() const override { return g_->n; }

    void alltoallv(const void* send, const size_t* send_off, const size_t* send_bytes, void* recv,
                   const size_t* recv_off, const size_t* recv_bytes, cudaStream_t st) override {
        const int n = g_->n;
        if (!ready_) {
            cuda_ok(cudaEventCreateWithFlags(&ready_, cudaEventDisableTiming), "cudaEventCreate");
            cuda_ok(cudaEventCreateWithFlags(&done_, cudaEventDisableTiming), "cudaEventCreate");
            std::lock_guard<std::mutex> lk(g_->mu);
            g_->ready[r_] = ready_;
            g_->done[r_] = done_;
        }
        const int par = (int)(calls_++ & 1);
        cuda_ok(cudaEventRecord(ready_, st), "cudaEventRecord");
        {
            std::lock_guard<std::mutex> lk(g_->mu);
            Group::Post& p = g_->post[par][r_];
            p.send = static_cast<const char*>(send);
            p.off.assign(send_off, send_off + n);
            p.bytes.assign(send_bytes, send_bytes + n);
        }
        g_->barrier(r_);
        // every post of this call is complete and stays unchanged until this
        // rank reaches the next barrier
        for (int p = 0; p < n; ++p) {
            const Group::Post& P = g_->post[par][p];
            if (P.bytes[r_] != recv_bytes[p]) {
                std::lock_guard<std::mutex> lk(g_->mu);
                g_->fail_locked("exchange sizes disagree between ranks " + std::to_string(p) + " and " +
                                std::to_string(r_));
                comm_fail("communicator failed: " + g_->why);
            }
            if (recv_bytes[p] == 0) continue;
            if (p != r_) cuda_ok(cudaStreamWaitEvent(st, g_->ready[p], 0), "cudaStreamWaitEvent");
            cuda_ok(cudaMemcpyAsync(static_cast<char*>(recv) + recv_off[p], P.send + P.off[r_], recv_bytes[p],
                                    cudaMemcpyDefault, st),
                    "exchange copy");
        }
        cuda_ok(cudaEventRecord(done_, st), "cudaEventRecord");
        g_->barrier(r_);
        // the peers have queued their reads of this rank's send buffer: later
        // work on this stream (which may overwrite it) waits for them
        for (int p = 0; p < n; ++p)
            if (p != r_) cuda_ok(cudaStreamWaitEvent(st, g_->done[p], 0), "cudaStreamWaitEvent");
    }

    void allreduce_max_u64(unsigned long long* v, int n, cudaStream_t st) override {
        const int R = g_->n;
        if (n <= 0) return;
        if ((size_t)n * R > scratch_cap_) {
            if (scratch_) {
                cuda_ok(cudaStreamSynchronize(st), "sync");
                cudaFree(scratch_);
            }
            cuda_ok(cudaMalloc(&scratch_, (size_t)n * R * 2 * sizeof(unsigned long long)), "cudaMalloc");
            scratch_cap_ = (size_t)n * R;
        }
        // the send copy keeps v's value stable while the peers read it
        unsigned long long* mine = scratch_ + scratch_cap_;
        cuda_ok(cudaMemcpyAsync(mine, v, (size_t)n * 8, cudaMemcpyDeviceToDevice, st), "copy");
        std::vector<size_t> so(R, 0), sb(R, (size_t)n * 8), ro(R), rb(R, (size_t)n * 8);
        for (int p = 0; p < R; ++p) ro[p] = (size_t)p * n * 8;
        alltoallv(mine, so.data(), sb.data(), scratch_, ro.data(), rb.data(), st);
        cuda_ok(launch_max_words(v, scratch_, n, R, st), "max");
    }

    void sync(cudaStream_t st) override { cuda_ok(cudaStreamSynchronize(st), "cudaStreamSynchronize"); }

    void abort(const std::string& why) override {
        std::lock_guard<std::mutex> lk(g_->mu);
        g_->fail_locked("rank " + std::to_string(r_) + ": " + why);
    }

  private:
    std::shared_ptr<Group> g_;
    int r_;
    uint64_t calls_ = 0;
    cudaEvent_t ready_ = nullptr, done_ = nullptr;
    unsigned long long* scratch_ = nullptr;
    size_t scratch_cap_ = 0;
};

// ---------------------------------------------------------------------------
// NCCL, loaded at run time (the process's own NCCL when it has one loaded)
// ---------------------------------------------------------------------------
struct NcclApi {
    void* h = nullptr;
    decltype(&ncclGetUniqueId) get_unique_id = nullptr;
    decltype(&ncclCommInitRankConfig) init_rank_config = nullptr;
    decltype(&ncclCommDestroy) destroy = nullptr;
    decltype(&ncclCommAbort) abort = nullptr;
    decltype(&ncclCommGetAsyncError) async_error = nullptr;
    decltype(&ncclGroupStart) group_start = nullptr;
    decltype(&ncclGroupEnd) group_end = nullptr;
    decltype(&ncclSend) send = nullptr;
    decltype(&ncclRecv) recv = nullptr;
    decltype(&ncclAllReduce) all_reduce = nullptr;
    decltype(&ncclGetErrorString) error_string = nullptr;
};

const NcclApi& nccl_api(const char* library) {
    static std::mutex mu;
    static NcclApi api;
    std::lock_guard<std::mutex> lk(mu);
    if (api.h) return api;
    const char* path = (library && *library) ? library : "libnccl.so.2";
    void* h = dlopen(path, RTLD_NOW | RTLD_GLOBAL);
    if (!h) comm_fail(std::string("cannot load NCCL (") + path + "): " + dlerror());
    auto sym = [&](auto& f, const char* name) {
        f = reinterpret_cast<std::remove_reference_t<decltype(f)>>(dlsym(h, name));
        if (!f) comm_fail(std::string("NCCL library lacks ") + name);
    };
    sym(api.get_unique_id, "ncclGetUniqueId");
    sym(api.init_rank_config, "ncclCommInitRankConfig");
    sym(api.destroy, "ncclCommDestroy");
    sym(api.abort, "ncclCommAbort");
    sym(api.async_error, "ncclCommGetAsyncError");
    sym(api.group_start, "ncclGroupStart");
    sym(api.group_end, "ncclGroupEnd");
    sym(api.send, "ncclSend");
    sym(api.recv, "ncclRecv");
    sym(api.all_reduce, "ncclAllReduce");
    sym(api.error_string, "ncclGetErrorString");
    api.h = h;
    return api;
}

class NcclComm final : public Comm {
  public:
    NcclComm(const char* library, const unsigned char id[128], int rank, int nranks, double timeout_s)
        : api_(nccl_api(library)), r_(rank), n_(nranks), timeout_(timeout_s) {
        ncclUniqueId uid;
        static_assert(sizeof(uid.internal) == 128, "ncclUniqueId is 128 bytes");
        std::memcpy(uid.internal, id, 128);
        ncclConfig_t cfg = NCCL_CONFIG_INITIALIZER;
        cfg.blocking = 0;  // every wait below is bounded
        ncclResult_t e = api_.init_rank_config(&comm_, nranks, uid, rank, &cfg);
        if (e != ncclSuccess && e != ncclInProgress) nccl_fail(e, "ncclCommInitRankConfig");
        wait_ready("ncclCommInitRankConfig");
    }
    ~NcclComm() override {
        if (comm_) api_.destroy(comm_);
    }
    int rank() const override { return r_; }
    int size() const override { return n_; }

    void alltoallv(const void* send, const size_t* send_off, const size_t* send_bytes, void* recv,
                   const size_t* recv_off, const size_t* recv_bytes, cudaStream_t st) override {
        if (failed_) comm_fail("communicator failed: " + why_);
        if (recv_bytes[r_] != send_bytes[r_]) fail("exchange sizes disagree on the rank itself");
        if (recv_bytes[r_])
            cuda_ok(cudaMemcpyAsync(static_cast<char*>(recv) + recv_off[r_],
                                    static_cast<const char*>(send) + send_off[r_], recv_bytes[r_],
                                    cudaMemcpyDeviceToDevice, st),
                    "exchange copy");
        check(api_.group_start(), "ncclGroupStart");
        for (int p = 0; p < n_; ++p) {
            if (p == r_) continue;
            if (send_bytes[p])
                check(api_.send(static_cast<const char*>(send) + send_off[p], send_bytes[p], ncclUint8, p, comm_, st),
                      "ncclSend");
            if (recv_bytes[p])
                check(api_.recv(static_cast<char*>(recv) + recv_off[p], recv_bytes[p], ncclUint8, p, comm_, st),
                      "ncclRecv");
        }
        ncclResult_t e = api_.group_end();
        if (e == ncclInProgress) wait_ready("ncclGroupEnd");
        else check(e, "ncclGroupEnd");
    }

    void allreduce_max_u64(unsigned long long* v, int n, cudaStream_t st) override {
        if (failed_) comm_fail("communicator failed: " + why_);
        ncclResult_t e = api_.all_reduce(v, v, (size_t)n, ncclUint64, ncclMax, comm_, st);
        if (e == ncclInProgress) wait_ready("ncclAllReduce");
        else check(e, "ncclAllReduce");
    }

    void sync(cudaStream_t st) override {
        const auto t0 = std::chrono::steady_clock::now();
        for (;;) {
            const cudaError_t q = cudaStreamQuery(st);
            if (q == cudaSuccess) return;
            if (q != cudaErrorNotReady) cuda_ok(q, "cudaStreamQuery");
            ncclResult_t ae = ncclSuccess;
            api_.async_error(comm_, &ae);
            if (ae != ncclSuccess && ae != ncclInProgress) nccl_fail(ae, "asynchronous NCCL error");
            if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > timeout_)
                fail("stream did not finish within " + std::to_string(timeout_) + " s");
            std::this_thread::sleep_for(std::chrono::microseconds(50));
        }
    }

    // ncclCommAbort ends the communicator's kernels still in flight
    void abort(const std::string& why) override {
        if (!failed_) {
            failed_ = true;
            why_ = why;
        }
        if (comm_) {
            api_.abort(comm_);
            comm_ = nullptr;
        }
    }

  private:
    [[noreturn]] void fail(const std::string& why) {
        abort(why);
        comm_fail("communicator failed: " + why_);
    }
    void check(ncclResult_t e, const char* what) {
        if (e != ncclSuccess) nccl_fail(e, what);
    }
    [[noreturn]] void nccl_fail(ncclResult_t e, const char* what) { fail(std::string(what) + ": " + api_.error_string(e)); }
    void wait_ready(const char* what) {
        const auto t0 = std::chrono::steady_clock::now();
        for (;;) {
            ncclResult_t ae = ncclSuccess;
            api_.async_error(comm_, &ae);
            if (ae == ncclSuccess) return;
            if (ae != ncclInProgress) nccl_fail(ae, what);
            if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > timeout_)
                fail(std::string(what) + " did not complete within " + std::to_string(timeout_) + " s");
            std::this_thread::sleep_for(std::chrono::microseconds(50));
        }
    }
    const NcclApi& api_;
    ncclComm_t comm_ = nullptr;
    int r_, n_;
    double timeout_;
    bool failed_ = false;
    std::string why_;
};
}  // namespace

std::vector<std::shared_ptr<Comm>> make_local_group(int n, double timeout_s) {
    if (n < 1) throw Error(FCB_ERR_INVALID, "a group needs at least one rank");
    if (!(timeout_s > 0.0)) throw Error(FCB_ERR_INVALID, "the time limit must be positive");
    auto g = std::make_shared<Group>();
    g->n = n;
    g->timeout = std::chrono::duration<double>(timeout_s);
    g->ready.assign(n, nullptr);
    g->done.assign(n, nullptr);
    g->post[0].resize(n);
    g->post[1].resize(n);
    std::vector<std::shared_ptr<Comm>> out;
    for (int r = 0; r < n; ++r) out.push_back(std::make_shared<LocalComm>(g, r));
    return out;
}

void nccl_unique_id(const char* library, unsigned char id[128]) {
    const NcclApi& api = nccl_api(library);
    ncclUniqueId uid;
    const ncclResult_t e = api.get_unique_id(&uid);
    if (e != ncclSuccess) comm_fail(std::string("ncclGetUniqueId: ") + api.error_string(e));
    std::memcpy(id, uid.internal, 128);
}

std::shared_ptr<Comm> make_nccl_comm(const char* library, const unsigned char id[128], int rank, int nranks,
                                     double timeout_s) {
    if (nranks < 1 || rank < 0 || rank >= nranks) throw Error(FCB_ERR_INVALID, "bad rank / number of ranks");
    if (!(timeout_s > 0.0)) throw Error(FCB_ERR_INVALID, "the time limit must be positive");
    return std::make_shared<NcclComm>(library, id, rank, nranks, timeout_s);
}

}  // namespace fcb
