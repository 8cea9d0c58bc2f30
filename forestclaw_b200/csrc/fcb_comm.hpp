// Communicators of a partitioned solve.  They carry the three collective steps
// of the reference's parallel path on device buffers, in stream order:
//   * the ghost-patch exchange (fclaw2d_exchange.c:308-413) and the patch
//     transfer after a repartition (fclaw2d_partition.c:113-197): alltoallv of
//     byte ranges;
//   * fclaw2d_domain_global_maximum (forestclaw2d.c:51) for the CFL number and
//     the gathered refinement tags: allreduce_max_u64 / alltoallv.
// Every rank makes the same calls in the same order.  Two implementations:
//   * LocalGroup: the ranks are contexts of one process, each driven by its own
//     host thread; data moves by device-to-device copies ordered by CUDA events,
//     and the ranks meet at host barriers with a time limit (no kernel ever
//     waits for another rank);
//   * NCCL (one process per GPU): grouped ncclSend/ncclRecv and ncclAllReduce
//     from the library loaded at run time, non-blocking communicator, every
//     wait bounded, a communicator that runs out of time is aborted.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <memory>
#include <string>
#include <vector>

namespace fcb {

class Comm {
  public:
    virtual ~Comm() = default;
    virtual int rank() const = 0;
    virtual int size() const = 0;
    // Sends send_bytes[p] bytes at send + send_off[p] to every rank p and
    // receives recv_bytes[p] bytes at recv + recv_off[p] from every rank p
    // (device memory, p = 0..size()-1, the rank itself included).
    virtual void alltoallv(const void* send, const size_t* send_off, const size_t* send_bytes, void* recv,
                           const size_t* recv_off, const size_t* recv_bytes, cudaStream_t st) = 0;
    // v[k] = max over ranks of v[k] for n unsigned 64-bit words in device memory
    // (the bit patterns of non-negative doubles order like the doubles).
    virtual void allreduce_max_u64(unsigned long long* v, int n, cudaStream_t st) = 0;
    // Waits for the stream; throws (and aborts the communicator) after the time limit.
    virtual void sync(cudaStream_t st) = 0;
    // Marks the communicator failed: every rank's next collective throws at once.
    virtual void abort(const std::string& why) = 0;
};

// n handles of one in-process group (timeout_s: limit of every host rendezvous).
std::vector<std::shared_ptr<Comm>> make_local_group(int n, double timeout_s);
// NCCL: unique id of a new communicator (128 bytes), and rank `rank` of it.
void nccl_unique_id(const char* library, unsigned char id[128]);
std::shared_ptr<Comm> make_nccl_comm(const char* library, const unsigned char id[128], int rank, int nranks,
                                     double timeout_s);

// In place: v[k] = max_r words[r * n + k], r < nranks (fcb_comm.cu).
cudaError_t launch_max_words(unsigned long long* v, const unsigned long long* words, int n, int nranks,
                             cudaStream_t st);
// items[k] = slot * 2 + array (0 q, 1 time-interpolated q): pack == true copies
// the psize doubles of each item into buf[k * psize]; false copies them back.
cudaError_t launch_pack_patches(double* q, double* qti, int64_t stride, const int32_t* items, int n, int64_t psize,
                                double* buf, bool pack, cudaStream_t st);

}  // namespace fcb
