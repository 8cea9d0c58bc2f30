// Mass sums that allocate nothing: fcb_conservation_sum_noalloc.
//
// Some callers cannot allocate device memory at the moment they want a mass
// diagnostic: a serving loop that has handed every byte of HBM to admitted
// solves under a fixed budget (an allocation could fail or overrun it), code
// that must not stall other streams (cudaMalloc and cudaFree can synchronise
// the device), and hosts that own all device memory through their own pool.
// This entry point takes the caller's patch arrays and output buffer and keeps
// its per-patch partial sums in the file-scope array below instead of in
// memory obtained at run time.
//
// The scratch array is sized for kMaxPatchSums = 262,144 per-patch partial sums
// (npatches * meqn), 2 MiB, and every GPU that loads this library holds it
// until the process exits.  All calls share it: two calls that overlap on the
// GPU (different streams, or different host threads) race on it and must be
// serialised by the caller.  Every entry a call reads is first written by the
// same call, so nothing in it has to start at zero and the previous call's
// contents never leak into a result.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/fclaw_b200.h"

namespace fcb {
void set_last_error(const std::string& msg);  // the message fcb_last_error() returns
}

namespace {

constexpr int kMaxPatchSums = 262144;
constexpr int kMaxDevices = 64;

// Per-patch Kahan partial sums, [patch][component].
static __device__ __align__(256) double g_patch_sums[kMaxPatchSums];

// Host-side device address of g_patch_sums for each device, found once per
// device with that device current.  The symbol's name in host code is only a
// stand-in and must never be handed to a kernel.  The address is kept for the
// life of the process: a cudaDeviceReset tears down the context that owns it,
// after which it would be stale, so a caller must not reset a device it has
// used this entry point on.
double* g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_setup_mutex;

// Kahan sum of q*area over the interior of each patch in the reference's loop
// order (fclaw2d_clawpatch46_diagnostics.f:13-58): component m, then j, then i.
__global__ void patch_sums_kernel(const double* __restrict__ q, size_t stride, int npatches, int mx, int my,
                                  int mbc, int meqn, const double* __restrict__ area, double* scratch) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npatches) return;
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc;
    const double* qp = q + (size_t)p * stride;
    const double a = area[p];
    for (int m = 0; m < meqn; ++m) {
        double sum = 0.0, c = 0.0;
        for (int j = 1; j <= my; ++j)
            for (int i = 1; i <= mx; ++i) {
                const double y = qp[((size_t)m * ny + j + mbc - 1) * nx + i + mbc - 1] * a - c;
                const double t = sum + y;
                c = (t - sum) - y;
                sum = t;
            }
        scratch[(size_t)p * meqn + m] = sum;
    }
}

// Kahan sum of the per-patch sums in patch order, one thread per component.
__global__ void combine_kernel(const double* scratch, int npatches, int meqn, double* sums) {
    const int m = threadIdx.x;
    if (m >= meqn) return;
    double s = 0.0, c = 0.0;
    for (int p = 0; p < npatches; ++p) {
        const double y = scratch[(size_t)p * meqn + m] - c;
        const double t = s + y;
        c = (t - s) - y;
        s = t;
    }
    sums[m] = s;
}

int fail(int code, const std::string& msg) {
    fcb::set_last_error(msg);
    return code;
}

// Once per device, with that device current: look up the device address of
// the scratch array.
int scratch_for_current_device(double** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(FCB_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(FCB_ERR_INVALID, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_patch_sums);
        if (e != cudaSuccess || p == nullptr)
            return fail(FCB_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_ptr[dev];
    return FCB_OK;
}

}  // namespace

extern "C" {

__attribute__((visibility("default"))) int fcb_conservation_sum_noalloc(const double* d_q, size_t patch_stride, int npatches, int mx, int my, int mbc,
                                 int meqn, const double* d_area, double* d_sums, void* cuda_stream) {
    if (!d_q || !d_area || !d_sums) return fail(FCB_ERR_INVALID, "null device pointer");
    if (npatches <= 0 || mx <= 0 || my <= 0 || mbc < 0 || meqn <= 0 || meqn > 1024)
        return fail(FCB_ERR_INVALID, "bad sizes");
    if (patch_stride < (size_t)meqn * (mx + 2 * mbc) * (my + 2 * mbc))
        return fail(FCB_ERR_INVALID, "patch_stride smaller than one patch");
    if ((long long)npatches * meqn > kMaxPatchSums)
        return fail(FCB_ERR_INVALID, "npatches * meqn = " + std::to_string((long long)npatches * meqn) +
                                         " exceeds the fixed scratch of " + std::to_string(kMaxPatchSums) +
                                         " per-patch sums; use fcb_conservation_check instead");
    double* scratch = nullptr;
    const int rc = scratch_for_current_device(&scratch);
    if (rc != FCB_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    patch_sums_kernel<<<(npatches + 127) / 128, 128, 0, st>>>(d_q, patch_stride, npatches, mx, my, mbc, meqn,
                                                                d_area, scratch);
    combine_kernel<<<1, 32 * ((meqn + 31) / 32), 0, st>>>(scratch, npatches, meqn, d_sums);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(FCB_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return FCB_OK;
}

}  // extern "C"
