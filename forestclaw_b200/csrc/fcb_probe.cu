// Floating-point issue rate of this GPU, for roofline reports beside the HBM
// one (no counterpart in the reference).  Every thread of one full wave of
// resident CTAs runs CHAINS independent multiply-then-add chains; each step is
// one multiply and one add instruction (explicitly rounded, never contracted to
// an FMA), the instruction mix of the patch step compiled without contraction.
// The rate is lane operations per second: one add or multiply of one thread.
#include <cuda_runtime.h>

#include <algorithm>

#include "fcb_runtime.hpp"

namespace fcb {
namespace {

constexpr int CHAINS = 8;
constexpr int ITERS = 4096;
constexpr int TPB = 256;

template <typename T>
__device__ __forceinline__ T mul_rn(T a, T b);
template <>
__device__ __forceinline__ double mul_rn<double>(double a, double b) { return __dmul_rn(a, b); }
template <>
__device__ __forceinline__ float mul_rn<float>(float a, float b) { return __fmul_rn(a, b); }
template <typename T>
__device__ __forceinline__ T add_rn(T a, T b);
template <>
__device__ __forceinline__ double add_rn<double>(double a, double b) { return __dadd_rn(a, b); }
template <>
__device__ __forceinline__ float add_rn<float>(float a, float b) { return __fadd_rn(a, b); }

template <typename T>
__global__ void __launch_bounds__(TPB) rate_kernel(T a, T b, T* out) {
    T x[CHAINS];
#pragma unroll
    for (int k = 0; k < CHAINS; ++k) x[k] = T(threadIdx.x) * T(1e-3) + T(k);
#pragma unroll 4
    for (int it = 0; it < ITERS; ++it) {
#pragma unroll
        for (int k = 0; k < CHAINS; ++k) x[k] = add_rn(mul_rn(x[k], a), b);
    }
    T s = T(0);
#pragma unroll
    for (int k = 0; k < CHAINS; ++k) s += x[k];
    out[(size_t)blockIdx.x * TPB + threadIdx.x] = s;
}

template <typename T>
cudaError_t measure(cudaStream_t st, double* rate) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rate_kernel<T>, TPB, 0);
    if (e != cudaSuccess) return e;
    const int blocks = sms * std::max(1, per_sm);
    T* out = nullptr;
    e = cudaMalloc(&out, (size_t)blocks * TPB * sizeof(T));
    if (e != cudaSuccess) return e;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const T a = T(0.999999), b = T(1e-6);
    float best = 1e30f;
    rate_kernel<T><<<blocks, TPB, 0, st>>>(a, b, out);  // warm-up
    for (int r = 0; r < 5 && e == cudaSuccess; ++r) {
        cudaEventRecord(e0, st);
        rate_kernel<T><<<blocks, TPB, 0, st>>>(a, b, out);
        cudaEventRecord(e1, st);
        e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        best = std::min(best, ms);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e == cudaSuccess) *rate = (double)blocks * TPB * ITERS * CHAINS * 2.0 / (best * 1e-3);
    return e;
}

}  // namespace

cudaError_t measure_fp_rate(bool fp64, cudaStream_t st, double* ops_per_second) {
    *ops_per_second = 0.0;
    return fp64 ? measure<double>(st, ops_per_second) : measure<float>(st, ops_per_second);
}

}  // namespace fcb
