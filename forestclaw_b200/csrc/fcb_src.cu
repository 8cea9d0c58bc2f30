// Source-term stage of clawpack46_update / clawpack5_update: src2 after the
// step when src_term > 0 (src/solvers/fc2d_clawpack4.6/fc2d_clawpack46.cpp:436-440,
// fc2d_clawpack5/fc2d_clawpack5.cpp:397-403).
//
// Source 1: the axisymmetric Euler source of euler/2d/shockbubble
// (user_4.6/src2.f, user_5.0/src2.f90, the same arithmetic): a two-stage
// Runge-Kutta step over the interior cells with the radius at the cell centre,
// rad = ylower + (j-0.5)*dy (shockbubble setaux.f stores exactly this in
// aux(i,j,1)); components 1-4 change, a tracer would not.  Compiled without
// FMA contraction; each expression keeps the Fortran association
// (a*b/c*d = ((a*b)/c)*d, (ndim-1) = 1 converted to double).
#include <cuda_runtime.h>

#include "fcb_device.h"

namespace fcb {

namespace {

__global__ void src2_axisymmetric_kernel(const StepArgs a, int mx, int my, int mbc, double gamma1) {
    const int pi = blockIdx.x;
    if (pi >= a.npatches) return;
    const int slot = a.slots[pi];
    const PatchMeta mt = a.meta[slot];
    const double dt = step_dt(a, mt.level);
    const double dt2 = dt / 2.0;
    const double ndim1 = 1.0;
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc;
    const int64_t plane = (int64_t)nx * ny;
    double* q = a.q + (int64_t)slot * a.q_stride;
    for (int k = threadIdx.x; k < mx * my; k += blockDim.x) {
        const int jj = k / mx, ii = k - jj * mx;  // 0-based interior indices: i = ii+1, j = jj+1
        const double rad = mt.ylower + ((jj + 1) - 0.5) * mt.dy;
        double* c = q + (int64_t)(jj + mbc) * nx + (ii + mbc);
        const double q1 = c[0], q2 = c[plane], q3 = c[2 * plane], q4 = c[3 * plane];
        double rho = q1;
        double u = q2 / q1;
        double v = q3 / q1;
        double press = gamma1 * (q4 - 0.5 * rho * (u * u + v * v));
        const double qs1 = q1 - dt2 * ndim1 / rad * q3;
        const double qs2 = q2 - dt2 * ndim1 / rad * (rho * u * v);
        const double qs3 = q3 - dt2 * ndim1 / rad * (rho * v * v);
        const double qs4 = q4 - dt2 * ndim1 / rad * v * (q4 + press);
        rho = qs1;
        u = qs2 / qs1;
        v = qs3 / qs1;
        press = gamma1 * (qs4 - 0.5 * rho * (u * u + v * v));
        c[0] = q1 - dt * ndim1 / rad * qs3;
        c[plane] = q2 - dt * ndim1 / rad * (rho * u * v);
        c[2 * plane] = q3 - dt * ndim1 / rad * (rho * v * v);
        c[3 * plane] = q4 - dt * ndim1 / rad * v * (qs4 + press);
    }
}

}  // namespace

// The source stage over the patches of one step launch (slots, levels and dt
// exactly as the step launch `a` had them).
cudaError_t launch_src2(int kind, const StepArgs& a, int mx, int my, int mbc, int meqn, cudaStream_t st) {
    if (a.npatches <= 0) return cudaSuccess;
    if (kind != 1 || meqn < 4 || a.desc) return cudaErrorInvalidValue;
    src2_axisymmetric_kernel<<<a.npatches, 256, 0, st>>>(a, mx, my, mbc, a.gamma1);
    return cudaGetLastError();
}

}  // namespace fcb
