// Ghost-cell fill kernels (copy / average / interpolate across faces and
// corners, physical boundary conditions) and time interpolation.
//
// A warp executes the records of one destination patch; a launch executes one "wave" of
// records that the host has proven independent (no record in a wave reads or
// writes cells another record of the same wave writes), so the result equals
// the reference's sequential order.
//
// References (clawpack 4.6 layout, same-block transforms):
//   copy:        src/patches/clawpatch/fort_4.6/fclaw2d_clawpatch46_copy.f:17-133
//   average:     fort_4.6/fclaw2d_clawpatch46_average.f:16-272
//   interpolate: fort_4.6/fclaw2d_clawpatch46_interpolate.f:30-314 (+ slopes,
//                fclaw2d_clawpatch_utils.f:11-66 with mth = 5)
//   physical BC: src/solvers/fc2d_clawpack4.6/fortran_source/clawpack46_bc2_default.f
//   time interp: fort_4.6/fclaw2d_clawpatch46_timeinterp.f:11-78
// Index transforms: src/forestclaw2d.c same-block branches; a copy maps
// (i,j) -> (i+dx, j+dy); a half-size map sends coarse (ic,jc) to the fine
// cells (2ic+dx+kx, 2jc+dy+ky), kx,ky in {0,1}.
#include <cuda_runtime.h>

#include "fcb_device.h"

namespace fcb {

namespace {

struct PatchView {
    double* p;
    int mx, my, mbc, nx, ny;
    __device__ __forceinline__ double& at(int i, int j, int m) const {
        return p[((int64_t)m * ny + (j + mbc - 1)) * nx + (i + mbc - 1)];
    }
};

// fclaw2d_clawpatch_compute_slopes, mth = 5 (SIGN(1,x) follows the sign bit).
template <typename R>
__device__ __forceinline__ R slope5(R sl, R sr) {
    const R sc = (sl + sr) / R(2);
    R m = 2 * fabs(sl);
    const R b = 2 * fabs(sr), cc = fabs(sc);
    if (b < m) m = b;
    if (cc < m) m = cc;
    const R s0 = copysign(R(1), sl * sr);
    return m * (s0 > R(0) ? s0 : R(0)) * copysign(R(1), sc);
}

// R = double: the reference's arithmetic; R = float: the mixed-precision form.
template <typename R>
__device__ __forceinline__ void interp_cell_t(const PatchView& C, const PatchView& F, int m, int ic, int jc,
                                              int i20, int j20) {
    const R qc = R(C.at(ic, jc, m));
    R sl = (qc - R(C.at(ic - 1, jc, m)));
    R sr = (R(C.at(ic + 1, jc, m)) - qc);
    const R gradx = slope5(sl, sr);
    sl = (qc - R(C.at(ic, jc - 1, m)));
    sr = (R(C.at(ic, jc + 1, m)) - qc);
    const R grady = slope5(sl, sr);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int ii = k & 1, jj = k >> 1;
        const R shiftx = (ii - R(0.5)) / R(2);
        const R shifty = (jj - R(0.5)) / R(2);
        F.at(i20 + ii, j20 + jj, m) = double(qc + gradx * shiftx + grady * shifty);
    }
}

__device__ __forceinline__ void interp_cell(bool fp32, const PatchView& C, const PatchView& F, int m, int ic,
                                            int jc, int i20, int j20) {
    if (fp32) interp_cell_t<float>(C, F, m, ic, jc, i20, j20);
    else interp_cell_t<double>(C, F, m, ic, jc, i20, j20);
}

// Patch shape of a launch: MXC > 0 fixes mx = my = MXC and mbc = 2 at compile
// time (index decoding by constant division), MXC == 0 reads the arguments.
template <int MXC>
__device__ __forceinline__ int gmx(const GhostArgs& a) { return MXC > 0 ? MXC : a.mx; }
template <int MXC>
__device__ __forceinline__ int gmy(const GhostArgs& a) { return MXC > 0 ? MXC : a.my; }
template <int MXC>
__device__ __forceinline__ int gmbc(const GhostArgs& a) { return MXC > 0 ? 2 : a.mbc; }

}  // namespace

// A physical-boundary record (clawpack46_bc2_default.f) executed by the 32
// lanes of a warp: its sides run in the reference's order, each reading cells
// the previous side may have written.  Every other record type goes through
// op_cell below.
template <int MXC>
__device__ __forceinline__ void physbc_op(const GhostArgs& a, const GhostOp& op, int lane) {
    const int mx = gmx<MXC>(a), my = gmy<MXC>(a), mbc = gmbc<MXC>(a), meqn = a.meqn;
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc;
    PatchView D{(op.dst_ti ? a.qti : a.q) + (int64_t)op.dst * a.stride, mx, my, mbc, nx, ny};
    for (int side = 0; side < 4; ++side) {
        const int mth = op.mthbc[side];
        if (mth == 1 || mth == 3) {
            const bool xside = side < 2;
            const int len = xside ? ny : nx;
            const int n = meqn * mbc * len;
            for (int k = lane; k < n; k += 32) {
                const int m = k / (mbc * len), rem = k - m * mbc * len;
                const int bc = rem / len + 1, t = rem % len + (1 - mbc);
                if (side == 0) {
                    double v = (mth == 1) ? D.at(1, t, m) : D.at(bc, t, m);
                    if (mth == 3 && m == 1) v = -v;
                    D.at(1 - bc, t, m) = v;
                } else if (side == 1) {
                    double v = (mth == 1) ? D.at(mx, t, m) : D.at(mx + 1 - bc, t, m);
                    if (mth == 3 && m == 1) v = -v;
                    D.at(mx + bc, t, m) = v;
                } else if (side == 2) {
                    double v = (mth == 1) ? D.at(t, 1, m) : D.at(t, bc, m);
                    if (mth == 3 && m == 2) v = -v;
                    D.at(t, 1 - bc, m) = v;
                } else {
                    double v = (mth == 1) ? D.at(t, my, m) : D.at(t, my + 1 - bc, m);
                    if (mth == 3 && m == 2) v = -v;
                    D.at(t, my + bc, m) = v;
                }
            }
        }
        __syncwarp();
    }
}

// Number of cells one lane-level work item of a record covers (0 for the
// physical-boundary record, which keeps its whole-warp form: its sides read
// cells that the previous side writes).
template <int MXC>
__device__ __forceinline__ int op_cells(const GhostArgs& a, const GhostOp& op) {
    const int mx = gmx<MXC>(a), my = gmy<MXC>(a), mbc = gmbc<MXC>(a), meqn = a.meqn;
    switch (op.type) {
        case OP_COPY_FACE: return (op.face < 2 ? mbc * my : mx * mbc) * meqn;
        case OP_COPY_CORNER:
        case OP_AVERAGE_CORNER: return mbc * mbc * meqn;
        case OP_AVERAGE_FACE: return (op.face < 2 ? my : mx) * mbc * meqn;
        case OP_INTERP_FACE: return mx * (mbc / 2) * meqn;
        case OP_INTERP_CORNER: return (mbc / 2) * (mbc / 2) * meqn;
        default: return 0;
    }
}

// Work item k of a record.  Copy
// and average items return their value and destination so the caller can
// issue several loads before the stores; interpolation items store their four
// fine cells themselves and return nullptr.
template <int MXC>
__device__ __forceinline__ double* op_cell(const GhostArgs& a, const GhostOp& op, int k, double& v) {
    const int mx = gmx<MXC>(a), my = gmy<MXC>(a), mbc = gmbc<MXC>(a);
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc;
    PatchView D{(op.dst_ti ? a.qti : a.q) + (int64_t)op.dst * a.stride, mx, my, mbc, nx, ny};
    PatchView S{(op.src_ti ? a.qti : a.q) + (int64_t)op.src * a.stride, mx, my, mbc, nx, ny};
    switch (op.type) {
        case OP_COPY_FACE: {
            int i0, j0, w, h;
            if (op.face == 0) { i0 = 1 - mbc; j0 = 1; w = mbc; h = my; }
            else if (op.face == 1) { i0 = mx + 1; j0 = 1; w = mbc; h = my; }
            else if (op.face == 2) { i0 = 1; j0 = 1 - mbc; w = mx; h = mbc; }
            else { i0 = 1; j0 = my + 1; w = mx; h = mbc; }
            const int m = k / (w * h), rem = k - m * w * h, jj = rem / w, ii = rem - jj * w;
            const int i = i0 + ii, j = j0 + jj;
            v = S.at(i + op.dx, j + op.dy, m);
            return &D.at(i, j, m);
        }
        case OP_COPY_CORNER:
        case OP_AVERAGE_CORNER: {
            const int m = k / (mbc * mbc), rem = k - m * mbc * mbc;
            const int ibc = rem / mbc + 1, jbc = rem % mbc + 1;
            int i1, j1;
            if (op.face == 0) { i1 = 1 - ibc; j1 = 1 - jbc; }
            else if (op.face == 1) { i1 = mx + ibc; j1 = 1 - jbc; }
            else if (op.face == 2) { i1 = 1 - ibc; j1 = my + jbc; }
            else { i1 = mx + ibc; j1 = my + jbc; }
            if (op.type == OP_COPY_CORNER) {
                v = S.at(i1 + op.dx, j1 + op.dy, m);
            } else {
                const int fi = 2 * i1 + op.dx, fj = 2 * j1 + op.dy;
                double sum = 0;
                sum = sum + S.at(fi, fj, m);
                sum = sum + S.at(fi + 1, fj, m);
                sum = sum + S.at(fi, fj + 1, m);
                sum = sum + S.at(fi + 1, fj + 1, m);
                v = sum / 4.0;
            }
            return &D.at(i1, j1, m);
        }
        case OP_AVERAGE_FACE: {
            const int idir = op.face / 2;
            const int along = idir == 0 ? my : mx;
            const int m = k / (along * mbc), rem = k - m * along * mbc;
            const int t = rem / mbc + 1, bc = rem % mbc + 1;
            int ic, jc;
            if (idir == 0) { jc = t; ic = (op.face == 0) ? 1 - bc : mx + bc; }
            else { ic = t; jc = (op.face == 2) ? 1 - bc : my + bc; }
            const int fi = 2 * ic + op.dx, fj = 2 * jc + op.dy;
            if (fi < 1 || fi + 1 > mx || fj < 1 || fj + 1 > my) return nullptr;  // is_valid_average
            double sum = 0;
            sum = sum + S.at(fi, fj, m);
            sum = sum + S.at(fi + 1, fj, m);
            sum = sum + S.at(fi, fj + 1, m);
            sum = sum + S.at(fi + 1, fj + 1, m);
            v = sum / 4.0;
            return &D.at(ic, jc, m);
        }
        case OP_INTERP_FACE: {
            const int idir = op.face / 2;
            const int nb = mbc / 2;
            const int along = mx;  // the reference loops jc = 1..mx for idir = 0 as well
            const int m = k / (along * nb), rem = k - m * along * nb;
            const int t = rem / nb + 1, b = rem % nb + 1;
            int ic, jc;
            if (idir == 0) { jc = t; ic = (op.face == 0) ? b : mx - b + 1; }
            else { ic = t; jc = (op.face == 2) ? b : my - b + 1; }
            const int fi = 2 * ic + op.dx, fj = 2 * jc + op.dy;
            if (fi < 1 - mbc || fi + 1 > mx + mbc || fj < 1 - mbc || fj + 1 > my + mbc) return nullptr;
            interp_cell(a.interp_fp32 != 0, S, D, m, ic, jc, fi, fj);
            return nullptr;
        }
        case OP_INTERP_CORNER: {
            const int nb = mbc / 2;
            const int m = k / (nb * nb), rem = k - m * nb * nb;
            const int ibc = rem / nb + 1, jbc = rem % nb + 1;
            int ic, jc;
            if (op.face == 0) { ic = ibc; jc = jbc; }
            else if (op.face == 1) { ic = mx - ibc + 1; jc = jbc; }
            else if (op.face == 2) { ic = ibc; jc = my - jbc + 1; }
            else { ic = mx - ibc + 1; jc = my - jbc + 1; }
            interp_cell(a.interp_fp32 != 0, S, D, m, ic, jc, 2 * ic + op.dx, 2 * jc + op.dy);
            return nullptr;
        }
        default: return nullptr;
    }
}

// One warp per group.  The records of a group share their destination patch;
// the host proved every record of a wave independent of the others (none reads
// or writes a cell another writes), so their work items may run in any order:
// the warp lays the items of up to 32 records out in one flat index range
// (prefix sum of op_cells over the lanes) and each lane takes items lane,
// lane+32, ...  UNROLL items per lane issue their loads before any store.
constexpr int GHOST_TPB = 256;
template <int GHOST_UNROLL, int MXC>
__global__ void __launch_bounds__(GHOST_TPB) ghost_wave_kernel(const GhostArgs a) {
    __shared__ GhostOp s_ops[GHOST_TPB / 32][32];
    __shared__ int s_end[GHOST_TPB / 32][32];
    const int wl = threadIdx.x >> 5;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= a.ngroups) return;
    const int b = a.groups[warp], e = a.groups[warp + 1];
    for (int base = b; base < e; base += 32) {
        const int cnt = min(32, e - base);
        int n = 0;
        bool phys = false;
        if (lane < cnt) {
            const GhostOp op = a.ops[base + lane];
            s_ops[wl][lane] = op;
            phys = op.type == OP_PHYSBC;
            n = op_cells<MXC>(a, op);
        }
        int incl = n;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        s_end[wl][lane] = incl;
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        __syncwarp();
        int r = 0;  // record of the current item; items are visited in increasing order
        for (int f0 = lane; f0 < total; f0 += 32 * GHOST_UNROLL) {
            double v[GHOST_UNROLL];
            double* dst[GHOST_UNROLL];
#pragma unroll
            for (int u = 0; u < GHOST_UNROLL; ++u) {
                const int f = f0 + 32 * u;
                dst[u] = nullptr;
                v[u] = 0.0;
                if (f < total) {
                    while (f >= s_end[wl][r]) ++r;
                    const int first = r > 0 ? s_end[wl][r - 1] : 0;
                    dst[u] = op_cell<MXC>(a, s_ops[wl][r], f - first, v[u]);
                }
            }
#pragma unroll
            for (int u = 0; u < GHOST_UNROLL; ++u)
                if (dst[u]) *dst[u] = v[u];
        }
        // physical-boundary records (independent of the items above)
        unsigned pm = __ballot_sync(0xffffffffu, phys);
        while (pm) {
            const int l = __ffs(pm) - 1;
            pm &= pm - 1;
            physbc_op<MXC>(a, s_ops[wl][l], lane);
        }
        __syncwarp();
    }
}

// unroll: work items per lane whose loads are issued before the stores (2, 4
// or 8; the autotuner picks one per patch shape)
namespace {
template <int MXC>
void launch_ghost_shape(const GhostArgs& a, cudaStream_t st, int unroll, int blocks) {
    switch (unroll) {
        case 2: ghost_wave_kernel<2, MXC><<<blocks, GHOST_TPB, 0, st>>>(a); break;
        case 8: ghost_wave_kernel<8, MXC><<<blocks, GHOST_TPB, 0, st>>>(a); break;
        default: ghost_wave_kernel<4, MXC><<<blocks, GHOST_TPB, 0, st>>>(a); break;
    }
}
}  // namespace

cudaError_t launch_ghost_wave(const GhostArgs& a, cudaStream_t st, int unroll) {
    if (a.ngroups <= 0) return cudaSuccess;
    const int blocks = (int)(((int64_t)a.ngroups * 32 + GHOST_TPB - 1) / GHOST_TPB);
    const int shape = (a.mbc == 2 && a.mx == a.my) ? a.mx : 0;
    switch (shape) {
        case 8: launch_ghost_shape<8>(a, st, unroll, blocks); break;
        case 16: launch_ghost_shape<16>(a, st, unroll, blocks); break;
        case 32: launch_ghost_shape<32>(a, st, unroll, blocks); break;
        case 64: launch_ghost_shape<64>(a, st, unroll, blocks); break;
        default: launch_ghost_shape<0>(a, st, unroll, blocks); break;
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Time interpolation on the interior band of width mbc (the four strips in the
// reference's order; every strip cell is written once, so order is free).
// ---------------------------------------------------------------------------
__global__ void timeinterp_kernel(double* q, const double* qlast, double* qti, int64_t stride,
                                  const int32_t* slots, int n, int mx, int my, int mbc, int meqn,
                                  double alpha) {
    const int p = blockIdx.x;
    if (p >= n) return;
    const int64_t base = (int64_t)slots[p] * stride;
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc;
    const int mint = mbc;
    const int total = meqn * mx * my;
    for (int k = threadIdx.x; k < total; k += blockDim.x) {
        const int m = k / (mx * my), rem = k - m * mx * my;
        const int j = rem / mx + 1, i = rem % mx + 1;
        const bool in_band = (i <= mint) || (i > mx - mint) || (j <= mint) || (j > my - mint);
        if (!in_band) continue;
        const int64_t idx = base + ((int64_t)m * ny + (j + mbc - 1)) * nx + (i + mbc - 1);
        qti[idx] = qlast[idx] + alpha * (q[idx] - qlast[idx]);
    }
}

cudaError_t launch_timeinterp(double* q, const double* qlast, double* qti, int64_t stride,
                              const int32_t* slots, int n, int mx, int my, int mbc, int meqn,
                              double alpha, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    timeinterp_kernel<<<n, 128, 0, st>>>(q, qlast, qti, stride, slots, n, mx, my, mbc, meqn, alpha);
    return cudaGetLastError();
}

}  // namespace fcb
