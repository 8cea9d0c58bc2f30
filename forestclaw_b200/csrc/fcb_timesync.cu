// Conservative time synchronisation on the device (the reference's
// time-sync = T path for the clawpack 4.6 shallow-water solver):
//
//   * before a level update, f(q) of the cells on both sides of every patch
//     face is accumulated into the face's edge-flux registers
//     (clawpack46_time_sync.f:37-157, clawpack46_time_sync_store_flux, with
//     shallow/2d/radialdam/rpn2cons_update.f);
//   * the boundary fluctuations fp, fm, gp, gm are accumulated by the step
//     kernel itself (fcb_step.cu, clawpack46_time_sync_accumulate_waves);
//   * at each synchronisation the same-size and fine-to-coarse corrections and
//     the register resets run as records, one CTA per patch, the records of a
//     patch in the reference's order (clawpack46_fort_time_sync_samesize,
//     clawpack46_fort_time_sync_f2c, fclaw2d_clawpatch_time_sync_reset).
//
// One block: every transform is a shift (same size) or a shift of the doubled
// index (half size) and the normal sign factors are 1.  Compiled without FMA
// contraction, so every correction rounds as the reference's.
#include <cuda_runtime.h>

#include "fcb_device.h"

namespace fcb {

namespace {

constexpr int TS_TPB = 128;

// rpn2_cons_update (shallow/2d/radialdam/rpn2cons_update.f)
__device__ __forceinline__ void swe_cons_flux(int idir, const double* q, double grav, double* flux) {
    const int mu = (idir == 0) ? 1 : 2;
    const int mv = (idir == 0) ? 2 : 1;
    const double hun = q[mu], hut = q[mv], h = q[0];
    const double un = hun / h;
    flux[0] = hun;
    flux[mu] = (hun * hun) / h + (0.5 * grav) * (h * h);
    flux[mv] = un * hut;
}

// One CTA per patch; thread k handles (face, cell, side) items.
__global__ void __launch_bounds__(TS_TPB) store_flux_kernel(const StepArgs a, int mx, int my, int mbc, int meqn) {
    const int pi = blockIdx.x;
    if (pi >= a.npatches) return;
    const int slot = a.slots[pi];
    const PatchMeta mt = a.meta[slot];
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc;
    const double* q = a.q + (int64_t)slot * a.q_stride;
    double* R = a.treg + (int64_t)slot * a.treg_stride;
    const RegLayout L{mx, my, meqn};
    const double dt = step_dt(a, mt.level);
    const int nitems = 2 * 2 * my + 2 * 2 * mx;  // faces 0, 1 (my cells) and 2, 3 (mx cells), two sides each
    for (int it = threadIdx.x; it < nitems; it += blockDim.x) {
        int face, cell, k;
        if (it < 4 * my) {
            face = it / (2 * my);
            const int r = it - face * 2 * my;
            cell = r >> 1;
            k = r & 1;
        } else {
            const int t = it - 4 * my;
            face = 2 + t / (2 * mx);
            const int r = t - (face - 2) * 2 * mx;
            cell = r >> 1;
            k = r & 1;
        }
        // Fortran cell of the item: face 0 -> (1-k, j), 1 -> (mx+k, j), 2 -> (i, 1-k), 3 -> (i, my+k)
        int i, j;
        if (face == 0) { i = 1 - k; j = cell + 1; }
        else if (face == 1) { i = mx + k; j = cell + 1; }
        else if (face == 2) { i = cell + 1; j = 1 - k; }
        else { i = cell + 1; j = my + k; }
        const int c = i + mbc - 1, r = j + mbc - 1;
        double qv[3], fl[3];
        for (int m = 0; m < 3; ++m) qv[m] = q[((int64_t)m * ny + r) * nx + c];
        swe_cons_flux(face / 2, qv, a.grav, fl);
        const double el = face < 2 ? mt.dy : mt.dx;  // edge lengths without a mapping
        const int len = face < 2 ? my : mx;
        for (int m = 0; m < meqn; ++m) {
            double& e = R[L.ef(face) + cell + len * (m + meqn * k)];
            e = e + (dt * el) * fl[m];
        }
    }
}

__device__ __forceinline__ double qat(const double* q, int nx, int ny, int mbc, int i, int j, int m) {
    return q[((int64_t)m * ny + (j + mbc - 1)) * nx + (i + mbc - 1)];
}

// qthis_dummy of clawpack46_fort_time_sync_samesize: the neighbour's registers
// placed one and two cells outside its own faces.
__device__ double dummy_same(const double* Rn, const RegLayout& L, int mx, int my, int i, int j, int m) {
    const int meqn = L.meqn;
    if (j >= 1 && j <= my) {
        const int k = (j - 1) + my * m;
        if (i == 0) return Rn[L.fm(0) + k];
        if (i == -1) return Rn[L.ef(0) + k + my * meqn];
        if (i == mx + 1) return Rn[L.fp(1) + k];
        if (i == mx + 2) return Rn[L.ef(1) + k + my * meqn];
    }
    if (i >= 1 && i <= mx) {
        const int k = (i - 1) + mx * m;
        if (j == 0) return Rn[L.gm(0) + k];
        if (j == -1) return Rn[L.ef(2) + k + mx * meqn];
        if (j == my + 1) return Rn[L.gp(1) + k];
        if (j == my + 2) return Rn[L.ef(3) + k + mx * meqn];
    }
    return 0.0;
}

// qfine_dummy of clawpack46_fort_time_sync_f2c: the fine patch's registers
// summed over pairs of fine edge cells, two cells deep outside each face, and
// the edge fluxes two further cells out.
__device__ double dummy_fine(const double* Rf, const RegLayout& L, int mx, int my, int i, int j, int m) {
    const int meqn = L.meqn;
    if (j >= 1 && j <= my) {
        const int j1 = ((j - 1) & ~1), k1 = j1 + my * m, k2 = k1 + 1;
        if (i == -1 || i == 0) return Rf[L.fm(0) + k1] + Rf[L.fm(0) + k2];
        if (i == -3 || i == -2) return Rf[L.ef(0) + k1 + my * meqn] + Rf[L.ef(0) + k2 + my * meqn];
        if (i == mx + 1 || i == mx + 2) return Rf[L.fp(1) + k1] + Rf[L.fp(1) + k2];
        if (i == mx + 3 || i == mx + 4) return Rf[L.ef(1) + k1 + my * meqn] + Rf[L.ef(1) + k2 + my * meqn];
    }
    if (i >= 1 && i <= mx) {
        const int i1 = ((i - 1) & ~1), k1 = i1 + mx * m, k2 = k1 + 1;
        if (j == -1 || j == 0) return Rf[L.gm(0) + k1] + Rf[L.gm(0) + k2];
        if (j == -3 || j == -2) return Rf[L.ef(2) + k1 + mx * meqn] + Rf[L.ef(2) + k2 + mx * meqn];
        if (j == my + 1 || j == my + 2) return Rf[L.gp(1) + k1] + Rf[L.gp(1) + k2];
        if (j == my + 3 || j == my + 4) return Rf[L.ef(3) + k1 + mx * meqn] + Rf[L.ef(3) + k2 + mx * meqn];
    }
    return 0.0;
}

// fc46_skip_this_grid: skip unless each of the four fine cells lies inside the
// fine patch in exactly one direction
__device__ __forceinline__ bool skip_grid(int di, int dj, int mx, int my) {
    for (int ky = 0; ky < 2; ++ky)
        for (int kx = 0; kx < 2; ++kx) {
            const bool iv = 1 <= di + kx && di + kx <= mx, jv = 1 <= dj + ky && dj + ky <= my;
            if (iv == jv) return true;
        }
    return false;
}

__device__ void apply_samesize(const TsArgs& a, const TsOp& o) {
    const int mx = a.mx, my = a.my, mbc = a.mbc, meqn = a.meqn;
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc;
    const RegLayout L{mx, my, meqn};
    const double* Rt = a.treg + (int64_t)o.slot * a.treg_stride;
    const double* Rn = a.treg + (int64_t)o.nbr * a.treg_stride;
    double* q = a.q + (int64_t)o.slot * a.q_stride;
    const PatchMeta mt = a.meta[o.slot];
    const double area = mt.dx * mt.dy;
    const int len = o.face < 2 ? my : mx;
    for (int it = threadIdx.x; it < len * meqn; it += blockDim.x) {
        const int m = it / len, cell = it - m * len;
        double delta;
        int i1, j1;
        if (o.face == 0) {
            i1 = 1; j1 = cell + 1;
            const int k = cell + my * m;
            const double fpv = dummy_same(Rn, L, mx, my, i1 + o.dx, j1 + o.dy, m);
            const double ef = dummy_same(Rn, L, mx, my, i1 + 1 + o.dx, j1 + o.dy, m);
            delta = (ef - Rt[L.ef(0) + k]) - (fpv - Rt[L.fp(0) + k]);
        } else if (o.face == 1) {
            i1 = mx; j1 = cell + 1;
            const int k = cell + my * m;
            const double fmv = dummy_same(Rn, L, mx, my, i1 + o.dx, j1 + o.dy, m);
            const double ef = dummy_same(Rn, L, mx, my, i1 - 1 + o.dx, j1 + o.dy, m);
            delta = (Rt[L.ef(1) + k] - ef) - (fmv - Rt[L.fm(1) + k]);
        } else if (o.face == 2) {
            i1 = cell + 1; j1 = 1;
            const int k = cell + mx * m;
            const double gpv = dummy_same(Rn, L, mx, my, i1 + o.dx, j1 + o.dy, m);
            const double ef = dummy_same(Rn, L, mx, my, i1 + o.dx, j1 + 1 + o.dy, m);
            delta = (ef - Rt[L.ef(2) + k]) - (gpv - Rt[L.gp(0) + k]);
        } else {
            i1 = cell + 1; j1 = my;
            const int k = cell + mx * m;
            const double gmv = dummy_same(Rn, L, mx, my, i1 + o.dx, j1 + o.dy, m);
            const double ef = dummy_same(Rn, L, mx, my, i1 + o.dx, j1 - 1 + o.dy, m);
            delta = (Rt[L.ef(3) + k] - ef) - (gmv - Rt[L.gm(1) + k]);
        }
        double& qv = q[((int64_t)m * ny + (j1 + mbc - 1)) * nx + (i1 + mbc - 1)];
        qv = qv + (0.5 * delta) / area;
    }
}

__device__ void apply_f2c(const TsArgs& a, const TsOp& o) {
    const int mx = a.mx, my = a.my, mbc = a.mbc, meqn = a.meqn;
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc;
    const RegLayout L{mx, my, meqn};
    const double* Rc = a.treg + (int64_t)o.slot * a.treg_stride;
    const double* Rf = a.treg + (int64_t)o.nbr * a.treg_stride;
    double* q = a.q + (int64_t)o.slot * a.q_stride;
    const PatchMeta mt = a.meta[o.slot];
    const double areac = mt.dx * mt.dy;
    const int len = o.face < 2 ? my : mx;
    for (int it = threadIdx.x; it < len * meqn; it += blockDim.x) {
        const int m = it / len, cell = it - m * len;
        int ic, jc;
        double deltac = 0;
        if (o.face < 2) {
            jc = cell + 1;
            ic = o.face == 0 ? 1 : mx;
            // fclaw2d_clawpatch_transform_face_half: first fine index 1 + D + 2*(c-1)
            const int di = 1 + o.dx + 2 * (ic - 1), dj = 1 + o.dy + 2 * (jc - 1);
            if (!skip_grid(di, dj, mx, my)) {
                const int k = cell + my * m;
                const double v = dummy_fine(Rf, L, mx, my, di, dj, m);
                if (o.face == 0) {
                    const double ef = dummy_fine(Rf, L, mx, my, di + 2, dj, m);
                    deltac = (ef - Rc[L.ef(0) + k]) - (v - Rc[L.fp(0) + k]);
                } else {
                    const double ef = dummy_fine(Rf, L, mx, my, di - 2, dj, m);
                    deltac = (Rc[L.ef(1) + k] - ef) - (v - Rc[L.fm(1) + k]);
                }
            }
        } else {
            ic = cell + 1;
            jc = o.face == 2 ? 1 : my;
            const int di = 1 + o.dx + 2 * (ic - 1), dj = 1 + o.dy + 2 * (jc - 1);
            if (!skip_grid(di, dj, mx, my)) {
                const int k = cell + mx * m;
                const double v = dummy_fine(Rf, L, mx, my, di, dj, m);
                if (o.face == 2) {
                    const double ef = dummy_fine(Rf, L, mx, my, di, dj + 2, m);
                    deltac = (ef - Rc[L.ef(2) + k]) - (v - Rc[L.gp(0) + k]);
                } else {
                    const double ef = dummy_fine(Rf, L, mx, my, di, dj - 2, m);
                    deltac = (Rc[L.ef(3) + k] - ef) - (v - Rc[L.gm(1) + k]);
                }
            }
        }
        double& qv = q[((int64_t)m * ny + (jc + mbc - 1)) * nx + (ic + mbc - 1)];
        qv = qv + deltac / areac;
    }
}

__device__ void apply_reset(const TsArgs& a, const TsOp& o) {
    const RegLayout L{a.mx, a.my, a.meqn};
    double* R = a.treg + (int64_t)o.slot * a.treg_stride;
    const int f = o.face;
    const int n = f < 2 ? L.ny() : L.nx();
    double* fpb = R + (f < 2 ? L.fp(f) : L.gp(f - 2));
    double* fmb = R + (f < 2 ? L.fm(f) : L.gm(f - 2));
    double* efb = R + L.ef(f);
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        fpb[k] = 0.0;
        fmb[k] = 0.0;
        efb[k] = 0.0;
        efb[k + n] = 0.0;
    }
}

// One CTA per patch group; its records in order, a barrier between records
// (consecutive records may update the same corner cell).
__global__ void __launch_bounds__(TS_TPB) ts_apply_kernel(const TsArgs a) {
    const int g = blockIdx.x;
    if (g >= a.ngroups) return;
    const int b = a.groups[g], e = a.groups[g + 1];
    for (int k = b; k < e; ++k) {
        const TsOp o = a.ops[k];
        if (o.type == TS_SAMESIZE) apply_samesize(a, o);
        else if (o.type == TS_F2C) apply_f2c(a, o);
        else apply_reset(a, o);
        __syncthreads();
    }
}

__global__ void zero_registers_kernel(double* treg, int64_t stride, const int32_t* slots, int n) {
    const int pi = blockIdx.x;
    if (pi >= n) return;
    double* R = treg + (int64_t)slots[pi] * stride;
    for (int64_t k = threadIdx.x; k < stride; k += blockDim.x) R[k] = 0.0;
}

}  // namespace

cudaError_t launch_ts_store_flux(const StepArgs& a, int mx, int my, int mbc, int meqn, cudaStream_t st) {
    if (a.npatches <= 0) return cudaSuccess;
    if (meqn != 3 || !a.treg) return cudaErrorInvalidValue;
    store_flux_kernel<<<a.npatches, TS_TPB, 0, st>>>(a, mx, my, mbc, meqn);
    return cudaGetLastError();
}

cudaError_t launch_ts_apply(const TsArgs& a, cudaStream_t st) {
    if (a.ngroups <= 0) return cudaSuccess;
    ts_apply_kernel<<<a.ngroups, TS_TPB, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_zero_registers(double* treg, int64_t stride, const int32_t* slots, int n, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    zero_registers_kernel<<<n, 128, 0, st>>>(treg, stride, slots, n);
    return cudaGetLastError();
}

}  // namespace fcb
