// Initial conditions, refinement tags, regrid transfers and the mass sum.
//
// References:
//   qinit:     applications/clawpack/advection/2d/swirl/user_4.6/qinit.f,
//              applications/clawpack/euler/2d/quadrants/user_4.6/qinit.f,
//              radial dam break (cell-centre test, as configured for this path),
//              applications/clawpack/shallow/2d/bump/user_4.6/qinit.f (hump),
//              applications/clawpack/advection/2d/periodic/user_4.6/qinit.f with fdisc.f
//   tagging:   src/patches/clawpatch/fort_4.6/fclaw2d_clawpatch46_tag4refinement.f,
//              fclaw2d_clawpatch46_tag4coarsening.f, fort_user/*_exceeds_th.f90.
//              Every criterion's verdict is order independent (a running
//              max-min only grows; the others are "any cell exceeds"), so the
//              device reduces per patch and the host combines families.
//   regrid:    fort_4.6/fclaw2d_clawpatch46_interpolate.f:324-400 (interpolate2fine),
//              fort_4.6/fclaw2d_clawpatch46_average.f:282-364 (average2coarse)
//   mass:      fort_4.6/fclaw2d_clawpatch46_diagnostics.f:13-58 (Kahan per patch)
#include <cuda_runtime.h>

#include "fcb_device.h"

namespace fcb {

// Bathymetry of the lake-at-rest problem at a cell centre.
__device__ __forceinline__ double bathy_b(double xc, double yc) {
    return -1.0 + 0.8 * exp(-((xc - 0.5) * (xc - 0.5) + (yc - 0.5) * (yc - 0.5)) / 0.02);
}

// radialdam/fdisc.f (no mapping) and cellave2.f (cellave2, fss, zeroin): the
// fraction of a cell inside the circle r < r0.  zeroin is Brent's method as the
// reference states it (netlib zeroin, with its "b = b - xm" step); it converges
// in a few tens of steps on [0, 1], and the loop stops after 1000 in any case.
// kind 0: radialdam's r^2 - r0^2; kind 1: advection/2d/periodic/fdisc.f,
// sqrt(x*x + y*y) - r0 (about (x0, y0); the application's disc is at the origin)
struct DiscD {
    double x0, y0, r0;
    int kind = 0;
    __device__ double f(double x, double y) const {
        const double r2 = (x - x0) * (x - x0) + (y - y0) * (y - y0);
        return kind == 0 ? r2 - r0 * r0 : sqrt(r2) - r0;
    }
};

__device__ double zeroin_d(const DiscD& dsc, double xc0, double yc0, double xc1, double yc1, double tol) {
    auto f = [&](double sv) { return dsc.f(xc0 + sv * (xc1 - xc0), yc0 + sv * (yc1 - yc0)); };
    double eps = 1.0, tol1;
    do {
        eps = eps / 2.0;
        tol1 = 1.0 + eps;
    } while (tol1 > 1.0);
    double a = 0.0, b = 1.0, fa = f(a), fb = f(b);
    double c = a, fc = fa, d = b - a, e = d;
    bool restart = false;  // label 20 (true) or 30 (false) at the top of the loop
    for (int it = 0; it < 1000; ++it) {
        if (restart) {
            c = a;
            fc = fa;
            d = b - a;
            e = d;
        }
        if (fabs(fc) < fabs(fb)) {
            a = b;
            b = c;
            c = a;
            fa = fb;
            fb = fc;
            fc = fa;
        }
        tol1 = (2.0 * eps) * fabs(b) + 0.5 * tol;
        const double xm = 0.5 * (c - b);
        if (fabs(xm) <= tol1) break;
        if (fb == 0.0) break;
        bool bisect = fabs(e) < tol1 || fabs(fa) <= fabs(fb);
        if (!bisect) {
            double p, qq;
            if (a == c) {
                const double sv = fb / fa;
                p = (2.0 * xm) * sv;
                qq = 1.0 - sv;
            } else {
                qq = fa / fc;
                const double r = fb / fc;
                const double sv = fb / fa;
                p = sv * (((2.0 * xm) * qq) * (qq - r) - (b - a) * (r - 1.0));
                qq = ((qq - 1.0) * (r - 1.0)) * (sv - 1.0);
            }
            if (p > 0.0) qq = -qq;
            p = fabs(p);
            if ((2.0 * p) >= ((3.0 * xm) * qq - fabs(tol1 * qq)) || p >= fabs((0.5 * e) * qq)) {
                bisect = true;
            } else {
                e = d;
                d = p / qq;
            }
        }
        if (bisect) {
            d = xm;
            e = d;
        }
        a = b;
        fa = fb;
        if (fabs(d) > tol1) b = b + d;
        if (fabs(d) <= tol1) {
            if (xm >= 0) b = b + tol1;
            else b = b - xm;
        }
        fb = f(b);
        restart = (fb * (fc / fabs(fc))) > 0.0;
    }
    return b;
}

__device__ double cellave2_d(const DiscD& dsc, double xlow, double ylow, double dx, double dy) {
    double xx[5], yy[5], x[10], y[10];
    bool fl[5];
    xx[0] = xlow; xx[1] = xlow; xx[2] = xlow + dx; xx[3] = xlow + dx; xx[4] = xx[0];
    yy[0] = ylow; yy[1] = ylow + dy; yy[2] = ylow + dy; yy[3] = ylow; yy[4] = yy[0];
    bool alll = true, allr = true;
    for (int i = 0; i < 4; ++i) {
        fl[i] = dsc.f(xx[i], yy[i]) < 0.0;
        alll = alll && fl[i];
        allr = allr && !fl[i];
    }
    fl[4] = fl[0];
    if (alll) return 1.0;
    if (allr) return 0.0;
    int iv = 0;
    for (int i = 0; i < 4; ++i) {
        if (fl[i]) {
            x[iv] = xx[i];
            y[iv] = yy[i];
            ++iv;
        }
        if (fl[i] != fl[i + 1]) {
            const double ss = zeroin_d(dsc, xx[i], yy[i], xx[i + 1], yy[i + 1], 1e-14);
            x[iv] = xx[i] + ss * (xx[i + 1] - xx[i]);
            y[iv] = yy[i] + ss * (yy[i + 1] - yy[i]);
            ++iv;
        }
    }
    if (iv == 0) return 0.0;
    x[iv] = x[0];
    y[iv] = y[0];
    double area = 0.0;
    for (int i = 0; i < iv; ++i) area = area + (0.5 * (y[i] + y[i + 1])) * (x[i + 1] - x[i]);
    return area / (dx * dy);
}

__global__ void qinit_kernel(const QinitArgs a) {
    const int pi = blockIdx.x;
    if (pi >= a.n) return;
    const int slot = a.slots[pi];
    const PatchMeta mt = a.meta[slot];
    const int nx = a.mx + 2 * a.mbc, ny = a.my + 2 * a.mbc;
    double* q = a.q + (int64_t)slot * a.stride;
    for (int k = threadIdx.x; k < nx * ny; k += blockDim.x) {
        const int r = k / nx, c = k - r * nx;
        const int i = c - a.mbc + 1, j = r - a.mbc + 1;
        const double xc = mt.xlower + (i - 0.5) * mt.dx;
        const double yc = mt.ylower + (j - 0.5) * mt.dy;
        if (a.problem == PROB_SWIRL) {
            for (int m = 0; m < a.meqn; ++m) q[((int64_t)m * ny + r) * nx + c] = (xc < 0.5) ? 1.0 : 0.0;
        } else if (a.problem == PROB_RADIALDAM) {
            const double x0 = a.p[0], y0 = a.p[1], r0 = a.p[2];
            const double rr = sqrt((xc - x0) * (xc - x0) + (yc - y0) * (yc - y0));
            q[((int64_t)0 * ny + r) * nx + c] = (rr < r0) ? a.p[3] : a.p[4];
            q[((int64_t)1 * ny + r) * nx + c] = 0.0;
            q[((int64_t)2 * ny + r) * nx + c] = 0.0;
        } else if (a.problem == PROB_QUADRANTS) {
            const double xs = a.p[16], ys = a.p[17];
            int iq = 0;
            if (xc >= xs && yc >= ys) iq = 0;
            if (xc < xs && yc >= ys) iq = 1;
            if (xc < xs && yc < ys) iq = 2;
            if (xc >= xs && yc < ys) iq = 3;
            const double rho = a.p[iq], u = a.p[4 + iq], v = a.p[8 + iq], pr = a.p[12 + iq];
            q[((int64_t)0 * ny + r) * nx + c] = rho;
            q[((int64_t)1 * ny + r) * nx + c] = rho * u;
            q[((int64_t)2 * ny + r) * nx + c] = rho * v;
            q[((int64_t)3 * ny + r) * nx + c] = pr / a.gamma1 + 0.5 * rho * (u * u + v * v);
        } else if (a.problem == PROB_RADIALDAM_CELLAVE) {
            const DiscD dsc{a.p[0], a.p[1], a.p[2]};
            const double win = cellave2_d(dsc, mt.xlower + (i - 1.0) * mt.dx, mt.ylower + (j - 1.0) * mt.dy, mt.dx,
                                          mt.dy);
            q[((int64_t)0 * ny + r) * nx + c] = a.p[3] * win + a.p[4] * (1.0 - win);
            q[((int64_t)1 * ny + r) * nx + c] = 0.0;
            q[((int64_t)2 * ny + r) * nx + c] = 0.0;
        } else if (a.problem == PROB_PERIODIC_DISC || a.problem == PROB_FILAMENT) {
            // advection/2d/periodic/user_4.6/qinit.f: q(i,j,1) = the cell's fraction inside the disc
            // (filament/user_4.6/qinit.f with its fdisc.f: the disc of radius 0.25 about (0.5, 1))
            DiscD dsc{a.p[2], a.p[3], a.p[4]};
            dsc.kind = 1;
            q[r * nx + c] = cellave2_d(dsc, mt.xlower + (i - 1.0) * mt.dx, mt.ylower + (j - 1.0) * mt.dy, mt.dx, mt.dy);
        } else if (a.problem == PROB_HUMP) {
            // q(i,j,1) = 0.1d0 + exp(-200.d0*r2), r2 = (xc-x0)**2 + (yc-y0)**2
            const double r2 = (xc - a.p[0]) * (xc - a.p[0]) + (yc - a.p[1]) * (yc - a.p[1]);
            q[((int64_t)0 * ny + r) * nx + c] = a.p[2] + exp(-(a.p[3] * r2));
            q[((int64_t)1 * ny + r) * nx + c] = 0.0;
            q[((int64_t)2 * ny + r) * nx + c] = 0.0;
        } else if (a.problem == PROB_BATHY) {
            const double r2 = (xc - a.p[0]) * (xc - a.p[0]) + (yc - a.p[1]) * (yc - a.p[1]);
            const double eta = a.p[2] * exp(-r2 / (a.p[3] * a.p[3]));
            const double b = bathy_b(xc, yc);
            q[((int64_t)0 * ny + r) * nx + c] = (eta - b > 0.0) ? eta - b : 0.0;  // max(0, eta - b)
            q[((int64_t)1 * ny + r) * nx + c] = 0.0;
            q[((int64_t)2 * ny + r) * nx + c] = 0.0;
        }
    }
}

// filament/psi.f: psi = (4/3) r**3 (r**3 as r*r*r), r = sqrt((x-1)**2 + (y-1)**2)
__device__ __forceinline__ double psi_filament(double x, double y) {
    const double r = sqrt((x - 1.0) * (x - 1.0) + (y - 1.0) * (y - 1.0));
    return (4.0 / 3.0) * (r * r * r);
}

// src/patches/metric/fortran_source2d/fclaw2d_metric_default_fort.f90
// get_area_approx with norm_cross: |T_xi x T_eta| at the centre of the bilinear
// cell with corners (x0 + ic*dx, y0 + jc*dy), z = 0 (compute_area_affine)
__device__ double area_affine(double x0, double y0, double dx, double dy) {
    double cx[2][2], cy[2][2];
    for (int ic = 0; ic < 2; ++ic)
        for (int jc = 0; jc < 2; ++jc) {
            cx[ic][jc] = x0 + ic * dx;
            cy[ic][jc] = y0 + jc * dy;
        }
    double a01[3], a10[3], a11[3], txi[3], teta[3];
    for (int m = 0; m < 3; ++m) {
        const double c00 = m == 0 ? cx[0][0] : (m == 1 ? cy[0][0] : 0.0);
        const double c10 = m == 0 ? cx[1][0] : (m == 1 ? cy[1][0] : 0.0);
        const double c01 = m == 0 ? cx[0][1] : (m == 1 ? cy[0][1] : 0.0);
        const double c11 = m == 0 ? cx[1][1] : (m == 1 ? cy[1][1] : 0.0);
        a01[m] = c10 - c00;
        a10[m] = c01 - c00;
        a11[m] = c11 - c10 - c01 + c00;
    }
    for (int m = 0; m < 3; ++m) {
        txi[m] = a01[m] + a11[m] * 0.5;
        teta[m] = a10[m] + a11[m] * 0.5;
    }
    const double w1 = txi[1] * teta[2] - txi[2] * teta[1];
    const double w2 = -txi[0] * teta[2] + txi[2] * teta[0];
    const double w3 = txi[0] * teta[1] - txi[1] * teta[0];
    return sqrt(w1 * w1 + w2 * w2 + w3 * w3);
}

// setaux for every listed slot, ghost cells included: the lake-at-rest
// problem's aux(i,j,1) = b at the cell centres; the periodic problem's
// aux(i,j,1) = uvel, aux(i,j,2) = vvel (advection/2d/periodic/user_4.6/
// clawpack46_setaux.f; further components 0, unused); the filament's
// (advection/2d/all/user46_setaux_manifold.f on the cart-mapped brick, whose
// nodes map to themselves exactly on this dyadic mesh) aux(i,j,1) =
// area/(dx*dy), aux(i,j,2) = (psi(node(i,j+1)) - psi(node(i,j)))/dy,
// aux(i,j,3) = -(psi(node(i+1,j)) - psi(node(i,j)))/dx; p[0] != 0 multiplies the
// capacity by 1 + p[0]*xc*yc (a test setting that makes dtdx1d vary by cell).
__global__ void setaux_kernel(int problem, int maux, double uvel, double vvel, double* aux, int64_t stride,
                              const int32_t* slots, const PatchMeta* meta, int n, int mx, int my, int mbc) {
    const int pi = blockIdx.x;
    if (pi >= n) return;
    const int slot = slots[pi];
    const PatchMeta mt = meta[slot];
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc;
    double* a = aux + (int64_t)slot * stride;
    for (int k = threadIdx.x; k < nx * ny; k += blockDim.x) {
        const int r = k / nx, c = k - r * nx;
        if (problem == PROB_BATHY) {
            const double xc = mt.xlower + (c - mbc + 1 - 0.5) * mt.dx;
            const double yc = mt.ylower + (r - mbc + 1 - 0.5) * mt.dy;
            a[k] = bathy_b(xc, yc);
        } else if (problem == PROB_FILAMENT) {
            const int i = c - mbc + 1, j = r - mbc + 1;
            const double xn = mt.xlower + (i - 1) * mt.dx, yn = mt.ylower + (j - 1) * mt.dy;
            a[k] = area_affine(xn, yn, mt.dx, mt.dy) / (mt.dx * mt.dy);
            if (uvel != 0.0)  // p[0]: the capacity modulation of the tests (0 in the application)
                a[k] = a[k] * (1.0 + uvel * ((mt.xlower + (i - 0.5) * mt.dx) * (mt.ylower + (j - 0.5) * mt.dy)));
            const double p00 = psi_filament(xn, yn);
            a[nx * ny + k] = (psi_filament(xn, mt.ylower + j * mt.dy) - p00) / mt.dy;
            a[2 * nx * ny + k] = -((psi_filament(mt.xlower + i * mt.dx, yn) - p00) / mt.dx);
        } else {
            a[k] = uvel;
            a[nx * ny + k] = vvel;
            for (int m = 2; m < maux; ++m) a[(int64_t)m * nx * ny + k] = 0.0;
        }
    }
}

cudaError_t launch_setaux(int problem, int maux, const double* params, double* aux, int64_t stride,
                          const int32_t* slots, const PatchMeta* meta, int n, int mx, int my, int mbc, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    setaux_kernel<<<n, 256, 0, st>>>(problem, maux, params[0], params[1], aux, stride, slots, meta, n, mx, my, mbc);
    return cudaGetLastError();
}

cudaError_t launch_qinit(const QinitArgs& a, cudaStream_t st) {
    if (a.n <= 0) return cudaSuccess;
    qinit_kernel<<<a.n, 256, 0, st>>>(a);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Tagging: per patch, the min/max of component ivar over all cells (ghosts
// included) and, for the "difference"/"gradient"/"value" criteria, whether any
// cell exceeds the refine and the coarsen threshold.
// out[4*p + 0] = qmin, [1] = qmax, [2] = refine-exceeds (0/1), [3] = coarsen-exceeds (0/1)
// ---------------------------------------------------------------------------
__global__ void tag_kernel(const TagArgs a) {
    const int pi = blockIdx.x;
    if (pi >= a.n) return;
    const int slot = a.slots[pi];
    const PatchMeta mt = a.meta[slot];
    const int nx = a.mx + 2 * a.mbc, ny = a.my + 2 * a.mbc;
    const double* q = a.q + (int64_t)slot * a.stride + (int64_t)a.ivar * nx * ny;
    double qmin = q[(a.mbc) * nx + a.mbc], qmax = qmin;
    int ex_r = 0, ex_c = 0;
    for (int k = threadIdx.x; k < nx * ny; k += blockDim.x) {
        const int r = k / nx, c = k - r * nx;
        const double v = q[k];
        qmin = v < qmin ? v : qmin;
        qmax = v > qmax ? v : qmax;
        const bool ghost = c < a.mbc || r < a.mbc || c >= a.mbc + a.mx || r >= a.mbc + a.my;
        if (a.criteria == TAG_VALUE) {
            ex_r |= (v > a.refine_th);
            ex_c |= (v > a.coarsen_th);
        } else if (!ghost && (a.criteria == TAG_DIFFERENCE || a.criteria == TAG_GRADIENT)) {
            const double e = q[k + 1], w = q[k - 1], n_ = q[k + nx], s = q[k - nx];
            if (a.criteria == TAG_DIFFERENCE) {
                const double dqx = fabs(e - w), dqy = fabs(n_ - s);
                const double dq = dqx > dqy ? dqx : dqy;
                ex_r |= (dq > a.refine_th);
                ex_c |= (dq > a.coarsen_th);
            } else {
                const double dx2 = 2 * mt.dx, dy2 = 2 * mt.dy;
                const double dqx = (e - w) / dx2, dqy = (n_ - s) / dy2;
                const double g3 = 0;
                const double ds = sqrt(dqx * dqx + dqy * dqy + g3 * g3);
                ex_r |= (ds > a.refine_th);
                ex_c |= (ds > a.coarsen_th);
            }
        }
    }
    __shared__ double smin[32], smax[32];
    __shared__ int sr[32], sc[32];
    for (int off = 16; off > 0; off >>= 1) {
        const double a1 = __shfl_xor_sync(0xffffffffu, qmin, off);
        const double a2 = __shfl_xor_sync(0xffffffffu, qmax, off);
        qmin = a1 < qmin ? a1 : qmin;
        qmax = a2 > qmax ? a2 : qmax;
        ex_r |= __shfl_xor_sync(0xffffffffu, ex_r, off);
        ex_c |= __shfl_xor_sync(0xffffffffu, ex_c, off);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { smin[w] = qmin; smax[w] = qmax; sr[w] = ex_r; sc[w] = ex_c; }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        for (int k = 1; k < nw; ++k) {
            qmin = smin[k] < qmin ? smin[k] : qmin;
            qmax = smax[k] > qmax ? smax[k] : qmax;
            ex_r |= sr[k];
            ex_c |= sc[k];
        }
        a.out[4 * pi + 0] = qmin;
        a.out[4 * pi + 1] = qmax;
        a.out[4 * pi + 2] = ex_r;
        a.out[4 * pi + 3] = ex_c;
    }
}

cudaError_t launch_tag(const TagArgs& a, cudaStream_t st) {
    if (a.n <= 0) return cudaSuccess;
    tag_kernel<<<a.n, 256, 0, st>>>(a);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Regrid transfers.  ops[3*k] = kind (0 = interpolate2fine, 1 = average2coarse),
// ops[3*k+1] = coarse slot, ops[3*k+2] = first of four consecutive entries in
// `fine` (the four children in z-order).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double slope5b(double sl, double sr) {
    const double sc = (sl + sr) / 2.0;
    double m = 2 * fabs(sl);
    const double b = 2 * fabs(sr), cc = fabs(sc);
    if (b < m) m = b;
    if (cc < m) m = cc;
    const double s0 = copysign(1.0, sl * sr);
    return m * (s0 > 0.0 ? s0 : 0.0) * copysign(1.0, sc);
}

__global__ void regrid_kernel(double* q, int64_t stride, const int32_t* ops, const int32_t* fine,
                              int nops, int mx, int my, int mbc, int meqn) {
    const int k = blockIdx.x >> 2;  // four CTAs per record: one per child
    const int igrid = blockIdx.x & 3;
    if (k >= nops) return;
    const int kind = ops[3 * k], cslot = ops[3 * k + 1];
    const int fslot = fine[ops[3 * k + 2] + igrid];
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc;
    double* qc = q + (int64_t)cslot * stride;
    double* qf = q + (int64_t)fslot * stride;
    auto C = [&](int i, int j, int m) -> double& { return qc[((int64_t)m * ny + j + mbc - 1) * nx + i + mbc - 1]; };
    auto F = [&](int i, int j, int m) -> double& { return qf[((int64_t)m * ny + j + mbc - 1) * nx + i + mbc - 1]; };
    const int ig = igrid % 2, jg = igrid / 2;
    if (kind == 0) {
        const int i1 = 1 - ig, i2 = mx / 2 + (1 - ig), ic_add = ig * mx / 2;
        const int j1 = 1 - jg, j2 = my / 2 + (1 - jg), jc_add = jg * my / 2;
        const int wi = i2 - i1 + 1, wj = j2 - j1 + 1;
        for (int t = threadIdx.x; t < meqn * wi * wj; t += blockDim.x) {
            const int m = t / (wi * wj), rem = t - m * wi * wj;
            const int j = j1 + rem / wi, i = i1 + rem % wi;
            const int ic = i + ic_add, jc = j + jc_add;
            const double qcv = C(ic, jc, m);
            double sl = (qcv - C(ic - 1, jc, m));
            double sr = (C(ic + 1, jc, m) - qcv);
            const double gradx = slope5b(sl, sr);
            sl = (qcv - C(ic, jc - 1, m));
            sr = (C(ic, jc + 1, m) - qcv);
            const double grady = slope5b(sl, sr);
            for (int ii = 1; ii <= 2; ++ii)
                for (int jj = 1; jj <= 2; ++jj) {
                    const double shiftx = (ii - 2 / 2.0 - 0.5) / 2;
                    const double shifty = (jj - 2 / 2.0 - 0.5) / 2;
                    F((i - 1) * 2 + ii, (j - 1) * 2 + jj, m) = qcv + shiftx * gradx + shifty * grady;
                }
        }
    } else {
        const int ic_add = ig * mx / 2, jc_add = jg * mx / 2;  // the reference uses mx for both
        const int wi = mx / 2, wj = my / 2;
        for (int t = threadIdx.x; t < meqn * wi * wj; t += blockDim.x) {
            const int m = t / (wi * wj), rem = t - m * wi * wj;
            const int j = 1 + rem / wi, i = 1 + rem % wi;
            double sum = 0;
            sum = sum + F((i - 1) * 2 + 1, (j - 1) * 2 + 1, m);
            sum = sum + F((i - 1) * 2 + 2, (j - 1) * 2 + 1, m);
            sum = sum + F((i - 1) * 2 + 1, (j - 1) * 2 + 2, m);
            sum = sum + F((i - 1) * 2 + 2, (j - 1) * 2 + 2, m);
            C(i + ic_add, j + jc_add, m) = sum / 4;
        }
    }
}

cudaError_t launch_regrid(double* q, int64_t stride, const int32_t* ops, const int32_t* fine, int nops,
                          int mx, int my, int mbc, int meqn, cudaStream_t st) {
    if (nops <= 0) return cudaSuccess;
    regrid_kernel<<<nops * 4, 128, 0, st>>>(q, stride, ops, fine, nops, mx, my, mbc, meqn);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Mass: Kahan-compensated sum of q*dx*dy over the interior of each patch, in
// the reference's loop order (m, j, i); out[p*meqn + m].
// ---------------------------------------------------------------------------
__global__ void mass_kernel(const double* q, int64_t stride, const int32_t* slots, const PatchMeta* meta,
                            int n, int mx, int my, int mbc, int meqn, double* out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int slot = slots[p];
    const double area = meta[slot].dx * meta[slot].dy;
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc;
    const double* qp = q + (int64_t)slot * stride;
    for (int m = 0; m < meqn; ++m) {
        double sum = 0.0, ck = 0.0;
        for (int j = 1; j <= my; ++j)
            for (int i = 1; i <= mx; ++i) {
                const double y = qp[((int64_t)m * ny + j + mbc - 1) * nx + i + mbc - 1] * area - ck;
                const double t = sum + y;
                ck = (t - sum) - y;
                sum = t;
            }
        out[(int64_t)p * meqn + m] = sum;
    }
}

cudaError_t launch_mass(const double* q, int64_t stride, const int32_t* slots, const PatchMeta* meta, int n,
                        int mx, int my, int mbc, int meqn, double* out, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    mass_kernel<<<(n + 127) / 128, 128, 0, st>>>(q, stride, slots, meta, n, mx, my, mbc, meqn, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Gather / scatter of whole patches between the slot arena and a contiguous
// buffer (leaf order), so that host transfers are one copy each way.
// ---------------------------------------------------------------------------
// meqn5 > 0: the staging side holds each patch in the clawpack 5 order q(m,i,j)
// (component fastest) while the arena keeps q(i,j,m).
__global__ void gather_kernel(const double* __restrict__ src, int64_t stride, const int32_t* slots, int n,
                              int64_t psize, double* __restrict__ dst, int scatter, int meqn5) {
    const int64_t ncell = meqn5 > 0 ? psize / meqn5 : psize;
    for (int p = blockIdx.x; p < n; p += gridDim.x) {
        const int64_t a = (int64_t)slots[p] * stride, b = (int64_t)p * psize;
        for (int64_t k = threadIdx.x; k < psize; k += blockDim.x) {
            int64_t h = k;
            if (meqn5 > 0) {
                const int64_t m = k / ncell, cell = k - m * ncell;
                h = cell * meqn5 + m;
            }
            if (scatter) const_cast<double*>(src)[a + k] = dst[b + h];
            else dst[b + h] = src[a + k];
        }
    }
}

cudaError_t launch_gather(const double* src, int64_t stride, const int32_t* slots, int n, int64_t psize,
                          double* dst, bool scatter, int meqn5, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int blocks = n < 148 * 16 ? n : 148 * 16;
    gather_kernel<<<blocks, 256, 0, st>>>(src, stride, slots, n, psize, dst, scatter ? 1 : 0, meqn5);
    return cudaGetLastError();
}

}  // namespace fcb
