// Batched Clawpack 4.6 patch update (step2 + flux2 + conservative update) for
// sm_100a.  One thread per patch column, several patches per CTA; the patch
// rows stream through a two-row pipeline so that q is read once and written
// once per step with no global flux scratch.
//
// Reference: src/solvers/fc2d_clawpack4.6/fortran_source/clawpack46_step2_wrap.f
// (conservative update over i,j = 1-mbc..mx+mbc-1), clawpack46_step2.f (x- and
// y-sweeps, fm/fp/gm/gp accumulation), clawpack46_flux2.f (Godunov, CFL,
// limiter, second-order and transverse corrections).
//
// Index map: cell (c, r) with c, r in [0, NX) holds Fortran cell
// (i, j) = (c - mbc + 1, r - mbc + 1).  x-interface c sits between cells c-1
// and c, y-interface r between rows r-1 and r.  With the reference's loop
// bounds this gives: x-sweep rows r in [1, NY-2], x-interfaces c in [1, NX-1],
// Godunov part for c <= NX-2, CFL and limiting for c in [mbc, mbc+mx];
// y-sweep columns c in [1, NX-2], interfaces r in [1, NY-1]; updated cells
// c in [0, NX-2], r in [0, NY-2].
//
// The flux accumulators are formed in the reference's order:
//   fm(i,j) = (FXm + GYu[col i-1]) + GYd[col i],   gm(i,j) = (GXu[row j-1] + GXd[row j]) + FYm
// (absent terms are +0, which leaves every sum unchanged), and
//   q = q - dtdx*(fm(i+1,j) - fp(i,j)) - dtdy*(gm(i,j+1) - gp(i,j)).
// This file is compiled without FMA contraction, so each result is rounded
// exactly as the reference's, operation by operation.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>

#include "fcb_device.h"
#include "fcb_solvers.cuh"

namespace fcb {

namespace {

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* p, double v) {
    // Non-negative doubles order like their bit patterns; NaN (large bits) wins
    // and is reported to the host.
    atomicMax(p, (unsigned long long)__double_as_longlong(v));
}

template <int NX, int NY, int PPB, int M, int W, int NAUX, bool PSI, int NC>
struct StepSmem {
    static constexpr int QROW = 0;
    static constexpr int XW = QROW + 3 * PPB * NX * M;
    static constexpr int XS = XW + PPB * NX * W * M;
    static constexpr int GL = XS + PPB * NX * W;
    static constexpr int FX = GL + PPB * NX * 2 * M;
    static constexpr int GY = FX + 3 * PPB * NX * 2 * M;
    static constexpr int CROW = GY + PPB * NX * 2 * M;
    static constexpr int GXR = CROW + 2 * PPB * NX * NC;
    static constexpr int AUX = GXR + 3 * PPB * NX * M;
    static constexpr int TAB = AUX + PPB * NAUX * NY * NX;
    static constexpr int PSIT = TAB + (PSI ? PPB * 2 * (NX + 1) : 0);
    static constexpr int TOTAL = PSIT + (PSI ? PPB * (NY + 1) * (NX + 1) : 0);
};

// LIM > 0: order (2, 2) and limiter LIM on every wave, fixed at compile time;
// LIM == 0: order and limiters read from the launch arguments.
template <int LIM>
struct MethodC {
    const StepArgs& a;
    __device__ __forceinline__ bool second_order() const { return LIM > 0 || a.order0 == 2; }
    __device__ __forceinline__ bool transverse() const { return LIM > 0 || a.order1 > 0; }
    __device__ __forceinline__ bool transverse2() const { return LIM > 0 || (a.order0 > 1 && a.order1 == 2); }
    __device__ __forceinline__ int lim(int mw) const { return LIM > 0 ? LIM : a.mthlim[mw]; }
};

}  // namespace

// AUXK: AUX_NONE, AUX_SWIRL (velocities computed from the swirl stream function),
// AUX_STORED (aux arena, NAUX components).
template <class SOL, int MX, int MBC, int AUXK, int NAUX, int TPB, int LIM>
__global__ void __launch_bounds__(TPB) step_kernel(const StepArgs a) {
    constexpr int M = SOL::M;
    constexpr int W = SOL::W;
    constexpr int NC = SOL::NC;
    constexpr int NX = MX + 2 * MBC;
    constexpr int NY = NX;
    constexpr int PPB = TPB / NX;
    using L = StepSmem<NX, NY, PPB, M, W, NAUX, AUXK == AUX_SWIRL, NC>;
    using Cell = typename SOL::Cell;
    // mapped grids: the Riemann solvers read aux from component KS on, and
    // aux(1) is the capacity kappa (dtdx1d(i) = dtdx / kappa(i), clawpack46_step2.f:122-126)
    constexpr int KS = AuxLayout<SOL>::SHIFT;
    constexpr bool CAPA = AuxLayout<SOL>::CAPA;
    // clawpack 5 (scalar advection here): clawpack5_inlinelimiter.f's computed
    // go to sends mthlim > 5 to its first branch (minmod), and
    // clawpack5_step2_wrap.f updates the interior cells 1..mx, 1..my only;
    // those read the interfaces 1..mx+1, whose fluxes are the same as 4.6's
    constexpr bool V5 = SOL::V5;
    auto LIMV = [](int l) { return (V5 && l > 5) ? 1 : l; };
    const MethodC<LIM> meth{a};
    extern __shared__ double smem[];
    double* s_qrow = smem + L::QROW;  // [3][PPB][NX][M]: rows s-2, s-1, s (slot row % 3)
    double* s_xw = smem + L::XW;      // [PPB][NX][W][M]
    double* s_xs = smem + L::XS;      // [PPB][NX][W]
    double* s_gl = smem + L::GL;      // [PPB][NX][2][M]
    double* s_fx = smem + L::FX;      // [3][PPB][NX][2][M]
    double* s_gy = smem + L::GY;      // [PPB][NX][2][M]
    double* s_crow = smem + L::CROW;  // [2][PPB][NX][NC]: the cell quantities of rows s-1 and s
    double* s_gxr = smem + L::GXR;    // [3][PPB][NX][M]: GXu(row-1) + GXd(row) of rows s-2, s-1, s (own column)
    double* s_aux = smem + L::AUX;    // [PPB][NAUX][NY][NX]
    double* s_tab = smem + L::TAB;    // [PPB][2][NX+1] (swirl)
    double* s_psi = smem + L::PSIT;   // [PPB][NY+1][NX+1] (swirl)

    const int t = threadIdx.x;
    const int pl = t / NX;
    const int c = t - pl * NX;
    // Row bands: band `band` of the patch group updates cell rows [R0, R1) and
    // streams rows s0..s1; it starts two rows early so that every carried
    // value its first own row needs (the raw y-interface R0-1, the x-row R0-1)
    // is computed inside the band.  Raw y-interfaces from before row s0+1 and
    // finalized ones before s0+2 would see rows the band did not load and are
    // skipped; the first band keeps the reference's boundary behaviour.
    // With band_first, the CTAs before it update whole patches in place and
    // the ones after it are the bands of the remaining patches.
    const int B0 = a.nbands > 1 ? a.band_first : 0;
    const bool banded = a.nbands > 1 && (int)blockIdx.x >= B0;
    const int nb = banded ? a.nbands : 1;
    const int rel = (int)blockIdx.x - B0;
    const int band = banded ? rel % nb : 0;
    const int pg = (banded ? B0 + rel / nb : (int)blockIdx.x) * PPB + pl;
    const int R0 = band * (NY - 1) / nb, R1 = (band + 1) * (NY - 1) / nb;
    const int s0 = band == 0 ? 0 : R0 - 2;
    const int s1 = band == nb - 1 ? NY : R1 + 1;
    const int ylo = band == 0 ? 1 : s0 + 1;
    const int flo = band == 0 ? 1 : s0 + 2;
    const int qlo = band == 0 ? 0 : R0, qhi = band == nb - 1 ? NY : R1;
    const bool active = (pl < PPB) && (pg < a.npatches);
    // a launch over the patches of several solves (serving) describes every
    // patch by its own arrays, geometry, dt and CFL slot
    const PatchDesc* D = (a.desc && active) ? a.desc + pg : nullptr;
    const int slot = (active && !a.desc) ? a.slots[pg] : 0;
    const PatchMeta meta = D ? D->meta : (active ? a.meta[slot] : PatchMeta{0, 0, 1, 1, 0, 0});
    const int req = D ? D->req : -1;
    double* __restrict__ q = D ? D->q : a.q + (int64_t)slot * a.q_stride;
    const double* __restrict__ qin = D ? D->q : (banded ? a.qsrc : a.q) + (int64_t)slot * a.q_stride;
    double* __restrict__ qlast = D ? D->qlast : a.qlast + (int64_t)slot * a.q_stride;
    const bool save_last = active && (meta.flags & PATCH_SAVE_LAST);
    const double pdt = D ? D->dt : step_dt(a, meta.level);
    const double dtdx = pdt / meta.dx;
    const double dtdy = pdt / meta.dy;
    const double dtdxave = 0.5 * (dtdx + dtdx);  // 0.5*(dtdx1d(i-1)+dtdx1d(i)), no capacity
    const double dtdyave = 0.5 * (dtdy + dtdy);
    SOL sol{a.grav, a.gamma, a.gamma1};

    // ---- aux tile ---------------------------------------------------------
    if constexpr (AUXK == AUX_SWIRL) {
        // swirl/user_4.6/b4step2.f with swirl/psi.f:
        //   u(i,j) = vty*(psi(xll,yll+dy) - psi(xll,yll)),  v(i,j) = -vtx*(psi(xll+dx,yll) - psi(xll,yll))
        //   psi(x,y) = (sin(pi x)**2 * sin(pi y)**2)/pi
        // On the dyadic unit-square mesh (mx a power of two) xll + dx is the next
        // node's xll exactly, so psi is evaluated once per node: P(c,r) at the
        // lower-left corner of cell (c,r), c in [0,NX], r in [0,NY].
        constexpr double pi = 3.141592653589793;  // 4*atan(1) in double precision
        double* tx = s_tab + pl * 2 * (NX + 1);
        double* ty = tx + (NX + 1);
        double* P = s_psi + pl * (NY + 1) * (NX + 1);
        if (active) {
            for (int n = c; n <= NX; n += NX) {
                const double x = meta.xlower + (double)(n - MBC) * meta.dx;
                const double y = meta.ylower + (double)(n - MBC) * meta.dy;
                const double sx = sin(pi * x), sy = sin(pi * y);
                tx[n] = sx * sx;
                ty[n] = sy * sy;
            }
        }
        __syncthreads();
        if (active) {
            for (int n = c; n <= NX; n += NX) {
                const double sx2 = tx[n];
                for (int r = 0; r <= NY; ++r) P[r * (NX + 1) + n] = (sx2 * ty[r]) / pi;
            }
        }
        __syncthreads();
        if (active) {
            const double pvt = D ? D->vt : step_vt(a, meta.level);
            const double vty = pvt / meta.dy;
            const double vtx = pvt / meta.dx;
            double* au = s_aux + (pl * NAUX + 0) * NY * NX;
            double* av = s_aux + (pl * NAUX + 1) * NY * NX;
            for (int r = 0; r < NY; ++r) {
                const double pij = P[r * (NX + 1) + c];
                au[r * NX + c] = vty * (P[(r + 1) * (NX + 1) + c] - pij);
                av[r * NX + c] = -vtx * (P[r * (NX + 1) + c + 1] - pij);
            }
        }
    } else if constexpr (AUXK == AUX_STORED) {
        if (active) {
            const double* ag = D ? D->aux : a.aux + (int64_t)slot * a.aux_stride;
            for (int k = 0; k < NAUX; ++k)
                for (int r = 0; r < NY; ++r)
                    s_aux[((pl * NAUX + k) * NY + r) * NX + c] = ag[(k * NY + r) * NX + c];
        }
    }
    __syncthreads();
    auto AUXV = [&](int k, int cc, int rr) -> double {
        if constexpr (NAUX > 0) return s_aux[((pl * NAUX + k) * NY + rr) * NX + cc];
        else return 0.0;
    };
    // dtdx1d / dtdy1d of cell (cc, rr)
    auto DTDX = [&](int cc, int rr) -> double {
        if constexpr (CAPA) return dtdx / AUXV(0, cc, rr);
        else return dtdx;
    };
    auto DTDY = [&](int cc, int rr) -> double {
        if constexpr (CAPA) return dtdy / AUXV(0, cc, rr);
        else return dtdy;
    };

    const bool ycol = active && c >= 1 && c <= NX - 2;
    double cfl = 0.0;

    // q rows s-2, s-1, s of this column
    double q_n[M];
    // y window: finalizing interface f = s-1 uses its raw waves (yw_f) and the
    // dot products with interfaces f-1 (ydotl) and f+1 (ydotr).
    double yw_f[W][M], ys_f[W], yam_f[M], yap_f[M], ydotl[W];
    typename SOL::Roe yR_f{};
    double yw_n[W][M], ys_n[W], yam_n[M], yap_n[M], ydotr[W];
    typename SOL::Roe yR_n{};
    double gRm_prev[M], gRp_prev[M];  // y transverse parts from interface f-1 into cell f-1
    double FYp_prev[M];               // faddp of interface s-2
    double GXu_prev[M];               // x-row s-1 "up" transverse part
    double GYd_r[M], GYu_r[M];        // y transverse parts for cell row s-2
#pragma unroll
    for (int m = 0; m < M; ++m) {
        q_n[m] = 0.0;
        yam_f[m] = yap_f[m] = yam_n[m] = yap_n[m] = 0.0;
        gRm_prev[m] = gRp_prev[m] = FYp_prev[m] = GXu_prev[m] = 0.0;
        GYd_r[m] = GYu_r[m] = 0.0;
    }
#pragma unroll
    for (int mw = 0; mw < W; ++mw) {
        ys_f[mw] = ys_n[mw] = ydotl[mw] = ydotr[mw] = 0.0;
#pragma unroll
        for (int m = 0; m < M; ++m) yw_f[mw][m] = yw_n[mw][m] = 0.0;
    }

    // q of (column cc, row rr) in the row ring
    auto QR = [&](int rr, int cc) -> double* { return s_qrow + (((rr % 3) * PPB + pl) * NX + cc) * M; };
    auto GXS = [&](int rr) -> double* { return s_gxr + (((rr % 3) * PPB + pl) * NX + c) * M; };
    double* xw = s_xw + pl * NX * W * M;
    double* xs = s_xs + pl * NX * W;
    double* gl = s_gl + pl * NX * 2 * M;
    double* gy = s_gy + pl * NX * 2 * M;

    // cell quantities of (column cc, row rr), shared by the interfaces of the cell
    auto CELL = [&](int rr, int cc) -> Cell* {
        return reinterpret_cast<Cell*>(s_crow + (((rr & 1) * PPB + pl) * NX + cc) * NC);
    };

    for (int s = s0; s <= s1; ++s) {
        // ---------------- phase 1: load row s; raw y-interface s ----------------
        if (s < NY && active) {
#pragma unroll
            for (int m = 0; m < M; ++m) {
                const int64_t k = ((int64_t)m * NY + s) * NX + c;
                q_n[m] = qin[k];
                if (save_last && s >= qlo && s < qhi) qlast[k] = q_n[m];
                QR(s, c)[m] = q_n[m];
            }
            Cell cn;
            sol.prep(q_n, cn);
            if constexpr (NC > 0) *CELL(s, c) = cn;
            if (ycol && s >= ylo) {
                double q_m1[M];
#pragma unroll
                for (int m = 0; m < M; ++m) q_m1[m] = QR(s - 1, c)[m];
                sol.rpn2c(2, q_m1, q_n, *CELL(s - 1, c), cn, AUXV(1 + KS, c, s), yw_n, ys_n, yam_n, yap_n, yR_n);
#pragma unroll
                for (int mw = 0; mw < W; ++mw) {
                    double d = yw_f[mw][0] * yw_n[mw][0];
#pragma unroll
                    for (int m = 1; m < M; ++m) d = d + yw_f[mw][m] * yw_n[mw][m];
                    ydotr[mw] = d;  // dot(w(s-1), w(s))
                }
            }
        }
        // ---------------- y: finalize interface f = s-1 (own column) ----------------
        double FYm_cur[M];
#pragma unroll
        for (int m = 0; m < M; ++m) { FYm_cur[m] = 0.0; GYd_r[m] = 0.0; GYu_r[m] = 0.0; }
        const int f = s - 1;
        if (ycol && f >= flo) {
            double w[W][M];
#pragma unroll
            for (int mw = 0; mw < W; ++mw)
#pragma unroll
                for (int m = 0; m < M; ++m) w[mw][m] = yw_f[mw][m];
            // dtdy1d of the cells below (f-1) and above (f) the interface
            const double dty_lo = DTDY(c, f - 1), dty_hi = DTDY(c, f);
            if (f >= MBC && f <= MBC + MX) {
#pragma unroll
                for (int mw = 0; mw < W; ++mw) cfl = nanmax(nanmax(cfl, dty_hi * ys_f[mw]), -dty_lo * ys_f[mw]);
            }
            const double dtyave = CAPA ? 0.5 * (dty_lo + dty_hi) : dtdyave;
            double cq[M];
#pragma unroll
            for (int m = 0; m < M; ++m) cq[m] = 0.0;
            if (meth.second_order()) {
                if (f >= MBC && f <= MBC + MX) {
#pragma unroll
                    for (int mw = 0; mw < W; ++mw) {
                        if (meth.lim(mw) == 0) continue;
                        double wn2 = yw_f[mw][0] * yw_f[mw][0];
#pragma unroll
                        for (int m = 1; m < M; ++m) wn2 = wn2 + yw_f[mw][m] * yw_f[mw][m];
                        if (wn2 == 0.0) continue;
                        const double r = (ys_f[mw] > 0.0) ? ydotl[mw] / wn2 : ydotr[mw] / wn2;
                        const double phi = limiter_phi(LIMV(meth.lim(mw)), r);
#pragma unroll
                        for (int m = 0; m < M; ++m) w[mw][m] = phi * w[mw][m];
                    }
                }
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    double acc;
                    {
                        const double as = fabs(ys_f[0]);
                        acc = as * (1.0 - as * dtyave) * w[0][m];
                    }
#pragma unroll
                    for (int mw = 1; mw < W; ++mw) {
                        const double as = fabs(ys_f[mw]);
                        acc = acc + as * (1.0 - as * dtyave) * w[mw][m];
                    }
                    cq[m] = acc;
                }
            }
            double fm_[M], fp_[M], am[M], ap[M];
#pragma unroll
            for (int m = 0; m < M; ++m) {
                double fmv = (f <= NY - 2) ? yam_f[m] : 0.0;
                double fpv = (f <= NY - 2) ? -yap_f[m] : 0.0;
                if (meth.second_order()) { fmv = fmv + 0.5 * cq[m]; fpv = fpv + 0.5 * cq[m]; }
                fm_[m] = fmv; fp_[m] = fpv;
                am[m] = yam_f[m]; ap[m] = yap_f[m];
                if (meth.transverse2() && f <= NY - 2) { am[m] = am[m] + cq[m]; ap[m] = ap[m] - cq[m]; }
                FYm_cur[m] = fmv;
            }
            double gLm[M], gLp[M], gRm[M], gRp[M];
            if (meth.transverse()) {
                double bm[M], bp[M];
                // imp = 1: aux2(j-1, kv=1), aux3(j-1, kv=1) = u at columns c, c+1, row f-1
                sol.rpt2(2, am, yR_f, AUXV(KS, c, f - 1), AUXV(KS, c + 1, f - 1), bm, bp);
#pragma unroll
                for (int m = 0; m < M; ++m) { gLm[m] = 0.5 * dty_lo * bm[m]; gLp[m] = 0.5 * dty_lo * bp[m]; }
                sol.rpt2(2, ap, yR_f, AUXV(KS, c, f), AUXV(KS, c + 1, f), bm, bp);
#pragma unroll
                for (int m = 0; m < M; ++m) { gRm[m] = 0.5 * dty_hi * bm[m]; gRp[m] = 0.5 * dty_hi * bp[m]; }
            } else {
#pragma unroll
                for (int m = 0; m < M; ++m) gLm[m] = gLp[m] = gRm[m] = gRp[m] = 0.0;
            }
            // cell row k = f-1 is now complete: gadd(k,.,1) = (0 - gL(k+1)) - gR(k)
            if (f - 1 >= 1) {
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    GYd_r[m] = -gLm[m] - gRm_prev[m];
                    GYu_r[m] = -gLp[m] - gRp_prev[m];
                }
            }
#pragma unroll
            for (int m = 0; m < M; ++m) { gRm_prev[m] = gRm[m]; gRp_prev[m] = gRp[m]; }
            // FYp of interface f is needed when updating cell row f (two steps on)
#pragma unroll
            for (int m = 0; m < M; ++m) { FYm_cur[m] = fm_[m]; }
            // rotate FYp below, after the update of row s-2 has used FYp(s-2)
#pragma unroll
            for (int m = 0; m < M; ++m) yap_f[m] = fp_[m];  // reuse slot: holds FYp(f) until rotation
        }
        // shift the y window: raw interface s becomes the one to finalize next
#pragma unroll
        for (int mw = 0; mw < W; ++mw) {
            ydotl[mw] = ydotr[mw];
            ys_f[mw] = ys_n[mw];
#pragma unroll
            for (int m = 0; m < M; ++m) yw_f[mw][m] = yw_n[mw][m];
        }
        double FYp_cur[M];
#pragma unroll
        for (int m = 0; m < M; ++m) {
            FYp_cur[m] = (ycol && f >= flo) ? yap_f[m] : 0.0;
            yam_f[m] = yam_n[m];
            yap_f[m] = yap_n[m];
        }
        yR_f = yR_n;
        __syncthreads();  // A

        // ---------------- phase 2: raw x-interface (c, s) ----------------
        const bool xrow = active && s >= 1 && s <= NY - 2;
        const bool xint = xrow && c >= 1;
        double xwl[W][M], xsl[W], xam[M], xap[M];
        typename SOL::Roe xR{};
        // dtdx1d of the cells left (c-1) and right (c) of the interface
        double dtx_lo = dtdx, dtx_hi = dtdx;
        if (xint) {
            dtx_lo = DTDX(c - 1, s);
            dtx_hi = DTDX(c, s);
            double qL[M];
#pragma unroll
            for (int m = 0; m < M; ++m) qL[m] = QR(s, c - 1)[m];
            sol.rpn2c(1, qL, q_n, *CELL(s, c - 1), *CELL(s, c), AUXV(KS, c, s), xwl, xsl, xam, xap, xR);
#pragma unroll
            for (int mw = 0; mw < W; ++mw) {
                xs[c * W + mw] = xsl[mw];
#pragma unroll
                for (int m = 0; m < M; ++m) xw[(c * W + mw) * M + m] = xwl[mw][m];
                if (c >= MBC && c <= MBC + MX) cfl = nanmax(nanmax(cfl, dtx_hi * xsl[mw]), -dtx_lo * xsl[mw]);
            }
        }

        __syncthreads();  // B

        // ---------------- phase 3: x limiter, corrections, transverse ----------------
        double* fxs = s_fx + ((s % 3) * PPB + pl) * NX * 2 * M;
        double gRmx[M], gRpx[M];
#pragma unroll
        for (int m = 0; m < M; ++m) gRmx[m] = gRpx[m] = 0.0;
        if (xint) {
            const double dtxave = CAPA ? 0.5 * (dtx_lo + dtx_hi) : dtdxave;
            double cq[M];
#pragma unroll
            for (int m = 0; m < M; ++m) cq[m] = 0.0;
            if (meth.second_order()) {
                if (c >= MBC && c <= MBC + MX) {
#pragma unroll
                    for (int mw = 0; mw < W; ++mw) {
                        if (meth.lim(mw) == 0) continue;
                        double wn2 = xwl[mw][0] * xwl[mw][0];
                        double dl = xw[((c - 1) * W + mw) * M + 0] * xwl[mw][0];
                        double dr = xwl[mw][0] * xw[((c + 1) * W + mw) * M + 0];
#pragma unroll
                        for (int m = 1; m < M; ++m) {
                            const double wc = xwl[mw][m];
                            wn2 = wn2 + wc * wc;
                            dl = dl + xw[((c - 1) * W + mw) * M + m] * wc;
                            dr = dr + wc * xw[((c + 1) * W + mw) * M + m];
                        }
                        if (wn2 == 0.0) continue;
                        const double r = (xsl[mw] > 0.0) ? dl / wn2 : dr / wn2;
                        const double phi = limiter_phi(LIMV(meth.lim(mw)), r);
#pragma unroll
                        for (int m = 0; m < M; ++m) xwl[mw][m] = phi * xwl[mw][m];
                    }
                }
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    double acc;
                    {
                        const double as = fabs(xsl[0]);
                        acc = as * (1.0 - as * dtxave) * xwl[0][m];
                    }
#pragma unroll
                    for (int mw = 1; mw < W; ++mw) {
                        const double as = fabs(xsl[mw]);
                        acc = acc + as * (1.0 - as * dtxave) * xwl[mw][m];
                    }
                    cq[m] = acc;
                }
            }
            double am[M], ap[M];
#pragma unroll
            for (int m = 0; m < M; ++m) {
                double fmv = (c <= NX - 2) ? xam[m] : 0.0;
                double fpv = (c <= NX - 2) ? -xap[m] : 0.0;
                if (meth.second_order()) { fmv = fmv + 0.5 * cq[m]; fpv = fpv + 0.5 * cq[m]; }
                fxs[(c * 2 + 0) * M + m] = fmv;
                fxs[(c * 2 + 1) * M + m] = fpv;
                am[m] = xam[m]; ap[m] = xap[m];
                if (meth.transverse2() && c <= NX - 2) { am[m] = am[m] + cq[m]; ap[m] = ap[m] - cq[m]; }
            }
            if (meth.transverse()) {
                double bm[M], bp[M];
                // imp = 1: aux2(i-1, kv=2), aux3(i-1, kv=2) = v at column c-1, rows s, s+1
                sol.rpt2(1, am, xR, AUXV(1 + KS, c - 1, s), AUXV(1 + KS, c - 1, s + 1), bm, bp);
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    gl[(c * 2 + 0) * M + m] = 0.5 * dtx_lo * bm[m];
                    gl[(c * 2 + 1) * M + m] = 0.5 * dtx_lo * bp[m];
                }
                sol.rpt2(1, ap, xR, AUXV(1 + KS, c, s), AUXV(1 + KS, c, s + 1), bm, bp);
#pragma unroll
                for (int m = 0; m < M; ++m) { gRmx[m] = 0.5 * dtx_hi * bm[m]; gRpx[m] = 0.5 * dtx_hi * bp[m]; }
            } else {
#pragma unroll
                for (int m = 0; m < M; ++m) { gl[(c * 2 + 0) * M + m] = 0.0; gl[(c * 2 + 1) * M + m] = 0.0; }
            }
        } else if (active) {
#pragma unroll
            for (int m = 0; m < M; ++m) {
                fxs[(c * 2 + 0) * M + m] = 0.0;
                fxs[(c * 2 + 1) * M + m] = 0.0;
                gl[(c * 2 + 0) * M + m] = 0.0;
                gl[(c * 2 + 1) * M + m] = 0.0;
            }
        }
        __syncthreads();  // C

        // ---------------- phase 4: complete GX(c, s); publish GY(c, s-2) ----------------
        // (idle threads of the CTA, pl == PPB, own no ring slot)
        double* GXs_n = GXS(s);
#pragma unroll
        for (int m = 0; m < M; ++m) {
            double gxd = 0.0, gxu = 0.0;
            if (xint) {
                if (c + 1 <= NX - 1) {
                    gxd = -gl[((c + 1) * 2 + 0) * M + m] - gRmx[m];
                    gxu = -gl[((c + 1) * 2 + 1) * M + m] - gRpx[m];
                } else {
                    gxd = -gRmx[m];
                    gxu = -gRpx[m];
                }
            }
            if (active) GXs_n[m] = GXu_prev[m] + gxd;
            GXu_prev[m] = gxu;
        }
        if (active) {
#pragma unroll
            for (int m = 0; m < M; ++m) {
                gy[(c * 2 + 0) * M + m] = GYd_r[m];
                gy[(c * 2 + 1) * M + m] = GYu_r[m];
            }
        }
        __syncthreads();  // D

        // ---------------- phase 5: update cell row r = s-2 ----------------
        const int r = s - 2;
        const bool upd = V5 ? (c >= MBC && c < MBC + MX && r >= MBC && r < MBC + MX) : (c <= NX - 2);
        if (active && r >= R0 && r < R1 && upd) {
            const double* fxr = s_fx + ((r % 3) * PPB + pl) * NX * 2 * M;
#pragma unroll
            for (int m = 0; m < M; ++m) {
                const double fxm1 = fxr[((c + 1) * 2 + 0) * M + m];
                const double fxp0 = fxr[(c * 2 + 1) * M + m];
                const double gyu_l = (c >= 1) ? gy[((c - 1) * 2 + 1) * M + m] : 0.0;
                const double gyd_r = gy[((c + 1) * 2 + 0) * M + m];
                const double fmv = (fxm1 + GYu_r[m]) + gyd_r;       // fm(i+1, j)
                const double fpv = (fxp0 + gyu_l) + GYd_r[m];       // fp(i, j)
                const double gmv = GXS(s - 1)[m] + FYm_cur[m];      // gm(i, j+1)
                const double gpv = GXS(r)[m] + FYp_prev[m];         // gp(i, j)
                double qv;
                if constexpr (CAPA)  // clawpack46_step2_wrap.f:118-121
                    qv = QR(r, c)[m] - (dtdx * (fmv - fpv) + dtdy * (gmv - gpv)) / AUXV(0, c, r);
                else
                    qv = QR(r, c)[m] - dtdx * (fmv - fpv) - dtdy * (gmv - gpv);
                q[((int64_t)m * NY + r) * NX + c] = qv;
                if (a.treg) {
                    // time-sync: boundary fluctuations scaled by dt and the edge
                    // length (clawpack46_time_sync_accumulate_waves); each
                    // register element has exactly one writer
                    const RegLayout RL{MX, MX, M};
                    double* R = a.treg + (int64_t)slot * a.treg_stride;
                    const int i = c - MBC + 1, j = r - MBC + 1;
                    const double dty = pdt * meta.dy, dtx = pdt * meta.dx;
                    if (j >= 1 && j <= MX) {
                        const int k = (j - 1) + MX * m;
                        if (i == 1) R[RL.fp(0) + k] = R[RL.fp(0) + k] - dty * fpv;
                        if (i == 0) R[RL.fm(0) + k] = R[RL.fm(0) + k] + dty * fmv;         // fm(1, j)
                        if (i == MX) R[RL.fm(1) + k] = R[RL.fm(1) + k] + dty * fmv;        // fm(mx+1, j)
                        if (i == MX + 1) R[RL.fp(1) + k] = R[RL.fp(1) + k] - dty * fpv;    // fp(mx+1, j)
                    }
                    if (i >= 1 && i <= MX) {
                        const int k = (i - 1) + MX * m;
                        if (j == 1) R[RL.gp(0) + k] = R[RL.gp(0) + k] - dtx * gpv;
                        if (j == 0) R[RL.gm(0) + k] = R[RL.gm(0) + k] + dtx * gmv;         // gm(i, 1)
                        if (j == MX) R[RL.gm(1) + k] = R[RL.gm(1) + k] + dtx * gmv;        // gm(i, my+1)
                        if (j == MX + 1) R[RL.gp(1) + k] = R[RL.gp(1) + k] - dtx * gpv;    // gp(i, my+1)
                    }
                }
            }
        }
        // rotate per-row registers
#pragma unroll
        for (int m = 0; m < M; ++m) {
            FYp_prev[m] = FYp_cur[m];
        }
    }

    // ---- CFL: warp max, one atomic per warp (per solve of a serving launch) ----
    if (a.desc) {
        // patches of different solves share warps: reduce over the lanes of each
        // solve (max of the non-negative bit patterns, high word then low word)
        const unsigned grp = __match_any_sync(0xffffffffu, req);
        const unsigned long long b = (unsigned long long)__double_as_longlong(active ? cfl : 0.0);
        const unsigned hi = __reduce_max_sync(grp, (unsigned)(b >> 32));
        const unsigned lo = __reduce_max_sync(grp, ((unsigned)(b >> 32) == hi) ? (unsigned)b : 0u);
        if (req >= 0 && (t & 31) == __ffs(grp) - 1 && a.cfl_out)
            atomicMax(a.cfl_out + req, ((unsigned long long)hi << 32) | lo);
        return;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) cfl = nanmax(cfl, __shfl_xor_sync(0xffffffffu, cfl, off));
    if ((t & 31) == 0 && a.cfl_out) atomic_max_nonneg(a.cfl_out, cfl);
}

// Copy the patches slots[0..n) of arena src into the same slots of dst
// (two-double vectors; the slot stride is a multiple of 256 bytes).
__global__ void copy_slots_kernel(const int32_t* __restrict__ slots, int n, const double* __restrict__ src,
                                  double* __restrict__ dst, int64_t stride) {
    const int64_t half = stride / 2;
    const int64_t total = (int64_t)n * half;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int p = (int)(k / half);
        const int64_t off = (int64_t)slots[p] * half + (k - (int64_t)p * half);
        reinterpret_cast<double2*>(dst)[off] = reinterpret_cast<const double2*>(src)[off];
    }
}

// ---------------------------------------------------------------------------
// Host-side launcher: dispatch on (solver, mx, aux kind).
// ---------------------------------------------------------------------------
namespace {

// A launch of G CTAs on an SM array that holds W at once ends with a wave of
// G mod W CTAs that lasts a whole patch sweep.  When that tail is small, its
// patches are split into nb row bands (nb CTAs of about 1/nb of a sweep each,
// nb * tail <= W, at most 4), so the last wave is shorter; the full waves run
// as before.  A launch of at most W / 2 CTAs is all tail.  Returns the number
// of leading unbanded CTAs and sets nb, or returns -1 when banding the tail
// does not pay.
int tail_plan(int groups, int per_wave, int* nb) {
    if (per_wave <= 0 || groups <= 0 || (groups <= per_wave && 2 * groups > per_wave)) return -1;
    const int tail = groups % per_wave;
    if (tail == 0) return -1;
    const int k = std::min(4, per_wave / tail);
    if (k < 2) return -1;
    *nb = k;
    return groups - tail;
}

template <class SOL, int MX, int MBC, int AUXK, int NAUX, int TPB, int LIM>
cudaError_t launch_one(const StepArgs& a, cudaStream_t st) {
    constexpr int NX = MX + 2 * MBC;
    constexpr int PPB = TPB / NX;
    static_assert(PPB >= 1, "patch wider than the CTA");
    using L = StepSmem<NX, NX, PPB, SOL::M, SOL::W, NAUX, AUXK == AUX_SWIRL, SOL::NC>;
    const size_t bytes = (size_t)L::TOTAL * sizeof(double);
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(step_kernel<SOL, MX, MBC, AUXK, NAUX, TPB, LIM>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    if (a.nbands <= 1 && a.qtail && !a.desc && !a.treg && a.npatches > 0) {
        // CTAs one SM array holds at once (the Roe forms: one per SM)
        static int per_wave = -1;
        if (per_wave < 0) {
            int dev = 0, sms = 0, occ = 0;
            if (cudaGetDevice(&dev) != cudaSuccess ||
                cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, step_kernel<SOL, MX, MBC, AUXK, NAUX, TPB, LIM>,
                                                              TPB, bytes) != cudaSuccess)
                return cudaErrorInvalidValue;
            per_wave = sms * occ;
        }
        int tb = 1;
        const int b0 = tail_plan((a.npatches + PPB - 1) / PPB, per_wave, &tb);
        if (b0 >= 0) {
            const int first = b0 * PPB, ntail = a.npatches - first;
            const int64_t vecs = (int64_t)ntail * (a.q_stride / 2);
            const int cb = (int)std::min<int64_t>((vecs + 255) / 256, 4096);
            copy_slots_kernel<<<cb, 256, 0, st>>>(a.slots + first, ntail, a.q, a.qtail, a.q_stride);
            StepArgs t = a;
            t.qsrc = a.qtail;
            t.nbands = tb;
            t.band_first = b0;
            t.qtail = nullptr;
            return launch_one<SOL, MX, MBC, AUXK, NAUX, TPB, LIM>(t, st);
        }
    }
    const int nb = a.nbands > 1 ? a.nbands : 1;
    if (nb > 1 && (!a.qsrc || a.qsrc == a.q || nb > 4 || a.desc)) return cudaErrorInvalidValue;
    if (a.desc && a.treg) return cudaErrorInvalidValue;
    const int groups = (a.npatches + PPB - 1) / PPB;
    const int b0 = nb > 1 ? a.band_first : 0;
    if (b0 < 0 || b0 > groups) return cudaErrorInvalidValue;
    const int blocks = b0 + (groups - b0) * nb;
    if (blocks == 0) return cudaSuccess;
    step_kernel<SOL, MX, MBC, AUXK, NAUX, TPB, LIM><<<blocks, TPB, bytes, st>>>(a);
    return cudaGetLastError();
}

// CTA size: the Roe systems run at the register limit (255 per thread), one
// 256-thread CTA per SM, which packs 7 patches of mx = 32 (252 of 256 threads
// busy) where 128 threads held 3 (108 busy) and left the last CTAs of a level
// as a second wave; 1.4-1.65x faster on levels of 1,024 patches of mx = 32.
// Scalar advection keeps 128 threads (its per-patch aux and stream-function
// tables would not fit 256 threads' worth of patches of mx = 64 in shared memory).
// The Roe systems with order (2, 2) and the MC limiter on every wave (the
// benchmarked configurations) get the method fixed at compile time.
template <class SOL, int MX, int AUXK, int NAUX, int TPB>
cudaError_t launch_lim(const StepArgs& a, cudaStream_t st) {
    if constexpr (SOL::M > 1) {
        bool mc = a.order0 == 2 && a.order1 == 2;
        for (int mw = 0; mw < SOL::W; ++mw) mc = mc && a.mthlim[mw] == 4;
        if (mc) return launch_one<SOL, MX, 2, AUXK, NAUX, TPB, 4>(a, st);
    }
    return launch_one<SOL, MX, 2, AUXK, NAUX, TPB, 0>(a, st);
}

template <class SOL, int AUXK, int NAUX>
cudaError_t launch_mx(int mx, int mbc, const StepArgs& a, cudaStream_t st) {
    constexpr int TPB = SOL::M > 1 ? 256 : 128;
    if (mbc != 2) return cudaErrorInvalidValue;
    switch (mx) {
        case 8: return launch_lim<SOL, 8, AUXK, NAUX, TPB>(a, st);
        case 16: return launch_lim<SOL, 16, AUXK, NAUX, TPB>(a, st);
        case 32: return launch_lim<SOL, 32, AUXK, NAUX, TPB>(a, st);
        case 64: return launch_lim<SOL, 64, AUXK, NAUX, TPB>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

// Returns cudaErrorInvalidValue for an unsupported (solver, mx, mbc, aux) combination.
cudaError_t launch_step(int solver, int aux_kind, int mwaves, int mx, int my, int mbc,
                        const StepArgs& a, cudaStream_t st, int claw_version) {
    if (mx != my) return cudaErrorInvalidValue;
    // clawpack 5 exists in this form for the manifold advection solver only
    if (claw_version == 5 && solver != SOLVER_ADVECTION_MANIFOLD) return cudaErrorInvalidValue;
    switch (solver) {
        case SOLVER_ADVECTION:
            if (mwaves != 1) return cudaErrorInvalidValue;
            if (aux_kind == AUX_SWIRL) return launch_mx<AdvectionSolver<1>, AUX_SWIRL, 2>(mx, mbc, a, st);
            if (aux_kind == AUX_STORED && a.maux >= 2)
                return launch_mx<AdvectionSolver<1>, AUX_STORED, 2>(mx, mbc, a, st);
            return cudaErrorInvalidValue;
        case SOLVER_SWE_ROE:
            if (mwaves != 3 || aux_kind != AUX_NONE) return cudaErrorInvalidValue;
            return launch_mx<SweRoeSolver, AUX_NONE, 0>(mx, mbc, a, st);
        case SOLVER_EULER4_ROE:
            if (mwaves != 4 || aux_kind != AUX_NONE) return cudaErrorInvalidValue;
            return launch_mx<Euler4RoeSolver, AUX_NONE, 0>(mx, mbc, a, st);
        case SOLVER_ADVECTION_MANIFOLD:
            // capacity in aux(1), edge velocities in aux(2:3)
            if (mwaves != 1 || aux_kind != AUX_STORED || a.maux < 3) return cudaErrorInvalidValue;
            if (claw_version == 5) return launch_mx<AdvectionManifoldSolver<1, true>, AUX_STORED, 3>(mx, mbc, a, st);
            return launch_mx<AdvectionManifoldSolver<1>, AUX_STORED, 3>(mx, mbc, a, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace fcb
