// Warp-synchronous form of the clawpack 4.6 patch update (same arithmetic as
// fcb_step.cu, same reference and the same operation order).
//
// Mapping: a patch of NX = mx + 2 mbc columns is handled by L = NX / CPL lanes,
// CPL consecutive columns per lane; G = floor(32 / L) patches share one warp.
// The rows stream through the same two-row pipeline as fcb_step.cu, but every
// neighbour exchange (left state of an x-interface, neighbouring waves for the
// limiter, transverse parts, flux terms of the update) is a warp shuffle, so
// there is no CTA barrier and no shared-memory round trip.
//
// Swirl velocities (swirl/user_4.6/b4step2.f, swirl/psi.f): on the dyadic
// unit-square mesh xll(i) + dx == xll(i+1) exactly, so psi(xll, yll+dy) and
// psi(xll+dx, yll) are the node values of the neighbouring nodes and one psi
// per node reproduces the reference's three evaluations per cell bit for bit.
// The host checks that the mesh is dyadic before selecting this kernel.
#include <cuda_runtime.h>

#include "fcb_device.h"
#include "fcb_solvers.cuh"

namespace fcb {

namespace {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ void atomic_max_nonneg_w(unsigned long long* p, double v) {
    atomicMax(p, (unsigned long long)__double_as_longlong(v));
}

template <int N>
__device__ __forceinline__ void shfl_up_arr(const double (&src)[N], double (&dst)[N]) {
#pragma unroll
    for (int i = 0; i < N; ++i) dst[i] = __shfl_up_sync(FULL, src[i], 1);
}
template <int N>
__device__ __forceinline__ void shfl_down_arr(const double (&src)[N], double (&dst)[N]) {
#pragma unroll
    for (int i = 0; i < N; ++i) dst[i] = __shfl_down_sync(FULL, src[i], 1);
}

}  // namespace

template <class SOL, int MX, int MBC, int CPL>
__global__ void __launch_bounds__(128) step_kernel_warp(const StepArgs a) {
    constexpr int M = SOL::M;
    constexpr int W = SOL::W;
    constexpr int NX = MX + 2 * MBC;
    constexpr int NY = NX;
    constexpr int L = NX / CPL;  // lanes per patch
    static_assert(NX % CPL == 0, "CPL must divide NX");
    static_assert(L <= 32, "patch wider than a warp");
    constexpr int G = 32 / L;    // patches per warp
    constexpr int WPB = 4;       // warps per CTA
    constexpr double pi = 3.141592653589793;  // 4*atan(1) in double precision

    // per patch: SX2 at node columns 0..NX, SY2 at node rows 0..NY
    __shared__ double s_tab[WPB][G][2][NX + 1];

    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane / L, k = lane - g * L;
    const int pg = (blockIdx.x * WPB + w) * G + g;
    const bool active = (g < G) && (pg < a.npatches);
    const int slot = active ? a.slots[pg] : 0;
    const PatchMeta meta = active ? a.meta[slot] : PatchMeta{0, 0, 1, 1, 0, 0};
    double* __restrict__ q = a.q + (int64_t)slot * a.q_stride;
    double* __restrict__ qlast = a.qlast + (int64_t)slot * a.q_stride;
    const bool save_last = active && (meta.flags & PATCH_SAVE_LAST);
    const double dtdx = step_dt(a, meta.level) / meta.dx, dtdy = step_dt(a, meta.level) / meta.dy;
    const double dtdxave = 0.5 * (dtdx + dtdx), dtdyave = 0.5 * (dtdy + dtdy);
    const double vty = step_vt(a, meta.level) / meta.dy, vtx = step_vt(a, meta.level) / meta.dx;
    const SOL sol{a.grav, a.gamma, a.gamma1};
    const int c0 = k * CPL;  // first own column

    // ---- sine tables ----
    if (active) {
        double* tx = &s_tab[w][g < G ? g : 0][0][0];
        double* ty = &s_tab[w][g < G ? g : 0][1][0];
        for (int n = k; n <= NX; n += L) {
            const double x = meta.xlower + (double)(n - MBC) * meta.dx;
            const double y = meta.ylower + (double)(n - MBC) * meta.dy;
            const double sx = sin(pi * x), sy = sin(pi * y);
            tx[n] = sx * sx;
            ty[n] = sy * sy;
        }
    }
    __syncwarp();
    const double* TX = &s_tab[w][g < G ? g : 0][0][0];
    const double* TY = &s_tab[w][g < G ? g : 0][1][0];

    // ---- per-column state ----
    double q_m2[CPL][M], q_m1[CPL][M], q_n[CPL][M];
    double Po[CPL], PoR;               // psi at node row s (own columns, right neighbour node)
    double u_m2[CPL], u_m1[CPL], u_s[CPL];
    double v_s[CPL], v_s1[CPL];        // v at rows s, s+1
    double yw_f[CPL][W][M], ys_f[CPL][W], yam_f[CPL][M], yap_f[CPL][M], ydotl[CPL][W];
    typename SOL::Roe yR_f[CPL];
    double gRm_prev[CPL][M], gRp_prev[CPL][M], FYp_prev[CPL][M], GXu_prev[CPL][M];
    double GXs_m2[CPL][M], GXs_m1[CPL][M];
    double FXm[3][CPL][M], FXp[3][CPL][M];  // x-row fluxes of rows s, s-1, s-2 (ring)
    double cfl = 0.0;
#pragma unroll
    for (int j = 0; j < CPL; ++j) {
        Po[j] = u_m2[j] = u_m1[j] = u_s[j] = v_s[j] = v_s1[j] = 0.0;
#pragma unroll
        for (int m = 0; m < M; ++m) {
            q_m2[j][m] = q_m1[j][m] = q_n[j][m] = 0.0;
            yam_f[j][m] = yap_f[j][m] = 0.0;
            gRm_prev[j][m] = gRp_prev[j][m] = FYp_prev[j][m] = GXu_prev[j][m] = 0.0;
            GXs_m2[j][m] = GXs_m1[j][m] = 0.0;
#pragma unroll
            for (int r = 0; r < 3; ++r) FXm[r][j][m] = FXp[r][j][m] = 0.0;
        }
#pragma unroll
        for (int mw = 0; mw < W; ++mw) {
            ys_f[j][mw] = ydotl[j][mw] = 0.0;
#pragma unroll
            for (int m = 0; m < M; ++m) yw_f[j][mw][m] = 0.0;
        }
        yR_f[j] = typename SOL::Roe{};
    }
    // node row 0 and v(., 0)
    PoR = 0.0;
    {
        const double ty0 = active ? TY[0] : 0.0;
#pragma unroll
        for (int j = 0; j < CPL; ++j) Po[j] = active ? (TX[c0 + j] * ty0) / pi : 0.0;
        double nb = __shfl_down_sync(FULL, Po[0], 1);
        if (k == L - 1) nb = active ? (TX[NX] * ty0) / pi : 0.0;
        PoR = nb;
#pragma unroll
        for (int j = 0; j < CPL; ++j) {
            const double right = (j + 1 < CPL) ? Po[j + 1] : PoR;
            v_s[j] = -vtx * (right - Po[j]);
        }
    }

    for (int s = 0; s <= NY; ++s) {
        // ------------- node row s+1: u(., s), v(., s+1) -------------
        {
            double Pn[CPL];
            const double ty = (active && s + 1 <= NY) ? TY[s + 1] : 0.0;
#pragma unroll
            for (int j = 0; j < CPL; ++j) Pn[j] = (active && s + 1 <= NY) ? (TX[c0 + j] * ty) / pi : 0.0;
            double PnR = __shfl_down_sync(FULL, Pn[0], 1);
            if (k == L - 1) PnR = (active && s + 1 <= NY) ? (TX[NX] * ty) / pi : 0.0;
#pragma unroll
            for (int j = 0; j < CPL; ++j) {
                u_s[j] = vty * (Pn[j] - Po[j]);
                const double right = (j + 1 < CPL) ? Pn[j + 1] : PnR;
                v_s1[j] = -vtx * (right - Pn[j]);
                Po[j] = Pn[j];
            }
            PoR = PnR;
        }

        // ------------- load row s; raw y-interface s -------------
        double yw_n[CPL][W][M], ys_n[CPL][W], yam_n[CPL][M], yap_n[CPL][M], ydotr[CPL][W];
        typename SOL::Roe yR_n[CPL];
#pragma unroll
        for (int j = 0; j < CPL; ++j) {
            const int c = c0 + j;
            if (s < NY && active) {
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    const int64_t kk = ((int64_t)m * NY + s) * NX + c;
                    q_n[j][m] = q[kk];
                    if (save_last) qlast[kk] = q_n[j][m];
                }
            }
#pragma unroll
            for (int mw = 0; mw < W; ++mw) {
                ys_n[j][mw] = 0.0; ydotr[j][mw] = 0.0;
#pragma unroll
                for (int m = 0; m < M; ++m) yw_n[j][mw][m] = 0.0;
            }
#pragma unroll
            for (int m = 0; m < M; ++m) yam_n[j][m] = yap_n[j][m] = 0.0;
            yR_n[j] = typename SOL::Roe{};
            if (active && s < NY && s >= 1 && c >= 1 && c <= NX - 2) {
                sol.rpn2(2, q_m1[j], q_n[j], v_s[j], yw_n[j], ys_n[j], yam_n[j], yap_n[j], yR_n[j]);
#pragma unroll
                for (int mw = 0; mw < W; ++mw) {
                    double d = yw_f[j][mw][0] * yw_n[j][mw][0];
#pragma unroll
                    for (int m = 1; m < M; ++m) d = d + yw_f[j][mw][m] * yw_n[j][mw][m];
                    ydotr[j][mw] = d;
                }
            }
        }

        // ------------- raw x-interfaces (c, s) -------------
        const bool xrow = active && s >= 1 && s <= NY - 2;
        double qleft[M];
        {
            double last[M];
#pragma unroll
            for (int m = 0; m < M; ++m) last[m] = q_n[CPL - 1][m];
            shfl_up_arr(last, qleft);
        }
        double xw[CPL][W][M], xs[CPL][W], xam[CPL][M], xap[CPL][M];
        typename SOL::Roe xR[CPL];
#pragma unroll
        for (int j = 0; j < CPL; ++j) {
            const int c = c0 + j;
#pragma unroll
            for (int mw = 0; mw < W; ++mw) {
                xs[j][mw] = 0.0;
#pragma unroll
                for (int m = 0; m < M; ++m) xw[j][mw][m] = 0.0;
            }
#pragma unroll
            for (int m = 0; m < M; ++m) xam[j][m] = xap[j][m] = 0.0;
            xR[j] = typename SOL::Roe{};
            if (xrow && c >= 1) {
                const double* qL = (j == 0) ? qleft : q_n[j - 1];
                sol.rpn2(1, qL, q_n[j], u_s[j], xw[j], xs[j], xam[j], xap[j], xR[j]);
                if (c >= MBC && c <= MBC + MX) {
#pragma unroll
                    for (int mw = 0; mw < W; ++mw) cfl = nanmax(nanmax(cfl, dtdx * xs[j][mw]), -dtdx * xs[j][mw]);
                }
            }
        }
        // neighbour raw waves for the limiter (lane-1's last column, lane+1's first column)
        double wl[W][M], wr[W][M];
#pragma unroll
        for (int mw = 0; mw < W; ++mw)
#pragma unroll
            for (int m = 0; m < M; ++m) {
                wl[mw][m] = __shfl_up_sync(FULL, xw[CPL - 1][mw][m], 1);
                wr[mw][m] = __shfl_down_sync(FULL, xw[0][mw][m], 1);
            }
        // v(c-1, s), v(c-1, s+1) for the first own column
        const double vl_s = __shfl_up_sync(FULL, v_s[CPL - 1], 1);
        const double vl_s1 = __shfl_up_sync(FULL, v_s1[CPL - 1], 1);
        // u(c+1, s-2), u(c+1, s-1) for the last own column (y transverse)
        const double ur_m2 = __shfl_down_sync(FULL, u_m2[0], 1);
        const double ur_m1 = __shfl_down_sync(FULL, u_m1[0], 1);

        // ------------- x: limiter, corrections, transverse -------------
        double gLm[CPL][M], gLp[CPL][M], gRmx[CPL][M], gRpx[CPL][M];
        const int ring = s % 3;
#pragma unroll
        for (int j = 0; j < CPL; ++j) {
            const int c = c0 + j;
#pragma unroll
            for (int m = 0; m < M; ++m) {
                gLm[j][m] = gLp[j][m] = gRmx[j][m] = gRpx[j][m] = 0.0;
                FXm[ring][j][m] = 0.0;
                FXp[ring][j][m] = 0.0;
            }
            if (!(xrow && c >= 1)) continue;
            double cq[M];
#pragma unroll
            for (int m = 0; m < M; ++m) cq[m] = 0.0;
            if (a.order0 == 2) {
                double wv[W][M];
#pragma unroll
                for (int mw = 0; mw < W; ++mw)
#pragma unroll
                    for (int m = 0; m < M; ++m) wv[mw][m] = xw[j][mw][m];
                if (c >= MBC && c <= MBC + MX) {
#pragma unroll
                    for (int mw = 0; mw < W; ++mw) {
                        if (a.mthlim[mw] == 0) continue;
                        double wn2 = 0.0, dl = 0.0, dr = 0.0;
#pragma unroll
                        for (int m = 0; m < M; ++m) {
                            const double wc = xw[j][mw][m];
                            const double wlv = (j == 0) ? wl[mw][m] : xw[j > 0 ? j - 1 : 0][mw][m];
                            const double wrv = (j == CPL - 1) ? wr[mw][m] : xw[j + 1 < CPL ? j + 1 : j][mw][m];
                            if (m == 0) {
                                wn2 = wc * wc;
                                dl = wlv * wc;
                                dr = wc * wrv;
                            } else {
                                wn2 = wn2 + wc * wc;
                                dl = dl + wlv * wc;
                                dr = dr + wc * wrv;
                            }
                        }
                        if (wn2 == 0.0) continue;
                        const double r = (xs[j][mw] > 0.0) ? dl / wn2 : dr / wn2;
                        const double phi = limiter_phi(a.mthlim[mw], r);
#pragma unroll
                        for (int m = 0; m < M; ++m) wv[mw][m] = phi * wv[mw][m];
                    }
                }
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    double acc;
                    {
                        const double as = fabs(xs[j][0]);
                        acc = as * (1.0 - as * dtdxave) * wv[0][m];
                    }
#pragma unroll
                    for (int mw = 1; mw < W; ++mw) {
                        const double as = fabs(xs[j][mw]);
                        acc = acc + as * (1.0 - as * dtdxave) * wv[mw][m];
                    }
                    cq[m] = acc;
                }
            }
            double am[M], ap[M];
#pragma unroll
            for (int m = 0; m < M; ++m) {
                double fmv = (c <= NX - 2) ? xam[j][m] : 0.0;
                double fpv = (c <= NX - 2) ? -xap[j][m] : 0.0;
                if (a.order0 == 2) { fmv = fmv + 0.5 * cq[m]; fpv = fpv + 0.5 * cq[m]; }
                FXm[ring][j][m] = fmv;
                FXp[ring][j][m] = fpv;
                am[m] = xam[j][m]; ap[m] = xap[j][m];
                if (a.order0 > 1 && a.order1 == 2 && c <= NX - 2) { am[m] = am[m] + cq[m]; ap[m] = ap[m] - cq[m]; }
            }
            if (a.order1 > 0) {
                double bm[M], bp[M];
                const double v_l = (j == 0) ? vl_s : v_s[j > 0 ? j - 1 : 0];
                const double v_l1 = (j == 0) ? vl_s1 : v_s1[j > 0 ? j - 1 : 0];
                sol.rpt2(1, am, xR[j], v_l, v_l1, bm, bp);
#pragma unroll
                for (int m = 0; m < M; ++m) { gLm[j][m] = 0.5 * dtdx * bm[m]; gLp[j][m] = 0.5 * dtdx * bp[m]; }
                sol.rpt2(1, ap, xR[j], v_s[j], v_s1[j], bm, bp);
#pragma unroll
                for (int m = 0; m < M; ++m) { gRmx[j][m] = 0.5 * dtdx * bm[m]; gRpx[j][m] = 0.5 * dtdx * bp[m]; }
            }
        }
        // gL of the column to the right (lane+1's first column for the last own column)
        double gLm_r[M], gLp_r[M];
        shfl_down_arr(gLm[0], gLm_r);
        shfl_down_arr(gLp[0], gLp_r);
        double GXs_n[CPL][M];
#pragma unroll
        for (int j = 0; j < CPL; ++j) {
            const int c = c0 + j;
#pragma unroll
            for (int m = 0; m < M; ++m) {
                double gxd = 0.0, gxu = 0.0;
                if (xrow && c >= 1) {
                    if (c + 1 <= NX - 1) {
                        const double glm = (j == CPL - 1) ? gLm_r[m] : gLm[j + 1 < CPL ? j + 1 : j][m];
                        const double glp = (j == CPL - 1) ? gLp_r[m] : gLp[j + 1 < CPL ? j + 1 : j][m];
                        gxd = -glm - gRmx[j][m];
                        gxu = -glp - gRpx[j][m];
                    } else {
                        gxd = -gRmx[j][m];
                        gxu = -gRpx[j][m];
                    }
                }
                GXs_n[j][m] = GXu_prev[j][m] + gxd;
                GXu_prev[j][m] = gxu;
            }
        }

        // ------------- y: finalize interface f = s-1 (own columns) -------------
        const int f = s - 1;
        double FYm_cur[CPL][M], FYp_cur[CPL][M], GYd_r[CPL][M], GYu_r[CPL][M];
#pragma unroll
        for (int j = 0; j < CPL; ++j) {
            const int c = c0 + j;
#pragma unroll
            for (int m = 0; m < M; ++m) FYm_cur[j][m] = FYp_cur[j][m] = GYd_r[j][m] = GYu_r[j][m] = 0.0;
            if (!(active && c >= 1 && c <= NX - 2 && f >= 1)) continue;
            double wv[W][M];
#pragma unroll
            for (int mw = 0; mw < W; ++mw)
#pragma unroll
                for (int m = 0; m < M; ++m) wv[mw][m] = yw_f[j][mw][m];
            if (f >= MBC && f <= MBC + MX) {
#pragma unroll
                for (int mw = 0; mw < W; ++mw) cfl = nanmax(nanmax(cfl, dtdy * ys_f[j][mw]), -dtdy * ys_f[j][mw]);
            }
            double cq[M];
#pragma unroll
            for (int m = 0; m < M; ++m) cq[m] = 0.0;
            if (a.order0 == 2) {
                if (f >= MBC && f <= MBC + MX) {
#pragma unroll
                    for (int mw = 0; mw < W; ++mw) {
                        if (a.mthlim[mw] == 0) continue;
                        double wn2 = yw_f[j][mw][0] * yw_f[j][mw][0];
#pragma unroll
                        for (int m = 1; m < M; ++m) wn2 = wn2 + yw_f[j][mw][m] * yw_f[j][mw][m];
                        if (wn2 == 0.0) continue;
                        const double r = (ys_f[j][mw] > 0.0) ? ydotl[j][mw] / wn2 : ydotr[j][mw] / wn2;
                        const double phi = limiter_phi(a.mthlim[mw], r);
#pragma unroll
                        for (int m = 0; m < M; ++m) wv[mw][m] = phi * wv[mw][m];
                    }
                }
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    double acc;
                    {
                        const double as = fabs(ys_f[j][0]);
                        acc = as * (1.0 - as * dtdyave) * wv[0][m];
                    }
#pragma unroll
                    for (int mw = 1; mw < W; ++mw) {
                        const double as = fabs(ys_f[j][mw]);
                        acc = acc + as * (1.0 - as * dtdyave) * wv[mw][m];
                    }
                    cq[m] = acc;
                }
            }
            double am[M], ap[M];
#pragma unroll
            for (int m = 0; m < M; ++m) {
                double fmv = (f <= NY - 2) ? yam_f[j][m] : 0.0;
                double fpv = (f <= NY - 2) ? -yap_f[j][m] : 0.0;
                if (a.order0 == 2) { fmv = fmv + 0.5 * cq[m]; fpv = fpv + 0.5 * cq[m]; }
                FYm_cur[j][m] = fmv;
                FYp_cur[j][m] = fpv;
                am[m] = yam_f[j][m]; ap[m] = yap_f[j][m];
                if (a.order0 > 1 && a.order1 == 2 && f <= NY - 2) { am[m] = am[m] + cq[m]; ap[m] = ap[m] - cq[m]; }
            }
            double gLmy[M], gLpy[M], gRmy[M], gRpy[M];
#pragma unroll
            for (int m = 0; m < M; ++m) gLmy[m] = gLpy[m] = gRmy[m] = gRpy[m] = 0.0;
            if (a.order1 > 0) {
                double bm[M], bp[M];
                const double u_r_m2 = (j == CPL - 1) ? ur_m2 : u_m2[j + 1 < CPL ? j + 1 : j];
                const double u_r_m1 = (j == CPL - 1) ? ur_m1 : u_m1[j + 1 < CPL ? j + 1 : j];
                // imp = 1: u at columns c, c+1, row f-1 = s-2; imp = 2: row f = s-1
                sol.rpt2(2, am, yR_f[j], u_m2[j], u_r_m2, bm, bp);
#pragma unroll
                for (int m = 0; m < M; ++m) { gLmy[m] = 0.5 * dtdy * bm[m]; gLpy[m] = 0.5 * dtdy * bp[m]; }
                sol.rpt2(2, ap, yR_f[j], u_m1[j], u_r_m1, bm, bp);
#pragma unroll
                for (int m = 0; m < M; ++m) { gRmy[m] = 0.5 * dtdy * bm[m]; gRpy[m] = 0.5 * dtdy * bp[m]; }
            }
            if (f - 1 >= 1) {
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    GYd_r[j][m] = -gLmy[m] - gRm_prev[j][m];
                    GYu_r[j][m] = -gLpy[m] - gRp_prev[j][m];
                }
            }
#pragma unroll
            for (int m = 0; m < M; ++m) { gRm_prev[j][m] = gRmy[m]; gRp_prev[j][m] = gRpy[m]; }
        }

        // ------------- update cell row r = s-2 -------------
        const int r = s - 2;
        const int ringr = (s + 1) % 3;  // == (s-2) % 3
        double fxm_r[M], gyd_r[M], gyu_l[M];
        shfl_down_arr(FXm[ringr][0], fxm_r);
        shfl_down_arr(GYd_r[0], gyd_r);
        shfl_up_arr(GYu_r[CPL - 1], gyu_l);
        if (active && r >= 0 && r <= NY - 2) {
#pragma unroll
            for (int j = 0; j < CPL; ++j) {
                const int c = c0 + j;
                if (c > NX - 2) continue;
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    const double fxm1 = (j == CPL - 1) ? fxm_r[m] : FXm[ringr][j + 1 < CPL ? j + 1 : j][m];
                    const double gydr = (j == CPL - 1) ? gyd_r[m] : GYd_r[j + 1 < CPL ? j + 1 : j][m];
                    const double gyul = (c >= 1) ? ((j == 0) ? gyu_l[m] : GYu_r[j > 0 ? j - 1 : 0][m]) : 0.0;
                    const double fmv = (fxm1 + GYu_r[j][m]) + gydr;
                    const double fpv = (FXp[ringr][j][m] + gyul) + GYd_r[j][m];
                    const double gmv = GXs_m1[j][m] + FYm_cur[j][m];
                    const double gpv = GXs_m2[j][m] + FYp_prev[j][m];
                    q[((int64_t)m * NY + r) * NX + c] = q_m2[j][m] - dtdx * (fmv - fpv) - dtdy * (gmv - gpv);
                }
            }
        }

        // ------------- rotate -------------
#pragma unroll
        for (int j = 0; j < CPL; ++j) {
#pragma unroll
            for (int m = 0; m < M; ++m) {
                q_m2[j][m] = q_m1[j][m];
                q_m1[j][m] = q_n[j][m];
                GXs_m2[j][m] = GXs_m1[j][m];
                GXs_m1[j][m] = GXs_n[j][m];
                FYp_prev[j][m] = FYp_cur[j][m];
                yam_f[j][m] = yam_n[j][m];
                yap_f[j][m] = yap_n[j][m];
            }
#pragma unroll
            for (int mw = 0; mw < W; ++mw) {
                ydotl[j][mw] = ydotr[j][mw];
                ys_f[j][mw] = ys_n[j][mw];
#pragma unroll
                for (int m = 0; m < M; ++m) yw_f[j][mw][m] = yw_n[j][mw][m];
            }
            yR_f[j] = yR_n[j];
            u_m2[j] = u_m1[j];
            u_m1[j] = u_s[j];
            v_s[j] = v_s1[j];
        }
    }

#pragma unroll
    for (int off = 16; off > 0; off >>= 1) cfl = nanmax(cfl, __shfl_xor_sync(FULL, cfl, off));
    if (lane == 0 && a.cfl_out) atomic_max_nonneg_w(a.cfl_out, cfl);
}

namespace {
template <class SOL, int MX, int MBC, int CPL>
cudaError_t launch_w(const StepArgs& a, cudaStream_t st) {
    constexpr int NX = MX + 2 * MBC;
    constexpr int G = 32 / (NX / CPL);
    constexpr int per_block = 4 * G;
    const int blocks = (a.npatches + per_block - 1) / per_block;
    if (blocks == 0) return cudaSuccess;
    step_kernel_warp<SOL, MX, MBC, CPL><<<blocks, 128, 0, st>>>(a);
    return cudaGetLastError();
}
}  // namespace

// Warp form for the swirl advection case; returns cudaErrorNotSupported when
// (mx, mbc) has no warp mapping, so the caller can fall back to the CTA form.
cudaError_t launch_step_warp_swirl(int mx, int mbc, const StepArgs& a, cudaStream_t st) {
    if (mbc != 2) return cudaErrorNotSupported;
    switch (mx) {
        case 8: return launch_w<AdvectionSolver<1>, 8, 2, 2>(a, st);    // 6 lanes/patch, 5 patches/warp
        case 16: return launch_w<AdvectionSolver<1>, 16, 2, 2>(a, st);  // 10 lanes/patch, 3 patches/warp
        case 32: return launch_w<AdvectionSolver<1>, 32, 2, 3>(a, st);  // 12 lanes/patch, 2 patches/warp
        default: return cudaErrorNotSupported;
    }
}

}  // namespace fcb
