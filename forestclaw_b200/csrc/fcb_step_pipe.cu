// Software-pipelined form of the batched Clawpack 4.6 patch update (step2 +
// flux2 + conservative update): one thread per patch column, several patches
// per CTA, the patch rows streamed top to bottom.  The arithmetic, operation
// order and loop bounds are those of fcb_step.cu (and of the reference:
// src/solvers/fc2d_clawpack4.6/fortran_source/clawpack46_step2.f,
// clawpack46_flux2.f, clawpack46_step2_wrap.f); only the schedule differs.
//
// Every exchange between neighbouring columns goes through a small ring of
// rows in shared memory (2 or 4 slots), and every consumer runs at least one
// row-iteration after its producer, so one CTA barrier per row separates all
// producer/consumer pairs.  In the steady state the row loop is unrolled by the
// ring period, which turns every ring slot into a compile-time offset.
// Iteration s runs, in this order (k = row index of the stage):
//   S4  x-row s-3: transverse parts from the right neighbour (ring GL) -> GX(c, s-3)
//   S5  cell row s-4: conservative update (rings FX, GY; own GX, FY)
//   S3  x-row s-2: limiter with the neighbours' waves (ring XW), second-order
//       and transverse corrections -> rings FX, GL
//   S2  x-row s-1: Riemann problem with the left neighbour's state (ring Q) -> ring XW
//   S1  row s: y-interface s (raw) and y-interface s-1 (final, own column);
//       y transverse parts -> ring GY; aux row s+1 -> ring AX
// with q(c, s+1) prefetched at the top of iteration s.  Stages that carry
// values to the next iteration run before their producers, so the carries
// need no register copies.
//
// Accumulation order (identical to fcb_step.cu):
//   fm(i,j) = (FXm + GYu[col i-1]) + GYd[col i],   gm(i,j) = (GXu[row j-1] + GXd[row j]) + FYm
//   q = q - dtdx*(fm(i+1,j) - fp(i,j)) - dtdy*(gm(i,j+1) - gp(i,j)).
// Compiled without FMA contraction.
#include <cuda_runtime.h>

#include "fcb_device.h"
#include "fcb_solvers.cuh"

namespace fcb {

namespace {

__device__ __forceinline__ void atomic_max_nonneg_p(unsigned long long* p, double v) {
    atomicMax(p, (unsigned long long)__double_as_longlong(v));
}

// LIM > 0: order (2, 2) and limiter LIM on every wave, fixed at compile time;
// LIM == 0: order and limiters read from the launch arguments.
template <int LIM>
struct Method {
    const StepArgs& a;
    __device__ __forceinline__ bool second_order() const { return LIM > 0 || a.order0 == 2; }
    __device__ __forceinline__ bool transverse() const { return LIM > 0 || a.order1 > 0; }
    __device__ __forceinline__ bool transverse2() const { return LIM > 0 || (a.order0 > 1 && a.order1 == 2); }
    __device__ __forceinline__ int lim(int mw) const { return LIM > 0 ? LIM : a.mthlim[mw]; }
};

template <int NX, int PPB, int M, int W, int NAUX, bool SWIRL>
struct PipeSmem {
    // one ring slot holds one row of every patch of the CTA
    static constexpr int QS = PPB * M * NX;
    static constexpr int XWS = PPB * W * M * NX;
    static constexpr int GLS = PPB * 2 * M * NX;
    static constexpr int FXS = PPB * 2 * M * NX;
    static constexpr int GYS = PPB * 2 * M * NX;
    static constexpr int AXS = PPB * NAUX * NX;
    static constexpr int NDS = PPB * (NX + 1);
    static constexpr int Q = 0;                                   // 2 slots: [PPB][M][NX]
    static constexpr int XW = Q + 2 * QS;                         // 2 slots: [PPB][W][M][NX]
    static constexpr int GL = XW + 2 * XWS;                       // 2 slots: [PPB][2][M][NX]
    static constexpr int FX = GL + 2 * GLS;                       // 4 slots: [PPB][2][M][NX]
    static constexpr int GY = FX + 4 * FXS;                       // 4 slots: [PPB][2][M][NX]
    static constexpr int AX = GY + 4 * GYS;                       // 4 slots: [PPB][NAUX][NX]
    static constexpr int TY = AX + 4 * AXS;                       // [PPB][NX+1]           (swirl)
    static constexpr int ND = TY + (SWIRL ? PPB * (NX + 1) : 0);  // 2 slots: [PPB][NX+1]  (swirl)
    static constexpr int TOTAL = ND + (SWIRL ? 2 * NDS : 0);
};

// Values a thread carries from one row-iteration to the next.
template <class SOL>
struct PipeState {
    static constexpr int M = SOL::M;
    static constexpr int W = SOL::W;
    double qcur[M], q_m1[M];                                   // q(c, s), q(c, s-1)
    double yw_f[W][M], ys_f[W], yam_f[M], yap_f[M], ydotl[W];  // raw y-interface s-1
    typename SOL::Roe yR_f;
    double gRm_prev[M], gRp_prev[M];                           // y transverse parts into row s-2
    double xwl[W][M], xsl[W], xam[M], xap[M];                  // S2 -> S3
    typename SOL::Roe xR;
    double gRmx[M], gRpx[M];                                   // S3 -> S4
    double GXu_prev[M], GXs_prev[M];                           // S4 -> S4, S4 -> S5
    double FYm1[M], FYm2[M], FYp1[M], FYp2[M], FYp3[M];        // y fluxes of the own column, delayed
    double pcur;                                               // swirl: psi at node (c, s+1)
    double cfl;
};

// Per-thread constants: column, flags and this thread's column in every ring.
struct PipeThread {
    double* q;        // q of the patch, offset to column c
    double* qlast;    // qlast of the patch, offset to column c
    const double* aux;
    double* Qb;
    double* XWb;
    double* GLb;
    double* FXb;
    double* GYb;
    double* AXb;
    double* NDb;
    const double* TYb;
    double dtdx, dtdy, dtdxave, dtdyave, vty, vtx, tx, txr;
    int c;
    bool active, save_last, ycol;
};

// ring slot of row s - d when s == J (mod D) is known at compile time
__host__ __device__ constexpr int cslot(int J, int d, int D) { return ((J - d) % D + D) % D; }

// One row-iteration.  J >= 0: s == J (mod 4) at compile time, so every ring
// slot is a constant; STEADY: s in [4, NY-2], where every stage is active for
// every row and the row-range tests vanish.
template <class SOL, int MX, int MBC, int AUXK, int NAUX, int PPB, int LIM, int J, bool STEADY>
__device__ __forceinline__ void pipe_iter(const StepArgs& a, const SOL& sol, const PipeThread& T,
                                          PipeState<SOL>& S, int s) {
    constexpr int M = SOL::M;
    constexpr int W = SOL::W;
    constexpr int NX = MX + 2 * MBC;
    constexpr int NY = NX;
    constexpr bool SWIRL = AUXK == AUX_SWIRL;
    using L = PipeSmem<NX, PPB, M, W, NAUX, SWIRL>;
    constexpr double pi = 3.141592653589793;  // 4*atan(1) in double precision
    const Method<LIM> meth{a};
    const int c = T.c;
    auto s2 = [&](int d) -> int { return J >= 0 ? cslot(J, d, 2) : ((s - d) & 1); };
    auto s4 = [&](int d) -> int { return J >= 0 ? cslot(J, d, 4) : ((s - d) & 3); };
    // aux component k of row s-d, column c+dc
    auto AUXV = [&](int k, int dc, int d) -> double {
        if constexpr (NAUX > 0) return T.AXb[s4(d) * L::AXS + k * NX + dc];
        else return 0.0;
    };

    // prefetch q(c, s+1)
    double qnext[M];
    {
        const bool on = T.active && (STEADY || s + 1 < NY);
#pragma unroll
        for (int m = 0; m < M; ++m) qnext[m] = on ? T.q[((int64_t)m * NY + s + 1) * NX] : 0.0;
    }

    // ---------------- S4: GX(c, k), k = s-3 ----------------
    double GXs_new[M];
    {
        const int k = s - 3;
        const bool xint = T.active && (STEADY || (k >= 1 && k <= NY - 2)) && c >= 1;
        const double* gl = T.GLb + s2(3) * L::GLS;
#pragma unroll
        for (int m = 0; m < M; ++m) {
            double gxd = 0.0, gxu = 0.0;
            if (xint) {
                if (c + 1 <= NX - 1) {
                    gxd = -gl[(0 * M + m) * NX + 1] - S.gRmx[m];
                    gxu = -gl[(1 * M + m) * NX + 1] - S.gRpx[m];
                } else {
                    gxd = -S.gRmx[m];
                    gxu = -S.gRpx[m];
                }
            }
            GXs_new[m] = S.GXu_prev[m] + gxd;  // GX(c, k) = GXu(row k-1) + GXd(row k)
            S.GXu_prev[m] = gxu;
        }
    }

    // ---------------- S5: update cell row r = s-4 ----------------
    {
        const int r = s - 4;
        if (T.active && (STEADY || (r >= 0 && r <= NY - 2)) && c <= NX - 2) {
            const double* fx = T.FXb + s4(4) * L::FXS;
            const double* gy = T.GYb + s4(4) * L::GYS;
#pragma unroll
            for (int m = 0; m < M; ++m) {
                double* qp = T.q + ((int64_t)m * NY + r) * NX;
                const double qold = *qp;
                const double fxm1 = fx[(0 * M + m) * NX + 1];
                const double fxp0 = fx[(1 * M + m) * NX];
                const double gyu_l = (c >= 1) ? gy[(1 * M + m) * NX - 1] : 0.0;
                const double gyd_r = gy[(0 * M + m) * NX + 1];
                const double gyd = gy[(0 * M + m) * NX];
                const double gyu = gy[(1 * M + m) * NX];
                const double fmv = (fxm1 + gyu) + gyd_r;   // fm(i+1, j)
                const double fpv = (fxp0 + gyu_l) + gyd;   // fp(i, j)
                const double gmv = GXs_new[m] + S.FYm2[m];   // gm(i, j+1)
                const double gpv = S.GXs_prev[m] + S.FYp3[m];  // gp(i, j)
                *qp = qold - T.dtdx * (fmv - fpv) - T.dtdy * (gmv - gpv);
            }
        }
#pragma unroll
        for (int m = 0; m < M; ++m) S.GXs_prev[m] = GXs_new[m];
    }

    // ---------------- S3: x-row k = s-2: limiter, corrections, transverse ----------------
    {
        const int k = s - 2;
        if (T.active && (STEADY || (k >= 0 && k <= NY - 2))) {
            double* fx = T.FXb + s4(2) * L::FXS;
            const bool xint = (STEADY || k >= 1) && c >= 1;
            if (xint) {
                const double* xw = T.XWb + s2(2) * L::XWS;
                double cq[M];
#pragma unroll
                for (int m = 0; m < M; ++m) cq[m] = 0.0;
                if (meth.second_order()) {
                    if (c >= MBC && c <= MBC + MX) {
#pragma unroll
                        for (int mw = 0; mw < W; ++mw) {
                            const int mth = meth.lim(mw);
                            if (mth == 0) continue;
                            double wn2 = S.xwl[mw][0] * S.xwl[mw][0];
                            double dl = xw[(mw * M + 0) * NX - 1] * S.xwl[mw][0];
                            double dr = S.xwl[mw][0] * xw[(mw * M + 0) * NX + 1];
#pragma unroll
                            for (int m = 1; m < M; ++m) {
                                const double wc = S.xwl[mw][m];
                                wn2 = wn2 + wc * wc;
                                dl = dl + xw[(mw * M + m) * NX - 1] * wc;
                                dr = dr + wc * xw[(mw * M + m) * NX + 1];
                            }
                            if (wn2 == 0.0) continue;
                            const double rr = (S.xsl[mw] > 0.0) ? dl / wn2 : dr / wn2;
                            const double phi = limiter_phi(mth, rr);
#pragma unroll
                            for (int m = 0; m < M; ++m) S.xwl[mw][m] = phi * S.xwl[mw][m];
                        }
                    }
#pragma unroll
                    for (int m = 0; m < M; ++m) {
                        double acc;
                        {
                            const double as = fabs(S.xsl[0]);
                            acc = as * (1.0 - as * T.dtdxave) * S.xwl[0][m];
                        }
#pragma unroll
                        for (int mw = 1; mw < W; ++mw) {
                            const double as = fabs(S.xsl[mw]);
                            acc = acc + as * (1.0 - as * T.dtdxave) * S.xwl[mw][m];
                        }
                        cq[m] = acc;
                    }
                }
                double am[M], ap[M];
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    double fmv = (c <= NX - 2) ? S.xam[m] : 0.0;
                    double fpv = (c <= NX - 2) ? -S.xap[m] : 0.0;
                    if (meth.second_order()) { fmv = fmv + 0.5 * cq[m]; fpv = fpv + 0.5 * cq[m]; }
                    fx[(0 * M + m) * NX] = fmv;
                    fx[(1 * M + m) * NX] = fpv;
                    am[m] = S.xam[m];
                    ap[m] = S.xap[m];
                    if (meth.transverse2() && c <= NX - 2) { am[m] = am[m] + cq[m]; ap[m] = ap[m] - cq[m]; }
                }
                double* gl = T.GLb + s2(2) * L::GLS;
                if (meth.transverse()) {
                    double bm[M], bp[M];
                    // imp = 1: aux2(i-1, kv=2), aux3(i-1, kv=2) = v at column c-1, rows k, k+1
                    sol.rpt2(1, am, S.xR, AUXV(1, -1, 2), AUXV(1, -1, 1), bm, bp);
#pragma unroll
                    for (int m = 0; m < M; ++m) {
                        gl[(0 * M + m) * NX] = 0.5 * T.dtdx * bm[m];
                        gl[(1 * M + m) * NX] = 0.5 * T.dtdx * bp[m];
                    }
                    sol.rpt2(1, ap, S.xR, AUXV(1, 0, 2), AUXV(1, 0, 1), bm, bp);
#pragma unroll
                    for (int m = 0; m < M; ++m) {
                        S.gRmx[m] = 0.5 * T.dtdx * bm[m];
                        S.gRpx[m] = 0.5 * T.dtdx * bp[m];
                    }
                } else {
#pragma unroll
                    for (int m = 0; m < M; ++m) {
                        gl[(0 * M + m) * NX] = 0.0;
                        gl[(1 * M + m) * NX] = 0.0;
                        S.gRmx[m] = S.gRpx[m] = 0.0;
                    }
                }
            } else {
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    fx[(0 * M + m) * NX] = 0.0;
                    fx[(1 * M + m) * NX] = 0.0;
                }
            }
        }
    }

    // ---------------- S2: x-row k = s-1: Riemann problem at x-interface c ----------------
    {
        const int k = s - 1;
        if (T.active && (STEADY || (k >= 1 && k <= NY - 2)) && c >= 1) {
            const double* qr = T.Qb + s2(1) * L::QS;
            double qL[M];
#pragma unroll
            for (int m = 0; m < M; ++m) qL[m] = qr[m * NX - 1];
            sol.rpn2(1, qL, S.q_m1, AUXV(0, 0, 1), S.xwl, S.xsl, S.xam, S.xap, S.xR);
            double* xw = T.XWb + s2(1) * L::XWS;
#pragma unroll
            for (int mw = 0; mw < W; ++mw) {
#pragma unroll
                for (int m = 0; m < M; ++m) xw[(mw * M + m) * NX] = S.xwl[mw][m];
                if (c >= MBC && c <= MBC + MX) S.cfl = dmax(dmax(S.cfl, T.dtdx * S.xsl[mw]), -T.dtdx * S.xsl[mw]);
            }
        }
    }

    // ---------------- S1: row s ----------------
    {
        double yw_n[W][M], ys_n[W], yam_n[M], yap_n[M], ydotr[W];
        typename SOL::Roe yR_n{};
#pragma unroll
        for (int mw = 0; mw < W; ++mw) {
            ys_n[mw] = ydotr[mw] = 0.0;
#pragma unroll
            for (int m = 0; m < M; ++m) yw_n[mw][m] = 0.0;
        }
#pragma unroll
        for (int m = 0; m < M; ++m) yam_n[m] = yap_n[m] = 0.0;
        if (T.active && (STEADY || s < NY)) {
            double* qr = T.Qb + s2(0) * L::QS;
#pragma unroll
            for (int m = 0; m < M; ++m) {
                if (T.save_last) T.qlast[((int64_t)m * NY + s) * NX] = S.qcur[m];
                qr[m * NX] = S.qcur[m];
            }
            // raw y-interface s (between rows s-1 and s)
            if (T.ycol && (STEADY || s >= 1)) {
                sol.rpn2(2, S.q_m1, S.qcur, AUXV(1, 0, 0), yw_n, ys_n, yam_n, yap_n, yR_n);
#pragma unroll
                for (int mw = 0; mw < W; ++mw) {
                    double d = S.yw_f[mw][0] * yw_n[mw][0];
#pragma unroll
                    for (int m = 1; m < M; ++m) d = d + S.yw_f[mw][m] * yw_n[mw][m];
                    ydotr[mw] = d;  // dot(w(s-1), w(s))
                }
            }
        }

        // finalize y-interface f = s-1 (own column)
        const int f = s - 1;
        double FYm_new[M], FYp_new[M], GYd[M], GYu[M];
#pragma unroll
        for (int m = 0; m < M; ++m) FYm_new[m] = FYp_new[m] = GYd[m] = GYu[m] = 0.0;
        if (T.ycol && (STEADY || (f >= 1 && f <= NY - 1))) {
            const bool inner = STEADY || (f >= MBC && f <= MBC + MX);
            const bool god = STEADY || f <= NY - 2;
            double w[W][M];
#pragma unroll
            for (int mw = 0; mw < W; ++mw)
#pragma unroll
                for (int m = 0; m < M; ++m) w[mw][m] = S.yw_f[mw][m];
            if (inner) {
#pragma unroll
                for (int mw = 0; mw < W; ++mw) S.cfl = dmax(dmax(S.cfl, T.dtdy * S.ys_f[mw]), -T.dtdy * S.ys_f[mw]);
            }
            double cq[M];
#pragma unroll
            for (int m = 0; m < M; ++m) cq[m] = 0.0;
            if (meth.second_order()) {
                if (inner) {
#pragma unroll
                    for (int mw = 0; mw < W; ++mw) {
                        const int mth = meth.lim(mw);
                        if (mth == 0) continue;
                        double wn2 = S.yw_f[mw][0] * S.yw_f[mw][0];
#pragma unroll
                        for (int m = 1; m < M; ++m) wn2 = wn2 + S.yw_f[mw][m] * S.yw_f[mw][m];
                        if (wn2 == 0.0) continue;
                        const double rr = (S.ys_f[mw] > 0.0) ? S.ydotl[mw] / wn2 : ydotr[mw] / wn2;
                        const double phi = limiter_phi(mth, rr);
#pragma unroll
                        for (int m = 0; m < M; ++m) w[mw][m] = phi * w[mw][m];
                    }
                }
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    double acc;
                    {
                        const double as = fabs(S.ys_f[0]);
                        acc = as * (1.0 - as * T.dtdyave) * w[0][m];
                    }
#pragma unroll
                    for (int mw = 1; mw < W; ++mw) {
                        const double as = fabs(S.ys_f[mw]);
                        acc = acc + as * (1.0 - as * T.dtdyave) * w[mw][m];
                    }
                    cq[m] = acc;
                }
            }
            double am[M], ap[M];
#pragma unroll
            for (int m = 0; m < M; ++m) {
                double fmv = god ? S.yam_f[m] : 0.0;
                double fpv = god ? -S.yap_f[m] : 0.0;
                if (meth.second_order()) { fmv = fmv + 0.5 * cq[m]; fpv = fpv + 0.5 * cq[m]; }
                FYm_new[m] = fmv;
                FYp_new[m] = fpv;
                am[m] = S.yam_f[m];
                ap[m] = S.yap_f[m];
                if (meth.transverse2() && god) { am[m] = am[m] + cq[m]; ap[m] = ap[m] - cq[m]; }
            }
            double gLm[M], gLp[M], gRm[M], gRp[M];
            if (meth.transverse()) {
                double bm[M], bp[M];
                // imp = 1: aux2(j-1, kv=1), aux3(j-1, kv=1) = u at columns c, c+1, row f-1
                sol.rpt2(2, am, S.yR_f, AUXV(0, 0, 2), AUXV(0, 1, 2), bm, bp);
#pragma unroll
                for (int m = 0; m < M; ++m) { gLm[m] = 0.5 * T.dtdy * bm[m]; gLp[m] = 0.5 * T.dtdy * bp[m]; }
                sol.rpt2(2, ap, S.yR_f, AUXV(0, 0, 1), AUXV(0, 1, 1), bm, bp);
#pragma unroll
                for (int m = 0; m < M; ++m) { gRm[m] = 0.5 * T.dtdy * bm[m]; gRp[m] = 0.5 * T.dtdy * bp[m]; }
            } else {
#pragma unroll
                for (int m = 0; m < M; ++m) gLm[m] = gLp[m] = gRm[m] = gRp[m] = 0.0;
            }
            // cell row f-1 is complete: gadd(f-1,.,1) = (0 - gL(f)) - gR(f-1)
            if (STEADY || f - 1 >= 1) {
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    GYd[m] = -gLm[m] - S.gRm_prev[m];
                    GYu[m] = -gLp[m] - S.gRp_prev[m];
                }
            }
#pragma unroll
            for (int m = 0; m < M; ++m) { S.gRm_prev[m] = gRm[m]; S.gRp_prev[m] = gRp[m]; }
        }
        // GY of cell row s-2 (zero outside the y-columns and for row 0)
        if (T.active && (STEADY || (s >= 2 && s - 2 <= NY - 2))) {
            double* gy = T.GYb + s4(2) * L::GYS;
#pragma unroll
            for (int m = 0; m < M; ++m) {
                gy[(0 * M + m) * NX] = GYd[m];
                gy[(1 * M + m) * NX] = GYu[m];
            }
        }
        // delay lines: FYm(f) serves row f-1 two iterations on, FYp(f) row f three on
#pragma unroll
        for (int m = 0; m < M; ++m) {
            S.FYm2[m] = S.FYm1[m];
            S.FYm1[m] = FYm_new[m];
            S.FYp3[m] = S.FYp2[m];
            S.FYp2[m] = S.FYp1[m];
            S.FYp1[m] = FYp_new[m];
        }
        // shift the y window
#pragma unroll
        for (int mw = 0; mw < W; ++mw) {
            S.ydotl[mw] = ydotr[mw];
            S.ys_f[mw] = ys_n[mw];
#pragma unroll
            for (int m = 0; m < M; ++m) S.yw_f[mw][m] = yw_n[mw][m];
        }
#pragma unroll
        for (int m = 0; m < M; ++m) {
            S.yam_f[m] = yam_n[m];
            S.yap_f[m] = yap_n[m];
            S.q_m1[m] = S.qcur[m];
            S.qcur[m] = qnext[m];
        }
        S.yR_f = yR_n;

        // aux row s+1
        if (STEADY || s + 1 <= NY - 1) {
            if constexpr (SWIRL) {
                double* Nn = T.NDb + s2(-2) * L::NDS;        // node row s+2
                const double* Nc = T.NDb + s2(-1) * L::NDS;  // node row s+1
                const double ty = T.TYb[s + 2];
                const double pn = (T.tx * ty) / pi;
                if (T.active) {
                    double* ax = T.AXb + s4(-1) * L::AXS;
                    ax[0 * NX] = T.vty * (pn - S.pcur);
                    ax[1 * NX] = -T.vtx * (Nc[1] - S.pcur);
                    Nn[0] = pn;
                    if (c == NX - 1) Nn[1] = (T.txr * ty) / pi;
                }
                S.pcur = pn;
            } else if constexpr (AUXK == AUX_STORED) {
                if (T.active) {
                    double* ax = T.AXb + s4(-1) * L::AXS;
#pragma unroll
                    for (int kk = 0; kk < NAUX; ++kk) ax[kk * NX] = T.aux[(kk * NY + s + 1) * NX];
                }
            }
        }
    }
    __syncthreads();
}

}  // namespace

template <class SOL, int MX, int MBC, int AUXK, int NAUX, int TPB, int LIM>
__global__ void __launch_bounds__(TPB) step_kernel_pipe(const StepArgs a) {
    constexpr int M = SOL::M;
    constexpr int W = SOL::W;
    constexpr int NX = MX + 2 * MBC;
    constexpr int NY = NX;
    constexpr int PPB = TPB / NX;
    constexpr bool SWIRL = AUXK == AUX_SWIRL;
    using L = PipeSmem<NX, PPB, M, W, NAUX, SWIRL>;
    extern __shared__ double smem[];

    const int t = threadIdx.x;
    const int pl = t / NX;
    const int c = t - pl * NX;
    const int pg = blockIdx.x * PPB + pl;
    const bool active = (pl < PPB) && (pg < a.npatches);
    const int pls = active ? pl : 0;  // idle threads of a partial CTA read (never write) patch 0's rows
    const int slot = active ? a.slots[pg] : 0;
    const PatchMeta meta = active ? a.meta[slot] : PatchMeta{0, 0, 1, 1, 0, 0};
    const SOL sol{a.grav, a.gamma, a.gamma1};

    PipeThread T;
    T.c = c;
    T.active = active;
    T.save_last = active && (meta.flags & PATCH_SAVE_LAST);
    T.ycol = active && c >= 1 && c <= NX - 2;
    T.q = a.q + (int64_t)slot * a.q_stride + c;
    T.qlast = a.qlast + (int64_t)slot * a.q_stride + c;
    T.aux = (AUXK == AUX_STORED && active) ? a.aux + (int64_t)slot * a.aux_stride + c : nullptr;
    T.Qb = smem + L::Q + pls * M * NX + c;
    T.XWb = smem + L::XW + pls * W * M * NX + c;
    T.GLb = smem + L::GL + pls * 2 * M * NX + c;
    T.FXb = smem + L::FX + pls * 2 * M * NX + c;
    T.GYb = smem + L::GY + pls * 2 * M * NX + c;
    T.AXb = smem + L::AX + pls * NAUX * NX + c;
    T.NDb = smem + L::ND + pls * (NX + 1) + c;
    T.TYb = smem + L::TY + pls * (NX + 1);
    T.dtdx = a.dt / meta.dx;
    T.dtdy = a.dt / meta.dy;
    T.dtdxave = 0.5 * (T.dtdx + T.dtdx);  // 0.5*(dtdx1d(i-1)+dtdx1d(i)), no capacity
    T.dtdyave = 0.5 * (T.dtdy + T.dtdy);
    T.vty = a.vt / meta.dy;
    T.vtx = a.vt / meta.dx;
    T.tx = T.txr = 0.0;

    PipeState<SOL> S;
#pragma unroll
    for (int m = 0; m < M; ++m) {
        S.qcur[m] = active ? T.q[(int64_t)m * NY * NX] : 0.0;
        S.q_m1[m] = 0.0;
        S.yam_f[m] = S.yap_f[m] = 0.0;
        S.gRm_prev[m] = S.gRp_prev[m] = 0.0;
        S.xam[m] = S.xap[m] = 0.0;
        S.gRmx[m] = S.gRpx[m] = 0.0;
        S.GXu_prev[m] = S.GXs_prev[m] = 0.0;
        S.FYm1[m] = S.FYm2[m] = S.FYp1[m] = S.FYp2[m] = S.FYp3[m] = 0.0;
    }
#pragma unroll
    for (int mw = 0; mw < W; ++mw) {
        S.ys_f[mw] = S.ydotl[mw] = S.xsl[mw] = 0.0;
#pragma unroll
        for (int m = 0; m < M; ++m) S.yw_f[mw][m] = S.xwl[mw][m] = 0.0;
    }
    S.yR_f = typename SOL::Roe{};
    S.xR = typename SOL::Roe{};
    S.pcur = 0.0;
    S.cfl = 0.0;

    // ---- prologue: aux row 0 ----
    if constexpr (SWIRL) {
        // swirl/user_4.6/b4step2.f with swirl/psi.f:
        //   u(i,j) = vty*(psi(xll,yll+dy) - psi(xll,yll)),  v(i,j) = -vtx*(psi(xll+dx,yll) - psi(xll,yll)),
        //   psi(x,y) = (sin(pi x)**2 * sin(pi y)**2)/pi.
        // The unit-square mesh with mx a power of two is dyadic (xll + dx is the
        // next node's xll exactly; checked on the host), so psi is evaluated
        // once per node: P(c,n) at the lower-left corner of cell (c,n).
        constexpr double pi = 3.141592653589793;
        double* TY = smem + L::TY + pls * (NX + 1);
        {
            const double x = meta.xlower + (double)(c - MBC) * meta.dx;
            const double y = meta.ylower + (double)(c - MBC) * meta.dy;
            const double sx = sin(pi * x), sy = sin(pi * y);
            T.tx = sx * sx;
            if (active) TY[c] = sy * sy;
            if (c == NX - 1) {
                const double xr = meta.xlower + (double)(NX - MBC) * meta.dx;
                const double yr = meta.ylower + (double)(NX - MBC) * meta.dy;
                const double sxr = sin(pi * xr), syr = sin(pi * yr);
                T.txr = sxr * sxr;
                if (active) TY[NX] = syr * syr;
            }
        }
        __syncthreads();
        double* N0 = T.NDb;              // node row 0
        double* N1 = T.NDb + L::NDS;     // node row 1
        const double p0 = (T.tx * TY[0]) / pi, p1 = (T.tx * TY[1]) / pi;
        if (active) {
            N0[0] = p0;
            N1[0] = p1;
            if (c == NX - 1) {
                N0[1] = (T.txr * TY[0]) / pi;
                N1[1] = (T.txr * TY[1]) / pi;
            }
        }
        __syncthreads();
        if (active) {
            T.AXb[0 * NX] = T.vty * (p1 - p0);
            T.AXb[1 * NX] = -T.vtx * (N0[1] - p0);
        }
        S.pcur = p1;
    } else if constexpr (AUXK == AUX_STORED) {
        if (active) {
#pragma unroll
            for (int k = 0; k < NAUX; ++k) T.AXb[k * NX] = T.aux[(k * NY + 0) * NX];
        }
    }
    __syncthreads();

    // ---- rows: ramp-up, steady state (unrolled by the ring period 4), ramp-down ----
    int s = 0;
    for (; s < 4; ++s) pipe_iter<SOL, MX, MBC, AUXK, NAUX, PPB, LIM, -1, false>(a, sol, T, S, s);
    constexpr int NSTEADY = NY - 5;  // s = 4 .. NY-2
    for (int rnd = 0; rnd < NSTEADY / 4; ++rnd, s += 4) {
        pipe_iter<SOL, MX, MBC, AUXK, NAUX, PPB, LIM, 0, true>(a, sol, T, S, s);
        pipe_iter<SOL, MX, MBC, AUXK, NAUX, PPB, LIM, 1, true>(a, sol, T, S, s + 1);
        pipe_iter<SOL, MX, MBC, AUXK, NAUX, PPB, LIM, 2, true>(a, sol, T, S, s + 2);
        pipe_iter<SOL, MX, MBC, AUXK, NAUX, PPB, LIM, 3, true>(a, sol, T, S, s + 3);
    }
    for (; s <= NY + 2; ++s) pipe_iter<SOL, MX, MBC, AUXK, NAUX, PPB, LIM, -1, false>(a, sol, T, S, s);

    // ---- CFL: warp max, one atomic per warp ----
    double cfl = S.cfl;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) cfl = dmax(cfl, __shfl_xor_sync(0xffffffffu, cfl, off));
    if ((t & 31) == 0 && a.cfl_out) atomic_max_nonneg_p(a.cfl_out, cfl);
}

// ---------------------------------------------------------------------------
// Host-side launcher
// ---------------------------------------------------------------------------
namespace {

template <class SOL, int MX, int MBC, int AUXK, int NAUX, int TPB, int LIM>
cudaError_t launch_pipe_one(const StepArgs& a, cudaStream_t st) {
    constexpr int NX = MX + 2 * MBC;
    constexpr int PPB = TPB / NX;
    static_assert(PPB >= 1, "patch wider than the CTA");
    using L = PipeSmem<NX, PPB, SOL::M, SOL::W, NAUX, AUXK == AUX_SWIRL>;
    const size_t bytes = (size_t)L::TOTAL * sizeof(double);
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(step_kernel_pipe<SOL, MX, MBC, AUXK, NAUX, TPB, LIM>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    const int blocks = (a.npatches + PPB - 1) / PPB;
    if (blocks == 0) return cudaSuccess;
    step_kernel_pipe<SOL, MX, MBC, AUXK, NAUX, TPB, LIM><<<blocks, TPB, bytes, st>>>(a);
    return cudaGetLastError();
}

// Limiter specialisation: every wave limited with the same code and order (2, 2).
template <class SOL>
int fixed_limiter(const StepArgs& a) {
    if (a.order0 != 2 || a.order1 != 2) return 0;
    const int l = a.mthlim[0];
    for (int mw = 1; mw < SOL::W; ++mw)
        if (a.mthlim[mw] != l) return 0;
    return (l == 3 || l == 4) ? l : 0;
}

template <class SOL, int MX, int AUXK, int NAUX>
cudaError_t launch_pipe_lim(const StepArgs& a, cudaStream_t st) {
    switch (fixed_limiter<SOL>(a)) {
        case 3: return launch_pipe_one<SOL, MX, 2, AUXK, NAUX, 128, 3>(a, st);
        case 4: return launch_pipe_one<SOL, MX, 2, AUXK, NAUX, 128, 4>(a, st);
        default: return launch_pipe_one<SOL, MX, 2, AUXK, NAUX, 128, 0>(a, st);
    }
}

template <class SOL, int AUXK, int NAUX>
cudaError_t launch_pipe_mx(int mx, int mbc, const StepArgs& a, cudaStream_t st) {
    if (mbc != 2) return cudaErrorNotSupported;
    switch (mx) {
        case 8: return launch_pipe_lim<SOL, 8, AUXK, NAUX>(a, st);
        case 16: return launch_pipe_lim<SOL, 16, AUXK, NAUX>(a, st);
        case 32: return launch_pipe_lim<SOL, 32, AUXK, NAUX>(a, st);
        default: return cudaErrorNotSupported;
    }
}

}  // namespace

// cudaErrorNotSupported: no pipelined form for this (solver, mx, mbc, aux).
cudaError_t launch_step_pipe(int solver, int aux_kind, int mwaves, int mx, int my, int mbc, const StepArgs& a,
                             cudaStream_t st) {
    if (mx != my) return cudaErrorNotSupported;
    switch (solver) {
        case SOLVER_ADVECTION:
            if (mwaves != 1) return cudaErrorNotSupported;
            if (aux_kind == AUX_SWIRL) return launch_pipe_mx<AdvectionSolver<1>, AUX_SWIRL, 2>(mx, mbc, a, st);
            if (aux_kind == AUX_STORED && a.maux == 2)
                return launch_pipe_mx<AdvectionSolver<1>, AUX_STORED, 2>(mx, mbc, a, st);
            return cudaErrorNotSupported;
        case SOLVER_SWE_ROE:
            if (mwaves != 3 || aux_kind != AUX_NONE) return cudaErrorNotSupported;
            return launch_pipe_mx<SweRoeSolver, AUX_NONE, 0>(mx, mbc, a, st);
        case SOLVER_EULER4_ROE:
            if (mwaves != 4 || aux_kind != AUX_NONE) return cudaErrorNotSupported;
            return launch_pipe_mx<Euler4RoeSolver, AUX_NONE, 0>(mx, mbc, a, st);
        default: return cudaErrorNotSupported;
    }
}

}  // namespace fcb
