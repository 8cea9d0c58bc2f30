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
// with q(c, s+2) prefetched at the top of iteration s.  Stages that carry
// values to the next iteration run before their producers, so the carries
// need no register copies.
//
// Accumulation order (identical to fcb_step.cu):
//   fm(i,j) = (FXm + GYu[col i-1]) + GYd[col i],   gm(i,j) = (GXu[row j-1] + GXd[row j]) + FYm
//   q = q - dtdx*(fm(i+1,j) - fp(i,j)) - dtdy*(gm(i,j+1) - gp(i,j)).
// The kernel is a template on the compute type R of the Riemann solves,
// limiters and transverse parts (SOL::Real): R = double is the FP64 form,
// compiled without FMA contraction (fcb_step_pipe.cu); R = float is the mixed
// form (fcb_step_mixed.cu), whose flux parts are widened to FP64 for the sums
// that form fm, fp, gm, gp and for the cell update.
#pragma once
#include <cuda_runtime.h>

#include <type_traits>

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

// psi at a node: (sin^2(pi x) sin^2(pi y))/pi.  The FP64 form divides as the
// reference does; the mixed form multiplies by 1/pi (one more rounding, far
// below its FP32 solves).
template <typename R>
__device__ __forceinline__ double psi_node(double tx, double ty) {
    constexpr double pi = 3.141592653589793;  // 4*atan(1) in double precision
    if constexpr (sizeof(R) == sizeof(double)) return (tx * ty) / pi;
    else return (tx * ty) * (1.0 / pi);
}

// Type of the state and aux rings: the compute type, except for the f-wave
// solver, whose hydrostatic part reads FP64 states and bathymetry; in its mixed
// form those two rings live in the FP64 region.
template <class SOL>
using ring_t = std::conditional_t<SOL::FWAVE, double, typename SOL::Real>;
template <class SOL>
constexpr bool ring_in_fp64 = SOL::FWAVE && !std::is_same_v<typename SOL::Real, double>;

template <int NX, int PPB, int M, int W, int NAUX, bool SWIRL, typename R, bool QDBL = false>
struct PipeSmem {
    // Rings are [slot][component][patch][column]: one thread's element of any
    // ring sits at (pl * NX + c) + a compile-time offset.
    static constexpr int PNX = PPB * NX;
    // rings in the compute type R (offsets in R elements); with QDBL the state
    // (Q) and aux (AX) rings are in the FP64 region instead
    static constexpr int XW = QDBL ? 0 : 2 * M * PNX; // 2 slots x W*M (after Q: 2 slots x M)
    static constexpr int GL = XW + 2 * W * M * PNX;   // 2 slots x 2M
    static constexpr int FX = GL + 2 * 2 * M * PNX;   // 4 slots x 2M
    static constexpr int AXR = FX + 4 * 2 * M * PNX;  // 4 slots x NAUX
    static constexpr int NR = QDBL ? AXR : AXR + 4 * NAUX * PNX;
    // FP64 region, from byte DBYTES on (offsets in doubles)
    static constexpr int DBYTES = ((NR * (int)sizeof(R) + 15) / 16) * 16;
    static constexpr int GY = 0;                      // 4 slots x 2M: y transverse sums
    static constexpr int NDS = PPB * (NX + 1);
    static constexpr int TY = GY + 4 * 2 * M * PNX;   // swirl: sin^2 of the node rows [patch][NX+1]
    static constexpr int ND = TY + (SWIRL ? NDS : 0); // swirl: psi node rows, 2 slots [patch][NX+1]
    static constexpr int NDEND = ND + (SWIRL ? 2 * NDS : 0);
    static constexpr int Q = QDBL ? NDEND : 0;
    static constexpr int AX = QDBL ? NDEND + 2 * M * PNX : AXR;
    static constexpr int BYTES = DBYTES + (QDBL ? NDEND + 2 * M * PNX + 4 * NAUX * PNX : NDEND) * 8;
};

// Values a thread carries from one row-iteration to the next.  R is the
// compute type of the Riemann solves, limiters and transverse parts; the
// sums that form fm, fp, gm, gp and the cell update stay in FP64.
template <class SOL>
struct PipeState {
    using R = typename SOL::Real;
    static constexpr int M = SOL::M;
    static constexpr int W = SOL::W;
    double qcur[M], q_m1[M];                             // q(c, s), q(c, s-1)
    double qpre[M];                                      // q(c, s+1), loaded one iteration ahead
    // scalar case: q(c, s-2..s-4) kept from their loads, so the update of row
    // s-4 reads its old value from registers instead of memory
    static constexpr bool DELAY = M == 1;
    double q_m2[M], q_m3[M], q_m4[M];
    R yw_f[W][M], ys_f[W], yam_f[M], yap_f[M], ydotl[W];  // raw y-interface s-1
    typename SOL::Roe yR_f;
    R gRm_prev[M], gRp_prev[M];                          // y transverse parts into row s-2
    R xwl[W][M], xsl[W], xam[M], xap[M];                 // S2 -> S3
    typename SOL::Roe xR;
    R gRmx[M], gRpx[M];                                  // S3 -> S4
    double GXu_prev[M], GXs_prev[M];                     // S4 -> S4, S4 -> S5
    R FYm1[M], FYm2[M], FYp1[M], FYp2[M], FYp3[M];       // y fluxes of the own column, delayed
    double pcur;                                         // swirl: psi at node (c, s+1)
    R smax_x, smax_y;  // largest |s| over the CFL interfaces of each direction
    bool bad;          // a Riemann problem the reference would stop on (reported as a NaN CFL)
};

// Per-thread constants: column, flags and this thread's element of the rings.
template <typename R>
struct PipeThread {
    double* q;        // q of the patch, offset to column c (fused: the patch in the arena written)
    double* qlast;    // qlast of the patch, offset to column c
    const double* qs; // fused: where rows MBC..MBC+MX-1 of column c are read (neighbour or own patch)
    unsigned negmid;  // fused: components negated on those rows (bit m: component m; solid walls)
    int slot;         // fused: the patch's slot
    const double* aux;
    R* rb;            // this thread's element of the R rings
    double* db;       // this thread's element of the FP64 rings
    double* nb;       // swirl: this thread's node in the psi node rows
    const double* ty; // swirl: sin^2 table of the patch's node rows
    double dtdx, dtdy, vty, vtx, tx;
    R rdtdx, rdtdy, rhdtdx, rhdtdy;
    double* treg;     // time-sync: the patch's conservation registers (nullptr: off)
    double tdy, tdx;  // time-sync: dt*dy and dt*dx
    int c;
    bool active, save_last, ycol, node;
};

// The pipelined form accumulates the time-sync registers for the
// shallow-water Roe solver in FP64, the one whose conservative flux
// (rpn2_cons_update) the flux store has.
template <class SOL, bool FUSED>
__host__ __device__ constexpr bool pipe_time_sync() {
    return !FUSED && std::is_same_v<SOL, SweRoeT<double, SOL::V5>>;
}

// ring slot of row s - d when s == J (mod D) is known at compile time
__host__ __device__ constexpr int cslot(int J, int d, int D) { return ((J - d) % D + D) % D; }

// Ghost-exchange fusion: where cell (c, s) of the patch in `slot` gets its
// value when the ghost update that precedes the step is folded into the step.
// On a mesh of one level that update (fclaw2d_ghost_update_async, one rank)
// first copies the same-size neighbours' interior cells into the face bands
// and corner blocks (fclaw2d_clawpatch46_fort_copy_face/_corner, the
// same-block transform a shift by mx), then applies the physical boundary
// conditions (clawpack46_bc2_default.f) left, right, bottom, top, each over the
// whole band including the corner cells.  The bottom/top conditions are
// applied last, so they are resolved first: a cell of a physical bottom band
// takes row 1 (extrapolation) or the mirrored row (wall, component 3 negated);
// then a physical left/right band takes column 1 / mx or the mirrored column
// (wall, component 2 negated); whatever still lies outside the interior is
// the copy from the face or corner neighbour that owns it.  *p receives the
// address of component 0 of the source cell in the arena qsrc; bit m of *neg
// says that component m is negated.
template <int MX, int MBC>
__device__ __forceinline__ void fused_src(const StepArgs& a, int slot, int c, int s, const double*& p,
                                          unsigned& neg) {
    constexpr int NX = MX + 2 * MBC;
    constexpr int HI = MBC + MX;  // first ghost row / column after the interior
    const FuseNbr* F = a.fuse + slot;
    int col = c, row = s, sl = slot;
    neg = 0u;
    if (row < MBC) {
        const int bc = __ldg(&F->bc[2]);
        if (bc == 3) { row = 2 * MBC - 1 - row; neg ^= 4u; }
        else if (bc != 0) row = MBC;
    } else if (row >= HI) {
        const int bc = __ldg(&F->bc[3]);
        if (bc == 3) { row = 2 * HI - 1 - row; neg ^= 4u; }
        else if (bc != 0) row = HI - 1;
    }
    if (col < MBC) {
        const int bc = __ldg(&F->bc[0]);
        if (bc == 3) { col = 2 * MBC - 1 - col; neg ^= 2u; }
        else if (bc != 0) col = MBC;
    } else if (col >= HI) {
        const int bc = __ldg(&F->bc[1]);
        if (bc == 3) { col = 2 * HI - 1 - col; neg ^= 2u; }
        else if (bc != 0) col = HI - 1;
    }
    const int h = col < MBC ? 0 : (col >= HI ? 2 : 1);
    const int v = row < MBC ? 0 : (row >= HI ? 2 : 1);
    if (h != 1 || v != 1) {
        int n;
        if (v == 1) n = __ldg(&F->face[h == 0 ? 0 : 1]);
        else if (h == 1) n = __ldg(&F->face[v == 0 ? 2 : 3]);
        else n = __ldg(&F->corner[(v == 0 ? 0 : 2) + (h == 0 ? 0 : 1)]);
        if (n >= 0) {  // always on a complete table; otherwise the patch's own (stale) ghost cell
            sl = n;
            col += h == 0 ? MX : (h == 2 ? -MX : 0);
            row += v == 0 ? MX : (v == 2 ? -MX : 0);
        }
    }
    p = a.qsrc + (int64_t)sl * a.q_stride + (int64_t)row * NX + col;
}

// Component m of row `row` of this thread's column as the step sees it.
template <int MX, int MBC, bool FUSED, typename R>
__device__ __forceinline__ double load_q(const StepArgs& a, const PipeThread<R>& T, int m, int row) {
    constexpr int NX = MX + 2 * MBC;
    constexpr int NY = NX;
    if constexpr (!FUSED) {
        return T.q[((int64_t)m * NY + row) * NX];
    } else {
        if (row >= MBC && row < MBC + MX) {
            const double v = T.qs[((int64_t)m * NY + row) * NX];
            return ((T.negmid >> m) & 1u) ? -v : v;
        }
        const double* p;
        unsigned neg;
        fused_src<MX, MBC>(a, T.slot, T.c, row, p, neg);
        const double v = p[(int64_t)m * NY * NX];
        return ((neg >> m) & 1u) ? -v : v;
    }
}

// One row-iteration.  J >= 0: s == J (mod 4) at compile time, so every ring
// slot is a constant; STEADY: s in [4, NY-2], where every stage is active for
// every row and the row-range tests vanish.
template <class SOL, int MX, int MBC, int AUXK, int NAUX, int PPB, int LIM, int J, bool STEADY, bool FUSED>
__device__ __forceinline__ void pipe_iter(const StepArgs& a, const SOL& sol,
                                          const PipeThread<typename SOL::Real>& T, PipeState<SOL>& S, int s) {
    using R = typename SOL::Real;
    using QT = ring_t<SOL>;
    constexpr int M = SOL::M;
    constexpr int W = SOL::W;
    constexpr int NX = MX + 2 * MBC;
    constexpr int NY = NX;
    constexpr bool SWIRL = AUXK == AUX_SWIRL;
    constexpr bool QDBL = ring_in_fp64<SOL>;
    using L = PipeSmem<NX, PPB, M, W, NAUX, SWIRL, R, QDBL>;
    QT* qb;  // this thread's element of the state and aux rings
    if constexpr (QDBL) qb = T.db;
    else qb = T.rb;
    const Method<LIM> meth{a};
    // clawpack 5 (clawpack5_flux2.f, clawpack5_step2.f90, clawpack5_step2_wrap.f):
    // fluxes at interfaces 1..mx+1 only, accumulated into cells 1..mx+1, and
    // only the interior cells updated
    constexpr bool V5 = SOL::V5;
    // f-waves (clawpack46_flux2fw.f): Godunov and correction terms on interfaces
    // 1..mx+1 only, corrections weighted by sign(s), no transverse part
    constexpr bool FWAVE = SOL::FWAVE;
    constexpr bool R15 = V5 || FWAVE;  // fluxes on interfaces MBC..MBC+MX only
    auto abs_sign = [](R sv) -> R {
        if constexpr (FWAVE) return copysign(R(1), sv);
        else return fabs(sv);
    };
    const int c = T.c;
    auto s2 = [&](int d) -> int { return J >= 0 ? cslot(J, d, 2) : ((s - d) & 1); };
    auto s4 = [&](int d) -> int { return J >= 0 ? cslot(J, d, 4) : ((s - d) & 3); };
    // aux component k of row s-d, column c+dc
    auto AUXV = [&](int k, int dc, int d) -> QT {
        if constexpr (NAUX > 0) return k < NAUX ? qb[L::AX + (s4(d) * NAUX + k) * L::PNX + dc] : QT(0);
        else return QT(0);
    };

    // prefetch q(c, s+2); the old value of q(c, s-4) for this iteration's update
    double qnext[M], qold[M];
    // a fused step writes the interior cells only: the ghost cells it would
    // update are overwritten by the ghost update that follows every step on a
    // mesh of one level, and that update is deferred until the ghost cells are read
    const bool upd = T.active && ((V5 || FUSED) ? (s - 4 >= MBC && s - 4 <= MBC + MX - 1 && c >= MBC && c <= MBC + MX - 1)
                                                : ((STEADY || (s - 4 >= 0 && s - 4 <= NY - 2)) && c <= NX - 2));
    {
        // prefetch two rows ahead; the last steady iteration (s = 4 + 4*((NY-5)/4) - 1)
        // still has row s+2 inside the patch for the patch sizes built here
        constexpr bool STEADY_IN = 4 + 4 * ((NY - 5) / 4) + 1 < NY;
        const bool on = T.active && ((STEADY && STEADY_IN) || s + 2 < NY);
#pragma unroll
        for (int m = 0; m < M; ++m) {
            qnext[m] = on ? load_q<MX, MBC, FUSED>(a, T, m, s + 2) : 0.0;
            if constexpr (PipeState<SOL>::DELAY) qold[m] = S.q_m4[m];
            else qold[m] = upd ? load_q<MX, MBC, FUSED>(a, T, m, s - 4) : 0.0;
        }
    }

    // ---------------- S4: GX(c, k), k = s-3 ----------------
    double GXs_new[M];
    {
        const int k = s - 3;
        const bool xint = T.active && (STEADY || (k >= 1 && k <= NY - 2)) && (V5 ? (c >= MBC && c <= MBC + MX) : c >= 1);
        const R* gl = T.rb + L::GL + s2(3) * (2 * M * L::PNX);
#pragma unroll
        for (int m = 0; m < M; ++m) {
            double gxd = 0.0, gxu = 0.0;
            if (xint) {
                if (c + 1 <= NX - 1) {
                    gxd = -(double)gl[(0 * M + m) * L::PNX + 1] - (double)S.gRmx[m];
                    gxu = -(double)gl[(1 * M + m) * L::PNX + 1] - (double)S.gRpx[m];
                } else {
                    gxd = -(double)S.gRmx[m];
                    gxu = -(double)S.gRpx[m];
                }
            }
            GXs_new[m] = S.GXu_prev[m] + gxd;  // GX(c, k) = GXu(row k-1) + GXd(row k)
            S.GXu_prev[m] = gxu;
        }
    }

    // ---------------- S5: update cell row r = s-4 ----------------
    {
        const int r = s - 4;
        // time-sync: the boundary fluctuations of the cells next to the patch
        // edges, inside and outside (clawpack46_time_sync_accumulate_waves,
        // clawpack5_time_sync_accumulate_waves), which the clawpack 5 update
        // computes but does not apply to the ghost cells
        constexpr bool TSYNC = pipe_time_sync<SOL, FUSED>();
        const int i = c - MBC + 1, j = r - MBC + 1;
        bool tsr = false;
        if constexpr (TSYNC) {
            const bool iin = i >= 1 && i <= MX, jin = j >= 1 && j <= MX;
            const bool iedge = i == 0 || i == 1 || i == MX || i == MX + 1;
            const bool jedge = j == 0 || j == 1 || j == MX || j == MX + 1;
            tsr = T.treg != nullptr && T.active && ((iedge && jin) || (jedge && iin));
        }
        if (upd || tsr) {
            const R* fx = T.rb + L::FX + s4(4) * (2 * M * L::PNX);
            const double* gy = T.db + L::GY + s4(4) * (2 * M * L::PNX);
#pragma unroll
            for (int m = 0; m < M; ++m) {
                double* qp = T.q + ((int64_t)m * NY + r) * NX;
                const double fxm1 = fx[(0 * M + m) * L::PNX + 1];  // FP32 flux parts widen exactly
                const double fxp0 = fx[(1 * M + m) * L::PNX];
                const double gyu_l = (c >= 1) ? gy[(1 * M + m) * L::PNX - 1] : 0.0;
                const double gyd_r = gy[(0 * M + m) * L::PNX + 1];
                const double gyd = gy[(0 * M + m) * L::PNX];
                const double gyu = gy[(1 * M + m) * L::PNX];
                const double fmv = (fxm1 + gyu) + gyd_r;   // fm(i+1, j)
                const double fpv = (fxp0 + gyu_l) + gyd;   // fp(i, j)
                const double gmv = GXs_new[m] + (double)S.FYm2[m];    // gm(i, j+1)
                const double gpv = S.GXs_prev[m] + (double)S.FYp3[m];  // gp(i, j)
                if (upd) *qp = qold[m] - T.dtdx * (fmv - fpv) - T.dtdy * (gmv - gpv);
                if constexpr (TSYNC) {
                    if (tsr) {
                        // each register element has exactly one writer
                        const RegLayout RL{MX, MX, M};
                        double* Rg = T.treg;
                        if (j >= 1 && j <= MX) {
                            const int k = (j - 1) + MX * m;
                            if (i == 1) Rg[RL.fp(0) + k] = Rg[RL.fp(0) + k] - T.tdy * fpv;
                            if (i == 0) Rg[RL.fm(0) + k] = Rg[RL.fm(0) + k] + T.tdy * fmv;       // fm(1, j)
                            if (i == MX) Rg[RL.fm(1) + k] = Rg[RL.fm(1) + k] + T.tdy * fmv;      // fm(mx+1, j)
                            if (i == MX + 1) Rg[RL.fp(1) + k] = Rg[RL.fp(1) + k] - T.tdy * fpv;  // fp(mx+1, j)
                        }
                        if (i >= 1 && i <= MX) {
                            const int k = (i - 1) + MX * m;
                            if (j == 1) Rg[RL.gp(0) + k] = Rg[RL.gp(0) + k] - T.tdx * gpv;
                            if (j == 0) Rg[RL.gm(0) + k] = Rg[RL.gm(0) + k] + T.tdx * gmv;       // gm(i, 1)
                            if (j == MX) Rg[RL.gm(1) + k] = Rg[RL.gm(1) + k] + T.tdx * gmv;      // gm(i, my+1)
                            if (j == MX + 1) Rg[RL.gp(1) + k] = Rg[RL.gp(1) + k] - T.tdx * gpv;  // gp(i, my+1)
                        }
                    }
                }
            }
        }
#pragma unroll
        for (int m = 0; m < M; ++m) S.GXs_prev[m] = GXs_new[m];
    }

    // ---------------- S3: x-row k = s-2: limiter, corrections, transverse ----------------
    {
        const int k = s - 2;
        if (T.active && (STEADY || (k >= 0 && k <= NY - 2))) {
            R* fx = T.rb + L::FX + s4(2) * (2 * M * L::PNX);
            const bool xint = (STEADY || k >= 1) && (R15 ? (c >= MBC && c <= MBC + MX) : c >= 1);
            if (xint) {
                const R* xw = T.rb + L::XW + s2(2) * (W * M * L::PNX);
                R cq[M];
#pragma unroll
                for (int m = 0; m < M; ++m) cq[m] = R(0);
                if (meth.second_order()) {
                    if (c >= MBC && c <= MBC + MX) {
#pragma unroll
                        for (int mw = 0; mw < W; ++mw) {
                            const int mth = meth.lim(mw);
                            if (mth == 0) continue;
                            R wn2 = S.xwl[mw][0] * S.xwl[mw][0];
                            R dl = xw[(mw * M + 0) * L::PNX - 1] * S.xwl[mw][0];
                            R dr = S.xwl[mw][0] * xw[(mw * M + 0) * L::PNX + 1];
#pragma unroll
                            for (int m = 1; m < M; ++m) {
                                const R wc = S.xwl[mw][m];
                                wn2 = wn2 + wc * wc;
                                dl = dl + xw[(mw * M + m) * L::PNX - 1] * wc;
                                dr = dr + wc * xw[(mw * M + m) * L::PNX + 1];
                            }
                            if (wn2 == R(0)) continue;
                            const R rr = (S.xsl[mw] > R(0)) ? dl / wn2 : dr / wn2;
                            const R phi = limiter_phi((SOL::V5 && mth > 5) ? 1 : mth, rr);
#pragma unroll
                            for (int m = 0; m < M; ++m) S.xwl[mw][m] = phi * S.xwl[mw][m];
                        }
                    }
#pragma unroll
                    for (int m = 0; m < M; ++m) {
                        R acc;
                        {
                            const R as = fabs(S.xsl[0]);
                            acc = abs_sign(S.xsl[0]) * (R(1) - as * T.rdtdx) * S.xwl[0][m];
                        }
#pragma unroll
                        for (int mw = 1; mw < W; ++mw) {
                            const R as = fabs(S.xsl[mw]);
                            acc = acc + abs_sign(S.xsl[mw]) * (R(1) - as * T.rdtdx) * S.xwl[mw][m];
                        }
                        cq[m] = acc;
                    }
                }
                R am[M], ap[M];
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    R fmv = (c <= NX - 2) ? S.xam[m] : R(0);
                    R fpv = (c <= NX - 2) ? -S.xap[m] : R(0);
                    if (meth.second_order()) { fmv = fmv + R(0.5) * cq[m]; fpv = fpv + R(0.5) * cq[m]; }
                    fx[(0 * M + m) * L::PNX] = fmv;
                    fx[(1 * M + m) * L::PNX] = fpv;
                    am[m] = S.xam[m];
                    ap[m] = S.xap[m];
                    if (meth.transverse2() && c <= NX - 2) { am[m] = am[m] + cq[m]; ap[m] = ap[m] - cq[m]; }
                }
                R* gl = T.rb + L::GL + s2(2) * (2 * M * L::PNX);
                if (meth.transverse()) {
                    R bm[M], bp[M];
                    // imp = 1: aux2(i-1, kv=2), aux3(i-1, kv=2) = v at column c-1, rows k, k+1
                    sol.rpt2(1, am, S.xR, AUXV(1, -1, 2), AUXV(1, -1, 1), bm, bp);
#pragma unroll
                    for (int m = 0; m < M; ++m) {
                        gl[(0 * M + m) * L::PNX] = T.rhdtdx * bm[m];
                        gl[(1 * M + m) * L::PNX] = T.rhdtdx * bp[m];
                    }
                    sol.rpt2(1, ap, S.xR, AUXV(1, 0, 2), AUXV(1, 0, 1), bm, bp);
#pragma unroll
                    for (int m = 0; m < M; ++m) {
                        S.gRmx[m] = T.rhdtdx * bm[m];
                        S.gRpx[m] = T.rhdtdx * bp[m];
                    }
                } else {
#pragma unroll
                    for (int m = 0; m < M; ++m) {
                        gl[(0 * M + m) * L::PNX] = R(0);
                        gl[(1 * M + m) * L::PNX] = R(0);
                        S.gRmx[m] = S.gRpx[m] = R(0);
                    }
                }
            } else {
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    fx[(0 * M + m) * L::PNX] = R(0);
                    fx[(1 * M + m) * L::PNX] = R(0);
                    if constexpr (R15) {  // read by the cell to the left (mx+1 at the right end)
                        R* gl = T.rb + L::GL + s2(2) * (2 * M * L::PNX);
                        gl[(0 * M + m) * L::PNX] = R(0);
                        gl[(1 * M + m) * L::PNX] = R(0);
                    }
                }
            }
        }
    }

    // ---------------- S2: x-row k = s-1: Riemann problem at x-interface c ----------------
    {
        const int k = s - 1;
        if (T.active && (STEADY || (k >= 1 && k <= NY - 2)) && c >= 1) {
            const QT* qr = qb + L::Q + s2(1) * (M * L::PNX);
            QT qL[M], qR[M];
#pragma unroll
            for (int m = 0; m < M; ++m) {
                qL[m] = qr[m * L::PNX - 1];
                qR[m] = QT(S.q_m1[m]);
            }
            if constexpr (FWAVE) {
                bool bad = false;
                sol.rpn2b(1, qL, qR, AUXV(0, -1, 1), AUXV(0, 0, 1), S.xwl, S.xsl, S.xam, S.xap, bad);
                S.bad = S.bad || bad;
            } else {
                sol.rpn2(1, qL, qR, AUXV(0, 0, 1), S.xwl, S.xsl, S.xam, S.xap, S.xR);
            }
            R* xw = T.rb + L::XW + s2(1) * (W * M * L::PNX);
#pragma unroll
            for (int mw = 0; mw < W; ++mw) {
#pragma unroll
                for (int m = 0; m < M; ++m) xw[(mw * M + m) * L::PNX] = S.xwl[mw][m];
                if (c >= MBC && c <= MBC + MX) S.smax_x = absmax(S.smax_x, S.xsl[mw]);
            }
        }
    }

    // ---------------- S1: row s ----------------
    {
        R yw_n[W][M], ys_n[W], yam_n[M], yap_n[M], ydotr[W];
        typename SOL::Roe yR_n{};
#pragma unroll
        for (int mw = 0; mw < W; ++mw) {
            ys_n[mw] = ydotr[mw] = R(0);
#pragma unroll
            for (int m = 0; m < M; ++m) yw_n[mw][m] = R(0);
        }
#pragma unroll
        for (int m = 0; m < M; ++m) yam_n[m] = yap_n[m] = R(0);
        if (T.active && (STEADY || s < NY)) {
            QT* qr = qb + L::Q + s2(0) * (M * L::PNX);
#pragma unroll
            for (int m = 0; m < M; ++m) {
                if (T.save_last) T.qlast[((int64_t)m * NY + s) * NX] = S.qcur[m];
                qr[m * L::PNX] = QT(S.qcur[m]);
            }
            // raw y-interface s (between rows s-1 and s)
            if (T.ycol && (STEADY || s >= 1)) {
                QT qD[M], qU[M];
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    qD[m] = QT(S.q_m1[m]);
                    qU[m] = QT(S.qcur[m]);
                }
                if constexpr (FWAVE) {
                    bool bad = false;
                    sol.rpn2b(2, qD, qU, AUXV(0, 0, 1), AUXV(0, 0, 0), yw_n, ys_n, yam_n, yap_n, bad);
                    S.bad = S.bad || bad;
                } else {
                    sol.rpn2(2, qD, qU, AUXV(1, 0, 0), yw_n, ys_n, yam_n, yap_n, yR_n);
                }
#pragma unroll
                for (int mw = 0; mw < W; ++mw) {
                    R d = S.yw_f[mw][0] * yw_n[mw][0];
#pragma unroll
                    for (int m = 1; m < M; ++m) d = d + S.yw_f[mw][m] * yw_n[mw][m];
                    ydotr[mw] = d;  // dot(w(s-1), w(s))
                }
            }
        }

        // finalize y-interface f = s-1 (own column)
        const int f = s - 1;
        R FYm_new[M], FYp_new[M];
        double GYd[M], GYu[M];
#pragma unroll
        for (int m = 0; m < M; ++m) {
            FYm_new[m] = FYp_new[m] = R(0);
            GYd[m] = GYu[m] = 0.0;
        }
        // clawpack 5: interfaces MBC..MBC+MX carry fluxes; f = MBC+MX+1 only
        // closes the transverse sum of cell row MBC+MX
        const bool yblk = T.ycol && (R15 ? (f >= MBC && f <= MBC + MX + 1) : (STEADY || (f >= 1 && f <= NY - 1)));
        if (yblk) {
            const bool fact = !R15 || f <= MBC + MX;
            const bool inner = R15 ? fact : (STEADY || (f >= MBC && f <= MBC + MX));
            const bool god = R15 ? fact : (STEADY || f <= NY - 2);
            R w[W][M];
#pragma unroll
            for (int mw = 0; mw < W; ++mw)
#pragma unroll
                for (int m = 0; m < M; ++m) w[mw][m] = S.yw_f[mw][m];
            if (inner) {
#pragma unroll
                for (int mw = 0; mw < W; ++mw) S.smax_y = absmax(S.smax_y, S.ys_f[mw]);
            }
            R cq[M];
#pragma unroll
            for (int m = 0; m < M; ++m) cq[m] = R(0);
            if (meth.second_order() && fact) {
                if (inner) {
#pragma unroll
                    for (int mw = 0; mw < W; ++mw) {
                        const int mth = meth.lim(mw);
                        if (mth == 0) continue;
                        R wn2 = S.yw_f[mw][0] * S.yw_f[mw][0];
#pragma unroll
                        for (int m = 1; m < M; ++m) wn2 = wn2 + S.yw_f[mw][m] * S.yw_f[mw][m];
                        if (wn2 == R(0)) continue;
                        const R rr = (S.ys_f[mw] > R(0)) ? S.ydotl[mw] / wn2 : ydotr[mw] / wn2;
                        const R phi = limiter_phi((SOL::V5 && mth > 5) ? 1 : mth, rr);
#pragma unroll
                        for (int m = 0; m < M; ++m) w[mw][m] = phi * w[mw][m];
                    }
                }
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    R acc;
                    {
                        const R as = fabs(S.ys_f[0]);
                        acc = abs_sign(S.ys_f[0]) * (R(1) - as * T.rdtdy) * w[0][m];
                    }
#pragma unroll
                    for (int mw = 1; mw < W; ++mw) {
                        const R as = fabs(S.ys_f[mw]);
                        acc = acc + abs_sign(S.ys_f[mw]) * (R(1) - as * T.rdtdy) * w[mw][m];
                    }
                    cq[m] = acc;
                }
            }
            R am[M], ap[M];
#pragma unroll
            for (int m = 0; m < M; ++m) {
                R fmv = god ? S.yam_f[m] : R(0);
                R fpv = god ? -S.yap_f[m] : R(0);
                if (meth.second_order()) { fmv = fmv + R(0.5) * cq[m]; fpv = fpv + R(0.5) * cq[m]; }
                FYm_new[m] = fmv;
                FYp_new[m] = fpv;
                am[m] = S.yam_f[m];
                ap[m] = S.yap_f[m];
                if (meth.transverse2() && god) { am[m] = am[m] + cq[m]; ap[m] = ap[m] - cq[m]; }
            }
            R gLm[M], gLp[M], gRm[M], gRp[M];
            if (meth.transverse() && fact) {
                R bm[M], bp[M];
                // imp = 1: aux2(j-1, kv=1), aux3(j-1, kv=1) = u at columns c, c+1, row f-1
                sol.rpt2(2, am, S.yR_f, AUXV(0, 0, 2), AUXV(0, 1, 2), bm, bp);
#pragma unroll
                for (int m = 0; m < M; ++m) { gLm[m] = T.rhdtdy * bm[m]; gLp[m] = T.rhdtdy * bp[m]; }
                sol.rpt2(2, ap, S.yR_f, AUXV(0, 0, 1), AUXV(0, 1, 1), bm, bp);
#pragma unroll
                for (int m = 0; m < M; ++m) { gRm[m] = T.rhdtdy * bm[m]; gRp[m] = T.rhdtdy * bp[m]; }
            } else {
#pragma unroll
                for (int m = 0; m < M; ++m) gLm[m] = gLp[m] = gRm[m] = gRp[m] = R(0);
            }
            // cell row f-1 is complete: gadd(f-1,.,1) = (0 - gL(f)) - gR(f-1)
            if (R15 ? (f - 1 >= MBC && f - 1 <= MBC + MX) : (STEADY || f - 1 >= 1)) {
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    GYd[m] = -(double)gLm[m] - (double)S.gRm_prev[m];
                    GYu[m] = -(double)gLp[m] - (double)S.gRp_prev[m];
                }
            }
#pragma unroll
            for (int m = 0; m < M; ++m) { S.gRm_prev[m] = gRm[m]; S.gRp_prev[m] = gRp[m]; }
        }
        // GY of cell row s-2 (zero outside the y-columns and for row 0)
        if (T.active && (STEADY || (s >= 2 && s - 2 <= NY - 2))) {
            double* gy = T.db + L::GY + s4(2) * (2 * M * L::PNX);
#pragma unroll
            for (int m = 0; m < M; ++m) {
                gy[(0 * M + m) * L::PNX] = GYd[m];
                gy[(1 * M + m) * L::PNX] = GYu[m];
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
            if constexpr (PipeState<SOL>::DELAY) {
                S.q_m4[m] = S.q_m3[m];
                S.q_m3[m] = S.q_m2[m];
                S.q_m2[m] = S.q_m1[m];
            }
            S.q_m1[m] = S.qcur[m];
            S.qcur[m] = S.qpre[m];
            S.qpre[m] = qnext[m];
        }
        S.yR_f = yR_n;

        // aux row s+1
        if (STEADY || s + 1 <= NY - 1) {
            if constexpr (SWIRL) {
                // node thread c (c in [0, NX]) computes psi at node (c, s+2)
                const double pn = psi_node<R>(T.tx, T.ty[s + 2]);
                if (T.node) T.nb[s2(-2) * L::NDS] = pn;
                if (T.active) {
                    QT* ax = qb + L::AX + s4(-1) * (NAUX * L::PNX);
                    ax[0 * L::PNX] = QT(T.vty * (pn - S.pcur));
                    ax[1 * L::PNX] = QT(-T.vtx * (T.nb[s2(-1) * L::NDS + 1] - S.pcur));
                }
                S.pcur = pn;
            } else if constexpr (AUXK == AUX_STORED) {
                if (T.active) {
                    QT* ax = qb + L::AX + s4(-1) * (NAUX * L::PNX);
#pragma unroll
                    for (int kk = 0; kk < NAUX; ++kk) ax[kk * L::PNX] = QT(T.aux[(kk * NY + s + 1) * NX]);
                }
            }
        }
    }
    __syncthreads();
}

template <int NX, bool SWIRL>
__host__ __device__ constexpr int pipe_threads_per_patch() { return SWIRL ? NX + 1 : NX; }

}  // namespace

// The mixed scalar form runs with the register budget cut for six resident
// 128-thread CTAs per SM (80 registers, a 32-byte spill): 3 % faster on the step
// than five at 93; seven (72 registers) and eight (64) spill more and are slower
// (B200, uniform swirl mx = 16).  Every other form keeps the compiler's choice:
// even an explicit minimum of one CTA changes its code (FP64 swirl step 18 %
// slower), so the body is shared by two kernels that differ only in the bound.
template <class SOL>
constexpr bool pipe_six_ctas() {
    return sizeof(typename SOL::Real) == 4 && SOL::M == 1;
}

template <class SOL, int MX, int MBC, int AUXK, int NAUX, int TPB, int LIM, bool FUSED>
__device__ __forceinline__ void step_pipe_body(const StepArgs& a) {
    constexpr int M = SOL::M;
    constexpr int W = SOL::W;
    constexpr int NX = MX + 2 * MBC;
    constexpr int NY = NX;
    constexpr bool SWIRL = AUXK == AUX_SWIRL;
    constexpr int TPP = pipe_threads_per_patch<NX, SWIRL>();
    constexpr int PPB = TPB / TPP;
    using R = typename SOL::Real;
    using QT = ring_t<SOL>;
    using L = PipeSmem<NX, PPB, M, W, NAUX, SWIRL, R, ring_in_fp64<SOL>>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* const rsm = reinterpret_cast<R*>(smem_raw);
    double* const dsm = reinterpret_cast<double*>(smem_raw + L::DBYTES);

    // Threads (pl, c): c in [0, NX) owns column c of patch pl; with the swirl
    // velocities one more thread per patch (c == NX) computes the last node
    // column of the stream function.
    const int t = threadIdx.x;
    const int pl = t / TPP;
    const int c = t - pl * TPP;
    const int pg = blockIdx.x * PPB + pl;
    const bool patch_ok = (pl < PPB) && (pg < a.npatches);
    const bool active = patch_ok && c < NX;
    const int pls = patch_ok ? pl : 0;  // threads without a patch read (never write) patch 0's rows
    const int cc = c < NX ? c : NX - 1;
    const PatchDesc* D = (a.desc && patch_ok) ? a.desc + pg : nullptr;  // mixed-solve launch
    const int slot = (patch_ok && !a.desc) ? a.slots[pg] : 0;
    const PatchMeta meta = D ? D->meta : (patch_ok ? a.meta[slot] : PatchMeta{0, 0, 1, 1, 0, 0});
    const int req = D ? D->req : -1;
    SOL sol{R(a.grav), R(a.gamma), R(a.gamma1), R(a.drytol)};
    if constexpr (SOL::FWAVE) {
        sol.gdbl = a.grav;
        sol.drytol_d = a.drytol;
    }

    PipeThread<R> T;
    T.c = cc;
    T.active = active;
    T.node = SWIRL && patch_ok;
    T.save_last = active && (meta.flags & PATCH_SAVE_LAST);
    T.ycol = active && c >= 1 && c <= NX - 2;
    T.q = (D ? D->q : a.q + (int64_t)slot * a.q_stride) + cc;
    T.qlast = (D ? D->qlast : a.qlast + (int64_t)slot * a.q_stride) + cc;
    T.slot = slot;
    T.qs = nullptr;
    T.negmid = 0u;
    if constexpr (FUSED) {
        // rows MBC..MBC+MX-1 of this column come from one place (own patch,
        // face neighbour, or the own patch's boundary column); rows outside are
        // resolved row by row in load_q
        T.save_last = false;  // a mesh of one level has no patch with finer neighbours
        if (active) {
            const double* p0;
            unsigned neg;
            fused_src<MX, MBC>(a, slot, cc, MBC, p0, neg);
            T.qs = p0 - (int64_t)MBC * NX;
            T.negmid = neg;
        }
    }
    T.aux = (AUXK == AUX_STORED && active) ? (D ? D->aux : a.aux + (int64_t)slot * a.aux_stride) + cc : nullptr;
    T.rb = rsm + pls * NX + cc;
    T.db = dsm + pls * NX + cc;
    T.nb = dsm + L::ND + pls * (NX + 1) + c;
    T.ty = dsm + L::TY + pls * (NX + 1);
    // dtdx1d is uniform without capacity, so 0.5*(dtdx1d(i-1)+dtdx1d(i)) == dtdx exactly
    const double dt = D ? D->dt : step_dt(a, meta.level), vt = D ? D->vt : step_vt(a, meta.level);
    T.dtdx = dt / meta.dx;
    T.dtdy = dt / meta.dy;
    T.rdtdx = R(T.dtdx);
    T.rdtdy = R(T.dtdy);
    T.rhdtdx = R(0.5 * T.dtdx);  // the reference's 0.5d0*dtdx*b, evaluated left to right
    T.rhdtdy = R(0.5 * T.dtdy);
    T.vty = vt / meta.dy;
    T.vtx = vt / meta.dx;
    T.tx = 0.0;
    T.treg = nullptr;
    T.tdy = T.tdx = 0.0;
    if constexpr (pipe_time_sync<SOL, FUSED>()) {
        if (a.treg && patch_ok && !D) {
            T.treg = a.treg + (int64_t)slot * a.treg_stride;
            T.tdy = dt * meta.dy;
            T.tdx = dt * meta.dx;
        }
    }

    PipeState<SOL> S;
#pragma unroll
    for (int m = 0; m < M; ++m) {
        S.qcur[m] = active ? load_q<MX, MBC, FUSED>(a, T, m, 0) : 0.0;
        S.qpre[m] = active ? load_q<MX, MBC, FUSED>(a, T, m, 1) : 0.0;
        S.q_m1[m] = 0.0;
        S.q_m2[m] = S.q_m3[m] = S.q_m4[m] = 0.0;
        S.yam_f[m] = S.yap_f[m] = R(0);
        S.gRm_prev[m] = S.gRp_prev[m] = R(0);
        S.xam[m] = S.xap[m] = R(0);
        S.gRmx[m] = S.gRpx[m] = R(0);
        S.GXu_prev[m] = S.GXs_prev[m] = 0.0;
        S.FYm1[m] = S.FYm2[m] = S.FYp1[m] = S.FYp2[m] = S.FYp3[m] = R(0);
    }
#pragma unroll
    for (int mw = 0; mw < W; ++mw) {
        S.ys_f[mw] = S.ydotl[mw] = S.xsl[mw] = R(0);
#pragma unroll
        for (int m = 0; m < M; ++m) S.yw_f[mw][m] = S.xwl[mw][m] = R(0);
    }
    S.yR_f = typename SOL::Roe{};
    S.xR = typename SOL::Roe{};
    S.pcur = 0.0;
    S.smax_x = S.smax_y = R(0);
    S.bad = false;

    // ---- prologue: aux row 0 ----
    if constexpr (SWIRL) {
        // swirl/user_4.6/b4step2.f with swirl/psi.f:
        //   u(i,j) = vty*(psi(xll,yll+dy) - psi(xll,yll)),  v(i,j) = -vtx*(psi(xll+dx,yll) - psi(xll,yll)),
        //   psi(x,y) = (sin(pi x)**2 * sin(pi y)**2)/pi.
        // The unit-square mesh with mx a power of two is dyadic (xll + dx is the
        // next node's xll exactly; checked on the host), so psi is evaluated
        // once per node: P(c,n) at the lower-left corner of cell (c,n).
        constexpr double pi = 3.141592653589793;
        {
            const double x = meta.xlower + (double)(c - MBC) * meta.dx;
            const double y = meta.ylower + (double)(c - MBC) * meta.dy;
            const double sx = sin(pi * x), sy = sin(pi * y);
            T.tx = sx * sx;
            if (T.node) dsm[L::TY + pls * (NX + 1) + c] = sy * sy;
        }
        __syncthreads();
        const double p0 = psi_node<R>(T.tx, T.ty[0]), p1 = psi_node<R>(T.tx, T.ty[1]);
        if (T.node) {
            T.nb[0] = p0;          // node row 0
            T.nb[L::NDS] = p1;     // node row 1
        }
        __syncthreads();
        if (active) {
            T.rb[L::AX + 0 * L::PNX] = QT(T.vty * (p1 - p0));
            T.rb[L::AX + 1 * L::PNX] = QT(-T.vtx * (T.nb[1] - p0));
        }
        S.pcur = p1;
    } else if constexpr (AUXK == AUX_STORED) {
        if (active) {
#pragma unroll
            for (int k = 0; k < NAUX; ++k) {
                if constexpr (ring_in_fp64<SOL>) T.db[L::AX + k * L::PNX] = T.aux[(k * NY + 0) * NX];
                else T.rb[L::AX + k * L::PNX] = QT(T.aux[(k * NY + 0) * NX]);
            }
        }
    }
    __syncthreads();

    // ---- rows: ramp-up, steady state (unrolled by the ring period 4), ramp-down ----
    int s = 0;
    for (; s < 4; ++s) pipe_iter<SOL, MX, MBC, AUXK, NAUX, PPB, LIM, -1, false, FUSED>(a, sol, T, S, s);
    constexpr int NSTEADY = NY - 5;  // s = 4 .. NY-2
    for (int rnd = 0; rnd < NSTEADY / 4; ++rnd, s += 4) {
        pipe_iter<SOL, MX, MBC, AUXK, NAUX, PPB, LIM, 0, true, FUSED>(a, sol, T, S, s);
        pipe_iter<SOL, MX, MBC, AUXK, NAUX, PPB, LIM, 1, true, FUSED>(a, sol, T, S, s + 1);
        pipe_iter<SOL, MX, MBC, AUXK, NAUX, PPB, LIM, 2, true, FUSED>(a, sol, T, S, s + 2);
        pipe_iter<SOL, MX, MBC, AUXK, NAUX, PPB, LIM, 3, true, FUSED>(a, sol, T, S, s + 3);
    }
    for (; s <= NY + 2; ++s) pipe_iter<SOL, MX, MBC, AUXK, NAUX, PPB, LIM, -1, false, FUSED>(a, sol, T, S, s);

    // ---- CFL: warp max, one atomic per warp ----
    // flux2: cfl = max(cfl, dtdx*s, -dtdx*s) over the interfaces.  Rounding is
    // monotone, so max_i fl(dtdx*|s_i|) == fl(dtdx * max_i |s_i|): one product
    // per direction gives the reference's value exactly.
    double cfl = (double)nanmax(T.rdtdx * S.smax_x, T.rdtdy * S.smax_y);
    if (S.bad) cfl = __longlong_as_double(0x7ff8000000000000LL);  // NaN: wins the max, reported by the host
    if (a.desc) {
        // patches of different solves share warps: reduce over the lanes of each
        // solve (max of the non-negative bit patterns, high word then low word)
        const unsigned grp = __match_any_sync(0xffffffffu, req);
        const unsigned long long b = (unsigned long long)__double_as_longlong(patch_ok ? cfl : 0.0);
        const unsigned hi = __reduce_max_sync(grp, (unsigned)(b >> 32));
        const unsigned lo = __reduce_max_sync(grp, ((unsigned)(b >> 32) == hi) ? (unsigned)b : 0u);
        if (req >= 0 && (t & 31) == __ffs(grp) - 1 && a.cfl_out)
            atomicMax(a.cfl_out + req, ((unsigned long long)hi << 32) | lo);
    } else {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) cfl = nanmax(cfl, __shfl_xor_sync(0xffffffffu, cfl, off));
        if ((t & 31) == 0 && a.cfl_out) atomic_max_nonneg_p(a.cfl_out, cfl);
    }
}

template <class SOL, int MX, int MBC, int AUXK, int NAUX, int TPB, int LIM, bool FUSED>
__global__ void __launch_bounds__(TPB) step_kernel_pipe(const StepArgs a) {
    step_pipe_body<SOL, MX, MBC, AUXK, NAUX, TPB, LIM, FUSED>(a);
}

template <class SOL, int MX, int MBC, int AUXK, int NAUX, int TPB, int LIM, bool FUSED>
__global__ void __launch_bounds__(TPB, 6) step_kernel_pipe_six(const StepArgs a) {
    step_pipe_body<SOL, MX, MBC, AUXK, NAUX, TPB, LIM, FUSED>(a);
}

// the one kernel of the two that a form uses (only that one is instantiated)
template <class SOL, int MX, int MBC, int AUXK, int NAUX, int TPB, int LIM, bool FUSED>
constexpr auto pipe_kernel() {
    if constexpr (pipe_six_ctas<SOL>()) return step_kernel_pipe_six<SOL, MX, MBC, AUXK, NAUX, TPB, LIM, FUSED>;
    else return step_kernel_pipe<SOL, MX, MBC, AUXK, NAUX, TPB, LIM, FUSED>;
}

// ---------------------------------------------------------------------------
// Host-side launcher
// ---------------------------------------------------------------------------
namespace {

template <class SOL, int MX, int MBC, int AUXK, int NAUX, int TPB, int LIM, bool FUSED>
cudaError_t launch_pipe_one(const StepArgs& a, cudaStream_t st) {
    constexpr int NX = MX + 2 * MBC;
    constexpr int PPB = TPB / pipe_threads_per_patch<NX, AUXK == AUX_SWIRL>();
    static_assert(PPB >= 1, "patch wider than the CTA");
    using L = PipeSmem<NX, PPB, SOL::M, SOL::W, NAUX, AUXK == AUX_SWIRL, typename SOL::Real, ring_in_fp64<SOL>>;
    const size_t bytes = (size_t)L::BYTES;
    constexpr auto kernel = pipe_kernel<SOL, MX, MBC, AUXK, NAUX, TPB, LIM, FUSED>();
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    const int blocks = (a.npatches + PPB - 1) / PPB;
    if (blocks == 0) return cudaSuccess;
    kernel<<<blocks, TPB, bytes, st>>>(a);
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

template <class SOL, int MX, int AUXK, int NAUX, bool FUSED>
cudaError_t launch_pipe_lim(const StepArgs& a, cudaStream_t st) {
    switch (fixed_limiter<SOL>(a)) {
        case 3: return launch_pipe_one<SOL, MX, 2, AUXK, NAUX, 128, 3, FUSED>(a, st);
        case 4: return launch_pipe_one<SOL, MX, 2, AUXK, NAUX, 128, 4, FUSED>(a, st);
        default: return launch_pipe_one<SOL, MX, 2, AUXK, NAUX, 128, 0, FUSED>(a, st);
    }
}

template <class SOL, int AUXK, int NAUX, bool FUSED>
cudaError_t launch_pipe_mx(int mx, int mbc, const StepArgs& a, cudaStream_t st) {
    if (mbc != 2) return cudaErrorNotSupported;
    switch (mx) {
        case 8: return launch_pipe_lim<SOL, 8, AUXK, NAUX, FUSED>(a, st);
        case 16: return launch_pipe_lim<SOL, 16, AUXK, NAUX, FUSED>(a, st);
        case 32: return launch_pipe_lim<SOL, 32, AUXK, NAUX, FUSED>(a, st);
        default: return cudaErrorNotSupported;
    }
}

}  // namespace

// cudaErrorNotSupported: no pipelined form for this (solver, mx, mbc, aux).
// R: compute type of the Riemann solves, limiters and transverse parts;
// V5: the clawpack 5 update (fc2d_clawpack5) instead of clawpack 4.6.
template <typename R, bool V5, bool FUSED>
cudaError_t launch_step_pipe_v(int solver, int aux_kind, int mwaves, int mx, int my, int mbc, const StepArgs& a,
                               cudaStream_t st) {
    if (mx != my) return cudaErrorNotSupported;
    switch (solver) {
        case SOLVER_ADVECTION:
            if (mwaves != 1) return cudaErrorNotSupported;
            if (aux_kind == AUX_SWIRL) return launch_pipe_mx<AdvectionSolver<1, R, V5>, AUX_SWIRL, 2, FUSED>(mx, mbc, a, st);
            if (aux_kind == AUX_STORED && a.maux >= 2)
                return launch_pipe_mx<AdvectionSolver<1, R, V5>, AUX_STORED, 2, FUSED>(mx, mbc, a, st);
            return cudaErrorNotSupported;
        case SOLVER_SWE_ROE:
            if (mwaves != 3 || aux_kind != AUX_NONE) return cudaErrorNotSupported;
            return launch_pipe_mx<SweRoeT<R, V5>, AUX_NONE, 0, FUSED>(mx, mbc, a, st);
        case SOLVER_EULER4_ROE:
            if (mwaves != 4 || aux_kind != AUX_NONE) return cudaErrorNotSupported;
            return launch_pipe_mx<Euler4RoeT<R, V5>, AUX_NONE, 0, FUSED>(mx, mbc, a, st);
        case SOLVER_GEOCLAW_FWAVE:
            if constexpr (!V5) {
                if (mwaves != 3 || aux_kind != AUX_STORED || a.maux != 1) return cudaErrorNotSupported;
                return launch_pipe_mx<GeoclawFwaveT<R>, AUX_STORED, 1, FUSED>(mx, mbc, a, st);
            }
            return cudaErrorNotSupported;
        default: return cudaErrorNotSupported;
    }
}

// FUSED: the ghost-exchange-fused form (a.fuse and a.qsrc set; mesh of one level)
template <typename R, bool FUSED>
cudaError_t launch_step_pipe_t(int solver, int aux_kind, int mwaves, int mx, int my, int mbc, int claw_version,
                               const StepArgs& a, cudaStream_t st) {
    if (FUSED != (a.fuse != nullptr) || (FUSED && (a.desc || !a.qsrc || a.qsrc == a.q))) return cudaErrorInvalidValue;
    if (claw_version == 5) return launch_step_pipe_v<R, true, FUSED>(solver, aux_kind, mwaves, mx, my, mbc, a, st);
    return launch_step_pipe_v<R, false, FUSED>(solver, aux_kind, mwaves, mx, my, mbc, a, st);
}

}  // namespace fcb
