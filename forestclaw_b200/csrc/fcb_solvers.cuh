// Point-wise Riemann solvers and the wave limiter for the device step kernel.
//
// Each solver restates one reference Fortran routine for a single interface
// (V5: the clawpack 5 twin of the routine where its arithmetic differs)
// (the reference loops over a whole 1-D slice; the per-interface arithmetic is
// the same).  The Roe averages that the reference passes from rpn2 to rpt2
// through COMMON /comroe/ travel here in an explicit per-interface struct.
// Association of every expression follows the Fortran source so that, compiled
// without FMA contraction, the results equal the reference's bit for bit.
#pragma once
#include <cuda_runtime.h>

namespace fcb {

template <typename T>
__device__ __forceinline__ T dmax(T a, T b) { return a > b ? a : b; }
template <typename T>
__device__ __forceinline__ T dmin(T a, T b) { return a < b ? a : b; }
// Maximum for the CFL number that keeps a NaN: a NaN wave speed (a negative
// depth, say) must reach the host as a NaN CFL, which the library reports as
// FCB_ERR_NUMERIC.  For numbers it equals dmax.
template <typename T>
__device__ __forceinline__ T nanmax(T a, T b) { return (b > a || b != b) ? b : a; }
// max(m, |s|) for m >= 0 as the unsigned maximum of the bit patterns: for
// non-negative numbers the same value as dmax, and a NaN (its magnitude's bits
// are the largest) is kept, at the cost of one integer compare-select.
__device__ __forceinline__ double absmax(double m, double s) {
    const unsigned long long a = (unsigned long long)__double_as_longlong(m);
    const unsigned long long b = (unsigned long long)__double_as_longlong(fabs(s));
    return __longlong_as_double((long long)(a > b ? a : b));
}
__device__ __forceinline__ float absmax(float m, float s) {
    const unsigned a = __float_as_uint(m), b = __float_as_uint(fabsf(s));
    return __uint_as_float(a > b ? a : b);
}

// ---------------------------------------------------------------------------
// Scalar advection: applications/clawpack/advection/2d/all/clawpack46_rpn2adv.f,
// clawpack46_rpt2adv.f.  The normal speed is the edge velocity aux(i,j,ixy);
// the transverse splitting uses the two edge velocities of the cell pair.
// ---------------------------------------------------------------------------
// clawpack5_rpn2adv.f90 / clawpack5_rpt2adv.f90 have the same arithmetic.
template <int W_, typename R = double, bool V5_ = false>
struct AdvectionSolver {
    using Real = R;
    static constexpr bool V5 = V5_;
    static constexpr bool FWAVE = false;
    static constexpr int M = 1;
    static constexpr int W = W_;
    struct Roe {};
    // no per-cell quantities to share between the interfaces of a cell
    struct Cell {};
    static constexpr int NC = 0;
    R grav, gamma, gamma1, drytol;  // unused
    __device__ __forceinline__ void prep(const R*, Cell&) const {}
    __device__ __forceinline__ void rpn2c(int ixy, const R* qL, const R* qR, const Cell&, const Cell&, R speed,
                                          R (*wave)[M], R* s, R* amdq, R* apdq, Roe& rr) const {
        rpn2(ixy, qL, qR, speed, wave, s, amdq, apdq, rr);
    }
    __device__ __forceinline__ void rpn2(int /*ixy*/, const R* qL, const R* qR, R speed,
                                         R (*wave)[M], R* s, R* amdq, R* apdq,
                                         Roe&) const {
        const R delta = qR[0] - qL[0];
#pragma unroll
        for (int mw = 0; mw < W; ++mw) {
            wave[mw][0] = delta;
            s[mw] = speed;
        }
        // the reference starts both sums at 0; starting at the first term differs
        // only in the sign of a zero result
        R am = dmin(s[0], R(0.0)) * wave[0][0];
        R ap = dmax(s[0], R(0.0)) * wave[0][0];
#pragma unroll
        for (int mw = 1; mw < W; ++mw) {
            am = am + dmin(s[mw], R(0.0)) * wave[mw][0];
            ap = ap + dmax(s[mw], R(0.0)) * wave[mw][0];
        }
        amdq[0] = am;
        apdq[0] = ap;
    }
    // aux_dn = aux2(i1,kv), aux_up = aux3(i1,kv)
    __device__ __forceinline__ void rpt2(int /*ixy*/, const R* asdq, const Roe&, R aux_dn,
                                         R aux_up, R* bm, R* bp) const {
        bm[0] = dmin(aux_dn, R(0.0)) * asdq[0];
        bp[0] = dmax(aux_up, R(0.0)) * asdq[0];
    }
};

// Scalar advection on a mapped grid: applications/clawpack/advection/2d/all/
// clawpack46_rpn2adv_manifold.f, clawpack46_rpt2adv_manifold.f.  The arithmetic
// of rpn2adv / rpt2adv with the edge velocities in aux(2:3), after the
// capacity kappa = area / (dx dy) in aux(1) (mcapa = 1), which the step then
// applies (clawpack46_step2.f:122-126,191-195, clawpack46_flux2.f:134-220,
// clawpack46_step2_wrap.f:118-121).
// V5: clawpack5_rpn2adv_manifold.f90 / rpt2adv_manifold.f90, the same arithmetic.
template <int W_, bool V5_ = false>
struct AdvectionManifoldSolver : AdvectionSolver<W_, double, V5_> {};

// Stored-aux layout of a solver: the first aux component its Riemann solvers
// read, and whether aux(1) is the capacity.
template <class SOL>
struct AuxLayout {
    static constexpr int SHIFT = 0;
    static constexpr bool CAPA = false;
};
template <int W_, bool V5_>
struct AuxLayout<AdvectionManifoldSolver<W_, V5_>> {
    static constexpr int SHIFT = 1;
    static constexpr bool CAPA = true;
};

// ---------------------------------------------------------------------------
// Shallow water, Roe with entropy fix:
// applications/clawpack/shallow/2d/rp/clawpack46_rpn2.f:1-247, clawpack46_rpt2.f:1-74
// ---------------------------------------------------------------------------
// V5: clawpack5_rpn2.f90, clawpack5_rpt2.f90 (a1, a3 scaled by 0.5/a instead
// of divided by 2a; the Roe averages clawpack5_rpt2 recomputes equal rpn2's).
template <typename R, bool V5_ = false>
struct SweRoeT {
    using Real = R;
    static constexpr bool V5 = V5_;
    static constexpr bool FWAVE = false;
    static constexpr int M = 3;
    static constexpr int W = 3;
    struct Roe { R u, v, a; };
    // Quantities of one cell that every Riemann problem it takes part in (two
    // x- and two y-interfaces) evaluates with the same operations on the same
    // operands: sqrt(h), hu/sqrt(h), hv/sqrt(h), hu/h, hv/h, sqrt(g h).  The
    // step kernels compute them once per cell; the values are bit-identical.
    struct Cell { R sq, rq[2], vel[2], c; };
    static constexpr int NC = 6;
    R grav, gamma, gamma1, drytol;  // drytol: GeoClaw only
    __device__ __forceinline__ void prep(const R* q, Cell& k) const {
        k.sq = sqrt(q[0]);
        k.rq[0] = q[1] / k.sq;
        k.rq[1] = q[2] / k.sq;
        k.vel[0] = q[1] / q[0];
        k.vel[1] = q[2] / q[0];
        k.c = sqrt(grav * q[0]);
    }
    __device__ __forceinline__ void rpn2(int ixy, const R* qL, const R* qR, R speed,
                                         R (*wave)[M], R* s, R* amdq, R* apdq,
                                         Roe& rr) const {
        Cell cl, cr;
        prep(qL, cl);
        prep(qR, cr);
        rpn2c(ixy, qL, qR, cl, cr, speed, wave, s, amdq, apdq, rr);
    }
    __device__ __forceinline__ void rpn2c(int ixy, const R* qL, const R* qR, const Cell& cl, const Cell& cr,
                                          R /*speed*/, R (*wave)[M], R* s, R* amdq, R* apdq,
                                          Roe& rr) const {
        const int mu = (ixy == 1) ? 1 : 2;
        const int mv = (ixy == 1) ? 2 : 1;
        const R h = (qL[0] + qR[0]) / R(2.0);
        const R hsq2 = cl.sq + cr.sq;                       // sqrt(qL(1)) + sqrt(qR(1))
        const R u = (cl.rq[mu - 1] + cr.rq[mu - 1]) / hsq2;  // (qL(mu)/hsqrtl + qR(mu)/hsqrtr)/hsq2
        const R v = (cl.rq[mv - 1] + cr.rq[mv - 1]) / hsq2;
        const R a = sqrt(grav * h);
        rr.u = u; rr.v = v; rr.a = a;
        const R d1 = qR[0] - qL[0];
        const R d2 = qR[mu] - qL[mu];
        const R d3 = qR[mv] - qL[mv];
        const R a1 = V5 ? ((u + a) * d1 - d2) * (R(0.5) / a) : ((u + a) * d1 - d2) / (R(2.0) * a);
        const R a2 = -(v * d1) + d3;
        const R a3 = V5 ? (-((u - a) * d1) + d2) * (R(0.5) / a) : (-((u - a) * d1) + d2) / (R(2.0) * a);
        wave[0][0] = a1; wave[0][mu] = a1 * (u - a); wave[0][mv] = a1 * v; s[0] = u - a;
        wave[1][0] = R(0.0); wave[1][mu] = R(0.0); wave[1][mv] = a2; s[1] = u;
        wave[2][0] = a3; wave[2][mu] = a3 * (u + a); wave[2][mv] = a3 * v; s[2] = u + a;
        // entropy fix
        R am[3];
        {
            const R s0 = cl.vel[mu - 1] - cl.c;  // qL(mu)/him1 - sqrt(g*him1)
            R sfract;
            if (s0 > R(0.0) && s[0] > R(0.0)) {
                am[0] = am[1] = am[2] = R(0.0);
                goto done;
            }
            {
                const R h1 = qL[0] + wave[0][0];
                const R hu1 = qL[mu] + wave[0][mu];
                const R s1 = hu1 / h1 - sqrt(grav * h1);
                if (s0 < R(0.0) && s1 > R(0.0)) sfract = s0 * ((s1 - s[0]) / (s1 - s0));
                else if (s[0] < R(0.0)) sfract = s[0];
                else sfract = R(0.0);
#pragma unroll
                for (int m = 0; m < 3; ++m) am[m] = sfract * wave[0][m];
            }
            if (s[1] > R(0.0)) goto done;
#pragma unroll
            for (int m = 0; m < 3; ++m) am[m] = am[m] + s[1] * wave[1][m];
            {
                const R s03 = cr.vel[mu - 1] + cr.c;  // qR(mu)/hi + sqrt(g*hi)
                const R h3 = qR[0] - wave[2][0];
                const R hu3 = qR[mu] - wave[2][mu];
                const R s3 = hu3 / h3 + sqrt(grav * h3);
                if (s3 < R(0.0) && s03 > R(0.0)) sfract = s3 * ((s03 - s[2]) / (s03 - s3));
                else if (s[2] < R(0.0)) sfract = s[2];
                else goto done;
#pragma unroll
                for (int m = 0; m < 3; ++m) am[m] = am[m] + sfract * wave[2][m];
            }
        }
    done:
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            R df = s[0] * wave[0][m];
#pragma unroll
            for (int mw = 1; mw < W; ++mw) df = df + s[mw] * wave[mw][m];
            amdq[m] = am[m];
            apdq[m] = df - am[m];
        }
    }
    __device__ __forceinline__ void rpt2(int ixy, const R* asdq, const Roe& rr, R, R,
                                         R* bm, R* bp) const {
        const int mu = (ixy == 1) ? 1 : 2;
        const int mv = (ixy == 1) ? 2 : 1;
        const R u = rr.u, v = rr.v, a = rr.a;
        const R a1 = V5 ? (R(0.5) / a) * ((v + a) * asdq[0] - asdq[mv]) : ((v + a) * asdq[0] - asdq[mv]) / (2 * a);
        const R a2 = asdq[mu] - u * asdq[0];
        const R a3 = V5 ? (R(0.5) / a) * (-((v - a) * asdq[0]) + asdq[mv]) : (-((v - a) * asdq[0]) + asdq[mv]) / (2 * a);
        R waveb[3][3], sb[3];
        waveb[0][0] = a1; waveb[mu][0] = a1 * u; waveb[mv][0] = a1 * (v - a); sb[0] = v - a;
        waveb[0][1] = R(0.0); waveb[mu][1] = a2; waveb[mv][1] = R(0.0); sb[1] = v;
        waveb[0][2] = a3; waveb[mu][2] = a3 * u; waveb[mv][2] = a3 * (v + a); sb[2] = v + a;
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            R m1 = dmin(sb[0], R(0.0)) * waveb[m][0], p1 = dmax(sb[0], R(0.0)) * waveb[m][0];
#pragma unroll
            for (int mw = 1; mw < 3; ++mw) {
                m1 = m1 + dmin(sb[mw], R(0.0)) * waveb[m][mw];
                p1 = p1 + dmax(sb[mw], R(0.0)) * waveb[m][mw];
            }
            bm[m] = m1;
            bp[m] = p1;
        }
    }
};

// ---------------------------------------------------------------------------
// Euler (4 equations), Roe with entropy fix:
// applications/clawpack/euler/2d/rp/clawpack46_rpn2_euler4.f:1-289,
// clawpack46_rpt2_euler4.f:290-386
// ---------------------------------------------------------------------------
// clawpack5_rpn2_euler4.f90 / clawpack5_rpt2_euler4.f90 have the same arithmetic.
template <typename R, bool V5_ = false>
struct Euler4RoeT {
    using Real = R;
    static constexpr bool V5 = V5_;
    static constexpr bool FWAVE = false;
    static constexpr int M = 4;
    static constexpr int W = 4;
    struct Roe { R u, v, a, enth, u2v2, g1a2, euv; };
    // Quantities of one cell shared by the four Riemann problems it takes part
    // in: sqrt(rho), rho u/sqrt(rho), rho v/sqrt(rho), (E + p)/sqrt(rho), u, v
    // and the sound speed sqrt(gamma p/rho).  The entropy fix's pressure sums
    // the squared momenta in the normal direction's order, which equals p
    // (addition commutes exactly), so every value is bit-identical.
    struct Cell { R sq, rq[2], rh, vel[2], c; };
    static constexpr int NC = 7;
    R grav, gamma, gamma1, drytol;  // drytol: GeoClaw only
    __device__ __forceinline__ void prep(const R* q, Cell& k) const {
        k.sq = sqrt(q[0]);
        const R p = gamma1 * (q[3] - R(0.5) * (q[1] * q[1] + q[2] * q[2]) / q[0]);
        k.rq[0] = q[1] / k.sq;
        k.rq[1] = q[2] / k.sq;
        k.rh = (q[3] + p) / k.sq;
        k.vel[0] = q[1] / q[0];
        k.vel[1] = q[2] / q[0];
        k.c = sqrt(gamma * p / q[0]);
    }
    __device__ __forceinline__ void rpn2(int ixy, const R* qL, const R* qR, R speed,
                                         R (*wave)[M], R* s, R* amdq, R* apdq,
                                         Roe& rr) const {
        Cell cl, cr;
        prep(qL, cl);
        prep(qR, cr);
        rpn2c(ixy, qL, qR, cl, cr, speed, wave, s, amdq, apdq, rr);
    }
    __device__ __forceinline__ void rpn2c(int ixy, const R* qL, const R* qR, const Cell& cl, const Cell& cr, R,
                                          R (*wave)[M], R* s, R* amdq, R* apdq,
                                          Roe& rr) const {
        const int mu = (ixy == 1) ? 1 : 2;
        const int mv = (ixy == 1) ? 2 : 1;
        const R rhsq2 = cl.sq + cr.sq;
        const R u = (cl.rq[mu - 1] + cr.rq[mu - 1]) / rhsq2;  // (qL(mu)/rhsqrtl + qR(mu)/rhsqrtr)/rhsq2
        const R v = (cl.rq[mv - 1] + cr.rq[mv - 1]) / rhsq2;
        const R enth = (cl.rh + cr.rh) / rhsq2;               // ((qL(4)+pl)/rhsqrtl + (qR(4)+pr)/rhsqrtr)/rhsq2
        const R u2v2 = u * u + v * v;
        const R a2s = gamma1 * (enth - R(0.5) * u2v2);
        const R a = sqrt(a2s);
        const R g1a2 = gamma1 / a2s;
        const R euv = enth - u2v2;
        rr.u = u; rr.v = v; rr.a = a; rr.enth = enth; rr.u2v2 = u2v2; rr.g1a2 = g1a2; rr.euv = euv;
        const R d1 = qR[0] - qL[0];
        const R d2 = qR[mu] - qL[mu];
        const R d3 = qR[mv] - qL[mv];
        const R d4 = qR[3] - qL[3];
        const R a3 = g1a2 * (euv * d1 + u * d2 + v * d3 - d4);
        const R a2 = d3 - v * d1;
        const R a4 = (d2 + (a - u) * d1 - a * a3) / (R(2.0) * a);
        const R a1 = d1 - a3 - a4;
        wave[0][0] = a1; wave[0][mu] = a1 * (u - a); wave[0][mv] = a1 * v; wave[0][3] = a1 * (enth - u * a);
        s[0] = u - a;
        wave[1][0] = R(0.0); wave[1][mu] = R(0.0); wave[1][mv] = a2; wave[1][3] = a2 * v; s[1] = u;
        wave[2][0] = a3; wave[2][mu] = a3 * u; wave[2][mv] = a3 * v; wave[2][3] = a3 * R(0.5) * u2v2; s[2] = u;
        wave[3][0] = a4; wave[3][mu] = a4 * (u + a); wave[3][mv] = a4 * v; wave[3][3] = a4 * (enth + u * a);
        s[3] = u + a;
        R am[4];
        {
            const R s0 = cl.vel[mu - 1] - cl.c;  // qL(mu)/rhoim1 - sqrt(gamma*pim1/rhoim1)
            R sfract;
            if (s0 >= R(0.0) && s[0] > R(0.0)) {
                am[0] = am[1] = am[2] = am[3] = R(0.0);
                goto done;
            }
            {
                const R rho1 = qL[0] + wave[0][0];
                const R rhou1 = qL[mu] + wave[0][mu];
                const R rhov1 = qL[mv] + wave[0][mv];
                const R en1 = qL[3] + wave[0][3];
                const R p1 = gamma1 * (en1 - R(0.5) * (rhou1 * rhou1 + rhov1 * rhov1) / rho1);
                const R c1 = sqrt(gamma * p1 / rho1);
                const R s1 = rhou1 / rho1 - c1;
                if (s0 < R(0.0) && s1 > R(0.0)) sfract = s0 * (s1 - s[0]) / (s1 - s0);
                else if (s[0] < R(0.0)) sfract = s[0];
                else sfract = R(0.0);
#pragma unroll
                for (int m = 0; m < 4; ++m) am[m] = sfract * wave[0][m];
            }
            if (s[1] >= R(0.0)) goto done;
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                am[m] = am[m] + s[1] * wave[1][m];
                am[m] = am[m] + s[2] * wave[2][m];
            }
            {
                const R s3 = cr.vel[mu - 1] + cr.c;  // qR(mu)/rhoi + sqrt(gamma*pi/rhoi)
                const R rho2 = qR[0] - wave[3][0];
                const R rhou2 = qR[mu] - wave[3][mu];
                const R rhov2 = qR[mv] - wave[3][mv];
                const R en2 = qR[3] - wave[3][3];
                const R p2 = gamma1 * (en2 - R(0.5) * (rhou2 * rhou2 + rhov2 * rhov2) / rho2);
                const R c2 = sqrt(gamma * p2 / rho2);
                const R s2 = rhou2 / rho2 + c2;
                if (s2 < R(0.0) && s3 > R(0.0)) sfract = s2 * (s3 - s[3]) / (s3 - s2);
                else if (s[3] < R(0.0)) sfract = s[3];
                else goto done;
#pragma unroll
                for (int m = 0; m < 4; ++m) am[m] = am[m] + sfract * wave[3][m];
            }
        }
    done:
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            R df = s[0] * wave[0][m];
#pragma unroll
            for (int mw = 1; mw < W; ++mw) df = df + s[mw] * wave[mw][m];
            amdq[m] = am[m];
            apdq[m] = df - am[m];
        }
    }
    __device__ __forceinline__ void rpt2(int ixy, const R* asdq, const Roe& rr, R, R,
                                         R* bm, R* bp) const {
        const int mu = (ixy == 1) ? 1 : 2;
        const int mv = (ixy == 1) ? 2 : 1;
        const R u = rr.u, v = rr.v, a = rr.a, enth = rr.enth;
        const R a3 = rr.g1a2 * (rr.euv * asdq[0] + u * asdq[mu] + v * asdq[mv] - asdq[3]);
        const R a2 = asdq[mu] - u * asdq[0];
        const R a4 = (asdq[mv] + (a - v) * asdq[0] - a * a3) / (R(2.0) * a);
        const R a1 = asdq[0] - a3 - a4;
        R waveb[4][3], sb[3];
        waveb[0][0] = a1; waveb[mu][0] = a1 * u; waveb[mv][0] = a1 * (v - a); waveb[3][0] = a1 * (enth - v * a);
        sb[0] = v - a;
        waveb[0][1] = a3; waveb[mu][1] = a3 * u + a2; waveb[mv][1] = a3 * v;
        waveb[3][1] = a3 * R(0.5) * rr.u2v2 + a2 * u; sb[1] = v;
        waveb[0][2] = a4; waveb[mu][2] = a4 * u; waveb[mv][2] = a4 * (v + a); waveb[3][2] = a4 * (enth + v * a);
        sb[2] = v + a;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            R m1 = dmin(sb[0], R(0.0)) * waveb[m][0], p1 = dmax(sb[0], R(0.0)) * waveb[m][0];
#pragma unroll
            for (int mw = 1; mw < 3; ++mw) {
                m1 = m1 + dmin(sb[mw], R(0.0)) * waveb[m][mw];
                p1 = p1 + dmax(sb[mw], R(0.0)) * waveb[m][mw];
            }
            bm[m] = m1;
            bp[m] = p1;
        }
    }
};

using SweRoeSolver = SweRoeT<double>;
using Euler4RoeSolver = Euler4RoeT<double>;


// ---------------------------------------------------------------------------
// GeoClaw f-wave solver: applications/clawpack/shallow/2d/rp/rpn2_geoclaw.f90
// with geoclaw_riemann_utils.f (riemanntype, riemann_aug_JCP, maxiter = 1).
// The reference stops on a negative depth or a sonic state; here such an
// interface sets `bad`, which the kernel reports as a NaN CFL.  The
// reference's rpt2_geoclaw stops on entry, so no transverse solver exists.
//
// R = double is the reference's arithmetic.  R = float is the mixed form: the
// speed estimates, the 3x3 f-wave solve and the waves in FP32, while the
// hydrostatic part stays FP64 -- the states, dry-state and wall handling, the
// bathymetry jump and the jumps del = (delh - deldelh, delhu, delphi -
// deldelphi) the waves are solved for -- so that a lake at rest gives del = 0
// and no waves.  Every R expression keeps the FP64 form's association, so
// R = double compiles to the same arithmetic.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double fsignd(double a, double b) { return signbit(b) ? -fabs(a) : fabs(a); }

template <typename R>
__device__ __forceinline__ void geo_riemanntype(R hL, R hR, R uL, R uR, R& hm, R& s1m, R& s2m, R drytol, R g) {
    const R h_min = fmin(hR, hL), h_max = fmax(hR, hL);
    const R delu = uR - uL;
    if (h_min <= drytol) {
        hm = R(0.0);
        s1m = uR + uL - R(2.0) * sqrt(g * hR) + R(2.0) * sqrt(g * hL);
        s2m = s1m;
    } else {
        const R F_min = delu + R(2.0) * (sqrt(g * h_min) - sqrt(g * h_max));
        const R F_max = delu + (h_max - h_min) * (sqrt(R(.5) * g * (h_max + h_min) / (h_max * h_min)));
        if (F_min > R(0.0)) {
            const R t = dmax(R(0.0), -delu + R(2.0) * (sqrt(g * hL) + sqrt(g * hR)));
            hm = (R(1.0) / (R(16.0) * g)) * (t * t);
            s1m = uL + R(2.0) * sqrt(g * hL) - R(3.0) * sqrt(g * hm);
            s2m = uR - R(2.0) * sqrt(g * hR) + R(3.0) * sqrt(g * hm);
        } else if (F_max <= R(0.0)) {
            R h0 = h_max;
            {
                const R gL = sqrt(R(.5) * g * (R(1) / h0 + R(1) / hL));
                const R gR = sqrt(R(.5) * g * (R(1) / h0 + R(1) / hR));
                const R F0 = delu + (h0 - hL) * gL + (h0 - hR) * gR;
                const R dfdh = gL - g * (h0 - hL) / (R(4.0) * (h0 * h0) * gL) + gR -
                               g * (h0 - hR) / (R(4.0) * (h0 * h0) * gR);
                const R slope = R(2.0) * sqrt(h0) * dfdh;
                const R t = sqrt(h0) - F0 / slope;
                h0 = t * t;
            }
            hm = h0;
            const R u1m = uL - (hm - hL) * sqrt((R(.5) * g) * (R(1) / hm + R(1) / hL));
            const R u2m = uR + (hm - hR) * sqrt((R(.5) * g) * (R(1) / hm + R(1) / hR));
            s1m = u1m - sqrt(g * hm);
            s2m = u2m + sqrt(g * hm);
        } else {
            R h0 = h_min;
            {
                const R F0 = delu + R(2.0) * (sqrt(g * h0) - sqrt(g * h_max)) +
                             (h0 - h_min) * sqrt(R(.5) * g * (R(1) / h0 + R(1) / h_min));
                const R slope = (F_max - F0) / (h_max - h_min);
                h0 = h0 - F0 / slope;
            }
            hm = h0;
            if (hL > hR) {
                s1m = uL + R(2.0) * sqrt(g * hL) - R(3.0) * sqrt(g * hm);
                s2m = uL + R(2.0) * sqrt(g * hL) - sqrt(g * hm);
            } else {
                s2m = uR - R(2.0) * sqrt(g * hR) + R(3.0) * sqrt(g * hm);
                s1m = uR - R(2.0) * sqrt(g * hR) + sqrt(g * hm);
            }
        }
    }
}

// riemann_aug_JCP with maxiter = 1 and rarecorrectortest = .false.; returns false on a sonic state
template <typename R>
__device__ __forceinline__ bool geo_riemann_aug(double hL, double hR, double huL, double huR, double bL, double bR,
                                                double uL, double uR, double vL, double vR, double phiL, double phiR,
                                                R sE1, R sE2, double drytol, double g, R sw[3], R fw[3][3]) {
    const double rho = -9999999.0, pL = 0.0, pR = 0.0;
    const double delh = hR - hL, delhu = huR - huL, delphi = phiR - phiL, delb = bR - bL, delP = pR - pL;
    R hm, s1m, s2m;
    geo_riemanntype<R>(R(hL), R(hR), R(uL), R(uR), hm, s1m, s2m, R(drytol), R(g));
    R lambda[3];
    lambda[0] = dmin(sE1, s2m);
    lambda[2] = dmax(sE2, s1m);
    sE1 = lambda[0];
    sE2 = lambda[2];
    const R hstarHLL = dmax((R(huL) - R(huR) + sE2 * R(hR) - sE1 * R(hL)) / (sE2 - sE1), R(0.0));
    R r[3][3];
#pragma unroll
    for (int mw = 0; mw < 3; ++mw) {
        r[0][mw] = R(1.0);
        r[1][mw] = (mw == 1) ? R(0.0) : lambda[mw];
        r[2][mw] = (mw == 1) ? R(0.0) : lambda[mw] * lambda[mw];
    }
    lambda[1] = R(0.5) * (lambda[0] + lambda[2]);
    r[0][1] = R(0.0);
    r[1][1] = R(0.0);
    r[2][1] = R(1.0);
    const double criticaltol = dmax(drytol * g, 1e-6);
    const double criticaltol_2 = sqrt(criticaltol);
    const double hbar = dmax(0.5 * (hL + hR), 0.0);
    const double s1s2bar = 0.25 * ((uL + uR) * (uL + uR)) - g * hbar;
    const double s1s2tilde = dmax(0.0, uL * uR) - g * hbar;
    const double dE1 = sE1, dE2 = sE2, ds1m = s1m, ds2m = s2m;
    bool sonic = false;
    if (fabs(s1s2bar) <= criticaltol) sonic = true;
    else if (s1s2bar * s1s2tilde <= criticaltol * criticaltol) sonic = true;
    else if (s1s2bar * dE1 * dE2 <= criticaltol * criticaltol) sonic = true;
    else if (dmin(fabs(dE1), fabs(dE2)) < criticaltol_2) sonic = true;
    else if (dE1 < criticaltol_2 && ds1m > -criticaltol_2) sonic = true;
    else if (dE2 > -criticaltol_2 && ds2m < criticaltol_2) sonic = true;
    else if ((uL + sqrt(g * hL)) * (uR + sqrt(g * hR)) < 0.0) sonic = true;
    else if ((uL - sqrt(g * hL)) * (uR - sqrt(g * hR)) < 0.0) sonic = true;
    double deldelh = delb * g * hbar / s1s2bar;
    if (dE1 < -criticaltol && dE2 > criticaltol) {
        deldelh = dmin(deldelh, (double)(hstarHLL * (sE2 - sE1) / sE2));
        deldelh = dmax(deldelh, (double)(hstarHLL * (sE2 - sE1) / sE1));
    } else if (dE1 >= criticaltol) {
        deldelh = dmin(deldelh, (double)(hstarHLL * (sE2 - sE1) / sE1));
        deldelh = dmax(deldelh, -hL);
    } else if (dE2 <= -criticaltol) {
        deldelh = dmin(deldelh, hR);
        deldelh = dmax(deldelh, (double)(hstarHLL * (sE2 - sE1) / sE2));
    }
    deldelh = deldelh - delP / (rho * g);
    double deldelphi = -(delb * g * hbar * s1s2tilde / s1s2bar);
    deldelphi = dmin(deldelphi, g * dmax(-hL * delb, -hR * delb));
    deldelphi = dmax(deldelphi, g * dmin(-hL * delb, -hR * delb));
    deldelphi = deldelphi - hbar * delP / rho;
    const R del[3] = {R(delh - deldelh), R(delhu), R(delphi - deldelphi)};
    R det1 = r[0][0] * (r[1][1] * r[2][2] - r[1][2] * r[2][1]);
    R det2 = r[0][1] * (r[1][0] * r[2][2] - r[1][2] * r[2][0]);
    R det3 = r[0][2] * (r[1][0] * r[2][1] - r[1][1] * r[2][0]);
    const R determinant = det1 - det2 + det3;
    R beta[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        R A[3][3];
#pragma unroll
        for (int mw = 0; mw < 3; ++mw)
#pragma unroll
            for (int m = 0; m < 3; ++m) A[m][mw] = (mw == k) ? del[m] : r[m][mw];
        det1 = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]);
        det2 = A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]);
        det3 = A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
        beta[k] = (det1 - det2 + det3) / determinant;
    }
#pragma unroll
    for (int mw = 0; mw < 3; ++mw) {
        sw[mw] = lambda[mw];
        fw[0][mw] = beta[mw] * r[1][mw];
        fw[1][mw] = beta[mw] * r[2][mw];
        fw[2][mw] = beta[mw] * r[1][mw];
    }
    fw[2][0] = fw[2][0] * R(vL);
    fw[2][2] = fw[2][2] * R(vR);
    fw[2][1] = R(0.0);
    const double hustar_interface = huL + (double)fw[0][0];
    const R dvflux = R(hR * uR * vR - hL * uL * vL);
    if (hustar_interface <= 0.0) fw[2][0] = fw[2][0] + (dvflux - fw[2][0] - fw[2][2]);
    else fw[2][2] = fw[2][2] + (dvflux - fw[2][0] - fw[2][2]);
    return !sonic;
}

template <typename R, bool V5_ = false>
struct GeoclawFwaveT {
    using Real = R;
    static constexpr bool V5 = V5_;
    static constexpr bool FWAVE = true;
    static constexpr int M = 3;
    static constexpr int W = 3;
    struct Roe {};
    R grav, gamma, gamma1, drytol;
    // one interface of rpn2_geoclaw.f90; the states and bL, bR (aux(1) of the
    // two cells) in FP64
    __device__ __forceinline__ void rpn2b(int ixy, const double* qL, const double* qR, double bL, double bR,
                                          R (*wave)[M], R* s, R* amdq, R* apdq, bool& bad) const {
        const int mu = (ixy == 1) ? 1 : 2;
        const int mv = (ixy == 1) ? 2 : 1;
        // the FP64 hydrostatic part reads gravity and the dry tolerance in FP64
        const double g = gdbl, dtol = drytol_d;
#pragma unroll
        for (int mw = 0; mw < 3; ++mw) {
            s[mw] = R(0.0);
            wave[mw][0] = R(0.0); wave[mw][1] = R(0.0); wave[mw][2] = R(0.0);
        }
        if (qL[0] < 0.0 || qR[0] < 0.0) bad = true;
        if (!(qL[0] <= dtol && qR[0] <= dtol)) {
            double hL = qL[0], hR = qR[0], huL = qL[mu], huR = qR[mu], hvL = qL[mv], hvR = qR[mv];
            double uR, vR, phiR, uL, vL, phiL;
            if (hR > dtol) {
                uR = huR / hR; vR = hvR / hR;
                phiR = 0.5 * g * (hR * hR) + (huR * huR) / hR;
            } else {
                hR = 0.0; huR = 0.0; hvR = 0.0; uR = 0.0; vR = 0; phiR = 0.0;
            }
            if (hL > dtol) {
                uL = huL / hL; vL = hvL / hL;
                phiL = 0.5 * g * (hL * hL) + (huL * huL) / hL;
            } else {
                hL = 0.0; huL = 0.0; hvL = 0.0; uL = 0.0; vL = 0.0; phiL = 0.0;
            }
            R wall[3] = {R(1.0), R(1.0), R(1.0)};
            double hstar, s1m, s2m;
            if (hR <= dtol) {
                geo_riemanntype<double>(hL, hL, uL, -uL, hstar, s1m, s2m, dtol, g);
                const double hstartest = dmax(hL, hstar);
                if (hstartest + bL < bR) {
                    wall[1] = R(0.0); wall[2] = R(0.0);
                    hR = hL; huR = -huL; bR = bL; phiR = phiL; uR = -uL; vL = vR;
                } else if (hL + bL < bR) {
                    bR = hL + bL;
                }
            } else if (hL <= dtol) {
                geo_riemanntype<double>(hR, hR, -uR, uR, hstar, s1m, s2m, dtol, g);
                const double hstartest = dmax(hR, hstar);
                if (hstartest + bR < bL) {
                    wall[0] = R(0.0); wall[1] = R(0.0);
                    hL = hR; huL = -huR; bL = bR; phiL = phiR; uL = -uR; vR = vL;
                } else if (hR + bR < bL) {
                    bL = hR + bR;
                }
            }
            const R rg = R(g);
            const R sL = R(uL) - sqrt(rg * R(hL));
            const R sR = R(uR) + sqrt(rg * R(hR));
            const R uhat = (sqrt(rg * R(hL)) * R(uL) + sqrt(rg * R(hR)) * R(uR)) / (sqrt(rg * R(hR)) + sqrt(rg * R(hL)));
            const R chat = sqrt(rg * R(0.5) * (R(hR) + R(hL)));
            const R sE1 = dmin(sL, uhat - chat), sE2 = dmax(sR, uhat + chat);
            R sw[3], fw[3][3];
            if (!geo_riemann_aug<R>(hL, hR, huL, huR, bL, bR, uL, uR, vL, vR, phiL, phiR, sE1, sE2, dtol, g, sw, fw))
                bad = true;
#pragma unroll
            for (int mw = 0; mw < 3; ++mw) {
                s[mw] = sw[mw] * wall[mw];
                wave[mw][0] = fw[0][mw] * wall[mw];
                wave[mw][mu] = fw[1][mw] * wall[mw];
                wave[mw][mv] = fw[2][mw] * wall[mw];
            }
        }
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            R am = R(0.0), ap = R(0.0);
#pragma unroll
            for (int mw = 0; mw < 3; ++mw) {
                if (s[mw] < R(0.0)) am = am + wave[mw][m];
                else if (s[mw] > R(0.0)) ap = ap + wave[mw][m];
                else {
                    am = am + R(0.5) * wave[mw][m];
                    ap = ap + R(0.5) * wave[mw][m];
                }
            }
            amdq[m] = am;
            apdq[m] = ap;
        }
    }
    double gdbl, drytol_d;  // gravity and dry tolerance in FP64, set by the step kernel
    // never called: order (2, 0) is enforced for this solver
    __device__ __forceinline__ void rpt2(int, const R* asdq, const Roe&, R, R, R* bm, R* bp) const {
#pragma unroll
        for (int m = 0; m < M; ++m) bm[m] = bp[m] = R(0) * asdq[m];
    }
    __device__ __forceinline__ void rpn2(int, const R*, const R*, R, R (*)[M], R*, R*, R*, Roe&) const {}
};

// clawpack46_inlinelimiter.f:4-118: phi(r) for limiter code `mth`
// (clawpack5_inlinelimiter.f:4-109 knows codes 1-5; callers map the others to 1).
template <typename R>
__device__ __forceinline__ R limiter_phi(int mth, R r) {
    switch (mth) {
        case 2: return dmax(dmax(R(0.0), dmin(R(1.0), R(2.0) * r)), dmin(R(2.0), r));
        case 3: return (r + fabs(r)) / (R(1.0) + fabs(r));
        case 4: {
            const R c = (R(1.0) + r) / R(2.0);
            return dmax(R(0.0), dmin(dmin(c, R(2.0)), R(2.0) * r));
        }
        case 5: return r;
        case 6: {
            const R th = R((double)1.3f);  // REAL*4 literal in the reference
            return dmax(R(0.0), dmin(dmin(th * r, (1 + r) / R(2.0)), th));
        }
        default: return dmax(R(0.0), dmin(R(1.0), r));
    }
}

}  // namespace fcb
