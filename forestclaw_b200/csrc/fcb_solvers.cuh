// Point-wise Riemann solvers and the wave limiter for the device step kernel.
//
// Each solver restates one reference Fortran routine for a single interface
// (the reference loops over a whole 1-D slice; the per-interface arithmetic is
// the same).  The Roe averages that the reference passes from rpn2 to rpt2
// through COMMON /comroe/ travel here in an explicit per-interface struct.
// Association of every expression follows the Fortran source so that, compiled
// without FMA contraction, the results equal the reference's bit for bit.
#pragma once
#include <cuda_runtime.h>

namespace fcb {

__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double dmin(double a, double b) { return a < b ? a : b; }

// ---------------------------------------------------------------------------
// Scalar advection: applications/clawpack/advection/2d/all/clawpack46_rpn2adv.f,
// clawpack46_rpt2adv.f.  The normal speed is the edge velocity aux(i,j,ixy);
// the transverse splitting uses the two edge velocities of the cell pair.
// ---------------------------------------------------------------------------
template <int W_>
struct AdvectionSolver {
    static constexpr int M = 1;
    static constexpr int W = W_;
    struct Roe {};
    double grav, gamma, gamma1;  // unused
    __device__ __forceinline__ void rpn2(int /*ixy*/, const double* qL, const double* qR, double speed,
                                         double (*wave)[M], double* s, double* amdq, double* apdq,
                                         Roe&) const {
        const double delta = qR[0] - qL[0];
#pragma unroll
        for (int mw = 0; mw < W; ++mw) {
            wave[mw][0] = delta;
            s[mw] = speed;
        }
        // the reference starts both sums at 0; starting at the first term differs
        // only in the sign of a zero result
        double am = dmin(s[0], 0.0) * wave[0][0];
        double ap = dmax(s[0], 0.0) * wave[0][0];
#pragma unroll
        for (int mw = 1; mw < W; ++mw) {
            am = am + dmin(s[mw], 0.0) * wave[mw][0];
            ap = ap + dmax(s[mw], 0.0) * wave[mw][0];
        }
        amdq[0] = am;
        apdq[0] = ap;
    }
    // aux_dn = aux2(i1,kv), aux_up = aux3(i1,kv)
    __device__ __forceinline__ void rpt2(int /*ixy*/, const double* asdq, const Roe&, double aux_dn,
                                         double aux_up, double* bm, double* bp) const {
        bm[0] = dmin(aux_dn, 0.0) * asdq[0];
        bp[0] = dmax(aux_up, 0.0) * asdq[0];
    }
};

// ---------------------------------------------------------------------------
// Shallow water, Roe with entropy fix:
// applications/clawpack/shallow/2d/rp/clawpack46_rpn2.f:1-247, clawpack46_rpt2.f:1-74
// ---------------------------------------------------------------------------
struct SweRoeSolver {
    static constexpr int M = 3;
    static constexpr int W = 3;
    struct Roe { double u, v, a; };
    double grav, gamma, gamma1;
    __device__ __forceinline__ void rpn2(int ixy, const double* qL, const double* qR, double /*speed*/,
                                         double (*wave)[M], double* s, double* amdq, double* apdq,
                                         Roe& R) const {
        const int mu = (ixy == 1) ? 1 : 2;
        const int mv = (ixy == 1) ? 2 : 1;
        const double h = (qL[0] + qR[0]) / 2.0;
        const double hsqrtl = sqrt(qL[0]);
        const double hsqrtr = sqrt(qR[0]);
        const double hsq2 = hsqrtl + hsqrtr;
        const double u = (qL[mu] / hsqrtl + qR[mu] / hsqrtr) / hsq2;
        const double v = (qL[mv] / hsqrtl + qR[mv] / hsqrtr) / hsq2;
        const double a = sqrt(grav * h);
        R.u = u; R.v = v; R.a = a;
        const double d1 = qR[0] - qL[0];
        const double d2 = qR[mu] - qL[mu];
        const double d3 = qR[mv] - qL[mv];
        const double a1 = ((u + a) * d1 - d2) / (2.0 * a);
        const double a2 = -(v * d1) + d3;
        const double a3 = (-((u - a) * d1) + d2) / (2.0 * a);
        wave[0][0] = a1; wave[0][mu] = a1 * (u - a); wave[0][mv] = a1 * v; s[0] = u - a;
        wave[1][0] = 0.0; wave[1][mu] = 0.0; wave[1][mv] = a2; s[1] = u;
        wave[2][0] = a3; wave[2][mu] = a3 * (u + a); wave[2][mv] = a3 * v; s[2] = u + a;
        // entropy fix
        double am[3];
        {
            const double him1 = qL[0];
            const double s0 = qL[mu] / him1 - sqrt(grav * him1);
            double sfract;
            if (s0 > 0.0 && s[0] > 0.0) {
                am[0] = am[1] = am[2] = 0.0;
                goto done;
            }
            {
                const double h1 = qL[0] + wave[0][0];
                const double hu1 = qL[mu] + wave[0][mu];
                const double s1 = hu1 / h1 - sqrt(grav * h1);
                if (s0 < 0.0 && s1 > 0.0) sfract = s0 * ((s1 - s[0]) / (s1 - s0));
                else if (s[0] < 0.0) sfract = s[0];
                else sfract = 0.0;
#pragma unroll
                for (int m = 0; m < 3; ++m) am[m] = sfract * wave[0][m];
            }
            if (s[1] > 0.0) goto done;
#pragma unroll
            for (int m = 0; m < 3; ++m) am[m] = am[m] + s[1] * wave[1][m];
            {
                const double hi = qR[0];
                const double s03 = qR[mu] / hi + sqrt(grav * hi);
                const double h3 = qR[0] - wave[2][0];
                const double hu3 = qR[mu] - wave[2][mu];
                const double s3 = hu3 / h3 + sqrt(grav * h3);
                if (s3 < 0.0 && s03 > 0.0) sfract = s3 * ((s03 - s[2]) / (s03 - s3));
                else if (s[2] < 0.0) sfract = s[2];
                else goto done;
#pragma unroll
                for (int m = 0; m < 3; ++m) am[m] = am[m] + sfract * wave[2][m];
            }
        }
    done:
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            double df = s[0] * wave[0][m];
#pragma unroll
            for (int mw = 1; mw < W; ++mw) df = df + s[mw] * wave[mw][m];
            amdq[m] = am[m];
            apdq[m] = df - am[m];
        }
    }
    __device__ __forceinline__ void rpt2(int ixy, const double* asdq, const Roe& R, double, double,
                                         double* bm, double* bp) const {
        const int mu = (ixy == 1) ? 1 : 2;
        const int mv = (ixy == 1) ? 2 : 1;
        const double u = R.u, v = R.v, a = R.a;
        const double a1 = ((v + a) * asdq[0] - asdq[mv]) / (2 * a);
        const double a2 = asdq[mu] - u * asdq[0];
        const double a3 = (-((v - a) * asdq[0]) + asdq[mv]) / (2 * a);
        double waveb[3][3], sb[3];
        waveb[0][0] = a1; waveb[mu][0] = a1 * u; waveb[mv][0] = a1 * (v - a); sb[0] = v - a;
        waveb[0][1] = 0.0; waveb[mu][1] = a2; waveb[mv][1] = 0.0; sb[1] = v;
        waveb[0][2] = a3; waveb[mu][2] = a3 * u; waveb[mv][2] = a3 * (v + a); sb[2] = v + a;
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            double m1 = dmin(sb[0], 0.0) * waveb[m][0], p1 = dmax(sb[0], 0.0) * waveb[m][0];
#pragma unroll
            for (int mw = 1; mw < 3; ++mw) {
                m1 = m1 + dmin(sb[mw], 0.0) * waveb[m][mw];
                p1 = p1 + dmax(sb[mw], 0.0) * waveb[m][mw];
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
struct Euler4RoeSolver {
    static constexpr int M = 4;
    static constexpr int W = 4;
    struct Roe { double u, v, a, enth, u2v2, g1a2, euv; };
    double grav, gamma, gamma1;
    __device__ __forceinline__ void rpn2(int ixy, const double* qL, const double* qR, double,
                                         double (*wave)[M], double* s, double* amdq, double* apdq,
                                         Roe& R) const {
        const int mu = (ixy == 1) ? 1 : 2;
        const int mv = (ixy == 1) ? 2 : 1;
        const double rhsqrtl = sqrt(qL[0]);
        const double rhsqrtr = sqrt(qR[0]);
        const double pl = gamma1 * (qL[3] - 0.5 * (qL[1] * qL[1] + qL[2] * qL[2]) / qL[0]);
        const double pr = gamma1 * (qR[3] - 0.5 * (qR[1] * qR[1] + qR[2] * qR[2]) / qR[0]);
        const double rhsq2 = rhsqrtl + rhsqrtr;
        const double u = (qL[mu] / rhsqrtl + qR[mu] / rhsqrtr) / rhsq2;
        const double v = (qL[mv] / rhsqrtl + qR[mv] / rhsqrtr) / rhsq2;
        const double enth = (((qL[3] + pl) / rhsqrtl + (qR[3] + pr) / rhsqrtr)) / rhsq2;
        const double u2v2 = u * u + v * v;
        const double a2s = gamma1 * (enth - 0.5 * u2v2);
        const double a = sqrt(a2s);
        const double g1a2 = gamma1 / a2s;
        const double euv = enth - u2v2;
        R.u = u; R.v = v; R.a = a; R.enth = enth; R.u2v2 = u2v2; R.g1a2 = g1a2; R.euv = euv;
        const double d1 = qR[0] - qL[0];
        const double d2 = qR[mu] - qL[mu];
        const double d3 = qR[mv] - qL[mv];
        const double d4 = qR[3] - qL[3];
        const double a3 = g1a2 * (euv * d1 + u * d2 + v * d3 - d4);
        const double a2 = d3 - v * d1;
        const double a4 = (d2 + (a - u) * d1 - a * a3) / (2.0 * a);
        const double a1 = d1 - a3 - a4;
        wave[0][0] = a1; wave[0][mu] = a1 * (u - a); wave[0][mv] = a1 * v; wave[0][3] = a1 * (enth - u * a);
        s[0] = u - a;
        wave[1][0] = 0.0; wave[1][mu] = 0.0; wave[1][mv] = a2; wave[1][3] = a2 * v; s[1] = u;
        wave[2][0] = a3; wave[2][mu] = a3 * u; wave[2][mv] = a3 * v; wave[2][3] = a3 * 0.5 * u2v2; s[2] = u;
        wave[3][0] = a4; wave[3][mu] = a4 * (u + a); wave[3][mv] = a4 * v; wave[3][3] = a4 * (enth + u * a);
        s[3] = u + a;
        double am[4];
        {
            const double rhoim1 = qL[0];
            const double pim1 = gamma1 * (qL[3] - 0.5 * (qL[mu] * qL[mu] + qL[mv] * qL[mv]) / rhoim1);
            const double cim1 = sqrt(gamma * pim1 / rhoim1);
            const double s0 = qL[mu] / rhoim1 - cim1;
            double sfract;
            if (s0 >= 0.0 && s[0] > 0.0) {
                am[0] = am[1] = am[2] = am[3] = 0.0;
                goto done;
            }
            {
                const double rho1 = qL[0] + wave[0][0];
                const double rhou1 = qL[mu] + wave[0][mu];
                const double rhov1 = qL[mv] + wave[0][mv];
                const double en1 = qL[3] + wave[0][3];
                const double p1 = gamma1 * (en1 - 0.5 * (rhou1 * rhou1 + rhov1 * rhov1) / rho1);
                const double c1 = sqrt(gamma * p1 / rho1);
                const double s1 = rhou1 / rho1 - c1;
                if (s0 < 0.0 && s1 > 0.0) sfract = s0 * (s1 - s[0]) / (s1 - s0);
                else if (s[0] < 0.0) sfract = s[0];
                else sfract = 0.0;
#pragma unroll
                for (int m = 0; m < 4; ++m) am[m] = sfract * wave[0][m];
            }
            if (s[1] >= 0.0) goto done;
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                am[m] = am[m] + s[1] * wave[1][m];
                am[m] = am[m] + s[2] * wave[2][m];
            }
            {
                const double rhoi = qR[0];
                const double pi = gamma1 * (qR[3] - 0.5 * (qR[mu] * qR[mu] + qR[mv] * qR[mv]) / rhoi);
                const double ci = sqrt(gamma * pi / rhoi);
                const double s3 = qR[mu] / rhoi + ci;
                const double rho2 = qR[0] - wave[3][0];
                const double rhou2 = qR[mu] - wave[3][mu];
                const double rhov2 = qR[mv] - wave[3][mv];
                const double en2 = qR[3] - wave[3][3];
                const double p2 = gamma1 * (en2 - 0.5 * (rhou2 * rhou2 + rhov2 * rhov2) / rho2);
                const double c2 = sqrt(gamma * p2 / rho2);
                const double s2 = rhou2 / rho2 + c2;
                if (s2 < 0.0 && s3 > 0.0) sfract = s2 * (s3 - s[3]) / (s3 - s2);
                else if (s[3] < 0.0) sfract = s[3];
                else goto done;
#pragma unroll
                for (int m = 0; m < 4; ++m) am[m] = am[m] + sfract * wave[3][m];
            }
        }
    done:
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            double df = s[0] * wave[0][m];
#pragma unroll
            for (int mw = 1; mw < W; ++mw) df = df + s[mw] * wave[mw][m];
            amdq[m] = am[m];
            apdq[m] = df - am[m];
        }
    }
    __device__ __forceinline__ void rpt2(int ixy, const double* asdq, const Roe& R, double, double,
                                         double* bm, double* bp) const {
        const int mu = (ixy == 1) ? 1 : 2;
        const int mv = (ixy == 1) ? 2 : 1;
        const double u = R.u, v = R.v, a = R.a, enth = R.enth;
        const double a3 = R.g1a2 * (R.euv * asdq[0] + u * asdq[mu] + v * asdq[mv] - asdq[3]);
        const double a2 = asdq[mu] - u * asdq[0];
        const double a4 = (asdq[mv] + (a - v) * asdq[0] - a * a3) / (2.0 * a);
        const double a1 = asdq[0] - a3 - a4;
        double waveb[4][3], sb[3];
        waveb[0][0] = a1; waveb[mu][0] = a1 * u; waveb[mv][0] = a1 * (v - a); waveb[3][0] = a1 * (enth - v * a);
        sb[0] = v - a;
        waveb[0][1] = a3; waveb[mu][1] = a3 * u + a2; waveb[mv][1] = a3 * v;
        waveb[3][1] = a3 * 0.5 * R.u2v2 + a2 * u; sb[1] = v;
        waveb[0][2] = a4; waveb[mu][2] = a4 * u; waveb[mv][2] = a4 * (v + a); waveb[3][2] = a4 * (enth + v * a);
        sb[2] = v + a;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            double m1 = dmin(sb[0], 0.0) * waveb[m][0], p1 = dmax(sb[0], 0.0) * waveb[m][0];
#pragma unroll
            for (int mw = 1; mw < 3; ++mw) {
                m1 = m1 + dmin(sb[mw], 0.0) * waveb[m][mw];
                p1 = p1 + dmax(sb[mw], 0.0) * waveb[m][mw];
            }
            bm[m] = m1;
            bp[m] = p1;
        }
    }
};

// clawpack46_inlinelimiter.f:4-118: phi(r) for limiter code `mth`.
__device__ __forceinline__ double limiter_phi(int mth, double r) {
    switch (mth) {
        case 2: return dmax(dmax(0.0, dmin(1.0, 2.0 * r)), dmin(2.0, r));
        case 3: return (r + fabs(r)) / (1.0 + fabs(r));
        case 4: {
            const double c = (1.0 + r) / 2.0;
            return dmax(0.0, dmin(dmin(c, 2.0), 2.0 * r));
        }
        case 5: return r;
        case 6: {
            const double th = (double)1.3f;  // REAL*4 literal in the reference
            return dmax(0.0, dmin(dmin(th * r, (1 + r) / 2.0), th));
        }
        default: return dmax(0.0, dmin(1.0, r));
    }
}

}  // namespace fcb
