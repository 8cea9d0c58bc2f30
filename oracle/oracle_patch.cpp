// ORACLE -- test infrastructure only (see oracle_patch.hpp).
//
// Every routine below restates one reference routine; the citation is given
// above each.  Expression association follows the Fortran source (left to
// right for * and /, as gfortran evaluates it) and the build uses
// -ffp-contract=off so that no fused multiply-add changes a rounding.
#include "oracle_patch.hpp"

#include <algorithm>
#include <stdexcept>

namespace orc {

namespace {

// One 1-D slice array with Fortran index range [1-mbc, maxm+mbc].
struct Slice {
    int L, mbc;
    Slice(int maxm, int mbc_) : L(maxm + 2 * mbc_), mbc(mbc_) {}
    inline int at(int i) const { return i + mbc - 1; }
};

// ---------------------------------------------------------------------------
// Riemann solvers.  Arrays are slice-major: a(i, m) -> a[m*L + at(i)],
// wave(i, m, mw) -> wave[(mw*meqn + m)*L + at(i)], s(i, mw) -> s[mw*L + at(i)].
// ---------------------------------------------------------------------------
struct RiemannState {
    // Fortran COMMON /comroe/ equivalents (Roe averages per interface).
    std::vector<double> u, v, a, h, u2v2, enth, g1a2, euv;
    void resize(int L) {
        u.assign(L, 0); v.assign(L, 0); a.assign(L, 0); h.assign(L, 0);
        u2v2.assign(L, 0); enth.assign(L, 0); g1a2.assign(L, 0); euv.assign(L, 0);
    }
};

// ---------------------------------------------------------------------------
// GeoClaw f-wave solver (applications/clawpack/shallow/2d/rp/rpn2_geoclaw.f90
// with geoclaw_riemann_utils.f: riemanntype, riemann_aug_JCP), called with
// maxiter = 1 as the reference does.  The reference stops (Fortran STOP) on a
// negative depth and on a sonic state; here those raise std::runtime_error.
// ---------------------------------------------------------------------------
inline double fsign(double a, double b) { return std::signbit(b) ? -std::fabs(a) : std::fabs(a); }

// geoclaw_riemann_utils.f: riemanntype
void riemanntype(double hL, double hR, double uL, double uR, double& hm, double& s1m, double& s2m,
                 bool& rare1, bool& rare2, int maxiter, double drytol, double g) {
    double um, u1m, u2m, h0, F0, slope, gL, gR, dfdh;
    const double h_min = std::min(hR, hL), h_max = std::max(hR, hL);
    const double delu = uR - uL;
    if (h_min <= drytol) {
        hm = 0.0;
        um = 0.0;
        s1m = uR + uL - 2.0 * std::sqrt(g * hR) + 2.0 * std::sqrt(g * hL);
        s2m = uR + uL - 2.0 * std::sqrt(g * hR) + 2.0 * std::sqrt(g * hL);
        if (hL <= 0.0) { rare2 = true; rare1 = false; }
        else { rare1 = true; rare2 = false; }
    } else {
        const double F_min = delu + 2.0 * (std::sqrt(g * h_min) - std::sqrt(g * h_max));
        const double F_max = delu + (h_max - h_min) * (std::sqrt(.5 * g * (h_max + h_min) / (h_max * h_min)));
        if (F_min > 0.0) {  // 2-rarefactions
            const double t = std::max(0.0, -delu + 2.0 * (std::sqrt(g * hL) + std::sqrt(g * hR)));
            hm = (1.0 / (16.0 * g)) * (t * t);
            um = fsign(1.0, hm) * (uL + 2.0 * (std::sqrt(g * hL) - std::sqrt(g * hm)));
            s1m = uL + 2.0 * std::sqrt(g * hL) - 3.0 * std::sqrt(g * hm);
            s2m = uR - 2.0 * std::sqrt(g * hR) + 3.0 * std::sqrt(g * hm);
            rare1 = true;
            rare2 = true;
        } else if (F_max <= 0.0) {  // 2 shocks
            h0 = h_max;
            for (int iter = 1; iter <= maxiter; ++iter) {
                gL = std::sqrt(.5 * g * (1 / h0 + 1 / hL));
                gR = std::sqrt(.5 * g * (1 / h0 + 1 / hR));
                F0 = delu + (h0 - hL) * gL + (h0 - hR) * gR;
                dfdh = gL - g * (h0 - hL) / (4.0 * (h0 * h0) * gL) + gR - g * (h0 - hR) / (4.0 * (h0 * h0) * gR);
                slope = 2.0 * std::sqrt(h0) * dfdh;
                const double t = std::sqrt(h0) - F0 / slope;
                h0 = t * t;
            }
            hm = h0;
            u1m = uL - (hm - hL) * std::sqrt((.5 * g) * (1 / hm + 1 / hL));
            u2m = uR + (hm - hR) * std::sqrt((.5 * g) * (1 / hm + 1 / hR));
            um = .5 * (u1m + u2m);
            s1m = u1m - std::sqrt(g * hm);
            s2m = u2m + std::sqrt(g * hm);
            rare1 = false;
            rare2 = false;
        } else {  // one shock one rarefaction
            h0 = h_min;
            for (int iter = 1; iter <= maxiter; ++iter) {
                F0 = delu + 2.0 * (std::sqrt(g * h0) - std::sqrt(g * h_max)) +
                     (h0 - h_min) * std::sqrt(.5 * g * (1 / h0 + 1 / h_min));
                slope = (F_max - F0) / (h_max - h_min);
                h0 = h0 - F0 / slope;
            }
            hm = h0;
            if (hL > hR) {
                um = uL + 2.0 * std::sqrt(g * hL) - 2.0 * std::sqrt(g * hm);
                s1m = uL + 2.0 * std::sqrt(g * hL) - 3.0 * std::sqrt(g * hm);
                s2m = uL + 2.0 * std::sqrt(g * hL) - std::sqrt(g * hm);
                rare1 = true;
                rare2 = false;
            } else {
                s2m = uR - 2.0 * std::sqrt(g * hR) + 3.0 * std::sqrt(g * hm);
                s1m = uR - 2.0 * std::sqrt(g * hR) + std::sqrt(g * hm);
                um = uR - 2.0 * std::sqrt(g * hR) + 2.0 * std::sqrt(g * hm);
                rare2 = true;
                rare1 = false;
            }
        }
    }
    (void)um;
}

// geoclaw_riemann_utils.f: riemann_aug_JCP (rarecorrectortest = .false.)
void riemann_aug_JCP(int maxiter, double hL, double hR, double huL, double huR, double hvL, double hvR,
                     double bL, double bR, double uL, double uR, double vL, double vR, double phiL,
                     double phiR, double pL, double pR, double sE1, double sE2, double drytol, double g,
                     double rho, double sw[3], double fw[3][3]) {
    (void)hvL; (void)hvR;
    double r[3][3], lambda[3], del[3], beta[3] = {0, 0, 0};
    const double delh = hR - hL, delhu = huR - huL, delphi = phiR - phiL, delb = bR - bL, delP = pR - pL;
    double delnorm = delh * delh + delphi * delphi;
    double hm, s1m, s2m;
    bool rare1, rare2;
    riemanntype(hL, hR, uL, uR, hm, s1m, s2m, rare1, rare2, 1, drytol, g);
    lambda[0] = std::min(sE1, s2m);
    lambda[2] = std::max(sE2, s1m);
    sE1 = lambda[0];
    sE2 = lambda[2];
    lambda[1] = 0.0;
    const double hstarHLL = std::max((huL - huR + sE2 * hR - sE1 * hL) / (sE2 - sE1), 0.0);
    const bool rarecorrector = false;
    for (int mw = 0; mw < 3; ++mw) {
        r[0][mw] = 1.0;
        r[1][mw] = lambda[mw];
        r[2][mw] = lambda[mw] * lambda[mw];
    }
    if (!rarecorrector) {
        lambda[1] = 0.5 * (lambda[0] + lambda[2]);
        r[0][1] = 0.0;
        r[1][1] = 0.0;
        r[2][1] = 1.0;
    }
    const double criticaltol = std::max(drytol * g, 1e-6);
    const double criticaltol_2 = std::sqrt(criticaltol);
    double deldelh = -delb;
    double deldelphi = -0.5 * (hR + hL) * (g * delb + delP / rho);
    double hLstar = hL, hRstar = hR, uLstar = uL, uRstar = uR;
    double huLstar = uLstar * hLstar, huRstar = uRstar * hRstar;
    const double convergencetol = 1e-6;
    for (int iter = 1; iter <= maxiter; ++iter) {
        const double hbar = std::max(0.5 * (hLstar + hRstar), 0.0);
        const double s1s2bar = 0.25 * ((uLstar + uRstar) * (uLstar + uRstar)) - g * hbar;
        const double s1s2tilde = std::max(0.0, uLstar * uRstar) - g * hbar;
        bool sonic = false;
        if (std::fabs(s1s2bar) <= criticaltol) sonic = true;
        else if (s1s2bar * s1s2tilde <= criticaltol * criticaltol) sonic = true;
        else if (s1s2bar * sE1 * sE2 <= criticaltol * criticaltol) sonic = true;
        else if (std::min(std::fabs(sE1), std::fabs(sE2)) < criticaltol_2) sonic = true;
        else if (sE1 < criticaltol_2 && s1m > -criticaltol_2) sonic = true;
        else if (sE2 > -criticaltol_2 && s2m < criticaltol_2) sonic = true;
        else if ((uL + std::sqrt(g * hL)) * (uR + std::sqrt(g * hR)) < 0.0) sonic = true;
        else if ((uL - std::sqrt(g * hL)) * (uR - std::sqrt(g * hR)) < 0.0) sonic = true;
        if (sonic) throw std::runtime_error("geoclaw_riemann_utils : sonic == true (the reference stops)");
        deldelh = delb * g * hbar / s1s2bar;
        if (sE1 < -criticaltol && sE2 > criticaltol) {
            deldelh = std::min(deldelh, hstarHLL * (sE2 - sE1) / sE2);
            deldelh = std::max(deldelh, hstarHLL * (sE2 - sE1) / sE1);
        } else if (sE1 >= criticaltol) {
            deldelh = std::min(deldelh, hstarHLL * (sE2 - sE1) / sE1);
            deldelh = std::max(deldelh, -hL);
        } else if (sE2 <= -criticaltol) {
            deldelh = std::min(deldelh, hR);
            deldelh = std::max(deldelh, hstarHLL * (sE2 - sE1) / sE2);
        }
        deldelh = deldelh - delP / (rho * g);
        deldelphi = -(delb * g * hbar * s1s2tilde / s1s2bar);
        deldelphi = std::min(deldelphi, g * std::max(-hLstar * delb, -hRstar * delb));
        deldelphi = std::max(deldelphi, g * std::min(-hLstar * delb, -hRstar * delb));
        deldelphi = deldelphi - hbar * delP / rho;
        del[0] = delh - deldelh;
        del[1] = delhu;
        del[2] = delphi - deldelphi;
        double det1 = r[0][0] * (r[1][1] * r[2][2] - r[1][2] * r[2][1]);
        double det2 = r[0][1] * (r[1][0] * r[2][2] - r[1][2] * r[2][0]);
        double det3 = r[0][2] * (r[1][0] * r[2][1] - r[1][1] * r[2][0]);
        const double determinant = det1 - det2 + det3;
        for (int k = 0; k < 3; ++k) {
            double A[3][3];
            for (int mw = 0; mw < 3; ++mw)
                for (int m = 0; m < 3; ++m) A[m][mw] = r[m][mw];
            A[0][k] = del[0];
            A[1][k] = del[1];
            A[2][k] = del[2];
            det1 = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]);
            det2 = A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]);
            det3 = A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
            beta[k] = (det1 - det2 + det3) / determinant;
        }
        if (std::fabs(del[0] * del[0] + del[2] * del[2] - delnorm) < convergencetol) break;
        delnorm = del[0] * del[0] + del[2] * del[2];
        hLstar = hL; hRstar = hR; uLstar = uL; uRstar = uR;
        huLstar = uLstar * hLstar;
        huRstar = uRstar * hRstar;
        for (int mw = 0; mw < 3; ++mw)
            if (lambda[mw] < 0.0) {
                hLstar = hLstar + beta[mw] * r[0][mw];
                huLstar = huLstar + beta[mw] * r[1][mw];
            }
        for (int mw = 2; mw >= 0; --mw)
            if (lambda[mw] > 0.0) {
                hRstar = hRstar - beta[mw] * r[0][mw];
                huRstar = huRstar - beta[mw] * r[1][mw];
            }
        if (hLstar > drytol) uLstar = huLstar / hLstar;
        else { hLstar = std::max(hLstar, 0.0); uLstar = 0.0; }
        if (hRstar > drytol) uRstar = huRstar / hRstar;
        else { hRstar = std::max(hRstar, 0.0); uRstar = 0.0; }
    }
    for (int mw = 0; mw < 3; ++mw) {
        sw[mw] = lambda[mw];
        fw[0][mw] = beta[mw] * r[1][mw];
        fw[1][mw] = beta[mw] * r[2][mw];
        fw[2][mw] = beta[mw] * r[1][mw];
    }
    fw[2][0] = fw[2][0] * vL;
    fw[2][2] = fw[2][2] * vR;
    fw[2][1] = 0.0;
    const double hustar_interface = huL + fw[0][0];
    if (hustar_interface <= 0.0) fw[2][0] = fw[2][0] + (hR * uR * vR - hL * uL * vL - fw[2][0] - fw[2][2]);
    else fw[2][2] = fw[2][2] + (hR * uR * vR - hL * uL * vL - fw[2][0] - fw[2][2]);
}

// rpn2_geoclaw.f90 (clawpack46 layout), use_simple = .false.
void rpn2_geoclaw(const Slice& S, double grav, double drytol, int ixy, int meqn, int mwaves, int mx,
                  const double* q, const double* aux2, double* wave, double* s, double* amdq, double* apdq) {
    const int L = S.L, mbc = S.mbc;
    const int mu = (ixy == 1) ? 1 : 2;
    const int mv = (ixy == 1) ? 2 : 1;
    auto Q = [&](int i, int m) { return q[m * L + S.at(i)]; };
    auto FW = [&](int i, int m, int mw) -> double& { return wave[(mw * meqn + m) * L + S.at(i)]; };
    const double g = grav, rho = -9999999.0, pL = 0, pR = 0;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        if (Q(i - 1, 0) < 0.0 || Q(i, 0) < 0.0) throw std::runtime_error("rpn2_geoclaw: negative input depth");
        for (int mw = 0; mw < mwaves; ++mw) {
            s[mw * L + S.at(i)] = 0.0;
            FW(i, 0, mw) = 0.0; FW(i, 1, mw) = 0.0; FW(i, 2, mw) = 0;
        }
        if (Q(i - 1, 0) <= drytol && Q(i, 0) <= drytol) continue;
        double hL = Q(i - 1, 0), hR = Q(i, 0), huL = Q(i - 1, mu), huR = Q(i, mu);
        double bL = aux2[0 * L + S.at(i - 1)], bR = aux2[0 * L + S.at(i)];
        double hvL = Q(i - 1, mv), hvR = Q(i, mv);
        double uR, vR, phiR, uL, vL, phiL;
        if (hR > drytol) {
            uR = huR / hR; vR = hvR / hR;
            phiR = 0.5 * grav * (hR * hR) + (huR * huR) / hR;
        } else {
            hR = 0.0; huR = 0.0; hvR = 0.0; uR = 0.0; vR = 0; phiR = 0.0;
        }
        if (hL > drytol) {
            uL = huL / hL; vL = hvL / hL;
            phiL = 0.5 * grav * (hL * hL) + (huL * huL) / hL;
        } else {
            hL = 0.0; huL = 0.0; hvL = 0.0; uL = 0.0; vL = 0.0; phiL = 0.0;
        }
        double wall[3] = {1.0, 1.0, 1.0};
        double hstar, s1m, s2m;
        bool rare1, rare2;
        if (hR <= drytol) {
            riemanntype(hL, hL, uL, -uL, hstar, s1m, s2m, rare1, rare2, 1, drytol, grav);
            const double hstartest = std::max(hL, hstar);
            if (hstartest + bL < bR) {
                wall[1] = 0.0; wall[2] = 0.0;
                hR = hL; huR = -huL; bR = bL; phiR = phiL; uR = -uL; vL = vR;
            } else if (hL + bL < bR) {
                bR = hL + bL;
            }
        } else if (hL <= drytol) {
            riemanntype(hR, hR, -uR, uR, hstar, s1m, s2m, rare1, rare2, 1, drytol, grav);
            const double hstartest = std::max(hR, hstar);
            if (hstartest + bR < bL) {
                wall[0] = 0.0; wall[1] = 0.0;
                hL = hR; huL = -huR; bL = bR; phiL = phiR; uL = -uR; vR = vL;
            } else if (hR + bR < bL) {
                bL = hR + bR;
            }
        }
        const double sL = uL - std::sqrt(grav * hL);
        const double sR = uR + std::sqrt(grav * hR);
        const double uhat = (std::sqrt(grav * hL) * uL + std::sqrt(grav * hR) * uR) /
                            (std::sqrt(grav * hR) + std::sqrt(grav * hL));
        const double chat = std::sqrt(grav * 0.5 * (hR + hL));
        const double sRoe1 = uhat - chat, sRoe2 = uhat + chat;
        const double sE1 = std::min(sL, sRoe1), sE2 = std::max(sR, sRoe2);
        double sw[3], fw[3][3];
        riemann_aug_JCP(1, hL, hR, huL, huR, hvL, hvR, bL, bR, uL, uR, vL, vR, phiL, phiR, pL, pR, sE1, sE2,
                        drytol, g, rho, sw, fw);
        for (int mw = 0; mw < mwaves; ++mw) {
            sw[mw] = sw[mw] * wall[mw];
            fw[0][mw] = fw[0][mw] * wall[mw];
            fw[1][mw] = fw[1][mw] * wall[mw];
            fw[2][mw] = fw[2][mw] * wall[mw];
        }
        for (int mw = 0; mw < mwaves; ++mw) {
            s[mw * L + S.at(i)] = sw[mw];
            FW(i, 0, mw) = fw[0][mw];
            FW(i, mu, mw) = fw[1][mw];
            FW(i, mv, mw) = fw[2][mw];
        }
    }
    for (int i = 2 - mbc; i <= mx + mbc; ++i)
        for (int m = 0; m < 3; ++m) {
            amdq[m * L + S.at(i)] = 0.0;
            apdq[m * L + S.at(i)] = 0.0;
        }
    for (int i = 2 - mbc; i <= mx + mbc; ++i)
        for (int mw = 0; mw < 3; ++mw) {
            const double sv = s[mw * L + S.at(i)];
            for (int m = 0; m < 3; ++m) {
                double& am = amdq[m * L + S.at(i)];
                double& ap = apdq[m * L + S.at(i)];
                if (sv < 0.0) am = am + FW(i, m, mw);
                else if (sv > 0.0) ap = ap + FW(i, m, mw);
                else {
                    am = am + 0.5 * FW(i, m, mw);
                    ap = ap + 0.5 * FW(i, m, mw);
                }
            }
        }
}

// applications/clawpack/advection/2d/all/clawpack46_rpn2adv.f:1-61; with
// shift = 1, clawpack46_rpn2adv_manifold.f:1-42 (s = auxl(i, 1+ixy): the edge
// velocities follow the capacity in aux(1)); clawpack5_rpn2adv(_manifold).f90
// have the same arithmetic
void rpn2_adv(const Slice& S, int ixy, int meqn, int mwaves, int mx, const double* q,
              const double* auxl, double* wave, double* s, double* amdq, double* apdq, int shift) {
    const int L = S.L, mbc = S.mbc;
    const int iface = ixy + shift;  // aux component 1 (+shift) = x velocity, 2 (+shift) = y velocity
    double delta[10];
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const int ii = S.at(i);
        for (int mq = 0; mq < meqn; ++mq)
            for (int mw = 0; mw < mwaves; ++mw) wave[(mw * meqn + mq) * L + ii] = 0.0;
        for (int mq = 0; mq < meqn; ++mq) {
            delta[mq] = q[mq * L + ii] - q[mq * L + ii - 1];
            for (int mw = 0; mw < mwaves; ++mw) wave[(mw * meqn + mq) * L + ii] = delta[mq];
        }
        for (int mw = 0; mw < mwaves; ++mw) s[mw * L + ii] = auxl[(iface - 1) * L + ii];
        for (int mq = 0; mq < meqn; ++mq) {
            amdq[mq * L + ii] = 0.0;
            apdq[mq * L + ii] = 0.0;
            for (int mw = 0; mw < mwaves; ++mw) {
                const double sw = s[mw * L + ii];
                const double w = wave[(mw * meqn + mq) * L + ii];
                amdq[mq * L + ii] = amdq[mq * L + ii] + dmin(sw, 0.0) * w;
                apdq[mq * L + ii] = apdq[mq * L + ii] + dmax(sw, 0.0) * w;
            }
        }
    }
}

// applications/clawpack/advection/2d/all/clawpack46_rpt2adv.f:62-89; with
// shift = 1, clawpack46_rpt2adv_manifold.f:1-44 (aux(i1, iface+1))
void rpt2_adv(const Slice& S, int ixy, int meqn, int mx, const double* aux2, const double* aux3,
              int imp, const double* asdq, double* bmasdq, double* bpasdq, int shift) {
    const int L = S.L, mbc = S.mbc;
    const int kv = 3 - ixy + shift;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const int ii = S.at(i);
        const int i1 = S.at(i - 2 + imp);
        for (int mq = 0; mq < meqn; ++mq) {
            bmasdq[mq * L + ii] = dmin(aux2[(kv - 1) * L + i1], 0.0) * asdq[mq * L + ii];
            bpasdq[mq * L + ii] = dmax(aux3[(kv - 1) * L + i1], 0.0) * asdq[mq * L + ii];
        }
    }
}

// applications/clawpack/shallow/2d/rp/clawpack46_rpn2.f:1-247 (entropy fix on)
// v5: applications/clawpack/shallow/2d/rp/clawpack5_rpn2.f90 (a1, a3 scaled by
// (0.5/a) instead of divided by 2a)
void rpn2_swe(const Slice& S, RiemannState& R, double grav, int ixy, int meqn, int mwaves, int mx,
              const double* q, double* wave, double* s, double* amdq, double* apdq, bool v5) {
    const int L = S.L, mbc = S.mbc;
    const int mu = (ixy == 1) ? 1 : 2;  // 0-based component of normal momentum
    const int mv = (ixy == 1) ? 2 : 1;
    auto Q = [&](int i, int m) { return q[m * L + S.at(i)]; };
    auto W = [&](int i, int m, int mw) -> double& { return wave[(mw * meqn + m) * L + S.at(i)]; };
    auto Sp = [&](int i, int mw) -> double& { return s[mw * L + S.at(i)]; };
    auto AM = [&](int i, int m) -> double& { return amdq[m * L + S.at(i)]; };
    auto AP = [&](int i, int m) -> double& { return apdq[m * L + S.at(i)]; };
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const int ii = S.at(i);
        R.h[ii] = (Q(i - 1, 0) + Q(i, 0)) / 2.0;
        const double hsqrtl = std::sqrt(Q(i - 1, 0));
        const double hsqrtr = std::sqrt(Q(i, 0));
        const double hsq2 = hsqrtl + hsqrtr;
        R.u[ii] = (Q(i - 1, mu) / hsqrtl + Q(i, mu) / hsqrtr) / hsq2;
        R.v[ii] = (Q(i - 1, mv) / hsqrtl + Q(i, mv) / hsqrtr) / hsq2;
        R.a[ii] = std::sqrt(grav * R.h[ii]);
    }
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const int ii = S.at(i);
        const double u = R.u[ii], v = R.v[ii], a = R.a[ii];
        const double d1 = Q(i, 0) - Q(i - 1, 0);
        const double d2 = Q(i, mu) - Q(i - 1, mu);
        const double d3 = Q(i, mv) - Q(i - 1, mv);
        const double a1 = v5 ? ((u + a) * d1 - d2) * (0.50 / a) : ((u + a) * d1 - d2) / (2.0 * a);
        const double a2 = -(v * d1) + d3;
        const double a3 = v5 ? (-((u - a) * d1) + d2) * (0.50 / a) : (-((u - a) * d1) + d2) / (2.0 * a);
        W(i, 0, 0) = a1; W(i, mu, 0) = a1 * (u - a); W(i, mv, 0) = a1 * v; Sp(i, 0) = u - a;
        W(i, 0, 1) = 0.0; W(i, mu, 1) = 0.0; W(i, mv, 1) = a2; Sp(i, 1) = u;
        W(i, 0, 2) = a3; W(i, mu, 2) = a3 * (u + a); W(i, mv, 2) = a3 * v; Sp(i, 2) = u + a;
    }
    // entropy fix (label 110)
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const double him1 = Q(i - 1, 0);
        const double s0 = Q(i - 1, mu) / him1 - std::sqrt(grav * him1);
        double sfract;
        if (s0 > 0.0 && Sp(i, 0) > 0.0) {
            for (int m = 0; m < 3; ++m) AM(i, m) = 0.0;
            goto done;
        }
        {
            const double h1 = Q(i - 1, 0) + W(i, 0, 0);
            const double hu1 = Q(i - 1, mu) + W(i, mu, 0);
            const double s1 = hu1 / h1 - std::sqrt(grav * h1);
            if (s0 < 0.0 && s1 > 0.0) sfract = s0 * ((s1 - Sp(i, 0)) / (s1 - s0));
            else if (Sp(i, 0) < 0.0) sfract = Sp(i, 0);
            else sfract = 0.0;
            for (int m = 0; m < 3; ++m) AM(i, m) = sfract * W(i, m, 0);
        }
        if (Sp(i, 1) > 0.0) goto done;
        for (int m = 0; m < 3; ++m) AM(i, m) = AM(i, m) + Sp(i, 1) * W(i, m, 1);
        {
            const double hi = Q(i, 0);
            const double s03 = Q(i, mu) / hi + std::sqrt(grav * hi);
            const double h3 = Q(i, 0) - W(i, 0, 2);
            const double hu3 = Q(i, mu) - W(i, mu, 2);
            const double s3 = hu3 / h3 + std::sqrt(grav * h3);
            if (s3 < 0.0 && s03 > 0.0) sfract = s3 * ((s03 - Sp(i, 2)) / (s03 - s3));
            else if (Sp(i, 2) < 0.0) sfract = Sp(i, 2);
            else goto done;
            for (int m = 0; m < 3; ++m) AM(i, m) = AM(i, m) + sfract * W(i, m, 2);
        }
    done:;
    }
    for (int m = 0; m < 3; ++m)
        for (int i = 2 - mbc; i <= mx + mbc; ++i) {
            double df = 0.0;
            for (int mw = 0; mw < mwaves; ++mw) df = df + Sp(i, mw) * W(i, m, mw);
            AP(i, m) = df - AM(i, m);
        }
}

// applications/clawpack/shallow/2d/rp/clawpack46_rpt2.f:1-74
// v5: clawpack5_rpt2.f90 (the Roe averages it recomputes equal rpn2's)
void rpt2_swe(const Slice& S, const RiemannState& R, int ixy, int meqn, int mwaves, int mx,
              const double* asdq, double* bmasdq, double* bpasdq, bool v5) {
    const int L = S.L, mbc = S.mbc;
    const int mu = (ixy == 1) ? 1 : 2;
    const int mv = (ixy == 1) ? 2 : 1;
    double waveb[3][3], sb[3];
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const int ii = S.at(i);
        const double u = R.u[ii], v = R.v[ii], a = R.a[ii];
        const double q1 = asdq[0 * L + ii], qmu = asdq[mu * L + ii], qmv = asdq[mv * L + ii];
        const double a1 = v5 ? (0.50 / a) * ((v + a) * q1 - qmv) : ((v + a) * q1 - qmv) / (2 * a);
        const double a2 = qmu - u * q1;
        const double a3 = v5 ? (0.50 / a) * (-((v - a) * q1) + qmv) : (-((v - a) * q1) + qmv) / (2 * a);
        waveb[0][0] = a1; waveb[mu][0] = a1 * u; waveb[mv][0] = a1 * (v - a); sb[0] = v - a;
        waveb[0][1] = 0.0; waveb[mu][1] = a2; waveb[mv][1] = 0.0; sb[1] = v;
        waveb[0][2] = a3; waveb[mu][2] = a3 * u; waveb[mv][2] = a3 * (v + a); sb[2] = v + a;
        for (int m = 0; m < meqn; ++m) {
            double bm = 0.0, bp = 0.0;
            for (int mw = 0; mw < mwaves; ++mw) {
                bm = bm + dmin(sb[mw], 0.0) * waveb[m][mw];
                bp = bp + dmax(sb[mw], 0.0) * waveb[m][mw];
            }
            bmasdq[m * L + ii] = bm;
            bpasdq[m * L + ii] = bp;
        }
    }
}

// applications/clawpack/euler/2d/rp/clawpack46_rpn2_euler4.f:1-289 (entropy fix on)
void rpn2_euler4(const Slice& S, RiemannState& R, double gamma, double gamma1, int ixy, int meqn,
                 int mwaves, int mx, const double* q, double* wave, double* s, double* amdq,
                 double* apdq) {
    const int L = S.L, mbc = S.mbc;
    const int mu = (ixy == 1) ? 1 : 2;
    const int mv = (ixy == 1) ? 2 : 1;
    auto Q = [&](int i, int m) { return q[m * L + S.at(i)]; };
    auto W = [&](int i, int m, int mw) -> double& { return wave[(mw * meqn + m) * L + S.at(i)]; };
    auto Sp = [&](int i, int mw) -> double& { return s[mw * L + S.at(i)]; };
    auto AM = [&](int i, int m) -> double& { return amdq[m * L + S.at(i)]; };
    auto AP = [&](int i, int m) -> double& { return apdq[m * L + S.at(i)]; };
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const int ii = S.at(i);
        const double rhsqrtl = std::sqrt(Q(i - 1, 0));
        const double rhsqrtr = std::sqrt(Q(i, 0));
        const double pl = gamma1 * (Q(i - 1, 3) - 0.5 * (Q(i - 1, 1) * Q(i - 1, 1) +
                                                          Q(i - 1, 2) * Q(i - 1, 2)) / Q(i - 1, 0));
        const double pr = gamma1 * (Q(i, 3) - 0.5 * (Q(i, 1) * Q(i, 1) + Q(i, 2) * Q(i, 2)) / Q(i, 0));
        const double rhsq2 = rhsqrtl + rhsqrtr;
        R.u[ii] = (Q(i - 1, mu) / rhsqrtl + Q(i, mu) / rhsqrtr) / rhsq2;
        R.v[ii] = (Q(i - 1, mv) / rhsqrtl + Q(i, mv) / rhsqrtr) / rhsq2;
        R.enth[ii] = (((Q(i - 1, 3) + pl) / rhsqrtl + (Q(i, 3) + pr) / rhsqrtr)) / rhsq2;
        R.u2v2[ii] = R.u[ii] * R.u[ii] + R.v[ii] * R.v[ii];
        const double a2 = gamma1 * (R.enth[ii] - 0.5 * R.u2v2[ii]);
        R.a[ii] = std::sqrt(a2);
        R.g1a2[ii] = gamma1 / a2;
        R.euv[ii] = R.enth[ii] - R.u2v2[ii];
    }
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const int ii = S.at(i);
        const double u = R.u[ii], v = R.v[ii], a = R.a[ii], enth = R.enth[ii];
        const double d1 = Q(i, 0) - Q(i - 1, 0);
        const double d2 = Q(i, mu) - Q(i - 1, mu);
        const double d3 = Q(i, mv) - Q(i - 1, mv);
        const double d4 = Q(i, 3) - Q(i - 1, 3);
        const double a3 = R.g1a2[ii] * (R.euv[ii] * d1 + u * d2 + v * d3 - d4);
        const double a2 = d3 - v * d1;
        const double a4 = (d2 + (a - u) * d1 - a * a3) / (2.0 * a);
        const double a1 = d1 - a3 - a4;
        W(i, 0, 0) = a1; W(i, mu, 0) = a1 * (u - a); W(i, mv, 0) = a1 * v;
        W(i, 3, 0) = a1 * (enth - u * a); Sp(i, 0) = u - a;
        W(i, 0, 1) = 0.0; W(i, mu, 1) = 0.0; W(i, mv, 1) = a2; W(i, 3, 1) = a2 * v; Sp(i, 1) = u;
        W(i, 0, 2) = a3; W(i, mu, 2) = a3 * u; W(i, mv, 2) = a3 * v;
        W(i, 3, 2) = a3 * 0.5 * R.u2v2[ii]; Sp(i, 2) = u;
        W(i, 0, 3) = a4; W(i, mu, 3) = a4 * (u + a); W(i, mv, 3) = a4 * v;
        W(i, 3, 3) = a4 * (enth + u * a); Sp(i, 3) = u + a;
    }
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const double rhoim1 = Q(i - 1, 0);
        const double pim1 = gamma1 * (Q(i - 1, 3) - 0.5 * (Q(i - 1, mu) * Q(i - 1, mu) +
                                                           Q(i - 1, mv) * Q(i - 1, mv)) / rhoim1);
        const double cim1 = std::sqrt(gamma * pim1 / rhoim1);
        const double s0 = Q(i - 1, mu) / rhoim1 - cim1;
        double sfract;
        if (s0 >= 0.0 && Sp(i, 0) > 0.0) {
            for (int m = 0; m < meqn; ++m) AM(i, m) = 0.0;
            goto done;
        }
        {
            const double rho1 = Q(i - 1, 0) + W(i, 0, 0);
            const double rhou1 = Q(i - 1, mu) + W(i, mu, 0);
            const double rhov1 = Q(i - 1, mv) + W(i, mv, 0);
            const double en1 = Q(i - 1, 3) + W(i, 3, 0);
            const double p1 = gamma1 * (en1 - 0.5 * (rhou1 * rhou1 + rhov1 * rhov1) / rho1);
            const double c1 = std::sqrt(gamma * p1 / rho1);
            const double s1 = rhou1 / rho1 - c1;
            if (s0 < 0.0 && s1 > 0.0) sfract = s0 * (s1 - Sp(i, 0)) / (s1 - s0);
            else if (Sp(i, 0) < 0.0) sfract = Sp(i, 0);
            else sfract = 0.0;
            for (int m = 0; m < meqn; ++m) AM(i, m) = sfract * W(i, m, 0);
        }
        if (Sp(i, 1) >= 0.0) goto done;
        for (int m = 0; m < meqn; ++m) {
            AM(i, m) = AM(i, m) + Sp(i, 1) * W(i, m, 1);
            AM(i, m) = AM(i, m) + Sp(i, 2) * W(i, m, 2);
        }
        {
            const double rhoi = Q(i, 0);
            const double pi = gamma1 * (Q(i, 3) - 0.5 * (Q(i, mu) * Q(i, mu) +
                                                         Q(i, mv) * Q(i, mv)) / rhoi);
            const double ci = std::sqrt(gamma * pi / rhoi);
            const double s3 = Q(i, mu) / rhoi + ci;
            const double rho2 = Q(i, 0) - W(i, 0, 3);
            const double rhou2 = Q(i, mu) - W(i, mu, 3);
            const double rhov2 = Q(i, mv) - W(i, mv, 3);
            const double en2 = Q(i, 3) - W(i, 3, 3);
            const double p2 = gamma1 * (en2 - 0.5 * (rhou2 * rhou2 + rhov2 * rhov2) / rho2);
            const double c2 = std::sqrt(gamma * p2 / rho2);
            const double s2 = rhou2 / rho2 + c2;
            if (s2 < 0.0 && s3 > 0.0) sfract = s2 * (s3 - Sp(i, 3)) / (s3 - s2);
            else if (Sp(i, 3) < 0.0) sfract = Sp(i, 3);
            else goto done;
            for (int m = 0; m < meqn; ++m) AM(i, m) = AM(i, m) + sfract * W(i, m, 3);
        }
    done:;
    }
    for (int m = 0; m < meqn; ++m)
        for (int i = 2 - mbc; i <= mx + mbc; ++i) {
            double df = 0.0;
            for (int mw = 0; mw < mwaves; ++mw) df = df + Sp(i, mw) * W(i, m, mw);
            AP(i, m) = df - AM(i, m);
        }
}

// applications/clawpack/euler/2d/rp/clawpack46_rpt2_euler4.f:290-386
void rpt2_euler4(const Slice& S, const RiemannState& R, int ixy, int meqn, int mx,
                 const double* asdq, double* bmasdq, double* bpasdq) {
    const int L = S.L, mbc = S.mbc;
    const int mu = (ixy == 1) ? 1 : 2;
    const int mv = (ixy == 1) ? 2 : 1;
    double waveb[4][3], sb[3];
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        const int ii = S.at(i);
        const double u = R.u[ii], v = R.v[ii], a = R.a[ii], enth = R.enth[ii];
        const double q1 = asdq[0 * L + ii], qmu = asdq[mu * L + ii], qmv = asdq[mv * L + ii],
                     q4 = asdq[3 * L + ii];
        const double a3 = R.g1a2[ii] * (R.euv[ii] * q1 + u * qmu + v * qmv - q4);
        const double a2 = qmu - u * q1;
        const double a4 = (qmv + (a - v) * q1 - a * a3) / (2.0 * a);
        const double a1 = q1 - a3 - a4;
        waveb[0][0] = a1; waveb[mu][0] = a1 * u; waveb[mv][0] = a1 * (v - a);
        waveb[3][0] = a1 * (enth - v * a); sb[0] = v - a;
        waveb[0][1] = a3; waveb[mu][1] = a3 * u + a2; waveb[mv][1] = a3 * v;
        waveb[3][1] = a3 * 0.5 * R.u2v2[ii] + a2 * u; sb[1] = v;
        waveb[0][2] = a4; waveb[mu][2] = a4 * u; waveb[mv][2] = a4 * (v + a);
        waveb[3][2] = a4 * (enth + v * a); sb[2] = v + a;
        for (int m = 0; m < meqn; ++m) {
            double bm = 0.0, bp = 0.0;
            for (int mw = 0; mw < 3; ++mw) {
                bm = bm + dmin(sb[mw], 0.0) * waveb[m][mw];
                bp = bp + dmax(sb[mw], 0.0) * waveb[m][mw];
            }
            bmasdq[m * L + ii] = bm;
            bpasdq[m * L + ii] = bp;
        }
    }
}

// src/solvers/fc2d_clawpack4.6/fortran_source/clawpack46_inlinelimiter.f:4-118
// v5: clawpack5_inlinelimiter.f:4-109 (codes 1-5; others fall to label 10)
void inlinelimiter(const Slice& S, int meqn, int mwaves, int mx, double* wave, const double* s,
                   const int* mthlim, bool v5) {
    const int L = S.L;
    auto W = [&](int i, int m, int mw) -> double& { return wave[(mw * meqn + m) * L + S.at(i)]; };
    for (int mw = 0; mw < mwaves; ++mw) {
        if (mthlim[mw] == 0) continue;
        double dotr = 0.0;
        for (int i = 0; i <= mx + 1; ++i) {
            double wnorm2 = 0.0;
            const double dotl = dotr;
            dotr = 0.0;
            for (int m = 0; m < meqn; ++m) {
                wnorm2 = wnorm2 + W(i, m, mw) * W(i, m, mw);
                dotr = dotr + W(i, m, mw) * W(i + 1, m, mw);
            }
            if (i == 0) continue;
            if (wnorm2 == 0.0) continue;
            const double r = (s[mw * L + S.at(i)] > 0.0) ? dotl / wnorm2 : dotr / wnorm2;
            double wlimitr;
            switch ((v5 && mthlim[mw] > 5) ? 1 : mthlim[mw]) {
                case 2: wlimitr = dmax(dmax(0.0, dmin(1.0, 2.0 * r)), dmin(2.0, r)); break;
                case 3: wlimitr = (r + std::fabs(r)) / (1.0 + std::fabs(r)); break;
                case 4: {
                    const double c = (1.0 + r) / 2.0;
                    wlimitr = dmax(0.0, dmin(dmin(c, 2.0), 2.0 * r));
                    break;
                }
                case 5: wlimitr = r; break;
                case 6: {
                    const double th = (double)1.3f;  // REAL*4 literal assigned to a double
                    wlimitr = dmax(0.0, dmin(dmin(th * r, (1 + r) / 2.0), th));
                    break;
                }
                default:  // 1 and out-of-range values fall to label 10 (minmod)
                    wlimitr = dmax(0.0, dmin(1.0, r));
                    break;
            }
            for (int m = 0; m < meqn; ++m) W(i, m, mw) = wlimitr * W(i, m, mw);
        }
    }
}

struct Work {
    Slice S;
    int meqn, maux, mwaves;
    bool v5 = false;  // clawpack 5 solver arithmetic
    std::vector<double> q1d, dtdx1d, dtdy1d, aux1, aux2, aux3, faddm, faddp, gaddm, gaddp;
    std::vector<double> wave, s, amdq, apdq, cqxx, bmasdq, bpasdq;
    RiemannState R;
    Work(int maxm, int mbc, int meqn_, int maux_, int mwaves_)
        : S(maxm, mbc), meqn(meqn_), maux(maux_), mwaves(mwaves_) {
        const int L = S.L;
        q1d.assign((size_t)L * meqn, 0); dtdx1d.assign(L, 0); dtdy1d.assign(L, 0);
        aux1.assign((size_t)L * std::max(maux, 1), 0); aux2 = aux1; aux3 = aux1;
        faddm.assign((size_t)L * meqn, 0); faddp = faddm;
        gaddm.assign((size_t)L * meqn * 2, 0); gaddp = gaddm;
        wave.assign((size_t)L * meqn * mwaves, 0); s.assign((size_t)L * mwaves, 0);
        amdq.assign((size_t)L * meqn, 0); apdq = amdq; cqxx = amdq; bmasdq = amdq; bpasdq = amdq;
        R.resize(L);
    }
};

void call_rpn2(const SolverParams& sp, Work& w, int ixy, int mx) {
    switch (sp.kind) {
        case SOLVER_ADVECTION:
        case SOLVER_ADVECTION_MANIFOLD:
            rpn2_adv(w.S, ixy, w.meqn, w.mwaves, mx, w.q1d.data(), w.aux2.data(), w.wave.data(),
                     w.s.data(), w.amdq.data(), w.apdq.data(), sp.kind == SOLVER_ADVECTION_MANIFOLD);
            break;
        case SOLVER_SWE_ROE:
            rpn2_swe(w.S, w.R, sp.grav, ixy, w.meqn, w.mwaves, mx, w.q1d.data(), w.wave.data(),
                     w.s.data(), w.amdq.data(), w.apdq.data(), w.v5);
            break;
        case SOLVER_EULER4_ROE:
            rpn2_euler4(w.S, w.R, sp.gamma, sp.gamma1, ixy, w.meqn, w.mwaves, mx, w.q1d.data(),
                        w.wave.data(), w.s.data(), w.amdq.data(), w.apdq.data());
            break;
        case SOLVER_GEOCLAW_FWAVE:
            rpn2_geoclaw(w.S, sp.grav, sp.drytol, ixy, w.meqn, w.mwaves, mx, w.q1d.data(), w.aux2.data(),
                         w.wave.data(), w.s.data(), w.amdq.data(), w.apdq.data());
            break;
        default: throw std::runtime_error("unknown solver kind");
    }
}

void call_rpt2(const SolverParams& sp, Work& w, int ixy, int mx, int imp, const double* asdq) {
    switch (sp.kind) {
        case SOLVER_ADVECTION:
        case SOLVER_ADVECTION_MANIFOLD:
            rpt2_adv(w.S, ixy, w.meqn, mx, w.aux2.data(), w.aux3.data(), imp, asdq,
                     w.bmasdq.data(), w.bpasdq.data(), sp.kind == SOLVER_ADVECTION_MANIFOLD);
            break;
        case SOLVER_SWE_ROE:
            rpt2_swe(w.S, w.R, ixy, w.meqn, w.mwaves, mx, asdq, w.bmasdq.data(), w.bpasdq.data(), w.v5);
            break;
        case SOLVER_EULER4_ROE:
            rpt2_euler4(w.S, w.R, ixy, w.meqn, mx, asdq, w.bmasdq.data(), w.bpasdq.data());
            break;
        default: throw std::runtime_error("unknown solver kind");
    }
}

// src/solvers/fc2d_clawpack4.6/fortran_source/clawpack46_flux2.f:4-228; with
// mp.version == 5, fc2d_clawpack5/fortran_source/clawpack5_flux2.f:4-235, whose
// Godunov, correction and transverse loops all run over i = 1..mx+1.
double flux2(const SolverParams& sp, const MethodParams& mp, Work& w, int ixy, int mx,
             const double* dtdx1d) {
    const Slice& S = w.S;
    const int L = S.L, mbc = S.mbc, meqn = w.meqn, mwaves = w.mwaves;
    const bool v5 = mp.version == 5;
    // f-waves: clawpack46_flux2fw.f (Godunov and cqxx over i = 1..mx+1, cqxx
    // weighted by sign(s); the reference's rpt2_geoclaw stops, so no transverse part)
    const bool fw = sp.kind == SOLVER_GEOCLAW_FWAVE;
    if (fw && mp.order1 > 0) throw std::runtime_error("rpt2_geoclaw stops in the reference: use order (2, 0)");
    const int god_lo = (v5 || fw) ? 1 : 2 - mbc, god_hi = (v5 || fw) ? mx + 1 : mx + mbc - 1;  // Godunov
    const int cq_lo = (v5 || fw) ? 1 : 2 - mbc, cq_hi = (v5 || fw) ? mx + 1 : mx + mbc;          // cqxx
    bool limit = false;
    for (int mw = 0; mw < mwaves; ++mw)
        if (mp.mthlim[mw] > 0) limit = true;
    for (int side = 0; side < 2; ++side)
        for (int m = 0; m < meqn; ++m)
            for (int i = 1 - mbc; i <= mx + mbc; ++i) {
                w.faddm[m * L + S.at(i)] = 0.0;
                w.faddp[m * L + S.at(i)] = 0.0;
                w.gaddm[(side * meqn + m) * L + S.at(i)] = 0.0;
                w.gaddp[(side * meqn + m) * L + S.at(i)] = 0.0;
            }
    call_rpn2(sp, w, ixy, mx);
    for (int i = god_lo; i <= god_hi; ++i)
        for (int m = 0; m < meqn; ++m) {
            const int k = m * L + S.at(i);
            w.faddp[k] = w.faddp[k] - w.apdq[k];
            w.faddm[k] = w.faddm[k] + w.amdq[k];
        }
    double cfl1d = 0.0;
    for (int mw = 0; mw < mwaves; ++mw)
        for (int i = 1; i <= mx + 1; ++i) {
            const double sw = w.s[mw * L + S.at(i)];
            cfl1d = dmax(dmax(cfl1d, dtdx1d[S.at(i)] * sw), -dtdx1d[S.at(i - 1)] * sw);
        }
    if (mp.order0 == 2) {
        if (limit) inlinelimiter(S, meqn, mwaves, mx, w.wave.data(), w.s.data(), mp.mthlim, w.v5);
        for (int i = cq_lo; i <= cq_hi; ++i) {
            const double dtdxave = 0.5 * (dtdx1d[S.at(i - 1)] + dtdx1d[S.at(i)]);
            for (int m = 0; m < meqn; ++m) {
                const int k = m * L + S.at(i);
                w.cqxx[k] = 0.0;
                for (int mw = 0; mw < mwaves; ++mw) {
                    const double sv = w.s[mw * L + S.at(i)];
                    const double as = std::fabs(sv);
                    const double abs_sign = fw ? fsign(1.0, sv) : as;
                    w.cqxx[k] = w.cqxx[k] + abs_sign * (1.0 - as * dtdxave) *
                                                w.wave[(mw * meqn + m) * L + S.at(i)];
                }
                w.faddm[k] = w.faddm[k] + 0.5 * w.cqxx[k];
                w.faddp[k] = w.faddp[k] + 0.5 * w.cqxx[k];
            }
        }
    }
    if (mp.order1 > 0) {
        if (mp.order0 > 1 && mp.order1 == 2)
            for (int i = god_lo; i <= god_hi; ++i)
                for (int m = 0; m < meqn; ++m) {
                    const int k = m * L + S.at(i);
                    w.amdq[k] = w.amdq[k] + w.cqxx[k];
                    w.apdq[k] = w.apdq[k] - w.cqxx[k];
                }
        call_rpt2(sp, w, ixy, mx, 1, w.amdq.data());
        for (int m = 0; m < meqn; ++m)
            for (int i = cq_lo; i <= cq_hi; ++i) {
                const int k = m * L + S.at(i);
                const int k1 = (0 * meqn + m) * L + S.at(i - 1);
                const int k2 = (1 * meqn + m) * L + S.at(i - 1);
                double gupdate = 0.5 * dtdx1d[S.at(i - 1)] * w.bmasdq[k];
                w.gaddm[k1] = w.gaddm[k1] - gupdate;
                w.gaddp[k1] = w.gaddp[k1] - gupdate;
                gupdate = 0.5 * dtdx1d[S.at(i - 1)] * w.bpasdq[k];
                w.gaddm[k2] = w.gaddm[k2] - gupdate;
                w.gaddp[k2] = w.gaddp[k2] - gupdate;
            }
        call_rpt2(sp, w, ixy, mx, 2, w.apdq.data());
        for (int m = 0; m < meqn; ++m)
            for (int i = cq_lo; i <= cq_hi; ++i) {
                const int k = m * L + S.at(i);
                const int k1 = (0 * meqn + m) * L + S.at(i);
                const int k2 = (1 * meqn + m) * L + S.at(i);
                double gupdate = 0.5 * dtdx1d[S.at(i)] * w.bmasdq[k];
                w.gaddm[k1] = w.gaddm[k1] - gupdate;
                w.gaddp[k1] = w.gaddp[k1] - gupdate;
                gupdate = 0.5 * dtdx1d[S.at(i)] * w.bpasdq[k];
                w.gaddm[k2] = w.gaddm[k2] - gupdate;
                w.gaddp[k2] = w.gaddp[k2] - gupdate;
            }
    }
    return cfl1d;
}

}  // namespace

double step2(const SolverParams& sp, const MethodParams& mp, int mx, int my, int mbc, int meqn,
             int maux, double* q, const double* aux, double dx, double dy, double dt, StepFluxArrays* keep) {
    const PatchIdx P(mx, my, mbc);
    const int maxm = std::max(mx, my);
    const int mwaves = mp.mwaves;
    const bool capa = mp.mcapa > 0;
    Work w(maxm, mbc, meqn, maux, mwaves);
    w.v5 = mp.version == 5;
    // accumulation ranges of fm/fp/gm/gp (clawpack46_step2.f:240-294 / clawpack5_step2.f90:
    // 1..mx+1) and of the update (clawpack46_step2_wrap.f:106-125 / clawpack5_step2_wrap.f:94-113)
    const int acc_lo = w.v5 ? 1 : 2 - mbc;
    const int accx_hi = w.v5 ? mx + 1 : mx + mbc, accy_hi = w.v5 ? my + 1 : my + mbc;
    const int upd_lo = w.v5 ? 1 : 1 - mbc;
    const int updx_hi = w.v5 ? mx : mx + mbc - 1, updy_hi = w.v5 ? my : my + mbc - 1;
    const Slice& S = w.S;
    const int L = S.L;
    const size_t n = (size_t)P.size(meqn);
    std::vector<double> fm(n, 0.0), fp(n, 0.0), gm(n, 0.0), gp(n, 0.0);

    double cflgrid = 0.0;
    const double dtdx = dt / dx, dtdy = dt / dy;
    if (!capa)
        for (int i = 1 - mbc; i <= maxm + mbc; ++i) {
            w.dtdx1d[S.at(i)] = dtdx;
            w.dtdy1d[S.at(i)] = dtdy;
        }

    // x-sweeps (clawpack46_step2.f:113-167)
    for (int j = 2 - mbc; j <= my + mbc - 1; ++j) {
        for (int m = 0; m < meqn; ++m)
            for (int i = 1 - mbc; i <= mx + mbc; ++i) w.q1d[m * L + S.at(i)] = q[P(i, j, m)];
        if (capa)
            for (int i = 1 - mbc; i <= mx + mbc; ++i)
                w.dtdx1d[S.at(i)] = dtdx / aux[P(i, j, mp.mcapa - 1)];
        if (maux > 0)
            for (int ma = 0; ma < maux; ++ma)
                for (int i = 1 - mbc; i <= mx + mbc; ++i) {
                    w.aux1[ma * L + S.at(i)] = aux[P(i, j - 1, ma)];
                    w.aux2[ma * L + S.at(i)] = aux[P(i, j, ma)];
                    w.aux3[ma * L + S.at(i)] = aux[P(i, j + 1, ma)];
                }
        const double cfl1d = flux2(sp, mp, w, 1, mx, w.dtdx1d.data());
        cflgrid = dmax(cflgrid, cfl1d);
        for (int m = 0; m < meqn; ++m)
            for (int i = acc_lo; i <= accx_hi; ++i) {
                const int k = m * L + S.at(i);
                fm[P(i, j, m)] = fm[P(i, j, m)] + w.faddm[k];
                fp[P(i, j, m)] = fp[P(i, j, m)] + w.faddp[k];
                gm[P(i, j, m)] = gm[P(i, j, m)] + w.gaddm[(0 * meqn + m) * L + S.at(i)];
                gp[P(i, j, m)] = gp[P(i, j, m)] + w.gaddp[(0 * meqn + m) * L + S.at(i)];
                gm[P(i, j + 1, m)] = gm[P(i, j + 1, m)] + w.gaddm[(1 * meqn + m) * L + S.at(i)];
                gp[P(i, j + 1, m)] = gp[P(i, j + 1, m)] + w.gaddp[(1 * meqn + m) * L + S.at(i)];
            }
    }
    // y-sweeps (clawpack46_step2.f:182-236)
    for (int i = 2 - mbc; i <= mx + mbc - 1; ++i) {
        for (int m = 0; m < meqn; ++m)
            for (int j = 1 - mbc; j <= my + mbc; ++j) w.q1d[m * L + S.at(j)] = q[P(i, j, m)];
        if (capa)
            for (int j = 1 - mbc; j <= my + mbc; ++j)
                w.dtdy1d[S.at(j)] = dtdy / aux[P(i, j, mp.mcapa - 1)];
        if (maux > 0)
            for (int ma = 0; ma < maux; ++ma)
                for (int j = 1 - mbc; j <= my + mbc; ++j) {
                    w.aux1[ma * L + S.at(j)] = aux[P(i - 1, j, ma)];
                    w.aux2[ma * L + S.at(j)] = aux[P(i, j, ma)];
                    w.aux3[ma * L + S.at(j)] = aux[P(i + 1, j, ma)];
                }
        const double cfl1d = flux2(sp, mp, w, 2, my, w.dtdy1d.data());
        cflgrid = dmax(cflgrid, cfl1d);
        for (int m = 0; m < meqn; ++m)
            for (int j = acc_lo; j <= accy_hi; ++j) {
                const int k = m * L + S.at(j);
                gm[P(i, j, m)] = gm[P(i, j, m)] + w.faddm[k];
                gp[P(i, j, m)] = gp[P(i, j, m)] + w.faddp[k];
                fm[P(i, j, m)] = fm[P(i, j, m)] + w.gaddm[(0 * meqn + m) * L + S.at(j)];
                fp[P(i, j, m)] = fp[P(i, j, m)] + w.gaddp[(0 * meqn + m) * L + S.at(j)];
                fm[P(i + 1, j, m)] = fm[P(i + 1, j, m)] + w.gaddm[(1 * meqn + m) * L + S.at(j)];
                fp[P(i + 1, j, m)] = fp[P(i + 1, j, m)] + w.gaddp[(1 * meqn + m) * L + S.at(j)];
            }
    }
    // conservative update (clawpack46_step2_wrap.f:106-125)
    for (int m = 0; m < meqn; ++m)
        for (int i = upd_lo; i <= updx_hi; ++i)
            for (int j = upd_lo; j <= updy_hi; ++j) {
                const double df = fm[P(i + 1, j, m)] - fp[P(i, j, m)];
                const double dg = gm[P(i, j + 1, m)] - gp[P(i, j, m)];
                if (!capa)
                    q[P(i, j, m)] = q[P(i, j, m)] - dtdx * df - dtdy * dg;
                else
                    q[P(i, j, m)] = q[P(i, j, m)] - (dtdx * df + dtdy * dg) / aux[P(i, j, mp.mcapa - 1)];
            }
    if (keep) {
        keep->fm = std::move(fm);
        keep->fp = std::move(fp);
        keep->gm = std::move(gm);
        keep->gp = std::move(gp);
    }
    return cflgrid;
}

void rpn2_cons_update_swe(int meqn, int idir, const double* q, double grav, double* flux) {
    (void)meqn;
    // mu, mv: normal and tangential momentum (1-based 2, 3 for idir 0)
    const int mu = (idir == 0) ? 1 : 2;
    const int mv = (idir == 0) ? 2 : 1;
    const double hun = q[mu], hut = q[mv], h = q[0];
    const double un = hun / h;
    flux[0] = hun;
    flux[mu] = (hun * hun) / h + (0.5 * grav) * (h * h);  // hun**2/h + 0.5*grav*h**2
    flux[mv] = un * hut;
}

namespace {

// radialdam/fdisc.f without a mapping: r^2 - r0^2 (kind 0); periodic/fdisc.f:
// sqrt(x*x + y*y) - r0 about (x0, y0) (kind 1)
struct Disc {
    double x0, y0, r0;
    int kind = 0;
    double fdisc(double x, double y) const {
        const double r2 = (x - x0) * (x - x0) + (y - y0) * (y - y0);
        return kind == 0 ? r2 - r0 * r0 : std::sqrt(r2) - r0;
    }
};

// cellave2.f zeroin: Brent's root finder as the reference states it (netlib
// zeroin), including its step "b = b - xm" where the published algorithm has
// b - tol1, and eps found by halving until 1 + eps == 1.
double zeroin(const Disc& dsc, double xc0, double yc0, double xc1, double yc1, double ax, double bx, double tol) {
    auto f = [&](double sv) {  // fss
        const double x = xc0 + sv * (xc1 - xc0);
        const double y = yc0 + sv * (yc1 - yc0);
        return dsc.fdisc(x, y);
    };
    double eps = 1.0, tol1;
    do {
        eps = eps / 2.0;
        tol1 = 1.0 + eps;
    } while (tol1 > 1.0);
    double a = ax, b = bx, fa = f(a), fb = f(b);
    double c, fc, d, e, xm, sv, p, qq, r;
    goto L20;
L20:
    c = a;
    fc = fa;
    d = b - a;
    e = d;
L30:
    if (std::fabs(fc) >= std::fabs(fb)) goto L40;
    a = b;
    b = c;
    c = a;
    fa = fb;
    fb = fc;
    fc = fa;
L40:
    tol1 = (2.0 * eps) * std::fabs(b) + 0.5 * tol;
    xm = 0.5 * (c - b);
    if (std::fabs(xm) <= tol1) goto L90;
    if (fb == 0.0) goto L90;
    if (std::fabs(e) < tol1) goto L70;
    if (std::fabs(fa) <= std::fabs(fb)) goto L70;
    if (a != c) goto L50;
    sv = fb / fa;
    p = (2.0 * xm) * sv;
    qq = 1.0 - sv;
    goto L60;
L50:
    qq = fa / fc;
    r = fb / fc;
    sv = fb / fa;
    p = sv * (((2.0 * xm) * qq) * (qq - r) - (b - a) * (r - 1.0));
    qq = ((qq - 1.0) * (r - 1.0)) * (sv - 1.0);
L60:
    if (p > 0.0) qq = -qq;
    p = std::fabs(p);
    if ((2.0 * p) >= ((3.0 * xm) * qq - std::fabs(tol1 * qq))) goto L70;
    if (p >= std::fabs((0.5 * e) * qq)) goto L70;
    e = d;
    d = p / qq;
    goto L80;
L70:
    d = xm;
    e = d;
L80:
    a = b;
    fa = fb;
    if (std::fabs(d) > tol1) b = b + d;
    if (std::fabs(d) <= tol1) {
        if (xm >= 0) b = b + tol1;
        else b = b - xm;
    }
    fb = f(b);
    if ((fb * (fc / std::fabs(fc))) > 0.0) goto L20;
    goto L30;
L90:
    return b;
}

// cellave2.f: fraction of the cell [xlow, xlow+dx] x [ylow, ylow+dy] where fdisc < 0
double cellave2(const Disc& dsc, double xlow, double ylow, double dx, double dy) {
    double xx[5], yy[5], x[10], y[10];
    bool fl[5];
    xx[0] = xlow; xx[1] = xlow; xx[2] = xlow + dx; xx[3] = xlow + dx; xx[4] = xx[0];
    yy[0] = ylow; yy[1] = ylow + dy; yy[2] = ylow + dy; yy[3] = ylow; yy[4] = yy[0];
    bool alll = true, allr = true;
    for (int i = 0; i < 4; ++i) {
        fl[i] = dsc.fdisc(xx[i], yy[i]) < 0.0;
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
            const double ss = zeroin(dsc, xx[i], yy[i], xx[i + 1], yy[i + 1], 0.0, 1.0, 1e-14);
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

}  // namespace

void qinit_radialdam_cellave(int mx, int my, int mbc, double xlower, double ylower, double dx, double dy,
                             double x0, double y0, double r0, double hin, double hout, double* q) {
    const PatchIdx P(mx, my, mbc);
    const Disc dsc{x0, y0, r0};
    for (int i = 1 - mbc; i <= mx + mbc; ++i) {
        const double xlow = xlower + (i - 1.0) * dx;
        for (int j = 1 - mbc; j <= my + mbc; ++j) {
            const double ylow = ylower + (j - 1.0) * dy;
            const double win = cellave2(dsc, xlow, ylow, dx, dy);
            q[P(i, j, 0)] = hin * win + hout * (1.0 - win);
            q[P(i, j, 1)] = 0.0;
            q[P(i, j, 2)] = 0.0;
        }
    }
}

void setaux_velocity(int mx, int my, int mbc, int maux, double uvel, double vvel, double* aux) {
    const PatchIdx P(mx, my, mbc);
    for (int i = 1 - mbc; i <= mx + mbc; ++i)
        for (int j = 1 - mbc; j <= my + mbc; ++j) {
            aux[P(i, j, 0)] = uvel;
            aux[P(i, j, 1)] = vvel;
            for (int k = 2; k < maux; ++k) aux[P(i, j, k)] = 0.0;  // not set by the reference (unused)
        }
}

namespace {

// filament/psi.f: psi = (4/3) r**3 (r**3 as r*r*r), r = sqrt((x-1)**2 + (y-1)**2)
double psi_filament(double x, double y) {
    const double r = std::sqrt((x - 1.0) * (x - 1.0) + (y - 1.0) * (y - 1.0));
    return (4.0 / 3.0) * (r * r * r);
}

// fclaw2d_metric_default_fort.f90 get_area_approx: |T_xi x T_eta| of the
// bilinear cell at its centre; corners q[icell][jcell] = (x, y), z = 0
double area_approx(const double q[2][2][2]) {
    double a01[3], a10[3], a11[3], txi[3], teta[3];
    for (int m = 0; m < 3; ++m) {
        const double c00 = m < 2 ? q[0][0][m] : 0.0, c10 = m < 2 ? q[1][0][m] : 0.0;
        const double c01 = m < 2 ? q[0][1][m] : 0.0, c11 = m < 2 ? q[1][1][m] : 0.0;
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
    return std::sqrt(w1 * w1 + w2 * w2 + w3 * w3);
}

}  // namespace

void setaux_filament(int mx, int my, int mbc, double xlower, double ylower, double dx, double dy, double kmod,
                     double* aux) {
    const PatchIdx P(mx, my, mbc);
    const double dxdy = dx * dy;
    auto nx = [&](int i) { return xlower + (i - 1) * dx; };
    auto ny = [&](int j) { return ylower + (j - 1) * dy; };
    for (int i = 1 - mbc; i <= mx + mbc; ++i)
        for (int j = 1 - mbc; j <= my + mbc; ++j) {
            double q[2][2][2];
            for (int ic = 0; ic < 2; ++ic)
                for (int jc = 0; jc < 2; ++jc) {
                    q[ic][jc][0] = nx(i) + ic * dx;  // xe + icell*dx
                    q[ic][jc][1] = ny(j) + jc * dy;
                }
            aux[P(i, j, 0)] = area_approx(q) / dxdy;
            if (kmod != 0.0)
                aux[P(i, j, 0)] = aux[P(i, j, 0)] * (1.0 + kmod * ((xlower + (i - 0.5) * dx) * (ylower + (j - 0.5) * dy)));
        }
    for (int i = 1 - mbc; i <= mx + mbc; ++i)
        for (int j = 1 - mbc; j <= my + mbc; ++j) {
            aux[P(i, j, 1)] = (psi_filament(nx(i), ny(j + 1)) - psi_filament(nx(i), ny(j))) / dy;
            aux[P(i, j, 2)] = -((psi_filament(nx(i + 1), ny(j)) - psi_filament(nx(i), ny(j))) / dx);
        }
}

void qinit_disc_fraction(int mx, int my, int mbc, int meqn, double xlower, double ylower, double dx, double dy,
                         double x0, double y0, double r0, double* q) {
    const PatchIdx P(mx, my, mbc);
    Disc dsc{x0, y0, r0};
    dsc.kind = 1;
    for (int m = 0; m < meqn; ++m)
        for (int i = 1 - mbc; i <= mx + mbc; ++i) {
            const double xlow = xlower + (i - 1.0) * dx;
            for (int j = 1 - mbc; j <= my + mbc; ++j) {
                const double ylow = ylower + (j - 1.0) * dy;
                q[P(i, j, 0)] = cellave2(dsc, xlow, ylow, dx, dy);  // qinit.f writes q(i,j,1) for every mq
            }
        }
}

void setaux_bathy(int mx, int my, int mbc, double xlower, double ylower, double dx, double dy, double* aux) {
    const PatchIdx P(mx, my, mbc);
    for (int j = 1 - mbc; j <= my + mbc; ++j)
        for (int i = 1 - mbc; i <= mx + mbc; ++i) {
            const double xc = xlower + (i - 0.5) * dx, yc = ylower + (j - 0.5) * dy;
            aux[P(i, j, 0)] = -1.0 + 0.8 * std::exp(-((xc - 0.5) * (xc - 0.5) + (yc - 0.5) * (yc - 0.5)) / 0.02);
        }
}

void qinit_bathy(int mx, int my, int mbc, double xlower, double ylower, double dx, double dy, const double* p,
                 double* q) {
    const PatchIdx P(mx, my, mbc);
    std::vector<double> b((size_t)P.size(1));
    setaux_bathy(mx, my, mbc, xlower, ylower, dx, dy, b.data());
    for (int j = 1 - mbc; j <= my + mbc; ++j)
        for (int i = 1 - mbc; i <= mx + mbc; ++i) {
            const double xc = xlower + (i - 0.5) * dx, yc = ylower + (j - 0.5) * dy;
            const double r2 = (xc - p[0]) * (xc - p[0]) + (yc - p[1]) * (yc - p[1]);
            const double eta = p[2] * std::exp(-r2 / (p[3] * p[3]));
            q[P(i, j, 0)] = std::max(0.0, eta - b[P(i, j, 0)]);
            q[P(i, j, 1)] = 0.0;
            q[P(i, j, 2)] = 0.0;
        }
}

void b4step2_swirl(int mx, int my, int mbc, int maux, double xlower, double ylower, double dx,
                   double dy, double t, double dt, double tperiod, double* aux) {
    (void)maux;
    const PatchIdx P(mx, my, mbc);
    if (tperiod == 0.0) return;
    const double pi = 4.0 * std::atan(1.0);
    const double pi2 = 2.0 * pi;
    // swirl/psi.f
    auto psi = [&](double xp, double yp) {
        const double sx = std::sin(pi * xp), sy = std::sin(pi * yp);
        return ((sx * sx) * (sy * sy)) / pi;
    };
    const double vt = std::cos(pi2 * (t + dt / 2.0) / tperiod);
    const double vty = vt / dy;
    const double vtx = vt / dx;
    for (int j = 1 - mbc; j <= my + mbc; ++j) {
        const double yll = ylower + (j - 1) * dy;
        for (int i = 1 - mbc; i <= mx + mbc; ++i) {
            const double xll = xlower + (i - 1) * dx;
            const double pij = psi(xll, yll);
            aux[P(i, j, 0)] = vty * (psi(xll, yll + dy) - pij);
            aux[P(i, j, 1)] = -vtx * (psi(xll + dx, yll) - pij);
        }
    }
}

void qinit_swirl(int mx, int my, int mbc, int meqn, double xlower, double ylower, double dx,
                 double dy, double* q) {
    (void)ylower; (void)dy;
    const PatchIdx P(mx, my, mbc);
    for (int mq = 0; mq < meqn; ++mq)
        for (int i = 1 - mbc; i <= mx + mbc; ++i) {
            const double xc = xlower + (i - 0.5) * dx;
            for (int j = 1 - mbc; j <= my + mbc; ++j) q[P(i, j, mq)] = (xc < 0.5) ? 1.0 : 0.0;
        }
}

void qinit_radialdam(int mx, int my, int mbc, double xlower, double ylower, double dx, double dy,
                     double x0, double y0, double r0, double hin, double hout, double* q) {
    const PatchIdx P(mx, my, mbc);
    for (int i = 1 - mbc; i <= mx + mbc; ++i) {
        const double xc = xlower + (i - 0.5) * dx;
        for (int j = 1 - mbc; j <= my + mbc; ++j) {
            const double yc = ylower + (j - 0.5) * dy;
            const double r = std::sqrt((xc - x0) * (xc - x0) + (yc - y0) * (yc - y0));
            q[P(i, j, 0)] = (r < r0) ? hin : hout;
            q[P(i, j, 1)] = 0.0;
            q[P(i, j, 2)] = 0.0;
        }
    }
}

void src2_axisymmetric(int mx, int my, int mbc, int meqn, double ylower, double dy, double gamma1, double dt,
                       double* q) {
    const PatchIdx P(mx, my, mbc);
    const double dt2 = dt / 2.0;
    const double ndim1 = 1.0;  // (ndim-1) with ndim = 2, converted to double
    for (int i = 1; i <= mx; ++i) {
        for (int j = 1; j <= my; ++j) {
            const double rad = ylower + (j - 0.5) * dy;
            double rho = q[P(i, j, 0)];
            double u = q[P(i, j, 1)] / q[P(i, j, 0)];
            double v = q[P(i, j, 2)] / q[P(i, j, 0)];
            double press = gamma1 * (q[P(i, j, 3)] - 0.5 * rho * (u * u + v * v));
            // Fortran a*b/c*d associates as ((a*b)/c)*d
            const double qs1 = q[P(i, j, 0)] - dt2 * ndim1 / rad * q[P(i, j, 2)];
            const double qs2 = q[P(i, j, 1)] - dt2 * ndim1 / rad * (rho * u * v);
            const double qs3 = q[P(i, j, 2)] - dt2 * ndim1 / rad * (rho * v * v);
            const double qs4 = q[P(i, j, 3)] - dt2 * ndim1 / rad * v * (q[P(i, j, 3)] + press);
            rho = qs1;
            u = qs2 / qs1;
            v = qs3 / qs1;
            press = gamma1 * (qs4 - 0.5 * rho * (u * u + v * v));
            q[P(i, j, 0)] = q[P(i, j, 0)] - dt * ndim1 / rad * qs3;
            q[P(i, j, 1)] = q[P(i, j, 1)] - dt * ndim1 / rad * (rho * u * v);
            q[P(i, j, 2)] = q[P(i, j, 2)] - dt * ndim1 / rad * (rho * v * v);
            q[P(i, j, 3)] = q[P(i, j, 3)] - dt * ndim1 / rad * v * (qs4 + press);
        }
    }
    (void)meqn;
}

void qinit_hump(int mx, int my, int mbc, double xlower, double ylower, double dx, double dy, double x0,
                double y0, double base, double coef, double* q) {
    const PatchIdx P(mx, my, mbc);
    for (int i = 1 - mbc; i <= mx + mbc; ++i) {
        const double xc = xlower + (i - 0.5) * dx;
        for (int j = 1 - mbc; j <= my + mbc; ++j) {
            const double yc = ylower + (j - 0.5) * dy;
            const double r2 = (xc - x0) * (xc - x0) + (yc - y0) * (yc - y0);
            q[P(i, j, 0)] = base + std::exp(-(coef * r2));  // 0.1d0 + exp(-200.d0*r2)
            q[P(i, j, 1)] = 0.0;
            q[P(i, j, 2)] = 0.0;
        }
    }
}

void qinit_quadrants(int mx, int my, int mbc, double xlower, double ylower, double dx, double dy,
                     double gamma1, const double* rpr, const double* rpu, const double* rpv,
                     const double* rpp, double xs, double ys, double* q) {
    const PatchIdx P(mx, my, mbc);
    for (int i = 1 - mbc; i <= mx + mbc; ++i) {
        const double xcell = xlower + (i - 0.5) * dx;
        for (int j = 1 - mbc; j <= my + mbc; ++j) {
            const double ycell = ylower + (j - 0.5) * dy;
            int iq = 0;
            if (xcell >= xs && ycell >= ys) iq = 0;
            if (xcell < xs && ycell >= ys) iq = 1;
            if (xcell < xs && ycell < ys) iq = 2;
            if (xcell >= xs && ycell < ys) iq = 3;
            q[P(i, j, 0)] = rpr[iq];
            q[P(i, j, 1)] = rpr[iq] * rpu[iq];
            q[P(i, j, 2)] = rpr[iq] * rpv[iq];
            q[P(i, j, 3)] = rpp[iq] / gamma1 + 0.5 * rpr[iq] * (rpu[iq] * rpu[iq] + rpv[iq] * rpv[iq]);
        }
    }
}

void bc2_default(int mx, int my, int mbc, int meqn, double* q, const int mthbc[4]) {
    const PatchIdx P(mx, my, mbc);
    auto bad = [](int k) {
        return k == 0 || k == 2;  // user BC without a routine, or periodic: an error in bc2
    };
    for (int k = 0; k < 4; ++k)
        if (bad(mthbc[k])) throw std::runtime_error("bc2_default: mthbc 0 or 2 not supported");
    // left
    if (mthbc[0] == 1) {
        for (int m = 0; m < meqn; ++m)
            for (int ibc = 1; ibc <= mbc; ++ibc)
                for (int j = 1 - mbc; j <= my + mbc; ++j) q[P(1 - ibc, j, m)] = q[P(1, j, m)];
    } else if (mthbc[0] == 3) {
        for (int m = 0; m < meqn; ++m)
            for (int ibc = 1; ibc <= mbc; ++ibc)
                for (int j = 1 - mbc; j <= my + mbc; ++j) q[P(1 - ibc, j, m)] = q[P(ibc, j, m)];
        for (int ibc = 1; ibc <= mbc; ++ibc)
            for (int j = 1 - mbc; j <= my + mbc; ++j) q[P(1 - ibc, j, 1)] = -q[P(ibc, j, 1)];
    }
    // right
    if (mthbc[1] == 1) {
        for (int m = 0; m < meqn; ++m)
            for (int ibc = 1; ibc <= mbc; ++ibc)
                for (int j = 1 - mbc; j <= my + mbc; ++j) q[P(mx + ibc, j, m)] = q[P(mx, j, m)];
    } else if (mthbc[1] == 3) {
        for (int m = 0; m < meqn; ++m)
            for (int ibc = 1; ibc <= mbc; ++ibc)
                for (int j = 1 - mbc; j <= my + mbc; ++j)
                    q[P(mx + ibc, j, m)] = q[P(mx + 1 - ibc, j, m)];
        for (int ibc = 1; ibc <= mbc; ++ibc)
            for (int j = 1 - mbc; j <= my + mbc; ++j)
                q[P(mx + ibc, j, 1)] = -q[P(mx + 1 - ibc, j, 1)];
    }
    // bottom
    if (mthbc[2] == 1) {
        for (int m = 0; m < meqn; ++m)
            for (int jbc = 1; jbc <= mbc; ++jbc)
                for (int i = 1 - mbc; i <= mx + mbc; ++i) q[P(i, 1 - jbc, m)] = q[P(i, 1, m)];
    } else if (mthbc[2] == 3) {
        for (int m = 0; m < meqn; ++m)
            for (int jbc = 1; jbc <= mbc; ++jbc)
                for (int i = 1 - mbc; i <= mx + mbc; ++i) q[P(i, 1 - jbc, m)] = q[P(i, jbc, m)];
        for (int jbc = 1; jbc <= mbc; ++jbc)
            for (int i = 1 - mbc; i <= mx + mbc; ++i) q[P(i, 1 - jbc, 2)] = -q[P(i, jbc, 2)];
    }
    // top
    if (mthbc[3] == 1) {
        for (int m = 0; m < meqn; ++m)
            for (int jbc = 1; jbc <= mbc; ++jbc)
                for (int i = 1 - mbc; i <= mx + mbc; ++i) q[P(i, my + jbc, m)] = q[P(i, my, m)];
    } else if (mthbc[3] == 3) {
        for (int m = 0; m < meqn; ++m)
            for (int jbc = 1; jbc <= mbc; ++jbc)
                for (int i = 1 - mbc; i <= mx + mbc; ++i)
                    q[P(i, my + jbc, m)] = q[P(i, my + 1 - jbc, m)];
        for (int jbc = 1; jbc <= mbc; ++jbc)
            for (int i = 1 - mbc; i <= mx + mbc; ++i)
                q[P(i, my + jbc, 2)] = -q[P(i, my + 1 - jbc, 2)];
    }
}

}  // namespace orc
