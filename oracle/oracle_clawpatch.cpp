// ORACLE -- test infrastructure only (see oracle_patch.hpp).
#include "oracle_clawpatch.hpp"

#include <stdexcept>

namespace orc {

void Transform::face(int i1, int j1, int& i2, int& j2) const {
    const double iwidth = (double)(1 << self.level);
    i2 = i1 + (int)((self.xlower - nbr.xlower) * iwidth * (double)mx);
    j2 = j1 + (int)((self.ylower - nbr.ylower) * iwidth * (double)my);
}

void Transform::face_half(int i1, int j1, int i2[4], int j2[4]) const {
    const int based = 1;
    const double owidth = (double)(1 << nbr.level);
    const int di = based + (int)((self.xlower - nbr.xlower) * owidth * (double)mx + 2. * (i1 - based));
    const int dj = based + (int)((self.ylower - nbr.ylower) * owidth * (double)my + 2. * (j1 - based));
    for (int ky = 0; ky < 2; ++ky)
        for (int kx = 0; kx < 2; ++kx) {
            i2[2 * ky + kx] = di + kx;
            j2[2 * ky + kx] = dj + ky;
        }
}

void Transform::corner(int i1, int j1, int& i2, int& j2) const {
    const double rx = (double)(1 << self.level) * (double)mx;
    const double ry = (double)(1 << self.level) * (double)my;
    i2 = i1 + (int)((self.xlower - nbr.xlower + 0.) * rx);
    j2 = j1 + (int)((self.ylower - nbr.ylower + 0.) * ry);
}

void Transform::corner_half(int i1, int j1, int i2[4], int j2[4]) const {
    const int based = 1;
    const double rx = (double)(1 << nbr.level) * (double)mx;
    const double ry = (double)(1 << nbr.level) * (double)my;
    const int di = based + (int)((self.xlower - nbr.xlower + 0.) * rx + 2. * (i1 - based));
    const int dj = based + (int)((self.ylower - nbr.ylower + 0.) * ry + 2. * (j1 - based));
    for (int kt = 0; kt < 2; ++kt)
        for (int kn = 0; kn < 2; ++kn) {
            i2[2 * kt + kn] = di + kn;
            j2[2 * kt + kn] = dj + kt;
        }
}

namespace {

// fclaw2d_clawpatch_utils.f:11-66 with mth = 5 (AMRClaw slopes).  Fortran
// SIGN(1.d0, x) follows the sign bit of x, as copysign does.
inline double compute_slopes(double sl, double sr) {
    const double sc = (sl + sr) / 2.0;
    const double a = std::fabs(sl), b = std::fabs(sr), c = std::fabs(sc);
    double m = 2 * a;
    if (2 * b < m) m = 2 * b;
    if (c < m) m = c;
    return m * dmax(0.0, std::copysign(1.0, sl * sr)) * std::copysign(1.0, sc);
}

inline bool is_valid_interp(int i, int j, int mx, int my, int mbc) {
    return (1 - mbc <= i && i <= mx + mbc) && (1 - mbc <= j && j <= my + mbc);
}
inline bool is_valid_average(int i, int j, int mx, int my) {
    return (1 <= i && i <= mx) && (1 <= j && j <= my);
}

}  // namespace

// fclaw2d_clawpatch_utils.f:76-169: recover A, F of T(ic,jc) = A(ic,jc) + F.
void build_transform_half(const Transform& t, int a[2][2], int f[2]) {
    int mi[4], mj[4];
    t.face_half(0, 0, mi, mj);
    f[0] = mi[0]; f[1] = mj[0];
    t.face_half(1, 0, mi, mj);
    a[0][0] = mi[0] - f[0]; a[1][0] = mj[0] - f[1];
    t.face_half(0, 1, mi, mj);
    a[0][1] = mi[0] - f[0]; a[1][1] = mj[0] - f[1];
}
void build_transform_same(const Transform& t, int a[2][2], int f[2]) {
    int mi, mj;
    t.face(0, 0, mi, mj);
    f[0] = mi; f[1] = mj;
    t.face(1, 0, mi, mj);
    a[0][0] = mi - f[0]; a[1][0] = mj - f[1];
    t.face(0, 1, mi, mj);
    a[0][1] = mi - f[0]; a[1][1] = mj - f[1];
}


void copy_face(int mx, int my, int mbc, int meqn, double* qthis, const double* qnbr, int iface,
               const Transform& t) {
    const PatchIdx P(mx, my, mbc);
    int a[2][2], f[2];
    build_transform_same(t, a, f);
    auto put = [&](int mq, int i1, int j1) {
        const int i2 = a[0][0] * i1 + a[0][1] * j1 + f[0];
        const int j2 = a[1][0] * i1 + a[1][1] * j1 + f[1];
        qthis[P(i1, j1, mq)] = qnbr[P(i2, j2, mq)];
    };
    for (int mq = 0; mq < meqn; ++mq) {
        if (iface == 0) {
            for (int j1 = 1; j1 <= my; ++j1) for (int i1 = 1 - mbc; i1 <= 0; ++i1) put(mq, i1, j1);
        } else if (iface == 1) {
            for (int j1 = 1; j1 <= my; ++j1) for (int i1 = mx + 1; i1 <= mx + mbc; ++i1) put(mq, i1, j1);
        } else if (iface == 2) {
            for (int j1 = 1 - mbc; j1 <= 0; ++j1) for (int i1 = 1; i1 <= mx; ++i1) put(mq, i1, j1);
        } else if (iface == 3) {
            for (int j1 = my + 1; j1 <= my + mbc; ++j1) for (int i1 = 1; i1 <= mx; ++i1) put(mq, i1, j1);
        }
    }
}

void copy_corner(int mx, int my, int mbc, int meqn, double* qthis, const double* qnbr, int icorner,
                 const Transform& t) {
    const PatchIdx P(mx, my, mbc);
    for (int mq = 0; mq < meqn; ++mq)
        for (int ibc = 1; ibc <= mbc; ++ibc)
            for (int jbc = 1; jbc <= mbc; ++jbc) {
                int i1, j1;
                if (icorner == 0) { i1 = 1 - ibc; j1 = 1 - jbc; }
                else if (icorner == 1) { i1 = mx + ibc; j1 = 1 - jbc; }
                else if (icorner == 2) { i1 = 1 - ibc; j1 = my + jbc; }
                else { i1 = mx + ibc; j1 = my + jbc; }
                int i2, j2;
                t.corner(i1, j1, i2, j2);
                qthis[P(i1, j1, mq)] = qnbr[P(i2, j2, mq)];
            }
}

void average_face(int mx, int my, int mbc, int meqn, double* qcoarse, const double* qfine, int idir,
                  int iface_coarse, const Transform& t) {
    const PatchIdx P(mx, my, mbc);
    const int r2 = 4;
    int i2[4], j2[4];
    auto avg = [&](int mq, int ic, int jc) {
        t.face_half(ic, jc, i2, j2);
        for (int m = 0; m < r2; ++m)
            if (!is_valid_average(i2[m], j2[m], mx, my)) return;
        double sum = 0;
        for (int m = 0; m < r2; ++m) sum = sum + qfine[P(i2[m], j2[m], mq)];
        qcoarse[P(ic, jc, mq)] = sum / (double)r2;
    };
    if (idir == 0) {
        for (int mq = 0; mq < meqn; ++mq)
            for (int jc = 1; jc <= my; ++jc)
                for (int ibc = 1; ibc <= mbc; ++ibc) {
                    const int ic = (iface_coarse == 0) ? 1 - ibc : mx + ibc;
                    avg(mq, ic, jc);
                }
    } else {
        for (int mq = 0; mq < meqn; ++mq)
            for (int jbc = 1; jbc <= mbc; ++jbc)
                for (int ic = 1; ic <= mx; ++ic) {
                    const int jc = (iface_coarse == 2) ? 1 - jbc : my + jbc;
                    avg(mq, ic, jc);
                }
    }
}

void average_corner(int mx, int my, int mbc, int meqn, double* qcoarse, const double* qfine,
                    int icorner_coarse, const Transform& t) {
    const PatchIdx P(mx, my, mbc);
    const int r2 = 4;
    int i2[4], j2[4];
    for (int ibc = 1; ibc <= mbc; ++ibc)
        for (int jbc = 1; jbc <= mbc; ++jbc) {
            int i1, j1;
            if (icorner_coarse == 0) { i1 = 1 - ibc; j1 = 1 - jbc; }
            else if (icorner_coarse == 1) { i1 = mx + ibc; j1 = 1 - jbc; }
            else if (icorner_coarse == 2) { i1 = 1 - ibc; j1 = my + jbc; }
            else { i1 = mx + ibc; j1 = my + jbc; }
            t.corner_half(i1, j1, i2, j2);
            for (int mq = 0; mq < meqn; ++mq) {
                double sum = 0;
                for (int m = 0; m < r2; ++m) sum = sum + qfine[P(i2[m], j2[m], mq)];
                qcoarse[P(i1, j1, mq)] = sum / (double)r2;
            }
        }
}

namespace {
// Shared body of the face and corner interpolation: fill the four fine cells
// under coarse cell (ic, jc).
inline void interp_cell(const PatchIdx& P, int mq, int ic, int jc, const double* qcoarse,
                        double* qfine, int i20, int j20, const int df[2][4], const double* shiftx,
                        const double* shifty) {
    const double qc = qcoarse[P(ic, jc, mq)];
    double sl = (qc - qcoarse[P(ic - 1, jc, mq)]);
    double sr = (qcoarse[P(ic + 1, jc, mq)] - qc);
    const double gradx = compute_slopes(sl, sr);
    sl = (qc - qcoarse[P(ic, jc - 1, mq)]);
    sr = (qcoarse[P(ic, jc + 1, mq)] - qc);
    const double grady = compute_slopes(sl, sr);
    for (int m = 0; m < 4; ++m) {
        const int iff = i20 + df[0][m];
        const int jff = j20 + df[1][m];
        const double value = qc + gradx * shiftx[m] + grady * shifty[m];
        qfine[P(iff, jff, mq)] = value;
    }
}
void interp_setup(const Transform& t, int df[2][4], double shiftx[4], double shifty[4]) {
    int a[2][2], f[2];
    build_transform_half(t, a, f);
    int m = 0;
    for (int jj = 0; jj <= 1; ++jj)
        for (int ii = 0; ii <= 1; ++ii) {
            df[0][m] = (a[0][0] * ii + a[0][1] * jj) / 2;
            df[1][m] = (a[1][0] * ii + a[1][1] * jj) / 2;
            shiftx[m] = (ii - 0.5) / 2.0;
            shifty[m] = (jj - 0.5) / 2.0;
            ++m;
        }
}
}  // namespace

void interpolate_face(int mx, int my, int mbc, int meqn, const double* qcoarse, double* qfine,
                      int idir, int iface_coarse, const Transform& t) {
    const PatchIdx P(mx, my, mbc);
    int df[2][4];
    double shiftx[4], shifty[4];
    interp_setup(t, df, shiftx, shifty);
    int i2[4], j2[4];
    for (int mq = 0; mq < meqn; ++mq) {
        if (idir == 0) {
            for (int ibc = 1; ibc <= mbc / 2; ++ibc) {
                int ic;
                if (iface_coarse == 0) ic = ibc;
                else if (iface_coarse == 1) ic = mx - ibc + 1;
                else throw std::runtime_error("interpolate_face: bad iface_coarse");
                for (int jc = 1; jc <= mx; ++jc) {
                    t.face_half(ic, jc, i2, j2);
                    bool skip = false;
                    for (int m = 0; m < 4; ++m)
                        if (!is_valid_interp(i2[m], j2[m], mx, my, mbc)) { skip = true; break; }
                    if (!skip) interp_cell(P, mq, ic, jc, qcoarse, qfine, i2[0], j2[0], df, shiftx, shifty);
                }
            }
        } else {
            for (int jbc = 1; jbc <= mbc / 2; ++jbc) {
                int jc;
                if (iface_coarse == 2) jc = jbc;
                else if (iface_coarse == 3) jc = my - jbc + 1;
                else throw std::runtime_error("interpolate_face: bad iface_coarse");
                for (int ic = 1; ic <= mx; ++ic) {
                    t.face_half(ic, jc, i2, j2);
                    bool skip = false;
                    for (int m = 0; m < 4; ++m)
                        if (!is_valid_interp(i2[m], j2[m], mx, my, mbc)) { skip = true; break; }
                    if (!skip) interp_cell(P, mq, ic, jc, qcoarse, qfine, i2[0], j2[0], df, shiftx, shifty);
                }
            }
        }
    }
}

void interpolate_corner(int mx, int my, int mbc, int meqn, const double* qcoarse, double* qfine,
                        int icorner_coarse, const Transform& t) {
    const PatchIdx P(mx, my, mbc);
    int df[2][4];
    double shiftx[4], shifty[4];
    interp_setup(t, df, shiftx, shifty);
    int i2[4], j2[4];
    for (int ibc = 1; ibc <= mbc / 2; ++ibc)
        for (int jbc = 1; jbc <= mbc / 2; ++jbc) {
            int ic, jc;
            if (icorner_coarse == 0) { ic = ibc; jc = jbc; }
            else if (icorner_coarse == 1) { ic = mx - ibc + 1; jc = jbc; }
            else if (icorner_coarse == 2) { ic = ibc; jc = my - jbc + 1; }
            else { ic = mx - ibc + 1; jc = my - jbc + 1; }
            t.corner_half(ic, jc, i2, j2);
            for (int mq = 0; mq < meqn; ++mq)
                interp_cell(P, mq, ic, jc, qcoarse, qfine, i2[0], j2[0], df, shiftx, shifty);
        }
}

int timeinterp(int mx, int my, int mbc, int meqn, int psize, const double* qcurr,
               const double* qlast, double* qinterp, double alpha) {
    const PatchIdx P(mx, my, mbc);
    const int mint = mbc;
    int k = 1;
    auto f = [&](int i, int j, int m) {
        qinterp[P(i, j, m)] = qlast[P(i, j, m)] + alpha * (qcurr[P(i, j, m)] - qlast[P(i, j, m)]);
        ++k;
    };
    for (int m = 0; m < meqn; ++m) {
        for (int j = 1; j <= my - mint; ++j) for (int i = 1; i <= mint; ++i) f(i, j, m);
        for (int j = 1; j <= mint; ++j) for (int i = mint + 1; i <= mx; ++i) f(i, j, m);
        for (int j = mint + 1; j <= my; ++j) for (int i = mx - mint + 1; i <= mx; ++i) f(i, j, m);
        for (int j = my - mint + 1; j <= my; ++j) for (int i = 1; i <= mx - mint; ++i) f(i, j, m);
    }
    return (k - 1 != psize) ? 2 : 0;
}

void interpolate2fine(int mx, int my, int mbc, int meqn, const double* qcoarse, double* qfine,
                      int igrid) {
    const PatchIdx P(mx, my, mbc);
    const int rf = 2, refratio = 2;
    const int ig = igrid % refratio;
    const int jg = (igrid - ig) / refratio;
    const int i1 = 1 - ig, i2 = mx / rf + (1 - ig), ic_add = ig * mx / rf;
    const int j1 = 1 - jg, j2 = my / rf + (1 - jg), jc_add = jg * my / rf;
    for (int mq = 0; mq < meqn; ++mq)
        for (int j = j1; j <= j2; ++j)
            for (int i = i1; i <= i2; ++i) {
                const int ic = i + ic_add, jc = j + jc_add;
                const double qc = qcoarse[P(ic, jc, mq)];
                double sl = (qc - qcoarse[P(ic - 1, jc, mq)]);
                double sr = (qcoarse[P(ic + 1, jc, mq)] - qc);
                const double gradx = compute_slopes(sl, sr);
                sl = (qc - qcoarse[P(ic, jc - 1, mq)]);
                sr = (qcoarse[P(ic, jc + 1, mq)] - qc);
                const double grady = compute_slopes(sl, sr);
                for (int ii = 1; ii <= refratio; ++ii)
                    for (int jj = 1; jj <= refratio; ++jj) {
                        const double shiftx = (ii - refratio / 2.0 - 0.5) / refratio;
                        const double shifty = (jj - refratio / 2.0 - 0.5) / refratio;
                        qfine[P((i - 1) * refratio + ii, (j - 1) * refratio + jj, mq)] =
                            qc + shiftx * gradx + shifty * grady;
                    }
            }
}

void average2coarse(int mx, int my, int mbc, int meqn, double* qcoarse, const double* qfine,
                    int igrid) {
    const PatchIdx P(mx, my, mbc);
    const int rf = 2, refratio = 2, r2 = 4;
    const int ig = igrid % refratio;
    const int jg = (igrid - ig) / refratio;
    const int ic_add = ig * mx / rf;
    const int jc_add = jg * mx / rf;  // the reference uses mx here as well
    for (int mq = 0; mq < meqn; ++mq)
        for (int j = 1; j <= my / rf; ++j)
            for (int i = 1; i <= mx / rf; ++i) {
                const int i1 = i + ic_add, j1 = j + jc_add;
                double sum = 0;
                for (int jj = 1; jj <= refratio; ++jj)
                    for (int ii = 1; ii <= refratio; ++ii)
                        sum = sum + qfine[P((i - 1) * refratio + ii, (j - 1) * refratio + jj, mq)];
                qcoarse[P(i1, j1, mq)] = sum / r2;
            }
}

namespace {
// fort_user/fclaw2d_clawpatch_{value,minmax,difference,gradient}_exceeds_th.f90
int exceeds_th(int criteria, int ivar, const double* qval, const double* qmin, const double* qmax,
               const double quad[3][3], double dx, double dy, double threshold, bool is_ghost) {
    (void)ivar;
    switch (criteria) {
        case TAG_VALUE: return (qval[0] > threshold) ? 1 : 0;
        case TAG_MINMAX: return (qmax[0] - qmin[0] > threshold) ? 1 : 0;
        case TAG_DIFFERENCE: {
            if (is_ghost) return -1;
            const double dqx = std::fabs(quad[2][1] - quad[0][1]);
            const double dqy = std::fabs(quad[1][2] - quad[1][0]);
            const double dq = dmax(dqx, dqy);
            return (dq > threshold) ? 1 : 0;
        }
        case TAG_GRADIENT: {
            if (is_ghost) return -1;
            const double dx2 = 2 * dx, dy2 = 2 * dy;
            const double dqx = (quad[2][1] - quad[0][1]) / dx2;
            const double dqy = (quad[1][2] - quad[1][0]) / dy2;
            const double g3 = 0;
            const double ds = std::sqrt(dqx * dqx + dqy * dqy + g3 * g3);
            return (ds > threshold) ? 1 : 0;
        }
        default: throw std::runtime_error("unknown refinement criteria");
    }
}
inline bool is_ghost(int i, int j, int mx, int my) { return i < 1 || j < 1 || i > mx || j > my; }
}  // namespace

// The criterion reads component `ivar` (0-based), so only that component's
// running min/max is kept; the other components never influence a tag.
int tag4refinement(int mx, int my, int mbc, int meqn, double dx, double dy, const double* q,
                   double threshold, int criteria, int ivar) {
    (void)meqn;
    const PatchIdx P(mx, my, mbc);
    double qmin = q[P(1, 1, ivar)], qmax = qmin;
    double quad[3][3] = {{0}};
    for (int j = 1 - mbc; j <= my + mbc; ++j)
        for (int i = 1 - mbc; i <= mx + mbc; ++i) {
            const double qv = q[P(i, j, ivar)];
            qmin = dmin(qmin, qv);
            qmax = dmax(qmax, qv);
            const bool g = is_ghost(i, j, mx, my);
            if (!g)
                for (int jj = -1; jj <= 1; ++jj)
                    for (int ii = -1; ii <= 1; ++ii) quad[ii + 1][jj + 1] = q[P(i + ii, j + jj, ivar)];
            if (exceeds_th(criteria, ivar, &qv, &qmin, &qmax, quad, dx, dy, threshold, g) > 0) return 1;
        }
    return 0;
}

int tag4coarsening(int mx, int my, int mbc, int meqn, double dx, double dy, const double* q[4],
                   double threshold, int criteria, int ivar, int initflag) {
    (void)meqn;
    if (initflag != 0) return 0;
    const PatchIdx P(mx, my, mbc);
    double qmin = q[0][P(1, 1, ivar)], qmax = qmin;
    double quad[3][3] = {{0}};
    for (int k = 0; k < 4; ++k) {
        const double* qk = q[k];
        for (int i = 1 - mbc; i <= mx + mbc; ++i)
            for (int j = 1 - mbc; j <= my + mbc; ++j) {
                const double qv = qk[P(i, j, ivar)];
                qmin = dmin(qv, qmin);
                qmax = dmax(qv, qmax);
                const bool g = is_ghost(i, j, mx, my);
                if (!g)
                    for (int ii = -1; ii <= 1; ++ii)
                        for (int jj = -1; jj <= 1; ++jj) quad[ii + 1][jj + 1] = qk[P(i + ii, j + jj, ivar)];
                if (exceeds_th(criteria, ivar, &qv, &qmin, &qmax, quad, dx, dy, threshold, g) > 0) return 0;
            }
    }
    return 1;
}

void conservation_sum(int mx, int my, int mbc, int meqn, double dx, double dy, const double* q,
                      double* sum, double* c_kahan) {
    const PatchIdx P(mx, my, mbc);
    const double area_ij = dx * dy;
    for (int m = 0; m < meqn; ++m)
        for (int j = 1; j <= my; ++j)
            for (int i = 1; i <= mx; ++i) {
                const double y = q[P(i, j, m)] * area_ij - c_kahan[m];
                const double t = sum[m] + y;
                c_kahan[m] = (t - sum[m]) - y;
                sum[m] = t;
            }
}

}  // namespace orc
