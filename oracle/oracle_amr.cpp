// ORACLE -- test infrastructure only (see oracle_patch.hpp).
#include "oracle_amr.hpp"

#include <algorithm>
#include <functional>
#include <cmath>
#include <stdexcept>

namespace orc {

// --------------------------------------------------------------------------
// Forest: leaves of one p4est tree in Morton order.
// --------------------------------------------------------------------------
uint64_t Forest::morton(int32_t x, int32_t y) {
    uint64_t k = 0;
    for (int b = 0; b < 31; ++b) {
        k |= (uint64_t)((x >> b) & 1) << (2 * b);
        k |= (uint64_t)((y >> b) & 1) << (2 * b + 1);
    }
    return k;
}

void Forest::sort_morton() {
    std::sort(leaves.begin(), leaves.end(), [](const Quad& a, const Quad& b) {
        return morton(a.x, a.y) < morton(b.x, b.y);
    });
    rebuild_index();
}

void Forest::uniform(int level) {
    leaves.clear();
    const int32_t hh = h(level);
    const int n = 1 << level;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) leaves.push_back(Quad{level, i * hh, j * hh});
    sort_morton();
}

void Forest::rebuild_index() {
    index_.clear();
    index_.reserve(leaves.size() * 2);
    for (size_t k = 0; k < leaves.size(); ++k) index_[key(leaves[k].level, leaves[k].x, leaves[k].y)] = (int)k;
}

int Forest::find(int level, int32_t x, int32_t y) const {
    if (level < 0 || level > kMaxLevel) return -1;
    auto it = index_.find(key(level, x, y));
    return it == index_.end() ? -1 : it->second;
}

int Forest::min_level() const {
    int m = kMaxLevel;
    for (auto& q : leaves) m = std::min(m, q.level);
    return m;
}
int Forest::max_level() const {
    int m = 0;
    for (auto& q : leaves) m = std::max(m, q.level);
    return m;
}

bool Forest::wrap(int32_t& x, int32_t& y, int img[2]) const {
    int ix = 0, iy = 0;
    if (x < 0 || x >= kRoot) {
        if (!periodic_x) return false;
        ix = x < 0 ? -1 : 1;
        x -= ix * kRoot;
    }
    if (y < 0 || y >= kRoot) {
        if (!periodic_y) return false;
        iy = y < 0 ? -1 : 1;
        y -= iy * kRoot;
    }
    if (img) { img[0] = ix; img[1] = iy; }
    return true;
}

// fclaw2d_patch_face_neighbors (src/forestclaw2d.c:443-541) on one tree; on a
// periodic brick the faces on the domain boundary connect to the opposite side
// (p4est brick connectivity with periodic_i / periodic_j).
int Forest::face_neighbors(int p, int face, int nbr[2], int* pos, int img[2]) const {
    const Quad& q = leaves[p];
    const int32_t hq = h(q.level);
    int32_t nx = q.x, ny = q.y;
    if (face == 0) nx -= hq;
    else if (face == 1) nx += hq;
    else if (face == 2) ny -= hq;
    else ny += hq;
    nbr[0] = nbr[1] = -1;
    *pos = -1;
    int im[2] = {0, 0};
    if (!wrap(nx, ny, im)) return REL_BOUNDARY;
    if (img) { img[0] = im[0]; img[1] = im[1]; }
    int k = find(q.level, nx, ny);
    if (k >= 0) { nbr[0] = k; return REL_SAMESIZE; }
    if (q.level > 0) {
        const int32_t mask = ~(2 * hq - 1);
        k = find(q.level - 1, nx & mask, ny & mask);
        if (k >= 0) {
            nbr[0] = k;
            const Quad& b = leaves[k];
            *pos = (face < 2) ? (q.y - b.y) / hq : (q.x - b.x) / hq;
            return REL_DOUBLESIZE;
        }
    }
    const int32_t hh = hq / 2;
    int32_t ax, ay, bx, by;
    if (face == 0) { ax = nx + hh; ay = ny; bx = nx + hh; by = ny + hh; }
    else if (face == 1) { ax = nx; ay = ny; bx = nx; by = ny + hh; }
    else if (face == 2) { ax = nx; ay = ny + hh; bx = nx + hh; by = ny + hh; }
    else { ax = nx; ay = ny; bx = nx + hh; by = ny; }
    nbr[0] = find(q.level + 1, ax, ay);
    nbr[1] = find(q.level + 1, bx, by);
    if (nbr[0] < 0 || nbr[1] < 0) throw std::runtime_error("forest is not 2:1 balanced (face)");
    return REL_HALFSIZE;
}

// fclaw2d_patch_corner_neighbors (src/forestclaw2d.c:986-1112) on one tree:
// hanging corners (the corner lies inside a larger neighbour's face) have no
// corner neighbour, as in p4est_mesh's quad_to_corner.
int Forest::corner_neighbor(int p, int corner, int* nbr, int img[2]) const {
    const Quad& q = leaves[p];
    const int32_t hq = h(q.level);
    const int sx = (corner & 1) ? 1 : -1, sy = (corner & 2) ? 1 : -1;
    int32_t cx = q.x + sx * hq, cy = q.y + sy * hq;
    *nbr = -1;
    int im[2] = {0, 0};
    if (!wrap(cx, cy, im)) return 0;
    if (img) { img[0] = im[0]; img[1] = im[1]; }
    int k = find(q.level, cx, cy);
    if (k >= 0) { *nbr = k; return REL_SAMESIZE; }
    if (q.level > 0) {
        const int32_t mask = ~(2 * hq - 1);
        const int32_t bx = cx & mask, by = cy & mask;
        k = find(q.level - 1, bx, by);
        if (k >= 0) {
            const int32_t X = q.x + (sx > 0 ? hq : 0), Y = q.y + (sy > 0 ? hq : 0);
            const int32_t bxa = bx + im[0] * kRoot, bya = by + im[1] * kRoot;  // adjacent image
            const bool is_corner = (X == bxa || X == bxa + 2 * hq) && (Y == bya || Y == bya + 2 * hq);
            if (!is_corner) return 0;  // hanging node
            *nbr = k;
            return REL_DOUBLESIZE;
        }
    }
    const int32_t hh = hq / 2;
    k = find(q.level + 1, cx + (sx < 0 ? hh : 0), cy + (sy < 0 ? hh : 0));
    if (k < 0) throw std::runtime_error("forest is not 2:1 balanced (corner)");
    *nbr = k;
    return REL_HALFSIZE;
}

int Forest::is_first_sibling(int p) const {
    const int n = (int)leaves.size();
    if (p + 4 > n) return 0;
    const Quad& q = leaves[p];
    if (q.level == 0) return 0;
    const int32_t hq = h(q.level);
    if ((q.x & (2 * hq - 1)) != 0 || (q.y & (2 * hq - 1)) != 0) return 0;
    for (int k = 1; k < 4; ++k) {
        const Quad& s = leaves[p + k];
        if (s.level != q.level) return 0;
        if (s.x != q.x + (k & 1) * hq || s.y != q.y + (k >> 1) * hq) return 0;
    }
    return 1;
}

// --------------------------------------------------------------------------
// Solver
// --------------------------------------------------------------------------
// A brick of b x b blocks (b a power of two) is kept as one tree: block level
// l is tree level l + log2(b), and the brick's patch corners
// (xv[block] + xc)/mi (fclaw2d_map_brick.c:75) are the tree's dyadic corners
// exactly; smooth-level and the level bounds move with the offset.
Solver::Solver(const Options& o) : opt(o) {
    int off = 0;
    if (opt.brick < 1 || (opt.brick & (opt.brick - 1)) != 0)
        throw std::runtime_error("brick must be a power of two (mi = mj)");
    while ((1 << off) < opt.brick) ++off;
    opt.minlevel += off;
    opt.maxlevel += off;
    opt.smooth_level += off;
    forest.periodic_x = opt.periodic_x != 0;
    forest.periodic_y = opt.periodic_y != 0;
    if (opt.time_sync && (opt.periodic_x || opt.periodic_y))
        throw std::runtime_error("time-sync is not built for periodic domains");
}

double Solver::xlower(int p) const { return (double)forest.leaves[p].x / (double)Forest::kRoot; }
double Solver::ylower(int p) const { return (double)forest.leaves[p].y / (double)Forest::kRoot; }
// fclaw2d_clawpatch.cpp clawpatch_define (no mapping): physical corner
// ax + (bx-ax)*x of the block coordinate, dx = (xupper - xlower)/mx.
double Solver::xphys(int p) const { return opt.ax + (opt.bx - opt.ax) * xlower(p); }
double Solver::yphys(int p) const { return opt.ay + (opt.by - opt.ay) * ylower(p); }
double Solver::dx(int p) const {
    const double xl = xlower(p);
    const double xu = (double)(forest.leaves[p].x + Forest::h(forest.leaves[p].level)) / (double)Forest::kRoot;
    return ((opt.ax + (opt.bx - opt.ax) * xu) - (opt.ax + (opt.bx - opt.ax) * xl)) / opt.mx;
}
double Solver::dy(int p) const {
    const double yl = ylower(p);
    const double yu = (double)(forest.leaves[p].y + Forest::h(forest.leaves[p].level)) / (double)Forest::kRoot;
    return ((opt.ay + (opt.by - opt.ay) * yu) - (opt.ay + (opt.by - opt.ay) * yl)) / opt.my;
}
PatchGeom Solver::geom(int p) const { return PatchGeom{xlower(p), ylower(p), forest.leaves[p].level}; }
// the periodic image of leaf p adjacent to the patch that found it across a
// face or corner (img from NeighborInfo; block-width shifts are exact)
PatchGeom Solver::geom_img(int p, const int img[2]) const {
    return PatchGeom{xlower(p) + img[0], ylower(p) + img[1], forest.leaves[p].level};
}

std::vector<int> Solver::patches_at_level(int level) const {
    std::vector<int> v;
    for (int p = 0; p < (int)forest.leaves.size(); ++p)
        if (forest.leaves[p].level == level) v.push_back(p);
    return v;
}

double* Solver::q_time_sync(int p, int time_interp) {
    return time_interp ? data[p].qinterp.data() : data[p].q.data();
}

void Solver::build_patch(int p, bool) {
    PatchData& d = data[p];
    d.q.assign(patch_size(), 0.0);
    d.qlast.assign(patch_size(), 0.0);
    d.qinterp.assign(patch_size(), 0.0);
    d.qsave.assign(patch_size(), 0.0);
    d.aux.assign(aux_size(), 0.0);
    // fclaw2d_clawpatch_time_sync_new: zeroed registers on every new patch
    const size_t ny = (size_t)opt.my * opt.meqn, nx = (size_t)opt.mx * opt.meqn;
    for (int k = 0; k < 2; ++k) {
        d.reg.fp[k].assign(ny, 0.0);
        d.reg.fm[k].assign(ny, 0.0);
        d.reg.gp[k].assign(nx, 0.0);
        d.reg.gm[k].assign(nx, 0.0);
        d.reg.ef[k].assign(2 * ny, 0.0);
        d.reg.ef[k + 2].assign(2 * nx, 0.0);
    }
}

void Solver::qinit_patch(int p) {
    const double* pp = opt.pparams;
    double* q = data[p].q.data();
    switch (opt.problem) {
        case PROB_SWIRL:
            qinit_swirl(opt.mx, opt.my, opt.mbc, opt.meqn, xphys(p), yphys(p), dx(p), dy(p), q);
            break;
        case PROB_RADIALDAM:
            qinit_radialdam(opt.mx, opt.my, opt.mbc, xphys(p), yphys(p), dx(p), dy(p), pp[0], pp[1],
                            pp[2], pp[3], pp[4], q);
            break;
        case PROB_RADIALDAM_CELLAVE:
            // pparams: x0, y0, r0, hin, hout
            qinit_radialdam_cellave(opt.mx, opt.my, opt.mbc, xphys(p), yphys(p), dx(p), dy(p), pp[0], pp[1],
                                    pp[2], pp[3], pp[4], q);
            break;
        case PROB_QUADRANTS:
            // pparams: rho[4], u[4], v[4], p[4], xs, ys
            qinit_quadrants(opt.mx, opt.my, opt.mbc, xphys(p), yphys(p), dx(p), dy(p),
                            opt.solver.gamma1, pp + 0, pp + 4, pp + 8, pp + 12, pp[16], pp[17], q);
            break;
        case PROB_PERIODIC_DISC:
        case PROB_FILAMENT:
            // pparams: uvel, vvel (periodic only), x0, y0, r0 (filament/fdisc.f: (0.5, 1), 0.25)
            qinit_disc_fraction(opt.mx, opt.my, opt.mbc, opt.meqn, xphys(p), yphys(p), dx(p), dy(p), pp[2], pp[3],
                                pp[4], q);
            break;
        case PROB_HUMP:
            // pparams: x0, y0, base, coef
            qinit_hump(opt.mx, opt.my, opt.mbc, xphys(p), yphys(p), dx(p), dy(p), pp[0], pp[1], pp[2], pp[3], q);
            break;
        case PROB_BATHY:
            qinit_bathy(opt.mx, opt.my, opt.mbc, xphys(p), yphys(p), dx(p), dy(p), pp, q);
            break;
        default: throw std::runtime_error("unknown problem");
    }
}

// setaux: the bathymetry depends on the cell centres only, so a new patch gets
// it from the formula (no transfer from its parent or children).
void Solver::setaux_patch(int p) {
    if (opt.problem == PROB_BATHY)
        setaux_bathy(opt.mx, opt.my, opt.mbc, xphys(p), yphys(p), dx(p), dy(p), data[p].aux.data());
    if (opt.problem == PROB_PERIODIC_DISC)  // pparams: uvel, vvel
        setaux_velocity(opt.mx, opt.my, opt.mbc, opt.maux, opt.pparams[0], opt.pparams[1], data[p].aux.data());
    if (opt.problem == PROB_FILAMENT)
        setaux_filament(opt.mx, opt.my, opt.mbc, xphys(p), yphys(p), dx(p), dy(p), opt.pparams[0],
                        data[p].aux.data());
}

// clawpack46_update (fc2d_clawpack46.cpp:403-444) for one patch.
double Solver::single_step_patch(int p, double t, double dt) {
    PatchData& d = data[p];
    if (opt.problem == PROB_SWIRL)
        b4step2_swirl(opt.mx, opt.my, opt.mbc, opt.maux, xphys(p), yphys(p), dx(p), dy(p), t, dt,
                      opt.pparams[0], d.aux.data());
    d.qlast = d.q;  // fclaw2d_clawpatch_save_current_step
    if (!opt.time_sync) {
        const double cfl = step2(opt.solver, opt.method, opt.mx, opt.my, opt.mbc, opt.meqn, opt.maux, d.q.data(),
                                 opt.maux > 0 ? d.aux.data() : nullptr, dx(p), dy(p), dt);
        // clawpack46_update: src2 after the step when src_term > 0 (fc2d_clawpack46.cpp:436-440)
        if (opt.src_term == 1)
            src2_axisymmetric(opt.mx, opt.my, opt.mbc, opt.meqn, yphys(p), dy(p), opt.solver.gamma1, dt, d.q.data());
        return cfl;
    }
    // clawpack46_step2 (fc2d_clawpack46.cpp:316-386): fluxes f(q) at the patch
    // edges before the update, boundary fluctuations after it
    time_sync_store_flux(p, dt);
    StepFluxArrays f;
    const double cfl = step2(opt.solver, opt.method, opt.mx, opt.my, opt.mbc, opt.meqn, opt.maux, d.q.data(),
                             opt.maux > 0 ? d.aux.data() : nullptr, dx(p), dy(p), dt, &f);
    time_sync_accumulate(p, dt, f);
    if (opt.src_term == 1)
        src2_axisymmetric(opt.mx, opt.my, opt.mbc, opt.meqn, yphys(p), dy(p), opt.solver.gamma1, dt, d.q.data());
    return cfl;
}

// --------------------------------------------------------------------------
// Conservative time synchronisation
// --------------------------------------------------------------------------

// clawpack46_time_sync.f:37-157 (clawpack46_time_sync_store_flux) with the
// shallow-water rpn2_cons_update; edge lengths dy (x faces) and dx (y faces)
// (clawpatch_time_sync_setup, fclaw2d_clawpatch_utils.f:259-310, no manifold).
void Solver::time_sync_store_flux(int p, double dt) {
    if (opt.solver.kind != SOLVER_SWE_ROE) throw std::runtime_error("time-sync: rpn2_cons for shallow water only");
    // clawpack5_time_sync.f has clawpack46_time_sync.f's arithmetic in the q(m,i,j)
    // layout; the registers take clawpack 5's flux arrays (fc2d_clawpack5.cpp:286-343)
    const int mx = opt.mx, my = opt.my, mbc = opt.mbc, meqn = opt.meqn;
    const PatchIdx P(mx, my, mbc);
    PatchData& d = data[p];
    const double* q = d.q.data();
    const double el_x = dy(p), el_y = dx(p);
    double qv[8], fl[8];
    auto cons = [&](int i, int j, int idir) {
        for (int m = 0; m < meqn; ++m) qv[m] = q[P(i, j, m)];
        rpn2_cons_update_swe(meqn, idir, qv, opt.solver.grav, fl);
    };
    for (int j = 1; j <= my; ++j) {
        for (int k = 0; k <= 1; ++k) {
            cons(1 - k, j, 0);
            for (int m = 0; m < meqn; ++m) {
                double& r = d.reg.ef[0][(j - 1) + my * (m + meqn * k)];
                r = r + (dt * el_x) * fl[m];
            }
        }
        for (int k = 0; k <= 1; ++k) {
            cons(mx + k, j, 0);
            for (int m = 0; m < meqn; ++m) {
                double& r = d.reg.ef[1][(j - 1) + my * (m + meqn * k)];
                r = r + (dt * el_x) * fl[m];
            }
        }
    }
    for (int i = 1; i <= mx; ++i) {
        for (int k = 0; k <= 1; ++k) {
            cons(i, 1 - k, 1);
            for (int m = 0; m < meqn; ++m) {
                double& r = d.reg.ef[2][(i - 1) + mx * (m + meqn * k)];
                r = r + (dt * el_y) * fl[m];
            }
        }
        for (int k = 0; k <= 1; ++k) {
            cons(i, my + k, 1);
            for (int m = 0; m < meqn; ++m) {
                double& r = d.reg.ef[3][(i - 1) + mx * (m + meqn * k)];
                r = r + (dt * el_y) * fl[m];
            }
        }
    }
}

// clawpack46_time_sync.f:163-243 (clawpack46_time_sync_accumulate_waves)
void Solver::time_sync_accumulate(int p, double dt, const StepFluxArrays& f) {
    const int mx = opt.mx, my = opt.my, mbc = opt.mbc, meqn = opt.meqn;
    const PatchIdx P(mx, my, mbc);
    Registers& r = data[p].reg;
    const double dtdy = dt * dy(p), dtdx = dt * dx(p);
    for (int j = 1; j <= my; ++j)
        for (int m = 0; m < meqn; ++m) {
            const int k = (j - 1) + my * m;
            r.fp[0][k] = r.fp[0][k] - dtdy * f.fp[P(1, j, m)];
            r.fm[0][k] = r.fm[0][k] + dtdy * f.fm[P(1, j, m)];
            r.fp[1][k] = r.fp[1][k] - dtdy * f.fp[P(mx + 1, j, m)];
            r.fm[1][k] = r.fm[1][k] + dtdy * f.fm[P(mx + 1, j, m)];
        }
    for (int i = 1; i <= mx; ++i)
        for (int m = 0; m < meqn; ++m) {
            const int k = (i - 1) + mx * m;
            r.gp[0][k] = r.gp[0][k] - dtdx * f.gp[P(i, 1, m)];
            r.gm[0][k] = r.gm[0][k] + dtdx * f.gm[P(i, 1, m)];
            r.gp[1][k] = r.gp[1][k] - dtdx * f.gp[P(i, my + 1, m)];
            r.gm[1][k] = r.gm[1][k] + dtdx * f.gm[P(i, my + 1, m)];
        }
}

namespace {
// clawpack46_time_sync.f fc46_is_valid_correct / fc46_skip_this_grid
bool skip_this_grid(const int i2[4], const int j2[4], int mx, int my) {
    for (int m = 0; m < 4; ++m) {
        const bool iv = 1 <= i2[m] && i2[m] <= mx, jv = 1 <= j2[m] && j2[m] <= my;
        if (!(iv != jv)) return true;
    }
    return false;
}
}  // namespace

// fclaw2d_clawpatch_time_sync_samesize (fclaw2d_clawpatch_conservation.c:410-470)
// -> clawpack46_fort_time_sync_samesize (clawpack46_time_sync.f:528-700):
// half of the mismatch between this patch's registers and its same-size
// neighbour's goes into this patch's edge cells.
void Solver::time_sync_samesize(int p, int iface) {
    const int mx = opt.mx, my = opt.my, mbc = opt.mbc, meqn = opt.meqn;
    const int n = nbrs[p].face_nbr[iface][0];
    const PatchIdx P(mx, my, mbc);
    const Transform t{geom(p), geom(n), mx, my};
    int a[2][2], f[2];
    build_transform_same(t, a, f);
    const Registers& rt = data[p].reg;
    const Registers& rn = data[n].reg;
    std::vector<double> dum((size_t)P.size(meqn), 0.0);
    for (int mq = 0; mq < meqn; ++mq) {
        for (int j = 1; j <= my; ++j) {
            const int k = (j - 1) + my * mq;
            dum[P(0, j, mq)] = rn.fm[0][k];
            dum[P(-1, j, mq)] = rn.ef[0][k + my * meqn];
            dum[P(mx + 1, j, mq)] = rn.fp[1][k];
            dum[P(mx + 2, j, mq)] = rn.ef[1][k + my * meqn];
        }
        for (int i = 1; i <= mx; ++i) {
            const int k = (i - 1) + mx * mq;
            dum[P(i, 0, mq)] = rn.gm[0][k];
            dum[P(i, -1, mq)] = rn.ef[2][k + mx * meqn];
            dum[P(i, my + 1, mq)] = rn.gp[1][k];
            dum[P(i, my + 2, mq)] = rn.ef[3][k + mx * meqn];
        }
    }
    double* q = data[p].q.data();
    const double area = dx(p) * dy(p);
    const int idir = iface / 2;
    int i2, j2;
    if (idir == 0) {
        const int sc = a[0][0] + a[1][0];
        for (int mq = 0; mq < meqn; ++mq)
            for (int j = 1; j <= my; ++j) {
                const int k = (j - 1) + my * mq;
                int i1 = 1;
                double delta;
                if (iface == 0) {
                    t.face(i1, j, i2, j2);
                    const double fpv = dum[P(i2, j2, mq)];
                    t.face(i1 + 1, j, i2, j2);
                    const double ef = (double)sc * dum[P(i2, j2, mq)];
                    delta = (ef - rt.ef[0][k]) - (fpv - rt.fp[0][k]);
                } else {
                    i1 = mx;
                    t.face(i1, j, i2, j2);
                    const double fmv = dum[P(i2, j2, mq)];
                    t.face(i1 - 1, j, i2, j2);
                    const double ef = (double)sc * dum[P(i2, j2, mq)];
                    delta = (rt.ef[1][k] - ef) - (fmv - rt.fm[1][k]);
                }
                q[P(i1, j, mq)] = q[P(i1, j, mq)] + (0.5 * delta) / area;
            }
    } else {
        const int sc = a[0][1] + a[1][1];
        for (int mq = 0; mq < meqn; ++mq)
            for (int i = 1; i <= mx; ++i) {
                const int k = (i - 1) + mx * mq;
                int j1 = 1;
                double delta;
                if (iface == 2) {
                    t.face(i, j1, i2, j2);
                    const double gpv = dum[P(i2, j2, mq)];
                    t.face(i, j1 + 1, i2, j2);
                    const double ef = (double)sc * dum[P(i2, j2, mq)];
                    delta = (ef - rt.ef[2][k]) - (gpv - rt.gp[0][k]);
                } else {
                    j1 = my;
                    t.face(i, j1, i2, j2);
                    const double gmv = dum[P(i2, j2, mq)];
                    t.face(i, j1 - 1, i2, j2);
                    const double ef = (double)sc * dum[P(i2, j2, mq)];
                    delta = (rt.ef[3][k] - ef) - (gmv - rt.gm[1][k]);
                }
                q[P(i, j1, mq)] = q[P(i, j1, mq)] + (0.5 * delta) / area;
            }
    }
}

// fclaw2d_clawpatch_time_sync_f2c (fclaw2d_clawpatch_conservation.c:344-405)
// -> clawpack46_fort_time_sync_f2c (clawpack46_time_sync.f:254-520): the fine
// patch's registers, summed over pairs of fine edge cells, replace the coarse
// patch's along the shared face.
void Solver::time_sync_f2c(int pc, int pf, int iface) {
    const int mx = opt.mx, my = opt.my, mbc = opt.mbc, meqn = opt.meqn;
    const PatchIdx P(mx, my, mbc);
    const int nx2 = mx + 4 * mbc, ny2 = my + 4 * mbc;
    // qfine_dummy(1-2mbc:mx+2mbc, 1-2mbc:my+2mbc, meqn)
    std::vector<double> dum((size_t)nx2 * ny2 * meqn, 0.0);
    auto D = [&](int i, int j, int m) -> double& {
        return dum[((size_t)m * ny2 + (j + 2 * mbc - 1)) * nx2 + (i + 2 * mbc - 1)];
    };
    const Transform t{geom(pc), geom(pf), mx, my};
    int a[2][2], f[2];
    build_transform_half(t, a, f);
    const Registers& rc = data[pc].reg;
    const Registers& rf = data[pf].reg;
    for (int mq = 0; mq < meqn; ++mq) {
        for (int j = 1; j <= my / 2; ++j) {
            const int jj1 = 2 * (j - 1) + 1, jj2 = 2 * (j - 1) + 2;
            const int k1 = (jj1 - 1) + my * mq, k2 = (jj2 - 1) + my * mq;
            double fm = rf.fm[0][k1] + rf.fm[0][k2];
            double ef = rf.ef[0][k1 + my * meqn] + rf.ef[0][k2 + my * meqn];
            for (int jj = jj1; jj <= jj2; ++jj)
                for (int ii = -1; ii <= 0; ++ii) {
                    D(ii, jj, mq) = fm;
                    D(ii - 2, jj, mq) = ef;
                }
            const double fp = rf.fp[1][k1] + rf.fp[1][k2];
            ef = rf.ef[1][k1 + my * meqn] + rf.ef[1][k2 + my * meqn];
            for (int jj = jj1; jj <= jj2; ++jj)
                for (int ii = 1; ii <= 2; ++ii) {
                    D(mx + ii, jj, mq) = fp;
                    D(mx + ii + 2, jj, mq) = ef;
                }
        }
        for (int i = 1; i <= mx / 2; ++i) {
            const int ii1 = 2 * (i - 1) + 1, ii2 = 2 * (i - 1) + 2;
            const int k1 = (ii1 - 1) + mx * mq, k2 = (ii2 - 1) + mx * mq;
            const double gm = rf.gm[0][k1] + rf.gm[0][k2];
            double ef = rf.ef[2][k1 + mx * meqn] + rf.ef[2][k2 + mx * meqn];
            for (int ii = ii1; ii <= ii2; ++ii)
                for (int jj = -1; jj <= 0; ++jj) {
                    D(ii, jj, mq) = gm;
                    D(ii, jj - 2, mq) = ef;
                }
            const double gp = rf.gp[1][k1] + rf.gp[1][k2];
            ef = rf.ef[3][k1 + mx * meqn] + rf.ef[3][k2 + mx * meqn];
            for (int ii = ii1; ii <= ii2; ++ii)
                for (int jj = 1; jj <= 2; ++jj) {
                    D(ii, my + jj, mq) = gp;
                    D(ii, my + jj + 2, mq) = ef;
                }
        }
    }
    double* q = data[pc].q.data();
    const double areac_v = dx(pc) * dy(pc);
    const int idir = iface / 2;
    int i2[4], j2[4];
    if (idir == 0) {
        const int sc = (a[0][0] + a[1][0]) / 2;
        for (int mq = 0; mq < meqn; ++mq)
            for (int jc = 1; jc <= my; ++jc) {
                const int k = (jc - 1) + my * mq;
                int ic = 1;
                double deltac = 0;
                double areac = 1;
                if (iface == 0) {
                    ic = 1;
                    t.face_half(ic, jc, i2, j2);
                    deltac = 0;
                    areac = areac_v;
                    if (!skip_this_grid(i2, j2, mx, my)) {
                        const double fp = D(i2[0], j2[0], mq);
                        t.face_half(ic + 1, jc, i2, j2);
                        const double ef = (double)sc * D(i2[0], j2[0], mq);
                        deltac = (ef - rc.ef[0][k]) - (fp - rc.fp[0][k]);
                    }
                } else if (iface == 1) {
                    ic = mx;
                    t.face_half(ic, jc, i2, j2);
                    deltac = 0;
                    areac = areac_v;
                    if (!skip_this_grid(i2, j2, mx, my)) {
                        const double fm = D(i2[0], j2[0], mq);
                        t.face_half(ic - 1, jc, i2, j2);
                        const double ef = (double)sc * D(i2[0], j2[0], mq);
                        deltac = (rc.ef[1][k] - ef) - (fm - rc.fm[1][k]);
                    }
                }
                q[P(ic, jc, mq)] = q[P(ic, jc, mq)] + deltac / areac;
            }
    } else {
        const int sc = (a[0][1] + a[1][1]) / 2;
        for (int mq = 0; mq < meqn; ++mq)
            for (int ic = 1; ic <= mx; ++ic) {
                const int k = (ic - 1) + mx * mq;
                int jc = 1;
                double deltac = 0;
                double areac = 1;
                if (iface == 2) {
                    jc = 1;
                    t.face_half(ic, jc, i2, j2);
                    deltac = 0;
                    areac = areac_v;
                    if (!skip_this_grid(i2, j2, mx, my)) {
                        const double gp = D(i2[0], j2[0], mq);
                        t.face_half(ic, jc + 1, i2, j2);
                        const double ef = (double)sc * D(i2[0], j2[0], mq);
                        deltac = (ef - rc.ef[2][k]) - (gp - rc.gp[0][k]);
                    }
                } else if (iface == 3) {
                    jc = my;
                    t.face_half(ic, jc, i2, j2);
                    deltac = 0;
                    areac = areac_v;
                    if (!skip_this_grid(i2, j2, mx, my)) {
                        const double gm = D(i2[0], j2[0], mq);
                        t.face_half(ic, jc - 1, i2, j2);
                        const double ef = (double)sc * D(i2[0], j2[0], mq);
                        deltac = (rc.ef[3][k] - ef) - (gm - rc.gm[1][k]);
                    }
                }
                q[P(ic, jc, mq)] = q[P(ic, jc, mq)] + deltac / areac;
            }
    }
}

// fclaw2d_clawpatch_time_sync_reset (fclaw2d_clawpatch_conservation.c:205-270)
void Solver::time_sync_reset(int p, int coarse_level, int mode) {
    const int fine_level = coarse_level + 1;
    const int level = forest.leaves[p].level;
    Registers& r = data[p].reg;
    for (int k = 0; k < 4; ++k) {
        const int rel = nbrs[p].face_rel[k];
        bool reset = false;
        if (mode == 1)  // FCLAW2D_TIME_SYNC_RESET_F2C
            reset = (rel == REL_HALFSIZE && level == coarse_level) || (rel == REL_DOUBLESIZE && level == fine_level);
        else if (mode == 2)  // FCLAW2D_TIME_SYNC_RESET_SAMESIZE
            reset = rel == REL_SAMESIZE && level == coarse_level;
        else  // FCLAW2D_TIME_SYNC_RESET_PHYS
            reset = rel == REL_BOUNDARY;
        if (!reset) continue;
        if (k < 2) {
            std::fill(r.fm[k].begin(), r.fm[k].end(), 0.0);
            std::fill(r.fp[k].begin(), r.fp[k].end(), 0.0);
        } else {
            std::fill(r.gm[k - 2].begin(), r.gm[k - 2].end(), 0.0);
            std::fill(r.gp[k - 2].begin(), r.gp[k - 2].end(), 0.0);
        }
        std::fill(r.ef[k].begin(), r.ef[k].end(), 0.0);
    }
}

// fclaw2d_time_sync (src/fclaw2d_time_sync.c:157-205) -> correct_coarse_cells
// (:115-155): per level from the finest option level down, same-size
// corrections then their register reset, then fine-to-coarse corrections at
// the level's coarse/fine faces and their reset; finally the physical-boundary
// registers of every level are cleared.
void Solver::time_sync(int minlevel, int maxlevel) {
    (void)maxlevel;
    for (int level = opt.maxlevel; level >= minlevel; --level) {
        const std::vector<int> ps = patches_at_level(level);
        for (int p : ps)
            for (int f = 0; f < 4; ++f)
                if (nbrs[p].face_rel[f] == REL_SAMESIZE) time_sync_samesize(p, f);
        for (int p : ps) time_sync_reset(p, level, 2);
        if (level < opt.maxlevel) {
            for (int p : ps)
                for (int f = 0; f < 4; ++f)
                    if (nbrs[p].face_rel[f] == REL_HALFSIZE)
                        for (int ig = 0; ig < 2; ++ig) time_sync_f2c(p, nbrs[p].face_nbr[f][ig], f);
            for (int p : ps) time_sync_reset(p, level, 1);
            for (int p : patches_at_level(level + 1)) time_sync_reset(p, level, 1);
        }
    }
    for (int level = opt.maxlevel; level >= minlevel; --level)
        for (int p : patches_at_level(level)) time_sync_reset(p, level, 3);
}

double Solver::update_single_step(int level, double t, double dt) {
    double maxcfl = 0;
    const std::vector<int> ps = patches_at_level(level);
#ifdef ORC_OPENMP
    // timing build: patches of one level are independent (max is order-free)
#pragma omp parallel for schedule(dynamic, 4) reduction(max : maxcfl)
    for (int k = 0; k < (int)ps.size(); ++k) maxcfl = std::fmax(single_step_patch(ps[k], t, dt), maxcfl);
    count_single_step += (long long)ps.size();
#else
    for (int p : ps) {
        const double cfl = single_step_patch(p, t, dt);
        ++count_single_step;
        maxcfl = std::fmax(cfl, maxcfl);
    }
#endif
    return maxcfl;
}

// cb_set_neighbor_types (fclaw2d_regrid.c:338-393) + fclaw2d_patch_neighbors_set
// (fclaw2d_patch.c:975-1040)
void Solver::set_neighbor_types() {
    nbrs.assign(forest.leaves.size(), NeighborInfo{});
    for (int p = 0; p < (int)forest.leaves.size(); ++p) {
        NeighborInfo& n = nbrs[p];
        for (int f = 0; f < 4; ++f) {
            n.face_img[f][0] = n.face_img[f][1] = 0;
            n.face_rel[f] = forest.face_neighbors(p, f, n.face_nbr[f], &n.face_pos[f], n.face_img[f]);
        }
        for (int c = 0; c < 4; ++c) {
            n.corner_img[c][0] = n.corner_img[c][1] = 0;
            n.corner_rel[c] = forest.corner_neighbor(p, c, &n.corner_nbr[c], n.corner_img[c]);
            n.corner_exists[c] = n.corner_rel[c] != 0;
        }
        n.has_finegrid_neighbors = 0;
        n.on_coarsefine_interface = 0;
        for (int f = 0; f < 4; ++f) {
            if (n.face_rel[f] == REL_HALFSIZE || n.face_rel[f] == REL_DOUBLESIZE) {
                n.on_coarsefine_interface = 1;
                if (n.face_rel[f] == REL_HALFSIZE) n.has_finegrid_neighbors = 1;
            }
        }
        for (int c = 0; c < 4; ++c) {
            if (!n.corner_exists[c]) continue;
            if (n.corner_rel[c] == REL_HALFSIZE || n.corner_rel[c] == REL_DOUBLESIZE) {
                n.on_coarsefine_interface = 1;
                if (n.corner_rel[c] == REL_HALFSIZE) n.has_finegrid_neighbors = 1;
            }
        }
    }
}

// --------------------------------------------------------------------------
// Ghost fill (fclaw2d_ghost_fill.c, face/corner dispatch in
// fclaw2d_face_neighbors.c:195-450 and fclaw2d_corner_neighbors.c:334-535)
// --------------------------------------------------------------------------
void Solver::copy2ghost(int level, int time_interp) {
    const int mx = opt.mx, my = opt.my, mbc = opt.mbc, meqn = opt.meqn;
    const auto ps = patches_at_level(level);
    for (int p : ps) {  // cb_face_fill, FCLAW2D_COPY
        for (int f = 0; f < 4; ++f) {
            if (nbrs[p].face_rel[f] != REL_SAMESIZE) continue;
            const int n = nbrs[p].face_nbr[f][0];
            Transform t{geom(p), geom_img(n, nbrs[p].face_img[f]), mx, my};
            copy_face(mx, my, mbc, meqn, q_time_sync(p, time_interp), q_time_sync(n, time_interp), f, t);
        }
    }
    for (int p : ps) {  // cb_corner_fill, FCLAW2D_COPY
        for (int c = 0; c < 4; ++c) {
            if (!nbrs[p].corner_exists[c] || nbrs[p].corner_rel[c] != REL_SAMESIZE) continue;
            const int n = nbrs[p].corner_nbr[c];
            Transform t{geom(p), geom_img(n, nbrs[p].corner_img[c]), mx, my};
            copy_corner(mx, my, mbc, meqn, q_time_sync(p, time_interp), q_time_sync(n, time_interp), c, t);
        }
    }
}

void Solver::average2ghost(int coarse_level, int time_interp) {
    const int mx = opt.mx, my = opt.my, mbc = opt.mbc, meqn = opt.meqn;
    const auto ps = patches_at_level(coarse_level);
    for (int p : ps) {
        if (!nbrs[p].on_coarsefine_interface) continue;
        for (int f = 0; f < 4; ++f) {
            if (nbrs[p].face_rel[f] != REL_HALFSIZE) continue;
            for (int ig = 0; ig < 2; ++ig) {
                const int n = nbrs[p].face_nbr[f][ig];
                Transform t{geom(p), geom_img(n, nbrs[p].face_img[f]), mx, my};
                average_face(mx, my, mbc, meqn, q_time_sync(p, time_interp), data[n].q.data(), f / 2, f, t);
            }
        }
    }
    for (int p : ps) {
        if (!nbrs[p].on_coarsefine_interface) continue;
        for (int c = 0; c < 4; ++c) {
            if (!nbrs[p].corner_exists[c] || nbrs[p].corner_rel[c] != REL_HALFSIZE) continue;
            const int n = nbrs[p].corner_nbr[c];
            Transform t{geom(p), geom_img(n, nbrs[p].corner_img[c]), mx, my};
            average_corner(mx, my, mbc, meqn, q_time_sync(p, time_interp), data[n].q.data(), c, t);
        }
    }
}

void Solver::interpolate2ghost(int coarse_level, int time_interp) {
    const int mx = opt.mx, my = opt.my, mbc = opt.mbc, meqn = opt.meqn;
    const auto ps = patches_at_level(coarse_level);
    for (int p : ps) {
        if (!nbrs[p].on_coarsefine_interface) continue;
        for (int f = 0; f < 4; ++f) {
            if (nbrs[p].face_rel[f] != REL_HALFSIZE) continue;
            for (int ig = 0; ig < 2; ++ig) {
                const int n = nbrs[p].face_nbr[f][ig];
                Transform t{geom(p), geom_img(n, nbrs[p].face_img[f]), mx, my};
                interpolate_face(mx, my, mbc, meqn, q_time_sync(p, time_interp), data[n].q.data(), f / 2, f, t);
            }
        }
    }
    for (int p : ps) {
        if (!nbrs[p].on_coarsefine_interface) continue;
        for (int c = 0; c < 4; ++c) {
            if (!nbrs[p].corner_exists[c] || nbrs[p].corner_rel[c] != REL_HALFSIZE) continue;
            const int n = nbrs[p].corner_nbr[c];
            Transform t{geom(p), geom_img(n, nbrs[p].corner_img[c]), mx, my};
            interpolate_corner(mx, my, mbc, meqn, q_time_sync(p, time_interp), data[n].q.data(), c, t);
        }
    }
}

// clawpack46_bc2 (fc2d_clawpack46.cpp:92-140) through cb_fclaw2d_physical_set_bc.
void Solver::physical_bc(int p, int time_interp) {
    int mthbc[4];
    for (int f = 0; f < 4; ++f) mthbc[f] = (nbrs[p].face_rel[f] == REL_BOUNDARY) ? opt.mthbc[f] : -1;
    bc2_default(opt.mx, opt.my, opt.mbc, opt.meqn, q_time_sync(p, time_interp), mthbc);
}

void Solver::setphysical(int level, int time_interp) {
    for (int p : patches_at_level(level)) physical_bc(p, time_interp);
}

// fclaw2d_ghost_update_async (fclaw2d_ghost_fill.c:611-831) on one rank: the
// "ghost only" passes touch no patch, the interior-only pass touches them all.
void Solver::ghost_update(int minlevel, int maxlevel, double, int time_interp) {
    const int mincoarse = minlevel, maxcoarse = maxlevel - 1;
    // average_fine2coarse_ghost
    for (int l = maxcoarse; l >= mincoarse; --l) average2ghost(l, 0);
    if (time_interp) average2ghost(mincoarse - 1, 1);
    // copy_samelevel
    for (int l = maxlevel; l >= minlevel; --l) copy2ghost(l, 0);
    if (time_interp) copy2ghost(minlevel - 1, 1);
    // fill_physical_ghost(mincoarse, maxcoarse)
    for (int l = maxcoarse; l >= mincoarse; --l) setphysical(l, 0);
    if (time_interp) setphysical(mincoarse - 1, 1);
    // interpolate_coarse2fine_ghost
    for (int l = maxcoarse; l >= mincoarse; --l) interpolate2ghost(l, 0);
    if (time_interp) interpolate2ghost(mincoarse - 1, 1);
    // fill_physical_ghost(minfine, maxfine)
    const int minfine = mincoarse + 1, maxfine = maxlevel;
    for (int l = maxfine; l >= minfine; --l) setphysical(l, 0);
    if (time_interp) setphysical(minfine - 1, 1);
    // final fill_physical_ghost(minlevel, maxlevel), all patches
    for (int l = maxlevel; l >= minlevel; --l) setphysical(l, 0);
    if (time_interp) setphysical(minlevel - 1, 1);
}

void Solver::timeinterp(int level, double alpha) {
    const int mint = 3 / 2 + 1;  // interp_stencil_width/2 + 1
    const int psize = (opt.mx * opt.my - (opt.mx - 2 * mint) * (opt.my - 2 * mint)) * opt.meqn;
    for (int p : patches_at_level(level)) {
        if (!nbrs[p].has_finegrid_neighbors) continue;
        PatchData& d = data[p];
        const int ierr = orc::timeinterp(opt.mx, opt.my, opt.mbc, opt.meqn, psize, d.q.data(),
                                         d.qlast.data(), d.qinterp.data(), alpha);
        if (ierr != 0) throw std::runtime_error("timeinterp: psize mismatch");
    }
}

// --------------------------------------------------------------------------
// Advance (fclaw2d_advance.c)
// --------------------------------------------------------------------------
namespace {
struct LevelCounter {
    int last_step = 0, step_inc = 0, total_steps = 0;
    double initial_time = 0, current_time = 0, dt_step = 0;
};
}  // namespace

double Solver::advance_all_levels(double t_curr, double dt) {
    const int gmin = forest.min_level(), gmax = forest.max_level();
    std::vector<LevelCounter> ts(opt.maxlevel + 1);
    for (int l = opt.minlevel; l <= opt.maxlevel; ++l) {
        ts[l].last_step = 0;
        ts[l].initial_time = t_curr;
        ts[l].current_time = t_curr;
    }
    if (opt.subcycle) {
        double dt_level = dt;
        int steps_inc = 1 << (gmax - opt.minlevel);
        int total_steps = 1;
        for (int l = opt.minlevel; l <= opt.maxlevel; ++l) {
            ts[l].dt_step = dt_level;
            ts[l].total_steps = total_steps;
            ts[l].step_inc = steps_inc;
            dt_level /= 2;
            steps_inc /= 2;
            total_steps *= 2;
        }
    } else {
        const int rf = 1 << (opt.maxlevel - opt.minlevel);
        for (int l = opt.minlevel; l <= opt.maxlevel; ++l) {
            ts[l].step_inc = 1;
            ts[l].dt_step = dt / rf;
            ts[l].total_steps = rf;
        }
    }
    // advance_level (fclaw2d_advance.c:188-241)
    std::function<double(int, int, double)> advance_level = [&](int level, int curr_fine_step,
                                                                 double maxcfl) -> double {
        const double t_level = ts[level].current_time;
        const double dt_level = ts[level].dt_step;
        const double cfl_step = update_single_step(level, t_level, dt_level);
        maxcfl = std::fmax(maxcfl, cfl_step);
        ts[level].last_step += ts[level].step_inc;
        ts[level].current_time += ts[level].dt_step;
        if (level > gmin) {
            const int last_coarse_step = ts[level - 1].last_step;
            if (last_coarse_step == curr_fine_step) {
                const double c2 = advance_level(level - 1, last_coarse_step, maxcfl);
                maxcfl = std::fmax(maxcfl, c2);
                if (opt.subcycle) {
                    const int coarse_inc = ts[level - 1].step_inc;
                    const int new_curr_step = ts[level].last_step;
                    const double alpha = ((double)(new_curr_step % coarse_inc)) / coarse_inc;
                    timeinterp(level - 1, alpha);
                }
            }
        }
        return maxcfl;
    };
    double maxcfl = 0;
    const int n_fine_steps = ts[gmax].total_steps;
    for (int nf = 0; nf < n_fine_steps; ++nf) {
        const double cfl_step = advance_level(gmax, nf, maxcfl);
        maxcfl = std::fmax(cfl_step, maxcfl);
        const int last_step = ts[gmax].last_step;
        if (last_step < ts[gmax].total_steps) {
            const double sync_time = ts[gmax].current_time;
            if (opt.subcycle) {
                int ti_level = gmax - 1;
                while (last_step % ts[ti_level].step_inc == 0) --ti_level;
                ghost_update(ti_level + 1, gmax, sync_time, 1);
                if (opt.time_sync) time_sync(ti_level + 1, gmax);
            } else {
                ghost_update(gmin, gmax, sync_time, 0);
                if (opt.time_sync) time_sync(gmin, gmax);
            }
        }
    }
    ghost_update(gmin, gmax, ts[gmax].current_time, 0);
    if (opt.time_sync) time_sync(gmin, gmax);
    ++count_amr_advance;
    return maxcfl;
}

// --------------------------------------------------------------------------
// Regrid
// --------------------------------------------------------------------------

// fclaw2d_domain_adapt (fclaw2d_convenience.c:498-680) followed by the
// p4est_wrap_adapt semantics: refine flagged leaves once, coarsen complete
// families whose four leaves are all flagged, then 2:1 balance across faces
// and corners when anything changed.
bool Solver::domain_adapt(std::vector<Quad>& new_leaves) {
    const int n = (int)forest.leaves.size();
    enum { F_REFINE = 1, F_COARSEN = 2 };
    std::vector<int> flags(n, 0);
    auto mark_refine = [&](int p) {
        if (forest.leaves[p].level < Forest::kMaxLevel) { flags[p] |= F_REFINE; flags[p] &= ~F_COARSEN; }
    };
    auto mark_coarsen = [&](int p) {
        flags[p] &= ~F_REFINE;
        if (forest.leaves[p].level > 0) flags[p] |= F_COARSEN;
    };
    if (opt.smooth_refine) {
        for (int p = 0; p < n; ++p) {
            const int level = forest.leaves[p].level;
            int max_tlevel = target_level[p];
            for (int f = 0; max_tlevel <= level && f < 4; ++f) {
                const int rel = nbrs[p].face_rel[f];
                if (rel == REL_SAMESIZE || rel == REL_DOUBLESIZE) {
                    const int q = nbrs[p].face_nbr[f][0];
                    if (forest.leaves[q].level >= opt.smooth_level) max_tlevel = std::max(max_tlevel, target_level[q]);
                } else if (rel == REL_HALFSIZE) {
                    for (int k = 0; k < 2; ++k) {
                        const int q = nbrs[p].face_nbr[f][k];
                        if (forest.leaves[q].level >= opt.smooth_level) max_tlevel = std::max(max_tlevel, target_level[q]);
                    }
                }
            }
            for (int c = 0; max_tlevel <= level && c < 4; ++c) {
                if (!nbrs[p].corner_exists[c]) continue;
                const int q = nbrs[p].corner_nbr[c];
                if (forest.leaves[q].level >= opt.smooth_level) max_tlevel = std::max(max_tlevel, target_level[q]);
            }
            if (max_tlevel < level) mark_coarsen(p);
            else if (max_tlevel > level) mark_refine(p);
        }
    } else {
        for (int p = 0; p < n; ++p) {
            if (target_level[p] > forest.leaves[p].level) mark_refine(p);
            else if (target_level[p] < forest.leaves[p].level) mark_coarsen(p);
        }
    }
    // refine
    bool changed = false;
    std::vector<Quad> after_refine;
    std::vector<int> after_flags;
    for (int p = 0; p < n; ++p) {
        const Quad& q = forest.leaves[p];
        if (flags[p] & F_REFINE) {
            changed = true;
            const int32_t hh = Forest::h(q.level + 1);
            for (int k = 0; k < 4; ++k) {
                after_refine.push_back(Quad{q.level + 1, q.x + (k & 1) * hh, q.y + (k >> 1) * hh});
                after_flags.push_back(flags[p] & ~F_REFINE);
            }
        } else {
            after_refine.push_back(q);
            after_flags.push_back(flags[p]);
        }
    }
    // coarsen complete families
    Forest tmp;
    tmp.leaves = after_refine;
    std::vector<Quad> after_coarsen;
    for (int p = 0; p < (int)after_refine.size();) {
        if (tmp.is_first_sibling(p) && (after_flags[p] & F_COARSEN) && (after_flags[p + 1] & F_COARSEN) &&
            (after_flags[p + 2] & F_COARSEN) && (after_flags[p + 3] & F_COARSEN)) {
            const Quad& q = after_refine[p];
            after_coarsen.push_back(Quad{q.level - 1, q.x, q.y});
            changed = true;
            p += 4;
        } else {
            after_coarsen.push_back(after_refine[p]);
            ++p;
        }
    }
    if (!changed) return false;
    // 2:1 balance across faces and corners (p4est_balance, P4EST_CONNECT_FULL)
    Forest f;
    f.periodic_x = forest.periodic_x;
    f.periodic_y = forest.periodic_y;
    f.leaves = after_coarsen;
    f.rebuild_index();
    for (;;) {
        std::vector<char> split(f.leaves.size(), 0);
        bool any = false;
        for (size_t p = 0; p < f.leaves.size(); ++p) {
            const Quad& q = f.leaves[p];
            if (q.level < 2) continue;
            const int32_t hq = Forest::h(q.level);
            for (int dyi = -1; dyi <= 1; ++dyi)
                for (int dxi = -1; dxi <= 1; ++dxi) {
                    if (dxi == 0 && dyi == 0) continue;
                    int32_t cx = q.x + dxi * hq, cy = q.y + dyi * hq;
                    if (!forest.wrap(cx, cy, nullptr)) continue;
                    for (int lv = q.level - 2; lv >= 0; --lv) {
                        const int32_t m = ~(Forest::h(lv) - 1);
                        const int k = f.find(lv, cx & m, cy & m);
                        if (k >= 0) { split[k] = 1; any = true; break; }
                    }
                }
        }
        if (!any) break;
        std::vector<Quad> nl;
        for (size_t p = 0; p < f.leaves.size(); ++p) {
            const Quad& q = f.leaves[p];
            if (split[p]) {
                const int32_t hh = Forest::h(q.level + 1);
                for (int k = 0; k < 4; ++k) nl.push_back(Quad{q.level + 1, q.x + (k & 1) * hh, q.y + (k >> 1) * hh});
            } else {
                nl.push_back(q);
            }
        }
        f.leaves = nl;
        f.rebuild_index();
    }
    f.sort_morton();
    new_leaves = f.leaves;
    return true;
}

// fclaw2d_domain_iterate_adapted (forestclaw2d.c:1453-1507) with
// cb_fclaw2d_regrid_repopulate (fclaw2d_regrid.c:114-230).
void Solver::iterate_adapted(const std::vector<Quad>& old_leaves, std::vector<PatchData>& old_data,
                             bool domain_init) {
    const int nn = (int)forest.leaves.size();
    data.assign(nn, PatchData{});
    int oj = 0, nj = 0;
    while (oj < (int)old_leaves.size()) {
        const Quad& o = old_leaves[oj];
        const Quad& nw = forest.leaves[nj];
        if (o.level < nw.level) {
            for (int k = 0; k < 4; ++k) {
                build_patch(nj + k, false);
                if (domain_init) { setaux_patch(nj + k); qinit_patch(nj + k); }
                else setaux_patch(nj + k);
            }
            if (!domain_init)
                for (int k = 0; k < 4; ++k)
                    interpolate2fine(opt.mx, opt.my, opt.mbc, opt.meqn, old_data[oj].q.data(),
                                     data[nj + k].q.data(), k);
            oj += 1;
            nj += 4;
        } else if (o.level > nw.level) {
            build_patch(nj, false);
            setaux_patch(nj);
            if (domain_init) qinit_patch(nj);
            else
                for (int k = 0; k < 4; ++k)
                    average2coarse(opt.mx, opt.my, opt.mbc, opt.meqn, data[nj].q.data(),
                                   old_data[oj + k].q.data(), k);
            oj += 4;
            nj += 1;
        } else {
            data[nj] = std::move(old_data[oj]);
            oj += 1;
            nj += 1;
        }
    }
    if (nj != nn) throw std::runtime_error("iterate_adapted: leaf count mismatch");
}

// Tagging (fclaw2d_regrid.c:45-106) and adaptation; returns whether the mesh changed.
void Solver::tag_and_adapt(bool domain_init, bool* changed) {
    const int n = (int)forest.leaves.size();
    target_level.assign(n, 0);
    for (int p = 0; p < n; ++p) target_level[p] = forest.leaves[p].level;
    const int initflag = domain_init ? 1 : 0;
    // families first (cb_regrid_tag4coarsening)
    for (int p = 0; p < n; ++p) {
        if (!forest.is_first_sibling(p)) continue;
        const int level = forest.leaves[p].level;
        if (level > opt.minlevel && opt.coarsen_threshold > 0) {
            const double* qs[4] = {data[p].q.data(), data[p + 1].q.data(), data[p + 2].q.data(),
                                   data[p + 3].q.data()};
            const int tag = tag4coarsening(opt.mx, opt.my, opt.mbc, opt.meqn, dx(p), dy(p), qs,
                                           opt.coarsen_threshold, opt.criteria, opt.ivar, initflag);
            if (tag == 1)
                for (int k = 0; k < 4; ++k) target_level[p + k] = std::max(forest.leaves[p + k].level - 1, 0);
        }
        p += 3;
    }
    // then patches (cb_fclaw2d_regrid_tag4refinement)
    for (int p = 0; p < n; ++p) {
        const int level = forest.leaves[p].level;
        if (level < opt.maxlevel) {
            int tag;
            if (opt.refine_threshold < 0) tag = 1;
            else tag = tag4refinement(opt.mx, opt.my, opt.mbc, opt.meqn, dx(p), dy(p), data[p].q.data(),
                                      opt.refine_threshold, opt.criteria, opt.ivar);
            if (tag == 1) target_level[p] = level + 1;
        }
    }
    std::vector<Quad> new_leaves;
    *changed = domain_adapt(new_leaves);
    if (!*changed) return;
    std::vector<Quad> old_leaves = forest.leaves;
    std::vector<PatchData> old_data = std::move(data);
    forest.leaves = new_leaves;
    forest.rebuild_index();
    iterate_adapted(old_leaves, old_data, domain_init);
    set_neighbor_types();
}

void Solver::regrid() {
    bool changed = false;
    tag_and_adapt(false, &changed);
    if (changed) {
        ghost_update(forest.min_level(), forest.max_level(), curr_time, 0);
        ++count_amr_new_domain;
    }
    ++count_amr_regrid;
}

void Solver::initialize() {
    forest.uniform(opt.minlevel);
    data.assign(forest.leaves.size(), PatchData{});
    for (int p = 0; p < (int)forest.leaves.size(); ++p) {
        build_patch(p, true);
        setaux_patch(p);
        qinit_patch(p);
    }
    set_neighbor_types();
    if (opt.init_ghostcell) ghost_update(forest.min_level(), forest.max_level(), 0.0, 0);
    if (opt.minlevel < opt.maxlevel) {
        for (int level = opt.minlevel; level <= opt.maxlevel; ++level) {
            bool changed = false;
            tag_and_adapt(true, &changed);
            if (!changed) break;
        }
    }
    if (opt.init_ghostcell) ghost_update(forest.min_level(), forest.max_level(), 0.0, 0);
}

// outstyle_1 (fclaw2d_run.c:120-290)
void Solver::run() {
    const double final_time = opt.tfinal;
    const int nout = opt.nout;
    double dt_minlevel = opt.initial_dt;
    const double t0 = 0;
    const double dt_outer = (final_time - t0) / ((double)nout);
    double t_curr = t0;
    int n_inner = 0;
    for (int n = 0; n < nout; ++n) {
        const double tstart = t_curr;
        curr_time = t_curr;
        const double tend = tstart + dt_outer;
        while (t_curr < tend) {
            if (!opt.use_fixed_dt)
                for (auto& d : data) d.qsave = d.q;  // save_time_step
            double dt_step = dt_minlevel;
            const double tol = 1e-2 * dt_step;
            int took_small_step = 0;
            const double dt_step_desired = dt_step;
            (void)dt_step_desired;
            if (!opt.use_fixed_dt) {
                const double small_step = tend - (t_curr + dt_step);
                if (small_step < tol) {
                    dt_step = tend - t_curr;
                    if (small_step < 0) took_small_step = 1;
                }
            }
            const double maxcfl_step = advance_all_levels(t_curr, dt_step);
            if ((maxcfl_step > opt.max_cfl) && opt.reduce_cfl) {
                if (!opt.use_fixed_dt) {
                    for (auto& d : data) d.q = d.qsave;  // restore_time_step
                    dt_minlevel = dt_minlevel * opt.desired_cfl / maxcfl_step;
                    continue;
                }
            }
            ++n_inner;
            t_curr += dt_step;
            if (!opt.use_fixed_dt) {
                const double dt_new = dt_minlevel * opt.desired_cfl / maxcfl_step;
                if (!took_small_step) dt_minlevel = dt_new;
            }
            curr_time = t_curr;
            if (opt.regrid_interval > 0 && n_inner % opt.regrid_interval == 0) regrid();
        }
        curr_time = t_curr;
    }
}

void Solver::conservation(std::vector<double>& sums) const {
    sums.assign(opt.meqn, 0.0);
    std::vector<double> c(opt.meqn, 0.0);
    for (int p = 0; p < (int)forest.leaves.size(); ++p)
        conservation_sum(opt.mx, opt.my, opt.mbc, opt.meqn, dx(p), dy(p), data[p].q.data(), sums.data(), c.data());
}

}  // namespace orc
