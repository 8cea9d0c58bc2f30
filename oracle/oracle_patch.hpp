// ORACLE -- test infrastructure only.
//
// CPU restatement of ForestClaw's Clawpack 4.6 patch arithmetic, written
// loop-for-loop after the reference Fortran so that loop bounds, accumulation
// order and ghost-region updates are the same.  It exists to check the CUDA
// path: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg
// may load it.  The product library never links it.
//
// Storage convention (the reference "46" layout): q(i,j,m) with Fortran
// indices i in [1-mbc, mx+mbc], j in [1-mbc, my+mbc], i fastest, then j, then m.
#pragma once
#include <cmath>
#include <cstdint>
#include <vector>

namespace orc {

enum SolverKind {
    SOLVER_ADVECTION = 0,   // clawpack46_rpn2adv / rpt2adv (swirl aux velocities)
    SOLVER_SWE_ROE = 1,     // shallow/2d/rp/clawpack46_rpn2.f / rpt2.f
    SOLVER_EULER4_ROE = 2,  // euler/2d/rp/clawpack46_rpn2_euler4.f / rpt2_euler4.f
    SOLVER_GEOCLAW_FWAVE = 3,  // shallow/2d/rp/rpn2_geoclaw.f90 (f-waves, clawpack46_flux2fw.f)
    SOLVER_ADVECTION_MANIFOLD = 4,  // advection/2d/all/clawpack46_rpn2adv_manifold.f / rpt2adv_manifold.f
                                    // (aux(1) capacity, aux(2:3) edge velocities)
};

struct SolverParams {
    int kind = SOLVER_ADVECTION;
    double grav = 1.0;      // /cparam/ grav (SWE)
    double gamma = 1.4;     // /cparam/ gamma (Euler)
    double gamma1 = 0.4;    // /cparam/ gamma1 = gamma - 1
    double drytol = 1e-3;   // /common_swe/ dry_tolerance (GeoClaw)
};

struct MethodParams {
    int order0 = 2;         // method(2): 1 = Godunov only, 2 = second-order corrections
    int order1 = 2;         // method(3): 0 none, 1 transverse increments, 2 + corrections
    int mcapa = 0;          // capacity index (0 = none)
    int mwaves = 1;
    int mthlim[8] = {4, 4, 4, 4, 4, 4, 4, 4};
    int version = 4;        // 4: clawpack 4.6 (fc2d_clawpack46), 5: clawpack 5 (fc2d_clawpack5)
};

// Index helper for one patch array with Fortran bounds.
struct PatchIdx {
    int mx, my, mbc, nx, ny;
    PatchIdx(int mx_, int my_, int mbc_) : mx(mx_), my(my_), mbc(mbc_),
        nx(mx_ + 2 * mbc_), ny(my_ + 2 * mbc_) {}
    inline int64_t operator()(int i, int j, int m) const {
        return ((int64_t)m * ny + (j + mbc - 1)) * nx + (i + mbc - 1);
    }
    inline int64_t size(int meqn) const { return (int64_t)meqn * nx * ny; }
};

// Fortran DMAX1/DMIN1 on non-NaN operands.
inline double dmax(double a, double b) { return a > b ? a : b; }
inline double dmin(double a, double b) { return a < b ? a : b; }

// clawpack46_step2_wrap.f:1-127 + clawpack46_step2.f:5-239 + clawpack46_flux2.f:4-228:
// updates q in place over i,j = 1-mbc..mx+mbc-1 and returns cflgrid.
// With mp.version == 5: clawpack5_step2_wrap.f:1-115 + clawpack5_step2.f90:1-172 +
// clawpack5_flux2.f:4-235 (interfaces 1..mx+1 only, interior update i,j = 1..mx,
// clawpack5_rpn2.f90 / clawpack5_rpt2.f90 arithmetic for the shallow-water solver).
// The flux accumulators fm, fp, gm, gp of one step (46 layout), kept for the
// time-sync registers (fc2d_clawpack46.cpp:369-386).
struct StepFluxArrays {
    std::vector<double> fm, fp, gm, gp;
};
double step2(const SolverParams& sp, const MethodParams& mp,
             int mx, int my, int mbc, int meqn, int maux,
             double* q, const double* aux, double dx, double dy, double dt,
             StepFluxArrays* keep = nullptr);

// shallow/2d/radialdam/rpn2cons_update.f: the physical flux f(q) (idir 0) or
// g(q) (idir 1) of the shallow-water equations at one cell.
void rpn2_cons_update_swe(int meqn, int idir, const double* q, double grav, double* flux);

// radialdam/user_4.6/qinit.f with src/fortran_source2d/cellave2.f (cellave2,
// fss, zeroin) and radialdam/fdisc.f (no mapping): h = hin*w + hout*(1-w),
// w the fraction of the cell inside the circle of radius r0 about (x0, y0).
void qinit_radialdam_cellave(int mx, int my, int mbc, double xlower, double ylower, double dx, double dy,
                             double x0, double y0, double r0, double hin, double hout, double* q);

// Shallow water over bathymetry: b(x,y) = -1 + 0.8 exp(-((x-.5)^2 + (y-.5)^2)/0.02)
// at cell centres (aux(i,j,1), ghost cells included), and a surface
// eta = amp exp(-((x-x0)^2 + (y-y0)^2)/width^2) on a lake at rest: h = max(0, eta - b),
// hu = hv = 0.  p = {x0, y0, amp, width}.
void setaux_bathy(int mx, int my, int mbc, double xlower, double ylower, double dx, double dy, double* aux);

// advection/2d/periodic: user_4.6/clawpack46_setaux.f (aux(i,j,1) = uvel,
// aux(i,j,2) = vvel over the whole patch) and user_4.6/qinit.f with fdisc.f
// (q = the fraction of each cell inside the disc sqrt((x-x0)^2+(y-y0)^2) < r0,
// cellave2.f; the application's disc is r0 = 0.25 about the origin).
void setaux_velocity(int mx, int my, int mbc, int maux, double uvel, double vvel, double* aux);

// advection/2d/filament, example 1 (a 2 x 2 brick under the cart mapping,
// manifold = T): all/user46_setaux_manifold.f with the metric's affine area
// (src/patches/metric/fortran_source2d/fclaw2d_metric_default_fort.f90:
// compute_area_affine, get_area_approx, norm_cross) and filament/psi.f:
//   aux(i,j,1) = area(i,j)/(dx*dy),
//   aux(i,j,2) = (psi(node(i,j+1)) - psi(node(i,j)))/dy,
//   aux(i,j,3) = -(psi(node(i+1,j)) - psi(node(i,j)))/dx,
// psi = (4/3) r^3, r = |(x,y) - (1,1)|, node(i,j) = (xlower+(i-1)dx, ylower+(j-1)dy).
// The brick and cart maps send every node of this dyadic mesh to the same
// point of [0,2]^2 exactly, so the nodes are the physical coordinates.
// kmod != 0 (a test setting; the application's is 0) multiplies the capacity
// by 1 + kmod*xc*yc at the cell centre, so that dtdx1d varies from cell to cell.
void setaux_filament(int mx, int my, int mbc, double xlower, double ylower, double dx, double dy, double kmod,
                     double* aux);
void qinit_disc_fraction(int mx, int my, int mbc, int meqn, double xlower, double ylower, double dx, double dy,
                         double x0, double y0, double r0, double* q);
void qinit_bathy(int mx, int my, int mbc, double xlower, double ylower, double dx, double dy, const double* p,
                 double* q);

// shallow/2d/bump/user_4.6/qinit.f (user_5.0/qinit.f90 computes the same):
// h = base + exp(-coef*r2), r2 = (xc-x0)**2 + (yc-y0)**2, hu = hv = 0 over the
// whole patch, ghost cells included.  The reference has x0 = y0 = 0,
// base = 0.1, coef = 200.
void qinit_hump(int mx, int my, int mbc, double xlower, double ylower, double dx, double dy, double x0,
                double y0, double base, double coef, double* q);

// euler/2d/shockbubble/user_4.6/src2.f (clawpack5: user_5.0/src2.f90, the
// same arithmetic): the axisymmetric source of the Euler equations over the
// interior cells, a two-stage Runge-Kutta step with radius rad = y at the cell
// centre (shockbubble setaux.f: aux(i,j,1) = ylower + (j-0.5)*dy); components
// 1-4 change, a tracer (component 5) does not.
void src2_axisymmetric(int mx, int my, int mbc, int meqn, double ylower, double dy, double gamma1, double dt,
                       double* q);

// swirl/user_4.6/b4step2.f (+ swirl/psi.f): time-dependent edge velocities.
void b4step2_swirl(int mx, int my, int mbc, int maux, double xlower, double ylower,
                   double dx, double dy, double t, double dt, double tperiod, double* aux);

// swirl/user_4.6/qinit.f
void qinit_swirl(int mx, int my, int mbc, int meqn, double xlower, double ylower,
                 double dx, double dy, double* q);
// Radial dam break (cell-centre test), hu = hv = 0.
void qinit_radialdam(int mx, int my, int mbc, double xlower, double ylower, double dx, double dy,
                     double x0, double y0, double r0, double hin, double hout, double* q);
// euler/2d/quadrants/user_4.6/qinit.f with the quadrant states as parameters
// (rho, u, v, p for quadrants 1..4) and the split point (xs, ys).
void qinit_quadrants(int mx, int my, int mbc, double xlower, double ylower, double dx, double dy,
                     double gamma1, const double* rpr, const double* rpu, const double* rpv,
                     const double* rpp, double xs, double ys, double* q);

// clawpack46_bc2_default.f: mthbc per side (left,right,bottom,top); -1 = skip.
void bc2_default(int mx, int my, int mbc, int meqn, double* q, const int mthbc[4]);

}  // namespace orc
