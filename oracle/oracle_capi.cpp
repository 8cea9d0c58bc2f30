// ORACLE -- test infrastructure only (see oracle_patch.hpp).
//
// Flat C entry points so that the Python tests can drive the oracle through
// ctypes.  Options travel as two arrays (ints, doubles) whose layout is fixed
// by orc_pack_layout() below and mirrored in tests/oracle.py.
#include <cstring>
#include <exception>
#include <string>

#include "oracle_amr.hpp"

using namespace orc;

namespace {
thread_local std::string g_err;

// Layout of the option arrays (indices into iopt / dopt).
enum IOpt {
    I_MX, I_MY, I_MBC, I_MEQN, I_MAUX, I_ORDER0, I_ORDER1, I_MCAPA, I_MWAVES,
    I_MTHLIM0, I_MTHLIM7 = I_MTHLIM0 + 7,
    I_MTHBC0, I_MTHBC3 = I_MTHBC0 + 3,
    I_MINLEVEL, I_MAXLEVEL, I_SUBCYCLE, I_REGRID_INTERVAL, I_SMOOTH_REFINE, I_SMOOTH_LEVEL,
    I_CRITERIA, I_IVAR, I_USE_FIXED_DT, I_NOUT, I_INIT_GHOSTCELL, I_REDUCE_CFL,
    I_SOLVER, I_PROBLEM, I_CLAW_VERSION, I_TIME_SYNC, I_SRC_TERM, I_BRICK, I_PERIODIC_X, I_PERIODIC_Y,
    I_COUNT
};
enum DOpt {
    D_REFINE_TH, D_COARSEN_TH, D_TFINAL, D_INITIAL_DT, D_MAX_CFL, D_DESIRED_CFL,
    D_GRAV, D_GAMMA, D_GAMMA1, D_DRYTOL, D_PPARAM0, D_AX = D_PPARAM0 + 32, D_BX, D_AY, D_BY, D_COUNT
};

Options unpack(const int* io, const double* d) {
    Options o;
    o.mx = io[I_MX]; o.my = io[I_MY]; o.mbc = io[I_MBC]; o.meqn = io[I_MEQN]; o.maux = io[I_MAUX];
    o.method.order0 = io[I_ORDER0]; o.method.order1 = io[I_ORDER1]; o.method.mcapa = io[I_MCAPA];
    o.method.mwaves = io[I_MWAVES];
    for (int k = 0; k < 8; ++k) o.method.mthlim[k] = io[I_MTHLIM0 + k];
    for (int k = 0; k < 4; ++k) o.mthbc[k] = io[I_MTHBC0 + k];
    o.minlevel = io[I_MINLEVEL]; o.maxlevel = io[I_MAXLEVEL]; o.subcycle = io[I_SUBCYCLE];
    o.regrid_interval = io[I_REGRID_INTERVAL]; o.smooth_refine = io[I_SMOOTH_REFINE];
    o.smooth_level = io[I_SMOOTH_LEVEL]; o.criteria = io[I_CRITERIA]; o.ivar = io[I_IVAR];
    o.use_fixed_dt = io[I_USE_FIXED_DT]; o.nout = io[I_NOUT]; o.init_ghostcell = io[I_INIT_GHOSTCELL];
    o.reduce_cfl = io[I_REDUCE_CFL];
    o.solver.kind = io[I_SOLVER]; o.problem = io[I_PROBLEM];
    o.method.version = io[I_CLAW_VERSION];
    o.time_sync = io[I_TIME_SYNC];
    o.src_term = io[I_SRC_TERM];
    o.brick = io[I_BRICK] > 0 ? io[I_BRICK] : 1;
    o.periodic_x = io[I_PERIODIC_X];
    o.periodic_y = io[I_PERIODIC_Y];
    o.ax = d[D_AX]; o.bx = d[D_BX]; o.ay = d[D_AY]; o.by = d[D_BY];
    o.refine_threshold = d[D_REFINE_TH]; o.coarsen_threshold = d[D_COARSEN_TH];
    o.tfinal = d[D_TFINAL]; o.initial_dt = d[D_INITIAL_DT]; o.max_cfl = d[D_MAX_CFL];
    o.desired_cfl = d[D_DESIRED_CFL];
    o.solver.grav = d[D_GRAV]; o.solver.gamma = d[D_GAMMA]; o.solver.gamma1 = d[D_GAMMA1];
    o.solver.drytol = d[D_DRYTOL];
    for (int k = 0; k < 32; ++k) o.pparams[k] = d[D_PPARAM0 + k];
    return o;
}

template <class F>
int guard(F&& f) {
    try {
        f();
        return 0;
    } catch (std::exception& e) {
        g_err = e.what();
        return 1;
    }
}
}  // namespace

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }
int orc_iopt_count() { return I_COUNT; }
// src2_axisymmetric on one patch (the source-term stage alone)
int orc_src2_axisymmetric(int mx, int my, int mbc, int meqn, double ylower, double dy, double gamma1, double dt,
                          double* q) {
    return guard([&] { src2_axisymmetric(mx, my, mbc, meqn, ylower, dy, gamma1, dt, q); });
}
int orc_dopt_count() { return D_COUNT; }

// ---- single-patch kernels --------------------------------------------------
int orc_step2(const int* iopt, const double* dopt, double* q, const double* aux, double dx, double dy,
              double dt, double* cfl) {
    return guard([&] {
        const Options o = unpack(iopt, dopt);
        *cfl = step2(o.solver, o.method, o.mx, o.my, o.mbc, o.meqn, o.maux, q, aux, dx, dy, dt);
    });
}
void orc_b4step2_swirl(int mx, int my, int mbc, int maux, double xlower, double ylower, double dx,
                       double dy, double t, double dt, double tperiod, double* aux) {
    b4step2_swirl(mx, my, mbc, maux, xlower, ylower, dx, dy, t, dt, tperiod, aux);
}
int orc_bc2(int mx, int my, int mbc, int meqn, double* q, const int* mthbc) {
    return guard([&] { bc2_default(mx, my, mbc, meqn, q, mthbc); });
}
void orc_qinit_swirl(int mx, int my, int mbc, int meqn, double xlower, double ylower, double dx,
                     double dy, double* q) {
    qinit_swirl(mx, my, mbc, meqn, xlower, ylower, dx, dy, q);
}
// geometry arrays: {xlower, ylower, level} for self and neighbour
static Transform mk(int mx, int my, const double* gs, const double* gn) {
    return Transform{PatchGeom{gs[0], gs[1], (int)gs[2]}, PatchGeom{gn[0], gn[1], (int)gn[2]}, mx, my};
}
void orc_copy_face(int mx, int my, int mbc, int meqn, double* qthis, const double* qnbr, int iface,
                   const double* gs, const double* gn) {
    copy_face(mx, my, mbc, meqn, qthis, qnbr, iface, mk(mx, my, gs, gn));
}
void orc_copy_corner(int mx, int my, int mbc, int meqn, double* qthis, const double* qnbr, int icorner,
                     const double* gs, const double* gn) {
    copy_corner(mx, my, mbc, meqn, qthis, qnbr, icorner, mk(mx, my, gs, gn));
}
void orc_average_face(int mx, int my, int mbc, int meqn, double* qc, const double* qf, int iface,
                      const double* gs, const double* gn) {
    average_face(mx, my, mbc, meqn, qc, qf, iface / 2, iface, mk(mx, my, gs, gn));
}
void orc_average_corner(int mx, int my, int mbc, int meqn, double* qc, const double* qf, int icorner,
                        const double* gs, const double* gn) {
    average_corner(mx, my, mbc, meqn, qc, qf, icorner, mk(mx, my, gs, gn));
}
void orc_interpolate_face(int mx, int my, int mbc, int meqn, const double* qc, double* qf, int iface,
                          const double* gs, const double* gn) {
    interpolate_face(mx, my, mbc, meqn, qc, qf, iface / 2, iface, mk(mx, my, gs, gn));
}
void orc_interpolate_corner(int mx, int my, int mbc, int meqn, const double* qc, double* qf,
                            int icorner, const double* gs, const double* gn) {
    interpolate_corner(mx, my, mbc, meqn, qc, qf, icorner, mk(mx, my, gs, gn));
}
void orc_interpolate2fine(int mx, int my, int mbc, int meqn, const double* qc, double* qf, int igrid) {
    interpolate2fine(mx, my, mbc, meqn, qc, qf, igrid);
}
void orc_average2coarse(int mx, int my, int mbc, int meqn, double* qc, const double* qf, int igrid) {
    average2coarse(mx, my, mbc, meqn, qc, qf, igrid);
}
int orc_timeinterp(int mx, int my, int mbc, int meqn, int psize, const double* qcurr,
                   const double* qlast, double* qinterp, double alpha) {
    return timeinterp(mx, my, mbc, meqn, psize, qcurr, qlast, qinterp, alpha);
}
int orc_tag4refinement(int mx, int my, int mbc, int meqn, double dx, double dy, const double* q,
                       double th, int criteria, int ivar) {
    return tag4refinement(mx, my, mbc, meqn, dx, dy, q, th, criteria, ivar);
}
int orc_tag4coarsening(int mx, int my, int mbc, int meqn, double dx, double dy, const double* q0,
                       const double* q1, const double* q2, const double* q3, double th, int criteria,
                       int ivar, int initflag) {
    const double* qs[4] = {q0, q1, q2, q3};
    return tag4coarsening(mx, my, mbc, meqn, dx, dy, qs, th, criteria, ivar, initflag);
}

// ---- whole-solver driver ----------------------------------------------------
void* orc_solver_new(const int* iopt, const double* dopt) {
    try {
        return new Solver(unpack(iopt, dopt));
    } catch (std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}
void orc_solver_free(void* s) { delete (Solver*)s; }
int orc_initialize(void* s) { return guard([&] { ((Solver*)s)->initialize(); }); }
int orc_run(void* s) { return guard([&] { ((Solver*)s)->run(); }); }
int orc_advance(void* s, double t, double dt, double* maxcfl) {
    return guard([&] { *maxcfl = ((Solver*)s)->advance_all_levels(t, dt); });
}
int orc_regrid(void* s) { return guard([&] { ((Solver*)s)->regrid(); }); }
int orc_ghost_update(void* s, int minlevel, int maxlevel, double t, int ti) {
    return guard([&] { ((Solver*)s)->ghost_update(minlevel, maxlevel, t, ti); });
}
int orc_update_single_step(void* s, int level, double t, double dt, double* maxcfl) {
    return guard([&] { *maxcfl = ((Solver*)s)->update_single_step(level, t, dt); });
}
int orc_timeinterp_level(void* s, int level, double alpha) {
    return guard([&] { ((Solver*)s)->timeinterp(level, alpha); });
}
int orc_num_patches(void* s) { return (int)((Solver*)s)->forest.leaves.size(); }
void orc_patch_info(void* s, int p, int* level, int* x, int* y) {
    const Quad& q = ((Solver*)s)->forest.leaves[p];
    *level = q.level; *x = q.x; *y = q.y;
}
void orc_get_q(void* s, int p, double* out) {
    const auto& v = ((Solver*)s)->data[p].q;
    std::memcpy(out, v.data(), v.size() * sizeof(double));
}
void orc_set_q(void* s, int p, const double* in) {
    auto& v = ((Solver*)s)->data[p].q;
    std::memcpy(v.data(), in, v.size() * sizeof(double));
}
void orc_get_qinterp(void* s, int p, double* out) {
    const auto& v = ((Solver*)s)->data[p].qinterp;
    std::memcpy(out, v.data(), v.size() * sizeof(double));
}
void orc_counters(void* s, long long* out) {
    Solver* S = (Solver*)s;
    out[0] = S->count_amr_advance;
    out[1] = S->count_amr_new_domain;
    out[2] = S->count_amr_regrid;
    out[3] = S->count_single_step;
}
void orc_conservation(void* s, double* sums) {
    std::vector<double> v;
    ((Solver*)s)->conservation(v);
    for (size_t k = 0; k < v.size(); ++k) sums[k] = v[k];
}
// Neighbour relations of patch p: face_rel[4], face_nbr[8], corner_rel[4] (0 = none), corner_nbr[4],
// flags[2] = {has_finegrid_neighbors, on_coarsefine_interface}.
void orc_neighbors(void* s, int p, int* out) {
    const NeighborInfo& n = ((Solver*)s)->nbrs[p];
    for (int f = 0; f < 4; ++f) {
        out[f] = n.face_rel[f];
        out[4 + 2 * f] = n.face_nbr[f][0];
        out[5 + 2 * f] = n.face_nbr[f][1];
        out[12 + f] = n.corner_rel[f];
        out[16 + f] = n.corner_nbr[f];
    }
    out[20] = n.has_finegrid_neighbors;
    out[21] = n.on_coarsefine_interface;
}

}  // extern "C"
