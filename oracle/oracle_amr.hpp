// ORACLE -- test infrastructure only (see oracle_patch.hpp).
//
// CPU restatement of the ForestClaw time-stepping core on one MPI rank and one
// unit-square block: the forest (leaf order, face/corner relations, smooth
// refinement, refine -> coarsen -> 2:1 corner balance), the subcycled level
// schedule, the ghost-fill phase order, time interpolation, regridding and
// the outstyle-1 run loop.  Each function cites the reference routine.
#pragma once
#include <cstdint>
#include <unordered_map>
#include <vector>

#include "oracle_clawpatch.hpp"

namespace orc {

enum Relation { REL_BOUNDARY = 0, REL_HALFSIZE = 1, REL_SAMESIZE = 2, REL_DOUBLESIZE = 3 };

enum Problem { PROB_SWIRL = 0, PROB_RADIALDAM = 1, PROB_QUADRANTS = 2, PROB_BATHY = 3, PROB_RADIALDAM_CELLAVE = 4, PROB_HUMP = 5, PROB_PERIODIC_DISC = 6, PROB_FILAMENT = 7 };

struct Options {
    // [clawpatch]
    int mx = 16, my = 16, mbc = 2, meqn = 1, maux = 2;
    // [clawpack46]
    MethodParams method;
    int mthbc[4] = {1, 1, 1, 1};
    // [Options]
    int minlevel = 4, maxlevel = 4;
    int subcycle = 1;
    int regrid_interval = 1;
    double refine_threshold = 0.5, coarsen_threshold = 0.1;
    int smooth_refine = 0, smooth_level = 0;
    int criteria = TAG_MINMAX;
    int ivar = 0;  // 0-based threshold-variable
    double tfinal = 1.0, initial_dt = 0.01, max_cfl = 1.0, desired_cfl = 0.9;
    int use_fixed_dt = 0;
    int nout = 1;
    int init_ghostcell = 0;
    int reduce_cfl = 1;
    // [Options] time-sync (flux-correction and fluctuation-correction on)
    int time_sync = 0;
    // [Options] mi = mj = brick (a power of two): a brick of brick x brick
    // blocks (fclaw2d_map_brick.c) whose leaves are kept as one tree with
    // levels offset by log2(brick); periodic_x / periodic_y wrap the domain
    int brick = 1;
    int periodic_x = 0, periodic_y = 0;
    // [clawpack46] src_term with the source of euler/2d/shockbubble/user_4.6/src2.f
    // (1: axisymmetric Euler source, radius aux(i,j,1) = y at the cell centre)
    int src_term = 0;
    // [Options] ax, bx, ay, by: the physical extent of the (unmapped) unit square
    double ax = 0.0, bx = 1.0, ay = 0.0, by = 1.0;
    // problem
    SolverParams solver;
    int problem = PROB_SWIRL;
    double pparams[32] = {0};
};

struct Quad {
    int level;
    int32_t x, y;  // lower-left corner in units of 2^-kMaxLevel
};

struct NeighborInfo {
    int face_rel[4];
    int face_nbr[4][2];
    int face_pos[4];  // DOUBLESIZE: which half of the big face this patch touches
    // periodic domains: the neighbour's position adjacent to this patch is its
    // stored position plus img * (block width) in x and y (0 unless the face or
    // corner crosses a periodic boundary)
    int face_img[4][2];
    int corner_img[4][2];
    int corner_exists[4];
    int corner_rel[4];
    int corner_nbr[4];
    int has_finegrid_neighbors = 0;
    int on_coarsefine_interface = 0;
};

// Leaves of one block in Morton (z-) order, as p4est stores a tree.
class Forest {
  public:
    static constexpr int kMaxLevel = 28;
    static constexpr int32_t kRoot = (int32_t)1 << kMaxLevel;
    std::vector<Quad> leaves;

    void uniform(int level);
    void rebuild_index();
    int find(int level, int32_t x, int32_t y) const;  // -1 if no leaf
    // Level of the leaf covering cell (level, x, y) searched at level-1..level+1 (-1 if none).
    int face_neighbors(int p, int face, int nbr[2], int* pos, int img[2] = nullptr) const;
    int corner_neighbor(int p, int corner, int* nbr, int img[2] = nullptr) const;  // relation, 0 if none
    // periodic domains: a point outside the block wraps into it (img receives
    // -1 / +1 per direction it wrapped); false if it lies outside a
    // non-periodic side
    bool wrap(int32_t& x, int32_t& y, int img[2]) const;
    bool periodic_x = false, periodic_y = false;
    int is_first_sibling(int p) const;
    void sort_morton();
    static uint64_t morton(int32_t x, int32_t y);
    static int32_t h(int level) { return (int32_t)1 << (kMaxLevel - level); }
    int min_level() const;
    int max_level() const;

  private:
    std::unordered_map<uint64_t, int> index_;
    static uint64_t key(int level, int32_t x, int32_t y) {
        return ((uint64_t)level << 58) | ((uint64_t)(uint32_t)x << 29) | (uint64_t)(uint32_t)y;
    }
};

// Conservation registers of one patch (fclaw2d_clawpatch_conservation.h,
// fclaw2d_clawpatch_time_sync_new): side k = 0 left, 1 right (fp, fm: my x
// meqn) and k = 0 bottom, 1 top (gp, gm: mx x meqn); edge_fluxes on faces
// 0..3 hold f(q) of the interior (0) and exterior (1) cell along the face
// (len x meqn x 2).  Fortran index order: (j, m) and (j, m, k).
struct Registers {
    std::vector<double> fp[2], fm[2], gp[2], gm[2], ef[4];
};

struct PatchData {
    std::vector<double> q, qlast, qinterp, qsave, aux;
    Registers reg;
};

class Solver {
  public:
    explicit Solver(const Options& o);
    Options opt;
    Forest forest;
    std::vector<PatchData> data;      // parallel to forest.leaves
    std::vector<NeighborInfo> nbrs;   // parallel to forest.leaves
    std::vector<int> target_level;
    // counters (fclaw2d_global_t)
    int count_amr_advance = 0, count_amr_new_domain = 0, count_amr_regrid = 0;
    long long count_single_step = 0;
    double curr_time = 0.0;

    void initialize();                                   // fclaw2d_initialize.c:75-248
    double advance_all_levels(double t, double dt);      // fclaw2d_advance.c:247-357
    double update_single_step(int level, double t, double dt);  // fclaw2d_update_single_step.c:73
    void ghost_update(int minlevel, int maxlevel, double sync_time, int time_interp);
    void timeinterp(int level, double alpha);            // fclaw2d_timeinterp.c:51
    void regrid();                                       // fclaw2d_regrid.c:234
    void run();                                          // fclaw2d_run.c outstyle_1
    void conservation(std::vector<double>& sums) const;  // diagnostics (Kahan)

    // geometry of a leaf
    double xlower(int p) const;  // block coordinates
    double ylower(int p) const;
    double xphys(int p) const;   // physical lower-left corner
    double yphys(int p) const;
    double dx(int p) const;
    double dy(int p) const;
    PatchGeom geom(int p) const;
    PatchGeom geom_img(int p, const int img[2]) const;

    size_t patch_size() const { return (size_t)opt.meqn * (opt.mx + 2 * opt.mbc) * (opt.my + 2 * opt.mbc); }
    size_t aux_size() const { return (size_t)opt.maux * (opt.mx + 2 * opt.mbc) * (opt.my + 2 * opt.mbc); }

    // exposed for tests
    void set_neighbor_types();
    void build_patch(int p, bool init);
    void qinit_patch(int p);
    void setaux_patch(int p);
    double single_step_patch(int p, double t, double dt);
    void physical_bc(int p, int time_interp);
    bool domain_adapt(std::vector<Quad>& new_leaves);
    // conservative time synchronisation (src/fclaw2d_time_sync.c)
    void time_sync(int minlevel, int maxlevel);

  private:
    void copy2ghost(int level, int time_interp);
    void average2ghost(int coarse_level, int time_interp);
    void interpolate2ghost(int coarse_level, int time_interp);
    void setphysical(int level, int time_interp);
    std::vector<int> patches_at_level(int level) const;
    double* q_time_sync(int p, int time_interp);
    void iterate_adapted(const std::vector<Quad>& old_leaves, std::vector<PatchData>& old_data,
                         bool domain_init);
    void tag_and_adapt(bool domain_init, bool* changed);
    void time_sync_store_flux(int p, double dt);
    void time_sync_accumulate(int p, double dt, const StepFluxArrays& f);
    void time_sync_samesize(int p, int iface);
    void time_sync_f2c(int pc, int pf, int iface);
    void time_sync_reset(int p, int coarse_level, int mode);
};

}  // namespace orc
