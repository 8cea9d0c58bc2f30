// Plain-old-data structures shared by the host runtime and the CUDA kernels.
#pragma once
#include <cstddef>
#include <cstdint>

namespace fcb {

// Per-slot patch geometry, uploaded after each regrid.
struct PatchMeta {
    double xlower, ylower, dx, dy;
    int32_t level;
    int32_t flags;  // PATCH_SAVE_LAST: write q into qlast before stepping
};
enum : int32_t { PATCH_SAVE_LAST = 1 };

enum SolverKind : int32_t {
    SOLVER_ADVECTION = 0,
    SOLVER_SWE_ROE = 1,
    SOLVER_EULER4_ROE = 2,
    SOLVER_GEOCLAW_FWAVE = 3,
    SOLVER_ADVECTION_MANIFOLD = 4
};
enum AuxKind : int32_t { AUX_NONE = 0, AUX_SWIRL = 1, AUX_STORED = 2 };

// One patch of a launch that mixes patches of several solves (ensemble
// serving): its arrays, geometry and time step travel with it.
struct PatchDesc {
    double* q;            // the patch's q (qlast at the same offset in its qlast arena)
    double* qlast;
    const double* aux;    // stored aux of the patch, or null
    PatchMeta meta;
    double dt, vt;        // step and swirl velocity scale of the patch's solve
    int32_t req;          // CFL slot: cfl_out[req]
    int32_t pad;
};

// Ghost-exchange fusion on a mesh of one level: per slot, the slots of its
// same-size neighbours across faces 0-3 (left, right, bottom, top) and corners
// 0-3 (bottom-left, bottom-right, top-left, top-right), -1 where there is none,
// and the physical boundary condition of each face (mthbc 1 or 3, 0 where the
// face has a neighbour).  A fused step reads its ghost cells from these
// neighbours' interiors instead of from its own ghost cells.
struct FuseNbr {
    int32_t face[4];
    int32_t corner[4];
    int32_t bc[4];
};

// Arguments of one batched step launch (all patches of one level).
struct StepArgs {
    double* q;             // arena base
    double* qlast;         // arena base
    const double* aux;     // stored-aux arena base (AUX_STORED), else null
    const int32_t* slots;  // patch list
    const PatchMeta* meta; // indexed by slot
    int64_t q_stride;      // doubles per slot in q / qlast
    int64_t aux_stride;    // doubles per slot in aux
    int32_t npatches;
    int32_t maux;
    int32_t order0, order1;
    int32_t mthlim[8];
    double dt;
    double vt;             // swirl: cos(2 pi (t + dt/2) / tperiod)
    const double* dyn;     // non-null: {dt, vt} read from device memory (one macro-step graph serves every step)
    const PatchDesc* desc; // non-null: per-patch arrays, geometry and dt (slots, meta, q, dt unused)
    double grav, gamma, gamma1;
    double drytol;         // GeoClaw dry tolerance
    unsigned long long* cfl_out;  // atomicMax on the bits of a non-negative double
    double* treg;          // time-sync: conservation-register arena (null: off)
    int64_t treg_stride;   // doubles per slot in treg
    // nlvl > 1: one launch over the level updates between two ghost updates;
    // dyn holds {dt, vt} for levels lvl0 .. lvl0 + nlvl - 1 and each patch reads
    // its own level's pair
    int32_t lvl0, nlvl;
    // ghost-exchange fusion (fuse non-null): the step reads the arena qsrc, its
    // ghost cells resolved through fuse[slot] to the neighbours' interiors and
    // the physical boundary conditions, and writes the updated interior cells to
    // the arena q (qsrc != q)
    const double* qsrc;
    const FuseNbr* fuse;
    // four-barrier form: nbands > 1 splits every patch's rows into that many
    // bands, one CTA each, which read the copy qsrc of the arena (bands
    // overlap in the rows they read) and update their own rows in q
    int32_t nbands;
    // with nbands > 1: the first band_first CTAs update whole patches in place
    // (from q) and only the patches after them are split into bands (the tail
    // of a launch that would otherwise leave a nearly empty last wave)
    int32_t band_first;
    // four-barrier form, nbands <= 1: a scratch arena (q's layout) that lets
    // the launcher split the last, partial wave of CTAs into row bands (the
    // patches of that tail are copied there and read from it); null: off
    double* qtail;
};

// Conservation registers of one slot (fclaw2d_clawpatch_registers_t), doubles
// at these offsets, Fortran index order (j, m) / (i, m) and (j|i, m, k):
//   fp[k], fm[k]: k = 0 left, 1 right, my x meqn
//   gp[k], gm[k]: k = 0 bottom, 1 top, mx x meqn
//   ef[f]: f(q) accumulated at the interior (k = 0) and exterior (k = 1) cell
//          along face f (len x meqn x 2)
struct RegLayout {
    int mx, my, meqn;
    __host__ __device__ int ny() const { return my * meqn; }
    __host__ __device__ int nx() const { return mx * meqn; }
    __host__ __device__ int fp(int k) const { return k * ny(); }
    __host__ __device__ int fm(int k) const { return 2 * ny() + k * ny(); }
    __host__ __device__ int gp(int k) const { return 4 * ny() + k * nx(); }
    __host__ __device__ int gm(int k) const { return 4 * ny() + 2 * nx() + k * nx(); }
    __host__ __device__ int ef(int f) const {
        const int b = 4 * ny() + 4 * nx();
        return f < 2 ? b + f * 2 * ny() : b + 4 * ny() + (f - 2) * 2 * nx();
    }
    __host__ __device__ int size() const { return 8 * ny() + 8 * nx(); }
};

// Time-synchronisation records (fclaw2d_time_sync.c correct_coarse_cells).
enum TsOpType : int32_t {
    TS_SAMESIZE = 0,  // clawpack46_fort_time_sync_samesize on (slot, face) from neighbour nbr
    TS_F2C = 1,       // clawpack46_fort_time_sync_f2c on coarse slot, face, from fine nbr
    TS_RESET = 2,     // zero the registers of (slot, face)
};
struct TsOp {
    int32_t type, slot, face, nbr;
    int32_t dx, dy;  // same size: index shift to the neighbour; f2c: fine-index offset D
};
struct TsArgs {
    double* q;
    double* treg;
    int64_t q_stride, treg_stride;
    const PatchMeta* meta;
    int mx, my, mbc, meqn;
    const TsOp* ops;
    const int32_t* groups;  // group k = records [groups[k], groups[k+1]), one patch each
    int ngroups;
};
#ifdef __CUDACC__
// {dt, vt} of a patch of `level` (clamped: threads without a patch read a valid entry)
__device__ __forceinline__ const double* step_dv(const StepArgs& a, int level) {
    int k = level - a.lvl0;
    k = a.nlvl > 1 ? (k < 0 ? 0 : (k >= a.nlvl ? a.nlvl - 1 : k)) : 0;
    return a.dyn + 2 * k;
}
__device__ __forceinline__ double step_dt(const StepArgs& a, int level) { return a.dyn ? step_dv(a, level)[0] : a.dt; }
__device__ __forceinline__ double step_vt(const StepArgs& a, int level) { return a.dyn ? step_dv(a, level)[1] : a.vt; }
#endif

// Ghost-cell operations, one record per reference kernel call.
enum GhostOpType : int32_t {
    OP_COPY_FACE = 0,
    OP_COPY_CORNER = 1,
    OP_AVERAGE_FACE = 2,
    OP_AVERAGE_CORNER = 3,
    OP_INTERP_FACE = 4,
    OP_INTERP_CORNER = 5,
    OP_PHYSBC = 6,
};
struct GhostOp {
    int32_t type;
    int32_t dst;       // slot written (this patch / coarse patch for average / fine patch for interp)
    int32_t src;       // slot read
    int32_t face;      // iface / icorner (relative to the coarse patch for average/interp)
    int32_t dx, dy;    // index shift (copy) or fine-index offset D (average/interp)
    int32_t dst_ti;    // 1: dst uses the time-interpolated array
    int32_t src_ti;    // 1: src uses the time-interpolated array
    int32_t mthbc[4];  // physbc: per side, -1 = not a physical boundary
};

// Arguments of one ghost-fill wave launch.
struct GhostArgs {
    double* q;        // arena of current solutions
    double* qti;      // arena of time-interpolated solutions
    int64_t stride;
    int mx, my, mbc, meqn;
    const GhostOp* ops;    // records of the wave, sorted by destination patch
    const int32_t* groups; // group k = records [groups[k], groups[k+1]) (absolute indices into ops)
    int ngroups;
    int interp_fp32;       // mixed precision: coarse-to-fine interpolation in FP32
};

enum Problem : int32_t {
    PROB_SWIRL = 0,
    PROB_RADIALDAM = 1,
    PROB_QUADRANTS = 2,
    PROB_BATHY = 3,
    PROB_RADIALDAM_CELLAVE = 4,  // radialdam/user_4.6/qinit.f with cellave2.f
    PROB_HUMP = 5,               // shallow/2d/bump/user_4.6/qinit.f
    PROB_PERIODIC_DISC = 6,      // advection/2d/periodic/user_4.6/qinit.f, fdisc.f
    PROB_FILAMENT = 7,           // advection/2d/filament (example 1): qinit.f, fdisc.f, user46_setaux_manifold.f
};

struct QinitArgs {
    double* q;
    int64_t stride;
    const int32_t* slots;
    const PatchMeta* meta;
    int n, mx, my, mbc, meqn, problem;
    double gamma1;
    double p[32];
};

enum TagCriteria : int32_t { TAG_VALUE = 0, TAG_MINMAX = 1, TAG_DIFFERENCE = 2, TAG_GRADIENT = 3 };

// out[4*p + 0] = qmin, [1] = qmax, [2] = refine-exceeds (0/1), [3] = coarsen-exceeds (0/1)
struct TagArgs {
    const double* q;
    int64_t stride;
    const int32_t* slots;
    const PatchMeta* meta;
    int n, mx, my, mbc, ivar, criteria;
    double refine_th, coarsen_th;
    double* out;
};

}  // namespace fcb
