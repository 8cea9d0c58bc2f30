/*
 * forestclaw-b200: C ABI of the B200 (sm_100a) patch hot path.
 *
 * One context holds one solve: the quadtree forest (single unit-square block,
 * p4est leaf-order semantics) on the host, and every patch array (q, the
 * pre-step copy used for time interpolation, the time-interpolated copy, the
 * CFL-retry copy, aux) resident in a pooled device arena indexed by slot.
 * Neighbour tables and ghost-fill operation lists are rebuilt on the host and
 * uploaded only after a regrid.
 *
 * Every entry point returns FCB_OK (0) or an error code and never exits the
 * process; fcb_last_error() returns the message of the last failure on the
 * calling thread.  Host buffers are plain pointers; patch arrays use the
 * reference's clawpack 4.6 layout q(i,j,m) with i fastest and Fortran ranges
 * i in [1-mbc, mx+mbc], j in [1-mbc, my+mbc].
 *
 * A context is used from one host thread at a time.  Work is enqueued on the
 * CUDA stream given at creation (or the legacy default stream for NULL).
 */
#ifndef FCLAW_B200_H
#define FCLAW_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FCB_ABI_VERSION 1

enum fcb_status {
    FCB_OK = 0,
    FCB_ERR_INVALID = 1,     /* bad argument or unsupported option combination */
    FCB_ERR_CUDA = 2,        /* a CUDA call failed */
    FCB_ERR_STATE = 3,       /* call out of order (e.g. step before initialize) */
    FCB_ERR_NUMERIC = 4,     /* NaN/Inf in the CFL number */
    FCB_ERR_INTERNAL = 5,
    FCB_ERR_COMM = 6         /* partitioned solve: a rank failed, sizes disagreed, or a
                              * collective outlasted the communicator's time limit */
};

/* Riemann solver families (fc2d_clawpack46_vtable_t rpn2/rpt2 pairs). */
enum fcb_solver_kind {
    FCB_SOLVER_ADVECTION = 0,  /* clawpack46_rpn2adv / rpt2adv (edge velocities in aux) */
    FCB_SOLVER_SWE_ROE = 1,    /* shallow water Roe with entropy fix (clawpack46_rpn2/rpt2) */
    FCB_SOLVER_EULER4_ROE = 2, /* Euler Roe with entropy fix (clawpack46_rpn2_euler4/rpt2_euler4) */
    FCB_SOLVER_GEOCLAW_FWAVE = 3, /* shallow water over bathymetry aux(1) = b: rpn2_geoclaw f-waves
                                   * with clawpack46_flux2fw; order (2, 0) only, because the
                                   * reference's rpt2_geoclaw stops; FP64 only */
    FCB_SOLVER_ADVECTION_MANIFOLD = 4 /* clawpack46_rpn2adv_manifold / rpt2adv_manifold on a mapped grid:
                                       * capacity aux(1) (mcapa = 1, clawpack46_step2.f / step2_wrap.f
                                       * capacity form), edge velocities aux(2:3); clawpack 4.6 and 5
                                       * (clawpack5_rpn2adv_manifold.f90, interior update), FP64 */
};

/* Initial conditions / b4step2 hooks of the configured applications. */
enum fcb_precision {
    FCB_PRECISION_FP64 = 0,  /* the reference's FP64 arithmetic */
    FCB_PRECISION_MIXED = 1  /* FP32 solves / limiters / ghost interpolation, FP64 sums and state */
};

enum fcb_problem {
    FCB_PROBLEM_SWIRL = 0,      /* advection/2d/swirl: qinit.f, b4step2.f velocities; p[0] = tperiod */
    FCB_PROBLEM_RADIALDAM = 1,  /* dam break: p = {x0, y0, r0, h_in, h_out} */
    FCB_PROBLEM_QUADRANTS = 2,  /* euler/2d/quadrants qinit.f: p = rho[4], u[4], v[4], p[4], xs, ys */
    FCB_PROBLEM_BATHY = 3,      /* lake at rest over b = -1 + 0.8 exp(-((x-.5)^2+(y-.5)^2)/0.02)
                                 * with a surface pulse p[2] exp(-((x-p[0])^2+(y-p[1])^2)/p[3]^2) */
    FCB_PROBLEM_RADIALDAM_CELLAVE = 4, /* the reference's radialdam qinit (radialdam/user_4.6/qinit.f):
                                 * depth p[3]*w + p[4]*(1-w), w the fraction of the cell inside the
                                 * circle about (p[0], p[1]) of radius p[2] (cellave2.f) */
    FCB_PROBLEM_HUMP = 5,       /* shallow/2d/bump qinit (user_4.6/qinit.f, user_5.0/qinit.f90):
                                 * depth p[2] + exp(-p[3]*r2), r2 = (xc-p[0])^2 + (yc-p[1])^2, at rest */
    FCB_PROBLEM_PERIODIC_DISC = 6, /* advection/2d/periodic (user_4.6/qinit.f, fdisc.f, clawpack46_setaux.f):
                                 * q = the cell's fraction inside the disc of radius p[4] about (p[2], p[3])
                                 * (cellave2.f), constant velocity (p[0], p[1]) in aux(1:2), maux >= 2 */
    FCB_PROBLEM_FILAMENT = 7    /* advection/2d/filament example 1 (cart-mapped 2 x 2 brick, extent [0, 2]^2):
                                 * q as FCB_PROBLEM_PERIODIC_DISC with the disc (p[2], p[3]), radius p[4]
                                 * (fdisc.f: (0.5, 1), 0.25); aux(1) = area/(dx dy) (the metric's affine
                                 * area), aux(2:3) = edge velocities of psi = (4/3) r^3 about (1, 1)
                                 * (user46_setaux_manifold.f, psi.f); manifold advection solver.
                                 * p[0] != 0 (0 in the application) multiplies the capacity by
                                 * 1 + p[0]*xc*yc at the cell centre (a test setting) */
};

/* Source terms (fc2d_clawpack46_vtable_t / fc2d_clawpack5_vtable_t src2). */
enum fcb_source {
    FCB_SOURCE_NONE = 0,
    FCB_SOURCE_AXISYMMETRIC_EULER = 1  /* euler/2d/shockbubble/user_4.6/src2.f: the axisymmetric Euler
                                        * source, radius y at the cell centre (its setaux.f); Euler
                                        * solver (meqn 4) */
};

/* Refinement criteria (fclaw2d_clawpatch_options "refinement-criteria"). */
enum fcb_criteria { FCB_TAG_VALUE = 0, FCB_TAG_MINMAX = 1, FCB_TAG_DIFFERENCE = 2, FCB_TAG_GRADIENT = 3 };

/*
 * The fields of fclaw_options_t, fclaw2d_clawpatch_options_t and
 * fc2d_clawpack46_options_t that the patch hot path reads (names as in the
 * reference's ini sections).  One unmapped block: the unit square, or
 * [ax, bx] x [ay, by] when those are set.
 */
typedef struct fcb_options {
    /* [clawpatch] */
    int mx, my, mbc, meqn, maux;
    int refinement_criteria;   /* enum fcb_criteria */
    int threshold_variable;    /* 1-based component used for tagging */
    /* [clawpack46] */
    int order[2];              /* method(2:3) */
    int mcapa;                 /* 0, or 1 with FCB_SOLVER_ADVECTION_MANIFOLD: capacity kappa in aux(1)
                                * (the four-barrier FP64 step form, clawpack 4.6 or 5) */
    int mwaves;
    int mthlim[8];
    int mthbc[4];              /* left, right, bottom, top: 1 extrapolation, 3 wall */
    /* [Options] */
    int minlevel, maxlevel;
    int subcycle;
    int regrid_interval;
    int smooth_refine, smooth_level;
    int use_fixed_dt;
    int nout;
    int init_ghostcell;
    int reduce_cfl;
    double refine_threshold, coarsen_threshold;
    double tfinal, initial_dt, max_cfl, desired_cfl;
    /* solver and problem */
    int solver_kind;           /* enum fcb_solver_kind */
    int problem;               /* enum fcb_problem */
    double grav;               /* SWE /cparam/ grav */
    double gamma;              /* Euler /cparam/ gamma; gamma1 = gamma - 1 */
    double problem_params[32];
    /* step kernel form: 0 = chosen by the library, 1 = one CTA per patch group
     * (rows through shared memory, four barriers per row), 2 = warp-synchronous
     * (swirl advection, mx = 8, 16, 32), 3 = software-pipelined CTA form (one
     * barrier per row; mx = 8, 16, 32), 4 and 5 = form 1 with every patch's
     * rows split into 2 or 3 bands of separate CTAs (Roe solvers; more, shorter
     * row sweeps); all give identical results */
    int step_variant;
    /* arithmetic of the patch update: 0 = FP64 throughout (the reference's
     * arithmetic), 1 = mixed: Riemann solves, limiters, transverse parts and
     * ghost interpolation in FP32, flux sums, cell update, state and mass sums
     * in FP64 (pipelined step form only); enum fcb_precision */
    int precision;
    /* 1: fcb_advance_all_levels replays the whole subcycled macro-step (level
     * updates, time interpolation, ghost fills) as one CUDA graph, captured on
     * the second call for a mesh; 0: every launch is issued from the host;
     * 2: automatic (the graph whenever a macro step updates a level) */
    int macro_graph;
    /* 4 (or 0): the fc2d_clawpack46 update; 5: the fc2d_clawpack5 update
     * (fluxes at interfaces 1..mx+1, interior cells updated, clawpack5 Riemann
     * solver arithmetic); fcb_get_q / fcb_set_q then use the clawpack 5 array
     * order q(m,i,j) for every patch (pipelined step form only) */
    int claw_version;
    /* GeoClaw /common_swe/ dry_tolerance */
    double dry_tolerance;
    /* [Options] time-sync: conservative correction of coarse cells at
     * coarse/fine faces and of edge cells at same-size faces after every
     * synchronisation of levels (fclaw2d_time_sync.c; flux-correction and
     * fluctuation-correction on).  Shallow-water Roe solver, clawpack 4.6 or 5,
     * FP64, the four-barrier or pipelined step form (step_variant 0, 1 or 3;
     * clawpack 5: 0 or 3). */
    int time_sync;
    /* [Options] ax, bx, ay, by: physical extent of the block; all four zero
     * means the unit square */
    double ax, bx, ay, by;
    /* [Options] weighted-partition: with subcycling, a partitioned solve
     * weighs a leaf of level l by 2^l (its updates per macro step) when it cuts
     * the Morton order into ranges (fclaw2d_partition.c:142) */
    int weighted_partition;
    /* Ghost-exchange fusion (no counterpart in the reference's options): on a
     * mesh of one level, fcb_advance_all_levels may fold the ghost update that
     * follows each step into the next step, which then reads its ghost cells
     * from the neighbours' interiors (the same values the copy and physical
     * boundary kernels would write).  The arrays move between two arenas, and
     * the last ghost update of a macro step is deferred until a call reads
     * ghost cells (fcb_get_q, fcb_regrid, a level update, ...), so every result
     * equals the unfused one bit for bit.  0: chosen by the autotuner (the
     * fused step against the best step form plus the ghost fill), 1: off,
     * 2: on whenever the mesh has one level (pipelined step form). */
    int ghost_fusion;
    /* [clawpack46] / [clawpack5] src_term: the src2 stage after every patch
     * step (clawpack46_update, fc2d_clawpack46.cpp:436-440; clawpack5_update,
     * fc2d_clawpack5.cpp:397-403), selected by enum fcb_source as the Riemann
     * solvers are (the device cannot call the host's Fortran src2 pointer). */
    int src_term;
    /* [Options] mi = mj: a brick of brick x brick unmapped blocks (a power of
     * two; 0 or 1: one block) on [ax, bx] x [ay, by] (fclaw2d_map_brick.c).
     * It is kept as one quadtree whose levels count from the whole domain:
     * minlevel/maxlevel/smooth_level are the brick's (per block), and
     * fcb_patch_info reports block level + log2(brick). */
    int brick;
    /* [Options] periodic_x / periodic_y: faces on the domain boundary connect
     * to the opposite side (one rank, no time-sync) */
    int periodic_x, periodic_y;
} fcb_options_t;

typedef struct fcb_counters {
    long long count_amr_advance;     /* fclaw2d_global_t counters of the same names */
    long long count_amr_new_domain;
    long long count_amr_regrid;
    long long count_single_step;     /* patch updates; x mx*my = cell updates */
    long long count_ghost_waves;     /* ghost-fill kernel launches */
    long long count_kernel_launches; /* all kernels launched by the library (graph replays included) */
    long long count_graph_replays;   /* macro steps replayed from a captured CUDA graph */
} fcb_counters_t;

typedef struct fcb_context fcb_context_t;

/* ---- context ---------------------------------------------------------------- */
/* Replaces the solver/patch setup of fc2d_clawpack46_solver_initialize
 * (src/solvers/fc2d_clawpack4.6/fc2d_clawpack46.cpp:483-537) and
 * fclaw2d_domain_new_unitsquare (src/fclaw2d_convenience.c:326). */
int fcb_context_create(const fcb_options_t* opt, void* cuda_stream, fcb_context_t** out);
int fcb_context_destroy(fcb_context_t* ctx);
const char* fcb_last_error(void);
int fcb_abi_version(void);

/* ---- time stepping core ---------------------------------------------------- */
/* fclaw2d_initialize (src/fclaw2d_initialize.c:75): uniform minlevel, qinit,
 * initial refinement up to maxlevel. */
int fcb_initialize(fcb_context_t* ctx);
/* fclaw2d_run outstyle 1 (src/fclaw2d_run.c:120-290): advance to tfinal with
 * adaptive dt, CFL rejection and regridding. */
int fcb_run(fcb_context_t* ctx);
/* fclaw2d_advance_all_levels (src/fclaw2d_advance.c:247): one subcycled
 * macro-step from t with coarse step dt; returns the max CFL over all updates. */
int fcb_advance_all_levels(fcb_context_t* ctx, double t, double dt, double* maxcfl);
/* The same macro step (fclaw2d_advance_all_levels, src/fclaw2d_advance.c:247)
 * without waiting for its CFL number: the call returns once the work is
 * enqueued on the context's stream, and the number goes into a running maximum
 * on the device.  fcb_read_max_cfl waits for the work enqueued so far, returns
 * the largest CFL number of the asynchronous macro steps since the last read
 * (0 if none) and resets it; a NaN there is FCB_ERR_NUMERIC.  For run loops
 * that need the CFL number only every few steps (fixed dt).  In a partitioned
 * solve both calls are per rank, as fcb_advance_all_levels is: the number is
 * the rank's maximum (fcb_global_maximum reduces it). */
int fcb_advance_all_levels_async(fcb_context_t* ctx, double t, double dt);
int fcb_read_max_cfl(fcb_context_t* ctx, double* maxcfl);
/* fclaw2d_update_single_step (src/fclaw2d_update_single_step.c:73): every patch
 * of `level` advanced by dt in one batched launch; returns the level max CFL. */
int fcb_update_single_step(fcb_context_t* ctx, int level, double t, double dt, double* maxcfl);
/* The batched level update of fcb_update_single_step without the CFL
 * read-back: the launch is only enqueued on the context's stream, and the
 * level max CFL is folded into the value fcb_advance_all_levels reports next.
 * For callers that pipeline several levels before synchronising. */
int fcb_update_single_step_async(fcb_context_t* ctx, int level, double t, double dt);
/* patch_vt->single_step_update (src/fclaw2d_patch.h:937-943, set at
 * fc2d_clawpack46.cpp:512) with the buffer_data protocol of
 * fclaw2d_update_single_step.h:47-71: calls with iter = 0..total_count-1 are
 * recorded; the call with iter == total_count-1 launches the batch and returns
 * the batch CFL in *cfl (the other calls return 0). */
int fcb_single_step_update(fcb_context_t* ctx, int patchno, double t, double dt, int iter,
                           int total_count, double* cfl);
/* fclaw2d_ghost_update (src/fclaw2d_ghost_fill.c:838), one rank. */
int fcb_ghost_update(fcb_context_t* ctx, int minlevel, int maxlevel, double sync_time, int time_interp);
/* fclaw2d_timeinterp (src/fclaw2d_timeinterp.c:51). */
int fcb_timeinterp(fcb_context_t* ctx, int level, double alpha);
/* fclaw2d_regrid (src/fclaw2d_regrid.c:234); *changed = 1 if the mesh changed. */
int fcb_regrid(fcb_context_t* ctx, int* changed);
/* fclaw2d_physical_set_bc (src/fclaw2d_physical_bc.c) for every patch of a level. */
int fcb_physical_set_bc(fcb_context_t* ctx, int level, int time_interp);

/* ---- queries and data movement ------------------------------------------------ */
int fcb_num_patches(fcb_context_t* ctx, int* n);
/* Leaf p in Morton order: level and lower-left corner in units of 2^-28. */
int fcb_patch_info(fcb_context_t* ctx, int p, int* level, int* x, int* y);
/* Neighbour relations of leaf p (layout: face_rel[4], face_nbr[4][2],
 * corner_rel[4] (0 = no corner neighbour), corner_nbr[4], has_fine, on_cf):
 * relation codes 0 boundary, 1 half size, 2 same size, 3 double size. */
int fcb_patch_neighbors(fcb_context_t* ctx, int p, int* out22);
/* Size in doubles of one patch array: meqn*(mx+2mbc)*(my+2mbc). */
int fcb_patch_size(fcb_context_t* ctx, size_t* n);
/* Copy all leaves' q (Morton order, patch after patch) to/from host memory. */
int fcb_get_q(fcb_context_t* ctx, double* host, size_t n);
int fcb_set_q(fcb_context_t* ctx, const double* host, size_t n);
/* Time-interpolated arrays of all leaves (same layout). */
int fcb_get_qinterp(fcb_context_t* ctx, double* host, size_t n);
int fcb_counters(fcb_context_t* ctx, fcb_counters_t* out);
/* Mass diagnostic (fclaw2d_clawpatch46_diagnostics.f:13-58): Kahan sum of
 * q*dx*dy per component over all leaves; sums has meqn entries. */
int fcb_conservation_check(fcb_context_t* ctx, double* sums);
/* Mass sums that allocate no device memory.  No counterpart in the reference:
 * it exists for callers that must not allocate while they run (a serving loop
 * whose HBM is fully committed to admitted solves, code that must not let a
 * cudaMalloc/cudaFree synchronise the device, hosts that own all device memory).
 * Inputs are the caller's device arrays: npatches patch arrays of
 * meqn*(mx+2mbc)*(my+2mbc) doubles in the layout above, patch_stride doubles
 * apart, and one cell area (dx*dy) per patch; d_sums receives meqn doubles
 * (Kahan over each patch's interior, then over the patches in order, the same
 * sequence as fcb_conservation_check).  Work is enqueued on cuda_stream.
 * Per-patch partial sums live in a fixed array of 262,144 doubles (2 MiB)
 * inside the library, held by every GPU that loads it; npatches*meqn above
 * that is rejected with FCB_ERR_INVALID.  The first call on each device looks
 * up that array's address, so make it before any stream capture; the address
 * is kept for the life of the process, so a cudaDeviceReset of that device
 * between calls leaves it stale (do not reset a device this entry point has
 * used).  All calls share the array: calls that overlap on the GPU race and
 * must be serialised by the caller. */
int fcb_conservation_sum_noalloc(const double* d_q, size_t patch_stride, int npatches, int mx, int my, int mbc,
                                 int meqn, const double* d_area, double* d_sums, void* cuda_stream);
/* Current time of the run loop. */
int fcb_curr_time(fcb_context_t* ctx, double* t);
/* Output frame `iframe` (0..9999) of all leaves in the reference's ASCII
 * format: dir/fort.tNNNN (time, meqn, ngrids, num_aux, num_dim) and
 * dir/fort.qNNNN (per patch a grid header, then the interior cells row by row)
 * (fclaw2d_clawpatch_output_ascii, src/patches/clawpatch/
 * fclaw2d_clawpatch_output_ascii.c; fort_4.6/fclaw2d_clawpatch46_output_ascii.f).
 * dir must exist; NULL means the working directory. */
int fcb_output_ascii(fcb_context_t* ctx, int iframe, const char* dir);
/* Autotuner choices of the last launches (no counterpart in the reference):
 * step_form 1 = one CTA per patch with four barriers per stage, 2 = one warp
 * per patch, 3 = pipelined row sweep; ghost_unroll = ghost records per thread
 * per pass (2, 4 or 8).  With step_variant 0 the library times the forms that
 * exist for the case on its first level update, on scratch copies of the
 * arrays, and keeps the fastest for the process; 0 before the first update. */
int fcb_autotune_info(fcb_context_t* ctx, int* step_form, int* ghost_unroll);
/* Device time of the step kernel that fcb_advance_all_levels launches for
 * the current mesh (no counterpart in the reference; for roofline reports):
 * `launches` launches over the finest level's patches at (t, dt), on scratch
 * copies of the patch arrays (the solve's state is untouched), timed with
 * CUDA events on the context's stream.  *fused = 1 when that is the
 * ghost-exchange-fused step (ghost cells read from the neighbours), 0 for the
 * step alone (the ghost fill is a separate launch).  *ms_per_launch receives
 * the mean time of one launch.  Synchronises the stream. */
int fcb_step_kernel_time(fcb_context_t* ctx, double t, double dt, int launches, int* fused, double* ms_per_launch);
/* Floating-point issue rate of the current GPU (no counterpart in the
 * reference; for roofline reports): lane add/multiply operations per second in
 * FP64 (fp64 != 0) or FP32, from independent multiply-then-add chains on one
 * full wave of resident CTAs, best of five launches on cuda_stream.  Allocates
 * and frees a small result array. */
int fcb_measure_fp_rate(int fp64, void* cuda_stream, double* ops_per_second);
/* Wait for all work of the context. */
int fcb_synchronize(fcb_context_t* ctx);

/* ---- partitioned solves ------------------------------------------------------
 * Replaces the MPI layer under fclaw2d_domain_new_unitsquare(mpicomm, ...):
 * every rank holds the whole forest (leaf metadata only) and the patch arrays
 * of its Morton range of leaves (p4est_partition with weights 2^level when
 * weighted_partition and subcycle are set, complete families never split)
 * plus a ghost layer of the face and corner neighbours of those leaves.
 * Ghost updates exchange the ghost layer (fclaw2d_exchange.c:308-413) in two
 * steps: the sources' interiors before the averages and copies, and after
 * them the coarse patches (ghost cells included) that the interpolations read.
 * Refinement tags are gathered so every rank adapts the forest identically;
 * after a regrid the leaves are repartitioned and the patch data moves to its
 * new owners with the regrid transfer (fclaw2d_partition.c:113-197).  The
 * state of every owned patch is bit-identical to a one-rank solve.
 *
 * Collective calls (all ranks, same order): fcb_initialize, fcb_run,
 * fcb_advance_all_levels, fcb_ghost_update, fcb_regrid,
 * fcb_conservation_check, fcb_global_maximum, fcb_output_ascii.  fcb_advance_all_levels returns
 * this rank's CFL maximum, as fclaw2d_advance_all_levels does; fcb_run takes
 * the global maximum itself (fclaw2d_run.c:206).  fcb_get_q / fcb_set_q /
 * fcb_get_qinterp move only the owned patches, at their places in the
 * all-leaves layout.  fcb_output_ascii is collective: rank 0 writes the
 * header, then every rank appends its patches in rank order (mpi_rank in the
 * grid headers).  The macro-step graph is not used; time-sync is rejected.  A failed rank marks the communicator failed, and
 * the others' next collective returns FCB_ERR_COMM. */
typedef struct fcb_comm fcb_comm_t;
/* nranks communicators of one in-process group: each rank's context is driven
 * by its own host thread; every rendezvous waits at most timeout_s seconds */
int fcb_comm_create_local(int nranks, double timeout_s, fcb_comm_t** comms);
/* NCCL (nccl_library: path of libnccl.so.2, NULL for the default search):
 * the 128-byte unique id made on one rank and sent to the others by the
 * caller, and one rank's communicator (one process per GPU, the device current
 * at the call); every wait is bounded by timeout_s, then the communicator is aborted */
int fcb_comm_nccl_unique_id(const char* nccl_library, unsigned char id[128]);
int fcb_comm_create_nccl(const char* nccl_library, const unsigned char id[128], int rank, int nranks,
                         double timeout_s, fcb_comm_t** out);
int fcb_comm_destroy(fcb_comm_t* comm);
/* a context that is rank comm.rank of a partitioned solve (the context keeps
 * its own reference to the communicator) */
int fcb_context_create_partitioned(const fcb_options_t* opt, void* cuda_stream, fcb_comm_t* comm,
                                   fcb_context_t** out);
/* this rank, the number of ranks, and the owned leaves [first, first + count) */
int fcb_partition_info(fcb_context_t* ctx, int* rank, int* nranks, int* first, int* count);
/* fclaw2d_domain_global_maximum: the maximum of value over the ranks */
int fcb_global_maximum(fcb_context_t* ctx, double value, double* out);
/* Planning query, host only (no device call, works without a GPU): rank `rank`
 * of `nranks` over nleaves leaves in Morton order (level, and the lower-left
 * corner x, y in units of 2^-28 of the block), partitioned as a partitioned
 * solve does: the owned leaves [first, first + count), the size of the ghost
 * layer, and per peer rank (arrays of nranks) the patches the ghost update
 * (minlevel, maxlevel, time_interp) sends and receives in its first exchange
 * (x1, before the averages and copies) and second (x2, before the
 * interpolations).  Rank a's x?_send[b] equals rank b's x?_recv[a]. */
int fcb_partition_plan(const fcb_options_t* opt, int nranks, int rank, int nleaves, const int* level, const int* x,
                       const int* y, int minlevel, int maxlevel, int time_interp, int* first, int* count,
                       int* ghosts, int* x1_send, int* x1_recv, int* x2_send, int* x2_recv);

/* ---- ensemble serving -----------------------------------------------------
 * No counterpart in the reference (ForestClaw runs one solve per process): a
 * server admits independent solves as they arrive, keeps their arrays on the
 * device, and advances them together.  A served solve runs to tfinal in one
 * output interval (nout = 1), subcycled or not (subcycle), with the four-barrier
 * or pipelined step form; a round advances every active solve by one fine step
 * of its macro step (the level updates between two of its ghost updates), with
 * the patches of all solves that share solver, patch shape, method and
 * precision in ONE step launch, each patch carrying its own dt.  Queued solves are admitted in arrival order while
 * their device arrays fit in budget_bytes (one solve is always admitted when
 * none runs).  A served solve's result equals fcb_run on the same options bit
 * for bit.  Work is enqueued on cuda_stream (NULL: the legacy default stream). */
typedef struct fcb_server fcb_server_t;
enum fcb_request_state { FCB_REQ_QUEUED = 0, FCB_REQ_ACTIVE = 1, FCB_REQ_DONE = 2, FCB_REQ_FAILED = 3 };
typedef struct fcb_request_status {
    int state;                /* enum fcb_request_state */
    int num_patches;          /* current leaves (0 unless active or done) */
    double t;                 /* simulated time reached */
    double submit_s, start_s, finish_s;  /* server clock (seconds since creation) */
    long long cell_updates;   /* interior cells advanced, summed over fine steps */
    long long count_amr_advance;
} fcb_request_status_t;
int fcb_server_create(size_t budget_bytes, void* cuda_stream, fcb_server_t** out);
int fcb_server_destroy(fcb_server_t* s);
/* Queue a solve; *id receives its handle. */
int fcb_server_submit(fcb_server_t* s, const fcb_options_t* opt, int* id);
/* Admit what fits, enqueue one fine step of every running solve; reports the
 * active and queued counts after the round.  The call does not wait for the
 * GPU (each admitted solve runs on its own stream; the step launch goes to
 * cuda_stream); it blocks only when every active solve waits for the end of
 * its macro step to reach the host. */
int fcb_server_round(fcb_server_t* s, int* active, int* queued);
int fcb_server_status(fcb_server_t* s, int id, fcb_request_status_t* out);
/* Patch arrays of a finished (or running) solve, as fcb_get_q. */
int fcb_server_get_q(fcb_server_t* s, int id, double* host, size_t n);
/* Forget a finished, failed or queued solve and free its device arrays. */
int fcb_server_release(fcb_server_t* s, int id);
/* Work limit (no counterpart in the reference): admit the next queued solve
 * only while the cells of the admitted solves' meshes (patches x mx x my,
 * re-counted after every regrid) plus its own stay within max_cells; 0 (the
 * default) sets no limit.  Admission stays in arrival order; a solve that
 * waits for the limit keeps its initialised state and device arrays. */
int fcb_server_set_work_limit(fcb_server_t* s, long long max_cells);
/* Seconds on the server clock; rounds and step launches so far. */
int fcb_server_clock(fcb_server_t* s, double* now, long long* rounds, long long* launches);

#ifdef __cplusplus
}
#endif
#endif /* FCLAW_B200_H */
