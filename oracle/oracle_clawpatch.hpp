// ORACLE -- test infrastructure only (see oracle_patch.hpp).
//
// Restatement of the clawpatch 4.6 ghost-cell, time-interpolation, regrid
// transfer, tagging and conservation kernels for patches that live in one
// block (the single unit-square block of every configuration exercised here).
#pragma once
#include "oracle_patch.hpp"

namespace orc {

// The part of fclaw2d_patch_t the same-block transforms read
// (src/forestclaw2d.h:97-150): lower-left corner in block coordinates and level.
struct PatchGeom {
    double xlower, ylower;
    int level;
};

// Same-block branches of src/forestclaw2d.c:
//   fclaw2d_patch_transform_face   (:609-745, branch :655-663)
//   fclaw2d_patch_transform_face2  (:748-977, branch :798-841)
//   fclaw2d_patch_transform_corner (:1128-1236, not a block boundary)
//   fclaw2d_patch_transform_corner2(:1239-1384, not a block boundary)
// all with based = 1 (cell-centred Fortran indices).
struct Transform {
    PatchGeom self, nbr;
    int mx, my;
    void face(int i1, int j1, int& i2, int& j2) const;
    void face_half(int i1, int j1, int i2[4], int j2[4]) const;
    void corner(int i1, int j1, int& i2, int& j2) const;
    void corner_half(int i1, int j1, int i2[4], int j2[4]) const;
};

// fclaw2d_clawpatch_utils.f:76-169: A and F of T(i,j) = A (i,j) + F for the
// half-size (coarse to first fine index) and same-size transforms.
void build_transform_half(const Transform& t, int a[2][2], int f[2]);
void build_transform_same(const Transform& t, int a[2][2], int f[2]);

// fort_4.6/fclaw2d_clawpatch46_copy.f:17-86
void copy_face(int mx, int my, int mbc, int meqn, double* qthis, const double* qnbr, int iface,
               const Transform& t);
// fort_4.6/fclaw2d_clawpatch46_copy.f:95-133
void copy_corner(int mx, int my, int mbc, int meqn, double* qthis, const double* qnbr, int icorner,
                 const Transform& t);
// fort_4.6/fclaw2d_clawpatch46_average.f:16-176 (non-manifold)
void average_face(int mx, int my, int mbc, int meqn, double* qcoarse, const double* qfine, int idir,
                  int iface_coarse, const Transform& t);
// fort_4.6/fclaw2d_clawpatch46_average.f:186-272 (non-manifold)
void average_corner(int mx, int my, int mbc, int meqn, double* qcoarse, const double* qfine,
                    int icorner_coarse, const Transform& t);
// fort_4.6/fclaw2d_clawpatch46_interpolate.f:30-199
void interpolate_face(int mx, int my, int mbc, int meqn, const double* qcoarse, double* qfine,
                      int idir, int iface_coarse, const Transform& t);
// fort_4.6/fclaw2d_clawpatch46_interpolate.f:208-314
void interpolate_corner(int mx, int my, int mbc, int meqn, const double* qcoarse, double* qfine,
                        int icorner_coarse, const Transform& t);
// fort_4.6/fclaw2d_clawpatch46_timeinterp.f:11-78; returns ierror.
int timeinterp(int mx, int my, int mbc, int meqn, int psize, const double* qcurr,
               const double* qlast, double* qinterp, double alpha);
// fort_4.6/fclaw2d_clawpatch46_interpolate.f:324-400 (non-manifold)
void interpolate2fine(int mx, int my, int mbc, int meqn, const double* qcoarse, double* qfine,
                      int igrid);
// fort_4.6/fclaw2d_clawpatch46_average.f:282-364 (non-manifold)
void average2coarse(int mx, int my, int mbc, int meqn, double* qcoarse, const double* qfine,
                    int igrid);

enum TagCriteria { TAG_VALUE = 0, TAG_MINMAX = 1, TAG_DIFFERENCE = 2, TAG_GRADIENT = 3 };

// fort_4.6/fclaw2d_clawpatch46_tag4refinement.f + fort_user/*_exceeds_th.f90
int tag4refinement(int mx, int my, int mbc, int meqn, double dx, double dy, const double* q,
                   double threshold, int criteria, int ivar);
// fort_4.6/fclaw2d_clawpatch46_tag4coarsening.f (families of four siblings)
int tag4coarsening(int mx, int my, int mbc, int meqn, double dx, double dy, const double* q[4],
                   double threshold, int criteria, int ivar, int initflag);

// fort_4.6/fclaw2d_clawpatch46_diagnostics.f:13-58: Kahan sum of q*dx*dy over the interior.
void conservation_sum(int mx, int my, int mbc, int meqn, double dx, double dy, const double* q,
                      double* sum, double* c_kahan);

}  // namespace orc
