// ASCII output frames in the reference's fort.tNNNN / fort.qNNNN format (fcb_output.cpp).
#pragma once
#include <cstddef>
#include <string>
#include <vector>

namespace fcb {

struct OutputPatch {
    int global_num, level;
    double xlower, ylower, dx, dy;  // physical lower-left corner and spacing
    int block = 0;  // block of a brick (fclaw2d's blockno), 0 on one block
};

// Fortran Ew.d edit descriptor (gfortran form: "0.d1..dd", exponent E+xx or +xxx)
std::string fortran_e(double x, int w, int d);

// Writes dir/fort.tNNNN and dir/fort.qNNNN; q holds the patches in order,
// patch_size doubles apart, each in the clawpack 4.6 layout q(i,j,m) with ghosts.
void write_ascii_frame(const std::string& dir, int iframe, double time, int meqn, int maux, int mx, int my, int mbc,
                       const std::vector<OutputPatch>& patches, const double* q, size_t patch_size);
// The two halves of a frame, as the ranks of a partitioned solve write it
// (fclaw2d_clawpatch_output_ascii): rank 0 writes fort.tNNNN and starts an
// empty fort.qNNNN, then every rank in turn appends its patches.
void write_ascii_header(const std::string& dir, int iframe, double time, int meqn, int maux, long ngrids);
void append_ascii_patches(const std::string& dir, int iframe, int meqn, int mx, int my, int mbc,
                          const std::vector<OutputPatch>& patches, const double* q, size_t patch_size, int mpi_rank);

}  // namespace fcb
