// ASCII output frames in the reference's format (fort.tNNNN / fort.qNNNN):
// src/patches/clawpatch/fclaw2d_clawpatch_output_ascii.c with
// fort_4.6/fclaw2d_clawpatch46_output_ascii.f (fclaw2d_clawpatch46_fort_header_ascii,
// _fort_output_ascii, _fort_write_grid_header).  Numbers follow the Fortran
// edit descriptors of those routines: Ew.d ("0.d1..dd" mantissa, two-digit
// exponent "E+xx", three-digit exponent without the E), Iw right-justified,
// list-directed ' ' as a record of two blanks.
#include "fcb_output.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>

namespace fcb {

std::string fortran_e(double x, int w, int d) {
    std::string body;
    if (std::isnan(x)) {
        body = "NaN";
    } else if (std::isinf(x)) {
        body = x < 0 ? "-Infinity" : "Infinity";
    } else {
        const bool neg = std::signbit(x) && x != 0.0;
        char digits[64];
        int e10 = 0;
        if (x == 0.0) {
            std::memset(digits, '0', (size_t)d);
            digits[d] = 0;
        } else {
            // d significant digits, correctly rounded: D.DDD...E+XX
            char buf[64];
            std::snprintf(buf, sizeof buf, "%.*E", d - 1, std::fabs(x));
            int k = 0;
            for (const char* c = buf; *c && *c != 'E'; ++c)
                if (*c != '.') digits[k++] = *c;
            digits[k] = 0;
            e10 = std::atoi(std::strchr(buf, 'E') + 1) + 1;  // 0.D... scaling
        }
        char ex[8];
        if (std::abs(e10) <= 99) std::snprintf(ex, sizeof ex, "E%c%02d", e10 < 0 ? '-' : '+', std::abs(e10));
        else std::snprintf(ex, sizeof ex, "%c%03d", e10 < 0 ? '-' : '+', std::abs(e10));
        body = std::string(neg ? "-" : "") + "0." + digits + ex;
    }
    if ((int)body.size() > w) return std::string((size_t)w, '*');
    return std::string((size_t)(w - (int)body.size()), ' ') + body;
}

namespace {
std::string fortran_i(long v, int w) {
    char buf[32];
    std::snprintf(buf, sizeof buf, "%*ld", w, v);
    std::string s(buf);
    if ((int)s.size() > w) return std::string((size_t)w, '*');
    return s;
}

FILE* open_or_throw(const std::string& path, const char* mode) {
    FILE* f = std::fopen(path.c_str(), mode);
    if (!f) throw std::runtime_error("cannot open " + path);
    return f;
}
}  // namespace

void write_ascii_header(const std::string& dir, int iframe, double time, int meqn, int maux, long ngrids) {
    char name[32];
    const std::string base = dir.empty() ? std::string(".") : dir;
    // fclaw2d_clawpatch46_fort_header_ascii: fort.t, and an empty fort.q
    std::snprintf(name, sizeof name, "fort.t%04d", iframe);
    FILE* ft = open_or_throw(base + "/" + name, "w");
    std::fprintf(ft, "%s    time\n", fortran_e(time, 30, 20).c_str());
    std::fprintf(ft, "%s                 meqn\n", fortran_i(meqn, 5).c_str());
    std::fprintf(ft, "%s                 ngrids\n", fortran_i(ngrids, 5).c_str());
    std::fprintf(ft, "%s                 num_aux\n", fortran_i(maux, 5).c_str());
    std::fprintf(ft, "%s                 num_dim\n", fortran_i(2, 5).c_str());
    std::fclose(ft);
    std::snprintf(name, sizeof name, "fort.q%04d", iframe);
    std::fclose(open_or_throw(base + "/" + name, "w"));
}

void write_ascii_frame(const std::string& dir, int iframe, double time, int meqn, int maux, int mx, int my, int mbc,
                       const std::vector<OutputPatch>& patches, const double* q, size_t patch_size) {
    write_ascii_header(dir, iframe, time, meqn, maux, (long)patches.size());
    append_ascii_patches(dir, iframe, meqn, mx, my, mbc, patches, q, patch_size, 0);
}

void append_ascii_patches(const std::string& dir, int iframe, int meqn, int mx, int my, int mbc,
                          const std::vector<OutputPatch>& patches, const double* q, size_t patch_size, int mpi_rank) {
    char name[32];
    const std::string base = dir.empty() ? std::string(".") : dir;
    std::snprintf(name, sizeof name, "fort.q%04d", iframe);
    FILE* fq = open_or_throw(base + "/" + name, "a");
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc;
    std::string line;
    for (size_t p = 0; p < patches.size(); ++p) {
        const OutputPatch& P = patches[p];
        // fclaw2d_clawpatch46_fort_write_grid_header
        std::fprintf(fq, "%s                 grid_number\n", fortran_i(P.global_num, 5).c_str());
        std::fprintf(fq, "%s                 AMR_level\n", fortran_i(P.level, 5).c_str());
        std::fprintf(fq, "%s                 block_number\n", fortran_i(P.block, 5).c_str());
        std::fprintf(fq, "%s                 mpi_rank\n", fortran_i(mpi_rank, 5).c_str());
        std::fprintf(fq, "%s                 mx\n", fortran_i(mx, 5).c_str());
        std::fprintf(fq, "%s                 my\n", fortran_i(my, 5).c_str());
        std::fprintf(fq, "%s    xlow\n", fortran_e(P.xlower, 24, 16).c_str());
        std::fprintf(fq, "%s    ylow\n", fortran_e(P.ylower, 24, 16).c_str());
        std::fprintf(fq, "%s    dx\n", fortran_e(P.dx, 24, 16).c_str());
        std::fprintf(fq, "%s    dy\n\n", fortran_e(P.dy, 24, 16).c_str());
        const double* qp = q + p * patch_size;
        for (int j = 1; j <= my; ++j) {
            for (int i = 1; i <= mx; ++i) {
                line.clear();
                for (int m = 0; m < meqn; ++m) {
                    double v = qp[((size_t)m * ny + (j + mbc - 1)) * nx + (i + mbc - 1)];
                    if (std::fabs(v) < 1e-99) v = 0.0;  // the reference zeroes tiny values
                    line += fortran_e(v, 26, 16);
                }
                std::fprintf(fq, "%s\n", line.c_str());
            }
            std::fprintf(fq, "  \n");  // write(matunit1,*) ' '
        }
    }
    std::fclose(fq);
}

}  // namespace fcb
