// ORACLE -- test infrastructure only.
//
// Instrumented build of the CPU restatement: oracle_patch.cpp compiled with its
// FP64 type replaced by a counting wrapper, which counts one operation per
// floating-point add/subtract, multiply, divide, square root and
// compare/select (relational operators, min, max, abs, sign tests), and the
// transcendental calls (sin, cos, exp, atan) apart.  Negation is a sign-bit
// flip and is not counted.  The counts are the algorithmic FP64 operations
// per interior cell update of the reference's patch step (clawpack46_step2_wrap
// + step2 + flux2 with the reference's loop ranges, ghost-region work
// included), for the FP64-pipe roofline beside the HBM one.
//
// Inputs are seeded and dense (every wave nonzero, so every limiter and
// transverse branch is taken): the counts are the per-(solver, order, mx)
// constants of the method, not of one solution.
//
// Build and run:  make -C oracle flopcount && oracle/flopcount
// Prints one JSON object per case.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

namespace fcnt {
struct Ops {
    long long add = 0, mul = 0, div = 0, sqrt = 0, cmp = 0, trans = 0;
    long long total() const { return add + mul + div + sqrt + cmp; }
};
inline Ops g;

struct CD {
    double v;
    CD() = default;
    CD(double x) : v(x) {}
    CD operator-() const { return CD(-v); }
    CD operator+() const { return *this; }
    CD& operator+=(CD b) { ++g.add; v += b.v; return *this; }
    CD& operator-=(CD b) { ++g.add; v -= b.v; return *this; }
    CD& operator*=(CD b) { ++g.mul; v *= b.v; return *this; }
    CD& operator/=(CD b) { ++g.div; v /= b.v; return *this; }
};
inline CD operator+(CD a, CD b) { ++g.add; return CD(a.v + b.v); }
inline CD operator-(CD a, CD b) { ++g.add; return CD(a.v - b.v); }
inline CD operator*(CD a, CD b) { ++g.mul; return CD(a.v * b.v); }
inline CD operator/(CD a, CD b) { ++g.div; return CD(a.v / b.v); }
inline bool operator<(CD a, CD b) { ++g.cmp; return a.v < b.v; }
inline bool operator>(CD a, CD b) { ++g.cmp; return a.v > b.v; }
inline bool operator<=(CD a, CD b) { ++g.cmp; return a.v <= b.v; }
inline bool operator>=(CD a, CD b) { ++g.cmp; return a.v >= b.v; }
inline bool operator==(CD a, CD b) { ++g.cmp; return a.v == b.v; }
inline bool operator!=(CD a, CD b) { ++g.cmp; return a.v != b.v; }
}  // namespace fcnt

namespace std {
inline fcnt::CD max(fcnt::CD a, fcnt::CD b) { return (a < b) ? b : a; }
inline fcnt::CD min(fcnt::CD a, fcnt::CD b) { return (b < a) ? b : a; }
inline fcnt::CD fabs(fcnt::CD a) { ++fcnt::g.cmp; return fcnt::CD(std::fabs(a.v)); }
inline bool signbit(fcnt::CD a) { ++fcnt::g.cmp; return std::signbit(a.v); }
inline fcnt::CD sqrt(fcnt::CD a) { ++fcnt::g.sqrt; return fcnt::CD(std::sqrt(a.v)); }
inline fcnt::CD sin(fcnt::CD a) { ++fcnt::g.trans; return fcnt::CD(std::sin(a.v)); }
inline fcnt::CD cos(fcnt::CD a) { ++fcnt::g.trans; return fcnt::CD(std::cos(a.v)); }
inline fcnt::CD exp(fcnt::CD a) { ++fcnt::g.trans; return fcnt::CD(std::exp(a.v)); }
inline fcnt::CD atan(fcnt::CD a) { ++fcnt::g.trans; return fcnt::CD(std::atan(a.v)); }
}  // namespace std

#define double fcnt::CD
#include "oracle_patch.hpp"
#include "oracle_patch.cpp"
#undef double

namespace {

using fcnt::CD;

struct Case {
    std::string name;
    int kind, mx, meqn, maux, mwaves, order0, order1, version;
};

void emit(const Case& c, const fcnt::Ops& o, const fcnt::Ops& aux, int cells) {
    const double n = (double)cells;
    std::printf("{\"case\": \"%s\", \"mx\": %d, \"claw_version\": %d, \"ops_per_cell\": %.4f, \"add\": %.4f, "
                "\"mul\": %.4f, \"div\": %.4f, \"sqrt\": %.4f, \"cmp\": %.4f, \"transcendental\": %.4f, "
                "\"aux_ops_per_cell\": %.4f, \"aux_transcendental_per_cell\": %.4f}\n",
                c.name.c_str(), c.mx, c.version, o.total() / n, o.add / n, o.mul / n, o.div / n, o.sqrt / n,
                o.cmp / n, o.trans / n, aux.total() / n, aux.trans / n);
}

void run(const Case& c, std::mt19937_64& rng) {
    const int mx = c.mx, my = c.mx, mbc = 2;
    const orc::PatchIdx P(mx, my, mbc);
    const double dx = 1.0 / 256, dy = dx, xlower = 0.25, ylower = 0.5;
    std::uniform_real_distribution<double> U(0.0, 1.0);
    std::vector<CD> q((size_t)P.size(c.meqn)), aux((size_t)P.size(std::max(c.maux, 1)));
    orc::SolverParams sp;
    sp.kind = c.kind;
    sp.grav = 1.0;
    sp.gamma = 1.4;
    sp.gamma1 = 0.4;
    orc::MethodParams mp;
    mp.order0 = c.order0;
    mp.order1 = c.order1;
    mp.mwaves = c.mwaves;
    mp.version = c.version;
    fcnt::Ops aux_ops;
    for (int j = 1 - mbc; j <= my + mbc; ++j)
        for (int i = 1 - mbc; i <= mx + mbc; ++i) {
            if (c.kind == orc::SOLVER_ADVECTION) {
                q[P(i, j, 0)] = U(rng);
            } else if (c.kind == orc::SOLVER_SWE_ROE) {
                q[P(i, j, 0)] = 1.0 + U(rng);
                q[P(i, j, 1)] = 0.4 * (U(rng) - 0.5);
                q[P(i, j, 2)] = 0.4 * (U(rng) - 0.5);
            } else if (c.kind == orc::SOLVER_EULER4_ROE) {
                const double rho = 1.0 + 0.5 * U(rng), u = 0.6 * (U(rng) - 0.5), v = 0.6 * (U(rng) - 0.5);
                const double p = 1.0 + 0.5 * U(rng);
                q[P(i, j, 0)] = rho;
                q[P(i, j, 1)] = rho * u;
                q[P(i, j, 2)] = rho * v;
                q[P(i, j, 3)] = p / 0.4 + 0.5 * rho * (u * u + v * v);
            }
        }
    if (c.kind == orc::SOLVER_ADVECTION) {
        fcnt::g = fcnt::Ops{};
        orc::b4step2_swirl(mx, my, mbc, c.maux, xlower, ylower, dx, dy, 0.1, 0.9 * dx, 1.0, aux.data());
        aux_ops = fcnt::g;
    } else if (c.kind == orc::SOLVER_GEOCLAW_FWAVE) {
        orc::setaux_bathy(mx, my, mbc, xlower, ylower, dx, dy, aux.data());
        for (int j = 1 - mbc; j <= my + mbc; ++j)
            for (int i = 1 - mbc; i <= mx + mbc; ++i) {
                const double b = aux[P(i, j, 0)].v;
                q[P(i, j, 0)] = 1e-3 * U(rng) - b;
                q[P(i, j, 1)] = 1e-3 * (U(rng) - 0.5);
                q[P(i, j, 2)] = 1e-3 * (U(rng) - 0.5);
            }
    }
    fcnt::g = fcnt::Ops{};
    orc::step2(sp, mp, mx, my, mbc, c.meqn, c.maux, q.data(), aux.data(), dx, dy, 0.2 * dx);
    emit(c, fcnt::g, aux_ops, mx * my);
}

}  // namespace

int main() {
    std::mt19937_64 rng(20241203);
    std::vector<Case> cases;
    for (int mx : {8, 16, 32}) cases.push_back({"advection_swirl_order22", orc::SOLVER_ADVECTION, mx, 1, 2, 1, 2, 2, 4});
    cases.push_back({"advection_swirl_order22", orc::SOLVER_ADVECTION, 16, 1, 2, 1, 2, 2, 5});
    for (int mx : {16, 32}) cases.push_back({"swe_roe_order22", orc::SOLVER_SWE_ROE, mx, 3, 0, 3, 2, 2, 4});
    for (int mx : {8, 16, 32, 64})
        cases.push_back({"euler4_roe_order22", orc::SOLVER_EULER4_ROE, mx, 4, 0, 4, 2, 2, 4});
    cases.push_back({"geoclaw_fwave_order20", orc::SOLVER_GEOCLAW_FWAVE, 32, 3, 1, 3, 2, 0, 4});
    for (const Case& c : cases) run(c, rng);
    return 0;
}
