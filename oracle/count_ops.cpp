// count_ops.cpp -- op-counting build of the FP64 oracle.
//
// TEST INFRASTRUCTURE ONLY: run by oracle/count_ops.py to tally the
// arithmetic of one reference step; the product library never links it.
//
// The oracle restatement (imhd_oracle.hpp: vanleer_mod.f90:279-3334,
// passive_mod.f90:118-627, turb_driver_mod.f90:130-192, 395-457) is compiled
// with every `double` replaced by Counted, a double whose operators add to a
// global tally: additions and subtractions, multiplications, divisions,
// square roots, comparisons (the reference's MAX/MIN expand to them, as do its
// limiter and upwind tests), ABS and SIGN.  Unary minus, copies and integer
// index arithmetic are not counted.  The values are computed exactly as the
// plain oracle computes them (same order, same IEEE operations), so the
// tallies follow the same branches.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <thread>
#include <vector>

namespace opcount {

struct Tally {
    unsigned long long add = 0, mul = 0, div = 0, sqrt = 0, cmp = 0, abs = 0, sign = 0, transc = 0;
};
inline Tally g_tally;

struct Counted {
    double v;
    constexpr Counted() : v(0.0) {}
    constexpr Counted(double x) : v(x) {}
    Counted& operator+=(Counted o) { ++g_tally.add; v += o.v; return *this; }
    Counted& operator-=(Counted o) { ++g_tally.add; v -= o.v; return *this; }
    Counted& operator*=(Counted o) { ++g_tally.mul; v *= o.v; return *this; }
    Counted& operator/=(Counted o) { ++g_tally.div; v /= o.v; return *this; }
    Counted operator-() const { return Counted(-v); }
    Counted operator+() const { return *this; }
};
inline Counted operator+(Counted a, Counted b) { ++g_tally.add; return Counted(a.v + b.v); }
inline Counted operator-(Counted a, Counted b) { ++g_tally.add; return Counted(a.v - b.v); }
inline Counted operator*(Counted a, Counted b) { ++g_tally.mul; return Counted(a.v * b.v); }
inline Counted operator/(Counted a, Counted b) { ++g_tally.div; return Counted(a.v / b.v); }
inline bool operator<(Counted a, Counted b) { ++g_tally.cmp; return a.v < b.v; }
inline bool operator>(Counted a, Counted b) { ++g_tally.cmp; return a.v > b.v; }
inline bool operator<=(Counted a, Counted b) { ++g_tally.cmp; return a.v <= b.v; }
inline bool operator>=(Counted a, Counted b) { ++g_tally.cmp; return a.v >= b.v; }
inline bool operator==(Counted a, Counted b) { ++g_tally.cmp; return a.v == b.v; }
inline bool operator!=(Counted a, Counted b) { ++g_tally.cmp; return a.v != b.v; }

}  // namespace opcount

namespace std {
inline opcount::Counted sqrt(opcount::Counted a) { ++opcount::g_tally.sqrt; return opcount::Counted(std::sqrt(a.v)); }
inline opcount::Counted fabs(opcount::Counted a) { ++opcount::g_tally.abs; return opcount::Counted(std::fabs(a.v)); }
inline opcount::Counted copysign(opcount::Counted a, opcount::Counted b) {
    ++opcount::g_tally.sign;
    return opcount::Counted(std::copysign(a.v, b.v));
}
inline opcount::Counted exp(opcount::Counted a) { ++opcount::g_tally.transc; return opcount::Counted(std::exp(a.v)); }
inline opcount::Counted log(opcount::Counted a) { ++opcount::g_tally.transc; return opcount::Counted(std::log(a.v)); }
inline opcount::Counted sin(opcount::Counted a) { ++opcount::g_tally.transc; return opcount::Counted(std::sin(a.v)); }
inline opcount::Counted cos(opcount::Counted a) { ++opcount::g_tally.transc; return opcount::Counted(std::cos(a.v)); }
inline opcount::Counted atan(opcount::Counted a) { ++opcount::g_tally.transc; return opcount::Counted(std::atan(a.v)); }
}  // namespace std

using opcount::Counted;
#define double Counted
#include "imhd_oracle.hpp"
#undef double

using imhd_oracle::Config;
using imhd_oracle::Solver;

extern "C" {

// Same layout and meaning as oracle_create / oracle_set_state in
// imhd_oracle_capi.cpp; one host thread (the tally is not synchronised).
void* ops_create(int nx, int ny, int nz, int riemann, int recon, int npass, double sound_speed) {
    Config c;
    c.nx = nx; c.ny = ny; c.nz = nz;
    c.riemann = riemann; c.ppm = recon & 1; c.prim = (recon >> 1) & 1; c.protect = (recon >> 2) & 1;
    c.npass = npass;
    c.sound_speed = sound_speed; c.nthreads = 1;
    c.nb = 6;
    if (nx < 2 * c.nb || ny < 2 * c.nb || nz < 2 * c.nb) return nullptr;
    return new Solver(c);
}

void ops_destroy(void* h) { delete static_cast<Solver*>(h); }

void ops_set_state(void* h, const double* q, const double* bface, const double* qpass) {
    auto* s = static_cast<Solver*>(h);
    long n = (long)s->nx * s->ny * s->nz;
    for (long k = 0; k < s->nz; ++k)
        for (long j = 0; j < s->ny; ++j)
            for (long i = 0; i < s->nx; ++i) {
                long c = i + s->nx * (j + s->ny * k);
                for (int v = 1; v <= 7; ++v) s->q(i + 1, j + 1, k + 1, v) = q[(v - 1) * n + c];
                for (int v = 1; v <= 3; ++v) s->bface(i + 1, j + 1, k + 1, v) = bface[(v - 1) * n + c];
                for (int v = 1; v <= s->cfg.npass; ++v) s->qpass(i + 1, j + 1, k + 1, v) = qpass[(v - 1) * n + c];
            }
    s->boundary_conditions();
}

// One undriven step of the reference driver loop; out[0..7] receive the
// step's tallies {add, mul, div, sqrt, cmp, abs, sign, transcendental}; the
// return value is cmax (dt = COUR*dx/cmax for the next step).
double ops_step(void* h, double dt, double* out) {
    auto* s = static_cast<Solver*>(h);
    opcount::g_tally = opcount::Tally{};
    double cmax = s->step(Counted(dt), false).v;
    const opcount::Tally& t = opcount::g_tally;
    const unsigned long long v[8] = {t.add, t.mul, t.div, t.sqrt, t.cmp, t.abs, t.sign, t.transc};
    for (int i = 0; i < 8; ++i) out[i] = (double)v[i];
    return cmax;
}

double ops_dx(void* h) { return static_cast<Solver*>(h)->dx.v; }

}  // extern "C"
