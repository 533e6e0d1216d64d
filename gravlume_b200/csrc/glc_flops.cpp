// Algorithmic operation counts of the trace kernel, taken by running the same templated device
// source (kn_rhs, dp5_attempt) on the host with a counting scalar. The counts back the roofline
// reported next to the measured throughput: FMA counts 2 flops, add/sub/mul 1, and the special
// functions (reciprocal, square root, reciprocal square root) are reported separately.
#include <cmath>
#include <cstdint>

#include "glc_dp54.cuh"
#include "glc_internal.h"

namespace {

struct Counts {
  uint64_t add = 0, mul = 0, special = 0, cmp = 0;
};
thread_local Counts g_counts;

struct CF {
  double v;
  CF() : v(0) {}
  CF(double x) : v(x) {}  // NOLINT: implicit from literals, like float
  explicit operator double() const { return v; }
};
inline CF operator+(CF a, CF b) { ++g_counts.add; return CF(a.v + b.v); }
inline CF operator-(CF a, CF b) { ++g_counts.add; return CF(a.v - b.v); }
inline CF operator*(CF a, CF b) { ++g_counts.mul; return CF(a.v * b.v); }
inline CF operator/(CF a, CF b) { ++g_counts.special; ++g_counts.mul; return CF(a.v / b.v); }
inline CF operator-(CF a) { return CF(-a.v); }
inline CF& operator+=(CF& a, CF b) { a = a + b; return a; }
inline bool operator>=(CF a, CF b) { ++g_counts.cmp; return a.v >= b.v; }
inline bool operator>(CF a, CF b) { ++g_counts.cmp; return a.v > b.v; }
inline bool operator<(CF a, CF b) { ++g_counts.cmp; return a.v < b.v; }
inline bool operator<=(CF a, CF b) { ++g_counts.cmp; return a.v <= b.v; }
inline bool operator==(CF a, CF b) { return a.v == b.v; }
// found by argument-dependent lookup from the templated device source
inline CF g_rsqrt(CF x) { ++g_counts.special; return CF(1.0 / std::sqrt(x.v)); }
inline CF g_rcp(CF x) { ++g_counts.special; return CF(1.0 / x.v); }
inline CF g_sqrt(CF x) { ++g_counts.special; return CF(std::sqrt(x.v)); }
inline CF g_abs(CF x) { return CF(std::fabs(x.v)); }
inline CF g_max(CF a, CF b) { ++g_counts.cmp; return CF(std::fmax(a.v, b.v)); }
inline CF g_min(CF a, CF b) { ++g_counts.cmp; return CF(std::fmin(a.v, b.v)); }
inline bool g_finite(CF x) { return std::isfinite(x.v); }

}  // namespace

namespace glc {

// flops[0] = flops per right-hand-side evaluation (FMA = 2: a multiply feeding an add counts as
// one FMA), flops[1] = special-function ops per evaluation, flops[2] = flops per attempted step
// including its six evaluations, flops[3] = special-function ops per attempted step.
void flop_model(double out[4]) {
  KN<CF> k{CF(0.9), CF(0.81), CF(-1.0), CF(-0.9), CF(0.09)};
  CF y[6] = {CF(30.0), CF(1.0), CF(8.0), CF(-0.9), CF(0.1), CF(-0.2)};
  CF d[7], r, vr;
  g_counts = Counts{};
  kn_rhs(k, y, CF(1.0), d, r, vr);
  const Counts one = g_counts;
  // adds and multiplies pair into FMAs wherever a product feeds a sum: count min(add, mul) FMAs
  auto flops = [](const Counts& c) {
    const uint64_t fma = c.add < c.mul ? c.add : c.mul;
    return double(2 * fma + (c.add - fma) + (c.mul - fma));
  };
  out[0] = flops(one);
  out[1] = double(one.special);
  CF k1[7] = {CF(-0.9), CF(0.1), CF(-0.2), CF(0.01), CF(0.0), CF(0.001), CF(1.1)};
  CF inc[6], dt, k7[7];
  Invariants<CF> inv;
  bool finite;
  const Tolerance tol{1e-6, 1e-8, 1e-6, 1e-8};
  g_counts = Counts{};
  dp5_attempt<CF, CF>(k, y, CF(1.0), CF(0.5), k1, CF(3.0), tol, inc, dt, k7, r, vr, inv, finite);
  const Counts step = g_counts;
  // the attempt includes the embedded error norm and the end-point invariants; the controller's
  // power and the state update add ~2 special ops and ~10 flops
  out[2] = flops(step) + 10.0;
  out[3] = double(step.special) + 2.0;
}

}  // namespace glc
