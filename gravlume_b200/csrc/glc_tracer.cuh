// Per-ray adaptive DP5(4) trace: one ray's state machine, shared by the one-thread-per-ray kernel
// and the persistent work-queue kernel.
//
// Semantics follow the reference's binary64 oracle loop (crates/gravlume-reference/src/geodesic.rs
// TraceExecution::run 129-212): accept/reject with the grouped infinity norm and the
// 0.9 * err^(-1/5) controller clamped to [0.2, 5] (policy.rs:137-173); relative coordinate time in
// the time error component (geodesic.rs:158-165); event arming (530-573), sign-change detection
// (702-708), bisection on the dense output to the affine tolerance (640-676), earliest event with
// tie candidates (722-740); radial turning points and equatorial crossings (330-383); azimuth
// winding (406-418); invariant drifts (575-598); escape direction (480-497); the Keplerian surface
// observable (surface.rs:75-146).
//
// Precision modes: S = storage type of the state accumulators, C = type of the right-hand side
// and stage combinations, T = S for the rare event path (root finding, observables).
//   FP32:  S = C = float.   FP64: S = C = double.
//   MIXED: S = double, C = float; a warp whose lanes are inside the shell r < shell radius steps
//          in double; the event path and the final null-constraint renormalisation are double.
//   MIXED as two kernels (the frame path): BULK steps in binary32 with the compensated pair state
//          (S = C = float) and leaves a ray at its first step that brackets a terminal event or
//          crosses the surface near or on it, or when it enters the shell; TAIL (S = C = double)
//          resumes the ray from its hand-off record, re-takes that step, and finishes the trace
//          in binary64 (event root-finding, shell steps, observables and the null-constraint
//          renormalisation). BULK counts crossings and turnings without roots where no event
//          root shares the step, and takes a pericentre's radius from the radial potential.
// In every mode, a step with no event root counts its equatorial crossing and an apocentre from
// the sign changes alone (their roots always exist on the dense output), and a surface crossing
// whose end radii both lie clear of the surface's radial interval is a miss without a root.
#pragma once

#include <cfloat>
#include <type_traits>

// Form of the DP5(4) attempt: 0 fully unrolled stages; 1 one rolled loop over a stage array (local
// memory); 2 streaming stage sums in registers around a rolled loop (dp5_attempt_stream). The
// kernels are bound by instruction fetch, so the small footprint of form 2 wins: 3840x2160 frames
// measured 144 -> 173 Mrays/s (binary32), 76 -> 92 (mixed), 133 -> 157 (binary64 at rtol 1e-6).
#ifndef GLC_ATTEMPT_FORM
#define GLC_ATTEMPT_FORM 2
#endif

#include "glc_dp54.cuh"
#include "glc_radiation.cuh"
#include "../../include/glc.h"

namespace glc {

enum Prec : int { kFP32 = 0, kMIXED = 1, kFP64 = 2, kBULK = 3, kTAIL = 4 };

template <int P>
struct PrecTraits;
template <>
struct PrecTraits<kFP32> {
  using S = float;
  using C = float;
};
template <>
struct PrecTraits<kMIXED> {
  using S = double;
  using C = float;
};
template <>
struct PrecTraits<kFP64> {
  using S = double;
  using C = double;
};
template <>
struct PrecTraits<kBULK> {
  using S = float;
  using C = float;
};
template <>
struct PrecTraits<kTAIL> {
  using S = double;
  using C = double;
};

// BULK hands a surface crossing to TAIL when its binary32 root radius lies within this relative
// margin of the surface's radial interval, so that TAIL's binary64 root decides hits near the edges.
constexpr double kBulkSurfaceMargin = 1e-4;
// A surface crossing whose step keeps the sign of its radial velocity, and whose end radii both lie
// outside the surface's radial interval widened by this relative margin (on the same side), misses
// the surface: it is decided without its root, in every precision.
constexpr double kSurfaceMissMargin = 1e-4;
// BULK localizes its non-terminal roots (pericentres, for the turning radius, and surface crossings
// near the surface) to at least this affine tolerance: binary32 cannot resolve the binary64
// presets' 2e-11.
constexpr double kBulkRootTolerance = 1e-6;

enum EventBit : uint32_t { kEvGuard = 0, kEvHorizon = 1, kEvSurface = 2, kEvEscape = 3 };

enum FlagBit : uint32_t {
  kFlagShellF64 = 1u << 0,     // MIXED: some steps ran in binary64
  kFlagRenormalized = 1u << 1, // MIXED: final momentum renormalized onto H = 0
  kFlagSurfaceInvalid = 1u << 2,  // surface hit but the circular emitter observable is undefined
  kFlagNoEscapeDirection = 1u << 3,
  kFlagCertified = 1u << 4,       // horizon capture proven by the tile's interval certificate
  kFlagReconstructed = 1u << 5,   // escape direction reconstructed from the escape-direction map
};

struct CompSum {
  template <class S>
  GLC_HD static void add(S& sum, S& corr, S v) {
    const S next = sum + v;
    corr += g_abs(sum) >= g_abs(v) ? (sum - next) + v : (v - next) + sum;
    sum = next;
  }
};

template <class S>
GLC_HD S wrapped_angle(S current, S previous) {
  const S pi = S(3.14159265358979323846);
  const S tau = S(6.28318530717958647692);
  S v = current - previous + pi;
  v = v - tau * g_floor(v / tau);
  return v - pi;
}

// Scene constants a lane needs for stepping and events (binary64 source, cast per use).
struct LaneScene {
  KN<double> kn;
  double horizon_r;   // horizon event radius (r_+ + offset), < 0 when absent
  double escape_r;    // 0 when absent
  double surf_in, surf_out;
  double shell_r;     // MIXED binary64 shell radius
  double frequency;
  uint32_t installed; // event bits installed
  // the packed scene, for the surface-transport constants: the result writer reads them after
  // the stepping loop, so that they do not occupy registers through it
  const glc_scene* src;
  // evaluate L_z, Carter's constant and the null residual at every accepted step for the drift
  // maxima; off when no drift output is wanted (they do not steer the integration)
  bool track;
};

GLC_HD LaneScene make_lane_scene(const glc_scene& s, double shell_factor, bool track = true) {
  LaneScene ls;
  ls.track = track;
  ls.kn.a = s.spin;
  ls.kn.a2 = s.spin * s.spin;
  ls.kn.s = s.chart_sign;
  ls.kn.sa = s.chart_sign * s.spin;
  ls.kn.q2 = s.charge * s.charge;
  ls.horizon_r = s.has_horizon ? s.horizon_event_radius : -1.0;
  ls.escape_r = s.has_escape ? s.escape_radius : 0.0;
  ls.surf_in = s.surface_inner;
  ls.surf_out = s.surface_outer;
  ls.shell_r = shell_factor * s.photon_shell_radius;
  ls.frequency = s.frequency;
  ls.src = &s;
  ls.installed = (1u << kEvGuard) | (s.has_horizon ? 1u << kEvHorizon : 0u) | (s.has_surface ? 1u << kEvSurface : 0u) |
                 (s.has_escape ? 1u << kEvEscape : 0u);
  return ls;
}

template <class T>
GLC_HD T event_value(int kind, const LaneScene& sc, double guard, T r, T z) {
  switch (kind) {
    case kEvGuard: {
      const T r2 = r * r;
      return r2 * r2 + T(sc.kn.a2) * z * z - T(guard);
    }
    case kEvHorizon: return r - T(sc.horizon_r);
    case kEvSurface: return z;
    default: return r - T(sc.escape_r);
  }
}

template <class T>
GLC_HD bool event_clears_band(int kind, T v, T band) {
  switch (kind) {
    case kEvGuard:
    case kEvHorizon: return v > band;
    case kEvSurface: return g_abs(v) > band;
    default: return v < -band;
  }
}

template <class T>
GLC_HD bool event_crosses(int kind, T s, T e) {
  switch (kind) {
    case kEvGuard:
    case kEvHorizon: return s > T(0) && e <= T(0);
    case kEvSurface: return (s < T(0) && e >= T(0)) || (s > T(0) && e <= T(0));
    default: return s < T(0) && e >= T(0);
  }
}

GLC_HD double event_scale(int kind, const LaneScene& sc) {
  switch (kind) {
    case kEvGuard: return 1.0;
    case kEvHorizon: return sc.horizon_r > 1.0 ? sc.horizon_r : 1.0;
    case kEvSurface: return 1.0;
    default: return sc.escape_r > 1.0 ? sc.escape_r : 1.0;
  }
}

// Earliest of n localized event roots (geodesic.rs:722-740): the smallest step fraction, the
// first in kind order (guard, horizon, surface, escape) on equal fractions, and as candidate bits
// every kind whose root lies within `tie` affine distance of it. Returns its index, -1 when n = 0.
template <class T>
GLC_HD int earliest_event(const int kinds[4], const T thetas[4], int n, T step_magnitude, T tie, uint32_t& cand) {
  int first = -1;
  for (int i = 0; i < n; ++i)
    if (first < 0 || thetas[i] < thetas[first]) first = i;
  cand = 0;
  if (first >= 0)
    for (int i = 0; i < n; ++i)
      if (g_abs(thetas[i] - thetas[first]) * step_magnitude <= tie) cand |= 1u << kinds[i];
  return first;
}

GLC_HD uint32_t termination_of_event(int kind) {
  return kind == kEvGuard ? GLC_TERM_SINGULARITY
                          : (kind == kEvSurface ? GLC_TERM_SURFACE : (kind == kEvEscape ? GLC_TERM_ESCAPE : GLC_TERM_HORIZON));
}

// Result of one ray, written by the tracer into the caller's SoA.
template <class S>
struct RayResult {
  uint32_t termination, failure, candidates, flags;
  S event_residual;
  S event_theta;  // fraction of the terminal step at the localized event (read by the adjoint)
  S escape_theta, escape_phi;
  S surface_r, surface_phi, g;
};

// Dense output of one step as four polynomial coefficient vectors in T (built once from the
// stages, then evaluated by Horner's rule): y(theta) = y0 + h theta (c1 + theta (c2 + theta (c3 +
// theta c4))).
template <class T>
struct DensePoly {
  T c[4][7];
  template <class TK>
  GLC_HD void build(const TK K[7][7]) {
    using namespace dp;
    const double d[7][4] = {{d10, d11, d12, d13}, {0, 0, 0, 0},     {0, d31, d32, d33}, {0, d41, d42, d43},
                            {0, d51, d52, d53},   {0, d61, d62, d63}, {0, d71, d72, d73}};
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int comp = 0; comp < 7; ++comp) {
        T s = T(0);
#pragma unroll
        for (int j = 0; j < 7; ++j) s += T(d[j][p]) * T(K[j][comp]);
        c[p][comp] = s;
      }
  }
  GLC_HD void eval(const T y0[6], T h, T th, T y[6], T& dt) const {
    for (int comp = 0; comp < 7; ++comp) {
      const T v = th * (c[0][comp] + th * (c[1][comp] + th * (c[2][comp] + th * c[3][comp])));
      if (comp < 6) y[comp] = y0[comp] + h * v;
      else dt = h * v;
    }
  }
};

// Root of an event function on the dense output between theta = 0 (value sv) and 1 (value ev).
// The reference's oracle bisects to the affine tolerance (geodesic.rs:640-676); this is the
// Illinois variant of regula falsi with a bisection guard, which reaches the same bracket width in
// a handful of evaluations. Like the oracle, it stops once the bracket, in affine units, is within
// `tol` and returns the bracket end with the smaller |value|. value_at(y, v) -> false on failure.
template <class T, class F>
GLC_HD bool localize(const T y0[6], T h, const DensePoly<T>& K, T tol, T sv, T ev, F value_at, T& theta, T yroot[6],
                     T& bracket) {
  T lo = T(0), hi = T(1), flo = sv, fhi = ev;  // true values at the bracket ends
  T slo = sv, shi = ev;                        // Illinois-scaled values used for interpolation
  int side = 0;
  T width2 = T(2);  // bracket width two iterations ago
  T width1 = T(1);
  const T ah = g_abs(h);
  for (int i = 0; i < 64; ++i) {
    const T width = hi - lo;
    if (width * ah <= tol) break;
    T mid;
    if (width > T(0.5) * width2) {
      mid = T(0.5) * (lo + hi);  // guard: the bracket stopped halving
      width2 = T(2) * width;
    } else {
      mid = (lo * shi - hi * slo) / (shi - slo);
      if (!(mid > lo && mid < hi)) mid = T(0.5) * (lo + hi);
      width2 = width1;
    }
    width1 = width;
    if (mid == lo || mid == hi) break;
    T ys[6], dt;
    K.eval(y0, h, mid, ys, dt);
    T v;
    if (!value_at(ys, v)) return false;
    if (g_signbit(flo) == g_signbit(v)) {
      lo = mid;
      flo = slo = v;
      if (side == -1) shi *= T(0.5);
      side = -1;
    } else {
      hi = mid;
      fhi = shi = v;
      if (side == 1) slo *= T(0.5);
      side = 1;
    }
    if (v == T(0)) {
      lo = hi = mid;
      flo = fhi = v;
      break;
    }
  }
  theta = g_abs(flo) <= g_abs(fhi) ? lo : hi;
  T dt;
  K.eval(y0, h, theta, yroot, dt);
  bracket = (hi - lo) * ah;
  for (int c = 0; c < 6; ++c)
    if (!g_finite(yroot[c])) return false;
  return true;
}

// Keplerian prograde circular emitter observable (surface.rs:75-146, M = 1). Returns false when
// the orbit is unavailable or not timelike.
// frequency_ratio: g of the emitter at radius r for a photon with energy E and state y (a, Q^2 and
// a^2 as T so that the adjoint can differentiate through them).
template <class T>
GLC_HD bool frequency_ratio(T a, T q2, T a2, double frequency, const T y[6], T E, T r, T& g) {
  const T crs = r - q2;
  if (!(crs >= T(0))) return false;
  const T cr = g_sqrt(crs);
  const T bs = a < T(0) ? T(-1) : T(1);
  const T r2 = r * r;
  const T avd = bs * a * cr + r2;
  if (!(avd > T(0))) return false;
  const T omega = bs * cr / avd;
  const T rn = T(2) * r - q2;
  const T tdisc = T(-3) * r + T(2) * bs * a * cr + T(2) * q2 + r2;
  if (!(tdisc > T(0))) return false;
  const T delta = r2 - T(2) * r + a2 + q2;
  const T gtt = T(-1) + rn / r2;
  const T gtp = -rn * a / r2;
  const T rf = r2 + a2;
  const T gpp = (rf * rf - a2 * delta) / r2;
  const T cn2 = omega * omega * gpp + T(2) * gtp * omega + gtt;
  if (!(cn2 < T(0))) return false;
  const T ut = T(1) / g_sqrt(-cn2);
  const T lz = y[0] * y[4] - y[1] * y[3];
  const T ef = ut * (E - omega * lz);
  if (!(ef > T(0))) return false;
  g = T(frequency) / ef;
  return g_finite(g) && g > T(0);
}

template <class T>
GLC_HD bool surface_observable(const LaneScene& sc, const T y[6], T E, T r, T& g, T& phi_s) {
  if (!frequency_ratio(T(sc.kn.a), T(sc.kn.q2), T(sc.kn.a2), sc.frequency, y, E, r, g)) return false;
  phi_s = wrapped_angle(g_atan2(y[1], y[0]), g_atan2(T(sc.kn.sa), r));
  return true;
}

// Renormalize the spatial momentum so that g^{mu nu} p_mu p_nu = 0 (scaling p_i by lambda closest
// to 1; E is untouched).
template <class T>
GLC_HD bool renormalize_null(const KN<T>& k, T y[6], T E) {
  int st;
  const T r = kn_radius(k, y[0], y[1], y[2], st);
  if (st != kGeomOk) return false;
  const T r2 = r * r;
  const T sigma = r2 + k.a2 * y[2] * y[2] / r2;
  const T f = (T(2) * r - k.q2) / sigma;
  const T A = r2 + k.a2;
  const T l[3] = {k.s * (r * y[0] + k.sa * y[1]) / A, k.s * (r * y[1] - k.sa * y[0]) / A, k.s * y[2] / r};
  const T lp = l[0] * y[3] + l[1] * y[4] + l[2] * y[5];
  const T pp = y[3] * y[3] + y[4] * y[4] + y[5] * y[5];
  // H(lambda) = -E^2 + lambda^2 pp - f (E + lambda lp)^2 = 0  (g^{tt} = -1 - f, g^{ti} = f l_i)
  const T qa = pp - f * lp * lp;
  const T qb = T(-2) * f * E * lp;
  const T qc = -E * E - f * E * E;
  const T disc = qb * qb - T(4) * qa * qc;
  if (!(disc >= T(0)) || qa == T(0)) return false;
  const T sd = g_sqrt(disc);
  const T l1 = (-qb + sd) / (T(2) * qa), l2 = (-qb - sd) / (T(2) * qa);
  const T lam = g_abs(l1 - T(1)) <= g_abs(l2 - T(1)) ? l1 : l2;
  if (!(g_abs(lam - T(1)) < T(1e-3))) return false;
  y[3] *= lam;
  y[4] *= lam;
  y[5] *= lam;
  return true;
}

template <int P>
struct Ray;

// Outputs of one accepted attempt that the commit and the event path need.
template <class C>
struct StepOutT {
  C inc[6], k7[7];
  C dt, r_end, vr_end, en;
  C z0, z1;
  Invariants<C> inv;
  uint32_t mask;
  bool stepped64;
};

// One binary64 DP5(4) attempt from a binary64 state (k1 evaluated at y0).
struct Attempt64 {
  double inc[6], k7[7];
  double dt, r_end, vr_end, en;
  Invariants<double> inv;
  bool finite;
};

GLC_HD void attempt64_body(const KN<double>& kd, const double y0[6], double E, double h, double t_start,
                           const Tolerance& tol, Attempt64* a) {
  double k1[7], rr, vv;
  kn_rhs(kd, y0, E, k1, rr, vv);
#if GLC_ATTEMPT_FORM == 2
  a->en = dp5_attempt_stream<double, double>(kd, y0, E, h, k1, t_start, tol, a->inc, a->dt, a->k7, a->r_end,
                                             a->vr_end, a->inv, a->finite);
#else
  a->en = dp5_attempt<double, double>(kd, y0, E, h, k1, t_start, tol, a->inc, a->dt, a->k7, a->r_end, a->vr_end,
                                      a->inv, a->finite);
#endif
}

#if defined(__CUDA_ARCH__)
__device__ __noinline__ void attempt64_outline(KN<double> kd, const double* y0, double E, double h, double t_start,
                                               Tolerance tol, Attempt64* a) {
  attempt64_body(kd, y0, E, h, t_start, tol, a);
}
GLC_HD void attempt64(const KN<double>& kd, const double y0[6], double E, double h, double t_start,
                      const Tolerance& tol, Attempt64* a) {
  attempt64_outline(kd, y0, E, h, t_start, tol, a);
}
#else
GLC_HD void attempt64(const KN<double>& kd, const double y0[6], double E, double h, double t_start,
                      const Tolerance& tol, Attempt64* a) {
  attempt64_body(kd, y0, E, h, t_start, tol, a);
}
#endif

// ----------------------------------------------------------------------------------------------
// One ray's trace state. The state (x, y, z, p_x, p_y, p_z), affine parameter and coordinate time
// are stepping-precision values; MIXED keeps each as a compensated binary32 pair (hi + lo, ~48
// significant bits) so that its accumulation error matches binary64 without binary64 arithmetic in
// the hot loop. S is the precision of the event path and observables (binary64 in MIXED).
template <int P>
struct Ray {
  using S = typename PrecTraits<P>::S;
  using C = typename PrecTraits<P>::C;
  static constexpr bool kPair = P == kMIXED || P == kBULK;
  using StepOut = StepOutT<C>;

  C yh[6], yl[6];  // state (yl: MIXED low parts, zero otherwise)
  C ah, al;        // affine parameter
  C th, tl;        // coordinate-time increment sum (compensated in every mode, like the reference)
  C Ec;            // energy in stepping precision
  S E;             // energy for the event path and observables
  S az0;           // initial azimuth; the advance is az_end - az0 + 2 pi * winding
  C h;
  C k1[7];         // FSAL derivative at the state
  C r, vr;         // event-function inputs at the state: the exact values the previous step's
                   // crossing checks used as end values (the sign chain every decision follows)
  C lz0, q0, dnull, dlz, dq;
  C turn_r;
  C dir;
  uint32_t accepted, rejected, f64steps, consecutive;
  uint32_t armed;
  uint32_t turnings, crossings;
  int32_t winding, polar;
  uint32_t flags;
  bool have_inv;
  bool pair;       // MIXED with mixed_pair_state: compensated accumulation of state and affine

  GLC_HD S ys(int c) const { return kPair ? S(yh[c]) + S(yl[c]) : S(yh[c]); }
  GLC_HD void state_s(S out[6]) const {
    for (int c = 0; c < 6; ++c) out[c] = ys(c);
  }
  template <class V>
  GLC_HD void set_state(const V v[6]) {
    for (int c = 0; c < 6; ++c) {
      yh[c] = C(v[c]);
      yl[c] = kPair && pair ? C(v[c] - V(yh[c])) : C(0);
    }
  }
  GLC_HD S travel() const { return S(dir) * (S(th) + S(tl)); }
  GLC_HD S affine() const { return kPair ? S(ah) + S(al) : S(ah); }

  GLC_HD void init(const LaneScene& sc, const glc_policy& pol, const double st8[8], double direction) {
    // the pair state splits the binary64 initial state into high and low parts
    using V = typename std::conditional<kPair, double, S>::type;
    V v[6];
    for (int c = 0; c < 3; ++c) {
      v[c] = V(st8[1 + c]);
      v[3 + c] = V(st8[5 + c]);
    }
    pair = kPair && pol.mixed_pair_state != 0u;
    set_state(v);
    E = S(-st8[4]);
    Ec = C(E);
    dir = C(direction);
    h = dir * C(pol.initial_step);
    ah = al = th = tl = C(0);
    accepted = rejected = f64steps = consecutive = 0;
    turnings = crossings = 0;
    winding = 0;
    flags = 0;
    polar = st8[3] > 0.0 ? 1 : (st8[3] < 0.0 ? -1 : 0);
    turn_r = C(NAN);
    az0 = P == kBULK ? S(0) : S(g_atan2(v[1], v[0]));  // BULK: the completion kernel derives it
    dnull = dlz = dq = C(0);
    // first derivative (FSAL seed), the invariants at the start and the event arming
    // (geodesic.rs:98-136, 536-544)
    const KN<C> kc = kn_cast<C>(sc.kn);
    C rr, vv;
    Invariants<C> inv;
    kn_rhs<C, true>(kc, yh, Ec, k1, rr, vv, &inv);
    r = rr;
    vr = vv;
    if (pair) pair_invariants(inv);
    have_inv = g_finite(rr) && g_finite(inv.lz) && g_finite(inv.carter) && g_finite(inv.null_residual);
    lz0 = inv.lz;
    q0 = inv.carter;
    armed = 0;
    if (have_inv) {
      dnull = inv.null_residual;
      for (int kind = 0; kind < 4; ++kind) {
        const C vk = event_value<C>(kind, sc, pol.singularity_guard, r, yh[2]);
        if (event_clears_band(kind, vk, C(pol.event_arming_band))) armed |= 1u << kind;
      }
    }
  }

  // MIXED: L_x, L_y, L_z from the compensated state (products of pairs), so that L_z and Carter's
  // constant keep binary32 relative accuracy in their own scale far from the hole.
  GLC_HD void pair_invariants(Invariants<C>& inv) const {
    if constexpr (kPair) {
      const float lx = ff_cross(yh[1], yl[1], yh[5], yl[5], yh[2], yl[2], yh[4], yl[4]);  // y p_z - z p_y
      const float ly = ff_cross(yh[2], yl[2], yh[3], yl[3], yh[0], yl[0], yh[5], yl[5]);  // z p_x - x p_z
      inv.lz = ff_cross(yh[0], yl[0], yh[4], yl[4], yh[1], yl[1], yh[3], yl[3]);          // x p_y - y p_x
      inv.carter = lx * lx + ly * ly + inv.abracket;
    }
  }

  template <class T>
  GLC_HD void update_drifts(const Invariants<T>& inv) {
    if (!have_inv) return;
    if (g_finite(inv.null_residual)) dnull = g_max(dnull, C(inv.null_residual));
    if (g_finite(inv.lz)) dlz = g_max(dlz, C(g_abs(T(inv.lz) - T(lz0)) / g_max(g_abs(T(lz0)), T(1))));
    if (g_finite(inv.carter)) dq = g_max(dq, C(g_abs(T(inv.carter) - T(q0)) / g_max(g_abs(T(q0)), T(1))));
  }

  GLC_HD C next_step(const glc_policy& pol, C mag, C en, bool accepted_step) const {
    const C maxf = accepted_step ? C(pol.maximum_factor) : C(1);
    C factor;
    if (en == C(0)) {
      factor = maxf;
    } else {
      factor = C(pol.safety) * g_pow_m02(en);
      factor = factor < C(pol.minimum_factor) ? C(pol.minimum_factor) : (factor > maxf ? maxf : factor);
    }
    C hn = mag * factor;
    hn = hn < C(pol.minimum_step) ? C(pol.minimum_step) : (hn > C(pol.maximum_step) ? C(pol.maximum_step) : hn);
    return hn;
  }

  // Winding of the azimuth about the z axis (geodesic.rs:406-418): a wrap of atan2(y, x) happens
  // only when y changes sign, so the azimuths are evaluated on those steps alone.
  GLC_HD void commit_azimuth(S x_old, S y_old, S x_new, S y_new) {
    if (g_signbit(y_old) == g_signbit(y_new)) return;
    const S raw = g_atan2(y_new, x_new) - g_atan2(y_old, x_old);
    const S pi = S(3.14159265358979323846);
    if (raw > pi) winding -= 1;
    else if (raw < -pi) winding += 1;
  }

  GLC_HD S azimuth_advance() const {
    return g_atan2(ys(1), ys(0)) - az0 + S(6.28318530717958647692) * S(winding);
  }

  GLC_HD void add_time(C v) { ff_add_any(th, tl, v); }
  GLC_HD static void ff_add_any(C& hi, C& lo, C v) {
    if constexpr (sizeof(C) == sizeof(float)) {
      ff_add(hi, lo, v);
    } else {
      CompSum::add(hi, lo, v);
    }
  }

  // Advance by one attempted step. Returns true when the ray terminated (result filled). use64
  // (MIXED only): take this step in binary64 (the warp has a lane inside the shell). One step body
  // serves both cases; only the attempt itself branches.
  // stages (optional, binary64 stepping only): where the attempt leaves its seven stage
  // derivatives, so that the event path builds the dense output from them instead of evaluating
  // the stages again
  // kUnroll: the attempt's stage loop unrolled (6) or rolled (1); unrolled by default only in
  // MIXED's bulk stepping, whose small footprint lets it pay.
  template <int kUnroll = (P == kBULK ? 6 : 1)>
  GLC_HD bool step(const LaneScene& sc, const glc_policy& pol, RayResult<S>& res, bool use64,
                   C (*stages)[7] = nullptr) {
    if (uint64_t(accepted) >= pol.maximum_accepted_steps) {
      finish_plain(res, GLC_TERM_STEP_EXHAUSTION, GLC_FAIL_NONE);
      return true;
    }
    if (P == kBULK && double(r) < sc.shell_r) return hand_off(res);
    const Tolerance tol{pol.position_rtol, pol.position_atol, pol.momentum_rtol, pol.momentum_atol};
    StepOut o;
    bool finite;
    const bool stepped64 = P == kMIXED && use64;
    if (stepped64) {
      // binary64 step inside the shell: double k1 at the state, double stages and error control
      // (out of line on the device, so the binary32 hot loop is not register-allocated for it)
      Attempt64 a;
      double yd[6];
      for (int c = 0; c < 6; ++c) yd[c] = double(ys(c));
      attempt64(sc.kn, yd, double(E), double(h), double(th) + double(tl), tol, &a);
      for (int c = 0; c < 6; ++c) o.inc[c] = C(yd[c] + a.inc[c] - ys(c));
      for (int c = 0; c < 7; ++c) o.k7[c] = C(a.k7[c]);
      o.dt = C(a.dt);
      o.r_end = C(a.r_end);
      o.vr_end = C(a.vr_end);
      o.inv.lz = C(a.inv.lz);
      o.inv.carter = C(a.inv.carter);
      o.inv.null_residual = C(a.inv.null_residual);
      o.inv.abracket = C(a.inv.abracket);
      o.en = C(a.en);
      finite = a.finite;
    } else {
      const KN<C> kc = kn_cast<C>(sc.kn);
#if GLC_ATTEMPT_FORM == 1
      o.en = dp5_attempt_compact<C, C, true>(kc, yh, Ec, h, k1, th + tl, tol, o.inc, o.dt, o.k7, o.r_end, o.vr_end,
                                             o.inv, finite);
#elif GLC_ATTEMPT_FORM == 2
      // MIXED's bulk kernel unrolls the stage loop (+5 % there; the one-kernel FP32 lost 13 % with
      // it, to instruction fetch, and so did the work-queue kernels, which inline it into more code)
      o.en = dp5_attempt_stream<C, C, true, std::is_same<C, double>::value, kUnroll>(
          kc, yh, Ec, h, k1, th + tl, tol, o.inc, o.dt, o.k7, o.r_end, o.vr_end, o.inv, finite, sc.track, stages);
#else
      o.en = dp5_attempt<C, C, true>(kc, yh, Ec, h, k1, th + tl, tol, o.inc, o.dt, o.k7, o.r_end, o.vr_end, o.inv,
                                     finite);
#endif
    }
    if (!finite || !g_finite(o.en)) {
      finish_plain(res, GLC_TERM_NUMERICAL_FAILURE, GLC_FAIL_NON_FINITE);
      return true;
    }
    if (o.en > C(1)) {
      rejected += 1;
      consecutive += 1;
      if (consecutive >= pol.maximum_consecutive_rejects) {
        finish_plain(res, GLC_TERM_REJECT_EXHAUSTION, GLC_FAIL_NONE);
        return true;
      }
      if (g_abs(h) <= C(pol.minimum_step)) {
        finish_plain(res, GLC_TERM_NUMERICAL_FAILURE, GLC_FAIL_MINIMUM_STEP);
        return true;
      }
      h = dir * next_step(pol, g_abs(h), o.en, false);
      return false;
    }
    // ---- crossing detection in the stepping precision; the start values are exactly the
    // previous step's end values, so every sign change between consecutive states is seen
    const double guard = pol.singularity_guard;
    o.z0 = yh[2];
    o.z1 = yh[2] + o.inc[2];
    if (pair) {
      C zl = yl[2], zh = yh[2];
      ff_add_any(zh, zl, o.inc[2]);
      o.z1 = zh;
    }
    uint32_t ev = 0;
    for (int kind = 0; kind < 4; ++kind) {
      if (!((armed >> kind) & 1u) || !((sc.installed >> kind) & 1u)) continue;
      const C sv = event_value<C>(kind, sc, guard, r, o.z0);
      const C evv = event_value<C>(kind, sc, guard, o.r_end, o.z1);
      if (event_crosses(kind, sv, evv)) ev |= 1u << kind;
    }
    const C vs = dir * vr, ve = dir * o.vr_end;
    if ((vs < C(0) && ve >= C(0)) || (vs > C(0) && ve <= C(0))) ev |= 1u << 4;
    if (event_crosses(kEvSurface, o.z0, o.z1)) ev |= 1u << 5;
    o.mask = ev;
    // BULK: a step that brackets a root of the singularity guard, the horizon or the escape sphere
    // is terminal whatever comes first in it; TAIL re-takes it in binary64
    constexpr uint32_t kTerminalBits = (1u << kEvGuard) | (1u << kEvHorizon) | (1u << kEvEscape);
    if (P == kBULK && (ev & kTerminalBits) != 0u) return hand_off(res);
    accepted += 1;
    consecutive = 0;
    if (stepped64 || P == kTAIL) {
      f64steps += 1;
      flags |= kFlagShellF64;
    }
    if (ev != 0u) {
      o.stepped64 = stepped64;
      // inline: with the streaming attempt the ray fits in registers, and copying it to local
      // memory for an out-of-line call measured 12-15 % slower in every precision
      if (event_path(sc, pol, res, o, stages)) return true;
    }
    commit(sc, pol, o, stepped64);
    return false;
  }

  // Plain commit of an accepted, non-terminal step.
  GLC_HD void commit(const LaneScene& sc, const glc_policy& pol, const StepOut& o, bool stepped64) {
    const C x_old = yh[0], y_old = yh[1];
    add_time(o.dt);
    if (pair) {
      for (int c = 0; c < 6; ++c) ff_add_any(yh[c], yl[c], o.inc[c]);
      ff_add_any(ah, al, h);
    } else {
      for (int c = 0; c < 6; ++c) yh[c] += o.inc[c];
      ah += h;
    }
    commit_azimuth(S(x_old), S(y_old), S(yh[0]), S(yh[1]));
    if (sc.track) {
      if (pair) {
        // L_z and Carter's constant from the committed pair state, on accepted steps only
        Invariants<C> inv = o.inv;
        pair_invariants(inv);
        update_drifts(inv);
      } else {
        update_drifts(o.inv);
      }
    }
    for (int c = 0; c < 7; ++c) k1[c] = o.k7[c];
    r = o.r_end;
    vr = o.vr_end;
    arm_update(sc, pol);
    h = dir * next_step(pol, g_abs(h), o.en, true);
    (void)stepped64;
  }

  GLC_HD void arm_update(const LaneScene& sc, const glc_policy& pol) {
    if (armed == 0xFu) return;
    for (int kind = 0; kind < 4; ++kind) {
      if ((armed >> kind) & 1u) continue;
      const C v = event_value<C>(kind, sc, pol.singularity_guard, r, yh[2]);
      if (event_clears_band(kind, v, C(pol.event_arming_band))) armed |= 1u << kind;
    }
  }

  GLC_HD void add_time_s(S v) {
    const C hi = C(v);
    add_time(hi);
    if (kPair) add_time(C(v - S(hi)));
  }
  GLC_HD void add_affine_s(S v) {
    const C hi = C(v);
    ff_add_any(ah, al, hi);
    if (kPair) ff_add_any(ah, al, C(v - S(hi)));
  }

  // Event path of an accepted step with a sign change (o.mask: bits 0-3 events, 4 radial turning,
  // 5 equator). The decisions are the stepping-precision sign tests already taken; here the roots
  // are localized on the step's dense output in precision S (binary64 in MIXED: a binary64 dense
  // polynomial from the stepping-precision stages), events are ordered and, for a terminal event,
  // the observables are evaluated in S. Returns true when the ray terminated; otherwise the caller
  // commits the step as a plain one.
  GLC_HD bool event_path(const LaneScene& sc, const glc_policy& pol, RayResult<S>& res, const StepOut& o,
                         const C (*stages)[7] = nullptr) {
    using T = S;
    uint32_t mask = o.mask;
    {
      // Decisions without the dense output. Outside the horizon a null geodesic's r has at most one
      // turning point, so on a step whose radial velocity keeps its sign r moves monotonically
      // between the end radii, and a surface crossing's radius lies between them: when both lie
      // outside the surface's radial interval (widened by the margin, on the same side), the
      // crossing misses the surface. Otherwise its root decides, below.
      const bool turning = (mask >> 4) & 1u;
      if (((mask >> kEvSurface) & 1u) && !turning) {
        const double lo = g_min(double(r), double(o.r_end)), hi = g_max(double(r), double(o.r_end));
        if (hi < sc.surf_in * (1.0 - kSurfaceMissMargin) || lo > sc.surf_out * (1.0 + kSurfaceMissMargin)) {
          mask &= ~(1u << kEvSurface);
        } else if (P == kBULK && lo > sc.surf_in * (1.0 + kBulkSurfaceMargin) &&
                   hi < sc.surf_out * (1.0 - kBulkSurfaceMargin)) {
          // BULK: the crossing lies on the surface, away from its edges, so TAIL takes the step
          // (the binary32 root would only confirm the hand-off)
          accepted -= 1;
          return hand_off(res);
        }
      }
      if ((mask & 0xFu) == 0u) {
        // No event root in the step, so nothing to order the crossings and turnings against. An
        // equatorial crossing's root always exists on the dense output (z changes sign between its
        // ends), so it is counted without localizing it.
        if ((mask >> 5) & 1u) crossings += 1;
        mask &= ~(1u << 5);
        if (!turning) return false;
        // an outward turning (apocentre) is counted likewise; a pericentre's radius needs its root
        if (!(dir * vr < C(0) && dir * o.vr_end >= C(0))) {
          turnings += 1;
          return false;
        }
        // MIXED's bulk kernel: the pericentre's radius from the radial potential instead of the
        // dense output. FP32 and FP64 keep the reference's root on the dense output: they follow
        // its algorithm wherever a shortcut would change a result, and this one moves the radius
        // by the drift of the constants of motion.
        C rp;
        if (P == kBULK && pericentre_radius(sc, o, rp)) {
          turnings += 1;
          turn_r = (turn_r == turn_r) ? g_min(turn_r, rp) : rp;
          return false;
        }
      }
    }
    const KN<T> kt = kn_cast<T>(sc.kn);
    T y[6];
    state_s(y);
    // stages for the dense output, in the stepping precision (binary64 on MIXED shell steps)
    DensePoly<T> dpoly;
    if (stages != nullptr) {
      dpoly.build(stages);
    } else if (o.stepped64) {
      double K[7][7], yk[6], rr, vv, ye[6];
      for (int c = 0; c < 6; ++c) yk[c] = double(y[c]);
      kn_rhs(sc.kn, yk, double(E), K[0], rr, vv);
      dp5_stages(sc.kn, yk, double(E), double(h), K, ye, rr, vv);
      dpoly.build(K);
    } else {
      const KN<C> kc = kn_cast<C>(sc.kn);
      C K[7][7], ye[6], rr, vv;
      for (int c = 0; c < 7; ++c) K[0][c] = k1[c];
      dp5_stages(kc, yh, Ec, h, K, ye, rr, vv);
      dpoly.build(K);
    }
    const T hh = T(h);
    const double guard = pol.singularity_guard;
    const T tol = T(P == kBULK && pol.event_affine_tolerance < kBulkRootTolerance ? kBulkRootTolerance
                                                                                 : pol.event_affine_tolerance);
    int n = 0;
    int kinds[4];
    T thetas[4], residuals[4], states[4][6];
    for (int kind = 0; kind < 4; ++kind) {
      if (P == kBULK && kind != kEvSurface) continue;  // the other events were handed off already
      if (!((mask >> kind) & 1u)) continue;
      const T sv = T(event_value<C>(kind, sc, guard, r, o.z0));
      const T evv = T(event_value<C>(kind, sc, guard, o.r_end, o.z1));
      T th_, yr[6], br;
      auto value_at = [&](const T* ys_, T& v) -> bool {
        int gs = kGeomOk;
        const T rr = kind == kEvSurface ? T(0) : kn_radius(kt, ys_[0], ys_[1], ys_[2], gs);
        if (gs != kGeomOk) return false;
        v = event_value<T>(kind, sc, guard, rr, ys_[2]);
        return true;
      };
      if (!localize(y, hh, dpoly, tol, sv, evv, value_at, th_, yr, br)) {
        finish_plain(res, GLC_TERM_NUMERICAL_FAILURE, GLC_FAIL_NON_FINITE);
        return true;
      }
      T rv;
      if (!value_at(yr, rv)) {
        finish_plain(res, GLC_TERM_NUMERICAL_FAILURE, GLC_FAIL_NON_FINITE);
        return true;
      }
      bool keep = true;
      if (kind == kEvSurface) {
        int gs;
        const T rr = kn_radius(kt, yr[0], yr[1], yr[2], gs);
        if (P == kBULK)
          keep = gs == kGeomOk && rr >= T(sc.surf_in * (1.0 - kBulkSurfaceMargin)) &&
                 rr <= T(sc.surf_out * (1.0 + kBulkSurfaceMargin));
        else
          keep = gs == kGeomOk && rr >= T(sc.surf_in) && rr <= T(sc.surf_out);
      }
      if (keep) {
        kinds[n] = kind;
        thetas[n] = th_;
        residuals[n] = g_abs(rv) / T(event_scale(kind, sc));
        for (int c = 0; c < 6; ++c) states[n][c] = yr[c];
        ++n;
      }
    }
    uint32_t cand = 0;
    const int first = earliest_event<T>(kinds, thetas, n, g_abs(hh), T(pol.event_tie_tolerance), cand);
    const bool has_event = first >= 0;
    if (P == kBULK && has_event) {
      // a surface crossing at or near the surface: TAIL re-takes the step (not counted here)
      accepted -= 1;
      return hand_off(res);
    }
    const T term_theta = has_event ? thetas[first] : T(1);
    // the replaced GPU kernel's gate: the terminal inside a turning point's root bracket
    bool turning_uncertain = false;
    // radial turning point (geodesic.rs:330-360)
    if ((mask >> 4) & 1u) {
      const T sv = T(dir * vr), evv = T(dir * o.vr_end);
      T th_, yr[6], br;
      auto vr_at = [&](const T* ys_, T& v) -> bool {
        C d[7], rr, vv, yy[6];
        for (int c = 0; c < 6; ++c) yy[c] = C(ys_[c]);
        kn_rhs(kn_cast<C>(sc.kn), yy, Ec, d, rr, vv);
        v = T(dir * vv);
        return g_finite(v);
      };
      const bool found = localize(y, hh, dpoly, tol, sv, evv, vr_at, th_, yr, br);
      if (found && (!has_event || th_ < term_theta)) {
        turnings += 1;
        if (sv < T(0) && evv >= T(0)) {
          int gs;
          const T rr = kn_radius(kt, yr[0], yr[1], yr[2], gs);
          if (gs == kGeomOk) turn_r = (turn_r == turn_r) ? C(g_min(T(turn_r), rr)) : C(rr);
        }
      }
      if (has_event && (!found || g_abs(th_ - term_theta) * g_abs(hh) <= br)) turning_uncertain = true;
    }
    // equatorial crossing (geodesic.rs:362-383)
    if ((mask >> 5) & 1u) {
      T th_, yr[6], br;
      auto z_at = [&](const T* ys_, T& v) -> bool {
        v = ys_[2];
        return true;
      };
      if (localize(y, hh, dpoly, tol, T(o.z0), T(o.z1), z_at, th_, yr, br) && (!has_event || th_ < term_theta))
        crossings += 1;
    }
    if (P == kBULK || !has_event) return false;
    // terminal commit at the event (precision S)
    T ycommit[6], dtc;
    {
      T ytmp[6];
      dpoly.eval(y, hh, term_theta, ytmp, dtc);
      for (int c = 0; c < 6; ++c) ycommit[c] = states[first][c];
    }
    add_time_s(dtc);
    commit_azimuth(y[0], y[1], ycommit[0], ycommit[1]);
    {
      int gs;
      const T rr = kn_radius(kt, ycommit[0], ycommit[1], ycommit[2], gs);
      if (sc.track && gs == kGeomOk) update_drifts(kn_invariants(kt, ycommit, E, rr));
    }
    add_affine_s(hh * term_theta);
    set_state(ycommit);
    const uint32_t term = termination_of_event(kinds[first]);
    finish_event(sc, pol, res, term, cand, residuals[first], ycommit);
    res.event_theta = term_theta;
    if (pol.uncertain_terminals) {
      const double limit = pol.uncertain_drift_limit;
      const bool drift = sc.track && (double(dnull) > limit || double(dlz) > limit || double(dq) > limit);
      if ((cand & (cand - 1u)) != 0u || turning_uncertain || drift) res.termination = GLC_TERM_UNCERTAIN;
    }
    return true;
  }

  // The radius of a pericentre inside the step, as the largest root of the radial potential
  //   R(r) = [E (r^2 + a^2) - a L_z]^2 - Delta [(L_z - a E)^2 + Q],  Delta = r^2 - 2 r + a^2 + Q_e^2
  // of the constants of motion at the step's start (Carter's Q in the same L-form as the drift
  // diagnostics). Outside the horizon the pericentre is R's largest root and lies below both end
  // radii, where R is positive and rising, so Newton's method from the smaller end radius descends
  // onto it. It takes a few binary32 evaluations where localizing the root of the radial velocity
  // on the dense output takes the step's six stages again and a right-hand side per iteration. The
  // radius differs from that root's by the drift of the constants (the frame tolerance's level).
  // Returns false when Newton does not settle below the end radii, as near a double root (a ray
  // grazing the photon orbit); the caller then localizes the root.
  GLC_HD bool pericentre_radius(const LaneScene& sc, const StepOut& o, C& rp) const {
    const C x = yh[0], y = yh[1], z = yh[2], px = yh[3], py = yh[4], pz = yh[5];
    const C a = C(sc.kn.a), a2 = C(sc.kn.a2), q2 = C(sc.kn.q2), E = Ec;
    const C L = x * py - y * px;
    const C Lx = y * pz - z * py, Ly = z * px - x * pz;
    const C r0 = r, r02 = r0 * r0;
    const C Q = Lx * Lx + Ly * Ly +
                a2 * (z * z / r02 * (px * px + py * py - E * E) - (x * x + y * y) / (r02 + a2) * pz * pz);
    const C K = (L - a * E) * (L - a * E) + Q;
    const C top = g_min(r0, C(o.r_end));
    C rr = top;
    for (int it = 0; it < 16; ++it) {
      const C w = E * (rr * rr + a2) - a * L;
      const C R = w * w - (rr * rr - C(2) * rr + a2 + q2) * K;
      const C dR = C(4) * E * rr * w - (C(2) * rr - C(2)) * K;
      if (!(dR > C(0))) return false;
      const C step = R / dR;
      rr -= step;
      if (!(rr > C(0.5) * top)) return false;
      if (g_abs(step) <= C(1e-7) * rr) {
        if (!(rr <= top * C(1.000001))) return false;
        rp = rr;
        return true;
      }
    }
    return false;
  }

  // BULK: leave the ray to TAIL at the current state (termination NONE: not finished).
  GLC_HD bool hand_off(RayResult<S>& res) {
    res.termination = GLC_TERM_NONE;
    res.failure = GLC_FAIL_NONE;
    return true;
  }

  GLC_HD void finish_plain(RayResult<S>& res, uint32_t term, uint32_t failure) {
    res.termination = term;
    res.failure = failure;
    res.candidates = 0;
    res.flags = flags;
    res.event_residual = S(NAN);
    res.event_theta = S(NAN);
    res.escape_theta = res.escape_phi = S(NAN);
    res.surface_r = res.surface_phi = res.g = S(NAN);
  }

  // Terminal observables at the committed event state y (precision S; binary64 in MIXED).
  GLC_HD void finish_event(const LaneScene& sc, const glc_policy& pol, RayResult<S>& res, uint32_t term,
                           uint32_t cand, S residual, const S ystate[6]) {
    using T = S;
    const KN<T> kt = kn_cast<T>(sc.kn);
    T ye[6];
    for (int c = 0; c < 6; ++c) ye[c] = ystate[c];
    if ((P == kMIXED || P == kTAIL) && pol.renormalize_null) {
      if (renormalize_null(kt, ye, E)) flags |= kFlagRenormalized;
    }
    res.termination = term;
    res.failure = GLC_FAIL_NONE;
    res.candidates = cand;
    res.event_residual = residual;
    res.escape_theta = res.escape_phi = S(NAN);
    res.surface_r = res.surface_phi = res.g = S(NAN);
    if (term == GLC_TERM_ESCAPE) {
      T d[7], rr, vv;
      kn_rhs(kt, ye, E, d, rr, vv);
      const T dx = T(dir) * d[0], dy = T(dir) * d[1], dz = T(dir) * d[2];
      const T nrm = g_sqrt(dx * dx + dy * dy + dz * dz);
      if (nrm > T(0) && g_finite(nrm)) {
        T cz = dz / nrm;
        cz = cz > T(1) ? T(1) : (cz < T(-1) ? T(-1) : cz);
        res.escape_theta = g_acos(cz);
        res.escape_phi = g_atan2(dy, dx);
      } else {
        flags |= kFlagNoEscapeDirection;
      }
    } else if (term == GLC_TERM_SURFACE) {
      int gs;
      const T rr = kn_radius(kt, ye[0], ye[1], ye[2], gs);
      T g, phi;
      if (gs == kGeomOk && surface_observable(sc, ye, E, rr, g, phi)) {
        res.surface_r = rr;
        res.surface_phi = phi;
        res.g = g;
      } else {
        flags |= kFlagSurfaceInvalid;
      }
    }
    res.flags = flags;
  }
};

// ---- MIXED as two kernels: the hand-off record of a ray from BULK to TAIL, 128 bytes (8 words of
// 16 bytes, which the kernels store word-major across the job's rays):
//   d[0..5] the state (x, y, z, p_x, p_y, p_z) in binary64 (the sum of the compensated pair),
//   d[6] the affine parameter, d[7] the coordinate-time increment sum;
//   f[0..7] step size with direction, L_z and Carter's constant at the start, minimum turning radius,
//   the null residual, L_z and Carter drift maxima, and the radius at the state as BULK's last
//   crossing checks saw it;
//   u[0..7] accepted, rejected, consecutive rejects, armed event bits, radial turnings, equatorial
//   crossings, winding, and polar side + 1 | flags << 4 | termination << 16 | failure << 24 |
//   sign of the radial velocity at the state (0 positive, 1 negative, 2 zero) << 28 |
//   invariants valid << 31.
// The radius and the sign of the radial velocity carry BULK's sign chain over to TAIL: the state's
// binary64 values can fall on the other side of an event (a state a few binary32 ulps inside the
// escape sphere whose binary64 radius is already outside it would never see the sphere crossed).
// E, the initial azimuth and the direction are not stored: TAIL re-derives them from the ray's
// initial state, exactly as BULK did.
struct alignas(16) HandoffRec {
  double d[8];
  float f[8];
  uint32_t u[8];
};
static_assert(sizeof(HandoffRec) == 128, "hand-off record is 8 words of 16 bytes");

GLC_HD void handoff_pack(const Ray<kBULK>& ray, const RayResult<float>& res, HandoffRec& rec) {
  for (int c = 0; c < 6; ++c) rec.d[c] = double(ray.yh[c]) + double(ray.yl[c]);
  rec.d[6] = double(ray.ah) + double(ray.al);
  rec.d[7] = double(ray.th) + double(ray.tl);
  rec.f[0] = ray.h;
  rec.f[1] = ray.lz0;
  rec.f[2] = ray.q0;
  rec.f[3] = ray.turn_r;
  rec.f[4] = ray.dnull;
  rec.f[5] = ray.dlz;
  rec.f[6] = ray.dq;
  rec.f[7] = ray.r;
  rec.u[0] = ray.accepted;
  rec.u[1] = ray.rejected;
  rec.u[2] = ray.consecutive;
  rec.u[3] = ray.armed;
  rec.u[4] = ray.turnings;
  rec.u[5] = ray.crossings;
  rec.u[6] = uint32_t(ray.winding);
  rec.u[7] = uint32_t(ray.polar + 1) | ((ray.flags & 0xFFFu) << 4) | ((res.termination & 0xFFu) << 16) |
             ((res.failure & 0xFu) << 24) | (ray.vr < 0.0f ? 1u << 28 : (ray.vr == 0.0f ? 2u << 28 : 0u)) |
             (ray.have_inv ? 1u << 31 : 0u);
}

// Resume a handed-off ray as a binary64 stepper: the stored state and counters, E and the initial
// azimuth from the ray's initial state st8, and the derivative, radius and radial velocity at the
// state re-evaluated in binary64. Returns the termination BULK recorded (NONE: continue stepping)
// and sets its failure kind.
GLC_HD uint32_t handoff_unpack(const HandoffRec& rec, Ray<kTAIL>& ray, const LaneScene& sc, const double st8[8],
                               double direction, uint32_t& failure) {
  ray.pair = false;
  ray.set_state(rec.d);
  ray.E = -st8[4];
  ray.Ec = ray.E;
  ray.dir = direction;
  ray.az0 = g_atan2(st8[2], st8[1]);
  ray.ah = rec.d[6];
  ray.al = 0.0;
  ray.th = rec.d[7];
  ray.tl = 0.0;
  ray.h = double(rec.f[0]);
  ray.lz0 = double(rec.f[1]);
  ray.q0 = double(rec.f[2]);
  ray.turn_r = double(rec.f[3]);
  ray.dnull = double(rec.f[4]);
  ray.dlz = double(rec.f[5]);
  ray.dq = double(rec.f[6]);
  ray.accepted = rec.u[0];
  ray.rejected = rec.u[1];
  ray.consecutive = rec.u[2];
  ray.armed = rec.u[3];
  ray.f64steps = 0;
  ray.turnings = rec.u[4];
  ray.crossings = rec.u[5];
  ray.winding = int32_t(rec.u[6]);
  const uint32_t w = rec.u[7];
  ray.polar = int32_t(w & 0xFu) - 1;
  ray.flags = (w >> 4) & 0xFFFu;
  ray.have_inv = (w >> 31) != 0u;
  failure = (w >> 24) & 0xFu;
  double rr, vv;
  kn_rhs(sc.kn, ray.yh, ray.Ec, ray.k1, rr, vv);
  // continue BULK's sign chain: its radius at the state, and a radial velocity of its sign
  ray.r = double(rec.f[7]);
  const uint32_t vs = (w >> 28) & 3u;
  if (vs == 2u) vv = 0.0;
  else if (vs == 1u && !(vv < 0.0)) vv = -DBL_MIN;
  else if (vs == 0u && !(vv > 0.0)) vv = DBL_MIN;
  ray.vr = vv;
  (void)rr;
  return (w >> 16) & 0xFFu;
}

}  // namespace glc
