// Binary32 restatement of the reference's own GPU trace kernel, the one the CUDA path replaces: the
// fixed-policy classical RK4 loop of crates/gravlume-render/src/shaders/geodesic_integration.wgsl
// (trace_initialized, 22-408) over the Kerr-Schild dynamics of kerr_schild_dynamics.wgsl (18-317)
// and the event, invariant, source and branch helpers of geodesic_events.wgsl (3-515), fed with the
// uniforms that TraceUniforms::from_observation_with_surface packs
// (crates/gravlume-render/src/trace/input.rs:85-131).
//
// TEST INFRASTRUCTURE ONLY. It is a second comparator: it shows what the reference's GPU algorithm
// yields on the rays the CUDA kernels trace, next to the binary64 oracle that checks them. It is
// pinned by the reference's own GPU-against-CPU gate (gpu_trace_tests.rs:544-627: terminal class,
// escape direction within 3.82e-4 rad, event residual 5e-3, travel time 1e-3 M, drifts 0.05).
//
// Binary32 throughout, as in WGSL; every product is unfused (the oracle builds with
// -ffp-contract=off), and inverseSqrt is 1/sqrt.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>

namespace gro {
namespace rk4 {

// TraceTermination discriminants (trace_protocol.wgsl; the same 1-7 as the CPU reference).
constexpr uint32_t kHorizon = 1, kEscape = 2, kSingularity = 3, kStepExhaustion = 4, kFailure = 5,
                   kUncertain = 6, kSurface = 7;
constexpr uint32_t kNonFinite = 1, kBadRadicand = 2, kBadDenominator = 4;           // failure flags
constexpr uint32_t kCandSingularity = 1, kCandHorizon = 2, kCandSurface = 4, kCandEscape = 8;
constexpr uint32_t kMaxSteps = 2048;           // MAXIMUM_STEPS
constexpr int kEventIterations = 6;            // EVENT_REFINEMENT_ITERATIONS
constexpr int kTurningIterations = 20;         // TURNING_REFINEMENT_ITERATIONS
constexpr float kDerivativeFloor = 0x1p-11f;   // EVENT_DERIVATIVE_RELATIVE_FLOOR
constexpr float kMaxFinite = std::numeric_limits<float>::max();

struct V3 {
  float x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline bool finite(float v) { return v == v && std::fabs(v) <= kMaxFinite; }
inline bool finite(V3 v) { return finite(v.x) && finite(v.y) && finite(v.z); }
inline float wgsl_sign(float v) { return v > 0.0f ? 1.0f : (v < 0.0f ? -1.0f : 0.0f); }

// Saturating helpers of trace_protocol.wgsl (products and sums clamp at the largest finite value).
inline float sat_product(float a, float b) {
  if (a == 0.0f || b == 0.0f) return 0.0f;
  if (a > 1.0f && b > kMaxFinite / a) return kMaxFinite;
  return a * b;
}
inline float sat_sum(float a, float b) { return a > kMaxFinite - b ? kMaxFinite : a + b; }
inline float sat_square(float v) { return sat_product(std::fabs(v), std::fabs(v)); }

// TraceUniforms, narrowed to binary32 (input.rs:85-131). The event surfaces are the job's.
struct Uniforms {
  float mass, spin, charge, chart;           // (M, a, Q, Kerr-Schild branch sign)
  V3 observer;                               // observer x, y, z
  float velocity[4], right[4], up[4], arrival[4];  // contravariant tetrad legs (t, x, y, z)
  float tan_half_fov, frequency;
  float escape, guard, horizon, tie;         // escape radius, 2^-40, capture radius, 2^-17 M
  float inner, outer, arming;                // surface radii, arming band 2^-12 M
  bool surface;
  float step_scale, step_min, step_max, drift_limit;  // 0.1, 0.005, 8, 0.05
};

struct Geometry {
  float radius = 0.0f, f = 0.0f;
  V3 df{0, 0, 0}, l{0, 0, 0}, dr{0, 0, 0};
  float inv_scale = 0.0f, inv_r = 0.0f, inv_oblate = 0.0f, sing = 0.0f;
  uint32_t flags = 0;
};
inline Geometry bad_geometry(uint32_t flags) {
  Geometry g;
  g.flags = flags;
  return g;
}

struct State {
  V3 x, p;
};
struct Rhs {
  float tdot = 0.0f;
  V3 xdot{0, 0, 0}, pdot{0, 0, 0};
  uint32_t flags = 0;
};

// Scaled oblate radius, f = (2Mr - Q^2)/Sigma and its gradient, the principal null direction and
// grad r (kerr_schild_dynamics.wgsl:18-163): coordinates are divided by max(|x|, |y|, |z|, |a|),
// with a closed form on the axis and the conjugate root where direct addition would cancel.
inline Geometry metric_geometry(const Uniforms& U, V3 pos) {
  const float scale = std::max(std::max(std::max(std::fabs(pos.x), std::fabs(pos.y)), std::fabs(pos.z)),
                               std::fabs(U.spin));
  if (!finite(scale) || scale == 0.0f) return bad_geometry(kBadDenominator);
  const float is = 1.0f / scale;
  const V3 c = is * pos;
  const float a = U.spin * is, a2 = a * a;
  const float m = U.mass * is, q = U.charge * is;
  Geometry g;
  g.inv_scale = is;
  if (c.x == 0.0f && c.y == 0.0f) {
    const float r = std::fabs(c.z), sigma = r * r + a2;
    if (r <= 0.0f || sigma <= 0.0f || !finite(sigma)) return bad_geometry(kBadDenominator);
    const float s = wgsl_sign(c.z);
    const float inv_sigma = 1.0f / sigma;
    g.f = (2.0f * m * r - q * q) * inv_sigma;
    g.dr = {0.0f, 0.0f, s};
    const V3 dsigma{0.0f, 0.0f, 2.0f * r * s};
    g.df = (inv_sigma * is) * ((2.0f * m) * g.dr - g.f * dsigma);
    g.l = {0.0f, 0.0f, U.chart * s};
    g.inv_r = 1.0f / r;
    g.inv_oblate = inv_sigma;
    g.radius = scale * r;
    if (!finite(g.radius) || !finite(g.f) || !finite(g.df) || !finite(g.inv_r) || !finite(g.inv_oblate))
      return bad_geometry(kNonFinite);
    return g;
  }
  const float rr3 = dot(c, c);
  const float off = rr3 - a2;
  const float rad = off * off + 4.0f * a2 * c.z * c.z;
  if (rad < 0.0f || !finite(rad)) return bad_geometry(kBadRadicand);
  const float sigma = std::sqrt(rad);
  float r2;
  if (off >= 0.0f) {
    r2 = 0.5f * (off + sigma);
  } else {
    const float den = sigma - off;
    if (den <= 0.0f || !finite(den)) return bad_geometry(kBadDenominator);
    r2 = 2.0f * a2 * c.z * c.z / den;
  }
  if (r2 <= 0.0f || !finite(r2)) return bad_geometry(kBadDenominator);
  const float r = std::sqrt(r2);
  if (r <= 0.0f || sigma <= 0.0f || !finite(sigma)) return bad_geometry(kBadDenominator);
  const float inv_r = 1.0f / r, inv_sigma = 1.0f / sigma;
  const float rs = r * inv_sigma;
  g.dr = {c.x * rs, c.y * rs, c.z * (r2 + a2) * inv_r * inv_sigma};
  g.f = (2.0f * m * r - q * q) * inv_sigma;
  const V3 dsigma = (2.0f * inv_sigma) * V3{off * c.x, off * c.y, c.z * (rr3 + a2)};
  g.df = (inv_sigma * is) * ((2.0f * m) * g.dr - g.f * dsigma);
  const float oblate = r2 + a2;
  if (oblate <= 0.0f || !finite(oblate)) return bad_geometry(kBadDenominator);
  const float io = 1.0f / oblate;
  const float ca = U.chart * a;
  g.l = U.chart * V3{(r * c.x + ca * c.y) * io, (r * c.y + ca * -c.x) * io, c.z * inv_r};
  g.inv_r = inv_r;
  g.inv_oblate = io;
  g.radius = scale * r;
  if (!finite(g.radius) || !finite(g.f) || !finite(g.df) || !finite(g.l) || !finite(g.dr) || !finite(is) ||
      !finite(g.inv_r) || !finite(g.inv_oblate))
    return bad_geometry(kNonFinite);
  return g;
}

// Geometry plus the singularity measure r^4 + a^2 z^2 that event tests need (165-175).
inline Geometry event_geometry(const Uniforms& U, V3 pos) {
  Geometry g = metric_geometry(U, pos);
  if (g.flags == 0) g.sing = sat_sum(sat_square(sat_square(g.radius)), sat_square(sat_product(std::fabs(U.spin), std::fabs(pos.z))));
  return g;
}

// p . d(l)/dx contracted with the principal null direction's gradient (211-235).
inline V3 principal_gradient(const Uniforms& U, const State& s, const Geometry& g) {
  const float is = g.inv_scale;
  const V3 c = is * s.x;
  const float r = g.radius * is, a = U.spin * is, ca = U.chart * a;
  const float ir2 = g.inv_r * g.inv_r, io = g.inv_oblate;
  const V3 p = s.p, lu = U.chart * g.l;
  const float radial = ((c.x * p.x + c.y * p.y) - 2.0f * r * (lu.x * p.x + lu.y * p.y)) * io - c.z * p.z * ir2;
  const V3 direct{(r * p.x + ca * -p.y) * io, (r * p.y + ca * p.x) * io, p.z * g.inv_r};
  return (U.chart * is) * (direct + radial * g.dr);
}

// Reduced Hamiltonian right-hand side at fixed E = -p_t (237-260).
inline Rhs hamilton_rhs(const Uniforms& U, const State& s, float E, const Geometry& g) {
  Rhs d;
  if (g.flags != 0) {
    d.flags = g.flags;
    return d;
  }
  const float k = E + dot(s.p, g.l);
  const float fk = g.f * k;
  d.xdot = s.p - fk * g.l;
  d.tdot = E + fk;
  d.pdot = fk * principal_gradient(U, s, g) + (0.5f * k * k) * g.df;
  if (!finite(d.xdot) || !finite(d.pdot) || !finite(d.tdot)) {
    Rhs bad;
    bad.flags = kNonFinite;
    return bad;
  }
  return d;
}

inline State advance(const State& s, const Rhs& d, float h) { return {s.x + h * d.xdot, s.p + h * d.pdot}; }

// One classical RK4 step of size h from s, with k1 the slope at s (282-317). Intermediate stages
// use the metric geometry only (no singularity measure).
inline uint32_t rk4_step(const Uniforms& U, const State& s, float E, const Rhs& k1, float h, State& next, float& dt) {
  if (k1.flags) return k1.flags;
  const State s1 = advance(s, k1, 0.5f * h);
  Rhs st = hamilton_rhs(U, s1, E, metric_geometry(U, s1.x));
  if (st.flags) return st.flags;
  float wt = k1.tdot + 2.0f * st.tdot;
  V3 wx = k1.xdot + 2.0f * st.xdot, wp = k1.pdot + 2.0f * st.pdot;
  const State s2 = advance(s, st, 0.5f * h);
  st = hamilton_rhs(U, s2, E, metric_geometry(U, s2.x));
  if (st.flags) return st.flags;
  wt = wt + 2.0f * st.tdot;
  wx = wx + 2.0f * st.xdot;
  wp = wp + 2.0f * st.pdot;
  const State s3 = advance(s, st, h);
  st = hamilton_rhs(U, s3, E, metric_geometry(U, s3.x));
  if (st.flags) return st.flags;
  wt = wt + st.tdot;
  wx = wx + st.xdot;
  wp = wp + st.pdot;
  const float w = h / 6.0f;
  next = {s.x + w * wx, s.p + w * wp};
  dt = w * wt;
  if (!finite(next.x) || !finite(next.p) || !finite(dt)) return kNonFinite;
  return 0;
}

// Cubic Hermite interpolation over a step (geodesic_events.wgsl:3-45).
struct Weights {
  float w0, w1, w2, w3;
};
inline Weights hermite_weights(float h, float u) {
  const float u2 = u * u, u3 = u2 * u;
  return {2.0f * u3 - 3.0f * u2 + 1.0f, h * (u3 - 2.0f * u2 + u), -2.0f * u3 + 3.0f * u2, h * (u3 - u2)};
}
inline State dense_state(const State& a, const State& b, const Rhs& da, const Rhs& db, const Weights& w) {
  return {w.w0 * a.x + w.w1 * da.xdot + w.w2 * b.x + w.w3 * db.xdot,
          w.w0 * a.p + w.w1 * da.pdot + w.w2 * b.p + w.w3 * db.pdot};
}
inline float dense_time(float dt, const Rhs& da, const Rhs& db, const Weights& w) {
  return w.w1 * da.tdot + w.w2 * dt + w.w3 * db.tdot;
}

// Slope of an event function along the step, per unit affine parameter (47-64).
inline float event_slope(const Uniforms& U, uint32_t term, const State& s, const Geometry& g, const Rhs& d) {
  if (term == kSurface) return d.xdot.z;
  const float vr = dot(g.dr, d.xdot);
  if (term != kSingularity) return vr;
  const float r = g.radius;
  return 4.0f * r * r * r * vr + 2.0f * U.spin * U.spin * s.x.z * d.xdot.z;
}

// Root fraction of an event residual over a step: the chord, refined by safeguarded Newton on the
// cubic Hermite residual when the slopes are monotone and well scaled (66-161).
inline float event_fraction(float e0, float e1, float s0, float s1) {
  const float span = e1 - e0;
  const float chord = std::min(std::max(-e0 / span, 0.0f), 1.0f);
  if (!finite(s0) || !finite(s1)) return chord;
  const float mid = 3.0f * span - s0 - s1;
  if (!finite(mid)) return chord;
  const float sg = wgsl_sign(span);
  const float c0 = sg * s0, c1 = sg * mid, c2 = sg * s1;
  if (c0 < 0.0f || c1 < 0.0f || c2 < 0.0f) return chord;
  const float k3 = 2.0f * (e0 - e1) + s0 + s1, k2 = 3.0f * (e1 - e0) - 2.0f * s0 - s1, k1 = s0, k0 = e0;
  const float floor_ = kDerivativeFloor * std::max(std::fabs(span), std::max(std::max(c0, c1), c2));
  float lo = 0.0f, hi = 1.0f, u = chord;
  const bool start_positive = e0 > 0.0f;
  for (int it = 0; it < kEventIterations; ++it) {
    const float cur = u;
    const float val = ((k3 * cur + k2) * cur + k1) * cur + k0;
    const float der = (3.0f * k3 * cur + 2.0f * k2) * cur + k1;
    if (!finite(val)) return chord;
    if (val == 0.0f) return cur;
    if ((val > 0.0f) == start_positive)
      lo = cur;
    else
      hi = cur;
    if (!finite(der) || std::fabs(der) <= floor_) return chord;
    u = 0.5f * (lo + hi);
    const float newton = cur - val / der;
    if (finite(newton) && newton > lo && newton < hi) u = newton;
  }
  return u;
}

struct Selection {
  uint32_t termination = 0;
  float fraction = 2.0f;
  uint32_t candidates = 0;
  bool ambiguous = false;
};

// Earliest candidate in protocol order (singularity, horizon, surface, escape; strict '<'), and the
// candidates within the tie tolerance of it in affine distance (200-248).
inline Selection select_earliest(const float ev[4], float step_magnitude, float tie) {
  static const uint32_t kTerm[4] = {kSingularity, kHorizon, kSurface, kEscape};
  static const uint32_t kBit[4] = {kCandSingularity, kCandHorizon, kCandSurface, kCandEscape};
  int best = 0;
  for (int i = 1; i < 4; ++i)
    if (ev[i] < ev[best]) best = i;
  Selection sel;
  sel.fraction = ev[best];
  if (sel.fraction > 1.0f) return sel;
  int n = 0;
  for (int i = 0; i < 4; ++i)
    if (ev[i] <= 1.0f && std::fabs(ev[i] - sel.fraction) * step_magnitude <= tie) {
      sel.candidates |= kBit[i];
      ++n;
    }
  sel.termination = kTerm[best];
  sel.ambiguous = n > 1;
  return sel;
}

// Null residual, E, L_z and Carter's constant at a state (346-391).
struct Invariants {
  float v[4] = {0, 0, 0, 0};
  uint32_t flags = 0;
};
inline Invariants invariants(const Uniforms& U, const State& s, float E, const Geometry& g, const Rhs& d) {
  Invariants out;
  if (g.flags || d.flags) {
    out.flags = g.flags | d.flags;
    return out;
  }
  const float a2 = U.spin * U.spin, r = g.radius, r2 = r * r;
  const float oblate = r2 + a2;
  if (oblate <= 0.0f || !finite(oblate)) {
    out.flags = kBadDenominator;
    return out;
  }
  const float lz = s.x.x * s.p.y - s.x.y * s.p.x;
  const float proj = s.x.x * s.p.x + s.x.y * s.p.y;
  const float pt2 = s.p.x * s.p.x + s.p.y * s.p.y;
  const V3 c = g.inv_scale * s.x;
  const float cosine = c.z * g.inv_r;
  const float w0 = cosine * cosine, w1 = (c.x * c.x + c.y * c.y) * g.inv_oblate;
  const float carter = w0 * (oblate * pt2 - a2 * E * E) - 2.0f * s.x.z * proj * s.p.z + r2 * w1 * s.p.z * s.p.z;
  const float contraction = -E * d.tdot + dot(s.p, d.xdot);
  const float norm = std::fabs(E * d.tdot) +
                     (std::fabs(s.p.x) * std::fabs(d.xdot.x) + std::fabs(s.p.y) * std::fabs(d.xdot.y) +
                      std::fabs(s.p.z) * std::fabs(d.xdot.z));
  out.v[0] = std::fabs(contraction) / std::max(1.0f, norm);
  out.v[1] = E;
  out.v[2] = lz;
  out.v[3] = carter;
  for (float x : out.v)
    if (!finite(x)) {
      Invariants bad;
      bad.flags = kNonFinite;
      return bad;
    }
  return out;
}
inline void accumulate_drift(float drift[4], const float v0[4], const float v[4]) {
  const float cur[4] = {v[0], 0.0f, std::fabs(v[2] - v0[2]) / std::max(1.0f, std::fabs(v0[2])),
                        std::fabs(v[3] - v0[3]) / std::max(1.0f, std::fabs(v0[3]))};
  for (int i = 0; i < 4; ++i) drift[i] = std::max(drift[i], cur[i]);
}

// Keplerian prograde emitter at the hit: (radius, source azimuth, g) (254-311).
inline uint32_t surface_source(const Uniforms& U, const State& s, const Geometry& g, const Invariants& inv,
                               float out[3]) {
  const float r = g.radius, a = U.spin, q2 = U.charge * U.charge;
  const float root2 = r - q2;
  if (root2 < 0.0f || !finite(root2)) return kBadRadicand;
  const float root = std::sqrt(root2);
  const float branch = a >= 0.0f ? 1.0f : -1.0f;
  const float r2 = r * r;
  const float den = r2 + branch * a * root;
  if (den <= 0.0f || !finite(den)) return kBadDenominator;
  const float omega = branch * root / den;
  const float num = 2.0f * r - q2, a2 = a * a;
  const float timelike = r2 - 3.0f * r + 2.0f * q2 + 2.0f * branch * a * root;
  if (timelike <= 0.0f || !finite(timelike)) return kBadDenominator;
  const float delta = r2 - 2.0f * r + a2 + q2;
  const float gtt = -1.0f + num / r2, gtp = -num * a / r2, rf = r2 + a2;
  const float gpp = (rf * rf - a2 * delta) / r2;
  const float norm2 = gtt + 2.0f * gtp * omega + gpp * omega * omega;
  if (norm2 >= 0.0f || !finite(norm2)) return kBadDenominator;
  const float ut = 1.0f / std::sqrt(-norm2);
  const float emitted = ut * (inv.v[1] - omega * inv.v[2]);
  if (emitted <= 0.0f || !finite(emitted)) return kBadDenominator;
  const float ratio = U.frequency / emitted;
  const float raw = std::atan2(s.x.y, s.x.x) - std::atan2(U.chart * a, r);
  const float pi = 3.141592653589793f, tau = 6.283185307179586f;
  const float azimuth = raw - tau * std::floor((raw + pi) / tau);
  if (ratio <= 0.0f || !finite(r) || !finite(azimuth) || !finite(ratio)) return kNonFinite;
  out[0] = r;
  out[1] = azimuth;
  out[2] = ratio;
  return 0;
}

inline float radial_velocity(const Geometry& g, const Rhs& d) { return -dot(g.dr, d.xdot); }

// Bisection bracket of a radial turning point on the dense output (417-490); valid == false when a
// sample fails.
inline bool turning_bracket(const Uniforms& U, const State& a, const State& b, const Rhs& da, const Rhs& db, float E,
                            float h, float v0, float& lo, float& hi) {
  lo = 0.0f;
  hi = 1.0f;
  float vlo = v0;
  for (int it = 0; it < kTurningIterations; ++it) {
    const float mid = 0.5f * (lo + hi);
    if (mid == lo || mid == hi) break;
    const State s = dense_state(a, b, da, db, hermite_weights(h, mid));
    if (!finite(s.x) || !finite(s.p)) return false;
    const Geometry g = event_geometry(U, s.x);
    const Rhs d = hamilton_rhs(U, s, E, g);
    if (g.flags || d.flags) return false;
    const float v = radial_velocity(g, d);
    if (!finite(v)) return false;
    if (v == 0.0f) {
      lo = hi = mid;
      return true;
    }
    if ((v < 0.0f) == (vlo < 0.0f)) {
      lo = mid;
      vlo = v;
    } else {
      hi = mid;
    }
  }
  return true;
}

inline int32_t update_winding(float previous, V3 pos, int32_t winding) {
  const float diff = std::atan2(pos.y, pos.x) - previous;
  if (diff > 3.141592653589793f) return winding - 1;
  if (diff < -3.141592653589793f) return winding + 1;
  return winding;
}

struct Result {
  uint32_t termination = 0, flags = 0, candidates = 0, steps = 0;
  float event_residual = 0.0f;
  float source[3] = {0, 0, 0};  // escape: unit -dx/dlambda; surface: (radius, azimuth, g)
  float travel_time = 0.0f;
  float drift[4] = {0, 0, 0, 0};
  uint32_t turnings = 0, crossings = 0;
  int32_t winding = 0;
};

inline Result failure(uint32_t flags, uint32_t steps, float travel_time, const float drift[4]) {
  Result r;
  r.termination = kFailure;
  r.flags = flags;
  r.steps = steps;
  r.travel_time = travel_time;
  for (int i = 0; i < 4; ++i) r.drift[i] = drift[i];
  return r;
}

inline uint32_t bump(uint32_t v) { return v == 0xffffffffu ? v : v + 1u; }

// One pixel: initial null covector at the observer (sight_direction, lower_momentum,
// initial_state_at: kerr_schild_dynamics.wgsl:177-205, geodesic_events.wgsl:313-344), then the
// fixed-step RK4 loop with h = clamp(0.1 r, 0.005, 8) traced backward in affine parameter.
inline Result trace_pixel(const Uniforms& U, uint32_t width, uint32_t height, uint32_t px, uint32_t py, float sx,
                          float sy) {
  const float zero4[4] = {0, 0, 0, 0};
  const float W = float(width), H = float(height);
  const float nx = 2.0f * (float(px) + sx) / W - 1.0f;
  const float ny = 1.0f - 2.0f * (float(py) + sy) / H;
  const float spx = W / H * U.tan_half_fov * nx, spy = U.tan_half_fov * ny;
  const float il = 1.0f / std::sqrt(1.0f + (spx * spx + spy * spy));
  float pu[4];
  for (int m = 0; m < 4; ++m) {
    const float sight = (spx * U.right[m] + spy * U.up[m] - U.arrival[m]) * il;
    pu[m] = U.frequency * (U.velocity[m] + -sight);
  }
  Geometry g = event_geometry(U, U.observer);
  uint32_t fl = g.flags;
  for (float v : pu)
    if (!finite(v)) fl |= kNonFinite;
  if (fl) return failure(fl, 0, 0.0f, zero4);
  const float contraction = pu[0] + g.l.x * pu[1] + g.l.y * pu[2] + g.l.z * pu[3];
  const float fc = g.f * contraction;
  const float pt = -pu[0] + fc;
  const V3 p{pu[1] + fc * g.l.x, pu[2] + fc * g.l.y, pu[3] + fc * g.l.z};
  if (!finite(pt) || !finite(p)) return failure(kNonFinite, 0, 0.0f, zero4);
  const float E = -pt;
  State s{U.observer, p};
  Rhs d = hamilton_rhs(U, s, E, g);
  if (d.flags) return failure(d.flags, 0, 0.0f, zero4);
  const Invariants inv0 = invariants(U, s, E, g, d);
  if (inv0.flags) return failure(inv0.flags, 0, 0.0f, zero4);

  float drift[4] = {inv0.v[0], 0.0f, 0.0f, 0.0f};
  float travel = 0.0f;
  uint32_t turnings = 0, crossings = 0;
  int32_t winding = 0;
  float prev_azimuth = std::atan2(s.x.y, s.x.x);
  bool armed = U.surface && std::fabs(s.x.z) > U.arming;
  for (uint32_t step = 0; step < kMaxSteps; ++step) {
    const Geometry g0 = g;
    if (g0.flags) return failure(g0.flags, step, travel, drift);
    if (g0.sing <= U.guard) {
      Result r;
      r.termination = kSingularity;
      r.candidates = kCandSingularity;
      r.steps = step;
      r.event_residual = (g0.sing - U.guard) / std::max(1.0f, U.guard);
      r.travel_time = travel;
      for (int i = 0; i < 4; ++i) r.drift[i] = drift[i];
      r.turnings = turnings;
      r.crossings = crossings;
      r.winding = winding;
      return r;
    }
    const float hm = std::min(std::max(U.step_scale * g0.radius, U.step_min), U.step_max);
    const float h = -hm;
    State s1;
    float dt = 0.0f;
    if (const uint32_t f = rk4_step(U, s, E, d, h, s1, dt)) return failure(f, step, travel, drift);
    const Geometry g1 = event_geometry(U, s1.x);
    if (g1.flags) return failure(g1.flags, step + 1, travel, drift);
    const Rhs d1 = hamilton_rhs(U, s1, E, g1);
    if (d1.flags) return failure(d1.flags, step + 1, travel, drift);
    const float v0 = radial_velocity(g0, d), v1 = radial_velocity(g1, d1);
    const bool turning = (v0 < 0.0f && v1 >= 0.0f) || (v0 > 0.0f && v1 <= 0.0f);
    float ev[4] = {2.0f, 2.0f, 2.0f, 2.0f};
    if (g1.sing <= U.guard)
      ev[0] = event_fraction(g0.sing - U.guard, g1.sing - U.guard, h * event_slope(U, kSingularity, s, g0, d),
                             h * event_slope(U, kSingularity, s1, g1, d1));
    if (U.horizon > 0.0f && g0.radius > U.horizon && g1.radius <= U.horizon)
      ev[1] = event_fraction(g0.radius - U.horizon, g1.radius - U.horizon, h * event_slope(U, kHorizon, s, g0, d),
                             h * event_slope(U, kHorizon, s1, g1, d1));
    if (g0.radius < U.escape && g1.radius >= U.escape)
      ev[3] = event_fraction(g0.radius - U.escape, g1.radius - U.escape, h * event_slope(U, kEscape, s, g0, d),
                             h * event_slope(U, kEscape, s1, g1, d1));
    const bool crosses = U.surface && ((s.x.z > 0.0f && s1.x.z <= 0.0f) || (s.x.z < 0.0f && s1.x.z >= 0.0f));
    float crossing_fraction = 2.0f;
    if (crosses) {
      const float u = event_fraction(s.x.z, s1.x.z, h * d.xdot.z, h * d1.xdot.z);
      crossing_fraction = u;
      if (armed) {
        const State ss = dense_state(s, s1, d, d1, hermite_weights(h, u));
        const Geometry gs = event_geometry(U, ss.x);
        if (gs.flags) return failure(gs.flags, step + 1, travel, drift);
        if (gs.radius >= U.inner && gs.radius <= U.outer) ev[2] = u;
      }
    }
    const Selection sel = select_earliest(ev, hm, U.tie);
    if (sel.termination != 0) {
      const Weights w = hermite_weights(h, sel.fraction);
      const State se = dense_state(s, s1, d, d1, w);
      const float te = dense_time(dt, d, d1, w);
      if (!finite(te)) return failure(kNonFinite, step + 1, travel, drift);
      const Geometry ge = event_geometry(U, se.x);
      const Rhs de = hamilton_rhs(U, se, E, ge);
      const Invariants ie = invariants(U, se, E, ge, de);
      if (const uint32_t f = ge.flags | de.flags | ie.flags) return failure(f, step + 1, travel, drift);
      Result r;
      r.travel_time = travel + std::fabs(te);
      for (int i = 0; i < 4; ++i) r.drift[i] = drift[i];
      accumulate_drift(r.drift, inv0.v, ie.v);
      if (!sel.ambiguous && sel.termination == kEscape) {
        const V3 m = -1.0f * de.xdot;
        const float len = std::sqrt(dot(m, m));
        r.source[0] = m.x / len;
        r.source[1] = m.y / len;
        r.source[2] = m.z / len;
      } else if (!sel.ambiguous && sel.termination == kSurface) {
        if (const uint32_t f = surface_source(U, se, ge, ie, r.source)) return failure(f, step + 1, travel, drift);
      }
      const bool is_sing = sel.termination == kSingularity, is_hor = sel.termination == kHorizon;
      const bool is_surf = sel.termination == kSurface;
      const float value = is_surf ? se.x.z : (is_sing ? ge.sing : ge.radius);
      const float target = is_surf ? 0.0f : (is_sing ? U.guard : (is_hor ? U.horizon : U.escape));
      r.event_residual = (value - target) / std::max(1.0f, std::fabs(target));
      uint32_t turn_count = turnings;
      bool turn_uncertain = false;
      if (turning) {
        float lo, hi;
        if (!turning_bracket(U, s, s1, d, d1, E, h, v0, lo, hi))
          turn_uncertain = true;
        else if (hi < sel.fraction)
          turn_count = bump(turn_count);
        else if (lo < sel.fraction)
          turn_uncertain = true;
      }
      r.crossings = crossing_fraction < sel.fraction ? bump(crossings) : crossings;
      bool over_budget = false;
      for (float x : r.drift) over_budget = over_budget || x > U.drift_limit;
      r.termination = (sel.ambiguous || turn_uncertain || over_budget) ? kUncertain : sel.termination;
      r.candidates = sel.candidates;
      r.steps = step + 1;
      r.turnings = turn_count;
      r.winding = update_winding(prev_azimuth, se.x, winding);
      return r;
    }
    const Invariants i1 = invariants(U, s1, E, g1, d1);
    if (i1.flags) return failure(i1.flags, step + 1, travel, drift);
    travel = travel + std::fabs(dt);
    accumulate_drift(drift, inv0.v, i1.v);
    if (turning) turnings = bump(turnings);
    if (crossing_fraction <= 1.0f) crossings = bump(crossings);
    winding = update_winding(prev_azimuth, s1.x, winding);
    prev_azimuth = std::atan2(s1.x.y, s1.x.x);
    if (U.surface) armed = armed || std::fabs(s1.x.z) > U.arming;
    s = s1;
    g = g1;
    d = d1;
  }
  Result r;
  r.termination = kStepExhaustion;
  r.steps = kMaxSteps;
  r.travel_time = travel;
  for (int i = 0; i < 4; ++i) r.drift[i] = drift[i];
  r.turnings = turnings;
  r.crossings = crossings;
  r.winding = winding;
  return r;
}

}  // namespace rk4
}  // namespace gro
