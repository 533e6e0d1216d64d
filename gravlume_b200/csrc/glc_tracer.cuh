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
#pragma once

#include "glc_dp54.cuh"
#include "../../include/glc.h"

namespace glc {

enum Prec : int { kFP32 = 0, kMIXED = 1, kFP64 = 2 };

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

enum EventBit : uint32_t { kEvGuard = 0, kEvHorizon = 1, kEvSurface = 2, kEvEscape = 3 };

enum FlagBit : uint32_t {
  kFlagShellF64 = 1u << 0,     // MIXED: some steps ran in binary64
  kFlagRenormalized = 1u << 1, // MIXED: final momentum renormalized onto H = 0
  kFlagSurfaceInvalid = 1u << 2,  // surface hit but the circular emitter observable is undefined
  kFlagNoEscapeDirection = 1u << 3,
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
};

GLC_HD LaneScene make_lane_scene(const glc_scene& s, double shell_factor) {
  LaneScene ls;
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

// Result of one ray, written by the tracer into the caller's SoA.
template <class S>
struct RayResult {
  uint32_t termination, failure, candidates, flags;
  S event_residual;
  S y[6];
  S escape_theta, escape_phi;
  S surface_r, surface_phi, g;
};

// Bisection on the dense output (geodesic.rs:640-676). value_at(y, v) -> false on failure.
template <class T, class F>
GLC_HD bool localize(const T y0[6], T h, const T K[7][7], T tol, T sv, T ev, F value_at, T& theta, T yroot[6],
                     T& bracket) {
  T lower = T(0), upper = T(1), lv = sv, uv = ev;
  const T ah = g_abs(h);
  for (int i = 0; i < 64; ++i) {
    if ((upper - lower) * ah <= tol) break;
    const T mid = T(0.5) * (lower + upper);
    if (mid == lower || mid == upper) break;
    T ys[6], dt;
    dense_eval(y0, h, K, mid, ys, dt);
    T v;
    if (!value_at(ys, v)) return false;
    if (g_signbit(lv) == g_signbit(v)) {
      lower = mid;
      lv = v;
    } else {
      upper = mid;
      uv = v;
    }
  }
  theta = g_abs(lv) <= g_abs(uv) ? lower : upper;
  T dt;
  dense_eval(y0, h, K, theta, yroot, dt);
  bracket = (upper - lower) * ah;
  for (int c = 0; c < 6; ++c)
    if (!g_finite(yroot[c])) return false;
  return true;
}

// Keplerian prograde circular emitter observable (surface.rs:75-146, M = 1). Returns false when
// the orbit is unavailable or not timelike.
template <class T>
GLC_HD bool surface_observable(const LaneScene& sc, const T y[6], T E, T r, T& g, T& phi_s) {
  const T a = T(sc.kn.a), q2 = T(sc.kn.q2), a2 = T(sc.kn.a2);
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
  g = T(sc.frequency) / ef;
  phi_s = wrapped_angle(g_atan2(y[1], y[0]), g_atan2(T(sc.kn.sa), r));
  return g_finite(g) && g > T(0);
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

// ----------------------------------------------------------------------------------------------
template <int P>
struct Ray {
  using S = typename PrecTraits<P>::S;
  using C = typename PrecTraits<P>::C;

  S y[6];
  S E;
  S h;
  S affine;
  S tsum, tcorr;
  S k1[7];
  S r, vr;
  S lz0, q0, dnull, dlz, dq;
  S az_prev, az_adv;
  S turn_r;
  S dir;
  uint32_t accepted, rejected, f64steps, consecutive;
  uint32_t armed;
  uint32_t k1_f64;
  uint32_t turnings, crossings;
  int32_t winding, polar;
  uint32_t flags;
  bool have_inv;

  // Initial state: y (position, covariant spatial momentum) and energy E = -p_t.
  GLC_HD void init(const LaneScene& sc, const glc_policy& pol, const double st8[8], double direction) {
    for (int c = 0; c < 3; ++c) {
      y[c] = S(st8[1 + c]);
      y[3 + c] = S(st8[5 + c]);
    }
    E = S(-st8[4]);
    dir = S(direction);
    h = dir * S(pol.initial_step);
    affine = S(0);
    tsum = S(0);
    tcorr = S(0);
    accepted = rejected = f64steps = consecutive = 0;
    turnings = crossings = 0;
    winding = 0;
    flags = 0;
    polar = st8[3] > 0.0 ? 1 : (st8[3] < 0.0 ? -1 : 0);
    turn_r = S(NAN);
    az_prev = g_atan2(y[1], y[0]);
    az_adv = S(0);
    dnull = dlz = dq = S(0);
    const KN<S> ks = kn_cast<S>(sc.kn);
    int gs;
    const S r0 = kn_radius(ks, y[0], y[1], y[2], gs);
    // initial invariants (geodesic.rs:101) and arming (geodesic.rs:536-544)
    have_inv = gs == kGeomOk;
    armed = 0;
    if (have_inv) {
      const Invariants<S> inv = kn_invariants(ks, y, E, r0);
      lz0 = inv.lz;
      q0 = inv.carter;
      have_inv = g_finite(inv.lz) && g_finite(inv.carter) && g_finite(inv.null_residual);
      for (int kind = 0; kind < 4; ++kind) {
        const S v = event_value<S>(kind, sc, pol.singularity_guard, r0, y[2]);
        if (event_clears_band(kind, v, S(pol.event_arming_band))) armed |= 1u << kind;
      }
    }
    // first derivative (FSAL seed)
    const KN<C> kc = kn_cast<C>(sc.kn);
    C yc[6], d[7], rr, vv;
    for (int c = 0; c < 6; ++c) yc[c] = C(y[c]);
    kn_rhs(kc, yc, C(E), d, rr, vv);
    for (int c = 0; c < 7; ++c) k1[c] = S(d[c]);
    r = S(rr);
    vr = S(vv);
    k1_f64 = (P == kFP64) ? 1u : 0u;
    if (have_inv) update_invariants(sc, y, r0);
  }

  GLC_HD void update_invariants(const LaneScene& sc, const S yy[6], S rr) {
    if (!have_inv) return;
    const Invariants<S> inv = kn_invariants(kn_cast<S>(sc.kn), yy, E, rr);
    if (g_finite(inv.null_residual)) dnull = g_max(dnull, inv.null_residual);
    if (g_finite(inv.lz)) dlz = g_max(dlz, g_abs(inv.lz - lz0) / g_max(g_abs(lz0), S(1)));
    if (g_finite(inv.carter)) dq = g_max(dq, g_abs(inv.carter - q0) / g_max(g_abs(q0), S(1)));
  }

  GLC_HD S next_step(const glc_policy& pol, S mag, S en, bool accepted_step) const {
    const S maxf = accepted_step ? S(pol.maximum_factor) : S(1);
    S factor;
    if (en == S(0)) {
      factor = maxf;
    } else {
      factor = S(pol.safety) * g_pow_m02(en);
      factor = factor < S(pol.minimum_factor) ? S(pol.minimum_factor) : (factor > maxf ? maxf : factor);
    }
    S hn = mag * factor;
    hn = hn < S(pol.minimum_step) ? S(pol.minimum_step) : (hn > S(pol.maximum_step) ? S(pol.maximum_step) : hn);
    return hn;
  }

  GLC_HD void commit_azimuth(const S yy[6]) {
    const S az = g_atan2(yy[1], yy[0]);
    const S raw = az - az_prev;
    const S pi = S(3.14159265358979323846);
    az_adv += wrapped_angle(az, az_prev);
    if (raw > pi) winding -= 1;
    else if (raw < -pi) winding += 1;
    az_prev = az;
  }

  // Compute one attempt in precision CC; results are returned in S.
  template <class CC>
  GLC_HD void attempt(const LaneScene& sc, S inc[6], S& dt, S err[7], S k7[7], S& r_end, S& vr_end, bool recompute_k1) {
    const KN<CC> kc = kn_cast<CC>(sc.kn);
    CC k1c[7];
    if (recompute_k1) {
      CC yc[6], rr, vv;
      for (int c = 0; c < 6; ++c) yc[c] = CC(y[c]);
      kn_rhs(kc, yc, CC(E), k1c, rr, vv);
    } else {
      for (int c = 0; c < 7; ++c) k1c[c] = CC(k1[c]);
    }
    CC incc[6], dtc, errc[7], k7c[7], rc, vc;
    dp5_attempt<CC, S>(kc, y, CC(E), CC(h), k1c, incc, dtc, errc, k7c, rc, vc);
    for (int c = 0; c < 6; ++c) inc[c] = S(incc[c]);
    for (int c = 0; c < 7; ++c) {
      err[c] = S(errc[c]);
      k7[c] = S(k7c[c]);
    }
    dt = S(dtc);
    r_end = S(rc);
    vr_end = S(vc);
  }

  // Advance by one attempted step. Returns true when the ray terminated (result filled).
  template <bool kUse64>
  GLC_HD bool step(const LaneScene& sc, const glc_policy& pol, RayResult<S>& res) {
    if (uint64_t(accepted) >= pol.maximum_accepted_steps) {
      finish_plain(res, GLC_TERM_STEP_EXHAUSTION, GLC_FAIL_NONE);
      return true;
    }
    S inc[6], dt, err[7], k7[7], r_end, vr_end;
    bool stepped64 = false;
    if (P == kMIXED && kUse64) {
      attempt<double>(sc, inc, dt, err, k7, r_end, vr_end, k1_f64 == 0u);
      stepped64 = true;
    } else {
      attempt<C>(sc, inc, dt, err, k7, r_end, vr_end, false);
    }
    // grouped infinity norm with the relative coordinate time (geodesic.rs:158-165)
    const S t_start = tsum + tcorr;
    S en = S(0);
    bool finite = g_finite(dt) && g_finite(r_end);
    for (int c = 0; c < 7; ++c) {
      S sc_, ec;
      if (c < 6) {
        sc_ = y[c];
        ec = y[c] + inc[c];
      } else {
        sc_ = t_start;
        ec = t_start + dt;
      }
      const bool pos = (c < 3) || (c == 6);
      const S rtol = pos ? S(pol.position_rtol) : S(pol.momentum_rtol);
      const S atol = pos ? S(pol.position_atol) : S(pol.momentum_atol);
      const S scale = rtol * g_max(g_abs(sc_), g_abs(ec)) + atol;
      const S q = g_abs(err[c]) / scale;
      finite = finite && g_finite(err[c]) && g_finite(inc[c > 5 ? 5 : c]);
      en = g_max(en, q);
    }
    if (!finite || !g_finite(en)) {
      finish_plain(res, GLC_TERM_NUMERICAL_FAILURE, GLC_FAIL_NON_FINITE);
      return true;
    }
    if (en > S(1)) {
      rejected += 1;
      consecutive += 1;
      if (consecutive >= pol.maximum_consecutive_rejects) {
        finish_plain(res, GLC_TERM_REJECT_EXHAUSTION, GLC_FAIL_NONE);
        return true;
      }
      if (g_abs(h) <= S(pol.minimum_step)) {
        finish_plain(res, GLC_TERM_NUMERICAL_FAILURE, GLC_FAIL_MINIMUM_STEP);
        return true;
      }
      h = dir * next_step(pol, g_abs(h), en, false);
      return false;
    }
    accepted += 1;
    consecutive = 0;
    if (stepped64) {
      f64steps += 1;
      flags |= kFlagShellF64;
    }
    S yend[6];
    for (int c = 0; c < 6; ++c) yend[c] = y[c] + inc[c];
    // ---- crossing detection at both ends (values from the FSAL evaluations)
    const double guard = pol.singularity_guard;
    uint32_t ev_mask = 0;
    for (int kind = 0; kind < 4; ++kind) {
      if (!((armed >> kind) & 1u) || !((sc.installed >> kind) & 1u)) continue;
      const S sv = event_value<S>(kind, sc, guard, r, y[2]);
      const S evv = event_value<S>(kind, sc, guard, r_end, yend[2]);
      if (event_crosses(kind, sv, evv)) ev_mask |= 1u << kind;
    }
    const S vs = dir * vr, ve = dir * vr_end;
    const bool turning = (vs < S(0) && ve >= S(0)) || (vs > S(0) && ve <= S(0));
    const bool equator = event_crosses(kEvSurface, y[2], yend[2]);
    if (ev_mask != 0u || turning || equator) {
      return rare_step(sc, pol, res, en);
    }
    // ---- plain commit
    CompSum::add(tsum, tcorr, dt);
    commit_azimuth(yend);
    S rc = r_end;
    if (P == kMIXED) {
      int gs;
      rc = kn_radius(kn_cast<S>(sc.kn), yend[0], yend[1], yend[2], gs);
    }
    update_invariants(sc, yend, rc);
    affine += h;
    for (int c = 0; c < 6; ++c) y[c] = yend[c];
    for (int c = 0; c < 7; ++c) k1[c] = k7[c];
    k1_f64 = (P == kFP64 || stepped64) ? 1u : 0u;
    r = r_end;
    vr = vr_end;
    arm_update(sc, pol);
    h = dir * next_step(pol, g_abs(h), en, true);
    return false;
  }

  GLC_HD void arm_update(const LaneScene& sc, const glc_policy& pol) {
    if (armed == 0xFu) return;
    for (int kind = 0; kind < 4; ++kind) {
      if ((armed >> kind) & 1u) continue;
      const S v = event_value<S>(kind, sc, pol.singularity_guard, r, y[2]);
      if (event_clears_band(kind, v, S(pol.event_arming_band))) armed |= 1u << kind;
    }
  }

  // Event path in S precision: recompute the stages for dense output, localize, commit.
  GLC_HD bool rare_step(const LaneScene& sc, const glc_policy& pol, RayResult<S>& res, S en) {
    using T = S;
    const KN<T> kt = kn_cast<T>(sc.kn);
    T K[7][7];
    T r0 = r, vr0 = vr;
    if (P == kMIXED && k1_f64 == 0u) {
      T rr, vv;
      kn_rhs(kt, y, E, K[0], rr, vv);
      r0 = rr;
      vr0 = vv;
    } else {
      for (int c = 0; c < 7; ++c) K[0][c] = k1[c];
    }
    const T hh = h;
    T yend[6], r_end, vr_end;
    dp5_stages(kt, y, E, hh, K, yend, r_end, vr_end);
    const double guard = pol.singularity_guard;
    const T tol = T(pol.event_affine_tolerance);
    bool fail = false;
    // events in the reference order: guard, horizon, surface, escape
    int n = 0;
    int kinds[4];
    T thetas[4], residuals[4], states[4][6];
    for (int kind = 0; kind < 4; ++kind) {
      if (!((armed >> kind) & 1u) || !((sc.installed >> kind) & 1u)) continue;
      const T sv = event_value<T>(kind, sc, guard, r0, y[2]);
      const T evv = event_value<T>(kind, sc, guard, r_end, yend[2]);
      if (!event_crosses(kind, sv, evv)) continue;
      T th, yr[6], br;
      auto value_at = [&](const T* ys, T& v) -> bool {
        int gs;
        const T rr = kind == kEvSurface ? T(0) : kn_radius(kt, ys[0], ys[1], ys[2], gs);
        if (kind != kEvSurface && gs != kGeomOk) return false;
        v = event_value<T>(kind, sc, guard, rr, ys[2]);
        return true;
      };
      if (!localize(y, hh, K, tol, sv, evv, value_at, th, yr, br)) {
        fail = true;
        break;
      }
      T rv;
      if (!value_at(yr, rv)) {
        fail = true;
        break;
      }
      bool keep = true;
      if (kind == kEvSurface) {
        int gs;
        const T rr = kn_radius(kt, yr[0], yr[1], yr[2], gs);
        keep = gs == kGeomOk && rr >= T(sc.surf_in) && rr <= T(sc.surf_out);
      }
      if (keep) {
        kinds[n] = kind;
        thetas[n] = th;
        residuals[n] = g_abs(rv) / T(event_scale(kind, sc));
        for (int c = 0; c < 6; ++c) states[n][c] = yr[c];
        ++n;
      }
    }
    if (fail) {
      finish_plain(res, GLC_TERM_NUMERICAL_FAILURE, GLC_FAIL_NON_FINITE);
      return true;
    }
    int first = -1;
    uint32_t cand = 0;
    for (int i = 0; i < n; ++i)
      if (first < 0 || thetas[i] < thetas[first]) first = i;
    if (first >= 0)
      for (int i = 0; i < n; ++i)
        if (g_abs(thetas[i] - thetas[first]) * g_abs(hh) <= T(pol.event_tie_tolerance)) cand |= 1u << kinds[i];
    const bool has_event = first >= 0;
    const T term_theta = has_event ? thetas[first] : T(1);
    // radial turning point (geodesic.rs:330-360)
    {
      const T sv = dir * vr0, evv = dir * vr_end;
      if ((sv < T(0) && evv >= T(0)) || (sv > T(0) && evv <= T(0))) {
        T th, yr[6], br;
        auto vr_at = [&](const T* ys, T& v) -> bool {
          T d[7], rr, vv;
          kn_rhs(kt, ys, E, d, rr, vv);
          v = dir * vv;
          return g_finite(v);
        };
        if (localize(y, hh, K, tol, sv, evv, vr_at, th, yr, br) && (!has_event || th < term_theta)) {
          turnings += 1;
          if (sv < T(0) && evv >= T(0)) {
            int gs;
            const T rr = kn_radius(kt, yr[0], yr[1], yr[2], gs);
            if (gs == kGeomOk) turn_r = (turn_r == turn_r) ? g_min(turn_r, rr) : rr;
          }
        }
      }
    }
    // equatorial crossing (geodesic.rs:362-383)
    if (event_crosses(kEvSurface, y[2], yend[2])) {
      T th, yr[6], br;
      auto z_at = [&](const T* ys, T& v) -> bool {
        v = ys[2];
        return true;
      };
      if (localize(y, hh, K, tol, y[2], yend[2], z_at, th, yr, br) && (!has_event || th < term_theta)) crossings += 1;
    }
    // commit at the terminal theta (or the step end)
    T ycommit[6], dtc;
    if (has_event) {
      T ytmp[6];
      dense_eval(y, hh, K, term_theta, ytmp, dtc);
      for (int c = 0; c < 6; ++c) ycommit[c] = states[first][c];
    } else {
      dense_eval(y, hh, K, T(1), ycommit, dtc);
      for (int c = 0; c < 6; ++c) ycommit[c] = yend[c];
    }
    CompSum::add(tsum, tcorr, dtc);
    commit_azimuth(ycommit);
    {
      int gs;
      const T rr = kn_radius(kt, ycommit[0], ycommit[1], ycommit[2], gs);
      if (gs == kGeomOk) update_invariants(sc, ycommit, rr);
    }
    if (has_event) {
      affine = hh * term_theta + affine;
      const int kind = kinds[first];
      uint32_t term = GLC_TERM_HORIZON;
      if (kind == kEvGuard) term = GLC_TERM_SINGULARITY;
      else if (kind == kEvSurface) term = GLC_TERM_SURFACE;
      else if (kind == kEvEscape) term = GLC_TERM_ESCAPE;
      finish_event(sc, pol, res, term, cand, residuals[first], ycommit);
      return true;
    }
    affine += hh;
    for (int c = 0; c < 6; ++c) y[c] = yend[c];
    for (int c = 0; c < 7; ++c) k1[c] = K[6][c];
    k1_f64 = (P == kFP32) ? 0u : 1u;
    r = r_end;
    vr = vr_end;
    arm_update(sc, pol);
    h = dir * next_step(pol, g_abs(h), en, true);
    return false;
  }

  GLC_HD void finish_plain(RayResult<S>& res, uint32_t term, uint32_t failure) {
    res.termination = term;
    res.failure = failure;
    res.candidates = 0;
    res.flags = flags;
    res.event_residual = S(NAN);
    for (int c = 0; c < 6; ++c) res.y[c] = y[c];
    res.escape_theta = res.escape_phi = S(NAN);
    res.surface_r = res.surface_phi = res.g = S(NAN);
  }

  GLC_HD void finish_event(const LaneScene& sc, const glc_policy& pol, RayResult<S>& res, uint32_t term,
                           uint32_t cand, S residual, S ye[6]) {
    using T = S;
    const KN<T> kt = kn_cast<T>(sc.kn);
    if (P == kMIXED && pol.renormalize_null) {
      if (renormalize_null(kt, ye, E)) flags |= kFlagRenormalized;
    }
    res.termination = term;
    res.failure = GLC_FAIL_NONE;
    res.candidates = cand;
    res.event_residual = residual;
    for (int c = 0; c < 6; ++c) res.y[c] = ye[c];
    res.escape_theta = res.escape_phi = S(NAN);
    res.surface_r = res.surface_phi = res.g = S(NAN);
    if (term == GLC_TERM_ESCAPE) {
      T d[7], rr, vv;
      kn_rhs(kt, ye, E, d, rr, vv);
      const T dx = dir * d[0], dy = dir * d[1], dz = dir * d[2];
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

}  // namespace glc
