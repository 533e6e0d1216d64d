// Host-side scene packing: validates a physical scene in the reference's terms and produces the
// binary64 glc_scene the kernels read.
//
// Mirrors TraceUniforms::from_observation_with_surface (crates/gravlume-render/src/trace/input.rs:
// 45-131) without its binary32 narrowing: normalization by M, the extremality-unchanged check
// (input.rs:84-91), the observer-frequency normalization check (input.rs:52-63) and the event
// envelope (crates/gravlume-reference/src/events.rs:61-84). The observer tetrad is the reference's
// stationary-observer construction (crates/gravlume-domain/src/observer.rs:106-183): u along the
// Killing time, sight projected and normalized in g, the up hint projected against the sight
// (falling back to the best coordinate axis), the right vector completed from the best coordinate
// axis and oriented so det(u, right, up, arrival) > 0. The camera basis has to be the same as the
// reference's for image parity, so the construction follows the same steps.
#include <cmath>
#include <cstring>
#include <limits>

#include "glc_internal.h"
#include "glc_radiation.cuh"

namespace glc {

namespace {

constexpr double kBasisTolerance = 1.0e-12;

// ---- exact sign of M^2 - (a^2 + Q^2): error-free products and a Shewchuk expansion sum ----
void two_product(double a, double b, double& hi, double& lo) {
  hi = a * b;
  lo = std::fma(a, b, -hi);
}
void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  const double bv = s - a;
  e = (a - (s - bv)) + (b - bv);
}
// Adds v into the nonoverlapping expansion e[0..n) (increasing magnitude); returns new length.
int grow_expansion(double* e, int n, double v) {
  double q = v;
  int m = 0;
  double h[16];
  for (int i = 0; i < n; ++i) {
    double s, err;
    two_sum(q, e[i], s, err);
    if (err != 0.0) h[m++] = err;
    q = s;
  }
  if (q != 0.0 || m == 0) h[m++] = q;
  std::memcpy(e, h, sizeof(double) * m);
  return m;
}

// Returns sign (-1, 0, +1) of M^2 - a^2 - Q^2 and an approximation of its value, exact up to the
// final rounding. Inputs are scaled by a common power of two so that no product under- or
// overflows for physically meaningful ratios.
int extremality_discriminant(double m, double a, double q, double& value) {
  const double big = std::fmax(std::fabs(m), std::fmax(std::fabs(a), std::fabs(q)));
  int ex = 0;
  std::frexp(big, &ex);
  const double sm = std::ldexp(m, -ex), sa = std::ldexp(a, -ex), sq = std::ldexp(q, -ex);
  double parts[6];
  two_product(sm, sm, parts[0], parts[1]);
  two_product(sa, sa, parts[2], parts[3]);
  two_product(sq, sq, parts[4], parts[5]);
  double e[16];
  int n = 0;
  const double terms[6] = {parts[1], -parts[3], -parts[5], parts[0], -parts[2], -parts[4]};
  for (double t : terms)
    if (t != 0.0) n = grow_expansion(e, n, t);
  double sum = 0.0;
  for (int i = 0; i < n; ++i) sum += e[i];
  value = std::ldexp(sum, 2 * ex);
  if (n == 0) return 0;
  const double top = e[n - 1];
  return top > 0.0 ? 1 : (top < 0.0 ? -1 : 0);
}

// ---- Kerr-Newman metric at a point (M = 1), g_{mu nu} = eta + f l_mu l_nu ----
struct PointMetric {
  double g[4][4];
  double f;
};

bool metric_at(double a, double q, double s, const double txyz[4], PointMetric& out) {
  const double x = txyz[1], y = txyz[2], z = txyz[3];
  const double a2 = a * a;
  const double b = x * x + y * y + z * z - a2;
  const double az2 = a2 * z * z;
  const double sq = std::sqrt(b * b + 4.0 * az2);
  const double r2 = b >= 0.0 ? 0.5 * (b + sq) : 2.0 * az2 / (sq - b);
  if (!(r2 > 0.0) || !std::isfinite(r2)) return false;
  const double r = std::sqrt(r2);
  const double sigma = r2 + az2 / r2;
  const double f = (2.0 * r - q * q) / sigma;
  const double A = r2 + a2;
  const double lc[4] = {1.0, s * (r * x + s * a * y) / A, s * (r * y - s * a * x) / A, s * z / r};
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      const double eta = i == j ? (i == 0 ? -1.0 : 1.0) : 0.0;
      out.g[i][j] = std::fma(f * lc[i], lc[j], eta);
    }
  out.f = f;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      if (!std::isfinite(out.g[i][j])) return false;
  return true;
}

double gdot(const PointMetric& m, const double u[4], const double v[4], double* term_norm = nullptr) {
  double s = 0.0, n = 0.0;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      const double t = m.g[i][j] * u[i] * v[j];
      s += t;
      n += std::fabs(t);
    }
  if (term_norm) *term_norm = n;
  return s;
}

bool project_normalize(const PointMetric& m, const double u[4], const double seed[4], const double (*ortho)[4],
                       int n_ortho, double out[4]) {
  double p[4];
  const double us = gdot(m, u, seed);
  for (int i = 0; i < 4; ++i) p[i] = seed[i] + u[i] * us;
  for (int k = 0; k < n_ortho; ++k) {
    const double c = gdot(m, p, ortho[k]);
    for (int i = 0; i < 4; ++i) p[i] -= ortho[k][i] * c;
  }
  const double n2 = gdot(m, p, p);
  if (!std::isfinite(n2) || n2 <= kBasisTolerance * kBasisTolerance) return false;
  const double inv = 1.0 / std::sqrt(n2);
  for (int i = 0; i < 4; ++i) {
    out[i] = p[i] * inv;
    if (!std::isfinite(out[i])) return false;
  }
  return true;
}

bool best_axis(const PointMetric& m, const double u[4], const double (*ortho)[4], int n_ortho, double out[4]) {
  bool found = false;
  double best = 0.0;
  for (int axis = 1; axis <= 3; ++axis) {
    double seed[4] = {0, 0, 0, 0};
    seed[axis] = 1.0;
    double cand[4];
    if (!project_normalize(m, u, seed, ortho, n_ortho, cand)) continue;
    const double score = std::fmax(std::fabs(cand[1]), std::fmax(std::fabs(cand[2]), std::fabs(cand[3])));
    if (!found || score >= best) {  // later axes win ties
      std::memcpy(out, cand, sizeof cand);
      best = score;
      found = true;
    }
  }
  return found;
}

double det4(const double c0[4], const double c1[4], const double c2[4], const double c3[4]) {
  double m[4][4];
  for (int r = 0; r < 4; ++r) {
    m[r][0] = c0[r];
    m[r][1] = c1[r];
    m[r][2] = c2[r];
    m[r][3] = c3[r];
  }
  double det = 1.0;
  for (int pc = 0; pc < 4; ++pc) {
    int pr = pc;
    for (int r = pc + 1; r < 4; ++r)
      if (std::fabs(m[r][pc]) >= std::fabs(m[pr][pc])) pr = r;
    if (m[pr][pc] == 0.0) return 0.0;
    if (pr != pc) {
      for (int c = 0; c < 4; ++c) std::swap(m[pr][c], m[pc][c]);
      det = -det;
    }
    det *= m[pc][pc];
    for (int r = pc + 1; r < 4; ++r) {
      const double fct = m[r][pc] / m[pc][pc];
      for (int c = pc + 1; c < 4; ++c) m[r][c] -= fct * m[pc][c];
    }
  }
  return det;
}

// Equatorial circular photon orbits of Kerr-Newman (M = 1): roots of
//   r^2 - 3 r + 2 Q^2 + sign * 2 |a| sqrt(r - Q^2) = 0
// (sign +1: prograde, the inner orbit; -1: retrograde, the outer one). The function is positive
// above the orbit; walk down from 6 M to the first non-positive value and bisect.
double photon_orbit(double a, double q, double sign) {
  const double q2 = q * q;
  auto fn = [&](double r) { return r * r - 3.0 * r + 2.0 * q2 + sign * 2.0 * std::fabs(a) * std::sqrt(r - q2); };
  double hi = 6.0;
  double probe = hi;
  while (probe > q2 + 1e-9 && fn(probe) > 0.0) {
    hi = probe;
    probe -= 0.005;
  }
  if (!(probe > q2) || fn(probe) > 0.0) return std::numeric_limits<double>::quiet_NaN();
  double lo = probe;
  for (int i = 0; i < 200; ++i) {
    const double mid = 0.5 * (lo + hi);
    if (fn(mid) > 0.0) hi = mid;
    else lo = mid;
  }
  return 0.5 * (lo + hi);
}

}  // namespace

// Prograde ISCO of Kerr-Newman (M = 1): the outermost root of
//   r (6 r - r^2 - 9 Q^2 + 3 a^2) + 4 Q^2 (Q^2 - a^2) - 8 |a| (r - Q^2)^(3/2) = 0,
// which is Bardeen-Press-Teukolsky's r^2 - 6 r + 8 a sqrt(r) - 3 a^2 = 0 at Q = 0 and the
// Reissner-Nordstrom r^3 - 6 r^2 + 9 Q^2 r - 4 Q^4 = 0 at a = 0.
double prograde_isco(double a, double q) {
  const double q2 = q * q;
  auto fn = [&](double r) {
    const double k = r - q2;
    return r * (6.0 * r - r * r - 9.0 * q2 + 3.0 * a * a) + 4.0 * q2 * (q2 - a * a) -
           8.0 * std::fabs(a) * k * std::sqrt(std::fmax(k, 0.0));
  };
  double hi = 10.0, lo = hi;
  while (lo > 1e-6 && fn(lo) < 0.0) lo *= 0.95;
  for (int i = 0; i < 200; ++i) {
    const double mid = 0.5 * (lo + hi);
    if (fn(mid) < 0.0) hi = mid;
    else lo = mid;
  }
  return 0.5 * (lo + hi);
}

glc_status pack_scene(const glc_scene_input& in, glc_scene& out) {
  std::memset(&out, 0, sizeof out);
  const double M = in.mass;
  if (!std::isfinite(M) || !std::isfinite(in.spin) || !std::isfinite(in.charge))
    return set_error(GLC_ERR_NON_FINITE, "spacetime parameters must be finite");
  if (M <= 0.0) return set_error(GLC_ERR_NON_POSITIVE, "mass scale must be positive");
  if (in.chart != GLC_CHART_INGOING && in.chart != GLC_CHART_OUTGOING)
    return set_error(GLC_ERR_INVALID_ARGUMENT, "chart must be ingoing or outgoing");
  for (int i = 0; i < 4; ++i)
    if (!std::isfinite(in.observer_txyz[i]) || !std::isfinite(in.target_txyz[i]))
      return set_error(GLC_ERR_NON_FINITE, "observer and target events must be finite");
  for (int i = 0; i < 3; ++i)
    if (!std::isfinite(in.up_hint_xyz[i])) return set_error(GLC_ERR_NON_FINITE, "up hint must be finite");
  if (!std::isfinite(in.measured_frequency)) return set_error(GLC_ERR_NON_FINITE, "measured frequency must be finite");
  if (in.measured_frequency <= 0.0) return set_error(GLC_ERR_NON_POSITIVE, "measured frequency must be positive");
  if (std::fabs(in.measured_frequency - 1.0) > 32.0 * std::numeric_limits<double>::epsilon())
    return set_error(GLC_ERR_NON_NORMALIZED, "observer frequency must be normalized to 1");
  if (in.width == 0 || in.height == 0) return set_error(GLC_ERR_INVALID_VIEW, "view size must be nonzero");
  if (!std::isfinite(in.vertical_fov) || in.vertical_fov <= 0.0 || in.vertical_fov >= M_PI)
    return set_error(GLC_ERR_INVALID_VIEW, "vertical field of view must lie in (0, pi)");
  const double tan_half = std::tan(0.5 * in.vertical_fov);
  if (!std::isfinite(tan_half)) return set_error(GLC_ERR_INVALID_VIEW, "non-finite view scale");
  if (!std::isfinite(in.escape_radius) || in.escape_radius < 0.0)
    return set_error(GLC_ERR_INVALID_ARGUMENT, "escape radius must be finite and non-negative (0 = none)");
  if (!std::isfinite(in.horizon_offset) || in.horizon_offset < 0.0)
    return set_error(GLC_ERR_INVALID_ARGUMENT, "horizon offset must be finite and non-negative");
  if (in.has_surface) {
    if (!std::isfinite(in.surface_inner) || !std::isfinite(in.surface_outer) || in.surface_inner <= 0.0 ||
        in.surface_outer < in.surface_inner || !std::isfinite(in.intensity_at_six) || in.intensity_at_six < 0.0)
      return set_error(GLC_ERR_INVALID_SURFACE, "surface radii must be finite, positive and ordered");
    if (in.escape_radius > 0.0 && in.surface_outer / M >= in.escape_radius / M)
      return set_error(GLC_ERR_SURFACE_OUTSIDE_ESCAPE, "surface must lie strictly inside the escape sphere");
  }
  // normalization by M; the extremality must survive it (input.rs:84-91)
  const double a = in.spin / M, q = in.charge / M;
  double d_phys, d_norm;
  const int e_phys = extremality_discriminant(M, in.spin, in.charge, d_phys);
  const int e_norm = extremality_discriminant(1.0, a, q, d_norm);
  if (e_phys != e_norm) return set_error(GLC_ERR_EXTREMALITY_CHANGED, "normalization by M changed the extremality");
  out.spin = a;
  out.charge = q;
  out.chart_sign = in.chart == GLC_CHART_INGOING ? 1.0 : -1.0;
  out.mass_scale = M;
  out.extremality = e_norm > 0 ? 0 : (e_norm == 0 ? 1 : 2);
  if (out.extremality == 2) {
    out.has_horizon = 0;
    out.outer_horizon = -1.0;
  } else {
    out.has_horizon = 1;
    out.outer_horizon = out.extremality == 1 ? 1.0 : 1.0 + std::sqrt(std::fmax(d_norm, 0.0));
    if (!std::isfinite(out.outer_horizon)) return set_error(GLC_ERR_NON_FINITE, "outer horizon radius must be representable");
  }
  out.horizon_event_radius = out.outer_horizon + in.horizon_offset / M;
  out.has_escape = in.escape_radius > 0.0;
  out.escape_radius = out.has_escape ? in.escape_radius / M : 0.0;
  out.has_surface = in.has_surface ? 1 : 0;
  out.surface_inner = in.has_surface ? in.surface_inner / M : 0.0;
  out.surface_outer = in.has_surface ? in.surface_outer / M : 0.0;
  out.intensity_at_six = in.has_surface ? in.intensity_at_six : 0.0;
  // surface emission and transport (EquatorialEmissionModel, SurfaceTransport)
  out.emission_model = 0;
  out.reserved = 0;
  out.temperature_at_six = 0.0;
  out.slab_transmittance = 1.0;
  out.slab_emission = 0.0;
  out.slab_bands[0] = out.slab_bands[1] = out.slab_bands[2] = 0.0;
  if (in.has_surface) {
    if (in.emission_model != 0 && in.emission_model != 1)
      return set_error(GLC_ERR_INVALID_SURFACE, "unknown surface emission model");
    out.emission_model = in.emission_model;
    if (in.emission_model == 1) {
      if (!std::isfinite(in.temperature_at_six) || !(in.temperature_at_six > 0.0))
        return set_error(GLC_ERR_INVALID_SURFACE, "blackbody temperature at 6 M must be finite and positive");
      out.temperature_at_six = in.temperature_at_six;
    }
    if (in.has_slab) {
      if (!std::isfinite(in.slab_optical_depth) || in.slab_optical_depth < 0.0 || !std::isfinite(in.slab_emission) ||
          in.slab_emission < 0.0)
        return set_error(GLC_ERR_INVALID_SURFACE, "slab optical depth and emission must be finite and non-negative");
      out.slab_transmittance = std::exp(-in.slab_optical_depth);
      out.slab_emission = in.slab_emission;
      if (in.emission_model == 1 && in.slab_emission > 0.0) {
        if (!std::isfinite(in.slab_temperature) || !(in.slab_temperature > 0.0))
          return set_error(GLC_ERR_INVALID_SURFACE, "slab temperature must be finite and positive");
        if (!blackbody_bands(in.slab_emission, in.slab_temperature, out.slab_bands))
          return set_error(GLC_ERR_INVALID_SURFACE, "slab spectrum is not representable");
      }
    }
  }
  // inner (prograde) circular photon orbit: the MIXED binary64 shell r < factor * r_ph hugs the
  // horizon and the co-rotating photon sphere
  out.photon_shell_radius = photon_orbit(a, q, +1.0);
  if (!std::isfinite(out.photon_shell_radius)) out.photon_shell_radius = 3.0 - 2.0 * std::fabs(a);
  out.isco_prograde = out.extremality == 2 ? std::numeric_limits<double>::quiet_NaN() : prograde_isco(a, q);
  double ev[4], tg[4];
  for (int i = 0; i < 4; ++i) {
    ev[i] = in.observer_txyz[i] / M;
    tg[i] = in.target_txyz[i] / M;
    out.observer_txyz[i] = ev[i];
  }
  // stationary observer tetrad (observer.rs:67-183)
  PointMetric pm;
  if (!metric_at(a, q, out.chart_sign, ev, pm)) return set_error(GLC_ERR_NON_STATIONARY, "metric undefined at the observer");
  const double gtt = -1.0 + pm.f;
  if (!(gtt < 0.0)) return set_error(GLC_ERR_NON_STATIONARY, "a stationary observer requires g_tt < 0");
  const double u[4] = {1.0 / std::sqrt(-gtt), 0.0, 0.0, 0.0};
  double seed[4], sight[4], up[4], right[4], arrival[4];
  for (int i = 0; i < 4; ++i) seed[i] = tg[i] - ev[i];
  if (!project_normalize(pm, u, seed, nullptr, 0, sight))
    return set_error(GLC_ERR_DEGENERATE_FRAME, "target does not define a spatial direction in the observer frame");
  for (int i = 0; i < 4; ++i) arrival[i] = -sight[i];
  const double up_seed[4] = {0.0, in.up_hint_xyz[0], in.up_hint_xyz[1], in.up_hint_xyz[2]};
  double so[2][4];
  std::memcpy(so[0], sight, sizeof sight);
  if (!project_normalize(pm, u, up_seed, so, 1, up)) {
    if (!best_axis(pm, u, so, 1, up)) return set_error(GLC_ERR_DEGENERATE_FRAME, "no stable image-up axis");
  }
  std::memcpy(so[1], up, sizeof up);
  if (!best_axis(pm, u, so, 2, right)) return set_error(GLC_ERR_DEGENERATE_FRAME, "observer tetrad could not be completed");
  if (det4(u, right, up, arrival) < 0.0)
    for (int i = 0; i < 4; ++i) right[i] = -right[i];
  // Gram check (observer.rs:171-181)
  const double* basis[4] = {u, right, up, arrival};
  double gram = 0.0;
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) {
      double tn;
      const double v = gdot(pm, basis[r], basis[c], &tn);
      const double expected = r == c ? (r == 0 ? -1.0 : 1.0) : 0.0;
      gram = std::fmax(gram, std::fabs(v - expected) / std::fmax(tn, 1.0));
    }
  if (!(gram <= kBasisTolerance)) return set_error(GLC_ERR_DEGENERATE_FRAME, "observer frame failed its Gram contract");
  for (int i = 0; i < 4; ++i) {
    out.four_velocity[i] = u[i];
    out.image_right[i] = right[i];
    out.image_up[i] = up[i];
    out.arrival[i] = arrival[i];
  }
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) out.metric_covariant[4 * i + j] = pm.g[i][j];
  out.frequency = in.measured_frequency;
  out.tangent_half_fov = tan_half;
  out.width = in.width;
  out.height = in.height;
  return GLC_OK;
}

}  // namespace glc
