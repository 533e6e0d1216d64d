// Oracle: stationary observer tetrad, perspective view and initial photon momentum (binary64).
//
// TEST INFRASTRUCTURE ONLY (see oracle_numerics.hpp).
//
// Follows crates/gravlume-domain/src/observer.rs (StationaryObserverInput::build 67-103,
// construct_frame 106-183, project_and_normalize 289-317, best_coordinate_axis 319-352,
// gram_residual 354-376, determinant4 378-408), view.rs (PerspectiveView::new 343-370,
// sight_plane 408-424) and scene.rs (Observation::initial_ray 211-270).
#pragma once

#include "oracle_spacetime.hpp"

namespace gro {

constexpr double BASIS_TOLERANCE = 1.0e-12;
constexpr double INITIAL_RAY_NULL_TOLERANCE = 2.0e-12;

struct FourVec {
  double v[4];
};
inline FourVec fv_add(const FourVec& a, const FourVec& b) {
  FourVec r;
  for (int i = 0; i < 4; ++i) r.v[i] = a.v[i] + b.v[i];
  return r;
}
inline FourVec fv_sub(const FourVec& a, const FourVec& b) {
  FourVec r;
  for (int i = 0; i < 4; ++i) r.v[i] = a.v[i] - b.v[i];
  return r;
}
inline FourVec fv_scale(const FourVec& a, double s) {
  FourVec r;
  for (int i = 0; i < 4; ++i) r.v[i] = a.v[i] * s;
  return r;
}
inline bool fv_finite(const FourVec& a) {
  for (int i = 0; i < 4; ++i)
    if (!std::isfinite(a.v[i])) return false;
  return true;
}

enum class ObserverError : int {
  None = 0,
  InvalidInput = 1,
  OutOfRange = 2,
  NonStationary = 3,
  DegenerateTarget = 4,
  DegenerateUp = 5,
  InternalInvariant = 6,
};

struct ObserverFrame {
  FourVec four_velocity, image_right, image_up, arrival;
  double gram_residual, orientation_determinant;
  bool used_up_fallback;
};

struct StationaryObserver {
  double event[4];
  ObserverFrame frame;
  double measured_frequency;
  double metric_g_tt;
  double metric_covariant[4][4];

  void lower(const FourVec& vec, double out[4]) const {
    for (int r = 0; r < 4; ++r) {
      double s = -0.0;
      for (int c = 0; c < 4; ++c) s += metric_covariant[r][c] * vec.v[c];
      out[r] = s;
    }
  }
};

// observer.rs:289-317
inline bool project_and_normalize(const Spacetime& st, const double ev[4], const FourVec& u, const FourVec& seed,
                                  const FourVec* ortho, int n_ortho, FourVec& out) {
  if (!fv_finite(seed)) return false;
  double uds, norm;
  if (st.metric_dot_and_term_norm(ev, u.v, seed.v, uds, norm) != GeometryError::None) return false;
  FourVec projected = fv_add(seed, fv_scale(u, uds));
  for (int i = 0; i < n_ortho; ++i) {
    double comp;
    if (st.metric_dot_and_term_norm(ev, projected.v, ortho[i].v, comp, norm) != GeometryError::None) return false;
    projected = fv_sub(projected, fv_scale(ortho[i], comp));
  }
  double n2;
  if (st.metric_dot_and_term_norm(ev, projected.v, projected.v, n2, norm) != GeometryError::None) return false;
  if (!std::isfinite(n2) || n2 <= BASIS_TOLERANCE * BASIS_TOLERANCE) return false;
  out = fv_scale(projected, 1.0 / std::sqrt(n2));
  return fv_finite(out);
}

// observer.rs:319-352 (Rust `max_by` keeps the last of equal maxima)
inline bool best_coordinate_axis(const Spacetime& st, const double ev[4], const FourVec& u, const FourVec* ortho,
                                 int n_ortho, FourVec& out) {
  const double axes[3][4] = {{0, 1, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}};
  bool found = false;
  double best_score = 0.0;
  for (int a = 0; a < 3; ++a) {
    FourVec seed{{axes[a][0], axes[a][1], axes[a][2], axes[a][3]}};
    FourVec cand;
    if (!project_and_normalize(st, ev, u, seed, ortho, n_ortho, cand)) continue;
    double score = 0.0;
    for (int i = 1; i < 4; ++i) score = std::fmax(score, std::fabs(cand.v[i]));
    if (!found || !(score < best_score)) {
      out = cand;
      best_score = score;
      found = true;
    }
  }
  return found;
}

// observer.rs:354-376
inline double gram_residual(const Spacetime& st, const double ev[4], const FourVec basis[4]) {
  double residual = 0.0;
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) {
      double actual, norm;
      if (st.metric_dot_and_term_norm(ev, basis[r].v, basis[c].v, actual, norm) != GeometryError::None)
        return std::numeric_limits<double>::infinity();
      const double expected = r == c ? (r == 0 ? -1.0 : 1.0) : 0.0;
      residual = std::fmax(residual, std::fabs(actual - expected) / std::fmax(norm, 1.0));
    }
  return residual;
}

// observer.rs:378-408 (columns are the basis vectors)
inline double determinant4(const FourVec cols[4]) {
  double m[4][4];
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) m[r][c] = cols[c].v[r];
  double det = 1.0;
  for (int pc = 0; pc < 4; ++pc) {
    int pr = pc;
    for (int r = pc; r < 4; ++r)
      if (!(std::fabs(m[r][pc]) < std::fabs(m[pr][pc]))) pr = r;  // max_by: last maximum
    if (m[pr][pc] == 0.0) return 0.0;
    if (pr != pc) {
      for (int c = 0; c < 4; ++c) std::swap(m[pr][c], m[pc][c]);
      det = -det;
    }
    const double pivot = m[pc][pc];
    det *= pivot;
    double pv[4];
    for (int c = 0; c < 4; ++c) pv[c] = m[pc][c];
    for (int r = pc + 1; r < 4; ++r) {
      const double factor = m[r][pc] / pivot;
      for (int c = pc + 1; c < 4; ++c) m[r][c] = std::fma(factor, -pv[c], m[r][c]);
    }
  }
  return det;
}

// observer.rs:17-103 StationaryObserverInput::{validate, build}
inline ObserverError build_observer(const Spacetime& st, const double event[4], const double target[4],
                                    const double up_hint[3], double frequency, StationaryObserver& out) {
  for (int i = 0; i < 4; ++i)
    if (!std::isfinite(event[i]) || !std::isfinite(target[i])) return ObserverError::InvalidInput;
  for (int i = 0; i < 3; ++i)
    if (!std::isfinite(up_hint[i])) return ObserverError::InvalidInput;
  if (!std::isfinite(frequency) || frequency <= 0.0) return ObserverError::InvalidInput;
  Geometry g;
  if (st.geometry(event, g) != GeometryError::None) return ObserverError::OutOfRange;
  const double gtt = -1.0 + g.scalar_f;
  if (gtt >= 0.0) return ObserverError::NonStationary;
  const FourVec u{{1.0 / std::sqrt(-gtt), 0.0, 0.0, 0.0}};
  // construct_frame, observer.rs:106-183
  FourVec seed;
  for (int i = 0; i < 4; ++i) seed.v[i] = target[i] - event[i];
  FourVec sight;
  if (!project_and_normalize(st, event, u, seed, nullptr, 0, sight)) return ObserverError::DegenerateTarget;
  const FourVec arrival = fv_scale(sight, -1.0);
  const FourVec requested{{0.0, up_hint[0], up_hint[1], up_hint[2]}};
  FourVec up;
  bool fallback = false;
  if (!project_and_normalize(st, event, u, requested, &sight, 1, up)) {
    if (!best_coordinate_axis(st, event, u, &sight, 1, up)) return ObserverError::DegenerateUp;
    fallback = true;
  }
  const FourVec so[2] = {sight, up};
  FourVec right;
  if (!best_coordinate_axis(st, event, u, so, 2, right)) return ObserverError::InternalInvariant;
  FourVec cols[4] = {u, right, up, arrival};
  double orientation = determinant4(cols);
  if (orientation < 0.0) {
    right = fv_scale(right, -1.0);
    orientation = -orientation;
  }
  const FourVec basis[4] = {u, right, up, arrival};
  ObserverFrame f{u, right, up, arrival, gram_residual(st, event, basis), orientation, fallback};
  if (!std::isfinite(f.gram_residual) || f.gram_residual > BASIS_TOLERANCE || !std::isfinite(f.orientation_determinant) ||
      f.orientation_determinant <= 0.0)
    return ObserverError::InternalInvariant;
  for (int i = 0; i < 4; ++i) out.event[i] = event[i];
  out.frame = f;
  out.measured_frequency = frequency;
  out.metric_g_tt = gtt;
  Spacetime::metric_covariant(g, out.metric_covariant);
  return ObserverError::None;
}

// view.rs:330-424
struct PerspectiveView {
  uint32_t width = 1, height = 1;
  double vertical_fov = 0.0, tangent_half_fov = 0.0;

  static bool make(uint32_t w, uint32_t h, double fov, PerspectiveView& out) {
    if (w == 0 || h == 0) return false;
    if (!std::isfinite(fov) || fov <= 0.0 || fov >= M_PI) return false;
    const double t = std::tan(fov * 0.5);
    if (!std::isfinite(t)) return false;
    out = {w, h, fov, t};
    return true;
  }
  bool valid_sample(uint32_t px, uint32_t py, double sx, double sy) const {
    if (px >= width || py >= height) return false;
    if (!std::isfinite(sx) || !std::isfinite(sy)) return false;
    return sx >= 0.0 && sx <= 1.0 && sy >= 0.0 && sy <= 1.0;
  }
  void sight_plane(uint32_t px, uint32_t py, double sx, double sy, double out[2]) const {
    const double w = double(width), h = double(height);
    const double nx = 2.0 * (double(px) + sx) / w - 1.0;
    const double ny = 1.0 - 2.0 * (double(py) + sy) / h;
    const double aspect = w / h;
    out[0] = aspect * tangent_half_fov * nx;
    out[1] = tangent_half_fov * ny;
  }
};

struct InitialRay {
  double state[8];
  double sight_direction[4];
  double observer_frequency;
  double normalized_null_residual;
};

enum class InitialRayError : int { None = 0, InvalidSample = 1, NonFinite = 2, InternalInvariant = 3 };

// scene.rs:211-270 Observation::initial_ray
inline InitialRayError initial_ray(const StationaryObserver& obs, const PerspectiveView& view, uint32_t px, uint32_t py,
                                   double sx, double sy, InitialRay& out) {
  if (!view.valid_sample(px, py, sx, sy)) return InitialRayError::InvalidSample;
  double sp[2];
  view.sight_plane(px, py, sx, sy, sp);
  const ObserverFrame& f = obs.frame;
  const double normalization = 1.0 / std::hypot(1.0, std::hypot(sp[0], sp[1]));
  const FourVec sight = fv_scale(fv_sub(fv_add(fv_scale(f.image_right, sp[0]), fv_scale(f.image_up, sp[1])), f.arrival),
                                 normalization);
  const FourVec arrival_direction = fv_scale(sight, -1.0);
  const FourVec mom = fv_scale(fv_add(f.four_velocity, arrival_direction), obs.measured_frequency);
  if (!fv_finite(mom)) return InitialRayError::NonFinite;
  double pc[4];
  obs.lower(mom, pc);
  const double residual = normalized_quadratic_form_residual(obs.metric_covariant, mom.v);
  double freq = -0.0;
  for (int i = 0; i < 4; ++i) freq += pc[i] * f.four_velocity.v[i];
  freq = -freq;
  for (int i = 0; i < 4; ++i)
    if (!std::isfinite(pc[i])) return InitialRayError::NonFinite;
  if (!std::isfinite(freq) || !std::isfinite(residual)) return InitialRayError::NonFinite;
  if (freq <= 0.0 || residual > INITIAL_RAY_NULL_TOLERANCE) return InitialRayError::InternalInvariant;
  for (int i = 0; i < 4; ++i) {
    out.state[i] = obs.event[i];
    out.state[4 + i] = pc[i];
    out.sight_direction[i] = sight.v[i];
  }
  out.observer_frequency = freq;
  out.normalized_null_residual = residual;
  return InitialRayError::None;
}

}  // namespace gro
