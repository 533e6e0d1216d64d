// Surface footprint (crates/gravlume-reference/src/footprint.rs). TEST INFRASTRUCTURE ONLY: the
// checker for the CUDA path's quarter-pixel and tangent footprints.
//
// surface_footprint restates ObservationTracer::surface_footprint_v1 (footprint.rs:74-150): the
// center and four neighbours a quarter pixel away (left, right, up, down; 154-195) are traced
// through the observation; the estimate is resolved only when all five end on an unambiguous
// observed surface (237-253) with the center's branch key, and its Jacobian is the central
// difference over the half-pixel span of the source radius and of the local azimuthal arc
// (center radius times the wrapped azimuth difference). footprint_metrics restates 203-235.
#pragma once

#include <cmath>
#include <cstdint>

#include "oracle_tracer.hpp"

namespace gro {

enum FootprintStatus : int {
  kFootprintNoSurface = 0,     // CenterSurfaceUnavailable (footprint.rs:264)
  kFootprintResolved = 1,      // SurfaceFootprintEstimate::Resolved
  kFootprintDiscontinuity = 2, // SurfaceFootprintEstimate::Discontinuity
  kFootprintNonFinite = 3,     // NonFiniteJacobian (footprint.rs:266)
};

struct FootprintMetrics {
  double determinant, squared_norm, major, minor;
};

// footprint.rs:203-235 (the `mul_add`s as std::fma; the sum of squares left to right).
inline bool footprint_metrics(const double J[4], FootprintMetrics& m) {
  for (int i = 0; i < 4; ++i)
    if (!std::isfinite(J[i])) return false;
  m.determinant = std::fma(J[0], J[3], -J[1] * J[2]);
  double n2 = 0.0;
  for (int i = 0; i < 4; ++i) n2 += J[i] * J[i];
  m.squared_norm = n2;
  const double disc = std::sqrt(std::fmax(std::fma(n2, n2, -4.0 * m.determinant * m.determinant), 0.0));
  m.major = std::sqrt(0.5 * (n2 + disc));
  m.minor = m.major == 0.0 ? 0.0 : std::fabs(m.determinant) / m.major;
  return std::isfinite(m.major) && std::isfinite(m.minor);
}

// footprint.rs:168-175: parity against the determinant floor 64 eps |J|_F^2.
inline int footprint_parity(const FootprintMetrics& m) {
  const double floor_ = 64.0 * 2.220446049250313e-16 * m.squared_norm;
  return m.determinant > floor_ ? 1 : (m.determinant < -floor_ ? -1 : 0);
}

// footprint.rs:237-253: an observed surface whose localized event has one candidate.
inline bool resolved_surface(const Outcome& o) {
  return o.termination == Termination::EquatorialSurface && o.surface_status == 1 &&
         __builtin_popcount(o.event_candidates) <= 1;
}

inline bool same_branch(const Outcome& a, const Outcome& b) {
  return a.polar_side == b.polar_side && a.radial_turnings == b.radial_turnings &&
         a.equatorial_crossings == b.equatorial_crossings && a.azimuth_winding == b.azimuth_winding;
}

// Footprint from the five outcomes (center, left, right, up, down). out8 = J (row-major: dr/dx,
// dr/dy, darc/dx, darc/dy, M per pixel), major, minor, determinant, parity; NaN unless resolved.
inline int surface_footprint(const Outcome o[5], double out8[8]) {
  for (int i = 0; i < 8; ++i) out8[i] = NAN;
  if (!resolved_surface(o[0])) return kFootprintNoSurface;
  for (int k = 1; k < 5; ++k)
    if (!resolved_surface(o[k]) || !same_branch(o[k], o[0])) return kFootprintDiscontinuity;
  const double rc = o[0].source_radius, pc = o[0].source_azimuth;
  auto arc = [&](const Outcome& n) { return rc * wrapped_angle_difference(n.source_azimuth, pc); };
  constexpr double kSpan = 0.5;
  const double J[4] = {(o[2].source_radius - o[1].source_radius) / kSpan,
                       (o[4].source_radius - o[3].source_radius) / kSpan, (arc(o[2]) - arc(o[1])) / kSpan,
                       (arc(o[4]) - arc(o[3])) / kSpan};
  FootprintMetrics m;
  if (!footprint_metrics(J, m)) return kFootprintNonFinite;
  for (int i = 0; i < 4; ++i) out8[i] = J[i];
  out8[4] = m.major;
  out8[5] = m.minor;
  out8[6] = m.determinant;
  out8[7] = double(footprint_parity(m));
  return kFootprintResolved;
}

}  // namespace gro
