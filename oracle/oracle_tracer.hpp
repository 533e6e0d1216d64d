// Oracle: the binary64 Dormand-Prince 5(4) geodesic tracer with events and observables.
//
// TEST INFRASTRUCTURE ONLY (see oracle_numerics.hpp).
//
// Follows crates/gravlume-reference/src/integrator.rs (tableau 6-98, attempt_step 153-190, dense
// output 128-143/192-209), policy.rs (regular_v1 28-48, strict_v1 51-66, error_norm 137-158,
// next_step_magnitude 160-173), events.rs (3-129), geodesic.rs (TraceExecution::run 129-212,
// find_event 233-265, record_turning_point 330-360, record_equatorial_crossing 362-383,
// commit_observables 406-418, escape_direction_xyz 480-497, CompensatedSum 508-528, EventArming
// 530-573, localize_dense_root 640-676, event_value_for 678-700, crosses 702-708,
// select_earliest_event 722-740), observation.rs (ObservationTracer::trace 189-231) and
// surface.rs (observable_at 12-73, surface_radius_and_frequency_ratio 75-146).
//
// Two parameters extend the reference's event configuration for the benchmark workloads and are
// neutral at their defaults: `horizon_offset_m` (capture at r_+ + offset; reference: 0) and the
// escape radius (reference observation baseline: 200 M).
#pragma once

#include <vector>

#include "oracle_observation.hpp"

namespace gro {

// ---------------------------------------------------------------- integrator.rs:6-98
namespace tableau {
constexpr double A[7][7] = {
    {0, 0, 0, 0, 0, 0, 0},
    {1.0 / 5.0, 0, 0, 0, 0, 0, 0},
    {3.0 / 40.0, 9.0 / 40.0, 0, 0, 0, 0, 0},
    {44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0, 0, 0, 0, 0},
    {19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0, 0, 0, 0},
    {9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0, -5103.0 / 18656.0, 0, 0},
    {35.0 / 384.0, 0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0, 0},
};
constexpr double B5[7] = {35.0 / 384.0, 0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0, 0};
constexpr double B4[7] = {5179.0 / 57600.0, 0, 7571.0 / 16695.0, 393.0 / 640.0, -92097.0 / 339200.0, 187.0 / 2100.0,
                          1.0 / 40.0};
constexpr double D[7][4] = {
    {1.0, -8048581381.0 / 2820520608.0, 8663915743.0 / 2820520608.0, -12715105075.0 / 11282082432.0},
    {0, 0, 0, 0},
    {0, 131558114200.0 / 32700410799.0, -68118460800.0 / 10900136933.0, 87487479700.0 / 32700410799.0},
    {0, -1754552775.0 / 470086768.0, 14199869525.0 / 1410260304.0, -10690763975.0 / 1880347072.0},
    {0, 127303824393.0 / 49829197408.0, -318862633887.0 / 49829197408.0, 701980252875.0 / 199316789632.0},
    {0, -282668133.0 / 205662961.0, 2019193451.0 / 616988883.0, -1453857185.0 / 822651844.0},
    {0, 40617522.0 / 29380423.0, -110615467.0 / 29380423.0, 69997945.0 / 29380423.0},
};
}  // namespace tableau

struct DenseOutput {
  double start[8];
  double step;
  double stages[7][8];

  double dense_derivative(int c, const double pw[4]) const {
    double s = -0.0;
    for (int j = 0; j < 7; ++j) {
      double cs = -0.0;
      for (int k = 0; k < 4; ++k) cs += tableau::D[j][k] * pw[k];
      s += cs * stages[j][c];
    }
    return s;
  }
  static void powers(double th, double pw[4]) {
    pw[0] = th;
    pw[1] = th * th;
    pw[2] = th * (th * th);
    pw[3] = (th * th) * (th * th);
  }
  void evaluate(double th, double out[8]) const {
    double pw[4];
    powers(th, pw);
    for (int c = 0; c < 8; ++c) out[c] = std::fma(step, dense_derivative(c, pw), start[c]);
  }
  double time_increment(double th) const {
    double pw[4];
    powers(th, pw);
    return step * dense_derivative(0, pw);
  }
};

struct StepAttempt {
  double end[8];
  double error[8];
  double end_derivative[8];
  DenseOutput dense;
};

inline double weighted_derivative(const double st[7][8], const double* w, int c) {
  double s = -0.0;
  for (int j = 0; j < 7; ++j) s += w[j] * st[j][c];
  return s;
}

// integrator.rs:153-190; returns the error and, on failure, the number of evaluations done.
inline GeometryError attempt_step(const Spacetime& sp, const double start[8], double step, const double k1[8],
                                  StepAttempt& out, int& evaluations) {
  double (*stages)[8] = out.dense.stages;
  for (int c = 0; c < 8; ++c) stages[0][c] = k1[c];
  for (int s = 1; s < 7; ++s) {
    double ss[8];
    for (int c = 0; c < 8; ++c) {
      double w = -0.0;
      for (int j = 0; j < s; ++j) w += tableau::A[s][j] * stages[j][c];
      ss[c] = std::fma(step, w, start[c]);
    }
    bool finite = true;
    for (int c = 0; c < 8; ++c) finite = finite && std::isfinite(ss[c]);
    GeometryError e = finite ? sp.hamiltonian_rhs(ss, stages[s]) : GeometryError::NonFinite;
    if (e != GeometryError::None) {
      evaluations = s;
      return e;
    }
  }
  double fourth[8];
  for (int c = 0; c < 8; ++c) {
    out.end[c] = std::fma(step, weighted_derivative(stages, tableau::B5, c), start[c]);
    fourth[c] = std::fma(step, weighted_derivative(stages, tableau::B4, c), start[c]);
  }
  for (int c = 0; c < 8; ++c) out.error[c] = out.end[c] - fourth[c];
  out.error[0] = step * weighted_derivative(stages, tableau::B5, 0) - step * weighted_derivative(stages, tableau::B4, 0);
  for (int c = 0; c < 8; ++c) {
    out.end_derivative[c] = stages[6][c];
    out.dense.start[c] = start[c];
  }
  out.dense.step = step;
  evaluations = 6;
  return GeometryError::None;
}

// ---------------------------------------------------------------- policy.rs
struct Policy {
  int id = 0;  // 0 = regular-v1, 1 = strict-v1, 2 = custom
  double position_rtol = 2.0e-12, position_atol = 2.0e-13;
  double momentum_rtol = 2.0e-12, momentum_atol = 2.0e-13;
  double initial_step = 1.0e-3;
  double minimum_step = 9.094947017729282e-13;
  double maximum_step = 0.5;
  double safety = 0.9, minimum_factor = 0.2, maximum_factor = 5.0;
  uint64_t maximum_accepted_steps = 200000;
  uint32_t maximum_consecutive_rejects = 64;
  double event_affine_tolerance = 2.0e-11;
  double event_tie_tolerance = 5.0e-11;
  double event_arming_band = 1.28e-9;
  double singularity_guard = 9.094947017729282e-13;  // 2^-40 (policy.rs:3)

  static Policy regular_v1() { return Policy{}; }
  static Policy strict_v1() {
    Policy r = regular_v1();
    Policy s = r;
    s.id = 1;
    s.position_rtol = r.position_rtol / 16.0;
    s.position_atol = r.position_atol / 16.0;
    s.momentum_rtol = r.momentum_rtol / 16.0;
    s.momentum_atol = r.momentum_atol / 16.0;
    s.maximum_step = 0.25;
    s.maximum_accepted_steps = r.maximum_accepted_steps * 2;
    s.maximum_consecutive_rejects = r.maximum_consecutive_rejects * 2;
    s.event_affine_tolerance = r.event_affine_tolerance / 4.0;
    s.event_tie_tolerance = r.event_tie_tolerance / 4.0;
    return s;
  }
  // policy.rs:137-158
  double error_norm(const double s[8], const double e[8], const double err[8]) const {
    double m = 0.0;
    for (int i = 0; i < 8; ++i) {
      const double rel = i < 4 ? position_rtol : momentum_rtol;
      const double abs_ = i < 4 ? position_atol : momentum_atol;
      m = std::fmax(m, std::fabs(err[i]) / std::fma(rel, std::fmax(std::fabs(s[i]), std::fabs(e[i])), abs_));
    }
    return m;
  }
  // policy.rs:160-173
  double next_step_magnitude(double current, double en, bool accepted) const {
    const double maxf = accepted ? maximum_factor : 1.0;
    double factor;
    if (en == 0.0) {
      factor = maxf;
    } else {
      factor = safety * std::pow(en, -0.2);
      if (factor < minimum_factor) factor = minimum_factor;
      else if (factor > maxf) factor = maxf;
    }
    double h = current * factor;
    if (h < minimum_step) h = minimum_step;
    else if (h > maximum_step) h = maximum_step;
    return h;
  }
};

// ---------------------------------------------------------------- events.rs
enum EventKind : int { kSingularity = 0, kHorizon = 1, kSurface = 2, kEscape = 3 };

struct EventConfig {
  bool has_escape = false;
  double escape_radius = 0.0;
  bool has_surface = false;
  double surface_inner = 0.0, surface_outer = 0.0;
  double horizon_offset = 0.0;
};

// ---------------------------------------------------------------- outcome.rs
enum class Termination : int {
  HorizonCrossing = 1,
  Escape = 2,
  SingularityGuard = 3,
  StepExhaustion = 4,
  NumericalFailure = 5,
  EquatorialSurface = 7,
  RejectExhaustion = 8,
};
enum class NumericalFailure : int { None = 0, NonFinite = 1, RingSingularity = 2, ChartBoundary = 3, InvalidDenominator = 4, MinimumStep = 5 };

inline NumericalFailure failure_of(GeometryError e) {
  switch (e) {
    case GeometryError::NonFinite: return NumericalFailure::NonFinite;
    case GeometryError::RingSingularity: return NumericalFailure::RingSingularity;
    case GeometryError::ChartBoundary: return NumericalFailure::ChartBoundary;
    case GeometryError::InvalidDenominator: return NumericalFailure::InvalidDenominator;
    default: return NumericalFailure::None;
  }
}

struct Outcome {
  Termination termination;
  NumericalFailure failure;
  int event_kind;             // -1 when the terminal has no localized event
  uint32_t event_candidates;  // bit k set: event kind k within tie tolerance
  double event_affine, event_bracket, event_residual;
  double event_theta;         // fraction of the terminal step at the event (the variational reference reads it)
  double state[8];
  double affine_parameter;
  bool has_turning_radius;
  double turning_radius;
  double azimuth_advance;
  double travel_time;
  int polar_side;  // -1, 0, +1
  uint32_t radial_turnings, equatorial_crossings;
  int32_t azimuth_winding;
  uint64_t accepted_steps, rejected_steps, rhs_evaluations;
  double minimum_step, maximum_step;  // NaN when no attempt was made
  double max_null_residual, max_energy_drift, max_lz_drift, max_carter_drift;
  bool has_escape_direction;
  double escape_direction[3];
  // Surface observable (observation traces with a surface only).
  int surface_status;  // 0 = not applicable, 1 = resolved, <0 = SurfaceObservableError code
  double source_radius, source_azimuth, frequency_ratio, emitted_intensity, observed_intensity;
};

inline double wrapped_angle_difference(double current, double previous) {
  const double v = current - previous + M_PI;
  const double tau = 2.0 * M_PI;
  double r = std::fmod(v, tau);
  if (r < 0.0) r += std::fabs(tau);
  return r - M_PI;
}

inline double relative_drift(double initial, double current) {
  return std::fabs(current - initial) / std::fmax(std::fabs(initial), 1.0);
}

struct CompensatedSum {
  double sum = 0.0, correction = 0.0;
  void add(double v) {
    const double next = sum + v;
    correction += std::fabs(sum) >= std::fabs(v) ? (sum - next) + v : (v - next) + sum;
    sum = next;
  }
  double total() const { return sum + correction; }
};

struct Tracer {
  Spacetime sp;
  Policy policy;
  EventConfig events;

  bool horizon_installed() const {
    double rp;
    return sp.outer_horizon_radius(rp);
  }
  double horizon_event_radius() const {
    double rp = 0.0;
    if (!sp.outer_horizon_radius(rp)) rp = 0.0;
    return rp + events.horizon_offset;
  }
  // geodesic.rs:678-700
  GeometryError event_value(int kind, const double st[8], double& v) const {
    switch (kind) {
      case kSingularity: {
        const double m2 = sp.mass_m * sp.mass_m;
        const double guard = policy.singularity_guard * m2 * m2;
        return sp.singularity_guard_residual(st, guard, v);
      }
      case kHorizon: {
        double r;
        GeometryError e = sp.radius(st, r);
        if (e == GeometryError::None) v = r - horizon_event_radius();
        return e;
      }
      case kSurface: v = st[3]; return GeometryError::None;
      default: {
        double r;
        GeometryError e = sp.radius(st, r);
        if (e == GeometryError::None) v = r - (events.has_escape ? events.escape_radius : 0.0);
        return e;
      }
    }
  }
  bool installed(int kind) const {
    switch (kind) {
      case kSingularity: return true;
      case kHorizon: return horizon_installed();
      case kSurface: return events.has_surface;
      default: return events.has_escape;
    }
  }
  double event_scale(int kind) const {
    switch (kind) {
      case kSingularity: return std::fmax((sp.mass_m * sp.mass_m) * (sp.mass_m * sp.mass_m), 1.0);
      case kHorizon: {
        double rp;
        if (!sp.outer_horizon_radius(rp)) rp = 1.0;
        return std::fmax(rp + events.horizon_offset, 1.0);
      }
      case kSurface: return std::fmax(sp.mass_m, 1.0);
      default: return std::fmax(events.has_escape ? events.escape_radius : 1.0, 1.0);
    }
  }
  static bool clears_band(int kind, double v, double band) {
    switch (kind) {
      case kSingularity:
      case kHorizon: return v > band;
      case kSurface: return std::fabs(v) > band;
      default: return v < -band;
    }
  }
  static bool crosses(int kind, double s, double e) {
    switch (kind) {
      case kSingularity:
      case kHorizon: return s > 0.0 && e <= 0.0;
      case kSurface: return (s < 0.0 && e >= 0.0) || (s > 0.0 && e <= 0.0);
      default: return s < 0.0 && e >= 0.0;
    }
  }
  bool surface_contains(const double st[8]) const {
    double r;
    if (sp.radius(st, r) != GeometryError::None) return false;
    return r >= events.surface_inner && r <= events.surface_outer;
  }

  // record: when given, receives the signed size of every accepted step. replay: when given, the
  // attempts take these sizes in order and are all accepted (no error test) while the list lasts,
  // then stepping is adaptive again. Together they give the traced map with its step sequence held
  // fixed, whose central differences are the internal numerical differentiation of the trace
  // (the check of the adjoint; not part of the reference).
  Outcome trace(const double initial[8], double direction_sign, std::vector<double>* record = nullptr,
                const std::vector<double>* replay = nullptr) const;
};

struct DenseRoot {
  double theta;
  double state[8];
  double bracket;
};

// geodesic.rs:640-676
template <class F>
inline GeometryError localize_dense_root(const DenseOutput& dense, double step, double tol, double sv, double ev,
                                         F&& value_at, DenseRoot& out) {
  double lower = 0.0, upper = 1.0, lv = sv, uv = ev;
  for (int i = 0; i < 64; ++i) {
    if ((upper - lower) * std::fabs(step) <= tol) break;
    const double middle = 0.5 * (lower + upper);
    double st[8];
    dense.evaluate(middle, st);
    for (int c = 0; c < 8; ++c)
      if (!std::isfinite(st[c])) return GeometryError::NonFinite;
    double v;
    GeometryError e = value_at(st, v);
    if (e != GeometryError::None) return e;
    if (std::signbit(lv) == std::signbit(v)) {
      lower = middle;
      lv = v;
    } else {
      upper = middle;
      uv = v;
    }
  }
  out.theta = std::fabs(lv) <= std::fabs(uv) ? lower : upper;
  dense.evaluate(out.theta, out.state);
  for (int c = 0; c < 8; ++c)
    if (!std::isfinite(out.state[c])) return GeometryError::NonFinite;
  out.bracket = (upper - lower) * std::fabs(step);
  return GeometryError::None;
}

struct LocalizedRoot {
  int kind;
  double theta;
  double state[8];
  double bracket;
  double residual;
};

// geodesic.rs:53-506 GeodesicTracer::trace / TraceExecution
inline Outcome Tracer::trace(const double initial[8], double sign, std::vector<double>* record,
                             const std::vector<double>* replay) const {
  Outcome o{};
  o.event_kind = -1;
  o.surface_status = 0;
  o.minimum_step = std::numeric_limits<double>::quiet_NaN();
  o.maximum_step = std::numeric_limits<double>::quiet_NaN();
  double state[8];
  for (int i = 0; i < 8; ++i) state[i] = initial[i];
  double affine = 0.0;
  double step = sign * policy.initial_step;
  uint64_t accepted = 0, rejected = 0, rhs = 0;
  uint32_t consecutive = 0;
  bool have_min = false;
  double hmin = 0.0, hmax = 0.0;
  Invariants init_inv;
  const bool have_init_inv = sp.invariants(state, init_inv) == GeometryError::None;
  double d_null = 0.0, d_e = 0.0, d_lz = 0.0, d_q = 0.0;
  bool armed[4];
  for (int k = 0; k < 4; ++k) {
    double v;
    armed[k] = event_value(k, state, v) == GeometryError::None && clears_band(k, v, policy.event_arming_band);
  }
  bool has_turning = false;
  double turning_radius = 0.0;
  uint32_t turnings = 0, crossings = 0;
  int32_t winding = 0;
  const int polar = state[3] > 0.0 ? 1 : (state[3] < 0.0 ? -1 : 0);
  double azimuth_advance = 0.0;
  double previous_azimuth = std::atan2(state[2], state[1]);
  CompensatedSum time_delta;

  auto update_invariants = [&](const double st[8]) {
    Invariants cur;
    if (have_init_inv && sp.invariants(st, cur) == GeometryError::None) {
      d_null = std::fmax(d_null, cur.normalized_null_residual);
      d_e = std::fmax(d_e, relative_drift(init_inv.energy, cur.energy));
      d_lz = std::fmax(d_lz, relative_drift(init_inv.angular_momentum_z, cur.angular_momentum_z));
      d_q = std::fmax(d_q, relative_drift(init_inv.carter_constant, cur.carter_constant));
    }
  };
  auto finish = [&](const double st[8], Termination term) {
    o.termination = term;
    for (int i = 0; i < 8; ++i) o.state[i] = st[i];
    o.affine_parameter = affine;
    o.has_turning_radius = has_turning;
    o.turning_radius = turning_radius;
    o.azimuth_advance = azimuth_advance;
    o.travel_time = sign * time_delta.total();
    o.polar_side = polar;
    o.radial_turnings = turnings;
    o.equatorial_crossings = crossings;
    o.azimuth_winding = winding;
    o.accepted_steps = accepted;
    o.rejected_steps = rejected;
    o.rhs_evaluations = rhs;
    if (have_min) {
      o.minimum_step = hmin;
      o.maximum_step = hmax;
    }
    o.max_null_residual = d_null;
    o.max_energy_drift = d_e;
    o.max_lz_drift = d_lz;
    o.max_carter_drift = d_q;
    return o;
  };
  auto finish_failure = [&](NumericalFailure f) {
    o.failure = f;
    return finish(state, Termination::NumericalFailure);
  };

  double k1[8];
  rhs += 1;
  GeometryError e0 = sp.hamiltonian_rhs(state, k1);
  if (e0 != GeometryError::None) return finish_failure(failure_of(e0));
  update_invariants(state);
  StepAttempt att;
  for (;;) {
    if (accepted >= policy.maximum_accepted_steps) return finish(state, Termination::StepExhaustion);
    const bool replaying = replay != nullptr && accepted < replay->size();
    if (replaying) step = (*replay)[accepted];
    const double mag = std::fabs(step);
    if (!have_min) {
      hmin = mag;
      hmax = mag;
      have_min = true;
    } else {
      hmin = std::fmin(hmin, mag);
      hmax = std::fmax(hmax, mag);
    }
    int evals = 0;
    GeometryError es = attempt_step(sp, state, step, k1, att, evals);
    rhs += uint64_t(evals);
    if (es != GeometryError::None) return finish_failure(failure_of(es));
    double es_start[8], es_end[8];
    for (int i = 0; i < 8; ++i) {
      es_start[i] = state[i];
      es_end[i] = att.end[i];
    }
    es_start[0] = time_delta.total();
    es_end[0] = es_start[0] + att.dense.time_increment(1.0);
    const double en = policy.error_norm(es_start, es_end, att.error);
    if (!std::isfinite(en)) return finish_failure(NumericalFailure::NonFinite);
    if (!replaying && en > 1.0) {
      rejected += 1;
      consecutive += 1;
      if (consecutive >= policy.maximum_consecutive_rejects) return finish(state, Termination::RejectExhaustion);
      if (std::fabs(step) <= policy.minimum_step) return finish_failure(NumericalFailure::MinimumStep);
      step = sign * policy.next_step_magnitude(std::fabs(step), en, false);
      continue;
    }
    accepted += 1;
    consecutive = 0;
    if (record) record->push_back(step);
    for (int i = 0; i < 8; ++i)
      if (!std::isfinite(att.end[i])) return finish_failure(NumericalFailure::NonFinite);
    const double* end_state = att.end;
    // find_event, geodesic.rs:233-265
    LocalizedRoot roots[4];
    int nroots = 0;
    for (int k = 0; k < 4; ++k) {
      if (!armed[k] || !installed(k)) continue;
      double sv, ev;
      GeometryError e = event_value(k, state, sv);
      if (e != GeometryError::None) return finish_failure(failure_of(e));
      e = event_value(k, end_state, ev);
      if (e != GeometryError::None) return finish_failure(failure_of(e));
      if (!crosses(k, sv, ev)) continue;
      DenseRoot dr;
      e = localize_dense_root(att.dense, step, policy.event_affine_tolerance, sv, ev,
                              [&](const double* st, double& v) { return event_value(k, st, v); }, dr);
      if (e != GeometryError::None) return finish_failure(failure_of(e));
      double rv;
      e = event_value(k, dr.state, rv);
      if (e != GeometryError::None) return finish_failure(failure_of(e));
      if (k != kSurface || surface_contains(dr.state)) {
        LocalizedRoot& lr = roots[nroots++];
        lr.kind = k;
        lr.theta = dr.theta;
        for (int c = 0; c < 8; ++c) lr.state[c] = dr.state[c];
        lr.bracket = dr.bracket;
        lr.residual = std::fabs(rv) / event_scale(k);
      }
    }
    int first = -1;
    uint32_t candidates = 0;
    if (nroots > 0) {
      first = 0;
      for (int i = 1; i < nroots; ++i)
        if (roots[i].theta < roots[first].theta) first = i;
      for (int i = 0; i < nroots; ++i)
        if (std::fabs(roots[i].theta - roots[first].theta) * std::fabs(step) <= policy.event_tie_tolerance)
          candidates |= 1u << roots[i].kind;
    }
    const bool has_event = first >= 0;
    const double terminal_theta = has_event ? roots[first].theta : 1.0;
    const double* committed = has_event ? roots[first].state : end_state;
    // record_turning_point, geodesic.rs:330-360
    {
      double sv = 0.0, ev = 0.0;
      rhs += 1;
      const bool ok_s = sp.radial_velocity(state, sv) == GeometryError::None;
      rhs += 1;
      const bool ok_e = sp.radial_velocity(end_state, ev) == GeometryError::None;
      sv *= sign;
      ev *= sign;
      if (ok_s && ok_e && ((sv < 0.0 && ev >= 0.0) || (sv > 0.0 && ev <= 0.0))) {
        DenseRoot dr;
        GeometryError e = localize_dense_root(att.dense, step, policy.event_affine_tolerance, sv, ev,
                                              [&](const double* st, double& v) {
                                                rhs += 1;
                                                GeometryError ee = sp.radial_velocity(st, v);
                                                v *= sign;
                                                return ee;
                                              },
                                              dr);
        if (e == GeometryError::None && (!has_event || dr.theta < terminal_theta)) {
          turnings += 1;
          double r;
          if (sv < 0.0 && ev >= 0.0 && sp.radius(dr.state, r) == GeometryError::None) {
            turning_radius = has_turning ? std::fmin(turning_radius, r) : r;
            has_turning = true;
          }
        }
      }
    }
    // record_equatorial_crossing, geodesic.rs:362-383
    {
      const double sz = state[3], ez = end_state[3];
      if (crosses(kSurface, sz, ez)) {
        DenseRoot dr;
        GeometryError e = localize_dense_root(att.dense, step, policy.event_affine_tolerance, sz, ez,
                                              [&](const double* st, double& v) {
                                                v = st[3];
                                                return GeometryError::None;
                                              },
                                              dr);
        if (e == GeometryError::None && (!has_event || dr.theta < terminal_theta)) crossings += 1;
      }
    }
    time_delta.add(att.dense.time_increment(has_event ? terminal_theta : 1.0));
    // commit_observables, geodesic.rs:406-418
    {
      const double az = std::atan2(committed[2], committed[1]);
      const double raw = az - previous_azimuth;
      azimuth_advance += wrapped_angle_difference(az, previous_azimuth);
      if (raw > M_PI) winding -= 1;
      else if (raw < -M_PI) winding += 1;
      previous_azimuth = az;
      update_invariants(committed);
    }
    if (has_event) {
      affine = std::fma(step, roots[first].theta, affine);
      const LocalizedRoot& r = roots[first];
      o.event_kind = r.kind;
      o.event_candidates = candidates;
      // geodesic.rs:201-202 updates the affine parameter before event_diagnostic adds step*theta
      // once more; the diagnostic keeps that value.
      o.event_affine = std::fma(step, r.theta, affine);
      o.event_bracket = r.bracket;
      o.event_residual = r.residual;
      o.event_theta = r.theta;
      Termination term = Termination::HorizonCrossing;
      switch (r.kind) {
        case kSingularity: term = Termination::SingularityGuard; break;
        case kHorizon: term = Termination::HorizonCrossing; break;
        case kSurface: term = Termination::EquatorialSurface; break;
        default: term = Termination::Escape; break;
      }
      if (r.kind == kEscape) {
        double d[8];
        rhs += 1;
        if (sp.hamiltonian_rhs(r.state, d) == GeometryError::None) {
          const double dir[3] = {sign * d[1], sign * d[2], sign * d[3]};
          const double norm = std::sqrt(std::fma(dir[0], dir[0], std::fma(dir[1], dir[1], dir[2] * dir[2])));
          if (norm > 0.0 && std::isfinite(norm)) {
            o.has_escape_direction = true;
            for (int c = 0; c < 3; ++c) o.escape_direction[c] = dir[c] / norm;
          }
        }
      }
      return finish(r.state, term);
    }
    affine += step;
    for (int i = 0; i < 8; ++i) {
      state[i] = end_state[i];
      k1[i] = att.end_derivative[i];
    }
    // EventArming::update, geodesic.rs:550-560
    for (int k = 0; k < 4; ++k) {
      double v;
      if (!armed[k] && event_value(k, state, v) == GeometryError::None && clears_band(k, v, policy.event_arming_band))
        armed[k] = true;
    }
    step = sign * policy.next_step_magnitude(std::fabs(step), en, true);
  }
}

// ---------------------------------------------------------------- surface.rs
enum SurfaceError : int {
  kSurfOk = 1,
  kSurfGeometry = -1,
  kSurfOutside = -2,
  kSurfCircularUnavailable = -3,
  kSurfNotTimelike = -4,
  kSurfNonPositiveEmitter = -5,
  kSurfInvalidObserverFrequency = -6,
  kSurfNonRepresentableRatio = -7,
  kSurfNonRepresentableEmitted = -8,
  kSurfNonRepresentableObserved = -9,
};

// surface.rs:75-146
inline int surface_radius_and_frequency_ratio(const Spacetime& sp, double inner, double outer, const double st[8],
                                              double observer_frequency, double& radius, double& ratio) {
  if (sp.radius(st, radius) != GeometryError::None) return kSurfGeometry;
  if (!(radius >= inner && radius <= outer)) return kSurfOutside;
  const double m = sp.mass_m, a = sp.spin_m;
  const double q2 = sp.charge_m * sp.charge_m;
  const double crs = std::fma(m, radius, -q2);
  if (!std::isfinite(crs) || crs < 0.0) return kSurfCircularUnavailable;
  const double cr = std::sqrt(crs);
  const double bs = a < 0.0 ? -1.0 : 1.0;
  const double r2 = radius * radius;
  const double avd = std::fma(bs * a, cr, r2);
  if (!std::isfinite(avd) || avd <= 0.0) return kSurfCircularUnavailable;
  const double omega = bs * cr / avd;
  const double rn = std::fma(2.0 * m, radius, -q2);
  const double a2 = a * a;
  const double tdisc = std::fma(-3.0 * m, radius, std::fma(2.0 * bs * a, cr, std::fma(2.0, q2, r2)));
  if (!std::isfinite(tdisc) || tdisc <= 0.0) return kSurfNotTimelike;
  const double delta = std::fma(r2, 1.0, std::fma(2.0 * m, -radius, a2 + q2));
  const double gtt = -1.0 + rn / r2;
  const double gtp = -rn * a / r2;
  const double rf = r2 + a2;
  const double gpp = std::fma(rf, rf, -a2 * delta) / r2;
  const double cn2 = std::fma(omega, omega * gpp, std::fma(2.0 * gtp, omega, gtt));
  if (!std::isfinite(cn2) || cn2 >= 0.0) return kSurfNotTimelike;
  const double tc = 1.0 / std::sqrt(-cn2);
  Invariants inv;
  if (sp.invariants(st, inv) != GeometryError::None) return kSurfGeometry;
  const double ef = tc * std::fma(omega, -inv.angular_momentum_z, inv.energy);
  if (!std::isfinite(ef) || ef <= 0.0) return kSurfNonPositiveEmitter;
  if (!std::isfinite(observer_frequency) || observer_frequency <= 0.0) return kSurfInvalidObserverFrequency;
  ratio = observer_frequency / ef;
  if (!std::isfinite(ratio) || ratio <= 0.0) return kSurfNonRepresentableRatio;
  return kSurfOk;
}

// surface.rs:12-73 restricted to the inverse-cube bolometric emitter in vacuum.
inline int observable_at(const Spacetime& sp, double inner, double outer, double intensity_at_six, const double st[8],
                         double observer_frequency, Outcome& o) {
  double radius, ratio;
  int s = surface_radius_and_frequency_ratio(sp, inner, outer, st, observer_frequency, radius, ratio);
  if (s != kSurfOk) return s;
  const double rr = radius / sp.mass_m / 6.0;
  if (!std::isfinite(rr) || rr <= 0.0) return kSurfNonRepresentableEmitted;
  double emitted = intensity_at_six;
  for (int i = 0; i < 3; ++i) emitted /= rr;
  if (!std::isfinite(emitted) || emitted < 0.0) return kSurfNonRepresentableEmitted;
  double observed = emitted;
  for (int i = 0; i < 4; ++i) observed *= ratio;
  if (!std::isfinite(observed) || observed < 0.0) return kSurfNonRepresentableObserved;
  const double cs = sp.chart == Chart::Ingoing ? sp.spin_m : -sp.spin_m;
  o.source_radius = radius;
  o.source_azimuth = wrapped_angle_difference(std::atan2(st[2], st[1]), std::atan2(cs, radius));
  o.frequency_ratio = ratio;
  o.emitted_intensity = emitted;
  o.observed_intensity = observed;
  return kSurfOk;
}

// observation.rs:189-231: backward trace of one image sample with the surface observable.
inline Outcome trace_observation(const Tracer& tr, const InitialRay& ray, double intensity_at_six) {
  Outcome o = tr.trace(ray.state, -1.0);
  if (tr.events.has_surface && o.termination == Termination::EquatorialSurface) {
    o.surface_status = observable_at(tr.sp, tr.events.surface_inner, tr.events.surface_outer, intensity_at_six, o.state,
                                     ray.observer_frequency, o);
  }
  return o;
}

// Kerr-Newman prograde ISCO: the root of M r (6 M r - r^2 - 9 Q^2 + 3 a^2) + 4 Q^2 (Q^2 - a^2)
// - 8 a (M r - Q^2)^(3/2) = 0 above the prograde photon orbit (new oracle code; reduces to the
// Bardeen-Press-Teukolsky Kerr ISCO at Q = 0 and to the Reissner-Nordstrom ISCO at a = 0).
inline double isco_function(double m, double a, double q, double r) {
  const double q2 = q * q;
  const double k = m * r - q2;
  return m * r * (6.0 * m * r - r * r - 9.0 * q2 + 3.0 * a * a) + 4.0 * q2 * (q2 - a * a) -
         8.0 * std::fabs(a) * k * std::sqrt(std::fmax(k, 0.0));
}
inline double prograde_isco(double m, double a, double q) {
  // The function is negative at large r and positive just outside the marginally stable region;
  // bracket from 9 M downwards and bisect.
  double hi = 9.0 * m + 1.0, lo = hi;
  while (lo > 1e-6 && isco_function(m, a, q, lo) < 0.0) lo *= 0.9;
  for (int i = 0; i < 200; ++i) {
    const double mid = 0.5 * (lo + hi);
    if (isco_function(m, a, q, mid) < 0.0) hi = mid;
    else lo = mid;
  }
  return 0.5 * (lo + hi);
}

}  // namespace gro
