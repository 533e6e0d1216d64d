// Oracle C ABI for the Python test harness (ctypes). TEST INFRASTRUCTURE ONLY: the parity tests,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg load this library as the checker; the
// product never does.
//
// gro_trace_* mirror the reference's CPU entry points: GeodesicTracer::trace
// (crates/gravlume-reference/src/geodesic.rs:53-62), ObservationTracer::trace
// (observation.rs:189-231) and the ordered rayon batch GeodesicBatch::trace_ordered
// (batch.rs:31-43), here as a std::thread pool that writes each outcome at its input index.
#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

#include "oracle_footprint.hpp"
#include "oracle_radiation.hpp"
#include "oracle_tracer.hpp"
#include "oracle_variational.hpp"
#include "oracle_wgsl_rk4.hpp"

using namespace gro;

template <class F>
static void parallel_for(int64_t n, int threads, F&& body) {
  if (threads <= 1 || n <= 1) {
    for (int64_t i = 0; i < n; ++i) body(i);
    return;
  }
  std::atomic<int64_t> next{0};
  std::vector<std::thread> pool;
  const int t = int(std::min<int64_t>(threads, n));
  for (int w = 0; w < t; ++w)
    pool.emplace_back([&] {
      for (;;) {
        const int64_t i = next.fetch_add(1);
        if (i >= n) break;
        body(i);
      }
    });
  for (auto& th : pool) th.join();
}

extern "C" {

struct gro_policy {
  double position_rtol, position_atol, momentum_rtol, momentum_atol;
  double initial_step, minimum_step, maximum_step;
  double safety, minimum_factor, maximum_factor;
  uint64_t maximum_accepted_steps;
  uint32_t maximum_consecutive_rejects;
  uint32_t policy_id;
  double event_affine_tolerance, event_tie_tolerance, event_arming_band, singularity_guard;
};

struct gro_events {
  int32_t has_escape;
  int32_t has_surface;
  double escape_radius;
  double surface_inner, surface_outer;
  double horizon_offset;
  double intensity_at_six;
};

struct gro_scene {
  double mass, spin, charge;
  int32_t chart;  // 0 ingoing, 1 outgoing
  int32_t pad;
  double observer_txyz[4];
  double target_txyz[4];
  double up_hint[3];
  double frequency;
  uint32_t width, height;
  double vertical_fov;
};

struct gro_observer_info {
  double event[4];
  double g_tt;
  double gram_residual;
  double orientation;
  int32_t used_up_fallback;
  int32_t extremality;
  double outer_horizon;  // NaN when absent
  double four_velocity[4], image_right[4], image_up[4], arrival[4];
  double metric_covariant[16];
  double tangent_half_fov;
};

enum { GRO_FIELDS = 43 };

int gro_fields() { return GRO_FIELDS; }

static Policy to_policy(const gro_policy& p) {
  Policy q;
  q.id = int(p.policy_id);
  q.position_rtol = p.position_rtol;
  q.position_atol = p.position_atol;
  q.momentum_rtol = p.momentum_rtol;
  q.momentum_atol = p.momentum_atol;
  q.initial_step = p.initial_step;
  q.minimum_step = p.minimum_step;
  q.maximum_step = p.maximum_step;
  q.safety = p.safety;
  q.minimum_factor = p.minimum_factor;
  q.maximum_factor = p.maximum_factor;
  q.maximum_accepted_steps = p.maximum_accepted_steps;
  q.maximum_consecutive_rejects = p.maximum_consecutive_rejects;
  q.event_affine_tolerance = p.event_affine_tolerance;
  q.event_tie_tolerance = p.event_tie_tolerance;
  q.event_arming_band = p.event_arming_band;
  q.singularity_guard = p.singularity_guard;
  return q;
}

void gro_policy_preset(int which, gro_policy* out) {
  const Policy p = which == 1 ? Policy::strict_v1() : Policy::regular_v1();
  *out = {p.position_rtol, p.position_atol, p.momentum_rtol, p.momentum_atol, p.initial_step, p.minimum_step,
          p.maximum_step, p.safety, p.minimum_factor, p.maximum_factor, p.maximum_accepted_steps,
          p.maximum_consecutive_rejects, uint32_t(p.id), p.event_affine_tolerance, p.event_tie_tolerance,
          p.event_arming_band, p.singularity_guard};
}

static EventConfig to_events(const gro_events& e) {
  EventConfig c;
  c.has_escape = e.has_escape != 0;
  c.escape_radius = e.escape_radius;
  c.has_surface = e.has_surface != 0;
  c.surface_inner = e.surface_inner;
  c.surface_outer = e.surface_outer;
  c.horizon_offset = e.horizon_offset;
  return c;
}

static void pack(const Outcome& o, double* f) {
  f[0] = double(int(o.termination));
  f[1] = double(int(o.failure));
  f[2] = double(o.event_kind);
  f[3] = double(o.event_candidates);
  f[4] = o.event_affine;
  f[5] = o.event_bracket;
  f[6] = o.event_residual;
  for (int i = 0; i < 8; ++i) f[7 + i] = o.state[i];
  f[15] = o.affine_parameter;
  f[16] = o.has_turning_radius ? 1.0 : 0.0;
  f[17] = o.turning_radius;
  f[18] = o.azimuth_advance;
  f[19] = o.travel_time;
  f[20] = double(o.polar_side);
  f[21] = double(o.radial_turnings);
  f[22] = double(o.equatorial_crossings);
  f[23] = double(o.azimuth_winding);
  f[24] = double(o.accepted_steps);
  f[25] = double(o.rejected_steps);
  f[26] = double(o.rhs_evaluations);
  f[27] = o.minimum_step;
  f[28] = o.maximum_step;
  f[29] = o.max_null_residual;
  f[30] = o.max_energy_drift;
  f[31] = o.max_lz_drift;
  f[32] = o.max_carter_drift;
  f[33] = o.has_escape_direction ? 1.0 : 0.0;
  for (int i = 0; i < 3; ++i) f[34 + i] = o.escape_direction[i];
  f[37] = double(o.surface_status);
  f[38] = o.source_radius;
  f[39] = o.source_azimuth;
  f[40] = o.frequency_ratio;
  f[41] = o.emitted_intensity;
  f[42] = o.observed_intensity;
}

int gro_hardware_threads() { return int(std::thread::hardware_concurrency()); }

// Spacetime validation + exact horizon (spacetime.rs:134-238). Returns 0 on success.
int gro_spacetime_info(double m, double a, double q, int chart, int* extremality, double* outer_horizon) {
  Spacetime sp;
  if (!Spacetime::make(m, a, q, chart ? Chart::Outgoing : Chart::Ingoing, sp)) return -1;
  *extremality = int(sp.extremality);
  double rp;
  *outer_horizon = sp.outer_horizon_radius(rp) ? rp : std::numeric_limits<double>::quiet_NaN();
  return 0;
}

void gro_oblate_to_cartesian(double a, int chart, double r, double polar, double azimuth, double out[3]) {
  Spacetime sp;
  sp.spin_m = a;
  sp.chart = chart ? Chart::Outgoing : Chart::Ingoing;
  sp.oblate_to_cartesian(r, polar, azimuth, out);
}

double gro_prograde_isco(double m, double a, double q) { return prograde_isco(m, a, q); }

static int build_scene(const gro_scene& s, Spacetime& sp, StationaryObserver& obs, PerspectiveView& view) {
  if (!Spacetime::make(s.mass, s.spin, s.charge, s.chart ? Chart::Outgoing : Chart::Ingoing, sp)) return -1;
  const ObserverError oe = build_observer(sp, s.observer_txyz, s.target_txyz, s.up_hint, s.frequency, obs);
  if (oe != ObserverError::None) return -10 - int(oe);
  if (!PerspectiveView::make(s.width, s.height, s.vertical_fov, view)) return -3;
  return 0;
}

int gro_observer_info(const gro_scene* s, gro_observer_info* out) {
  Spacetime sp;
  StationaryObserver obs;
  PerspectiveView view;
  const int rc = build_scene(*s, sp, obs, view);
  if (rc != 0) return rc;
  for (int i = 0; i < 4; ++i) {
    out->event[i] = obs.event[i];
    out->four_velocity[i] = obs.frame.four_velocity.v[i];
    out->image_right[i] = obs.frame.image_right.v[i];
    out->image_up[i] = obs.frame.image_up.v[i];
    out->arrival[i] = obs.frame.arrival.v[i];
  }
  out->g_tt = obs.metric_g_tt;
  out->gram_residual = obs.frame.gram_residual;
  out->orientation = obs.frame.orientation_determinant;
  out->used_up_fallback = obs.frame.used_up_fallback;
  out->extremality = int(sp.extremality);
  double rp;
  out->outer_horizon = sp.outer_horizon_radius(rp) ? rp : std::numeric_limits<double>::quiet_NaN();
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) out->metric_covariant[r * 4 + c] = obs.metric_covariant[r][c];
  out->tangent_half_fov = view.tangent_half_fov;
  return 0;
}

// Initial rays for image samples (scene.rs:211-270). status[i] = 0 on success.
int gro_initial_rays(const gro_scene* s, int64_t n, const uint32_t* px, const uint32_t* py, const double* sx,
                     const double* sy, double* states, double* frequency, double* residual, int32_t* status) {
  Spacetime sp;
  StationaryObserver obs;
  PerspectiveView view;
  const int rc = build_scene(*s, sp, obs, view);
  if (rc != 0) return rc;
  for (int64_t i = 0; i < n; ++i) {
    InitialRay ray;
    const InitialRayError e = initial_ray(obs, view, px[i], py[i], sx[i], sy[i], ray);
    status[i] = int(e);
    if (e == InitialRayError::None) {
      for (int c = 0; c < 8; ++c) states[8 * i + c] = ray.state[c];
      frequency[i] = ray.observer_frequency;
      residual[i] = ray.normalized_null_residual;
    }
  }
  return 0;
}

// GeodesicTracer::trace over explicit states (geodesic.rs:53-62), ordered batch (batch.rs:31-43).
int gro_trace_states(double m, double a, double q, int chart, const gro_policy* pol, const gro_events* ev, int64_t n,
                     const double* states, double direction, int threads, double* out) {
  Spacetime sp;
  if (!Spacetime::make(m, a, q, chart ? Chart::Outgoing : Chart::Ingoing, sp)) return -1;
  if (bits_of(sp.mass_m) != bits_of(1.0)) return -2;  // geodesic.rs:33-35
  Tracer tr{sp, to_policy(*pol), to_events(*ev)};
  parallel_for(n, threads, [&](int64_t i) { pack(tr.trace(states + 8 * i, direction), out + GRO_FIELDS * i); });
  return 0;
}

// ObservationTracer::trace over image samples (observation.rs:189-231).
int gro_trace_pixels(const gro_scene* s, const gro_policy* pol, const gro_events* ev, int64_t n, const uint32_t* px,
                     const uint32_t* py, const double* sx, const double* sy, int threads, double* out,
                     int32_t* status) {
  Spacetime sp;
  StationaryObserver obs;
  PerspectiveView view;
  const int rc = build_scene(*s, sp, obs, view);
  if (rc != 0) return rc;
  if (bits_of(sp.mass_m) != bits_of(1.0)) return -2;
  Tracer tr{sp, to_policy(*pol), to_events(*ev)};
  if (tr.events.has_surface && tr.events.has_escape && tr.events.surface_outer >= tr.events.escape_radius)
    return -4;  // events.rs:73-78
  parallel_for(n, threads, [&](int64_t i) {
    InitialRay ray;
    const InitialRayError e = initial_ray(obs, view, px[i], py[i], sx[i], sy[i], ray);
    status[i] = int(e);
    if (e != InitialRayError::None) return;
    if (std::fabs(ray.observer_frequency - 1.0) > 32.0 * 2.220446049250313e-16) {
      status[i] = 100;  // observation.rs:200-202
      return;
    }
    const Outcome o = trace_observation(tr, ray, ev->intensity_at_six);
    pack(o, out + GRO_FIELDS * i);
  });
  return 0;
}

// surface.rs:12-146 for one terminal state (bolometric vacuum emitter).
int gro_surface_observable(double m, double a, double q, int chart, double inner, double outer, double intensity,
                           const double* state, double observer_frequency, double* out5) {
  Spacetime sp;
  if (!Spacetime::make(m, a, q, chart ? Chart::Outgoing : Chart::Ingoing, sp)) return -100;
  Outcome o{};
  const int s = observable_at(sp, inner, outer, intensity, state, observer_frequency, o);
  out5[0] = o.source_radius;
  out5[1] = o.source_azimuth;
  out5[2] = o.frequency_ratio;
  out5[3] = o.emitted_intensity;
  out5[4] = o.observed_intensity;
  return s;
}

// Invariants and normalized null residual of one state (spacetime.rs:345-401).
int gro_invariants(double m, double a, double q, int chart, const double* state, double* out4) {
  Spacetime sp;
  if (!Spacetime::make(m, a, q, chart ? Chart::Outgoing : Chart::Ingoing, sp)) return -100;
  Invariants inv;
  const GeometryError e = sp.invariants(state, inv);
  if (e != GeometryError::None) return int(e);
  out4[0] = inv.energy;
  out4[1] = inv.angular_momentum_z;
  out4[2] = inv.carter_constant;
  out4[3] = inv.normalized_null_residual;
  return 0;
}

// Canonical Hamilton right-hand side of one state (spacetime.rs:305-338).
int gro_hamiltonian_rhs(double m, double a, double q, int chart, const double* state, double* out8) {
  Spacetime sp;
  if (!Spacetime::make(m, a, q, chart ? Chart::Outgoing : Chart::Ingoing, sp)) return -100;
  return int(sp.hamiltonian_rhs(state, out8));
}

// Surface radiation model (radiation.rs, surface.rs): Planck integral, band split, radiance.
double gro_planck_integral(double lo, double hi) { return integrate_planck(lo, hi); }

int gro_blackbody_bands(double intensity, double temperature, double* out3) {
  return blackbody_bands(intensity, temperature, out3) ? 1 : 0;
}

int gro_surface_radiance(int model, double i6, double t6, int slab, double tau, double s, double tslab, double r,
                         double g, double* out5) {
  return surface_radiance(model, i6, t6, slab != 0, tau, s, tslab, r, g, out5) ? 1 : 0;
}

// Surface footprint (footprint.rs:74-150) of n pixel samples: the center and its four quarter-pixel
// neighbours traced through the observation. out8 per sample as gro::surface_footprint; status =
// FootprintStatus, or -100 - InitialRayError for a sample whose rays cannot be set up.
int gro_surface_footprint(const gro_scene* s, const gro_policy* pol, const gro_events* ev, int64_t n,
                          const uint32_t* px, const uint32_t* py, const double* sx, const double* sy, int threads,
                          double* out8, int32_t* status) {
  Spacetime sp;
  StationaryObserver obs;
  PerspectiveView view;
  const int rc = build_scene(*s, sp, obs, view);
  if (rc != 0) return rc;
  if (bits_of(sp.mass_m) != bits_of(1.0)) return -2;
  Tracer tr{sp, to_policy(*pol), to_events(*ev)};
  if (tr.events.has_surface && tr.events.has_escape && tr.events.surface_outer >= tr.events.escape_radius)
    return -4;
  for (int64_t i = 0; i < n; ++i)
    if (!(sx[i] >= 0.25 && sx[i] <= 0.75 && sy[i] >= 0.25 && sy[i] <= 0.75)) return -5;  // footprint.rs:82-86
  parallel_for(n, threads, [&](int64_t i) {
    const double off[5][2] = {{0.0, 0.0}, {-0.25, 0.0}, {0.25, 0.0}, {0.0, -0.25}, {0.0, 0.25}};
    Outcome o[5];
    for (int k = 0; k < 5; ++k) {
      InitialRay ray;
      const InitialRayError e = initial_ray(obs, view, px[i], py[i], sx[i] + off[k][0], sy[i] + off[k][1], ray);
      if (e != InitialRayError::None) {
        status[i] = -100 - int(e);
        for (int j = 0; j < 8; ++j) out8[8 * i + j] = NAN;
        return;
      }
      o[k] = trace_observation(tr, ray, ev->intensity_at_six);
    }
    status[i] = surface_footprint(o, out8 + 8 * i);
  });
  return 0;
}

// footprint.rs:203-235 on one Jacobian: out4 = determinant, squared norm, major, minor.
int gro_footprint_metrics(const double* J, double* out4) {
  FootprintMetrics m;
  if (!footprint_metrics(J, m)) return 0;
  out4[0] = m.determinant;
  out4[1] = m.squared_norm;
  out4[2] = m.major;
  out4[3] = m.minor;
  return 1;
}

// Internal numerical differentiation of traces (the check of the discrete adjoint; not part of the
// reference): for each ray, the observables (source radius and g at a surface hit with g's observer
// frequency 1; escape polar and azimuthal angle of the coordinate direction at an escape) and their
// central differences with respect to p_t, p_x, p_y, p_z of the initial state and to a and Q of the
// spacetime, every perturbed trace replaying the unperturbed trace's accepted step sizes.
// out: 30 doubles per ray = termination, ok, the 4 observables, then d(4 observables)/d(param) for
// the 6 parameters in that order (param-major). h_rel: step relative to |p| (momenta) or absolute
// (a, Q).
int gro_ind_gradients(double m, double a, double q, int chart, const gro_policy* pol, const gro_events* ev, int64_t n,
                      const double* states, double direction, double h_rel, int threads, double* out) {
  Spacetime sp;
  if (!Spacetime::make(m, a, q, chart ? Chart::Outgoing : Chart::Ingoing, sp)) return -100;
  const Policy policy = to_policy(*pol);
  const EventConfig events = to_events(*ev);
  auto observe = [&](const Tracer& tr, const Outcome& o, double obs[4]) {
    for (int k = 0; k < 4; ++k) obs[k] = NAN;
    if (o.termination == Termination::EquatorialSurface) {
      if (tr.sp.radius(o.state, obs[0]) != GeometryError::None) return false;
      Outcome so{};
      if (observable_at(tr.sp, events.surface_inner, events.surface_outer, 1.0, o.state, 1.0, so) != 1) return false;
      obs[1] = so.frequency_ratio;
      return true;
    }
    if (o.termination == Termination::Escape && o.has_escape_direction) {
      obs[2] = std::acos(std::fmax(-1.0, std::fmin(1.0, o.escape_direction[2])));
      obs[3] = std::atan2(o.escape_direction[1], o.escape_direction[0]);
      return true;
    }
    return false;
  };
  parallel_for(n, threads, [&](int64_t i) {
    double* row = out + 30 * i;
    for (int k = 0; k < 30; ++k) row[k] = 0.0;
    const double* st = states + 8 * i;
    const Tracer base{sp, policy, events};
    std::vector<double> steps;
    const Outcome o0 = base.trace(st, direction, &steps, nullptr);
    row[0] = double(int(o0.termination));
    double obs0[4];
    if (!observe(base, o0, obs0)) return;
    for (int k = 0; k < 4; ++k) row[2 + k] = obs0[k];
    const double pn = std::sqrt(st[5] * st[5] + st[6] * st[6] + st[7] * st[7]);
    for (int p = 0; p < 6; ++p) {
      double d[2][4];
      const double h = p < 4 ? h_rel * pn : h_rel;
      for (int sgn = 0; sgn < 2; ++sgn) {
        const double hs = sgn == 0 ? h : -h;
        double s2[8];
        for (int c = 0; c < 8; ++c) s2[c] = st[c];
        Spacetime sp2 = sp;
        if (p < 4) {
          s2[4 + p] += hs;
        } else if (!Spacetime::make(m, p == 4 ? a + hs : a, p == 5 ? q + hs : q, sp.chart, sp2)) {
          return;
        }
        const Tracer tr{sp2, policy, events};
        const Outcome o = tr.trace(s2, direction, nullptr, &steps);
        if (o.termination != o0.termination || o.accepted_steps != o0.accepted_steps || !observe(tr, o, d[sgn])) return;
      }
      for (int k = 0; k < 4; ++k) {
        double diff = d[0][k] - d[1][k];
        if (k == 3) diff = std::remainder(diff, 2.0 * M_PI);
        row[6 + 4 * p + k] = std::isfinite(diff) ? diff / (2.0 * h) : 0.0;
      }
    }
    row[1] = 1.0;
  });
  return 0;
}

// Variational-equation reference gradients (oracle_variational.hpp): per ray (termination, ok, the
// 4 observables of gro_ind_gradients, then their derivatives with respect to (p_t, p_x, p_y, p_z,
// a, Q), param-major), the same 30-column layout as gro_ind_gradients.
int gro_variational_gradients(double m, double a, double q, int chart, const gro_policy* pol, const gro_events* ev,
                              int64_t n, const double* states, double direction, int threads, double* out) {
  Spacetime sp;
  if (!Spacetime::make(m, a, q, chart ? Chart::Outgoing : Chart::Ingoing, sp)) return -100;
  const Tracer base{sp, to_policy(*pol), to_events(*ev)};
  parallel_for(n, threads, [&](int64_t i) {
    double* row = out + 30 * i;
    Termination term;
    double obs[4], grad[kVarParams][4];
    const bool ok = variational_gradient(base, states + 8 * i, direction, term, obs, grad);
    row[0] = double(int(term));
    row[1] = ok ? 1.0 : 0.0;
    for (int k = 0; k < 4; ++k) row[2 + k] = obs[k];
    for (int p = 0; p < kVarParams; ++p)
      for (int k = 0; k < 4; ++k) row[6 + 4 * p + k] = ok ? grad[p][k] : 0.0;
  });
  return 0;
}

// KerrNewmanSpacetime::metric_covariant_at (spacetime.rs:485-490): g_{mu nu} = eta + f l l at a
// Cartesian Kerr-Schild event; out16 row-major. Returns 0, or -1 for invalid parameters and
// -2 where the geometry is singular.
int gro_metric_covariant(double m, double a, double q, int chart, const double* txyz, double* out16) {
  Spacetime sp;
  if (!Spacetime::make(m, a, q, chart ? Chart::Outgoing : Chart::Ingoing, sp)) return -1;
  Geometry g;
  if (sp.geometry(txyz, g) != GeometryError::None) return -2;
  double mm[4][4];
  Spacetime::metric_covariant(g, mm);
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) out16[4 * r + c] = mm[r][c];
  return 0;
}

// The reference's GPU RK4 kernel restated in binary32 (oracle_wgsl_rk4.hpp) over image samples,
// with the uniforms input.rs:64-131 packs: M = 1, the chart as +1 ingoing / -1 outgoing, the tetrad
// legs and tan(fov/2) narrowed from binary64, guard 2^-40, tie tolerance 2^-17 M, arming band
// 2^-12 M, step policy (0.1, 0.005, 8) and drift limit 0.05. The event surfaces are the job's
// (escape radius; capture at the outer horizon of the narrowed spacetime plus the job's offset;
// surface radii). out: 16 doubles per ray = termination, failure flags, event candidates, steps,
// event residual, source[3] (escape: unit -dx/dlambda; surface: radius, azimuth, g), travel time,
// drift[4] (null residual, 0, L_z, Carter), radial turnings, equatorial crossings, azimuth winding.
int gro_rk4_pixels(const gro_scene* s, const gro_events* ev, int64_t n, const uint32_t* px, const uint32_t* py,
                   const double* sx, const double* sy, int threads, double* out) {
  Spacetime sp;
  StationaryObserver obs;
  PerspectiveView view;
  const int rc = build_scene(*s, sp, obs, view);
  if (rc != 0) return rc;
  if (bits_of(sp.mass_m) != bits_of(1.0)) return -2;
  if (!ev->has_escape) return -5;
  rk4::Uniforms U{};
  U.mass = 1.0f;
  U.spin = float(s->spin);
  U.charge = float(s->charge);
  U.chart = s->chart ? -1.0f : 1.0f;
  U.observer = {float(obs.event[1]), float(obs.event[2]), float(obs.event[3])};
  for (int i = 0; i < 4; ++i) {
    U.velocity[i] = float(obs.frame.four_velocity.v[i]);
    U.right[i] = float(obs.frame.image_right.v[i]);
    U.up[i] = float(obs.frame.image_up.v[i]);
    U.arrival[i] = float(obs.frame.arrival.v[i]);
  }
  U.tan_half_fov = float(view.tangent_half_fov);
  U.frequency = 1.0f;
  Spacetime narrowed;
  double rp = -1.0;
  if (Spacetime::make(1.0, double(U.spin), double(U.charge), sp.chart, narrowed) && narrowed.outer_horizon_radius(rp))
    rp += ev->horizon_offset;
  else
    rp = -1.0;
  U.escape = float(ev->escape_radius);
  U.guard = 0x1p-40f;
  U.horizon = float(rp);
  U.tie = 0x1p-17f;
  U.surface = ev->has_surface != 0;
  U.inner = U.surface ? float(ev->surface_inner) : 0.0f;
  U.outer = U.surface ? float(ev->surface_outer) : 0.0f;
  U.arming = U.surface ? 0x1p-12f : 0.0f;
  U.step_scale = 0.1f;
  U.step_min = 0.005f;
  U.step_max = 8.0f;
  U.drift_limit = 0.05f;
  parallel_for(n, threads, [&](int64_t i) {
    const rk4::Result r = rk4::trace_pixel(U, s->width, s->height, px[i], py[i], float(sx[i]), float(sy[i]));
    double* row = out + 16 * i;
    row[0] = r.termination;
    row[1] = r.flags;
    row[2] = r.candidates;
    row[3] = r.steps;
    row[4] = r.event_residual;
    for (int k = 0; k < 3; ++k) row[5 + k] = r.source[k];
    row[8] = r.travel_time;
    for (int k = 0; k < 4; ++k) row[9 + k] = r.drift[k];
    row[13] = r.turnings;
    row[14] = r.crossings;
    row[15] = r.winding;
  });
  return 0;
}

}  // extern "C"
