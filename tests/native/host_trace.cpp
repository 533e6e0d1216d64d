// Test harness (not product code): runs the device tracer's per-ray state machine
// (gravlume_b200/csrc/glc_tracer.cuh, compiled here for the host) over explicit initial states so
// that the kernel logic -- event arming and localization, mixed-precision consistency, turning
// points, crossings -- can be checked against the oracle without a GPU. The MIXED shell decision is
// taken per ray here (the kernels take it per warp).
#include <cstdint>

#include <vector>

#include "../../gravlume_b200/csrc/glc_adjoint.cuh"

using namespace glc;

namespace {
template <int P>
void run(const glc_scene& sc, const glc_policy& pol, int64_t n, const double* st, double dir, double* out, int nf) {
  const LaneScene ls = make_lane_scene(sc, pol.mixed_shell_factor);
  for (int64_t i = 0; i < n; ++i) {
    Ray<P> ray;
    ray.init(ls, pol, st + 8 * i, dir);
    RayResult<typename PrecTraits<P>::S> res;
    for (;;) {
      const bool use64 = P == kMIXED && double(ray.r) < ls.shell_r;
      const bool done = ray.step(ls, pol, res, use64);
      if (done) break;
    }
    double* o = out + nf * i;
    o[0] = res.termination;
    o[1] = res.failure;
    o[2] = res.candidates;
    o[3] = res.flags;
    o[4] = ray.accepted;
    o[5] = ray.rejected;
    o[6] = ray.turnings;
    o[7] = ray.crossings;
    o[8] = ray.winding;
    o[9] = double(res.escape_theta);
    o[10] = double(res.escape_phi);
    o[11] = double(res.surface_r);
    o[12] = double(res.surface_phi);
    o[13] = double(res.g);
    o[14] = double(ray.travel());
    o[15] = double(res.event_residual);
    o[16] = double(ray.affine());
    o[17] = double(ray.dnull);
    o[18] = double(ray.dlz);
    o[19] = double(ray.dq);
    o[20] = double(ray.turn_r);
    o[21] = double(ray.azimuth_advance());
    for (int c = 0; c < 6; ++c) o[22 + c] = double(ray.ys(c));
    o[28] = ray.f64steps;
  }
}
// MIXED as two kernels: BULK steps each ray until it hands off, the record is packed and unpacked
// as between the kernels, and TAIL finishes the ray (the outputs are TAIL's).
void run_split(const glc_scene& sc, const glc_policy& pol, int64_t n, const double* st, double dir, double* out,
               int nf) {
  const LaneScene ls = make_lane_scene(sc, pol.mixed_shell_factor);
  for (int64_t i = 0; i < n; ++i) {
    Ray<kBULK> bulk;
    bulk.init(ls, pol, st + 8 * i, dir);
    RayResult<float> bres;
    while (!bulk.step(ls, pol, bres, false)) {
    }
    HandoffRec rec;
    handoff_pack(bulk, bres, rec);
    Ray<kTAIL> ray;
    uint32_t failure = 0;
    const uint32_t term = handoff_unpack(rec, ray, ls, st + 8 * i, dir, failure);
    RayResult<double> res;
    if (term != GLC_TERM_NONE) {
      ray.finish_plain(res, term, failure);
    } else {
      while (!ray.step(ls, pol, res, false)) {
      }
    }
    double* o = out + nf * i;
    o[0] = res.termination;
    o[1] = res.failure;
    o[2] = res.candidates;
    o[3] = res.flags;
    o[4] = ray.accepted;
    o[5] = ray.rejected;
    o[6] = ray.turnings;
    o[7] = ray.crossings;
    o[8] = ray.winding;
    o[9] = res.escape_theta;
    o[10] = res.escape_phi;
    o[11] = res.surface_r;
    o[12] = res.surface_phi;
    o[13] = res.g;
    o[14] = ray.travel();
    o[15] = res.event_residual;
    o[16] = ray.affine();
    o[17] = ray.dnull;
    o[18] = ray.dlz;
    o[19] = ray.dq;
    o[20] = ray.turn_r;
    o[21] = ray.azimuth_advance();
    for (int c = 0; c < 6; ++c) o[22 + c] = ray.ys(c);
    o[28] = ray.f64steps;
  }
}
}  // namespace

extern "C" int host_trace_fields() { return 29; }

// precision 0 FP32, 1 MIXED (one kernel), 2 FP64, 3 MIXED as two kernels (BULK + TAIL)
extern "C" int host_trace_split(const glc_scene* sc, const glc_policy* pol, int64_t n, const double* states,
                                double dir, double* out) {
  run_split(*sc, *pol, n, states, dir, out, 29);
  return 0;
}

extern "C" int host_trace_states(const glc_scene* sc, const glc_policy* pol, int64_t n, const double* states,
                                 double dir, double* out) {
  switch (pol->precision) {
    case 0: run<kFP32>(*sc, *pol, n, states, dir, out, 29); return 0;
    case 1: run<kMIXED>(*sc, *pol, n, states, dir, out, 29); return 0;
    case 2: run<kFP64>(*sc, *pol, n, states, dir, out, 29); return 0;
  }
  return -1;
}

// Discrete adjoint of whole traces, every accepted step recorded (no checkpoints): for each ray,
// dL/d(initial x, y, z, p_x, p_y, p_z), dL/dE, dL/da, dL/dQ^2 for the observable weights wobs
// (source radius, g, escape theta, escape phi). out: 9 gradients, termination, ok, accepted steps.
namespace {
template <int P>
void adjoint(const glc_scene& sc, const glc_policy& pol, int64_t n, const double* st, double dir, const double* wobs,
             double* out) {
  const LaneScene ls = make_lane_scene(sc, pol.mixed_shell_factor);
  const KN<D4> kd = kn_dual_vjp(ls.kn);
  for (int64_t i = 0; i < n; ++i) {
    Ray<P> ray;
    ray.init(ls, pol, st + 8 * i, dir);
    RayResult<typename PrecTraits<P>::S> res;
    std::vector<double> tape;  // per accepted step: y0[6], h
    double y0[6], h0 = 0.0;
    for (;;) {
      for (int c = 0; c < 6; ++c) y0[c] = double(ray.ys(c));
      h0 = double(ray.h);
      const uint32_t acc = ray.accepted;
      const bool use64 = P == kMIXED && double(ray.r) < ls.shell_r;
      if (ray.step(ls, pol, res, use64)) break;
      if (ray.accepted != acc) {
        tape.insert(tape.end(), y0, y0 + 6);
        tape.push_back(h0);
      }
    }
    double* o = out + 12 * i;
    for (int c = 0; c < 12; ++c) o[c] = 0.0;
    o[9] = res.termination;
    o[11] = double(tape.size() / 7);
    double lam[6], g[3] = {0, 0, 0};
    const double E = double(ray.E);
    if (!terminal_reverse(ls, y0, E, h0, double(res.event_theta), dir, res.termination, wobs + kObs * i, lam, g))
      continue;
    double w[7];
    step_weights(w);
    for (size_t m = tape.size() / 7; m-- > 0;) {
      const double* rec = tape.data() + 7 * m;
      double l0[6];
      dp5_reverse(ls.kn, kd, rec, E, rec[6], w, lam, l0, g);
      for (int c = 0; c < 6; ++c) lam[c] = l0[c];
    }
    for (int c = 0; c < 6; ++c) o[c] = lam[c];
    o[6] = g[0];
    o[7] = g[1];
    o[8] = g[2];
    o[10] = 1.0;
  }
}

// Observables of traces under a scene whose spin and squared charge are shifted by (da, dq2) in the
// dynamics only (the initial states are given): termination, source radius, g, escape theta, phi.
template <int P>
void perturbed(const glc_scene& sc, const glc_policy& pol, int64_t n, const double* st, double dir, double da,
               double dq2, double* out) {
  LaneScene ls = make_lane_scene(sc, pol.mixed_shell_factor);
  ls.kn.a += da;
  ls.kn.a2 = ls.kn.a * ls.kn.a;
  ls.kn.sa = ls.kn.s * ls.kn.a;
  ls.kn.q2 += dq2;
  for (int64_t i = 0; i < n; ++i) {
    Ray<P> ray;
    ray.init(ls, pol, st + 8 * i, dir);
    RayResult<typename PrecTraits<P>::S> res;
    for (;;) {
      const bool use64 = P == kMIXED && double(ray.r) < ls.shell_r;
      if (ray.step(ls, pol, res, use64)) break;
    }
    double* o = out + 5 * i;
    o[0] = res.termination;
    o[1] = double(res.surface_r);
    o[2] = double(res.g);
    o[3] = double(res.escape_theta);
    o[4] = double(res.escape_phi);
  }
}
}  // namespace

extern "C" int host_adjoint_states(const glc_scene* sc, const glc_policy* pol, int64_t n, const double* states,
                                   double dir, const double* wobs, double* out) {
  switch (pol->precision) {
    case 1: adjoint<kMIXED>(*sc, *pol, n, states, dir, wobs, out); return 0;
    case 2: adjoint<kFP64>(*sc, *pol, n, states, dir, wobs, out); return 0;
  }
  return -1;
}

extern "C" int host_trace_perturbed(const glc_scene* sc, const glc_policy* pol, int64_t n, const double* states,
                                    double dir, double da, double dq2, double* out) {
  switch (pol->precision) {
    case 1: perturbed<kMIXED>(*sc, *pol, n, states, dir, da, dq2, out); return 0;
    case 2: perturbed<kFP64>(*sc, *pol, n, states, dir, da, dq2, out); return 0;
  }
  return -1;
}

// The device's surface transport (glc_radiation.cuh) for the CPU checks.
extern "C" int host_blackbody_bands(double intensity, double temperature, double* out3) {
  return blackbody_bands(intensity, temperature, out3) ? 1 : 0;
}

extern "C" int host_surface_radiance(int model, double i6, double t6, int slab, double tau, double s, double tslab,
                                     double r, double g, double* out5) {
  double bands[3] = {0.0, 0.0, 0.0};
  if (slab && model == 1 && s > 0.0 && !blackbody_bands(s, tslab, bands)) return 0;
  const double trans = slab ? std::exp(-tau) : 1.0;
  double em, ob, rgb[3];
  if (!surface_radiance(model, i6, t6, trans, slab ? s : 0.0, bands, r, g, em, ob, rgb)) return 0;
  out5[0] = em;
  out5[1] = ob;
  for (int b = 0; b < 3; ++b) out5[2 + b] = rgb[b];
  return 1;
}

// Both stage VJPs at n states (rows of 6) with energy E and cotangents kbar (rows of 6): out rows of
// 18 = (ybar, g) from the 4-channel Hamiltonian form, then (ybar, g) from the 9-channel Jacobian.
extern "C" int host_rhs_vjp_pair(const glc_scene* sc, int64_t n, const double* y, const double* E,
                                 const double* kbar, double* out) {
  const LaneScene ls = make_lane_scene(*sc, 3.0);
  const KN<D4> k4 = kn_dual_vjp(ls.kn);
  const KN<D9> k9 = kn_dual(ls.kn);
  for (int64_t i = 0; i < n; ++i) {
    double* o = out + 18 * i;
    for (int c = 0; c < 18; ++c) o[c] = 0.0;
    rhs_vjp(k4, y + 6 * i, E[i], kbar + 6 * i, o, o + 6);
    rhs_vjp_jacobian(k9, y + 6 * i, E[i], kbar + 6 * i, o + 9, o + 15);
  }
  return 0;
}
