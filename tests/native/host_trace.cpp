// Test harness (not product code): runs the device tracer's per-ray state machine
// (gravlume_b200/csrc/glc_tracer.cuh, compiled here for the host) over explicit initial states so
// that the kernel logic -- event arming and localization, mixed-precision consistency, turning
// points, crossings -- can be checked against the oracle without a GPU. The MIXED shell decision is
// taken per ray here (the kernels take it per warp).
#include <cstdint>

#include "../../gravlume_b200/csrc/glc_tracer.cuh"

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
}  // namespace

extern "C" int host_trace_fields() { return 29; }

extern "C" int host_trace_states(const glc_scene* sc, const glc_policy* pol, int64_t n, const double* states,
                                 double dir, double* out) {
  switch (pol->precision) {
    case 0: run<kFP32>(*sc, *pol, n, states, dir, out, 29); return 0;
    case 1: run<kMIXED>(*sc, *pol, n, states, dir, out, 29); return 0;
    case 2: run<kFP64>(*sc, *pol, n, states, dir, out, 29); return 0;
  }
  return -1;
}
