// Trace kernels: ray setup from a camera, result stores, the one-thread-per-ray kernel and the
// persistent work-queue kernel with warp-level refill of finished lanes.
#pragma once

#include <cuda_runtime.h>

#include "glc_tracer.cuh"

namespace glc {

// Device view of one trace job: scenes, cameras and the prefix of their (padded) ray counts.
struct JobView {
  const glc_scene* scenes;
  const glc_camera* cams;
  const unsigned long long* begin;  // n_cams + 1 entries
  int n_cams;
  unsigned long long total;
  const unsigned long long* cert_begin;  // n_cams + 1 entries: first 16x16-tile word of each camera
  const uint32_t* cert;                  // per-tile capture certificates, or null when not evaluated
};

// Initial state of ray gi of the job. Image rays are generated in binary64 from the camera basis
// (scene.rs:211-270, view.rs:408-424): sight = (s_x right + s_y up - arrival) / |.|,
// p^mu = omega (u^mu - sight^mu), p_mu = g_{mu nu} p^nu at the observer. Returns false for tile
// padding outside the image.
__device__ __forceinline__ bool ray_setup(const JobView& job, const glc_policy& pol, unsigned long long gi,
                                          double st8[8], double& dir, unsigned long long& slot, int& scene_idx,
                                          bool& certified) {
  certified = false;
  int lo = 0, hi = job.n_cams - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (job.begin[mid] <= gi) lo = mid;
    else hi = mid - 1;
  }
  const glc_camera* cam = job.cams + lo;
  const unsigned long long j = gi - job.begin[lo];
  scene_idx = cam->scene_index;
  if (cam->kind == GLC_CAMERA_RAYLIST) {
    const double2* src = reinterpret_cast<const double2*>(cam->ray_states + 8ull * j);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const double2 v = __ldg(src + i);
      st8[2 * i] = v.x;
      st8[2 * i + 1] = v.y;
    }
    dir = cam->affine_direction;
    slot = cam->result_offset + j;
    return true;
  }
  const uint32_t W = cam->width, H = cam->height;
  const uint32_t tw = pol.tile_w, th = pol.tile_h;
  const uint32_t tiles_x = (W + tw - 1) / tw;
  const unsigned long long per_tile = (unsigned long long)tw * th;
  const unsigned long long tile = j / per_tile;
  const uint32_t within = uint32_t(j - tile * per_tile);
  const uint32_t px = uint32_t(tile % tiles_x) * tw + within % tw;
  const uint32_t py = uint32_t(tile / tiles_x) * th + within / tw;
  if (px >= W || py >= H) return false;
  slot = cam->result_offset + (unsigned long long)py * W + px;
  dir = -1.0;
  if (job.cert) {
    const unsigned long long t = job.cert_begin[lo] + (unsigned long long)(py >> 4) * ((W + 15u) >> 4) + (px >> 4);
    if (job.cert[t]) {
      certified = true;
      return true;
    }
  }
  const glc_scene* sc = job.scenes + scene_idx;
  double sight[4];
  if (cam->kind == GLC_CAMERA_PINHOLE) {
    const double w = double(W), h = double(H);
    const double nx = 2.0 * (double(px) + cam->subpixel_x) / w - 1.0;
    const double ny = 1.0 - 2.0 * (double(py) + cam->subpixel_y) / h;
    const double sx = (w / h) * sc->tangent_half_fov * nx;
    const double sy = sc->tangent_half_fov * ny;
    const double nrm = 1.0 / hypot(1.0, hypot(sx, sy));
#pragma unroll
    for (int i = 0; i < 4; ++i) sight[i] = (sc->image_right[i] * sx + sc->image_up[i] * sy - sc->arrival[i]) * nrm;
  } else {
    // equirectangular full sphere in the observer frame: longitude about image-up, zero along
    // the sight axis (-arrival), latitude towards image-up
    const double lon = 2.0 * M_PI * ((double(px) + cam->subpixel_x) / double(W)) - M_PI;
    const double lat = 0.5 * M_PI - M_PI * ((double(py) + cam->subpixel_y) / double(H));
    double sl, cl, sb, cb;
    sincos(lon, &sl, &cl);
    sincos(lat, &sb, &cb);
#pragma unroll
    for (int i = 0; i < 4; ++i)
      sight[i] = cb * sl * sc->image_right[i] + sb * sc->image_up[i] - cb * cl * sc->arrival[i];
  }
  double pc[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) pc[i] = sc->frequency * (sc->four_velocity[i] - sight[i]);
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < 4; ++c) s += sc->metric_covariant[4 * r + c] * pc[c];
    st8[4 + r] = s;
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) st8[i] = sc->observer_txyz[i];
  return true;
}

template <int P>
__device__ __forceinline__ void write_result(const glc_results& o, unsigned long long slot, const Ray<P>& ray,
                                             const RayResult<typename PrecTraits<P>::S>& res, const LaneScene& ls) {
  using S = typename PrecTraits<P>::S;
  const uint32_t code = (res.termination & 0xFFu) | ((res.failure & 0xFu) << 8) | ((res.candidates & 0xFu) << 12) |
                        (uint32_t(ray.polar + 1) << 16) | ((res.flags & 0xFFFu) << 20);
  if (o.code) reinterpret_cast<uint4*>(o.code)[slot] = make_uint4(code, ray.accepted, ray.rejected, ray.f64steps);
  if (o.branch)
    reinterpret_cast<int4*>(o.branch)[slot] =
        make_int4(int(ray.turnings), int(ray.crossings), ray.winding, ray.turn_r == ray.turn_r ? 1 : 0);
  if (o.escape) reinterpret_cast<double2*>(o.escape)[slot] = make_double2(double(res.escape_theta), double(res.escape_phi));
  if (o.surface) reinterpret_cast<double2*>(o.surface)[slot] = make_double2(double(res.surface_r), double(res.surface_phi));
  const S travel = ray.travel();
  if (o.redshift_time) reinterpret_cast<double2*>(o.redshift_time)[slot] = make_double2(double(res.g), double(travel));
  if (o.event) reinterpret_cast<double2*>(o.event)[slot] = make_double2(double(res.event_residual), double(ray.affine()));
  if (o.drift_a) reinterpret_cast<double2*>(o.drift_a)[slot] = make_double2(double(ray.dnull), 0.0);
  if (o.drift_b) reinterpret_cast<double2*>(o.drift_b)[slot] = make_double2(double(ray.dlz), double(ray.dq));
  if (o.turning)
    reinterpret_cast<double2*>(o.turning)[slot] = make_double2(double(ray.turn_r), double(ray.azimuth_advance()));
  if (o.position_xy) reinterpret_cast<double2*>(o.position_xy)[slot] = make_double2(double(ray.ys(0)), double(ray.ys(1)));
  if (o.position_zr) {
    int gs;
    const double r = kn_radius(ls.kn, double(ray.ys(0)), double(ray.ys(1)), double(ray.ys(2)), gs);
    reinterpret_cast<double2*>(o.position_zr)[slot] = make_double2(double(ray.ys(2)), r);
  }
}

// A ray of a certified tile: horizon capture proven without integration (flag bit 2, code bit
// 22); the integration observables are NaN and the counters zero.
__device__ __forceinline__ void write_certified(const glc_results& o, unsigned long long slot) {
  const double nan = __longlong_as_double(0x7ff8000000000000ll);
  const uint32_t code = uint32_t(GLC_TERM_HORIZON) | (1u << 16) | (4u << 20);
  if (o.code) reinterpret_cast<uint4*>(o.code)[slot] = make_uint4(code, 0u, 0u, 0u);
  if (o.branch) reinterpret_cast<int4*>(o.branch)[slot] = make_int4(0, 0, 0, 0);
  const double2 nn = make_double2(nan, nan);
  if (o.escape) reinterpret_cast<double2*>(o.escape)[slot] = nn;
  if (o.surface) reinterpret_cast<double2*>(o.surface)[slot] = nn;
  if (o.redshift_time) reinterpret_cast<double2*>(o.redshift_time)[slot] = nn;
  if (o.event) reinterpret_cast<double2*>(o.event)[slot] = nn;
  if (o.drift_a) reinterpret_cast<double2*>(o.drift_a)[slot] = make_double2(0.0, 0.0);
  if (o.drift_b) reinterpret_cast<double2*>(o.drift_b)[slot] = make_double2(0.0, 0.0);
  if (o.turning) reinterpret_cast<double2*>(o.turning)[slot] = nn;
  if (o.position_xy) reinterpret_cast<double2*>(o.position_xy)[slot] = nn;
  if (o.position_zr) reinterpret_cast<double2*>(o.position_zr)[slot] = nn;
}

// Register budget per precision: binary32 fits 128 registers (16 warps per SM); the binary64 and
// mixed kernels carry binary64 event and shell paths and run at 2 blocks of 128 threads per SM.
#ifndef GLC_MIN_BLOCKS_FP32
#define GLC_MIN_BLOCKS_FP32 4
#endif
#ifndef GLC_MIN_BLOCKS_MIXED
#define GLC_MIN_BLOCKS_MIXED 2
#endif
#ifndef GLC_MIN_BLOCKS_FP64
#define GLC_MIN_BLOCKS_FP64 2
#endif
template <int P>
struct LaunchShape {
  static constexpr int kMinBlocks =
      P == kFP32 ? GLC_MIN_BLOCKS_FP32 : (P == kMIXED ? GLC_MIN_BLOCKS_MIXED : GLC_MIN_BLOCKS_FP64);
};

template <int P>
__device__ __forceinline__ bool ray_step(Ray<P>& ray, const LaneScene& ls, const glc_policy& pol,
                                         RayResult<typename PrecTraits<P>::S>& res, bool use64) {
  return ray.step(ls, pol, res, P == kMIXED && use64);
}

// One ray from set-up to result (the body of the one-thread-per-ray kernels).
template <int P>
__device__ __forceinline__ void trace_one(const JobView& job, const glc_policy& pol, const glc_results& out,
                                          unsigned long long gi) {
  using S = typename PrecTraits<P>::S;
  if (gi >= job.total) return;
  double st8[8], dir;
  unsigned long long slot;
  int scene_idx;
  bool certified;
  if (!ray_setup(job, pol, gi, st8, dir, slot, scene_idx, certified)) return;
  if (certified) {
    write_certified(out, slot);
    return;
  }
  const LaneScene ls = make_lane_scene(job.scenes[scene_idx], pol.mixed_shell_factor);
  Ray<P> ray;
  ray.init(ls, pol, st8, dir);
  RayResult<S> res;
  for (;;) {
    bool use64 = false;
    if (P == kMIXED) use64 = __any_sync(__activemask(), double(ray.r) < ls.shell_r);
    if (ray_step<P>(ray, ls, pol, res, use64)) break;
  }
  write_result<P>(out, slot, ray, res, ls);
}

// One thread per ray; rays in tile order so a warp covers a compact pixel tile.
template <int P>
__global__ void __launch_bounds__(128, LaunchShape<P>::kMinBlocks) trace_simple_kernel(JobView job, glc_policy pol, glc_results out) {
  trace_one<P>(job, pol, out, (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// Work-queue kernel with warp-granular grabs: a grid of SMs x occupancy whose warps take
// `rays_per_grab` consecutive rays at a time from a global atomic counter and trace them 32 at a
// time with the one-thread-per-ray body. Load balances uneven jobs (many scenes, rays of very
// different cost) at warp granularity without interleaving ray set-up with stepping inside a warp.
template <int P>
__global__ void __launch_bounds__(128, LaunchShape<P>::kMinBlocks) trace_queue_kernel(JobView job, glc_policy pol,
                                                                                      glc_results out,
                                                                                      unsigned long long* queue) {
  const unsigned FULL = 0xffffffffu;
  const unsigned lane = threadIdx.x & 31u;
  const unsigned grab = pol.rays_per_grab < 32u ? 32u : (pol.rays_per_grab & ~31u);
  for (;;) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(queue, (unsigned long long)grab);
    base = __shfl_sync(FULL, base, 0);
    if (base >= job.total) break;
    for (unsigned k = 0; k < grab; k += 32u) trace_one<P>(job, pol, out, base + k + lane);
  }
}

// Persistent kernel: every warp loops until the job's queue is drained. Idle lanes are refilled
// from a warp-private range of `rays_per_grab` consecutive ray indices taken from a global atomic
// counter. A refill happens on every `refill_interval`-th step once at least `refill_min_idle`
// lanes are idle (or at once when the whole warp is idle), so ray set-up runs for several lanes
// together rather than diverging lane by lane. The counter is the only scratch memory; the loop
// has no waits on other warps or blocks.
template <int P>
__global__ void __launch_bounds__(128, LaunchShape<P>::kMinBlocks) trace_persistent_kernel(JobView job, glc_policy pol, glc_results out,
                                                               unsigned long long* queue) {
  using S = typename PrecTraits<P>::S;
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  Ray<P> ray;
  RayResult<S> res;
  LaneScene ls;
  unsigned long long slot = 0;
  bool active = false;
  unsigned long long grab_next = 0, grab_end = 0;
  bool drained = false;
  const unsigned grab = pol.rays_per_grab < 32 ? 32u : pol.rays_per_grab;
  const unsigned interval = pol.refill_interval == 0 ? 1u : pol.refill_interval;
  const unsigned min_idle = pol.refill_min_idle == 0 ? 1u : (pol.refill_min_idle > 32 ? 32u : pol.refill_min_idle);
  unsigned iter = 0;
  for (;;) {
    unsigned idle = __ballot_sync(FULL, !active);
    const bool any_active = idle != FULL;
    if (!drained && (!any_active || (iter % interval == 0u && unsigned(__popc(idle)) >= min_idle))) {
      while (idle != 0u) {
        if (grab_next >= grab_end) {
          unsigned long long base = 0;
          if (lane == 0) base = atomicAdd(queue, (unsigned long long)grab);
          base = __shfl_sync(FULL, base, 0);
          if (base >= job.total) {
            drained = true;
            break;
          }
          grab_next = base;
          grab_end = base + grab < job.total ? base + grab : job.total;
        }
        const unsigned avail = unsigned(grab_end - grab_next);
        const unsigned n_idle = __popc(idle);
        const unsigned take = avail < n_idle ? avail : n_idle;
        const unsigned rank = __popc(idle & lt_mask);
        const bool mine = ((idle >> lane) & 1u) && rank < take;
        if (mine) {
          double st8[8], dir;
          int scene_idx;
          bool certified;
          if (ray_setup(job, pol, grab_next + rank, st8, dir, slot, scene_idx, certified)) {
            if (certified) {
              write_certified(out, slot);
            } else {
              ls = make_lane_scene(job.scenes[scene_idx], pol.mixed_shell_factor);
              ray.init(ls, pol, st8, dir);
              active = true;
            }
          }
        }
        const unsigned took = __ballot_sync(FULL, mine);
        idle &= ~took;
        grab_next += take;
      }
    }
    if (!__any_sync(FULL, active)) {
      if (drained) break;
      continue;
    }
    bool use64 = false;
    if (P == kMIXED) use64 = __any_sync(FULL, active && double(ray.r) < ls.shell_r);
    if (active) {
      if (ray_step<P>(ray, ls, pol, res, use64)) {
        write_result<P>(out, slot, ray, res, ls);
        active = false;
      }
    }
    ++iter;
  }
}

}  // namespace glc
