// Node pass of the escape-direction map: the rays of every 4th pixel of each axis of each image
// camera, traced in full (their results are stored like any other pixel's) and packed into the map
// the main pass reconstructs stable 8x8 tiles from (crates/gravlume-render/src/shaders/
// geodesic_acceleration.wgsl:497-520, trace_escape_map_nodes).
#pragma once

#include "glc_kernels.cuh"

namespace glc {

template <int P>
__global__ void __launch_bounds__(128, LaunchShape<P>::kMinBlocks) escape_map_nodes_kernel(JobView job, glc_policy pol,
                                                                                           glc_results out,
                                                                                           uint32_t* nodes) {
  using S = typename PrecTraits<P>::S;
  const unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= job.emap_begin[job.n_cams]) return;
  int lo = 0, hi = job.n_cams - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (job.emap_begin[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  const glc_camera& cam = job.cams[lo];
  const uint32_t W = cam.width, H = cam.height, gw = map_grid_w(W);
  const unsigned long long j = t - job.emap_begin[lo];
  const uint32_t px = uint32_t(j % gw) * kMapNodeStep, py = uint32_t(j / gw) * kMapNodeStep;
  // a tile region needs the nodes of its 8x8 tiles' stencils, which reach one node row and column
  // past its last tile; node pixels outside the region are traced for the map but not stored
  const PixelRect rc = camera_rect(cam);
  const bool whole = cam.tile_count[0] == 0u && cam.tile_count[1] == 0u;
  const uint32_t xe = (whole ? (W + kRegionTile - 1) / kRegionTile : cam.tile_origin[0] + cam.tile_count[0]) * kRegionTile;
  const uint32_t ye = (whole ? (H + kRegionTile - 1) / kRegionTile : cam.tile_origin[1] + cam.tile_count[1]) * kRegionTile;
  if (px < rc.x0 || py < rc.y0 || px > xe || py > ye) return;
  const bool store = px < rc.x1 && py < rc.y1;
  glc_results none{};
  const glc_results& dst = store ? out : none;
  uint32_t packed = 0u;
  if (px < W && py < H) {
    const unsigned long long slot = cam.result_offset + (unsigned long long)py * W + px;
    if (job.cert && job.cert[job.cert_begin[lo] + (unsigned long long)(py >> 4) * ((W + 15u) >> 4) + (px >> 4)]) {
      write_certified(dst, slot);
      packed = kMapTagHorizon << kMapTagShift;
    } else {
      const glc_scene& sc = job.scenes[cam.scene_index];
      double st8[8];
      image_state(&sc, &cam, px, py, st8);
      const LaneScene ls = make_lane_scene(sc, pol.mixed_shell_factor, out.drift_a || out.drift_b || pol.uncertain_terminals);
      Ray<P> ray;
      ray.init(ls, pol, st8, -1.0);
      RayResult<S> res;
      for (;;) {
        bool use64 = false;
        // per ray (not per warp): a node's result must not depend on which other nodes share its
        // warp, so that a frame traced in tile batches equals the frame traced at once
        if (P == kMIXED) use64 = double(ray.r) < ls.shell_r;
        if (ray_step<P>(ray, ls, pol, res, use64)) break;
      }
      write_result<P>(dst, slot, ray, res, ls);
      if (res.termination == GLC_TERM_ESCAPE) {
        const double th = double(res.escape_theta), ph = double(res.escape_phi);
        if (isfinite(th) && isfinite(ph)) {
          double s, c, sp, cp;
          sincos(th, &s, &c);
          sincos(ph, &sp, &cp);
          packed = map_pack_escape(s * cp, s * sp, c);
        }
      } else if (res.termination == GLC_TERM_HORIZON) {
        packed = kMapTagHorizon << kMapTagShift;
      }
    }
  }
  nodes[t] = packed;
}

}  // namespace glc
