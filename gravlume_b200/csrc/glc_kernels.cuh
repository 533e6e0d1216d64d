// Trace kernels: ray setup from a camera, result stores, the one-thread-per-ray kernel and the
// persistent work-queue kernel with warp-level refill of finished lanes.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "glc_tracer.cuh"

namespace glc {

// Pixel rectangle [x0, x1) x [y0, y1) an image camera traces: its tile region of 8x8-pixel tiles
// (TileRegion, crates/gravlume-render/src/trace.rs:799-857, TRACE_WORKGROUP_AXIS = 8), or the whole
// view when tile_count is {0, 0}. The host validates the region against the view's tile grid.
constexpr uint32_t kRegionTile = 8;
struct PixelRect {
  uint32_t x0, y0, x1, y1;
};
__host__ __device__ __forceinline__ PixelRect camera_rect(const glc_camera& c) {
  if (c.tile_count[0] == 0u && c.tile_count[1] == 0u) return {0u, 0u, c.width, c.height};
  const uint32_t x0 = c.tile_origin[0] * kRegionTile, y0 = c.tile_origin[1] * kRegionTile;
  const uint32_t x1 = (c.tile_origin[0] + c.tile_count[0]) * kRegionTile;
  const uint32_t y1 = (c.tile_origin[1] + c.tile_count[1]) * kRegionTile;
  return {x0, y0, x1 < c.width ? x1 : c.width, y1 < c.height ? y1 : c.height};
}

// Device view of one trace job: scenes, cameras and the prefix of their (padded) ray counts.
struct JobView {
  const glc_scene* scenes;
  const glc_camera* cams;
  const unsigned long long* begin;  // n_cams + 1 entries
  int n_cams;
  unsigned long long total;
  const unsigned long long* cert_begin;  // n_cams + 1 entries: first 16x16-tile word of each camera
  const uint32_t* cert;                  // per-tile capture certificates, or null when not evaluated
  const unsigned long long* emap_begin;  // n_cams + 1 entries: first escape-map node of each camera
  const uint32_t* emap;                  // packed escape-map nodes, or null when not traced
};

// ---- escape-direction map (crates/gravlume-render/src/shaders/geodesic_acceleration.wgsl:330-586)
// Nodes sit on every 4th pixel of each axis; 8x8 pixel tiles see a 3x3 stencil of nodes. A node is
// packed into 32 bits like the reference's map: tag << 30 (1 escape, 2 horizon, 0 anything else)
// and, for escapes, the octahedral projection of the unit escape direction in 15 + 15 bits.
constexpr uint32_t kMapNodeStep = 4, kMapTile = 8, kMapTagShift = 30, kMapTagEscape = 1, kMapTagHorizon = 2;
constexpr uint32_t kMapOctMax = 0x7fffu;
constexpr double kMapMaxStencilError = 3.0e-4;  // room inside the 3.82e-4 rad direction budget

__host__ __device__ __forceinline__ uint32_t map_grid_w(uint32_t w) { return 2u * ((w + kMapTile - 1) / kMapTile) + 1u; }
__host__ __device__ __forceinline__ uint32_t map_grid_h(uint32_t h) { return 2u * ((h + kMapTile - 1) / kMapTile) + 1u; }

__device__ __forceinline__ float oct_sign(float v) { return v >= 0.0f ? 1.0f : -1.0f; }

__device__ __forceinline__ uint32_t map_pack_escape(double dx, double dy, double dz) {
  const double l1 = fabs(dx) + fabs(dy) + fabs(dz);
  if (!(l1 > 0.0) || !isfinite(l1)) return 0u;
  float px = float(dx / l1), py = float(dy / l1);
  if (dz < 0.0) {
    const float qx = (1.0f - fabsf(py)) * oct_sign(px), qy = (1.0f - fabsf(px)) * oct_sign(py);
    px = qx;
    py = qy;
  }
  const float ex = fminf(fmaxf(0.5f * px + 0.5f, 0.0f), 1.0f), ey = fminf(fmaxf(0.5f * py + 0.5f, 0.0f), 1.0f);
  const uint32_t ux = uint32_t(rintf(ex * float(kMapOctMax))), uy = uint32_t(rintf(ey * float(kMapOctMax)));
  return ux | (uy << 15) | (kMapTagEscape << kMapTagShift);
}

// Unpacked node: tag and unit direction (escapes only).
__device__ __forceinline__ uint32_t map_unpack(uint32_t packed, float d[3]) {
  const uint32_t tag = packed >> kMapTagShift;
  d[0] = d[1] = d[2] = 0.0f;
  if (tag != kMapTagEscape) return tag;
  float px = 2.0f * float(packed & kMapOctMax) / float(kMapOctMax) - 1.0f;
  float py = 2.0f * float((packed >> 15) & kMapOctMax) / float(kMapOctMax) - 1.0f;
  const float z = 1.0f - fabsf(px) - fabsf(py);
  if (z < 0.0f) {
    const float qx = (1.0f - fabsf(py)) * oct_sign(px), qy = (1.0f - fabsf(px)) * oct_sign(py);
    px = qx;
    py = qy;
  }
  const float n = rsqrtf(px * px + py * py + z * z);
  d[0] = px * n;
  d[1] = py * n;
  d[2] = z * n;
  return tag;
}

__device__ __forceinline__ void map_bilerp(const float a[3], const float b[3], const float c[3], const float e[3],
                                           float u, float v, float out[3]) {
  float n2 = 0.0f;
  for (int i = 0; i < 3; ++i) {
    const float top = a[i] + (b[i] - a[i]) * u, bot = c[i] + (e[i] - c[i]) * u;
    out[i] = top + (bot - top) * v;
    n2 += out[i] * out[i];
  }
  const float n = rsqrtf(n2);
  for (int i = 0; i < 3; ++i) out[i] *= n;
}

// Escape direction of pixel (px, py) reconstructed from its tile's 3x3 stencil, when the tile is
// stable: all nine nodes escaped and the five inner nodes lie within min(half a pixel, 3e-4 rad)
// of the bilinear interpolation of the four corners (escape_map_tile_is_stable). Returns false
// otherwise.
__device__ inline bool map_reconstruct(const uint32_t* nodes, uint32_t gw, uint32_t px, uint32_t py,
                                       double half_pixel, double dir[3]) {
  const uint32_t tx = px / kMapTile, ty = py / kMapTile;
  float st[9][3];
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) {
      const uint32_t packed = nodes[(2u * ty + uint32_t(j)) * gw + 2u * tx + uint32_t(i)];
      if (map_unpack(packed, st[3 * j + i]) != kMapTagEscape) return false;
    }
  const float tol = float(fmin(half_pixel, kMapMaxStencilError));
  const float tol2 = tol * tol;
  // inner nodes (1, 3, 4, 5, 7) at tile coordinates (1/2, 0), (0, 1/2), (1/2, 1/2), (1, 1/2), (1/2, 1)
  const int inner[5] = {1, 3, 4, 5, 7};
  const float iu[5] = {0.5f, 0.0f, 0.5f, 1.0f, 0.5f}, iv[5] = {0.0f, 0.5f, 0.5f, 0.5f, 1.0f};
  for (int k = 0; k < 5; ++k) {
    float pr[3];
    map_bilerp(st[0], st[2], st[6], st[8], iu[k], iv[k], pr);
    const float dx = pr[0] - st[inner[k]][0], dy = pr[1] - st[inner[k]][1], dz = pr[2] - st[inner[k]][2];
    const float e2 = dx * dx + dy * dy + dz * dz;
    if (!(e2 <= tol2)) return false;
  }
  // the pixel's 2x2 sub-cell of the stencil
  const uint32_t lx = px - tx * kMapTile, ly = py - ty * kMapTile;
  const uint32_t cx = min(lx / kMapNodeStep, 1u), cy = min(ly / kMapNodeStep, 1u);
  const float u = float(lx - cx * kMapNodeStep) / float(kMapNodeStep);
  const float v = float(ly - cy * kMapNodeStep) / float(kMapNodeStep);
  const int f = int(cy * 3u + cx);
  float d[3];
  map_bilerp(st[f], st[f + 1], st[f + 3], st[f + 4], u, v, d);
  for (int i = 0; i < 3; ++i) dir[i] = double(d[i]);
  return true;
}

// Ways a ray of an image camera can be settled without its own integration.
enum RayShortcut : int { kShortNone = 0, kShortCertified = 1, kShortMapNode = 2, kShortReconstructed = 3 };

// Initial state of ray gi of the job. Image rays are generated in binary64 from the camera basis
// (scene.rs:211-270, view.rs:408-424): sight = (s_x right + s_y up - arrival) / |.|,
// p^mu = omega (u^mu - sight^mu), p_mu = g_{mu nu} p^nu at the observer. Returns false for tile
// padding outside the image.
__device__ __forceinline__ void image_state(const glc_scene* sc, const glc_camera* cam, uint32_t px, uint32_t py,
                                            double st8[8]);

__device__ __forceinline__ bool ray_setup(const JobView& job, const glc_policy& pol, unsigned long long gi,
                                          double st8[8], double& dir, unsigned long long& slot, int& scene_idx,
                                          int& shortcut, double rdir[3]) {
  shortcut = kShortNone;
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
  const PixelRect rc = camera_rect(*cam);
  const uint32_t tw = pol.tile_w, th = pol.tile_h;
  const uint32_t tiles_x = (rc.x1 - rc.x0 + tw - 1) / tw;
  const unsigned long long per_tile = (unsigned long long)tw * th;
  const unsigned long long tile = j / per_tile;
  const uint32_t within = uint32_t(j - tile * per_tile);
  const uint32_t px = rc.x0 + uint32_t(tile % tiles_x) * tw + within % tw;
  const uint32_t py = rc.y0 + uint32_t(tile / tiles_x) * th + within / tw;
  if (px >= rc.x1 || py >= rc.y1) return false;
  slot = cam->result_offset + (unsigned long long)py * W + px;
  dir = -1.0;
  if (job.cert) {
    const unsigned long long t = job.cert_begin[lo] + (unsigned long long)(py >> 4) * ((W + 15u) >> 4) + (px >> 4);
    if (job.cert[t]) {
      shortcut = kShortCertified;
      return true;
    }
  }
  const glc_scene* sc = job.scenes + scene_idx;
  if (job.emap) {
    // node pixels were traced by the node pass; stable tiles take the interpolated direction
    if (px % kMapNodeStep == 0u && py % kMapNodeStep == 0u) {
      shortcut = kShortMapNode;
      return true;
    }
    if (!sc->has_surface) {
      const double half_pixel = cam->kind == GLC_CAMERA_PINHOLE ? sc->tangent_half_fov / double(H)
                                                                : 0.5 * 3.141592653589793 / double(H);
      if (map_reconstruct(job.emap + job.emap_begin[lo], map_grid_w(W), px, py, half_pixel, rdir)) {
        shortcut = kShortReconstructed;
        return true;
      }
    }
  }
  image_state(sc, cam, px, py, st8);
  return true;
}

// Initial state of pixel (px, py) of an image camera (pinhole sight plane or equirectangular map).
__device__ __forceinline__ void image_state(const glc_scene* sc, const glc_camera* cam, uint32_t px, uint32_t py,
                                            double st8[8]) {
  const uint32_t W = cam->width, H = cam->height;
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
}

// Binary16 bits of a non-negative intensity, saturating at the largest finite binary16.
__device__ __forceinline__ unsigned short half_bits(double v) {
  const float f = v > 65504.0 ? 65504.0f : (v > 0.0 ? float(v) : 0.0f);
  return __half_as_ushort(__float2half_rn(f));
}

// intensity and radiance stores of one ray (surface transport; zero radiance elsewhere)
__device__ __forceinline__ void write_radiance(const glc_results& o, unsigned long long slot, double emitted,
                                               double observed, const double rgb[3]) {
  const bool hit = isfinite(observed);
  if (o.intensity)
    reinterpret_cast<double2*>(o.intensity)[slot] =
        hit ? make_double2(observed, emitted) : make_double2(__longlong_as_double(0x7ff8000000000000ll),
                                                             __longlong_as_double(0x7ff8000000000000ll));
  if (o.radiance) {
    ushort4 v = make_ushort4(0, 0, 0, 0);
    if (hit) v = make_ushort4(half_bits(rgb[0]), half_bits(rgb[1]), half_bits(rgb[2]), half_bits(2.0));
    reinterpret_cast<ushort4*>(o.radiance)[slot] = v;
  }
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
  // post-hit transport (surface.rs:12-72) after the stepping loop: a function of the hit radius and
  // g alone, evaluated where the loop's state is no longer live
  const double nan = __longlong_as_double(0x7ff8000000000000ll);
  double emitted = nan, observed = nan, rgb[3] = {0.0, 0.0, 0.0};
  if ((o.intensity || o.radiance) && res.termination == GLC_TERM_SURFACE && isfinite(double(res.g))) {
    const glc_scene& sp = *ls.src;
    if (!surface_radiance(sp.emission_model, sp.intensity_at_six, sp.temperature_at_six, sp.slab_transmittance,
                          sp.slab_emission, sp.slab_bands, double(res.surface_r), double(res.g), emitted, observed,
                          rgb))
      emitted = observed = nan;
  }
  write_radiance(o, slot, emitted, observed, rgb);
}

// A ray of a certified tile: horizon capture proven without integration (kFlagCertified); the
// integration observables are NaN and the counters zero.
__device__ __forceinline__ void write_certified(const glc_results& o, unsigned long long slot) {
  const double nan = __longlong_as_double(0x7ff8000000000000ll);
  // like the reference's certified sample (geodesic_acceleration.wgsl:299-311): horizon, with the
  // horizon event as its candidate
  const uint32_t code = uint32_t(GLC_TERM_HORIZON) | ((1u << kEvHorizon) << 12) | (1u << 16) |
                        (uint32_t(kFlagCertified) << 20);
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
  const double none[3] = {0.0, 0.0, 0.0};
  write_radiance(o, slot, nan, nan, none);
}

// A ray of a stable escape-map tile: an escape whose direction is interpolated from the tile's
// nodes (kFlagReconstructed); the other observables are NaN and the counters zero.
__device__ __forceinline__ void write_reconstructed(const glc_results& o, unsigned long long slot, const double d[3]) {
  const double nan = __longlong_as_double(0x7ff8000000000000ll);
  // like the reference's reconstructed sample (geodesic_acceleration.wgsl:549-560): escape, with the
  // escape event as its candidate
  const uint32_t code = uint32_t(GLC_TERM_ESCAPE) | ((1u << kEvEscape) << 12) | (1u << 16) |
                        (uint32_t(kFlagReconstructed) << 20);
  if (o.code) reinterpret_cast<uint4*>(o.code)[slot] = make_uint4(code, 0u, 0u, 0u);
  if (o.branch) reinterpret_cast<int4*>(o.branch)[slot] = make_int4(0, 0, 0, 0);
  const double2 nn = make_double2(nan, nan);
  const double cz = fmin(fmax(d[2], -1.0), 1.0);
  if (o.escape) reinterpret_cast<double2*>(o.escape)[slot] = make_double2(acos(cz), atan2(d[1], d[0]));
  if (o.surface) reinterpret_cast<double2*>(o.surface)[slot] = nn;
  if (o.redshift_time) reinterpret_cast<double2*>(o.redshift_time)[slot] = nn;
  if (o.event) reinterpret_cast<double2*>(o.event)[slot] = nn;
  if (o.drift_a) reinterpret_cast<double2*>(o.drift_a)[slot] = make_double2(0.0, 0.0);
  if (o.drift_b) reinterpret_cast<double2*>(o.drift_b)[slot] = make_double2(0.0, 0.0);
  if (o.turning) reinterpret_cast<double2*>(o.turning)[slot] = nn;
  if (o.position_xy) reinterpret_cast<double2*>(o.position_xy)[slot] = nn;
  if (o.position_zr) reinterpret_cast<double2*>(o.position_zr)[slot] = nn;
  const double none[3] = {0.0, 0.0, 0.0};
  write_radiance(o, slot, nan, nan, none);
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
#ifndef GLC_MIN_BLOCKS_BULK
#define GLC_MIN_BLOCKS_BULK 4
#endif
#ifndef GLC_MIN_BLOCKS_TAIL
#define GLC_MIN_BLOCKS_TAIL 2
#endif
template <int P>
struct LaunchShape {
  static constexpr int kMinBlocks =
      P == kFP32 ? GLC_MIN_BLOCKS_FP32
                 : (P == kBULK ? GLC_MIN_BLOCKS_BULK
                               : (P == kMIXED ? GLC_MIN_BLOCKS_MIXED
                                              : (P == kTAIL ? GLC_MIN_BLOCKS_TAIL : GLC_MIN_BLOCKS_FP64)));
};

template <int P>
__device__ __forceinline__ bool ray_step(Ray<P>& ray, const LaneScene& ls, const glc_policy& pol,
                                         RayResult<typename PrecTraits<P>::S>& res, bool use64) {
  // rolled stage loop: the work-queue kernels and the one-kernel modes
  return ray.template step<1>(ls, pol, res, P == kMIXED && use64);
}

// One ray from set-up to result (the body of the one-thread-per-ray kernels).
template <int P>
__device__ __forceinline__ void trace_one(const JobView& job, const glc_policy& pol, const glc_results& out,
                                          unsigned long long gi) {
  using S = typename PrecTraits<P>::S;
  if (gi >= job.total) return;
  double st8[8], dir;
  unsigned long long slot;
  int scene_idx, shortcut;
  double rdir[3];
  if (!ray_setup(job, pol, gi, st8, dir, slot, scene_idx, shortcut, rdir)) return;
  if (shortcut != kShortNone) {
    if (shortcut == kShortCertified) write_certified(out, slot);
    else if (shortcut == kShortReconstructed) write_reconstructed(out, slot, rdir);
    return;
  }
  // the drift maxima are evaluated only when a drift array is wanted
  const LaneScene ls = make_lane_scene(job.scenes[scene_idx], pol.mixed_shell_factor, out.drift_a || out.drift_b || pol.uncertain_terminals);
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
__global__ void __launch_bounds__(128, LaunchShape<P>::kMinBlocks) trace_simple_kernel(JobView job, glc_policy pol, glc_results out,
                                                                                       unsigned long long base) {
  trace_one<P>(job, pol, out, base + (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// ---- MIXED as two kernels: the hand-off records (HandoffRec, glc_tracer.cuh) of a job's rays are
// stored word-major, word w of ray gi at rec[w * n + gi], so that a warp's stores and loads of one
// word are contiguous 16-byte accesses.
struct Handoff {
  uint4* rec;
  unsigned long long n;  // rays of the job (the stride between words)
};
constexpr int kHandoffWords = int(sizeof(HandoffRec) / sizeof(uint4));

__device__ __forceinline__ void handoff_store(const Handoff& hv, unsigned long long gi, const Ray<kBULK>& ray,
                                              const RayResult<float>& res) {
  HandoffRec rec;
  handoff_pack(ray, res, rec);
  const uint4* w = reinterpret_cast<const uint4*>(&rec);
#pragma unroll
  for (int k = 0; k < kHandoffWords; ++k) hv.rec[k * hv.n + gi] = w[k];
}

__device__ __forceinline__ uint32_t handoff_resume(const Handoff& hv, unsigned long long gi, Ray<kTAIL>& ray,
                                                   const LaneScene& sc, const double st8[8], double direction,
                                                   uint32_t& failure) {
  HandoffRec rec;
  uint4* w = reinterpret_cast<uint4*>(&rec);
#pragma unroll
  for (int k = 0; k < kHandoffWords; ++k) w[k] = hv.rec[k * hv.n + gi];
  return handoff_unpack(rec, ray, sc, st8, direction, failure);
}

// MIXED, first kernel: binary32 stepping with the compensated pair state at the binary32 register
// budget. Non-terminal turning points and equatorial crossings are handled here; a ray leaves at the
// start of its first step that brackets a terminal event (or a surface crossing near the surface),
// or when it enters the binary64 shell, or when it fails, by storing its hand-off record.
// Certified and map-reconstructed pixels are written here. bulk_one is one ray of it, shared by
// the one-thread-per-ray kernel and the work-queue kernels.
template <int kUnroll = 6>
__device__ __forceinline__ void bulk_one(const JobView& job, const glc_policy& pol, const glc_results& out,
                                         const Handoff& hv, unsigned long long gi) {
  if (gi >= job.total) return;
  double st8[8], dir;
  unsigned long long slot;
  int scene_idx, shortcut;
  double rdir[3];
  if (!ray_setup(job, pol, gi, st8, dir, slot, scene_idx, shortcut, rdir)) return;
  if (shortcut != kShortNone) {
    if (shortcut == kShortCertified) write_certified(out, slot);
    else if (shortcut == kShortReconstructed) write_reconstructed(out, slot, rdir);
    return;
  }
  const LaneScene ls = make_lane_scene(job.scenes[scene_idx], pol.mixed_shell_factor, out.drift_a || out.drift_b || pol.uncertain_terminals);
  Ray<kBULK> ray;
  ray.init(ls, pol, st8, dir);
  RayResult<float> res;
  while (!ray.template step<kUnroll>(ls, pol, res, false)) {
  }
  handoff_store(hv, gi, ray, res);
}

template <int P = kBULK>
__global__ void __launch_bounds__(128, LaunchShape<P>::kMinBlocks)
    trace_bulk_kernel(JobView job, glc_policy pol, glc_results out, Handoff hv, unsigned long long base) {
  static_assert(P == kBULK, "the bulk kernel steps the BULK precision");
  bulk_one(job, pol, out, hv, base + (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// MIXED, second kernel: one thread per ray of the same job; resumes each handed-off ray in binary64
// (re-taking the step it left at, with binary64 error control, root-finding and observables, the
// shell steps, and the renormalization of the final momentum) and writes its result.
template <int P = kTAIL>
__global__ void __launch_bounds__(128, LaunchShape<P>::kMinBlocks)
    trace_tail_kernel(JobView job, glc_policy pol, glc_results out, Handoff hv, unsigned long long base) {
  static_assert(P == kTAIL, "the completion kernel steps the TAIL precision");
  const unsigned long long gi = base + (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gi >= job.total) return;
  double st8[8], dir;
  unsigned long long slot;
  int scene_idx, shortcut;
  double rdir[3];
  if (!ray_setup(job, pol, gi, st8, dir, slot, scene_idx, shortcut, rdir)) return;
  if (shortcut != kShortNone) return;
  const LaneScene ls = make_lane_scene(job.scenes[scene_idx], pol.mixed_shell_factor, out.drift_a || out.drift_b || pol.uncertain_terminals);
  Ray<kTAIL> ray;
  uint32_t failure = GLC_FAIL_NONE;
  const uint32_t term = handoff_resume(hv, gi, ray, ls, st8, dir, failure);
  RayResult<double> res;
  if (term != GLC_TERM_NONE) {
    ray.finish_plain(res, term, failure);
  } else {
    // the stages of each attempt, kept (in local memory) for the terminal step's dense output
    double stages[7][7];
    while (!ray.step(ls, pol, res, false, stages)) {
    }
  }
  write_result<kTAIL>(out, slot, ray, res, ls);
}

// Work-queue kernel with warp-granular grabs: a grid of SMs x occupancy whose warps take
// `rays_per_grab` consecutive rays at a time from a global atomic counter and trace them 32 at a
// time with the one-thread-per-ray body. Load balances uneven jobs (many scenes, rays of very
// different cost) at warp granularity without interleaving ray set-up with stepping inside a warp.
template <int P>
__global__ void __launch_bounds__(128, LaunchShape<P>::kMinBlocks) trace_queue_kernel(JobView job, glc_policy pol,
                                                                                      glc_results out,
                                                                                      unsigned long long* queue,
                                                                                      Handoff hv) {
  const unsigned FULL = 0xffffffffu;
  const unsigned lane = threadIdx.x & 31u;
  const unsigned grab = pol.rays_per_grab < 32u ? 32u : (pol.rays_per_grab & ~31u);
  for (;;) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(queue, (unsigned long long)grab);
    base = __shfl_sync(FULL, base, 0);
    if (base >= job.total) break;
    for (unsigned k = 0; k < grab; k += 32u) {
      if constexpr (P == kBULK) bulk_one<1>(job, pol, out, hv, base + k + lane);
      else trace_one<P>(job, pol, out, base + k + lane);
    }
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
                                                               unsigned long long* queue, Handoff hv) {
  using S = typename PrecTraits<P>::S;
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  Ray<P> ray;
  RayResult<S> res;
  LaneScene ls;
  unsigned long long slot = 0, ray_index = 0;
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
          double st8[8], dir, rdir[3];
          int scene_idx, shortcut;
          if (ray_setup(job, pol, grab_next + rank, st8, dir, slot, scene_idx, shortcut, rdir)) {
            if (shortcut != kShortNone) {
              if (shortcut == kShortCertified) write_certified(out, slot);
              else if (shortcut == kShortReconstructed) write_reconstructed(out, slot, rdir);
            } else {
              ls = make_lane_scene(job.scenes[scene_idx], pol.mixed_shell_factor, out.drift_a || out.drift_b || pol.uncertain_terminals);
              ray.init(ls, pol, st8, dir);
              ray_index = grab_next + rank;
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
        if constexpr (P == kBULK) handoff_store(hv, ray_index, ray, res);
        else write_result<P>(out, slot, ray, res, ls);
        active = false;
      }
    }
    ++iter;
  }
}

}  // namespace glc
