// Surface footprint (crates/gravlume-reference/src/footprint.rs): the local source Jacobian of an
// image pixel that ends on the surface, rows (source radius, local azimuthal arc r_c dphi), columns
// (screen x, screen y), in M per image pixel, with its singular values and parity (203-235).
//
// Two kernels follow a classification pass that lists the pixels whose primary trace is an
// unambiguous observed surface hit (footprint.rs:237-253); the others get NO_SURFACE without work.
//  - footprint_quarter_kernel is the reference's estimate (74-150): four lanes per listed pixel
//    trace the neighbours a quarter pixel left, right, up and down; a neighbour that is not an
//    unambiguous surface hit with the center's branch key makes the pixel a DISCONTINUITY, and the
//    Jacobian is the central difference over the half-pixel span, gathered by warp shuffles.
//  - footprint_tangent_kernel is the exact derivative of the computed trace: two tangent channels
//    (d/dx, d/dy of the image point) are seeded through the ray set-up, carried across every
//    accepted DP5(4) step by re-evaluating its stages in dual arithmetic at the step's frozen size,
//    and through the terminal step's dense output with the implicit derivative of the event time
//    (z = 0 at the hit). One re-trace per listed pixel.
#pragma once

#include <type_traits>

#include "glc_adjoint.cuh"
#include "glc_kernels.cuh"

namespace glc {

using D2 = Dual<2>;

// footprint.rs:203-235 on J (row-major), with every product and sum rounded as written (no FMA
// contraction beyond the reference's two mul_adds) so that equal Jacobians give equal metrics.
__device__ __forceinline__ void footprint_finish(const double J[4], glc_footprint& f) {
  const double nan = __longlong_as_double(0x7ff8000000000000ll);
  bool finite = true;
  for (int i = 0; i < 4; ++i) finite = finite && isfinite(J[i]);
  double major = nan, minor = nan, det = nan, n2 = nan;
  if (finite) {
    det = __fma_rn(J[0], J[3], __dmul_rn(-J[1], J[2]));
    n2 = 0.0;
    for (int i = 0; i < 4; ++i) n2 = __dadd_rn(n2, __dmul_rn(J[i], J[i]));
    const double disc = sqrt(fmax(__fma_rn(n2, n2, __dmul_rn(__dmul_rn(-4.0, det), det)), 0.0));
    major = sqrt(__dmul_rn(0.5, __dadd_rn(n2, disc)));
    minor = major == 0.0 ? 0.0 : fabs(det) / major;
    finite = isfinite(major) && isfinite(minor);
  }
  if (!finite) {
    for (int i = 0; i < 4; ++i) f.jacobian[i] = nan;
    f.singular_values[0] = f.singular_values[1] = f.determinant = nan;
    f.status = GLC_FOOTPRINT_NON_FINITE;
    f.parity = 0;
    return;
  }
  for (int i = 0; i < 4; ++i) f.jacobian[i] = J[i];
  f.singular_values[0] = major;
  f.singular_values[1] = minor;
  f.determinant = det;
  const double floor_ = __dmul_rn(64.0 * 2.220446049250313e-16, n2);
  f.status = GLC_FOOTPRINT_RESOLVED;
  f.parity = det > floor_ ? 1 : (det < -floor_ ? -1 : 0);
}

__device__ __forceinline__ void footprint_store(glc_footprint* out, const glc_footprint& f) {
  const double4* s = reinterpret_cast<const double4*>(&f);
  double4* w = reinterpret_cast<double4*>(out);
  w[0] = s[0];
  w[1] = s[1];
}

__device__ __forceinline__ void footprint_unresolved(glc_footprint* out, int status) {
  const double nan = __longlong_as_double(0x7ff8000000000000ll);
  glc_footprint f;
  for (int i = 0; i < 4; ++i) f.jacobian[i] = nan;
  f.singular_values[0] = f.singular_values[1] = f.determinant = nan;
  f.status = status;
  f.parity = 0;
  footprint_store(out, f);
}

// footprint.rs:237-253 on a code word: an observed surface hit (no undefined-emitter flag) with one
// event candidate.
__device__ __forceinline__ bool resolved_surface_code(uint32_t code) {
  const uint32_t term = code & 0xFFu, cand = (code >> 12) & 0xFu, flags = (code >> 20) & 0xFFFu;
  return term == GLC_TERM_SURFACE && (flags & kFlagSurfaceInvalid) == 0u && __popc(cand) <= 1;
}

// footprint.rs:318-320 (surface.rs): (left - right + pi) rem_euclid tau - pi.
__device__ __forceinline__ double wrapped_difference(double left, double right) {
  const double pi = 3.14159265358979323846, tau = 6.28318530717958647692;
  double r = fmod(__dadd_rn(__dsub_rn(left, right), pi), tau);
  if (r < 0.0) r = __dadd_rn(r, tau);
  return __dsub_rn(r, pi);
}

// List the pixels of image camera c whose primary trace is a resolved surface hit; every other
// pixel's footprint is written NO_SURFACE here.
__global__ void footprint_classify_kernel(JobView job, int c, const uint4* code, glc_footprint* out,
                                          unsigned long long* list, unsigned int* count, unsigned int capacity) {
  const glc_camera& cam = job.cams[c];
  const unsigned long long p = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= (unsigned long long)cam.width * cam.height) return;
  const unsigned long long slot = cam.result_offset + p;
  if (!resolved_surface_code(code[slot].x)) {
    footprint_unresolved(out + slot, GLC_FOOTPRINT_NO_SURFACE);
    return;
  }
  const unsigned int k = atomicAdd(count, 1u);
  if (k < capacity) list[k] = ((unsigned long long)c << 32) | p;
}

// Four lanes per listed pixel: lane k traces neighbour k (left, right, up, down, footprint.rs:
// 154-195) and the group's first lane combines them. The stride loop runs on the warp-uniform base
// index so that all 32 lanes reach the shuffles.
template <int P>
__global__ void __launch_bounds__(128, LaunchShape<P>::kMinBlocks) footprint_quarter_kernel(
    JobView job, glc_policy pol, const unsigned long long* list, const unsigned int* count, unsigned int capacity,
    const uint4* code, const int4* branch, const double2* surface, glc_footprint* out) {
  using S = typename PrecTraits<P>::S;
  const unsigned FULL = 0xffffffffu;
  const unsigned int n = min(*count, capacity);
  const unsigned lane = threadIdx.x & 31u;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < 4ull * n;
       base += stride) {
    const unsigned long long t = base + lane;
    const int k = int(t & 3u);
    unsigned ok = 0u;
    double r = 0.0, phi = 0.0;
    unsigned long long slot = 0;
    if (t < 4ull * n) {
      const unsigned long long entry = list[t >> 2];
      glc_camera cam = job.cams[entry >> 32];
      const unsigned long long p = entry & 0xffffffffull;
      slot = cam.result_offset + p;
      const uint32_t px = uint32_t(p % cam.width), py = uint32_t(p / cam.width);
      if (k < 2) cam.subpixel_x += k == 0 ? -0.25 : 0.25;
      else cam.subpixel_y += k == 2 ? -0.25 : 0.25;
      const glc_scene& sc = job.scenes[cam.scene_index];
      double st8[8];
      image_state(&sc, &cam, px, py, st8);
      const LaneScene ls = make_lane_scene(sc, pol.mixed_shell_factor, pol.uncertain_terminals != 0u);  // drifts only for the Uncertain gate
      Ray<P> ray;
      ray.init(ls, pol, st8, -1.0);
      RayResult<S> res;
      for (;;) {
        bool use64 = false;
        if (P == kMIXED) use64 = __any_sync(__activemask(), double(ray.r) < ls.shell_r);
        if (ray_step<P>(ray, ls, pol, res, use64)) break;
      }
      // the neighbour's code word and branch key, as write_result packs them
      const uint32_t w = (res.termination & 0xFFu) | ((res.candidates & 0xFu) << 12) |
                         (uint32_t(ray.polar + 1) << 16) | ((res.flags & 0xFFFu) << 20);
      const uint32_t cw = code[slot].x;
      const int4 cb = branch[slot];
      ok = resolved_surface_code(w) && ((w >> 16) & 0xFu) == ((cw >> 16) & 0xFu) && int(ray.turnings) == cb.x &&
                   int(ray.crossings) == cb.y && ray.winding == cb.z
               ? 1u
               : 0u;
      r = double(res.surface_r);
      phi = double(res.surface_phi);
    }
    __syncwarp(FULL);
    const unsigned g0 = lane & ~3u;
    double rn[4], pn[4];
    unsigned all = 1u;
    for (int q = 0; q < 4; ++q) {
      rn[q] = __shfl_sync(FULL, r, g0 + q);
      pn[q] = __shfl_sync(FULL, phi, g0 + q);
      all &= __shfl_sync(FULL, ok, g0 + q);
    }
    if (t < 4ull * n && k == 0) {
      if (!all) {
        footprint_unresolved(out + slot, GLC_FOOTPRINT_DISCONTINUITY);
      } else {
        // footprint.rs:111-134
        const double2 c = surface[slot];
        const double a[4] = {__dmul_rn(c.x, wrapped_difference(pn[0], c.y)), __dmul_rn(c.x, wrapped_difference(pn[1], c.y)),
                             __dmul_rn(c.x, wrapped_difference(pn[2], c.y)), __dmul_rn(c.x, wrapped_difference(pn[3], c.y))};
        const double J[4] = {__dsub_rn(rn[1], rn[0]) / 0.5, __dsub_rn(rn[3], rn[2]) / 0.5, __dsub_rn(a[1], a[0]) / 0.5,
                             __dsub_rn(a[3], a[2]) / 0.5};
        glc_footprint f;
        footprint_finish(J, f);
        footprint_store(out + slot, f);
      }
    }
  }
}

// Slopes K_i, i < kStages, of the step from y0 with size h (frozen), in the dual arithmetic D.
template <int kStages, class D>
__device__ __forceinline__ void dual_stages(const KN<double>& k, const D y0[6], const D& E, double h, D K[kStages][6]) {
  const KN<D> kt{D(k.a), D(k.a2), D(k.s), D(k.sa), D(k.q2)};
  for (int i = 0; i < kStages; ++i) {
    D Y[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      D s(0.0);
      for (int j = 0; j < i; ++j) s += dp_coef(i, j) * K[j][c];
      Y[c] = y0[c] + h * s;
    }
    D d[7], r, vr;
    kn_rhs(kt, Y, E, d, r, vr);
#pragma unroll
    for (int c = 0; c < 6; ++c) K[i][c] = d[c];
  }
}

// Tangent of an accepted step: y <- y + h sum_i b_i K_i with the stages in dual arithmetic (the
// seventh stage, the slope at the end point, has weight 0).
template <class D>
__device__ __noinline__ void step_tangent(const KN<double>& k, D y[6], const D& E, double h) {
  D K[6][6];
  dual_stages<6>(k, y, E, h, K);
  double w[7];
  step_weights(w);
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    D s(0.0);
#pragma unroll
    for (int i = 0; i < 6; ++i) s += w[i] * K[i][c];
    y[c] = y[c] + h * s;
  }
}

// Tangent of the state at the terminal surface event, dense-output fraction theta: y(theta) with the
// event time moving so that z stays 0 (d theta = -dz / zdot).
template <class D>
__device__ __noinline__ void hit_tangent(const KN<double>& k, D y[6], const D& E, double h, double theta) {
  D K[7][6];
  dual_stages<7>(k, y, E, h, K);
  double w[7], dw[7];
  dense_weights_at(theta, w, dw);
  D ys[6];
  double ydot[6];
  for (int c = 0; c < 6; ++c) {
    D s(0.0);
    double sd = 0.0;
    for (int i = 0; i < 7; ++i) {
      s += w[i] * K[i][c];
      sd += dw[i] * double(K[i][c].v);
    }
    ys[c] = y[c] + h * s;
    ydot[c] = h * sd;
  }
  for (int ch = 0; ch < 2; ++ch) {
    const double dtheta = -double(ys[2].d[ch]) / ydot[2];
    for (int c = 0; c < 6; ++c) ys[c].d[ch] += decltype(ys[c].v)(ydot[c] * dtheta);
  }
  for (int c = 0; c < 6; ++c) y[c] = ys[c];
}

// A binary64 dual rounded to the dual type D.
template <class D>
__device__ __forceinline__ D dual_cast(const D2& x) {
  D r(x.v);
  r.d[0] = decltype(r.v)(x.d[0]);
  r.d[1] = decltype(r.v)(x.d[1]);
  return r;
}

// The set-up of image_state on the dual image point (u, v) = pixel + subpixel, seeded d/du, d/dv:
// the spatial state and E = -p_t with their tangents.
__device__ __noinline__ void image_state_tangent(const glc_scene& sc, const glc_camera& cam, double u, double v,
                                                 D2 y[6], D2& E) {
  const double W = double(cam.width), H = double(cam.height);
  const D2 ud = D2::seed(u, 0), vd = D2::seed(v, 1);
  D2 sight[4];
  if (cam.kind == GLC_CAMERA_PINHOLE) {
    const D2 nx = 2.0 * ud / W - 1.0, ny = 1.0 - 2.0 * vd / H;
    const D2 sx = (W / H) * sc.tangent_half_fov * nx, sy = sc.tangent_half_fov * ny;
    const D2 nrm = 1.0 / g_sqrt(1.0 + sx * sx + sy * sy);
    for (int i = 0; i < 4; ++i) sight[i] = (sc.image_right[i] * sx + sc.image_up[i] * sy - sc.arrival[i]) * nrm;
  } else {
    const double lon = 2.0 * M_PI * (u / W) - M_PI, lat = 0.5 * M_PI - M_PI * (v / H);
    double sl, cl, sb, cb;
    sincos(lon, &sl, &cl);
    sincos(lat, &sb, &cb);
    // d lon / du = 2 pi / W, d lat / dv = -pi / H
    D2 SL(sl), CL(cl), SB(sb), CB(cb);
    SL.d[0] = cl * (2.0 * M_PI / W);
    CL.d[0] = -sl * (2.0 * M_PI / W);
    SB.d[1] = cb * (-M_PI / H);
    CB.d[1] = -sb * (-M_PI / H);
    for (int i = 0; i < 4; ++i) sight[i] = CB * SL * sc.image_right[i] + SB * sc.image_up[i] - CB * CL * sc.arrival[i];
  }
  D2 p[4];
  for (int r = 0; r < 4; ++r) {
    D2 s(0.0);
    for (int c = 0; c < 4; ++c) s += sc.metric_covariant[4 * r + c] * (sc.frequency * (sc.four_velocity[c] - sight[c]));
    p[r] = s;
  }
  for (int c = 0; c < 3; ++c) {
    y[c] = D2(sc.observer_txyz[1 + c]);
    y[3 + c] = p[1 + c];
  }
  E = -p[0];
}

// One thread per listed pixel (grid-stride): the center re-traced with tangents.
template <int P>
__global__ void __launch_bounds__(128, 2) footprint_tangent_kernel(
    JobView job, glc_policy pol, const unsigned long long* list, const unsigned int* count, unsigned int capacity,
    glc_footprint* out) {
  using S = typename PrecTraits<P>::S;
  const unsigned int n = min(*count, capacity);
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride) {
    const unsigned long long entry = list[t];
    const glc_camera cam = job.cams[entry >> 32];
    const unsigned long long p = entry & 0xffffffffull;
    const unsigned long long slot = cam.result_offset + p;
    const uint32_t px = uint32_t(p % cam.width), py = uint32_t(p / cam.width);
    const glc_scene& sc = job.scenes[cam.scene_index];
    double st8[8];
    image_state(&sc, &cam, px, py, st8);
    const LaneScene ls = make_lane_scene(sc, pol.mixed_shell_factor, pol.uncertain_terminals != 0u);  // drifts only for the Uncertain gate
    Ray<P> ray;
    ray.init(ls, pol, st8, -1.0);
    RayResult<S> res;
    // the tangents in the trace's own stage precision: binary32 duals for FP32 and MIXED (whose
    // stages are binary32), binary64 for FP64
    using D = typename std::conditional<P == kFP64, D2, Dual<2, float>>::type;
    using R = decltype(D::v);
    D ty[6], E;
    {
      D2 t2[6], e2;
      image_state_tangent(sc, cam, double(px) + cam.subpixel_x, double(py) + cam.subpixel_y, t2, e2);
      for (int c = 0; c < 6; ++c) ty[c] = dual_cast<D>(t2[c]);
      E = dual_cast<D>(e2);
    }
    E.v = R(ray.E);
    bool hit = false;
    for (;;) {
      double y0[6];
      for (int c = 0; c < 6; ++c) y0[c] = double(ray.ys(c));
      const double h0 = double(ray.h);
      const uint32_t acc = ray.accepted;
      bool use64 = false;
      if (P == kMIXED) use64 = __any_sync(__activemask(), double(ray.r) < ls.shell_r);
      if (ray_step<P>(ray, ls, pol, res, use64)) {
        const uint32_t w = (res.termination & 0xFFu) | ((res.candidates & 0xFu) << 12) | ((res.flags & 0xFFFu) << 20);
        if (resolved_surface_code(w)) {
          for (int c = 0; c < 6; ++c) ty[c].v = R(y0[c]);
          hit_tangent(ls.kn, ty, E, h0, double(res.event_theta));
          hit = true;
        }
        break;
      }
      if (ray.accepted != acc) {
        for (int c = 0; c < 6; ++c) ty[c].v = R(y0[c]);
        step_tangent(ls.kn, ty, E, h0);
      }
    }
    if (!hit) {
      footprint_unresolved(out + slot, GLC_FOOTPRINT_NO_SURFACE);
      continue;
    }
    // source radius and oblate azimuth phi = atan2(y, x) - atan2(s a, r) at the hit (the observable's
    // own expressions), differentiated; arc = r_c dphi
    const KN<D> kd{D(ls.kn.a), D(ls.kn.a2), D(ls.kn.s), D(ls.kn.sa), D(ls.kn.q2)};
    int gs;
    const D r = kn_radius(kd, ty[0], ty[1], ty[2], gs);
    const D phi = g_atan2(ty[1], ty[0]) - g_atan2(D(ls.kn.sa), r);
    const double rc = double(res.surface_r);
    const double J[4] = {double(r.d[0]), double(r.d[1]), rc * double(phi.d[0]), rc * double(phi.d[1])};
    glc_footprint f;
    footprint_finish(J, f);
    footprint_store(out + slot, f);
  }
}

}  // namespace glc
