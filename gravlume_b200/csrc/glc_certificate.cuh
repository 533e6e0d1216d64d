// Interval capture certificates on 16x16 pixel tiles.
//
// A tile is certified captured when, for every ray whose pixel lies in the tile, the radial
// potential of Kerr-Newman null geodesics
//   R(r) = [E (r^2 + a^2) - a L]^2 - Delta [(L - a E)^2 + Q],   Delta = r^2 - 2 r + a^2 + Q_e^2,
// is positive on [r_+, r_obs] and the backward-traced ray starts inward. Then dr/dlambda never
// vanishes, the ray reaches r_+ (so the horizon event at r_+ + offset) with r decreasing, and no
// other event of a surface-free scene can fire first (escape needs r to grow, the singularity
// guard lies inside r_+). This is the test of the reference's per-ray certificate
// (crates/gravlume-render/src/shaders/geodesic_acceleration.wgsl:115-279: degree-4 Bernstein bounds
// of R per radial segment), applied once per tile to the whole pixel rectangle, with R kept in its
// structured form q^2 - Delta S (see segment_positive).
//
// Soundness: every quantity is a binary32 interval evaluated with directed rounding
// (__fadd_rd/__fadd_ru, __fmul_rd/__fmul_ru, __fdiv_rd/__fdiv_ru, __fsqrt_rd/__fsqrt_ru), starting
// from the tile's image-plane rectangle and the scene's binary64 constants rounded outward. The
// intervals of E, L_z and Carter's Q therefore contain the exact invariants of every ray of the
// tile. They are further widened by 2^-30 (|v| + 1) so that they also contain the invariants of the
// binary64 initial states the tracer actually integrates, whose rounding is ~1e-16 relative. A
// segment is accepted only when the lower bounds of all five Bernstein coefficients are positive,
// which bounds R away from zero on the segment; anything inconclusive (a non-finite interval, a
// non-positive bound, an ineligible scene) leaves the tile to the full integration.
#pragma once

#include <cuda_runtime.h>

#include <cmath>

#include "glc_kernels.cuh"

namespace glc {

struct Iv {
  float lo, hi;
};

__device__ __forceinline__ float next_down(float v) { return nextafterf(v, -INFINITY); }
__device__ __forceinline__ float next_up(float v) { return nextafterf(v, INFINITY); }

// Binary64 value, or a binary64 range, to a binary32 interval rounded outward by one further ulp.
__device__ __forceinline__ Iv iv_d(double v) { return {next_down(__double2float_rd(v)), next_up(__double2float_ru(v))}; }
__device__ __forceinline__ Iv iv_d(double lo, double hi) {
  return {next_down(__double2float_rd(lo)), next_up(__double2float_ru(hi))};
}
__device__ __forceinline__ Iv iv_add(Iv a, Iv b) { return {__fadd_rd(a.lo, b.lo), __fadd_ru(a.hi, b.hi)}; }
__device__ __forceinline__ Iv iv_sub(Iv a, Iv b) { return {__fsub_rd(a.lo, b.hi), __fsub_ru(a.hi, b.lo)}; }
__device__ __forceinline__ Iv iv_neg(Iv a) { return {-a.hi, -a.lo}; }
__device__ __forceinline__ Iv iv_mul(Iv a, Iv b) {
  const float l = fminf(fminf(__fmul_rd(a.lo, b.lo), __fmul_rd(a.lo, b.hi)), fminf(__fmul_rd(a.hi, b.lo), __fmul_rd(a.hi, b.hi)));
  const float h = fmaxf(fmaxf(__fmul_ru(a.lo, b.lo), __fmul_ru(a.lo, b.hi)), fmaxf(__fmul_ru(a.hi, b.lo), __fmul_ru(a.hi, b.hi)));
  return {l, h};
}
__device__ __forceinline__ Iv iv_sqr(Iv a) {
  const float l2 = __fmul_rd(a.lo, a.lo), h2 = __fmul_rd(a.hi, a.hi);
  const float l2u = __fmul_ru(a.lo, a.lo), h2u = __fmul_ru(a.hi, a.hi);
  if (a.lo <= 0.0f && a.hi >= 0.0f) return {0.0f, fmaxf(l2u, h2u)};
  return {fminf(l2, h2), fmaxf(l2u, h2u)};
}
// Division by a positive exact scalar.
__device__ __forceinline__ Iv iv_div(Iv a, float s) { return {__fdiv_rd(a.lo, s), __fdiv_ru(a.hi, s)}; }
__device__ __forceinline__ Iv iv_scale(Iv a, float s) { return iv_mul(a, Iv{s, s}); }
// 1 / sqrt(a) for a > 0.
__device__ __forceinline__ Iv iv_rsqrt(Iv a) { return {__fdiv_rd(1.0f, __fsqrt_ru(a.hi)), __fdiv_ru(1.0f, __fsqrt_rd(a.lo))}; }
__device__ __forceinline__ Iv iv_widen(Iv a, float rel) {
  const float pad = __fmul_ru(rel, __fadd_ru(fmaxf(fabsf(a.lo), fabsf(a.hi)), 1.0f));
  return {__fsub_rd(a.lo, pad), __fadd_ru(a.hi, pad)};
}
__device__ __forceinline__ bool iv_ok(Iv a) { return isfinite(a.lo) && isfinite(a.hi) && a.lo <= a.hi; }

// Range of sin and cos over [lo, hi] (|lo|, |hi| <= 2 pi, hi - lo < pi), from binary64 endpoint
// values widened by 2^-40 (far above the few-ulp error of the binary64 functions) and from the
// interior extrema the interval contains.
__device__ __forceinline__ void sincos_range(double lo, double hi, Iv& s, Iv& c) {
  double sl, cl, sh, ch;
  sincos(lo, &sl, &cl);
  sincos(hi, &sh, &ch);
  double smin = fmin(sl, sh), smax = fmax(sl, sh), cmin = fmin(cl, ch), cmax = fmax(cl, ch);
  const double kPi = 3.141592653589793, kHalf = 1.5707963267948966;
  for (int k = -2; k <= 2; ++k) {
    const double peak = kHalf + 2.0 * kPi * k, trough = -kHalf + 2.0 * kPi * k;
    const double cpeak = 2.0 * kPi * k, ctrough = kPi + 2.0 * kPi * k;
    // the extrema positions carry binary64 rounding; test with a margin so an extremum near an end
    // is always included
    if (lo <= peak + 1e-12 && peak - 1e-12 <= hi) smax = 1.0;
    if (lo <= trough + 1e-12 && trough - 1e-12 <= hi) smin = -1.0;
    if (lo <= cpeak + 1e-12 && cpeak - 1e-12 <= hi) cmax = 1.0;
    if (lo <= ctrough + 1e-12 && ctrough - 1e-12 <= hi) cmin = -1.0;
  }
  const double pad = 0x1p-40;
  s = iv_d(smin - pad, smax + pad);
  c = iv_d(cmin - pad, cmax + pad);
}

// Positive on the whole segment [lo, hi] (binary32 endpoints). R is kept in the structured form
// R(r) = q(r)^2 - Delta(r) S with q = E (r^2 + a^2) - a L and S = (L - a E)^2 + Q, so that the wide
// interval S multiplies only the narrow Bernstein coefficients of Delta (which vanish at r_+) instead
// of entering three expanded coefficients independently. With r = lo + w t, t in [0, 1]:
//   q:      degree-2 Bernstein coefficients from q(lo), 2 E lo w, E w^2;
//   q^2:    the degree-4 product coefficients q0^2, q0 q1, (q0 q2 + 2 q1^2)/3, q1 q2, q2^2;
//   Delta:  degree 2 from Delta(lo), (2 lo - 2) w, w^2, elevated to degree 4.
// R > 0 on the segment when every q^2_k - S Delta_k has a positive lower bound.
__device__ __forceinline__ bool segment_positive(float lo, float hi, Iv E, Iv L, Iv S, Iv a, Iv a2q2) {
  const Iv r{lo, lo};
  const Iv w{__fsub_rd(hi, lo), __fsub_ru(hi, lo)};
  const Iv r2 = iv_sqr(r);
  const Iv q0 = iv_sub(iv_mul(E, iv_add(r2, iv_sqr(a))), iv_mul(a, L));
  const Iv a1 = iv_scale(iv_mul(iv_mul(E, r), w), 2.0f);
  const Iv a2 = iv_mul(E, iv_sqr(w));
  const Iv q1 = iv_add(q0, iv_scale(a1, 0.5f));
  const Iv q2 = iv_add(iv_add(q0, a1), a2);
  const Iv P[5] = {iv_sqr(q0), iv_mul(q0, q1), iv_div(iv_add(iv_mul(q0, q2), iv_scale(iv_sqr(q1), 2.0f)), 3.0f),
                   iv_mul(q1, q2), iv_sqr(q2)};
  const Iv e0 = iv_add(iv_sub(r2, iv_scale(r, 2.0f)), a2q2);
  const Iv d1 = iv_mul(iv_sub(iv_scale(r, 2.0f), Iv{2.0f, 2.0f}), w);
  const Iv e1 = iv_add(e0, iv_scale(d1, 0.5f));
  const Iv e2 = iv_add(iv_add(e0, d1), iv_sqr(w));
  const Iv D[5] = {e0, iv_scale(iv_add(e0, e1), 0.5f), iv_div(iv_add(iv_add(e0, iv_scale(e1, 4.0f)), e2), 6.0f),
                   iv_scale(iv_add(e1, e2), 0.5f), e2};
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const Iv R = iv_sub(P[k], iv_mul(S, D[k]));
    if (!iv_ok(R) || !(R.lo > 0.0f)) return false;
  }
  return true;
}

constexpr int kCertTile = 16;
constexpr int kCertSegments = 24;

// The certificate for pixels [x0, x1] x [y0, y1] of an image camera of scene sc.
__device__ inline bool tile_certified(const glc_scene& sc, const glc_camera& cam, uint32_t x0, uint32_t x1,
                                      uint32_t y0, uint32_t y1) {
  if (sc.has_surface || sc.extremality != 0 || !(sc.outer_horizon > 0.0)) return false;
  const double xo = sc.observer_txyz[1], yo = sc.observer_txyz[2], zo = sc.observer_txyz[3];
  const double a = sc.spin, a2 = a * a;
  // observer radius and radial gradient in binary64 (kn_rhs's formulas), then outward intervals
  const double R2 = xo * xo + yo * yo + zo * zo, bb = R2 - a2, az2 = a2 * zo * zo;
  const double sq = sqrt(bb * bb + 4.0 * az2);
  const double r2d = bb >= 0.0 ? 0.5 * (bb + sq) : 2.0 * az2 / (sq - bb);
  const double rd = sqrt(r2d);
  const double sigma = r2d + az2 / r2d;
  if (!(rd > sc.horizon_event_radius) || !(rd < 1.0e4)) return false;
  const double Ad = r2d + a2;
  const double grd[3] = {xo * rd / sigma, yo * rd / sigma, zo * Ad / (rd * sigma)};
  const float env = 0x1p-30f;

  // image-plane box of the tile's sample points, then the sight direction
  Iv sight[4];
  const double u0 = double(x0) + cam.subpixel_x, u1 = double(x1) + cam.subpixel_x;
  const double v0 = double(y0) + cam.subpixel_y, v1 = double(y1) + cam.subpixel_y;
  if (cam.kind == GLC_CAMERA_PINHOLE) {
    const double w = double(cam.width), h = double(cam.height);
    const Iv nx = iv_d(2.0 * u0 / w - 1.0, 2.0 * u1 / w - 1.0);
    const Iv ny = iv_d(1.0 - 2.0 * v1 / h, 1.0 - 2.0 * v0 / h);
    const Iv sx = iv_mul(iv_d((w / h) * sc.tangent_half_fov), nx);
    const Iv sy = iv_mul(iv_d(sc.tangent_half_fov), ny);
    const Iv nrm = iv_rsqrt(iv_add(Iv{1.0f, 1.0f}, iv_add(iv_sqr(sx), iv_sqr(sy))));
#pragma unroll
    for (int i = 0; i < 4; ++i)
      sight[i] = iv_mul(iv_sub(iv_add(iv_mul(iv_d(sc.image_right[i]), sx), iv_mul(iv_d(sc.image_up[i]), sy)),
                               iv_d(sc.arrival[i])),
                        nrm);
  } else if (cam.kind == GLC_CAMERA_EQUIRECT) {
    const double kPi = 3.141592653589793;
    const double lon0 = 2.0 * kPi * (u0 / double(cam.width)) - kPi, lon1 = 2.0 * kPi * (u1 / double(cam.width)) - kPi;
    const double lat1 = 0.5 * kPi - kPi * (v0 / double(cam.height)), lat0 = 0.5 * kPi - kPi * (v1 / double(cam.height));
    if (!(lon1 - lon0 < 3.0) || !(lat1 - lat0 < 3.0)) return false;
    Iv sl, cl, sb, cb;
    sincos_range(lon0 - 1e-12, lon1 + 1e-12, sl, cl);
    sincos_range(lat0 - 1e-12, lat1 + 1e-12, sb, cb);
#pragma unroll
    for (int i = 0; i < 4; ++i)
      sight[i] = iv_sub(iv_add(iv_mul(iv_mul(cb, sl), iv_d(sc.image_right[i])), iv_mul(sb, iv_d(sc.image_up[i]))),
                        iv_mul(iv_mul(cb, cl), iv_d(sc.arrival[i])));
  } else {
    return false;
  }
  // p^mu = omega (u^mu - sight^mu), p_mu = g_{mu nu} p^nu
  Iv pc[4], p[4];
  const Iv om = iv_d(sc.frequency);
#pragma unroll
  for (int i = 0; i < 4; ++i) pc[i] = iv_mul(om, iv_sub(iv_d(sc.four_velocity[i]), sight[i]));
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    Iv s{0.0f, 0.0f};
#pragma unroll
    for (int n = 0; n < 4; ++n) s = iv_add(s, iv_mul(iv_d(sc.metric_covariant[4 * m + n]), pc[n]));
    p[m] = s;
  }
  // the backward trace must start inward: the future-directed dr/dlambda = grad r . p^i > 0
  Iv vr = iv_mul(iv_d(grd[0]), pc[1]);
  vr = iv_add(vr, iv_mul(iv_d(grd[1]), pc[2]));
  vr = iv_add(vr, iv_mul(iv_d(grd[2]), pc[3]));
  if (!iv_ok(vr) || !(vr.lo > 0.0f)) return false;

  const Iv x = iv_d(xo), y = iv_d(yo), z = iv_d(zo);
  const Iv E = iv_widen(iv_neg(p[0]), env);
  const Iv px = p[1], py = p[2], pz = p[3];
  const Iv L = iv_widen(iv_sub(iv_mul(x, py), iv_mul(y, px)), env);
  const Iv Lx = iv_sub(iv_mul(y, pz), iv_mul(z, py)), Ly = iv_sub(iv_mul(z, px), iv_mul(x, pz));
  const Iv rinv2 = iv_d(1.0 / r2d), Ainv = iv_d(1.0 / Ad);  // exact reciprocals lie within one binary32 ulp
  const Iv bracket = iv_sub(iv_mul(iv_mul(iv_sqr(z), rinv2), iv_sub(iv_add(iv_sqr(px), iv_sqr(py)), iv_sqr(E))),
                            iv_mul(iv_mul(iv_add(iv_sqr(x), iv_sqr(y)), Ainv), iv_sqr(pz)));
  const Iv Q = iv_widen(iv_add(iv_add(iv_sqr(Lx), iv_sqr(Ly)), iv_mul(iv_d(a2), bracket)), env);
  if (!iv_ok(E) || !iv_ok(L) || !iv_ok(Q) || !(E.lo > 0.0f)) return false;

  const Iv A = iv_d(a), a2q2 = iv_d(a2 + sc.charge * sc.charge);
  const Iv S = iv_add(iv_sqr(iv_sub(L, iv_mul(A, E))), Q);
  if (!iv_ok(S)) return false;

  // geometric segments from r_+ (rounded down) to r_obs (rounded up); consecutive segments share
  // the same binary32 endpoint, so together they cover [r_+, r_obs]
  const float r_lo = next_down(__double2float_rd(sc.outer_horizon));
  const float r_hi = next_up(__double2float_ru(rd));
  const double ratio = double(r_hi) / double(r_lo);
  float prev = r_lo;
  for (int k = 1; k <= kCertSegments; ++k) {
    const float e = k == kCertSegments ? r_hi : float(double(r_lo) * pow(ratio, double(k) / kCertSegments));
    if (!(e > prev)) return false;
    if (!segment_positive(prev, e, E, L, S, A, a2q2)) return false;
    prev = e;
  }
  return true;
}

// One thread per 16x16 tile of every image camera; writes 1 to cert[tile] when certified.
__global__ void certify_tiles_kernel(JobView job, uint32_t* cert) {
  const unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= job.cert_begin[job.n_cams]) return;
  int lo = 0, hi = job.n_cams - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (job.cert_begin[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  const glc_camera& cam = job.cams[lo];
  const unsigned long long j = t - job.cert_begin[lo];
  const uint32_t tiles_x = (cam.width + kCertTile - 1) / kCertTile;
  const uint32_t tx = uint32_t(j % tiles_x), ty = uint32_t(j / tiles_x);
  const uint32_t x0 = tx * kCertTile, y0 = ty * kCertTile;
  const uint32_t x1 = min(x0 + kCertTile - 1, cam.width - 1), y1 = min(y0 + kCertTile - 1, cam.height - 1);
  cert[t] = tile_certified(job.scenes[cam.scene_index], cam, x0, x1, y0, y1) ? 1u : 0u;
}

}  // namespace glc
