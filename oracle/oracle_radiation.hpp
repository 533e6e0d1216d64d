// Oracle (test infrastructure, not the product): binary64 restatement of the reference's surface
// radiation model, the checker of the CUDA path's post-hit transport.
//   Planck band integrals: crates/gravlume-reference/src/radiation.rs:84-170 (80 unit intervals of
//     adaptive Simpson quadrature to 8 eps, depth 20; logarithmic x^3 e^-x tail at x >= 50)
//   band split and slab transport: radiation.rs:13-78 (visible boxcar bands 600-700, 500-600,
//     400-500 nm from gravlume-domain/src/radiation.rs:4-8)
//   emitter profiles: crates/gravlume-reference/src/surface.rs:148-200
#pragma once

#include <cfloat>
#include <cmath>

namespace gro {

constexpr double kC2 = 0.014387768775039337;  // second radiation constant, m K
inline double planck_norm() { return std::pow(M_PI, 4) / 15.0; }

inline double planck_kernel(double x) {
  if (x == 0.0) return 0.0;
  if (x > 50.0) {
    const double e = std::exp(-x);
    return x * x * x * e / (1.0 - e);
  }
  return x * x * x / std::expm1(x);
}

inline double simpson_rule(double a, double b, double fa, double fm, double fb) {
  return (b - a) * (std::fma(4.0, fm, fa) + fb) / 6.0;
}

// radiation.rs:139-161
inline double adaptive_simpson_rule(double a, double b, double whole, double tol, unsigned depth) {
  const double m = 0.5 * (a + b), lm = 0.5 * (a + m), rm = 0.5 * (m + b);
  const double left = simpson_rule(a, m, planck_kernel(a), planck_kernel(lm), planck_kernel(m));
  const double right = simpson_rule(m, b, planck_kernel(m), planck_kernel(rm), planck_kernel(b));
  const double refined = left + right, corr = refined - whole;
  if (depth == 0 || std::fabs(corr) <= 15.0 * tol) return refined + corr / 15.0;
  return adaptive_simpson_rule(a, m, left, 0.5 * tol, depth - 1) +
         adaptive_simpson_rule(m, b, right, 0.5 * tol, depth - 1);
}

// radiation.rs:113-132: unit intervals [i, i+1] of [0, 80] clipped to [lo, hi]
inline double integrate_planck(double lo, double hi) {
  double sum = 0.0;
  for (unsigned i = 0; i < 80; ++i) {
    const double l = std::fmax(lo, double(i)), r = std::fmin(hi, double(i + 1));
    if (!(l < r)) continue;
    const double m = 0.5 * (l + r);
    const double whole = simpson_rule(l, r, planck_kernel(l), planck_kernel(m), planck_kernel(r));
    const double tol = 8.0 * DBL_EPSILON * std::fmax(std::fabs(whole), DBL_MIN);
    sum += adaptive_simpson_rule(l, r, whole, tol, 20);
  }
  return sum;
}

// radiation.rs:126-137
inline double log_planck_tail(double x) {
  const double inv = 1.0 / x;
  const double poly = inv * std::fma(inv, std::fma(6.0, inv, 6.0), 3.0);
  return std::fma(3.0, std::log(x), -x) + std::log1p(poly);
}

// radiation.rs:84-101
inline bool band_log2_fraction(double T, double lo_nm, double hi_nm, double& out) {
  const double xl = kC2 / (hi_nm * 1.0e-9 * T), xh = kC2 / (lo_nm * 1.0e-9 * T);
  if (!std::isfinite(xl) || !std::isfinite(xh) || xl < 0.0 || xh <= xl) return false;
  double log_integral;
  if (xl >= 50.0) {
    const double a = log_planck_tail(xl), b = log_planck_tail(xh);
    log_integral = a + std::log1p(-std::exp(b - a));
  } else {
    log_integral = std::log(integrate_planck(xl, xh));
  }
  out = (log_integral - std::log(planck_norm())) / M_LN2;
  return std::isfinite(out) && out <= 0.0;
}

// radiation.rs:103-111
inline bool scale_log2(double v, double l2, double& out) {
  const double s = std::exp2(l2);
  out = (s == 0.0 && v > 0.0) ? std::exp2(std::log2(v) + l2) : v * s;
  return std::isfinite(out) && out >= 0.0;
}

// radiation.rs:13-31
inline bool blackbody_bands(double I, double T, double out[3]) {
  if (!std::isfinite(I) || I < 0.0 || !std::isfinite(T) || T <= 0.0) return false;
  const double lo[3] = {600.0, 500.0, 400.0}, hi[3] = {700.0, 600.0, 500.0};
  for (int b = 0; b < 3; ++b) {
    double l2;
    if (!band_log2_fraction(T, lo[b], hi[b], l2) || !scale_log2(I, l2, out[b])) return false;
  }
  return true;
}

// surface.rs:12-72 after the frequency ratio: emitted and observed bolometric intensity, and the
// observed bands (blackbody) or the observed bolometric intensity (bolometric), with the slab.
inline bool surface_radiance(int model, double I6, double T6, bool slab, double tau, double S, double Tslab,
                             double r, double g, double out[5]) {
  const double ratio = r / 6.0;
  if (!std::isfinite(ratio) || ratio <= 0.0) return false;
  double em = I6;
  for (int i = 0; i < 3; ++i) em /= ratio;
  double vac = em;
  for (int i = 0; i < 4; ++i) vac *= g;
  const double trans = slab ? std::exp(-tau) : 1.0, src = slab ? S : 0.0;
  const double obs = std::fma(vac, trans, src);
  out[0] = em;
  out[1] = obs;
  if (model == 1) {
    const double Tem = T6 / std::sqrt(ratio * std::sqrt(ratio));
    double bands[3], sb[3] = {0.0, 0.0, 0.0};
    if (!blackbody_bands(vac, Tem * g, bands)) return false;
    if (slab && S > 0.0 && !blackbody_bands(S, Tslab, sb)) return false;
    for (int b = 0; b < 3; ++b) out[2 + b] = std::fma(bands[b], trans, sb[b]);
  } else {
    out[2] = out[3] = out[4] = obs;
  }
  return true;
}

}  // namespace gro
