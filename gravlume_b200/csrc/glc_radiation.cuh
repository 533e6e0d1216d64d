// Post-hit surface transport (crates/gravlume-reference/src/surface.rs:12-200 and radiation.rs:13-120):
// the inverse-cube bolometric emitter I_em(r) = I_6 (r/6)^-3, its vacuum observed intensity
// I_em g^4, the inverse-cube blackbody temperature T_em(r) = T_6 (r/6)^-3/4 observed at g T_em, the
// observed blackbody intensity split into the three visible boxcar bands (600-700, 500-600,
// 400-500 nm) by Planck band fractions, and the homogeneous scalar slab in front of the surface
// (incoming e^-tau + its integrated emission, itself blackbody-split for the bands).
//
// The band fraction is the Planck integral int_{x_lo}^{x_hi} t^3 / (e^t - 1) dt / (pi^4 / 15) over
// x = c_2 / (lambda T). The reference evaluates it by adaptive Simpson quadrature (and a
// logarithmic tail above x = 50). Here, so that a surface hit costs a few hundred flops and no
// lookup table, the integral comes from closed forms of F(x) = int_x^inf t^3 / (e^t - 1) dt:
//   x >= 2:  F(x) = sum_k e^{-k x} (x^3/k + 3 x^2/k^2 + 6 x/k^3 + 6/k^4)   (exponential series),
//   x < 2:   F(x) = pi^4/15 - G(x),  G(x) = x^3/3 - x^4/8 + sum_m B_2m / (2m)! x^{2m+3} / (2m+3)
//            (Bernoulli series of t^3 / (e^t - 1), radius 2 pi); a band whose ends both lie below
//            2 is G(x_hi) - G(x_lo), which keeps its relative accuracy at high temperatures,
//   x > 50:  the reference's logarithmic tail, ln F = 3 ln x - x + ln(1 + 3/x + 6/x^2 + 6/x^3).
// Both series are truncated where their terms fall below 1e-16 of the sum.
#pragma once

#include "glc_geometry.cuh"

namespace glc {

constexpr double kSecondRadiationConstant = 0.014387768775039337;  // c_2 = h c / k_B, m K
constexpr double kPlanckIntegral = 6.4939394022668291;             // pi^4 / 15
constexpr double kLn2 = 0.69314718055994531;

GLC_HD double rad_exp(double x) {
#if defined(__CUDA_ARCH__)
  return exp(x);
#else
  return std::exp(x);
#endif
}
GLC_HD double rad_log(double x) {
#if defined(__CUDA_ARCH__)
  return log(x);
#else
  return std::log(x);
#endif
}
GLC_HD double rad_log1p(double x) {
#if defined(__CUDA_ARCH__)
  return log1p(x);
#else
  return std::log1p(x);
#endif
}

// G(x) = int_0^x t^3 / (e^t - 1) dt for 0 <= x < 2 (Bernoulli series).
GLC_HD double planck_head(double x) {
  // B_2m / (2m)! / (2m + 3), m = 1 .. 16
  const double c[16] = {1.66666666666666664e-02,  -1.98412698412698413e-04, 3.67430922986478553e-06,
                        -7.51563251563251607e-08, 1.60590438368216149e-09,  -3.52279342579166215e-11,
                        7.87208031216745774e-13,  -1.78404226122241216e-14, 4.08860097917992578e-16,
                        -9.45595086329592140e-18, 2.20360113134409181e-19,  -5.16832025400463853e-21,
                        1.21886449642395423e-22,  -2.88823142807662809e-24, 6.87258318890207039e-26,
                        -1.64136876253491499e-27};
  const double x2 = x * x;
  double s = 0.0;
  for (int m = 15; m >= 0; --m) s = s * x2 + c[m];
  return x * x2 * (1.0 / 3.0 - x / 8.0 + x2 * s);
}

// ln F(x) = ln int_x^inf t^3 / (e^t - 1) dt, x > 0.
GLC_HD double planck_log_tail(double x) {
  if (x > 50.0) {
    const double inv = 1.0 / x;
    return 3.0 * rad_log(x) - x + rad_log1p(inv * (3.0 + inv * (6.0 + 6.0 * inv)));
  }
  if (x >= 2.0) {
    double sum = 0.0;
    const double q = rad_exp(-x);
    double qk = q;
    const int terms = int(40.0 / x) + 1;
    for (int k = 1; k <= terms; ++k) {
      const double ik = 1.0 / double(k);
      sum += qk * ik * (x * x * x + ik * (3.0 * x * x + ik * (6.0 * x + 6.0 * ik)));
      qk *= q;
    }
    return rad_log(sum);
  }
  return rad_log(kPlanckIntegral - planck_head(x));
}

// ln int_{x_lo}^{x_hi} t^3 / (e^t - 1) dt, 0 < x_lo < x_hi: from G where both ends lie in the
// series' range (no cancellation against pi^4 / 15), else from F.
GLC_HD double planck_log_band(double x_lo, double x_hi) {
  if (x_hi < 2.0) return rad_log(planck_head(x_hi) - planck_head(x_lo));
  const double a = planck_log_tail(x_lo), b = planck_log_tail(x_hi);
  return a + rad_log1p(-rad_exp(b - a));
}

// log2 of the fraction of the blackbody intensity at temperature T (K) inside the wavelength band
// [lo_nm, hi_nm]; returns false when not representable.
GLC_HD bool blackbody_band_log2_fraction(double T, double lo_nm, double hi_nm, double& log2_fraction) {
  const double x_lo = kSecondRadiationConstant / (hi_nm * 1.0e-9 * T);
  const double x_hi = kSecondRadiationConstant / (lo_nm * 1.0e-9 * T);
  if (!(x_lo > 0.0) || !(x_hi > x_lo) || !g_finite(x_hi)) return false;
  const double log_integral = planck_log_band(x_lo, x_hi);
  log2_fraction = (log_integral - rad_log(kPlanckIntegral)) / kLn2;
  return g_finite(log2_fraction) && log2_fraction <= 0.0;
}

// The three visible boxcar bands (red 600-700, green 500-600, blue 400-500 nm) of a bolometric
// intensity I at temperature T.
GLC_HD bool blackbody_bands(double I, double T, double out[3]) {
  const double lo[3] = {600.0, 500.0, 400.0}, hi[3] = {700.0, 600.0, 500.0};
  if (!(I >= 0.0) || !g_finite(I) || !(T > 0.0) || !g_finite(T)) return false;
  for (int b = 0; b < 3; ++b) {
    double l2;
    if (!blackbody_band_log2_fraction(T, lo[b], hi[b], l2)) return false;
    out[b] = I > 0.0 ? rad_exp((rad_log(I) / kLn2 + l2) * kLn2) : 0.0;
  }
  return true;
}

// Surface radiance of a hit at radius r with frequency ratio g (M = 1). model 0: inverse-cube
// bolometric, 1: inverse-cube blackbody with T_6 = temp6. The slab (transmittance, integrated
// emission, its band split) is applied after the vacuum transport. Outputs: emitted and observed
// bolometric intensity; rgb = observed band intensities (blackbody) or the observed bolometric
// intensity in all three (bolometric).
GLC_HD bool surface_radiance(int model, double I6, double temp6, double transmittance, double slab_emission,
                             const double slab_bands[3], double r, double g, double& emitted, double& observed,
                             double rgb[3]) {
  const double rr = r / 6.0;
  if (!(rr > 0.0) || !g_finite(rr) || !(g > 0.0)) return false;
  emitted = I6 / (rr * rr * rr);
  const double vac = emitted * g * g * g * g;
  observed = vac * transmittance + slab_emission;
  if (!g_finite(observed) || observed < 0.0) return false;
  if (model == 1) {
    const double T = g * temp6 / g_sqrt(rr * g_sqrt(rr));
    double bands[3];
    if (!blackbody_bands(vac, T, bands)) return false;
    for (int b = 0; b < 3; ++b) rgb[b] = bands[b] * transmittance + slab_bands[b];
  } else {
    rgb[0] = rgb[1] = rgb[2] = observed;
  }
  return true;
}

}  // namespace glc
