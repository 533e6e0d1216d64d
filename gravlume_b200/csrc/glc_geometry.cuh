// Kerr-Newman geometry and the reduced Hamilton right-hand side in Cartesian Kerr-Schild
// coordinates, templated on the arithmetic type (float / double) and compiled for both the
// device and the host (host builds back glc_rhs_host and the CPU checks).
//
// Metric: g^{mu nu} = eta^{mu nu} - f l^mu l^nu with l^mu = (-1, l_x, l_y, l_z), M = 1,
//   r^2 = (b + sqrt(b^2 + 4 a^2 z^2)) / 2, b = x^2 + y^2 + z^2 - a^2 (conjugate root when b < 0),
//   f = (2 r - Q^2) r^2 / (r^4 + a^2 z^2),
//   l = s ((r x + s a y) / (r^2 + a^2), (r y - s a x) / (r^2 + a^2), z / r), s = +1 ingoing, -1 outgoing.
// With q = E + l.p (E = -p_t) the exact reduced system is
//   x' = p - f q l,  p' = f q w + q^2 grad(f) / 2,  t' = E + f q,   w_i = p_j d_i l_j = e_i + C d_i r,
//   e = ((s r p_x - a p_y) / A, (a p_x + s r p_y) / A, s p_z / r), A = r^2 + a^2,
//   C = [(s x - 2 r l_x) p_x + (s y - 2 r l_y) p_y] / A - s z p_z / r^2.
// This is the contraction of the full null-vector Jacobian that the reference's binary64 oracle
// builds explicitly (crates/gravlume-domain/src/spacetime.rs:492-582, hamiltonian_rhs 305-338);
// the reference derives the same contracted form in docs/physics.md section 4. The state carries
// (x, y, z, p_x, p_y, p_z) and the relative coordinate time; E is constant per ray.
#pragma once

#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define GLC_HD __host__ __device__ __forceinline__
#else
#define GLC_HD inline
#endif

namespace glc {

// ---------------------------------------------------------------- precision helpers
GLC_HD float g_rsqrt(float x) {
#if defined(__CUDA_ARCH__)
  return rsqrtf(x);
#else
  return 1.0f / std::sqrt(x);
#endif
}
GLC_HD double g_rsqrt(double x) {
#if defined(__CUDA_ARCH__)
  return rsqrt(x);
#else
  return 1.0 / std::sqrt(x);
#endif
}
GLC_HD float g_rcp(float x) {
#if defined(__CUDA_ARCH__)
  return __fdividef(1.0f, x);
#else
  return 1.0f / x;
#endif
}
GLC_HD double g_rcp(double x) {
#if defined(__CUDA_ARCH__)
  return __drcp_rn(x);
#else
  return 1.0 / x;
#endif
}
GLC_HD float g_sqrt(float x) {
#if defined(__CUDA_ARCH__)
  return sqrtf(x);
#else
  return std::sqrt(x);
#endif
}
GLC_HD double g_sqrt(double x) {
#if defined(__CUDA_ARCH__)
  return sqrt(x);
#else
  return std::sqrt(x);
#endif
}
#if defined(__CUDA_ARCH__)
GLC_HD float g_abs(float x) { return fabsf(x); }
GLC_HD double g_abs(double x) { return fabs(x); }
GLC_HD float g_max(float a, float b) { return fmaxf(a, b); }
GLC_HD double g_max(double a, double b) { return fmax(a, b); }
GLC_HD float g_min(float a, float b) { return fminf(a, b); }
GLC_HD double g_min(double a, double b) { return fmin(a, b); }
GLC_HD bool g_finite(float x) { return isfinite(x); }
GLC_HD bool g_finite(double x) { return isfinite(x); }
GLC_HD bool g_signbit(float x) { return signbit(x); }
GLC_HD bool g_signbit(double x) { return signbit(x); }
GLC_HD float g_floor(float x) { return floorf(x); }
GLC_HD double g_floor(double x) { return floor(x); }
GLC_HD float g_atan2(float y, float x) { return atan2f(y, x); }
GLC_HD double g_atan2(double y, double x) { return atan2(y, x); }
GLC_HD float g_acos(float x) { return acosf(x); }
GLC_HD double g_acos(double x) { return acos(x); }
#else
GLC_HD float g_abs(float x) { return std::fabs(x); }
GLC_HD double g_abs(double x) { return std::fabs(x); }
GLC_HD float g_max(float a, float b) { return std::fmax(a, b); }
GLC_HD double g_max(double a, double b) { return std::fmax(a, b); }
GLC_HD float g_min(float a, float b) { return std::fmin(a, b); }
GLC_HD double g_min(double a, double b) { return std::fmin(a, b); }
GLC_HD bool g_finite(float x) { return std::isfinite(x); }
GLC_HD bool g_finite(double x) { return std::isfinite(x); }
GLC_HD bool g_signbit(float x) { return std::signbit(x); }
GLC_HD bool g_signbit(double x) { return std::signbit(x); }
GLC_HD float g_floor(float x) { return std::floor(x); }
GLC_HD double g_floor(double x) { return std::floor(x); }
GLC_HD float g_atan2(float y, float x) { return std::atan2(y, x); }
GLC_HD double g_atan2(double y, double x) { return std::atan2(y, x); }
GLC_HD float g_acos(float x) { return std::acos(x); }
GLC_HD double g_acos(double x) { return std::acos(x); }
#endif
// err^(-1/5) for the step controller.
GLC_HD float g_pow_m02(float x) {
#if defined(__CUDA_ARCH__)
  return exp2f(-0.2f * __log2f(x));
#else
  return std::pow(x, -0.2f);
#endif
}
GLC_HD double g_pow_m02(double x) {
#if defined(__CUDA_ARCH__)
  return pow(x, -0.2);
#else
  return std::pow(x, -0.2);
#endif
}

// ---------------------------------------------------------------- spacetime constants
template <class T>
struct KN {
  T a, a2, s, sa, q2;  // spin, spin^2, chart sign, s*a, charge^2  (M = 1)
};

template <class T, class U>
GLC_HD KN<T> kn_cast(const KN<U>& k) {
  return KN<T>{T(k.a), T(k.a2), T(k.s), T(k.sa), T(k.q2)};
}

enum GeomStatus : int { kGeomOk = 0, kGeomRing = 2, kGeomChart = 3, kGeomDenominator = 4 };

// Kerr-Schild radius squared from Cartesian position (stable root selection).
template <class T>
GLC_HD T kn_radius_squared(const KN<T>& k, T x, T y, T z, int& status) {
  const T R2 = x * x + y * y + z * z;
  const T b = R2 - k.a2;
  const T az2 = k.a2 * z * z;
  const T sq = g_sqrt(b * b + T(4) * az2);
  T r2;
  if (b >= T(0)) {
    r2 = T(0.5) * (b + sq);
  } else {
    r2 = T(2) * az2 / (sq - b);
  }
  status = r2 > T(0) ? kGeomOk : (b == T(0) ? kGeomRing : kGeomChart);
  return r2;
}

template <class T>
GLC_HD T kn_radius(const KN<T>& k, T x, T y, T z, int& status) {
  const T r2 = kn_radius_squared(k, x, y, z, status);
  return g_sqrt(r2);
}

// Reduced right-hand side. y = (x, y, z, p_x, p_y, p_z); d = (x', y', z', p_x', p_y', p_z', t').
// Also returns r and the radial velocity dr/dlambda = grad(r) . x'. Non-finite values propagate
// as NaN into the step's error norm, which the stepper turns into a numerical failure.
// L_z, Carter's constant, the normalized null residual and the spin term of Carter's constant
// (Q = L_x^2 + L_y^2 + abracket, see kn_invariants).
template <class T>
struct Invariants {
  T lz, carter, null_residual, abracket;
};

// kInv: also evaluate L_z, Carter's constant and the normalized null residual at this point from
// the same geometry (used on the end-of-step evaluation, whose point is the committed state).
template <class T, bool kInv = false>
GLC_HD void kn_rhs(const KN<T>& k, const T y[6], T E, T d[7], T& r_out, T& vr_out, Invariants<T>* inv = nullptr) {
  const T x = y[0], yy = y[1], z = y[2], px = y[3], py = y[4], pz = y[5];
  // the radius exactly as kn_radius_squared forms it, so both give the same r
  const T R2 = x * x + yy * yy + z * z;
  const T b = R2 - k.a2;
  const T az2 = k.a2 * z * z;
  const T sq = g_sqrt(b * b + T(4) * az2);
  T r2;
  if (b >= T(0)) {
    r2 = T(0.5) * (b + sq);
  } else {
    r2 = T(2) * az2 * g_rcp(sq - b);
  }
  const T inv_r = g_rsqrt(r2);
  const T r = r2 * inv_r;
  const T inv_r2 = inv_r * inv_r;
  const T A = r2 + k.a2;
  const T m = az2 * inv_r2;  // a^2 z^2 / r^2
  const T sigma = r2 + m;    // (r^4 + a^2 z^2) / r^2
  // one reciprocal for both denominators: 1/A = sigma/(A sigma), 1/sigma = A/(A sigma)
  const T inv_As = g_rcp(A * sigma);
  const T inv_A = sigma * inv_As;
  const T inv_sigma = A * inv_As;
  // The chart sign s = +-1 factors out of the null vector l = s lt, of e = s et and of C = s Ct
  // (s^2 = 1 turns s a into sa inside them), so it enters once, through q and fqs = f q s.
  // lt = ((r x + sa y) / A, (r y - sa x) / A, z / r)
  const T lzt = z * inv_r;
  const T lxt = (r * x + k.sa * yy) * inv_A;
  const T lyt = (r * yy - k.sa * x) * inv_A;
  // grad r = (x r, y r, z A / r) / sigma
  const T rs = r * inv_sigma;
  const T grx = x * rs, gry = yy * rs, grz = lzt * (A * inv_sigma);
  // f = (2 r - Q^2) / sigma; grad f = c1 grad r - (0, 0, 2 a^2 z f / (r^2 sigma)) with
  // c1 = (2 - 2 f (r - a^2 z^2 / r^3)) / sigma, carried as c1h = c1 / 2
  const T f = (T(2) * r - k.q2) * inv_sigma;
  const T c1h = (T(1) - f * (r - m * inv_r)) * inv_sigma;
  // q = E + l . p
  const T lxy = lxt * px + lyt * py;
  const T lzp = lzt * pz;
  const T q = E + k.s * (lxy + lzp);
  const T fq = f * q;
  const T fqs = k.s * fq;
  // Ct = ((x - 2 r lt_x) p_x + (y - 2 r lt_y) p_y) / A - z p_z / r^2
  const T Ct = (x * px + yy * py - (r + r) * lxy) * inv_A - lzp * inv_r;
  // p' = f q (e + C grad r) + q^2 / 2 grad f = fqs et + K grad r - q^2 (0, 0, a^2 z f / (r^2 sigma))
  // with et = ((r p_x - sa p_y) / A, (sa p_x + r p_y) / A, p_z / r) and K = fqs Ct + q^2 c1h
  const T qq = q * q;
  const T K = fqs * Ct + qq * c1h;
  const T W = fqs * inv_A;
  const T gz = f * inv_sigma * lzt * inv_r * k.a2;
  d[0] = px - fqs * lxt;
  d[1] = py - fqs * lyt;
  d[2] = pz - fqs * lzt;
  d[3] = W * (r * px - k.sa * py) + K * grx;
  d[4] = W * (k.sa * px + r * py) + K * gry;
  d[5] = (fqs * inv_r) * pz + K * grz - qq * gz;
  d[6] = E + fq;
  r_out = r;
  vr_out = grx * d[0] + gry * d[1] + grz * d[2];
  if (kInv && inv != nullptr) {
    // Carter's constant as Q = L_x^2 + L_y^2 + a^2 [(z^2/r^2)(P_perp^2 - E^2) - (rho^2/A) p_z^2]
    // (see kn_invariants): no r^2-sized terms cancel, so binary32 keeps its relative accuracy far out
    const T rho2 = x * x + yy * yy;
    const T pp2 = px * px + py * py;
    const T Lx = yy * pz - z * py, Ly = z * px - x * pz;
    inv->lz = x * py - yy * px;
    inv->abracket = k.a2 * (z * z * inv_r2 * (pp2 - E * E) - rho2 * inv_A * pz * pz);
    inv->carter = Lx * Lx + Ly * Ly + inv->abracket;
    // g^{mu nu} p_mu p_nu with m = eta - f l l and u_i = l^i p_i (u_0 = E): diagonal terms
    // eta_ii p_i^2 - f u_i^2, off-diagonal -f u_i u_j (only u_i^2 and |u_i| enter, so lt serves)
    const T u1 = lxt * px, u2 = lyt * py, u3 = lzp;
    const T sum = -E * E + pp2 + pz * pz - f * qq;
    const T au = g_abs(E) + g_abs(u1) + g_abs(u2) + g_abs(u3);
    const T su2 = E * E + u1 * u1 + u2 * u2 + u3 * u3;
    const T norm = E * E * g_abs(T(1) + f) + g_abs(px * px - f * u1 * u1) + g_abs(py * py - f * u2 * u2) +
                   g_abs(pz * pz - f * u3 * u3) + g_abs(f) * (au * au - su2);
    inv->null_residual = norm > T(0) ? g_abs(sum) * g_rcp(norm) * g_min(norm, T(1)) : T(0);
  }
}

// Conserved quantities and the normalized null residual (the reference's drift diagnostics,
// crates/gravlume-domain/src/spacetime.rs:345-401 and numerics.rs:3-35). Carter's constant uses the
// Cartesian form
//   Q = L_x^2 + L_y^2 + a^2 [(z^2 / r^2)(P_perp^2 - E^2) - (rho^2 / A) p_z^2],
//   L = x cross p, P_perp^2 = p_x^2 + p_y^2, rho^2 = x^2 + y^2, A = r^2 + a^2,
// which equals the oracle's trigonometric form p_theta^2 + cos^2(theta)(L_z^2/sin^2 - a^2 E^2)
// identically (z^2 P_perp^2 - 2 z (x p_x + y p_y) p_z + rho^2 p_z^2 = L_x^2 + L_y^2) and is regular
// on the axis.
template <class T>
GLC_HD Invariants<T> kn_invariants(const KN<T>& k, const T y[6], T E, T r) {
  const T x = y[0], yy = y[1], z = y[2], px = y[3], py = y[4], pz = y[5];
  Invariants<T> out;
  out.lz = x * py - yy * px;
  const T r2 = r * r;
  const T A = r2 + k.a2;
  const T rho2 = x * x + yy * yy;
  const T pp2 = px * px + py * py;
  const T Lx = yy * pz - z * py, Ly = z * px - x * pz;
  out.abracket = k.a2 * (z * z / r2 * (pp2 - E * E) - rho2 / A * pz * pz);
  out.carter = Lx * Lx + Ly * Ly + out.abracket;
  // g^{mu nu} p_mu p_nu with g^{mu nu} = eta - f l l, p = (-E, p_x, p_y, p_z), l = (-1, l_x, l_y, l_z).
  const T inv_r = T(1) / r;
  const T sigma = r2 + k.a2 * z * z / r2;
  const T f = (T(2) * r - k.q2) / sigma;
  const T inv_A = T(1) / A;
  const T l[4] = {T(-1), k.s * (r * x + k.sa * yy) * inv_A, k.s * (r * yy - k.sa * x) * inv_A, k.s * z * inv_r};
  const T p[4] = {-E, px, py, pz};
  T sum = T(0), norm = T(0);
  for (int i = 0; i < 4; ++i) {
    for (int j = 0; j < 4; ++j) {
      const T eta = i == j ? (i == 0 ? T(-1) : T(1)) : T(0);
      const T m = eta - f * l[i] * l[j];
      const T term = m * p[i] * p[j];
      sum += term;
      norm += g_abs(term);
    }
  }
  // |sum| / norm * min(norm, 1): the reference's scale-normalized residual
  // (numerics.rs:3-35) with its overflow-safe product collapsed for finite moderate inputs.
  out.null_residual = norm > T(0) ? g_abs(sum) / norm * g_min(norm, T(1)) : T(0);
  return out;
}

// Binary64 reciprocal from a binary32 seed and one Newton step (relative error ~1e-14): the
// MIXED path's binary64 quantities without binary64 division sequences.
GLC_HD double rcp_refined(double x) {
  const double r0 = double(g_rcp(float(x)));
  return r0 * (2.0 - x * r0);
}

// ---- compensated binary32 (a pair hi + lo with |lo| <= ulp(hi) / 2) ----
// TwoSum (Knuth): s + e == a + b exactly.
GLC_HD void two_sum(float a, float b, float& s, float& e) {
  s = a + b;
  const float bv = s - a;
  e = (a - (s - bv)) + (b - bv);
}
// hi + lo += v, renormalized.
GLC_HD void ff_add(float& hi, float& lo, float v) {
  float s, e;
  two_sum(hi, v, s, e);
  e += lo;
  hi = s + e;
  lo = e - (hi - s);
}
// (ah + al)(bh + bl) as a pair; the al * bl term is below the pair's precision.
GLC_HD void ff_mul(float ah, float al, float bh, float bl, float& ph, float& pl) {
  const float p = ah * bh;
  const float e = fmaf(ah, bh, -p);
  pl = e + (ah * bl + al * bh);
  ph = p + pl;
  pl = pl - (ph - p);
}
// Cross-product component a1 b2 - a2 b1 of pairs, returned as a float accurate to its own scale.
GLC_HD float ff_cross(float a1h, float a1l, float b2h, float b2l, float a2h, float a2l, float b1h, float b1l) {
  float p1h, p1l, p2h, p2l;
  ff_mul(a1h, a1l, b2h, b2l, p1h, p1l);
  ff_mul(a2h, a2l, b1h, b1l, p2h, p2l);
  return (p1h - p2h) + (p1l - p2l);
}

}  // namespace glc
