// Forward-mode dual numbers with N tangent channels, for the Jacobians the discrete adjoint needs
// (right-hand side, radius, event functions and observables). Overloads of the precision helpers
// (g_sqrt, g_rcp, ...) live in this namespace, so the geometry templates (kn_rhs, kn_radius,
// frequency_ratio) instantiate on Dual<N> unchanged.
#pragma once

#include "glc_geometry.cuh"

namespace glc {

template <int N>
struct Dual {
  double v;
  double d[N];
  GLC_HD Dual() : v(0.0) {
#pragma unroll
    for (int i = 0; i < N; ++i) d[i] = 0.0;
  }
  GLC_HD Dual(double x) : v(x) {
#pragma unroll
    for (int i = 0; i < N; ++i) d[i] = 0.0;
  }
  // value x with unit tangent on channel i
  static GLC_HD Dual seed(double x, int i) {
    Dual r(x);
    r.d[i] = 1.0;
    return r;
  }
  GLC_HD Dual& operator+=(const Dual& b) {
    v += b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) d[i] += b.d[i];
    return *this;
  }
  GLC_HD Dual& operator-=(const Dual& b) {
    v -= b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) d[i] -= b.d[i];
    return *this;
  }
  GLC_HD Dual& operator*=(const Dual& b) {
#pragma unroll
    for (int i = 0; i < N; ++i) d[i] = d[i] * b.v + v * b.d[i];
    v *= b.v;
    return *this;
  }
};

// chain rule helper: f(a) with value fv and derivative df
template <int N>
GLC_HD Dual<N> dual_apply(const Dual<N>& a, double fv, double df) {
  Dual<N> r(fv);
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = df * a.d[i];
  return r;
}

template <int N>
GLC_HD Dual<N> operator+(Dual<N> a, const Dual<N>& b) {
  a += b;
  return a;
}
template <int N>
GLC_HD Dual<N> operator-(Dual<N> a, const Dual<N>& b) {
  a -= b;
  return a;
}
template <int N>
GLC_HD Dual<N> operator*(Dual<N> a, const Dual<N>& b) {
  a *= b;
  return a;
}
template <int N>
GLC_HD Dual<N> operator-(const Dual<N>& a) {
  return dual_apply(a, -a.v, -1.0);
}
template <int N>
GLC_HD Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
  const double q = a.v / b.v;
  Dual<N> r(q);
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - q * b.d[i]) / b.v;
  return r;
}
template <int N>
GLC_HD Dual<N> operator+(const Dual<N>& a, double b) { return a + Dual<N>(b); }
template <int N>
GLC_HD Dual<N> operator+(double a, const Dual<N>& b) { return Dual<N>(a) + b; }
template <int N>
GLC_HD Dual<N> operator-(const Dual<N>& a, double b) { return a - Dual<N>(b); }
template <int N>
GLC_HD Dual<N> operator-(double a, const Dual<N>& b) { return Dual<N>(a) - b; }
template <int N>
GLC_HD Dual<N> operator*(const Dual<N>& a, double b) { return dual_apply(a, a.v * b, b); }
template <int N>
GLC_HD Dual<N> operator*(double a, const Dual<N>& b) { return dual_apply(b, a * b.v, a); }
template <int N>
GLC_HD Dual<N> operator/(const Dual<N>& a, double b) { return dual_apply(a, a.v / b, 1.0 / b); }
template <int N>
GLC_HD Dual<N> operator/(double a, const Dual<N>& b) { return Dual<N>(a) / b; }

template <int N>
GLC_HD bool operator<(const Dual<N>& a, const Dual<N>& b) { return a.v < b.v; }
template <int N>
GLC_HD bool operator>(const Dual<N>& a, const Dual<N>& b) { return a.v > b.v; }
template <int N>
GLC_HD bool operator<=(const Dual<N>& a, const Dual<N>& b) { return a.v <= b.v; }
template <int N>
GLC_HD bool operator>=(const Dual<N>& a, const Dual<N>& b) { return a.v >= b.v; }
template <int N>
GLC_HD bool operator==(const Dual<N>& a, const Dual<N>& b) { return a.v == b.v; }
template <int N>
GLC_HD bool operator!=(const Dual<N>& a, const Dual<N>& b) { return a.v != b.v; }

template <int N>
GLC_HD Dual<N> g_sqrt(const Dual<N>& a) {
  const double s = g_sqrt(a.v);
  return dual_apply(a, s, 0.5 / s);
}
template <int N>
GLC_HD Dual<N> g_rcp(const Dual<N>& a) {
  const double r = 1.0 / a.v;
  return dual_apply(a, r, -r * r);
}
template <int N>
GLC_HD Dual<N> g_rsqrt(const Dual<N>& a) {
  const double r = 1.0 / g_sqrt(a.v);
  return dual_apply(a, r, -0.5 * r * r * r);
}
template <int N>
GLC_HD Dual<N> g_abs(const Dual<N>& a) {
  return a.v < 0.0 ? -a : a;
}
template <int N>
GLC_HD Dual<N> g_min(const Dual<N>& a, const Dual<N>& b) {
  return b.v < a.v ? b : a;
}
template <int N>
GLC_HD Dual<N> g_max(const Dual<N>& a, const Dual<N>& b) {
  return b.v > a.v ? b : a;
}
template <int N>
GLC_HD bool g_finite(const Dual<N>& a) {
  return g_finite(a.v);
}
template <int N>
GLC_HD Dual<N> g_acos(const Dual<N>& a) {
  return dual_apply(a, g_acos(a.v), -1.0 / g_sqrt(1.0 - a.v * a.v));
}
template <int N>
GLC_HD Dual<N> g_atan2(const Dual<N>& y, const Dual<N>& x) {
  const double den = x.v * x.v + y.v * y.v;
  Dual<N> r(g_atan2(y.v, x.v));
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = (x.v * y.d[i] - y.v * x.d[i]) / den;
  return r;
}
template <int N>
GLC_HD Dual<N> g_hypot(const Dual<N>& a, const Dual<N>& b) {
  return g_sqrt(a * a + b * b);
}

}  // namespace glc
