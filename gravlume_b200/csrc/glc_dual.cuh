// Forward-mode dual numbers with N tangent channels over the scalar type R (binary64 by default),
// for the Jacobians the discrete adjoint and the footprint tangents need (right-hand side, radius,
// event functions and observables). Overloads of the precision helpers (g_sqrt, g_rcp, ...) live
// in this namespace, so the geometry templates (kn_rhs, kn_radius, frequency_ratio) instantiate on
// Dual<N, R> unchanged. Scalars enter as double and are rounded to R.
#pragma once

#include "glc_geometry.cuh"

namespace glc {

template <int N, class R = double>
struct Dual {
  R v;
  R d[N];
  GLC_HD Dual() : v(R(0)) {
#pragma unroll
    for (int i = 0; i < N; ++i) d[i] = R(0);
  }
  GLC_HD Dual(double x) : v(R(x)) {
#pragma unroll
    for (int i = 0; i < N; ++i) d[i] = R(0);
  }
  // value x with unit tangent on channel i
  static GLC_HD Dual seed(double x, int i) {
    Dual r(x);
    r.d[i] = R(1);
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
template <int N, class R>
GLC_HD Dual<N, R> dual_apply(const Dual<N, R>& a, R fv, R df) {
  Dual<N, R> r;
  r.v = fv;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = df * a.d[i];
  return r;
}

template <int N, class R>
GLC_HD Dual<N, R> operator+(Dual<N, R> a, const Dual<N, R>& b) {
  a += b;
  return a;
}
template <int N, class R>
GLC_HD Dual<N, R> operator-(Dual<N, R> a, const Dual<N, R>& b) {
  a -= b;
  return a;
}
template <int N, class R>
GLC_HD Dual<N, R> operator*(Dual<N, R> a, const Dual<N, R>& b) {
  a *= b;
  return a;
}
template <int N, class R>
GLC_HD Dual<N, R> operator-(const Dual<N, R>& a) {
  return dual_apply(a, -a.v, R(-1));
}
template <int N, class R>
GLC_HD Dual<N, R> operator/(const Dual<N, R>& a, const Dual<N, R>& b) {
  const R q = a.v / b.v;
  Dual<N, R> r;
  r.v = q;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - q * b.d[i]) / b.v;
  return r;
}
template <int N, class R>
GLC_HD Dual<N, R> operator+(const Dual<N, R>& a, double b) { return a + Dual<N, R>(b); }
template <int N, class R>
GLC_HD Dual<N, R> operator+(double a, const Dual<N, R>& b) { return Dual<N, R>(a) + b; }
template <int N, class R>
GLC_HD Dual<N, R> operator-(const Dual<N, R>& a, double b) { return a - Dual<N, R>(b); }
template <int N, class R>
GLC_HD Dual<N, R> operator-(double a, const Dual<N, R>& b) { return Dual<N, R>(a) - b; }
template <int N, class R>
GLC_HD Dual<N, R> operator*(const Dual<N, R>& a, double b) { return dual_apply(a, a.v * R(b), R(b)); }
template <int N, class R>
GLC_HD Dual<N, R> operator*(double a, const Dual<N, R>& b) { return dual_apply(b, R(a) * b.v, R(a)); }
template <int N, class R>
GLC_HD Dual<N, R> operator/(const Dual<N, R>& a, double b) { return dual_apply(a, a.v / R(b), R(1) / R(b)); }
template <int N, class R>
GLC_HD Dual<N, R> operator/(double a, const Dual<N, R>& b) { return Dual<N, R>(a) / b; }

template <int N, class R>
GLC_HD bool operator<(const Dual<N, R>& a, const Dual<N, R>& b) { return a.v < b.v; }
template <int N, class R>
GLC_HD bool operator>(const Dual<N, R>& a, const Dual<N, R>& b) { return a.v > b.v; }
template <int N, class R>
GLC_HD bool operator<=(const Dual<N, R>& a, const Dual<N, R>& b) { return a.v <= b.v; }
template <int N, class R>
GLC_HD bool operator>=(const Dual<N, R>& a, const Dual<N, R>& b) { return a.v >= b.v; }
template <int N, class R>
GLC_HD bool operator==(const Dual<N, R>& a, const Dual<N, R>& b) { return a.v == b.v; }
template <int N, class R>
GLC_HD bool operator!=(const Dual<N, R>& a, const Dual<N, R>& b) { return a.v != b.v; }

template <int N, class R>
GLC_HD Dual<N, R> g_sqrt(const Dual<N, R>& a) {
  const R s = g_sqrt(a.v);
  return dual_apply(a, s, R(0.5) / s);
}
template <int N, class R>
GLC_HD Dual<N, R> g_rcp(const Dual<N, R>& a) {
  const R r = R(1) / a.v;
  return dual_apply(a, r, -r * r);
}
template <int N, class R>
GLC_HD Dual<N, R> g_rsqrt(const Dual<N, R>& a) {
  const R r = R(1) / g_sqrt(a.v);
  return dual_apply(a, r, R(-0.5) * r * r * r);
}
template <int N, class R>
GLC_HD Dual<N, R> g_abs(const Dual<N, R>& a) {
  return a.v < R(0) ? -a : a;
}
template <int N, class R>
GLC_HD Dual<N, R> g_min(const Dual<N, R>& a, const Dual<N, R>& b) {
  return b.v < a.v ? b : a;
}
template <int N, class R>
GLC_HD Dual<N, R> g_max(const Dual<N, R>& a, const Dual<N, R>& b) {
  return b.v > a.v ? b : a;
}
template <int N, class R>
GLC_HD bool g_finite(const Dual<N, R>& a) {
  return g_finite(a.v);
}
template <int N, class R>
GLC_HD Dual<N, R> g_acos(const Dual<N, R>& a) {
  return dual_apply(a, g_acos(a.v), R(-1) / g_sqrt(R(1) - a.v * a.v));
}
template <int N, class R>
GLC_HD Dual<N, R> g_atan2(const Dual<N, R>& y, const Dual<N, R>& x) {
  const R den = x.v * x.v + y.v * y.v;
  Dual<N, R> r;
  r.v = g_atan2(y.v, x.v);
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = (x.v * y.d[i] - y.v * x.d[i]) / den;
  return r;
}
template <int N, class R>
GLC_HD Dual<N, R> g_hypot(const Dual<N, R>& a, const Dual<N, R>& b) {
  return g_sqrt(a * a + b * b);
}

}  // namespace glc
