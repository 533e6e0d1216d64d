// TEST INFRASTRUCTURE ONLY (the checker of the adjoint's gradients; the product never uses it).
//
// Binary64 variational-equation reference for per-ray gradients. The oracle traces a ray with its
// own adaptive DP5(4) loop (oracle_tracer.hpp, after crates/gravlume-reference/src/integrator.rs
// 153-190 and geodesic.rs:129-212) and records the signed size of every accepted step. The same
// steps are then replayed on the state augmented with its sensitivities: every quantity carries
// its derivatives with respect to the initial covariant momentum (p_t, p_x, p_y, p_z) and to the
// spin a and charge Q in the dynamics (forward-mode dual numbers). For an explicit Runge-Kutta
// method with frozen step sizes this is the variational equation Phi' = (df/dy) Phi + df/dtheta
// integrated by the same tableau, i.e. the exact derivative of the discrete trace. The terminal
// event time follows from the implicit-function rule on the terminal step's dense output,
// dtheta*/dp = -(dg/dy . dy/dp) / (dg/dy . dy/dtheta), so the observables at the event (source
// radius and g at the surface, escape polar angle and azimuth at the escape sphere) get total
// derivatives. The right-hand side and the surface observable are restated here for a generic
// scalar from the oracle's binary64 code (Spacetime::geometry / hamiltonian_rhs, spacetime.rs
// 492-582 and 305-338; surface_radius_and_frequency_ratio, surface.rs:75-146).
#pragma once

#include <cmath>
#include <vector>

#include "oracle_tracer.hpp"

namespace gro {

// ---------------------------------------------------------------- dual numbers
template <int M>
struct Dual {
  double v;
  double d[M];
  Dual() : v(0.0) {
    for (int i = 0; i < M; ++i) d[i] = 0.0;
  }
  Dual(double x) : v(x) {  // NOLINT: constants promote implicitly
    for (int i = 0; i < M; ++i) d[i] = 0.0;
  }
  static Dual seed(double x, int k) {
    Dual r(x);
    r.d[k] = 1.0;
    return r;
  }
};

template <int M>
inline Dual<M> operator+(const Dual<M>& a, const Dual<M>& b) {
  Dual<M> r(a.v + b.v);
  for (int i = 0; i < M; ++i) r.d[i] = a.d[i] + b.d[i];
  return r;
}
template <int M>
inline Dual<M> operator-(const Dual<M>& a, const Dual<M>& b) {
  Dual<M> r(a.v - b.v);
  for (int i = 0; i < M; ++i) r.d[i] = a.d[i] - b.d[i];
  return r;
}
template <int M>
inline Dual<M> operator-(const Dual<M>& a) {
  Dual<M> r(-a.v);
  for (int i = 0; i < M; ++i) r.d[i] = -a.d[i];
  return r;
}
template <int M>
inline Dual<M> operator*(const Dual<M>& a, const Dual<M>& b) {
  Dual<M> r(a.v * b.v);
  for (int i = 0; i < M; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
template <int M>
inline Dual<M> operator/(const Dual<M>& a, const Dual<M>& b) {
  const double q = a.v / b.v;
  Dual<M> r(q);
  for (int i = 0; i < M; ++i) r.d[i] = (a.d[i] - q * b.d[i]) / b.v;
  return r;
}
template <int M> inline Dual<M> operator+(const Dual<M>& a, double b) { return a + Dual<M>(b); }
template <int M> inline Dual<M> operator+(double a, const Dual<M>& b) { return Dual<M>(a) + b; }
template <int M> inline Dual<M> operator-(const Dual<M>& a, double b) { return a - Dual<M>(b); }
template <int M> inline Dual<M> operator-(double a, const Dual<M>& b) { return Dual<M>(a) - b; }
template <int M> inline Dual<M> operator*(const Dual<M>& a, double b) {
  Dual<M> r(a.v * b);
  for (int i = 0; i < M; ++i) r.d[i] = a.d[i] * b;
  return r;
}
template <int M> inline Dual<M> operator*(double a, const Dual<M>& b) { return b * a; }
template <int M> inline Dual<M> operator/(const Dual<M>& a, double b) { return a / Dual<M>(b); }
template <int M> inline Dual<M> operator/(double a, const Dual<M>& b) { return Dual<M>(a) / b; }

inline double value(double x) { return x; }
template <int M> inline double value(const Dual<M>& x) { return x.v; }

inline double vsqrt(double x) { return std::sqrt(x); }
template <int M>
inline Dual<M> vsqrt(const Dual<M>& a) {
  const double s = std::sqrt(a.v);
  Dual<M> r(s);
  for (int i = 0; i < M; ++i) r.d[i] = a.d[i] / (2.0 * s);
  return r;
}
inline double vfabs(double x) { return std::fabs(x); }
template <int M> inline Dual<M> vfabs(const Dual<M>& a) { return a.v < 0.0 ? -a : a; }
inline double vacos(double x) { return std::acos(x); }
template <int M>
inline Dual<M> vacos(const Dual<M>& a) {
  Dual<M> r(std::acos(a.v));
  const double k = -1.0 / std::sqrt(1.0 - a.v * a.v);
  for (int i = 0; i < M; ++i) r.d[i] = k * a.d[i];
  return r;
}
inline double vatan2(double y, double x) { return std::atan2(y, x); }
template <int M>
inline Dual<M> vatan2(const Dual<M>& y, const Dual<M>& x) {
  Dual<M> r(std::atan2(y.v, x.v));
  const double n = x.v * x.v + y.v * y.v;
  for (int i = 0; i < M; ++i) r.d[i] = (x.v * y.d[i] - y.v * x.d[i]) / n;
  return r;
}
template <class T> inline T vfma(const T& a, const T& b, const T& c) { return a * b + c; }
inline double vfma(double a, double b, double c) { return std::fma(a, b, c); }

// ---------------------------------------------------------------- geometry for a generic scalar
template <class T>
struct GeometryT {
  T radius;
  T radius_gradient[3];
  T scalar_f;
  T scalar_f_gradient[3];
  T null_vector[4];
  T null_vector_gradient[3][4];
};

// Spacetime::geometry (spacetime.rs:492-582) off the spin axis, with spin and charge as scalars of
// type T (mass 1 in the oracle's units is passed as `mass`); returns false where the oracle takes
// its axis branch or meets a singular denominator.
template <class T>
bool geometry_t(double mass_m, const T& spin_m, const T& charge_m, double branch_sign, const T txyz[4],
                GeometryT<T>& g) {
  const T px = txyz[1], py = txyz[2], pz = txyz[3];
  // the oracle's scale: the largest magnitude of the coordinates and the spin (a normalization
  // that cancels, so its derivative may follow whichever argument is largest)
  T scale = vfabs(px);
  if (vfabs(py).v > scale.v) scale = vfabs(py);
  if (vfabs(pz).v > scale.v) scale = vfabs(pz);
  if (vfabs(spin_m).v > scale.v) scale = vfabs(spin_m);
  if (!(scale.v > 0.0)) return false;
  const T x = px / scale, y = py / scale, z = pz / scale;
  if (x.v == 0.0 && y.v == 0.0) return false;
  const T spin = spin_m / scale;
  const T spin_squared = spin * spin;
  const T r3 = x * x + (y * y + z * z);
  const T b = r3 - spin_squared;
  const T disc = b * b + 4.0 * spin_squared * z * z;
  if (!(disc.v >= 0.0)) return false;
  const T root = vsqrt(disc);
  T radius_squared;
  if (b.v >= 0.0) {
    radius_squared = 0.5 * (b + root);
  } else {
    const T den = root - b;
    if (!(den.v > 0.0)) return false;
    radius_squared = 2.0 * spin_squared * z * z / den;
  }
  if (!(radius_squared.v > 0.0)) return false;
  const T r = vsqrt(radius_squared);
  const T sigma = radius_squared + spin_squared * z * z / radius_squared;
  if (!(sigma.v > 0.0)) return false;
  const T rg[3] = {x * r / sigma, y * r / sigma, z * (radius_squared + spin_squared) / (r * sigma)};
  const T mass = mass_m / scale, charge = charge_m / scale;
  const T numerator = 2.0 * mass * r - charge * charge;
  const T vertical_sigma = spin_squared * z * z / radius_squared;
  const T srf = 2.0 * (r - vertical_sigma / r);
  const T sg[3] = {srf * rg[0], srf * rg[1], srf * rg[2] + 2.0 * spin_squared * z / radius_squared};
  g.radius = scale * r;
  for (int i = 0; i < 3; ++i) g.radius_gradient[i] = rg[i];
  g.scalar_f = numerator / sigma;
  for (int i = 0; i < 3; ++i) {
    const T ng = rg[i] * (2.0 * mass);
    g.scalar_f_gradient[i] = (ng * sigma - sg[i] * numerator) / (sigma * sigma * scale);
  }
  const T rd = radius_squared + spin_squared;
  if (!(rd.v > 0.0)) return false;
  const double bs = branch_sign;
  const T cs = bs * spin;
  const T ns[3] = {bs * ((cs * y + r * x) / rd), bs * ((r * y - cs * x) / rd), bs * (z / r)};
  g.null_vector[0] = T(-1.0);
  for (int i = 0; i < 3; ++i) g.null_vector[i + 1] = ns[i];
  const T coords[3] = {x, y, z};
  for (int i = 0; i < 3; ++i) {
    const T ri = rg[i];
    const double dx = i == 0 ? 1.0 : 0.0, dy = i == 1 ? 1.0 : 0.0, dz = i == 2 ? 1.0 : 0.0;
    const T nx = cs * dy + (ri * x + r * dx);
    const T ny = cs * (-dx) + (ri * y + r * dy);
    const T radial_derivative = 2.0 * r * ri;
    const T der_x = ((-bs) * ns[0] * radial_derivative / rd + nx / rd) / scale;
    const T der_y = ((-bs) * ns[1] * radial_derivative / rd + ny / rd) / scale;
    const T der_z = (dz / r - coords[2] * ri / radius_squared) / scale;
    g.null_vector_gradient[i][0] = T(0.0);
    g.null_vector_gradient[i][1] = bs * der_x;
    g.null_vector_gradient[i][2] = bs * der_y;
    g.null_vector_gradient[i][3] = bs * der_z;
  }
  return true;
}

// Spacetime::hamiltonian_rhs (spacetime.rs:305-338) for a generic scalar; state = (t, x, y, z, p_t,
// p_x, p_y, p_z).
template <class T>
bool hamiltonian_rhs_t(double mass_m, const T& spin_m, const T& charge_m, double branch_sign, const T st[8], T d[8]) {
  GeometryT<T> g;
  if (!geometry_t(mass_m, spin_m, charge_m, branch_sign, st, g)) return false;
  const T* p = st + 4;
  const T contraction = g.null_vector[0] * p[0] + g.null_vector[1] * p[1] + g.null_vector[2] * p[2] +
                        g.null_vector[3] * p[3];
  const T mr[4] = {-p[0], p[1], p[2], p[3]};
  const T fc = g.scalar_f * contraction;
  for (int i = 0; i < 4; ++i) d[i] = mr[i] - fc * g.null_vector[i];
  d[4] = T(0.0);
  for (int i = 0; i < 3; ++i) {
    const T ndc = p[0] * g.null_vector_gradient[i][0] + p[1] * g.null_vector_gradient[i][1] +
                  p[2] * g.null_vector_gradient[i][2] + p[3] * g.null_vector_gradient[i][3];
    d[5 + i] = fc * ndc + 0.5 * contraction * contraction * g.scalar_f_gradient[i];
  }
  for (int i = 0; i < 8; ++i)
    if (!std::isfinite(value(d[i]))) return false;
  return true;
}

// surface_radius_and_frequency_ratio (surface.rs:75-146) for a generic scalar: g of the prograde
// Keplerian emitter at the state's radius (no interval test: the base trace decided the hit).
template <class T>
bool frequency_ratio_t(double mass_m, const T& a, const T& charge, const T& radius, const T st[8],
                       double observer_frequency, T& ratio) {
  const double m = mass_m;
  const T q2 = charge * charge;
  const T crs = m * radius - q2;
  if (!(crs.v >= 0.0)) return false;
  const T cr = vsqrt(crs);
  const double bs = a.v < 0.0 ? -1.0 : 1.0;
  const T r2 = radius * radius;
  const T avd = bs * a * cr + r2;
  if (!(avd.v > 0.0)) return false;
  const T omega = bs * cr / avd;
  const T rn = 2.0 * m * radius - q2;
  const T a2 = a * a;
  const T tdisc = -3.0 * m * radius + (2.0 * bs * a * cr + (2.0 * q2 + r2));
  if (!(tdisc.v > 0.0)) return false;
  const T delta = r2 + ((-2.0 * m) * radius + (a2 + q2));
  const T gtt = -1.0 + rn / r2;
  const T gtp = -rn * a / r2;
  const T rf = r2 + a2;
  const T gpp = (rf * rf - a2 * delta) / r2;
  const T cn2 = omega * (omega * gpp) + (2.0 * gtp * omega + gtt);
  if (!(cn2.v < 0.0)) return false;
  const T tc = 1.0 / vsqrt(-cn2);
  const T energy = -st[4];
  const T lz = st[1] * st[6] - st[2] * st[5];
  const T ef = tc * (energy - omega * lz);
  if (!(ef.v > 0.0)) return false;
  ratio = observer_frequency / ef;
  return ratio.v > 0.0;
}

// ---------------------------------------------------------------- the reference gradient
// Per-ray observables and their gradients: obs[4] = source radius, g, escape polar angle, escape
// azimuth (NaN where not applicable); grad[6][4] = d(obs)/d(p_t, p_x, p_y, p_z, a, Q). Returns the
// termination of the base trace and whether the gradient is defined (a surface hit with its
// observable, or an escape with its direction, through a localized event).
constexpr int kVarParams = 6;
using VD = Dual<kVarParams>;

inline bool variational_gradient(const Tracer& base, const double initial[8], double sign, Termination& term,
                                 double obs[4], double grad[kVarParams][4]) {
  for (int k = 0; k < 4; ++k) obs[k] = NAN;
  for (int p = 0; p < kVarParams; ++p)
    for (int k = 0; k < 4; ++k) grad[p][k] = 0.0;
  std::vector<double> steps;
  const Outcome o = base.trace(initial, sign, &steps, nullptr);
  term = o.termination;
  const bool surface = o.termination == Termination::EquatorialSurface;
  const bool escape = o.termination == Termination::Escape && o.has_escape_direction;
  if ((!surface && !escape) || steps.empty()) return false;
  const Spacetime& sp = base.sp;
  const double bs = sp.branch_sign();
  const VD spin = VD::seed(sp.spin_m, 4), charge = VD::seed(sp.charge_m, 5);
  VD y[8];
  for (int c = 0; c < 8; ++c) y[c] = VD(initial[c]);
  for (int c = 0; c < 4; ++c) y[4 + c] = VD::seed(initial[4 + c], c);
  VD stages[7][8];
  if (!hamiltonian_rhs_t(sp.mass_m, spin, charge, bs, y, stages[0])) return false;
  const size_t last = steps.size() - 1;
  for (size_t k = 0; k <= last; ++k) {
    const double h = steps[k];
    for (int s = 1; s < 7; ++s) {
      VD ss[8];
      for (int c = 0; c < 8; ++c) {
        VD w(-0.0);
        for (int j = 0; j < s; ++j) w = w + tableau::A[s][j] * stages[j][c];
        ss[c] = h * w + y[c];
      }
      if (!hamiltonian_rhs_t(sp.mass_m, spin, charge, bs, ss, stages[s])) return false;
    }
    if (k < last) {
      for (int c = 0; c < 8; ++c) {
        VD w(-0.0);
        for (int j = 0; j < 7; ++j) w = w + tableau::B5[j] * stages[j][c];
        y[c] = h * w + y[c];
      }
      for (int c = 0; c < 8; ++c) stages[0][c] = stages[6][c];
      continue;
    }
    // terminal step: the event on the dense output at the base trace's theta
    const double th = o.event_theta;
    double pw[4], dpw[4];
    DenseOutput::powers(th, pw);
    dpw[0] = 1.0;
    dpw[1] = 2.0 * th;
    dpw[2] = 3.0 * th * th;
    dpw[3] = 4.0 * th * th * th;
    VD ye[8];
    double ydot[8];
    for (int c = 0; c < 8; ++c) {
      VD s(-0.0);
      double sd = 0.0;
      for (int j = 0; j < 7; ++j) {
        double cj = 0.0, cdj = 0.0;
        for (int q = 0; q < 4; ++q) {
          cj += tableau::D[j][q] * pw[q];
          cdj += tableau::D[j][q] * dpw[q];
        }
        s = s + cj * stages[j][c];
        sd += cdj * stages[j][c].v;
      }
      ye[c] = h * s + y[c];
      ydot[c] = h * sd;
    }
    // event function g(y): z on the surface, r - R at the escape sphere; dg/dtheta along the dense output
    VD gv;
    double gdot;
    if (surface) {
      gv = ye[3];
      gdot = ydot[3];
    } else {
      GeometryT<VD> gg;
      if (!geometry_t(sp.mass_m, spin, charge, bs, ye, gg)) return false;
      gv = gg.radius;
      gdot = gg.radius_gradient[0].v * ydot[1] + gg.radius_gradient[1].v * ydot[2] + gg.radius_gradient[2].v * ydot[3];
    }
    if (!(std::fabs(gdot) > 0.0)) return false;
    for (int c = 0; c < 8; ++c)
      for (int p = 0; p < kVarParams; ++p) ye[c].d[p] -= ydot[c] * gv.d[p] / gdot;
    for (int c = 0; c < 8; ++c) y[c] = ye[c];
  }
  VD out[4];
  if (surface) {
    GeometryT<VD> gg;
    if (!geometry_t(sp.mass_m, spin, charge, bs, y, gg)) return false;
    VD ratio;
    if (!frequency_ratio_t(sp.mass_m, spin, charge, gg.radius, y, 1.0, ratio)) return false;
    out[0] = gg.radius;
    out[1] = ratio;
    out[2] = out[3] = VD(0.0);
  } else {
    VD d[8];
    if (!hamiltonian_rhs_t(sp.mass_m, spin, charge, bs, y, d)) return false;
    const VD dir[3] = {sign * d[1], sign * d[2], sign * d[3]};
    const VD n = vsqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
    out[0] = out[1] = VD(0.0);
    out[2] = vacos(dir[2] / n);
    out[3] = vatan2(dir[1], dir[0]);
  }
  for (int k = 0; k < 4; ++k) {
    const bool used = surface ? k < 2 : k >= 2;
    obs[k] = used ? out[k].v : NAN;
    for (int p = 0; p < kVarParams; ++p) grad[p][k] = used ? out[k].d[p] : 0.0;
  }
  return true;
}

}  // namespace gro
