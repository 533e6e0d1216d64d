// Oracle: CPU restatement of the Kerr-Newman Cartesian Kerr-Schild geometry in binary64.
//
// TEST INFRASTRUCTURE ONLY (see oracle_numerics.hpp).
//
// Follows crates/gravlume-domain/src/spacetime.rs step for step: scaled coordinates
// (spacetime.rs:637-712), the off-axis geometry with the full null-vector Jacobian
// (spacetime.rs:492-582), the axis branch (spacetime.rs:584-635), the canonical Hamilton
// right-hand side (spacetime.rs:305-338), invariants (spacetime.rs:345-386), the normalized null
// residual (spacetime.rs:393-401), radial velocity (spacetime.rs:408-414), the singularity-guard
// residual (spacetime.rs:437-451) and the exact outer horizon radius (spacetime.rs:227-238).
#pragma once

#include "oracle_numerics.hpp"

namespace gro {

enum class GeometryError : int { None = 0, NonFinite = 1, RingSingularity = 2, ChartBoundary = 3, InvalidDenominator = 4 };
enum class Extremality : int { Subextremal = 0, Extremal = 1, Superextremal = 2 };
enum class Chart : int { Ingoing = 0, Outgoing = 1 };

struct Geometry {
  double radius;
  double radius_gradient[3];
  double scalar_f;
  double scalar_f_gradient[3];
  double null_covector[4];
  double null_vector[4];
  double null_vector_gradient[3][4];
};

struct ScaledCoordinates {
  double scale, x, y, z, spin, radius_squared, radius, sigma;
  double singularity_measure() const {
    const double spin_squared = spin * spin;
    return positive_product(std::array<double, 5>{
        scale, scale, scale, scale, std::fma(radius_squared, radius_squared, spin_squared * z * z)});
  }
};

struct Invariants {
  double energy, angular_momentum_z, carter_constant, normalized_null_residual;
};

inline double dot4(const double a[4], const double b[4]) {
  // Rust `.sum()` over four products, left to right.
  double s = -0.0;
  for (int i = 0; i < 4; ++i) s += a[i] * b[i];
  return s;
}

struct Spacetime {
  double mass_m = 1.0, spin_m = 0.0, charge_m = 0.0;
  Chart chart = Chart::Ingoing;
  Extremality extremality = Extremality::Subextremal;

  double branch_sign() const { return chart == Chart::Ingoing ? 1.0 : -1.0; }

  // spacetime.rs:143-199 (validated_with_prefix); returns false on invalid input.
  static bool make(double m, double a, double q, Chart chart, Spacetime& out) {
    if (!std::isfinite(m) || m <= 0.0 || !std::isfinite(a) || !std::isfinite(q)) return false;
    out.mass_m = m;
    out.spin_m = a;
    out.charge_m = q;
    out.chart = chart;
    const int c = ExactBinary::square(m).compare(ExactBinary::sum_of_squares(a, q));
    out.extremality = c > 0 ? Extremality::Subextremal : (c == 0 ? Extremality::Extremal : Extremality::Superextremal);
    double rp;
    if (out.outer_horizon_radius(rp) && !std::isfinite(rp)) return false;
    return true;
  }

  // spacetime.rs:227-238
  bool outer_horizon_radius(double& r) const {
    switch (extremality) {
      case Extremality::Superextremal: return false;
      case Extremality::Extremal: r = mass_m; return true;
      default: {
        const ExactBinary m2 = ExactBinary::square(mass_m);
        const ExactBinary a2 = ExactBinary::sum_of_squares(spin_m, charge_m);
        r = mass_m + m2.subtract(a2).square_root();
        return true;
      }
    }
  }

  // spacetime.rs:245-254
  void oblate_to_cartesian(double radius, double polar, double azimuth, double out[3]) const {
    const double st = std::sin(polar), ct = std::cos(polar);
    const double sp = std::sin(azimuth), cp = std::cos(azimuth);
    const double cs = branch_sign() * spin_m;
    out[0] = std::fma(cs, -sp, radius * cp) * st;
    out[1] = std::fma(cs, cp, radius * sp) * st;
    out[2] = radius * ct;
  }

  // spacetime.rs:637-712
  GeometryError scaled_coordinates(const double txyz[4], ScaledCoordinates& s) const {
    const double px = txyz[1], py = txyz[2], pz = txyz[3];
    if (!std::isfinite(px) || !std::isfinite(py) || !std::isfinite(pz)) return GeometryError::NonFinite;
    const double scale = std::fmax(std::fmax(std::fmax(std::fabs(px), std::fabs(py)), std::fabs(pz)), std::fabs(spin_m));
    if (scale == 0.0) return GeometryError::RingSingularity;
    const double x = px / scale, y = py / scale, z = pz / scale;
    const double spin = spin_m / scale;
    const double spin_squared = spin * spin;
    if (px == 0.0 && py == 0.0 && pz != 0.0) {
      const double radius = std::fabs(z);
      const double radius_squared = radius * radius;
      const double sigma = radius_squared + spin_squared;
      if (radius > 0.0 && std::isfinite(sigma) && sigma > 0.0) {
        s = {scale, x, y, z, spin, radius_squared, radius, sigma};
        return GeometryError::None;
      }
    }
    const double r3 = std::fma(x, x, std::fma(y, y, z * z));
    const double b = r3 - spin_squared;
    const double disc = std::fma(b, b, 4.0 * spin_squared * z * z);
    if (!std::isfinite(disc) || disc < 0.0) return GeometryError::InvalidDenominator;
    const double root = std::sqrt(disc);
    double radius_squared;
    if (b >= 0.0) {
      radius_squared = 0.5 * (b + root);
    } else {
      const double denominator = root - b;
      if (denominator <= 0.0 || !std::isfinite(denominator)) return GeometryError::InvalidDenominator;
      radius_squared = 2.0 * spin_squared * z * z / denominator;
    }
    if (!std::isfinite(radius_squared)) return GeometryError::InvalidDenominator;
    if (radius_squared <= 0.0) return b == 0.0 ? GeometryError::RingSingularity : GeometryError::ChartBoundary;
    const double radius = std::sqrt(radius_squared);
    const double sigma = radius_squared + spin_squared * z * z / radius_squared;
    if (!std::isfinite(sigma) || sigma <= 0.0) return GeometryError::InvalidDenominator;
    s = {scale, x, y, z, spin, radius_squared, radius, sigma};
    return GeometryError::None;
  }

  static GeometryError validate(const Geometry& g) {
    bool ok = std::isfinite(g.scalar_f);
    for (int i = 0; i < 3; ++i) ok = ok && std::isfinite(g.radius_gradient[i]) && std::isfinite(g.scalar_f_gradient[i]);
    for (int i = 0; i < 4; ++i) ok = ok && std::isfinite(g.null_covector[i]);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 4; ++j) ok = ok && std::isfinite(g.null_vector_gradient[i][j]);
    return ok ? GeometryError::None : GeometryError::NonFinite;
  }

  // spacetime.rs:584-635
  GeometryError axis_geometry(const ScaledCoordinates& s, Geometry& g) const {
    const double scale = s.scale, z = s.z, spin = s.spin, r = s.radius, sigma = s.sigma;
    const double radius = scale * r;
    if (!std::isfinite(radius) || r <= 0.0 || sigma <= 0.0) return GeometryError::InvalidDenominator;
    const double axis_sign = std::signbit(z) ? -1.0 : 1.0;
    g.radius = radius;
    g.radius_gradient[0] = 0.0;
    g.radius_gradient[1] = 0.0;
    g.radius_gradient[2] = axis_sign;
    const double mass = mass_m / scale, charge = charge_m / scale;
    const double numerator = std::fma(-charge, charge, 2.0 * mass * r);
    g.scalar_f = numerator / sigma;
    const double sg[3] = {0.0, 0.0, 2.0 * r * axis_sign};
    for (int i = 0; i < 3; ++i) {
      const double ng = g.radius_gradient[i] * (2.0 * mass);
      g.scalar_f_gradient[i] = (ng * sigma - sg[i] * numerator) / (sigma * sigma * scale);
    }
    const double s_ = branch_sign();
    g.null_covector[0] = 1.0;
    g.null_covector[1] = 0.0;
    g.null_covector[2] = 0.0;
    g.null_covector[3] = s_ * axis_sign;
    g.null_vector[0] = -1.0;
    g.null_vector[1] = 0.0;
    g.null_vector[2] = 0.0;
    g.null_vector[3] = s_ * axis_sign;
    const double inv = (1.0 / sigma) / scale;
    const double row0[4] = {0.0, s_ * r * inv, -spin * inv, 0.0};
    const double row1[4] = {0.0, spin * inv, s_ * r * inv, 0.0};
    for (int j = 0; j < 4; ++j) {
      g.null_vector_gradient[0][j] = row0[j];
      g.null_vector_gradient[1][j] = row1[j];
      g.null_vector_gradient[2][j] = 0.0;
    }
    return validate(g);
  }

  // spacetime.rs:492-582
  GeometryError geometry(const double txyz[4], Geometry& g) const {
    ScaledCoordinates s;
    GeometryError e = scaled_coordinates(txyz, s);
    if (e != GeometryError::None) return e;
    if (s.x == 0.0 && s.y == 0.0) return axis_geometry(s, g);
    const double scale = s.scale, x = s.x, y = s.y, z = s.z, spin = s.spin;
    const double radius_squared = s.radius_squared, r = s.radius, sigma = s.sigma;
    const double radius = scale * r;
    if (!std::isfinite(radius)) return GeometryError::InvalidDenominator;
    const double spin_squared = spin * spin;
    const double rg[3] = {x * r / sigma, y * r / sigma, z * (radius_squared + spin_squared) / (r * sigma)};
    const double mass = mass_m / scale, charge = charge_m / scale;
    const double numerator = std::fma(-charge, charge, 2.0 * mass * r);
    const double scalar_f = numerator / sigma;
    const double vertical_sigma = spin_squared * z * z / radius_squared;
    const double srf = 2.0 * (r - vertical_sigma / r);
    const double sg[3] = {srf * rg[0], srf * rg[1], std::fma(srf, rg[2], 2.0 * spin_squared * z / radius_squared)};
    g.radius = radius;
    for (int i = 0; i < 3; ++i) g.radius_gradient[i] = rg[i];
    g.scalar_f = scalar_f;
    for (int i = 0; i < 3; ++i) {
      const double ng = rg[i] * (2.0 * mass);
      g.scalar_f_gradient[i] = (ng * sigma - sg[i] * numerator) / (sigma * sigma * scale);
    }
    const double rd = radius_squared + spin_squared;
    if (rd <= 0.0 || !std::isfinite(rd)) return GeometryError::InvalidDenominator;
    const double bs = branch_sign();
    const double cs = bs * spin;
    const double ns[3] = {bs * (std::fma(cs, y, r * x) / rd), bs * (std::fma(cs, -x, r * y) / rd), bs * (z / r)};
    g.null_covector[0] = 1.0;
    g.null_vector[0] = -1.0;
    for (int i = 0; i < 3; ++i) {
      g.null_covector[i + 1] = ns[i];
      g.null_vector[i + 1] = ns[i];
    }
    const double coords[3] = {x, y, z};
    for (int i = 0; i < 3; ++i) {
      const double ri = rg[i];
      const double dx = i == 0 ? 1.0 : 0.0, dy = i == 1 ? 1.0 : 0.0, dz = i == 2 ? 1.0 : 0.0;
      const double nx = std::fma(cs, dy, std::fma(ri, x, r * dx));
      const double ny = std::fma(cs, -dx, std::fma(ri, y, r * dy));
      const double radial_derivative = 2.0 * r * ri;
      const double der_x = std::fma(-bs * ns[0] * radial_derivative, 1.0 / rd, nx / rd) / scale;
      const double der_y = std::fma(-bs * ns[1] * radial_derivative, 1.0 / rd, ny / rd) / scale;
      const double der_z = (dz / r - coords[2] * ri / radius_squared) / scale;
      g.null_vector_gradient[i][0] = 0.0;
      g.null_vector_gradient[i][1] = bs * der_x;
      g.null_vector_gradient[i][2] = bs * der_y;
      g.null_vector_gradient[i][3] = bs * der_z;
    }
    return validate(g);
  }

  GeometryError radius(const double txyz[4], double& r) const {
    Geometry g;
    GeometryError e = geometry(txyz, g);
    if (e == GeometryError::None) r = g.radius;
    return e;
  }

  // spacetime.rs:305-338; state = (t, x, y, z, p_t, p_x, p_y, p_z)
  GeometryError hamiltonian_rhs(const double st[8], double d[8]) const {
    Geometry g;
    GeometryError e = geometry(st, g);
    if (e != GeometryError::None) return e;
    const double* p = st + 4;
    const double contraction = dot4(g.null_vector, p);
    const double mr[4] = {-p[0], p[1], p[2], p[3]};
    double v[4], md[3];
    for (int i = 0; i < 4; ++i) v[i] = std::fma(g.scalar_f * contraction, -g.null_vector[i], mr[i]);
    for (int i = 0; i < 3; ++i) {
      const double ndc = dot4(p, g.null_vector_gradient[i]);
      md[i] = std::fma(g.scalar_f * contraction, ndc, 0.5 * contraction * contraction * g.scalar_f_gradient[i]);
    }
    const double out[8] = {v[0], v[1], v[2], v[3], 0.0, md[0], md[1], md[2]};
    for (int i = 0; i < 8; ++i) {
      if (!std::isfinite(out[i])) return GeometryError::NonFinite;
    }
    for (int i = 0; i < 8; ++i) d[i] = out[i];
    return GeometryError::None;
  }

  static void metric_inverse(const Geometry& g, double m[4][4]) {
    for (int r = 0; r < 4; ++r)
      for (int c = 0; c < 4; ++c) {
        const double mink = r == c ? (r == 0 ? -1.0 : 1.0) : 0.0;
        m[r][c] = std::fma(-g.scalar_f * g.null_vector[r], g.null_vector[c], mink);
      }
  }
  static void metric_covariant(const Geometry& g, double m[4][4]) {
    for (int r = 0; r < 4; ++r)
      for (int c = 0; c < 4; ++c) {
        const double mink = r == c ? (r == 0 ? -1.0 : 1.0) : 0.0;
        m[r][c] = std::fma(g.scalar_f * g.null_covector[r], g.null_covector[c], mink);
      }
  }

  // spacetime.rs:393-401
  GeometryError normalized_null_residual(const double st[8], double& out) const {
    Geometry g;
    GeometryError e = geometry(st, g);
    if (e != GeometryError::None) return e;
    double m[4][4];
    metric_inverse(g, m);
    const double res = normalized_quadratic_form_residual(m, st + 4);
    if (!std::isfinite(res)) return GeometryError::NonFinite;
    out = res;
    return GeometryError::None;
  }

  // spacetime.rs:345-386
  GeometryError invariants(const double st[8], Invariants& inv) const {
    double radius;
    GeometryError e = this->radius(st, radius);
    if (e != GeometryError::None) return e;
    const double x = st[1], y = st[2], z = st[3];
    const double* p = st + 4;
    const double energy = -p[0];
    const double lz = std::fma(y, -p[1], x * p[2]);
    const double rho = std::hypot(x, y);
    const double spin_squared = spin_m * spin_m;
    double carter;
    if (rho == 0.0) {
      const double tps = std::fma(p[1], p[1], p[2] * p[2]);
      const double leading = std::fma(radius, radius, spin_squared) * tps;
      carter = std::fma(-spin_squared * energy, energy, leading);
    } else {
      const double ct = z / radius;
      const double stt = rho / std::sqrt(std::fma(radius, radius, spin_squared));
      const double proj = std::fma(x, p[1], y * p[2]);
      const double p_theta = std::fma(-radius * stt, p[3], (ct / stt) * proj);
      const double lzs = lz / stt;
      const double angular = std::fma(-spin_squared * energy, energy, lzs * lzs);
      carter = std::fma(ct * ct, angular, p_theta * p_theta);
    }
    double nr;
    e = normalized_null_residual(st, nr);
    if (e != GeometryError::None) return e;
    if (!std::isfinite(energy) || !std::isfinite(lz) || !std::isfinite(carter) || !std::isfinite(nr))
      return GeometryError::NonFinite;
    inv = {energy, lz, carter, nr};
    return GeometryError::None;
  }

  // spacetime.rs:408-414
  GeometryError radial_velocity(const double st[8], double& out) const {
    Geometry g;
    GeometryError e = geometry(st, g);
    if (e != GeometryError::None) return e;
    double d[8];
    e = hamiltonian_rhs(st, d);
    if (e != GeometryError::None) return e;
    out = g.radius_gradient[0] * d[1] + g.radius_gradient[1] * d[2] + g.radius_gradient[2] * d[3];
    return GeometryError::None;
  }

  // spacetime.rs:437-451
  GeometryError singularity_guard_residual(const double txyz[4], double guard, double& out) const {
    if (!std::isfinite(guard) || guard <= 0.0) return GeometryError::InvalidDenominator;
    ScaledCoordinates s;
    GeometryError e = scaled_coordinates(txyz, s);
    if (e != GeometryError::None) return e;
    const double m = s.singularity_measure();
    out = std::isinf(m) ? std::numeric_limits<double>::max() : m - guard;
    return GeometryError::None;
  }

  // spacetime.rs:463-483 metric_dot_and_term_norm
  GeometryError metric_dot_and_term_norm(const double txyz[4], const double l[4], const double r[4], double& sum,
                                         double& norm) const {
    Geometry g;
    GeometryError e = geometry(txyz, g);
    if (e != GeometryError::None) return e;
    double m[4][4];
    metric_covariant(g, m);
    sum = 0.0;
    norm = 0.0;
    for (int row = 0; row < 4; ++row)
      for (int col = 0; col < 4; ++col) {
        const double term = m[row][col] * l[row] * r[col];
        sum = sum + term;
        norm = norm + std::fabs(term);
      }
    if (!std::isfinite(sum) || !std::isfinite(norm)) return GeometryError::NonFinite;
    return GeometryError::None;
  }
};

}  // namespace gro
