// Oracle: CPU restatement of Gravlume's binary64 numerics helpers.
//
// TEST INFRASTRUCTURE ONLY. This directory is the checker for the CUDA trace path: only
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it. Nothing in the
// product (gravlume_b200/) links, imports or calls it.
//
// Follows crates/gravlume-domain/src/numerics.rs (term-normalized residuals, exact binary
// decomposition) and crates/gravlume-domain/src/spacetime/exact_binary.rs (exact M^2-(a^2+Q^2)).
// Every `mul_add` of the reference is `std::fma` here; the translation unit is compiled with
// -ffp-contract=off so no other product is fused.
#pragma once

#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>

namespace gro {

inline uint64_t bits_of(double v) {
  uint64_t b;
  std::memcpy(&b, &v, sizeof b);
  return b;
}
inline double from_bits(uint64_t b) {
  double v;
  std::memcpy(&v, &b, sizeof v);
  return v;
}

// numerics.rs:137-151 binary64_magnitude
inline void binary64_magnitude(double value, uint64_t& significand, int& exponent) {
  const uint64_t b = bits_of(value);
  const uint64_t stored = (b >> 52) & 0x7ff;
  const uint64_t fraction = b & ((uint64_t(1) << 52) - 1);
  if (stored == 0) {
    significand = fraction;
    exponent = -1074;
  } else {
    significand = (uint64_t(1) << 52) | fraction;
    exponent = int(stored) - 1075;
  }
}

// numerics.rs:153-171 binary_power
inline double binary_power(int exponent) {
  if (exponent < -1074) return 0.0;
  if (exponent < -1022) return from_bits(uint64_t(1) << unsigned(exponent + 1074));
  const long stored = long(exponent) + 1023;
  if (stored >= 0x7ff) return std::numeric_limits<double>::infinity();
  return from_bits(uint64_t(stored) << 52);
}

// numerics.rs:127-136 positive_binary_decomposition (value assumed positive, finite)
inline void positive_binary_decomposition(double value, double& significand, int& exponent) {
  uint64_t s;
  int e;
  binary64_magnitude(value, s, e);
  if (s == 0) {
    significand = std::numeric_limits<double>::quiet_NaN();
    exponent = 0;
    return;
  }
  const int highest_bit = 63 - __builtin_clzll(s);
  exponent = e + highest_bit;
  significand = value / binary_power(exponent);
}

// numerics.rs:103-125 positive_product
template <size_t N>
inline double positive_product(const std::array<double, N>& factors) {
  for (double f : factors)
    if (f == 0.0) return 0.0;
  double significand = 1.0;
  int exponent = 0;
  for (double f : factors) {
    double fs;
    int fe;
    positive_binary_decomposition(f, fs, fe);
    significand *= fs;
    exponent += fe;
    if (significand >= 2.0) {
      significand *= 0.5;
      exponent += 1;
    }
  }
  if (exponent < -1075) return 0.0;
  if (exponent == -1075) return (significand * 0.5) * from_bits(1);
  return significand * binary_power(exponent);
}

// numerics.rs:3-35 normalized_quadratic_form_residual
inline double normalized_quadratic_form_residual(const double m[4][4], const double v[4]) {
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c)
      if (!std::isfinite(m[r][c])) return std::numeric_limits<double>::quiet_NaN();
  for (int i = 0; i < 4; ++i)
    if (!std::isfinite(v[i])) return std::numeric_limits<double>::quiet_NaN();
  double matrix_scale = 0.0;
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) matrix_scale = std::fmax(matrix_scale, std::fabs(m[r][c]));
  double vector_scale = 0.0;
  for (int i = 0; i < 4; ++i) vector_scale = std::fmax(vector_scale, std::fabs(v[i]));
  if (matrix_scale == 0.0 || vector_scale == 0.0) return 0.0;
  double sv[4];
  for (int i = 0; i < 4; ++i) sv[i] = v[i] / vector_scale;
  double contraction = 0.0, term_norm = 0.0;
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) {
      const double term = (m[r][c] / matrix_scale) * sv[r] * sv[c];
      contraction += term;
      term_norm += std::fabs(term);
    }
  if (term_norm == 0.0) return 0.0;
  const double relative = std::fabs(contraction) / term_norm;
  const double denominator_scale = std::fmin(
      positive_product(std::array<double, 4>{term_norm, matrix_scale, vector_scale, vector_scale}),
      1.0);
  return relative * denominator_scale;
}

// exact_binary.rs:12-122 ExactBinary: 66 64-bit limbs hold the exact sum of two squared
// binary64 magnitudes (exponent range [-2148, ...]).
struct ExactBinary {
  static constexpr int LIMBS = 66;
  static constexpr int MIN_SQUARED_EXPONENT = -2148;
  uint64_t limbs[LIMBS];

  ExactBinary() { std::memset(limbs, 0, sizeof limbs); }

  static ExactBinary square(double v) {
    ExactBinary r;
    r.add_square(v);
    return r;
  }
  static ExactBinary sum_of_squares(double a, double b) {
    ExactBinary r;
    r.add_square(a);
    r.add_square(b);
    return r;
  }
  void add_word(int index, uint64_t value) {
    while (value != 0) {
      const uint64_t sum = limbs[index] + value;
      const bool carry = sum < value;
      limbs[index] = sum;
      value = carry ? 1 : 0;
      ++index;
    }
  }
  void add_shifted(unsigned __int128 coefficient, size_t shift) {
    const size_t word = shift / 64, bit = shift % 64;
    const uint64_t low = uint64_t(coefficient), high = uint64_t(coefficient >> 64);
    if (bit == 0) {
      add_word(int(word), low);
      add_word(int(word + 1), high);
    } else {
      add_word(int(word), low << bit);
      add_word(int(word + 1), low >> (64 - bit));
      add_word(int(word + 1), high << bit);
      add_word(int(word + 2), high >> (64 - bit));
    }
  }
  void add_square(double value) {
    uint64_t s;
    int e;
    binary64_magnitude(std::fabs(value), s, e);
    if (s == 0) return;
    const unsigned __int128 c = (unsigned __int128)s * s;
    const long shift = 2L * e - MIN_SQUARED_EXPONENT;
    add_shifted(c, shift < 0 ? 0 : size_t(shift));
  }
  ExactBinary subtract(const ExactBinary& smaller) const {
    ExactBinary r;
    bool borrow = false;
    for (int i = 0; i < LIMBS; ++i) {
      const uint64_t d1 = limbs[i] - smaller.limbs[i];
      const bool b1 = limbs[i] < smaller.limbs[i];
      const uint64_t d2 = d1 - (borrow ? 1 : 0);
      const bool b2 = borrow && d1 == 0;
      r.limbs[i] = d2;
      borrow = b1 || b2;
    }
    return r;
  }
  int highest_bit() const {
    for (int w = LIMBS - 1; w >= 0; --w)
      if (limbs[w] != 0) return w * 64 + (63 - __builtin_clzll(limbs[w]));
    return -1;
  }
  bool bit(long index) const { return (limbs[index / 64] >> (index % 64)) & 1; }
  double square_root() const {
    int hb = highest_bit();
    if (hb < 0) hb = 0;
    uint64_t significand = 0;
    for (int off = 0; off < 53; ++off) {
      significand <<= 1;
      if (hb >= off && bit(hb - off)) significand |= 1;
    }
    const long discarded = hb > 52 ? hb - 52 : 0;
    if (discarded > 0) {
      const bool guard = bit(discarded - 1);
      bool sticky = false;
      for (long b = 0; b < discarded - 1 && !sticky; ++b) sticky = bit(b);
      if (guard && (sticky || (significand & 1))) significand += 1;
    }
    const double high = double(uint32_t(significand >> 32));
    const double low = double(uint32_t(significand & 0xffffffffu));
    const double normalized = std::fma(high, 4294967296.0, low) / 4503599627370496.0;
    const int exponent = MIN_SQUARED_EXPONENT + hb;
    if ((exponent & 1) == 0) return std::sqrt(normalized) * binary_power(exponent / 2);
    return std::sqrt(2.0 * normalized) * binary_power((exponent - 1) / 2);
  }
  int compare(const ExactBinary& o) const {
    for (int i = LIMBS - 1; i >= 0; --i) {
      if (limbs[i] < o.limbs[i]) return -1;
      if (limbs[i] > o.limbs[i]) return 1;
    }
    return 0;
  }
};

}  // namespace gro
