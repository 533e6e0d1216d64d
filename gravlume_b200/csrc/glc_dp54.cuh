// Dormand-Prince 5(4) with FSAL, embedded error estimate and Shampine's quartic dense output.
// Coefficients are the published Dormand-Prince (1980) tableau and the dense-output polynomial the
// reference's oracle uses (crates/gravlume-reference/src/integrator.rs:6-98); they are compile-time
// constants here, so every stage combination is an FMA with an immediate operand.
#pragma once

#include <type_traits>

#include "glc_geometry.cuh"

namespace glc {
namespace dp {
// stage matrix A[i][j], i = 1..6 (stage 7 row equals the fifth-order weights B5)
constexpr double a21 = 1.0 / 5.0;
constexpr double a31 = 3.0 / 40.0, a32 = 9.0 / 40.0;
constexpr double a41 = 44.0 / 45.0, a42 = -56.0 / 15.0, a43 = 32.0 / 9.0;
constexpr double a51 = 19372.0 / 6561.0, a52 = -25360.0 / 2187.0, a53 = 64448.0 / 6561.0, a54 = -212.0 / 729.0;
constexpr double a61 = 9017.0 / 3168.0, a62 = -355.0 / 33.0, a63 = 46732.0 / 5247.0, a64 = 49.0 / 176.0,
                 a65 = -5103.0 / 18656.0;
constexpr double b1 = 35.0 / 384.0, b3 = 500.0 / 1113.0, b4 = 125.0 / 192.0, b5 = -2187.0 / 6784.0, b6 = 11.0 / 84.0;
// fourth-order weights
constexpr double c1 = 5179.0 / 57600.0, c3 = 7571.0 / 16695.0, c4 = 393.0 / 640.0, c5 = -92097.0 / 339200.0,
                 c6 = 187.0 / 2100.0, c7 = 1.0 / 40.0;
// error weights e = b - c
constexpr double e1 = b1 - c1, e3 = b3 - c3, e4 = b4 - c4, e5 = b5 - c5, e6 = b6 - c6, e7 = -c7;
// dense output: y(theta) = y0 + h sum_j (sum_k d_jk theta^(k+1)) K_j (stage 2 has no weight)
constexpr double d10 = 1.0, d11 = -8048581381.0 / 2820520608.0, d12 = 8663915743.0 / 2820520608.0,
                 d13 = -12715105075.0 / 11282082432.0;
constexpr double d31 = 131558114200.0 / 32700410799.0, d32 = -68118460800.0 / 10900136933.0,
                 d33 = 87487479700.0 / 32700410799.0;
constexpr double d41 = -1754552775.0 / 470086768.0, d42 = 14199869525.0 / 1410260304.0,
                 d43 = -10690763975.0 / 1880347072.0;
constexpr double d51 = 127303824393.0 / 49829197408.0, d52 = -318862633887.0 / 49829197408.0,
                 d53 = 701980252875.0 / 199316789632.0;
constexpr double d61 = -282668133.0 / 205662961.0, d62 = 2019193451.0 / 616988883.0,
                 d63 = -1453857185.0 / 822651844.0;
constexpr double d71 = 40617522.0 / 29380423.0, d72 = -110615467.0 / 29380423.0, d73 = 69997945.0 / 29380423.0;
}  // namespace dp

// Stage matrix as a table for the compact attempt (row s: coefficients of stages 0..s-1; row 6 is
// the fifth-order weights, so stage 7's point is the end state), and the error weights b - b*.
#define GLC_DP_A(T)                                                                                   \
  {{T(0), T(0), T(0), T(0), T(0), T(0)},                                                              \
   {T(dp::a21), T(0), T(0), T(0), T(0), T(0)},                                                        \
   {T(dp::a31), T(dp::a32), T(0), T(0), T(0), T(0)},                                                  \
   {T(dp::a41), T(dp::a42), T(dp::a43), T(0), T(0), T(0)},                                            \
   {T(dp::a51), T(dp::a52), T(dp::a53), T(dp::a54), T(0), T(0)},                                      \
   {T(dp::a61), T(dp::a62), T(dp::a63), T(dp::a64), T(dp::a65), T(0)},                                \
   {T(dp::b1), T(0), T(dp::b3), T(dp::b4), T(dp::b5), T(dp::b6)}}

// Streaming form of the stage matrix: after the slope of stage j (0-based) is known it is added,
// with weight kStreamA[j][m] = A[j+1+m][j], into the pending point sum of stage j+1+m; the sums
// rotate so that the next stage's sum is always first (row 6, after the end-point slope, is zero).
// kStreamE / kStreamB are the error weights b - b* and the fifth-order weights b per stage.
#define GLC_STREAM_A(T)                                                                                  \
  {{T(dp::a21), T(dp::a31), T(dp::a41), T(dp::a51), T(dp::a61), T(dp::b1)},                             \
   {T(dp::a32), T(dp::a42), T(dp::a52), T(dp::a62), T(0), T(0)},                                         \
   {T(dp::a43), T(dp::a53), T(dp::a63), T(dp::b3), T(0), T(0)},                                          \
   {T(dp::a54), T(dp::a64), T(dp::b4), T(0), T(0), T(0)},                                                \
   {T(dp::a65), T(dp::b5), T(0), T(0), T(0), T(0)},                                                      \
   {T(dp::b6), T(0), T(0), T(0), T(0), T(0)},                                                            \
   {T(0), T(0), T(0), T(0), T(0), T(0)}}
#define GLC_STREAM_E(T) {T(dp::e1), T(0), T(dp::e3), T(dp::e4), T(dp::e5), T(dp::e6), T(dp::e7)}
#define GLC_STREAM_B(T) {T(dp::b1), T(0), T(dp::b3), T(dp::b4), T(dp::b5), T(dp::b6), T(0)}

// The device reads constant memory at a warp-uniform index; host code (the host builds of these
// templates, and the host pass of nvcc) reads ordinary static copies of the same tables.
#if defined(__CUDACC__)
__constant__ double kDpA[7][6] = GLC_DP_A(double);
__constant__ float kDpAf[7][6] = GLC_DP_A(float);
__constant__ float kStreamAf[7][6] = GLC_STREAM_A(float);
__constant__ double kStreamAd[7][6] = GLC_STREAM_A(double);
__constant__ float kStreamEf[7] = GLC_STREAM_E(float);
__constant__ double kStreamEd[7] = GLC_STREAM_E(double);
__constant__ float kStreamBf[7] = GLC_STREAM_B(float);
__constant__ double kStreamBd[7] = GLC_STREAM_B(double);
#endif
static const double kDpAHost[7][6] = GLC_DP_A(double);
static const float kDpAfHost[7][6] = GLC_DP_A(float);
static const float kStreamAfHost[7][6] = GLC_STREAM_A(float);
static const double kStreamAdHost[7][6] = GLC_STREAM_A(double);
static const float kStreamEfHost[7] = GLC_STREAM_E(float);
static const double kStreamEdHost[7] = GLC_STREAM_E(double);
static const float kStreamBfHost[7] = GLC_STREAM_B(float);
static const double kStreamBdHost[7] = GLC_STREAM_B(double);
#undef GLC_DP_A
#undef GLC_STREAM_A
#undef GLC_STREAM_E
#undef GLC_STREAM_B

#if defined(__CUDA_ARCH__)
#define GLC_COEF(table) table
#else
#define GLC_COEF(table) table##Host
#endif

template <class T>
GLC_HD T dp_a(int s, int j);
template <>
GLC_HD float dp_a<float>(int s, int j) { return GLC_COEF(kDpAf)[s][j]; }
template <>
GLC_HD double dp_a<double>(int s, int j) { return GLC_COEF(kDpA)[s][j]; }

template <class T>
struct StreamCoef;
template <>
struct StreamCoef<float> {
  static GLC_HD float a(int j, int m) { return GLC_COEF(kStreamAf)[j][m]; }
  static GLC_HD float e(int j) { return GLC_COEF(kStreamEf)[j]; }
  static GLC_HD float b(int j) { return GLC_COEF(kStreamBf)[j]; }
};
template <>
struct StreamCoef<double> {
  static GLC_HD double a(int j, int m) { return GLC_COEF(kStreamAd)[j][m]; }
  static GLC_HD double e(int j) { return GLC_COEF(kStreamEd)[j]; }
  static GLC_HD double b(int j) { return GLC_COEF(kStreamBd)[j]; }
};
#undef GLC_COEF

struct Tolerance {
  double pos_rtol, pos_atol, mom_rtol, mom_atol;
};

// One attempt. y0 is the state in storage precision S, the stages run in compute precision C.
// Returns the grouped infinity norm of the embedded error (the reference's error_norm with the
// relative coordinate time in the time slot, crates/gravlume-reference/src/policy.rs:137-158 and
// geodesic.rs:158-165). Outputs: inc = fifth-order increment of the six state components
// (y1 = y0 + inc in S), dt = coordinate-time increment, k7 = derivative at the end (FSAL) with
// r, dr/dlambda and the invariants there; `finite` is false if anything overflowed or became NaN.
template <class C, class S, bool kInv = true>
GLC_HD C dp5_attempt(const KN<C>& k, const S y0[6], C E, C h, const C k1[7], C t_start, const Tolerance& tol,
                     C inc[6], C& dt, C k7[7], C& r_end, C& vr_end, Invariants<C>& inv, bool& finite) {
  using namespace dp;
  C y0c[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) y0c[c] = C(y0[c]);
  C k2[7], k3[7], k4[7], k5[7], k6[7], ys[6], rr, vv;
#pragma unroll
  for (int c = 0; c < 6; ++c) ys[c] = y0c[c] + h * (C(a21) * k1[c]);
  kn_rhs(k, ys, E, k2, rr, vv);
#pragma unroll
  for (int c = 0; c < 6; ++c) ys[c] = y0c[c] + h * (C(a31) * k1[c] + C(a32) * k2[c]);
  kn_rhs(k, ys, E, k3, rr, vv);
#pragma unroll
  for (int c = 0; c < 6; ++c) ys[c] = y0c[c] + h * (C(a41) * k1[c] + C(a42) * k2[c] + C(a43) * k3[c]);
  kn_rhs(k, ys, E, k4, rr, vv);
#pragma unroll
  for (int c = 0; c < 6; ++c)
    ys[c] = y0c[c] + h * (C(a51) * k1[c] + C(a52) * k2[c] + C(a53) * k3[c] + C(a54) * k4[c]);
  kn_rhs(k, ys, E, k5, rr, vv);
#pragma unroll
  for (int c = 0; c < 6; ++c)
    ys[c] = y0c[c] + h * (C(a61) * k1[c] + C(a62) * k2[c] + C(a63) * k3[c] + C(a64) * k4[c] + C(a65) * k5[c]);
  kn_rhs(k, ys, E, k6, rr, vv);
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    inc[c] = h * (C(b1) * k1[c] + C(b3) * k3[c] + C(b4) * k4[c] + C(b5) * k5[c] + C(b6) * k6[c]);
    ys[c] = y0c[c] + inc[c];
  }
  kn_rhs<C, kInv>(k, ys, E, k7, r_end, vr_end, &inv);
  dt = h * (C(b1) * k1[6] + C(b3) * k3[6] + C(b4) * k4[6] + C(b5) * k5[6] + C(b6) * k6[6]);
  C chk = dt + r_end;
  if (kInv) chk += inv.lz + inv.carter;
  // max_c |err_c| / scale_c with a single reciprocal: keep the running maximum as a fraction
  // (num, den) and compare fractions by cross-multiplication (all scales are positive)
  C num = C(0), den = C(1);
#pragma unroll
  for (int c = 0; c < 7; ++c) {
    const C err = h * (C(e1) * k1[c] + C(e3) * k3[c] + C(e4) * k4[c] + C(e5) * k5[c] + C(e6) * k6[c] + C(e7) * k7[c]);
    const C sv = c < 6 ? y0c[c] : t_start;
    const C ev = c < 6 ? ys[c] : t_start + dt;
    const bool pos = c < 3 || c == 6;
    const C scale = C(pos ? tol.pos_rtol : tol.mom_rtol) * g_max(g_abs(sv), g_abs(ev)) + C(pos ? tol.pos_atol : tol.mom_atol);
    const C ae = g_abs(err);
    const bool larger = ae * den > num * scale;
    num = larger ? ae : num;
    den = larger ? scale : den;
    chk += err + k7[c];
  }
  finite = g_finite(chk);
  return num * g_rcp(den);
}

// The same attempt with the stage loop kept rolled: one inlined right-hand side serves all six
// evaluations and the stages live in a per-thread array (local memory, L1-resident), so the hot
// loop's instruction footprint is a fraction of the unrolled form's.
template <class C, class S, bool kInv = true>
GLC_HD C dp5_attempt_compact(const KN<C>& k, const S y0[6], C E, C h, const C k1[7], C t_start,
                             const Tolerance& tol, C inc[6], C& dt, C k7[7], C& r_end, C& vr_end,
                             Invariants<C>& inv, bool& finite) {
  using namespace dp;
  C K[7][7];
  C y0c[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) y0c[c] = C(y0[c]);
#pragma unroll
  for (int c = 0; c < 7; ++c) K[0][c] = k1[c];
  C ys[6], rr = C(0), vv = C(0);
#pragma unroll 1
  for (int s = 1; s < 7; ++s) {
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      C w = C(0);
#pragma unroll 1
      for (int j = 0; j < s; ++j) w += dp_a<C>(s, j) * K[j][c];
      ys[c] = y0c[c] + h * w;
    }
    C d[7];
    if (s < 6) {
      kn_rhs<C, false>(k, ys, E, d, rr, vv);
    } else {
      kn_rhs<C, kInv>(k, ys, E, d, rr, vv, &inv);
    }
#pragma unroll
    for (int c = 0; c < 7; ++c) K[s][c] = d[c];
  }
  r_end = rr;
  vr_end = vv;
#pragma unroll
  for (int c = 0; c < 6; ++c) inc[c] = ys[c] - y0c[c];
  dt = h * (C(b1) * K[0][6] + C(b3) * K[2][6] + C(b4) * K[3][6] + C(b5) * K[4][6] + C(b6) * K[5][6]);
#pragma unroll
  for (int c = 0; c < 7; ++c) k7[c] = K[6][c];
  C chk = dt + r_end;
  if (kInv) chk += inv.lz + inv.carter;
  C num = C(0), den = C(1);
#pragma unroll
  for (int c = 0; c < 7; ++c) {
    const C err =
        h * (C(e1) * K[0][c] + C(e3) * K[2][c] + C(e4) * K[3][c] + C(e5) * K[4][c] + C(e6) * K[5][c] + C(e7) * K[6][c]);
    const C sv = c < 6 ? y0c[c] : t_start;
    const C ev = c < 6 ? ys[c] : t_start + dt;
    const bool pos = c < 3 || c == 6;
    const C scale = C(pos ? tol.pos_rtol : tol.mom_rtol) * g_max(g_abs(sv), g_abs(ev)) + C(pos ? tol.pos_atol : tol.mom_atol);
    const C ae = g_abs(err);
    const bool larger = ae * den > num * scale;
    num = larger ? ae : num;
    den = larger ? scale : den;
    chk += err + K[6][c];
  }
  finite = g_finite(chk);
  return num * g_rcp(den);
}

// The same attempt in streaming form: all six evaluations (five interior stages and the end point)
// run through one rolled loop around a single inlined right-hand side, whose invariants block runs
// on the last pass only. The pending stage sums stay at fixed register positions (no local memory)
// and the coefficients come from constant memory at the warp-uniform stage index, so the hot
// loop's instruction footprint is about a sixth of the unrolled form's.
// kFold: the end-point evaluation is the loop's sixth pass (one right-hand-side body; measured
// faster in binary64) or follows the loop as its own call (measured faster in binary32).
// kUnroll: the stage loop unrolled (the binary32 bulk kernel of MIXED, whose instruction footprint
// is small enough that the coefficients as immediates pay) or rolled (1; every other kernel, where
// the unrolled footprint measured slower: instruction fetch).
template <class C, class S, bool kInv = true, bool kFold = std::is_same<C, double>::value, int kUnroll = 1>
GLC_HD C dp5_attempt_stream(const KN<C>& k, const S y0[6], C E, C h, const C k1[7], C t_start, const Tolerance& tol,
                            C inc[6], C& dt, C k7[7], C& r_end, C& vr_end, Invariants<C>& inv, bool& finite,
                            bool track = true, C (*stages)[7] = nullptr) {
  using Coef = StreamCoef<C>;
  // stages (optional): the seven stage derivatives of this attempt, for a dense output built
  // without evaluating them again
  if (stages != nullptr)
    for (int c = 0; c < 7; ++c) stages[0][c] = k1[c];
  C y0c[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) y0c[c] = C(y0[c]);
  C P[6][6], err[7], bt;
#pragma unroll
  for (int m = 0; m < 6; ++m)
#pragma unroll
    for (int c = 0; c < 6; ++c) P[m][c] = Coef::a(0, m) * k1[c];
#pragma unroll
  for (int c = 0; c < 7; ++c) err[c] = Coef::e(0) * k1[c];
  bt = Coef::b(0) * k1[6];
  C ys[6], rr = C(0), vv = C(0), d[7];
  constexpr int kPasses = kFold ? 7 : 6;
#pragma unroll kUnroll
  for (int j = 1; j < kPasses; ++j) {
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      if constexpr (kFold) {
        inc[c] = h * P[0][c];
        ys[c] = y0c[c] + inc[c];
      } else {
        ys[c] = y0c[c] + h * P[0][c];
      }
    }
    if constexpr (kFold) {
      kn_rhs<C, kInv>(k, ys, E, d, rr, vv, (track && j == 6) ? &inv : nullptr);
    } else {
      kn_rhs<C, false>(k, ys, E, d, rr, vv);
    }
    if (stages != nullptr)
      for (int c = 0; c < 7; ++c) stages[j][c] = d[c];
    // pending sums of the stages still ahead (stage j + 2 + m <= 7); the rest would only add
    // zero coefficients
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      if (m + j > 5) break;
#pragma unroll
      for (int c = 0; c < 6; ++c) P[m][c] = P[m + 1][c] + Coef::a(j, m) * d[c];
    }
    const C ej = Coef::e(j);
#pragma unroll
    for (int c = 0; c < 7; ++c) err[c] += ej * d[c];
    bt += Coef::b(j) * d[6];
  }
  if constexpr (!kFold) {
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      inc[c] = h * P[0][c];
      ys[c] = y0c[c] + inc[c];
    }
    kn_rhs<C, kInv>(k, ys, E, d, rr, vv, track ? &inv : nullptr);
    if (stages != nullptr)
      for (int c = 0; c < 7; ++c) stages[6][c] = d[c];
#pragma unroll
    for (int c = 0; c < 7; ++c) err[c] += Coef::e(6) * d[c];
  }
#pragma unroll
  for (int c = 0; c < 7; ++c) k7[c] = d[c];
  r_end = rr;
  vr_end = vv;
  dt = h * bt;
  C chk = dt + r_end;
  if (kInv && track) chk += inv.lz + inv.carter;
  C num = C(0), den = C(1);
#pragma unroll
  for (int c = 0; c < 7; ++c) {
    const C e = h * err[c];
    const C sv = c < 6 ? y0c[c] : t_start;
    const C ev = c < 6 ? ys[c] : t_start + dt;
    const bool pos = c < 3 || c == 6;
    const C scale = C(pos ? tol.pos_rtol : tol.mom_rtol) * g_max(g_abs(sv), g_abs(ev)) + C(pos ? tol.pos_atol : tol.mom_atol);
    const C ae = g_abs(e);
    const bool larger = ae * den > num * scale;
    num = larger ? ae : num;
    den = larger ? scale : den;
    chk += e + k7[c];
  }
  finite = g_finite(chk);
  return num * g_rcp(den);
}

// Full stage set for dense output (the rare event path). K[0] must hold k1 on entry. The last
// stage is evaluated at the fifth-order end state, returned in yend with r and dr/dlambda there.
template <class T>
GLC_HD void dp5_stages(const KN<T>& k, const T y0[6], T E, T h, T K[7][7], T yend[6], T& r_end, T& vr_end) {
  using namespace dp;
  const double A[7][6] = {{0, 0, 0, 0, 0, 0},       {a21, 0, 0, 0, 0, 0},       {a31, a32, 0, 0, 0, 0},
                          {a41, a42, a43, 0, 0, 0}, {a51, a52, a53, a54, 0, 0}, {a61, a62, a63, a64, a65, 0},
                          {b1, 0, b3, b4, b5, b6}};
  T ys[6], rr, vv;
#pragma unroll
  for (int s = 1; s < 7; ++s) {
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      T w = T(0);
#pragma unroll
      for (int j = 0; j < s; ++j) w += T(A[s][j]) * K[j][c];
      ys[c] = y0[c] + h * w;
    }
    kn_rhs(k, ys, E, K[s], rr, vv);
  }
#pragma unroll
  for (int c = 0; c < 6; ++c) yend[c] = ys[c];
  r_end = rr;
  vr_end = vv;
}

template <class T>
GLC_HD void dense_weights(T th, T w[7]) {
  using namespace dp;
  const T p1 = th, p2 = th * th, p3 = p2 * th, p4 = p2 * p2;
  w[0] = T(d10) * p1 + T(d11) * p2 + T(d12) * p3 + T(d13) * p4;
  w[1] = T(0);
  w[2] = T(d31) * p2 + T(d32) * p3 + T(d33) * p4;
  w[3] = T(d41) * p2 + T(d42) * p3 + T(d43) * p4;
  w[4] = T(d51) * p2 + T(d52) * p3 + T(d53) * p4;
  w[5] = T(d61) * p2 + T(d62) * p3 + T(d63) * p4;
  w[6] = T(d71) * p2 + T(d72) * p3 + T(d73) * p4;
}

// Dense state (six components) and coordinate-time increment at theta.
template <class T>
GLC_HD void dense_eval(const T y0[6], T h, const T K[7][7], T th, T y[6], T& dt) {
  T w[7];
  dense_weights(th, w);
#pragma unroll
  for (int c = 0; c < 7; ++c) {
    T s = T(0);
#pragma unroll
    for (int j = 0; j < 7; ++j) s += w[j] * K[j][c];
    if (c < 6) y[c] = y0[c] + h * s;
    else dt = h * s;
  }
}

// Dense output with stages in TK accumulated in T (binary64 dense state from binary32 stages in
// the MIXED event path).
template <class T, class TK>
GLC_HD void dense_eval_mixed(const T y0[6], T h, const TK K[7][7], T th, T y[6], T& dt) {
  T w[7];
  dense_weights(th, w);
#pragma unroll
  for (int c = 0; c < 7; ++c) {
    T s = T(0);
#pragma unroll
    for (int j = 0; j < 7; ++j) s += w[j] * T(K[j][c]);
    if (c < 6) y[c] = y0[c] + h * s;
    else dt = h * s;
  }
}

template <class T>
GLC_HD T dense_component(const T y0[6], T h, const T K[7][7], T th, int c) {
  T w[7];
  dense_weights(th, w);
  T s = T(0);
#pragma unroll
  for (int j = 0; j < 7; ++j) s += w[j] * K[j][c];
  return y0[c] + h * s;
}

}  // namespace glc
