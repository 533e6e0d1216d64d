// Discrete adjoint of the DP5(4) trace: reverse sweeps of accepted steps and of the terminal event,
// compiled for the device (the adjoint kernels) and for the host (the adjoint's CPU checks).
//
// The forward map of one accepted step with frozen step size h is
//   Y_1 = y0,  Y_i = y0 + h sum_{j<i} a_ij k_j,  k_i = F(Y_i; E, a, Q^2),  y1 = y0 + h sum_i w_i k_i,
// with w = the fifth-order weights b (stage 7 unused), and for the terminal step of a trace the
// dense-output weights w_i(theta*) at the localized event (stage 7 is F at the fifth-order end
// point). Its adjoint, for lambda = dL/dy1:
//   kbar_i = h w_i lambda;  for i = 7 .. 1:  Ybar_i = J_i^T kbar_i,  kbar_j += h a_ij Ybar_i (j < i),
//   lambda0 = lambda + sum_i Ybar_i,  and dL/d(E, a, Q^2) += sum_i (dF/d(E, a, Q^2))^T kbar_i,
// where J_i is the Jacobian of the reduced right-hand side at stage point Y_i, taken in forward mode
// with 9 dual channels (6 state, E, a, Q^2). The event time theta* of the terminal step depends on
// the inputs through the event condition e(y(theta*)) = 0; its implicit derivative turns the
// observable adjoint mu into mu - (mu . ydot) / (grad e . ydot) grad e before the dense-output sweep.
//
// The step sizes are the forward pass's accepted steps, held fixed (the controller's accept/reject
// decisions are piecewise constant), which is the standard discrete adjoint of an adaptive
// integrator: its gradient is the exact derivative of the computed map and agrees with the
// derivative of the exact flow to the integration tolerance.
#pragma once

#include "glc_dual.cuh"
#include "glc_tracer.cuh"

namespace glc {

using D9 = Dual<9>;
constexpr int kChE = 6, kChA = 7, kChQ2 = 8;

GLC_HD double g_hypot(double a, double b) {
#if defined(__CUDA_ARCH__)
  return hypot(a, b);
#else
  return std::hypot(a, b);
#endif
}

GLC_HD KN<D9> kn_dual(const KN<double>& k) {
  KN<D9> o;
  o.a = D9::seed(k.a, kChA);
  o.a2 = o.a * o.a;
  o.s = D9(k.s);
  o.sa = o.s * o.a;
  o.q2 = D9::seed(k.q2, kChQ2);
  return o;
}

// Stage-matrix row i (0-based stage), coefficient of stage j < i; row 6 holds the fifth-order
// weights (stage 7's point is the end state). The device reads the constant-memory table (a local
// array indexed at run time would be rebuilt in local memory on every call).
GLC_HD double dp_coef(int i, int j) { return dp_a<double>(i, j); }

// Weights of the fifth-order end point (stage 7 unused).
GLC_HD void step_weights(double w[7]) {
  using namespace dp;
  const double b[7] = {b1, 0.0, b3, b4, b5, b6, 0.0};
  for (int i = 0; i < 7; ++i) w[i] = b[i];
}

// Dense-output weights at theta, y(theta) = y0 + h sum_j w_j K_j, and their theta-derivatives.
GLC_HD void dense_weights_at(double th, double w[7], double dw[7]) {
  using namespace dp;
  const double d[7][4] = {{d10, d11, d12, d13}, {0, 0, 0, 0},     {0, d31, d32, d33}, {0, d41, d42, d43},
                          {0, d51, d52, d53},   {0, d61, d62, d63}, {0, d71, d72, d73}};
  for (int j = 0; j < 7; ++j) {
    w[j] = th * (d[j][0] + th * (d[j][1] + th * (d[j][2] + th * d[j][3])));
    dw[j] = d[j][0] + th * (2.0 * d[j][1] + th * (3.0 * d[j][2] + th * 4.0 * d[j][3]));
  }
}

// Stage points Y_i and slopes K_i (binary64) of the step from y0 with size h.
GLC_HD void dp5_stage_points(const KN<double>& k, const double y0[6], double E, double h, double Y[7][6],
                             double K[7][6]) {
  for (int i = 0; i < 7; ++i) {
    for (int c = 0; c < 6; ++c) {
      double s = 0.0;
      for (int j = 0; j < i; ++j) s += dp_coef(i, j) * K[j][c];
      Y[i][c] = y0[c] + h * s;
    }
    double d[7], r, vr;
    kn_rhs(k, Y[i], E, d, r, vr);
    for (int c = 0; c < 6; ++c) K[i][c] = d[c];
  }
}

// kbar -> Ybar += J_y^T kbar and g (E, a, Q^2) += J_p^T kbar at stage point Y, from the full
// 9-channel Jacobian (kept as the cross-check of rhs_vjp).
GLC_HD void rhs_vjp_jacobian(const KN<D9>& kd, const double Y[6], double E, const double kbar[6], double ybar[6],
                             double g[3]) {
  D9 y[6];
  for (int c = 0; c < 6; ++c) y[c] = D9::seed(Y[c], c);
  D9 d[7], r, vr;
  kn_rhs(kd, y, D9::seed(E, kChE), d, r, vr);
  for (int c = 0; c < 6; ++c) {
    const double kb = kbar[c];
    for (int i = 0; i < 6; ++i) ybar[i] += d[c].d[i] * kb;
    g[0] += d[c].d[kChE] * kb;
    g[1] += d[c].d[kChA] * kb;
    g[2] += d[c].d[kChQ2] * kb;
  }
}

// The same product from 4 channels. The reduced system is Hamiltonian, F = J grad H with
// J = [[0, I], [-I, 0]] and H = g^{mu nu} p_mu p_nu / 2 at fixed p_t = -E, so its state Jacobian is
// J Hess(H) and J_y^T kbar = Hess(H) u with u = J^T kbar = (-kbar_p, kbar_x). Hess(H) u is the
// derivative of grad H = (-F_p, F_x) along u: one tangent channel seeded with u. Channels 1-3 carry
// E, a and Q^2 for the parameter part.
using D4 = Dual<4>;
constexpr int kVjpDir = 0, kVjpE = 1, kVjpA = 2, kVjpQ2 = 3;

// The spacetime constants with their a and Q^2 channels, over the scalar type R of the sweep.
template <class R = double>
GLC_HD KN<Dual<4, R>> kn_dual_vjp(const KN<double>& k) {
  using V = Dual<4, R>;
  KN<V> o;
  o.a = V::seed(k.a, kVjpA);
  o.a2 = o.a * o.a;
  o.s = V(k.s);
  o.sa = o.s * o.a;
  o.q2 = V::seed(k.q2, kVjpQ2);
  return o;
}

template <class R>
GLC_HD void rhs_vjp(const KN<Dual<4, R>>& kd, const double Y[6], double E, const double kbar[6], double ybar[6],
                    double g[3]) {
  using V = Dual<4, R>;
  V y[6];
  for (int c = 0; c < 3; ++c) {
    y[c] = V(Y[c]);
    y[c].d[kVjpDir] = R(-kbar[3 + c]);
    y[3 + c] = V(Y[3 + c]);
    y[3 + c].d[kVjpDir] = R(kbar[c]);
  }
  V d[7], r, vr;
  kn_rhs(kd, y, V::seed(E, kVjpE), d, r, vr);
  for (int c = 0; c < 3; ++c) {
    ybar[c] -= double(d[3 + c].d[kVjpDir]);
    ybar[3 + c] += double(d[c].d[kVjpDir]);
  }
  for (int c = 0; c < 6; ++c) {
    const double kb = kbar[c];
    g[0] += double(d[c].d[kVjpE]) * kb;
    g[1] += double(d[c].d[kVjpA]) * kb;
    g[2] += double(d[c].d[kVjpQ2]) * kb;
  }
}

// Reverse sweep over the stages of y_out = y0 + h sum_i w_i K_i, given the stage points Y:
// lam0 = dL/dy0 from lam = dL/dy_out, g += dL/d(E, a, Q^2).
template <class R>
GLC_HD void stages_reverse(const KN<Dual<4, R>>& kd, const double Y[7][6], double E, double h, const double w[7],
                           const double lam[6], double lam0[6], double g[3]) {
  double kb[7][6];
  for (int i = 0; i < 7; ++i)
    for (int c = 0; c < 6; ++c) kb[i][c] = h * w[i] * lam[c];
  double out[6];
  for (int c = 0; c < 6; ++c) out[c] = lam[c];
  for (int i = 6; i >= 0; --i) {
    bool nz = false;
    for (int c = 0; c < 6; ++c) nz = nz || kb[i][c] != 0.0;
    if (!nz) continue;
    double yb[6] = {0, 0, 0, 0, 0, 0};
    rhs_vjp(kd, Y[i], E, kb[i], yb, g);
    for (int c = 0; c < 6; ++c) out[c] += yb[c];
    for (int j = 0; j < i; ++j) {
      const double cf = h * dp_coef(i, j);
      if (cf == 0.0) continue;
      for (int c = 0; c < 6; ++c) kb[j][c] += cf * yb[c];
    }
  }
  for (int c = 0; c < 6; ++c) lam0[c] = out[c];
}

// Adjoint of one accepted step from y0 with size h (stage points recomputed in binary64, the stage
// products in the scalar type of kd).
// Stage points of the step in binary32, as the MIXED forward pass formed them (from the binary32
// high part of its state): the dual products that follow are binary32 anyway.
GLC_HD void dp5_stage_points_f32(const KN<double>& k, const double y0[6], double E, double h, double Y[7][6]) {
  const KN<float> kf = kn_cast<float>(k);
  const float hf = float(h), Ef = float(E);
  float y0f[6], K[7][6];
  for (int c = 0; c < 6; ++c) y0f[c] = float(y0[c]);
  for (int i = 0; i < 7; ++i) {
    float ys[6];
    for (int c = 0; c < 6; ++c) {
      float s = 0.0f;
      for (int j = 0; j < i; ++j) s += dp_a<float>(i, j) * K[j][c];
      ys[c] = y0f[c] + hf * s;
      Y[i][c] = double(ys[c]);
    }
    float d[7], r, vr;
    kn_rhs(kf, ys, Ef, d, r, vr);
    for (int c = 0; c < 6; ++c) K[i][c] = d[c];
  }
}

template <class R>
GLC_HD void dp5_reverse(const KN<double>& k, const KN<Dual<4, R>>& kd, const double y0[6], double E, double h,
                        const double w[7], const double lam[6], double lam0[6], double g[3]) {
  double Y[7][6];
  if constexpr (std::is_same<R, float>::value) {
    dp5_stage_points_f32(k, y0, E, h, Y);
  } else {
    double K[7][6];
    dp5_stage_points(k, y0, E, h, Y, K);
  }
  stages_reverse(kd, Y, E, h, w, lam, lam0, g);
}

// Observables the adjoint differentiates, slot order of dL/dobs: source (hit) radius, frequency
// ratio g, escape theta, escape phi.
constexpr int kObs = 4;

// Adjoint of the terminal step (a surface hit or an escape at dense-output fraction theta of the
// step from y0 with size h). wobs = dL/dobs. Returns false when the event geometry is degenerate.
GLC_HD bool terminal_reverse(const LaneScene& sc, const double y0[6], double E, double h, double theta, double dir,
                             uint32_t term, const double wobs[kObs], double lam0[6], double g[3]) {
  const KN<double>& k = sc.kn;
  const KN<D9> kd = kn_dual(k);
  double Y[7][6], K[7][6], w[7], dw[7];
  dp5_stage_points(k, y0, E, h, Y, K);
  dense_weights_at(theta, w, dw);
  double ys[6], ydot[6];
  for (int c = 0; c < 6; ++c) {
    double s = 0.0, sd = 0.0;
    for (int j = 0; j < 7; ++j) {
      s += w[j] * K[j][c];
      sd += dw[j] * K[j][c];
    }
    ys[c] = y0[c] + h * s;
    ydot[c] = h * sd;
  }
  D9 yd[6];
  for (int c = 0; c < 6; ++c) yd[c] = D9::seed(ys[c], c);
  const D9 Ed = D9::seed(E, kChE);
  double mu[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  D9 ev;
  if (term == GLC_TERM_SURFACE) {
    int gs;
    const D9 r = kn_radius(kd, yd[0], yd[1], yd[2], gs);
    if (gs != kGeomOk) return false;
    D9 gf;
    if (!frequency_ratio(kd.a, kd.q2, kd.a2, sc.frequency, yd, Ed, r, gf)) return false;
    for (int i = 0; i < 9; ++i) mu[i] = wobs[0] * r.d[i] + wobs[1] * gf.d[i];
    ev = yd[2];
  } else if (term == GLC_TERM_ESCAPE) {
    D9 d[7], rr, vr;
    kn_rhs(kd, yd, Ed, d, rr, vr);
    const D9 dx = dir * d[0], dy = dir * d[1], dz = dir * d[2];
    const D9 nrm = g_sqrt(dx * dx + dy * dy + dz * dz);
    const D9 th = g_acos(dz / nrm), ph = g_atan2(dy, dx);
    for (int i = 0; i < 9; ++i) mu[i] = wobs[2] * th.d[i] + wobs[3] * ph.d[i];
    int gs;
    ev = kn_radius(kd, yd[0], yd[1], yd[2], gs);
    if (gs != kGeomOk) return false;
  } else {
    return false;
  }
  // implicit event time: theta* moves with the inputs so that e(y(theta*)) stays 0
  double num = 0.0, den = 0.0;
  for (int c = 0; c < 6; ++c) {
    num += mu[c] * ydot[c];
    den += ev.d[c] * ydot[c];
  }
  if (!(den != 0.0) || !g_finite(den)) return false;
  const double s = num / den;
  for (int i = 0; i < 9; ++i) mu[i] -= s * ev.d[i];
  g[0] += mu[kChE];
  g[1] += mu[kChA];
  g[2] += mu[kChQ2];
  // dense output with theta* fixed (its variation is already folded into mu)
  stages_reverse(kn_dual_vjp(k), Y, E, h, w, mu, lam0, g);
  return true;
}

// Scene constants the initial state of an image ray depends on, in this order: observer event (4),
// four-velocity (4), image right (4), image up (4), arrival (4), metric at the observer (16),
// frequency, tan(fov / 2).
constexpr int kSceneConsts = 38;

GLC_HD void gather_scene_consts(const glc_scene& s, double c[kSceneConsts]) {
  for (int i = 0; i < 4; ++i) {
    c[i] = s.observer_txyz[i];
    c[4 + i] = s.four_velocity[i];
    c[8 + i] = s.image_right[i];
    c[12 + i] = s.image_up[i];
    c[16 + i] = s.arrival[i];
  }
  for (int i = 0; i < 16; ++i) c[20 + i] = s.metric_covariant[i];
  c[36] = s.frequency;
  c[37] = s.tangent_half_fov;
}

// Initial state (t, x, y, z, p_t, p_x, p_y, p_z) of the pinhole sample at (px, py) (pixel index plus
// subpixel offset): the arithmetic of the trace kernels' ray set-up, on scene constants of type T
// (dual numbers carry their derivatives).
template <class T>
GLC_HD void pinhole_state(const T c[kSceneConsts], double px, double py, double W, double H, T st8[8]) {
  const double nx = 2.0 * px / W - 1.0;
  const double ny = 1.0 - 2.0 * py / H;
  const T sx = (W / H) * c[37] * nx;
  const T sy = c[37] * ny;
  const T nrm = T(1.0) / g_hypot(T(1.0), g_hypot(sx, sy));
  T pc[4];
  for (int i = 0; i < 4; ++i) pc[i] = c[36] * (c[4 + i] - (c[8 + i] * sx + c[12 + i] * sy - c[16 + i]) * nrm);
  for (int r = 0; r < 4; ++r) {
    T s = T(0.0);
    for (int q = 0; q < 4; ++q) s += c[20 + 4 * r + q] * pc[q];
    st8[4 + r] = s;
  }
  for (int i = 0; i < 4; ++i) st8[i] = c[i];
}

}  // namespace glc
