// dspw_math.cuh -- precision policy and the per-face mathematics of the
// SP-WENO / DSP-WENO TeCNO stage, templated on the arithmetic type.
//
// FP64 (the plain form) keeps the order of floating-point operations of the
// reference C++ (cited per function) and its translation unit is compiled with
// --fmad=false, so results differ from the reference only where CUDA's
// log/exp/tanh round differently from glibc's.  FP32 uses the hardware
// reciprocal, log2, exp2 and tanh units.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#define DSPW_HD __device__ __forceinline__

namespace dspw {

template <typename T> struct Mth;

template <> struct Mth<double> {
  static DSPW_HD double div(double a, double b) { return a / b; }
  static DSPW_HD double rcp(double a) { return 1.0 / a; }
  static DSPW_HD double log(double a) { return ::log(a); }
  static DSPW_HD double exp(double a) { return ::exp(a); }
  static DSPW_HD double tanh(double a) { return ::tanh(a); }
  static DSPW_HD double sqrt(double a) { return ::sqrt(a); }
  static DSPW_HD double abs(double a) { return ::fabs(a); }
  static DSPW_HD double min(double a, double b) { return ::fmin(a, b); }
  static DSPW_HD double max(double a, double b) { return ::fmax(a, b); }
  static DSPW_HD double cube(double a) { return a * a * a; }
};

template <> struct Mth<float> {
  static DSPW_HD float div(float a, float b) { return __fdividef(a, b); }
  static DSPW_HD float rcp(float a) { return __frcp_rn(a); }
  static DSPW_HD float log(float a) { return __logf(a); }
  static DSPW_HD float exp(float a) { return __expf(a); }
  // 2^a on the special-function unit (one instruction; the FP32 network's
  // last layer is scaled by log2 e so that its softmax needs no other factor)
  static DSPW_HD float exp2(float a) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
    return r;
  }
  static DSPW_HD float tanh(float a) {
    float r;
    asm("tanh.approx.f32 %0, %1;" : "=f"(r) : "f"(a));
    return r;
  }
  static DSPW_HD float sqrt(float a) { return ::sqrtf(a); }
  static DSPW_HD float abs(float a) { return ::fabsf(a); }
  static DSPW_HD float min(float a, float b) { return ::fminf(a, b); }
  static DSPW_HD float max(float a, float b) { return ::fmaxf(a, b); }
  static DSPW_HD float cube(float a) { return a * a * a; }
};

// ---------------------------------------------------------------- log mean --
// logavg, enflo/src/misc_func.h:14-32: (a+b)/2 / F with F = 1 + u/3 + u^2/5 +
// u^3/7 for u = ((xi-1)/(xi+1))^2 < 1e-2, else ln(xi) / (2 f).
template <typename T>
DSPW_HD T logavg(T a, T b) {
  typedef Mth<T> m;
  T xi = m::div(b, a);
  T f = m::div(xi - T(1.0), xi + T(1.0));
  T u = f * f;
  T F;
  if (u < T(1.0e-2)) {
    T u2 = u * u;
    T u3 = u2 * u;
    F = T(1.0) + m::div(u, T(3.0)) + m::div(u2, T(5.0)) + m::div(u3, T(7.0));
  } else {
    F = m::div(m::div(m::log(xi), T(2.0)), f);
  }
  return m::div(T(0.5) * (a + b), F);
}

// --------------------------------------------------------------- SP-WENO --
constexpr double SPW_EPS = 1.0e-13;   // enflo/src/limiter.h:14

// fp, enflo/src/limiter.h:103-118
template <typename T>
DSPW_HD T spw_fp(T t0, T t1) {
  typedef Mth<T> m;
  const T eps = T(SPW_EPS);
  T psi = (m::abs(t0 - T(1.0)) < eps) ? T(0.0) : m::div(T(1) - t1, T(1) - t0);
  return (m::abs(t0 - T(1.0)) > eps && m::abs(psi + T(1.0)) > eps) ? m::div(T(1.0), T(1.0) + psi) : T(1.0);
}

// Cp, enflo/src/limiter.h:153-187
template <typename T>
DSPW_HD void spw_cp(T t0, T t1, T del1, T scale, T& C, T& corr) {
  typedef Mth<T> m;
  const T eps = T(SPW_EPS);
  T psi = (m::abs(t0 - T(1.0)) < eps || m::abs(t1 - T(1.0)) < eps) ? T(0.0) : m::div(T(1) - t1, T(1) - t0);
  corr = T(0.0);
  if (m::abs(psi + T(1.0)) > eps && m::abs(t0 - T(1.0)) > eps && psi < T(0)) {
    T a = spw_fp(t0, t1), b = spw_fp(t1, t0);
    C = m::div(m::div(a, a * a + b * b), T(8.0));
    T mm = m::min(m::abs(m::div(del1, scale)), m::abs(del1));
    corr += m::div(T(-0.25) * m::cube(mm), T(1.0) - t0);
  } else if (m::abs(t0 - T(1.0)) > eps && m::abs(psi + T(1.0)) < eps) {
    C = T(0.0);
  } else if (m::abs(t0 - T(1.0)) < eps || (psi > -eps && m::abs(t0) < T(1) + eps)) {
    C = T(-3.0 / 8.0);
  } else if (psi > -eps && m::abs(t0) > T(1)) {
    C = T(1.0 / 8.0);
  }
}

// The reference's lower-order reconstructions of one component
// (enflo/src/reconstruct.cc): kind 4 first order (:14-30), 5 unlimited MUSCL
// with kappa = 1/3 (:35-56), 6 / 7 MUSCL with the minmod / minabs limited slope
// 0.5 * limiter(outer jump, face jump) (:61-79, limited_slope :162-186,
// minmod / minabs enflo/src/limiter.h:22-57), 8 point-wise ENO of level 2
// (:84-110).
template <typename T>
DSPW_HD T eno2_side(T q0, T q1, T q2) {
  // eno_pw with eno_level 2 (enflo/src/limiter.h:63-96, ENO2_COEF :8-9): the
  // stencil shifts left when the right divided difference is larger
  typedef Mth<T> m;
  T res = T(0);
  if (m::abs(q2 - q1) > m::abs(q1 - q0)) {
    res += T(-0.5) * q0;
    res += T(1.5) * q1;
  } else {
    res += T(0.5) * q1;
    res += T(0.5) * q2;
  }
  return res;
}

// eno_pw with eno_level 3 (enflo/src/limiter.h:63-96, ENO3_COEF :10-12) of
// five values: the stencil shifts left once for the first-order and once for
// the second-order divided difference whose right member is the larger in
// magnitude, then the three-point interpolation of the chosen stencil, summed
// in the reference's order.  Selects, not indexing: no local memory.
template <typename T>
DSPW_HD T eno3_side(T q0, T q1, T q2, T q3, T q4) {
  typedef Mth<T> m;
  const T d10 = q1 - q0, d11 = q2 - q1, d12 = q3 - q2, d13 = q4 - q3;
  const T d20 = d11 - d10, d21 = d12 - d11, d22 = d13 - d12;
  const bool s1 = m::abs(d12) > m::abs(d11);
  // second order: r = 0 compares d22 with d21, r = 1 compares d21 with d20
  const bool s2 = s1 ? (m::abs(d21) > m::abs(d20)) : (m::abs(d22) > m::abs(d21));
  const int r = (int)s1 + (int)s2;
  T a, b, c, x, y, z;
  if (r == 0) { a = T(0.375); b = T(0.75); c = T(-0.125); x = q2; y = q3; z = q4; }
  else if (r == 1) { a = T(-0.125); b = T(0.75); c = T(0.375); x = q1; y = q2; z = q3; }
  else { a = T(0.375); b = T(-1.25); c = T(1.875); x = q0; y = q1; z = q2; }
  T res = T(0);
  res += a * x;
  res += b * y;
  res += c * z;
  return res;
}

// point-wise ENO of level 3 at the middle face of a six-cell stencil
// (reconstruct_eno_pw, enflo/src/reconstruct.cc:84-110): left state from
// s0..s4, right state from s5..s1
template <typename T>
DSPW_HD void eno3_recon(T s0, T s1, T s2, T s3, T s4, T s5, T& recl, T& recr) {
  recl = eno3_side<T>(s0, s1, s2, s3, s4);
  recr = eno3_side<T>(s5, s4, s3, s2, s1);
}

template <typename T>
DSPW_HD void simple_recon(int kind, T s0, T s1, T s2, T s3, T& recl, T& recr) {
  typedef Mth<T> m;
  if (kind == 4) { recl = s1; recr = s2; return; }
  if (kind == 8) { recl = eno2_side<T>(s0, s1, s2); recr = eno2_side<T>(s3, s2, s1); return; }
  const T ds = s2 - s1, dl = s1 - s0, dr = s3 - s2;
  if (kind == 5) {
    const T K = T(1.0 / 3.0);
    recl = s1 + (dl * (T(1.0) - K) + ds * (T(1.0) + K)) * T(0.25);
    recr = s2 - (dr * (T(1.0) - K) + ds * (T(1.0) + K)) * T(0.25);
    return;
  }
  T sl, sr;
  if (kind == 6) {
    sl = (dl * ds > T(0.0)) ? m::min(m::abs(dl), m::abs(ds)) * ((dl < T(0)) ? T(-1) : T(1)) : T(0.0);
    sr = (dr * ds > T(0.0)) ? m::min(m::abs(dr), m::abs(ds)) * ((dr < T(0)) ? T(-1) : T(1)) : T(0.0);
  } else {
    sl = (m::abs(dl) > m::abs(ds)) ? ds : dl;
    sr = (m::abs(dr) > m::abs(ds)) ? ds : dr;
  }
  recl = s1 + T(0.5) * sl;
  recr = s2 - T(0.5) * sr;
}

// sp_weno_rec, enflo/src/limiter.h:193-252.  corr: 0 sp_weno, 1 sp_wenoc, 2 sp_weno_corr2
template <typename T>
DSPW_HD void sp_weno(T s0, T s1, T s2, T s3, int corr, T& recl, T& recr) {
  typedef Mth<T> m;
  T del0 = s1 - s0, del1 = s2 - s1, del2 = s3 - s2;
  if (m::abs(del1) < T(SPW_EPS)) {
    recl = s1;
    recr = s2;
    return;
  }
  T tp = m::div(del0, del1);
  T tm = m::div(del2, del1);
  T scale = T(0.5) * (m::abs(s1) + m::abs(s2));
  T C1 = 0, C2 = 0, C1c = 0, C2c = 0;
  spw_cp(tp, tm, del1, scale, C1, C1c);
  spw_cp(tm, tp, del1, scale, C2, C2c);
  if (corr > 0) {
    T C1n = C1 + C1c, C2n = C2 + C2c;
    if (corr == 1) { C1 = C1n; C2 = C2n; }
    C1 = m::min(m::max(C1, T(-3.0 / 8.0)), T(1.0 / 8.0));
    C2 = m::min(m::max(C2, T(-3.0 / 8.0)), T(1.0 / 8.0));
  }
  T w0 = T(3.0 / 4.0) + T(2) * C1;
  T w0t = T(1.0 / 4.0) - T(2) * C2;
  recl = w0 * T(0.5) * (s1 + s2) + (T(1) - w0) * (T(-0.5) * s0 + T(1.5) * s1);
  recr = (T(1) - w0t) * T(0.5) * (s1 + s2) + w0t * (T(-0.5) * s3 + T(1.5) * s2);
}

// -------------------------------------------------------------- DSP-WENO --
// Network weights as read by Neural_Network::load_network
// (enflo/src/neural_network.cc:82-130): W[l][out][in], b[l][out].
struct NetParams {
  double w[4][5][5];
  double b[4][5];
  // FP32 copies for the tensor-core form; the last layer (l = 3) times log2 e,
  // so that its logits are base-2 (nn_finish)
  float wf[4][5][5];
  float bf[4][5];
  float feat_lo[5], feat_hi[5];   // training box of the network inputs (FP32 form fallback)
  int use_box;
};

// The network's inputs: scale (neural_network.cc:300-313), theta and deltas;
// tm, tp and the largest delta md feed the vertices (nn_vertices)
template <typename T>
DSPW_HD void nn_inputs(T u0, T u1, T u2, T u3, T feat[5], T& tm_out, T& tp_out, T& md_out) {
  typedef Mth<T> m;
  T mx = T(1.0);
  mx = m::max(mx, m::abs(u0)); mx = m::max(mx, m::abs(u1));
  mx = m::max(mx, m::abs(u2)); mx = m::max(mx, m::abs(u3));
  T c0, c1, c2, c3, tm, tp;
  if constexpr (sizeof(T) == 4) {
    // FP32 form: one reciprocal per divisor, shared by its quotients
    const T rm = m::div(T(1), mx);
    c0 = u0 * rm; c1 = u1 * rm; c2 = u2 * rm; c3 = u3 * rm;
    const T r21 = m::div(T(1), c2 - c1);
    tm = (c3 - c2) * r21;
    tp = (c1 - c0) * r21;
  } else {
    c0 = m::div(u0, mx); c1 = m::div(u1, mx); c2 = m::div(u2, mx); c3 = m::div(u3, mx);
    tm = m::div(c3 - c2, c2 - c1);
    tp = m::div(c1 - c0, c2 - c1);
  }
  T d1 = m::abs(c1 - c0), d2 = m::abs(c2 - c1), d3 = m::abs(c3 - c2);
  T md = m::max(m::max(d1, d2), d3);
  feat[0] = m::tanh(tm); feat[1] = m::tanh(tp);
  feat[2] = d1; feat[3] = d2; feat[4] = d3;
  tm_out = tm;
  tp_out = tp;
  md_out = md;
}

// The feasible-region vertices of compute_vertices with vertex_mode 2 /
// permutation 2 (neural_network.cc:135-260) from tm, tp and md
template <typename T>
DSPW_HD void nn_vertices(T tm, T tp, T md, T vx[5], T vy[5]) {
  typedef Mth<T> m;
  const T thr = T(1e-8);
  T psi_p, psi_m;
  if constexpr (sizeof(T) == 4) {
    const T a = T(1) - tm, b = T(1) - tp;
    psi_p = a * m::div(T(1), b);
    psi_m = b * m::div(T(1), a);
  } else {
    psi_p = m::div(T(1) - tm, T(1) - tp);
    psi_m = m::div(T(1), psi_p);
  }
  T g1 = m::min(md, T(1.0 / 8.0));
  T g2 = -m::min(md, T(3.0 / 8.0));
  T x1 = T(1.0 / 8.0) * (T(1) + psi_p) - g1 * psi_p;
  T y1 = T(1.0 / 8.0) * (T(1) + psi_m) - g2 * psi_m;
  T x2 = T(1.0 / 8.0) * (T(1) + psi_p) - g2 * psi_p;
  T y2 = T(1.0 / 8.0) * (T(1) + psi_m) - g1 * psi_m;
  const T e = T(1.0 / 8.0), t = T(-3.0 / 8.0), o = T(-1.0 / 8.0);
#define DSPW_SET5(a, v0, v1, v2, v3, v4) { a[0] = v0; a[1] = v1; a[2] = v2; a[3] = v3; a[4] = v4; }
  if ((tm - T(1.0)) > thr && (tp - T(1.0)) > thr) {
    DSPW_SET5(vx, e, e, e, e, e) DSPW_SET5(vy, e, e, e, e, e)
  } else if ((tm - T(1.0)) > thr && (tp - T(1.0)) < T(-1.0) * thr) {
    if (psi_p < T(-1.0)) {
      if (x1 < g2) {
        T nx = m::div((psi_m * psi_m) + psi_m, T(8) * ((psi_m * psi_m) + T(1)));
        T ny = T(1.0 / 8.0) * (T(1) + psi_m) - nx * psi_m;
        DSPW_SET5(vx, nx, nx, nx, nx, nx) DSPW_SET5(vy, ny, ny, ny, ny, ny)
      } else {
        T cx = m::div(T(2) * g2 + x1, T(3.0)), cy = m::div(T(2) * g1 + y2, T(3.0));
        DSPW_SET5(vx, g2, x1, g2, cx, cx) DSPW_SET5(vy, g1, g1, y2, cy, cy)
      }
    } else {
      if (y2 < g2) { DSPW_SET5(vx, g2, g1, g2, g1, T(0)) DSPW_SET5(vy, g1, g1, g2, g2, T(0)) }
      else { DSPW_SET5(vx, g2, g1, g2, g1, x2) DSPW_SET5(vy, g1, g1, g2, y2, g2) }
    }
  } else if ((tm - T(1.0)) < T(-1.0) * thr && (tp - T(1.0)) > thr) {
    if (psi_p < T(-1.0)) {
      if (x1 < g2) { DSPW_SET5(vx, g2, g1, g2, g1, T(0)) DSPW_SET5(vy, g1, g1, g2, g2, T(0)) }
      else { DSPW_SET5(vx, g1, g1, g2, x1, g2) DSPW_SET5(vy, g2, g1, g2, g1, y1) }
    } else {
      if (y2 < g2) {
        T nx = m::div((psi_m * psi_m) + psi_m, T(8) * ((psi_m * psi_m) + T(1)));
        T ny = T(1.0 / 8.0) * (T(1) + psi_m) - nx * psi_m;
        DSPW_SET5(vx, nx, nx, nx, nx, nx) DSPW_SET5(vy, ny, ny, ny, ny, ny)
      } else {
        T cx = m::div(T(2) * g1 + x1, T(3.0)), cy = m::div(T(2) * g2 + y2, T(3.0));
        DSPW_SET5(vx, g1, x1, g1, cx, cx) DSPW_SET5(vy, g2, g2, y2, cy, cy)
      }
    }
  } else if (m::abs(tm - T(1.0)) < thr && (tp - T(1.0)) > thr) {
    DSPW_SET5(vx, e, e, e, e, e) DSPW_SET5(vy, t, e, e, t, o)
  } else if (m::abs(tp - T(1.0)) < thr && (tm - T(1.0)) > thr) {
    DSPW_SET5(vx, e, e, t, t, o) DSPW_SET5(vy, e, e, e, e, e)
  } else {
    DSPW_SET5(vx, e, e, t, t, o) DSPW_SET5(vy, e, t, t, e, o)
  }
#undef DSPW_SET5
}

// inputs and vertices of one stencil (the reference's forward computes both
// before the network)
template <typename T>
DSPW_HD void nn_features(T u0, T u1, T u2, T u3, T feat[5], T vx[5], T vy[5]) {
  T tm, tp, md;
  nn_inputs<T>(u0, u1, u2, u3, feat, tm, tp, md);
  nn_vertices<T>(tm, tp, md, vx, vy);
}

// softmax (neural_network.cc:276-295) and the vertex combination / weights /
// compute_recon (:62-76, :320-325) from the 5 output logits.  The FP32 form's
// logits are in base 2 (its last layer carries the factor log2 e, NetParams),
// so its softmax weights are 2^(lg - max): the same weights as e^(lg' - max')
// of the unscaled logits lg'.
template <typename T>
DSPW_HD void nn_finish(const T lg[5], const T vx[5], const T vy[5], T u0, T u1, T u2, T u3, T& recl,
                       T& recr) {
  typedef Mth<T> m;
  T s[5];
  T mxv = T(0.0);
#pragma unroll
  for (int i = 0; i < 5; i++) mxv = m::max(mxv, lg[i]);
  T sum = T(0);
#pragma unroll
  for (int i = 0; i < 5; i++) {
    if constexpr (sizeof(T) == 4) s[i] = m::exp2(lg[i] - mxv);
    else s[i] = m::exp(lg[i] - mxv);
    sum += s[i];
  }
  T C1 = T(0.0), C2 = T(0.0);
  if constexpr (sizeof(T) == 4) {
    // FP32 form: normalise the two weighted sums instead of the five weights
#pragma unroll
    for (int i = 0; i < 5; i++) { C1 += s[i] * vx[i]; C2 += s[i] * vy[i]; }
    const T rs = m::div(T(1), sum);
    C1 *= rs;
    C2 *= rs;
  } else {
#pragma unroll
    for (int i = 0; i < 5; i++) s[i] = m::div(s[i], sum);
#pragma unroll
    for (int i = 0; i < 5; i++) { C1 += s[i] * vx[i]; C2 += s[i] * vy[i]; }
  }
  T w1 = T(1.0 / 4.0) - T(2) * C1;
  T tw0 = T(1.0 / 4.0) - T(2) * C2;
  T wt0 = T(1.0) - w1, wt3 = T(1.0) - tw0;
  recl = wt0 * T(0.5) * (u1 + u2) + w1 * (T(-0.5) * u0 + T(1.5) * u1);
  recr = wt3 * T(0.5) * (u1 + u2) + tw0 * (T(-0.5) * u3 + T(1.5) * u2);
}

// scalar-lane MLP (neural_network.cc:40-60), used by the FP64 form
DSPW_HD void nn_layers_fp64(const NetParams& P, double st[5]) {
  double tmp[5];
#pragma unroll
  for (int l = 0; l < 4; l++) {
#pragma unroll
    for (int j = 0; j < 5; j++) {
      double dot = 0.0;
#pragma unroll
      for (int k = 0; k < 5; k++) dot += P.w[l][j][k] * st[k];
      tmp[j] = dot;
    }
#pragma unroll
    for (int j = 0; j < 5; j++) st[j] = tmp[j] + P.b[l][j];
    if (l != 3) {
#pragma unroll
      for (int j = 0; j < 5; j++) st[j] = ::fmax(0.0, st[j]);
    }
  }
}

// Neural_Network::forward with the |u2-u1| < 1e-15 guard of
// reconstruct_sp_weno_dl (enflo/src/reconstruct.cc:138-157), FP64
DSPW_HD void dsp_weno_fp64(const NetParams& P, double u0, double u1, double u2, double u3, double& l,
                           double& r) {
  if (::fabs(u2 - u1) < 1e-15) { l = 0.0; r = 0.0; return; }
  double st[5], vx[5], vy[5];
  nn_features<double>(u0, u1, u2, u3, st, vx, vy);
  nn_layers_fp64(P, st);
  nn_finish<double>(st, vx, vy, u0, u1, u2, u3, l, r);
}

}  // namespace dspw
