/*
 * dspw_oracle.c -- TEST INFRASTRUCTURE (the checker, never the product).
 *
 * Plain-C FP64 restatement of the reference's per-stage path.  Every function
 * names the reference file:line it restates and keeps that code's order of
 * floating-point operations, so that compiled like the reference (gcc -O3, no
 * FMA contraction) it reproduces the reference bit for bit.  Used by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg only.
 */
#include "dspw_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ghost width of the state `s` in scope: max(flux_ng, rec_ng), 3 for eno 3 and
 * 2 otherwise (enflo/src/parameter.cc:156-206,315-318, enflo/src/fv.cc:26) */
#define NG (s->ng)
#define SPW_EPS 1.0e-13       /* enflo/src/limiter.h:14 */
#define NN_THRESHOLD 1e-8     /* enflo/src/neural_network.cc:137 */

static const double ARK[3] = {0.0, 3.0 / 4.0, 1.0 / 3.0};   /* enflo/src/ext_constants.h:7 */
static const double BRK[3] = {1.0, 1.0 / 4.0, 2.0 / 3.0};   /* enflo/src/ext_constants.h:8 */
static const double JRK[4] = {1.0 / 4.0, 1.0 / 3.0, 1.0 / 2.0, 1.0};   /* jameson_rks, :9 */
static const double RK4C[4] = {1.0, 1.0 / 2.0, 1.0 / 2.0, 1.0};        /* rk4_rks, :10 */

struct or_state {
  dspw_desc d;
  int scalar, nvar;
  int ng;                       /* ghost width; face stencils hold 2 ng cells */
  int nx, ny, nz, px, py, pz;   /* interior and padded sizes */
  double dx, dy, dz;
  double *P, *V;                /* padded primitive / entropy variables, 5 per cell */
  double *U, *Uold, *R;         /* interior conserved, 5 per cell (scalar: 1 used) */
  double* R2;                   /* classic RK4: weighted sum of the stage residuals */
  double ke_diss_pr;            /* -sum(|u|^2/2 R_mass + u.R_mom) of the last inviscid residual */
  double ke_diss_stress;        /* viscous-stress KE dissipation of the last viscous residual */
  double time, dt, t_interval, t_save;
  int iter;
};

static inline size_t pidx(const or_state* s, int i, int j, int k) {  /* padded coords */
  return ((size_t)k * s->py + j) * s->px + i;
}
static inline size_t cidx(const or_state* s, int i, int j, int k) {  /* interior coords */
  return ((size_t)k * s->ny + j) * s->nx + i;
}

/* ---------------------------------------------------------------- helpers -- */

/* logavg, enflo/src/misc_func.h:14-32 */
double or_logavg(double a, double b) {
  double xi = b / a;
  double f = (xi - 1.0) / (xi + 1.0);
  double u = f * f;
  double F;
  if (u < 1.0e-2) {
    double u2 = u * u;
    double u3 = u2 * u;
    F = 1.0 + u / 3.0 + u2 / 5.0 + u3 / 7.0;
  } else {
    F = log(xi) / 2.0 / f;
  }
  return 0.5 * (a + b) / F;
}

static inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline double sq3(const double* a) { return a[0] * a[0] + a[1] * a[1] + a[2] * a[2]; }

/* fp, enflo/src/limiter.h:103-118 */
static double spw_fp(double theta0, double theta1) {
  double psi, val;
  if (fabs(theta0 - 1.0) < SPW_EPS) psi = 0.0;
  else psi = (1 - theta1) / (1 - theta0);
  if (fabs(theta0 - 1.0) > SPW_EPS && fabs(psi + 1.0) > SPW_EPS) val = 1.0 / (1.0 + psi);
  else val = 1.0;
  return val;
}

/* Cp, enflo/src/limiter.h:153-187 */
static void spw_cp(double theta0, double theta1, double del1, double scale, double* C, double* corr) {
  double psi;
  if (fabs(theta0 - 1.0) < SPW_EPS || fabs(theta1 - 1.0) < SPW_EPS) psi = 0.0;
  else psi = (1 - theta1) / (1 - theta0);
  *corr = 0.0;
  if (fabs(psi + 1.0) > SPW_EPS && fabs(theta0 - 1.0) > SPW_EPS && psi < 0) {
    double a = spw_fp(theta0, theta1), b = spw_fp(theta1, theta0);
    *C = (a / (pow(a, 2.0) + pow(b, 2.0))) / 8.0;
    double m = fmin(fabs(del1 / scale), fabs(del1));
    *corr += -0.25 * pow(m, 3.0) / (1.0 - theta0);
  } else if (fabs(theta0 - 1.0) > SPW_EPS && fabs(psi + 1.0) < SPW_EPS) {
    *C = 0.0;
  } else if (fabs(theta0 - 1.0) < SPW_EPS || (psi > -SPW_EPS && fabs(theta0) < 1 + SPW_EPS)) {
    *C = -3.0 / 8.0;
  } else if (psi > -SPW_EPS && fabs(theta0) > 1) {
    *C = 1.0 / 8.0;
  }
  /* else: the reference prints a warning and leaves C unchanged */
}

/* sp_weno_rec, enflo/src/limiter.h:193-252 */
void or_sp_weno(const double s[4], int corr_type, double* recl, double* recr) {
  double del0 = s[1] - s[0];
  double del1 = s[2] - s[1];
  double del2 = s[3] - s[2];
  if (fabs(del1) < SPW_EPS) {
    *recl = s[1];
    *recr = s[2];
    return;
  }
  double tp = del0 / del1;
  double tm = del2 / del1;
  double scale = 0.5 * (fabs(s[1]) + fabs(s[2]));
  double C1 = 0, C2 = 0, C1c = 0, C2c = 0;
  spw_cp(tp, tm, del1, scale, &C1, &C1c);
  spw_cp(tm, tp, del1, scale, &C2, &C2c);
  if (corr_type > 0) {
    double C1n = C1 + C1c, C2n = C2 + C2c;
    if (corr_type == 1) { C1 = C1n; C2 = C2n; }
    C1 = fmin(fmax(C1, -3.0 / 8.0), 1.0 / 8.0);
    C2 = fmin(fmax(C2, -3.0 / 8.0), 1.0 / 8.0);
  }
  double w0 = 3.0 / 4.0 + 2 * C1;
  double w0t = 1.0 / 4.0 - 2 * C2;
  *recl = w0 * 0.5 * (s[1] + s[2]) + (1 - w0) * (-0.5 * s[0] + 1.5 * s[1]);
  *recr = (1 - w0t) * 0.5 * (s[1] + s[2]) + w0t * (-0.5 * s[3] + 1.5 * s[2]);
}

/* ------------------------------------------------------------ DSP-WENO net -- */

/* compute_vertices with vertex_mode 2 and permutation 2, enflo/src/neural_network.cc:135-260 */
static void nn_vertices(double tm, double tp, double max_delta, double vx[5], double vy[5]) {
  const double thr = NN_THRESHOLD;
  double psi_p = (1 - tm) / (1 - tp);
  double psi_m = 1 / psi_p;
  double g1 = fmin(max_delta, 1.0 / 8.0);
  double g2 = -fmin(max_delta, 3.0 / 8.0);
  double x1 = 1.0 / 8.0 * (1 + psi_p) - g1 * psi_p;
  double y1 = 1.0 / 8.0 * (1 + psi_m) - g2 * psi_m;
  double x2 = 1.0 / 8.0 * (1 + psi_p) - g2 * psi_p;
  double y2 = 1.0 / 8.0 * (1 + psi_m) - g1 * psi_m;
  const double e = 1.0 / 8.0, t = -3.0 / 8.0, o = -1.0 / 8.0;
#define SET5(a, v0, v1, v2, v3, v4) do { a[0] = v0; a[1] = v1; a[2] = v2; a[3] = v3; a[4] = v4; } while (0)
  if ((tm - 1.0) > thr && (tp - 1.0) > thr) {
    SET5(vx, e, e, e, e, e); SET5(vy, e, e, e, e, e);
  } else if ((tm - 1.0) > thr && (tp - 1.0) < -1.0 * thr) {
    if (psi_p < -1.0) {
      if (x1 < g2) {
        double nxv = ((psi_m * psi_m) + psi_m) / (8 * ((psi_m * psi_m) + 1));
        double nyv = 1.0 / 8.0 * (1 + psi_m) - nxv * psi_m;
        SET5(vx, nxv, nxv, nxv, nxv, nxv); SET5(vy, nyv, nyv, nyv, nyv, nyv);
      } else {
        double cx = (2 * g2 + x1) / 3.0, cy = (2 * g1 + y2) / 3.0;
        SET5(vx, g2, x1, g2, cx, cx); SET5(vy, g1, g1, y2, cy, cy);
      }
    } else {
      if (y2 < g2) { SET5(vx, g2, g1, g2, g1, 0.0); SET5(vy, g1, g1, g2, g2, 0.0); }
      else { SET5(vx, g2, g1, g2, g1, x2); SET5(vy, g1, g1, g2, y2, g2); }
    }
  } else if ((tm - 1.0) < -1.0 * thr && (tp - 1.0) > thr) {
    if (psi_p < -1.0) {
      if (x1 < g2) { SET5(vx, g2, g1, g2, g1, 0.0); SET5(vy, g1, g1, g2, g2, 0.0); }
      else { SET5(vx, g1, g1, g2, x1, g2); SET5(vy, g2, g1, g2, g1, y1); }
    } else {
      if (y2 < g2) {
        double nxv = ((psi_m * psi_m) + psi_m) / (8 * ((psi_m * psi_m) + 1));
        double nyv = 1.0 / 8.0 * (1 + psi_m) - nxv * psi_m;
        SET5(vx, nxv, nxv, nxv, nxv, nxv); SET5(vy, nyv, nyv, nyv, nyv, nyv);
      } else {
        double cx = (2 * g1 + x1) / 3.0, cy = (2 * g2 + y2) / 3.0;
        SET5(vx, g1, x1, g1, cx, cx); SET5(vy, g2, g2, y2, cy, cy);
      }
    }
  } else if (fabs(tm - 1.0) < thr && (tp - 1.0) > thr) {
    SET5(vx, e, e, e, e, e); SET5(vy, t, e, e, t, o);
  } else if (fabs(tp - 1.0) < thr && (tm - 1.0) > thr) {
    SET5(vx, e, e, t, t, o); SET5(vy, e, e, e, e, e);
  } else {
    SET5(vx, e, e, t, t, o); SET5(vy, e, t, t, e, o);
  }
#undef SET5
}

/* scale + features + vertices, enflo/src/neural_network.cc:21-37,300-313 */
void or_nn_features(const double u[4], double feat[5], double vx[5], double vy[5]) {
  double c[4];
  double max_val = 1.0;
  for (int i = 0; i < 4; i++) c[i] = u[i];
  for (int i = 0; i < 4; i++) max_val = fmax(max_val, fabs(c[i]));
  for (int i = 0; i < 4; i++) c[i] /= max_val;
  double tm = (c[3] - c[2]) / (c[2] - c[1]);
  double tp = (c[1] - c[0]) / (c[2] - c[1]);
  double d1 = fabs(c[1] - c[0]);
  double d2 = fabs(c[2] - c[1]);
  double d3 = fabs(c[3] - c[2]);
  double max_del = fmax(fmax(d1, d2), d3);
  feat[0] = tanh(tm);
  feat[1] = tanh(tp);
  feat[2] = d1;
  feat[3] = d2;
  feat[4] = d3;
  nn_vertices(tm, tp, max_del, vx, vy);
}

/* Neural_Network::forward, enflo/src/neural_network.cc:16-77 (relu :265-271,
 * softmax :276-295, compute_recon :320-325) */
void or_nn_forward(const dspw_desc* d, const double u[4], double* recl, double* recr) {
  double st[5], vx[5], vy[5], tmp[5];
  or_nn_features(u, st, vx, vy);
  for (int l = 0; l < 4; l++) {
    for (int j = 0; j < 5; j++) {
      double dot = 0.0;
      for (int k = 0; k < 5; k++) dot += d->nn_w[l][j][k] * st[k];
      tmp[j] = dot;
    }
    for (int j = 0; j < 5; j++) st[j] = tmp[j] + d->nn_b[l][j];
    if (l != 3)
      for (int j = 0; j < 5; j++) st[j] = fmax(0.0, st[j]);
  }
  double max_val = 0.0;
  for (int i = 0; i < 5; i++) max_val = fmax(max_val, st[i]);
  double sum = 0;
  for (int i = 0; i < 5; i++) { st[i] = exp(st[i] - max_val); sum += st[i]; }
  for (int i = 0; i < 5; i++) st[i] /= sum;
  double C1 = 0.0, C2 = 0.0;
  for (int i = 0; i < 5; i++) { C1 += st[i] * vx[i]; C2 += st[i] * vy[i]; }
  double w1 = 1.0 / 4.0 - 2 * C1;
  double tw0 = 1.0 / 4.0 - 2 * C2;
  double w[4] = {1.0 - w1, w1, tw0, 1.0 - tw0};
  *recl = w[0] * 0.5 * (u[1] + u[2]) + w[1] * (-0.5 * u[0] + 1.5 * u[1]);
  *recr = w[3] * 0.5 * (u[1] + u[2]) + w[2] * (-0.5 * u[3] + 1.5 * u[2]);
}

/* eno_pw with eno_level 3 on five values q[0..4] (enflo/src/limiter.h:63-96,
 * ENO3_COEF :10-12): divided differences of order 1 and 2, the stencil shifted
 * left once per order whose right difference is the larger in magnitude, then
 * the three-point interpolation of the chosen stencil. */
static double eno3_pw(const double q[5]) {
  static const double coef[3][3] = {{0.375, -1.25, 1.875}, {-0.125, 0.75, 0.375}, {0.375, 0.75, -0.125}};
  double dd1[4], dd2[3];
  for (int j = 0; j < 4; j++) dd1[j] = q[j + 1] - q[j];
  for (int j = 0; j < 3; j++) dd2[j] = dd1[j + 1] - dd1[j];
  int r = 0;
  if (fabs(dd1[2 - r]) > fabs(dd1[1 - r])) r++;
  if (fabs(dd2[2 - r]) > fabs(dd2[1 - r])) r++;
  double res = 0;
  for (int i = 0; i < 3; i++) res += coef[2 - r][i] * q[2 - r + i];
  return res;
}

/* reconstruct dispatch for one component, enflo/src/reconstruct.cc:115-157,192-239.
 * s holds the face stencil: 4 values, 6 for eno 3 (reconstruct_eno_pw,
 * reconstruct.cc:84-110: left from s[0..4], right from s[5..1]). */
static void reconstruct1(const dspw_desc* d, const double* s, double* l, double* r) {
  if (d->recon == DSPW_REC_ENO3) {
    const double L[5] = {s[0], s[1], s[2], s[3], s[4]}, Rr[5] = {s[5], s[4], s[3], s[2], s[1]};
    *l = eno3_pw(L);
    *r = eno3_pw(Rr);
    return;
  }
  switch (d->recon) {
    case DSPW_REC_SP_WENO: or_sp_weno(s, 0, l, r); break;
    case DSPW_REC_SP_WENOC: or_sp_weno(s, 1, l, r); break;
    case DSPW_REC_SP_WENO_CORR2: or_sp_weno(s, 2, l, r); break;
    case DSPW_REC_SP_WENO_DL:
      if (fabs(s[2] - s[1]) < 1e-15) { *l = 0.0; *r = 0.0; }
      else or_nn_forward(d, s, l, r);
      break;
    case DSPW_REC_FIRST:            /* reconstruct_first, enflo/src/reconstruct.cc:14-30 */
      *l = s[1]; *r = s[2]; break;
    case DSPW_REC_SECOND: {         /* reconstruct_second_muscl, kappa = 1/3 */
      double ds = s[2] - s[1], dl = s[1] - s[0], dr = s[3] - s[2];
      const double K = 1.0 / 3.0;
      *l = s[1] + (dl * (1.0 - K) + ds * (1.0 + K)) * 0.25;
      *r = s[2] - (dr * (1.0 - K) + ds * (1.0 + K)) * 0.25;
      break;
    }
    case DSPW_REC_MINMOD:
    case DSPW_REC_MINABS: {         /* reconstruct_muscl_limited + limited_slope */
      double ds = s[2] - s[1], dl = s[1] - s[0], dr = s[3] - s[2];
      double sl, sr;
      if (d->recon == DSPW_REC_MINMOD) {
        sl = (dl * ds > 0.0) ? fmin(fabs(dl), fabs(ds)) * ((dl < 0) ? -1 : 1) : 0.0;
        sr = (dr * ds > 0.0) ? fmin(fabs(dr), fabs(ds)) * ((dr < 0) ? -1 : 1) : 0.0;
      } else {
        sl = (fabs(dl) > fabs(ds)) ? ds : dl;
        sr = (fabs(dr) > fabs(ds)) ? ds : dr;
      }
      *l = s[1] + 0.5 * sl;
      *r = s[2] - 0.5 * sr;
      break;
    }
    case DSPW_REC_ENO2: {           /* reconstruct_eno_pw + eno_pw, eno_level 2 (limiter.h:63-96) */
      const double c[2][2] = {{-0.5, 1.5}, {0.5, 0.5}};   /* ENO2_COEF, limiter.h:8-9 */
      const double L[3] = {s[0], s[1], s[2]}, Rr[3] = {s[3], s[2], s[1]};
      const double* st[2] = {L, Rr};
      double out[2];
      for (int side = 0; side < 2; side++) {
        const double* q = st[side];
        int r = 0;
        if (fabs(q[2] - q[1]) > fabs(q[1] - q[0])) r++;
        double res = 0;
        for (int i = 0; i < 2; i++) res += c[1 - r][i] * q[1 - r + i];
        out[side] = res;
      }
      *l = out[0]; *r = out[1];
      break;
    }
    default: *l = s[1]; *r = s[2];
  }
}

/* ------------------------------------------------------------ Euler pieces -- */

/* kepec_flux, enflo/src/kepec.cc:10-48.  Pl,Pr: (rho,u,v,w,p). */
static void kepec_flux(const dspw_desc* d, const double* Pl, const double* Pr, const double* n,
                       double area, double* F) {
  double R = d->gas_const, G = d->gamma;
  double rhol = Pl[0], rhor = Pr[0];
  double rho = or_logavg(rhol, rhor);
  double templ = Pl[4] / (R * rhol);
  double tempr = Pr[4] / (R * rhor);
  double vel2 = 0.5 * (sq3(Pl + 1) + sq3(Pr + 1));
  double betal = 0.5 / (R * templ);
  double betar = 0.5 / (R * tempr);
  double beta = or_logavg(betal, betar);
  double p = 0.5 * (rhol + rhor) / (betal + betar);
  double vel[3] = {Pl[1] * 0.5 + Pr[1] * 0.5, Pl[2] * 0.5 + Pr[2] * 0.5, Pl[3] * 0.5 + Pr[3] * 0.5};
  double vn = dot3(vel, n);
  F[0] = rho * vn;
  for (int c = 0; c < 3; c++) F[1 + c] = n[c] * p + vel[c] * F[0];
  F[4] = 0.5 * (1.0 / ((G - 1.0) * beta) - vel2) * F[0] + dot3(F + 1, vel);
  for (int c = 0; c < 5; c++) F[c] *= area;
}

/* Enthalpy, enflo/src/fv.cc:565-569 */
static double enthalpy(const dspw_desc* d, const double* P) {
  double a = sqrt(d->gamma * P[4] / P[0]);
  return a * a / (d->gamma - 1.0) + 0.5 * sq3(P + 1);
}

/* kep_flux, enflo/src/kep.cc:10-44 */
static void kep_flux(const dspw_desc* d, const double* Pl, const double* Pr, const double* n, double area,
                     double* F) {
  double rho = 0.5 * (Pl[0] + Pr[0]);
  double p = 0.5 * (Pl[4] + Pr[4]);
  double vel[3] = {Pl[1] * 0.5 + Pr[1] * 0.5, Pl[2] * 0.5 + Pr[2] * 0.5, Pl[3] * 0.5 + Pr[3] * 0.5};
  double H = 0.5 * (enthalpy(d, Pl) + enthalpy(d, Pr));
  double vn = dot3(vel, n);
  F[0] = rho * vn;
  for (int c = 0; c < 3; c++) F[1 + c] = n[c] * p + vel[c] * F[0];
  F[4] = rho * H * vn;
  for (int c = 0; c < 5; c++) F[c] *= area;
}

/* roe_ec_flux, enflo/src/roe_ec.cc:10-69 */
static void roe_ec_flux(const dspw_desc* d, const double* Pl, const double* Pr, const double* n,
                        double area, double* F) {
  double G = d->gamma;
  double rhol = Pl[0], rhor = Pr[0], pl = Pl[4], pr = Pr[4];
  double bl = sqrt(rhol / pl);
  double br = sqrt(rhor / pr);
  double z1b = 0.5 * (bl + br);
  double zvb[3] = {Pl[1] * (0.5 * bl) + Pr[1] * (0.5 * br), Pl[2] * (0.5 * bl) + Pr[2] * (0.5 * br),
                   Pl[3] * (0.5 * bl) + Pr[3] * (0.5 * br)};
  double z5b = 0.5 * (bl * pl + br * pr);
  double zn = dot3(zvb, n);
  double z1l = or_logavg(bl, br);
  double z5l = or_logavg(bl * pl, br * pr);
  F[0] = z5l * zn;
  double c1 = z5b / z1b, c2 = F[0] / z1b;
  for (int c = 0; c < 3; c++) F[1 + c] = n[c] * c1 + zvb[c] * c2;
  F[4] = 0.5 * ((G + 1.0) / (G - 1.0) * F[0] / z1l + dot3(F + 1, zvb)) / z1b;
  for (int c = 0; c < 5; c++) F[c] *= area;
}

/* keps_flux, enflo/src/keps.cc:10-48: arithmetic means of rho and beta */
static void keps_flux(const dspw_desc* d, const double* Pl, const double* Pr, const double* n,
                      double area, double* F) {
  double R = d->gas_const, G = d->gamma;
  double rhol = Pl[0], rhor = Pr[0];
  double rho = 0.5 * (rhol + rhor);
  double templ = Pl[4] / (R * rhol);
  double tempr = Pr[4] / (R * rhor);
  double vel2 = 0.5 * (sq3(Pl + 1) + sq3(Pr + 1));
  double betal = 0.5 / (R * templ);
  double betar = 0.5 / (R * tempr);
  double beta = 0.5 * (betal + betar);
  double p = 0.5 * rho / beta;
  double vel[3] = {Pl[1] * 0.5 + Pr[1] * 0.5, Pl[2] * 0.5 + Pr[2] * 0.5, Pl[3] * 0.5 + Pr[3] * 0.5};
  double vn = dot3(vel, n);
  F[0] = rho * vn;
  for (int c = 0; c < 3; c++) F[1 + c] = n[c] * p + vel[c] * F[0];
  F[4] = 0.5 * (1.0 / ((G - 1.0) * beta) - vel2) * F[0] + dot3(F + 1, vel);
  for (int c = 0; c < 5; c++) F[c] *= area;
}

/* roe_flux (Roe's flux without entropy fix), enflo/src/roe.cc:10-86 */
static void roe_flux(const dspw_desc* d, const double* Pl, const double* Pr, const double* n,
                     double area, double* F) {
  double G = d->gamma;
  double rhol = Pl[0], rhor = Pr[0], pl = Pl[4], pr = Pr[4];
  double hl = G * pl / rhol / (G - 1.0) + 0.5 * sq3(Pl + 1);
  double hr = G * pr / rhor / (G - 1.0) + 0.5 * sq3(Pr + 1);
  double rls = sqrt(rhol), rrs = sqrt(rhor);
  double fl = rls / (rls + rrs);
  double fr = 1.0 - fl;
  double rho = rls * rrs;
  double vel[3] = {Pl[1] * fl + Pr[1] * fr, Pl[2] * fl + Pr[2] * fr, Pl[3] * fl + Pr[3] * fr};
  double h = hl * fl + hr * fr;
  double vn = dot3(vel, n);
  double a = sqrt((G - 1.0) * (h - 0.5 * sq3(vel)));
  double dp = pr - pl;
  double vln = dot3(Pl + 1, n), vrn = dot3(Pr + 1, n);
  double dV = vrn - vln;
  if (vn >= 0.0) {
    double lambda = vn - a;
    double coeff = 0.5 * (dp - rho * a * dV) / (a * a);
    double factor = ((0.0 < lambda) ? 0.0 : lambda) * coeff;   /* std::min(lambda, 0.0) */
    F[0] = rhol * vln;
    for (int c = 0; c < 3; c++) F[1 + c] = n[c] * pl + Pl[1 + c] * (rhol * vln);
    F[4] = hl * F[0];
    F[0] += factor;
    for (int c = 0; c < 3; c++) F[1 + c] += vel[c] * factor + n[c] * (-a * factor);
    F[4] += (h - a * vn) * factor;
  } else {
    double lambda = vn + a;
    double coeff = 0.5 * (dp + rho * a * dV) / (a * a);
    double factor = ((lambda < 0.0) ? 0.0 : lambda) * coeff;   /* std::max(lambda, 0.0) */
    F[0] = rhor * vrn;
    for (int c = 0; c < 3; c++) F[1 + c] = n[c] * pr + Pr[1 + c] * (rhor * vrn);
    F[4] = hr * F[0];
    F[0] -= factor;
    for (int c = 0; c < 3; c++) F[1 + c] += vel[c] * (-factor) + n[c] * (-a * factor);
    F[4] -= (h + a * vn) * factor;
  }
  for (int c = 0; c < 5; c++) F[c] *= area;
}

typedef void (*two_point_fn)(const dspw_desc*, const double*, const double*, const double*, double, double*);

/* kepec4 / roe_ec4 / kep4 combination, enflo/src/kepec4.cc:10-38, roe_ec4.cc:10-34 */
static void four_point(const dspw_desc* d, two_point_fn f2, const double* P, const double* n, double area,
                       double* F) {
  double f0[5];
  for (int c = 0; c < 5; c++) F[c] = 0.0;
  f2(d, P + 5 * 1, P + 5 * 2, n, area, f0);
  for (int c = 0; c < 5; c++) F[c] += f0[c] * (4.0 / 3.0);
  double fact = -1.0 / 6.0;
  f2(d, P + 5 * 0, P + 5 * 2, n, area, f0);
  for (int c = 0; c < 5; c++) F[c] += f0[c] * fact;
  f2(d, P + 5 * 1, P + 5 * 3, n, area, f0);
  for (int c = 0; c < 5; c++) F[c] += f0[c] * fact;
}

/* Entropy variables of one primitive state, enflo/src/fv.cc:427-433 and Entropy :557-560 */
static void prim_to_ent1(const dspw_desc* d, const double* P, double* V) {
  double G = d->gamma;
  double beta = P[0] / (2 * P[4]);
  double s = log(P[4]) - G * log(P[0]);
  V[0] = (G - s) / (G - 1) - (sq3(P + 1)) * beta;
  V[1] = P[1] * (2 * beta);
  V[2] = P[2] * (2 * beta);
  V[3] = P[3] * (2 * beta);
  V[4] = -2 * beta;
}

/* The TeCNO family: central part + eigenvector-scaled entropy dissipation on the
 * reconstructed scaled entropy variables.  kepes_tecno4_roe_flux
 * (enflo/src/kepes_tecno4_roe.cc:10-176) is the template; the variants differ in
 * the central flux (kepes_tecno_roe.cc:51-54, kep_tecno_roe.cc:53, roe_tecno*_roe.cc)
 * and in Lambda (kepes_tecno4_rusanov.cc:83-85). */
static void tecno_flux(const dspw_desc* d, const double* Pst, const double* V, int ns, const double* n,
                       double area, double h, double* flux) {
  (void)h;
  double G = d->gamma, Rg = d->gas_const;
  const double* P = Pst + 5 * (ns / 2 - 2);   /* the four cells around the face */
  const double* Pl = P + 5;
  const double* Pr = P + 10;
  double rhol = Pl[0], rhor = Pr[0];
  double rho = or_logavg(rhol, rhor);
  double templ = Pl[4] / (Rg * rhol);
  double tempr = Pr[4] / (Rg * rhor);
  double betal = 0.5 / (Rg * templ);
  double betar = 0.5 / (Rg * tempr);
  double beta = or_logavg(betal, betar);
  double p = 0.5 * (rhol + rhor) / (betal + betar);
  double vel[3] = {Pl[1] * 0.5 + Pr[1] * 0.5, Pl[2] * 0.5 + Pr[2] * 0.5, Pl[3] * 0.5 + Pr[3] * 0.5};
  double vn = dot3(vel, n);

  int roe_lambda = 1, ec1 = 0;
  switch (d->flux) {
    case DSPW_KEPES_TECNO4_ROE: four_point(d, kepec_flux, P, n, area, flux); ec1 = d->ec1_fix; break;
    case DSPW_KEPES_TECNO4_RUSANOV: four_point(d, kepec_flux, P, n, area, flux); roe_lambda = 0; break;
    case DSPW_KEPES_TECNO_ROE: kepec_flux(d, Pl, Pr, n, area, flux); ec1 = d->ec1_fix; break;
    case DSPW_KEPES_TECNO_RUSANOV: kepec_flux(d, Pl, Pr, n, area, flux); roe_lambda = 0; break;
    case DSPW_KEP_TECNO_ROE: kep_flux(d, Pl, Pr, n, area, flux); break;
    case DSPW_ROE_TECNO_ROE: roe_ec_flux(d, Pl, Pr, n, area, flux); ec1 = d->ec1_fix; break;
    case DSPW_ROE_TECNO4_ROE: four_point(d, roe_ec_flux, P, n, area, flux); ec1 = d->ec1_fix; break;
    default: for (int c = 0; c < 5; c++) flux[c] = 0.0;
  }
  for (int c = 0; c < 5; c++) flux[c] *= (1 / area);

  double a = sqrt(0.5 * G / beta);
  double H = a * a / (G - 1.0) + 0.5 * sq3(vel);
  double v1 = vel[0] * n[1] - vel[1] * n[0];
  double v2 = vel[2] * n[0] - vel[0] * n[2];
  double Rm[5][5] = {
      {1, 1, 0, 0, 1},
      {vel[0] - a * n[0], vel[0], n[1], -n[2], vel[0] + a * n[0]},
      {vel[1] - a * n[1], vel[1], -n[0], 0, vel[1] + a * n[1]},
      {vel[2] - a * n[2], vel[2], 0, n[0], vel[2] + a * n[2]},
      {H - a * vn, 0.5 * sq3(vel), v1, v2, H + a * vn}};
  double const1 = sqrt(rho / G);
  double psqrt = sqrt(p);
  double S[5] = {sqrt(0.5) * const1, sqrt(G - 1.0) * const1, psqrt, psqrt, sqrt(0.5) * const1};
  for (int i = 0; i < 5; i++)
    for (int j = 0; j < 5; j++) Rm[j][i] *= S[i];

  double Lam[5];
  if (roe_lambda) {
    double vnl = dot3(Pl + 1, n);
    double vnr = dot3(Pr + 1, n);
    double al = sqrt(0.5 * G / betal);
    double ar = sqrt(0.5 * G / betar);
    double LL[5] = {vnl - al, vnl, vnl, vnl, vnl + al};
    double LR[5] = {vnr - ar, vnr, vnr, vnr, vnr + ar};
    double l2 = fabs(vn);
    double mb = 0.0 / 6.0, ma = 0.0 / 6.0;
    if (ec1) ma = 1.0 / 6.0;
    Lam[0] = (1 + mb) * fabs(vn - a) + ma * fabs(LL[0] - LR[0]);
    Lam[1] = l2; Lam[2] = l2; Lam[3] = l2;
    Lam[4] = (1 + mb) * fabs(vn + a) + ma * fabs(LL[3] - LR[3]);
  } else {
    double lr = fabs(vn) + fabs(a);
    for (int i = 0; i < 5; i++) Lam[i] = lr;
  }

  double Z[6][5];
  for (int k = 0; k < ns; k++)
    for (int i = 0; i < 5; i++) {
      const double* Vk = V + 5 * k;
      Z[k][i] = 0.0;
      Z[k][i] += Rm[0][i] * Vk[0] + Rm[1][i] * Vk[1] + Rm[2][i] * Vk[2] + Rm[3][i] * Vk[3] + Rm[4][i] * Vk[4];
    }
  double Zij[5], Zji[5];
  for (int i = 0; i < 5; i++) {
    double sk[6];
    for (int k = 0; k < ns; k++) sk[k] = Z[k][i];
    reconstruct1(d, sk, &Zij[i], &Zji[i]);
  }
  double dZ[5], Diff[5];
  for (int i = 0; i < 5; i++) { dZ[i] = Zji[i] - Zij[i]; Diff[i] = 0; }
  for (int i = 0; i < 5; i++)
    for (int j = 0; j < 5; j++) Diff[i] += Rm[i][j] * Lam[j] * dZ[j];
  flux[0] -= 0.5 * Diff[0];
  flux[1] -= 0.5 * Diff[1];
  flux[2] -= 0.5 * Diff[2];
  flux[2] -= 0.5 * Diff[3];   /* momentum y, not z: as in the reference (kepes_tecno4_roe.cc:170) */
  flux[4] -= 0.5 * Diff[4];
  for (int c = 0; c < 5; c++) flux[c] *= area;
}

/* num_flux dispatch, enflo/src/num_flux.cc:12-72 */
static void euler_num_flux(const dspw_desc* d, const double* Pst, const double* V, int ns, int dir, double dx,
                           double dy, double dz, double* F) {
  const double* P = Pst + 5 * (ns / 2 - 2);   /* central fluxes read the four middle cells */
  double n[3] = {0, 0, 0};
  n[dir] = 1;
  double area = dir == 0 ? dy * dz : (dir == 1 ? dx * dz : dx * dy);
  double h = dir == 0 ? dx : (dir == 1 ? dy : dz);
  switch (d->flux) {
    case DSPW_KEPEC: kepec_flux(d, P + 5, P + 10, n, area, F); break;
    case DSPW_KEPEC4: four_point(d, kepec_flux, P, n, area, F); break;
    case DSPW_KEP: kep_flux(d, P + 5, P + 10, n, area, F); break;
    case DSPW_KEP4: four_point(d, kep_flux, P, n, area, F); break;
    case DSPW_ROE_EC: roe_ec_flux(d, P + 5, P + 10, n, area, F); break;
    case DSPW_ROE_EC4: four_point(d, roe_ec_flux, P, n, area, F); break;
    case DSPW_KEPS: keps_flux(d, P + 5, P + 10, n, area, F); break;
    case DSPW_KEPS4: four_point(d, keps_flux, P, n, area, F); break;
    case DSPW_ROE: roe_flux(d, P + 5, P + 10, n, area, F); break;
    default: tecno_flux(d, Pst, V, ns, n, area, h, F);
  }
}

/* cells of a face stencil: 2 ng */
static int stencil_cells(const dspw_desc* d) { return d->recon == DSPW_REC_ENO3 ? 6 : 4; }

void or_euler_face_flux(const dspw_desc* d, const double* P, int dir, double dx, double dy, double dz,
                        double* V, double flux[5]) {
  const int ns = stencil_cells(d);
  for (int k = 0; k < ns; k++) prim_to_ent1(d, P + 5 * k, V + 5 * k);
  euler_num_flux(d, P, V, ns, dir, dx, dy, dz, flux);
}

/* ----------------------------------------------------------- scalar pieces -- */

/* lin_ec / bur_ec two-point fluxes, enflo_scalar/src_scalar/lin_ec.cc:10-20, bur_ec.cc:10-19 */
static double lin_ec(const double* vel, const double* n, double ul, double ur) {
  double v = n[0] * vel[0] + n[1] * vel[1] + n[2] * vel[2];
  return 0.5 * v * (ul + ur);
}
static double bur_ec(double ul, double ur) { return (ul * ul + ur * ur + ul * ur) / 6.0; }

/* num_flux and the lin_ and bur_ fluxes, enflo_scalar/src_scalar/num_flux.cc:12-57,
 * lin_tecno4.cc:10-31, lin_ec4.cc:10-34, bur_tecno4.cc:10-35, bur_ec4.cc:10-34 */
double or_scalar_face_flux(const dspw_desc* d, const double* ust, int dir, double dx, double dy, double dz) {
  const double* u = ust + (stencil_cells(d) / 2 - 2);   /* central fluxes read the four middle cells */
  double n[3] = {0, 0, 0};
  n[dir] = 1;
  double area = dir == 0 ? dy * dz : (dir == 1 ? dx * dz : dx * dy);
  const double* vel = d->lin_vel;
  double flux = 0.0, f0, l, r;
  switch (d->flux) {
    case DSPW_LIN_EC: flux = lin_ec(vel, n, u[1], u[2]); break;
    case DSPW_LIN_EC4:
    case DSPW_LIN_TECNO4:
      flux = 0.0;
      f0 = lin_ec(vel, n, u[1], u[2]); flux += f0 * 4.0 / 3.0;
      f0 = lin_ec(vel, n, u[0], u[2]); flux += f0 * (-1.0 / 6.0);
      f0 = lin_ec(vel, n, u[1], u[3]); flux += f0 * (-1.0 / 6.0);
      break;
    case DSPW_LIN_TECNO: flux = lin_ec(vel, n, u[1], u[2]); break;
    case DSPW_BUR_EC: flux = bur_ec(u[1], u[2]); break;
    case DSPW_BUR_EC4:
    case DSPW_BUR_TECNO4:
      flux = 0.0;
      f0 = bur_ec(u[1], u[2]); flux += f0 * (4.0 / 3.0);
      f0 = bur_ec(u[0], u[2]); flux += f0 * (-1.0 / 6.0);
      f0 = bur_ec(u[1], u[3]); flux += f0 * (-1.0 / 6.0);
      break;
    case DSPW_BUR_TECNO: flux = bur_ec(u[1], u[2]); break;
  }
  if (d->flux == DSPW_LIN_TECNO || d->flux == DSPW_LIN_TECNO4) {
    double D = fabs(n[0] * vel[0] + n[1] * vel[1] + n[2] * vel[2]);
    reconstruct1(d, ust, &l, &r);
    flux -= 0.5 * D * (r - l);
  } else if (d->flux == DSPW_BUR_TECNO || d->flux == DSPW_BUR_TECNO4) {
    double D = 0.5 * (fabs(u[1]) + fabs(u[2]));
    reconstruct1(d, ust, &l, &r);
    flux -= 0.5 * D * (r - l);
  }
  flux *= area;
  return flux;
}

/* ------------------------------------------------------------ solver state -- */

or_state* or_create(const dspw_desc* d) {
  or_state* s = (or_state*)calloc(1, sizeof(or_state));
  s->d = *d;
  s->scalar = (d->model == DSPW_LINADV || d->model == DSPW_BURGERS);
  s->nvar = s->scalar ? 1 : 5;
  s->nx = d->nx; s->ny = d->ny; s->nz = d->nz;
  s->ng = d->recon == DSPW_REC_ENO3 ? 3 : 2;
  s->px = d->nx + 2 * NG; s->py = d->ny + 2 * NG; s->pz = d->nz + 2 * NG;
  s->dx = (d->xmax - d->xmin) / d->nx;   /* enflo/src/fv.cc:29-31 */
  s->dy = (d->ymax - d->ymin) / d->ny;
  s->dz = (d->zmax - d->zmin) / d->nz;
  size_t np = (size_t)s->px * s->py * s->pz, nc = (size_t)s->nx * s->ny * s->nz;
  s->P = (double*)calloc(np * 5, sizeof(double));
  s->V = (double*)calloc(np * 5, sizeof(double));
  s->U = (double*)calloc(nc * 5, sizeof(double));
  s->Uold = (double*)calloc(nc * 5, sizeof(double));
  s->R2 = (double*)calloc(nc * 5, sizeof(double));
  s->R = (double*)calloc(nc * 5, sizeof(double));
  s->t_interval = d->final_time / (d->t_stamps > 0 ? d->t_stamps : 1);
  s->t_save = s->t_interval;
  return s;
}

void or_destroy(or_state* s) {
  if (!s) return;
  free(s->P); free(s->V); free(s->U); free(s->Uold); free(s->R); free(s->R2);
  free(s);
}

/* apply_bc, enflo/src/fv.cc:121-361 (systems, on primitive variables) and
 * enflo_scalar/src_scalar/fv.cc:110-281 (scalar).  The ghost value of a cell
 * is copied from `src` (periodic/neumann/wall) with the wall sign flip on the
 * face-normal velocity (systems) or on u (scalar); DIRICHLET uses bc_state. */
static void ghost_from(or_state* s, size_t dst, size_t src, int face, int kind) {
  int nv = s->scalar ? 1 : 5;
  double* D = s->P + 5 * dst;
  const double* S = s->P + 5 * src;
  if (kind == DSPW_BC_DIRICHLET) {
    for (int c = 0; c < nv; c++) D[c] = s->d.bc_state[face][c];
    return;
  }
  for (int c = 0; c < nv; c++) D[c] = S[c];
  if (kind == DSPW_BC_WALL) {
    if (s->scalar) D[0] = -S[0];
    else D[1 + face / 2] = -S[1 + face / 2];
  }
}

static void apply_bc(or_state* s) {
  const int g = NG, Nx = s->nx, Ny = s->ny, Nz = s->nz;
  const int* bc = s->d.bc;
  /* x faces */
  for (int i = 0; i < g; ++i)
    for (int j = 0; j < Ny; ++j)
      for (int k = 0; k < Nz; ++k) {
        size_t dst = pidx(s, i, g + j, g + k), src;
        if (bc[0] == DSPW_BC_PERIODIC) src = pidx(s, Nx + i, g + j, g + k);
        else if (bc[0] == DSPW_BC_WALL) src = pidx(s, 2 * g - 1 - i, g + j, g + k);
        else src = pidx(s, g, g + j, g + k);
        ghost_from(s, dst, src, 0, bc[0]);
      }
  for (int i = 0; i < g; ++i)
    for (int j = 0; j < Ny; ++j)
      for (int k = 0; k < Nz; ++k) {
        size_t dst = pidx(s, Nx + g + i, g + j, g + k), src;
        if (bc[1] == DSPW_BC_PERIODIC) src = pidx(s, g + i, g + j, g + k);
        else if (bc[1] == DSPW_BC_WALL) src = pidx(s, Nx + g - 1 - i, g + j, g + k);
        else src = pidx(s, Nx + g - 1, g + j, g + k);
        ghost_from(s, dst, src, 1, bc[1]);
      }
  /* y faces */
  for (int i = 0; i < Nx; ++i)
    for (int j = 0; j < g; ++j)
      for (int k = 0; k < Nz; ++k) {
        size_t dst = pidx(s, g + i, j, g + k), src;
        if (bc[2] == DSPW_BC_PERIODIC) src = pidx(s, g + i, Ny + j, g + k);
        else if (bc[2] == DSPW_BC_WALL) src = pidx(s, g + i, 2 * g - 1 - j, g + k);
        else src = pidx(s, g + i, g, g + k);
        ghost_from(s, dst, src, 2, bc[2]);
      }
  for (int i = 0; i < Nx; ++i)
    for (int j = 0; j < g; ++j)
      for (int k = 0; k < Nz; ++k) {
        size_t dst = pidx(s, g + i, Ny + g + j, g + k), src;
        if (bc[3] == DSPW_BC_PERIODIC) src = pidx(s, g + i, g + j, g + k);
        else if (bc[3] == DSPW_BC_WALL) src = pidx(s, g + i, Ny + g - 1 - j, g + k);
        else src = pidx(s, g + i, Ny + g - 1, g + k);
        ghost_from(s, dst, src, 3, bc[3]);
      }
  /* z faces */
  for (int i = 0; i < Nx; ++i)
    for (int j = 0; j < Ny; ++j)
      for (int k = 0; k < g; ++k) {
        size_t dst = pidx(s, g + i, g + j, k), src;
        if (bc[4] == DSPW_BC_PERIODIC) src = pidx(s, g + i, g + j, Nz + k);
        else if (bc[4] == DSPW_BC_WALL) src = pidx(s, g + i, g + j, 2 * g - 1 - k);
        else src = pidx(s, g + i, g + j, g);
        ghost_from(s, dst, src, 4, bc[4]);
      }
  for (int i = 0; i < Nx; ++i)
    for (int j = 0; j < Ny; ++j)
      for (int k = 0; k < g; ++k) {
        size_t dst = pidx(s, g + i, g + j, Nz + g + k), src;
        if (bc[5] == DSPW_BC_PERIODIC) src = pidx(s, g + i, g + j, g + k);
        else if (bc[5] == DSPW_BC_WALL) src = pidx(s, g + i, g + j, Nz + g - 1 - k);
        else src = pidx(s, g + i, g + j, Nz + g - 1);
        ghost_from(s, dst, src, 5, bc[5]);
      }
  if (s->scalar) return;
  /* edges and corners, periodic wrap (enflo/src/fv.cc:317-358); only the
   * viscous node stencil reads them */
  for (int k = -1; k <= Nz; ++k)
    for (int j = -1; j <= Ny; ++j)
      for (int i = -1; i <= Nx; ++i) {
        int out = (i < 0 || i >= Nx) + (j < 0 || j >= Ny) + (k < 0 || k >= Nz);
        if (out < 2) continue;
        int si = (i + Nx) % Nx, sj = (j + Ny) % Ny, sk = (k + Nz) % Nz;
        memcpy(s->P + 5 * pidx(s, g + i, g + j, g + k), s->P + 5 * pidx(s, g + si, g + sj, g + sk),
               5 * sizeof(double));
      }
}

/* prim_to_con, enflo/src/fv.cc:405-416 */
static void prim_to_con(or_state* s) {
  double G = s->d.gamma;
  for (int k = 0; k < s->nz; ++k)
    for (int j = 0; j < s->ny; ++j)
      for (int i = 0; i < s->nx; ++i) {
        const double* P = s->P + 5 * pidx(s, i + NG, j + NG, k + NG);
        double* U = s->U + 5 * cidx(s, i, j, k);
        U[0] = P[0];
        U[1] = P[1] * P[0]; U[2] = P[2] * P[0]; U[3] = P[3] * P[0];
        U[4] = 0.5 * P[0] * sq3(P + 1) + P[4] / (G - 1.0);
      }
}

/* con_to_prim, enflo/src/fv.cc:388-400 */
static void con_to_prim(or_state* s) {
  double G = s->d.gamma;
  for (int k = 0; k < s->nz; ++k)
    for (int j = 0; j < s->ny; ++j)
      for (int i = 0; i < s->nx; ++i) {
        double* P = s->P + 5 * pidx(s, i + NG, j + NG, k + NG);
        const double* U = s->U + 5 * cidx(s, i, j, k);
        P[0] = U[0];
        double r = 1.0 / U[0];
        P[1] = U[1] * r; P[2] = U[2] * r; P[3] = U[3] * r;
        P[4] = (G - 1.0) * (U[4] - 0.5 * sq3(U + 1) / U[0]);
      }
  apply_bc(s);
}

/* prim_to_ent over interior and ghost cells, enflo/src/fv.cc:421-552 */
static void prim_to_ent(or_state* s) {
  for (int k = -NG; k < s->nz + NG; ++k)
    for (int j = -NG; j < s->ny + NG; ++j)
      for (int i = -NG; i < s->nx + NG; ++i) {
        int out = (i < 0 || i >= s->nx) + (j < 0 || j >= s->ny) + (k < 0 || k >= s->nz);
        int inner_ring = (i >= -1 && i <= s->nx && j >= -1 && j <= s->ny && k >= -1 && k <= s->nz);
        if (out >= 2 && !inner_ring) continue;
        size_t c = pidx(s, i + NG, j + NG, k + NG);
        if (s->P[5 * c] == 0.0 && s->P[5 * c + 4] == 0.0) continue;
        prim_to_ent1(&s->d, s->P + 5 * c, s->V + 5 * c);
      }
}

void or_set_prim(or_state* s, const double* prim) {
  size_t nc = (size_t)s->nx * s->ny * s->nz;
  for (int k = 0; k < s->nz; ++k)
    for (int j = 0; j < s->ny; ++j)
      for (int i = 0; i < s->nx; ++i) {
        size_t c = cidx(s, i, j, k);
        double* P = s->P + 5 * pidx(s, i + NG, j + NG, k + NG);
        if (s->scalar) P[0] = prim[c];
        else for (int v = 0; v < 5; v++) P[v] = prim[v * nc + c];
      }
  apply_bc(s);
  if (s->scalar) {
    for (int k = 0; k < s->nz; ++k)
      for (int j = 0; j < s->ny; ++j)
        for (int i = 0; i < s->nx; ++i)
          s->U[5 * cidx(s, i, j, k)] = s->P[5 * pidx(s, i + NG, j + NG, k + NG)];
  } else {
    prim_to_con(s);
    prim_to_ent(s);
  }
  s->time = 0.0;
  s->iter = 0;
  s->t_save = s->t_interval;
}

void or_get_prim(const or_state* s, double* prim) {
  size_t nc = (size_t)s->nx * s->ny * s->nz;
  for (int k = 0; k < s->nz; ++k)
    for (int j = 0; j < s->ny; ++j)
      for (int i = 0; i < s->nx; ++i) {
        size_t c = cidx(s, i, j, k);
        const double* P = s->P + 5 * pidx(s, i + NG, j + NG, k + NG);
        for (int v = 0; v < s->nvar; v++) prim[v * nc + c] = P[v];
      }
}

void or_get_cons(const or_state* s, double* cons) {
  size_t nc = (size_t)s->nx * s->ny * s->nz;
  for (size_t c = 0; c < nc; c++)
    for (int v = 0; v < s->nvar; v++) cons[v * nc + c] = s->U[5 * c + v];
}

/* scalar state lives in P[.][0] (with ghosts) and U[.][0] (interior copy) */
static void scalar_sync_from_P(or_state* s) {
  for (int k = 0; k < s->nz; ++k)
    for (int j = 0; j < s->ny; ++j)
      for (int i = 0; i < s->nx; ++i)
        s->U[5 * cidx(s, i, j, k)] = s->P[5 * pidx(s, i + NG, j + NG, k + NG)];
}

/* Viscosity, enflo/src/parameter.cc:646-663 */
static double viscosity(const dspw_desc* d, double T) {
  switch (d->mu_model) {
    case DSPW_MU_SUTHERLAND: return d->mu_ref * pow(T / d->T_ref, 1.5) * (d->T_ref + d->T_0) / (T + d->T_0);
    case DSPW_MU_POWER: return d->mu_ref * pow(T / d->T_ref, d->omega);
    default: return d->mu_ref;
  }
}

/* compute_dt, enflo/src/fv.cc:366-383 and enflo_scalar/src_scalar/fv.cc:286-311 */
double or_compute_dt(or_state* s) {
  double dt = 1.0e20;
  double hmin = fmin(s->dx, fmin(s->dy, s->dz));
  for (int i = 0; i < s->nx; ++i)
    for (int j = 0; j < s->ny; ++j)
      for (int k = 0; k < s->nz; ++k) {
        const double* P = s->P + 5 * pidx(s, i + NG, j + NG, k + NG);
        double speed;
        if (s->d.model == DSPW_LINADV) speed = sqrt(sq3(s->d.lin_vel));
        else if (s->d.model == DSPW_BURGERS) speed = fabs(P[0]);
        else {
          speed = sqrt(sq3(P + 1)) + sqrt(s->d.gamma * P[4] / P[0]);
          if (s->d.model == DSPW_NS_ES || s->d.model == DSPW_NS_KEP)
            speed += viscosity(&s->d, P[4] / (s->d.gas_const * P[0])) / P[0] / hmin;
        }
        dt = fmin(dt, hmin / speed);
      }
  dt *= s->d.cfl;
  s->dt = dt;
  return dt;
}

/* ------------------------------------------------------- residual assembly -- */

/* cell of the face stencil along direction dir of line (a, b), in padded
 * coordinates: face f reads cells f .. f + 2 ng - 1 along dir */
static void line_cell(const or_state* s, int dir, int f, int a, int b, int* i, int* j, int* k) {
  if (dir == 0) { *i = f; *j = a; *k = b; }
  else if (dir == 1) { *i = a; *j = f; *k = b; }
  else { *i = a; *j = b; *k = f; }
  (void)s;
}

/* compute_inv_residual, enflo/src/fv.cc:608-767; scalar compute_residual,
 * enflo_scalar/src_scalar/fv.cc:317-457.  Faces of each direction in the
 * reference's order: left boundary face, interior faces, right boundary face. */
static void inviscid_residual(or_state* s) {
  int nc = s->nx * s->ny * s->nz;
  memset(s->R, 0, sizeof(double) * 5 * nc);
  int N[3] = {s->nx, s->ny, s->nz};
  int nv = s->nvar;
  for (int dir = 0; dir < 3; dir++) {
    /* A direction with a single cell is not swept: the reference always
     * carries at least two cells there (1-D and 2-D problems use Ny=Nz=2,
     * README.md:152-160); the single-cell layout is this project's reduced
     * form, in which the degenerate sweeps are dropped. */
    if (N[dir] == 1) continue;
    int o1 = dir == 0 ? 1 : 0, o2 = dir == 2 ? 1 : 2;   /* the two other directions */
    for (int a = 0; a < N[o1]; a++)
      for (int b = 0; b < N[o2]; b++) {
        const int ns = 2 * NG;
        for (int f = 0; f <= N[dir]; f++) {   /* face f between cells f-1 and f */
          double Pst[30], Vst[30], F[5];
          for (int l = 0; l < ns; l++) {
            int i, j, k;
            int coord[3];
            coord[dir] = f + l;          /* padded: cells f-ng..f+ng-1 */
            coord[o1] = a + NG;
            coord[o2] = b + NG;
            line_cell(s, 0, coord[0], coord[1], coord[2], &i, &j, &k);
            size_t c = pidx(s, i, j, k);
            memcpy(Pst + 5 * l, s->P + 5 * c, 5 * sizeof(double));
            memcpy(Vst + 5 * l, s->V + 5 * c, 5 * sizeof(double));
          }
          if (s->scalar) {
            double us[6];
            for (int l = 0; l < ns; l++) us[l] = Pst[5 * l];
            F[0] = or_scalar_face_flux(&s->d, us, dir, s->dx, s->dy, s->dz);
          } else {
            euler_num_flux(&s->d, Pst, Vst, ns, dir, s->dx, s->dy, s->dz, F);
          }
          int cl[3], cr[3];
          cl[dir] = f - 1; cl[o1] = a; cl[o2] = b;
          cr[dir] = f; cr[o1] = a; cr[o2] = b;
          if (f == 0) {
            double* R = s->R + 5 * cidx(s, cr[0], cr[1], cr[2]);
            for (int v = 0; v < nv; v++) R[v] -= F[v];
          } else if (f == N[dir]) {
            double* R = s->R + 5 * cidx(s, cl[0], cl[1], cl[2]);
            for (int v = 0; v < nv; v++) R[v] += F[v];
          } else {
            double* Rl = s->R + 5 * cidx(s, cl[0], cl[1], cl[2]);
            double* Rr = s->R + 5 * cidx(s, cr[0], cr[1], cr[2]);
            for (int v = 0; v < nv; v++) { Rl[v] += F[v]; Rr[v] -= F[v]; }
          }
        }
      }
    /* the reference visits faces direction by direction with the other two
     * indices outermost in (i,j,k) order; per cell the sum order is the same */
  }
  /* KE dissipation of the inviscid residual, enflo/src/fv.cc:756-764 */
  s->ke_diss_pr = 0.0;
  if (s->scalar) return;
  for (int i = 0; i < s->nx; ++i)
    for (int j = 0; j < s->ny; ++j)
      for (int k = 0; k < s->nz; ++k) {
        const double* P = s->P + 5 * pidx(s, i + NG, j + NG, k + NG);
        const double* R = s->R + 5 * cidx(s, i, j, k);
        s->ke_diss_pr -= 0.5 * sq3(P + 1) * R[0] + dot3(P + 1, R + 1);
      }
}

/* nodal_vlux_ES, enflo/src/vflux_ES.cc:15-151, node (i,j,k) at (i+1/2, j+1/2,
 * k+1/2) in interior coordinates (i in -1..Nx-1).  Returns the effective x, y
 * and z fluxes: the y flux keeps only its K22,K23 terms and the z flux only
 * K33, because the reference overwrites the earlier accumulations. */
static void nodal_flux_es(or_state* s, int i, int j, int k, double* xf, double* yf, double* zf) {
  const dspw_desc* d = &s->d;
#define VV(a, b, c) (s->V + 5 * pidx(s, NG + i + (a), NG + j + (b), NG + k + (c)))
  const double f1 = 1.0 / 8.0;
  double avg[5], Tx[5], Ty[5], Tz[5];
  double fx = 1.0 / 4.0 / s->dx, fy = 1.0 / 4.0 / s->dy, fz = 1.0 / 4.0 / s->dz;
  for (int c = 0; c < 5; c++) {
    avg[c] = VV(1, 1, 1)[c] * f1 + VV(0, 1, 1)[c] * f1 + VV(1, 0, 1)[c] * f1 + VV(1, 1, 0)[c] * f1;
    avg[c] += VV(0, 0, 1)[c] * f1 + VV(0, 1, 0)[c] * f1 + VV(1, 0, 0)[c] * f1 + VV(0, 0, 0)[c] * f1;
    Tx[c] = VV(1, 1, 1)[c] * fx + VV(1, 1, 0)[c] * fx + VV(1, 0, 1)[c] * fx + VV(1, 0, 0)[c] * fx;
    Tx[c] += VV(0, 1, 1)[c] * -fx + VV(0, 1, 0)[c] * -fx + VV(0, 0, 1)[c] * -fx + VV(0, 0, 0)[c] * -fx;
    Ty[c] = VV(1, 1, 1)[c] * fy + VV(1, 1, 0)[c] * fy + VV(0, 1, 1)[c] * fy + VV(0, 1, 0)[c] * fy;
    Ty[c] += VV(1, 0, 1)[c] * -fy + VV(1, 0, 0)[c] * -fy + VV(0, 0, 1)[c] * -fy + VV(0, 0, 0)[c] * -fy;
    Tz[c] = VV(1, 1, 1)[c] * fz + VV(1, 0, 1)[c] * fz + VV(0, 1, 1)[c] * fz + VV(0, 0, 1)[c] * fz;
    Tz[c] += VV(1, 1, 0)[c] * -fz + VV(1, 0, 0)[c] * -fz + VV(0, 1, 0)[c] * -fz + VV(0, 0, 0)[c] * -fz;
  }
#undef VV
  double Cp = d->gamma * d->gas_const / (d->gamma - 1.0);
  double T = -1 / avg[4] / d->gas_const;
  double mu = viscosity(d, T);
  double kappa = mu * Cp / d->prandtl;
  double c1 = 4.0 * mu / 3.0, c2 = -2.0 * mu / 3.0, c3 = kappa / d->gas_const, e4 = 1.0 / avg[4];
  double e1 = avg[1] * e4, e2 = avg[2] * e4, e3 = avg[3] * e4;
  /* x flux: K11 Vx + K12 Vy + K13 Vz */
  xf[0] = 0.0;
  xf[1] = c1 * e4 * (-Tx[1] + e1 * Tx[4]);
  xf[2] = mu * e4 * (-Tx[2] + e2 * Tx[4]);
  xf[3] = mu * e4 * (-Tx[3] + e3 * Tx[4]);
  xf[4] = e4 * (c1 * e1 * Tx[1] + mu * e2 * Tx[2] + mu * e3 * Tx[3] +
                (-c1 * e1 * e1 - mu * (e2 * e2 + e3 * e3) + c3 * e4) * Tx[4]);
  xf[1] += c2 * e4 * (-Ty[2] + e2 * Ty[4]);
  xf[2] += mu * e4 * (-Ty[1] + e1 * Ty[4]);
  xf[3] += 0;
  xf[4] += e4 * (mu * e2 * Ty[1] + c2 * e1 * Ty[2] - (mu + c2) * e1 * e2 * Ty[4]);
  xf[1] += c2 * e4 * (-Tz[3] + e3 * Tz[4]);
  xf[2] += 0;
  xf[3] += mu * e4 * (-Tz[1] + e1 * Tz[4]);
  xf[4] += e4 * (mu * e3 * Tz[1] + c2 * e1 * Tz[3] - (mu + c2) * e1 * e3 * Tz[4]);
  /* y flux: K22 Vy + K23 Vz (the K21 terms are overwritten in the reference) */
  yf[0] = 0.0;
  yf[1] = mu * e4 * (-Ty[1] + e1 * Ty[4]);
  yf[2] = c1 * e4 * (-Ty[2] + e2 * Ty[4]);
  yf[3] = mu * e4 * (-Ty[3] + e3 * Ty[4]);
  yf[4] = e4 * (mu * e1 * Ty[1] + c1 * e2 * Ty[2] + mu * e3 * Ty[3] +
                (-c1 * e2 * e2 - mu * (e1 * e1 + e3 * e3) + c3 * e4) * Ty[4]);
  yf[1] += 0;
  yf[2] += c2 * e4 * (-Tz[3] + e3 * Tz[4]);
  yf[3] += mu * e4 * (-Tz[2] + e2 * Tz[4]);
  yf[4] += e4 * (mu * e3 * Tz[2] + c2 * e2 * Tz[3] - (mu + c2) * e2 * e3 * Tz[4]);
  /* z flux: K33 Vz only */
  zf[0] = 0.0;
  zf[1] = mu * e4 * (-Tz[1] + e1 * Tz[4]);
  zf[2] = mu * e4 * (-Tz[2] + e2 * Tz[4]);
  zf[3] = c1 * e4 * (-Tz[3] + e3 * Tz[4]);
  zf[4] = e4 * (mu * e1 * Tz[1] + mu * e2 * Tz[2] + c1 * e3 * Tz[3] +
                (-c1 * e3 * e3 - mu * (e1 * e1 + e2 * e2) + c3 * e4) * Tz[4]);
  double ax = -(s->dy * s->dz), ay = -(s->dx * s->dz), az = -(s->dx * s->dy);
  for (int c = 0; c < 5; c++) { xf[c] *= ax; yf[c] *= ay; zf[c] *= az; }
}

/* nodal_vlux_KE, enflo/src/vflux_KE.cc:15-96, with the node average and the
 * velocity derivatives of nodal_avg_and_vel_derivatives
 * (enflo/src/nodal_avg_and_der.cc:16-82; note its 1/(4 dx) against the
 * 1/4/dx of the temperature derivatives) and Temperature (enflo/src/fv.cc:1329-1332). */
static double temp_of(const or_state* s, const double* P) { return P[4] / (s->d.gas_const * P[0]); }

/* velocity derivatives at node (i,j,k) (i in -1..Nx-1) from the 8 cells around
 * it, nodal_avg_and_vel_derivatives, enflo/src/nodal_avg_and_der.cc:37-81:
 * Tx[c] = d(u_c)/dx, Ty, Tz likewise */
static void node_vel_derivatives(const or_state* s, int i, int j, int k, double* Tx, double* Ty, double* Tz) {
#define PP(a, b, c) (s->P + 5 * pidx(s, NG + i + (a), NG + j + (b), NG + k + (c)))
  const double vx = 1.0 / (4.0 * s->dx), vy = 1.0 / (4.0 * s->dy), vz = 1.0 / (4.0 * s->dz);
  for (int c = 0; c < 3; c++) {
    const int v = 1 + c;
    Tx[c] = PP(1, 1, 1)[v] * vx + PP(1, 1, 0)[v] * vx + PP(1, 0, 1)[v] * vx + PP(1, 0, 0)[v] * vx;
    Tx[c] += PP(0, 1, 1)[v] * -vx + PP(0, 1, 0)[v] * -vx + PP(0, 0, 1)[v] * -vx + PP(0, 0, 0)[v] * -vx;
    Ty[c] = PP(1, 1, 1)[v] * vy + PP(1, 1, 0)[v] * vy + PP(0, 1, 1)[v] * vy + PP(0, 1, 0)[v] * vy;
    Ty[c] += PP(1, 0, 1)[v] * -vy + PP(1, 0, 0)[v] * -vy + PP(0, 0, 1)[v] * -vy + PP(0, 0, 0)[v] * -vy;
    Tz[c] = PP(1, 1, 1)[v] * vz + PP(1, 0, 1)[v] * vz + PP(0, 1, 1)[v] * vz + PP(0, 0, 1)[v] * vz;
    Tz[c] += PP(1, 1, 0)[v] * -vz + PP(1, 0, 0)[v] * -vz + PP(0, 1, 0)[v] * -vz + PP(0, 0, 0)[v] * -vz;
  }
#undef PP
}

static void nodal_flux_ke(or_state* s, int i, int j, int k, double* xf, double* yf, double* zf) {
  const dspw_desc* d = &s->d;
#define PP(a, b, c) (s->P + 5 * pidx(s, NG + i + (a), NG + j + (b), NG + k + (c)))
  const double f1 = 1.0 / 8.0;
  double avg[5], Tx[3], Ty[3], Tz[3];
  for (int c = 0; c < 5; c++) {
    avg[c] = PP(1, 1, 1)[c] * f1 + PP(0, 1, 1)[c] * f1 + PP(1, 0, 1)[c] * f1 + PP(1, 1, 0)[c] * f1;
    avg[c] += PP(0, 0, 1)[c] * f1 + PP(0, 1, 0)[c] * f1 + PP(1, 0, 0)[c] * f1 + PP(0, 0, 0)[c] * f1;
  }
  node_vel_derivatives(s, i, j, k, Tx, Ty, Tz);
  const double T_avg = avg[4] / (d->gas_const * avg[0]);
  const double mu = viscosity(d, T_avg);
  const double Cp = d->gamma * d->gas_const / (d->gamma - 1.0);
  const double kappa = mu * Cp / d->prandtl;
  const double fx = 1.0 / 4.0 / s->dx, fy = 1.0 / 4.0 / s->dy, fz = 1.0 / 4.0 / s->dz;
  const double t111 = temp_of(s, PP(1, 1, 1)), t110 = temp_of(s, PP(1, 1, 0)), t101 = temp_of(s, PP(1, 0, 1));
  const double t100 = temp_of(s, PP(1, 0, 0)), t011 = temp_of(s, PP(0, 1, 1)), t010 = temp_of(s, PP(0, 1, 0));
  const double t001 = temp_of(s, PP(0, 0, 1)), t000 = temp_of(s, PP(0, 0, 0));
#undef PP
  const double Tt_x = fx * (t111 + t110 + t101 + t100 - t011 - t010 - t001 - t000);
  const double Tt_y = fy * (t111 + t110 + t011 + t010 - t101 - t100 - t001 - t000);
  const double Tt_z = fz * (t111 + t101 + t011 + t001 - t110 - t100 - t010 - t000);
  const double grad = Tx[0] + Ty[1] + Tz[2];
  const double txx = mu * (2 * Tx[0] - (2.0 / 3.0) * grad);
  const double tyy = mu * (2 * Ty[1] - (2.0 / 3.0) * grad);
  const double tzz = mu * (2 * Tz[2] - (2.0 / 3.0) * grad);
  const double txy = mu * (Ty[0] + Tx[1]);
  const double txz = mu * (Tx[2] + Tz[0]);
  const double tyz = mu * (Ty[2] + Tz[1]);
  const double* u = avg + 1;
  xf[0] = 0.0; xf[1] = txx; xf[2] = txy; xf[3] = txz;
  xf[4] = (u[0] * txx + u[1] * txy + u[2] * txz) + kappa * Tt_x;
  yf[0] = 0.0; yf[1] = txy; yf[2] = tyy; yf[3] = tyz;
  yf[4] = (u[0] * txy + u[1] * tyy + u[2] * tyz) + kappa * Tt_y;
  zf[0] = 0.0; zf[1] = txz; zf[2] = tyz; zf[3] = tzz;
  zf[4] = (u[0] * txz + u[1] * tyz + u[2] * tzz) + kappa * Tt_z;
  double ax = -(s->dy * s->dz), ay = -(s->dx * s->dz), az = -(s->dx * s->dy);
  for (int c = 0; c < 5; c++) { xf[c] *= ax; yf[c] *= ay; zf[c] *= az; }
}

/* node weight of find_node_weights, enflo/src/find_node_weights.cc:19-66:
 * halved on each periodic domain face the node lies on; (a,b,c) in 0..N */
static double node_weight(const or_state* s, int a, int b, int c) {
  double w = 1.0;
  const int* bc = s->d.bc;
  if (a == 0 && bc[0] == DSPW_BC_PERIODIC) w /= 2.0;
  if (a == s->nx && bc[1] == DSPW_BC_PERIODIC) w /= 2.0;
  if (b == 0 && bc[2] == DSPW_BC_PERIODIC) w /= 2.0;
  if (b == s->ny && bc[3] == DSPW_BC_PERIODIC) w /= 2.0;
  if (c == 0 && bc[4] == DSPW_BC_PERIODIC) w /= 2.0;
  if (c == s->nz && bc[5] == DSPW_BC_PERIODIC) w /= 2.0;
  return w;
}

/* scatter one node's fluxes into its interior cells with weights +-1/4
 * (nodal_vlux, enflo/src/fv.cc:773-780: ES for ns_es, KE otherwise), and add
 * the node's viscous-stress KE dissipation -(Tx.F_x dx + Ty.F_y dy + Tz.F_z dz) w
 * (enflo/src/fv.cc:810-814).  The derivatives and the weight are those of node
 * (ti,tj,tk), which is (i,j,k) except at two corners (viscous_residual). */
static void scatter_node_at(or_state* s, int i, int j, int k, int ti, int tj, int tk) {
  const int Nx = s->nx, Ny = s->ny, Nz = s->nz;
  double xf[5], yf[5], zf[5];
  if (s->d.model == DSPW_NS_ES) nodal_flux_es(s, i, j, k, xf, yf, zf);
  else nodal_flux_ke(s, i, j, k, xf, yf, zf);
  {
    double Tx[3], Ty[3], Tz[3];
    const double wt = node_weight(s, ti + 1, tj + 1, tk + 1);
    node_vel_derivatives(s, ti, tj, tk, Tx, Ty, Tz);
    s->ke_diss_stress -= (dot3(Tx, xf + 1) * s->dx + dot3(Ty, yf + 1) * s->dy + dot3(Tz, zf + 1) * s->dz) * wt;
  }
  for (int l = 0; l < 2; ++l)
    for (int m = 0; m < 2; ++m)
      for (int n = 0; n < 2; ++n) {
        int ci = i + l, cj = j + m, ck = k + n;
        if (ci < 0 || ci >= Nx || cj < 0 || cj >= Ny || ck < 0 || ck >= Nz) continue;
        double cx = (l ? -1.0 : 1.0) / 4.0, cy = (m ? -1.0 : 1.0) / 4.0, cz = (n ? -1.0 : 1.0) / 4.0;
        double* R = s->R + 5 * cidx(s, ci, cj, ck);
        for (int c = 0; c < 5; c++) R[c] += xf[c] * cx + yf[c] * cy + zf[c] * cz;
      }
}

static void scatter_node(or_state* s, int i, int j, int k) { scatter_node_at(s, i, j, k, i, j, k); }

/* compute_visc_residual, enflo/src/fv.cc:786-1157.  Nodes are visited in the
 * reference's order: interior nodes, then for each domain face (x-right,
 * x-left, y-right, y-left, z-right, z-left) its face nodes and two families of
 * edge nodes, then the 8 corners.  Every edge node line therefore appears in
 * two face blocks (e.g. (Nx-1, Ny-1, k) in the x-right block :867-870 and again
 * in the y-right block :930-937), and its contribution is added twice; this
 * restatement keeps that. */
static void viscous_residual(or_state* s) {
  const int X = s->nx - 1, Y = s->ny - 1, Z = s->nz - 1;
  s->ke_diss_stress = 0.0;
  for (int i = 0; i < X; i++)
    for (int j = 0; j < Y; j++)
      for (int k = 0; k < Z; k++) scatter_node(s, i, j, k);
  /* x-right, x-left */
  for (int side = 0; side < 2; side++) {
    int ib = side == 0 ? X : -1;
    for (int j = 0; j < Y; j++)
      for (int k = 0; k < Z; k++) scatter_node(s, ib, j, k);
    for (int j = 0; j < Y; j++) { scatter_node(s, ib, j, -1); scatter_node(s, ib, j, Z); }
    for (int k = 0; k < Z; k++) { scatter_node(s, ib, -1, k); scatter_node(s, ib, Y, k); }
  }
  /* y-right, y-left */
  for (int side = 0; side < 2; side++) {
    int jb = side == 0 ? Y : -1;
    for (int i = 0; i < X; i++)
      for (int k = 0; k < Z; k++) scatter_node(s, i, jb, k);
    for (int i = 0; i < X; i++) { scatter_node(s, i, jb, -1); scatter_node(s, i, jb, Z); }
    for (int k = 0; k < Z; k++) { scatter_node(s, -1, jb, k); scatter_node(s, X, jb, k); }
  }
  /* z-right, z-left */
  for (int side = 0; side < 2; side++) {
    int kb = side == 0 ? Z : -1;
    for (int i = 0; i < X; i++)
      for (int j = 0; j < Y; j++) scatter_node(s, i, j, kb);
    for (int i = 0; i < X; i++) { scatter_node(s, i, -1, kb); scatter_node(s, i, Y, kb); }
    for (int j = 0; j < Y; j++) { scatter_node(s, -1, j, kb); scatter_node(s, X, j, kb); }
  }
  /* corners, :1116-1150 */
  scatter_node(s, -1, -1, -1);
  scatter_node(s, X, -1, -1);
  scatter_node(s, -1, Y, -1);
  scatter_node(s, -1, -1, Z);
  scatter_node(s, X, Y, -1);
  scatter_node(s, X, -1, Z);
  /* the corners (0,N,N) and (N,N,N) take their derivatives and weight at
   * j = Nz-1 in place of Ny-1 (:1141-1150); the same node when Ny == Nz.  With
   * Nz > Ny that index lies outside the reference's node arrays; the corner's
   * own node is used then. */
  const int Yq = s->nz <= s->ny ? Z : Y;
  scatter_node_at(s, -1, Y, Z, -1, Yq, Z);
  scatter_node_at(s, X, Y, Z, X, Yq, Z);
}

void or_residual(or_state* s, int rk, double* res) {
  (void)rk;
  if (!s->scalar) prim_to_ent(s);
  inviscid_residual(s);
  if (s->d.model == DSPW_NS_ES || s->d.model == DSPW_NS_KEP) viscous_residual(s);
  if (res) {
    size_t nc = (size_t)s->nx * s->ny * s->nz;
    for (size_t c = 0; c < nc; c++)
      for (int v = 0; v < s->nvar; v++) res[v * nc + c] = s->R[5 * c + v];
  }
}

/* update_solution, enflo/src/fv.cc:1163-1175 (systems) and
 * enflo_scalar/src_scalar/fv.cc:463-476 (scalar) */
static void update(or_state* s, int rk) {
  double factor = s->dt / (s->dx * s->dy * s->dz);
  size_t nc = (size_t)s->nx * s->ny * s->nz;
  const int ts = s->d.time_scheme;
  if (ts == DSPW_JAMESON_RK4) {   /* fv.cc:1176-1184, scalar fv.cc:477-486 */
    for (size_t c = 0; c < nc; c++)
      for (int v = 0; v < (s->scalar ? 1 : 5); v++) {
        double* u = s->U + 5 * c + v;
        if (s->scalar) *u = (s->Uold[5 * c] - factor * JRK[rk] * s->R[5 * c]);
        else *u = s->Uold[5 * c + v] * 1.0 + s->R[5 * c + v] * (-factor * JRK[rk]);
      }
    return;
  }
  if (ts == DSPW_RK4) {           /* fv.cc:1185-1197, scalar fv.cc:487-499 */
    for (size_t c = 0; c < nc; c++)
      for (int v = 0; v < (s->scalar ? 1 : 5); v++) {
        double* u = s->U + 5 * c + v;
        double* r2 = s->R2 + 5 * c + v;
        const double Rv = s->R[5 * c + v], old = s->Uold[5 * c + v];
        if (s->scalar) {
          *r2 += (Rv / RK4C[rk]);
          if (rk < 3) *u = (old - factor * RK4C[rk + 1] * Rv);
          else *u = (old - factor * *r2 / 6.0);
        } else {
          *r2 += Rv * (1.0 / RK4C[rk]);
          if (rk < 3) *u = old * 1.0 + Rv * (-factor * RK4C[rk + 1]);
          else *u = old * 1.0 + *r2 * (-factor / 6.0);
        }
      }
    return;
  }
  double a = ARK[rk], b = BRK[rk];
  if (s->scalar) {
    for (size_t c = 0; c < nc; c++) {
      double* u = s->U + 5 * c;
      u[0] *= b;
      u[0] += (s->Uold[5 * c] * a - factor * b * s->R[5 * c]);
    }
  } else {
    for (size_t c = 0; c < nc; c++) {
      double* u = s->U + 5 * c;
      for (int v = 0; v < 5; v++) u[v] *= b;
      for (int v = 0; v < 5; v++) u[v] += s->Uold[5 * c + v] * a + s->R[5 * c + v] * (-factor * b);
    }
  }
}

static void scalar_to_P(or_state* s) {
  for (int k = 0; k < s->nz; ++k)
    for (int j = 0; j < s->ny; ++j)
      for (int i = 0; i < s->nx; ++i)
        s->P[5 * pidx(s, i + NG, j + NG, k + NG)] = s->U[5 * cidx(s, i, j, k)];
  apply_bc(s);
}

/* Enstrophy of compute_global (enflo/src/compute_global.cc:33-65) from the
 * node vorticity of find_vorticity (enflo/src/find_vort.cc:18-28), nodes
 * (i,j,k) in 0..N, ghost cells included */
static double enstrophy(const or_state* s) {
  const double f1 = 1.0 / 8.0;
  double ens = 0.0;
  for (int i = 0; i < s->nx + 1; ++i)
    for (int j = 0; j < s->ny + 1; ++j)
      for (int k = 0; k < s->nz + 1; ++k) {
#define RHO(a, b, c) s->P[5 * pidx(s, NG + i + (a), NG + j + (b), NG + k + (c))]
        double den = f1 * (RHO(-1, -1, -1) + RHO(0, -1, -1) + RHO(-1, 0, -1) + RHO(-1, -1, 0) + RHO(0, 0, -1) +
                           RHO(0, -1, 0) + RHO(-1, 0, 0) + RHO(0, 0, 0));
#undef RHO
        double Tx[3], Ty[3], Tz[3], w[3];
        node_vel_derivatives(s, i - 1, j - 1, k - 1, Tx, Ty, Tz);
        w[0] = Ty[2] - Tz[1];
        w[1] = Tz[0] - Tx[2];
        w[2] = Tx[1] - Ty[0];
        ens += den * sq3(w) * node_weight(s, i, j, k);
      }
  const dspw_desc* d = &s->d;
  double nodal_volume = (d->xmax - d->xmin) / (s->nx + 1) * (d->ymax - d->ymin) / (s->ny + 1) *
                        (d->zmax - d->zmin) / (s->nz + 1);
  return ens * (0.5 * nodal_volume);
}

/* compute_global's cell sums, enflo/src/compute_global.cc:18-28,58-64 and
 * enflo_scalar/src_scalar/compute_global.cc:12-21 */
static void cell_globals(const or_state* s, double* total_ent, double* ke) {
  double ent = 0.0, k_e = 0.0;
  for (int i = 0; i < s->nx; ++i)
    for (int j = 0; j < s->ny; ++j)
      for (int k = 0; k < s->nz; ++k) {
        const double* P = s->P + 5 * pidx(s, i + NG, j + NG, k + NG);
        if (s->scalar) {
          ent += 0.5 * pow(P[0], 2);
        } else {
          double sv = log(P[4]) - s->d.gamma * log(P[0]);
          ent += -P[0] * sv / (s->d.gamma - 1.0);
          k_e += P[0] * sq3(P + 1);
        }
      }
  double cell_volume = s->dx * s->dy * s->dz;
  *total_ent = ent * cell_volume;
  *ke = k_e * (0.5 * cell_volume);
}

/* compute_residual_norm, enflo/src/fv.cc:1204-1226 (per component, scaled by
 * the cell volume) and enflo_scalar/src_scalar/fv.cc:505-517 */
static void residual_norm(const or_state* s, double* out) {
  double r[5] = {0, 0, 0, 0, 0};
  for (int i = 0; i < s->nx; ++i)
    for (int j = 0; j < s->ny; ++j)
      for (int k = 0; k < s->nz; ++k) {
        const double* R = s->R + 5 * cidx(s, i, j, k);
        if (s->scalar) r[0] += pow(R[0], 2);
        else
          for (int v = 0; v < 5; v++) r[v] += pow(R[v] / s->dx / s->dy / s->dz, 2);
      }
  for (int v = 0; v < 5; v++) out[v] = sqrt(r[v]);
  if (!s->scalar)
    for (int v = 0; v < 5; v++) out[v] *= (s->dx * s->dy * s->dz);
}

int or_step(or_state* s, int nsteps, double fixed_dt) { return or_step_diag(s, nsteps, fixed_dt, NULL); }

/* loop body of FV::run, enflo/src/fv.cc:1262-1313 and
 * enflo_scalar/src_scalar/fv.cc:553-597.  or_step_diag also records, per step, the row of global diagnostics FV::run
 * computes (OR_DIAG_COLS doubles: iter, time, total entropy, KE, KE_diss_pr,
 * KE_diss_stress, enstrophy, residual norm per component).  Systems: the
 * values of compute_global at stage 0 (fv.cc:1280-1281), i.e. of U^n at t^n,
 * and the residual norm of the step's last stage.  Scalar: compute_global
 * after the step (enflo_scalar/src_scalar/fv.cc:573-576), i.e. t^(n+1). */
int or_step_diag(or_state* s, int nsteps, double fixed_dt, double* rows) {
  int taken = 0;
  size_t nc = (size_t)s->nx * s->ny * s->nz;
  const int ts = s->d.time_scheme;
  int nrk = ts == DSPW_RK1 ? 1 : (ts == DSPW_SSPRK3 ? 3 : 4);
  while (taken < nsteps && s->time < s->d.final_time && s->iter < s->d.max_iter) {
    memcpy(s->Uold, s->U, sizeof(double) * 5 * nc);
    if (ts == DSPW_RK4) memset(s->R2, 0, sizeof(double) * 5 * nc);   /* fv.cc:1268-1275 */
    if (fixed_dt > 0) s->dt = fixed_dt; else or_compute_dt(s);
    if (s->time + s->dt > s->t_save) s->dt = s->t_save - s->time;
    double* row = rows ? rows + (size_t)OR_DIAG_COLS * taken : NULL;
    if (row) memset(row, 0, sizeof(double) * OR_DIAG_COLS);
    for (int rk = 0; rk < nrk; ++rk) {
      or_residual(s, rk, NULL);
      if (row && rk == 0 && !s->scalar) {
        row[0] = s->iter;
        row[1] = s->time;
        cell_globals(s, &row[2], &row[3]);
        row[4] = s->ke_diss_pr;
        row[5] = (s->d.model == DSPW_NS_ES || s->d.model == DSPW_NS_KEP) ? s->ke_diss_stress : 0.0;
        row[6] = enstrophy(s);
      }
      update(s, rk);
      if (s->scalar) scalar_to_P(s);
      else con_to_prim(s);
    }
    s->time += s->dt;
    ++s->iter;
    if (row) {
      residual_norm(s, row + 7);
      if (s->scalar) {
        double ke;
        row[0] = s->iter;
        row[1] = s->time;
        cell_globals(s, &row[2], &ke);
      }
    }
    if (s->time == s->t_save) s->t_save += s->t_interval;
    ++taken;
  }
  (void)scalar_sync_from_P;
  return taken;
}

void or_time(const or_state* s, double* t, int* iter, double* dt) {
  if (t) *t = s->time;
  if (iter) *iter = s->iter;
  if (dt) *dt = s->dt;
}

/* compute_global, enflo/src/compute_global.cc:18-28 and
 * enflo_scalar/src_scalar/compute_global.cc:12-21, plus conserved totals */
void or_globals(or_state* s, double* total_entropy, double* cons5, double* ke) {
  double vol = s->dx * s->dy * s->dz;
  double ent = 0.0, k_e = 0.0, tot[5] = {0, 0, 0, 0, 0};
  for (int i = 0; i < s->nx; ++i)
    for (int j = 0; j < s->ny; ++j)
      for (int k = 0; k < s->nz; ++k) {
        const double* P = s->P + 5 * pidx(s, i + NG, j + NG, k + NG);
        const double* U = s->U + 5 * cidx(s, i, j, k);
        if (s->scalar) {
          ent += 0.5 * pow(P[0], 2);
          tot[0] += U[0];
        } else {
          double sv = log(P[4]) - s->d.gamma * log(P[0]);
          ent += -P[0] * sv / (s->d.gamma - 1.0);
          k_e += 0.5 * P[0] * sq3(P + 1);
          for (int v = 0; v < 5; v++) tot[v] += U[v];
        }
      }
  *total_entropy = ent * vol;
  if (ke) *ke = k_e * vol;
  for (int v = 0; v < 5; v++) cons5[v] = tot[v] * vol;
}
