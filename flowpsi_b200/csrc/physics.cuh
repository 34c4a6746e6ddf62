// physics.cuh -- device face physics of the implicit path (FP64 arithmetic).
//
// Primitive states are q = [T, u, v, w, pg] (pg = gauge pressure).  The
// preconditioned Roe scheme of flowPsi is written here around one object,
// the 5x5 matrix K(l1,l2,l3) of RoeJacobian (fluxInviscid.loci:1019-1090):
//   * roeCT_flux  (:869-1014)  = central flux - area/2 * K(|l|) dq
//   * roeCT_jacobian (:1092-1168) = area * K(l+-) with smoothed eigenvalues
// so the flux dissipation and the flux Jacobians share one coefficient set.
#pragma once
#include <cuda_runtime.h>

namespace fpsi {
namespace dev {

struct Gas {
  double gamma, Rt, pamb;
};

struct Q5 {
  double T, u, v, w, p;
};

__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double dmin(double a, double b) { return a < b ? a : b; }

// Roe-averaged state of roeCT_flux / roeCT_jacobian (:875-915, :1098-1139)
struct RoeAvg {
  double rl, rr, rel, rer;   // densities and total energies per volume
  double r, U, V, W, h0;     // Roe density, velocity, total enthalpy
  double un, unA;            // U.n - us_n, U.n
  double a, sigma, eta;
};

__device__ __forceinline__ RoeAvg roe_average(const Q5& L, const Q5& R, double nx, double ny,
                                              double nz, const Gas& g, double us_n,
                                              double eta) {
  RoeAvg s;
  const double gm1 = g.gamma - 1.0;
  const double pl = L.p + g.pamb, pr = R.p + g.pamb;
  s.rl = pl / (g.Rt * L.T);
  s.rr = pr / (g.Rt * R.T);
  s.rel = s.rl * (g.Rt * L.T / gm1 + 0.5 * (L.u * L.u + L.v * L.v + L.w * L.w));
  s.rer = s.rr * (g.Rt * R.T / gm1 + 0.5 * (R.u * R.u + R.v * R.v + R.w * R.w));
  const double h0l = (s.rel + pl) / s.rl;
  const double h0r = (s.rer + pr) / s.rr;
  s.r = sqrt(s.rl * s.rr);
  const double wl = sqrt(s.rl), wr = sqrt(s.rr);
  const double iw = 1.0 / (wl + wr);
  s.U = (L.u * wl + R.u * wr) * iw;
  s.V = (L.v * wl + R.v * wr) * iw;
  s.W = (L.w * wl + R.w * wr) * iw;
  s.unA = s.U * nx + s.V * ny + s.W * nz;
  s.un = s.unA - us_n;
  s.h0 = (h0l * wl + h0r * wr) * iw;
  const double h = s.h0 - 0.5 * (s.U * s.U + s.V * s.V + s.W * s.W);
  // strong pressure jumps switch preconditioning off (:914-915)
  if (fabs(pl - pr) / (pl + pr + 1e-33) > 0.1) eta = 1.0;
  s.eta = eta;
  s.a = sqrt(dmax(gm1 * h, 1e-30));
  const double em = eta - 1.0;
  s.sigma = sqrt(s.un * s.un * em * em + 4.0 * eta * s.a * s.a);
  return s;
}

// Coefficients of K for eigenvalues (l1, l2, l3): the entries are
//   K[0][T]=l1*rT  K[0][m]=n_m*c7          K[0][p]=c8
//   K[r][T]=l1*rT*U_r   K[r][m]=n_m*(c7*U_r+n_r*c4)+l1*rho*delta_rm
//   K[r][p]=c8*U_r-n_r*c1
//   K[e][T]=l1*c9  K[e][m]=n_m*c10+l1*rho*U_m   K[e][p]=c11
struct RoeK {
  double l1, rT, c7, c8, c9, c10, c11, c4, c1, rho, t4, d23;
};

// ---- eta == 1 with a fixed grid (us_n == 0): the form every mesh kernel
// evaluates.  The preconditioning parameter is 1 for Minf >= 0.5
// (fluxInviscid.loci:97-112), the only range the library accepts, and the
// grid does not move.  Then sigma = sqrt(4 a^2) = 2 a and every (beta - 1)
// term of roeCT_flux / RoeJacobian vanishes, so the coefficient set needs
// the reciprocals of a and of rT instead of a dozen divisions.  Results
// differ from the general form by a few ulp of their terms.
__device__ __forceinline__ RoeAvg roe_average1(const Q5& L, const Q5& R, double nx, double ny,
                                               double nz, const Gas& g) {
  RoeAvg s;
  const double gm1 = g.gamma - 1.0;
  const double pl = L.p + g.pamb, pr = R.p + g.pamb;
  const double RTl = g.Rt * L.T, RTr = g.Rt * R.T;
  s.rl = pl / RTl;
  s.rr = pr / RTr;
  const double kl = 0.5 * (L.u * L.u + L.v * L.v + L.w * L.w);
  const double kr = 0.5 * (R.u * R.u + R.v * R.v + R.w * R.w);
  const double igm1 = 1.0 / gm1;
  s.rel = s.rl * (RTl * igm1 + kl);
  s.rer = s.rr * (RTr * igm1 + kr);
  // h0 = (rho e0 + p) / rho = gamma R T / (gamma - 1) + |u|^2 / 2
  const double h0l = g.gamma * RTl * igm1 + kl;
  const double h0r = g.gamma * RTr * igm1 + kr;
  const double wl = sqrt(s.rl), wr = sqrt(s.rr);
  s.r = wl * wr;
  const double iw = 1.0 / (wl + wr);
  s.U = (L.u * wl + R.u * wr) * iw;
  s.V = (L.v * wl + R.v * wr) * iw;
  s.W = (L.w * wl + R.w * wr) * iw;
  s.unA = s.U * nx + s.V * ny + s.W * nz;
  s.un = s.unA;
  s.h0 = (h0l * wl + h0r * wr) * iw;
  const double h = s.h0 - 0.5 * (s.U * s.U + s.V * s.V + s.W * s.W);
  s.eta = 1.0;
  s.a = sqrt(dmax(gm1 * h, 1e-30));
  s.sigma = 2.0 * s.a;
  return s;
}

// roe_k at eta == 1; isg receives 1/sigma for the flux's dissipation
__device__ __forceinline__ RoeK roe_k1(double l1, double l2, double l3, const RoeAvg& s,
                                       const Gas& g, double& isg) {
  const double gm1 = g.gamma - 1.0;
  const double ia = 1.0 / s.a;
  const double ia2 = ia * ia;
  isg = 0.5 * ia;
  const double d23 = l2 - l3;
  const double s23 = l2 + l3 - 2.0 * l1;
  const double t3 = -0.25 * s.r * s.sigma;  // r (0 - sigma^2) / (4 sigma)
  const double t5 = 0.5 * s23;              // (s23 sigma) / (2 sigma)
  const double t6 = 0.5 * (l2 + l3);
  const double cp = g.gamma * g.Rt / gm1;
  const double rT = -g.gamma * g.Rt * s.r * ia2;  // -gamma R rho / ((gamma - 1) h)
  const double irT = 1.0 / rT;
  RoeK k;
  k.l1 = l1;
  k.rT = rT;
  k.rho = s.r;
  const double dt3 = d23 * t3 * ia2;
  k.c7 = dt3;
  k.c8 = (g.gamma * t6 - gm1 * t5) * ia2;
  k.c9 = cp * s.r + s.h0 * rT;
  const double x1 = g.gamma * s.h0 * dt3;
  const double x2 = -gm1 * dt3 * k.c9 * irT;
  const double x3 = -d23 * t3;
  const double x4 = 0.5 * s.r * s23 * s.unA;  // r t4 unA / (2 sigma), t4 = s23 sigma
  k.c10 = (x1 + x2 + x3 + x4);
  k.c11 = (ia2 * s.h0 + (k.c9 - s.r * cp) * ia2 * gm1 * irT - 1.0) * t6 -
          gm1 * ia2 * k.c9 * t5 * irT - s.unA * d23 * isg;
  k.c4 = 0.5 * s.r * s23;  // r t4 / (2 sigma)
  k.c1 = d23 * isg;
  k.t4 = s23 * s.sigma;
  k.d23 = d23;
  return k;
}

__device__ __forceinline__ RoeK roe_k(double l1, double l2, double l3, const RoeAvg& s,
                                      const Gas& g) {
  const double beta = s.eta, sg = s.sigma, un = s.un;
  const double bm = beta - 1.0;
  const double d23 = l2 - l3;
  const double s23 = l2 + l3 - 2.0 * l1;
  const double t3 = s.r * (bm * bm * un * un - sg * sg) / (4.0 * sg);
  const double t4 = s23 * sg + bm * d23 * un;
  const double t5 = (s23 * sg - bm * d23 * un) / (2.0 * sg);
  const double t6 = ((l2 + l3) * sg - bm * d23 * un) / (2.0 * sg);
  const double gm1 = g.gamma - 1.0;
  const double cp = g.gamma * g.Rt / gm1;
  const double rT = -g.gamma * g.Rt * s.r /
                    ((s.h0 - 0.5 * (s.U * s.U + s.V * s.V + s.W * s.W)) * gm1);
  const double ib = 1.0 / beta;
  const double ia2 = 1.0 / (s.a * s.a);
  RoeK k;
  k.l1 = l1;
  k.rT = rT;
  k.rho = s.r;
  k.c7 = ib * d23 * t3 * ia2;
  k.c8 = (((ib - 1.0) + g.gamma) * t6 - gm1 * t5) * ia2;
  k.c9 = cp * s.r + s.h0 * rT;
  const double x1 = g.gamma * s.h0 * d23 * t3 * ia2 * ib;
  const double x2 = -ib * gm1 * d23 * t3 * k.c9 * ia2 / rT;
  const double x3 = -d23 * t3 * ib;
  const double x4 = 0.5 * s.r * t4 * s.unA / sg;
  k.c10 = (x1 + x2 + x3 + x4);
  k.c11 = (ib * ia2 * s.h0 + (k.c9 - s.r * ib * cp) * ia2 * gm1 / rT - ib) * t6 -
          gm1 * ia2 * k.c9 * t5 / rT - s.unA * d23 / sg;
  k.c4 = s.r * t4 / (2.0 * sg);
  k.c1 = d23 / sg;
  k.t4 = t4;
  k.d23 = d23;
  return k;
}

// y = K dq
__device__ __forceinline__ void roe_k_apply(const RoeK& k, const RoeAvg& s, double nx,
                                            double ny, double nz, const double dq[5],
                                            double y[5]) {
  const double dun = nx * dq[1] + ny * dq[2] + nz * dq[3];
  const double Ud = s.U * dq[1] + s.V * dq[2] + s.W * dq[3];
  const double a1 = k.l1 * k.rT * dq[0];
  y[0] = a1 + k.c7 * dun + k.c8 * dq[4];
  y[1] = a1 * s.U + (k.c7 * s.U + nx * k.c4) * dun + k.l1 * k.rho * dq[1] +
         (k.c8 * s.U - nx * k.c1) * dq[4];
  y[2] = a1 * s.V + (k.c7 * s.V + ny * k.c4) * dun + k.l1 * k.rho * dq[2] +
         (k.c8 * s.V - ny * k.c1) * dq[4];
  y[3] = a1 * s.W + (k.c7 * s.W + nz * k.c4) * dun + k.l1 * k.rho * dq[3] +
         (k.c8 * s.W - nz * k.c1) * dq[4];
  y[4] = k.l1 * k.c9 * dq[0] + k.c10 * dun + k.l1 * k.rho * Ud + k.c11 * dq[4];
}

// M = area * K, row-major
template <class TB>
__device__ __forceinline__ void roe_k_matrix(const RoeK& k, const RoeAvg& s, double nx,
                                             double ny, double nz, double area, TB* M) {
  const double n[3] = {nx, ny, nz};
  const double U[3] = {s.U, s.V, s.W};
  M[0] = TB(area * (k.l1 * k.rT));
#pragma unroll
  for (int m = 0; m < 3; ++m) M[1 + m] = TB(area * (n[m] * k.c7));
  M[4] = TB(area * k.c8);
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    M[5 * (1 + r)] = TB(area * (k.l1 * k.rT * U[r]));
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      double v = n[m] * (k.c7 * U[r] + n[r] * k.c4);
      if (r == m) v += k.l1 * k.rho;
      M[5 * (1 + r) + 1 + m] = TB(area * v);
    }
    M[5 * (1 + r) + 4] = TB(area * (k.c8 * U[r] - n[r] * k.c1));
  }
  M[20] = TB(area * (k.l1 * k.c9));
#pragma unroll
  for (int m = 0; m < 3; ++m) M[21 + m] = TB(area * (n[m] * k.c10 + k.l1 * k.rho * U[m]));
  M[24] = TB(area * k.c11);
}

// roeCT_flux: central part plus K(|l|) dissipation with the Harten-Hyman
// entropy fix on the acoustic waves (:918-962).
__device__ __forceinline__ void flux_roe(const Q5& L, const Q5& R, double nx, double ny,
                                         double nz, double area, const Gas& g, double us_n,
                                         double eta, double F[5]) {
  const RoeAvg s = roe_average(L, R, nx, ny, nz, g, us_n, eta);
  const double ep = s.eta + 1.0, em = s.eta - 1.0;
  const double l2s = 0.5 * (s.un * ep - s.sigma);
  const double l3s = 0.5 * (s.un * ep + s.sigma);
  double l1 = fabs(s.un), l2 = fabs(l2s), l3 = fabs(l3s);
  const double unlA = L.u * nx + L.v * ny + L.w * nz, unrA = R.u * nx + R.v * ny + R.w * nz;
  const double unl = unlA - us_n, unr = unrA - us_n;
  const double sl = sqrt(unl * unl * em * em + 4.0 * s.eta * g.gamma * g.Rt * L.T);
  const double sr = sqrt(unr * unr * em * em + 4.0 * s.eta * g.gamma * g.Rt * R.T);
  const double w2 = dmax(0.0, dmax(l2s - 0.5 * (unl * ep - sl), 0.5 * (unr * ep - sr) - l2s));
  const double w3 = dmax(0.0, dmax(l3s - 0.5 * (unl * ep + sl), 0.5 * (unr * ep + sr) - l3s));
  if (l2 < w2) l2 = 0.5 * ((l2s * l2s) / w2 + w2);
  if (l3 < w3) l3 = 0.5 * ((l3s * l3s) / w3 + w3);
  const RoeK k = roe_k(l1, l2, l3, s, g);
  // K(|l|) dq with the association of fluxInviscid.loci:985-1004 (the
  // quotients by sigma below share one reciprocal), so the FP64 flux agrees
  // with the reference to within a few ulp of its terms
  const double dT = R.T - L.T, dp = R.p - L.p;
  const double du = R.u - L.u, dv = R.v - L.v, dw = R.w - L.w;
  const double uj = du * nx + dv * ny + dw * nz;
  // the six quotients by sigma and 2 sigma share one reciprocal (each term
  // moves by at most an ulp against the division)
  const double isg = 1.0 / s.sigma;
  const double dsg = k.d23 * isg, tsg = s.r * k.t4 * uj * (0.5 * isg);
  double d[5];
  d[0] = dp * k.c8 + uj * k.c7 + l1 * dT * k.rT;
  d[1] = s.U * k.c7 * uj + l1 * (s.U * dT * k.rT + s.r * du) + dp * (k.c8 * s.U - nx * dsg) + nx * tsg;
  d[2] = s.V * k.c7 * uj + l1 * (s.V * dT * k.rT + s.r * dv) + dp * (k.c8 * s.V - ny * dsg) + ny * tsg;
  d[3] = s.W * k.c7 * uj + l1 * (s.W * dT * k.rT + s.r * dw) + dp * (k.c8 * s.W - nz * dsg) + nz * tsg;
  d[4] = dp * k.c11 + k.c10 * uj + l1 * (k.c9 * dT + s.r * (s.U * du + s.V * dv + s.W * dw));
  const double ah = 0.5 * area;
  const double ml = s.rl * unl, mr = s.rr * unr;
  const double pl = L.p + g.pamb, pr = R.p + g.pamb;
  F[0] = ah * (ml + mr - d[0]);
  F[1] = ah * (L.u * ml + R.u * mr + nx * (L.p + R.p) - d[1]);
  F[2] = ah * (L.v * ml + R.v * mr + ny * (L.p + R.p) - d[2]);
  F[3] = ah * (L.w * ml + R.w * mr + nz * (L.p + R.p) - d[3]);
  F[4] = ah * ((s.rel * unl + pl * unlA) + (s.rer * unr + pr * unrA) - d[4]);
}

// roeCT_flux at eta == 1 on a fixed grid (see roe_average1)
__device__ __forceinline__ void flux_roe1(const Q5& L, const Q5& R, double nx, double ny,
                                          double nz, double area, const Gas& g, double F[5]) {
  const RoeAvg s = roe_average1(L, R, nx, ny, nz, g);
  const double l2s = s.un - s.a;  // (un (eta + 1) - sigma) / 2
  const double l3s = s.un + s.a;
  double l1 = fabs(s.un), l2 = fabs(l2s), l3 = fabs(l3s);
  const double unl = L.u * nx + L.v * ny + L.w * nz, unr = R.u * nx + R.v * ny + R.w * nz;
  const double hl = sqrt(g.gamma * g.Rt * L.T), hr = sqrt(g.gamma * g.Rt * R.T);  // sigma / 2
  const double w2 = dmax(0.0, dmax(l2s - (unl - hl), (unr - hr) - l2s));
  const double w3 = dmax(0.0, dmax(l3s - (unl + hl), (unr + hr) - l3s));
  if (l2 < w2) l2 = 0.5 * ((l2s * l2s) / w2 + w2);
  if (l3 < w3) l3 = 0.5 * ((l3s * l3s) / w3 + w3);
  double isg;
  const RoeK k = roe_k1(l1, l2, l3, s, g, isg);
  const double dT = R.T - L.T, dp = R.p - L.p;
  const double du = R.u - L.u, dv = R.v - L.v, dw = R.w - L.w;
  const double uj = du * nx + dv * ny + dw * nz;
  const double dsg = k.d23 * isg, tsg = s.r * k.t4 * uj * (0.5 * isg);
  double d[5];
  d[0] = dp * k.c8 + uj * k.c7 + l1 * dT * k.rT;
  d[1] = s.U * k.c7 * uj + l1 * (s.U * dT * k.rT + s.r * du) + dp * (k.c8 * s.U - nx * dsg) + nx * tsg;
  d[2] = s.V * k.c7 * uj + l1 * (s.V * dT * k.rT + s.r * dv) + dp * (k.c8 * s.V - ny * dsg) + ny * tsg;
  d[3] = s.W * k.c7 * uj + l1 * (s.W * dT * k.rT + s.r * dw) + dp * (k.c8 * s.W - nz * dsg) + nz * tsg;
  d[4] = dp * k.c11 + k.c10 * uj + l1 * (k.c9 * dT + s.r * (s.U * du + s.V * dv + s.W * dw));
  const double ah = 0.5 * area;
  const double ml = s.rl * unl, mr = s.rr * unr;
  const double pl = L.p + g.pamb, pr = R.p + g.pamb;
  F[0] = ah * (ml + mr - d[0]);
  F[1] = ah * (L.u * ml + R.u * mr + nx * (L.p + R.p) - d[1]);
  F[2] = ah * (L.v * ml + R.v * mr + ny * (L.p + R.p) - d[2]);
  F[3] = ah * (L.w * ml + R.w * mr + nz * (L.p + R.p) - d[3]);
  F[4] = ah * ((s.rel * unl + pl * unl) + (s.rer * unr + pr * unr) - d[4]);
}

// smoothed eigenvalue Jacobian coefficients at eta == 1 (roe_k_smoothed)
__device__ __forceinline__ RoeK roe_k_smoothed1(const RoeAvg& s, const Gas& g, int dir) {
  double l1 = s.un;
  double l2 = s.un - s.a;
  double l3 = s.un + s.a;
  const double hi = dmax(l1, dmax(l2, l3)), lo = dmin(l1, dmin(l2, l3));
  const double e = 0.02 * (hi - lo);
  const double e2 = e * e;
  const double d = dir < 0 ? -1.0 : 1.0;
  l1 = 0.5 * (l1 + d * sqrt(l1 * l1 + e2));
  l2 = 0.5 * (l2 + d * sqrt(l2 * l2 + e2));
  l3 = 0.5 * (l3 + d * sqrt(l3 * l3 + e2));
  double isg;
  return roe_k1(l1, l2, l3, s, g, isg);
}

// Smoothed one-sided eigenvalue Jacobian, roeCT_jacobian (:1141-1167):
// l -> (l +- sqrt(l^2 + (0.02 (lmax - lmin))^2)) / 2.
__device__ __forceinline__ RoeK roe_k_smoothed(const RoeAvg& s, const Gas& g, int dir) {
  const double ep = s.eta + 1.0;
  double l1 = s.un;
  double l2 = 0.5 * (s.un * ep - s.sigma);
  double l3 = 0.5 * (s.un * ep + s.sigma);
  const double hi = dmax(l1, dmax(l2, l3)), lo = dmin(l1, dmin(l2, l3));
  const double e = 0.02 * (hi - lo);
  const double e2 = e * e;
  const double d = dir < 0 ? -1.0 : 1.0;
  l1 = 0.5 * (l1 + d * sqrt(l1 * l1 + e2));
  l2 = 0.5 * (l2 + d * sqrt(l2 * l2 + e2));
  l3 = 0.5 * (l3 + d * sqrt(l3 * l3 + e2));
  return roe_k(l1, l2, l3, s, g);
}

template <class TB>
__device__ __forceinline__ void jac_roe(const RoeAvg& s, double nx, double ny, double nz,
                                        double area, const Gas& g, int dir, TB* M) {
  roe_k_matrix<TB>(roe_k_smoothed(s, g, dir), s, nx, ny, nz, area, M);
}

template <class TB>
__device__ __forceinline__ void jac_roe1(const RoeAvg& s, double nx, double ny, double nz,
                                         double area, const Gas& g, int dir, TB* M) {
  roe_k_matrix<TB>(roe_k_smoothed1(s, g, dir), s, nx, ny, nz, area, M);
}

// Compact form of area * K: nine per-direction coefficients (area folded in)
// with which, for x = (x0, x_m, x4) and dun = n . x_m,
//   y0  = a1 x0 + c7 dun + c8 x4
//   y_r = U_r y0 + n_r (c4 dun - c1 x4) + lr x_r          (r = 1..3)
//   y4  = l9 x0 + c10 dun + lr (U . x_m) + c11 x4
// is y = area K x.  With U and n, which both directions of a face share,
// 15 numbers hold the matrix that roe_k_matrix spells out in 25.
// A face record holds both directions: [+ (9) | - (9) | U (3) | n (3)];
// a sweep slot holds one: [dir (9) | U (3) | n (3)].
enum { CK_A1, CK_C7, CK_C8, CK_C4, CK_C1, CK_LR, CK_L9, CK_C10, CK_C11, CK_DIR };
constexpr int CK_FACE = 2 * CK_DIR + 6;  // 24
constexpr int CK_SLOT = CK_DIR + 6;      // 15

template <class TB, bool ETA1 = false>
__device__ __forceinline__ void jac_roe_compact(const RoeAvg& s, double area, const Gas& g, int dir,
                                                TB* c) {
  const RoeK k = ETA1 ? roe_k_smoothed1(s, g, dir) : roe_k_smoothed(s, g, dir);
  c[CK_A1] = TB(area * (k.l1 * k.rT));
  c[CK_C7] = TB(area * k.c7);
  c[CK_C8] = TB(area * k.c8);
  c[CK_C4] = TB(area * k.c4);
  c[CK_C1] = TB(area * k.c1);
  c[CK_LR] = TB(area * (k.l1 * k.rho));
  c[CK_L9] = TB(area * (k.l1 * k.c9));
  c[CK_C10] = TB(area * k.c10);
  c[CK_C11] = TB(area * k.c11);
}

// The 25 entries (row-major) of the matrix held by direction coefficients
// c[9] and the face's U[3], n[3]; each entry evaluated in FP64 and rounded
// once, as roe_k_matrix does.
template <class TB>
__device__ __forceinline__ void compact_expand(const TB* c, const TB* Uf, const TB* nf, TB* M) {
  const double a1 = c[CK_A1], c7 = c[CK_C7], c8 = c[CK_C8], c4 = c[CK_C4], c1 = c[CK_C1];
  const double lr = c[CK_LR], l9 = c[CK_L9], c10 = c[CK_C10], c11 = c[CK_C11];
  const double U[3] = {double(Uf[0]), double(Uf[1]), double(Uf[2])};
  const double n[3] = {double(nf[0]), double(nf[1]), double(nf[2])};
  M[0] = TB(a1);
#pragma unroll
  for (int m = 0; m < 3; ++m) M[1 + m] = TB(n[m] * c7);
  M[4] = TB(c8);
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    M[5 * (1 + r)] = TB(a1 * U[r]);
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      double v = n[m] * (c7 * U[r] + n[r] * c4);
      if (r == m) v += lr;
      M[5 * (1 + r) + 1 + m] = TB(v);
    }
    M[5 * (1 + r) + 4] = TB(c8 * U[r] - n[r] * c1);
  }
  M[20] = TB(l9);
#pragma unroll
  for (int m = 0; m < 3; ++m) M[21 + m] = TB(n[m] * c10 + lr * U[m]);
  M[24] = TB(c11);
}

// y += M x for the matrix of one sweep slot s[15] (coefficients, U, n), in
// the iterate's precision
template <class TB, class TX>
__device__ __forceinline__ void compact_apply(const TB* s, const TX* x, TX* y) {
  const TX a1 = TX(s[CK_A1]), c7 = TX(s[CK_C7]), c8 = TX(s[CK_C8]), c4 = TX(s[CK_C4]);
  const TX c1 = TX(s[CK_C1]), lr = TX(s[CK_LR]), l9 = TX(s[CK_L9]), c10 = TX(s[CK_C10]);
  const TX c11 = TX(s[CK_C11]);
  const TX U0 = TX(s[CK_DIR]), U1 = TX(s[CK_DIR + 1]), U2 = TX(s[CK_DIR + 2]);
  const TX n0 = TX(s[CK_DIR + 3]), n1 = TX(s[CK_DIR + 4]), n2 = TX(s[CK_DIR + 5]);
  const TX dun = n0 * x[1] + n1 * x[2] + n2 * x[3];
  const TX y0 = a1 * x[0] + c7 * dun + c8 * x[4];
  const TX w = c4 * dun - c1 * x[4];
  y[0] += y0;
  y[1] += U0 * y0 + n0 * w + lr * x[1];
  y[2] += U1 * y0 + n1 * w + lr * x[2];
  y[3] += U2 * y0 + n2 * w + lr * x[3];
  y[4] += l9 * x[0] + c10 * dun + lr * (U0 * x[1] + U1 * x[2] + U2 * x[3]) + c11 * x[4];
}

// hllc_flux (fluxInviscid.loci:157-256) and the HLL two-wave flux built on
// the same SL/SR estimates.
struct Waves {
  double rl, rr, el, er, unlA, unrA, unl, unr, SL, SR;
};
__device__ __forceinline__ Waves hll_waves(const Q5& L, const Q5& R, double nx, double ny,
                                           double nz, const Gas& g, double us_n, double eta) {
  Waves w;
  const double gm1 = g.gamma - 1.0;
  w.rl = (L.p + g.pamb) / (g.Rt * L.T);
  w.rr = (R.p + g.pamb) / (g.Rt * R.T);
  const double h0l = g.Rt * L.T * g.gamma / gm1 + 0.5 * (L.u * L.u + L.v * L.v + L.w * L.w);
  const double h0r = g.Rt * R.T * g.gamma / gm1 + 0.5 * (R.u * R.u + R.v * R.v + R.w * R.w);
  w.el = h0l - g.Rt * L.T;
  w.er = h0r - g.Rt * R.T;
  const double wl = sqrt(w.rl), wr = sqrt(w.rr), iw = 1.0 / (wl + wr);
  const double U = (L.u * wl + R.u * wr) * iw, V = (L.v * wl + R.v * wr) * iw,
               W = (L.w * wl + R.w * wr) * iw;
  const double un = U * nx + V * ny + W * nz - us_n;
  const double h0 = (h0l * wl + h0r * wr) * iw;
  const double a = sqrt(dmax(gm1 * (h0 - 0.5 * (U * U + V * V + W * W)), 0.0));
  const double ep = eta + 1.0, em = eta - 1.0;
  const double sg = sqrt(dmax(un * un * em * em + 4.0 * eta * a * a, 1e-30));
  w.unlA = L.u * nx + L.v * ny + L.w * nz;
  w.unrA = R.u * nx + R.v * ny + R.w * nz;
  w.unl = w.unlA - us_n;
  w.unr = w.unrA - us_n;
  const double sr = sqrt(dmax(w.unr * w.unr * em * em + 4.0 * eta * g.gamma * g.Rt * R.T, 0.0));
  const double sl = sqrt(dmax(w.unl * w.unl * em * em + 4.0 * eta * g.gamma * g.Rt * L.T, 0.0));
  w.SL = dmin(0.5 * (un * ep - sg), 0.5 * (w.unl * ep - sl));
  w.SR = dmax(0.5 * (un * ep + sg), 0.5 * (w.unr * ep + sr));
  return w;
}

__device__ __forceinline__ void flux_hllc(const Q5& L, const Q5& R, double nx, double ny,
                                          double nz, double area, const Gas& g, double us_n,
                                          double eta, double F[5]) {
  const Waves w = hll_waves(L, R, nx, ny, nz, g, us_n, eta);
  const double SL = w.SL, SR = w.SR, rl = w.rl, rr = w.rr;
  const double ml = rl * w.unl, mr = rr * w.unr;
  const double pl = L.p + g.pamb, pr = R.p + g.pamb;
  const double c = 0.5 * area;
  const double AL = c * ((SL > 0) ? (SR < 0 ? 1. : 2.) : (SR < 0 ? 0. : 1.));
  const double AR = c * ((SR < 0) ? (SL > 0 ? 1. : 2.) : (SL > 0 ? 0. : 1.));
  const double AM = c * ((SL > 0 || SR < 0) ? 0. : 1.);
  F[0] = AL * ml + AR * mr;
  F[1] = AL * ml * L.u + AR * mr * R.u + nx * (AL * L.p + AR * R.p);
  F[2] = AL * ml * L.v + AR * mr * R.v + ny * (AL * L.p + AR * R.p);
  F[3] = AL * ml * L.w + AR * mr * R.w + nz * (AL * L.p + AR * R.p);
  F[4] = AL * (ml * w.el + pl * w.unlA) + AR * (mr * w.er + pr * w.unrA);
  F[0] -= AM * (SL * rl + SR * rr);
  F[1] -= AM * (SL * rl * L.u + SR * rr * R.u);
  F[2] -= AM * (SL * rl * L.v + SR * rr * R.v);
  F[3] -= AM * (SL * rl * L.w + SR * rr * R.w);
  F[4] -= AM * (SL * rl * w.el + SR * rr * w.er);
  const double unl = w.unl, unr = w.unr;
  const double SM = ((rr * unr * (SR - unr) - rl * unl * (SL - unl) + L.p - R.p) /
                     (rr * (SR - unr) - rl * (SL - unl)));
  const double il = 1.0 / (SL - SM), ir = 1.0 / (SR - SM);
  const double pgs = rl * (unl - SL) * (unl - SM) + L.p;
  const double ps = pgs + g.pamb;
  const double CR = SR - fabs(SM), CL = SL + fabs(SM);
  const double fl = (SL - unl) * rl, fr = (SR - unr) * rr;
  // star states U*_L, U*_R (conserved), weighted by CL, CR; the ten
  // quotients by SR - SM and SL - SM share two reciprocals
  F[0] += AM * (CR * (fr * ir) + CL * (fl * il));
  F[1] += AM * (CR * ((fr * R.u + (pgs - R.p) * nx) * ir) + CL * ((fl * L.u + (pgs - L.p) * nx) * il));
  F[2] += AM * (CR * ((fr * R.v + (pgs - R.p) * ny) * ir) + CL * ((fl * L.v + (pgs - L.p) * ny) * il));
  F[3] += AM * (CR * ((fr * R.w + (pgs - R.p) * nz) * ir) + CL * ((fl * L.w + (pgs - L.p) * nz) * il));
  F[4] += AM * (CR * ((fr * w.er - pr * unr + ps * SM) * ir) +
                CL * ((fl * w.el - pl * unl + ps * SM) * il));
}

__device__ __forceinline__ void analytic_flux(const Q5& q, double rho, double e0, double unA,
                                              double un, double nx, double ny, double nz,
                                              double area, const Gas& g, double f[5]) {
  const double m = area * rho * un;
  f[0] = m;
  f[1] = m * q.u + area * q.p * nx;
  f[2] = m * q.v + area * q.p * ny;
  f[3] = m * q.w + area * q.p * nz;
  f[4] = m * e0 + area * (q.p + g.pamb) * unA;
}

__device__ __forceinline__ void flux_hlle(const Q5& L, const Q5& R, double nx, double ny,
                                          double nz, double area, const Gas& g, double us_n,
                                          double eta, double F[5]) {
  const Waves w = hll_waves(L, R, nx, ny, nz, g, us_n, eta);
  double fl[5], fr[5];
  analytic_flux(L, w.rl, w.el, w.unlA, w.unl, nx, ny, nz, area, g, fl);
  analytic_flux(R, w.rr, w.er, w.unrA, w.unr, nx, ny, nz, area, g, fr);
  if (w.SL >= 0) {
#pragma unroll
    for (int i = 0; i < 5; ++i) F[i] = fl[i];
    return;
  }
  if (w.SR <= 0) {
#pragma unroll
    for (int i = 0; i < 5; ++i) F[i] = fr[i];
    return;
  }
  const double ql[5] = {w.rl, w.rl * L.u, w.rl * L.v, w.rl * L.w, w.rl * w.el};
  const double qr[5] = {w.rr, w.rr * R.u, w.rr * R.v, w.rr * R.w, w.rr * w.er};
  const double id = 1.0 / (w.SR - w.SL);
  const double ss = area * w.SL * w.SR;
#pragma unroll
  for (int i = 0; i < 5; ++i) F[i] = (w.SR * fl[i] - w.SL * fr[i] + ss * (qr[i] - ql[i])) * id;
}

__device__ __forceinline__ void riemann(int kind, const Q5& L, const Q5& R, double nx,
                                        double ny, double nz, double area, const Gas& g,
                                        double us_n, double eta, double F[5]) {
  if (kind == 1)
    flux_roe(L, R, nx, ny, nz, area, g, us_n, eta, F);
  else if (kind == 2)
    flux_hlle(L, R, nx, ny, nz, area, g, us_n, eta, F);
  else
    flux_hllc(L, R, nx, ny, nz, area, g, us_n, eta, F);
}

// the face flux of the mesh kernels: eta == 1, fixed grid
__device__ __forceinline__ void riemann1(int kind, const Q5& L, const Q5& R, double nx,
                                         double ny, double nz, double area, const Gas& g,
                                         double F[5]) {
  if (kind == 1)
    flux_roe1(L, R, nx, ny, nz, area, g, F);
  else if (kind == 2)
    flux_hlle(L, R, nx, ny, nz, area, g, 0.0, 1.0, F);
  else
    flux_hllc(L, R, nx, ny, nz, area, g, 0.0, 1.0, F);
}

// ---- low-dissipation (KEC) flux, fluxLowDiss.loci -----------------------
// The central kinetic-energy-consistent flux of two states through a face of
// area A (kec_flux, fluxLowDiss.loci:258-298), added to F: the mean velocity
// and gauge pressure, the density-averaged temperature, the internal energy
// of the mean temperature and the kinetic energy |u_f|^2 - (|u_l|^2 + |u_r|^2)/4.
__device__ __forceinline__ void kec_flux_add(const Q5& l, const Q5& r, double nx, double ny,
                                             double nz, double A, const Gas& g, double F[5]) {
  const double ux = 0.5 * (l.u + r.u), uy = 0.5 * (l.v + r.v), uz = 0.5 * (l.w + r.w);
  const double ufn = ux * nx + uy * ny + uz * nz;
  const double pgf = 0.5 * (l.p + r.p);
  const double tf =
      l.T * r.T * (l.p + r.p + 2 * g.pamb) / ((l.p + g.pamb) * r.T + (r.p + g.pamb) * l.T);
  const double rf = (pgf + g.pamb) / (g.Rt * tf);
  const double mdot = rf * ufn;
  F[0] += A * mdot;
  F[1] += A * (mdot * ux + pgf * nx);
  F[2] += A * (mdot * uy + pgf * ny);
  F[3] += A * (mdot * uz + pgf * nz);
  const double ei = 0.5 * g.Rt * (l.T + r.T) / (g.gamma - 1);
  const double ke = (ux * ux + uy * uy + uz * uz) -
                    0.25 * ((l.u * l.u + l.v * l.v + l.w * l.w) + (r.u * r.u + r.v * r.v + r.w * r.w));
  F[4] += A * (mdot * (ke + ei) + ufn * (pgf + g.pamb));
}

// KEC::iflux of an interior face (fluxLowDiss.loci:320-431).  L, R: the
// MUSCL face states with their floors; qa, qb: the two cell states; ga, gb:
// their gradient (15) and limiter (5) records; dv = x_f - (x_l + x_r) / 2;
// aa, ab: the cells' alpha_diss; ag: the face's alpha_geom_f.  The upwind
// part is hllc_flux (inviscidRiemannFlux, inviscidFlux.h:82-90) of the
// Thornber-preconditioned states on the area A alpha, the central part
// kec_flux of the states reconstructed to dv on the area A (1 - alpha).
__device__ __forceinline__ void kec_face(const Q5& L, const Q5& R, const Q5& qa, const Q5& qb,
                                         const double* ga, const double* gb, double dvx,
                                         double dvy, double dvz, double aa, double ab, double ag,
                                         double nx, double ny, double nz, double A, const Gas& g,
                                         double F[5]) {
  const double pglim = 0.1 * dmin(qa.p, qb.p) + -0.9 * g.pamb;
  const double tlim = 0.1 * dmin(qa.T, qb.T);
  const double rl = (L.p + g.pamb) / (g.Rt * L.T), rr = (R.p + g.pamb) / (g.Rt * R.T);
  const double al2 = g.gamma * g.Rt * L.T, ar2 = g.gamma * g.Rt * R.T;
  const double dp = 2. * fabs(L.p - R.p) / dmax(rl * al2, rr * ar2);
  const double alpha_c = dmax(dmax(aa, ab), dmin(1.0, dp * 1.0 - 0.5));
  const double alpha = dmax(alpha_c, ag);
#pragma unroll
  for (int i = 0; i < 5; ++i) F[i] = 0.0;
  if (alpha > 1e-10) {
    const double amin = sqrt(dmin(al2, ar2));
    const double utmax = dmax(fabs(L.u * nx + L.v * ny + L.w * nz), fabs(R.u * nx + R.v * ny + R.w * nz));
    const double Ma = dmax(alpha_c, dmin(1.0, utmax / amin + 1e-4));
    const double h = 0.5 * (1. - Ma);
    Q5 Lp = L, Rp = R;
    Lp.u = L.u + h * (R.u - L.u), Lp.v = L.v + h * (R.v - L.v), Lp.w = L.w + h * (R.w - L.w);
    Rp.u = R.u + h * (L.u - R.u), Rp.v = R.v + h * (L.v - R.v), Rp.w = R.w + h * (L.w - R.w);
    flux_hllc(Lp, Rp, nx, ny, nz, A * alpha, g, 0.0, 1.0, F);
  }
  auto at = [&](const Q5& c, const double* gr, Q5& o) {
    const double* ph = gr + 15;
    double d[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) d[k] = gr[3 * k] * dvx + gr[3 * k + 1] * dvy + gr[3 * k + 2] * dvz;
    o.p = dmax(c.p + ph[4] * d[4], pglim);
    o.T = dmax(c.T + ph[0] * d[0], tlim);
    o.u = c.u + ph[1] * d[1];
    o.v = c.v + ph[2] * d[2];
    o.w = c.w + ph[3] * d[3];
  };
  Q5 l, r;
  at(qa, ga, l);
  at(qb, gb, r);
  kec_flux_add(l, r, nx, ny, nz, A * (1. - alpha), g, F);
}

// The Roe-type dissipation of two states (roedis, fluxLowDiss.loci:180-270)
// on the area `area`, subtracted from F: eigenvalues of the Roe-averaged
// state with the face sound speed a^2 = 2 a_l^2 a_r^2 / (a_l^2 + a_r^2),
// applied to the jumps in p, u and T.
__device__ __forceinline__ void roe_dissipation_sub(const Q5& l, const Q5& r, double nx, double ny,
                                                    double nz, double area, const Gas& g,
                                                    double F[5]) {
  const double pl = l.p + g.pamb, pr = r.p + g.pamb;
  const double rl = pl / (g.Rt * l.T), rr = pr / (g.Rt * r.T);
  const double rgm1 = 1. / (g.gamma - 1);
  const double el = g.Rt * rgm1 * l.T, er = g.Rt * rgm1 * r.T;
  const double re0l = rl * el + 0.5 * rl * (l.u * l.u + l.v * l.v + l.w * l.w);
  const double re0r = rr * er + 0.5 * rr * (r.u * r.u + r.v * r.v + r.w * r.w);
  const double h0l = (re0l + pl) / rl, h0r = (re0r + pr) / rr;
  const double rho = sqrt(rl * rr);
  const double wl = sqrt(rl), wr = sqrt(rr), iw = 1. / (wl + wr);
  const double U = (l.u * wl + r.u * wr) * iw, V = (l.v * wl + r.v * wr) * iw,
               W = (l.w * wl + r.w * wr) * iw;
  const double un = U * nx + V * ny + W * nz;  // fixed grid: the relative and absolute speeds agree
  const double h0 = (h0l * wl + h0r * wr) * iw;
  const double al2 = g.gamma * g.Rt * l.T, ar2 = g.gamma * g.Rt * r.T;
  const double af2 = dmax(2. * al2 * ar2 / (al2 + ar2), 1e-30);
  const double cp = g.Rt * g.gamma * rgm1;
  const double Tm = (l.T * ar2 + r.T * al2) * af2 / (2. * ar2 * al2);
  const double rT = -rho / Tm;
  const double a = sqrt(af2);
  const double ev1 = fabs(un), ev2 = fabs(un - a), ev3 = fabs(un + a);
  const double ujx = r.u - l.u, ujy = r.v - l.v, ujz = r.w - l.w;
  const double utj = ujx * nx + ujy * ny + ujz * nz;
  const double pj = r.p - l.p, Tj = r.T - l.T;
  const double t1 = ev2 - ev3, t2 = (ev2 + ev3 - 2 * ev1), t3 = -rho * a / 2.;
  const double t4 = 2. * t2 * a, t5 = t2 / 2., t6 = (ev2 + ev3) / 2.;
  const double c1 = (1 - g.gamma) / rT;
  const double ra2 = 1. / (a * a);
  const double gm1 = g.gamma - 1;
  const double t7 = (1 + gm1 + c1 * rT) * t1 * t3 * ra2;
  const double t8 = (g.gamma * t6 + c1 * rT * t5) * ra2;
  const double t9 = cp * rho + h0 * rT;
  const double x1 = g.gamma * h0 * t1 * t3 * ra2;
  const double x2 = c1 * t1 * t3 * t9 * ra2;
  const double x3 = rT * Tm * t1 * t3 * 1 / rho;
  const double x4 = .25 * rho * t4 * un / a;
  const double t10 = (x1 + x2 + x3 + x4);
  const double t11 = (ra2 * h0 + (t9 - rho * cp) * ra2 * gm1 / rT + rT * Tm / rho) * t6 +
                     ra2 * t9 * t5 * c1 - .5 * un * t1 / a;
  const double coef = 0.5 * area;
  const double md = coef * (pj * t8 + utj * t7 + ev1 * Tj * rT);
  F[0] -= md;
  const double fp = .5 * (.5 * rho * t4 * utj - pj * t1) / a;
  F[1] -= md * U + coef * (ev1 * rho * ujx + fp * nx);
  F[2] -= md * V + coef * (ev1 * rho * ujy + fp * ny);
  F[3] -= md * W + coef * (ev1 * rho * ujz + fp * nz);
  F[4] -= coef * (pj * t11 + t10 * utj + ev1 * (t9 * Tj + rho * (U * ujx + V * ujy + W * ujz)));
}

// SSF::iflux of an interior face (fluxLowDiss.loci:436-640): the 4th-order
// skew-symmetric scheme.  Arguments as kec_face, plus d2 = x_r - x_l, the
// SSF coefficient and the MILES filter level.  Upwind part as KEC's but
// switched by alpha_c alone; central part: kec_flux of (l, r) on (1 + 2C)
// A (1 - alpha) and of (l, rr) and (ll, r) on -C A (1 - alpha), C = coeff/6,
// with ll, rr extrapolated along d2; then the Roe dissipation of the cubic
// face values (1/3, 5/6, -1/6), Thornber-preconditioned, on the area
// max(alpha_geom_f, filter) A (1 - alpha).
__device__ __forceinline__ void ssf_face(const Q5& L, const Q5& R, const Q5& qa, const Q5& qb,
                                         const double* ga, const double* gb, double dvx,
                                         double dvy, double dvz, double d2x, double d2y, double d2z,
                                         double aa, double ab, double ag, double coeff,
                                         double filter, double nx, double ny, double nz, double A,
                                         const Gas& g, double F[5]) {
  const double pglim = 0.1 * dmin(qa.p, qb.p) + -0.9 * g.pamb;
  const double tlim = 0.1 * dmin(qa.T, qb.T);
  const double rl = (L.p + g.pamb) / (g.Rt * L.T), rr = (R.p + g.pamb) / (g.Rt * R.T);
  const double al2 = g.gamma * g.Rt * L.T, ar2 = g.gamma * g.Rt * R.T;
  const double dp = 2. * fabs(L.p - R.p) / dmax(rl * al2, rr * ar2);
  const double alpha_c = dmax(dmax(aa, ab), dmin(1.0, dp * 1.0 - 0.5));
  const double alpha = alpha_c;
  const double amin = sqrt(dmin(al2, ar2));
#pragma unroll
  for (int i = 0; i < 5; ++i) F[i] = 0.0;
  if (alpha > 1e-10) {
    const double utmax = dmax(fabs(L.u * nx + L.v * ny + L.w * nz), fabs(R.u * nx + R.v * ny + R.w * nz));
    const double Ma = dmax(alpha_c, dmin(1.0, utmax / amin + 1e-4));
    const double h = 0.5 * (1. - Ma);
    Q5 Lp = L, Rp = R;
    Lp.u = L.u + h * (R.u - L.u), Lp.v = L.v + h * (R.v - L.v), Lp.w = L.w + h * (R.w - L.w);
    Rp.u = R.u + h * (L.u - R.u), Rp.v = R.v + h * (L.v - R.v), Rp.w = R.w + h * (L.w - R.w);
    flux_hllc(Lp, Rp, nx, ny, nz, A * alpha, g, 0.0, 1.0, F);
  }
  auto dot3 = [](const double* gr, double x, double y, double z) { return gr[0] * x + gr[1] * y + gr[2] * z; };
  auto at = [&](const Q5& c, const double* gr, Q5& o) {
    const double* ph = gr + 15;
    o.p = dmax(c.p + ph[4] * dot3(gr + 12, dvx, dvy, dvz), pglim);
    o.T = dmax(c.T + ph[0] * dot3(gr, dvx, dvy, dvz), tlim);
    o.u = c.u + ph[1] * dot3(gr + 3, dvx, dvy, dvz);
    o.v = c.v + ph[2] * dot3(gr + 6, dvx, dvy, dvz);
    o.w = c.w + ph[3] * dot3(gr + 9, dvx, dvy, dvz);
  };
  Q5 l, r, ll, rx;
  at(qa, ga, l);
  at(qb, gb, r);
  // ll from r with the left cell's gradient, rr from l with the right one's
  ll.p = dmax(r.p - 2. * dot3(ga + 12, d2x, d2y, d2z), pglim);
  rx.p = dmax(l.p + 2. * dot3(gb + 12, d2x, d2y, d2z), pglim);
  ll.T = dmax(r.T - 2. * dot3(ga, d2x, d2y, d2z), tlim);
  rx.T = dmax(l.T + 2. * dot3(gb, d2x, d2y, d2z), tlim);
  ll.u = r.u - 2. * dot3(ga + 3, d2x, d2y, d2z);
  ll.v = r.v - 2. * dot3(ga + 6, d2x, d2y, d2z);
  ll.w = r.w - 2. * dot3(ga + 9, d2x, d2y, d2z);
  rx.u = l.u + 2. * dot3(gb + 3, d2x, d2y, d2z);
  rx.v = l.v + 2. * dot3(gb + 6, d2x, d2y, d2z);
  rx.w = l.w + 2. * dot3(gb + 9, d2x, d2y, d2z);
  const double CC = coeff / 6.0;
  const double sada = A * (1. - alpha);
  kec_flux_add(l, r, nx, ny, nz, (1. + 2. * CC) * sada, g, F);
  kec_flux_add(l, rx, nx, ny, nz, -CC * sada, g, F);
  kec_flux_add(ll, r, nx, ny, nz, -CC * sada, g, F);
  // cubic extrapolation to the face
  const double a0 = 1. / 3., a1 = 5. / 6., a2 = -1. / 6.;
  Q5 lq, rq;
  lq.p = dmax(pglim, a0 * r.p + a1 * l.p + a2 * ll.p);
  rq.p = dmax(pglim, a0 * l.p + a1 * r.p + a2 * rx.p);
  lq.T = dmax(tlim, a0 * r.T + a1 * l.T + a2 * ll.T);
  rq.T = dmax(tlim, a0 * l.T + a1 * r.T + a2 * rx.T);
  lq.u = a0 * r.u + a1 * l.u + a2 * ll.u, lq.v = a0 * r.v + a1 * l.v + a2 * ll.v,
  lq.w = a0 * r.w + a1 * l.w + a2 * ll.w;
  rq.u = a0 * l.u + a1 * r.u + a2 * rx.u, rq.v = a0 * l.v + a1 * r.v + a2 * rx.v,
  rq.w = a0 * l.w + a1 * r.w + a2 * rx.w;
  const double cf = dmax(ag, filter) * sada;
  const double utmax = dmax(fabs(lq.u * nx + lq.v * ny + lq.w * nz), fabs(rq.u * nx + rq.v * ny + rq.w * nz));
  const double Ma = dmin(1.0, utmax / amin + 1e-4);
  const double h = 0.5 * (1. - Ma);
  Q5 lp = lq, rp = rq;
  lp.u = lq.u + h * (rq.u - lq.u), lp.v = lq.v + h * (rq.v - lq.v), lp.w = lq.w + h * (rq.w - lq.w);
  rp.u = rq.u + h * (lq.u - rq.u), rp.v = rq.v + h * (lq.v - rq.v), rp.w = rq.w + h * (lq.w - rq.w);
  roe_dissipation_sub(lp, rp, nx, ny, nz, cf, g, F);
}

// ---- boundary states from total conditions or a mass flux ---------------
// Each returns the face state (T, u, v, w, pg) from the cell-centre state qi
// of the face's cell; n is the outward unit normal, the flow direction of
// the inflows is -n, the grid does not move.

// The analytic flux of one state through a face (inviscidFlux,
// inviscidFlux.h:25-45): momentum with the gauge pressure, energy with the
// absolute one.
__device__ __forceinline__ void state_flux(const Q5& q, double nx, double ny, double nz,
                                           double area, const Gas& g, double F[5]) {
  const double gm1 = g.gamma - 1.0;
  const double rho = (q.p + g.pamb) / (g.Rt * q.T);
  const double h0 = g.Rt * q.T * g.gamma / gm1 + 0.5 * (q.u * q.u + q.v * q.v + q.w * q.w);
  const double e0 = h0 - g.Rt * q.T;
  const double ut = q.u * nx + q.v * ny + q.w * nz;
  const double m = area * rho * ut;
  F[0] = m;
  F[1] = m * q.u + area * q.p * nx;
  F[2] = m * q.v + area * q.p * ny;
  F[3] = m * q.w + area * q.p * nz;
  F[4] = m * e0 + area * (q.p + g.pamb) * ut;
}

// Isentropic inflow at total pressure p0 (absolute) and temperature T0
// (bcIsentropic.loci:52-160): the boundary sound speed from the outgoing
// Riemann invariant, the Mach number capped at 1, isentropic relations, and a
// blend towards the inside sound speed when the boundary would be much
// hotter than the inside.
__device__ __forceinline__ void isentropic_state(const Q5& qi, double nx, double ny, double nz,
                                                 double p0, double T0, const Gas& g, Q5& qb) {
  const double gm1 = g.gamma - 1.0;
  const double a0 = sqrt(g.gamma * g.Rt * T0);
  const double ai = sqrt(g.gamma * g.Rt * qi.T);
  const double dx = -nx, dy = -ny, dz = -nz;  // flow direction
  const double uit = qi.u * dx + qi.v * dy + qi.w * dz;
  // boundary sound speed ab and normal velocity unb: the root of a quadratic
  const double rim = uit - 2.0 * ai / gm1;
  const double qa = 2.0 / gm1 + 1.0, qb2 = 2.0 * rim, qc = 0.5 * gm1 * rim * rim - a0 * a0;
  const double D = qb2 * qb2 - 4.0 * qa * qc;
  double ab, unb;
  if (D < 0) {
    ab = a0;
  } else {
    ab = (-qb2 + sqrt(D)) / (2.0 * qa);
    ab = dmax(ab, 0.25 * a0);
  }
  unb = rim + 2.0 * ab / gm1;
  auto finish = [&](double ab_, double unb_, double& Tb, double& pb, double& un_out) {
    double M = fabs(unb_) / ab_;
    un_out = unb_;
    if (M > 1.0) {  // choked: Mach 1 from the total conditions
      M = 1.0;
      const double utot = M * a0 / sqrt(1.0 + 0.5 * gm1 * M * M);
      un_out = sqrt(dmax(utot * utot, 0.0));
    }
    const double fm = 1.0 + 0.5 * gm1 * M * M;
    Tb = T0 / fm;
    pb = p0 * pow(fm, -g.gamma / gm1);
  };
  double Tb, pb, un;
  finish(ab, unb, Tb, pb, un);
  double f = (Tb - qi.T) / dmax(qi.T, Tb) - 0.1;
  if (f > 0) {
    f = sqrt(f);
    ab = (1.0 - f) * ab + f * a0;
    unb = (1.0 - f) * unb + f * uit;
    finish(ab, unb, Tb, pb, un);
  }
  qb.u = un * dx, qb.v = un * dy, qb.w = un * dz;
  qb.T = Tb;
  qb.p = pb - g.pamb;
}

// Fixed mass-flux inflow at total temperature T0 (bcFixedMass.loci:84-135):
// the boundary temperature by fixed-point iteration (at most 1000 steps, to
// 1e-9 of the inside temperature) at the inside pressure.  Returns false
// when the iteration did not converge.
__device__ __forceinline__ bool fixed_mass_state(const Q5& qi, double nx, double ny, double nz,
                                                 double mflux, double T0, const Gas& g, Q5& qb) {
  const double pin = qi.p + g.pamb;
  const double gp1 = g.gamma + 1.0, gm1 = g.gamma - 1.0;
  double T = qi.T;
  const double eps = qi.T * 1e-9;
  bool ok = false;
  for (int it = 0; it < 1000; ++it) {
    const double rho = pin / (g.Rt * T);
    const double a = sqrt(g.gamma * g.Rt * T);
    const double M = (mflux / rho) / a;
    const double lam = sqrt((gp1 * M * M) / (gm1 * M * M + 2.0));
    const double base = 1.0 - (gm1 / gp1) * lam * lam;
    const double p0 = pin * pow(base, -g.gamma / gm1);
    const double rho0 = p0 / (g.Rt * T0);
    const double rho1 = rho0 * pow(base, 1.0 / gm1);
    const double T1 = pin / (rho1 * g.Rt);
    if (fabs(T1 - T) < eps) {
      ok = true;
      break;
    }
    T = T1;
  }
  const double vel = mflux / (pin / (g.Rt * T));
  // u = d (-vel / (d . n)) with the flow direction d = -n: -vel n
  qb.u = -vel * nx, qb.v = -vel * ny, qb.w = -vel * nz;
  qb.T = T;
  qb.p = qi.p;
  return ok;
}

// Fixed mass-flux outflow (bcFixedMassOutflow.loci:86-132): the target
// mass flux (1 - relax) rho_i u_i.n + relax mflux, bounded by the choked
// flux, reached by the normal velocity at the inside total conditions.
__device__ __forceinline__ void fixed_mass_outflow_state(const Q5& qi, double nx, double ny,
                                                         double nz, double mflux, double relax,
                                                         const Gas& g, Q5& qb) {
  const double gm1 = g.gamma - 1.0, gp1 = g.gamma + 1.0;
  const double pin = qi.p + g.pamb;
  const double rhoin = pin / (g.Rt * qi.T);
  const double cin = sqrt(g.gamma * g.Rt * qi.T);
  const double uin_n = qi.u * nx + qi.v * ny + qi.w * nz;
  const double target = (1.0 - relax) * rhoin * uin_n + relax * mflux;
  const double M2 = (qi.u * qi.u + qi.v * qi.v + qi.w * qi.w) / (cin * cin);
  double fm = 1.0 + 0.5 * gm1 * M2;
  const double p0 = pin * pow(fm, g.gamma / gm1);
  const double T0 = qi.T * fm;
  const double rho0 = rhoin * pow(fm, 1.0 / gm1);
  const double rhos = rho0 * pow(2.0 / gp1, 1.0 / gm1);
  double cstar = cin * sqrt(2.0 * fm / gp1);
  double u = dmin(target, rhos * cstar) / rhoin;
  fm = 1.0 + 0.5 * gm1 * (u / cin) * (u / cin);
  cstar = cin * sqrt(2.0 * fm / gp1);
  u = dmin(u, cstar);
  const double lam = u / cstar;
  const double fl = 1.0 - (gm1 / gp1) * lam * lam;
  const double p = p0 * pow(fl, g.gamma / gm1);
  if (u < cin) {
    const double du = u - uin_n;
    qb.u = qi.u + du * nx, qb.v = qi.v + du * ny, qb.w = qi.w + du * nz;
    qb.T = T0 * fl;
    qb.p = p - g.pamb;
  } else {
    qb = qi;
  }
}

// Characteristic boundary states, cv_inflow / cv_outflow (bcTools.h:25-81).// Characteristic boundary states, cv_inflow / cv_outflow (bcTools.h:25-81).
__device__ __forceinline__ void cv_state(bool outflow, const Q5& qi, const Q5& q0, double nx,
                                         double ny, double nz, double us_n, const Gas& g,
                                         double beta, Q5& qb) {
  const double uit = qi.u * nx + qi.v * ny + qi.w * nz - us_n;
  const double u0t = q0.u * nx + q0.v * ny + q0.w * nz - us_n;
  const double a02 = g.gamma * g.Rt * q0.T;
  const double r0 = (q0.p + g.pamb) / (g.Rt * q0.T);
  const double bm = 0.5 * (1.0 - beta);
  const double ub = uit * (1.0 - beta);
  const double sg = sqrt(ub * ub + 4.0 * beta * a02);
  const double rel = ((qi.p - q0.p) + r0 * (uit - u0t) * uit * bm) * uit * bm / (2.0 * sg);
  double pb;
  if (outflow) {
    pb = 0.5 * (qi.p + q0.p - 0.5 * r0 * sg * (u0t - uit)) + rel;
    pb = dmax(pb, 0.1 * (qi.p + g.pamb) - g.pamb);
    const double s = 2.0 * (qi.p - pb) / (r0 * (sg + uit * bm));
    qb.u = qi.u + s * nx;
    qb.v = qi.v + s * ny;
    qb.w = qi.w + s * nz;
    const double rb = r0 + (pb - qi.p) * (sg - uit * bm) / (beta * a02 * (sg + uit * bm));
    qb.T = (pb + g.pamb) / (g.Rt * rb);
  } else {
    pb = 0.5 * (q0.p + qi.p - 0.5 * r0 * sg * (u0t - uit)) - rel;
    pb = dmax(pb, 0.1 * (q0.p + g.pamb) - g.pamb);
    const double s = 2.0 * (pb - q0.p) / (r0 * (sg + uit * bm));
    qb.u = q0.u + s * nx;
    qb.v = q0.v + s * ny;
    qb.w = q0.w + s * nz;
    const double rb = r0 + (pb - q0.p) * (sg - uit * bm) / (beta * a02 * (sg + uit * bm));
    qb.T = (pb + g.pamb) / (g.Rt * rb);
  }
  qb.p = pb;
}

}  // namespace dev
}  // namespace fpsi
