// oracle.cpp -- CPU restatement of flowPsi's steady implicit hot path.
//
// TEST INFRASTRUCTURE ONLY (the checker): called by tests/, the smoke check
// and the CPU-baseline leg of bench.py; never linked by the product library.
//
// Scalar C++ that follows the reference rule by rule, in the reference's own
// evaluation order where the order changes rounding (face-order scatter,
// upper-then-lower accumulation, FP32 stores for real_fj blocks).
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct V3 {
  double x, y, z;
};
inline V3 mk(double x, double y, double z) { return V3{x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator*(double s, V3 a) { return mk(s * a.x, s * a.y, s * a.z); }
inline V3 operator*(V3 a, double s) { return mk(s * a.x, s * a.y, s * a.z); }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline double norm(V3 a) { return std::sqrt(dot(a, a)); }

// ---------------------------------------------------------------------------
// Face physics
// ---------------------------------------------------------------------------

// inviscidFlux, inviscidFlux.h:25-45: analytic flux of one state.
void analytic_flux(double f[5], double pg, double T, V3 U, V3 an, double area,
                   double pamb, double Rt, double gamma, double Us_n) {
  double gm1 = gamma - 1;
  double rho = (pg + pamb) / (Rt * T);
  double h0 = Rt * T * gamma / gm1 + 0.5 * dot(U, U);
  double e0 = h0 - Rt * T;
  double uta = dot(U, an);
  double ut = uta - Us_n;
  double mdot = area * rho * ut;
  double p = pg + pamb;
  f[0] = mdot;
  f[1] = mdot * U.x + area * pg * an.x;
  f[2] = mdot * U.y + area * pg * an.y;
  f[3] = mdot * U.z + area * pg * an.z;
  f[4] = mdot * e0 + area * p * uta;
}

// hllc_flux, fluxInviscid.loci:157-256.
void hllc_flux(double F[5], double pgl, double Tl, V3 Ul, double pgr, double Tr, V3 Ur,
               V3 an, double area, double pamb, double Rt, double gamma, double Us_n,
               double Eta) {
  double gm1 = gamma - 1;
  double rl = (pgl + pamb) / (Rt * Tl);
  double rr = (pgr + pamb) / (Rt * Tr);
  double h0l = Rt * Tl * gamma / gm1 + 0.5 * dot(Ul, Ul);
  double h0r = Rt * Tr * gamma / gm1 + 0.5 * dot(Ur, Ur);
  double e0l = h0l - Rt * Tl;
  double e0r = h0r - Rt * Tr;
  double srl = std::sqrt(rl), srr = std::sqrt(rr);
  double rf = 1. / (srl + srr);
  V3 U_ = (Ul * srl + Ur * srr) * rf;
  double ut_ = dot(U_, an) - Us_n;
  double h0_ = (h0l * srl + h0r * srr) * rf;
  double a_ = std::sqrt(std::max(gm1 * (h0_ - 0.5 * dot(U_, U_)), 0.0));
  double EtaP = Eta + 1., EtaM = Eta - 1.;
  double sigma = std::sqrt(std::max(ut_ * ut_ * EtaM * EtaM + 4. * Eta * a_ * a_, 1e-30));
  double evl_ = 0.5 * (ut_ * EtaP - sigma);
  double evr_ = 0.5 * (ut_ * EtaP + sigma);
  double utla = dot(Ul, an), utra = dot(Ur, an);
  double utl = utla - Us_n, utr = utra - Us_n;
  double al2 = gamma * Rt * Tl, ar2 = gamma * Rt * Tr;
  double sigmar = std::sqrt(std::max(utr * utr * EtaM * EtaM + 4. * Eta * ar2, 0.0));
  double sigmal = std::sqrt(std::max(utl * utl * EtaM * EtaM + 4. * Eta * al2, 0.0));
  double SL = std::min(evl_, .5 * (utl * EtaP - sigmal));
  double SR = std::max(evr_, .5 * (utr * EtaP + sigmar));
  double lmdot = rl * utl, rmdot = rr * utr;
  double pl = pgl + pamb, pr = pgr + pamb;
  double coef = 0.5 * area;
  double AL = coef * ((SL > 0) ? (SR < 0 ? 1. : 2.) : (SR < 0 ? 0. : 1.));
  double AR = coef * ((SR < 0) ? (SL > 0 ? 1. : 2.) : (SL > 0 ? 0. : 1.));
  double AM = coef * ((SL > 0 || SR < 0) ? 0. : 1.);
  F[0] = AL * lmdot + AR * rmdot;
  F[1] = AL * lmdot * Ul.x + AR * rmdot * Ur.x + an.x * (AL * pgl + AR * pgr);
  F[2] = AL * lmdot * Ul.y + AR * rmdot * Ur.y + an.y * (AL * pgl + AR * pgr);
  F[3] = AL * lmdot * Ul.z + AR * rmdot * Ur.z + an.z * (AL * pgl + AR * pgr);
  F[4] = AL * (lmdot * e0l + pl * utla) + AR * (rmdot * e0r + pr * utra);
  F[0] -= AM * (SL * rl + SR * rr);
  F[1] -= AM * (SL * rl * Ul.x + SR * rr * Ur.x);
  F[2] -= AM * (SL * rl * Ul.y + SR * rr * Ur.y);
  F[3] -= AM * (SL * rl * Ul.z + SR * rr * Ur.z);
  F[4] -= AM * (SL * rl * e0l + SR * rr * e0r);
  double SM = ((rr * utr * (SR - utr) - rl * utl * (SL - utl) + pgl - pgr) /
               (rr * (SR - utr) - rl * (SL - utl)));
  double rl_s = rl * (SL - utl) / (SL - SM);
  double rr_s = rr * (SR - utr) / (SR - SM);
  double pg_s = rl * (utl - SL) * (utl - SM) + pgl;
  double p_s = pg_s + pamb;
  double rul = ((SL - utl) * rl * Ul.x + (pg_s - pgl) * an.x) / (SL - SM);
  double rvl = ((SL - utl) * rl * Ul.y + (pg_s - pgl) * an.y) / (SL - SM);
  double rwl = ((SL - utl) * rl * Ul.z + (pg_s - pgl) * an.z) / (SL - SM);
  double rur = ((SR - utr) * rr * Ur.x + (pg_s - pgr) * an.x) / (SR - SM);
  double rvr = ((SR - utr) * rr * Ur.y + (pg_s - pgr) * an.y) / (SR - SM);
  double rwr = ((SR - utr) * rr * Ur.z + (pg_s - pgr) * an.z) / (SR - SM);
  double rel = ((SL - utl) * rl * e0l - pl * utl + p_s * SM) / (SL - SM);
  double rer = ((SR - utr) * rr * e0r - pr * utr + p_s * SM) / (SR - SM);
  double CR = SR - std::fabs(SM), CL = SL + std::fabs(SM);
  F[0] += AM * (CR * rr_s + CL * rl_s);
  F[1] += AM * (CR * rur + CL * rul);
  F[2] += AM * (CR * rvr + CL * rvl);
  F[3] += AM * (CR * rwr + CL * rwl);
  F[4] += AM * (CR * rer + CL * rel);
}

// HLLE: no counterpart in the reference.  Two-wave HLL flux whose wave
// speeds are hllc_flux's SL/SR (fluxInviscid.loci:173-204).
void hlle_flux(double F[5], double pgl, double Tl, V3 Ul, double pgr, double Tr, V3 Ur,
               V3 an, double area, double pamb, double Rt, double gamma, double Us_n,
               double Eta) {
  double gm1 = gamma - 1;
  double rl = (pgl + pamb) / (Rt * Tl);
  double rr = (pgr + pamb) / (Rt * Tr);
  double h0l = Rt * Tl * gamma / gm1 + 0.5 * dot(Ul, Ul);
  double h0r = Rt * Tr * gamma / gm1 + 0.5 * dot(Ur, Ur);
  double srl = std::sqrt(rl), srr = std::sqrt(rr);
  double rf = 1. / (srl + srr);
  V3 U_ = (Ul * srl + Ur * srr) * rf;
  double ut_ = dot(U_, an) - Us_n;
  double h0_ = (h0l * srl + h0r * srr) * rf;
  double a_ = std::sqrt(std::max(gm1 * (h0_ - 0.5 * dot(U_, U_)), 0.0));
  double EtaP = Eta + 1., EtaM = Eta - 1.;
  double sigma = std::sqrt(std::max(ut_ * ut_ * EtaM * EtaM + 4. * Eta * a_ * a_, 1e-30));
  double utl = dot(Ul, an) - Us_n, utr = dot(Ur, an) - Us_n;
  double al2 = gamma * Rt * Tl, ar2 = gamma * Rt * Tr;
  double sigmar = std::sqrt(std::max(utr * utr * EtaM * EtaM + 4. * Eta * ar2, 0.0));
  double sigmal = std::sqrt(std::max(utl * utl * EtaM * EtaM + 4. * Eta * al2, 0.0));
  double SL = std::min(0.5 * (ut_ * EtaP - sigma), .5 * (utl * EtaP - sigmal));
  double SR = std::max(0.5 * (ut_ * EtaP + sigma), .5 * (utr * EtaP + sigmar));
  double fl[5], fr[5];
  analytic_flux(fl, pgl, Tl, Ul, an, area, pamb, Rt, gamma, Us_n);
  analytic_flux(fr, pgr, Tr, Ur, an, area, pamb, Rt, gamma, Us_n);
  if (SL >= 0) {
    for (int i = 0; i < 5; ++i) F[i] = fl[i];
    return;
  }
  if (SR <= 0) {
    for (int i = 0; i < 5; ++i) F[i] = fr[i];
    return;
  }
  double e0l = h0l - Rt * Tl, e0r = h0r - Rt * Tr;
  double ql[5] = {rl, rl * Ul.x, rl * Ul.y, rl * Ul.z, rl * e0l};
  double qr[5] = {rr, rr * Ur.x, rr * Ur.y, rr * Ur.z, rr * e0r};
  double rd = 1. / (SR - SL);
  for (int i = 0; i < 5; ++i)
    F[i] = (SR * fl[i] - SL * fr[i] + area * SL * SR * (qr[i] - ql[i])) * rd;
}

// The 5x5 matrix of the preconditioned Roe scheme, RoeJacobian in
// fluxInviscid.loci:1019-1090.  roeCT_flux (:869-1014) applies the same
// coefficients, with |eigenvalues|, to the primitive jumps.
struct RoeCoef {
  double ev1, rT, T7, T8, T9, T10, T11, T4s, rho, T1s;
};
RoeCoef roe_coef(double ev1, double ev2, double ev3, V3 U, double un, double a,
                 double beta, double sigma, double gamma, double Rt, double rho, double h0,
                 V3 n) {
  const double BM = beta - 1.;
  const double una = dot(U, n);
  const double T1 = ev2 - ev3;
  const double T2 = (ev2 + ev3 - 2 * ev1);
  const double T3 = rho * (BM * BM * un * un - sigma * sigma) / (4. * sigma);
  const double T4 = T2 * sigma + BM * T1 * un;
  const double T5 = (T2 * sigma - BM * T1 * un) / (2. * sigma);
  const double T6 = ((ev2 + ev3) * sigma - BM * T1 * un) / (2. * sigma);
  const double gm1 = gamma - 1.0;
  const double Cp = gamma * Rt / gm1;
  const double rT = -gamma * Rt * rho / ((h0 - 0.5 * dot(U, U)) * gm1);
  const double rbeta = 1. / beta;
  const double ra2 = 1. / (a * a);
  const double T7 = rbeta * T1 * T3 * ra2;
  const double T8 = (((rbeta - 1) + gamma) * T6 - gm1 * T5) * ra2;
  const double T9 = Cp * rho + h0 * rT;
  const double x1 = gamma * h0 * T1 * T3 * ra2 * rbeta;
  const double x2 = -rbeta * gm1 * T1 * T3 * T9 * ra2 / rT;
  const double x3 = -T1 * T3 * rbeta;
  const double x4 = .5 * rho * T4 * una / sigma;
  const double T10 = (x1 + x2 + x3 + x4);
  const double T11 = (rbeta * ra2 * h0 + (T9 - rho * rbeta * Cp) * ra2 * gm1 / rT - rbeta) * T6 -
                     gm1 * ra2 * T9 * T5 / rT - una * T1 / sigma;
  RoeCoef c;
  c.ev1 = ev1;
  c.rT = rT;
  c.T7 = T7;
  c.T8 = T8;
  c.T9 = T9;
  c.T10 = T10;
  c.T11 = T11;
  c.T4s = rho * T4 / (2. * sigma);
  c.rho = rho;
  c.T1s = T1 / sigma;
  return c;
}

// RoeJacobian (fluxInviscid.loci:1019-1090): Fj += area*K, accumulated in TB.
template <class TB>
void roe_matrix_accum(TB Fj[25], const RoeCoef& c, V3 U, V3 n, double area) {
  const int Ti = 0, Pi = 4, mi = 1, ei = 4;
  double u[3] = {U.x, U.y, U.z}, nn[3] = {n.x, n.y, n.z};
#define FJ(i, j) Fj[(i)*5 + (j)]
  FJ(0, Ti) += area * c.ev1 * c.rT;
  for (int k = 0; k < 3; ++k) FJ(0, mi + k) += area * nn[k] * c.T7;
  FJ(0, Pi) += area * c.T8;
  for (int k = 0; k < 3; ++k) FJ(mi + k, Ti) += area * c.ev1 * c.rT * u[k];
  for (int r = 0; r < 3; ++r)
    for (int k = 0; k < 3; ++k) {
      double v = nn[k] * (c.T7 * u[r] + nn[r] * c.T4s);
      if (r == k) v += c.ev1 * c.rho;
      FJ(mi + r, mi + k) += area * v;
    }
  for (int r = 0; r < 3; ++r) FJ(mi + r, Pi) += area * (c.T8 * u[r] - nn[r] * c.T1s);
  FJ(ei, Ti) += area * c.ev1 * c.T9;
  for (int k = 0; k < 3; ++k) FJ(ei, mi + k) += area * (nn[k] * c.T10 + c.ev1 * c.rho * u[k]);
  FJ(ei, Pi) += area * c.T11;
#undef FJ
}

struct RoeState {
  double rl, rr, re0l, re0r, pl, pr, r_, srl, srr, h0_, h_, ut_, uta_, a_, sigma, Eta;
  V3 U_;
};
// Roe averages shared by roeCT_flux (:875-915) and roeCT_jacobian (:1098-1139).
RoeState roe_state(double pgl, double Tl, V3 Ul, double pgr, double Tr, V3 Ur, V3 an,
                   double pamb, double Rt, double gamma, double Us_n, double Eta) {
  RoeState s;
  double gm1 = gamma - 1.;
  s.pl = pgl + pamb;
  s.pr = pgr + pamb;
  s.rl = s.pl / (Rt * Tl);
  s.rr = s.pr / (Rt * Tr);
  s.re0l = s.rl * (Rt * Tl / gm1 + 0.5 * dot(Ul, Ul));
  s.re0r = s.rr * (Rt * Tr / gm1 + 0.5 * dot(Ur, Ur));
  double h0l = (s.re0l + s.pl) / s.rl;
  double h0r = (s.re0r + s.pr) / s.rr;
  s.r_ = std::sqrt(s.rl * s.rr);
  s.srl = std::sqrt(s.rl);
  s.srr = std::sqrt(s.rr);
  double rf = 1. / (s.srl + s.srr);
  s.U_ = (Ul * s.srl + Ur * s.srr) * rf;
  s.ut_ = dot(s.U_, an) - Us_n;
  s.uta_ = dot(s.U_, an);
  double q2_ = dot(s.U_, s.U_);
  s.h0_ = (h0l * s.srl + h0r * s.srr) * rf;
  s.h_ = s.h0_ - 0.5 * q2_;
  if (std::fabs(s.pl - s.pr) / (s.pl + s.pr + 1e-33) > .1) Eta = 1.;
  s.Eta = Eta;
  double af2 = std::max(gm1 * s.h_, 1e-30);
  s.a_ = std::sqrt(af2);
  double EtaM = Eta - 1.;
  s.sigma = std::sqrt(s.ut_ * s.ut_ * EtaM * EtaM + 4. * Eta * s.a_ * s.a_);
  return s;
}

// roeCT_flux, fluxInviscid.loci:869-1014 (with the Harten-Hyman fix :940-962).
void roe_flux(double F[5], double pgl, double Tl, V3 Ul, double pgr, double Tr, V3 Ur, V3 an,
              double area, double pamb, double Rt, double gamma, double Us_n, double Eta) {
  RoeState s = roe_state(pgl, Tl, Ul, pgr, Tr, Ur, an, pamb, Rt, gamma, Us_n, Eta);
  Eta = s.Eta;
  const double EtaP = Eta + 1., EtaM = Eta - 1.;
  const double ut_ = s.ut_, sigma = s.sigma;
  double ev1 = std::fabs(ut_);
  double ev2 = std::fabs(ut_ * EtaP - sigma) / 2.;
  double ev3 = std::fabs(ut_ * EtaP + sigma) / 2.;
  const double al2 = gamma * Rt * Tl, ar2 = gamma * Rt * Tr;
  const double utla = dot(Ul, an), utra = dot(Ur, an);
  const double utl = utla - Us_n, utr = utra - Us_n;
  double sigmal = std::sqrt(utl * utl * EtaM * EtaM + 4. * Eta * al2);
  double sigmar = std::sqrt(utr * utr * EtaM * EtaM + 4. * Eta * ar2);
  const double e2l = (utl * EtaP - sigmal) / 2., e2r = (utr * EtaP - sigmar) / 2.;
  const double e3l = (utl * EtaP + sigmal) / 2., e3r = (utr * EtaP + sigmar) / 2.;
  const double ev2s = (ut_ * EtaP - sigma) / 2., ev3s = (ut_ * EtaP + sigma) / 2.;
  const double eps2 = std::max(0.0, std::max(ev2s - e2l, e2r - ev2s));
  const double eps3 = std::max(0.0, std::max(ev3s - e3l, e3r - ev3s));
  ev2 = ev2 < eps2 ? 0.5 * ((ev2s * ev2s) / eps2 + eps2) : ev2;
  ev3 = ev3 < eps3 ? 0.5 * ((ev3s * ev3s) / eps3 + eps3) : ev3;
  // dissipation, written with the association of :985-1004
  const V3 U_ = s.U_;
  const double r_ = s.r_, h0_ = s.h0_, uta_ = s.uta_;
  const V3 Uj = Ur - Ul;
  const double utj = dot(Uj, an);
  const double pj = pgr - pgl, Tj = Tr - Tl;
  const double BM = EtaM;
  const double T1 = ev2 - ev3;
  const double T2 = (ev2 + ev3 - 2 * ev1);
  const double T3 = r_ * (BM * BM * ut_ * ut_ - sigma * sigma) / (4. * sigma);
  const double T4 = T2 * sigma + BM * T1 * ut_;
  const double T5 = (T2 * sigma - BM * T1 * ut_) / (2. * sigma);
  const double T6 = ((ev2 + ev3) * sigma - BM * T1 * ut_) / (2. * sigma);
  const double gm1 = gamma - 1.;
  const double Cp = gamma * Rt / gm1;
  const double rT_ = -gamma * Rt * r_ / (s.h_ * gm1);
  const double rbeta = 1. / Eta;
  const double ra2 = 1. / (s.a_ * s.a_);
  const double T7 = rbeta * T1 * T3 * ra2;
  const double T8 = (((rbeta - 1) + gamma) * T6 - gm1 * T5) * ra2;
  const double T9 = Cp * r_ + h0_ * rT_;
  const double x1 = gamma * h0_ * T1 * T3 * ra2 * rbeta;
  const double x2 = -rbeta * gm1 * T1 * T3 * T9 * ra2 / rT_;
  const double x3 = -T1 * T3 * rbeta;
  const double x4 = .5 * r_ * T4 * uta_ / sigma;
  const double T10 = (x1 + x2 + x3 + x4);
  const double T11 = (rbeta * ra2 * h0_ + (T9 - r_ * rbeta * Cp) * ra2 * gm1 / rT_ - rbeta) * T6 -
                     gm1 * ra2 * T9 * T5 / rT_ - uta_ * T1 / sigma;
  double d[5];
  d[0] = pj * T8 + utj * T7 + ev1 * Tj * rT_;
  d[1] = U_.x * T7 * utj + ev1 * (U_.x * Tj * rT_ + r_ * Uj.x) + pj * (T8 * U_.x - an.x * T1 / sigma) +
         an.x * r_ * T4 * utj / (2. * sigma);
  d[2] = U_.y * T7 * utj + ev1 * (U_.y * Tj * rT_ + r_ * Uj.y) + pj * (T8 * U_.y - an.y * T1 / sigma) +
         an.y * r_ * T4 * utj / (2. * sigma);
  d[3] = U_.z * T7 * utj + ev1 * (U_.z * Tj * rT_ + r_ * Uj.z) + pj * (T8 * U_.z - an.z * T1 / sigma) +
         an.z * r_ * T4 * utj / (2. * sigma);
  d[4] = pj * T11 + T10 * utj + ev1 * (T9 * Tj + r_ * dot(U_, Uj));
  const double Ah = 0.5 * area;
  F[0] = Ah * (s.rl * utl + s.rr * utr - d[0]);
  F[1] = Ah * (Ul.x * s.rl * utl + Ur.x * s.rr * utr + an.x * (pgl + pgr) - d[1]);
  F[2] = Ah * (Ul.y * s.rl * utl + Ur.y * s.rr * utr + an.y * (pgl + pgr) - d[2]);
  F[3] = Ah * (Ul.z * s.rl * utl + Ur.z * s.rr * utr + an.z * (pgl + pgr) - d[3]);
  F[4] = Ah * ((s.re0l * utl + s.pl * utla) + (s.re0r * utr + s.pr * utra) - d[4]);
}

// roeCT_jacobian, fluxInviscid.loci:1092-1168 (eigenvalue smoothing :1141-1164).
template <class TB>
void roe_jacobian(TB Fj[25], double pgl, double Tl, V3 Ul, double pgr, double Tr, V3 Ur,
                  V3 an, double area, double pamb, double Rt, double gamma, double Us_n,
                  double Eta, int dir) {
  RoeState s = roe_state(pgl, Tl, Ul, pgr, Tr, Ur, an, pamb, Rt, gamma, Us_n, Eta);
  Eta = s.Eta;
  const double EtaP = Eta + 1.;
  double ev1 = s.ut_;
  double ev2 = (s.ut_ * EtaP - s.sigma) / 2.;
  double ev3 = (s.ut_ * EtaP + s.sigma) / 2.;
  double d = (dir < 0) ? -1 : 1;
  const double mxv = std::max(ev1, std::max(ev2, ev3));
  const double mnv = std::min(ev1, std::min(ev2, ev3));
  const double eps = 0.02 * (mxv - mnv);
  const double eps2 = eps * eps;
  ev1 = .5 * (ev1 + d * std::sqrt(ev1 * ev1 + eps2));
  ev2 = .5 * (ev2 + d * std::sqrt(ev2 * ev2 + eps2));
  ev3 = .5 * (ev3 + d * std::sqrt(ev3 * ev3 + eps2));
  RoeCoef c = roe_coef(ev1, ev2, ev3, s.U_, s.ut_, s.a_, Eta, s.sigma, gamma, Rt, s.r_, s.h0_, an);
  roe_matrix_accum<TB>(Fj, c, s.U_, an, area);
}

void riemann_flux(int kind, double F[5], double pgl, double Tl, V3 Ul, double pgr, double Tr,
                  V3 Ur, V3 an, double area, double pamb, double Rt, double gamma, double Us_n,
                  double Eta) {
  if (kind == FPSI_FLUX_ROE)
    roe_flux(F, pgl, Tl, Ul, pgr, Tr, Ur, an, area, pamb, Rt, gamma, Us_n, Eta);
  else if (kind == FPSI_FLUX_HLLE)
    hlle_flux(F, pgl, Tl, Ul, pgr, Tr, Ur, an, area, pamb, Rt, gamma, Us_n, Eta);
  else
    hllc_flux(F, pgl, Tl, Ul, pgr, Tr, Ur, an, area, pamb, Rt, gamma, Us_n, Eta);
}

// cv_inflow / cv_outflow, bcTools.h:25-81.
void cv_inflow(double& pgb, double& Tb, V3& ub, double pgi, double Ti, V3 ui, double pg0,
               double T0, V3 u0, V3 n, double us_n, double pamb, double gamma, double Rt,
               double Beta) {
  (void)Ti;
  const double uit = dot(ui, n) - us_n, u0t = dot(u0, n) - us_n;
  const double a0 = std::sqrt(gamma * Rt * T0);
  const double r0 = (pg0 + pamb) / (Rt * T0);
  const double MinP = 0.1 * (pg0 + pamb) - pamb;
  const double BetaM = 0.5 * (1.0 - Beta);
  const double uitBeta = uit * (1. - Beta);
  const double sigma = std::sqrt(uitBeta * uitBeta + 4. * Beta * a0 * a0);
  pgb = 0.5 * (pg0 + pgi - 0.5 * r0 * sigma * (u0t - uit)) -
        ((pgi - pg0) + r0 * (uit - u0t) * uit * BetaM) * uit * BetaM / (2. * sigma);
  pgb = std::max(pgb, MinP);
  ub = u0 + 2. * n * (pgb - pg0) * (1.0 / (r0 * (sigma + uit * BetaM)));
  double rhob = r0 + (pgb - pg0) * (sigma - uit * BetaM) / (Beta * a0 * a0 * (sigma + uit * BetaM));
  Tb = (pgb + pamb) / (Rt * rhob);
}
void cv_outflow(double& pgb, double& Tb, V3& ub, double pgi, double Ti, V3 ui, double pg0,
                double T0, V3 u0, V3 n, double us_n, double pamb, double gamma, double Rt,
                double Beta) {
  (void)Ti;
  const double uit = dot(ui, n) - us_n, u0t = dot(u0, n) - us_n;
  const double a0 = std::sqrt(gamma * Rt * T0);
  const double r0 = (pg0 + pamb) / (Rt * T0);
  const double MinP = 0.1 * (pgi + pamb) - pamb;
  const double BetaM = 0.5 * (1.0 - Beta);
  const double uitBeta = uit * (1. - Beta);
  const double sigma = std::sqrt(uitBeta * uitBeta + 4. * Beta * a0 * a0);
  pgb = .5 * (pgi + pg0 - 0.5 * r0 * sigma * (u0t - uit)) +
        ((pgi - pg0) + r0 * (uit - u0t) * uit * BetaM) * uit * BetaM / (2. * sigma);
  pgb = std::max(pgb, MinP);
  ub = ui + 2. * n * (pgi - pgb) * (1.0 / (r0 * (sigma + uit * BetaM)));
  const double rhob = r0 + (pgb - pgi) * (sigma - uit * BetaM) / (Beta * a0 * a0 * (sigma + uit * BetaM));
  Tb = (pgb + pamb) / (Rt * rhob);
}

// ---------------------------------------------------------------------------
// 5x5 LU with partial pivoting (textbook Doolittle; Loci's decompose_lu_pivot
// is not vendored) and the solve used by linearSolverSGS.loci:43-69.
// ---------------------------------------------------------------------------
template <class TB>
bool lu5(TB A[25], int piv[5]) {
  bool ok = true;
  for (int k = 0; k < 5; ++k) {
    int p = k;
    TB best = std::fabs(A[k * 5 + k]);
    for (int i = k + 1; i < 5; ++i)
      if (std::fabs(A[i * 5 + k]) > best) {
        best = std::fabs(A[i * 5 + k]);
        p = i;
      }
    piv[k] = p;
    if (p != k)
      for (int j = 0; j < 5; ++j) std::swap(A[k * 5 + j], A[p * 5 + j]);
    if (A[k * 5 + k] == TB(0)) {
      ok = false;
      continue;
    }
    for (int i = k + 1; i < 5; ++i) {
      A[i * 5 + k] /= A[k * 5 + k];
      TB l = A[i * 5 + k];
      for (int j = k + 1; j < 5; ++j) A[i * 5 + j] -= l * A[k * 5 + j];
    }
  }
  return ok;
}
template <class TB, class TX>
void lu5_solve(const TB A[25], const int piv[5], const TX b[5], TX x[5]) {
  TX y[5];
  for (int i = 0; i < 5; ++i) y[i] = b[i];
  for (int k = 0; k < 5; ++k)
    if (piv[k] != k) std::swap(y[k], y[piv[k]]);
  for (int i = 1; i < 5; ++i)
    for (int j = 0; j < i; ++j) y[i] -= TX(A[i * 5 + j]) * y[j];
  for (int i = 4; i >= 0; --i) {
    for (int j = i + 1; j < 5; ++j) y[i] -= TX(A[i * 5 + j]) * y[j];
    y[i] /= TX(A[i * 5 + i]);
  }
  for (int i = 0; i < 5; ++i) x[i] = y[i];
}

}  // namespace

// ---------------------------------------------------------------------------
// Mesh-level oracle
// ---------------------------------------------------------------------------
struct orc_ctx {
  fpsi_params P;
  int64_t nc = 0, nf = 0;
  std::vector<int32_t> cl, cr;
  std::vector<fpsi_bc> bcs;
  // geometry
  std::vector<double> vol, cc;          // nc, nc*3
  std::vector<double> an, area, fc;     // nf*3, nf, nf*3
  std::vector<double> rL, rR;           // nf*3: x_f - x_cl, x_f - x_cr(image)
  std::vector<double> Minv;             // nc*6 LSQ inverse (xx,xy,xz,yy,yz,zz)
  double vol_tot = 0;
  // cell -> faces (upper = faces with cl==c, lower = cr==c, bnd = boundary)
  std::vector<int64_t> up_off, lo_off, bd_off;
  std::vector<int64_t> up, lo, bd;
  // state & results
  std::vector<double> T, pg, u;         // nc, nc, nc*3
  std::vector<double> tmu;              // nc eddy viscosity (turbulent regime)
  std::vector<double> qb;               // nbf... stored per face (nf*5): boundary face state
  std::vector<double> bc_pmean;         // per condition: area-weighted mean gauge pressure
  bool bcs_from_mdot = false;           // fixed-mass mass fluxes still to derive from mdot
  uint64_t bc_err = 0;                  // boundary-condition error bits of the last residual
  std::vector<double> grad, phi;        // nc*15, nc*5
  std::vector<double> F, maxev;         // nf*5, nf
  std::vector<double> src, dtau;        // nc*5, nc
  // time-accurate BDF2: primitive states of time levels n and n-1
  std::vector<double> Tn, pgn, un, Tm, pgm, um;
  bool have_levels = false;
  bool have_resid = false, have_asm = false, have_dq = false;
  // blocks (both precisions kept; the active one is selected by P.precision)
  std::vector<float> fjp32, fjm32, D32, LU32, B32;
  std::vector<double> fjp64, fjm64, D64, LU64, B64;
  std::vector<int> piv;                 // nc*5
  std::vector<double> dq;               // nc*5 (FP64 copy of the result)
  // Spalart-Allmaras working variable and its scalar system
  std::vector<double> nut, wdist;       // nc
  std::vector<double> sa_grad, sa_phi;  // nc*3, nc
  std::vector<double> sa_src, sa_D;     // nc
  std::vector<double> sa_fjp, sa_fjm;   // nf
  std::vector<double> sa_dq;            // nc
  bool have_sa = false, have_sa_dq = false;
};

static int g_threads = 1;

extern "C" int orc_set_threads(int n) {
  g_threads = n < 1 ? 1 : n;
#ifdef _OPENMP
  omp_set_num_threads(g_threads);
#endif
  return g_threads;
}

static inline V3 v3(const double* p) { return mk(p[0], p[1], p[2]); }

// Face and cell geometry (Loci FVM's area, facecenter, vol, cellcenter;
// restated: fan triangulation about the node average, divergence theorem).
static void compute_geometry(orc_ctx* o, const fpsi_mesh* m) {
  const int64_t nc = m->ncells, nf = m->nfaces;
  o->an.assign(nf * 3, 0);
  o->area.assign(nf, 0);
  o->fc.assign(nf * 3, 0);
  std::vector<double> Avec(nf * 3);
  for (int64_t f = 0; f < nf; ++f) {
    int64_t b = m->face_off[f], e = m->face_off[f + 1];
    int k = int(e - b);
    V3 xa = mk(0, 0, 0);
    for (int64_t i = b; i < e; ++i) xa = xa + v3(m->xyz + 3 * m->face_nodes[i]);
    xa = (1.0 / k) * xa;
    V3 A = mk(0, 0, 0), C = mk(0, 0, 0);
    double W = 0;
    for (int i = 0; i < k; ++i) {
      V3 p0 = v3(m->xyz + 3 * m->face_nodes[b + i]);
      V3 p1 = v3(m->xyz + 3 * m->face_nodes[b + (i + 1) % k]);
      V3 a = 0.5 * cross(p0 - xa, p1 - xa);
      A = A + a;
      double w = norm(a);
      C = C + (w / 3.0) * (xa + p0 + p1);
      W += w;
    }
    C = (1.0 / W) * C;
    double s = norm(A);
    o->area[f] = s;
    o->an[3 * f] = A.x / s;
    o->an[3 * f + 1] = A.y / s;
    o->an[3 * f + 2] = A.z / s;
    o->fc[3 * f] = C.x;
    o->fc[3 * f + 1] = C.y;
    o->fc[3 * f + 2] = C.z;
    Avec[3 * f] = A.x;
    Avec[3 * f + 1] = A.y;
    Avec[3 * f + 2] = A.z;
  }
  // reference point per cell: mean of its face centres (in its own frame)
  std::vector<double> xr(nc * 3, 0);
  std::vector<int> cnt(nc, 0);
  for (int64_t f = 0; f < nf; ++f) {
    V3 x = v3(&o->fc[3 * f]);
    int c = m->cl[f];
    xr[3 * c] += x.x, xr[3 * c + 1] += x.y, xr[3 * c + 2] += x.z, cnt[c]++;
    if (m->cr[f] >= 0) {
      int d = m->cr[f];
      V3 s = m->pshift ? v3(m->pshift + 3 * f) : mk(0, 0, 0);
      V3 y = x - s;
      xr[3 * d] += y.x, xr[3 * d + 1] += y.y, xr[3 * d + 2] += y.z, cnt[d]++;
    }
  }
  for (int64_t c = 0; c < nc; ++c)
    for (int i = 0; i < 3; ++i) xr[3 * c + i] /= cnt[c];
  o->vol.assign(nc, 0);
  o->cc.assign(nc * 3, 0);
  // pyramids on the fan triangles of every face, seen from each adjacent cell
  for (int64_t f = 0; f < nf; ++f) {
    int64_t b = m->face_off[f], e = m->face_off[f + 1];
    int k = int(e - b);
    V3 xa = mk(0, 0, 0);
    for (int64_t i = b; i < e; ++i) xa = xa + v3(m->xyz + 3 * m->face_nodes[i]);
    xa = (1.0 / k) * xa;
    for (int side = 0; side < 2; ++side) {
      int c = side == 0 ? m->cl[f] : m->cr[f];
      if (c < 0) continue;
      V3 s = (side == 1 && m->pshift) ? v3(m->pshift + 3 * f) : mk(0, 0, 0);
      double sg = side == 0 ? 1.0 : -1.0;
      V3 x0 = v3(&xr[3 * c]);
      for (int i = 0; i < k; ++i) {
        V3 p0 = v3(m->xyz + 3 * m->face_nodes[b + i]) - s;
        V3 p1 = v3(m->xyz + 3 * m->face_nodes[b + (i + 1) % k]) - s;
        V3 pa = xa - s;
        double v = sg * dot(pa - x0, cross(p0 - x0, p1 - x0)) / 6.0;
        V3 cen = 0.25 * (x0 + pa + p0 + p1);
        o->vol[c] += v;
        o->cc[3 * c] += v * cen.x;
        o->cc[3 * c + 1] += v * cen.y;
        o->cc[3 * c + 2] += v * cen.z;
      }
    }
  }
  for (int64_t c = 0; c < nc; ++c)
    for (int i = 0; i < 3; ++i) o->cc[3 * c + i] /= o->vol[c];
  o->vol_tot = 0;
  for (int64_t c = 0; c < nc; ++c) o->vol_tot += o->vol[c];
  o->rL.assign(nf * 3, 0);
  o->rR.assign(nf * 3, 0);
  for (int64_t f = 0; f < nf; ++f) {
    V3 x = v3(&o->fc[3 * f]);
    V3 a = x - v3(&o->cc[3 * m->cl[f]]);
    o->rL[3 * f] = a.x, o->rL[3 * f + 1] = a.y, o->rL[3 * f + 2] = a.z;
    if (m->cr[f] >= 0) {
      V3 s = m->pshift ? v3(m->pshift + 3 * f) : mk(0, 0, 0);
      V3 bb = x - (v3(&o->cc[3 * m->cr[f]]) + s);
      o->rR[3 * f] = bb.x, o->rR[3 * f + 1] = bb.y, o->rR[3 * f + 2] = bb.z;
    }
  }
}

static void wall_distance(orc_ctx* o, const fpsi_mesh* m);
static void sa_tmu(orc_ctx* o);

extern "C" int orc_create(orc_ctx** out, const fpsi_mesh* m, const fpsi_params* p) {
  if (!out || !m || !p) return FPSI_E_INVALID;
  orc_ctx* o = new orc_ctx();
  o->P = *p;
  o->nc = m->ncells;
  o->nf = m->nfaces;
  o->cl.assign(m->cl, m->cl + m->nfaces);
  o->cr.assign(m->cr, m->cr + m->nfaces);
  o->bcs.assign(m->bcs, m->bcs + m->nbc);
  o->bcs_from_mdot = true;
  compute_geometry(o, m);
  const int64_t nc = o->nc, nf = o->nf;
  // cell -> face lists in face order (the order Loci's upper/lower maps keep)
  o->up_off.assign(nc + 1, 0);
  o->lo_off.assign(nc + 1, 0);
  o->bd_off.assign(nc + 1, 0);
  for (int64_t f = 0; f < nf; ++f) {
    if (o->cr[f] >= 0) {
      o->up_off[o->cl[f] + 1]++;
      o->lo_off[o->cr[f] + 1]++;
    } else {
      o->bd_off[o->cl[f] + 1]++;
    }
  }
  for (int64_t c = 0; c < nc; ++c) {
    o->up_off[c + 1] += o->up_off[c];
    o->lo_off[c + 1] += o->lo_off[c];
    o->bd_off[c + 1] += o->bd_off[c];
  }
  o->up.resize(o->up_off[nc]);
  o->lo.resize(o->lo_off[nc]);
  o->bd.resize(o->bd_off[nc]);
  {
    std::vector<int64_t> pu(o->up_off.begin(), o->up_off.end() - 1),
        pl(o->lo_off.begin(), o->lo_off.end() - 1), pb(o->bd_off.begin(), o->bd_off.end() - 1);
    for (int64_t f = 0; f < nf; ++f) {
      if (o->cr[f] >= 0) {
        o->up[pu[o->cl[f]]++] = f;
        o->lo[pl[o->cr[f]]++] = f;
      } else {
        o->bd[pb[o->cl[f]]++] = f;
      }
    }
  }
  // LSQ normal matrices M = sum d d^T over face neighbours (boundary: face centre)
  o->Minv.assign(nc * 6, 0);
  for (int64_t c = 0; c < nc; ++c) {
    double M[6] = {0, 0, 0, 0, 0, 0};
    auto add = [&](V3 d) {
      M[0] += d.x * d.x, M[1] += d.x * d.y, M[2] += d.x * d.z;
      M[3] += d.y * d.y, M[4] += d.y * d.z, M[5] += d.z * d.z;
    };
    for (int64_t k = o->up_off[c]; k < o->up_off[c + 1]; ++k) {
      int64_t f = o->up[k];
      add(v3(&o->rL[3 * f]) - v3(&o->rR[3 * f]));
    }
    for (int64_t k = o->lo_off[c]; k < o->lo_off[c + 1]; ++k) {
      int64_t f = o->lo[k];
      add(v3(&o->rR[3 * f]) - v3(&o->rL[3 * f]));
    }
    for (int64_t k = o->bd_off[c]; k < o->bd_off[c + 1]; ++k) add(v3(&o->rL[3 * o->bd[k]]));
    double a = M[0], b = M[1], cc = M[2], d = M[3], e = M[4], f = M[5];
    double A00 = d * f - e * e, A01 = cc * e - b * f, A02 = b * e - cc * d;
    double A11 = a * f - cc * cc, A12 = b * cc - a * e, A22 = a * d - b * b;
    double det = a * A00 + b * A01 + cc * A02;
    double r = 1.0 / det;
    double* mi = &o->Minv[6 * c];
    mi[0] = A00 * r, mi[1] = A01 * r, mi[2] = A02 * r;
    mi[3] = A11 * r, mi[4] = A12 * r, mi[5] = A22 * r;
  }
  o->T.assign(nc, 0);
  o->pg.assign(nc, 0);
  o->u.assign(nc * 3, 0);
  o->tmu.assign(nc, 0);
  o->nut.assign(nc, 1e-6);  // nuTilde_ic default (SA_ic.loci:39-50)
  wall_distance(o, m);
  *out = o;
  return FPSI_OK;
}

extern "C" void orc_destroy(orc_ctx* o) { delete o; }

extern "C" int orc_set_params(orc_ctx* o, const fpsi_params* p) {
  o->P = *p;
  o->have_asm = false;
  o->have_levels = false;
  return FPSI_OK;
}

extern "C" int orc_get_geometry(orc_ctx* o, double* vol, double* cellcenter, double* face_an,
                                double* face_area, double* facecenter) {
  if (vol) std::memcpy(vol, o->vol.data(), sizeof(double) * o->nc);
  if (cellcenter) std::memcpy(cellcenter, o->cc.data(), sizeof(double) * o->nc * 3);
  if (face_an)
    for (int64_t f = 0; f < o->nf; ++f)
      for (int i = 0; i < 3; ++i) face_an[3 * f + i] = o->an[3 * f + i] * o->area[f];
  if (face_area) std::memcpy(face_area, o->area.data(), sizeof(double) * o->nf);
  if (facecenter) std::memcpy(facecenter, o->fc.data(), sizeof(double) * o->nf * 3);
  return FPSI_OK;
}

extern "C" int orc_set_state(orc_ctx* o, const double* T, const double* pg, const double* u) {
  std::memcpy(o->T.data(), T, sizeof(double) * o->nc);
  std::memcpy(o->pg.data(), pg, sizeof(double) * o->nc);
  std::memcpy(o->u.data(), u, sizeof(double) * o->nc * 3);
  o->have_resid = o->have_asm = o->have_dq = false;
  o->have_levels = false;
  return FPSI_OK;
}
extern "C" int orc_get_state(orc_ctx* o, double* T, double* pg, double* u) {
  std::memcpy(T, o->T.data(), sizeof(double) * o->nc);
  std::memcpy(pg, o->pg.data(), sizeof(double) * o->nc);
  std::memcpy(u, o->u.data(), sizeof(double) * o->nc * 3);
  return FPSI_OK;
}

// ---- total-pressure and fixed-mass conditions (their own form) ----------
// analytic flux of one state, inviscidFlux (inviscidFlux.h:25-45)
static void state_flux(double F[5], double pg, double T, V3 U, V3 an, double area, double pamb,
                       double Rt, double gamma) {
  const double gm1 = gamma - 1;
  const double rho = (pg + pamb) / (Rt * T);
  const double h0 = Rt * T * gamma / gm1 + 0.5 * dot(U, U);
  const double e0 = h0 - Rt * T;
  const double uta = dot(U, an);
  const double mdot = area * rho * uta;
  F[0] = mdot;
  F[1] = mdot * U.x + area * pg * an.x;
  F[2] = mdot * U.y + area * pg * an.y;
  F[3] = mdot * U.z + area * pg * an.z;
  F[4] = mdot * e0 + area * (pg + pamb) * uta;
}

// isentropic inflow from p0 (absolute), T0 and the inside state, flow along
// dir (= -n): bcIsentropic.loci:52-160
static void isentropic_bc(double& pb, double& Tb, V3& ub, double T0, double p0, double gamma,
                          double Rt, V3 ui, double Ti, V3 dir) {
  const double gm1 = gamma - 1.;
  const double a0 = std::sqrt(gamma * Rt * T0), ai = std::sqrt(gamma * Rt * Ti);
  const double uit = dot(ui, dir);
  double unb = uit, ab = a0;
  {  // fixed_p0t0_bc: outgoing invariant and the energy equation
    const double rim = uit - 2. * ai / gm1;
    const double a = 2. / gm1 + 1, b = 2. * rim, c = 0.5 * gm1 * rim * rim - a0 * a0;
    const double D = b * b - 4. * a * c;
    if (D < 0) {
      ab = a0;
      unb = rim + 2. * ab / gm1;
    } else {
      ab = std::max((-b + std::sqrt(D)) / (2. * a), .25 * a0);
      unb = rim + 2. * ab / gm1;
    }
  }
  auto relations = [&](double abx, double unx) {
    ub = unx * dir;
    double M = norm(ub) / abx;
    if (M > 1.0) {
      M = 1.0;
      const double utot = M * a0 / std::sqrt(1 + .5 * gm1 * M * M);
      ub = std::sqrt(std::max(utot * utot, 0.0)) * dir;
    }
    Tb = T0 / (1 + .5 * gm1 * M * M);
    pb = p0 * std::pow(1. + .5 * gm1 * M * M, -gamma / gm1);
  };
  relations(ab, unb);
  double f = (Tb - Ti) / std::max(Ti, Tb) - .1;
  if (f > 0) {
    f = std::pow(f, .5);
    ab = (1 - f) * ab + f * a0;
    unb = (1 - f) * unb + f * uit;
    relations(ab, unb);
  }
}

// fixed mass-flux inflow at total temperature Tstag: bcFixedMass.loci:84-135;
// returns false when the temperature iteration did not converge
static bool fixed_mass_bc(V3& ub, double& Tb, double& pgb, double pin, double Tin, double mflux,
                          V3 dir, V3 n, double Tstag, double pamb, double gamma, double Rt) {
  double T = Tin;
  const double eps = Tin * 1e-9;
  int iter;
  for (iter = 0; iter < 1000; ++iter) {
    const double rho = pin / (Rt * T);
    const double a = std::sqrt(gamma * Rt * T);
    const double M = (mflux / rho) / a;
    const double lam = std::sqrt(((gamma + 1.0) * M * M) / ((gamma - 1.0) * M * M + 2));
    const double p0 = pin * std::pow((1. - ((gamma - 1.) / (gamma + 1.)) * lam * lam), -gamma / (gamma - 1.0));
    const double rho0 = p0 / (Rt * Tstag);
    const double rho1 = rho0 * std::pow((1. - (gamma - 1.0) / (gamma + 1.0) * lam * lam), 1.0 / (gamma - 1.0));
    const double T1 = pin / (rho1 * Rt);
    if (std::fabs(T1 - T) < eps) break;
    T = T1;
  }
  const double vel = mflux / (pin / (Rt * T));
  ub = dir * (-vel / dot(dir, n));
  Tb = T;
  pgb = pin - pamb;
  return iter < 1000;
}

// fixed mass-flux outflow: bcFixedMassOutflow.loci:86-132
static void fixed_mass_outflow_bc(V3& ub, double& Tb, double& pgb, double rhoin, double pin,
                                  double Tin, V3 uin, double gam, double cin, double mflux,
                                  double pamb, V3 n) {
  const double M2 = dot(uin, uin) / (cin * cin);
  double fm = 1. + 0.5 * (gam - 1.) * M2;
  const double p0 = pin * std::pow(fm, gam / (gam - 1.));
  const double T0 = Tin * fm;
  const double rho0 = rhoin * std::pow(fm, 1. / (gam - 1.));
  const double rhos = rho0 * std::pow(2. / (gam + 1.), 1. / (gam - 1.));
  double cstar = cin * std::sqrt(2. * fm / (gam + 1.));
  double u = std::min(mflux, rhos * cstar) / rhoin;
  fm = 1. + 0.5 * (gam - 1.) * (u / cin) * (u / cin);
  cstar = cin * std::sqrt(2. * fm / (gam + 1.));
  u = std::min(u, cstar);
  const double lambda = u / cstar;
  const double fl = 1. - ((gam - 1.) / (gam + 1.)) * lambda * lambda;
  const double p = p0 * std::pow(fl, gam / (gam - 1.));
  if (u < cin) {
    ub = uin + (u - dot(uin, n)) * n;
    Tb = T0 * fl;
    pgb = p - pamb;
  } else {
    ub = uin;
    Tb = Tin;
    pgb = pin - pamb;
  }
}

// boundary face state (gagePressure_f, temperature_f, u_f) from the cell
// centre state: farfield bcInflow.loci:311-344, supersonicInflow :270-278,
// extrapolate bcOutflow.loci:84-95, supersonicOutflow :127-142, outflow at a
// back pressure :206-244, reflecting (mirror of the normal velocity)
// bcImpermeable.loci:48-140.  Returns the boundary-condition error bits.
static uint64_t bc_face_state(const orc_ctx* o, int64_t f, double q[5]) {
  const fpsi_params& P = o->P;
  int c = o->cl[f];
  const fpsi_bc& bc = o->bcs[-o->cr[f] - 1];
  V3 n = v3(&o->an[3 * f]);
  double Ti = o->T[c], pgi = o->pg[c];
  V3 ui = v3(&o->u[3 * c]);
  V3 u0 = v3(bc.u);
  double pgb = pgi, Tb = Ti;
  V3 ub = ui;
  const double us_n = 0, Eta = 1.0;
  switch (bc.kind) {
    case FPSI_BC_FARFIELD: {
      double uit = dot(ui, n) - us_n;
      double ai = std::sqrt(P.gamma * P.Rtilde * Ti);
      double a0 = std::sqrt(P.gamma * P.Rtilde * bc.T);
      if (uit > 0) {
        if (uit > ai) {
          pgb = pgi, Tb = Ti, ub = ui;
        } else {
          cv_outflow(pgb, Tb, ub, pgi, Ti, ui, bc.pg, bc.T, u0, n, us_n, P.Pambient, P.gamma,
                     P.Rtilde, Eta);
        }
      } else {
        if (-uit > a0) {
          pgb = bc.pg, Tb = bc.T, ub = u0;
        } else {
          cv_inflow(pgb, Tb, ub, pgi, Ti, ui, bc.pg, bc.T, u0, n, us_n, P.Pambient, P.gamma,
                    P.Rtilde, Eta);
        }
      }
      break;
    }
    case FPSI_BC_INFLOW: {  // bcInflow.loci:376-401: Dirichlet where the flow leaves
      double uit = dot(ui, n) - us_n;
      double a0 = std::sqrt(P.gamma * P.Rtilde * bc.T);
      if (uit > 0 || -uit > a0) {
        pgb = bc.pg, Tb = bc.T, ub = u0;
      } else {
        cv_inflow(pgb, Tb, ub, pgi, Ti, ui, bc.pg, bc.T, u0, n, us_n, P.Pambient, P.gamma,
                  P.Rtilde, Eta);
      }
      break;
    }
    case FPSI_BC_SUPERSONIC_INFLOW:
      pgb = bc.pg, Tb = bc.T, ub = u0;
      break;
    case FPSI_BC_SUPERSONIC_OUTFLOW: {
      double ai = std::sqrt(P.gamma * P.Rtilde * Ti);
      double ut = dot(n, ui) - us_n;
      pgb = pgi;
      if (ut < ai) pgb -= (pgi + P.Pambient) * .1;
      Tb = Ti, ub = ui;
      break;
    }
    case FPSI_BC_REFLECTING: {
      double un = dot(ui, n);
      ub = ui - 2.0 * un * n;
      break;
    }
    case FPSI_BC_VISCOUS_WALL:  // stationary adiabatic wall (bcViscousWall.loci:148-218)
      ub = mk(0, 0, 0);
      break;
    case FPSI_BC_OUTFLOW:
    case FPSI_BC_OUTFLOW_MEAN: {
      // pBoundary - Pambient: p_BC, or (pMean) the cell's pressure plus the
      // difference of pMean and the boundary's mean pressure (:174-204)
      const double pref = bc.kind == FPSI_BC_OUTFLOW
                              ? bc.pg
                              : pgi + (bc.pg - o->bc_pmean[-o->cr[f] - 1]);
      const double uit = dot(ui, n) - us_n;
      const double ai = std::sqrt(P.gamma * P.Rtilde * Ti);
      const double rhoi = (pgi + P.Pambient) / (P.Rtilde * Ti);
      if (uit >= 0) {
        if (!(uit > ai)) {
          pgb = pref;
          Tb = (pgb + P.Pambient) / (P.Rtilde * rhoi);
        }
      } else {
        ub = mk(0, 0, 0);
        pgb = pgi - .05 * (pgi + P.Pambient);
        Tb = Ti;
        q[0] = Tb, q[1] = ub.x, q[2] = ub.y, q[3] = ub.z, q[4] = pgb;
        return FPSI_BCERR_OUTFLOW_BECAME_INFLOW;
      }
      break;
    }
    case FPSI_BC_ISENTROPIC_INFLOW: {
      double pb;
      isentropic_bc(pb, Tb, ub, bc.T, bc.pg + P.Pambient, P.gamma, P.Rtilde, ui, Ti, -1.0 * n);
      pgb = pb - P.Pambient;
      break;
    }
    case FPSI_BC_FIXED_MASS_INFLOW: {
      const bool ok = fixed_mass_bc(ub, Tb, pgb, pgi + P.Pambient, Ti, bc.mass_flux, -1.0 * n, n,
                                    bc.T, P.Pambient, P.gamma, P.Rtilde);
      q[0] = Tb, q[1] = ub.x, q[2] = ub.y, q[3] = ub.z, q[4] = pgb;
      return ok ? 0 : FPSI_BCERR_FIXED_MASS_FAILED_CONVERGENCE;
    }
    case FPSI_BC_FIXED_MASS_OUTFLOW: {
      const double pin = pgi + P.Pambient, rhoin = pin / (P.Rtilde * Ti);
      const double t = bc.mass_relax;
      const double mfb = (1. - t) * rhoin * dot(ui, n) + t * bc.mass_flux;
      fixed_mass_outflow_bc(ub, Tb, pgb, rhoin, pin, Ti, ui, P.gamma,
                            std::sqrt(P.gamma * P.Rtilde * Ti), mfb, P.Pambient, n);
      break;
    }
    default:  // extrapolate
      break;
  }
  q[0] = Tb, q[1] = ub.x, q[2] = ub.y, q[3] = ub.z, q[4] = pgb;
  return 0;
}

static inline void cell_q(const orc_ctx* o, int64_t c, double q[5]) {
  q[0] = o->T[c], q[1] = o->u[3 * c], q[2] = o->u[3 * c + 1], q[3] = o->u[3 * c + 2],
  q[4] = o->pg[c];
}

// Least-squares cell gradients (Loci FVM grads/gradv3d; method named in
// guide/inviscidFlux.tex:234-236) and per-variable limiters (Loci FVM
// limiters/limiterv3d; options guide/guide.tex:495-518).
static void gradients_and_limiters(orc_ctx* o) {
  const int64_t nc = o->nc;
  const int lim = o->P.limiter;
  const double Kl = o->P.Kl;
  o->grad.assign(nc * 15, 0);
  o->phi.assign(nc * 5, 0);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < nc; ++c) {
    double qc[5];
    cell_q(o, c, qc);
    double b[15] = {0};
    double qmax[5], qmin[5];
    for (int k = 0; k < 5; ++k) qmax[k] = qmin[k] = qc[k];
    auto nb = [&](V3 d, const double* qn) {
      for (int k = 0; k < 5; ++k) {
        double dq = qn[k] - qc[k];
        b[3 * k] += d.x * dq, b[3 * k + 1] += d.y * dq, b[3 * k + 2] += d.z * dq;
        qmax[k] = std::max(qmax[k], qn[k]);
        qmin[k] = std::min(qmin[k], qn[k]);
      }
    };
    for (int64_t k = o->up_off[c]; k < o->up_off[c + 1]; ++k) {
      int64_t f = o->up[k];
      double qn[5];
      cell_q(o, o->cr[f], qn);
      nb(v3(&o->rL[3 * f]) - v3(&o->rR[3 * f]), qn);
    }
    for (int64_t k = o->lo_off[c]; k < o->lo_off[c + 1]; ++k) {
      int64_t f = o->lo[k];
      double qn[5];
      cell_q(o, o->cl[f], qn);
      nb(v3(&o->rR[3 * f]) - v3(&o->rL[3 * f]), qn);
    }
    for (int64_t k = o->bd_off[c]; k < o->bd_off[c + 1]; ++k) {
      int64_t f = o->bd[k];
      nb(v3(&o->rL[3 * f]), &o->qb[5 * f]);
    }
    const double* mi = &o->Minv[6 * c];
    double* g = &o->grad[15 * c];
    for (int k = 0; k < 5; ++k) {
      double bx = b[3 * k], by = b[3 * k + 1], bz = b[3 * k + 2];
      g[3 * k] = mi[0] * bx + mi[1] * by + mi[2] * bz;
      g[3 * k + 1] = mi[1] * bx + mi[3] * by + mi[4] * bz;
      g[3 * k + 2] = mi[2] * bx + mi[4] * by + mi[5] * bz;
    }
    double* ph = &o->phi[5 * c];
    if (lim == FPSI_LIMITER_NONE) {
      for (int k = 0; k < 5; ++k) ph[k] = 1.0;
      continue;
    }
    if (lim == FPSI_LIMITER_ZERO) {
      for (int k = 0; k < 5; ++k) ph[k] = 0.0;
      continue;
    }
    const double h = std::cbrt(o->vol[c]);
    const double eps2 = (Kl * h) * (Kl * h) * (Kl * h);
    for (int k = 0; k < 5; ++k) ph[k] = 1.0;
    auto face = [&](V3 r) {
      for (int k = 0; k < 5; ++k) {
        double d2 = g[3 * k] * r.x + g[3 * k + 1] * r.y + g[3 * k + 2] * r.z;
        double p = 1.0;
        if (d2 != 0.0) {
          double d1 = d2 > 0 ? qmax[k] - qc[k] : qmin[k] - qc[k];
          if (lim == FPSI_LIMITER_BARTH) {
            p = std::min(1.0, d1 / d2);
          } else {
            double num = (d1 * d1 + eps2) + 2.0 * d2 * d1;
            double den = d1 * d1 + 2.0 * d2 * d2 + d1 * d2 + eps2;
            p = std::min(1.0, num / den);
          }
        }
        ph[k] = std::min(ph[k], p);
      }
    };
    for (int64_t k = o->up_off[c]; k < o->up_off[c + 1]; ++k) face(v3(&o->rL[3 * o->up[k]]));
    for (int64_t k = o->lo_off[c]; k < o->lo_off[c + 1]; ++k) face(v3(&o->rR[3 * o->lo[k]]));
    for (int64_t k = o->bd_off[c]; k < o->bd_off[c + 1]; ++k) face(v3(&o->rL[3 * o->bd[k]]));
  }
}

// MUSCL states leftsP/rightsP/leftv3d/rightv3d (Loci FVM), restated in the
// form flowPsi itself writes out at fluxLowDiss.loci:338-356: q_c + phi *
// grad.(x_f - x_c), with floors 0.1*min(T) and 0.1*min(pg) - 0.9*Pambient.
static void face_states(const orc_ctx* o, int64_t f, double qL[5], double qR[5]) {
  int c = o->cl[f];
  double qc[5];
  cell_q(o, c, qc);
  double qo[5];
  const bool bnd = o->cr[f] < 0;
  if (bnd) {
    for (int k = 0; k < 5; ++k) qo[k] = o->qb[5 * f + k];
  } else {
    cell_q(o, o->cr[f], qo);
  }
  const double tlim = 0.1 * std::min(qc[0], qo[0]);
  const double plim = 0.1 * std::min(qc[4], qo[4]) - 0.9 * o->P.Pambient;
  V3 r = v3(&o->rL[3 * f]);
  const double* g = &o->grad[15 * c];
  const double* ph = &o->phi[5 * c];
  for (int k = 0; k < 5; ++k)
    qL[k] = qc[k] + ph[k] * (g[3 * k] * r.x + g[3 * k + 1] * r.y + g[3 * k + 2] * r.z);
  qL[0] = std::max(qL[0], tlim);
  qL[4] = std::max(qL[4], plim);
  if (bnd) {
    for (int k = 0; k < 5; ++k) qR[k] = qo[k];
    return;
  }
  int d = o->cr[f];
  V3 s = v3(&o->rR[3 * f]);
  const double* gr = &o->grad[15 * d];
  const double* pr = &o->phi[5 * d];
  for (int k = 0; k < 5; ++k)
    qR[k] = qo[k] + pr[k] * (gr[3 * k] * s.x + gr[3 * k + 1] * s.y + gr[3 * k + 2] * s.z);
  qR[0] = std::max(qR[0], tlim);
  qR[4] = std::max(qR[4], plim);
}

static int bc_kind_of(const orc_ctx* o, int64_t f) {
  return o->cr[f] >= 0 ? 0 : o->bcs[-o->cr[f] - 1].kind;
}

// viscous face flux, fluxViscous.loci:112-292 (+ bcViscousWall.loci:172-184
// on adiabatic walls, no viscous flux on symmetry planes :294-297).  Face
// gradients (Loci FVM gradv3d_f / grads_f, not vendored): mean of the two
// cell gradients with the component along d = x_R - x_L replaced by the
// difference quotient; at boundary faces the cell gradient corrected the
// same way towards the face state.
struct VFace {
  double vf[4], uf[3], muT, kT, dist;
};
static double suth(double T, double a1, double a2, double a3) {
  return a1 * std::pow(T, a2) / (T + a3);
}
static VFace viscous_face(const orc_ctx* o, int64_t f) {
  const fpsi_params& P = o->P;
  VFace v;
  V3 n = v3(&o->an[3 * f]);
  const double A = o->area[f];
  const int64_t a = o->cl[f];
  double qa[5];
  cell_q(o, a, qa);
  const double* ga = &o->grad[15 * a];
  double gf[4][3];
  double muf, kf, tmuf = 0;
  const int kind = bc_kind_of(o, f);
  if (kind == 0) {
    const int64_t b = o->cr[f];
    double qc[5];
    cell_q(o, b, qc);
    const double* gb = &o->grad[15 * b];
    const double vl = o->vol[a], vr = o->vol[b];
    muf = (vl * suth(qc[0], P.mu_a1, P.mu_a2, P.mu_a3) + vr * suth(qa[0], P.mu_a1, P.mu_a2, P.mu_a3)) /
          (vl + vr);
    kf = (vl * suth(qc[0], P.k_a1, P.k_a2, P.k_a3) + vr * suth(qa[0], P.k_a1, P.k_a2, P.k_a3)) /
         (vl + vr);
    if (P.viscous == 2) tmuf = (o->tmu[b] * vl + o->tmu[a] * vr) / (vr + vl);
    const double factor = 1. / (vl + vr);
    for (int k = 0; k < 3; ++k) v.uf[k] = factor * (vl * qc[1 + k] + vr * qa[1 + k]);
    V3 d = v3(&o->rL[3 * f]) - v3(&o->rR[3 * f]);
    v.dist = dot(n, d);
    const double dd[3] = {d.x, d.y, d.z};
    const double d2 = dot(d, d);
    for (int w = 0; w < 4; ++w) {
      double gm[3];
      for (int k = 0; k < 3; ++k) gm[k] = 0.5 * (ga[3 * w + k] + gb[3 * w + k]);
      const double c = ((qc[w] - qa[w]) - (gm[0] * dd[0] + gm[1] * dd[1] + gm[2] * dd[2])) / d2;
      for (int k = 0; k < 3; ++k) gf[w][k] = gm[k] + c * dd[k];
    }
  } else {
    const double* qf = &o->qb[5 * f];
    muf = suth(qf[0], P.mu_a1, P.mu_a2, P.mu_a3);
    kf = suth(qf[0], P.k_a1, P.k_a2, P.k_a3);
    if (P.viscous == 2 && kind != FPSI_BC_VISCOUS_WALL) tmuf = o->tmu[a];
    for (int k = 0; k < 3; ++k) v.uf[k] = qf[1 + k];
    V3 r = v3(&o->rL[3 * f]);
    v.dist = dot(n, r);
    const double rr[3] = {r.x, r.y, r.z};
    const double r2 = dot(r, r);
    for (int w = 0; w < 4; ++w) {
      const double* gv = ga + 3 * w;
      const double c = ((qf[w] - qa[w]) - (gv[0] * rr[0] + gv[1] * rr[1] + gv[2] * rr[2])) / r2;
      for (int k = 0; k < 3; ++k) gf[w][k] = gv[k] + c * rr[k];
    }
  }
  v.muT = muf + tmuf;
  v.kT = kf + (P.viscous == 2 ? tmuf * (P.gamma * P.Rtilde / (P.gamma - 1.0)) / P.Prt : 0.0);
  if (kind == FPSI_BC_REFLECTING) {
    for (int k = 0; k < 4; ++k) v.vf[k] = 0;
    return v;
  }
  // tau, fluxViscous.loci:217-238
  const double mt = v.muT;
  const double dudx = gf[1][0], dvdy = gf[2][1], dwdz = gf[3][2];
  const double dvdx = gf[2][0], dwdx = gf[3][0], dwdy = gf[3][1];
  const double dudy = gf[1][1], dudz = gf[1][2], dvdz = gf[2][2];
  const double divm = (dudx + dvdy + dwdz) * (1. / 3.);
  const double txx = 2.0 * mt * (dudx - divm), tyy = 2.0 * mt * (dvdy - divm),
               tzz = 2.0 * mt * (dwdz - divm);
  const double txy = mt * (dudy + dvdx), txz = mt * (dudz + dwdx), tyz = mt * (dvdz + dwdy);
  // vflux, fluxViscous.loci:279-292
  v.vf[0] = (txx * n.x + txy * n.y + txz * n.z) * A;
  v.vf[1] = (txy * n.x + tyy * n.y + tyz * n.z) * A;
  v.vf[2] = (txz * n.x + tyz * n.y + tzz * n.z) * A;
  v.vf[3] = (v.uf[0] * v.vf[0] + v.uf[1] * v.vf[1] + v.uf[2] * v.vf[2]);
  if (kind != FPSI_BC_VISCOUS_WALL)
    v.vf[3] += (gf[0][0] * n.x + gf[0][1] * n.y + gf[0][2] * n.z) * v.kT * A;
  return v;
}

// thin-layer viscous Jacobian, fluxViscous.loci:315-448: Fj += sgn * J,
// each term added separately as the reference's += on real_fj blocks
template <class TB>
static void add_visc_jac(TB* M, const VFace& v, V3 n3, double A, double sgn) {
  const double n[3] = {n3.x, n3.y, n3.z};
  const double coef = v.muT * A / v.dist, third = 1.0 / 3.0;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      const double t = coef * ((r == c ? 1.0 : 0.0) + n[r] * n[c] * third);
      M[5 * (1 + r) + 1 + c] = TB(double(M[5 * (1 + r) + 1 + c]) + sgn * t);
    }
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) {
      const double t = v.uf[r] * coef * ((r == c ? 1.0 : 0.0) + n[r] * n[c] * third);
      M[21 + c] = TB(double(M[21 + c]) + sgn * t);
    }
  for (int c = 0; c < 3; ++c) M[21 + c] = TB(double(M[21 + c]) + sgn * 0.5 * v.vf[c]);
  M[20] = TB(double(M[20]) + sgn * (v.kT * A / v.dist));
}

extern "C" int orc_set_eddy_viscosity(orc_ctx* o, const double* tmu) {
  std::memcpy(o->tmu.data(), tmu, sizeof(double) * o->nc);
  o->have_resid = o->have_asm = o->have_dq = false;
  return FPSI_OK;
}

// ---- low-dissipation (KEC) flux, fluxLowDiss.loci ----------------------
// alpha_geom_f (fluxLowDiss.loci:122-138), rounded to FP32 (store<realF>).
// With rL = x_f - x_l and rR = x_f - x_r: df = x_r - x_l = rL - rR and
// dv = x_f - (x_l + x_r)/2 = (rL + rR)/2.
static float alpha_geom(const orc_ctx* o, int64_t f) {
  const V3 rl = v3(&o->rL[3 * f]), rr = v3(&o->rR[3 * f]);
  const V3 df = rl - rr, dv = 0.5 * (rl + rr);
  const double ndv = norm(dv), ndf = norm(df);
  const double cosa = std::min(std::sqrt(std::max(1. - 2. * ndv / ndf, 0.0)),
                               dot(v3(&o->an[3 * f]), df) / ndf);
  const double scale = o->P.lds_nonsym_coeff;
  const double s = o->P.lds_nonsym_factor / std::max(scale, 1.0);
  const double x = std::min(scale * (1. - cosa), 1.0);
  const double x2 = x * x, x3 = x2 * x;
  return float(x2 + s * (x3 - 2. * x2 + x));
}

// alpha_diss of every cell (fluxLowDiss.loci:141-176): veldiv from ufn
// (fluxLowDiss.loci:61-78) summed over the cell's faces, + on the cl side,
// in the cell's face order (upper, lower, boundary); interior faces use the
// face gradient of u of the viscous terms (viscous_face), boundary faces the
// boundary velocity.  vortMag from the cell gradient (solverTurbulence.loci:45-79).
static void alpha_diss(const orc_ctx* o, std::vector<double>& ad) {
  const int64_t nc = o->nc;
  const fpsi_params& P = o->P;
  ad.assign(nc, 0.0);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < nc; ++c) {
    double veldiv = 0.0, maxd2 = 0.0;
    auto interior = [&](int64_t f, double sign) {
      const int64_t a = o->cl[f], b = o->cr[f];
      const V3 rl = v3(&o->rL[3 * f]), rr = v3(&o->rR[3 * f]);
      const V3 d = rl - rr, dv = 0.5 * (rl + rr);
      const double d2 = dot(d, d);
      const double* ga = &o->grad[15 * a];
      const double* gb = &o->grad[15 * b];
      double uf[3];
      for (int v = 1; v < 4; ++v) {
        const V3 gm = 0.5 * (v3(ga + 3 * v) + v3(gb + 3 * v));
        const double ua = o->u[3 * a + v - 1], ub = o->u[3 * b + v - 1];
        const double cq = ((ub - ua) - dot(gm, d)) / d2;
        const V3 gf = gm + cq * d;
        uf[v - 1] = 0.5 * (ua + ub) + dot(gf, dv);
      }
      const double ufn = dot(mk(uf[0], uf[1], uf[2]), v3(&o->an[3 * f])) * o->area[f];
      veldiv += sign * ufn;
    };
    for (int64_t k = o->up_off[c]; k < o->up_off[c + 1]; ++k) {
      const int64_t f = o->up[k];
      maxd2 = std::max(maxd2, dot(v3(&o->rL[3 * f]), v3(&o->rL[3 * f])));
      interior(f, 1.0);
    }
    for (int64_t k = o->lo_off[c]; k < o->lo_off[c + 1]; ++k) {
      const int64_t f = o->lo[k];
      maxd2 = std::max(maxd2, dot(v3(&o->rR[3 * f]), v3(&o->rR[3 * f])));
      interior(f, -1.0);
    }
    for (int64_t k = o->bd_off[c]; k < o->bd_off[c + 1]; ++k) {
      const int64_t f = o->bd[k];
      maxd2 = std::max(maxd2, dot(v3(&o->rL[3 * f]), v3(&o->rL[3 * f])));
      const double* qb = &o->qb[5 * f];
      veldiv += dot(mk(qb[1], qb[2], qb[3]), v3(&o->an[3 * f])) * o->area[f];
    }
    const double V = o->vol[c];
    const double len = 2. * std::sqrt(maxd2);
    const double a = std::sqrt(P.gamma * P.Rtilde * o->T[c]);
    const double factor = P.lds_comp_factor * std::fabs(veldiv) * len / (a * V);
    const double alpha_comp = factor * factor;
    const double theta_2 = veldiv * veldiv / (V * V);
    const double* g = &o->grad[15 * c];
    const V3 w = mk(g[10] - g[8], g[5] - g[9], g[6] - g[4]);
    const double vm = norm(w);
    const double alpha_ducro = P.lds_ducros_factor * theta_2 / (theta_2 + vm * vm + 1e-10);
    double al = std::max(alpha_ducro, alpha_comp);
    al = std::min(al, P.lds_dissipation_limit);
    ad[c] = std::max(al, P.lds_use_upwind);
  }
}

// kec_flux (fluxLowDiss.loci:258-298), added to F
static void kec_flux(double F[5], double pgl, double Tl, V3 Ul, double pgr, double Tr, V3 Ur,
                     V3 an, double area, double pamb, double Rt, double gamma) {
  const V3 uf = 0.5 * (Ul + Ur);
  const double ufn = dot(uf, an);
  const double pgf = 0.5 * (pgl + pgr);
  const double tf = Tl * Tr * (pgl + pgr + 2 * pamb) / ((pgl + pamb) * Tr + (pgr + pamb) * Tl);
  const double rf = (pgf + pamb) / (Rt * tf);
  const double mdot = rf * ufn;
  F[0] += area * mdot;
  F[1] += area * (mdot * uf.x + pgf * an.x);
  F[2] += area * (mdot * uf.y + pgf * an.y);
  F[3] += area * (mdot * uf.z + pgf * an.z);
  const double e_internalf = 0.5 * Rt * (Tl + Tr) / (gamma - 1);
  const double ke_f = dot(uf, uf) - 0.25 * (dot(Ul, Ul) + dot(Ur, Ur));
  F[4] += area * (mdot * (ke_f + e_internalf) + ufn * (pgf + pamb));
}

// KEC::iflux of interior face f (fluxLowDiss.loci:320-431); qL, qR are the
// MUSCL face states with their floors (face_states)
static void kec_iflux(const orc_ctx* o, int64_t f, const double qL[5], const double qR[5],
                      const std::vector<double>& ad, double F[5]) {
  const fpsi_params& P = o->P;
  const int64_t a = o->cl[f], b = o->cr[f];
  const V3 an = v3(&o->an[3 * f]);
  const double A = o->area[f];
  const double pglim = 0.1 * std::min(o->pg[a], o->pg[b]) + -0.9 * P.Pambient;
  const double tlim = 0.1 * std::min(o->T[a], o->T[b]);
  const double pgL = qL[4], pgR = qR[4], tL = qL[0], tR = qR[0];
  const double rL = (pgL + P.Pambient) / (P.Rtilde * tL);
  const double rR = (pgR + P.Pambient) / (P.Rtilde * tR);
  const double al2 = P.gamma * P.Rtilde * tL, ar2 = P.gamma * P.Rtilde * tR;
  const double dp = 2. * std::fabs(pgL - pgR) / std::max(rL * al2, rR * ar2);
  const double alpha_c = std::max(std::max(ad[a], ad[b]), std::min(1.0, dp * 1.0 - 0.5));
  const double alpha = std::max(alpha_c, double(alpha_geom(o, f)));
  for (int i = 0; i < 5; ++i) F[i] = 0;
  if (alpha > 1e-10) {
    const V3 uL = mk(qL[1], qL[2], qL[3]), uR = mk(qR[1], qR[2], qR[3]);
    const double amin = std::sqrt(std::min(al2, ar2));
    const double utmax = std::max(std::fabs(dot(uL, an)), std::fabs(dot(uR, an)));
    const double Ma = std::max(alpha_c, std::min(1.0, utmax / amin + 1e-4));
    const V3 uLp = uL + 0.5 * (1. - Ma) * (uR - uL);
    const V3 uRp = uR + 0.5 * (1. - Ma) * (uL - uR);
    hllc_flux(F, pgL, tL, uLp, pgR, tR, uRp, an, A * alpha, P.Pambient, P.Rtilde, P.gamma, 0.0, 1.0);
  }
  const V3 dv = 0.5 * (v3(&o->rL[3 * f]) + v3(&o->rR[3 * f]));
  auto at = [&](int64_t c, double& pg, double& t, V3& u) {
    const double* g = &o->grad[15 * c];
    const double* ph = &o->phi[5 * c];
    pg = std::max(o->pg[c] + ph[4] * dot(v3(g + 12), dv), pglim);
    t = std::max(o->T[c] + ph[0] * dot(v3(g), dv), tlim);
    u = mk(o->u[3 * c] + ph[1] * dot(v3(g + 3), dv), o->u[3 * c + 1] + ph[2] * dot(v3(g + 6), dv),
           o->u[3 * c + 2] + ph[3] * dot(v3(g + 9), dv));
  };
  double pg_l, t_l, pg_r, t_r;
  V3 u_l, u_r;
  at(a, pg_l, t_l, u_l);
  at(b, pg_r, t_r, u_r);
  kec_flux(F, pg_l, t_l, u_l, pg_r, t_r, u_r, an, A * (1. - alpha), P.Pambient, P.Rtilde, P.gamma);
}

// roedis (fluxLowDiss.loci:180-270): Roe-type dissipation of two states on
// the area `sada`, subtracted from F
static void roe_dissipation(double F[5], double pg_l, V3 Ul, double Tl, double pg_r, V3 Ur,
                            double Tr, double Rt, double gamma, double pamb, V3 an, double sada) {
  const double pl = pg_l + pamb, pr = pg_r + pamb;
  const double rl = pl / (Rt * Tl), rr = pr / (Rt * Tr);
  const double rgm1 = 1. / (gamma - 1);
  const double el = Rt * rgm1 * Tl, er = Rt * rgm1 * Tr;
  const double re0l = rl * el + 0.5 * rl * dot(Ul, Ul);
  const double re0r = rr * er + 0.5 * rr * dot(Ur, Ur);
  const double h0l = (re0l + pl) / rl, h0r = (re0r + pr) / rr;
  const double rho = std::sqrt(rl * rr);
  const double srl = std::sqrt(rl), srr = std::sqrt(rr), f = 1. / (srl + srr);
  const V3 U = (Ul * srl + Ur * srr) * f;
  const double un = dot(U, an);
  const double h0 = (h0l * srl + h0r * srr) * f;
  const double al2 = gamma * Rt * Tl, ar2 = gamma * Rt * Tr;
  const double af2 = std::max(2. * al2 * ar2 / (al2 + ar2), 1e-30);
  const double cp = Rt * gamma * rgm1;
  const double Tm = (Tl * ar2 + Tr * al2) * af2 / (2. * ar2 * al2);
  const double rT = -rho / Tm;
  const double a = std::sqrt(af2);
  const double ev1 = std::fabs(un), ev2 = std::fabs(un - a), ev3 = std::fabs(un + a);
  const V3 Uj = Ur - Ul;
  const double utj = dot(Uj, an), pj = pg_r - pg_l, Tj = Tr - Tl;
  const double t1 = ev2 - ev3, t2 = (ev2 + ev3 - 2 * ev1), t3 = -rho * a / 2.;
  const double t4 = 2. * t2 * a, t5 = t2 / 2., t6 = (ev2 + ev3) / 2.;
  const double c1 = (1 - gamma) / rT, ra2 = 1. / (a * a), gm1 = gamma - 1;
  const double t7 = (1 + gm1 + c1 * rT) * t1 * t3 * ra2;
  const double t8 = (gamma * t6 + c1 * rT * t5) * ra2;
  const double t9 = cp * rho + h0 * rT;
  const double x1 = gamma * h0 * t1 * t3 * ra2, x2 = c1 * t1 * t3 * t9 * ra2;
  const double x3 = rT * Tm * t1 * t3 * 1 / rho, x4 = .25 * rho * t4 * un / a;
  const double t10 = (x1 + x2 + x3 + x4);
  const double t11 = (ra2 * h0 + (t9 - rho * cp) * ra2 * gm1 / rT + rT * Tm / rho) * t6 +
                     ra2 * t9 * t5 * c1 - .5 * un * t1 / a;
  const double coef = 0.5 * sada;
  const double md = coef * (pj * t8 + utj * t7 + ev1 * Tj * rT);
  F[0] -= md;
  const double fp = .5 * (.5 * rho * t4 * utj - pj * t1) / a;
  F[1] -= md * U.x + coef * (ev1 * rho * Uj.x + fp * an.x);
  F[2] -= md * U.y + coef * (ev1 * rho * Uj.y + fp * an.y);
  F[3] -= md * U.z + coef * (ev1 * rho * Uj.z + fp * an.z);
  F[4] -= coef * (pj * t11 + t10 * utj + ev1 * (t9 * Tj + rho * dot(U, Uj)));
}

// SSF::iflux of interior face f (fluxLowDiss.loci:436-640, the cubic
// extrapolation variant that the file compiles)
static void ssf_iflux(const orc_ctx* o, int64_t f, const double qL[5], const double qR[5],
                      const std::vector<double>& ad, double F[5]) {
  const fpsi_params& P = o->P;
  const int64_t a = o->cl[f], b = o->cr[f];
  const V3 an = v3(&o->an[3 * f]);
  const double A = o->area[f];
  const double pglim = 0.1 * std::min(o->pg[a], o->pg[b]) + -0.9 * P.Pambient;
  const double tlim = 0.1 * std::min(o->T[a], o->T[b]);
  const double pgL = qL[4], pgR = qR[4], tL = qL[0], tR = qR[0];
  const double rL = (pgL + P.Pambient) / (P.Rtilde * tL);
  const double rR = (pgR + P.Pambient) / (P.Rtilde * tR);
  const double al2 = P.gamma * P.Rtilde * tL, ar2 = P.gamma * P.Rtilde * tR;
  const double dp = 2. * std::fabs(pgL - pgR) / std::max(rL * al2, rR * ar2);
  const double alpha_c = std::max(std::max(ad[a], ad[b]), std::min(1.0, dp * 1.0 - 0.5));
  const double alpha = alpha_c;
  const double amin = std::sqrt(std::min(al2, ar2));
  for (int i = 0; i < 5; ++i) F[i] = 0;
  if (alpha > 1e-10) {
    const V3 uL = mk(qL[1], qL[2], qL[3]), uR = mk(qR[1], qR[2], qR[3]);
    const double utmax = std::max(std::fabs(dot(uL, an)), std::fabs(dot(uR, an)));
    const double Ma = std::max(alpha_c, std::min(1.0, utmax / amin + 1e-4));
    const V3 uLp = uL + 0.5 * (1. - Ma) * (uR - uL);
    const V3 uRp = uR + 0.5 * (1. - Ma) * (uL - uR);
    hllc_flux(F, pgL, tL, uLp, pgR, tR, uRp, an, A * alpha, P.Pambient, P.Rtilde, P.gamma, 0.0, 1.0);
  }
  const V3 rl = v3(&o->rL[3 * f]), rr = v3(&o->rR[3 * f]);
  const V3 dv = 0.5 * (rl + rr), dv2 = rl - rr;
  const double* ga = &o->grad[15 * a];
  const double* gb = &o->grad[15 * b];
  auto at = [&](int64_t c, double& pg, double& t, V3& u) {
    const double* g = &o->grad[15 * c];
    const double* ph = &o->phi[5 * c];
    pg = std::max(o->pg[c] + ph[4] * dot(v3(g + 12), dv), pglim);
    t = std::max(o->T[c] + ph[0] * dot(v3(g), dv), tlim);
    u = mk(o->u[3 * c] + ph[1] * dot(v3(g + 3), dv), o->u[3 * c + 1] + ph[2] * dot(v3(g + 6), dv),
           o->u[3 * c + 2] + ph[3] * dot(v3(g + 9), dv));
  };
  double pg_l, t_l, pg_r, t_r;
  V3 u_l, u_r;
  at(a, pg_l, t_l, u_l);
  at(b, pg_r, t_r, u_r);
  const double pg_ll = std::max(pg_r - 2. * dot(v3(ga + 12), dv2), pglim);
  const double pg_rr = std::max(pg_l + 2. * dot(v3(gb + 12), dv2), pglim);
  const double t_ll = std::max(t_r - 2. * dot(v3(ga), dv2), tlim);
  const double t_rr = std::max(t_l + 2. * dot(v3(gb), dv2), tlim);
  const V3 u_ll = u_r - mk(2. * dot(v3(ga + 3), dv2), 2. * dot(v3(ga + 6), dv2), 2. * dot(v3(ga + 9), dv2));
  const V3 u_rr = u_l + mk(2. * dot(v3(gb + 3), dv2), 2. * dot(v3(gb + 6), dv2), 2. * dot(v3(gb + 9), dv2));
  const double CC = P.ssf_coeff / 6.0;
  const double sada = A * (1. - alpha);
  kec_flux(F, pg_l, t_l, u_l, pg_r, t_r, u_r, an, (1. + 2. * CC) * sada, P.Pambient, P.Rtilde, P.gamma);
  kec_flux(F, pg_l, t_l, u_l, pg_rr, t_rr, u_rr, an, -CC * sada, P.Pambient, P.Rtilde, P.gamma);
  kec_flux(F, pg_ll, t_ll, u_ll, pg_r, t_r, u_r, an, -CC * sada, P.Pambient, P.Rtilde, P.gamma);
  const double a0 = 1. / 3., a1 = 5. / 6., a2 = -1. / 6.;
  const double pg_lq = std::max(pglim, a0 * pg_r + a1 * pg_l + a2 * pg_ll);
  const double pg_rq = std::max(pglim, a0 * pg_l + a1 * pg_r + a2 * pg_rr);
  const double t_lq = std::max(tlim, a0 * t_r + a1 * t_l + a2 * t_ll);
  const double t_rq = std::max(tlim, a0 * t_l + a1 * t_r + a2 * t_rr);
  const V3 u_lq = a0 * u_r + a1 * u_l + a2 * u_ll;
  const V3 u_rq = a0 * u_l + a1 * u_r + a2 * u_rr;
  const double coef = std::max(double(alpha_geom(o, f)), P.lds_miles_filter) * sada;
  const double utmax = std::max(std::fabs(dot(u_lq, an)), std::fabs(dot(u_rq, an)));
  const double Ma = std::min(1.0, utmax / amin + 1e-4);
  const V3 u_lqp = u_lq + 0.5 * (1. - Ma) * (u_rq - u_lq);
  const V3 u_rqp = u_rq + 0.5 * (1. - Ma) * (u_lq - u_rq);
  roe_dissipation(F, pg_lq, u_lqp, t_lq, pg_rq, u_rqp, t_rq, P.Rtilde, P.gamma, P.Pambient, an, coef);
}

extern "C" int orc_residual(orc_ctx* o, double* src_out, fpsi_resid* norms) {
  const int64_t nc = o->nc, nf = o->nf;
  const fpsi_params& P = o->P;
  if (P.Minf < 0.5) return FPSI_E_UNSUPPORTED;
  if (P.viscous == 2 && P.turbulence == FPSI_TURB_SA) sa_tmu(o);
  o->have_sa = o->have_sa_dq = false;
  if (P.time_accurate && !o->have_levels) {  // first time step: Q(n-1) = Q(n) = Q
    o->Tn = o->Tm = o->T;
    o->pgn = o->pgm = o->pg;
    o->un = o->um = o->u;
    o->have_levels = true;
  }
  if (o->bcs_from_mdot) {  // massFlux_BC = mdot_BC / boundary_area (bcFixedMass.loci:227-230)
    std::vector<double> barea(o->bcs.size(), 0.0);
    for (int64_t f = 0; f < nf; ++f)
      if (o->cr[f] < 0) barea[-o->cr[f] - 1] += o->area[f];
    for (size_t b = 0; b < o->bcs.size(); ++b) {
      fpsi_bc& bc = o->bcs[b];
      const bool fm = bc.kind == FPSI_BC_FIXED_MASS_INFLOW || bc.kind == FPSI_BC_FIXED_MASS_OUTFLOW;
      if (fm && !(bc.mass_flux > 0) && barea[b] > 0) bc.mass_flux = bc.mdot / barea[b];
    }
    o->bcs_from_mdot = false;
  }
  o->qb.assign(nf * 5, 0);
  // area-weighted mean gauge pressure next to each condition (areaPressure /
  // boundary_area, bcOutflow.loci:178-198), in face order
  {
    std::vector<double> ap(o->bcs.size(), 0.0), aa(o->bcs.size(), 0.0);
    for (int64_t f = 0; f < nf; ++f)
      if (o->cr[f] < 0) {
        const int b = -o->cr[f] - 1;
        ap[b] += o->area[f] * o->pg[o->cl[f]];
        aa[b] += o->area[f];
      }
    o->bc_pmean.assign(o->bcs.size(), 0.0);
    for (size_t b = 0; b < o->bcs.size(); ++b) o->bc_pmean[b] = aa[b] > 0 ? ap[b] / aa[b] : 0.0;
  }
  o->bc_err = 0;
  for (int64_t f = 0; f < nf; ++f)
    if (o->cr[f] < 0) o->bc_err |= bc_face_state(o, f, &o->qb[5 * f]);
  gradients_and_limiters(o);
  const bool kec = P.flux == FPSI_FLUX_KEC || P.flux == FPSI_FLUX_SSF;
  std::vector<double> adiss;
  if (kec) alpha_diss(o, adiss);
  o->F.assign(nf * 5, 0);
  o->maxev.assign(nf, 0);
#pragma omp parallel for schedule(static)
  for (int64_t f = 0; f < nf; ++f) {
    double qL[5], qR[5];
    face_states(o, f, qL, qR);
    V3 n = v3(&o->an[3 * f]);
    if (bc_kind_of(o, f) == FPSI_BC_VISCOUS_WALL) {
      // wall iflux: pressure only, cell-centre pressure (bcViscousWall.loci:220-230)
      const double p = o->qb[5 * f + 4];
      const V3 a = n * o->area[f];
      double* F = &o->F[5 * f];
      F[0] = 0, F[1] = p * a.x, F[2] = p * a.y, F[3] = p * a.z, F[4] = 0;
    } else if (bc_kind_of(o, f) >= FPSI_BC_ISENTROPIC_INFLOW) {
      // analytic flux of the boundary state (bcIsentropic.loci:162-167,
      // bcFixedMass.loci:155-160, bcFixedMassOutflow.loci:152-157)
      const double* b = &o->qb[5 * f];
      state_flux(&o->F[5 * f], b[4], b[0], mk(b[1], b[2], b[3]), n, o->area[f], P.Pambient,
                 P.Rtilde, P.gamma);
    } else if (kec && o->cr[f] >= 0) {
      if (P.flux == FPSI_FLUX_KEC)
        kec_iflux(o, f, qL, qR, adiss, &o->F[5 * f]);
      else
        ssf_iflux(o, f, qL, qR, adiss, &o->F[5 * f]);
    } else {
      // boundary faces of the KEC scheme: inviscidRiemannFlux (inviscidFlux.h:82-90)
      riemann_flux(kec ? FPSI_FLUX_HLLC : P.flux, &o->F[5 * f], qL[4], qL[0],
                   mk(qL[1], qL[2], qL[3]), qR[4], qR[0], mk(qR[1], qR[2], qR[3]), n, o->area[f],
                   P.Pambient, P.Rtilde, P.gamma, 0.0, 1.0);
    }
    if (P.viscous) {
      // src[cl] += vflux, src[cr] -= vflux (fluxViscous.loci:299-310)
      const VFace v = viscous_face(o, f);
      for (int k = 0; k < 4; ++k) o->F[5 * f + 1 + k] -= v.vf[k];
    }
    // maxev_f, solverSetup.loci:81-105 (eta == 1)
    double ql[5], qr[5];
    cell_q(o, o->cl[f], ql);
    if (o->cr[f] >= 0)
      cell_q(o, o->cr[f], qr);
    else
      for (int k = 0; k < 5; ++k) qr[k] = o->qb[5 * f + k];
    const double eta = 1.0, EP = eta + 1., EM = eta - 1.;
    double utl = ql[1] * n.x + ql[2] * n.y + ql[3] * n.z;
    double utr = qr[1] * n.x + qr[2] * n.y + qr[3] * n.z;
    double al = std::sqrt(P.gamma * P.Rtilde * ql[0]);
    double ar = std::sqrt(P.gamma * P.Rtilde * qr[0]);
    double sl = std::sqrt(utl * utl * EM * EM + 4. * eta * al * al);
    double sr = std::sqrt(utr * utr * EM * EM + 4. * eta * ar * ar);
    double ml = 0.5 * std::max(std::fabs(utl * EP - sl), std::fabs(utl * EP + sl));
    double mr = 0.5 * std::max(std::fabs(utr * EP - sr), std::fabs(utr * EP + sr));
    o->maxev[f] = (o->cr[f] >= 0) ? std::max(ml, mr) : mr;
  }
  // scatter in face order: src[cl] -= F, src[cr] += F (fluxInviscid.loci:1253-1268),
  // done as a per-cell gather over the cell's faces in increasing face order.
  o->src.assign(nc * 5, 0);
  o->dtau.assign(nc, 0);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < nc; ++c) {
    // merge upper, lower, boundary lists by face index
    int64_t iu = o->up_off[c], il = o->lo_off[c], ib = o->bd_off[c];
    double s[5] = {0, 0, 0, 0, 0};
    double meva = 0;
    while (true) {
      int64_t fu = iu < o->up_off[c + 1] ? o->up[iu] : INT64_MAX;
      int64_t fl = il < o->lo_off[c + 1] ? o->lo[il] : INT64_MAX;
      int64_t fb = ib < o->bd_off[c + 1] ? o->bd[ib] : INT64_MAX;
      int64_t f = std::min(fu, std::min(fl, fb));
      if (f == INT64_MAX) break;
      if (f == fl) {
        for (int k = 0; k < 5; ++k) s[k] += o->F[5 * f + k];
        ++il;
      } else {
        for (int k = 0; k < 5; ++k) s[k] -= o->F[5 * f + k];
        if (f == fu)
          ++iu;
        else
          ++ib;
      }
    }
    // cflpdt (solverSetup.loci:107-119): lower, upper, boundary order
    for (int64_t k = o->lo_off[c]; k < o->lo_off[c + 1]; ++k)
      meva += o->maxev[o->lo[k]] * o->area[o->lo[k]];
    for (int64_t k = o->up_off[c]; k < o->up_off[c + 1]; ++k)
      meva += o->maxev[o->up[k]] * o->area[o->up[k]];
    for (int64_t k = o->bd_off[c]; k < o->bd_off[c + 1]; ++k)
      meva += o->maxev[o->bd[k]] * o->area[o->bd[k]];
    for (int k = 0; k < 5; ++k) o->src[5 * c + k] = s[k];
    double cflpdt = 0.5 * meva / o->vol[c];
    // dtcfl + dtau (solverTimestep.loci:289-329), eta == 1
    double dt = P.dtmax;
    if (P.cflmax > 0) dt = std::min(dt, P.cflmax / cflpdt);
    const double rvol = 1. / o->vol[c];
    const double p = o->pg[c] + P.Pambient, T = o->T[c], Rt = P.Rtilde;
    const double rP = 1. / (Rt * T);
    const double rho = (o->pg[c] + P.Pambient) * rP;
    const double rT = -rho / T, g = P.gamma;
    V3 U = v3(&o->u[3 * c]);
    const double q = 0.5 * dot(U, U);
    const double fT = rT * q, fP = (1. / (g - 1) + rP * q);
    const double reta = 1.0, a2 = g * Rt * T;
    const double pterm = (1. - reta) * (g - 1.) / a2;
    const double cterm = fP * rT * reta - fT * rP * reta;
    const double q2 = 2. * q;
    const double dsu = s[1] * U.x + s[2] * U.y + s[3] * U.z;
    const double dtemp = rvol * (s[0] * (fP * rT * reta + fT * pterm) +
                                 (dsu - s[4] - q2 * s[0]) * (rT * (pterm + rP * reta))) /
                         (cterm * rT);
    dt = std::min(dt, P.urelax * T / (std::fabs(dtemp) + 1e-30));
    const double dp = rvol * (rT * (q2 * s[0] - dsu + s[4]) - fT * s[0]);
    dt = std::min(dt, P.urelax * p / (std::fabs(dp) + 1e-30));
    o->dtau[c] = dt;
    if (P.time_accurate) {
      // rhs of the BDF2 Newton iteration (solverTimestep.loci:397-428)
      const double Pa = P.Pambient;
      const double rhon = (o->pgn[c] + Pa) / (Rt * o->Tn[c]);
      const double rhonm1 = (o->pgm[c] + Pa) / (Rt * o->Tm[c]);
      const double rhonp1 = (o->pg[c] + Pa) / (Rt * o->T[c]);
      const double rdtvol = o->vol[c] / P.dtmax;
      const double w = 0.5, w1 = (1.0 + w) * rdtvol, w2 = w * rdtvol;
      double* r = &o->src[5 * c];
      r[0] = (r[0] - w1 * (rhonp1 - rhon) + w2 * (rhon - rhonm1));
      const V3 Un = v3(&o->un[3 * c]), Um = v3(&o->um[3 * c]);
      const V3 runp1 = rhonp1 * U, run = rhon * Un, runm1 = rhonm1 * Um;
      r[1] = (r[1] - w1 * (runp1.x - run.x) + w2 * (run.x - runm1.x));
      r[2] = (r[2] - w1 * (runp1.y - run.y) + w2 * (run.y - runm1.y));
      r[3] = (r[3] - w1 * (runp1.z - run.z) + w2 * (run.z - runm1.z));
      const double re0np1 = rhonp1 * (Rt * o->T[c] / (g - 1.) + .5 * dot(U, U));
      const double re0n = rhon * (Rt * o->Tn[c] / (g - 1.) + .5 * dot(Un, Un));
      const double re0nm1 = rhonm1 * (Rt * o->Tm[c] / (g - 1.) + .5 * dot(Um, Um));
      r[4] = (r[4] - w1 * (re0np1 - re0n) + w2 * (re0n - re0nm1));
    }
  }
  // residual norms, solverResidual.loci:74-112 joined in cell order
  fpsi_resid r;
  std::memset(&r, 0, sizeof(r));
  double rt = 0, et = 0, mt = 0;
  for (int64_t c = 0; c < nc; ++c) {
    const double* s = &o->src[5 * c];
    double rvol = 1. / o->vol[c];
    double w = o->vol[c] / o->vol_tot;
    double a0 = rvol * s[0];
    rt += w * (a0 * a0);
    double mm = 0, mmax = 0;
    for (int i = 0; i < 3; ++i) {
      double a = rvol * s[1 + i];
      if (std::fabs(mmax) < std::fabs(a)) mmax = a;
      mm += a * a;
    }
    mt += mm * (w / 3.0);
    double a4 = rvol * s[4];
    et += w * (a4 * a4);
    if (std::fabs(r.rtmax) < std::fabs(a0)) {
      r.rtmax = a0;
      for (int i = 0; i < 3; ++i) r.ccmaxr_center[i] = o->cc[3 * c + i];
    }
    if (std::fabs(r.etmax) < std::fabs(a4)) {
      r.etmax = a4;
      for (int i = 0; i < 3; ++i) r.ccmaxe_center[i] = o->cc[3 * c + i];
    }
    if (std::fabs(r.mtmax) < std::fabs(mmax)) r.mtmax = mmax;
  }
  r.rtrms = std::sqrt(rt);
  r.etrms = std::sqrt(et);
  r.mtrms = std::sqrt(mt);
  o->have_resid = true;
  o->have_asm = false;
  if (src_out) std::memcpy(src_out, o->src.data(), sizeof(double) * nc * 5);
  r.bcErrorCode = o->bc_err;
  if (norms) *norms = r;
  if (r.rtrms != r.rtrms || r.etrms != r.etrms || r.mtrms != r.mtrms) return FPSI_E_NAN;
  return FPSI_OK;
}

extern "C" int orc_get_reconstruction(orc_ctx* o, double* grad, double* limiter) {
  if (!o->have_resid) return FPSI_E_STATE;
  if (grad) std::memcpy(grad, o->grad.data(), sizeof(double) * o->nc * 15);
  if (limiter) std::memcpy(limiter, o->phi.data(), sizeof(double) * o->nc * 5);
  return FPSI_OK;
}
extern "C" int orc_get_dtau(orc_ctx* o, double* dtau) {
  if (!o->have_resid) return FPSI_E_STATE;
  std::memcpy(dtau, o->dtau.data(), sizeof(double) * o->nc);
  return FPSI_OK;
}

// Jacobians (fluxInviscid.loci:1190-1221, BC srcJ e.g. bcInflow.loci:357-375),
// srcJ sum (solverLinearSystem.loci:106-121), steady fluid_D (:176-224),
// fluid_B (:45-55) and the LU (linearSolverSGS.loci:43-50).
template <class TB>
static int assemble_t(orc_ctx* o, std::vector<TB>& fjp, std::vector<TB>& fjm,
                      std::vector<TB>& D, std::vector<TB>& LU, std::vector<TB>& B) {
  const int64_t nc = o->nc, nf = o->nf;
  const fpsi_params& P = o->P;
  fjp.assign(nf * 25, TB(0));
  fjm.assign(nf * 25, TB(0));
#pragma omp parallel for schedule(static)
  for (int64_t f = 0; f < nf; ++f) {
    double qL[5], qR[5];
    face_states(o, f, qL, qR);
    V3 n = v3(&o->an[3 * f]);
    if (bc_kind_of(o, f) == FPSI_BC_VISCOUS_WALL) {
      // srcJ -= d(wall pressure flux)/dq (bcViscousWall.loci:232-240), u_f.n = 0
      TB* J = &fjp[25 * f];
      J[9] = TB(n.x * o->area[f]), J[14] = TB(n.y * o->area[f]), J[19] = TB(n.z * o->area[f]);
    } else if (bc_kind_of(o, f) == FPSI_BC_ISENTROPIC_INFLOW ||
               bc_kind_of(o, f) == FPSI_BC_FIXED_MASS_INFLOW) {
      // one-sided differences of the boundary flux in the cell-centre state
      // (bcIsentropic.loci:196-239, bcFixedMass.loci:163-224)
      const fpsi_bc& bc = o->bcs[-o->cr[f] - 1];
      const int c = o->cl[f];
      double vals[5] = {o->T[c], o->u[3 * c], o->u[3 * c + 1], o->u[3 * c + 2], o->pg[c]};
      auto bflux = [&](double F[5]) {
        double pgb, Tb;
        V3 ub;
        const V3 ui = mk(vals[1], vals[2], vals[3]);
        if (bc.kind == FPSI_BC_ISENTROPIC_INFLOW) {
          double pb;
          isentropic_bc(pb, Tb, ub, bc.T, bc.pg + P.Pambient, P.gamma, P.Rtilde, ui, vals[0],
                        -1.0 * n);
          pgb = pb - P.Pambient;
        } else {
          fixed_mass_bc(ub, Tb, pgb, vals[4] + P.Pambient, vals[0], bc.mass_flux, -1.0 * n, n,
                        bc.T, P.Pambient, P.gamma, P.Rtilde);
        }
        state_flux(F, pgb, Tb, ub, n, o->area[f], P.Pambient, P.Rtilde, P.gamma);
      };
      double F[5], F2[5];
      bflux(F);
      const double eps = 1e-5, ai = std::sqrt(P.gamma * P.Rtilde * vals[0]);
      const double deltas[5] = {vals[0] * eps, ai * eps, ai * eps, ai * eps, ai * ai * eps};
      for (int j = 0; j < 5; ++j) {
        const double tmp = vals[j];
        vals[j] += deltas[j];
        bflux(F2);
        const double rh = 1. / (tmp - vals[j]);
        for (int i = 0; i < 5; ++i) fjp[25 * f + 5 * i + j] = TB((F[i] - F2[i]) * rh);
        vals[j] = tmp;
      }
    } else {
      roe_jacobian<TB>(&fjp[25 * f], qL[4], qL[0], mk(qL[1], qL[2], qL[3]), qR[4], qR[0],
                       mk(qR[1], qR[2], qR[3]), n, o->area[f], P.Pambient, P.Rtilde, P.gamma,
                       0.0, 1.0, 1);
    }
    if (o->cr[f] >= 0)
      roe_jacobian<TB>(&fjm[25 * f], qL[4], qL[0], mk(qL[1], qL[2], qL[3]), qR[4], qR[0],
                       mk(qR[1], qR[2], qR[3]), n, o->area[f], P.Pambient, P.Rtilde, P.gamma,
                       0.0, 1.0, -1);
    if (P.viscous) {
      const VFace v = viscous_face(o, f);
      add_visc_jac<TB>(&fjp[25 * f], v, n, o->area[f], +1.0);
      if (o->cr[f] >= 0) add_visc_jac<TB>(&fjm[25 * f], v, n, o->area[f], -1.0);
    }
  }
  D.assign(nc * 25, TB(0));
  LU.assign(nc * 25, TB(0));
  B.assign(nc * 5, TB(0));
  o->piv.assign(nc * 5, 0);
  int bad = 0;
#pragma omp parallel for schedule(static) reduction(+ : bad)
  for (int64_t c = 0; c < nc; ++c) {
    TB sJ[25];
    for (int i = 0; i < 25; ++i) sJ[i] = TB(0);
    for (int64_t k = o->up_off[c]; k < o->up_off[c + 1]; ++k)
      for (int i = 0; i < 25; ++i) sJ[i] -= fjp[25 * o->up[k] + i];
    for (int64_t k = o->lo_off[c]; k < o->lo_off[c + 1]; ++k)
      for (int i = 0; i < 25; ++i) sJ[i] += fjm[25 * o->lo[k] + i];
    for (int64_t k = o->bd_off[c]; k < o->bd_off[c + 1]; ++k)
      for (int i = 0; i < 25; ++i) sJ[i] -= fjp[25 * o->bd[k] + i];
    TB* d = &D[25 * c];
    for (int i = 0; i < 25; ++i) d[i] = -sJ[i];
    // V / dtau (steady), 1.5 V / dtau (BDF2, solverLinearSystem.loci:389)
    const double coef = (o->P.time_accurate ? 1.5 : 1.0) * o->vol[c] / o->dtau[c];
    const double Rt = P.Rtilde, T = o->T[c];
    const double rP = 1. / (Rt * T);
    const double rho = (o->pg[c] + P.Pambient) * rP;
    const double rT = -rho / T;
    V3 U = v3(&o->u[3 * c]);
    const double q = 0.5 * dot(U, U);
    const double fT = rT * q, g = P.gamma, fP = (1. / (g - 1) + rP * q);
    const double reta = 1.0, a2 = g * Rt * T;
    const double pterm = (1. - reta) * (g - 1.) / a2;
#define DD(i, j) d[(i)*5 + (j)]
    DD(0, 0) += coef * rT;
    DD(1, 0) += coef * rT * U.x;
    DD(2, 0) += coef * rT * U.y;
    DD(3, 0) += coef * rT * U.z;
    DD(4, 0) += coef * fT;
    DD(0, 4) += coef * (pterm + rP * reta);
    DD(1, 4) += coef * (pterm + rP * reta) * U.x;
    DD(2, 4) += coef * (pterm + rP * reta) * U.y;
    DD(3, 4) += coef * (pterm + rP * reta) * U.z;
    DD(4, 4) += coef * (fT * pterm / rT + fP * reta);
    DD(1, 1) += coef * rho;
    DD(4, 1) += coef * rho * U.x;
    DD(2, 2) += coef * rho;
    DD(4, 2) += coef * rho * U.y;
    DD(3, 3) += coef * rho;
    DD(4, 3) += coef * rho * U.z;
#undef DD
    for (int i = 0; i < 25; ++i) LU[25 * c + i] = d[i];
    if (!lu5<TB>(&LU[25 * c], &o->piv[5 * c])) bad += 1;
    for (int k = 0; k < 5; ++k) B[5 * c + k] = TB(o->src[5 * c + k]);
  }
  o->have_asm = true;
  return bad ? FPSI_E_SINGULAR : FPSI_OK;
}

extern "C" int orc_assemble(orc_ctx* o) {
  if (!o->have_resid) return FPSI_E_STATE;
  if (o->P.precision == FPSI_PREC_FP64)
    return assemble_t<double>(o, o->fjp64, o->fjm64, o->D64, o->LU64, o->B64);
  return assemble_t<float>(o, o->fjp32, o->fjm32, o->D32, o->LU32, o->B32);
}

extern "C" int orc_get_blocks(orc_ctx* o, void* D, void* fjp, void* fjm, void* B) {
  if (!o->have_asm) return FPSI_E_STATE;
  const bool d64 = o->P.precision == FPSI_PREC_FP64;
  const size_t es = d64 ? 8 : 4;
  if (D) std::memcpy(D, d64 ? (void*)o->D64.data() : (void*)o->D32.data(), es * o->nc * 25);
  if (fjp) std::memcpy(fjp, d64 ? (void*)o->fjp64.data() : (void*)o->fjp32.data(), es * o->nf * 25);
  if (fjm) std::memcpy(fjm, d64 ? (void*)o->fjm64.data() : (void*)o->fjm32.data(), es * o->nf * 25);
  if (B) std::memcpy(B, d64 ? (void*)o->B64.data() : (void*)o->B32.data(), es * o->nc * 5);
  return FPSI_OK;
}

// One cell of a Gauss-Seidel sweep (gseidel_forward::calculate,
// linearSolverSGS.loci:186-207): t = -B + sum_upper U x(cr) + sum_lower L x(cl),
// x_c = D^-1 (-t), with U = fjm and L = -fjp (solverLinearSystem.loci:57-77).
template <class TB, class TX>
static inline void gs_cell(const orc_ctx* o, int64_t c, const std::vector<TB>& fjp,
                           const std::vector<TB>& fjm, const std::vector<TB>& LU,
                           const std::vector<TB>& B, TX* x) {
  TX t[5];
  for (int i = 0; i < 5; ++i) t[i] = -TX(B[5 * c + i]);
  for (int64_t k = o->up_off[c]; k < o->up_off[c + 1]; ++k) {
    int64_t f = o->up[k];
    const TB* U = &fjm[25 * f];
    const TX* xn = &x[5 * o->cr[f]];
    for (int i = 0; i < 5; ++i)
      for (int j = 0; j < 5; ++j) t[i] += TX(U[5 * i + j]) * xn[j];
  }
  for (int64_t k = o->lo_off[c]; k < o->lo_off[c + 1]; ++k) {
    int64_t f = o->lo[k];
    const TB* Lp = &fjp[25 * f];
    const TX* xn = &x[5 * o->cl[f]];
    for (int i = 0; i < 5; ++i)
      for (int j = 0; j < 5; ++j) t[i] += TX(-Lp[5 * i + j]) * xn[j];
  }
  TX v[5];
  for (int i = 0; i < 5; ++i) v[i] = -t[i];
  lu5_solve<TB, TX>(&LU[25 * c], &o->piv[5 * c], v, &x[5 * c]);
}

template <class TB, class TX>
static int solve_t(orc_ctx* o, const int32_t* colour, const double* x0,
                   const std::vector<TB>& fjp, const std::vector<TB>& fjm,
                   const std::vector<TB>& LU, const std::vector<TB>& B) {
  const int64_t nc = o->nc;
  std::vector<TX> x(nc * 5);
  const bool fsgs = o->P.solver == FPSI_SOLVER_FSGS;
  if (x0) {
    for (int64_t i = 0; i < nc * 5; ++i) x[i] = TX(x0[i]);
  } else if (fsgs) {
    // FSGS starts from zero (linearSolverFSGS.loci:1611)
    std::fill(x.begin(), x.end(), TX(0));
  } else {
    // block Jacobi start D x = B (linearSolverSGS.loci:57-69)
    for (int64_t c = 0; c < nc; ++c) {
      TX b[5];
      for (int i = 0; i < 5; ++i) b[i] = TX(B[5 * c + i]);
      lu5_solve<TB, TX>(&LU[25 * c], &o->piv[5 * c], b, &x[5 * c]);
    }
  }
  const int nit = o->P.gauss_seidel_iter;
  if (!colour) {
    // the sequential order: cell order for SGS; for FSGS the breadth-first
    // order of its single-cell lines (linearSolverFSGS.loci:808-845): from
    // the lowest unvisited cell, level by level, each level in increasing
    // cell number
    std::vector<int64_t> order(nc);
    if (fsgs) {
      std::vector<char> seen(nc, 0);
      int64_t cnt = 0, sp = 0;
      std::vector<int64_t> level, next;
      while (cnt < nc) {
        if (level.empty()) {
          while (seen[sp]) ++sp;
          level.push_back(sp);
          seen[sp] = 1;
        }
        next.clear();
        for (int64_t c : level) {
          order[cnt++] = c;
          auto visit = [&](int64_t n) {
            if (!seen[n]) seen[n] = 1, next.push_back(n);
          };
          for (int64_t k = o->lo_off[c]; k < o->lo_off[c + 1]; ++k) visit(o->cl[o->lo[k]]);
          for (int64_t k = o->up_off[c]; k < o->up_off[c + 1]; ++k) visit(o->cr[o->up[k]]);
        }
        std::sort(next.begin(), next.end());
        level.swap(next);
      }
    } else {
      for (int64_t c = 0; c < nc; ++c) order[c] = c;
    }
    for (int it = 0; it < nit; ++it) {
      for (int64_t i = 0; i < nc; ++i) gs_cell<TB, TX>(o, order[i], fjp, fjm, LU, B, x.data());
      for (int64_t i = nc - 1; i >= 0; --i) gs_cell<TB, TX>(o, order[i], fjp, fjm, LU, B, x.data());
    }
  } else {
    int ncol = 0;
    for (int64_t c = 0; c < nc; ++c) ncol = std::max(ncol, colour[c] + 1);
    std::vector<std::vector<int64_t>> byc(ncol);
    for (int64_t c = 0; c < nc; ++c) byc[colour[c]].push_back(c);
    for (int it = 0; it < nit; ++it) {
      for (int k = 0; k < ncol; ++k) {
        const auto& L = byc[k];
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < (int64_t)L.size(); ++i)
          gs_cell<TB, TX>(o, L[i], fjp, fjm, LU, B, x.data());
      }
      for (int k = ncol - 1; k >= 0; --k) {
        const auto& L = byc[k];
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < (int64_t)L.size(); ++i)
          gs_cell<TB, TX>(o, L[i], fjp, fjm, LU, B, x.data());
      }
    }
  }
  o->dq.resize(nc * 5);
  for (int64_t i = 0; i < nc * 5; ++i) o->dq[i] = double(x[i]);
  o->have_dq = true;
  return FPSI_OK;
}

extern "C" int orc_linear_solve(orc_ctx* o, const int32_t* colour, const double* x0,
                                double* dq, fpsi_lsinfo* info) {
  if (!o->have_asm) return FPSI_E_STATE;
  int rc;
  switch (o->P.precision) {
    case FPSI_PREC_FP64:
      rc = solve_t<double, double>(o, colour, x0, o->fjp64, o->fjm64, o->LU64, o->B64);
      break;
    case FPSI_PREC_MIXED:
      rc = solve_t<float, float>(o, colour, x0, o->fjp32, o->fjm32, o->LU32, o->B32);
      break;
    default:
      rc = solve_t<float, double>(o, colour, x0, o->fjp32, o->fjm32, o->LU32, o->B32);
  }
  if (dq) std::memcpy(dq, o->dq.data(), sizeof(double) * o->nc * 5);
  if (info) {
    info->iterations = o->P.gauss_seidel_iter;
    info->status = rc;
    info->resid0 = info->resid = 0;
  }
  return rc;
}

// ---------------------------------------------------------------------------
// Line SGS, linearSolverLSGS.loci:1465-1572 (line kernels) and :1692-1954
// (solve loop), over given lines.  Lines are processed in the given order,
// or, with line colours, colour by colour (forward 0..K-1, backward K-1..0).
// ---------------------------------------------------------------------------
template <class T>
static void lu_nopiv(T* A) {  // decompose_lu
  for (int k = 0; k < 5; ++k)
    for (int i = k + 1; i < 5; ++i) {
      A[5 * i + k] /= A[5 * k + k];
      for (int j = k + 1; j < 5; ++j) A[5 * i + j] -= A[5 * i + k] * A[5 * k + j];
    }
}
template <class T, class V>
static void lu_nopiv_solve(const T* A, V* y) {  // solve_lu
  for (int i = 1; i < 5; ++i)
    for (int j = 0; j < i; ++j) y[i] -= V(A[5 * i + j]) * y[j];
  for (int i = 4; i >= 0; --i) {
    for (int j = i + 1; j < 5; ++j) y[i] -= V(A[5 * i + j]) * y[j];
    y[i] /= V(A[5 * i + i]);
  }
}

template <class TB, class TD, class TX>
static int lsgs_t(orc_ctx* o, int64_t nlines, const int64_t* loff, const int32_t* lcells,
                  const int32_t* lcolour, const std::vector<TB>& fjp, const std::vector<TB>& fjm,
                  const std::vector<TB>& D, const std::vector<TB>& B, const double* x0,
                  fpsi_lsinfo* info) {
  const int64_t nc = o->nc;
  std::vector<int32_t> line_of(nc, -1), pos(nc, -1);
  for (int64_t l = 0; l < nlines; ++l)
    for (int64_t k = loff[l]; k < loff[l + 1]; ++k) {
      line_of[lcells[k]] = int32_t(l);
      pos[lcells[k]] = int32_t(k - loff[l]);
    }
  for (int64_t c = 0; c < nc; ++c)
    if (line_of[c] < 0) return FPSI_E_INVALID;
  // coupling block of row c to neighbour n through face f
  auto coupling = [&](int64_t c, int64_t f, TB* out) {
    if (o->cl[f] == c)
      for (int k = 0; k < 25; ++k) out[k] = fjm[25 * f + k];
    else
      for (int k = 0; k < 25; ++k) out[k] = -fjp[25 * f + k];
  };
  // line matrices: D' (TD), L (row p to p-1), U (row p to p+1), outer list
  std::vector<TD> Dp(nc * 25);
  std::vector<TB> Lb(nc * 25, TB(0)), Ub(nc * 25, TB(0));
  struct Outer {
    int64_t row, col;
    TB F[25];
  };
  std::vector<std::vector<Outer>> outer(nlines);
  auto nbr_of = [&](int64_t c, int64_t f) { return o->cl[f] == c ? o->cr[f] : o->cl[f]; };
  for (int64_t c = 0; c < nc; ++c) {
    for (int k = 0; k < 25; ++k) Dp[25 * c + k] = TD(D[25 * c + k]);
    const int64_t l = line_of[c];
    const int64_t p = pos[c];
    const int64_t len = loff[l + 1] - loff[l];
    const int64_t prv = p > 0 ? lcells[loff[l] + p - 1] : -1;
    const int64_t nxt = p + 1 < len ? lcells[loff[l] + p + 1] : -1;
    bool hp = false, hn = false;
    auto face = [&](int64_t f) {
      const int64_t n = nbr_of(c, f);
      TB blk[25];
      coupling(c, f, blk);
      if (n == prv && !hp) {
        hp = true;
        for (int k = 0; k < 25; ++k) Lb[25 * c + k] = blk[k];
      } else if (n == nxt && !hn) {
        hn = true;
        for (int k = 0; k < 25; ++k) Ub[25 * c + k] = blk[k];
      } else {
        Outer ou;
        ou.row = c, ou.col = n;
        for (int k = 0; k < 25; ++k) ou.F[k] = blk[k];
        outer[l].push_back(ou);
      }
    };
    for (int64_t k = o->up_off[c]; k < o->up_off[c + 1]; ++k) face(o->up[k]);
    for (int64_t k = o->lo_off[c]; k < o->lo_off[c + 1]; ++k) face(o->lo[k]);
  }
  // preprocessLine (:1465-1495): Schur products with real_fj intermediates
  for (int64_t l = 0; l < nlines; ++l) {
    const int64_t len = loff[l + 1] - loff[l];
    lu_nopiv<TD>(&Dp[25 * lcells[loff[l]]]);
    for (int64_t i = 1; i < len; ++i) {
      const int64_t cm = lcells[loff[l] + i - 1], cn = lcells[loff[l] + i];
      const TD* Dm = &Dp[25 * cm];
      TD* Dn = &Dp[25 * cn];
      const TB* Lm = &Lb[25 * cn];
      const TB* Um = &Ub[25 * cm];
      for (int j = 0; j < 5; ++j) {
        TD v[5];
        for (int k = 0; k < 5; ++k) v[k] = TD(Um[5 * k + j]);
        lu_nopiv_solve<TD, TD>(Dm, v);
        TB t[5], w[5];
        for (int k = 0; k < 5; ++k) t[k] = TB(v[k]), w[k] = TB(0);
        for (int k = 0; k < 5; ++k)
          for (int m = 0; m < 5; ++m) w[k] += Lm[5 * k + m] * t[m];
        for (int k = 0; k < 5; ++k) Dn[5 * k + j] -= TD(w[k]);
      }
      lu_nopiv<TD>(Dn);
    }
  }
  std::vector<TX> X(nc * 5, TX(0)), xt(nc * 5, TX(0));
  // lineSolve (:1523-1572) with right-hand side r (r = B - sum_outer F X)
  auto line_solve = [&](int64_t l, bool with_outer, bool save) {
    const int64_t len = loff[l + 1] - loff[l];
    std::vector<TX> r(len * 5);
    for (int64_t i = 0; i < len; ++i)
      for (int k = 0; k < 5; ++k) r[5 * i + k] = TX(B[5 * lcells[loff[l] + i] + k]);
    if (with_outer)
      for (const Outer& ou : outer[l]) {
        const int64_t i = pos[ou.row];
        for (int k = 0; k < 5; ++k)
          for (int j = 0; j < 5; ++j) r[5 * i + k] -= TX(ou.F[5 * k + j]) * X[5 * ou.col + j];
      }
    if (save)
      for (int64_t i = 0; i < len; ++i)
        for (int k = 0; k < 5; ++k) xt[5 * lcells[loff[l] + i] + k] = X[5 * lcells[loff[l] + i] + k];
    std::vector<TX> y(len * 5);
    for (int k = 0; k < 5; ++k) y[k] = r[k];
    for (int64_t i = 1; i < len; ++i) {
      TX v[5];
      for (int k = 0; k < 5; ++k) v[k] = y[5 * (i - 1) + k];
      lu_nopiv_solve<TD, TX>(&Dp[25 * lcells[loff[l] + i - 1]], v);
      const TB* Lm = &Lb[25 * lcells[loff[l] + i]];
      for (int k = 0; k < 5; ++k) {
        TX a = r[5 * i + k];
        for (int j = 0; j < 5; ++j) a -= TX(Lm[5 * k + j]) * v[j];
        y[5 * i + k] = a;
      }
    }
    for (int64_t i = len - 1; i >= 0; --i) {
      TX v[5];
      for (int k = 0; k < 5; ++k) v[k] = y[5 * i + k];
      if (i < len - 1) {
        const TB* Um = &Ub[25 * lcells[loff[l] + i]];
        const int64_t cn = lcells[loff[l] + i + 1];
        for (int k = 0; k < 5; ++k)
          for (int j = 0; j < 5; ++j) v[k] -= TX(Um[5 * k + j]) * X[5 * cn + j];
      }
      lu_nopiv_solve<TD, TX>(&Dp[25 * lcells[loff[l] + i]], v);
      for (int k = 0; k < 5; ++k) X[5 * lcells[loff[l] + i] + k] = v[k];
    }
  };
  if (x0) {
    for (int64_t i = 0; i < nc * 5; ++i) X[i] = TX(x0[i]);
  } else {
    for (int64_t l = 0; l < nlines; ++l) line_solve(l, false, false);  // (:1708-1728)
  }
  std::vector<int64_t> order;
  if (lcolour) {
    int ncol = 0;
    for (int64_t l = 0; l < nlines; ++l) ncol = std::max(ncol, lcolour[l] + 1);
    for (int k = 0; k < ncol; ++k)
      for (int64_t l = 0; l < nlines; ++l)
        if (lcolour[l] == k) order.push_back(l);
  } else {
    for (int64_t l = 0; l < nlines; ++l) order.push_back(l);
  }
  double w = o->P.lsgs_relaxation, zero = 1.0, resid = 0.0;
  int iter = 0;
  for (; iter < o->P.lsgs_max_iter;) {
    for (int64_t l : order) line_solve(l, true, false);
    for (auto it = order.rbegin(); it != order.rend(); ++it) line_solve(*it, true, true);
    double s = 0;
    for (int64_t i = 0; i < nc * 5; ++i) {
      X[i] = TX(w * double(X[i]) + (1. - w) * double(xt[i]));
      const double r = double(X[i]) - double(xt[i]);
      s += r * r;
    }
    resid = std::sqrt(s);
    if (iter == 0) zero = std::max(resid, 1e-16);
    const double rel = resid / zero;
    if (rel > 1.0) w *= 1. / rel;
    ++iter;
    if (resid < o->P.lsgs_abs_tol || rel < o->P.lsgs_rel_tol) break;
  }
  o->dq.resize(nc * 5);
  for (int64_t i = 0; i < nc * 5; ++i) o->dq[i] = double(X[i]);
  o->have_dq = true;
  if (info) {
    info->iterations = iter;
    info->status = FPSI_OK;
    info->resid0 = zero;
    info->resid = resid;
  }
  return FPSI_OK;
}

extern "C" int orc_lsgs_solve(orc_ctx* o, int64_t nlines, const int64_t* line_off,
                              const int32_t* line_cells, const int32_t* line_colour,
                              const double* x0, double* dq, fpsi_lsinfo* info) {
  if (!o->have_asm) return FPSI_E_STATE;
  int rc;
  switch (o->P.precision) {
    case FPSI_PREC_FP64:
      rc = lsgs_t<double, double, double>(o, nlines, line_off, line_cells, line_colour, o->fjp64,
                                          o->fjm64, o->D64, o->B64, x0, info);
      break;
    case FPSI_PREC_MIXED:
      rc = lsgs_t<float, float, float>(o, nlines, line_off, line_cells, line_colour, o->fjp32,
                                       o->fjm32, o->D32, o->B32, x0, info);
      break;
    default:
      rc = lsgs_t<float, double, double>(o, nlines, line_off, line_cells, line_colour, o->fjp32,
                                         o->fjm32, o->D32, o->B32, x0, info);
  }
  if (!rc && dq) std::memcpy(dq, o->dq.data(), sizeof(double) * o->nc * 5);
  return rc;
}

// ||B - A dq|| with A from the unfactored blocks
template <class TB>
static void linres_t(orc_ctx* o, const std::vector<TB>& fjp, const std::vector<TB>& fjm,
                     const std::vector<TB>& D, const std::vector<TB>& B, double* nb, double* nr) {
  double sb = 0, sr = 0;
  for (int64_t c = 0; c < o->nc; ++c) {
    double r[5];
    for (int i = 0; i < 5; ++i) r[i] = double(B[5 * c + i]);
    const double* x = &o->dq[5 * c];
    for (int i = 0; i < 5; ++i)
      for (int j = 0; j < 5; ++j) r[i] -= double(D[25 * c + 5 * i + j]) * x[j];
    for (int64_t k = o->up_off[c]; k < o->up_off[c + 1]; ++k) {
      int64_t f = o->up[k];
      const double* xn = &o->dq[5 * o->cr[f]];
      for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5; ++j) r[i] -= double(fjm[25 * f + 5 * i + j]) * xn[j];
    }
    for (int64_t k = o->lo_off[c]; k < o->lo_off[c + 1]; ++k) {
      int64_t f = o->lo[k];
      const double* xn = &o->dq[5 * o->cl[f]];
      for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5; ++j) r[i] += double(fjp[25 * f + 5 * i + j]) * xn[j];
    }
    for (int i = 0; i < 5; ++i) {
      sb += double(B[5 * c + i]) * double(B[5 * c + i]);
      sr += r[i] * r[i];
    }
  }
  *nb = std::sqrt(sb);
  *nr = std::sqrt(sr);
}

extern "C" int orc_linear_residual(orc_ctx* o, double* norm_b, double* norm_r) {
  if (!o->have_dq) return FPSI_E_STATE;
  double nb, nr;
  if (o->P.precision == FPSI_PREC_FP64)
    linres_t<double>(o, o->fjp64, o->fjm64, o->D64, o->B64, &nb, &nr);
  else
    linres_t<float>(o, o->fjp32, o->fjm32, o->D32, o->B32, &nb, &nr);
  if (norm_b) *norm_b = nb;
  if (norm_r) *norm_r = nr;
  return FPSI_OK;
}

// Steady Newton update with positivity clip, solverNewton.loci:62-78.
extern "C" int orc_update(orc_ctx* o, double* min_alpha) {
  if (!o->have_dq) return FPSI_E_STATE;
  double amin = 1.0;
  for (int64_t c = 0; c < o->nc; ++c) {
    const double* d = &o->dq[5 * c];
    double alpha = 1.0;
    if (o->P.time_accurate) {  // BDF2, solverNewton.loci:163-182
      const double relax = 0.75;
      alpha = std::min(alpha, relax * (o->pg[c] + o->P.Pambient) / std::max(std::fabs(d[4]), 1e-30));
      alpha = std::min(alpha, relax * o->T[c] / std::max(std::fabs(d[0]), 1e-30));
    } else {
      alpha = std::min(alpha, 0.9 * o->T[c] / (std::fabs(d[0]) + 1e-30));
      alpha = std::min(alpha, 0.9 * (o->pg[c] + o->P.Pambient) / (std::fabs(d[4]) + 1e-30));
    }
    o->T[c] += alpha * d[0];
    o->pg[c] += alpha * d[4];
    for (int i = 0; i < 3; ++i) o->u[3 * c + i] += alpha * d[1 + i];
    amin = std::min(amin, alpha);
  }
  if (min_alpha) *min_alpha = amin;
  o->have_resid = o->have_asm = o->have_dq = false;
  return FPSI_OK;
}

extern "C" int orc_sa_residual(orc_ctx* o, double* src_out);
extern "C" int orc_sa_solve(orc_ctx* o, const int32_t* colour, double* dq);
extern "C" int orc_sa_update(orc_ctx* o);

// one implicit step; with the SA model the nu~ system is built from the same
// residual state and its update applied after the mean flow's
extern "C" int orc_newton_step(orc_ctx* o, const int32_t* colour, fpsi_stepinfo* info) {
  fpsi_stepinfo si;
  std::memset(&si, 0, sizeof(si));
  int rc = orc_residual(o, nullptr, &si.resid);
  if (rc) return rc;
  si.dtau_min = *std::min_element(o->dtau.begin(), o->dtau.end());
  si.dtau_max = *std::max_element(o->dtau.begin(), o->dtau.end());
  const bool sa = o->P.viscous == 2 && o->P.turbulence == FPSI_TURB_SA;
  if (sa) {
    if ((rc = orc_sa_residual(o, nullptr))) return rc;
    if ((rc = orc_sa_solve(o, colour, nullptr))) return rc;
  }
  rc = orc_assemble(o);
  if (rc) return rc;
  rc = orc_linear_solve(o, colour, nullptr, nullptr, &si.ls);
  if (rc) return rc;
  rc = orc_update(o, &si.min_alpha);
  if (!rc && sa) rc = orc_sa_update(o);
  if (info) *info = si;
  return rc;
}

// One BDF2 time step (timeStepAccurate, timeStepSchemeBDF2): newton_iters
// Newton iterations (solverNewton.loci:200-219), then the time levels move
// on (the in-place copy of :190-198).
extern "C" int orc_time_step(orc_ctx* o, const int32_t* colour, fpsi_resid* norms) {
  if (!o->P.time_accurate) return FPSI_E_STATE;
  for (int it = 0; it < o->P.newton_iters; ++it) {
    fpsi_stepinfo si;
    const int rc = orc_newton_step(o, colour, &si);
    if (norms) norms[it] = si.resid;
    if (rc) return rc;
  }
  o->Tm = o->Tn, o->pgm = o->pgn, o->um = o->un;
  o->Tn = o->T, o->pgn = o->pg, o->un = o->u;
  return FPSI_OK;
}

// ---------------------------------------------------------------------------
// Batched face functions
// ---------------------------------------------------------------------------
extern "C" int orc_face_flux(int32_t kind, int64_t n, const double* qL, const double* qR,
                             const double* an, const double* area, double pamb, double Rt,
                             double gamma, double us_n, double eta, double* flux) {
  for (int64_t i = 0; i < n; ++i) {
    const double* l = qL + 5 * i;
    const double* r = qR + 5 * i;
    riemann_flux(kind, flux + 5 * i, l[0], l[1], mk(l[2], l[3], l[4]), r[0], r[1],
                 mk(r[2], r[3], r[4]), v3(an + 3 * i), area[i], pamb, Rt, gamma, us_n, eta);
  }
  return FPSI_OK;
}

extern "C" int orc_face_jacobian(int64_t n, const double* qL, const double* qR,
                                 const double* an, const double* area, double pamb, double Rt,
                                 double gamma, double us_n, double eta, int32_t dir,
                                 int32_t as_double, void* out) {
  for (int64_t i = 0; i < n; ++i) {
    const double* l = qL + 5 * i;
    const double* r = qR + 5 * i;
    if (as_double) {
      double* J = (double*)out + 25 * i;
      for (int k = 0; k < 25; ++k) J[k] = 0;
      roe_jacobian<double>(J, l[0], l[1], mk(l[2], l[3], l[4]), r[0], r[1],
                           mk(r[2], r[3], r[4]), v3(an + 3 * i), area[i], pamb, Rt, gamma,
                           us_n, eta, dir);
    } else {
      float* J = (float*)out + 25 * i;
      for (int k = 0; k < 25; ++k) J[k] = 0;
      roe_jacobian<float>(J, l[0], l[1], mk(l[2], l[3], l[4]), r[0], r[1],
                          mk(r[2], r[3], r[4]), v3(an + 3 * i), area[i], pamb, Rt, gamma, us_n,
                          eta, dir);
    }
  }
  return FPSI_OK;
}

extern "C" int orc_cv_state(int32_t outflow, int64_t n, const double* qi, const double* q0,
                            const double* an, double us_n, double pamb, double gamma, double Rt,
                            double beta, double* out) {
  for (int64_t i = 0; i < n; ++i) {
    const double* a = qi + 5 * i;
    const double* b = q0 + 5 * i;
    double pgb, Tb;
    V3 ub;
    if (outflow)
      cv_outflow(pgb, Tb, ub, a[0], a[1], mk(a[2], a[3], a[4]), b[0], b[1], mk(b[2], b[3], b[4]),
                 v3(an + 3 * i), us_n, pamb, gamma, Rt, beta);
    else
      cv_inflow(pgb, Tb, ub, a[0], a[1], mk(a[2], a[3], a[4]), b[0], b[1], mk(b[2], b[3], b[4]),
                v3(an + 3 * i), us_n, pamb, gamma, Rt, beta);
    double* o = out + 5 * i;
    o[0] = pgb, o[1] = Tb, o[2] = ub.x, o[3] = ub.y, o[4] = ub.z;
  }
  return FPSI_OK;
}

// ---------------------------------------------------------------------------
// Spalart-Allmaras nu~ transport (turbulence/SA/SA_turb.loci, baseline model,
// standard production) in the reference's scalar transport
// (solverScalarTransport.loci), steady pseudo time, one Newton iteration per
// step.
// ---------------------------------------------------------------------------
namespace {
struct SAConst {  // Spa_All_param, SA_param.h:28-40
  double cb1 = 0.1355, k = 0.41, cv1 = 7.1, cb2 = 0.622, cw2 = 0.3, cw3 = 2.0, sigma = 2. / 3.;
};
constexpr double SA_FACTORX = 2, SA_FACTORY = .5;  // SA_turb.loci:426-427
}  // namespace

// Nearest no-slip wall face by its edge-weighted centre from each cell's
// area-weighted face-centre average (find_mind, gridSetup.loci:418-640; ties:
// lowest face), then |(x_f - x_c).n| with the finite-volume centres
// (dist_noslip, solverTurbulence.loci:133-137).  No walls: 1e30.
static void wall_distance(orc_ctx* o, const fpsi_mesh* m) {
  const int64_t nc = o->nc, nf = o->nf;
  o->wdist.assign(nc, 1e30);
  std::vector<int64_t> walls;
  for (int64_t f = 0; f < nf; ++f)
    if (o->cr[f] < 0 && o->bcs[-o->cr[f] - 1].kind == FPSI_BC_VISCOUS_WALL) walls.push_back(f);
  if (walls.empty()) return;
  std::vector<double> fce(nf * 3), fa(nf);
  for (int64_t f = 0; f < nf; ++f) {
    const int64_t a = m->face_off[f], b = m->face_off[f + 1];
    const int n = int(b - a);
    V3 ns = mk(0, 0, 0);
    double ls = 0;
    for (int i = 0; i < n; ++i) {
      V3 p1 = v3(&m->xyz[3 * int64_t(m->face_nodes[a + i])]);
      V3 p2 = v3(&m->xyz[3 * int64_t(m->face_nodes[a + (i + 1) % n])]);
      const double len = norm(p1 - p2);
      ns = ns + len * (0.5 * (p1 + p2));
      ls += len;
    }
    V3 c = (1.0 / ls) * ns;
    V3 s = mk(0, 0, 0);
    for (int i = 0; i < n; ++i) {
      V3 p1 = v3(&m->xyz[3 * int64_t(m->face_nodes[a + i])]);
      V3 p2 = v3(&m->xyz[3 * int64_t(m->face_nodes[a + (i + 1) % n])]);
      s = s + cross(p1 - c, p2 - c);
    }
    fce[3 * f] = c.x, fce[3 * f + 1] = c.y, fce[3 * f + 2] = c.z;
    fa[f] = 0.5 * norm(s);
  }
  std::vector<double> csum(nc * 3, 0), asum(nc, 0);
  for (int64_t f = 0; f < nf; ++f) {
    for (int side = 0; side < 2; ++side) {
      const int64_t c = side ? o->cr[f] : o->cl[f];
      if (c < 0) continue;
      for (int k = 0; k < 3; ++k) csum[3 * c + k] += fce[3 * f + k] * fa[f];
      asum[c] += fa[f];
    }
  }
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < nc; ++c) {
    const V3 p = (1.0 / asum[c]) * v3(&csum[3 * c]);
    double best = 1e300;
    int64_t bf = -1;
    for (int64_t w : walls) {
      const V3 d = v3(&fce[3 * w]) - p;
      const double d2 = dot(d, d);
      if (d2 < best) best = d2, bf = w;
    }
    const V3 dist = v3(&o->fc[3 * bf]) - v3(&o->cc[3 * c]);
    o->wdist[c] = std::fabs(dot(dist, v3(&o->an[3 * bf])));
  }
}

static inline double sa_rho(const orc_ctx* o, int64_t c) {
  return (o->pg[c] + o->P.Pambient) / (o->P.Rtilde * o->T[c]);
}
static inline double sa_mu(const orc_ctx* o, int64_t c) {
  return suth(o->T[c], o->P.mu_a1, o->P.mu_a2, o->P.mu_a3);
}

// tmu = nu~ f_v1 rho (SA_turb.loci:91-107)
static void sa_tmu(orc_ctx* o) {
  const SAConst S;
  for (int64_t c = 0; c < o->nc; ++c) {
    const double rho = sa_rho(o, c), mu = sa_mu(o, c);
    const double x = rho * o->nut[c] / mu;
    const double fv1 = std::pow(x, 3) / (std::pow(x, 3) + std::pow(S.cv1, 3));
    o->tmu[c] = o->nut[c] * fv1 * rho;
  }
}

// nu~ on a boundary face: 0 on no-slip walls (:181-183), the inside value
// where the face velocity leaves or on symmetry planes, else the boundary's
// nu_t (solverScalarTransport.loci:423-466, SA_turb.loci:167-179)
static double sa_face_bc(const orc_ctx* o, int64_t f) {
  const fpsi_bc& bc = o->bcs[-o->cr[f] - 1];
  const int64_t a = o->cl[f];
  if (bc.kind == FPSI_BC_VISCOUS_WALL) return 0.0;
  if (bc.kind == FPSI_BC_REFLECTING) return o->nut[a];
  const double* qf = &o->qb[5 * f];
  const double uit = o->an[3 * f] * qf[1] + o->an[3 * f + 1] * qf[2] + o->an[3 * f + 2] * qf[3];
  if (uit >= -0.0) return o->nut[a];
  return bc.nu_t > 0 ? bc.nu_t : 5e-9;
}

extern "C" int orc_set_nutilde(orc_ctx* o, const double* nut) {
  std::memcpy(o->nut.data(), nut, sizeof(double) * o->nc);
  o->have_resid = o->have_asm = o->have_dq = o->have_sa = o->have_sa_dq = false;
  return FPSI_OK;
}
extern "C" int orc_get_nutilde(orc_ctx* o, double* nut) {
  std::memcpy(nut, o->nut.data(), sizeof(double) * o->nc);
  return FPSI_OK;
}
extern "C" int orc_get_eddy_viscosity(orc_ctx* o, double* tmu) {
  std::memcpy(tmu, o->tmu.data(), sizeof(double) * o->nc);
  return FPSI_OK;
}
extern "C" int orc_get_wall_distance(orc_ctx* o, double* d) {
  std::memcpy(d, o->wdist.data(), sizeof(double) * o->nc);
  return FPSI_OK;
}

// SA sources, convection, diffusion and their Jacobians into X_src, X_D,
// X_fjp, X_fjm (SA_turb.loci:85-476, solverScalarTransport.loci:457-700)
extern "C" int orc_sa_residual(orc_ctx* o, double* src_out) {
  if (!o->have_resid) return FPSI_E_STATE;
  const fpsi_params& P = o->P;
  if (!(P.viscous == 2 && P.turbulence == FPSI_TURB_SA)) return FPSI_E_STATE;
  const SAConst S;
  const int64_t nc = o->nc, nf = o->nf;
  // gradient and limiter of nu~, boundary values at the boundary faces
  std::vector<double> nub(nf, 0.0);
  for (int64_t f = 0; f < nf; ++f)
    if (o->cr[f] < 0) nub[f] = sa_face_bc(o, f);
  o->sa_grad.assign(nc * 3, 0);
  o->sa_phi.assign(nc, 1.0);
  const int lim = P.limiter;
  for (int64_t c = 0; c < nc; ++c) {
    const double xc = o->nut[c];
    double b[3] = {0, 0, 0}, xmax = xc, xmin = xc;
    auto nb = [&](V3 d, double xn) {
      const double dx = xn - xc;
      b[0] += d.x * dx, b[1] += d.y * dx, b[2] += d.z * dx;
      xmax = std::max(xmax, xn), xmin = std::min(xmin, xn);
    };
    for (int64_t k = o->up_off[c]; k < o->up_off[c + 1]; ++k) {
      const int64_t f = o->up[k];
      nb(v3(&o->rL[3 * f]) - v3(&o->rR[3 * f]), o->nut[o->cr[f]]);
    }
    for (int64_t k = o->lo_off[c]; k < o->lo_off[c + 1]; ++k) {
      const int64_t f = o->lo[k];
      nb(v3(&o->rR[3 * f]) - v3(&o->rL[3 * f]), o->nut[o->cl[f]]);
    }
    for (int64_t k = o->bd_off[c]; k < o->bd_off[c + 1]; ++k) {
      const int64_t f = o->bd[k];
      nb(v3(&o->rL[3 * f]), nub[f]);
    }
    const double* mi = &o->Minv[6 * c];
    double* g = &o->sa_grad[3 * c];
    g[0] = mi[0] * b[0] + mi[1] * b[1] + mi[2] * b[2];
    g[1] = mi[1] * b[0] + mi[3] * b[1] + mi[4] * b[2];
    g[2] = mi[2] * b[0] + mi[4] * b[1] + mi[5] * b[2];
    double ph = lim == FPSI_LIMITER_ZERO ? 0.0 : 1.0;
    if (lim == FPSI_LIMITER_VENKATAKRISHNAN || lim == FPSI_LIMITER_BARTH) {
      const double h = std::cbrt(o->vol[c]);
      const double kh = P.Kl * h, eps2 = kh * kh * kh;
      auto side = [&](V3 r) {
        const double d2 = g[0] * r.x + g[1] * r.y + g[2] * r.z;
        double p = 1.0;
        if (d2 != 0.0) {
          const double d1 = d2 > 0 ? xmax - xc : xmin - xc;
          if (lim == FPSI_LIMITER_BARTH) {
            p = std::min(1.0, d1 / d2);
          } else {
            const double num = (d1 * d1 + eps2) + 2.0 * d2 * d1;
            const double den = d1 * d1 + 2.0 * d2 * d2 + d1 * d2 + eps2;
            p = std::min(1.0, num / den);
          }
        }
        ph = std::min(ph, p);
      };
      for (int64_t k = o->up_off[c]; k < o->up_off[c + 1]; ++k) side(v3(&o->rL[3 * o->up[k]]));
      for (int64_t k = o->lo_off[c]; k < o->lo_off[c + 1]; ++k) side(v3(&o->rR[3 * o->lo[k]]));
      for (int64_t k = o->bd_off[c]; k < o->bd_off[c + 1]; ++k) side(v3(&o->rL[3 * o->bd[k]]));
    }
    o->sa_phi[c] = ph;
  }
  std::vector<double> rho(nc), mu(nc);
  for (int64_t c = 0; c < nc; ++c) rho[c] = sa_rho(o, c), mu[c] = sa_mu(o, c);
  // per-cell accumulators
  std::vector<double> src(nc, 0.0), srcJ(nc, 0.0), rhodot(nc, 0.0), divn(nc, 0.0);
  o->sa_fjp.assign(nf, 0.0);
  o->sa_fjm.assign(nf, 0.0);
  for (int64_t f = 0; f < nf; ++f) {
    const int64_t a = o->cl[f];
    const V3 n = v3(&o->an[3 * f]);
    const double A = o->area[f];
    const double mdot = o->F[5 * f];  // scalar_mdot_f = iflux[0]
    const double* ga = &o->sa_grad[3 * a];
    const V3 rl = v3(&o->rL[3 * f]);
    const double xl = o->nut[a] + o->sa_phi[a] * (ga[0] * rl.x + ga[1] * rl.y + ga[2] * rl.z);
    if (o->cr[f] >= 0) {
      const int64_t b = o->cr[f];
      const double* gb = &o->sa_grad[3 * b];
      const V3 rr = v3(&o->rR[3 * f]);
      const double xr = o->nut[b] + o->sa_phi[b] * (gb[0] * rr.x + gb[1] * rr.y + gb[2] * rr.z);
      const double vl = o->vol[a], vr = o->vol[b];
      const double nuf = (vr * o->nut[a] + vl * o->nut[b]) * (1.0 / (vr + vl));
      const double muf = (vl * mu[b] + vr * mu[a]) / (vl + vr);
      const double rhof = (1. / (vl + vr)) * (vl * rho[b] + vr * rho[a]);
      // face gradient: mean + correction along d = x_b - x_a
      const V3 d = rl - rr;
      const double d2 = dot(d, d);
      double gm[3];
      for (int k = 0; k < 3; ++k) gm[k] = 0.5 * (ga[k] + gb[k]);
      const double cc = ((o->nut[b] - o->nut[a]) - (gm[0] * d.x + gm[1] * d.y + gm[2] * d.z)) / d2;
      const V3 gf = mk(gm[0] + cc * d.x, gm[1] + cc * d.y, gm[2] + cc * d.z);
      const double divf = dot(gf, n) * A;
      double diff1 = dot(gf, n) * A;
      diff1 = (diff1 * (muf / rhof + (1. + S.cb2) * nuf)) / S.sigma;
      // convection (inviscid_fluxP(X,Zero))
      const double xv = mdot < 0.0 ? xr : xl;
      const double conv = mdot * std::max(xv, 0.0);
      src[a] -= conv, src[b] += conv;
      rhodot[a] -= mdot, rhodot[b] += mdot;
      src[a] += rho[a] * diff1, src[b] -= rho[b] * diff1;
      divn[a] += divf, divn[b] -= divf;
      // Jacobians
      double fjp = 0.0, fjm = 0.0;
      fjp += std::max(mdot, 0.0);
      fjm += std::min(mdot, 0.0);
      const double rbar = .5 * (rho[a] + rho[b]);
      const double C = (muf + (1. + S.cb2) * rbar * nuf) * A;
      const double dd = dot(d, n);  // (x_b - x_a).n
      fjp -= -C / (dd * S.sigma);
      fjm += -C / (dd * S.sigma);
      const double C2 = S.cb2 * A, d2s = S.sigma * dd;
      const double sU = -SA_FACTORX * (C2 / d2s) * rho[a] * o->nut[a];
      const double sL = -SA_FACTORX * (C2 / d2s) * rho[b] * o->nut[b];
      fjp += sL;
      fjm -= sU;
      srcJ[a] += SA_FACTORX * SA_FACTORY * (C2 / d2s) * rho[a] * o->nut[a];
      srcJ[b] += SA_FACTORX * SA_FACTORY * (C2 / d2s) * rho[b] * o->nut[b];
      // X_srcJ += -sum_upper fjp + sum_lower fjm, minus the L/U
      // non-conservative parts (SA_turb.loci:745-752)
      srcJ[a] -= fjp, srcJ[b] += fjm;
      srcJ[a] += sL, srcJ[b] += sU;
      o->sa_fjp[f] = fjp, o->sa_fjm[f] = fjm;
    } else {
      const int kind = o->bcs[-o->cr[f] - 1].kind;
      const double* qf = &o->qb[5 * f];
      const double nuf = nub[f];
      const double muf = suth(qf[0], P.mu_a1, P.mu_a2, P.mu_a3);
      const double rhof = (qf[4] + P.Pambient) / (P.Rtilde * qf[0]);  // solverEoS.loci:53-56
      const V3 r = rl;
      const double r2 = dot(r, r);
      const double cc = ((nuf - o->nut[a]) - (ga[0] * r.x + ga[1] * r.y + ga[2] * r.z)) / r2;
      const V3 gf = mk(ga[0] + cc * r.x, ga[1] + cc * r.y, ga[2] + cc * r.z);
      const double divf = dot(gf, n) * A;
      double diff1 = dot(gf, n) * A;
      diff1 = (diff1 * (muf / rhof + (1. + S.cb2) * nuf)) / S.sigma;
      const double xv = mdot < 0.0 ? nuf : xl;
      const double conv = mdot * std::max(xv, 0.0);
      src[a] -= conv;
      rhodot[a] -= mdot;
      src[a] += rho[a] * diff1;
      divn[a] += divf;
      srcJ[a] -= std::max(mdot, 0.0);
      if (kind != FPSI_BC_REFLECTING) {  // no_symmetry_BC
        const double C = (muf + (1. + S.cb2) * rhof * nuf) * A;
        const double db = dot(r, n);
        srcJ[a] += -C / (db * S.sigma);
        const double C2 = S.cb2 * A, d2s = S.sigma * db;
        srcJ[a] += SA_FACTORX * SA_FACTORY * (C2 / d2s) * rho[a] * o->nut[a];
      }
    }
  }
  // cell terms
  const double k2 = S.k * S.k;
  const double cw1 = (S.cb1) / (k2) + (1.0 + (S.cb2)) / (S.sigma);
  const double cw36 = std::pow(S.cw3, 6);
  const double cv13 = S.cv1 * S.cv1 * S.cv1;
  o->sa_src.assign(nc, 0.0);
  o->sa_D.assign(nc, 0.0);
  for (int64_t c = 0; c < nc; ++c) {
    const double nu = o->nut[c], r0 = rho[c], V = o->vol[c], y = o->wdist[c];
    const double* gu = &o->grad[15 * c + 3];  // rows u, v, w: d u_i / d x_j
    const double wx = gu[3 * 2 + 1] - gu[3 * 1 + 2];
    const double wy = gu[3 * 0 + 2] - gu[3 * 2 + 0];
    const double wz = gu[3 * 1 + 0] - gu[3 * 0 + 1];
    const double vort = std::sqrt(wx * wx + wy * wy + wz * wz);
    const double x = r0 * nu / mu[c];
    const double fv1 = std::pow(x, 3) / (std::pow(x, 3) + std::pow(S.cv1, 3));
    const double fv2 = 1.0 - (x / (1.0 + x * fv1));
    const double denom = k2 * y * y;
    double St = 0.0;
    St += vort;
    St += nu * fv2 / denom;
    const double Sl = std::max(St, 0.3 * vort);
    double rc;
    if (Sl < nu / (10 * denom))
      rc = 10;
    else
      rc = nu / (Sl * denom);
    const double r2 = rc * rc, r6 = r2 * r2 * r2;
    const double gc = rc + S.cw2 * (r6 - rc);
    const double g2 = gc * gc, g6 = g2 * g2 * g2;
    const double fw = gc * std::pow((1.0 + cw36) / (g6 + cw36), 1.0 / 6.0);
    double s = src[c];
    s += r0 * nu * Sl * S.cb1 * V;
    const double t = nu / y;
    s -= r0 * fw * cw1 * t * t * V;
    s += -r0 * nu * divn[c] * S.cb2 / S.sigma;
    s -= nu * rhodot[c];
    // destruction Jacobian (:275-357)
    double rp;
    if (Sl < nu / (9e6 * denom)) {
      rp = 0;
    } else {
      const double chi = x, chiP = 1. / mu[c];
      const double chi3 = chi * chi * chi, chi4 = chi3 * chi, chi6 = chi3 * chi3;
      const double fv2p = chi * (4 * (chi3 * chiP) / (chi3 + cv13) -
                                 3 * (chi6 * chiP) / std::pow(chi3 + cv13, 2)) /
                              std::pow(chi4 / (chi3 + cv13) + 1, 2) -
                          chiP / (chi4 / (chi3 + cv13) + 1);
      const double Stp = (fv2 / r0 + nu * fv2p) / (denom);
      rp = 1. / (r0 * denom * Sl) - nu * Stp / (denom * Sl * Sl);
    }
    const double gp = rp + S.cw2 * (6. * std::pow(rc, 5) * rp - rp);
    const double term = std::pow((cw36 + 1.) / (cw36 + g6), 1. / 6.);
    const double term2 = term * term, term5 = term2 * term2 * term;
    const double rterm5 = 1. / term5, rsum = 1. / (g6 + cw36);
    const double fwp = gp * term - gp * ((cw36 + 1) * g6) * rsum * rsum * rterm5;
    double sJ = srcJ[c];
    sJ -= V * cw1 * r0 * nu * (r0 * nu * fwp + 2. * fw) / (y * y);
    sJ += -rhodot[c];
    o->sa_src[c] = s;
    o->sa_D[c] = -sJ + r0 * (V / o->dtau[c]);
  }
  if (src_out) std::memcpy(src_out, o->sa_src.data(), sizeof(double) * nc);
  o->have_sa = true;
  o->have_sa_dq = false;
  return FPSI_OK;
}

extern "C" int orc_sa_get_system(orc_ctx* o, double* D, double* fjp, double* fjm) {
  if (!o->have_sa) return FPSI_E_STATE;
  if (D) std::memcpy(D, o->sa_D.data(), sizeof(double) * o->nc);
  if (fjp) std::memcpy(fjp, o->sa_fjp.data(), sizeof(double) * o->nf);
  if (fjm) std::memcpy(fjm, o->sa_fjm.data(), sizeof(double) * o->nf);
  return FPSI_OK;
}

// scalar SGS (linearSolverSGS.loci:333-470): x = B/D, then per sweep the
// forward and backward passes x_c = Dinv (B - sum_upper U x_cr - sum_lower L x_cl)
// with L = -fjp, U = fjm; colour == NULL: sequential order, else multi-colour
extern "C" int orc_sa_solve(orc_ctx* o, const int32_t* colour, double* dq) {
  if (!o->have_sa) return FPSI_E_STATE;
  const int64_t nc = o->nc;
  std::vector<double> Dinv(nc), x(nc);
  for (int64_t c = 0; c < nc; ++c) {
    Dinv[c] = 1. / o->sa_D[c];
    x[c] = Dinv[c] * o->sa_src[c];
  }
  auto gs = [&](int64_t c) {
    double t = -o->sa_src[c];
    for (int64_t k = o->up_off[c]; k < o->up_off[c + 1]; ++k) {
      const int64_t f = o->up[k];
      t += x[o->cr[f]] * o->sa_fjm[f];
    }
    for (int64_t k = o->lo_off[c]; k < o->lo_off[c + 1]; ++k) {
      const int64_t f = o->lo[k];
      t += x[o->cl[f]] * (-o->sa_fjp[f]);
    }
    x[c] = Dinv[c] * (-t);
  };
  std::vector<int64_t> order(nc);
  for (int64_t c = 0; c < nc; ++c) order[c] = c;
  if (colour) {
    std::stable_sort(order.begin(), order.end(),
                     [&](int64_t a, int64_t b) { return colour[a] < colour[b]; });
  }
  for (int it = 0; it < o->P.gauss_seidel_iter; ++it) {
    for (int64_t i = 0; i < nc; ++i) gs(order[i]);
    for (int64_t i = nc - 1; i >= 0; --i) gs(order[i]);
  }
  o->sa_dq = x;
  if (dq) std::memcpy(dq, x.data(), sizeof(double) * nc);
  o->have_sa_dq = true;
  return FPSI_OK;
}

// X_next = max(X + min(1, urelax X / (|dq| + 1e-15)) dq, 1e-15)
// (solverScalarTransport.loci:397-405)
extern "C" int orc_sa_update(orc_ctx* o) {
  if (!o->have_sa_dq) return FPSI_E_STATE;
  const double relax = o->P.urelax;
  for (int64_t c = 0; c < o->nc; ++c) {
    double tscale = 1.0;
    tscale = std::min(tscale, relax * o->nut[c] / (std::fabs(o->sa_dq[c]) + 1e-15));
    double xn = o->nut[c] + tscale * o->sa_dq[c];
    o->nut[c] = std::max(xn, 1e-15);
  }
  o->have_sa = o->have_sa_dq = false;
  return FPSI_OK;
}
