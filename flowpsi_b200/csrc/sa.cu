// sa.cu -- Spalart-Allmaras working variable nu~ on the GPU: the baseline
// model with standard production (turbulence/SA/SA_turb.loci:85-476) inside
// the reference's steady scalar transport (solverScalarTransport.loci:36-700),
// solved segregated from the mean flow once per implicit step.
//
// Data (RCM cell order, faces sorted as the mean flow's):
//   nut [nc], wdist [nc], sgrad [nc][3], sphi [nc]      FP64
//   nub [nbf]      nu~ on the boundary faces
//   per face, SoA [7][nf]: conv, diff, divn, fjp, fjm, jl, jr
//     conv = mdot max(X_upwind, 0)      (inviscid_fluxP(X,Zero))
//     diff = diff1_f / rho              (added times the cell's rho)
//     divn = grads_f(nu~).n A           (div_nuTilde)
//     fjp, fjm: X_fjp, X_fjm (interior faces; L = -fjp, U = fjm)
//     jl, jr:   contributions of the face to X_srcJ of cl and cr
//   B [nc] = X_src, D [nc] = X_D, Dinv [nc], x [nc] iterate
// Each cell gathers its faces in its fixed face-list order: no atomics.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "fpsi_internal.h"
#include "kernels.cuh"

namespace fpsi {
namespace sa {

// Spa_All_param (SA_param.h:28-40)
constexpr double CB1 = 0.1355, KAPPA = 0.41, CV1 = 7.1, CB2 = 0.622, CW2 = 0.3, CW3 = 2.0;
constexpr double SIGMA = 2. / 3.;
constexpr double FACTORX = 2, FACTORY = .5;  // SA_turb.loci:426-427

struct Geo {
  int64_t nc, nf, nfi;
  const int32_t *cl, *cr, *cf_off, *cf;
  const double *n, *area, *rL, *rR, *vol, *Minv;
  const fpsi_bc* bcs;
};

struct Gas {
  double gamma, Rt, pamb, a1, a2, a3;
};

__device__ __forceinline__ double suth(double T, const Gas& g) {
  return g.a1 * pow(T, g.a2) / (T + g.a3);
}
__device__ __forceinline__ double rho_of(const double* q, int64_t c, const Gas& g) {
  return (q[5 * c + 4] + g.pamb) / (g.Rt * q[5 * c]);
}

// tmu = nu~ f_v1 rho (SA_turb.loci:91-107)
__global__ void k_sa_tmu(int64_t nc, const double* __restrict__ q, const double* __restrict__ nut,
                         Gas g, double* __restrict__ tmu) {
  const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const double rho = rho_of(q, c, g), mu = suth(q[5 * c], g);
  const double x = rho * nut[c] / mu;
  const double fv1 = pow(x, 3) / (pow(x, 3) + pow(CV1, 3));
  tmu[c] = nut[c] * fv1 * rho;
}

// nu~ on boundary faces: 0 on no-slip walls (SA_turb.loci:181-183), the
// inside value on symmetry planes or where the face velocity leaves, else
// the boundary's nu_t (solverScalarTransport.loci:423-466, SA_turb.loci:167-179)
__global__ void k_sa_bface(Geo G, const double* __restrict__ qb, const double* __restrict__ nut,
                           double* __restrict__ nub) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t f = G.nfi + i;
  if (f >= G.nf) return;
  const fpsi_bc bc = G.bcs[-G.cr[f] - 1];
  const int64_t a = G.cl[f];
  double v;
  if (bc.kind == FPSI_BC_VISCOUS_WALL) {
    v = 0.0;
  } else if (bc.kind == FPSI_BC_REFLECTING) {
    v = nut[a];
  } else {
    const double* qf = qb + 5 * i;
    const double uit = G.n[f] * qf[1] + G.n[G.nf + f] * qf[2] + G.n[2 * G.nf + f] * qf[3];
    v = uit >= -0.0 ? nut[a] : (bc.nu_t > 0 ? bc.nu_t : 5e-9);
  }
  nub[i] = v;
}

// least-squares gradient of nu~ and its limiter (the method of the mean
// flow's k_grad_limiter, one variable)
__global__ void k_sa_grad(Geo G, const double* __restrict__ nut, const double* __restrict__ nub,
                          int limiter, double Kl, double* __restrict__ sgrad,
                          double* __restrict__ sphi) {
  const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= G.nc) return;
  const int64_t nf = G.nf;
  const double xc = nut[c];
  double b0 = 0, b1 = 0, b2 = 0, xmax = xc, xmin = xc;
  const int32_t e0 = G.cf_off[c], e1 = G.cf_off[c + 1];
  for (int32_t e = e0; e < e1; ++e) {
    const int32_t ent = G.cf[e];
    const int64_t f = ent >> 1;
    double xn, d0, d1, d2;
    if (f >= G.nfi) {
      xn = nub[f - G.nfi];
      d0 = G.rL[f], d1 = G.rL[nf + f], d2 = G.rL[2 * nf + f];
    } else {
      const bool lower = ent & 1;
      xn = nut[lower ? G.cl[f] : G.cr[f]];
      const double sg = lower ? -1.0 : 1.0;
      d0 = sg * (G.rL[f] - G.rR[f]);
      d1 = sg * (G.rL[nf + f] - G.rR[nf + f]);
      d2 = sg * (G.rL[2 * nf + f] - G.rR[2 * nf + f]);
    }
    const double dx = xn - xc;
    b0 += d0 * dx, b1 += d1 * dx, b2 += d2 * dx;
    xmax = fmax(xmax, xn), xmin = fmin(xmin, xn);
  }
  const int64_t nc = G.nc;
  const double m0 = G.Minv[c], m1 = G.Minv[nc + c], m2 = G.Minv[2 * nc + c], m3 = G.Minv[3 * nc + c],
               m4 = G.Minv[4 * nc + c], m5 = G.Minv[5 * nc + c];
  const double g0 = m0 * b0 + m1 * b1 + m2 * b2;
  const double g1 = m1 * b0 + m3 * b1 + m4 * b2;
  const double g2 = m2 * b0 + m4 * b1 + m5 * b2;
  double ph = limiter == FPSI_LIMITER_ZERO ? 0.0 : 1.0;
  if (limiter == FPSI_LIMITER_VENKATAKRISHNAN || limiter == FPSI_LIMITER_BARTH) {
    const double h = cbrt(G.vol[c]);
    const double kh = Kl * h, eps2 = kh * kh * kh;
    for (int32_t e = e0; e < e1; ++e) {
      const int32_t ent = G.cf[e];
      const int64_t f = ent >> 1;
      const double* r = (ent & 1) ? G.rR : G.rL;
      const double dd = g0 * r[f] + g1 * r[nf + f] + g2 * r[2 * nf + f];
      double p = 1.0;
      if (dd != 0.0) {
        const double d1 = dd > 0 ? xmax - xc : xmin - xc;
        if (limiter == FPSI_LIMITER_BARTH) {
          p = fmin(1.0, d1 / dd);
        } else {
          const double num = (d1 * d1 + eps2) + 2.0 * dd * d1;
          const double den = d1 * d1 + 2.0 * dd * dd + d1 * dd + eps2;
          p = fmin(1.0, num / den);
        }
      }
      ph = fmin(ph, p);
    }
  }
  sgrad[3 * c] = g0, sgrad[3 * c + 1] = g1, sgrad[3 * c + 2] = g2;
  sphi[c] = ph;
}

// per face: convection, diffusion, divergence and Jacobian pieces
// (SA_turb.loci:185-476, solverScalarTransport.loci:107-133,494-552,565-612)
__global__ void k_sa_face(Geo G, const double* __restrict__ q, const double* __restrict__ qb,
                          const double* __restrict__ F, const double* __restrict__ nut,
                          const double* __restrict__ nub, const double* __restrict__ sgrad,
                          const double* __restrict__ sphi, Gas g, double* __restrict__ out) {
  const int64_t f = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t nf = G.nf;
  if (f >= nf) return;
  const double n0 = G.n[f], n1 = G.n[nf + f], n2 = G.n[2 * nf + f];
  const double A = G.area[f];
  const double mdot = F[FREC * f];  // scalar_mdot_f = iflux[0]
  const int64_t a = G.cl[f];
  const double* ga = sgrad + 3 * a;
  const double rl0 = G.rL[f], rl1 = G.rL[nf + f], rl2 = G.rL[2 * nf + f];
  const double xl = nut[a] + sphi[a] * (ga[0] * rl0 + ga[1] * rl1 + ga[2] * rl2);
  const double rho_a = rho_of(q, a, g);
  double conv, diff, divn, fjp = 0.0, fjm = 0.0, jl, jr = 0.0;
  if (f < G.nfi) {
    const int64_t b = G.cr[f];
    const double* gb = sgrad + 3 * b;
    const double rr0 = G.rR[f], rr1 = G.rR[nf + f], rr2 = G.rR[2 * nf + f];
    const double xr = nut[b] + sphi[b] * (gb[0] * rr0 + gb[1] * rr1 + gb[2] * rr2);
    const double vl = G.vol[a], vr = G.vol[b];
    const double rho_b = rho_of(q, b, g);
    const double nuf = (vr * nut[a] + vl * nut[b]) * (1.0 / (vr + vl));
    const double muf = (vl * suth(q[5 * b], g) + vr * suth(q[5 * a], g)) / (vl + vr);
    const double rhof = (1. / (vl + vr)) * (vl * rho_b + vr * rho_a);
    const double d0 = rl0 - rr0, d1 = rl1 - rr1, d2 = rl2 - rr2;
    const double dsq = d0 * d0 + d1 * d1 + d2 * d2;
    const double gm0 = 0.5 * (ga[0] + gb[0]), gm1 = 0.5 * (ga[1] + gb[1]), gm2 = 0.5 * (ga[2] + gb[2]);
    const double cc = ((nut[b] - nut[a]) - (gm0 * d0 + gm1 * d1 + gm2 * d2)) / dsq;
    const double gf0 = gm0 + cc * d0, gf1 = gm1 + cc * d1, gf2 = gm2 + cc * d2;
    const double gn = gf0 * n0 + gf1 * n1 + gf2 * n2;
    divn = gn * A;
    diff = gn * A;
    diff = (diff * (muf / rhof + (1. + CB2) * nuf)) / SIGMA;
    const double xv = mdot < 0.0 ? xr : xl;
    conv = mdot * fmax(xv, 0.0);
    fjp += fmax(mdot, 0.0);
    fjm += fmin(mdot, 0.0);
    const double rbar = .5 * (rho_a + rho_b);
    const double C = (muf + (1. + CB2) * rbar * nuf) * A;
    const double dd = d0 * n0 + d1 * n1 + d2 * n2;  // (x_b - x_a).n
    fjp -= -C / (dd * SIGMA);
    fjm += -C / (dd * SIGMA);
    const double C2 = CB2 * A, d2s = SIGMA * dd;
    const double sU = -FACTORX * (C2 / d2s) * rho_a * nut[a];
    const double sL = -FACTORX * (C2 / d2s) * rho_b * nut[b];
    fjp += sL;
    fjm -= sU;
    // X_srcJ: -fjp / +fjm of the generic sum, the cb2 diagonal terms and
    // the removal of the non-conservative L/U parts (SA_turb.loci:745-752)
    jl = FACTORX * FACTORY * (C2 / d2s) * rho_a * nut[a];
    jl -= fjp;
    jl += sL;
    jr = FACTORX * FACTORY * (C2 / d2s) * rho_b * nut[b];
    jr += fjm;
    jr += sU;
  } else {
    const int kind = G.bcs[-G.cr[f] - 1].kind;
    const double* qf = qb + 5 * (f - G.nfi);
    const double nuf = nub[f - G.nfi];
    const double muf = suth(qf[0], g);
    const double rhof = (qf[4] + g.pamb) / (g.Rt * qf[0]);  // solverEoS.loci:53-56
    const double rsq = rl0 * rl0 + rl1 * rl1 + rl2 * rl2;
    const double cc = ((nuf - nut[a]) - (ga[0] * rl0 + ga[1] * rl1 + ga[2] * rl2)) / rsq;
    const double gf0 = ga[0] + cc * rl0, gf1 = ga[1] + cc * rl1, gf2 = ga[2] + cc * rl2;
    const double gn = gf0 * n0 + gf1 * n1 + gf2 * n2;
    divn = gn * A;
    diff = gn * A;
    diff = (diff * (muf / rhof + (1. + CB2) * nuf)) / SIGMA;
    const double xv = mdot < 0.0 ? nuf : xl;
    conv = mdot * fmax(xv, 0.0);
    jl = -fmax(mdot, 0.0);
    if (kind != FPSI_BC_REFLECTING) {  // no_symmetry_BC
      const double C = (muf + (1. + CB2) * rhof * nuf) * A;
      const double db = rl0 * n0 + rl1 * n1 + rl2 * n2;
      jl += -C / (db * SIGMA);
      const double C2 = CB2 * A, d2s = SIGMA * db;
      jl += FACTORX * FACTORY * (C2 / d2s) * rho_a * nut[a];
    }
  }
  out[f] = conv;
  out[nf + f] = diff;
  out[2 * nf + f] = divn;
  out[3 * nf + f] = fjp;
  out[4 * nf + f] = fjm;
  out[5 * nf + f] = jl;
  out[6 * nf + f] = jr;
}

// per cell: production, destruction and its Jacobian, the gathered face
// terms, the cb2 divergence term, the continuity term; B = X_src,
// D = -X_srcJ + rho V / dtau (SA_turb.loci:109-357,420-424,
// solverScalarTransport.loci:504-530,614-681)
__global__ void k_sa_cell(Geo G, const double* __restrict__ q, const double* __restrict__ grad,
                          const double* __restrict__ F, const double* __restrict__ dtau,
                          const double* __restrict__ nut, const double* __restrict__ wdist,
                          const double* __restrict__ fo, Gas g, double* __restrict__ B,
                          double* __restrict__ D, double* __restrict__ Dinv) {
  const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= G.nc) return;
  const int64_t nf = G.nf;
  const double r0 = rho_of(q, c, g);
  double src = 0.0, srcJ = 0.0, rhodot = 0.0, divn = 0.0;
  for (int32_t e = G.cf_off[c]; e < G.cf_off[c + 1]; ++e) {
    const int32_t ent = G.cf[e];
    const int64_t f = ent >> 1;
    const double mdot = F[FREC * f];
    if (ent & 1) {  // lower face: this cell is cr
      src += fo[f];
      rhodot += mdot;
      src -= r0 * fo[nf + f];
      divn -= fo[2 * nf + f];
      srcJ += fo[6 * nf + f];
    } else {
      src -= fo[f];
      rhodot -= mdot;
      src += r0 * fo[nf + f];
      divn += fo[2 * nf + f];
      srcJ += fo[5 * nf + f];
    }
  }
  const double nu = nut[c], V = G.vol[c], y = wdist[c];
  const double mu = suth(q[5 * c], g);
  const double* gu = grad + GPREC * c + 3;  // rows u, v, w: d u_i / d x_j
  const double wx = gu[3 * 2 + 1] - gu[3 * 1 + 2];
  const double wy = gu[3 * 0 + 2] - gu[3 * 2 + 0];
  const double wz = gu[3 * 1 + 0] - gu[3 * 0 + 1];
  const double vort = sqrt(wx * wx + wy * wy + wz * wz);
  const double x = r0 * nu / mu;
  const double fv1 = pow(x, 3) / (pow(x, 3) + pow(CV1, 3));
  const double fv2 = 1.0 - (x / (1.0 + x * fv1));
  const double k2 = KAPPA * KAPPA;
  const double denom = k2 * y * y;
  double St = 0.0;
  St += vort;
  St += nu * fv2 / denom;
  const double Sl = fmax(St, 0.3 * vort);
  double rc;
  if (Sl < nu / (10 * denom))
    rc = 10;
  else
    rc = nu / (Sl * denom);
  const double cw36 = pow(CW3, 6);
  const double rr2 = rc * rc, r6 = rr2 * rr2 * rr2;
  const double gc = rc + CW2 * (r6 - rc);
  const double g2 = gc * gc, g6 = g2 * g2 * g2;
  const double fw = gc * pow((1.0 + cw36) / (g6 + cw36), 1.0 / 6.0);
  const double cw1 = (CB1) / (k2) + (1.0 + (CB2)) / (SIGMA);
  src += r0 * nu * Sl * CB1 * V;
  const double t = nu / y;
  src -= r0 * fw * cw1 * t * t * V;
  src += -r0 * nu * divn * CB2 / SIGMA;
  src -= nu * rhodot;
  const double cv13 = CV1 * CV1 * CV1;
  double rp;
  if (Sl < nu / (9e6 * denom)) {
    rp = 0;
  } else {
    const double chi = x, chiP = 1. / mu;
    const double chi3 = chi * chi * chi, chi4 = chi3 * chi, chi6 = chi3 * chi3;
    const double fv2p = chi * (4 * (chi3 * chiP) / (chi3 + cv13) - 3 * (chi6 * chiP) / pow(chi3 + cv13, 2)) /
                            pow(chi4 / (chi3 + cv13) + 1, 2) -
                        chiP / (chi4 / (chi3 + cv13) + 1);
    const double Stp = (fv2 / r0 + nu * fv2p) / (denom);
    rp = 1. / (r0 * denom * Sl) - nu * Stp / (denom * Sl * Sl);
  }
  const double gp = rp + CW2 * (6. * pow(rc, 5) * rp - rp);
  const double term = pow((cw36 + 1.) / (cw36 + g6), 1. / 6.);
  const double term2 = term * term, term5 = term2 * term2 * term;
  const double rterm5 = 1. / term5, rsum = 1. / (g6 + cw36);
  const double fwp = gp * term - gp * ((cw36 + 1) * g6) * rsum * rsum * rterm5;
  srcJ -= V * cw1 * r0 * nu * (r0 * nu * fwp + 2. * fw) / (y * y);
  srcJ += -rhodot;
  const double d = -srcJ + r0 * (V / dtau[c]);
  B[c] = src;
  D[c] = d;
  Dinv[c] = 1. / d;
}

__global__ void k_sa_jacobi(int64_t nc, const double* __restrict__ B, const double* __restrict__ Dinv,
                            double* __restrict__ x) {
  const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c < nc) x[c] = Dinv[c] * B[c];
}

// one colour of a scalar Gauss-Seidel pass (linearSolverSGS.loci:365-420):
// t = -B + sum_upper U x_cr + sum_lower L x_cl, x = Dinv (-t)
__global__ void k_sa_gs(Geo G, const int32_t* __restrict__ cells, int64_t n,
                        const double* __restrict__ B, const double* __restrict__ Dinv,
                        const double* __restrict__ fo, double* __restrict__ x) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t c = cells[i];
  const int64_t nf = G.nf;
  double t = -B[c];
  for (int32_t e = G.cf_off[c]; e < G.cf_off[c + 1]; ++e) {
    const int32_t ent = G.cf[e];
    const int64_t f = ent >> 1;
    if (f >= G.nfi) continue;
    if (ent & 1)
      t += x[G.cl[f]] * (-fo[3 * nf + f]);
    else
      t += x[G.cr[f]] * fo[4 * nf + f];
  }
  x[c] = Dinv[c] * (-t);
}

// X_next = max(X + min(1, urelax X / (|dq| + 1e-15)) dq, 1e-15)
// (solverScalarTransport.loci:397-405)
// guard (may be null): the mean flow's norms of this step; NaN norms leave
// nu~ unchanged, as the mean-flow update does
__global__ void k_sa_update(int64_t nc, double urelax, const double* __restrict__ dq,
                            double* __restrict__ nut, const double* __restrict__ guard) {
  const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  if (guard && (isnan(guard[0]) || isnan(guard[1]) || isnan(guard[2]))) return;
  double tscale = 1.0;
  tscale = fmin(tscale, urelax * nut[c] / (fabs(dq[c]) + 1e-15));
  const double xn = nut[c] + tscale * dq[c];
  nut[c] = fmax(xn, 1e-15);
}

}  // namespace sa

namespace {
inline unsigned nblk(int64_t n, int t) { return unsigned((n + t - 1) / t); }

sa::Geo geo(const fpsi_ctx* x) {
  sa::Geo G;
  G.nc = x->H.nc, G.nf = x->H.nf, G.nfi = x->H.nfi;
  G.cl = x->d_cl, G.cr = x->d_cr, G.cf_off = x->d_cf_off, G.cf = x->d_cf;
  G.n = x->d_n, G.area = x->d_area, G.rL = x->d_rL, G.rR = x->d_rR, G.vol = x->d_vol;
  G.Minv = x->d_Minv;
  G.bcs = x->d_bcs;
  return G;
}
sa::Gas sgas(const fpsi_ctx* x) {
  return sa::Gas{x->P.gamma, x->P.Rtilde, x->P.Pambient, x->P.mu_a1, x->P.mu_a2, x->P.mu_a3};
}
}  // namespace

bool sa_active(const fpsi_ctx* x) {
  return x->P.viscous == 2 && x->P.turbulence == FPSI_TURB_SA;
}

int sa_launch_tmu(fpsi_ctx* x) {
  prof_begin(x, "sa_tmu");
  sa::k_sa_tmu<<<nblk(x->H.nc, 256), 256, 0, x->stream>>>(x->H.nc, x->d_q, x->d_nut, sgas(x),
                                                          x->d_tmu);
  prof_end(x);
  FPSI_CUDA_TRY(cudaGetLastError());
  return FPSI_OK;
}

int sa_launch_residual(fpsi_ctx* x) {
  const sa::Geo G = geo(x);
  const sa::Gas g = sgas(x);
  cudaStream_t s = x->stream;
  prof_begin(x, "sa_grad");
  if (x->H.nbf > 0)
    sa::k_sa_bface<<<nblk(x->H.nbf, 256), 256, 0, s>>>(G, x->d_qb, x->d_nut, x->d_sa_nub);
  sa::k_sa_grad<<<nblk(G.nc, 128), 128, 0, s>>>(G, x->d_nut, x->d_sa_nub, x->P.limiter, x->P.Kl,
                                                x->d_sa_grad, x->d_sa_phi);
  prof_end(x);
  prof_begin(x, "sa_face");
  sa::k_sa_face<<<nblk(G.nf, 128), 128, 0, s>>>(G, x->d_q, x->d_qb, x->d_F, x->d_nut, x->d_sa_nub,
                                                x->d_sa_grad, x->d_sa_phi, g, x->d_sa_face);
  prof_end(x);
  prof_begin(x, "sa_cell");
  sa::k_sa_cell<<<nblk(G.nc, 128), 128, 0, s>>>(G, x->d_q, x->d_grad, x->d_F, x->d_dtau, x->d_nut,
                                                x->d_wdist, x->d_sa_face, g, x->d_sa_B, x->d_sa_D,
                                                x->d_sa_Dinv);
  prof_end(x);
  FPSI_CUDA_TRY(cudaGetLastError());
  return FPSI_OK;
}

int sa_launch_solve(fpsi_ctx* x) {
  const sa::Geo G = geo(x);
  cudaStream_t s = x->stream;
  const HostMesh& H = x->H;
  prof_begin(x, "sa_sgs");
  sa::k_sa_jacobi<<<nblk(G.nc, 256), 256, 0, s>>>(G.nc, x->d_sa_B, x->d_sa_Dinv, x->d_sa_x);
  // a colour directly following itself would rewrite the same values
  // (its cells read only other colours): skipped, the result is unchanged
  int last = -1;
  for (int it = 0; it < x->P.gauss_seidel_iter; ++it)
    for (int pass = 0; pass < 2; ++pass)
      for (int kk = 0; kk < H.ncolours; ++kk) {
        const int k = pass == 0 ? kk : H.ncolours - 1 - kk;
        const int64_t b = H.colour_off[k], n = H.colour_off[k + 1] - b;
        if (n == 0 || k == last) continue;
        last = k;
        sa::k_sa_gs<<<nblk(n, 128), 128, 0, s>>>(G, x->d_colour_cells + b, n, x->d_sa_B,
                                                 x->d_sa_Dinv, x->d_sa_face, x->d_sa_x);
      }
  prof_end(x);
  FPSI_CUDA_TRY(cudaGetLastError());
  return FPSI_OK;
}

int sa_launch_update(fpsi_ctx* x, const double* guard) {
  prof_begin(x, "sa_update");
  sa::k_sa_update<<<nblk(x->H.nc, 256), 256, 0, x->stream>>>(x->H.nc, x->P.urelax, x->d_sa_x,
                                                             x->d_nut, guard);
  prof_end(x);
  FPSI_CUDA_TRY(cudaGetLastError());
  return FPSI_OK;
}

}  // namespace fpsi
