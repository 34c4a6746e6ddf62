// kernels.cu -- sm_100a kernels of the steady implicit step.
//
// Data layout in HBM (RCM cell order, faces sorted by cl, interior first):
//   q      [nc][5]  FP64  T,u,v,w,pg          (AoS: every gather is one 40 B record)
//   grad   [nc][20] FP64  dT/dx.. dpg/dz (15), then the limiter per variable
//                         (5, phi = grad + 15): one 160 B record per cell
//   F      [nf][6]  FP64  face flux (5) and maxev_f*area: one 48 B record,
//                         three 16 B accesses
//   src    [nc][5]  FP64, dtau [nc]
//   fjp/fjm [nf][25] TB   (TB = float in REF/MIXED precision, double in FP64)
//   sweeps, colour order (ci = position of the cell in its colour's list):
//     luc  [25][n_k] TB per colour   LU of fluid_D;   bc [5][n_k] TB  fluid_B
//     aoff [m_k][25][n_k] TB per colour: off-diagonal block of each slot
//     nbr  [m_k][n_k] int32 per colour: ci of the slot's neighbour
//     x    [nc][5]  TX (ci order)   (TX = double in FP64/REF, float in MIXED)
// geometry is SoA: n[3][nf], area[nf], rL[3][nf], rR[3][nf], Minv[6][nc].
//
// Every reduction has a fixed order (per-cell loops over a fixed face list,
// fixed-shape block trees), so results are bitwise reproducible run to run.
#include <cuda_runtime.h>

#include <cstdint>

#include "fpsi_internal.h"
#include "kernels.cuh"
#include "physics.cuh"

namespace fpsi {
namespace dev {

struct MeshView {
  int64_t nc, nf, nfi;
  const int32_t* cl;
  const int32_t* cr;
  const double* n;     // [3][nf]
  const double* area;  // [nf]
  const double* rL;    // [3][nf]
  const double* rR;    // [3][nf]
  const double* vol;
  const double* Minv;  // [6][nc]
  const int32_t* cf_off;
  const int32_t* cf;
  int32_t K;           // largest face count of a cell
  const int32_t* ecf;  // [K][nc] cf entries entry-major, -1 past the last
  const int32_t* enb;  // [K][nc] interior neighbour of the entry, -1 on boundary faces
  const fpsi_bc* bcs;
};

__device__ __forceinline__ Q5 load_q(const double* q, int64_t c) {
  const double* p = q + 5 * c;
  Q5 r;
  r.T = __ldg(p + 0);
  r.u = __ldg(p + 1);
  r.v = __ldg(p + 2);
  r.w = __ldg(p + 3);
  r.p = __ldg(p + 4);
  return r;
}
__device__ __forceinline__ void q_arr(const Q5& q, double a[5]) {
  a[0] = q.T, a[1] = q.u, a[2] = q.v, a[3] = q.w, a[4] = q.p;
}

// ---------------------------------------------------------------------------
// boundary face states (bcInflow.loci:270-344, bcOutflow.loci:84-142,
// bcImpermeable.loci:48-140); eta == 1
// ---------------------------------------------------------------------------
// Area-weighted mean gauge pressure of the cells next to each boundary
// condition (areaPressure / boundary_area, bcOutflow.loci:178-198), for the
// pMean outflow: block b sums over the faces of condition b in a fixed
// order (per-thread strided sums, then a tree), out[2b] = sum A pg,
// out[2b+1] = sum A.
constexpr int BCM_THREADS = 256;
__global__ void __launch_bounds__(BCM_THREADS)
k_bc_mean(MeshView M, const double* __restrict__ q, double* __restrict__ out) {
  const int b = blockIdx.x;
  __shared__ double sp[BCM_THREADS], sa[BCM_THREADS];
  double ap = 0, aa = 0;
  for (int64_t f = M.nfi + threadIdx.x; f < M.nf; f += BCM_THREADS) {
    if (-M.cr[f] - 1 != b) continue;
    const double A = M.area[f];
    ap += A * q[5 * int64_t(M.cl[f]) + 4];
    aa += A;
  }
  sp[threadIdx.x] = ap, sa[threadIdx.x] = aa;
  __syncthreads();
  for (int st = BCM_THREADS / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) sp[threadIdx.x] += sp[threadIdx.x + st], sa[threadIdx.x] += sa[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[2 * b] = sp[0], out[2 * b + 1] = sa[0];
}

// bcmean: k_bc_mean's sums (read by pMean outflows only); bcflags: error
// bits of this residual (OUTFLOW_BECAME_INFLOW)
__global__ void k_bc_state(MeshView M, const double* __restrict__ q, const fpsi_bc* __restrict__ bcs,
                           Gas g, const double* __restrict__ bcmean, int32_t* __restrict__ bcflags,
                           double* __restrict__ qb) {
  const int64_t b = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t nbf = M.nf - M.nfi;
  if (b >= nbf) return;
  const int64_t f = M.nfi + b;
  const int32_t c = M.cl[f];
  const fpsi_bc bc = bcs[-M.cr[f] - 1];
  const double nx = M.n[f], ny = M.n[M.nf + f], nz = M.n[2 * M.nf + f];
  const Q5 qi = load_q(q, c);
  Q5 q0;
  q0.T = bc.T, q0.u = bc.u[0], q0.v = bc.u[1], q0.w = bc.u[2], q0.p = bc.pg;
  Q5 r = qi;
  switch (bc.kind) {
    case FPSI_BC_FARFIELD: {
      const double uit = qi.u * nx + qi.v * ny + qi.w * nz;
      const double ai = sqrt(g.gamma * g.Rt * qi.T);
      const double a0 = sqrt(g.gamma * g.Rt * q0.T);
      if (uit > 0) {
        if (!(uit > ai)) cv_state(true, qi, q0, nx, ny, nz, 0.0, g, 1.0, r);
      } else {
        if (-uit > a0)
          r = q0;
        else
          cv_state(false, qi, q0, nx, ny, nz, 0.0, g, 1.0, r);
      }
      break;
    }
    case FPSI_BC_INFLOW: {  // bcInflow.loci:376-401
      const double uit = qi.u * nx + qi.v * ny + qi.w * nz;
      const double a0 = sqrt(g.gamma * g.Rt * q0.T);
      if (uit > 0 || -uit > a0)
        r = q0;
      else
        cv_state(false, qi, q0, nx, ny, nz, 0.0, g, 1.0, r);
      break;
    }
    case FPSI_BC_SUPERSONIC_INFLOW:
      r = q0;
      break;
    case FPSI_BC_SUPERSONIC_OUTFLOW: {
      const double ai = sqrt(g.gamma * g.Rt * qi.T);
      const double ut = qi.u * nx + qi.v * ny + qi.w * nz;
      if (ut < ai) r.p -= (qi.p + g.pamb) * 0.1;
      break;
    }
    case FPSI_BC_VISCOUS_WALL:  // adiabatic no-slip wall, bcViscousWall.loci:148-218
      r.u = r.v = r.w = 0.0;
      break;
    case FPSI_BC_REFLECTING: {
      const double un = qi.u * nx + qi.v * ny + qi.w * nz;
      r.u = qi.u - 2.0 * un * nx;
      r.v = qi.v - 2.0 * un * ny;
      r.w = qi.w - 2.0 * un * nz;
      break;
    }
    case FPSI_BC_OUTFLOW:
    case FPSI_BC_OUTFLOW_MEAN: {  // bcOutflow.loci:206-244, us_n = 0
      // back pressure (gauge): 'p', or the cell's pressure shifted so that
      // the boundary's area-weighted mean becomes 'pMean' (:200-204)
      double pref = bc.pg;
      if (bc.kind == FPSI_BC_OUTFLOW_MEAN) {
        const int bi = -M.cr[f] - 1;
        pref = qi.p + (bc.pg - bcmean[2 * bi] / bcmean[2 * bi + 1]);
      }
      const double uit = qi.u * nx + qi.v * ny + qi.w * nz;
      const double ai = sqrt(g.gamma * g.Rt * qi.T);
      const double rhoi = (qi.p + g.pamb) / (g.Rt * qi.T);
      if (uit >= 0) {
        if (!(uit > ai)) {  // subsonic: the back pressure at the cell's density
          r.p = pref;
          r.T = (pref + g.pamb) / (g.Rt * rhoi);
        }
      } else {  // the outflow became an inflow
        r.u = r.v = r.w = 0.0;
        r.p = qi.p - 0.05 * (qi.p + g.pamb);
        atomicOr(bcflags, FPSI_BCERR_OUTFLOW_BECAME_INFLOW);
      }
      break;
    }
    case FPSI_BC_ISENTROPIC_INFLOW:  // total conditions: p0 = pg + Pambient, T0 = T
      isentropic_state(qi, nx, ny, nz, bc.pg + g.pamb, bc.T, g, r);
      break;
    case FPSI_BC_FIXED_MASS_INFLOW:
      if (!fixed_mass_state(qi, nx, ny, nz, bc.mass_flux, bc.T, g, r))
        atomicOr(bcflags, FPSI_BCERR_FIXED_MASS_FAILED_CONVERGENCE);
      break;
    case FPSI_BC_FIXED_MASS_OUTFLOW:
      fixed_mass_outflow_state(qi, nx, ny, nz, bc.mass_flux, bc.mass_relax, g, r);
      break;
    default:
      break;
  }
  double* o = qb + 5 * b;
  o[0] = r.T, o[1] = r.u, o[2] = r.v, o[3] = r.w, o[4] = r.p;
}

// ---------------------------------------------------------------------------
// least-squares gradient + limiter, one thread per cell.  Each cell's
// gradient (15) and limiter (5) form one 160 B record; the CTA's 128
// records are contiguous, staged in shared memory and written back with
// consecutive threads on consecutive addresses.
// ---------------------------------------------------------------------------
constexpr int GRAD_THREADS = 128;
// a cell's gradient-and-limiter record staged in shared memory with a
// stride of GPREC + 1 doubles, so that the 32 lanes' stores of one value
// fall into different banks
constexpr int GPS = GPREC + 1;
// The cell's faces are taken four at a time from the entry-major lists:
// the four entries and neighbours are loaded together (entry j of a warp's
// 32 cells is one coalesced line), then the four neighbour states and face
// vectors, then they are summed in the cell's face order.  Padding entries
// (-1) read cell 0 and face 0 and are not summed.
constexpr int ECH = 4;
struct EChunk {
  int32_t ent[ECH];
  int64_t f[ECH];
  int32_t nb[ECH];
};
__device__ __forceinline__ void load_chunk(const MeshView& M, int64_t c, int j0, EChunk& k,
                                           bool with_nb) {
#pragma unroll
  for (int i = 0; i < ECH; ++i) {
    const bool in = j0 + i < M.K;
    k.ent[i] = in ? __ldg(M.ecf + int64_t(j0 + i) * M.nc + c) : -1;
    k.nb[i] = in && with_nb ? __ldg(M.enb + int64_t(j0 + i) * M.nc + c) : -1;
  }
#pragma unroll
  for (int i = 0; i < ECH; ++i) k.f[i] = k.ent[i] >= 0 ? int64_t(k.ent[i] >> 1) : 0;
}
// the state across face i of the chunk: the neighbour's, or the boundary state
__device__ __forceinline__ const double* across(const MeshView& M, const double* q,
                                                const double* qb, const EChunk& k, int i) {
  return k.f[i] >= M.nfi ? qb + 5 * (k.f[i] - M.nfi) : q + 5 * int64_t(k.nb[i] < 0 ? 0 : k.nb[i]);
}

__device__ __forceinline__ void grad_limiter_cell(const MeshView& M, const double* __restrict__ q,
                                                  const double* __restrict__ qb, int limiter,
                                                  double Kl, int64_t c, double* go, double* po) {
  double qc[5];
  q_arr(load_q(q, c), qc);
  double b[15];
  double qmax[5], qmin[5];
#pragma unroll
  for (int k = 0; k < 15; ++k) b[k] = 0.0;
#pragma unroll
  for (int k = 0; k < 5; ++k) qmax[k] = qmin[k] = qc[k];
  const int64_t nf = M.nf;
  for (int j0 = 0; j0 < M.K; j0 += ECH) {
    EChunk ch;
    load_chunk(M, c, j0, ch, true);
    double qn[ECH][5], d[ECH][3];
#pragma unroll
    for (int i = 0; i < ECH; ++i) {
      const double* p = across(M, q, qb, ch, i);
#pragma unroll
      for (int k = 0; k < 5; ++k) qn[i][k] = __ldg(p + k);
      const bool bnd = ch.f[i] >= M.nfi;
      const double sg = (ch.ent[i] & 1) ? -1.0 : 1.0;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double l = M.rL[k * nf + ch.f[i]], r = M.rR[k * nf + ch.f[i]];
        d[i][k] = bnd ? l : sg * (l - r);
      }
    }
#pragma unroll
    for (int i = 0; i < ECH; ++i) {
      if (ch.ent[i] < 0) continue;
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        const double dq = qn[i][k] - qc[k];
        b[3 * k] += d[i][0] * dq;
        b[3 * k + 1] += d[i][1] * dq;
        b[3 * k + 2] += d[i][2] * dq;
        qmax[k] = dmax(qmax[k], qn[i][k]);
        qmin[k] = dmin(qmin[k], qn[i][k]);
      }
    }
  }
  const double m0 = M.Minv[c], m1 = M.Minv[M.nc + c], m2 = M.Minv[2 * M.nc + c],
               m3 = M.Minv[3 * M.nc + c], m4 = M.Minv[4 * M.nc + c], m5 = M.Minv[5 * M.nc + c];
  double g[15];
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const double bx = b[3 * k], by = b[3 * k + 1], bz = b[3 * k + 2];
    g[3 * k] = m0 * bx + m1 * by + m2 * bz;
    g[3 * k + 1] = m1 * bx + m3 * by + m4 * bz;
    g[3 * k + 2] = m2 * bx + m4 * by + m5 * bz;
  }
  double ph[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) ph[k] = limiter == FPSI_LIMITER_ZERO ? 0.0 : 1.0;
  if (limiter == FPSI_LIMITER_VENKATAKRISHNAN || limiter == FPSI_LIMITER_BARTH) {
    const double h = cbrt(M.vol[c]);
    const double kh = Kl * h;
    const double eps2 = kh * kh * kh;
    for (int j0 = 0; j0 < M.K; j0 += ECH) {
      EChunk ch;
      load_chunk(M, c, j0, ch, false);
      double rv[ECH][3];
#pragma unroll
      for (int i = 0; i < ECH; ++i) {
        const double* r = (ch.ent[i] & 1) ? M.rR : M.rL;
#pragma unroll
        for (int k = 0; k < 3; ++k) rv[i][k] = r[k * nf + ch.f[i]];
      }
#pragma unroll
      for (int i = 0; i < ECH; ++i) {
        if (ch.ent[i] < 0) continue;
#pragma unroll
        for (int k = 0; k < 5; ++k) {
          const double d2 = g[3 * k] * rv[i][0] + g[3 * k + 1] * rv[i][1] + g[3 * k + 2] * rv[i][2];
          // min(1, a / b) divides only where the ratio is below 1 (a
          // correctly rounded quotient is >= 1 exactly when a >= b for b > 0),
          // so the result is the same bit for bit
          double p = 1.0;
          if (d2 != 0.0) {
            const double d1 = d2 > 0 ? qmax[k] - qc[k] : qmin[k] - qc[k];
            if (limiter == FPSI_LIMITER_BARTH) {
              if (d2 > 0 ? d1 < d2 : d1 > d2) p = d1 / d2;
            } else {
              const double num = (d1 * d1 + eps2) + 2.0 * d2 * d1;
              const double den = d1 * d1 + 2.0 * d2 * d2 + d1 * d2 + eps2;
              if (num < den) p = num / den;
            }
          }
          ph[k] = dmin(ph[k], p);
        }
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 15; ++k) go[k] = g[k];
#pragma unroll
  for (int k = 0; k < 5; ++k) po[k] = ph[k];
}

// The face states of one cell's faces: MUSCL q_c + phi grad.(x_f - x_c)
// with the floors 0.1 min(T) and 0.1 min(pg) - 0.9 Pambient over the face's
// two cells (the form of fluxLowDiss.loci:338-356), and the side's spectral
// radius 0.5 max(|2 u.n - 2a|, |2 u.n + 2a|) of the cell-centre state
// (maxev_f, solverSetup.loci:81-105, eta == 1).  The cell writes its own
// side of every face; on a boundary face also the other side, the boundary
// state (not reconstructed) and its spectral radius.
__device__ __forceinline__ void side_record(double* o, const double l[5], double m) {
  double2* o2 = reinterpret_cast<double2*>(o);
  o2[0] = make_double2(l[0], l[1]);
  o2[1] = make_double2(l[2], l[3]);
  o2[2] = make_double2(l[4], m);
}
__device__ __forceinline__ double side_maxev(const double s[5], double nx, double ny, double nz,
                                             const Gas& gas) {
  const double ut = s[1] * nx + s[2] * ny + s[3] * nz;
  const double a2 = 2.0 * sqrt(gas.gamma * gas.Rt * s[0]);  // sqrt(4 a^2) of the reference, to an ulp
  return 0.5 * dmax(fabs(2.0 * ut - a2), fabs(2.0 * ut + a2));
}
__device__ __forceinline__ void face_states_cell(const MeshView& M, const double* __restrict__ q,
                                                 const double* __restrict__ qb, const Gas& gas,
                                                 int64_t c, const double g[15], const double ph[5],
                                                 double* __restrict__ qf) {
  double qc[5];
  q_arr(load_q(q, c), qc);
  const int64_t nf = M.nf;
  for (int j0 = 0; j0 < M.K; j0 += ECH) {
    EChunk ch;
    load_chunk(M, c, j0, ch, true);
    double Tn[ECH], pn[ECH], rv[ECH][3], nv[ECH][3];
#pragma unroll
    for (int i = 0; i < ECH; ++i) {
      const double* p = across(M, q, qb, ch, i);
      Tn[i] = __ldg(p), pn[i] = __ldg(p + 4);
      const double* r = (ch.ent[i] & 1) ? M.rR : M.rL;
#pragma unroll
      for (int k = 0; k < 3; ++k) rv[i][k] = r[k * nf + ch.f[i]], nv[i][k] = M.n[k * nf + ch.f[i]];
    }
#pragma unroll
    for (int i = 0; i < ECH; ++i) {
      if (ch.ent[i] < 0) continue;
      const int64_t f = ch.f[i];
      const int side = ch.ent[i] & 1;
      double l[5];
#pragma unroll
      for (int k = 0; k < 5; ++k)
        l[k] = qc[k] + ph[k] * (g[3 * k] * rv[i][0] + g[3 * k + 1] * rv[i][1] + g[3 * k + 2] * rv[i][2]);
      l[0] = dmax(l[0], 0.1 * dmin(side ? Tn[i] : qc[0], side ? qc[0] : Tn[i]));
      l[4] = dmax(l[4], 0.1 * dmin(side ? pn[i] : qc[4], side ? qc[4] : pn[i]) - 0.9 * gas.pamb);
      double* o = qf + int64_t(QFREC) * f;
      side_record(o + (QFREC / 2) * side, l, side_maxev(qc, nv[i][0], nv[i][1], nv[i][2], gas));
      if (f >= M.nfi) {
        double qbs[5];
        const double* p = qb + 5 * (f - M.nfi);
#pragma unroll
        for (int k = 0; k < 5; ++k) qbs[k] = __ldg(p + k);
        side_record(o + QFREC / 2, qbs, side_maxev(qbs, nv[i][0], nv[i][1], nv[i][2], gas));
      }
    }
  }
}

// WREC: also the cell's gradient-and-limiter record (viscous terms, the SA
// model and fpsi_get_reconstruction read it)
template <bool WREC>
__global__ void __launch_bounds__(GRAD_THREADS, 4)
k_grad_limiter(MeshView M, const double* __restrict__ q, const double* __restrict__ qb, int limiter,
               double Kl, Gas gas, double* __restrict__ grad, double* __restrict__ qf) {
  __shared__ double sr[WREC ? GRAD_THREADS * GPS : 1];
  const int64_t c0 = int64_t(blockIdx.x) * GRAD_THREADS;
  const int64_t c = c0 + threadIdx.x;
  if (c < M.nc) {
    double rec[GPREC];
    grad_limiter_cell(M, q, qb, limiter, Kl, c, rec, rec + 15);
    face_states_cell(M, q, qb, gas, c, rec, rec + 15, qf);
    if (WREC) {
#pragma unroll
      for (int k = 0; k < GPREC; ++k) sr[GPS * threadIdx.x + k] = rec[k];
    }
  }
  if (WREC) {
    __syncthreads();
    // one record per cell: the gradient (15) then the limiter (5)
    const int cnt = int(min(int64_t(GRAD_THREADS), M.nc - c0));
    for (int i = threadIdx.x; i < GPREC * cnt; i += GRAD_THREADS)
      grad[GPREC * c0 + i] = sr[GPS * (i / GPREC) + i % GPREC];
  }
}

// The same three passes with the per-face data of the last two staged in
// shared memory by the first: the first pass loads, for every face of the
// cell, the neighbour state, rL, rR and the normal, and keeps the cell's own
// face vector x_f - x_c, the normal and the neighbour's T and pg; the
// limiter and face-state passes then read those instead of walking the
// face lists again (two rounds of dependent gathers fewer).  Layout
// [entry][value][thread], so a warp's accesses are consecutive doubles.
// For cells of at most KS_MAX faces (the launcher falls back to
// k_grad_limiter otherwise).
constexpr int KS_MAX = 8;
constexpr int KS_VALS = 8;  // r_own 3, n 3, T and pg across the face
__host__ __device__ inline size_t grad_staged_smem(int K, bool wrec) {
  return size_t(K) * GRAD_THREADS * (KS_VALS * sizeof(double) + sizeof(int32_t)) +
         (wrec ? size_t(GRAD_THREADS) * GPS * sizeof(double) : 0);
}
template <bool WREC>
__global__ void __launch_bounds__(GRAD_THREADS, 4)
k_grad_staged(MeshView M, const double* __restrict__ q, const double* __restrict__ qb, int limiter,
              double Kl, Gas gas, double* __restrict__ grad, double* __restrict__ qf) {
  extern __shared__ __align__(16) unsigned char gsm[];
  const int K = M.K;
  const int t = threadIdx.x;
  double* sv = reinterpret_cast<double*>(gsm);                                 // [K][8][T]
  int32_t* se = reinterpret_cast<int32_t*>(sv + size_t(K) * KS_VALS * GRAD_THREADS);  // [K][T]
  double* sr = WREC ? reinterpret_cast<double*>(gsm + size_t(K) * GRAD_THREADS * (KS_VALS * 8 + 4)) : nullptr;
  auto V = [&](int j, int v) -> double& { return sv[(size_t(j) * KS_VALS + v) * GRAD_THREADS + t]; };
  const int64_t c0 = int64_t(blockIdx.x) * GRAD_THREADS;
  const int64_t c = c0 + t;
  const int64_t nf = M.nf;
  if (c < M.nc) {
    double qc[5];
    q_arr(load_q(q, c), qc);
    double b[15], qmax[5], qmin[5];
#pragma unroll
    for (int k = 0; k < 15; ++k) b[k] = 0.0;
#pragma unroll
    for (int k = 0; k < 5; ++k) qmax[k] = qmin[k] = qc[k];
    // ---- pass 1: gradient sums and bounds; stage the face data.  All
    // entries and neighbours first (coalesced), then the faces two at a time
    int32_t ents[KS_MAX], nbs[KS_MAX];
#pragma unroll
    for (int j = 0; j < KS_MAX; ++j) {
      const bool in = j < K;
      ents[j] = in ? __ldg(M.ecf + int64_t(j) * M.nc + c) : -1;
      nbs[j] = in ? __ldg(M.enb + int64_t(j) * M.nc + c) : -1;
    }
#pragma unroll
    for (int j = 0; j < KS_MAX; ++j) {
      if (j >= K) break;
      const int32_t ent = ents[j];
      se[size_t(j) * GRAD_THREADS + t] = ent;
      if (ent < 0) continue;
      const int64_t f = ent >> 1;
      const int side = ent & 1;
      const bool bnd = f >= M.nfi;
      const double* p = bnd ? qb + 5 * (f - M.nfi) : q + 5 * int64_t(nbs[j] < 0 ? 0 : nbs[j]);
      double qn[5], d[3];
#pragma unroll
      for (int k = 0; k < 5; ++k) qn[k] = __ldg(p + k);
      const double sg = side ? -1.0 : 1.0;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double l = M.rL[k * nf + f], r = M.rR[k * nf + f];
        d[k] = bnd ? l : sg * (l - r);
        V(j, k) = side ? r : l;
        V(j, 3 + k) = M.n[k * nf + f];
      }
      V(j, 6) = qn[0];
      V(j, 7) = qn[4];
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        const double dq = qn[k] - qc[k];
        b[3 * k] += d[0] * dq;
        b[3 * k + 1] += d[1] * dq;
        b[3 * k + 2] += d[2] * dq;
        qmax[k] = dmax(qmax[k], qn[k]);
        qmin[k] = dmin(qmin[k], qn[k]);
      }
    }
    const double m0 = M.Minv[c], m1 = M.Minv[M.nc + c], m2 = M.Minv[2 * M.nc + c],
                 m3 = M.Minv[3 * M.nc + c], m4 = M.Minv[4 * M.nc + c], m5 = M.Minv[5 * M.nc + c];
    double g[15];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      const double bx = b[3 * k], by = b[3 * k + 1], bz = b[3 * k + 2];
      g[3 * k] = m0 * bx + m1 * by + m2 * bz;
      g[3 * k + 1] = m1 * bx + m3 * by + m4 * bz;
      g[3 * k + 2] = m2 * bx + m4 * by + m5 * bz;
    }
    // ---- pass 2: limiter over the staged face vectors
    double ph[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) ph[k] = limiter == FPSI_LIMITER_ZERO ? 0.0 : 1.0;
    if (limiter == FPSI_LIMITER_VENKATAKRISHNAN || limiter == FPSI_LIMITER_BARTH) {
      const double h = cbrt(M.vol[c]);
      const double kh = Kl * h;
      const double eps2 = kh * kh * kh;
      for (int j = 0; j < K; ++j) {
        if (se[size_t(j) * GRAD_THREADS + t] < 0) continue;
        const double rx = V(j, 0), ry = V(j, 1), rz = V(j, 2);
#pragma unroll
        for (int k = 0; k < 5; ++k) {
          const double d2 = g[3 * k] * rx + g[3 * k + 1] * ry + g[3 * k + 2] * rz;
          // min(1, a / b) divides only where the ratio is below 1
          double p = 1.0;
          if (d2 != 0.0) {
            const double d1 = d2 > 0 ? qmax[k] - qc[k] : qmin[k] - qc[k];
            if (limiter == FPSI_LIMITER_BARTH) {
              if (d2 > 0 ? d1 < d2 : d1 > d2) p = d1 / d2;
            } else {
              const double num = (d1 * d1 + eps2) + 2.0 * d2 * d1;
              const double den = d1 * d1 + 2.0 * d2 * d2 + d1 * d2 + eps2;
              if (num < den) p = num / den;
            }
          }
          ph[k] = dmin(ph[k], p);
        }
      }
    }
    // ---- pass 3: face states from the staged data
    for (int j = 0; j < K; ++j) {
      const int32_t ent = se[size_t(j) * GRAD_THREADS + t];
      if (ent < 0) continue;
      const int64_t f = ent >> 1;
      const int side = ent & 1;
      const double rx = V(j, 0), ry = V(j, 1), rz = V(j, 2);
      const double nx = V(j, 3), ny = V(j, 4), nz = V(j, 5);
      const double Tn = V(j, 6), pn = V(j, 7);
      double l[5];
#pragma unroll
      for (int k = 0; k < 5; ++k) l[k] = qc[k] + ph[k] * (g[3 * k] * rx + g[3 * k + 1] * ry + g[3 * k + 2] * rz);
      l[0] = dmax(l[0], 0.1 * dmin(side ? Tn : qc[0], side ? qc[0] : Tn));
      l[4] = dmax(l[4], 0.1 * dmin(side ? pn : qc[4], side ? qc[4] : pn) - 0.9 * gas.pamb);
      double* o = qf + int64_t(QFREC) * f;
      side_record(o + (QFREC / 2) * side, l, side_maxev(qc, nx, ny, nz, gas));
      if (f >= M.nfi) {
        double qbs[5];
        const double* p = qb + 5 * (f - M.nfi);
#pragma unroll
        for (int k = 0; k < 5; ++k) qbs[k] = __ldg(p + k);
        side_record(o + QFREC / 2, qbs, side_maxev(qbs, nx, ny, nz, gas));
      }
    }
    if (WREC) {
#pragma unroll
      for (int k = 0; k < 15; ++k) sr[GPS * t + k] = g[k];
#pragma unroll
      for (int k = 0; k < 5; ++k) sr[GPS * t + 15 + k] = ph[k];
    }
  }
  if (WREC) {
    __syncthreads();
    const int cnt = int(min(int64_t(GRAD_THREADS), M.nc - c0));
    for (int i = t; i < GPREC * cnt; i += GRAD_THREADS) grad[GPREC * c0 + i] = sr[GPS * (i / GPREC) + i % GPREC];
  }
}

// The two reconstructed states of a face and their spectral radii, from
// the face record the gradient kernel wrote (six aligned 16 B loads).
struct FaceStates {
  Q5 L, R;
  double mL, mR;
};
__device__ __forceinline__ void load_face_states(const double* __restrict__ qf, int64_t f,
                                                 FaceStates& s) {
  const double2* p = reinterpret_cast<const double2*>(qf + int64_t(QFREC) * f);
  const double2 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
  const double2 d = __ldg(p + 3), e = __ldg(p + 4), h = __ldg(p + 5);
  s.L.T = a.x, s.L.u = a.y, s.L.v = b.x, s.L.w = b.y, s.L.p = c.x, s.mL = c.y;
  s.R.T = d.x, s.R.u = d.y, s.R.v = e.x, s.R.w = e.y, s.R.p = h.x, s.mR = h.y;
}

// ---------------------------------------------------------------------------
// viscous face flux (fluxViscous.loci:112-310) and its thin-layer Jacobian
// (:315-448).  Face gradients (Loci FVM gradv3d_f / grads_f) are the mean of
// the two cell gradients with the component along d = x_R - x_L replaced
// by the difference quotient; at boundary faces the cell gradient corrected
// the same way towards the face state.
// ---------------------------------------------------------------------------
struct Visc {
  int on;  // 0 inviscid, 1 laminar, 2 turbulent
  double a1, a2, a3, k1, k2, k3, cp_prt;
  const double* tmu;
};

struct VFace {
  double vf[4];   // momentum x,y,z and energy (added to src[cl], taken from src[cr])
  double uf[3];
  double muT, kT, dist;
};

__device__ __forceinline__ double suth(double T, double a1, double a2, double a3) {
  return a1 * pow(T, a2) / (T + a3);
}

__device__ __forceinline__ int bc_kind(const MeshView& M, int64_t f) {
  return f >= M.nfi ? M.bcs[-M.cr[f] - 1].kind : 0;
}

__device__ VFace viscous_face(const MeshView& M, const double* __restrict__ q,
                              const double* __restrict__ qb, const double* __restrict__ grad,
                              const Visc& V, int64_t f) {
  VFace o;
  const int64_t nf = M.nf;
  const double n[3] = {M.n[f], M.n[nf + f], M.n[2 * nf + f]};
  const double A = M.area[f];
  const int64_t a = M.cl[f];
  double qa[5];
  q_arr(load_q(q, a), qa);
  const double* ga = grad + GPREC * a;
  // face gradients of T, u, v, w (rows 0..3 of the cell gradient)
  double gf[4][3];
  double muf, kf, tmuf = 0.0;
  const int kind = bc_kind(M, f);
  if (kind == 0) {
    const int64_t b = M.cr[f];
    double qc[5];
    q_arr(load_q(q, b), qc);
    const double* gb = grad + GPREC * b;
    const double vl = M.vol[a], vr = M.vol[b];
    const double iv = 1.0 / (vl + vr);
    muf = (vl * suth(qc[0], V.a1, V.a2, V.a3) + vr * suth(qa[0], V.a1, V.a2, V.a3)) / (vl + vr);
    kf = (vl * suth(qc[0], V.k1, V.k2, V.k3) + vr * suth(qa[0], V.k1, V.k2, V.k3)) / (vl + vr);
    if (V.on == 2) tmuf = (V.tmu[b] * vl + V.tmu[a] * vr) / (vr + vl);
    for (int k = 0; k < 3; ++k) o.uf[k] = iv * (vl * qc[1 + k] + vr * qa[1 + k]);
    double d[3], d2 = 0;
    for (int k = 0; k < 3; ++k) {
      d[k] = M.rL[k * nf + f] - M.rR[k * nf + f];
      d2 += d[k] * d[k];
    }
    o.dist = n[0] * d[0] + n[1] * d[1] + n[2] * d[2];
    for (int v = 0; v < 4; ++v) {
      double gm[3];
      for (int k = 0; k < 3; ++k) gm[k] = 0.5 * (ga[3 * v + k] + gb[3 * v + k]);
      const double c = ((qc[v] - qa[v]) - (gm[0] * d[0] + gm[1] * d[1] + gm[2] * d[2])) / d2;
      for (int k = 0; k < 3; ++k) gf[v][k] = gm[k] + c * d[k];
    }
  } else {
    const double* pb = qb + 5 * (f - M.nfi);
    double qf[5];
    for (int k = 0; k < 5; ++k) qf[k] = pb[k];
    muf = suth(qf[0], V.a1, V.a2, V.a3);
    kf = suth(qf[0], V.k1, V.k2, V.k3);
    if (V.on == 2 && kind != FPSI_BC_VISCOUS_WALL) tmuf = V.tmu[a];
    for (int k = 0; k < 3; ++k) o.uf[k] = qf[1 + k];
    double r[3], r2 = 0;
    for (int k = 0; k < 3; ++k) {
      r[k] = M.rL[k * nf + f];
      r2 += r[k] * r[k];
    }
    o.dist = n[0] * r[0] + n[1] * r[1] + n[2] * r[2];
    for (int v = 0; v < 4; ++v) {
      const double* gv = ga + 3 * v;
      const double c = ((qf[v] - qa[v]) - (gv[0] * r[0] + gv[1] * r[1] + gv[2] * r[2])) / r2;
      for (int k = 0; k < 3; ++k) gf[v][k] = gv[k] + c * r[k];
    }
  }
  o.muT = muf + tmuf;
  o.kT = kf + (V.on == 2 ? tmuf * V.cp_prt : 0.0);
  if (kind == FPSI_BC_REFLECTING) {  // symmetry: no viscous flux (fluxViscous.loci:294-297)
    for (int k = 0; k < 4; ++k) o.vf[k] = 0.0;
    return o;
  }
  const double mt = o.muT;
  const double dudx = gf[1][0], dvdy = gf[2][1], dwdz = gf[3][2];
  const double dvdx = gf[2][0], dwdx = gf[3][0], dwdy = gf[3][1];
  const double dudy = gf[1][1], dudz = gf[1][2], dvdz = gf[2][2];
  const double divm = (dudx + dvdy + dwdz) * (1. / 3.);
  const double txx = 2.0 * mt * (dudx - divm), tyy = 2.0 * mt * (dvdy - divm),
               tzz = 2.0 * mt * (dwdz - divm);
  const double txy = mt * (dudy + dvdx), txz = mt * (dudz + dwdx), tyz = mt * (dvdz + dwdy);
  o.vf[0] = (txx * n[0] + txy * n[1] + txz * n[2]) * A;
  o.vf[1] = (txy * n[0] + tyy * n[1] + tyz * n[2]) * A;
  o.vf[2] = (txz * n[0] + tyz * n[1] + tzz * n[2]) * A;
  o.vf[3] = (o.uf[0] * o.vf[0] + o.uf[1] * o.vf[1] + o.uf[2] * o.vf[2]);
  // conduction; an adiabatic wall carries -qwall*A = 0 instead (bcViscousWall.loci:172-184)
  if (kind != FPSI_BC_VISCOUS_WALL)
    o.vf[3] += (gf[0][0] * n[0] + gf[0][1] * n[1] + gf[0][2] * n[2]) * o.kT * A;
  return o;
}

// Adds sgn * (thin-layer viscous Jacobian) to a block stored in TB, one
// rounding per term as the reference's += on real_fj blocks.
template <class TB>
__device__ __forceinline__ void add_visc_jac(TB* M, const VFace& v, const double n[3], double A,
                                             double sgn) {
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

// ---------------------------------------------------------------------------
// face flux + spectral radius, one thread per face
// ---------------------------------------------------------------------------
// KIND: the Riemann solver (fpsi_flux_kind), a template parameter so that
// each instantiation holds only its own solver's registers
// the low-dissipation fluxes' switches (fluxLowDiss.loci:82-120, 434-437)
struct Lds {
  double comp, dlim, ducros, upwind, nscoeff, nsfactor, filter, ssf;
};

// The inviscid flux of face f from its two face states: the pressure of a
// viscous wall, the analytic flux of the total-pressure and fixed-mass
// conditions' boundary state, the low-dissipation fluxes on interior faces
// (HLLC on boundary faces), or the Riemann solver KIND.
template <int KIND>
__device__ __forceinline__ void inviscid_face_flux(const MeshView& M, const double* __restrict__ q,
                                                   const double* __restrict__ grad, const FaceStates& s,
                                                   int64_t f, double nx, double ny, double nz, double A,
                                                   const Gas& g, const double* __restrict__ adiss,
                                                   const float* __restrict__ ageom, const Lds& P,
                                                   double fl[5]) {
  const int bk = bc_kind(M, f);
  if (bk == FPSI_BC_VISCOUS_WALL) {
    // pressure only, from the cell-centre pressure (bcViscousWall.loci:220-230),
    // which the wall's boundary state carries
    const double p = s.R.p;
    fl[0] = 0.0, fl[1] = p * nx * A, fl[2] = p * ny * A, fl[3] = p * nz * A, fl[4] = 0.0;
  } else if (bk >= FPSI_BC_ISENTROPIC_INFLOW) {
    // the total-pressure and fixed-mass conditions take the analytic flux of
    // their boundary state (bcIsentropic.loci:162-167, bcFixedMass.loci:155-160,
    // bcFixedMassOutflow.loci:152-157)
    state_flux(s.R, nx, ny, nz, A, g, fl);
  } else if (KIND == FPSI_FLUX_KEC || KIND == FPSI_FLUX_SSF) {
    if (f < M.nfi) {
      const int64_t a = M.cl[f], b = M.cr[f];
      const double lx = M.rL[f], ly = M.rL[M.nf + f], lz = M.rL[2 * M.nf + f];
      const double rx = M.rR[f], ry = M.rR[M.nf + f], rz = M.rR[2 * M.nf + f];
      // dv = x_f - (x_l + x_r)/2, d2 = x_r - x_l
      const double dvx = 0.5 * (lx + rx), dvy = 0.5 * (ly + ry), dvz = 0.5 * (lz + rz);
      if (KIND == FPSI_FLUX_KEC)
        kec_face(s.L, s.R, load_q(q, a), load_q(q, b), grad + GPREC * a, grad + GPREC * b, dvx, dvy,
                 dvz, adiss[a], adiss[b], double(ageom[f]), nx, ny, nz, A, g, fl);
      else
        ssf_face(s.L, s.R, load_q(q, a), load_q(q, b), grad + GPREC * a, grad + GPREC * b, dvx, dvy,
                 dvz, lx - rx, ly - ry, lz - rz, adiss[a], adiss[b], double(ageom[f]), P.ssf,
                 P.filter, nx, ny, nz, A, g, fl);
    } else {
      riemann1(FPSI_FLUX_HLLC, s.L, s.R, nx, ny, nz, A, g, fl);  // inviscidRiemannFlux
    }
  } else {
    riemann1(KIND, s.L, s.R, nx, ny, nz, A, g, fl);
  }
}

template <bool VIS, int KIND>
__global__ void k_face_flux(MeshView M, const double* __restrict__ q,
                            const double* __restrict__ qb, const double* __restrict__ grad,
                            const double* __restrict__ qf, Gas g, Visc V, double* __restrict__ F,
                            const double* __restrict__ adiss, const float* __restrict__ ageom,
                            Lds P) {
  const int64_t f = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (f >= M.nf) return;
  FaceStates s;
  load_face_states(qf, f, s);
  const double nx = M.n[f], ny = M.n[M.nf + f], nz = M.n[2 * M.nf + f];
  const double A = M.area[f];
  double fl[5];
  inviscid_face_flux<KIND>(M, q, grad, s, f, nx, ny, nz, A, g, adiss, ageom, P, fl);
  if constexpr (VIS) {
    const VFace v = viscous_face(M, q, qb, grad, V, f);
#pragma unroll
    for (int k = 0; k < 4; ++k) fl[1 + k] -= v.vf[k];
  }
  // maxev_f (solverSetup.loci:81-105): the larger spectral radius of the
  // two sides; a boundary face has only its boundary state's
  const double m = f < M.nfi ? dmax(s.mL, s.mR) : s.mR;
  double2* o = reinterpret_cast<double2*>(F + FREC * f);
  o[0] = make_double2(fl[0], fl[1]);
  o[1] = make_double2(fl[2], fl[3]);
  o[2] = make_double2(fl[4], m * A);
}

// ---------------------------------------------------------------------------
// low-dissipation (KEC) switches
// ---------------------------------------------------------------------------

// alpha_geom_f (fluxLowDiss.loci:122-138) of each interior face, stored in
// FP32 like the reference's store<realF>: with df = x_r - x_l and dv = x_f -
// (x_l + x_r)/2, cos a = min(sqrt(max(1 - 2|dv|/|df|, 0)), n.df/|df|),
// x = min(c (1 - cos a), 1), alpha = x^2 + s (x^3 - 2 x^2 + x), s = factor/max(c, 1)
__global__ void k_alpha_geom(MeshView M, Lds P, float* __restrict__ ag) {
  const int64_t f = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (f >= M.nfi) return;
  const int64_t nf = M.nf;
  double df[3], dv[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double l = M.rL[k * nf + f], r = M.rR[k * nf + f];
    df[k] = l - r;
    dv[k] = 0.5 * (l + r);
  }
  const double ndv = sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
  const double ndf = sqrt(df[0] * df[0] + df[1] * df[1] + df[2] * df[2]);
  const double ndotdf = M.n[f] * df[0] + M.n[nf + f] * df[1] + M.n[2 * nf + f] * df[2];
  const double cosa = dmin(sqrt(dmax(1. - 2. * ndv / ndf, 0.0)), ndotdf / ndf);
  const double scale = P.nscoeff;
  const double sf = P.nsfactor / dmax(scale, 1.0);
  const double x = dmin(scale * (1. - cosa), 1.0);
  const double x2 = x * x, x3 = x2 * x;
  ag[f] = float(x2 + sf * (x3 - 2. * x2 + x));
}

// alpha_diss (fluxLowDiss.loci:141-176) of each cell from its velocity
// divergence veldiv, the sum over its faces of +-ufn (fluxLowDiss.loci:61-78;
// interior faces: the mean velocity plus the face gradient of u times dv =
// x_f - (x_l + x_r)/2, boundary faces: the boundary velocity; dotted with the
// area vector, + on the cl side), the vorticity magnitude of the cell
// gradient (solverTurbulence.loci:45-79), the sound speed and twice the
// largest distance from the cell centre to its face centres.
constexpr int AD_THREADS = 128;
__global__ void __launch_bounds__(AD_THREADS)
k_alpha_diss(MeshView M, const double* __restrict__ q, const double* __restrict__ qb,
             const double* __restrict__ grad, Gas g, Lds P, double* __restrict__ adiss) {
  const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= M.nc) return;
  const int64_t nf = M.nf;
  double veldiv = 0.0, maxd2 = 0.0;
  // the cell's own velocity and velocity gradient rows, loaded once
  double uo[5], go[12];
  q_arr(load_q(q, c), uo);
#pragma unroll
  for (int k = 0; k < 12; ++k) go[k] = grad[GPREC * c + k];
  for (int j0 = 0; j0 < M.K; j0 += ECH) {
    EChunk ch;
    load_chunk(M, c, j0, ch, true);
#pragma unroll
    for (int i = 0; i < ECH; ++i) {
      if (ch.ent[i] < 0) continue;
      const int64_t f = ch.f[i];
      const int side = ch.ent[i] & 1;
      double rl[3], rr[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) rl[k] = M.rL[k * nf + f], rr[k] = M.rR[k * nf + f];
      const double* ro = side ? rr : rl;
      maxd2 = dmax(maxd2, ro[0] * ro[0] + ro[1] * ro[1] + ro[2] * ro[2]);
      const double n[3] = {M.n[f], M.n[nf + f], M.n[2 * nf + f]};
      const double A = M.area[f];
      double ufn;
      if (f < M.nfi) {
        // the neighbour's velocity and gradient rows; l is the cl side
        double qnb[5], gn[12];
        q_arr(load_q(q, ch.nb[i]), qnb);
#pragma unroll
        for (int k = 0; k < 12; ++k) gn[k] = grad[GPREC * int64_t(ch.nb[i]) + k];
        const double* ua = side ? qnb : uo;
        const double* ub = side ? uo : qnb;
        const double* ga = side ? gn : go;
        const double* gb = side ? go : gn;
        double d[3], d2 = 0.0, dv[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          d[k] = rl[k] - rr[k];
          d2 += d[k] * d[k];
          dv[k] = 0.5 * (rl[k] + rr[k]);
        }
        double un = 0.0;
#pragma unroll
        for (int v = 1; v < 4; ++v) {
          double gm[3];
#pragma unroll
          for (int k = 0; k < 3; ++k) gm[k] = 0.5 * (ga[3 * v + k] + gb[3 * v + k]);
          const double cq = ((ub[v] - ua[v]) - (gm[0] * d[0] + gm[1] * d[1] + gm[2] * d[2])) / d2;
          double gf[3];
#pragma unroll
          for (int k = 0; k < 3; ++k) gf[k] = gm[k] + cq * d[k];
          const double uf = 0.5 * (ua[v] + ub[v]) + (gf[0] * dv[0] + gf[1] * dv[1] + gf[2] * dv[2]);
          un += uf * n[v - 1];
        }
        ufn = un * A;
      } else {
        const double* pb = qb + 5 * (f - M.nfi);
        ufn = (pb[1] * n[0] + pb[2] * n[1] + pb[3] * n[2]) * A;
      }
      veldiv += side ? -ufn : ufn;
    }
  }
  const Q5 qc = load_q(q, c);
  const double* gc = grad + GPREC * c;
  const double V = M.vol[c];
  const double len = 2. * sqrt(maxd2);
  const double snd = sqrt(g.gamma * g.Rt * qc.T);
  const double factor = P.comp * fabs(veldiv) * len / (snd * V);
  const double alpha_comp = factor * factor;
  const double theta2 = veldiv * veldiv / (V * V);
  const double wx = gc[10] - gc[8], wy = gc[5] - gc[9], wz = gc[6] - gc[4];
  const double vm = sqrt(wx * wx + wy * wy + wz * wz);
  const double alpha_ducro = P.ducros * theta2 / (theta2 + vm * vm + 1e-10);
  double al = dmax(alpha_ducro, alpha_comp);
  al = dmin(al, P.dlim);
  adiss[c] = dmax(al, P.upwind);
}

// ---------------------------------------------------------------------------
// per-cell residual gather, local time step and norm partials
// ---------------------------------------------------------------------------
constexpr int NORM_THREADS = 256;

template <bool BDF>
__global__ void __launch_bounds__(NORM_THREADS)
// qn, qnm1 (time-accurate BDF2, else null): the states of time levels n
// and n-1; src then receives the rhs with the time terms
// (solverTimestep.loci:397-428), and the norms are the rhs's
// (solverResidual.loci:113-150), while dtau is still the spatial src's
k_cell_residual(MeshView M, const double* __restrict__ q, const double* __restrict__ F,
                Gas g, double urelax, double dtmax,
                double cflmax, double vol_tot, const double* __restrict__ qn,
                const double* __restrict__ qnm1, double* __restrict__ src,
                double* __restrict__ dtau, double* __restrict__ part) {
  const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  double rt = 0, et = 0, mt = 0, rmax = 0, emax = 0, mmax = 0;
  double rloc = -1, eloc = -1;
  if (c < M.nc) {
    // the cell's own state and volume are requested before its face records
    const Q5 qc = load_q(q, c);
    const double V = M.vol[c];
    double s[5] = {0, 0, 0, 0, 0};
    double meva = 0;
    // the face records four at a time from the entry-major lists, all four
    // requested before any is summed, then summed in the cell's face order
    auto add = [&](int32_t en, const double2* r3) {
      const double p[5] = {r3[0].x, r3[0].y, r3[1].x, r3[1].y, r3[2].x};
      if (en & 1) {
#pragma unroll
        for (int k = 0; k < 5; ++k) s[k] += p[k];
      } else {
#pragma unroll
        for (int k = 0; k < 5; ++k) s[k] -= p[k];
      }
      meva += r3[2].y;
    };
    for (int j0 = 0; j0 < M.K; j0 += ECH) {
      int32_t ent[ECH];
#pragma unroll
      for (int i = 0; i < ECH; ++i)
        ent[i] = j0 + i < M.K ? __ldg(M.ecf + int64_t(j0 + i) * M.nc + c) : -1;
      double2 rec[ECH][3];
#pragma unroll
      for (int i = 0; i < ECH; ++i) {
        const double2* p2 =
            reinterpret_cast<const double2*>(F + FREC * int64_t(ent[i] >= 0 ? ent[i] >> 1 : 0));
        rec[i][0] = __ldg(p2), rec[i][1] = __ldg(p2 + 1), rec[i][2] = __ldg(p2 + 2);
      }
#pragma unroll
      for (int i = 0; i < ECH; ++i)
        if (ent[i] >= 0) add(ent[i], rec[i]);
    }
    const double cflpdt = 0.5 * meva / V;
    double dt = dtmax;
    if (cflmax > 0) dt = dmin(dt, cflmax / cflpdt);
    // dtau, solverTimestep.loci:302-329 with eta == 1
    const double rvol = 1.0 / V;
    const double p = qc.p + g.pamb, T = qc.T;
    const double rP = 1.0 / (g.Rt * T);
    const double rho = p * rP;
    const double rT = -rho / T;
    const double qk = 0.5 * (qc.u * qc.u + qc.v * qc.v + qc.w * qc.w);
    const double fT = rT * qk, fP = 1.0 / (g.gamma - 1.0) + rP * qk;
    const double cterm = fP * rT - fT * rP;
    const double dsu = s[1] * qc.u + s[2] * qc.v + s[3] * qc.w;
    const double dtemp =
        rvol * (s[0] * (fP * rT) + (dsu - s[4] - 2.0 * qk * s[0]) * (rT * rP)) / (cterm * rT);
    dt = dmin(dt, urelax * T / (fabs(dtemp) + 1e-30));
    const double dp = rvol * (rT * (2.0 * qk * s[0] - dsu + s[4]) - fT * s[0]);
    dt = dmin(dt, urelax * p / (fabs(dp) + 1e-30));
    dtau[c] = dt;
    if (BDF) {
      // BDF2: s - 1.5 (Q(n+1) - Q(n)) V/dt + 0.5 (Q(n) - Q(n-1)) V/dt
      const Q5 a = load_q(qn, c), b = load_q(qnm1, c);
      const double rdtvol = V / dtmax;
      const double w1 = 1.5 * rdtvol, w2 = 0.5 * rdtvol;
      const double rhon = (a.p + g.pamb) / (g.Rt * a.T);
      const double rhonm1 = (b.p + g.pamb) / (g.Rt * b.T);
      const double rhonp1 = rho;
      s[0] = s[0] - w1 * (rhonp1 - rhon) + w2 * (rhon - rhonm1);
      const double up1[3] = {qc.u, qc.v, qc.w}, un[3] = {a.u, a.v, a.w}, um1[3] = {b.u, b.v, b.w};
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const double r1 = rhonp1 * up1[i], r0 = rhon * un[i], rm = rhonm1 * um1[i];
        s[1 + i] = s[1 + i] - w1 * (r1 - r0) + w2 * (r0 - rm);
      }
      const double igm1 = 1.0 / (g.gamma - 1.0);
      const double e1 = rhonp1 * (g.Rt * qc.T * igm1 + qk);
      const double e0 = rhon * (g.Rt * a.T * igm1 + 0.5 * (a.u * a.u + a.v * a.v + a.w * a.w));
      const double em = rhonm1 * (g.Rt * b.T * igm1 + 0.5 * (b.u * b.u + b.v * b.v + b.w * b.w));
      s[4] = s[4] - w1 * (e1 - e0) + w2 * (e0 - em);
    }
    double* so = src + 5 * c;
#pragma unroll
    for (int k = 0; k < 5; ++k) so[k] = s[k];
    // norms (solverResidual.loci:74-112)
    const double w = V / vol_tot;
    const double a0 = rvol * s[0], a4 = rvol * s[4];
    rt = w * (a0 * a0);
    et = w * (a4 * a4);
    double mm = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double a = rvol * s[1 + i];
      if (fabs(mmax) < fabs(a)) mmax = a;
      mm += a * a;
    }
    mt = mm * (w / 3.0);
    rmax = a0, emax = a4;
    rloc = double(c), eloc = double(c);
  }
  // fixed-shape reduction: sums and signed max-abs with lowest-index ties,
  // first across each warp's lanes (shuffles), then across the 8 warps
  const unsigned full = 0xffffffffu;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  auto combine = [&](double& v, double& loc, double ov, double oloc) {
    if (fabs(ov) > fabs(v) || (fabs(ov) == fabs(v) && loc < 0)) v = ov, loc = oloc;
  };
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    rt += __shfl_down_sync(full, rt, off);
    et += __shfl_down_sync(full, et, off);
    mt += __shfl_down_sync(full, mt, off);
    const double orm = __shfl_down_sync(full, rmax, off), orl = __shfl_down_sync(full, rloc, off);
    const double oem = __shfl_down_sync(full, emax, off), oel = __shfl_down_sync(full, eloc, off);
    const double omm = __shfl_down_sync(full, mmax, off);
    combine(rmax, rloc, orm, orl);
    combine(emax, eloc, oem, oel);
    if (fabs(omm) > fabs(mmax)) mmax = omm;
  }
  constexpr int NW = NORM_THREADS / 32;
  __shared__ double sw[8][NW];
  if (lane == 0) {
    sw[0][warp] = rt, sw[1][warp] = et, sw[2][warp] = mt, sw[3][warp] = rmax;
    sw[4][warp] = rloc, sw[5][warp] = emax, sw[6][warp] = eloc, sw[7][warp] = mmax;
  }
  __syncthreads();
  if (warp == 0) {
    const bool in = lane < NW;
    rt = in ? sw[0][lane] : 0.0, et = in ? sw[1][lane] : 0.0, mt = in ? sw[2][lane] : 0.0;
    rmax = in ? sw[3][lane] : 0.0, rloc = in ? sw[4][lane] : -1.0;
    emax = in ? sw[5][lane] : 0.0, eloc = in ? sw[6][lane] : -1.0, mmax = in ? sw[7][lane] : 0.0;
#pragma unroll
    for (int off = NW / 2; off > 0; off >>= 1) {
      rt += __shfl_down_sync(full, rt, off);
      et += __shfl_down_sync(full, et, off);
      mt += __shfl_down_sync(full, mt, off);
      const double orm = __shfl_down_sync(full, rmax, off), orl = __shfl_down_sync(full, rloc, off);
      const double oem = __shfl_down_sync(full, emax, off), oel = __shfl_down_sync(full, eloc, off);
      const double omm = __shfl_down_sync(full, mmax, off);
      combine(rmax, rloc, orm, orl);
      combine(emax, eloc, oem, oel);
      if (fabs(omm) > fabs(mmax)) mmax = omm;
    }
    if (lane == 0) {
      double* o = part + 8 * int64_t(blockIdx.x);
      o[0] = rt, o[1] = et, o[2] = mt, o[3] = rmax, o[4] = rloc, o[5] = emax, o[6] = eloc, o[7] = mmax;
    }
  }
}

// out[0..2] = rms (sqrt of sums), out[3..4] rtmax/loc, out[5..6] etmax/loc,
// out[7] mtmax; written to slot `step` of a per-run history
__global__ void k_norm_final(const double* __restrict__ part, int nblk,
                             int32_t* __restrict__ bcflags, double* __restrict__ out) {
  __shared__ double sh[8][NORM_THREADS];
  const int t = threadIdx.x;
  double a[8] = {0, 0, 0, 0, -1, 0, -1, 0};
  for (int i = t; i < nblk; i += NORM_THREADS) {
    const double* p = part + 8 * int64_t(i);
    a[0] += p[0], a[1] += p[1], a[2] += p[2];
    if (fabs(p[3]) > fabs(a[3]) || (fabs(p[3]) == fabs(a[3]) && a[4] < 0)) a[3] = p[3], a[4] = p[4];
    if (fabs(p[5]) > fabs(a[5]) || (fabs(p[5]) == fabs(a[5]) && a[6] < 0)) a[5] = p[5], a[6] = p[6];
    if (fabs(p[7]) > fabs(a[7])) a[7] = p[7];
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) sh[k][t] = a[k];
  __syncthreads();
  for (int st = NORM_THREADS / 2; st > 0; st >>= 1) {
    if (t < st) {
      sh[0][t] += sh[0][t + st];
      sh[1][t] += sh[1][t + st];
      sh[2][t] += sh[2][t + st];
      if (fabs(sh[3][t + st]) > fabs(sh[3][t]) ||
          (fabs(sh[3][t + st]) == fabs(sh[3][t]) && sh[4][t + st] >= 0 &&
           (sh[4][t] < 0 || sh[4][t + st] < sh[4][t]))) {
        sh[3][t] = sh[3][t + st];
        sh[4][t] = sh[4][t + st];
      }
      if (fabs(sh[5][t + st]) > fabs(sh[5][t]) ||
          (fabs(sh[5][t + st]) == fabs(sh[5][t]) && sh[6][t + st] >= 0 &&
           (sh[6][t] < 0 || sh[6][t + st] < sh[6][t]))) {
        sh[5][t] = sh[5][t + st];
        sh[6][t] = sh[6][t + st];
      }
      if (fabs(sh[7][t + st]) > fabs(sh[7][t])) sh[7][t] = sh[7][t + st];
    }
    __syncthreads();
  }
  if (t == 0) {
    out[0] = sqrt(sh[0][0]);
    out[1] = sqrt(sh[1][0]);
    out[2] = sqrt(sh[2][0]);
#pragma unroll
    for (int k = 3; k < 8; ++k) out[k] = sh[k][0];
    // the boundary-condition error bits of this residual, cleared for the next
    out[8] = double(*bcflags);
    out[9] = 0.0;
    *bcflags = 0;
  }
}

// ---------------------------------------------------------------------------
// Boundary conditions whose state comes from total conditions or a mass
// flux and whose flux is the state's analytic flux: the Jacobian block of a
// face is the one-sided difference of that flux in the cell-centre state,
// steps 1e-5 of T, a, a, a and a^2 (bcIsentropic.loci:196-239,
// bcFixedMass.loci:163-224); bjac[b] receives the block that srcJ loses.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool fd_jacobian_kind(int kind) {
  return kind == FPSI_BC_ISENTROPIC_INFLOW || kind == FPSI_BC_FIXED_MASS_INFLOW;
}
__device__ __forceinline__ void fd_bc_flux(const fpsi_bc& bc, const double v[5], double nx,
                                           double ny, double nz, double A, const Gas& g,
                                           double F[5]) {
  Q5 qi, qb;
  qi.T = v[0], qi.u = v[1], qi.v = v[2], qi.w = v[3], qi.p = v[4];
  if (bc.kind == FPSI_BC_ISENTROPIC_INFLOW)
    isentropic_state(qi, nx, ny, nz, bc.pg + g.pamb, bc.T, g, qb);
  else
    fixed_mass_state(qi, nx, ny, nz, bc.mass_flux, bc.T, g, qb);
  state_flux(qb, nx, ny, nz, A, g, F);
}
template <class TB>
__global__ void k_bc_fdjac(MeshView M, const double* __restrict__ q, Gas g, TB* __restrict__ bjac) {
  const int64_t b = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b >= M.nf - M.nfi) return;
  const int64_t f = M.nfi + b;
  const fpsi_bc bc = M.bcs[-M.cr[f] - 1];
  if (!fd_jacobian_kind(bc.kind)) return;
  const double nx = M.n[f], ny = M.n[M.nf + f], nz = M.n[2 * M.nf + f], A = M.area[f];
  double v[5];
  q_arr(load_q(q, M.cl[f]), v);
  double F[5], F2[5];
  fd_bc_flux(bc, v, nx, ny, nz, A, g, F);
  const double ai = sqrt(g.gamma * g.Rt * v[0]);
  const double eps = 1e-5;
  const double d[5] = {v[0] * eps, ai * eps, ai * eps, ai * eps, ai * ai * eps};
  TB* J = bjac + 25 * b;
  for (int j = 0; j < 5; ++j) {
    const double t = v[j];
    v[j] += d[j];
    fd_bc_flux(bc, v, nx, ny, nz, A, g, F2);
    const double rh = 1.0 / (t - v[j]);
#pragma unroll
    for (int i = 0; i < 5; ++i) J[5 * i + j] = TB((F[i] - F2[i]) * rh);
    v[j] = t;
  }
}

// ---------------------------------------------------------------------------
// face Jacobians fjp (dir +1) and fjm (dir -1), one thread per face// ---------------------------------------------------------------------------
// face Jacobians fjp (dir +1) and fjm (dir -1), one thread per face
// ---------------------------------------------------------------------------
// The 25 entries of each thread's block are staged in shared memory and the
// CTA's contiguous range of blocks is written back with consecutive threads
// on consecutive addresses (a thread storing its own 100/200 B block would
// touch 25 cache lines per instruction across the warp).
constexpr int JAC_THREADS = 128;

template <class TB, bool VIS>
__global__ void __launch_bounds__(JAC_THREADS)
k_face_jacobian(MeshView M, const double* __restrict__ q, const double* __restrict__ qb,
                const double* __restrict__ grad, const double* __restrict__ qf, Gas g, Visc V,
                TB* __restrict__ fjp, TB* __restrict__ fjm) {
  __shared__ TB stage[JAC_THREADS * 25];
  const int64_t f0 = int64_t(blockIdx.x) * JAC_THREADS;
  const int64_t f = f0 + threadIdx.x;
  const int64_t cnt = min(int64_t(JAC_THREADS), M.nf - f0) * 25;
  const bool live = f < M.nf;
  RoeAvg ra;
  double nx = 0, ny = 0, nz = 0, A = 0;
  if (live) {
    FaceStates s;
    load_face_states(qf, f, s);
    nx = M.n[f], ny = M.n[M.nf + f], nz = M.n[2 * M.nf + f];
    A = M.area[f];
    ra = roe_average1(s.L, s.R, nx, ny, nz, g);
    TB* st = stage + 25 * threadIdx.x;
    const int bk = bc_kind(M, f);
    if (bk == FPSI_BC_VISCOUS_WALL) {
      // d(pressure flux)/dq of the wall (bcViscousWall.loci:232-240); u_f.n = 0
#pragma unroll
      for (int k = 0; k < 25; ++k) st[k] = TB(0);
      st[9] = TB(nx * A), st[14] = TB(ny * A), st[19] = TB(nz * A);
    } else if (fd_jacobian_kind(bk)) {  // the difference block comes from k_bc_fdjac
#pragma unroll
      for (int k = 0; k < 25; ++k) st[k] = TB(0);
    } else {
      jac_roe1<TB>(ra, nx, ny, nz, A, g, +1, st);
    }
    if constexpr (VIS) {
      const double nn[3] = {nx, ny, nz};
      add_visc_jac<TB>(st, viscous_face(M, q, qb, grad, V, f), nn, A, +1.0);
    }
  }
  __syncthreads();
  for (int64_t k = threadIdx.x; k < cnt; k += JAC_THREADS) fjp[25 * f0 + k] = stage[k];
  __syncthreads();
  if (live && f < M.nfi) {
    jac_roe1<TB>(ra, nx, ny, nz, A, g, -1, stage + 25 * threadIdx.x);
    if constexpr (VIS) {
      const double nn[3] = {nx, ny, nz};
      add_visc_jac<TB>(stage + 25 * threadIdx.x, viscous_face(M, q, qb, grad, V, f), nn, A, -1.0);
    }
  }
  __syncthreads();
  // boundary faces have no fjm; their slots are written with whatever the
  // stage holds and never read
  for (int64_t k = threadIdx.x; k < cnt; k += JAC_THREADS) fjm[25 * f0 + k] = stage[k];
}

// Compact face Jacobians of an inviscid system: per face the coefficients of
// fjp (+) and fjm (-) and the shared U, n (CK_FACE values), staged and
// written back like the explicit blocks.  A viscous-wall face's pressure
// block d(p n A)/dpg is c1 = -A with every other coefficient zero.
// One face's compact Jacobian record (CK_FACE values) from its two states:
// the fjp direction (zero on viscous walls but -A on c1, zero on the faces
// whose difference block comes from k_bc_fdjac), the fjm direction on
// interior faces, then the Roe velocity and the normal.
template <class TB>
__device__ __forceinline__ void compact_record(const MeshView& M, int64_t f, const FaceStates& s,
                                               double nx, double ny, double nz, double A, const Gas& g,
                                               TB* st) {
  const RoeAvg ra = roe_average1(s.L, s.R, nx, ny, nz, g);
  const int bk = bc_kind(M, f);
  if (bk == FPSI_BC_VISCOUS_WALL) {
#pragma unroll
    for (int k = 0; k < CK_DIR; ++k) st[k] = TB(0);
    st[CK_C1] = TB(-A);
  } else if (fd_jacobian_kind(bk)) {  // the difference block comes from k_bc_fdjac
#pragma unroll
    for (int k = 0; k < CK_DIR; ++k) st[k] = TB(0);
  } else {
    jac_roe_compact<TB, true>(ra, A, g, +1, st);
  }
  if (f < M.nfi) {
    jac_roe_compact<TB, true>(ra, A, g, -1, st + CK_DIR);
  } else {
#pragma unroll
    for (int k = 0; k < CK_DIR; ++k) st[CK_DIR + k] = TB(0);
  }
  st[2 * CK_DIR] = TB(ra.U), st[2 * CK_DIR + 1] = TB(ra.V), st[2 * CK_DIR + 2] = TB(ra.W);
  st[2 * CK_DIR + 3] = TB(nx), st[2 * CK_DIR + 4] = TB(ny), st[2 * CK_DIR + 5] = TB(nz);
}

template <class TB>
__global__ void __launch_bounds__(JAC_THREADS)
k_face_jacobian_c(MeshView M, const double* __restrict__ qf, Gas g, TB* __restrict__ fjc) {
  __shared__ TB stage[JAC_THREADS * CK_FACE];
  const int64_t f0 = int64_t(blockIdx.x) * JAC_THREADS;
  const int64_t f = f0 + threadIdx.x;
  const int64_t cnt = min(int64_t(JAC_THREADS), M.nf - f0) * CK_FACE;
  if (f < M.nf) {
    FaceStates s;
    load_face_states(qf, f, s);
    const double nx = M.n[f], ny = M.n[M.nf + f], nz = M.n[2 * M.nf + f];
    compact_record<TB>(M, f, s, nx, ny, nz, M.area[f], g, stage + CK_FACE * threadIdx.x);
  }
  __syncthreads();
  for (int64_t k = threadIdx.x; k < cnt; k += JAC_THREADS) fjc[CK_FACE * f0 + k] = stage[k];
}

// The inviscid face flux and the compact Jacobian record of each face in one
// pass over the face-state records (the SGS systems without viscous terms):
// the face states, normal and area are read once, and the flux record and
// the Jacobian record are both written (the latter staged for coalesced
// stores), so the assembly does not launch k_face_jacobian_c.
template <int KIND, class TB>
__global__ void __launch_bounds__(JAC_THREADS)
k_face_flux_jac(MeshView M, const double* __restrict__ q, const double* __restrict__ grad,
                const double* __restrict__ qf, Gas g, double* __restrict__ F,
                const double* __restrict__ adiss, const float* __restrict__ ageom, Lds P,
                TB* __restrict__ fjc) {
  __shared__ TB stage[JAC_THREADS * CK_FACE];
  const int64_t f0 = int64_t(blockIdx.x) * JAC_THREADS;
  const int64_t f = f0 + threadIdx.x;
  const int64_t cnt = min(int64_t(JAC_THREADS), M.nf - f0) * CK_FACE;
  if (f < M.nf) {
    FaceStates s;
    load_face_states(qf, f, s);
    const double nx = M.n[f], ny = M.n[M.nf + f], nz = M.n[2 * M.nf + f];
    const double A = M.area[f];
    double fl[5];
    inviscid_face_flux<KIND>(M, q, grad, s, f, nx, ny, nz, A, g, adiss, ageom, P, fl);
    const double m = f < M.nfi ? dmax(s.mL, s.mR) : s.mR;
    double2* o = reinterpret_cast<double2*>(F + FREC * f);
    o[0] = make_double2(fl[0], fl[1]);
    o[1] = make_double2(fl[2], fl[3]);
    o[2] = make_double2(fl[4], m * A);
    compact_record<TB>(M, f, s, nx, ny, nz, A, g, stage + CK_FACE * threadIdx.x);
  }
  __syncthreads();
  for (int64_t k = threadIdx.x; k < cnt; k += JAC_THREADS) fjc[CK_FACE * f0 + k] = stage[k];
}

// explicit fjp/fjm from the compact face records (boundary faces: fjp only)
template <class TB>
__global__ void k_expand_blocks(int64_t nf, int64_t nfi, const TB* __restrict__ fjc,
                                TB* __restrict__ fjp, TB* __restrict__ fjm) {
  const int64_t f = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  TB r[CK_FACE];
#pragma unroll
  for (int k = 0; k < CK_FACE; ++k) r[k] = fjc[CK_FACE * f + k];
  TB Mb[25];
  compact_expand<TB>(r, r + 2 * CK_DIR, r + 2 * CK_DIR + 3, Mb);
#pragma unroll
  for (int k = 0; k < 25; ++k) fjp[25 * f + k] = Mb[k];
  if (f < nfi) {
    compact_expand<TB>(r + CK_DIR, r + 2 * CK_DIR, r + 2 * CK_DIR + 3, Mb);
#pragma unroll
    for (int k = 0; k < 25; ++k) fjm[25 * f + k] = Mb[k];
  }
}

// ---------------------------------------------------------------------------
// 5x5 LU with partial pivoting and its solve
// ---------------------------------------------------------------------------
template <class TB>
__device__ __forceinline__ bool lu5(TB* A, int* piv) {
  bool ok = true;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    int p = k;
    TB best = fabs(A[5 * k + k]);
#pragma unroll
    for (int i = k + 1; i < 5; ++i) {
      const TB v = fabs(A[5 * i + k]);
      if (v > best) best = v, p = i;
    }
    piv[k] = p;
    if (p != k) {
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        // pivot rows are selected with p known only at run time: swap via
        // a predicated pass over the candidate rows to keep A in registers
        TB tk = A[5 * k + j];
        TB tp = tk;
#pragma unroll
        for (int i = k + 1; i < 5; ++i)
          if (i == p) tp = A[5 * i + j];
#pragma unroll
        for (int i = k + 1; i < 5; ++i)
          if (i == p) A[5 * i + j] = tk;
        A[5 * k + j] = tp;
      }
    }
    const TB d = A[5 * k + k];
    if (d == TB(0)) {
      ok = false;
      continue;
    }
#pragma unroll
    for (int i = k + 1; i < 5; ++i) {
      A[5 * i + k] /= d;
      const TB l = A[5 * i + k];
#pragma unroll
      for (int j = k + 1; j < 5; ++j) A[5 * i + j] -= l * A[5 * k + j];
    }
  }
  return ok;
}

template <class TB, class TX>
__device__ __forceinline__ void lu5_solve(const TB* A, int pv, TX* y) {
  // pivots packed 3 bits each
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const int p = (pv >> (3 * k)) & 7;
    if (p != k) {
      TX tk = y[k], tp = tk;
#pragma unroll
      for (int i = k + 1; i < 5; ++i)
        if (i == p) tp = y[i];
#pragma unroll
      for (int i = k + 1; i < 5; ++i)
        if (i == p) y[i] = tk;
      y[k] = tp;
    }
  }
#pragma unroll
  for (int i = 1; i < 5; ++i)
#pragma unroll
    for (int j = 0; j < i; ++j) y[i] -= TX(A[5 * i + j]) * y[j];
#pragma unroll
  for (int i = 4; i >= 0; --i) {
#pragma unroll
    for (int j = i + 1; j < 5; ++j) y[i] -= TX(A[5 * i + j]) * y[j];
    y[i] /= TX(A[5 * i + i]);
  }
}

// ---------------------------------------------------------------------------
// diagonal block assembly (srcJ sum, steady fluid_D), LU, B and the block
// Jacobi start x0 = D^-1 B; one thread per cell
// ---------------------------------------------------------------------------
struct SweepView {
  const int32_t* ci;     // RCM cell -> colour-order index
  const int32_t* ccol;   // RCM cell -> colour
  const ColInfo* col;    // per colour
};

// Also scatters the off-diagonal blocks into the colour-order slots: row c
// couples to its upper neighbour with U = fjm and to its lower neighbour
// with L = -fjp (solverLinearSystem.loci:57-77).  Threads run in RCM order;
// the cells of one colour inside a warp have consecutive colour positions,
// so every slot store fills whole 32 B sectors.
//
// Face blocks reach the threads through shared memory: for face entry e of
// its 32 cells, a warp copies the (fjp, fjm) pairs with consecutive lanes on
// consecutive words of each 25-entry block, then every thread adds its own
// pair.  Each cell still sums its faces in list order.
constexpr int ASM_THREADS = 128;
constexpr int ASM_STRIDE = 33;  // shared row stride: 32 cells + 1 (no bank conflicts)
constexpr int ASM_BATCH = 10;   // loads in flight per lane while staging
template <class TB>
constexpr size_t asm_smem_bytes() {
  return size_t(ASM_THREADS / 32) * 50 * ASM_STRIDE * sizeof(TB);
}

// CPT: the face blocks come as compact records (fjc, CK_FACE values per
// face) and the slots are written compact (CK_SLOT values); otherwise as
// explicit (fjp, fjm) pairs into 25-value slots.
template <class TB, class TX, bool CPT>
__global__ void __launch_bounds__(ASM_THREADS, sizeof(TB) == 4 ? (CPT ? 5 : 6) : 4)
k_assemble(MeshView M, SweepView S, const double* __restrict__ q, const double* __restrict__ src,
           const double* __restrict__ dtau, const TB* __restrict__ fjp, const TB* __restrict__ fjm,
           const TB* __restrict__ fjc, Gas g, TB* __restrict__ luc, TB* __restrict__ bcv,
           int32_t* __restrict__ pvv, TB* __restrict__ aoff, TB* __restrict__ Dout, TX* __restrict__ x,
           int32_t* __restrict__ err, double dcoef, const TB* __restrict__ bjac) {
  constexpr int RW = 50;  // words staged per face (explicit blocks)
  // compact records move in 16 B units: U16 per record, stored record-major
  // with an odd stride of RS16 units so that a quarter warp's 16 B accesses
  // hit distinct banks
  constexpr int U16 = int(CK_FACE * sizeof(TB) / 16), RS16 = U16 + 1;
  static_assert(CK_FACE * sizeof(TB) % 16 == 0, "a compact record is whole 16 B units");
  static_assert(32 * RS16 * 16 <= 50 * ASM_STRIDE * sizeof(TB), "fits the warp's staging area");
  extern __shared__ __align__(16) unsigned char asm_smem[];
  TB* st = reinterpret_cast<TB*>(asm_smem) + (threadIdx.x >> 5) * (50 * ASM_STRIDE);
  uint4* st4 = reinterpret_cast<uint4*>(asm_smem + (threadIdx.x >> 5) * size_t(32 * RS16 * 16));
  const int lane = threadIdx.x & 31;
  const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const bool active = c < M.nc;
  int32_t e0 = 0, deg = 0;
  int64_t ci = 0, i = 0, ld = 0;
  ColInfo ck{};
  if (active) {
    e0 = M.cf_off[c];
    deg = M.cf_off[c + 1] - e0;
    ci = S.ci[c];
    ck = S.col[S.ccol[c]];
    i = ci - ck.cb;
    ld = ck.ld;
  }
  const int maxdeg = __reduce_max_sync(0xffffffffu, deg);
  TB sJ[25];
#pragma unroll
  for (int k = 0; k < 25; ++k) sJ[k] = TB(0);
  int64_t slot = 0;
  for (int e = 0; e < maxdeg; ++e) {
    const int32_t my_ent = e < deg ? M.cf[e0 + e] : -1;
    if constexpr (CPT) {
      // the warp's 32 records as 32 * U16 units of 16 B, U16 per lane, all
      // in flight together (lanes without an entry read face 0; their units
      // are never used)
      constexpr int HALF = U16 > 6 ? U16 / 2 : U16;  // units held in registers at once
#pragma unroll
      for (int h = 0; h < U16; h += HALF) {
        uint4 v[HALF];
#pragma unroll
        for (int u = 0; u < HALF; ++u) {
          const int idx = lane + 32 * (h + u);
          const int L = idx / U16, j = idx - U16 * L;
          const int32_t ent = __shfl_sync(0xffffffffu, my_ent, L);
          const int64_t f = ent >= 0 ? int64_t(ent >> 1) : 0;
          v[u] = __ldg(reinterpret_cast<const uint4*>(fjc + CK_FACE * f) + j);
        }
#pragma unroll
        for (int u = 0; u < HALF; ++u) {
          const int idx = lane + 32 * (h + u);
          const int L = idx / U16, j = idx - U16 * L;
          st4[L * RS16 + j] = v[u];
        }
      }
    } else {
      // 32 RW words per round, RW per lane, in batches of ASM_BATCH
      // independent loads (fjm is allocated for every face, so every address
      // is valid; lanes without an entry read face 0 and their words are
      // never used)
#pragma unroll 1
      for (int b = 0; b < RW / ASM_BATCH; ++b) {
        TB v[ASM_BATCH];
#pragma unroll
        for (int u = 0; u < ASM_BATCH; ++u) {
          const int idx = lane + 32 * (ASM_BATCH * b + u);
          const int L = idx / RW, k = idx - RW * L;
          const int32_t ent = __shfl_sync(0xffffffffu, my_ent, L);
          const int64_t f = ent >= 0 ? int64_t(ent >> 1) : 0;
          v[u] = k < 25 ? __ldg(fjp + 25 * f + k) : __ldg(fjm + 25 * f + (k - 25));
        }
#pragma unroll
        for (int u = 0; u < ASM_BATCH; ++u) {
          const int idx = lane + 32 * (ASM_BATCH * b + u);
          const int L = idx / RW, k = idx - RW * L;
          st[k * ASM_STRIDE + L] = v[u];
        }
      }
    }
    __syncwarp();
    if (CPT && my_ent >= 0) {
      // L = -fjp to the lower neighbour, U = fjm to the upper one, as below,
      // with the slots written compact
      const int64_t f = my_ent >> 1;
      TB r[CK_FACE];
#pragma unroll
      for (int j = 0; j < U16; ++j) reinterpret_cast<uint4*>(r)[j] = st4[lane * RS16 + j];
      TB* ao = aoff ? aoff + CK_SLOT * ck.ebp + slot * CK_SLOT * ld + i : nullptr;
      TB Mb[25];
      if (my_ent & 1) {
        compact_expand<TB>(r + CK_DIR, r + 2 * CK_DIR, r + 2 * CK_DIR + 3, Mb);
#pragma unroll
        for (int k = 0; k < 25; ++k) sJ[k] += Mb[k];
        if (ao) {
#pragma unroll
          for (int k = 0; k < CK_DIR; ++k) ao[k * ld] = -r[k];
#pragma unroll
          for (int k = 0; k < 6; ++k) ao[(CK_DIR + k) * ld] = r[2 * CK_DIR + k];
        }
        ++slot;
      } else {
        compact_expand<TB>(r, r + 2 * CK_DIR, r + 2 * CK_DIR + 3, Mb);
#pragma unroll
        for (int k = 0; k < 25; ++k) sJ[k] -= Mb[k];
        if (f < M.nfi) {
          if (ao) {
#pragma unroll
            for (int k = 0; k < CK_DIR; ++k) ao[k * ld] = r[CK_DIR + k];
#pragma unroll
            for (int k = 0; k < 6; ++k) ao[(CK_DIR + k) * ld] = r[2 * CK_DIR + k];
          }
          ++slot;
        }
      }
    }
    if (!CPT && my_ent >= 0) {
      const int64_t f = my_ent >> 1;
      const TB* sp = st + lane;                    // fjp of the face
      const TB* sm = st + 25 * ASM_STRIDE + lane;  // fjm of the face
      TB* ao = aoff ? aoff + 25 * ck.ebp + slot * 25 * ld + i : nullptr;
      if (my_ent & 1) {
#pragma unroll
        for (int k = 0; k < 25; ++k) sJ[k] += sm[k * ASM_STRIDE];
        if (ao) {
#pragma unroll
          for (int k = 0; k < 25; ++k) ao[k * ld] = -sp[k * ASM_STRIDE];
        }
        ++slot;
      } else {
#pragma unroll
        for (int k = 0; k < 25; ++k) sJ[k] -= sp[k * ASM_STRIDE];
        if (f < M.nfi) {
          if (ao) {
#pragma unroll
            for (int k = 0; k < 25; ++k) ao[k * ld] = sm[k * ASM_STRIDE];
          }
          ++slot;
        }
      }
    }
    __syncwarp();
  }
  if (!active) return;
  if (bjac) {  // difference blocks of the total-pressure and fixed-mass inflows
    for (int e = 0; e < deg; ++e) {
      const int64_t f = M.cf[e0 + e] >> 1;
      if (f < M.nfi || !fd_jacobian_kind(M.bcs[-M.cr[f] - 1].kind)) continue;
      const TB* J = bjac + 25 * (f - M.nfi);
#pragma unroll
      for (int k = 0; k < 25; ++k) sJ[k] -= J[k];
    }
  }
  TB D[25];
#pragma unroll
  for (int i = 0; i < 25; ++i) D[i] = -sJ[i];
  const Q5 qc = load_q(q, c);
  // V / dtau (steady, solverLinearSystem.loci:176-215), 1.5 V / dtau (BDF2, :376-435)
  const double coef = dcoef * M.vol[c] / dtau[c];
  const double T = qc.T, rP = 1.0 / (g.Rt * T);
  const double rho = (qc.p + g.pamb) * rP;
  const double rT = -rho / T;
  const double qk = 0.5 * (qc.u * qc.u + qc.v * qc.v + qc.w * qc.w);
  const double fT = rT * qk, fP = 1.0 / (g.gamma - 1.0) + rP * qk;
  // M P^-1 (solverLinearSystem.loci:176-215) with reta == 1, pterm == 0
  const double U[3] = {qc.u, qc.v, qc.w};
  D[0] = TB(double(D[0]) + coef * rT);
#pragma unroll
  for (int r = 0; r < 3; ++r) D[5 * (1 + r)] = TB(double(D[5 * (1 + r)]) + coef * rT * U[r]);
  D[20] = TB(double(D[20]) + coef * fT);
  D[4] = TB(double(D[4]) + coef * rP);
#pragma unroll
  for (int r = 0; r < 3; ++r)
    D[5 * (1 + r) + 4] = TB(double(D[5 * (1 + r) + 4]) + coef * rP * U[r]);
  D[24] = TB(double(D[24]) + coef * fP);
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    D[6 * (1 + r)] = TB(double(D[6 * (1 + r)]) + coef * rho);
    D[21 + r] = TB(double(D[21 + r]) + coef * rho * U[r]);
  }
  if (Dout) {
    TB* o = Dout + 25 * c;
#pragma unroll
    for (int i = 0; i < 25; ++i) o[i] = D[i];
  }
  int piv[5];
  if (!lu5<TB>(D, piv)) atomicOr(err, 1);
  int pv = 0;
#pragma unroll
  for (int k = 0; k < 5; ++k) pv |= piv[k] << (3 * k);
  TB Bv[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) Bv[k] = TB(src[5 * c + k]);
  TB* lo = luc + 25 * ck.cbp + i;
#pragma unroll
  for (int k = 0; k < 25; ++k) lo[k * ld] = D[k];
  TB* bo = bcv + 5 * ck.cbp + i;
#pragma unroll
  for (int k = 0; k < 5; ++k) bo[k * ld] = Bv[k];
  pvv[ci] = pv;
  // block Jacobi start D x = B (linearSolverSGS.loci:57-69)
  TX y[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) y[k] = TX(Bv[k]);
  lu5_solve<TB, TX>(D, pv, y);
  TX* xo = x + 5 * ci;
#pragma unroll
  for (int k = 0; k < 5; ++k) xo[k] = y[k];
}

// block Jacobi start alone (a second solve on an assembled system)
template <class TB, class TX>
__global__ void k_jacobi_start(ColInfo ck, const TB* __restrict__ luc,
                               const TB* __restrict__ bcv, const int32_t* __restrict__ pvv,
                               TX* __restrict__ x) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= ck.n) return;
  TB LU[25];
#pragma unroll
  for (int k = 0; k < 25; ++k) LU[k] = luc[25 * ck.cbp + k * ck.ld + i];
  TX y[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) y[k] = TX(bcv[5 * ck.cbp + k * ck.ld + i]);
  lu5_solve<TB, TX>(LU, pvv[ck.cb + i], y);
#pragma unroll
  for (int k = 0; k < 5; ++k) x[5 * (ck.cb + i) + k] = y[k];
}

// ---------------------------------------------------------------------------
// one colour of a Gauss-Seidel sweep (gseidel_forward/backward,
// linearSolverSGS.loci:186-207, 277-298):
//   x_c = D^-1 (B - sum_upper fjm x_cr + sum_lower fjp x_cl)
// ---------------------------------------------------------------------------
// One thread per cell of colour k; every per-cell stream (slots, LU, B,
// pivots, own iterate) is read with consecutive threads on consecutive
// addresses; only the neighbours' iterates are gathered.  The one-pass
// streams are loaded with the streaming hint (evict first) so that the
// iterate, which every colour re-reads, stays resident in L2.
// CPT: slots hold the compact form (CK_SLOT values), applied without
// spelling out the 25 entries.
template <class TB, class TX, bool CPT>
__global__ void k_sgs_colour(ColInfo ck, const int32_t* __restrict__ nbr,
                             const TB* __restrict__ aoff, const TB* __restrict__ luc,
                             const TB* __restrict__ bcv, const int32_t* __restrict__ pvv,
                             TX* __restrict__ x) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t n = ck.n, ld = ck.ld;
  if (i >= n) return;
  // the cell's LU factors and pivots are loaded first, so that they are in
  // flight while the slots are walked; each slot's neighbour id is read one
  // slot ahead
  TB LU[25];
#pragma unroll
  for (int k = 0; k < 25; ++k) LU[k] = __ldcs(luc + 25 * ck.cbp + k * ld + i);
  const int32_t pv = __ldcs(pvv + ck.cb + i);
  TX t[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) t[k] = -TX(__ldcs(bcv + 5 * ck.cbp + k * ld + i));
  int32_t o = ck.m > 0 ? __ldcs(nbr + ck.ebp + i) : -1;
  for (int64_t s = 0; s < ck.m && o >= 0; ++s) {
    const int32_t onext = s + 1 < ck.m ? __ldcs(nbr + ck.ebp + (s + 1) * ld + i) : -1;
    TX xv[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) xv[k] = x[5 * int64_t(o) + k];
    if constexpr (CPT) {
      const TB* A = aoff + CK_SLOT * ck.ebp + s * CK_SLOT * ld + i;
      TB c[CK_SLOT];
#pragma unroll
      for (int k = 0; k < CK_SLOT; ++k) c[k] = __ldcs(A + k * ld);
      compact_apply<TB, TX>(c, xv, t);
    } else {
      const TB* A = aoff + 25 * ck.ebp + s * 25 * ld + i;
#pragma unroll
      for (int r = 0; r < 5; ++r)
#pragma unroll
        for (int j = 0; j < 5; ++j) t[r] += TX(__ldcs(A + (5 * r + j) * ld)) * xv[j];
    }
    o = onext;
  }
  TX y[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) y[k] = -t[k];
  lu5_solve<TB, TX>(LU, pv, y);
  TX* xo = x + 5 * (ck.cb + i);
#pragma unroll
  for (int k = 0; k < 5; ++k) xo[k] = y[k];
}

// ||B - A x||^2 and ||B||^2 per block (A from the unfactored D kept by
// k_assemble and the face blocks)
template <class TB, class TX>
__global__ void __launch_bounds__(NORM_THREADS)
k_linres(MeshView M, const int32_t* __restrict__ xmap, const TB* __restrict__ D,
         const double* __restrict__ src, const TB* __restrict__ fjp, const TB* __restrict__ fjm,
         const TX* __restrict__ x, double* __restrict__ part) {
  const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  double sb = 0, sr = 0;
  if (c < M.nc) {
    const int64_t ci = xmap[c];
    double r[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) r[k] = double(TB(src[5 * c + k]));
#pragma unroll
    for (int k = 0; k < 5; ++k) sb += r[k] * r[k];
#pragma unroll
    for (int i = 0; i < 5; ++i)
#pragma unroll
      for (int j = 0; j < 5; ++j) r[i] -= double(D[25 * c + 5 * i + j]) * double(x[5 * ci + j]);
    for (int32_t e = M.cf_off[c]; e < M.cf_off[c + 1]; ++e) {
      const int32_t ent = M.cf[e];
      const int64_t f = ent >> 1;
      if (f >= M.nfi) continue;
      if (ent & 1) {
        const TX* xn = x + 5 * int64_t(xmap[M.cl[f]]);
#pragma unroll
        for (int i = 0; i < 5; ++i)
#pragma unroll
          for (int j = 0; j < 5; ++j) r[i] += double(fjp[25 * f + 5 * i + j]) * double(xn[j]);
      } else {
        const TX* xn = x + 5 * int64_t(xmap[M.cr[f]]);
#pragma unroll
        for (int i = 0; i < 5; ++i)
#pragma unroll
          for (int j = 0; j < 5; ++j) r[i] -= double(fjm[25 * f + 5 * i + j]) * double(xn[j]);
      }
    }
#pragma unroll
    for (int k = 0; k < 5; ++k) sr += r[k] * r[k];
  }
  __shared__ double sh[2][NORM_THREADS];
  const int t = threadIdx.x;
  sh[0][t] = sb, sh[1][t] = sr;
  __syncthreads();
  for (int st = NORM_THREADS / 2; st > 0; st >>= 1) {
    if (t < st) sh[0][t] += sh[0][t + st], sh[1][t] += sh[1][t + st];
    __syncthreads();
  }
  if (t == 0) part[2 * blockIdx.x] = sh[0][0], part[2 * blockIdx.x + 1] = sh[1][0];
}

__global__ void k_sum2(const double* __restrict__ part, int nblk, double* __restrict__ out) {
  __shared__ double sh[2][NORM_THREADS];
  const int t = threadIdx.x;
  double a = 0, b = 0;
  for (int i = t; i < nblk; i += NORM_THREADS) a += part[2 * i], b += part[2 * i + 1];
  sh[0][t] = a, sh[1][t] = b;
  __syncthreads();
  for (int st = NORM_THREADS / 2; st > 0; st >>= 1) {
    if (t < st) sh[0][t] += sh[0][t + st], sh[1][t] += sh[1][t + st];
    __syncthreads();
  }
  if (t == 0) out[0] = sqrt(sh[0][0]), out[1] = sqrt(sh[1][0]);
}

// ---------------------------------------------------------------------------
// clipped Newton update (solverNewton.loci:62-78)
// ---------------------------------------------------------------------------
// guard (may be null): the norms of the residual this system was built
// from; when they are NaN the state is left as it is, so a run that meets a
// NaN residual keeps the state of that step (solverResidual.loci:203-208
// aborts there)
template <class TX>
__global__ void __launch_bounds__(NORM_THREADS)
// relax: 0.9 (steady, solverNewton.loci:62-78) or 0.75 of T and p (BDF2,
// :163-182, whose floor is max(|d|, 1e-30) instead of |d| + 1e-30)
k_update(int64_t nc, double pamb, const int32_t* __restrict__ ci, const TX* __restrict__ x, double* __restrict__ q,
         double* __restrict__ amin_part, const double* __restrict__ guard, bool bdf,
         const int32_t* __restrict__ flag0, const int32_t* __restrict__ flag1) {
  const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  double alpha = 1.0;
  // the state stays as it is for a step with NaN norms, or (flags given)
  // whose assembly or learned start raised an error bit
  const bool halt = (guard && (isnan(guard[0]) || isnan(guard[1]) || isnan(guard[2]))) ||
                    (flag0 && *flag0 != 0) || (flag1 && *flag1 != 0);
  if (c < nc && !halt) {
    double* qc = q + 5 * c;
    const TX* d = x + 5 * int64_t(ci[c]);
    const double dT = double(d[0]), dp = double(d[4]);
    if (bdf) {
      alpha = dmin(alpha, 0.75 * (qc[4] + pamb) / dmax(fabs(dp), 1e-30));
      alpha = dmin(alpha, 0.75 * qc[0] / dmax(fabs(dT), 1e-30));
    } else {
      alpha = dmin(alpha, 0.9 * qc[0] / (fabs(dT) + 1e-30));
      alpha = dmin(alpha, 0.9 * (qc[4] + pamb) / (fabs(dp) + 1e-30));
    }
    qc[0] += alpha * dT;
    qc[1] += alpha * double(d[1]);
    qc[2] += alpha * double(d[2]);
    qc[3] += alpha * double(d[3]);
    qc[4] += alpha * dp;
  }
  // block minimum: warp shuffles, then one exchange across the warps
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) alpha = dmin(alpha, __shfl_down_sync(0xffffffffu, alpha, off));
  __shared__ double sw[NORM_THREADS / 32];
  if (lane == 0) sw[warp] = alpha;
  __syncthreads();
  if (t == 0) {
    double a = sw[0];
#pragma unroll
    for (int w = 1; w < NORM_THREADS / 32; ++w) a = dmin(a, sw[w]);
    amin_part[blockIdx.x] = a;
  }
}

// caller-order state (T[nc], pg[nc], u[3nc]) <-> device q[nc][5] (RCM order)
__global__ void k_state_in(int64_t nc, const int32_t* __restrict__ perm,
                           const double* __restrict__ stage, double* __restrict__ q) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= nc) return;
  const int64_t c = perm[i];
  double* o = q + 5 * i;
  o[0] = stage[c];
  o[1] = stage[2 * nc + 3 * c];
  o[2] = stage[2 * nc + 3 * c + 1];
  o[3] = stage[2 * nc + 3 * c + 2];
  o[4] = stage[nc + c];
}
__global__ void k_state_out(int64_t nc, const int32_t* __restrict__ perm,
                            const double* __restrict__ q, double* __restrict__ stage) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= nc) return;
  const int64_t c = perm[i];
  const double* p = q + 5 * i;
  stage[c] = p[0];
  stage[2 * nc + 3 * c] = p[1];
  stage[2 * nc + 3 * c + 1] = p[2];
  stage[2 * nc + 3 * c + 2] = p[3];
  stage[nc + c] = p[4];
}

// batched face functions (inviscidFlux.h entry points)
__global__ void k_batch_flux(int kind, int64_t n, const double* __restrict__ qL,
                             const double* __restrict__ qR, const double* __restrict__ an,
                             const double* __restrict__ area, Gas g, double us_n, double eta,
                             double* __restrict__ F) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Q5 L, R;
  L.p = qL[5 * i], L.T = qL[5 * i + 1], L.u = qL[5 * i + 2], L.v = qL[5 * i + 3], L.w = qL[5 * i + 4];
  R.p = qR[5 * i], R.T = qR[5 * i + 1], R.u = qR[5 * i + 2], R.v = qR[5 * i + 3], R.w = qR[5 * i + 4];
  double f[5];
  riemann(kind, L, R, an[3 * i], an[3 * i + 1], an[3 * i + 2], area[i], g, us_n, eta, f);
#pragma unroll
  for (int k = 0; k < 5; ++k) F[5 * i + k] = f[k];
}

template <class TB>
__global__ void k_batch_jac(int64_t n, const double* __restrict__ qL,
                            const double* __restrict__ qR, const double* __restrict__ an,
                            const double* __restrict__ area, Gas g, double us_n, double eta,
                            int dir, TB* __restrict__ out) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Q5 L, R;
  L.p = qL[5 * i], L.T = qL[5 * i + 1], L.u = qL[5 * i + 2], L.v = qL[5 * i + 3], L.w = qL[5 * i + 4];
  R.p = qR[5 * i], R.T = qR[5 * i + 1], R.u = qR[5 * i + 2], R.v = qR[5 * i + 3], R.w = qR[5 * i + 4];
  const double nx = an[3 * i], ny = an[3 * i + 1], nz = an[3 * i + 2];
  const RoeAvg s = roe_average(L, R, nx, ny, nz, g, us_n, eta);
  TB blk[25];
  jac_roe<TB>(s, nx, ny, nz, area[i], g, dir, blk);
#pragma unroll
  for (int k = 0; k < 25; ++k) out[25 * i + k] = blk[k];
}

}  // namespace dev

// ===========================================================================
// host launchers
// ===========================================================================
namespace {
inline unsigned blocks_for(int64_t n, int t) { return unsigned((n + t - 1) / t); }

dev::MeshView view(const fpsi_ctx* x) {
  dev::MeshView M;
  M.nc = x->H.nc;
  M.nf = x->H.nf;
  M.nfi = x->H.nfi;
  M.cl = x->d_cl;
  M.cr = x->d_cr;
  M.n = x->d_n;
  M.area = x->d_area;
  M.rL = x->d_rL;
  M.rR = x->d_rR;
  M.vol = x->d_vol;
  M.Minv = x->d_Minv;
  M.cf_off = x->d_cf_off;
  M.cf = x->d_cf;
  M.K = x->H.ell_k;
  M.ecf = x->d_ecf;
  M.enb = x->d_enb;
  M.bcs = x->d_bcs;
  return M;
}
dev::Visc visc(const fpsi_ctx* x) {
  dev::Visc V;
  V.on = x->P.viscous;
  V.a1 = x->P.mu_a1, V.a2 = x->P.mu_a2, V.a3 = x->P.mu_a3;
  V.k1 = x->P.k_a1, V.k2 = x->P.k_a2, V.k3 = x->P.k_a3;
  V.cp_prt = x->P.gamma * x->P.Rtilde / (x->P.gamma - 1.0) / x->P.Prt;
  V.tmu = x->d_tmu;
  return V;
}
dev::Lds lds(const fpsi_ctx* x) {
  dev::Lds L;
  L.comp = x->P.lds_comp_factor;
  L.dlim = x->P.lds_dissipation_limit;
  L.ducros = x->P.lds_ducros_factor;
  L.upwind = x->P.lds_use_upwind;
  L.nscoeff = x->P.lds_nonsym_coeff;
  L.nsfactor = x->P.lds_nonsym_factor;
  L.filter = x->P.lds_miles_filter;
  L.ssf = x->P.ssf_coeff;
  return L;
}
dev::Gas gas(const fpsi_ctx* x) {
  dev::Gas g;
  g.gamma = x->P.gamma;
  g.Rt = x->P.Rtilde;
  g.pamb = x->P.Pambient;
  return g;
}
}  // namespace

// the gradient, limiter and face-state kernel: the shared-memory staged
// form for cells of at most KS_MAX faces, else the general one
template <bool WREC>
void launch_grad(fpsi_ctx* x, const dev::MeshView& M, cudaStream_t s) {
  const unsigned nb = blocks_for(M.nc, dev::GRAD_THREADS);
  if (M.K <= dev::KS_MAX) {
    static bool attr = false;
    if (!attr) {
      cudaFuncSetAttribute(dev::k_grad_staged<WREC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           int(dev::grad_staged_smem(dev::KS_MAX, true)));
      attr = true;
    }
    dev::k_grad_staged<WREC><<<nb, dev::GRAD_THREADS, dev::grad_staged_smem(M.K, WREC), s>>>(
        M, x->d_q, x->d_qb, x->P.limiter, x->P.Kl, gas(x), x->d_grad, x->d_qf);
  } else {
    dev::k_grad_limiter<WREC><<<nb, dev::GRAD_THREADS, 0, s>>>(M, x->d_q, x->d_qb, x->P.limiter,
                                                               x->P.Kl, gas(x), x->d_grad, x->d_qf);
  }
}

int launch_grad_records(fpsi_ctx* x) {
  const dev::MeshView M = view(x);
  launch_grad<true>(x, M, x->stream);
  FPSI_CUDA_TRY(cudaGetLastError());
  x->grad_valid = true;
  return FPSI_OK;
}

int launch_residual(fpsi_ctx* x, double* resid_slot) {
  const dev::MeshView M = view(x);
  const dev::Gas g = gas(x);
  cudaStream_t s = x->stream;
  const int T = 256;
  if (x->H.nbf > 0) {
    prof_begin(x, "bc_state");
    if (x->any_pmean)
      dev::k_bc_mean<<<unsigned(x->bcs.size()), dev::BCM_THREADS, 0, s>>>(M, x->d_q, x->d_bcmean);
    dev::k_bc_state<<<blocks_for(x->H.nbf, T), T, 0, s>>>(M, x->d_q, x->d_bcs, g, x->d_bcmean,
                                                         x->d_err + 1, x->d_qb);
    prof_end(x);
  }
  const bool kec = x->P.flux == FPSI_FLUX_KEC || x->P.flux == FPSI_FLUX_SSF;
  if (kec) {
    if (!x->d_adiss) {
      FPSI_CUDA_TRY(cudaMalloc(&x->d_adiss, size_t(M.nc) * sizeof(double)));
      FPSI_CUDA_TRY(cudaMalloc(&x->d_ageom, size_t(std::max<int64_t>(M.nfi, 1)) * sizeof(float)));
    }
    if (x->ageom_coeff != x->P.lds_nonsym_coeff || x->ageom_factor != x->P.lds_nonsym_factor) {
      if (M.nfi > 0)
        dev::k_alpha_geom<<<blocks_for(M.nfi, T), T, 0, s>>>(M, lds(x), x->d_ageom);
      x->ageom_coeff = x->P.lds_nonsym_coeff;
      x->ageom_factor = x->P.lds_nonsym_factor;
    }
  }
  prof_begin(x, "grad_limiter");
  // the gradient records are written every residual only where the viscous
  // terms, the SA model and the KEC flux read them
  x->grad_valid = x->P.viscous != 0 || kec;
  if (x->grad_valid)
    launch_grad<true>(x, M, s);
  else
    launch_grad<false>(x, M, s);
  if (kec)
    dev::k_alpha_diss<<<blocks_for(M.nc, dev::AD_THREADS), dev::AD_THREADS, 0, s>>>(
        M, x->d_q, x->d_qb, x->d_grad, g, lds(x), x->d_adiss);
  prof_end(x);
  // an inviscid system relaxed by SGS gets its compact face Jacobian records
  // from the flux kernel, in the same pass over the face states
  x->jac_fresh = 0;
  if (!x->P.viscous && x->P.solver != FPSI_SOLVER_LSGS && x->d_fjc) {
    prof_begin(x, "face_flux_jac");
    const unsigned nb = blocks_for(M.nf, dev::JAC_THREADS);
    const bool f64 = x->P.precision == FPSI_PREC_FP64;
#define FPSI_FLUXJ(K)                                                                              \
  do {                                                                                             \
    if (f64)                                                                                       \
      dev::k_face_flux_jac<K, double><<<nb, dev::JAC_THREADS, 0, s>>>(                             \
          M, x->d_q, x->d_grad, x->d_qf, g, x->d_F, x->d_adiss, x->d_ageom, lds(x), (double*)x->d_fjc); \
    else                                                                                           \
      dev::k_face_flux_jac<K, float><<<nb, dev::JAC_THREADS, 0, s>>>(                              \
          M, x->d_q, x->d_grad, x->d_qf, g, x->d_F, x->d_adiss, x->d_ageom, lds(x), (float*)x->d_fjc); \
  } while (0)
    if (x->P.flux == FPSI_FLUX_ROE) FPSI_FLUXJ(FPSI_FLUX_ROE);
    else if (x->P.flux == FPSI_FLUX_HLLE) FPSI_FLUXJ(FPSI_FLUX_HLLE);
    else if (x->P.flux == FPSI_FLUX_KEC) FPSI_FLUXJ(FPSI_FLUX_KEC);
    else if (x->P.flux == FPSI_FLUX_SSF) FPSI_FLUXJ(FPSI_FLUX_SSF);
    else FPSI_FLUXJ(FPSI_FLUX_HLLC);
#undef FPSI_FLUXJ
    x->jac_fresh = f64 ? 8 : 4;
    prof_end(x);
  } else {
  prof_begin(x, "face_flux");
    // the viscous terms and each Riemann solver are separate instantiations:
    // the inviscid Roe kernel does not carry the others' registers
    {
      const unsigned nb = blocks_for(M.nf, 128);
      const dev::Visc Vv = visc(x);
      double* F = x->d_F;
  #define FPSI_FLUX(VIS, K)                                                                     \
    dev::k_face_flux<VIS, K><<<nb, 128, 0, s>>>(M, x->d_q, x->d_qb, x->d_grad, x->d_qf, g, Vv, F, \
                                                x->d_adiss, x->d_ageom, lds(x))
      if (x->P.viscous) {
        if (x->P.flux == FPSI_FLUX_ROE) FPSI_FLUX(true, FPSI_FLUX_ROE);
        else if (x->P.flux == FPSI_FLUX_HLLE) FPSI_FLUX(true, FPSI_FLUX_HLLE);
        else if (x->P.flux == FPSI_FLUX_KEC) FPSI_FLUX(true, FPSI_FLUX_KEC);
        else if (x->P.flux == FPSI_FLUX_SSF) FPSI_FLUX(true, FPSI_FLUX_SSF);
        else FPSI_FLUX(true, FPSI_FLUX_HLLC);
      } else {
        if (x->P.flux == FPSI_FLUX_ROE) FPSI_FLUX(false, FPSI_FLUX_ROE);
        else if (x->P.flux == FPSI_FLUX_HLLE) FPSI_FLUX(false, FPSI_FLUX_HLLE);
        else if (x->P.flux == FPSI_FLUX_KEC) FPSI_FLUX(false, FPSI_FLUX_KEC);
        else if (x->P.flux == FPSI_FLUX_SSF) FPSI_FLUX(false, FPSI_FLUX_SSF);
        else FPSI_FLUX(false, FPSI_FLUX_HLLC);
      }
  #undef FPSI_FLUX
    }
    prof_end(x);
  }
  prof_begin(x, "cell_residual");
  const bool bdf = x->P.time_accurate != 0;
  if (bdf && !x->have_levels) {
    // the first time step after a new state: Q(n-1) = Q(n) = that state
    FPSI_CUDA_TRY(cudaMemcpyAsync(x->d_qn, x->d_q, size_t(M.nc) * 5 * sizeof(double),
                                  cudaMemcpyDeviceToDevice, s));
    FPSI_CUDA_TRY(cudaMemcpyAsync(x->d_qnm1, x->d_q, size_t(M.nc) * 5 * sizeof(double),
                                  cudaMemcpyDeviceToDevice, s));
    x->have_levels = true;
  }
  if (bdf)
    dev::k_cell_residual<true><<<x->nblk_norm, dev::NORM_THREADS, 0, s>>>(
        M, x->d_q, x->d_F, g, x->P.urelax, x->P.dtmax, x->P.cflmax, x->H.vol_tot, x->d_qn, x->d_qnm1,
        x->d_src, x->d_dtau, x->d_part);
  else
    dev::k_cell_residual<false><<<x->nblk_norm, dev::NORM_THREADS, 0, s>>>(
        M, x->d_q, x->d_F, g, x->P.urelax, x->P.dtmax, x->P.cflmax, x->H.vol_tot, nullptr, nullptr,
        x->d_src, x->d_dtau, x->d_part);
  dev::k_norm_final<<<1, dev::NORM_THREADS, 0, s>>>(x->d_part, x->nblk_norm, x->d_err + 1, resid_slot);
  prof_end(x);
  FPSI_CUDA_TRY(cudaGetLastError());
  return FPSI_OK;
}

static ColInfo col_info(const fpsi_ctx* x, int k) {
  const HostMesh& H = x->H;
  return ColInfo{H.col_cb[k], H.col_n[k], H.col_m[k], H.col_ld[k], H.col_cbp[k], H.col_ebp[k]};
}

static dev::SweepView sweep_view(const fpsi_ctx* x) {
  dev::SweepView S;
  S.ci = x->d_ci;
  S.ccol = x->d_ccol;
  S.col = x->d_colinfo;
  return S;
}

// Inviscid systems relaxed by multi-colour SGS keep their face Jacobians in
// the compact Roe form (15 values per sweep slot instead of 25); viscous
// terms and the line solver need the explicit blocks.
static bool compact_blocks(const fpsi_ctx* x) {
  return !x->P.viscous && x->P.solver != FPSI_SOLVER_LSGS;
}

template <class TB, class TX, bool CPT>
static void launch_assemble_kernel(fpsi_ctx* x, const dev::MeshView& M, const dev::Gas& g) {
  constexpr size_t smem = dev::asm_smem_bytes<TB>();
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(dev::k_assemble<TB, TX, CPT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         int(smem));
  dev::k_assemble<TB, TX, CPT><<<blocks_for(M.nc, dev::ASM_THREADS), dev::ASM_THREADS, smem, x->stream>>>(
      M, sweep_view(x), x->d_q, x->d_src, x->d_dtau, (const TB*)x->d_fjp, (const TB*)x->d_fjm,
      (const TB*)x->d_fjc, g, (TB*)x->d_luc, (TB*)x->d_bc, x->d_pv,
      x->P.solver == FPSI_SOLVER_LSGS ? nullptr : (TB*)x->d_aoff, x->keep_D ? (TB*)x->d_D : nullptr,
      (TX*)x->d_x, x->d_err, x->P.time_accurate ? 1.5 : 1.0,
      x->any_fdbc ? (const TB*)x->d_bjac : nullptr);
}

template <class TB, class TX>
static int launch_assemble_t(fpsi_ctx* x) {
  const dev::MeshView M = view(x);
  const dev::Gas g = gas(x);
  cudaStream_t s = x->stream;
  TB* fjp = (TB*)x->d_fjp;
  TB* fjm = (TB*)x->d_fjm;
  const bool cpt = compact_blocks(x);
  x->asm_compact = cpt;
  x->have_explicit = !cpt;
  // compact records the flux kernel wrote with this residual are kept
  const bool fresh = cpt && x->jac_fresh == int(sizeof(TB));
  if (x->any_fdbc || !fresh) {
    prof_begin(x, "face_jacobian");
    if (x->any_fdbc)
      dev::k_bc_fdjac<TB><<<blocks_for(x->H.nbf, 128), 128, 0, s>>>(M, x->d_q, g, (TB*)x->d_bjac);
    if (!cpt && x->P.viscous)
      dev::k_face_jacobian<TB, true><<<blocks_for(M.nf, dev::JAC_THREADS), dev::JAC_THREADS, 0, s>>>(
          M, x->d_q, x->d_qb, x->d_grad, x->d_qf, g, visc(x), fjp, fjm);
    else if (!cpt)
      dev::k_face_jacobian<TB, false><<<blocks_for(M.nf, dev::JAC_THREADS), dev::JAC_THREADS, 0, s>>>(
          M, x->d_q, x->d_qb, x->d_grad, x->d_qf, g, visc(x), fjp, fjm);
    else if (!fresh)
      dev::k_face_jacobian_c<TB><<<blocks_for(M.nf, dev::JAC_THREADS), dev::JAC_THREADS, 0, s>>>(
          M, x->d_qf, g, (TB*)x->d_fjc);
    prof_end(x);
  }
  prof_begin(x, "assemble_lu");
  if (cpt)
    launch_assemble_kernel<TB, TX, true>(x, M, g);
  else
    launch_assemble_kernel<TB, TX, false>(x, M, g);
  prof_end(x);
  FPSI_CUDA_TRY(cudaGetLastError());
  return FPSI_OK;
}

int launch_assemble(fpsi_ctx* x) {
  int rc;
  switch (x->P.precision) {
    case FPSI_PREC_FP64:
      rc = launch_assemble_t<double, double>(x);
      break;
    case FPSI_PREC_MIXED:
      rc = launch_assemble_t<float, float>(x);
      break;
    default:
      rc = launch_assemble_t<float, double>(x);
  }
  // FSGS starts its sweeps from zero (linearSolverFSGS.loci:1611), the
  // others from the block Jacobi solution the assembly left in x
  if (!rc && x->P.solver == FPSI_SOLVER_FSGS)
    FPSI_CUDA_TRY(cudaMemsetAsync(x->d_x, 0, size_t(x->H.nc) * 5 * x->x_bytes, x->stream));
  return rc;
}

template <class TB, class TX>
static int launch_jacobi_t(fpsi_ctx* x) {
  for (int k = 0; k < x->H.ncolours; ++k) {
    const ColInfo ck = col_info(x, k);
    if (ck.n == 0) continue;
    dev::k_jacobi_start<TB, TX><<<blocks_for(ck.n, 128), 128, 0, x->stream>>>(
        ck, (const TB*)x->d_luc, (const TB*)x->d_bc, x->d_pv, (TX*)x->d_x);
  }
  FPSI_CUDA_TRY(cudaGetLastError());
  return FPSI_OK;
}

int launch_jacobi_start(fpsi_ctx* x) {
  switch (x->P.precision) {
    case FPSI_PREC_FP64:
      return launch_jacobi_t<double, double>(x);
    case FPSI_PREC_MIXED:
      return launch_jacobi_t<float, float>(x);
    default:
      return launch_jacobi_t<float, double>(x);
  }
}

template <class TB, class TX>
// Forward then backward over the colours, `sweeps` times.  A colour's cells
// read only other colours' iterates, so a colour that directly follows
// itself (the turn of each sweep, and the step from one sweep to the next)
// would reproduce the values it just wrote: those launches are skipped and
// the iterate is bitwise the same as with every launch made.
static int launch_sgs_t(fpsi_ctx* x, int sweeps) {
  cudaStream_t s = x->stream;
  const int T = 128;
  const int K = x->H.ncolours;
  int last = -1;
  for (int it = 0; it < sweeps; ++it) {
    for (int pass = 0; pass < 2; ++pass)
      for (int kk = 0; kk < K; ++kk) {
        const int k = pass == 0 ? kk : K - 1 - kk;
        const ColInfo ck = col_info(x, k);
        if (ck.n == 0 || k == last) continue;
        last = k;
        prof_begin(x, "sgs_colour");
        if (x->asm_compact)
          dev::k_sgs_colour<TB, TX, true><<<blocks_for(ck.n, T), T, 0, s>>>(
              ck, x->d_nbr, (const TB*)x->d_aoff, (const TB*)x->d_luc, (const TB*)x->d_bc, x->d_pv,
              (TX*)x->d_x);
        else
          dev::k_sgs_colour<TB, TX, false><<<blocks_for(ck.n, T), T, 0, s>>>(
              ck, x->d_nbr, (const TB*)x->d_aoff, (const TB*)x->d_luc, (const TB*)x->d_bc, x->d_pv,
              (TX*)x->d_x);
        prof_end(x);
      }
  }
  FPSI_CUDA_TRY(cudaGetLastError());
  return FPSI_OK;
}

int launch_sgs(fpsi_ctx* x, int sweeps) {
  switch (x->P.precision) {
    case FPSI_PREC_FP64:
      return launch_sgs_t<double, double>(x, sweeps);
    case FPSI_PREC_MIXED:
      return launch_sgs_t<float, float>(x, sweeps);
    default:
      return launch_sgs_t<float, double>(x, sweeps);
  }
}

template <class TB>
static int expand_blocks_t(fpsi_ctx* x) {
  dev::k_expand_blocks<TB><<<blocks_for(x->H.nf, 128), 128, 0, x->stream>>>(
      x->H.nf, x->H.nfi, (const TB*)x->d_fjc, (TB*)x->d_fjp, (TB*)x->d_fjm);
  FPSI_CUDA_TRY(cudaGetLastError());
  FPSI_CUDA_TRY(cudaStreamSynchronize(x->stream));
  x->have_explicit = true;
  return FPSI_OK;
}

int ensure_explicit_blocks(fpsi_ctx* x) {
  if (x->have_explicit || !x->asm_compact) return FPSI_OK;
  return x->P.precision == FPSI_PREC_FP64 ? expand_blocks_t<double>(x) : expand_blocks_t<float>(x);
}

template <class TB, class TX>
static int launch_linres_t(fpsi_ctx* x, double* out2) {
  const int rc = ensure_explicit_blocks(x);
  if (rc) return rc;
  const dev::MeshView M = view(x);
  const bool lsgs = x->P.solver == FPSI_SOLVER_LSGS;
  dev::k_linres<TB, TX><<<x->nblk_norm, dev::NORM_THREADS, 0, x->stream>>>(
      M, lsgs ? x->d_lt : x->d_ci, (const TB*)x->d_D, x->d_src, (const TB*)x->d_fjp,
      (const TB*)x->d_fjm, (const TX*)(lsgs ? x->d_lx : x->d_x), x->d_part);
  dev::k_sum2<<<1, dev::NORM_THREADS, 0, x->stream>>>(x->d_part, x->nblk_norm, out2);
  FPSI_CUDA_TRY(cudaGetLastError());
  return FPSI_OK;
}

int launch_linres(fpsi_ctx* x, double* out2) {
  switch (x->P.precision) {
    case FPSI_PREC_FP64:
      return launch_linres_t<double, double>(x, out2);
    case FPSI_PREC_MIXED:
      return launch_linres_t<float, float>(x, out2);
    default:
      return launch_linres_t<float, double>(x, out2);
  }
}

int launch_update(fpsi_ctx* x, const double* guard, const int32_t* flag0, const int32_t* flag1) {
  const int64_t nc = x->H.nc;
  const bool lsgs = x->P.solver == FPSI_SOLVER_LSGS;
  const int32_t* map = lsgs ? x->d_lt : x->d_ci;
  const void* xv = lsgs ? x->d_lx : x->d_x;
  prof_begin(x, "update");
  if (x->P.precision == FPSI_PREC_MIXED)
    dev::k_update<float><<<x->nblk_norm, dev::NORM_THREADS, 0, x->stream>>>(
        nc, x->P.Pambient, map, (const float*)xv, x->d_q, x->d_amin, guard, x->P.time_accurate != 0,
        flag0, flag1);
  else
    dev::k_update<double><<<x->nblk_norm, dev::NORM_THREADS, 0, x->stream>>>(
        nc, x->P.Pambient, map, (const double*)xv, x->d_q, x->d_amin, guard, x->P.time_accurate != 0,
        flag0, flag1);
  prof_end(x);
  FPSI_CUDA_TRY(cudaGetLastError());
  if (x->keep_prev && x->d_xprev && !lsgs) {
    FPSI_CUDA_TRY(cudaMemcpyAsync(x->d_xprev, x->d_x, size_t(nc) * 5 * x->x_bytes,
                                  cudaMemcpyDeviceToDevice, x->stream));
    x->have_xprev = true;
  }
  return FPSI_OK;
}

int launch_state(fpsi_ctx* x, bool in) {
  const int64_t nc = x->H.nc;
  if (in)
    dev::k_state_in<<<blocks_for(nc, 256), 256, 0, x->stream>>>(nc, x->d_perm, x->d_stage, x->d_q);
  else
    dev::k_state_out<<<blocks_for(nc, 256), 256, 0, x->stream>>>(nc, x->d_perm, x->d_q, x->d_stage);
  FPSI_CUDA_TRY(cudaGetLastError());
  return FPSI_OK;
}

int launch_batch_flux(int kind, int64_t n, const double* qL, const double* qR, const double* an,
                      const double* area, double pamb, double Rt, double gamma, double us_n,
                      double eta, double* F, cudaStream_t s) {
  dev::Gas g{gamma, Rt, pamb};
  dev::k_batch_flux<<<blocks_for(n, 128), 128, 0, s>>>(kind, n, qL, qR, an, area, g, us_n, eta, F);
  FPSI_CUDA_TRY(cudaGetLastError());
  return FPSI_OK;
}

int launch_batch_jac(int64_t n, const double* qL, const double* qR, const double* an,
                     const double* area, double pamb, double Rt, double gamma, double us_n,
                     double eta, int dir, int as_double, void* out, cudaStream_t s) {
  dev::Gas g{gamma, Rt, pamb};
  if (as_double)
    dev::k_batch_jac<double><<<blocks_for(n, 128), 128, 0, s>>>(n, qL, qR, an, area, g, us_n,
                                                                  eta, dir, (double*)out);
  else
    dev::k_batch_jac<float><<<blocks_for(n, 128), 128, 0, s>>>(n, qL, qR, an, area, g, us_n, eta,
                                                                 dir, (float*)out);
  FPSI_CUDA_TRY(cudaGetLastError());
  return FPSI_OK;
}

}  // namespace fpsi
