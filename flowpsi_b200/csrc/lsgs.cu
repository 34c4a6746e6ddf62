// lsgs.cu -- line symmetric Gauss-Seidel (linearSolverLSGS.loci) on the GPU.
//
// Lines are solved as batched block-tridiagonal systems (block Thomas
// algorithm, one thread per line, 32 lines per group stored position-major
// so that the group's threads read coalesced rows).  Lines are coloured so
// that the lines of one colour are independent; a sweep runs the colours in
// order (forward) and in reverse (backward).  The iteration is the
// reference's solve loop (linearSolverLSGS.loci:1692-1954):
//   * start: every line solved with its own right-hand side B (:1708-1728);
//   * per iteration: forward sweep, backward sweep, relaxation
//     X = w X + (1-w) X_t with X_t the iterate before the backward line solve
//     (:1868-1874), residual ||X - X_t||, w *= 1/rel when rel > 1 (:1935),
//     stop on the absolute or relative tolerance (:1944-1947).
// The stopping test runs on the device (no host round trip per iteration);
// once it fires, the remaining launches of the solve return at entry.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <vector>

#include "fpsi_internal.h"
#include "kernels.cuh"

namespace fpsi {

// ---------------------------------------------------------------------------
// host: lines, colours, groups, roles of the cell's faces
// ---------------------------------------------------------------------------
namespace {

// default lines: link cells that are mutually among each other's two
// strongest couplings, measured geometrically by area / centre distance,
// keeping a second link only when it is within a factor 25 of the first
// (the test of linearSolverLSGS.loci:620).
std::vector<std::vector<int32_t>> default_lines(const HostMesh& H) {
  const int64_t nc = H.nc;
  std::vector<std::array<int32_t, 2>> best(nc, {-1, -1});
  std::vector<std::array<double, 2>> bw(nc, {0.0, 0.0});
  for (int64_t c = 0; c < nc; ++c) {
    for (int32_t e = H.cf_off[c]; e < H.cf_off[c + 1]; ++e) {
      const int64_t f = H.cf[e] >> 1;
      if (H.cr[f] < 0) continue;
      const int32_t o = (H.cf[e] & 1) ? H.cl[f] : H.cr[f];
      double d2 = 0;
      for (int k = 0; k < 3; ++k) {
        const double d = H.rL[3 * f + k] - H.rR[3 * f + k];
        d2 += d * d;
      }
      const double w = H.area[f] / std::sqrt(d2);
      if (w > bw[c][0]) {
        bw[c][1] = bw[c][0], best[c][1] = best[c][0];
        bw[c][0] = w, best[c][0] = o;
      } else if (w > bw[c][1]) {
        bw[c][1] = w, best[c][1] = o;
      }
    }
    if (best[c][1] >= 0 && bw[c][1] * 25.0 <= bw[c][0]) best[c][1] = -1;
  }
  auto mutual = [&](int32_t a, int32_t b) {
    return best[b][0] == a || best[b][1] == a;
  };
  std::vector<std::array<int32_t, 2>> link(nc, {-1, -1});
  for (int64_t c = 0; c < nc; ++c)
    for (int s = 0; s < 2; ++s) {
      const int32_t o = best[c][s];
      if (o >= 0 && mutual(int32_t(c), o)) link[c][s] = o;
    }
  std::vector<char> seen(nc, 0);
  std::vector<std::vector<int32_t>> lines;
  auto degree = [&](int64_t c) { return (link[c][0] >= 0) + (link[c][1] >= 0); };
  // paths from their ends first, then what is left (cycles) cut anywhere
  for (int pass = 0; pass < 2; ++pass)
    for (int64_t s0 = 0; s0 < nc; ++s0) {
      if (seen[s0] || (pass == 0 && degree(s0) > 1)) continue;
      std::vector<int32_t> L;
      int32_t prev = -1, cur = int32_t(s0);
      while (cur >= 0 && !seen[cur]) {
        seen[cur] = 1;
        L.push_back(cur);
        int32_t nxt = -1;
        for (int s = 0; s < 2; ++s)
          if (link[cur][s] >= 0 && link[cur][s] != prev && !seen[link[cur][s]]) {
            nxt = link[cur][s];
            break;
          }
        prev = cur;
        cur = nxt;
      }
      lines.push_back(std::move(L));
    }
  return lines;
}

}  // namespace

int build_lines(fpsi_ctx* x, const std::vector<std::vector<int32_t>>* given) {
  const HostMesh& H = x->H;
  LineLayout& Y = x->LY;
  const int64_t nc = H.nc;
  std::vector<std::vector<int32_t>> lines = given ? *given : default_lines(H);
  // cells not covered become single-cell lines
  std::vector<int32_t> line_of(nc, -1), pos(nc, -1);
  for (size_t l = 0; l < lines.size(); ++l)
    for (size_t p = 0; p < lines[l].size(); ++p) {
      const int32_t c = lines[l][p];
      if (c < 0 || c >= nc || line_of[c] >= 0) {
        set_error("lines: cell %d missing or repeated", c);
        return FPSI_E_INVALID;
      }
      line_of[c] = int32_t(l), pos[c] = int32_t(p);
    }
  for (int64_t c = 0; c < nc; ++c)
    if (line_of[c] < 0) {
      line_of[c] = int32_t(lines.size()), pos[c] = 0;
      lines.push_back({int32_t(c)});
    }
  const int64_t nl = int64_t(lines.size());
  // consecutive cells of a line must share an interior face
  auto coupled = [&](int32_t a, int32_t b) {
    for (int32_t e = H.cf_off[a]; e < H.cf_off[a + 1]; ++e) {
      const int64_t f = H.cf[e] >> 1;
      if (H.cr[f] < 0) continue;
      if (((H.cf[e] & 1) ? H.cl[f] : H.cr[f]) == b) return true;
    }
    return false;
  };
  for (const auto& L : lines)
    for (size_t p = 1; p < L.size(); ++p)
      if (!coupled(L[p - 1], L[p])) {
        set_error("lines: consecutive cells %d and %d share no face", L[p - 1], L[p]);
        return FPSI_E_INVALID;
      }
  // greedy colouring of the line graph in line order
  std::vector<int32_t> lcol(nl, -1);
  std::vector<int64_t> mark;
  int ncol = 0;
  for (int64_t l = 0; l < nl; ++l) {
    for (int32_t c : lines[l])
      for (int32_t e = H.cf_off[c]; e < H.cf_off[c + 1]; ++e) {
        const int64_t f = H.cf[e] >> 1;
        if (H.cr[f] < 0) continue;
        const int32_t o = (H.cf[e] & 1) ? H.cl[f] : H.cr[f];
        const int32_t ol = line_of[o];
        if (ol == l || lcol[ol] < 0) continue;
        if (lcol[ol] >= int32_t(mark.size())) mark.resize(lcol[ol] + 1, -1);
        mark[lcol[ol]] = l;
      }
    int k = 0;
    while (k < int(mark.size()) && mark[k] == l) ++k;
    lcol[l] = k;
    ncol = std::max(ncol, k + 1);
  }
  // groups of 32 lines per colour, lines ordered by their first cell
  Y = LineLayout();
  Y.nlines = nl;
  Y.ncolours = ncol;
  Y.col_goff.assign(ncol + 1, 0);
  Y.t_of.assign(nc, -1);
  Y.line_of = line_of;
  Y.line_colour = lcol;
  int64_t row = 0;
  for (int k = 0; k < ncol; ++k) {
    std::vector<int32_t> ls;
    for (int64_t l = 0; l < nl; ++l)
      if (lcol[l] == k) ls.push_back(int32_t(l));
    std::sort(ls.begin(), ls.end(), [&](int32_t a, int32_t b) { return lines[a][0] < lines[b][0]; });
    Y.col_goff[k] = Y.ngroups;
    for (size_t g0 = 0; g0 < ls.size(); g0 += 32) {
      int32_t glen = 0;
      for (size_t j = g0; j < std::min(ls.size(), g0 + 32); ++j)
        glen = std::max<int32_t>(glen, int32_t(lines[ls[j]].size()));
      Y.grp_row0.push_back(row);
      Y.grp_len.push_back(glen);
      for (int lane = 0; lane < 32; ++lane) {
        const size_t j = g0 + lane;
        if (j >= ls.size()) {
          Y.lane_len.push_back(0);
          continue;
        }
        const auto& L = lines[ls[j]];
        Y.lane_len.push_back(int32_t(L.size()));
        for (size_t p = 0; p < L.size(); ++p) Y.t_of[L[p]] = int32_t((row + p) * 32 + lane);
      }
      row += glen;
      Y.ngroups++;
    }
  }
  Y.col_goff[ncol] = Y.ngroups;
  Y.nrows = row;
  if (row * 32 >= (int64_t(1) << 31)) {
    set_error("lines: padded size too large");
    return FPSI_E_INVALID;
  }
  Y.c_of_t.assign(size_t(row * 32), -1);
  for (int64_t c = 0; c < nc; ++c) Y.c_of_t[Y.t_of[c]] = int32_t(c);
  // roles of the cell's faces and outer slots
  Y.role.assign(H.cf.size(), 0);
  int mout = 0;
  std::vector<int32_t> nout(nc, 0);
  for (int64_t c = 0; c < nc; ++c) {
    const auto& L = lines[line_of[c]];
    const int32_t p = pos[c];
    const int32_t prv = p > 0 ? L[p - 1] : -1;
    const int32_t nxt = p + 1 < int32_t(L.size()) ? L[p + 1] : -1;
    bool hp = false, hn = false;
    for (int32_t e = H.cf_off[c]; e < H.cf_off[c + 1]; ++e) {
      const int64_t f = H.cf[e] >> 1;
      if (H.cr[f] < 0) continue;
      const int32_t o = (H.cf[e] & 1) ? H.cl[f] : H.cr[f];
      if (o == prv && !hp) {
        Y.role[e] = 1, hp = true;
      } else if (o == nxt && !hn) {
        Y.role[e] = 2, hn = true;
      } else {
        if (nout[c] > 120) {
          set_error("lines: cell %lld has too many outer couplings", (long long)c);
          return FPSI_E_INVALID;
        }
        Y.role[e] = int8_t(3 + nout[c]++);
      }
    }
    mout = std::max(mout, nout[c]);
  }
  Y.mout = std::max(mout, 1);
  Y.onbr.assign(size_t(row) * Y.mout * 32, -1);
  for (int64_t c = 0; c < nc; ++c) {
    const int64_t t = Y.t_of[c], r = t / 32, lane = t % 32;
    for (int32_t e = H.cf_off[c]; e < H.cf_off[c + 1]; ++e) {
      if (Y.role[e] < 3) continue;
      const int64_t f = H.cf[e] >> 1;
      const int32_t o = (H.cf[e] & 1) ? H.cl[f] : H.cr[f];
      Y.onbr[(r * Y.mout + (Y.role[e] - 3)) * 32 + lane] = Y.t_of[o];
    }
  }
  Y.built = true;
  return FPSI_OK;
}

// ---------------------------------------------------------------------------
// device
// ---------------------------------------------------------------------------
namespace dev {

struct LineView {
  const int32_t* t_of;       // RCM cell -> t
  const int8_t* role;        // per cf entry
  const int32_t* onbr;       // [(row*mout+s)*32+lane]
  const int32_t* lane_len;   // [g*32+lane]
  const int64_t* grp_row0;
  int mout;
};

struct LsgsCtl {
  double w, zero, resid;
  int32_t iter, done;
};

// Gather the line-ordered system: raw diagonal block, in-line couplings
// (row p to p-1 in L, to p+1 in U), outer couplings and B.  The coupling of
// row c to neighbour n through face f is fjm_f when c = cl(f), -fjp_f when
// c = cr(f) (solverLinearSystem.loci:57-77).  One thread per line slot t,
// so that the 32 lanes of a row store 32 consecutive words of every stream;
// padding slots are left as they are (never read as data).
template <class TB, class TD>
__global__ void k_lsgs_scatter(int64_t nt, const int32_t* __restrict__ c_of_t,
                               const int32_t* __restrict__ cf_off, const int32_t* __restrict__ cf,
                               LineView V, const TB* __restrict__ D, const TB* __restrict__ fjp,
                               const TB* __restrict__ fjm, const double* __restrict__ src,
                               TD* __restrict__ lD, TB* __restrict__ lL, TB* __restrict__ lU,
                               TB* __restrict__ lF, TB* __restrict__ lB) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const int64_t c = c_of_t[t];
  if (c < 0) return;
  const int64_t r = t >> 5, lane = t & 31;
#pragma unroll
  for (int e = 0; e < 25; ++e) lD[(r * 25 + e) * 32 + lane] = TD(__ldg(D + 25 * c + e));
#pragma unroll
  for (int k = 0; k < 5; ++k) lB[(r * 5 + k) * 32 + lane] = TB(__ldg(src + 5 * c + k));
  for (int32_t e = cf_off[c]; e < cf_off[c + 1]; ++e) {
    const int ro = V.role[e];
    if (ro == 0) continue;
    const int32_t ent = cf[e];
    const int64_t f = ent >> 1;
    const bool neg = ent & 1;
    const TB* A = neg ? fjp + 25 * f : fjm + 25 * f;
    TB* o;
    if (ro == 1)
      o = lL + r * 25 * 32 + lane;
    else if (ro == 2)
      o = lU + r * 25 * 32 + lane;
    else
      o = lF + (r * V.mout + (ro - 3)) * 25 * 32 + lane;
#pragma unroll
    for (int k = 0; k < 25; ++k) o[k * 32] = neg ? TB(-__ldg(A + k)) : __ldg(A + k);
  }
}

// 5x5 LU without pivoting (decompose_lu of linearSolverLSGS.loci:1474) and
// its solve, on a block held in registers
template <class T>
__device__ __forceinline__ bool lu5_nopiv(T* A) {
  bool ok = true;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const T d = A[5 * k + k];
    if (d == T(0)) ok = false;
#pragma unroll
    for (int i = k + 1; i < 5; ++i) {
      A[5 * i + k] /= d;
#pragma unroll
      for (int j = k + 1; j < 5; ++j) A[5 * i + j] -= A[5 * i + k] * A[5 * k + j];
    }
  }
  return ok;
}
template <class T, class TV>
__device__ __forceinline__ void lu5_nopiv_solve(const T* A, TV* y) {
#pragma unroll
  for (int i = 1; i < 5; ++i)
#pragma unroll
    for (int j = 0; j < i; ++j) y[i] -= TV(A[5 * i + j]) * y[j];
#pragma unroll
  for (int i = 4; i >= 0; --i) {
#pragma unroll
    for (int j = i + 1; j < 5; ++j) y[i] -= TV(A[5 * i + j]) * y[j];
    y[i] /= TV(A[5 * i + i]);
  }
}

// block Thomas preprocessing (preprocessLine, linearSolverLSGS.loci:1465-1495):
// D'_0 = D_0, D'_p = D_p - L_p D'_{p-1}^{-1} U_{p-1}; each D' factored in
// place.  As in the reference the Schur product is formed with real_fj
// (TB) intermediates.
template <class TB, class TD>
__global__ void k_lsgs_prep(int64_t ngroups, LineView V, TD* __restrict__ lD,
                            const TB* __restrict__ lL, const TB* __restrict__ lU,
                            int32_t* __restrict__ err) {
  const int64_t gl = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (gl >= ngroups * 32) return;
  const int64_t g = gl >> 5, lane = gl & 31;
  const int len = V.lane_len[gl];
  const int64_t r0 = V.grp_row0[g];
  TD prev[25];
  for (int p = 0; p < len; ++p) {
    const int64_t r = r0 + p;
    TD Dp[25];
#pragma unroll
    for (int e = 0; e < 25; ++e) Dp[e] = lD[(r * 25 + e) * 32 + lane];
    if (p > 0) {
      TB Lm[25], Um[25];
#pragma unroll
      for (int e = 0; e < 25; ++e) {
        Lm[e] = lL[(r * 25 + e) * 32 + lane];
        Um[e] = lU[((r - 1) * 25 + e) * 32 + lane];
      }
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        TD v[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) v[k] = TD(Um[5 * k + j]);
        lu5_nopiv_solve<TD, TD>(prev, v);
        TB tt[5], w[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) tt[k] = TB(v[k]), w[k] = TB(0);
#pragma unroll
        for (int k = 0; k < 5; ++k)
#pragma unroll
          for (int m = 0; m < 5; ++m) w[k] += Lm[5 * k + m] * tt[m];
#pragma unroll
        for (int k = 0; k < 5; ++k) Dp[5 * k + j] -= TD(w[k]);
      }
    }
    if (!lu5_nopiv<TD>(Dp)) atomicOr(err, 2);
#pragma unroll
    for (int e = 0; e < 25; ++e) {
      lD[(r * 25 + e) * 32 + lane] = Dp[e];
      prev[e] = Dp[e];
    }
  }
}

// right-hand side of the rows of one colour: B - sum_outer F x_outer
template <class TB, class TX>
__global__ void k_lsgs_rhs(int64_t row_begin, int64_t nrows, LineView V,
                           const TB* __restrict__ lF, const TB* __restrict__ lB,
                           const TX* __restrict__ x, TX* __restrict__ rhs,
                           const LsgsCtl* __restrict__ ctl) {
  if (ctl->done) return;
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= nrows * 32) return;
  const int64_t r = row_begin + (i >> 5), lane = i & 31;
  TX b[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) b[k] = TX(__ldcs(lB + (r * 5 + k) * 32 + lane));
  for (int s = 0; s < V.mout; ++s) {
    const int32_t o = V.onbr[(r * V.mout + s) * 32 + lane];
    if (o < 0) break;
    TX xo[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) xo[k] = x[5 * int64_t(o) + k];
    const TB* F = lF + (r * V.mout + s) * 25 * 32 + lane;
#pragma unroll
    for (int k = 0; k < 5; ++k)
#pragma unroll
      for (int j = 0; j < 5; ++j) b[k] -= TX(__ldcs(F + (5 * k + j) * 32)) * xo[j];
  }
#pragma unroll
  for (int k = 0; k < 5; ++k) rhs[(r * 5 + k) * 32 + lane] = b[k];
}

// ---- bulk-copy pipeline (TMA engine, no multicast) -------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait: false after ~2^24 polls (each poll may suspend the warp)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (uint32_t it = 0; it < (1u << 24); ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

constexpr int LSGS_NST = 4;  // pipeline depth (rows in flight per group)

template <class TB, class TD, class TX>
struct ThomasStage {
  static constexpr uint32_t d_bytes = 25 * 32 * sizeof(TD);
  static constexpr uint32_t m_bytes = 25 * 32 * sizeof(TB);  // L (forward) or U (backward)
  static constexpr uint32_t b_bytes = 5 * 32 * (sizeof(TX) > sizeof(TB) ? sizeof(TX) : sizeof(TB));
  static constexpr uint32_t x_bytes = 5 * 32 * sizeof(TX);  // one row of the iterate
  static constexpr uint32_t bytes = d_bytes + m_bytes + b_bytes + x_bytes;  // multiple of 16
};
template <class TB, class TD, class TX>
constexpr size_t thomas_smem_bytes() {
  return size_t(LSGS_NST) * ThomasStage<TB, TD, TX>::bytes + 16 * LSGS_NST;
}

// block Thomas solve of the lines of groups [g0, g0+ng) (lineSolve,
// linearSolverLSGS.loci:1523-1572), one warp per group of 32 lines, one
// line per lane.  use_B: right-hand side B (start); save_xt: keep the
// iterate before the solve for the relaxation.
//
// A group's rows are contiguous ([row][entry][32 lanes]), so each row's
// factored diagonal block, coupling block and right-hand side arrive as
// bulk copies into shared memory, LSGS_NST rows ahead of the recurrence.
// The iterate's row comes the same way: before the forward solve
// overwrites it (kept for the relaxation) and, in the back substitution,
// the forward result (written by this warp, then made visible to the copy
// engine by a proxy fence).  Lane 0 issues the copies; every wait is
// bounded and a wait that gives up sets bit 4 of err and ends the kernel
// once the copies in flight landed.
template <class TB, class TD, class TX>
__global__ void __launch_bounds__(32)
k_lsgs_thomas(int64_t g0, LineView V, const TD* __restrict__ lD, const TB* __restrict__ lL,
              const TB* __restrict__ lU, const TX* __restrict__ rhs, const TB* __restrict__ lB,
              int use_B, int save_xt, TX* __restrict__ x, TX* __restrict__ xt,
              const LsgsCtl* __restrict__ ctl, int32_t* __restrict__ err) {
  using S = ThomasStage<TB, TD, TX>;
  if (ctl && ctl->done) return;
  extern __shared__ __align__(128) unsigned char th_smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(th_smem + size_t(LSGS_NST) * S::bytes);
  auto stage = [&](int s) { return th_smem + size_t(s) * S::bytes; };
  const int lane = threadIdx.x;
  const int64_t g = g0 + blockIdx.x;
  const int len = V.lane_len[g * 32 + lane];
  const int glen = __reduce_max_sync(0xffffffffu, len);
  const int64_t r0 = V.grp_row0[g];
  if (lane == 0)
    for (int s = 0; s < LSGS_NST; ++s) mbar_init(bar + s);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  __syncwarp();
  uint32_t phase = 0;  // bit s: parity of the next completion of stage s
  int inflight = 0;    // bit s: stage s has copies outstanding
  bool ok = true;

  // forward stage for row p: D'_{p-1}, L_p (p > 0) and the right-hand side
  auto issue_fwd = [&](int p) {
    const int s = p % LSGS_NST;
    const int64_t r = r0 + p;
    unsigned char* st = stage(s);
    const uint32_t bb = 5 * 32 * uint32_t(use_B ? sizeof(TB) : sizeof(TX));
    mbar_expect_tx(bar + s, (p > 0 ? S::d_bytes + S::m_bytes : 0) + bb + (save_xt ? S::x_bytes : 0));
    if (save_xt) bulk_g2s(st + S::d_bytes + S::m_bytes + S::b_bytes, x + r * 32 * 5, S::x_bytes, bar + s);
    if (p > 0) {
      bulk_g2s(st, lD + (r - 1) * 25 * 32, S::d_bytes, bar + s);
      bulk_g2s(st + S::d_bytes, lL + r * 25 * 32, S::m_bytes, bar + s);
    }
    if (use_B)
      bulk_g2s(st + S::d_bytes + S::m_bytes, lB + r * 5 * 32, bb, bar + s);
    else
      bulk_g2s(st + S::d_bytes + S::m_bytes, rhs + r * 5 * 32, bb, bar + s);
  };
  // backward stage for row p: D'_p, U_p and the forward result y_p
  auto issue_bwd = [&](int p) {
    const int s = (glen - 1 - p) % LSGS_NST;
    const int64_t r = r0 + p;
    unsigned char* st = stage(s);
    mbar_expect_tx(bar + s, S::d_bytes + S::m_bytes + S::x_bytes);
    bulk_g2s(st, lD + r * 25 * 32, S::d_bytes, bar + s);
    bulk_g2s(st + S::d_bytes, lU + r * 25 * 32, S::m_bytes, bar + s);
    bulk_g2s(st + S::d_bytes + S::m_bytes + S::b_bytes, x + r * 32 * 5, S::x_bytes, bar + s);
  };
  auto wait_stage = [&](int s) {
    const bool got = mbar_wait(bar + s, (phase >> s) & 1u);
    if (got) {
      phase ^= 1u << s;
      inflight &= ~(1 << s);
    }
    return got;
  };

  // forward elimination: y_p = rhs_p - L_p D'_{p-1}^{-1} y_{p-1}
  for (int p = 0; p < min(glen, LSGS_NST); ++p) {
    if (lane == 0) issue_fwd(p);
    inflight |= 1 << (p % LSGS_NST);
  }
  TX y[5];
  for (int p = 0; p < glen && ok; ++p) {
    const int s = p % LSGS_NST;
    ok = __all_sync(0xffffffffu, wait_stage(s));
    if (!ok) break;
    const unsigned char* st = stage(s);
    const TD* sD = reinterpret_cast<const TD*>(st) + lane;
    const TB* sL = reinterpret_cast<const TB*>(st + S::d_bytes) + lane;
    const int64_t t = (r0 + p) * 32 + lane;
    TX yn[5];
    if (use_B) {
      const TB* sb = reinterpret_cast<const TB*>(st + S::d_bytes + S::m_bytes) + lane;
#pragma unroll
      for (int k = 0; k < 5; ++k) yn[k] = TX(sb[k * 32]);
    } else {
      const TX* sb = reinterpret_cast<const TX*>(st + S::d_bytes + S::m_bytes) + lane;
#pragma unroll
      for (int k = 0; k < 5; ++k) yn[k] = sb[k * 32];
    }
    if (p > 0 && p < len) {
      TD Dm[25];
#pragma unroll
      for (int e = 0; e < 25; ++e) Dm[e] = sD[e * 32];
      lu5_nopiv_solve<TD, TX>(Dm, y);
#pragma unroll
      for (int k = 0; k < 5; ++k)
#pragma unroll
        for (int j = 0; j < 5; ++j) yn[k] -= TX(sL[(5 * k + j) * 32]) * y[j];
    }
    TX xo[5];
    if (save_xt) {
      const TX* sx = reinterpret_cast<const TX*>(st + S::d_bytes + S::m_bytes + S::b_bytes) + 5 * lane;
#pragma unroll
      for (int k = 0; k < 5; ++k) xo[k] = sx[k];
    }
    __syncwarp();
    if (lane == 0 && p + LSGS_NST < glen) issue_fwd(p + LSGS_NST);
    if (p + LSGS_NST < glen) inflight |= 1 << s;
    if (p < len) {
      if (save_xt) {
#pragma unroll
        for (int k = 0; k < 5; ++k) xt[5 * t + k] = xo[k];
      }
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        y[k] = yn[k];
        x[5 * t + k] = yn[k];
      }
    }
  }
  // back substitution: x_p = D'_p^{-1} (y_p - U_p x_{p+1}); the forward
  // results are read back through the copy engine
  asm volatile("fence.proxy.async.global;" ::: "memory");
  __syncwarp();
  if (ok) {
    for (int q = 0; q < min(glen, LSGS_NST); ++q) {
      if (lane == 0) issue_bwd(glen - 1 - q);
      inflight |= 1 << (q % LSGS_NST);
    }
    TX xn[5];
    for (int q = 0; q < glen && ok; ++q) {
      const int p = glen - 1 - q;
      const int s = q % LSGS_NST;
      ok = __all_sync(0xffffffffu, wait_stage(s));
      if (!ok) break;
      const unsigned char* st = stage(s);
      const TD* sD = reinterpret_cast<const TD*>(st) + lane;
      const TB* sU = reinterpret_cast<const TB*>(st + S::d_bytes) + lane;
      const int64_t t = (r0 + p) * 32 + lane;
      TX v[5];
      TD Dp[25];
      if (p < len) {
        const TX* sx = reinterpret_cast<const TX*>(st + S::d_bytes + S::m_bytes + S::b_bytes) + 5 * lane;
#pragma unroll
        for (int k = 0; k < 5; ++k) v[k] = sx[k];
        if (p < len - 1) {
#pragma unroll
          for (int k = 0; k < 5; ++k)
#pragma unroll
            for (int j = 0; j < 5; ++j) v[k] -= TX(sU[(5 * k + j) * 32]) * xn[j];
        }
#pragma unroll
        for (int e = 0; e < 25; ++e) Dp[e] = sD[e * 32];
      }
      __syncwarp();
      if (lane == 0 && q + LSGS_NST < glen) issue_bwd(p - LSGS_NST);
      if (q + LSGS_NST < glen) inflight |= 1 << s;
      if (p < len) {
        lu5_nopiv_solve<TD, TX>(Dp, v);
#pragma unroll
        for (int k = 0; k < 5; ++k) {
          x[5 * t + k] = v[k];
          xn[k] = v[k];
        }
      }
    }
  }
  if (!ok) {
    if (lane == 0) atomicOr(err, 4);
    // let the copies in flight land before the block's shared memory goes
    for (int s = 0; s < LSGS_NST; ++s)
      if (inflight & (1 << s)) mbar_wait(bar + s, (phase >> s) & 1u);
  }
}

constexpr int RELAX_THREADS = 256;

// X = w X + (1-w) X_t and the block partial of ||X - X_t||^2 (:1868-1874)
template <class TX>
__global__ void __launch_bounds__(RELAX_THREADS)
k_lsgs_relax(int64_t nt, TX* __restrict__ x, const TX* __restrict__ xt,
             const LsgsCtl* __restrict__ ctl, double* __restrict__ part) {
  if (ctl->done) return;
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const double w = ctl->w;
  double s = 0;
  if (t < nt) {
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      const TX xo = xt[5 * t + k];
      const TX xv = TX(w * double(x[5 * t + k]) + (1.0 - w) * double(xo));
      x[5 * t + k] = xv;
      const double d = double(xv) - double(xo);
      s += d * d;
    }
  }
  __shared__ double sh[RELAX_THREADS];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int st = RELAX_THREADS / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// residual, adaptive relaxation and stopping test (:1923-1947)
__global__ void k_lsgs_control(const double* __restrict__ part, int nblk, double abs_tol,
                               double rel_tol, LsgsCtl* __restrict__ ctl) {
  if (ctl->done) return;
  __shared__ double sh[RELAX_THREADS];
  double s = 0;
  for (int i = threadIdx.x; i < nblk; i += RELAX_THREADS) s += part[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int st = RELAX_THREADS / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double resid = sqrt(sh[0]);
    if (ctl->iter == 0) ctl->zero = fmax(resid, 1e-16);
    const double rel = resid / ctl->zero;
    if (rel > 1.0) ctl->w *= 1.0 / rel;
    ctl->resid = resid;
    ctl->iter += 1;
    if (resid < abs_tol || rel < rel_tol) ctl->done = 1;
  }
}

__global__ void k_lsgs_init(LsgsCtl* ctl, double w) {
  ctl->w = w;
  ctl->zero = 1.0;
  ctl->resid = 0.0;
  ctl->iter = 0;
  ctl->done = 0;
}

}  // namespace dev

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
namespace {
inline unsigned nblocks(int64_t n, int t) { return unsigned((n + t - 1) / t); }

dev::LineView line_view(const fpsi_ctx* x) {
  dev::LineView V;
  V.t_of = x->d_lt;
  V.role = x->d_lrole;
  V.onbr = x->d_lonbr;
  V.lane_len = x->d_llen;
  V.grp_row0 = x->d_lrow0;
  V.mout = x->LY.mout;
  return V;
}
}  // namespace

template <class TB, class TD, class TX>
static int lsgs_assemble_t(fpsi_ctx* x) {
  const LineLayout& Y = x->LY;
  cudaStream_t s = x->stream;
  const dev::LineView V = line_view(x);
  prof_begin(x, "lsgs_scatter");
  dev::k_lsgs_scatter<TB, TD><<<nblocks(Y.nrows * 32, 128), 128, 0, s>>>(
      Y.nrows * 32, x->d_lct, x->d_cf_off, x->d_cf, V, (const TB*)x->d_D, (const TB*)x->d_fjp,
      (const TB*)x->d_fjm, x->d_src, (TD*)x->d_lD, (TB*)x->d_lL, (TB*)x->d_lU, (TB*)x->d_lF,
      (TB*)x->d_lB);
  prof_end(x);
  prof_begin(x, "lsgs_prep");
  dev::k_lsgs_prep<TB, TD><<<nblocks(Y.ngroups * 32, 64), 64, 0, s>>>(
      Y.ngroups, V, (TD*)x->d_lD, (const TB*)x->d_lL, (const TB*)x->d_lU, x->d_err);
  prof_end(x);
  FPSI_CUDA_TRY(cudaGetLastError());
  return FPSI_OK;
}

int lsgs_assemble(fpsi_ctx* x) {
  switch (x->P.precision) {
    case FPSI_PREC_FP64:
      return lsgs_assemble_t<double, double, double>(x);
    case FPSI_PREC_MIXED:
      return lsgs_assemble_t<float, float, float>(x);
    default:
      return lsgs_assemble_t<float, double, double>(x);
  }
}

template <class TB, class TD, class TX>
static int lsgs_solve_t(fpsi_ctx* x, bool jacobi_start) {
  const LineLayout& Y = x->LY;
  cudaStream_t s = x->stream;
  const dev::LineView V = line_view(x);
  dev::LsgsCtl* ctl = (dev::LsgsCtl*)x->d_lctl;
  const int64_t nt = Y.nrows * 32;
  TX* X = (TX*)x->d_lx;
  TX* XT = (TX*)x->d_lxt;
  dev::k_lsgs_init<<<1, 1, 0, s>>>(ctl, x->P.lsgs_relaxation);
  constexpr size_t th_smem = dev::thomas_smem_bytes<TB, TD, TX>();
  if (th_smem > 48 * 1024)
    FPSI_CUDA_TRY(cudaFuncSetAttribute(dev::k_lsgs_thomas<TB, TD, TX>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, int(th_smem)));
  if (jacobi_start) {
    prof_begin(x, "lsgs_thomas");
    dev::k_lsgs_thomas<TB, TD, TX><<<unsigned(Y.ngroups), 32, th_smem, s>>>(
        0, V, (const TD*)x->d_lD, (const TB*)x->d_lL, (const TB*)x->d_lU, nullptr,
        (const TB*)x->d_lB, 1, 0, X, XT, nullptr, x->d_err);
    prof_end(x);
  }
  const int K = Y.ncolours;
  const int nblk = int(nblocks(nt, dev::RELAX_THREADS));
  for (int it = 0; it < x->P.lsgs_max_iter; ++it) {
    for (int pass = 0; pass < 2; ++pass)
      for (int kk = 0; kk < K; ++kk) {
        const int k = pass == 0 ? kk : K - 1 - kk;
        const int64_t g0 = Y.col_goff[k], ng = Y.col_goff[k + 1] - g0;
        if (ng == 0) continue;
        const int64_t rb = Y.grp_row0[g0];
        const int64_t re = Y.grp_row0[g0 + ng - 1] + Y.grp_len[g0 + ng - 1];
        prof_begin(x, "lsgs_rhs");
        dev::k_lsgs_rhs<TB, TX><<<nblocks((re - rb) * 32, 128), 128, 0, s>>>(
            rb, re - rb, V, (const TB*)x->d_lF, (const TB*)x->d_lB, X, (TX*)x->d_lrhs, ctl);
        prof_end(x);
        prof_begin(x, "lsgs_thomas");
        dev::k_lsgs_thomas<TB, TD, TX><<<unsigned(ng), 32, th_smem, s>>>(
            g0, V, (const TD*)x->d_lD, (const TB*)x->d_lL, (const TB*)x->d_lU,
            (const TX*)x->d_lrhs, (const TB*)x->d_lB, 0, pass == 1 ? 1 : 0, X, XT, ctl, x->d_err);
        prof_end(x);
      }
    prof_begin(x, "lsgs_relax");
    dev::k_lsgs_relax<TX><<<nblk, dev::RELAX_THREADS, 0, s>>>(nt, X, XT, ctl, x->d_lpart);
    dev::k_lsgs_control<<<1, dev::RELAX_THREADS, 0, s>>>(x->d_lpart, nblk, x->P.lsgs_abs_tol,
                                                         x->P.lsgs_rel_tol, ctl);
    prof_end(x);
  }
  FPSI_CUDA_TRY(cudaGetLastError());
  return FPSI_OK;
}

int lsgs_solve(fpsi_ctx* x, bool jacobi_start) {
  switch (x->P.precision) {
    case FPSI_PREC_FP64:
      return lsgs_solve_t<double, double, double>(x, jacobi_start);
    case FPSI_PREC_MIXED:
      return lsgs_solve_t<float, float, float>(x, jacobi_start);
    default:
      return lsgs_solve_t<float, double, double>(x, jacobi_start);
  }
}

}  // namespace fpsi
