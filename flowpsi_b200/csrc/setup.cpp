// setup.cpp -- host-side preparation of a mesh for the device path.
//
//  * geometry in FP64 (Loci FVM's area, facecenter, vol, cellcenter):
//    fan triangulation of each face about its node average; cell volume and
//    centroid from the pyramids on those triangles (divergence theorem);
//  * reverse Cuthill-McKee renumbering of the cells;
//  * faces sorted by (cl, cr) in the new numbering, interior faces first;
//  * cell -> face lists (upper, lower, boundary) and least-squares normal
//    matrices of the cell gradient;
//  * greedy distance-1 colouring of the cell graph for the multi-colour
//    Gauss-Seidel sweeps.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <numeric>

#include "fpsi_internal.h"

namespace fpsi {

namespace {
thread_local char g_err[512] = "";
}

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}
const char* last_error() { return g_err; }

namespace {

struct P3 {
  double v[3];
};
inline P3 p3(const double* a) { return P3{{a[0], a[1], a[2]}}; }

// Cuthill-McKee from a pseudo-peripheral start in every connected component,
// neighbours visited by increasing degree; reversed at the end.
std::vector<int32_t> rcm_order(int64_t n, const std::vector<int64_t>& off,
                               const std::vector<int32_t>& adj) {
  std::vector<int32_t> order;
  order.reserve(size_t(n));
  std::vector<char> seen(size_t(n), 0);
  std::vector<int32_t> level(size_t(n), -1);
  auto deg = [&](int32_t c) { return int32_t(off[c + 1] - off[c]); };
  auto bfs_far = [&](int32_t s, std::vector<int32_t>& comp) {
    // returns a node of the last BFS level with minimum degree
    comp.clear();
    comp.push_back(s);
    level[s] = 0;
    size_t h = 0;
    while (h < comp.size()) {
      int32_t c = comp[h++];
      for (int64_t k = off[c]; k < off[c + 1]; ++k) {
        int32_t m = adj[k];
        if (level[m] < 0) {
          level[m] = level[c] + 1;
          comp.push_back(m);
        }
      }
    }
    int32_t last = level[comp.back()];
    int32_t best = comp.back();
    for (size_t i = comp.size(); i-- > 0;) {
      if (level[comp[i]] != last) break;
      if (deg(comp[i]) < deg(best)) best = comp[i];
    }
    for (int32_t c : comp) level[c] = -1;
    return std::make_pair(best, last);
  };
  std::vector<int32_t> comp, nb;
  for (int64_t s0 = 0; s0 < n; ++s0) {
    if (seen[s0]) continue;
    int32_t start = int32_t(s0);
    auto r = bfs_far(start, comp);
    for (int it = 0; it < 2; ++it) {
      auto r2 = bfs_far(r.first, comp);
      if (r2.second <= r.second && it > 0) break;
      start = r.first;
      r = r2;
    }
    size_t h = order.size();
    order.push_back(start);
    seen[start] = 1;
    while (h < order.size()) {
      int32_t c = order[h++];
      nb.clear();
      for (int64_t k = off[c]; k < off[c + 1]; ++k)
        if (!seen[adj[k]]) {
          seen[adj[k]] = 1;
          nb.push_back(adj[k]);
        }
      std::stable_sort(nb.begin(), nb.end(),
                       [&](int32_t a, int32_t b) { return deg(a) < deg(b); });
      order.insert(order.end(), nb.begin(), nb.end());
    }
  }
  std::reverse(order.begin(), order.end());
  return order;
}

}  // namespace

int build_host_mesh(const fpsi_mesh* m, HostMesh& h) {
  const int64_t nc = m->ncells, nf = m->nfaces;
  if (nc <= 0 || nf <= 0 || !m->xyz || !m->face_off || !m->face_nodes || !m->cl || !m->cr) {
    set_error("mesh: empty or missing arrays");
    return FPSI_E_INVALID;
  }
  if (nc >= (int64_t(1) << 31) || 2 * nf >= (int64_t(1) << 30)) {
    set_error("mesh: too large for 32-bit indices");
    return FPSI_E_INVALID;
  }
  for (int64_t f = 0; f < nf; ++f) {
    int32_t a = m->cl[f], b = m->cr[f];
    if (a < 0 || a >= nc || b >= nc || (b < 0 && -b - 1 >= m->nbc) || a == b) {
      set_error("mesh: face %lld has invalid cl/cr (%d, %d)", (long long)f, a, b);
      return FPSI_E_INVALID;
    }
    int64_t k = m->face_off[f + 1] - m->face_off[f];
    if (k < 3) {
      set_error("mesh: face %lld has %lld nodes", (long long)f, (long long)k);
      return FPSI_E_INVALID;
    }
  }
  h.nc = nc;
  h.nf = nf;
  // ---- geometry in caller order ----
  std::vector<double> A(nf * 3), fc(nf * 3), ar(nf);
  for (int64_t f = 0; f < nf; ++f) {
    const int64_t b = m->face_off[f], e = m->face_off[f + 1];
    const int k = int(e - b);
    double xa[3] = {0, 0, 0};
    for (int64_t i = b; i < e; ++i)
      for (int d = 0; d < 3; ++d) xa[d] += m->xyz[3 * int64_t(m->face_nodes[i]) + d];
    for (int d = 0; d < 3; ++d) xa[d] /= k;
    double Av[3] = {0, 0, 0}, C[3] = {0, 0, 0}, W = 0;
    for (int i = 0; i < k; ++i) {
      const double* p0 = m->xyz + 3 * int64_t(m->face_nodes[b + i]);
      const double* p1 = m->xyz + 3 * int64_t(m->face_nodes[b + (i + 1) % k]);
      double u[3], v[3];
      for (int d = 0; d < 3; ++d) u[d] = p0[d] - xa[d], v[d] = p1[d] - xa[d];
      double t[3] = {0.5 * (u[1] * v[2] - u[2] * v[1]), 0.5 * (u[2] * v[0] - u[0] * v[2]),
                     0.5 * (u[0] * v[1] - u[1] * v[0])};
      double w = std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
      for (int d = 0; d < 3; ++d) {
        Av[d] += t[d];
        C[d] += (w / 3.0) * (xa[d] + p0[d] + p1[d]);
      }
      W += w;
    }
    double s = std::sqrt(Av[0] * Av[0] + Av[1] * Av[1] + Av[2] * Av[2]);
    if (!(s > 0)) {
      set_error("mesh: face %lld has zero area", (long long)f);
      return FPSI_E_INVALID;
    }
    ar[f] = s;
    for (int d = 0; d < 3; ++d) {
      A[3 * f + d] = Av[d];
      fc[3 * f + d] = C[d] / W;
    }
  }
  auto shift = [&](int64_t f, int d) { return m->pshift ? m->pshift[3 * f + d] : 0.0; };
  std::vector<double> xr(nc * 3, 0.0), vol(nc, 0.0), cc(nc * 3, 0.0);
  std::vector<int32_t> nfc(nc, 0);
  for (int64_t f = 0; f < nf; ++f) {
    int32_t a = m->cl[f], b = m->cr[f];
    for (int d = 0; d < 3; ++d) xr[3 * a + d] += fc[3 * f + d];
    nfc[a]++;
    if (b >= 0) {
      for (int d = 0; d < 3; ++d) xr[3 * b + d] += fc[3 * f + d] - shift(f, d);
      nfc[b]++;
    }
  }
  for (int64_t c = 0; c < nc; ++c)
    for (int d = 0; d < 3; ++d) xr[3 * c + d] /= nfc[c];
  for (int64_t f = 0; f < nf; ++f) {
    const int64_t b = m->face_off[f], e = m->face_off[f + 1];
    const int k = int(e - b);
    double xa[3] = {0, 0, 0};
    for (int64_t i = b; i < e; ++i)
      for (int d = 0; d < 3; ++d) xa[d] += m->xyz[3 * int64_t(m->face_nodes[i]) + d];
    for (int d = 0; d < 3; ++d) xa[d] /= k;
    for (int side = 0; side < 2; ++side) {
      int32_t c = side ? m->cr[f] : m->cl[f];
      if (c < 0) continue;
      double sg = side ? -1.0 : 1.0;
      double sh[3] = {side ? shift(f, 0) : 0, side ? shift(f, 1) : 0, side ? shift(f, 2) : 0};
      const double* x0 = &xr[3 * c];
      for (int i = 0; i < k; ++i) {
        const double* q0 = m->xyz + 3 * int64_t(m->face_nodes[b + i]);
        const double* q1 = m->xyz + 3 * int64_t(m->face_nodes[b + (i + 1) % k]);
        double pa[3], p0[3], p1[3];
        for (int d = 0; d < 3; ++d) {
          pa[d] = xa[d] - sh[d] - x0[d];
          p0[d] = q0[d] - sh[d] - x0[d];
          p1[d] = q1[d] - sh[d] - x0[d];
        }
        double cr3[3] = {p0[1] * p1[2] - p0[2] * p1[1], p0[2] * p1[0] - p0[0] * p1[2],
                         p0[0] * p1[1] - p0[1] * p1[0]};
        double v = sg * (pa[0] * cr3[0] + pa[1] * cr3[1] + pa[2] * cr3[2]) / 6.0;
        vol[c] += v;
        for (int d = 0; d < 3; ++d)
          cc[3 * c + d] += v * 0.25 * (4 * x0[d] + pa[d] + p0[d] + p1[d]);
      }
    }
  }
  for (int64_t c = 0; c < nc; ++c) {
    if (!(vol[c] > 0)) {
      set_error("mesh: cell %lld has non-positive volume %g", (long long)c, vol[c]);
      return FPSI_E_INVALID;
    }
    for (int d = 0; d < 3; ++d) cc[3 * c + d] /= vol[c];
  }
  h.an_caller = A;
  h.area_caller = ar;
  h.fc_caller = fc;

  // ---- RCM ----
  std::vector<int64_t> aoff(nc + 1, 0);
  for (int64_t f = 0; f < nf; ++f)
    if (m->cr[f] >= 0) {
      aoff[m->cl[f] + 1]++;
      aoff[m->cr[f] + 1]++;
    }
  for (int64_t c = 0; c < nc; ++c) aoff[c + 1] += aoff[c];
  std::vector<int32_t> adj(aoff[nc]);
  {
    std::vector<int64_t> pos(aoff.begin(), aoff.end() - 1);
    for (int64_t f = 0; f < nf; ++f)
      if (m->cr[f] >= 0) {
        adj[pos[m->cl[f]]++] = m->cr[f];
        adj[pos[m->cr[f]]++] = m->cl[f];
      }
  }
  h.perm = rcm_order(nc, aoff, adj);
  h.iperm.assign(nc, 0);
  for (int64_t i = 0; i < nc; ++i) h.iperm[h.perm[i]] = int32_t(i);

  // ---- faces: interior by (cl, cr) then boundary by (cl, bc) ----
  std::vector<int64_t> fo(nf);
  std::iota(fo.begin(), fo.end(), 0);
  auto key = [&](int64_t f) {
    int64_t a = h.iperm[m->cl[f]];
    int64_t b = m->cr[f] >= 0 ? int64_t(h.iperm[m->cr[f]]) : (int64_t(1) << 40) - m->cr[f];
    int64_t bnd = m->cr[f] < 0 ? 1 : 0;
    return std::make_tuple(bnd, a, b, f);
  };
  std::sort(fo.begin(), fo.end(), [&](int64_t x, int64_t y) { return key(x) < key(y); });
  h.fperm = fo;
  h.cl.resize(nf);
  h.cr.resize(nf);
  h.n.resize(nf * 3);
  h.area.resize(nf);
  h.rL.assign(nf * 3, 0.0);
  h.rR.assign(nf * 3, 0.0);
  h.nfi = 0;
  for (int64_t i = 0; i < nf; ++i) {
    int64_t f = fo[i];
    int32_t a = m->cl[f], b = m->cr[f];
    h.cl[i] = h.iperm[a];
    h.cr[i] = b >= 0 ? h.iperm[b] : b;
    if (b >= 0) h.nfi++;
    h.area[i] = ar[f];
    for (int d = 0; d < 3; ++d) {
      h.n[3 * i + d] = A[3 * f + d] / ar[f];
      h.rL[3 * i + d] = fc[3 * f + d] - cc[3 * a + d];
      if (b >= 0) h.rR[3 * i + d] = fc[3 * f + d] - (cc[3 * b + d] + shift(f, d));
    }
  }
  h.nbf = nf - h.nfi;
  h.vol.resize(nc);
  h.cc.resize(nc * 3);
  h.vol_tot = 0;
  for (int64_t i = 0; i < nc; ++i) {
    int32_t c = h.perm[i];
    h.vol[i] = vol[c];
    for (int d = 0; d < 3; ++d) h.cc[3 * i + d] = cc[3 * c + d];
  }
  for (int64_t c = 0; c < nc; ++c) h.vol_tot += vol[c];

  // ---- cell -> faces (upper, lower, boundary; each in face order) ----
  std::vector<int32_t> nu(nc, 0), nl(nc, 0), nb(nc, 0);
  for (int64_t f = 0; f < nf; ++f) {
    if (h.cr[f] >= 0) {
      nu[h.cl[f]]++;
      nl[h.cr[f]]++;
    } else {
      nb[h.cl[f]]++;
    }
  }
  h.cf_off.assign(nc + 1, 0);
  for (int64_t c = 0; c < nc; ++c) h.cf_off[c + 1] = h.cf_off[c] + nu[c] + nl[c] + nb[c];
  h.cf.assign(h.cf_off[nc], 0);
  {
    std::vector<int32_t> pu(nc), pl(nc), pb(nc);
    for (int64_t c = 0; c < nc; ++c) {
      pu[c] = h.cf_off[c];
      pl[c] = h.cf_off[c] + nu[c];
      pb[c] = h.cf_off[c] + nu[c] + nl[c];
    }
    for (int64_t f = 0; f < nf; ++f) {
      int32_t e = int32_t(f) << 1;
      if (h.cr[f] >= 0) {
        h.cf[pu[h.cl[f]]++] = e;
        h.cf[pl[h.cr[f]]++] = e | 1;
      } else {
        h.cf[pb[h.cl[f]]++] = e;
      }
    }
  }
  // ---- the same lists entry-major ----
  h.ell_k = 0;
  for (int64_t c = 0; c < nc; ++c) h.ell_k = std::max(h.ell_k, h.cf_off[c + 1] - h.cf_off[c]);
  h.ecf.assign(size_t(h.ell_k) * nc, -1);
  h.enb.assign(size_t(h.ell_k) * nc, -1);
  for (int64_t c = 0; c < nc; ++c)
    for (int32_t e = h.cf_off[c]; e < h.cf_off[c + 1]; ++e) {
      const size_t at = size_t(e - h.cf_off[c]) * nc + c;
      const int64_t f = h.cf[e] >> 1;
      h.ecf[at] = h.cf[e];
      if (h.cr[f] >= 0) h.enb[at] = (h.cf[e] & 1) ? h.cl[f] : h.cr[f];
    }
  // ---- least-squares normal matrices (inverse, symmetric 6 entries) ----
  h.Minv.assign(nc * 6, 0.0);
  for (int64_t c = 0; c < nc; ++c) {
    double M[6] = {0, 0, 0, 0, 0, 0};
    for (int32_t k = h.cf_off[c]; k < h.cf_off[c + 1]; ++k) {
      int64_t f = h.cf[k] >> 1;
      int side = h.cf[k] & 1;
      double dv[3];
      for (int d = 0; d < 3; ++d) {
        if (h.cr[f] < 0)
          dv[d] = h.rL[3 * f + d];
        else
          dv[d] = side ? h.rR[3 * f + d] - h.rL[3 * f + d] : h.rL[3 * f + d] - h.rR[3 * f + d];
      }
      M[0] += dv[0] * dv[0], M[1] += dv[0] * dv[1], M[2] += dv[0] * dv[2];
      M[3] += dv[1] * dv[1], M[4] += dv[1] * dv[2], M[5] += dv[2] * dv[2];
    }
    double a = M[0], b = M[1], cq = M[2], d = M[3], e = M[4], ff = M[5];
    double A00 = d * ff - e * e, A01 = cq * e - b * ff, A02 = b * e - cq * d;
    double A11 = a * ff - cq * cq, A12 = b * cq - a * e, A22 = a * d - b * b;
    double det = a * A00 + b * A01 + cq * A02;
    if (!(std::fabs(det) > 0)) {
      set_error("mesh: singular least-squares matrix in cell %lld", (long long)c);
      return FPSI_E_INVALID;
    }
    double r = 1.0 / det;
    double* mi = &h.Minv[6 * c];
    mi[0] = A00 * r, mi[1] = A01 * r, mi[2] = A02 * r;
    mi[3] = A11 * r, mi[4] = A12 * r, mi[5] = A22 * r;
  }
  // ---- greedy colouring in the new order ----
  h.colour.assign(nc, -1);
  int ncol = 0;
  std::vector<int64_t> mark(64, -1);
  for (int64_t c = 0; c < nc; ++c) {
    for (int32_t k = h.cf_off[c]; k < h.cf_off[c + 1]; ++k) {
      int64_t f = h.cf[k] >> 1;
      if (h.cr[f] < 0) continue;
      int32_t o = (h.cf[k] & 1) ? h.cl[f] : h.cr[f];
      int32_t col = h.colour[o];
      if (col >= 0) {
        if (col >= (int)mark.size()) mark.resize(col + 1, -1);
        mark[col] = c;
      }
    }
    int col = 0;
    while (col < (int)mark.size() && mark[col] == c) ++col;
    h.colour[c] = col;
    ncol = std::max(ncol, col + 1);
  }
  h.ncolours = ncol;
  h.colour_off.assign(ncol + 1, 0);
  for (int64_t c = 0; c < nc; ++c) h.colour_off[h.colour[c] + 1]++;
  for (int k = 0; k < ncol; ++k) h.colour_off[k + 1] += h.colour_off[k];
  h.colour_cells.assign(nc, 0);
  {
    std::vector<int32_t> pos(h.colour_off.begin(), h.colour_off.end() - 1);
    for (int64_t c = 0; c < nc; ++c) h.colour_cells[pos[h.colour[c]]++] = int32_t(c);
  }
  // ---- colour-order slot structure for the sweeps ----
  h.ci_of.assign(nc, 0);
  for (int64_t j = 0; j < nc; ++j) h.ci_of[h.colour_cells[j]] = int32_t(j);
  h.col_n.assign(ncol, 0);
  h.col_cb.assign(ncol, 0);
  h.col_m.assign(ncol, 0);
  h.col_ld.assign(ncol, 0);
  h.col_cbp.assign(ncol, 0);
  h.col_ebp.assign(ncol, 0);
  auto ninterior = [&](int64_t c) {
    int32_t k = 0;
    for (int32_t e = h.cf_off[c]; e < h.cf_off[c + 1]; ++e)
      if (h.cr[h.cf[e] >> 1] >= 0) ++k;
    return k;
  };
  int64_t eb = 0, cbp = 0;
  for (int k = 0; k < ncol; ++k) {
    h.col_cb[k] = h.colour_off[k];
    h.col_n[k] = h.colour_off[k + 1] - h.colour_off[k];
    h.col_ld[k] = (h.col_n[k] + 31) / 32 * 32;
    int64_t m = 0;
    for (int32_t j = h.colour_off[k]; j < h.colour_off[k + 1]; ++j)
      m = std::max<int64_t>(m, ninterior(h.colour_cells[j]));
    h.col_m[k] = m;
    h.col_cbp[k] = cbp;
    h.col_ebp[k] = eb;
    cbp += h.col_ld[k];
    eb += m * h.col_ld[k];
  }
  h.ncp = cbp;
  h.nslots = eb;
  h.nbr.assign(size_t(eb), -1);
  for (int k = 0; k < ncol; ++k)
    for (int64_t i = 0; i < h.col_n[k]; ++i) {
      const int32_t c = h.colour_cells[h.col_cb[k] + i];
      int64_t s = 0;
      for (int32_t e = h.cf_off[c]; e < h.cf_off[c + 1]; ++e) {
        const int64_t f = h.cf[e] >> 1;
        if (h.cr[f] < 0) continue;
        const int32_t o = (h.cf[e] & 1) ? h.cl[f] : h.cr[f];
        h.nbr[h.col_ebp[k] + s * h.col_ld[k] + i] = h.ci_of[o];
        ++s;
      }
    }
  return FPSI_OK;
}


// ---------------------------------------------------------------------------
// distance to the nearest no-slip wall (find_mind, gridSetup.loci:418-640;
// dist_noslip, solverTurbulence.loci:133-137): the wall face is chosen by the
// distance between its edge-length weighted centre and the cell's area
// weighted face-centre average (ties: lowest face), the distance is
// |(x_f - x_c).n| with the finite-volume centres.  k-d tree over the wall
// faces.  Result in the context's (RCM) cell order; 1e30 without walls.
// ---------------------------------------------------------------------------
namespace {
struct WallTree {
  std::vector<double> p;     // 3 per wall face (search centres)
  std::vector<int64_t> id;   // caller face id
  std::vector<int32_t> ord;  // tree order: node k = ord[k]
  std::vector<int8_t> axis;  // per tree position
  void build(int64_t lo, int64_t hi) {
    if (hi - lo <= 0) return;
    double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
    for (int64_t k = lo; k < hi; ++k)
      for (int d = 0; d < 3; ++d) {
        mn[d] = std::min(mn[d], p[3 * ord[k] + d]);
        mx[d] = std::max(mx[d], p[3 * ord[k] + d]);
      }
    int ax = 0;
    for (int d = 1; d < 3; ++d)
      if (mx[d] - mn[d] > mx[ax] - mn[ax]) ax = d;
    const int64_t mid = lo + (hi - lo) / 2;
    std::nth_element(ord.begin() + lo, ord.begin() + mid, ord.begin() + hi, [&](int32_t a, int32_t b) {
      const double va = p[3 * a + ax], vb = p[3 * b + ax];
      return va < vb || (va == vb && id[a] < id[b]);
    });
    axis[mid] = int8_t(ax);
    build(lo, mid);
    build(mid + 1, hi);
  }
  void query(int64_t lo, int64_t hi, const double q[3], double& bd, int64_t& bid, int32_t& bk) const {
    if (hi - lo <= 0) return;
    const int64_t mid = lo + (hi - lo) / 2;
    const int32_t k = ord[mid];
    double d2 = 0;
    for (int d = 0; d < 3; ++d) {
      const double t = p[3 * k + d] - q[d];
      d2 += t * t;
    }
    if (d2 < bd || (d2 == bd && id[k] < bid)) bd = d2, bid = id[k], bk = k;
    const int ax = axis[mid];
    const double diff = q[ax] - p[3 * k + ax];
    const bool left_first = diff <= 0;
    if (left_first) {
      query(lo, mid, q, bd, bid, bk);
      if (diff * diff <= bd) query(mid + 1, hi, q, bd, bid, bk);
    } else {
      query(mid + 1, hi, q, bd, bid, bk);
      if (diff * diff <= bd) query(lo, mid, q, bd, bid, bk);
    }
  }
};
}  // namespace

void wall_distance(const fpsi_mesh* m, const HostMesh& H, std::vector<double>& out) {
  const int64_t nc = m->ncells, nf = m->nfaces;
  out.assign(nc, 1e30);
  std::vector<int64_t> walls;
  for (int64_t f = 0; f < nf; ++f)
    if (m->cr[f] < 0 && m->bcs[-m->cr[f] - 1].kind == FPSI_BC_VISCOUS_WALL) walls.push_back(f);
  if (walls.empty()) return;
  // search centres (caller numbering)
  std::vector<double> fce(nf * 3), fa(nf);
  for (int64_t f = 0; f < nf; ++f) {
    const int64_t a = m->face_off[f], b = m->face_off[f + 1];
    const int n = int(b - a);
    double ns[3] = {0, 0, 0}, ls = 0;
    for (int i = 0; i < n; ++i) {
      const double* p1 = m->xyz + 3 * int64_t(m->face_nodes[a + i]);
      const double* p2 = m->xyz + 3 * int64_t(m->face_nodes[a + (i + 1) % n]);
      const double len = std::sqrt((p1[0] - p2[0]) * (p1[0] - p2[0]) + (p1[1] - p2[1]) * (p1[1] - p2[1]) +
                                   (p1[2] - p2[2]) * (p1[2] - p2[2]));
      for (int d = 0; d < 3; ++d) ns[d] += len * (0.5 * (p1[d] + p2[d]));
      ls += len;
    }
    double c[3];
    for (int d = 0; d < 3; ++d) c[d] = (1.0 / ls) * ns[d];
    double sx = 0, sy = 0, sz = 0;
    for (int i = 0; i < n; ++i) {
      const double* p1 = m->xyz + 3 * int64_t(m->face_nodes[a + i]);
      const double* p2 = m->xyz + 3 * int64_t(m->face_nodes[a + (i + 1) % n]);
      const double u0 = p1[0] - c[0], u1 = p1[1] - c[1], u2 = p1[2] - c[2];
      const double v0 = p2[0] - c[0], v1 = p2[1] - c[1], v2 = p2[2] - c[2];
      sx += u1 * v2 - u2 * v1, sy += u2 * v0 - u0 * v2, sz += u0 * v1 - u1 * v0;
    }
    for (int d = 0; d < 3; ++d) fce[3 * f + d] = c[d];
    fa[f] = 0.5 * std::sqrt(sx * sx + sy * sy + sz * sz);
  }
  std::vector<double> csum(nc * 3, 0.0), asum(nc, 0.0);
  for (int64_t f = 0; f < nf; ++f)
    for (int side = 0; side < 2; ++side) {
      const int64_t c = side ? m->cr[f] : m->cl[f];
      if (c < 0) continue;
      for (int d = 0; d < 3; ++d) csum[3 * c + d] += fce[3 * f + d] * fa[f];
      asum[c] += fa[f];
    }
  WallTree T;
  const int64_t nw = int64_t(walls.size());
  T.p.resize(3 * nw);
  T.id.resize(nw);
  T.ord.resize(nw);
  T.axis.assign(nw, 0);
  for (int64_t k = 0; k < nw; ++k) {
    for (int d = 0; d < 3; ++d) T.p[3 * k + d] = fce[3 * walls[k] + d];
    T.id[k] = walls[k];
    T.ord[k] = int32_t(k);
  }
  T.build(0, nw);
  std::vector<double> cc_caller(nc * 3);
  for (int64_t i = 0; i < nc; ++i)
    for (int d = 0; d < 3; ++d) cc_caller[3 * H.perm[i] + d] = H.cc[3 * i + d];
  std::vector<double> dc(nc);
  for (int64_t c = 0; c < nc; ++c) {
    double q[3];
    for (int d = 0; d < 3; ++d) q[d] = (1.0 / asum[c]) * csum[3 * c + d];
    double bd = 1e300;
    int64_t bid = -1;
    int32_t bk = -1;
    T.query(0, nw, q, bd, bid, bk);
    const int64_t w = bid;
    double dot = 0;
    for (int d = 0; d < 3; ++d)
      dot += (H.fc_caller[3 * w + d] - cc_caller[3 * c + d]) * (H.an_caller[3 * w + d] / H.area_caller[w]);
    dc[c] = std::fabs(dot);
  }
  for (int64_t i = 0; i < nc; ++i) out[i] = dc[H.perm[i]];
}

}  // namespace fpsi
