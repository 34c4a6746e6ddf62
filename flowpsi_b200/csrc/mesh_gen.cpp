// mesh_gen.cpp -- synthetic grids for the benchmark configurations.
//
// kind 0: structured hex box (configs: 32^3 farfield cube, 256^3 shock cube)
// kind 1: hex box, each hex split into 6 Kuhn tetrahedra along its main
//         diagonal, nodes jittered; periodic (128^3 Taylor-Green case) or
//         bounded sides (the steady farfield tet case)
// kind 2: boundary-layer hex block with geometric wall-normal stretching
// kind 3: hex box (as kind 0, periodic sides allowed) with each hex split
//         into two triangular prisms across the diagonal v000-v110 of its
//         z-faces: 5 faces per cell, triangles and quads mixed
//
// Faces are produced directly from the structured topology (no hashing), with
// interior faces oriented cl < cr and node order giving a cl->cr normal.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <new>
#include <vector>

#include "fpsi_internal.h"

namespace {

struct OwnedMesh {
  fpsi_mesh m;
  std::vector<double> xyz, pshift;
  std::vector<int64_t> face_off;
  std::vector<int32_t> face_nodes, cl, cr;
  std::vector<fpsi_bc> bcs;
};

// SplitMix64: counter-based, identical on every host.
inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
inline double u01(uint64_t seed, uint64_t i) {
  return double(splitmix64(seed * 0x100000001B3ull + i) >> 11) * (1.0 / 9007199254740992.0);
}

void finish(OwnedMesh* o) {
  fpsi_mesh& m = o->m;
  m.nnodes = int64_t(o->xyz.size() / 3);
  m.ncells = 0;
  m.nfaces = int64_t(o->cl.size());
  m.xyz = o->xyz.data();
  m.face_off = o->face_off.data();
  m.face_nodes = o->face_nodes.data();
  m.cl = o->cl.data();
  m.cr = o->cr.data();
  m.pshift = o->pshift.empty() ? nullptr : o->pshift.data();
  m.nbc = int32_t(o->bcs.size());
  m.bcs = o->bcs.data();
}

// Hex box.  Node (i,j,k) = i + (nx+1)*(j + (ny+1)*k); cell (i,j,k) =
// i + nx*(j + ny*k).  Periodic directions reuse node index i mod n for the
// face of the last layer and record the translation in pshift.
// With `prism` each hex c becomes prisms 2c (P0: corners v000 v100 v110 and
// the three above) and 2c+1 (P1: v000 v110 v010 and above).  P0 owns the
// hex's x-max and y-min faces, P1 its x-min and y-max faces; z-faces split
// into two triangles (P0's and P1's), and the diagonal quad separates P0
// from P1 with its normal towards P1.
int gen_hex(const fpsi_mesh_spec* s, OwnedMesh* o, bool stretched, bool prism = false) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  if (nx < 2 || ny < 2 || nz < 2) return FPSI_E_INVALID;
  const bool per[3] = {s->bc_side[0] < 0, s->bc_side[2] < 0, s->bc_side[4] < 0};
  for (int d = 0; d < 3; ++d)
    if ((s->bc_side[2 * d] < 0) != (s->bc_side[2 * d + 1] < 0)) return FPSI_E_INVALID;
  const int64_t NX = nx + 1, NY = ny + 1, NZ = nz + 1;
  o->xyz.resize(size_t(NX * NY * NZ * 3));
  std::vector<double> yc(NY);
  if (stretched) {
    double y = 0;
    for (int j = 0; j < NY; ++j) {
      yc[j] = y;
      y += s->dy0 * std::pow(s->growth, j);
    }
  } else {
    for (int j = 0; j < NY; ++j) yc[j] = s->Ly * j / ny;
  }
  for (int64_t k = 0; k < NZ; ++k)
    for (int64_t j = 0; j < NY; ++j)
      for (int64_t i = 0; i < NX; ++i) {
        int64_t id = i + NX * (j + NY * k);
        o->xyz[3 * id] = s->Lx * i / nx;
        o->xyz[3 * id + 1] = yc[j];
        o->xyz[3 * id + 2] = s->Lz * k / nz;
      }
  auto node = [&](int64_t i, int64_t j, int64_t k) -> int32_t {
    return int32_t(i + NX * (j + NY * k));
  };
  auto cell = [&](int64_t i, int64_t j, int64_t k) -> int32_t {
    return int32_t(i + int64_t(nx) * (j + int64_t(ny) * k));
  };
  const int64_t nc = int64_t(nx) * ny * nz;
  o->face_off.push_back(0);
  bool anyper = per[0] || per[1] || per[2];
  auto add_poly = [&](std::initializer_list<int32_t> nodes, int32_t L, int32_t R, double sx,
                      double sy, double sz) {
    for (int32_t v : nodes) o->face_nodes.push_back(v);
    o->face_off.push_back(int64_t(o->face_nodes.size()));
    o->cl.push_back(L);
    o->cr.push_back(R);
    if (anyper) {
      o->pshift.push_back(sx);
      o->pshift.push_back(sy);
      o->pshift.push_back(sz);
    }
  };
  // where = 0 interior (+d node order), 1 emitted at p = 0 (reversed
  // order; R is the last layer's hex on a periodic seam, else a boundary
  // code), 2 the boundary at p = n_d
  int cur_d = 0, where = 0;
  auto add_face = [&](int32_t a, int32_t b, int32_t c, int32_t d, int32_t L, int32_t R,
                      double sx, double sy, double sz) {
    if (prism) {
      const bool rb = R < 0;  // boundary code
      auto P = [](int32_t h, int side) { return 2 * h + side; };
      if (cur_d == 2) {
        // triangles (a,b,c) and (a,c,d); in +z order the first is P0's
        const int sa = where == 1 ? 1 : 0, sb = 1 - sa;
        add_poly({a, b, c}, P(L, sa), rb ? R : P(R, sa), sx, sy, sz);
        add_poly({a, c, d}, P(L, sb), rb ? R : P(R, sb), sx, sy, sz);
      } else {
        // the face's side of the hex on each side: x-max and y-min in P0
        const int lo_side = cur_d == 0 ? 1 : 0;  // the hex's min-plane face
        const int hi_side = 1 - lo_side;         // the hex's max-plane face
        const int sl = where == 1 ? lo_side : hi_side;  // cl's face: min plane at p = 0
        const int sr = where == 1 ? hi_side : lo_side;
        add_poly({a, b, c, d}, P(L, sl), rb ? R : P(R, sr), sx, sy, sz);
      }
      return;
    }
    o->face_nodes.push_back(a);
    o->face_nodes.push_back(b);
    o->face_nodes.push_back(c);
    o->face_nodes.push_back(d);
    o->face_off.push_back(int64_t(o->face_nodes.size()));
    o->cl.push_back(L);
    o->cr.push_back(R);
    if (anyper) {
      o->pshift.push_back(sx);
      o->pshift.push_back(sy);
      o->pshift.push_back(sz);
    }
  };
  const double Ly = stretched ? yc[ny] : s->Ly;
  // Faces normal to direction d at plane index p.  The +d node cycle is
  // (t0,t1), (t0+1,t1), (t0+1,t1+1), (t0,t1+1) over the two transverse
  // directions in cyclic order.  A periodic seam is emitted once, at p = 0,
  // with cl = first layer, cr = last layer, nodes in cl's frame, normal -d
  // and pshift = -L_d * e_d (cr's image sits below the min plane).
  const int64_t Nn[3] = {nx, ny, nz};
  const double Ld[3] = {s->Lx, Ly, s->Lz};
  for (int d = 0; d < 3; ++d) {
    const int t0 = (d + 1) % 3, t1 = (d + 2) % 3;
    for (int64_t b = 0; b < Nn[t1]; ++b)
      for (int64_t a = 0; a < Nn[t0]; ++a)
        for (int64_t p = 0; p <= Nn[d]; ++p) {
          auto nid = [&](int64_t pp, int64_t aa, int64_t bb) {
            int64_t ijk[3];
            ijk[d] = pp, ijk[t0] = aa, ijk[t1] = bb;
            return node(ijk[0], ijk[1], ijk[2]);
          };
          auto cid = [&](int64_t pp) {
            int64_t ijk[3];
            ijk[d] = pp, ijk[t0] = a, ijk[t1] = b;
            return cell(ijk[0], ijk[1], ijk[2]);
          };
          int32_t n0 = nid(p, a, b), n1 = nid(p, a + 1, b), n2 = nid(p, a + 1, b + 1),
                  n3 = nid(p, a, b + 1);
          double sh[3] = {0, 0, 0};
          cur_d = d;
          where = (p > 0 && p < Nn[d]) ? 0 : (p == 0 ? 1 : 2);
          if (p > 0 && p < Nn[d]) {
            add_face(n0, n1, n2, n3, cid(p - 1), cid(p), 0, 0, 0);
          } else if (per[d]) {
            if (p == 0) {
              sh[d] = -Ld[d];
              add_face(n0, n3, n2, n1, cid(0), cid(Nn[d] - 1), sh[0], sh[1], sh[2]);
            }
          } else if (p == 0) {
            add_face(n0, n3, n2, n1, cid(0), -1 - s->bc_side[2 * d], 0, 0, 0);
          } else {
            add_face(n0, n1, n2, n3, cid(Nn[d] - 1), -1 - s->bc_side[2 * d + 1], 0, 0, 0);
          }
        }
  }
  if (prism) {
    // the diagonal quad of every hex, P0 -> P1
    for (int64_t k = 0; k < nz; ++k)
      for (int64_t j = 0; j < ny; ++j)
        for (int64_t i = 0; i < nx; ++i) {
          const int32_t c = cell(i, j, k);
          add_poly({node(i, j, k), node(i, j, k + 1), node(i + 1, j + 1, k + 1), node(i + 1, j + 1, k)},
                   2 * c, 2 * c + 1, 0, 0, 0);
        }
  }
  const int64_t ncells = prism ? 2 * nc : nc;
  o->m.ncells = ncells;
  o->bcs.assign(s->bcs, s->bcs + s->nbc);
  finish(o);
  o->m.ncells = ncells;
  return FPSI_OK;
}

// Kuhn split of each hex of a box into 6 tetrahedra.  For the permutation
// (a,b,c) of the axes, tet = {v0, v0+e_a, v0+e_a+e_b, v0+1}.  Face sharing
// is analytic:
//   opposite v7         <-> tet (c,a,b) of the hex at -e_c   (cube-face)
//   opposite v0         <-> tet (b,c,a) of the hex at +e_a   (cube-face)
//   opposite v0+e_a     <-> tet (b,a,c) of the same hex      (internal)
//   opposite v0+e_a+e_b <-> tet (a,c,b) of the same hex      (internal)
// The split conforms across opposite sides of the box, so every direction
// may be periodic (bc_side < 0: the neighbour hex wraps around) or bounded
// (a cube-face tet face on the side becomes a boundary face of that side's
// condition).  Node coordinates are jittered by U(-jitter,+jitter) of the
// spacing, except the normal component of nodes on a bounded side, so the
// sides stay plane.  A periodic direction has one node layer per hex layer
// (periodic images share their node and its jitter).
int gen_kuhn(const fpsi_mesh_spec* s, OwnedMesh* o) {
  const int64_t nx = s->nx, ny = s->ny, nz = s->nz;
  if (nx < 2 || ny < 2 || nz < 2) return FPSI_E_INVALID;
  bool per[3];
  for (int d = 0; d < 3; ++d) {
    per[d] = s->bc_side[2 * d] < 0;
    if ((s->bc_side[2 * d] < 0) != (s->bc_side[2 * d + 1] < 0)) return FPSI_E_INVALID;
  }
  const bool anyper = per[0] || per[1] || per[2];
  static const int PERM[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  auto perm_id = [&](int a, int b, int c) {
    for (int p = 0; p < 6; ++p)
      if (PERM[p][0] == a && PERM[p][1] == b && PERM[p][2] == c) return p;
    return -1;
  };
  const double h[3] = {s->Lx / nx, s->Ly / ny, s->Lz / nz};
  const double L[3] = {s->Lx, s->Ly, s->Lz};
  const int64_t N[3] = {nx, ny, nz};
  // node layers per direction: n (periodic) or n + 1 (bounded)
  const int64_t NN[3] = {per[0] ? nx : nx + 1, per[1] ? ny : ny + 1, per[2] ? nz : nz + 1};
  const int64_t nn = NN[0] * NN[1] * NN[2];
  o->xyz.resize(size_t(nn * 3));
  for (int64_t k = 0; k < NN[2]; ++k)
    for (int64_t j = 0; j < NN[1]; ++j)
      for (int64_t i = 0; i < NN[0]; ++i) {
        int64_t id = i + NN[0] * (j + NN[1] * k);
        int64_t ijk[3] = {i, j, k};
        for (int d = 0; d < 3; ++d) {
          const bool on_side = !per[d] && (ijk[d] == 0 || ijk[d] == N[d]);
          double jt = on_side ? 0.0
                              : s->jitter * h[d] * (2.0 * u01(s->seed, uint64_t(3 * id + d)) - 1.0);
          o->xyz[3 * id + d] = h[d] * ijk[d] + jt;
        }
      }
  auto nodeid = [&](int64_t i, int64_t j, int64_t k) {
    if (per[0]) i = (i + nx) % nx;
    if (per[1]) j = (j + ny) % ny;
    if (per[2]) k = (k + nz) % nz;
    return i + NN[0] * (j + NN[1] * k);
  };
  auto hexid = [&](int64_t i, int64_t j, int64_t k) {
    i = (i + nx) % nx, j = (j + ny) % ny, k = (k + nz) % nz;
    return i + nx * (j + ny * k);
  };
  const int64_t ncell = 6 * nx * ny * nz;
  o->face_off.push_back(0);
  for (int64_t k = 0; k < nz; ++k)
    for (int64_t j = 0; j < ny; ++j)
      for (int64_t i = 0; i < nx; ++i) {
        const int64_t hx = i + nx * (j + ny * k);
        const int64_t base[3] = {i, j, k};
        for (int p = 0; p < 6; ++p) {
          const int a = PERM[p][0], b = PERM[p][1], c = PERM[p][2];
          int off[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {1, 1, 1}};
          off[1][a] = 1;
          off[2][a] = 1;
          off[2][b] = 1;
          const int32_t me = int32_t(6 * hx + p);
          // the four faces: (opposite vertex, neighbour tet, shift of neighbour hex)
          for (int opp = 0; opp < 4; ++opp) {
            int np;
            int dshift[3] = {0, 0, 0};
            if (opp == 3) {
              dshift[c] = -1;
              np = perm_id(c, a, b);
            } else if (opp == 0) {
              dshift[a] = 1;
              np = perm_id(b, c, a);
            } else if (opp == 1) {
              np = perm_id(b, a, c);
            } else {
              np = perm_id(a, c, b);
            }
            // a neighbour hex across a bounded side: boundary face
            int32_t bcode = 0;
            for (int d = 0; d < 3; ++d) {
              const int64_t u = base[d] + dshift[d];
              if (!per[d] && u < 0) bcode = -1 - s->bc_side[2 * d];
              if (!per[d] && u >= N[d]) bcode = -1 - s->bc_side[2 * d + 1];
            }
            int32_t other = bcode;
            if (!bcode) {
              const int64_t nh = hexid(i + dshift[0], j + dshift[1], k + dshift[2]);
              other = int32_t(6 * nh + np);
              // emit each interior face once, from the smaller cell id (cl < cr)
              if (other < me) continue;
              if (other == me) return FPSI_E_INVALID;
            }
            // nodes of the face (the three vertices other than opp)
            int32_t ids[3];
            int q = 0;
            for (int v = 0; v < 4; ++v) {
              if (v == opp) continue;
              ids[q++] = int32_t(nodeid(base[0] + off[v][0], base[1] + off[v][1], base[2] + off[v][2]));
            }
            // orientation: normal must point away from the opposite vertex.
            // positions (unjittered is enough for the sign; jitter < h/2)
            double P[3][3], Vo[3];
            q = 0;
            for (int v = 0; v < 4; ++v) {
              double x[3] = {h[0] * (base[0] + off[v][0]), h[1] * (base[1] + off[v][1]),
                             h[2] * (base[2] + off[v][2])};
              if (v == opp) {
                for (int d = 0; d < 3; ++d) Vo[d] = x[d];
              } else {
                for (int d = 0; d < 3; ++d) P[q][d] = x[d];
                ++q;
              }
            }
            double e1[3], e2[3], nrm[3];
            for (int d = 0; d < 3; ++d) e1[d] = P[1][d] - P[0][d], e2[d] = P[2][d] - P[0][d];
            nrm[0] = e1[1] * e2[2] - e1[2] * e2[1];
            nrm[1] = e1[2] * e2[0] - e1[0] * e2[2];
            nrm[2] = e1[0] * e2[1] - e1[1] * e2[0];
            double sd = 0;
            for (int d = 0; d < 3; ++d) sd += nrm[d] * (P[0][d] - Vo[d]);
            if (sd < 0) std::swap(ids[1], ids[2]);
            o->cl.push_back(me);
            o->cr.push_back(other);
            // x_cr_image = x_cr + pshift: the wrap of the neighbour hex
            if (anyper)
              for (int d = 0; d < 3; ++d) {
                const int64_t u = base[d] + dshift[d];
                double s2 = 0;
                if (!bcode && u < 0) s2 = -L[d];
                if (!bcode && u >= N[d]) s2 = L[d];
                o->pshift.push_back(s2);
              }
            for (int v = 0; v < 3; ++v) o->face_nodes.push_back(ids[v]);
            o->face_off.push_back(int64_t(o->face_nodes.size()));
          }
        }
      }
  // Faces reference wrapped node ids; a face whose vertices straddle a
  // periodic seam is expressed in cl's frame through private node copies
  // (appended after the shared nodes).
  const int64_t nf = int64_t(o->cl.size());
  if (anyper)
    for (int64_t f = 0; f < nf; ++f) {
      const int64_t hx = o->cl[f] / 6;
      const int64_t bb[3] = {hx % nx, (hx / nx) % ny, hx / (nx * ny)};
      const int64_t b = o->face_off[f];
      for (int q = 0; q < 3; ++q) {
        const int64_t nd = o->face_nodes[b + q];
        const int64_t v[3] = {nd % NN[0], (nd / NN[0]) % NN[1], nd / (NN[0] * NN[1])};
        // the vertex belongs to hex base + {0,1}: unwrap relative to base
        double add[3] = {0, 0, 0};
        bool wrap = false;
        for (int d = 0; d < 3; ++d)
          if (per[d] && v[d] < bb[d]) {
            add[d] = L[d];
            wrap = true;
          }
        if (!wrap) continue;
        const int64_t newid = int64_t(o->xyz.size() / 3);
        for (int d = 0; d < 3; ++d) o->xyz.push_back(o->xyz[3 * nd + d] + add[d]);
        o->face_nodes[b + q] = int32_t(newid);
      }
    }
  o->bcs.assign(s->bcs, s->bcs + s->nbc);
  o->m.ncells = ncell;
  finish(o);
  o->m.ncells = ncell;
  return FPSI_OK;
}

}  // namespace

extern "C" int fpsi_mesh_generate(const fpsi_mesh_spec* s, fpsi_mesh** out) {
  if (!s || !out) return FPSI_E_INVALID;
  OwnedMesh* o = new (std::nothrow) OwnedMesh();
  if (!o) return FPSI_E_NOMEM;
  std::memset(&o->m, 0, sizeof(o->m));
  int rc;
  try {
    if (s->kind == 0)
      rc = gen_hex(s, o, false);
    else if (s->kind == 1)
      rc = gen_kuhn(s, o);
    else if (s->kind == 2)
      rc = gen_hex(s, o, true);
    else if (s->kind == 3)
      rc = gen_hex(s, o, false, true);
    else
      rc = FPSI_E_INVALID;
  } catch (const std::bad_alloc&) {
    rc = FPSI_E_NOMEM;
  }
  if (rc) {
    delete o;
    return rc;
  }
  static_assert(offsetof(OwnedMesh, m) == 0, "fpsi_mesh must lead OwnedMesh");
  *out = &o->m;
  return FPSI_OK;
}

extern "C" void fpsi_mesh_free(fpsi_mesh* m) {
  if (!m) return;
  delete reinterpret_cast<OwnedMesh*>(m);
}
