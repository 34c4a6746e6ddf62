// fpsi_internal.h -- device context of the B200 implicit path (not part of the ABI).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/fpsi.h"

namespace fpsi {

// doubles per face record of the flux array: the flux (5) and maxev_f*area,
// 48 B so that the record is three aligned 16 B accesses
constexpr int FREC = 6;
// doubles per cell record of the reconstruction array: the gradient (15,
// d(T,u,v,w,pg)/dx, y, z) then the limiter (5); 160 B, ten aligned 16 B
// accesses
constexpr int GPREC = 20;
// doubles per face of the reconstructed face states: per side (cl, then cr
// or the boundary state) T, u, v, w, pg at the face and the side's spectral
// radius |u.n| + a of its cell-centre state; 96 B, six aligned 16 B accesses
constexpr int QFREC = 12;
// doubles per residual-norm record: rtrms, etrms, mtrms, rtmax, its cell,
// etmax, its cell, mtmax, the boundary-condition error bits of that
// residual (flowPsiIO.h:212-215), one spare
constexpr int NREC = 10;

void set_error(const char* fmt, ...);

#define FPSI_CUDA_TRY(expr)                                                          \
  do {                                                                               \
    cudaError_t e_ = (expr);                                                         \
    if (e_ != cudaSuccess) {                                                         \
      ::fpsi::set_error("%s:%d %s: %s", __FILE__, __LINE__, #expr, cudaGetErrorString(e_)); \
      return FPSI_E_CUDA;                                                            \
    }                                                                                \
  } while (0)

// Host-side mesh after setup: RCM cell order, faces sorted by (cl, cr) with
// interior faces first and boundary faces last.
struct HostMesh {
  int64_t nc = 0, nf = 0, nfi = 0, nbf = 0;
  std::vector<int32_t> perm;     // new cell id -> caller cell id
  std::vector<int32_t> iperm;    // caller cell id -> new cell id
  std::vector<int64_t> fperm;    // new face id -> caller face id
  std::vector<int32_t> cl, cr;   // new numbering; cr < 0 = -(bc)-1
  std::vector<double> n, area;   // n: nf*3 (AoS on host)
  std::vector<double> rL, rR;    // nf*3
  std::vector<double> vol, cc;   // nc, nc*3
  std::vector<double> Minv;      // nc*6
  std::vector<double> an_caller, area_caller, fc_caller;  // caller order, for export
  std::vector<int32_t> cf_off;   // nc+1
  std::vector<int32_t> cf;       // (face << 1) | side ; upper, lower, boundary order
  // the same lists entry-major: entry j of cell c at [j * nc + c], j below
  // ell_k (the largest face count of a cell), -1 past a cell's last face;
  // a warp's 32 consecutive cells read entry j as one coalesced 128 B line
  int32_t ell_k = 0;
  std::vector<int32_t> ecf;      // ell_k * nc: cf entries
  std::vector<int32_t> enb;      // ell_k * nc: the interior neighbour, -1 on boundary faces
  std::vector<int32_t> colour;   // nc (new numbering)
  int ncolours = 0;
  std::vector<int32_t> colour_off;   // ncolours+1 into colour_cells
  std::vector<int32_t> colour_cells; // cells of each colour, increasing
  // colour order: ci = position in colour_cells.  The sweeps keep every
  // per-cell array of one colour contiguous (structure of arrays inside the
  // colour) and the off-diagonal blocks in slots: slot s of colour k holds,
  // for each of its n_k cells, the block coupling to the s-th interior
  // neighbour (upper faces first, then lower faces, as the cell's face list).
  // Every structure-of-arrays row of a colour has a leading dimension ld_k
  // = n_k rounded up to 32, so a warp's 32 consecutive cells read whole
  // aligned 128 B lines (FP32) and no DRAM burst straddles two rows.
  std::vector<int32_t> ci_of;        // RCM cell -> colour-order index
  std::vector<int64_t> col_n, col_cb, col_m, col_ld, col_cbp, col_ebp;
  std::vector<int32_t> nbr;          // padded slots: ci of the slot's neighbour, -1 = empty
  int64_t ncp = 0;                   // sum ld_k  (padded cells)
  int64_t nslots = 0;                // sum m_k ld_k  (padded slots)
  double vol_tot = 0;
};

// per-colour description passed to the kernels: cb = first ci of the colour
// (iterate, pivots), n cells, m slots per cell, ld row stride, cbp and ebp
// padded bases of the per-cell rows and of the slots
struct ColInfo {
  int64_t cb, n, m, ld, cbp, ebp;
};

int build_host_mesh(const fpsi_mesh* m, HostMesh& h);

// Line structure of the line-SGS solver.  Lines are coloured (no two lines
// of one colour couple) and packed 32 to a group; a group's cells are stored
// position-major: cell p of lane l of group g sits at t = (row0_g + p)*32 + l,
// so the 32 threads walking the group's lines read coalesced rows.
struct LineLayout {
  bool built = false;
  int64_t nlines = 0, ngroups = 0, nrows = 0;   // nrows = sum of group lengths
  int ncolours = 0;
  std::vector<int64_t> col_goff;   // ncolours+1: groups of colour k
  std::vector<int64_t> grp_row0;   // per group: first row
  std::vector<int32_t> grp_len;    // per group: longest line
  std::vector<int32_t> lane_len;   // per group*32+lane: line length (0 = empty lane)
  std::vector<int32_t> t_of;       // RCM cell -> t
  std::vector<int32_t> c_of_t;     // t -> RCM cell, -1 for padding
  std::vector<int8_t> role;        // per cf entry: 0 boundary, 1 prev, 2 next, 3+s outer slot s
  int mout = 0;                    // outer slots per cell
  std::vector<int32_t> onbr;       // [(row*mout + s)*32 + lane]: t of the outer neighbour or -1
  std::vector<int32_t> line_of;    // RCM cell -> line id (caller-visible order)
  std::vector<int32_t> line_colour;  // per line id
};

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
};

}  // namespace fpsi

struct fpsi_prof_rec {
  const char* name;
  cudaEvent_t a, b;
};

struct fpsi_ctx {
  fpsi_params P;
  fpsi::HostMesh H;
  std::vector<fpsi_bc> bcs;
  int device = 0;
  cudaStream_t stream = nullptr;
  // ---- device arrays (new numbering) ----
  // geometry
  int32_t *d_cl = nullptr, *d_cr = nullptr;
  double *d_n = nullptr, *d_area = nullptr;      // SoA: n[3][nf], area[nf]
  double *d_rL = nullptr, *d_rR = nullptr;       // SoA: [3][nf]
  double *d_vol = nullptr, *d_cc = nullptr;      // vol[nc], cc[3][nc]
  double* d_Minv = nullptr;                      // [6][nc]
  int32_t *d_cf_off = nullptr, *d_cf = nullptr;
  int32_t *d_ecf = nullptr, *d_enb = nullptr;  // entry-major cell-face lists
  // low-dissipation (KEC) flux: alpha_diss per cell, alpha_geom_f per
  // interior face (FP32) and the switches it was computed with
  double* d_adiss = nullptr;
  float* d_ageom = nullptr;
  double ageom_coeff = -1.0, ageom_factor = -1.0;
  int32_t* d_colour_cells = nullptr;
  fpsi_bc* d_bcs = nullptr;
  double* d_bcmean = nullptr;  // [nbc][2]: sum of A pg and of A over each condition's faces
  bool any_pmean = false;      // a pMean outflow is present
  bool any_fdbc = false;       // a total-pressure or fixed-mass inflow is present
  void* d_bjac = nullptr;      // [nbf][25] TB: their difference Jacobian blocks
  // state and residual
  double* d_q = nullptr;       // [nc][5]  T,u,v,w,pg
  // time-accurate mode: the states of time levels n and n-1 (as d_q)
  double* d_qn = nullptr;
  double* d_qnm1 = nullptr;
  bool have_levels = false;
  double* d_qb = nullptr;      // [nbf][5] boundary face states
  double* d_grad = nullptr;    // [nc][GPREC]: gradient (15) and limiter (5) per cell
  bool grad_valid = false;     // d_grad holds the last residual's records (viscous runs
                               // write them every residual, others on request)
  double* d_qf = nullptr;      // [nf][QFREC]: reconstructed face states of the last residual
  double* d_F = nullptr;       // [nf][FREC]: face flux (5) and maxev_f * area
  double* d_src = nullptr;     // [nc][5]
  double* d_dtau = nullptr;    // [nc]
  double* d_tmu = nullptr;     // [nc] eddy viscosity (flowRegime turbulent)
  double* d_part = nullptr;    // per-block partial norms
  double* d_resid = nullptr;   // 16 doubles: final norms
  double* h_resid = nullptr;   // pinned mirror
  // pinned: a learned step's error bits ([0] assembly, [1] the model) and
  // the update's per-block step fractions, read after its one synchronisation
  int32_t* h_flags = nullptr;
  double* h_amin = nullptr;
  // residual history of fpsi_run / fpsi_run_timed: 8 norms per step on the
  // device and their pinned host mirror, kept for the context's life (grown
  // only for a longer run than any before)
  double* d_hist = nullptr;
  double* h_hist = nullptr;
  int64_t hist_cap = 0;
  // state copy of fpsi_newton_step_ex, to undo a rejected update
  double* d_qsave = nullptr;   // [nc][5]
  int nblk_norm = 0;
  // implicit system (block type depends on precision)
  void* d_fjp = nullptr;       // [nf][25] TB
  void* d_fjm = nullptr;       // [nf][25] TB
  // compact face Jacobians (inviscid SGS): per face [+ (9) | - (9) | U | n] TB;
  // the explicit fjp/fjm are then filled only on request
  void* d_fjc = nullptr;       // [nf][24] TB
  bool asm_compact = false;    // the assembled system's slots are compact
  int jac_fresh = 0;           // block bytes of compact face records written with the
                               // current residual (the fused flux kernel), else 0
  bool have_explicit = false;  // fjp/fjm hold the assembled system's blocks
  void* d_D = nullptr;         // [nc][25] TB (only when keep_D)
  // colour-order arrays of the sweeps (see HostMesh)
  void* d_luc = nullptr;       // per colour [25][n_k] TB: LU factors of fluid_D
  void* d_bc = nullptr;        // per colour [5][n_k] TB: fluid_B
  int32_t* d_pv = nullptr;     // [nc] packed pivots, colour order
  void* d_aoff = nullptr;      // per colour [m_k][25 or 15][n_k] TB: off-diagonal blocks
  int32_t* d_nbr = nullptr;    // per colour [m_k][n_k] neighbour ci
  int32_t* d_ci = nullptr;     // RCM cell -> ci
  int32_t* d_ccol = nullptr;   // RCM cell -> colour
  fpsi::ColInfo* d_colinfo = nullptr;
  void* d_x = nullptr;         // [nc][5] TX, colour order
  double* d_amin = nullptr;    // per-block min alpha
  int32_t* d_err = nullptr;    // error flags (singular pivots, ...)
  int blk_bytes = 4;           // sizeof(TB)
  int x_bytes = 8;             // sizeof(TX)
  int alloc_prec = -1;
  bool keep_D = true;
  bool have_resid = false, have_asm = false, have_dq = false;
  bool x_preset = false;       // the iterate holds a caller-provided start
  // interior-face cell graph (RCM order, CSR), built on first use by the
  // learned start
  int32_t *d_cnb_off = nullptr, *d_cnb = nullptr;
  int64_t cnb_n = 0;
  // copy of the last applied update (colour order, TX), kept once a learned
  // start has used this context: the next system's start uses it as input
  void* d_xprev = nullptr;     // nc * 5 * 8 bytes
  bool keep_prev = false, have_xprev = false;
  // Spalart-Allmaras working variable (RCM order) and its scalar system
  std::vector<double> h_wdist;   // wall distance, RCM order
  double *d_nut = nullptr, *d_wdist = nullptr, *d_sa_grad = nullptr, *d_sa_phi = nullptr;
  double *d_sa_nub = nullptr, *d_sa_face = nullptr;  // [nbf], [7][nf]
  double *d_sa_B = nullptr, *d_sa_D = nullptr, *d_sa_Dinv = nullptr, *d_sa_x = nullptr;
  bool have_sa = false, have_sa_dq = false;
  int64_t device_bytes = 0;
  // caller-order staging for state transfers (T, pg, u) and the permutation
  int32_t* d_perm = nullptr;   // new cell id -> caller cell id
  double* d_stage = nullptr;   // [nc] T, [nc] pg, [3 nc] u (caller order)
  // line SGS (solver == LSGS)
  fpsi::LineLayout LY;
  int32_t *d_lt = nullptr, *d_lonbr = nullptr, *d_llen = nullptr;
  int32_t* d_lct = nullptr;    // line slot t -> RCM cell (-1: padding)
  int8_t* d_lrole = nullptr;
  int64_t* d_lrow0 = nullptr;
  void *d_lD = nullptr, *d_lL = nullptr, *d_lU = nullptr, *d_lF = nullptr, *d_lB = nullptr;
  void *d_lrhs = nullptr, *d_lx = nullptr, *d_lxt = nullptr;
  void* d_lctl = nullptr;
  double* d_lpart = nullptr;
  int lsgs_prec = -1;
  // per-kernel timing (fpsi_kernel_times)
  bool profiling = false;
  std::vector<fpsi_prof_rec> prof;
  std::vector<cudaEvent_t> evpool;
  size_t evnext = 0;
};

namespace fpsi {
void prof_begin(fpsi_ctx* x, const char* name);
void prof_end(fpsi_ctx* x);
// line SGS: layout from caller lines (RCM ids) or the default rule
int build_lines(fpsi_ctx* x, const std::vector<std::vector<int32_t>>* lines);
int lsgs_assemble(fpsi_ctx* x);
int lsgs_solve(fpsi_ctx* x, bool jacobi_start);
// distance to the nearest no-slip wall per cell (RCM order)
void wall_distance(const fpsi_mesh* m, const HostMesh& H, std::vector<double>& out);
// Spalart-Allmaras nu~ (sa.cu)
bool sa_active(const fpsi_ctx* x);
int sa_launch_tmu(fpsi_ctx* x);
int sa_launch_residual(fpsi_ctx* x);
int gnn_predict_launch(fpsi_gnn* m, fpsi_ctx* x, double* dx0, bool jacobi_in_iterate = false);
int32_t* gnn_error_bits(fpsi_gnn* m);  // the model's device error word
int sa_launch_solve(fpsi_ctx* x);
int sa_launch_update(fpsi_ctx* x, const double* guard);
}  // namespace fpsi
