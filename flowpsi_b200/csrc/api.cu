// api.cu -- the C ABI (include/fpsi.h) over the device path.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "fpsi_internal.h"
#include "kernels.cuh"

using fpsi::HostMesh;

namespace fpsi {
static cudaEvent_t prof_event(fpsi_ctx* x) {
  if (x->evnext == x->evpool.size()) {
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    x->evpool.push_back(e);
  }
  return x->evpool[x->evnext++];
}
void prof_begin(fpsi_ctx* x, const char* name) {
  if (!x->profiling) return;
  fpsi_prof_rec r;
  r.name = name;
  r.a = prof_event(x);
  r.b = prof_event(x);
  cudaEventRecord(r.a, x->stream);
  x->prof.push_back(r);
}
void prof_end(fpsi_ctx* x) {
  if (!x->profiling || x->prof.empty()) return;
  cudaEventRecord(x->prof.back().b, x->stream);
}
}  // namespace fpsi

namespace {

template <class T>
int dalloc(fpsi_ctx* x, T** p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess) {
    fpsi::set_error("cudaMalloc(%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
    *p = nullptr;
    return e == cudaErrorMemoryAllocation ? FPSI_E_NOMEM : FPSI_E_CUDA;
  }
  x->device_bytes += int64_t(n * sizeof(T));
  return FPSI_OK;
}

template <class T>
int upload(fpsi_ctx* x, T** p, const std::vector<T>& h) {
  int rc = dalloc(x, p, h.size());
  if (rc) return rc;
  if (!h.empty()) FPSI_CUDA_TRY(cudaMemcpy(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  return FPSI_OK;
}

// AoS [n][3] -> SoA [3][n]
std::vector<double> soa3(const std::vector<double>& a, int64_t n) {
  std::vector<double> r(3 * n);
  for (int64_t i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) r[d * n + i] = a[3 * i + d];
  return r;
}

void free_system(fpsi_ctx* x) {
  void* ps[] = {x->d_fjp, x->d_fjm, x->d_fjc, x->d_D, x->d_x, x->d_luc, x->d_bc, x->d_pv, x->d_aoff,
                x->d_bjac};
  for (void* p : ps)
    if (p) cudaFree(p);
  x->d_fjp = x->d_fjm = x->d_fjc = x->d_D = x->d_x = x->d_luc = x->d_bc = x->d_aoff = nullptr;
  x->d_bjac = nullptr;
  x->d_pv = nullptr;
}

int alloc_system(fpsi_ctx* x) {
  if (x->alloc_prec == x->P.precision) return FPSI_OK;
  free_system(x);
  const int tb = x->P.precision == FPSI_PREC_FP64 ? 8 : 4;
  const int tx = x->P.precision == FPSI_PREC_MIXED ? 4 : 8;
  x->blk_bytes = tb;
  x->x_bytes = tx;
  const size_t nf = size_t(x->H.nf), nc = size_t(x->H.nc);
  int rc;
  if ((rc = dalloc(x, (char**)&x->d_fjp, nf * 25 * tb))) return rc;
  if ((rc = dalloc(x, (char**)&x->d_fjm, nf * 25 * tb))) return rc;
  if ((rc = dalloc(x, (char**)&x->d_fjc, nf * 24 * tb))) return rc;
  const size_t ncp = size_t(x->H.ncp);
  if ((rc = dalloc(x, (char**)&x->d_luc, ncp * 25 * tb))) return rc;
  if ((rc = dalloc(x, (char**)&x->d_bc, ncp * 5 * tb))) return rc;
  if ((rc = dalloc(x, &x->d_pv, nc))) return rc;
  if ((rc = dalloc(x, (char**)&x->d_aoff, size_t(x->H.nslots) * 25 * tb))) return rc;
  if (x->keep_D)
    if ((rc = dalloc(x, (char**)&x->d_D, nc * 25 * tb))) return rc;
  if ((rc = dalloc(x, (char**)&x->d_x, nc * 5 * tx))) return rc;
  if (x->any_fdbc && (rc = dalloc(x, (char**)&x->d_bjac, size_t(std::max<int64_t>(x->H.nbf, 1)) * 25 * tb)))
    return rc;
  x->alloc_prec = x->P.precision;
  x->have_asm = x->have_dq = false;
  return FPSI_OK;
}

void free_lsgs(fpsi_ctx* x) {
  void* ps[] = {x->d_lt, x->d_lct, x->d_lonbr, x->d_llen, x->d_lrole, x->d_lrow0, x->d_lD, x->d_lL,
                x->d_lU, x->d_lF, x->d_lB, x->d_lrhs, x->d_lx, x->d_lxt, x->d_lctl, x->d_lpart};
  for (void* p : ps)
    if (p) cudaFree(p);
  x->d_lt = x->d_lct = x->d_lonbr = x->d_llen = nullptr;
  x->d_lrole = nullptr;
  x->d_lrow0 = nullptr;
  x->d_lD = x->d_lL = x->d_lU = x->d_lF = x->d_lB = x->d_lrhs = x->d_lx = x->d_lxt = nullptr;
  x->d_lctl = nullptr;
  x->d_lpart = nullptr;
  x->lsgs_prec = -1;
}

// device arrays of the line solver for the current line layout and precision
void free_sa(fpsi_ctx* x) {
  double* ps[] = {x->d_nut, x->d_wdist, x->d_sa_grad, x->d_sa_phi, x->d_sa_nub,
                  x->d_sa_face, x->d_sa_B, x->d_sa_D, x->d_sa_Dinv, x->d_sa_x};
  for (double* p : ps)
    if (p) cudaFree(p);
  x->d_nut = x->d_wdist = x->d_sa_grad = x->d_sa_phi = x->d_sa_nub = nullptr;
  x->d_sa_face = x->d_sa_B = x->d_sa_D = x->d_sa_Dinv = x->d_sa_x = nullptr;
  x->have_sa = x->have_sa_dq = false;
}

// Spalart-Allmaras arrays, on first use of the model; nu~ starts at the
// reference's nuTilde_ic default 1e-6 (SA_ic.loci:39-50)
int alloc_sa(fpsi_ctx* x) {
  if (!fpsi::sa_active(x) || x->d_nut) return FPSI_OK;
  const int64_t nc = x->H.nc, nf = x->H.nf;
  int rc;
  if ((rc = dalloc(x, &x->d_nut, nc))) return rc;
  if ((rc = dalloc(x, &x->d_wdist, nc))) return rc;
  if ((rc = dalloc(x, &x->d_sa_grad, nc * 3))) return rc;
  if ((rc = dalloc(x, &x->d_sa_phi, nc))) return rc;
  if ((rc = dalloc(x, &x->d_sa_nub, std::max<int64_t>(x->H.nbf, 1)))) return rc;
  if ((rc = dalloc(x, &x->d_sa_face, nf * 7))) return rc;
  if ((rc = dalloc(x, &x->d_sa_B, nc))) return rc;
  if ((rc = dalloc(x, &x->d_sa_D, nc))) return rc;
  if ((rc = dalloc(x, &x->d_sa_Dinv, nc))) return rc;
  if ((rc = dalloc(x, &x->d_sa_x, nc))) return rc;
  std::vector<double> v(nc, 1e-6);
  FPSI_CUDA_TRY(cudaMemcpy(x->d_nut, v.data(), nc * sizeof(double), cudaMemcpyHostToDevice));
  FPSI_CUDA_TRY(cudaMemcpy(x->d_wdist, x->h_wdist.data(), nc * sizeof(double), cudaMemcpyHostToDevice));
  return FPSI_OK;
}

int alloc_lsgs(fpsi_ctx* x) {
  if (x->P.solver != FPSI_SOLVER_LSGS) return FPSI_OK;
  int rc;
  if (!x->LY.built && (rc = fpsi::build_lines(x, nullptr))) return rc;
  if (x->lsgs_prec == x->P.precision && x->d_lt) return FPSI_OK;
  free_lsgs(x);
  const fpsi::LineLayout& Y = x->LY;
  const int tb = x->P.precision == FPSI_PREC_FP64 ? 8 : 4;
  const int td = x->P.precision == FPSI_PREC_MIXED ? 4 : 8;
  const int tx = td;
  const size_t nt = size_t(Y.nrows) * 32;
  if ((rc = upload(x, &x->d_lt, Y.t_of))) return rc;
  if ((rc = upload(x, &x->d_lct, Y.c_of_t))) return rc;
  if ((rc = upload(x, &x->d_lrole, Y.role))) return rc;
  if ((rc = upload(x, &x->d_lonbr, Y.onbr))) return rc;
  if ((rc = upload(x, &x->d_llen, Y.lane_len))) return rc;
  if ((rc = upload(x, &x->d_lrow0, Y.grp_row0))) return rc;
  if ((rc = dalloc(x, (char**)&x->d_lD, nt * 25 * td))) return rc;
  if ((rc = dalloc(x, (char**)&x->d_lL, nt * 25 * tb))) return rc;
  if ((rc = dalloc(x, (char**)&x->d_lU, nt * 25 * tb))) return rc;
  if ((rc = dalloc(x, (char**)&x->d_lF, nt * size_t(Y.mout) * 25 * tb))) return rc;
  if ((rc = dalloc(x, (char**)&x->d_lB, nt * 5 * tb))) return rc;
  if ((rc = dalloc(x, (char**)&x->d_lrhs, nt * 5 * tx))) return rc;
  if ((rc = dalloc(x, (char**)&x->d_lx, nt * 5 * tx))) return rc;
  if ((rc = dalloc(x, (char**)&x->d_lxt, nt * 5 * tx))) return rc;
  if ((rc = dalloc(x, (char**)&x->d_lctl, 64))) return rc;
  if ((rc = dalloc(x, &x->d_lpart, (nt + 255) / 256 + 1))) return rc;
  // padding cells must read as zero in the relaxation and the residual
  FPSI_CUDA_TRY(cudaMemset(x->d_lx, 0, nt * 5 * tx));
  FPSI_CUDA_TRY(cudaMemset(x->d_lxt, 0, nt * 5 * tx));
  FPSI_CUDA_TRY(cudaMemset(x->d_lB, 0, nt * 5 * tb));
  x->lsgs_prec = x->P.precision;
  x->keep_D = true;  // the line preprocessing starts from the unfactored blocks
  return FPSI_OK;
}

// residual history for runs of up to n steps (8 doubles per step)
int ensure_hist(fpsi_ctx* x, int64_t n) {
  if (n <= x->hist_cap) return FPSI_OK;
  if (x->d_hist) {
    x->device_bytes -= x->hist_cap * fpsi::NREC * int64_t(sizeof(double));
    cudaFree(x->d_hist);
    x->d_hist = nullptr;
  }
  if (x->h_hist) cudaFreeHost(x->h_hist);
  x->h_hist = nullptr;
  x->hist_cap = 0;
  int rc = dalloc(x, &x->d_hist, size_t(n) * fpsi::NREC);
  if (rc) return rc;
  if (cudaMallocHost((void**)&x->h_hist, size_t(n) * fpsi::NREC * sizeof(double)) != cudaSuccess) {
    fpsi::set_error("cudaMallocHost of the residual history failed");
    return FPSI_E_NOMEM;
  }
  x->hist_cap = n;
  return FPSI_OK;
}

bool is_lsgs(const fpsi_ctx* x) { return x->P.solver == FPSI_SOLVER_LSGS; }

int check_params(const fpsi_params* p) {
  if (!p) return FPSI_E_INVALID;
  if (!(p->gamma > 1.0) || !(p->Rtilde > 0) || p->flux < 0 || p->flux > FPSI_FLUX_SSF || p->limiter < 0 ||
      p->limiter > 3 || p->precision < 0 || p->precision > 2 || p->gauss_seidel_iter < 0) {
    fpsi::set_error("invalid parameter value");
    return FPSI_E_INVALID;
  }
  if (p->Minf < 0.5) {
    fpsi::set_error("low-Mach preconditioning (Minf < 0.5) is not on the device path");
    return FPSI_E_UNSUPPORTED;
  }
  if (p->solver != FPSI_SOLVER_SGS && p->solver != FPSI_SOLVER_LSGS && p->solver != FPSI_SOLVER_FSGS) {
    fpsi::set_error("fluidLinearSolver: 'sgs', 'lsgs' or 'fsgs'");
    return FPSI_E_INVALID;
  }
  if (p->solver == FPSI_SOLVER_LSGS && (p->lsgs_max_iter < 0 || !(p->lsgs_relaxation > 0))) {
    fpsi::set_error("LSGS controls out of range");
    return FPSI_E_INVALID;
  }
  if (p->viscous < 0 || p->viscous > 2 ||
      (p->viscous && (!(p->mu_a1 > 0) || !(p->k_a1 > 0) || !(p->Prt > 0)))) {
    fpsi::set_error("flowRegime / Sutherland parameters out of range");
    return FPSI_E_INVALID;
  }
  if (p->turbulence < 0 || p->turbulence > 1 || (p->turbulence == FPSI_TURB_SA && p->viscous != 2)) {
    fpsi::set_error("turbulence: 0 (given eddy viscosity) or 1 (SA, needs viscous = 2)");
    return FPSI_E_INVALID;
  }
  if (p->time_accurate < 0 || p->time_accurate > 1 || (p->time_accurate && p->newton_iters < 1)) {
    fpsi::set_error("time_accurate: 0 (steady) or 1 (BDF2, newton_iters >= 1)");
    return FPSI_E_INVALID;
  }
  if (p->time_accurate && p->turbulence == FPSI_TURB_SA && p->viscous == 2) {
    fpsi::set_error("the SA model is advanced in steady mode only");
    return FPSI_E_UNSUPPORTED;
  }
  if ((p->flux == FPSI_FLUX_KEC || p->flux == FPSI_FLUX_SSF) &&
      (!(p->lds_comp_factor >= 0) || !(p->lds_dissipation_limit >= 0) || !(p->lds_ducros_factor >= 0) ||
       !(p->lds_use_upwind >= 0) || !(p->lds_nonsym_coeff > 0) || !(p->lds_nonsym_factor >= 0) ||
       !(p->lds_miles_filter >= 0) || !(p->ssf_coeff == p->ssf_coeff))) {
    fpsi::set_error("low-dissipation flux switches out of range");
    return FPSI_E_INVALID;
  }
  if (p->step_graphs < 0 || p->step_graphs > 1) {
    fpsi::set_error("step_graphs must be 0 or 1");
    return FPSI_E_INVALID;
  }
  return FPSI_OK;
}

int sync(fpsi_ctx* x) {
  FPSI_CUDA_TRY(cudaStreamSynchronize(x->stream));
  return FPSI_OK;
}

void fill_norms(const fpsi_ctx* x, const double* r, fpsi_resid* n) {
  std::memset(n, 0, sizeof(*n));
  n->rtrms = r[0];
  n->etrms = r[1];
  n->mtrms = r[2];
  n->rtmax = r[3];
  n->etmax = r[5];
  n->mtmax = r[7];
  n->bcErrorCode = uint64_t(r[8]);
  const int64_t cr = int64_t(r[4]), ce = int64_t(r[6]);
  if (cr >= 0 && cr < x->H.nc)
    for (int d = 0; d < 3; ++d) n->ccmaxr_center[d] = x->H.cc[3 * cr + d];
  if (ce >= 0 && ce < x->H.nc)
    for (int d = 0; d < 3; ++d) n->ccmaxe_center[d] = x->H.cc[3 * ce + d];
}

bool has_nan(const double* r) { return r[0] != r[0] || r[1] != r[1] || r[2] != r[2]; }

template <class T>
void unpermute_cells(const fpsi_ctx* x, const T* dev_order, int w, T* caller) {
  const int64_t nc = x->H.nc;
  for (int64_t i = 0; i < nc; ++i) {
    const int64_t c = x->H.perm[i];
    for (int k = 0; k < w; ++k) caller[w * c + k] = dev_order[w * i + k];
  }
}

}  // namespace

extern "C" {

void fpsi_default_params(fpsi_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->gamma = 1.4;
  p->Rtilde = 8314.4621 / 28.96;
  p->Pambient = 0.0;
  p->Minf = 1.0;
  p->flux = FPSI_FLUX_HLLC;
  p->limiter = FPSI_LIMITER_VENKATAKRISHNAN;
  p->Kl = 1.0;
  p->urelax = 0.2;
  p->dtmax = 1.0;
  p->cflmax = 0.0;
  p->solver = FPSI_SOLVER_LSGS;
  p->gauss_seidel_iter = 6;
  p->lsgs_relaxation = 0.25;
  p->lsgs_abs_tol = 1e-10;
  p->lsgs_rel_tol = 0.1;
  p->lsgs_max_iter = 10;
  p->precision = FPSI_PREC_REF;
  p->viscous = 0;
  p->Prt = 0.9;
  p->mu_a1 = 1.458e-6;
  p->mu_a2 = 1.5;
  p->mu_a3 = 110.4;
  p->k_a1 = 2.495e-3;
  p->k_a2 = 1.5;
  p->k_a3 = 194.0;
  p->time_accurate = 0;
  p->newton_iters = 6;
  p->lds_comp_factor = 5.0;
  p->lds_dissipation_limit = 1.0;
  p->lds_ducros_factor = 0.0;
  p->lds_use_upwind = 0.0;
  p->lds_nonsym_coeff = 2.0;
  p->lds_nonsym_factor = 1.0;
  p->lds_miles_filter = 0.1;
  p->ssf_coeff = 1.0;
  p->step_graphs = 1;
}

const char* fpsi_strerror(int code) {
  switch (code) {
    case FPSI_OK: return "ok";
    case FPSI_E_INVALID: return "invalid argument";
    case FPSI_E_CUDA: return "CUDA error";
    case FPSI_E_NOMEM: return "out of memory";
    case FPSI_E_UNSUPPORTED: return "unsupported option";
    case FPSI_E_SINGULAR: return "singular diagonal block";
    case FPSI_E_NAN: return "NaN residual";
    case FPSI_E_TIMEOUT: return "device wait timed out";
    case FPSI_E_STATE: return "call out of order";
    default: return "unknown error";
  }
}

const char* fpsi_last_error(void) { return fpsi::last_error(); }

int fpsi_device_available(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n > 0;
}

int fpsi_destroy(fpsi_ctx* x) {
  if (!x) return FPSI_OK;
  free_system(x);
  free_lsgs(x);
  free_sa(x);
  void* ps[] = {x->d_cl, x->d_cr, x->d_n, x->d_area, x->d_rL, x->d_rR, x->d_vol, x->d_cc,
                x->d_Minv, x->d_cf_off, x->d_cf, x->d_ecf, x->d_enb, x->d_colour_cells, x->d_bcs, x->d_bcmean, x->d_q,
                x->d_qn, x->d_qnm1, x->d_qb, x->d_grad, x->d_qf, x->d_F, x->d_src, x->d_dtau, x->d_tmu,
                x->d_part, x->d_resid, x->d_amin, x->d_err, x->d_perm, x->d_stage, x->d_ci, x->d_ccol,
                x->d_nbr, x->d_colinfo, x->d_cnb_off, x->d_cnb, x->d_xprev, x->d_qsave, x->d_adiss, x->d_ageom};
  for (void* p : ps)
    if (p) cudaFree(p);
  if (x->h_resid) cudaFreeHost(x->h_resid);
  if (x->h_flags) cudaFreeHost(x->h_flags);
  if (x->h_amin) cudaFreeHost(x->h_amin);
  if (x->d_hist) cudaFree(x->d_hist);
  if (x->h_hist) cudaFreeHost(x->h_hist);
  for (cudaEvent_t e : x->evpool) cudaEventDestroy(e);
  if (x->stream) cudaStreamDestroy(x->stream);
  delete x;
  return FPSI_OK;
}

int fpsi_create(fpsi_ctx** out, const fpsi_mesh* mesh, const fpsi_params* params) {
  if (!out || !mesh || !params) return FPSI_E_INVALID;
  *out = nullptr;
  int rc = check_params(params);
  if (rc) return rc;
  if (!fpsi_device_available()) {
    fpsi::set_error("no CUDA device");
    return FPSI_E_CUDA;
  }
  fpsi_ctx* x = new (std::nothrow) fpsi_ctx();
  if (!x) return FPSI_E_NOMEM;
  x->P = *params;
  try {
    rc = fpsi::build_host_mesh(mesh, x->H);
  } catch (const std::bad_alloc&) {
    rc = FPSI_E_NOMEM;
  }
  if (rc) {
    delete x;
    return rc;
  }
  x->bcs.assign(mesh->bcs, mesh->bcs + mesh->nbc);
  for (const fpsi_bc& b : x->bcs)
    if (b.kind < FPSI_BC_FARFIELD || b.kind > FPSI_BC_INFLOW) {
      fpsi::set_error("boundary condition kind %d is not on the device path", b.kind);
      delete x;
      return FPSI_E_UNSUPPORTED;
    }
  const HostMesh& H = x->H;
  const int64_t nc = H.nc, nf = H.nf;
#define TRY(e)                \
  do {                        \
    int rc_ = (e);            \
    if (rc_) {                \
      fpsi_destroy(x);        \
      return rc_;             \
    }                         \
  } while (0)
  if (cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking) != cudaSuccess) {
    fpsi::set_error("cudaStreamCreate failed");
    delete x;
    return FPSI_E_CUDA;
  }
  TRY(upload(x, &x->d_cl, H.cl));
  TRY(upload(x, &x->d_cr, H.cr));
  TRY(upload(x, &x->d_n, soa3(H.n, nf)));
  TRY(upload(x, &x->d_area, H.area));
  TRY(upload(x, &x->d_rL, soa3(H.rL, nf)));
  TRY(upload(x, &x->d_rR, soa3(H.rR, nf)));
  TRY(upload(x, &x->d_vol, H.vol));
  TRY(upload(x, &x->d_cc, soa3(H.cc, nc)));
  {
    std::vector<double> m(6 * nc);
    for (int64_t c = 0; c < nc; ++c)
      for (int k = 0; k < 6; ++k) m[k * nc + c] = H.Minv[6 * c + k];
    TRY(upload(x, &x->d_Minv, m));
  }
  TRY(upload(x, &x->d_cf_off, H.cf_off));
  TRY(upload(x, &x->d_cf, H.cf));
  TRY(upload(x, &x->d_ecf, H.ecf));
  TRY(upload(x, &x->d_enb, H.enb));
  TRY(upload(x, &x->d_colour_cells, H.colour_cells));
  TRY(upload(x, &x->d_perm, H.perm));
  TRY(upload(x, &x->d_ci, H.ci_of));
  TRY(upload(x, &x->d_ccol, H.colour));
  TRY(upload(x, &x->d_nbr, H.nbr));
  {
    std::vector<fpsi::ColInfo> ci(H.ncolours);
    for (int k = 0; k < H.ncolours; ++k)
      ci[k] = fpsi::ColInfo{H.col_cb[k], H.col_n[k], H.col_m[k], H.col_ld[k], H.col_cbp[k],
                            H.col_ebp[k]};
    TRY(upload(x, &x->d_colinfo, ci));
  }
  TRY(dalloc(x, &x->d_stage, nc * 5));
  // fixed-mass conditions given by mdot: the mass flux over the condition's
  // area (massFlux_BC = mdot_BC / boundary_area, bcFixedMass.loci:227-230)
  {
    std::vector<double> barea(x->bcs.size(), 0.0);
    for (int64_t f = H.nfi; f < H.nf; ++f) barea[-H.cr[f] - 1] += H.area[f];
    for (size_t b = 0; b < x->bcs.size(); ++b) {
      fpsi_bc& bc = x->bcs[b];
      const bool fm = bc.kind == FPSI_BC_FIXED_MASS_INFLOW || bc.kind == FPSI_BC_FIXED_MASS_OUTFLOW;
      if (fm && !(bc.mass_flux > 0) && barea[b] > 0) bc.mass_flux = bc.mdot / barea[b];
      x->any_fdbc = x->any_fdbc || bc.kind == FPSI_BC_ISENTROPIC_INFLOW ||
                    bc.kind == FPSI_BC_FIXED_MASS_INFLOW;
    }
  }
  TRY(upload(x, &x->d_bcs, x->bcs));
  TRY(dalloc(x, &x->d_bcmean, std::max<size_t>(x->bcs.size(), 1) * 2));
  for (const fpsi_bc& b : x->bcs) x->any_pmean = x->any_pmean || b.kind == FPSI_BC_OUTFLOW_MEAN;
  TRY(dalloc(x, &x->d_q, nc * 5));
  TRY(dalloc(x, &x->d_qn, nc * 5));
  TRY(dalloc(x, &x->d_qnm1, nc * 5));
  TRY(dalloc(x, &x->d_qb, std::max<int64_t>(H.nbf, 1) * 5));
  TRY(dalloc(x, &x->d_grad, nc * fpsi::GPREC));
  TRY(dalloc(x, &x->d_qf, nf * fpsi::QFREC));
  TRY(dalloc(x, &x->d_F, nf * fpsi::FREC));
  TRY(dalloc(x, &x->d_src, nc * 5));
  TRY(dalloc(x, &x->d_dtau, nc));
  TRY(dalloc(x, &x->d_tmu, nc));
  if (cudaMemset(x->d_tmu, 0, nc * sizeof(double)) != cudaSuccess) {
    fpsi_destroy(x);
    return FPSI_E_CUDA;
  }
  x->nblk_norm = int((nc + 255) / 256);
  TRY(dalloc(x, &x->d_part, size_t(x->nblk_norm) * 8));
  TRY(dalloc(x, &x->d_resid, 32));
  TRY(dalloc(x, &x->d_amin, size_t(x->nblk_norm)));
  TRY(dalloc(x, &x->d_err, 4));
  if (cudaMallocHost((void**)&x->h_resid, 32 * sizeof(double)) != cudaSuccess ||
      cudaMallocHost((void**)&x->h_flags, 4 * sizeof(int32_t)) != cudaSuccess ||
      cudaMallocHost((void**)&x->h_amin, size_t(x->nblk_norm) * sizeof(double)) != cudaSuccess) {
    fpsi_destroy(x);
    return FPSI_E_NOMEM;
  }
  if (cudaMemset(x->d_err, 0, 4 * sizeof(int32_t)) != cudaSuccess) {
    fpsi_destroy(x);
    return FPSI_E_CUDA;
  }
  TRY(ensure_hist(x, 4096));
  if (params->solver == FPSI_SOLVER_LSGS) x->keep_D = true;
  TRY(alloc_system(x));
  TRY(alloc_lsgs(x));
  fpsi::wall_distance(mesh, x->H, x->h_wdist);
  TRY(alloc_sa(x));
#undef TRY
  *out = x;
  return FPSI_OK;
}

int fpsi_set_params(fpsi_ctx* x, const fpsi_params* p) {
  if (!x) return FPSI_E_INVALID;
  int rc = check_params(p);
  if (rc) return rc;
  x->P = *p;
  x->have_asm = x->have_dq = x->have_xprev = false;
  x->have_levels = false;
  if (is_lsgs(x) && !x->keep_D) {
    x->keep_D = true;
    x->alloc_prec = -1;
  }
  rc = alloc_system(x);
  if (rc) return rc;
  if ((rc = alloc_sa(x))) return rc;
  x->have_sa = x->have_sa_dq = false;
  return alloc_lsgs(x);
}

int fpsi_info(fpsi_ctx* x, int64_t* nc, int64_t* nf, int32_t* ncol, int64_t* bytes) {
  if (!x) return FPSI_E_INVALID;
  if (nc) *nc = x->H.nc;
  if (nf) *nf = x->H.nf;
  if (ncol) *ncol = x->H.ncolours;
  if (bytes) *bytes = x->device_bytes;
  return FPSI_OK;
}

int fpsi_get_geometry(fpsi_ctx* x, double* vol, double* cellcenter, double* face_an,
                      double* face_area, double* facecenter) {
  if (!x) return FPSI_E_INVALID;
  if (vol) unpermute_cells(x, x->H.vol.data(), 1, vol);
  if (cellcenter) unpermute_cells(x, x->H.cc.data(), 3, cellcenter);
  if (face_an) std::memcpy(face_an, x->H.an_caller.data(), sizeof(double) * 3 * x->H.nf);
  if (face_area) std::memcpy(face_area, x->H.area_caller.data(), sizeof(double) * x->H.nf);
  if (facecenter) std::memcpy(facecenter, x->H.fc_caller.data(), sizeof(double) * 3 * x->H.nf);
  return FPSI_OK;
}

int fpsi_get_colours(fpsi_ctx* x, int32_t* colour) {
  if (!x || !colour) return FPSI_E_INVALID;
  unpermute_cells(x, x->H.colour.data(), 1, colour);
  return FPSI_OK;
}

int fpsi_set_lines(fpsi_ctx* x, int64_t nlines, const int64_t* line_off,
                   const int32_t* line_cells) {
  if (!x || nlines < 0 || (nlines > 0 && (!line_off || !line_cells))) return FPSI_E_INVALID;
  std::vector<std::vector<int32_t>> lines(nlines);
  for (int64_t l = 0; l < nlines; ++l) {
    if (line_off[l + 1] < line_off[l]) return FPSI_E_INVALID;
    for (int64_t k = line_off[l]; k < line_off[l + 1]; ++k) {
      const int32_t c = line_cells[k];
      if (c < 0 || c >= x->H.nc) {
        fpsi::set_error("fpsi_set_lines: cell %d out of range", c);
        return FPSI_E_INVALID;
      }
      lines[l].push_back(x->H.iperm[c]);
    }
  }
  int rc = fpsi::build_lines(x, &lines);
  if (rc) return rc;
  x->lsgs_prec = -1;
  x->have_asm = x->have_dq = false;
  return alloc_lsgs(x);
}

int fpsi_get_lines(fpsi_ctx* x, int32_t* line_of_cell, int32_t* position, int32_t* line_colour,
                   int64_t* nlines) {
  if (!x) return FPSI_E_INVALID;
  if (!x->LY.built) {
    int rc = fpsi::build_lines(x, nullptr);
    if (rc) return rc;
  }
  const fpsi::LineLayout& Y = x->LY;
  if (nlines) *nlines = Y.nlines;
  for (int64_t i = 0; i < x->H.nc; ++i) {
    const int64_t c = x->H.perm[i];
    if (line_of_cell) line_of_cell[c] = Y.line_of[i];
    if (position) {
      // position along the line from the padded row of the cell
      const int64_t t = Y.t_of[i], r = t / 32, g_lane = t % 32;
      int64_t g = std::upper_bound(Y.grp_row0.begin(), Y.grp_row0.end(), r) - Y.grp_row0.begin() - 1;
      (void)g_lane;
      position[c] = int32_t(r - Y.grp_row0[g]);
    }
  }
  if (line_colour)
    for (int64_t l = 0; l < Y.nlines; ++l) line_colour[l] = Y.line_colour[l];
  return FPSI_OK;
}

int fpsi_set_eddy_viscosity(fpsi_ctx* x, const double* tmu) {
  if (!x || !tmu) return FPSI_E_INVALID;
  std::vector<double> t(x->H.nc);
  for (int64_t i = 0; i < x->H.nc; ++i) t[i] = tmu[x->H.perm[i]];
  FPSI_CUDA_TRY(cudaMemcpy(x->d_tmu, t.data(), t.size() * sizeof(double), cudaMemcpyHostToDevice));
  x->have_resid = x->have_asm = x->have_dq = false;
  return FPSI_OK;
}

// ---- Spalart-Allmaras nu~ -------------------------------------------------
static int sa_down(fpsi_ctx* x, const double* d, double* out) {
  std::vector<double> h(x->H.nc);
  FPSI_CUDA_TRY(cudaMemcpyAsync(h.data(), d, h.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                x->stream));
  int rc = sync(x);
  if (rc) return rc;
  for (int64_t i = 0; i < x->H.nc; ++i) out[x->H.perm[i]] = h[i];
  return FPSI_OK;
}

int fpsi_set_nutilde(fpsi_ctx* x, const double* nut) {
  if (!x || !nut) return FPSI_E_INVALID;
  if (!x->d_nut) return FPSI_E_STATE;
  std::vector<double> t(x->H.nc);
  for (int64_t i = 0; i < x->H.nc; ++i) t[i] = nut[x->H.perm[i]];
  FPSI_CUDA_TRY(cudaMemcpy(x->d_nut, t.data(), t.size() * sizeof(double), cudaMemcpyHostToDevice));
  x->have_resid = x->have_asm = x->have_dq = x->have_sa = x->have_sa_dq = false;
  return FPSI_OK;
}

int fpsi_get_nutilde(fpsi_ctx* x, double* nut) {
  if (!x || !nut) return FPSI_E_INVALID;
  if (!x->d_nut) return FPSI_E_STATE;
  return sa_down(x, x->d_nut, nut);
}

int fpsi_get_eddy_viscosity(fpsi_ctx* x, double* tmu) {
  if (!x || !tmu) return FPSI_E_INVALID;
  return sa_down(x, x->d_tmu, tmu);
}

int fpsi_get_wall_distance(fpsi_ctx* x, double* d) {
  if (!x || !d) return FPSI_E_INVALID;
  for (int64_t i = 0; i < x->H.nc; ++i) d[x->H.perm[i]] = x->h_wdist[i];
  return FPSI_OK;
}

int fpsi_sa_residual(fpsi_ctx* x, double* src) {
  if (!x) return FPSI_E_INVALID;
  if (!fpsi::sa_active(x)) return FPSI_E_STATE;
  if (!x->have_resid) return FPSI_E_STATE;
  int rc = fpsi::sa_launch_residual(x);
  if (rc) return rc;
  if (src) {
    if ((rc = sa_down(x, x->d_sa_B, src))) return rc;
  } else if ((rc = sync(x))) {
    return rc;
  }
  x->have_sa = true;
  x->have_sa_dq = false;
  return FPSI_OK;
}

int fpsi_sa_get_system(fpsi_ctx* x, double* D, double* fjp, double* fjm) {
  if (!x) return FPSI_E_INVALID;
  if (!x->have_sa) return FPSI_E_STATE;
  int rc;
  if (D && (rc = sa_down(x, x->d_sa_D, D))) return rc;
  const int64_t nf = x->H.nf;
  for (int w = 0; w < 2; ++w) {
    double* dst = w ? fjm : fjp;
    if (!dst) continue;
    std::vector<double> h(nf);
    FPSI_CUDA_TRY(cudaMemcpy(h.data(), x->d_sa_face + (3 + w) * nf, nf * sizeof(double),
                             cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < nf; ++i) dst[x->H.fperm[i]] = h[i];
  }
  return FPSI_OK;
}

int fpsi_sa_solve(fpsi_ctx* x, double* dq) {
  if (!x) return FPSI_E_INVALID;
  if (!x->have_sa) return FPSI_E_STATE;
  int rc = fpsi::sa_launch_solve(x);
  if (rc) return rc;
  if (dq) {
    if ((rc = sa_down(x, x->d_sa_x, dq))) return rc;
  } else if ((rc = sync(x))) {
    return rc;
  }
  x->have_sa_dq = true;
  return FPSI_OK;
}

int fpsi_sa_update(fpsi_ctx* x) {
  if (!x) return FPSI_E_INVALID;
  if (!x->have_sa_dq) return FPSI_E_STATE;
  int rc = fpsi::sa_launch_update(x, x->d_resid);
  if (rc) return rc;
  if ((rc = sync(x))) return rc;
  x->have_sa = x->have_sa_dq = false;
  return FPSI_OK;
}

int fpsi_set_state(fpsi_ctx* x, const double* T, const double* pg, const double* u) {
  if (!x || !T || !pg || !u) return FPSI_E_INVALID;
  const int64_t nc = x->H.nc;
  const size_t b = size_t(nc) * sizeof(double);
  FPSI_CUDA_TRY(cudaMemcpyAsync(x->d_stage, T, b, cudaMemcpyHostToDevice, x->stream));
  FPSI_CUDA_TRY(cudaMemcpyAsync(x->d_stage + nc, pg, b, cudaMemcpyHostToDevice, x->stream));
  FPSI_CUDA_TRY(cudaMemcpyAsync(x->d_stage + 2 * nc, u, 3 * b, cudaMemcpyHostToDevice, x->stream));
  int rc = fpsi::launch_state(x, true);
  if (rc) return rc;
  x->have_resid = x->have_asm = x->have_dq = x->have_xprev = false;
  x->have_levels = false;
  return sync(x);
}

int fpsi_get_state(fpsi_ctx* x, double* T, double* pg, double* u) {
  if (!x || !T || !pg || !u) return FPSI_E_INVALID;
  const int64_t nc = x->H.nc;
  const size_t b = size_t(nc) * sizeof(double);
  int rc = fpsi::launch_state(x, false);
  if (rc) return rc;
  FPSI_CUDA_TRY(cudaMemcpyAsync(T, x->d_stage, b, cudaMemcpyDeviceToHost, x->stream));
  FPSI_CUDA_TRY(cudaMemcpyAsync(pg, x->d_stage + nc, b, cudaMemcpyDeviceToHost, x->stream));
  FPSI_CUDA_TRY(cudaMemcpyAsync(u, x->d_stage + 2 * nc, 3 * b, cudaMemcpyDeviceToHost, x->stream));
  return sync(x);
}

int fpsi_keep_blocks(fpsi_ctx* x, int32_t keep) {
  if (!x) return FPSI_E_INVALID;
  if (is_lsgs(x)) return keep ? FPSI_OK : FPSI_E_UNSUPPORTED;  // lines need fluid_D
  if (bool(keep) == x->keep_D) return FPSI_OK;
  x->keep_D = keep != 0;
  x->alloc_prec = -1;  // reallocate the system arrays
  return alloc_system(x);
}

int fpsi_residual(fpsi_ctx* x, double* src, fpsi_resid* norms) {
  if (!x) return FPSI_E_INVALID;
  int rc;
  x->have_sa = x->have_sa_dq = false;
  if (fpsi::sa_active(x) && (rc = fpsi::sa_launch_tmu(x))) return rc;
  rc = fpsi::launch_residual(x, x->d_resid);
  if (rc) return rc;
  FPSI_CUDA_TRY(cudaMemcpyAsync(x->h_resid, x->d_resid, fpsi::NREC * sizeof(double),
                                cudaMemcpyDeviceToHost, x->stream));
  std::vector<double> s;
  if (src) {
    s.resize(5 * x->H.nc);
    FPSI_CUDA_TRY(cudaMemcpyAsync(s.data(), x->d_src, s.size() * sizeof(double),
                                  cudaMemcpyDeviceToHost, x->stream));
  }
  if ((rc = sync(x))) return rc;
  if (src) unpermute_cells(x, s.data(), 5, src);
  if (norms) fill_norms(x, x->h_resid, norms);
  x->have_resid = true;
  x->have_asm = x->have_dq = x->x_preset = false;
  return has_nan(x->h_resid) ? FPSI_E_NAN : FPSI_OK;
}

int fpsi_get_reconstruction(fpsi_ctx* x, double* grad, double* limiter) {
  if (!x) return FPSI_E_INVALID;
  if (!x->have_resid) return FPSI_E_STATE;
  const int64_t nc = x->H.nc;
  // device records hold the gradient (15) and the limiter (5) of a cell;
  // an inviscid residual does not write them, so they are made on request
  if (!x->grad_valid) {
    int rc = fpsi::launch_grad_records(x);
    if (!rc) rc = sync(x);
    if (rc) return rc;
  }
  std::vector<double> rec(size_t(nc) * fpsi::GPREC), part;
  if (grad || limiter)
    FPSI_CUDA_TRY(cudaMemcpy(rec.data(), x->d_grad, rec.size() * sizeof(double), cudaMemcpyDeviceToHost));
  auto split = [&](int k0, int w, double* out) {
    part.resize(size_t(nc) * w);
    for (int64_t i = 0; i < nc; ++i)
      for (int k = 0; k < w; ++k) part[size_t(i) * w + k] = rec[size_t(i) * fpsi::GPREC + k0 + k];
    unpermute_cells(x, part.data(), w, out);
  };
  if (grad) split(0, 15, grad);
  if (limiter) split(15, 5, limiter);
  return FPSI_OK;
}

int fpsi_get_dtau(fpsi_ctx* x, double* dtau) {
  if (!x || !dtau) return FPSI_E_INVALID;
  if (!x->have_resid) return FPSI_E_STATE;
  std::vector<double> d(x->H.nc);
  FPSI_CUDA_TRY(cudaMemcpy(d.data(), x->d_dtau, d.size() * sizeof(double), cudaMemcpyDeviceToHost));
  unpermute_cells(x, d.data(), 1, dtau);
  return FPSI_OK;
}

static int finish_assemble(fpsi_ctx* x) {
  int32_t err = 0;
  FPSI_CUDA_TRY(cudaMemcpyAsync(&err, x->d_err, sizeof(int32_t), cudaMemcpyDeviceToHost, x->stream));
  int rc = sync(x);
  if (rc) return rc;
  if (err) {
    FPSI_CUDA_TRY(cudaMemset(x->d_err, 0, sizeof(int32_t)));
    if (err & 4) {
      fpsi::set_error("a line solve gave up waiting for its staged rows");
      return FPSI_E_TIMEOUT;
    }
    fpsi::set_error("zero pivot in a diagonal block LU");
    return FPSI_E_SINGULAR;
  }
  return FPSI_OK;
}

int fpsi_assemble(fpsi_ctx* x) {
  if (!x) return FPSI_E_INVALID;
  if (!x->have_resid) return FPSI_E_STATE;
  int rc = fpsi::launch_assemble(x);
  if (rc) return rc;
  if (is_lsgs(x) && (rc = fpsi::lsgs_assemble(x))) return rc;
  if ((rc = finish_assemble(x))) return rc;
  x->have_asm = true;
  x->have_dq = false;
  return FPSI_OK;
}

int fpsi_get_blocks(fpsi_ctx* x, void* D, void* fjp, void* fjm, void* B) {
  if (!x) return FPSI_E_INVALID;
  if (!x->have_asm) return FPSI_E_STATE;
  const int tb = x->blk_bytes;
  const int64_t nc = x->H.nc, nf = x->H.nf;
  std::vector<char> h;
  if (D) {
    if (!x->d_D) return FPSI_E_STATE;
    h.resize(size_t(nc) * 25 * tb);
    FPSI_CUDA_TRY(cudaMemcpy(h.data(), x->d_D, h.size(), cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < nc; ++i)
      std::memcpy((char*)D + size_t(x->H.perm[i]) * 25 * tb, h.data() + size_t(i) * 25 * tb, 25 * tb);
  }
  if ((fjp || fjm) && !x->have_explicit) {
    const int rc = fpsi::ensure_explicit_blocks(x);
    if (rc) return rc;
  }
  std::vector<char> hb;  // difference blocks of the total-pressure and fixed-mass inflows
  if (fjp && x->any_fdbc) {
    hb.resize(size_t(std::max<int64_t>(x->H.nbf, 1)) * 25 * tb);
    FPSI_CUDA_TRY(cudaMemcpy(hb.data(), x->d_bjac, hb.size(), cudaMemcpyDeviceToHost));
  }
  for (int w = 0; w < 2; ++w) {
    void* dst = w ? fjm : fjp;
    if (!dst) continue;
    h.resize(size_t(nf) * 25 * tb);
    FPSI_CUDA_TRY(cudaMemcpy(h.data(), w ? x->d_fjm : x->d_fjp, h.size(), cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < nf; ++i) {
      char* o = (char*)dst + size_t(x->H.fperm[i]) * 25 * tb;
      if (w && i >= x->H.nfi) {
        std::memset(o, 0, 25 * tb);  // no fjm on boundary faces
      } else if (!w && i >= x->H.nfi && !hb.empty()) {
        const int kind = x->bcs[-x->H.cr[i] - 1].kind;
        const bool fd = kind == FPSI_BC_ISENTROPIC_INFLOW || kind == FPSI_BC_FIXED_MASS_INFLOW;
        const char* a = h.data() + size_t(i) * 25 * tb;
        const char* b = hb.data() + size_t(i - x->H.nfi) * 25 * tb;
        std::memcpy(o, a, 25 * tb);
        // the block srcJ loses is the face's (viscous part, if any) plus the difference block
        for (int k = 0; fd && k < 25; ++k) {
          if (tb == 4)
            reinterpret_cast<float*>(o)[k] += reinterpret_cast<const float*>(b)[k];
          else
            reinterpret_cast<double*>(o)[k] += reinterpret_cast<const double*>(b)[k];
        }
      } else {
        std::memcpy(o, h.data() + size_t(i) * 25 * tb, 25 * tb);
      }
    }
  }
  if (B) {
    h.resize(size_t(x->H.ncp) * 5 * tb);
    FPSI_CUDA_TRY(cudaMemcpy(h.data(), x->d_bc, h.size(), cudaMemcpyDeviceToHost));
    const HostMesh& H = x->H;
    for (int k = 0; k < H.ncolours; ++k)
      for (int64_t i = 0; i < H.col_n[k]; ++i) {
        const int64_t c = H.colour_cells[H.col_cb[k] + i];
        char* o = (char*)B + size_t(H.perm[c]) * 5 * tb;
        for (int j = 0; j < 5; ++j)
          std::memcpy(o + j * tb, h.data() + (size_t(5 * H.col_cbp[k]) + j * H.col_ld[k] + i) * tb,
                      tb);
      }
  }
  return FPSI_OK;
}

static int upload_x(fpsi_ctx* x, const double* x0) {
  const int64_t nc = x->H.nc;
  if (is_lsgs(x)) {
    const size_t nt = size_t(x->LY.nrows) * 32;
    std::vector<double> v(5 * nt, 0.0);
    for (int64_t i = 0; i < nc; ++i)
      for (int k = 0; k < 5; ++k)
        v[5 * int64_t(x->LY.t_of[i]) + k] = x0[5 * int64_t(x->H.perm[i]) + k];
    if (x->x_bytes == 8 && x->P.precision != FPSI_PREC_MIXED) {
      FPSI_CUDA_TRY(cudaMemcpy(x->d_lx, v.data(), v.size() * 8, cudaMemcpyHostToDevice));
    } else {
      std::vector<float> f(v.begin(), v.end());
      FPSI_CUDA_TRY(cudaMemcpy(x->d_lx, f.data(), f.size() * 4, cudaMemcpyHostToDevice));
    }
    return FPSI_OK;
  }
  if (x->x_bytes == 8) {
    std::vector<double> v(5 * nc);
    for (int64_t i = 0; i < nc; ++i)
      for (int k = 0; k < 5; ++k)
        v[5 * int64_t(x->H.ci_of[i]) + k] = x0[5 * int64_t(x->H.perm[i]) + k];
    FPSI_CUDA_TRY(cudaMemcpy(x->d_x, v.data(), v.size() * 8, cudaMemcpyHostToDevice));
  } else {
    std::vector<float> v(5 * nc);
    for (int64_t i = 0; i < nc; ++i)
      for (int k = 0; k < 5; ++k)
        v[5 * int64_t(x->H.ci_of[i]) + k] = float(x0[5 * int64_t(x->H.perm[i]) + k]);
    FPSI_CUDA_TRY(cudaMemcpy(x->d_x, v.data(), v.size() * 4, cudaMemcpyHostToDevice));
  }
  return FPSI_OK;
}

static int download_x(fpsi_ctx* x, double* dq) {
  const int64_t nc = x->H.nc;
  if (is_lsgs(x)) {
    const size_t nt = size_t(x->LY.nrows) * 32;
    std::vector<double> v(5 * nt);
    if (x->P.precision != FPSI_PREC_MIXED) {
      FPSI_CUDA_TRY(cudaMemcpy(v.data(), x->d_lx, v.size() * 8, cudaMemcpyDeviceToHost));
    } else {
      std::vector<float> f(5 * nt);
      FPSI_CUDA_TRY(cudaMemcpy(f.data(), x->d_lx, f.size() * 4, cudaMemcpyDeviceToHost));
      for (size_t i = 0; i < f.size(); ++i) v[i] = f[i];
    }
    for (int64_t i = 0; i < nc; ++i)
      for (int k = 0; k < 5; ++k)
        dq[5 * int64_t(x->H.perm[i]) + k] = v[5 * int64_t(x->LY.t_of[i]) + k];
    return FPSI_OK;
  }
  std::vector<double> v(5 * nc);
  if (x->x_bytes == 8) {
    FPSI_CUDA_TRY(cudaMemcpy(v.data(), x->d_x, v.size() * 8, cudaMemcpyDeviceToHost));
  } else {
    std::vector<float> f(5 * nc);
    FPSI_CUDA_TRY(cudaMemcpy(f.data(), x->d_x, f.size() * 4, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < f.size(); ++i) v[i] = f[i];
  }
  for (int64_t i = 0; i < nc; ++i)
    for (int k = 0; k < 5; ++k)
      dq[5 * int64_t(x->H.perm[i]) + k] = v[5 * int64_t(x->H.ci_of[i]) + k];
  return FPSI_OK;
}

int fpsi_linear_solve(fpsi_ctx* x, const double* x0, double* dq, fpsi_lsinfo* info) {
  if (!x) return FPSI_E_INVALID;
  if (!x->have_asm) return FPSI_E_STATE;
  int rc;
  if (is_lsgs(x)) {
    if (x0 && (rc = upload_x(x, x0))) return rc;
    if ((rc = fpsi::lsgs_solve(x, x0 == nullptr))) return rc;
    struct {
      double w, zero, resid;
      int32_t iter, done;
    } ctl;
    FPSI_CUDA_TRY(cudaMemcpyAsync(&ctl, x->d_lctl, sizeof(ctl), cudaMemcpyDeviceToHost, x->stream));
    if ((rc = finish_assemble(x))) return rc;
    x->have_dq = true;
    if (dq && (rc = download_x(x, dq))) return rc;
    if (info) {
      info->iterations = ctl.iter;
      info->status = FPSI_OK;
      info->resid0 = ctl.zero;
      info->resid = ctl.resid;
    }
    return FPSI_OK;
  }
  if (x0) {
    if ((rc = upload_x(x, x0))) return rc;
  } else if (x->have_dq && !x->x_preset) {
    // iterate was consumed by an earlier solve: rebuild the reference start
    if (x->P.solver == FPSI_SOLVER_FSGS) {
      FPSI_CUDA_TRY(cudaMemsetAsync(x->d_x, 0, size_t(x->H.nc) * 5 * x->x_bytes, x->stream));
    } else if ((rc = fpsi::launch_jacobi_start(x))) {
      return rc;
    }
  }
  x->x_preset = false;
  if ((rc = fpsi::launch_sgs(x, x->P.gauss_seidel_iter))) return rc;
  if ((rc = sync(x))) return rc;
  x->have_dq = true;
  if (dq && (rc = download_x(x, dq))) return rc;
  if (info) {
    info->iterations = x->P.gauss_seidel_iter;
    info->status = FPSI_OK;
    info->resid0 = info->resid = 0;
  }
  return FPSI_OK;
}

int fpsi_set_iterate(fpsi_ctx* x, const double* x0) {
  if (!x || !x0) return FPSI_E_INVALID;
  if (!x->have_asm) return FPSI_E_STATE;
  int rc = upload_x(x, x0);
  if (rc) return rc;
  x->x_preset = true;
  return FPSI_OK;
}

int fpsi_get_iterate(fpsi_ctx* x, double* dq) {
  if (!x || !dq) return FPSI_E_INVALID;
  if (!x->have_asm) return FPSI_E_STATE;
  return download_x(x, dq);
}

int fpsi_linear_sweeps(fpsi_ctx* x, int32_t nsweeps) {
  if (!x || nsweeps < 0) return FPSI_E_INVALID;
  if (!x->have_asm) return FPSI_E_STATE;
  if (is_lsgs(x)) return FPSI_E_UNSUPPORTED;
  int rc = fpsi::launch_sgs(x, nsweeps);
  if (rc) return rc;
  if ((rc = sync(x))) return rc;
  x->have_dq = true;
  x->x_preset = false;
  return FPSI_OK;
}

int fpsi_linear_residual(fpsi_ctx* x, double* norm_b, double* norm_r) {
  if (!x) return FPSI_E_INVALID;
  if (!x->have_asm || !x->d_D) return FPSI_E_STATE;
  int rc = fpsi::launch_linres(x, x->d_resid + 16);
  if (rc) return rc;
  FPSI_CUDA_TRY(cudaMemcpyAsync(x->h_resid + 16, x->d_resid + 16, 2 * sizeof(double),
                                cudaMemcpyDeviceToHost, x->stream));
  if ((rc = sync(x))) return rc;
  if (norm_b) *norm_b = x->h_resid[16];
  if (norm_r) *norm_r = x->h_resid[17];
  return FPSI_OK;
}

int fpsi_update(fpsi_ctx* x, double* min_alpha) {
  if (!x) return FPSI_E_INVALID;
  if (!x->have_dq) return FPSI_E_STATE;
  int rc = fpsi::launch_update(x, x->d_resid);
  if (rc) return rc;
  std::vector<double> a(x->nblk_norm);
  FPSI_CUDA_TRY(cudaMemcpyAsync(a.data(), x->d_amin, a.size() * sizeof(double),
                                cudaMemcpyDeviceToHost, x->stream));
  if ((rc = sync(x))) return rc;
  if (min_alpha) *min_alpha = *std::min_element(a.begin(), a.end());
  x->have_resid = x->have_asm = x->have_dq = false;
  return FPSI_OK;
}

int fpsi_newton_step(fpsi_ctx* x, fpsi_stepinfo* info) {
  if (!x) return FPSI_E_INVALID;
  int rc;
  const bool sa = fpsi::sa_active(x);
  if (sa && (rc = fpsi::sa_launch_tmu(x))) return rc;
  if ((rc = fpsi::launch_residual(x, x->d_resid))) return rc;
  if (sa && ((rc = fpsi::sa_launch_residual(x)) || (rc = fpsi::sa_launch_solve(x)))) return rc;
  if ((rc = fpsi::launch_assemble(x))) return rc;
  if (is_lsgs(x)) {
    if ((rc = fpsi::lsgs_assemble(x))) return rc;
    if ((rc = fpsi::lsgs_solve(x, true))) return rc;
  } else if ((rc = fpsi::launch_sgs(x, x->P.gauss_seidel_iter))) {
    return rc;
  }
  if ((rc = fpsi::launch_update(x, x->d_resid))) return rc;
  if (sa && (rc = fpsi::sa_launch_update(x, x->d_resid))) return rc;
  FPSI_CUDA_TRY(cudaMemcpyAsync(x->h_resid, x->d_resid, fpsi::NREC * sizeof(double),
                                cudaMemcpyDeviceToHost, x->stream));
  std::vector<double> a(x->nblk_norm);
  FPSI_CUDA_TRY(cudaMemcpyAsync(a.data(), x->d_amin, a.size() * sizeof(double),
                                cudaMemcpyDeviceToHost, x->stream));
  if ((rc = sync(x))) return rc;
  x->have_resid = x->have_asm = x->have_dq = false;
  if (info) {
    std::memset(info, 0, sizeof(*info));
    fill_norms(x, x->h_resid, &info->resid);
    info->ls.iterations = x->P.gauss_seidel_iter;
    info->min_alpha = *std::min_element(a.begin(), a.end());
  }
  if (has_nan(x->h_resid)) {
    // the state was left unchanged; a system built from NaN norms may have
    // flagged zero pivots too
    FPSI_CUDA_TRY(cudaMemset(x->d_err, 0, sizeof(int32_t)));
    fpsi::set_error("NaN residual norms; the state is unchanged");
    return FPSI_E_NAN;
  }
  return finish_assemble(x);
}

// ---- one step with a chosen start, a linear tolerance and rejection -----
namespace {
// sweeps of the assembled system: exactly gauss_seidel_iter, or until the
// linear residual falls below lin_rtol ||B|| (checked every check_every
// sweeps); info gets the count and the residuals measured
int ex_sweeps(fpsi_ctx* x, const fpsi_step_opts& o, fpsi_lsinfo* info) {
  int rc;
  info->status = FPSI_OK;
  info->resid0 = info->resid = 0;
  if (o.lin_rtol <= 0) {
    if ((rc = fpsi::launch_sgs(x, x->P.gauss_seidel_iter))) return rc;
    info->iterations = x->P.gauss_seidel_iter;
    return FPSI_OK;
  }
  const int every = std::max(1, o.check_every);
  int done = 0;
  for (bool first = true;; first = false) {
    if ((rc = fpsi::launch_linres(x, x->d_resid + 16))) return rc;
    FPSI_CUDA_TRY(cudaMemcpyAsync(x->h_resid + 16, x->d_resid + 16, 2 * sizeof(double),
                                  cudaMemcpyDeviceToHost, x->stream));
    if ((rc = sync(x))) return rc;
    const double nb = x->h_resid[16], nr = x->h_resid[17];
    if (first) info->resid0 = nr;
    info->resid = nr;
    if (!(nr > o.lin_rtol * nb) || done >= o.max_sweeps) break;
    const int k = std::min(every, o.max_sweeps - done);
    if ((rc = fpsi::launch_sgs(x, k))) return rc;
    done += k;
  }
  info->iterations = done;
  return FPSI_OK;
}

// residual of the current state into d_resid and h_resid
int ex_residual(fpsi_ctx* x) {
  int rc = fpsi::launch_residual(x, x->d_resid);
  if (rc) return rc;
  FPSI_CUDA_TRY(cudaMemcpyAsync(x->h_resid, x->d_resid, fpsi::NREC * sizeof(double),
                                cudaMemcpyDeviceToHost, x->stream));
  if ((rc = sync(x))) return rc;
  x->have_resid = true;
  x->have_asm = x->have_dq = x->x_preset = false;
  return FPSI_OK;
}

// assemble, start, relax and update from the residual in d_resid, queued
// with no host synchronisation (unless the sweeps run to a tolerance).  The
// update leaves the state alone when the assembly (a zero pivot) or the
// learned start (a wait that gave up) raised an error bit; the bits and the
// update's step fractions are copied to pinned memory behind the kernels
// and checked by ex_finish after the next residual's synchronisation.
int ex_attempt(fpsi_ctx* x, fpsi_gnn* model, const fpsi_step_opts& o, int start,
               fpsi_stepinfo* info) {
  x->h_flags[0] = x->h_flags[1] = 0;
  int rc = fpsi::launch_assemble(x);
  if (rc) return rc;
  x->have_asm = true;
  int32_t* merr = nullptr;
  if (start == FPSI_START_ZERO) {
    FPSI_CUDA_TRY(cudaMemsetAsync(x->d_x, 0, size_t(x->H.nc) * 5 * x->x_bytes, x->stream));
  } else if (start == FPSI_START_LEARNED) {
    if ((rc = fpsi::gnn_predict_launch(model, x, nullptr, x->P.solver == FPSI_SOLVER_SGS))) return rc;
    merr = fpsi::gnn_error_bits(model);
  }
  if ((rc = ex_sweeps(x, o, &info->ls))) return rc;
  if ((rc = fpsi::launch_update(x, x->d_resid, x->d_err, merr))) return rc;
  FPSI_CUDA_TRY(cudaMemcpyAsync(x->h_flags, x->d_err, sizeof(int32_t), cudaMemcpyDeviceToHost, x->stream));
  FPSI_CUDA_TRY(cudaMemsetAsync(x->d_err, 0, sizeof(int32_t), x->stream));
  if (merr) {
    FPSI_CUDA_TRY(cudaMemcpyAsync(x->h_flags + 1, merr, sizeof(int32_t), cudaMemcpyDeviceToHost, x->stream));
    FPSI_CUDA_TRY(cudaMemsetAsync(merr, 0, sizeof(int32_t), x->stream));
  }
  FPSI_CUDA_TRY(cudaMemcpyAsync(x->h_amin, x->d_amin, size_t(x->nblk_norm) * sizeof(double),
                                cudaMemcpyDeviceToHost, x->stream));
  x->have_resid = x->have_asm = x->have_dq = x->x_preset = false;
  return FPSI_OK;
}

// after ex_attempt and the synchronisation of the residual that follows it
int ex_finish(fpsi_ctx* x, fpsi_stepinfo* info) {
  const int32_t ea = x->h_flags[0], em = x->h_flags[1];
  if (ea & 4) {
    fpsi::set_error("a line solve gave up waiting for its staged rows");
    return FPSI_E_TIMEOUT;
  }
  if (ea) {
    fpsi::set_error("zero pivot in a diagonal block LU");
    return FPSI_E_SINGULAR;
  }
  if (em) {
    fpsi::set_error("learned start: a tensor-core wait timed out");
    return FPSI_E_TIMEOUT;
  }
  info->min_alpha = *std::min_element(x->h_amin, x->h_amin + x->nblk_norm);
  return FPSI_OK;
}
}  // namespace

int fpsi_newton_step_ex(fpsi_ctx* x, fpsi_gnn* model, const fpsi_step_opts* opts,
                        fpsi_stepinfo* info) {
  if (!x || !opts) return FPSI_E_INVALID;
  const fpsi_step_opts o = *opts;
  if (o.start < FPSI_START_JACOBI || o.start > FPSI_START_LEARNED ||
      (o.start == FPSI_START_LEARNED && !model) || (o.lin_rtol > 0 && o.max_sweeps < 0)) {
    fpsi::set_error("fpsi_newton_step_ex: bad options");
    return FPSI_E_INVALID;
  }
  if (is_lsgs(x) || fpsi::sa_active(x)) {
    fpsi::set_error("fpsi_newton_step_ex: multi-colour SGS without the SA model only");
    return FPSI_E_UNSUPPORTED;
  }
  if ((o.start == FPSI_START_LEARNED || o.lin_rtol > 0) && !x->d_D) {
    fpsi::set_error("fpsi_newton_step_ex: keep the diagonal blocks (fpsi_keep_blocks)");
    return FPSI_E_STATE;
  }
  const int64_t nc = x->H.nc;
  const size_t qb = size_t(nc) * 5 * sizeof(double);
  const bool may_reject = o.reject && o.start != FPSI_START_JACOBI;
  int rc;
  if (may_reject && !x->d_qsave && (rc = dalloc(x, &x->d_qsave, size_t(nc) * 5))) return rc;
  fpsi_stepinfo si;
  std::memset(&si, 0, sizeof(si));
  // the residual of the current state: kept from the previous call, or new
  if (!x->have_resid && (rc = ex_residual(x))) return rc;
  double r_start[fpsi::NREC];
  std::memcpy(r_start, x->h_resid, sizeof(r_start));
  fill_norms(x, r_start, &si.resid);
  if (has_nan(r_start)) {
    fpsi::set_error("NaN residual norms; the state is unchanged");
    return FPSI_E_NAN;
  }
  if (may_reject)
    FPSI_CUDA_TRY(cudaMemcpyAsync(x->d_qsave, x->d_q, qb, cudaMemcpyDeviceToDevice, x->stream));
  si.start_used = o.start;
  if ((rc = ex_attempt(x, model, o, o.start, &si))) return rc;
  if ((rc = ex_residual(x))) return rc;
  if ((rc = ex_finish(x, &si))) return rc;
  if (may_reject && !(x->h_resid[0] < r_start[0])) {
    // the step did not lower the FP64 density residual: undo it and take
    // the reference's step from D^-1 B
    FPSI_CUDA_TRY(cudaMemcpyAsync(x->d_q, x->d_qsave, qb, cudaMemcpyDeviceToDevice, x->stream));
    if ((rc = ex_residual(x))) return rc;
    si.rejected = 1;
    si.start_used = FPSI_START_JACOBI;
    if ((rc = ex_attempt(x, model, o, FPSI_START_JACOBI, &si))) return rc;
    if ((rc = ex_residual(x))) return rc;
    if ((rc = ex_finish(x, &si))) return rc;
  }
  fill_norms(x, x->h_resid, &si.resid_after);
  if (info) *info = si;
  if (has_nan(x->h_resid)) {
    fpsi::set_error("NaN residual norms after the step");
    return FPSI_E_NAN;
  }
  return FPSI_OK;
}

// One implicit step's launches on the stream, its norms into slot (device)
// and, when hdst is given, by a copy queued behind the residual into hdst
// (pinned host).
static int launch_step(fpsi_ctx* x, double* slot, double* hdst, bool sa) {
  int rc = FPSI_OK;
  if (sa) rc = fpsi::sa_launch_tmu(x);
  if (!rc) rc = fpsi::launch_residual(x, slot);
  if (!rc && hdst &&
      cudaMemcpyAsync(hdst, slot, fpsi::NREC * sizeof(double), cudaMemcpyDeviceToHost, x->stream) !=
          cudaSuccess)
    rc = FPSI_E_CUDA;
  if (!rc && sa) rc = fpsi::sa_launch_residual(x);
  if (!rc && sa) rc = fpsi::sa_launch_solve(x);
  if (!rc) rc = fpsi::launch_assemble(x);
  if (!rc && is_lsgs(x)) {
    rc = fpsi::lsgs_assemble(x);
    if (!rc) rc = fpsi::lsgs_solve(x, true);
  } else if (!rc) {
    rc = fpsi::launch_sgs(x, x->P.gauss_seidel_iter);
  }
  if (!rc) rc = fpsi::launch_update(x, slot);
  if (!rc && sa) rc = fpsi::sa_launch_update(x, slot);
  return rc;
}

// The launches of one step captured as a CUDA graph, with its norms going to
// the fixed slot; null when the capture or the instantiation fails (the
// caller then launches the step itself).  Nothing of a captured step runs
// until the graph is launched.
static cudaGraphExec_t capture_step(fpsi_ctx* x, double* fixed) {
  if (cudaStreamBeginCapture(x->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  const int rc = launch_step(x, fixed, nullptr, fpsi::sa_active(x));
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(x->stream, &g);
  cudaGraphExec_t ge = nullptr;
  if (rc == FPSI_OK && e == cudaSuccess && g &&
      cudaGraphInstantiate(&ge, g, 0) != cudaSuccess)
    ge = nullptr;
  if (g) cudaGraphDestroy(g);
  cudaGetLastError();
  return ge;
}

// nsteps implicit steps on the stream; with the SA model nu~ is advanced in
// each step from the same residual state, after the mean flow's solve.  The
// norms of step s go to d_hist[NREC s] and, by a copy queued behind the
// residual, to the pinned h_hist[NREC s] (whose rtrms slot starts at -1).
// Before each launch the host looks at the copies that have landed and stops
// launching once one holds NaN norms; steps already queued behind it leave
// the state alone (the update kernels test their step's norms), so the state
// is the one of the first NaN step.  With step_graphs step 0 runs as
// launches, which makes every buffer the step uses, and steps
// 1.. replay one captured graph whose norms land in d_hist[NREC nsteps]
// (the history holds nsteps + 1 records) and are copied from there into
// the step's slots behind the graph.
// Returns the number of steps launched.
static int run_steps(fpsi_ctx* x, int32_t nsteps, int32_t* launched) {
  int rc = FPSI_OK;
  const bool sa = fpsi::sa_active(x);
  const bool graphs = x->P.step_graphs && !x->profiling && nsteps > 2;
  double* fixed = x->d_hist + fpsi::NREC * int64_t(nsteps);
  cudaGraphExec_t ge = nullptr;
  volatile double* hh = x->h_hist;
  for (int32_t s = 0; s < nsteps; ++s) hh[fpsi::NREC * int64_t(s)] = -1.0;
  int32_t seen = 0, s = 0;
  for (; s < nsteps && !rc; ++s) {
    bool nan = false;
    while (seen < s && !nan) {
      const double r = hh[fpsi::NREC * int64_t(seen)];
      if (r == -1.0) break;  // not landed yet
      const int64_t o = fpsi::NREC * int64_t(seen);
      nan = r != r || hh[o + 1] != hh[o + 1] || hh[o + 2] != hh[o + 2];
      ++seen;
    }
    if (nan) break;
    double* slot = x->d_hist + fpsi::NREC * int64_t(s);
    double* hdst = x->h_hist + fpsi::NREC * int64_t(s);
    if (graphs && s == 1) ge = capture_step(x, fixed);
    if (ge) {
      if (cudaGraphLaunch(ge, x->stream) != cudaSuccess ||
          cudaMemcpyAsync(slot, fixed, fpsi::NREC * sizeof(double), cudaMemcpyDeviceToDevice,
                          x->stream) != cudaSuccess ||
          cudaMemcpyAsync(hdst, fixed, fpsi::NREC * sizeof(double), cudaMemcpyDeviceToHost,
                          x->stream) != cudaSuccess)
        rc = FPSI_E_CUDA;
    } else {
      rc = launch_step(x, slot, hdst, sa);
    }
  }
  if (ge) cudaGraphExecDestroy(ge);
  *launched = s;
  x->have_sa = x->have_sa_dq = false;
  return rc;
}

// norms of a finished run; a NaN step ends the history (later entries NaN)
static int finish_run(fpsi_ctx* x, int32_t nsteps, int32_t launched, fpsi_resid* norms) {
  int32_t first_nan = -1;
  for (int32_t s = 0; s < launched && first_nan < 0; ++s)
    if (has_nan(&x->h_hist[fpsi::NREC * int64_t(s)])) first_nan = s;
  if (launched < nsteps && first_nan < 0) {
    fpsi::set_error("the run stopped after %d of %d steps without a NaN residual", launched, nsteps);
    return FPSI_E_STATE;
  }
  const int32_t last = first_nan < 0 ? nsteps : first_nan + 1;
  if (norms) {
    for (int32_t s = 0; s < last; ++s) fill_norms(x, &x->h_hist[fpsi::NREC * int64_t(s)], &norms[s]);
    const double q = std::nan("");
    const double nanrec[fpsi::NREC] = {q, q, q, q, -1, q, -1, q, 0, 0};
    for (int32_t s = last; s < nsteps; ++s) fill_norms(x, nanrec, &norms[s]);
  }
  if (first_nan >= 0) {
    // the systems built from NaN norms may have flagged zero pivots too
    FPSI_CUDA_TRY(cudaMemset(x->d_err, 0, sizeof(int32_t)));
    fpsi::set_error("NaN residual norms at step %d of %d; the state is that step's", first_nan,
                    nsteps);
    return FPSI_E_NAN;
  }
  return finish_assemble(x);
}

int fpsi_run(fpsi_ctx* x, int32_t nsteps, fpsi_resid* norms) {
  if (!x || nsteps < 0) return FPSI_E_INVALID;
  if (nsteps == 0) return FPSI_OK;
  int rc = ensure_hist(x, nsteps + 1);
  if (rc) return rc;
  int32_t launched = 0;
  rc = run_steps(x, nsteps, &launched);
  if (!rc) rc = sync(x);
  x->have_resid = x->have_asm = x->have_dq = false;
  if (rc) return rc;
  return finish_run(x, nsteps, launched, norms);
}

int fpsi_time_step(fpsi_ctx* x, fpsi_resid* norms) {
  if (!x) return FPSI_E_INVALID;
  if (!x->P.time_accurate) {
    fpsi::set_error("fpsi_time_step needs params.time_accurate = 1");
    return FPSI_E_STATE;
  }
  const int32_t nit = x->P.newton_iters;
  int rc = ensure_hist(x, nit + 1);
  if (rc) return rc;
  int32_t launched = 0;
  rc = run_steps(x, nit, &launched);
  if (!rc) rc = sync(x);
  x->have_resid = x->have_asm = x->have_dq = false;
  if (rc) return rc;
  if ((rc = finish_run(x, nit, launched, norms))) return rc;
  // the converged state becomes time level n+1: Q(n-1) = Q(n), Q(n) = Q(n+1)
  const size_t b = size_t(x->H.nc) * 5 * sizeof(double);
  std::swap(x->d_qn, x->d_qnm1);
  FPSI_CUDA_TRY(cudaMemcpyAsync(x->d_qn, x->d_q, b, cudaMemcpyDeviceToDevice, x->stream));
  return sync(x);
}

int fpsi_run_timed(fpsi_ctx* x, int32_t nsteps, fpsi_resid* norms, double* device_ms) {
  if (!x || nsteps <= 0 || !device_ms) return FPSI_E_INVALID;
  int rc = ensure_hist(x, nsteps + 1);
  if (rc) return rc;
  cudaEvent_t a = nullptr, b = nullptr;
  if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) rc = FPSI_E_CUDA;
  if (!rc && cudaEventRecord(a, x->stream) != cudaSuccess) rc = FPSI_E_CUDA;
  int32_t launched = 0;
  if (!rc) rc = run_steps(x, nsteps, &launched);
  if (!rc && cudaEventRecord(b, x->stream) != cudaSuccess) rc = FPSI_E_CUDA;
  if (!rc) rc = sync(x);
  float ms = 0;
  if (!rc && cudaEventElapsedTime(&ms, a, b) != cudaSuccess) rc = FPSI_E_CUDA;
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  x->have_resid = x->have_asm = x->have_dq = false;
  if (rc) return rc;
  *device_ms = ms;
  return finish_run(x, nsteps, launched, norms);
}

int fpsi_kernel_times(fpsi_ctx* x, int32_t nsteps, int32_t cap, char* names, double* ms,
                      int64_t* launches, int32_t* count) {
  if (!x || nsteps <= 0 || cap < 0 || !count) return FPSI_E_INVALID;
  int rc = ensure_hist(x, nsteps + 1);
  if (rc) return rc;
  x->prof.clear();
  x->evnext = 0;
  x->profiling = true;
  int32_t launched = 0;
  rc = run_steps(x, nsteps, &launched);
  x->profiling = false;
  if (!rc) rc = sync(x);
  x->have_resid = x->have_asm = x->have_dq = false;
  if (rc) return rc;
  if ((rc = finish_run(x, nsteps, launched, nullptr))) return rc;
  std::vector<std::string> keys;
  std::vector<double> tot;
  std::vector<int64_t> cnt;
  for (const fpsi_prof_rec& r : x->prof) {
    float t = 0;
    FPSI_CUDA_TRY(cudaEventElapsedTime(&t, r.a, r.b));
    size_t k = 0;
    while (k < keys.size() && keys[k] != r.name) ++k;
    if (k == keys.size()) {
      keys.push_back(r.name);
      tot.push_back(0);
      cnt.push_back(0);
    }
    tot[k] += t;
    cnt[k] += 1;
  }
  x->prof.clear();
  *count = int32_t(keys.size());
  for (size_t k = 0; k < keys.size() && int32_t(k) < cap; ++k) {
    if (names) {
      std::memset(names + 32 * k, 0, 32);
      std::strncpy(names + 32 * k, keys[k].c_str(), 31);
    }
    if (ms) ms[k] = tot[k];
    if (launches) launches[k] = cnt[k];
  }
  return FPSI_OK;
}

// ---- batched face functions ----------------------------------------------
static int batch_common(int64_t n, const double* qL, const double* qR, const double* an,
                        const double* area, double** dL, double** dR, double** dA,
                        double** dS) {
  if (n <= 0 || !qL || !qR || !an || !area) return FPSI_E_INVALID;
  if (!fpsi_device_available()) {
    fpsi::set_error("no CUDA device");
    return FPSI_E_CUDA;
  }
  FPSI_CUDA_TRY(cudaMalloc((void**)dL, n * 5 * sizeof(double)));
  FPSI_CUDA_TRY(cudaMalloc((void**)dR, n * 5 * sizeof(double)));
  FPSI_CUDA_TRY(cudaMalloc((void**)dA, n * 3 * sizeof(double)));
  FPSI_CUDA_TRY(cudaMalloc((void**)dS, n * sizeof(double)));
  FPSI_CUDA_TRY(cudaMemcpy(*dL, qL, n * 5 * sizeof(double), cudaMemcpyHostToDevice));
  FPSI_CUDA_TRY(cudaMemcpy(*dR, qR, n * 5 * sizeof(double), cudaMemcpyHostToDevice));
  FPSI_CUDA_TRY(cudaMemcpy(*dA, an, n * 3 * sizeof(double), cudaMemcpyHostToDevice));
  FPSI_CUDA_TRY(cudaMemcpy(*dS, area, n * sizeof(double), cudaMemcpyHostToDevice));
  return FPSI_OK;
}

int fpsi_face_flux(int32_t kind, int64_t n, const double* qL, const double* qR,
                   const double* an, const double* area, double pambient, double Rt,
                   double gamma, double us_n, double eta, double* flux) {
  if (kind < 0 || kind > 2 || !flux) return FPSI_E_INVALID;
  double *dL = nullptr, *dR = nullptr, *dA = nullptr, *dS = nullptr, *dF = nullptr;
  int rc = batch_common(n, qL, qR, an, area, &dL, &dR, &dA, &dS);
  if (!rc && cudaMalloc((void**)&dF, n * 5 * sizeof(double)) != cudaSuccess) rc = FPSI_E_NOMEM;
  if (!rc) rc = fpsi::launch_batch_flux(kind, n, dL, dR, dA, dS, pambient, Rt, gamma, us_n, eta, dF, 0);
  if (!rc && cudaMemcpy(flux, dF, n * 5 * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = FPSI_E_CUDA;
  cudaFree(dL), cudaFree(dR), cudaFree(dA), cudaFree(dS), cudaFree(dF);
  return rc;
}

int fpsi_face_jacobian(int64_t n, const double* qL, const double* qR, const double* an,
                       const double* area, double pambient, double Rt, double gamma,
                       double us_n, double eta, int32_t dir, int32_t as_double, void* out) {
  if (!out || (dir != 1 && dir != -1)) return FPSI_E_INVALID;
  double *dL = nullptr, *dR = nullptr, *dA = nullptr, *dS = nullptr;
  void* dO = nullptr;
  const size_t ob = size_t(n) * 25 * (as_double ? 8 : 4);
  int rc = batch_common(n, qL, qR, an, area, &dL, &dR, &dA, &dS);
  if (!rc && cudaMalloc(&dO, ob) != cudaSuccess) rc = FPSI_E_NOMEM;
  if (!rc)
    rc = fpsi::launch_batch_jac(n, dL, dR, dA, dS, pambient, Rt, gamma, us_n, eta, dir, as_double,
                                dO, 0);
  if (!rc && cudaMemcpy(out, dO, ob, cudaMemcpyDeviceToHost) != cudaSuccess) rc = FPSI_E_CUDA;
  cudaFree(dL), cudaFree(dR), cudaFree(dA), cudaFree(dS), cudaFree(dO);
  return rc;
}

}  // extern "C"
