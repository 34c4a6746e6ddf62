/*
 * fpsi.h -- C ABI of the B200-native implicit residual-and-relaxation path.
 *
 * The library replaces, on one GPU, the chain of Loci rules that flowPsi runs
 * once per Newton iteration of a steady implicit step:
 *
 *   residual      src = -sum(iflux)                 fluxInviscid.loci:1170-1188,1253-1268
 *   time step     cflpdt, dtcfl, dtau, rhs = src    solverSetup.loci:81-119,
 *                                                   solverTimestep.loci:289-338
 *   Jacobians     fjp / fjm (smoothed Roe)          fluxInviscid.loci:1190-1221
 *   assembly      fluid_L/U/D/B                     solverLinearSystem.loci:45-224
 *   relaxation    SGSBlockedSSolve / LSGS           linearSolverSGS.loci:43-329,
 *                                                   linearSolverLSGS.loci:1692-1954
 *   update        clipped Newton update             solverNewton.loci:62-91
 *   norms         residual (rtrms, etrms, ...)      solverResidual.loci:74-112
 *
 * Conventions (all shared with the reference):
 *   - primitive variables q = [T, u, v, w, p_g] (column order of every 5x5
 *     block; rows are the rho, rho u, rho v, rho w, rho e0 equations);
 *   - blocks are row-major, 25 contiguous values per entity;
 *   - interior face normals point from cl to cr; boundary faces have cr < 0
 *     and name boundary condition -cr-1;
 *   - host arrays are in the caller's (Loci) entity order and AoS layout; the
 *     library keeps its own RCM order and SoA layout on the device and
 *     translates at this boundary.
 *
 * Every function returns 0 on success or a negative FPSI_E_* code; no C++
 * exception crosses the ABI.  There is no CPU fallback: without a usable CUDA
 * device every compute entry point returns FPSI_E_CUDA.
 */
#ifndef FPSI_H
#define FPSI_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes -------------------------------------------------------- */
#define FPSI_OK              0
#define FPSI_E_INVALID      -1   /* bad argument or inconsistent mesh        */
#define FPSI_E_CUDA         -2   /* CUDA runtime failure / no device          */
#define FPSI_E_NOMEM        -3   /* device or host allocation failed          */
#define FPSI_E_UNSUPPORTED  -4   /* option not implemented on this path       */
#define FPSI_E_SINGULAR     -5   /* zero pivot in a 5x5 block LU              */
#define FPSI_E_NAN          -6   /* NaN residual (solverResidual.loci:203-208)*/
#define FPSI_E_TIMEOUT      -7   /* a bounded device wait gave up             */
#define FPSI_E_STATE        -8   /* call out of order (e.g. solve before assemble) */

/* ---- options (names and defaults follow the reference's vars) ----------- */
enum fpsi_flux_kind {          /* inviscidRiemannFlux, inviscidFlux.h:82-90 */
  FPSI_FLUX_HLLC = 0,          /* hllc_flux, fluxInviscid.loci:157-256 (reference default) */
  FPSI_FLUX_ROE  = 1,          /* roeCT_flux, fluxInviscid.loci:869-1014 */
  FPSI_FLUX_HLLE = 2,          /* two-wave HLL with hllc_flux's SL/SR (no reference counterpart) */
  FPSI_FLUX_KEC  = 3,          /* inviscidFlux "KEC": kinetic-energy-consistent low-dissipation
                                  flux on interior faces (KEC::iflux, fluxLowDiss.loci:320-431),
                                  hllc_flux on boundary faces */
  FPSI_FLUX_SSF  = 4           /* inviscidFlux "SSF": 4th-order skew-symmetric low-dissipation
                                  flux with a Roe-type MILES filter on interior faces
                                  (SSF::iflux, fluxLowDiss.loci:436-640), hllc_flux on boundary faces */
};
enum fpsi_limiter_kind {       /* vars 'limiter' (guide.tex:495-518) */
  FPSI_LIMITER_VENKATAKRISHNAN = 0,
  FPSI_LIMITER_BARTH = 1,
  FPSI_LIMITER_NONE = 2,
  FPSI_LIMITER_ZERO = 3
};
enum fpsi_solver_kind {        /* vars 'fluidLinearSolver' (solverNewton.loci:222-249) */
  FPSI_SOLVER_SGS = 0,         /* multi-colour block SGS */
  FPSI_SOLVER_LSGS = 1,        /* line SGS (batched block-tridiagonal lines) */
  FPSI_SOLVER_FSGS = 2         /* 'fsgs' (linearSolverFSGS.loci:1601-1700): gauss_seidel_iter
                                  symmetric sweeps from a zero start; the reference sweeps
                                  single cells in breadth-first order with an unpivoted block
                                  LU, this path the colours with the pivoted LU of SGS */
};
enum fpsi_precision {
  FPSI_PREC_FP64 = 0,          /* every block and iterate in FP64 */
  FPSI_PREC_REF = 1,           /* reference precision: FP32 blocks and B, FP64 iterate */
  FPSI_PREC_MIXED = 2          /* FP32 blocks, LU and sweeps (defect correction) */
};
enum fpsi_turbulence_kind {
  FPSI_TURB_EDDY_VISCOSITY = 0,    /* tmu given by fpsi_set_eddy_viscosity */
  FPSI_TURB_SA = 1                 /* Spalart-Allmaras nu~ transport, turbulence/SA/SA_turb.loci */
};
enum fpsi_bc_kind {
  FPSI_BC_FARFIELD = 1,            /* bcInflow.loci:311-375 */
  FPSI_BC_SUPERSONIC_INFLOW = 2,   /* bcInflow.loci:270-309 */
  FPSI_BC_SUPERSONIC_OUTFLOW = 3,  /* bcOutflow.loci:127-165 */
  FPSI_BC_EXTRAPOLATE = 4,         /* bcOutflow.loci:84-120 */
  FPSI_BC_REFLECTING = 5,          /* symmetry / slip wall, bcImpermeable.loci:48-140 */
  FPSI_BC_VISCOUS_WALL = 6,        /* adiabatic no-slip wall, bcViscousWall.loci:146-240 */
  FPSI_BC_OUTFLOW = 7,             /* subsonic outflow at back pressure 'p' (gauge: fpsi_bc.pg),
                                      bcOutflow.loci:174-273 */
  FPSI_BC_OUTFLOW_MEAN = 8,        /* outflow whose area-weighted mean pressure is 'pMean'
                                      (gauge: fpsi_bc.pg), bcOutflow.loci:178-204 */
  FPSI_BC_ISENTROPIC_INFLOW = 9,   /* total pressure p0 (gauge: fpsi_bc.pg) and temperature
                                      T0 (fpsi_bc.T), bcIsentropic.loci:40-240 */
  FPSI_BC_FIXED_MASS_INFLOW = 10,  /* mass flux (fpsi_bc.mass_flux) at total temperature T0
                                      (fpsi_bc.T), bcFixedMass.loci:84-235 */
  FPSI_BC_FIXED_MASS_OUTFLOW = 11, /* mass flux (fpsi_bc.mass_flux) relaxed by mass_relax,
                                      bcFixedMassOutflow.loci:72-186 */
  FPSI_BC_INFLOW = 12              /* subsonic inflow at the reference state (T, pg, u),
                                      bcInflow.loci:376-431: the farfield's inflow state
                                      where the flow enters, the reference state itself
                                      where it leaves */
};
/* fpsi_resid.bcErrorCode bits (flowPsiIO.h:212-215) */
#define FPSI_BCERR_OUTFLOW_BECAME_INFLOW 1
#define FPSI_BCERR_FIXED_MASS_FAILED_CONVERGENCE 4

typedef struct fpsi_params {
  double gamma;            /* 1.4                                  solverEoS.loci:31 */
  double Rtilde;           /* 8314.4621/28.96                      solverEoS.loci:34-37 */
  double Pambient;         /* p0 = 0                               solverEoS.loci:39-47 */
  double Minf;             /* 1; eta == 1 for Minf >= 0.5          fluxInviscid.loci:97-112 */
  int32_t flux;            /* fpsi_flux_kind, default HLLC */
  int32_t limiter;         /* fpsi_limiter_kind, default venkatakrishnan */
  double Kl;               /* Venkatakrishnan threshold, default 1 */
  double urelax;           /* 0.2                                  solverTimestep.loci:281-283 */
  double dtmax;            /* 1.0                                  solverTimestep.loci:285-287 */
  double cflmax;           /* <= 0 disables the CFL time step      solverTimestep.loci:294-297 */
  int32_t solver;          /* fpsi_solver_kind, default LSGS */
  int32_t gauss_seidel_iter; /* 6                                  linearSolverSGS.loci:39-41 */
  double lsgs_relaxation;  /* 0.25                                 linearSolverLSGS.loci:96-108 */
  double lsgs_abs_tol;     /* 1e-10 */
  double lsgs_rel_tol;     /* 0.1 */
  int32_t lsgs_max_iter;   /* 10 */
  int32_t precision;       /* fpsi_precision, default FPSI_PREC_REF */
  int32_t viscous;         /* flowRegime: 0 inviscid, 1 laminar, 2 turbulent
                                                                   fluxViscous.loci:28-52 */
  int32_t turbulence;      /* fpsi_turbulence_kind (viscous == 2): where tmu comes from */
  double Prt;              /* turbulentPrandtlNumber 0.9           fluxViscous.loci:268-270 */
  double mu_a1, mu_a2, mu_a3; /* Sutherland mu = a1 T^a2/(T+a3): 1.458e-6, 1.5, 110.4 */
  double k_a1, k_a2, k_a3;    /* conductivity k = k1 T^k2/(T+k3): 2.495e-3, 1.5, 194
                                 (sutherlandParameters, fluxViscous.loci:58-80) */
  int32_t time_accurate;   /* timeSteppingMode: 0 steady (pseudo-time, one Newton
                              iteration per step), 1 time accurate with the BDF2 scheme
                              (solverTimestep.loci:397-428); dtmax is then the time step */
  int32_t newton_iters;    /* newtonMaxIter: Newton iterations per time step, 6
                                                                   solverNewton.loci:200-210 */
  /* the low-dissipation (KEC) flux's switches, fluxLowDiss.loci:82-120 */
  double lds_comp_factor;       /* LDS_compFactor 5 */
  double lds_dissipation_limit; /* LDS_dissipationLimit 1 */
  double lds_ducros_factor;     /* LDS_ducrosFactor 0 */
  double lds_use_upwind;        /* LDS_useUpwind 0 */
  double lds_nonsym_coeff;      /* LDS_nonSymmetricCoeff 2 */
  double lds_nonsym_factor;     /* LDS_nonSymmetricFactor 1 */
  double lds_miles_filter;      /* LDS_MILES_filter 0.1 (SSF) */
  double ssf_coeff;             /* SSF_Coeff 1 (SSF) */
  int32_t step_graphs;     /* 1 (default): fpsi_run, fpsi_run_timed and
                              fpsi_time_step run the first step of a call
                              as launches, capture the second as a CUDA
                              graph and replay it for the rest (same
                              kernels, same results bit for bit); 0: every
                              step as launches */
  int32_t reserved2;
} fpsi_params;

typedef struct fpsi_bc {
  int32_t kind;            /* fpsi_bc_kind */
  int32_t reserved;
  double T, pg, u[3];      /* reference state (temperatureRef, gagePressureRef, uRef) */
  double nu_t;             /* SA nu~ entering through the boundary (BC option nu_t,
                              SA_turb.loci:167-179); <= 0 selects the default 5e-9 */
  double mass_flux;        /* fixed-mass conditions: 'massFlux' (kg/s/m^2), or <= 0 to use
                              mdot over the condition's area (massFlux_BC, bcFixedMass.loci:227-230) */
  double mdot;             /* fixed-mass conditions: 'mdot' (kg/s) */
  double mass_relax;       /* fixedMassOutflow 'massRelax' (default 1, bcFixedMassOutflow.loci:72-78) */
} fpsi_bc;

/* Unstructured mesh in the caller's numbering.  Face nodes are ordered so
 * that the right-hand-rule normal points from cl to cr.  For periodic faces
 * (translation only) pshift[3f..3f+2] is the vector that moves cell cr next to
 * cl (x_cr_image = x_cr + pshift); NULL means no periodic faces. */
typedef struct fpsi_mesh {
  int64_t nnodes, ncells, nfaces;
  const double*  xyz;          /* nnodes*3 */
  const int64_t* face_off;     /* nfaces+1 */
  const int32_t* face_nodes;   /* face_off[nfaces] */
  const int32_t* cl;           /* nfaces */
  const int32_t* cr;           /* nfaces; < 0 => boundary condition -cr-1 */
  const double*  pshift;       /* nfaces*3 or NULL */
  int32_t nbc;
  int32_t reserved;
  const fpsi_bc* bcs;          /* nbc */
} fpsi_mesh;

typedef struct fpsi_resid {    /* flowPsi::residual, flowTypes.h:421-427 (rms already square-rooted) */
  double rtrms, etrms, mtrms;  /* volume-weighted RMS of src/V: density, energy, momentum */
  double rtmax, etmax, mtmax;  /* signed L-inf values */
  double ccmaxr_center[3];
  double ccmaxe_center[3];
  uint64_t bcErrorCode;
} fpsi_resid;

typedef struct fpsi_lsinfo {
  int32_t iterations;          /* symmetric sweeps (SGS) or line iterations (LSGS) */
  int32_t status;
  double resid0, resid;        /* ||B - A x|| before / after (if measured) */
} fpsi_lsinfo;

typedef struct fpsi_stepinfo {
  fpsi_resid resid;            /* norms of the residual the step started from */
  fpsi_lsinfo ls;
  double min_alpha;            /* smallest Newton clip factor applied */
  double dtau_min, dtau_max;
  /* fpsi_newton_step_ex only: */
  fpsi_resid resid_after;      /* norms of the residual of the new state */
  int32_t start_used;          /* fpsi_start_kind the accepted update started from */
  int32_t rejected;            /* 1: the first attempt's update was rejected */
} fpsi_stepinfo;

typedef struct fpsi_ctx fpsi_ctx;
typedef struct fpsi_gnn fpsi_gnn;   /* learned starting iterate, below */

/* ---- parameters / errors -------------------------------------------------- */
void        fpsi_default_params(fpsi_params* p);
const char* fpsi_strerror(int code);
const char* fpsi_last_error(void);   /* detail of the last failure in this thread */
int         fpsi_device_available(void);

/* ---- synthetic meshes (host memory, caller frees with fpsi_mesh_free) ------
 * kind 0: nx*ny*nz hex box [0,Lx]x[0,Ly]x[0,Lz], boundary condition of the six
 *         sides bc_side[0..5] = (xmin, xmax, ymin, ymax, zmin, zmax); an entry
 *         of -1 makes that direction periodic (both sides).
 * kind 1: nx*ny*nz hexes each split into 6 Kuhn tetrahedra on the box
 *         [0,Lx]x[0,Ly]x[0,Lz], sides periodic (-1) or bounded as kind 0;
 *         nodes jittered by U(-jitter,+jitter)*h (not normal to a bounded
 *         side, so the sides stay plane).
 * kind 2: boundary-layer hex block: y spacing dy0*growth^j.
 * kind 3: the kind-0 box with each hex split into two triangular prisms
 *         across the diagonal of its z-faces (cells 2c and 2c+1 of hex c):
 *         five faces per cell, triangular and quadrilateral faces mixed.
 * Returns an fpsi_mesh whose arrays are owned by the library. */
typedef struct fpsi_mesh_spec {
  int32_t kind;
  int32_t nx, ny, nz;
  double Lx, Ly, Lz;
  double jitter;              /* fraction of the spacing */
  double dy0, growth;         /* kind 2 */
  uint64_t seed;
  int32_t bc_side[6];         /* index into bcs, or -1 (periodic) */
  int32_t nbc;
  int32_t reserved;
  fpsi_bc bcs[8];
} fpsi_mesh_spec;
int  fpsi_mesh_generate(const fpsi_mesh_spec* spec, fpsi_mesh** out);
void fpsi_mesh_free(fpsi_mesh* m);

/* ---- context -------------------------------------------------------------- */
int fpsi_create(fpsi_ctx** out, const fpsi_mesh* mesh, const fpsi_params* params);
int fpsi_destroy(fpsi_ctx* ctx);
int fpsi_set_params(fpsi_ctx* ctx, const fpsi_params* params);
int fpsi_info(fpsi_ctx* ctx, int64_t* ncells, int64_t* nfaces, int32_t* ncolours,
              int64_t* device_bytes);

/* geometry as the library computed it (caller order): cell volumes and
 * centroids, face area vectors (n*|A|) and centroids; any pointer may be NULL */
int fpsi_get_geometry(fpsi_ctx* ctx, double* vol, double* cellcenter,
                      double* face_an, double* face_area, double* facecenter);
/* keep (1, default) or drop (0) the unfactored diagonal blocks after the LU;
 * fpsi_linear_residual and the D export of fpsi_get_blocks need them */
int fpsi_keep_blocks(fpsi_ctx* ctx, int32_t keep);
/* Lines of the line-SGS solver (fluidLinearSolver 'lsgs',
 * linearSolverLSGS.loci:361-1110), caller order: line l is
 * line_cells[line_off[l] .. line_off[l+1]); consecutive cells must share a
 * face; cells left out become single-cell lines.  Without this call the
 * library links cells that are mutually among each other's two strongest
 * couplings (face area over centre distance; a second link only within a
 * factor 25 of the first, as linearSolverLSGS.loci:620).  Lines are coloured
 * so the lines of one colour are solved together. */
int fpsi_set_lines(fpsi_ctx* ctx, int64_t nlines, const int64_t* line_off,
                   const int32_t* line_cells);
/* per caller cell its line and position on the line; per line its colour */
int fpsi_get_lines(fpsi_ctx* ctx, int32_t* line_of_cell, int32_t* position,
                   int32_t* line_colour, int64_t* nlines);
/* cell colour used by the multi-colour sweeps (caller order) */
int fpsi_get_colours(fpsi_ctx* ctx, int32_t* colour);

/* turbulent eddy viscosity tmu[nc] (caller order) used by flowRegime
 * turbulent (muTotal = mu + tmu, kTotal = k + tmu Cp/Prt,
 * fluxViscous.loci:179-201,268-277); zero until set */
int fpsi_set_eddy_viscosity(fpsi_ctx* ctx, const double* tmu);

/* state in Loci layout: T[nc], pg[nc], u[nc*3] (AoS) */
int fpsi_set_state(fpsi_ctx* ctx, const double* T, const double* pg, const double* u);
int fpsi_get_state(fpsi_ctx* ctx, double* T, double* pg, double* u);

/* residual of the current state.  src (nc*5, AoS, may be NULL) receives
 * the reference's 'src' store; norms may be NULL.  grad (nc*15: dT/dx..,
 * du/dx.., dv/dx.., dw/dx.., dp/dx..) and limiter (nc*5) are optional views
 * of the reconstruction inputs. */
int fpsi_residual(fpsi_ctx* ctx, double* src, fpsi_resid* norms);
int fpsi_get_reconstruction(fpsi_ctx* ctx, double* grad, double* limiter);

/* local pseudo time step from the last residual (solverTimestep.loci:302-329) */
int fpsi_get_dtau(fpsi_ctx* ctx, double* dtau);

/* Jacobians and diagonal blocks for the last residual's state and dtau,
 * followed by the batched LU of the diagonal blocks. */
int fpsi_assemble(fpsi_ctx* ctx);
/* optional export of the assembled blocks (caller order, row-major 25 per
 * entity, as float in REF/MIXED and as double in FP64 precision):
 * D (nc*25, before factorisation), fjp and fjm (nfaces*25), B (nc*5).
 * An inviscid system relaxed by multi-colour SGS keeps its face Jacobians
 * in the compact Roe form (9 coefficients per direction plus the face's
 * Roe velocity and normal); fjp and fjm are then expanded from it on this
 * call, each entry evaluated in FP64 and rounded once. */
int fpsi_get_blocks(fpsi_ctx* ctx, void* D, void* fjp, void* fjm, void* B);

/* relaxation of  A dq = B.  x0 (nc*5 AoS) NULL selects the reference start
 * (block Jacobi D^-1 B).  dq (nc*5 AoS) may be NULL (result stays on the
 * device for fpsi_update). */
int fpsi_linear_solve(fpsi_ctx* ctx, const double* x0, double* dq, fpsi_lsinfo* info);
/* set the device iterate (caller order nc*5) of the assembled system: the
 * next fpsi_linear_solve(ctx, NULL, ...) or fpsi_linear_sweeps starts there */
int fpsi_set_iterate(fpsi_ctx* ctx, const double* x0);
/* the current device iterate (caller order nc*5) */
int fpsi_get_iterate(fpsi_ctx* ctx, double* x);
/* nsweeps more symmetric multi-colour sweeps from the current device iterate
 * (no restart), e.g. to run a solve to a tolerance with fpsi_linear_residual */
int fpsi_linear_sweeps(fpsi_ctx* ctx, int32_t nsweeps);
/* || B - A x || (2-norm over all cells) of the device iterate */
int fpsi_linear_residual(fpsi_ctx* ctx, double* norm_b, double* norm_r);
/* clipped Newton update with the device dq (solverNewton.loci:62-78) */
int fpsi_update(fpsi_ctx* ctx, double* min_alpha);

/* one steady implicit step: residual -> dtau -> assemble -> solve -> update.
 * NaN residual norms return FPSI_E_NAN and leave the state unchanged. */
int fpsi_newton_step(fpsi_ctx* ctx, fpsi_stepinfo* info);
/* Starting iterate of the relaxation and the rule that keeps a step.
 *   start       FPSI_START_JACOBI: the reference's D^-1 B
 *               (linearSolverSGS.loci:57-69); FPSI_START_ZERO; or
 *               FPSI_START_LEARNED: the model's start (fpsi_gnn_predict).
 *   reject      1: when the FP64 density residual (rtrms) of the new state is
 *               not below the one the step started from, a step that did not
 *               start from D^-1 B is undone and redone from D^-1 B, which is
 *               kept whatever its residual (the reference's step).
 *   lin_rtol    > 0: sweep until ||B - A x|| <= lin_rtol ||B||, measured every
 *               check_every sweeps, at most max_sweeps; <= 0: exactly
 *               gauss_seidel_iter sweeps.
 * The step is queued on the device and synchronises with the host once,
 * to read its new residual (more often when sweeping to lin_rtol).  A zero
 * pivot (FPSI_E_SINGULAR) or a model wait that gave up (FPSI_E_TIMEOUT)
 * leaves the state unchanged: the update kernel reads their error bits. */
enum fpsi_start_kind {
  FPSI_START_JACOBI = 0,
  FPSI_START_ZERO = 1,
  FPSI_START_LEARNED = 2
};
typedef struct fpsi_step_opts {
  int32_t start;               /* fpsi_start_kind */
  int32_t reject;
  double lin_rtol;
  int32_t max_sweeps;
  int32_t check_every;
} fpsi_step_opts;
/* one steady implicit step as fpsi_newton_step, with a chosen starting
 * iterate, an optional linear tolerance and the rejection rule above.  The
 * step ends with the residual of the new state (info->resid_after), which
 * the next call reuses as its starting residual.  model may be NULL unless
 * start is FPSI_START_LEARNED.  Multi-colour SGS without the SA model; the
 * learned start and a linear tolerance need the diagonal blocks kept
 * (fpsi_keep_blocks). */
int fpsi_newton_step_ex(fpsi_ctx* ctx, fpsi_gnn* model, const fpsi_step_opts* opts,
                        fpsi_stepinfo* info);
/* nsteps steps without host round trips; norms[k] of each step (may be NULL).
 * A step whose residual norms are NaN ends the run there, as
 * solverResidual.loci:203-208 aborts: the state stays the one that step
 * started from, norms[] is filled up to that step and NaN after it, and
 * the call returns FPSI_E_NAN (fpsi_last_error names the step).  The norm
 * history lives in the context (no allocation per call up to 4096 steps). */
int fpsi_run(fpsi_ctx* ctx, int32_t nsteps, fpsi_resid* norms);
/* ---- time-accurate stepping (params.time_accurate = 1, BDF2) -------------
 * One time step of size dtmax: params.newton_iters Newton iterations on the
 * state q(n+1), each with the residual rhs = src - (1.5 (Q(n+1) - Q(n)) -
 * 0.5 (Q(n) - Q(n-1))) V / dtmax of the conserved variables Q = (rho, rho u,
 * rho e0) (solverTimestep.loci:397-428), the diagonal blocks -srcJ +
 * 1.5 V / dtau dQ/dq (solverLinearSystem.loci:376-435), the linear solve and
 * the update clipped at 0.75 of T and p (solverNewton.loci:163-198); then
 * Q(n-1) = Q(n), Q(n) = Q(n+1).  The first step after fpsi_set_state takes
 * Q(n-1) = Q(n) = the set state.  norms (newton_iters entries, may be NULL)
 * receive the norms of each iteration's rhs.  In this mode fpsi_residual's
 * src is that rhs, and fpsi_newton_step is one Newton iteration of the
 * current time step. */
int fpsi_time_step(fpsi_ctx* ctx, fpsi_resid* norms);
/* fpsi_run timed on the device: CUDA events recorded on the library's
 * stream around the nsteps steps; device_ms receives the elapsed time. */
int fpsi_run_timed(fpsi_ctx* ctx, int32_t nsteps, fpsi_resid* norms, double* device_ms);
/* Per-kernel device time of nsteps steps (CUDA events around every launch
 * group on the library's stream).  Fills up to cap entries of names (32
 * chars each), total ms and launch counts; *count receives the number of
 * kernel kinds. */
int fpsi_kernel_times(fpsi_ctx* ctx, int32_t nsteps, int32_t cap, char* names, double* ms,
                      int64_t* launches, int32_t* count);

/* ---- learned starting iterate ---------------------------------------------
 * No counterpart in the reference; the hook is the starting iterate of the
 * relaxation (linearSolverSGS.loci:57-69).  A message-passing network over
 * the cell graph (3 layers of width 64, GELU, linear head; BF16 weights,
 * FP32 accumulation) maps each cell's fluid_B, fluid_D, block Jacobi
 * solution D^-1 B and the context's previous update (kept on the device
 * from the first use of a model with the context on; zero before), made
 * scale free per system, to a correction d of the block Jacobi start:
 * x0 = D^-1 B + xs * d (xs = RMS of D^-1 B per component).  The weights do not depend on the mesh: one model serves any
 * context.  Training pairs come from the solver: fpsi_gnn_add_snapshot takes
 * the features of an assembled system, its cell graph and its converged dq
 * (caller order).  The model runs on its own stream. */
int fpsi_gnn_create(fpsi_gnn** out, uint64_t seed);
int fpsi_gnn_destroy(fpsi_gnn* m);
int64_t fpsi_gnn_num_params(const fpsi_gnn* m);
/* FP32 master weights, flat: per layer l: Ws[64][fin], Wn[64][fin], b[64]
 * (fin = 40, 64, 64), then head Wo[5][64], bo[5] */
int fpsi_gnn_get_params(fpsi_gnn* m, float* w);
int fpsi_gnn_set_params(fpsi_gnn* m, const float* w);
int fpsi_gnn_add_snapshot(fpsi_gnn* m, fpsi_ctx* ctx, const double* dq);
/* a snapshot of the cells of ctx's assembled system whose centroids lie in
 * the box lo <= x < hi: their features (those of the whole system), the
 * graph among them, dq and the Jacobi start; the loss counts only cells
 * more than `halo` hops from every cell outside the box, whose network
 * inputs the box holds in full (halo = 3 for the three layers).  Keeps the
 * training set of a large grid small; its cells are listed in the
 * library's order (fpsi_gnn_get_snapshot). */
int fpsi_gnn_add_snapshot_region(fpsi_gnn* m, fpsi_ctx* ctx, const double* dq, const double* lo,
                                 const double* hi, int32_t halo);
int fpsi_gnn_clear_snapshots(fpsi_gnn* m);
int fpsi_gnn_num_snapshots(const fpsi_gnn* m);
/* cells of snapshot s (-1 when s is out of range) */
int64_t fpsi_gnn_snapshot_cells(const fpsi_gnn* m, int32_t s);
/* features (nc*40), targets (nc*5), Jacobi start (nc*5), scales rs[5] xs[5] */
int fpsi_gnn_get_snapshot(fpsi_gnn* m, int32_t s, float* feat, float* target, float* xjac,
                          float* scales);
/* mean squared error and its gradient (flat, as the parameters) on snapshot
 * s over a batch of about `batch` cells chosen by seed (all when batch >= nc) */
int fpsi_gnn_loss_grad(fpsi_gnn* m, int32_t s, int64_t batch, uint64_t seed, double* loss,
                       float* grad);
/* nsteps Adam steps (lr; beta 0.9/0.999) on random snapshots and batches */
int fpsi_gnn_train(fpsi_gnn* m, int32_t nsteps, int64_t batch, uint64_t seed, double lr,
                   double* losses);
/* learned start for ctx's assembled system: the next fpsi_linear_solve(ctx,
 * NULL, ...) or fpsi_linear_sweeps starts from it; x0 (caller order) optional */
int fpsi_gnn_predict(fpsi_gnn* m, fpsi_ctx* ctx, double* x0);

/* ---- Spalart-Allmaras turbulence model ----------------------------------
 * With params.viscous = 2 and params.turbulence = FPSI_TURB_SA the context
 * owns the working variable nu~ (nuTilde; baseline model, standard
 * production, SA_turb.loci:85-476).  fpsi_residual first sets the eddy
 * viscosity tmu = rho nu~ f_v1 (:105-107) from it.  fpsi_newton_step and
 * fpsi_run advance nu~ once per step, segregated from the mean flow as the
 * reference's scalar transport (solverScalarTransport.loci:36-700): upwind
 * convection by the mean flow's mass flux, production, destruction and
 * diffusion, the steady pseudo-time term with the mean flow's dtau, scalar
 * multi-colour SGS (linearSolverSGS.loci:333-470) and the relaxed positive
 * update (:397-405).  The wall distance is the distance from the cell centre
 * to the plane of the nearest no-slip wall face (gridSetup.loci:418-640,
 * solverTurbulence.loci:133-137); without walls it is 1e30. */
int fpsi_set_nutilde(fpsi_ctx* ctx, const double* nut);      /* caller order, nc */
int fpsi_get_nutilde(fpsi_ctx* ctx, double* nut);
int fpsi_get_eddy_viscosity(fpsi_ctx* ctx, double* tmu);     /* as last used */
int fpsi_get_wall_distance(fpsi_ctx* ctx, double* dist);
/* after fpsi_residual: nuTilde_src (the scalar right-hand side), optional */
int fpsi_sa_residual(fpsi_ctx* ctx, double* src);
/* scalar system of the last fpsi_sa_residual: X_D (nc), X_fjp and X_fjm
 * (nf; L = -fjp, U = fjm), any may be NULL; caller order */
int fpsi_sa_get_system(fpsi_ctx* ctx, double* D, double* fjp, double* fjm);
/* Jacobi start and gauss_seidel_iter symmetric sweeps; dq optional */
int fpsi_sa_solve(fpsi_ctx* ctx, double* dq);
int fpsi_sa_update(fpsi_ctx* ctx);

/* ---- residual norms without allocation -----------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * (a host code that hands out device buffers from its own pool and forbids
 * allocations behind it, or a step that must not block or fail on an
 * allocation): the norms of fpsi_residual computed from caller-owned device
 * buffers -- d_src (nc*5 doubles, the 'src' store), d_vol (nc doubles) --
 * into d_out (8 doubles: rtrms, etrms, mtrms, rtmax, cell of rtmax, etmax,
 * cell of etmax, mtmax).  stream is a cudaStream_t or NULL.
 * Allocates nothing: the block partials live in a static 1 MiB __device__
 * array that every GPU loading the library keeps until exit, so nc is
 * limited to 16,777,216 cells (larger sizes return FPSI_E_INVALID).  Each
 * call outside a stream capture looks the array's address up on the current
 * device (no allocation), which also follows a module reloaded after
 * cudaDeviceReset; a call inside a capture reuses the address found last,
 * so make the first call on a device before any stream capture (else
 * FPSI_E_STATE).  Every call overwrites
 * the partials it reads, so nothing must start at zero; calls that overlap
 * on the GPU share the array and race. */
int fpsi_residual_norms_noalloc(const double* d_src, const double* d_vol, int64_t nc,
                                double vol_tot, double* d_out, void* stream);

/* ---- face functions on batches (inviscidFlux.h entry points) --------------
 * States are packed per face as [pg, T, u, v, w] (n*5), normals n*3 (unit),
 * area n.  Host pointers; copies and one kernel launch inside. */
int fpsi_face_flux(int32_t kind, int64_t n, const double* qL, const double* qR,
                   const double* an, const double* area, double pambient,
                   double Rt, double gamma, double us_n, double eta, double* flux);
/* roeCT_jacobian (fluxInviscid.loci:1092-1168); dir = +1 (fjp) or -1 (fjm).
 * out is n*25 float (real_fj) or double when as_double != 0. */
int fpsi_face_jacobian(int64_t n, const double* qL, const double* qR,
                       const double* an, const double* area, double pambient,
                       double Rt, double gamma, double us_n, double eta,
                       int32_t dir, int32_t as_double, void* out);

#ifdef __cplusplus
}
#endif
#endif /* FPSI_H */
