/*
 * oracle.h -- CPU restatement of flowPsi's implicit residual-and-relaxation
 * path.  TEST INFRASTRUCTURE ONLY: the parity tests, the smoke check and the
 * CPU-baseline leg of the benchmark call it as the checker; the product
 * library (libfpsi) never links or calls it.
 *
 * Each function cites the reference file:line it restates.  Where the
 * reference's arithmetic lives in the (unvendored) Loci FVM module -- LSQ
 * gradients, limiters, MUSCL reconstruction, geometry -- the published method
 * is restated and parity is unpinned.
 */
#ifndef FPSI_ORACLE_H
#define FPSI_ORACLE_H
#include "../include/fpsi.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_ctx orc_ctx;

int  orc_create(orc_ctx** out, const fpsi_mesh* mesh, const fpsi_params* params);
void orc_destroy(orc_ctx* o);
int  orc_set_params(orc_ctx* o, const fpsi_params* params);
int  orc_get_geometry(orc_ctx* o, double* vol, double* cellcenter, double* face_an,
                      double* face_area, double* facecenter);
int  orc_set_state(orc_ctx* o, const double* T, const double* pg, const double* u);
int  orc_set_eddy_viscosity(orc_ctx* o, const double* tmu);
int  orc_get_state(orc_ctx* o, double* T, double* pg, double* u);
int  orc_residual(orc_ctx* o, double* src, fpsi_resid* norms);
int  orc_get_reconstruction(orc_ctx* o, double* grad, double* limiter);
int  orc_get_dtau(orc_ctx* o, double* dtau);
int  orc_assemble(orc_ctx* o);
int  orc_get_blocks(orc_ctx* o, void* D, void* fjp, void* fjm, void* B);
/* colour == NULL: the reference's sequential forward/backward order
 * (linearSolverSGS.loci:150-305); otherwise the multi-colour order. */
int  orc_linear_solve(orc_ctx* o, const int32_t* colour, const double* x0, double* dq,
                      fpsi_lsinfo* info);
int  orc_linear_residual(orc_ctx* o, double* norm_b, double* norm_r);
/* line SGS (linearSolverLSGS.loci:1465-1954) over caller lines; with
 * line_colour the lines are swept colour by colour, else in line order */
int  orc_lsgs_solve(orc_ctx* o, int64_t nlines, const int64_t* line_off,
                    const int32_t* line_cells, const int32_t* line_colour, const double* x0,
                    double* dq, fpsi_lsinfo* info);
int  orc_update(orc_ctx* o, double* min_alpha);
int  orc_newton_step(orc_ctx* o, const int32_t* colour, fpsi_stepinfo* info);
/* Spalart-Allmaras nu~ transport (turbulence/SA/SA_turb.loci), as
 * fpsi_set_nutilde ... fpsi_sa_update; orc_sa_solve takes the sweep order
 * like orc_linear_solve */
int  orc_set_nutilde(orc_ctx* o, const double* nut);
int  orc_get_nutilde(orc_ctx* o, double* nut);
int  orc_get_eddy_viscosity(orc_ctx* o, double* tmu);
int  orc_get_wall_distance(orc_ctx* o, double* dist);
int  orc_sa_residual(orc_ctx* o, double* src);
int  orc_sa_get_system(orc_ctx* o, double* D, double* fjp, double* fjm);
int  orc_sa_solve(orc_ctx* o, const int32_t* colour, double* dq);
int  orc_sa_update(orc_ctx* o);
/* number of OpenMP threads the oracle loops use (1 = scalar) */
int  orc_set_threads(int n);

/* face functions on batches, same packing as fpsi_face_flux */
int orc_face_flux(int32_t kind, int64_t n, const double* qL, const double* qR,
                  const double* an, const double* area, double pambient, double Rt,
                  double gamma, double us_n, double eta, double* flux);
int orc_face_jacobian(int64_t n, const double* qL, const double* qR, const double* an,
                      const double* area, double pambient, double Rt, double gamma,
                      double us_n, double eta, int32_t dir, int32_t as_double, void* out);
/* characteristic boundary states cv_inflow / cv_outflow (bcTools.h:25-81),
 * qi and q0 packed [pg,T,u,v,w]; out packed the same way */
int orc_cv_state(int32_t outflow, int64_t n, const double* qi, const double* q0,
                 const double* an, double us_n, double pambient, double gamma,
                 double Rt, double beta, double* out);

#ifdef __cplusplus
}
#endif
#endif
