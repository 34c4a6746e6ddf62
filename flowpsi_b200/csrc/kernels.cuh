// kernels.cuh -- host launchers of the device path (internal).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

struct fpsi_ctx;

namespace fpsi {

// residual chain: boundary states, gradient+limiter, face flux, per-cell
// gather (src, dtau), norms into resid_slot[8] (device)
int launch_residual(fpsi_ctx* x, double* resid_slot);
// the gradient-and-limiter records of the last residual's state (written
// by the residual itself only for viscous runs)
int launch_grad_records(fpsi_ctx* x);
// face Jacobians, diagonal blocks, LU, B and the starting iterate
// (the starting iterate is the block Jacobi start D^-1 B)
int launch_assemble(fpsi_ctx* x);
// block Jacobi start x = D^-1 B on an assembled system
int launch_jacobi_start(fpsi_ctx* x);
// `sweeps` symmetric multi-colour Gauss-Seidel sweeps on the device iterate
int launch_sgs(fpsi_ctx* x, int sweeps);
// out2[0] = ||B||, out2[1] = ||B - A x|| (device)
int launch_linres(fpsi_ctx* x, double* out2);
// fills fjp/fjm from the compact face records of the assembled system (a
// no-op when they already hold it)
int ensure_explicit_blocks(fpsi_ctx* x);
// clipped Newton update; per-block minimum alpha into d_amin.  guard
// (device, may be null): the norms of the residual the system came from;
// NaN norms leave the state unchanged
int launch_update(fpsi_ctx* x, const double* guard, const int32_t* flag0 = nullptr,
                  const int32_t* flag1 = nullptr);
// caller-order staging buffer <-> device state (in = staging -> q)
int launch_state(fpsi_ctx* x, bool in);

int launch_batch_flux(int kind, int64_t n, const double* qL, const double* qR, const double* an,
                      const double* area, double pamb, double Rt, double gamma, double us_n,
                      double eta, double* F, cudaStream_t s);
int launch_batch_jac(int64_t n, const double* qL, const double* qR, const double* an,
                     const double* area, double pamb, double Rt, double gamma, double us_n,
                     double eta, int dir, int as_double, void* out, cudaStream_t s);

const char* last_error();

}  // namespace fpsi
