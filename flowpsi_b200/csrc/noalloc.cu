// noalloc.cu -- residual norms for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: a host code that hands the library
// buffers from its own memory pool (and forbids allocations behind the
// pool's back), or code running where a device allocation would be a
// synchronising, failure-prone call in a step that must not fail.  This
// entry point computes the same norms as fpsi_residual from caller-owned
// device buffers and allocates nothing.  Its block partials live in one
// file-scope __device__ array of fixed size (1 MiB), which every GPU that
// loads the library holds until the process exits.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "fpsi_internal.h"

namespace {

constexpr int NA_THREADS = 256;
constexpr int NA_CELLS_PER_THREAD = 4;
constexpr int64_t NA_CELLS_PER_BLOCK = int64_t(NA_THREADS) * NA_CELLS_PER_THREAD;
constexpr int64_t NA_MAX_BLOCKS = 16384;
constexpr int64_t NA_MAX_CELLS = NA_MAX_BLOCKS * NA_CELLS_PER_BLOCK;  // 16,777,216

// 8 partial values per block: three weighted sums, signed maxima of the
// density and energy residuals with their cell indices, momentum maximum.
static __device__ __align__(256) double g_norm_scratch[NA_MAX_BLOCKS * 8];

__device__ __forceinline__ bool take(double v, double loc, double cur, double cloc) {
  return fabs(v) > fabs(cur) || (fabs(v) == fabs(cur) && loc >= 0 && (cloc < 0 || loc < cloc));
}

__global__ void __launch_bounds__(NA_THREADS)
k_norm_partial(const double* __restrict__ src, const double* __restrict__ vol, int64_t nc,
               double vol_tot, double* __restrict__ scratch) {
  double a[8] = {0, 0, 0, 0, -1, 0, -1, 0};
  const int64_t base = int64_t(blockIdx.x) * NA_CELLS_PER_BLOCK;
  for (int r = 0; r < NA_CELLS_PER_THREAD; ++r) {
    const int64_t c = base + int64_t(r) * NA_THREADS + threadIdx.x;
    if (c >= nc) break;
    const double* s = src + 5 * c;
    const double V = vol[c];
    const double rv = 1.0 / V, w = V / vol_tot;
    const double a0 = rv * s[0], a4 = rv * s[4];
    a[0] += w * (a0 * a0);
    a[1] += w * (a4 * a4);
    double mm = 0, mmax = 0;
    for (int i = 0; i < 3; ++i) {
      const double m = rv * s[1 + i];
      if (fabs(mmax) < fabs(m)) mmax = m;
      mm += m * m;
    }
    a[2] += mm * (w / 3.0);
    if (take(a0, double(c), a[3], a[4])) a[3] = a0, a[4] = double(c);
    if (take(a4, double(c), a[5], a[6])) a[5] = a4, a[6] = double(c);
    if (fabs(mmax) > fabs(a[7])) a[7] = mmax;
  }
  __shared__ double sh[8][NA_THREADS];
  const int t = threadIdx.x;
  for (int k = 0; k < 8; ++k) sh[k][t] = a[k];
  __syncthreads();
  for (int st = NA_THREADS / 2; st > 0; st >>= 1) {
    if (t < st) {
      sh[0][t] += sh[0][t + st];
      sh[1][t] += sh[1][t + st];
      sh[2][t] += sh[2][t + st];
      if (take(sh[3][t + st], sh[4][t + st], sh[3][t], sh[4][t]))
        sh[3][t] = sh[3][t + st], sh[4][t] = sh[4][t + st];
      if (take(sh[5][t + st], sh[6][t + st], sh[5][t], sh[6][t]))
        sh[5][t] = sh[5][t + st], sh[6][t] = sh[6][t + st];
      if (fabs(sh[7][t + st]) > fabs(sh[7][t])) sh[7][t] = sh[7][t + st];
    }
    __syncthreads();
  }
  if (t == 0)
    for (int k = 0; k < 8; ++k) scratch[8 * int64_t(blockIdx.x) + k] = sh[k][0];
}

__global__ void __launch_bounds__(NA_THREADS)
k_norm_combine(const double* __restrict__ scratch, int64_t nblk, double* __restrict__ out) {
  __shared__ double sh[8][NA_THREADS];
  const int t = threadIdx.x;
  double a[8] = {0, 0, 0, 0, -1, 0, -1, 0};
  for (int64_t i = t; i < nblk; i += NA_THREADS) {
    const double* p = scratch + 8 * i;
    a[0] += p[0], a[1] += p[1], a[2] += p[2];
    if (take(p[3], p[4], a[3], a[4])) a[3] = p[3], a[4] = p[4];
    if (take(p[5], p[6], a[5], a[6])) a[5] = p[5], a[6] = p[6];
    if (fabs(p[7]) > fabs(a[7])) a[7] = p[7];
  }
  for (int k = 0; k < 8; ++k) sh[k][t] = a[k];
  __syncthreads();
  for (int st = NA_THREADS / 2; st > 0; st >>= 1) {
    if (t < st) {
      sh[0][t] += sh[0][t + st];
      sh[1][t] += sh[1][t + st];
      sh[2][t] += sh[2][t + st];
      if (take(sh[3][t + st], sh[4][t + st], sh[3][t], sh[4][t]))
        sh[3][t] = sh[3][t + st], sh[4][t] = sh[4][t + st];
      if (take(sh[5][t + st], sh[6][t + st], sh[5][t], sh[6][t]))
        sh[5][t] = sh[5][t + st], sh[6][t] = sh[6][t + st];
      if (fabs(sh[7][t + st]) > fabs(sh[7][t])) sh[7][t] = sh[7][t + st];
    }
    __syncthreads();
  }
  if (t == 0) {
    out[0] = sqrt(sh[0][0]);
    out[1] = sqrt(sh[1][0]);
    out[2] = sqrt(sh[2][0]);
    for (int k = 3; k < 8; ++k) out[k] = sh[k][0];
  }
}

// Device address of g_norm_scratch.  In host code the symbol itself is
// only a host-side stand-in: a kernel given it would fault or silently use
// the wrong memory.  The address is looked up on every call made outside a
// stream capture (the lookup allocates nothing), so a module reloaded after
// cudaDeviceReset is followed; a call inside a capture uses the address the
// last uncaptured call on that device found.
constexpr int NA_MAX_DEVICES = 64;
std::mutex g_mu;
double* g_scratch_ptr[NA_MAX_DEVICES] = {nullptr};

int scratch_for_current_device(cudaStream_t s, double** out) {
  int dev = 0;
  FPSI_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NA_MAX_DEVICES) {
    fpsi::set_error("device ordinal %d beyond the %d supported", dev, NA_MAX_DEVICES);
    return FPSI_E_UNSUPPORTED;
  }
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  FPSI_CUDA_TRY(cudaStreamIsCapturing(s, &cap));
  std::lock_guard<std::mutex> lk(g_mu);
  if (cap != cudaStreamCaptureStatusNone && !g_scratch_ptr[dev]) {
    fpsi::set_error("fpsi_residual_norms_noalloc: the first call on a device must come before "
                    "any stream capture");
    return FPSI_E_STATE;
  }
  if (cap == cudaStreamCaptureStatusNone) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_norm_scratch);
    if (e != cudaSuccess || !p) {
      fpsi::set_error("cudaGetSymbolAddress(g_norm_scratch): %s", cudaGetErrorString(e));
      return FPSI_E_CUDA;
    }
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[dev];
  return FPSI_OK;
}

}  // namespace

extern "C" int fpsi_residual_norms_noalloc(const double* d_src, const double* d_vol, int64_t nc,
                                           double vol_tot, double* d_out, void* stream) {
  if (!d_src || !d_vol || !d_out || nc <= 0 || !(vol_tot > 0)) {
    fpsi::set_error("fpsi_residual_norms_noalloc: null buffer, empty mesh or vol_tot <= 0");
    return FPSI_E_INVALID;
  }
  if (nc > NA_MAX_CELLS) {
    fpsi::set_error("fpsi_residual_norms_noalloc: %lld cells exceed the static scratch limit "
                    "of %lld cells", (long long)nc, (long long)NA_MAX_CELLS);
    return FPSI_E_INVALID;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* scratch = nullptr;
  int rc = scratch_for_current_device(s, &scratch);
  if (rc) return rc;
  const int64_t nblk = (nc + NA_CELLS_PER_BLOCK - 1) / NA_CELLS_PER_BLOCK;
  k_norm_partial<<<unsigned(nblk), NA_THREADS, 0, s>>>(d_src, d_vol, nc, vol_tot, scratch);
  k_norm_combine<<<1, NA_THREADS, 0, s>>>(scratch, nblk, d_out);
  FPSI_CUDA_TRY(cudaGetLastError());
  return FPSI_OK;
}
