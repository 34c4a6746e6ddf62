// gnn.cu -- learned starting iterate for the block relaxation.
//
// No counterpart in the reference: the hook is the starting iterate of the
// SGS/LSGS solve (linearSolverSGS.loci:57-69, linearSolverLSGS.loci:1708-1728),
// which the reference sets to the block Jacobi solution x_J = D^-1 B.
//
// Model.  Per cell c the 40 inputs are the right-hand side B_c (5), the
// diagonal block D_c (25), the block Jacobi solution x_J,c = D_c^-1 B_c (5)
// and the context's previous update dq_prev,c (5; zero before the first
// update), made scale free per system: B by its RMS per component (rs),
// x_J and dq_prev by the RMS of x_J per component (xs), D_ij by xs_j/rs_i (so
// that the scaled blocks map the scaled x_J onto the scaled B).  Neighbour
// information enters through the mean aggregation of every layer.  Three
// message-passing layers
//     h' = GELU(W_s h + W_n mean_{n in N(c)} h + b)        (40 -> 64 -> 64 -> 64)
// and a linear head (64 -> 5) give d, and the starting iterate is
//     x0 = x_J + xs * d,
// so a network that outputs zero reproduces the reference's start.  Weights
// and activations are BF16, accumulation FP32: each message-passing layer is
// one tcgen05 tensor-core GEMM per 128-cell tile ([h | agg] times
// [Ws | Wn]^T, accumulator in tensor memory) with bias and GELU applied as
// the accumulator is read back.  FP32 master weights and Adam moments are
// kept for training.  Training targets are (dq - x_J)/xs for
// solver-generated converged dq.  All reductions (weight gradients, loss)
// are per-block partials summed in a fixed order: training is reproducible.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <type_traits>
#include <vector>

#include "fpsi_internal.h"
#include "kernels.cuh"

namespace {

constexpr int NIN = 40;
constexpr int W = 64;  // hidden width
constexpr int NOUT = 5;
constexpr int NLAYER = 3;
constexpr int GT = 128;  // threads per block for the per-cell kernels

// flat parameter layout (FP32 masters)
struct Layout {
  int64_t ws[NLAYER], wn[NLAYER], b[NLAYER], wo, bo, total;
  int fan_in[NLAYER];
};
Layout layout() {
  Layout L;
  int64_t o = 0;
  for (int l = 0; l < NLAYER; ++l) {
    const int fin = l == 0 ? NIN : W;
    L.fan_in[l] = fin;
    L.ws[l] = o, o += int64_t(W) * fin;
    L.wn[l] = o, o += int64_t(W) * fin;
    L.b[l] = o, o += W;
  }
  L.wo = o, o += int64_t(NOUT) * W;
  L.bo = o, o += NOUT;
  L.total = o;
  return L;
}

// cell graph of one mesh: interior-face neighbours in RCM order (CSR) and
// the RCM -> caller cell map
struct Graph {
  int64_t nc = 0;
  const int32_t* off = nullptr;
  const int32_t* nb = nullptr;
  // the same graph entry-major (a context's mesh): [K][nc], -1 = no neighbour
  const int32_t* ell = nullptr;
  int K = 0;
};

struct Snapshot {
  int64_t nc = 0;
  int32_t *d_off = nullptr, *d_nb = nullptr;  // own copy of the system's graph
  std::vector<int32_t> perm;
  float* feat = nullptr;    // [nc][40]
  float* target = nullptr;  // [nc][5]  (dq - xJ)/xs
  float* xj = nullptr;      // [nc][5]
  float* mask = nullptr;    // [nc] 1 where the loss counts (region snapshots), or null: all
  float xs[5], rs[5];
  Graph graph() const { return Graph{nc, d_off, d_nb}; }
};

}  // namespace

struct fpsi_gnn {
  Layout L;
  float *d_w = nullptr, *d_m = nullptr, *d_v = nullptr, *d_g = nullptr;
  __nv_bfloat16* d_wb = nullptr;
  int64_t adam_t = 0;
  // activations for one full-graph pass, sized for `cap` cells
  int64_t cap = 0;
  // BF16 activations (h[0] is the FP32 feature array of the pass), FP32
  // pre-activations for the backward pass
  __nv_bfloat16 *d_h[NLAYER + 1] = {nullptr}, *d_agg[NLAYER] = {nullptr};
  float* d_z[NLAYER] = {nullptr};
  float *d_y = nullptr, *d_dh = nullptr, *d_dh2 = nullptr, *d_dz = nullptr, *d_dagg = nullptr;
  float* d_part = nullptr;  // weight-gradient partials
  double* d_lpart = nullptr;
  std::vector<Snapshot> snaps;
  cudaStream_t stream = nullptr;
  int nsm = 148;                  // multiprocessors of the device (grid of the layer GEMM)
  int32_t* d_err = nullptr;       // bit 1: a tensor-core wait gave up
  float* d_fac = nullptr;         // inference: scales rs|xs (10) then the 40 feature factors
};

namespace {

// GELU in the tanh form of Hendrycks and Gimpel ("Gaussian Error Linear
// Units", 2016):  0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))).  Since
// 1 + tanh(u) = 2 / (1 + exp(-2u)) it is x / (1 + exp(-2u)): one base-2
// exponential and one fast division on the special-function unit, against
// the twenty-odd instructions of erff.  The tanh form differs from the erf
// form by at most 4.8e-4 (at |x| = 2.7); the network is trained with it.
constexpr float GELU_K = 0.7978845608028654f;  // sqrt(2/pi)
constexpr float GELU_C = 0.044715f;
// -2 sqrt(2/pi) log2(e): exp(-2u) = 2^(GELU_T x (1 + GELU_C x^2))
constexpr float GELU_T = -2.0f * 0.7978845608028654f * 1.4426950408889634f;
__device__ __forceinline__ float ex2_approx(float t) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(t));
  return r;
}
__device__ __forceinline__ float gelu(float x) {
  const float e = ex2_approx(GELU_T * x * fmaf(GELU_C, x * x, 1.0f));
  return __fdividef(x, 1.0f + e);
}
// d/dx [x s(x)], s = 1 / (1 + exp(-2u)):  s + x s (1 - s) 2 sqrt(2/pi) (1 + 3 GELU_C x^2)
__device__ __forceinline__ float gelu_grad(float x) {
  const float x2 = x * x;
  const float e = ex2_approx(GELU_T * x * fmaf(GELU_C, x2, 1.0f));
  const float sg = __fdividef(1.0f, 1.0f + e);
  return sg + x * sg * (1.0f - sg) * (2.0f * GELU_K) * fmaf(3.0f * GELU_C, x2, 1.0f);
}

// a layer input as the tensor cores multiply it (FP32 features rounded to BF16)
__device__ __forceinline__ float as_operand(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }
__device__ __forceinline__ float as_operand(__nv_bfloat16 v) { return __bfloat162float(v); }

// ---- tcgen05 helpers (single-CTA MMA, no multicast) ----------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// shared-memory matrix descriptor, K-major without swizzle: 8-row core
// matrices of 16 B rows; SBO = byte step between 8-row groups, LBO = byte
// step between the two 8-element K halves of one MMA (version 1, base 0)
__device__ __forceinline__ uint64_t umma_desc(const void* p, uint32_t lbo, uint32_t sbo) {
  const uint64_t a = (smem_u32(p) & 0x3FFFFu) >> 4;
  return a | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) | (uint64_t((sbo >> 4) & 0x3FFFu) << 32) |
         (uint64_t(1) << 46);
}
// instruction descriptor: BF16 x BF16 -> FP32, both K-major, M = 128, N = 64
constexpr uint32_t UMMA_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(W >> 3) << 17) |
                                (uint32_t(128 >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(UMMA_IDESC), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void mbar_init1(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}
// bounded wait on an mbarrier phase: false after ~2^24 polls
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (uint32_t it = 0; it < (1u << 24); ++it) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
// 32 lanes x 32 FP32 columns of the accumulator for this warp
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
      "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
      "[%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
        "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
        "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
        "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

// 8 consecutive elements of a layer input (one 16 B operand chunk), held
// as loaded so that many loads can be in flight before they are used
template <class T>
struct Chunk8;
template <>
struct Chunk8<__nv_bfloat16> {
  uint4 u;
  __device__ __forceinline__ void load(const __nv_bfloat16* p) { u = __ldg(reinterpret_cast<const uint4*>(p)); }
  __device__ __forceinline__ void get(float* v) const {
    const __nv_bfloat162* q = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float2 f = __bfloat1622float2(q[k]);
      v[2 * k] = f.x;
      v[2 * k + 1] = f.y;
    }
  }
};
template <>
struct Chunk8<float> {
  float4 a, b;
  __device__ __forceinline__ void load(const float* p) {
    a = __ldg(reinterpret_cast<const float4*>(p));
    b = __ldg(reinterpret_cast<const float4*>(p) + 1);
  }
  __device__ __forceinline__ void get(float* v) const {
    v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w, v[4] = b.x, v[5] = b.y, v[6] = b.z, v[7] = b.w;
  }
};
// a layer input value as the network sees it: FP32 features are rounded to
// BF16 (the own row and every neighbour row before their mean), BF16
// activations are already
template <class TIn>
__device__ __forceinline__ float as_input(float x) {
  return std::is_same<TIn, float>::value ? __bfloat162float(__float2bfloat16_rn(x)) : x;
}
__device__ __forceinline__ uint4 pack8(const float* v) {
  uint4 u;
  __nv_bfloat162* q = reinterpret_cast<__nv_bfloat162*>(&u);
#pragma unroll
  for (int k = 0; k < 4; ++k) q[k] = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
  return u;
}

constexpr int TC_ROWS = 128;     // cells per tile (the MMA's M)
constexpr int TC_COLS = 64;      // tensor-memory columns held per CTA (the MMA's N)
constexpr int TC_THREADS = 256;  // 8 warps: two per accumulator lane quarter
constexpr int TC_OSTRIDE = 144;  // bytes per row of the staged BF16 output tile (128 + 16 pad)
constexpr int NB_FAST = 6;       // neighbours per cell gathered with all loads in flight

struct TcSmem {  // byte offsets of the layer kernel's dynamic shared memory
  size_t a, b, o, y, wo, bar, slot, bias, total;
};
__host__ __device__ inline TcSmem tc_smem(int fin) {
  const size_t nch = size_t(2 * fin / 8);  // 16 B chunks of one operand row
  TcSmem s;
  s.a = 0;
  s.b = s.a + nch * TC_ROWS * 16;
  s.o = s.b + nch * W * 16;
  s.y = s.o + size_t(TC_ROWS) * TC_OSTRIDE;
  s.wo = s.y + size_t(TC_ROWS) * 8 * sizeof(float);
  s.bar = s.wo + size_t(NOUT * W + 8) * sizeof(float);
  s.slot = s.bar + 8;
  s.bias = s.slot + 8;
  s.total = s.bias + W * sizeof(float);
  return s;
}

// One message-passing layer, aggregation included, on the tensor cores,
// persistent over 128-cell tiles:
//   A = [h | mean over graph neighbours of h]   (BF16, staged from global)
//   z = A [Ws | Wn]^T + b                         (tcgen05, FP32 in tensor memory)
//   h_out = BF16(GELU(z))
// and, for the last layer, the head y = Wo h_out + bo.  z, the neighbour
// means and h_out are written only where the caller asks (training keeps
// them for the backward pass).
// Operands sit in shared memory chunk-major: chunk c (8 K-elements, 16 B)
// of row r at (c * rows + r) * 16, so one MMA (K = 16) reads chunks 2s and
// 2s+1 with SBO = 128 B and LBO = rows * 16 B.  fin is 40 or 64 (K = 80 or
// 128).  Staging: warp w fills rows 16w..16w+15, lane = (row 0..7, chunk
// group 0..3); the epilogue's warp w reads accumulator lanes 32(w%4).. and
// columns 32(w/4)...  Every wait is bounded; a wait that gives up sets bit 1
// of err, waits once more for the MMAs in flight and frees the tensor memory.
// CTAs per SM: three for the BF16 layers (80 registers), two for the
// first layer, whose FP32 input chunks need more registers
template <class TIn>
constexpr int tc_ctas_per_sm() {
  return sizeof(TIn) == 2 ? 3 : 2;
}

template <class TIn, bool HEAD>
__global__ void __launch_bounds__(TC_THREADS, tc_ctas_per_sm<TIn>())
k_layer_tc(int64_t nc, int fin, const TIn* __restrict__ h, const int32_t* __restrict__ off,
           const int32_t* __restrict__ nb, const __nv_bfloat16* __restrict__ ws,
           const __nv_bfloat16* __restrict__ wn, const __nv_bfloat16* __restrict__ bias,
           const __nv_bfloat16* __restrict__ wo, const __nv_bfloat16* __restrict__ bo,
           __nv_bfloat16* __restrict__ agg_out, float* __restrict__ z, __nv_bfloat16* __restrict__ hout,
           float* __restrict__ y, int32_t* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char tsm[];
  const TcSmem L = tc_smem(fin);
  const int nch = 2 * fin / 8, hch = fin / 8;
  unsigned char* sA = tsm + L.a;
  unsigned char* sB = tsm + L.b;
  unsigned char* sO = tsm + L.o;
  float* sY = reinterpret_cast<float*>(tsm + L.y);
  float* sWo = reinterpret_cast<float*>(tsm + L.wo);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(tsm + L.bar);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(tsm + L.slot);
  float* sbias = reinterpret_cast<float*>(tsm + L.bias);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // B = [Ws | Wn]: row j (output feature), chunk c of 8 elements
  for (int idx = tid; idx < W * nch; idx += TC_THREADS) {
    const int j = idx / nch, c = idx - nch * (idx / nch);
    const __nv_bfloat16* src = c < hch ? ws + j * fin + 8 * c : wn + j * fin + 8 * (c - hch);
    *reinterpret_cast<uint4*>(sB + (size_t(c) * W + j) * 16) = *reinterpret_cast<const uint4*>(src);
  }
  if (tid < W) sbias[tid] = __bfloat162float(bias[tid]);
  if (HEAD) {
    for (int i = tid; i < NOUT * W; i += TC_THREADS) sWo[i] = __bfloat162float(wo[i]);
    if (tid < NOUT) sWo[NOUT * W + tid] = __bfloat162float(bo[tid]);
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(uint32_t(TC_COLS))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init1(mbar);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  uint32_t phase = 0;
  bool ok = true, pending = false;
  const int64_t ntiles = (nc + TC_ROWS - 1) / TC_ROWS;
  const int rs = lane & 7, cg = lane >> 3;     // staging: row within 8, chunk group
  const int q = warp & 3, hf = warp >> 2;      // epilogue: lane quarter, column half
  constexpr int CPI = 1;  // chunks of a row gathered together
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t row0 = t * TC_ROWS;
    // ---- stage A = [h | neighbour mean] for rows 16 warp .. 16 warp + 15.
    // The row bounds and the first NB_FAST neighbour ids of both rows are
    // loaded first, then every chunk of a row at once, so that each lane has
    // up to 2 (NB_FAST + 1) loads in flight.
    int32_t e0[2], e1[2], nbi[2][NB_FAST];
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      const int64_t cell = row0 + 16 * warp + 8 * p + rs;
      e0[p] = e1[p] = 0;
      if (cell < nc) {
        e0[p] = __ldg(off + cell);
        e1[p] = __ldg(off + cell + 1);
      }
    }
#pragma unroll
    for (int p = 0; p < 2; ++p)
#pragma unroll
      for (int k = 0; k < NB_FAST; ++k) nbi[p][k] = e0[p] + k < e1[p] ? __ldg(nb + e0[p] + k) : -1;
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      const int r = 16 * warp + 8 * p + rs;
      const int64_t cell = row0 + r;
      if (cell < nc) {
        const float inv = e1[p] > e0[p] ? 1.0f / float(e1[p] - e0[p]) : 0.f;
#pragma unroll 1
        for (int c = cg; c < hch; c += 4 * CPI) {
          // chunks c + 4 i, i < CPI, of the row and of its neighbours
          Chunk8<TIn> own[CPI], u[NB_FAST][CPI];
#pragma unroll
          for (int i = 0; i < CPI; ++i)
            if (c + 4 * i < hch) own[i].load(h + cell * fin + 8 * (c + 4 * i));
#pragma unroll
          for (int k = 0; k < NB_FAST; ++k)
#pragma unroll
            for (int i = 0; i < CPI; ++i)
              if (nbi[p][k] >= 0 && c + 4 * i < hch) u[k][i].load(h + int64_t(nbi[p][k]) * fin + 8 * (c + 4 * i));
#pragma unroll
          for (int i = 0; i < CPI; ++i) {
            const int ci = c + 4 * i;
            if (ci >= hch) break;
            float v[8], sum[8];
            own[i].get(v);
            *reinterpret_cast<uint4*>(sA + (size_t(ci) * TC_ROWS + r) * 16) = pack8(v);
#pragma unroll
            for (int q8 = 0; q8 < 8; ++q8) sum[q8] = 0.f;
#pragma unroll
            for (int k = 0; k < NB_FAST; ++k)
              if (nbi[p][k] >= 0) {
                u[k][i].get(v);
#pragma unroll
                for (int q8 = 0; q8 < 8; ++q8) sum[q8] += as_input<TIn>(v[q8]);
              }
            for (int32_t e = e0[p] + NB_FAST; e < e1[p]; ++e) {  // cells with many neighbours
              Chunk8<TIn> x;
              x.load(h + int64_t(__ldg(nb + e)) * fin + 8 * ci);
              x.get(v);
#pragma unroll
              for (int q8 = 0; q8 < 8; ++q8) sum[q8] += as_input<TIn>(v[q8]);
            }
#pragma unroll
            for (int q8 = 0; q8 < 8; ++q8) sum[q8] *= inv;
            const uint4 m = pack8(sum);
            *reinterpret_cast<uint4*>(sA + (size_t(hch + ci) * TC_ROWS + r) * 16) = m;
            if (agg_out) *reinterpret_cast<uint4*>(agg_out + cell * fin + 8 * ci) = m;
          }
        }
      } else {
        for (int c = cg; c < nch; c += 4)
          *reinterpret_cast<uint4*>(sA + (size_t(c) * TC_ROWS + r) * 16) = make_uint4(0, 0, 0, 0);
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // ---- z = A B^T on the tensor cores
    if (tid == 0) {
      for (int st = 0; st < nch / 2; ++st) {
        const uint64_t ad = umma_desc(sA + size_t(2 * st) * TC_ROWS * 16, TC_ROWS * 16, 128);
        const uint64_t bd = umma_desc(sB + size_t(2 * st) * W * 16, W * 16, 128);
        umma_bf16(tmem, ad, bd, st > 0 ? 1u : 0u);
      }
      umma_commit(mbar);
    }
    pending = true;
    __syncwarp();
    // warp 0 polls the barrier, the others wait at the thread barrier
    const bool got = warp == 0 ? mbar_wait_bounded(mbar, phase) : true;
    ok = __syncthreads_and(got) != 0;
    if (!ok) break;
    pending = false;
    phase ^= 1u;
    tc_fence_after();
    // ---- epilogue: row 32 q + lane, columns 32 hf .. 32 hf + 31
    const int r = 32 * q + lane;
    const int64_t cell = row0 + r;
    float v[32];
    tmem_ld32(tmem + (uint32_t(32 * q) << 16) + uint32_t(32 * hf), v);
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] += sbias[32 * hf + j];
    if (z && cell < nc) {
      float4* zo = reinterpret_cast<float4*>(z + cell * W + 32 * hf);
#pragma unroll
      for (int j = 0; j < 8; ++j) zo[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
    }
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __bfloat162float(__float2bfloat16_rn(gelu(v[j])));
    if (hout) {
#pragma unroll
      for (int j = 0; j < 4; ++j)
        *reinterpret_cast<uint4*>(sO + size_t(r) * TC_OSTRIDE + 64 * hf + 16 * j) = pack8(v + 8 * j);
    }
    if (HEAD) {
      float yp[NOUT];
#pragma unroll
      for (int k = 0; k < NOUT; ++k) {
        float s = 0.f;
#pragma unroll
        for (int j = 0; j < 32; ++j) s += sWo[k * W + 32 * hf + j] * v[j];
        yp[k] = s;
      }
      if (hf == 1)
#pragma unroll
        for (int k = 0; k < NOUT; ++k) sY[r * 8 + k] = yp[k];
      __syncthreads();
      if (hf == 0 && cell < nc)
#pragma unroll
        for (int k = 0; k < NOUT; ++k) y[cell * NOUT + k] = (yp[k] + sY[r * 8 + k]) + sWo[NOUT * W + k];
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // ---- coalesced copy of the BF16 output tile
    if (hout) {
      const int64_t nrow = nc - row0 < TC_ROWS ? nc - row0 : int64_t(TC_ROWS);
      for (int idx = tid; idx < TC_ROWS * 8; idx += TC_THREADS) {
        const int rr = idx >> 3, c16 = idx & 7;
        if (rr < nrow)
          *reinterpret_cast<uint4*>(hout + (row0 + rr) * W + 8 * c16) =
              *reinterpret_cast<const uint4*>(sO + size_t(rr) * TC_OSTRIDE + 16 * c16);
      }
    }
    // sO is rewritten only after the next tile's staging barrier
  }
  if (!ok) {
    if (tid == 0) atomicOr(err, 2);
    if (pending && warp == 0) mbar_wait_bounded(mbar, phase);  // let the MMAs in flight finish
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(uint32_t(TC_COLS))
                 : "memory");
}

// ---- inference layer, warp-specialised ------------------------------------
// The same layer as k_layer_tc (A = [h | neighbour mean] in BF16, z = A
// [Ws | Wn]^T + b on the tensor cores, GELU, BF16 out; the last layer also
// the head), with the roles split and two tiles in flight:
//   warps 0..WS_PROD-1   gather A of tile k into shared buffer k % 2;
//   warp WS_PROD         one thread issues the tile's MMAs into tensor-memory
//                        accumulator k % 2 and commits them;
//   warps WS_PROD+1..+4  read accumulator k % 2 (one lane quarter each), apply
//                        bias and GELU and store the tile (or the head).
// Hand-offs are mbarriers: full[b] (gatherers -> MMA), done[b] (MMA
// completion -> epilogue, and -> gatherers: buffer b may be refilled),
// tfree[b] (epilogue has read accumulator b -> MMA may overwrite it).  A
// phase of done[b] cannot complete twice before both of its waiters saw it,
// because the next MMA on b needs both of them first.  Every wait is
// bounded: a wait that gives up sets the CTA's abort flag and bit 1 of err,
// every role then leaves its loop, the MMA thread lets its last commits
// land (bounded) and the tensor memory is freed.
constexpr int WS_PROD = 8;                         // gathering warps, 16 rows each
constexpr int WS_EPI = 4;                          // epilogue warps
constexpr int WS_THREADS = 32 * (WS_PROD + 1 + WS_EPI);
constexpr int WS_NB = 4;                           // neighbour rows per cell in flight
// Bytes between the K-chunk blocks of an A tile: the 128 rows' 16 B units
// of one chunk plus 32 B, so that chunk c starts 2c units (of 16 B) further
// round the 8 bank groups.  A quarter warp of gathering lanes holds chunks
// qc + 4i of two rows r, r + 1, whose units then fall into the 8 groups
// (2 qc + r) mod 8 once each: conflict-free stores.  The MMA reads the skew
// through its descriptor's K-chunk step (LBO).
constexpr int WS_ACH = TC_ROWS * 16 + 32;

struct WsSmem {
  size_t a0, a1, b, o, wo, bias, bar, slot, abort, total;
};
__host__ __device__ inline WsSmem ws_smem(int fin) {
  const size_t nch = size_t(2 * fin / 8);
  WsSmem s;
  s.a0 = 0;
  s.a1 = s.a0 + nch * WS_ACH;
  s.b = s.a1 + nch * WS_ACH;
  s.o = s.b + nch * W * 16;
  s.wo = s.o + size_t(WS_EPI) * 32 * TC_OSTRIDE;
  s.bias = s.wo + size_t(NOUT * W + 8) * sizeof(float);
  s.bar = s.bias + W * sizeof(float);
  s.slot = s.bar + 6 * 8;
  s.abort = s.slot + 8;
  s.total = s.abort + 8;
  return s;
}

__device__ __forceinline__ void mbar_init_n(uint64_t* bar, uint32_t n) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(n) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

template <bool HEAD>
__global__ void __launch_bounds__(WS_THREADS, 2)
k_layer_ws(int64_t nc, int fin, const __nv_bfloat16* __restrict__ h, const int32_t* __restrict__ ell,
           int K, const __nv_bfloat16* __restrict__ ws,
           const __nv_bfloat16* __restrict__ wn, const __nv_bfloat16* __restrict__ bias,
           const __nv_bfloat16* __restrict__ wo, const __nv_bfloat16* __restrict__ bo,
           __nv_bfloat16* __restrict__ hout, float* __restrict__ y, int32_t* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char wsm[];
  const WsSmem L = ws_smem(fin);
  const int nch = 2 * fin / 8, hch = fin / 8;
  unsigned char* sA[2] = {wsm + L.a0, wsm + L.a1};
  unsigned char* sB = wsm + L.b;
  float* sWo = reinterpret_cast<float*>(wsm + L.wo);
  float* sbias = reinterpret_cast<float*>(wsm + L.bias);
  uint64_t* bar = reinterpret_cast<uint64_t*>(wsm + L.bar);  // full[2], done[2], tfree[2]
  uint64_t *full = bar, *done = bar + 2, *tfree = bar + 4;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(wsm + L.slot);
  volatile int32_t* abort_flag = reinterpret_cast<volatile int32_t*>(wsm + L.abort);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  for (int idx = tid; idx < W * nch; idx += WS_THREADS) {
    const int j = idx / nch, c = idx - nch * (idx / nch);
    const __nv_bfloat16* src = c < hch ? ws + j * fin + 8 * c : wn + j * fin + 8 * (c - hch);
    *reinterpret_cast<uint4*>(sB + (size_t(c) * W + j) * 16) = *reinterpret_cast<const uint4*>(src);
  }
  if (tid < W) sbias[tid] = __bfloat162float(bias[tid]);
  if (HEAD) {
    for (int i = tid; i < NOUT * W; i += WS_THREADS) sWo[i] = __bfloat162float(wo[i]);
    if (tid < NOUT) sWo[NOUT * W + tid] = __bfloat162float(bo[tid]);
  }
  if (warp == WS_PROD) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(uint32_t(2 * TC_COLS))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int b = 0; b < 2; ++b) {
      mbar_init_n(full + b, 32 * WS_PROD);
      mbar_init_n(done + b, 1);
      mbar_init_n(tfree + b, 32 * WS_EPI);
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const int64_t ntiles = (nc + TC_ROWS - 1) / TC_ROWS;
  auto give_up = [&]() {
    *abort_flag = 1;
    atomicOr(err, 2);
  };

  if (warp < WS_PROD) {
    // ---- gather: warp w fills rows 16 w .. 16 w + 15, eight rows at a
    // time; lane = 4 row slot (0..7) + quarter holds chunks quarter and
    // quarter + 4 of its row and of the row's first WS_NB neighbours, all
    // loading at once: four consecutive lanes read 64 contiguous bytes of a
    // row, which costs the L1 less than eight lanes on eight rows (measured:
    // 314 against 389 us a layer at 64^3 x 6); the A tile's skewed chunk
    // blocks (WS_ACH) keep this mapping's stores free of bank conflicts.  The
    // neighbours come from the entry-major lists in the cell's face order
    // (boundary entries are -1 and skipped), so the mean sums them in the
    // order of the face graph.
    const int sl = lane >> 2, qc = lane & 3;
    int k = 0;
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x, ++k) {
      const int b = k & 1;
      if (k >= 2 && !mbar_wait_bounded(done + b, uint32_t(((k >> 1) - 1) & 1))) give_up();
      if (*abort_flag) break;
      unsigned char* A = sA[b];
#pragma unroll 1
      for (int g = 0; g < 2; ++g) {
        const int r = 16 * warp + 8 * g + sl;
        const int64_t cell = t * TC_ROWS + r;
        int32_t nbi[WS_NB];
#pragma unroll
        for (int j = 0; j < WS_NB; ++j) nbi[j] = cell < nc && j < K ? __ldg(ell + j * nc + cell) : -1;
        if (cell >= nc) {
          for (int c = qc; c < nch; c += 4)
            *reinterpret_cast<uint4*>(A + size_t(c) * WS_ACH + size_t(r) * 16) = make_uint4(0, 0, 0, 0);
          continue;
        }
        int deg = 0;
#pragma unroll
        for (int j = 0; j < WS_NB; ++j) deg += nbi[j] >= 0;
        for (int j = WS_NB; j < K; ++j) deg += __ldg(ell + j * nc + cell) >= 0;
        const float inv = deg > 0 ? 1.0f / float(deg) : 0.f;
        for (int c0 = qc; c0 < hch; c0 += 8) {
          // chunks c0 and c0 + 4 of the row and of its neighbours
          Chunk8<__nv_bfloat16> own[2], u[2][WS_NB];
#pragma unroll
          for (int i = 0; i < 2; ++i) {
            const int c = c0 + 4 * i;
            if (c < hch) {
              own[i].load(h + cell * fin + 8 * c);
#pragma unroll
              for (int j = 0; j < WS_NB; ++j)
                if (nbi[j] >= 0) u[i][j].load(h + int64_t(nbi[j]) * fin + 8 * c);
            }
          }
#pragma unroll
          for (int i = 0; i < 2; ++i) {
            const int c = c0 + 4 * i;
            if (c >= hch) break;
            float v[8], sum[8];
            own[i].get(v);
            *reinterpret_cast<uint4*>(A + size_t(c) * WS_ACH + size_t(r) * 16) = pack8(v);
#pragma unroll
            for (int q8 = 0; q8 < 8; ++q8) sum[q8] = 0.f;
#pragma unroll
            for (int j = 0; j < WS_NB; ++j)
              if (nbi[j] >= 0) {
                u[i][j].get(v);
#pragma unroll
                for (int q8 = 0; q8 < 8; ++q8) sum[q8] += v[q8];
              }
            for (int j = WS_NB; j < K; ++j) {  // cells with more faces
              const int32_t o = __ldg(ell + j * nc + cell);
              if (o < 0) continue;
              Chunk8<__nv_bfloat16> x;
              x.load(h + int64_t(o) * fin + 8 * c);
              x.get(v);
#pragma unroll
              for (int q8 = 0; q8 < 8; ++q8) sum[q8] += v[q8];
            }
#pragma unroll
            for (int q8 = 0; q8 < 8; ++q8) sum[q8] *= inv;
            *reinterpret_cast<uint4*>(A + size_t(hch + c) * WS_ACH + size_t(r) * 16) = pack8(sum);
          }
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(full + b);
    }
  } else if (warp == WS_PROD) {
    // ---- MMA issue (one thread)
    int k = 0;
    int last[2] = {-1, -1};  // last tile index committed on each accumulator
    if (lane == 0) {
      for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x, ++k) {
        const int b = k & 1;
        if (!mbar_wait_bounded(full + b, uint32_t((k >> 1) & 1))) give_up();
        if (!*abort_flag && k >= 2 && !mbar_wait_bounded(tfree + b, uint32_t(((k >> 1) - 1) & 1)))
          give_up();
        if (*abort_flag) break;
        tc_fence_after();
        for (int st = 0; st < nch / 2; ++st) {
          const uint64_t ad = umma_desc(sA[b] + size_t(2 * st) * WS_ACH, WS_ACH, 128);
          const uint64_t bd = umma_desc(sB + size_t(2 * st) * W * 16, W * 16, 128);
          umma_bf16(tmem + uint32_t(TC_COLS * b), ad, bd, st > 0 ? 1u : 0u);
        }
        umma_commit(done + b);
        last[b] = k;
      }
      // let every committed MMA land before the tensor memory is freed
      for (int b = 0; b < 2; ++b)
        if (last[b] >= 0) mbar_wait_bounded(done + b, uint32_t((last[b] >> 1) & 1));
    }
    __syncwarp();
  } else {
    // ---- epilogue: warp quarter q holds accumulator lanes 32 q .. 32 q + 31
    const int ew = warp - WS_PROD - 1;
    const int q = warp & 3;
    unsigned char* sO = wsm + L.o + size_t(ew) * 32 * TC_OSTRIDE;
    int k = 0;
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x, ++k) {
      const int b = k & 1;
      if (!mbar_wait_bounded(done + b, uint32_t((k >> 1) & 1))) give_up();
      if (*abort_flag) break;
      tc_fence_after();
      // the accumulator's two 32-column halves in turn (fewer registers:
      // two CTAs share an SM); it is released after the second is read
      const uint32_t ta = tmem + (uint32_t(32 * q) << 16) + uint32_t(TC_COLS * b);
      const int64_t cell = t * TC_ROWS + 32 * q + lane;
      float ys[2][NOUT];
#pragma unroll
      for (int hf = 0; hf < 2; ++hf) {
        float v[32];
        tmem_ld32(ta + 32 * hf, v);
        if (hf == 1) {
          tc_fence_before();
          mbar_arrive(tfree + b);
        }
        // bias and head weights are read as 16 B vectors (one shared load
        // per four values, the same address in every lane)
        const float4* b4 = reinterpret_cast<const float4*>(sbias + 32 * hf);
#pragma unroll
        for (int j4 = 0; j4 < 8; ++j4) {
          const float4 bb = b4[j4];
          v[4 * j4] = __bfloat162float(__float2bfloat16_rn(gelu(v[4 * j4] + bb.x)));
          v[4 * j4 + 1] = __bfloat162float(__float2bfloat16_rn(gelu(v[4 * j4 + 1] + bb.y)));
          v[4 * j4 + 2] = __bfloat162float(__float2bfloat16_rn(gelu(v[4 * j4 + 2] + bb.z)));
          v[4 * j4 + 3] = __bfloat162float(__float2bfloat16_rn(gelu(v[4 * j4 + 3] + bb.w)));
        }
        if (HEAD) {
#pragma unroll
          for (int o = 0; o < NOUT; ++o) {
            const float4* w4 = reinterpret_cast<const float4*>(sWo + o * W + 32 * hf);
            float sacc = 0.f;
#pragma unroll
            for (int j4 = 0; j4 < 8; ++j4) {
              const float4 ww = w4[j4];
              sacc += ww.x * v[4 * j4];
              sacc += ww.y * v[4 * j4 + 1];
              sacc += ww.z * v[4 * j4 + 2];
              sacc += ww.w * v[4 * j4 + 3];
            }
            ys[hf][o] = sacc;
          }
        } else {
#pragma unroll
          for (int j = 0; j < 4; ++j)
            *reinterpret_cast<uint4*>(sO + size_t(lane) * TC_OSTRIDE + 64 * hf + 16 * j) = pack8(v + 8 * j);
        }
      }
      if (HEAD) {
        if (cell < nc)
#pragma unroll
          for (int o = 0; o < NOUT; ++o) y[cell * NOUT + o] = (ys[0][o] + ys[1][o]) + sWo[NOUT * W + o];
      } else {
        __syncwarp();
        const int64_t row0 = t * TC_ROWS + 32 * q;
        for (int idx = lane; idx < 32 * 8; idx += 32) {
          const int rr = idx >> 3, c16 = idx & 7;
          if (row0 + rr < nc)
            *reinterpret_cast<uint4*>(hout + (row0 + rr) * W + 8 * c16) =
                *reinterpret_cast<const uint4*>(sO + size_t(rr) * TC_OSTRIDE + 16 * c16);
        }
        __syncwarp();
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == WS_PROD)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(uint32_t(2 * TC_COLS))
                 : "memory");
}

// batch membership: a counter-based hash of (seed, cell) below the threshold
__device__ __forceinline__ bool in_batch(uint64_t seed, int64_t c, uint64_t thr) {
  uint64_t x = seed * 0x9E3779B97F4A7C15ull + uint64_t(c) + 0x632BE59BD9B4E019ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  x ^= x >> 31;
  return x <= thr;
}

// dy = 2 (y - t) / (5 n_batch) on the batch, 0 elsewhere; block partials of
// the squared error and of the batch count
__global__ void __launch_bounds__(GT) k_loss(int64_t nc, const float* __restrict__ y,
                                             const float* __restrict__ t, uint64_t seed, uint64_t thr,
                                             const float* __restrict__ mask, float* __restrict__ dy,
                                             double* __restrict__ part) {
  const int64_t c = int64_t(blockIdx.x) * GT + threadIdx.x;
  double se = 0, cnt = 0;
  if (c < nc) {
    const bool m = in_batch(seed, c, thr) && (!mask || mask[c] > 0.f);
#pragma unroll
    for (int k = 0; k < NOUT; ++k) {
      const float d = y[c * NOUT + k] - t[c * NOUT + k];
      dy[c * NOUT + k] = m ? d : 0.f;  // scaled later by 2/(5 n)
      if (m) se += double(d) * double(d);
    }
    cnt = m ? 1.0 : 0.0;
  }
  __shared__ double s1[GT], s2[GT];
  s1[threadIdx.x] = se, s2[threadIdx.x] = cnt;
  __syncthreads();
  for (int st = GT / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) s1[threadIdx.x] += s1[threadIdx.x + st], s2[threadIdx.x] += s2[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[2 * blockIdx.x] = s1[0], part[2 * blockIdx.x + 1] = s2[0];
}

__global__ void k_scale(int64_t n, float* __restrict__ a, const double* __restrict__ loss_cnt) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double cnt = loss_cnt[1];
  a[i] = float(double(a[i]) * (cnt > 0 ? 2.0 / (5.0 * cnt) : 0.0));
}

// sum of the loss partials: out[0] = mean squared error, out[1] = batch size
__global__ void k_loss_final(const double* __restrict__ part, int nblk, double* __restrict__ out) {
  __shared__ double s1[256], s2[256];
  double a = 0, b = 0;
  for (int i = threadIdx.x; i < nblk; i += 256) a += part[2 * i], b += part[2 * i + 1];
  s1[threadIdx.x] = a, s2[threadIdx.x] = b;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st) s1[threadIdx.x] += s1[threadIdx.x + st], s2[threadIdx.x] += s2[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = s2[0] > 0 ? s1[0] / (5.0 * s2[0]) : 0.0;
    out[1] = s2[0];
  }
}

// weight-gradient partials over blocks of RB cells:
// part[blk][j][i] = sum_c dz[c][j] * a[c][i]   (a = h or agg, as the forward
// GEMM used it), and bias sums
constexpr int RB = 256;
template <class TA>
__global__ void k_wgrad_partial(int64_t nc, int nout, int fin, const float* __restrict__ dz,
                                const TA* __restrict__ a, float* __restrict__ part) {
  const int64_t c0 = int64_t(blockIdx.x) * RB;
  const int64_t c1 = min(nc, c0 + RB);
  float* o = part + int64_t(blockIdx.x) * nout * (fin + 1);
  for (int w = threadIdx.x; w < nout * (fin + 1); w += blockDim.x) {
    const int j = w / (fin + 1), i = w % (fin + 1);
    float s = 0.f;
    if (i < fin) {
      for (int64_t c = c0; c < c1; ++c) s += dz[c * nout + j] * as_operand(a[c * fin + i]);
    } else {
      for (int64_t c = c0; c < c1; ++c) s += dz[c * nout + j];
    }
    o[w] = s;
  }
}
// g[wofs + j*fin + i] (and g[bofs + j] when bofs >= 0) = sum over blocks
__global__ void k_wgrad_reduce(int nblk, int nout, int fin, const float* __restrict__ part,
                               float* __restrict__ g, int64_t wofs, int64_t bofs) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nout * (fin + 1)) return;
  const int j = w / (fin + 1), i = w % (fin + 1);
  double s = 0;
  for (int b = 0; b < nblk; ++b) s += part[int64_t(b) * nout * (fin + 1) + w];
  if (i < fin)
    g[wofs + j * fin + i] = float(s);
  else if (bofs >= 0)
    g[bofs + j] = float(s);
}

// dh[c][i] = sum_j W[j][i] dz[c][j]   (W: nout x fin, bf16)
__global__ void __launch_bounds__(GT) k_back_dense(int64_t nc, int nout, int fin,
                                                   const __nv_bfloat16* __restrict__ w,
                                                   const float* __restrict__ dz,
                                                   float* __restrict__ dh) {
  __shared__ float sw[W * W];
  for (int i = threadIdx.x; i < nout * fin; i += GT) sw[i] = __bfloat162float(w[i]);
  __syncthreads();
  const int64_t c = int64_t(blockIdx.x) * GT + threadIdx.x;
  if (c >= nc) return;
  for (int i0 = 0; i0 < fin; i0 += 16) {
    float acc[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) acc[i] = 0.f;
    for (int j = 0; j < nout; ++j) {
      const float d = dz[c * nout + j];
#pragma unroll
      for (int i = 0; i < 16; ++i)
        if (i0 + i < fin) acc[i] += sw[j * fin + i0 + i] * d;
    }
#pragma unroll
    for (int i = 0; i < 16; ++i)
      if (i0 + i < fin) dh[c * fin + i0 + i] = acc[i];
  }
}

// dh[n] += sum_{c in N(n)} dagg[c] / deg(c)  (the graph is symmetric)
__global__ void k_back_aggregate(int64_t nc, int fin, const int32_t* __restrict__ off,
                                 const int32_t* __restrict__ nb, const float* __restrict__ dagg,
                                 float* __restrict__ dh) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= nc * fin) return;
  const int64_t n = i / fin;
  const int k = int(i % fin);
  float s = 0.f;
  for (int32_t e = off[n]; e < off[n + 1]; ++e) {
    const int32_t c = nb[e];
    const int32_t deg = off[c + 1] - off[c];
    s += dagg[int64_t(c) * fin + k] / float(deg);
  }
  dh[i] += s;
}

// dz = dh * GELU'(z)
__global__ void k_back_gelu(int64_t n, const float* __restrict__ dh, const float* __restrict__ z,
                            float* __restrict__ dz) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) dz[i] = dh[i] * gelu_grad(z[i]);
}

__global__ void k_adam(int64_t n, float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ g, __nv_bfloat16* __restrict__ wb, float lr,
                       float b1, float b2, float eps, float c1, float c2) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi, v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  wb[i] = __float2bfloat16_rn(wi);
}

__global__ void k_to_bf16(int64_t n, const float* __restrict__ w, __nv_bfloat16* __restrict__ wb) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) wb[i] = __float2bfloat16_rn(w[i]);
}

constexpr int FCB = 128;  // cells per block of the feature kernels

// features of one assembled system (RCM order): B = float(src), D, x_J
// gathered from the colour-order iterate right after assembly, dq_prev from
// the colour-order copy of the last update (null: zero)
template <class TB, class TX>
__global__ void k_features_raw(int64_t nc, const double* __restrict__ src, const TB* __restrict__ D,
                               const TX* __restrict__ xj_ci, const TX* __restrict__ xprev_ci,
                               const int32_t* __restrict__ ci,
                               float* __restrict__ raw /* [nc][40]: B, D, zero, dq_prev */,
                               float* __restrict__ xj) {
  // a block per FCB cells, a thread per 4 feature elements (float4 stores;
  // 40 = 10 x 4, so a float4 never straddles two cells), unrolled so that
  // each thread has several loads in flight
  const int64_t c0 = int64_t(blockIdx.x) * FCB;
  const int ncb = int(nc - c0 < FCB ? nc - c0 : FCB);
  float4* raw4 = reinterpret_cast<float4*>(raw + c0 * NIN);
#pragma unroll 5
  for (int j = threadIdx.x; j < ncb * (NIN / 4); j += blockDim.x) {
    const int cl = j / (NIN / 4), k0 = 4 * (j - (NIN / 4) * cl);
    const int64_t c = c0 + cl;
    float v[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int k = k0 + e;
      v[e] = 0.f;
      if (k < 5)
        v[e] = float(src[5 * c + k]);
      else if (k < 30)
        v[e] = float(D[25 * c + k - 5]);
      else if (k >= 35 && xprev_ci)
        v[e] = float(xprev_ci[5 * int64_t(ci[c]) + k - 35]);
    }
    raw4[j] = make_float4(v[0], v[1], v[2], v[3]);
  }
  for (int j = threadIdx.x; j < ncb * 5; j += blockDim.x) {
    const int cl = j / 5, k = j - 5 * cl;
    xj[c0 * 5 + j] = float(xj_ci[5 * int64_t(ci[c0 + cl]) + k]);
  }
}

// per-component sums of squares of B (raw[:,0:5]) and x_J, block partials
__global__ void k_rms_partial(int64_t nc, const float* __restrict__ raw, const float* __restrict__ xj,
                              double* __restrict__ part) {
  const int64_t c = int64_t(blockIdx.x) * GT + threadIdx.x;
  __shared__ double sh[10][GT];
  for (int k = 0; k < 5; ++k) {
    const double b = c < nc ? double(raw[c * NIN + k]) : 0.0;
    const double x = c < nc ? double(xj[c * 5 + k]) : 0.0;
    sh[k][threadIdx.x] = b * b;
    sh[5 + k][threadIdx.x] = x * x;
  }
  __syncthreads();
  for (int st = GT / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int k = 0; k < 10; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 10; ++k) part[10 * blockIdx.x + k] = sh[k][0];
}

// Scales rs, xs from the per-block sums of squares, and the 40 per-feature
// factors of k_features_norm, in one block: thread t sums blocks t, t + T,
// ... in order, then a fixed tree combines the threads, so the scales are
// the same on every call for the same system (training features and
// inference features use this one kernel).  fac[0..9] = rs|xs,
// fac[10..49] the factors.
constexpr int FS_THREADS = 512;
__global__ void __launch_bounds__(FS_THREADS) k_feat_scales(const double* __restrict__ part, int nblk,
                                                         int64_t nc, float* __restrict__ fac) {
  __shared__ double sh[10][FS_THREADS];
  __shared__ float scl[10];
  const int t = threadIdx.x;
  double a[10];
#pragma unroll
  for (int k = 0; k < 10; ++k) a[k] = 0.0;
  for (int b = t; b < nblk; b += FS_THREADS) {
#pragma unroll
    for (int k = 0; k < 10; ++k) a[k] += part[10 * int64_t(b) + k];
  }
#pragma unroll
  for (int k = 0; k < 10; ++k) sh[k][t] = a[k];
  __syncthreads();
  for (int st = FS_THREADS / 2; st > 0; st >>= 1) {
    if (t < st)
#pragma unroll
      for (int k = 0; k < 10; ++k) sh[k][t] += sh[k][t + st];
    __syncthreads();
  }
  if (t < 10) {
    scl[t] = float(sqrt(sh[t][0] / double(nc)) + 1e-30);
    fac[t] = scl[t];
  }
  __syncthreads();
  if (t < NIN) {
    const float* rs = scl;
    const float* xs = scl + 5;
    float f;
    if (t < 5)
      f = 1.0f / rs[t];
    else if (t < 30)
      f = xs[(t - 5) % 5] / rs[(t - 5) / 5];
    else if (t < 35)
      f = 1.0f / xs[t - 30];
    else
      f = 1.0f / xs[t - 35];
    fac[10 + t] = f;
  }
}

// normalise: B/rs, D_ij xs_j / rs_i, x_J/xs, dq_prev/xs, each as one// normalise: B/rs, D_ij xs_j / rs_i, x_J/xs, dq_prev/xs, each as one
// multiplication by a per-feature factor (feature 30..34 read from x_J)
__global__ void k_features_norm(int64_t nc, const float* __restrict__ raw, const float* __restrict__ xj,
                                const float* __restrict__ scl /*rs[5],xs[5]*/, float* __restrict__ feat) {
  // a block per FCB cells, a thread per 4 feature elements (float4 loads
  // and stores), unrolled so that each thread has several loads in flight;
  // no branch depends on the feature index
  const int64_t c0 = int64_t(blockIdx.x) * FCB;
  const int ncb = int(nc - c0 < FCB ? nc - c0 : FCB);
  __shared__ float fac[NIN];
  if (threadIdx.x < NIN) {
    const int k = threadIdx.x;
    const float* rs = scl;
    const float* xs = scl + 5;
    float f;
    if (k < 5)
      f = 1.0f / rs[k];
    else if (k < 30)
      f = xs[(k - 5) % 5] / rs[(k - 5) / 5];
    else if (k < 35)
      f = 1.0f / xs[k - 30];
    else
      f = 1.0f / xs[k - 35];
    fac[k] = f;
  }
  __syncthreads();
  const float4* raw4 = reinterpret_cast<const float4*>(raw + c0 * NIN);
  float4* feat4 = reinterpret_cast<float4*>(feat + c0 * NIN);
#pragma unroll 5
  for (int j = threadIdx.x; j < ncb * (NIN / 4); j += blockDim.x) {
    const int cl = j / (NIN / 4), k0 = 4 * (j - (NIN / 4) * cl);
    const float4 r4 = raw4[j];
    float v[4] = {r4.x, r4.y, r4.z, r4.w};
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int k = k0 + e;
      if (k >= 30 && k < 35) v[e] = xj[(c0 + cl) * 5 + k - 30];
      v[e] *= fac[k];
    }
    feat4[j] = make_float4(v[0], v[1], v[2], v[3]);
  }
}

inline unsigned nb_(int64_t n, int t) { return unsigned((n + t - 1) / t); }


// forward over the whole graph from features; returns head output in
// m->d_y.  keep stores what the backward pass needs: neighbour means, FP32
// pre-activations and every layer's activations.
static_assert(NLAYER >= 2, "the head is fused into the last hidden layer");
// feat16 (BF16 [nc][40], inference): used instead of feat by the first
// layer, which rounds every input row to BF16 anyway (its own and each
// neighbour's before their mean), so the result is the same
int forward(fpsi_gnn* m, const Graph& G, const float* feat, bool keep,
            const __nv_bfloat16* feat16 = nullptr, cudaStream_t stream = nullptr) {
  cudaStream_t s = stream ? stream : m->stream;
  const int64_t nc = G.nc;
  const int64_t ntiles = (nc + TC_ROWS - 1) / TC_ROWS;
  if (!keep && feat16 && G.ell) {
    // inference: the warp-specialised layer, two CTAs per SM
    const unsigned gws = unsigned(std::max<int64_t>(1, std::min<int64_t>(ntiles, 2 * int64_t(m->nsm))));
    const __nv_bfloat16 *wo = m->d_wb + m->L.wo, *bo = m->d_wb + m->L.bo;
    for (int l = 0; l < NLAYER; ++l) {
      const int fin = m->L.fan_in[l];
      const size_t smem = ws_smem(fin).total;
      const __nv_bfloat16 *ws = m->d_wb + m->L.ws[l], *wn = m->d_wb + m->L.wn[l], *b = m->d_wb + m->L.b[l];
      const __nv_bfloat16* hin = l == 0 ? feat16 : m->d_h[l];
      if (l == NLAYER - 1)
        k_layer_ws<true><<<gws, WS_THREADS, smem, s>>>(nc, fin, hin, G.ell, G.K, ws, wn, b, wo, bo, nullptr,
                                                      m->d_y, m->d_err);
      else
        k_layer_ws<false><<<gws, WS_THREADS, smem, s>>>(nc, fin, hin, G.ell, G.K, ws, wn, b, wo, bo,
                                                       m->d_h[l + 1], nullptr, m->d_err);
    }
    FPSI_CUDA_TRY(cudaGetLastError());
    return FPSI_OK;
  }
  auto grid_for = [&](int per_sm) {
    return unsigned(std::max<int64_t>(1, std::min<int64_t>(ntiles, int64_t(per_sm) * m->nsm)));
  };
  const unsigned grid = grid_for(tc_ctas_per_sm<__nv_bfloat16>());
  const unsigned grid0 = grid_for(tc_ctas_per_sm<float>());
  const __nv_bfloat16 *wo = m->d_wb + m->L.wo, *bo = m->d_wb + m->L.bo;
  for (int l = 0; l < NLAYER; ++l) {
    const int fin = m->L.fan_in[l];
    const size_t smem = tc_smem(fin).total;
    const __nv_bfloat16 *ws = m->d_wb + m->L.ws[l], *wn = m->d_wb + m->L.wn[l], *b = m->d_wb + m->L.b[l];
    __nv_bfloat16* agg = keep ? m->d_agg[l] : nullptr;
    float* z = keep ? m->d_z[l] : nullptr;
    const bool last = l == NLAYER - 1;
    __nv_bfloat16* hout = (last && !keep) ? nullptr : m->d_h[l + 1];
    if (l == 0 && feat16)
      k_layer_tc<__nv_bfloat16, false><<<grid, TC_THREADS, smem, s>>>(nc, fin, feat16, G.off, G.nb, ws, wn, b,
                                                                      wo, bo, agg, z, hout, nullptr, m->d_err);
    else if (l == 0)
      k_layer_tc<float, false><<<grid0, TC_THREADS, smem, s>>>(nc, fin, feat, G.off, G.nb, ws, wn, b, wo, bo, agg,
                                                              z, hout, nullptr, m->d_err);
    else if (!last)
      k_layer_tc<__nv_bfloat16, false><<<grid, TC_THREADS, smem, s>>>(nc, fin, m->d_h[l], G.off, G.nb, ws, wn, b,
                                                                      wo, bo, agg, z, hout, nullptr, m->d_err);
    else
      k_layer_tc<__nv_bfloat16, true><<<grid, TC_THREADS, smem, s>>>(nc, fin, m->d_h[l], G.off, G.nb, ws, wn, b,
                                                                     wo, bo, agg, z, hout, m->d_y, m->d_err);
  }
  FPSI_CUDA_TRY(cudaGetLastError());
  return FPSI_OK;
}

// after the stream is synchronised: a tensor-core wait that gave up is an
// error of the pass (flag cleared for the next one)
int take_error(fpsi_gnn* m) {
  int32_t e = 0;
  FPSI_CUDA_TRY(cudaMemcpy(&e, m->d_err, sizeof(e), cudaMemcpyDeviceToHost));
  if (!e) return FPSI_OK;
  FPSI_CUDA_TRY(cudaMemset(m->d_err, 0, sizeof(int32_t)));
  fpsi::set_error("learned start: a tensor-core wait timed out");
  return FPSI_E_TIMEOUT;
}

// loss over the batch and full gradient into m->d_g; loss_out (device) [2]
int backward(fpsi_gnn* m, const Graph& G, const float* feat, const float* target, const float* mask,
             uint64_t seed, uint64_t thr, double* loss_out) {
  cudaStream_t s = m->stream;
  const int64_t nc = G.nc;
  const int nblk = int(nb_(nc, GT));
  float* dy = m->d_dz;  // [nc][5] fits in the [nc][64] buffer
  k_loss<<<nblk, GT, 0, s>>>(nc, m->d_y, target, seed, thr, mask, dy, m->d_lpart);
  k_loss_final<<<1, 256, 0, s>>>(m->d_lpart, nblk, loss_out);
  k_scale<<<nb_(nc * NOUT, 256), 256, 0, s>>>(nc * NOUT, dy, loss_out);
  const int rb = int(nb_(nc, RB));
  // head
  k_wgrad_partial<__nv_bfloat16><<<rb, 256, 0, s>>>(nc, NOUT, W, dy, m->d_h[NLAYER], m->d_part);
  k_wgrad_reduce<<<nb_(NOUT * (W + 1), 256), 256, 0, s>>>(rb, NOUT, W, m->d_part, m->d_g, m->L.wo, m->L.bo);
  k_back_dense<<<nb_(nc, GT), GT, 0, s>>>(nc, NOUT, W, m->d_wb + m->L.wo, dy, m->d_dh);
  for (int l = NLAYER - 1; l >= 0; --l) {
    const int fin = m->L.fan_in[l];
    k_back_gelu<<<nb_(nc * W, 256), 256, 0, s>>>(nc * W, m->d_dh, m->d_z[l], m->d_dz);
    if (l == 0)
      k_wgrad_partial<float><<<rb, 256, 0, s>>>(nc, W, fin, m->d_dz, feat, m->d_part);
    else
      k_wgrad_partial<__nv_bfloat16><<<rb, 256, 0, s>>>(nc, W, fin, m->d_dz, m->d_h[l], m->d_part);
    k_wgrad_reduce<<<nb_(W * (fin + 1), 256), 256, 0, s>>>(rb, W, fin, m->d_part, m->d_g, m->L.ws[l],
                                                          m->L.b[l]);
    k_wgrad_partial<__nv_bfloat16><<<rb, 256, 0, s>>>(nc, W, fin, m->d_dz, m->d_agg[l], m->d_part);
    k_wgrad_reduce<<<nb_(W * (fin + 1), 256), 256, 0, s>>>(rb, W, fin, m->d_part, m->d_g, m->L.wn[l], -1);
    if (l > 0) {
      // dh_in = Ws^T dz + scatter(Wn^T dz)
      k_back_dense<<<nb_(nc, GT), GT, 0, s>>>(nc, W, fin, m->d_wb + m->L.wn[l], m->d_dz, m->d_dagg);
      k_back_dense<<<nb_(nc, GT), GT, 0, s>>>(nc, W, fin, m->d_wb + m->L.ws[l], m->d_dz, m->d_dh2);
      k_back_aggregate<<<nb_(nc * fin, 256), 256, 0, s>>>(nc, fin, G.off, G.nb, m->d_dagg, m->d_dh2);
      std::swap(m->d_dh, m->d_dh2);
    }
  }
  FPSI_CUDA_TRY(cudaGetLastError());
  return FPSI_OK;
}

template <class T>
int galloc(T** p, size_t n) {
  if (cudaMalloc((void**)p, (n ? n : 1) * sizeof(T)) != cudaSuccess) {
    fpsi::set_error("cudaMalloc failed in the learned-start model");
    *p = nullptr;
    return FPSI_E_NOMEM;
  }
  return FPSI_OK;
}

void free_activations(fpsi_gnn* m) {
  void* ps[] = {m->d_y, m->d_dh, m->d_dh2, m->d_dz, m->d_dagg, m->d_part, m->d_lpart};
  for (void* p : ps)
    if (p) cudaFree(p);
  m->d_y = m->d_dh = m->d_dh2 = m->d_dz = m->d_dagg = m->d_part = nullptr;
  m->d_lpart = nullptr;
  for (int l = 0; l <= NLAYER; ++l) {
    if (m->d_h[l]) cudaFree(m->d_h[l]);
    m->d_h[l] = nullptr;
  }
  for (int l = 0; l < NLAYER; ++l) {
    if (m->d_agg[l]) cudaFree(m->d_agg[l]);
    if (m->d_z[l]) cudaFree(m->d_z[l]);
    m->d_agg[l] = nullptr;
    m->d_z[l] = nullptr;
  }
  m->cap = 0;
}

// activation buffers for graphs of up to nc cells
int ensure_capacity(fpsi_gnn* m, int64_t nc) {
  if (nc <= m->cap) return FPSI_OK;
  if (cudaStreamSynchronize(m->stream) != cudaSuccess) return FPSI_E_CUDA;
  free_activations(m);
  int rc = FPSI_OK;
#define G(e) \
  if (!rc) rc = (e)
  for (int l = 1; l <= NLAYER; ++l) G(galloc(&m->d_h[l], nc * W));
  for (int l = 0; l < NLAYER; ++l) {
    G(galloc(&m->d_agg[l], nc * W));
    G(galloc(&m->d_z[l], nc * W));
  }
  G(galloc(&m->d_y, nc * NOUT));
  G(galloc(&m->d_dh, nc * W));
  G(galloc(&m->d_dh2, nc * W));
  G(galloc(&m->d_dz, nc * W));
  G(galloc(&m->d_dagg, nc * W));
  G(galloc(&m->d_part, ((nc + RB - 1) / RB) * W * (W + 1)));
  G(galloc(&m->d_lpart, ((nc + GT - 1) / GT) * 10 + 16));
#undef G
  if (rc) {
    free_activations(m);
    return rc;
  }
  m->cap = nc;
  return FPSI_OK;
}

// the context's interior-face cell graph (RCM order), built on first use
int ctx_graph(fpsi_ctx* x, Graph* G) {
  const int64_t nc = x->H.nc;
  if (!x->d_cnb_off) {
    std::vector<int32_t> off(nc + 1, 0), nb;
    for (int64_t c = 0; c < nc; ++c) {
      for (int32_t e = x->H.cf_off[c]; e < x->H.cf_off[c + 1]; ++e) {
        const int64_t f = x->H.cf[e] >> 1;
        if (x->H.cr[f] < 0) continue;
        nb.push_back((x->H.cf[e] & 1) ? x->H.cl[f] : x->H.cr[f]);
      }
      off[c + 1] = int32_t(nb.size());
    }
    int rc = galloc(&x->d_cnb_off, off.size());
    if (!rc) rc = galloc(&x->d_cnb, nb.size());
    if (rc) {
      cudaFree(x->d_cnb_off), cudaFree(x->d_cnb);
      x->d_cnb_off = x->d_cnb = nullptr;
      return rc;
    }
    FPSI_CUDA_TRY(cudaMemcpy(x->d_cnb_off, off.data(), off.size() * 4, cudaMemcpyHostToDevice));
    if (!nb.empty())
      FPSI_CUDA_TRY(cudaMemcpy(x->d_cnb, nb.data(), nb.size() * 4, cudaMemcpyHostToDevice));
    x->cnb_n = int64_t(nb.size());
  }
  *G = Graph{nc, x->d_cnb_off, x->d_cnb, x->d_enb, x->H.ell_k};
  return FPSI_OK;
}

void free_snapshot(Snapshot& s) {
  void* ps[] = {s.d_off, s.d_nb, s.feat, s.target, s.xj, s.mask};
  for (void* p : ps)
    if (p) cudaFree(p);
  s.d_off = s.d_nb = nullptr;
  s.feat = s.target = s.xj = s.mask = nullptr;
}

}  // namespace

extern "C" {

int fpsi_gnn_create(fpsi_gnn** out, uint64_t seed) {
  if (!out) return FPSI_E_INVALID;
  *out = nullptr;
  fpsi_gnn* m = new (std::nothrow) fpsi_gnn();
  if (!m) return FPSI_E_NOMEM;
  m->L = layout();
  if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete m;
    fpsi::set_error("learned start: cudaStreamCreate failed");
    return FPSI_E_CUDA;
  }
  const int64_t np = m->L.total;
  int rc = FPSI_OK;
#define G(e) \
  if (!rc) rc = (e)
  G(galloc(&m->d_w, np));
  G(galloc(&m->d_m, np));
  G(galloc(&m->d_v, np));
  G(galloc(&m->d_g, np));
  G(galloc(&m->d_wb, np));
  G(galloc(&m->d_err, 1));
  G(galloc(&m->d_fac, 64));
#undef G
  if (!rc && cudaMemset(m->d_err, 0, sizeof(int32_t)) != cudaSuccess) rc = FPSI_E_CUDA;
  int dev = 0;
  if (!rc && (cudaGetDevice(&dev) != cudaSuccess ||
              cudaDeviceGetAttribute(&m->nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
              cudaFuncSetAttribute(k_layer_tc<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(tc_smem(W).total)) != cudaSuccess ||
              cudaFuncSetAttribute(k_layer_tc<__nv_bfloat16, false>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(tc_smem(W).total)) != cudaSuccess ||
              cudaFuncSetAttribute(k_layer_tc<__nv_bfloat16, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(tc_smem(W).total)) != cudaSuccess ||
              cudaFuncSetAttribute(k_layer_ws<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(ws_smem(W).total)) != cudaSuccess ||
              cudaFuncSetAttribute(k_layer_ws<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(ws_smem(W).total)) != cudaSuccess)) {
    fpsi::set_error("learned start: device query failed");
    rc = FPSI_E_CUDA;
  }
  if (rc) {
    fpsi_gnn_destroy(m);
    return rc;
  }
  // He-style uniform initialisation from a counter-based generator; the
  // head starts at zero so the untrained model gives the Jacobi start
  std::vector<float> w(np, 0.f);
  auto u01 = [&](uint64_t i) {
    uint64_t z = seed * 0x100000001B3ull + i + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return double(z >> 11) * (1.0 / 9007199254740992.0);
  };
  for (int l = 0; l < NLAYER; ++l) {
    const int fin = m->L.fan_in[l];
    const double a = std::sqrt(3.0 / (2.0 * fin));
    for (int64_t i = 0; i < int64_t(W) * fin; ++i) {
      w[m->L.ws[l] + i] = float(a * (2 * u01(m->L.ws[l] + i) - 1));
      w[m->L.wn[l] + i] = float(a * (2 * u01(m->L.wn[l] + i) - 1));
    }
  }
  rc = fpsi_gnn_set_params(m, w.data());
  if (rc) {
    fpsi_gnn_destroy(m);
    return rc;
  }
  *out = m;
  return FPSI_OK;
}

int fpsi_gnn_clear_snapshots(fpsi_gnn* m) {
  if (!m) return FPSI_E_INVALID;
  if (m->stream) cudaStreamSynchronize(m->stream);
  for (Snapshot& s : m->snaps) free_snapshot(s);
  m->snaps.clear();
  return FPSI_OK;
}

int fpsi_gnn_destroy(fpsi_gnn* m) {
  if (!m) return FPSI_OK;
  fpsi_gnn_clear_snapshots(m);
  free_activations(m);
  void* ps[] = {m->d_w, m->d_m, m->d_v, m->d_g, m->d_wb, m->d_err, m->d_fac};
  for (void* p : ps)
    if (p) cudaFree(p);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
  return FPSI_OK;
}

int64_t fpsi_gnn_num_params(const fpsi_gnn* m) { return m ? m->L.total : 0; }

int fpsi_gnn_get_params(fpsi_gnn* m, float* w) {
  if (!m || !w) return FPSI_E_INVALID;
  FPSI_CUDA_TRY(cudaMemcpy(w, m->d_w, m->L.total * 4, cudaMemcpyDeviceToHost));
  return FPSI_OK;
}

int fpsi_gnn_set_params(fpsi_gnn* m, const float* w) {
  if (!m || !w) return FPSI_E_INVALID;
  FPSI_CUDA_TRY(cudaMemcpy(m->d_w, w, m->L.total * 4, cudaMemcpyHostToDevice));
  FPSI_CUDA_TRY(cudaMemset(m->d_m, 0, m->L.total * 4));
  FPSI_CUDA_TRY(cudaMemset(m->d_v, 0, m->L.total * 4));
  m->adam_t = 0;
  k_to_bf16<<<nb_(m->L.total, 256), 256, 0, m->stream>>>(m->L.total, m->d_w, m->d_wb);
  FPSI_CUDA_TRY(cudaStreamSynchronize(m->stream));
  return FPSI_OK;
}

// features of ctx's assembled system into (feat, xj, scales)
// (activation buffers must hold x's cells)
static int make_features(fpsi_gnn* m, fpsi_ctx* x, float* feat, float* xj, float* rs, float* xs) {
  if (!x->have_asm || !x->d_D || x->P.solver == FPSI_SOLVER_LSGS) {
    fpsi::set_error("learned start: needs an assembled SGS system with the diagonal blocks kept");
    return FPSI_E_STATE;
  }
  const int64_t nc = x->H.nc;
  if (nc > m->cap) return FPSI_E_INVALID;
  // from now on the context keeps a copy of each applied update
  if (!x->d_xprev) {
    if (cudaMalloc(&x->d_xprev, size_t(nc) * 5 * 8) != cudaSuccess) {
      x->d_xprev = nullptr;
      fpsi::set_error("cudaMalloc failed for the previous-update copy");
      return FPSI_E_NOMEM;
    }
    x->have_xprev = false;
  }
  x->keep_prev = true;
  const void* xprev = x->have_xprev ? x->d_xprev : nullptr;
  // x_J = D^-1 B from the factored blocks (the iterate may hold a solve)
  FPSI_CUDA_TRY(cudaStreamSynchronize(m->stream));
  int rc0 = fpsi::launch_jacobi_start(x);
  if (rc0) return rc0;
  FPSI_CUDA_TRY(cudaStreamSynchronize(x->stream));
  float* raw = m->d_dagg;  // [nc][40] scratch inside an [nc][64] buffer
  if (x->P.precision == FPSI_PREC_FP64)
    k_features_raw<double, double><<<nb_(nc, FCB), 256, 0, m->stream>>>(
        nc, x->d_src, (const double*)x->d_D, (const double*)x->d_x, (const double*)xprev, x->d_ci, raw,
        xj);
  else if (x->P.precision == FPSI_PREC_MIXED)
    k_features_raw<float, float><<<nb_(nc, FCB), 256, 0, m->stream>>>(
        nc, x->d_src, (const float*)x->d_D, (const float*)x->d_x, (const float*)xprev, x->d_ci, raw, xj);
  else
    k_features_raw<float, double><<<nb_(nc, FCB), 256, 0, m->stream>>>(
        nc, x->d_src, (const float*)x->d_D, (const double*)x->d_x, (const double*)xprev, x->d_ci, raw,
        xj);
  const int nblk = int(nb_(nc, GT));
  k_rms_partial<<<nblk, GT, 0, m->stream>>>(nc, raw, xj, m->d_lpart);
  k_feat_scales<<<1, FS_THREADS, 0, m->stream>>>(m->d_lpart, nblk, nc, m->d_fac);
  float scl[10];
  FPSI_CUDA_TRY(cudaMemcpyAsync(scl, m->d_fac, sizeof(scl), cudaMemcpyDeviceToHost, m->stream));
  k_features_norm<<<nb_(nc, FCB), 256, 0, m->stream>>>(nc, raw, xj, m->d_fac, feat);
  FPSI_CUDA_TRY(cudaStreamSynchronize(m->stream));
  for (int k = 0; k < 5; ++k) rs[k] = scl[k], xs[k] = scl[5 + k];
  FPSI_CUDA_TRY(cudaGetLastError());
  return FPSI_OK;
}

__global__ void k_target(int64_t nc, const double* __restrict__ dq_rcm, const float* __restrict__ xj,
                         const float* __restrict__ scl, float* __restrict__ t) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= nc * 5) return;
  const int k = int(i % 5);
  t[i] = float((dq_rcm[i] - double(xj[i])) / double(scl[k]));
}

int fpsi_gnn_add_snapshot(fpsi_gnn* m, fpsi_ctx* x, const double* dq) {
  if (!m || !x || !dq) return FPSI_E_INVALID;
  Snapshot s;
  const int64_t nc = x->H.nc;
  Graph G;
  int rc = ensure_capacity(m, nc);
  if (!rc) rc = ctx_graph(x, &G);
  if (!rc) rc = galloc(&s.d_off, nc + 1);
  if (!rc) rc = galloc(&s.d_nb, x->cnb_n);
  if (!rc) rc = galloc(&s.feat, nc * NIN);
  if (!rc) rc = galloc(&s.target, nc * 5);
  if (!rc) rc = galloc(&s.xj, nc * 5);
  if (!rc) rc = make_features(m, x, s.feat, s.xj, s.rs, s.xs);
  double* dd = nullptr;
  if (!rc) rc = galloc(&dd, nc * 5);
  if (rc) {
    free_snapshot(s);
    return rc;
  }
  s.nc = nc;
  s.perm = x->H.perm;
  // target in RCM order
  std::vector<double> d(nc * 5);
  for (int64_t i = 0; i < nc; ++i)
    for (int k = 0; k < 5; ++k) d[5 * i + k] = dq[5 * int64_t(s.perm[i]) + k];
  float* dscl = reinterpret_cast<float*>(m->d_lpart);
  bool ok = cudaMemcpyAsync(s.d_off, G.off, (nc + 1) * 4, cudaMemcpyDeviceToDevice, m->stream) == cudaSuccess &&
            (x->cnb_n == 0 || cudaMemcpyAsync(s.d_nb, G.nb, x->cnb_n * 4, cudaMemcpyDeviceToDevice,
                                              m->stream) == cudaSuccess) &&
            cudaMemcpyAsync(dd, d.data(), d.size() * 8, cudaMemcpyHostToDevice, m->stream) == cudaSuccess &&
            cudaMemcpyAsync(dscl, s.xs, 5 * sizeof(float), cudaMemcpyHostToDevice, m->stream) == cudaSuccess;
  if (ok) {
    k_target<<<nb_(nc * 5, 256), 256, 0, m->stream>>>(nc, dd, s.xj, dscl, s.target);
    ok = cudaStreamSynchronize(m->stream) == cudaSuccess;
  }
  cudaFree(dd);
  if (!ok) {
    free_snapshot(s);
    fpsi::set_error("learned start: snapshot upload failed");
    return FPSI_E_CUDA;
  }
  m->snaps.push_back(std::move(s));
  return FPSI_OK;
}

__global__ void k_gather_rows(int64_t n, const int32_t* __restrict__ idx, int w,
                              const float* __restrict__ src, float* __restrict__ dst) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n * w) return;
  const int64_t r = i / w;
  dst[i] = src[int64_t(idx[r]) * w + (i - r * w)];
}

int fpsi_gnn_add_snapshot_region(fpsi_gnn* m, fpsi_ctx* x, const double* dq, const double* lo,
                                 const double* hi, int32_t halo) {
  if (!m || !x || !dq || !lo || !hi || halo < 0) return FPSI_E_INVALID;
  const int64_t nc = x->H.nc;
  Graph G;
  int rc = ensure_capacity(m, nc);
  if (!rc) rc = ctx_graph(x, &G);
  if (rc) return rc;
  // features of the whole system in the backward pass's scratch
  float* ffull = m->d_dz;
  float* xfull = m->d_dh;
  float rs[5], xs[5];
  if ((rc = make_features(m, x, ffull, xfull, rs, xs))) return rc;
  // cells of the box (RCM order) and their interior-face neighbours
  const fpsi::HostMesh& H = x->H;
  std::vector<int32_t> sel, newid(nc, -1);
  for (int64_t c = 0; c < nc; ++c) {
    bool in = true;
    for (int d = 0; d < 3; ++d) in = in && H.cc[3 * c + d] >= lo[d] && H.cc[3 * c + d] < hi[d];
    if (in) {
      newid[c] = int32_t(sel.size());
      sel.push_back(int32_t(c));
    }
  }
  const int64_t ns = int64_t(sel.size());
  if (ns == 0) {
    fpsi::set_error("learned start: no cell centre inside the snapshot box");
    return FPSI_E_INVALID;
  }
  auto nbrs = [&](int64_t c, auto&& fn) {
    for (int32_t e = H.cf_off[c]; e < H.cf_off[c + 1]; ++e) {
      const int64_t f = H.cf[e] >> 1;
      if (H.cr[f] < 0) continue;
      fn(int64_t((H.cf[e] & 1) ? H.cl[f] : H.cr[f]));
    }
  };
  // hops from each box cell to the nearest cell outside the box (up to halo+1)
  std::vector<int32_t> dist(nc, -1), front, next;
  for (int64_t c = 0; c < nc; ++c)
    if (newid[c] < 0) dist[c] = 0;
  for (int64_t c : sel) {
    bool edge = false;
    nbrs(c, [&](int64_t o) { edge = edge || newid[o] < 0; });
    if (edge) dist[c] = 1, front.push_back(int32_t(c));
  }
  for (int h = 2; h <= halo + 1 && !front.empty(); ++h) {
    next.clear();
    for (int32_t c : front)
      nbrs(c, [&](int64_t o) {
        if (dist[o] < 0) dist[o] = h, next.push_back(int32_t(o));
      });
    front.swap(next);
  }
  std::vector<float> mask(ns);
  std::vector<int32_t> off(ns + 1, 0), nb;
  for (int64_t j = 0; j < ns; ++j) {
    const int64_t c = sel[j];
    mask[j] = (dist[c] < 0 || dist[c] > halo) ? 1.f : 0.f;
    nbrs(c, [&](int64_t o) {
      if (newid[o] >= 0) nb.push_back(newid[o]);
    });
    off[j + 1] = int32_t(nb.size());
  }
  Snapshot s;
  int32_t* didx = nullptr;
  double* dd = nullptr;
  rc = galloc(&s.d_off, ns + 1);
  if (!rc) rc = galloc(&s.d_nb, std::max<size_t>(nb.size(), 1));
  if (!rc) rc = galloc(&s.feat, ns * NIN);
  if (!rc) rc = galloc(&s.target, ns * 5);
  if (!rc) rc = galloc(&s.xj, ns * 5);
  if (!rc) rc = galloc(&s.mask, ns);
  if (!rc) rc = galloc(&didx, ns);
  if (!rc) rc = galloc(&dd, ns * 5);
  std::vector<double> d(ns * 5);
  for (int64_t j = 0; j < ns; ++j)
    for (int k = 0; k < 5; ++k) d[5 * j + k] = dq[5 * int64_t(H.perm[sel[j]]) + k];
  float* dscl = reinterpret_cast<float*>(m->d_lpart);
  bool ok = !rc;
  cudaStream_t st = m->stream;
  ok = ok && cudaMemcpyAsync(s.d_off, off.data(), off.size() * 4, cudaMemcpyHostToDevice, st) == cudaSuccess;
  ok = ok && (nb.empty() ||
              cudaMemcpyAsync(s.d_nb, nb.data(), nb.size() * 4, cudaMemcpyHostToDevice, st) == cudaSuccess);
  ok = ok && cudaMemcpyAsync(s.mask, mask.data(), ns * 4, cudaMemcpyHostToDevice, st) == cudaSuccess;
  ok = ok && cudaMemcpyAsync(didx, sel.data(), ns * 4, cudaMemcpyHostToDevice, st) == cudaSuccess;
  ok = ok && cudaMemcpyAsync(dd, d.data(), d.size() * 8, cudaMemcpyHostToDevice, st) == cudaSuccess;
  ok = ok && cudaMemcpyAsync(dscl, xs, 5 * sizeof(float), cudaMemcpyHostToDevice, st) == cudaSuccess;
  if (ok) {
    k_gather_rows<<<nb_(ns * NIN, 256), 256, 0, st>>>(ns, didx, NIN, ffull, s.feat);
    k_gather_rows<<<nb_(ns * 5, 256), 256, 0, st>>>(ns, didx, 5, xfull, s.xj);
    k_target<<<nb_(ns * 5, 256), 256, 0, st>>>(ns, dd, s.xj, dscl, s.target);
    ok = cudaGetLastError() == cudaSuccess && cudaStreamSynchronize(st) == cudaSuccess;
  }
  cudaFree(didx);
  cudaFree(dd);
  if (!ok) {
    free_snapshot(s);
    if (!rc) fpsi::set_error("learned start: region snapshot upload failed");
    return rc ? rc : FPSI_E_CUDA;
  }
  s.nc = ns;
  s.perm.resize(ns);
  for (int64_t j = 0; j < ns; ++j) s.perm[j] = int32_t(j);  // snapshot order
  for (int k = 0; k < 5; ++k) s.rs[k] = rs[k], s.xs[k] = xs[k];
  m->snaps.push_back(std::move(s));
  return FPSI_OK;
}

int fpsi_gnn_num_snapshots(const fpsi_gnn* m) { return m ? int(m->snaps.size()) : 0; }

int64_t fpsi_gnn_snapshot_cells(const fpsi_gnn* m, int32_t si) {
  if (!m || si < 0 || si >= int32_t(m->snaps.size())) return -1;
  return m->snaps[si].nc;
}

int fpsi_gnn_get_snapshot(fpsi_gnn* m, int32_t si, float* feat, float* target, float* xj,
                          float* scales) {
  if (!m || si < 0 || si >= int32_t(m->snaps.size())) return FPSI_E_INVALID;
  const Snapshot& s = m->snaps[si];
  const int64_t nc = s.nc;
  auto fetch = [&](const float* dsrc, int w, float* dst) -> int {
    if (!dst) return FPSI_OK;
    std::vector<float> h(nc * w);
    FPSI_CUDA_TRY(cudaMemcpy(h.data(), dsrc, h.size() * 4, cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < nc; ++i)
      for (int k = 0; k < w; ++k) dst[int64_t(s.perm[i]) * w + k] = h[i * w + k];
    return FPSI_OK;
  };
  int rc = fetch(s.feat, NIN, feat);
  if (!rc) rc = fetch(s.target, 5, target);
  if (!rc) rc = fetch(s.xj, 5, xj);
  if (scales)
    for (int k = 0; k < 5; ++k) scales[k] = s.rs[k], scales[5 + k] = s.xs[k];
  return rc;
}

// loss (batch = cells whose hash is below the threshold; batch >= nc: all)
static uint64_t threshold(int64_t nc, int64_t batch) {
  if (batch >= nc) return ~uint64_t(0);
  return uint64_t((long double)batch / (long double)nc * 18446744073709551615.0L);
}

int fpsi_gnn_loss_grad(fpsi_gnn* m, int32_t si, int64_t batch, uint64_t seed, double* loss,
                       float* grad) {
  if (!m || si < 0 || si >= int32_t(m->snaps.size())) return FPSI_E_INVALID;
  const Snapshot& s = m->snaps[si];
  int rc = ensure_capacity(m, s.nc);
  if (!rc) rc = forward(m, s.graph(), s.feat, true);
  if (rc) return rc;
  double* dl = m->d_lpart + ((s.nc + GT - 1) / GT) * 2 + 2;
  if ((rc = backward(m, s.graph(), s.feat, s.target, s.mask, seed, threshold(s.nc, batch), dl))) return rc;
  double h[2];
  FPSI_CUDA_TRY(cudaMemcpyAsync(h, dl, sizeof(h), cudaMemcpyDeviceToHost, m->stream));
  FPSI_CUDA_TRY(cudaStreamSynchronize(m->stream));
  if ((rc = take_error(m))) return rc;
  if (loss) *loss = h[0];
  if (grad) FPSI_CUDA_TRY(cudaMemcpy(grad, m->d_g, m->L.total * 4, cudaMemcpyDeviceToHost));
  return FPSI_OK;
}

int fpsi_gnn_train(fpsi_gnn* m, int32_t nsteps, int64_t batch, uint64_t seed, double lr,
                   double* losses) {
  if (!m || nsteps < 0 || m->snaps.empty()) return FPSI_E_INVALID;
  const int64_t np = m->L.total;
  const int ns = int(m->snaps.size());
  int64_t ncmax = 0;
  for (const Snapshot& s : m->snaps) ncmax = std::max(ncmax, s.nc);
  int rc0 = ensure_capacity(m, ncmax);
  if (rc0) return rc0;
  double* dhist = nullptr;
  if (losses && galloc(&dhist, size_t(nsteps) + 1)) return FPSI_E_NOMEM;
  for (int32_t it = 0; it < nsteps; ++it) {
    const uint64_t sd = seed * 1000003ull + uint64_t(it);
    const Snapshot& s = m->snaps[size_t(sd % uint64_t(ns))];
    double* dl = m->d_lpart + ((s.nc + GT - 1) / GT) * 2 + 2;
    int rc = forward(m, s.graph(), s.feat, true);
    if (!rc) rc = backward(m, s.graph(), s.feat, s.target, s.mask, sd, threshold(s.nc, batch), dl);
    if (rc) {
      cudaFree(dhist);
      return rc;
    }
    m->adam_t += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = float(1.0 - std::pow(double(b1), double(m->adam_t)));
    const float c2 = float(1.0 - std::pow(double(b2), double(m->adam_t)));
    k_adam<<<nb_(np, 256), 256, 0, m->stream>>>(np, m->d_w, m->d_m, m->d_v, m->d_g, m->d_wb,
                                                float(lr), b1, b2, 1e-8f, c1, c2);
    if (dhist) cudaMemcpyAsync(dhist + it, dl, 8, cudaMemcpyDeviceToDevice, m->stream);
  }
  FPSI_CUDA_TRY(cudaGetLastError());
  if (dhist) {
    FPSI_CUDA_TRY(cudaMemcpyAsync(losses, dhist, size_t(nsteps) * 8, cudaMemcpyDeviceToHost, m->stream));
  }
  FPSI_CUDA_TRY(cudaStreamSynchronize(m->stream));
  cudaFree(dhist);
  return take_error(m);
}

}  // extern "C"

namespace {
// ---- inference features in two passes, with no host round trip ----------
// Per-block sums of squares of B (= float(src)) and x_J (= float of the
// colour-order iterate), GT cells per block and the same tree as
// k_rms_partial, so the partials are the ones the training features use.
template <class TX>
__global__ void k_feat_stats(int64_t nc, const double* __restrict__ src, const TX* __restrict__ x_ci,
                             const int32_t* __restrict__ ci, double* __restrict__ part) {
  const int64_t c = int64_t(blockIdx.x) * GT + threadIdx.x;
  __shared__ double sh[10][GT];
  const int64_t i = c < nc ? int64_t(ci[c]) : 0;
  for (int k = 0; k < 5; ++k) {
    const double b = c < nc ? double(float(src[5 * c + k])) : 0.0;
    const double x = c < nc ? double(float(x_ci[5 * i + k])) : 0.0;
    sh[k][threadIdx.x] = b * b;
    sh[5 + k][threadIdx.x] = x * x;
  }
  __syncthreads();
  for (int st = GT / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int k = 0; k < 10; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 10; ++k) part[10 * blockIdx.x + k] = sh[k][0];
}

// the 40 normalised features of a cell straight from the system, rounded
// to BF16 (B, D, x_J, dq_prev; the same float products as
// k_features_raw + k_features_norm), one 16 B chunk of 8 per thread
template <class TB, class TX>
__global__ void k_features_bf16(int64_t nc, const double* __restrict__ src, const TB* __restrict__ D,
                                const TX* __restrict__ x_ci, const TX* __restrict__ xprev_ci,
                                const int32_t* __restrict__ ci, const float* __restrict__ fac,
                                __nv_bfloat16* __restrict__ feat) {
  __shared__ float f[NIN];
  if (threadIdx.x < NIN) f[threadIdx.x] = fac[10 + threadIdx.x];
  __syncthreads();
  const int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;  // chunk
  if (j >= nc * (NIN / 8)) return;
  const int64_t c = j / (NIN / 8);
  const int k0 = 8 * int(j - (NIN / 8) * c);
  const int64_t i = ci[c];
  float v[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    const int k = k0 + e;
    float r;
    if (k < 5)
      r = float(src[5 * c + k]);
    else if (k < 30)
      r = float(D[25 * c + k - 5]);
    else if (k < 35)
      r = float(x_ci[5 * i + k - 30]);
    else
      r = xprev_ci ? float(xprev_ci[5 * i + k - 35]) : 0.f;
    v[e] = r * f[k];
  }
  *reinterpret_cast<uint4*>(feat + c * NIN + k0) = pack8(v);
}

// x0 = x_J + xs * d into ctx's colour-order iterate, which holds x_J (the
// next linear solve starts from it); x0_out (RCM order) optional
template <class TX>
__global__ void k_apply_start(int64_t nc, const float* __restrict__ y, const float* __restrict__ fac,
                              const int32_t* __restrict__ ci, TX* __restrict__ x, double* __restrict__ x0) {
  const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const int64_t i = ci[c];
  for (int k = 0; k < 5; ++k) {
    const float xj = float(x[5 * i + k]);
    const double v = double(xj) + double(fac[5 + k]) * double(y[c * 5 + k]);
    x[5 * i + k] = TX(v);
    if (x0) x0[5 * c + k] = v;
  }
}

template <class TB, class TX>
void launch_features16(fpsi_gnn* m, fpsi_ctx* x, __nv_bfloat16* feat, cudaStream_t s) {
  const int64_t nc = x->H.nc;
  const int nblk = int(nb_(nc, GT));
  const TX* xv = static_cast<const TX*>(x->d_x);
  const TX* xp = x->have_xprev ? static_cast<const TX*>(x->d_xprev) : nullptr;
  k_feat_stats<TX><<<nblk, GT, 0, s>>>(nc, x->d_src, xv, x->d_ci, m->d_lpart);
  k_feat_scales<<<1, FS_THREADS, 0, s>>>(m->d_lpart, nblk, nc, m->d_fac);
  k_features_bf16<TB, TX><<<nb_(nc * (NIN / 8), 256), 256, 0, s>>>(
      nc, x->d_src, static_cast<const TB*>(x->d_D), xv, xp, x->d_ci, m->d_fac, feat);
}
}  // namespace

extern "C" {

// Inference runs on the context's stream: the Jacobi start D^-1 B, the
// features (two kernels and a one-block scale kernel, no host round trip),
// the three layers with the head, and the start written over D^-1 B.
int fpsi_gnn_predict(fpsi_gnn* m, fpsi_ctx* x, double* x0) {
  if (!m || !x) return FPSI_E_INVALID;
  const int64_t nc = x->H.nc;
  double* dx0 = nullptr;
  int rc = FPSI_OK;
  if (x0 && (rc = galloc(&dx0, nc * 5))) return rc;
  rc = fpsi::gnn_predict_launch(m, x, dx0);
  if (!rc && cudaStreamSynchronize(x->stream) != cudaSuccess) rc = FPSI_E_CUDA;
  if (!rc) rc = take_error(m);
  if (!rc && x0) {
    std::vector<double> h(nc * 5);
    if (cudaMemcpy(h.data(), dx0, h.size() * 8, cudaMemcpyDeviceToHost) != cudaSuccess) rc = FPSI_E_CUDA;
    for (int64_t i = 0; !rc && i < nc; ++i)
      for (int k = 0; k < 5; ++k) x0[5 * int64_t(x->H.perm[i]) + k] = h[5 * i + k];
  }
  cudaFree(dx0);
  return rc;
}

}  // extern "C"
namespace fpsi {
// Inference queued on the context's stream with no host synchronisation:
// the Jacobi start, the features, the layers and the start written into the
// iterate (and, with dx0, a copy in RCM order).  The model's error bits
// (gnn_error_bits) are left for the caller to read.  jacobi_in_iterate: the
// iterate already holds D^-1 B (an SGS assembly has just written it).
int32_t* gnn_error_bits(fpsi_gnn* m) { return m->d_err; }
int gnn_predict_launch(fpsi_gnn* m, fpsi_ctx* x, double* dx0, bool jacobi_in_iterate) {
  if (!x->have_asm || !x->d_D || x->P.solver == FPSI_SOLVER_LSGS) {
    set_error("learned start: needs an assembled SGS system with the diagonal blocks kept");
    return FPSI_E_STATE;
  }
  const int64_t nc = x->H.nc;
  Graph G;
  int rc = ensure_capacity(m, nc);
  if (!rc) rc = ctx_graph(x, &G);
  if (rc) return rc;
  // from now on the context keeps a copy of each applied update
  if (!x->d_xprev) {
    if (cudaMalloc(&x->d_xprev, size_t(nc) * 5 * 8) != cudaSuccess) {
      x->d_xprev = nullptr;
      set_error("cudaMalloc failed for the previous-update copy");
      return FPSI_E_NOMEM;
    }
    x->have_xprev = false;
  }
  x->keep_prev = true;
  FPSI_CUDA_TRY(cudaStreamSynchronize(m->stream));  // no training pass in flight
  cudaStream_t s = x->stream;
  // x_J = D^-1 B from the factored blocks (the iterate may hold a solve)
  if (!jacobi_in_iterate && (rc = launch_jacobi_start(x))) return rc;
  // BF16 features [nc][40] in a backward-pass buffer an inference pass does
  // not use ([nc][64] FP32)
  __nv_bfloat16* feat16 = reinterpret_cast<__nv_bfloat16*>(m->d_dz);
  if (x->P.precision == FPSI_PREC_FP64)
    launch_features16<double, double>(m, x, feat16, s);
  else if (x->P.precision == FPSI_PREC_MIXED)
    launch_features16<float, float>(m, x, feat16, s);
  else
    launch_features16<float, double>(m, x, feat16, s);
  if ((rc = forward(m, G, nullptr, false, feat16, s))) return rc;
  if (x->P.precision == FPSI_PREC_MIXED)
    k_apply_start<float><<<nb_(nc, 256), 256, 0, s>>>(nc, m->d_y, m->d_fac, x->d_ci, (float*)x->d_x, dx0);
  else
    k_apply_start<double><<<nb_(nc, 256), 256, 0, s>>>(nc, m->d_y, m->d_fac, x->d_ci, (double*)x->d_x, dx0);
  FPSI_CUDA_TRY(cudaGetLastError());
  x->x_preset = true;
  return FPSI_OK;
}
}  // namespace fpsi

