// mlp.cu -- the density-compensation regressor: a multilayer perceptron
// 18 -> 64 -> 64 -> 64 -> 1 (ReLU), BF16 weights, FP32 activations and
// accumulation, trained on the device by hand-written forward / backward
// kernels with Adam on FP32 master weights; inference on the tensor cores
// (mlp_infer_mma_kernel).
//
// Parameters, one flat FP32 vector (row-major, out x in):
//   W1[64][18] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[64] b4
// The forward and backward passes use the BF16 rounding (nearest even) of the
// master weights, refreshed after every Adam update.
//
// Kernel layout.  A CTA of 256 threads takes 64 samples: the weights (as FP32)
// and the 64 samples' activations and back-propagated errors live in shared
// memory (rows padded to 65 floats, so a warp's 32 neurons hit 32 banks while
// a sample row is a broadcast).  Thread t owns neuron i = t mod 64 of samples
// t / 64 + 4k, k < 16, in every layer; for the weight gradients it owns entries
// (i, t / 64 + 4k).  Each CTA writes its partial gradient; one reduction
// kernel sums the partials in CTA order (deterministic) and applies Adam.
#include "../../include/mirt_b200.h"

#include <cuda_bf16.h>

#include <cmath>
#include <string>
#include <new>
#include <vector>

#include "runtime.cuh"

using namespace mirt;

namespace {

#define MCK(call)                                                                     \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return api_fail(e_ == cudaErrorMemoryAllocation ? MIRT_ERR_ALLOC : MIRT_ERR_CUDA, \
                      std::string(#call) + ": " + cudaGetErrorString(e_));            \
  } while (0)

constexpr int NIN = MIRT_DCF_NFEAT;
constexpr int HID = 64;
constexpr int NS = 64;       // samples per CTA
constexpr int NT = 256;      // threads per CTA
constexpr int KS = NS / 4;   // samples per thread
constexpr int LD = HID + 1;  // padded row
constexpr int LDI = NIN + 1;
constexpr int P_W1 = 0, P_B1 = P_W1 + HID * NIN, P_W2 = P_B1 + HID, P_B2 = P_W2 + HID * HID,
              P_W3 = P_B2 + HID, P_B3 = P_W3 + HID * HID, P_W4 = P_B3 + HID, P_B4 = P_W4 + HID,
              NPARAM = P_B4 + 1;
static_assert(NPARAM == MIRT_MLP_NPARAM, "parameter count");

struct Weights {  // shared-memory FP32 copy of the BF16 weights
  float W1[HID][LDI];
  float b1[HID];
  float W2[HID][LD];
  float b2[HID];
  float W3[HID][LD];
  float b3[HID];
  float W4[HID];
  float b4;
};

struct Acts {
  float X[NS][LDI];
  float H1[NS][LD], H2[NS][LD], H3[NS][LD];
  float out[NS], dout[NS];
};

struct Errs {
  float D1[NS][LD], D2[NS][LD], D3[NS][LD];
};

__device__ void load_weights(Weights &w, const __nv_bfloat16 *__restrict__ p) {
  for (int e = threadIdx.x; e < HID * NIN; e += NT) w.W1[e / NIN][e % NIN] = __bfloat162float(p[P_W1 + e]);
  for (int e = threadIdx.x; e < HID * HID; e += NT) {
    w.W2[e / HID][e % HID] = __bfloat162float(p[P_W2 + e]);
    w.W3[e / HID][e % HID] = __bfloat162float(p[P_W3 + e]);
  }
  for (int e = threadIdx.x; e < HID; e += NT) {
    w.b1[e] = __bfloat162float(p[P_B1 + e]);
    w.b2[e] = __bfloat162float(p[P_B2 + e]);
    w.b3[e] = __bfloat162float(p[P_B3 + e]);
    w.W4[e] = __bfloat162float(p[P_W4 + e]);
  }
  if (threadIdx.x == 0) w.b4 = __bfloat162float(p[P_B4]);
}

// H[s][i] = relu(b[i] + sum_j W[i][j] Hin[s][j]) for the thread's 16 samples
template <int NJ, int LDW, int LDH>
__device__ __forceinline__ void dense_relu(const float (*W)[LDW], const float *b,
                                           const float (*Hin)[LDH], float (*H)[LD]) {
  const int i = threadIdx.x & (HID - 1), s0 = threadIdx.x >> 6;
  float acc[KS];
#pragma unroll
  for (int k = 0; k < KS; k++) acc[k] = b[i];
  for (int j = 0; j < NJ; j++) {
    const float wij = W[i][j];
#pragma unroll
    for (int k = 0; k < KS; k++) acc[k] = fmaf(wij, Hin[s0 + 4 * k][j], acc[k]);
  }
#pragma unroll
  for (int k = 0; k < KS; k++) H[s0 + 4 * k][i] = fmaxf(acc[k], 0.f);
}

// forward through the three hidden layers and the output unit
__device__ void forward(const Weights &w, Acts &a) {
  dense_relu<NIN, LDI, LDI>(w.W1, w.b1, a.X, a.H1);
  __syncthreads();
  dense_relu<HID, LD, LD>(w.W2, w.b2, a.H1, a.H2);
  __syncthreads();
  dense_relu<HID, LD, LD>(w.W3, w.b3, a.H2, a.H3);
  __syncthreads();
  if (threadIdx.x < NS) {
    float acc = w.b4;
    for (int j = 0; j < HID; j++) acc = fmaf(w.W4[j], a.H3[threadIdx.x][j], acc);
    a.out[threadIdx.x] = acc;
  }
  __syncthreads();
}

// counter-based index hash (splitmix64 finaliser)
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

struct GradArgs {
  const float *x;        // [n][NIN]
  const float *y;        // [n]
  long long n;
  const long long *idx;  // explicit sample list [batch] (or null: hashed draw)
  int batch;
  unsigned long long seed;
  const int *step;       // device step counter (hashed draw)
  const __nv_bfloat16 *wb;
  float *part;           // [nblk][NPARAM]
  float *loss_part;      // [nblk]
};

// one CTA: forward + backward of up to 64 samples, partial gradient of the
// mean squared error over the whole batch
__global__ void __launch_bounds__(NT) mlp_grad_kernel(GradArgs g) {
  extern __shared__ __align__(16) unsigned char smem[];
  Weights &w = *reinterpret_cast<Weights *>(smem);
  Acts &a = *reinterpret_cast<Acts *>(smem + sizeof(Weights));
  Errs &d = *reinterpret_cast<Errs *>(smem + sizeof(Weights) + sizeof(Acts));
  load_weights(w, g.wb);
  const int b0 = blockIdx.x * NS;
  const int cnt = min(NS, g.batch - b0);
  const int st = g.step ? *g.step : 0;
  __shared__ long long src[NS];
  __shared__ float yv[NS];
  if (threadIdx.x < NS) {
    long long m = 0;
    if (threadIdx.x < cnt) {
      const long long r = b0 + threadIdx.x;
      m = g.idx ? g.idx[r]
                : (long long)(mix64(g.seed ^ ((unsigned long long)st << 32) ^ (unsigned long long)r) %
                              (unsigned long long)g.n);
    }
    src[threadIdx.x] = m;
    yv[threadIdx.x] = threadIdx.x < cnt ? g.y[m] : 0.f;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < NS * NIN; e += NT) {
    const int s = e / NIN, j = e % NIN;
    a.X[s][j] = s < cnt ? g.x[src[s] * NIN + j] : 0.f;
  }
  __syncthreads();
  forward(w, a);
  const float inv_b = 1.f / (float)g.batch;
  if (threadIdx.x < NS) {
    const float r = threadIdx.x < cnt ? a.out[threadIdx.x] - yv[threadIdx.x] : 0.f;
    a.dout[threadIdx.x] = 2.f * r * inv_b;
    a.out[threadIdx.x] = r * r;  // squared residual, summed below
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float l = 0.f;
    for (int s = 0; s < NS; s++) l += a.out[s];
    g.loss_part[blockIdx.x] = l * inv_b;
  }
  const int i = threadIdx.x & (HID - 1), s0 = threadIdx.x >> 6;
  // back-propagated errors
#pragma unroll
  for (int k = 0; k < KS; k++) {
    const int s = s0 + 4 * k;
    d.D3[s][i] = a.H3[s][i] > 0.f ? w.W4[i] * a.dout[s] : 0.f;
  }
  __syncthreads();
  {
    float acc[KS];
#pragma unroll
    for (int k = 0; k < KS; k++) acc[k] = 0.f;
    for (int kk = 0; kk < HID; kk++) {
      const float wk = w.W3[kk][i];
#pragma unroll
      for (int k = 0; k < KS; k++) acc[k] = fmaf(wk, d.D3[s0 + 4 * k][kk], acc[k]);
    }
#pragma unroll
    for (int k = 0; k < KS; k++) {
      const int s = s0 + 4 * k;
      d.D2[s][i] = a.H2[s][i] > 0.f ? acc[k] : 0.f;
    }
  }
  __syncthreads();
  {
    float acc[KS];
#pragma unroll
    for (int k = 0; k < KS; k++) acc[k] = 0.f;
    for (int kk = 0; kk < HID; kk++) {
      const float wk = w.W2[kk][i];
#pragma unroll
      for (int k = 0; k < KS; k++) acc[k] = fmaf(wk, d.D2[s0 + 4 * k][kk], acc[k]);
    }
#pragma unroll
    for (int k = 0; k < KS; k++) {
      const int s = s0 + 4 * k;
      d.D1[s][i] = a.H1[s][i] > 0.f ? acc[k] : 0.f;
    }
  }
  __syncthreads();
  // partial weight gradients: entry (i, j) with j = s0 + 4k
  float *part = g.part + (size_t)blockIdx.x * NPARAM;
  auto outer = [&](const float (*Dl)[LD], const float *Hp, int ldh, int nj, int pw) {
    float acc[KS];
#pragma unroll
    for (int k = 0; k < KS; k++) acc[k] = 0.f;
    for (int s = 0; s < NS; s++) {
      const float dv = Dl[s][i];
      const float *hrow = Hp + s * ldh;
#pragma unroll
      for (int k = 0; k < KS; k++) {
        const int j = s0 + 4 * k;
        if (j < nj) acc[k] = fmaf(dv, hrow[j], acc[k]);
      }
    }
#pragma unroll
    for (int k = 0; k < KS; k++) {
      const int j = s0 + 4 * k;
      if (j < nj) part[pw + i * nj + j] = acc[k];
    }
  };
  outer(d.D3, &a.H2[0][0], LD, HID, P_W3);
  outer(d.D2, &a.H1[0][0], LD, HID, P_W2);
  outer(d.D1, &a.X[0][0], LDI, NIN, P_W1);
  if (threadIdx.x < HID) {
    float gb1 = 0.f, gb2 = 0.f, gb3 = 0.f, gw4 = 0.f;
    for (int s = 0; s < NS; s++) {
      gb1 += d.D1[s][i];
      gb2 += d.D2[s][i];
      gb3 += d.D3[s][i];
      gw4 += a.dout[s] * a.H3[s][i];
    }
    part[P_B1 + i] = gb1;
    part[P_B2 + i] = gb2;
    part[P_B3 + i] = gb3;
    part[P_W4 + i] = gw4;
  }
  if (threadIdx.x == 0) {
    float gb4 = 0.f;
    for (int s = 0; s < NS; s++) gb4 += a.dout[s];
    part[P_B4] = gb4;
  }
}

struct AdamArgs {
  const float *part;
  const float *loss_part;
  int nblk;
  float *master, *m, *v;
  __nv_bfloat16 *wb;
  float *grad_out;  // optional: the summed gradient
  float *loss_hist;
  int *step;
  float lr, beta1, beta2, eps;
  int apply;        // 0: only sum the gradient (and loss)
};

// sum the partial gradients in CTA order; Adam on the FP32 master weights
__global__ void mlp_adam_kernel(AdamArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int t = *a.step + 1;
  if (p < NPARAM) {
    float g = 0.f;
    for (int b = 0; b < a.nblk; b++) g += a.part[(size_t)b * NPARAM + p];
    if (a.grad_out) a.grad_out[p] = g;
    if (a.apply) {
      const float m = a.beta1 * a.m[p] + (1.f - a.beta1) * g;
      const float v = a.beta2 * a.v[p] + (1.f - a.beta2) * g * g;
      a.m[p] = m;
      a.v[p] = v;
      const float mh = m / (1.f - powf(a.beta1, (float)t));
      const float vh = v / (1.f - powf(a.beta2, (float)t));
      const float th = a.master[p] - a.lr * mh / (sqrtf(vh) + a.eps);
      a.master[p] = th;
      a.wb[p] = __float2bfloat16_rn(th);
    }
  }
  if (p == 0) {
    float l = 0.f;
    for (int b = 0; b < a.nblk; b++) l += a.loss_part[b];
    if (a.loss_hist) a.loss_hist[t - 1] = l;
  }
}

__global__ void mlp_step_kernel(int *step) { *step += 1; }

__global__ void to_bf16_kernel(const float *__restrict__ m, __nv_bfloat16 *__restrict__ wb, int n) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) wb[p] = __float2bfloat16_rn(m[p]);
}

// inference: w = exp(sigma * out + mu) per sample
__global__ void __launch_bounds__(NT) mlp_infer_kernel(const float *__restrict__ x, long long n,
                                                       const __nv_bfloat16 *__restrict__ wb,
                                                       float mu, float sigma,
                                                       float *__restrict__ yhat,
                                                       double *__restrict__ wout) {
  extern __shared__ __align__(16) unsigned char smem[];
  Weights &w = *reinterpret_cast<Weights *>(smem);
  Acts &a = *reinterpret_cast<Acts *>(smem + sizeof(Weights));
  load_weights(w, wb);
  for (long long b0 = (long long)blockIdx.x * NS; b0 < n; b0 += (long long)gridDim.x * NS) {
    const int cnt = (int)min((long long)NS, n - b0);
    __syncthreads();
    for (int e = threadIdx.x; e < NS * NIN; e += NT) {
      const int s = e / NIN, j = e % NIN;
      a.X[s][j] = s < cnt ? x[(b0 + s) * NIN + j] : 0.f;
    }
    __syncthreads();
    forward(w, a);
    if (threadIdx.x < cnt) {
      const float o = a.out[threadIdx.x];
      if (yhat) yhat[b0 + threadIdx.x] = o;
      if (wout) wout[b0 + threadIdx.x] = exp((double)sigma * (double)o + (double)mu);
    }
  }
}

// ------------------------------------------------------------------------
// Inference on the tensor cores: mma.sync m16n8k16, BF16 operands, FP32
// accumulation.  A warp takes 16 samples at a time; the weights are exact
// BF16 (B operands, row-major W[out][in] is the column-major B the
// instruction wants), the FP32 activations enter as the sum of NTERM BF16
// terms (hi, then the BF16 rounding of each remainder), smallest term first,
// so that the products carry the activations to about 8 NTERM bits.  The D
// fragments of n-tiles 2k and 2k+1 are the A fragment of k-tile k of the next
// layer, so the activations stay in registers from layer to layer.
// Fragment layout (PTX ISA, m16n8k16 .bf16): g = lane / 4, t = lane % 4;
// A: a0 (row g, cols 2t, 2t+1), a1 (row g + 8), a2 (cols 2t + 8, 2t + 9),
// a3 (row g + 8, cols 2t + 8, 2t + 9); B: b0 (k 2t, 2t+1; n g), b1 (k 2t + 8,
// 2t + 9; n g); C/D: c0, c1 (row g, cols 2t, 2t+1), c2, c3 (row g + 8).
constexpr int MW1 = 40;  // W1 rows in shared memory: 18 inputs, zero-padded to 32, + 8 pad
constexpr int MWH = 72;  // W2, W3 rows: 64 + 8 pad (conflict-free B loads)

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// the NTERM BF16 terms of (v0, v1) packed as pairs, term 0 the largest
template <int NTERM>
__device__ __forceinline__ void split_pair(float v0, float v1, uint32_t (&t)[NTERM]) {
#pragma unroll
  for (int k = 0; k < NTERM; k++) {
    const __nv_bfloat16 h0 = __float2bfloat16_rn(v0), h1 = __float2bfloat16_rn(v1);
    t[k] = pack_bf16(h0, h1);
    v0 -= __bfloat162float(h0);
    v1 -= __bfloat162float(h1);
  }
}

// A fragments (NTERM terms) of k-tile kt from the previous layer's D fragments
template <int NTERM>
__device__ __forceinline__ void a_from_d(const float (&h)[8][4], int kt, uint32_t (&a)[NTERM][4]) {
  uint32_t t0[NTERM], t1[NTERM], t2[NTERM], t3[NTERM];
  split_pair<NTERM>(h[2 * kt][0], h[2 * kt][1], t0);
  split_pair<NTERM>(h[2 * kt][2], h[2 * kt][3], t1);
  split_pair<NTERM>(h[2 * kt + 1][0], h[2 * kt + 1][1], t2);
  split_pair<NTERM>(h[2 * kt + 1][2], h[2 * kt + 1][3], t3);
#pragma unroll
  for (int k = 0; k < NTERM; k++) {
    a[k][0] = t0[k];
    a[k][1] = t1[k];
    a[k][2] = t2[k];
    a[k][3] = t3[k];
  }
}

// out[8][4] = bias + A W^T over KT k-tiles (A given per k-tile by `afrag`)
template <int NTERM, int KT, int LDW, class AF>
__device__ __forceinline__ void mma_layer(const __nv_bfloat16 *__restrict__ W, const float *bias,
                                          AF afrag, float (&out)[8][4]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int nt = 0; nt < 8; nt++) {
    const float b0 = bias[nt * 8 + 2 * t], b1 = bias[nt * 8 + 2 * t + 1];
    out[nt][0] = b0;
    out[nt][1] = b1;
    out[nt][2] = b0;
    out[nt][3] = b1;
  }
#pragma unroll
  for (int kt = 0; kt < KT; kt++) {
    uint32_t a[NTERM][4];
    afrag(kt, a);
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
      const __nv_bfloat16 *wr = W + (nt * 8 + g) * LDW + kt * 16 + 2 * t;
      const uint32_t b0 = *reinterpret_cast<const uint32_t *>(wr);
      const uint32_t b1 = *reinterpret_cast<const uint32_t *>(wr + 8);
#pragma unroll
      for (int k = NTERM - 1; k >= 0; k--) mma_bf16(out[nt], a[k], b0, b1);
    }
  }
}

__device__ __forceinline__ void relu8(float (&h)[8][4]) {
#pragma unroll
  for (int nt = 0; nt < 8; nt++)
#pragma unroll
    for (int e = 0; e < 4; e++) h[nt][e] = fmaxf(h[nt][e], 0.f);
}

template <int NTERM>
__global__ void __launch_bounds__(NT, 2) mlp_infer_mma_kernel(const float *__restrict__ x, long long n,
                                                           const __nv_bfloat16 *__restrict__ wb,
                                                           float mu, float sigma,
                                                           float *__restrict__ yhat,
                                                           double *__restrict__ wout) {
  __shared__ __align__(16) __nv_bfloat16 sW1[HID * MW1];
  __shared__ __align__(16) __nv_bfloat16 sW2[HID * MWH];
  __shared__ __align__(16) __nv_bfloat16 sW3[HID * MWH];
  __shared__ float sb1[HID], sb2[HID], sb3[HID], sW4[HID];
  __shared__ float sb4;
  for (int e = threadIdx.x; e < HID * 32; e += NT) {
    const int r = e / 32, k = e % 32;
    sW1[r * MW1 + k] = k < NIN ? wb[P_W1 + r * NIN + k] : __float2bfloat16_rn(0.f);
  }
  for (int e = threadIdx.x; e < HID * HID; e += NT) {
    sW2[(e / HID) * MWH + e % HID] = wb[P_W2 + e];
    sW3[(e / HID) * MWH + e % HID] = wb[P_W3 + e];
  }
  for (int e = threadIdx.x; e < HID; e += NT) {
    sb1[e] = __bfloat162float(wb[P_B1 + e]);
    sb2[e] = __bfloat162float(wb[P_B2 + e]);
    sb3[e] = __bfloat162float(wb[P_B3 + e]);
    sW4[e] = __bfloat162float(wb[P_W4 + e]);
  }
  if (threadIdx.x == 0) sb4 = __bfloat162float(wb[P_B4]);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const long long ngrp = (n + 15) / 16;
  for (long long grp = (long long)blockIdx.x * (NT / 32) + warp; grp < ngrp;
       grp += (long long)gridDim.x * (NT / 32)) {
    const long long r0 = grp * 16 + g, r1 = r0 + 8;
    // the features of rows r0, r1 at this lane's columns (zero past 18 and past n)
    auto feat = [&](long long r, int k) -> float {
      return (r < n && k < NIN) ? __ldg(x + r * NIN + k) : 0.f;
    };
    float h1[8][4], h2[8][4];
    mma_layer<NTERM, 2, MW1>(sW1, sb1, [&](int kt, uint32_t (&a)[NTERM][4]) {
      const int k0 = kt * 16 + 2 * t;
      uint32_t t0[NTERM], t1[NTERM], t2[NTERM], t3[NTERM];
      split_pair<NTERM>(feat(r0, k0), feat(r0, k0 + 1), t0);
      split_pair<NTERM>(feat(r1, k0), feat(r1, k0 + 1), t1);
      split_pair<NTERM>(feat(r0, k0 + 8), feat(r0, k0 + 9), t2);
      split_pair<NTERM>(feat(r1, k0 + 8), feat(r1, k0 + 9), t3);
#pragma unroll
      for (int k = 0; k < NTERM; k++) {
        a[k][0] = t0[k];
        a[k][1] = t1[k];
        a[k][2] = t2[k];
        a[k][3] = t3[k];
      }
    }, h1);
    relu8(h1);
    mma_layer<NTERM, 4, MWH>(sW2, sb2, [&](int kt, uint32_t (&a)[NTERM][4]) {
      a_from_d<NTERM>(h1, kt, a);
    }, h2);
    relu8(h2);
    mma_layer<NTERM, 4, MWH>(sW3, sb3, [&](int kt, uint32_t (&a)[NTERM][4]) {
      a_from_d<NTERM>(h2, kt, a);
    }, h1);
    relu8(h1);
    // output unit: the quad of lanes sharing g holds all 64 columns of rows r0, r1
    float o0 = 0.f, o1 = 0.f;
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
      const float w0 = sW4[nt * 8 + 2 * t], w1 = sW4[nt * 8 + 2 * t + 1];
      o0 = fmaf(w0, h1[nt][0], fmaf(w1, h1[nt][1], o0));
      o1 = fmaf(w0, h1[nt][2], fmaf(w1, h1[nt][3], o1));
    }
    o0 += __shfl_xor_sync(0xffffffffu, o0, 1);
    o1 += __shfl_xor_sync(0xffffffffu, o1, 1);
    o0 += __shfl_xor_sync(0xffffffffu, o0, 2);
    o1 += __shfl_xor_sync(0xffffffffu, o1, 2);
    if (t == 0) {
      o0 += sb4;
      o1 += sb4;
      if (r0 < n) {
        if (yhat) yhat[r0] = o0;
        if (wout) wout[r0] = exp((double)sigma * (double)o0 + (double)mu);
      }
      if (r1 < n) {
        if (yhat) yhat[r1] = o1;
        if (wout) wout[r1] = exp((double)sigma * (double)o1 + (double)mu);
      }
    }
  }
}

constexpr size_t kGradSmem = sizeof(Weights) + sizeof(Acts) + sizeof(Errs);
constexpr size_t kInferSmem = sizeof(Weights) + sizeof(Acts);

}  // namespace

struct mirt_mlp {
  DMem master, m, v, wb, part, loss_part, step, grad, losses, idx;
  int nblk_cap = 0;
  int tensor_cores = 1;  // inference on mma.sync (1) or on the FP32 pipes (0)
  float lr = 1e-3f, beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
};

namespace {

int ensure_batch(mirt_mlp *q, int batch) {
  const int nblk = (batch + NS - 1) / NS;
  if (nblk > q->nblk_cap) {
    MCK(q->part.alloc((size_t)nblk * NPARAM * sizeof(float)));
    MCK(q->loss_part.alloc((size_t)nblk * sizeof(float)));
    q->nblk_cap = nblk;
  }
  return MIRT_OK;
}

int set_attrs() {
  static bool done = false;
  if (done) return MIRT_OK;
  MCK(cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)kGradSmem));
  MCK(cudaFuncSetAttribute(mlp_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)kInferSmem));
  done = true;
  return MIRT_OK;
}

GradArgs grad_args(mirt_mlp *q, const float *x, const float *y, long long n, const long long *idx,
                   int batch, unsigned long long seed) {
  GradArgs g{};
  g.x = x;
  g.y = y;
  g.n = n;
  g.idx = idx;
  g.batch = batch;
  g.seed = seed;
  g.step = q->step.as<int>();
  g.wb = q->wb.as<__nv_bfloat16>();
  g.part = q->part.as<float>();
  g.loss_part = q->loss_part.as<float>();
  return g;
}

AdamArgs adam_args(mirt_mlp *q, int nblk, int apply, float *grad_out, float *loss_hist) {
  AdamArgs a{};
  a.part = q->part.as<float>();
  a.loss_part = q->loss_part.as<float>();
  a.nblk = nblk;
  a.master = q->master.as<float>();
  a.m = q->m.as<float>();
  a.v = q->v.as<float>();
  a.wb = q->wb.as<__nv_bfloat16>();
  a.grad_out = grad_out;
  a.loss_hist = loss_hist;
  a.step = q->step.as<int>();
  a.lr = q->lr;
  a.beta1 = q->beta1;
  a.beta2 = q->beta2;
  a.eps = q->eps;
  a.apply = apply;
  return a;
}

}  // namespace

extern "C" {

int mirt_mlp_create(mirt_mlp **out, const float *params) {
  if (!out || !params) return api_fail(MIRT_ERR_ARG, "NULL argument");
  *out = nullptr;
  int rc = set_attrs();
  if (rc) return rc;
  auto *q = new mirt_mlp();
  auto bail = [&](int code) {
    delete q;
    return code;
  };
  if (q->master.alloc(NPARAM * sizeof(float)) || q->m.alloc(NPARAM * sizeof(float)) ||
      q->v.alloc(NPARAM * sizeof(float)) || q->wb.alloc(NPARAM * sizeof(__nv_bfloat16)) ||
      q->step.alloc(sizeof(int)) || q->grad.alloc(NPARAM * sizeof(float)))
    return bail(api_fail(MIRT_ERR_ALLOC, "MLP parameter buffers"));
  cudaError_t e = cudaMemcpy(q->master.p, params, NPARAM * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(q->m.p, 0, NPARAM * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(q->v.p, 0, NPARAM * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(q->step.p, 0, sizeof(int));
  if (e == cudaSuccess) {
    to_bf16_kernel<<<(NPARAM + 255) / 256, 256>>>(q->master.as<float>(),
                                                  q->wb.as<__nv_bfloat16>(), NPARAM);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return bail(api_fail(MIRT_ERR_CUDA, cudaGetErrorString(e)));
  *out = q;
  return MIRT_OK;
}

int mirt_mlp_params(mirt_mlp *q, float *params) {
  if (!q || !params) return api_fail(MIRT_ERR_ARG, "NULL argument");
  MCK(cudaMemcpy(params, q->master.p, NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
  return MIRT_OK;
}

int mirt_mlp_grad(mirt_mlp *q, const float *x, const float *y, int64_t n, float *grad,
                  float *loss, void *stream) try {
  if (!q || !x || !y || !grad) return api_fail(MIRT_ERR_ARG, "NULL argument");
  if (n < 1 || n > (1 << 30)) return api_fail(MIRT_ERR_ARG, "need 1 <= n <= 2^30");
  cudaStream_t st = as_stream(stream);
  int rc = ensure_batch(q, (int)n);
  if (rc) return rc;
  DMem idx, lh;
  std::vector<long long> hidx(n);
  for (long long i = 0; i < n; i++) hidx[i] = i;
  MCK(idx.alloc(n * sizeof(long long)));
  MCK(lh.alloc(sizeof(float)));
  MCK(cudaMemcpyAsync(idx.p, hidx.data(), n * sizeof(long long), cudaMemcpyHostToDevice, st));
  const int nblk = (int)((n + NS - 1) / NS);
  // a fixed-list gradient must not advance the step counter: use a scratch one
  DMem st0;
  MCK(st0.alloc(sizeof(int)));
  MCK(cudaMemsetAsync(st0.p, 0, sizeof(int), st));
  GradArgs g = grad_args(q, x, y, n, idx.as<long long>(), (int)n, 0);
  g.step = st0.as<int>();
  mlp_grad_kernel<<<nblk, NT, kGradSmem, st>>>(g);
  MCK(cudaGetLastError());
  AdamArgs a = adam_args(q, nblk, 0, q->grad.as<float>(), lh.as<float>());
  a.step = st0.as<int>();
  mlp_adam_kernel<<<(NPARAM + 255) / 256, 256, 0, st>>>(a);
  MCK(cudaGetLastError());
  MCK(cudaMemcpyAsync(grad, q->grad.p, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, st));
  float l = 0.f;
  MCK(cudaMemcpyAsync(&l, lh.p, sizeof(float), cudaMemcpyDeviceToHost, st));
  MCK(cudaStreamSynchronize(st));
  if (loss) *loss = l;
  return MIRT_OK;
} catch (const std::bad_alloc &) {
  return api_fail(MIRT_ERR_ALLOC, "out of host memory");
}

int mirt_mlp_train(mirt_mlp *q, const float *x, const float *y, int64_t n, int32_t batch,
                   int32_t steps, float lr, uint64_t seed, float *loss_hist, void *stream) try {
  if (!q || !x || !y) return api_fail(MIRT_ERR_ARG, "NULL argument");
  if (n < 1 || batch < 1 || batch > (1 << 24) || steps < 0 || !(lr > 0.f))
    return api_fail(MIRT_ERR_ARG, "need n >= 1, 1 <= batch <= 2^24, steps >= 0, lr > 0");
  cudaStream_t st = as_stream(stream);
  int rc = ensure_batch(q, batch);
  if (rc) return rc;
  q->lr = lr;
  int step0 = 0;
  MCK(cudaMemcpyAsync(&step0, q->step.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  MCK(cudaStreamSynchronize(st));
  MCK(q->losses.alloc((size_t)(step0 + steps + 1) * sizeof(float)));
  const int nblk = (batch + NS - 1) / NS;
  GradArgs g = grad_args(q, x, y, n, nullptr, batch, seed);
  AdamArgs a = adam_args(q, nblk, 1, nullptr, q->losses.as<float>());
  // one training step = three launches; capture a block of steps in a CUDA
  // graph and replay it (the step counter lives on the device)
  const int chunk = steps < 64 ? steps : 64;
  cudaGraphExec_t exec = nullptr;
  if (chunk > 0) {
    cudaStream_t cs;
    MCK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t graph;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    for (int i = 0; i < chunk && e == cudaSuccess; i++) {
      mlp_grad_kernel<<<nblk, NT, kGradSmem, cs>>>(g);
      mlp_adam_kernel<<<(NPARAM + 255) / 256, 256, 0, cs>>>(a);
      mlp_step_kernel<<<1, 1, 0, cs>>>(q->step.as<int>());
    }
    cudaError_t e2 = cudaStreamEndCapture(cs, &graph);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    if (e2 == cudaSuccess) cudaGraphDestroy(graph);
    cudaStreamDestroy(cs);
    if (e != cudaSuccess) return api_fail(MIRT_ERR_CUDA, std::string("training graph: ") + cudaGetErrorString(e));
  }
  int done = 0;
  cudaError_t e = cudaSuccess;
  while (e == cudaSuccess && done + chunk <= steps && chunk > 0) {
    e = cudaGraphLaunch(exec, st);
    done += chunk;
  }
  for (; e == cudaSuccess && done < steps; done++) {
    mlp_grad_kernel<<<nblk, NT, kGradSmem, st>>>(g);
    mlp_adam_kernel<<<(NPARAM + 255) / 256, 256, 0, st>>>(a);
    mlp_step_kernel<<<1, 1, 0, st>>>(q->step.as<int>());
    e = cudaGetLastError();
  }
  if (exec) cudaGraphExecDestroy(exec);
  MCK(e);
  if (loss_hist && steps > 0)
    MCK(cudaMemcpyAsync(loss_hist, q->losses.as<float>() + step0, steps * sizeof(float),
                        cudaMemcpyDeviceToHost, st));
  MCK(cudaStreamSynchronize(st));
  return MIRT_OK;
} catch (const std::bad_alloc &) {
  return api_fail(MIRT_ERR_ALLOC, "out of host memory");
}

int mirt_mlp_infer(mirt_mlp *q, const float *x, int64_t n, float mu, float sigma, float *yhat,
                   double *w, void *stream) {
  if (!q || !x || (!yhat && !w)) return api_fail(MIRT_ERR_ARG, "NULL argument");
  if (n < 0) return api_fail(MIRT_ERR_ARG, "n must be >= 0");
  if (n == 0) return MIRT_OK;
  cudaStream_t st = as_stream(stream);
  if (q->tensor_cores) {
    // tensor-core inference: 8 warps of 16 samples per CTA and pass
    long long nb = (n + 127) / 128;
    if (nb > 148 * 8) nb = 148 * 8;
    mlp_infer_mma_kernel<3><<<(unsigned)nb, NT, 0, st>>>(x, n, q->wb.as<__nv_bfloat16>(), mu,
                                                          sigma, yhat, w);
  } else {
    long long nb = (n + NS - 1) / NS;
    if (nb > 148 * 8) nb = 148 * 8;
    mlp_infer_kernel<<<(unsigned)nb, NT, kInferSmem, st>>>(x, n, q->wb.as<__nv_bfloat16>(), mu,
                                                            sigma, yhat, w);
  }
  MCK(cudaGetLastError());
  return MIRT_OK;
}

int mirt_mlp_set_tensor_cores(mirt_mlp *q, int32_t on) {
  if (!q) return api_fail(MIRT_ERR_ARG, "NULL argument");
  q->tensor_cores = on ? 1 : 0;
  return MIRT_OK;
}

int mirt_mlp_destroy(mirt_mlp *q) {
  if (q) {
    cudaDeviceSynchronize();
    delete q;
  }
  return MIRT_OK;
}

}  // extern "C"
