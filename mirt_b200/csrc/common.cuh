// common.cuh -- shared definitions for the mirt_b200 sm_100a kernels.
//
// Device data layout (all FP32, complex = float2 interleaved):
//   grid   ck[k][b]   k = ((k3*K2 + k2)*K1 + k1) (K1 fastest, as MATLAB's
//                     column-major [K1,K2,K3]); b = column (coil) fastest.
//   samples fm[m][b]  m = sample, b = column fastest.
//   coords tm[d*M + m] FP64, the caller's column-major [M, D] array.
// Columns are innermost so that one warp can serve one sample for 32 coils
// with a single 256-byte coalesced access per tap.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

#define MIRT_DMAX 3
#define MIRT_JMAX 16

namespace mirt {

// Per-dimension geometry handed to the kernels by value.
struct Geom {
  int D;                  // 1..3
  int K[MIRT_DMAX];       // grid size per dimension
  int J[MIRT_DMAX];       // neighbours per dimension
  int L[MIRT_DMAX];       // table oversampling per dimension
  int ncenter[MIRT_DMAX]; // floor(J*L/2): table index of t - k == 0
  int tlen[MIRT_DMAX];    // J*L + 1
  long long kstride[MIRT_DMAX];  // grid point stride of each dimension
};

// Index selection exactly as the reference computes it in FP64
// (nufft/table/interp2_table1_for.c:63-71, def,table2.h:7-8):
//   koff = 1 + floor(t - J/2),  p = (t - k) * L,
//   order 0: n = floor(p + 0.5);  order 1: n = floor(p), a = p - n.
// The _rn intrinsics keep nvcc from contracting (t-k)*L + 0.5 into an FMA,
// which would round differently from the reference's separate mul and add.
__device__ __forceinline__ int koff_of(double t, int J) {
  return 1 + (int)floor(__dsub_rn(t, (double)J * 0.5));
}

__device__ __forceinline__ int tab0_index(double t, int k, int L) {
  const double p = __dmul_rn(__dsub_rn(t, (double)k), (double)L);
  return (int)floor(__dadd_rn(p, 0.5));
}

__device__ __forceinline__ int tab1_index(double t, int k, int L, float *alf) {
  const double p = __dmul_rn(__dsub_rn(t, (double)k), (double)L);
  const double n = floor(p);
  *alf = (float)__dsub_rn(p, n);
  return (int)n;
}

// k mod K into [0, K) for any integer k (the reference's mymod).
__device__ __forceinline__ int wrapk(int k, int K) {
  int r = k % K;
  return r < 0 ? r + K : r;
}

// The roundings are spelled out (one product, then one fused multiply-add per
// part) so that every kernel computing a product gets the same bits, whatever
// contraction the compiler would otherwise choose.
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(__fmaf_rn(a.x, b.x, -__fmul_rn(a.y, b.y)),
                     __fmaf_rn(a.x, b.y, __fmul_rn(a.y, b.x)));
}
// conj(a) * b
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(__fmaf_rn(a.x, b.x, __fmul_rn(a.y, b.y)),
                     __fmaf_rn(a.x, b.y, -__fmul_rn(a.y, b.x)));
}

// Static loop: f(std::integral_constant<int, i>{}) for i = 0 .. N-1, so that
// the index is a compile-time constant inside the body.
template <class F, int... I>
__device__ __forceinline__ void sfor_impl(F &f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, I>{}), ...);
}
template <int N, class F>
__device__ __forceinline__ void sfor(F &&f) {
  sfor_impl(f, std::make_integer_sequence<int, N>{});
}

}  // namespace mirt
