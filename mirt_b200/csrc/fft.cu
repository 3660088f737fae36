// fft.cu -- batched DFT passes of the NUFFT's oversampled FFT (see fft.cuh).
//
// A pass transforms lines of length n = R1 * R2 in two radix stages (the
// four-step factorisation): with k = R2 k1 + q and p = p1 + R1 p2,
//   X[p1 + R1 p2] = sum_q W_R2^{p2 q} W_n^{p1 q} sum_k1 W_R1^{p1 k1} x[R2 k1 + q].
// Stage 1 loads the R1 elements of one (line, q) from global memory into
// registers, runs the radix-R1 DFT, multiplies by the twiddles W_n^{p1 q} and
// stores to shared memory; stage 2 reads the R2 values of one (line, p1),
// runs the radix-R2 DFT and stores the outputs to global memory.  Every
// element is read from global memory once and written once, and every read of
// a line precedes the block barrier that precedes its writes, so the passes
// along dimensions >= 2 run in place.
//
// A line's elements are vectors of vw consecutive complex values (coils, or
// consecutive grid points of the faster dimensions); lane v of a group serves
// element v of the vector, so every global access of a warp is a run of
// consecutive complex values and every shared-memory access is conflict-free
// (rows padded when vw < 16).
//
// Zero padding and crop: the forward passes read only the nin < n input
// elements that hold data; when nin <= n/2 the radix-R1 stage drops its first
// decimation-in-frequency butterfly level (half its inputs are zero).  The
// adjoint passes write only the nout outputs the crop keeps; when nout <= n/2
// the radix-R2 stage forms only the first half of its outputs.
//
// In-register DFTs: recursive radix-4/2 decimation in time with the twiddle
// constants cos(2 pi e/R), sin(2 pi e/R) evaluated by the compiler from their
// Taylor series in FP64; the pass twiddles W_n^{p1 q} come from an FP64-built
// table.  Arithmetic is FP32.
#include <utility>

#include "common.cuh"
#include "fft.cuh"

namespace mirt {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxLpb = 32;

// ---- compile-time twiddle constants ---------------------------------------
constexpr double kTwoPi = 6.283185307179586476925286766559;

__host__ __device__ constexpr double ct_cos(double x) {
  double s = 1.0, t = 1.0;
  for (int k = 1; k <= 24; k++) {
    t = -t * x * x / ((2.0 * k - 1.0) * (2.0 * k));
    s += t;
  }
  return s;
}

__host__ __device__ constexpr double ct_sin(double x) {
  double s = x, t = x;
  for (int k = 1; k <= 24; k++) {
    t = -t * x * x / ((2.0 * k) * (2.0 * k + 1.0));
    s += t;
  }
  return s;
}

// 2 pi e / R with e reduced into (-R/2, R/2], so |angle| <= pi
template <int R, int E>
struct Angle {
  static constexpr int e0 = ((E % R) + R) % R;
  static constexpr int e = 2 * e0 > R ? e0 - R : e0;
  static constexpr double value = kTwoPi * e / R;
};

__device__ __forceinline__ float2 cadd(float2 a, float2 b) {
  return make_float2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
  return make_float2(a.x - b.x, a.y - b.y);
}

// v * W_R^E with W_R = exp(-2 pi i / R) (forward) or exp(+2 pi i / R) (INV)
template <int R, int E, bool INV>
__device__ __forceinline__ float2 twmul(float2 v) {
  constexpr int e = ((E % R) + R) % R;
  if constexpr (e == 0) {
    return v;
  } else if constexpr (2 * e == R) {
    return make_float2(-v.x, -v.y);
  } else if constexpr (4 * e == R) {  // -i (forward), +i (inverse)
    return INV ? make_float2(-v.y, v.x) : make_float2(v.y, -v.x);
  } else if constexpr (4 * e == 3 * R) {  // +i (forward), -i (inverse)
    return INV ? make_float2(v.y, -v.x) : make_float2(-v.y, v.x);
  } else {
    constexpr float c = (float)ct_cos(Angle<R, E>::value);
    constexpr float s0 = (float)ct_sin(Angle<R, E>::value);
    constexpr float s = INV ? s0 : -s0;
    return make_float2(__fmaf_rn(v.x, c, -__fmul_rn(v.y, s)), __fmaf_rn(v.x, s, __fmul_rn(v.y, c)));
  }
}

// In-place DFT of R values in natural order.  R = A * B: A DFTs of length B on
// the stride-A subsequences, twiddles W_R^{a k1}, then B DFTs of length A.
template <int R, bool INV>
struct Dft {
  static __device__ __forceinline__ void run(float2 *x) {
    if constexpr (R == 1) {
    } else if constexpr (R == 2) {
      const float2 a = x[0], b = x[1];
      x[0] = cadd(a, b);
      x[1] = csub(a, b);
    } else if constexpr (R == 4) {
      const float2 t0 = cadd(x[0], x[2]), t1 = csub(x[0], x[2]);
      const float2 t2 = cadd(x[1], x[3]), t3 = twmul<4, 1, INV>(csub(x[1], x[3]));
      x[0] = cadd(t0, t2);
      x[2] = csub(t0, t2);
      x[1] = cadd(t1, t3);
      x[3] = csub(t1, t3);
    } else {
      constexpr int A = (R % 16 == 0) ? 4 : 2;
      constexpr int B = R / A;
      float2 y[A][B];
      sfor<A>([&](auto a) { sfor<B>([&](auto b) { y[a][b] = x[A * b + a]; }); });
      sfor<A>([&](auto a) { Dft<B, INV>::run(y[a]); });
      sfor<A>([&](auto a) {
        sfor<B>([&](auto k) {
          y[a][k] = twmul<R, decltype(a)::value * decltype(k)::value, INV>(y[a][k]);
        });
      });
      sfor<B>([&](auto k1) {
        float2 z[A];
        sfor<A>([&](auto a) { z[a] = y[a][k1]; });
        Dft<A, INV>::run(z);
        sfor<A>([&](auto k2) { x[k1 + B * k2] = z[k2]; });
      });
    }
  }
};

// DFT of R values whose upper half is zero: X[2m] = DFT_{R/2}(x)[m],
// X[2m+1] = DFT_{R/2}(x[j] W_R^j)[m].
template <int R, bool INV>
__device__ __forceinline__ void dft_half_in(float2 *x) {
  constexpr int H = R / 2;
  float2 a[H], b[H];
  sfor<H>([&](auto j) {
    a[j] = x[j];
    b[j] = twmul<R, decltype(j)::value, INV>(x[j]);
  });
  Dft<H, INV>::run(a);
  Dft<H, INV>::run(b);
  sfor<H>([&](auto k) {
    x[2 * k] = a[k];
    x[2 * k + 1] = b[k];
  });
}

// The first R/2 outputs of a DFT of R values: X[k] = E[k] + W_R^k O[k] (E, O the
// DFTs of the even and odd samples).
template <int R, bool INV>
__device__ __forceinline__ void dft_half_out(float2 *x) {
  constexpr int H = R / 2;
  float2 e[H], o[H];
  sfor<H>([&](auto j) {
    e[j] = x[2 * j];
    o[j] = x[2 * j + 1];
  });
  Dft<H, INV>::run(e);
  Dft<H, INV>::run(o);
  sfor<H>([&](auto k) { x[k] = cadd(e[k], twmul<R, decltype(k)::value, INV>(o[k])); });
}

// ---- the pass kernel ---------------------------------------------------------
// PRUNE: forward with nin <= n/2, or inverse with nout <= n/2.  VW: the vector
// width at compile time (8 or 16) with the element counts exactly the transform's
// (nin = n/2 pruned or n, nout = n/2 pruned or n: no bounds tests), or 0 (any
// width and counts, read from the pass).
template <int R1, int R2, bool INV, bool PRUNE, int VW>
__global__ void __launch_bounds__(kThreads, VW == 16 ? 3 : VW == 8 ? 2 : 1)
    fft_pass_kernel(FftPass P, int lpb, int pitch_rt) {
  constexpr bool EXACT = VW != 0;
  extern __shared__ __align__(16) float2 sm[];
  __shared__ long long base_in[kMaxLpb], base_out[kMaxLpb];
  __shared__ int snrow[kMaxLpb];
  const int vw = VW ? VW : P.vw;
  const int lvw = VW ? (VW == 16 ? 4 : 3) : __ffs(vw) - 1;
  const int pitch = VW ? R2 * VW + (VW < 16 ? VW : 0) : pitch_rt;
  const int nlines = P.nslice * P.nr2 * P.nr1 * P.nvec;
  const int g0 = blockIdx.x * lpb;
  if (threadIdx.x < lpb) {
    const int gl = g0 + threadIdx.x;
    long long bi = -1, bo = -1;
    int row = 0;
    if (gl < nlines) {
      int o = gl / P.nvec;
      const int w = gl - o * P.nvec;
      const int r1 = o % P.nr1;
      o /= P.nr1;
      const int r2 = o % P.nr2;
      const int s = o / P.nr2;
      bi = s * P.is[0] + r2 * P.is[1] + r1 * P.is[2] + (long long)w * vw;
      bo = s * P.os[0] + r2 * P.os[1] + r1 * P.os[2] + (long long)w * vw;
      row = r2 * P.nr1 + r1;
    }
    base_in[threadIdx.x] = bi;
    base_out[threadIdx.x] = bo;
    snrow[threadIdx.x] = row;
  }
  __syncthreads();

  // stage 1
  constexpr int KH = (PRUNE && !INV) ? R1 / 2 : R1;
  const int n1 = (lpb * R2) << lvw;
#pragma unroll 1
  for (int i = threadIdx.x; i < n1; i += kThreads) {
    const int v = i & (vw - 1);
    const int q = (i >> lvw) % R2;
    const int g = (i >> lvw) / R2;
    const long long bi = base_in[g];
    if (bi < 0) continue;
    const float2 *src = P.in + bi + v;
    float2 x[R1];
    if constexpr (EXACT) {
      // element k = R2 k1 + q at a running pointer (no hoisted per-element offsets)
      const float2 *sp = src + (long long)q * P.es_in;
      const long long st = (long long)R2 * P.es_in;
#pragma unroll
      for (int k1 = 0; k1 < R1; k1++) {
        x[k1] = make_float2(0.f, 0.f);
        if (k1 < KH) {
          x[k1] = *sp;
          sp += st;
        }
      }
    } else {
#pragma unroll
      for (int k1 = 0; k1 < R1; k1++) {
        const int k = R2 * k1 + q;
        x[k1] = make_float2(0.f, 0.f);
        if (k1 < KH && k < P.nin) x[k1] = src[(long long)k * P.es_in];
      }
    }
    if (P.sn_in) {
      const float2 *sr = P.sn_in + (long long)snrow[g] * P.nin + q;
#pragma unroll
      for (int k1 = 0; k1 < KH; k1++) {
        const int k = R2 * k1 + q;
        if (EXACT || k < P.nin) x[k1] = cmul(x[k1], __ldg(sr + R2 * k1));
      }
    }
    if (P.ph_in) {
#pragma unroll
      for (int k1 = 0; k1 < KH; k1++) x[k1] = cmulc(__ldg(P.ph_in + R2 * k1 + q), x[k1]);
    }
    if constexpr (PRUNE && !INV) {
      dft_half_in<R1, INV>(x);
    } else {
      Dft<R1, INV>::run(x);
    }
    {
      // this column's twiddles, two per 16-byte load
      const float4 *tw4 = reinterpret_cast<const float4 *>(P.tw) + q * (R1 / 2);
#pragma unroll
      for (int j = 0; j < R1 / 2; j++) {
        const float4 t = __ldg(tw4 + j);
        if (j > 0 || !P.tw_unit0) x[2 * j] = cmul(x[2 * j], make_float2(t.x, t.y));
        x[2 * j + 1] = cmul(x[2 * j + 1], make_float2(t.z, t.w));
      }
    }
    float2 *d = sm + (size_t)(g * R1) * pitch + (q << lvw) + v;
#pragma unroll
    for (int p1 = 0; p1 < R1; p1++) d[p1 * pitch] = x[p1];
  }
  __syncthreads();

  // stage 2
  constexpr int PH = (PRUNE && INV) ? R2 / 2 : R2;
  const int n2 = (lpb * R1) << lvw;
#pragma unroll 1
  for (int i = threadIdx.x; i < n2; i += kThreads) {
    const int v = i & (vw - 1);
    const int p1 = (i >> lvw) % R1;
    const int g = (i >> lvw) / R1;
    const long long bo = base_out[g];
    if (bo < 0) continue;
    float2 y[R2];
    const float2 *s = sm + (size_t)(g * R1 + p1) * pitch + v;
#pragma unroll
    for (int k2 = 0; k2 < R2; k2++) y[k2] = s[k2 << lvw];
    if constexpr (PRUNE && INV) {
      dft_half_out<R2, INV>(y);
    } else {
      Dft<R2, INV>::run(y);
    }
    float2 *dst = P.out + bo + v;
    const float2 *sr = P.sn_out ? P.sn_out + (long long)snrow[g] * P.nout : nullptr;
    if (EXACT && !sr && !P.ph_out) {
      float2 *dp = dst + (long long)p1 * P.es_out;
      const long long st = (long long)R1 * P.es_out;
#pragma unroll
      for (int p2 = 0; p2 < PH; p2++) {
        *dp = y[p2];
        dp += st;
      }
    } else {
#pragma unroll
      for (int p2 = 0; p2 < PH; p2++) {
        const int p = p1 + R1 * p2;
        if (EXACT || p < P.nout) {
          float2 val = y[p2];
          if (P.ph_out) val = cmul(val, __ldg(P.ph_out + p));
          if (sr) val = cmulc(__ldg(sr + p), val);
          dst[(long long)p * P.es_out] = val;
        }
      }
    }
  }
}

template <int R1, int R2>
cudaError_t launch_r(const FftPass &P, cudaStream_t st) {
  const int vw = P.vw;
  int lpb = kThreads / ((R1 < R2 ? R1 : R2) * vw);
  if (lpb < 1) lpb = 1;
  if (lpb > kMaxLpb) lpb = kMaxLpb;
  const int pitch = R2 * vw + (vw < 16 ? vw : 0);
  const size_t smem = (size_t)lpb * R1 * pitch * sizeof(float2);
  const long long nlines = (long long)P.nslice * P.nr2 * P.nr1 * P.nvec;
  if (nlines <= 0) return cudaSuccess;
  const unsigned grid = (unsigned)((nlines + lpb - 1) / lpb);
  const bool prune = P.inverse ? (2 * P.nout <= P.n) : (2 * P.nin <= P.n);
  auto pick = [&](auto kern) -> cudaError_t {
    cudaError_t e =
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, kThreads, smem, st>>>(P, lpb, pitch);
    return cudaGetLastError();
  };
  // the exact forms: 16- or 8-wide vectors, inputs and outputs exactly the
  // (pruned) halves or all n
  const int hin = prune && !P.inverse ? P.n / 2 : P.n, hout = prune && P.inverse ? P.n / 2 : P.n;
  const int exact = (P.nin == hin && P.nout == hout && (vw == 16 || vw == 8)) ? vw : 0;
  auto by_width = [&](auto k16, auto k8, auto k0) -> cudaError_t {
    return exact == 16 ? pick(k16) : exact == 8 ? pick(k8) : pick(k0);
  };
  if (P.inverse)
    return prune ? by_width(fft_pass_kernel<R1, R2, true, true, 16>,
                            fft_pass_kernel<R1, R2, true, true, 8>,
                            fft_pass_kernel<R1, R2, true, true, 0>)
                 : by_width(fft_pass_kernel<R1, R2, true, false, 16>,
                            fft_pass_kernel<R1, R2, true, false, 8>,
                            fft_pass_kernel<R1, R2, true, false, 0>);
  return prune ? by_width(fft_pass_kernel<R1, R2, false, true, 16>,
                          fft_pass_kernel<R1, R2, false, true, 8>,
                          fft_pass_kernel<R1, R2, false, true, 0>)
               : by_width(fft_pass_kernel<R1, R2, false, false, 16>,
                          fft_pass_kernel<R1, R2, false, false, 8>,
                          fft_pass_kernel<R1, R2, false, false, 0>);
}

// largest power of two dividing v, at most 16
int vec_width(long long v) {
  int w = 1;
  while (w < 16 && v % (2 * w) == 0) w *= 2;
  return w;
}

FftPass base_pass(const NufftFft &f, int d, int s0, int s1, bool inverse) {
  FftPass p{};
  p.nslice = s1 - s0;
  p.nr1 = p.nr2 = 1;
  p.n = f.g.K[d];
  p.inverse = inverse ? 1 : 0;
  p.tw = inverse ? f.twa[d] : f.twf[d];
  p.tw_unit0 = !inverse || !f.phase_folded;  // entry p1 = 0 is 1 for every column
  const float2 *ph = (f.gp && f.gp->tab[0] && !f.phase_folded) ? f.gp->tab[d] : nullptr;
  if (inverse)
    p.ph_in = ph;
  else
    p.ph_out = ph;
  return p;
}

}  // namespace

bool fft_len_ok(int n) { return n >= 64 && n <= 1024 && (n & (n - 1)) == 0; }

cudaError_t launch_fft_pass(const FftPass &p, cudaStream_t st) {
  if (p.vw < 1 || p.vw > 32 || (p.vw & (p.vw - 1)) || p.nr1 < 1 || p.nr2 < 1 || p.nvec < 1)
    return cudaErrorInvalidValue;
  if ((long long)p.nslice * p.nr2 * p.nr1 * p.nvec >= (1ll << 31)) return cudaErrorInvalidValue;
  switch (p.n) {
    case 64: return launch_r<8, 8>(p, st);
    case 128: return launch_r<8, 16>(p, st);
    case 256: return launch_r<16, 16>(p, st);
    case 512: return launch_r<16, 32>(p, st);
    case 1024: return launch_r<32, 32>(p, st);
    default: return cudaErrorInvalidValue;
  }
}

void fft_radix(int n, int *r1, int *r2) {
  int a = 0, b = 0;
  switch (n) {
    case 64: a = 8, b = 8; break;
    case 128: a = 8, b = 16; break;
    case 256: a = 16, b = 16; break;
    case 512: a = 16, b = 32; break;
    case 1024: a = 32, b = 32; break;
    default: break;
  }
  *r1 = a;
  *r2 = b;
}

int fft_nufft_passes(const NufftFft &f) { return f.g.D; }

cudaError_t fft_nufft_forward(const NufftFft &f, const float2 *x, float2 *grid, int s0, int s1,
                              cudaStream_t st) {
  const GlueGeom &g = f.g;
  const long long C = f.C, xs = g.npix * C, gs = g.ngrid * C;
  if (s1 <= s0 || C == 0) return cudaSuccess;
  const int N1 = g.N[0], N2 = g.N[1], N3 = g.N[2];
  const int K1 = g.K[0], K2 = g.K[1];
  float2 *gd = grid + s0 * gs;
  // dimension 1: image rows -> grid rows (times sn)
  {
    FftPass p = base_pass(f, 0, s0, s1, false);
    p.in = x + s0 * xs;
    p.out = gd;
    p.nr1 = g.D > 1 ? N2 : 1;
    p.nr2 = g.D > 2 ? N3 : 1;
    p.is[0] = xs;
    p.is[1] = (long long)N2 * N1 * C;
    p.is[2] = (long long)N1 * C;
    p.os[0] = gs;
    p.os[1] = (long long)K2 * K1 * C;
    p.os[2] = (long long)K1 * C;
    p.es_in = p.es_out = C;
    p.vw = vec_width(C);
    p.nvec = (int)(C / p.vw);
    p.nin = N1;
    p.nout = K1;
    p.sn_in = f.sn;
    cudaError_t e = launch_fft_pass(p, st);
    if (e != cudaSuccess || g.D == 1) return e;
  }
  // dimension 2, in place: the image rows of every plane n3 < N3
  {
    FftPass p = base_pass(f, 1, s0, s1, false);
    p.in = p.out = gd;
    p.nr1 = g.D > 2 ? N3 : 1;
    p.is[0] = p.os[0] = gs;
    p.is[2] = p.os[2] = (long long)K2 * K1 * C;
    p.es_in = p.es_out = (long long)K1 * C;
    p.vw = vec_width((long long)K1 * C);
    p.nvec = (int)((long long)K1 * C / p.vw);
    p.nin = N2;
    p.nout = K2;
    cudaError_t e = launch_fft_pass(p, st);
    if (e != cudaSuccess || g.D == 2) return e;
  }
  // dimension 3, in place
  {
    FftPass p = base_pass(f, 2, s0, s1, false);
    p.in = p.out = gd;
    p.is[0] = p.os[0] = gs;
    p.es_in = p.es_out = (long long)K2 * K1 * C;
    p.vw = vec_width(p.es_in);
    p.nvec = (int)(p.es_in / p.vw);
    p.nin = N3;
    p.nout = g.K[2];
    return launch_fft_pass(p, st);
  }
}

cudaError_t fft_nufft_adjoint(const NufftFft &f, float2 *grid, float2 *x, int s0, int s1,
                              cudaStream_t st) {
  const GlueGeom &g = f.g;
  const long long C = f.C, xs = g.npix * C, gs = g.ngrid * C;
  if (s1 <= s0 || C == 0) return cudaSuccess;
  const int N1 = g.N[0], N2 = g.N[1], N3 = g.N[2];
  const int K1 = g.K[0], K2 = g.K[1];
  float2 *gd = grid + s0 * gs;
  cudaError_t e = cudaSuccess;
  if (g.D > 2) {  // dimension 3, in place: planes n3 < N3 kept
    FftPass p = base_pass(f, 2, s0, s1, true);
    p.in = p.out = gd;
    p.is[0] = p.os[0] = gs;
    p.es_in = p.es_out = (long long)K2 * K1 * C;
    p.vw = vec_width(p.es_in);
    p.nvec = (int)(p.es_in / p.vw);
    p.nin = g.K[2];
    p.nout = N3;
    e = launch_fft_pass(p, st);
    if (e != cudaSuccess) return e;
  }
  if (g.D > 1) {  // dimension 2, in place: rows n2 < N2 of planes n3 < N3 kept
    FftPass p = base_pass(f, 1, s0, s1, true);
    p.in = p.out = gd;
    p.nr1 = g.D > 2 ? N3 : 1;
    p.is[0] = p.os[0] = gs;
    p.is[2] = p.os[2] = (long long)K2 * K1 * C;
    p.es_in = p.es_out = (long long)K1 * C;
    p.vw = vec_width((long long)K1 * C);
    p.nvec = (int)((long long)K1 * C / p.vw);
    p.nin = K2;
    p.nout = N2;
    e = launch_fft_pass(p, st);
    if (e != cudaSuccess) return e;
  }
  // dimension 1: grid rows -> image rows, cropped, times conj(sn)
  FftPass p = base_pass(f, 0, s0, s1, true);
  p.in = gd;
  p.out = x + s0 * xs;
  p.nr1 = g.D > 1 ? N2 : 1;
  p.nr2 = g.D > 2 ? N3 : 1;
  p.is[0] = gs;
  p.is[1] = (long long)K2 * K1 * C;
  p.is[2] = (long long)K1 * C;
  p.os[0] = xs;
  p.os[1] = (long long)N2 * N1 * C;
  p.os[2] = (long long)N1 * C;
  p.es_in = p.es_out = C;
  p.vw = vec_width(C);
  p.nvec = (int)(C / p.vw);
  p.nin = K1;
  p.nout = N1;
  p.sn_out = f.sn;
  return launch_fft_pass(p, st);
}

}  // namespace mirt
