// toeplitz.cu -- the Gram operator T = G'WG of a 2D table NUFFT as a Toeplitz
// matrix embedded in a 2N1 x 2N2 circulant (systems/Gnufft_gram.m).
//
// Kernel (Gnufft_gram_init2, :183-198): the lags t[l] = sum_m w_m
// exp(i omega_m . l), |l_d| < N_d, come from two adjoint NUFFTs of w without
// phase shift: block1 = G1' w (lags l >= 0) and block2 = G2' w with omega_1
// negated (lags l1 <= 0, l2 >= 0); the other quadrants are their conjugates.
// The lag -N_d slots are zero, the kernel is made Hermitian by averaging with
// its conjugate mirror (systems/private/dsft_gram_hermitify.m) and
// transformed once.  Applying T (Gnufft_gram_mult, :339-348): zero-pad to
// 2N, FFT, multiply, inverse FFT, crop -- two FFTs of the padded image per
// column instead of a NUFFT pair.
//
// The same spectrum gives a circulant preconditioner for the regularised
// SENSE normal equations: P = crop C pad with C the circulant of spectrum
// 1 / max(lam Re H + r, floor), lam the mean coil power, r the spectrum of the
// quadratic first-order penalty, floor = 1e-3 max(lam Re H).  P is Hermitian
// positive definite (a compression of a positive circulant).
#include "../../include/mirt_b200.h"

#include <cmath>
#include <new>
#include <string>
#include <vector>

#include "toeplitz.cuh"

using namespace mirt;

namespace {

#define TCK(call)                                                                     \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return api_fail(e_ == cudaErrorMemoryAllocation ? MIRT_ERR_ALLOC : MIRT_ERR_CUDA, \
                      std::string(#call) + ": " + cudaGetErrorString(e_));            \
  } while (0)

#define TCF(call)                                                                     \
  do {                                                                                \
    cufftResult r_ = (call);                                                          \
    if (r_ != CUFFT_SUCCESS)                                                          \
      return api_fail(MIRT_ERR_FFT, std::string(#call) + " failed: " + std::to_string((int)r_)); \
  } while (0)

unsigned nblk(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  return (unsigned)(b < 1 ? 1 : b);
}

__global__ void k_w_to_c64(const double *__restrict__ w, long long M, float2 *__restrict__ f) {
  for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < M;
       m += (long long)gridDim.x * blockDim.x)
    f[m] = make_float2(w ? (float)w[m] : 1.f, 0.f);
}

__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }

// t at circular index (q1, q2) of the 2N grid, from the two blocks
__device__ __forceinline__ float2 lag(const float2 *b1, const float2 *b2, int q1, int q2, int N1,
                                      int N2) {
  if (q1 == N1 || q2 == N2) return make_float2(0.f, 0.f);
  const int l1 = q1 < N1 ? q1 : q1 - 2 * N1;
  const int l2 = q2 < N2 ? q2 : q2 - 2 * N2;
  if (l1 >= 0 && l2 >= 0) return b1[(long long)l2 * N1 + l1];
  if (l1 < 0 && l2 >= 0) return b2[(long long)l2 * N1 - l1];
  if (l1 >= 0) return conjf2(l1 == 0 ? b1[(long long)(-l2) * N1] : b2[(long long)(-l2) * N1 + l1]);
  return conjf2(b1[(long long)(-l2) * N1 - l1]);
}

// Hermitian circulant kernel [S][2N2][2N1]
__global__ void k_assemble(const float2 *__restrict__ b1, const float2 *__restrict__ b2,
                           float2 *__restrict__ c, int S, int N1, int N2) {
  const long long P = 4ll * N1 * N2, np = (long long)N1 * N2;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < S * P;
       e += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(e / P);
    const long long r = e - s * P;
    const int q1 = (int)(r % (2 * N1)), q2 = (int)(r / (2 * N1));
    const float2 *B1 = b1 + s * np, *B2 = b2 + s * np;
    const float2 a = lag(B1, B2, q1, q2, N1, N2);
    const float2 b = conjf2(lag(B1, B2, (2 * N1 - q1) % (2 * N1), (2 * N2 - q2) % (2 * N2), N1, N2));
    c[e] = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y + b.y));
  }
}

// u[s*nc + c][r2][r1] = x[s][r2][r1][c] (zero outside N), optionally times sens
__global__ void k_pad(const float2 *__restrict__ x, const float2 *__restrict__ sens,
                      float2 *__restrict__ u, int S, int nc, int N1, int N2, int xcols) {
  const long long P = 4ll * N1 * N2;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)S * nc * P;
       e += (long long)gridDim.x * blockDim.x) {
    const long long sc = e / P;
    const long long r = e - sc * P;
    const int r1 = (int)(r % (2 * N1)), r2 = (int)(r / (2 * N1));
    const int s = (int)(sc / nc), c = (int)(sc - (long long)s * nc);
    float2 v = make_float2(0.f, 0.f);
    if (r1 < N1 && r2 < N2) {
      const long long p = ((long long)s * N2 + r2) * N1 + r1;
      if (sens) {
        const float2 a = x[p], b = sens[p * nc + c];
        v = make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
      } else {
        v = x[p * xcols + c];
      }
    }
    u[e] = v;
  }
}

// u[s*nc + c] *= H[s] (complex) or Hp[s] (real)
__global__ void k_mul(float2 *__restrict__ u, const float2 *__restrict__ H,
                      const float *__restrict__ Hp, int S, int nc, long long P) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)S * nc * P;
       e += (long long)gridDim.x * blockDim.x) {
    const long long sc = e / P, k = e - sc * P;
    const int s = (int)(sc / nc);
    const float2 a = u[e];
    if (Hp) {
      const float h = Hp[s * P + k];
      u[e] = make_float2(a.x * h, a.y * h);
    } else {
      const float2 h = H[s * P + k];
      u[e] = make_float2(a.x * h.x - a.y * h.y, a.x * h.y + a.y * h.x);
    }
  }
}

// y[s][r2][r1][c] = scale u[s*nc + c][r2][r1] over the N1 x N2 corner
__global__ void k_crop(const float2 *__restrict__ u, float2 *__restrict__ y, int S, int nc,
                       int N1, int N2, float scale) {
  const long long np = (long long)N1 * N2, P = 4 * np;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)S * np * nc;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e % nc);
    const long long p = e / nc;
    const int s = (int)(p / np);
    const long long q = p - s * np;
    const int r1 = (int)(q % N1), r2 = (int)(q / N1);
    const float2 a = u[((long long)s * nc + c) * P + (long long)r2 * 2 * N1 + r1];
    y[e] = make_float2(scale * a.x, scale * a.y);
  }
}

// out[s][p] = scale sum_c conj(sens[s][p][c]) u[s*nc + c][p]
__global__ void k_crop_combine(const float2 *__restrict__ u, const float2 *__restrict__ sens,
                               float2 *__restrict__ out, int S, int nc, int N1, int N2,
                               float scale) {
  const long long np = (long long)N1 * N2, P = 4 * np;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < (long long)S * np;
       p += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(p / np);
    const long long q = p - s * np;
    const long long off = (long long)(q / N1) * 2 * N1 + q % N1;
    float ar = 0.f, ai = 0.f;
    for (int c = 0; c < nc; c++) {
      const float2 a = sens[p * nc + c], b = u[((long long)s * nc + c) * P + off];
      ar = fmaf(a.x, b.x, fmaf(a.y, b.y, ar));
      ai = fmaf(a.x, b.y, fmaf(-a.y, b.x, ai));
    }
    out[p] = make_float2(scale * ar, scale * ai);
  }
}

// per-slice max of lam_s Re H over the spectrum (one CTA per slice)
__global__ void k_specmax(const float2 *__restrict__ H, const double *__restrict__ lam, long long P,
                          float *__restrict__ mx) {
  __shared__ float part[256];
  const int s = blockIdx.x;
  float m = 0.f;
  for (long long k = threadIdx.x; k < P; k += blockDim.x)
    m = fmaxf(m, (float)lam[s] * H[s * P + k].x);
  part[threadIdx.x] = m;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) part[threadIdx.x] = fmaxf(part[threadIdx.x], part[threadIdx.x + h]);
    __syncthreads();
  }
  if (threadIdx.x == 0) mx[s] = part[0];
}

// Hp = 1 / max(lam Re H + r, 1e-3 max), r = beta [(2-2cos a) + (2-2cos b) +
// ((2-2cos(a+b)) + (2-2cos(b-a))) / sqrt(2)]
__global__ void k_precon(const float2 *__restrict__ H, const double *__restrict__ lam,
                         const double *__restrict__ beta, const float *__restrict__ mx,
                         float *__restrict__ Hp, int S, int N1, int N2) {
  const long long P = 4ll * N1 * N2;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < S * P;
       e += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(e / P);
    const long long k = e - s * P;
    const int f1 = (int)(k % (2 * N1)), f2 = (int)(k / (2 * N1));
    const double a = M_PI * f1 / N1, b = M_PI * f2 / N2;
    const double r = beta[s] * ((2 - 2 * cos(a)) + (2 - 2 * cos(b)) +
                                ((2 - 2 * cos(a + b)) + (2 - 2 * cos(b - a))) / sqrt(2.0));
    const double v = fmax(lam[s] * (double)H[e].x + r, 1e-3 * (double)mx[s]);
    Hp[e] = (float)(1.0 / v);
  }
}

// per slice: mean of max(Re Hw, 1e-3 max Re Hw) and of P1
__global__ void k_dcf_means(const float2 *__restrict__ Hw, const float *__restrict__ mxw,
                            const float *__restrict__ P1, long long P, double *__restrict__ mean) {
  __shared__ double pw[256], p1[256];
  const int s = blockIdx.x;
  const float fl = 1e-3f * mxw[s];
  double a = 0, b = 0;
  for (long long k = threadIdx.x; k < P; k += blockDim.x) {
    a += (double)fmaxf(Hw[s * P + k].x, fl);
    b += (double)P1[s * P + k];
  }
  pw[threadIdx.x] = a;
  p1[threadIdx.x] = b;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      pw[threadIdx.x] += pw[threadIdx.x + h];
      p1[threadIdx.x] += p1[threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    mean[2 * s] = pw[0] / (double)P;
    mean[2 * s + 1] = p1[0] / (double)P;
  }
}

__global__ void k_dcf_blend(const float2 *__restrict__ Hw, const float *__restrict__ mxw,
                            const float *__restrict__ P1, const double *__restrict__ mean,
                            double blend, float *__restrict__ Hp, int S, long long P) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < S * P;
       e += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(e / P);
    const double pw = (double)fmaxf(Hw[e].x, 1e-3f * mxw[s]);
    Hp[e] = (float)(blend * pw / mean[2 * s] + (1.0 - blend) * (double)P1[e] / mean[2 * s + 1]);
  }
}

int make_plan(cufftHandle *h, int N1, int N2, int batch) {
  int n[2] = {2 * N2, 2 * N1};
  const int P = 4 * N1 * N2;
  TCF(cufftPlanMany(h, 2, n, nullptr, 1, P, nullptr, 1, P, CUFFT_C2C, batch));
  return MIRT_OK;
}

int fft(cufftHandle h, float2 *u, int dir, cudaStream_t st) {
  TCF(cufftSetStream(h, st));
  TCF(cufftExecC2C(h, reinterpret_cast<cufftComplex *>(u), reinterpret_cast<cufftComplex *>(u),
                   dir));
  return MIRT_OK;
}

}  // namespace

namespace mirt {

int toep_create(mirt_toeplitz **out, const double *om, long long M, const long long *moff,
                int nslice, const int *Nd, const int *Kd, const int *Jd, const int *Ld,
                const double *w, int ncol, cudaStream_t st) try {
  if (!out || !om || !Nd || !Kd || !Jd || !Ld) return api_fail(MIRT_ERR_ARG, "NULL argument");
  *out = nullptr;
  if (ncol < 1 || nslice < 1) return api_fail(MIRT_ERR_ARG, "need ncol >= 1 and nslice >= 1");
  // the two adjoint NUFFTs without phase shift: omega and omega with omega_1 negated
  std::vector<double> om2(om, om + 2 * M);
  for (long long m = 0; m < M; m++) om2[m] = -om2[m];
  const double zero[2] = {0.0, 0.0};
  std::vector<int64_t> mo;
  if (moff) mo.assign(moff, moff + nslice + 1);
  mirt_nufft *g1 = nullptr, *g2 = nullptr;
  int rc = mirt_nufft_create(&g1, 2, Nd, Kd, Jd, Ld, zero, om, M, moff ? mo.data() : nullptr,
                             nslice, 1, st);
  if (rc) return rc;
  rc = mirt_nufft_create(&g2, 2, Nd, Kd, Jd, Ld, zero, om2.data(), M,
                         moff ? mo.data() : nullptr, nslice, 1, st);
  if (rc) {
    mirt_nufft_destroy(g1);
    return rc;
  }
  auto *T = new mirt_toeplitz();
  T->S = nslice;
  T->N1 = Nd[0];
  T->N2 = Nd[1];
  T->ncol = ncol;
  const long long np = (long long)T->N1 * T->N2, P = 4 * np;
  DMem f, b1, b2;
  auto fin = [&](int code) {
    mirt_nufft_destroy(g1);
    mirt_nufft_destroy(g2);
    if (code) delete T;
    return code;
  };
  if (f.alloc(std::max<long long>(M, 1) * sizeof(float2)) ||
      b1.alloc(nslice * np * sizeof(float2)) || b2.alloc(nslice * np * sizeof(float2)) ||
      T->H.alloc(nslice * P * sizeof(float2)) ||
      T->pad.alloc((size_t)nslice * ncol * P * sizeof(float2)))
    return fin(api_fail(MIRT_ERR_ALLOC, "Toeplitz buffers"));
  k_w_to_c64<<<nblk(M), 256, 0, st>>>(w, M, f.as<float2>());
  rc = mirt_nufft_adjoint(g1, f.p, b1.p, st);
  if (!rc) rc = mirt_nufft_adjoint(g2, f.p, b2.p, st);
  if (rc) return fin(rc);
  k_assemble<<<nblk(nslice * P), 256, 0, st>>>(b1.as<float2>(), b2.as<float2>(), T->H.as<float2>(),
                                               nslice, T->N1, T->N2);
  if (cudaGetLastError() != cudaSuccess) return fin(api_fail(MIRT_ERR_CUDA, "kernel assembly"));
  rc = make_plan(&T->fft_1, T->N1, T->N2, nslice);
  if (rc) return fin(rc);
  T->ok_1 = true;
  if (ncol > 1) {
    rc = make_plan(&T->fft_n, T->N1, T->N2, nslice * ncol);
    if (rc) return fin(rc);
    T->ok_n = true;
  }
  rc = fft(T->fft_1, T->H.as<float2>(), CUFFT_FORWARD, st);
  if (rc) return fin(rc);
  if (cudaStreamSynchronize(st) != cudaSuccess) return fin(api_fail(MIRT_ERR_CUDA, "Toeplitz set-up"));
  *out = T;
  return fin(MIRT_OK);
} catch (const std::bad_alloc &) {
  return api_fail(MIRT_ERR_ALLOC, "out of host memory");
}

int toep_gram_sense(mirt_toeplitz *T, const float2 *x, const float2 *sens, float2 *out,
                    cudaStream_t st) {
  const int S = T->S, nc = T->ncol;
  const long long P = 4ll * T->N1 * T->N2;
  cufftHandle h = nc > 1 ? T->fft_n : T->fft_1;
  float2 *u = T->pad.as<float2>();
  k_pad<<<nblk(S * nc * P), 256, 0, st>>>(x, sens, u, S, nc, T->N1, T->N2, 1);
  int rc = fft(h, u, CUFFT_FORWARD, st);
  if (rc) return rc;
  k_mul<<<nblk(S * nc * P), 256, 0, st>>>(u, T->H.as<float2>(), nullptr, S, nc, P);
  rc = fft(h, u, CUFFT_INVERSE, st);
  if (rc) return rc;
  k_crop_combine<<<nblk((long long)S * T->N1 * T->N2), 256, 0, st>>>(u, sens, out, S, nc, T->N1,
                                                                     T->N2, 1.f / (float)P);
  TCK(cudaGetLastError());
  return MIRT_OK;
}

int toep_precon_build(mirt_toeplitz *T, const double *lam, const double *beta, cudaStream_t st) {
  const int S = T->S;
  const long long P = 4ll * T->N1 * T->N2;
  DMem dl, db, mx;
  TCK(dl.alloc(S * sizeof(double)));
  TCK(db.alloc(S * sizeof(double)));
  TCK(mx.alloc(S * sizeof(float)));
  TCK(T->Hp.alloc(S * P * sizeof(float)));
  TCK(cudaMemcpyAsync(dl.p, lam, S * sizeof(double), cudaMemcpyHostToDevice, st));
  TCK(cudaMemcpyAsync(db.p, beta, S * sizeof(double), cudaMemcpyHostToDevice, st));
  k_specmax<<<S, 256, 0, st>>>(T->H.as<float2>(), dl.as<double>(), P, mx.as<float>());
  k_precon<<<nblk(S * P), 256, 0, st>>>(T->H.as<float2>(), dl.as<double>(), db.as<double>(),
                                        mx.as<float>(), T->Hp.as<float>(), S, T->N1, T->N2);
  TCK(cudaGetLastError());
  TCK(cudaStreamSynchronize(st));
  return MIRT_OK;
}

int toep_precon_dcf(mirt_toeplitz *T, const mirt_toeplitz *Tw, double blend, cudaStream_t st) {
  const int S = T->S;
  const long long P = 4ll * T->N1 * T->N2;
  if (!T->Hp.p || !Tw || Tw->S != S || Tw->N1 != T->N1 || Tw->N2 != T->N2)
    return api_fail(MIRT_ERR_ARG, "preconditioner kernels of different shapes");
  if (!T->Hp1.p) {  // keep the unweighted spectrum the first time
    TCK(T->Hp1.alloc(S * P * sizeof(float)));
    TCK(cudaMemcpyAsync(T->Hp1.p, T->Hp.p, S * P * sizeof(float), cudaMemcpyDeviceToDevice, st));
  }
  DMem one, mx, mean;
  std::vector<double> ones(S, 1.0);
  TCK(one.alloc(S * sizeof(double)));
  TCK(mx.alloc(S * sizeof(float)));
  TCK(mean.alloc(2 * S * sizeof(double)));
  TCK(cudaMemcpyAsync(one.p, ones.data(), S * sizeof(double), cudaMemcpyHostToDevice, st));
  k_specmax<<<S, 256, 0, st>>>(Tw->H.as<float2>(), one.as<double>(), P, mx.as<float>());
  k_dcf_means<<<S, 256, 0, st>>>(Tw->H.as<float2>(), mx.as<float>(), T->Hp1.as<float>(), P,
                                 mean.as<double>());
  k_dcf_blend<<<nblk(S * P), 256, 0, st>>>(Tw->H.as<float2>(), mx.as<float>(), T->Hp1.as<float>(),
                                           mean.as<double>(), blend, T->Hp.as<float>(), S, P);
  TCK(cudaGetLastError());
  TCK(cudaStreamSynchronize(st));
  return MIRT_OK;
}

int toep_precon_apply(mirt_toeplitz *T, const float2 *x, float2 *out, cudaStream_t st) {
  const int S = T->S;
  const long long P = 4ll * T->N1 * T->N2;
  float2 *u = T->pad.as<float2>();  // the first S planes of the work grid
  k_pad<<<nblk(S * P), 256, 0, st>>>(x, nullptr, u, S, 1, T->N1, T->N2, 1);
  int rc = fft(T->fft_1, u, CUFFT_FORWARD, st);
  if (rc) return rc;
  k_mul<<<nblk(S * P), 256, 0, st>>>(u, nullptr, T->Hp.as<float>(), S, 1, P);
  rc = fft(T->fft_1, u, CUFFT_INVERSE, st);
  if (rc) return rc;
  k_crop<<<nblk((long long)S * T->N1 * T->N2), 256, 0, st>>>(u, out, S, 1, T->N1, T->N2,
                                                            1.f / (float)P);
  TCK(cudaGetLastError());
  return MIRT_OK;
}

}  // namespace mirt

extern "C" {

int mirt_toeplitz_create(mirt_toeplitz **out, const double *om, int64_t M,
                         const int64_t *slice_moff, int32_t nslice, const int32_t *Nd,
                         const int32_t *Kd, const int32_t *Jd, const int32_t *Ld, const double *w,
                         int32_t ncol, void *stream) {
  std::vector<long long> mo;
  if (slice_moff) mo.assign(slice_moff, slice_moff + nslice + 1);
  return toep_create(out, om, M, slice_moff ? mo.data() : nullptr, nslice, Nd, Kd, Jd, Ld, w,
                     ncol, as_stream(stream));
}

int mirt_toeplitz_apply(mirt_toeplitz *T, const void *x, void *y, void *stream) {
  if (!T || !x || !y) return api_fail(MIRT_ERR_ARG, "NULL argument");
  cudaStream_t st = as_stream(stream);
  const int S = T->S, nc = T->ncol;
  const long long P = 4ll * T->N1 * T->N2;
  cufftHandle h = nc > 1 ? T->fft_n : T->fft_1;
  float2 *u = T->pad.as<float2>();
  k_pad<<<nblk(S * nc * P), 256, 0, st>>>(static_cast<const float2 *>(x), nullptr, u, S, nc, T->N1,
                                          T->N2, nc);
  int rc = fft(h, u, CUFFT_FORWARD, st);
  if (rc) return rc;
  k_mul<<<nblk(S * nc * P), 256, 0, st>>>(u, T->H.as<float2>(), nullptr, S, nc, P);
  rc = fft(h, u, CUFFT_INVERSE, st);
  if (rc) return rc;
  k_crop<<<nblk((long long)S * T->N1 * T->N2 * nc), 256, 0, st>>>(
      u, static_cast<float2 *>(y), S, nc, T->N1, T->N2, 1.f / (float)P);
  TCK(cudaGetLastError());
  return MIRT_OK;
}

int mirt_toeplitz_destroy(mirt_toeplitz *T) {
  if (T) {
    cudaDeviceSynchronize();
    delete T;
  }
  return MIRT_OK;
}

}  // extern "C"
