// sense.cu -- batched CG-SENSE on the device NUFFT.
//
// System (systems/Asense.m:53-56): A = [G diag(s_1); ...; G diag(s_C)], G the
// table NUFFT of the plan (one slice per problem, ncol = C coils).  Penalty
// (penalty/Reg1.m with its defaults: first-order differences, offsets
// [1 nx nx+1 nx-1] of penalty/penalty_offsets.m, 'tight' edges and
// distance_power 1 of penalty/Rweights.m): R = C'C = sum_m C_m' diag(w_m) C_m,
// w_m = beta / |offset_m|, over pixel pairs that are both inside the image.
// Solver (wls/qpwls_pcg1.m:94-189 with precon = 1): Fletcher-Reeves directions
// and the real step (ddir' ngrad) / (Adir' W Adir + ddir' R ddir), with Ax
// and R x carried along as the reference carries Ax and Cx.
//
// Every problem of the batch has its own scalars; all reductions are FP64
// (deterministic: one CTA per problem, fixed order); vectors are complex64.
// The iteration runs without host round trips.
#include "../../include/mirt_b200.h"

#include <cmath>
#include <new>
#include <string>
#include <vector>

#include "runtime.cuh"
#include "toeplitz.cuh"

using namespace mirt;

namespace {

#define SCK(call)                                                                     \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return api_fail(e_ == cudaErrorMemoryAllocation ? MIRT_ERR_ALLOC : MIRT_ERR_CUDA, \
                      std::string(#call) + ": " + cudaGetErrorString(e_));            \
  } while (0)

enum { SC_NEW = 0, SC_OLD, SC_GAMMA, SC_STEP, SC_DEN, SC_NUM, SC_DENR, SC_N };

unsigned nblocks(long long n, int t = 256) {
  long long b = (n + t - 1) / t;
  if (b > 148 * 16) b = 148 * 16;
  return (unsigned)(b < 1 ? 1 : b);
}

// z[s][p][c] = sens[s][p][c] x[s][p]
__global__ void k_expand(const float2 *__restrict__ x, const float2 *__restrict__ sens,
                         float2 *__restrict__ z, long long n, int C) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const float2 v = x[e / C], s = sens[e];
    z[e] = make_float2(s.x * v.x - s.y * v.y, s.x * v.y + s.y * v.x);
  }
}

// out[s][p] = sum_c conj(sens) z  (- sub[s][p] when sub is given)
__global__ void k_combine(const float2 *__restrict__ z, const float2 *__restrict__ sens,
                          const float2 *__restrict__ sub, float2 *__restrict__ out, long long np,
                          int C) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np;
       p += (long long)gridDim.x * blockDim.x) {
    float ar = 0.f, ai = 0.f;
    const float2 *zp = z + p * C, *sp = sens + p * C;
    for (int c = 0; c < C; c++) {
      const float2 a = sp[c], b = zp[c];
      ar = fmaf(a.x, b.x, fmaf(a.y, b.y, ar));
      ai = fmaf(a.x, b.y, fmaf(-a.y, b.x, ai));
    }
    if (sub) {
      ar -= sub[p].x;
      ai -= sub[p].y;
    }
    out[p] = make_float2(ar, ai);
  }
}

// r = W (y - Ax), W per sample (all coils) or 1
__global__ void k_resid(const float2 *__restrict__ y, const float2 *__restrict__ Ax,
                        const float *__restrict__ W, float2 *__restrict__ r, long long n, int C) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const float w = W ? W[e / C] : 1.f;
    r[e] = make_float2(w * (y[e].x - Ax[e].x), w * (y[e].y - Ax[e].y));
  }
}

// out = C'C x for the four offsets (1,0) (0,1) (1,1) (-1,1) in (n1, n2)
__global__ void k_reg(const float2 *__restrict__ x, float2 *__restrict__ out, int S, int N1,
                      int N2, const double *__restrict__ beta) {
  const long long np = (long long)N1 * N2;
  const long long n = (long long)S * np;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(e / np);
    const long long q = e - (long long)s * np;
    const int i1 = (int)(q % N1), i2 = (int)(q / N1);
    const float b = (float)beta[s];
    const float bd = (float)(beta[s] / sqrt(2.0));
    const float2 *xs = x + (long long)s * np;
    const float2 v = xs[q];
    float ar = 0.f, ai = 0.f;
    const int d1[4] = {1, 0, 1, -1}, d2[4] = {0, 1, 1, 1};
#pragma unroll
    for (int m = 0; m < 4; m++) {
      const float w = m < 2 ? b : bd;
      // pair (n, n - d)
      int j1 = i1 - d1[m], j2 = i2 - d2[m];
      if (j1 >= 0 && j1 < N1 && j2 >= 0) {
        const float2 u = xs[(long long)j2 * N1 + j1];
        ar += w * (v.x - u.x);
        ai += w * (v.y - u.y);
      }
      // pair (n + d, n)
      j1 = i1 + d1[m];
      j2 = i2 + d2[m];
      if (j1 >= 0 && j1 < N1 && j2 < N2) {
        const float2 u = xs[(long long)j2 * N1 + j1];
        ar += w * (v.x - u.x);
        ai += w * (v.y - u.y);
      }
    }
    out[e] = make_float2(ar, ai);
  }
}

// out[s] = Re sum conj(a) b over [off[s], off[s+1]) in FP64 (weights per
// element group of C when W is given), one CTA per segment, fixed order
__global__ void k_segdot(const float2 *__restrict__ a, const float2 *__restrict__ b,
                         const long long *__restrict__ off, const float *__restrict__ W, int C,
                         double *__restrict__ out, int stride) {
  __shared__ double part[256];
  const int s = blockIdx.x;
  const long long e0 = off[s], e1 = off[s + 1];
  double acc = 0.0;
  for (long long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
    const float2 u = a[e], v = b[e];
    double t = (double)u.x * v.x + (double)u.y * v.y;
    if (W) t *= (double)W[e / C];
    acc += t;
  }
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) part[threadIdx.x] += part[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[s * stride] = part[0];
}

// out = b - u - v (the negative gradient of the Gram form)
__global__ void k_sub2(const float2 *__restrict__ b, const float2 *__restrict__ u,
                       const float2 *__restrict__ v, float2 *__restrict__ out, long long n) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x)
    out[e] = make_float2(b[e].x - u[e].x - v[e].x, b[e].y - u[e].y - v[e].y);
}

// Fletcher-Reeves: gamma = new / old (0 on the first iteration or old = 0);
// ddir = pregrad + gamma ddir; old = new
__global__ void k_dir(const float2 *__restrict__ ngrad, float2 *__restrict__ ddir,
                      const double *__restrict__ sc, long long np, int S, int first) {
  const long long n = (long long)S * np;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(e / np);
    const double *c = sc + s * SC_N;
    double g = 0.0;
    if (!first && c[SC_OLD] != 0.0) g = c[SC_NEW] / c[SC_OLD];
    const float gf = (float)g;
    const float2 q = ngrad[e];
    float2 d = first ? q : ddir[e];
    if (!first) d = make_float2(q.x + gf * d.x, q.y + gf * d.y);
    ddir[e] = d;
  }
}

__global__ void k_scal_dir(double *sc, int S, int first) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  double *c = sc + s * SC_N;
  c[SC_GAMMA] = (first || c[SC_OLD] == 0.0) ? 0.0 : c[SC_NEW] / c[SC_OLD];
  c[SC_OLD] = c[SC_NEW];
}

__global__ void k_scal_step(double *sc, int S) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  double *c = sc + s * SC_N;
  const double den = c[SC_DEN] + c[SC_DENR];
  c[SC_STEP] = den == 0.0 ? 0.0 : c[SC_NUM] / den;
}

// v += step_s d over image vectors ([S][np]) or sample vectors (slice_of[m])
__global__ void k_axpy(float2 *__restrict__ v, const float2 *__restrict__ d,
                       const double *__restrict__ sc, long long n, long long np,
                       const int *__restrict__ slice_of, int C) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int s = slice_of ? slice_of[e / C] : (int)(e / np);
    const float st = (float)sc[s * SC_N + SC_STEP];
    const float2 a = v[e], b = d[e];
    v[e] = make_float2(fmaf(st, b.x, a.x), fmaf(st, b.y, a.y));
  }
}

// per-slice ||x - xref||^2 (FP64), one CTA per slice
__global__ void k_errnorm(const float2 *__restrict__ x, const float2 *__restrict__ xr,
                          long long np, double *__restrict__ out) {
  __shared__ double part[256];
  const int s = blockIdx.x;
  const float2 *a = x + (long long)s * np, *b = xr + (long long)s * np;
  double acc = 0.0;
  for (long long e = threadIdx.x; e < np; e += blockDim.x) {
    const double dx = (double)a[e].x - b[e].x, dy = (double)a[e].y - b[e].y;
    acc += dx * dx + dy * dy;
  }
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) part[threadIdx.x] += part[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[s] = part[0];
}

}  // namespace

struct mirt_sense {
  mirt_nufft *G = nullptr;
  int S = 0, C = 0, N1 = 0, N2 = 0;
  long long np = 0, M = 0;
  DMem sens, beta, z, ioff, soff, slice_of;
  std::vector<double> beta_host;
  mirt_toeplitz *T = nullptr;  // Gram operator and preconditioner (mirt_sense_toeplitz)
  ~mirt_sense() { delete T; }
};

namespace {

int sense_A(mirt_sense *op, const float2 *x, float2 *y, cudaStream_t st) {
  const long long n = (long long)op->S * op->np * op->C;
  k_expand<<<nblocks(n), 256, 0, st>>>(x, op->sens.as<float2>(), op->z.as<float2>(), n, op->C);
  SCK(cudaGetLastError());
  return mirt_nufft_forward(op->G, op->z.p, y, st);
}

int sense_At(mirt_sense *op, const float2 *y, float2 *x, const float2 *sub, cudaStream_t st) {
  int rc = mirt_nufft_adjoint(op->G, y, op->z.p, st);
  if (rc) return rc;
  const long long np = (long long)op->S * op->np;
  k_combine<<<nblocks(np), 256, 0, st>>>(op->z.as<float2>(), op->sens.as<float2>(), sub, x, np,
                                         op->C);
  SCK(cudaGetLastError());
  return MIRT_OK;
}

int sense_R(mirt_sense *op, const float2 *x, float2 *rx, cudaStream_t st) {
  const long long n = (long long)op->S * op->np;
  k_reg<<<nblocks(n), 256, 0, st>>>(x, rx, op->S, op->N1, op->N2, op->beta.as<double>());
  SCK(cudaGetLastError());
  return MIRT_OK;
}

}  // namespace

extern "C" {

int mirt_sense_create(mirt_sense **out, mirt_nufft *G, const void *sens, const double *beta,
                      void *stream) {
  if (!out || !G || !sens || !beta) return api_fail(MIRT_ERR_ARG, "NULL argument");
  *out = nullptr;
  if (G->gg.D != 2) return api_fail(MIRT_ERR_ARG, "CG-SENSE is provided for 2D plans");
  if (G->nslice > 1024) return api_fail(MIRT_ERR_ARG, "at most 1024 problems per plan");
  cudaStream_t st = as_stream(stream);
  auto *op = new mirt_sense();
  auto bail = [&](int code) {
    delete op;
    return code;
  };
  op->G = G;
  op->S = G->nslice;
  op->C = G->C;
  op->N1 = G->gg.N[0];
  op->N2 = G->gg.N[1];
  op->np = G->gg.npix;
  op->M = G->Mtot;
  const size_t nimg = (size_t)op->S * op->np;
  if (op->sens.alloc(nimg * op->C * sizeof(float2)) || op->beta.alloc(op->S * sizeof(double)) ||
      op->z.alloc(nimg * op->C * sizeof(float2)) ||
      op->ioff.alloc((op->S + 1) * sizeof(long long)) ||
      op->soff.alloc((op->S + 1) * sizeof(long long)) ||
      op->slice_of.alloc(std::max<long long>(op->M, 1) * sizeof(int)))
    return bail(api_fail(MIRT_ERR_ALLOC, "CG-SENSE buffers"));
  std::vector<long long> io(op->S + 1), so(op->S + 1);
  for (int s = 0; s <= op->S; s++) {
    io[s] = (long long)s * op->np;
    so[s] = G->ip->moff_host[s] * op->C;
  }
  cudaError_t e = cudaMemcpyAsync(op->sens.p, sens, nimg * op->C * sizeof(float2),
                                  cudaMemcpyDeviceToDevice, st);
  op->beta_host.assign(beta, beta + op->S);
  if (!e) e = cudaMemcpyAsync(op->beta.p, beta, op->S * sizeof(double), cudaMemcpyHostToDevice, st);
  if (!e) e = cudaMemcpyAsync(op->ioff.p, io.data(), io.size() * sizeof(long long),
                              cudaMemcpyHostToDevice, st);
  if (!e) e = cudaMemcpyAsync(op->soff.p, so.data(), so.size() * sizeof(long long),
                              cudaMemcpyHostToDevice, st);
  if (!e && op->S > 1)
    e = launch_fill_slice(G->ip->moff.as<long long>(), op->S, op->M, op->slice_of.as<int>(), st);
  else if (!e)
    e = cudaMemsetAsync(op->slice_of.p, 0, std::max<long long>(op->M, 1) * sizeof(int), st);
  if (!e) e = cudaStreamSynchronize(st);
  if (e) return bail(api_fail(MIRT_ERR_CUDA, cudaGetErrorString(e)));
  *out = op;
  return MIRT_OK;
}

int mirt_sense_forward(mirt_sense *op, const void *x, void *y, void *stream) {
  if (!op || !x || !y) return api_fail(MIRT_ERR_ARG, "NULL argument");
  return sense_A(op, static_cast<const float2 *>(x), static_cast<float2 *>(y), as_stream(stream));
}

int mirt_sense_adjoint(mirt_sense *op, const void *y, void *x, void *stream) {
  if (!op || !x || !y) return api_fail(MIRT_ERR_ARG, "NULL argument");
  return sense_At(op, static_cast<const float2 *>(y), static_cast<float2 *>(x), nullptr,
                  as_stream(stream));
}

int mirt_sense_reg(mirt_sense *op, const void *x, void *rx, void *stream) {
  if (!op || !x || !rx) return api_fail(MIRT_ERR_ARG, "NULL argument");
  return sense_R(op, static_cast<const float2 *>(x), static_cast<float2 *>(rx), as_stream(stream));
}

int mirt_sense_pcg(mirt_sense *op, void *x_, const void *y_, const float *W, int32_t niter,
                   int32_t flags, const void *xref_, double *nrmse, float *ms, void *stream) try {
  if (!op || !x_ || !y_) return api_fail(MIRT_ERR_ARG, "NULL argument");
  if (niter < 0) return api_fail(MIRT_ERR_ARG, "niter must be >= 0");
  const bool precon = flags & MIRT_PCG_CIRCULANT, gram = flags & MIRT_PCG_TOEPLITZ;
  if ((precon || gram) && !op->T)
    return api_fail(MIRT_ERR_ARG, "attach the Toeplitz operator first (mirt_sense_toeplitz)");
  if (gram && W) return api_fail(MIRT_ERR_ARG, "the Toeplitz Gram form takes no data weights");
  cudaStream_t st = as_stream(stream);
  const int S = op->S, C = op->C;
  const long long ni = (long long)S * op->np, ns = op->M * C;
  float2 *x = static_cast<float2 *>(x_);
  const float2 *y = static_cast<const float2 *>(y_);
  const float2 *xref = static_cast<const float2 *>(xref_);
  // data-side vectors: Ax, Adir, residual (form 1) or A'y, Gx, Gdir (Gram form)
  DMem Ax, Adir, r, Rx, Rdir, ngrad, pgrad, ddir, sc, err, refn;
  if (gram) {
    SCK(Ax.alloc(ni * sizeof(float2)));    // G x
    SCK(Adir.alloc(ni * sizeof(float2)));  // G ddir
    SCK(r.alloc(ni * sizeof(float2)));     // b = A'y
  } else {
    SCK(Ax.alloc(std::max<long long>(ns, 1) * sizeof(float2)));
    SCK(Adir.alloc(std::max<long long>(ns, 1) * sizeof(float2)));
    SCK(r.alloc(std::max<long long>(ns, 1) * sizeof(float2)));
  }
  SCK(Rx.alloc(ni * sizeof(float2)));
  SCK(Rdir.alloc(ni * sizeof(float2)));
  SCK(ngrad.alloc(ni * sizeof(float2)));
  if (precon) SCK(pgrad.alloc(ni * sizeof(float2)));
  SCK(ddir.alloc(ni * sizeof(float2)));
  SCK(sc.alloc(S * SC_N * sizeof(double)));
  SCK(cudaMemsetAsync(sc.p, 0, S * SC_N * sizeof(double), st));
  const bool track = xref && nrmse;
  if (track) {
    SCK(err.alloc((size_t)(niter + 1) * S * sizeof(double)));
    SCK(refn.alloc(S * sizeof(double)));
    DMem zero;
    SCK(zero.alloc(ni * sizeof(float2)));
    SCK(cudaMemsetAsync(zero.p, 0, ni * sizeof(float2), st));
    k_errnorm<<<S, 256, 0, st>>>(xref, zero.as<float2>(), op->np, refn.as<double>());
    k_errnorm<<<S, 256, 0, st>>>(x, xref, op->np, err.as<double>());
    SCK(cudaGetLastError());
  }
  std::vector<cudaEvent_t> ev;
  if (ms) {
    ev.resize(niter + 1);
    for (auto &e : ev) SCK(cudaEventCreate(&e));
    SCK(cudaEventRecord(ev[0], st));
  }
  auto cleanup = [&]() {
    for (auto &e : ev) cudaEventDestroy(e);
  };
  auto gram_apply = [&](const float2 *v, float2 *out) {
    return toep_gram_sense(op->T, v, op->sens.as<float2>(), out, st);
  };
  // data term and penalty of the initial estimate
  int rc = MIRT_OK;
  if (gram) {
    rc = sense_At(op, y, r.as<float2>(), nullptr, st);  // b = A'y
    if (!rc) rc = gram_apply(x, Ax.as<float2>());
  } else {
    rc = sense_A(op, x, Ax.as<float2>(), st);
  }
  if (!rc) rc = sense_R(op, x, Rx.as<float2>(), st);
  const long long *ioff = op->ioff.as<long long>(), *soff = op->soff.as<long long>();
  double *scp = sc.as<double>();
  for (int it = 1; it <= niter && !rc; it++) {
    const int first = it == 1;
    // negative gradient
    if (gram) {
      k_sub2<<<nblocks(ni), 256, 0, st>>>(r.as<float2>(), Ax.as<float2>(), Rx.as<float2>(),
                                          ngrad.as<float2>(), ni);
    } else {
      k_resid<<<nblocks(ns), 256, 0, st>>>(y, Ax.as<float2>(), W, r.as<float2>(), ns, C);
      rc = sense_At(op, r.as<float2>(), ngrad.as<float2>(), Rx.as<float2>(), st);
      if (rc) break;
    }
    // preconditioned gradient and the Fletcher-Reeves direction
    const float2 *pg = ngrad.as<float2>();
    if (precon) {
      rc = toep_precon_apply(op->T, ngrad.as<float2>(), pgrad.as<float2>(), st);
      if (rc) break;
      pg = pgrad.as<float2>();
    }
    k_segdot<<<S, 256, 0, st>>>(ngrad.as<float2>(), pg, ioff, nullptr, 1, scp + SC_NEW, SC_N);
    k_dir<<<nblocks(ni), 256, 0, st>>>(pg, ddir.as<float2>(), scp, op->np, S, first);
    k_scal_dir<<<1, 64 * ((S + 63) / 64), 0, st>>>(scp, S, first);
    // step: (ddir' ngrad) / (data curvature + ddir' R ddir)
    if (gram) {
      rc = gram_apply(ddir.as<float2>(), Adir.as<float2>());
    } else {
      rc = sense_A(op, ddir.as<float2>(), Adir.as<float2>(), st);
    }
    if (!rc) rc = sense_R(op, ddir.as<float2>(), Rdir.as<float2>(), st);
    if (rc) break;
    if (gram)
      k_segdot<<<S, 256, 0, st>>>(ddir.as<float2>(), Adir.as<float2>(), ioff, nullptr, 1,
                                  scp + SC_DEN, SC_N);
    else
      k_segdot<<<S, 256, 0, st>>>(Adir.as<float2>(), Adir.as<float2>(), soff, W, C, scp + SC_DEN,
                                  SC_N);
    k_segdot<<<S, 256, 0, st>>>(ddir.as<float2>(), Rdir.as<float2>(), ioff, nullptr, 1,
                                scp + SC_DENR, SC_N);
    k_segdot<<<S, 256, 0, st>>>(ddir.as<float2>(), ngrad.as<float2>(), ioff, nullptr, 1,
                                scp + SC_NUM, SC_N);
    k_scal_step<<<1, 64 * ((S + 63) / 64), 0, st>>>(scp, S);
    if (gram)
      k_axpy<<<nblocks(ni), 256, 0, st>>>(Ax.as<float2>(), Adir.as<float2>(), scp, ni, op->np,
                                          nullptr, 1);
    else
      k_axpy<<<nblocks(ns), 256, 0, st>>>(Ax.as<float2>(), Adir.as<float2>(), scp, ns, 0,
                                          op->slice_of.as<int>(), C);
    k_axpy<<<nblocks(ni), 256, 0, st>>>(Rx.as<float2>(), Rdir.as<float2>(), scp, ni, op->np,
                                        nullptr, 1);
    k_axpy<<<nblocks(ni), 256, 0, st>>>(x, ddir.as<float2>(), scp, ni, op->np, nullptr, 1);
    if (track) k_errnorm<<<S, 256, 0, st>>>(x, xref, op->np, err.as<double>() + (size_t)it * S);
    cudaError_t e = cudaGetLastError();
    if (e) rc = api_fail(MIRT_ERR_CUDA, std::string("CG iteration: ") + cudaGetErrorString(e));
    if (ms) cudaEventRecord(ev[it], st);
  }
  if (rc) {
    cleanup();
    return rc;
  }
  cudaError_t e = cudaStreamSynchronize(st);
  if (e) {
    cleanup();
    return api_fail(MIRT_ERR_CUDA, cudaGetErrorString(e));
  }
  if (ms)
    for (int it = 1; it <= niter; it++) cudaEventElapsedTime(&ms[it - 1], ev[0], ev[it]);
  cleanup();
  if (track) {
    std::vector<double> h((size_t)(niter + 1) * S), rn(S);
    SCK(cudaMemcpy(h.data(), err.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
    SCK(cudaMemcpy(rn.data(), refn.p, S * sizeof(double), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < h.size(); i++) {
      const double d = rn[i % S];
      nrmse[i] = d > 0 ? std::sqrt(h[i] / d) : std::sqrt(h[i]);
    }
  }
  return MIRT_OK;
} catch (const std::bad_alloc &) {
  return api_fail(MIRT_ERR_ALLOC, "out of host memory");
}

int mirt_sense_cg(mirt_sense *op, void *x, const void *y, const float *W, int32_t niter,
                  const void *xref, double *nrmse, float *ms, void *stream) {
  return mirt_sense_pcg(op, x, y, W, niter, 0, xref, nrmse, ms, stream);
}

namespace {
__global__ void k_square(const double *__restrict__ w, double *__restrict__ w2, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    w2[i] = w[i] * w[i];
}
}  // namespace

int mirt_sense_precon_dcf(mirt_sense *op, const double *om, const double *w, double blend,
                          void *stream) {
  if (!op || !om || !w) return api_fail(MIRT_ERR_ARG, "NULL argument");
  if (!op->T) return api_fail(MIRT_ERR_ARG, "mirt_sense_toeplitz must run first");
  if (!(blend >= 0.0 && blend <= 1.0)) return api_fail(MIRT_ERR_ARG, "blend must be in [0, 1]");
  cudaStream_t st = as_stream(stream);
  mirt_interp_plan *P = op->G->ip;
  const int Nd[2] = {op->N1, op->N2}, Kd[2] = {P->a.g.K[0], P->a.g.K[1]};
  const int Jd[2] = {P->a.g.J[0], P->a.g.J[1]}, Ld[2] = {P->a.g.L[0], P->a.g.L[1]};
  DMem w2;
  cudaError_t e = w2.alloc(std::max<long long>(op->M, 1) * sizeof(double));
  if (e) return api_fail(MIRT_ERR_ALLOC, "DCF preconditioner weights");
  if (op->M > 0) {
    long long nb = (op->M + 255) / 256;
    if (nb > 148 * 16) nb = 148 * 16;
    k_square<<<(unsigned)nb, 256, 0, st>>>(w, w2.as<double>(), op->M);
    e = cudaGetLastError();
    if (e) return api_fail(MIRT_ERR_CUDA, cudaGetErrorString(e));
  }
  mirt_toeplitz *Tw = nullptr;
  int rc = toep_create(&Tw, om, op->M, P->moff_host.data(), op->S, Nd, Kd, Jd, Ld,
                       w2.as<double>(), 1, st);
  if (rc) return rc;
  rc = toep_precon_dcf(op->T, Tw, blend, st);
  delete Tw;
  return rc;
}

int mirt_sense_toeplitz(mirt_sense *op, const double *om, void *stream) {
  if (!op || !om) return api_fail(MIRT_ERR_ARG, "NULL argument");
  cudaStream_t st = as_stream(stream);
  mirt_interp_plan *P = op->G->ip;
  const int Nd[2] = {op->N1, op->N2}, Kd[2] = {P->a.g.K[0], P->a.g.K[1]};
  const int Jd[2] = {P->a.g.J[0], P->a.g.J[1]}, Ld[2] = {P->a.g.L[0], P->a.g.L[1]};
  mirt_toeplitz *T = nullptr;
  int rc = toep_create(&T, om, op->M, P->moff_host.data(), op->S, Nd, Kd, Jd, Ld, nullptr, op->C,
                       st);
  if (rc) return rc;
  // mean coil power per problem, for the preconditioner
  std::vector<long long> off(op->S + 1);
  for (int s = 0; s <= op->S; s++) off[s] = (long long)s * op->np * op->C;
  DMem doff, pw;
  cudaError_t e = doff.alloc((op->S + 1) * sizeof(long long));
  if (!e) e = pw.alloc(op->S * sizeof(double));
  if (!e) e = cudaMemcpyAsync(doff.p, off.data(), off.size() * sizeof(long long),
                              cudaMemcpyHostToDevice, st);
  if (e) {
    delete T;
    return api_fail(MIRT_ERR_CUDA, cudaGetErrorString(e));
  }
  k_segdot<<<op->S, 256, 0, st>>>(op->sens.as<float2>(), op->sens.as<float2>(),
                                  doff.as<long long>(), nullptr, 1, pw.as<double>(), 1);
  std::vector<double> lam(op->S);
  e = cudaMemcpyAsync(lam.data(), pw.p, op->S * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (!e) e = cudaStreamSynchronize(st);
  if (e) {
    delete T;
    return api_fail(MIRT_ERR_CUDA, cudaGetErrorString(e));
  }
  for (auto &v : lam) v /= (double)op->np;
  rc = toep_precon_build(T, lam.data(), op->beta_host.data(), st);
  if (rc) {
    delete T;
    return rc;
  }
  delete op->T;
  op->T = T;
  return MIRT_OK;
}

int mirt_sense_warm_start(mirt_sense *op, void *x_, const void *y_, const float *W,
                          void *stream) {
  if (!op || !x_ || !y_) return api_fail(MIRT_ERR_ARG, "NULL argument");
  cudaStream_t st = as_stream(stream);
  const int S = op->S, C = op->C;
  const long long ni = (long long)S * op->np, ns = op->M * C;
  float2 *x = static_cast<float2 *>(x_);
  const float2 *y = static_cast<const float2 *>(y_);
  DMem zero, r, Ax, sc;
  SCK(zero.alloc(std::max<long long>(ns, 1) * sizeof(float2)));
  SCK(r.alloc(std::max<long long>(ns, 1) * sizeof(float2)));
  SCK(Ax.alloc(std::max<long long>(ns, 1) * sizeof(float2)));
  SCK(sc.alloc(S * SC_N * sizeof(double)));
  SCK(cudaMemsetAsync(zero.p, 0, std::max<long long>(ns, 1) * sizeof(float2), st));
  // x = A'(W y): the density-compensated "conjugate phase" image
  k_resid<<<nblocks(ns), 256, 0, st>>>(y, zero.as<float2>(), W, r.as<float2>(), ns, C);
  int rc = sense_At(op, r.as<float2>(), x, nullptr, st);
  if (!rc) rc = sense_A(op, x, Ax.as<float2>(), st);
  if (rc) return rc;
  // per problem: x *= Re<Ax, y> / ||Ax||^2 (the least-squares scale)
  double *scp = sc.as<double>();
  k_segdot<<<S, 256, 0, st>>>(Ax.as<float2>(), y, op->soff.as<long long>(), nullptr, 1,
                              scp + SC_NUM, SC_N);
  k_segdot<<<S, 256, 0, st>>>(Ax.as<float2>(), Ax.as<float2>(), op->soff.as<long long>(),
                              nullptr, 1, scp + SC_DEN, SC_N);
  k_scal_step<<<1, 64 * ((S + 63) / 64), 0, st>>>(scp, S);
  // x = 0 + step x
  DMem xc;
  SCK(xc.alloc(ni * sizeof(float2)));
  SCK(cudaMemcpyAsync(xc.p, x, ni * sizeof(float2), cudaMemcpyDeviceToDevice, st));
  SCK(cudaMemsetAsync(x, 0, ni * sizeof(float2), st));
  k_axpy<<<nblocks(ni), 256, 0, st>>>(x, xc.as<float2>(), scp, ni, op->np, nullptr, 1);
  SCK(cudaGetLastError());
  SCK(cudaStreamSynchronize(st));
  return MIRT_OK;
}

int mirt_sense_destroy(mirt_sense *op) {
  if (op) {
    cudaDeviceSynchronize();
    delete op;
  }
  return MIRT_OK;
}

}  // extern "C"
