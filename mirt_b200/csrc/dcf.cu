// dcf.cu -- density compensation weights on the project's NUFFT.
//
// Pipe & Menon iteration (mri/ir_mri_density_comp.m:203-281): starting from
// w = 1, repeat  goal = real(P P' w),  w = w ./ goal  until
// max |goal - 1| <= thresh, with at most niter + 1 updates (the reference
// tests `iter > niter` after the update), then scale w so that the point
// spread function G' w sums to prod(N ./ fov).  P is the table interpolator
// with the NUFFT's phase shift (nufft/nufft_table_interp.m:75-78 and
// nufft/nufft_table_adj.m:47-50), G the full NUFFT.  The one-step weights
// w = 1 ./ real(P (P' 1)) of ir_mri_dcf_jackson (:160-180) are here too.
//
// Precision: the spread / gather run in FP32 (the plan's kernels); the weights,
// the ratio update, the residual and the scaling sums are FP64.  A batch of
// slices (trajectories of uneven length in one plan) iterates together in one
// launch sequence; each slice stops on its own residual and is then frozen on
// the device, so no host round trip is needed per iteration.
#include "../../include/mirt_b200.h"

#include <cmath>
#include <string>
#include <vector>

#include "runtime.cuh"

using namespace mirt;

namespace {

#define DCK(call)                                                                     \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return api_fail(e_ == cudaErrorMemoryAllocation ? MIRT_ERR_ALLOC : MIRT_ERR_CUDA, \
                      std::string(#call) + ": " + cudaGetErrorString(e_));            \
  } while (0)

constexpr int kRun = 16;  // samples per thread in the update (one residual flush per run)

__global__ void fill_ones_kernel(double *w, long long M) {
  for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < M;
       m += (long long)gridDim.x * blockDim.x)
    w[m] = 1.0;
}

// FP64 weights -> complex64 samples for the spread
__global__ void w_to_c64_kernel(const double *__restrict__ w, long long M, float2 *__restrict__ f) {
  for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < M;
       m += (long long)gridDim.x * blockDim.x)
    f[m] = make_float2((float)w[m], 0.f);
}

// w <- w / real(g) on the active slices; residual max |goal - 1| per slice by
// an atomic max on the bit pattern (order-free for non-negative doubles).
__global__ void pipe_update_kernel(const float2 *__restrict__ g, const int *__restrict__ slice_of,
                                   long long M, const int *__restrict__ active,
                                   double *__restrict__ w, unsigned long long *resid_bits,
                                   int *bad) {
  const long long m0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) * kRun;
  if (m0 >= M) return;
  const long long m1 = min(M, m0 + kRun);
  int cur = -1;
  double rmax = 0.0;
  for (long long m = m0; m < m1; m++) {
    const int s = slice_of ? slice_of[m] : 0;
    if (s != cur) {
      if (cur >= 0 && active[cur])
        atomicMax(resid_bits + cur, (unsigned long long)__double_as_longlong(rmax));
      cur = s;
      rmax = 0.0;
    }
    if (!active[s]) continue;
    const double goal = (double)g[m].x;
    if (!(goal > 0.0)) {
      atomicOr(bad, 1);
      continue;
    }
    w[m] = w[m] / goal;
    rmax = fmax(rmax, fabs(goal - 1.0));
  }
  if (cur >= 0 && active[cur])
    atomicMax(resid_bits + cur, (unsigned long long)__double_as_longlong(rmax));
}

// After update `it`: record the residual and iteration of each active slice,
// freeze the slices that met the threshold, count the ones still active.
__global__ void pipe_finalize_kernel(int nslice, int it, double thresh, int *active,
                                     unsigned long long *resid_bits, double *resid, int *iters,
                                     int *nactive) {
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  for (int s = threadIdx.x; s < nslice; s += blockDim.x) {
    if (active[s]) {
      const double r = __longlong_as_double((long long)resid_bits[s]);
      resid[s] = r;
      iters[s] = it;
      if (r <= thresh)
        active[s] = 0;
      else
        atomicAdd(&cnt, 1);
    }
    resid_bits[s] = 0ull;
  }
  __syncthreads();
  if (threadIdx.x == 0) *nactive = cnt;
}

// Per-slice FP64 sum of real(x) over npix pixels, fixed summation order.
__global__ void psf_sum_kernel(const float2 *__restrict__ x, long long npix,
                               double *__restrict__ sums) {
  __shared__ double part[256];
  const float2 *xs = x + (long long)blockIdx.x * npix;
  double acc = 0.0;
  for (long long i = threadIdx.x; i < npix; i += blockDim.x) acc += (double)xs[i].x;
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) part[threadIdx.x] += part[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) sums[blockIdx.x] = part[0];
}

// w <- (target / sum_s) w per slice
__global__ void dcf_scale_kernel(double *__restrict__ w, const int *__restrict__ slice_of,
                                 long long M, const double *__restrict__ sums, double target) {
  for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < M;
       m += (long long)gridDim.x * blockDim.x) {
    const int s = slice_of ? slice_of[m] : 0;
    w[m] *= target / sums[s];
  }
}

__global__ void recip_real_kernel(const float2 *__restrict__ g, long long M, double *__restrict__ w,
                                  int *bad) {
  for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < M;
       m += (long long)gridDim.x * blockDim.x) {
    const double v = (double)g[m].x;
    if (v == 0.0) atomicOr(bad, 1);
    w[m] = 1.0 / v;
  }
}

unsigned grid_for(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > 148 * 32) b = 148 * 32;
  return (unsigned)b;
}

struct DcfBuffers {
  DMem f, g, slice_of;
  int alloc(mirt_nufft *p, cudaStream_t st) {
    const long long M = p->Mtot;
    DCK(f.alloc(std::max<long long>(M, 1) * sizeof(float2)));
    DCK(g.alloc(std::max<long long>(M, 1) * sizeof(float2)));
    if (p->nslice > 1) {
      DCK(slice_of.alloc(std::max<long long>(M, 1) * sizeof(int)));
      DCK(launch_fill_slice(p->ip->moff.as<long long>(), p->nslice, M, slice_of.as<int>(), st));
    }
    return MIRT_OK;
  }
};

// g = P P' f  (spread into the plan's grid, gather back; phase applied by the plan)
int ppt(mirt_nufft *p, const float2 *f, float2 *g, cudaStream_t st) {
  mirt_interp_plan *P = p->ip;
  DCK(launch_spread(P->a, P->t, P->ls, P->bin_start.as<int>(), f, p->grid.as<float2>(), st));
  DCK(launch_gather(P->ag, P->lg, p->grid.as<float2>(), g, st));
  return MIRT_OK;
}

// scale: sum(real(G' w)) = prod(N ./ fov) per slice (mri/ir_mri_density_comp.m:258-261)
int scale_to_psf(mirt_nufft *p, double *w, const double *fov, DcfBuffers &b, cudaStream_t st) {
  const long long M = p->Mtot;
  const int S = p->nslice;
  double target = 1.0;
  for (int d = 0; d < p->gg.D; d++) {
    const double fv = fov ? fov[d] : 1.0;
    if (!(fv > 0.0)) return api_fail(MIRT_ERR_ARG, "fov must be positive");
    target *= p->gg.N[d] / fv;
  }
  DMem x, sums;
  DCK(x.alloc((size_t)S * p->gg.npix * sizeof(float2)));
  DCK(sums.alloc(S * sizeof(double)));
  w_to_c64_kernel<<<grid_for(M, 256), 256, 0, st>>>(w, M, b.f.as<float2>());
  DCK(cudaGetLastError());
  int rc = mirt_nufft_adjoint(p, b.f.p, x.p, st);
  if (rc) return rc;
  psf_sum_kernel<<<S, 256, 0, st>>>(x.as<float2>(), p->gg.npix, sums.as<double>());
  DCK(cudaGetLastError());
  const int *slice_of = S > 1 ? b.slice_of.as<int>() : nullptr;
  dcf_scale_kernel<<<grid_for(M, 256), 256, 0, st>>>(w, slice_of, M, sums.as<double>(), target);
  DCK(cudaGetLastError());
  return MIRT_OK;
}

int check_plan(mirt_nufft *p, const double *w) {
  if (!p) return api_fail(MIRT_ERR_ARG, "nufft is NULL");
  if (!w) return api_fail(MIRT_ERR_ARG, "w is NULL");
  if (p->C != 1)
    return api_fail(MIRT_ERR_ARG,
                    "density compensation needs a single-column NUFFT plan (ncol = 1)");
  return MIRT_OK;
}

}  // namespace

extern "C" {

int mirt_dcf_pipe(mirt_nufft *p, double *w, int32_t init_ones, int32_t niter, double thresh,
                  const double *fov, int32_t *iters, double *resid, void *stream) {
  int rc = check_plan(p, w);
  if (rc) return rc;
  if (niter < 0 || !(thresh >= 0.0)) return api_fail(MIRT_ERR_ARG, "need niter >= 0, thresh >= 0");
  cudaStream_t st = as_stream(stream);
  const long long M = p->Mtot;
  const int S = p->nslice;
  DcfBuffers b;
  rc = b.alloc(p, st);
  if (rc) return rc;
  DMem active, rbits, rdev, idev, flags;
  DCK(active.alloc(S * sizeof(int)));
  DCK(rbits.alloc(S * sizeof(unsigned long long)));
  DCK(rdev.alloc(S * sizeof(double)));
  DCK(idev.alloc(S * sizeof(int)));
  DCK(flags.alloc(2 * sizeof(int)));  // [0] non-positive goal seen, [1] slices still active
  {
    std::vector<int> ones(S, 1);
    DCK(cudaMemcpyAsync(active.p, ones.data(), S * sizeof(int), cudaMemcpyHostToDevice, st));
  }
  DCK(cudaMemsetAsync(rbits.p, 0, S * sizeof(unsigned long long), st));
  DCK(cudaMemsetAsync(rdev.p, 0, S * sizeof(double), st));
  DCK(cudaMemsetAsync(idev.p, 0, S * sizeof(int), st));
  DCK(cudaMemsetAsync(flags.p, 0, 2 * sizeof(int), st));
  const int *slice_of = p->nslice > 1 ? b.slice_of.as<int>() : nullptr;
  if (init_ones) fill_ones_kernel<<<grid_for(M, 256), 256, 0, st>>>(w, M);
  DCK(cudaGetLastError());
  const long long nrun = (M + kRun - 1) / kRun;
  for (int it = 1; it <= niter + 1; it++) {
    w_to_c64_kernel<<<grid_for(M, 256), 256, 0, st>>>(w, M, b.f.as<float2>());
    DCK(cudaGetLastError());
    rc = ppt(p, b.f.as<float2>(), b.g.as<float2>(), st);
    if (rc) return rc;
    if (M > 0) {
      pipe_update_kernel<<<(unsigned)((nrun + 255) / 256), 256, 0, st>>>(
          b.g.as<float2>(), slice_of, M, active.as<int>(), w, rbits.as<unsigned long long>(),
          flags.as<int>());
      DCK(cudaGetLastError());
    }
    pipe_finalize_kernel<<<1, 256, 0, st>>>(S, it, thresh, active.as<int>(),
                                            rbits.as<unsigned long long>(), rdev.as<double>(),
                                            idev.as<int>(), flags.as<int>() + 1);
    DCK(cudaGetLastError());
    if (it % 4 == 0 || it == niter + 1) {
      int h[2];
      DCK(cudaMemcpyAsync(h, flags.p, sizeof h, cudaMemcpyDeviceToHost, st));
      DCK(cudaStreamSynchronize(st));
      if (h[0]) return api_fail(MIRT_ERR_ARG, "pipe bug: non-positive P P' w");
      if (h[1] == 0) break;
    }
  }
  {
    int h[2];
    DCK(cudaMemcpyAsync(h, flags.p, sizeof h, cudaMemcpyDeviceToHost, st));
    DCK(cudaStreamSynchronize(st));
    if (h[0]) return api_fail(MIRT_ERR_ARG, "pipe bug: non-positive P P' w");
  }
  rc = scale_to_psf(p, w, fov, b, st);
  if (rc) return rc;
  if (iters) DCK(cudaMemcpyAsync(iters, idev.p, S * sizeof(int), cudaMemcpyDeviceToHost, st));
  if (resid) DCK(cudaMemcpyAsync(resid, rdev.p, S * sizeof(double), cudaMemcpyDeviceToHost, st));
  DCK(cudaStreamSynchronize(st));
  return MIRT_OK;
}

int mirt_dcf_scale(mirt_nufft *p, double *w, const double *fov, void *stream) {
  int rc = check_plan(p, w);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  DcfBuffers b;
  rc = b.alloc(p, st);
  if (rc) return rc;
  rc = scale_to_psf(p, w, fov, b, st);
  if (rc) return rc;
  DCK(cudaStreamSynchronize(st));
  return MIRT_OK;
}

int mirt_dcf_jackson(mirt_nufft *p, double *w, void *stream) {
  int rc = check_plan(p, w);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  const long long M = p->Mtot;
  DcfBuffers b;
  rc = b.alloc(p, st);
  if (rc) return rc;
  DMem flags;
  DCK(flags.alloc(sizeof(int)));
  DCK(cudaMemsetAsync(flags.p, 0, sizeof(int), st));
  fill_ones_kernel<<<grid_for(M, 256), 256, 0, st>>>(w, M);
  w_to_c64_kernel<<<grid_for(M, 256), 256, 0, st>>>(w, M, b.f.as<float2>());
  DCK(cudaGetLastError());
  rc = ppt(p, b.f.as<float2>(), b.g.as<float2>(), st);
  if (rc) return rc;
  recip_real_kernel<<<grid_for(M, 256), 256, 0, st>>>(b.g.as<float2>(), M, w, flags.as<int>());
  DCK(cudaGetLastError());
  int h = 0;
  DCK(cudaMemcpyAsync(&h, flags.p, sizeof h, cudaMemcpyDeviceToHost, st));
  DCK(cudaStreamSynchronize(st));
  if (h) return api_fail(MIRT_ERR_ARG, "jackson: P P' 1 has a zero entry");
  return MIRT_OK;
}

}  // extern "C"
