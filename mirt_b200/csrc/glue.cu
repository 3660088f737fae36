// glue.cu -- elementwise kernels around the interpolation and the FFT.
//
//   deapod_image_cm x .* sn into the coil-major FFT input, zero-padded at the end of
//                   every dimension to Kd (nufft/nufft.m:139-140, nufft/fftn_fast.m:22-26);
//                   the padding is written once, this kernel writes the image region
//   crop_deapod_cm  crop [Kd] -> [Nd] and multiply by conj(sn) (nufft/nufft_adj.m:63-80),
//                   from the coil-major FFT output back to the coil-innermost image
//   transpose_cols  coil-major <-> coil-innermost grid between the FFT and the
//                   interpolation, optionally times newfft's phase_before over the
//                   grid or its conjugate (nufft/newfft.m:511-520,
//                   nufft/private/newfft_approx_for.m:32-34, newfft_approx_adj.m:56-58)
//   om_to_tm     tm = om / (2 pi / K) in FP64 and the n_shift phase
//                exp(i om . n_shift) (nufft/nufft_table_interp.m:36-40,
//                nufft/nufft_table_init.m:48-50)
//   split <-> interleaved conversions for the FP64 split-complex mex layout
//                (column n of [*, N] <-> innermost column of the device layout)
#include "glue.cuh"

namespace mirt {

// Image tiles of 32 n1 x 32 coils of one image row (n2 + N2 n3) of one slice:
// blockIdx.x = image row (slices outer), y = n1 block, z = coil block.  The
// grid row of an image row is its own index in the K grid (the image sits at
// the start of every dimension).
struct ImageTile {
  long long s, r, krow;
  int n1_0, c0;
};

__device__ __forceinline__ ImageTile image_tile(const GlueGeom &g) {
  ImageTile t;
  const long long row = blockIdx.x;
  const long long rows_per_slice = g.npix / g.N[0];
  t.s = row / rows_per_slice;
  t.r = row - t.s * rows_per_slice;
  t.n1_0 = blockIdx.y * 32;
  t.c0 = blockIdx.z * 32;
  long long kstr = 1, rem = t.r;
  t.krow = 0;
  for (int d = 1; d < g.D; d++) {
    const long long nd = rem % g.N[d];
    rem /= g.N[d];
    t.krow += nd * kstr;
    kstr *= g.K[d];
  }
  return t;
}

// x[s][n][c] (coil innermost) .* sn  ->  pad[s][c][k] on the image region only;
// the rest of pad is the zero padding, written once when the plan is made.
__global__ void __launch_bounds__(256) deapod_image_cm_kernel(const float2 *__restrict__ x,
                                                              const float2 *__restrict__ sn,
                                                              float2 *__restrict__ pad,
                                                              GlueGeom g, int C) {
  __shared__ float2 tile[32][33];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const long long krows = g.ngrid / g.K[0];
  const ImageTile t = image_tile(g);
  for (int i = ty; i < 32; i += 8) {
    const int n1 = t.n1_0 + i;
    const int c = t.c0 + tx;
    float2 v = make_float2(0.f, 0.f);
    if (c < C && n1 < g.N[0]) {
      const long long n = t.r * g.N[0] + n1;
      const float2 a = x[(t.s * g.npix + n) * C + c];
      const float2 b = sn[n];
      v = make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
    }
    tile[i][tx] = v;
  }
  __syncthreads();
  for (int i = ty; i < 32; i += 8) {
    const int c = t.c0 + i;
    const int n1 = t.n1_0 + tx;
    if (c < C && n1 < g.N[0]) pad[((t.s * C + c) * krows + t.krow) * g.K[0] + n1] = tile[tx][i];
  }
}

// grid[s][c][k] (coil outermost)  ->  crop to N, .* conj(sn)  ->  x[s][n][c]
__global__ void __launch_bounds__(256) crop_deapod_cm_kernel(const float2 *__restrict__ grid,
                                                             const float2 *__restrict__ sn,
                                                             float2 *__restrict__ x, GlueGeom g,
                                                             int C) {
  __shared__ float2 tile[32][33];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const long long krows = g.ngrid / g.K[0];
  const ImageTile t = image_tile(g);
  for (int i = ty; i < 32; i += 8) {
    const int c = t.c0 + i;
    const int n1 = t.n1_0 + tx;
    float2 v = make_float2(0.f, 0.f);
    if (c < C && n1 < g.N[0]) v = grid[((t.s * C + c) * krows + t.krow) * g.K[0] + n1];
    tile[i][tx] = v;
  }
  __syncthreads();
  for (int i = ty; i < 32; i += 8) {
    const int n1 = t.n1_0 + i;
    const int c = t.c0 + tx;
    if (c < C && n1 < g.N[0]) {
      const long long n = t.r * g.N[0] + n1;
      const float2 a = tile[tx][i];
      const float2 b = sn[n];
      // a * conj(b)
      x[(t.s * g.npix + n) * C + c] = make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
    }
  }
}

// grid phase prod_d tab[d][k_d] of grid point p (k1 fastest)
__device__ __forceinline__ float2 grid_phase(const GridPhase &ph, long long p) {
  float2 v = make_float2(1.f, 0.f);
  long long r = p;
  for (int d = 0; d < ph.D; d++) {
    const int k = (int)(r % ph.K[d]);
    r /= ph.K[d];
    const float2 t = ph.tab[d][k];
    v = make_float2(v.x * t.x - v.y * t.y, v.x * t.y + v.y * t.x);
  }
  return v;
}

// [B][P] <-> [P][B] per slice: out[s][p][b] = in[s][b][p] (to_cl) or the reverse;
// PH: times the grid phase of p (to_cl) or its conjugate (the reverse).
template <bool PH>
__global__ void transpose_cols_kernel(const float2 *__restrict__ in, float2 *__restrict__ out,
                                      long long P, int B, int to_cl, GridPhase ph) {
  __shared__ float2 tile[32][33];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const long long p0 = (long long)blockIdx.x * 32;
  const int b0 = blockIdx.y * 32;
  const long long s = blockIdx.z;
  const float2 *src = in + s * P * B;
  float2 *dst = out + s * P * B;
  if (to_cl) {
    // src [B][P] -> dst [P][B]
    for (int i = ty; i < 32; i += 8) {
      const int b = b0 + i;
      const long long p = p0 + tx;
      if (b < B && p < P) tile[i][tx] = src[(long long)b * P + p];
    }
    __syncthreads();
    for (int i = ty; i < 32; i += 8) {
      const long long p = p0 + i;
      const int b = b0 + tx;
      if (b < B && p < P) {
        float2 v = tile[tx][i];
        if (PH) {
          const float2 q = grid_phase(ph, p);
          v = make_float2(v.x * q.x - v.y * q.y, v.x * q.y + v.y * q.x);
        }
        dst[p * B + b] = v;
      }
    }
  } else {
    // src [P][B] -> dst [B][P]
    for (int i = ty; i < 32; i += 8) {
      const long long p = p0 + i;
      const int b = b0 + tx;
      if (b < B && p < P) tile[i][tx] = src[p * B + b];
    }
    __syncthreads();
    for (int i = ty; i < 32; i += 8) {
      const int b = b0 + i;
      const long long p = p0 + tx;
      if (b < B && p < P) {
        float2 v = tile[tx][i];
        if (PH) {
          const float2 q = grid_phase(ph, p);  // v * conj(q)
          v = make_float2(v.x * q.x + v.y * q.y, v.y * q.x - v.x * q.y);
        }
        dst[(long long)b * P + p] = v;
      }
    }
  }
}

__global__ void om_to_tm_kernel(const double *__restrict__ om, long long M, int D,
                                const double *gam, const double *n_shift, int want_phase,
                                double *__restrict__ tm, float2 *__restrict__ phase) {
  const long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (m >= M) return;
  double arg = 0.0;
  for (int d = 0; d < D; d++) {
    const double o = om[d * M + m];
    tm[d * M + m] = o / gam[d];
    arg += o * n_shift[d];
  }
  if (want_phase) {
    double s, c;
    sincos(arg, &s, &c);
    phase[m] = make_float2((float)c, (float)s);
  }
}

// split FP64 [npts, N] (column n contiguous) -> float2 [npts][N]
__global__ void split_to_il_kernel(const double *__restrict__ re, const double *__restrict__ im,
                                   long long npts, int N, float2 *__restrict__ out) {
  __shared__ float2 tile[32][33];
  const long long p0 = (long long)blockIdx.x * 32;
  const int n0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int r = ty; r < 32; r += 8) {
    const long long p = p0 + tx;
    const int n = n0 + r;
    if (p < npts && n < N) {
      const long long idx = (long long)n * npts + p;
      tile[r][tx] = make_float2((float)re[idx], im ? (float)im[idx] : 0.f);
    }
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const long long p = p0 + r;
    const int n = n0 + tx;
    if (p < npts && n < N) out[p * N + n] = tile[tx][r];
  }
}

// float2 [npts][N] -> split FP64 [npts, N]
__global__ void il_to_split_kernel(const float2 *__restrict__ in, long long npts, int N,
                                   double *__restrict__ re, double *__restrict__ im) {
  __shared__ float2 tile[32][33];
  const long long p0 = (long long)blockIdx.x * 32;
  const int n0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int r = ty; r < 32; r += 8) {
    const long long p = p0 + r;
    const int n = n0 + tx;
    if (p < npts && n < N) tile[r][tx] = in[p * N + n];
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const long long p = p0 + tx;
    const int n = n0 + r;
    if (p < npts && n < N) {
      const long long idx = (long long)n * npts + p;
      const float2 v = tile[tx][r];
      re[idx] = (double)v.x;
      im[idx] = (double)v.y;
    }
  }
}

__global__ void tab_to_f32_kernel(const double *__restrict__ re, const double *__restrict__ im,
                                  int n, void *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (im)
    static_cast<float2 *>(out)[i] = make_float2((float)re[i], (float)im[i]);
  else
    static_cast<float *>(out)[i] = (float)re[i];
}

__global__ void fill_slice_kernel(const long long *moff, int nslice, int *slice_id) {
  const int s = blockIdx.y;
  if (s >= nslice) return;
  const long long beg = moff[s], end = moff[s + 1];
  for (long long m = beg + blockIdx.x * (long long)blockDim.x + threadIdx.x; m < end;
       m += (long long)gridDim.x * blockDim.x)
    slice_id[m] = s;
}

// gather the per-sample arrays into bin-sorted order: out[pos] = in[perm[pos]]
__global__ void permute_samples_kernel(const double *__restrict__ tm_in,
                                       const int *__restrict__ slice_in,
                                       const float2 *__restrict__ ph_in,
                                       const int *__restrict__ perm, long long M, int D,
                                       double *__restrict__ tm_out, int *__restrict__ slice_out,
                                       float2 *__restrict__ ph_out) {
  const long long pos = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (pos >= M) return;
  const int m = perm[pos];
  for (int d = 0; d < D; d++) tm_out[d * M + pos] = tm_in[d * M + m];
  if (slice_in) slice_out[pos] = slice_in[m];
  if (ph_in) ph_out[pos] = ph_in[m];
}

namespace {
dim3 image_grid(const GlueGeom &g, int C, int nslice) {
  return dim3((unsigned)(g.npix / g.N[0] * nslice), (unsigned)((g.N[0] + 31) / 32),
              (unsigned)((C + 31) / 32));
}
}  // namespace

cudaError_t launch_deapod_image_cm(const float2 *x, const float2 *sn, float2 *pad,
                                   const GlueGeom &g, int C, int nslice, cudaStream_t st) {
  if (nslice == 0 || C == 0) return cudaSuccess;
  deapod_image_cm_kernel<<<image_grid(g, C, nslice), dim3(32, 8), 0, st>>>(x, sn, pad, g, C);
  return cudaGetLastError();
}

cudaError_t launch_crop_deapod_cm(const float2 *grid, const float2 *sn, float2 *x,
                                  const GlueGeom &g, int C, int nslice, cudaStream_t st) {
  if (nslice == 0 || C == 0) return cudaSuccess;
  crop_deapod_cm_kernel<<<image_grid(g, C, nslice), dim3(32, 8), 0, st>>>(grid, sn, x, g, C);
  return cudaGetLastError();
}

cudaError_t launch_transpose_cols(const float2 *in, float2 *out, long long P, int B, int nslice,
                                  int to_cl, cudaStream_t st, const GridPhase *ph) {
  if (P == 0 || B == 0 || nslice == 0) return cudaSuccess;
  dim3 grid_dim((unsigned)((P + 31) / 32), (unsigned)((B + 31) / 32), (unsigned)nslice);
  if (ph && ph->tab[0])
    transpose_cols_kernel<true><<<grid_dim, dim3(32, 8), 0, st>>>(in, out, P, B, to_cl, *ph);
  else
    transpose_cols_kernel<false><<<grid_dim, dim3(32, 8), 0, st>>>(in, out, P, B, to_cl,
                                                                   GridPhase{});
  return cudaGetLastError();
}

cudaError_t launch_om_to_tm(const double *om, long long M, int D, const double *gam_dev,
                            const double *nshift_dev, int want_phase, double *tm, float2 *phase,
                            cudaStream_t st) {
  if (M == 0) return cudaSuccess;
  om_to_tm_kernel<<<(unsigned)((M + 255) / 256), 256, 0, st>>>(om, M, D, gam_dev, nshift_dev,
                                                              want_phase, tm, phase);
  return cudaGetLastError();
}

cudaError_t launch_split_to_il(const double *re, const double *im, long long npts, int N,
                               float2 *out, cudaStream_t st) {
  if (npts == 0 || N == 0) return cudaSuccess;
  dim3 grid((unsigned)((npts + 31) / 32), (unsigned)((N + 31) / 32));
  split_to_il_kernel<<<grid, dim3(32, 8), 0, st>>>(re, im, npts, N, out);
  return cudaGetLastError();
}

cudaError_t launch_il_to_split(const float2 *in, long long npts, int N, double *re, double *im,
                               cudaStream_t st) {
  if (npts == 0 || N == 0) return cudaSuccess;
  dim3 grid((unsigned)((npts + 31) / 32), (unsigned)((N + 31) / 32));
  il_to_split_kernel<<<grid, dim3(32, 8), 0, st>>>(in, npts, N, re, im);
  return cudaGetLastError();
}

cudaError_t launch_tab_to_f32(const double *re, const double *im, int n, void *out,
                              cudaStream_t st) {
  tab_to_f32_kernel<<<(n + 255) / 256, 256, 0, st>>>(re, im, n, out);
  return cudaGetLastError();
}

cudaError_t launch_permute_samples(const double *tm_in, const int *slice_in, const float2 *ph_in,
                                   const int *perm, long long M, int D, double *tm_out,
                                   int *slice_out, float2 *ph_out, cudaStream_t st) {
  if (M == 0) return cudaSuccess;
  permute_samples_kernel<<<(unsigned)((M + 255) / 256), 256, 0, st>>>(
      tm_in, slice_in, ph_in, perm, M, D, tm_out, slice_out, ph_out);
  return cudaGetLastError();
}

cudaError_t launch_fill_slice(const long long *moff_dev, int nslice, long long Mtot, int *slice_id,
                              cudaStream_t st) {
  if (Mtot == 0) return cudaSuccess;
  dim3 grid(64, (unsigned)nslice);
  fill_slice_kernel<<<grid, 256, 0, st>>>(moff_dev, nslice, slice_id);
  return cudaGetLastError();
}

}  // namespace mirt
