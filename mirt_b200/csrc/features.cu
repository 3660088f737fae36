// features.cu -- per-sample trajectory features for the learned density
// compensation: normalised radius |omega| / pi, angle atan2(omega_2,
// omega_1) / pi, and log1p of a 16-bin histogram of the distances to the
// other samples of the same trajectory within 2 grid cells (bins of 1/8
// cell, distances in units of the oversampled grid, t = omega / (2 pi / K),
// no periodic wrap).
//
// Samples are bucketed into 2 x 2-cell hash cells by the library's stable
// radix sort (slice-major keys), so the neighbours of a sample lie in the 3 x
// 3 hash cells around its own; the scan reads the sorted coordinate copy
// contiguously.  Squared distances are formed in FP64 with explicitly rounded
// operations and compared with the exact squared bin edges, so the counts are
// reproducible bit for bit by an FP64 restatement.
#include "../../include/mirt_b200.h"

#include <new>
#include <string>

#include "runtime.cuh"

using namespace mirt;

namespace {

#define FCK(call)                                                                     \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return api_fail(e_ == cudaErrorMemoryAllocation ? MIRT_ERR_ALLOC : MIRT_ERR_CUDA, \
                      std::string(#call) + ": " + cudaGetErrorString(e_));            \
  } while (0)

struct FeatGeom {
  double scale[2];  // K / (2 pi): omega -> grid units
  int K[2];
  int nc[2];        // hash cells per dimension (2 grid units each)
  int ncells;       // nc[0] * nc[1]
};

__device__ __forceinline__ int cell_of(double t, int K, int nc) {
  // t in [-K/2, K/2) for omega in [-pi, pi); clamp the rest onto the edge cells
  int c = (int)floor((t + 0.5 * K) * 0.5);
  return c < 0 ? 0 : (c >= nc ? nc - 1 : c);
}

// grid coordinates and sort key (slice-major, then hash cell) of each sample
__global__ void feat_keys_kernel(const double *__restrict__ om, long long M,
                                 const int *__restrict__ slice_of, FeatGeom g,
                                 double2 *__restrict__ t, uint32_t *__restrict__ keys) {
  const long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (m >= M) return;
  const double t0 = __dmul_rn(om[m], g.scale[0]);
  const double t1 = __dmul_rn(om[M + m], g.scale[1]);
  t[m] = make_double2(t0, t1);
  const int s = slice_of ? slice_of[m] : 0;
  const int c = cell_of(t0, g.K[0], g.nc[0]) + g.nc[0] * cell_of(t1, g.K[1], g.nc[1]);
  keys[m] = (uint32_t)((long long)s * g.ncells + c);
}

__global__ void feat_gather_kernel(const double2 *__restrict__ t, const int *__restrict__ perm,
                                   long long M, double2 *__restrict__ ts) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p < M) ts[p] = t[perm[p]];
}

// one thread per sorted position
__global__ void feat_hist_kernel(const double *__restrict__ om, const double2 *__restrict__ ts,
                                 const int *__restrict__ perm, const int *__restrict__ bin_start,
                                 const int *__restrict__ slice_of, long long M, FeatGeom g,
                                 float *__restrict__ feat) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= M) return;
  const int m = perm[p];
  const double2 tp = ts[p];
  const int s = slice_of ? slice_of[m] : 0;
  const int c0 = cell_of(tp.x, g.K[0], g.nc[0]);
  const int c1 = cell_of(tp.y, g.K[1], g.nc[1]);
  int h[16];
#pragma unroll
  for (int b = 0; b < 16; b++) h[b] = 0;
  const long long sbase = (long long)s * g.ncells;
  for (int d1 = -1; d1 <= 1; d1++) {
    const int cc1 = c1 + d1;
    if (cc1 < 0 || cc1 >= g.nc[1]) continue;
    // the three cells of this row are contiguous in the sort order
    const int ca = max(c0 - 1, 0), cb = min(c0 + 1, g.nc[0] - 1);
    const long long q0 = bin_start[sbase + (long long)cc1 * g.nc[0] + ca];
    const long long q1 = bin_start[sbase + (long long)cc1 * g.nc[0] + cb + 1];
    for (long long q = q0; q < q1; q++) {
      if (q == p) continue;
      const double2 tq = ts[q];
      const double dx = __dsub_rn(tq.x, tp.x), dy = __dsub_rn(tq.y, tp.y);
      const double d2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
      if (d2 < 4.0) {
        // bin b: (b/8)^2 <= d2 < ((b+1)/8)^2, edges exact in binary
        int b = 0;
#pragma unroll
        for (int e = 1; e < 16; e++) b += d2 >= (e * 0.125) * (e * 0.125) ? 1 : 0;
#pragma unroll
        for (int e = 0; e < 16; e++) h[e] += (e == b) ? 1 : 0;
      }
    }
  }
  const double w0 = om[m], w1 = om[M + m];
  float *f = feat + (long long)m * MIRT_DCF_NFEAT;
  f[0] = (float)(sqrt(w0 * w0 + w1 * w1) / M_PI);
  f[1] = (float)(atan2(w1, w0) / M_PI);
#pragma unroll
  for (int b = 0; b < 16; b++) f[2 + b] = log1pf((float)h[b]);
}

}  // namespace

extern "C" int mirt_dcf_features(const double *om, int64_t M, const int64_t *slice_moff,
                                 int32_t nslice, const int32_t *K, float *feat, void *stream) try {
  if (!om || !K || !feat) return api_fail(MIRT_ERR_ARG, "NULL argument");
  if (M < 0 || nslice < 1) return api_fail(MIRT_ERR_ARG, "need M >= 0 and nslice >= 1");
  if (M >= (1ll << 31)) return api_fail(MIRT_ERR_ARG, "M too large");
  if (K[0] < 2 || K[1] < 2) return api_fail(MIRT_ERR_ARG, "K must be >= 2");
  FeatGeom g{};
  for (int d = 0; d < 2; d++) {
    g.K[d] = K[d];
    g.scale[d] = K[d] / (2.0 * M_PI);
    g.nc[d] = (K[d] + 1) / 2;
  }
  g.ncells = g.nc[0] * g.nc[1];
  const long long nbins = (long long)g.ncells * nslice;
  if (nbins >= (1ll << 31) - 1) return api_fail(MIRT_ERR_ARG, "too many hash cells (K, nslice)");
  std::vector<long long> moff(nslice + 1);
  if (slice_moff) {
    for (int s = 0; s <= nslice; s++) moff[s] = slice_moff[s];
    if (moff[0] != 0 || moff[nslice] != M)
      return api_fail(MIRT_ERR_ARG, "slice offsets must start at 0 and end at M");
    for (int s = 0; s < nslice; s++)
      if (moff[s + 1] < moff[s]) return api_fail(MIRT_ERR_ARG, "slice offsets must not decrease");
  } else if (nslice != 1) {
    return api_fail(MIRT_ERR_ARG, "slice offsets required for nslice > 1");
  }
  if (M == 0) return MIRT_OK;
  cudaStream_t st = as_stream(stream);
  DMem dmoff, slice, t, ts, keys, perm, bstart, tmp;
  const int *slice_of = nullptr;
  if (nslice > 1) {
    FCK(dmoff.alloc((nslice + 1) * sizeof(long long)));
    FCK(cudaMemcpyAsync(dmoff.p, moff.data(), (nslice + 1) * sizeof(long long),
                        cudaMemcpyHostToDevice, st));
    FCK(slice.alloc(M * sizeof(int)));
    FCK(launch_fill_slice(dmoff.as<long long>(), nslice, M, slice.as<int>(), st));
    slice_of = slice.as<int>();
  }
  FCK(t.alloc(M * sizeof(double2)));
  FCK(ts.alloc(M * sizeof(double2)));
  FCK(keys.alloc(M * sizeof(uint32_t)));
  FCK(perm.alloc(M * sizeof(int)));
  FCK(bstart.alloc((nbins + 1) * sizeof(int)));
  FCK(tmp.alloc(radix_sort_tmp_bytes(M)));
  const unsigned blk = (unsigned)((M + 255) / 256);
  feat_keys_kernel<<<blk, 256, 0, st>>>(om, M, slice_of, g, t.as<double2>(), keys.as<uint32_t>());
  FCK(cudaGetLastError());
  FCK(radix_sort_bins(keys.as<uint32_t>(), M, (int)nbins, tmp.p, perm.as<int>(), bstart.as<int>(),
                      st));
  feat_gather_kernel<<<blk, 256, 0, st>>>(t.as<double2>(), perm.as<int>(), M, ts.as<double2>());
  FCK(cudaGetLastError());
  feat_hist_kernel<<<blk, 256, 0, st>>>(om, ts.as<double2>(), perm.as<int>(), bstart.as<int>(),
                                        slice_of, M, g, feat);
  FCK(cudaGetLastError());
  FCK(cudaStreamSynchronize(st));
  return MIRT_OK;
} catch (const std::bad_alloc &) {
  return mirt::api_fail(MIRT_ERR_ALLOC, "out of host memory");
}
