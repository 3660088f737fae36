// glue.cuh -- launchers of the elementwise kernels in glue.cu.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace mirt {

struct GlueGeom {
  int D;
  int N[3];            // image size per dimension (N1 fastest)
  int K[3];            // oversampled grid size per dimension
  long long npix;      // prod(N)
  long long ngrid;     // prod(K)
};

cudaError_t launch_deapod_pad(const float2 *x, const float2 *sn, float2 *grid, const GlueGeom &g,
                              int C, int nslice, cudaStream_t st);
cudaError_t launch_crop_deapod(const float2 *grid, const float2 *sn, float2 *x, const GlueGeom &g,
                               int C, int nslice, cudaStream_t st);
cudaError_t launch_om_to_tm(const double *om, long long M, int D, const double *gam_dev,
                            const double *nshift_dev, int want_phase, double *tm, float2 *phase,
                            cudaStream_t st);
cudaError_t launch_split_to_il(const double *re, const double *im, long long npts, int N,
                               float2 *out, cudaStream_t st);
cudaError_t launch_il_to_split(const float2 *in, long long npts, int N, double *re, double *im,
                               cudaStream_t st);
cudaError_t launch_tab_to_f32(const double *re, const double *im, int n, void *out,
                              cudaStream_t st);
cudaError_t launch_permute_samples(const double *tm_in, const int *slice_in, const float2 *ph_in,
                                   const int *perm, long long M, int D, double *tm_out,
                                   int *slice_out, float2 *ph_out, cudaStream_t st);
cudaError_t launch_fill_slice(const long long *moff_dev, int nslice, long long Mtot, int *slice_id,
                              cudaStream_t st);

}  // namespace mirt
