// glue.cuh -- launchers of the elementwise kernels in glue.cu.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace mirt {

// Separable phase on the oversampled grid, prod_d tab[d][k_d] (k1 fastest):
// newfft's phase_before = exp(i 2 pi sum_d k_d Nmid_d / K_d) as one table
// of K_d values per dimension.
struct GridPhase {
  int D;
  int K[3];
  const float2 *tab[3];
};

struct GlueGeom {
  int D;
  int N[3];            // image size per dimension (N1 fastest)
  int K[3];            // oversampled grid size per dimension
  long long npix;      // prod(N)
  long long ngrid;     // prod(K)
};

// image x[s][n][c] .* sn -> the image region of the coil-major zero-padded grid
// pad[s][c][k] (its padding is zero already and stays so)
cudaError_t launch_deapod_image_cm(const float2 *x, const float2 *sn, float2 *pad,
                                   const GlueGeom &g, int C, int nslice, cudaStream_t st);
// coil-major grid[s][c][k] -> cropped, conj(sn)-scaled image x[s][n][c]
cudaError_t launch_crop_deapod_cm(const float2 *grid, const float2 *sn, float2 *x,
                                  const GlueGeom &g, int C, int nslice, cudaStream_t st);
// per slice: to_cl = 1: [B][P] -> [P][B]; to_cl = 0: [P][B] -> [B][P]; with ph,
// times the grid phase (to_cl = 1) or its conjugate (to_cl = 0)
cudaError_t launch_transpose_cols(const float2 *in, float2 *out, long long P, int B, int nslice,
                                  int to_cl, cudaStream_t st, const GridPhase *ph = nullptr);
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
