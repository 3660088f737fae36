// fft.cuh -- the oversampled FFT of the table NUFFT as fused passes over the
// coil-innermost grid (fft.cu).
//
// nufft.m:139-140 forms fftn(x .* sn, Kd) (the image zero-padded at the end of
// every dimension) and nufft_adj.m:63-80 prod(Kd) * ifftn(Xk), cropped to Nd
// and times conj(sn).  Here each is one pass per dimension over the grid the
// interpolation reads and writes (coil index innermost), so that no coil-major
// copy and no transpose is needed:
//   * the forward pass along dimension 1 reads the image, multiplies it by sn
//     and writes the image rows of the grid; the passes along dimensions 2 and
//     3 transform the grid in place, reading only the rows and planes that hold
//     data (the zero padding is never read) and writing every grid point;
//   * the adjoint runs the passes in the other order, in place, writing only
//     the rows and planes the crop keeps; its last pass writes the image times
//     conj(sn).
// newfft's phase_before (a separable grid phase) is applied to the output of
// each forward pass and, conjugated, to the input of each adjoint pass.
#pragma once
#include <cuda_runtime.h>

#include "glue.cuh"

namespace mirt {

// One pass: a batch of 1D DFTs of length n.  A line is (outer index o, vector
// chunk w); o = (s, r2, r1) with r1 < nr1, r2 < nr2 and s < nslice.  Its k-th
// input element is the vector of vw complex values at
//   in + s*is[0] + r2*is[1] + r1*is[2] + w*vw + k*es_in       (k < nin; zero beyond)
// and output p (p < nout) goes to the same form with os[] and es_out.
struct FftPass {
  const float2 *in;
  float2 *out;
  int nslice, nr2, nr1, nvec, vw;
  long long is[3], os[3], es_in, es_out;
  int n, nin, nout;
  int inverse;               // 0: exp(-2 pi i k p / n); 1: exp(+...), unnormalised
  const float2 *tw;          // exp(-2 pi i k / n), k < n (FP64-built)
  // deapodisation: sn_in scales input k of line (r2, r1) by sn[(r2*nr1 + r1)*nin + k];
  // sn_out scales output p by conj(sn[(r2*nr1 + r1)*nout + p])
  const float2 *sn_in, *sn_out;
  // grid phase of this dimension: ph_out[p] on outputs, conj(ph_in[k]) on inputs
  const float2 *ph_out, *ph_in;
};

// Transform lengths the passes handle (powers of two from 64 to 1024).
bool fft_len_ok(int n);

cudaError_t launch_fft_pass(const FftPass &p, cudaStream_t st);

// Geometry of the NUFFT's FFT: image N, grid K, C columns, per-dimension
// twiddle tables (device, FP64-built), the deapodisation sn [npix] and the
// optional grid phase.
struct NufftFft {
  GlueGeom g;
  int C;
  const float2 *tw[3];
  const float2 *sn;
  const GridPhase *gp;       // null or tab[0] null: no grid phase
};

// fftn(x .* sn, K) of slices [s0, s1): x [s][n][c] -> grid [s][k][c]
cudaError_t fft_nufft_forward(const NufftFft &f, const float2 *x, float2 *grid, int s0, int s1,
                              cudaStream_t st);
// prod(K) ifftn(grid), cropped, .* conj(sn), slices [s0, s1): grid is overwritten
cudaError_t fft_nufft_adjoint(const NufftFft &f, float2 *grid, float2 *x, int s0, int s1,
                              cudaStream_t st);
// launches of one forward or adjoint (for launch counts)
int fft_nufft_passes(const NufftFft &f);

}  // namespace mirt
