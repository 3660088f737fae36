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
  // stage-1 twiddles, [q][p1] (q < R2, p1 < R1 for n = R1 R2, fft_radix):
  // W^{p1 q}, W = exp(-+2 pi i / n) in the pass's direction, times any grid
  // phase folded in (FP64-built; see NufftFft)
  const float2 *tw;
  int tw_unit0;              // 1: the twiddle of p1 = 0 is 1 in every column (skipped)
  // deapodisation: sn_in scales input k of line (r2, r1) by sn[(r2*nr1 + r1)*nin + k];
  // sn_out scales output p by conj(sn[(r2*nr1 + r1)*nout + p])
  const float2 *sn_in, *sn_out;
  // grid phase of this dimension: ph_out[p] on outputs, conj(ph_in[k]) on inputs
  const float2 *ph_out, *ph_in;
};

// Transform lengths the passes handle (powers of two from 64 to 1024), and
// the two radices n = R1 R2 of a length.
bool fft_len_ok(int n);
void fft_radix(int n, int *r1, int *r2);

cudaError_t launch_fft_pass(const FftPass &p, cudaStream_t st);

// Geometry of the NUFFT's FFT: image N, grid K, C columns, per-dimension
// stage-1 twiddle tables of the forward and the adjoint passes (device,
// FP64-built), the deapodisation sn [npix] and the optional grid phase.
// When the grid phase is a sequence of quarter turns, exp(2 pi i k Nmid / K)
// = i^(k m) with m = 4 Nmid / K an integer (K = 2N, Nmid = N/2: m = 1), it is
// folded into the twiddles: the forward pass's output p = p1 + R1 p2 turns by
// i^(p1 m) (R1 is a multiple of 4), the same for every output of a stage-2
// thread, and the adjoint pass's input k = R2 k1 + q by i^(-q m), the same for
// every input of a stage-1 thread; both are exact rotations and pass through
// the linear DFT stages.  phase_folded = 1: no phase multiplies in the passes.
struct NufftFft {
  GlueGeom g;
  int C;
  const float2 *twf[3], *twa[3];
  const float2 *sn;
  const GridPhase *gp;       // null or tab[0] null: no grid phase
  int phase_folded;
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
