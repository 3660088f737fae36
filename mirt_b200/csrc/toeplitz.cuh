// toeplitz.cuh -- Toeplitz embedding of the 2D NUFFT Gram operator, shared by
// toeplitz.cu (the C ABI) and sense.cu (CG-SENSE in Gram form and the
// circulant preconditioner).
#pragma once

#include <cufft.h>

#include "runtime.cuh"

// Gram operator G'WG of a batched 2D plan: per slice the FFT of the (2N1 x
// 2N2) circulant kernel in which the Toeplitz matrix is embedded.
struct mirt_toeplitz {
  int S = 0, N1 = 0, N2 = 0, ncol = 0;
  mirt::DMem H;    // complex64 [S][2N2][2N1]: FFT of the circulant kernel
  mirt::DMem Hp;   // float [S][2N2][2N1]: circulant preconditioner spectrum (or empty)
  mirt::DMem Hp1;  // float [S][2N2][2N1]: the unweighted spectrum, kept when Hp is blended
  mirt::DMem pad;  // complex64 [S * ncol][2N2][2N1]: work grid
  cufftHandle fft_n = 0, fft_1 = 0;  // batches S * ncol and S
  bool ok_n = false, ok_1 = false;
  ~mirt_toeplitz() {
    if (ok_n) cufftDestroy(fft_n);
    if (ok_1) cufftDestroy(fft_1);
  }
};

namespace mirt {

int toep_create(mirt_toeplitz **out, const double *om, long long M, const long long *moff,
                int nslice, const int *Nd, const int *Kd, const int *Jd, const int *Ld,
                const double *w, int ncol, cudaStream_t st);

// out[s][p] = sum_c conj(sens[s][p][c]) (T_s (sens_c x_s))[p]   (ncol = C)
int toep_gram_sense(mirt_toeplitz *T, const float2 *x, const float2 *sens, float2 *out,
                    cudaStream_t st);

// Circulant preconditioner spectrum 1 / max(lam_s Re H_s + r_s, floor_s),
// r_s the spectrum of the quadratic first-order penalty with weight beta_s
// (host arrays of S values).
int toep_precon_build(mirt_toeplitz *T, const double *lam, const double *beta, cudaStream_t st);

// Circulant preconditioner spectrum from the learned density compensation:
// Tw = G' diag(w^2) G (its spectrum approximates the inverse sampling density
// where the trajectory samples), floored at 1e-3 of its maximum per slice so
// that it stays positive (a Hermitian positive definite preconditioner keeps
// the unweighted minimiser), blended with T's unweighted spectrum P1 (kept in
// Hp1): Hp = blend Pw / mean(Pw) + (1 - blend) P1 / mean(P1).  T's
// toep_precon_build must have run; blend in [0, 1].
int toep_precon_dcf(mirt_toeplitz *T, const mirt_toeplitz *Tw, double blend, cudaStream_t st);

// out = crop(IFFT(Hp FFT(pad(x)))) per slice, single column
int toep_precon_apply(mirt_toeplitz *T, const float2 *x, float2 *out, cudaStream_t st);

}  // namespace mirt
