// interp4.cu -- 4D table interpolation, the work of
// nufft/table/interp4_table1_for.c and interp4_table1_adj.c, on the 3D plan.
//
// A sample's 4D interpolation is J4 weighted 3D interpolations, one on each
// hyperplane k4 that its 4th-dimension taps reach:
//   f(t) = sum_{j4} h4(t4 - k4_j) G3(ck[:, :, :, k4_j mod K4], t1, t2, t3)
// (interp4_table1_for.c:92-140 nests the same sums with j4 outermost).  The
// 4D plan is therefore a 3D plan over the batch of nslice * K4 hyperplanes:
// sub-slice s * K4 + k4 is hyperplane k4 of slice s, whose grid block is
// exactly that hyperplane of the [K1, K2, K3, K4] grid; its samples are the
// (sample, tap j4) pairs whose tap lands on k4, with the tap's coefficient
// (times the caller's phase) as the 3D plan's per-sample phase.  Then
//   forward  fm[m] = sum_{j4} out3[pos(m, j4)]        (j4 in fixed order)
//   adjoint  in3[e] = fm[src(e)],  ck = adjoint3(in3)  (conj(phase) applied)
// and the 3D plan keeps its sort, spreads, gathers and autotuner.  The 4th
// dimension's taps are selected on the host in FP64 with the reference's
// index rules (interp4_table1_for.c:92-99; order 1: :389-394) and any K4
// (general modulo), so the coefficients carry FP64 table values rounded once.
#include "../../include/mirt_b200.h"

#include <cmath>
#include <complex>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "runtime.cuh"

namespace mirt {

int api_fail(int code, const std::string &msg);

namespace {

#define CK4(call)                                                                    \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess)                                                           \
      return api_fail(e_ == cudaErrorMemoryAllocation ? MIRT_ERR_ALLOC : MIRT_ERR_CUDA, \
                      std::string(#call) + ": " + cudaGetErrorString(e_));          \
  } while (0)

// fm[m][c] = sum over j4 of out3[pos[m J4 + j4]][c], j4 = 0, 1, ... in order
__global__ void x4_sum_kernel(const float2 *__restrict__ out3, const int *__restrict__ pos,
                              int J4, long long M4, int C, float2 *__restrict__ fm) {
  const long long n = M4 * C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long m = i / C;
    const int c = (int)(i - m * C);
    const int *p = pos + m * J4;
    float2 v = out3[(long long)__ldg(p) * C + c];
    for (int j = 1; j < J4; j++) {
      const float2 w = out3[(long long)__ldg(p + j) * C + c];
      v.x += w.x;
      v.y += w.y;
    }
    fm[i] = v;
  }
}

// in3[e][c] = fm[src[e]][c]
__global__ void x4_expand_kernel(const float2 *__restrict__ fm, const int *__restrict__ src,
                                 long long Me, int C, float2 *__restrict__ in3) {
  const long long n = Me * C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long e = i / C;
    const int c = (int)(i - e * C);
    in3[i] = fm[(long long)__ldg(src + e) * C + c];
  }
}

int grid_of(long long n) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long b = (n + 255) / 256;
  return (int)std::max(1ll, std::min(b, (long long)sms * 8));
}

// coefficient of 4th-dimension tap k for coordinate t: the table entry
// nearest (t - k) L4 (order 0) or the linear blend of the two entries around
// it (order 1, real tables), indices relative to the table centre nc
std::complex<double> coef4(double t, int k, const double *hr, const double *hi, int nc, int tl,
                           int L, int order) {
  const double p = (t - (double)k) * (double)L;
  if (order == 0) {
    int n = nc + (int)std::floor(p + 0.5);
    n = std::min(std::max(n, 0), tl - 1);
    return {hr[n], hi ? hi[n] : 0.0};
  }
  const double nf = std::floor(p);
  const double alf = p - nf;
  int n = nc + (int)nf;
  n = std::min(std::max(n, 0), tl - 1);
  const double h1 = n + 1 < tl ? hr[n + 1] : 0.0;
  return {(1 - alf) * hr[n] + alf * h1, 0.0};
}

int plan4_build(mirt_interp_plan **out, const int *K, const int *J, const int *L,
                const double *const *h_re, const double *const *h_im, int order,
                const double *tm, long long M4, const long long *moff, int nslice, int C,
                const double *ph_re, const double *ph_im, cudaStream_t st) {
  const int K4 = K[3], J4 = J[3], L4 = L[3];
  const long long Me = M4 * J4;
  if (Me >= (1ll << 31)) return api_fail(MIRT_ERR_ARG, "4D plan: samples times J4 must be < 2^31");
  const long long nsub = (long long)nslice * K4;
  if (nsub >= (1ll << 31)) return api_fail(MIRT_ERR_ARG, "4D plan: slices times K4 too large");
  const bool cplx = h_im != nullptr && h_im[0] != nullptr;
  const double *hr4 = h_re[3], *hi4 = cplx ? h_im[3] : nullptr;
  const int nc = (int)std::floor(J4 * L4 / 2.);
  const int tl = J4 * L4 + 1;
  const double *t4 = tm + 3 * M4;

  // first tap of each sample (interp4_table1_for.c:92), wrapped into [0, K4)
  std::vector<int> koff(M4), k0(M4);
  std::vector<long long> cnt(nsub + 1, 0);
  for (int s = 0; s < nslice; s++)
    for (long long m = moff[s]; m < moff[s + 1]; m++) {
      koff[m] = 1 + (int)std::floor(t4[m] - J4 / 2.);
      k0[m] = (int)(((long long)koff[m] % K4 + K4) % K4);
      for (int j = 0; j < J4; j++) cnt[(long long)s * K4 + (k0[m] + j) % K4]++;
    }
  std::vector<int64_t> moff3(nsub + 1, 0);
  for (long long i = 0; i < nsub; i++) moff3[i + 1] = moff3[i] + cnt[i];
  std::vector<long long> next(moff3.begin(), moff3.end() - 1);
  std::vector<double> tm3(std::max(Me, 1ll) * 3), p3r(std::max(Me, 1ll)), p3i(std::max(Me, 1ll));
  std::vector<int> src(std::max(Me, 1ll)), pos(std::max(Me, 1ll));
  for (int s = 0; s < nslice; s++)
    for (long long m = moff[s]; m < moff[s + 1]; m++) {
      const std::complex<double> ph(ph_re ? ph_re[m] : 1.0, ph_re && ph_im ? ph_im[m] : 0.0);
      for (int j = 0; j < J4; j++) {
        const long long e = next[(long long)s * K4 + (k0[m] + j) % K4]++;
        for (int d = 0; d < 3; d++) tm3[d * Me + e] = tm[d * M4 + m];
        const std::complex<double> w = coef4(t4[m], koff[m] + j, hr4, hi4, nc, tl, L4, order) * ph;
        p3r[e] = w.real();
        p3i[e] = w.imag();
        src[e] = (int)m;
        pos[m * J4 + j] = (int)e;
      }
    }

  const double *hr3[3] = {h_re[0], h_re[1], h_re[2]};
  const double *hi3[3] = {cplx ? h_im[0] : nullptr, cplx ? h_im[1] : nullptr,
                          cplx ? h_im[2] : nullptr};
  mirt_interp_plan *sub = nullptr;
  int rc = mirt_interp_plan_create(&sub, 3, K, J, L, hr3, cplx ? hi3 : nullptr, order, tm3.data(),
                                   Me, moff3.data(), (int32_t)nsub, C, p3r.data(), p3i.data(), st);
  if (rc) return rc;
  std::unique_ptr<mirt_interp_plan> owned(sub);
  auto *P = new mirt_interp_plan();
  P->sub4 = owned.release();
  P->a.g.D = 4;
  P->a.C = C;
  P->a.Mtot = M4;
  P->J4 = J4;
  P->Me = Me;
  cudaError_t e = P->x4_src.alloc(std::max(Me, 1ll) * sizeof(int));
  if (e == cudaSuccess) e = P->x4_pos.alloc(std::max(Me, 1ll) * sizeof(int));
  if (e == cudaSuccess) e = P->x4_buf.alloc(std::max(Me * C, 1ll) * sizeof(float2));
  if (e == cudaSuccess && Me)
    e = cudaMemcpyAsync(P->x4_src.p, src.data(), Me * sizeof(int), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && Me)
    e = cudaMemcpyAsync(P->x4_pos.p, pos.data(), Me * sizeof(int), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    delete P;
    return api_fail(e == cudaErrorMemoryAllocation ? MIRT_ERR_ALLOC : MIRT_ERR_CUDA,
                    std::string("4D plan: ") + cudaGetErrorString(e));
  }
  *out = P;
  return MIRT_OK;
}

}  // namespace

// The host expansion holds 8 * (3 + 2 + 2) bytes per (sample, tap) pair: a
// failed host allocation returns MIRT_ERR_ALLOC instead of leaving the C ABI
// as an exception.
int plan4_create(mirt_interp_plan **out, const int *K, const int *J, const int *L,
                 const double *const *h_re, const double *const *h_im, int order,
                 const double *tm, long long M4, const long long *moff, int nslice, int C,
                 const double *ph_re, const double *ph_im, cudaStream_t st) {
  try {
    return plan4_build(out, K, J, L, h_re, h_im, order, tm, M4, moff, nslice, C, ph_re, ph_im,
                       st);
  } catch (const std::bad_alloc &) {
    return api_fail(MIRT_ERR_ALLOC, "4D plan: out of host memory for the expanded samples");
  }
}

int plan4_forward(mirt_interp_plan *P, const float2 *ck, float2 *fm, cudaStream_t st) {
  float2 *buf = P->x4_buf.as<float2>();
  int rc = mirt_interp_plan_forward(P->sub4, ck, buf, st);
  if (rc) return rc;
  const long long n = P->a.Mtot * P->a.C;
  if (n) {
    x4_sum_kernel<<<grid_of(n), 256, 0, st>>>(buf, P->x4_pos.as<int>(), P->J4, P->a.Mtot, P->a.C,
                                              fm);
    CK4(cudaGetLastError());
  }
  return MIRT_OK;
}

int plan4_adjoint(mirt_interp_plan *P, const float2 *fm, float2 *ck, cudaStream_t st) {
  float2 *buf = P->x4_buf.as<float2>();
  const long long n = P->Me * P->a.C;
  if (n) {
    x4_expand_kernel<<<grid_of(n), 256, 0, st>>>(fm, P->x4_src.as<int>(), P->Me, P->a.C, buf);
    CK4(cudaGetLastError());
  }
  return mirt_interp_plan_adjoint(P->sub4, buf, ck, st);
}

}  // namespace mirt
