// capi.cu -- the C ABI of include/mirt_b200.h.
//
// The mex drop-ins reproduce the gateways' argument checks and messages
// (nufft/table/interp{1,2,3}_table{,_adj}_mex.c) and their column semantics,
// then run the whole call on the GPU: FP64 split-complex host arrays are
// copied in, converted to the device's interleaved FP32 layout, bin-sorted,
// interpolated, converted back and copied out before the call returns.
#include "../../include/mirt_b200.h"

#include <cufft.h>

#include <cstdio>
#include <cstdlib>

#include <cmath>
#include <complex>
#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <set>
#include <string>
#include <vector>

#include "glue.cuh"
#include "interp.cuh"
#include "runtime.cuh"

namespace mirt {
bool minmax_kb_table(int N, int J, int K, int L, std::vector<std::complex<double>> &h);
void alpha_kb_fit(int N, int J, int K, std::vector<double> &alphas, double &beta);
std::vector<std::complex<double>> scale1(int N, int K, const std::vector<double> &alpha,
                                         double beta);
void kb_table(int J, int L, std::vector<double> &h);
std::vector<double> kb_scale(int N, int J, int K, double nmid);
void kb_table_alpha(int J, int L, double alpha_full, std::vector<double> &h);
std::vector<double> kb_scale_alpha(int N, int J, int K, double nmid, double alpha);
double kb_beatty_alpha(int N, int J, int K);
void diric_table(int J, int K, int L, std::vector<double> &h);
bool minmax_kb_table_real(int N, int J, int K, int L, std::vector<double> &h);
std::vector<double> minmax_kb_scale_real(int N, int J, int K, double Nmid);
bool minmax_table_real_ab(int N, int J, int K, int L, const std::vector<double> &alpha, double beta,
                          std::vector<double> &h);
std::vector<double> minmax_scale_real_ab(int N, int K, const std::vector<double> &alpha,
                                         double beta, double Nmid);
bool best_alpha(int J, int N, int K, std::vector<double> &alpha, double &beta);
void linear_table(int J, int L, std::vector<double> &h);
std::vector<double> linear_scale(int N, int J, int K, double Nmid);
void kb_user_table(int J, int L, double alpha_full, int m, std::vector<double> &h);
void kb_table_complex(int N, int J, int K, int L, double alpha_full, int m,
                      std::vector<std::complex<double>> &h);
bool minmax_table_complex_ab(int N, int J, int K, int L, const std::vector<double> &alpha,
                             double beta, std::vector<std::complex<double>> &h);
void diric_table_complex(int N, int J, int K, int L, std::vector<std::complex<double>> &h);
void linear_table_complex(int N, int J, int K, int L, std::vector<std::complex<double>> &h);
bool nufft_table_ktype(int kt, int N, int J, int K, int L, double kb_alf, int kb_m,
                       const std::vector<double> &alpha, double beta,
                       std::vector<std::complex<double>> &h);
bool nufft_scale_ktype(int kt, int N, int J, int K, double kb_alf, int kb_m,
                       const std::vector<double> &alpha, double beta,
                       std::vector<std::complex<double>> &sn);
std::vector<double> kb_user_scale(int N, int J, int K, double nmid, double alpha, int m);
int plan4_create(mirt_interp_plan **out, const int *K, const int *J, const int *L,
                 const double *const *h_re, const double *const *h_im, int order,
                 const double *tm, long long M4, const long long *moff, int nslice, int C,
                 const double *ph_re, const double *ph_im, cudaStream_t st);
int plan4_forward(mirt_interp_plan *P, const float2 *ck, float2 *fm, cudaStream_t st);
int plan4_adjoint(mirt_interp_plan *P, const float2 *fm, float2 *ck, cudaStream_t st);
}  // namespace mirt

using namespace mirt;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

#define CK(call)                                                                      \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return fail(e_ == cudaErrorMemoryAllocation ? MIRT_ERR_ALLOC : MIRT_ERR_CUDA,   \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                \
  } while (0)

int device_ok() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(MIRT_ERR_CUDA, "no CUDA device available");
  }
  return MIRT_OK;
}

}  // namespace

namespace mirt {
// Record an error for mirt_last_error() from another translation unit.
int api_fail(int code, const std::string &msg) { return fail(code, msg); }

// ---------------------------------------------------------------------------
// caching device allocator: blocks are rounded up to a power of two and kept
// for reuse, so repeated mex calls do not pay cudaMalloc / cudaFree.
// ---------------------------------------------------------------------------
namespace {
std::mutex g_cache_mu;
std::multimap<std::pair<int, size_t>, void *> g_free;
}  // namespace

size_t round_block(size_t b) {
  size_t r = 256;
  while (r < b) r <<= 1;
  return r;
}

cudaError_t dalloc(void **p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) return cudaSuccess;
  int dev = 0;
  cudaGetDevice(&dev);
  const size_t r = round_block(bytes);
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    auto it = g_free.find({dev, r});
    if (it != g_free.end()) {
      *p = it->second;
      g_free.erase(it);
      return cudaSuccess;
    }
  }
  cudaError_t e = cudaMalloc(p, r);
  if (e != cudaSuccess) {
    cudaGetLastError();
    // release the cache and retry once
    std::lock_guard<std::mutex> lk(g_cache_mu);
    for (auto &kv : g_free) cudaFree(kv.second);
    g_free.clear();
    e = cudaMalloc(p, r);
  }
  return e;
}

void dfree(void *p, size_t bytes) {
  if (!p) return;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_cache_mu);
  g_free.insert({{dev, round_block(bytes)}, p});
}

}  // namespace mirt


namespace mirt_plan_kernels {
// records of position gorder[i] to slot i (the gather's order)
__global__ void gather_records_kernel(const int *__restrict__ gorder, long long M, int SJ,
                                      const float2 *__restrict__ W, const int4 *__restrict__ K0,
                                      const int *__restrict__ perm, const float2 *__restrict__ ph,
                                      float2 *__restrict__ Wg, int4 *__restrict__ K0g,
                                      int *__restrict__ permg, float2 *__restrict__ phg) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= M) return;
  const long long p = gorder[i];
  K0g[i] = K0[p];
  permg[i] = perm ? perm[p] : (int)p;
  if (ph) phg[i] = ph[p];
  for (int j = 0; j < SJ; j++) Wg[i * SJ + j] = W[p * SJ + j];
}

// Tap records of the staged 2D row sweep (J = 6): per position, the six
// first-dimension taps as FFMA2 operand pairs (wr, wr, wi, -wi), then the six
// second-dimension taps two per float4.
__global__ void sweep_records_kernel(const float2 *__restrict__ W, long long M,
                                     float4 *__restrict__ out) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= M) return;
  const float2 *w = W + p * 12;
  float4 *o = out + p * 9;
  for (int j = 0; j < 6; j++) o[j] = make_float4(w[j].x, w[j].x, w[j].y, -w[j].y);
  for (int k = 0; k < 3; k++) o[6 + k] = make_float4(w[6 + 2 * k].x, w[6 + 2 * k].y,
                                                      w[7 + 2 * k].x, w[7 + 2 * k].y);
}

// Output records of the TMA gather, in the gather order: (caller's sample
// index, 0, phase re, phase im as bits); phase (1, 0) where there is none.
__global__ void out_records_kernel(long long M, const int *__restrict__ permg,
                                   const float2 *__restrict__ phg, int4 *__restrict__ out) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= M) return;
  const float2 ph = phg ? phg[i] : make_float2(1.f, 0.f);
  out[i] = make_int4(permg[i], 0, __float_as_int(ph.x), __float_as_int(ph.y));
}
}  // namespace mirt_plan_kernels

namespace {

// Launch shapes and tiling.  Samples are binned on one-point bins of their
// first tap; the spread runs one warp per tile by default (lanes = coils; the
// tile accumulator is sized to keep several CTAs resident per SM).
// The spread's range path serves wrapping taps when no tile can meet a
// sample's taps both before and after their periodic wrap.
// The ownership spread needs: 2D, J = 6, one-point bins, tiles of at least
// J - 1 points, an even number (>= 2) of tiles per dimension and a last tile
// of at least J - 1 points, so that a padded tile reaches only the next tile
// and tiles of one colour (index parities) never overlap, wrap included.
int own_ok(const InterpArgs &a, const Tiling &t) {
  if (a.g.D != 2) return 0;
  for (int d = 0; d < 2; d++) {
    const int K = a.g.K[d], T = t.T[d];
    if (a.g.J[d] != 6 || t.B[d] != 1 || T < 5 || K < T + 5) return 0;
    const int nb = (K + T - 1) / T;
    if (nb < 2 || nb % 2 || K - (nb - 1) * T < 5) return 0;
  }
  return 1;
}

// The row-sweep spread needs: 2D, J = 6, one-point bins, K >= J per dimension
// (each bin row and column reaches a grid row or column through one tap).
int sweep_ok(const InterpArgs &a, const Tiling &t) {
  if (a.g.D != 2) return 0;
  for (int d = 0; d < 2; d++)
    if (a.g.J[d] != 6 || t.B[d] != 1 || a.g.K[d] < 6) return 0;
  return 1;
}

// The 3D line sweep needs: 3D, J = 6, one-point bins, K >= 6 per dimension,
// and coil chunks of 8, 16 or 32 lanes (blocks of 2 x 2, 2 x 1 or 1 lines).
int sweep3_ok(const InterpArgs &a, const Tiling &t, int cw) {
  if (a.g.D != 3 || (cw != 8 && cw != 16 && cw != 32)) return 0;
  for (int d = 0; d < 3; d++)
    if (a.g.J[d] != 6 || t.B[d] != 1 || a.g.K[d] < 6) return 0;
  return 1;
}

// The row sweep's copy of the samples in plan order (allocated when the sweep
// is first selected, outside any launch).
int sweep_buffer(mirt_interp_plan *P) {
  const size_t bytes = (size_t)std::max<long long>(P->a.Mtot, 1) * std::max(P->a.C, 1) *
                       sizeof(float2);
  if (P->swept.bytes < bytes) CK(P->swept.alloc(bytes));
  P->t.sorted = P->swept.as<float2>();
  return MIRT_OK;
}

// Balanced row-sweep teams: each band of `rows` grid rows of each slice is
// cut into column segments of about equal cost, cost = visits (samples of the
// rows + 5 bin rows in the segment's columns and its five warm-up columns)
// + 2 per column step; segments of at least 8 columns, about `target` teams
// in all, in grid order (neighbouring bands read the same samples, so they
// run together; heaviest-first order measured slower at full size).  Teams
// write disjoint points, each summed in the same fixed order.
// bins with at least this many samples are summed into patches before a sweep
constexpr int kDenseBin = 16;

// Visits per bin column of every band of `rows` grid rows: vb[(s * nband +
// band) * K1 + x] = samples in bin column x of the band's rows + 5 bin rows.
int sweep_band_visits(mirt_interp_plan *P, int rows, cudaStream_t st, std::vector<float> &vb) {
  const InterpArgs &a = P->a;
  const Tiling &t = P->t;
  const int K1 = a.g.K[0], K2 = a.g.K[1], S = t.nslice, NQ = rows + 5;
  const long long nb = (long long)t.nbins * S;
  std::vector<int> bs(nb + 1);
  CK(cudaMemcpyAsync(bs.data(), P->bin_start.p, (nb + 1) * sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  const int nband = (K2 + rows - 1) / rows;
  vb.assign((size_t)S * nband * K1, 0.f);
  for (int s = 0; s < S; s++) {
    const int *b = bs.data() + (size_t)s * t.nbins;
    for (int bi = 0; bi < nband; bi++) {
      float *v = vb.data() + ((size_t)s * nband + bi) * K1;
      for (int q = 0; q < NQ; q++) {
        int r = (bi * rows - 5 + q) % K2;
        if (r < 0) r += K2;
        const int *br = b + (size_t)r * K1;
        for (int x = 0; x < K1; x++) {
          const int n = br[x + 1] - br[x];
          // a dense bin costs its patch rows, not its samples
          v[x] += (float)(P->t.dense_of && n >= kDenseBin ? 6 : n);
        }
      }
    }
  }
  return MIRT_OK;
}

// cost of a team: its visits (five warm-up columns included) + 2 per column step
constexpr double kSweepColumnCost = 2.0;

double sweep_team_cost(const float *v, int K1, int x0, int x1) {
  double c = 0;
  for (int x = x0 - 5; x < x1; x++) c += v[(x % K1 + K1) % K1] + kSweepColumnCost;
  return c;
}

// The sweep's work queue: teams heaviest first (ties in index order), and the
// queue counter.  Teams are the list (t.sweep < 0) or the uniform segments.
int build_sweep_order(mirt_interp_plan *P, const std::vector<float> &vb, cudaStream_t st) {
  const InterpArgs &a = P->a;
  Tiling &t = P->t;
  const int K1 = a.g.K[0], K2 = a.g.K[1], rows = t.sweep_rows;
  const int nband = (K2 + rows - 1) / rows;
  std::vector<int4> tk;
  if (t.sweep < 0) {
    tk = P->team_host;
  } else {
    const int nseg = t.sweep, sw = (K1 + nseg - 1) / nseg;
    for (int s = 0; s < t.nslice; s++)
      for (int bi = 0; bi < nband; bi++)
        for (int g = 0; g < nseg; g++)
          tk.push_back(make_int4(s, bi * rows, g * sw, std::min(K1, g * sw + sw)));
  }
  std::vector<double> cost(tk.size());
  for (size_t i = 0; i < tk.size(); i++) {
    const int4 k = tk[i];
    cost[i] = k.z < k.w ? sweep_team_cost(vb.data() + ((size_t)k.x * nband + k.y / rows) * K1, K1,
                                          k.z, k.w)
                        : 0.0;
  }
  std::vector<int> order(tk.size());
  for (size_t i = 0; i < order.size(); i++) order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost[x] > cost[y]; });
  if (P->team_order.bytes < std::max<size_t>(order.size(), 1) * sizeof(int))
    CK(P->team_order.alloc(std::max<size_t>(order.size(), 1) * sizeof(int)));
  if (!order.empty())
    CK(cudaMemcpyAsync(P->team_order.p, order.data(), order.size() * sizeof(int),
                       cudaMemcpyHostToDevice, st));
  // one queue counter per coil chunk
  const size_t nq = (size_t)std::max(1, (a.C + P->ls.cw - 1) / std::max(P->ls.cw, 1));
  if (P->team_next.bytes < nq * sizeof(int)) CK(P->team_next.alloc(nq * sizeof(int)));
  CK(cudaStreamSynchronize(st));
  t.team_order = P->team_order.as<int>();
  t.team_next = P->team_next.as<int>();
  return MIRT_OK;
}

// Balanced row-sweep teams: each band of `rows` grid rows of each slice is
// cut into column segments of about equal cost (sweep_team_cost), segments of
// at least 8 columns, about `target` teams in all.  Teams write disjoint
// points, each summed in the same fixed order.
int build_sweep_teams(mirt_interp_plan *P, int rows, long long target, cudaStream_t st) {
  const InterpArgs &a = P->a;
  Tiling &t = P->t;
  const int K1 = a.g.K[0], K2 = a.g.K[1], S = t.nslice;
  std::vector<float> vb;
  int rc = sweep_band_visits(P, rows, st, vb);
  if (rc) return rc;
  const double alpha = kSweepColumnCost;
  const int nband = (K2 + rows - 1) / rows;
  double total = 0;
  for (float v : vb) total += v + alpha;
  const double T = std::max(1.0, total / (double)std::max<long long>(target, 1));
  std::vector<int4> tk;  // (slice, first row, x0, x1), in grid order
  for (int s = 0; s < S; s++)
    for (int bi = 0; bi < nband; bi++) {
      const float *v = vb.data() + ((size_t)s * nband + bi) * K1;
      auto vx = [&](int x) { return (double)v[(x % K1 + K1) % K1]; };
      int x0 = 0;
      while (x0 < K1) {
        double c = 5 * alpha;
        for (int x = x0 - 5; x < x0; x++) c += vx(x);
        int x1 = x0;
        while (x1 < K1) {
          const double add = vx(x1) + alpha;
          if (x1 - x0 >= 8 && c + add > T) break;
          c += add;
          x1++;
        }
        if (K1 - x1 < 8) x1 = K1;  // a short tail joins this segment
        tk.push_back(make_int4(s, bi * rows, x0, x1));
        x0 = x1;
      }
    }
  if (P->sweep_teams.bytes < tk.size() * sizeof(int4)) CK(P->sweep_teams.alloc(tk.size() * sizeof(int4)));
  CK(cudaMemcpyAsync(P->sweep_teams.p, tk.data(), tk.size() * sizeof(int4), cudaMemcpyHostToDevice,
                     st));
  CK(cudaStreamSynchronize(st));
  P->team_host = tk;
  t.sweep_team = P->sweep_teams.as<int4>();
  t.nteams = (int)tk.size();
  t.sweep = -1;
  t.sweep_rows = rows;
  return build_sweep_order(P, vb, st);
}

// The sweeps' dense bins: bins with at least `minc` samples (0: none), their
// index map and patch buffer (J^D taps x C per dense bin).
int build_dense(mirt_interp_plan *P, int minc, cudaStream_t st) {
  const InterpArgs &a = P->a;
  Tiling &t = P->t;
  t.dense_of = nullptr;
  t.dense_bin = nullptr;
  t.patch = nullptr;
  t.dense0 = 0;
  t.ndense = 0;
  t.dense_min = minc;
  t.dense_chunk = nullptr;
  t.dense_part0 = nullptr;
  t.patch_part = nullptr;
  t.chunk0 = 0;
  t.nchunks = 0;
  P->dense_slice.assign(t.nslice + 1, 0);
  // (a chunk's sample rows are staged in shared memory: at most 256 columns)
  if (minc <= 0 || a.C == 0 || a.C > 256) return MIRT_OK;
  const long long nb = (long long)t.nbins * t.nslice;
  std::vector<int> bs(nb + 1);
  CK(cudaMemcpyAsync(bs.data(), P->bin_start.p, (nb + 1) * sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  std::vector<int> db;
  for (long long b = 0; b < nb; b++) {
    if (b % t.nbins == 0) P->dense_slice[b / t.nbins] = (int)db.size();
    if (bs[b + 1] - bs[b] >= minc) db.push_back((int)b);
  }
  P->dense_slice[t.nslice] = (int)db.size();
  if (db.empty()) return MIRT_OK;
  int taps = 1;
  for (int d = 0; d < a.g.D; d++) taps *= 6;
  // chunks of at most 64 samples per dense bin, summed apart, then per bin
  constexpr int kChunk = 64;
  std::vector<int4> chunks;
  std::vector<int> part0(db.size() + 1, 0);
  for (size_t d = 0; d < db.size(); d++) {
    part0[d] = (int)chunks.size();
    for (int p = bs[db[d]]; p < bs[db[d] + 1]; p += kChunk)
      chunks.push_back(make_int4((int)d, p, std::min(p + kChunk, bs[db[d] + 1]),
                                 (int)chunks.size()));
  }
  part0[db.size()] = (int)chunks.size();
  CK(P->dense_of.alloc(nb * sizeof(int)));
  CK(P->dense_bin.alloc(db.size() * sizeof(int)));
  CK(P->patch.alloc(db.size() * (size_t)taps * a.C * sizeof(float2)));
  CK(P->dense_chunk.alloc(chunks.size() * sizeof(int4)));
  CK(P->dense_part0.alloc(part0.size() * sizeof(int)));
  CK(P->patch_part.alloc(chunks.size() * (size_t)taps * a.C * sizeof(float2)));
  CK(cudaMemcpyAsync(P->dense_chunk.p, chunks.data(), chunks.size() * sizeof(int4),
                     cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(P->dense_part0.p, part0.data(), part0.size() * sizeof(int),
                     cudaMemcpyHostToDevice, st));
  P->dense_part0_host = part0;
  CK(cudaMemsetAsync(P->dense_of.p, 0xff, nb * sizeof(int), st));
  CK(cudaMemcpyAsync(P->dense_bin.p, db.data(), db.size() * sizeof(int), cudaMemcpyHostToDevice,
                     st));
  CK(launch_mark_dense(P->dense_bin.as<int>(), (int)db.size(), P->dense_of.as<int>(), st));
  CK(cudaStreamSynchronize(st));
  t.dense_of = P->dense_of.as<int>();
  t.dense_bin = P->dense_bin.as<int>();
  t.patch = P->patch.as<float2>();
  t.ndense = (int)db.size();
  t.dense_chunk = P->dense_chunk.as<int4>();
  t.dense_part0 = P->dense_part0.as<int>();
  t.patch_part = P->patch_part.as<float2>();
  t.chunk0 = 0;
  t.nchunks = (int)chunks.size();
  return MIRT_OK;
}

// 3D line sweep with nseg uniform segments per line block: the work queue of
// its teams, heaviest first (cost: the samples of the block's bin lines in
// the segment and its warm-up columns + 2 per column step).
int set_line_sweep3(mirt_interp_plan *P, int nseg, cudaStream_t st) {
  const InterpArgs &a = P->a;
  Tiling &t = P->t;
  const int K1 = a.g.K[0], K2 = a.g.K[1], K3 = a.g.K[2], S = t.nslice;
  const int nl = 32 / P->ls.cw, B2 = nl >= 2 ? 2 : 1, B3 = nl / B2;
  const int nby = (K2 + B2 - 1) / B2, nbz = (K3 + B3 - 1) / B3;
  const long long nb = (long long)t.nbins * S;
  std::vector<int> bs(nb + 1);
  CK(cudaMemcpyAsync(bs.data(), P->bin_start.p, (nb + 1) * sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  const int sw = (K1 + nseg - 1) / nseg;
  const long long nteam = (long long)S * nbz * nby * nseg;
  std::vector<double> cost(nteam, 0.0);
  for (long long team = 0; team < nteam; team++) {
    const int seg = (int)(team % nseg);
    long long rest = team / nseg;
    const int by = (int)(rest % nby);
    rest /= nby;
    const int bz = (int)(rest % nbz);
    const int s = (int)(rest / nbz);
    const int x0 = seg * sw, x1 = std::min(K1, x0 + sw);
    if (x0 >= x1) continue;
    double c = kSweepColumnCost * (x1 - x0 + 5);
    for (int q3 = 0; q3 < B3 + 5; q3++)
      for (int q2 = 0; q2 < B2 + 5; q2++) {
        const int r = ((by * B2 - 5 + q2) % K2 + K2) % K2;
        const int z = ((bz * B3 - 5 + q3) % K3 + K3) % K3;
        const int *br = bs.data() + (size_t)s * t.nbins + ((size_t)z * K2 + r) * K1;
        const int xs = x0 - 5;
        if (xs < 0) c += br[K1] - br[xs + K1];
        c += br[x1] - br[std::max(xs, 0)];
      }
    cost[team] = c;
  }
  std::vector<int> order(nteam);
  for (long long i = 0; i < nteam; i++) order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost[x] > cost[y]; });
  if (P->team_order.bytes < std::max<size_t>(order.size(), 1) * sizeof(int))
    CK(P->team_order.alloc(std::max<size_t>(order.size(), 1) * sizeof(int)));
  if (!order.empty())
    CK(cudaMemcpyAsync(P->team_order.p, order.data(), order.size() * sizeof(int),
                       cudaMemcpyHostToDevice, st));
  const size_t nq = (size_t)std::max(1, (a.C + P->ls.cw - 1) / std::max(P->ls.cw, 1));
  if (P->team_next.bytes < nq * sizeof(int)) CK(P->team_next.alloc(nq * sizeof(int)));
  CK(cudaStreamSynchronize(st));
  t.team_order = P->team_order.as<int>();
  t.team_next = P->team_next.as<int>();
  t.sweep = nseg;
  t.sweep_rows = 1;
  return MIRT_OK;
}

// Uniform segments: the work queue of their teams.
int set_uniform_sweep(mirt_interp_plan *P, int nseg, int rows, cudaStream_t st) {
  P->t.sweep = nseg;
  P->t.sweep_rows = rows;
  std::vector<float> vb;
  int rc = sweep_band_visits(P, rows, st, vb);
  if (rc) return rc;
  return build_sweep_order(P, vb, st);
}

// The plan's gather over slices [s0, s1) (all: s1 < 0): the TMA-staged tiles
// when the plan has them, else the plain gather over the slices' positions.
cudaError_t plan_gather(mirt_interp_plan *P, const float2 *ck, float2 *fm, cudaStream_t st,
                        int s0 = 0, int s1 = -1) {
  const int S = P->t.nslice;
  if (s1 < 0) s1 = S;
  if (P->gtma) {
    const long long i0 = P->gitem_slice[s0], i1 = P->gitem_slice[s1];
    return launch_gather_tma(P->ag, P->gbk, S, i0, i1 - i0, ck, fm, P->gfault.as<int>(), st,
                             P->gfault_test, P->gtma == 2 ? 16 : 32);
  }
  InterpArgs ag = P->ag;
  if (s0 > 0 || s1 < S) {
    const long long q0 = P->moff_host[s0], nq = P->moff_host[s1] - q0;
    ag.Mtot = nq;
    ag.W += q0 * ag.SJ;
    ag.K0 += q0;
    if (ag.perm) ag.perm += q0;
    if (ag.phase) ag.phase += q0;
  }
  return launch_gather(ag, P->lg, ck, fm, st);
}

int wrap_ok(const InterpArgs &a, const Tiling &t) {
  for (int d = 0; d < a.g.D; d++)
    if (a.g.K[d] < t.T[d] + a.g.J[d]) return 0;
  return 1;
}

void choose_config(mirt_interp_plan *P) {
  InterpArgs &a = P->a;
  Tiling &t = P->t;
  const int C = a.C, D = a.g.D;
  const int cw = C >= 32 ? 32 : C >= 8 ? 8 : C >= 4 ? 4 : 1;
  const int threads = 256;
  Launch &lg = P->lg;
  lg.threads = threads;
  lg.cw = cw;
  lg.sb = 0;
  lg.grid = 0;

  // one-point sort bins: a tile's source samples in one row of bins are one
  // contiguous range, and every visit has taps in the tile
  int B[MIRT_DMAX] = {1, 1, 1}, T[MIRT_DMAX] = {1, 1, 1};
  if (D == 1) {
    T[0] = cw == 32 ? 64 : 256;
  } else if (D == 2) {
    const int e = cw == 32 ? 8 : cw == 8 ? 16 : 32;
    T[0] = T[1] = e;
  } else {
    T[0] = T[1] = T[2] = 8;
    if (cw <= 4) T[0] = 16;
  }
  for (int d = 0; d < D; d++) {
    if (B[d] > a.g.K[d]) B[d] = a.g.K[d];
    const int kr = (a.g.K[d] + B[d] - 1) / B[d] * B[d];
    if (T[d] > kr) T[d] = kr;
    T[d] = (T[d] + B[d] - 1) / B[d] * B[d];
  }
  lg.atomic = 0;
  Launch &ls = P->ls;
  ls.threads = 32;
  ls.cw = cw;
  ls.sb = 0;
  ls.grid = 0;
  ls.atomic = 0;
  // no spare tile columns by default; the autotuner also tries J1 - 1
  t.padc = 0;
  t.own = 0;
  t.sweep = 0;
  t.sweep_rows = 1;
  t.sorted = nullptr;
  t.slice0 = 0;
  t.pos0 = 0;
  t.npos = -1;
  t.sweep_team = nullptr;
  t.nteams = 0;
  t.team_order = nullptr;
  t.team_next = nullptr;
  t.dense_of = nullptr;
  t.dense_bin = nullptr;
  t.patch = nullptr;
  t.dense0 = 0;
  t.ndense = 0;
  t.dense_min = 0;
  t.dense_on = 0;
  t.dense_chunk = nullptr;
  t.dense_part0 = nullptr;
  t.patch_part = nullptr;
  t.chunk0 = 0;
  t.nchunks = 0;
  t.nbins = 1;
  t.ntiles = 1;
  for (int d = 0; d < MIRT_DMAX; d++) {
    t.B[d] = d < D ? B[d] : 1;
    t.nbin[d] = d < D ? (a.g.K[d] + B[d] - 1) / B[d] : 1;
    t.T[d] = d < D ? T[d] : 1;
    t.nb[d] = d < D ? (a.g.K[d] + T[d] - 1) / T[d] : 1;
    t.nbins *= t.nbin[d];
    t.ntiles *= t.nb[d];
  }
  t.wrap_ok = wrap_ok(a, t);
}

// Source bins per dimension: bins whose samples (binned by the first tap
// koff mod K) can have a tap inside tile b, i.e. koff in [lo-J+1, hi-1] mod K.
int build_sources(mirt_interp_plan *P, cudaStream_t st) {
  const InterpArgs &a = P->a;
  Tiling &t = P->t;
  std::vector<int> src[MIRT_DMAX], nsrc[MIRT_DMAX];
  std::vector<int4> run0(t.nb[0], make_int4(0, 1, 0, 0));
  for (int d = 0; d < MIRT_DMAX; d++) {
    const int nb = t.nb[d];
    src[d].assign((size_t)nb * MIRT_SRCMAX, 0);
    nsrc[d].assign(nb, 1);
    if (d >= a.g.D) continue;
    const int K = a.g.K[d], T = t.T[d], B = t.B[d], J = a.g.J[d];
    for (int b = 0; b < nb; b++) {
      const int lo = b * T, hi = std::min(lo + T, K);
      const long long n = (long long)(hi - lo) + J - 1;
      std::vector<int> list;
      if (n >= K) {
        for (int i = 0; i < t.nbin[d]; i++) list.push_back(i);
      } else {
        const int x0 = ((lo - J + 1) % K + K) % K;
        std::set<int> seen;
        for (long long i = 0; i < n; i++) {
          const int bb = (int)((x0 + i) % K) / B;
          if (!seen.count(bb)) {
            seen.insert(bb);
            list.push_back(bb);
          }
        }
      }
      if (d == 0) {
        // consecutive bins in order, split where the periodic wrap restarts at 0
        int4 r = make_int4(list[0], 1, 0, 0);
        size_t i = 1;
        for (; i < list.size() && list[i] == list[i - 1] + 1; i++) r.y++;
        if (i < list.size()) {
          r.z = list[i];
          r.w = 1;
          for (i++; i < list.size(); i++) {
            if (list[i] != list[i - 1] + 1) return fail(MIRT_ERR_ARG, "spread source runs");
            r.w++;
          }
        }
        run0[b] = r;
        continue;
      }
      if ((int)list.size() > MIRT_SRCMAX)
        return fail(MIRT_ERR_ARG, "spread tile spans too many sort bins");
      nsrc[d][b] = (int)list.size();
      for (size_t i = 0; i < list.size(); i++) src[d][(size_t)b * MIRT_SRCMAX + i] = list[i];
    }
  }
  CK(P->run0.alloc(run0.size() * sizeof(int4)));
  CK(cudaMemcpyAsync(P->run0.p, run0.data(), run0.size() * sizeof(int4), cudaMemcpyHostToDevice,
                     st));
  t.run0 = P->run0.as<int4>();
  for (int d = 0; d < MIRT_DMAX; d++) {
    CK(P->src[d].alloc(src[d].size() * sizeof(int)));
    CK(P->nsrc[d].alloc(nsrc[d].size() * sizeof(int)));
    CK(cudaMemcpyAsync(P->src[d].p, src[d].data(), src[d].size() * sizeof(int),
                       cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(P->nsrc[d].p, nsrc[d].data(), nsrc[d].size() * sizeof(int),
                       cudaMemcpyHostToDevice, st));
    t.src[d] = P->src[d].as<int>();
    t.nsrc[d] = P->nsrc[d].as<int>();
  }
  // the host vectors are released at scope exit: wait for the copies
  CK(cudaStreamSynchronize(st));
  return MIRT_OK;
}

// Fill geometry and upload tables.  Tables arrive as host FP64.
int plan_geometry(mirt_interp_plan *P, int D, const int *K, const int *J, const int *L,
                  const double *const *h_re, const double *const *h_im, int order, int C,
                  cudaStream_t st) {
  InterpArgs &a = P->a;
  a.g.D = D;
  long long stride = 1;
  const bool cplx = h_im != nullptr && h_im[0] != nullptr;
  a.real_tab = cplx ? 0 : 1;
  a.order = order;
  a.C = C;
  for (int d = 0; d < MIRT_DMAX; d++) {
    if (d < D) {
      a.g.K[d] = K[d];
      a.g.J[d] = J[d];
      a.g.L[d] = L[d];
      a.g.ncenter[d] = (int)std::floor(J[d] * L[d] / 2.);
      a.g.tlen[d] = J[d] * L[d] + 1;
      a.g.kstride[d] = stride;
      stride *= K[d];
    } else {
      a.g.K[d] = 1;
      a.g.J[d] = 1;
      a.g.L[d] = 1;
      a.g.ncenter[d] = 0;
      a.g.tlen[d] = 1;
      a.g.kstride[d] = stride;
    }
  }
  a.grid_elems = stride * C;
  for (int d = 0; d < D; d++) {
    const int n = a.g.tlen[d];
    if (cplx) {
      std::vector<float2> h(n);
      for (int i = 0; i < n; i++) h[i] = make_float2((float)h_re[d][i], (float)h_im[d][i]);
      CK(P->tab[d].alloc(n * sizeof(float2)));
      CK(cudaMemcpyAsync(P->tab[d].p, h.data(), n * sizeof(float2), cudaMemcpyHostToDevice, st));
      CK(cudaStreamSynchronize(st));
    } else {
      std::vector<float> h(n);
      for (int i = 0; i < n; i++) h[i] = (float)h_re[d][i];
      CK(P->tab[d].alloc(n * sizeof(float)));
      CK(cudaMemcpyAsync(P->tab[d].p, h.data(), n * sizeof(float), cudaMemcpyHostToDevice, st));
      CK(cudaStreamSynchronize(st));
    }
    a.tab[d] = P->tab[d].p;
  }
  return MIRT_OK;
}

// Spread work list.  The work of a tile is the number of sample visits over
// its source bins.  Tiles with more than split_chunk visits (the dense k-space
// centre of radial and kooshball trajectories) are split into tasks of
// split_chunk visits whose partial tiles a reduction sums in fixed order, so
// no single CTA serialises a dense tile.  Tasks run heaviest first.
int build_tasks(mirt_interp_plan *P, cudaStream_t st) {
  Tiling &t = P->t;
  const int D = P->a.g.D;
  const long long ntile_all = (long long)t.ntiles * t.nslice;
  const long long nbin_all = (long long)t.nbins * t.nslice;
  std::vector<int> bs(nbin_all + 1);
  CK(cudaMemcpyAsync(bs.data(), P->bin_start.p, (nbin_all + 1) * sizeof(int),
                     cudaMemcpyDeviceToHost, st));
  std::vector<int> src[MIRT_DMAX], nsrc[MIRT_DMAX];
  for (int d = 0; d < MIRT_DMAX; d++) {
    src[d].resize((size_t)t.nb[d] * MIRT_SRCMAX);
    nsrc[d].resize(t.nb[d]);
    CK(cudaMemcpyAsync(src[d].data(), t.src[d], src[d].size() * sizeof(int),
                       cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(nsrc[d].data(), t.nsrc[d], nsrc[d].size() * sizeof(int),
                       cudaMemcpyDeviceToHost, st));
  }
  std::vector<int4> run0(t.nb[0]);
  CK(cudaMemcpyAsync(run0.data(), t.run0, run0.size() * sizeof(int4), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  const long long chunk = std::max(32, P->split_chunk);
  struct Task {
    long long work;
    int tile, v0, v1, slot, color;
  };
  std::vector<int> red_color;
  std::vector<Task> tasks;
  std::vector<int4> red;
  int nslot = 0;
  for (long long task = 0; task < ntile_all; task++) {
    const int tile = (int)(task % t.ntiles);
    const long long slice = task / t.ntiles;
    int b[MIRT_DMAX] = {0, 0, 0}, r = tile;
    for (int d = 0; d < D; d++) {
      b[d] = r % t.nb[d];
      r /= t.nb[d];
    }
    long long w = 0;
    int color = 0;
    if (t.own) {
      // the tile's own samples: first tap inside the tile, one range per row
      const int lo0 = b[0] * t.T[0], lo1 = b[1] * t.T[1];
      const int ext0 = std::min(t.T[0], P->a.g.K[0] - lo0);
      const int ext1 = std::min(t.T[1], P->a.g.K[1] - lo1);
      for (int i1 = 0; i1 < ext1; i1++) {
        const long long key = slice * t.nbins + (long long)(lo1 + i1) * t.nbin[0] + lo0;
        w += bs[key + ext0] - bs[key];
      }
      color = (b[0] & 1) | ((b[1] & 1) << 1);
    } else {
    const int n1 = D > 1 ? nsrc[1][b[1]] : 1, n2 = D > 2 ? nsrc[2][b[2]] : 1;
    const int4 rr = run0[b[0]];
    for (int i2 = 0; i2 < n2; i2++)
      for (int i1 = 0; i1 < n1; i1++)
        for (int k = 0; k < 2; k++) {
          const int rs = k ? rr.z : rr.x, rl = k ? rr.w : rr.y;
          if (rl == 0) continue;
          long long row = 0;
          if (D > 1) row += (long long)src[1][b[1] * MIRT_SRCMAX + i1] * t.nbin[0];
          if (D > 2) row += (long long)src[2][b[2] * MIRT_SRCMAX + i2] * t.nbin[0] * t.nbin[1];
          const long long bin = slice * t.nbins + row + rs;
          w += bs[bin + rl] - bs[bin];
        }
    }
    if (w >= (1ll << 31)) return fail(MIRT_ERR_ARG, "too many samples in one tile");
    if (w <= chunk) {
      tasks.push_back({w, (int)task, 0, (int)w, -1, color});
    } else {
      const int np = (int)((w + chunk - 1) / chunk);
      red.push_back(make_int4((int)task, nslot, np, 0));
      red_color.push_back(color);
      for (int i = 0; i < np; i++) {
        const long long v0 = i * chunk, v1 = std::min(w, v0 + chunk);
        tasks.push_back({v1 - v0, (int)task, (int)v0, (int)v1, nslot + i, color});
      }
      nslot += np;
    }
  }
  if (P->heavy_first)
    std::stable_sort(tasks.begin(), tasks.end(),
                     [](const Task &x, const Task &y) { return x.work > y.work; });
  for (int c = 0; c < 9; c++) t.color_beg[c] = t.red_beg[c] = 0;
  if (t.own) {
    // colour-major (each colour one launch), the order above within a colour
    std::stable_sort(tasks.begin(), tasks.end(),
                     [](const Task &x, const Task &y) { return x.color < y.color; });
    std::vector<int> idx(red.size());
    for (size_t i = 0; i < idx.size(); i++) idx[i] = (int)i;
    std::stable_sort(idx.begin(), idx.end(),
                     [&](int x, int y) { return red_color[x] < red_color[y]; });
    std::vector<int4> red2(red.size());
    for (size_t i = 0; i < idx.size(); i++) red2[i] = red[idx[i]];
    red.swap(red2);
    for (int c = 0; c < 4; c++) {
      t.color_beg[c + 1] = t.color_beg[c];
      for (const Task &k : tasks) t.color_beg[c + 1] += k.color == c;
      t.red_beg[c + 1] = t.red_beg[c];
      for (int rc : red_color) t.red_beg[c + 1] += rc == c;
    }
  }
  const size_t nt = tasks.size();
  std::vector<int> tt(nt), ts(nt);
  std::vector<int2> tr(nt);
  for (size_t i = 0; i < nt; i++) {
    tt[i] = tasks[i].tile;
    tr[i] = make_int2(tasks[i].v0, tasks[i].v1);
    ts[i] = tasks[i].slot;
  }
  CK(P->task_tile.alloc(std::max<size_t>(nt, 1) * sizeof(int)));
  CK(P->task_range.alloc(std::max<size_t>(nt, 1) * sizeof(int2)));
  CK(P->task_slot.alloc(std::max<size_t>(nt, 1) * sizeof(int)));
  CK(P->red.alloc(std::max<size_t>(red.size(), 1) * sizeof(int4)));
  if (nt) {
    CK(cudaMemcpyAsync(P->task_tile.p, tt.data(), nt * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(P->task_range.p, tr.data(), nt * sizeof(int2), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(P->task_slot.p, ts.data(), nt * sizeof(int), cudaMemcpyHostToDevice, st));
  }
  if (!red.empty())
    CK(cudaMemcpyAsync(P->red.p, red.data(), red.size() * sizeof(int4), cudaMemcpyHostToDevice,
                       st));
  size_t npts = 1;
  for (int d = 0; d < D; d++) npts *= t.T[d];
  if (t.own) npts = (size_t)(t.T[0] + 5) * (t.T[1] + 5);
  const int cw = P->ls.cw;
  const size_t nchunk = (P->a.C + cw - 1) / cw;
  const size_t sbytes = (size_t)nslot * nchunk * npts * cw * sizeof(float2);
  if (P->scratch.bytes < sbytes) CK(P->scratch.alloc(sbytes));
  CK(cudaStreamSynchronize(st));
  t.ntask = (int)nt;
  t.task_tile = P->task_tile.as<int>();
  t.task_range = P->task_range.as<int2>();
  t.task_slot = P->task_slot.as<int>();
  t.nred = (int)red.size();
  t.red = P->red.as<int4>();
  t.scratch = P->scratch.as<float2>();
  return MIRT_OK;
}

// Slices, tiling, bin sort.  P->tm must hold the FP64 coordinates on device.
int plan_finish(mirt_interp_plan *P, long long Mtot, const long long *moff, int nslice,
                cudaStream_t st) {
  InterpArgs &a = P->a;
  a.Mtot = Mtot;
  a.tm = P->tm.as<double>();
  P->t.nslice = nslice;
  P->moff_host.assign(moff, moff + nslice + 1);
  if (nslice > 1) {
    CK(P->moff.alloc((nslice + 1) * sizeof(long long)));
    CK(cudaMemcpyAsync(P->moff.p, moff, (nslice + 1) * sizeof(long long),
                       cudaMemcpyHostToDevice, st));
    CK(P->slice.alloc(Mtot * sizeof(int)));
    CK(launch_fill_slice(P->moff.as<long long>(), nslice, Mtot, P->slice.as<int>(), st));
    a.slice_id = P->slice.as<int>();
  } else {
    a.slice_id = nullptr;
  }
  choose_config(P);
  int rc = build_sources(P, st);
  if (rc) return rc;
  const long long nbins = (long long)P->t.nbins * nslice;
  if (nbins >= (1ll << 31)) return fail(MIRT_ERR_ARG, "too many grid tiles");
  CK(P->keys.alloc(std::max<long long>(Mtot, 1) * sizeof(uint32_t)));
  CK(P->perm.alloc(std::max<long long>(Mtot, 1) * sizeof(int)));
  CK(P->bin_start.alloc((nbins + 1) * sizeof(int)));
  CK(P->sorttmp.alloc(radix_sort_tmp_bytes(Mtot)));
  CK(launch_bin_keys(a, P->t, P->keys.as<uint32_t>(), st));
  CK(radix_sort_bins(P->keys.as<uint32_t>(), Mtot, (int)nbins, P->sorttmp.p, P->perm.as<int>(),
                     P->bin_start.as<int>(), st));
  // per-sample arrays into sorted order, so that staging reads are coalesced
  {
    DMem tm2, sl2, ph2;
    CK(tm2.alloc(std::max<long long>(Mtot, 1) * a.g.D * sizeof(double)));
    if (a.slice_id) CK(sl2.alloc(std::max<long long>(Mtot, 1) * sizeof(int)));
    if (a.phase) CK(ph2.alloc(std::max<long long>(Mtot, 1) * sizeof(float2)));
    CK(launch_permute_samples(a.tm, a.slice_id, a.phase, P->perm.as<int>(), Mtot, a.g.D,
                              tm2.as<double>(), sl2.as<int>(), ph2.as<float2>(), st));
    CK(cudaStreamSynchronize(st));
    swap_mem(P->tm, tm2);
    a.tm = P->tm.as<double>();
    if (a.slice_id) {
      swap_mem(P->slice, sl2);
      a.slice_id = P->slice.as<int>();
    }
    if (a.phase) {
      swap_mem(P->phase, ph2);
      a.phase = P->phase.as<float2>();
    }
  }
  a.perm = P->perm.as<int>();
  P->sorttmp.release();
  // tap coefficients and first taps of every position, once per trajectory
  a.SJ = 0;
  for (int d = 0; d < a.g.D; d++) a.SJ += a.g.J[d];
  CK(P->wtap.alloc(std::max<long long>(Mtot, 1) * a.SJ * sizeof(float2)));
  CK(P->k0tap.alloc(std::max<long long>(Mtot, 1) * sizeof(int4)));
  CK(launch_prep_taps(a, P->wtap.as<float2>(), P->k0tap.as<int4>(), st));
  a.W = P->wtap.as<float2>();
  a.K0 = P->k0tap.as<int4>();
  // gather order: the sorted positions re-sorted (stably) by 4-point blocks
  // of their first taps, so that a CTA's consecutive samples share grid rows
  // in every dimension; the gather gets its own copy of the records in that
  // order, read sequentially
  P->ag = a;
  P->gtma = 0;
  if (a.g.D > 1 && Mtot > 0) {
    // 8-point blocks where the gather runs on TMA-staged tiles (2D, J = 6,
    // 32-coil chunks), 4-point blocks otherwise
    const int gbs = (gather_tma_ok(a) && P->lg.cw == 32) ? gather_tma_block() : 4;
    Tiling t4 = P->t;
    t4.nbins = 1;
    for (int d = 0; d < MIRT_DMAX; d++) {
      t4.B[d] = d < a.g.D ? std::min(gbs, a.g.K[d]) : 1;
      t4.nbin[d] = d < a.g.D ? (a.g.K[d] + t4.B[d] - 1) / t4.B[d] : 1;
      t4.nbins *= t4.nbin[d];
    }
    const long long nb4 = (long long)t4.nbins * nslice;
    DMem keys4, tmp4;
    DMem &bs4 = P->gblk;
    CK(keys4.alloc(Mtot * sizeof(uint32_t)));
    CK(bs4.alloc((nb4 + 1) * sizeof(int)));
    CK(tmp4.alloc(radix_sort_tmp_bytes(Mtot)));
    DMem gorder;
    CK(gorder.alloc(Mtot * sizeof(int)));
    CK(launch_bin_keys(a, t4, keys4.as<uint32_t>(), st));  // a.tm, a.slice_id already sorted
    CK(radix_sort_bins(keys4.as<uint32_t>(), Mtot, (int)nb4, tmp4.p, gorder.as<int>(),
                       bs4.as<int>(), st));
    CK(P->wtap_g.alloc(Mtot * a.SJ * sizeof(float2)));
    CK(P->k0tap_g.alloc(Mtot * sizeof(int4)));
    CK(P->perm_g.alloc(Mtot * sizeof(int)));
    if (a.phase) CK(P->phase_g.alloc(Mtot * sizeof(float2)));
    mirt_plan_kernels::gather_records_kernel<<<(unsigned)((Mtot + 255) / 256), 256, 0, st>>>(
        gorder.as<int>(), Mtot, a.SJ, a.W, a.K0, a.perm, a.phase, P->wtap_g.as<float2>(),
        P->k0tap_g.as<int4>(), P->perm_g.as<int>(), P->phase_g.as<float2>());
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    P->ag.W = P->wtap_g.as<float2>();
    P->ag.K0 = P->k0tap_g.as<int4>();
    P->ag.perm = P->perm_g.as<int>();
    P->ag.phase = a.phase ? P->phase_g.as<float2>() : nullptr;
    const bool tma3 = a.g.D == 3 && gather_tma3_ok(a) && gbs == gather_tma3_block();
    if ((gbs == gather_tma_block() && a.g.D == 2) || tma3) {
      // work items: up to gather_tma_item() (3D: gather_tma3_item()) samples of
      // one non-empty block
      std::vector<int> hb(nb4 + 1);
      CK(cudaMemcpy(hb.data(), bs4.p, (nb4 + 1) * sizeof(int), cudaMemcpyDeviceToHost));
      const int rc_n = tma3 ? gather_tma3_item() : gather_tma_item();
      const long long per = (long long)t4.nbins;
      std::vector<int2> items;
      P->gitem_slice.assign(nslice + 1, 0);
      for (long long bk = 0; bk < nb4; bk++) {
        if (bk % per == 0) P->gitem_slice[bk / per] = (long long)items.size();
        for (int p0 = hb[bk]; p0 < hb[bk + 1]; p0 += rc_n) items.push_back(make_int2((int)bk, p0));
      }
      P->gitem_slice[nslice] = (long long)items.size();
      CK(P->gitem.alloc(std::max<size_t>(items.size(), 1) * sizeof(int2)));
      if (!items.empty())
        CK(cudaMemcpy(P->gitem.p, items.data(), items.size() * sizeof(int2), cudaMemcpyHostToDevice));
      CK(P->orec_g.alloc(Mtot * sizeof(int4)));
      mirt_plan_kernels::out_records_kernel<<<(unsigned)((Mtot + 255) / 256), 256, 0, st>>>(
          Mtot, P->ag.perm, P->ag.phase, P->orec_g.as<int4>());
      CK(cudaGetLastError());
      CK(cudaStreamSynchronize(st));
      P->gbk = GatherBlocks{P->gblk.as<int>(), P->gitem.as<int2>(), P->orec_g.as<int4>(), gbs,
                            t4.nbin[0], t4.nbin[1], t4.nbin[2]};
      CK(P->gfault.alloc(sizeof(int)));
      CK(cudaMemset(P->gfault.p, 0, sizeof(int)));
      P->gtma = 1;  // the default where it applies; the autotuner times both
    }
  }
  int rc2 = build_tasks(P, st);
  if (rc2) return rc2;
  CK(query_gather_grid(a, P->lg));
  // 2D, J = 6, 32-coil chunks: the row sweep by default, one grid row per
  // team, balanced segments (about 64k teams, heaviest first)
  if (sweep_ok(a, P->t) || sweep3_ok(a, P->t, P->ls.cw)) {
    int rc3 = build_dense(P, kDenseBin, st);
    if (rc3) return rc3;
    P->t.dense_on = P->t.dense_of ? 1 : 0;
  }
  if (sweep_ok(a, P->t) && P->ls.cw == 32) {
    int rc3 = sweep_buffer(P);
    if (rc3) return rc3;
    rc3 = build_sweep_teams(P, 1, 65536, st);
    if (rc3) return rc3;
    // the staged sweep's records (FFMA2 operand pairs of the taps)
    CK(P->wsw.alloc(std::max<long long>(Mtot, 1) * 9 * sizeof(float4)));
    if (Mtot > 0)
      mirt_plan_kernels::sweep_records_kernel<<<(unsigned)((Mtot + 255) / 256), 256, 0, st>>>(
          a.W, Mtot, P->wsw.as<float4>());
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    P->t.wsw = P->wsw.as<float4>();
  }
  // 3D, J = 6, coil chunks of 8, 16 or 32: the line sweep, two segments per line
  if (sweep3_ok(a, P->t, P->ls.cw)) {
    int rc3 = sweep_buffer(P);
    if (rc3) return rc3;
    rc3 = set_line_sweep3(P, 2, st);
    if (rc3) return rc3;
  }
  return MIRT_OK;
}

// Re-tile the spread (tiles of T[d] points, multiples of the sort bins) and
// rebuild its source lists and CTA order; the sort itself is unchanged.
int set_spread_tiles(mirt_interp_plan *P, const int *T, cudaStream_t st) {
  Tiling &t = P->t;
  const int D = P->a.g.D;
  t.ntiles = 1;
  for (int d = 0; d < MIRT_DMAX; d++) {
    t.T[d] = d < D ? T[d] : 1;
    t.nb[d] = d < D ? (P->a.g.K[d] + t.T[d] - 1) / t.T[d] : 1;
    t.ntiles *= t.nb[d];
  }
  t.wrap_ok = wrap_ok(P->a, t);
  if (t.own && !own_ok(P->a, t)) t.own = 0;
  int rc = build_sources(P, st);
  if (rc) return rc;
  return build_tasks(P, st);
}

struct SpreadCand {
  int T[MIRT_DMAX];
  int threads, padc, atomic, own, sweep, sweep_rows;
  int dense = 0;  // 2D row sweep with dense-bin patches (one-row bands)
  int staged = 0;  // 2D row sweep staged per column (1), reading the caller's samples (2)
};

// spare columns the J = 6 row update can use (0 elsewhere)
int padc_max(const InterpArgs &a) {
  if (a.g.D < 2) return 0;
  for (int d = 0; d < a.g.D; d++)
    if (a.g.J[d] != 6) return 0;
  return 5;
}

// MIRT_AUTOTUNE_LOG=1 in the environment: the autotuner prints every
// candidate's time to stderr.
bool autotune_log() {
  const char *v = std::getenv("MIRT_AUTOTUNE_LOG");
  return v && v[0] && v[0] != '0';
}

// Time `fn` (one launch) on the stream: one warm-up, then the best of 3.
template <class F>
int time_launch(F fn, cudaStream_t st, float *ms) {
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  *ms = 1e30f;
  for (int it = 0; it < 4; it++) {
    CK(cudaEventRecord(e0, st));
    cudaError_t e = fn();
    if (e != cudaSuccess) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      cudaGetLastError();
      return fail(MIRT_ERR_CUDA, std::string("autotune launch: ") + cudaGetErrorString(e));
    }
    CK(cudaEventRecord(e1, st));
    CK(cudaEventSynchronize(e1));
    float t = 0;
    CK(cudaEventElapsedTime(&t, e0, e1));
    if (it > 0 && t < *ms) *ms = t;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return MIRT_OK;
}

int validate_geometry(int D, const int *K, const int *J, const int *L, int order, bool cplx,
                      long long Mtot, int C) {
  if (D < 1 || D > MIRT_DMAX) return fail(MIRT_ERR_ARG, "D must be 1, 2 or 3");
  for (int d = 0; d < D; d++) {
    if (K[d] < 1) return fail(MIRT_ERR_ARG, "K must be positive");
    if (J[d] < 1 || J[d] > MIRT_JMAX) return fail(MIRT_ERR_ARG, "J must be in 1..16");
    if (L[d] < 1) return fail(MIRT_ERR_ARG, "L must be positive");
    if ((long long)J[d] * L[d] + 1 > (1ll << 30)) return fail(MIRT_ERR_ARG, "table too long");
    // the kernels wrap a tap index k0 + j (k0 in [0, K)) at most once
    if (J[d] > K[d]) return fail(MIRT_ERR_ARG, "J must not exceed K in any dimension");
  }
  if (order != 0 && order != 1) return fail(MIRT_ERR_ARG, "bad order");
  if (cplx && order) return fail(MIRT_ERR_ARG, "only 0th order implemented for complex");
  if (Mtot < 0 || Mtot >= (1ll << 31)) return fail(MIRT_ERR_ARG, "too many samples");
  if (C < 0) return fail(MIRT_ERR_ARG, "bad column count");
  long long g = C;
  for (int d = 0; d < D; d++) g *= K[d];
  if (g >= (1ll << 31)) return fail(MIRT_ERR_ARG, "grid too large for one slice");
  return MIRT_OK;
}

}  // namespace

// The plan whose launches a setter tunes: a 4D plan's 3D plan, else the plan.
static mirt_interp_plan *launch_plan(mirt_interp_plan *P) { return P->sub4 ? P->sub4 : P; }

extern "C" {

const char *mirt_last_error(void) { return g_err.c_str(); }

int mirt_version(void) { return 100; }

int mirt_interp_plan_create(mirt_interp_plan **plan, int32_t D, const int32_t *K,
                            const int32_t *J, const int32_t *L, const double *const *h_re,
                            const double *const *h_im, int32_t order, const double *tm,
                            int64_t Mtot, const int64_t *slice_moff, int32_t nslice,
                            int32_t ncol, const double *phase_re, const double *phase_im,
                            void *stream) try {
  if (!plan) return fail(MIRT_ERR_ARG, "plan pointer is NULL");
  *plan = nullptr;
  if (!K || !J || !L || !h_re || (Mtot > 0 && !tm)) return fail(MIRT_ERR_ARG, "NULL argument");
  if (D < 1 || D > 4) return fail(MIRT_ERR_ARG, "D must be 1, 2, 3 or 4");
  const bool cplx = h_im != nullptr && h_im[0] != nullptr;
  for (int d = 0; d < D; d++)
    if (!h_re[d] || (cplx && !h_im[d])) return fail(MIRT_ERR_ARG, "NULL table");
  if (nslice < 1) return fail(MIRT_ERR_ARG, "nslice must be >= 1");
  if (D == 4) {
    // the 4th dimension's taps are wrapped on the host by a general modulo
    if (K[3] < 1) return fail(MIRT_ERR_ARG, "K must be positive");
    if (J[3] < 1 || J[3] > MIRT_JMAX) return fail(MIRT_ERR_ARG, "J must be in 1..16");
    if (L[3] < 1) return fail(MIRT_ERR_ARG, "L must be positive");
    if ((long long)J[3] * L[3] + 1 > (1ll << 30)) return fail(MIRT_ERR_ARG, "table too long");
  }
  int rc = validate_geometry(D == 4 ? 3 : D, K, J, L, order, cplx, Mtot, ncol);
  if (rc) return rc;
  std::vector<long long> moff(nslice + 1);
  if (slice_moff) {
    for (int s = 0; s <= nslice; s++) moff[s] = slice_moff[s];
    if (moff[0] != 0 || moff[nslice] != Mtot)
      return fail(MIRT_ERR_ARG, "slice offsets must start at 0 and end at Mtot");
    for (int s = 0; s < nslice; s++)
      if (moff[s + 1] < moff[s]) return fail(MIRT_ERR_ARG, "slice offsets must not decrease");
  } else {
    if (nslice != 1) return fail(MIRT_ERR_ARG, "slice offsets required for nslice > 1");
    moff[0] = 0;
    moff[1] = Mtot;
  }
  rc = device_ok();
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  if (D == 4)
    return plan4_create(plan, K, J, L, h_re, h_im, order, tm, Mtot, moff.data(), nslice, ncol,
                        phase_re, phase_im, st);
  auto *P = new mirt_interp_plan();
  rc = plan_geometry(P, D, K, J, L, h_re, h_im, order, ncol, st);
  if (!rc) {
    cudaError_t e = P->tm.alloc(std::max<long long>(Mtot, 1) * D * sizeof(double));
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(P->tm.p, tm, Mtot * D * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && phase_re) {
      std::vector<float2> ph(Mtot);
      for (long long m = 0; m < Mtot; m++)
        ph[m] = make_float2((float)phase_re[m], phase_im ? (float)phase_im[m] : 0.f);
      e = P->phase.alloc(std::max<long long>(Mtot, 1) * sizeof(float2));
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(P->phase.p, ph.data(), Mtot * sizeof(float2), cudaMemcpyHostToDevice,
                            st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      P->a.phase = P->phase.as<float2>();
    }
    if (e != cudaSuccess) rc = fail(MIRT_ERR_CUDA, std::string("plan upload: ") + cudaGetErrorString(e));
  }
  if (!rc) rc = plan_finish(P, Mtot, moff.data(), nslice, st);
  if (!rc) {
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = fail(MIRT_ERR_CUDA, std::string("plan: ") + cudaGetErrorString(e));
  }
  if (rc) {
    delete P;
    return rc;
  }
  *plan = P;
  return MIRT_OK;
} catch (const std::bad_alloc &) {
  return fail(MIRT_ERR_ALLOC, "out of host memory");
}

int mirt_interp_plan_forward(mirt_interp_plan *P, const void *ck, void *fm, void *stream) {
  if (!P) return fail(MIRT_ERR_ARG, "plan is NULL");
  if (P->sub4)
    return plan4_forward(P, static_cast<const float2 *>(ck), static_cast<float2 *>(fm),
                         as_stream(stream));
  CK(plan_gather(P, static_cast<const float2 *>(ck), static_cast<float2 *>(fm),
                   as_stream(stream)));
  return MIRT_OK;
}

int mirt_interp_plan_adjoint(mirt_interp_plan *P, const void *fm, void *ck, void *stream) {
  if (!P) return fail(MIRT_ERR_ARG, "plan is NULL");
  if (P->sub4)
    return plan4_adjoint(P, static_cast<const float2 *>(fm), static_cast<float2 *>(ck),
                         as_stream(stream));
  CK(launch_spread(P->a, P->t, P->ls, P->bin_start.as<int>(), static_cast<const float2 *>(fm),
                   static_cast<float2 *>(ck), as_stream(stream)));
  return MIRT_OK;
}

int mirt_interp_plan_autotune(mirt_interp_plan *P, void *stream) try {
  if (!P) return fail(MIRT_ERR_ARG, "plan is NULL");
  P = launch_plan(P);
  cudaStream_t st = as_stream(stream);
  const InterpArgs &a = P->a;
  const int D = a.g.D, cw = P->ls.cw;
  const long long ngrid = (long long)P->t.nslice * a.grid_elems;
  const long long nsamp = a.Mtot * (long long)a.C;
  if (ngrid == 0 || nsamp == 0) return MIRT_OK;
  DMem grid, samp;
  CK(grid.alloc(ngrid * sizeof(float2)));
  CK(samp.alloc(nsamp * sizeof(float2)));
  CK(cudaMemsetAsync(samp.p, 0, nsamp * sizeof(float2), st));
  CK(cudaMemsetAsync(grid.p, 0, ngrid * sizeof(float2), st));
  // spread candidates: tile shape (multiples of the sort bins), warps
  std::vector<SpreadCand> cands;
  const int pmax = padc_max(a);
  auto add = [&](int t0, int t1, int t2, int threads) {
    const int npc = pmax ? 2 : 1;
    for (int ip = 0; ip < npc; ip++) {
      const int pc = ip ? pmax : 0;
      SpreadCand c{{t0, t1, t2}, threads, pc, 0, 0, 0, 1};
      for (int d = 0; d < D; d++) {
        const int kr = (a.g.K[d] + P->t.B[d] - 1) / P->t.B[d] * P->t.B[d];
        if (c.T[d] > kr) c.T[d] = kr;
        c.T[d] = (c.T[d] + P->t.B[d] - 1) / P->t.B[d] * P->t.B[d];
      }
      size_t npts = (size_t)c.T[0] + 2 * pc;
      for (int d = 1; d < D; d++) npts *= c.T[d];
      if (npts * cw * 8 <= 160 * 1024) {
        cands.push_back(c);
        // shared-tile variant: every warp takes whole visits, atomic adds
        if (!P->deterministic)
          for (int th : {128, 256}) {
            SpreadCand ca = c;
            ca.threads = th;
            ca.atomic = 1;
            cands.push_back(ca);
          }
      }
    }
    // ownership spread (2D, J = 6): padded tile, warps on bands of its rows
    if (D == 2 && pmax) {
      Tiling tt = P->t;
      tt.T[0] = t0;
      tt.T[1] = t1;
      const size_t pts = (size_t)(t0 + 5) * (t1 + 5);
      if (own_ok(a, tt) && pts * cw * 8 <= 160 * 1024 && threads == 32)
        for (int th = 32; th <= 256 && th / 32 <= t1 + 5; th *= 2)
          cands.push_back(SpreadCand{{t0, t1, 1}, th, 0, 0, 1, 0, 1});
    }
  };
  if (D == 1) {
    for (int t0 : {64, 128, 256, 512})
      for (int th : {32, 64}) add(t0, 1, 1, th);
  } else if (D == 2) {
    // warps per tile: each owns a band of at least one row
    for (int t0 : {8, 16, 32})
      for (int t1 : {8, 16, 32})
        for (int th = 32; th <= 256 && th / 32 <= t1; th *= 2) add(t0, t1, 1, th);
  } else {
    // each warp owns a band of at least one plane
    for (int t0 : {8, 16})
      for (int t1 : {8, 16})
        for (int t2 : {8, 16})
          for (int th = 32; th <= 256 && th / 32 <= t2; th *= 2) add(t0, t1, t2, th);
  }
  // row sweep (no tiles): bands of 1, 2 or 4 rows, whole rows or uniform
  // segments of at least 32 columns, or balanced teams (sweep = -1)
  if (sweep_ok(a, P->t) && sweep_buffer(P) == MIRT_OK)
    for (int dense : {0, 1})
      for (int rows : {1, 2, 4})
        for (int nseg = -1; nseg <= 16 && (nseg <= 1 || a.g.K[0] / nseg >= 32);
             nseg = nseg < 0 ? 1 : nseg * 2)
          if (!dense || (rows == 1 && P->t.dense_of))
            for (int staged : {0, 1, 2})
              if (!staged || (cw == 32 && !dense && P->t.wsw))
                cands.push_back(SpreadCand{{P->t.T[0], P->t.T[1], P->t.T[2]}, P->ls.threads, 0,
                                           0, 0, nseg, rows, dense, staged});
  // 3D line sweep: 1, 2, 4 or 8 segments per line block
  if (sweep3_ok(a, P->t, cw) && sweep_buffer(P) == MIRT_OK)
    for (int nseg : {1, 2, 4, 8})
      cands.push_back(SpreadCand{{P->t.T[0], P->t.T[1], P->t.T[2]}, P->ls.threads, 0, 0, 0,
                                 nseg, 1});
  SpreadCand best{};
  float best_ms = 1e30f;
  int built_rows = 0;  // rows of the team list last built
  for (const SpreadCand &c : cands) {
    P->t.own = c.own;
    P->t.sweep = c.sweep;
    P->t.sweep_rows = c.sweep_rows;
    P->t.dense_on = c.dense;
    P->t.sweep_staged = c.staged;
    if (c.sweep < 0 && built_rows != c.sweep_rows) {
      int rc = build_sweep_teams(P, c.sweep_rows, 65536, st);
      if (rc) return rc;
      built_rows = c.sweep_rows;
    } else if (c.sweep > 0) {
      int rc = D == 3 ? set_line_sweep3(P, c.sweep, st)
                      : set_uniform_sweep(P, c.sweep, c.sweep_rows, st);
      if (rc) return rc;
      built_rows = 0;  // the work queue now orders uniform segments
    }
    int rc = set_spread_tiles(P, c.T, st);
    if (rc) continue;
    P->ls.threads = c.threads;
    P->t.padc = c.padc;
    P->ls.atomic = c.atomic;
    float ms = 0;
    rc = time_launch([&]() {
      return launch_spread(P->a, P->t, P->ls, P->bin_start.as<int>(), samp.as<float2>(),
                           grid.as<float2>(), st);
    }, st, &ms);
    if (rc) return rc;
    if (autotune_log())
      std::fprintf(stderr,
                   "mirt autotune spread: tile %dx%dx%d threads %d padc %d atomic %d own %d "
                   "sweep %d rows %d dense %d staged %d: %.3f ms\n",
                   c.T[0], c.T[1], c.T[2], c.threads, c.padc, c.atomic, c.own, c.sweep,
                   c.sweep_rows, c.dense, c.staged, ms);
    if (ms < best_ms) {
      best_ms = ms;
      best = c;
    }
  }
  if (best_ms < 1e30f) {
    P->t.own = best.own;
    P->t.sweep = best.sweep;
    P->t.sweep_rows = best.sweep_rows;
    P->t.dense_on = best.dense;
    P->t.sweep_staged = best.staged;
    if (best.sweep < 0 && built_rows != best.sweep_rows) {
      int rc = build_sweep_teams(P, best.sweep_rows, 65536, st);
      if (rc) return rc;
    } else if (best.sweep > 0) {
      int rc = D == 3 ? set_line_sweep3(P, best.sweep, st)
                      : set_uniform_sweep(P, best.sweep, best.sweep_rows, st);
      if (rc) return rc;
    }
    int rc = set_spread_tiles(P, best.T, st);
    if (rc) return rc;
    P->ls.threads = best.threads;
    P->t.padc = best.padc;
    P->ls.atomic = best.atomic;
  }
  // split size of heavy tiles (sample visits per spread task)
  if (!P->t.sweep) {
    int best_chunk = P->split_chunk;
    float bc_ms = 1e30f;
    for (int chunk : {256, 512, 1024, 2048, 4096, 16384}) {
      P->split_chunk = chunk;
      int rc = build_tasks(P, st);
      if (rc) return rc;
      float ms = 0;
      rc = time_launch([&]() {
        return launch_spread(P->a, P->t, P->ls, P->bin_start.as<int>(), samp.as<float2>(),
                             grid.as<float2>(), st);
      }, st, &ms);
      if (rc) return rc;
      if (ms < bc_ms) {
        bc_ms = ms;
        best_chunk = chunk;
      }
    }
    P->split_chunk = best_chunk;
    // task order: heaviest first (load balance) or grid order (L2 reuse of
    // neighbouring bins)
    float order_ms[2] = {1e30f, 1e30f};
    for (int hf = 0; hf < 2; hf++) {
      P->heavy_first = hf;
      int rc = build_tasks(P, st);
      if (rc) return rc;
      rc = time_launch([&]() {
        return launch_spread(P->a, P->t, P->ls, P->bin_start.as<int>(), samp.as<float2>(),
                             grid.as<float2>(), st);
      }, st, &order_ms[hf]);
      if (rc) return rc;
    }
    P->heavy_first = order_ms[1] <= order_ms[0] ? 1 : 0;
    int rc = build_tasks(P, st);
    if (rc) return rc;
  }
  // gather candidates: CTA size of the plain gather, and the TMA-staged gather
  Launch bestg = P->lg;
  float bestg_ms = 1e30f;
  const int had_tma = P->gbk.item != nullptr;
  int best_tma = 0;
  P->gtma = 0;
  for (int threads : {64, 128, 256}) {
    Launch l = P->lg;
    l.threads = threads;
    l.grid = 0;
    CK(query_gather_grid(P->a, l));
    float ms = 0;
    int rc = time_launch([&]() {
      return launch_gather(P->ag, l, grid.as<float2>(), samp.as<float2>(), st);
    }, st, &ms);
    if (rc) return rc;
    if (ms < bestg_ms) {
      bestg_ms = ms;
      bestg = l;
    }
  }
  if (had_tma)
    for (int mode : {1, 2}) {  // tiles of 32 or 16 coils (3D: of 8 coils, mode 1 only)
      if (mode == 2 && a.g.D == 3) continue;
      P->gtma = mode;
      float ms = 0;
      int rc = time_launch([&]() {
        return plan_gather(P, grid.as<float2>(), samp.as<float2>(), st);
      }, st, &ms);
      if (rc) return rc;
      if (autotune_log())
        std::fprintf(stderr, "mirt autotune gather: TMA tiles of %d coils: %.3f ms\n",
                     a.g.D == 3 ? 8 : mode == 2 ? 16 : 32, ms);
      if (ms < bestg_ms) {
        bestg_ms = ms;
        best_tma = mode;
      }
    }
  P->gtma = best_tma;
  P->lg = bestg;
  CK(cudaStreamSynchronize(st));
  return MIRT_OK;
} catch (const std::bad_alloc &) {
  return fail(MIRT_ERR_ALLOC, "out of host memory");
}

int mirt_interp_plan_config(mirt_interp_plan *P, int32_t *out, int32_t n) {
  if (!P || !out) return fail(MIRT_ERR_ARG, "NULL argument");
  P = launch_plan(P);
  const int32_t v[23] = {P->t.T[0], P->t.T[1], P->t.T[2], P->ls.threads, P->heavy_first, P->ls.cw,
                         P->lg.threads, P->lg.sb, P->lg.grid, P->t.B[0], P->t.B[1], P->t.B[2],
                         P->split_chunk, P->t.ntask, P->t.padc, P->t.nred, P->ls.atomic,
                         P->t.own, P->t.sweep, P->t.sweep_rows, P->gtma, P->t.dense_on,
                         P->t.sweep_staged};
  for (int i = 0; i < n && i < 23; i++) out[i] = v[i];
  return MIRT_OK;
}

int mirt_interp_plan_set_gather(mirt_interp_plan *P, int32_t tma) {
  if (!P) return fail(MIRT_ERR_ARG, "plan is NULL");
  P = launch_plan(P);
  if (tma < 0 || tma > 2) return fail(MIRT_ERR_ARG, "gather mode must be 0, 1 or 2");
  if (tma && !P->gbk.item)
    return fail(MIRT_ERR_ARG, "TMA gather needs J = 6 and, in 2D, an even C >= 32 and K >= 13, "
                              "in 3D an even C >= 8 and K >= 9");
  if (tma == 2 && P->a.g.D == 3)
    return fail(MIRT_ERR_ARG, "gather mode 2 (16-coil tiles) is 2D only");
  P->gtma = tma;
  return MIRT_OK;
}

int mirt_interp_plan_set_fault_test(mirt_interp_plan *P, int32_t on) {
  if (!P) return fail(MIRT_ERR_ARG, "plan is NULL");
  P = launch_plan(P);
  if (on && !P->gtma) return fail(MIRT_ERR_ARG, "the plan's gather does not use TMA stages");
  P->gfault_test = on ? 1 : 0;
  return MIRT_OK;
}

int mirt_interp_plan_fault(mirt_interp_plan *P, int32_t *fault) {
  if (!P || !fault) return fail(MIRT_ERR_ARG, "NULL argument");
  P = launch_plan(P);
  *fault = 0;
  if (P->gfault.p) {
    CK(cudaDeviceSynchronize());
    int f = 0;
    CK(cudaMemcpy(&f, P->gfault.p, sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemset(P->gfault.p, 0, sizeof(int)));
    *fault = f;
  }
  return MIRT_OK;
}

int mirt_interp_plan_set_sweep(mirt_interp_plan *P, int32_t segments, int32_t rows) try {
  if (!P) return fail(MIRT_ERR_ARG, "plan is NULL");
  P = launch_plan(P);
  if (P->a.g.D == 3) {
    if (segments && !sweep3_ok(P->a, P->t, P->ls.cw))
      return fail(MIRT_ERR_ARG, "3D line sweep needs J = 6, K >= 6 per dimension and coil "
                                "chunks of 8, 16 or 32");
    if (segments < 0 || segments > P->a.g.K[0])
      return fail(MIRT_ERR_ARG, "3D line-sweep segments must be in 1..K1 (0: off)");
    if (segments) {
      int rc = sweep_buffer(P);
      if (rc) return rc;
      return set_line_sweep3(P, segments, as_stream(nullptr));
    }
    P->t.sweep = 0;
    return MIRT_OK;
  }
  if (segments && !sweep_ok(P->a, P->t))
    return fail(MIRT_ERR_ARG, "row-sweep spread needs 2D, J = 6 and K >= 6 per dimension");
  if (segments < -1 || (segments > 0 && segments > P->a.g.K[0]))
    return fail(MIRT_ERR_ARG, "row-sweep segments must be in 1..K1 (0: off, -1: balanced)");
  if (segments && rows != 1 && rows != 2 && rows != 4)
    return fail(MIRT_ERR_ARG, "row-sweep rows per band must be 1, 2 or 4");
  if (segments) {
    int rc = sweep_buffer(P);
    if (rc) return rc;
  }
  if (segments < 0) {
    int rc = build_sweep_teams(P, rows, 65536, as_stream(nullptr));
    if (rc) return rc;
  } else if (segments > 0) {
    int rc = set_uniform_sweep(P, segments, rows, as_stream(nullptr));
    if (rc) return rc;
  }
  P->t.sweep = segments;
  if (segments) P->t.sweep_rows = rows;
  if (segments) {
    P->t.own = 0;
    P->ls.atomic = 0;
  }
  return MIRT_OK;
} catch (const std::bad_alloc &) {
  return fail(MIRT_ERR_ALLOC, "out of host memory");
}

int mirt_interp_plan_set_dense(mirt_interp_plan *P, int32_t on) {
  if (!P) return fail(MIRT_ERR_ARG, "plan is NULL");
  P = launch_plan(P);
  if (on && !P->t.dense_of) return fail(MIRT_ERR_ARG, "the plan has no dense bins");
  P->t.dense_on = on ? 1 : 0;
  return MIRT_OK;
}

int mirt_interp_plan_set_staged(mirt_interp_plan *P, int32_t mode) {
  if (!P) return fail(MIRT_ERR_ARG, "plan is NULL");
  P = launch_plan(P);
  if (mode < 0 || mode > 2) return fail(MIRT_ERR_ARG, "staged mode must be 0, 1 or 2");
  if (mode && (P->ls.cw != 32 || !P->t.wsw))
    return fail(MIRT_ERR_ARG, "the staged row sweep needs 32-coil lanes (C >= 32)");
  P->t.sweep_staged = mode;
  return MIRT_OK;
}

int mirt_interp_plan_set_ownership(mirt_interp_plan *P, int32_t own, void *stream) try {
  if (!P) return fail(MIRT_ERR_ARG, "plan is NULL");
  P = launch_plan(P);
  if (own && !own_ok(P->a, P->t))
    return fail(MIRT_ERR_ARG, "ownership spread needs 2D, J = 6, tiles of >= 5 points and an "
                              "even number of tiles (last one >= 5 points) per dimension");
  P->t.own = own ? 1 : 0;
  if (own) {
    P->ls.atomic = 0;
    P->t.sweep = 0;
  }
  int T[MIRT_DMAX] = {P->t.T[0], P->t.T[1], P->t.T[2]};
  int rc = set_spread_tiles(P, T, as_stream(stream));
  if (rc) return rc;
  CK(cudaStreamSynchronize(as_stream(stream)));
  return MIRT_OK;
} catch (const std::bad_alloc &) {
  return fail(MIRT_ERR_ALLOC, "out of host memory");
}

int mirt_interp_plan_set_deterministic(mirt_interp_plan *P, int32_t deterministic) {
  if (!P) return fail(MIRT_ERR_ARG, "plan is NULL");
  P = launch_plan(P);
  P->deterministic = deterministic ? 1 : 0;
  if (deterministic) {
    P->ls.atomic = 0;
    if (P->ls.threads > 32 * P->t.T[P->a.g.D - 1]) P->ls.threads = 32;
  } else {
    P->ls.atomic = 1;
    P->ls.threads = 256;
  }
  return MIRT_OK;
}

int mirt_interp_plan_set_spread(mirt_interp_plan *P, const int32_t *T, int32_t threads,
                                int32_t padc, void *stream) try {
  if (!P || !T) return fail(MIRT_ERR_ARG, "NULL argument");
  P = launch_plan(P);
  const int D = P->a.g.D;
  if (threads < 32 || threads > 1024 || threads % 32)
    return fail(MIRT_ERR_ARG, "spread threads must be a multiple of 32 in [32, 1024]");
  if (padc != 0 && padc != padc_max(P->a))
    return fail(MIRT_ERR_ARG, "padc must be 0 or J1 - 1 (J = 6 kernels in 2D/3D)");
  int Tn[MIRT_DMAX] = {1, 1, 1};
  size_t npts = 1;
  for (int d = 0; d < D; d++) {
    const int B = P->t.B[d];
    const int kr = (P->a.g.K[d] + B - 1) / B * B;
    if (T[d] < B || T[d] % B || T[d] > kr)
      return fail(MIRT_ERR_ARG, "tile extents must be multiples of the sort bin, at most the "
                                "grid extent rounded up to a bin");
    Tn[d] = T[d];
    npts *= (size_t)(d == 0 ? T[0] + 2 * padc : T[d]);
  }
  if (npts * P->ls.cw * 8 > 200 * 1024) return fail(MIRT_ERR_ARG, "tile exceeds shared memory");
  cudaStream_t st = as_stream(stream);
  P->t.padc = padc;
  P->ls.threads = threads;
  P->t.sweep = 0;
  int rc = set_spread_tiles(P, Tn, st);
  if (rc) return rc;
  CK(cudaStreamSynchronize(st));
  return MIRT_OK;
} catch (const std::bad_alloc &) {
  return fail(MIRT_ERR_ALLOC, "out of host memory");
}

int mirt_interp_plan_destroy(mirt_interp_plan *P) {
  if (P) {
    cudaDeviceSynchronize();
    delete P;
  }
  return MIRT_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// mex gateway drop-ins
// ---------------------------------------------------------------------------
namespace {

struct Tab {
  const double *re, *im;
  int64_t rows, cols;
};

struct MexCall {
  const char *gateway;  // the gateway's mexFail() text
  int D;
  bool adj;
  int K[4], J[4], L[4];  // up to the 4D gateways
  Tab h[4];
  int order;
  long long M;
  int N;
  const double *tm;
  const double *in_re, *in_im;
  double *out_re, *out_im;
};

int mex_fail(const MexCall &c, const std::string &why) {
  return fail(MIRT_ERR_ARG, std::string(c.gateway) + ": " + why);
}

std::mutex g_mex_mu;
cudaStream_t g_mex_stream = nullptr;

// Table kind and order checks shared by all gateways, in the gateways' order
// (e.g. nufft/table/interp2_table_mex.c:78-126).
int mex_check_tables(MexCall &c, const int32_t *flips, int64_t flips_numel) {
  bool all_cx = true, all_re = true;
  for (int d = 0; d < c.D; d++) {
    if (c.h[d].im) all_re = false;
    else all_cx = false;
  }
  if (all_cx) {
    if (c.order) return mex_fail(c, "only 0th order implemented for complex");
  } else if (all_re) {
    if (c.order != 0 && c.order != 1) return mex_fail(c, "bad order");
    if (flips)
      for (int64_t i = 0; i < flips_numel; i++)
        if (flips[i]) return mex_fail(c, "flip not compiled");
  } else {
    return mex_fail(c, "h must be real or complex double (preferably real)");
  }
  for (int d = 0; d < c.D; d++) {
    if (c.J[d] < 1 || c.J[d] > MIRT_JMAX)
      return mex_fail(c, "J outside 1..16 is not supported by the GPU kernels");
    if (c.L[d] < 1) return mex_fail(c, "L must be positive");
    if (c.K[d] < 1) return mex_fail(c, "K must be positive");
    // the first three dimensions run in the GPU kernels, which wrap a tap once
    if (d < 3 && c.J[d] > c.K[d])
      return mex_fail(c, "J larger than K is not supported by the GPU kernels");
  }
  return MIRT_OK;
}

int mex_run(MexCall &c) {
  // No samples or no columns: the reference's adjoint returns the zeroed
  // grid and its forward an empty fm (interp2_table1_adj.c:57-58 clears ck
  // before the sample loop), with no device work here either.
  if (c.M == 0 || c.N == 0) {
    if (c.adj && c.N > 0) {
      long long nk = 1;
      for (int d = 0; d < c.D; d++) nk *= c.K[d];
      std::fill(c.out_re, c.out_re + nk * c.N, 0.0);
      std::fill(c.out_im, c.out_im + nk * c.N, 0.0);
    }
    return MIRT_OK;
  }
  int rc = device_ok();
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(g_mex_mu);
  if (!g_mex_stream) CK(cudaStreamCreateWithFlags(&g_mex_stream, cudaStreamNonBlocking));
  cudaStream_t st = g_mex_stream;
  long long nk = 1;
  for (int d = 0; d < c.D; d++) nk *= c.K[d];
  const long long M = c.M;
  const int N = c.N;
  {
    long long g = (long long)N;
    for (int d = 0; d < c.D; d++) g *= c.K[d];
    if (g >= (1ll << 31)) return mex_fail(c, "grid times columns too large");
    if (M >= (1ll << 31)) return mex_fail(c, "too many samples");
  }
  const bool cplx = c.h[0].im != nullptr;
  const double *hr[4] = {nullptr, nullptr, nullptr, nullptr};
  const double *hi[4] = {nullptr, nullptr, nullptr, nullptr};
  for (int d = 0; d < c.D; d++) {
    hr[d] = c.h[d].re;
    hi[d] = c.h[d].im;
  }
  mirt_interp_plan P;
  // 4D: the 4D plan over its 3D plan of hyperplanes (interp4.cu)
  std::unique_ptr<mirt_interp_plan> P4;
  if (c.D == 4) {
    mirt_interp_plan *p4 = nullptr;
    rc = mirt_interp_plan_create(&p4, 4, c.K, c.J, c.L, hr, cplx ? hi : nullptr, c.order, c.tm,
                                 M, nullptr, 1, N, nullptr, nullptr, st);
    if (rc) return rc;
    P4.reset(p4);
  } else {
    rc = plan_geometry(&P, c.D, c.K, c.J, c.L, hr, cplx ? hi : nullptr, c.order, N, st);
    if (rc) return rc;
    CK(P.tm.alloc(std::max<long long>(M, 1) * c.D * sizeof(double)));
    if (M) CK(cudaMemcpyAsync(P.tm.p, c.tm, M * c.D * sizeof(double), cudaMemcpyHostToDevice, st));
    const long long moff[2] = {0, M};
    rc = plan_finish(&P, M, moff, 1, st);
    if (rc) return rc;
  }

  const long long nin = c.adj ? M : nk;
  const long long nout = c.adj ? nk : M;
  DMem in_split, in_il, out_il, out_split;
  CK(in_split.alloc(std::max<long long>(nin * N, 1) * 2 * sizeof(double)));
  CK(in_il.alloc(std::max<long long>(nin * N, 1) * sizeof(float2)));
  CK(out_il.alloc(std::max<long long>(nout * N, 1) * sizeof(float2)));
  CK(out_split.alloc(std::max<long long>(nout * N, 1) * 2 * sizeof(double)));
  double *ir = in_split.as<double>(), *ii = ir + nin * N;
  double *orr = out_split.as<double>(), *oi = orr + nout * N;
  if (nin > 0 && N > 0) {
    CK(cudaMemcpyAsync(ir, c.in_re, nin * N * sizeof(double), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ii, c.in_im, nin * N * sizeof(double), cudaMemcpyHostToDevice, st));
  }
  CK(launch_split_to_il(ir, ii, nin, N, in_il.as<float2>(), st));
  if (P4) {
    rc = c.adj ? mirt_interp_plan_adjoint(P4.get(), in_il.p, out_il.p, st)
               : mirt_interp_plan_forward(P4.get(), in_il.p, out_il.p, st);
    if (rc) return rc;
  } else if (c.adj)
    CK(launch_spread(P.a, P.t, P.ls, P.bin_start.as<int>(), in_il.as<float2>(),
                     out_il.as<float2>(), st));
  else
    CK(launch_gather(P.ag, P.lg, in_il.as<float2>(), out_il.as<float2>(), st));
  CK(launch_il_to_split(out_il.as<float2>(), nout, N, orr, oi, st));
  if (nout > 0 && N > 0) {
    CK(cudaMemcpyAsync(c.out_re, orr, nout * N * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(c.out_im, oi, nout * N * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  CK(cudaStreamSynchronize(st));
  return MIRT_OK;
}

// table size check of the gateways: "hD size problem" (2D/3D) / "h size problem" (1D)
bool tab_len_ok(const Tab &h, int J, int L) { return h.rows == (int64_t)J * L + 1 && h.cols == 1; }

}  // namespace

extern "C" {

int mirt_interp1_table_mex(const double *ck_re, const double *ck_im, int64_t ck_rows,
                           int64_t ck_cols, const double *h_re, const double *h_im,
                           int64_t h_rows, int64_t h_cols, const int32_t *J, int64_t J_numel,
                           const int32_t *L, int64_t L_numel, const double *tm, int64_t tm_rows,
                           int64_t tm_cols, const int32_t *order, int64_t order_numel,
                           const int32_t *flips, int64_t flips_numel, double *fm_re,
                           double *fm_im) {
  MexCall c{};
  c.gateway = "interp1_table_mex() failed";
  c.D = 1;
  c.adj = false;
  if (!ck_re || !ck_im) return mex_fail(c, "mxIsComplexDouble");
  if (!tm) return mex_fail(c, "mxIsRealDouble");
  if (!J || J_numel != 1) return mex_fail(c, "J must be scalar int32");
  if (!L || L_numel != 1) return mex_fail(c, "L must be scalar int32");
  if (order && order_numel != 1) return mex_fail(c, "order must be scalar int32 (0 | 1)");
  if (flips && flips_numel != 1) return mex_fail(c, "flips must be scalar int32 (0 | 1)");
  c.J[0] = J[0];
  c.L[0] = L[0];
  c.h[0] = Tab{h_re, h_im, h_rows, h_cols};
  if (!h_re || !tab_len_ok(c.h[0], c.J[0], c.L[0])) return mex_fail(c, "h size problem");
  if (tm_cols != 1) return mex_fail(c, "t_m must be col vector.");
  c.K[0] = (int)ck_rows;
  c.N = (int)ck_cols;
  c.M = tm_rows;
  c.order = order ? order[0] : 0;
  int rc = mex_check_tables(c, flips, flips_numel);
  if (rc) return rc;
  c.tm = tm;
  c.in_re = ck_re;
  c.in_im = ck_im;
  c.out_re = fm_re;
  c.out_im = fm_im;
  return mex_run(c);
}

int mirt_interp2_table_mex(const double *ck_re, const double *ck_im, const int64_t *ck_dims,
                           int32_t ck_ndim, const double *h1_re, const double *h1_im,
                           int64_t h1_rows, int64_t h1_cols, const double *h2_re,
                           const double *h2_im, int64_t h2_rows, int64_t h2_cols,
                           const int32_t *J, int64_t J_numel, const int32_t *L, int64_t L_numel,
                           const double *tm, int64_t tm_rows, int64_t tm_cols,
                           const int32_t *order, int64_t order_numel, const int32_t *flips,
                           int64_t flips_numel, double *fm_re, double *fm_im) {
  MexCall c{};
  c.gateway = "interp2_table_mex failed";
  c.D = 2;
  c.adj = false;
  if (!ck_re || !ck_im) return mex_fail(c, "mxIsComplexDouble");
  if (!tm) return mex_fail(c, "mxIsRealDouble");
  if (!J || J_numel != 2) return mex_fail(c, "J must be [1,2]");
  if (!L || L_numel != 2) return mex_fail(c, "L must be [1,2]");
  if (order && order_numel != 1) return mex_fail(c, "order must be scalar int32 (0 | 1)");
  if (flips && flips_numel != 2) return mex_fail(c, "flips must be [1 2] int32 (0 | 1)");
  for (int d = 0; d < 2; d++) {
    c.J[d] = J[d];
    c.L[d] = L[d];
  }
  c.h[0] = Tab{h1_re, h1_im, h1_rows, h1_cols};
  c.h[1] = Tab{h2_re, h2_im, h2_rows, h2_cols};
  if (!h1_re || !tab_len_ok(c.h[0], c.J[0], c.L[0])) return mex_fail(c, "h1 size problem");
  if (!h2_re || !tab_len_ok(c.h[1], c.J[1], c.L[1])) return mex_fail(c, "h2 size problem");
  if (tm_cols != 2) return mex_fail(c, "tm must have 2 columns");
  c.K[0] = ck_ndim > 0 ? (int)ck_dims[0] : 1;
  c.K[1] = ck_ndim > 1 ? (int)ck_dims[1] : 1;
  c.N = ck_ndim > 2 ? (int)ck_dims[2] : 1;
  c.M = tm_rows;
  c.order = order ? order[0] : 0;
  int rc = mex_check_tables(c, flips, flips_numel);
  if (rc) return rc;
  c.tm = tm;
  c.in_re = ck_re;
  c.in_im = ck_im;
  c.out_re = fm_re;
  c.out_im = fm_im;
  return mex_run(c);
}

int mirt_interp3_table_mex(const double *ck_re, const double *ck_im, const int64_t *ck_dims,
                           int32_t ck_ndim, const double *h1_re, const double *h1_im,
                           int64_t h1_rows, int64_t h1_cols, const double *h2_re,
                           const double *h2_im, int64_t h2_rows, int64_t h2_cols,
                           const double *h3_re, const double *h3_im, int64_t h3_rows,
                           int64_t h3_cols, const int32_t *J, int64_t J_numel, const int32_t *L,
                           int64_t L_numel, const double *tm, int64_t tm_rows, int64_t tm_cols,
                           const int32_t *order, int64_t order_numel, const int32_t *flips,
                           int64_t flips_numel, double *fm_re, double *fm_im) {
  MexCall c{};
  c.gateway = "interp3_table_mex failed";
  c.D = 3;
  c.adj = false;
  if (!ck_re || !ck_im) return mex_fail(c, "mxIsComplexDouble");
  if (!tm) return mex_fail(c, "mxIsRealDouble");
  if (!J || J_numel != 3) return mex_fail(c, "J must be [1,3]");
  if (!L || L_numel != 3) return mex_fail(c, "L must be [1,3]");
  if (order && order_numel != 1) return mex_fail(c, "order must be scalar int32 (0 | 1)");
  if (flips && flips_numel != 3) return mex_fail(c, "flips must be [1 3] int32 (0 | 1)");
  for (int d = 0; d < 3; d++) {
    c.J[d] = J[d];
    c.L[d] = L[d];
  }
  c.h[0] = Tab{h1_re, h1_im, h1_rows, h1_cols};
  c.h[1] = Tab{h2_re, h2_im, h2_rows, h2_cols};
  c.h[2] = Tab{h3_re, h3_im, h3_rows, h3_cols};
  if (!h1_re || !tab_len_ok(c.h[0], c.J[0], c.L[0])) return mex_fail(c, "h1 size problem");
  if (!h2_re || !tab_len_ok(c.h[1], c.J[1], c.L[1])) return mex_fail(c, "h2 size problem");
  if (!h3_re || !tab_len_ok(c.h[2], c.J[2], c.L[2])) return mex_fail(c, "h3 size problem");
  if (tm_cols != 3) return mex_fail(c, "tm must have 3 columns");
  c.K[0] = ck_ndim > 0 ? (int)ck_dims[0] : 1;
  c.K[1] = ck_ndim > 1 ? (int)ck_dims[1] : 1;
  c.K[2] = ck_ndim > 2 ? (int)ck_dims[2] : 1;
  c.N = ck_ndim > 3 ? (int)ck_dims[3] : 1;
  c.M = tm_rows;
  c.order = order ? order[0] : 0;
  int rc = mex_check_tables(c, flips, flips_numel);
  if (rc) return rc;
  c.tm = tm;
  c.in_re = ck_re;
  c.in_im = ck_im;
  c.out_re = fm_re;
  c.out_im = fm_im;
  return mex_run(c);
}

int mirt_interp1_table_adj_mex(const double *fm_re, const double *fm_im, int64_t fm_rows,
                               int64_t fm_cols, const double *h_re, const double *h_im,
                               int64_t h_rows, int64_t h_cols, const int32_t *J, int64_t J_numel,
                               const int32_t *L, int64_t L_numel, const double *tm,
                               int64_t tm_rows, int64_t tm_cols, const int32_t *K,
                               int64_t K_numel, const int32_t *order, int64_t order_numel,
                               const int32_t *flips, int64_t flips_numel, double *ck_re,
                               double *ck_im) {
  MexCall c{};
  c.gateway = "interp1_table_adj_mex() failed";
  c.D = 1;
  c.adj = true;
  if (!fm_re || !fm_im) return mex_fail(c, "mxIsComplexDouble");
  if (!tm) return mex_fail(c, "mxIsRealDouble");
  if (!J || J_numel != 1) return mex_fail(c, "J must be scalar int32");
  if (!K || K_numel != 1) return mex_fail(c, "K must be scalar int32");
  if (!L || L_numel != 1) return mex_fail(c, "L must be scalar int32");
  if (order && order_numel != 1) return mex_fail(c, "order must be scalar int32 (0 | 1)");
  if (flips && flips_numel != 1) return mex_fail(c, "flips must be scalar int32 (0 | 1)");
  c.J[0] = J[0];
  c.L[0] = L[0];
  c.K[0] = K[0];
  c.h[0] = Tab{h_re, h_im, h_rows, h_cols};
  if (!h_re || h_rows != (int64_t)c.J[0] * c.L[0] + 1) return mex_fail(c, "h size problem");
  if (h_cols != 1) return mex_fail(c, "h must be col vector");
  if (fm_rows != tm_rows || tm_cols != 1) return mex_fail(c, "t_m must be Mx1 col vector");
  c.M = fm_rows;
  c.N = (int)fm_cols;
  c.order = order ? order[0] : 0;
  int rc = mex_check_tables(c, flips, flips_numel);
  if (rc) return rc;
  c.tm = tm;
  c.in_re = fm_re;
  c.in_im = fm_im;
  c.out_re = ck_re;
  c.out_im = ck_im;
  return mex_run(c);
}

int mirt_interp2_table_adj_mex(const double *fm_re, const double *fm_im, int64_t fm_rows,
                               int64_t fm_cols, const double *h1_re, const double *h1_im,
                               int64_t h1_rows, int64_t h1_cols, const double *h2_re,
                               const double *h2_im, int64_t h2_rows, int64_t h2_cols,
                               const int32_t *J, int64_t J_numel, const int32_t *L,
                               int64_t L_numel, const double *tm, int64_t tm_rows,
                               int64_t tm_cols, const int32_t *K, int64_t K_numel,
                               const int32_t *order, int64_t order_numel, const int32_t *flips,
                               int64_t flips_numel, double *ck_re, double *ck_im) {
  MexCall c{};
  c.gateway = "interp2_table_adj_mex() failed";
  c.D = 2;
  c.adj = true;
  if (!fm_re || !fm_im) return mex_fail(c, "mxIsComplexDouble");
  if (!tm) return mex_fail(c, "mxIsRealDouble");
  if (!J || J_numel != 2) return mex_fail(c, "J must be int32 [1,2]");
  if (!L || L_numel != 2) return mex_fail(c, "L must be int32 [1,2]");
  if (!K || K_numel != 2) return mex_fail(c, "K must be int32 [1,2]");
  if (order && order_numel != 1) return mex_fail(c, "order must be scalar int32 (0 | 1)");
  if (flips && flips_numel != 2) return mex_fail(c, "flips must be [1 2] int32 (0 | 1)");
  for (int d = 0; d < 2; d++) {
    c.J[d] = J[d];
    c.L[d] = L[d];
    c.K[d] = K[d];
  }
  c.h[0] = Tab{h1_re, h1_im, h1_rows, h1_cols};
  c.h[1] = Tab{h2_re, h2_im, h2_rows, h2_cols};
  if (!h1_re || !tab_len_ok(c.h[0], c.J[0], c.L[0])) return mex_fail(c, "h1 size problem");
  if (!h2_re || !tab_len_ok(c.h[1], c.J[1], c.L[1])) return mex_fail(c, "h2 size problem");
  if (fm_rows != tm_rows || tm_cols != 2) return mex_fail(c, "t_m must be Mx2 matrix");
  c.M = fm_rows;
  c.N = (int)fm_cols;
  c.order = order ? order[0] : 0;
  int rc = mex_check_tables(c, flips, flips_numel);
  if (rc) return rc;
  c.tm = tm;
  c.in_re = fm_re;
  c.in_im = fm_im;
  c.out_re = ck_re;
  c.out_im = ck_im;
  return mex_run(c);
}

int mirt_interp3_table_adj_mex(const double *fm_re, const double *fm_im, int64_t fm_rows,
                               int64_t fm_cols, const double *h1_re, const double *h1_im,
                               int64_t h1_rows, int64_t h1_cols, const double *h2_re,
                               const double *h2_im, int64_t h2_rows, int64_t h2_cols,
                               const double *h3_re, const double *h3_im, int64_t h3_rows,
                               int64_t h3_cols, const int32_t *J, int64_t J_numel,
                               const int32_t *L, int64_t L_numel, const double *tm,
                               int64_t tm_rows, int64_t tm_cols, const int32_t *K,
                               int64_t K_numel, const int32_t *order, int64_t order_numel,
                               const int32_t *flips, int64_t flips_numel, double *ck_re,
                               double *ck_im) {
  MexCall c{};
  c.gateway = "interp3_table_adj_mex() failed";
  c.D = 3;
  c.adj = true;
  if (!fm_re || !fm_im) return mex_fail(c, "mxIsComplexDouble");
  if (!tm) return mex_fail(c, "mxIsRealDouble");
  if (!J || J_numel != 3) return mex_fail(c, "J must be int32 [1,3]");
  if (!L || L_numel != 3) return mex_fail(c, "L must be int32 [1,3]");
  if (!K || K_numel != 3) return mex_fail(c, "K must be int32 [1,3]");
  if (order && order_numel != 1) return mex_fail(c, "order must be scalar int32 (0 | 1)");
  if (flips && flips_numel != 3) return mex_fail(c, "flips must be [1 3] int32 (0 | 1)");
  for (int d = 0; d < 3; d++) {
    c.J[d] = J[d];
    c.L[d] = L[d];
    c.K[d] = K[d];
  }
  c.h[0] = Tab{h1_re, h1_im, h1_rows, h1_cols};
  c.h[1] = Tab{h2_re, h2_im, h2_rows, h2_cols};
  c.h[2] = Tab{h3_re, h3_im, h3_rows, h3_cols};
  if (!h1_re || !tab_len_ok(c.h[0], c.J[0], c.L[0])) return mex_fail(c, "h1 size problem");
  if (!h2_re || !tab_len_ok(c.h[1], c.J[1], c.L[1])) return mex_fail(c, "h2 size problem");
  if (!h3_re || !tab_len_ok(c.h[2], c.J[2], c.L[2])) return mex_fail(c, "h3 size problem");
  if (fm_rows != tm_rows || tm_cols != 3) return mex_fail(c, "t_m must be Mx3 matrix");
  c.M = fm_rows;
  c.N = (int)fm_cols;
  c.order = order ? order[0] : 0;
  int rc = mex_check_tables(c, flips, flips_numel);
  if (rc) return rc;
  c.tm = tm;
  c.in_re = fm_re;
  c.in_im = fm_im;
  c.out_re = ck_re;
  c.out_im = ck_im;
  return mex_run(c);
}

/* The 4D gateways: nufft/table/interp4_table_mex.c:12-163 and
 * interp4_table_adj_mex.c:12-166, their checks in order and their texts
 * (the forward gateway's own failure text names interp3_table_mex,
 * interp4_table_mex.c:182). */
int mirt_interp4_table_mex(const double *ck_re, const double *ck_im, const int64_t *ck_dims,
                           int32_t ck_ndim, const double *h1_re, const double *h1_im,
                           int64_t h1_rows, int64_t h1_cols, const double *h2_re,
                           const double *h2_im, int64_t h2_rows, int64_t h2_cols,
                           const double *h3_re, const double *h3_im, int64_t h3_rows,
                           int64_t h3_cols, const double *h4_re, const double *h4_im,
                           int64_t h4_rows, int64_t h4_cols, const int32_t *J, int64_t J_numel,
                           const int32_t *L, int64_t L_numel, const double *tm, int64_t tm_rows,
                           int64_t tm_cols, const int32_t *order, int64_t order_numel,
                           const int32_t *flips, int64_t flips_numel, double *fm_re,
                           double *fm_im) {
  MexCall c{};
  c.gateway = "interp3_table_mex failed";
  c.D = 4;
  c.adj = false;
  if (!ck_re || !ck_im) return mex_fail(c, "mxIsComplexDouble");
  if (!tm) return mex_fail(c, "mxIsRealDouble");
  if (!J || J_numel != 4) return mex_fail(c, "J must be [1,4]");
  if (!L || L_numel != 4) return mex_fail(c, "L must be [1,4]");
  if (order && order_numel != 1) return mex_fail(c, "order must be scalar int32 (0 | 1)");
  if (flips && flips_numel != 4) return mex_fail(c, "flips must be [1 4] int32 (0 | 1)");
  for (int d = 0; d < 4; d++) {
    c.J[d] = J[d];
    c.L[d] = L[d];
  }
  c.h[0] = Tab{h1_re, h1_im, h1_rows, h1_cols};
  c.h[1] = Tab{h2_re, h2_im, h2_rows, h2_cols};
  c.h[2] = Tab{h3_re, h3_im, h3_rows, h3_cols};
  c.h[3] = Tab{h4_re, h4_im, h4_rows, h4_cols};
  if (!h1_re || !tab_len_ok(c.h[0], c.J[0], c.L[0])) return mex_fail(c, "h1 size problem");
  if (!h2_re || !tab_len_ok(c.h[1], c.J[1], c.L[1])) return mex_fail(c, "h2 size problem");
  if (!h3_re || !tab_len_ok(c.h[2], c.J[2], c.L[2])) return mex_fail(c, "h3 size problem");
  if (!h4_re || !tab_len_ok(c.h[3], c.J[3], c.L[3])) return mex_fail(c, "h4 size problem");
  if (tm_cols != 4) return mex_fail(c, "tm must have 4 columns");
  for (int d = 0; d < 4; d++) c.K[d] = ck_ndim > d ? (int)ck_dims[d] : 1;
  // the reference gateway stops at N > 1 ("N=1 done only"); this one runs every column
  c.N = ck_ndim > 4 ? (int)ck_dims[4] : 1;
  c.M = tm_rows;
  c.order = order ? order[0] : 0;
  int rc = mex_check_tables(c, flips, flips_numel);
  if (rc) return rc;
  c.tm = tm;
  c.in_re = ck_re;
  c.in_im = ck_im;
  c.out_re = fm_re;
  c.out_im = fm_im;
  return mex_run(c);
}

int mirt_interp4_table_adj_mex(const double *fm_re, const double *fm_im, int64_t fm_rows,
                               int64_t fm_cols, const double *h1_re, const double *h1_im,
                               int64_t h1_rows, int64_t h1_cols, const double *h2_re,
                               const double *h2_im, int64_t h2_rows, int64_t h2_cols,
                               const double *h3_re, const double *h3_im, int64_t h3_rows,
                               int64_t h3_cols, const double *h4_re, const double *h4_im,
                               int64_t h4_rows, int64_t h4_cols, const int32_t *J,
                               int64_t J_numel, const int32_t *L, int64_t L_numel,
                               const double *tm, int64_t tm_rows, int64_t tm_cols,
                               const int32_t *K, int64_t K_numel, const int32_t *order,
                               int64_t order_numel, const int32_t *flips, int64_t flips_numel,
                               double *ck_re, double *ck_im) {
  MexCall c{};
  c.gateway = "interp4_table_adj_mex() failed";
  c.D = 4;
  c.adj = true;
  if (!fm_re || !fm_im) return mex_fail(c, "mxIsComplexDouble");
  if (!tm) return mex_fail(c, "mxIsRealDouble");
  if (!J || J_numel != 4) return mex_fail(c, "J must be int32 [1,4]");
  if (!L || L_numel != 4) return mex_fail(c, "L must be int32 [1,4]");
  if (!K || K_numel != 4) return mex_fail(c, "K must be int32 [1,4]");
  if (order && order_numel != 1) return mex_fail(c, "order must be scalar int32 (0 | 1)");
  if (flips && flips_numel != 4) return mex_fail(c, "flips must be [1 4] int32 (0 | 1)");
  for (int d = 0; d < 4; d++) {
    c.J[d] = J[d];
    c.L[d] = L[d];
    c.K[d] = K[d];
  }
  c.h[0] = Tab{h1_re, h1_im, h1_rows, h1_cols};
  c.h[1] = Tab{h2_re, h2_im, h2_rows, h2_cols};
  c.h[2] = Tab{h3_re, h3_im, h3_rows, h3_cols};
  c.h[3] = Tab{h4_re, h4_im, h4_rows, h4_cols};
  if (!h1_re || !tab_len_ok(c.h[0], c.J[0], c.L[0])) return mex_fail(c, "h1 size problem");
  if (!h2_re || !tab_len_ok(c.h[1], c.J[1], c.L[1])) return mex_fail(c, "h2 size problem");
  if (!h3_re || !tab_len_ok(c.h[2], c.J[2], c.L[2])) return mex_fail(c, "h3 size problem");
  if (!h4_re || !tab_len_ok(c.h[3], c.J[3], c.L[3])) return mex_fail(c, "h4 size problem");
  if (fm_rows != tm_rows || tm_cols != 4) return mex_fail(c, "t_m must be Mx4 matrix");
  c.M = fm_rows;
  c.N = (int)fm_cols;
  c.order = order ? order[0] : 0;
  int rc = mex_check_tables(c, flips, flips_numel);
  if (rc) return rc;
  c.tm = tm;
  c.in_re = fm_re;
  c.in_im = fm_im;
  c.out_re = ck_re;
  c.out_im = ck_im;
  return mex_run(c);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// NUFFT
// ---------------------------------------------------------------------------

namespace {

#define CF(call)                                                                   \
  do {                                                                             \
    cufftResult r_ = (call);                                                       \
    if (r_ != CUFFT_SUCCESS)                                                       \
      return fail(MIRT_ERR_FFT, std::string(#call) + " failed: " + std::to_string((int)r_)); \
  } while (0)

// one batched C2C execution over every slice and coil of the coil-major grid:
// forward out of place from the zero-padded input, inverse in place
int nufft_fft(mirt_nufft *p, int dir, cudaStream_t st) {
  CF(cufftSetStream(p->fft, st));
  cufftComplex *g = reinterpret_cast<cufftComplex *>(p->grid_cm.as<float2>());
  cufftComplex *src = dir == CUFFT_FORWARD ? reinterpret_cast<cufftComplex *>(p->pad.as<float2>()) : g;
  CF(cufftExecC2C(p->fft, src, g, dir));
  return MIRT_OK;
}

}  // namespace

extern "C" {

int mirt_minmax_kb_table(int32_t N, int32_t J, int32_t K, int32_t L, double *h_re, double *h_im) {
  if (N < 1 || J < 1 || K < 1 || L < 1) return fail(MIRT_ERR_ARG, "N, J, K, L must be positive");
  std::vector<std::complex<double>> h;
  if (!minmax_kb_table(N, J, K, L, h)) return fail(MIRT_ERR_ARG, "singular min-max system");
  for (size_t i = 0; i < h.size(); i++) {
    h_re[i] = h[i].real();
    h_im[i] = h[i].imag();
  }
  return MIRT_OK;
}

int mirt_minmax_kb_scale(int32_t N, int32_t J, int32_t K, double *sn_re, double *sn_im) {
  if (N < 1 || J < 1 || K < 1) return fail(MIRT_ERR_ARG, "N, J, K must be positive");
  std::vector<double> alpha;
  double beta;
  alpha_kb_fit(N, J, K, alpha, beta);
  std::vector<std::complex<double>> s = scale1(N, K, alpha, beta);
  for (int i = 0; i < N; i++) {
    sn_re[i] = s[i].real();
    sn_im[i] = s[i].imag();
  }
  return MIRT_OK;
}

}  // extern "C"

namespace {

// Geometry checks shared by the NUFFT constructors; fills the slice offsets.
int nufft_check(int D, const int32_t *Nd, const int32_t *Kd, const int32_t *Jd, const int32_t *Ld,
                int order, bool cplx, int64_t Mtot, const int64_t *slice_moff, int nslice,
                int ncol, std::vector<long long> &moff) {
  int rc = device_ok();
  if (rc) return rc;
  if (nslice < 1) return fail(MIRT_ERR_ARG, "nslice must be >= 1");
  rc = validate_geometry(D, Kd, Jd, Ld, order, cplx, Mtot, ncol);
  if (rc) return rc;
  for (int d = 0; d < D; d++)
    if (Nd[d] < 1 || Nd[d] > Kd[d]) return fail(MIRT_ERR_ARG, "need 1 <= N <= K per dimension");
  moff.assign(nslice + 1, 0);
  if (slice_moff) {
    for (int s = 0; s <= nslice; s++) moff[s] = slice_moff[s];
    if (moff[0] != 0 || moff[nslice] != Mtot)
      return fail(MIRT_ERR_ARG, "slice offsets must start at 0 and end at Mtot");
    for (int s = 0; s < nslice; s++)
      if (moff[s + 1] < moff[s]) return fail(MIRT_ERR_ARG, "slice offsets must not decrease");
  } else {
    if (nslice != 1) return fail(MIRT_ERR_ARG, "slice offsets required for nslice > 1");
    moff[0] = 0;
    moff[1] = Mtot;
  }
  return MIRT_OK;
}

// The plan once its tables and scaling factors are known: device tables,
// sn, tm = om / (2 pi / K) with the per-sample phase exp(i om . ns), the
// grid phase prod_d exp(i 2 pi k_d nmid_d / K_d) when nmid is given, the
// sorted interpolation plan, the grids and the batched FFT.
int nufft_finish(mirt_nufft *p, int D, const int32_t *Nd, const int32_t *Kd, const int32_t *Jd,
                 const int32_t *Ld, const double *const *hr, const double *const *hi, int order,
                 const std::vector<std::complex<double>> &sn, const double *ns_in,
                 const double *nmid, const double *om, int64_t Mtot,
                 const std::vector<long long> &moff, int nslice, int ncol, cudaStream_t st) {
  p->C = ncol;
  p->nslice = nslice;
  p->Mtot = Mtot;
  p->gg.D = D;
  p->gg.npix = 1;
  p->gg.ngrid = 1;
  for (int d = 0; d < 3; d++) {
    p->gg.N[d] = d < D ? Nd[d] : 1;
    p->gg.K[d] = d < D ? Kd[d] : 1;
    p->gg.npix *= p->gg.N[d];
    p->gg.ngrid *= p->gg.K[d];
  }
  p->ip = new mirt_interp_plan();
  mirt_interp_plan *P = p->ip;
  int rc = plan_geometry(P, D, Kd, Jd, Ld, hr, hi, order, ncol, st);
  if (rc) return rc;
  {
    std::vector<float2> snf(sn.size());
    for (size_t i = 0; i < sn.size(); i++)
      snf[i] = make_float2((float)sn[i].real(), (float)sn[i].imag());
    cudaError_t e = p->sn.alloc(snf.size() * sizeof(float2));
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(p->sn.p, snf.data(), snf.size() * sizeof(float2),
                          cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(MIRT_ERR_CUDA, cudaGetErrorString(e));
  }
  bool any_mid = false;
  for (int d = 0; d < D; d++)
    if (nmid && nmid[d] != 0) any_mid = true;
  if (any_mid) {
    // phase_before per dimension in FP64: angle 2 pi frac(k nmid / K)
    std::vector<float2> ph;
    for (int d = 0; d < D; d++)
      for (int k = 0; k < Kd[d]; k++) {
        const double f = std::fmod((double)k * nmid[d], (double)Kd[d]) / Kd[d];
        ph.push_back(make_float2((float)std::cos(2 * M_PI * f), (float)std::sin(2 * M_PI * f)));
      }
    cudaError_t e = p->phtab.alloc(ph.size() * sizeof(float2));
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(p->phtab.p, ph.data(), ph.size() * sizeof(float2),
                          cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(MIRT_ERR_CUDA, cudaGetErrorString(e));
    p->gp.D = D;
    long long off = 0;
    for (int d = 0; d < 3; d++) {
      p->gp.K[d] = d < D ? Kd[d] : 1;
      p->gp.tab[d] = d < D ? p->phtab.as<float2>() + off : nullptr;
      if (d < D) off += Kd[d];
    }
  }
  // om -> tm (FP64, om / (2 pi / K)) and the per-sample phase on the device
  bool any_shift = false;
  double gam[3] = {1, 1, 1}, ns[3] = {0, 0, 0};
  for (int d = 0; d < D; d++) {
    gam[d] = 2 * M_PI / Kd[d];
    ns[d] = ns_in ? ns_in[d] : 0.0;
    if (ns[d] != 0) any_shift = true;
  }
  {
    DMem om_d, par;
    cudaError_t e = om_d.alloc(std::max<long long>(Mtot, 1) * D * sizeof(double));
    if (e == cudaSuccess) e = par.alloc(6 * sizeof(double));
    if (e == cudaSuccess) e = P->tm.alloc(std::max<long long>(Mtot, 1) * D * sizeof(double));
    if (e == cudaSuccess && any_shift) e = P->phase.alloc(std::max<long long>(Mtot, 1) * sizeof(float2));
    double hp[6] = {gam[0], gam[1], gam[2], ns[0], ns[1], ns[2]};
    if (e == cudaSuccess && Mtot)
      e = cudaMemcpyAsync(om_d.p, om, Mtot * D * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(par.p, hp, sizeof hp, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = launch_om_to_tm(om_d.as<double>(), Mtot, D, par.as<double>(), par.as<double>() + 3,
                          any_shift ? 1 : 0, P->tm.as<double>(), P->phase.as<float2>(), st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(MIRT_ERR_CUDA, cudaGetErrorString(e));
    P->a.phase = any_shift ? P->phase.as<float2>() : nullptr;
  }
  rc = plan_finish(P, Mtot, moff.data(), nslice, st);
  if (rc) return rc;
  p->own_fft = ncol > 0;
  for (int d = 0; d < D; d++)
    if (!fft_len_ok(Kd[d])) p->own_fft = false;
  if (p->own_fft) {
    // fused FFT passes over the interpolation grid.  Stage-1 twiddles per
    // dimension and direction, [q][p1], in FP64: forward exp(-2 pi i p1 q / K)
    // and adjoint exp(+2 pi i p1 q / K); a grid phase of quarter turns i^(k m)
    // is folded in (forward: times i^(p1 m), adjoint: times i^(-q m))
    int qm[3] = {0, 0, 0};
    bool fold = any_mid;
    for (int d = 0; d < D && fold; d++) {
      const long long m4 = 4ll * (nmid ? nmid[d] : 0);
      if (m4 % Kd[d] != 0) fold = false;
      else qm[d] = (int)(((m4 / Kd[d]) % 4 + 4) % 4);
    }
    std::vector<float2> tw;
    long long offf[3] = {0, 0, 0}, offa[3] = {0, 0, 0};
    auto rot = [](float2 w, int e) {  // w * i^e, exact
      for (int r = 0; r < (e & 3); r++) w = make_float2(-w.y, w.x);
      return w;
    };
    for (int d = 0; d < D; d++) {
      int r1 = 0, r2 = 0;
      fft_radix(Kd[d], &r1, &r2);
      for (int dir = 0; dir < 2; dir++) {
        (dir ? offa : offf)[d] = (long long)tw.size();
        for (int q = 0; q < r2; q++)
          for (int p1 = 0; p1 < r1; p1++) {
            const long long j = ((long long)p1 * q) % Kd[d];
            const double a = 2 * M_PI * (double)j / Kd[d];
            float2 w = make_float2((float)std::cos(a), (float)(dir ? std::sin(a) : -std::sin(a)));
            if (fold) w = rot(w, dir ? -(q * qm[d]) : p1 * qm[d]);
            tw.push_back(w);
          }
      }
    }
    cudaError_t e = p->twtab.alloc(tw.size() * sizeof(float2));
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(p->twtab.p, tw.data(), tw.size() * sizeof(float2),
                          cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = p->grid.alloc((size_t)nslice * p->gg.ngrid * ncol * sizeof(float2));
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(MIRT_ERR_ALLOC, "NUFFT grid buffers");
    p->nf.g = p->gg;
    p->nf.C = ncol;
    for (int d = 0; d < 3; d++) {
      p->nf.twf[d] = d < D ? p->twtab.as<float2>() + offf[d] : nullptr;
      p->nf.twa[d] = d < D ? p->twtab.as<float2>() + offa[d] : nullptr;
    }
    p->nf.phase_folded = fold ? 1 : 0;
    p->nf.sn = p->sn.as<float2>();
    p->nf.gp = &p->gp;
    return MIRT_OK;
  }
  {
    cudaError_t e = p->grid.alloc((size_t)nslice * p->gg.ngrid * ncol * sizeof(float2));
    if (e == cudaSuccess) e = p->grid_cm.alloc((size_t)nslice * p->gg.ngrid * ncol * sizeof(float2));
    if (e == cudaSuccess) e = p->pad.alloc((size_t)nslice * p->gg.ngrid * ncol * sizeof(float2));
    if (e == cudaSuccess)
      e = cudaMemsetAsync(p->pad.p, 0, (size_t)nslice * p->gg.ngrid * ncol * sizeof(float2), st);
    if (e != cudaSuccess) return fail(MIRT_ERR_ALLOC, "NUFFT grid buffers");
  }
  // contiguous C2C transforms, one per (slice, coil) plane of the coil-major grid
  int n[3];
  for (int d = 0; d < D; d++) n[d] = Kd[D - 1 - d];
  if (ncol > 0) {
    const long long batch = (long long)nslice * ncol;
    if (batch >= (1ll << 31)) return fail(MIRT_ERR_ARG, "too many FFT planes");
    cufftResult r = cufftPlanMany(&p->fft, D, n, nullptr, 1, (int)p->gg.ngrid, nullptr, 1,
                                  (int)p->gg.ngrid, CUFFT_C2C, (int)batch);
    if (r != CUFFT_SUCCESS)
      return fail(MIRT_ERR_FFT, "cufftPlanMany failed: " + std::to_string((int)r));
    p->fft_ok = true;
  }
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(MIRT_ERR_CUDA, cudaGetErrorString(e));
  return MIRT_OK;
}

}  // namespace

extern "C" {

int mirt_nufft_create(mirt_nufft **out, int32_t D, const int32_t *Nd, const int32_t *Kd,
                      const int32_t *Jd, const int32_t *Ld, const double *n_shift,
                      const double *om, int64_t Mtot, const int64_t *slice_moff, int32_t nslice,
                      int32_t ncol, void *stream) try {
  if (!out) return fail(MIRT_ERR_ARG, "output pointer is NULL");
  *out = nullptr;
  std::vector<long long> moff;
  int rc = nufft_check(D, Nd, Kd, Jd, Ld, 0, true, Mtot, slice_moff, nslice, ncol, moff);
  if (rc) return rc;
  // tables (FP64 host), scaling factors as the outer product of conj(1D factors)
  std::vector<std::vector<double>> hre(D), him(D);
  std::vector<std::complex<double>> sn(1, 1.0);
  for (int d = 0; d < D; d++) {
    std::vector<std::complex<double>> h;
    if (!minmax_kb_table(Nd[d], Jd[d], Kd[d], Ld[d], h))
      return fail(MIRT_ERR_ARG, "singular min-max system");
    hre[d].resize(h.size());
    him[d].resize(h.size());
    for (size_t i = 0; i < h.size(); i++) {
      hre[d][i] = h[i].real();
      him[d][i] = h[i].imag();
    }
    std::vector<double> alpha;
    double beta;
    alpha_kb_fit(Nd[d], Jd[d], Kd[d], alpha, beta);
    std::vector<std::complex<double>> s1 = scale1(Nd[d], Kd[d], alpha, beta);
    std::vector<std::complex<double>> nsn(sn.size() * Nd[d]);
    for (int n = 0; n < Nd[d]; n++)
      for (size_t i = 0; i < sn.size(); i++) nsn[i + sn.size() * n] = sn[i] * std::conj(s1[n]);
    sn.swap(nsn);
  }
  const double *hr[MIRT_DMAX] = {nullptr, nullptr, nullptr};
  const double *hi[MIRT_DMAX] = {nullptr, nullptr, nullptr};
  for (int d = 0; d < D; d++) {
    hr[d] = hre[d].data();
    hi[d] = him[d].data();
  }
  auto *p = new mirt_nufft();
  rc = nufft_finish(p, D, Nd, Kd, Jd, Ld, hr, hi, 0, sn, n_shift, nullptr, om, Mtot, moff,
                    nslice, ncol, as_stream(stream));
  if (rc) {
    delete p;
    return rc;
  }
  *out = p;
  return MIRT_OK;
} catch (const std::bad_alloc &) {
  return fail(MIRT_ERR_ALLOC, "out of host memory");
}

int mirt_newfft_create(mirt_nufft **out, int32_t D, const int32_t *Nd, const int32_t *Kd,
                       const int32_t *Jd, const int32_t *Ld, const double *const *h_re,
                       const double *const *h_im, int32_t order, const double *sn_re,
                       const double *sn_im, const double *nmid, const double *n_shift,
                       const double *om, int64_t Mtot, const int64_t *slice_moff, int32_t nslice,
                       int32_t ncol, void *stream) try {
  if (!out) return fail(MIRT_ERR_ARG, "output pointer is NULL");
  *out = nullptr;
  if (!h_re || !sn_re) return fail(MIRT_ERR_ARG, "tables and scaling factors are required");
  const bool cplx = h_im != nullptr && h_im[0] != nullptr;
  std::vector<long long> moff;
  int rc = nufft_check(D, Nd, Kd, Jd, Ld, order, cplx, Mtot, slice_moff, nslice, ncol, moff);
  if (rc) return rc;
  for (int d = 0; d < D; d++) {
    if (!h_re[d]) return fail(MIRT_ERR_ARG, "table of a dimension is NULL");
    if (cplx && !h_im[d]) return fail(MIRT_ERR_ARG, "complex tables need every imaginary part");
  }
  long long npix = 1;
  for (int d = 0; d < D; d++) npix *= Nd[d];
  std::vector<std::complex<double>> sn(npix);
  for (long long i = 0; i < npix; i++) sn[i] = {sn_re[i], sn_im ? sn_im[i] : 0.0};
  // phase_after = exp(i om . (n_shift - nmid)) per sample
  double ns[3] = {0, 0, 0};
  for (int d = 0; d < D; d++) ns[d] = (n_shift ? n_shift[d] : 0.0) - (nmid ? nmid[d] : 0.0);
  auto *p = new mirt_nufft();
  rc = nufft_finish(p, D, Nd, Kd, Jd, Ld, h_re, cplx ? h_im : nullptr, order, sn, ns, nmid, om,
                    Mtot, moff, nslice, ncol, as_stream(stream));
  if (rc) {
    delete p;
    return rc;
  }
  *out = p;
  return MIRT_OK;
} catch (const std::bad_alloc &) {
  return fail(MIRT_ERR_ALLOC, "out of host memory");
}

int mirt_newfft_kb_table(int32_t J, int32_t L, double *h) {
  if (J < 1 || J > MIRT_JMAX || L < 1) return fail(MIRT_ERR_ARG, "J must be in 1..16, L positive");
  if (!h) return fail(MIRT_ERR_ARG, "output pointer is NULL");
  std::vector<double> t;
  kb_table(J, L, t);
  std::copy(t.begin(), t.end(), h);
  return MIRT_OK;
}

int mirt_newfft_kb_scale(int32_t N, int32_t J, int32_t K, double nmid, double *sn) {
  if (N < 1 || J < 1 || J > MIRT_JMAX || K < 1)
    return fail(MIRT_ERR_ARG, "N, K must be positive, J in 1..16");
  if (!sn) return fail(MIRT_ERR_ARG, "output pointer is NULL");
  std::vector<double> s = kb_scale(N, J, K, nmid);
  std::copy(s.begin(), s.end(), sn);
  return MIRT_OK;
}

int mirt_newfft_ktype_table(int32_t ktype, int32_t N, int32_t J, int32_t K, int32_t L, double *h) try {
  if (N < 1 || J < 1 || J > MIRT_JMAX || K < 1 || L < 1)
    return fail(MIRT_ERR_ARG, "N, K, L must be positive, J in 1..16");
  if (!h) return fail(MIRT_ERR_ARG, "output pointer is NULL");
  std::vector<double> t;
  switch (ktype) {
    case MIRT_KTYPE_KB_MINMAX: kb_table(J, L, t); break;
    case MIRT_KTYPE_KB_BEATTY: {
      const double a = kb_beatty_alpha(N, J, K);
      if (!(a > 0)) return fail(MIRT_ERR_ARG, "kb:beatty has no real shape for this J, K/N");
      kb_table_alpha(J, L, a, t);
      break;
    }
    case MIRT_KTYPE_DIRIC: diric_table(J, K, L, t); break;
    case MIRT_KTYPE_MINMAX_KB:
      if (N > K) return fail(MIRT_ERR_ARG, "minmax:kb needs N <= K");
      if (!minmax_kb_table_real(N, J, K, L, t))
        return fail(MIRT_ERR_ARG, "singular min-max matrix for this N, J, K");
      break;
    case MIRT_KTYPE_MINMAX_UNIF:
    case MIRT_KTYPE_MINMAX_TUNED: {
      if (N > K) return fail(MIRT_ERR_ARG, "minmax:* needs N <= K");
      std::vector<double> alpha{1.0};
      double beta = 0.0;
      if (ktype == MIRT_KTYPE_MINMAX_TUNED && !best_alpha(J, N, K, alpha, beta))
        return fail(MIRT_ERR_ARG, "minmax:tuned: unknown J,K/N");
      if (!minmax_table_real_ab(N, J, K, L, alpha, beta, t))
        return fail(MIRT_ERR_ARG, "singular min-max matrix for this N, J, K");
      break;
    }
    case MIRT_KTYPE_LINEAR: linear_table(J, L, t); break;
    default: return fail(MIRT_ERR_ARG, "unknown ktype");
  }
  std::copy(t.begin(), t.end(), h);
  return MIRT_OK;
} catch (const std::bad_alloc &) {
  return fail(MIRT_ERR_ALLOC, "out of host memory");
}

int mirt_newfft_ktype_scale(int32_t ktype, int32_t N, int32_t J, int32_t K, double nmid,
                            double *sn) try {
  if (N < 1 || J < 1 || J > MIRT_JMAX || K < 1)
    return fail(MIRT_ERR_ARG, "N, K must be positive, J in 1..16");
  if (!sn) return fail(MIRT_ERR_ARG, "output pointer is NULL");
  std::vector<double> s;
  switch (ktype) {
    case MIRT_KTYPE_KB_MINMAX: s = kb_scale(N, J, K, nmid); break;
    case MIRT_KTYPE_KB_BEATTY: {
      const double a = kb_beatty_alpha(N, J, K);
      if (!(a > 0)) return fail(MIRT_ERR_ARG, "kb:beatty has no real shape for this J, K/N");
      s = kb_scale_alpha(N, J, K, nmid, a);
      break;
    }
    case MIRT_KTYPE_DIRIC: s.assign(N, 1.0); break;
    case MIRT_KTYPE_MINMAX_KB: s = minmax_kb_scale_real(N, J, K, nmid); break;
    case MIRT_KTYPE_MINMAX_UNIF: s = minmax_scale_real_ab(N, K, {1.0}, 0.0, nmid); break;
    case MIRT_KTYPE_MINMAX_TUNED: {
      std::vector<double> alpha;
      double beta;
      if (!best_alpha(J, N, K, alpha, beta))
        return fail(MIRT_ERR_ARG, "minmax:tuned: unknown J,K/N");
      s = minmax_scale_real_ab(N, K, alpha, beta, nmid);
      break;
    }
    case MIRT_KTYPE_LINEAR: s = linear_scale(N, J, K, nmid); break;
    default: return fail(MIRT_ERR_ARG, "unknown ktype");
  }
  std::copy(s.begin(), s.end(), sn);
  return MIRT_OK;
} catch (const std::bad_alloc &) {
  return fail(MIRT_ERR_ALLOC, "out of host memory");
}

int mirt_newfft_table_complex(int32_t ktype, int32_t N, int32_t J, int32_t K, int32_t L,
                              double kb_alf, int32_t kb_m, const double *alpha, int32_t nalpha,
                              double beta, double *h_re, double *h_im) try {
  if (N < 1 || J < 1 || J > MIRT_JMAX || K < 1 || L < 1)
    return fail(MIRT_ERR_ARG, "N, K, L must be positive, J in 1..16");
  if (!h_re || !h_im) return fail(MIRT_ERR_ARG, "output pointer is NULL");
  std::vector<std::complex<double>> t;
  const bool minmax = ktype == MIRT_KTYPE_MINMAX_KB || ktype == MIRT_KTYPE_MINMAX_UNIF ||
                      ktype == MIRT_KTYPE_MINMAX_TUNED || ktype == MIRT_KTYPE_MINMAX_USER;
  if (minmax && N > K) return fail(MIRT_ERR_ARG, "minmax:* needs N <= K");
  switch (ktype) {
    case MIRT_KTYPE_KB_MINMAX: kb_table_complex(N, J, K, L, 2.34 * J, 0, t); break;
    case MIRT_KTYPE_KB_BEATTY: {
      const double a = kb_beatty_alpha(N, J, K);
      if (!(a > 0)) return fail(MIRT_ERR_ARG, "kb:beatty has no real shape for this J, K/N");
      kb_table_complex(N, J, K, L, a, 0, t);
      break;
    }
    case MIRT_KTYPE_KB_USER:
      if (!(kb_alf >= 0) || kb_m < 0 || kb_m > 32)
        return fail(MIRT_ERR_ARG, "kb:user needs alpha >= 0 and an integer kb_m in 0..32");
      kb_table_complex(N, J, K, L, kb_alf, kb_m, t);
      break;
    case MIRT_KTYPE_DIRIC: diric_table_complex(N, J, K, L, t); break;
    case MIRT_KTYPE_LINEAR: linear_table_complex(N, J, K, L, t); break;
    case MIRT_KTYPE_MINMAX_KB:
    case MIRT_KTYPE_MINMAX_UNIF:
    case MIRT_KTYPE_MINMAX_TUNED:
    case MIRT_KTYPE_MINMAX_USER: {
      std::vector<double> a{1.0};
      double b = 0.0;
      if (ktype == MIRT_KTYPE_MINMAX_KB) {
        alpha_kb_fit(N, J, K, a, b);  // Nmid = (N - 1) / 2 with phasing 'complex'
      } else if (ktype == MIRT_KTYPE_MINMAX_TUNED) {
        if (!best_alpha(J, N, K, a, b)) return fail(MIRT_ERR_ARG, "minmax:tuned: unknown J,K/N");
      } else if (ktype == MIRT_KTYPE_MINMAX_USER) {
        if (!alpha || nalpha < 1) return fail(MIRT_ERR_ARG, "user must provide alpha/beta");
        a.assign(alpha, alpha + nalpha);
        b = beta;
      }
      if (!minmax_table_complex_ab(N, J, K, L, a, b, t))
        return fail(MIRT_ERR_ARG, "singular min-max matrix for this N, J, K");
      break;
    }
    default: return fail(MIRT_ERR_ARG, "unknown ktype");
  }
  for (size_t i = 0; i < t.size(); i++) {
    h_re[i] = t[i].real();
    h_im[i] = t[i].imag();
  }
  return MIRT_OK;
} catch (const std::bad_alloc &) {
  return fail(MIRT_ERR_ALLOC, "out of host memory");
}

namespace {
// the argument checks of mirt_nufft_ktype_table / _scale
int nufft_ktype_args(int32_t ktype, int32_t N, int32_t J, int32_t K, double kb_alf, int32_t kb_m,
                     const double *alpha, int32_t nalpha, std::vector<double> &al) {
  if (N < 1 || J < 1 || J > MIRT_JMAX || K < 1)
    return fail(MIRT_ERR_ARG, "N, K must be positive, J in 1..16");
  switch (ktype) {
    case MIRT_KTYPE_KB_MINMAX:
    case MIRT_KTYPE_LINEAR:
      break;
    case MIRT_KTYPE_KB_USER:
      if (!(kb_alf >= 0) || kb_m < 0 || kb_m > 32)
        return fail(MIRT_ERR_ARG, "kaiser needs alpha >= 0 and an integer m in 0..32");
      break;
    case MIRT_KTYPE_MINMAX_KB:
    case MIRT_KTYPE_MINMAX_UNIF:
    case MIRT_KTYPE_MINMAX_TUNED:
    case MIRT_KTYPE_MINMAX_USER:
      if (N > K) return fail(MIRT_ERR_ARG, "N > K");
      if (ktype == MIRT_KTYPE_MINMAX_USER) {
        if (!alpha || nalpha < 1) return fail(MIRT_ERR_ARG, "user must provide alpha/beta");
        al.assign(alpha, alpha + nalpha);
      }
      break;
    default: return fail(MIRT_ERR_ARG, "not an interpolator of nufft_init");
  }
  return MIRT_OK;
}
}  // namespace

int mirt_nufft_ktype_table(int32_t ktype, int32_t N, int32_t J, int32_t K, int32_t L,
                           double kb_alf, int32_t kb_m, const double *alpha, int32_t nalpha,
                           double beta, double *h_re, double *h_im) try {
  if (!h_re || !h_im) return fail(MIRT_ERR_ARG, "output pointer is NULL");
  if (L < 1) return fail(MIRT_ERR_ARG, "L must be positive");
  std::vector<double> al;
  int rc = nufft_ktype_args(ktype, N, J, K, kb_alf, kb_m, alpha, nalpha, al);
  if (rc) return rc;
  std::vector<std::complex<double>> t;
  if (!nufft_table_ktype(ktype, N, J, K, L, kb_alf, kb_m, al, beta, t))
    return fail(MIRT_ERR_ARG, ktype == MIRT_KTYPE_MINMAX_TUNED ? "unknown J,K/N"
                                                                : "singular min-max matrix");
  for (size_t i = 0; i < t.size(); i++) {
    h_re[i] = t[i].real();
    h_im[i] = t[i].imag();
  }
  return MIRT_OK;
} catch (const std::bad_alloc &) {
  return fail(MIRT_ERR_ALLOC, "out of host memory");
}

int mirt_nufft_ktype_scale(int32_t ktype, int32_t N, int32_t J, int32_t K, double kb_alf,
                           int32_t kb_m, const double *alpha, int32_t nalpha, double beta,
                           double *sn_re, double *sn_im) try {
  if (!sn_re || !sn_im) return fail(MIRT_ERR_ARG, "output pointer is NULL");
  std::vector<double> al;
  int rc = nufft_ktype_args(ktype, N, J, K, kb_alf, kb_m, alpha, nalpha, al);
  if (rc) return rc;
  std::vector<std::complex<double>> s;
  if (!nufft_scale_ktype(ktype, N, J, K, kb_alf, kb_m, al, beta, s))
    return fail(MIRT_ERR_ARG, "unknown J,K/N");
  for (int n = 0; n < N; n++) {
    sn_re[n] = s[n].real();
    sn_im[n] = s[n].imag();
  }
  return MIRT_OK;
} catch (const std::bad_alloc &) {
  return fail(MIRT_ERR_ALLOC, "out of host memory");
}

int mirt_newfft_kb_user_table(int32_t J, int32_t L, double alpha, int32_t m, double *h) try {
  if (J < 1 || J > MIRT_JMAX || L < 1) return fail(MIRT_ERR_ARG, "L must be positive, J in 1..16");
  if (!h) return fail(MIRT_ERR_ARG, "output pointer is NULL");
  if (!(alpha >= 0) || m < 0 || m > 32)
    return fail(MIRT_ERR_ARG, "kb:user needs alpha >= 0 and an integer kb_m in 0..32");
  std::vector<double> t;
  kb_user_table(J, L, alpha, m, t);
  std::copy(t.begin(), t.end(), h);
  return MIRT_OK;
} catch (const std::bad_alloc &) {
  return fail(MIRT_ERR_ALLOC, "out of host memory");
}

int mirt_newfft_kb_user_scale(int32_t N, int32_t J, int32_t K, double nmid, double alpha,
                              int32_t m, double *sn) try {
  if (N < 1 || J < 1 || J > MIRT_JMAX || K < 1)
    return fail(MIRT_ERR_ARG, "N, K must be positive, J in 1..16");
  if (!sn) return fail(MIRT_ERR_ARG, "output pointer is NULL");
  if (!(alpha >= 0) || m < 0 || m > 32)
    return fail(MIRT_ERR_ARG, "kb:user needs alpha >= 0 and an integer kb_m in 0..32");
  const std::vector<double> s = kb_user_scale(N, J, K, nmid, alpha, m);
  std::copy(s.begin(), s.end(), sn);
  return MIRT_OK;
} catch (const std::bad_alloc &) {
  return fail(MIRT_ERR_ALLOC, "out of host memory");
}

int mirt_newfft_minmax_user_table(int32_t N, int32_t J, int32_t K, int32_t L,
                                  const double *alpha, int32_t nalpha, double beta, double *h) try {
  if (N < 1 || J < 1 || J > MIRT_JMAX || K < 1 || L < 1)
    return fail(MIRT_ERR_ARG, "N, K, L must be positive, J in 1..16");
  if (!h || !alpha || nalpha < 1) return fail(MIRT_ERR_ARG, "NULL argument or empty alpha");
  if (N > K) return fail(MIRT_ERR_ARG, "minmax:* needs N <= K");
  std::vector<double> t;
  if (!minmax_table_real_ab(N, J, K, L, std::vector<double>(alpha, alpha + nalpha), beta, t))
    return fail(MIRT_ERR_ARG, "singular min-max matrix for this N, J, K");
  std::copy(t.begin(), t.end(), h);
  return MIRT_OK;
} catch (const std::bad_alloc &) {
  return fail(MIRT_ERR_ALLOC, "out of host memory");
}

int mirt_newfft_minmax_user_scale(int32_t N, int32_t K, double nmid, const double *alpha,
                                  int32_t nalpha, double beta, double *sn) try {
  if (N < 1 || K < 1) return fail(MIRT_ERR_ARG, "N, K must be positive");
  if (!sn || !alpha || nalpha < 1) return fail(MIRT_ERR_ARG, "NULL argument or empty alpha");
  const std::vector<double> s =
      minmax_scale_real_ab(N, K, std::vector<double>(alpha, alpha + nalpha), beta, nmid);
  std::copy(s.begin(), s.end(), sn);
  return MIRT_OK;
} catch (const std::bad_alloc &) {
  return fail(MIRT_ERR_ALLOC, "out of host memory");
}

int mirt_nufft_forward(mirt_nufft *p, const void *x, void *X, void *stream) {
  if (!p) return fail(MIRT_ERR_ARG, "nufft is NULL");
  if (p->C == 0) return MIRT_OK;
  cudaStream_t st = as_stream(stream);
  if (p->own_fft) {
    CK(fft_nufft_forward(p->nf, static_cast<const float2 *>(x), p->grid.as<float2>(), 0,
                         p->nslice, st));
    CK(plan_gather(p->ip, p->grid.as<float2>(), static_cast<float2 *>(X), st));
    return MIRT_OK;
  }
  CK(launch_deapod_image_cm(static_cast<const float2 *>(x), p->sn.as<float2>(),
                            p->pad.as<float2>(), p->gg, p->C, p->nslice, st));
  int rc = nufft_fft(p, CUFFT_FORWARD, st);
  if (rc) return rc;
  CK(launch_transpose_cols(p->grid_cm.as<float2>(), p->grid.as<float2>(), p->gg.ngrid, p->C,
                           p->nslice, 1, st, &p->gp));
  CK(plan_gather(p->ip, p->grid.as<float2>(), static_cast<float2 *>(X), st));
  return MIRT_OK;
}

int mirt_nufft_adjoint(mirt_nufft *p, const void *X, void *x, void *stream) {
  if (!p) return fail(MIRT_ERR_ARG, "nufft is NULL");
  if (p->C == 0) return MIRT_OK;
  cudaStream_t st = as_stream(stream);
  mirt_interp_plan *P = p->ip;
  CK(launch_spread(P->a, P->t, P->ls, P->bin_start.as<int>(), static_cast<const float2 *>(X),
                   p->grid.as<float2>(), st));
  if (p->own_fft) {
    CK(fft_nufft_adjoint(p->nf, p->grid.as<float2>(), static_cast<float2 *>(x), 0, p->nslice, st));
    return MIRT_OK;
  }
  CK(launch_transpose_cols(p->grid.as<float2>(), p->grid_cm.as<float2>(), p->gg.ngrid, p->C,
                           p->nslice, 0, st, &p->gp));
  int rc = nufft_fft(p, CUFFT_INVERSE, st);
  if (rc) return rc;
  CK(launch_crop_deapod_cm(p->grid_cm.as<float2>(), p->sn.as<float2>(), static_cast<float2 *>(x),
                           p->gg, p->C, p->nslice, st));
  return MIRT_OK;
}

}  // extern "C"

namespace {

// Slices [s0, s1) of the forward NUFFT on the plan's full-size buffers (x, X:
// the whole batch's device image and samples), with `fft` made for s1 - s0
// slices.
int nufft_forward_range(mirt_nufft *p, int s0, int s1, const float2 *x, float2 *X,
                        cufftHandle fft, cudaStream_t st) {
  const int ns = s1 - s0, C = p->C;
  const long long gi = p->gg.ngrid * C, xi = p->gg.npix * C;
  if (p->own_fft) {
    CK(fft_nufft_forward(p->nf, x, p->grid.as<float2>(), s0, s1, st));
    CK(plan_gather(p->ip, p->grid.as<float2>(), X, st, s0, s1));
    return MIRT_OK;
  }
  float2 *pad = p->pad.as<float2>() + s0 * gi;
  float2 *gcm = p->grid_cm.as<float2>() + s0 * gi;
  CK(launch_deapod_image_cm(x + s0 * xi, p->sn.as<float2>(), pad, p->gg, C, ns, st));
  CF(cufftSetStream(fft, st));
  CF(cufftExecC2C(fft, reinterpret_cast<cufftComplex *>(pad), reinterpret_cast<cufftComplex *>(gcm),
                  CUFFT_FORWARD));
  CK(launch_transpose_cols(gcm, p->grid.as<float2>() + s0 * gi, p->gg.ngrid, C, ns, 1, st,
                           &p->gp));
  // the gather over the chunk's slices (slice-major in the gather order)
  CK(plan_gather(p->ip, p->grid.as<float2>(), X, st, s0, s1));
  return MIRT_OK;
}

// Slices [s0, s1) of the adjoint NUFFT (row-sweep spread) on the full-size
// buffers.
int nufft_adjoint_range(mirt_nufft *p, int s0, int s1, const float2 *X, float2 *x,
                        cufftHandle fft, cudaStream_t st) {
  const int ns = s1 - s0, C = p->C;
  const long long gi = p->gg.ngrid * C, xi = p->gg.npix * C;
  mirt_interp_plan *P = p->ip;
  Tiling t = P->t;
  if (t.sweep < 0) t.sweep = 2;  // a chunk: uniform halves of rows (same sums)
  t.team_order = nullptr;        // the chunk's teams in index order
  if (t.ndense > 0) {            // the chunk's dense bins and their sample chunks
    t.dense0 = P->dense_slice[s0];
    t.ndense = P->dense_slice[s1] - t.dense0;
    t.chunk0 = P->dense_part0_host[t.dense0];
    t.nchunks = P->dense_part0_host[t.dense0 + t.ndense] - t.chunk0;
  }
  t.slice0 = s0;
  t.nslice = ns;
  t.pos0 = P->moff_host[s0];
  t.npos = P->moff_host[s1] - t.pos0;
  CK(launch_spread(P->a, t, P->ls, P->bin_start.as<int>(), X, p->grid.as<float2>(), st));
  if (p->own_fft) {
    CK(fft_nufft_adjoint(p->nf, p->grid.as<float2>(), x, s0, s1, st));
    return MIRT_OK;
  }
  float2 *gcm = p->grid_cm.as<float2>() + s0 * gi;
  CK(launch_transpose_cols(p->grid.as<float2>() + s0 * gi, gcm, p->gg.ngrid, C, ns, 0, st,
                           &p->gp));
  CF(cufftSetStream(fft, st));
  CF(cufftExecC2C(fft, reinterpret_cast<cufftComplex *>(gcm), reinterpret_cast<cufftComplex *>(gcm),
                  CUFFT_INVERSE));
  CK(launch_crop_deapod_cm(gcm, p->sn.as<float2>(), x + s0 * xi, p->gg, C, ns, st));
  return MIRT_OK;
}

// Chunks of a host-buffer call: up to 8, of ch slices (the last may be smaller).
int host_chunks(const mirt_nufft *p, int *ch) {
  const int nch = std::min(p->nslice, 8);
  *ch = (p->nslice + nch - 1) / nch;
  return (p->nslice + *ch - 1) / *ch;
}

// Streams, events and the chunk-size FFT plans for the pipelined host calls.
int host_pipeline_setup(mirt_nufft *p) {
  if (!p->cs_in) CK(cudaStreamCreateWithFlags(&p->cs_in, cudaStreamNonBlocking));
  if (!p->cs_out) CK(cudaStreamCreateWithFlags(&p->cs_out, cudaStreamNonBlocking));
  int ch = 0;
  const int nch = host_chunks(p, &ch);
  while ((int)p->ev.size() < 2 * nch + 1) {
    cudaEvent_t e;
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    p->ev.push_back(e);
  }
  if (p->own_fft) return MIRT_OK;  // the FFT passes take slice ranges directly
  const int sizes[2] = {ch, p->nslice - (nch - 1) * ch};
  int n[3];
  for (int d = 0; d < p->gg.D; d++) n[d] = p->gg.K[p->gg.D - 1 - d];
  for (int i = 0; i < 2; i++) {
    if (p->ch_n[i] == sizes[i]) continue;
    if (p->ch_n[i]) cufftDestroy(p->fft_ch[i]);
    p->ch_n[i] = 0;
    cufftResult r = cufftPlanMany(&p->fft_ch[i], p->gg.D, n, nullptr, 1, (int)p->gg.ngrid, nullptr,
                                  1, (int)p->gg.ngrid, CUFFT_C2C, sizes[i] * p->C);
    if (r != CUFFT_SUCCESS)
      return fail(MIRT_ERR_FFT, "cufftPlanMany failed: " + std::to_string((int)r));
    p->ch_n[i] = sizes[i];
  }
  return MIRT_OK;
}

// Host-buffer call pipelined over slice chunks: the copy in of chunk i + 1 and
// the copy out of chunk i - 1 overlap the compute of chunk i (copy streams
// cs_in / cs_out, compute on the caller's stream, ordered by events).
template <bool FWD>
int host_pipelined(mirt_nufft *p, const float *in, float *out, cudaStream_t st) {
  int rc = host_pipeline_setup(p);
  if (rc) return rc;
  int ch = 0;
  const int nch = host_chunks(p, &ch);
  const long long C = p->C, xi = p->gg.npix * C;
  const std::vector<long long> &mo = p->ip->moff_host;
  const float2 *hin = reinterpret_cast<const float2 *>(in);
  float2 *hout = reinterpret_cast<float2 *>(out);
  float2 *din = FWD ? p->hx.as<float2>() : p->hX.as<float2>();
  float2 *dout = FWD ? p->hX.as<float2>() : p->hx.as<float2>();
  // earlier work on the caller's stream comes first
  CK(cudaEventRecord(p->ev[2 * nch], st));
  CK(cudaStreamWaitEvent(p->cs_in, p->ev[2 * nch], 0));
  for (int i = 0; i < nch; i++) {
    const int s0 = i * ch, s1 = std::min(p->nslice, s0 + ch);
    const long long i0 = FWD ? s0 * xi : mo[s0] * C, i1 = FWD ? s1 * xi : mo[s1] * C;
    const long long o0 = FWD ? mo[s0] * C : s0 * xi, o1 = FWD ? mo[s1] * C : s1 * xi;
    if (i1 > i0)
      CK(cudaMemcpyAsync(din + i0, hin + i0, (i1 - i0) * sizeof(float2), cudaMemcpyHostToDevice,
                         p->cs_in));
    CK(cudaEventRecord(p->ev[2 * i], p->cs_in));
    CK(cudaStreamWaitEvent(st, p->ev[2 * i], 0));
    cufftHandle f = p->fft_ch[(s1 - s0) == p->ch_n[0] ? 0 : 1];
    rc = FWD ? nufft_forward_range(p, s0, s1, din, dout, f, st)
             : nufft_adjoint_range(p, s0, s1, din, dout, f, st);
    if (rc) return rc;
    CK(cudaEventRecord(p->ev[2 * i + 1], st));
    CK(cudaStreamWaitEvent(p->cs_out, p->ev[2 * i + 1], 0));
    if (o1 > o0)
      CK(cudaMemcpyAsync(hout + o0, dout + o0, (o1 - o0) * sizeof(float2), cudaMemcpyDeviceToHost,
                         p->cs_out));
  }
  CK(cudaStreamSynchronize(p->cs_out));
  CK(cudaStreamSynchronize(st));
  return MIRT_OK;
}

// the chunked path needs several slices and, for the adjoint, the row sweep
bool host_pipeline_ok(const mirt_nufft *p, bool fwd) {
  return p->nslice > 1 && p->C > 0 && (fwd || p->ip->t.sweep != 0);
}

}  // namespace

extern "C" {

int mirt_nufft_forward_host(mirt_nufft *p, const float *x, float *X, void *stream) {
  if (!p) return fail(MIRT_ERR_ARG, "nufft is NULL");
  cudaStream_t st = as_stream(stream);
  const size_t bx = (size_t)p->nslice * p->gg.npix * p->C * sizeof(float2);
  const size_t bX = (size_t)p->Mtot * p->C * sizeof(float2);
  if (p->hx.bytes < bx) CK(p->hx.alloc(bx));
  if (p->hX.bytes < bX) CK(p->hX.alloc(bX));
  if (host_pipeline_ok(p, true)) return host_pipelined<true>(p, x, X, st);
  CK(cudaMemcpyAsync(p->hx.p, x, bx, cudaMemcpyHostToDevice, st));
  int rc = mirt_nufft_forward(p, p->hx.p, p->hX.p, stream);
  if (rc) return rc;
  CK(cudaMemcpyAsync(X, p->hX.p, bX, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return MIRT_OK;
}

int mirt_nufft_adjoint_host(mirt_nufft *p, const float *X, float *x, void *stream) {
  if (!p) return fail(MIRT_ERR_ARG, "nufft is NULL");
  cudaStream_t st = as_stream(stream);
  const size_t bx = (size_t)p->nslice * p->gg.npix * p->C * sizeof(float2);
  const size_t bX = (size_t)p->Mtot * p->C * sizeof(float2);
  if (p->hx.bytes < bx) CK(p->hx.alloc(bx));
  if (p->hX.bytes < bX) CK(p->hX.alloc(bX));
  if (host_pipeline_ok(p, false)) return host_pipelined<false>(p, X, x, st);
  CK(cudaMemcpyAsync(p->hX.p, X, bX, cudaMemcpyHostToDevice, st));
  int rc = mirt_nufft_adjoint(p, p->hX.p, p->hx.p, stream);
  if (rc) return rc;
  CK(cudaMemcpyAsync(x, p->hx.p, bx, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return MIRT_OK;
}

mirt_interp_plan *mirt_nufft_interp_plan(mirt_nufft *p) { return p ? p->ip : nullptr; }

}  // extern "C"

struct mirt_graph {
  cudaGraphExec_t exec = nullptr;
  ~mirt_graph() {
    if (exec) cudaGraphExecDestroy(exec);
  }
};

extern "C" {

int mirt_nufft_capture(mirt_nufft *p, const void *x, void *X, void *xa, mirt_graph **out) {
  if (!p || !out || !X || (!x && !xa)) return fail(MIRT_ERR_ARG, "NULL argument");
  *out = nullptr;
  cudaStream_t cs;
  CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  int rc = MIRT_OK;
  if (e == cudaSuccess) {
    if (x) rc = mirt_nufft_forward(p, x, X, cs);
    if (!rc && xa) rc = mirt_nufft_adjoint(p, X, xa, cs);
    const cudaError_t e2 = cudaStreamEndCapture(cs, &graph);
    if (!rc && e2 != cudaSuccess) e = e2;
  }
  cudaGraphExec_t exec = nullptr;
  if (!rc && e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
  if (graph) cudaGraphDestroy(graph);
  cudaStreamDestroy(cs);
  if (rc) return rc;
  if (e != cudaSuccess)
    return fail(MIRT_ERR_CUDA, std::string("NUFFT graph capture: ") + cudaGetErrorString(e));
  auto *g = new mirt_graph();
  g->exec = exec;
  *out = g;
  return MIRT_OK;
}

int mirt_graph_launch(mirt_graph *g, void *stream) {
  if (!g) return fail(MIRT_ERR_ARG, "graph is NULL");
  CK(cudaGraphLaunch(g->exec, as_stream(stream)));
  return MIRT_OK;
}

int mirt_graph_destroy(mirt_graph *g) {
  delete g;
  return MIRT_OK;
}

int mirt_nufft_autotune(mirt_nufft *p, void *stream) {
  if (!p) return fail(MIRT_ERR_ARG, "nufft is NULL");
  return mirt_interp_plan_autotune(p->ip, stream);
}

static bool a3d(const mirt_nufft *p) { return p->gg.D == 3; }

int mirt_nufft_config(mirt_nufft *p, int32_t *out, int32_t n) {
  if (!p || !out) return fail(MIRT_ERR_ARG, "NULL argument");
  const Tiling &t = p->ip->t;
  // gather: one launch (TMA-staged or plain)
  const int fwd = (p->own_fft ? p->gg.D : 2) + 1;
  int spread = 1;
  if (t.sweep != 0) {
    // ordering pass, dense-bin patches (chunk sums, per-bin sums), sweep (and a
    // memset of the queue counters)
    const bool dense = t.ndense > 0 && (a3d(p) || (t.dense_on && t.sweep_rows == 1));
    spread = 2 + (dense ? 2 : 0);
    // the staged 2D sweep reading the caller's samples has no ordering pass
    const bool staged2 = !a3d(p) && t.sweep_staged == 2 && p->ip->ls.cw == 32 &&
                         !(t.dense_on && t.dense_of && t.sweep_rows == 1);
    if (staged2) spread = 1;
  } else if (t.own) {
    spread = 1;  // the clearing memset, then per colour a launch and a reduction
    for (int c = 0; c < 4; c++)
      spread += (t.color_beg[c + 1] > t.color_beg[c]) + (t.red_beg[c + 1] > t.red_beg[c]);
  } else {
    spread = (t.ntask > 0) + (t.nred > 0);
  }
  const int adj = spread + (p->own_fft ? p->gg.D : 2);
  const int32_t v[3] = {p->own_fft ? 1 : 0, fwd, adj};
  for (int i = 0; i < n && i < 3; i++) out[i] = v[i];
  return MIRT_OK;
}

int mirt_nufft_destroy(mirt_nufft *p) {
  if (p) {
    cudaDeviceSynchronize();
    delete p;
  }
  return MIRT_OK;
}

}  // extern "C"
