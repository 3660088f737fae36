// interp.cu -- bin keys, the stable bin sort, and the public launchers of the
// table-interpolation kernels (templates in interp_impl.cuh, instantiated per
// dimension in interp_d{1,2,3}.cu).
#include "interp_impl.cuh"

namespace mirt {
// ------------------------------------------------------------------------
// bin keys
// ------------------------------------------------------------------------
__global__ void bin_keys_kernel(InterpArgs a, Tiling t, uint32_t *keys) {
  const long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (m >= a.Mtot) return;
  int bin = 0, mul = 1;
  for (int d = 0; d < a.g.D; d++) {
    const double td = a.tm[(long long)d * a.Mtot + m];
    const int k0 = wrapk(koff_of(td, a.g.J[d]), a.g.K[d]);
    bin += (k0 / t.B[d]) * mul;
    mul *= t.nbin[d];
  }
  const int s = a.slice_id ? a.slice_id[m] : 0;
  keys[m] = (uint32_t)s * (uint32_t)t.nbins + (uint32_t)bin;
}

cudaError_t launch_bin_keys(const InterpArgs &a, const Tiling &t, uint32_t *keys,
                            cudaStream_t st) {
  if (a.Mtot == 0) return cudaSuccess;
  const int thr = 256;
  const long long blocks = (a.Mtot + thr - 1) / thr;
  bin_keys_kernel<<<(unsigned)blocks, thr, 0, st>>>(a, t, keys);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------
// stable LSD radix sort of bin keys (8-bit digits), deterministic
// ------------------------------------------------------------------------
namespace {
constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_CHUNK = 4096;  // elements per block
constexpr unsigned FULL = 0xffffffffu;

__global__ void rs_hist(const uint32_t *keys, long long n, int shift, int nblk, int *hist) {
  __shared__ int cnt[256];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  const long long beg = (long long)blockIdx.x * RS_CHUNK;
  const long long end = min(beg + RS_CHUNK, n);
  for (long long i = beg + threadIdx.x; i < end; i += RS_THREADS)
    atomicAdd(&cnt[(keys[i] >> shift) & 255u], 1);
  __syncthreads();
  hist[threadIdx.x * nblk + blockIdx.x] = cnt[threadIdx.x];
}

// exclusive scan of n ints in one block of 1024 threads
__global__ void rs_scan(int *v, int n) {
  __shared__ int part[1024];
  const int seg = (n + 1023) / 1024;
  const int beg = threadIdx.x * seg;
  const int end = min(beg + seg, n);
  int s = 0;
  for (int i = beg; i < end; i++) s += v[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    int x = threadIdx.x >= off ? part[threadIdx.x - off] : 0;
    __syncthreads();
    part[threadIdx.x] += x;
    __syncthreads();
  }
  int run = part[threadIdx.x] - s;
  for (int i = beg; i < end; i++) {
    const int x = v[i];
    v[i] = run;
    run += x;
  }
}

// Stable scatter: elements keep their input order within a digit.  Each warp
// ranks its 32 elements with match_any; warps are then ordered by a per-digit
// prefix over the warp counts, and the block's running digit offsets advance.
__global__ void rs_scatter(const uint32_t *kin, const int *vin, long long n, int shift, int nblk,
                           const int *offs, uint32_t *kout, int *vout) {
  __shared__ int run[256];
  __shared__ int wcnt[RS_WARPS][256];
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  run[tid] = offs[tid * nblk + blockIdx.x];
  const long long beg = (long long)blockIdx.x * RS_CHUNK;
  const long long end = min(beg + RS_CHUNK, n);
  const unsigned lt = (1u << lane) - 1u;
  for (long long base = beg; base < end; base += RS_THREADS) {
    for (int i = tid; i < RS_WARPS * 256; i += RS_THREADS) (&wcnt[0][0])[i] = 0;
    __syncthreads();
    const long long i = base + tid;
    const bool valid = i < end;
    const uint32_t key = valid ? kin[i] : 0u;
    const int val = valid ? (vin ? vin[i] : (int)i) : 0;
    const unsigned dig = valid ? ((key >> shift) & 255u) : 256u;
    const unsigned peers = __match_any_sync(FULL, dig);
    const int rank = __popc(peers & lt);
    if (valid && rank == 0) wcnt[w][dig] = __popc(peers);
    __syncthreads();
    {
      int acc = run[tid];
      for (int ww = 0; ww < RS_WARPS; ww++) {
        const int c = wcnt[ww][tid];
        wcnt[ww][tid] = acc;
        acc += c;
      }
      run[tid] = acc;
    }
    __syncthreads();
    if (valid) {
      const int pos = wcnt[w][dig] + rank;
      kout[pos] = key;
      vout[pos] = val;
    }
    __syncthreads();
  }
}

__global__ void rs_bin_start(const uint32_t *ks, long long n, int nbins, int *bin_start) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long long k = ks[i];
  const long long kp = i > 0 ? (long long)ks[i - 1] : -1;
  for (long long b = kp + 1; b <= k; b++) bin_start[b] = (int)i;
  if (i == n - 1)
    for (long long b = k + 1; b <= nbins; b++) bin_start[b] = (int)n;
}

__global__ void fill_int(int *p, int n, int v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}
}  // namespace

size_t radix_sort_tmp_bytes(long long n) {
  const long long nblk = (n + RS_CHUNK - 1) / RS_CHUNK + 1;
  return (size_t)(4 * n * 4) + (size_t)(256 * nblk * 4) + 1024;
}

cudaError_t radix_sort_bins(const uint32_t *keys, long long n, int nbins, void *tmp, int *perm,
                            int *bin_start, cudaStream_t st) {
  if (n == 0) {
    fill_int<<<(nbins + 1 + 255) / 256, 256, 0, st>>>(bin_start, nbins + 1, 0);
    return cudaGetLastError();
  }
  const int nblk = (int)((n + RS_CHUNK - 1) / RS_CHUNK);
  char *p = static_cast<char *>(tmp);
  uint32_t *kA = reinterpret_cast<uint32_t *>(p);
  uint32_t *kB = kA + n;
  int *vA = reinterpret_cast<int *>(kB + n);
  int *vB = vA + n;
  int *hist = vB + n;
  int bits = 1;
  while (bits < 32 && (1ll << bits) < (long long)nbins) bits++;
  const int npass = (bits + 7) / 8;
  const uint32_t *kin = keys;
  const int *vin = nullptr;
  for (int ps = 0; ps < npass; ps++) {
    const int shift = 8 * ps;
    uint32_t *kout = (ps & 1) ? kB : kA;
    int *vout = (ps == npass - 1) ? perm : ((ps & 1) ? vB : vA);
    rs_hist<<<nblk, RS_THREADS, 0, st>>>(kin, n, shift, nblk, hist);
    rs_scan<<<1, 1024, 0, st>>>(hist, 256 * nblk);
    rs_scatter<<<nblk, RS_THREADS, 0, st>>>(kin, vin, n, shift, nblk, hist, kout, vout);
    kin = kout;
    vin = vout;
  }
  rs_bin_start<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(kin, n, nbins, bin_start);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------
// per-position tap data
// ------------------------------------------------------------------------
cudaError_t launch_prep_taps(const InterpArgs &a, float2 *W, int4 *K0, cudaStream_t st) {
  if (a.Mtot == 0) return cudaSuccess;
  const unsigned blocks = (unsigned)((a.Mtot + 255) / 256);
  if (a.real_tab)
    detail::prep_taps_kernel<true><<<blocks, 256, 0, st>>>(a, W, K0);
  else
    detail::prep_taps_kernel<false><<<blocks, 256, 0, st>>>(a, W, K0);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------
// public launchers
// ------------------------------------------------------------------------
namespace {
cudaError_t dispatch(detail::Req &r) {
  switch (r.a->g.D) {
    case 1: return detail::dispatch_d1(r);
    case 2: return detail::dispatch_d2(r);
    case 3: return detail::dispatch_d3(r);
    default: return cudaErrorInvalidValue;
  }
}
}  // namespace

cudaError_t query_gather_grid(const InterpArgs &a, Launch &l) {
  detail::Req r{detail::GATHER_GRID, &a, nullptr, &l, nullptr, nullptr, nullptr, 0};
  return dispatch(r);
}

cudaError_t launch_gather(const InterpArgs &a, const Launch &l, const float2 *ck, float2 *fm,
                          cudaStream_t st) {
  if (a.Mtot == 0 || a.C == 0) return cudaSuccess;
  Launch lc = l;
  detail::Req r{detail::GATHER, &a, nullptr, &lc, nullptr, ck, fm, st};
  return dispatch(r);
}

namespace {
__global__ void mark_dense_kernel(const int *__restrict__ dense_bin, int n, int *dense_of) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dense_of[dense_bin[i]] = i;
}
}  // namespace

cudaError_t launch_mark_dense(const int *dense_bin, int n, int *dense_of, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  mark_dense_kernel<<<(n + 255) / 256, 256, 0, st>>>(dense_bin, n, dense_of);
  return cudaGetLastError();
}

cudaError_t launch_spread(const InterpArgs &a, const Tiling &t, const Launch &l,
                          const int *bin_start, const float2 *fm, float2 *ck, cudaStream_t st) {
  if (a.C == 0) return cudaSuccess;
  Launch lc = l;
  detail::Req r{detail::SPREAD, &a, &t, &lc, bin_start, fm, ck, st};
  return dispatch(r);
}

}  // namespace mirt
