// noalloc.cu -- a forward gather that allocates no device memory.
//
// Some callers cannot allocate GPU memory: code that runs while a stream is
// being captured into a CUDA graph, hosts that hand all device memory to their
// own pool (e.g. a MATLAB or framework allocator) and forbid cudaMalloc after
// start-up, and real-time loops where an allocation could stall.  For them,
// mirt_interp_gather_noalloc runs the table gather on buffers the caller
// already owns.  The only scratch it needs -- the per-sample tap coefficients
// and wrapped first taps, the same data an interpolation plan keeps -- lives
// in the fixed array below, which is part of the library image: every GPU that
// loads the library holds these MIRT_NOALLOC_SCRATCH_BYTES until the process
// exits.
#include "../../include/mirt_b200.h"

#include <mutex>
#include <string>

#include "interp.cuh"

namespace {

// 32 MiB of tap scratch.  Per sample it holds 8 * (J1 + ... + JD) bytes of
// coefficients and 16 bytes of first taps (112 bytes for J = 6 in 2D, 160 in 3D).
static __device__ __align__(256) unsigned char g_noalloc_scratch[MIRT_NOALLOC_SCRATCH_BYTES];

std::mutex g_noalloc_mu;
void *g_noalloc_ptr[256] = {nullptr};

}  // namespace

namespace mirt {
int api_fail(int code, const std::string &msg);  // capi.cu: sets mirt_last_error()
}  // namespace mirt

static int noalloc_fail(int code, const std::string &msg) { return mirt::api_fail(code, msg); }

extern "C" int mirt_interp_gather_noalloc(int32_t D, const int32_t *K, const int32_t *J,
                                          const int32_t *L, const void *const *tab,
                                          int32_t real_tab, int32_t order, const double *tm,
                                          int64_t M, int32_t ncol, const void *ck, void *fm,
                                          void *stream) {
  using namespace mirt;
  if (D < 1 || D > MIRT_DMAX) return noalloc_fail(MIRT_ERR_ARG, "D must be 1, 2 or 3");
  if (!K || !J || !L || !tab || !tm || !ck || !fm)
    return noalloc_fail(MIRT_ERR_ARG, "NULL argument");
  if (order != 0 && order != 1) return noalloc_fail(MIRT_ERR_ARG, "bad order");
  if (!real_tab && order) return noalloc_fail(MIRT_ERR_ARG, "only 0th order implemented for complex");
  if (M < 0 || ncol < 1) return noalloc_fail(MIRT_ERR_ARG, "M must be >= 0 and ncol >= 1");
  int SJ = 0;
  long long grid = ncol;
  for (int d = 0; d < D; d++) {
    if (K[d] < 1 || J[d] < 1 || J[d] > MIRT_JMAX || J[d] > K[d] || L[d] < 1)
      return noalloc_fail(MIRT_ERR_ARG, "need 1 <= J <= min(K, 16) and L >= 1");
    SJ += J[d];
    grid *= K[d];
  }
  if (grid >= (1ll << 31)) return noalloc_fail(MIRT_ERR_ARG, "grid too large");
  const size_t per_sample = (size_t)SJ * sizeof(float2) + sizeof(int4);
  const long long m_max = (long long)((MIRT_NOALLOC_SCRATCH_BYTES - 256) / per_sample);
  if (M > m_max)
    return noalloc_fail(MIRT_ERR_ARG,
                        "mirt_interp_gather_noalloc: M = " + std::to_string(M) +
                            " exceeds the fixed scratch (" + std::to_string(m_max) +
                            " samples for this J)");
  if (M == 0) return MIRT_OK;

  // device address of the scratch array, looked up once per device with that
  // device current (the host-side symbol is only a stand-in)
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 256)
    return noalloc_fail(MIRT_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  unsigned char *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess)
        return noalloc_fail(MIRT_ERR_CUDA,
                            std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_noalloc_ptr[dev] = p;
    }
    scratch = static_cast<unsigned char *>(g_noalloc_ptr[dev]);
  }
  // K0 first (16-byte records), then the coefficients
  int4 *K0 = reinterpret_cast<int4 *>(scratch);
  float2 *W = reinterpret_cast<float2 *>(scratch + (((size_t)M * sizeof(int4) + 255) & ~(size_t)255));

  InterpArgs a{};
  a.g.D = D;
  long long stride = 1;
  for (int d = 0; d < MIRT_DMAX; d++) {
    if (d < D) {
      a.g.K[d] = K[d];
      a.g.J[d] = J[d];
      a.g.L[d] = L[d];
      a.g.ncenter[d] = (int)((long long)J[d] * L[d] / 2);
      a.g.tlen[d] = J[d] * L[d] + 1;
      a.g.kstride[d] = stride;
      stride *= K[d];
      a.tab[d] = tab[d];
    } else {
      a.g.K[d] = a.g.J[d] = a.g.L[d] = a.g.tlen[d] = 1;
      a.g.ncenter[d] = 0;
      a.g.kstride[d] = stride;
    }
  }
  a.real_tab = real_tab ? 1 : 0;
  a.order = order;
  a.C = ncol;
  a.Mtot = M;
  a.tm = tm;
  a.slice_id = nullptr;
  a.perm = nullptr;
  a.phase = nullptr;
  a.grid_elems = grid;
  a.SJ = SJ;
  a.W = W;
  a.K0 = K0;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  e = launch_prep_taps(a, W, K0, st);
  if (e != cudaSuccess)
    return noalloc_fail(MIRT_ERR_CUDA, std::string("tap set-up: ") + cudaGetErrorString(e));
  Launch l{};
  l.threads = 256;
  l.cw = ncol >= 32 ? 32 : ncol >= 8 ? 8 : ncol >= 4 ? 4 : 1;
  l.sb = 0;
  l.grid = 0;
  e = launch_gather(a, l, static_cast<const float2 *>(ck), static_cast<float2 *>(fm), st);
  if (e != cudaSuccess)
    return noalloc_fail(MIRT_ERR_CUDA, std::string("gather: ") + cudaGetErrorString(e));
  return MIRT_OK;
}
