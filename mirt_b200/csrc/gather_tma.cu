// gather_tma.cu -- the forward gather (nufft/table/interp2_table1_for.c) for 2D
// plans with J = 6 and 32-coil chunks, over grid tiles and sample records
// staged in shared memory by the Tensor Memory Accelerator.
//
// The gather order groups the samples by 8 x 8 blocks of their first taps
// (slice-major, then block rows, then block columns); a work item is up to
// TG_RC consecutive samples of one block.  A CTA takes one item at a time:
// one thread issues, on one mbarrier, a cp.async.bulk.tensor of the block's
// 13 x 13 grid points x 32 coils and 1-D bulk copies of the item's tap
// coefficients and first taps (contiguous in the gather order) into one of
// two shared-memory stages, and issues the next item's copies into the other
// stage before the current one is used, so the loads overlap the arithmetic.
// The CTA's eight warps take the item's samples in turn (lane = coil) and
// read their records and all 36 taps from shared memory; only the output
// index and phase come from global memory.  Blocks whose taps wrap past K
// (the last block row and column) read the grid from global memory instead.
// Per sample the taps are summed in the order of the plain gather (columns
// inner, rows outer, packed FP32x2 MACs), so the two give identical results.
//
// Waits are bounded: when a stage does not arrive within the limit the CTA
// sets the plan's fault flag, waits (bounded) for its other stage in flight
// and stops; the host reads the flag (mirt_interp_plan_fault).
#include <cuda.h>
#include <cudaTypedefs.h>

#include "interp_impl.cuh"

namespace mirt {
namespace {

constexpr int TG_GB = 8;               // block of first taps per dimension
constexpr int TG_TW = TG_GB + 5;       // tile extent per dimension (J = 6)
constexpr int TG_CW = 32;              // coils per tile (lanes)
constexpr unsigned TG_TILE_BYTES = TG_TW * TG_TW * TG_CW * 8;   // 43,264
constexpr int TG_RC = 96;              // samples per work item
constexpr unsigned TG_W_BYTES = TG_RC * 12 * 8;                 // 9,216
constexpr unsigned TG_K_BYTES = TG_RC * 16;                     // 1,536
constexpr unsigned TG_STAGE = TG_TILE_BYTES + TG_W_BYTES + TG_K_BYTES;  // 54,016 = 422 x 128
constexpr int TG_THREADS = 256;
constexpr long long TG_WAIT_LIMIT = 1ll << 22;
constexpr long long TG_TEST_WAIT_LIMIT = 1ll << 12;

__device__ __forceinline__ unsigned smem_addr(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// 4-D tile copy into this CTA's own shared memory
__device__ __forceinline__ void tile_copy(const CUtensorMap *tm, void *dst, uint64_t *bar, int x,
                                          int y, int z, int w) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_addr(bar))
      : "memory");
}

// 1-D bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned)
__device__ __forceinline__ void bulk_copy(void *dst, const void *src, unsigned bytes,
                                          uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// wait for phase `parity` of the barrier, at most `limit` polls
__device__ __forceinline__ bool stage_wait(uint64_t *bar, unsigned parity, long long limit) {
  for (long long it = 0; it < limit; it++) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

struct Item {
  int slice, bx, by, p0, n;
  bool interior;
};

__device__ __forceinline__ Item item_of(const GatherBlocks &g, const InterpArgs &a, long long i) {
  const int2 it = g.item[i];
  Item r;
  const long long per = (long long)g.nbx * g.nby;
  r.slice = (int)(it.x / per);
  const int q = (int)(it.x - (long long)r.slice * per);
  r.by = q / g.nbx;
  r.bx = q - r.by * g.nbx;
  r.p0 = it.y;
  r.n = min(TG_RC, g.start[it.x + 1] - it.y);
  r.interior = r.bx * TG_GB + TG_TW <= a.g.K[0] && r.by * TG_GB + TG_TW <= a.g.K[1];
  return r;
}

// one thread: arm the stage's barrier and start its copies.  no_copy (the
// test of the bounded waits): arm the barrier for bytes that no copy will
// deliver and issue no copy, so that its wait runs out with nothing in flight.
__device__ __forceinline__ void stage_issue(const CUtensorMap *tm, const InterpArgs &a,
                                            unsigned char *st, uint64_t *bar, const Item &r,
                                            int chunk, bool no_copy) {
  const unsigned wb = (unsigned)r.n * 96u, kb = (unsigned)r.n * 16u;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (no_copy) {
    mbar_expect(bar, 16u);
    return;
  }
  mbar_expect(bar, (r.interior ? TG_TILE_BYTES : 0u) + wb + kb);
  if (r.interior)
    tile_copy(tm, st, bar, chunk * 2 * TG_CW, r.bx * TG_GB, r.by * TG_GB, r.slice);
  bulk_copy(st + TG_TILE_BYTES, a.W + (long long)r.p0 * 12, wb, bar);
  bulk_copy(st + TG_TILE_BYTES + TG_W_BYTES, a.K0 + r.p0, kb, bar);
}

template <bool REAL>
__global__ void __launch_bounds__(TG_THREADS, 2)
    gather_tma_kernel(const __grid_constant__ CUtensorMap tmap, InterpArgs a, GatherBlocks g,
                      long long it0, long long nit, const float2 *__restrict__ ck,
                      float2 *__restrict__ fm, int *__restrict__ fault, int no_copy,
                      long long wait_limit) {
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + 2 * TG_STAGE);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarp = TG_THREADS / 32;
  const int C = a.C;
  const int chunk = blockIdx.y;
  const int c = chunk * TG_CW + lane;
  const bool on = c < C;
  const int K1 = a.g.K[0], K2 = a.g.K[1];
  if (threadIdx.x == 0) {
    mbar_init(&bar[0]);
    mbar_init(&bar[1]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  unsigned par0 = 0u, par1 = 0u;  // wait parity of each stage's barrier
  const long long end = it0 + nit;
  long long i = it0 + blockIdx.x;
  if (threadIdx.x == 0 && i < end)
    stage_issue(&tmap, a, smem, &bar[0], item_of(g, a, i), chunk, no_copy);
  for (int k = 0; i < end; i += gridDim.x, k++) {
    const int s = k & 1;
    const long long inx = i + gridDim.x;
    if (threadIdx.x == 0 && inx < end)
      stage_issue(&tmap, a, smem + (s ^ 1) * TG_STAGE, &bar[s ^ 1], item_of(g, a, inx), chunk,
                  no_copy);
    const Item r = item_of(g, a, i);
    const bool ready = stage_wait(&bar[s], s ? par1 : par0, wait_limit);
    if (s) par1 ^= 1u;
    else par0 ^= 1u;
    if (__syncthreads_or(!ready)) {
      // a stage did not arrive in time: flag it, let the other stage land
      // (bounded), and stop this CTA
      if (threadIdx.x == 0) {
        atomicExch(fault, 1);
        if (inx < end) stage_wait(&bar[s ^ 1], s ? par0 : par1, wait_limit);
      }
      return;
    }
    const unsigned char *st = smem + s * TG_STAGE;
    const float2 *tile = reinterpret_cast<const float2 *>(st);
    const float2 *Wst = reinterpret_cast<const float2 *>(st + TG_TILE_BYTES);
    const int4 *Kst = reinterpret_cast<const int4 *>(st + TG_TILE_BYTES + TG_W_BYTES);
    const int x0 = r.bx * TG_GB, y0 = r.by * TG_GB;
    const float2 *gs = ck + (long long)r.slice * a.grid_elems + c;
    for (int q = warp; q < r.n; q += nwarp) {
      const int pos = r.p0 + q;
      // output row and phase: global, used last
      const int m = a.perm ? __ldg(a.perm + pos) : pos;
      const float2 ph = a.phase ? __ldg(a.phase + pos) : make_float2(1.f, 0.f);
      const int4 k0 = Kst[q];
      const float2 *Ws = Wst + q * 12;
      float2 w1[6];
#pragma unroll
      for (int j = 0; j < 6; j++) w1[j] = Ws[j];
      detail::CAcc s2;
      detail::cacc_zero(s2);
      if (r.interior) {
        const float2 *tl = tile + ((k0.y - y0) * TG_TW + (k0.x - x0)) * TG_CW + lane;
#pragma unroll
        for (int j2 = 0; j2 < 6; j2++) {
          detail::CAcc s1;
          detail::cacc_zero(s1);
#pragma unroll
          for (int j1 = 0; j1 < 6; j1++)
            detail::cacc_mac<REAL>(s1, w1[j1], tl[(j2 * TG_TW + j1) * TG_CW]);
          detail::cacc_mac<false>(s2, Ws[6 + j2], detail::cacc_get<REAL>(s1));
        }
      } else if (on) {
#pragma unroll 1
        for (int j2 = 0; j2 < 6; j2++) {
          const float2 *row = gs + (long long)detail::tap_k(k0.y, j2, K2) * K1 * C;
          detail::CAcc s1;
          detail::cacc_zero(s1);
#pragma unroll
          for (int j1 = 0; j1 < 6; j1++)
            detail::cacc_mac<REAL>(s1, w1[j1], __ldg(row + (long long)detail::tap_k(k0.x, j1, K1) * C));
          detail::cacc_mac<false>(s2, Ws[6 + j2], detail::cacc_get<REAL>(s1));
        }
      }
      float2 out = detail::cacc_get<false>(s2);
      if (a.phase) out = cmul(out, ph);
      if (on) fm[(long long)m * C + c] = out;
    }
    __syncthreads();  // the stage is free before the next-but-one item is copied into it
  }
}

// the driver's tensor-map encoder, looked up once (thread-safe static init)
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = []() {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    return static_cast<PFN_cuTensorMapEncodeTiled_v12000>(nullptr);
  }();
  return fn;
}

}  // namespace

bool gather_tma_ok(const InterpArgs &a) {
  if (a.g.D != 2 || a.C < TG_CW || (a.C & 1)) return false;
  for (int d = 0; d < 2; d++)
    if (a.g.J[d] != 6 || a.g.K[d] < TG_TW) return false;
  return true;
}

int gather_tma_block() { return TG_GB; }
int gather_tma_item() { return TG_RC; }

cudaError_t launch_gather_tma(const InterpArgs &a, const GatherBlocks &g, int nslice,
                              long long it0, long long nit, const float2 *ck, float2 *fm,
                              int *fault, cudaStream_t st, int fault_test) {
  if (a.Mtot == 0 || a.C == 0 || nit <= 0) return cudaSuccess;
  if (!gather_tma_ok(a) || g.gb != TG_GB || a.SJ != 12) return cudaErrorInvalidValue;
  PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
  if (!enc) return cudaErrorNotSupported;
  // the grid as floats [S][K2][K1][2C]: dims innermost first, strides in bytes
  CUtensorMap tm;
  const cuuint64_t dims[4] = {(cuuint64_t)2 * a.C, (cuuint64_t)a.g.K[0], (cuuint64_t)a.g.K[1],
                              (cuuint64_t)nslice};
  const cuuint64_t row = (cuuint64_t)2 * a.C * 4;
  const cuuint64_t strides[3] = {row, row * a.g.K[0], row * a.g.K[0] * a.g.K[1]};
  const cuuint32_t box[4] = {2 * TG_CW, TG_TW, TG_TW, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = enc(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float2 *>(ck), dims, strides,
                   box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
  const size_t smem = 2 * (size_t)TG_STAGE + 2 * sizeof(uint64_t);
  auto kern = a.real_tab ? gather_tma_kernel<true> : gather_tma_kernel<false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  long long ctas = (long long)nsm * 2;
  if (ctas > nit) ctas = nit;
  const unsigned nchunk = (unsigned)((a.C + TG_CW - 1) / TG_CW);
  // the test of the bounded waits: no copies, and a short wait limit
  const long long limit = fault_test ? TG_TEST_WAIT_LIMIT : TG_WAIT_LIMIT;
  kern<<<dim3((unsigned)ctas, nchunk), TG_THREADS, smem, st>>>(tm, a, g, it0, nit, ck, fm, fault,
                                                              fault_test ? 1 : 0, limit);
  return cudaGetLastError();
}

}  // namespace mirt
