// gather_tma.cu -- the forward gather (nufft/table/interp2_table1_for.c) for 2D
// plans with J = 6 and 32-coil chunks, over grid tiles and sample records
// staged in shared memory by the Tensor Memory Accelerator.
//
// The gather order groups the samples by 8 x 8 blocks of their first taps
// (slice-major, then block rows, then block columns); a work item is up to
// TG_RC consecutive samples of one block.  A CTA's items alternate between
// two shared-memory stages; an item's copies -- on one mbarrier, a
// cp.async.bulk.tensor of the block's 13 x 13 grid points x 32 (or 16) coils
// and 1-D bulk copies of the item's tap coefficients and first taps
// (contiguous in the gather order) -- are issued while the item before it is
// summed: the first two at the CTA's start, each later one by the last warp to
// finish the item two before it, into the stage that item frees.  No CTA-wide
// barrier: warps do not wait for the slowest warp of every item.  The CTA's
// eight warps take the item's samples in turn (lane = coil; two samples per
// warp with 16-coil tiles), starting from a warp that rotates from item to
// item, and read their records, output rows and phases and all 36 taps from
// shared memory.  Blocks whose taps wrap past
// K (the last block row and column) read the grid from global memory instead.
// Per sample the taps are summed in the order of the plain gather (columns
// inner, rows outer, packed FP32x2 MACs), so the two give identical results.
//
// Waits are bounded: when a stage does not arrive within the limit the warp
// sets the plan's fault flag, waits (bounded) for the other stage's copy in
// flight and stops; the stage is then never released, so no further copy is
// issued, and the other warps' waits run out in turn.  The host reads the
// flag (mirt_interp_plan_fault).
#include <cuda.h>
#include <cudaTypedefs.h>

#include "interp_impl.cuh"

namespace mirt {
namespace {

constexpr int TG_GB = 8;               // block of first taps per dimension
constexpr int TG_TW = TG_GB + 5;       // tile extent per dimension (J = 6)
constexpr int TG_RC = 96;              // samples per work item
constexpr unsigned TG_W_BYTES = TG_RC * 12 * 8;                 // 9,216
constexpr unsigned TG_K_BYTES = TG_RC * 16;                     // 1,536
constexpr unsigned TG_O_BYTES = TG_RC * 16;                     // 1,536
constexpr int TG_THREADS = 256;
constexpr long long TG_WAIT_LIMIT = 1ll << 22;
constexpr long long TG_TEST_WAIT_LIMIT = 1ll << 12;
// Tiles of TCW coils: 32 (a warp per sample, lane = coil) or 16 (a half-warp
// per sample: smaller stages, three CTAs per SM instead of two).
template <int TCW>
struct TgShape {
  static constexpr unsigned TILE = TG_TW * TG_TW * TCW * 8;         // 43,264 / 21,632
  static constexpr unsigned STAGE = TILE + TG_W_BYTES + TG_K_BYTES + TG_O_BYTES;  // 55,552 / 33,920
  static constexpr int CTAS_PER_SM = TCW == 32 ? 2 : 3;
  static_assert(TILE % 128 == 0 && STAGE % 128 == 0, "stages must stay 128-byte aligned");
};

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

// one thread: record the item in the stage's header, arm the stage's barrier
// (its arrival publishes the header to the waiting warps) and start its
// copies.  no_copy (the test of the bounded waits): arm the barrier for bytes
// that no copy will deliver and issue no copy, so that its wait runs out with
// nothing in flight.
template <int TCW>
__device__ __forceinline__ void stage_issue(const CUtensorMap *tm, const InterpArgs &a,
                                            const int4 *orec, unsigned char *st, uint64_t *bar,
                                            Item *hdr, const Item &r, int chunk, bool no_copy) {
  constexpr unsigned TILE = TgShape<TCW>::TILE;
  const unsigned wb = (unsigned)r.n * 96u, kb = (unsigned)r.n * 16u;
  *hdr = r;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (no_copy) {
    mbar_expect(bar, 16u);
    return;
  }
  mbar_expect(bar, (r.interior ? TILE : 0u) + wb + 2 * kb);
  if (r.interior)
    tile_copy(tm, st, bar, chunk * 2 * TCW, r.bx * TG_GB, r.by * TG_GB, r.slice);
  bulk_copy(st + TILE, a.W + (long long)r.p0 * 12, wb, bar);
  bulk_copy(st + TILE + TG_W_BYTES, a.K0 + r.p0, kb, bar);
  bulk_copy(st + TILE + TG_W_BYTES + TG_K_BYTES, orec + r.p0, kb, bar);
}

template <bool REAL, int TCW>
__global__ void __launch_bounds__(TG_THREADS, TgShape<TCW>::CTAS_PER_SM)
    gather_tma_kernel(const __grid_constant__ CUtensorMap tmap, InterpArgs a, GatherBlocks g,
                      long long it0, long long nit, const float2 *__restrict__ ck,
                      float2 *__restrict__ fm, int *__restrict__ fault, int no_copy,
                      long long wait_limit) {
  constexpr unsigned TILE = TgShape<TCW>::TILE, STAGE = TgShape<TCW>::STAGE;
  constexpr int SPW = 32 / TCW;  // samples per warp at a time
  constexpr int NWARP = TG_THREADS / 32;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + 2 * STAGE);
  Item *hdr = reinterpret_cast<Item *>(bar + 2);  // each stage's item
  int *done = reinterpret_cast<int *>(hdr + 2);   // warps finished with each stage's item
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = lane / TCW, cl = lane % TCW;
  const int C = a.C;
  const int chunk = blockIdx.y;
  const int c = chunk * TCW + cl;
  const bool on = c < C;
  const int K1 = a.g.K[0], K2 = a.g.K[1];
  const long long end = it0 + nit;
  if (threadIdx.x == 0) {
    mbar_init(&bar[0]);
    mbar_init(&bar[1]);
    done[0] = done[1] = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // the CTA's items are it0 + blockIdx.x + k gridDim.x, k = 0, 1, ...; item k
  // goes to stage k & 1.  The first two are issued here; after that the last
  // warp to finish item k issues item k + 2 into the stage it frees, so no
  // warp waits for another except through the two stages.
  if (threadIdx.x == 0)
    for (int k = 0; k < 2; k++) {
      const long long i = it0 + blockIdx.x + (long long)k * gridDim.x;
      if (i < end)
        stage_issue<TCW>(&tmap, a, g.orec, smem + k * STAGE, &bar[k], &hdr[k], item_of(g, a, i),
                         chunk, no_copy);
    }
  for (int k = 0;; k++) {
    const long long i = it0 + blockIdx.x + (long long)k * gridDim.x;
    if (i >= end) break;
    const int s = k & 1;
    if (!stage_wait(&bar[s], (unsigned)(k >> 1) & 1u, wait_limit)) {
      // the stage did not arrive in time: flag it, let the other stage's copy
      // land (bounded), and stop this warp; the stage is never released, so
      // no further copy is issued
      if (lane == 0) {
        atomicExch(fault, 1);
        if (i + gridDim.x < end)
          stage_wait(&bar[s ^ 1], (unsigned)((k + 1) >> 1) & 1u, wait_limit);
      }
      return;
    }
    const Item r = hdr[s];
    const unsigned char *st = smem + s * STAGE;
    const float2 *tile = reinterpret_cast<const float2 *>(st);
    const float2 *Wst = reinterpret_cast<const float2 *>(st + TILE);
    const int4 *Kst = reinterpret_cast<const int4 *>(st + TILE + TG_W_BYTES);
    const int4 *Ost = reinterpret_cast<const int4 *>(st + TILE + TG_W_BYTES + TG_K_BYTES);
    const int x0 = r.bx * TG_GB, y0 = r.by * TG_GB;
    const float2 *gs = ck + (long long)r.slice * a.grid_elems + c;
    // the warps' share of the item rotates from item to item
    const int wr = (warp + NWARP - (k % NWARP)) % NWARP;
    for (int q = wr * SPW + sub; q < r.n; q += NWARP * SPW) {
      const int4 o = Ost[q];  // output row and phase
      const int m = o.x;
      const float2 ph = make_float2(__int_as_float(o.z), __int_as_float(o.w));
      const int4 k0 = Kst[q];
      const float2 *Ws = Wst + q * 12;
      float2 w1[6];
#pragma unroll
      for (int j = 0; j < 6; j++) w1[j] = Ws[j];
      detail::CAcc s2;
      detail::cacc_zero(s2);
      if (r.interior) {
        const float2 *tl = tile + ((k0.y - y0) * TG_TW + (k0.x - x0)) * TCW + cl;
#pragma unroll
        for (int j2 = 0; j2 < 6; j2++) {
          detail::CAcc s1;
          detail::cacc_zero(s1);
#pragma unroll
          for (int j1 = 0; j1 < 6; j1++)
            detail::cacc_mac<REAL>(s1, w1[j1], tl[(j2 * TG_TW + j1) * TCW]);
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
    // release the stage; the last warp out refills it with item k + 2
    __syncwarp();
    if (lane == 0) {
      __threadfence_block();
      if (atomicAdd(&done[s], 1) == NWARP - 1) {
        done[s] = 0;
        __threadfence_block();
        const long long i2 = i + 2ll * gridDim.x;
        if (i2 < end)
          stage_issue<TCW>(&tmap, a, g.orec, smem + s * STAGE, &bar[s], &hdr[s],
                           item_of(g, a, i2), chunk, no_copy);
      }
    }
  }
}

// ------------------------------------------------------------------------
// 3D: 4 x 4 x 4 blocks of first taps, 9 x 9 x 9 x 8-coil tiles
// ------------------------------------------------------------------------
// The same pipeline for 3D plans (J = 6, an even C >= 8): the gather order's
// 4 x 4 x 4 blocks of first taps, items of up to 32 samples, one 5-D tile copy
// of the block's 9 x 9 x 9 grid points x 8 coils per item; a warp serves four
// samples at a time (lane = 8 coils x 4 samples), eight warps the item's 32.
// Per sample the taps are summed in the order of the plain gather (j1 inner,
// then j2, then j3; packed FP32x2 MACs): identical results.
constexpr int T3_GB = 4, T3_TW = T3_GB + 5, T3_CW = 8, T3_RC = 32;
constexpr unsigned T3_TILE_RAW = T3_TW * T3_TW * T3_TW * T3_CW * 8;            // 46,656
constexpr unsigned T3_TILE = (T3_TILE_RAW + 127) / 128 * 128;                   // 46,720
constexpr unsigned T3_W_BYTES = T3_RC * 18 * 8;                                 // 4,608
constexpr unsigned T3_K_BYTES = T3_RC * 16;                                     // 512
constexpr unsigned T3_STAGE = T3_TILE + T3_W_BYTES + 2 * T3_K_BYTES;            // 52,352
static_assert(T3_STAGE % 128 == 0, "stages must stay 128-byte aligned");

struct Item3 {
  int slice, bx, by, bz, p0, n;
  bool interior;
};

__device__ __forceinline__ Item3 item3_of(const GatherBlocks &g, const InterpArgs &a, long long i) {
  const int2 it = g.item[i];
  Item3 r;
  const long long per = (long long)g.nbx * g.nby * g.nbz;
  r.slice = (int)(it.x / per);
  int q = (int)(it.x - (long long)r.slice * per);
  r.bz = q / (g.nbx * g.nby);
  q -= r.bz * g.nbx * g.nby;
  r.by = q / g.nbx;
  r.bx = q - r.by * g.nbx;
  r.p0 = it.y;
  r.n = min(T3_RC, g.start[it.x + 1] - it.y);
  r.interior = r.bx * T3_GB + T3_TW <= a.g.K[0] && r.by * T3_GB + T3_TW <= a.g.K[1] &&
               r.bz * T3_GB + T3_TW <= a.g.K[2];
  return r;
}

// 5-D tile copy into this CTA's own shared memory
__device__ __forceinline__ void tile_copy5(const CUtensorMap *tm, void *dst, uint64_t *bar, int x,
                                           int y, int z, int w, int v) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(v),
      "r"(smem_addr(bar))
      : "memory");
}

// FLAT (C = 8): the grid rows' (k1, coil) pairs are contiguous, and the tile is
// copied as 9 x 9 rows of 9 x 8 coils (4-D map, 576-byte rows) instead of
// 9 x 9 x 9 rows of 8 coils (5-D map, 64-byte rows); the same layout in shared
// memory.
template <bool FLAT>
__device__ __forceinline__ void stage3_issue(const CUtensorMap *tm, const InterpArgs &a,
                                             const int4 *orec, unsigned char *st, uint64_t *bar,
                                             Item3 *hdr, const Item3 &r, int chunk, bool no_copy) {
  const unsigned wb = (unsigned)r.n * 144u, kb = (unsigned)r.n * 16u;
  *hdr = r;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (no_copy) {
    mbar_expect(bar, 16u);
    return;
  }
  mbar_expect(bar, (r.interior ? T3_TILE_RAW : 0u) + wb + 2 * kb);
  if (r.interior) {
    if (FLAT)
      tile_copy(tm, st, bar, r.bx * T3_GB * 2 * T3_CW, r.by * T3_GB, r.bz * T3_GB, r.slice);
    else
      tile_copy5(tm, st, bar, chunk * 2 * T3_CW, r.bx * T3_GB, r.by * T3_GB, r.bz * T3_GB, r.slice);
  }
  bulk_copy(st + T3_TILE, a.W + (long long)r.p0 * 18, wb, bar);
  bulk_copy(st + T3_TILE + T3_W_BYTES, a.K0 + r.p0, kb, bar);
  bulk_copy(st + T3_TILE + T3_W_BYTES + T3_K_BYTES, orec + r.p0, kb, bar);
}

template <bool REAL, bool FLAT>
__global__ void __launch_bounds__(TG_THREADS, 2)
    gather_tma3_kernel(const __grid_constant__ CUtensorMap tmap, InterpArgs a, GatherBlocks g,
                       long long it0, long long nit, const float2 *__restrict__ ck,
                       float2 *__restrict__ fm, int *__restrict__ fault, int no_copy,
                       long long wait_limit) {
  constexpr int SPW = 32 / T3_CW;  // samples per warp at a time
  constexpr int NWARP = TG_THREADS / 32;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + 2 * T3_STAGE);
  Item3 *hdr = reinterpret_cast<Item3 *>(bar + 2);
  int *done = reinterpret_cast<int *>(hdr + 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = lane / T3_CW, cl = lane % T3_CW;
  const int C = a.C;
  const int chunk = blockIdx.y;
  const int c = chunk * T3_CW + cl;
  const bool on = c < C;
  const int K1 = a.g.K[0], K2 = a.g.K[1], K3 = a.g.K[2];
  const long long rstr = (long long)K1 * C, pstr = (long long)K2 * K1 * C;
  const long long end = it0 + nit;
  if (threadIdx.x == 0) {
    mbar_init(&bar[0]);
    mbar_init(&bar[1]);
    done[0] = done[1] = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int k = 0; k < 2; k++) {
      const long long i = it0 + blockIdx.x + (long long)k * gridDim.x;
      if (i < end)
        stage3_issue<FLAT>(&tmap, a, g.orec, smem + k * T3_STAGE, &bar[k], &hdr[k],
                           item3_of(g, a, i), chunk, no_copy);
    }
  for (int k = 0;; k++) {
    const long long i = it0 + blockIdx.x + (long long)k * gridDim.x;
    if (i >= end) break;
    const int s = k & 1;
    if (!stage_wait(&bar[s], (unsigned)(k >> 1) & 1u, wait_limit)) {
      if (lane == 0) {
        atomicExch(fault, 1);
        if (i + gridDim.x < end)
          stage_wait(&bar[s ^ 1], (unsigned)((k + 1) >> 1) & 1u, wait_limit);
      }
      return;
    }
    const Item3 r = hdr[s];
    // the descriptor of item k + 2, loaded now in case this warp releases the stage
    const long long i2 = i + 2ll * gridDim.x;
    Item3 r2{};
    if (lane == 0 && i2 < end) r2 = item3_of(g, a, i2);
    const unsigned char *st = smem + s * T3_STAGE;
    const float2 *tile = reinterpret_cast<const float2 *>(st);
    const float2 *Wst = reinterpret_cast<const float2 *>(st + T3_TILE);
    const int4 *Kst = reinterpret_cast<const int4 *>(st + T3_TILE + T3_W_BYTES);
    const int4 *Ost = reinterpret_cast<const int4 *>(st + T3_TILE + T3_W_BYTES + T3_K_BYTES);
    const int x0 = r.bx * T3_GB, y0 = r.by * T3_GB, z0 = r.bz * T3_GB;
    const float2 *gs = ck + (long long)r.slice * a.grid_elems + c;
    const int wr = (warp + NWARP - (k % NWARP)) % NWARP;
    for (int q = wr * SPW + sub; q < r.n; q += NWARP * SPW) {
      const int4 o = Ost[q];
      const int m = o.x;
      const float2 ph = make_float2(__int_as_float(o.z), __int_as_float(o.w));
      const int4 k0 = Kst[q];
      const float2 *Ws = Wst + q * 18;
      float2 w1[6];
#pragma unroll
      for (int j = 0; j < 6; j++) w1[j] = Ws[j];
      detail::CAcc s3;
      detail::cacc_zero(s3);
      if (r.interior) {
        const float2 *tl =
            tile + (((k0.z - z0) * T3_TW + (k0.y - y0)) * T3_TW + (k0.x - x0)) * T3_CW + cl;
#pragma unroll 2
        for (int j3 = 0; j3 < 6; j3++) {
          detail::CAcc s2;
          detail::cacc_zero(s2);
#pragma unroll
          for (int j2 = 0; j2 < 6; j2++) {
            const float2 *row = tl + (j3 * T3_TW + j2) * T3_TW * T3_CW;
            detail::CAcc s1;
            detail::cacc_zero(s1);
#pragma unroll
            for (int j1 = 0; j1 < 6; j1++) detail::cacc_mac<REAL>(s1, w1[j1], row[j1 * T3_CW]);
            detail::cacc_mac<false>(s2, Ws[6 + j2], detail::cacc_get<REAL>(s1));
          }
          detail::cacc_mac<false>(s3, Ws[12 + j3], detail::cacc_get<false>(s2));
        }
      } else if (on) {
#pragma unroll 1
        for (int j3 = 0; j3 < 6; j3++) {
          const float2 *pl = gs + (long long)detail::tap_k(k0.z, j3, K3) * pstr;
          detail::CAcc s2;
          detail::cacc_zero(s2);
#pragma unroll 1
          for (int j2 = 0; j2 < 6; j2++) {
            const float2 *row = pl + (long long)detail::tap_k(k0.y, j2, K2) * rstr;
            detail::CAcc s1;
            detail::cacc_zero(s1);
#pragma unroll
            for (int j1 = 0; j1 < 6; j1++)
              detail::cacc_mac<REAL>(s1, w1[j1],
                                     __ldg(row + (long long)detail::tap_k(k0.x, j1, K1) * C));
            detail::cacc_mac<false>(s2, Ws[6 + j2], detail::cacc_get<REAL>(s1));
          }
          detail::cacc_mac<false>(s3, Ws[12 + j3], detail::cacc_get<false>(s2));
        }
      }
      float2 out = detail::cacc_get<false>(s3);
      if (a.phase) out = cmul(out, ph);
      if (on) fm[(long long)m * C + c] = out;
    }
    __syncwarp();
    if (lane == 0) {
      __threadfence_block();
      if (atomicAdd(&done[s], 1) == NWARP - 1) {
        done[s] = 0;
        __threadfence_block();
        if (i2 < end)
          stage3_issue<FLAT>(&tmap, a, g.orec, smem + s * T3_STAGE, &bar[s], &hdr[s], r2, chunk,
                             no_copy);
      }
    }
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
  if (a.g.D != 2 || a.C < 32 || (a.C & 1)) return false;
  for (int d = 0; d < 2; d++)
    if (a.g.J[d] != 6 || a.g.K[d] < TG_TW) return false;
  return true;
}

int gather_tma_block() { return TG_GB; }
int gather_tma_item() { return TG_RC; }

bool gather_tma3_ok(const InterpArgs &a) {
  if (a.g.D != 3 || a.C < T3_CW || (a.C & 1)) return false;
  for (int d = 0; d < 3; d++)
    if (a.g.J[d] != 6 || a.g.K[d] < T3_TW) return false;
  return true;
}

int gather_tma3_block() { return T3_GB; }
int gather_tma3_item() { return T3_RC; }

namespace {
cudaError_t launch_gather_tma3(const InterpArgs &a, const GatherBlocks &g, int nslice,
                               long long it0, long long nit, const float2 *ck, float2 *fm,
                               int *fault, cudaStream_t st, int fault_test) {
  if (!gather_tma3_ok(a) || g.gb != T3_GB || a.SJ != 18) return cudaErrorInvalidValue;
  PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
  if (!enc) return cudaErrorNotSupported;
  // the grid as floats [S][K3][K2][K1][2C]: dims innermost first, strides in
  // bytes; with C = 8, k1 and the coils as one dimension of 2 C K1 floats
  CUtensorMap tm;
  const bool flat = a.C == T3_CW;
  const cuuint64_t row = (cuuint64_t)2 * a.C * 4;
  const cuuint64_t K1 = a.g.K[0], K2 = a.g.K[1], K3 = a.g.K[2];
  const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  CUresult r;
  if (flat) {
    const cuuint64_t dims[4] = {(cuuint64_t)2 * a.C * K1, K2, K3, (cuuint64_t)nslice};
    const cuuint64_t strides[3] = {row * K1, row * K1 * K2, row * K1 * K2 * K3};
    const cuuint32_t box[4] = {(cuuint32_t)(2 * T3_CW * T3_TW), T3_TW, T3_TW, 1};
    r = enc(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float2 *>(ck), dims, strides, box,
            estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  } else {
    const cuuint64_t dims[5] = {(cuuint64_t)2 * a.C, K1, K2, K3, (cuuint64_t)nslice};
    const cuuint64_t strides[4] = {row, row * K1, row * K1 * K2, row * K1 * K2 * K3};
    const cuuint32_t box[5] = {(cuuint32_t)(2 * T3_CW), T3_TW, T3_TW, T3_TW, 1};
    r = enc(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, const_cast<float2 *>(ck), dims, strides, box,
            estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  }
  if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
  auto kern = a.real_tab ? (flat ? gather_tma3_kernel<true, true> : gather_tma3_kernel<true, false>)
                         : (flat ? gather_tma3_kernel<false, true> : gather_tma3_kernel<false, false>);
  const size_t smem = 2 * (size_t)T3_STAGE + 2 * sizeof(uint64_t) + 2 * sizeof(Item3) +
                      2 * sizeof(int);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  long long ctas = (long long)nsm * 2;
  if (ctas > nit) ctas = nit;
  const unsigned nchunk = (unsigned)((a.C + T3_CW - 1) / T3_CW);
  const long long limit = fault_test ? TG_TEST_WAIT_LIMIT : TG_WAIT_LIMIT;
  kern<<<dim3((unsigned)ctas, nchunk), TG_THREADS, smem, st>>>(tm, a, g, it0, nit, ck, fm, fault,
                                                              fault_test ? 1 : 0, limit);
  return cudaGetLastError();
}
}  // namespace

cudaError_t launch_gather_tma(const InterpArgs &a, const GatherBlocks &g, int nslice,
                              long long it0, long long nit, const float2 *ck, float2 *fm,
                              int *fault, cudaStream_t st, int fault_test, int tcw) {
  if (a.Mtot == 0 || a.C == 0 || nit <= 0) return cudaSuccess;
  if (a.g.D == 3) return launch_gather_tma3(a, g, nslice, it0, nit, ck, fm, fault, st, fault_test);
  if (!gather_tma_ok(a) || g.gb != TG_GB || a.SJ != 12 || (tcw != 32 && tcw != 16))
    return cudaErrorInvalidValue;
  PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
  if (!enc) return cudaErrorNotSupported;
  // the grid as floats [S][K2][K1][2C]: dims innermost first, strides in bytes
  CUtensorMap tm;
  const cuuint64_t dims[4] = {(cuuint64_t)2 * a.C, (cuuint64_t)a.g.K[0], (cuuint64_t)a.g.K[1],
                              (cuuint64_t)nslice};
  const cuuint64_t row = (cuuint64_t)2 * a.C * 4;
  const cuuint64_t strides[3] = {row, row * a.g.K[0], row * a.g.K[0] * a.g.K[1]};
  const cuuint32_t box[4] = {(cuuint32_t)(2 * tcw), TG_TW, TG_TW, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = enc(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float2 *>(ck), dims, strides,
                   box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
  auto go = [&](auto kern, unsigned stage, int per_sm, int cw) -> cudaError_t {
    const size_t smem = 2 * (size_t)stage + 2 * sizeof(uint64_t) + 2 * sizeof(Item) +
                        2 * sizeof(int);
    cudaError_t e =
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    long long ctas = (long long)nsm * per_sm;
    if (ctas > nit) ctas = nit;
    const unsigned nchunk = (unsigned)((a.C + cw - 1) / cw);
    // the test of the bounded waits: no copies, and a short wait limit
    const long long limit = fault_test ? TG_TEST_WAIT_LIMIT : TG_WAIT_LIMIT;
    kern<<<dim3((unsigned)ctas, nchunk), TG_THREADS, smem, st>>>(tm, a, g, it0, nit, ck, fm, fault,
                                                                fault_test ? 1 : 0, limit);
    return cudaGetLastError();
  };
  if (tcw == 32)
    return go(a.real_tab ? gather_tma_kernel<true, 32> : gather_tma_kernel<false, 32>,
              TgShape<32>::STAGE, TgShape<32>::CTAS_PER_SM, 32);
  return go(a.real_tab ? gather_tma_kernel<true, 16> : gather_tma_kernel<false, 16>,
            TgShape<16>::STAGE, TgShape<16>::CTAS_PER_SM, 16);
}

}  // namespace mirt
