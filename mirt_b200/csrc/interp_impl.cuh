// interp_impl.cuh -- device templates of the gather and spread kernels and
// the launch dispatch, included by one translation unit per dimension
// (interp_d1.cu, interp_d2.cu, interp_d3.cu) so that they compile in parallel.
//
// Forward gather replaces nufft/table/interp{1,2,3}_table1_for.c; the
// adjoint spread replaces nufft/table/interp{1,2,3}_table1_adj.c.
// Table-entry selection and grid wrap are FP64, exactly as the reference
// (common.cuh); taps are accumulated in FP32 with packed FP32x2 FMAs.
//
// Both kernels stage, per CTA, a batch of `sb` samples: one thread per
// (sample, dimension, tap) computes the table coefficient and the wrapped grid
// coordinate once, so that the FP64 index arithmetic is not repeated by every
// coil lane.  Coil lanes then run the taps with coalesced column accesses.
#pragma once
#include "interp.cuh"

namespace mirt {
namespace detail {

// ------------------------------------------------------------------------
// small helpers
// ------------------------------------------------------------------------
// k mod K for any k, cheap when k is within one period of [0, K)
__device__ __forceinline__ int wrap_fast(int k, int K) {
  if (k < 0) k += K;
  else if (k >= K) k -= K;
  if ((unsigned)k >= (unsigned)K) k = wrapk(k, K);
  return k;
}

// k0 + j for a wrapped first tap k0 in [0, K) and 0 <= j < J <= K
__device__ __forceinline__ int tap_k(int k0, int j, int K) {
  const int x = k0 + j;
  return x >= K ? x - K : x;
}

// Coefficient of tap (d, k) for coordinate t: the reference's 0th-order
// lookup or 1st-order linear interpolation of the table.  The index is
// clamped into the table, which changes nothing for |t - k| <= J/2.
template <bool REAL>
__device__ __forceinline__ float2 tap_coef(const InterpArgs &a, int d, double t, int k) {
  const int L = a.g.L[d];
  const int nc = a.g.ncenter[d];
  const int tl = a.g.tlen[d];
  if (REAL) {
    const float *h = static_cast<const float *>(a.tab[d]);
    if (a.order == 0) {
      int n = nc + tab0_index(t, k, L);
      n = min(max(n, 0), tl - 1);
      return make_float2(__ldg(h + n), 0.f);
    }
    float alf;
    int n = nc + tab1_index(t, k, L, &alf);
    n = min(max(n, 0), tl - 1);
    const float h0 = __ldg(h + n);
    // the reference reads one entry past the table end here, times alf = 0
    const float h1 = (n + 1 < tl) ? __ldg(h + n + 1) : 0.f;
    return make_float2((1.f - alf) * h0 + alf * h1, 0.f);
  } else {
    const float2 *h = static_cast<const float2 *>(a.tab[d]);
    int n = nc + tab0_index(t, k, L);
    n = min(max(n, 0), tl - 1);
    return __ldg(h + n);
  }
}

// One thread per position: every tap coefficient and the wrapped first taps.
template <bool REAL>
__global__ void prep_taps_kernel(InterpArgs a, float2 *__restrict__ W, int4 *__restrict__ K0) {
  const long long pos = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (pos >= a.Mtot) return;
  int k0[MIRT_DMAX] = {0, 0, 0};
  float2 *w = W + pos * a.SJ;
  for (int d = 0; d < a.g.D; d++) {
    const double t = a.tm[(long long)d * a.Mtot + pos];
    const int koff = koff_of(t, a.g.J[d]);
    for (int j = 0; j < a.g.J[d]; j++) *w++ = tap_coef<REAL>(a, d, t, koff + j);
    k0[d] = wrap_fast(koff, a.g.K[d]);
  }
  K0[pos] = make_int4(k0[0], k0[1], k0[2], a.slice_id ? a.slice_id[pos] : 0);
}

// Complex accumulator held as two packed pairs: with w = (wr, wi) and
// v = (vr, vi), A += (wr, wr) * v and B += (wi, wi) * v, so that
// sum w * v = (A.x - B.y, A.y + B.x).  Two FFMA2 per complex MAC.
struct CAcc {
  float2 A, B;
};
__device__ __forceinline__ void cacc_zero(CAcc &c) {
  c.A = make_float2(0.f, 0.f);
  c.B = make_float2(0.f, 0.f);
}
template <bool REAL>
__device__ __forceinline__ void cacc_mac(CAcc &c, float2 w, float2 v) {
  c.A = __ffma2_rn(make_float2(w.x, w.x), v, c.A);
  if (!REAL) c.B = __ffma2_rn(make_float2(w.y, w.y), v, c.B);
}
template <bool REAL>
__device__ __forceinline__ float2 cacc_get(const CAcc &c) {
  if (REAL) return c.A;
  return make_float2(c.A.x - c.B.y, c.A.y + c.B.x);
}

// conj(w) * v
template <bool REAL>
__device__ __forceinline__ float2 cw_mul(float2 w, float2 v) {
  if (REAL) return make_float2(w.x * v.x, w.x * v.y);
  return cmulc(w, v);
}

// A += conj(w) * v as two FFMA2: (wr, wr) * (vr, vi) + (wi, -wi) * (vi, vr)
template <bool REAL>
__device__ __forceinline__ float2 cw_fma(float2 w, float2 v, float2 vs, float2 A) {
  A = __ffma2_rn(make_float2(w.x, w.x), v, A);
  if (!REAL) A = __ffma2_rn(make_float2(w.y, -w.y), vs, A);
  return A;
}

// acc += conj(w) * v as four scalar FMAs in the order (re: wr vr, wi vi;
// im: wr vi, -wi vr) -- the roundings of cw_fma.
template <bool REAL>
__device__ __forceinline__ void cmac_conj(float2 &acc, float2 w, float2 v) {
  acc.x = __fmaf_rn(w.x, v.x, acc.x);
  acc.y = __fmaf_rn(w.x, v.y, acc.y);
  if (!REAL) {
    acc.x = __fmaf_rn(w.y, v.y, acc.x);
    acc.y = __fmaf_rn(-w.y, v.x, acc.y);
  }
}

// *p += (wr, wr) v2 + (wi, -wi) v2s: a read-modify-write by the point's one
// owner, or (ATOMIC) two shared-memory atomic adds when warps share the tile
template <bool ATOMIC, bool REAL>
__device__ __forceinline__ void acc_pair(float2 *p, float2 wr, float2 wi, float2 v2, float2 v2s) {
  if constexpr (ATOMIC) {
    float2 c = __fmul2_rn(wr, v2);
    if (!REAL) c = __ffma2_rn(wi, v2s, c);
    atomicAdd(&p->x, c.x);
    atomicAdd(&p->y, c.y);
  } else {
    float2 A = *p;
    A = __ffma2_rn(wr, v2, A);
    if (!REAL) A = __ffma2_rn(wi, v2s, A);
    *p = A;
  }
}

// *p += conj(w) v (vs = (vi, vr))
template <bool ATOMIC, bool REAL>
__device__ __forceinline__ void acc_cw(float2 *p, float2 w, float2 v, float2 vs) {
  acc_pair<ATOMIC, REAL>(p, make_float2(w.x, w.x), make_float2(w.y, -w.y), v, vs);
}

// ------------------------------------------------------------------------
// forward gather
// ------------------------------------------------------------------------
// Persistent CTAs sweep the bin-sorted positions; a group of CW lanes serves
// one position at a time, lane li the columns li, li+CW, ..., and each tap is
// one coalesced column segment of the grid.  The tap coefficients come from
// the plan's per-position table (one broadcast load each).  When the J1 taps
// of a row do not wrap they sit at a constant stride from one row pointer (a
// compile-time stride when C == CW, CX).
template <int D, int CW, int JT, bool REAL, bool CX>
__global__ void __launch_bounds__(256, D == 3 ? 2 : 4) gather_kernel(InterpArgs a, const float2 *__restrict__ ck,
                                                     float2 *__restrict__ fm) {
  const Geom &g = a.g;
  int Jd[MIRT_DMAX] = {1, 1, 1};
#pragma unroll
  for (int d = 0; d < D; d++) Jd[d] = JT > 0 ? JT : g.J[d];
  const int SJ = a.SJ;
  const int gpc = blockDim.x / CW;
  const int li = threadIdx.x % CW;
  const long long ngr = (long long)gridDim.x * gpc;
  const int C = a.C;
  const int cstr = CX ? CW : C;  // grid stride between neighbouring k1
  const long long rstr = (long long)g.kstride[D > 1 ? 1 : 0] * C;
  const long long pstr = (long long)g.kstride[D > 2 ? 2 : 0] * C;
  const int K1 = g.K[0];
  const int K2 = g.K[D > 1 ? 1 : 0];
  const int K3 = g.K[D > 2 ? 2 : 0];

  for (long long pos = (long long)blockIdx.x * gpc + threadIdx.x / CW; pos < a.Mtot;
       pos += ngr) {
    const int4 k0 = a.K0[pos];
    const int m = a.perm ? a.perm[pos] : (int)pos;
    const float2 *Ws = a.W + pos * SJ;
    const float2 *gb = ck + (long long)k0.w * a.grid_elems;
    const float2 ph = a.phase ? a.phase[pos] : make_float2(1.f, 0.f);
    if constexpr (JT > 0) {
      // column coefficients stay in registers; row / plane coefficients are
      // loaded per row (broadcast L1 hits), keeping register pressure low
      float2 w1[JT];
      if constexpr ((JT & 1) == 0) {
        const float4 *W4 = reinterpret_cast<const float4 *>(Ws);
#pragma unroll
        for (int q = 0; q < JT / 2; q++) {
          const float4 v = __ldg(W4 + q);
          w1[2 * q] = make_float2(v.x, v.y);
          w1[2 * q + 1] = make_float2(v.z, v.w);
        }
      } else {
#pragma unroll
        for (int j = 0; j < JT; j++) w1[j] = __ldg(Ws + j);
      }
      const bool fast = k0.x + JT <= K1;
      const int c10 = k0.x * C;
      for (int c = li; c < C; c += CW) {
        const float2 *gc = gb + c;
        // sum over j1 of one grid row (the reference's innermost loop)
        auto rowsum = [&](const float2 *row) -> float2 {
          CAcc s1;
          cacc_zero(s1);
          if (fast) {
            const float2 *p = row + c10;
#pragma unroll
            for (int j1 = 0; j1 < JT; j1++) cacc_mac<REAL>(s1, w1[j1], __ldg(p + j1 * cstr));
          } else {
#pragma unroll
            for (int j1 = 0; j1 < JT; j1++)
              cacc_mac<REAL>(s1, w1[j1], __ldg(row + tap_k(k0.x, j1, K1) * C));
          }
          return cacc_get<REAL>(s1);
        };
        float2 out;
        if constexpr (D == 1) {
          out = rowsum(gc);
        } else if constexpr (D == 2) {
          CAcc s2;
          cacc_zero(s2);
#pragma unroll 3
          for (int j2 = 0; j2 < JT; j2++)
            cacc_mac<false>(s2, __ldg(Ws + JT + j2), rowsum(gc + tap_k(k0.y, j2, K2) * rstr));
          out = cacc_get<false>(s2);
        } else {
          CAcc s3;
          cacc_zero(s3);
#pragma unroll 2
          for (int j3 = 0; j3 < JT; j3++) {
            const float2 *pl = gc + tap_k(k0.z, j3, K3) * pstr;
            CAcc s2;
            cacc_zero(s2);
            // the plane's JT rows at once: all JT x JT tap loads in flight together
#pragma unroll
            for (int j2 = 0; j2 < JT; j2++)
              cacc_mac<false>(s2, __ldg(Ws + JT + j2), rowsum(pl + tap_k(k0.y, j2, K2) * rstr));
            cacc_mac<false>(s3, __ldg(Ws + 2 * JT + j3), cacc_get<false>(s2));
          }
          out = cacc_get<false>(s3);
        }
        if (a.phase) out = cmul(out, ph);
        fm[(long long)m * C + c] = out;
      }
    } else {
      // any J: coefficients read per tap, runtime loops
      for (int c = li; c < C; c += CW) {
        const float2 *gc = gb + c;
        auto rowsum = [&](const float2 *row) -> float2 {
          CAcc s1;
          cacc_zero(s1);
          for (int j1 = 0; j1 < Jd[0]; j1++)
            cacc_mac<REAL>(s1, __ldg(Ws + j1), __ldg(row + (long long)tap_k(k0.x, j1, K1) * C));
          return cacc_get<REAL>(s1);
        };
        float2 out;
        if constexpr (D == 1) {
          out = rowsum(gc);
        } else if constexpr (D == 2) {
          CAcc s2;
          cacc_zero(s2);
          for (int j2 = 0; j2 < Jd[1]; j2++)
            cacc_mac<false>(s2, __ldg(Ws + Jd[0] + j2), rowsum(gc + tap_k(k0.y, j2, K2) * rstr));
          out = cacc_get<false>(s2);
        } else {
          CAcc s3;
          cacc_zero(s3);
          for (int j3 = 0; j3 < Jd[2]; j3++) {
            const float2 *pl = gc + tap_k(k0.z, j3, K3) * pstr;
            CAcc s2;
            cacc_zero(s2);
            for (int j2 = 0; j2 < Jd[1]; j2++)
              cacc_mac<false>(s2, __ldg(Ws + Jd[0] + j2),
                              rowsum(pl + tap_k(k0.y, j2, K2) * rstr));
            cacc_mac<false>(s3, __ldg(Ws + Jd[0] + Jd[1] + j3), cacc_get<false>(s2));
          }
          out = cacc_get<false>(s3);
        }
        if (a.phase) out = cmul(out, ph);
        fm[(long long)m * C + c] = out;
      }
    }
  }
}

// ------------------------------------------------------------------------
// adjoint spread: owner-computes over grid tiles, deterministic
// ------------------------------------------------------------------------
// CTA (tile, slice, coil chunk) accumulates its tile in shared memory and
// writes it once.  Ownership of the accumulators:
//   * warp w owns a contiguous band of the tile's slowest tiled dimension
//     (rows l2 in 2D, planes l3 in 3D, columns l1 in 1D);
//   * lane (s, c), s < SUB = 32/CW, c < CW, owns coil c0 + c of the columns
//     l1 = s (mod SUB).
// Every accumulator therefore has exactly one writer, and every warp walks the
// tile's samples in the same fixed order (source bins in fixed order, samples
// in stable bin-sorted order).  The sum at each grid point is formed in a
// fixed order: no atomics, bitwise reproducible.  A warp skips a sample whose
// taps miss its band with one warp-uniform test.  There is no halo merge
// pass: samples of neighbouring bins whose taps reach into the tile are read.

// Mask of taps j < J whose local coordinate lies in [lo_b, hi_b) and, when
// SUB > 1, is congruent to s modulo SUB.  The taps of a sample are the grid
// points k0w + j (mod K), which in tile-local coordinates form at most two
// runs: base + j before the periodic wrap and base - K + j after it.
template <int SUB>
__host__ __device__ __forceinline__ unsigned tap_mask(int k0w, int J, int K, int lo_tile, int lo_b,
                                                      int hi_b, int s) {
  const int base = k0w - lo_tile;
  const int jw = K - k0w;  // first tap index after the wrap
  unsigned m = 0;
  {
    const int ja = max(0, lo_b - base), jb = min(min(J, jw), hi_b - base);
    if (jb > ja) m |= ((1u << jb) - 1u) & ~((1u << ja) - 1u);
  }
  {
    const int b2 = base - K;
    const int ja = max(jw, lo_b - b2), jb = min(J, hi_b - b2);
    if (jb > ja) m |= ((1u << jb) - 1u) & ~((1u << ja) - 1u);
  }
  if (SUB > 1 && m) {
    // bit j kept iff (base + j) = s (mod SUB); after the wrap base - K + j,
    // and K need not be a multiple of SUB, so test each run separately
    unsigned keep = 0;
    const unsigned all = (J >= 32) ? 0xffffffffu : ((1u << J) - 1u);
    const unsigned pre = (jw >= 32) ? all : (all & ((1u << max(jw, 0)) - 1u));
    {
      const int r = (s - base) & (SUB - 1);
      unsigned p = 0;
      for (int j = r; j < 32; j += SUB) p |= 1u << j;
      keep |= p & pre;
    }
    {
      const int r = (s - (base - K)) & (SUB - 1);
      unsigned p = 0;
      for (int j = r; j < 32; j += SUB) p |= 1u << j;
      keep |= p & ~pre;
    }
    m &= keep;
  }
  return m;
}

__host__ __device__ __forceinline__ int tap_local(int k0w, int j, int K, int lo_tile) {
  int x = k0w + j;
  if (x >= K) x -= K;
  return x - lo_tile;
}

// One grid row of the tile for one sample: acc[l1][lane coil] += conj(w1) v2
// for the lane's taps.  Fast path when all J1 taps lie inside the tile.
template <int CW, int JT, bool REAL, bool ATOMIC>
__device__ __forceinline__ void spread_row(float2 *row, const float2 *Ws, int J1, bool fast1,
                                           int l10, unsigned m1, int k10, int K1, int lo1,
                                           int ls, float2 v2) {
  constexpr int SUB = 32 / CW;
  const float2 v2s = make_float2(v2.y, v2.x);
  if (fast1) {
    for (int j1 = (ls - l10) & (SUB - 1); j1 < J1; j1 += SUB) {
      float2 *p = row + (l10 + j1) * CW;
      acc_cw<ATOMIC, REAL>(p, __ldg(Ws + j1), v2, v2s);
    }
  } else {
    unsigned mm = m1;
    while (mm) {
      const int j1 = __ffs(mm) - 1;
      mm &= mm - 1;
      float2 *p = row + tap_local(k10, j1, K1, lo1) * CW;
      acc_cw<ATOMIC, REAL>(p, __ldg(Ws + j1), v2, v2s);
    }
  }
}

template <int D, int CW, int JT, bool REAL, bool ATOMIC>
__global__ void __launch_bounds__(256) spread_kernel(InterpArgs a, Tiling t,
                                                     const int *__restrict__ bin_start,
                                                     const float2 *__restrict__ fm,
                                                     float2 *__restrict__ ck) {
  constexpr int SUB = 32 / CW;
  extern __shared__ __align__(16) unsigned char smem[];
  const Geom &g = a.g;

  int npts = 1;
#pragma unroll
  for (int d = 0; d < D; d++) npts *= t.T[d];
  // shared tile: rows of RS = T0 + 2 pc points, point (l1, l2, l3) at
  // ((l3 T1 + l2) RS + pc + l1) CW + coil
  const int pc = D > 1 ? t.padc : 0;
  const int RS = t.T[0] + 2 * pc;
  const int nsm = npts / t.T[0] * RS;
  float2 *acc = reinterpret_cast<float2 *>(smem);
  int Jd[MIRT_DMAX] = {1, 1, 1};
#pragma unroll
  for (int d = 0; d < D; d++) Jd[d] = JT > 0 ? JT : g.J[d];
  const int SJ = a.SJ;

  const int task = t.task_tile[blockIdx.x];
  const int2 vr = t.task_range[blockIdx.x];
  const int slot = t.task_slot[blockIdx.x];
  const int tile = task % t.ntiles;
  const int slice = task / t.ntiles;
  const int c0 = blockIdx.y * CW;
  int b[MIRT_DMAX] = {0, 0, 0}, lo[MIRT_DMAX] = {0, 0, 0}, ext[MIRT_DMAX] = {1, 1, 1};
  {
    int r = tile;
#pragma unroll
    for (int d = 0; d < D; d++) {
      b[d] = r % t.nb[d];
      r /= t.nb[d];
      lo[d] = b[d] * t.T[d];
      ext[d] = min(t.T[d], g.K[d] - lo[d]);
    }
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarp = blockDim.x >> 5;
  const int ls = lane / CW;   // column class
  const int lc = lane % CW;   // coil within the chunk
  constexpr int BD = D - 1;   // band dimension
  // deterministic: warp w owns a band of the slowest tiled dimension and walks
  // every visit; ATOMIC: every warp owns the whole tile and takes every
  // nwarp-th visit
  const int per = ATOMIC ? t.T[BD] : (t.T[BD] + nwarp - 1) / nwarp;
  const int band_lo = ATOMIC ? 0 : min(warp * per, ext[BD]);
  const int band_hi = ATOMIC ? ext[BD] : min(band_lo + per, ext[BD]);
  for (int e = threadIdx.x; e < nsm * CW; e += blockDim.x) acc[e] = make_float2(0.f, 0.f);
  __syncthreads();

  // source rows (dimensions >= 1) x the two dimension-0 runs
  const int ns1 = D > 1 ? t.nsrc[1][b[1]] : 1, ns2 = D > 2 ? t.nsrc[2][b[2]] : 1;
  const int4 run = t.run0[b[0]];
  const int nsrc_tot = ns1 * ns2 * 2;
  const int C = a.C;
  const int T0 = t.T[0];
  const int T1 = D > 1 ? t.T[1] : 1;
  const int jb0 = D == 1 ? 0 : (D == 2 ? Jd[0] : Jd[0] + Jd[1]);  // first tap of dim BD
  const bool lane_on = c0 + lc < C;

  long long vbase = 0, vcta = 0;
  for (int si = 0; si < nsrc_tot && vbase < vr.y && band_lo < band_hi; si++) {
    const int kr = si & 1, rest = si >> 1;
    const int rs = kr ? run.z : run.x, rl = kr ? run.w : run.y;
    if (rl == 0) continue;
    int row = 0;
    if (D > 1) row += t.src[1][b[1] * MIRT_SRCMAX + rest % ns1] * t.nbin[0];
    if (D > 2) row += t.src[2][b[2] * MIRT_SRCMAX + rest / ns1] * t.nbin[0] * t.nbin[1];
    const int bin = slice * t.nbins + row + rs;
    const long long b0 = bin_start[bin], b1 = bin_start[bin + rl];
    // this task's share of the tile's visit sequence
    const long long beg = b0 + max(0ll, (long long)vr.x - vbase);
    const long long end = b0 + min(b1 - b0, (long long)vr.y - vbase);
    vbase += b1 - b0;
    if (beg >= end) continue;
    // ATOMIC: warp w takes the task's visits w, w + nwarp, ...
    const int stp = ATOMIC ? nwarp : 1;
    long long first = beg;
    if (ATOMIC) {
      first = beg + ((warp - (int)(vcta % nwarp)) % nwarp + nwarp) % nwarp;
      vcta += end - beg;
    }
    if (first >= end) continue;
    // one position ahead: its first taps and sample index are in flight
    int4 kn = a.K0[first];
    int mn = a.perm ? a.perm[first] : (int)first;
    for (long long pos = first; pos < end; pos += stp) {
      const int4 k = kn;
      const int m = mn;
      if (pos + stp < end) {
        kn = a.K0[pos + stp];
        mn = a.perm ? a.perm[pos + stp] : (int)(pos + stp);
      }
      const int kb = D == 1 ? k.x : (D == 2 ? k.y : k.z);
      const int l10 = k.x - lo[0];
      const float2 *Ws = a.W + pos * SJ;
      if constexpr (JT > 0 && D >= 2) {
        // The in-tile taps of each dimension are one index range, walked with
        // unrolled loops.  With K >= T + J per dimension a tile meets a
        // sample's taps either before or after their periodic wrap, never
        // both, so the tile-local first tap is k0 - lo, or k0 - lo - K when
        // the taps reach the tile only after the wrap.  A visit whose ranges
        // are empty ends before any coefficient is loaded.
        if (t.wrap_ok) {
          auto rel = [&](int k0, int d) {
            const int l = k0 - lo[d];
            return l >= ext[d] ? l - g.K[d] : l;
          };
          const int f10 = rel(k.x, 0);
          const int ja1 = max(0, -f10), jb1 = min(JT, ext[0] - f10);
          const int lb = rel(kb, BD);
          const int jab = max(0, band_lo - lb), jbb = min(JT, band_hi - lb);
          const int l20 = rel(k.y, 1);
          const int ja2 = D == 3 ? max(0, -l20) : 0, jb2 = D == 3 ? min(JT, ext[1] - l20) : 1;
          if (ja1 >= jb1 || jab >= jbb || ja2 >= jb2) continue;
          float2 f = make_float2(0.f, 0.f);
          if (lane_on) {
            f = __ldg(fm + (long long)m * C + c0 + lc);
            if (a.phase) f = cmulc(__ldg(a.phase + pos), f);
          }
          float2 wr[JT], wi[JT];
          if constexpr (SUB == 1) {
#pragma unroll
            for (int j1 = 0; j1 < JT; j1++) {
              const float2 w = __ldg(Ws + j1);
              wr[j1] = make_float2(w.x, w.x);
              wi[j1] = make_float2(w.y, -w.y);
            }
          }
          // lane's first column tap (class ls of SUB), then every SUB-th
          const int j1s = ja1 + ((ls - f10 - ja1) & (SUB - 1));
          const bool padded = pc >= JT - 1;
          const int j1p = (ls - f10) & (SUB - 1);
          auto row = [&](float2 *p, float2 v2) {
            const float2 v2s = make_float2(v2.y, v2.x);
            if (padded) {
              // every column tap has a slot (spare columns take the ones
              // outside the tile): no bounds tests
              if constexpr (SUB == 1) {
#pragma unroll
                for (int j1 = 0; j1 < JT; j1++) {
                  acc_pair<ATOMIC, REAL>(p + j1 * CW, wr[j1], wi[j1], v2, v2s);
                }
              } else {
                for (int j1 = j1p; j1 < JT; j1 += SUB) {
                  acc_cw<ATOMIC, REAL>(p + j1 * CW, __ldg(Ws + j1), v2, v2s);
                }
              }
            } else if constexpr (SUB == 1) {
#pragma unroll
              for (int j1 = 0; j1 < JT; j1++) {
                if (j1 >= ja1 && j1 < jb1) {
                  acc_pair<ATOMIC, REAL>(p + j1 * CW, wr[j1], wi[j1], v2, v2s);
                }
              }
            } else {
              for (int j1 = j1s; j1 < jb1; j1 += SUB) {
                acc_cw<ATOMIC, REAL>(p + j1 * CW, __ldg(Ws + j1), v2, v2s);
              }
            }
          };
          float2 *base = acc + (pc + f10) * CW + lc;
          if constexpr (D == 2) {
            for (int j2 = jab; j2 < jbb; j2++) {
              const float2 v2 = cw_mul<REAL>(__ldg(Ws + JT + j2), f);
              row(base + (size_t)(lb + j2) * RS * CW, v2);
            }
          } else {
            for (int j3 = jab; j3 < jbb; j3++) {
              const float2 v3 = cw_mul<REAL>(__ldg(Ws + 2 * JT + j3), f);
              float2 *pl = base + (size_t)(lb + j3) * T1 * RS * CW;
              for (int j2 = ja2; j2 < jb2; j2++) {
                const float2 v2 = cw_mul<REAL>(__ldg(Ws + JT + j2), v3);
                row(pl + (size_t)(l20 + j2) * RS * CW, v2);
              }
            }
          }
          continue;
        }
      }
      // general path (periodic wrap inside the patch, or any J)
      const unsigned mb = tap_mask<1>(kb, Jd[BD], g.K[BD], lo[BD], band_lo, band_hi, 0);
      if (!mb) continue;
      float2 f = make_float2(0.f, 0.f);
      if (lane_on) {
        f = __ldg(fm + (long long)m * C + c0 + lc);
        if (a.phase) f = cmulc(__ldg(a.phase + pos), f);
      }
      if constexpr (D == 1) {
        const unsigned m1 = tap_mask<SUB>(k.x, Jd[0], g.K[0], lo[0], band_lo, band_hi, ls);
        spread_row<CW, JT, REAL, ATOMIC>(acc + lc, Ws, Jd[0], false, l10, m1, k.x, g.K[0], lo[0], ls, f);
      } else {
        // lane's columns: fast when the J1 taps do not leave the tile
        const bool fast1 = l10 >= 0 && l10 + Jd[0] <= ext[0];
        const unsigned m1 = fast1 ? 0u : tap_mask<SUB>(k.x, Jd[0], g.K[0], lo[0], 0, ext[0], ls);
        if (!fast1 && !m1) continue;
        if constexpr (D == 2) {
          if constexpr (JT > 0 && SUB == 1) {
            if (fast1) {
              // all J1 columns inside the tile: coefficient pairs in registers,
              // LDS.64 + 2 FFMA2 + STS.64 per tap at compile-time strides
              float2 wr[JT], wi[JT];
#pragma unroll
              for (int j1 = 0; j1 < JT; j1++) {
                const float2 w = __ldg(Ws + j1);
                wr[j1] = make_float2(w.x, w.x);
                wi[j1] = make_float2(w.y, -w.y);
              }
              float2 *base = acc + (pc + l10) * CW + lc;
              unsigned m2 = mb;
              while (m2) {
                const int j2 = __ffs(m2) - 1;
                m2 &= m2 - 1;
                const int l2 = tap_local(k.y, j2, g.K[1], lo[1]);
                const float2 v2 = cw_mul<REAL>(__ldg(Ws + JT + j2), f);
                const float2 v2s = make_float2(v2.y, v2.x);
                float2 *p = base + (size_t)l2 * RS * CW;
#pragma unroll
                for (int j1 = 0; j1 < JT; j1++) {
                  acc_pair<ATOMIC, REAL>(p + j1 * CW, wr[j1], wi[j1], v2, v2s);
                }
              }
              continue;
            }
          }
          unsigned m2 = mb;
          while (m2) {
            const int j2 = __ffs(m2) - 1;
            m2 &= m2 - 1;
            const int l2 = tap_local(k.y, j2, g.K[1], lo[1]);
            const float2 v2 = cw_mul<REAL>(__ldg(Ws + Jd[0] + j2), f);
            spread_row<CW, JT, REAL, ATOMIC>(acc + ((size_t)l2 * RS + pc) * CW + lc, Ws, Jd[0], fast1, l10,
                                     m1, k.x, g.K[0], lo[0], ls, v2);
          }
        } else {
          const unsigned m2all = tap_mask<1>(k.y, Jd[1], g.K[1], lo[1], 0, ext[1], 0);
          if (!m2all) continue;
          unsigned m3 = mb;
          while (m3) {
            const int j3 = __ffs(m3) - 1;
            m3 &= m3 - 1;
            const int l3 = tap_local(k.z, j3, g.K[2], lo[2]);
            const float2 v3 = cw_mul<REAL>(__ldg(Ws + jb0 + j3), f);
            unsigned m2 = m2all;
            while (m2) {
              const int j2 = __ffs(m2) - 1;
              m2 &= m2 - 1;
              const int l2 = tap_local(k.y, j2, g.K[1], lo[1]);
              const float2 v2 = cw_mul<REAL>(__ldg(Ws + Jd[0] + j2), v3);
              spread_row<CW, JT, REAL, ATOMIC>(acc + (((size_t)l3 * T1 + l2) * RS + pc) * CW + lc, Ws,
                                       Jd[0], fast1, l10, m1, k.x, g.K[0], lo[0], ls, v2);
            }
          }
        }
      }
    }
  }
  __syncthreads();
  if (slot >= 0) {
    // partial tile of a split heavy tile: summed later in fixed order
    float2 *part = t.scratch + ((size_t)slot * gridDim.y + blockIdx.y) * npts * CW;
    for (int e = threadIdx.x; e < npts * CW; e += blockDim.x) {
      const int pt = e / CW, cc = e - pt * CW;
      const int l1 = pt % T0, r = pt / T0;
      part[e] = acc[(r * RS + pc + l1) * CW + cc];
    }
    return;
  }
  float2 *gout = ck + (long long)slice * a.grid_elems;
  for (int e = threadIdx.x; e < npts * CW; e += blockDim.x) {
    const int pt = e / CW, cc = e - pt * CW;
    const int l1 = pt % T0;
    const int l2 = D > 1 ? (pt / T0) % T1 : 0;
    const int l3 = D > 2 ? pt / (T0 * T1) : 0;
    if (l1 >= ext[0] || l2 >= ext[1] || l3 >= ext[2] || c0 + cc >= C) continue;
    long long kk = lo[0] + l1;
    if (D > 1) kk += (long long)(lo[1] + l2) * g.kstride[1];
    if (D > 2) kk += (long long)(lo[2] + l3) * g.kstride[2];
    gout[kk * C + c0 + cc] = acc[((pt / T0) * RS + pc + l1) * CW + cc];
  }
}

// Row-sweep spread (2D, J = 6 in both dimensions, one-point bins, K1, K2 >= 6).
// A team of CW lanes (lane = coil) owns a band of R grid rows y0 .. y0 + R - 1
// (rows past K2 - 1 in the last band are computed and dropped) and a segment
// [x0, x1) of their columns, of one slice and coil chunk.  The samples with a
// tap in the band are those binned (by their wrapped first tap) in bin rows
// y0 - 5 + q, q = 0 .. R + 4 (modulo K2); bin row q reaches band row r through
// tap row j2 = r - q + 5 when 0 <= j2 < 6, a static set per q.  The team sweeps
// bin columns xb = x0 - 5 .. x1 - 1 (modulo K1: five warm-up columns, wrapped
// when x0 < 5) and keeps the accumulators of grid columns xb .. xb + 5 of its R
// rows in registers; after bin column xb, column xb has all its contributions
// and is stored if it lies in the segment.  Summation order per grid point:
// bin columns ascending, bin rows ascending, samples in the stable sort order
// -- fixed, and the same for every R and segmentation, so the result is
// bitwise reproducible and independent of both.
// sorted[p][c] = conj(phase[p]) fm[perm[p]][c]: the samples in plan order, so
// that the sweep reads each bin's samples as one contiguous block.
template <int CW>
__global__ void __launch_bounds__(256) sweep_order_kernel(InterpArgs a, const float2 *__restrict__ fm,
                                                          float2 *__restrict__ sorted,
                                                          long long pos0, long long npos) {
  const long long e0 = pos0 * a.C, n = npos * (long long)a.C;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long e = e0 + i;
    const long long p = e / a.C;
    const int c = (int)(e - p * a.C);
    const int m = a.perm ? __ldg(a.perm + p) : (int)p;
    float2 v = __ldg(fm + (long long)m * a.C + c);
    if (a.phase) v = cmulc(__ldg(a.phase + p), v);
    sorted[e] = v;
  }
}

// The sweep of one team (see spread_sweep_kernel).  DENSE: bins with at least
// dense_min samples add their patches (dense_part/reduce_kernel) instead.
template <int CW, int R, bool REAL, bool DENSE>
__device__ __forceinline__ void sweep_team(const InterpArgs &a, const Tiling &t,
                                           const int *__restrict__ bin_start,
                                           const float2 *__restrict__ fs,
                                           float2 *__restrict__ ck, long long team) {
  constexpr int NQ = R + 5;  // bin rows reaching the band
  const int K1 = a.g.K[0], K2 = a.g.K[1];
  int slice, y0, x0, x1;
  if (t.sweep < 0) {
    const int4 tk = t.sweep_team[team];
    slice = tk.x;
    y0 = tk.y;
    x0 = tk.z;
    x1 = tk.w;
  } else {
    const int nseg = t.sweep;
    const int nband = (K2 + R - 1) / R;
    const int seg = (int)(team % nseg);
    const long long bandid = team / nseg;
    const int sl = (int)(bandid / nband);
    y0 = (int)(bandid - (long long)sl * nband) * R;
    slice = t.slice0 + sl;
    const int sw = (K1 + nseg - 1) / nseg;
    x0 = seg * sw;
    x1 = min(K1, x0 + sw);
  }
  if (x0 >= x1) return;
  const int C = a.C;
  const int c = blockIdx.y * CW + (int)(threadIdx.x % CW);
  const bool on = c < C;
  const int *bs = bin_start + (long long)slice * t.nbins;
  int row[NQ];
#pragma unroll
  for (int q = 0; q < NQ; q++) {
    int b = (y0 - 5 + q) % K2;
    if (b < 0) b += K2;
    row[q] = b * K1;  // one-point bins: K1 bins per row
  }
  const int xs = x0 - 5;
  int beg[NQ];
#pragma unroll
  for (int q = 0; q < NQ; q++) beg[q] = __ldg(bs + row[q] + (xs < 0 ? xs + K1 : xs));
  float2 acc[R][6];
#pragma unroll
  for (int r = 0; r < R; r++)
#pragma unroll
    for (int j = 0; j < 6; j++) acc[r][j] = make_float2(0.f, 0.f);
  float2 *out = ck + (long long)slice * a.grid_elems + (long long)y0 * K1 * C + c;
  for (int xb = xs; xb < x1; xb++) {
    const int xw = xb < 0 ? xb + K1 : xb;
    if (xb == 0 && xs < 0) {
#pragma unroll
      for (int q = 0; q < NQ; q++) beg[q] = __ldg(bs + row[q]);
    }
    int end[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) end[q] = __ldg(bs + row[q] + xw + 1);
#pragma unroll
    for (int q = 0; q < NQ; q++) {
      const int pe = end[q];
      if constexpr (DENSE) {
        if (pe - beg[q] >= t.dense_min) {
          // a dense bin: the sums of its samples, from its patch
          const int dn = __ldg(t.dense_of + (long long)slice * t.nbins + row[q] + xw);
          if (on) {
#pragma unroll
            for (int r = 0; r < R; r++) {
              const int j2 = r - q + 5;
              if (j2 >= 0 && j2 < 6) {
                const float2 *pp = t.patch + ((long long)dn * 36 + j2 * 6) * C + c;
#pragma unroll
                for (int j = 0; j < 6; j++) {
                  const float2 v = __ldg(pp + (long long)j * C);
                  acc[r][j].x += v.x;
                  acc[r][j].y += v.y;
                }
              }
            }
          }
          beg[q] = pe;
          continue;
        }
      }
      for (int p = beg[q]; p < pe; p++) {
        const float2 f = on ? __ldg(fs + (long long)p * C + c) : make_float2(0.f, 0.f);
        const float2 *Ws = a.W + (long long)p * 12;
        const float4 *W4 = reinterpret_cast<const float4 *>(Ws);
        float4 w1[3];
#pragma unroll
        for (int h = 0; h < 3; h++) w1[h] = __ldg(W4 + h);
#pragma unroll
        for (int r = 0; r < R; r++) {
          const int j2 = r - q + 5;  // compile-time after unrolling
          if (j2 >= 0 && j2 < 6) {
            const float2 v = cw_mul<REAL>(__ldg(Ws + 6 + j2), f);
            const float2 vs = make_float2(v.y, v.x);
#pragma unroll
            for (int h = 0; h < 3; h++) {
              acc[r][2 * h] = cw_fma<REAL>(make_float2(w1[h].x, w1[h].y), v, vs, acc[r][2 * h]);
              acc[r][2 * h + 1] =
                  cw_fma<REAL>(make_float2(w1[h].z, w1[h].w), v, vs, acc[r][2 * h + 1]);
            }
          }
        }
      }
      beg[q] = end[q];
    }
    if (xb >= x0 && on) {
#pragma unroll
      for (int r = 0; r < R; r++)
        if (y0 + r < K2) out[((long long)r * K1 + xb) * C] = acc[r][0];
    }
#pragma unroll
    for (int r = 0; r < R; r++) {
#pragma unroll
      for (int j = 0; j < 5; j++) acc[r][j] = acc[r][j + 1];
      acc[r][5] = make_float2(0.f, 0.f);
    }
  }
}

// Persistent row sweep: every warp takes 32 / CW teams at a time from the
// plan's work queue (heaviest teams first) until the queue is empty, so warps
// do not sit idle behind a heavy team of their block.  Each team's sums are
// independent of which warp runs it: deterministic.
template <int CW, int R, bool REAL, bool DENSE>
__global__ void __launch_bounds__(256) spread_sweep_kernel(InterpArgs a, Tiling t,
                                                           const int *__restrict__ bin_start,
                                                           const float2 *__restrict__ fs,
                                                           float2 *__restrict__ ck) {
  constexpr int G = 32 / CW;
  const int lane = threadIdx.x & 31;
  const long long nteam =
      t.sweep < 0 ? (long long)t.nteams
                  : (long long)t.nslice * ((a.g.K[1] + R - 1) / R) * t.sweep;
  for (;;) {
    int base = 0;
    if (lane == 0) base = atomicAdd(t.team_next + blockIdx.y, G);  // queue of this coil chunk
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= nteam) break;
    const long long qi = (long long)base + lane / CW;
    if (qi < nteam) {
      const long long team = t.team_order ? (long long)__ldg(t.team_order + qi) : qi;
      sweep_team<CW, R, REAL, DENSE>(a, t, bin_start, fs, ck, team);
    }
  }
}

// Dense-bin patches for the sweeps (J = 6, D = 2 or 3), in two launches.
// dense_part_kernel: block i takes chunk i of a dense bin (up to DP_CH of its
// samples, plan order, already times conj(phase) in fs), copies their tap
// records and sample rows into shared memory and sums them, one thread per
// row (j3, j2, c) of six j1 taps, in the sweeps' per-sample operation order
// and the samples' sort order, into patch_part[i].  dense_reduce_kernel:
// block d adds its bin's chunk sums in chunk order into patch[d].
constexpr int DP_CH = 64;
template <int D, bool REAL>
__global__ void __launch_bounds__(256) dense_part_kernel(InterpArgs a, Tiling t,
                                                         const float2 *__restrict__ fs) {
  constexpr int NR = D == 3 ? 36 : 6;  // (j3, j2) rows of a patch
  constexpr int SJ = D == 3 ? 18 : 12;
  extern __shared__ __align__(16) float2 dsm[];
  const int4 ch = t.dense_chunk[t.chunk0 + blockIdx.x];  // (dense bin, p0, p1, part)
  const int n = ch.z - ch.y;
  const int C = a.C;
  float2 *sw = dsm;                 // [DP_CH][SJ]
  float2 *sf = dsm + DP_CH * SJ;    // [DP_CH][C]
  for (int e = threadIdx.x; e < n * SJ; e += blockDim.x) sw[e] = __ldg(a.W + (long long)ch.y * SJ + e);
  for (int e = threadIdx.x; e < n * C; e += blockDim.x) sf[e] = __ldg(fs + (long long)ch.y * C + e);
  __syncthreads();
  float2 *out = t.patch_part + (long long)ch.w * NR * 6 * C;
  for (int row = threadIdx.x; row < NR * C; row += blockDim.x) {
    const int c = row % C, jr = row / C;
    const int j2 = jr % 6, j3 = jr / 6;
    float2 acc[6];
#pragma unroll
    for (int j = 0; j < 6; j++) acc[j] = make_float2(0.f, 0.f);
    for (int q = 0; q < n; q++) {
      const float2 *w = sw + q * SJ;
      float2 v = sf[q * C + c];
      if (D == 3) v = cw_mul<REAL>(w[12 + j3], v);
      v = cw_mul<REAL>(w[6 + j2], v);
#pragma unroll
      for (int j = 0; j < 6; j++) cmac_conj<REAL>(acc[j], w[j], v);
    }
#pragma unroll
    for (int j = 0; j < 6; j++) out[((long long)jr * 6 + j) * C + c] = acc[j];
  }
}

template <int D>
__global__ void __launch_bounds__(256) dense_reduce_kernel(InterpArgs a, Tiling t) {
  constexpr int NP = D == 3 ? 216 : 36;
  const int d = t.dense0 + blockIdx.x;
  const int q0 = __ldg(t.dense_part0 + d), q1 = __ldg(t.dense_part0 + d + 1);
  const long long pn = (long long)NP * a.C;
  float2 *out = t.patch + (long long)d * pn;
  for (long long e = threadIdx.x; e < pn; e += blockDim.x) {
    const float2 *src = t.patch_part + e;
    float2 v = src[(long long)q0 * pn];
    int q = q0 + 1;
    // eight chunk partials loaded ahead, added in chunk order (the same sums)
    for (; q + 8 <= q1; q += 8) {
      float2 w[8];
#pragma unroll
      for (int u = 0; u < 8; u++) w[u] = src[(long long)(q + u) * pn];
#pragma unroll
      for (int u = 0; u < 8; u++) {
        v.x += w[u].x;
        v.y += w[u].y;
      }
    }
    for (; q < q1; q++) {
      const float2 w = src[(long long)q * pn];
      v.x += w.x;
      v.y += w.y;
    }
    out[e] = v;
  }
}

// the two launches of the patches of dense bins [dense0, dense0 + ndense)
template <int D, bool REAL>
cudaError_t launch_dense_patches(const InterpArgs &a, const Tiling &t, const float2 *fs,
                                 cudaStream_t st) {
  if (!t.dense_of || t.ndense <= 0 || t.nchunks <= 0) return cudaSuccess;
  constexpr int SJ = D == 3 ? 18 : 12;
  const size_t sm = (size_t)DP_CH * (SJ + a.C) * sizeof(float2);
  auto k1 = dense_part_kernel<D, REAL>;
  cudaError_t e = cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  k1<<<(unsigned)t.nchunks, 256, sm, st>>>(a, t, fs);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  dense_reduce_kernel<D><<<(unsigned)t.ndense, 256, 0, st>>>(a, t);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------
// 3D line sweep (J = 6 in every dimension, one-point bins, K >= 6)
// ------------------------------------------------------------------------
// cp.async copies into this thread's CTA's shared memory, and their wait
__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
// all but the most recent group complete
__device__ __forceinline__ void cp_async_wait_group1() {
  asm volatile("cp.async.wait_group 1;" ::: "memory");
}

constexpr int SW3_CAP = 32;  // visits staged per batch and warp
template <int CW>
constexpr int sweep3_warp_bytes() {
  return 2 * SW3_CAP * 4 + SW3_CAP * 18 * 8 + SW3_CAP * CW * 8;
}

// A warp owns a block of B2 x B3 grid lines along k1 (rows y0 .. y0 + B2 - 1
// of planes z0 .. z0 + B3 - 1; lanes = CW coils x the block's 32 / CW lines:
// 2 x 2 lines for 8 coils, 2 x 1 for 16, one line for 32) and a segment
// [x0, x1) of their columns.  The samples with taps in the block are those
// binned in the Q2 x Q3 = (B2 + 5) x (B3 + 5) bin lines around it; lane l
// keeps the bin pointers of bin lines l and l + 32, and loads those of the
// next column while the current one is summed.  Per bin column the warp
// lists the column's samples (bin lines in index order, samples in sort
// order), copies their tap records and sample rows into its shared-memory
// stage with cp.async (all in flight at once), and then every lane adds each
// sample's six k1 taps into the six-column window of its own line (when the
// line is within the sample's 6 x 6 tap rows), with the same FP32 operation
// order per tap as the tiled spread (conj(w3) f, then conj(w2), then
// conj(w1)).  Dense bins (at least dense_min samples) add their patches after
// the column's samples, in bin-line order.  After bin column x, grid column x
// of every line is complete and is stored once.  The summation order per
// grid point is fixed and independent of the segments: bitwise reproducible.
template <int CW, bool REAL>
__device__ __forceinline__ void sweep3_team(const InterpArgs &a, const Tiling &t,
                                            const int *__restrict__ bin_start,
                                            const float2 *__restrict__ fs,
                                            float2 *__restrict__ ck, long long team,
                                            unsigned char *wsm) {
  constexpr unsigned FULLM = 0xffffffffu;
  constexpr int NL = 32 / CW;             // lines per warp
  constexpr int B2 = NL >= 2 ? 2 : 1;
  constexpr int B3 = NL / B2;
  constexpr int Q2 = B2 + 5, Q3 = B3 + 5, NBL = Q2 * Q3;  // bin lines, at most 49
  static_assert(NBL <= 64, "bin lines must fit two per lane");
  int *spos = reinterpret_cast<int *>(wsm);
  int *slin = spos + SW3_CAP;
  float2 *srec = reinterpret_cast<float2 *>(wsm + 2 * SW3_CAP * 4);
  float2 *sf = srec + SW3_CAP * 18;
  const int K1 = a.g.K[0], K2 = a.g.K[1], K3 = a.g.K[2];
  const int nseg = t.sweep;
  const int nby = (K2 + B2 - 1) / B2, nbz = (K3 + B3 - 1) / B3;
  const int seg = (int)(team % nseg);
  long long rest = team / nseg;
  const int by = (int)(rest % nby);
  rest /= nby;
  const int bz = (int)(rest % nbz);
  const int slice = t.slice0 + (int)(rest / nbz);
  const int y0 = by * B2, z0 = bz * B3;
  const int sw = (K1 + nseg - 1) / nseg;
  const int x0 = seg * sw, x1 = min(K1, x0 + sw);
  if (x0 >= x1) return;
  const int lane = threadIdx.x & 31;
  const int li = lane / CW, cl = lane % CW;
  const int dy = li % B2, dz = li / B2;
  const int C = a.C;
  const int c0 = blockIdx.y * CW;
  const bool on = c0 + cl < C;
  const int *bs = bin_start + (long long)slice * t.nbins;
  const int *dof = t.dense_of ? t.dense_of + (long long)slice * t.nbins : nullptr;
  const int dmin = t.dense_of ? t.dense_min : 0x7fffffff;
  auto line_base = [&](int l) -> long long {
    int r = (y0 - 5 + l % Q2) % K2;
    if (r < 0) r += K2;
    int z = (z0 - 5 + l / Q2) % K3;
    if (z < 0) z += K3;
    return ((long long)z * K2 + r) * K1;
  };
  const long long base0 = lane < NBL ? line_base(lane) : -1;
  const long long base1 = lane + 32 < NBL ? line_base(lane + 32) : -1;
  const int xs = x0 - 5;
  auto wrapx = [&](int x) { return x < 0 ? x + K1 : x; };
  int beg0 = base0 >= 0 ? __ldg(bs + base0 + wrapx(xs)) : 0;
  int beg1 = base1 >= 0 ? __ldg(bs + base1 + wrapx(xs)) : 0;
  // end of each bin line's samples
  const int rend0 = base0 >= 0 ? __ldg(bs + base0 + K1) : 0;
  const int rend1 = base1 >= 0 ? __ldg(bs + base1 + K1) : 0;
  // end pointers of the next column (and the row starts where the sweep wraps)
  int e0n = base0 >= 0 ? __ldg(bs + base0 + wrapx(xs) + 1) : beg0;
  int e1n = base1 >= 0 ? __ldg(bs + base1 + wrapx(xs) + 1) : beg1;
  int r0n = 0, r1n = 0;
  float2 acc[6];
#pragma unroll
  for (int j = 0; j < 6; j++) acc[j] = make_float2(0.f, 0.f);
  const bool out_ok = on && y0 + dy < K2 && z0 + dz < K3;
  float2 *out = ck + (long long)slice * a.grid_elems +
                ((long long)(z0 + dz) * K2 + (y0 + dy)) * K1 * C + c0 + cl;
  for (int xb = xs; xb < x1; xb++) {
    const int end0 = e0n, end1 = e1n;
    if (xb == 0 && xs < 0) {
      beg0 = r0n;
      beg1 = r1n;
    }
    if (xb + 1 < x1) {
      const int xn = wrapx(xb + 1);
      if (base0 >= 0) e0n = __ldg(bs + base0 + xn + 1);
      if (base1 >= 0) e1n = __ldg(bs + base1 + xn + 1);
      if (xb + 1 == 0) {
        if (base0 >= 0) r0n = __ldg(bs + base0);
        if (base1 >= 0) r1n = __ldg(bs + base1);
      }
    }
    const int n0 = end0 - beg0, n1 = end1 - beg1;
    const int s0 = n0 >= dmin ? 0 : n0, s1 = n1 >= dmin ? 0 : n1;
    // the column's sparse samples: line 0 .. 31, then 32 .. 48, in lane order
    int i0 = s0, i1 = s1;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u0 = __shfl_up_sync(FULLM, i0, o), u1 = __shfl_up_sync(FULLM, i1, o);
      if (lane >= o) {
        i0 += u0;
        i1 += u1;
      }
    }
    const int tot0 = __shfl_sync(FULLM, i0, 31);
    const int V = tot0 + __shfl_sync(FULLM, i1, 31);
    const int ex0 = i0 - s0, ex1 = tot0 + i1 - s1;
    for (int vb = 0; vb < V; vb += SW3_CAP) {
      const int nb = min(SW3_CAP, V - vb);
      for (int k = max(0, vb - ex0); k < s0 && ex0 + k < vb + SW3_CAP; k++) {
        spos[ex0 + k - vb] = beg0 + k;
        slin[ex0 + k - vb] = lane;
      }
      for (int k = max(0, vb - ex1); k < s1 && ex1 + k < vb + SW3_CAP; k++) {
        spos[ex1 + k - vb] = beg1 + k;
        slin[ex1 + k - vb] = lane + 32;
      }
      __syncwarp();
      for (int ch = lane; ch < nb * 9; ch += 32) {
        const int v = ch / 9, k = ch - 9 * v;
        cp_async16(srec + v * 18 + 2 * k, a.W + (long long)spos[v] * 18 + 2 * k);
      }
      for (int ch = lane; ch < nb * CW; ch += 32) {
        const int v = ch / CW, k = ch - CW * v;
        if (c0 + k < C)
          cp_async8(sf + v * CW + k, fs + (long long)spos[v] * C + c0 + k);
        else
          sf[v * CW + k] = make_float2(0.f, 0.f);
      }
      cp_async_wait_all();
      __syncwarp();
      for (int v = 0; v < nb; v++) {
        const int L = slin[v];
        const int j2 = dy - L % Q2 + 5, j3 = dz - L / Q2 + 5;
        if (j2 >= 0 && j2 < 6 && j3 >= 0 && j3 < 6) {
          const float2 *rv = srec + v * 18;
          const float2 v3 = cw_mul<REAL>(rv[12 + j3], sf[v * CW + cl]);
          const float2 vv = cw_mul<REAL>(rv[6 + j2], v3);
#pragma unroll
          for (int j = 0; j < 6; j++) cmac_conj<REAL>(acc[j], rv[j], vv);
        }
      }
      __syncwarp();  // the stage is read before the next batch refills it
    }
    // dense bins: their patches, in bin-line order
    unsigned md0 = __ballot_sync(FULLM, n0 >= dmin && n0 > 0);
    unsigned md1 = __ballot_sync(FULLM, n1 >= dmin && n1 > 0);
    const bool had_dense = (md0 | md1) != 0;
    while (md0 | md1) {
      int L;
      long long bb;
      if (md0) {
        L = __ffs(md0) - 1;
        md0 &= md0 - 1;
        bb = __shfl_sync(FULLM, base0, L);
      } else {
        const int l = __ffs(md1) - 1;
        md1 &= md1 - 1;
        bb = __shfl_sync(FULLM, base1, l);
        L = l + 32;
      }
      const int dn = __ldg(dof + bb + wrapx(xb));
      const int j2 = dy - L % Q2 + 5, j3 = dz - L / Q2 + 5;
      if (on && j2 >= 0 && j2 < 6 && j3 >= 0 && j3 < 6) {
        const float2 *pp = t.patch + ((long long)dn * 216 + (j3 * 6 + j2) * 6) * C + c0 + cl;
#pragma unroll
        for (int j = 0; j < 6; j++) {
          const float2 v = __ldg(pp + (long long)j * C);
          acc[j].x += v.x;
          acc[j].y += v.y;
        }
      }
    }
    beg0 = end0;
    beg1 = end1;
    if (xb >= x0 && out_ok) out[(long long)xb * C] = acc[0];
#pragma unroll
    for (int j = 0; j < 5; j++) acc[j] = acc[j + 1];
    acc[5] = make_float2(0.f, 0.f);
    // skip-ahead: after a column with no sample, jump to the next column in
    // which any of the bin lines holds one (the first tap column of each
    // line's next sample); the columns in between receive nothing
    if (V == 0 && !had_dense && xb >= 0 && xb + 1 < x1) {
      const int nc0 = beg0 < rend0 ? __ldg(&a.K0[beg0].x) : x1;
      const int nc1 = beg1 < rend1 ? __ldg(&a.K0[beg1].x) : x1;
      const int xn = min(__reduce_min_sync(FULLM, min(nc0, nc1)), x1);
      if (xn > xb + 1) {
        int x = xb + 1;
        for (int k = 0; k < 6 && x < xn; k++, x++) {
          if (x >= x0 && out_ok) out[(long long)x * C] = acc[0];
#pragma unroll
          for (int j = 0; j < 5; j++) acc[j] = acc[j + 1];
          acc[5] = make_float2(0.f, 0.f);
        }
        for (; x < xn; x++)
          if (x >= x0 && out_ok) out[(long long)x * C] = make_float2(0.f, 0.f);
        xb = xn - 1;  // the loop moves on to column xn
        if (xn < x1) {
          if (base0 >= 0) e0n = __ldg(bs + base0 + xn + 1);
          if (base1 >= 0) e1n = __ldg(bs + base1 + xn + 1);
        }
      }
    }
  }
}

// Persistent 3D line sweep over the plan's heaviest-first work queue (one
// counter per coil chunk); a warp is one team, with its own shared-memory stage.
template <int CW, bool REAL>
__global__ void __launch_bounds__(256) spread_sweep3_kernel(InterpArgs a, Tiling t,
                                                            const int *__restrict__ bin_start,
                                                            const float2 *__restrict__ fs,
                                                            float2 *__restrict__ ck) {
  extern __shared__ __align__(16) unsigned char sm3[];
  constexpr int NL = 32 / CW;
  constexpr int B2 = NL >= 2 ? 2 : 1;
  constexpr int B3 = NL / B2;
  const int lane = threadIdx.x & 31;
  unsigned char *wsm = sm3 + (threadIdx.x >> 5) * sweep3_warp_bytes<CW>();
  const long long nteam = (long long)t.nslice * ((a.g.K[1] + B2 - 1) / B2) *
                          ((a.g.K[2] + B3 - 1) / B3) * t.sweep;
  for (;;) {
    int qi = 0;
    if (lane == 0) qi = atomicAdd(t.team_next + blockIdx.y, 1);
    qi = __shfl_sync(0xffffffffu, qi, 0);
    if (qi >= nteam) break;
    const long long team = t.team_order ? (long long)__ldg(t.team_order + qi) : qi;
    sweep3_team<CW, REAL>(a, t, bin_start, fs, ck, team, wsm);
  }
}

// ------------------------------------------------------------------------
// 2D row sweep with per-column staging (J = 6, one-point bins, 32-coil chunks)
// ------------------------------------------------------------------------
// The team of spread_sweep_kernel (one warp, lane = coil; R grid rows, a
// segment of their columns), with the samples of each bin column staged in the
// warp's shared memory by cp.async, three columns in flight: while column xb
// is summed, the sample rows of column xb + 1 and the tap records of column
// xb + 2 are on their way.  Per column, lane q < R + 5 holds the bounds of bin
// row q (the next column's end loaded a column ahead); the warp lists the
// column's samples (bin rows in order, samples in sort order; the first
// SW2_CAP of them staged ahead, the rest of a crowded column staged when it is
// summed).  DIRECT: the sample rows are read in the caller's order through perm
// (staged with the records) and times conj(phase) here, so the ordering pass
// is not needed.  Same operations in the same order as spread_sweep_kernel:
// the same bits.
constexpr int SW2_CAP = 16;
// one column's list: positions, caller rows, phases; lane bounds
struct Sw2Meta {
  int pos[SW2_CAP];
  int row[SW2_CAP];
  float2 ph[SW2_CAP];
  int beg[16], ex[16];
};
// per warp: three lists, two blocks of tap records (9 float4 per visit) and
// two blocks of sample rows
template <bool DIRECT>
constexpr int sweep2_warp_bytes() {
  return 3 * (int)sizeof(Sw2Meta) + 2 * SW2_CAP * 9 * 16 + 2 * SW2_CAP * 32 * 8;
}

template <int R, bool REAL, bool DIRECT>
__device__ __forceinline__ void sweep2s_team(const InterpArgs &a, const Tiling &t,
                                             const int *__restrict__ bin_start,
                                             const float2 *__restrict__ fs,
                                             float2 *__restrict__ ck, long long team,
                                             unsigned char *wsm) {
  constexpr unsigned FULLM = 0xffffffffu;
  constexpr int NQ = R + 5;
  Sw2Meta *meta = reinterpret_cast<Sw2Meta *>(wsm);
  float4 *srec = reinterpret_cast<float4 *>(wsm + 3 * sizeof(Sw2Meta));
  float2 *sf = reinterpret_cast<float2 *>(srec + 2 * SW2_CAP * 9);
  const int K1 = a.g.K[0], K2 = a.g.K[1];
  int slice, y0, x0, x1;
  if (t.sweep < 0) {
    const int4 tk = t.sweep_team[team];
    slice = tk.x;
    y0 = tk.y;
    x0 = tk.z;
    x1 = tk.w;
  } else {
    const int nseg = t.sweep;
    const int nband = (K2 + R - 1) / R;
    const int seg = (int)(team % nseg);
    const long long bandid = team / nseg;
    const int sl = (int)(bandid / nband);
    y0 = (int)(bandid - (long long)sl * nband) * R;
    slice = t.slice0 + sl;
    const int sw = (K1 + nseg - 1) / nseg;
    x0 = seg * sw;
    x1 = min(K1, x0 + sw);
  }
  if (x0 >= x1) return;
  const int lane = threadIdx.x & 31;
  const int C = a.C;
  const int c0 = blockIdx.y * 32;
  const bool on = c0 + lane < C;
  const int *bs = bin_start + (long long)slice * t.nbins;
  long long rowb = -1;
  if (lane < NQ) {
    int b = (y0 - 5 + lane) % K2;
    if (b < 0) b += K2;
    rowb = (long long)b * K1;
  }
  const int xs = x0 - 5;
  auto wrapx = [&](int x) { return x < 0 ? x + K1 : x; };
  // lane bounds of the next column to list: start lb, end le (loaded ahead)
  int lb = rowb >= 0 ? __ldg(bs + rowb + wrapx(xs)) : 0;
  int le = rowb >= 0 ? __ldg(bs + rowb + wrapx(xs) + 1) : lb;
  int rn = 0;
  // caller rows and phases of the listed visits [0, nb) (DIRECT)
  auto issue_meta = [&](Sw2Meta &m, int nb) {
    if (DIRECT && lane < nb) {
      const int p = m.pos[lane];
      if (a.perm)
        cp_async4(&m.row[lane], a.perm + p);
      else
        m.row[lane] = p;
      if (a.phase) cp_async8(&m.ph[lane], a.phase + p);
    }
  };
  // tap records (9 x 16 bytes each) and sample rows of the listed visits [0, nb)
  auto issue_data = [&](const Sw2Meta &m, float4 *rec, float2 *f, int nb) {
    for (int ch = lane; ch < nb * 9; ch += 32) {
      const int v = ch / 9, k = ch - 9 * v;
      cp_async16(rec + ch, t.wsw + (long long)m.pos[v] * 9 + k);
    }
    for (int v = 0; v < nb; v++) {
      const long long row = DIRECT ? (long long)m.row[v] : (long long)m.pos[v];
      if (on)
        cp_async8(f + v * 32 + lane, fs + row * C + c0 + lane);
      else
        f[v * 32 + lane] = make_float2(0.f, 0.f);
    }
  };
  // list visits [vb, vb + SW2_CAP) of a column from the lanes' bounds
  auto list_part = [&](Sw2Meta &m, int beg, int n, int ex, int vb) {
    for (int k = max(0, vb - ex); k < n && ex + k < vb + SW2_CAP; k++) m.pos[ex + k - vb] = beg + k;
  };
  // list column xc into list slot m and issue its caller rows and phases;
  // returns its visits
  auto list_col = [&](int xc, Sw2Meta &m) -> int {
    const int end = le;
    if (xc == 0 && xs < 0) lb = rn;
    if (xc + 1 < x1 && rowb >= 0) {
      le = __ldg(bs + rowb + wrapx(xc + 1) + 1);
      if (xc + 1 == 0) rn = __ldg(bs + rowb);
    }
    const int n = end - lb;
    int inc = n;
#pragma unroll
    for (int o = 1; o < 16; o <<= 1) {
      const int u = __shfl_up_sync(FULLM, inc, o);
      if (lane >= o) inc += u;
    }
    const int V = __shfl_sync(FULLM, inc, 15);
    if (lane < 16) {
      m.beg[lane] = lb;
      m.ex[lane] = inc - n;
    }
    list_part(m, lb, n, inc - n, 0);
    lb = end;
    __syncwarp();
    issue_meta(m, min(V, SW2_CAP));
    cp_async_commit();
    return V;
  };
  // accumulators of grid columns xb .. xb + 5 (slot j: column xb + j)
  float2 acc[R][6];
#pragma unroll
  for (int r = 0; r < R; r++)
#pragma unroll
    for (int j = 0; j < 6; j++) acc[r][j] = make_float2(0.f, 0.f);
  // staged visits [vb, vb + nb) of the column; bin row q's visits are
  // [ex[q], ex[q + 1]), each reaching band rows r = q - 5 .. q.  The records'
  // operand pairs (wr, wr) and (wi, -wi) feed cw_fma's two FFMA2 directly.
  auto sum_chunk = [&](const Sw2Meta &m, const int *exq, const float4 *rec, const float2 *f,
                       int vb, int nb) {
    sfor<NQ>([&](auto QQ) {
      constexpr int Q = decltype(QQ)::value;
      const int lo = max(exq[Q] - vb, 0), hi = min(exq[Q + 1] - vb, nb);
      for (int v = lo; v < hi; v++) {
        float2 fv = f[v * 32 + lane];
        if (DIRECT && a.phase) fv = cmulc(m.ph[v], fv);
        const float4 *r4 = rec + v * 9;
        float4 wp[6];
#pragma unroll
        for (int j = 0; j < 6; j++) wp[j] = r4[j];
        sfor<R>([&](auto RR) {
          constexpr int r = decltype(RR)::value;
          constexpr int j2 = r - Q + 5;
          if constexpr (j2 >= 0 && j2 < 6) {
            const float4 w2p = r4[6 + j2 / 2];
            const float2 w2 = (j2 & 1) ? make_float2(w2p.z, w2p.w) : make_float2(w2p.x, w2p.y);
            const float2 vv = cw_mul<REAL>(w2, fv);
            const float2 vsw = make_float2(vv.y, vv.x);
            sfor<6>([&](auto JJ) {
              constexpr int j = decltype(JJ)::value;
              float2 A = __ffma2_rn(make_float2(wp[j].x, wp[j].y), vv, acc[r][j]);
              if (!REAL) A = __ffma2_rn(make_float2(wp[j].z, wp[j].w), vsw, A);
              acc[r][j] = A;
            });
          }
        });
      }
    });
  };
  float2 *out = ck + (long long)slice * a.grid_elems + (long long)y0 * K1 * C + c0 + lane;
  // prologue: lists of the first two columns, records and rows of the first
  int Vc = list_col(xs, meta[0]);
  int Vn = list_col(xs + 1, meta[1]);
  cp_async_wait_group1();
  __syncwarp();
  issue_data(meta[0], srec, sf, min(Vc, SW2_CAP));
  cp_async_commit();
  int sc = 0, fb = 0;  // list slot (of 3) and data block (of 2) of the column being summed
  for (int xb = xs; xb < x1; xb++) {
    const int s1 = sc == 2 ? 0 : sc + 1, s2 = sc == 0 ? 2 : sc - 1;
    int Vnn = 0;
    if (xb + 2 < x1)
      Vnn = list_col(xb + 2, meta[s2]);
    else
      cp_async_commit();
    cp_async_wait_group1();  // list of xb + 1, records and rows of xb
    __syncwarp();
    if (xb + 1 < x1)
      issue_data(meta[s1], srec + (1 - fb) * SW2_CAP * 9, sf + (1 - fb) * SW2_CAP * 32,
                 min(Vn, SW2_CAP));
    cp_async_commit();
    Sw2Meta &m = meta[sc];
    float4 *rec = srec + fb * SW2_CAP * 9;
    float2 *f = sf + fb * SW2_CAP * 32;
    int exq[NQ + 1];
#pragma unroll
    for (int q = 0; q <= NQ; q++) exq[q] = m.ex[q];
    // the first SW2_CAP visits are staged; the rest of a crowded column is
    // staged here, SW2_CAP at a time
    for (int vb = 0; vb < Vc; vb += SW2_CAP) {
      const int nb = min(SW2_CAP, Vc - vb);
      if (vb > 0) {
        int beg = 0, ex = 0;
        if (lane < 16) {
          beg = m.beg[lane];
          ex = m.ex[lane];
        }
        const int exn = __shfl_down_sync(FULLM, ex, 1);
        const int n = lane < 15 ? exn - ex : 0;
        __syncwarp();
        list_part(m, beg, n, ex, vb);
        __syncwarp();
        issue_meta(m, nb);
        cp_async_commit();
        cp_async_wait_all();
        __syncwarp();
        issue_data(m, rec, f, nb);
        cp_async_commit();
        cp_async_wait_all();
        __syncwarp();
      }
      sum_chunk(m, exq, rec, f, vb, nb);
      __syncwarp();
    }
    // grid column xb is complete
    if (xb >= x0 && on) {
#pragma unroll
      for (int r = 0; r < R; r++)
        if (y0 + r < K2) out[((long long)r * K1 + xb) * C] = acc[r][0];
    }
#pragma unroll
    for (int r = 0; r < R; r++) {
#pragma unroll
      for (int j = 0; j < 5; j++) acc[r][j] = acc[r][j + 1];
      acc[r][5] = make_float2(0.f, 0.f);
    }
    __syncwarp();  // list slot sc is listed again two columns on, data block fb one column on
    Vc = Vn;
    Vn = Vnn;
    sc = s1;
    fb ^= 1;
  }
  cp_async_wait_all();
  __syncwarp();
}

template <int R, bool REAL, bool DIRECT>
__global__ void __launch_bounds__(256) spread_sweep2s_kernel(InterpArgs a, Tiling t,
                                                             const int *__restrict__ bin_start,
                                                             const float2 *__restrict__ fs,
                                                             float2 *__restrict__ ck) {
  extern __shared__ __align__(16) unsigned char sm2[];
  const int lane = threadIdx.x & 31;
  unsigned char *wsm = sm2 + (threadIdx.x >> 5) * sweep2_warp_bytes<DIRECT>();
  const long long nteam =
      t.sweep < 0 ? (long long)t.nteams
                  : (long long)t.nslice * ((a.g.K[1] + R - 1) / R) * t.sweep;
  for (;;) {
    int qi = 0;
    if (lane == 0) qi = atomicAdd(t.team_next + blockIdx.y, 1);
    qi = __shfl_sync(0xffffffffu, qi, 0);
    if (qi >= nteam) break;
    const long long team = t.team_order ? (long long)__ldg(t.team_order + qi) : qi;
    sweep2s_team<R, REAL, DIRECT>(a, t, bin_start, fs, ck, team, wsm);
  }
}

// Sum the partial tiles of each split heavy tile, in slot order, into the grid.
template <int D, int CW>
__global__ void __launch_bounds__(256) spread_reduce_kernel(InterpArgs a, Tiling t,
                                                            float2 *__restrict__ ck) {
  const int4 it = t.red[blockIdx.x];
  const int task = it.x, first = it.y, nparts = it.z;
  const int tile = task % t.ntiles;
  const int slice = task / t.ntiles;
  const Geom &g = a.g;
  int npts = 1;
  int lo[MIRT_DMAX] = {0, 0, 0}, ext[MIRT_DMAX] = {1, 1, 1};
  {
    int r = tile;
#pragma unroll
    for (int d = 0; d < D; d++) {
      const int bd = r % t.nb[d];
      r /= t.nb[d];
      lo[d] = bd * t.T[d];
      ext[d] = min(t.T[d], g.K[d] - lo[d]);
      npts *= t.T[d];
    }
  }
  const int T0 = t.T[0];
  const int T1 = D > 1 ? t.T[1] : 1;
  const int c0 = blockIdx.y * CW;
  const size_t stride = (size_t)gridDim.y * npts * CW;
  const float2 *part = t.scratch + ((size_t)first * gridDim.y + blockIdx.y) * npts * CW;
  float2 *gout = ck + (long long)slice * a.grid_elems;
  for (int e = threadIdx.x; e < npts * CW; e += blockDim.x) {
    const int pt = e / CW, cc = e - pt * CW;
    const int l1 = pt % T0;
    const int l2 = D > 1 ? (pt / T0) % T1 : 0;
    const int l3 = D > 2 ? pt / (T0 * T1) : 0;
    if (l1 >= ext[0] || l2 >= ext[1] || l3 >= ext[2] || c0 + cc >= a.C) continue;
    float2 v = part[e];
    for (int p = 1; p < nparts; p++) {
      const float2 w = part[p * stride + e];
      v.x += w.x;
      v.y += w.y;
    }
    long long kk = lo[0] + l1;
    if (D > 1) kk += (long long)(lo[1] + l2) * g.kstride[1];
    if (D > 2) kk += (long long)(lo[2] + l3) * g.kstride[2];
    gout[kk * a.C + c0 + cc] = v;
  }
}

// ------------------------------------------------------------------------
// ownership spread (2D, J = 6)
// ------------------------------------------------------------------------
// A CTA takes the samples whose wrapped first tap lies in its tile (rows of
// the tile: one contiguous range of the one-point sort each) and adds all 36
// taps into a shared tile of (T0 + 5) x (T1 + 5) points -- no bounds tests,
// no wrap tests.  Warps own bands of padded rows (a sample is skipped by the
// warps whose band its six rows miss).  The padded tile is then added into
// the grid (periodic wrap) or, for a split heavy tile, written as a partial.
// Within one launch (one colour) no two padded tiles overlap, so the adds
// need no atomics; colours run in a fixed order: deterministic.
// grid[(lo + p) mod K] += sum over parts of src[part][p] for the q0 x q1
// points p of a padded tile (src: [P1][P0][CW], parts `pstride` apart);
// U grid values are loaded before any is written back, so a thread keeps U
// independent loads in flight.
template <int CW, int U>
__device__ __forceinline__ void own_add_tile(const float2 *src, int P0, int q0, int q1, int lo0,
                                             int lo1, int c0, int C, int K0, int K1,
                                             float2 *gout, int nparts, size_t pstride) {
  const int n = q0 * q1 * CW;
  for (int e0 = threadIdx.x; e0 < n; e0 += U * blockDim.x) {
    float2 o[U];
    float2 *q[U];
    size_t pe[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int e = e0 + u * blockDim.x;
      q[u] = nullptr;
      if (e < n) {
        const int cc = e % CW, pt = e / CW;
        const int p0 = pt % q0, p1 = pt / q0;
        if (c0 + cc < C) {
          int g0 = lo0 + p0, g1 = lo1 + p1;
          if (g0 >= K0) g0 -= K0;
          if (g1 >= K1) g1 -= K1;
          q[u] = gout + ((long long)g1 * K0 + g0) * C + c0 + cc;
          pe[u] = ((size_t)p1 * P0 + p0) * CW + cc;
          o[u] = *q[u];
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      if (!q[u]) continue;
      for (int p = 0; p < nparts; p++) {
        const float2 v = src[p * pstride + pe[u]];
        o[u].x += v.x;
        o[u].y += v.y;
      }
      *q[u] = o[u];
    }
  }
}

template <int CW, bool REAL>
__global__ void __launch_bounds__(256) spread_own_kernel(InterpArgs a, Tiling t,
                                                         const int *__restrict__ bin_start,
                                                         const float2 *__restrict__ fm,
                                                         float2 *__restrict__ ck, int task0) {
  constexpr int SUB = 32 / CW, JT = 6;
  extern __shared__ __align__(16) unsigned char smem[];
  float2 *acc = reinterpret_cast<float2 *>(smem);
  const Geom &g = a.g;
  const int T0 = t.T[0], T1 = t.T[1];
  const int P0 = T0 + JT - 1, P1 = T1 + JT - 1;
  const int ti = task0 + blockIdx.x;
  const int task = t.task_tile[ti];
  const int2 vr = t.task_range[ti];
  const int slot = t.task_slot[ti];
  const int tile = task % t.ntiles, slice = task / t.ntiles;
  const int bx = tile % t.nb[0], by = tile / t.nb[0];
  const int lo0 = bx * T0, lo1 = by * T1;
  const int ext0 = min(T0, g.K[0] - lo0), ext1 = min(T1, g.K[1] - lo1);
  const int c0 = blockIdx.y * CW;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarp = blockDim.x >> 5;
  const int ls = lane / CW, lc = lane % CW;
  const int per = (P1 + nwarp - 1) / nwarp;
  const int band_lo = min(warp * per, P1), band_hi = min(band_lo + per, P1);
  for (int e = threadIdx.x; e < P0 * P1 * CW; e += blockDim.x) acc[e] = make_float2(0.f, 0.f);
  __syncthreads();
  const int C = a.C;
  const bool lane_on = c0 + lc < C;
  const int SJ = a.SJ;
  long long vbase = 0;
  for (int i1 = 0; i1 < ext1 && vbase < vr.y && band_lo < band_hi; i1++) {
    const int key = slice * t.nbins + (lo1 + i1) * t.nbin[0] + lo0;
    const long long b0 = bin_start[key], b1 = bin_start[key + ext0];
    const long long beg = b0 + max(0ll, (long long)vr.x - vbase);
    const long long end = b0 + min(b1 - b0, (long long)vr.y - vbase);
    vbase += b1 - b0;
    // every sample of this row has l2 = i1: rows l2 .. l2 + 5 of the padded tile
    const int jab = max(0, band_lo - i1), jbb = min(JT, band_hi - i1);
    if (beg >= end || jab >= jbb) continue;
    int4 kn = a.K0[beg];
    int mn = a.perm ? a.perm[beg] : (int)beg;
    for (long long pos = beg; pos < end; pos++) {
      const int4 k = kn;
      const int m = mn;
      if (pos + 1 < end) {
        kn = a.K0[pos + 1];
        mn = a.perm ? a.perm[pos + 1] : (int)(pos + 1);
      }
      const int l1 = k.x - lo0;
      const float2 *Ws = a.W + pos * SJ;
      float2 f = make_float2(0.f, 0.f);
      if (lane_on) {
        f = __ldg(fm + (long long)m * C + c0 + lc);
        if (a.phase) f = cmulc(__ldg(a.phase + pos), f);
      }
      float2 *base = acc + ((size_t)i1 * P0 + l1) * CW + lc;
      if constexpr (SUB == 1) {
        float2 wr[JT], wi[JT];
#pragma unroll
        for (int j1 = 0; j1 < JT; j1++) {
          const float2 w = __ldg(Ws + j1);
          wr[j1] = make_float2(w.x, w.x);
          wi[j1] = make_float2(w.y, -w.y);
        }
        for (int j2 = jab; j2 < jbb; j2++) {
          const float2 v2 = cw_mul<REAL>(__ldg(Ws + JT + j2), f);
          const float2 v2s = make_float2(v2.y, v2.x);
          float2 *p = base + (size_t)j2 * P0 * CW;
#pragma unroll
          for (int j1 = 0; j1 < JT; j1++) {
            float2 A = p[j1 * CW];
            A = __ffma2_rn(wr[j1], v2, A);
            if (!REAL) A = __ffma2_rn(wi[j1], v2s, A);
            p[j1 * CW] = A;
          }
        }
      } else {
        // lane class ls takes the padded columns l1 + j1 = ls (mod SUB)
        const int j1s = (ls - l1) & (SUB - 1);
        for (int j2 = jab; j2 < jbb; j2++) {
          const float2 v2 = cw_mul<REAL>(__ldg(Ws + JT + j2), f);
          const float2 v2s = make_float2(v2.y, v2.x);
          float2 *p = base + (size_t)j2 * P0 * CW;
          for (int j1 = j1s; j1 < JT; j1 += SUB) {
            float2 A = p[j1 * CW];
            A = cw_fma<REAL>(__ldg(Ws + j1), v2, v2s, A);
            p[j1 * CW] = A;
          }
        }
      }
    }
  }
  __syncthreads();
  if (slot >= 0) {
    float2 *part = t.scratch + ((size_t)slot * gridDim.y + blockIdx.y) * P0 * P1 * CW;
    for (int e = threadIdx.x; e < P0 * P1 * CW; e += blockDim.x) part[e] = acc[e];
    return;
  }
  float2 *gout = ck + (long long)slice * a.grid_elems;
  const int q0 = ext0 + JT - 1, q1 = ext1 + JT - 1;
  own_add_tile<CW, 8>(acc, P0, q0, q1, lo0, lo1, c0, C, g.K[0], g.K[1], gout, 1, 0);
}

// Sum the partial padded tiles of each split tile of one colour, in slot
// order, into the grid.
template <int CW>
__global__ void __launch_bounds__(256) spread_own_reduce_kernel(InterpArgs a, Tiling t,
                                                                float2 *__restrict__ ck,
                                                                int red0) {
  constexpr int JT = 6;
  const int4 it = t.red[red0 + blockIdx.x];
  const int task = it.x, first = it.y, nparts = it.z;
  const int tile = task % t.ntiles, slice = task / t.ntiles;
  const Geom &g = a.g;
  const int T0 = t.T[0], T1 = t.T[1];
  const int P0 = T0 + JT - 1, P1 = T1 + JT - 1;
  const int lo0 = (tile % t.nb[0]) * T0, lo1 = (tile / t.nb[0]) * T1;
  const int ext0 = min(T0, g.K[0] - lo0), ext1 = min(T1, g.K[1] - lo1);
  const int c0 = blockIdx.y * CW;
  const size_t stride = (size_t)gridDim.y * P0 * P1 * CW;
  const float2 *part = t.scratch + ((size_t)first * gridDim.y + blockIdx.y) * P0 * P1 * CW;
  float2 *gout = ck + (long long)slice * a.grid_elems;
  const int q0 = ext0 + JT - 1, q1 = ext1 + JT - 1;
  own_add_tile<CW, 4>(part, P0, q0, q1, lo0, lo1, c0, a.C, g.K[0], g.K[1], gout, nparts, stride);
}

// ------------------------------------------------------------------------
// launch dispatch
// ------------------------------------------------------------------------
enum What { GATHER = 0, GATHER_GRID = 1, SPREAD = 2 };

struct Req {
  What what;
  const InterpArgs *a;
  const Tiling *t;
  Launch *l;
  const int *bin_start;
  const float2 *in;
  float2 *out;
  cudaStream_t st;
};

inline size_t spread_smem_bytes(const InterpArgs &a, const Tiling &t, const Launch &l) {
  if (t.own) return (size_t)(t.T[0] + 5) * (t.T[1] + 5) * l.cw * 8;
  size_t npts = a.g.D > 1 ? t.T[0] + 2 * t.padc : t.T[0];
  for (int d = 1; d < a.g.D; d++) npts *= t.T[d];
  return npts * l.cw * 8;
}

template <int D, int CW, int JT, bool REAL, bool CX>
cudaError_t run(Req &r) {
  const InterpArgs &a = *r.a;
  Launch &l = *r.l;
  if (r.what == GATHER || r.what == GATHER_GRID) {
    auto kern = gather_kernel<D, CW, JT, REAL, CX>;
    cudaError_t e = cudaSuccess;
    if (r.what == GATHER_GRID || l.grid <= 0) {
      int per_sm = 0, dev = 0, nsm = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, l.threads, 0);
      if (e != cudaSuccess) return e;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
      const long long groups = (a.Mtot + (l.threads / CW) - 1) / (l.threads / CW);
      long long gsz = (long long)nsm * (per_sm > 0 ? per_sm : 1);
      if (gsz > groups) gsz = groups;
      l.grid = (int)(gsz > 0 ? gsz : 1);
      if (r.what == GATHER_GRID) return cudaSuccess;
    }
    kern<<<l.grid, l.threads, 0, r.st>>>(a, r.in, r.out);
    return cudaGetLastError();
  }
  if constexpr (CX) {
    return cudaErrorInvalidValue;  // the spread has no CX variant
  } else {
    const Tiling &t = *r.t;
    const size_t sm = spread_smem_bytes(a, t, l);
    if constexpr (D == 3 && JT == 6 && (CW == 8 || CW == 16 || CW == 32)) {
      if (t.sweep > 0) {
        const unsigned nchunk = (unsigned)((a.C + CW - 1) / CW);
        if (!t.sorted || !t.team_next) return cudaErrorInvalidValue;
        if (a.Mtot > 0) {
          const long long p0 = t.npos < 0 ? 0 : t.pos0;
          const long long np = t.npos < 0 ? a.Mtot : t.npos;
          const long long n = np * (long long)a.C;
          long long nb = (n + 255) / 256;
          if (nb > 148 * 16) nb = 148 * 16;
          if (n > 0)
            sweep_order_kernel<CW><<<(unsigned)nb, 256, 0, r.st>>>(a, r.in, t.sorted, p0, np);
          cudaError_t e = cudaGetLastError();
          if (e != cudaSuccess) return e;
        }
        {
          cudaError_t e = launch_dense_patches<3, REAL>(a, t, t.sorted, r.st);
          if (e != cudaSuccess) return e;
        }
        auto kern = spread_sweep3_kernel<CW, REAL>;
        const size_t smem3 = 8 * (size_t)sweep3_warp_bytes<CW>();
        int per_sm = 0, dev = 0, nsm = 0;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem3);
        if (e != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, smem3);
        if (e != cudaSuccess) return e;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        constexpr int NL = 32 / CW, B2 = NL >= 2 ? 2 : 1, B3 = NL / B2;
        const long long teams = (long long)t.nslice * ((a.g.K[1] + B2 - 1) / B2) *
                                ((a.g.K[2] + B3 - 1) / B3) * t.sweep;
        long long nb = (long long)nsm * (per_sm > 0 ? per_sm : 1);
        if (nb > (teams + 7) / 8) nb = (teams + 7) / 8;
        if (nb < 1) nb = 1;
        e = cudaMemsetAsync(t.team_next, 0, nchunk * sizeof(int), r.st);
        if (e != cudaSuccess) return e;
        kern<<<dim3((unsigned)nb, nchunk), 256, smem3, r.st>>>(a, t, r.bin_start, t.sorted, r.out);
        return cudaGetLastError();
      }
    }
    if constexpr (D == 2 && JT == 6) {
      if (t.sweep != 0) {
        const long long nband = (a.g.K[1] + t.sweep_rows - 1) / max(t.sweep_rows, 1);
        const long long teams =
            t.sweep < 0 ? t.nteams : (long long)t.nslice * nband * t.sweep;
        const long long thr = teams * CW;
        const unsigned nchunk = (unsigned)((a.C + CW - 1) / CW);
        if (thr == 0) return cudaSuccess;
        if (t.sweep_staged && CW == 32 && !(t.dense_on && t.dense_of && t.sweep_rows == 1)) {
          // staged sweep: reads the plan-order copy (1) or the caller's samples (2)
          if (!t.wsw) return cudaErrorInvalidValue;
          const bool direct = t.sweep_staged == 2;
          if (!direct) {
            if (!t.sorted) return cudaErrorInvalidValue;
            const long long p0 = t.npos < 0 ? 0 : t.pos0;
            const long long np = t.npos < 0 ? a.Mtot : t.npos;
            const long long n = np * (long long)a.C;
            long long nb = (n + 255) / 256;
            if (nb > 148 * 16) nb = 148 * 16;
            if (n > 0)
              sweep_order_kernel<CW><<<(unsigned)nb, 256, 0, r.st>>>(a, r.in, t.sorted, p0, np);
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return e;
          }
          if (!t.team_next) return cudaErrorInvalidValue;
          const float2 *fsrc = direct ? r.in : t.sorted;
          auto go2 = [&](auto kern, size_t smem) -> cudaError_t {
            int per_sm = 0, dev = 0, nsm = 0;
            cudaError_t e =
                cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, smem);
            if (e != cudaSuccess) return e;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
            long long nb = (long long)nsm * (per_sm > 0 ? per_sm : 1);
            const long long need = (teams + 7) / 8;
            if (nb > need) nb = need;
            e = cudaMemsetAsync(t.team_next, 0, nchunk * sizeof(int), r.st);
            if (e != cudaSuccess) return e;
            kern<<<dim3((unsigned)nb, nchunk), 256, smem, r.st>>>(a, t, r.bin_start, fsrc, r.out);
            return cudaGetLastError();
          };
          const size_t smd = 8 * (size_t)sweep2_warp_bytes<true>();
          const size_t sms = 8 * (size_t)sweep2_warp_bytes<false>();
          switch (t.sweep_rows) {
            case 1: return direct ? go2(spread_sweep2s_kernel<1, REAL, true>, smd)
                                  : go2(spread_sweep2s_kernel<1, REAL, false>, sms);
            case 2: return direct ? go2(spread_sweep2s_kernel<2, REAL, true>, smd)
                                  : go2(spread_sweep2s_kernel<2, REAL, false>, sms);
            case 4: return direct ? go2(spread_sweep2s_kernel<4, REAL, true>, smd)
                                  : go2(spread_sweep2s_kernel<4, REAL, false>, sms);
            default: return cudaErrorInvalidValue;
          }
        }
        if (!t.sorted) return cudaErrorInvalidValue;
        {
          const long long p0 = t.npos < 0 ? 0 : t.pos0;
          const long long np = t.npos < 0 ? a.Mtot : t.npos;
          const long long n = np * (long long)a.C;
          long long nb = (n + 255) / 256;
          if (nb > 148 * 16) nb = 148 * 16;
          if (n > 0)
            sweep_order_kernel<CW><<<(unsigned)nb, 256, 0, r.st>>>(a, r.in, t.sorted, p0, np);
          cudaError_t e = cudaGetLastError();
          if (e != cudaSuccess) return e;
        }
        if (!t.team_next) return cudaErrorInvalidValue;
        const float2 *fs = t.sorted;
        auto go = [&](auto kern) -> cudaError_t {
          // persistent: the blocks that fit on the GPU at once (per coil chunk)
          int per_sm = 0, dev = 0, nsm = 0;
          cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0);
          if (e != cudaSuccess) return e;
          cudaGetDevice(&dev);
          cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
          long long nb = (long long)nsm * (per_sm > 0 ? per_sm : 1);
          const long long need = (thr + 255) / 256;
          if (nb > need) nb = need;
          e = cudaMemsetAsync(t.team_next, 0, nchunk * sizeof(int), r.st);
          if (e != cudaSuccess) return e;
          kern<<<dim3((unsigned)nb, nchunk), 256, 0, r.st>>>(a, t, r.bin_start, fs, r.out);
          return cudaGetLastError();
        };
        if (t.dense_on && t.dense_of && t.sweep_rows == 1) {
          // one-row bands with dense-bin patches
          cudaError_t e = launch_dense_patches<2, REAL>(a, t, t.sorted, r.st);
          if (e != cudaSuccess) return e;
          return go(spread_sweep_kernel<CW, 1, REAL, true>);
        }
        switch (t.sweep_rows) {
          case 1: return go(spread_sweep_kernel<CW, 1, REAL, false>);
          case 2: return go(spread_sweep_kernel<CW, 2, REAL, false>);
          case 4: return go(spread_sweep_kernel<CW, 4, REAL, false>);
          default: return cudaErrorInvalidValue;
        }
      }
      if (t.own) {
        // cleared grid, then one launch (and one reduction) per colour
        auto kern = spread_own_kernel<CW, REAL>;
        cudaError_t e =
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        e = cudaMemsetAsync(r.out, 0, (size_t)t.nslice * a.grid_elems * sizeof(float2), r.st);
        if (e != cudaSuccess) return e;
        const unsigned nchunk = (unsigned)((a.C + CW - 1) / CW);
        for (int c = 0; c < 4; c++) {
          const int n = t.color_beg[c + 1] - t.color_beg[c];
          if (n > 0) {
            kern<<<dim3((unsigned)n, nchunk), l.threads, sm, r.st>>>(a, t, r.bin_start, r.in, r.out,
                                                                    t.color_beg[c]);
            e = cudaGetLastError();
            if (e != cudaSuccess) return e;
          }
          const int nr = t.red_beg[c + 1] - t.red_beg[c];
          if (nr > 0) {
            spread_own_reduce_kernel<CW><<<dim3((unsigned)nr, nchunk), 256, 0, r.st>>>(
                a, t, r.out, t.red_beg[c]);
            e = cudaGetLastError();
            if (e != cudaSuccess) return e;
          }
        }
        return cudaSuccess;
      }
    }
    auto kern = l.atomic ? spread_kernel<D, CW, JT, REAL, true> : spread_kernel<D, CW, JT, REAL, false>;
    cudaError_t e =
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    const unsigned nchunk = (unsigned)((a.C + CW - 1) / CW);
    if (t.ntask > 0) {
      kern<<<dim3((unsigned)t.ntask, nchunk), l.threads, sm, r.st>>>(a, t, r.bin_start, r.in,
                                                                     r.out);
      e = cudaGetLastError();
      if (e != cudaSuccess) return e;
    }
    if (t.nred > 0) {
      spread_reduce_kernel<D, CW><<<dim3((unsigned)t.nred, nchunk), 256, 0, r.st>>>(a, t, r.out);
      e = cudaGetLastError();
    }
    return e;
  }
}

template <int D, int CW, int JT, bool REAL>
cudaError_t by_cx(Req &r) {
  if ((r.what == GATHER || r.what == GATHER_GRID) && JT > 0 && r.a->C == CW)
    return run<D, CW, JT, REAL, true>(r);
  return run<D, CW, JT, REAL, false>(r);
}

template <int D, int CW, int JT>
cudaError_t by_real(Req &r) {
  return r.a->real_tab ? by_cx<D, CW, JT, true>(r) : by_cx<D, CW, JT, false>(r);
}

inline bool all_j(const Geom &g, int j) {
  for (int d = 0; d < g.D; d++)
    if (g.J[d] != j) return false;
  return true;
}

template <int D, int CW>
cudaError_t by_j(Req &r) {
  if (all_j(r.a->g, 6)) return by_real<D, CW, 6>(r);
  return by_real<D, CW, 0>(r);
}

template <int D>
cudaError_t by_cw(Req &r) {
  switch (r.l->cw) {
    case 1: return by_j<D, 1>(r);
    case 4: return by_j<D, 4>(r);
    case 8: return by_j<D, 8>(r);
    case 16: return by_j<D, 16>(r);
    case 32: return by_j<D, 32>(r);
    default: return cudaErrorInvalidValue;
  }
}

// one per dimension, each in its own translation unit
cudaError_t dispatch_d1(Req &r);
cudaError_t dispatch_d2(Req &r);
cudaError_t dispatch_d3(Req &r);

}  // namespace detail
}  // namespace mirt
