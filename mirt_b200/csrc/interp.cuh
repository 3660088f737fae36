// interp.cuh -- host-side interface of the table-interpolation kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "common.cuh"

namespace mirt {

// Everything the gather / spread kernels need about one batch of samples.
// A batch is nslice independent trajectories ("slices") sharing K, J, L,
// tables and column count C.  Slice s owns grid block s (prod(K)*C points)
// and samples [moff[s], moff[s+1]) of the concatenated coordinate array.
struct InterpArgs {
  Geom g;
  int real_tab;          // 1: real tables (order 0 or 1); 0: complex tables
  int order;             // 0 or 1 (1 only with real tables)
  int C;                 // columns (coils) per slice
  long long Mtot;        // samples over all slices
  // Per-sample arrays are indexed by processing position pos.  Before the
  // bin sort perm == nullptr and pos is the sample index; after it the plan
  // stores tm / slice_id / phase permuted into sorted order and perm[pos]
  // gives the caller's sample index (the row of fm).
  const double *tm;      // [D][Mtot] FP64 coordinates t = om / (2 pi / K)
  const int *slice_id;   // [Mtot] slice of each sample, or nullptr (all 0)
  const int *perm;       // [Mtot] caller's sample index of each position, or nullptr
  const void *tab[MIRT_DMAX];  // device tables: float2 (complex) or float (real)
  const float2 *phase;   // [Mtot] per-sample phase (nullptr = none)
  long long grid_elems;  // prod(K) * C  (one slice's grid, in float2)
  // Per-position tap data, computed once per trajectory by prep_taps():
  //   W[pos * SJ + (sum of J[<d]) + j]  coefficient of tap j of dimension d
  //                                     (real tables: .y = 0)
  //   K0[pos] = (first tap k1, k2, k3 wrapped into [0, K), slice)
  int SJ;                // J[0] + ... + J[D-1]
  const float2 *W;
  const int4 *K0;
};

// Tiling of the grid.  Samples are sorted into bins of B[d] grid points per
// dimension (by the slice and the wrapped first tap of each sample); the
// spread works on tiles of T[d] = multiple of B[d] points, so the tile shape
// can be tuned without re-sorting.
struct Tiling {
  int B[MIRT_DMAX];      // bin extent per dimension
  int nbin[MIRT_DMAX];   // bins per dimension
  int nbins;             // prod(nbin): bins per slice
  int T[MIRT_DMAX];      // spread tile extent per dimension (multiple of B)
  int wrap_ok;           // K[d] >= T[d] + J[d] in every dimension: the spread's
                         // range path also serves samples whose taps wrap
  // Ownership spread (2D, J = 6): the tile holding a sample's wrapped first
  // tap owns it and accumulates all its taps in a shared tile padded by J - 1
  // points; tiles are processed by colour (tile index parities), one launch
  // per colour, adding their padded tiles into the cleared grid.  Tasks are
  // sorted by colour: colour c is tasks [color_beg[c], color_beg[c+1]) and
  // reductions [red_beg[c], red_beg[c+1]).
  int own;
  // Row-sweep spread (2D, J = 6, one-point bins, K1, K2 >= 6): a team of
  // lanes owns a band of sweep_rows grid rows (1, 2 or 4) and one of `sweep`
  // segments of their columns, and sweeps the bin columns of the bin rows
  // that reach the band, with six grid columns of accumulators per row in
  // registers; every grid point is written once, in a fixed summation order.
  // No tiles, shared memory or reductions (the tiling fields are unused).
  // sweep = 0: the tiled spread; -1: the team list below.
  int sweep;
  int sweep_rows;
  float2 *sorted;        // row sweep: [Mtot][C] samples in plan order times conj(phase)
  // Row sweep over part of the batch: slices [slice0, slice0 + nslice), whose
  // samples are positions [pos0, pos0 + npos) (npos < 0: the whole batch).
  int slice0;
  long long pos0, npos;
  // Row sweep with a team list (sweep = -1): team i covers band rows from
  // sweep_team[i].y of slice .x, columns [.z, .w); nteams entries, heaviest
  // first (segments of about equal visit counts, from the sort's bins).
  const int4 *sweep_team;
  int nteams;
  // Row sweep work queue: teams are taken by warps in the order team_order
  // (heaviest first; null: index order) through the counters team_next[coil
  // chunk], which are cleared before every launch.
  const int *team_order;
  int *team_next;
  // Dense bins (the sweeps): bins holding at least a threshold of samples.
  // Before a sweep, dense_part/reduce_kernel sum each dense bin's samples into its
  // patch of J^D taps x C (patch[d][tap][c], tap = (j3 J + j2) J + j1), and
  // the sweep adds the patch where it meets the bin instead of its samples.
  // dense_of[global bin] = its dense index or -1; dense_bin[d] = the global
  // bin; a launch covers dense bins [dense0, dense0 + ndense).
  const int *dense_of;
  const int *dense_bin;
  float2 *patch;
  int dense0, ndense;
  int dense_min;         // samples that make a bin dense
  int dense_on;          // 2D row sweep: use the patches (one-row bands only)
  // 2D row sweep with 32-coil chunks: 0 the classic kernel; 1 staged per column
  // (spread_sweep2s_kernel) after the ordering pass; 2 staged, reading the
  // caller's samples directly (no ordering pass)
  int sweep_staged;
  // the staged sweep's tap records, 9 float4 per position (plan order): the
  // six first-dimension taps as FFMA2 operand pairs (wr, wr, wi, -wi), then
  // the six second-dimension taps (two per float4)
  const float4 *wsw;
  // the patches are summed in chunks of at most 64 samples: chunk i =
  // dense_chunk[i] = (dense bin, first position, end position, part index);
  // dense bin d's chunk sums are patch_part[dense_part0[d] .. dense_part0[d+1]);
  // a launch covers chunks [chunk0, chunk0 + nchunks)
  const int4 *dense_chunk;
  const int *dense_part0;
  float2 *patch_part;
  int chunk0, nchunks;
  int color_beg[9];
  int red_beg[9];
  int padc;              // spread: spare columns on each side of a tile row in
                         // shared memory (0, or J1 - 1 so that every column
                         // tap of a visiting sample has a slot and the row
                         // update needs no bounds tests; never written out)
  int nb[MIRT_DMAX];     // tiles per dimension
  int ntiles;            // prod(nb): tiles per slice
  int nslice;
  // source bins per dimension: for tile index b of dimension d >= 1,
  // src[d][b*MIRT_SRCMAX + i], i < nsrc[d][b], are the bins whose samples
  // (binned by their first tap) can have a tap in tile b; in dimension 0 the
  // source bins are at most two runs of consecutive bins (two when the
  // periodic wrap splits them), run0[b] = (first, count, first, count), so
  // that for each source row the samples of a run are one contiguous range
  // of the sort order.  Visit order: rows (dimension 1 sources inner), then
  // the two runs.
  const int *src[MIRT_DMAX];
  const int *nsrc[MIRT_DMAX];
  const int4 *run0;
  // Spread work list, heaviest first.  Task i covers the sample visits
  // [task_range[i].x, task_range[i].y) of tile task_tile[i] (= slice * ntiles
  // + tile; a tile's visits are its source bins' samples in fixed order).  A
  // tile with one task is written to the grid directly (task_slot = -1);
  // a heavy tile split into several tasks writes partial tiles to
  // scratch[slot] and reduction item r sums its red[r].z partials from slot
  // red[r].y in order into tile red[r].x.  Fixed at plan time: deterministic.
  int ntask;
  const int *task_tile;
  const int2 *task_range;
  const int *task_slot;
  int nred;
  const int4 *red;
  float2 *scratch;       // [slots][coil chunks][prod(T)][cw]
};
#define MIRT_SRCMAX 48

// Launch tuning chosen by the host (autotuned per geometry).
struct Launch {
  int threads;   // CTA size (multiple of 32); the spread gives each warp a band
  int cw;        // coil lanes per sample group
  int sb;        // samples per staged batch (even)
  int grid;      // CTAs for the persistent gather (0: size from occupancy)
  int atomic;    // spread: warps share the tile and add with shared-memory
                 // atomics (not bitwise reproducible); 0: one owner per point
};

// The gather over TMA-staged grid tiles and records (gather_tma.cu): 2D, J = 6,
// C even and >= 32, K >= 13 per dimension; or 3D, J = 6, C even and >= 8,
// K >= 9 per dimension.  Samples in the gather order are grouped by blocks of
// gb points per dimension of their first taps; start[b] is the first position
// of block b = ((slice * nbz + bz) * nby + by) * nbx + bx (start[nblocks] =
// Mtot); a work item (block, first position) covers up to gather_tma_item()
// (3D: gather_tma3_item()) samples of one block, items in block order;
// orec[pos] = (caller's sample index, 0, phase as float bits), staged with the
// tap records.
struct GatherBlocks {
  const int *start;
  const int2 *item;
  const int4 *orec;
  int gb, nbx, nby, nbz;
};
bool gather_tma_ok(const InterpArgs &a);
int gather_tma_block();
int gather_tma_item();
bool gather_tma3_ok(const InterpArgs &a);
int gather_tma3_block();
int gather_tma3_item();
// items [it0, it0 + nit) of a batch of nslice slices; *fault is set when a
// stage does not arrive within the kernel's wait limit.  fault_test: the test
// of that path (no copies are issued, every wait runs out, nothing computed).
// tcw: coils per tile, 32 (a warp per sample) or 16 (a half-warp per sample);
// 3D plans always use tiles of 8 coils (a quarter-warp per sample).
cudaError_t launch_gather_tma(const InterpArgs &a, const GatherBlocks &g, int nslice,
                              long long it0, long long nit, const float2 *ck, float2 *fm,
                              int *fault, cudaStream_t st, int fault_test = 0, int tcw = 32);

// Compute the sort key of every sample: slice * nbins + bin of its first tap.
cudaError_t launch_bin_keys(const InterpArgs &a, const Tiling &t, uint32_t *keys,
                            cudaStream_t st);

// Tap coefficients (FP64 index selection, FP32 table values) and wrapped
// first taps of every position, in the plan's sorted order.
cudaError_t launch_prep_taps(const InterpArgs &a, float2 *W, int4 *K0, cudaStream_t st);

// Stable LSD radix sort of (keys, 0..n-1) by key; writes the permutation
// (sorted position -> sample) and bin_start[nbins+1].  tmp must hold
// radix_sort_tmp_bytes(n) bytes.
size_t radix_sort_tmp_bytes(long long n);
cudaError_t radix_sort_bins(const uint32_t *keys, long long n, int nbins, void *tmp,
                            int *perm, int *bin_start, cudaStream_t st);

// Size the persistent gather grid (l.grid) from the kernel's occupancy.
cudaError_t query_gather_grid(const InterpArgs &a, Launch &l);

// fm[m][c] = sum_taps h * ck   for every sample (forward gather)
cudaError_t launch_gather(const InterpArgs &a, const Launch &l, const float2 *ck,
                          float2 *fm, cudaStream_t st);

// dense_of[dense_bin[i]] = i for i < n (dense_of cleared to -1 first)
cudaError_t launch_mark_dense(const int *dense_bin, int n, int *dense_of, cudaStream_t st);

// ck = adjoint of the gather; deterministic owner-computes spread over tiles
cudaError_t launch_spread(const InterpArgs &a, const Tiling &t, const Launch &l,
                          const int *bin_start, const float2 *fm, float2 *ck,
                          cudaStream_t st);

}  // namespace mirt
