// runtime.cuh -- host-side state shared by the translation units of the C ABI:
// the caching device allocator, device buffers, and the interpolation and
// NUFFT plan objects behind the opaque handles of include/mirt_b200.h.
#pragma once

#include <cufft.h>

#include <string>
#include <utility>
#include <vector>

#include "fft.cuh"
#include "glue.cuh"
#include "interp.cuh"

namespace mirt {

// Record an error for mirt_last_error(); returns `code`.
int api_fail(int code, const std::string &msg);

// Caching device allocator: blocks are rounded up to a power of two and kept
// for reuse, so repeated calls do not pay cudaMalloc / cudaFree.
cudaError_t dalloc(void **p, size_t bytes);
void dfree(void *p, size_t bytes);

struct DMem {
  void *p = nullptr;
  size_t bytes = 0;
  DMem() = default;
  DMem(const DMem &) = delete;
  DMem &operator=(const DMem &) = delete;
  ~DMem() { release(); }
  void release() {
    dfree(p, bytes);
    p = nullptr;
    bytes = 0;
  }
  cudaError_t alloc(size_t b) {
    release();
    bytes = b;
    return dalloc(&p, b);
  }
  template <class T>
  T *as() const {
    return static_cast<T *>(p);
  }
};

inline void swap_mem(DMem &x, DMem &y) {
  std::swap(x.p, y.p);
  std::swap(x.bytes, y.bytes);
}

inline cudaStream_t as_stream(void *s) { return static_cast<cudaStream_t>(s); }

}  // namespace mirt

// Interpolation plan: geometry, tables, sorted trajectory, tap records, spread
// tiling and work list, launch shapes.
struct mirt_interp_plan {
  mirt::InterpArgs a{};
  mirt::Tiling t{};
  mirt::Launch lg{}, ls{};
  mirt::DMem tm, slice, perm, bin_start, tab[MIRT_DMAX], phase, src[MIRT_DMAX], nsrc[MIRT_DMAX];
  mirt::DMem keys, sorttmp, moff;
  mirt::DMem task_tile, task_range, task_slot, red, scratch, wtap, k0tap, run0;
  // the gather's copy of the per-position records, in its own order (4-point
  // blocks of the first tap); ag is `a` with these arrays
  mirt::InterpArgs ag{};
  mirt::DMem wtap_g, k0tap_g, perm_g, phase_g;
  mirt::DMem orec_g;        // TMA gather: output records (sample index, phase) in gather order
  mirt::DMem wsw;           // staged 2D row sweep: tap records with FFMA2 operand pairs, plan order
  mirt::DMem swept;        // row-sweep spread: the samples in plan order, [Mtot][C]
  mirt::DMem sweep_teams;  // row-sweep spread: balanced team list (int4 per team)
  std::vector<int4> team_host;  // the same list on the host
  mirt::DMem team_order, team_next;  // row-sweep work queue: heaviest-first order, counter
  mirt::DMem dense_of, dense_bin, patch;  // the sweeps' dense bins and their patches
  mirt::DMem dense_chunk, dense_part0, patch_part;  // chunks of the patch sums
  std::vector<int> dense_slice;           // first dense bin of each slice (+ total)
  std::vector<int> dense_part0_host;      // first chunk of each dense bin (+ total)
  // TMA gather: first position of each block of the gather order, work items
  // (block, first position), the first item of each slice, fault flag
  mirt::DMem gblk, gitem, gfault;
  std::vector<long long> gitem_slice;
  mirt::GatherBlocks gbk{};
  int gtma = 0;            // 1: the gather runs on TMA-staged tiles
  int gfault_test = 0;     // 1: test of the TMA gather's bounded waits (no copies)
  int split_chunk = 1024;  // sample visits per spread task before a tile is split
  int heavy_first = 1;     // spread task order: 1 heaviest first, 0 grid order
  int deterministic = 1;   // 0: the spread may use shared-memory atomics
  std::vector<long long> moff_host;
  // 4D plan (interp4.cu): a 3D plan over the nslice * K4 hyperplanes whose
  // samples are the (sample, 4th-dimension tap) pairs; x4_pos[m J4 + j4] is
  // the 3D position of pair (m, j4), x4_src[e] the 4D sample of 3D sample e,
  // x4_buf the [Me][C] samples of the 3D plan
  mirt_interp_plan *sub4 = nullptr;
  int J4 = 0;
  long long Me = 0;
  mirt::DMem x4_pos, x4_src, x4_buf;
  mirt_interp_plan() = default;
  mirt_interp_plan(const mirt_interp_plan &) = delete;
  mirt_interp_plan &operator=(const mirt_interp_plan &) = delete;
  ~mirt_interp_plan() { delete sub4; }
};

// NUFFT plan: an interpolation plan plus scaling factors, grids and the FFT.
struct mirt_nufft {
  mirt_interp_plan *ip = nullptr;
  mirt::GlueGeom gg{};
  int C = 0, nslice = 0;
  long long Mtot = 0;
  mirt::DMem sn, grid, grid_cm, hx, hX;  // grid: coil innermost (interp); grid_cm: coil-major (FFT)
  mirt::DMem pad;                        // coil-major FFT input: image region rewritten per
                                         // call, zero padding written once
  mirt::DMem phtab;                      // newfft phase_before per dimension, float2 [sum K_d]
  mirt::GridPhase gp{};                  // tables into phtab (tab[0] null: no grid phase)
  cufftHandle fft = 0;
  bool fft_ok = false;
  // power-of-two grids from 64 to 1024 points per dimension: the FFT runs as
  // fused passes over `grid` itself (fft.cu) and grid_cm / pad / cuFFT are unused
  bool own_fft = false;
  mirt::DMem twtab;                      // exp(-2 pi i k / K_d) per dimension, float2 [sum K_d]
  mirt::NufftFft nf{};
  // host-buffer calls, pipelined by slice chunks: copy streams, per-chunk
  // events and the FFT plans of the chunk sizes (made at the first such call)
  cudaStream_t cs_in = nullptr, cs_out = nullptr;
  std::vector<cudaEvent_t> ev;
  cufftHandle fft_ch[2] = {0, 0};
  int ch_n[2] = {0, 0};  // slices per chunk of fft_ch[i] (0: not made)
  ~mirt_nufft() {
    if (fft_ok) cufftDestroy(fft);
    for (int i = 0; i < 2; i++)
      if (ch_n[i]) cufftDestroy(fft_ch[i]);
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
    if (cs_in) cudaStreamDestroy(cs_in);
    if (cs_out) cudaStreamDestroy(cs_out);
    delete ip;
  }
};
