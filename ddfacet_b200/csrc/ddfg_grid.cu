// BDA W-projection gridder for B200 (sm_100a).
//
// Restates DDFacet's gridder<> (DDFacet/Gridder/gridder.h:78-377) as a warp-cooperative kernel:
//
//  * one lane owns one BDA block (a baseline, rows r in R, channels [c0, c1)) and walks its
//    visibilities exactly like the reference's hot loop 1 (gridder.h:182-301): first-corr flag,
//    facet phasor exp(i nu angle) with an FP64 argument, per-antenna Jones J_p^H V J_q,
//    weights, smearing factor, and the block means of (u + w Cu, v + w Cv, w, nu) in FP64 in
//    the reference's summation order (so the integer grid indices agree bit-for-bit);
//  * the block's Stokes value and footprint are then broadcast to the whole warp, whose 32
//    lanes lay the S x S convolution taps (hot loop 2, gridder.h:353-375) onto the facet grid
//    with vector complex atomics, consecutive lanes on consecutive cells of a CF row;
//  * per-band weight sums and the Jones normalisation sums are reduced in shared memory and
//    flushed once per CTA and facet.
//
// One launch takes up to DDFG_FACETS_PER_LAUNCH facet descriptors as a kernel parameter; the
// CTAs walk the facets one after the other, each over the whole block list, so the working set
// in L2 is one facet's grid and CF tables at a time.
#include <cuda_runtime.h>

#include "ddfg_common.cuh"
#include "ddfg_gridblock.cuh"
#include "ddfg_internal.h"
#include "ddfg_taps.cuh"

namespace ddfg {

template <int NPOL, int SLOTS, bool SINGLE>
__global__ void __launch_bounds__(256) grid_kernel(const ddfg_vis vs, const ddfg_jones js, const FacetPack pack,
                                                   const GridParams gp) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ddfg_facet *sf = (ddfg_facet *)smem_raw;
  double *s_acc = (double *)(sf + pack.n);
  stage_facets(pack, sf);
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  const int64_t nstripes = (vs.nblocks + 31) / 32;

  for (int fi = 0; fi < pack.n; ++fi) {
    __syncthreads();
    const ddfg_facet &f = sf[fi];
    const int npol_used = min(gp.nvispol, f.npol);
    const int nsw = f.nband * f.npol;
    double *s_sumwt = s_acc;                  // [nband][npol]
    double *s_sumj = s_acc + nsw;             // [2][nband]
    double *s_chan = s_sumj + 2 * f.nband;    // [2][nchan]
    const int nacc = nsw + 2 * f.nband + 2 * vs.nchan;
    for (int i = threadIdx.x; i < nacc; i += blockDim.x) s_acc[i] = 0.;
    __syncthreads();

    const double n0m1 = sqrt(1. - f.l0 * f.l0 - f.m0 * f.m0) - 1.;
    JonesCache jc;
    LaneTaps<SLOTS> lt;
    lt.reset();

    for (int64_t s = (int64_t)blockIdx.x * nwarps + warp; s < nstripes; s += (int64_t)gridDim.x * nwarps) {
      const int64_t b = s * 32 + lane;
      GridRecord<NPOL> rec;
      rec.valid = false;
      if (b < vs.nblocks) {
        if (SINGLE) grid_single_record<NPOL>(vs, js, f, gp, b, n0m1, rec);
        else grid_block_record<NPOL>(vs, js, f, gp, b, n0m1, rec, jc);
      }

      warp_add_block_sums<NPOL, SINGLE>(vs, js, f, gp, b, rec, npol_used, s_sumwt, s_sumj, s_chan, jc);

      scatter_records<NPOL, SLOTS>(rec, f, npol_used, lt, lane);
    }
    __syncthreads();
    // Flush this CTA's sums for facet fi.
    for (int i = threadIdx.x; i < nsw; i += blockDim.x)
      if (f.sumwt && s_sumwt[i] != 0.) atomicAdd(&f.sumwt[i], s_sumwt[i]);
    if (js.mode != 0) {
      for (int i = threadIdx.x; i < 2 * f.nband; i += blockDim.x)
        if (f.sumjones && s_sumj[i] != 0.) atomicAdd(&f.sumjones[i], s_sumj[i]);
      for (int i = threadIdx.x; i < 2 * vs.nchan; i += blockDim.x)
        if (f.sumjones_chan && s_chan[i] != 0.) atomicAdd(&f.sumjones_chan[i], s_chan[i]);
    }
    __syncthreads();
  }
}

// Averaged BDA blocks, facet-inner: each warp walks its 32 blocks for every facet of the launch
// in turn (grid_block_record resets its Jones cache per block, so the order is free), so a
// block's rows, visibilities, flags and weights are read from DRAM once per launch and from L1
// for the other facets; per-facet shared accumulators hold the weight and Jones sums.  The block
// walk needs ~170 registers: CTAs of 128 threads, three per SM (12 warps; 256-thread CTAs at the
// unconstrained 212 registers fit once, 8 warps).
template <int NPOL, int SLOTS>
__global__ void __launch_bounds__(128, 3) grid_block_fi_kernel(const ddfg_vis vs, const ddfg_jones js,
                                                            const FacetPack pack, const GridParams gp,
                                                            int acc_stride) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ddfg_facet *sf = (ddfg_facet *)smem_raw;
  double *s_n0m1 = (double *)(sf + DDFG_FACETS_PER_LAUNCH);
  double *s_acc = s_n0m1 + DDFG_FACETS_PER_LAUNCH;
  stage_facets(pack, sf);
  for (int i = threadIdx.x; i < pack.n * acc_stride; i += blockDim.x) s_acc[i] = 0.;
  __syncthreads();
  if (threadIdx.x < pack.n) {
    const ddfg_facet &f = sf[threadIdx.x];
    s_n0m1[threadIdx.x] = sqrt(1. - f.l0 * f.l0 - f.m0 * f.m0) - 1.;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  const int64_t nstripes = (vs.nblocks + 31) / 32;
  JonesCache jc;
  LaneTaps<SLOTS> lt;
  lt.reset();
  for (int64_t s = (int64_t)blockIdx.x * nwarps + warp; s < nstripes; s += (int64_t)gridDim.x * nwarps) {
    const int64_t b = s * 32 + lane;
    // blocks of the large-block list are left to the second loop
    const bool mine = b < vs.nblocks && !(vs.nlarge > 0 && block_nvis(vs, b) > vs.large_min_vis);
    for (int fi = 0; fi < pack.n; ++fi) {
      const ddfg_facet &f = sf[fi];
      const int npol_used = min(gp.nvispol, f.npol);
      double *a = s_acc + (size_t)fi * acc_stride;
      GridRecord<NPOL> rec;
      rec.valid = false;
      if (mine) grid_block_record<NPOL>(vs, js, f, gp, b, s_n0m1[fi], rec, jc);
      warp_add_block_sums<NPOL, false>(vs, js, f, gp, b, rec, npol_used, a, a + f.nband * f.npol,
                                       a + f.nband * f.npol + 2 * f.nband, jc);
      scatter_records<NPOL, SLOTS>(rec, f, npol_used, lt, lane);
    }
  }
  // Large blocks, one warp each: lane 0 walks the FP64 means in the reference's order, the warp
  // the rest (grid_block_record_warp); lane 0 holds the record the warp then lays down.
  for (int64_t t = (int64_t)blockIdx.x * nwarps + warp; t < vs.nlarge; t += (int64_t)gridDim.x * nwarps) {
    const int64_t bl = vs.large_blocks[t];
    if (vs.sparsification && !vs.sparsification[bl]) continue;
    for (int fi = 0; fi < pack.n; ++fi) {
      const ddfg_facet &f = sf[fi];
      const int npol_used = min(gp.nvispol, f.npol);
      double *a = s_acc + (size_t)fi * acc_stride;
      double *a_chan = a + f.nband * f.npol + 2 * f.nband;
      BlockMeans bm{};
      if (lane == 0) bm = grid_block_means(vs, f, bl);
      GridRecord<NPOL> rec;
      rec.valid = false;
      rec.single_chan = true;
      grid_block_record_warp<NPOL>(vs, js, f, gp, bl, bm, s_n0m1[fi], 0, lane, npol_used, a_chan, rec);
      warp_add_block_sums<NPOL, false>(vs, js, f, gp, bl, rec, npol_used, a, a + f.nband * f.npol, a_chan, jc,
                                       !rec.single_chan);
      scatter_records<NPOL, SLOTS>(rec, f, npol_used, lt, lane);
    }
  }
  __syncthreads();
  for (int fi = 0; fi < pack.n; ++fi) {
    const ddfg_facet &f = sf[fi];
    const double *a = s_acc + (size_t)fi * acc_stride;
    const int nsw = f.nband * f.npol;
    for (int i = threadIdx.x; i < nsw; i += blockDim.x)
      if (f.sumwt && a[i] != 0.) atomicAdd(&f.sumwt[i], a[i]);
    if (js.mode != 0) {
      for (int i = threadIdx.x; i < 2 * f.nband; i += blockDim.x)
        if (f.sumjones && a[nsw + i] != 0.) atomicAdd(&f.sumjones[i], a[nsw + i]);
      for (int i = threadIdx.x; i < 2 * vs.nchan; i += blockDim.x)
        if (f.sumjones_chan && a[nsw + 2 * f.nband + i] != 0.) atomicAdd(&f.sumjones_chan[i], a[nsw + 2 * f.nband + i]);
    }
  }
}

// Single-visibility blocks, facet-inner: each warp loads its 32 visibilities' facet-independent
// inputs (map entries, uvw, flags, weights, visibilities, Jones indices) once and grids them onto
// every facet of the launch in turn, instead of re-reading them once per facet.  Per-facet weight
// and Jones sums have their own shared-memory accumulators (acc_stride doubles each).
template <int NPOL, int SLOTS>
__global__ void __launch_bounds__(256) grid_single_fi_kernel(const ddfg_vis vs, const ddfg_jones js,
                                                             const FacetPack pack, const GridParams gp,
                                                             int acc_stride) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ddfg_facet *sf = (ddfg_facet *)smem_raw;
  double *s_n0m1 = (double *)(sf + DDFG_FACETS_PER_LAUNCH);
  double *s_acc = s_n0m1 + DDFG_FACETS_PER_LAUNCH;
  stage_facets(pack, sf);
  for (int i = threadIdx.x; i < pack.n * acc_stride; i += blockDim.x) s_acc[i] = 0.;
  __syncthreads();
  if (threadIdx.x < pack.n) {
    const ddfg_facet &f = sf[threadIdx.x];
    s_n0m1[threadIdx.x] = sqrt(1. - f.l0 * f.l0 - f.m0 * f.m0) - 1.;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  const int64_t nstripes = (vs.nblocks + 31) / 32;
  JonesCache jc;  // not used by single-visibility blocks
  LaneTaps<SLOTS> lt;
  lt.reset();

  for (int64_t s = (int64_t)blockIdx.x * nwarps + warp; s < nstripes; s += (int64_t)gridDim.x * nwarps) {
    const int64_t b = s * 32 + lane;
    SingleIn in;
    in.valid = false;
    if (b < vs.nblocks) load_single(vs, js, gp, b, in);
    if (!__any_sync(0xffffffffu, in.valid)) continue;
    for (int fi = 0; fi < pack.n; ++fi) {
      const ddfg_facet &f = sf[fi];
      const int npol_used = min(gp.nvispol, f.npol);
      double *a = s_acc + (size_t)fi * acc_stride;
      double *a_sumwt = a;                      // [nband][npol]
      double *a_sumj = a + f.nband * f.npol;    // [2][nband]
      double *a_chan = a_sumj + 2 * f.nband;    // [2][nchan]
      GridRecord<NPOL> rec;
      grid_single_facet<NPOL>(in, vs, js, f, gp, s_n0m1[fi], rec);
      warp_add_block_sums<NPOL, true>(vs, js, f, gp, b, rec, npol_used, a_sumwt, a_sumj, a_chan, jc);
      scatter_records<NPOL, SLOTS>(rec, f, npol_used, lt, lane);
    }
  }
  __syncthreads();
  // Flush this CTA's sums for every facet of the launch.
  for (int fi = 0; fi < pack.n; ++fi) {
    const ddfg_facet &f = sf[fi];
    const double *a = s_acc + (size_t)fi * acc_stride;
    const int nsw = f.nband * f.npol;
    for (int i = threadIdx.x; i < nsw; i += blockDim.x)
      if (f.sumwt && a[i] != 0.) atomicAdd(&f.sumwt[i], a[i]);
    if (js.mode != 0) {
      for (int i = threadIdx.x; i < 2 * f.nband; i += blockDim.x)
        if (f.sumjones && a[nsw + i] != 0.) atomicAdd(&f.sumjones[i], a[nsw + i]);
      for (int i = threadIdx.x; i < 2 * vs.nchan; i += blockDim.x)
        if (f.sumjones_chan && a[nsw + 2 * f.nband + i] != 0.) atomicAdd(&f.sumjones_chan[i], a[nsw + 2 * f.nband + i]);
    }
  }
}

}  // namespace ddfg

using namespace ddfg;

int ddfg_launch_grid(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_facet *facets, int nfacets, int policy,
                     int nvispol, int dopsf, int num_ctas, cudaStream_t stream) {
  int max_support = 1;
  for (int i = 0; i < nfacets; ++i) max_support = max(max_support, facets[i].max_support);
  const int slots = tap_slots(max_support);
  GridParams gp;
  gp.policy = policy;
  gp.nvispol = nvispol;
  gp.dopsf = dopsf;
  gp.freq_mean0 = vs->freq_mean;
  int max_band = 1;
  for (int i = 0; i < nfacets; ++i) max_band = max(max_band, facets[i].nband * (facets[i].npol + 2));
  const size_t smem = sizeof(ddfg_facet) * DDFG_FACETS_PER_LAUNCH + sizeof(double) * ((size_t)max_band + 2 * (size_t)vs->nchan);
  if (smem > 160 * 1024) return ddfg_set_error(DDFG_ESIZE, "grid: too many bands/channels for the shared accumulators");
  // Facet-inner single-visibility kernel when every facet's accumulators fit in shared memory.
  const int acc_stride = max_band + 2 * vs->nchan;
  const size_t smem_fi = sizeof(ddfg_facet) * DDFG_FACETS_PER_LAUNCH + sizeof(double) * DDFG_FACETS_PER_LAUNCH +
                         sizeof(double) * (size_t)DDFG_FACETS_PER_LAUNCH * (size_t)acc_stride;
  const bool facet_inner = vs->single_vis_blocks && smem_fi <= 64 * 1024;
  const bool block_fi = !vs->single_vis_blocks && smem_fi <= 64 * 1024;
  for (int f0 = 0; f0 < nfacets; f0 += DDFG_FACETS_PER_LAUNCH) {
    FacetPack pack;
    pack.n = min(DDFG_FACETS_PER_LAUNCH, nfacets - f0);
    for (int i = 0; i < pack.n; ++i) pack.f[i] = facets[f0 + i];
    const int npol = nvispol;
    cudaError_t e;
    if (block_fi) {
#define LAUNCH_B1(NP, SL)                                                                                          \
  do {                                                                                                             \
    if (smem_fi > 48 * 1024)                                                                                       \
      cudaFuncSetAttribute(grid_block_fi_kernel<NP, SL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_fi); \
    grid_block_fi_kernel<NP, SL><<<ddfg_one_wave(grid_block_fi_kernel<NP, SL>, 128, smem_fi), 128, smem_fi, stream>>>( \
        *vs, *js, pack, gp, acc_stride);                                                                           \
  } while (0)
#define LAUNCH_B_NP(SL)              \
  switch (npol) {                    \
    case 1: LAUNCH_B1(1, SL); break; \
    case 2: LAUNCH_B1(2, SL); break; \
    case 3: LAUNCH_B1(3, SL); break; \
    default: LAUNCH_B1(4, SL); break; \
  }
      if (slots == 2) { LAUNCH_B_NP(2) } else if (slots == 4) { LAUNCH_B_NP(4) } else { LAUNCH_B_NP(8) }
#undef LAUNCH_B_NP
#undef LAUNCH_B1
      e = cudaGetLastError();
      if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "grid launch: %s", cudaGetErrorString(e));
      continue;
    }
    if (facet_inner) {
#define LAUNCH_F1(NP, SL)                                                                                          \
  do {                                                                                                             \
    if (smem_fi > 48 * 1024)                                                                                       \
      cudaFuncSetAttribute(grid_single_fi_kernel<NP, SL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_fi); \
    grid_single_fi_kernel<NP, SL><<<num_ctas, 256, smem_fi, stream>>>(*vs, *js, pack, gp, acc_stride);             \
  } while (0)
#define LAUNCH_F_NP(SL)              \
  switch (npol) {                    \
    case 1: LAUNCH_F1(1, SL); break; \
    case 2: LAUNCH_F1(2, SL); break; \
    case 3: LAUNCH_F1(3, SL); break; \
    default: LAUNCH_F1(4, SL); break; \
  }
      if (slots == 2) { LAUNCH_F_NP(2) } else if (slots == 4) { LAUNCH_F_NP(4) } else { LAUNCH_F_NP(8) }
#undef LAUNCH_F_NP
#undef LAUNCH_F1
      e = cudaGetLastError();
      if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "grid launch: %s", cudaGetErrorString(e));
      continue;
    }
#define LAUNCH_G1(NP, SL, SG)                                                                                 \
  do {                                                                                                        \
    if (smem > 48 * 1024)                                                                                     \
      cudaFuncSetAttribute(grid_kernel<NP, SL, SG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);  \
    grid_kernel<NP, SL, SG><<<num_ctas, 256, smem, stream>>>(*vs, *js, pack, gp);                             \
  } while (0)
#define LAUNCH_G(NP, SL)                                 \
  do {                                                   \
    if (vs->single_vis_blocks) LAUNCH_G1(NP, SL, true);  \
    else LAUNCH_G1(NP, SL, false);                       \
  } while (0)
#define LAUNCH_G_NP(SL)            \
  switch (npol) {                  \
    case 1: LAUNCH_G(1, SL); break; \
    case 2: LAUNCH_G(2, SL); break; \
    case 3: LAUNCH_G(3, SL); break; \
    default: LAUNCH_G(4, SL); break; \
  }
    if (slots == 2) { LAUNCH_G_NP(2) } else if (slots == 4) { LAUNCH_G_NP(4) } else { LAUNCH_G_NP(8) }
#undef LAUNCH_G_NP
#undef LAUNCH_G
#undef LAUNCH_G1
    e = cudaGetLastError();
    if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "grid launch: %s", cudaGetErrorString(e));
  }
  return DDFG_OK;
}
