// BDA W-projection gridder for B200 (sm_100a).
//
// Restates DDFacet's gridder<> (DDFacet/Gridder/gridder.h:78-377) as persistent, queue-driven,
// facet-inner kernels (ddfg_queue.cuh):
//
//  * one lane owns one BDA block (a baseline, rows r in R, channels [c0, c1)) and walks its
//    visibilities exactly like the reference's hot loop 1 (gridder.h:182-301): first-corr flag,
//    facet phasor exp(i nu angle) with an FP64 argument, per-antenna Jones J_p^H V J_q,
//    weights, smearing factor, and the block means of (u + w Cu, v + w Cv, w, nu) in FP64 in
//    the reference's summation order (so the integer grid indices agree bit-for-bit);
//  * the warp applies every facet of its pack to its stripe of 32 blocks in turn: the block's
//    facet-independent inputs come from DRAM once per pack, the facet-dependent record (position,
//    Jones, phasor, Stokes) is formed per facet, and the 32 lanes lay each record's S x S taps
//    (hot loop 2, gridder.h:353-375) onto the facet grid with vector atomics (scatter_q: runs of
//    records on the same cells merged in registers; into an FP64 accumulator when the facet
//    has a grid_acc buffer, folded into the float32 grid at the end of the call);
//  * per-band weight sums and the Jones normalisation sums are reduced per warp into shared
//    accumulators of the pack's facets and flushed when the CTA moves to another pack.
//
// Single-visibility maps (every block one row and one channel) load the visibility's inputs once
// per stripe (load_single); averaged blocks are walked per facet (their rows stay L1/L2-hot), and
// blocks of the optional large-block list are walked by a whole warp each.
#include <cuda_runtime.h>

#include "ddfg_common.cuh"
#include "ddfg_gridblock.cuh"
#include "ddfg_internal.h"
#include "ddfg_queue.cuh"

namespace ddfg {

// The warp's records onto facet f: through the warp's tile when there is one and the records
// qualify (one Stokes plane), else directly.
template <int NPOL, int SLOTS>
__device__ __forceinline__ void scatter_any(const GridRecord<NPOL> &rec, const ddfg_facet &f, int npol_used,
                                            LaneTaps<SLOTS> &lt, LaneTaps<SLOTS> &ltt, int lane, float2 *wtile) {
  if constexpr (NPOL == 1) {
    if (wtile && scatter_tile<SLOTS>(rec, f, ltt, lane, wtile)) return;
  }
  scatter_q<NPOL, SLOTS>(rec, f, npol_used, lt, lane);
}

// Adds the CTA's shared sums of the pack's npk facets to their float64 outputs.  Each facet's
// accumulators are one copy of the weight and Jones sums per warp (updated by that warp alone, so
// its lanes never contend with other warps for them), then the per-channel Jones sums.
__device__ __forceinline__ void flush_grid_sums(const ddfg_facet *sf, int npk, const double *s_acc, const Sched &sc,
                                                const ddfg_jones &js, int nchan) {
  const int nwarps = blockDim.x >> 5;
  for (int fi = 0; fi < npk; ++fi) {
    const ddfg_facet &f = sf[fi];
    const double *a = s_acc + (size_t)fi * sc.acc_stride;
    const double *a_chan = a + nwarps * sc.small_stride;
    const int nsw = f.nband * f.npol;
    const int nsmall = nsw + (js.mode != 0 ? 2 * f.nband : 0);
    for (int i = threadIdx.x; i < nsmall; i += blockDim.x) {
      double v = 0.;
      for (int w = 0; w < nwarps; ++w) v += a[w * sc.small_stride + i];
      double *dst = i < nsw ? f.sumwt + i : (f.sumjones ? f.sumjones + (i - nsw) : nullptr);
      if (i < nsw && !f.sumwt) dst = nullptr;
      if (dst && v != 0.) atomicAdd(dst, v);
    }
    if (js.mode != 0)
      for (int i = threadIdx.x; i < 2 * nchan; i += blockDim.x)
        if (f.sumjones_chan && a_chan[i] != 0.) atomicAdd(&f.sumjones_chan[i], a_chan[i]);
  }
}

// Moves the CTA to pack `pack` if it is not there yet: flushes the old pack's sums, stages the new
// pack's descriptors and zeroes its accumulators.  All threads call it, after queue_next.
__device__ __forceinline__ void enter_pack(const FacetTable &tab, const Sched &sc, const ddfg_jones &js, int nchan,
                                           int pack, int &cur, int &npk, ddfg_facet *sf, double *s_n0m1,
                                           double *s_acc) {
  if (pack == cur) return;
  if (cur >= 0) flush_grid_sums(sf, npk, s_acc, sc, js, nchan);
  __syncthreads();
  npk = stage_pack(tab, sc, pack, sf, s_n0m1);
  for (int i = threadIdx.x; i < npk * sc.acc_stride; i += blockDim.x) s_acc[i] = 0.;
  cur = pack;
  __syncthreads();
}

// Single-visibility blocks: each warp loads its 32 visibilities' facet-independent inputs (map
// entries, uvw, flags, weights, visibilities, Jones indices) once and grids them onto every facet
// of the pack in turn.
template <int NPOL, int SLOTS>
__global__ void __launch_bounds__(256) grid_single_q(const ddfg_vis vs, const ddfg_jones js,
                                                     const __grid_constant__ FacetTable tab, const GridParams gp,
                                                     const Sched sc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2 *wtile = (float2 *)smem_raw + (threadIdx.x >> 5) * kTileCells;  // [warps][kTileCells] if sc.tiles
  ddfg_facet *sf = (ddfg_facet *)(smem_raw + (sc.tiles ? (blockDim.x >> 5) * kTileCells * sizeof(float2) : 0));
  double *s_n0m1 = (double *)(sf + sc.max_pack);
  double *s_acc = s_n0m1 + sc.max_pack;
  __shared__ QueueSmem q;
  const int lane = threadIdx.x & 31;
  JonesCache jc;  // not used by single-visibility blocks
  LaneTaps<SLOTS> lt, ltt;
  lt.reset();
  ltt.reset();
  long long static_next = blockIdx.x;
  int cur = -1, npk = 0;
  for (;;) {
    const long long item = queue_next(sc, &q, static_next);
    if (item >= sc.nitems) break;
    const int pack = (int)(item / sc.items_per_pack);
    const long long s0 = slot_stripe(sc, item - (long long)pack * sc.items_per_pack - sc.large_items);
    enter_pack(tab, sc, js, vs.nchan, pack, cur, npk, sf, s_n0m1, s_acc);
    const int ns = (int)min(sc.spi, sc.nstripes - s0);
    for (int k; (k = warp_take(&q, ns, lane)) >= 0;) {
      const int64_t b = (s0 + k) * 32 + lane;
      SingleIn in;
      in.valid = false;
      if (b < vs.nblocks) load_single(vs, js, gp, b, in);
      if (!__any_sync(0xffffffffu, in.valid)) continue;
      for (int fi = 0; fi < npk; ++fi) {
        const ddfg_facet &f = sf[fi];
        const int npol_used = min(gp.nvispol, f.npol);
        double *a = s_acc + (size_t)fi * sc.acc_stride + (threadIdx.x >> 5) * sc.small_stride;  // this warp's sums
        double *a_chan = s_acc + (size_t)fi * sc.acc_stride + (blockDim.x >> 5) * sc.small_stride;
        GridRecord<NPOL> rec;
        grid_single_facet<NPOL>(in, vs, js, f, gp, s_n0m1[fi], rec);
        warp_add_block_sums<NPOL, true>(vs, js, f, gp, b, rec, npol_used, a, a + f.nband * f.npol, a_chan, jc);
        scatter_any<NPOL, SLOTS>(rec, f, npol_used, lt, ltt, lane, sc.tiles ? wtile : nullptr);
      }
    }
  }
  if (cur >= 0) flush_grid_sums(sf, npk, s_acc, sc, js, vs.nchan);
}

// Averaged BDA blocks: each warp walks its 32 blocks for every facet of the pack in turn
// (grid_block_record resets its Jones cache per block, so the order is free); a block's rows,
// visibilities, flags and weights come from DRAM once per pack and from L1/L2 for the other
// facets.  Large-block items give each listed block to one warp: lane 0 walks the FP64 means in
// the reference's order, the warp the rest (grid_block_record_warp).  The block walk needs ~170
// registers: CTAs of 128 threads, three per SM.
template <int NPOL, int SLOTS>
__global__ void __launch_bounds__(128, 3) grid_block_q(const ddfg_vis vs, const ddfg_jones js,
                                                       const __grid_constant__ FacetTable tab, const GridParams gp,
                                                       const Sched sc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ddfg_facet *sf = (ddfg_facet *)smem_raw;
  double *s_n0m1 = (double *)(sf + sc.max_pack);
  double *s_acc = s_n0m1 + sc.max_pack;
  __shared__ QueueSmem q;
  const int lane = threadIdx.x & 31;
  JonesCache jc;
  LaneTaps<SLOTS> lt;
  lt.reset();
  long long static_next = blockIdx.x;
  int cur = -1, npk = 0;
  for (;;) {
    const long long item = queue_next(sc, &q, static_next);
    if (item >= sc.nitems) break;
    const int pack = (int)(item / sc.items_per_pack);
    const long long r = item - (long long)pack * sc.items_per_pack;
    enter_pack(tab, sc, js, vs.nchan, pack, cur, npk, sf, s_n0m1, s_acc);
    if (r < sc.large_items) {
      const long long t0 = r * sc.large_per_item;
      const int nt = (int)min((long long)sc.large_per_item, vs.nlarge - t0);
      for (int k; (k = warp_take(&q, nt, lane)) >= 0;) {
        const int64_t bl = vs.large_blocks[t0 + k];
        // entries that are out of range or not above the threshold belong to the stripes
        if (bl < 0 || bl >= vs.nblocks || block_nvis(vs, bl) <= vs.large_min_vis) continue;
        if (vs.sparsification && !vs.sparsification[bl]) continue;
        for (int fi = 0; fi < npk; ++fi) {
          const ddfg_facet &f = sf[fi];
          const int npol_used = min(gp.nvispol, f.npol);
          double *a = s_acc + (size_t)fi * sc.acc_stride + (threadIdx.x >> 5) * sc.small_stride;
          double *a_chan = s_acc + (size_t)fi * sc.acc_stride + (blockDim.x >> 5) * sc.small_stride;
          BlockMeans bm{};
          if (lane == 0) bm = grid_block_means(vs, f, bl);
          GridRecord<NPOL> rec;
          rec.valid = false;
          rec.single_chan = true;
          grid_block_record_warp<NPOL>(vs, js, f, gp, bl, bm, s_n0m1[fi], 0, lane, npol_used, a_chan, rec);
          warp_add_block_sums<NPOL, false>(vs, js, f, gp, bl, rec, npol_used, a, a + f.nband * f.npol, a_chan, jc,
                                           !rec.single_chan);
          scatter_q<NPOL, SLOTS, false>(rec, f, npol_used, lt, lane);
        }
      }
      continue;
    }
    const long long s0 = slot_stripe(sc, r - sc.large_items);
    const int ns = (int)min(sc.spi, sc.nstripes - s0);
    for (int k; (k = warp_take(&q, ns, lane)) >= 0;) {
      const int64_t b = (s0 + k) * 32 + lane;
      // blocks above the large-block threshold are the large items' work
      const bool mine = b < vs.nblocks && !(vs.nlarge > 0 && block_nvis(vs, b) > vs.large_min_vis);
      for (int fi = 0; fi < npk; ++fi) {
        const ddfg_facet &f = sf[fi];
        const int npol_used = min(gp.nvispol, f.npol);
        double *a = s_acc + (size_t)fi * sc.acc_stride + (threadIdx.x >> 5) * sc.small_stride;
        double *a_chan = s_acc + (size_t)fi * sc.acc_stride + (blockDim.x >> 5) * sc.small_stride;
        GridRecord<NPOL> rec;
        rec.valid = false;
        if (mine) grid_block_record<NPOL>(vs, js, f, gp, b, s_n0m1[fi], rec, jc);
        warp_add_block_sums<NPOL, false>(vs, js, f, gp, b, rec, npol_used, a, a + f.nband * f.npol, a_chan, jc);
        scatter_q<NPOL, SLOTS, false>(rec, f, npol_used, lt, lane);
      }
    }
  }
  if (cur >= 0) flush_grid_sums(sf, npk, s_acc, sc, js, vs.nchan);
}

// grid = fl(grid + acc); acc = 0, for every facet of the table that has an FP64 accumulator.
__global__ void fold_acc_kernel(const __grid_constant__ FacetTable tab, int nfacets) {
  const int fi = blockIdx.y;
  if (fi >= nfacets) return;
  const ddfg_facet &f = tab.f[fi];
  if (!f.grid_acc) return;
  float2 *grid = (float2 *)f.grid;
  double2 *acc = (double2 *)f.grid_acc;
  const int64_t n = (int64_t)f.nband * f.npol * f.ny * f.nx;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double2 a = acc[i];
    if (a.x != 0. || a.y != 0.) {
      const float2 g = grid[i];
      grid[i] = make_float2((float)((double)g.x + a.x), (float)((double)g.y + a.y));
      acc[i] = make_double2(0., 0.);
    }
  }
}

}  // namespace ddfg

using namespace ddfg;

namespace {

template <int NP, int SL>
int launch_grid_table(const ddfg_vis *vs, const ddfg_jones *js, const FacetTable &tab, const GridParams &gp,
                      Sched sc, const ddfg_batch *batch, cudaStream_t stream) {
  const bool single = vs->single_vis_blocks != 0;
  const int threads = single ? 256 : 128;
  const size_t smem = (sc.tiles ? (size_t)(threads / 32) * kTileCells * sizeof(float2) : 0) +
                      (sizeof(ddfg_facet) + sizeof(double)) * (size_t)sc.max_pack +
                      sizeof(double) * (size_t)sc.max_pack * (size_t)sc.acc_stride;
  const void *kern = single ? (const void *)grid_single_q<NP, SL> : (const void *)grid_block_q<NP, SL>;
  int per_sm = 0;
  int rc = ddfg_kernel_prepare(kern, threads, smem, &per_sm);
  if (rc) return rc;
  if (batch && batch->ctas_per_sm > 0) per_sm = min(per_sm, (int)batch->ctas_per_sm);
  const int ctas = ddfg_num_ctas(per_sm);
  sched_set_regions(sc, (batch && (batch->flags & 4)) ? ctas : 1);
  if (single) grid_single_q<NP, SL><<<ctas, threads, smem, stream>>>(*vs, *js, tab, gp, sc);
  else grid_block_q<NP, SL><<<ctas, threads, smem, stream>>>(*vs, *js, tab, gp, sc);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "grid launch: %s", cudaGetErrorString(e));
  return DDFG_OK;
}

}  // namespace

int ddfg_launch_grid(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_facet *facets, int nfacets, int policy,
                     int nvispol, int dopsf, const ddfg_batch *batch, cudaStream_t stream) {
  int max_support = 1, max_band = 1;
  bool any_acc = false;
  for (int i = 0; i < nfacets; ++i) {
    max_support = max(max_support, facets[i].max_support);
    max_band = max(max_band, facets[i].nband * (facets[i].npol + 2));
    any_acc = any_acc || facets[i].grid_acc != nullptr;
  }
  const int slots = tap_slots(max_support);
  GridParams gp;
  gp.policy = policy;
  gp.nvispol = nvispol;
  gp.dopsf = dopsf;
  gp.freq_mean0 = vs->freq_mean;
  const int nwarps_cta = vs->single_vis_blocks ? 8 : 4;
  const int acc_stride = nwarps_cta * max_band + 2 * vs->nchan;
  const size_t per_facet_smem = sizeof(ddfg_facet) + sizeof(double) + sizeof(double) * (size_t)acc_stride;
  // Shared memory per CTA: two 256-thread CTAs (single-visibility maps) or three 128-thread CTAs
  // (averaged blocks) per SM, each with the warps' grid tiles (one Stokes plane) and the shared
  // accumulators of a pack.
  const bool single = vs->single_vis_blocks != 0;
  const size_t budget = single ? 110 * 1024 : 74 * 1024;
  const size_t tile_bytes = (size_t)(single ? 8 : 4) * kTileCells * sizeof(float2);
  // warp tiles: single-visibility maps (a stripe is one row's neighbouring channels) only
  int tiles = (single && nvispol == 1 && batch && (batch->flags & 2)) ? 1 : 0;
  if (tiles && budget < tile_bytes + per_facet_smem) tiles = 0;
  const int max_fit = (int)((budget - (tiles ? tile_bytes : 0)) / per_facet_smem);
  if (max_fit < 1) return ddfg_set_error(DDFG_ESIZE, "grid: too many bands/channels for the shared accumulators");
  int want = (batch && batch->facets_per_pack > 0) ? batch->facets_per_pack : 16;
  want = max(1, min(want, max_fit));
  unsigned long long *counters = nullptr;
  const int ngroups = (nfacets + DDFG_TABLE_FACETS - 1) / DDFG_TABLE_FACETS;
  if (batch && !(batch->flags & 1)) {
    counters = (unsigned long long *)batch->workspace;
    const cudaError_t e = cudaMemsetAsync(counters, 0, sizeof(unsigned long long) * ngroups, stream);
    if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "grid: %s", cudaGetErrorString(e));
  }
  const long long nstripes = (vs->nblocks + 31) / 32;
  const int nlarge = vs->single_vis_blocks ? 0 : (int)(vs->nlarge < (1LL << 30) ? vs->nlarge : (1LL << 30));
  FacetTable tab_tl;  // host staging of the parameter table (copied into the launch)
  for (int g = 0; g < ngroups; ++g) {
    const int f0 = (int)(((long long)g * nfacets) / ngroups), f1 = (int)(((long long)(g + 1) * nfacets) / ngroups);
    const int n = f1 - f0;
    for (int i = 0; i < n; ++i) tab_tl.f[i] = facets[f0 + i];
    Sched sc;
    sc.nfacets = n;
    sc.npacks = (n + want - 1) / want;
    sc.max_pack = (n + sc.npacks - 1) / sc.npacks;
    sc.acc_stride = acc_stride;
    sc.small_stride = max_band;
    sc.tiles = tiles;
    sc.nstripes = nstripes;
    // default: items of 16-256 stripes, about four per resident CTA and pack
    const long long spi = (batch && batch->stripes_per_item > 0) ? batch->stripes_per_item
                                                                 : max(16LL, min(256LL, nstripes / 1184));
    sc.spi = max(1LL, spi);
    sc.stripe_items = (nstripes + sc.spi - 1) / sc.spi;
    sc.large_per_item = vs->single_vis_blocks ? 8 : 4;
    sc.large_items = (nlarge + sc.large_per_item - 1) / sc.large_per_item;
    sched_set_regions(sc, 1);
    sc.counter = counters ? counters + g : nullptr;
    int rc;
#define LG(NP, SL) rc = launch_grid_table<NP, SL>(vs, js, tab_tl, gp, sc, batch, stream)
#define LG_NP(SL)                \
  switch (nvispol) {             \
    case 1: LG(1, SL); break;    \
    case 2: LG(2, SL); break;    \
    case 3: LG(3, SL); break;    \
    default: LG(4, SL); break;   \
  }
    if (slots == 2) { LG_NP(2) } else if (slots == 4) { LG_NP(4) } else { LG_NP(8) }
#undef LG_NP
#undef LG
    if (rc) return rc;
    if (any_acc) {
      int64_t cells = 0;
      for (int i = 0; i < n; ++i)
        {
          const int64_t c = (int64_t)tab_tl.f[i].nband * tab_tl.f[i].npol * tab_tl.f[i].ny * tab_tl.f[i].nx;
          if (c > cells) cells = c;
        }
      const int bx = (int)((cells + 255) / 256 < 1024 ? (cells + 255) / 256 : 1024);
      fold_acc_kernel<<<dim3(bx, n), 256, 0, stream>>>(tab_tl, n);
      const cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "grid fold: %s", cudaGetErrorString(e));
    }
  }
  return DDFG_OK;
}
