// BDA W-projection degridder for B200 (sm_100a).
//
// Restates DDFacet's degridder<> (DDFacet/Gridder/degridder.h:55-267) as persistent,
// queue-driven, facet-inner kernels (ddfg_queue.cuh):
//
//  * one lane owns one BDA block: band, mean frequency over the block's channels and the
//    unweighted row means of (u + w Cu, v + w Cv, w) in FP64 (degridder.h:138-167), then the
//    W plane, grid location and oversampling phase (degridder.h:170-200);
//  * the warp gathers each block's S x S footprint cooperatively -- lanes on consecutive cells
//    of a CF row, one coalesced load per lane and tap -- and reduces the partial sums
//    (degridder.h:202-212);
//  * the owning lane converts Stokes to correlations, applies the per-block or per-visibility
//    Jones, the facet phasor exp(+i nu angle) (FP64 argument) and the smearing factor, and
//    subtracts the prediction from the visibilities (degridder.h:214-264).
//
// Every facet of a pack is applied to a stripe by the warp that owns it, so the read-modify-write
// of a visibility never races and the result does not depend on scheduling; the reference
// serialises the same update across facet processes with named semaphores (degridder.h:236-263).
// Single-visibility maps sum the pack's predictions in registers and subtract once per pack.
#include <cuda_runtime.h>

#include "ddfg_common.cuh"
#include "ddfg_degridblock.cuh"
#include "ddfg_internal.h"
#include "ddfg_queue.cuh"
#include "ddfg_taps.cuh"

namespace ddfg {

// Single-visibility blocks: the warp loads its 32 visibilities' facet-independent inputs once,
// sums the predictions of every facet of the pack in registers, and subtracts the sum from each
// visibility once (one read-modify-write per pack).  Supports up to 8 (two taps per lane) run
// three CTAs per SM (80 registers, a few spilled): 4.5 % faster than two CTAs at 126 registers on
// the combined at-scale chunk.
template <int NPOL, int SLOTS>
__global__ void __launch_bounds__(256, SLOTS == 2 ? 3 : 1)
    degrid_single_q(const ddfg_vis vs, const ddfg_jones js, const __grid_constant__ FacetTable tab,
                    const DegridParams dp, const Sched sc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2 *partial = (float2 *)smem_raw;  // [8 warps][32][32], NPOL == 1 only
  ddfg_facet *sf = (ddfg_facet *)(smem_raw + (NPOL == 1 ? 8 * kPartialBytesPerWarp : 0));
  double *s_n0m1 = (double *)(sf + sc.max_pack);
  __shared__ QueueSmem q;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  float2 *wpart = partial + warp * 32 * 32;
  LaneTaps<SLOTS> lt;
  lt.reset();
  long long static_next = blockIdx.x;
  int cur = -1, npk = 0;
  for (;;) {
    const long long item = queue_next(sc, &q, static_next);
    if (item >= sc.nitems) break;
    const int pack = (int)(item / sc.items_per_pack);
    const long long s0 = slot_stripe(sc, item - (long long)pack * sc.items_per_pack - sc.large_items);
    if (pack != cur) {
      npk = stage_pack(tab, sc, pack, sf, s_n0m1);
      cur = pack;
      __syncthreads();
    }
    const int ns = (int)min(sc.spi, sc.nstripes - s0);
    for (int k; (k = warp_take(&q, ns, lane)) >= 0;) {
      const int64_t b = (s0 + k) * 32 + lane;
      DSingleIn in;
      in.valid = false;
      if (b < vs.nblocks) degrid_load_single(vs, js, b, in);
      if (!__any_sync(0xffffffffu, in.valid)) continue;
      M2 sum;
#pragma unroll
      for (int p = 0; p < 4; ++p) sum.v[p] = czero();
      bool any = false;
      for (int fi = 0; fi < npk; ++fi) {
        const ddfg_facet &f = sf[fi];
        BlockGeom g;
        const bool valid = degrid_single_geom_in(in, f, g);
        TapJob job;
        if (valid) job = tap_job(g, in.gridchan, f);
        float2 mine[NPOL];
        gather_records<NPOL, SLOTS>(valid, job, f, lt, wpart, lane, mine);
        if (valid) {
          const M2 vb = degrid_single_pred<NPOL>(in, vs, js, f, dp, s_n0m1[fi], mine);
#pragma unroll
          for (int p = 0; p < 4; ++p) sum.v[p] = cadd(sum.v[p], vb.v[p]);
          any = true;
        }
      }
      if (any) {
        float2 *vp = (float2 *)vs.vis + (in.irow * vs.nchan + in.ch) * (int64_t)vs.ncorr;
        if (vs.ncorr == 4) {
          float4 a = *(float4 *)vp, c = *(float4 *)(vp + 2);
          a.x -= sum.v[0].x; a.y -= sum.v[0].y; a.z -= sum.v[1].x; a.w -= sum.v[1].y;
          c.x -= sum.v[2].x; c.y -= sum.v[2].y; c.z -= sum.v[3].x; c.w -= sum.v[3].y;
          *(float4 *)vp = a;
          *(float4 *)(vp + 2) = c;
        } else if (vs.ncorr == 2) {
          vp[0] = csub(vp[0], sum.v[0]);
          vp[1] = csub(vp[1], sum.v[3]);
        } else {
          vp[0] = csub(vp[0], sum.v[0]);
        }
      }
    }
  }
}

// Averaged BDA blocks: each lane reads its block's header once per stripe, then every facet of
// the pack forms the footprint, gathers and applies its prediction.  Large-block items give each
// listed block to one warp: lane 0 forms the footprint (row means in the reference's order), the
// warp gathers the taps and applies the prediction lane-strided (degrid_block_apply_warp).
template <int NPOL, int SLOTS>
__global__ void __launch_bounds__(256) degrid_block_q(const ddfg_vis vs, const ddfg_jones js,
                                                      const __grid_constant__ FacetTable tab, const DegridParams dp,
                                                      const Sched sc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2 *partial = (float2 *)smem_raw;  // [8 warps][32][32], NPOL == 1 only
  ddfg_facet *sf = (ddfg_facet *)(smem_raw + (NPOL == 1 ? 8 * kPartialBytesPerWarp : 0));
  double *s_n0m1 = (double *)(sf + sc.max_pack);
  __shared__ QueueSmem q;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  float2 *wpart = partial + warp * 32 * 32;
  LaneTaps<SLOTS> lt;
  lt.reset();
  long long static_next = blockIdx.x;
  int cur = -1, npk = 0;
  for (;;) {
    const long long item = queue_next(sc, &q, static_next);
    if (item >= sc.nitems) break;
    const int pack = (int)(item / sc.items_per_pack);
    const long long r = item - (long long)pack * sc.items_per_pack;
    if (pack != cur) {
      npk = stage_pack(tab, sc, pack, sf, s_n0m1);
      cur = pack;
      __syncthreads();
    }
    if (r < sc.large_items) {
      const long long t0 = r * sc.large_per_item;
      const int nt = (int)min((long long)sc.large_per_item, vs.nlarge - t0);
      for (int k; (k = warp_take(&q, nt, lane)) >= 0;) {
        const int64_t bl = vs.large_blocks[t0 + k];
        if (bl < 0 || bl >= vs.nblocks || block_nvis(vs, bl) <= vs.large_min_vis) continue;
        DegridBlock d;
        degrid_block_header(vs, bl, d);
        for (int fi = 0; fi < npk; ++fi) {
          const ddfg_facet &f = sf[fi];
          BlockGeom g;
          const bool valid = lane == 0 && degrid_block_geom(vs, f, d, g);
          TapJob job;
          if (valid) job = tap_job(g, d.gridchan, f);
          float2 pred[NPOL];
          gather_records<NPOL, SLOTS>(valid, job, f, lt, wpart, lane, pred);
          if (__shfl_sync(0xffffffffu, valid, 0)) degrid_block_apply_warp<NPOL>(vs, js, f, dp, d, pred, 0, lane);
        }
      }
      continue;
    }
    const long long s0 = slot_stripe(sc, r - sc.large_items);
    const int ns = (int)min(sc.spi, sc.nstripes - s0);
    for (int k; (k = warp_take(&q, ns, lane)) >= 0;) {
      const int64_t b = (s0 + k) * 32 + lane;
      const bool inrange = b < vs.nblocks;
      DegridBlock d;
      if (inrange) degrid_block_header(vs, b, d);
      // blocks above the large-block threshold are the large items' work
      const bool mine = inrange && !(vs.nlarge > 0 && (int64_t)d.nrows * (d.ch1 - d.ch0) > vs.large_min_vis);
      for (int fi = 0; fi < npk; ++fi) {
        const ddfg_facet &f = sf[fi];
        BlockGeom g;
        const bool valid = mine && degrid_block_geom(vs, f, d, g);
        TapJob job;
        if (valid) job = tap_job(g, d.gridchan, f);
        float2 pred[NPOL];
        gather_records<NPOL, SLOTS>(valid, job, f, lt, wpart, lane, pred);
        if (valid) degrid_block_apply<NPOL>(vs, js, f, dp, d, pred);
      }
    }
  }
}

}  // namespace ddfg

using namespace ddfg;

namespace {

template <int NP, int SL>
int launch_degrid_table(const ddfg_vis *vs, const ddfg_jones *js, const FacetTable &tab, const DegridParams &dp,
                        Sched sc, const ddfg_batch *batch, cudaStream_t stream) {
  const bool single = vs->single_vis_blocks != 0;
  const size_t smem = (NP == 1 ? 8 * kPartialBytesPerWarp : 0) + (sizeof(ddfg_facet) + sizeof(double)) * sc.max_pack;
  const void *kern = single ? (const void *)degrid_single_q<NP, SL> : (const void *)degrid_block_q<NP, SL>;
  int per_sm = 0;
  int rc = ddfg_kernel_prepare(kern, 256, smem, &per_sm);
  if (rc) return rc;
  if (batch && batch->ctas_per_sm > 0) per_sm = min(per_sm, (int)batch->ctas_per_sm);
  const int ctas = ddfg_num_ctas(per_sm);
  sched_set_regions(sc, (batch && (batch->flags & 4)) ? ctas : 1);
  if (single) degrid_single_q<NP, SL><<<ctas, 256, smem, stream>>>(*vs, *js, tab, dp, sc);
  else degrid_block_q<NP, SL><<<ctas, 256, smem, stream>>>(*vs, *js, tab, dp, sc);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "degrid launch: %s", cudaGetErrorString(e));
  return DDFG_OK;
}

}  // namespace

int ddfg_launch_degrid(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_facet *facets, int nfacets, int policy,
                       int nvispol, const ddfg_batch *batch, cudaStream_t stream) {
  DegridParams dp;
  dp.policy = policy;
  dp.nvispol = nvispol;
  int max_support = 1;
  for (int i = 0; i < nfacets; ++i) max_support = max(max_support, facets[i].max_support);
  const int slots = tap_slots(max_support);
  // One launch per pack: two packs of one launch could update the same visibility at once.
  // Default: every facet of a call in one pack (each visibility read and written once).
  const int per_launch = (batch && batch->facets_per_pack > 0) ? min((int)batch->facets_per_pack, DDFG_TABLE_FACETS)
                                                               : DDFG_TABLE_FACETS;
  const int ngroups = (nfacets + per_launch - 1) / per_launch;  // <= DDFG_MAX_FACETS
  unsigned long long *counters = nullptr;
  if (batch && !(batch->flags & 1)) {
    // counters after the gridder's (a grid and a degrid call may share one workspace)
    counters = (unsigned long long *)batch->workspace + kGridCounters;
    const cudaError_t e = cudaMemsetAsync(counters, 0, sizeof(unsigned long long) * ngroups, stream);
    if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "degrid: %s", cudaGetErrorString(e));
  }
  const long long nstripes = (vs->nblocks + 31) / 32;
  const int nlarge = vs->single_vis_blocks ? 0 : (int)(vs->nlarge < (1LL << 30) ? vs->nlarge : (1LL << 30));
  FacetTable tab;
  for (int g = 0; g < ngroups; ++g) {
    const int f0 = (int)(((long long)g * nfacets) / ngroups), f1 = (int)(((long long)(g + 1) * nfacets) / ngroups);
    const int n = f1 - f0;
    for (int i = 0; i < n; ++i) tab.f[i] = facets[f0 + i];
    Sched sc;
    sc.nfacets = n;
    sc.npacks = 1;
    sc.max_pack = n;
    sc.acc_stride = 0;
    sc.small_stride = 0;
    sc.tiles = 0;
    sc.nstripes = nstripes;
    const long long spi = (batch && batch->stripes_per_item > 0) ? batch->stripes_per_item
                                                                 : max(16LL, min(256LL, nstripes / 1184));
    sc.spi = max(1LL, spi);
    sc.stripe_items = (nstripes + sc.spi - 1) / sc.spi;
    sc.large_per_item = 8;
    sc.large_items = (nlarge + sc.large_per_item - 1) / sc.large_per_item;
    sched_set_regions(sc, 1);
    sc.counter = counters ? counters + g : nullptr;
    int rc;
#define LD(NP, SL) rc = launch_degrid_table<NP, SL>(vs, js, tab, dp, sc, batch, stream)
#define LD_NP(SL)                \
  switch (nvispol) {             \
    case 1: LD(1, SL); break;    \
    case 2: LD(2, SL); break;    \
    case 3: LD(3, SL); break;    \
    default: LD(4, SL); break;   \
  }
    if (slots == 2) { LD_NP(2) } else if (slots == 4) { LD_NP(4) } else { LD_NP(8) }
#undef LD_NP
#undef LD
    if (rc) return rc;
  }
  return DDFG_OK;
}
