// BDA W-projection degridder for B200 (sm_100a).
//
// Restates DDFacet's degridder<> (DDFacet/Gridder/degridder.h:55-267):
//
//  * one lane owns one BDA block: band, mean frequency over the block's channels and the
//    unweighted row means of (u + w Cu, v + w Cv, w) in FP64 (degridder.h:138-167), then the
//    W plane, grid location and oversampling phase (degridder.h:170-200);
//  * the warp gathers each block's S x S footprint cooperatively -- lanes on consecutive cells
//    of a CF row, one coalesced load per lane and tap -- and reduces the partial sums with
//    butterfly shuffles (degridder.h:202-212);
//  * the owning lane converts Stokes to correlations, applies the per-block or per-visibility
//    Jones, the facet phasor exp(+i nu angle) (FP64 argument) and the smearing factor, and
//    subtracts the prediction from the visibilities (degridder.h:214-264).
//
// Facets of one call are applied one after the other by the warp that owns a block, so the
// read-modify-write of a visibility never races and the result does not depend on scheduling;
// the reference serialises the same update across facet processes with named semaphores
// (degridder.h:236-263).
#include <cuda_runtime.h>

#include "ddfg_common.cuh"
#include "ddfg_degridblock.cuh"
#include "ddfg_internal.h"
#include "ddfg_taps.cuh"

namespace ddfg {

template <int NPOL, int SLOTS, bool SINGLE>
__global__ void __launch_bounds__(256) degrid_kernel(const ddfg_vis vs, const ddfg_jones js,
                                                        const FacetPackD pack, const DegridParams dp) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ddfg_facet *sf = (ddfg_facet *)smem_raw;
  float2 *partial = (float2 *)(smem_raw + sizeof(ddfg_facet) * DDFG_FACETS_PER_LAUNCH);
  stage_facets(pack, sf);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  const int64_t nstripes = (vs.nblocks + 31) / 32;
  float2 *wpart = partial + warp * 32 * 32;   // [block][lane], NPOL == 1 only
  LaneTaps<SLOTS> lt;
  lt.reset();

  for (int64_t s = (int64_t)blockIdx.x * nwarps + warp; s < nstripes; s += (int64_t)gridDim.x * nwarps) {
    const int64_t b = s * 32 + lane;
    const bool inrange = b < vs.nblocks;
    DegridBlock d;
    if (inrange && !SINGLE) degrid_block_header(vs, b, d);
    // blocks of the large-block list are left to the second loop
    const bool mine = inrange && (SINGLE || !(vs.nlarge > 0 && (int64_t)d.nrows * (d.ch1 - d.ch0) > vs.large_min_vis));
    for (int fi = 0; fi < pack.n; ++fi) {
      const ddfg_facet &f = sf[fi];
      BlockGeom g;
      int sch = 0, sgc = 0;
      int64_t srow = 0;
      bool valid;
      if (SINGLE) valid = inrange && degrid_single_geom(vs, f, b, sch, srow, sgc, g);
      else valid = mine && degrid_block_geom(vs, f, d, g);
      TapJob job;
      if (valid) job = tap_job(g, SINGLE ? sgc : d.gridchan, f);

      float2 pred[NPOL];
      gather_records<NPOL, SLOTS>(valid, job, f, lt, wpart, lane, pred);
      if (valid) {
        if (SINGLE) degrid_single_apply<NPOL>(vs, js, f, dp, sch, srow, pred);
        else degrid_block_apply<NPOL>(vs, js, f, dp, d, pred);
      }
    }
  }
  if (SINGLE) return;
  // Large blocks, one warp each: lane 0 forms the footprint (row means in the reference's
  // order), the warp gathers the taps and applies the prediction to the block's visibilities
  // lane-strided (degrid_block_apply_warp).
  for (int64_t t = (int64_t)blockIdx.x * nwarps + warp; t < vs.nlarge; t += (int64_t)gridDim.x * nwarps) {
    DegridBlock d;
    degrid_block_header(vs, vs.large_blocks[t], d);
    for (int fi = 0; fi < pack.n; ++fi) {
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
}

// Single-visibility blocks: the warp loads its 32 visibilities' facet-independent inputs once,
// sums the predictions of every facet of the launch in registers, and subtracts the sum from
// each visibility once (one read-modify-write per launch instead of one per facet).
template <int NPOL, int SLOTS>
__global__ void __launch_bounds__(256, SLOTS == 2 ? 2 : 1) degrid_single_fi_kernel(const ddfg_vis vs, const ddfg_jones js,
                                                               const FacetPackD pack, const DegridParams dp) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ddfg_facet *sf = (ddfg_facet *)smem_raw;
  double *s_n0m1 = (double *)(sf + DDFG_FACETS_PER_LAUNCH);
  float2 *partial = (float2 *)(s_n0m1 + DDFG_FACETS_PER_LAUNCH);
  stage_facets(pack, sf);
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
  float2 *wpart = partial + warp * 32 * 32;  // [block][lane], NPOL == 1 only
  LaneTaps<SLOTS> lt;
  lt.reset();

  for (int64_t s = (int64_t)blockIdx.x * nwarps + warp; s < nstripes; s += (int64_t)gridDim.x * nwarps) {
    const int64_t b = s * 32 + lane;
    DSingleIn in;
    in.valid = false;
    if (b < vs.nblocks) degrid_load_single(vs, js, b, in);
    if (!__any_sync(0xffffffffu, in.valid)) continue;
    M2 sum;
#pragma unroll
    for (int p = 0; p < 4; ++p) sum.v[p] = czero();
    bool any = false;
    for (int fi = 0; fi < pack.n; ++fi) {
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

}  // namespace ddfg

using namespace ddfg;

int ddfg_launch_degrid(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_facet *facets, int nfacets, int policy,
                       int nvispol, int num_ctas, cudaStream_t stream) {
  DegridParams dp;
  dp.policy = policy;
  dp.nvispol = nvispol;
  int max_support = 1;
  for (int i = 0; i < nfacets; ++i) max_support = max(max_support, facets[i].max_support);
  const int slots = tap_slots(max_support);
  for (int f0 = 0; f0 < nfacets; f0 += DDFG_FACETS_PER_LAUNCH) {
    FacetPackD pack;
    pack.n = min(DDFG_FACETS_PER_LAUNCH, nfacets - f0);
    for (int i = 0; i < pack.n; ++i) pack.f[i] = facets[f0 + i];
    const size_t smem = sizeof(ddfg_facet) * DDFG_FACETS_PER_LAUNCH + (nvispol == 1 ? 8 * kPartialBytesPerWarp : 0);
    const size_t smem_fi = smem + sizeof(double) * DDFG_FACETS_PER_LAUNCH;
#define LAUNCH_D1(NP, SL)                                                                                          \
  do {                                                                                                             \
    cudaFuncSetAttribute(degrid_kernel<NP, SL, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);    \
    degrid_kernel<NP, SL, false><<<ddfg_one_wave(degrid_kernel<NP, SL, false>, 256, smem), 256, smem, stream>>>( \
        *vs, *js, pack, dp);                                                                                       \
  } while (0)
#define LAUNCH_DS(NP, SL)                                                                                          \
  do {                                                                                                             \
    cudaFuncSetAttribute(degrid_single_fi_kernel<NP, SL>, cudaFuncAttributeMaxDynamicSharedMemorySize,             \
                         (int)smem_fi);                                                                            \
    degrid_single_fi_kernel<NP, SL><<<num_ctas, 256, smem_fi, stream>>>(*vs, *js, pack, dp);                       \
  } while (0)
#define LAUNCH_D(NP, SL)                              \
  do {                                                \
    if (vs->single_vis_blocks) LAUNCH_DS(NP, SL);     \
    else LAUNCH_D1(NP, SL);                           \
  } while (0)
#define LAUNCH_D_NP(SL)             \
  switch (nvispol) {                \
    case 1: LAUNCH_D(1, SL); break; \
    case 2: LAUNCH_D(2, SL); break; \
    case 3: LAUNCH_D(3, SL); break; \
    default: LAUNCH_D(4, SL); break; \
  }
    if (slots == 2) { LAUNCH_D_NP(2) } else if (slots == 4) { LAUNCH_D_NP(4) } else { LAUNCH_D_NP(8) }
#undef LAUNCH_D_NP
#undef LAUNCH_D
#undef LAUNCH_DS
#undef LAUNCH_D1
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "degrid launch: %s", cudaGetErrorString(e));
  }
  return DDFG_OK;
}
