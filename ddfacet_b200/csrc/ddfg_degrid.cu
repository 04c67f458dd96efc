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

namespace ddfg {

template <int NPOL>
__global__ void __launch_bounds__(256) degrid_kernel(const ddfg_vis vs, const ddfg_jones js, const FacetPackD pack,
                                                     const DegridParams dp) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ddfg_facet *sf = (ddfg_facet *)smem_raw;
  stage_facets(pack, sf);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  const int64_t nstripes = (vs.nblocks + 31) / 32;

  for (int64_t s = (int64_t)blockIdx.x * nwarps + warp; s < nstripes; s += (int64_t)gridDim.x * nwarps) {
    const int64_t b = s * 32 + lane;
    const bool inrange = b < vs.nblocks;
    DegridBlock d;
    if (inrange) degrid_block_header(vs, b, d);
    for (int fi = 0; fi < pack.n; ++fi) {
      const ddfg_facet &f = sf[fi];
      BlockGeom g;
      const bool valid = inrange && degrid_block_geom(vs, f, d, g);
      const int gridchan = inrange ? d.gridchan : 0;

      // Cooperative gather of every valid block's taps (degridder.h:202-212).
      float2 mine[NPOL];
#pragma unroll
      for (int p = 0; p < NPOL; ++p) mine[p] = czero();
      const size_t plane_sz = (size_t)f.nx * f.ny;
      const float2 *grid = (const float2 *)f.grid;
      unsigned mask = __ballot_sync(0xffffffffu, valid);
      while (mask) {
        const int src = __ffs(mask) - 1;
        mask &= mask - 1;
        const int locx = __shfl_sync(0xffffffffu, g.locx, src);
        const int locy = __shfl_sync(0xffffffffu, g.locy, src);
        const int S = __shfl_sync(0xffffffffu, g.S, src);
        const unsigned inv = __shfl_sync(0xffffffffu, g.inv, src);
        const int gch = __shfl_sync(0xffffffffu, gridchan, src);
        const float2 *cf = (const float2 *)__shfl_sync(0xffffffffu, (unsigned long long)g.cf, src);
        const int sup = (S - 1) >> 1;
        const int ntap = S * S;
        const float2 *g0 = grid + (size_t)gch * f.npol * plane_sz + (size_t)(locy - sup) * f.nx + (locx - sup);
        float2 acc[NPOL];
#pragma unroll
        for (int p = 0; p < NPOL; ++p) acc[p] = czero();
        for (int t = lane; t < ntap; t += 32) {
          const int sy = (int)(((unsigned)t * inv) >> 16);
          const int sx = t - sy * S;
          const float2 c = __ldg(cf + t);
          const float2 *cell = g0 + (size_t)sy * f.nx + sx;
#pragma unroll
          for (int p = 0; p < NPOL; ++p) acc[p] = cadd(acc[p], cmul(__ldg(cell + (size_t)p * plane_sz), c));
        }
#pragma unroll
        for (int p = 0; p < NPOL; ++p) {
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) {
            acc[p].x += __shfl_xor_sync(0xffffffffu, acc[p].x, o);
            acc[p].y += __shfl_xor_sync(0xffffffffu, acc[p].y, o);
          }
        }
        if (lane == src) {
#pragma unroll
          for (int p = 0; p < NPOL; ++p) mine[p] = acc[p];
        }
      }
      if (valid) degrid_block_apply<NPOL>(vs, js, f, dp, d, mine);
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
  for (int f0 = 0; f0 < nfacets; f0 += DDFG_FACETS_PER_LAUNCH) {
    FacetPackD pack;
    pack.n = min(DDFG_FACETS_PER_LAUNCH, nfacets - f0);
    for (int i = 0; i < pack.n; ++i) pack.f[i] = facets[f0 + i];
    const size_t smem = sizeof(ddfg_facet) * pack.n;
    switch (nvispol) {
      case 1: degrid_kernel<1><<<num_ctas, 256, smem, stream>>>(*vs, *js, pack, dp); break;
      case 2: degrid_kernel<2><<<num_ctas, 256, smem, stream>>>(*vs, *js, pack, dp); break;
      case 3: degrid_kernel<3><<<num_ctas, 256, smem, stream>>>(*vs, *js, pack, dp); break;
      default: degrid_kernel<4><<<num_ctas, 256, smem, stream>>>(*vs, *js, pack, dp); break;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "degrid launch: %s", cudaGetErrorString(e));
  }
  return DDFG_OK;
}
