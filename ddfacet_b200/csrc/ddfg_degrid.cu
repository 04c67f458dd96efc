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
#include "ddfg_internal.h"

namespace ddfg {

struct FacetPackD {
  ddfg_facet f[DDFG_FACETS_PER_LAUNCH];
  int n;
};

struct DegridParams {
  int policy;   // DegridPolicy
  int nvispol;  // Stokes planes read from the model grid
};

template <int NPOL>
__global__ void __launch_bounds__(256) degrid_kernel(const ddfg_vis vs, const ddfg_jones js, const FacetPackD pack,
                                                     const DegridParams dp) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  const int64_t nstripes = (vs.nblocks + 31) / 32;
  const int nchan = vs.nchan, ncorr = vs.ncorr;
  float2 *visd = (float2 *)vs.vis;

  for (int64_t s = (int64_t)blockIdx.x * nwarps + warp; s < nstripes; s += (int64_t)gridDim.x * nwarps) {
    const int64_t b = s * 32 + lane;
    const bool inrange = b < vs.nblocks;
    int64_t start = 0;
    int nrows_blk = 0, ch0 = 0, ch1 = 0;
    const int32_t *rows = nullptr;
    if (inrange) {
      start = vs.block_start[b];
      nrows_blk = vs.bda_map[2 + b] - 2;
      ch0 = vs.bda_map[start];
      ch1 = vs.bda_map[start + 1];
      rows = vs.bda_map + start + 2;
    }
    // Facet-independent block means (degridder.h:141-167).
    double freqmean = 0., umean0 = 0., vmean0 = 0., wmean = 0.;
    int nv = 0;
    if (inrange) {
      for (int c = ch0; c < ch1; ++c) freqmean = dadd(freqmean, vs.freqs[c]);
      freqmean = freqmean / (double)(ch1 - ch0);
    }

    for (int fi = 0; fi < pack.n; ++fi) {
      const ddfg_facet &f = pack.f[fi];
      bool valid = false;
      BlockGeom g;
      int gridchan = 0;
      if (inrange) {
        gridchan = vs.chan_map[ch0];
        if (gridchan >= 0 && gridchan < f.nband) {
          double um = 0., vm = 0.;
          wmean = 0.;
          nv = 0;
          for (int inx = 0; inx < nrows_blk; ++inx) {
            const double *up = vs.uvw + 3 * (int64_t)rows[inx];
            um = dadd(um, dadd(up[0], dmul(up[2], f.cu)));
            vm = dadd(vm, dadd(up[1], dmul(up[2], f.cv)));
            wmean = dadd(wmean, up[2]);
            ++nv;
          }
          if (nv > 0) {
            const double dn = (double)nv;
            umean0 = um / dn;
            vmean0 = vm / dn;
            const double wm = wmean / dn;
            valid = block_geometry(f, umean0, vmean0, wm, freqmean / kC, g);
          }
        }
      }

      // Cooperative gather of every valid block's taps.
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
        const int gch = __shfl_sync(0xffffffffu, gridchan, src);
        const float2 *cf = (const float2 *)__shfl_sync(0xffffffffu, (unsigned long long)g.cf, src);
        const int sup = (S - 1) >> 1;
        const int ntap = S * S;
        const unsigned inv = (65536u + (unsigned)S - 1u) / (unsigned)S;
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
      if (!valid) continue;

      // Stokes -> correlations (degridder.h:215), per-block Jones (:216-222).
      M2 corr_vis = corr_from_stokes(dp.policy, mine);
      JonesCache jc;
      jc.reset();
      const int mid = rows[nrows_blk / 2];
      if (js.mode == 2) {
        const double *up = vs.uvw + 3 * (int64_t)mid;
        jc.update(js, f.idir_kms, f.idir_beam, mid, (ch0 + ch1) / 2, up[0], up[1]);
        corr_vis = m2_times(m2_times(jc.j0, corr_vis), jc.j1h);
      }
      const float dec = (float)decorr_factor(vs, f, freqmean, mid);
      const double n0m1 = sqrt(1. - f.l0 * f.l0 - f.m0 * f.m0) - 1.;
      for (int inx = 0; inx < nrows_blk; ++inx) {
        const int64_t irow = rows[inx];
        const double *up = vs.uvw + 3 * irow;
        const double dot = up[0] * f.l0 + up[1] * f.m0 + up[2] * n0m1;
        for (int ch = ch0; ch < ch1; ++ch) {
          float2 ph = phasor_turns(vs.freqs[ch] * dot / kC);
          ph = cscale(ph, dec);
          M2 vb;
          if (js.mode == 1) {
            jc.update(js, f.idir_kms, f.idir_beam, irow, ch, up[0], up[1]);
            vb = m2_times(m2_times(jc.j0, corr_vis), jc.j1h);
            vb = m2_scale(vb, ph);
          } else {
            vb = m2_scale(corr_vis, ph);
          }
          float2 *vp = visd + (irow * nchan + ch) * (int64_t)ncorr;
          // subtractVis<nVisCorr> (degridder.h:43-53)
          if (ncorr == 4) {
            vp[0] = csub(vp[0], vb.v[0]);
            vp[1] = csub(vp[1], vb.v[1]);
            vp[2] = csub(vp[2], vb.v[2]);
            vp[3] = csub(vp[3], vb.v[3]);
          } else if (ncorr == 2) {
            vp[0] = csub(vp[0], vb.v[0]);
            vp[1] = csub(vp[1], vb.v[3]);
          } else {
            vp[0] = csub(vp[0], vb.v[0]);
          }
        }
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
  for (int f0 = 0; f0 < nfacets; f0 += DDFG_FACETS_PER_LAUNCH) {
    FacetPackD pack;
    pack.n = min(DDFG_FACETS_PER_LAUNCH, nfacets - f0);
    for (int i = 0; i < pack.n; ++i) pack.f[i] = facets[f0 + i];
    switch (nvispol) {
      case 1: degrid_kernel<1><<<num_ctas, 256, 0, stream>>>(*vs, *js, pack, dp); break;
      case 2: degrid_kernel<2><<<num_ctas, 256, 0, stream>>>(*vs, *js, pack, dp); break;
      case 3: degrid_kernel<3><<<num_ctas, 256, 0, stream>>>(*vs, *js, pack, dp); break;
      default: degrid_kernel<4><<<num_ctas, 256, 0, stream>>>(*vs, *js, pack, dp); break;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "degrid launch: %s", cudaGetErrorString(e));
  }
  return DDFG_OK;
}
