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
#include "ddfg_internal.h"

namespace ddfg {

struct FacetPack {
  ddfg_facet f[DDFG_FACETS_PER_LAUNCH];
  int n;
};

struct GridParams {
  int policy;       // GridPolicy
  int nvispol;      // Stokes products formed by the policy
  int dopsf;
  double freq_mean0;  // mean of all channel frequencies (gridder.h:164-171)
};

// Result of one lane's block walk.
template <int NPOL>
struct GridRecord {
  bool valid;
  int gridchan;
  BlockGeom g;
  float2 stokes[NPOL];
  double weight;          // ThisWeight
  double sumjones;        // ThisSumJones
  double sumsqw;          // ThisSumSqWeights
};

// Walk one block for one facet: gridder.h:184-351.
template <int NPOL>
__device__ __forceinline__ void grid_block_record(const ddfg_vis &vs, const ddfg_jones &js, const ddfg_facet &f,
                                                  const GridParams &gp, int64_t b, double n0m1,
                                                  GridRecord<NPOL> &rec, JonesCache &jc) {
  rec.valid = false;
  if (vs.sparsification && !vs.sparsification[b]) return;
  const int64_t start = vs.block_start[b];
  const int nrows_blk = vs.bda_map[2 + b] - 2;
  const int ch0 = vs.bda_map[start], ch1 = vs.bda_map[start + 1];
  const int32_t *rows = vs.bda_map + start + 2;
  const int nchan = vs.nchan, ncorr = vs.ncorr;
  if (nrows_blk <= 0) return;  // no rows: the reference grids nothing either (gridder.h:283)

  jc.reset();
  const double dec = decorr_factor(vs, f, gp.freq_mean0, rows[nrows_blk / 2]);
  const float decf = (float)dec;

  M2 vis_acc;
#pragma unroll
  for (int p = 0; p < 4; ++p) vis_acc.v[p] = czero();
  M2 vmeas;
  vmeas.v[0] = make_float2(decf, 0.f);
  vmeas.v[1] = czero();
  vmeas.v[2] = czero();
  vmeas.v[3] = make_float2(decf, 0.f);
  bool have_psf = false;

  double umean = 0., vmean = 0., wmean = 0., freqmean = 0., thisweight = 0., sumjones = 0., sumsqw = 0.;
  double chanmean = 0.;
  int nvis = 0;
  const float2 *visd = (const float2 *)vs.vis;

  for (int inx = 0; inx < nrows_blk; ++inx) {
    const int64_t irow = rows[inx];
    const double *up = vs.uvw + 3 * irow;
    const double U = up[0], V = up[1], W = up[2];
    // angle = -2 pi (U l0 + V m0 + W n0) / c  ->  phase in turns = -nu * dot / c
    const double dot = U * f.l0 + V * f.m0 + W * n0m1;
    for (int ch = ch0; ch < ch1; ++ch) {
      const int64_t doff = (irow * nchan + ch) * (int64_t)ncorr;
      if (vs.flags[doff]) continue;
      const double nu = vs.freqs[ch];
      const float2 corr = gp.dopsf ? make_float2(1.f, 0.f) : phasor_turns(-nu * dot / kC);
      if (js.mode == 1) {
        const bool chg = jc.update(js, f.idir_kms, f.idir_beam, irow, ch, U, V);
        if ((chg || !have_psf) && gp.dopsf) {
          vmeas = m2_times(jc.j0, jc.j1h);
          vmeas = m2_times(m2_times(jc.j0h, vmeas), jc.j1);
          vmeas = m2_scale(vmeas, make_float2(decf, 0.f));
          have_psf = true;
        }
      }
      if (!gp.dopsf) {
        // Read_4Corr / Read_2Corr_Pad / Read_1Corr_Pad (gridder.h:44-60)
        const float2 *vp = visd + doff;
        if (ncorr == 4) {
          vmeas.v[0] = vp[0]; vmeas.v[1] = vp[1]; vmeas.v[2] = vp[2]; vmeas.v[3] = vp[3];
        } else if (ncorr == 2) {
          vmeas.v[0] = vp[0]; vmeas.v[1] = czero(); vmeas.v[2] = czero(); vmeas.v[3] = vp[1];
        } else {
          vmeas.v[0] = vp[0]; vmeas.v[1] = czero(); vmeas.v[2] = czero(); vmeas.v[3] = vp[0];
        }
      }
      const double fw = (double)vs.weights[irow * nchan + ch];  // * WeightVaryJJ (=1)
      const float2 wgt = cscale(corr, (float)fw);
      const double fwd = fw * dec * dec;
      sumsqw += fwd;
      if (js.mode == 1) {
        if (!gp.dopsf) vmeas = m2_times(m2_times(jc.j0h, vmeas), jc.j1);
        sumjones += (double)jc.bb * fwd;
      }
      // Mulaccum_{4Corr,2Corr_Unpad,1Corr_Unpad} (gridder.h:63-76)
      vis_acc.v[0] = cadd(vis_acc.v[0], cmul(vmeas.v[0], wgt));
      if (ncorr == 4) {
        vis_acc.v[1] = cadd(vis_acc.v[1], cmul(vmeas.v[1], wgt));
        vis_acc.v[2] = cadd(vis_acc.v[2], cmul(vmeas.v[2], wgt));
      }
      if (ncorr >= 2) vis_acc.v[3] = cadd(vis_acc.v[3], cmul(vmeas.v[3], wgt));
      // Block means (gridder.h:272-279), FP64, uncontracted, reference order.
      umean = dadd(umean, dadd(U, dmul(W, f.cu)));
      vmean = dadd(vmean, dadd(V, dmul(W, f.cv)));
      wmean = dadd(wmean, W);
      freqmean = dadd(freqmean, nu);
      thisweight += fw;
      chanmean += (double)vs.chan_map[ch];
      ++nvis;
    }
  }
  if (nvis == 0) return;
  const double dn = (double)nvis;
  umean = umean / dn;
  vmean = vmean / dn;
  wmean = wmean / dn;
  freqmean = freqmean / dn;
  (void)chanmean;

  if (js.mode == 2) {
    // BDAJones: one Jones pair per block at the middle row / middle channel (gridder.h:291-301)
    jc.reset();
    jc.update(js, f.idir_kms, f.idir_beam, rows[nrows_blk / 2], (ch0 + ch1) / 2, umean, vmean);
    if (gp.dopsf) vis_acc = m2_times(m2_times(jc.j0, vis_acc), jc.j1h);
    vis_acc = m2_times(m2_times(jc.j0h, vis_acc), jc.j1);
    sumjones = sumsqw * (double)jc.bb;
  }
  const int gridchan = vs.chan_map[ch0];
  if (gridchan < 0 || gridchan >= f.nband) return;
  const double recip_wvl = freqmean / kC;
  if (!block_geometry(f, umean, vmean, wmean, recip_wvl, rec.g)) return;

  float2 st[4];
  stokes_from_corr(gp.policy, vis_acc, st);
#pragma unroll
  for (int p = 0; p < NPOL; ++p) rec.stokes[p] = st[p];
  rec.valid = true;
  rec.gridchan = gridchan;
  rec.weight = thisweight;
  rec.sumjones = sumjones;
  rec.sumsqw = sumsqw;
}

// Second walk of a valid block for the per-channel Jones sums (gridder.h:254-263, 299-300,
// 369-373), added straight into the CTA's shared accumulators.
__device__ __forceinline__ void grid_block_chan_sums(const ddfg_vis &vs, const ddfg_jones &js, const ddfg_facet &f,
                                                     const GridParams &gp, int64_t b, float block_bb, double mult,
                                                     double *s_chan, JonesCache &jc) {
  const int64_t start = vs.block_start[b];
  const int nrows_blk = vs.bda_map[2 + b] - 2;
  const int ch0 = vs.bda_map[start], ch1 = vs.bda_map[start + 1];
  const int32_t *rows = vs.bda_map + start + 2;
  const double dec = decorr_factor(vs, f, gp.freq_mean0, rows[nrows_blk / 2]);
  const int nchan = vs.nchan;
  jc.reset();
  for (int inx = 0; inx < nrows_blk; ++inx) {
    const int64_t irow = rows[inx];
    const double *up = vs.uvw + 3 * irow;
    for (int ch = ch0; ch < ch1; ++ch) {
      const int64_t doff = (irow * nchan + ch) * (int64_t)vs.ncorr;
      if (vs.flags[doff]) continue;
      const double fwd = (double)vs.weights[irow * nchan + ch] * dec * dec;
      double bbv = (double)block_bb;
      if (js.mode == 1) {
        jc.update(js, f.idir_kms, f.idir_beam, irow, ch, up[0], up[1]);
        bbv = (double)jc.bb;
      }
      atomicAdd(&s_chan[ch], mult * bbv * fwd);
      atomicAdd(&s_chan[nchan + ch], mult * fwd);
    }
  }
}

template <int NPOL>
__global__ void __launch_bounds__(256) grid_kernel(const ddfg_vis vs, const ddfg_jones js, const FacetPack pack,
                                                   const GridParams gp) {
  extern __shared__ double s_acc[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  const int64_t nstripes = (vs.nblocks + 31) / 32;

  for (int fi = 0; fi < pack.n; ++fi) {
    const ddfg_facet &f = pack.f[fi];
    const int npol_used = min(gp.nvispol, f.npol);
    const int nsw = f.nband * f.npol;
    double *s_sumwt = s_acc;                  // [nband][npol]
    double *s_sumj = s_acc + nsw;             // [2][nband]
    double *s_chan = s_sumj + 2 * f.nband;    // [2][nchan]
    const int nacc = nsw + 2 * f.nband + 2 * vs.nchan;
    for (int i = threadIdx.x; i < nacc; i += blockDim.x) s_acc[i] = 0.;
    __syncthreads();

    const double n0m1 = sqrt(1. - f.l0 * f.l0 - f.m0 * f.m0) - 1.;
    float2 *grid = (float2 *)f.grid;
    const size_t plane_sz = (size_t)f.nx * f.ny;
    JonesCache jc;

    for (int64_t s = (int64_t)blockIdx.x * nwarps + warp; s < nstripes; s += (int64_t)gridDim.x * nwarps) {
      const int64_t b = s * 32 + lane;
      GridRecord<NPOL> rec;
      rec.valid = false;
      if (b < vs.nblocks) grid_block_record<NPOL>(vs, js, f, gp, b, n0m1, rec, jc);

      if (rec.valid) {
        for (int p = 0; p < npol_used; ++p) atomicAdd(&s_sumwt[rec.gridchan * f.npol + p], rec.weight);
        if (js.mode != 0) {
          const double m = (double)npol_used;
          atomicAdd(&s_sumj[rec.gridchan], m * rec.sumjones);
          atomicAdd(&s_sumj[f.nband + rec.gridchan], m * rec.sumsqw);
          const float block_bb = jc.bb;  // the block's Jones after a BDAJones walk
          grid_block_chan_sums(vs, js, f, gp, b, block_bb, m, s_chan, jc);
        }
      }

      // Warp-cooperative tap scatter of the 32 records (gridder.h:353-362).
      unsigned mask = __ballot_sync(0xffffffffu, rec.valid);
      while (mask) {
        const int src = __ffs(mask) - 1;
        mask &= mask - 1;
        const int locx = __shfl_sync(0xffffffffu, rec.g.locx, src);
        const int locy = __shfl_sync(0xffffffffu, rec.g.locy, src);
        const int S = __shfl_sync(0xffffffffu, rec.g.S, src);
        const int gch = __shfl_sync(0xffffffffu, rec.gridchan, src);
        const float2 *cf = (const float2 *)__shfl_sync(0xffffffffu, (unsigned long long)rec.g.cf, src);
        float2 sv[NPOL];
#pragma unroll
        for (int p = 0; p < NPOL; ++p) {
          sv[p].x = __shfl_sync(0xffffffffu, rec.stokes[p].x, src);
          sv[p].y = __shfl_sync(0xffffffffu, rec.stokes[p].y, src);
        }
        const int sup = (S - 1) >> 1;
        const int ntap = S * S;
        const unsigned inv = (65536u + (unsigned)S - 1u) / (unsigned)S;  // exact t/S for t < S*S, S <= 63
        float2 *g0 = grid + (size_t)gch * f.npol * plane_sz + (size_t)(locy - sup) * f.nx + (locx - sup);
        for (int t = lane; t < ntap; t += 32) {
          const int sy = (int)(((unsigned)t * inv) >> 16);
          const int sx = t - sy * S;
          const float2 c = __ldg(cf + t);
          float2 *cell = g0 + (size_t)sy * f.nx + sx;
#pragma unroll
          for (int p = 0; p < NPOL; ++p) {
            if (p < npol_used) atomicAdd(cell + (size_t)p * plane_sz, cmul(sv[p], c));
          }
        }
      }
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

}  // namespace ddfg

using namespace ddfg;

int ddfg_launch_grid(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_facet *facets, int nfacets, int policy,
                     int nvispol, int dopsf, int num_ctas, cudaStream_t stream) {
  GridParams gp;
  gp.policy = policy;
  gp.nvispol = nvispol;
  gp.dopsf = dopsf;
  gp.freq_mean0 = vs->freq_mean;
  int max_band = 1;
  for (int i = 0; i < nfacets; ++i) max_band = max(max_band, facets[i].nband * (facets[i].npol + 2));
  const size_t smem = sizeof(double) * ((size_t)max_band + 2 * (size_t)vs->nchan);
  if (smem > 160 * 1024) return ddfg_set_error(DDFG_ESIZE, "grid: too many bands/channels for the shared accumulators");
  for (int f0 = 0; f0 < nfacets; f0 += DDFG_FACETS_PER_LAUNCH) {
    FacetPack pack;
    pack.n = min(DDFG_FACETS_PER_LAUNCH, nfacets - f0);
    for (int i = 0; i < pack.n; ++i) pack.f[i] = facets[f0 + i];
    const int npol = nvispol;
    cudaError_t e;
#define LAUNCH_G(NP)                                                                                   \
  do {                                                                                                 \
    if (smem > 48 * 1024)                                                                              \
      cudaFuncSetAttribute(grid_kernel<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);   \
    grid_kernel<NP><<<num_ctas, 256, smem, stream>>>(*vs, *js, pack, gp);                              \
  } while (0)
    switch (npol) {
      case 1: LAUNCH_G(1); break;
      case 2: LAUNCH_G(2); break;
      case 3: LAUNCH_G(3); break;
      default: LAUNCH_G(4); break;
    }
#undef LAUNCH_G
    e = cudaGetLastError();
    if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "grid launch: %s", cudaGetErrorString(e));
  }
  return DDFG_OK;
}
