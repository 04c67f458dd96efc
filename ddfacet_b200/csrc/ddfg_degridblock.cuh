// The degridder's per-block steps (shared by the direct and the tile-sorted kernels):
// block means and footprint (degridder.h:138-200) and the per-visibility correction and
// subtraction (degridder.h:214-264).
#pragma once
#include "ddfg_common.cuh"

namespace ddfg {

struct FacetPackD {
  ddfg_facet f[DDFG_FACETS_PER_LAUNCH];
  int n;
};

struct DegridParams {
  int policy;   // DegridPolicy
  int nvispol;  // Stokes planes read from the model grid
};

struct DegridBlock {
  int64_t start;
  int nrows, ch0, ch1;
  const int32_t *rows;
  int gridchan;
  double freqmean;
};

__device__ __forceinline__ void degrid_block_header(const ddfg_vis &vs, int64_t b, DegridBlock &d) {
  d.start = vs.block_start[b];
  d.nrows = vs.bda_map[2 + b] - 2;
  d.ch0 = vs.bda_map[d.start];
  d.ch1 = vs.bda_map[d.start + 1];
  d.rows = vs.bda_map + d.start + 2;
  d.gridchan = vs.chan_map[d.ch0 < vs.nchan ? d.ch0 : 0];
  double fm = 0.;
  for (int c = d.ch0; c < d.ch1; ++c) fm = dadd(fm, vs.freqs[c]);
  const int nc = d.ch1 - d.ch0;
  d.freqmean = (nc == 1) ? fm : fm / (double)nc;
}

// Footprint of block b on facet f; false when the reference skips it.
__device__ __forceinline__ bool degrid_block_geom(const ddfg_vis &vs, const ddfg_facet &f, const DegridBlock &d,
                                                  BlockGeom &g, int *dbg = nullptr) {
  if (d.ch1 <= d.ch0 || d.nrows <= 0) return false;
  if (d.gridchan < 0 || d.gridchan >= f.nband) return false;
  double um = 0., vm = 0., wm = 0.;
  for (int inx = 0; inx < d.nrows; ++inx) {
    const double *up = vs.uvw + 3 * (int64_t)d.rows[inx];
    um = dadd(um, dadd(up[0], dmul(up[2], f.cu)));
    vm = dadd(vm, dadd(up[1], dmul(up[2], f.cv)));
    wm = dadd(wm, up[2]);
  }
  if (d.nrows > 1) {
    const double dn = (double)d.nrows;
    um = um / dn;
    vm = vm / dn;
    wm = wm / dn;
  }
  const double rw = (d.ch1 - d.ch0 == 1 && vs.recip_wvl) ? vs.recip_wvl[d.ch0] : d.freqmean / kC;
  return block_geometry(f, um, vm, wm, rw, g, dbg);
}

// The block's Stokes -> correlation prediction with the per-block Jones (BDAJones), smearing
// factor and facet term n0 - 1: what every visibility of the block is derived from.
struct DegridBlockPred {
  M2 corr_vis;
  float dec;
  double n0m1;
};

template <int NPOL>
__device__ __forceinline__ DegridBlockPred degrid_block_pred(const ddfg_vis &vs, const ddfg_jones &js,
                                                             const ddfg_facet &f, const DegridParams &dp,
                                                             const DegridBlock &d, const float2 *pred,
                                                             JonesCache &jc) {
  float2 s[4];
#pragma unroll
  for (int p = 0; p < 4; ++p) s[p] = (p < NPOL) ? pred[p] : czero();
  DegridBlockPred bp;
  bp.corr_vis = corr_from_stokes(dp.policy, s);
  jc.reset();
  const int mid = d.rows[d.nrows / 2];
  if (js.mode == 2) {
    const double *up = vs.uvw + 3 * (int64_t)mid;
    jc.update(js, f.idir_kms, f.idir_beam, mid, (d.ch0 + d.ch1) / 2, up[0], up[1]);
    bp.corr_vis = m2_times(m2_times(jc.j0, bp.corr_vis), m2_herm(jc.j1));
  }
  bp.dec = (float)decorr_factor(vs, f, d.freqmean, mid);
  bp.n0m1 = sqrt(1. - f.l0 * f.l0 - f.m0 * f.m0) - 1.;
  return bp;
}

// One visibility of a block: per-visibility Jones, phasor exp(+i nu angle) and smearing, then
// vis -= (subtractVis<nVisCorr>, degridder.h:43-53, 227-261).
__device__ __forceinline__ void degrid_vis_update(const ddfg_vis &vs, const ddfg_jones &js, const ddfg_facet &f,
                                                  const DegridBlockPred &bp, int64_t irow, int ch,
                                                  JonesCache &jc) {
  const double *up = vs.uvw + 3 * irow;
  const double dot = up[0] * f.l0 + up[1] * f.m0 + up[2] * bp.n0m1;
  const float2 ph = cscale(phasor_turns(vs.freqs[ch] * dot * kInvC), bp.dec);
  M2 vb;
  if (js.mode == 1) {
    jc.update(js, f.idir_kms, f.idir_beam, irow, ch, up[0], up[1]);
    vb = m2_scale(m2_times(m2_times(jc.j0, bp.corr_vis), m2_herm(jc.j1)), ph);
  } else {
    vb = m2_scale(bp.corr_vis, ph);
  }
  float2 *vp = (float2 *)vs.vis + (irow * vs.nchan + ch) * (int64_t)vs.ncorr;
  if (vs.ncorr == 4) {
    float4 a = *(float4 *)vp, c = *(float4 *)(vp + 2);
    a.x -= vb.v[0].x; a.y -= vb.v[0].y; a.z -= vb.v[1].x; a.w -= vb.v[1].y;
    c.x -= vb.v[2].x; c.y -= vb.v[2].y; c.z -= vb.v[3].x; c.w -= vb.v[3].y;
    *(float4 *)vp = a;
    *(float4 *)(vp + 2) = c;
  } else if (vs.ncorr == 2) {
    vp[0] = csub(vp[0], vb.v[0]);
    vp[1] = csub(vp[1], vb.v[3]);
  } else {
    vp[0] = csub(vp[0], vb.v[0]);
  }
}

// Stokes prediction -> correlations, Jones, smearing, phasor; subtract from the visibilities.
template <int NPOL>
__device__ __forceinline__ void degrid_block_apply(const ddfg_vis &vs, const ddfg_jones &js, const ddfg_facet &f,
                                                   const DegridParams &dp, const DegridBlock &d, const float2 *pred) {
  JonesCache jc;
  const DegridBlockPred bp = degrid_block_pred<NPOL>(vs, js, f, dp, d, pred, jc);
  for (int inx = 0; inx < d.nrows; ++inx) {
    const int64_t irow = d.rows[inx];
    for (int ch = d.ch0; ch < d.ch1; ++ch) degrid_vis_update(vs, js, f, bp, irow, ch, jc);
  }
}

// degrid_block_apply of lane src's block by the whole warp (all 32 lanes call it): lanes take the
// block's visibilities in row-major order, lane-strided.  Every visibility's update is
// independent, and with uv-independent Jones terms (no DoScaleJones) a lane's own cache gives the
// values the owner's walk would, so the result is the same.
template <int NPOL>
__device__ __forceinline__ void degrid_block_apply_warp(const ddfg_vis &vs, const ddfg_jones &js,
                                                        const ddfg_facet &f, const DegridParams &dp,
                                                        const DegridBlock &own, const float2 *own_pred, int src,
                                                        int lane) {
  DegridBlock d;
  d.start = __shfl_sync(0xffffffffu, own.start, src);
  d.nrows = __shfl_sync(0xffffffffu, own.nrows, src);
  d.ch0 = __shfl_sync(0xffffffffu, own.ch0, src);
  d.ch1 = __shfl_sync(0xffffffffu, own.ch1, src);
  d.gridchan = __shfl_sync(0xffffffffu, own.gridchan, src);
  d.freqmean = __shfl_sync(0xffffffffu, own.freqmean, src);
  d.rows = vs.bda_map + d.start + 2;
  float2 pred[NPOL];
#pragma unroll
  for (int p = 0; p < NPOL; ++p) {
    pred[p].x = __shfl_sync(0xffffffffu, own_pred[p].x, src);
    pred[p].y = __shfl_sync(0xffffffffu, own_pred[p].y, src);
  }
  JonesCache jc;
  const DegridBlockPred bp = degrid_block_pred<NPOL>(vs, js, f, dp, d, pred, jc);
  const int nch = d.ch1 - d.ch0;
  const int64_t total = (int64_t)d.nrows * nch;
  for (int64_t k = lane; k < total; k += 32) {
    const int inx = (int)(k / nch);
    degrid_vis_update(vs, js, f, bp, d.rows[inx], d.ch0 + (int)(k - (int64_t)inx * nch), jc);
  }
}

// Single-visibility blocks (one row, one channel): degridder.h:138-264 without the loops.
__device__ __forceinline__ bool degrid_single_geom(const ddfg_vis &vs, const ddfg_facet &f, int64_t b, int &ch,
                                                   int64_t &irow, int &gridchan, BlockGeom &g) {
  const int64_t start = vs.block_start[b];
  ch = vs.bda_map[start];
  irow = vs.bda_map[start + 2];
  gridchan = vs.chan_map[ch];
  if (gridchan < 0 || gridchan >= f.nband) return false;
  const double *up = vs.uvw + 3 * irow;
  const double W = up[2];
  const double um = dadd(up[0], dmul(W, f.cu));
  const double vm = dadd(up[1], dmul(W, f.cv));
  const double rw = vs.recip_wvl ? vs.recip_wvl[ch] : vs.freqs[ch] / kC;
  return block_geometry(f, um, vm, W, rw, g);
}

// Facet-independent inputs of a single-visibility block for the degridder, loaded once and
// shared by every facet of a launch.
struct DSingleIn {
  bool valid;
  int ch, gridchan;
  int64_t irow;
  double U, V, W, recip, nu;
  JonesIdx jx;  // valid when js.mode != 0
};

__device__ __forceinline__ void degrid_load_single(const ddfg_vis &vs, const ddfg_jones &js, int64_t b,
                                                   DSingleIn &in) {
  const int64_t start = vs.block_start[b];
  in.ch = vs.bda_map[start];
  in.irow = vs.bda_map[start + 2];
  in.gridchan = vs.chan_map[in.ch];
  in.valid = in.gridchan >= 0;
  const double *up = vs.uvw + 3 * in.irow;
  in.U = up[0];
  in.V = up[1];
  in.W = up[2];
  in.recip = vs.recip_wvl ? vs.recip_wvl[in.ch] : vs.freqs[in.ch] / kC;
  in.nu = vs.freqs[in.ch];
  if (js.mode != 0) in.jx = jones_idx(js, in.irow, in.ch);
}

// degrid_single_geom from preloaded inputs.
__device__ __forceinline__ bool degrid_single_geom_in(const DSingleIn &in, const ddfg_facet &f, BlockGeom &g) {
  if (!in.valid || in.gridchan >= f.nband) return false;
  const double um = dadd(in.U, dmul(in.W, f.cu));
  const double vm = dadd(in.V, dmul(in.W, f.cv));
  return block_geometry(f, um, vm, in.W, in.recip, g);
}

// The prediction of facet f for a single visibility (what degrid_single_apply subtracts):
// Stokes -> correlations, J0 M J1^H, phasor exp(+i nu angle) and smearing (degridder.h:214-261).
template <int NPOL>
__device__ __forceinline__ M2 degrid_single_pred(const DSingleIn &in, const ddfg_vis &vs, const ddfg_jones &js,
                                                 const ddfg_facet &f, const DegridParams &dp, double n0m1,
                                                 const float2 *pred) {
  float2 s[4];
#pragma unroll
  for (int p = 0; p < 4; ++p) s[p] = (p < NPOL) ? pred[p] : czero();
  M2 cv = corr_from_stokes(dp.policy, s);
  if (js.mode != 0) {
    M2 j0, j1;
    float bb;
    jones_pair_at(js, f.idir_kms, f.idir_beam, in.jx, in.U, in.V, j0, j1, bb);
    cv = m2_times(m2_times(j0, cv), m2_herm(j1));
  }
  const float dec = (float)decorr_factor(vs, f, in.nu, in.irow);
  const float2 ph = cscale(phasor_turns(in.nu * (in.U * f.l0 + in.V * f.m0 + in.W * n0m1) * kInvC), dec);
  return m2_scale(cv, ph);
}

template <int NPOL>
__device__ __forceinline__ void degrid_single_apply(const ddfg_vis &vs, const ddfg_jones &js, const ddfg_facet &f,
                                                    const DegridParams &dp, int ch, int64_t irow, const float2 *pred) {
  float2 s[4];
#pragma unroll
  for (int p = 0; p < 4; ++p) s[p] = (p < NPOL) ? pred[p] : czero();
  M2 cv = corr_from_stokes(dp.policy, s);
  const double *up = vs.uvw + 3 * irow;
  const double nu = vs.freqs[ch];
  if (js.mode != 0) {
    M2 j0, j1;
    float bb;
    jones_pair(js, f.idir_kms, f.idir_beam, irow, ch, up[0], up[1], j0, j1, bb);
    cv = m2_times(m2_times(j0, cv), m2_herm(j1));
  }
  const float dec = (float)decorr_factor(vs, f, nu, irow);
  const double n0m1 = sqrt(1. - f.l0 * f.l0 - f.m0 * f.m0) - 1.;
  const float2 ph = cscale(phasor_turns(nu * (up[0] * f.l0 + up[1] * f.m0 + up[2] * n0m1) * kInvC), dec);
  const M2 vb = m2_scale(cv, ph);
  float2 *vp = (float2 *)vs.vis + (irow * vs.nchan + ch) * (int64_t)vs.ncorr;
  if (vs.ncorr == 4) {
    float4 a = *(float4 *)vp, c = *(float4 *)(vp + 2);
    a.x -= vb.v[0].x; a.y -= vb.v[0].y; a.z -= vb.v[1].x; a.w -= vb.v[1].y;
    c.x -= vb.v[2].x; c.y -= vb.v[2].y; c.z -= vb.v[3].x; c.w -= vb.v[3].y;
    *(float4 *)vp = a;
    *(float4 *)(vp + 2) = c;
  } else if (vs.ncorr == 2) {
    vp[0] = csub(vp[0], vb.v[0]);
    vp[1] = csub(vp[1], vb.v[3]);
  } else {
    vp[0] = csub(vp[0], vb.v[0]);
  }
}

}  // namespace ddfg
