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
                                                  BlockGeom &g) {
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
  return block_geometry(f, um, vm, wm, rw, g);
}

// Stokes prediction -> correlations, Jones, smearing, phasor; subtract from the visibilities.
template <int NPOL>
__device__ __forceinline__ void degrid_block_apply(const ddfg_vis &vs, const ddfg_jones &js, const ddfg_facet &f,
                                                   const DegridParams &dp, const DegridBlock &d, const float2 *pred) {
  float2 s[4];
#pragma unroll
  for (int p = 0; p < 4; ++p) s[p] = (p < NPOL) ? pred[p] : czero();
  M2 corr_vis = corr_from_stokes(dp.policy, s);
  JonesCache jc;
  jc.reset();
  const int mid = d.rows[d.nrows / 2];
  if (js.mode == 2) {
    const double *up = vs.uvw + 3 * (int64_t)mid;
    jc.update(js, f.idir_kms, f.idir_beam, mid, (d.ch0 + d.ch1) / 2, up[0], up[1]);
    corr_vis = m2_times(m2_times(jc.j0, corr_vis), m2_herm(jc.j1));
  }
  const float dec = (float)decorr_factor(vs, f, d.freqmean, mid);
  const double n0m1 = sqrt(1. - f.l0 * f.l0 - f.m0 * f.m0) - 1.;
  const int nchan = vs.nchan, ncorr = vs.ncorr;
  float2 *visd = (float2 *)vs.vis;
  for (int inx = 0; inx < d.nrows; ++inx) {
    const int64_t irow = d.rows[inx];
    const double *up = vs.uvw + 3 * irow;
    const double dot = up[0] * f.l0 + up[1] * f.m0 + up[2] * n0m1;
    for (int ch = d.ch0; ch < d.ch1; ++ch) {
      const float2 ph = cscale(phasor_turns(vs.freqs[ch] * dot * kInvC), dec);
      M2 vb;
      if (js.mode == 1) {
        jc.update(js, f.idir_kms, f.idir_beam, irow, ch, up[0], up[1]);
        vb = m2_scale(m2_times(m2_times(jc.j0, corr_vis), m2_herm(jc.j1)), ph);
      } else {
        vb = m2_scale(corr_vis, ph);
      }
      float2 *vp = visd + (irow * nchan + ch) * (int64_t)ncorr;
      // subtractVis<nVisCorr> (degridder.h:43-53)
      if (ncorr == 4) {
        float4 a = *(float4 *)vp, c = *(float4 *)(vp + 2);
        a.x -= vb.v[0].x; a.y -= vb.v[0].y; a.z -= vb.v[1].x; a.w -= vb.v[1].y;
        c.x -= vb.v[2].x; c.y -= vb.v[2].y; c.z -= vb.v[3].x; c.w -= vb.v[3].y;
        *(float4 *)vp = a;
        *(float4 *)(vp + 2) = c;
      } else if (ncorr == 2) {
        vp[0] = csub(vp[0], vb.v[0]);
        vp[1] = csub(vp[1], vb.v[3]);
      } else {
        vp[0] = csub(vp[0], vb.v[0]);
      }
    }
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
