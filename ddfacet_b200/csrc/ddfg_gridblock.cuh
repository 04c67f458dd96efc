// The gridder's per-block walk (shared by the direct and the tile-sorted gridding kernels).
#pragma once
#include "ddfg_common.cuh"

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
  int ch0;                // first channel of the block
  bool single_chan;       // one channel: its channel sums are the block sums
};

// Facet-independent inputs of a single-visibility block (one row, one channel), loaded once
// and shared by every facet of a launch.
struct SingleIn {
  bool valid;
  int ch, gridchan;
  int64_t irow;
  double U, V, W, recip, nu, fw;
  M2 vm;        // the visibilities (unused for the PSF)
  JonesIdx jx;  // valid when js.mode != 0
};

__device__ __forceinline__ void load_single(const ddfg_vis &vs, const ddfg_jones &js, const GridParams &gp, int64_t b,
                                            SingleIn &in) {
  in.valid = false;
  if (vs.sparsification && !vs.sparsification[b]) return;
  const int64_t start = vs.block_start[b];
  const int ch = vs.bda_map[start];
  const int64_t irow = vs.bda_map[start + 2];
  const int64_t doff = (irow * vs.nchan + ch) * (int64_t)vs.ncorr;
  if (vs.flags[doff]) return;
  const int gridchan = vs.chan_map[ch];
  if (gridchan < 0) return;
  in.ch = ch;
  in.irow = irow;
  in.gridchan = gridchan;
  in.U = vs.uvw[3 * irow];
  in.V = vs.uvw[3 * irow + 1];
  in.W = vs.uvw[3 * irow + 2];
  in.recip = vs.recip_wvl ? vs.recip_wvl[ch] : vs.freqs[ch] / kC;
  in.nu = vs.freqs[ch];
  in.fw = (double)vs.weights[irow * vs.nchan + ch];
  if (!gp.dopsf) {
    const float2 *vp = (const float2 *)vs.vis + doff;
    if (vs.ncorr == 4) {
      const float4 a = *(const float4 *)vp, c = *(const float4 *)(vp + 2);
      in.vm.v[0] = make_float2(a.x, a.y); in.vm.v[1] = make_float2(a.z, a.w);
      in.vm.v[2] = make_float2(c.x, c.y); in.vm.v[3] = make_float2(c.z, c.w);
    } else if (vs.ncorr == 2) {
      in.vm.v[0] = vp[0]; in.vm.v[1] = czero(); in.vm.v[2] = czero(); in.vm.v[3] = vp[1];
    } else {
      in.vm.v[0] = vp[0]; in.vm.v[1] = czero(); in.vm.v[2] = czero(); in.vm.v[3] = vp[0];
    }
  }
  if (js.mode != 0) in.jx = jones_idx(js, irow, ch);
  in.valid = true;
}

// The facet-dependent part of a single-visibility block: the walk of gridder.h:184-351 with its
// loops, means and cache collapsed.  Sums over one term equal that term exactly (0 + x == x,
// x / 1 == x), so the FP64 index inputs are the same as the reference's.
template <int NPOL>
__device__ __forceinline__ void grid_single_facet(const SingleIn &in, const ddfg_vis &vs, const ddfg_jones &js,
                                                  const ddfg_facet &f, const GridParams &gp, double n0m1,
                                                  GridRecord<NPOL> &rec) {
  rec.valid = false;
  if (!in.valid || in.gridchan >= f.nband) return;
  const double U = in.U, V = in.V, W = in.W;
  const double umean = dadd(U, dmul(W, f.cu));
  const double vmean = dadd(V, dmul(W, f.cv));
  if (!block_geometry(f, umean, vmean, W, in.recip, rec.g)) return;

  const double dec = decorr_factor(vs, f, gp.freq_mean0, in.irow);
  const float decf = (float)dec;
  M2 vm;
  if (gp.dopsf) {
    vm.v[0] = make_float2(decf, 0.f); vm.v[1] = czero(); vm.v[2] = czero(); vm.v[3] = make_float2(decf, 0.f);
  } else {
    vm = in.vm;
  }
  const double fw = in.fw;
  const double fwd = fw * dec * dec;
  double sumjones = 0.;
  if (js.mode != 0) {
    M2 j0, j1;
    float bb;
    // mode 1 normalises with the row's uvw, mode 2 with the block mean (gridder.h:236, 294)
    jones_pair_at(js, f.idir_kms, f.idir_beam, in.jx, js.mode == 1 ? U : umean, js.mode == 1 ? V : vmean, j0, j1,
                  bb);
    // PSF: J0^H J0 J1^H J1 times the smearing factor in both modes (gridder.h:236-242, 295-297)
    if (gp.dopsf) vm = m2_scale(m2_times(m2_times(m2_herm(j0), m2_times(j0, m2_herm(j1))), j1), make_float2(decf, 0.f));
    else vm = m2_times(m2_times(m2_herm(j0), vm), j1);
    sumjones = (double)bb * fwd;
  }
  const float2 corr = gp.dopsf ? make_float2(1.f, 0.f)
                               : phasor_turns(-in.nu * (U * f.l0 + V * f.m0 + W * n0m1) * kInvC);
  const float2 wgt = cscale(corr, (float)fw);
  M2 acc;
  acc.v[0] = cmul(vm.v[0], wgt);
  acc.v[1] = vs.ncorr == 4 ? cmul(vm.v[1], wgt) : czero();
  acc.v[2] = vs.ncorr == 4 ? cmul(vm.v[2], wgt) : czero();
  acc.v[3] = vs.ncorr >= 2 ? cmul(vm.v[3], wgt) : czero();
  float2 st[4];
  stokes_from_corr(gp.policy, acc, st);
#pragma unroll
  for (int p = 0; p < NPOL; ++p) rec.stokes[p] = st[p];
  rec.valid = true;
  rec.gridchan = in.gridchan;
  rec.weight = fw;
  rec.sumjones = sumjones;
  rec.sumsqw = fwd;
  rec.ch0 = in.ch;
  rec.single_chan = true;
}

// A block of exactly one row and one channel (every block of a map built without averaging).
template <int NPOL>
__device__ __forceinline__ void grid_single_record(const ddfg_vis &vs, const ddfg_jones &js, const ddfg_facet &f,
                                                   const GridParams &gp, int64_t b, double n0m1,
                                                   GridRecord<NPOL> &rec) {
  SingleIn in;
  load_single(vs, js, gp, b, in);
  grid_single_facet<NPOL>(in, vs, js, f, gp, n0m1, rec);
}

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
  int nvis = 0, last_ch = ch0;
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
      const float2 corr = gp.dopsf ? make_float2(1.f, 0.f) : phasor_turns(-nu * dot * kInvC);
      if (js.mode == 1) {
        const bool chg = jc.update(js, f.idir_kms, f.idir_beam, irow, ch, U, V);
        if ((chg || !have_psf) && gp.dopsf) {
          vmeas = m2_times(jc.j0, m2_herm(jc.j1));
          vmeas = m2_times(m2_times(m2_herm(jc.j0), vmeas), jc.j1);
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
        if (!gp.dopsf) vmeas = m2_times(m2_times(m2_herm(jc.j0), vmeas), jc.j1);
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
      last_ch = ch;
      ++nvis;
    }
  }
  if (nvis == 0) return;
  if (nvis > 1) {  // x / 1.0 == x exactly, so single-visibility blocks skip the divisions
    const double dn = (double)nvis;
    umean = umean / dn;
    vmean = vmean / dn;
    wmean = wmean / dn;
    freqmean = freqmean / dn;
  }

  if (js.mode == 2) {
    // BDAJones: one Jones pair per block at the middle row / middle channel (gridder.h:291-301)
    jc.reset();
    jc.update(js, f.idir_kms, f.idir_beam, rows[nrows_blk / 2], (ch0 + ch1) / 2, umean, vmean);
    if (gp.dopsf) vis_acc = m2_times(m2_times(jc.j0, vis_acc), m2_herm(jc.j1));
    vis_acc = m2_times(m2_times(m2_herm(jc.j0), vis_acc), jc.j1);
    sumjones = sumsqw * (double)jc.bb;
  }
  const int gridchan = vs.chan_map[ch0];
  if (gridchan < 0 || gridchan >= f.nband) return;
  // FreqMean / C; a single-visibility block's mean is its channel frequency, whose quotient
  // the host tabulated with the same IEEE division.
  const double recip_wvl = (nvis == 1 && vs.recip_wvl) ? vs.recip_wvl[last_ch] : freqmean / kC;
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
  rec.ch0 = ch0;
  rec.single_chan = (ch1 - ch0 == 1);
}

// Per-channel Jones sums of a valid block (gridder.h:254-263, 299-300, 369-373) into the CTA's
// shared accumulators: the block sums for a single-channel block, else a second walk.
template <int NPOL>
__device__ __forceinline__ void grid_block_add_chan_sums(const ddfg_vis &vs, const ddfg_jones &js,
                                                         const ddfg_facet &f, const GridParams &gp, int64_t b,
                                                         const GridRecord<NPOL> &rec, double mult, double *s_chan,
                                                         JonesCache &jc);

// Second walk of a valid block for the per-channel Jones sums.
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
__device__ __forceinline__ void grid_block_add_chan_sums(const ddfg_vis &vs, const ddfg_jones &js,
                                                         const ddfg_facet &f, const GridParams &gp, int64_t b,
                                                         const GridRecord<NPOL> &rec, double mult, double *s_chan,
                                                         JonesCache &jc) {
  if (rec.single_chan) {
    atomicAdd(&s_chan[rec.ch0], mult * rec.sumjones);
    atomicAdd(&s_chan[vs.nchan + rec.ch0], mult * rec.sumsqw);
  } else {
    const float block_bb = jc.bb;
    grid_block_chan_sums(vs, js, f, gp, b, block_bb, mult, s_chan, jc);
  }
}

// The warp's 32 records' contributions to the weight and Jones sums (gridder.h:363-373): one
// shared-memory update per warp when every valid lane grids into the same band, per lane
// otherwise.  Must be called by all 32 lanes.
template <int NPOL, bool SINGLE = false>
__device__ __forceinline__ void warp_add_block_sums(const ddfg_vis &vs, const ddfg_jones &js, const ddfg_facet &f,
                                                    const GridParams &gp, int64_t b, const GridRecord<NPOL> &rec,
                                                    int npol_used, double *a_sumwt, double *a_sumj, double *a_chan,
                                                    JonesCache &jc, bool chan_sums_done = false) {
  const unsigned vmask = __ballot_sync(0xffffffffu, rec.valid);
  if (!vmask) return;
  const int lane = threadIdx.x & 31;
  const int g0 = __shfl_sync(0xffffffffu, rec.gridchan, __ffs(vmask) - 1);
  const bool same = __all_sync(0xffffffffu, !rec.valid || rec.gridchan == g0);
  double wsum = rec.valid ? rec.weight : 0., jsum = rec.valid ? rec.sumjones : 0., qsum = rec.valid ? rec.sumsqw : 0.;
  if (same) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
      if (js.mode != 0) {
        jsum += __shfl_xor_sync(0xffffffffu, jsum, o);
        qsum += __shfl_xor_sync(0xffffffffu, qsum, o);
      }
    }
  }
  if ((same && lane == 0) || (!same && rec.valid)) {
    const int g = same ? g0 : rec.gridchan;
    for (int p = 0; p < npol_used; ++p) atomicAdd(&a_sumwt[g * f.npol + p], wsum);
    if (js.mode != 0) {
      atomicAdd(&a_sumj[g], (double)npol_used * jsum);
      atomicAdd(&a_sumj[f.nband + g], (double)npol_used * qsum);
    }
  }
  if (js.mode != 0 && rec.valid && !chan_sums_done) {
    if (SINGLE) {
      atomicAdd(&a_chan[rec.ch0], (double)npol_used * rec.sumjones);
      atomicAdd(&a_chan[vs.nchan + rec.ch0], (double)npol_used * rec.sumsqw);
    } else {
      grid_block_add_chan_sums<NPOL>(vs, js, f, gp, b, rec, (double)npol_used, a_chan, jc);
    }
  }
}

// Visibilities of block b (rows x channels, flagged ones included).
__device__ __forceinline__ int64_t block_nvis(const ddfg_vis &vs, int64_t b) {
  const int64_t start = vs.block_start[b];
  return (int64_t)(vs.bda_map[2 + b] - 2) * (vs.bda_map[start + 1] - vs.bda_map[start]);
}

// The FP64 block means of grid_block_record in the reference's order (gridder.h:272-279): one
// lane, only the flags read per visibility.  Keeping this sum sequential keeps every integer index
// derived from it bit-exact.
struct BlockMeans {
  double u, v, w, nu;
  int nvis, last_ch;
};

__device__ __forceinline__ BlockMeans grid_block_means(const ddfg_vis &vs, const ddfg_facet &f, int64_t b) {
  BlockMeans m;
  m.u = m.v = m.w = m.nu = 0.;
  m.nvis = 0;
  const int64_t start = vs.block_start[b];
  const int nrows_blk = vs.bda_map[2 + b] - 2;
  const int ch0 = vs.bda_map[start], ch1 = vs.bda_map[start + 1];
  m.last_ch = ch0;
  const int32_t *rows = vs.bda_map + start + 2;
  for (int inx = 0; inx < nrows_blk; ++inx) {
    const int64_t irow = rows[inx];
    const double *up = vs.uvw + 3 * irow;
    const double W = up[2];
    const double tu = dadd(up[0], dmul(W, f.cu)), tv = dadd(up[1], dmul(W, f.cv));
    const unsigned char *fl = vs.flags + irow * vs.nchan * (int64_t)vs.ncorr;
    for (int ch = ch0; ch < ch1; ++ch) {
      if (fl[(int64_t)ch * vs.ncorr]) continue;
      m.u = dadd(m.u, tu);
      m.v = dadd(m.v, tv);
      m.w = dadd(m.w, W);
      m.nu = dadd(m.nu, vs.freqs[ch]);
      m.last_ch = ch;
      ++m.nvis;
    }
  }
  return m;
}

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

__device__ __forceinline__ float warp_sum(float x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// grid_block_record of lane src's block b by the whole warp (all 32 lanes call it; the Jones
// terms must not depend on uv, i.e. no DoScaleJones): lanes take the block's visibilities in
// row-major order, lane-strided, and the weighted visibility and weight sums are reduced across
// the warp; the FP64 means come from the owner's sequential walk (grid_block_means, passed in by
// lane src).  With uv-independent Jones terms every lane's cache gives the owner's values.  Lane src receives the record.  When the
// block is valid and carries Jones sums over several channels, the per-channel sums are added to
// a_chan here (the caller passes chan_sums_done to warp_add_block_sums).
template <int NPOL>
__device__ __forceinline__ void grid_block_record_warp(const ddfg_vis &vs, const ddfg_jones &js, const ddfg_facet &f,
                                                       const GridParams &gp, int64_t b_own, const BlockMeans &m_own,
                                                       double n0m1, int src, int lane, int npol_used, double *a_chan,
                                                       GridRecord<NPOL> &rec) {
  const int64_t b = __shfl_sync(0xffffffffu, b_own, src);
  BlockMeans bm;
  bm.u = __shfl_sync(0xffffffffu, m_own.u, src);
  bm.v = __shfl_sync(0xffffffffu, m_own.v, src);
  bm.w = __shfl_sync(0xffffffffu, m_own.w, src);
  bm.nu = __shfl_sync(0xffffffffu, m_own.nu, src);
  bm.nvis = __shfl_sync(0xffffffffu, m_own.nvis, src);
  bm.last_ch = __shfl_sync(0xffffffffu, m_own.last_ch, src);
  const int64_t start = vs.block_start[b];
  const int nrows_blk = vs.bda_map[2 + b] - 2;
  const int ch0 = vs.bda_map[start], ch1 = vs.bda_map[start + 1];
  const int32_t *rows = vs.bda_map + start + 2;
  const int nchan = vs.nchan, ncorr = vs.ncorr;
  const int nch = ch1 - ch0;
  const int64_t total = (int64_t)nrows_blk * nch;
  const double dec = decorr_factor(vs, f, gp.freq_mean0, rows[nrows_blk / 2]);
  const float decf = (float)dec;
  JonesCache jc;
  jc.reset();
  M2 vis_acc;
#pragma unroll
  for (int p = 0; p < 4; ++p) vis_acc.v[p] = czero();
  M2 vmeas;
  vmeas.v[0] = make_float2(decf, 0.f);
  vmeas.v[1] = czero();
  vmeas.v[2] = czero();
  vmeas.v[3] = make_float2(decf, 0.f);
  bool have_psf = false;
  double thisweight = 0., sumjones = 0., sumsqw = 0.;
  const float2 *visd = (const float2 *)vs.vis;
  for (int64_t k = lane; k < total; k += 32) {
    const int inx = (int)(k / nch);
    const int ch = ch0 + (int)(k - (int64_t)inx * nch);
    const int64_t irow = rows[inx];
    const int64_t doff = (irow * nchan + ch) * (int64_t)ncorr;
    if (vs.flags[doff]) continue;
    const double *up = vs.uvw + 3 * irow;
    const double U = up[0], V = up[1], W = up[2];
    const double dot = U * f.l0 + V * f.m0 + W * n0m1;
    const double nu = vs.freqs[ch];
    const float2 corr = gp.dopsf ? make_float2(1.f, 0.f) : phasor_turns(-nu * dot * kInvC);
    if (js.mode == 1) {
      const bool chg = jc.update(js, f.idir_kms, f.idir_beam, irow, ch, U, V);
      if ((chg || !have_psf) && gp.dopsf) {
        vmeas = m2_times(jc.j0, m2_herm(jc.j1));
        vmeas = m2_times(m2_times(m2_herm(jc.j0), vmeas), jc.j1);
        vmeas = m2_scale(vmeas, make_float2(decf, 0.f));
        have_psf = true;
      }
    }
    if (!gp.dopsf) {
      const float2 *vp = visd + doff;
      if (ncorr == 4) {
        vmeas.v[0] = vp[0]; vmeas.v[1] = vp[1]; vmeas.v[2] = vp[2]; vmeas.v[3] = vp[3];
      } else if (ncorr == 2) {
        vmeas.v[0] = vp[0]; vmeas.v[1] = czero(); vmeas.v[2] = czero(); vmeas.v[3] = vp[1];
      } else {
        vmeas.v[0] = vp[0]; vmeas.v[1] = czero(); vmeas.v[2] = czero(); vmeas.v[3] = vp[0];
      }
    }
    const double fw = (double)vs.weights[irow * nchan + ch];
    const float2 wgt = cscale(corr, (float)fw);
    const double fwd = fw * dec * dec;
    sumsqw += fwd;
    if (js.mode == 1) {
      if (!gp.dopsf) vmeas = m2_times(m2_times(m2_herm(jc.j0), vmeas), jc.j1);
      sumjones += (double)jc.bb * fwd;
    }
    vis_acc.v[0] = cadd(vis_acc.v[0], cmul(vmeas.v[0], wgt));
    if (ncorr == 4) {
      vis_acc.v[1] = cadd(vis_acc.v[1], cmul(vmeas.v[1], wgt));
      vis_acc.v[2] = cadd(vis_acc.v[2], cmul(vmeas.v[2], wgt));
    }
    if (ncorr >= 2) vis_acc.v[3] = cadd(vis_acc.v[3], cmul(vmeas.v[3], wgt));
    thisweight += fw;
  }
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    vis_acc.v[p].x = warp_sum(vis_acc.v[p].x);
    vis_acc.v[p].y = warp_sum(vis_acc.v[p].y);
  }
  thisweight = warp_sum(thisweight);
  sumsqw = warp_sum(sumsqw);
  if (js.mode == 1) sumjones = warp_sum(sumjones);
  if (bm.nvis == 0) return;
  double umean = bm.u, vmean = bm.v, wmean = bm.w, freqmean = bm.nu;
  if (bm.nvis > 1) {
    const double dn = (double)bm.nvis;
    umean = umean / dn;
    vmean = vmean / dn;
    wmean = wmean / dn;
    freqmean = freqmean / dn;
  }
  if (js.mode == 2) {
    jc.reset();
    jc.update(js, f.idir_kms, f.idir_beam, rows[nrows_blk / 2], (ch0 + ch1) / 2, umean, vmean);
    if (gp.dopsf) vis_acc = m2_times(m2_times(jc.j0, vis_acc), m2_herm(jc.j1));
    vis_acc = m2_times(m2_times(m2_herm(jc.j0), vis_acc), jc.j1);
    sumjones = sumsqw * (double)jc.bb;
  }
  const int gridchan = vs.chan_map[ch0];
  if (gridchan < 0 || gridchan >= f.nband) return;
  const double recip_wvl = (bm.nvis == 1 && vs.recip_wvl) ? vs.recip_wvl[bm.last_ch] : freqmean / kC;
  BlockGeom g;
  if (!block_geometry(f, umean, vmean, wmean, recip_wvl, g)) return;
  // per-channel Jones sums of the valid block (grid_block_chan_sums), lane-strided
  if (js.mode != 0 && nch > 1) {
    const float block_bb = jc.bb;
    JonesCache jc2;
    jc2.reset();
    const double mult = (double)npol_used;
    for (int64_t k = lane; k < total; k += 32) {
      const int inx = (int)(k / nch);
      const int ch = ch0 + (int)(k - (int64_t)inx * nch);
      const int64_t irow = rows[inx];
      if (vs.flags[(irow * nchan + ch) * (int64_t)ncorr]) continue;
      const double fwd = (double)vs.weights[irow * nchan + ch] * dec * dec;
      double bbv = (double)block_bb;
      if (js.mode == 1) {
        const double *up = vs.uvw + 3 * irow;
        jc2.update(js, f.idir_kms, f.idir_beam, irow, ch, up[0], up[1]);
        bbv = (double)jc2.bb;
      }
      atomicAdd(&a_chan[ch], mult * bbv * fwd);
      atomicAdd(&a_chan[nchan + ch], mult * fwd);
    }
  }
  if (lane == src) {
    float2 st[4];
    stokes_from_corr(gp.policy, vis_acc, st);
#pragma unroll
    for (int p = 0; p < NPOL; ++p) rec.stokes[p] = st[p];
    rec.g = g;
    rec.valid = true;
    rec.gridchan = gridchan;
    rec.weight = thisweight;
    rec.sumjones = sumjones;
    rec.sumsqw = sumsqw;
    rec.ch0 = ch0;
    rec.single_chan = (nch == 1);
  }
}

}  // namespace ddfg
