// Backward passes of the degridder, for differentiating a visibility prediction.
//
// The degridder's prediction of facet f at visibility v of block b is linear in the facet's
// model grid G_f:
//     P_v = d ph_v J0 L(s_b) J1^H,   s_b,p = sum_t CF[t] G_f[p][cell_t(b)],
// with L the Stokes -> correlation map of the policy (Stokes.h:101-192), J0/J1 the antenna Jones
// terms, ph_v = exp(+i nu angle) and d the smearing factor (degridder.h:202-261).  Given the
// gradient g = dLoss/dP* of a real loss, the backward passes are:
//   * model grids (the adjoint, exact in exact arithmetic): G_f[p][cell_t] += conj(CF[t]) *
//     L^H(d conj(ph_v) J0^H g J1)_p -- a gridding pass with conjugated taps, the adjoint Stokes
//     map (no 1/2 factors) and no weights;
//   * Jones terms (J = J_kMS, nearest direction, no amplitude/phase normalisation): with
//     Q = d ph L(s) J1^H and R = d ph J0 L(s), dLoss/dJ0* += g Q^H and dLoss/dJ1* += g^H R.
// For averaged blocks the footprint is the block's (row means) and the adjoint value sums the
// block's visibilities; with per-block Jones (BDAJones) J0, J1 are the block's middle-row pair and
// the sums over the block come first.  Phases, smearing and Jones terms are recomputed from the
// same inputs as the forward pass.
#include <cuda_runtime.h>

#include "ddfg_common.cuh"
#include "ddfg_degridblock.cuh"
#include "ddfg_gridblock.cuh"
#include "ddfg_internal.h"
#include "ddfg_taps.cuh"

namespace ddfg {

// g as a 2x2 correlation matrix, the way the degridder maps its 2x2 prediction onto the
// visibility's correlations (4: all; 2: [0] and [3]; 1: [0]).
__device__ __forceinline__ M2 load_corr_matrix(const ddfg_vis &vs, int64_t irow, int ch) {
  const float2 *vp = (const float2 *)vs.vis + (irow * vs.nchan + ch) * (int64_t)vs.ncorr;
  M2 g;
  g.v[1] = czero();
  g.v[2] = czero();
  if (vs.ncorr == 4) {
    const float4 a = *(const float4 *)vp, c = *(const float4 *)(vp + 2);
    g.v[0] = make_float2(a.x, a.y); g.v[1] = make_float2(a.z, a.w);
    g.v[2] = make_float2(c.x, c.y); g.v[3] = make_float2(c.z, c.w);
  } else if (vs.ncorr == 2) {
    g.v[0] = vp[0]; g.v[3] = vp[1];
  } else {
    g.v[0] = vp[0]; g.v[3] = czero();
  }
  return g;
}

// L^H: the adjoint of corr_from_stokes, column by column.
template <int NPOL>
__device__ __forceinline__ void stokes_adjoint(int pol, const M2 &g, float2 *s) {
#pragma unroll
  for (int p = 0; p < NPOL; ++p) {
    float2 e[4] = {czero(), czero(), czero(), czero()};
    e[p] = make_float2(1.f, 0.f);
    const M2 col = corr_from_stokes(pol, e);
    float2 acc = czero();
#pragma unroll
    for (int c = 0; c < 4; ++c) acc = cadd(acc, cmul(cconj(col.v[c]), g.v[c]));
    s[p] = acc;
  }
}

// The adjoint record of visibility `in` on facet f: footprint by the degridder's geometry and
// value L^H(d conj(ph) J0^H g J1).
template <int NPOL>
__device__ __forceinline__ void adjoint_record(const DSingleIn &in, const ddfg_vis &vs, const ddfg_jones &js,
                                               const ddfg_facet &f, int policy, double n0m1, GridRecord<NPOL> &rec) {
  rec.valid = false;
  if (!degrid_single_geom_in(in, f, rec.g)) return;
  M2 gm = load_corr_matrix(vs, in.irow, in.ch);
  if (js.mode != 0) {
    M2 j0, j1;
    float bb;
    jones_pair_at(js, f.idir_kms, f.idir_beam, in.jx, in.U, in.V, j0, j1, bb);
    gm = m2_times(m2_times(m2_herm(j0), gm), j1);
  }
  const float dec = (float)decorr_factor(vs, f, in.nu, in.irow);
  const float2 ph = cscale(phasor_turns(in.nu * (in.U * f.l0 + in.V * f.m0 + in.W * n0m1) * kInvC), dec);
  gm = m2_scale(gm, cconj(ph));
  float2 s[4];
  stokes_adjoint<NPOL>(policy, gm, s);
#pragma unroll
  for (int p = 0; p < NPOL; ++p) rec.stokes[p] = s[p];
  rec.valid = true;
  rec.gridchan = in.gridchan;
}

// The adjoint record of averaged block d on facet f: footprint by the degridder's block geometry
// (row means, degridder.h:138-200), value L^H(J0m^H [sum over the block's visibilities of
// d conj(ph) J0^H g J1] J1m) -- per-visibility Jones (mode 1) inside the sum, the per-block Jones
// of the middle row and channel (mode 2) outside it, each looked up exactly as the forward pass
// does (same cache, same walk order).
template <int NPOL>
__device__ __forceinline__ void adjoint_block_record(const DegridBlock &d, const ddfg_vis &vs, const ddfg_jones &js,
                                                     const ddfg_facet &f, int policy, double n0m1,
                                                     GridRecord<NPOL> &rec) {
  rec.valid = false;
  if (!degrid_block_geom(vs, f, d, rec.g)) return;
  const int mid = d.rows[d.nrows / 2];
  const float dec = (float)decorr_factor(vs, f, d.freqmean, mid);
  JonesCache jc;
  jc.reset();
  M2 acc;
#pragma unroll
  for (int p = 0; p < 4; ++p) acc.v[p] = czero();
  for (int inx = 0; inx < d.nrows; ++inx) {
    const int64_t irow = d.rows[inx];
    const double *up = vs.uvw + 3 * irow;
    const double dot = up[0] * f.l0 + up[1] * f.m0 + up[2] * n0m1;
    for (int ch = d.ch0; ch < d.ch1; ++ch) {
      const float2 ph = cscale(phasor_turns(vs.freqs[ch] * dot * kInvC), dec);
      M2 g = load_corr_matrix(vs, irow, ch);
      if (js.mode == 1) {
        jc.update(js, f.idir_kms, f.idir_beam, irow, ch, up[0], up[1]);
        g = m2_times(m2_times(m2_herm(jc.j0), g), jc.j1);
      }
      g = m2_scale(g, cconj(ph));
#pragma unroll
      for (int p = 0; p < 4; ++p) acc.v[p] = cadd(acc.v[p], g.v[p]);
    }
  }
  if (js.mode == 2) {
    const double *up = vs.uvw + 3 * (int64_t)mid;
    jc.update(js, f.idir_kms, f.idir_beam, mid, (d.ch0 + d.ch1) / 2, up[0], up[1]);
    acc = m2_times(m2_times(m2_herm(jc.j0), acc), jc.j1);
  }
  float2 s[4];
  stokes_adjoint<NPOL>(policy, acc, s);
#pragma unroll
  for (int p = 0; p < NPOL; ++p) rec.stokes[p] = s[p];
  rec.valid = true;
  rec.gridchan = d.gridchan;
}

// Averaged blocks: each lane walks its block per facet and the warp lays the 32 adjoint records
// down with conjugated taps (the gridder's scatter).
template <int NPOL, int SLOTS>
__global__ void __launch_bounds__(256) degrid_adjoint_block_kernel(const ddfg_vis vs, const ddfg_jones js,
                                                                   const FacetPack pack, int policy) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ddfg_facet *sf = (ddfg_facet *)smem_raw;
  double *s_n0m1 = (double *)(sf + DDFG_FACETS_PER_LAUNCH);
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
  LaneTaps<SLOTS> lt;
  lt.reset();
  for (int64_t s = (int64_t)blockIdx.x * nwarps + warp; s < nstripes; s += (int64_t)gridDim.x * nwarps) {
    const int64_t b = s * 32 + lane;
    const bool inrange = b < vs.nblocks;
    DegridBlock d;
    if (inrange) degrid_block_header(vs, b, d);
    for (int fi = 0; fi < pack.n; ++fi) {
      const ddfg_facet &f = sf[fi];
      GridRecord<NPOL> rec;
      rec.valid = false;
      if (inrange) adjoint_block_record<NPOL>(d, vs, js, f, policy, s_n0m1[fi], rec);
      scatter_records<NPOL, SLOTS, true>(rec, f, min(NPOL, f.npol), lt, lane);
    }
  }
}

template <int NPOL, int SLOTS>
__global__ void __launch_bounds__(256) degrid_adjoint_kernel(const ddfg_vis vs, const ddfg_jones js,
                                                             const FacetPack pack, int policy) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ddfg_facet *sf = (ddfg_facet *)smem_raw;
  double *s_n0m1 = (double *)(sf + DDFG_FACETS_PER_LAUNCH);
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
  LaneTaps<SLOTS> lt;
  lt.reset();
  for (int64_t s = (int64_t)blockIdx.x * nwarps + warp; s < nstripes; s += (int64_t)gridDim.x * nwarps) {
    const int64_t b = s * 32 + lane;
    DSingleIn in;
    in.valid = false;
    if (b < vs.nblocks) degrid_load_single(vs, js, b, in);
    if (!__any_sync(0xffffffffu, in.valid)) continue;
    for (int fi = 0; fi < pack.n; ++fi) {
      const ddfg_facet &f = sf[fi];
      GridRecord<NPOL> rec;
      adjoint_record<NPOL>(in, vs, js, f, policy, s_n0m1[fi], rec);
      scatter_records<NPOL, SLOTS, true>(rec, f, min(NPOL, f.npol), lt, lane);
    }
  }
}

__device__ __forceinline__ size_t kms_offset(const ddfg_jones &js, int t, int dir, int a, int c) {
  const size_t nd = (size_t)js.kms_dims[1], na = (size_t)js.kms_dims[2], nch = (size_t)js.kms_dims[3];
  return (((size_t)t * nd + (size_t)dir) * na + (size_t)a) * nch * 4 + (size_t)c * 4;
}

__device__ __forceinline__ M2 load_m2(const float2 *J, size_t o) {
  M2 m;
#pragma unroll
  for (int p = 0; p < 4; ++p) m.v[p] = J[o + p];
  return m;
}

// The kMS gradient's view of the forward Jones: J = K . B (JonesServer.cc:276-289), so with a
// beam P = K0 (B0 M B1^H) K1^H and the kMS terms see M' = B0 M B1^H; the beam's own terms come
// from give_jones exactly as the forward takes them.  In interpolation mode 1 give_jones returns
// (sum of the coefficients)^2 times the stored matrix (its loop reads one direction once per
// non-zero coefficient), so the kMS matrices and their gradient carry that factor (kfac).
__device__ __forceinline__ M2 beam_sandwich(const ddfg_jones &js, int idir_beam, int tb, int cb, int a0, int a1,
                                            const M2 &m) {
  if (!js.beam) return m;
  const M2 b0 = give_jones((const float2 *)js.beam, js.beam_dims, js.interp_coefs, tb, a0, idir_beam, cb,
                           js.interp_mode);
  const M2 b1 = give_jones((const float2 *)js.beam, js.beam_dims, js.interp_coefs, tb, a1, idir_beam, cb,
                           js.interp_mode);
  return m2_times(m2_times(b0, m), m2_herm(b1));
}

__device__ __forceinline__ float kms_interp_factor(const ddfg_jones &js) {
  if (js.interp_mode != 1 || !js.interp_coefs) return 1.f;
  float c = 0.f;
  for (int d = 0; d < js.kms_dims[1]; ++d) c += js.interp_coefs[d];
  return c * c;
}

// The kMS matrix the forward applies, from the interpolated one z: the normalisation of
// norm_jones at the uv the forward uses (amplitude scaling depends on it).
__device__ __forceinline__ M2 kms_forward(const M2 &z, const ddfg_jones &js, double u, double v) {
  M2 k = z;
  norm_jones(k, js, u, v);
  return k;
}

// dL/dz* for f = z/|z|, given G = dL/df* (the Wirtinger chain rule dL/dz* = conj(G) df/dz* +
// G conj(df/dz)): G/(2|z|) - conj(G) z^2/(2|z|^3); at z = 0 the forward leaves z unchanged.
__device__ __forceinline__ float2 unit_grad(float2 z, float2 G) {
  const float r = cabs2(z);
  if (r == 0.f) return G;
  const float2 t = cmul(cconj(G), cmul(z, z));
  const float inv2r = 0.5f / r, inv2r3 = 0.5f / (r * r * r);
  return make_float2(G.x * inv2r - t.x * inv2r3, G.y * inv2r - t.y * inv2r3);
}

// dL/dz* of one Jones element through norm_jones (JonesServer.cc:25-52), given G = dL/df* for its
// output: the forward applies z1 = amplitude normalisation (z/|z|, without ApplyAmp), z2 = phase
// removal (|z1|, without ApplyPhase), z3 = amplitude scaling z2 ((1 - alpha)/|z2| + alpha)
// (DoScaleJones), and the chain rule runs back through the three: scaling gives
// (1 - alpha) unit_grad + alpha G, phase removal Re(G) z1/|z1|, amplitude normalisation unit_grad.
__device__ __forceinline__ float2 norm_grad1(float2 z, float2 G, bool amp, bool phase, bool scale, float alpha) {
  float2 z1 = z;
  if (!amp) {
    const float a = cabs2(z);
    if (a != 0.f) z1 = cscale(z, 1.f / a);
  }
  const float2 z2 = phase ? z1 : make_float2(cabs2(z1), 0.f);
  float2 g = G;
  if (scale) {
    const float2 u = unit_grad(z2, g);
    g = cabs2(z2) == 0.f ? g : make_float2((1.f - alpha) * u.x + alpha * g.x, (1.f - alpha) * u.y + alpha * g.y);
  }
  if (!phase) {
    const float r = cabs2(z1);
    g = r == 0.f ? czero() : cscale(z1, g.x / r);
  }
  if (!amp) g = unit_grad(z, g);
  return g;
}

// The amplitude-scaling factor alpha of norm_jones at (u, v).
__device__ __forceinline__ float scale_alpha(const ddfg_jones &js, double u, double v) {
  const double r2 = (u * u + v * v) / (js.wavelength_mean * js.wavelength_mean);
  return (float)exp(-2. * kPi * js.calib_error * js.calib_error * r2);
}

// dL/d(stored kMS matrix)* from dL/dK*: the normalisation's chain rule at (u, v), then the
// interpolation factor (the stored matrix z_s enters as z = kfac z_s).
__device__ __forceinline__ M2 kms_chain(const M2 &dK, const M2 &z, const ddfg_jones &js, float kfac, double u,
                                        double v) {
  M2 out;
  const bool amp = js.apply_amp != 0, phase = js.apply_phase != 0, scale = js.scale_jones != 0;
  if (amp && phase && !scale) {
#pragma unroll
    for (int p = 0; p < 4; ++p) out.v[p] = cscale(dK.v[p], kfac);
    return out;
  }
  const float alpha = scale ? scale_alpha(js, u, v) : 0.f;
#pragma unroll
  for (int p = 0; p < 4; ++p) out.v[p] = cscale(norm_grad1(z.v[p], dK.v[p], amp, phase, scale, alpha), kfac);
  return out;
}

__device__ __forceinline__ M2 m2_zero() {
  M2 m;
#pragma unroll
  for (int p = 0; p < 4; ++p) m.v[p] = czero();
  return m;
}

__device__ __forceinline__ M2 m2_add(const M2 &a, const M2 &b) {
  M2 m;
#pragma unroll
  for (int p = 0; p < 4; ++p) m.v[p] = cadd(a.v[p], b.v[p]);
  return m;
}

// One 2x2 gradient cell (32-byte aligned: Jones cells are 4 complex64) += d, two vector reductions.
__device__ __forceinline__ void red_add_m2(float2 *p, const M2 &d) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(d.v[0].x), "f"(d.v[0].y),
               "f"(d.v[1].x), "f"(d.v[1].y) : "memory");
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p + 2), "f"(d.v[2].x), "f"(d.v[2].y),
               "f"(d.v[3].x), "f"(d.v[3].y) : "memory");
}

// grad[o0] += d0 and grad[o1] += d1 for every active lane; called by the whole warp.  When every
// active lane targets the same two cells (a row's channels, a baseline's consecutive blocks in
// one Jones slot) the warp sums first and one lane adds, instead of 32 lanes adding to the same
// addresses.
__device__ __forceinline__ void warp_add_jones_grad(float2 *grad, bool active, size_t o0, size_t o1, M2 d0, M2 d1,
                                                    int lane) {
  const unsigned act = __ballot_sync(0xffffffffu, active);
  if (!act) return;
  const int first = __ffs(act) - 1;
  const unsigned long long f0 = __shfl_sync(0xffffffffu, (unsigned long long)o0, first);
  const unsigned long long f1 = __shfl_sync(0xffffffffu, (unsigned long long)o1, first);
  if (__all_sync(0xffffffffu, !active || ((unsigned long long)o0 == f0 && (unsigned long long)o1 == f1))) {
    if (!active) {
      d0 = m2_zero();
      d1 = m2_zero();
    }
#pragma unroll
    for (int p = 0; p < 4; ++p) {
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        d0.v[p].x += __shfl_xor_sync(0xffffffffu, d0.v[p].x, off);
        d0.v[p].y += __shfl_xor_sync(0xffffffffu, d0.v[p].y, off);
        d1.v[p].x += __shfl_xor_sync(0xffffffffu, d1.v[p].x, off);
        d1.v[p].y += __shfl_xor_sync(0xffffffffu, d1.v[p].y, off);
      }
    }
    if (lane == first) {
      red_add_m2(grad + f0, d0);
      red_add_m2(grad + f1, d1);
    }
  } else if (active) {
    red_add_m2(grad + o0, d0);
    red_add_m2(grad + o1, d1);
  }
}

// dLoss/dJ_kMS* for every visibility and facet: the forward gather of the model grid, then the
// two antenna terms, reduced into the gradient array (same layout as the Jones array).
template <int NPOL, int SLOTS>
__global__ void __launch_bounds__(256) jones_grad_kernel(const ddfg_vis vs, const ddfg_jones js,
                                                         const FacetPackD pack, int policy, float2 *grad) {
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
  float2 *wpart = partial + warp * 32 * 32;
  LaneTaps<SLOTS> lt;
  lt.reset();
  const float2 *J = (const float2 *)js.kms;
  const float kfac = kms_interp_factor(js);
  for (int64_t s = (int64_t)blockIdx.x * nwarps + warp; s < nstripes; s += (int64_t)gridDim.x * nwarps) {
    const int64_t b = s * 32 + lane;
    DSingleIn in;
    in.valid = false;
    if (b < vs.nblocks) degrid_load_single(vs, js, b, in);
    if (!__any_sync(0xffffffffu, in.valid)) continue;
    M2 g;
    if (in.valid) g = load_corr_matrix(vs, in.irow, in.ch);
    for (int fi = 0; fi < pack.n; ++fi) {
      const ddfg_facet &f = sf[fi];
      BlockGeom geo;
      const bool valid = degrid_single_geom_in(in, f, geo);
      TapJob job;
      if (valid) job = tap_job(geo, in.gridchan, f);
      float2 mine[NPOL];
      gather_records<NPOL, SLOTS>(valid, job, f, lt, wpart, lane, mine);
      size_t o0 = 0, o1 = 0;
      M2 d0 = m2_zero(), d1 = m2_zero();
      if (valid) {
        float2 sv[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) sv[p] = (p < NPOL) ? mine[p] : czero();
        const M2 m = beam_sandwich(js, f.idir_beam, in.jx.tb, in.jx.cb, in.jx.a0, in.jx.a1,
                                   corr_from_stokes(policy, sv));
        o0 = kms_offset(js, in.jx.tk, f.idir_kms, in.jx.a0, in.jx.ck);
        o1 = kms_offset(js, in.jx.tk, f.idir_kms, in.jx.a1, in.jx.ck);
        const M2 z0 = m2_scale(load_m2(J, o0), make_float2(kfac, 0.f));
        const M2 z1 = m2_scale(load_m2(J, o1), make_float2(kfac, 0.f));
        const M2 j0 = kms_forward(z0, js, in.U, in.V), j1 = kms_forward(z1, js, in.U, in.V);
        const float dec = (float)decorr_factor(vs, f, in.nu, in.irow);
        const float2 ph = cscale(phasor_turns(in.nu * (in.U * f.l0 + in.V * f.m0 + in.W * s_n0m1[fi]) * kInvC), dec);
        const M2 q = m2_scale(m2_times(m, m2_herm(j1)), ph);  // d ph M' K1^H
        const M2 r = m2_scale(m2_times(j0, m), ph);           // d ph K0 M'
        d0 = kms_chain(m2_times(g, m2_herm(q)), z0, js, kfac, in.U, in.V);
        d1 = kms_chain(m2_times(m2_herm(g), r), z1, js, kfac, in.U, in.V);
      }
      warp_add_jones_grad(grad, valid, o0, o1, d0, d1, lane);
    }
  }
}

// dLoss/dJ_kMS* for averaged blocks: the block's model sample M = L(s) is gathered once per facet;
// per visibility (mode 1) g Q^H and g^H R are reduced into the visibility's Jones cells, or
// (mode 2, one Jones pair per block at its middle row and channel) G (M J1^H)^H and
// G^H J0 M with G = sum over the block of d conj(ph) g.
template <int NPOL, int SLOTS>
__global__ void __launch_bounds__(256) jones_grad_block_kernel(const ddfg_vis vs, const ddfg_jones js,
                                                               const FacetPackD pack, int policy, float2 *grad) {
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
  float2 *wpart = partial + warp * 32 * 32;
  LaneTaps<SLOTS> lt;
  lt.reset();
  const float2 *J = (const float2 *)js.kms;
  const float kfac = kms_interp_factor(js);
  for (int64_t s = (int64_t)blockIdx.x * nwarps + warp; s < nstripes; s += (int64_t)gridDim.x * nwarps) {
    const int64_t b = s * 32 + lane;
    const bool inrange = b < vs.nblocks;
    DegridBlock d;
    if (inrange) degrid_block_header(vs, b, d);
    for (int fi = 0; fi < pack.n; ++fi) {
      const ddfg_facet &f = sf[fi];
      BlockGeom geo;
      const bool valid = inrange && degrid_block_geom(vs, f, d, geo);
      TapJob job;
      if (valid) job = tap_job(geo, d.gridchan, f);
      float2 mine[NPOL];
      gather_records<NPOL, SLOTS>(valid, job, f, lt, wpart, lane, mine);
      // the lane's pending sums for one pair of Jones cells (o0, o1): visibilities of a row share
      // them, so the lane adds once per run and the warp combines the last runs
      size_t o0 = 0, o1 = 0;
      M2 d0 = m2_zero(), d1 = m2_zero();
      bool pending = false;
      if (valid) {
        float2 sv[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) sv[p] = (p < NPOL) ? mine[p] : czero();
        const M2 m = corr_from_stokes(policy, sv);
        const int mid = d.rows[d.nrows / 2];
        const float dec = (float)decorr_factor(vs, f, d.freqmean, mid);
        M2 G = m2_zero();
        double uk = 0., vk = 0.;
        for (int inx = 0; inx < d.nrows; ++inx) {
          const int64_t irow = d.rows[inx];
          const double *up = vs.uvw + 3 * irow;
          const double dot = up[0] * f.l0 + up[1] * f.m0 + up[2] * s_n0m1[fi];
          for (int ch = d.ch0; ch < d.ch1; ++ch) {
            const float2 ph = cscale(phasor_turns(vs.freqs[ch] * dot * kInvC), dec);
            const M2 g = load_corr_matrix(vs, irow, ch);
            if (js.mode == 1) {
              const JonesIdx x = jones_idx(js, irow, ch);
              const size_t p0 = kms_offset(js, x.tk, f.idir_kms, x.a0, x.ck);
              const size_t p1 = kms_offset(js, x.tk, f.idir_kms, x.a1, x.ck);
              if (!pending || p0 != o0 || p1 != o1) {
                if (pending) {
                  red_add_m2(grad + o0, d0);
                  red_add_m2(grad + o1, d1);
                  d0 = m2_zero();
                  d1 = m2_zero();
                }
                // the forward's Jones cache (reset per block) recomputes the kMS terms, and reads
                // the uv its amplitude scaling uses, at the visibility where they change
                uk = up[0];
                vk = up[1];
              }
              o0 = p0;
              o1 = p1;
              pending = true;
              const M2 mb = beam_sandwich(js, f.idir_beam, x.tb, x.cb, x.a0, x.a1, m);
              const M2 z0 = m2_scale(load_m2(J, p0), make_float2(kfac, 0.f));
              const M2 z1 = m2_scale(load_m2(J, p1), make_float2(kfac, 0.f));
              const M2 j0 = kms_forward(z0, js, uk, vk), j1 = kms_forward(z1, js, uk, vk);
              const M2 q = m2_scale(m2_times(mb, m2_herm(j1)), ph);  // d ph M' K1^H
              const M2 r = m2_scale(m2_times(j0, mb), ph);           // d ph K0 M'
              d0 = m2_add(d0, kms_chain(m2_times(g, m2_herm(q)), z0, js, kfac, uk, vk));
              d1 = m2_add(d1, kms_chain(m2_times(m2_herm(g), r), z1, js, kfac, uk, vk));
            } else {
              G = m2_add(G, m2_scale(g, cconj(ph)));
            }
          }
        }
        if (js.mode == 2) {
          const JonesIdx x = jones_idx(js, mid, (d.ch0 + d.ch1) / 2);
          o0 = kms_offset(js, x.tk, f.idir_kms, x.a0, x.ck);
          o1 = kms_offset(js, x.tk, f.idir_kms, x.a1, x.ck);
          const M2 mb = beam_sandwich(js, f.idir_beam, x.tb, x.cb, x.a0, x.a1, m);
          const float2 kf = make_float2(kfac, 0.f);
          const M2 z0 = m2_scale(load_m2(J, o0), kf), z1 = m2_scale(load_m2(J, o1), kf);
          const double *um = vs.uvw + 3 * (int64_t)mid;  // the forward normalises at the middle row
          const M2 j0 = kms_forward(z0, js, um[0], um[1]), j1 = kms_forward(z1, js, um[0], um[1]);
          d0 = kms_chain(m2_times(G, m2_herm(m2_times(mb, m2_herm(j1)))), z0, js, kfac, um[0], um[1]);
          d1 = kms_chain(m2_times(m2_herm(G), m2_times(j0, mb)), z1, js, kfac, um[0], um[1]);
          pending = true;
        }
      }
      warp_add_jones_grad(grad, pending, o0, o1, d0, d1, lane);
    }
  }
}

}  // namespace ddfg

using namespace ddfg;

int ddfg_launch_degrid_adjoint(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_facet *facets, int nfacets,
                               int policy, int nvispol, int num_ctas, cudaStream_t stream) {
  int max_support = 1;
  for (int i = 0; i < nfacets; ++i) max_support = max(max_support, facets[i].max_support);
  const int slots = tap_slots(max_support);
  const size_t smem = sizeof(ddfg_facet) * DDFG_FACETS_PER_LAUNCH + sizeof(double) * DDFG_FACETS_PER_LAUNCH;
  const int npacks = (nfacets + DDFG_FACETS_PER_LAUNCH - 1) / DDFG_FACETS_PER_LAUNCH;  // balanced packs
  for (int ip = 0; ip < npacks; ++ip) {
    const int f0 = (int)(((long long)ip * nfacets) / npacks);
    FacetPack pack;
    pack.n = (int)(((long long)(ip + 1) * nfacets) / npacks) - f0;
    for (int i = 0; i < pack.n; ++i) pack.f[i] = facets[f0 + i];
#define LAUNCH_A(NP, SL)                                                                      \
  do {                                                                                        \
    if (vs->single_vis_blocks)                                                                \
      degrid_adjoint_kernel<NP, SL><<<num_ctas, 256, smem, stream>>>(*vs, *js, pack, policy);       \
    else                                                                                      \
      degrid_adjoint_block_kernel<NP, SL><<<num_ctas, 256, smem, stream>>>(*vs, *js, pack, policy); \
  } while (0)
#define LAUNCH_A_NP(SL)              \
  switch (nvispol) {                 \
    case 1: LAUNCH_A(1, SL); break;  \
    case 2: LAUNCH_A(2, SL); break;  \
    case 3: LAUNCH_A(3, SL); break;  \
    default: LAUNCH_A(4, SL); break; \
  }
    if (slots == 2) { LAUNCH_A_NP(2) } else if (slots == 4) { LAUNCH_A_NP(4) } else { LAUNCH_A_NP(8) }
#undef LAUNCH_A_NP
#undef LAUNCH_A
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "degrid_adjoint launch: %s", cudaGetErrorString(e));
  }
  return DDFG_OK;
}

int ddfg_launch_jones_grad(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_facet *facets, int nfacets,
                           int policy, int nvispol, void *grad, int num_ctas, cudaStream_t stream) {
  int max_support = 1;
  for (int i = 0; i < nfacets; ++i) max_support = max(max_support, facets[i].max_support);
  const int slots = tap_slots(max_support);
  const size_t smem = sizeof(ddfg_facet) * DDFG_FACETS_PER_LAUNCH + sizeof(double) * DDFG_FACETS_PER_LAUNCH +
                      (nvispol == 1 ? 8 * kPartialBytesPerWarp : 0);
  float2 *g = (float2 *)grad;
  int per_sm = 0;
  const int npacks = (nfacets + DDFG_FACETS_PER_LAUNCH - 1) / DDFG_FACETS_PER_LAUNCH;  // balanced packs
  for (int ip = 0; ip < npacks; ++ip) {
    const int f0 = (int)(((long long)ip * nfacets) / npacks);
    FacetPackD pack;
    pack.n = (int)(((long long)(ip + 1) * nfacets) / npacks) - f0;
    for (int i = 0; i < pack.n; ++i) pack.f[i] = facets[f0 + i];
#define LAUNCH_J(NP, SL)                                                                                   \
  do {                                                                                                     \
    if (vs->single_vis_blocks) {                                                                           \
      ddfg_kernel_prepare((const void *)jones_grad_kernel<NP, SL>, 256, smem, &per_sm);                     \
      jones_grad_kernel<NP, SL><<<num_ctas, 256, smem, stream>>>(*vs, *js, pack, policy, g);                 \
    } else {                                                                                               \
      ddfg_kernel_prepare((const void *)jones_grad_block_kernel<NP, SL>, 256, smem, &per_sm);               \
      jones_grad_block_kernel<NP, SL><<<num_ctas, 256, smem, stream>>>(*vs, *js, pack, policy, g);           \
    }                                                                                                      \
  } while (0)
#define LAUNCH_J_NP(SL)              \
  switch (nvispol) {                 \
    case 1: LAUNCH_J(1, SL); break;  \
    case 2: LAUNCH_J(2, SL); break;  \
    case 3: LAUNCH_J(3, SL); break;  \
    default: LAUNCH_J(4, SL); break; \
  }
    if (slots == 2) { LAUNCH_J_NP(2) } else if (slots == 4) { LAUNCH_J_NP(4) } else { LAUNCH_J_NP(8) }
#undef LAUNCH_J_NP
#undef LAUNCH_J
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "jones_grad launch: %s", cudaGetErrorString(e));
  }
  return DDFG_OK;
}
