// Device-side building blocks shared by the gridding and degridding kernels.
//
// Everything here restates the per-visibility physics of DDFacet's BDA gridder for the GPU:
// complex 2x2 algebra (JonesServer.h:38-81), the Jones fetch/normalise/compose rules
// (JonesServer.cc:25-298), the smearing factor (DecorrelationHelper.cc:42-63), the facet phasor
// (CorrelationCalculator.h:37-65) and the correlation <-> Stokes policies (Stokes.h:18-226).
//
// Precision: the phase argument (u l0 + v m0 + w (n0-1)) * nu / c and every quantity that feeds
// an integer grid index (block means, positions, w-plane) are FP64; FP64 additions/products that
// decide an index use explicit _rn intrinsics so they are not contracted into FMAs and round the
// way the reference's scalar C++ does.  Everything else is FP32.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "ddfg.h"

namespace ddfg {

constexpr double kC = 299792458.0;                      // common.h:9
constexpr double kPi = 3.141592653589793238462643383279502884197;
constexpr double kInvC = 1.0 / 299792458.0;  // phase arguments only; index arithmetic divides by kC

// ----------------------------------------------------------------------------------------
// complex helpers (float2 = complex64)
// ----------------------------------------------------------------------------------------
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float cabs2(float2 a) { return sqrtf(a.x * a.x + a.y * a.y); }
__device__ __forceinline__ float2 cmuli(float2 a) { return make_float2(-a.y, a.x); }  // a * i
__device__ __forceinline__ float2 czero() { return make_float2(0.f, 0.f); }

// grid[cell] += v as one vector reduction without a return value (red.global.add.v2.f32,
// sm_90+): the same addition as atomicAdd(float2*), which is issued as a returning atomic, but
// the issuing warp does not wait for the L2 round trip.
__device__ __forceinline__ void red_add(float2 *p, float2 v) {
  asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(v.x), "f"(v.y) : "memory");
}

// 2x2 complex matrix, element order [0]=(0,0) [1]=(0,1) [2]=(1,0) [3]=(1,1) (JonesServer.h:38-81)
struct M2 {
  float2 v[4];
};
__device__ __forceinline__ M2 m2_unity() {
  M2 m;
  m.v[0] = make_float2(1.f, 0.f);
  m.v[1] = czero();
  m.v[2] = czero();
  m.v[3] = make_float2(1.f, 0.f);
  return m;
}
__device__ __forceinline__ M2 m2_times(const M2 &a, const M2 &b) {
  M2 r;
  r.v[0] = cadd(cmul(a.v[0], b.v[0]), cmul(a.v[1], b.v[2]));
  r.v[1] = cadd(cmul(a.v[0], b.v[1]), cmul(a.v[1], b.v[3]));
  r.v[2] = cadd(cmul(a.v[2], b.v[0]), cmul(a.v[3], b.v[2]));
  r.v[3] = cadd(cmul(a.v[2], b.v[1]), cmul(a.v[3], b.v[3]));
  return r;
}
__device__ __forceinline__ M2 m2_herm(const M2 &a) {
  M2 r;
  r.v[0] = cconj(a.v[0]);
  r.v[1] = cconj(a.v[2]);
  r.v[2] = cconj(a.v[1]);
  r.v[3] = cconj(a.v[3]);
  return r;
}
__device__ __forceinline__ M2 m2_scale(const M2 &a, float2 s) {
  M2 r;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.v[i] = cmul(a.v[i], s);
  return r;
}

// ----------------------------------------------------------------------------------------
// FP64 index arithmetic without contraction
// ----------------------------------------------------------------------------------------
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ long long lrint_d(double x) { return __double2ll_rn(x); }

// exp(i * 2*pi * turns): FP64 range reduction, FP32 sincospi of the fraction.
__device__ __forceinline__ float2 phasor_turns(double turns) {
  double frac = turns - rint(turns);
  float s, c;
  sincospif(2.0f * (float)frac, &s, &c);
  return make_float2(c, s);
}

// ----------------------------------------------------------------------------------------
// Jones server (JonesServer.cc:54-95 GiveJones, :25-52 NormJones, :193-298 updateJones)
// ----------------------------------------------------------------------------------------
__device__ __forceinline__ M2 give_jones(const float2 *__restrict__ J, const int32_t *dims,
                                         const float *__restrict__ coefs, int it, int ant, int idir,
                                         int ich, int mode) {
  const size_t nd = (size_t)dims[1], na = (size_t)dims[2], nch = (size_t)dims[3];
  const size_t off = (size_t)it * nd * na * nch * 4 + (size_t)idir * na * nch * 4 + (size_t)ant * nch * 4 +
                     (size_t)ich * 4;
  M2 out;
  if (mode == 0) {
#pragma unroll
    for (int p = 0; p < 4; ++p) out.v[p] = J[off + p];
    return out;
  }
  // Mode 1 (JonesServer.cc:71-93): the reference's loop reads the SAME direction (offJ0 does
  // not depend on idir) once per non-zero coefficient; restated literally.
  float jabs[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
  for (int p = 0; p < 4; ++p) out.v[p] = czero();
  for (size_t d = 0; d < nd; ++d) {
    const float c = coefs[d];
    if (c == 0.f) continue;
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      const float2 val = J[off + p];
      const float a = cabs2(val);
      out.v[p] = cadd(out.v[p], cscale(val, c / a));
      jabs[p] += c * a;
    }
  }
#pragma unroll
  for (int p = 0; p < 4; ++p) out.v[p] = cscale(out.v[p], jabs[p]);
  return out;
}

__device__ __forceinline__ void norm_jones(M2 &j, const ddfg_jones &js, double u, double v) {
  if (!js.apply_amp) {
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      const float a = cabs2(j.v[p]);
      if (a != 0.f) j.v[p] = cscale(j.v[p], 1.f / a);
    }
  }
  if (!js.apply_phase) {
#pragma unroll
    for (int p = 0; p < 4; ++p) j.v[p] = make_float2(cabs2(j.v[p]), 0.f);
  }
  if (js.scale_jones) {
    const double r2 = (u * u + v * v) / (js.wavelength_mean * js.wavelength_mean);
    const float alpha = (float)exp(-2. * kPi * js.calib_error * js.calib_error * r2);
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      const float a = cabs2(j.v[p]);
      if (a != 0.f) j.v[p] = cscale(j.v[p], (1.f - alpha) / a + alpha);
    }
  }
}

// Cached Jones state of one block walk.  The reference recomputes the beam and DD Jones only
// when the antennas, the time slot or the Jones channel change; the DD Jones normalisation
// reads the uvw of the visibility at which that happened, which is kept so the cached and
// recomputed values agree even with scale_jones set.
struct JonesCache {
  int ant0, ant1, tk, ck, tb, cb;
  double uk, vk;
  M2 j0, j1;
  float bb;
  __device__ __forceinline__ void reset() {
    ant0 = ant1 = -1;
    tk = ck = tb = cb = -1;
    uk = vk = 0.;
    j0 = j1 = m2_unity();
    bb = 1.f;
  }
  // Returns true when J0/J1 changed (JonesServer.cc:193-298).
  __device__ __forceinline__ bool update(const ddfg_jones &js, int ifacet_dir_kms, int ifacet_dir_beam,
                                         int64_t irow, int ichan, double u, double v) {
    const int a0 = js.a0[irow], a1 = js.a1[irow];
    const bool bl_changed = (a0 != ant0) || (a1 != ant1);
    ant0 = a0;
    ant1 = a1;
    bool changed = false;
    if (js.beam) {
      const int t = js.beam_tmap[irow], c = js.beam_cmap[ichan];
      if (bl_changed || t != tb || c != cb) {
        tb = t;
        cb = c;
        changed = true;
      }
    }
    if (js.kms) {
      const int t = js.kms_tmap[irow], c = js.kms_cmap[ichan];
      if (bl_changed || t != tk || c != ck) {
        tk = t;
        ck = c;
        uk = u;
        vk = v;
        changed = true;
      }
    }
    if (changed) {
      M2 a = m2_unity(), b = m2_unity();
      if (js.beam) {
        a = give_jones((const float2 *)js.beam, js.beam_dims, js.interp_coefs, tb, ant0, ifacet_dir_beam, cb,
                       js.interp_mode);
        b = give_jones((const float2 *)js.beam, js.beam_dims, js.interp_coefs, tb, ant1, ifacet_dir_beam, cb,
                       js.interp_mode);
      }
      if (js.kms) {
        M2 k0 = give_jones((const float2 *)js.kms, js.kms_dims, js.interp_coefs, tk, ant0, ifacet_dir_kms, ck,
                           js.interp_mode);
        M2 k1 = give_jones((const float2 *)js.kms, js.kms_dims, js.interp_coefs, tk, ant1, ifacet_dir_kms, ck,
                           js.interp_mode);
        norm_jones(k0, js, uk, vk);
        norm_jones(k1, js, uk, vk);
        a = js.beam ? m2_times(k0, a) : k0;
        b = js.beam ? m2_times(k1, b) : k1;
      }
      j0 = a;
      j1 = b;
      const float t = (cabs2(j0.v[0]) * cabs2(j1.v[0]) + cabs2(j0.v[3]) * cabs2(j1.v[3])) * 0.5f;
      bb = t * t;
    }
    return changed;
  }
};

// The row/channel indices a visibility's Jones lookup needs (antennas, time slots, Jones
// channels), loaded once and reused for every facet of a launch.
struct JonesIdx {
  int a0, a1, tk, ck, tb, cb;
};
__device__ __forceinline__ JonesIdx jones_idx(const ddfg_jones &js, int64_t irow, int ichan) {
  JonesIdx x;
  x.a0 = js.a0[irow];
  x.a1 = js.a1[irow];
  x.tk = js.kms ? js.kms_tmap[irow] : 0;
  x.ck = js.kms ? js.kms_cmap[ichan] : 0;
  x.tb = js.beam ? js.beam_tmap[irow] : 0;
  x.cb = js.beam ? js.beam_cmap[ichan] : 0;
  return x;
}

// J0, J1 and BB of one visibility without a cache: what JonesCache::update computes after a
// reset (every single-visibility block resets the reference's cache, gridder.h:184), with the
// indices already loaded.
__device__ __forceinline__ void jones_pair_at(const ddfg_jones &js, int idir_kms, int idir_beam, const JonesIdx &x,
                                              double u, double v, M2 &j0, M2 &j1, float &bb) {
  const int a0 = x.a0, a1 = x.a1;
  M2 a = m2_unity(), b = m2_unity();
  if (js.beam) {
    const int t = x.tb, c = x.cb;
    a = give_jones((const float2 *)js.beam, js.beam_dims, js.interp_coefs, t, a0, idir_beam, c, js.interp_mode);
    b = give_jones((const float2 *)js.beam, js.beam_dims, js.interp_coefs, t, a1, idir_beam, c, js.interp_mode);
  }
  if (js.kms) {
    const int t = x.tk, c = x.ck;
    M2 k0 = give_jones((const float2 *)js.kms, js.kms_dims, js.interp_coefs, t, a0, idir_kms, c, js.interp_mode);
    M2 k1 = give_jones((const float2 *)js.kms, js.kms_dims, js.interp_coefs, t, a1, idir_kms, c, js.interp_mode);
    norm_jones(k0, js, u, v);
    norm_jones(k1, js, u, v);
    // J = J_kMS . J_beam; without a beam J_beam is the identity (JonesServer.cc:276-289)
    a = js.beam ? m2_times(k0, a) : k0;
    b = js.beam ? m2_times(k1, b) : k1;
  }
  j0 = a;
  j1 = b;
  const float t = (cabs2(a.v[0]) * cabs2(b.v[0]) + cabs2(a.v[3]) * cabs2(b.v[3])) * 0.5f;
  bb = t * t;
}

// The same, loading the indices of row irow and channel ichan.
__device__ __forceinline__ void jones_pair(const ddfg_jones &js, int idir_kms, int idir_beam, int64_t irow, int ichan,
                                           double u, double v, M2 &j0, M2 &j1, float &bb) {
  jones_pair_at(js, idir_kms, idir_beam, jones_idx(js, irow, ichan), u, v, j0, j1, bb);
}

// ----------------------------------------------------------------------------------------
// Smearing factor (DecorrelationHelper.cc:42-63)
// ----------------------------------------------------------------------------------------
__device__ __forceinline__ double decorr_factor(const ddfg_vis &vs, const ddfg_facet &f, double nu, int64_t irow) {
  if (!vs.uvw_dt) return 1.0;
  const double l = f.decorr_l, m = f.decorr_m;
  const double n0 = sqrt(1. - l * l - m * m) - 1.;
  double fac = 1.0;
  if (vs.do_fsmear) {
    const double *p = vs.uvw + 3 * irow;
    const double ph = p[0] * l + p[1] * m + p[2] * n0;
    const double phi = kPi * vs.dnu / kC * ph;
    fac *= (phi == 0.) ? 1.0 : sin(phi) / phi;
  }
  if (vs.do_tsmear) {
    const double *p = vs.uvw_dt + 3 * irow;
    const double dph = (p[0] * l + p[1] * m + p[2] * n0) * vs.dt;
    const double phi = kPi * nu / kC * dph;
    fac *= (phi == 0.) ? 1.0 : sin(phi) / phi;
  }
  return fac;
}

// ----------------------------------------------------------------------------------------
// Correlation <-> Stokes policies (Stokes.h)
// ----------------------------------------------------------------------------------------
// Gridding policies: visibility 2x2 accumulator -> Stokes vector (Stokes.h:18-77).
enum GridPolicy : int {
  G_I_FROM_I = 0,
  G_I_LIN2, G_IQ_LIN2,                     // XX,YY
  G_I_CIRC2, G_IV_CIRC2,                   // RR,LL
  G_I_LIN4, G_Q_LIN4, G_U_LIN4, G_V_LIN4,  // XX,XY,YX,YY
  G_IQ_LIN4, G_IV_LIN4, G_QU_LIN4, G_IQU_LIN4, G_IQUV_LIN4,
  G_I_CIRC4, G_IQ_CIRC4, G_IU_CIRC4, G_IV_CIRC4, G_QU_CIRC4, G_IQU_CIRC4, G_IQUV_CIRC4,
};

// Degridding policies: Stokes vector -> 2x2 correlations (Stokes.h:90-226).
enum DegridPolicy : int {
  D_DIAG_FROM_I = 0,  // XX=YY=I (all I-only modes)
  D_LIN4_FROM_Q, D_LIN4_FROM_U, D_LIN4_FROM_V,
  D_CIRC4_FROM_IQUV, D_CIRC4_FROM_IQ, D_CIRC4_FROM_IU, D_CIRC4_FROM_IQU,
  D_LIN4_FROM_IQUV, D_LIN4_FROM_IQ, D_LIN4_FROM_IU, D_LIN4_FROM_IV, D_LIN4_FROM_QU, D_LIN4_FROM_IQU,
  D_CIRC4_FROM_IV, D_LIN2_FROM_IQ, D_CIRC2_FROM_IV,
};

__device__ __forceinline__ void stokes_from_corr(int pol, const M2 &V, float2 *s) {
  const float2 ipp = cscale(cadd(V.v[0], V.v[3]), 0.5f);  // (V0+V3)/2
  const float2 imm = cscale(csub(V.v[0], V.v[3]), 0.5f);  // (V0-V3)/2
  const float2 xpp = cscale(cadd(V.v[1], V.v[2]), 0.5f);  // (V1+V2)/2
  // -(V1-V2)*0.5i
  const float2 xmm = cmuli(cscale(csub(V.v[1], V.v[2]), -0.5f));
  switch (pol) {
    case G_I_FROM_I: s[0] = V.v[0]; break;
    case G_I_LIN2: case G_I_CIRC2: case G_I_LIN4: case G_I_CIRC4: s[0] = ipp; break;
    case G_IQ_LIN2: case G_IV_CIRC2: s[0] = ipp; s[1] = imm; break;
    case G_Q_LIN4: s[0] = imm; break;
    case G_U_LIN4: s[0] = xpp; break;
    case G_V_LIN4: s[0] = xmm; break;
    case G_IQ_LIN4: s[0] = ipp; s[1] = imm; break;
    case G_IV_LIN4: s[0] = ipp; s[1] = xmm; break;
    case G_QU_LIN4: s[0] = imm; s[1] = xpp; break;
    case G_IQU_LIN4: s[0] = ipp; s[1] = imm; s[2] = xpp; break;
    case G_IQUV_LIN4: s[0] = ipp; s[1] = imm; s[2] = xpp; s[3] = xmm; break;
    case G_IQ_CIRC4: s[0] = ipp; s[1] = xpp; break;
    case G_IU_CIRC4: s[0] = ipp; s[1] = xmm; break;
    case G_IV_CIRC4: s[0] = ipp; s[1] = imm; break;
    case G_QU_CIRC4: s[0] = xpp; s[1] = xmm; break;
    case G_IQU_CIRC4: s[0] = ipp; s[1] = xpp; s[2] = xmm; break;
    case G_IQUV_CIRC4: s[0] = ipp; s[1] = xpp; s[2] = xmm; s[3] = imm; break;
    default: break;
  }
}

__device__ __forceinline__ M2 corr_from_stokes(int pol, const float2 *s) {
  M2 r;
  const float2 z = czero();
  switch (pol) {
    case D_DIAG_FROM_I: r.v[0] = s[0]; r.v[1] = z; r.v[2] = z; r.v[3] = s[0]; break;
    case D_LIN4_FROM_Q: r.v[0] = s[0]; r.v[1] = z; r.v[2] = z; r.v[3] = cscale(s[0], -1.f); break;
    case D_LIN4_FROM_U: r.v[0] = z; r.v[1] = s[0]; r.v[2] = s[0]; r.v[3] = z; break;
    case D_LIN4_FROM_V: r.v[0] = z; r.v[1] = cmuli(s[0]); r.v[2] = cscale(cmuli(s[0]), -1.f); r.v[3] = z; break;
    case D_CIRC4_FROM_IQUV:
      r.v[0] = cadd(s[0], s[3]); r.v[1] = cadd(s[1], cmuli(s[2]));
      r.v[2] = csub(s[1], cmuli(s[2])); r.v[3] = csub(s[0], s[3]); break;
    case D_CIRC4_FROM_IQ: r.v[0] = s[0]; r.v[1] = s[1]; r.v[2] = s[1]; r.v[3] = s[0]; break;
    case D_CIRC4_FROM_IU:
      r.v[0] = s[0]; r.v[1] = cmuli(s[1]); r.v[2] = cscale(cmuli(s[1]), -1.f); r.v[3] = s[0]; break;
    case D_CIRC4_FROM_IQU:
      r.v[0] = s[0]; r.v[1] = cadd(s[1], cmuli(s[2])); r.v[2] = csub(s[1], cmuli(s[2])); r.v[3] = s[0]; break;
    case D_LIN4_FROM_IQUV:
      r.v[0] = cadd(s[0], s[1]); r.v[1] = cadd(s[2], cmuli(s[3]));
      r.v[2] = csub(s[2], cmuli(s[3])); r.v[3] = csub(s[0], s[1]); break;
    case D_LIN4_FROM_IQ: case D_LIN2_FROM_IQ: case D_CIRC4_FROM_IV: case D_CIRC2_FROM_IV:
      r.v[0] = cadd(s[0], s[1]); r.v[1] = z; r.v[2] = z; r.v[3] = csub(s[0], s[1]); break;
    case D_LIN4_FROM_IU: r.v[0] = s[0]; r.v[1] = s[1]; r.v[2] = s[1]; r.v[3] = s[0]; break;
    case D_LIN4_FROM_IV:
      r.v[0] = s[0]; r.v[1] = cmuli(s[1]); r.v[2] = cscale(cmuli(s[1]), -1.f); r.v[3] = s[0]; break;
    case D_LIN4_FROM_QU: r.v[0] = s[0]; r.v[1] = s[1]; r.v[2] = s[1]; r.v[3] = cscale(s[0], -1.f); break;
    case D_LIN4_FROM_IQU:
      r.v[0] = cadd(s[0], s[1]); r.v[1] = s[2]; r.v[2] = s[2]; r.v[3] = csub(s[0], s[1]); break;
    default: r = m2_unity(); break;
  }
  return r;
}

// ----------------------------------------------------------------------------------------
// Block geometry: W plane, grid location and oversampling phase (gridder.h:321-351,
// degridder.h:168-200).  Returns false when the reference would skip the block.
// ----------------------------------------------------------------------------------------
struct BlockGeom {
  int locx, locy;  // centre cell
  int sup;         // (S-1)/2
  int S;           // support
  unsigned inv;    // ceil(65536 / S): t / S == (t * inv) >> 16 for every tap t < S*S (S <= 63)
  const float2 *cf;  // first tap of the [io][jo] sub-kernel (S*S taps, row-major sy, sx)
  int cfoff;       // the same tap as an element offset from cf_data
};

// Footprint of a block packed for a warp broadcast: cell index of the footprint's first tap in
// the facet grid array, CF element offset, and support with its reciprocal.
struct TapJob {
  int base;        // ((band * npol) * ny + locy - sup) * nx + locx - sup
  int cfoff;
  int s_inv;       // S | inv << 8
};
__device__ __forceinline__ TapJob tap_job(const BlockGeom &g, int band, const ddfg_facet &f) {
  TapJob j;
  j.base = ((band * f.npol) * f.ny + g.locy - g.sup) * f.nx + g.locx - g.sup;
  j.cfoff = g.cfoff;
  j.s_inv = g.S | (int)(g.inv << 8);
  return j;
}
__device__ __forceinline__ TapJob shfl_job(const TapJob &j, int src) {
  TapJob o;
  o.base = __shfl_sync(0xffffffffu, j.base, src);
  o.cfoff = __shfl_sync(0xffffffffu, j.cfoff, src);
  o.s_inv = __shfl_sync(0xffffffffu, j.s_inv, src);
  return o;
}

// Register slots per lane that hold a footprint of the given support (S*S taps over 32 lanes).
inline int tap_slots(int max_support) {
  const int t = max_support * max_support;
  return t <= 64 ? 2 : (t <= 128 ? 4 : 8);
}

// Per-lane tap offsets for the current support and grid width, recomputed when either changes:
// lane l owns taps t = l + 32 k (k < SLOTS), at cell offset (t / S) * nx + t % S.
template <int SLOTS>
struct LaneTaps {
  int S, NX;
  int off[SLOTS];
  __device__ __forceinline__ void reset() { S = -1; NX = -1; }
  // The offsets depend on the grid width too: facets of one launch may differ in size.
  __device__ __forceinline__ void set(int s_inv, int nx, int lane) {
    const int s = s_inv & 255;
    if (s == S && nx == NX) return;
    S = s;
    NX = nx;
    const unsigned inv = (unsigned)s_inv >> 8;
#pragma unroll
    for (int k = 0; k < SLOTS; ++k) {
      const int t = lane + 32 * k;
      const int sy = (int)(((unsigned)t * inv) >> 16);
      off[k] = (t < s * s) ? sy * nx + (t - sy * s) : -1;
    }
  }
};

// dbg (nullable, [7]): the intermediate integers {iw, plane, locx, locy, offx, offy, k} as far as
// they were formed (the rest untouched) -- ddfg_block_geometry reports them; the kernels pass NULL.
__device__ __forceinline__ bool block_geometry(const ddfg_facet &f, double umean, double vmean, double wmean,
                                               double recip_wvl, BlockGeom &g, int *dbg = nullptr) {
  const double nwd = (double)f.nw;
  // iwplane = lrint((Nw-1)*|W|*(RefWave*recipWvl)/wmax)
  const double t0 = dmul(nwd - 1.0, fabs(wmean));
  const double t1 = dmul(f.ref_wave, recip_wvl);
  const long long iw = lrint_d(dmul(t0, t1) / f.wmax);
  if (dbg) dbg[0] = iw > 0x7fffffffLL ? 0x7fffffff : (int)iw;
  if (iw >= f.nw) return false;
  if (iw < 0) return false;
  const int plane = (wmean > 0.) ? (int)iw : f.nw + (int)iw;
  if (dbg) dbg[1] = plane;
  const int S = f.cf_support[plane];
  const int O = f.overs;
  const int nconv = S * O;
  const int sup = (S - 1) / 2;  // (nConvX/OverS-1)/2
  // pos = (nGridX*incr) * Umean * recipWvl + nGrid/2 ; both axes scale by nGridX (gridder.h:142)
  const double scx = dmul((double)f.nx, f.incr_x);
  const double scy = dmul((double)f.nx, f.incr_y);
  const double posx = dadd(dmul(dmul(scx, umean), recip_wvl), (double)(f.nx / 2));
  const double posy = dadd(dmul(dmul(scy, vmean), recip_wvl), (double)(f.ny / 2));
  const long long lx = lrint_d(posx), ly = lrint_d(posy);
  if (dbg) {
    dbg[2] = (int)lx;
    dbg[3] = (int)ly;
  }
  if (lx - sup < 0 || lx + sup >= f.nx || ly - sup < 0 || ly + sup >= f.ny) return false;
  const int offx = (int)lrint_d(dmul(dsub((double)lx, posx), (double)O)) + (nconv - 1) / 2;
  const int offy = (int)lrint_d(dmul(dsub((double)ly, posy), (double)O)) + (nconv - 1) / 2;
  const int io = offy - sup * O;
  const int jo = offx - sup * O;
  const int k = io * O + jo;
  if (dbg) {
    dbg[4] = offx;
    dbg[5] = offy;
    dbg[6] = k;
  }
  // A position exactly half-way between cells makes the reference read the neighbouring
  // sub-kernel; past either end of the plane it would read outside it, so skip those.
  if (k < 0 || k >= O * O) return false;
  g.locx = (int)lx;
  g.locy = (int)ly;
  g.sup = sup;
  g.S = S;
  g.inv = (65536u + (unsigned)S - 1u) / (unsigned)S;
  g.cfoff = (int)(f.cf_offset[plane] + (int64_t)k * S * S);
  g.cf = (const float2 *)f.cf_data + g.cfoff;
  return true;
}

// Facet descriptors of a launch, copied to shared memory once per CTA: indexing them in the
// kernel parameter space with a loop index would go through local memory.
template <typename Pack>
__device__ __forceinline__ void stage_facets(const Pack &pack, ddfg_facet *sf) {
  const int words = pack.n * (int)(sizeof(ddfg_facet) / sizeof(int));
  const int *src = (const int *)pack.f;
  int *dst = (int *)sf;
  for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
}

}  // namespace ddfg
