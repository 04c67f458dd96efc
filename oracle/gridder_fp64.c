/*
 * FP64 restatement of DDFacet's BDA gridder and degridder -- TEST INFRASTRUCTURE ONLY.
 *
 * This is the "FP64 oracle": the same algorithm as DDFacet/Gridder/gridder.h:78-377 and
 * degridder.h:55-267 (with JonesServer.cc:25-298, DecorrelationHelper.cc:42-63,
 * CorrelationCalculator.h:37-65, Stokes.h:18-226), but every product and every sum in double
 * precision and the grid accumulated in complex128.  The CF taps, visibilities and Jones
 * matrices are the complex64 inputs promoted to double.  The phasor is exp(i nu angle) evaluated
 * directly in double for every channel (the reference's equidistant-channel recurrence differs
 * from it by rounding only).  The GPU results are compared with it to state their error against
 * an FP64 computation; it is never linked into the product.
 *
 * Built by oracle/build_fp64.sh into oracle/_build/libddfg_fp64.so; driven by oracle/fp64.py.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex dc;
typedef float complex fc;

static const double C_LIGHT = 299792458.;
static const double PI_D = 3.141592653589793238462643383279502884197;

typedef struct { dc v[4]; } M;

static M m_times(M a, M b) {
  M r;
  r.v[0] = a.v[0] * b.v[0] + a.v[1] * b.v[2];
  r.v[1] = a.v[0] * b.v[1] + a.v[1] * b.v[3];
  r.v[2] = a.v[2] * b.v[0] + a.v[3] * b.v[2];
  r.v[3] = a.v[2] * b.v[1] + a.v[3] * b.v[3];
  return r;
}
static M m_herm(M a) {
  M r;
  r.v[0] = conj(a.v[0]);
  r.v[1] = conj(a.v[2]);
  r.v[2] = conj(a.v[1]);
  r.v[3] = conj(a.v[3]);
  return r;
}
static M m_unity(void) {
  M r = {{1, 0, 0, 1}};
  return r;
}

/* Jones inputs (LJones, ClassDDEGridMachine.py:665-677) */
typedef struct {
  int mode; /* 0 none, 1 per visibility, 2 per block */
  const fc *kms;
  int kdims[4];
  const int *ktmap, *kcmap;
  const fc *beam;
  int bdims[4];
  const int *btmap, *bcmap;
  const int *a0, *a1;
  int idir_kms, idir_beam;
  const float *coefs;
  int interp_mode, apply_amp, apply_phase, scale;
  double calib_err, wl_mean;
} JonesIn;

typedef struct {
  const double *uvw_dt; /* NULL: no smearing */
  double dt, dnu, l, m;
  int do_t, do_f;
} SmearIn;

static M give_jones(const fc *J, const int *d, const float *coefs, int it, int ant, int idir, int ich, int mode) {
  size_t nd = (size_t)d[1], na = (size_t)d[2], nch = (size_t)d[3];
  size_t off = (size_t)it * nd * na * nch * 4 + (size_t)idir * na * nch * 4 + (size_t)ant * nch * 4 + (size_t)ich * 4;
  M out;
  if (mode == 0) {
    for (int p = 0; p < 4; ++p) out.v[p] = J[off + p];
    return out;
  }
  double jabs[4] = {0, 0, 0, 0};
  for (int p = 0; p < 4; ++p) out.v[p] = 0;
  for (size_t k = 0; k < nd; ++k) {
    double c = coefs[k];
    if (c == 0) continue;
    for (int p = 0; p < 4; ++p) {
      dc val = J[off + p];
      double a = cabs(val);
      out.v[p] += c / a * val;
      jabs[p] += c * a;
    }
  }
  for (int p = 0; p < 4; ++p) out.v[p] *= jabs[p];
  return out;
}

static void norm_jones(M *j, const JonesIn *js, const double *uvw) {
  if (!js->apply_amp)
    for (int p = 0; p < 4; ++p) {
      double a = cabs(j->v[p]);
      if (a != 0) j->v[p] /= a;
    }
  if (!js->apply_phase)
    for (int p = 0; p < 4; ++p) j->v[p] = cabs(j->v[p]);
  if (js->scale) {
    double r2 = (uvw[0] * uvw[0] + uvw[1] * uvw[1]) / (js->wl_mean * js->wl_mean);
    double al = exp(-2. * PI_D * js->calib_err * js->calib_err * r2);
    for (int p = 0; p < 4; ++p) {
      double a = cabs(j->v[p]);
      if (a != 0) j->v[p] *= (1. - al) / a + al;
    }
  }
}

/* J0, J1 and BB for a row/channel (JonesServer.cc:193-298, without the cache). */
static void jones_at(const JonesIn *js, int64_t row, int ch, const double *uvw, M *j0, M *j1, double *bb) {
  int a0 = js->a0[row], a1 = js->a1[row];
  M A = m_unity(), B = m_unity();
  if (js->beam) {
    int t = js->btmap[row], c = js->bcmap[ch];
    A = give_jones(js->beam, js->bdims, js->coefs, t, a0, js->idir_beam, c, js->interp_mode);
    B = give_jones(js->beam, js->bdims, js->coefs, t, a1, js->idir_beam, c, js->interp_mode);
  }
  if (js->kms) {
    int t = js->ktmap[row], c = js->kcmap[ch];
    M k0 = give_jones(js->kms, js->kdims, js->coefs, t, a0, js->idir_kms, c, js->interp_mode);
    M k1 = give_jones(js->kms, js->kdims, js->coefs, t, a1, js->idir_kms, c, js->interp_mode);
    norm_jones(&k0, js, uvw);
    norm_jones(&k1, js, uvw);
    A = m_times(k0, A);
    B = m_times(k1, B);
  }
  *j0 = A;
  *j1 = B;
  double t = (cabs(A.v[0]) * cabs(B.v[0]) + cabs(A.v[3]) * cabs(B.v[3])) / 2.;
  *bb = t * t;
}

static double decorr(const SmearIn *sm, const double *uvw, double nu, int64_t idx) {
  if (!sm->uvw_dt) return 1.;
  double l = sm->l, m = sm->m, n0 = sqrt(1. - l * l - m * m) - 1., f = 1.;
  if (sm->do_f) {
    double ph = uvw[3 * idx] * l + uvw[3 * idx + 1] * m + uvw[3 * idx + 2] * n0;
    double phi = PI_D * sm->dnu / C_LIGHT * ph;
    f *= (phi == 0.) ? 1. : sin(phi) / phi;
  }
  if (sm->do_t) {
    const double *p = sm->uvw_dt + 3 * idx;
    double dph = (p[0] * l + p[1] * m + p[2] * n0) * sm->dt;
    double phi = PI_D * nu / C_LIGHT * dph;
    f *= (phi == 0.) ? 1. : sin(phi) / phi;
  }
  return f;
}

/* ---------------- correlation / Stokes dispatch (GridderSmearPols.cc:98-348) ---------------- */
enum { C_BAD = -1, C_I, C_LIN2, C_CIRC2, C_LIN4, C_CIRC4 };
static int corr_set(const int *c, int n) {
  if (n == 1 && c[0] == 1) return C_I;
  if (n == 2 && c[0] == 9 && c[1] == 12) return C_LIN2;
  if (n == 2 && c[0] == 5 && c[1] == 8) return C_CIRC2;
  if (n == 4 && c[0] == 9 && c[1] == 10 && c[2] == 11 && c[3] == 12) return C_LIN4;
  if (n == 4 && c[0] == 5 && c[1] == 6 && c[2] == 7 && c[3] == 8) return C_CIRC4;
  return C_BAD;
}
static void sstr(const int *s, int n, char *out) {
  const char *nm = "?IQUV";
  for (int i = 0; i < n; ++i) out[i] = (s[i] >= 1 && s[i] <= 4) ? nm[s[i]] : '?';
  out[n] = 0;
}

/* Stokes from the accumulated 2x2 (Stokes.h:18-77).  Returns 0 if unsupported. */
static int stokes_grid(int cs, const char *st, M V, dc *out) {
  dc ipp = (V.v[0] + V.v[3]) * .5, imm = (V.v[0] - V.v[3]) * .5, xpp = (V.v[1] + V.v[2]) * .5;
  dc xmm = -(V.v[1] - V.v[2]) * (.5 * I);
  if (cs == C_I && !strcmp(st, "I")) { out[0] = V.v[0]; return 1; }
  if (cs == C_LIN2 || cs == C_CIRC2) {
    if (!strcmp(st, "I")) { out[0] = ipp; return 1; }
    if (cs == C_LIN2 && !strcmp(st, "IQ")) { out[0] = ipp; out[1] = imm; return 1; }
    if (cs == C_CIRC2 && !strcmp(st, "IV")) { out[0] = ipp; out[1] = imm; return 1; }
    return 0;
  }
  if (cs == C_LIN4) {
    if (!strcmp(st, "I")) { out[0] = ipp; return 1; }
    if (!strcmp(st, "Q")) { out[0] = imm; return 1; }
    if (!strcmp(st, "U")) { out[0] = xpp; return 1; }
    if (!strcmp(st, "V")) { out[0] = xmm; return 1; }
    if (!strcmp(st, "IQ") || !strcmp(st, "IU")) { out[0] = ipp; out[1] = imm; return 1; }
    if (!strcmp(st, "IV")) { out[0] = ipp; out[1] = xmm; return 1; }
    if (!strcmp(st, "QU")) { out[0] = imm; out[1] = xpp; return 1; }
    if (!strcmp(st, "IQU")) { out[0] = ipp; out[1] = imm; out[2] = xpp; return 1; }
    if (!strcmp(st, "IQUV")) { out[0] = ipp; out[1] = imm; out[2] = xpp; out[3] = xmm; return 1; }
    return 0;
  }
  if (cs == C_CIRC4) {
    if (!strcmp(st, "I")) { out[0] = ipp; return 1; }
    if (!strcmp(st, "IQ")) { out[0] = ipp; out[1] = xpp; return 1; }
    if (!strcmp(st, "IU")) { out[0] = ipp; out[1] = xmm; return 1; }
    if (!strcmp(st, "IV")) { out[0] = ipp; out[1] = imm; return 1; }
    if (!strcmp(st, "QU")) { out[0] = xpp; out[1] = xmm; return 1; }
    if (!strcmp(st, "IQU")) { out[0] = ipp; out[1] = xpp; out[2] = xmm; return 1; }
    if (!strcmp(st, "IQUV")) { out[0] = ipp; out[1] = xpp; out[2] = xmm; out[3] = imm; return 1; }
    return 0;
  }
  return 0;
}

/* Correlations from Stokes (Stokes.h:90-226).  Returns 0 if unsupported. */
static int corr_degrid(int cs, const char *st, const dc *s, M *r) {
  dc z = 0;
  if (!strcmp(st, "I") && cs != C_BAD) { *r = (M){{s[0], z, z, s[0]}}; return 1; }
  if (cs == C_LIN4) {
    if (!strcmp(st, "Q")) { *r = (M){{s[0], z, z, -s[0]}}; return 1; }
    if (!strcmp(st, "U")) { *r = (M){{z, s[0], s[0], z}}; return 1; }
    if (!strcmp(st, "V")) { *r = (M){{z, I * s[0], -I * s[0], z}}; return 1; }
    if (!strcmp(st, "IQUV")) { *r = (M){{s[0] + s[1], s[2] + I * s[3], s[2] - I * s[3], s[0] - s[1]}}; return 1; }
    if (!strcmp(st, "IQ")) { *r = (M){{s[0] + s[1], z, z, s[0] - s[1]}}; return 1; }
    if (!strcmp(st, "IU")) { *r = (M){{s[0], s[1], s[1], s[0]}}; return 1; }
    if (!strcmp(st, "IV")) { *r = (M){{s[0], I * s[1], -I * s[1], s[0]}}; return 1; }
    if (!strcmp(st, "QU")) { *r = (M){{s[0], s[1], s[1], -s[0]}}; return 1; }
    if (!strcmp(st, "IQU")) { *r = (M){{s[0] + s[1], s[2], s[2], s[0] - s[1]}}; return 1; }
  }
  if (cs == C_CIRC4) {
    if (!strcmp(st, "IQUV")) { *r = (M){{s[0] + s[3], s[1] + I * s[2], s[1] - I * s[2], s[0] - s[3]}}; return 1; }
    if (!strcmp(st, "IQ")) { *r = (M){{s[0], s[1], s[1], s[0]}}; return 1; }
    if (!strcmp(st, "IU")) { *r = (M){{s[0], I * s[1], -I * s[1], s[0]}}; return 1; }
    if (!strcmp(st, "IV")) { *r = (M){{s[0] + s[1], z, z, s[0] - s[1]}}; return 1; }
    if (!strcmp(st, "IQU")) { *r = (M){{s[0], s[1] + I * s[2], s[1] - I * s[2], s[0]}}; return 1; }
  }
  if (cs == C_LIN2 && !strcmp(st, "IQ")) { *r = (M){{s[0] + s[1], z, z, s[0] - s[1]}}; return 1; }
  if (cs == C_CIRC2 && !strcmp(st, "IV")) { *r = (M){{s[0] + s[1], z, z, s[0] - s[1]}}; return 1; }
  return 0;
}

/* W plane, location and CF offset (gridder.h:321-351).  Returns 0 to skip.  dbg (nullable, [7])
 * receives {iw, plane, locx, locy, offx, offy, k} as far as they are formed. */
static int geometry(double nw, int overs, double ref_wave, double wmax, const int64_t *cf_off, const int *cf_sup,
                    int nx, int ny, double incr_x, double incr_y, double U, double V, double W, double recip,
                    int64_t *cfo, int *lx, int *ly, int *S, int *dbg) {
  long iw = lrint((nw - 1) * fabs(W) * (ref_wave * recip) / wmax);
  if (dbg) dbg[0] = iw > 0x7fffffffL ? 0x7fffffff : (int)iw;
  if (iw >= (long)nw || iw < 0) return 0;
  int plane = (W > 0) ? (int)iw : (int)nw + (int)iw;
  if (dbg) dbg[1] = plane;
  int s = cf_sup[plane], nconv = s * overs, sup = (s - 1) / 2;
  double posx = nx * incr_x * U * recip + (double)(nx / 2);
  double posy = nx * incr_y * V * recip + (double)(ny / 2);
  long locx = lrint(posx), locy = lrint(posy);
  if (dbg) { dbg[2] = (int)locx; dbg[3] = (int)locy; }
  if (locx - sup < 0 || locx + sup >= nx || locy - sup < 0 || locy + sup >= ny) return 0;
  int offx = (int)(lrint((locx - posx) * overs) + (nconv - 1) / 2);
  int offy = (int)(lrint((locy - posy) * overs) + (nconv - 1) / 2);
  int k = (offy - sup * overs) * overs + (offx - sup * overs);
  if (dbg) { dbg[4] = offx; dbg[5] = offy; dbg[6] = k; }
  if (k < 0 || k >= overs * overs) return 0;
  *cfo = cf_off[plane] + (int64_t)k * s * s;
  *lx = (int)locx;
  *ly = (int)locy;
  *S = s;
  return 1;
}

/* Word index of every block record of a packed map (the sequential walk of gridder.h:144-148). */
static int64_t *block_starts(const int *bmap, size_t nb) {
  int64_t *st = malloc(sizeof(int64_t) * (nb ? nb : 1));
  int64_t w = 2 + (int64_t)nb;
  for (size_t b = 0; b < nb; ++b) {
    st[b] = w;
    w += bmap[2 + b];
  }
  return st;
}

/* {status, iw, plane, locx, locy, offx, offy, k} of every block, from the gridder's block means
 * (unflagged visibilities, gridder.h:272-289) or, with degrid_means, the degridder's (rows and
 * channels, degridder.h:138-167): the integer indices the GPU's ddfg_block_geometry reports. */
int fp64_block_indices(const double *uvw, const uint8_t *flags, int nchan, int ncorr, const double *freqs,
                       const int *chan_map, const int *bmap, const int64_t *cf_off, const int *cf_sup, int nw,
                       int overs, double ref_wave, double wmax, int nx, int ny, int nband, double incr_x,
                       double incr_y, double cu, double cv, int degrid_means, int *out) {
  size_t nb = (size_t)(uint32_t)bmap[0] + ((size_t)bmap[1] << 32);
  int64_t *st = block_starts(bmap, nb);
#pragma omp parallel for schedule(dynamic, 4096)
  for (size_t b = 0; b < nb; ++b) {
    const int *p = bmap + st[b];
    int nr = bmap[2 + b] - 2, c0 = p[0], c1 = p[1];
    const int *rows = p + 2;
    int dbg[7] = {-1, -1, -1, -1, -1, -1, -1}, ok = 0;
    int64_t cfo;
    int lx, ly, S;
    double um = 0, vmn = 0, wm = 0, fm = 0;
    int gch = chan_map[c0 < nchan ? c0 : 0];
    if (degrid_means) {
      if (gch >= 0 && gch < nband && nr > 0 && c1 > c0) {
        for (int c = c0; c < c1; ++c) fm += freqs[c];
        if (c1 - c0 > 1) fm /= (c1 - c0);
        for (int i = 0; i < nr; ++i) {
          const double *u = uvw + 3 * (int64_t)rows[i];
          um += u[0] + u[2] * cu;
          vmn += u[1] + u[2] * cv;
          wm += u[2];
        }
        if (nr > 1) { um /= nr; vmn /= nr; wm /= nr; }
        ok = geometry(nw, overs, ref_wave, wmax, cf_off, cf_sup, nx, ny, incr_x, incr_y, um, vmn, wm, fm / C_LIGHT,
                      &cfo, &lx, &ly, &S, dbg);
      }
    } else {
      int n = 0;
      for (int i = 0; i < nr; ++i) {
        const double *u = uvw + 3 * (int64_t)rows[i];
        for (int c = c0; c < c1; ++c) {
          if (flags[((int64_t)rows[i] * nchan + c) * ncorr]) continue;
          um += u[0] + u[2] * cu;
          vmn += u[1] + u[2] * cv;
          wm += u[2];
          fm += freqs[c];
          ++n;
        }
      }
      if (n > 0 && gch >= 0 && gch < nband) {
        if (n > 1) { um /= n; vmn /= n; wm /= n; fm /= n; }
        ok = geometry(nw, overs, ref_wave, wmax, cf_off, cf_sup, nx, ny, incr_x, incr_y, um, vmn, wm, fm / C_LIGHT,
                      &cfo, &lx, &ly, &S, dbg);
      }
    }
    int *o = out + 8 * b;
    o[0] = ok;
    for (int i = 0; i < 7; ++i) o[1 + i] = dbg[i];
  }
  free(st);
  return 0;
}

/* Returns 0, or -2 for an unsupported correlation/Stokes combination. */
int fp64_grid(dc *grid, int nband, int npol, int ny, int nx, const fc *vis, const double *uvw, const uint8_t *flags,
              const float *weights, int64_t nrow, int nchan, int ncorr, const double *freqs, const int *chan_map,
              const int *bmap, const fc *cf, const int64_t *cf_off, const int *cf_sup, int nw, int overs,
              double ref_wave, double wmax, double incr_x, double incr_y, double cu, double cv, double l0, double m0,
              const int *corr_ids, int ncorr_ids, const int *stokes_ids, int nstokes, int dopsf, const JonesIn *js,
              const SmearIn *sm, const uint8_t *sparsification, double *sumwt, double *sumjones,
              double *sumjones_chan) {
  char st[8];
  sstr(stokes_ids, nstokes, st);
  int cs = corr_set(corr_ids, ncorr_ids);
  { dc tmp[4]; M z = m_unity(); if (!stokes_grid(cs, st, z, tmp)) return -2; }
  double n0 = sqrt(1 - l0 * l0 - m0 * m0) - 1, fm0 = 0;
  for (int c = 0; c < nchan; ++c) fm0 += freqs[c];
  fm0 /= nchan;
  size_t nb = (size_t)(uint32_t)bmap[0] + ((size_t)bmap[1] << 32);
  const int *sizes = bmap + 2;
  int64_t *starts = block_starts(bmap, nb);
  const size_t gcells = (size_t)nband * npol * nx * ny;
  /* Large maps run on all host threads, each into its own complex128 grid and sums (added in
   * thread order at the end); small ones on one thread. */
  int nthr = 1;
#ifdef _OPENMP
  if (nb > 200000) nthr = omp_get_max_threads();
#endif
#pragma omp parallel num_threads(nthr)
  {
  int tid = 0;
#ifdef _OPENMP
  tid = omp_get_thread_num();
#endif
  dc *tgrid = tid == 0 ? grid : calloc(gcells, sizeof(dc));
  double *tsumwt = calloc((size_t)nband * npol, sizeof(double));
  double *tsj = calloc(2 * (size_t)nband, sizeof(double));
  double *tsjc = calloc(2 * (size_t)nchan, sizeof(double));
  double *chj = calloc((size_t)nchan, sizeof(double)), *chq = calloc((size_t)nchan, sizeof(double));
#pragma omp for schedule(dynamic, 2048)
  for (size_t b = 0; b < nb; ++b) {
    const int *p = bmap + starts[b];
    int nr = sizes[b] - 2, c0 = p[0], c1 = p[1];
    const int *rows = p + 2;
    if (sparsification && !sparsification[b]) continue;
    if (nr <= 0) continue;
    memset(chj, 0, sizeof(double) * nchan);
    memset(chq, 0, sizeof(double) * nchan);
    double dec = decorr(sm, uvw, fm0, rows[nr / 2]);
    M acc = {{0, 0, 0, 0}}, vm = {{dec, 0, 0, dec}};
    double um = 0, vmn = 0, wm = 0, fm = 0, tw = 0, sj = 0, sq = 0;
    int n = 0;
    for (int i = 0; i < nr; ++i) {
      int64_t r = rows[i];
      const double *u = uvw + 3 * r;
      double ang = -2. * PI_D * (u[0] * l0 + u[1] * m0 + u[2] * n0) / C_LIGHT;
      for (int c = c0; c < c1; ++c) {
        int64_t off = (r * nchan + c) * ncorr;
        if (flags[off]) continue;
        dc corr = dopsf ? 1. : cexp(I * freqs[c] * ang);
        M j0, j1;
        double bb = 1;
        if (js->mode == 1) {
          jones_at(js, r, c, u, &j0, &j1, &bb);
          if (dopsf) {
            vm = m_times(j0, m_herm(j1));
            vm = m_times(m_times(m_herm(j0), vm), j1);
            for (int q = 0; q < 4; ++q) vm.v[q] *= dec;
          }
        }
        if (!dopsf) {
          const fc *vp = vis + off;
          if (ncorr == 4) vm = (M){{vp[0], vp[1], vp[2], vp[3]}};
          else if (ncorr == 2) vm = (M){{vp[0], 0, 0, vp[1]}};
          else vm = (M){{vp[0], 0, 0, vp[0]}};
        }
        double fw = weights[r * nchan + c], fwd = fw * dec * dec;
        dc w = fw * corr;
        sq += fwd;
        chq[c] += fwd;
        M x = vm;
        if (js->mode == 1) {
          if (!dopsf) x = m_times(m_times(m_herm(j0), vm), j1);
          sj += bb * fwd;
          chj[c] += bb * fwd;
        }
        acc.v[0] += x.v[0] * w;
        if (ncorr == 4) { acc.v[1] += x.v[1] * w; acc.v[2] += x.v[2] * w; }
        if (ncorr >= 2) acc.v[3] += x.v[3] * w;
        um += u[0] + u[2] * cu;
        vmn += u[1] + u[2] * cv;
        wm += u[2];
        fm += freqs[c];
        tw += fw;
        ++n;
      }
    }
    if (n == 0) continue;
    um /= n; vmn /= n; wm /= n; fm /= n;
    if (js->mode == 2) {
      double uvwm[3] = {um, vmn, wm}, bb;
      M j0, j1;
      jones_at(js, rows[nr / 2], (c0 + c1) / 2, uvwm, &j0, &j1, &bb);
      if (dopsf) acc = m_times(m_times(j0, acc), m_herm(j1));
      acc = m_times(m_times(m_herm(j0), acc), j1);
      sj = sq * bb;
      for (int c = c0; c < c1; ++c) chj[c] = chq[c] * bb;
    }
    int gch = chan_map[c0];
    if (gch < 0 || gch >= nband) continue;
    int64_t cfo;
    int lx, ly, S;
    if (!geometry(nw, overs, ref_wave, wmax, cf_off, cf_sup, nx, ny, incr_x, incr_y, um, vmn, wm, fm / C_LIGHT, &cfo,
                  &lx, &ly, &S, NULL))
      continue;
    dc sv[4];
    stokes_grid(cs, st, acc, sv);
    int sup = (S - 1) / 2;
    for (int ip = 0; ip < nstokes; ++ip) {
      if (ip >= npol) continue;
      dc *g = tgrid + ((size_t)gch * npol + ip) * (size_t)nx * ny;
      const fc *c = cf + cfo;
      for (int sy = -sup; sy <= sup; ++sy)
        for (int sx = -sup; sx <= sup; ++sx) g[(size_t)(ly + sy) * nx + lx + sx] += sv[ip] * (dc)(*c++);
      tsumwt[ip + gch * npol] += tw;
      if (js->mode) {
        tsj[gch] += sj;
        tsj[gch + nband] += sq;
        for (int cc = c0; cc < c1; ++cc) {
          tsjc[cc] += chj[cc];
          tsjc[nchan + cc] += chq[cc];
        }
      }
    }
  }
  /* thread order: deterministic for a given thread count */
  for (int t = 0; t < nthr; ++t) {
#pragma omp barrier
    if (t == tid) {
      if (tid != 0)
        for (size_t i = 0; i < gcells; ++i) grid[i] += tgrid[i];
      for (int i = 0; i < nband * npol; ++i) sumwt[i] += tsumwt[i];
      if (js->mode) {
        for (int i = 0; i < 2 * nband; ++i) sumjones[i] += tsj[i];
        for (int i = 0; i < 2 * nchan; ++i) sumjones_chan[i] += tsjc[i];
      }
    }
  }
  if (tid != 0) free(tgrid);
  free(tsumwt);
  free(tsj);
  free(tsjc);
  free(chj);
  free(chq);
  }
  free(starts);
  return 0;
}

/* Subtracts the prediction from vis (complex128 [nrow][nchan][ncorr]).  cf planes in the
 * degridder's order (WplanesConj first, as ClassDDEGridMachine.get passes them). */
int fp64_degrid(const fc *grid, int nband, int npol, int ny, int nx, dc *vis, const double *uvw, int64_t nrow,
                int nchan, int ncorr, const double *freqs, const int *chan_map, const int *bmap, const fc *cf,
                const int64_t *cf_off, const int *cf_sup, int nw, int overs, double ref_wave, double wmax,
                double incr_x, double incr_y, double cu, double cv, double l0, double m0, const int *corr_ids,
                int ncorr_ids, const int *stokes_ids, int nstokes, const JonesIn *js, const SmearIn *sm) {
  char st[8];
  sstr(stokes_ids, nstokes, st);
  int cs = corr_set(corr_ids, ncorr_ids);
  { dc tmp[4] = {0, 0, 0, 0}; M r; if (!corr_degrid(cs, st, tmp, &r)) return -2; }
  (void)nrow;
  double n0 = sqrt(1 - l0 * l0 - m0 * m0) - 1;
  size_t nb = (size_t)(uint32_t)bmap[0] + ((size_t)bmap[1] << 32);
  const int *sizes = bmap + 2;
  int64_t *starts = block_starts(bmap, nb);
  int nthr = 1;
#ifdef _OPENMP
  if (nb > 200000) nthr = omp_get_max_threads();
#endif
  /* blocks of one map hold disjoint visibilities: parallel over blocks on large maps */
#pragma omp parallel for num_threads(nthr) schedule(dynamic, 2048)
  for (size_t b = 0; b < nb; ++b) {
    const int *p = bmap + starts[b];
    int nr = sizes[b] - 2, c0 = p[0], c1 = p[1];
    const int *rows = p + 2;
    int gch = chan_map[c0 < nchan ? c0 : 0];
    if (gch < 0 || gch >= nband || nr <= 0 || c1 <= c0) continue;
    double fm = 0, um = 0, vmn = 0, wm = 0;
    for (int c = c0; c < c1; ++c) fm += freqs[c];
    fm /= (c1 - c0);
    for (int i = 0; i < nr; ++i) {
      const double *u = uvw + 3 * (int64_t)rows[i];
      um += u[0] + u[2] * cu;
      vmn += u[1] + u[2] * cv;
      wm += u[2];
    }
    um /= nr; vmn /= nr; wm /= nr;
    int64_t cfo;
    int lx, ly, S;
    if (!geometry(nw, overs, ref_wave, wmax, cf_off, cf_sup, nx, ny, incr_x, incr_y, um, vmn, wm, fm / C_LIGHT, &cfo,
                  &lx, &ly, &S, NULL))
      continue;
    int sup = (S - 1) / 2;
    dc sv[4] = {0, 0, 0, 0};
    for (int ip = 0; ip < nstokes; ++ip) {
      const fc *g = grid + ((size_t)gch * npol + ip) * (size_t)nx * ny;
      const fc *c = cf + cfo;
      dc a = 0;
      for (int sy = -sup; sy <= sup; ++sy)
        for (int sx = -sup; sx <= sup; ++sx) a += (dc)g[(size_t)(ly + sy) * nx + lx + sx] * (dc)(*c++);
      sv[ip] = a;
    }
    M cv_;
    corr_degrid(cs, st, sv, &cv_);
    int mid = rows[nr / 2];
    if (js->mode == 2) {
      M j0, j1;
      double bb;
      jones_at(js, mid, (c0 + c1) / 2, uvw + 3 * (int64_t)mid, &j0, &j1, &bb);
      cv_ = m_times(m_times(j0, cv_), m_herm(j1));
    }
    double dec = decorr(sm, uvw, fm, mid);
    for (int i = 0; i < nr; ++i) {
      int64_t r = rows[i];
      const double *u = uvw + 3 * r;
      double ang = 2. * PI_D * (u[0] * l0 + u[1] * m0 + u[2] * n0) / C_LIGHT;
      for (int c = c0; c < c1; ++c) {
        dc corr = cexp(I * freqs[c] * ang) * dec;
        M vb = cv_;
        if (js->mode == 1) {
          M j0, j1;
          double bb;
          jones_at(js, r, c, u, &j0, &j1, &bb);
          vb = m_times(m_times(j0, cv_), m_herm(j1));
        }
        dc *vp = vis + (r * nchan + c) * ncorr;
        if (ncorr == 4) for (int q = 0; q < 4; ++q) vp[q] -= vb.v[q] * corr;
        else if (ncorr == 2) { vp[0] -= vb.v[0] * corr; vp[1] -= vb.v[3] * corr; }
        else vp[0] -= vb.v[0] * corr;
      }
    }
  }
  free(starts);
  return 0;
}
