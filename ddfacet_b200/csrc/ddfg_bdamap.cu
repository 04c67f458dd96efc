// BDA block maps (mode 1, DDFacet's default) built on the GPU, bit-exact.
//
// Restates GiveBlocksRowsListBL_old (DDFacet/Data/ClassSmearMapping.py:496-625) with one thread
// per baseline (a baseline's blocks depend on a running sum along its rows):
//   * Duv = C dPhi / (pi l nu_max), C = 3e8 (ClassSmearMapping.py:509);
//   * along the baseline's rows: |uvw| -> dnu = (C / pi) dPhi / (|uvw| l), the running minimum of
//     dnu / dFreq, and the running sum of |uvw[i+1] - uvw[i]| (the last difference repeated, 1e-30
//     for a one-row baseline); a block of rows closes when the sum exceeds Duv or the rows end;
//   * its channel blocks: step = max(min dnu/dFreq, 1); ch = arange(0, nchan, step) (+ nchan if
//     absent); chblock = int32(linspace(0, nchan, len(ch))); cut at every change of (channel
//     block, grid band), plus nchan; one block [c0, c1, rows...] per cut interval.
// Every FP64 operation is written with explicit round-to-nearest intrinsics in numpy's
// evaluation order (no contraction), and arange / linspace are evaluated the way numpy fills
// them (value i = i * step; linspace's last value = stop), so the maps equal the host builder's
// word for word.  Two passes: counts per baseline, then the words at scanned offsets.
#include <cuda_runtime.h>

#include "ddfg_internal.h"

namespace {

constexpr double kCBda = 3e8;
constexpr double kPiD = 3.141592653589793;

struct BlKernelArgs {
  const double *uvw;
  const int32_t *rows;      // rows grouped by baseline (key-string order), ascending within one
  const int64_t *bl_off;    // [nbl + 1]
  int32_t nbl;
  int32_t nchan;
  const int32_t *chan_map;  // [nchan] channel -> grid band
  double dfreq, dphi, l, nu0;
  int64_t *nblk, *nwords;                 // pass 1 out: [nbl]
  const int64_t *blk_off, *word_off;      // pass 2 in: [nbl] exclusive scans
  int32_t *sizes, *body;                  // pass 2 out
};

__device__ __forceinline__ double d3norm(double a, double b, double c) {
  return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(c, c)));
}

template <bool WRITE>
__global__ void bda_mode1_kernel(const BlKernelArgs a) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < a.nbl; b += gridDim.x * blockDim.x) {
    const int64_t r0 = a.bl_off[b], n = a.bl_off[b + 1] - r0;
    const double duv = __ddiv_rn(__dmul_rn(kCBda, a.dphi), __dmul_rn(__dmul_rn(kPiD, a.l), a.nu0));
    const double c_over_pi = __ddiv_rn(kCBda, kPiD);
    double nbm = 1e3, duvtot = 0.;
    int64_t start = 0, nb = 0, nw = 0;
    for (int64_t i = 0; i < n; ++i) {
      const int64_t row = a.rows[r0 + i];
      const double u = a.uvw[3 * row], v = a.uvw[3 * row + 1], w = a.uvw[3 * row + 2];
      double du, dv, dw;
      if (n == 1) {
        du = dv = dw = 1e-30;
      } else {
        const int64_t j = (i < n - 1) ? i : n - 2;  // the last difference repeats
        const int64_t ra = a.rows[r0 + j], rb = a.rows[r0 + j + 1];
        du = __dsub_rn(a.uvw[3 * rb], a.uvw[3 * ra]);
        dv = __dsub_rn(a.uvw[3 * rb + 1], a.uvw[3 * ra + 1]);
        dw = __dsub_rn(a.uvw[3 * rb + 2], a.uvw[3 * ra + 2]);
      }
      double uv = d3norm(u, v, w);
      if (1e-10 > uv) uv = 1e-10;
      const double dnu = __ddiv_rn(__dmul_rn(c_over_pi, a.dphi), __dmul_rn(uv, a.l));
      const double ncb = __ddiv_rn(dnu, a.dfreq);
      if (ncb < nbm) nbm = ncb;
      duvtot = __dadd_rn(duvtot, d3norm(du, dv, dw));
      if (duvtot > duv || i == n - 1) {
        const double step = (nbm > 1.) ? nbm : 1.;
        const double fn = (double)a.nchan;
        const int64_t len = (int64_t)ceil(__ddiv_rn(fn, step));
        bool has = false;
        for (int64_t k = len - 3 < 0 ? 0 : len - 3; k < len; ++k) has |= (__dmul_rn((double)k, step) == fn);
        const int64_t nchb = len + (has ? 0 : 1);
        const double lstep = __ddiv_rn(fn, (double)(nchb - 1));
        auto chblock = [&](int64_t jj) -> int { return jj == nchb - 1 ? a.nchan : (int)__dmul_rn((double)jj, lstep); };
        // Cuts at each change of (channel block, band), then nchan; a block per interval.
        const int64_t nrows_blk = i - start + 1;
        int64_t ib = 0;
        int prev_r = -1, prev_b = -1, c_prev = -1;
        for (int ic = 0; ic <= a.nchan; ++ic) {
          bool cut;
          if (ic < a.nchan) {
            while (ib + 1 < nchb - 1 && ic >= chblock(ib + 1)) ++ib;
            const int r = (int)ib, bnd = a.chan_map[ic];
            cut = (r != prev_r || bnd != prev_b);
            prev_r = r;
            prev_b = bnd;
          } else {
            cut = true;  // chblock[-1] = nchan closes the last interval
          }
          if (!cut) continue;
          if (c_prev >= 0) {
            if (WRITE) {
              a.sizes[a.blk_off[b] + nb] = (int32_t)(2 + nrows_blk);
              int32_t *o = a.body + a.word_off[b] + nw;
              o[0] = c_prev;
              o[1] = ic;
              for (int64_t k = 0; k < nrows_blk; ++k) o[2 + k] = a.rows[r0 + start + k];
            }
            ++nb;
            nw += 2 + nrows_blk;
          }
          c_prev = ic;
        }
        nbm = 1e3;
        duvtot = 0.;
        start = i + 1;
      }
    }
    if (!WRITE) {
      a.nblk[b] = nb;
      a.nwords[b] = nw;
    }
  }
}

// Mode 2 (GiveBlocksRowsListBL, ClassSmearMapping.py:348-491) for one baseline per thread:
//   * delta_phase[i] = (2 pi nu0 / C) (|(du, dv)| l_max + |dw| n_max) with duvw[i] = uvw[i] - uvw[i+1]
//     (the last difference repeated), n_max = |sqrt(1 - l_max^2) - 1|;
//   * time blocks: runs of equal int32(cumsum(delta_phase) / dPhi) (every row its own block when
//     dPhi is 0);
//   * per time block: fracmin = max(min over its rows of dnu / dFreq, 1), dnu = (C / 2 pi) dPhi /
//     (|(u, v)| l_max + |w| n_max); size = int32(ceil(nchan / ceil(nchan / fracmin))); channel
//     intervals cut wherever (int32(c / size), band) changes; one block [c0, c1, rows...] each.
// A baseline with a single row is refused (the reference indexes duvw[-2] there and fails): the
// count pass marks it with nblk = -1.
template <bool WRITE>
__global__ void bda_mode2_kernel(const BlKernelArgs a) {
  const double two_pi = 6.283185307179586;  // 2 * np.pi
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < a.nbl; b += gridDim.x * blockDim.x) {
    const int64_t r0 = a.bl_off[b], n = a.bl_off[b + 1] - r0;
    if (n < 2) {
      if (!WRITE) {
        a.nblk[b] = -1;
        a.nwords[b] = 0;
      }
      continue;
    }
    const double l_max = a.l;
    const double n_max = fabs(__dsub_rn(__dsqrt_rn(__dsub_rn(1., __dmul_rn(l_max, l_max))), 1.));
    const double coef = __ddiv_rn(__dmul_rn(two_pi, a.nu0), kCBda);
    const double c2pi_dphi = __dmul_rn(__ddiv_rn(kCBda, two_pi), a.dphi);
    const bool by_phase = __ddiv_rn(__dmul_rn(kCBda, a.dphi), __dmul_rn(two_pi, a.nu0)) != 0.;  // "if Duv"
    auto rowblock = [&](int64_t i, double cum) -> long long {
      return by_phase ? (long long)(int32_t)__ddiv_rn(cum, a.dphi) : i;
    };
    double cum = 0.;
    int64_t start = 0, nb = 0, nw = 0;
    long long cur_blk = 0;
    double fmin = 0.;
    for (int64_t i = 0; i < n; ++i) {
      const int64_t row = a.rows[r0 + i];
      const double *p = a.uvw + 3 * row;
      const int64_t j = (i < n - 1) ? i : n - 2;  // the last difference repeats
      const double *pa = a.uvw + 3 * (int64_t)a.rows[r0 + j], *pb = a.uvw + 3 * (int64_t)a.rows[r0 + j + 1];
      const double du = __dsub_rn(pa[0], pb[0]), dv = __dsub_rn(pa[1], pb[1]), dw = __dsub_rn(pa[2], pb[2]);
      const double dph = __dmul_rn(coef, __dadd_rn(__dmul_rn(__dsqrt_rn(__dadd_rn(__dmul_rn(du, du), __dmul_rn(dv, dv))), l_max),
                                                  __dmul_rn(fabs(dw), n_max)));
      cum = __dadd_rn(cum, dph);
      const long long rb = rowblock(i, cum);
      const double uv = __dadd_rn(__dmul_rn(__dsqrt_rn(__dadd_rn(__dmul_rn(p[0], p[0]), __dmul_rn(p[1], p[1]))), l_max),
                                  __dmul_rn(fabs(p[2]), n_max));
      const double frac = __ddiv_rn(__ddiv_rn(c2pi_dphi, uv), a.dfreq);
      if (i == 0) {
        cur_blk = rb;
        fmin = frac;
      } else if (rb != cur_blk) {
        // rows [start, i) form a time block
        const double fm = fmin > 1. ? fmin : 1.;
        const double ncb = ceil(__ddiv_rn((double)a.nchan, fm));
        const int size = (int)ceil(__ddiv_rn((double)a.nchan, ncb));
        const int64_t nr = i - start;
        int prev_q = -1, prev_b = -1, c_prev = -1;
        for (int ic = 0; ic <= a.nchan; ++ic) {
          bool cut;
          if (ic < a.nchan) {
            const int q = (int)__ddiv_rn((double)ic, (double)size), bnd = a.chan_map[ic];
            cut = (q != prev_q || bnd != prev_b);
            prev_q = q;
            prev_b = bnd;
          } else {
            cut = true;
          }
          if (!cut) continue;
          if (c_prev >= 0) {
            if (WRITE) {
              a.sizes[a.blk_off[b] + nb] = (int32_t)(2 + nr);
              int32_t *o = a.body + a.word_off[b] + nw;
              o[0] = c_prev;
              o[1] = ic;
              for (int64_t k = 0; k < nr; ++k) o[2 + k] = a.rows[r0 + start + k];
            }
            ++nb;
            nw += 2 + nr;
          }
          c_prev = ic;
        }
        start = i;
        cur_blk = rb;
        fmin = frac;
      } else if (frac < fmin) {
        fmin = frac;
      }
    }
    {  // the last time block
      const double fm = fmin > 1. ? fmin : 1.;
      const double ncb = ceil(__ddiv_rn((double)a.nchan, fm));
      const int size = (int)ceil(__ddiv_rn((double)a.nchan, ncb));
      const int64_t nr = n - start;
      int prev_q = -1, prev_b = -1, c_prev = -1;
      for (int ic = 0; ic <= a.nchan; ++ic) {
        bool cut;
        if (ic < a.nchan) {
          const int q = (int)__ddiv_rn((double)ic, (double)size), bnd = a.chan_map[ic];
          cut = (q != prev_q || bnd != prev_b);
          prev_q = q;
          prev_b = bnd;
        } else {
          cut = true;
        }
        if (!cut) continue;
        if (c_prev >= 0) {
          if (WRITE) {
            a.sizes[a.blk_off[b] + nb] = (int32_t)(2 + nr);
            int32_t *o = a.body + a.word_off[b] + nw;
            o[0] = c_prev;
            o[1] = ic;
            for (int64_t k = 0; k < nr; ++k) o[2 + k] = a.rows[r0 + start + k];
          }
          ++nb;
          nw += 2 + nr;
        }
        c_prev = ic;
      }
    }
    if (!WRITE) {
      a.nblk[b] = nb;
      a.nwords[b] = nw;
    }
  }
}

}  // namespace

extern "C" int ddfg_bda_mode2_count(const double *uvw, const int32_t *rows, const int64_t *bl_off, int32_t nbl,
                                    int32_t nchan, const int32_t *chan_map, double dfreq, double dphi, double l_max,
                                    double nu0, int64_t *nblk, int64_t *nwords, void *stream) {
  if (nbl < 0 || nchan < 1) return ddfg_set_error(DDFG_EINVAL, "bda_mode2: bad sizes");
  if (nbl == 0) return DDFG_OK;
  if (!uvw || !rows || !bl_off || !chan_map || !nblk || !nwords)
    return ddfg_set_error(DDFG_EINVAL, "bda_mode2: null pointer");
  BlKernelArgs a{uvw, rows, bl_off, nbl, nchan, chan_map, dfreq, dphi, l_max, nu0, nblk, nwords,
                 nullptr, nullptr, nullptr, nullptr};
  bda_mode2_kernel<false><<<(nbl + 127) / 128, 128, 0, (cudaStream_t)stream>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "bda_mode2 count: %s", cudaGetErrorString(e));
  return DDFG_OK;
}

extern "C" int ddfg_bda_mode2_write(const double *uvw, const int32_t *rows, const int64_t *bl_off, int32_t nbl,
                                    int32_t nchan, const int32_t *chan_map, double dfreq, double dphi, double l_max,
                                    double nu0, const int64_t *blk_off, const int64_t *word_off, int32_t *sizes,
                                    int32_t *body, void *stream) {
  if (nbl < 0 || nchan < 1) return ddfg_set_error(DDFG_EINVAL, "bda_mode2: bad sizes");
  if (nbl == 0) return DDFG_OK;
  if (!uvw || !rows || !bl_off || !chan_map || !blk_off || !word_off || !sizes || !body)
    return ddfg_set_error(DDFG_EINVAL, "bda_mode2: null pointer");
  BlKernelArgs a{uvw, rows, bl_off, nbl, nchan, chan_map, dfreq, dphi, l_max, nu0, nullptr, nullptr,
                 blk_off, word_off, sizes, body};
  bda_mode2_kernel<true><<<(nbl + 127) / 128, 128, 0, (cudaStream_t)stream>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "bda_mode2 write: %s", cudaGetErrorString(e));
  return DDFG_OK;
}

extern "C" int ddfg_bda_mode1_count(const double *uvw, const int32_t *rows, const int64_t *bl_off, int32_t nbl,
                                    int32_t nchan, const int32_t *chan_map, double dfreq, double dphi, double l,
                                    double nu0, int64_t *nblk, int64_t *nwords, void *stream) {
  if (nbl < 0 || nchan < 1) return ddfg_set_error(DDFG_EINVAL, "bda_mode1: bad sizes");
  if (nbl == 0) return DDFG_OK;
  if (!uvw || !rows || !bl_off || !chan_map || !nblk || !nwords)
    return ddfg_set_error(DDFG_EINVAL, "bda_mode1: null pointer");
  BlKernelArgs a{uvw, rows, bl_off, nbl, nchan, chan_map, dfreq, dphi, l, nu0, nblk, nwords,
                 nullptr, nullptr, nullptr, nullptr};
  bda_mode1_kernel<false><<<(nbl + 127) / 128, 128, 0, (cudaStream_t)stream>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "bda_mode1 count: %s", cudaGetErrorString(e));
  return DDFG_OK;
}

extern "C" int ddfg_bda_mode1_write(const double *uvw, const int32_t *rows, const int64_t *bl_off, int32_t nbl,
                                    int32_t nchan, const int32_t *chan_map, double dfreq, double dphi, double l,
                                    double nu0, const int64_t *blk_off, const int64_t *word_off, int32_t *sizes,
                                    int32_t *body, void *stream) {
  if (nbl < 0 || nchan < 1) return ddfg_set_error(DDFG_EINVAL, "bda_mode1: bad sizes");
  if (nbl == 0) return DDFG_OK;
  if (!uvw || !rows || !bl_off || !chan_map || !blk_off || !word_off || !sizes || !body)
    return ddfg_set_error(DDFG_EINVAL, "bda_mode1: null pointer");
  BlKernelArgs a{uvw, rows, bl_off, nbl, nchan, chan_map, dfreq, dphi, l, nu0, nullptr, nullptr,
                 blk_off, word_off, sizes, body};
  bda_mode1_kernel<true><<<(nbl + 127) / 128, 128, 0, (cudaStream_t)stream>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "bda_mode1 write: %s", cudaGetErrorString(e));
  return DDFG_OK;
}
