// Warp-cooperative tap loops shared by the gridding, degridding and adjoint kernels.
#pragma once
#include "ddfg_common.cuh"
#include "ddfg_gridblock.cuh"

namespace ddfg {

// Warp-cooperative tap scatter of the warp's 32 records onto facet f (gridder.h:353-362): each
// record's footprint, CF offset and support travel in three shuffles; each lane keeps the cell
// offsets of its taps for as long as the support and grid width stay the same.  Up to four
// records of equal support are issued together so their CF loads are in flight at once.
// CONJ lays down conj(CF) (the adjoint of the degridder's gather).  Must be called by all 32
// lanes.
template <int NPOL, int SLOTS, bool CONJ = false>
__device__ __forceinline__ void scatter_records(const GridRecord<NPOL> &rec, const ddfg_facet &f, int npol_used,
                                                LaneTaps<SLOTS> &lt, int lane) {
  float2 *grid = (float2 *)f.grid;
  const float2 *cfd = (const float2 *)f.cf_data;
  const int plane_sz = f.nx * f.ny;
  TapJob job;
  if (rec.valid) job = tap_job(rec.g, rec.gridchan, f);
  unsigned mask = __ballot_sync(0xffffffffu, rec.valid);
  if (!mask) return;
  // Fast path: every valid record of the stripe has the same support, which fits the slots (the
  // usual case: a stripe is one row's channels, all on one W plane).  The lane's tap pointers
  // are formed once, and each record costs three shuffles, its CF loads and the reductions.
  const int first = __ffs(mask) - 1;
  const int s_inv0 = __shfl_sync(0xffffffffu, rec.valid ? job.s_inv : 0, first);
  const int S0 = s_inv0 & 255;
  if (S0 * S0 <= 32 * SLOTS && __all_sync(0xffffffffu, !rec.valid || (job.s_inv & 255) == S0)) {
    lt.set(s_inv0, f.nx, lane);
    const float2 *cf_lane = cfd + lane;
    float2 *g_lane[SLOTS];
    bool on[SLOTS];
#pragma unroll
    for (int k = 0; k < SLOTS; ++k) {
      on[k] = lt.off[k] >= 0;
      g_lane[k] = grid + (on[k] ? lt.off[k] : 0);
    }
    while (mask) {
      int src[4];
      int nr = 0;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        src[r] = mask ? __ffs(mask) - 1 : src[0];
        if (mask) {
          mask &= mask - 1;
          ++nr;
        }
      }
      int base[4], cfo[4];
      float2 sv[4][NPOL];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        base[r] = __shfl_sync(0xffffffffu, job.base, src[r]);
        cfo[r] = __shfl_sync(0xffffffffu, job.cfoff, src[r]);
#pragma unroll
        for (int p = 0; p < NPOL; ++p) {
          sv[r][p].x = __shfl_sync(0xffffffffu, rec.stokes[p].x, src[r]);
          sv[r][p].y = __shfl_sync(0xffffffffu, rec.stokes[p].y, src[r]);
        }
      }
      float2 c[4][SLOTS];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int k = 0; k < SLOTS; ++k) c[r][k] = on[k] ? __ldg(cf_lane + cfo[r] + 32 * k) : czero();
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        if (r < nr) {
#pragma unroll
          for (int k = 0; k < SLOTS; ++k) {
            if (on[k]) {
              float2 *cell = g_lane[k] + base[r];
#pragma unroll
              for (int p = 0; p < NPOL; ++p)
                if (NPOL == 1 || p < npol_used) red_add(cell + (size_t)p * plane_sz, cmul(sv[r][p], CONJ ? cconj(c[r][k]) : c[r][k]));
            }
          }
        }
      }
    }
    return;
  }
  while (mask) {
    int src[4];
    int nr = 0;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      src[r] = mask ? __ffs(mask) - 1 : -1;
      if (mask) {
        mask &= mask - 1;
        ++nr;
      }
    }
    TapJob j[4];
    float2 sv[4][NPOL];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int sr = src[r] >= 0 ? src[r] : src[0];
      j[r] = shfl_job(job, sr);
#pragma unroll
      for (int p = 0; p < NPOL; ++p) {
        sv[r][p].x = __shfl_sync(0xffffffffu, rec.stokes[p].x, sr);
        sv[r][p].y = __shfl_sync(0xffffffffu, rec.stokes[p].y, sr);
      }
    }
    const int S = j[0].s_inv & 255;
    bool same = S * S <= 32 * SLOTS;
#pragma unroll
    for (int r = 1; r < 4; ++r) same = same && (r >= nr || (j[r].s_inv & 255) == S);
    if (same) {
      lt.set(j[0].s_inv, f.nx, lane);
      float2 c[4][SLOTS];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int k = 0; k < SLOTS; ++k)
          c[r][k] = (r < nr && lt.off[k] >= 0) ? __ldg(cfd + j[r].cfoff + lane + 32 * k) : czero();
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        if (r >= nr) break;
#pragma unroll
        for (int k = 0; k < SLOTS; ++k) {
          if (lt.off[k] >= 0) {
            float2 *cell = grid + (j[r].base + lt.off[k]);
#pragma unroll
            for (int p = 0; p < NPOL; ++p)
              if (p < npol_used) red_add(cell + (size_t)p * plane_sz, cmul(sv[r][p], CONJ ? cconj(c[r][k]) : c[r][k]));
          }
        }
      }
    } else {
      for (int r = 0; r < nr; ++r) {
        const int Sr = j[r].s_inv & 255;
        const unsigned inv = (unsigned)j[r].s_inv >> 8;
        for (int t = lane; t < Sr * Sr; t += 32) {
          const int sy = (int)(((unsigned)t * inv) >> 16);
          const float2 cv = __ldg(cfd + j[r].cfoff + t);
          float2 *cell = grid + (j[r].base + sy * f.nx + (t - sy * Sr));
#pragma unroll
          for (int p = 0; p < NPOL; ++p)
            if (p < npol_used) red_add(cell + (size_t)p * plane_sz, cmul(sv[r][p], CONJ ? cconj(cv) : cv));
        }
      }
    }
  }
}

// Lane partial sums of the warp's 32 blocks, staged in shared memory and reduced by column:
// lane j adds the 32 partials of block j (one pass instead of a butterfly per block).
constexpr int kPartialBytesPerWarp = 32 * 32 * 8;

// Cooperative gather of every valid record's taps on facet f (degridder.h:202-212): four
// records of equal support at once, lanes on consecutive taps of a CF row; the sum of record r
// ends in lane r's mine[].  For one Stokes plane the lane partials are reduced through the
// warp's shared-memory tile wpart (one column per record); otherwise by butterflies.
// Must be called by all 32 lanes.
template <int NPOL, int SLOTS>
__device__ __forceinline__ void gather_records(bool valid, const TapJob &job, const ddfg_facet &f,
                                               LaneTaps<SLOTS> &lt, float2 *wpart, int lane, float2 *mine) {
#pragma unroll
  for (int p = 0; p < NPOL; ++p) mine[p] = czero();
  const int plane_sz = f.nx * f.ny;
  const float2 *grid = (const float2 *)f.grid;
  const float2 *cfd = (const float2 *)f.cf_data;
  const unsigned vmask = __ballot_sync(0xffffffffu, valid);
  unsigned mask = vmask;
  // Fast path: every valid record has the same support, which fits the slots: the lane's tap
  // pointers are formed once; each record costs two shuffles and its CF and model loads.
  const int first = mask ? __ffs(mask) - 1 : 0;
  const int s_inv0 = __shfl_sync(0xffffffffu, valid ? job.s_inv : 0, first);
  const int S0 = s_inv0 & 255;
  if (mask && S0 * S0 <= 32 * SLOTS && __all_sync(0xffffffffu, !valid || (job.s_inv & 255) == S0)) {
    lt.set(s_inv0, f.nx, lane);
    const float2 *cf_lane = cfd + lane;
    const float2 *g_lane[SLOTS];
    bool on[SLOTS];
#pragma unroll
    for (int k = 0; k < SLOTS; ++k) {
      on[k] = lt.off[k] >= 0;
      g_lane[k] = grid + (on[k] ? lt.off[k] : 0);
    }
    while (mask) {
      int src[4];
      int nr = 0;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        src[r] = mask ? __ffs(mask) - 1 : src[0];
        if (mask) {
          mask &= mask - 1;
          ++nr;
        }
      }
      int base[4], cfo[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        base[r] = __shfl_sync(0xffffffffu, job.base, src[r]);
        cfo[r] = __shfl_sync(0xffffffffu, job.cfoff, src[r]);
      }
      float2 c[4][SLOTS], gv[4][SLOTS][NPOL];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int k = 0; k < SLOTS; ++k) {
          c[r][k] = on[k] ? __ldg(cf_lane + cfo[r] + 32 * k) : czero();
#pragma unroll
          for (int p = 0; p < NPOL; ++p)
            gv[r][k][p] = on[k] ? __ldg(g_lane[k] + base[r] + (size_t)p * plane_sz) : czero();
        }
      float2 acc[4][NPOL];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int p = 0; p < NPOL; ++p) {
          acc[r][p] = czero();
#pragma unroll
          for (int k = 0; k < SLOTS; ++k) acc[r][p] = cadd(acc[r][p], cmul(gv[r][k][p], c[r][k]));
        }
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        if (r >= nr) break;
        if (NPOL == 1) {
          wpart[src[r] * 32 + lane] = acc[r][0];
        } else {
#pragma unroll
          for (int p = 0; p < NPOL; ++p) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
              acc[r][p].x += __shfl_xor_sync(0xffffffffu, acc[r][p].x, o);
              acc[r][p].y += __shfl_xor_sync(0xffffffffu, acc[r][p].y, o);
            }
          }
          if (lane == src[r]) {
#pragma unroll
            for (int p = 0; p < NPOL; ++p) mine[p] = acc[r][p];
          }
        }
      }
    }
  }
  while (mask) {
    // Up to four records of equal support at once: their CF and grid loads overlap.
    int src[4];
    int nr = 0;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      src[r] = mask ? __ffs(mask) - 1 : -1;
      if (mask) {
        mask &= mask - 1;
        ++nr;
      }
    }
    TapJob j[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) j[r] = shfl_job(job, src[r] >= 0 ? src[r] : src[0]);
    const int S = j[0].s_inv & 255;
    bool same = S * S <= 32 * SLOTS;
#pragma unroll
    for (int r = 1; r < 4; ++r) same = same && (r >= nr || (j[r].s_inv & 255) == S);
    float2 acc[4][NPOL];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int p = 0; p < NPOL; ++p) acc[r][p] = czero();
    if (same) {
      lt.set(j[0].s_inv, f.nx, lane);
      float2 c[4][SLOTS], gv[4][SLOTS][NPOL];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int k = 0; k < SLOTS; ++k) {
          const bool on = r < nr && lt.off[k] >= 0;
          c[r][k] = on ? __ldg(cfd + j[r].cfoff + lane + 32 * k) : czero();
#pragma unroll
          for (int p = 0; p < NPOL; ++p)
            gv[r][k][p] = on ? __ldg(grid + (j[r].base + lt.off[k]) + (size_t)p * plane_sz) : czero();
        }
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int k = 0; k < SLOTS; ++k)
#pragma unroll
          for (int p = 0; p < NPOL; ++p) acc[r][p] = cadd(acc[r][p], cmul(gv[r][k][p], c[r][k]));
    } else {
      for (int r = 0; r < nr; ++r) {
        const int Sr = j[r].s_inv & 255;
        const unsigned inv = (unsigned)j[r].s_inv >> 8;
        for (int t = lane; t < Sr * Sr; t += 32) {
          const int sy = (int)(((unsigned)t * inv) >> 16);
          const float2 cv = __ldg(cfd + j[r].cfoff + t);
          const float2 *cell = grid + (j[r].base + sy * f.nx + (t - sy * Sr));
#pragma unroll
          for (int p = 0; p < NPOL; ++p) acc[r][p] = cadd(acc[r][p], cmul(__ldg(cell + (size_t)p * plane_sz), cv));
        }
      }
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      if (r >= nr) break;
      if (NPOL == 1) {
        wpart[src[r] * 32 + lane] = acc[r][0];
      } else {
#pragma unroll
        for (int p = 0; p < NPOL; ++p) {
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) {
            acc[r][p].x += __shfl_xor_sync(0xffffffffu, acc[r][p].x, o);
            acc[r][p].y += __shfl_xor_sync(0xffffffffu, acc[r][p].y, o);
          }
        }
        if (lane == src[r]) {
#pragma unroll
          for (int p = 0; p < NPOL; ++p) mine[p] = acc[r][p];
        }
      }
    }
  }
  if (NPOL == 1) {
    __syncwarp();
    if (valid) {
      float2 t = czero();
#pragma unroll 8
      for (int i = 0; i < 32; ++i) t = cadd(t, wpart[lane * 32 + ((i + lane) & 31)]);
      mine[0] = t;
    }
    __syncwarp();
  }
}

}  // namespace ddfg
