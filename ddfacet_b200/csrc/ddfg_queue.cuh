// Persistent, queue-driven scheduling of the gridding and degridding kernels, and the tap
// scatter they share (run merging, optional FP64 accumulation).
//
// One launch takes up to DDFG_TABLE_FACETS facet descriptors as a __grid_constant__ parameter
// table.  The facets are split into packs of balanced size; a work item is a run of stripes
// (32 consecutive blocks) of one pack, or a few large blocks of one pack.  Items are numbered
// pack by pack (large-block items of a pack first, so the longest work starts first); a CTA takes
// the next item number from a counter in device memory (or, without a counter, every gridDim.x-th
// item), stages the pack's descriptors in shared memory when the pack changes, and its warps take
// the item's stripes one at a time from a shared-memory counter.  The pack-major order keeps the
// grids of one pack at a time live in L2, and the queue balances facets and blocks of unequal cost
// across the GPU without a host-side plan.
#pragma once
#include "ddfg_common.cuh"
#include "ddfg_gridblock.cuh"

namespace ddfg {

struct FacetTable {
  ddfg_facet f[DDFG_TABLE_FACETS];
};

struct Sched {
  int nfacets;               // facets of this launch
  int npacks;
  int max_pack;              // most facets in one pack (shared-memory sizing)
  int acc_stride;            // doubles of one facet's shared accumulators (gridding), 0 otherwise:
                             // [warps][small_stride] weight/Jones sums, then [2][nchan] channel sums
  int small_stride;          // doubles of one warp's weight and Jones sums of one facet
  int tiles;                 // 1: the warps have grid tiles (scatter_tile) at the start of shared memory
  long long nstripes;        // stripes of 32 blocks
  long long spi;             // stripes per item
  long long stripe_items;    // ceil(nstripes / spi)
  int large_per_item;        // large blocks per item
  long long large_items;     // ceil(nlarge / large_per_item)
  long long regions;         // stripe items interleaved over this many regions (1: in order)
  long long per_region;      // ceil(stripe_items / regions)
  long long items_per_pack;  // large_items + stripe item slots (regions * per_region)
  long long nitems;          // npacks * items_per_pack
  unsigned long long *counter;  // item counter (zeroed before the launch), or NULL: static order
};

// Host: spreads a pack's stripe items over `regions` contiguous regions of the block order, taken
// in turn, so that CTAs holding consecutive item numbers work far apart in the map (for a map in
// uv-cell order: far apart on the grids, which keeps concurrent grid additions off the same
// cells).  With the static order and as many regions as CTAs, each CTA walks one region.
inline void sched_set_regions(Sched &sc, long long regions) {
  regions = regions < 1 ? 1 : (regions > sc.stripe_items ? sc.stripe_items : regions);
  if (regions < 1) regions = 1;
  sc.regions = regions;
  sc.per_region = (sc.stripe_items + regions - 1) / regions;
  sc.items_per_pack = sc.large_items + (regions > 1 ? regions * sc.per_region : sc.stripe_items);
  sc.nitems = sc.items_per_pack * sc.npacks;
}

// First stripe of stripe-item slot rr of a pack (0 <= rr < items_per_pack - large_items); slots
// past the last stripe give a start >= nstripes (an empty item).
__device__ __forceinline__ long long slot_stripe(const Sched &sc, long long rr) {
  const long long it = sc.regions > 1 ? (rr % sc.regions) * sc.per_region + rr / sc.regions : rr;
  return it * sc.spi;
}

__device__ __forceinline__ int pack_first(const Sched &sc, int p) {
  return (int)(((long long)p * sc.nfacets) / sc.npacks);
}

// Shared state of a CTA's walk over the queue.
struct QueueSmem {
  long long item;
  int next;  // next stripe (or large block) of the current item
};

// Takes the CTA's next item (all threads call it; returns the same value to all).
__device__ __forceinline__ long long queue_next(const Sched &sc, QueueSmem *q, long long &static_next) {
  __syncthreads();  // every thread has finished the previous item and read q->item
  if (threadIdx.x == 0) {
    q->item = sc.counter ? (long long)atomicAdd(sc.counter, 1ull) : static_next;
    q->next = 0;
  }
  static_next += gridDim.x;
  __syncthreads();
  return q->item;
}

// The warp's next unit of the current item (stripe or large block), or -1 when it is exhausted.
__device__ __forceinline__ int warp_take(QueueSmem *q, int limit, int lane) {
  int k = 0;
  if (lane == 0) k = atomicAdd(&q->next, 1);
  k = __shfl_sync(0xffffffffu, k, 0);
  return k < limit ? k : -1;
}

// Copies pack p's descriptors into shared memory (all threads call it).
__device__ __forceinline__ int stage_pack(const FacetTable &tab, const Sched &sc, int p, ddfg_facet *sf,
                                          double *s_n0m1) {
  const int f0 = pack_first(sc, p), f1 = pack_first(sc, p + 1);
  const int n = f1 - f0;
  const int words = n * (int)(sizeof(ddfg_facet) / sizeof(int));
  const int *src = (const int *)&tab.f[f0];
  int *dst = (int *)sf;
  for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const ddfg_facet &f = tab.f[f0 + i];
    s_n0m1[i] = sqrt(1. - f.l0 * f.l0 - f.m0 * f.m0) - 1.;
  }
  return n;
}

// ----------------------------------------------------------------------------------------
// Grid additions
// ----------------------------------------------------------------------------------------

// Adds v to a grid cell: into the facet's FP64 accumulator when it has one (two non-returning
// FP64 atomics; the float32 grid is untouched until the fold), else into the float32 cell.  The
// accumulator cell of grid cell c is found without the cell's index: with acc_off =
// addr(acc) - 2 addr(grid), addr(acc[c]) = 2 addr(grid[c]) + acc_off (16-byte cells for 8-byte
// ones; addresses are below 2^48, so the doubling cannot overflow).
__device__ __forceinline__ void grid_add(float2 *cell, bool acc, ptrdiff_t acc_off, float2 v) {
  if (acc) {
    double *d = (double *)(2 * (intptr_t)cell + acc_off);
    asm volatile("red.global.add.f64 [%0], %1;" ::"l"(d), "d"((double)v.x) : "memory");
    asm volatile("red.global.add.f64 [%0], %1;" ::"l"(d + 1), "d"((double)v.y) : "memory");
  } else {
    red_add(cell, v);
  }
}

__device__ __forceinline__ ptrdiff_t acc_offset(const ddfg_facet &f) {
  return f.grid_acc ? (ptrdiff_t)((intptr_t)f.grid_acc - 2 * (intptr_t)f.grid) : 0;
}

// Warp-cooperative tap scatter of the warp's 32 records onto facet f (gridder.h:353-362).
// As scatter_records (ddfg_taps.cuh), plus:
//  * run merging: consecutive records (lane order) with the same footprint origin and support
//    add their products into the lane's registers and reach the grid as one addition per tap
//    (consecutive channels of a row often fall on the same cell); the comparison is warp-uniform;
//  * FP64 accumulation when the facet has a grid_acc buffer (grid_add).
// MERGE = false drops the run merging (its accumulators cost registers that the averaged-block
// kernels, whose stripes rarely repeat a footprint, cannot spare).
// Must be called by all 32 lanes.
template <int NPOL, int SLOTS, bool MERGE = true>
__device__ __forceinline__ void scatter_q(const GridRecord<NPOL> &rec, const ddfg_facet &f, int npol_used,
                                          LaneTaps<SLOTS> &lt, int lane) {
  float2 *grid = (float2 *)f.grid;
  const bool comp = f.grid_acc != nullptr;
  const ptrdiff_t lo_off = acc_offset(f);
  const float2 *cfd = (const float2 *)f.cf_data;
  const int plane_sz = f.nx * f.ny;
  TapJob job;
  if (rec.valid) job = tap_job(rec.g, rec.gridchan, f);
  unsigned mask = __ballot_sync(0xffffffffu, rec.valid);
  if (!mask) return;
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
    if constexpr (!MERGE) {
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
                  if (NPOL == 1 || p < npol_used) grid_add(cell + (size_t)p * plane_sz, comp, lo_off, cmul(sv[r][p], c[r][k]));
              }
            }
          }
        }
      }
      return;
    }
    int run_base = -1;
    float2 acc[SLOTS][NPOL];
#pragma unroll
    for (int k = 0; k < SLOTS; ++k)
#pragma unroll
      for (int p = 0; p < NPOL; ++p) acc[k][p] = czero();
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
          if (base[r] != run_base) {  // warp-uniform: flush the previous run
            if (run_base >= 0) {
#pragma unroll
              for (int k = 0; k < SLOTS; ++k) {
                if (on[k]) {
                  float2 *cell = g_lane[k] + run_base;
#pragma unroll
                  for (int p = 0; p < NPOL; ++p)
                    if (NPOL == 1 || p < npol_used) grid_add(cell + (size_t)p * plane_sz, comp, lo_off, acc[k][p]);
                }
#pragma unroll
                for (int p = 0; p < NPOL; ++p) acc[k][p] = czero();
              }
            }
            run_base = base[r];
          }
#pragma unroll
          for (int k = 0; k < SLOTS; ++k)
#pragma unroll
            for (int p = 0; p < NPOL; ++p) acc[k][p] = cadd(acc[k][p], cmul(sv[r][p], c[r][k]));
        }
      }
    }
#pragma unroll
    for (int k = 0; k < SLOTS; ++k) {
      if (on[k]) {
        float2 *cell = g_lane[k] + run_base;
#pragma unroll
        for (int p = 0; p < NPOL; ++p)
          if (NPOL == 1 || p < npol_used) grid_add(cell + (size_t)p * plane_sz, comp, lo_off, acc[k][p]);
      }
    }
    return;
  }
  // Records of different supports (several W planes in one stripe): up to four records of equal
  // support at a time, so their CF loads overlap; otherwise one at a time.
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
              if (p < npol_used) grid_add(cell + (size_t)p * plane_sz, comp, lo_off, cmul(sv[r][p], c[r][k]));
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
            if (p < npol_used) grid_add(cell + (size_t)p * plane_sz, comp, lo_off, cmul(sv[r][p], cv));
        }
      }
    }
  }
}

// ----------------------------------------------------------------------------------------
// Warp-private grid tiles
// ----------------------------------------------------------------------------------------
// A stripe's 32 records usually lie close together on the grid (a row's consecutive channels move
// the footprint by a fraction of a cell each), so their S x S footprints overlap heavily.  The warp
// first sums the stripe's taps into its own shared-memory tile covering the footprints' bounding
// box -- plain loads and stores, no atomics: within one record every lane owns different cells,
// and a __syncwarp orders one record's updates before the next's -- and then adds every touched
// tile cell to the grid once.  The grid sees one addition per touched cell instead of one per tap
// (S^2 per record).
// Pitch 39 = 7 (mod 16): with 8-byte cells a 128-byte shared-memory wavefront holds 16 cells, and
// the rows of a 7 x 7 footprint (lanes 0-6 row 0, 7-13 row 1, ...) then fall on distinct banks.
constexpr int kTileW = 32, kTileH = 32, kTilePitch = 39;
constexpr int kTileCells = kTileH * kTilePitch;

// Lays the warp's records onto facet f through the warp's tile; returns false (having done
// nothing) when the records do not qualify -- different supports or bands, or a bounding box
// larger than the tile -- and the caller scatters them directly (scatter_q).  Single Stokes
// plane.  Must be called by all 32 lanes.
template <int SLOTS>
__device__ __forceinline__ bool scatter_tile(const GridRecord<1> &rec, const ddfg_facet &f, LaneTaps<SLOTS> &ltt,
                                             int lane, float2 *tile) {
  const unsigned mask0 = __ballot_sync(0xffffffffu, rec.valid);
  if (!mask0) return true;
  const int first = __ffs(mask0) - 1;
  const int S0 = __shfl_sync(0xffffffffu, rec.valid ? rec.g.S : 0, first);
  const int g0 = __shfl_sync(0xffffffffu, rec.valid ? rec.gridchan : 0, first);
  if (S0 * S0 > 32 * SLOTS || !__all_sync(0xffffffffu, !rec.valid || (rec.g.S == S0 && rec.gridchan == g0)))
    return false;
  const int sup = (S0 - 1) / 2;
  const int x0 = __reduce_min_sync(0xffffffffu, rec.valid ? rec.g.locx - sup : 0x7fffffff);
  const int y0 = __reduce_min_sync(0xffffffffu, rec.valid ? rec.g.locy - sup : 0x7fffffff);
  const int x1 = __reduce_max_sync(0xffffffffu, rec.valid ? rec.g.locx - sup : -1);
  const int y1 = __reduce_max_sync(0xffffffffu, rec.valid ? rec.g.locy - sup : -1);
  const int bw = x1 - x0 + S0, bh = y1 - y0 + S0;
  if (bw > kTileW || bh > kTileH) return false;
  // the bbox's cells lane-strided over all 32 lanes: cell i is row i / bw, column i % bw
  const int ncell = bw * bh;
  const unsigned inv_bw = (65536u + (unsigned)bw - 1u) / (unsigned)bw;  // i / bw == (i * inv_bw) >> 16, i < 1024
  for (int i = lane; i < ncell; i += 32) {
    const int r = (int)(((unsigned)i * inv_bw) >> 16);
    tile[r * kTilePitch + (i - r * bw)] = czero();
  }
  const int s_inv0 = S0 | (int)(((65536u + (unsigned)S0 - 1u) / (unsigned)S0) << 8);
  ltt.set(s_inv0, kTilePitch, lane);
  const float2 *cf_lane = (const float2 *)f.cf_data + lane;
  bool on[SLOTS];
#pragma unroll
  for (int k = 0; k < SLOTS; ++k) on[k] = ltt.off[k] >= 0;
  const int tb = rec.valid ? (rec.g.locy - sup - y0) * kTilePitch + (rec.g.locx - sup - x0) : 0;
  const int cfo_own = rec.valid ? rec.g.cfoff : 0;
  unsigned mask = mask0;
  __syncwarp();
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
    int tbase[4], cfo[4];
    float2 sv[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      tbase[r] = __shfl_sync(0xffffffffu, tb, src[r]);
      cfo[r] = __shfl_sync(0xffffffffu, cfo_own, src[r]);
      sv[r].x = __shfl_sync(0xffffffffu, rec.stokes[0].x, src[r]);
      sv[r].y = __shfl_sync(0xffffffffu, rec.stokes[0].y, src[r]);
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
            float2 *t = tile + tbase[r] + ltt.off[k];
            *t = cadd(*t, cmul(sv[r], c[r][k]));
          }
        }
        __syncwarp();
      }
    }
  }
  // one grid addition per touched tile cell (cells no tap reached hold an exact zero)
  float2 *gbase = (float2 *)f.grid + ((size_t)(g0 * f.npol) * f.ny + y0) * f.nx + x0;
  const bool comp = f.grid_acc != nullptr;
  const ptrdiff_t acc_off = acc_offset(f);
  for (int i = lane; i < ncell; i += 32) {
    const int r = (int)(((unsigned)i * inv_bw) >> 16), c = i - r * bw;
    const float2 v = tile[r * kTilePitch + c];
    if (v.x != 0.f || v.y != 0.f) grid_add(gbase + (size_t)r * f.nx + c, comp, acc_off, v);
  }
  __syncwarp();
  return true;
}

}  // namespace ddfg
