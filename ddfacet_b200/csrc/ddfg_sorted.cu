// Cell-sorted gridding and degridding (the batched path).
//
// Plan (once per visibility set): every BDA block gets a facet-independent key
//   (grid band, support of its W plane, grid row, grid column)
// of its mean position on a reference facet grid, and the blocks are sorted by it with a
// stable radix sort.  Neighbouring blocks in that order sit on the same or adjacent cells of
// every facet (the facets' uvw shifts w*Cu, w*Cv change slowly with w).
//
// Gridding: each warp takes chunks of consecutive sorted blocks.  Lane j walks block j
// exactly like the reference's hot loop 1 (gridder.h:182-351).  The warp then lays the
// blocks' taps with lanes over the S*S footprint, but keeps the tap sums in registers for as
// long as consecutive blocks share cell, support and band, and adds them to the facet grid with
// vector atomics only when that run ends.  This is Romein's work distribution for convolutional
// gridding moved to the warp level; with hundreds of blocks per cell, global read-modify-writes
// fall from one per tap (gridder.h:360-362) to one per run.  With compensation on, each register
// sum carries a TwoSum error term.
//
// Degridding: the warp keeps the footprint's model-grid values in registers while consecutive
// blocks share cell and support, multiplies them by each block's CF taps and reduces over lanes
// (degridder.h:202-212); lane j then applies block j's corrections and subtracts
// (degridder.h:214-264).  Every block belongs to one chunk, so visibilities are updated without
// atomics and the result is deterministic.
#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include <climits>

#include "ddfg_common.cuh"
#include "ddfg_degridblock.cuh"
#include "ddfg_gridblock.cuh"
#include "ddfg_internal.h"

namespace ddfg {

// ------------------------------------------------------------------------------------------
// plan keys
// ------------------------------------------------------------------------------------------
__global__ void sort_key_kernel(const ddfg_vis vs, const ddfg_facet f, uint64_t *keys, int64_t *vals,
                                unsigned long long *nvalid) {
  unsigned long long cnt = 0;
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < vs.nblocks;
       b += (int64_t)gridDim.x * blockDim.x) {
    vals[b] = b;
    DegridBlock d;
    degrid_block_header(vs, b, d);
    uint64_t key = ~0ull;
    if (d.ch1 > d.ch0 && d.nrows > 0 && d.gridchan >= 0 && d.gridchan < f.nband) {
      double um = 0., vm = 0., wm = 0.;
      for (int i = 0; i < d.nrows; ++i) {
        const double *up = vs.uvw + 3 * (int64_t)d.rows[i];
        um += up[0];
        vm += up[1];
        wm += up[2];
      }
      um /= d.nrows;
      vm /= d.nrows;
      wm /= d.nrows;
      const double rw = d.freqmean / kC;
      const double x = (double)f.nx * f.incr_x * um * rw + (double)(f.nx / 2);
      const double y = (double)f.nx * f.incr_y * vm * rw + (double)(f.ny / 2);
      long long cx = llrint(x), cy = llrint(y);
      cx = min(max(cx, 0LL), (1LL << 21) - 1);
      cy = min(max(cy, 0LL), (1LL << 21) - 1);
      long long iw = llrint(((double)f.nw - 1.0) * fabs(wm) * (f.ref_wave * rw) / f.wmax);
      iw = min(max(iw, 0LL), (long long)f.nw - 1);
      const int S = f.cf_support[wm > 0. ? (int)iw : f.nw + (int)iw];
      key = ((uint64_t)d.gridchan << 48) | ((uint64_t)(S & 63) << 42) | ((uint64_t)cy << 21) | (uint64_t)cx;
      ++cnt;
    }
    keys[b] = key;
  }
  if (cnt) atomicAdd(nvalid, cnt);
}

// ------------------------------------------------------------------------------------------
// shared helpers
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ float2 shfl2(float2 v, int src) {
  return make_float2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

// ------------------------------------------------------------------------------------------
// gridding
// ------------------------------------------------------------------------------------------
template <int NPOL, int SLOTS, bool COMP>
struct TapAcc {
  float2 hi[SLOTS][NPOL];
  float2 lo[COMP ? SLOTS : 1][NPOL];
};

template <int NPOL, int SLOTS, bool COMP>
__device__ __forceinline__ void acc_zero(TapAcc<NPOL, SLOTS, COMP> &a) {
#pragma unroll
  for (int k = 0; k < SLOTS; ++k)
#pragma unroll
    for (int p = 0; p < NPOL; ++p) {
      a.hi[k][p] = czero();
      if (COMP) a.lo[k][p] = czero();
    }
}

__device__ __forceinline__ void two_sum_acc(float &s, float &e, float x) {
  const float t = s + x;
  const float bb = t - s;
  e += (s - (t - bb)) + (x - bb);
  s = t;
}

template <int NPOL, int SLOTS, bool COMP>
__device__ __forceinline__ void acc_flush(TapAcc<NPOL, SLOTS, COMP> &a, float2 *grid, size_t plane_sz, int nx,
                                          int lx, int ly, int S, unsigned inv, int npol_used, int lane) {
  const int sup = (S - 1) >> 1;
  float2 *g0 = grid + (size_t)(ly - sup) * nx + (lx - sup);
#pragma unroll
  for (int k = 0; k < SLOTS; ++k) {
    const int t = lane + 32 * k;
    if (t < S * S) {
      const int sy = (int)(((unsigned)t * inv) >> 16);
      const int sx = t - sy * S;
      float2 *cell = g0 + (size_t)sy * nx + sx;
#pragma unroll
      for (int p = 0; p < NPOL; ++p) {
        if (p < npol_used) {
          float2 v = a.hi[k][p];
          if (COMP) {
            v.x += a.lo[k][p].x;
            v.y += a.lo[k][p].y;
          }
          if (v.x != 0.f || v.y != 0.f) red_add(cell + (size_t)p * plane_sz, v);
        }
      }
    }
  }
}

template <int NPOL, int SLOTS, bool COMP>
__global__ void __launch_bounds__(256) grid_sorted_kernel(const ddfg_vis vs, const ddfg_jones js, const FacetPack pack,
                                                          const GridParams gp, const int64_t *__restrict__ perm,
                                                          int64_t nplanned, int chunk) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ddfg_facet *sf = (ddfg_facet *)smem_raw;
  double *acc = (double *)(sf + pack.n);
  stage_facets(pack, sf);
  const int fstride = pack.f[0].nband * pack.f[0].npol + 2 * pack.f[0].nband + 2 * vs.nchan;
  for (int i = threadIdx.x; i < pack.n * fstride; i += blockDim.x) acc[i] = 0.;
  __syncthreads();

  const int lane = threadIdx.x & 31;
  const int wpc = blockDim.x >> 5;
  const int64_t gw = (int64_t)blockIdx.x * wpc + (threadIdx.x >> 5);
  const int64_t nwarps = (int64_t)gridDim.x * wpc;
  const int64_t nchunks = (nplanned + chunk - 1) / chunk;
  JonesCache jc;

  for (int64_t c = gw; c < nchunks; c += nwarps) {
    const int64_t r0 = c * chunk;
    const int64_t r1 = min(r0 + chunk, nplanned);
    for (int fi = 0; fi < pack.n; ++fi) {
      const ddfg_facet &f = sf[fi];
      const double n0m1 = sqrt(1. - f.l0 * f.l0 - f.m0 * f.m0) - 1.;
      const int npol_used = min(gp.nvispol, f.npol);
      const size_t plane_sz = (size_t)f.nx * f.ny;
      double *a_sumwt = acc + fi * fstride;
      double *a_sumj = a_sumwt + f.nband * f.npol;
      double *a_chan = a_sumj + 2 * f.nband;
      TapAcc<NPOL, SLOTS, COMP> ta;
      acc_zero(ta);
      int cur_lx = INT_MIN, cur_ly = 0, cur_S = 0, cur_g = 0;
      unsigned cur_inv = 0;

      for (int64_t base = r0; base < r1; base += 32) {
        GridRecord<NPOL> rec;
        rec.valid = false;
        int64_t b = -1;
        if (base + lane < r1) {
          b = perm[base + lane];
          grid_block_record<NPOL>(vs, js, f, gp, b, n0m1, rec, jc);
        }
        warp_add_block_sums<NPOL>(vs, js, f, gp, b, rec, npol_used, a_sumwt, a_sumj, a_chan, jc);
        const unsigned vmask = __ballot_sync(0xffffffffu, rec.valid);
        // Tap accumulation, run by run.
        unsigned mask = vmask;
        while (mask) {
          const int src = __ffs(mask) - 1;
          mask &= mask - 1;
          const int lx = __shfl_sync(0xffffffffu, rec.g.locx, src);
          const int ly = __shfl_sync(0xffffffffu, rec.g.locy, src);
          const int S = __shfl_sync(0xffffffffu, rec.g.S, src);
          const unsigned inv = __shfl_sync(0xffffffffu, rec.g.inv, src);
          const int gch = __shfl_sync(0xffffffffu, rec.gridchan, src);
          const float2 *cf = (const float2 *)__shfl_sync(0xffffffffu, (unsigned long long)rec.g.cf, src);
          float2 sv[NPOL];
#pragma unroll
          for (int p = 0; p < NPOL; ++p) sv[p] = shfl2(rec.stokes[p], src);
          if (lx != cur_lx || ly != cur_ly || S != cur_S || gch != cur_g) {
            if (cur_lx != INT_MIN)
              acc_flush(ta, (float2 *)f.grid + (size_t)cur_g * f.npol * plane_sz, plane_sz, f.nx, cur_lx, cur_ly,
                        cur_S, cur_inv, npol_used, lane);
            acc_zero(ta);
            cur_lx = lx;
            cur_ly = ly;
            cur_S = S;
            cur_inv = inv;
            cur_g = gch;
          }
          if (S * S <= 32 * SLOTS) {
#pragma unroll
            for (int k = 0; k < SLOTS; ++k) {
              const int t = lane + 32 * k;
              if (t < S * S) {
                const float2 cv = __ldg(cf + t);
#pragma unroll
                for (int p = 0; p < NPOL; ++p) {
                  const float2 v = cmul(sv[p], cv);
                  if (COMP) {
                    two_sum_acc(ta.hi[k][p].x, ta.lo[k][p].x, v.x);
                    two_sum_acc(ta.hi[k][p].y, ta.lo[k][p].y, v.y);
                  } else {
                    ta.hi[k][p].x += v.x;
                    ta.hi[k][p].y += v.y;
                  }
                }
              }
            }
          } else {
            // Support larger than the register footprint: taps go straight to the grid.
            const int sup = (S - 1) >> 1;
            float2 *g0 = (float2 *)f.grid + (size_t)gch * f.npol * plane_sz + (size_t)(ly - sup) * f.nx + (lx - sup);
            for (int t = lane; t < S * S; t += 32) {
              const int sy = (int)(((unsigned)t * inv) >> 16);
              const int sx = t - sy * S;
              const float2 cv = __ldg(cf + t);
#pragma unroll
              for (int p = 0; p < NPOL; ++p)
                if (p < npol_used) atomicAdd(g0 + (size_t)p * plane_sz + (size_t)sy * f.nx + sx, cmul(sv[p], cv));
            }
          }
        }
      }
      if (cur_lx != INT_MIN && cur_S * cur_S <= 32 * SLOTS)
        acc_flush(ta, (float2 *)f.grid + (size_t)cur_g * f.npol * plane_sz, plane_sz, f.nx, cur_lx, cur_ly, cur_S,
                  cur_inv, npol_used, lane);
    }
  }
  __syncthreads();
  for (int fi = 0; fi < pack.n; ++fi) {
    const ddfg_facet &f = sf[fi];
    const double *a = acc + fi * fstride;
    const int nsw = f.nband * f.npol;
    for (int i = threadIdx.x; i < nsw; i += blockDim.x)
      if (f.sumwt && a[i] != 0.) atomicAdd(&f.sumwt[i], a[i]);
    if (js.mode != 0) {
      for (int i = threadIdx.x; i < 2 * f.nband; i += blockDim.x)
        if (f.sumjones && a[nsw + i] != 0.) atomicAdd(&f.sumjones[i], a[nsw + i]);
      for (int i = threadIdx.x; i < 2 * vs.nchan; i += blockDim.x)
        if (f.sumjones_chan && a[nsw + 2 * f.nband + i] != 0.) atomicAdd(&f.sumjones_chan[i], a[nsw + 2 * f.nband + i]);
    }
  }
}

// ------------------------------------------------------------------------------------------
// degridding
// ------------------------------------------------------------------------------------------
template <int NPOL, int SLOTS>
__global__ void __launch_bounds__(256, 1) degrid_sorted_kernel(const ddfg_vis vs, const ddfg_jones js,
                                                            const FacetPackD pack, const DegridParams dp,
                                                            const int64_t *__restrict__ perm, int64_t nplanned,
                                                            int chunk) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ddfg_facet *sf = (ddfg_facet *)smem_raw;
  stage_facets(pack, sf);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int wpc = blockDim.x >> 5;
  const int64_t gw = (int64_t)blockIdx.x * wpc + (threadIdx.x >> 5);
  const int64_t nwarps = (int64_t)gridDim.x * wpc;
  const int64_t nchunks = (nplanned + chunk - 1) / chunk;

  for (int64_t c = gw; c < nchunks; c += nwarps) {
    const int64_t r0 = c * chunk;
    const int64_t r1 = min(r0 + chunk, nplanned);
    for (int fi = 0; fi < pack.n; ++fi) {
      const ddfg_facet &f = sf[fi];
      const size_t plane_sz = (size_t)f.nx * f.ny;
      float2 gv[SLOTS][NPOL];
      int cur_lx = INT_MIN, cur_ly = 0, cur_S = 0, cur_g = 0;
      for (int64_t base = r0; base < r1; base += 32) {
        DegridBlock d;
        BlockGeom g;
        bool valid = false;
        if (base + lane < r1) {
          degrid_block_header(vs, perm[base + lane], d);
          valid = degrid_block_geom(vs, f, d, g);
        }
        float2 mine[NPOL];
#pragma unroll
        for (int p = 0; p < NPOL; ++p) mine[p] = czero();
        unsigned mask = __ballot_sync(0xffffffffu, valid);
        while (mask) {
          const int src = __ffs(mask) - 1;
          mask &= mask - 1;
          const int lx = __shfl_sync(0xffffffffu, g.locx, src);
          const int ly = __shfl_sync(0xffffffffu, g.locy, src);
          const int S = __shfl_sync(0xffffffffu, g.S, src);
          const unsigned inv = __shfl_sync(0xffffffffu, g.inv, src);
          const int gch = __shfl_sync(0xffffffffu, d.gridchan, src);
          const float2 *cf = (const float2 *)__shfl_sync(0xffffffffu, (unsigned long long)g.cf, src);
          const int sup = (S - 1) >> 1;
          const float2 *g0 = (const float2 *)f.grid + (size_t)gch * f.npol * plane_sz + (size_t)(ly - sup) * f.nx +
                             (lx - sup);
          float2 a[NPOL];
#pragma unroll
          for (int p = 0; p < NPOL; ++p) a[p] = czero();
          if (S * S <= 32 * SLOTS) {
            if (lx != cur_lx || ly != cur_ly || S != cur_S || gch != cur_g) {
#pragma unroll
              for (int k = 0; k < SLOTS; ++k) {
                const int t = lane + 32 * k;
                const int sy = (int)(((unsigned)t * inv) >> 16);
                const int sx = t - sy * S;
#pragma unroll
                for (int p = 0; p < NPOL; ++p)
                  gv[k][p] = (t < S * S) ? __ldg(g0 + (size_t)p * plane_sz + (size_t)sy * f.nx + sx) : czero();
              }
              cur_lx = lx;
              cur_ly = ly;
              cur_S = S;
              cur_g = gch;
            }
#pragma unroll
            for (int k = 0; k < SLOTS; ++k) {
              const int t = lane + 32 * k;
              if (t < S * S) {
                const float2 cv = __ldg(cf + t);
#pragma unroll
                for (int p = 0; p < NPOL; ++p) a[p] = cadd(a[p], cmul(gv[k][p], cv));
              }
            }
          } else {
            for (int t = lane; t < S * S; t += 32) {
              const int sy = (int)(((unsigned)t * inv) >> 16);
              const int sx = t - sy * S;
              const float2 cv = __ldg(cf + t);
#pragma unroll
              for (int p = 0; p < NPOL; ++p)
                a[p] = cadd(a[p], cmul(__ldg(g0 + (size_t)p * plane_sz + (size_t)sy * f.nx + sx), cv));
            }
          }
#pragma unroll
          for (int p = 0; p < NPOL; ++p) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
              a[p].x += __shfl_xor_sync(0xffffffffu, a[p].x, o);
              a[p].y += __shfl_xor_sync(0xffffffffu, a[p].y, o);
            }
          }
          if (lane == src) {
#pragma unroll
            for (int p = 0; p < NPOL; ++p) mine[p] = a[p];
          }
        }
        if (valid) degrid_block_apply<NPOL>(vs, js, f, dp, d, mine);
      }
    }
  }
}

}  // namespace ddfg

using namespace ddfg;

// ------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------
namespace {
size_t sort_temp_bytes(int64_t n) {
  size_t bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const uint64_t *)nullptr, (uint64_t *)nullptr,
                                  (const int64_t *)nullptr, (int64_t *)nullptr, (int)(n > 0 ? n : 1));
  return bytes;
}
size_t al(size_t x) { return (x + 255) / 256 * 256; }
size_t nz(int64_t n) { return (size_t)(n > 0 ? n : 1); }
}  // namespace

extern "C" size_t ddfg_sort_plan_workspace_size(int64_t nblocks) {
  return al(sort_temp_bytes(nblocks)) + 2 * al(8 * nz(nblocks)) + al(8 * nz(nblocks)) + 256;
}

extern "C" int ddfg_sort_plan_build(const ddfg_vis *vs, const ddfg_facet *ref, ddfg_sort_plan *plan, void *workspace,
                                    size_t workspace_bytes, void *stream_) {
  cudaStream_t stream = (cudaStream_t)stream_;
  if (!vs || !ref || !plan || !plan->perm || !workspace) return ddfg_set_error(DDFG_EINVAL, "sort_plan: null argument");
  if (vs->nblocks > 0x7FFFFFFF) return ddfg_set_error(DDFG_ESIZE, "sort_plan: more than 2^31-1 blocks");
  if (!ref->cf_support || ref->nw <= 0 || ref->nx <= 0 || ref->ny <= 0 || ref->nband <= 0)
    return ddfg_set_error(DDFG_EINVAL, "sort_plan: bad reference facet");
  if (ref->nband >= (1 << 15)) return ddfg_set_error(DDFG_ESIZE, "sort_plan: too many bands");
  const size_t need = ddfg_sort_plan_workspace_size(vs->nblocks);
  if (workspace_bytes < need) return ddfg_set_error(DDFG_ESIZE, "sort_plan: workspace %zu < %zu", workspace_bytes, need);
  const int64_t nb = vs->nblocks;
  char *w = (char *)workspace;
  const size_t tb = al(sort_temp_bytes(nb));
  uint64_t *kin = (uint64_t *)(w + tb);
  uint64_t *kout = (uint64_t *)(w + tb + al(8 * nz(nb)));
  int64_t *vin = (int64_t *)(w + tb + 2 * al(8 * nz(nb)));
  unsigned long long *nvalid = (unsigned long long *)(w + tb + 3 * al(8 * nz(nb)));
  cudaError_t e = cudaMemsetAsync(nvalid, 0, sizeof(unsigned long long), stream);
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "sort_plan: %s", cudaGetErrorString(e));
  if (nb > 0) {
    sort_key_kernel<<<ddfg_num_ctas(8), 256, 0, stream>>>(*vs, *ref, kin, vin, nvalid);
    size_t tmpb = tb;
    e = cub::DeviceRadixSort::SortPairs(w, tmpb, kin, kout, vin, plan->perm, (int)nb, 0, 64, stream);
    if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "sort_plan sort: %s", cudaGetErrorString(e));
  }
  unsigned long long hv = 0;
  e = cudaMemcpyAsync(&hv, nvalid, sizeof(hv), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "sort_plan: %s", cudaGetErrorString(e));
  plan->nplanned = (int64_t)hv;
  plan->gref = ref->nx;
  if (plan->chunk <= 0) plan->chunk = 1024;
  return DDFG_OK;
}

namespace {
int slots_for(int max_support) {
  const int t = max_support * max_support;
  if (t <= 64) return 2;
  if (t <= 128) return 4;
  return 8;
}
}  // namespace

int ddfg_launch_grid_sorted(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_facet *facets, int nfacets, int policy,
                            int nvispol, int dopsf, const ddfg_sort_plan *plan, int compensated, int max_support,
                            int facets_per_launch, cudaStream_t stream) {
  GridParams gp;
  gp.policy = policy;
  gp.nvispol = nvispol;
  gp.dopsf = dopsf;
  gp.freq_mean0 = vs->freq_mean;
  if (plan->nplanned == 0) return DDFG_OK;
  const int per = facets_per_launch > 0 ? min(facets_per_launch, DDFG_FACETS_PER_LAUNCH) : DDFG_FACETS_PER_LAUNCH;
  const int slots = slots_for(max_support);
  const int chunk = plan->chunk > 0 ? plan->chunk : 1024;
  for (int f0 = 0; f0 < nfacets; f0 += per) {
    FacetPack pack;
    pack.n = min(per, nfacets - f0);
    for (int i = 0; i < pack.n; ++i) pack.f[i] = facets[f0 + i];
    for (int i = 0; i < pack.n; ++i)
      if (pack.f[i].nband != pack.f[0].nband || pack.f[i].npol != pack.f[0].npol)
        return ddfg_set_error(DDFG_EINVAL, "grid_sorted: facets of one call must share nband and npol");
    const int fstride = pack.f[0].nband * pack.f[0].npol + 2 * pack.f[0].nband + 2 * vs->nchan;
    const size_t smem = sizeof(ddfg_facet) * pack.n + sizeof(double) * (size_t)pack.n * fstride + 16;
    if (smem > 200 * 1024) return ddfg_set_error(DDFG_ESIZE, "grid_sorted: %zu bytes of shared accumulators", smem);
    const int nctas = ddfg_num_ctas(2);
#define LAUNCH_GS(NP, SL, CP)                                                                                    \
  do {                                                                                                           \
    if (smem > 48 * 1024)                                                                                        \
      cudaFuncSetAttribute(grid_sorted_kernel<NP, SL, CP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
    grid_sorted_kernel<NP, SL, CP><<<nctas, 256, smem, stream>>>(*vs, *js, pack, gp, plan->perm, plan->nplanned, \
                                                                 chunk);                                         \
  } while (0)
#define LAUNCH_GS_NP(SL, CP)        \
  switch (nvispol) {                \
    case 1: LAUNCH_GS(1, SL, CP); break; \
    case 2: LAUNCH_GS(2, SL, CP); break; \
    case 3: LAUNCH_GS(3, SL, CP); break; \
    default: LAUNCH_GS(4, SL, CP); break; \
  }
    if (compensated) {
      if (slots == 2) { LAUNCH_GS_NP(2, true) } else if (slots == 4) { LAUNCH_GS_NP(4, true) } else { LAUNCH_GS_NP(8, true) }
    } else {
      if (slots == 2) { LAUNCH_GS_NP(2, false) } else if (slots == 4) { LAUNCH_GS_NP(4, false) } else { LAUNCH_GS_NP(8, false) }
    }
#undef LAUNCH_GS_NP
#undef LAUNCH_GS
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "grid_sorted launch: %s", cudaGetErrorString(e));
  }
  return DDFG_OK;
}

int ddfg_launch_degrid_sorted(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_facet *facets, int nfacets,
                              int policy, int nvispol, const ddfg_sort_plan *plan, int max_support,
                              int facets_per_launch, cudaStream_t stream) {
  DegridParams dp;
  dp.policy = policy;
  dp.nvispol = nvispol;
  if (plan->nplanned == 0) return DDFG_OK;
  const int per = facets_per_launch > 0 ? min(facets_per_launch, DDFG_FACETS_PER_LAUNCH) : DDFG_FACETS_PER_LAUNCH;
  const int slots = slots_for(max_support);
  const int chunk = plan->chunk > 0 ? plan->chunk : 1024;
  const int nctas = ddfg_num_ctas(2);
  for (int f0 = 0; f0 < nfacets; f0 += per) {
    FacetPackD pack;
    pack.n = min(per, nfacets - f0);
    for (int i = 0; i < pack.n; ++i) pack.f[i] = facets[f0 + i];
    const size_t smem = sizeof(ddfg_facet) * pack.n + 16;
#define LAUNCH_DS(NP, SL)                                                                                     \
  degrid_sorted_kernel<NP, SL><<<nctas, 256, smem, stream>>>(*vs, *js, pack, dp, plan->perm, plan->nplanned, chunk)
#define LAUNCH_DS_NP(SL)             \
  switch (nvispol) {                 \
    case 1: LAUNCH_DS(1, SL); break; \
    case 2: LAUNCH_DS(2, SL); break; \
    case 3: LAUNCH_DS(3, SL); break; \
    default: LAUNCH_DS(4, SL); break; \
  }
    if (slots == 2) { LAUNCH_DS_NP(2) } else if (slots == 4) { LAUNCH_DS_NP(4) } else { LAUNCH_DS_NP(8) }
#undef LAUNCH_DS_NP
#undef LAUNCH_DS
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "degrid_sorted launch: %s", cudaGetErrorString(e));
  }
  return DDFG_OK;
}
