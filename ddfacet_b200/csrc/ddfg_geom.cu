// Check entry points: the integer footprint of every block as the kernels compute it, and the
// validation of a large-block list.
#include <cuda_runtime.h>

#include "ddfg_common.cuh"
#include "ddfg_degridblock.cuh"
#include "ddfg_gridblock.cuh"
#include "ddfg_internal.h"

using namespace ddfg;

namespace {

// out[b] = {status, iw, plane, locx, locy, offx, offy, k}: the gridder's block means
// (grid_block_means: unflagged visibilities, gridder.h:272-289) or the degridder's (row means and
// channel-mean frequency, degridder.h:138-167), then block_geometry with its intermediate values.
__global__ void block_geometry_kernel(const ddfg_vis vs, const ddfg_facet f, int degrid_means, int32_t *out) {
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < vs.nblocks;
       b += (int64_t)gridDim.x * blockDim.x) {
    int dbg[7] = {-1, -1, -1, -1, -1, -1, -1};
    bool ok = false;
    BlockGeom g;
    if (degrid_means) {
      DegridBlock d;
      degrid_block_header(vs, b, d);
      ok = degrid_block_geom(vs, f, d, g, dbg);
    } else {
      const BlockMeans m = grid_block_means(vs, f, b);
      const int64_t start = vs.block_start[b];
      const int gridchan = vs.chan_map[vs.bda_map[start]];
      if (m.nvis > 0 && gridchan >= 0 && gridchan < f.nband) {
        double um = m.u, vm = m.v, wm = m.w, fm = m.nu;
        if (m.nvis > 1) {
          const double dn = (double)m.nvis;
          um = um / dn;
          vm = vm / dn;
          wm = wm / dn;
          fm = fm / dn;
        }
        const double rw = (m.nvis == 1 && vs.recip_wvl) ? vs.recip_wvl[m.last_ch] : fm / kC;
        ok = block_geometry(f, um, vm, wm, rw, g, dbg);
      }
    }
    int32_t *o = out + 8 * b;
    o[0] = ok ? 1 : 0;
#pragma unroll
    for (int i = 0; i < 7; ++i) o[1 + i] = dbg[i];
  }
}

__global__ void large_mark_kernel(const ddfg_vis vs, unsigned int *bits, unsigned int *err) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < vs.nlarge;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t bl = vs.large_blocks[t];
    if (bl < 0 || bl >= vs.nblocks) {
      atomicOr(err, 1u);
      continue;
    }
    const unsigned int bit = 1u << (unsigned)(bl & 31);
    if (atomicOr(&bits[bl >> 5], bit) & bit) atomicOr(err, 2u);
    if (block_nvis(vs, bl) <= vs.large_min_vis) atomicOr(err, 4u);
  }
}

__global__ void large_check_kernel(const ddfg_vis vs, const unsigned int *bits, unsigned int *err) {
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < vs.nblocks;
       b += (int64_t)gridDim.x * blockDim.x) {
    const bool listed = (bits[b >> 5] >> (unsigned)(b & 31)) & 1u;
    if (!listed && block_nvis(vs, b) > vs.large_min_vis) atomicOr(err, 8u);
  }
}

// Jones time slot of every row: the last slot [t0, t1) that contains the row's time, 0 if none
// (ClassJones.GiveTimeMapping, ClassJones.py:415-439).
__global__ void jones_time_map_kernel(const double *times, int64_t nrow, const double *t0, const double *t1, int nt,
                                      int32_t *out) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nrow; r += (int64_t)gridDim.x * blockDim.x) {
    const double t = times[r];
    int v = 0;
    for (int it = 0; it < nt; ++it)
      if (t >= t0[it] && t < t1[it]) v = it;
    out[r] = v;
  }
}

}  // namespace

extern "C" int ddfg_jones_time_map(const double *times, int64_t nrow, const double *t0, const double *t1, int32_t nt,
                                   int32_t *out, void *stream) {
  if (nrow < 0 || nt < 0 || (nrow > 0 && (!times || !out)) || (nt > 0 && (!t0 || !t1)))
    return ddfg_set_error(DDFG_EINVAL, "jones_time_map: null pointer or negative size");
  if (nrow == 0) return DDFG_OK;
  jones_time_map_kernel<<<ddfg_num_ctas(4), 256, 0, (cudaStream_t)stream>>>(times, nrow, t0, t1, nt, out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "jones_time_map: %s", cudaGetErrorString(e));
  return DDFG_OK;
}

extern "C" int ddfg_block_geometry(const ddfg_vis *vs, const ddfg_facet *facet, int degrid_means, int32_t *out,
                                   void *stream) {
  if (!vs || !facet || (vs->nblocks > 0 && !out)) return ddfg_set_error(DDFG_EINVAL, "block_geometry: null argument");
  if (vs->nblocks == 0) return DDFG_OK;
  if (!vs->uvw || !vs->freqs || !vs->chan_map || !vs->bda_map || !vs->block_start || !vs->flags)
    return ddfg_set_error(DDFG_EINVAL, "block_geometry: null visibility-set pointer");
  if (!facet->cf_support || facet->nw <= 0 || facet->overs <= 0 || facet->wmax == 0.)
    return ddfg_set_error(DDFG_EINVAL, "block_geometry: bad facet");
  block_geometry_kernel<<<ddfg_num_ctas(4), 256, 0, (cudaStream_t)stream>>>(*vs, *facet, degrid_means, out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "block_geometry: %s", cudaGetErrorString(e));
  return DDFG_OK;
}

extern "C" size_t ddfg_check_large_blocks_workspace_size(int64_t nblocks) {
  return (size_t)((nblocks + 31) / 32) * sizeof(unsigned int) + 256;
}

extern "C" int ddfg_check_large_blocks(const ddfg_vis *vs, void *workspace, size_t workspace_bytes, void *stream_) {
  cudaStream_t stream = (cudaStream_t)stream_;
  if (!vs || !workspace) return ddfg_set_error(DDFG_EINVAL, "check_large_blocks: null argument");
  if (vs->nlarge == 0) return DDFG_OK;
  if (vs->nlarge < 0 || !vs->large_blocks || vs->large_min_vis < 1 || !vs->bda_map || !vs->block_start)
    return ddfg_set_error(DDFG_EINVAL, "check_large_blocks: bad large-block list");
  const size_t need = ddfg_check_large_blocks_workspace_size(vs->nblocks);
  if (workspace_bytes < need)
    return ddfg_set_error(DDFG_ESIZE, "check_large_blocks: workspace %zu < %zu bytes", workspace_bytes, need);
  unsigned int *bits = (unsigned int *)workspace;
  unsigned int *err = (unsigned int *)((char *)workspace + need - 256);
  cudaError_t e = cudaMemsetAsync(workspace, 0, need, stream);
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "check_large_blocks: %s", cudaGetErrorString(e));
  const int ctas = ddfg_num_ctas(4);
  large_mark_kernel<<<ctas, 256, 0, stream>>>(*vs, bits, err);
  large_check_kernel<<<ctas, 256, 0, stream>>>(*vs, bits, err);
  e = cudaGetLastError();
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "check_large_blocks: %s", cudaGetErrorString(e));
  unsigned int herr = 0;
  e = cudaMemcpyAsync(&herr, err, sizeof(herr), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "check_large_blocks: %s", cudaGetErrorString(e));
  if (herr & 1u) return ddfg_set_error(DDFG_EMAP, "check_large_blocks: an entry is not a block index");
  if (herr & 2u) return ddfg_set_error(DDFG_EMAP, "check_large_blocks: a block is listed twice");
  if (herr & 4u) return ddfg_set_error(DDFG_EMAP, "check_large_blocks: a listed block is not above large_min_vis");
  if (herr & 8u) return ddfg_set_error(DDFG_EMAP, "check_large_blocks: a block above large_min_vis is not listed");
  return DDFG_OK;
}
