// Imaging weights on the GPU: the uv-density grid behind uniform and Briggs weighting.
//
// Restates DDFacet's weight pipeline (DDFacet/Data/ClassVisServer.py, GridderSmearPols.cc):
//   index     -- _uv_to_index (ClassVisServer.py:981-1003): v < 0 flips (u, v); the uv cell is
//                floor(u nu / c / cell) + xymax, floor(v nu / c / cell) on a [npixx x npixy] half
//                plane, plus band * npix with per-band grids; zero weights point at cell 0.
//                FP64 uncontracted, so the indices are bit-exact.
//   accumulate-- pyAccumulateWeightsOntoGrid(NoSem) (GridderSmearPols.cc:32-74): grid[index] +=
//                weight (float64 atomics; the reference serialises with semaphores per cell).
//   robust    -- the Briggs step (ClassVisServer.py:897-904): per band g = 1 + g s^2 / avgW with
//                avgW = sum g^2 / sum g.
//   finalize  -- _finalizeWeights_handler (ClassVisServer.py:1036-1043): weight /= grid[index].
// All HBM-bound passes (a few bytes per visibility).
#include <cuda_runtime.h>

#include "ddfg_internal.h"

namespace {

constexpr double kC = 299792458.0;

__global__ void weights_index_kernel(const double *uvw, int64_t nrow, const double *freqs, int32_t nchan,
                                     const float *weights, const int32_t *band_of_chan, int32_t nbands, double cell,
                                     int64_t xymax, int64_t npixx, int64_t npix, int32_t *index) {
  const int64_t n = nrow * nchan;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / nchan;
    const int c = (int)(i - r * nchan);
    double u = uvw[3 * r], v = uvw[3 * r + 1];
    if (v < 0.) {
      u = -u;
      v = -v;
    }
    const double f = freqs[c];
    const double ul = __ddiv_rn(__dmul_rn(u, f), kC);
    const double vl = __ddiv_rn(__dmul_rn(v, f), kC);
    const int64_t x = (int64_t)floor(__ddiv_rn(ul, cell)) + xymax;
    const int64_t y = (int64_t)floor(__ddiv_rn(vl, cell));
    int64_t idx = y * npixx + x;
    if (nbands > 1) idx += (int64_t)band_of_chan[c] * npix;
    if (weights[i] == 0.f) idx = 0;
    index[i] = (int32_t)idx;
  }
}

__global__ void weights_accumulate_kernel(double *grid, int64_t grid_len, const float *weights,
                                          const int32_t *index, int64_t n, unsigned int *bad) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float w = weights[i];
    if (w == 0.f) continue;
    const int64_t k = index[i];
    if (k < 0 || k >= grid_len) {
      atomicOr(bad, 1u);
      continue;
    }
    atomicAdd(grid + k, (double)w);
  }
}

// sums[2 b] = sum g, sums[2 b + 1] = sum g^2 over band b.
__global__ void weights_sums_kernel(const double *grid, int64_t npix, int32_t nbands, double *sums) {
  for (int b = 0; b < nbands; ++b) {
    double s = 0., s2 = 0.;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += (int64_t)gridDim.x * blockDim.x) {
      const double g = grid[(int64_t)b * npix + i];
      s += g;
      s2 += g * g;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s += __shfl_xor_sync(0xffffffffu, s, o);
      s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(sums + 2 * b, s);
      atomicAdd(sums + 2 * b + 1, s2);
    }
  }
}

__global__ void weights_robust_kernel(double *grid, int64_t npix, int32_t nbands, const double *sums,
                                      double numerator_sqrt) {
  const int64_t n = npix * nbands;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = i / npix;
    const double avg_w = sums[2 * b + 1] / sums[2 * b];
    const double s_sq = numerator_sqrt * numerator_sqrt / avg_w;
    grid[i] = 1. + grid[i] * s_sq;
  }
}

__global__ void weights_finalize_kernel(float *weights, const int32_t *index, int64_t n, const double *grid,
                                        int64_t grid_len) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t k = index[i];
    if (k >= grid_len || k < 0) k = 0;
    weights[i] = (float)((double)weights[i] / grid[k]);
  }
}

int launch_check(const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "%s: %s", what, cudaGetErrorString(e));
  return DDFG_OK;
}

}  // namespace

extern "C" int ddfg_weights_uv_index(const double *uvw, int64_t nrow, const double *freqs, int32_t nchan,
                                     const float *weights, const int32_t *band_of_chan, int32_t nbands, double cell,
                                     int64_t xymax, int64_t npixx, int64_t npix, int32_t *index, void *stream) {
  if (nrow < 0 || nchan < 0 || nbands < 1 || !(cell > 0.))
    return ddfg_set_error(DDFG_EINVAL, "weights_uv_index: bad sizes or cell");
  if (nrow * (int64_t)nchan == 0) return DDFG_OK;
  if (!uvw || !freqs || !weights || !index || (nbands > 1 && !band_of_chan))
    return ddfg_set_error(DDFG_EINVAL, "weights_uv_index: null pointer");
  if ((int64_t)nbands * npix > INT32_MAX) return ddfg_set_error(DDFG_ESIZE, "weights_uv_index: grid exceeds int32 indices");
  weights_index_kernel<<<ddfg_num_ctas(8), 256, 0, (cudaStream_t)stream>>>(uvw, nrow, freqs, nchan, weights,
                                                                          band_of_chan, nbands, cell, xymax, npixx,
                                                                          npix, index);
  return launch_check("weights_uv_index");
}

extern "C" int ddfg_weights_accumulate(double *grid, int64_t grid_len, const float *weights, const int32_t *index,
                                       int64_t n, unsigned int *bad, void *stream) {
  if (n < 0 || grid_len < 1) return ddfg_set_error(DDFG_EINVAL, "weights_accumulate: bad sizes");
  if (n == 0) return DDFG_OK;
  if (!grid || !weights || !index || !bad) return ddfg_set_error(DDFG_EINVAL, "weights_accumulate: null pointer");
  weights_accumulate_kernel<<<ddfg_num_ctas(8), 256, 0, (cudaStream_t)stream>>>(grid, grid_len, weights, index, n,
                                                                               bad);
  return launch_check("weights_accumulate");
}

extern "C" int ddfg_weights_robust(double *grid, int64_t npix, int32_t nbands, double numerator_sqrt,
                                   double *workspace, void *stream) {
  if (npix < 1 || nbands < 1) return ddfg_set_error(DDFG_EINVAL, "weights_robust: bad sizes");
  if (!grid || !workspace) return ddfg_set_error(DDFG_EINVAL, "weights_robust: null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(workspace, 0, sizeof(double) * 2 * (size_t)nbands, st);
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "weights_robust: %s", cudaGetErrorString(e));
  weights_sums_kernel<<<ddfg_num_ctas(4), 256, 0, st>>>(grid, npix, nbands, workspace);
  int rc = launch_check("weights_robust sums");
  if (rc) return rc;
  weights_robust_kernel<<<ddfg_num_ctas(8), 256, 0, st>>>(grid, npix, nbands, workspace, numerator_sqrt);
  return launch_check("weights_robust");
}

extern "C" int ddfg_weights_finalize(float *weights, const int32_t *index, int64_t n, const double *grid,
                                     int64_t grid_len, void *stream) {
  if (n < 0 || grid_len < 1) return ddfg_set_error(DDFG_EINVAL, "weights_finalize: bad sizes");
  if (n == 0) return DDFG_OK;
  if (!weights || !index || !grid) return ddfg_set_error(DDFG_EINVAL, "weights_finalize: null pointer");
  weights_finalize_kernel<<<ddfg_num_ctas(8), 256, 0, (cudaStream_t)stream>>>(weights, index, n, grid, grid_len);
  return launch_check("weights_finalize");
}
