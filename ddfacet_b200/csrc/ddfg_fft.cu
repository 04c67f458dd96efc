// Per-facet transforms between grids and images, and stitching into the main image.
//
//  * grid -> dirty facet image: GridToIm (ClassDDEGridMachine.py:1186-1190) is
//    Grid *= OverS^2; fftshift(ifft2(ifftshift(Grid))) * N^2 (ModFFTW.py:584-599), i.e. the
//    unnormalised inverse DFT of the centred grid.  One shift+scale kernel, a batched cuFFT
//    C2C inverse over every (band, pol) plane, one shift kernel back.
//  * stitching: FacetsToIm_Channel (ClassFacetMachine.py:1331-1416): real part times InvSphe times
//    the facet's spatial weight over (sum of weights x sqrt(sum of Jones)), zero where the taper
//    is below 1e-3, flipped and transposed ([::-1,:].T), cropped with GiveEdges (GiveEdges.py:
//    29-80) and added into the main image; then the main image is divided by the facet norm
//    (:1411-1414).  One fused kernel per facet; facets are added one after the other on the
//    stream, so overlapping padded facets add in a fixed order.
//  * model image -> facet grid: GiveModelTessel(ToGrid=True) (ClassImToGrid.py:138-264): crop
//    the padded facet box, divide by the facet norm, multiply by the spatial weight, divide by
//    the taper (zero where it is below 1e-3), transpose and flip (.T[::-1,:]), scale by
//    (OverS N)^2 and take fftshift(fft2(ifftshift(.))) / N^2 (ModFFTW.py:557-582).  One fused
//    gather+shift kernel, cuFFT forward, one shift+scale kernel.
//
// The facet's 2-D arrays (taper, spatial weight) are [N][N] float32 in the orientation named in
// each entry point.  cuFFT is the only library call; every other pass is a kernel here.
#include <cuda_runtime.h>
#include <cufft.h>

#include "ddfg_common.cuh"
#include "ddfg_internal.h"

struct ddfg_fft_plan {
  cufftHandle h;
  int n, batch;
};

namespace {

// (i + s) mod n for 0 <= i < n, 0 <= s < n
__device__ __forceinline__ int wrap(int i, int s, int n) {
  const int j = i + s;
  return j >= n ? j - n : j;
}

// out[p][y][x] = in[p][(y + h) % n][(x + h) % n] * scale   (ifftshift with h = n / 2)
__global__ void ishift_scale_kernel(const float2 *__restrict__ in, float2 *__restrict__ out, int n, int planes,
                                    float scale) {
  const int h = n / 2;
  const int64_t total = (int64_t)planes * n * n;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = i / ((int64_t)n * n);
    const int r = (int)((i / n) % n), c = (int)(i % n);
    const float2 v = in[p * n * n + (int64_t)wrap(r, h, n) * n + wrap(c, h, n)];
    out[i] = make_float2(v.x * scale, v.y * scale);
  }
}

// out[p][r][c] = in[p][(r - h) mod n][(c - h) mod n] * scale   (fftshift)
__global__ void shift_scale_kernel(const float2 *__restrict__ in, float2 *__restrict__ out, int n, int planes,
                                   float scale) {
  const int h = n / 2;
  const int64_t total = (int64_t)planes * n * n;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = i / ((int64_t)n * n);
    const int r = (int)((i / n) % n), c = (int)(i % n);
    const float2 v = in[p * n * n + (int64_t)wrap(r, n - h, n) * n + wrap(c, n - h, n)];
    out[i] = make_float2(v.x * scale, v.y * scale);
  }
}

struct Edges {
  int x0m, x1m, y0m, y1m, x0f, x1f, y0f, y1f;
};

// GiveEdges(xc, yc, M, n//2, n//2, n) (GiveEdges.py:29-80), no parity argument.
Edges give_edges(int xc, int yc, int m, int n) {
  Edges e;
  const int mx0 = xc - n / 2;
  e.x0m = mx0 > 0 ? mx0 : 0;
  e.x0f = e.x0m - mx0;
  const int mx1 = xc + n / 2;
  int x1m = mx1 < m - 1 ? mx1 : m - 1;
  e.x1f = n - (mx1 - x1m);
  e.x1m = x1m + 1;
  const int my0 = yc - n / 2;
  e.y0m = my0 > 0 ? my0 : 0;
  e.y0f = e.y0m - my0;
  const int my1 = yc + n / 2;
  int y1m = my1 < m - 1 ? my1 : m - 1;
  e.y1f = n - (my1 - y1m);
  e.y1m = y1m + 1;
  return e;
}

// image[b][p][x0m + a][y0m + c] += Im[n-1-(y0f+c)][x0f+a]
// with Im[r][q] = Re(dirty[b][p][r][q]) * invsphe[r][q] * sw[r][q] / w[b][p], 0 where sphe < 1e-3
__global__ void stitch_kernel(const float2 *__restrict__ dirty, int nband, int npol, int n,
                              const float *__restrict__ sphe, const float *__restrict__ invsphe,
                              const float *__restrict__ sw, const double *__restrict__ weights,
                              float *__restrict__ image, int m, Edges e) {
  const int wa = e.x1m - e.x0m, wb = e.y1m - e.y0m;
  const int64_t per = (int64_t)wa * wb;
  const int64_t total = per * nband * npol;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t plane = i / per;
    const int64_t k = i - plane * per;
    const int a = (int)(k / wb), c = (int)(k - (int64_t)(k / wb) * wb);
    const int r = n - 1 - (e.y0f + c), q = e.x0f + a;
    const float s = sphe[(int64_t)r * n + q];
    float v = 0.f;
    if (!(s < 1e-3f)) {
      double w = weights[plane];
      if (w == 0.) w = 1.;
      // numexpr evaluates Im*InvSPhe*SpacialWeigth/weights in float64 (ClassFacetMachine.py:1393-1396)
      v = (float)((double)dirty[plane * n * n + (int64_t)r * n + q].x * (double)invsphe[(int64_t)r * n + q] *
                  (double)sw[(int64_t)r * n + q] / w);
    }
    image[plane * (int64_t)m * m + (int64_t)(e.x0m + a) * m + (e.y0m + c)] += v;
  }
}

__global__ void normalise_kernel(float *image, int planes, int m, const float *__restrict__ norm) {
  const int64_t mm = (int64_t)m * m, total = mm * planes;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
    image[i] = image[i] / norm[i % mm];
}

// work[p][y][x] = M2[p][(y+h)%n][(x+h)%n] * scale with M2[i][j] = ModelIm[j][n-1-i] and ModelIm
// the normalised crop of the main image (zero outside the GiveEdges box and where sphe < 1e-3).
__global__ void model_gather_kernel(const float *__restrict__ image, int planes, int m, const float *__restrict__ norm,
                                    const float *__restrict__ sw, const float *__restrict__ sphe, int n, Edges e,
                                    float scale, float2 *__restrict__ work) {
  const int h = n / 2;
  const int64_t nn = (int64_t)n * n, total = nn * planes;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = idx / nn;
    const int y = (int)((idx / n) % n), x = (int)(idx % n);
    const int i = wrap(y, h, n), j = wrap(x, h, n);
    const int pr = j, pc = n - 1 - i;  // ModelIm[pr][pc]
    float v = 0.f;
    if (pr >= e.x0f && pr < e.x1f && pc >= e.y0f && pc < e.y1f) {
      const float s = sphe[(int64_t)pr * n + pc];
      if (!(s < 1e-3f)) {
        const int64_t mi = (int64_t)(e.x0m + (pr - e.x0f)) * m + (e.y0m + (pc - e.y0f));
        v = image[p * (int64_t)m * m + mi] / norm[mi] * sw[(int64_t)pr * n + pc] / s;
      }
    }
    work[idx] = make_float2(v * scale, 0.f);
  }
}

// The adjoint of model_gather_kernel with respect to the real image, accumulated:
// grad[p][x0m + a][y0m + c] += scale * Re(work[p][(i - h) mod n][(j - h) mod n]) * coef(pr, pc)
// with pr = x0f + a, pc = y0f + c, (i, j) = (n-1-pc, pr) and coef = sw / sphe / norm (0 where
// sphe < 1e-3): every image pixel of the facet box reads the one grid cell its value went to.
__global__ void model_gather_adjoint_kernel(const float2 *__restrict__ work, int planes, int m,
                                            const float *__restrict__ norm, const float *__restrict__ sw,
                                            const float *__restrict__ sphe, int n, Edges e, float scale,
                                            float *__restrict__ grad) {
  const int h = n / 2;
  const int wa = e.x1m - e.x0m, wb = e.y1m - e.y0m;
  const int64_t per = (int64_t)wa * wb, total = per * planes, nn = (int64_t)n * n;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = idx / per;
    const int64_t k = idx - p * per;
    const int a = (int)(k / wb), c = (int)(k - (int64_t)a * wb);
    const int pr = e.x0f + a, pc = e.y0f + c;
    const float s = sphe[(int64_t)pr * n + pc];
    if (s < 1e-3f) continue;
    const int y = wrap(n - 1 - pc, n - h, n), x = wrap(pr, n - h, n);
    const int64_t mi = (int64_t)(e.x0m + a) * m + (e.y0m + c);
    const float v = work[p * nn + (int64_t)y * n + x].x * scale;
    grad[p * (int64_t)m * m + mi] += v / norm[mi] * sw[(int64_t)pr * n + pc] / s;
  }
}

int nctas_for(int64_t total) {
  const int64_t b = (total + 255) / 256;
  const int64_t cap = ddfg_num_ctas(8);
  return (int)(b < cap ? (b > 0 ? b : 1) : cap);
}

}  // namespace

extern "C" int ddfg_fft_plan_create(int32_t n, int32_t batch, ddfg_fft_plan **out) {
  if (!out || n <= 0 || batch <= 0) return ddfg_set_error(DDFG_EINVAL, "fft_plan_create: bad argument");
  ddfg_fft_plan *p = new ddfg_fft_plan;
  p->n = n;
  p->batch = batch;
  int dims[2] = {n, n};
  cufftResult r = cufftPlanMany(&p->h, 2, dims, nullptr, 1, n * n, nullptr, 1, n * n, CUFFT_C2C, batch);
  if (r != CUFFT_SUCCESS) {
    delete p;
    return ddfg_set_error(DDFG_ECUDA, "fft_plan_create: cufftPlanMany failed (%d)", (int)r);
  }
  *out = p;
  return DDFG_OK;
}

extern "C" int ddfg_fft_plan_destroy(ddfg_fft_plan *p) {
  if (!p) return DDFG_OK;
  cufftDestroy(p->h);
  delete p;
  return DDFG_OK;
}

extern "C" int ddfg_grid_to_image(ddfg_fft_plan *p, void *grid, double scale, void *work, void *stream_) {
  cudaStream_t stream = (cudaStream_t)stream_;
  if (!p || !grid || !work) return ddfg_set_error(DDFG_EINVAL, "grid_to_image: null argument");
  const int64_t total = (int64_t)p->batch * p->n * p->n;
  ishift_scale_kernel<<<nctas_for(total), 256, 0, stream>>>((const float2 *)grid, (float2 *)work, p->n, p->batch,
                                                              (float)scale);
  if (cufftSetStream(p->h, stream) != CUFFT_SUCCESS) return ddfg_set_error(DDFG_ECUDA, "grid_to_image: cufftSetStream");
  if (cufftExecC2C(p->h, (cufftComplex *)work, (cufftComplex *)work, CUFFT_INVERSE) != CUFFT_SUCCESS)
    return ddfg_set_error(DDFG_ECUDA, "grid_to_image: cufftExecC2C failed");
  shift_scale_kernel<<<nctas_for(total), 256, 0, stream>>>((const float2 *)work, (float2 *)grid, p->n, p->batch, 1.f);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "grid_to_image: %s", cudaGetErrorString(e));
  return DDFG_OK;
}

extern "C" int ddfg_fft_centred(ddfg_fft_plan *p, void *data, int32_t inverse, double scale, void *work,
                                void *stream_) {
  cudaStream_t stream = (cudaStream_t)stream_;
  if (!p || !data || !work) return ddfg_set_error(DDFG_EINVAL, "fft_centred: null argument");
  const int64_t total = (int64_t)p->batch * p->n * p->n;
  ishift_scale_kernel<<<nctas_for(total), 256, 0, stream>>>((const float2 *)data, (float2 *)work, p->n, p->batch, 1.f);
  if (cufftSetStream(p->h, stream) != CUFFT_SUCCESS) return ddfg_set_error(DDFG_ECUDA, "fft_centred: cufftSetStream");
  if (cufftExecC2C(p->h, (cufftComplex *)work, (cufftComplex *)work, inverse ? CUFFT_INVERSE : CUFFT_FORWARD) !=
      CUFFT_SUCCESS)
    return ddfg_set_error(DDFG_ECUDA, "fft_centred: cufftExecC2C failed");
  shift_scale_kernel<<<nctas_for(total), 256, 0, stream>>>((const float2 *)work, (float2 *)data, p->n, p->batch,
                                                             (float)scale);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "fft_centred: %s", cudaGetErrorString(e));
  return DDFG_OK;
}

extern "C" int ddfg_stitch_facet(const void *dirty, int32_t nband, int32_t npol, int32_t n, const float *sphe,
                                 const float *invsphe, const float *sw_grid, const double *weights, float *image,
                                 int32_t m, int32_t xc, int32_t yc, void *stream_) {
  if (!dirty || !sphe || !invsphe || !sw_grid || !weights || !image || n <= 0 || m <= 0)
    return ddfg_set_error(DDFG_EINVAL, "stitch_facet: bad argument");
  const Edges e = give_edges(xc, yc, m, n);
  if (e.x1m <= e.x0m || e.y1m <= e.y0m) return DDFG_OK;  // facet box outside the image
  const int64_t total = (int64_t)(e.x1m - e.x0m) * (e.y1m - e.y0m) * nband * npol;
  stitch_kernel<<<nctas_for(total), 256, 0, (cudaStream_t)stream_>>>((const float2 *)dirty, nband, npol, n, sphe,
                                                                       invsphe, sw_grid, weights, image, m, e);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "stitch_facet: %s", cudaGetErrorString(err));
  return DDFG_OK;
}

extern "C" int ddfg_image_normalise(float *image, int32_t planes, int32_t m, const float *facet_norm, void *stream_) {
  if (!image || !facet_norm || planes <= 0 || m <= 0) return ddfg_set_error(DDFG_EINVAL, "image_normalise: bad argument");
  const int64_t total = (int64_t)planes * m * m;
  normalise_kernel<<<nctas_for(total), 256, 0, (cudaStream_t)stream_>>>(image, planes, m, facet_norm);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "image_normalise: %s", cudaGetErrorString(err));
  return DDFG_OK;
}

extern "C" int ddfg_image_to_grid(ddfg_fft_plan *p, const float *image, int32_t m, const float *norm_image,
                                  const float *sw_img, const float *sphe, int32_t xc, int32_t yc, double overs,
                                  void *grid_out, void *work, void *stream_) {
  cudaStream_t stream = (cudaStream_t)stream_;
  if (!p || !image || !norm_image || !sw_img || !sphe || !grid_out || !work || m <= 0)
    return ddfg_set_error(DDFG_EINVAL, "image_to_grid: bad argument");
  const int n = p->n;
  const Edges e = give_edges(xc, yc, m, n);
  const int64_t total = (int64_t)p->batch * n * n;
  const double s = overs * (double)n;
  model_gather_kernel<<<nctas_for(total), 256, 0, stream>>>(image, p->batch, m, norm_image, sw_img, sphe, n, e,
                                                              (float)(s * s), (float2 *)work);
  if (cufftSetStream(p->h, stream) != CUFFT_SUCCESS) return ddfg_set_error(DDFG_ECUDA, "image_to_grid: cufftSetStream");
  if (cufftExecC2C(p->h, (cufftComplex *)work, (cufftComplex *)work, CUFFT_FORWARD) != CUFFT_SUCCESS)
    return ddfg_set_error(DDFG_ECUDA, "image_to_grid: cufftExecC2C failed");
  shift_scale_kernel<<<nctas_for(total), 256, 0, stream>>>((const float2 *)work, (float2 *)grid_out, n, p->batch,
                                                             (float)(1.0 / ((double)n * n)));
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "image_to_grid: %s", cudaGetErrorString(err));
  return DDFG_OK;
}

extern "C" int ddfg_image_to_grid_adjoint(ddfg_fft_plan *p, const void *grid_grad, int32_t m, const float *norm_image,
                                          const float *sw_img, const float *sphe, int32_t xc, int32_t yc,
                                          double overs, float *image_grad, void *work, void *stream_) {
  cudaStream_t stream = (cudaStream_t)stream_;
  if (!p || !grid_grad || !norm_image || !sw_img || !sphe || !image_grad || !work || m <= 0)
    return ddfg_set_error(DDFG_EINVAL, "image_to_grid_adjoint: bad argument");
  const int n = p->n;
  const Edges e = give_edges(xc, yc, m, n);
  if (e.x1m <= e.x0m || e.y1m <= e.y0m) return DDFG_OK;  // facet box outside the image
  const int64_t total = (int64_t)p->batch * n * n;
  // adjoint of (fftshift, times 1/N^2): ifftshift, times 1/N^2
  ishift_scale_kernel<<<nctas_for(total), 256, 0, stream>>>((const float2 *)grid_grad, (float2 *)work, n, p->batch,
                                                              (float)(1.0 / ((double)n * n)));
  if (cufftSetStream(p->h, stream) != CUFFT_SUCCESS)
    return ddfg_set_error(DDFG_ECUDA, "image_to_grid_adjoint: cufftSetStream");
  // adjoint of the unnormalised forward DFT: the unnormalised inverse DFT
  if (cufftExecC2C(p->h, (cufftComplex *)work, (cufftComplex *)work, CUFFT_INVERSE) != CUFFT_SUCCESS)
    return ddfg_set_error(DDFG_ECUDA, "image_to_grid_adjoint: cufftExecC2C failed");
  const double s = overs * (double)n;
  const int64_t pix = (int64_t)(e.x1m - e.x0m) * (e.y1m - e.y0m) * p->batch;
  model_gather_adjoint_kernel<<<nctas_for(pix), 256, 0, stream>>>((const float2 *)work, p->batch, m, norm_image,
                                                                    sw_img, sphe, n, e, (float)(s * s), image_grad);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "image_to_grid_adjoint: %s", cudaGetErrorString(err));
  return DDFG_OK;
}
