// BDA block-map planning: the word index of every block record, and a full validity check.
//
// The reference walks the packed map sequentially (gridder.h:144-148, 185-190; degridder.h:
// 107-136), so it needs no index; the GPU kernels give one lane per block and need each
// block's start, which is an exclusive prefix sum of the block sizes:
//   start[b] = 2 + NB + sum_{i<b} NRowBlocks[i].
// The check rejects maps the reference would read out of bounds (a row index equal to nrow
// passes its `irow > nrows` guard, gridder.h:214) instead of running them.
#include <cub/device/device_scan.cuh>
#include <cuda_runtime.h>

#include "ddfg_internal.h"

namespace {

__global__ void widen_sizes_kernel(const int32_t *sizes, int64_t n, int64_t *out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (int64_t)sizes[i];
}

__global__ void plan_check_kernel(const int32_t *map, int64_t len, int64_t nblocks, int64_t nrow, int32_t nchan,
                                  int64_t *start, unsigned int *err) {
  const int64_t base = 2 + nblocks;
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nblocks; b += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = start[b] + base;
    start[b] = s;
    const int32_t sz = map[2 + b];
    if (sz < 2 || s + sz > len) {
      atomicOr(err, 1u);
      continue;
    }
    const int32_t c0 = map[s], c1 = map[s + 1];
    if (c0 < 0 || c1 < c0 || c1 > nchan) atomicOr(err, 2u);
    if (sz != 3 || c1 != c0 + 1) atomicOr(err, 16u);  // not a single-visibility block
    for (int32_t i = 2; i < sz; ++i) {
      const int32_t r = map[s + i];
      if (r < 0 || (int64_t)r >= nrow) {
        atomicOr(err, 4u);
        break;
      }
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const int64_t nb = (int64_t)(uint32_t)map[0] + ((int64_t)map[1] << 32);
    if (nb != nblocks) atomicOr(err, 8u);
  }
}

size_t scan_bytes(int64_t nblocks) {
  size_t bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, bytes, (int64_t *)nullptr, (int64_t *)nullptr, nblocks);
  return bytes;
}

}  // namespace

extern "C" size_t ddfg_bda_plan_workspace_size(int64_t nblocks) {
  return ((scan_bytes(nblocks > 0 ? nblocks : 1) + 255) / 256) * 256 + 256;
}

extern "C" int ddfg_bda_plan(const int32_t *bda_map, int64_t bda_len, int64_t nblocks, int64_t nrow, int32_t nchan,
                             int64_t *block_start, void *workspace, size_t workspace_bytes, void *stream_,
                             int32_t *single_out) {
  cudaStream_t stream = (cudaStream_t)stream_;
  if (!bda_map || bda_len < 2 || nblocks < 0 || (nblocks > 0 && !block_start) || !workspace)
    return ddfg_set_error(DDFG_EINVAL, "bda_plan: null pointer or bad length");
  if (bda_len < 2 + nblocks) return ddfg_set_error(DDFG_EMAP, "bda_plan: map shorter than its block table");
  const size_t need = ddfg_bda_plan_workspace_size(nblocks);
  if (workspace_bytes < need) return ddfg_set_error(DDFG_ESIZE, "bda_plan: workspace %zu < %zu bytes", workspace_bytes, need);
  size_t tmp_bytes = need - 256;
  unsigned int *err = (unsigned int *)((char *)workspace + tmp_bytes);
  cudaError_t e = cudaMemsetAsync(err, 0, sizeof(unsigned int), stream);
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "bda_plan: %s", cudaGetErrorString(e));
  if (nblocks > 0) {
    widen_sizes_kernel<<<ddfg_num_ctas(4), 256, 0, stream>>>(bda_map + 2, nblocks, block_start);
    e = cub::DeviceScan::ExclusiveSum(workspace, tmp_bytes, block_start, block_start, nblocks, stream);
    if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "bda_plan scan: %s", cudaGetErrorString(e));
  }
  const int ctas = ddfg_num_ctas(4);
  plan_check_kernel<<<ctas, 256, 0, stream>>>(bda_map, bda_len, nblocks, nrow, nchan, block_start, err);
  e = cudaGetLastError();
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "bda_plan check: %s", cudaGetErrorString(e));
  unsigned int herr = 0;
  e = cudaMemcpyAsync(&herr, err, sizeof(herr), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "bda_plan: %s", cudaGetErrorString(e));
  if (herr & 8u) return ddfg_set_error(DDFG_EMAP, "bda_plan: map header block count differs from nblocks");
  if (herr & 1u) return ddfg_set_error(DDFG_EMAP, "bda_plan: a block size is < 2 or runs past the map end");
  if (herr & 2u) return ddfg_set_error(DDFG_EMAP, "bda_plan: a block's channel range is outside [0, nchan]");
  if (herr & 4u) return ddfg_set_error(DDFG_EMAP, "bda_plan: a block names a row outside [0, nrow)");
  if (single_out) *single_out = (herr & 16u) ? 0 : 1;
  return DDFG_OK;
}

// ------------------------------------------------------------------------------------------
// Allocation-free variant of ddfg_bda_plan.
//
// Some callers cannot allocate device memory when they plan a block map: a host application
// that hands every byte of the GPU to its own pool allocator, a real-time pipeline that forbids
// allocation after start-up, or a caller that has no workspace to offer at that point.  For
// them ddfg_bda_plan_noalloc keeps its scratch (the prefix-sum temporaries and the check's error
// word) in the fixed array below, which every GPU that loads the library holds until the
// process exits.  The array's address is looked up with the device current on every call made
// outside stream capture; a call made during capture reuses the last address, so the first call
// on a device should come before any stream capture.  All calls on a device share the array: two calls that overlap on the GPU
// (different streams, or different host threads) race, so callers serialise them.
// ------------------------------------------------------------------------------------------
#include <mutex>

namespace {

constexpr size_t kNoallocScratchBytes = size_t(1) << 20;  // 1 MiB per device
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
void *g_noalloc_addr[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device.  It is looked up again on every
// call made outside stream capture (so a context re-created after cudaDeviceReset gets its own
// address), and the last address is kept for calls made while the stream is being captured.
int noalloc_scratch(void **out, cudaStream_t stream) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "bda_plan_noalloc: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return ddfg_set_error(DDFG_ESIZE, "bda_plan_noalloc: device %d >= %d", dev, kMaxDevices);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(stream, &cap);
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "bda_plan_noalloc: %s", cudaGetErrorString(e));
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_addr[dev] || cap == cudaStreamCaptureStatusNone) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return ddfg_set_error(DDFG_ECUDA, "bda_plan_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return DDFG_OK;
}

}  // namespace

extern "C" int ddfg_bda_plan_noalloc(const int32_t *bda_map, int64_t bda_len, int64_t nblocks, int64_t nrow,
                                     int32_t nchan, int64_t *block_start, void *stream_, int32_t *single_out) {
  cudaStream_t stream = (cudaStream_t)stream_;
  if (nblocks > DDFG_BDA_PLAN_NOALLOC_MAX_BLOCKS)
    return ddfg_set_error(DDFG_ESIZE, "bda_plan_noalloc: %lld blocks exceed the fixed scratch limit of %d blocks",
                          (long long)nblocks, DDFG_BDA_PLAN_NOALLOC_MAX_BLOCKS);
  if (!bda_map || bda_len < 2 || nblocks < 0 || (nblocks > 0 && !block_start))
    return ddfg_set_error(DDFG_EINVAL, "bda_plan_noalloc: null pointer or bad length");
  if (bda_len < 2 + nblocks) return ddfg_set_error(DDFG_EMAP, "bda_plan_noalloc: map shorter than its block table");
  void *scratch = nullptr;
  int rc = noalloc_scratch(&scratch, stream);
  if (rc) return rc;
  // Layout: [prefix-sum temporaries ... | error word in the last 256 bytes]
  size_t tmp_bytes = 0;
  cudaError_t e = cudaSuccess;
  if (nblocks > 0) {
    e = cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, block_start, block_start, nblocks, stream);
    if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "bda_plan_noalloc: %s", cudaGetErrorString(e));
  }
  if (tmp_bytes > kNoallocScratchBytes - 256)
    return ddfg_set_error(DDFG_ESIZE, "bda_plan_noalloc: scan needs %zu bytes, fixed scratch holds %zu", tmp_bytes,
                          kNoallocScratchBytes - 256);
  unsigned int *err = (unsigned int *)((char *)scratch + kNoallocScratchBytes - 256);
  // The array keeps the previous call's contents: the error word must start at zero.
  e = cudaMemsetAsync(err, 0, sizeof(unsigned int), stream);
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "bda_plan_noalloc: %s", cudaGetErrorString(e));
  if (nblocks > 0) {
    widen_sizes_kernel<<<ddfg_num_ctas(4), 256, 0, stream>>>(bda_map + 2, nblocks, block_start);
    e = cub::DeviceScan::ExclusiveSum(scratch, tmp_bytes, block_start, block_start, nblocks, stream);
    if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "bda_plan_noalloc scan: %s", cudaGetErrorString(e));
  }
  plan_check_kernel<<<ddfg_num_ctas(4), 256, 0, stream>>>(bda_map, bda_len, nblocks, nrow, nchan, block_start, err);
  e = cudaGetLastError();
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "bda_plan_noalloc check: %s", cudaGetErrorString(e));
  unsigned int herr = 0;
  e = cudaMemcpyAsync(&herr, err, sizeof(herr), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "bda_plan_noalloc: %s", cudaGetErrorString(e));
  if (herr & 8u) return ddfg_set_error(DDFG_EMAP, "bda_plan_noalloc: map header block count differs from nblocks");
  if (herr & 1u) return ddfg_set_error(DDFG_EMAP, "bda_plan_noalloc: a block size is < 2 or runs past the map end");
  if (herr & 2u) return ddfg_set_error(DDFG_EMAP, "bda_plan_noalloc: a block's channel range is outside [0, nchan]");
  if (herr & 4u) return ddfg_set_error(DDFG_EMAP, "bda_plan_noalloc: a block names a row outside [0, nrow)");
  if (single_out) *single_out = (herr & 16u) ? 0 : 1;
  return DDFG_OK;
}
