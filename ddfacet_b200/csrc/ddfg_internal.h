// Internal declarations shared by the translation units of libddfg.so (not part of the ABI).
#pragma once
#include <cuda_runtime.h>

#include "ddfg.h"

// Records the message of the failing call for ddfg_last_error() and returns code.
int ddfg_set_error(int code, const char *fmt, ...);
// CTAs for a persistent launch on the current device (a multiple of the SM count).
int ddfg_num_ctas(int ctas_per_sm);

// One wave of a kernel: as many CTAs as can be resident at once on the current device (SMs x
// resident CTAs per SM), for grid-stride kernels whose CTAs do unequal work -- with more CTAs
// than fit, the later ones start as earlier ones finish and the last, partial wave sets the end.
template <typename K>
int ddfg_one_wave(K kernel, int threads, size_t smem) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  return ddfg_num_ctas(per_sm);
}

// Sets the kernel's dynamic shared-memory limit when smem needs more than the default and
// returns its resident CTAs per SM for (threads, smem) in *per_sm; both are cached per kernel,
// device and size, so a launch inside a captured step does no repeated host work.
int ddfg_kernel_prepare(const void *kernel, int threads, size_t smem, int *per_sm);

// Queue counters in a ddfg_batch workspace: the gridder's (one per launch of up to
// DDFG_TABLE_FACETS facets) then the degridder's (one per launch, at most one per facet).
constexpr int kGridCounters = (DDFG_MAX_FACETS + DDFG_TABLE_FACETS - 1) / DDFG_TABLE_FACETS;
constexpr int kDegridCounters = DDFG_MAX_FACETS;

// batch NULL: static item order, default packs (ddfg_grid / ddfg_degrid).
int ddfg_launch_grid(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_facet *facets, int nfacets, int policy,
                     int nvispol, int dopsf, const ddfg_batch *batch, cudaStream_t stream);
int ddfg_launch_degrid(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_facet *facets, int nfacets, int policy,
                       int nvispol, const ddfg_batch *batch, cudaStream_t stream);
int ddfg_launch_degrid_adjoint(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_facet *facets, int nfacets,
                               int policy, int nvispol, int num_ctas, cudaStream_t stream);
int ddfg_launch_jones_grad(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_facet *facets, int nfacets,
                           int policy, int nvispol, void *grad, int num_ctas, cudaStream_t stream);
