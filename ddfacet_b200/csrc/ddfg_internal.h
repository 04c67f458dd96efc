// Internal declarations shared by the translation units of libddfg.so (not part of the ABI).
#pragma once
#include <cuda_runtime.h>

#include "ddfg.h"

// Records the message of the failing call for ddfg_last_error() and returns code.
int ddfg_set_error(int code, const char *fmt, ...);
// CTAs for a persistent launch on the current device (a multiple of the SM count).
int ddfg_num_ctas(int ctas_per_sm);

int ddfg_launch_grid(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_facet *facets, int nfacets, int policy,
                     int nvispol, int dopsf, int num_ctas, cudaStream_t stream);
int ddfg_launch_degrid(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_facet *facets, int nfacets, int policy,
                       int nvispol, int num_ctas, cudaStream_t stream);
int ddfg_launch_grid_sorted(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_facet *facets, int nfacets, int policy,
                            int nvispol, int dopsf, const ddfg_sort_plan *plan, int compensated, int max_support,
                            int facets_per_launch, cudaStream_t stream);
int ddfg_launch_degrid_sorted(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_facet *facets, int nfacets,
                              int policy, int nvispol, const ddfg_sort_plan *plan, int max_support,
                              int facets_per_launch, cudaStream_t stream);
int ddfg_launch_degrid_adjoint(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_facet *facets, int nfacets,
                               int policy, int nvispol, int num_ctas, cudaStream_t stream);
int ddfg_launch_jones_grad(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_facet *facets, int nfacets,
                           int policy, int nvispol, void *grad, int num_ctas, cudaStream_t stream);
