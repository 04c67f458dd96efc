/*
 * ddfg.h -- C ABI of the B200 facet gridder/degridder (libddfg.so).
 *
 * Plain C: every argument is a pointer, an integer or a double.  Every data pointer is a
 * DEVICE pointer (CUDA global memory on the current device) unless a comment says "host".
 * Calls are asynchronous on the given stream (cudaStream_t passed as void*; NULL = legacy
 * default stream); they never allocate device memory and never synchronise.  Every entry point
 * returns DDFG_OK (0) or a negative DDFG_E* code; ddfg_last_error() then gives the message of the
 * failing call on this host thread.
 *
 * Arrays follow the reference's numpy layouts (C order):
 *   grid     complex64 [nband][npol][ny][nx]
 *   vis      complex64 [nrow][nchan][ncorr]
 *   uvw      float64   [nrow][3]           (metres)
 *   flags    uint8     [nrow][nchan][ncorr] (numpy bool)
 *   weights  float32   [nrow][nchan]
 *   BDA map  int32     [2 + NB + sum_b NRowBlocks[b]]  (DDFacet's packed block map)
 *   Jones    complex64 [nt][nd][na][nch][2][2]
 *   CF       complex64, each plane [S*OverS][S*OverS] re-ordered as [OverS][OverS][S][S]
 */
#ifndef DDFG_H
#define DDFG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DDFG_OK 0
#define DDFG_EINVAL (-1)       /* bad argument (null pointer, bad shape)                  */
#define DDFG_EUNSUPPORTED (-2) /* correlation / Stokes combination not handled            */
#define DDFG_ECUDA (-3)        /* a CUDA runtime or cuFFT call failed                     */
#define DDFG_EMAP (-4)         /* malformed BDA block map (row or channel out of range)   */
#define DDFG_ESIZE (-5)        /* a size exceeds a documented maximum                     */

/* Maximum number of facets one ddfg_grid / ddfg_degrid call may take. */
#define DDFG_MAX_FACETS 1024
/* Facets whose descriptors travel in one kernel launch of the backward passes (the rest go in
 * further launches of balanced size). */
#define DDFG_FACETS_PER_LAUNCH 16
/* Facets whose descriptors travel in one launch of ddfg_grid / ddfg_degrid and their batched
 * variants (a __grid_constant__ kernel parameter table); a call with more facets makes further
 * launches of balanced size. */
#define DDFG_TABLE_FACETS 128

/* One facet: its grid, geometry, W-projection tables and outputs.
 * Replaces the per-facet arguments of pyGridderWPol / pyDeGridderWPol
 * (DDFacet/Gridder/GridderSmearPols.cc:76-97, 212-233): grid, sumwt, Lcfs, LcfsConj, WInfos,
 * increment, Lmaps[1] (FacetInfos) and LJones[6], LJones[8], LJones[17], LJones[18]. */
typedef struct ddfg_facet {
  void *grid;                  /* complex64 [nband][npol][ny][nx]                         */
  int32_t nband, npol, ny, nx; /* grid shape                                              */
  double incr_x, incr_y;       /* increment[0..1] in radians ([-cell, +cell])             */
  double cu, cv, l0, m0;       /* FacetInfos[0..3]: uvw shift and facet centre            */
  /* W-projection tables.  Plane p < nw is Lcfs[p] (used when the block's mean w > 0),
   * plane nw + p is LcfsConj[p] (used when w <= 0).  cf_offset gives each plane's first
   * complex element in cf_data; cf_support its support S (plane side = S * overs).        */
  const void *cf_data;
  const int64_t *cf_offset;    /* [2*nw] */
  const int32_t *cf_support;   /* [2*nw] */
  int32_t nw, overs;
  int32_t max_support;         /* largest cf_support[] value (host copy)                  */
  double ref_wave, wmax;       /* WInfos[0], WInfos[1]                                    */
  int32_t idir_kms, idir_beam; /* Jones direction of this facet (LJones[6][0], [8][0])    */
  double decorr_l, decorr_m;   /* LSmearing[5..6]: lm at which smearing is evaluated      */
  /* Outputs of ddfg_grid, accumulated (+=), float64; NULL to skip. */
  double *sumwt;               /* [nband][npol]   (sumwt)                                 */
  double *sumjones;            /* [2][nband]      (LJones[17])                            */
  double *sumjones_chan;       /* [2][nchan]      (LJones[18])                            */
  /* FP64 accumulation (optional; NULL = float32 atomic additions into grid).  A complex128 buffer
   * [nband][npol][ny][nx], all zero on entry: ddfg_grid / ddfg_grid_batched add every tap product
   * into it with FP64 atomics instead of into grid, and at the end of the call add it into grid
   * (one float32 rounding per cell: grid = fl(grid + acc)) and zero it again.  The grid then holds
   * the float32 rounding of the call's sum instead of the sum of ~10^4-10^6 successively rounded
   * float32 additions per cell, as the reference's FP64 products would give if its grid were
   * wider (gridder.h:360-362 adds them into the float grid one by one). */
  void *grid_acc;
} ddfg_facet;

/* The visibilities and everything indexed by row/channel (facet independent). */
typedef struct ddfg_vis {
  void *vis;                   /* complex64 [nrow][nchan][ncorr]; ddfg_degrid subtracts   */
  const double *uvw;           /* [nrow][3]                                               */
  const uint8_t *flags;        /* [nrow][nchan][ncorr]; only corr 0 is read (gridder.h:229)*/
  const float *weights;        /* [nrow][nchan]                                           */
  const double *freqs;         /* [nchan] Hz                                              */
  double freq_mean;            /* mean of freqs[] (host value; gridder.h:164-171)         */
  const double *recip_wvl;     /* [nchan] freqs[c] / 299792458 computed on the host, or NULL */
  const int32_t *chan_map;     /* [nchan] visibility channel -> grid band                 */
  int64_t nrow;
  int32_t nchan, ncorr;
  int32_t chan_equidistant;    /* LOptimisation[1]                                        */
  int32_t single_vis_blocks;   /* 1 only if every block is one row x one channel, as
                                  ddfg_bda_plan reports it; selects the lighter kernels    */
  const int32_t *bda_map;      /* packed block map                                        */
  int64_t bda_len;             /* words in bda_map                                        */
  const int64_t *block_start;  /* [nblocks] word index of each block's [ch0,ch1,rows...]  */
  int64_t nblocks;
  const uint8_t *sparsification; /* [nblocks] (gridding only) or NULL                     */
  /* Smearing (LSmearing, DecorrelationHelper.cc:19-40); uvw_dt NULL disables it. */
  const double *uvw_dt;        /* [nrow][3]                                               */
  double dt, dnu;
  int32_t do_tsmear, do_fsmear;
  /* Large blocks (optional; nlarge 0 disables): large_blocks[nlarge] must list, in any order,
     exactly the blocks of more than large_min_vis visibilities (rows x channels).  The
     averaged-block kernels of ddfg_grid / ddfg_degrid take them out of the one-lane-per-block
     walks and give each to one warp, its lanes strided over the block's visibilities; the
     FP64 block means keep the reference's sequential order, so indices stay bit-exact.
     Needs Jones terms that do not depend on uv (no scale_jones). */
  const int64_t *large_blocks;
  int64_t nlarge;
  int64_t large_min_vis;
} ddfg_vis;

/* Direction-dependent Jones terms (LJones, ClassDDEGridMachine.py:665-677). */
typedef struct ddfg_jones {
  int32_t mode;                /* 0 none, 1 per visibility, 2 per BDA block (DoApplyJones)*/
  const void *kms;             /* complex64 [nt][nd][na][nch][2][2] or NULL               */
  int32_t kms_dims[4];         /* nt, nd, na, nch                                         */
  const int32_t *kms_tmap;     /* [nrow] row -> Jones time slot                           */
  const int32_t *kms_cmap;     /* [nchan] channel -> Jones channel                        */
  const void *beam;            /* complex64 [nt][nd][na][nch][2][2] or NULL               */
  int32_t beam_dims[4];
  const int32_t *beam_tmap;
  const int32_t *beam_cmap;
  const int32_t *a0, *a1;      /* [nrow] antennas                                         */
  const float *interp_coefs;   /* [nd] (interp_mode 1) or NULL                            */
  int32_t interp_mode;         /* 0 nearest, 1 weighted                                   */
  int32_t apply_amp, apply_phase, scale_jones;
  double calib_error;          /* radians                                                 */
  double wavelength_mean;      /* mean over channels of c/nu                              */
} ddfg_jones;

/* Correlation and Stokes ids use casacore's numbering: I=1 Q=2 U=3 V=4 RR=5 RL=6 LR=7 LL=8
 * XX=9 XY=10 YX=11 YY=12 (DDFacet/Data/ClassStokes.py:39). */
typedef struct ddfg_pol {
  int32_t ncorr, npol;
  int32_t corr_ids[4];
  int32_t stokes_ids[4];
} ddfg_pol;

/* Scheduling of ddfg_grid_batched / ddfg_degrid_batched: one persistent launch per call (per
 * DDFG_TABLE_FACETS facets) whose CTAs take work items from a queue in device memory.  An item
 * is a run of stripes (32 consecutive blocks) of one facet pack; the warps of a CTA apply every
 * facet of the pack to a stripe in turn (its inputs are read once per pack).  Items are ordered
 * pack by pack, the large-block items of a pack first (the longest work starts first).  Zero
 * fields take the library's defaults (or the autotuner's choice, ddfacet_b200.autotune). */
typedef struct ddfg_batch {
  void *workspace;             /* >= ddfg_batch_workspace_size() bytes of device scratch, 8-byte aligned */
  size_t workspace_bytes;
  int32_t facets_per_pack;     /* facets applied to a stripe before the next stripe (0: default) */
  int32_t stripes_per_item;    /* stripes of one queue item (0: default)                   */
  int32_t ctas_per_sm;         /* resident CTAs per SM of the persistent launch (0: occupancy) */
  int32_t flags;               /* bit 0: static item order instead of the queue (for
                                  measurements); bit 1: the gridder's warps sum each stripe into a
                                  shared-memory tile and add the touched cells to the grid once
                                  (one Stokes plane; pays when a stripe's footprints overlap);
                                  bit 2: spread the items over as many contiguous regions of the
                                  block order as the launch has CTAs, taken in turn (CTAs work far
                                  apart: for maps in uv-cell order, on distant grid cells) */
} ddfg_batch;

/* Library and device checks. */
int ddfg_version(void);
int ddfg_last_error(char *buf, int len);

/* Bytes of device scratch ddfg_bda_plan needs for a map of nblocks blocks. */
size_t ddfg_bda_plan_workspace_size(int64_t nblocks);

/* single_out (host, may be NULL) receives 1 when every block has exactly one row and one
 * channel (the map of unaveraged data), else 0.
 * Reads the map's block sizes, writes the word index of every block record into block_start
 * (device, int64 [nblocks]) and checks that the header's block count is nblocks, every block
 * lies inside the map, 0 <= ch0 <= ch1 <= nchan and every row is in [0, nrow).  A plan call,
 * not a hot one: it synchronises the stream to read the check's result, and returns DDFG_EMAP
 * for a malformed map.  Replaces the sequential block walk of gridder.h:144-148, 185-190 and
 * degridder.h:107-136. */
int ddfg_bda_plan(const int32_t *bda_map, int64_t bda_len, int64_t nblocks, int64_t nrow, int32_t nchan,
                  int64_t *block_start, void *workspace, size_t workspace_bytes, void *stream,
                  int32_t *single_out);

/* Grid the visibility set onto every facet's grid (accumulating), with W-projection, facet
 * phase shift, per-antenna Jones, smearing and corr->Stokes conversion.
 * Replaces pyGridderWPol32 (DDFacet/Gridder/GridderSmearPols.cc:76-209, gridder.h:78-377),
 * called once per facet by ClassDDEGridMachine.put (ClassDDEGridMachine.py:681-861).
 * facets: HOST array of nfacets descriptors (copied into the launches). */
int ddfg_grid(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_pol *pol,
              const ddfg_facet *facets, int nfacets, int dopsf, void *stream);

/* Predict every facet's model grid and SUBTRACT the prediction from vs->vis in place.
 * Replaces pyDeGridderWPol (GridderSmearPols.cc:212-348, degridder.h:55-267), called by
 * ClassDDEGridMachine.get (ClassDDEGridMachine.py:922-1152).  The reference serialises the
 * subtraction of concurrent facets with named semaphores (Semaphores.cc:27-29); here every
 * facet of a call is applied by the warp that owns the block, so the result is deterministic. */
int ddfg_degrid(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_pol *pol,
                const ddfg_facet *facets, int nfacets, void *stream);

/* Backward pass of ddfg_degrid for the model grids.  ddfg_degrid subtracts a prediction P that
 * is linear in the facets' model grids; given vs->vis = dLoss/dP* (the gradient of a real loss,
 * complex64 [nrow][nchan][ncorr], read only), this adds P's adjoint applied to it to each
 * facets[i].grid (+=): conj(CF) taps at the degridder's footprint, the adjoint Stokes map (for
 * Stokes I from XX/YY: g_XX + g_YY), conj(phasor), J0^H g J1 and the smearing factor.  The
 * facets carry the degridder's CF order (as for ddfg_degrid).  Averaged BDA blocks sum their
 * visibilities' back-projected gradients at the block's footprint; per-block Jones (BDAJones)
 * are applied to that sum.  No counterpart in the reference, whose degridder has no
 * derivative. */
int ddfg_degrid_adjoint(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_pol *pol,
                        const ddfg_facet *facets, int nfacets, void *stream);

/* Backward pass of ddfg_degrid for the kMS Jones terms: with vs->vis = dLoss/dP* as above and
 * facets[i].grid the model grids of the forward pass, adds dLoss/dJ* to grad_kms (complex64,
 * the layout of js->kms, 16-byte aligned, +=).  kMS Jones alone or times a beam (the beam is a
 * constant: J = K.B, so the kMS terms see B0 M B1^H), nearest or weighted directions
 * (interpolation mode 1 scales the stored matrices by the squared sum of the coefficients, as
 * the forward does), through NormJones (amplitude / phase normalisation and amplitude scaling,
 * the latter at the uv the forward's Jones cache reads); needs kMS Jones (DDFG_EUNSUPPORTED
 * otherwise); any BDA map, per-visibility or per-block (BDAJones) Jones.  No counterpart in the
 * reference. */
int ddfg_degrid_jones_grad(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_pol *pol,
                           const ddfg_facet *facets, int nfacets, void *grad_kms, void *stream);

/* ---- Imaging weights (uniform / Briggs uv-density grid) ------------------------------------
 * The weight grid is float64 [nbands][npix] over the half uv-plane: npixx = 2 xymax + 1 cells in
 * u (offset by xymax), xymax + 1 in v, npix = npixx (xymax + 1), cell = 1 / (SuperUniform FOV).
 *
 * ddfg_weights_uv_index replaces ClassVisServer._uv_to_index (DDFacet/Data/ClassVisServer.py:
 * 981-1003): index[r][c] of every visibility (v < 0 flips (u, v); floor(u nu / c / cell) +
 * xymax and floor(v nu / c / cell); + band_of_chan[c] * npix when nbands > 1; 0 where the weight
 * is 0).  uvw [nrow][3] float64, freqs [nchan], weights float32 [nrow][nchan] with flagged
 * visibilities already 0, index int32 [nrow][nchan] out.  Unlike the reference it does not flip
 * the caller's uvw in place. */
int ddfg_weights_uv_index(const double *uvw, int64_t nrow, const double *freqs, int32_t nchan,
                          const float *weights, const int32_t *band_of_chan, int32_t nbands, double cell,
                          int64_t xymax, int64_t npixx, int64_t npix, int32_t *index, void *stream);

/* grid[index[i]] += weights[i] for every non-zero weight (pyAccumulateWeightsOntoGrid /
 * ...NoSem, GridderSmearPols.cc:32-74).  Indices outside [0, grid_len) are skipped and set bit 0
 * of *bad (a device word the caller clears and reads). */
int ddfg_weights_accumulate(double *grid, int64_t grid_len, const float *weights, const int32_t *index,
                            int64_t n, unsigned int *bad, void *stream);

/* Briggs weighting (ClassVisServer.py:897-904): per band, grid = 1 + grid * s2 / avgW with
 * s2 = numerator_sqrt^2 (numerator_sqrt = 5 * 10^-Robust) and avgW = sum grid^2 / sum grid.
 * workspace: 2 * nbands doubles of device scratch. */
int ddfg_weights_robust(double *grid, int64_t npix, int32_t nbands, double numerator_sqrt, double *workspace,
                        void *stream);

/* weights[i] /= grid[index[i]] (indices >= grid_len read cell 0), the uniform / Briggs
 * normalisation of _finalizeWeights_handler (ClassVisServer.py:1036-1043). */
int ddfg_weights_finalize(float *weights, const int32_t *index, int64_t n, const double *grid, int64_t grid_len,
                          void *stream);

/* ---- BDA block maps on the GPU (mode 1) -----------------------------------------------------
 * Replace GiveBlocksRowsListBL_old (DDFacet/Data/ClassSmearMapping.py:496-625), run per baseline
 * by the reference's process pool, and collectSmearMapping's packing (:83-135): the map's words
 * are identical.  rows: the visibility rows grouped by baseline in "a0:a1" key-string order,
 * ascending within a baseline (autocorrelations left out); bl_off [nbl + 1] the group bounds;
 * uvw [nrow][3]; chan_map [nchan] channel -> grid band; dfreq the channel width; dphi =
 * sqrt(6 (1 - Decorr)); l the field radius; nu0 = max frequency.
 * ddfg_bda_mode1_count writes each baseline's block and word counts ([nbl] int64 each);
 * ddfg_bda_mode1_write writes the block sizes (sizes, from the map's word 2) and blocks (body,
 * after the sizes) at the exclusive scans blk_off / word_off of those counts. */
int ddfg_bda_mode1_count(const double *uvw, const int32_t *rows, const int64_t *bl_off, int32_t nbl,
                         int32_t nchan, const int32_t *chan_map, double dfreq, double dphi, double l, double nu0,
                         int64_t *nblk, int64_t *nwords, void *stream);
int ddfg_bda_mode1_write(const double *uvw, const int32_t *rows, const int64_t *bl_off, int32_t nbl,
                         int32_t nchan, const int32_t *chan_map, double dfreq, double dphi, double l, double nu0,
                         const int64_t *blk_off, const int64_t *word_off, int32_t *sizes, int32_t *body,
                         void *stream);

/* ---- BDA block maps on the GPU (mode 2) -----------------------------------------------------
 * Replace GiveBlocksRowsListBL (DDFacet/Data/ClassSmearMapping.py:348-491), per baseline: time
 * blocks are the runs of equal int32(cumsum(delta_phase) / dphi) with delta_phase the phase change
 * between consecutive rows at the field edge (2 pi nu0 / 3e8 (|(du, dv)| l_max + |dw| n_max)),
 * channel blocks of int32(ceil(nchan / ceil(nchan / max(min dnu / dfreq, 1)))) channels cut where
 * the grid band changes.  Same arguments and two passes as mode 1 (l_max in place of l); the count
 * pass sets nblk[b] = -1 for a baseline with a single row, which the reference cannot map either
 * (it reads the second-to-last row difference). */
int ddfg_bda_mode2_count(const double *uvw, const int32_t *rows, const int64_t *bl_off, int32_t nbl,
                         int32_t nchan, const int32_t *chan_map, double dfreq, double dphi, double l_max, double nu0,
                         int64_t *nblk, int64_t *nwords, void *stream);
int ddfg_bda_mode2_write(const double *uvw, const int32_t *rows, const int64_t *bl_off, int32_t nbl,
                         int32_t nchan, const int32_t *chan_map, double dfreq, double dphi, double l_max, double nu0,
                         const int64_t *blk_off, const int64_t *word_off, int32_t *sizes, int32_t *body,
                         void *stream);

/* Most blocks ddfg_bda_plan_noalloc accepts. */
#define DDFG_BDA_PLAN_NOALLOC_MAX_BLOCKS (1 << 24)

/* ddfg_bda_plan for callers that cannot allocate device memory.  It has no counterpart in the
 * reference.  Same inputs, outputs and checks as ddfg_bda_plan, but no workspace argument: its
 * scratch is a fixed 1 MiB array inside the library, held by every GPU that loads the library
 * until the process exits, so maps are limited to DDFG_BDA_PLAN_NOALLOC_MAX_BLOCKS blocks
 * (DDFG_ESIZE above that).  It allocates nothing.  Each call made outside stream capture looks
 * up that array's device address (with the device current); a call made while the stream is
 * being captured reuses the last address, so make the first call on a device before any stream
 * capture (and, after a cudaDeviceReset, one more call outside capture).  Calls share the array: calls that overlap on the GPU race and must be serialised by
 * the caller. */
int ddfg_bda_plan_noalloc(const int32_t *bda_map, int64_t bda_len, int64_t nblocks, int64_t nrow, int32_t nchan,
                          int64_t *block_start, void *stream, int32_t *single_out);

/* Bytes of device scratch ddfg_grid_batched / ddfg_degrid_batched need (the queue counters). */
size_t ddfg_batch_workspace_size(void);

/* ddfg_grid as one persistent, queue-driven launch per DDFG_TABLE_FACETS facets (see
 * ddfg_batch): same inputs, outputs and checks.  The work queue balances uneven facets and
 * blocks (averaged BDA blocks of very different sizes) across the GPU; every call first resets
 * its counters (one cudaMemsetAsync), so the call can be captured in a CUDA graph.  Replaces the
 * per-facet gridding jobs of ClassFacetMachine (ClassFacetMachine.py:1574-1592). */
int ddfg_grid_batched(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_pol *pol, const ddfg_facet *facets,
                      int nfacets, int dopsf, const ddfg_batch *batch, void *stream);

/* ddfg_degrid the same way (ClassFacetMachine.py:1912-1944).  With facets_per_pack >= nfacets
 * every visibility is read and written once per call. */
int ddfg_degrid_batched(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_pol *pol, const ddfg_facet *facets,
                        int nfacets, const ddfg_batch *batch, void *stream);

/* The integer footprint of every block on one facet, as the gridder (degrid_means 0) or the
 * degridder (1) computes it (gridder.h:321-351, degridder.h:168-200): out int32 [nblocks][8] =
 * {status, iw, plane, locx, locy, offx, offy, cf sub-kernel index} where iw is the w-plane
 * index lrint((Nw-1)|W|RefWave nu/c/wmax), plane the CF table used (iw for W > 0, nw + iw for
 * LcfsConj), (locx, locy) the centre cell and (offx, offy) the oversampling offsets; status 1 =
 * gridded/degridded, 0 = skipped (no unflagged visibility, band outside the grid, w beyond
 * wmax, support outside the grid), in which case the later fields are -1 from the first skipped
 * step on.  Uses the kernels' own index code.  A check entry point: the reference exposes these
 * indices only inside its loops. */
int ddfg_block_geometry(const ddfg_vis *vs, const ddfg_facet *facet, int degrid_means, int32_t *out, void *stream);

/* Jones time slot of every row (ClassJones.GiveTimeMapping, DDFacet/Data/ClassJones.py:415-439):
 * out[r] = the last it with t0[it] <= times[r] < t1[it], 0 when no slot contains the row; the times
 * need not be sorted.  times float64 [nrow]; t0, t1 float64 [nt] (the solutions' slot bounds);
 * out int32 [nrow] (LJones[1] / LJones[3], the time maps ddfg_jones.kms_tmap / beam_tmap take). */
int ddfg_jones_time_map(const double *times, int64_t nrow, const double *t0, const double *t1, int32_t nt,
                        int32_t *out, void *stream);

/* Bytes of device scratch ddfg_check_large_blocks needs. */
size_t ddfg_check_large_blocks_workspace_size(int64_t nblocks);

/* Checks vs->large_blocks: every entry a block index in [0, nblocks), listed once, and the list
 * holds exactly the blocks of more than large_min_vis visibilities.  A plan call: it synchronises
 * the stream and returns DDFG_EMAP for a bad list.  (The kernels also skip list entries that are
 * out of range or not above the threshold, so a bad list cannot make them read out of bounds or
 * grid a small block twice.) */
int ddfg_check_large_blocks(const ddfg_vis *vs, void *workspace, size_t workspace_bytes, void *stream);

/* ---- per-facet transforms and stitching --------------------------------------------- */

/* A batched N x N complex64 FFT plan (cuFFT).  Creating one allocates; using one does not. */
typedef struct ddfg_fft_plan ddfg_fft_plan;
int ddfg_fft_plan_create(int32_t n, int32_t batch, ddfg_fft_plan **out);
int ddfg_fft_plan_destroy(ddfg_fft_plan *plan);

/* GridToIm in place on grid[batch][N][N] (ClassDDEGridMachine.py:1186-1190, ModFFTW.py:584-599):
 * grid <- fftshift(IDFT(ifftshift(grid * scale))) with the unnormalised inverse DFT (numpy's
 * ifft2 times N^2); scale is OverS^2 for GridToIm.  work: a second [batch][N][N] buffer. */
int ddfg_grid_to_image(ddfg_fft_plan *plan, void *grid, double scale, void *work, void *stream);

/* data[batch][N][N] <- fftshift(DFT(ifftshift(data))) * scale, forward or (inverse != 0)
 * unnormalised inverse DFT: ModFFTW.FFTW_2Donly.fft/ifft (ModFFTW.py:557-599) with scale 1/N^2
 * (fft) or 1 (ifft times N^2).  work: a second [batch][N][N] buffer. */
int ddfg_fft_centred(ddfg_fft_plan *plan, void *data, int32_t inverse, double scale, void *work, void *stream);

/* Adds one facet's dirty image (complex64 [nband][npol][N][N] from ddfg_grid_to_image) into the
 * main image float32 [nband][npol][M][M] (FacetsToIm_Channel, ClassFacetMachine.py:1331-1410):
 * Re(dirty) * invsphe * sw_grid / weights[band][pol] (weights 0 counts as 1), zero where
 * sphe < 1e-3, flipped and transposed, cropped by GiveEdges around the facet centre pixel
 * (xc, yc).  sphe, invsphe (float32 of 1/taper) and sw_grid are [N][N] in grid orientation;
 * weights is float64
 * [nband][npol] = SumWeights * sqrt(SumJonesNorm). */
int ddfg_stitch_facet(const void *dirty, int32_t nband, int32_t npol, int32_t n, const float *sphe,
                      const float *invsphe, const float *sw_grid, const double *weights, float *image, int32_t m,
                      int32_t xc, int32_t yc, void *stream);

/* image[plane] /= facet_norm (ClassFacetMachine.py:1411-1414); facet_norm is [M][M]. */
int ddfg_image_normalise(float *image, int32_t planes, int32_t m, const float *facet_norm, void *stream);

/* GiveModelTessel(ToGrid=True) for one facet (ClassImToGrid.py:138-264): crops the main model
 * image float32 [batch][M][M] around (xc, yc), divides by norm_image [M][M], multiplies by
 * sw_img [N][N] (image orientation), divides by sphe [N][N] (zero where sphe < 1e-3),
 * transposes and flips, scales by (overs N)^2 and writes fftshift(DFT(ifftshift(.))) / N^2
 * into grid_out complex64 [batch][N][N].  work: a [batch][N][N] complex64 scratch buffer. */
int ddfg_image_to_grid(ddfg_fft_plan *plan, const float *image, int32_t m, const float *norm_image,
                       const float *sw_img, const float *sphe, int32_t xc, int32_t yc, double overs, void *grid_out,
                       void *work, void *stream);

/* The adjoint of ddfg_image_to_grid with respect to the (real) model image, for differentiating a
 * prediction through the model image (no reference counterpart: the reference has no derivative).
 * image_grad float32 [batch][M][M] += Re(A^H grid_grad) where A is ddfg_image_to_grid's linear map
 * with the same arguments; grid_grad is complex64 [batch][N][N] (PyTorch's gradient convention).
 * Pixels outside the facet's GiveEdges box or where sphe < 1e-3 receive nothing.  work: a
 * [batch][N][N] complex64 scratch buffer. */
int ddfg_image_to_grid_adjoint(ddfg_fft_plan *plan, const void *grid_grad, int32_t m, const float *norm_image,
                               const float *sw_img, const float *sphe, int32_t xc, int32_t yc, double overs,
                               float *image_grad, void *work, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* DDFG_H */
