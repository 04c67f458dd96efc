// C entry points of libddfg.so: argument checks, correlation/Stokes dispatch, error reporting.
//
// The dispatch tables restate pyGridderWPol / pyDeGridderWPol (DDFacet/Gridder/
// GridderSmearPols.cc:98-209 and :234-348): the same accepted (correlations, Stokes)
// combinations, the same quirk that gridding (I, U) from linear feeds uses the (I, Q) policy
// (GridderSmearPols.cc:142-143), and the same error texts.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <mutex>
#include <unordered_map>

#include "ddfg_common.cuh"
#include "ddfg_internal.h"

using namespace ddfg;

namespace {
thread_local char g_err[512] = "";

enum Corr { C_BAD = -1, C_I = 0, C_LIN2, C_CIRC2, C_LIN4, C_CIRC4 };

int corr_set(const ddfg_pol *p) {
  const int *c = p->corr_ids;
  if (p->ncorr == 1 && c[0] == 1) return C_I;
  if (p->ncorr == 2 && c[0] == 9 && c[1] == 12) return C_LIN2;
  if (p->ncorr == 2 && c[0] == 5 && c[1] == 8) return C_CIRC2;
  if (p->ncorr == 4 && c[0] == 9 && c[1] == 10 && c[2] == 11 && c[3] == 12) return C_LIN4;
  if (p->ncorr == 4 && c[0] == 5 && c[1] == 6 && c[2] == 7 && c[3] == 8) return C_CIRC4;
  return C_BAD;
}

// Stokes set as a string of letters, e.g. "IQUV".
void stokes_str(const ddfg_pol *p, char *out) {
  static const char *names = "?IQUV";
  int n = 0;
  for (int i = 0; i < p->npol && i < 4; ++i) {
    const int id = p->stokes_ids[i];
    out[n++] = (id >= 1 && id <= 4) ? names[id] : '?';
  }
  out[n] = 0;
}

bool corr_ids_ok(const ddfg_pol *p) {
  if (p->ncorr < 1 || p->ncorr > 4) return false;
  for (int i = 0; i < p->ncorr; ++i) {
    const int id = p->corr_ids[i];
    if (!((id >= 5 && id <= 12) || id == 1)) return false;
  }
  return true;
}

int grid_policy(const ddfg_pol *p) {
  char s[8];
  stokes_str(p, s);
  switch (corr_set(p)) {
    case C_LIN4:
      if (!strcmp(s, "I")) return G_I_LIN4;
      if (!strcmp(s, "Q")) return G_Q_LIN4;
      if (!strcmp(s, "U")) return G_U_LIN4;
      if (!strcmp(s, "V")) return G_V_LIN4;
      if (!strcmp(s, "IQ")) return G_IQ_LIN4;
      if (!strcmp(s, "IU")) return G_IQ_LIN4;  // GridderSmearPols.cc:142-143
      if (!strcmp(s, "IV")) return G_IV_LIN4;
      if (!strcmp(s, "QU")) return G_QU_LIN4;
      if (!strcmp(s, "IQU")) return G_IQU_LIN4;
      if (!strcmp(s, "IQUV")) return G_IQUV_LIN4;
      break;
    case C_CIRC4:
      if (!strcmp(s, "I")) return G_I_CIRC4;
      if (!strcmp(s, "IQ")) return G_IQ_CIRC4;
      if (!strcmp(s, "IU")) return G_IU_CIRC4;
      if (!strcmp(s, "IV")) return G_IV_CIRC4;
      if (!strcmp(s, "QU")) return G_QU_CIRC4;
      if (!strcmp(s, "IQU")) return G_IQU_CIRC4;
      if (!strcmp(s, "IQUV")) return G_IQUV_CIRC4;
      break;
    case C_LIN2:
      if (!strcmp(s, "I")) return G_I_LIN2;
      if (!strcmp(s, "IQ")) return G_IQ_LIN2;
      break;
    case C_CIRC2:
      if (!strcmp(s, "I")) return G_I_CIRC2;
      if (!strcmp(s, "IV")) return G_IV_CIRC2;
      break;
    case C_I:
      if (!strcmp(s, "I")) return G_I_FROM_I;
      break;
    default: break;
  }
  return -1;
}

int degrid_policy(const ddfg_pol *p) {
  char s[8];
  stokes_str(p, s);
  const int c = corr_set(p);
  if (!strcmp(s, "I")) {
    if (c == C_LIN4 || c == C_LIN2 || c == C_CIRC4 || c == C_CIRC2 || c == C_I) return D_DIAG_FROM_I;
  } else if (!strcmp(s, "Q")) {
    if (c == C_LIN4) return D_LIN4_FROM_Q;
  } else if (!strcmp(s, "U")) {
    if (c == C_LIN4) return D_LIN4_FROM_U;
  } else if (!strcmp(s, "V")) {
    if (c == C_LIN4) return D_LIN4_FROM_V;
  } else if (!strcmp(s, "IQUV")) {
    if (c == C_LIN4) return D_LIN4_FROM_IQUV;
    if (c == C_CIRC4) return D_CIRC4_FROM_IQUV;
  } else if (!strcmp(s, "IQ")) {
    if (c == C_LIN4) return D_LIN4_FROM_IQ;
    if (c == C_CIRC4) return D_CIRC4_FROM_IQ;
    if (c == C_LIN2) return D_LIN2_FROM_IQ;
  } else if (!strcmp(s, "IU")) {
    if (c == C_LIN4) return D_LIN4_FROM_IU;
    if (c == C_CIRC4) return D_CIRC4_FROM_IU;
  } else if (!strcmp(s, "IV")) {
    if (c == C_CIRC4) return D_CIRC4_FROM_IV;
    if (c == C_LIN4) return D_LIN4_FROM_IV;
    if (c == C_CIRC2) return D_CIRC2_FROM_IV;
  } else if (!strcmp(s, "QU")) {
    if (c == C_LIN4) return D_LIN4_FROM_QU;
  } else if (!strcmp(s, "IQU")) {
    if (c == C_LIN4) return D_LIN4_FROM_IQU;
    if (c == C_CIRC4) return D_CIRC4_FROM_IQU;
  }
  return -1;
}

int check_common(const char *who, const ddfg_vis *vs, const ddfg_jones *js, const ddfg_pol *pol,
                 const ddfg_facet *facets, int nfacets) {
  if (!vs || !js || !pol || !facets) return ddfg_set_error(DDFG_EINVAL, "%s: null argument", who);
  if (nfacets < 0 || nfacets > DDFG_MAX_FACETS)
    return ddfg_set_error(DDFG_ESIZE, "%s: nfacets=%d outside [0, %d]", who, nfacets, DDFG_MAX_FACETS);
  if (vs->ncorr != pol->ncorr) return ddfg_set_error(DDFG_EINVAL, "%s: vis has %d correlations, pol lists %d", who, vs->ncorr, pol->ncorr);
  if (vs->nblocks > 0 && (!vs->vis || !vs->uvw || !vs->freqs || !vs->chan_map || !vs->bda_map || !vs->block_start))
    return ddfg_set_error(DDFG_EINVAL, "%s: null visibility-set pointer", who);
  if (js->mode < 0 || js->mode > 2) return ddfg_set_error(DDFG_EINVAL, "%s: Jones mode %d", who, js->mode);
  if (js->mode != 0) {
    if (!js->kms && !js->beam)
      return ddfg_set_error(DDFG_EINVAL, "Jones matricies specified but neither E or DD Jones are applied. This is a bug!");
    if (!js->a0 || !js->a1) return ddfg_set_error(DDFG_EINVAL, "%s: Jones without antenna arrays", who);
    if (js->kms && (!js->kms_tmap || !js->kms_cmap)) return ddfg_set_error(DDFG_EINVAL, "%s: DD Jones maps missing", who);
    if (js->beam && (!js->beam_tmap || !js->beam_cmap)) return ddfg_set_error(DDFG_EINVAL, "%s: beam Jones maps missing", who);
    if (js->interp_mode == 1 && !js->interp_coefs) return ddfg_set_error(DDFG_EINVAL, "%s: interpolation coefficients missing", who);
  }
  for (int i = 0; i < nfacets; ++i) {
    const ddfg_facet &f = facets[i];
    if (!f.grid || !f.cf_data || !f.cf_offset || !f.cf_support)
      return ddfg_set_error(DDFG_EINVAL, "%s: facet %d has a null grid or CF pointer", who, i);
    if (f.nx <= 0 || f.ny <= 0 || f.nband <= 0 || f.npol <= 0 || f.nw <= 0 || f.overs <= 0)
      return ddfg_set_error(DDFG_EINVAL, "%s: facet %d has a bad shape", who, i);
    if (f.wmax == 0.) return ddfg_set_error(DDFG_EINVAL, "%s: facet %d has wmax = 0", who, i);
    if (((uintptr_t)f.grid & 7) || ((uintptr_t)f.grid_acc & 15))
      return ddfg_set_error(DDFG_EINVAL, "%s: facet %d grid (8 bytes) or FP64 accumulator (16 bytes) misaligned",
                            who, i);
    if (f.max_support <= 0 || f.max_support > 63)
      return ddfg_set_error(DDFG_EINVAL, "%s: facet %d max_support %d outside [1, 63]", who, i, f.max_support);
  }
  if (vs->nlarge < 0 || (vs->nlarge > 0 && (!vs->large_blocks || vs->large_min_vis < 1)))
    return ddfg_set_error(DDFG_EINVAL, "%s: bad large-block list", who);
  if (vs->nlarge > 0 && js && js->mode != 0 && js->scale_jones)
    return ddfg_set_error(DDFG_EUNSUPPORTED, "%s: a large-block list needs Jones terms that do not depend on uv "
                          "(no scale_jones)", who);
  if (vs->ncorr == 4 && ((uintptr_t)vs->vis & 15))
    return ddfg_set_error(DDFG_EINVAL, "%s: 4-correlation visibilities must be 16-byte aligned", who);
  if ((uintptr_t)vs->vis & 7) return ddfg_set_error(DDFG_EINVAL, "%s: visibilities must be 8-byte aligned", who);
  return DDFG_OK;
}
}  // namespace

int ddfg_set_error(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

int ddfg_num_ctas(int ctas_per_sm) {
  static thread_local int cached_dev = -1, cached_sms = 0;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148 * ctas_per_sm;
  if (dev != cached_dev) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    cached_dev = dev;
    cached_sms = sms;
  }
  return cached_sms * ctas_per_sm;
}

namespace {
struct PrepKey {
  const void *kernel;
  int device, threads;
  size_t smem;
  bool operator==(const PrepKey &o) const {
    return kernel == o.kernel && device == o.device && threads == o.threads && smem == o.smem;
  }
};
struct PrepHash {
  size_t operator()(const PrepKey &k) const {
    return std::hash<const void *>()(k.kernel) ^ (std::hash<size_t>()(k.smem) * 31u) ^
           (size_t)(k.device * 1315423911u) ^ (size_t)k.threads;
  }
};
std::mutex g_prep_mutex;
std::unordered_map<PrepKey, int, PrepHash> g_prep;
// Dynamic shared-memory limit set so far per (kernel, device): it only ever grows, since a
// launch needing more than the kernel's current limit fails.
std::unordered_map<PrepKey, size_t, PrepHash> g_smem_limit;
}  // namespace

int ddfg_kernel_prepare(const void *kernel, int threads, size_t smem, int *per_sm) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "kernel prepare: %s", cudaGetErrorString(e));
  const PrepKey key{kernel, dev, threads, smem};
  {
    std::lock_guard<std::mutex> lock(g_prep_mutex);
    auto it = g_prep.find(key);
    if (it != g_prep.end()) {
      *per_sm = it->second;
      return DDFG_OK;
    }
  }
  std::lock_guard<std::mutex> lock(g_prep_mutex);
  const PrepKey kkey{kernel, dev, 0, 0};
  size_t &limit = g_smem_limit[kkey];
  if (smem > 48 * 1024 && smem > limit) {
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
      return ddfg_set_error(DDFG_ECUDA, "kernel prepare: %zu bytes of shared memory: %s", smem, cudaGetErrorString(e));
    limit = smem;
  }
  int n = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem);
  if (e != cudaSuccess) return ddfg_set_error(DDFG_ECUDA, "kernel prepare: %s", cudaGetErrorString(e));
  if (n < 1) return ddfg_set_error(DDFG_ESIZE, "kernel prepare: %zu bytes of shared memory do not fit an SM", smem);
  g_prep[key] = n;
  *per_sm = n;
  return DDFG_OK;
}

extern "C" int ddfg_version(void) { return 2; }

extern "C" int ddfg_last_error(char *buf, int len) {
  if (!buf || len <= 0) return (int)strlen(g_err);
  snprintf(buf, (size_t)len, "%s", g_err);
  return (int)strlen(g_err);
}

namespace {
int grid_checks(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_pol *pol, const ddfg_facet *facets, int nfacets,
                int *policy) {
  int rc = check_common("grid", vs, js, pol, facets, nfacets);
  if (rc) return rc;
  if (!corr_ids_ok(pol))
    return ddfg_set_error(DDFG_EUNSUPPORTED, "Only accepts I,RR,RL,LR,LL,XX,XY,YX,YY as correlation input type");
  for (int i = 0; i < pol->npol; ++i)
    if (pol->stokes_ids[i] < 1 || pol->stokes_ids[i] > 4)
      return ddfg_set_error(DDFG_EUNSUPPORTED, "Only accepts I,Q,U,V as polarization output type");
  *policy = grid_policy(pol);
  if (*policy < 0)
    return ddfg_set_error(DDFG_EUNSUPPORTED, "Cannot convert input correlations to desired output Stokes parameters.");
  if (vs->nblocks > 0 && (!vs->flags || !vs->weights)) return ddfg_set_error(DDFG_EINVAL, "grid: null flags or weights");
  return DDFG_OK;
}
int degrid_checks(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_pol *pol, const ddfg_facet *facets,
                  int nfacets, int *policy) {
  int rc = check_common("degrid", vs, js, pol, facets, nfacets);
  if (rc) return rc;
  if (!corr_ids_ok(pol))
    return ddfg_set_error(DDFG_EUNSUPPORTED, "Only accepts I,RR,RL,LR,LL,XX,XY,YX,YY as correlation output types");
  *policy = degrid_policy(pol);
  if (*policy < 0)
    return ddfg_set_error(DDFG_EUNSUPPORTED, "Cannot convert input Stokes parameter to desired output correlations.");
  for (int i = 0; i < nfacets; ++i)
    if (facets[i].npol < pol->npol)
      return ddfg_set_error(DDFG_EINVAL, "degrid: facet %d grid has %d Stokes planes, %d needed", i, facets[i].npol,
                            pol->npol);
  return DDFG_OK;
}
}  // namespace

extern "C" int ddfg_grid(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_pol *pol, const ddfg_facet *facets,
                         int nfacets, int dopsf, void *stream) {
  g_err[0] = 0;
  int policy = -1;
  int rc = grid_checks(vs, js, pol, facets, nfacets, &policy);
  if (rc) return rc;
  if (nfacets == 0 || vs->nblocks == 0) return DDFG_OK;
  return ddfg_launch_grid(vs, js, facets, nfacets, policy, pol->npol, dopsf, nullptr, (cudaStream_t)stream);
}

extern "C" size_t ddfg_batch_workspace_size(void) {
  return sizeof(unsigned long long) * (size_t)(kGridCounters + kDegridCounters);
}

namespace {
int batch_checks(const ddfg_batch *batch, const char *who) {
  if (!batch) return ddfg_set_error(DDFG_EINVAL, "%s: null batch", who);
  if (batch->facets_per_pack < 0 || batch->stripes_per_item < 0 || batch->ctas_per_sm < 0)
    return ddfg_set_error(DDFG_EINVAL, "%s: negative batch parameter", who);
  if (!(batch->flags & 1)) {
    if (!batch->workspace || batch->workspace_bytes < ddfg_batch_workspace_size())
      return ddfg_set_error(DDFG_ESIZE, "%s: workspace %zu < %zu bytes", who, batch->workspace_bytes,
                            ddfg_batch_workspace_size());
    if ((uintptr_t)batch->workspace & 7) return ddfg_set_error(DDFG_EINVAL, "%s: workspace not 8-byte aligned", who);
  }
  return DDFG_OK;
}
}  // namespace

extern "C" int ddfg_grid_batched(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_pol *pol,
                                 const ddfg_facet *facets, int nfacets, int dopsf, const ddfg_batch *batch,
                                 void *stream) {
  g_err[0] = 0;
  int policy = -1;
  int rc = grid_checks(vs, js, pol, facets, nfacets, &policy);
  if (rc) return rc;
  rc = batch_checks(batch, "grid_batched");
  if (rc) return rc;
  if (nfacets == 0 || vs->nblocks == 0) return DDFG_OK;
  return ddfg_launch_grid(vs, js, facets, nfacets, policy, pol->npol, dopsf, batch, (cudaStream_t)stream);
}

extern "C" int ddfg_degrid_batched(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_pol *pol,
                                   const ddfg_facet *facets, int nfacets, const ddfg_batch *batch, void *stream) {
  g_err[0] = 0;
  int policy = -1;
  int rc = degrid_checks(vs, js, pol, facets, nfacets, &policy);
  if (rc) return rc;
  rc = batch_checks(batch, "degrid_batched");
  if (rc) return rc;
  if (nfacets == 0 || vs->nblocks == 0) return DDFG_OK;
  return ddfg_launch_degrid(vs, js, facets, nfacets, policy, pol->npol, batch, (cudaStream_t)stream);
}

extern "C" int ddfg_degrid(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_pol *pol, const ddfg_facet *facets,
                           int nfacets, void *stream) {
  g_err[0] = 0;
  int policy = -1;
  int rc = degrid_checks(vs, js, pol, facets, nfacets, &policy);
  if (rc) return rc;
  if (nfacets == 0 || vs->nblocks == 0) return DDFG_OK;
  return ddfg_launch_degrid(vs, js, facets, nfacets, policy, pol->npol, nullptr, (cudaStream_t)stream);
}

extern "C" int ddfg_degrid_adjoint(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_pol *pol,
                                   const ddfg_facet *facets, int nfacets, void *stream) {
  g_err[0] = 0;
  int policy = -1;
  int rc = degrid_checks(vs, js, pol, facets, nfacets, &policy);
  if (rc) return rc;
  if (nfacets == 0 || vs->nblocks == 0) return DDFG_OK;
  return ddfg_launch_degrid_adjoint(vs, js, facets, nfacets, policy, pol->npol, ddfg_num_ctas(4),
                                    (cudaStream_t)stream);
}

extern "C" int ddfg_degrid_jones_grad(const ddfg_vis *vs, const ddfg_jones *js, const ddfg_pol *pol,
                                      const ddfg_facet *facets, int nfacets, void *grad_kms, void *stream) {
  g_err[0] = 0;
  int policy = -1;
  int rc = degrid_checks(vs, js, pol, facets, nfacets, &policy);
  if (rc) return rc;
  if (js->mode == 0 || !js->kms) return ddfg_set_error(DDFG_EUNSUPPORTED, "degrid_jones_grad: needs kMS Jones");
  if (!grad_kms) return ddfg_set_error(DDFG_EINVAL, "degrid_jones_grad: null gradient array");
  if ((uintptr_t)grad_kms & 15)
    return ddfg_set_error(DDFG_EINVAL, "degrid_jones_grad: the gradient array must be 16-byte aligned");
  if (nfacets == 0 || vs->nblocks == 0) return DDFG_OK;
  return ddfg_launch_jones_grad(vs, js, facets, nfacets, policy, pol->npol, grad_kms, ddfg_num_ctas(4),
                                (cudaStream_t)stream);
}
