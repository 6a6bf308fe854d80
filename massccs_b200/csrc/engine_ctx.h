// engine_ctx.h -- internal to libmassccs_gpu.so: the context behind the
// opaque ccs_ctx handle of include/massccs_gpu.h and the helpers the engine's
// translation units share (the trajectory engine in ccs_engine.cu, the
// learned field in field.cu, the field's trajectory kernels in traj_field.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "../../include/massccs_gpu.h"
#include "ccs_device.cuh"

struct FieldState;  // the learned field of a context (field.cu)

struct ccs_ctx {
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[10] = {};  // [0..4] ccs_run, [5..7] passes, [8..9] autotuner
  ccs_params p{};
  bool have_params = false, have_target = false;
  std::string err;
  // engine grid
  int nx = 0, ny = 0, nz = 0, natoms = 0, max_cell = 0;
  int lcap = 2048;  // warp-pass candidate-list entries (ccs::LCAP .. ccs::LCAP_MAX)
  double h = 0, origin[3] = {0, 0, 0}, bb_lo[3] = {0, 0, 0}, bb_hi[3] = {0, 0, 0}, reach = 0;
  int charged = 0, allpairs = 0, coul_on = 0, dip_on = 0;
  float4 *d_xyzq32 = nullptr;
  float2 *d_ab32 = nullptr, *d_abc32 = nullptr;
  double4 *d_xyzq64 = nullptr;
  double2 *d_ab64 = nullptr, *d_abc64 = nullptr;
  int *d_cell_start = nullptr;
  // speed table
  double *d_vtab_v = nullptr, *d_vtab_s = nullptr;
  int vtab_n = 0;
  // per-run scratch
  unsigned long long *d_work = nullptr;  // [0] work counter, [1..7] stats, [8] clock, [9] parked, [10] resumed
  int *d_error = nullptr;
  double *d_rnd = nullptr;
  size_t rnd_cap = 0;
  int8_t *d_status = nullptr;
  double *d_omc = nullptr;
  uint32_t *d_steps = nullptr, *d_visits = nullptr;
  size_t out_cap = 0;
  // longest-first processing order
  float *d_key = nullptr, *d_key2 = nullptr;
  uint32_t *d_idx = nullptr, *d_idx2 = nullptr;
  void *d_sort_tmp = nullptr;
  size_t order_cap = 0, sort_tmp_bytes = 0;
  // parked long trajectories (lane pass -> warp pass)
  void *d_park = nullptr;
  size_t park_bytes = 0;
  // speculative retries: records and try outcomes
  ccs::SpecRec *d_spec_rec = nullptr;
  ccs::SpecOut *d_spec_out = nullptr;
  size_t spec_cap = 0;
  // device copy of the launch parameters (read by the non-inlined set-up code)
  ccs::KParams *d_kparams = nullptr;
  ccs::KParams h_kparams{};
  // batched runs led by this context: the ions' parameters and first trajectories
  ccs::KParams *d_bkp = nullptr;
  unsigned long long *d_bstart = nullptr;
  size_t bkp_cap = 0;
  int batch_G = 0;                        // tuned lanes for the last batch shape
  size_t batch_nions = 0, batch_total = 0;
  // launch choice
  int tuned_G = 0, tuned_block = 0;
  ccs_stats last{};
  // where the last run keeps its counters and error flag (the context's own
  // buffers, or the static scratch of ccs_run_device_noalloc)
  unsigned long long *run_work = nullptr;
  int *run_error = nullptr;
  // learned field (null until ccs_field_train); runs use it while field_on
  FieldState *field = nullptr;
  bool field_on = false;
};

namespace ccs_internal {

// Copies and fills ordered on the context's stream.  The stream is created
// non-blocking, so the legacy-stream cudaMemcpy / cudaMemset are not ordered
// with its kernels (a device memset may still run, and a pageable host-to-
// device copy may still be in flight, when the next kernel on the stream
// starts).  Host-to-device copies from pageable memory are staged before the
// call returns, so the source may be freed; to_host waits for the stream.
inline cudaError_t to_dev(const ccs_ctx *c, void *dst, const void *src, size_t bytes);
inline cudaError_t to_host(const ccs_ctx *c, void *dst, const void *src, size_t bytes);
inline cudaError_t zero_dev(const ccs_ctx *c, void *p, size_t bytes);

inline int fail(ccs_ctx *c, int code, const char *fmt, ...) {
  if (c) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    c->err = buf;
  }
  return code;
}

#define CK(call)                                                                       \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail(c, CCS_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_),    \
                  __FILE__, __LINE__);                                                 \
  } while (0)

template <typename P> inline void dfree(P *&p) {
  if (p) cudaFree((void *)p);
  p = nullptr;
}


inline bool is_molecule(int gas) { return gas == CCS_GAS_N2 || gas == CCS_GAS_CO2; }
inline int gas_kind(int gas) { return gas == CCS_GAS_N2 ? ccs::GAS_N2 : gas == CCS_GAS_CO2 ? ccs::GAS_CO2 : ccs::GAS_ATOM; }

using KernelFn = void (*)(ccs::KParams, const ccs::KParams *);
// The trajectory kernels with the learned field (traj_field.cu): lane pass
// with G lanes per exact evaluation, warp pass with nt threads.
KernelFn pick_traj_field(int gas, bool hasq, int G);
KernelFn pick_resume_field(int gas, bool hasq, int nt);

// Launch parameters of a context's target and scalars (ccs_engine.cu).
ccs::KParams base_params(const ccs_ctx *c);
// Site force and energy of gas site `site` at npts device positions (x, y, z
// doubles), into device arrays f (npts x 3) and U (npts); asynchronous on s.
int eval_site_forces_device(ccs_ctx *c, size_t npts, int site, const double *d_pos, double *d_f, double *d_U,
                            cudaStream_t s);
// The learned field's launch parameters and memory (field.cu).
void field_kparams(const ccs_ctx *c, ccs::KParams &k);
void field_free(ccs_ctx *c);

inline cudaError_t to_dev(const ccs_ctx *c, void *dst, const void *src, size_t bytes) {
  return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream);
}
inline cudaError_t to_host(const ccs_ctx *c, void *dst, const void *src, size_t bytes) {
  const cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream);
  return e != cudaSuccess ? e : cudaStreamSynchronize(c->stream);
}
inline cudaError_t zero_dev(const ccs_ctx *c, void *p, size_t bytes) {
  return cudaMemsetAsync(p, 0, bytes, c->stream);
}

}  // namespace ccs_internal
