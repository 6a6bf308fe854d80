// ccs_engine.cu -- host side of libmassccs_gpu.so: the C-ABI of
// include/massccs_gpu.h, the engine's cell grid, the speed-sampler table,
// the launch autotuner and the kernel instantiations.
//
// Reference counterparts (cces-cepid/massccs):
//   ccs_set_target  <- MoleculeTarget arrays + LinkedCell (src/LinkedCell.cpp:19-440)
//   ccs_set_params  <- System members and Force ctor arguments (src/System.cpp:19-144,
//                      src/Force.cpp:20-26)
//   ccs_run         <- the OpenMP trajectory loop (src/System.cpp:204-285)
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cub/device/device_radix_sort.cuh>

#include "engine_ctx.h"

using namespace ccs;

namespace {
using namespace ccs_internal;

void free_target(ccs_ctx *c) {
  field_free(c);  // the learned field belongs to this target and these parameters
  dfree(c->d_xyzq32); dfree(c->d_ab32); dfree(c->d_abc32);
  dfree(c->d_xyzq64); dfree(c->d_ab64); dfree(c->d_abc64);
  dfree(c->d_cell_start);
  c->have_target = false;
  c->tuned_G = 0;
  c->batch_G = 0;
}


// GasBuffer::gas_properties (GasBuffer.cpp:58-192): site charges, masses, z offsets.
void gas_table(int gas, double q[3], double m[3], double z[3], double &mass) {
  for (int k = 0; k < 3; k++) q[k] = m[k] = z[k] = 0.0;
  switch (gas) {
    case CCS_GAS_HE: m[0] = 4.0026; mass = m[0]; break;
    case CCS_GAS_AR: m[0] = 39.948; mass = m[0]; break;
    case CCS_GAS_CO2_1SITE: m[0] = 44.0098; mass = m[0]; break;
    case CCS_GAS_N2:
      z[0] = 0.5488; z[1] = -0.5488; q[0] = q[1] = -0.4825; q[2] = 0.965;
      m[0] = m[1] = 14.007; mass = m[0] + m[1];
      break;
    default:  // CO2
      z[0] = -1.149; z[2] = 1.149; q[0] = q[2] = -0.3256; q[1] = 0.6512;
      m[0] = m[2] = 15.999; m[1] = 12.011; mass = m[0] + m[1] + m[2];
      break;
  }
}

// Speed sampler table of System::velGenerator (System.cpp:1523-1555): the
// same running sums in the same order, so a binary search for the first
// S[k] >= u returns the speed the reference's linear scan returns.
void vel_table(double m_amu, double T, std::vector<double> &V, std::vector<double> &S) {
  const double AMU_TO_KG = 1.66053904E-27, KB = 1.38064E-23, ANG_TO_M = 1.0E-10, FS_TO_S = 1.0E-15;
  auto distr = [&](double v) {
    double m = m_amu * AMU_TO_KG;
    v = v * ANG_TO_M / FS_TO_S;
    return std::pow(v, 5.0) * std::pow((m / (2.0 * KB * T)), 3.0) *
           std::exp(-(m * std::pow(v, 2.0)) / (2.0 * KB * T));
  };
  V.clear(); S.clear();
  double v = 0.0, dv = 1.0E-5, s = distr(v);
  V.push_back(v); S.push_back(s);
  // until the CDF covers u = 1, or the density underflows (then the last entry
  // answers every larger u; the reference would scan forever there)
  while (s < 1.0 && V.size() < 4000000) {
    v += dv;
    const double pv = distr(v);
    s += pv;
    V.push_back(v); S.push_back(s);
    if (pv == 0.0 && v * ANG_TO_M / FS_TO_S > 1.0e3) break;
  }
}

template <typename T, int GAS, bool HASQ> KernelFn resume_ptr(int nt) {
  return nt == 32 ? resume_kernel<T, GAS, HASQ, 32, false>
                  : nt == 64 ? resume_kernel<T, GAS, HASQ, 64, false> : resume_kernel<T, GAS, HASQ, 128, false>;
}
using ForceFn = void (*)(KParams, int, size_t, const double *, double *, double *, uint32_t *);

template <typename T, int G, int GAS, bool HASQ> KernelFn traj_ptr() { return traj_kernel<T, G, GAS, HASQ, false>; }
template <typename T, int G, int GAS, bool HASQ> ForceFn force_ptr() {
  return force_points_kernel<T, G, GAS, HASQ>;
}

int g_index(int G) { int i = 0; while ((1 << i) < G) i++; return i; }

template <typename T, int GAS, bool HASQ> KernelFn pick_traj_g(int gi) {
  switch (gi) {
    case 0: return traj_ptr<T, 1, GAS, HASQ>();
    case 2: return traj_ptr<T, 4, GAS, HASQ>();
    case 3: return traj_ptr<T, 8, GAS, HASQ>();
    case 4: return traj_ptr<T, 16, GAS, HASQ>();
    default: return traj_ptr<T, 32, GAS, HASQ>();
  }
}
template <typename T, int GAS, bool HASQ> ForceFn pick_force_g(int gi) {
  switch (gi) {
    case 0: return force_ptr<T, 1, GAS, HASQ>();
    case 3: return force_ptr<T, 8, GAS, HASQ>();
    default: return force_ptr<T, 32, GAS, HASQ>();
  }
}
template <typename T> KernelFn pick_traj_t(int gas, bool hasq, int gi) {
  if (gas == GAS_ATOM) return hasq ? pick_traj_g<T, GAS_ATOM, true>(gi) : pick_traj_g<T, GAS_ATOM, false>(gi);
  if (gas == GAS_N2) return hasq ? pick_traj_g<T, GAS_N2, true>(gi) : pick_traj_g<T, GAS_N2, false>(gi);
  return hasq ? pick_traj_g<T, GAS_CO2, true>(gi) : pick_traj_g<T, GAS_CO2, false>(gi);
}
template <typename T> ForceFn pick_force_t(int gas, bool hasq, int gi) {
  if (gas == GAS_ATOM) return hasq ? pick_force_g<T, GAS_ATOM, true>(gi) : pick_force_g<T, GAS_ATOM, false>(gi);
  if (gas == GAS_N2) return hasq ? pick_force_g<T, GAS_N2, true>(gi) : pick_force_g<T, GAS_N2, false>(gi);
  return hasq ? pick_force_g<T, GAS_CO2, true>(gi) : pick_force_g<T, GAS_CO2, false>(gi);
}
KernelFn pick_traj(const ccs_ctx *c, int G) {
  const int gas = gas_kind(c->p.gas);
  const bool hasq = c->coul_on || c->dip_on;
  return c->p.precision == CCS_PREC_FP64 ? pick_traj_t<double>(gas, hasq, g_index(G))
                                         : pick_traj_t<float>(gas, hasq, g_index(G));
}
// threads per trajectory in the warp pass
// Threads per warp-pass trajectory: the configured value, else 32 for
// molecules on targets whose candidate lists fit the smallest list (one warp
// per trajectory, no cross-warp reduction: measured 1.90 against 1.98 s per
// 3e5 trajectories on the 1231-atom N2 globule), else RBLOCK (64).
int resume_threads(const ccs_ctx *c) {
  const int b = c->p.resume_block;
  if (b == 32 || b == 64 || b == 128) return b;
  if (is_molecule(c->p.gas) && c->p.precision != CCS_PREC_FP64 && c->lcap <= LCAP && !c->allpairs) return 32;
  return RBLOCK;
}

KernelFn pick_resume(const ccs_ctx *c) {
  const int gas = gas_kind(c->p.gas);
  const bool hasq = c->coul_on || c->dip_on;
  const int nt = resume_threads(c);
  if (c->p.precision == CCS_PREC_FP64) {
    if (gas == GAS_ATOM) return hasq ? resume_ptr<double, GAS_ATOM, true>(nt) : resume_ptr<double, GAS_ATOM, false>(nt);
    if (gas == GAS_N2) return hasq ? resume_ptr<double, GAS_N2, true>(nt) : resume_ptr<double, GAS_N2, false>(nt);
    return hasq ? resume_ptr<double, GAS_CO2, true>(nt) : resume_ptr<double, GAS_CO2, false>(nt);
  }
  if (gas == GAS_ATOM) return hasq ? resume_ptr<float, GAS_ATOM, true>(nt) : resume_ptr<float, GAS_ATOM, false>(nt);
  if (gas == GAS_N2) return hasq ? resume_ptr<float, GAS_N2, true>(nt) : resume_ptr<float, GAS_N2, false>(nt);
  return hasq ? resume_ptr<float, GAS_CO2, true>(nt) : resume_ptr<float, GAS_CO2, false>(nt);
}
ForceFn pick_force(const ccs_ctx *c, int G) {
  const int gas = gas_kind(c->p.gas);
  const bool hasq = c->coul_on || c->dip_on;
  return c->p.precision == CCS_PREC_FP64 ? pick_force_t<double>(gas, hasq, g_index(G))
                                         : pick_force_t<float>(gas, hasq, g_index(G));
}

}  // namespace

KParams ccs_internal::base_params(const ccs_ctx *c) {
  const ccs_params &p = c->p;
  KParams k;
  std::memset(&k, 0, sizeof k);
  k.xyzq32 = c->d_xyzq32; k.ab32 = c->d_ab32; k.abc32 = c->d_abc32 ? c->d_abc32 : c->d_ab32;
  k.xyzq64 = c->d_xyzq64; k.ab64 = c->d_ab64; k.abc64 = c->d_abc64 ? c->d_abc64 : c->d_ab64;
  k.cell_start = c->d_cell_start;
  k.nx = c->nx; k.ny = c->ny; k.nz = c->nz; k.natoms = c->natoms;
  k.ox = c->origin[0]; k.oy = c->origin[1]; k.oz = c->origin[2];
  k.h = c->h; k.inv_h = 1.0 / c->h;
  for (int d = 0; d < 3; d++) { k.bb_lo[d] = c->bb_lo[d]; k.bb_hi[d] = c->bb_hi[d]; }
  k.reach = c->reach;
  k.lcap = c->lcap;
  k.allpairs = c->allpairs;
  k.coul_on = c->coul_on;
  k.dip_on = c->dip_on;
  double gq[3], gm[3], gz[3], gmass;
  gas_table(p.gas, gq, gm, gz, gmass);
  for (int s = 0; s < 3; s++) { k.q_site[s] = gq[s]; k.gas_m[s] = gm[s]; k.gas_z[s] = gz[s]; }
  k.gas_mass = gmass;
  if (c->allpairs) {
    k.rlj2 = INFINITY; k.rc2 = INFINITY;
    k.rc6inv = k.rc12inv = k.rc3inv = k.c1 = k.c2 = 0.0;
  } else {
    const double rl = p.lj_cutoff, rc = p.coul_cutoff;
    k.rlj2 = rl * rl;
    k.rc2 = rc * rc;
    k.rc6inv = 1.0 / std::pow(rl, 6);
    k.rc12inv = k.rc6inv * k.rc6inv;
    k.rc3inv = 1.0 / std::pow(rc, 3);
    k.c1 = 1.5 / rc;
    k.c2 = 0.5 / std::pow(rc, 3);
  }
  k.alpha = p.alpha;
  // reference grid: cells of lj_cutoff + skin over the box (LinkedCell.cpp:48-90)
  const double rh = p.lj_cutoff + p.skin;
  k.ref_h = rh;
  k.ref_inv_h = 1.0 / rh;
  k.ref_nx = (int)std::ceil(2.0 * p.a / rh);
  k.ref_ny = (int)std::ceil(2.0 * p.b / rh);
  k.ref_nz = (int)std::ceil(2.0 * p.c / rh);
  k.ref_corner[0] = -0.5 * (k.ref_nx * rh);
  k.ref_corner[1] = -0.5 * (k.ref_ny * rh);
  k.ref_corner[2] = -0.5 * (k.ref_nz * rh);
  k.ref_check = c->allpairs ? 0 : 1;
  k.gas = p.gas;
  k.dt = p.dt; k.mu = p.mu; k.temperature = p.temperature; k.gas_inertia = p.gas_inertia;
  k.d_bond = p.d_bond; k.a = p.a; k.b = p.b; k.c = p.c; k.bmax = p.bmax;
  k.lx = p.lx; k.ly = p.ly; k.lz = p.lz;
  k.inv_a = 1.0 / p.a; k.inv_b = 1.0 / p.b; k.inv_c = 1.0 / p.c;
  k.etol = p.gas == CCS_GAS_N2 ? 1.0 : p.gas == CCS_GAS_CO2 ? 20.0 : 0.5;
  {
    // the moving pair: atoms integrate the reduced mass; N2 the two N; CO2 the two O
    const double m1 = is_molecule(p.gas) ? gm[0] : p.mu;
    const double m2 = is_molecule(p.gas) ? (p.gas == CCS_GAS_CO2 ? gm[2] : gm[1]) : p.mu;
    const double kc = KCALMOLANGAMU_TO_ANGFS2;
    k.half_kconv_over_m1 = 0.5 * kc / m1;
    k.half_kconv_over_m2 = 0.5 * kc / m2;
    k.inv_m1 = 1.0 / m1;
    k.inv_m2 = 1.0 / m2;
    k.mu12 = m1 * m2 / (m1 + m2);
    k.mu12_over_m1 = k.mu12 / m1;
    k.mu12_over_m2 = k.mu12 / m2;
  }
  k.quirks = p.quirks;
  k.max_steps = p.max_steps_per_try ? p.max_steps_per_try : 2000000u;
  k.vtab_v = c->d_vtab_v; k.vtab_s = c->d_vtab_s; k.vtab_n = c->vtab_n;
  k.work = c->d_work;
  k.stats = c->d_work + 1;
  k.error = c->d_error;
  return k;
}

namespace {

// Park-buffer capacity of a run of n trajectories: every trajectory up to
// 131,072, half of them beyond (a full buffer keeps the rest in their lanes)
size_t park_capacity(size_t n) { return std::min<size_t>(n, std::max<size_t>(131072, n / 2)); }

// Speculative-retry buffers for up to cap records (the park capacity) and
// the counters d_work[11] (records), d_work[12] (next speculative try) and
// d_work[13] (parked trajectories still running).
int setup_spec(ccs_ctx *c, KParams &k, size_t cap, cudaStream_t s) {
  // records come only from warp passes with at most 2 parked trajectories per
  // CTA slot (a few thousand); an overflow falls back to tries in sequence
  cap = std::min<size_t>(cap, 65536);
  if (cap > c->spec_cap) {
    dfree(c->d_spec_rec); dfree(c->d_spec_out);
    c->spec_cap = 0;
    CK(cudaMalloc(&c->d_spec_rec, cap * sizeof(SpecRec)));
    CK(cudaMalloc(&c->d_spec_out, cap * SPEC_SLOTS * sizeof(SpecOut)));
    c->spec_cap = cap;
  }
  k.spec_rec = c->d_spec_rec;
  k.spec_out = c->d_spec_out;
  k.spec_count = c->d_work + 11;
  k.spec_next = c->d_work + 12;
  k.park_active = c->d_work + 13;
  k.spec_cap = cap;
  k.spec_phase = 0;
  k.spec_from = std::max(SPEC_FROM_MIN, c->p.spec_tries > 0 ? c->p.spec_tries : 2);
  if (c->p.spec_tries < 0) k.spec_rec = nullptr;  // speculation off
  CK(cudaMemsetAsync(c->d_work + 11, 0, 3 * sizeof(unsigned long long), s));
  // every record unpublished (phase-0 CTAs claim only published records' tries)
  if (k.spec_rec) CK(cudaMemsetAsync(c->d_spec_rec, 0, cap * sizeof(SpecRec), s));
  return CCS_OK;
}

// The warp pass: parked trajectories (phase 0), the speculative tries of
// those that failed spec_from tries there (phase 1), their verdicts.
template <bool BATCH>
int launch_warp_pass(ccs_ctx *c, KernelFn rfn, int rnt, KParams k, cudaStream_t s) {
  int rper_sm = 0;
  // the candidate list (and with the learned field the near-part list)
  const size_t dyn = (size_t)(k.lcap + (k.field.on ? LCAP : 0)) * sizeof(int);
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&rper_sm, (const void *)rfn, rnt, dyn));
  const unsigned rgrid = (unsigned)((size_t)std::max(rper_sm, 1) * c->sm_count);
  k.spec_max_parked = 2ull * rgrid;  // measured: 448 parked of 3e5 (60 atoms, He) 1.7x faster, 52,241 (1231 atoms, N2) slower
  rfn<<<rgrid, rnt, dyn, s>>>(k, c->d_kparams);
  CK(cudaGetLastError());
  if (k.spec_rec) {
    k.spec_phase = 1;
    rfn<<<rgrid, rnt, dyn, s>>>(k, c->d_kparams);
    CK(cudaGetLastError());
    spec_resolve_kernel<BATCH><<<(unsigned)((k.spec_cap + 255) / 256), 256, 0, s>>>(k);
    CK(cudaGetLastError());
  }
  return CCS_OK;
}

int ensure_run_buffers(ccs_ctx *c, size_t n, bool need_rnd) {
  if (need_rnd && n > c->rnd_cap) {
    dfree(c->d_rnd);
    CK(cudaMalloc(&c->d_rnd, 9 * n * sizeof(double)));
    CK(cudaMemsetAsync(c->d_rnd, 0, 9 * n * sizeof(double), c->stream));
    c->rnd_cap = n;
  }
  if (n > c->out_cap) {
    dfree(c->d_status); dfree(c->d_omc); dfree(c->d_steps); dfree(c->d_visits);
    CK(cudaMalloc(&c->d_status, n));
    CK(cudaMalloc(&c->d_omc, n * sizeof(double)));
    CK(cudaMalloc(&c->d_steps, n * sizeof(uint32_t)));
    CK(cudaMalloc(&c->d_visits, n * sizeof(uint32_t)));
    c->out_cap = n;
  }
  return CCS_OK;
}

// The watchdog deadline of a run: now + watchdog_s, set on the device at the
// head of the run (stream-ordered, so the host never waits for the clock).
int arm_deadline(ccs_ctx *c, unsigned long long *word, cudaStream_t s) {
  const double wd = c->p.watchdog_s > 0 ? c->p.watchdog_s : 600.0;
  arm_watchdog<<<1, 1, 0, s>>>(word, (unsigned long long)(wd * 1e9));
  CK(cudaGetLastError());
  return CCS_OK;
}

// Full asynchronous run on device buffers (no host synchronisation).
int run_device(ccs_ctx *c, size_t n, const double *d_rnd, size_t stride, int8_t *d_status,
               double *d_omc, uint32_t *d_steps, uint32_t *d_visits, cudaStream_t s, int G,
               int block) {
  KParams k = base_params(c);
  k.rnd = d_rnd;
  k.rnd_stride = stride;
  k.ntraj = n;
  k.status = d_status;
  k.omc = d_omc;
  k.steps = d_steps;
  k.visits = d_visits;
  int rc = CCS_OK;
  field_kparams(c, k);  // the learned field, when on
  const bool surr = k.field.on != 0;
  const bool hasq = c->coul_on || c->dip_on;
  KernelFn fn = surr ? pick_traj_field(gas_kind(c->p.gas), hasq, G) : pick_traj(c, G);
  const int dyn = surr ? TC_SMEM_BYTES : 0;  // the MLP tiles of the lane pass
  if (surr) CK(cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)fn, block, dyn));
  if (per_sm < 1) per_sm = 1;
  size_t grid = (size_t)per_sm * c->sm_count;
  const size_t max_useful = (n + block - 1) / block;  // one trajectory per lane
  if (grid > max_useful) grid = std::max<size_t>(1, max_useful);
  k.deadline = c->d_work + 8;
  // longest-expected-first processing order (a radix sort of the length keys)
  if (n > 1 && c->p.schedule == 1) {
    if (n > c->order_cap) {
      dfree(c->d_key); dfree(c->d_key2); dfree(c->d_idx); dfree(c->d_idx2); dfree(c->d_sort_tmp);
      c->order_cap = 0;
      CK(cudaMalloc(&c->d_key, n * sizeof(float)));
      CK(cudaMalloc(&c->d_key2, n * sizeof(float)));
      CK(cudaMalloc(&c->d_idx, n * sizeof(uint32_t)));
      CK(cudaMalloc(&c->d_idx2, n * sizeof(uint32_t)));
      size_t tmp = 0;
      CK(cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp, c->d_key, c->d_key2, c->d_idx, c->d_idx2, (int)n));
      CK(cudaMalloc(&c->d_sort_tmp, tmp));
      c->sort_tmp_bytes = tmp;
      c->order_cap = n;
    }
    order_key_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(k, c->d_key, c->d_idx);
    CK(cudaGetLastError());
    size_t tmp = c->sort_tmp_bytes;
    CK(cub::DeviceRadixSort::SortPairsDescending(c->d_sort_tmp, tmp, c->d_key, c->d_key2, c->d_idx, c->d_idx2,
                                                 (int)n, 0, 32, s));
    k.order = c->d_idx2;
  }
  // parking buffer for trajectories that outlast park_steps in the lane pass
  const size_t state_bytes = c->p.precision == CCS_PREC_FP64 ? sizeof(LaneState<double>) : sizeof(LaneState<float>);
  // room for half the trajectories: a trajectory that finds the buffer full
  // keeps running in its lane at the lane pass's per-step cost (measured: a
  // park threshold that wanted 75,000+ slots of 75,000 tripled the run)
  const size_t cap = park_capacity(n);
  if (cap * state_bytes > c->park_bytes) {
    dfree(c->d_park);
    c->park_bytes = 0;
    CK(cudaMalloc(&c->d_park, cap * state_bytes));
    c->park_bytes = cap * state_bytes;
  }
  k.park = c->d_park;
  k.park_cap = cap;
  k.park_steps = c->p.park_steps ? c->p.park_steps : 2048u;
  k.park_drained = c->p.schedule == 2;
  k.park_count = c->d_work + 9;
  k.park_next = c->d_work + 10;
  rc = setup_spec(c, k, cap, s);
  if (rc) return rc;
  // d_work: [0] work counter, [1..7] statistics, [8] watchdog deadline, [9] parked, [10] resumed,
  // [11] speculative records, [12] next speculative try
  CK(cudaMemsetAsync(c->d_work, 0, 8 * sizeof(unsigned long long), s));
  CK(cudaMemsetAsync(c->d_work + 9, 0, 2 * sizeof(unsigned long long), s));
  CK(cudaMemsetAsync(c->d_error, 0, sizeof(int), s));
  rc = arm_deadline(c, c->d_work + 8, s);
  if (rc) return rc;
  c->run_work = c->d_work;
  c->run_error = c->d_error;
  c->h_kparams = k;
  CK(cudaMemcpyAsync(c->d_kparams, &c->h_kparams, sizeof(KParams), cudaMemcpyHostToDevice, s));
  CK(cudaEventRecord(c->ev[5], s));
  fn<<<(unsigned)grid, block, dyn, s>>>(k, c->d_kparams);
  CK(cudaGetLastError());
  CK(cudaEventRecord(c->ev[6], s));
  // warp pass over the parked trajectories (exits at once when none were parked)
  KernelFn rfn = surr ? pick_resume_field(gas_kind(c->p.gas), hasq, resume_threads(c)) : pick_resume(c);
  rc = launch_warp_pass<false>(c, rfn, resume_threads(c), k, s);
  if (rc) return rc;
  CK(cudaEventRecord(c->ev[7], s));
  c->last.grid_size = (int32_t)grid;
  c->last.block_size = block;
  c->last.lanes_per_traj = G;
  return CCS_OK;
}

int read_stats(ccs_ctx *c, ccs_stats *st, size_t n) {
  unsigned long long h[12];  // work[1..12]: statistics, deadline, park and speculation counters
  int herr = 0;
  unsigned long long *work = c->run_work ? c->run_work : c->d_work;
  int *error = c->run_error ? c->run_error : c->d_error;
  {
    float a = 0, b = 0;
    CK(cudaEventSynchronize(c->ev[7]));
    CK(cudaEventElapsedTime(&a, c->ev[5], c->ev[6]));
    CK(cudaEventElapsedTime(&b, c->ev[6], c->ev[7]));
    c->last.lane_ms = a;
    c->last.warp_ms = b;
  }
  CK(cudaMemcpyAsync(h, work + 1, sizeof h, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(&herr, error, sizeof herr, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->last.ntraj = n;
  c->last.nfree = h[0]; c->last.nscatter = h[1]; c->last.nlost = h[2]; c->last.ncapped = h[3];
  c->last.steps = h[4]; c->last.visits = h[5]; c->last.parked = h[6];
  c->last.speculated = work == c->d_work ? (int32_t)std::min<unsigned long long>(h[10], c->spec_cap) : 0;
  if (st) *st = c->last;
  if (herr == 2) return fail(c, CCS_ERR_CUDA, "a tensor-core stage of the learned field did not complete");
  if (herr) return fail(c, CCS_ERR_TIMEOUT, "device watchdog expired after %.0f s",
                        c->p.watchdog_s > 0 ? c->p.watchdog_s : 600.0);
  return CCS_OK;
}

// Autotuner: times each lanes-per-trajectory choice on a slice of the run and
// keeps the fastest (trajectories are independent, so a slice is a fair sample).
int autotune(ccs_ctx *c, size_t n, size_t stride, int block) {
  if (c->p.lanes_per_traj > 0) { c->tuned_G = c->p.lanes_per_traj; c->tuned_block = block; return CCS_OK; }
  if (c->tuned_G) return CCS_OK;
  const int cand[4] = {1, 8, 16, 32};
  size_t slice = std::min<size_t>(n, (size_t)c->sm_count * 256);
  float best = 1e30f;
  int bestG = 32;
  for (int G : cand) {
    for (int rep = 0; rep < 2; rep++) {  // first pass warms caches and code
      CK(cudaEventRecord(c->ev[8], c->stream));
      int rc = run_device(c, slice, c->d_rnd, stride, c->d_status, c->d_omc, nullptr, nullptr,
                          c->stream, G, block);
      if (rc) return rc;
      CK(cudaEventRecord(c->ev[9], c->stream));
      CK(cudaEventSynchronize(c->ev[9]));
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, c->ev[8], c->ev[9]));
      if (rep == 1 && ms < best) { best = ms; bestG = G; }
    }
  }
  c->tuned_G = bestG;
  c->tuned_block = block;
  return CCS_OK;
}


// ---------------------------------------------------------------------------
// Batched ions: one launch of each pass over the trajectories of many ions.
// Every ion keeps its own context (parameters, target tables, cell grid); the
// kernels pick the ion's parameters per trajectory from a device array.
template <typename T, int G, int GAS, bool HASQ> KernelFn traj_batch_ptr() {
  return traj_kernel<T, G, GAS, HASQ, true>;
}
template <typename T, int GAS, bool HASQ> KernelFn pick_traj_batch_g(int G) {
  return G <= 8 ? traj_batch_ptr<T, 8, GAS, HASQ>()
                : G == 16 ? traj_batch_ptr<T, 16, GAS, HASQ>() : traj_batch_ptr<T, 32, GAS, HASQ>();
}
template <typename T> KernelFn pick_traj_batch_t(int gas, bool hasq, int G) {
  if (gas == GAS_ATOM) return hasq ? pick_traj_batch_g<T, GAS_ATOM, true>(G) : pick_traj_batch_g<T, GAS_ATOM, false>(G);
  if (gas == GAS_N2) return hasq ? pick_traj_batch_g<T, GAS_N2, true>(G) : pick_traj_batch_g<T, GAS_N2, false>(G);
  return hasq ? pick_traj_batch_g<T, GAS_CO2, true>(G) : pick_traj_batch_g<T, GAS_CO2, false>(G);
}
template <typename T> KernelFn pick_resume_batch_t(int gas, bool hasq) {
  if (gas == GAS_ATOM)
    return hasq ? resume_kernel<T, GAS_ATOM, true, RBLOCK, true> : resume_kernel<T, GAS_ATOM, false, RBLOCK, true>;
  if (gas == GAS_N2)
    return hasq ? resume_kernel<T, GAS_N2, true, RBLOCK, true> : resume_kernel<T, GAS_N2, false, RBLOCK, true>;
  return hasq ? resume_kernel<T, GAS_CO2, true, RBLOCK, true> : resume_kernel<T, GAS_CO2, false, RBLOCK, true>;
}
int batch_lanes(int G) { return G <= 8 ? 8 : G <= 16 ? 16 : 32; }

// Both passes over trajectories [0, m[i]) of every ion i, whose random rows
// and outputs start at column off[i] of the lead context's buffers (row
// stride `stride`).  Asynchronous on the lead's stream; events ev[5..7].
int run_batch_device(ccs_ctx *lead, ccs_ctx *const *ions, size_t nions, const size_t *m, const size_t *off,
                     size_t stride, bool want_steps, bool want_visits, int G) {
  ccs_ctx *c = lead;  // error reports go to the lead context
  cudaStream_t s = lead->stream;
  std::vector<KParams> kv(nions);
  std::vector<unsigned long long> st(nions + 1);
  unsigned long long total = 0;
  bool hasq = false;
  for (size_t i = 0; i < nions; i++) {
    const ccs_ctx *ci = ions[i];
    KParams k = base_params(ci);
    k.rnd = lead->d_rnd + off[i];
    k.rnd_stride = stride;
    k.ntraj = m[i];
    k.status = lead->d_status + off[i];
    k.omc = lead->d_omc + off[i];
    k.steps = want_steps ? lead->d_steps + off[i] : nullptr;
    k.visits = want_visits ? lead->d_visits + off[i] : nullptr;
    k.order = nullptr;
    kv[i] = k;
    st[i] = total;
    total += m[i];
    hasq |= ci->coul_on || ci->dip_on;
  }
  st[nions] = total;
  if (total == 0) return CCS_OK;
  if (nions > lead->bkp_cap) {
    dfree(lead->d_bkp); dfree(lead->d_bstart);
    lead->bkp_cap = 0;
    CK(cudaMalloc(&lead->d_bkp, nions * sizeof(KParams)));
    CK(cudaMalloc(&lead->d_bstart, (nions + 1) * sizeof(unsigned long long)));
    lead->bkp_cap = nions;
  }
  for (size_t i = 0; i < nions; i++) kv[i].deadline = lead->d_work + 8;
  CK(to_dev(lead, lead->d_bkp, kv.data(), nions * sizeof(KParams)));
  CK(to_dev(lead, lead->d_bstart, st.data(), (nions + 1) * sizeof(unsigned long long)));
  KParams k = base_params(lead);
  for (size_t i = 0; i < nions; i++) k.lcap = std::max(k.lcap, ions[i]->lcap);  // one list size per launch
  k.ntraj = total;
  k.ions = lead->d_bkp;
  k.ion_start = lead->d_bstart;
  k.nions = (int)nions;
  int rc = CCS_OK;
  k.deadline = lead->d_work + 8;
  const size_t state_bytes =
      lead->p.precision == CCS_PREC_FP64 ? sizeof(LaneState<double>) : sizeof(LaneState<float>);
  const size_t cap = park_capacity(total);
  if (cap * state_bytes > lead->park_bytes) {
    dfree(lead->d_park);
    lead->park_bytes = 0;
    CK(cudaMalloc(&lead->d_park, cap * state_bytes));
    lead->park_bytes = cap * state_bytes;
  }
  k.park = lead->d_park;
  k.park_cap = cap;
  k.park_steps = lead->p.park_steps ? lead->p.park_steps : 2048u;
  k.park_drained = lead->p.schedule == 2;
  k.park_count = lead->d_work + 9;
  k.park_next = lead->d_work + 10;
  rc = setup_spec(lead, k, cap, s);
  if (rc) return rc;
  CK(cudaMemsetAsync(lead->d_work, 0, 8 * sizeof(unsigned long long), s));
  CK(cudaMemsetAsync(lead->d_work + 9, 0, 2 * sizeof(unsigned long long), s));
  CK(cudaMemsetAsync(lead->d_error, 0, sizeof(int), s));
  rc = arm_deadline(lead, lead->d_work + 8, s);
  if (rc) return rc;
  lead->run_work = lead->d_work;
  lead->run_error = lead->d_error;
  lead->h_kparams = k;
  CK(cudaMemcpyAsync(lead->d_kparams, &lead->h_kparams, sizeof(KParams), cudaMemcpyHostToDevice, s));
  const int gas = gas_kind(lead->p.gas);
  const bool fp64 = lead->p.precision == CCS_PREC_FP64;
  const int Gb = batch_lanes(G);
  KernelFn fn = fp64 ? pick_traj_batch_t<double>(gas, hasq, Gb) : pick_traj_batch_t<float>(gas, hasq, Gb);
  KernelFn rfn = fp64 ? pick_resume_batch_t<double>(gas, hasq) : pick_resume_batch_t<float>(gas, hasq);
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)fn, BLOCK, 0));
  size_t grid = (size_t)std::max(per_sm, 1) * lead->sm_count;
  grid = std::min(grid, std::max<size_t>(1, (total + BLOCK - 1) / BLOCK));
  CK(cudaEventRecord(lead->ev[5], s));
  fn<<<(unsigned)grid, BLOCK, 0, s>>>(k, lead->d_kparams);
  CK(cudaGetLastError());
  CK(cudaEventRecord(lead->ev[6], s));
  rc = launch_warp_pass<true>(lead, rfn, RBLOCK, k, s);
  if (rc) return rc;
  CK(cudaEventRecord(lead->ev[7], s));
  lead->last.grid_size = (int32_t)grid;
  lead->last.block_size = BLOCK;
  lead->last.lanes_per_traj = Gb;
  return CCS_OK;
}

// Lanes per force evaluation for a batch: the lead's setting, else the
// fastest of 8, 16 and 32 on a sub-batch of every ion's first trajectories.
int autotune_batch(ccs_ctx *lead, ccs_ctx *const *ions, size_t nions, const size_t *n, const size_t *off,
                   size_t stride, int &G) {
  ccs_ctx *c = lead;  // error reports go to the lead context
  if (lead->p.lanes_per_traj > 0) { G = batch_lanes(lead->p.lanes_per_traj); return CCS_OK; }
  size_t total = 0;
  for (size_t i = 0; i < nions; i++) total += n[i];
  if (lead->batch_G && lead->batch_nions == nions && lead->batch_total == total) {
    G = lead->batch_G;  // the same batch shape as last time
    return CCS_OK;
  }
  const size_t per = std::max<size_t>(1, ((size_t)lead->sm_count * 256) / std::max<size_t>(1, nions));
  std::vector<size_t> m(nions);
  for (size_t i = 0; i < nions; i++) m[i] = std::min(n[i], per);
  float best = 1e30f;
  G = 32;
  for (int cand : {8, 16, 32}) {
    for (int rep = 0; rep < 2; rep++) {  // first pass warms caches and code
      CK(cudaEventRecord(lead->ev[8], lead->stream));
      int rc = run_batch_device(lead, ions, nions, m.data(), off, stride, false, false, cand);
      if (rc) return rc;
      CK(cudaEventRecord(lead->ev[9], lead->stream));
      CK(cudaEventSynchronize(lead->ev[9]));
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, lead->ev[8], lead->ev[9]));
      if (rep == 1 && ms < best) { best = ms; G = cand; }
    }
  }
  lead->batch_G = G;
  lead->batch_nions = nions;
  lead->batch_total = total;
  return CCS_OK;
}
}  // namespace

// ===========================================================================
extern "C" {

int ccs_version(int32_t *abi) {
  if (abi) *abi = CCS_ABI_VERSION;
  return CCS_OK;
}

void ccs_params_default(ccs_params *p) {
  if (!p) return;
  std::memset(p, 0, sizeof *p);
  p->gas = CCS_GAS_HE;
  p->force_type = 4;
  p->dt = 10.0;           // Constants.h:72
  p->temperature = 298.0; // Constants.h:73
  p->lj_cutoff = 12.0;    // Constants.h:75
  p->coul_cutoff = 25.0;  // Constants.h:77
  p->skin = 0.01;         // Constants.h:74
  p->precision = CCS_PREC_FP32;
  p->watchdog_s = 600.0;
}

int ccs_create(ccs_ctx **out, int device) {
  if (!out) return CCS_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return CCS_ERR_NODEVICE; }
  if (device < 0 || device >= ndev) return CCS_ERR_INVALID;
  ccs_ctx *c = new (std::nothrow) ccs_ctx();
  if (!c) return CCS_ERR_NOMEM;
  ccs_params_default(&c->p);
  c->device = device;
  auto bail = [&](int code) { ccs_destroy(c); return code; };
  if (cudaSetDevice(device) != cudaSuccess) return bail(CCS_ERR_CUDA);
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return bail(CCS_ERR_CUDA);
  if (prop.major < 10) return bail(CCS_ERR_NODEVICE);  // built for sm_100a only
  c->sm_count = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(CCS_ERR_CUDA);
  for (auto &e : c->ev)
    if (cudaEventCreate(&e) != cudaSuccess) return bail(CCS_ERR_CUDA);
  if (cudaMalloc(&c->d_work, 14 * sizeof(unsigned long long)) != cudaSuccess) return bail(CCS_ERR_NOMEM);
  if (cudaMalloc(&c->d_error, sizeof(int)) != cudaSuccess) return bail(CCS_ERR_NOMEM);
  if (cudaMalloc(&c->d_kparams, sizeof(KParams)) != cudaSuccess) return bail(CCS_ERR_NOMEM);
  *out = c;
  return CCS_OK;
}

void ccs_destroy(ccs_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  free_target(c);
  dfree(c->d_vtab_v); dfree(c->d_vtab_s);
  dfree(c->d_work); dfree(c->d_error); dfree(c->d_rnd); dfree(c->d_kparams); dfree(c->d_park);
  dfree(c->d_bkp); dfree(c->d_bstart);
  dfree(c->d_spec_rec); dfree(c->d_spec_out);
  dfree(c->d_key); dfree(c->d_key2); dfree(c->d_idx); dfree(c->d_idx2); dfree(c->d_sort_tmp);
  dfree(c->d_status); dfree(c->d_omc); dfree(c->d_steps); dfree(c->d_visits);
  for (auto &e : c->ev)
    if (e) cudaEventDestroy(e);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

int ccs_set_params(ccs_ctx *c, const ccs_params *p) {
  if (!c || !p) return CCS_ERR_INVALID;
  if (p->gas < 1 || p->gas > 5) return fail(c, CCS_ERR_INVALID, "gas must be 1..5");
  if (p->force_type < 1 || p->force_type > 6) return fail(c, CCS_ERR_INVALID, "force_type must be 1..6");
  if (!is_molecule(p->gas) && p->force_type > 4)
    return fail(c, CCS_ERR_INVALID, "atomic gases use force_type 1..4");
  if (!(p->dt > 0) || !(p->temperature > 0) || !(p->mu > 0) || !(p->bmax > 0) || !(p->a > 0) ||
      !(p->b > 0) || !(p->c > 0) || !(p->lx > 0) || !(p->ly > 0) || !(p->lz > 0))
    return fail(c, CCS_ERR_INVALID, "dt, temperature, mu, a, b, c, bmax and box must be positive");
  if (!(p->lj_cutoff > 0) || !(p->coul_cutoff > 0))
    return fail(c, CCS_ERR_INVALID, "cutoffs must be positive");
  if (is_molecule(p->gas) && (!(p->gas_inertia > 0) || !(p->d_bond > 0)))
    return fail(c, CCS_ERR_INVALID, "molecular gases need gas_inertia and d_bond");
  if (p->precision != CCS_PREC_FP32 && p->precision != CCS_PREC_FP64)
    return fail(c, CCS_ERR_INVALID, "precision must be FP32 or FP64");
  const int G = p->lanes_per_traj;
  if (G != 0 && G != 1 && G != 4 && G != 8 && G != 16 && G != 32)
    return fail(c, CCS_ERR_INVALID, "lanes_per_traj must be 0, 1, 4, 8, 16 or 32");
  if (p->block_size != 0 && p->block_size != BLOCK)
    return fail(c, CCS_ERR_INVALID, "block_size must be 0 or %d", BLOCK);
  if (cudaSetDevice(c->device) != cudaSuccess) return fail(c, CCS_ERR_CUDA, "cudaSetDevice");
  const bool vel_changed = !c->have_params || c->p.mu != p->mu || c->p.temperature != p->temperature;
  c->p = *p;
  c->have_params = true;
  free_target(c);
  if (vel_changed) {
    std::vector<double> V, S;
    vel_table(p->mu, p->temperature, V, S);
    dfree(c->d_vtab_v); dfree(c->d_vtab_s);
    CK(cudaMalloc(&c->d_vtab_v, V.size() * sizeof(double)));
    CK(cudaMalloc(&c->d_vtab_s, S.size() * sizeof(double)));
    CK(to_dev(c, c->d_vtab_v, V.data(), V.size() * sizeof(double)));
    CK(to_dev(c, c->d_vtab_s, S.data(), S.size() * sizeof(double)));
    CK(cudaStreamSynchronize(c->stream));  // runs may launch on other streams
    c->vtab_n = (int)V.size();
  }
  return CCS_OK;
}

// Warp-pass candidate-list size: the most atoms that the column runs of a
// list sphere (radius reach + 2.5 A: the skin and a site's offset from the
// probe centre) can hold around one of up to 256 atoms spread through the
// target, plus an eighth, rounded up to 256, in [LCAP, LCAP_MAX].  A column
// run reaches at most a column diagonal beyond the sphere sideways, so an
// atom counts when (d_xy - h sqrt 2)_+^2 + d_z^2 <= R^2.  Steps with more
// candidates than the list holds flatten them chunk by chunk.
static int list_capacity(const ccs_ctx *c, const double *x, const double *y, const double *z,
                         const std::vector<int> &order, const std::vector<int> &start, const int *dims) {
  const size_t n = order.size();
  if (c->allpairs || n <= (size_t)ccs::LCAP) return ccs::LCAP;
  const double R = c->reach + 2.5, w = c->h * std::sqrt(2.0);
  const int reach_cells = (int)std::ceil((R + w) / c->h);
  const size_t samples = std::min<size_t>(256, n);
  int most = 0;
  for (size_t t = 0; t < samples; t++) {
    const int a = order[t * n / samples];
    const double ax = x[a], ay = y[a], az = z[a];
    int ci[3];
    const double v[3] = {ax, ay, az};
    for (int d = 0; d < 3; d++) ci[d] = std::min(dims[d] - 1, std::max(0, (int)std::floor((v[d] - c->origin[d]) / c->h)));
    int cnt = 0;
    for (int i = std::max(0, ci[0] - reach_cells); i <= std::min(dims[0] - 1, ci[0] + reach_cells); i++)
      for (int j = std::max(0, ci[1] - reach_cells); j <= std::min(dims[1] - 1, ci[1] + reach_cells); j++) {
        const size_t col = ((size_t)i * dims[1] + j) * dims[2];
        const int k0 = std::max(0, ci[2] - reach_cells), k1 = std::min(dims[2] - 1, ci[2] + reach_cells);
        for (int q = start[col + k0]; q < start[col + k1 + 1]; q++) {
          const int b = order[(size_t)q];
          const double dx = x[b] - ax, dy = y[b] - ay, dz = z[b] - az;
          const double e = std::max(0.0, std::sqrt(dx * dx + dy * dy) - w);
          cnt += e * e + dz * dz <= R * R;
        }
      }
    most = std::max(most, cnt);
  }
  const int want = (most + most / 8 + 255) / 256 * 256;
  return std::min(ccs::LCAP_MAX, std::max(ccs::LCAP, want));
}

int ccs_set_target(ccs_ctx *c, size_t n, const double *x, const double *y, const double *z,
                   const double *q, const double *eps, const double *sig, const double *eps_c,
                   const double *sig_c) {
  if (!c) return CCS_ERR_INVALID;
  if (!c->have_params) return fail(c, CCS_ERR_INVALID, "ccs_set_params must come first");
  if (n == 0 || !x || !y || !z || !q || !eps || !sig)
    return fail(c, CCS_ERR_INVALID, "target arrays missing or empty");
  if (n > (size_t)1 << 30) return fail(c, CCS_ERR_INVALID, "too many atoms");
  const ccs_params &p = c->p;
  if (p.gas == CCS_GAS_CO2 && (!eps_c || !sig_c))
    return fail(c, CCS_ERR_INVALID, "CO2 needs the carbon-site eps_c/sig_c");
  if (cudaSetDevice(c->device) != cudaSuccess) return fail(c, CCS_ERR_CUDA, "cudaSetDevice");
  free_target(c);
  const int ft = p.force_type;
  bool charged = false;
  for (size_t i = 0; i < n; i++) {
    if (!std::isfinite(x[i]) || !std::isfinite(y[i]) || !std::isfinite(z[i]) || !std::isfinite(q[i]))
      return fail(c, CCS_ERR_INVALID, "non-finite target coordinate or charge at atom %zu", i);
    charged |= q[i] != 0.0;
  }
  const bool mol = is_molecule(p.gas);
  c->charged = charged;
  c->allpairs = (ft == 1 || ft == 3 || ft == 5);
  c->coul_on = mol && ft >= 3 && charged;
  c->dip_on = charged && (mol ? (ft == 5 || ft == 6) : (ft == 3 || ft == 4));
  const bool hasq = c->coul_on || c->dip_on;
  c->reach = std::max(p.lj_cutoff, hasq ? p.coul_cutoff : 0.0);
  // engine cell edge: a fraction of the reach keeps the clipped columns close
  // to the cutoff sphere; the autotuner picks lanes per trajectory on top
  double h = p.cell_size > 0 ? p.cell_size : std::min(6.0, std::max(2.5, c->reach / 6.0));
  double lo[3] = {x[0], y[0], z[0]}, hi[3] = {x[0], y[0], z[0]};
  for (size_t i = 0; i < n; i++) {
    lo[0] = std::min(lo[0], x[i]); hi[0] = std::max(hi[0], x[i]);
    lo[1] = std::min(lo[1], y[i]); hi[1] = std::max(hi[1], y[i]);
    lo[2] = std::min(lo[2], z[i]); hi[2] = std::max(hi[2], z[i]);
  }
  int dims[3];
  for (int d = 0; d < 3; d++) {
    c->bb_lo[d] = lo[d];
    c->bb_hi[d] = hi[d];
    c->origin[d] = lo[d] - 1e-6;
    dims[d] = (int)std::floor((hi[d] - c->origin[d]) / h) + 1;
  }
  const long long ncell = (long long)dims[0] * dims[1] * dims[2];
  if (ncell > (1ll << 28)) return fail(c, CCS_ERR_INVALID, "engine grid too large; raise cell_size");
  c->nx = dims[0]; c->ny = dims[1]; c->nz = dims[2]; c->h = h; c->natoms = (int)n;
  // counting sort by flat cell (i*ny + j)*nz + k, stable in input order
  std::vector<int> cell(n), start((size_t)ncell + 1, 0), order(n);
  for (size_t i = 0; i < n; i++) {
    int ijk[3];
    const double v[3] = {x[i], y[i], z[i]};
    for (int d = 0; d < 3; d++)
      ijk[d] = std::min(dims[d] - 1, std::max(0, (int)std::floor((v[d] - c->origin[d]) / h)));
    cell[i] = (ijk[0] * c->ny + ijk[1]) * c->nz + ijk[2];
    start[(size_t)cell[i] + 1]++;
  }
  for (long long k = 0; k < ncell; k++) start[(size_t)k + 1] += start[(size_t)k];
  std::vector<int> fill(start.begin(), start.end() - 1);
  for (size_t i = 0; i < n; i++) order[(size_t)fill[(size_t)cell[i]]++] = (int)i;
  c->max_cell = 0;
  for (long long k = 0; k < ncell; k++) c->max_cell = std::max(c->max_cell, start[(size_t)k + 1] - start[(size_t)k]);
  c->lcap = list_capacity(c, x, y, z, order, start, dims);
  // packed atom tables: A = 4 eps sig^12, B = 4 eps sig^6 (the lj2, lj1 of Force.cpp:89-90)
  std::vector<float4> xq32(n);
  std::vector<float2> ab32(n), abc32(p.gas == CCS_GAS_CO2 ? n : 0);
  std::vector<double4> xq64(n);
  std::vector<double2> ab64(n), abc64(p.gas == CCS_GAS_CO2 ? n : 0);
  for (size_t s = 0; s < n; s++) {
    const int i = order[s];
    const double qq = (ft == 1 || ft == 2) ? 0.0 : q[i];
    xq64[s] = make_double4(x[i], y[i], z[i], qq);
    xq32[s] = make_float4((float)x[i], (float)y[i], (float)z[i], (float)qq);
    const double s6 = std::pow(sig[i], 6.0), B = 4.0 * eps[i] * s6, A = B * s6;
    ab64[s] = make_double2(A, B);
    ab32[s] = make_float2((float)A, (float)B);
    if (p.gas == CCS_GAS_CO2) {
      const double c6 = std::pow(sig_c[i], 6.0), Bc = 4.0 * eps_c[i] * c6, Ac = Bc * c6;
      abc64[s] = make_double2(Ac, Bc);
      abc32[s] = make_float2((float)Ac, (float)Bc);
    }
  }
  const bool fp64 = p.precision == CCS_PREC_FP64;
  if (fp64) {
    CK(cudaMalloc(&c->d_xyzq64, n * sizeof(double4)));
    CK(cudaMalloc(&c->d_ab64, n * sizeof(double2)));
    CK(to_dev(c, c->d_xyzq64, xq64.data(), n * sizeof(double4)));
    CK(to_dev(c, c->d_ab64, ab64.data(), n * sizeof(double2)));
    if (p.gas == CCS_GAS_CO2) {
      CK(cudaMalloc(&c->d_abc64, n * sizeof(double2)));
      CK(to_dev(c, c->d_abc64, abc64.data(), n * sizeof(double2)));
    }
  } else {
    CK(cudaMalloc(&c->d_xyzq32, n * sizeof(float4)));
    CK(cudaMalloc(&c->d_ab32, n * sizeof(float2)));
    CK(to_dev(c, c->d_xyzq32, xq32.data(), n * sizeof(float4)));
    CK(to_dev(c, c->d_ab32, ab32.data(), n * sizeof(float2)));
    if (p.gas == CCS_GAS_CO2) {
      CK(cudaMalloc(&c->d_abc32, n * sizeof(float2)));
      CK(to_dev(c, c->d_abc32, abc32.data(), n * sizeof(float2)));
    }
  }
  CK(cudaMalloc(&c->d_cell_start, start.size() * sizeof(int)));
  CK(to_dev(c, c->d_cell_start, start.data(), start.size() * sizeof(int)));
  CK(cudaStreamSynchronize(c->stream));  // runs may launch on other streams
  c->have_target = true;
  c->tuned_G = 0;
  c->batch_G = 0;
  return CCS_OK;
}

int ccs_get_info(ccs_ctx *c, ccs_info *info) {
  if (!c || !info) return CCS_ERR_INVALID;
  std::memset(info, 0, sizeof *info);
  info->nx = c->nx; info->ny = c->ny; info->nz = c->nz; info->natoms = c->natoms;
  info->cell_size = c->h; info->reach = c->reach;
  for (int d = 0; d < 3; d++) info->origin[d] = c->origin[d];
  info->charged = c->charged; info->allpairs = c->allpairs; info->max_cell_atoms = c->max_cell;
  info->vel_table_len = c->vtab_n; info->sm_count = c->sm_count;
  info->reserved = c->tuned_G;
  return CCS_OK;
}

int ccs_run_device(ccs_ctx *c, size_t n, const double *d_rnd, size_t stride, int8_t *d_status,
                   double *d_omc, uint32_t *d_steps, uint32_t *d_visits, void *stream) {
  if (!c) return CCS_ERR_INVALID;
  if (!c->have_target) return fail(c, CCS_ERR_INVALID, "no target set");
  if (n == 0) return CCS_OK;
  if (!d_rnd || !d_status || !d_omc || stride < n) return fail(c, CCS_ERR_INVALID, "bad device buffers");
  if (cudaSetDevice(c->device) != cudaSuccess) return fail(c, CCS_ERR_CUDA, "cudaSetDevice");
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  const int block = BLOCK;
  if (!c->tuned_G) {
    // tune on the caller's inputs (outputs land in the context's own buffers)
    int rc = ensure_run_buffers(c, std::min<size_t>(n, (size_t)c->sm_count * 256), false);
    if (rc) return rc;
    if (c->p.lanes_per_traj > 0) c->tuned_G = c->p.lanes_per_traj;
    else {
      CK(cudaStreamSynchronize(s));
      const double *save = c->d_rnd;
      c->d_rnd = const_cast<double *>(d_rnd);
      rc = autotune(c, n, stride, block);
      c->d_rnd = const_cast<double *>(save);
      if (rc) return rc;
    }
  }
  CK(cudaEventRecord(c->ev[2], s));
  int rc = run_device(c, n, d_rnd, stride, d_status, d_omc, d_steps, d_visits, s, c->tuned_G, block);
  if (rc) return rc;
  CK(cudaEventRecord(c->ev[3], s));
  c->last.ntraj = n;
  return CCS_OK;
}

int ccs_sync_stats(ccs_ctx *c, ccs_stats *st) {
  if (!c) return CCS_ERR_INVALID;
  CK(cudaEventSynchronize(c->ev[3]));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]));
  c->last.kernel_ms = ms;
  return read_stats(c, st, c->last.ntraj);
}

int ccs_run(ccs_ctx *c, size_t n, const double *const rnd[9], int8_t *status, double *omc,
            uint32_t *steps, uint32_t *visits, ccs_stats *st) {
  if (!c) return CCS_ERR_INVALID;
  if (!c->have_target) return fail(c, CCS_ERR_INVALID, "no target set");
  if (n == 0) { if (st) { std::memset(st, 0, sizeof *st); } return CCS_OK; }
  if (!rnd || !status || !omc) return fail(c, CCS_ERR_INVALID, "rnd, status and one_minus_cos are required");
  const int nrows = is_molecule(c->p.gas) ? 9 : 5;
  for (int k = 0; k < nrows; k++)
    if (!rnd[k]) return fail(c, CCS_ERR_INVALID, "rnd[%d] is NULL", k);
  if (cudaSetDevice(c->device) != cudaSuccess) return fail(c, CCS_ERR_CUDA, "cudaSetDevice");
  int rc = ensure_run_buffers(c, n, true);
  if (rc) return rc;
  CK(cudaEventRecord(c->ev[0], c->stream));
  for (int k = 0; k < nrows; k++)
    CK(cudaMemcpyAsync(c->d_rnd + (size_t)k * n, rnd[k], n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaEventRecord(c->ev[1], c->stream));
  const int block = BLOCK;
  rc = autotune(c, n, n, block);
  if (rc) return rc;
  CK(cudaEventRecord(c->ev[2], c->stream));
  rc = run_device(c, n, c->d_rnd, n, c->d_status, c->d_omc, steps ? c->d_steps : nullptr,
                  visits ? c->d_visits : nullptr, c->stream, c->tuned_G, block);
  if (rc) return rc;
  CK(cudaEventRecord(c->ev[3], c->stream));
  CK(cudaMemcpyAsync(status, c->d_status, n, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(omc, c->d_omc, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (steps) CK(cudaMemcpyAsync(steps, c->d_steps, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
  if (visits) CK(cudaMemcpyAsync(visits, c->d_visits, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaEventRecord(c->ev[4], c->stream));
  CK(cudaStreamSynchronize(c->stream));
  float t01 = 0, t23 = 0, t34 = 0;
  CK(cudaEventElapsedTime(&t01, c->ev[0], c->ev[1]));
  CK(cudaEventElapsedTime(&t23, c->ev[2], c->ev[3]));
  CK(cudaEventElapsedTime(&t34, c->ev[3], c->ev[4]));
  c->last.h2d_ms = t01;
  c->last.kernel_ms = t23;
  c->last.d2h_ms = t34;
  return read_stats(c, st, n);
}

int ccs_run_batch(ccs_ctx *const *ions, size_t nions, const size_t *ntraj, const double *const rnd[9],
                  int8_t *status, double *omc, uint32_t *steps, uint32_t *visits, ccs_stats *st) {
  if (!ions || nions == 0 || !ions[0]) return CCS_ERR_INVALID;
  ccs_ctx *lead = ions[0];
  if (!ntraj) return fail(lead, CCS_ERR_INVALID, "ntraj is required");
  const int gas = gas_kind(lead->p.gas);
  size_t total = 0;
  std::vector<size_t> off(nions);
  for (size_t i = 0; i < nions; i++) {
    const ccs_ctx *ci = ions[i];
    if (!ci) return fail(lead, CCS_ERR_INVALID, "ion %zu has no context", i);
    if (!ci->have_target) return fail(lead, CCS_ERR_INVALID, "ion %zu has no target", i);
    if (ci->device != lead->device) return fail(lead, CCS_ERR_INVALID, "ion %zu is on another device", i);
    if (gas_kind(ci->p.gas) != gas) return fail(lead, CCS_ERR_INVALID, "ion %zu: atomic and molecular gases mixed", i);
    if (ci->p.precision != lead->p.precision) return fail(lead, CCS_ERR_INVALID, "ion %zu: precision differs", i);
    off[i] = total;
    total += ntraj[i];
  }
  if (total == 0) { if (st) { std::memset(st, 0, sizeof *st); } return CCS_OK; }
  if (!rnd || !status || !omc) return fail(lead, CCS_ERR_INVALID, "rnd, status and one_minus_cos are required");
  const int nrows = gas == GAS_ATOM ? 5 : 9;
  for (int k = 0; k < nrows; k++)
    if (!rnd[k]) return fail(lead, CCS_ERR_INVALID, "rnd[%d] is NULL", k);
  if (cudaSetDevice(lead->device) != cudaSuccess) return fail(lead, CCS_ERR_CUDA, "cudaSetDevice");
  ccs_ctx *c = lead;  // error reports go to the lead context
  int rc = ensure_run_buffers(lead, total, true);
  if (rc) return rc;
  cudaStream_t s = lead->stream;
  CK(cudaEventRecord(lead->ev[0], s));
  for (int k = 0; k < nrows; k++)
    CK(cudaMemcpyAsync(lead->d_rnd + (size_t)k * total, rnd[k], total * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaEventRecord(lead->ev[1], s));
  int G = 32;
  rc = autotune_batch(lead, ions, nions, ntraj, off.data(), total, G);
  if (rc) return rc;
  CK(cudaEventRecord(lead->ev[2], s));
  rc = run_batch_device(lead, ions, nions, ntraj, off.data(), total, steps != nullptr, visits != nullptr, G);
  if (rc) return rc;
  CK(cudaEventRecord(lead->ev[3], s));
  CK(cudaMemcpyAsync(status, lead->d_status, total, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(omc, lead->d_omc, total * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (steps) CK(cudaMemcpyAsync(steps, lead->d_steps, total * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  if (visits) CK(cudaMemcpyAsync(visits, lead->d_visits, total * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  CK(cudaEventRecord(lead->ev[4], s));
  CK(cudaStreamSynchronize(s));
  float t01 = 0, t23 = 0, t34 = 0;
  CK(cudaEventElapsedTime(&t01, lead->ev[0], lead->ev[1]));
  CK(cudaEventElapsedTime(&t23, lead->ev[2], lead->ev[3]));
  CK(cudaEventElapsedTime(&t34, lead->ev[3], lead->ev[4]));
  lead->last.h2d_ms = t01;
  lead->last.kernel_ms = t23;
  lead->last.d2h_ms = t34;
  return read_stats(lead, st, total);
}

int ccs_eval_site_forces(ccs_ctx *c, size_t npts, int site, const double *pos, double *f, double *U,
                         uint32_t *visits) {
  if (!c) return CCS_ERR_INVALID;
  if (!c->have_target) return fail(c, CCS_ERR_INVALID, "no target set");
  const int ns = is_molecule(c->p.gas) ? 3 : 1;
  if (site < 0 || site >= ns) return fail(c, CCS_ERR_INVALID, "site out of range");
  if (npts == 0) return CCS_OK;
  if (!pos || !f || !U) return fail(c, CCS_ERR_INVALID, "pos, f and U are required");
  if (cudaSetDevice(c->device) != cudaSuccess) return fail(c, CCS_ERR_CUDA, "cudaSetDevice");
  double *dp = nullptr, *df = nullptr, *dU = nullptr;
  uint32_t *dv = nullptr;
  auto cleanup = [&]() { cudaFree(dp); cudaFree(df); cudaFree(dU); cudaFree(dv); };
  if (cudaMalloc(&dp, npts * 3 * sizeof(double)) || cudaMalloc(&df, npts * 3 * sizeof(double)) ||
      cudaMalloc(&dU, npts * sizeof(double)) || cudaMalloc(&dv, npts * sizeof(uint32_t))) {
    cleanup();
    return fail(c, CCS_ERR_NOMEM, "cudaMalloc for force points");
  }
  int rc = CCS_OK;
  do {
    if (to_dev(c, dp, pos, npts * 3 * sizeof(double))) { rc = CCS_ERR_CUDA; break; }
    KParams k = base_params(c);
    const int G = c->p.lanes_per_traj == 1 ? 1 : c->p.lanes_per_traj == 8 ? 8 : 32;
    ForceFn fn = pick_force(c, G);
    const int block = 128;
    const size_t grid = std::min<size_t>((npts * G + block - 1) / block, (size_t)c->sm_count * 16);
    fn<<<(unsigned)grid, block, 0, c->stream>>>(k, site, npts, dp, df, dU, dv);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(c->stream) != cudaSuccess) { rc = CCS_ERR_CUDA; break; }
    if (to_host(c, f, df, npts * 3 * sizeof(double)) ||
        to_host(c, U, dU, npts * sizeof(double))) { rc = CCS_ERR_CUDA; break; }
    if (visits && to_host(c, visits, dv, npts * sizeof(uint32_t))) { rc = CCS_ERR_CUDA; break; }
  } while (0);
  cleanup();
  if (rc) return fail(c, rc, "force evaluation failed: %s", cudaGetErrorString(cudaGetLastError()));
  return CCS_OK;
}

int ccs_eval_setup(ccs_ctx *c, size_t n, const double *const rnd[9], int8_t *hit, double *pos, double *vel) {
  if (!c) return CCS_ERR_INVALID;
  if (!c->have_params || !c->vtab_n) return fail(c, CCS_ERR_INVALID, "ccs_set_params must come first");
  if (n == 0) return CCS_OK;
  if (!rnd || !hit || !pos || !vel) return fail(c, CCS_ERR_INVALID, "missing buffers");
  const int nrows = is_molecule(c->p.gas) ? 9 : 5;
  for (int k = 0; k < nrows; k++)
    if (!rnd[k]) return fail(c, CCS_ERR_INVALID, "rnd[%d] is NULL", k);
  if (cudaSetDevice(c->device) != cudaSuccess) return fail(c, CCS_ERR_CUDA, "cudaSetDevice");
  int rc = ensure_run_buffers(c, n, true);
  if (rc) return rc;
  double *dpos = nullptr, *dvel = nullptr;
  if (cudaMalloc(&dpos, n * 9 * sizeof(double)) || cudaMalloc(&dvel, n * 9 * sizeof(double))) {
    cudaFree(dpos); cudaFree(dvel);
    return fail(c, CCS_ERR_NOMEM, "cudaMalloc for setup");
  }
  for (int k = 0; k < nrows; k++)
    if (to_dev(c, c->d_rnd + (size_t)k * n, rnd[k], n * sizeof(double))) rc = CCS_ERR_CUDA;
  if (!rc) {
    KParams k = base_params(c);
    k.rnd = c->d_rnd;
    k.rnd_stride = n;
    k.ntraj = n;
    setup_kernel<<<(unsigned)((n + 127) / 128), 128, 0, c->stream>>>(k, c->d_status, dpos, dvel);
    if (cudaGetLastError() || cudaStreamSynchronize(c->stream)) rc = CCS_ERR_CUDA;
  }
  if (!rc && (to_host(c, hit, c->d_status, n) ||
              to_host(c, pos, dpos, n * 9 * sizeof(double)) ||
              to_host(c, vel, dvel, n * 9 * sizeof(double))))
    rc = CCS_ERR_CUDA;
  cudaFree(dpos);
  cudaFree(dvel);
  if (rc) return fail(c, rc, "setup evaluation failed");
  return CCS_OK;
}

}  // extern "C"

// FP32 FMA throughput kernel: 8 independent chains per thread, each step one FMA.
__global__ void fma_peak_kernel(float *out, int iters, float a, float b) {
  float x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6,
        x7 = x0 + 7;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int u = 0; u < 16; u++) {
      x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
      x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
    }
  }
  const float s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == 123.456f) out[blockIdx.x] = s;  // keeps the chains live
}

extern "C" {

int ccs_measure_fp32_peak(int device, double ms, double *tflops) {
  if (!tflops) return CCS_ERR_INVALID;
  ccs_ctx *c = nullptr;  // CK() reports into no context here
  if (cudaSetDevice(device) != cudaSuccess) return CCS_ERR_NODEVICE;
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, device));
  float *out = nullptr;
  CK(cudaMalloc(&out, 4096 * sizeof(float)));
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const int threads = 256, blocks = prop.multiProcessorCount * 8;
  int iters = 256;
  float best = 0;
  for (int rep = 0; rep < 6; rep++) {
    CK(cudaEventRecord(e0));
    fma_peak_kernel<<<blocks, threads>>>(out, iters, 0.999999f, 1e-7f);
    CK(cudaEventRecord(e1));
    CK(cudaEventSynchronize(e1));
    float t = 0;
    CK(cudaEventElapsedTime(&t, e0, e1));
    const double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
    best = std::max(best, (float)(flops / (t * 1e-3) / 1e12));
    if (t < ms && rep < 5) iters = (int)std::min<double>(1 << 22, iters * std::max(1.0, ms / std::max(t, 0.01f)));
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  *tflops = best;
  return CCS_OK;
}

const char *ccs_status_string(int s) {
  switch (s) {
    case CCS_OK: return "ok";
    case CCS_ERR_INVALID: return "invalid argument";
    case CCS_ERR_NOMEM: return "out of memory";
    case CCS_ERR_CUDA: return "CUDA error";
    case CCS_ERR_TIMEOUT: return "device watchdog expired";
    case CCS_ERR_NODEVICE: return "no usable CUDA device";
    case CCS_ERR_UNSUPPORTED: return "unsupported configuration";
    default: return "unknown status";
  }
}

const char *ccs_last_error(ccs_ctx *c) { return c ? c->err.c_str() : "no context"; }

}  // extern "C"

int ccs_internal::eval_site_forces_device(ccs_ctx *c, size_t npts, int site, const double *d_pos, double *d_f,
                                          double *d_U, cudaStream_t s) {
  if (npts == 0) return CCS_OK;
  KParams k = base_params(c);
  ForceFn fn = pick_force(c, 32);
  const int block = 128;
  const size_t grid = std::min<size_t>((npts * 32 + block - 1) / block, (size_t)c->sm_count * 16);
  fn<<<(unsigned)grid, block, 0, s>>>(k, site, npts, d_pos, d_f, d_U, nullptr);
  CK(cudaGetLastError());
  return CCS_OK;
}

// ===========================================================================
// ccs_run_device_noalloc: the trajectory passes with no device allocation.
//
// Some callers cannot allocate device memory while they run: a host that has
// handed the whole device heap to its own pool allocator, a real-time or
// embedded service whose memory budget is fixed at start-up, or code running
// where a cudaMalloc would synchronise the device or fail.  For them the
// scratch of the trajectory passes (work counter, statistics, watchdog
// deadline, the device copy of the launch parameters and the park buffer of
// long trajectories) lives in this file-scope array instead of per-context
// allocations.  Every GPU that loads the library holds it until the process
// exits.
namespace {
constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(40) << 20;  // 40 MiB per device
constexpr size_t NOALLOC_HEADER_BYTES = 256;                // counters, deadline and the error flag
constexpr size_t NOALLOC_PARAMS_BYTES = 4096;               // the launch-parameter copy
constexpr size_t NOALLOC_MAX_TRAJ = size_t(1) << 18;        // 262144 trajectories per call
// park capacity: the rule of ccs_run_device (park_capacity) at the largest n
constexpr size_t NOALLOC_PARK_CAP = NOALLOC_MAX_TRAJ / 2;
static_assert(sizeof(KParams) <= NOALLOC_PARAMS_BYTES, "launch parameters do not fit");
static_assert(NOALLOC_HEADER_BYTES + NOALLOC_PARAMS_BYTES + NOALLOC_PARK_CAP * sizeof(LaneState<double>) <=
                  NOALLOC_SCRATCH_BYTES,
              "park buffer does not fit");
static_assert(12 * sizeof(unsigned long long) + sizeof(int) <= NOALLOC_HEADER_BYTES, "header does not fit");
}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// The device-side copy of the launch parameters, written by a kernel so that
// no host staging is involved.
__global__ void copy_params_kernel(KParams k, KParams *dst) { *dst = k; }

namespace {
// device address of g_noalloc_scratch, looked up once per device (with that
// device current); host code may not use the symbol itself as an address
struct NoallocSlot {
  std::once_flag once;
  unsigned char *ptr = nullptr;
  cudaError_t err = cudaSuccess;
};
NoallocSlot g_noalloc_slots[64];

unsigned char *noalloc_scratch(int device, cudaError_t &err) {
  if (device < 0 || device >= 64) {
    err = cudaErrorInvalidDevice;
    return nullptr;
  }
  NoallocSlot &slot = g_noalloc_slots[device];
  std::call_once(slot.once, [&]() {
    void *p = nullptr;
    slot.err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    slot.ptr = slot.err == cudaSuccess ? static_cast<unsigned char *>(p) : nullptr;
  });
  err = slot.err;
  return slot.ptr;
}
}  // namespace

extern "C" int ccs_run_device_noalloc(ccs_ctx *c, size_t n, const double *d_rnd, size_t stride, int8_t *d_status,
                                      double *d_omc, uint32_t *d_steps, uint32_t *d_visits, void *stream,
                                      ccs_stats *stats) {
  if (!c) return CCS_ERR_INVALID;
  if (!c->have_target) return fail(c, CCS_ERR_INVALID, "no target set");
  if (n == 0) return CCS_OK;
  if (n > NOALLOC_MAX_TRAJ)
    return fail(c, CCS_ERR_INVALID,
                "ccs_run_device_noalloc: %zu trajectories exceed the maximum of %zu per call (the fixed scratch "
                "holds the park buffer for that many); split the run or use ccs_run_device",
                n, NOALLOC_MAX_TRAJ);
  if (!d_rnd || !d_status || !d_omc || stride < n) return fail(c, CCS_ERR_INVALID, "bad device buffers");
  if (cudaSetDevice(c->device) != cudaSuccess) return fail(c, CCS_ERR_CUDA, "cudaSetDevice");
  cudaError_t serr = cudaSuccess;
  unsigned char *base = noalloc_scratch(c->device, serr);
  if (!base) return fail(c, CCS_ERR_CUDA, "cudaGetSymbolAddress(g_noalloc_scratch): %s", cudaGetErrorString(serr));
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  // header: [0] work counter [1..7] statistics [8] watchdog deadline [9] parked [10] resumed, then the error flag
  unsigned long long *work = reinterpret_cast<unsigned long long *>(base);
  int *error = reinterpret_cast<int *>(base + 12 * sizeof(unsigned long long));
  KParams *kparams = reinterpret_cast<KParams *>(base + NOALLOC_HEADER_BYTES);
  void *park = base + NOALLOC_HEADER_BYTES + NOALLOC_PARAMS_BYTES;
  // lanes per force evaluation: the configured or already tuned value (no autotuning here)
  const int G = c->p.lanes_per_traj > 0 ? c->p.lanes_per_traj : (c->tuned_G ? c->tuned_G : 32);
  const int block = BLOCK;
  KParams k = base_params(c);
  k.rnd = d_rnd;
  k.rnd_stride = stride;
  k.ntraj = n;
  k.status = d_status;
  k.omc = d_omc;
  k.steps = d_steps;
  k.visits = d_visits;
  k.order = nullptr;  // index order (the processing order never changes a result)
  k.work = work;
  k.stats = work + 1;
  k.error = error;
  k.deadline = work + 8;
  k.park = park;
  k.park_cap = park_capacity(n);
  k.park_steps = c->p.park_steps ? c->p.park_steps : 2048u;
  k.park_drained = c->p.schedule == 2;
  k.park_count = work + 9;
  k.park_next = work + 10;
  // everything that must start at zero: counters, statistics, park counters, error flag
  CK(cudaMemsetAsync(base, 0, NOALLOC_HEADER_BYTES, s));
  int rc = arm_deadline(c, work + 8, s);
  if (rc) return rc;
  copy_params_kernel<<<1, 1, 0, s>>>(k, kparams);
  CK(cudaGetLastError());
  KernelFn fn = pick_traj(c, G);
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)fn, block, 0));
  size_t grid = (size_t)std::max(per_sm, 1) * c->sm_count;
  grid = std::min(grid, std::max<size_t>(1, (n + block - 1) / block));
  CK(cudaEventRecord(c->ev[2], s));
  CK(cudaEventRecord(c->ev[5], s));
  fn<<<(unsigned)grid, block, 0, s>>>(k, kparams);
  CK(cudaGetLastError());
  CK(cudaEventRecord(c->ev[6], s));
  KernelFn rfn = pick_resume(c);
  int rper_sm = 0;
  const int rnt = resume_threads(c);
  const size_t rdyn = (size_t)k.lcap * sizeof(int);
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&rper_sm, (const void *)rfn, rnt, rdyn));
  rfn<<<(unsigned)((size_t)std::max(rper_sm, 1) * c->sm_count), rnt, rdyn, s>>>(k, kparams);
  CK(cudaGetLastError());
  CK(cudaEventRecord(c->ev[7], s));
  CK(cudaEventRecord(c->ev[3], s));
  // ccs_sync_stats reads this run's counters and error flag from the scratch
  c->run_work = work;
  c->run_error = error;
  c->last.ntraj = n;
  c->last.grid_size = (int32_t)grid;
  c->last.block_size = block;
  c->last.lanes_per_traj = G;
  if (stats) return ccs_sync_stats(c, stats);
  return CCS_OK;
}
