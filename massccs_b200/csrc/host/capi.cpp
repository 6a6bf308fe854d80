// capi.cpp -- the C-ABI of include/massccs_host.h over the host set-up, and
// mh_run: the reference's whole run (System.cpp:19-326) with the trajectory
// loop replaced by ccs_run.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <memory>
#include <thread>
#include <vector>

#include "massccs_host.h"
#include "setup.h"

struct mh_system {
  std::unique_ptr<massccs::SystemSetup> S;
};

namespace {
void copy_err(char *err, size_t len, const char *msg) {
  if (err && len) std::snprintf(err, len, "%s", msg);
}
}  // namespace

extern "C" {

int mh_open(mh_system **out, const char *input_json, int print, char *err, size_t errlen) {
  if (!out || !input_json) return CCS_ERR_INVALID;
  *out = nullptr;
  try {
    auto sys = std::make_unique<mh_system>();
    sys->S = std::make_unique<massccs::SystemSetup>(input_json, print != 0);
    *out = sys.release();
    return CCS_OK;
  } catch (const std::exception &e) {
    copy_err(err, errlen, e.what());
    return CCS_ERR_INVALID;
  }
}

void mh_close(mh_system *sys) { delete sys; }

int mh_get_info(const mh_system *sys, mh_info *o) {
  if (!sys || !o) return CCS_ERR_INVALID;
  const auto &S = *sys->S;
  std::memset(o, 0, sizeof *o);
  o->gas_flag = S.in.gas_buffer_flag;
  o->force_type = S.force_type;
  o->natoms = S.target.natoms;
  o->gas_natoms = S.gas.natoms;
  o->nprobe = S.in.nProbe; o->niter = S.in.nIter; o->seed = S.in.seed; o->nthreads = S.in.nthreads;
  o->short_range_cutoff = S.in.short_range_cutoff; o->long_range_flag = S.in.long_range_flag;
  o->long_range_cutoff = S.in.long_range_cutoff; o->polarizability_flag = S.in.polarizability_flag;
  o->equipotential_flag = S.in.equipotential_flag; o->user_ff_flag = S.in.user_ff_flag;
  o->dt = S.in.dt; o->temperature = S.in.temperatureTarget; o->skin = S.in.skin;
  o->lj_cutoff = S.in.lj_cutoff; o->coul_cutoff = S.in.coul_cutoff; o->alpha = S.alpha;
  o->mu = S.mu; o->target_mass = S.target.mass; o->target_charge = S.target.Q;
  o->gas_mass = S.gas.mass; o->gas_inertia = S.gas_inertia; o->d_bond = S.d_bond;
  o->a = S.a; o->b = S.b; o->c = S.c; o->bmax = S.bmax;
  o->lx = S.lx; o->ly = S.ly; o->lz = S.lz;
  o->Nx = S.Nx; o->Ny = S.Ny; o->Nz = S.Nz; o->Ncells = S.Nx * S.Ny * S.Nz;
  o->cell_size = S.cell_size;
  o->max_x = S.target.maxX; o->max_y = S.target.maxY; o->max_z = S.target.maxZ;
  o->radius = S.target.radius;
  return CCS_OK;
}

int mh_get_target(const mh_system *sys, double *x, double *y, double *z, double *q, double *m, double *eps,
                  double *sig, double *eps_c, double *sig_c) {
  if (!sys) return CCS_ERR_INVALID;
  const auto &t = sys->S->target;
  const size_t n = (size_t)t.natoms * sizeof(double);
  const std::vector<double> *src[9] = {&t.x, &t.y, &t.z, &t.q, &t.m, &t.eps, &t.sig, &t.eps_c, &t.sig_c};
  double *dst[9] = {x, y, z, q, m, eps, sig, eps_c, sig_c};
  for (int k = 0; k < 9; k++)
    if (dst[k]) std::memcpy(dst[k], src[k]->data(), n);
  return CCS_OK;
}

int mh_fill_params(const mh_system *sys, ccs_params *p) {
  if (!sys || !p) return CCS_ERR_INVALID;
  const auto &S = *sys->S;
  ccs_params_default(p);
  p->gas = S.in.gas_buffer_flag;
  p->force_type = S.force_type;
  p->dt = S.in.dt;
  p->temperature = S.in.temperatureTarget;
  p->mu = S.mu;
  p->gas_inertia = S.gas_inertia;
  p->d_bond = S.d_bond;
  p->alpha = S.alpha;
  p->lj_cutoff = S.in.lj_cutoff;
  p->coul_cutoff = S.in.coul_cutoff;
  p->skin = S.in.skin;
  p->a = S.a; p->b = S.b; p->c = S.c; p->bmax = S.bmax;
  p->lx = S.lx; p->ly = S.ly; p->lz = S.lz;
  p->precision = S.in.precision == "fp64" ? CCS_PREC_FP64 : CCS_PREC_FP32;
  p->quirks = S.in.ref_quirks ? CCS_QUIRK_CO2_VCM : 0;
  return CCS_OK;
}

int mh_predraw(const mh_system *sys, uint32_t seed, size_t n, double *rnd) {
  if (!sys || (!rnd && n)) return CCS_ERR_INVALID;
  massccs::predraw(*sys->S, seed, n, rnd);
  return CCS_OK;
}

int mh_reduce(size_t niter, size_t nprobe, const int8_t *status, const double *omc, double bmax, double *omega,
              int32_t *nfree, int32_t *nscatter, int32_t *nlost, double *ccs, double *err) {
  if (!status || !omc || niter == 0) return CCS_ERR_INVALID;
  const auto R = massccs::reduce(niter, nprobe, status, omc, bmax);
  for (size_t i = 0; i < niter; i++) {
    if (omega) omega[i] = R.omega[i];
    if (nfree) nfree[i] = R.nfree[i];
    if (nscatter) nscatter[i] = R.nscatter[i];
    if (nlost) nlost[i] = R.nlost[i];
  }
  if (ccs) *ccs = R.ccs;
  if (err) *err = R.err;
  return CCS_OK;
}

}  // extern "C"

namespace {
using CtxPtr = std::unique_ptr<ccs_ctx, void (*)(ccs_ctx *)>;

int make_context(const massccs::SystemSetup &S, int device, const ccs_params &p, CtxPtr &out, int print) {
  ccs_ctx *ctx = nullptr;
  int rc = ccs_create(&ctx, device);
  if (rc) {
    if (print) std::cerr << "ccs_create (GPU " << device << "): " << ccs_status_string(rc) << std::endl;
    return rc;
  }
  out.reset(ctx);
  if ((rc = ccs_set_params(ctx, &p)) ||
      (rc = ccs_set_target(ctx, (size_t)S.target.natoms, S.target.x.data(), S.target.y.data(), S.target.z.data(),
                           S.target.q.data(), S.target.eps.data(), S.target.sig.data(),
                           S.in.gas_buffer_flag == 3 ? S.target.eps_c.data() : nullptr,
                           S.in.gas_buffer_flag == 3 ? S.target.sig_c.data() : nullptr))) {
    if (print) std::cerr << "massccs: " << ccs_last_error(ctx) << std::endl;
    return rc;
  }
  return CCS_OK;
}

// The whole run over one or several GPUs: one pre-draw, contiguous slices of
// the trajectory numbers per GPU (every trajectory keeps its random numbers,
// so the split changes no initial condition), one fixed-order reduction.
// With several GPUs the lanes per force evaluation are tuned once (GPU 0, on
// the run's first trajectories) and used by every GPU.
int run_impl(mh_system *sys, const std::vector<int> &devices, const ccs_params *overrides, int print,
             double *ccs_out, double *err_out, double *seconds) {
  const auto &S = *sys->S;
  const size_t niter = S.in.nIter, nprobe = S.in.nProbe, n = niter * nprobe;
  if (n == 0 || devices.empty()) return CCS_ERR_INVALID;
  const size_t nd = devices.size();
  ccs_params p;
  if (overrides) p = *overrides;
  else mh_fill_params(sys, &p);
  std::vector<CtxPtr> ctxs;
  for (size_t r = 0; r < nd; r++) {
    ctxs.emplace_back(nullptr, ccs_destroy);
    int rc = make_context(S, devices[r], p, ctxs.back(), print);
    if (rc) return rc;
  }
  ccs_ctx *ctx = ctxs[0].get();
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<double> rnd(9 * n);
  massccs::predraw(S, S.in.seed, n, rnd.data());
  if (print) {
    std::cout << "*********************************************************" << std::endl;
    std::cout << "Trajectory calculations " << std::endl;
    std::cout << "*********************************************************" << std::endl;
  }
  const double *rows[9];
  for (int k = 0; k < 9; k++) rows[k] = rnd.data() + (size_t)k * n;
  std::vector<int8_t> status(n);
  std::vector<double> omc(n);
  ccs_stats st;
  std::memset(&st, 0, sizeof st);
  int rc = CCS_OK;
  if (nd == 1) {
    rc = ccs_run(ctx, n, rows, status.data(), omc.data(), nullptr, nullptr, &st);
  } else {
    if (p.lanes_per_traj == 0) {  // tune once, on GPU 0, then fix the choice everywhere
      const size_t m = std::min<size_t>(n, 148 * 256);
      std::vector<int8_t> s0(m);
      std::vector<double> o0(m);
      ccs_info info;
      if ((rc = ccs_run(ctx, m, rows, s0.data(), o0.data(), nullptr, nullptr, nullptr)) ||
          (rc = ccs_get_info(ctx, &info))) {
        if (print) std::cerr << "massccs: " << ccs_last_error(ctx) << std::endl;
        return rc;
      }
      p.lanes_per_traj = info.reserved;  // the tuned lanes per force evaluation
      for (size_t r = 0; r < nd; r++)
        if ((rc = make_context(S, devices[r], p, ctxs[r], print))) return rc;
      ctx = ctxs[0].get();
    }
    std::vector<ccs_stats> sts(nd);
    std::vector<int> rcs(nd, CCS_OK);
    std::vector<std::thread> th;
    for (size_t r = 0; r < nd; r++) {
      th.emplace_back([&, r]() {
        const size_t lo = n * r / nd, hi = n * (r + 1) / nd;
        const double *rr[9];
        for (int k = 0; k < 9; k++) rr[k] = rows[k] + lo;
        rcs[r] = hi > lo ? ccs_run(ctxs[r].get(), hi - lo, rr, status.data() + lo, omc.data() + lo, nullptr, nullptr,
                                   &sts[r])
                         : CCS_OK;
      });
    }
    for (auto &t : th) t.join();
    for (size_t r = 0; r < nd; r++) {
      if (rcs[r]) {
        if (print) std::cerr << "massccs (GPU " << devices[r] << "): " << ccs_last_error(ctxs[r].get()) << std::endl;
        return rcs[r];
      }
      const ccs_stats &a = sts[r];
      st.ntraj += a.ntraj; st.nfree += a.nfree; st.nscatter += a.nscatter; st.nlost += a.nlost;
      st.ncapped += a.ncapped; st.steps += a.steps; st.visits += a.visits; st.parked += a.parked;
      st.kernel_ms = std::max(st.kernel_ms, a.kernel_ms);
      st.lane_ms = std::max(st.lane_ms, a.lane_ms);
      st.warp_ms = std::max(st.warp_ms, a.warp_ms);
      st.lanes_per_traj = a.lanes_per_traj;
    }
  }
  if (rc) {
    if (print) std::cerr << "massccs: " << ccs_last_error(ctx) << std::endl;
    return rc;
  }
  const auto R = massccs::reduce(niter, nprobe, status.data(), omc.data(), S.bmax);
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (print) {
    for (size_t i = 0; i < niter; i++) {  // System.cpp:303-307
      std::printf("Ntraj: %i\n", (int)nprobe);
      std::printf("Nfree: %i\n", R.nfree[i]);
      std::printf("Nscatter: %i\n", R.nscatter[i]);
      std::printf("Nlost: %i\n", R.nlost[i]);
      std::printf("omega: %g\n", R.omega[i]);
    }
    std::fflush(stdout);
    std::cout << "CCS time: " << secs << " s" << std::endl;
    std::cout << "*********************************************************" << std::endl;
    std::cout << "average value of CCS = " << R.ccs << " Ang^2" << std::endl;
    std::cout << "error value of CCS = " << R.err << " Ang^2" << std::endl;
    std::cout << "*********************************************************" << std::endl;
    std::cout << "B200 engine: " << (p.precision == CCS_PREC_FP64 ? "FP64" : "FP32") << ", " << nd
              << (nd == 1 ? " GPU, " : " GPUs, ") << st.lanes_per_traj << " lanes per force evaluation, "
              << st.kernel_ms << " ms on the device (" << st.lane_ms << " lane pass, " << st.warp_ms
              << " warp pass, " << st.parked << " long trajectories), " << (double)n / (st.kernel_ms * 1e-3)
              << " trajectories/s" << std::endl;
    if (st.ncapped)
      std::cout << "warning: " << st.ncapped << " trajectories reached the step cap and were counted as lost"
                << std::endl;
  }
  // The FP32 result's error against FP64: the first trajectories again in the
  // engine's FP64 mode on the same initial conditions, compared pairwise
  // (dOmega of free and scattered trajectories, the reference's estimator).
  const size_t m = std::min<size_t>(n, S.in.fp64_check);
  if (print && m > 1 && p.precision == CCS_PREC_FP32) {
    ccs_params p64 = p;
    p64.precision = CCS_PREC_FP64;
    std::vector<int8_t> st64(m);
    std::vector<double> om64(m);
    ccs_stats s64;
    if ((rc = ccs_set_params(ctx, &p64)) ||
        (rc = ccs_set_target(ctx, (size_t)S.target.natoms, S.target.x.data(), S.target.y.data(), S.target.z.data(),
                             S.target.q.data(), S.target.eps.data(), S.target.sig.data(),
                             S.in.gas_buffer_flag == 3 ? S.target.eps_c.data() : nullptr,
                             S.in.gas_buffer_flag == 3 ? S.target.sig_c.data() : nullptr)) ||
        (rc = ccs_run(ctx, m, rows, st64.data(), om64.data(), nullptr, nullptr, &s64))) {
      std::cerr << "massccs: FP64 check: " << ccs_last_error(ctx) << std::endl;
      return rc;
    }
    const double w = M_PI * S.bmax * S.bmax;
    double sa = 0, sb = 0, sd = 0, sdd = 0;
    size_t k = 0, agree = 0;
    for (size_t j = 0; j < m; j++) {
      agree += st64[j] == status[j];
      if (st64[j] > 1 || status[j] > 1) continue;  // lost in either: outside the estimator
      const double a = st64[j] == 1 ? w * om64[j] : 0.0, b = status[j] == 1 ? w * omc[j] : 0.0;
      sa += a; sb += b; sd += b - a; sdd += (b - a) * (b - a);
      k++;
    }
    if (k > 1 && sa > 0) {
      const double mean_d = sd / k, var = (sdd - k * mean_d * mean_d) / (k - 1);
      std::printf("FP64 check: the first %zu trajectories again in FP64: CCS %.6g (FP32) vs %.6g (FP64) Ang^2, "
                  "relative difference %+.3f %% +- %.3f %% (paired), status agreement %.2f %%\n",
                  m, sb / k, sa / k, 100.0 * mean_d / (sa / k), 100.0 * std::sqrt(std::max(var, 0.0) / k) / (sa / k),
                  100.0 * agree / m);
      std::fflush(stdout);
    }
  }
  if (ccs_out) *ccs_out = R.ccs;
  if (err_out) *err_out = R.err;
  if (seconds) *seconds = secs;
  return CCS_OK;
}
}  // namespace

extern "C" {

int mh_run(mh_system *sys, int device, const ccs_params *overrides, int print, double *ccs_out, double *err_out,
           double *seconds) {
  if (!sys) return CCS_ERR_INVALID;
  return run_impl(sys, std::vector<int>{device}, overrides, print, ccs_out, err_out, seconds);
}

int mh_run_devices(mh_system *sys, size_t ndevices, const int *devices, const ccs_params *overrides, int print,
                   double *ccs_out, double *err_out, double *seconds) {
  if (!sys || ndevices == 0 || !devices) return CCS_ERR_INVALID;
  return run_impl(sys, std::vector<int>(devices, devices + ndevices), overrides, print, ccs_out, err_out, seconds);
}

int mh_get_devices(const mh_system *sys, int *devices, size_t cap, size_t *count) {
  if (!sys || !count) return CCS_ERR_INVALID;
  const auto &d = sys->S->in.devices;
  *count = d.size();
  for (size_t k = 0; k < d.size() && k < cap && devices; k++) devices[k] = d[k];
  return CCS_OK;
}

}  // extern "C"
