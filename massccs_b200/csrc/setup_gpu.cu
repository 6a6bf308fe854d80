// setup_gpu.cu -- the equipotential ellipsoid's ray marches on the GPU
// (ccs_equipotential_points in include/massccs_gpu.h).
//
// Reference: cces-cepid/massccs src/Equipotential.cpp:86-200 (the z-extent
// march and the rays towards the z-axis) with the all-atom potentials of
// :203-557.  Every march step needs the probe's potential summed over all
// target atoms without cutoffs, so a multi-million-atom target makes this the
// costliest part of the set-up (O(rays x steps x atoms)).  Here one CTA
// marches one ray: its threads sum the atoms in a fixed strided order and a
// fixed-order block reduction gives every step the same FP64 value on every
// run; the stepping rules, thresholds and crossing points are the
// reference's.  The least-squares fit and the final growth stay on the host
// (csrc/host/equipotential.cpp), which calls this for large targets.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "engine_ctx.h"

using namespace ccs_internal;

namespace {

constexpr int EQ_THREADS = 256;
constexpr double EQ_KCOUL = 332.06348078020324;  // Constants.h: KCOUL
constexpr double EQ_KT500 = 1.38064E-23 * 500.0 * 6.242E18 * 23.061;  // kB * 500 K in kcal/mol
constexpr long long EQ_MAX_STEPS = 200000;  // bound on one march (20 km of 0.1 A steps; the reference's loops are unbounded)

struct EqAtoms {
  const double *x, *y, *z, *q, *lj1, *lj2, *lj1c, *lj2c;  // lj1 = 4 eps sig^6, lj2 = lj1 sig^6
  int n;
  int gas;      // ccs_gas
  int polar;
  double alpha;
};

// Fixed-order block sum of NV values per thread (warp shuffles, then the
// warps in order); every thread returns with the totals in v.
template <int NV> __device__ __forceinline__ void block_sum(double (&v)[NV], double *sm) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; k++)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; k++) sm[w * NV + k] = v[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NV; k++) {
    double s = 0.0;
    for (int q = 0; q < EQ_THREADS / 32; q++) s += sm[q * NV + k];
    v[k] = s;
  }
  __syncthreads();
}

__device__ __forceinline__ double lj_pair(double dx, double dy, double dz, double l1, double l2) {
  const double r2inv = 1.0 / (dx * dx + dy * dy + dz * dz);
  const double r6inv = r2inv * r2inv * r2inv;
  return r6inv * (l2 * r6inv - l1);
}

// The probe's potential at p (Equipotential.cpp:203-557): atoms directly;
// N2 and CO2 in the three axis-aligned orientations, Boltzmann-averaged at
// 500 K.  All threads call it; all return the same value.
__device__ double eq_potential(const EqAtoms &A, const double p[3], double *sm) {
  const bool mol = A.gas == CCS_GAS_N2 || A.gas == CCS_GAS_CO2;
  if (!mol) {
    double v[4] = {0.0, 0.0, 0.0, 0.0};  // U, E
    for (int i = threadIdx.x; i < A.n; i += EQ_THREADS) {
      const double dx = p[0] - A.x[i], dy = p[1] - A.y[i], dz = p[2] - A.z[i];
      v[0] += lj_pair(dx, dy, dz, A.lj1[i], A.lj2[i]);
      if (A.polar) {
        const double r2inv = 1.0 / (dx * dx + dy * dy + dz * dz);
        const double r3inv = sqrt(r2inv) * r2inv;
        v[1] += A.q[i] * dx * r3inv;
        v[2] += A.q[i] * dy * r3inv;
        v[3] += A.q[i] * dz * r3inv;
      }
    }
    block_sum<4>(v, sm);
    double U = v[0];
    if (A.polar) U -= 0.5 * A.alpha * (v[1] * v[1] + v[2] * v[2] + v[3] * v[3]);
    return U;
  }
  const bool co2 = A.gas == CCS_GAS_CO2;
  const double qc = co2 ? 0.6512 : 0.965, qe = -0.5 * qc, d = co2 ? 1.149 : 0.5488;
  double v[17];  // Ulj[6], Uq[6], Ulj_c, Uq_c, E[3]
#pragma unroll
  for (int k = 0; k < 17; k++) v[k] = 0.0;
  for (int i = threadIdx.x; i < A.n; i += EQ_THREADS) {
    const double ax = A.x[i], ay = A.y[i], az = A.z[i], q = A.q[i];
#pragma unroll
    for (int k = 0; k < 6; k++) {
      const int axis = k / 2;
      const double s = (k % 2 == 0) ? d : -d;
      const double dx = p[0] + (axis == 0 ? s : 0.0) - ax;
      const double dy = p[1] + (axis == 1 ? s : 0.0) - ay;
      const double dz = p[2] + (axis == 2 ? s : 0.0) - az;
      v[k] += lj_pair(dx, dy, dz, A.lj1[i], A.lj2[i]);
      if (A.polar) v[6 + k] += qe * q * sqrt(1.0 / (dx * dx + dy * dy + dz * dz)) * EQ_KCOUL;
    }
    const double dx = p[0] - ax, dy = p[1] - ay, dz = p[2] - az;
    const double r2 = dx * dx + dy * dy + dz * dz;
    if (co2) v[12] += lj_pair(dx, dy, dz, A.lj1c[i], A.lj2c[i]);
    if (A.polar) {
      const double rinv = 1.0 / sqrt(r2);
      v[13] += qc * q * rinv * EQ_KCOUL;
      const double r3inv = rinv * (1.0 / r2);
      v[14] += dx * q * r3inv;
      v[15] += dy * q * r3inv;
      v[16] += dz * q * r3inv;
    }
  }
  block_sum<17>(v, sm);
  const double Uind = -0.5 * A.alpha * (v[14] * v[14] + v[15] * v[15] + v[16] * v[16]);
  double Um[3];
  for (int o = 0; o < 3; o++)
    Um[o] = v[2 * o] + v[2 * o + 1] + v[6 + 2 * o] + v[6 + 2 * o + 1] + Uind + (co2 ? v[12] : 0.0) + v[13];
  const double Umin = fmin(Um[0], fmin(Um[1], Um[2]));
  double Z = 0.0;
  for (int o = 0; o < 3; o++) Z += exp(-(Um[o] - Umin) / EQ_KT500);
  double U = 0.0;
  for (int o = 0; o < 3; o++) U += exp(-(Um[o] - Umin) / EQ_KT500) / Z * Um[o];
  return U;
}

// The z-extent march (Equipotential.cpp:86-120): from (0, 0, z0) in 0.5 A
// steps until the threshold is crossed.  One CTA.
__global__ void __launch_bounds__(EQ_THREADS) eq_zmax_kernel(EqAtoms A, double ek, double z0, double *zmax,
                                                             int *error) {
  __shared__ double sm[(EQ_THREADS / 32) * 17];
  double pos[3] = {0.0, 0.0, z0};
  const double slope = (eq_potential(A, pos, sm) + ek < 0.0) ? -1.0 : 1.0;
  for (long long it = 0;; it++) {
    if (it >= EQ_MAX_STEPS) {
      if (threadIdx.x == 0) { *error = 1; *zmax = 0.0; }
      return;
    }
    const double prev = pos[2];
    pos[2] -= 0.5 * slope;
    if ((eq_potential(A, pos, sm) + ek) * slope < 0.0) {
      if (threadIdx.x == 0) *zmax = fmax(pos[2], prev);
      return;
    }
  }
}

// The rays (Equipotential.cpp:122-200): one CTA per ray, in (level,
// rotation) order; the crossing step's farther point, or (0, 0, 0).
// rot[n] = {start x, start y, step x, step y} of rotation n (the host's
// cos/sin of the reference's angles, so both marches start identically).
__global__ void __launch_bounds__(EQ_THREADS) eq_rays_kernel(EqAtoms A, double ek, double zmax, int levels, int nrot,
                                                             const double *__restrict__ rot, double *pts, int *error) {
  __shared__ double sm[(EQ_THREADS / 32) * 17];
  const int ray = blockIdx.x;
  const int i = ray / nrot, nn = ray % nrot;
  const double zInc = 2 * zmax / levels;
  const double zPos = -zmax + i * zInc;
  const double startX = rot[4 * nn], startY = rot[4 * nn + 1];
  double p[3] = {startX, startY, zPos}, pp[3] = {0.0, 0.0, 0.0};
  double vel[3] = {rot[4 * nn + 2], rot[4 * nn + 3], 0.0};
  const double s = (eq_potential(A, p, sm) + ek < 0.0) ? -1.0 : 1.0;
  for (int k = 0; k < 3; k++) vel[k] *= s;
  double hit[3] = {0.0, 0.0, 0.0};
  for (long long it = 0;; it++) {
    if (it >= EQ_MAX_STEPS) {
      if (threadIdx.x == 0) *error = 1;
      break;
    }
    if ((eq_potential(A, p, sm) + ek) * s < 0.0) {
      const double np = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
      const double npp = sqrt(pp[0] * pp[0] + pp[1] * pp[1] + pp[2] * pp[2]);
      const double *far = npp > np ? pp : p;
      hit[0] = far[0]; hit[1] = far[1]; hit[2] = far[2];
      break;
    }
    if ((startX == 0 && startY / p[1] <= 0) || (startY == 0 && startX / p[0] <= 0) ||
        (startX / p[0] <= 0 && startY / p[1] <= 0))
      break;
    for (int k = 0; k < 3; k++) { pp[k] = p[k]; p[k] += vel[k]; }
  }
  if (threadIdx.x == 0) {
    pts[3 * ray] = hit[0]; pts[3 * ray + 1] = hit[1]; pts[3 * ray + 2] = hit[2];
  }
}

template <typename P> void dfree_(P *&p) {
  if (p) cudaFree((void *)p);
  p = nullptr;
}

}  // namespace

extern "C" int ccs_equipotential_points(int device, size_t natoms, const double *x, const double *y,
                                        const double *z, const double *q, const double *eps, const double *sig,
                                        const double *eps_c, const double *sig_c, int gas, int polar,
                                        double alpha, double ek, double max_x, double max_y, double max_z,
                                        size_t cap, double *pts, size_t *npts, double *zmax_out) {
  if (natoms == 0 || natoms > (size_t)1 << 30 || !x || !y || !z || !q || !eps || !sig || !pts || !npts)
    return CCS_ERR_INVALID;
  if (gas == CCS_GAS_CO2 && (!eps_c || !sig_c)) return CCS_ERR_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return CCS_ERR_NODEVICE;
  const size_t n = natoms;
  std::vector<double> l1(n), l2(n), l1c, l2c;
  for (size_t i = 0; i < n; i++) {  // the reference's lj1 = 4 eps sig^6, lj2 = lj1 sig^6 (Equipotential.cpp:215-218)
    l1[i] = 4.0 * eps[i] * std::pow(sig[i], 6);
    l2[i] = l1[i] * std::pow(sig[i], 6);
  }
  if (gas == CCS_GAS_CO2) {
    l1c.resize(n);
    l2c.resize(n);
    for (size_t i = 0; i < n; i++) {
      l1c[i] = 4.0 * eps_c[i] * std::pow(sig_c[i], 6);
      l2c[i] = l1c[i] * std::pow(sig_c[i], 6);
    }
  }
  double *d[8] = {};
  double *dpts = nullptr, *dz = nullptr, *drot = nullptr;
  int *derr = nullptr;
  auto cleanup = [&]() {
    for (auto &p : d) dfree_(p);
    dfree_(dpts); dfree_(dz); dfree_(drot); dfree_(derr);
  };
  const double *src[8] = {x, y, z, q, l1.data(), l2.data(), gas == CCS_GAS_CO2 ? l1c.data() : nullptr,
                          gas == CCS_GAS_CO2 ? l2c.data() : nullptr};
  for (int k = 0; k < 8; k++) {
    if (!src[k]) continue;
    if (cudaMalloc(&d[k], n * sizeof(double)) != cudaSuccess ||
        cudaMemcpy(d[k], src[k], n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
      cleanup();
      cudaGetLastError();
      return CCS_ERR_NOMEM;
    }
  }
  if (cudaMalloc(&dz, sizeof(double)) != cudaSuccess || cudaMalloc(&derr, sizeof(int)) != cudaSuccess ||
      cudaMemset(derr, 0, sizeof(int)) != cudaSuccess) {
    cleanup();
    cudaGetLastError();
    return CCS_ERR_NOMEM;
  }
  EqAtoms A{d[0], d[1], d[2], d[3], d[4], d[5], d[6], d[7], (int)n, gas, polar ? 1 : 0, alpha};
  // the z extent from maxZ + 20 A (Equipotential.cpp:86-120)
  eq_zmax_kernel<<<1, EQ_THREADS>>>(A, ek, std::fabs(max_z) + 20.0, dz, derr);
  double zMax = 0.0;
  int herr = 0;
  if (cudaGetLastError() != cudaSuccess || cudaMemcpy(&zMax, dz, sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
    cleanup();
    return CCS_ERR_CUDA;
  }
  if (herr) {
    cleanup();
    return CCS_ERR_TIMEOUT;
  }
  // the ray set (Equipotential.cpp:122-135)
  const int nrot = 20;
  zMax *= 1.3;
  const double posMag = std::fabs(std::max(std::fabs(max_x), std::fabs(max_y))) + std::fabs(zMax - std::fabs(max_z));
  const int levels = (int)std::ceil((double)std::max(25, (int)std::ceil(zMax)));
  const size_t nrays = (size_t)(levels + 1) * nrot;
  *npts = nrays;
  if (zmax_out) *zmax_out = zMax;
  if (nrays > cap) {
    cleanup();
    return CCS_ERR_INVALID;
  }
  std::vector<double> rot(4 * nrot);
  for (int k = 0; k < nrot; k++) {  // Equipotential.cpp:138-150
    const double theta = k * 2.0 * M_PI / (double)nrot;
    rot[4 * k] = posMag * std::cos(theta);
    rot[4 * k + 1] = posMag * std::sin(theta);
    rot[4 * k + 2] = -0.1 * std::cos(theta);
    rot[4 * k + 3] = -0.1 * std::sin(theta);
  }
  if (cudaMalloc(&dpts, nrays * 3 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&drot, rot.size() * sizeof(double)) != cudaSuccess ||
      cudaMemcpy(drot, rot.data(), rot.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
    cleanup();
    cudaGetLastError();
    return CCS_ERR_NOMEM;
  }
  eq_rays_kernel<<<(unsigned)nrays, EQ_THREADS>>>(A, ek, zMax, levels, nrot, drot, dpts, derr);
  const bool ok = cudaGetLastError() == cudaSuccess && cudaDeviceSynchronize() == cudaSuccess &&
                  cudaMemcpy(pts, dpts, nrays * 3 * sizeof(double), cudaMemcpyDeviceToHost) == cudaSuccess &&
                  cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess;
  cleanup();
  if (!ok) return CCS_ERR_CUDA;
  return herr ? CCS_ERR_TIMEOUT : CCS_OK;
}
