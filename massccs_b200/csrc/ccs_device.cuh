// ccs_device.cuh -- device code of the B200 trajectory engine.
//
// One persistent kernel runs the reference's trajectory loop
// (cces-cepid/massccs src/System.cpp:204-285): each group of G lanes
// (G = 1..32, a power of two) owns one trajectory at a time, takes the next
// trajectory index from a global work counter when it finishes, and runs
//   System::setup            (src/System.cpp:1397-1518, in FP64)
//   run_He / run_N2 / run_CO2 (src/System.cpp:338-1392, in T = float or double)
// with every site force of a step evaluated in one fused pass over the target
// atoms near the probe (src/Force.cpp:34-1725 semantics: LJ inside lj_cutoff,
// shifted Coulomb and the smoothed ion-induced dipole inside coul_cutoff).
//
// The reference walks 12.01 A cells with a fixed stencil; the physics it
// computes is the cutoff sum over all atoms closer than the cutoffs.  The
// engine enumerates a superset of those atoms from its own grid (z-sorted
// cells, one contiguous atom run per (x,y) column clipped to the sphere of
// the largest reach around the probe) and applies the exact cutoff tests per
// pair, so it sums the same set.  The reference's "site outside the cell grid
// -> zero force" rule (Force.cpp:58-66) is kept per site.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ccs {

constexpr int GAS_ATOM = 0;  // He, Ar, "co2": one site
constexpr int GAS_N2 = 1;    // N, N, central charge
constexpr int GAS_CO2 = 2;   // O, C, O

constexpr double KCALMOLANGAMU_TO_ANGFS2 = 1.0 / 48.88821291 / 48.88821291;
constexpr double AMUANGFS2_TO_KCAL_MOL = 2390.07;
constexpr double KCOUL = 332.06348078020324;
constexpr double BOLTZMANN_K = 1.38064E-23;
constexpr double OMEGA_TO_FS_INV = 2.45400505E8;
constexpr double PI_D = 3.14159265358979323846;

// Per-launch parameters (passed by value).
struct KParams {
  // target atoms, sorted by engine cell (z fastest within a column)
  const float4 *xyzq32;   // x, y, z, q
  const float2 *ab32;     // A = 4 eps sig^12, B = 4 eps sig^6 (primary LJ sites)
  const float2 *abc32;    // same for the CO2 carbon site
  const double4 *xyzq64;
  const double2 *ab64;
  const double2 *abc64;
  const int *cell_start;  // nx*ny*nz + 1
  int nx, ny, nz, natoms;
  double ox, oy, oz, h, inv_h;
  double bb_lo[3], bb_hi[3];
  double reach;           // largest site reach (cutoff of any active term), A
  int allpairs;           // force types 1/3/5: no cutoffs, no shifts
  int coul_on, dip_on;    // Coulomb / dipole terms present (and target charged)
  double q_site[3];
  double rlj2, rc2, rc6inv, rc12inv, rc3inv, c1, c2, alpha;
  // reference grid (LinkedCell.cpp:48-90) for the out-of-grid rule
  double ref_corner[3], ref_h;
  int ref_nx, ref_ny, ref_nz, ref_check;
  // dynamics
  int gas;                // ccs_gas numbering (1..5)
  double dt, mu, temperature, gas_inertia, d_bond, a, b, c, bmax, lx, ly, lz;
  double gas_m[3], gas_z[3], gas_mass;
  double etol;            // energy tolerance in percent
  int quirks;
  uint32_t max_steps;
  unsigned long long deadline_ns;
  // speed sampler table (System.cpp:1537-1555)
  const double *vtab_v, *vtab_s;
  int vtab_n;
  // work
  const double *rnd;
  size_t rnd_stride, ntraj;
  int8_t *status;
  double *omc;
  uint32_t *steps;
  uint32_t *visits;
  unsigned long long *work;   // [0] next trajectory
  unsigned long long *stats;  // nfree, nscatter, nlost, ncapped, steps, visits, force_calls
  int *error;                 // 1 = watchdog
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Watchdog test with one answer for the whole group (lane 0 reads the clock),
// so every lane of a group takes the same branch.
template <int G>
__device__ __forceinline__ bool group_expired(const KParams &kp, int g, unsigned mask);

template <typename T> struct Real;
template <> struct Real<float> {
  static __device__ __forceinline__ float rsq(float x) { return rsqrtf(x); }
  static __device__ __forceinline__ float sq(float x) { return sqrtf(x); }
};
template <> struct Real<double> {
  static __device__ __forceinline__ double rsq(double x) { return rsqrt(x); }
  static __device__ __forceinline__ double sq(double x) { return sqrt(x); }
};

template <typename T> struct Atom { T x, y, z, q, A, B, Ac, Bc; };

template <typename T, int GAS>
__device__ __forceinline__ Atom<T> load_atom(const KParams &kp, int i) {
  Atom<T> a;
  if constexpr (sizeof(T) == 4) {
    float4 p = __ldg(&kp.xyzq32[i]);
    float2 ab = __ldg(&kp.ab32[i]);
    a.x = p.x; a.y = p.y; a.z = p.z; a.q = p.w; a.A = ab.x; a.B = ab.y;
    if constexpr (GAS == GAS_CO2) { float2 c = __ldg(&kp.abc32[i]); a.Ac = c.x; a.Bc = c.y; }
  } else {
    double4 p = kp.xyzq64[i];
    double2 ab = kp.ab64[i];
    a.x = p.x; a.y = p.y; a.z = p.z; a.q = p.w; a.A = ab.x; a.B = ab.y;
    if constexpr (GAS == GAS_CO2) { double2 c = kp.abc64[i]; a.Ac = c.x; a.Bc = c.y; }
  }
  return a;
}

template <int GAS> struct GasShape;
template <> struct GasShape<GAS_ATOM> { static constexpr int NS = 1, DIP = 0; };
template <> struct GasShape<GAS_N2> { static constexpr int NS = 3, DIP = 2; };
template <> struct GasShape<GAS_CO2> { static constexpr int NS = 3, DIP = 1; };

// Site layout: which sites carry LJ, and with which parameter set.
template <int GAS> __device__ __forceinline__ constexpr int site_lj(int s) {
  return GAS == GAS_ATOM ? 1 : GAS == GAS_N2 ? (s < 2 ? 1 : 0) : (s == 1 ? 2 : 1);
}
template <int GAS> __device__ __forceinline__ constexpr bool site_coul(int s) {
  return GAS != GAS_ATOM;  // atomic probes are neutral
}

// Accumulators of one fused force evaluation.
template <typename T, int NS> struct Acc {
  T f[NS][3], U[NS];
  T E[3], G[6];  // field and symmetric gradient (xx yy zz xy xz yz) at the dipole site
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int s = 0; s < NS; s++) { f[s][0] = f[s][1] = f[s][2] = U[s] = T(0); }
#pragma unroll
    for (int k = 0; k < 3; k++) E[k] = T(0);
#pragma unroll
    for (int k = 0; k < 6; k++) G[k] = T(0);
  }
};

// Group-wide xor reduction: every lane ends with the same bits (a+b == b+a).
template <int G, typename T> __device__ __forceinline__ T group_sum(T v, unsigned mask) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, G);
  return v;
}

// One target atom against every active site (the pair terms of Force.cpp).
template <typename T, int GAS, bool HASQ>
__device__ __forceinline__ void visit_atom(const KParams &kp, const T (&p)[GasShape<GAS>::NS][3],
                                           const bool (&act)[GasShape<GAS>::NS], const Atom<T> &a,
                                           Acc<T, GasShape<GAS>::NS> &acc) {
  constexpr int NS = GasShape<GAS>::NS;
  const T rlj2 = T(kp.rlj2), rc2 = T(kp.rc2);
#pragma unroll
  for (int s = 0; s < NS; s++) {
    if (!act[s]) continue;
    const T dx = p[s][0] - a.x, dy = p[s][1] - a.y, dz = p[s][2] - a.z;
    const T r2 = dx * dx + dy * dy + dz * dz;
    const int lj = site_lj<GAS>(s);
    const bool in_lj = lj != 0 && r2 < rlj2;
    const bool in_c = HASQ && r2 < rc2;
    if (!(in_lj || in_c)) continue;
    const T ir = Real<T>::rsq(r2);
    const T ir2 = ir * ir;
    if (in_lj) {
      // Force.cpp:83-102: U = A/r^12 - B/r^6 - (A/rc^12 - B/rc^6), F = (12A/r^12 - 6B/r^6)/r^2 * d
      const T A = lj == 2 ? a.Ac : a.A, B = lj == 2 ? a.Bc : a.B;
      const T ir6 = ir2 * ir2 * ir2;
      acc.U[s] += ir6 * (A * ir6 - B) - (A * T(kp.rc12inv) - B * T(kp.rc6inv));
      const T fl = ir6 * (T(12) * A * ir6 - T(6) * B) * ir2;
      acc.f[s][0] += fl * dx; acc.f[s][1] += fl * dy; acc.f[s][2] += fl * dz;
    }
    if constexpr (HASQ) {
      if (in_c) {
        const T ir3 = ir * ir2;
        if (site_coul<GAS>(s) && kp.coul_on) {
          // Force.cpp:671-683: U = k qi qj (1/r - 3/(2rc) + r^2/(2rc^3)), F = k qi qj (1/r^3 - 1/rc^3) d
          const T kq = T(KCOUL * kp.q_site[s]) * a.q;
          acc.U[s] += kq * (ir - T(kp.c1) + T(kp.c2) * r2);
          const T fc = kq * (ir3 - T(kp.rc3inv));
          acc.f[s][0] += fc * dx; acc.f[s][1] += fc * dy; acc.f[s][2] += fc * dz;
        }
        if (s == GasShape<GAS>::DIP && kp.dip_on) {
          // Force.cpp:393-426: E += q (1/r^3 - 1/rc^3) d ; dE_ab += q (1/r^3 - 1/rc^3) delta_ab - 3 q d_a d_b / r^5
          const T sq = a.q * (ir3 - T(kp.rc3inv));
          const T tq = T(-3) * a.q * ir3 * ir2;
          acc.E[0] += sq * dx; acc.E[1] += sq * dy; acc.E[2] += sq * dz;
          const T tx = tq * dx, ty = tq * dy;
          acc.G[0] += sq + tx * dx;
          acc.G[1] += sq + ty * dy;
          acc.G[2] += sq + tq * dz * dz;
          acc.G[3] += tx * dy;
          acc.G[4] += tx * dz;
          acc.G[5] += ty * dz;
        }
      }
    }
  }
}

// Reference-grid test of Force.cpp:56-66 (LinkedCell::calculateIndex, LinkedCell.cpp:117-129).
template <typename T>
__device__ __forceinline__ bool ref_inside(const KParams &kp, T x, T y, T z) {
  if (!kp.ref_check) return true;
  const double h = kp.ref_h;
  const long i = (long)floor(((double)x - kp.ref_corner[0]) / h);
  const long j = (long)floor(((double)y - kp.ref_corner[1]) / h);
  const long k = (long)floor(((double)z - kp.ref_corner[2]) / h);
  const long idx = k + (long)kp.ref_nz * j + (long)kp.ref_nz * kp.ref_ny * i;
  return idx >= 0 && idx < (long)kp.ref_nx * kp.ref_ny * kp.ref_nz;
}

// Site forces of one probe configuration.  All G lanes of the group call it
// with identical arguments; each lane gets the identical result.
//   p       site positions, act: sites that feel the target
//   cen     centre of the sites, off: largest |p_s - cen|
template <typename T, int G, int GAS, bool HASQ>
__device__ __forceinline__ void eval_forces(const KParams &kp, const T (&p)[GasShape<GAS>::NS][3],
                                         const bool (&act)[GasShape<GAS>::NS], const T (&cen)[3],
                                         T off, T (&f)[GasShape<GAS>::NS][3],
                                         T (&U)[GasShape<GAS>::NS], uint32_t &visits, int g,
                                         unsigned mask, int *sm_end, int *sm_del) {
  constexpr int NS = GasShape<GAS>::NS;
  Acc<T, NS> acc;
  acc.zero();
  bool any = false;
#pragma unroll
  for (int s = 0; s < NS; s++) any |= act[s];
  uint32_t nvis = 0;
  if (any) {
    // candidate sphere around the centre; +1e-3 A so rounding never drops a pair
    const T R = kp.allpairs ? T(INFINITY) : T(kp.reach) + off + T(1e-3);
    const T cx = cen[0], cy = cen[1], cz = cen[2];
    const T ex = fmax(fmax(T(kp.bb_lo[0]) - cx, cx - T(kp.bb_hi[0])), T(0));
    const T ey = fmax(fmax(T(kp.bb_lo[1]) - cy, cy - T(kp.bb_hi[1])), T(0));
    const T ez = fmax(fmax(T(kp.bb_lo[2]) - cz, cz - T(kp.bb_hi[2])), T(0));
    if (ex * ex + ey * ey + ez * ez <= R * R) {
      const T ih = T(kp.inv_h), h = T(kp.h), ox = T(kp.ox), oy = T(kp.oy), oz = T(kp.oz);
      const int i0 = (int)fmax(T(0), floor((cx - R - ox) * ih));
      const int i1 = (int)fmin(T(kp.nx - 1), floor((cx + R - ox) * ih));
      const int j0 = (int)fmax(T(0), floor((cy - R - oy) * ih));
      const int j1 = (int)fmin(T(kp.ny - 1), floor((cy + R - oy) * ih));
      const int nj = j1 - j0 + 1;
      const int ncol = (i1 >= i0 && nj > 0) ? (i1 - i0 + 1) * nj : 0;
      for (int base = 0; base < ncol; base += G) {
        const int cidx = base + g;
        int b = 0, len = 0;
        if (cidx < ncol) {
          const int i = i0 + cidx / nj, j = j0 + cidx % nj;
          const T xlo = ox + T(i) * h, ylo = oy + T(j) * h;
          const T dxc = fmax(fmax(xlo - cx, cx - (xlo + h)), T(0));
          const T dyc = fmax(fmax(ylo - cy, cy - (ylo + h)), T(0));
          const T rem = R * R - dxc * dxc - dyc * dyc;
          if (rem >= T(0)) {
            const T zr = Real<T>::sq(rem);
            const int k0 = (int)fmax(T(0), floor((cz - zr - oz) * ih));
            const int k1 = (int)fmin(T(kp.nz - 1), floor((cz + zr - oz) * ih));
            if (k0 <= k1) {
              const int cb = (i * kp.ny + j) * kp.nz;
              b = __ldg(&kp.cell_start[cb + k0]);
              len = __ldg(&kp.cell_start[cb + k1 + 1]) - b;
            }
          }
        }
        if constexpr (G == 1) {
          nvis += (uint32_t)len;
          for (int ai = b; ai < b + len; ai++) {
            const Atom<T> a = load_atom<T, GAS>(kp, ai);
            visit_atom<T, GAS, HASQ>(kp, p, act, a, acc);
          }
        } else {
          // flatten the G runs of this chunk: inclusive scan of run lengths
          int incl = len;
#pragma unroll
          for (int o = 1; o < G; o <<= 1) {
            const int v = __shfl_up_sync(mask, incl, o, G);
            if (g >= o) incl += v;
          }
          const int total = __shfl_sync(mask, incl, G - 1, G);
          if (total == 0) continue;
          sm_end[g] = incl;
          sm_del[g] = b - (incl - len);
          __syncwarp(mask);
          int r = 0, cur_end = sm_end[0], cur_del = sm_del[0];
          for (int t = g; t < total; t += G) {
            while (t >= cur_end) { ++r; cur_end = sm_end[r]; cur_del = sm_del[r]; }
            const Atom<T> a = load_atom<T, GAS>(kp, t + cur_del);
            visit_atom<T, GAS, HASQ>(kp, p, act, a, acc);
          }
          if (g == 0) nvis += (uint32_t)total;
          __syncwarp(mask);
        }
      }
    }
  }
  if constexpr (G > 1) {
#pragma unroll
    for (int s = 0; s < NS; s++) {
      acc.U[s] = group_sum<G>(acc.U[s], mask);
#pragma unroll
      for (int k = 0; k < 3; k++) acc.f[s][k] = group_sum<G>(acc.f[s][k], mask);
    }
    if (HASQ && kp.dip_on) {
#pragma unroll
      for (int k = 0; k < 3; k++) acc.E[k] = group_sum<G>(acc.E[k], mask);
#pragma unroll
      for (int k = 0; k < 6; k++) acc.G[k] = group_sum<G>(acc.G[k], mask);
    }
  }
#pragma unroll
  for (int s = 0; s < NS; s++) {
    f[s][0] = acc.f[s][0]; f[s][1] = acc.f[s][1]; f[s][2] = acc.f[s][2]; U[s] = acc.U[s];
  }
  if (HASQ && kp.dip_on) {
    // Force.cpp:483-487: f += alpha (E . grad) E ; U -= alpha/2 |E|^2
    constexpr int d = GasShape<GAS>::DIP;
    const T al = T(kp.alpha);
    const T *E = acc.E, *Gr = acc.G;
    f[d][0] += al * (E[0] * Gr[0] + E[1] * Gr[3] + E[2] * Gr[4]);
    f[d][1] += al * (E[0] * Gr[3] + E[1] * Gr[1] + E[2] * Gr[5]);
    f[d][2] += al * (E[0] * Gr[4] + E[1] * Gr[5] + E[2] * Gr[2]);
    U[d] -= T(0.5) * al * (E[0] * E[0] + E[1] * E[1] + E[2] * E[2]);
  }
#pragma unroll
  for (int s = 0; s < NS; s++)
    if (!act[s]) { f[s][0] = f[s][1] = f[s][2] = U[s] = T(0); }
  visits += nvis;
}

// ---- initial conditions: System::setup (System.cpp:1397-1518), FP64 -------
__device__ __forceinline__ double vel_sample(const KParams &kp, double u) {
  // smallest k with S[k] >= u (the reference's linear scan, System.cpp:1549-1552)
  int lo = 0, hi = kp.vtab_n - 1;
  if (!(kp.vtab_s[hi] >= u)) return kp.vtab_v[hi];
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (kp.vtab_s[mid] >= u) hi = mid;
    else lo = mid + 1;
  }
  return kp.vtab_v[lo];
}

// Rz(gamma) Ry(phi) Rz(theta) as System::rotate (System.cpp:1583-1619)
__device__ __forceinline__ void rot3(double r[3], double v[3], double a0, double a1, double a2) {
  double c = cos(a0), s = sin(a0);
  double x = r[0] * c - r[1] * s, y = r[0] * s + r[1] * c;
  r[0] = x; r[1] = y;
  x = v[0] * c - v[1] * s; y = v[0] * s + v[1] * c;
  v[0] = x; v[1] = y;
  c = cos(a1); s = sin(a1);
  x = r[0] * c + r[2] * s; double z = r[0] * -s + r[2] * c;
  r[0] = x; r[2] = z;
  x = v[0] * c + v[2] * s; z = v[0] * -s + v[2] * c;
  v[0] = x; v[2] = z;
  c = cos(a2); s = sin(a2);
  x = r[0] * c - r[1] * s; y = r[0] * s + r[1] * c;
  r[0] = x; r[1] = y;
  x = v[0] * c - v[1] * s; y = v[0] * s + v[1] * c;
  v[0] = x; v[1] = y;
}
// Ry(theta) then Rz(phi) as System::rotate_gas (System.cpp:1624-1638)
__device__ __forceinline__ void rot_gas(double v[3], double theta, double phi) {
  double c = cos(theta), s = sin(theta);
  double x = v[0] * c + v[2] * s, z = v[0] * -s + v[2] * c;
  v[0] = x; v[2] = z;
  c = cos(phi); s = sin(phi);
  x = v[0] * c - v[1] * s; double y = v[0] * s + v[1] * c;
  v[0] = x; v[1] = y;
}

struct Init {
  double pos[3][3], vel[3][3], rcm[3], vcm[3];
};

__device__ bool setup_probe(const KParams &kp, size_t j, Init &I) {
  const double *u = kp.rnd;
  const size_t st = kp.rnd_stride;
  double rcm[3] = {u[j], 0.0, kp.bmax};
  const double vi = vel_sample(kp, u[st + j]);
  double vcm[3] = {0.0, 0.0, -vi};
  rot3(rcm, vcm, 2.0 * PI_D * u[2 * st + j], asin(2.0 * u[3 * st + j] - 1.0) + 0.5 * PI_D,
       2.0 * PI_D * u[4 * st + j]);
  // ray / ellipsoid intersection (System.cpp:1430-1459)
  const double ur[3] = {rcm[0] / kp.a, rcm[1] / kp.b, rcm[2] / kp.c};
  const double uv[3] = {vcm[0] / kp.a, vcm[1] / kp.b, vcm[2] / kp.c};
  const double cr0 = ur[1] * uv[2] - ur[2] * uv[1], cr1 = ur[2] * uv[0] - ur[0] * uv[2],
               cr2 = ur[0] * uv[1] - ur[1] * uv[0];
  const double uvuv = uv[0] * uv[0] + uv[1] * uv[1] + uv[2] * uv[2];
  const double delta = -(cr0 * cr0 + cr1 * cr1 + cr2 * cr2) + uvuv;
  if (delta < 0) return false;
  const double lambda = -(ur[0] * uv[0] + ur[1] * uv[1] + ur[2] * uv[2]) / uvuv - sqrt(delta) / uvuv;
  for (int k = 0; k < 3; k++) { rcm[k] = rcm[k] + lambda * vcm[k]; I.rcm[k] = rcm[k]; I.vcm[k] = vcm[k]; }
  if (kp.gas == 2 || kp.gas == 3) {
    const double theta = asin(2.0 * u[5 * st + j] - 1.0) + 0.5 * PI_D;
    const double phi = 2.0 * PI_D * u[6 * st + j];
    const double psi = 2.0 * PI_D * u[7 * st + j];
    const double omega =
        sqrt(2.0 * BOLTZMANN_K * kp.temperature / kp.gas_inertia * log(1. / (1. - u[8 * st + j]))) *
        OMEGA_TO_FS_INV;
    double w[3] = {omega * cos(psi), omega * sin(psi), 0.0};
    rot_gas(w, theta, phi);
    for (int s = 0; s < 3; s++) {
      double r[3] = {0.0, 0.0, kp.gas_z[s]};
      rot_gas(r, theta, phi);
      I.pos[s][0] = r[0] + rcm[0]; I.pos[s][1] = r[1] + rcm[1]; I.pos[s][2] = r[2] + rcm[2];
      I.vel[s][0] = (w[1] * r[2] - w[2] * r[1]) + vcm[0];
      I.vel[s][1] = (w[2] * r[0] - w[0] * r[2]) + vcm[1];
      I.vel[s][2] = (w[0] * r[1] - w[1] * r[0]) + vcm[2];
    }
  } else {
    for (int k = 0; k < 3; k++) { I.pos[0][k] = rcm[k]; I.vel[0][k] = vcm[k]; }
  }
  return true;
}

template <int G>
__device__ __forceinline__ bool group_expired(const KParams &kp, int g, unsigned mask) {
  int e = 0;
  if (g == 0) e = global_ns() > kp.deadline_ns;
  if constexpr (G > 1) e = __shfl_sync(mask, e, 0, G);
  return e != 0;
}

// ---- shared integrator pieces -----------------------------------------------
template <typename T> __device__ __forceinline__ T dot3(const T a[3], const T b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
// angle between position vectors (System::anglevec, System.cpp:1566-1579).
// FP64 keeps the reference's acos form; FP32 uses atan2(|a x b|, a.b), the
// same angle without acos's loss near 0.
template <typename T> __device__ __forceinline__ T angle3(const T a[3], const T b[3]) {
  if constexpr (sizeof(T) == 8) {
    const double arg = dot3(a, b) / (sqrt(dot3(a, a)) * sqrt(dot3(b, b)));
    return fabs(arg) > 1.0 ? 0.0 : acos(arg);
  } else {
    const float cx = a[1] * b[2] - a[2] * b[1], cy = a[2] * b[0] - a[0] * b[2],
                cz = a[0] * b[1] - a[1] * b[0];
    return atan2f(sqrtf(cx * cx + cy * cy + cz * cz), dot3(a, b));
  }
}
// 1 - cos(chi) between the initial and final centre-of-mass velocities.
// FP64 mode: 1 - cos(acos(arg)) as the reference (System.cpp:220);
// FP32 mode: |u_i - u_f|^2 / 2 of the unit vectors, in FP64 (no cancellation).
template <typename T>
__device__ __forceinline__ double one_minus_cos(const double vi[3], const T vf[3]) {
  const double f[3] = {(double)vf[0], (double)vf[1], (double)vf[2]};
  const double ni = sqrt(vi[0] * vi[0] + vi[1] * vi[1] + vi[2] * vi[2]);
  const double nf = sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
  if constexpr (sizeof(T) == 8) {
    const double arg = (vi[0] * f[0] + vi[1] * f[1] + vi[2] * f[2]) / (ni * nf);
    const double chi = fabs(arg) > 1.0 ? 0.0 : acos(arg);
    return 1.0 - cos(chi);
  } else {
    const double d0 = vi[0] / ni - f[0] / nf, d1 = vi[1] / ni - f[1] / nf, d2 = vi[2] / ni - f[2] / nf;
    return 0.5 * (d0 * d0 + d1 * d1 + d2 * d2);
  }
}
template <typename T> __device__ __forceinline__ bool outside_box(const KParams &kp, const T r[3]) {
  if (fabs(r[0]) >= T(kp.lx) || fabs(r[1]) >= T(kp.ly) || fabs(r[2]) >= T(kp.lz)) return true;
  const T ux = r[0] / T(kp.a), uy = r[1] / T(kp.b), uz = r[2] / T(kp.c);
  return ux * ux + uy * uy + uz * uz > T(1);
}

struct TrajOut {
  int8_t status;
  double omc;
  uint32_t steps, visits, calls;
};

// ---- run_He (System.cpp:338-511): He, Ar, "co2" ------------------------------
template <typename T, int G, bool HASQ>
__device__ void run_atom(const KParams &kp, size_t j, int g, unsigned mask, int *sm_e, int *sm_d,
                         TrajOut &o) {
  Init I;
  if (!setup_probe(kp, j, I)) { o.status = 0; return; }
  const double vi64[3] = {I.vel[0][0], I.vel[0][1], I.vel[0][2]};
  const T ri[3] = {T(I.pos[0][0]), T(I.pos[0][1]), T(I.pos[0][2])};
  const T vi[3] = {T(vi64[0]), T(vi64[1]), T(vi64[2])};
  const T mu = T(kp.mu), kconv = T(KCALMOLANGAMU_TO_ANGFS2), ke = T(AMUANGFS2_TO_KCAL_MOL);
  T p[1][3], f[1][3], U[1], fi[3];
  bool act[1];
  for (int k = 0; k < 3; k++) p[0][k] = ri[k];
  act[0] = ref_inside(kp, p[0][0], p[0][1], p[0][2]);
  eval_forces<T, G, GAS_ATOM, HASQ>(kp, p, act, p[0], T(0), f, U, o.visits, g, mask, sm_e, sm_d);
  o.calls++;
  for (int k = 0; k < 3; k++) fi[k] = f[0][k];
  const T Ei = U[0] + T(0.5) * mu * dot3(vi, vi) * ke;
  const T theta_max = T(1.5 * PI_D);
  T r[3], rlo[3], v[3], rold[3], dtheta = T(0);
  T dt = T(kp.dt);
  int tries = 0, maxTries = 8;
  uint32_t stepcount = 0;
  while (tries < maxTries && maxTries < 10) {
    if (stepcount == 0) {
      for (int k = 0; k < 3; k++) { r[k] = ri[k]; rlo[k] = T(0); v[k] = vi[k]; rold[k] = ri[k]; f[0][k] = fi[k]; }
      dtheta = T(0);
    }
    const T kick = T(0.5) * dt / mu * kconv;
    for (int k = 0; k < 3; k++) {
      v[k] += kick * f[0][k];
      // compensated position update (Kahan): r + rlo tracks the exact sum
      const T y = dt * v[k] - rlo[k];
      const T t = r[k] + y;
      rlo[k] = (t - r[k]) - y;
      r[k] = t;
    }
    dtheta += angle3(r, rold);
    for (int k = 0; k < 3; k++) { rold[k] = r[k]; p[0][k] = r[k]; }
    act[0] = ref_inside(kp, r[0], r[1], r[2]);
    eval_forces<T, G, GAS_ATOM, HASQ>(kp, p, act, p[0], T(0), f, U, o.visits, g, mask, sm_e, sm_d);
    o.calls++;
    for (int k = 0; k < 3; k++) v[k] += kick * f[0][k];
    stepcount++;
    o.steps++;
    if (dtheta > theta_max) {
      tries++;
      dt = T(kp.dt / (tries + 1));
      stepcount = 0;
      continue;
    }
    if (outside_box(kp, r)) {
      const double E = (double)U[0] + (double)(T(0.5) * mu * dot3(v, v) * ke);
      const double dE = fabs(E - (double)Ei) / (double)Ei * 100.0;
      if (dE > kp.etol) {
        tries++;
        maxTries++;
        dt = T(kp.dt / (tries + 1));
        stepcount = 0;
        continue;
      }
      o.status = 1;
      o.omc = one_minus_cos<T>(vi64, v);
      return;
    }
    if (stepcount >= kp.max_steps) { o.status = 3; return; }
    if ((o.steps & 4095u) == 0 && group_expired<G>(kp, g, mask)) {
      if (g == 0) atomicExch(kp.error, 1);
      o.status = 3;
      return;
    }
  }
  o.status = 2;
}

// ---- run_N2 (System.cpp:514-945) and run_CO2 (System.cpp:948-1392) ----------
template <typename T, int G, int GAS, bool HASQ>
__device__ void run_molecule(const KParams &kp, size_t j, int g, unsigned mask, int *sm_e,
                             int *sm_d, TrajOut &o) {
  constexpr bool co2 = GAS == GAS_CO2;
  constexpr int pa = 0, pb = co2 ? 2 : 1, pc = co2 ? 1 : 2;
  Init I;
  if (!setup_probe(kp, j, I)) { o.status = 0; return; }
  double vcm_i[3] = {I.vcm[0], I.vcm[1], I.vcm[2]};
  if (co2 && (kp.quirks & 1)) vcm_i[0] = I.vcm[1];  // System.cpp:1012
  const T ma = T(kp.gas_m[pa]), mb = T(kp.gas_m[pb]), mc = T(kp.gas_m[pc]), M = T(kp.gas_mass);
  const T kconv = T(KCALMOLANGAMU_TO_ANGFS2), ke = T(AMUANGFS2_TO_KCAL_MOL);
  const T d2 = T(kp.d_bond * kp.d_bond), theta_max = T(1.5 * PI_D);
  T ri[3], rj[3], vi[3], vj[3], fg[3][3], Ug[3], pos[3][3], rold[3], rilo[3], rjlo[3];
  bool act[3];
  T Ei = T(0), dtheta = T(0), dt = T(kp.dt);
  int tries = 0, maxTries = 8;
  uint32_t stepcount = 0;
  bool first = true;
  while (tries < maxTries && maxTries < 10) {
    if (stepcount == 0) {
      // restart from the initial conditions (recomputed: identical bits every time)
      if (!first) setup_probe(kp, j, I);
      for (int s = 0; s < 3; s++)
        for (int k = 0; k < 3; k++) pos[s][k] = T(I.pos[s][k]);
      for (int k = 0; k < 3; k++) {
        ri[k] = pos[pa][k]; rj[k] = pos[pb][k]; rilo[k] = rjlo[k] = T(0);
        vi[k] = T(I.vel[pa][k]); vj[k] = T(I.vel[pb][k]); rold[k] = T(I.rcm[k]);
      }
      for (int s = 0; s < 3; s++) act[s] = kp.allpairs || ref_inside(kp, pos[s][0], pos[s][1], pos[s][2]);
      const T cen[3] = {pos[pc][0], pos[pc][1], pos[pc][2]};
      eval_forces<T, G, GAS, HASQ>(kp, pos, act, cen, T(0.5) * T(kp.d_bond), fg, Ug, o.visits, g,
                                   mask, sm_e, sm_d);
      o.calls += 3;
      if (first) {
        // initial energy: every site's kinetic energy (System.cpp:648-660, 1076-1088)
        T ek = T(0);
        for (int s = 0; s < 3; s++) {
          const T vs[3] = {T(I.vel[s][0]), T(I.vel[s][1]), T(I.vel[s][2])};
          ek += T(0.5) * T(kp.gas_m[s]) * dot3(vs, vs) * ke;
        }
        Ei = Ug[0] + Ug[1] + Ug[2] + ek;
        first = false;
      }
      dtheta = T(0);
    }
    // pair forces: N2 splits the central charge half/half (System.cpp:736-739);
    // CO2 redistributes the carbon force (Ciccotti, System.cpp:1154-1158)
    T fi[3], fj[3];
    if constexpr (co2) {
      const T m2M = mc / M, m0M = ma / M;
      for (int k = 0; k < 3; k++) {
        fi[k] = (T(1) - T(0.5) * m2M) * fg[0][k] + m0M * fg[1][k] - T(0.5) * m2M * fg[2][k];
        fj[k] = (T(1) - T(0.5) * m2M) * fg[2][k] + m0M * fg[1][k] - T(0.5) * m2M * fg[0][k];
      }
    } else {
      for (int k = 0; k < 3; k++) { fi[k] = fg[0][k] + T(0.5) * fg[2][k]; fj[k] = fg[1][k] + T(0.5) * fg[2][k]; }
    }
    // first half of the constrained Verlet (System.cpp:1700-1739)
    {
      const T mu_ij = ma * mb / (ma + mb);
      T vci[3], vcj[3], rij[3], rcij[3];
      for (int k = 0; k < 3; k++) {
        vci[k] = vi[k] + T(0.5) * dt / ma * fi[k] * kconv;
        vcj[k] = vj[k] + T(0.5) * dt / mb * fj[k] * kconv;
        rij[k] = ri[k] - rj[k];
        rcij[k] = rij[k] + dt * (vci[k] - vcj[k]);
      }
      const T r2ij = dot3(rij, rij), rc2ij = dot3(rcij, rcij), rr = dot3(rcij, rij);
      T det = rr * rr - r2ij * (rc2ij - d2);
      if (det < T(0)) det = T(0);
      const T lam = (rr - Real<T>::sq(det)) / r2ij;
      const T ca = mu_ij / ma * lam, cb = mu_ij / ma * lam;  // the reference uses mi twice (:1735-1736)
      for (int k = 0; k < 3; k++) {
        vi[k] = vci[k] - mu_ij / (ma * dt) * lam * rij[k];
        vj[k] = vcj[k] + mu_ij / (mb * dt) * lam * rij[k];
        // compensated position updates
        T y = (dt * vci[k] - ca * rij[k]) - rilo[k];
        T t = ri[k] + y;
        rilo[k] = (t - ri[k]) - y;
        ri[k] = t;
        y = (dt * vcj[k] + cb * rij[k]) - rjlo[k];
        t = rj[k] + y;
        rjlo[k] = (t - rj[k]) - y;
        rj[k] = t;
      }
    }
    T rcm[3], vcm[3];
    for (int k = 0; k < 3; k++) { rcm[k] = T(0.5) * (ri[k] + rj[k]); vcm[k] = T(0.5) * (vi[k] + vj[k]); }
    dtheta += angle3(rcm, rold);
    for (int k = 0; k < 3; k++) {
      rold[k] = rcm[k];
      pos[pa][k] = ri[k]; pos[pb][k] = rj[k]; pos[pc][k] = rcm[k];
    }
    for (int s = 0; s < 3; s++) act[s] = kp.allpairs || ref_inside(kp, pos[s][0], pos[s][1], pos[s][2]);
    {
      T hd[3] = {ri[0] - rj[0], ri[1] - rj[1], ri[2] - rj[2]};
      const T off = T(0.5) * Real<T>::sq(dot3(hd, hd));
      eval_forces<T, G, GAS, HASQ>(kp, pos, act, rcm, off, fg, Ug, o.visits, g, mask, sm_e, sm_d);
      o.calls += 3;
    }
    if constexpr (co2) {
      const T m2M = mc / M, m0M = ma / M;
      for (int k = 0; k < 3; k++) {
        fi[k] = (T(1) - T(0.5) * m2M) * fg[0][k] + m0M * fg[1][k] - T(0.5) * m2M * fg[2][k];
        fj[k] = (T(1) - T(0.5) * m2M) * fg[2][k] + m0M * fg[1][k] - T(0.5) * m2M * fg[0][k];
      }
    } else {
      for (int k = 0; k < 3; k++) { fi[k] = fg[0][k] + T(0.5) * fg[2][k]; fj[k] = fg[1][k] + T(0.5) * fg[2][k]; }
    }
    // second half (RATTLE velocity correction, System.cpp:1741-1767)
    {
      const T mu_ij = ma * mb / (ma + mb);
      T vci[3], vcj[3], rij[3], vcij[3];
      for (int k = 0; k < 3; k++) {
        vci[k] = vi[k] + T(0.5) * dt / ma * fi[k] * kconv;
        vcj[k] = vj[k] + T(0.5) * dt / mb * fj[k] * kconv;
        rij[k] = ri[k] - rj[k];
        vcij[k] = vci[k] - vcj[k];
      }
      const T lam = mu_ij * dot3(rij, vcij) / dot3(rij, rij);
      for (int k = 0; k < 3; k++) { vi[k] = vci[k] - lam / ma * rij[k]; vj[k] = vcj[k] + lam / mb * rij[k]; }
    }
    for (int k = 0; k < 3; k++) vcm[k] = T(0.5) * (vi[k] + vj[k]);
    stepcount++;
    o.steps++;
    if (dtheta > theta_max) {
      tries++;
      dt = T(kp.dt / (tries + 1));
      stepcount = 0;
      continue;
    }
    if (outside_box(kp, rcm)) {
      // N2: kinetic energy of the two N atoms (System.cpp:890-896);
      // CO2: all three sites, the carbon moving with the centre (System.cpp:1333-1339)
      T ek = T(0.5) * ma * dot3(vi, vi) * ke + T(0.5) * mb * dot3(vj, vj) * ke;
      if (co2) ek += T(0.5) * mc * dot3(vcm, vcm) * ke;
      const double E = (double)Ug[0] + (double)Ug[1] + (double)Ug[2] + (double)ek;
      const double dE = fabs((E - (double)Ei) / (double)Ei) * 100.0;
      if (dE > kp.etol) {
        tries++;
        maxTries++;
        dt = T(kp.dt / (tries + 1));
        stepcount = 0;
        continue;
      }
      o.status = 1;
      o.omc = one_minus_cos<T>(vcm_i, vcm);
      return;
    }
    if (stepcount >= kp.max_steps) { o.status = 3; return; }
    if ((o.steps & 4095u) == 0 && group_expired<G>(kp, g, mask)) {
      if (g == 0) atomicExch(kp.error, 1);
      o.status = 3;
      return;
    }
  }
  o.status = 2;
}

// ---- the persistent trajectory kernel ----------------------------------------
constexpr int MAX_BLOCK = 256;

template <typename T, int G, int GAS, bool HASQ>
__global__ void __launch_bounds__(MAX_BLOCK) traj_kernel(KParams kp) {
  __shared__ int sm_end[MAX_BLOCK], sm_del[MAX_BLOCK];
  __shared__ unsigned long long blk[7];
  if (threadIdx.x < 7) blk[threadIdx.x] = 0ull;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int g = lane & (G - 1);
  const unsigned mask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << (lane & ~(G - 1)));
  int *sme = sm_end + (threadIdx.x & ~(G - 1));
  int *smd = sm_del + (threadIdx.x & ~(G - 1));
  unsigned long long cnt[7] = {0, 0, 0, 0, 0, 0, 0};
  for (;;) {
    // lane 0 takes the next trajectory (or stops the group after a watchdog
    // expiry); the decision is broadcast so the whole group leaves together
    unsigned long long jj = 0;
    if (g == 0) jj = *(volatile int *)kp.error ? kp.ntraj : atomicAdd(kp.work, 1ull);
    if constexpr (G > 1) jj = __shfl_sync(mask, jj, 0, G);
    if (jj >= kp.ntraj) break;
    const size_t j = (size_t)jj;
    TrajOut o{0, 0.0, 0u, 0u, 0u};
    if constexpr (GAS == GAS_ATOM) run_atom<T, G, HASQ>(kp, j, g, mask, sme, smd, o);
    else run_molecule<T, G, GAS, HASQ>(kp, j, g, mask, sme, smd, o);
    if (g == 0) {
      kp.status[j] = o.status;
      kp.omc[j] = o.status == 1 ? o.omc : 0.0;
      if (kp.steps) kp.steps[j] = o.steps;
      if (kp.visits) kp.visits[j] = o.visits;
      cnt[o.status < 4 ? o.status : 3]++;
      cnt[4] += o.steps;
      cnt[5] += o.visits;
      cnt[6] += o.calls;
    }
  }
  if (g == 0) {
    for (int k = 0; k < 7; k++)
      if (cnt[k]) atomicAdd(&blk[k], cnt[k]);
  }
  __syncthreads();
  if (threadIdx.x < 7 && blk[threadIdx.x]) atomicAdd(&kp.stats[threadIdx.x], blk[threadIdx.x]);
}

// Site-force evaluation at given points (ccs_eval_site_forces): one group per point.
template <typename T, int G, int GAS, bool HASQ>
__global__ void __launch_bounds__(MAX_BLOCK)
    force_points_kernel(KParams kp, int site, size_t npts, const double *pts, double *f, double *U,
                        uint32_t *vis) {
  constexpr int NS = GasShape<GAS>::NS;
  __shared__ int sm_end[MAX_BLOCK], sm_del[MAX_BLOCK];
  const int lane = threadIdx.x & 31;
  const int g = lane & (G - 1);
  const unsigned mask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << (lane & ~(G - 1)));
  const size_t grp = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
  const size_t ngrp = ((size_t)gridDim.x * blockDim.x) / G;
  for (size_t i = grp; i < npts; i += ngrp) {
    T p[NS][3], ff[NS][3], UU[NS], cen[3];
    bool act[NS];
    for (int k = 0; k < 3; k++) cen[k] = T(pts[3 * i + k]);
    for (int s = 0; s < NS; s++) {
      for (int k = 0; k < 3; k++) p[s][k] = cen[k];
      act[s] = (s == site) && (kp.allpairs || ref_inside(kp, cen[0], cen[1], cen[2]));
    }
    uint32_t v = 0;
    eval_forces<T, G, GAS, HASQ>(kp, p, act, cen, T(0), ff, UU, v, g, mask,
                                 sm_end + (threadIdx.x & ~(G - 1)), sm_del + (threadIdx.x & ~(G - 1)));
    if (g == 0) {
      for (int k = 0; k < 3; k++) f[3 * i + k] = (double)ff[site][k];
      U[i] = (double)UU[site];
      if (vis) vis[i] = v;
    }
  }
}

// Initial conditions (ccs_eval_setup): one thread per trajectory.
__global__ void setup_kernel(KParams kp, int8_t *hit, double *pos, double *vel) {
  const size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= kp.ntraj) return;
  Init I;
  const bool h = setup_probe(kp, j, I);
  hit[j] = h ? 1 : 0;
  for (int s = 0; s < 3; s++)
    for (int k = 0; k < 3; k++) {
      pos[9 * j + 3 * s + k] = h ? I.pos[s][k] : 0.0;
      vel[9 * j + 3 * s + k] = h ? I.vel[s][k] : 0.0;
    }
}

}  // namespace ccs
