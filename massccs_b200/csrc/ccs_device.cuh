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

#include "field_device.cuh"

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
  double ref_corner[3], ref_h, ref_inv_h;
  int ref_nx, ref_ny, ref_nz, ref_check;
  // dynamics
  int gas;                // ccs_gas numbering (1..5)
  double dt, mu, temperature, gas_inertia, d_bond, a, b, c, bmax, lx, ly, lz;
  double inv_a, inv_b, inv_c;
  double gas_m[3], gas_z[3], gas_mass;
  double etol;            // energy tolerance in percent
  // integrator constants of the moving pair (atoms: m1 = mu)
  double half_kconv_over_m1, half_kconv_over_m2, inv_m1, inv_m2, mu12, mu12_over_m1, mu12_over_m2;
  int quirks;
  uint32_t max_steps;
  // watchdog: the %globaltimer value after which the kernels stop, written on
  // the device by arm_watchdog just before the passes (no host round trip)
  const unsigned long long *deadline;
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
  const uint32_t *order;      // processing order of the trajectories (longest expected first)
  unsigned long long *work;   // [0] next trajectory
  unsigned long long *stats;  // nfree, nscatter, nlost, ncapped, steps, visits, parked
  // parking of long trajectories (lane pass -> warp pass)
  void *park;                       // LaneState<T>[park_cap]
  unsigned long long *park_count;   // parked so far
  unsigned long long *park_next;    // next parked trajectory to resume
  unsigned long long park_cap;
  uint32_t park_steps;
  int park_drained;                 // 1: park only once every trajectory has been taken
  int lcap;                         // warp pass: candidate-list entries (dynamic shared memory)
  // batched ions: per-ion parameters (their rnd/status/omc/steps/visits point
  // at the ion's first trajectory) and the global index of each ion's first
  // trajectory (nions + 1 entries); unused by single-ion runs
  const struct KParams *ions;
  const unsigned long long *ion_start;
  int nions;
  // speculative retries (see resume_kernel): records of trajectories that
  // failed their second try in the warp pass, the outcome of each remaining
  // try, and the phase of the warp-pass launch (0: parked trajectories,
  // 1: the speculative tries); spec_rec == nullptr: no speculation
  struct SpecRec *spec_rec;
  struct SpecOut *spec_out;
  unsigned long long *spec_count, *spec_next;
  unsigned long long *park_active;  // parked trajectories taken and not yet finished or recorded
  unsigned long long spec_cap;
  int spec_phase;
  int spec_from;  // failed tries after which a warp-pass trajectory is handed over
  unsigned long long spec_max_parked;  // speculate only when at most this many were parked
  int *error;                 // 1 = watchdog, 2 = a tensor-core stage timed out
  FieldK field;               // learned field (field.on == 0: every force exact)
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Sets the run's watchdog deadline to now + budget_ns (one thread, enqueued on
// the run's stream before the trajectory passes).
static __global__ void arm_watchdog(unsigned long long *deadline, unsigned long long budget_ns) {
  *deadline = global_ns() + budget_ns;
}

// A trajectory handed to the speculative phase: it failed try tries - 1 and
// will run tries tries..8 (the reference never runs a tenth: tries < maxTries
// <= 9), all at once, one CTA each.
struct SpecRec {
  double Ei;                  // initial total energy (the same for every try)
  unsigned long long j;
  uint32_t ion, nsteps, nvis; // steps and visits of the tries before
  int tries, maxTries;
  int ready;                  // set (after a fence) once the fields above are written
};

// A record's fields as its writer published them: read past L1 (a record
// is written by another CTA during the same launch).
__device__ __forceinline__ SpecRec load_spec_rec(const SpecRec *p) {
  SpecRec R;
  R.Ei = __ldcg(&p->Ei);
  R.j = __ldcg(&p->j);
  R.ion = __ldcg(&p->ion);
  R.nsteps = __ldcg(&p->nsteps);
  R.nvis = __ldcg(&p->nvis);
  R.tries = __ldcg(&p->tries);
  R.maxTries = __ldcg(&p->maxTries);
  R.ready = 1;
  return R;
}
// The end of one speculative try: 1 scatter (omc valid), 3 capped or watchdog,
// 4 failed the angle test, 5 failed the energy test.
struct SpecOut {
  double omc;
  uint32_t steps, nvis;
  int code, pad;
};
constexpr int SPEC_FROM_MIN = 2;  // the fewest failed tries after which speculation starts
constexpr int SPEC_SLOTS = 9 - SPEC_FROM_MIN;  // tries tries..tries+6 (those above 8 are skipped)

template <typename T> struct Real;
template <> struct Real<float> {
  static __device__ __forceinline__ float rsq(float x) { return rsqrtf(x); }
  static __device__ __forceinline__ float sq(float x) { return sqrtf(x); }
  // quotient for the FP32 integrator (2 ulp; the operands are O(1) and positive-definite)
  static __device__ __forceinline__ float div(float a, float b) { return __fdividef(a, b); }
};
template <> struct Real<double> {
  static __device__ __forceinline__ double rsq(double x) { return rsqrt(x); }
  static __device__ __forceinline__ double sq(double x) { return sqrt(x); }
  static __device__ __forceinline__ double div(double a, double b) { return a / b; }
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

// Accumulators of one fused force evaluation.  In FP32 the site energies
// are summed with Kahan compensation (Uc holds each sum's running rounding
// error): the energy test compares totals of ~1e3 terms to 0.5-1 %, so their
// rounding must stay far below that.
template <typename T, int NS> struct Acc {
  T f[NS][3], U[NS], Uc[NS];
  T E[3], G[6];  // field and symmetric gradient (xx yy zz xy xz yz) at the dipole site
  __device__ __forceinline__ void addU(int s, T v) {
    if constexpr (sizeof(T) == 4) {
      const T y = v - Uc[s];
      const T t = U[s] + y;
      Uc[s] = (t - U[s]) - y;
      U[s] = t;
    } else {
      U[s] += v;
    }
  }
  // the compensated sum of site s
  __device__ __forceinline__ T Usum(int s) const { return sizeof(T) == 4 ? U[s] - Uc[s] : U[s]; }
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int s = 0; s < NS; s++) { f[s][0] = f[s][1] = f[s][2] = U[s] = Uc[s] = T(0); }
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
// Branch-free over the cutoff tests: every term is computed and the ones
// outside their cutoff are selected away (a select, never a multiply, so an
// infinite or NaN term of an excluded pair cannot leak into the sums).  The
// lanes of a warp therefore never diverge on a pair's distance.
//
// SPLIT: the near part of the learned field's range separation -- every term
// weighted by the switch S(r) (field_device.cuh), its force by
// -grad(S u) = S F - u S'(r) d / r, the dipole's field by S e and its
// Jacobian by grad(S e) (still symmetric, since e is along d).
template <typename T, int GAS, bool HASQ, bool SPLIT = false>
__device__ __forceinline__ void visit_atom(const KParams &kp, const T (&p)[GasShape<GAS>::NS][3],
                                           const bool (&act)[GasShape<GAS>::NS], const Atom<T> &a,
                                           Acc<T, GasShape<GAS>::NS> &acc) {
  constexpr int NS = GasShape<GAS>::NS;
  const T rlj2 = T(kp.rlj2), rc2 = T(kp.rc2);
#pragma unroll
  for (int s = 0; s < NS; s++) {
    if (!act[s]) continue;
    T us = T(0);  // this pair's energy at site s (one compensated addition per site)
    const T dx = p[s][0] - a.x, dy = p[s][1] - a.y, dz = p[s][2] - a.z;
    const T r2 = dx * dx + dy * dy + dz * dz;
    const int lj = site_lj<GAS>(s);
    const T ir = Real<T>::rsq(r2);
    const T ir2 = ir * ir;
    T sw = T(1), dsw = T(0);  // S and S'(r) / r
    if constexpr (SPLIT) {
      T dS;
      range_switch(r2 * ir, T(kp.field.r_in), T(kp.field.r_out), sw, dS);
      dsw = dS * ir;
    }
    if (lj != 0) {
      // Force.cpp:83-102: U = A/r^12 - B/r^6 - (A/rc^12 - B/rc^6), F = (12A/r^12 - 6B/r^6)/r^2 * d
      const bool in_lj = r2 < rlj2;
      const T A = lj == 2 ? a.Ac : a.A, B = lj == 2 ? a.Bc : a.B;
      const T ir6 = ir2 * ir2 * ir2;
      const T u = in_lj ? ir6 * (A * ir6 - B) - (A * T(kp.rc12inv) - B * T(kp.rc6inv)) : T(0);
      T fl = in_lj ? ir6 * (T(12) * A * ir6 - T(6) * B) * ir2 : T(0);
      if constexpr (SPLIT) {
        fl = sw * fl - u * dsw;
        us += sw * u;
      } else {
        us += u;
      }
      acc.f[s][0] += fl * dx; acc.f[s][1] += fl * dy; acc.f[s][2] += fl * dz;
    }
    if constexpr (HASQ) {
      const bool in_c = r2 < rc2;
      const T ir3 = ir * ir2;
      if (site_coul<GAS>(s) && kp.coul_on) {
        // Force.cpp:671-683: U = k qi qj (1/r - 3/(2rc) + r^2/(2rc^3)), F = k qi qj (1/r^3 - 1/rc^3) d
        const T kq = T(KCOUL * kp.q_site[s]) * a.q;
        const T u = in_c ? kq * (ir - T(kp.c1) + T(kp.c2) * r2) : T(0);
        T fc = in_c ? kq * (ir3 - T(kp.rc3inv)) : T(0);
        if constexpr (SPLIT) {
          fc = sw * fc - u * dsw;
          us += sw * u;
        } else {
          us += u;
        }
        acc.f[s][0] += fc * dx; acc.f[s][1] += fc * dy; acc.f[s][2] += fc * dz;
      }
      if (s == GasShape<GAS>::DIP && kp.dip_on) {
        // Force.cpp:393-426: E += q (1/r^3 - 1/rc^3) d ; dE_ab += q (1/r^3 - 1/rc^3) delta_ab - 3 q d_a d_b / r^5
        T sq = in_c ? a.q * (ir3 - T(kp.rc3inv)) : T(0);
        T tq = in_c ? T(-3) * a.q * ir3 * ir2 : T(0);
        if constexpr (SPLIT) {  // E = S e, grad E = S grad e + (S'/r) e d^T
          tq = sw * tq + sq * dsw;
          sq = sw * sq;
        }
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
    acc.addU(s, us);
  }
}

// Reference-grid test of Force.cpp:56-66 (LinkedCell::calculateIndex, LinkedCell.cpp:117-129).
template <typename T>
__device__ __forceinline__ bool ref_inside(const KParams &kp, T x, T y, T z) {
  if (!kp.ref_check) return true;
  const T ih = T(kp.ref_inv_h);
  const int i = (int)floor((x - T(kp.ref_corner[0])) * ih);
  const int j = (int)floor((y - T(kp.ref_corner[1])) * ih);
  const int k = (int)floor((z - T(kp.ref_corner[2])) * ih);
  const long long idx = k + (long long)kp.ref_nz * j + (long long)kp.ref_nz * kp.ref_ny * i;
  return idx >= 0 && idx < (long long)kp.ref_nx * kp.ref_ny * kp.ref_nz;
}

// Column (i,j) number cidx of the ncol columns meeting the sphere of radius Rr
// around c: its z-run of atoms [b, b + len) clipped to the sphere.
template <typename T>
__device__ __forceinline__ void column_run(const KParams &kp, int cidx, int ncol, int i0, int j0, int nj,
                                           float inv_nj, T cx, T cy, T cz, T Rr, int &b, int &len) {
  b = 0;
  len = 0;
  if (cidx >= ncol) return;
  const T ih = T(kp.inv_h), h = T(kp.h), ox = T(kp.ox), oy = T(kp.oy), oz = T(kp.oz);
  const int di = (int)(((float)cidx + 0.5f) * inv_nj);  // exact: cidx < 2^20
  const int i = i0 + di, j = j0 + (cidx - di * nj);
  const T xlo = ox + T(i) * h, ylo = oy + T(j) * h;
  const T dxc = fmax(fmax(xlo - cx, cx - (xlo + h)), T(0));
  const T dyc = fmax(fmax(ylo - cy, cy - (ylo + h)), T(0));
  const T rem = Rr * Rr - dxc * dxc - dyc * dyc;
  if (rem < T(0)) return;
  const T zr = Real<T>::sq(rem);
  const int k0 = (int)fmax(T(0), floor((cz - zr - oz) * ih));
  const int k1 = (int)fmin(T(kp.nz - 1), floor((cz + zr - oz) * ih));
  if (k0 > k1) return;
  const int cb = (i * kp.ny + j) * kp.nz;
  b = __ldg(&kp.cell_start[cb + k0]);
  len = __ldg(&kp.cell_start[cb + k1 + 1]) - b;
}

// The (i,j) column range of the sphere of radius Rr around c.
template <typename T>
__device__ __forceinline__ int column_range(const KParams &kp, T cx, T cy, T Rr, int &i0, int &j0, int &nj,
                                            float &inv_nj) {
  const T ih = T(kp.inv_h), ox = T(kp.ox), oy = T(kp.oy);
  i0 = (int)fmax(T(0), floor((cx - Rr - ox) * ih));
  const int i1 = (int)fmin(T(kp.nx - 1), floor((cx + Rr - ox) * ih));
  j0 = (int)fmax(T(0), floor((cy - Rr - oy) * ih));
  const int j1 = (int)fmin(T(kp.ny - 1), floor((cy + Rr - oy) * ih));
  nj = j1 - j0 + 1;
  inv_nj = 1.0f / (float)(nj > 0 ? nj : 1);
  return (i1 >= i0 && nj > 0) ? (i1 - i0 + 1) * nj : 0;
}

// Raw sums of one force evaluation, in row order: per site f (3) and U, then
// the field (3) and its gradient (xx yy zz xy xz yz) at the dipole site.
template <typename T, int NS> __device__ __forceinline__ T acc_value(const Acc<T, NS> &acc, int k) {
  return k < 4 * NS ? (k % 4 == 3 ? acc.Usum(k / 4) : acc.f[k / 4][k % 4])
                    : (k < 4 * NS + 3 ? acc.E[k - 4 * NS] : acc.G[k - 4 * NS - 3]);
}

// Site forces and energies from a row of raw sums: the induced-dipole force
// alpha (E . grad) E and energy -alpha/2 |E|^2 (Force.cpp:483-487) at the
// dipole site; sites outside the reference grid feel nothing.
template <typename T, int GAS, bool HASQ>
__device__ __forceinline__ void finish_row(const KParams &kp, const T *row, const bool (&act)[GasShape<GAS>::NS],
                                           T (&f)[GasShape<GAS>::NS][3], T (&U)[GasShape<GAS>::NS]) {
  constexpr int NS = GasShape<GAS>::NS;
#pragma unroll
  for (int s = 0; s < NS; s++) {
    f[s][0] = row[4 * s]; f[s][1] = row[4 * s + 1]; f[s][2] = row[4 * s + 2]; U[s] = row[4 * s + 3];
  }
  if (HASQ && kp.dip_on) {
    constexpr int d = GasShape<GAS>::DIP;
    const T al = T(kp.alpha);
    const T *E = row + 4 * NS, *Gr = row + 4 * NS + 3;
    f[d][0] += al * (E[0] * Gr[0] + E[1] * Gr[3] + E[2] * Gr[4]);
    f[d][1] += al * (E[0] * Gr[3] + E[1] * Gr[1] + E[2] * Gr[5]);
    f[d][2] += al * (E[0] * Gr[4] + E[1] * Gr[5] + E[2] * Gr[2]);
    U[d] -= T(0.5) * al * (E[0] * E[0] + E[1] * E[1] + E[2] * E[2]);
  }
#pragma unroll
  for (int s = 0; s < NS; s++)
    if (!act[s]) { f[s][0] = f[s][1] = f[s][2] = U[s] = T(0); }
}

// Site forces and energies of a learned-field step: the exact near sums of
// the range separation (row, as finish_row reads it) plus the far parts --
// per site its far potential ufar and force ffar; at the dipole site the
// field E = E_near + E_far and its Jacobian J = J_near + J_far
// (Jf[a][b] = d E_far_a / d x_b), giving the induced-dipole force
// alpha J^T E and energy -alpha/2 |E|^2 (Force.cpp:483-487).
template <typename T, int GAS, bool HASQ>
__device__ __forceinline__ void finish_split(const KParams &kp, const T *row, const float (&ufar)[GasShape<GAS>::NS],
                                             const float (&ffar)[GasShape<GAS>::NS][3], const float (&Ef)[3],
                                             const float (&Jf)[3][3], const bool (&act)[GasShape<GAS>::NS],
                                             T (&f)[GasShape<GAS>::NS][3], T (&U)[GasShape<GAS>::NS]) {
  constexpr int NS = GasShape<GAS>::NS;
#pragma unroll
  for (int s = 0; s < NS; s++) {
#pragma unroll
    for (int k = 0; k < 3; k++) f[s][k] = row[4 * s + k] + T(ffar[s][k]);
    U[s] = row[4 * s + 3] + T(ufar[s]);
  }
  if (HASQ && kp.dip_on) {
    constexpr int d = GasShape<GAS>::DIP;
    const T al = T(kp.alpha);
    const T *En = row + 4 * NS, *Gn = row + 4 * NS + 3;  // near E; near Jacobian xx yy zz xy xz yz
    const T E[3] = {En[0] + T(Ef[0]), En[1] + T(Ef[1]), En[2] + T(Ef[2])};
    const T Jt[3][3] = {{Gn[0] + T(Jf[0][0]), Gn[3] + T(Jf[0][1]), Gn[4] + T(Jf[0][2])},
                        {Gn[3] + T(Jf[1][0]), Gn[1] + T(Jf[1][1]), Gn[5] + T(Jf[1][2])},
                        {Gn[4] + T(Jf[2][0]), Gn[5] + T(Jf[2][1]), Gn[2] + T(Jf[2][2])}};
#pragma unroll
    for (int a = 0; a < 3; a++) f[d][a] += al * (E[0] * Jt[0][a] + E[1] * Jt[1][a] + E[2] * Jt[2][a]);
    U[d] -= T(0.5) * al * (E[0] * E[0] + E[1] * E[1] + E[2] * E[2]);
  }
#pragma unroll
  for (int s = 0; s < NS; s++)
    if (!act[s]) { f[s][0] = f[s][1] = f[s][2] = U[s] = T(0); }
}

// Candidate visits of one probe configuration by a group of G lanes (G = 1:
// one lane alone).  All lanes of the group call it with identical arguments;
// each accumulates its share of the candidates into acc.
//   p       site positions, act: sites that feel the target
//   cen     centre of the sites, off: largest |p_s - cen|
//   glist   the group's candidate buffer in shared memory, GCAP_PER_LANE * G ints
constexpr int GCAP_PER_LANE = 8;
template <typename T, int G, int GAS, bool HASQ, bool SPLIT = false>
__device__ __forceinline__ void accumulate_group(const KParams &kp, const T (&p)[GasShape<GAS>::NS][3],
                                                 const bool (&act)[GasShape<GAS>::NS], const T (&cen)[3], T off,
                                                 Acc<T, GasShape<GAS>::NS> &acc, uint32_t &visits, int g,
                                                 unsigned mask, int *glist) {
  constexpr int NS = GasShape<GAS>::NS;
  constexpr int GCAP = GCAP_PER_LANE * G;
  bool any = false;
#pragma unroll
  for (int s = 0; s < NS; s++) any |= act[s];
  if (!any) return;
  uint32_t nvis = 0;
  // candidate sphere around the centre; +1e-3 A so rounding never drops a pair
  // (the near part of the range separation reaches r_out only)
  const T R = kp.allpairs ? T(INFINITY) : (SPLIT ? T(kp.field.r_out) : T(kp.reach)) + off + T(1e-3);
  const T cx = cen[0], cy = cen[1], cz = cen[2];
  const T ex = fmax(fmax(T(kp.bb_lo[0]) - cx, cx - T(kp.bb_hi[0])), T(0));
  const T ey = fmax(fmax(T(kp.bb_lo[1]) - cy, cy - T(kp.bb_hi[1])), T(0));
  const T ez = fmax(fmax(T(kp.bb_lo[2]) - cz, cz - T(kp.bb_hi[2])), T(0));
  const T fx = fmax(cx - T(kp.bb_lo[0]), T(kp.bb_hi[0]) - cx);
  const T fy = fmax(cy - T(kp.bb_lo[1]), T(kp.bb_hi[1]) - cy);
  const T fz = fmax(cz - T(kp.bb_lo[2]), T(kp.bb_hi[2]) - cz);
  if ((G > 1 && kp.natoms <= 2 * G) || fx * fx + fy * fy + fz * fz <= R * R) {
    // the whole target inside the reach sphere, or a target of at most two
    // atoms per lane of the group: every atom is a candidate
    for (int ai = g; ai < kp.natoms; ai += G) {
      const Atom<T> a = load_atom<T, GAS>(kp, ai);
      visit_atom<T, GAS, HASQ, SPLIT>(kp, p, act, a, acc);
    }
    if (G == 1 || g == 0) nvis += (uint32_t)kp.natoms;
  } else if (ex * ex + ey * ey + ez * ez <= R * R) {
    int i0, j0, nj;
    float inv_nj;
    const int ncol = column_range(kp, cx, cy, R, i0, j0, nj, inv_nj);
    for (int base = 0; base < ncol; base += G) {
      int b, len;
      column_run(kp, base + g, ncol, i0, j0, nj, inv_nj, cx, cy, cz, R, b, len);
      if constexpr (G == 1) {
        nvis += (uint32_t)len;
        for (int ai = b; ai < b + len; ai++) {
          const Atom<T> a = load_atom<T, GAS>(kp, ai);
          visit_atom<T, GAS, HASQ, SPLIT>(kp, p, act, a, acc);
        }
      } else {
        // flatten the G runs of this chunk into the group's list: exclusive scan of run lengths
        int incl = len;
#pragma unroll
        for (int o = 1; o < G; o <<= 1) {
          const int v = __shfl_up_sync(mask, incl, o, G);
          if (g >= o) incl += v;
        }
        const int total = __shfl_sync(mask, incl, G - 1, G);
        const int excl = incl - len;
        for (int cs = 0; cs < total; cs += GCAP) {
          const int lo = max(excl, cs), hi = min(excl + len, cs + GCAP);
          for (int q = lo; q < hi; q++) glist[q - cs] = b + (q - excl);
          __syncwarp(mask);
          const int m = min(GCAP, total - cs);
          for (int t = g; t < m; t += G) {
            const Atom<T> a = load_atom<T, GAS>(kp, glist[t]);
            visit_atom<T, GAS, HASQ, SPLIT>(kp, p, act, a, acc);
          }
          __syncwarp(mask);  // the list is rewritten next
        }
        if (g == 0) nvis += (uint32_t)total;
      }
    }
  }
  visits += nvis;
}

// Site forces of one probe configuration by a group of G lanes; every lane of
// the group gets the identical result (xor-butterfly sums).  Used by the
// force-evaluation entry point; the lane pass uses accumulate_group +
// reduce_group_row instead.
template <typename T, int G, int GAS, bool HASQ>
__device__ __forceinline__ void eval_forces(const KParams &kp, const T (&p)[GasShape<GAS>::NS][3],
                                         const bool (&act)[GasShape<GAS>::NS], const T (&cen)[3],
                                         T off, T (&f)[GasShape<GAS>::NS][3],
                                         T (&U)[GasShape<GAS>::NS], uint32_t &visits, int g,
                                         unsigned mask, int *glist) {
  constexpr int NS = GasShape<GAS>::NS;
  constexpr int NV = 4 * NS + 9;
  Acc<T, NS> acc;
  acc.zero();
  accumulate_group<T, G, GAS, HASQ>(kp, p, act, cen, off, acc, visits, g, mask, glist);
  T row[NV];
#pragma unroll
  for (int k = 0; k < NV; k++) row[k] = G > 1 ? group_sum<G>(acc_value(acc, k), mask) : acc_value(acc, k);
  finish_row<T, GAS, HASQ>(kp, row, act, f, U);
}

// Sum of P values over the 32 lanes of a warp, scattered: a reduce-scatter
// butterfly in which each exchange sends half of the values still held, so
// the warp spends 2P - 1 shuffles (not 5P).  Afterwards lane l holds in v[0]
// the warp sum of value index (l >> (5 - log2 P)); lanes that share an index
// hold identical bits (each pairwise sum is commutative).
template <int O, int C, int P, typename T> __device__ __forceinline__ void rs_level(T (&v)[P], int lane) {
  if constexpr (C == 1) {
    v[0] += __shfl_xor_sync(0xffffffffu, v[0], O);
  } else {
    constexpr int H = C / 2;
    const bool up = (lane & O) != 0;
#pragma unroll
    for (int i = 0; i < H; i++) {
      const T send = up ? v[i] : v[i + H];
      const T keep = up ? v[i + H] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, O);
    }
  }
  if constexpr (O > 1) rs_level<O / 2, (C == 1 ? 1 : C / 2), P>(v, lane);
}
template <int P, typename T> __device__ __forceinline__ void warp_reduce_scatter(T (&v)[P], int lane) {
  static_assert(P >= 1 && P <= 32 && (P & (P - 1)) == 0, "P must be a power of two <= 32");
  rs_level<16, P, P>(v, lane);
}
template <int P> constexpr int log2_of() { return P <= 1 ? 0 : 1 + log2_of<P / 2>(); }

// values reduced per force evaluation: per site f (3) and U, then the field
// (3) and its gradient (6) at the dipole site; padded to a power of two
template <int GAS> struct RedShape {
  static constexpr int NV = 4 * GasShape<GAS>::NS + 9;
  static constexpr int P = NV <= 16 ? 16 : 32;
};
// Raw sums of a group's evaluation into row[0..NV) (shared memory).  A full
// warp reduce-scatters (2P - 1 shuffles, each lane stores the value it ends
// with); smaller groups sum every value by xor butterfly and lane 0 stores.
template <typename T, int G, int GAS>
__device__ __forceinline__ void reduce_group_row(const Acc<T, GasShape<GAS>::NS> &acc, int g, unsigned mask,
                                                 T *row) {
  constexpr int NV = RedShape<GAS>::NV;
  if constexpr (G == 32) {
    constexpr int P = RedShape<GAS>::P;
    T v[P];
#pragma unroll
    for (int k = 0; k < P; k++) v[k] = k < NV ? acc_value(acc, k) : T(0);
    warp_reduce_scatter<P>(v, g);
    constexpr int SH = 5 - log2_of<P>();
    if ((g & ((1 << SH) - 1)) == 0 && (g >> SH) < NV) row[g >> SH] = v[0];
  } else {
#pragma unroll
    for (int k = 0; k < NV; k++) {
      const T x = G > 1 ? group_sum<G>(acc_value(acc, k), mask) : acc_value(acc, k);
      if (g == 0) row[k] = x;
    }
  }
}

constexpr int LCAP = 2048;  // least candidate-list entries kept in shared memory per CTA (the
                            // launch's kp.lcap, sized to the target's densest sphere, can be more)
constexpr int LCAP_MAX = 8192;
constexpr float LSKIN = 1.0f;  // A: the list's margin; reused while the probe moves less

// Block-wide exclusive scan of len; total receives the block sum.  Ends
// after one __syncthreads; sm_wsum may be rewritten only after another.
template <int NT>
__device__ __forceinline__ int block_excl_scan(int len, int lane, int w, int *sm_wsum, int &total) {
  constexpr int NW = NT / 32;
  int incl = len;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) sm_wsum[w] = incl;
  __syncthreads();
  int wofs = 0;
  total = 0;
#pragma unroll
  for (int k = 0; k < NW; k++) {
    const int ws = sm_wsum[k];
    wofs += k < w ? ws : 0;
    total += ws;
  }
  return incl + wofs - len;
}

// Visit candidates list[0..m) (list == nullptr: atoms 0..m): thread tid
// takes t, t+NT, ... two per iteration for instruction-level parallelism.
template <typename T, int NT, int GAS, bool HASQ, bool SPLIT = false>
__device__ __forceinline__ void visit_list(const KParams &kp, const T (&p)[GasShape<GAS>::NS][3],
                                           const bool (&act)[GasShape<GAS>::NS], const int *list, int m, int tid,
                                           Acc<T, GasShape<GAS>::NS> &acc) {
  int t = tid;
  for (; t + NT < m; t += 2 * NT) {
    const Atom<T> a1 = load_atom<T, GAS>(kp, list ? list[t] : t);
    const Atom<T> a2 = load_atom<T, GAS>(kp, list ? list[t + NT] : t + NT);
    visit_atom<T, GAS, HASQ, SPLIT>(kp, p, act, a1, acc);
    visit_atom<T, GAS, HASQ, SPLIT>(kp, p, act, a2, acc);
  }
  if (t < m) {
    const Atom<T> a1 = load_atom<T, GAS>(kp, list ? list[t] : t);
    visit_atom<T, GAS, HASQ, SPLIT>(kp, p, act, a1, acc);
  }
}

// Steps whose candidates do not fit the list: the runs of the reach sphere,
// flattened chunk by chunk.  Kept out of line (large targets only) and given
// copies of the probe, so the common step's code stays compact and its
// registers never need an address.
template <typename T, int GAS> struct ProbeSites {
  T p[GasShape<GAS>::NS][3];
  bool act[GasShape<GAS>::NS];
};
template <typename T, int NT, int GAS, bool HASQ, bool SPLIT = false>
__device__ __noinline__ Acc<T, GasShape<GAS>::NS> chunked_visits(const KParams *__restrict__ kpg,
                                                                 const ProbeSites<T, GAS> ps, T cx, T cy, T cz,
                                                                 T R, int tid, int *sm_list, int lcap,
                                                                 int *sm_wsum, uint32_t *nvis_out) {
  const KParams &kp = *kpg;
  const int lane = tid & 31, w = tid >> 5;
  Acc<T, GasShape<GAS>::NS> acc;
  acc.zero();
  uint32_t nvis = 0;
  int i0, j0, nj;
  float inv_nj;
  const int ncol = column_range(kp, cx, cy, R, i0, j0, nj, inv_nj);
  for (int base = 0; base < ncol; base += NT) {
    int b, len, total;
    column_run(kp, base + tid, ncol, i0, j0, nj, inv_nj, cx, cy, cz, R, b, len);
    const int excl = block_excl_scan<NT>(len, lane, w, sm_wsum, total);
    for (int cs = 0; cs < total; cs += lcap) {
      // this thread's run, as far as it falls into the chunk [cs, cs + lcap)
      const int lo = max(excl, cs), hi = min(excl + len, cs + lcap);
      for (int q = lo; q < hi; q++) sm_list[q - cs] = b + (q - excl);
      __syncthreads();
      visit_list<T, NT, GAS, HASQ, SPLIT>(kp, ps.p, ps.act, sm_list, min(lcap, total - cs), tid, acc);
      __syncthreads();  // the chunk is rewritten next
    }
    if (total == 0) __syncthreads();  // sm_wsum is rewritten next (block-uniform branch)
    nvis += (uint32_t)total;
  }
  *nvis_out = nvis;
  return acc;
}

// Block-cooperative site forces for the warp pass: all NT threads of a CTA
// evaluate one probe configuration.
//
// Candidates: small targets, and probes whose reach sphere holds the whole
// target, visit every atom.  Otherwise the CTA keeps a candidate list in
// shared memory (a Verlet list): the z-runs of the columns meeting a sphere
// LSKIN wider than the reach, flattened by an exclusive block scan of the
// run lengths.  While the probe's centre stays within LSKIN of where the list
// was built, the sphere of the current step lies inside the list's sphere, so
// the list is reused as is; the per-site cutoff tests then pick exactly the
// pairs the reference sums.  A list longer than lcap is not kept: such steps
// flatten the runs of the reach sphere chunk by chunk.
//
// The sums are reduced per warp with a reduce-scatter butterfly and then
// across warps in shared memory in a fixed order, so every thread ends with
// identical bits.  All threads call this with identical arguments.
//   sm_list: lcap ints; sm_wsum: NT/32 ints; sm_red: (NT/32) * RedShape<GAS>::P values, a
//   buffer the caller alternates between consecutive calls (one barrier per
//   call: a warp can reach the next call's barrier only after every warp has
//   read this call's sums, so the other buffer is free when it is written)
//   list_n, list_c: the CTA's list state (list_n < 0: no valid list)
//   SPLIT: the near part of the range separation (candidates within r_out);
//   the raw sums (per site f and U, then E and its gradient) go to raw[] and
//   the induced dipole is left to the caller, who adds the far parts first.
template <typename T, int NT, int GAS, bool HASQ, bool SPLIT = false>
__device__ __forceinline__ void eval_forces_block(const KParams &kp, const T (&p)[GasShape<GAS>::NS][3],
                                                  const bool (&act)[GasShape<GAS>::NS], const T (&cen)[3],
                                                  T off, T (&f)[GasShape<GAS>::NS][3],
                                                  T (&U)[GasShape<GAS>::NS], uint32_t &visits, int tid,
                                                  int *sm_list, int lcap, int *sm_wsum, T *sm_red, int &list_n,
                                                  T (&list_c)[3], const KParams *__restrict__ kpg,
                                                  T *raw = nullptr) {
  constexpr int NS = GasShape<GAS>::NS;
  constexpr int NW = NT / 32;
  constexpr int NV = RedShape<GAS>::NV;
  constexpr int P = RedShape<GAS>::P;
  const int lane = tid & 31, w = tid >> 5;
  Acc<T, NS> acc;
  acc.zero();
  bool any = false;
#pragma unroll
  for (int s = 0; s < NS; s++) any |= act[s];
  uint32_t nvis = 0;
  if (any) {
    const T R = kp.allpairs ? T(INFINITY) : (SPLIT ? T(kp.field.r_out) : T(kp.reach)) + off + T(1e-3);
    const T cx = cen[0], cy = cen[1], cz = cen[2];
    const T ex = fmax(fmax(T(kp.bb_lo[0]) - cx, cx - T(kp.bb_hi[0])), T(0));
    const T ey = fmax(fmax(T(kp.bb_lo[1]) - cy, cy - T(kp.bb_hi[1])), T(0));
    const T ez = fmax(fmax(T(kp.bb_lo[2]) - cz, cz - T(kp.bb_hi[2])), T(0));
    const T fx = fmax(cx - T(kp.bb_lo[0]), T(kp.bb_hi[0]) - cx);
    const T fy = fmax(cy - T(kp.bb_lo[1]), T(kp.bb_hi[1]) - cy);
    const T fz = fmax(cz - T(kp.bb_lo[2]), T(kp.bb_hi[2]) - cz);
    const int *lst = nullptr;  // candidates: atoms 0..m (nullptr) or lst[0..m)
    int m = 0;
    if (kp.natoms <= 2 * NT || fx * fx + fy * fy + fz * fz <= R * R) {
      // the whole target inside the reach sphere, or a target of at most two
      // atoms per thread: every atom is a candidate (the cutoff tests are exact)
      m = kp.natoms;
    } else if (ex * ex + ey * ey + ez * ez <= R * R) {
      const T dcx = cx - list_c[0], dcy = cy - list_c[1], dcz = cz - list_c[2];
      if (list_n < 0 || dcx * dcx + dcy * dcy + dcz * dcz > T(LSKIN) * T(LSKIN)) {
        // rebuild the list for the sphere of radius R + LSKIN around the centre
        const T RL = R + T(LSKIN);
        int i0, j0, nj;
        float inv_nj;
        const int ncol = column_range(kp, cx, cy, RL, i0, j0, nj, inv_nj);
        int filled = 0;  // block-uniform
        for (int base = 0; base < ncol; base += NT) {
          int b, len, total;
          column_run(kp, base + tid, ncol, i0, j0, nj, inv_nj, cx, cy, cz, RL, b, len);
          const int excl = block_excl_scan<NT>(len, lane, w, sm_wsum, total);
          if (filled + total <= lcap)
            for (int q = 0; q < len; q++) sm_list[filled + excl + q] = b + q;
          filled += total;
          __syncthreads();  // the runs are in place; sm_wsum may be rewritten
        }
        list_n = filled <= lcap ? filled : -1;
        list_c[0] = cx; list_c[1] = cy; list_c[2] = cz;
      }
      if (list_n >= 0) {
        lst = sm_list;
        m = list_n;
      } else {
        ProbeSites<T, GAS> ps;
#pragma unroll
        for (int s = 0; s < NS; s++) {
          ps.act[s] = act[s];
#pragma unroll
          for (int k = 0; k < 3; k++) ps.p[s][k] = p[s][k];
        }
        uint32_t nc = 0;
        acc = chunked_visits<T, NT, GAS, HASQ, SPLIT>(kpg, ps, cx, cy, cz, R, tid, sm_list, lcap, sm_wsum, &nc);
        nvis += nc;
      }
    }
    visit_list<T, NT, GAS, HASQ, SPLIT>(kp, p, act, lst, m, tid, acc);
    nvis += (uint32_t)m;
  }
  // reduce-scatter per warp, then the warps in a fixed order
  T v[P];
#pragma unroll
  for (int s = 0; s < NS; s++) {
    v[4 * s] = acc.f[s][0]; v[4 * s + 1] = acc.f[s][1]; v[4 * s + 2] = acc.f[s][2]; v[4 * s + 3] = acc.Usum(s);
  }
#pragma unroll
  for (int k = 0; k < 3; k++) v[4 * NS + k] = acc.E[k];
#pragma unroll
  for (int k = 0; k < 6; k++) v[4 * NS + 3 + k] = acc.G[k];
#pragma unroll
  for (int k = NV; k < P; k++) v[k] = T(0);
  warp_reduce_scatter<P>(v, lane);
  constexpr int SH = 5 - log2_of<P>();  // lanes per value index = 1 << SH
  T out[NV];
  if constexpr (NW > 1) {
    if ((lane & ((1 << SH) - 1)) == 0) sm_red[w * P + (lane >> SH)] = v[0];
    __syncthreads();
    // every thread sums the warps' partials in the same fixed order
#pragma unroll
    for (int k = 0; k < NV; k++) {
      T sum = sm_red[k];
#pragma unroll
      for (int q = 1; q < NW; q++) sum += sm_red[q * P + k];
      out[k] = sum;
    }
  } else {
#pragma unroll
    for (int k = 0; k < NV; k++) out[k] = __shfl_sync(0xffffffffu, v[0], k << SH);
  }
  if constexpr (SPLIT) {
#pragma unroll
    for (int k = 0; k < NV; k++) raw[k] = out[k];
    visits += nvis;
    return;
  }
#pragma unroll
  for (int s = 0; s < NS; s++) {
    f[s][0] = out[4 * s]; f[s][1] = out[4 * s + 1]; f[s][2] = out[4 * s + 2]; U[s] = out[4 * s + 3];
  }
  if (HASQ && kp.dip_on) {
    constexpr int d = GasShape<GAS>::DIP;
    const T al = T(kp.alpha);
    const T *E = out + 4 * NS, *Gr = out + 4 * NS + 3;
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

__device__ __forceinline__ bool setup_probe(const KParams &kp, size_t j, Init &I) {
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
    const float sn = sqrtf(cx * cx + cy * cy + cz * cz), cs = dot3(a, b);
    // one step turns the probe by a small angle: there atan(t), t = sn/cs <
    // 1/8, is its Maclaurin series to t^9 (truncation below 1.2e-11, far
    // under FP32 rounding); atan2f elsewhere
    if (cs > 0.f && sn < 0.125f * cs) {
      const float t = __fdividef(sn, cs), t2 = t * t;
      return t * (1.f + t2 * (-1.f / 3.f + t2 * (1.f / 5.f + t2 * (-1.f / 7.f + t2 * (1.f / 9.f)))));
    }
    return atan2f(sn, cs);
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
  const T ux = r[0] * T(kp.inv_a), uy = r[1] * T(kp.inv_b), uz = r[2] * T(kp.inv_c);
  return ux * ux + uy * uy + uz * uz > T(1);
}

// ---- trajectory kernels ------------------------------------------------------
// Two passes share one integrator (the step of run_He / run_N2 / run_CO2):
//
//  lane pass  every lane owns one trajectory; a warp advances 32 independent
//             trajectories in SIMT.  The force phase is cooperative: lanes
//             publish their site positions in shared memory, the lanes whose
//             probe is within reach of the target are collected with a ballot,
//             and subgroups of G lanes evaluate those probes (G = 1: every lane
//             its own).  Probes out of reach feel exactly zero force.  A lane
//             whose trajectory passes `park_steps` integration steps saves the
//             exact integrator state to HBM ("parks" it) and takes new work.
//  warp pass  parked trajectories resume one per CTA (64 threads by
//             default): the force phase of a step uses every thread and the
//             integrator runs CTA-uniform, so the long trajectories (captured
//             orbits with up to ~3e5 steps) advance at the lowest per-step
//             latency instead of sharing a warp with 31 others; failed tries
//             can run at once (speculative retries, see resume_kernel).
//
// Finished trajectories write status / 1-cos(chi) / steps / visits at their
// own index.  Restarts rebuild the initial state from the trajectory's random
// numbers (System::setup is deterministic), so no copy of the initial state is
// kept.
enum : int { M_IDLE = 0, M_INIT = 1, M_RESTART = 2, M_STEP = 3 };
constexpr int BLOCK = 128;
// Resident CTAs per SM the register allocation must allow.  Lane pass: 3.
// Warp pass: molecules run 512 threads per SM (8 CTAs of 64 at <= 128
// registers; measured 2.58 -> 2.07 s on the 1231-atom N2 workload, whose
// warp pass is throughput-bound), atoms are left unconstrained (their warp
// pass is bound by the latency of the longest trajectory), and so is the
// FP64 parity mode (128 registers would spill).
#ifndef CCS_LANE_MIN_BLOCKS
#define CCS_LANE_MIN_BLOCKS 3
#endif
#ifndef CCS_WARP_MIN_BLOCKS
#define CCS_WARP_MIN_BLOCKS(T, nt, gas) ((gas) == GAS_ATOM || sizeof(T) == 8 ? 1 : 512 / (nt))
#endif

__device__ __forceinline__ int nth_set_bit(unsigned m, int n) {
  for (int k = 0; k < n; k++) m &= m - 1u;
  return __ffs(m) - 1;
}

// Integrator state of one trajectory between force phases.  Atoms use
// r1/v1/r1lo; molecules keep the constrained pair (r1, r2) and the pair forces
// (f1, f2) of the last force phase; site positions are derived from it.
template <typename T> struct LaneState {
  T r1[3], r2[3], v1[3], v2[3], r1lo[3], r2lo[3];
  T f1[3], f2[3];
  T U, rold[3], dtheta, dt, Ei;
  uint32_t stepcount, nsteps, nvis;
  int tries, maxTries, mode;
  uint32_t ion;  // batched runs: the trajectory's ion (j is its index within that ion)
  unsigned long long j;
};

template <int GAS> struct Sites {
  static constexpr int NS = GasShape<GAS>::NS;
  static constexpr int pa = 0, pb = GAS == GAS_CO2 ? 2 : 1, pc = GAS == GAS_CO2 ? 1 : 2;
  static constexpr int cs = GAS == GAS_ATOM ? 0 : pc;  // reference point of the reach sphere
};

template <typename T, int GAS>
__device__ __forceinline__ void site_positions(const LaneState<T> &L, T (&p)[GasShape<GAS>::NS][3]) {
  using S = Sites<GAS>;
  if constexpr (GAS == GAS_ATOM) {
#pragma unroll
    for (int k = 0; k < 3; k++) p[0][k] = L.r1[k];
  } else {
#pragma unroll
    for (int k = 0; k < 3; k++) {
      p[S::pa][k] = L.r1[k];
      p[S::pb][k] = L.r2[k];
      p[S::pc][k] = T(0.5) * (L.r1[k] + L.r2[k]);
    }
  }
}

// half the pair distance: how far a site can sit from the reference point
template <typename T, int GAS>
__device__ __forceinline__ T site_offset(const T (&p)[GasShape<GAS>::NS][3]) {
  if constexpr (GAS == GAS_ATOM) {
    return T(0);
  } else {
    using S = Sites<GAS>;
    const T hd[3] = {p[S::pa][0] - p[S::pb][0], p[S::pa][1] - p[S::pb][1], p[S::pa][2] - p[S::pb][2]};
    return T(0.5) * Real<T>::sq(dot3(hd, hd));
  }
}

// the reach test (bounding box of the target) and the reference's grid rule
template <typename T, int GAS>
__device__ __forceinline__ bool probe_near(const KParams &kp, const T (&p)[GasShape<GAS>::NS][3],
                                           unsigned &actbits) {
  using S = Sites<GAS>;
  actbits = 0;
#pragma unroll
  for (int s = 0; s < S::NS; s++)
    if (ref_inside(kp, p[s][0], p[s][1], p[s][2])) actbits |= 1u << s;
  const T R = (kp.allpairs ? T(INFINITY) : T(kp.reach) + T(1e-3)) + site_offset<T, GAS>(p);
  const T ex = fmax(fmax(T(kp.bb_lo[0]) - p[S::cs][0], p[S::cs][0] - T(kp.bb_hi[0])), T(0));
  const T ey = fmax(fmax(T(kp.bb_lo[1]) - p[S::cs][1], p[S::cs][1] - T(kp.bb_hi[1])), T(0));
  const T ez = fmax(fmax(T(kp.bb_lo[2]) - p[S::cs][2], p[S::cs][2] - T(kp.bb_hi[2])), T(0));
  return actbits != 0 && ex * ex + ey * ey + ez * ez <= R * R;
}

// pair forces from the site forces: N2 splits the central charge half/half
// (System.cpp:736-739); CO2 redistributes the carbon force (Ciccotti,
// System.cpp:1154-1158); an atom keeps its own force.  Also sums U.
template <typename T, int GAS>
__device__ __forceinline__ void absorb_forces(const KParams &kp, const T (&fs)[GasShape<GAS>::NS][3],
                                              const T (&Us)[GasShape<GAS>::NS], LaneState<T> &L) {
  T u = T(0);
#pragma unroll
  for (int s = 0; s < GasShape<GAS>::NS; s++) u += Us[s];
  L.U = u;
  if constexpr (GAS == GAS_CO2) {
    const T M = T(kp.gas_mass), m2M = T(kp.gas_m[1]) / M, m0M = T(kp.gas_m[0]) / M;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      L.f1[k] = (T(1) - T(0.5) * m2M) * fs[0][k] + m0M * fs[1][k] - T(0.5) * m2M * fs[2][k];
      L.f2[k] = (T(1) - T(0.5) * m2M) * fs[2][k] + m0M * fs[1][k] - T(0.5) * m2M * fs[0][k];
    }
  } else if constexpr (GAS == GAS_N2) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
      L.f1[k] = fs[0][k] + T(0.5) * fs[2][k];
      L.f2[k] = fs[1][k] + T(0.5) * fs[2][k];
    }
  } else {
#pragma unroll
    for (int k = 0; k < 3; k++) L.f1[k] = fs[0][k];
  }
}

// Initial state of a trajectory (System::setup) and the initial kinetic
// energy of every site (System.cpp:376-383, 648-660, 1076-1088).  Not inlined
// (it runs once per trajectory and per retry); it returns by value so the
// caller's integrator state never needs an address and stays in registers.
template <typename T> struct InitState {
  T r1[3], r2[3], v1[3], v2[3], rcm[3], ek;
  int hit;
};

template <typename T, int GAS>
__device__ __noinline__ InitState<T> lane_setup(const KParams *__restrict__ kpg, unsigned long long j) {
  const KParams &kp = *kpg;
  constexpr bool MOL = GAS != GAS_ATOM;
  using S = Sites<GAS>;
  InitState<T> o;
  Init I;
  o.hit = setup_probe(kp, (size_t)j, I) ? 1 : 0;
  for (int k = 0; k < 3; k++) {
    o.r1[k] = T(I.pos[S::pa][k]); o.v1[k] = T(I.vel[S::pa][k]);
    o.r2[k] = T(I.pos[S::pb][k]); o.v2[k] = T(I.vel[S::pb][k]);
    o.rcm[k] = T(I.rcm[k]);
  }
  T e = T(0);
  for (int s = 0; s < (MOL ? 3 : 1); s++) {
    const T vs[3] = {T(I.vel[s][0]), T(I.vel[s][1]), T(I.vel[s][2])};
    e += T(0.5) * T(MOL ? kp.gas_m[s] : kp.mu) * dot3(vs, vs) * T(AMUANGFS2_TO_KCAL_MOL);
  }
  o.ek = e;
  return o;
}

template <typename T, int GAS>
__device__ __forceinline__ void load_init(LaneState<T> &L, const InitState<T> &I) {
#pragma unroll
  for (int k = 0; k < 3; k++) {
    L.r1[k] = I.r1[k]; L.v1[k] = I.v1[k]; L.r1lo[k] = T(0);
    if constexpr (GAS != GAS_ATOM) { L.r2[k] = I.r2[k]; L.v2[k] = I.v2[k]; L.r2lo[k] = T(0); }
    L.rold[k] = I.rcm[k];
  }
  L.dtheta = T(0);
  L.stepcount = 0;
}

// 1 - cos(chi) against the initial centre-of-mass velocity, rebuilt in FP64
// from the trajectory's random numbers.
template <typename T, int GAS>
__device__ __noinline__ double lane_chi(const KParams *__restrict__ kpg, unsigned long long j, T vx, T vy, T vz) {
  const KParams &kp = *kpg;
  Init I;
  setup_probe(kp, (size_t)j, I);
  double vref[3];
  if constexpr (GAS == GAS_ATOM) {
    for (int k = 0; k < 3; k++) vref[k] = I.vel[0][k];
  } else {
    for (int k = 0; k < 3; k++) vref[k] = I.vcm[k];
    if (GAS == GAS_CO2 && (kp.quirks & 1)) vref[0] = I.vcm[1];  // System.cpp:1012
  }
  const T vf[3] = {vx, vy, vz};
  return one_minus_cos<T>(vref, vf);
}

// First half of a step: kick, drift (constrained for molecules), angle.
template <typename T, int GAS>
__device__ __forceinline__ void first_half(const KParams &kp, LaneState<T> &L) {
  using S = Sites<GAS>;
  const T dt = L.dt, kconv = T(KCALMOLANGAMU_TO_ANGFS2);
  if constexpr (GAS == GAS_ATOM) {
    const T kick = dt * T(kp.half_kconv_over_m1);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      L.v1[k] += kick * L.f1[k];
      const T y = dt * L.v1[k] - L.r1lo[k];  // compensated position update
      const T t = L.r1[k] + y;
      L.r1lo[k] = (t - L.r1[k]) - y;
      L.r1[k] = t;
    }
    L.dtheta += angle3(L.r1, L.rold);
#pragma unroll
    for (int k = 0; k < 3; k++) L.rold[k] = L.r1[k];
  } else {
    // constrained Verlet, first half (System.cpp:1700-1739)
    const T d2 = T(kp.d_bond * kp.d_bond);
    const T ka = dt * T(kp.half_kconv_over_m1), kb = dt * T(kp.half_kconv_over_m2);
    T vci[3], vcj[3], rij[3], rcij[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      vci[k] = L.v1[k] + ka * L.f1[k];
      vcj[k] = L.v2[k] + kb * L.f2[k];
      rij[k] = L.r1[k] - L.r2[k];
      rcij[k] = rij[k] + dt * (vci[k] - vcj[k]);
    }
    const T r2ij = dot3(rij, rij), rc2ij = dot3(rcij, rcij), rr = dot3(rcij, rij);
    T det = rr * rr - r2ij * (rc2ij - d2);
    if (det < T(0)) det = T(0);
    const T lam = Real<T>::div(rr - Real<T>::sq(det), r2ij);
    const T cpos = T(kp.mu12_over_m1) * lam;  // the reference uses mi for both atoms (:1735-1736)
    const T inv_dt = Real<T>::div(T(1), dt);
    const T ca = cpos * inv_dt, cb = T(kp.mu12_over_m2) * lam * inv_dt;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      L.v1[k] = vci[k] - ca * rij[k];
      L.v2[k] = vcj[k] + cb * rij[k];
      T y = (dt * vci[k] - cpos * rij[k]) - L.r1lo[k];
      T t = L.r1[k] + y;
      L.r1lo[k] = (t - L.r1[k]) - y;
      L.r1[k] = t;
      y = (dt * vcj[k] + cpos * rij[k]) - L.r2lo[k];
      t = L.r2[k] + y;
      L.r2lo[k] = (t - L.r2[k]) - y;
      L.r2[k] = t;
    }
    T rcm[3];
#pragma unroll
    for (int k = 0; k < 3; k++) rcm[k] = T(0.5) * (L.r1[k] + L.r2[k]);
    L.dtheta += angle3(rcm, L.rold);
#pragma unroll
    for (int k = 0; k < 3; k++) L.rold[k] = rcm[k];
  }
}

enum : int { S_CONTINUE = 0, S_RETRY_ANGLE = 1, S_RETRY_ENERGY = 2, S_SCATTER = 3, S_CAPPED = 4 };

// Second half of a step and the exit tests (System.cpp:441-506, 835-940,
// 1268-1387).  vc receives the centre-of-mass velocity for chi.
template <typename T, int GAS>
__device__ __forceinline__ int second_half(const KParams &kp, LaneState<T> &L, T vc[3]) {
  using S = Sites<GAS>;
  const T dt = L.dt, kconv = T(KCALMOLANGAMU_TO_ANGFS2), ke = T(AMUANGFS2_TO_KCAL_MOL);
  T rc[3], ek;
  if constexpr (GAS == GAS_ATOM) {
    const T kick = dt * T(kp.half_kconv_over_m1);
#pragma unroll
    for (int k = 0; k < 3; k++) { L.v1[k] += kick * L.f1[k]; vc[k] = L.v1[k]; rc[k] = L.r1[k]; }
    ek = T(0.5) * T(kp.mu) * dot3(L.v1, L.v1) * ke;
  } else {
    // RATTLE velocity correction (System.cpp:1741-1767)
    const T ma = T(kp.gas_m[S::pa]), mb = T(kp.gas_m[S::pb]);
    const T ka = dt * T(kp.half_kconv_over_m1), kb = dt * T(kp.half_kconv_over_m2);
    T vci[3], vcj[3], rij[3], vcij[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      vci[k] = L.v1[k] + ka * L.f1[k];
      vcj[k] = L.v2[k] + kb * L.f2[k];
      rij[k] = L.r1[k] - L.r2[k];
      vcij[k] = vci[k] - vcj[k];
    }
    const T lam = Real<T>::div(T(kp.mu12) * dot3(rij, vcij), dot3(rij, rij));
    const T la = lam * T(kp.inv_m1), lb = lam * T(kp.inv_m2);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      L.v1[k] = vci[k] - la * rij[k];
      L.v2[k] = vcj[k] + lb * rij[k];
      vc[k] = T(0.5) * (L.v1[k] + L.v2[k]);
      rc[k] = T(0.5) * (L.r1[k] + L.r2[k]);
    }
    // N2: the two N atoms (System.cpp:890-896); CO2: all sites, carbon at vcm (:1333-1339)
    ek = T(0.5) * ma * dot3(L.v1, L.v1) * ke + T(0.5) * mb * dot3(L.v2, L.v2) * ke;
    if (GAS == GAS_CO2) ek += T(0.5) * T(kp.gas_m[S::pc]) * dot3(vc, vc) * ke;
  }
  L.stepcount++;
  L.nsteps++;
  if (L.dtheta > T(1.5 * PI_D)) return S_RETRY_ANGLE;
  if (outside_box(kp, rc)) {
    const double E = (double)L.U + (double)ek;
    const double dE = fabs((E - (double)L.Ei) / (double)L.Ei) * 100.0;
    return dE > kp.etol ? S_RETRY_ENERGY : S_SCATTER;
  }
  return L.stepcount >= kp.max_steps ? S_CAPPED : S_CONTINUE;
}

// Result of one trajectory.
template <typename T>
__device__ __forceinline__ void write_result(const KParams &kp, const LaneState<T> &L, int8_t st, double omc,
                                             unsigned long long *blk) {
  kp.status[L.j] = st;
  kp.omc[L.j] = st == 1 ? omc : 0.0;
  if (kp.steps) kp.steps[L.j] = L.nsteps;
  if (kp.visits) kp.visits[L.j] = L.nvis;
  atomicAdd(&blk[st], 1ull);
  atomicAdd(&blk[4], (unsigned long long)L.nsteps);
  atomicAdd(&blk[5], (unsigned long long)L.nvis);
}

// Parameters of the ion that trajectory state L belongs to: the launch's own
// (constant bank) for single-ion runs, the ion's entry of kp.ions for batches.
template <bool BATCH>
__device__ __forceinline__ const KParams &ion_params(const KParams &kp, uint32_t ion) {
  if constexpr (BATCH) return kp.ions[ion]; else return kp;
}
template <bool BATCH>
__device__ __forceinline__ const KParams *ion_params_ptr(const KParams &kp, const KParams *kpg, uint32_t ion) {
  if constexpr (BATCH) return kp.ions + ion; else return kpg;
}

// SURR: the learned field evaluates the probes outside its exact zone (see
// field_device.cuh): the loop then runs CTA-synchronously, because each step's
// MLP tile spans the CTA's 128 lanes; probes in the exact zone take the
// exact path below as before.
template <typename T, int G, int GAS, bool HASQ, bool BATCH, bool SURR = false>
__global__ void __launch_bounds__(BLOCK, SURR ? 2 : CCS_LANE_MIN_BLOCKS)
    traj_kernel(KParams kp, const KParams *__restrict__ kpg) {
  using S = Sites<GAS>;
  constexpr int NS = S::NS;
  static_assert(!SURR || (sizeof(T) == 4 && !BATCH), "the learned field runs in FP32 single-ion launches");
  constexpr int NSUB = 32 / G;
  constexpr unsigned FULL = 0xffffffffu;
  constexpr int NV = RedShape<GAS>::NV;
  __shared__ T sm_pos[BLOCK][NS][3];
  __shared__ T sm_row[BLOCK][NV];
  __shared__ uint32_t sm_vis[BLOCK];
  __shared__ unsigned sm_act[BLOCK];
  __shared__ uint32_t sm_ion[BATCH ? BLOCK : 1];
  __shared__ int sm_glist[BLOCK * GCAP_PER_LANE];
  __shared__ unsigned long long blk[8];
  if (threadIdx.x < 8) blk[threadIdx.x] = 0ull;
  __syncthreads();

  const int lane = threadIdx.x & 31;
  const int wbase = threadIdx.x & ~31;
  const int g = lane & (G - 1);
  const int sub = lane / G;
  const unsigned gmask = G == 32 ? FULL : (((1u << G) - 1u) << (sub * G));

  LaneState<T> L;
  L.mode = M_IDLE;
  L.ion = 0;
  const unsigned long long deadline = *(volatile const unsigned long long *)kp.deadline;
  bool park_full = false;  // the park buffer filled up: stop asking for slots (it only fills)
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  uint32_t tmem = 0, tc_phase = 0;
  if constexpr (SURR) tmem = tc_setup(kp.field, tc_smem);

  // take trajectories until one hits the ellipsoid (misses are written as free)
  auto grab = [&]() {
    for (;;) {
      const unsigned long long jj = atomicAdd(kp.work, 1ull);
      if (jj >= kp.ntraj || *(volatile int *)kp.error) { L.mode = M_IDLE; return; }
      if constexpr (BATCH) {  // the ion holding global trajectory jj (bisection of the ion starts)
        int lo = 0, hi = kp.nions;
        while (hi - lo > 1) {
          const int mid = (lo + hi) >> 1;
          if (__ldg(&kp.ion_start[mid]) <= jj) lo = mid; else hi = mid;
        }
        L.ion = (uint32_t)lo;
        L.j = jj - __ldg(&kp.ion_start[lo]);
      } else {
        L.ion = 0;
        L.j = kp.order ? (unsigned long long)__ldg(&kp.order[jj]) : jj;
      }
      const KParams &K = ion_params<BATCH>(kp, L.ion);
      L.nsteps = 0;
      L.nvis = 0;
      const InitState<T> I = lane_setup<T, GAS>(ion_params_ptr<BATCH>(kp, kpg, L.ion), L.j);
      if (!I.hit) { write_result(K, L, 0, 0.0, blk); continue; }
      load_init<T, GAS>(L, I);
      L.Ei = I.ek;  // completed with the initial potential energy by the first force phase
      L.tries = 0;
      L.maxTries = 8;
      L.dt = T(K.dt);
      L.mode = M_INIT;
      return;
    }
  };

  grab();
  unsigned it = 0;
  for (;;) {
    if ((++it & 127u) == 0) {  // watchdog, one answer per warp
      int e = 0;
      if (lane == 0) e = global_ns() > deadline || *(volatile int *)kp.error;
      e = __shfl_sync(FULL, e, 0);
      if (e) {
        if (lane == 0) atomicExch(kp.error, 1);
        if (L.mode != M_IDLE) write_result(ion_params<BATCH>(kp, L.ion), L, 3, 0.0, blk);
        L.mode = M_IDLE;
      }
    }
    if constexpr (SURR) {
      if (__syncthreads_and(L.mode == M_IDLE)) break;
    } else {
      if (__all_sync(FULL, L.mode == M_IDLE)) break;
    }
    const KParams &K = ion_params<BATCH>(kp, L.ion);  // this lane's ion

    if (L.mode == M_STEP) first_half<T, GAS>(K, L);

    // ---- force phase
    bool near = false, surr = false;
    unsigned actbits = 0;
    T fs[NS][3], Us[NS];
    T p[NS][3];
    if (L.mode != M_IDLE) {
      site_positions<T, GAS>(L, p);
      near = probe_near<T, GAS>(K, p, actbits);
      if constexpr (SURR) {
        if (near) {
          surr = true;
#pragma unroll
          for (int s = 0; s < NS; s++)
            if ((actbits >> s) & 1u) surr &= !field_exact(kp.field, (float)p[s][0], (float)p[s][1], (float)p[s][2]);
        }
      }
      if (near) {
        if constexpr (G == 1) {
          bool act[NS];
#pragma unroll
          for (int s = 0; s < NS; s++) act[s] = (actbits >> s) & 1u;
          if (!surr)
            eval_forces<T, 1, GAS, HASQ>(K, p, act, p[S::cs], site_offset<T, GAS>(p), fs, Us, L.nvis, 0,
                                         1u << lane, nullptr);
        } else {
#pragma unroll
          for (int s = 0; s < NS; s++)
#pragma unroll
            for (int k = 0; k < 3; k++) sm_pos[threadIdx.x][s][k] = p[s][k];
          sm_act[threadIdx.x] = actbits;
          if constexpr (BATCH) sm_ion[threadIdx.x] = L.ion;
        }
      }
    }
    if constexpr (G > 1) {
      __syncwarp();
      const unsigned bal = __ballot_sync(FULL, near && !surr);
      const int nn = __popc(bal);
      for (int idx = sub; idx < nn; idx += NSUB) {
        const int t = wbase + nth_set_bit(bal, idx);
        T P[NS][3];
        bool act[NS];
        const unsigned ab = sm_act[t];
#pragma unroll
        for (int s = 0; s < NS; s++) {
          act[s] = (ab >> s) & 1u;
#pragma unroll
          for (int k = 0; k < 3; k++) P[s][k] = sm_pos[t][s][k];
        }
        uint32_t nv = 0;
        Acc<T, NS> acc;
        acc.zero();
        const KParams &Kt = ion_params<BATCH>(kp, BATCH ? sm_ion[t] : 0u);  // the probe's ion
        accumulate_group<T, G, GAS, HASQ>(Kt, P, act, P[S::cs], site_offset<T, GAS>(P), acc, nv, g, gmask,
                                          sm_glist + (wbase + sub * G) * GCAP_PER_LANE);
        reduce_group_row<T, G, GAS>(acc, g, gmask, sm_row[t]);
        if (g == 0) sm_vis[t] = nv;
      }
      __syncwarp();
      if (near && !surr) {  // the probe's own lane finishes its forces from the raw sums
        bool act[NS];
#pragma unroll
        for (int s = 0; s < NS; s++) act[s] = (actbits >> s) & 1u;
        finish_row<T, GAS, HASQ>(K, sm_row[threadIdx.x], act, fs, Us);
        L.nvis += sm_vis[threadIdx.x];
      }
    }
    if constexpr (SURR) {
      // the learned field for every probe outside the exact zone: the
      // switched exact sums over the atoms within r_out ...
      bool act[NS];
#pragma unroll
      for (int s = 0; s < NS; s++) act[s] = (actbits >> s) & 1u;
      T raw[NV];
      if constexpr (G == 1) {
        if (surr) {
          Acc<T, NS> acc;
          acc.zero();
          uint32_t nv = 0;
          accumulate_group<T, 1, GAS, HASQ, true>(K, p, act, p[S::cs], site_offset<T, GAS>(p), acc, nv, 0, 1u << lane,
                                                  nullptr);
#pragma unroll
          for (int k = 0; k < NV; k++) raw[k] = acc_value(acc, k);
          L.nvis += nv;
        }
      } else {
        __syncwarp();
        const unsigned bal2 = __ballot_sync(FULL, surr);
        const int n2 = __popc(bal2);
        for (int idx = sub; idx < n2; idx += NSUB) {
          const int t = wbase + nth_set_bit(bal2, idx);
          T P[NS][3];
          bool at[NS];
          const unsigned ab = sm_act[t];
#pragma unroll
          for (int s = 0; s < NS; s++) {
            at[s] = (ab >> s) & 1u;
#pragma unroll
            for (int k = 0; k < 3; k++) P[s][k] = sm_pos[t][s][k];
          }
          uint32_t nv = 0;
          Acc<T, NS> acc;
          acc.zero();
          accumulate_group<T, G, GAS, HASQ, true>(kp, P, at, P[S::cs], site_offset<T, GAS>(P), acc, nv, g, gmask,
                                                  sm_glist + (wbase + sub * G) * GCAP_PER_LANE);
          reduce_group_row<T, G, GAS>(acc, g, gmask, sm_row[t]);
          if (g == 0) sm_vis[t] = nv;
        }
        __syncwarp();
        if (surr) {
#pragma unroll
          for (int k = 0; k < NV; k++) raw[k] = sm_row[threadIdx.x][k];
          L.nvis += sm_vis[threadIdx.x];
        }
      }
      // ... plus the far parts from the network: one MLP tile of the CTA's
      // 128 lanes per site (the dipole's site also gives the far field)
      float ufar[NS], ffar[NS][3], Ef[3] = {0.f, 0.f, 0.f}, Jf[3][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
#pragma unroll
      for (int s = 0; s < NS; s++) { ufar[s] = 0.f; ffar[s][0] = ffar[s][1] = ffar[s][2] = 0.f; }
      if (__syncthreads_or(surr)) {
        bool ok = true;
#pragma unroll 1
        for (int s = 0; s < NS && ok; s++) {
          const bool use = surr && act[s];
          float x[3] = {0.f, 0.f, 0.f};
          if (use) { x[0] = (float)p[s][0]; x[1] = (float)p[s][1]; x[2] = (float)p[s][2]; }
          int fl[FL_SITE_FIELDS];
          const int nfo = site_fields(kp.field, s, fl);
          float e[FL_E], J[FL_E][3], u[FL_SITE_FIELDS], gr[FL_SITE_FIELDS][3];
          field_encode(kp.field, x, e, J);
          ok = tc_site(kp.field, tc_smem, tmem, tc_phase, use, e, J, nfo, fl, u, gr);
          if (use) {
            ufar[s] = u[0];
            ffar[s][0] = gr[0][0]; ffar[s][1] = gr[0][1]; ffar[s][2] = gr[0][2];
            if (nfo == 4)
#pragma unroll
              for (int a = 0; a < 3; a++) {
                Ef[a] = u[1 + a];
#pragma unroll
                for (int b = 0; b < 3; b++) Jf[a][b] = -gr[1 + a][b];
              }
          }
        }
        if (!ok) {  // a tensor-core stage never completed (uniform): stop the kernel
          if (threadIdx.x == 0) atomicExch(kp.error, 2);
          if (L.mode != M_IDLE) write_result(K, L, 3, 0.0, blk);
          break;
        }
      }
      if (surr) finish_split<T, GAS, HASQ>(K, raw, ufar, ffar, Ef, Jf, act, fs, Us);
    }
    if (L.mode == M_IDLE) continue;
    if (!near) {
#pragma unroll
      for (int s = 0; s < NS; s++) fs[s][0] = fs[s][1] = fs[s][2] = Us[s] = T(0);
    }
    absorb_forces<T, GAS>(K, fs, Us, L);

    // ---- second half, exit tests, retries, parking
    if (L.mode == M_INIT) {
      L.Ei += L.U;
      L.mode = M_STEP;
    } else if (L.mode == M_RESTART) {
      L.mode = M_STEP;
    } else {
      T vc[3];
      const int r = second_half<T, GAS>(K, L, vc);
      if (r == S_SCATTER) {
        write_result(K, L, 1, lane_chi<T, GAS>(ion_params_ptr<BATCH>(kp, kpg, L.ion), L.j, vc[0], vc[1], vc[2]), blk);
        grab();
      } else if (r == S_CAPPED) {
        write_result(K, L, 3, 0.0, blk);
        grab();
      } else if (r != S_CONTINUE) {
        // a failed try: smaller time step and a fresh start (System.cpp:453-458, 468-473)
        L.tries++;
        if (r == S_RETRY_ENERGY) L.maxTries++;
        L.dt = T(K.dt / (L.tries + 1));
        if (!(L.tries < L.maxTries && L.maxTries < 10)) {
          write_result(K, L, 2, 0.0, blk);
          grab();
        } else {
          load_init<T, GAS>(L, lane_setup<T, GAS>(ion_params_ptr<BATCH>(kp, kpg, L.ion), L.j));
          L.mode = M_RESTART;
        }
      } else if (kp.park && !park_full && L.nsteps >= kp.park_steps &&
                 (!kp.park_drained ||
                  ((L.nsteps & 63u) == 0 && *(volatile const unsigned long long *)kp.work >= kp.ntraj))) {
        const unsigned long long slot = atomicAdd(kp.park_count, 1ull);
        if (slot < kp.park_cap) {
          reinterpret_cast<LaneState<T> *>(kp.park)[slot] = L;
          atomicAdd(&blk[7], 1ull);
          grab();
        } else {
          park_full = true;  // the trajectory stays in its lane
        }
      }
    }
  }
  if constexpr (SURR) tc_teardown(tmem);
  __syncthreads();
  if (threadIdx.x < 6 && blk[threadIdx.x]) atomicAdd(&kp.stats[threadIdx.x], blk[threadIdx.x]);
  if (threadIdx.x == 7 && blk[7]) atomicAdd(&kp.stats[6], blk[7]);
}

// Warp pass: parked trajectories resume one per CTA (all NT threads hold
// the same state; the force phase is block-cooperative).
//
// Speculative retries.  A failed try restarts the trajectory from its
// initial state with the step dt0/(k+1) (System.cpp:453-458); the tries of a
// trajectory are therefore independent computations, and only the decision
// which one counts is sequential.  Captured orbits fail try after try, each
// longer than the last, and set the end of a run.  So once a warp-pass
// trajectory has failed spec_from tries (phase 0), it is recorded and left;
// a second launch (phase 1) runs each recorded trajectory's remaining tries
// at once, one CTA each, from the same code; spec_resolve_kernel then walks
// every record's tries in order with the reference's rules.  Every try runs
// the same instructions as it would in sequence, so the results are those of
// the sequential path.
constexpr int RBLOCK = 64;  // default threads per trajectory in the warp pass

// SURR: steps whose sites all lie outside the learned field's exact zone are
// evaluated by the field, one warp per site (field_site_warp).
template <typename T, int GAS, bool HASQ, int NT, bool BATCH, bool SURR = false>
__global__ void __launch_bounds__(NT, CCS_WARP_MIN_BLOCKS(T, NT, GAS)) resume_kernel(KParams kp, const KParams *__restrict__ kpg) {
  using S = Sites<GAS>;
  constexpr int NS = S::NS;
  static_assert(!SURR || (sizeof(T) == 4 && !BATCH), "the learned field runs in FP32 single-ion launches");
  __shared__ float sm_site[NS][4 * FL_SITE_FIELDS];
  extern __shared__ int sm_list[];  // kp.lcap entries (+ LCAP with the field; dynamic shared memory)
  __shared__ int sm_wsum[NT / 32];
  __shared__ T sm_red[2][(NT / 32) * RedShape<GAS>::P];  // alternating reduction buffers
  int red = 0;
  __shared__ unsigned long long blk[8];
  __shared__ unsigned long long sm_idx;
  if (threadIdx.x < 8) blk[threadIdx.x] = 0ull;
  __syncthreads();
  const int tid = threadIdx.x;
  const bool spec_launch = kp.spec_phase != 0;
  const unsigned long long deadline = *(volatile const unsigned long long *)kp.deadline;
  unsigned long long np;
  if (spec_launch) {
    np = *(volatile unsigned long long *)kp.spec_count;
    if (np > kp.spec_cap) np = kp.spec_cap;
    np *= SPEC_SLOTS;
  } else {
    np = *(volatile unsigned long long *)kp.park_count;
    if (np > kp.park_cap) np = kp.park_cap;
  }
  unsigned long long *next = spec_launch ? kp.spec_next : kp.park_next;
  // speculation pays when the warp pass is bound by its longest chains of
  // tries, not while parked trajectories wait for a CTA (then the extra
  // tries only add work): a failed try is handed over when few trajectories
  // were parked at all, or once every parked trajectory has been taken
  const bool may_spec = kp.spec_rec && !spec_launch;
  // Phase-0 CTAs that find the park queue drained stay and run the
  // speculative tries as their records are published, until no parked
  // trajectory is still running (then every record is final); the phase-1
  // launch runs whatever is left (records beyond this, or after a timeout).
  // The wait polls with a sleep and ends at the watchdog's deadline.
  bool park_done = spec_launch;
  __shared__ int sm_kind;
  for (;;) {
    if (tid == 0) {
      unsigned long long v = ~0ull;
      int kind = spec_launch ? 1 : 0;
      if (!*(volatile int *)kp.error) {
        if (!park_done) {
          if (may_spec) atomicAdd(kp.park_active, 1ull);  // before taking: a poller never misses it
          v = atomicAdd(next, 1ull);
          if (v >= np) {
            v = ~0ull;
            park_done = true;
            if (may_spec) atomicAdd(kp.park_active, ~0ull);  // minus one
          }
        } else if (spec_launch) {
          v = atomicAdd(next, 1ull);
          if (v >= np) v = ~0ull;
        }
        if (v == ~0ull && may_spec) {
          kind = 1;
          for (unsigned poll = 0; poll < (1u << 26); poll++) {
            if ((poll & 255u) == 255u && (global_ns() > deadline || *(volatile int *)kp.error)) {
              atomicExch(kp.error, 1);  // the watchdog: stop waiting
              break;
            }
            // the running count first: once it is zero every record is published
            const unsigned long long active = *(volatile unsigned long long *)kp.park_active;
            __threadfence();
            unsigned long long cnt = *(volatile unsigned long long *)kp.spec_count;
            if (cnt > kp.spec_cap) cnt = kp.spec_cap;
            const unsigned long long cur = *(volatile unsigned long long *)kp.spec_next;
            if (cur < cnt * SPEC_SLOTS) {
              if (*(volatile int *)&kp.spec_rec[cur / SPEC_SLOTS].ready &&
                  atomicCAS(kp.spec_next, cur, cur + 1) == cur) {
                v = cur;
                break;
              }
              continue;  // being published, or another CTA took it: look again
            }
            if (active == 0) break;  // nothing left to come
            __nanosleep(2000);
          }
          __threadfence();  // the record's fields after its ready flag
        }
      }
      sm_idx = v;
      sm_kind = kind;
    }
    __syncthreads();
    const unsigned long long idx = sm_idx;
    const bool spec = sm_kind != 0;  // this item is a speculative try
    __syncthreads();
    if (idx == ~0ull) break;
    LaneState<T> L;
    unsigned long long rec = 0;
    if (spec) {  // try k of record rec, from the trajectory's initial state
      rec = idx / SPEC_SLOTS;
      const SpecRec R = load_spec_rec(kp.spec_rec + rec);
      const int k = R.tries + (int)(idx % SPEC_SLOTS);
      if (k > 8) continue;  // beyond the reference's last try (block-uniform)
      L.j = R.j;
      L.ion = R.ion;
      load_init<T, GAS>(L, lane_setup<T, GAS>(ion_params_ptr<BATCH>(kp, kpg, L.ion), L.j));
      L.Ei = T(R.Ei);
      L.tries = k;
      L.maxTries = R.maxTries;
      L.dt = T(ion_params<BATCH>(kp, L.ion).dt / (k + 1));
      L.mode = M_RESTART;
      L.nsteps = 0;
      L.nvis = 0;
    } else {
      L = reinterpret_cast<const LaneState<T> *>(kp.park)[idx];
    }
    const KParams &K = ion_params<BATCH>(kp, L.ion);
    const KParams *Kg = ion_params_ptr<BATCH>(kp, kpg, L.ion);
    int list_n = -1;  // this trajectory's candidate list (none yet)
    T list_c[3] = {T(0), T(0), T(0)};
    // with the learned field, the near part of the range separation keeps a
    // second list (radius r_out) after the first one's kp.lcap entries, so
    // steps that move between the exact and the field zone rebuild neither
    int near_n = -1;
    T near_c[3] = {T(0), T(0), T(0)};
    for (unsigned it = 1;; it++) {
      int r = S_CONTINUE;
      double omc = 0.0;
      if ((it & 1023u) == 0) {
        if (tid == 0) sm_idx = (global_ns() > deadline || *(volatile int *)kp.error) ? 1ull : 0ull;
        __syncthreads();
        const bool e = sm_idx != 0;
        __syncthreads();
        if (e) {
          if (tid == 0) atomicExch(kp.error, 1);
          r = S_CAPPED;
        }
      }
      if (r == S_CONTINUE) {
        if (L.mode == M_STEP) first_half<T, GAS>(K, L);
        T p[NS][3], fs[NS][3], Us[NS];
        site_positions<T, GAS>(L, p);
        unsigned actbits;
        if (probe_near<T, GAS>(K, p, actbits)) {
          bool act[NS];
#pragma unroll
          for (int s = 0; s < NS; s++) act[s] = (actbits >> s) & 1u;
          bool surr = false;  // block-uniform: every thread holds the same state
          if constexpr (SURR) {
            surr = true;
#pragma unroll
            for (int s = 0; s < NS; s++)
              if (act[s]) surr &= !field_exact(kp.field, (float)p[s][0], (float)p[s][1], (float)p[s][2]);
          }
          if (surr) {
            if constexpr (SURR) {
              // the switched exact sums over the atoms within r_out ...
              T raw[RedShape<GAS>::NV];
              eval_forces_block<T, NT, GAS, HASQ, true>(K, p, act, p[S::cs], site_offset<T, GAS>(p), fs, Us, L.nvis,
                                                        tid, sm_list + kp.lcap, LCAP, sm_wsum, sm_red[red], near_n, near_c, Kg, raw);
              red ^= 1;
              // ... plus the far parts from the network, one warp per site
              for (int s = tid >> 5; s < NS; s += NT / 32) {
                int fl[FL_SITE_FIELDS];
                const int nfo = site_fields(kp.field, s, fl);
                float u[FL_SITE_FIELDS] = {0.f, 0.f, 0.f, 0.f}, gr[FL_SITE_FIELDS][3] = {};
                if (act[s]) {
                  const float x[3] = {(float)p[s][0], (float)p[s][1], (float)p[s][2]};
                  field_site_warp(kp.field, x, nfo, fl, u, gr);
                }
                if ((tid & 31) == 0)
                  for (int k = 0; k < FL_SITE_FIELDS; k++) {
                    sm_site[s][4 * k] = u[k];
                    sm_site[s][4 * k + 1] = gr[k][0]; sm_site[s][4 * k + 2] = gr[k][1]; sm_site[s][4 * k + 3] = gr[k][2];
                  }
              }
              __syncthreads();
              float ufar[NS], ffar[NS][3], Ef[3] = {0.f, 0.f, 0.f}, Jf[3][3];
  #pragma unroll
              for (int s = 0; s < NS; s++) {
                ufar[s] = sm_site[s][0];
                ffar[s][0] = sm_site[s][1]; ffar[s][1] = sm_site[s][2]; ffar[s][2] = sm_site[s][3];
              }
              const int ds = kp.field.dip_site;
  #pragma unroll
              for (int a = 0; a < 3; a++) {
                Ef[a] = ds >= 0 ? sm_site[ds < NS ? ds : 0][4 * (1 + a)] : 0.f;
  #pragma unroll
                for (int b = 0; b < 3; b++) Jf[a][b] = ds >= 0 ? -sm_site[ds < NS ? ds : 0][4 * (1 + a) + 1 + b] : 0.f;
              }
              __syncthreads();
              finish_split<T, GAS, HASQ>(K, raw, ufar, ffar, Ef, Jf, act, fs, Us);
            }
          } else {
            eval_forces_block<T, NT, GAS, HASQ>(K, p, act, p[S::cs], site_offset<T, GAS>(p), fs, Us, L.nvis,
                                                  tid, sm_list, kp.lcap, sm_wsum, sm_red[red], list_n, list_c, Kg);
            red ^= 1;
          }
        } else {
#pragma unroll
          for (int s = 0; s < NS; s++) fs[s][0] = fs[s][1] = fs[s][2] = Us[s] = T(0);
        }
        absorb_forces<T, GAS>(K, fs, Us, L);
        if (L.mode == M_INIT) { L.Ei += L.U; L.mode = M_STEP; continue; }
        if (L.mode == M_RESTART) { L.mode = M_STEP; continue; }
        T vc[3];
        r = second_half<T, GAS>(K, L, vc);
        if (r == S_CONTINUE) continue;
        if (r == S_SCATTER) omc = lane_chi<T, GAS>(Kg, L.j, vc[0], vc[1], vc[2]);
      }
      // the try has ended: scatter, capped (or watchdog), or a failed test
      if (spec) {
        if (tid == 0) {
          SpecOut o;
          o.omc = omc;
          o.steps = L.nsteps;
          o.nvis = L.nvis;
          o.code = r == S_SCATTER ? 1 : r == S_CAPPED ? 3 : r == S_RETRY_ANGLE ? 4 : 5;
          o.pad = 0;
          kp.spec_out[rec * SPEC_SLOTS + (L.tries - __ldcg(&kp.spec_rec[rec].tries))] = o;
        }
        break;
      }
      if (r == S_SCATTER) {
        if (tid == 0) write_result(K, L, 1, omc, blk);
        break;
      }
      if (r == S_CAPPED) {
        if (tid == 0) write_result(K, L, 3, 0.0, blk);
        break;
      }
      L.tries++;
      if (r == S_RETRY_ENERGY) L.maxTries++;
      L.dt = T(K.dt / (L.tries + 1));
      if (!(L.tries < L.maxTries && L.maxTries < 10)) {
        if (tid == 0) write_result(K, L, 2, 0.0, blk);
        break;
      }
      if (may_spec && !spec && L.tries >= kp.spec_from) {  // hand the remaining tries to the speculative phase
        if (tid == 0) {
          const bool drained = np <= kp.spec_max_parked || *(volatile unsigned long long *)kp.park_next >= np;
          const unsigned long long slot = drained ? atomicAdd(kp.spec_count, 1ull) : ~0ull;
          sm_idx = slot;
          if (slot < kp.spec_cap) {
            SpecRec R;
            R.Ei = (double)L.Ei;
            R.j = L.j;
            R.ion = L.ion;
            R.nsteps = L.nsteps;
            R.nvis = L.nvis;
            R.tries = L.tries;
            R.maxTries = L.maxTries;
            R.ready = 0;
            kp.spec_rec[slot] = R;
            __threadfence();  // the fields before the flag that publishes them
            *(volatile int *)&kp.spec_rec[slot].ready = 1;
          }
        }
        __syncthreads();
        const bool recorded = sm_idx < kp.spec_cap;
        __syncthreads();
        if (recorded) break;
      }
      load_init<T, GAS>(L, lane_setup<T, GAS>(Kg, L.j));
      L.mode = M_RESTART;
      list_n = -1;
      near_n = -1;
    }
    // a parked trajectory has ended (or its record is published): one fewer running
    if (tid == 0 && !spec && may_spec) {
      __threadfence();
      atomicAdd(kp.park_active, ~0ull);
    }
    __syncthreads();
  }
  __syncthreads();
  if (threadIdx.x < 6 && blk[threadIdx.x]) atomicAdd(&kp.stats[threadIdx.x], blk[threadIdx.x]);
}

// The speculative tries' verdict, one thread per record: the tries in order,
// with the reference's rules (System.cpp:453-473): a failed energy test
// grants one more try, at most 9 tries and 2 such grants; the first try that
// scatters decides.  Steps and visits add up over the tries that ran in
// sequence (those after the deciding one are not counted).  After a
// watchdog stop every record is reported capped.
template <bool BATCH>
__global__ void spec_resolve_kernel(KParams kp) {
  __shared__ unsigned long long blk[8];
  if (threadIdx.x < 8) blk[threadIdx.x] = 0ull;
  __syncthreads();
  unsigned long long n = *(volatile unsigned long long *)kp.spec_count;
  if (n > kp.spec_cap) n = kp.spec_cap;
  const unsigned long long r = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n) {
    const SpecRec R = kp.spec_rec[r];
    const KParams &K = ion_params<BATCH>(kp, R.ion);
    const bool stopped = *(volatile int *)kp.error != 0;
    uint32_t steps = R.nsteps, nvis = R.nvis;
    int tries = R.tries, maxTries = R.maxTries, st = stopped ? 3 : 2;
    double omc = 0.0;
    for (int k = R.tries; k <= 8 && !stopped; k++) {
      const SpecOut o = kp.spec_out[r * SPEC_SLOTS + (k - R.tries)];
      steps += o.steps;
      nvis += o.nvis;
      if (o.code == 1) { st = 1; omc = o.omc; break; }
      if (o.code == 3) { st = 3; break; }
      tries = k + 1;
      if (o.code == 5) maxTries++;
      if (!(tries < maxTries && maxTries < 10)) { st = 2; break; }
    }
    K.status[R.j] = (int8_t)st;
    K.omc[R.j] = st == 1 ? omc : 0.0;
    if (K.steps) K.steps[R.j] = steps;
    if (K.visits) K.visits[R.j] = nvis;
    atomicAdd(&blk[st], 1ull);
    atomicAdd(&blk[4], (unsigned long long)steps);
    atomicAdd(&blk[5], (unsigned long long)nvis);
  }
  __syncthreads();
  if (threadIdx.x < 6 && blk[threadIdx.x]) atomicAdd(&kp.stats[threadIdx.x], blk[threadIdx.x]);
}

// Site-force evaluation at given points (ccs_eval_site_forces): one group per point.
template <typename T, int G, int GAS, bool HASQ>
__global__ void __launch_bounds__(BLOCK)
    force_points_kernel(KParams kp, int site, size_t npts, const double *pts, double *f, double *U,
                        uint32_t *vis) {
  constexpr int NS = GasShape<GAS>::NS;
  __shared__ int sm_glist[BLOCK * GCAP_PER_LANE];
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
                                 sm_glist + (threadIdx.x & ~(G - 1)) * GCAP_PER_LANE);
    if (g == 0) {
      for (int k = 0; k < 3; k++) f[3 * i + k] = (double)ff[site][k];
      U[i] = (double)UU[site];
      if (vis) vis[i] = v;
    }
  }
}

// Expected-length key of every trajectory for longest-first scheduling:
// the chord through the ellipsoid's bounding sphere over the sampled speed.
// Slow probes with small impact parameters run longest (they are the ones
// captured into orbits and retried); starting them first keeps the longest
// serial chains off the end of the launch.  Only the order changes, never a result.
static __global__ void order_key_kernel(KParams kp, float *key, uint32_t *idx) {
  const size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= kp.ntraj) return;
  const double v = vel_sample(kp, kp.rnd[kp.rnd_stride + j]);
  const double b = kp.rnd[j] / kp.bmax;
  const double chord = sqrt(fmax(1.0 - b * b, 0.01));
  key[j] = (float)(chord / fmax(v, 1e-12));
  idx[j] = (uint32_t)j;
}

// Initial conditions (ccs_eval_setup): one thread per trajectory.
static __global__ void setup_kernel(KParams kp, int8_t *hit, double *pos, double *vel) {
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
