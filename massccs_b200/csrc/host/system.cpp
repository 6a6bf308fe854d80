// system.cpp -- System::System up to the trajectory loop, the pre-draw and
// the reduction (cces-cepid/massccs src/System.cpp:19-326, 1640-1698).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <iostream>
#include <random>
#include <vector>

#include "setup.h"

namespace massccs {

namespace {
double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace

std::string resolve_path(const std::string &json_path, const std::string &file) {
  if (!file.empty() && file[0] == '/') return file;
  const size_t slash = json_path.find_last_of('/');
  if (slash == std::string::npos) return file;
  return json_path.substr(0, slash) + "/" + file;
}

int select_force_type(const Input &in) {  // System.cpp:49-87
  const int g = in.gas_buffer_flag, s = in.short_range_cutoff, l = in.long_range_flag,
            lc = in.long_range_cutoff, p = in.polarizability_flag;
  if (g == 1 || g == 4 || g == 5) {
    if (s == 0 && l == 0) return 1;
    if (s == 1 && l == 0) return 2;
    if (s == 0 && p == 1 && lc == 0) return 3;
    if (s == 1 && p == 1 && lc == 1) return 4;
    return 2;
  }
  if (s == 0 && l == 0 && p == 0) return 1;
  if (s == 1 && l == 0 && p == 0) return 2;
  if (s == 0 && l == 1 && lc == 0 && p == 0) return 3;
  if (s == 1 && l == 1 && lc == 1 && p == 0) return 4;
  if (s == 0 && l == 1 && lc == 0 && p == 1) return 5;
  if (s == 1 && l == 1 && lc == 1 && p == 1) return 6;
  return 2;
}

namespace {
Input read_and_print(const std::string &json_path, bool print) {
  Input in(json_path);
  if (print) in.print();
  return in;
}
MoleculeTarget build_target(const Input &in, const std::string &json_path, bool print, double &t) {
  const double t0 = now_s();
  const std::string ff = in.user_ff_flag ? resolve_path(json_path, in.user_ff) : std::string();
  MoleculeTarget tg(resolve_path(json_path, in.targetFilename), in.gas_buffer_flag, ff, in.user_ff_flag != 0,
                    select_force_type(in));
  t = now_s() - t0;
  if (print) {
    tg.printFF(in.gas_buffer_flag);
    tg.print();
    std::cout << "orientation time of molecule target: " << t << " s" << std::endl;
  }
  return tg;
}
}  // namespace

SystemSetup::SystemSetup(const std::string &json_path, bool print)
    : in(read_and_print(json_path, print)),
      gas(in.gas_buffer_flag),
      target(build_target(in, json_path, print, t_orient)) {
  force_type = select_force_type(in);
  const int g = in.gas_buffer_flag;
  // reduced mass, molecular inertia (System.cpp:97-114)
  if (g == 1 || g == 4 || g == 5) {
    mu = target.mass * gas.mass / (target.mass + gas.mass);
  } else {
    mu = gas.mass;
    gas_inertia = 0.0;
    for (int i = 0; i < gas.natoms; i++) gas_inertia += gas.m[i] * std::pow(gas.z[i], 2);
    d_bond = gas.d;
  }
  if (print) {
    std::cout << "target mass: " << target.mass << " amu" << std::endl;
    std::cout << "gas mass: " << gas.mass << " amu" << std::endl;
    std::cout << "reduce mass: " << mu << " amu" << std::endl;
    std::cout << "charge state: " << target.Q << " e" << std::endl;
  }
  alpha = in.alpha * 331.842254885;  // ALPHA_TO_KCAL_MOL (System.cpp:117)

  double t0 = now_s();
  if (in.equipotential_flag == 1) {  // System.cpp:120-126
    // the rays' all-atom potentials on the GPU for large targets (setup_device)
    const bool gpu = in.setup_device == "gpu" || (in.setup_device == "auto" && target.natoms >= 20000);
    const int dev = gpu ? (in.devices.empty() ? 0 : in.devices[0]) : -1;
    equipotential_ellipsoid(target, g, in.polarizability_flag, in.temperatureTarget, mu, alpha,
                            (int)std::max(1u, in.nthreads), print, a, b, c, dev);
    if (print) std::cout << "ellipsoid axis length: " << a << "  " << b << "  " << c << "  Ang" << std::endl;
  } else {
    geometric_ellipsoid(print);
  }
  t_ellipsoid = now_s() - t0;
  if (print) std::cout << "ellipsoid calculation time: " << t_ellipsoid << " s" << std::endl;
  bmax = std::fmax(std::fmax(a, b), c);
  if (print) std::cout << "maximal impact parameter: " << bmax << " Ang" << std::endl;

  // the reference's cell box (LinkedCell.cpp:48-90); its statistics are
  // reported as the reference does (LinkedCell.cpp:443-480)
  t0 = now_s();
  cell_size = in.lj_cutoff + in.skin;
  Nx = (int)std::ceil(2.0 * a / cell_size);
  Ny = (int)std::ceil(2.0 * b / cell_size);
  Nz = (int)std::ceil(2.0 * c / cell_size);
  const double Lx = Nx * cell_size, Ly = Ny * cell_size, Lz = Nz * cell_size;
  lx = 0.5 * Lx;
  ly = 0.5 * Ly;
  lz = 0.5 * Lz;
  if (print) {
    std::vector<int> count((size_t)Nx * Ny * Nz, 0);
    for (int i = 0; i < target.natoms; i++) {
      const int ci = (int)std::floor((target.x[i] + lx) / cell_size);
      const int cj = (int)std::floor((target.y[i] + ly) / cell_size);
      const int ck = (int)std::floor((target.z[i] + lz) / cell_size);
      const long idx = ck + (long)Nz * cj + (long)Nz * Ny * ci;
      if (idx >= 0 && idx < (long)count.size()) count[(size_t)idx]++;
    }
    int filled = 0, empty = 0, sum = 0, mx = 0, mn = target.natoms;
    for (int n : count) {
      if (n == 0) { empty++; continue; }
      filled++;
      sum += n;
      mx = std::max(mx, n);
      mn = std::min(mn, n);
    }
    t_cells = now_s() - t0;
    std::cout << "*********************************************************" << std::endl;
    std::cout << "Linked-cell: " << std::endl;
    std::cout << "Numbers of cells: " << (long)Nx * Ny * Nz << std::endl;
    std::cout << "Nx: " << Nx << " Ny: " << Ny << " Nz: " << Nz << std::endl;
    std::cout << "Filled cells: " << filled << std::endl;
    std::cout << "Empty cells: " << empty << std::endl;
    std::cout << "Average atoms per cell: " << ((float)sum) / ((float)filled) << std::endl;
    std::cout << "Maximum atoms per cell: " << mx << std::endl;
    std::cout << "Minimum atoms per cell: " << mn << std::endl;
    std::cout << "Simulation box: " << std::endl;
    std::cout << "lx: " << Lx << " Ang" << std::endl;
    std::cout << "ly: " << Ly << " Ang" << std::endl;
    std::cout << "lz: " << Lz << " Ang" << std::endl;
    std::cout << "linked-cell calculation time: " << t_cells << " s" << std::endl;
  }
}

// System::geometric_ellipsoid (System.cpp:1640-1698)
void SystemSetup::geometric_ellipsoid(bool print) {
  // geometric ellipsoid (System.cpp:1640-1698): axes grown in 0.01 A steps
  // until every atom pushed outward by radius + d lies inside
  const double mX = std::fabs(target.maxX), mY = std::fabs(target.maxY), mZ = std::fabs(target.maxZ);
  const double d = gas.d;
  const double radius = in.long_range_flag == 1 ? 2.0 * in.coul_cutoff : 2.0 * in.lj_cutoff;
  if (print) {
    std::cout << "*********************************************************" << std::endl;
    std::cout << "Geometric Ellipsoid: " << std::endl;
    std::cout << "*********************************************************" << std::endl;
    std::cout << "maximal distances: " << mX << "  " << mY << "  " << mZ << "  Ang" << std::endl;
  }
  a = mX + radius + in.skin + d;
  b = mY + radius + in.skin + d;
  c = mZ + radius + in.skin + d;
  if (print) std::cout << "Initial axis length: " << a << "  " << b << "  " << c << "  Ang" << std::endl;
  for (int i = 0; i < target.natoms; i++) {
    const double xi = target.x[i], yi = target.y[i], zi = target.z[i];
    const double ri = std::sqrt(xi * xi + yi * yi + zi * zi);
    const double px = xi + (radius + d) * (xi / ri), py = yi + (radius + d) * (yi / ri),
                 pz = zi + (radius + d) * (zi / ri);
    while (std::pow(px / a, 2) + std::pow(py / b, 2) + std::pow(pz / c, 2) > 1.0) {
      a += 0.01;
      b += 0.01;
      c += 0.01;
    }
  }
  if (print) std::cout << "Ellipsoid axis length: " << a << "  " << b << "  " << c << "  Ang" << std::endl;
}

namespace {
// MT19937 (Matsumoto and Nishimura, 1998), the generator the reference draws
// from (std::mt19937 in RandomNumber.cpp:19-29), producing whole blocks of
// 624 tempered words: the bulk form of the same sequence.  The twist is
// split where its index wraps, so both halves and the tempering vectorise.
constexpr int MT_N = 624, MT_M = 397;

inline uint32_t mt_mix(uint32_t a, uint32_t b, uint32_t c) {
  const uint32_t y = (a & 0x80000000u) | (b & 0x7fffffffu);
  return c ^ (y >> 1) ^ ((0u - (y & 1u)) & 0x9908b0dfu);
}

__attribute__((target_clones("avx2", "default")))
void mt_block(uint32_t *__restrict s, uint32_t *__restrict out) {
  for (int i = 0; i < MT_N - MT_M; i++) s[i] = mt_mix(s[i], s[i + 1], s[i + MT_M]);
  for (int i = MT_N - MT_M; i < MT_N - 1; i++) s[i] = mt_mix(s[i], s[i + 1], s[i + MT_M - MT_N]);
  s[MT_N - 1] = mt_mix(s[MT_N - 1], s[0], s[MT_M - 1]);
  for (int i = 0; i < MT_N; i++) {
    uint32_t y = s[i];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    out[i] = y;
  }
}

struct Mt19937Bulk {
  static constexpr int N = MT_N;
  uint32_t s[MT_N];
  explicit Mt19937Bulk(uint32_t seed) {
    s[0] = seed;
    for (int i = 1; i < MT_N; i++) s[i] = 1812433253u * (s[i - 1] ^ (s[i - 1] >> 30)) + (uint32_t)i;
  }
  void block(uint32_t *out) { mt_block(s, out); }  // the next 624 outputs
};
}  // namespace

void predraw(const SystemSetup &S, uint32_t seed, size_t n, double *rnd) {
  // System.cpp:185-197: per trajectory u1 (as sqrt(bmax^2 u1)), u2..u5, and
  // u6..u9 for N2/CO2, in trajectory order; u = (r - min) / max
  // (RandomNumber::getRandomNumber, RandomNumber.cpp:27-29).  The words are
  // generated in bulk (the sequence is serial), then converted in parallel:
  // the same divisions and square roots, so the same bits.
  const bool mol = S.in.gas_buffer_flag == 2 || S.in.gas_buffer_flag == 3;
  const size_t K = mol ? 9 : 5;
  const size_t total = K * n, blocks = (total + Mt19937Bulk::N - 1) / Mt19937Bulk::N;
  std::vector<uint32_t> raw(blocks * Mt19937Bulk::N);
  Mt19937Bulk mt(seed);
  for (size_t b = 0; b < blocks; b++) mt.block(raw.data() + b * Mt19937Bulk::N);
  const double mn = (double)std::mt19937::min(), mx = (double)std::mt19937::max();
  const double bmax2 = S.bmax * S.bmax;
#pragma omp parallel for schedule(static) num_threads((int)std::max(1u, S.in.nthreads))
  for (long long jj = 0; jj < (long long)n; jj++) {
    const size_t j = (size_t)jj;
    const uint32_t *r = raw.data() + j * K;
    rnd[j] = std::sqrt(bmax2 * (((double)r[0] - mn) / mx));
    for (size_t k = 1; k < K; k++) rnd[k * n + j] = ((double)r[k] - mn) / mx;
    if (!mol)
      for (size_t k = 5; k < 9; k++) rnd[k * n + j] = 0.0;
  }
}

Reduction reduce(size_t niter, size_t nprobe, const int8_t *status, const double *omc, double bmax) {
  Reduction R;
  R.omega.resize(niter);
  R.nfree.resize(niter);
  R.nscatter.resize(niter);
  R.nlost.resize(niter);
  double Om = 0.0, Om2 = 0.0;
  size_t count = 0;
  const double pi = 3.14159265358979323846;
  for (size_t i = 0; i < niter; i++) {
    double dOmega = 0.0;
    int ns = 0, nf = 0, nl = 0;
    for (size_t j = 0; j < nprobe; j++, count++) {
      if (status[count] == 1) dOmega += pi * omc[count] * std::pow(bmax, 2.0);
      ns += status[count] == 1;
      nf += status[count] == 0;
      nl += status[count] >= 2;  // lost, and capped (which the reference would never finish)
    }
    const double w = 1.0 / ((double)(float)(ns + nf)) * dOmega;  // float() as System.cpp:301
    Om += w;
    Om2 += std::pow(w, 2.0);
    R.omega[i] = w;
    R.nfree[i] = nf;
    R.nscatter[i] = ns;
    R.nlost[i] = nl;
  }
  R.ccs = Om / niter;
  const double sig2 = Om2 / niter - std::pow(R.ccs, 2.0);
  R.err = std::sqrt(sig2 / (double)(float)niter);
  return R;
}

}  // namespace massccs
