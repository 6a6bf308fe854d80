// equipotential.cpp -- the equipotential ellipsoid (cces-cepid/massccs
// src/Equipotential.cpp:19-715): the trajectories' start/end surface fitted
// to the points where the probe's potential energy falls to 1 % of the
// kinetic energy of a slow gas particle, instead of the geometric ellipsoid.
//
// Steps kept as the reference takes them (they define a, b, c):
//  - the energy threshold: Ek_min of the Maxwell-Boltzmann speed two
//    standard deviations below the mean speed, times 0.01 (:31-37, :99);
//  - the extent along z: from maxZ + 20 A in 0.5 A steps (:86-120), then
//    zMax x 1.3 and max(25, ceil(zMax)) z-levels;
//  - per z-level, 20 rays towards the z-axis in 0.1 A steps, from outside or
//    (when the start is inside the boundary) from inside out, keeping the
//    point of the crossing step farther from the origin (:128-200);
//  - a least-squares fit of x^2/a^2 + y^2/b^2 + z^2/c^2 = 1 (:560-640), then
//    all three axes grown in 0.01 A steps until every boundary point is
//    inside, at most to 3a (:668-715).
// The potentials are all-atom sums without cutoffs (:203-557); for N2 and CO2
// the three axis-aligned orientations of the probe are Boltzmann-averaged at
// 500 K.  The sums run in atom order (the reference's OpenMP reduction order
// depends on its thread count).
#include <algorithm>
#include <array>
#include <cmath>
#include <iostream>
#include <vector>

#include "massccs_gpu.h"
#include "setup.h"

namespace massccs {

namespace {
constexpr double kB = 1.38064E-23;       // BOLTZMANN_K (Constants.h:31)
constexpr double kAmuKg = 1.66053904E-27; // AMU_TO_KG (Constants.h:25)
constexpr double kJeV = 6.242E18;        // J_TO_eV (Constants.h:52)
constexpr double kEvKcal = 23.061;       // eV_TO_KCAL_MOL (Constants.h:54)
constexpr double kCoul = 332.06348078020324;  // KCOUL (Constants.h:63)

struct Probe {
  const MoleculeTarget &t;
  int gas;
  bool polar;
  double alpha;  // kcal/mol units

  double lj(double dx, double dy, double dz, double eps, double sig) const {
    const double r2inv = 1.0 / (dx * dx + dy * dy + dz * dz);
    const double r6inv = r2inv * r2inv * r2inv;
    const double lj1 = 4.0 * eps * std::pow(sig, 6), lj2 = lj1 * std::pow(sig, 6);
    return r6inv * (lj2 * r6inv - lj1);
  }

  // He, Ar and the one-site co2 (Equipotential.cpp:203-244)
  double atom(const double p[3]) const {
    double U = 0, E[3] = {0, 0, 0};
    for (int i = 0; i < t.natoms; i++) {
      const double dx = p[0] - t.x[i], dy = p[1] - t.y[i], dz = p[2] - t.z[i];
      U += lj(dx, dy, dz, t.eps[i], t.sig[i]);
      if (polar) {
        const double r2inv = 1.0 / (dx * dx + dy * dy + dz * dz);
        const double r3inv = std::sqrt(r2inv) * r2inv;
        E[0] += t.q[i] * dx * r3inv;
        E[1] += t.q[i] * dy * r3inv;
        E[2] += t.q[i] * dz * r3inv;
      }
    }
    if (polar) U -= 0.5 * alpha * (E[0] * E[0] + E[1] * E[1] + E[2] * E[2]);
    return U;
  }

  // N2 (:246-388) and CO2 (:391-557): end sites at +-d along each axis, the
  // central site at p; the three orientations weighted by exp(-dU/kT), 500 K
  double molecule(const double p[3]) const {
    const bool co2 = gas == 3;
    const double qc = co2 ? 0.6512 : 0.965, qe = -0.5 * qc, d = co2 ? 1.149 : 0.5488;
    double Ulj[6] = {0}, Uq[6] = {0}, Ulj_c = 0, Uq_c = 0, E[3] = {0, 0, 0};
    for (int i = 0; i < t.natoms; i++) {
      const double ax = t.x[i], ay = t.y[i], az = t.z[i], q = t.q[i];
      for (int k = 0; k < 6; k++) {
        const int axis = k / 2;
        const double s = (k % 2 == 0) ? d : -d;
        const double dx = p[0] + (axis == 0 ? s : 0.0) - ax;
        const double dy = p[1] + (axis == 1 ? s : 0.0) - ay;
        const double dz = p[2] + (axis == 2 ? s : 0.0) - az;
        Ulj[k] += lj(dx, dy, dz, t.eps[i], t.sig[i]);
        if (polar) Uq[k] += qe * q * std::sqrt(1.0 / (dx * dx + dy * dy + dz * dz)) * kCoul;
      }
      const double dx = p[0] - ax, dy = p[1] - ay, dz = p[2] - az;
      const double r2 = dx * dx + dy * dy + dz * dz;
      if (co2) Ulj_c += lj(dx, dy, dz, t.eps_c[i], t.sig_c[i]);
      if (polar) {
        const double rinv = 1.0 / std::sqrt(r2);
        Uq_c += qc * q * rinv * kCoul;
        const double r3inv = rinv * (1.0 / r2);
        E[0] += dx * q * r3inv;
        E[1] += dy * q * r3inv;
        E[2] += dz * q * r3inv;
      }
    }
    const double Uind = -0.5 * alpha * (E[0] * E[0] + E[1] * E[1] + E[2] * E[2]);
    double Umol[3];
    for (int o = 0; o < 3; o++)
      Umol[o] = Ulj[2 * o] + Ulj[2 * o + 1] + Uq[2 * o] + Uq[2 * o + 1] + Uind + (co2 ? Ulj_c : 0.0) + Uq_c;
    const double Umin = std::min(Umol[0], std::min(Umol[1], Umol[2]));
    const double kT = kB * 500.0 * kJeV * kEvKcal;
    double Z = 0;
    for (double u : Umol) Z += std::exp(-(u - Umin) / kT);
    double U = 0;
    for (double u : Umol) U += std::exp(-(u - Umin) / kT) / Z * u;
    return U;
  }

  double operator()(const double p[3]) const { return (gas == 2 || gas == 3) ? molecule(p) : atom(p); }
};

double norm3(const double p[3]) { return std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]); }
}  // namespace

void equipotential_ellipsoid(const MoleculeTarget &t, int gas, int polarizability_flag, double temperature,
                             double mu, double alpha, int nthreads, bool print, double &a, double &b, double &c,
                             int gpu_device) {
  const Probe U{t, gas, polarizability_flag != 0, alpha};
  // the energy threshold (Equipotential.cpp:31-37)
  const double v_mb = 2.0 * std::sqrt((2.0 * kB * temperature) / (M_PI * mu * kAmuKg));
  const double v2_mb = 3.0 * kB * temperature / (mu * kAmuKg);
  const double v_min = v_mb - 2.0 * std::sqrt(v2_mb - v_mb * v_mb);
  const double ek = 0.01 * (0.5 * mu * kAmuKg * std::pow(v_min, 2.0) * kJeV * kEvKcal);

  std::vector<std::array<double, 3>> pts;
  if (gpu_device >= 0) {
    // the marches on the GPU (ccs_equipotential_points): the same rays and
    // rules, each step's all-atom potential summed there
    const size_t cap = 64 * 20 + (size_t)(1.3 * (std::fabs(t.maxZ) + 20.0) + 64) * 20 * 4;
    std::vector<double> hits(3 * cap);
    size_t nh = 0;
    double zm = 0.0;
    const int rc = ccs_equipotential_points(gpu_device, (size_t)t.natoms, t.x.data(), t.y.data(), t.z.data(),
                                            t.q.data(), t.eps.data(), t.sig.data(),
                                            gas == 3 ? t.eps_c.data() : nullptr, gas == 3 ? t.sig_c.data() : nullptr,
                                            gas, polarizability_flag, alpha, ek, t.maxX, t.maxY, t.maxZ, cap,
                                            hits.data(), &nh, &zm);
    if (rc) throw std::runtime_error(std::string("equipotential on the GPU: ") + ccs_status_string(rc));
    for (size_t k = 0; k < nh; k++)
      if (!(hits[3 * k] == 0 && hits[3 * k + 1] == 0 && hits[3 * k + 2] == 0))
        pts.push_back({hits[3 * k], hits[3 * k + 1], hits[3 * k + 2]});
  } else {
    // extent along z (:86-120)
    double pos[3] = {0.0, 0.0, std::fabs(t.maxZ) + 20.0}, prev[3];
    double slope = (U(pos) + ek < 0.0) ? -1.0 : 1.0;
    double zMax = 0.0;
    for (;;) {
      std::copy(pos, pos + 3, prev);
      pos[2] -= 0.5 * slope;
      if ((U(pos) + ek) * slope < 0.0) {
        zMax = std::max(pos[2], prev[2]);
        break;
      }
    }

    // rays towards the z-axis on every z-level (:122-200)
    const int nrot = 20;
    const double velMag = 0.1;
    zMax *= 1.3;
    const double posMag = std::fabs(std::max(std::fabs(t.maxX), std::fabs(t.maxY))) + std::fabs(zMax - std::fabs(t.maxZ));
    const int levels = (int)std::ceil((double)std::max(25, (int)std::ceil(zMax)));
    const double zInc = 2 * zMax / levels;
    // every ray is independent: they run in parallel, each in sequence, and
    // the points keep the reference's (level, rotation) order
    const int nrays = (levels + 1) * nrot;
    std::vector<std::array<double, 3>> hits((size_t)nrays, std::array<double, 3>{0.0, 0.0, 0.0});
  #pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int ray = 0; ray < nrays; ray++) {
      const int i = ray / nrot, n = ray % nrot;
      const double zPos = -zMax + i * zInc;
      const double theta = n * 2.0 * M_PI / (double)nrot;
      const double startX = posMag * std::cos(theta), startY = posMag * std::sin(theta);
      double p[3] = {startX, startY, zPos}, pp[3] = {0.0, 0.0, 0.0};
      double vel[3] = {-velMag * std::cos(theta), -velMag * std::sin(theta), 0.0};
      const double s = (U(p) + ek < 0.0) ? -1.0 : 1.0;  // inside the boundary: search outwards
      for (double &v : vel) v *= s;
      for (;;) {
        if ((U(p) + ek) * s < 0.0) {
          const double *far = norm3(pp) > norm3(p) ? pp : p;  // the crossing step's farther point
          hits[(size_t)ray] = {far[0], far[1], far[2]};
          break;
        }
        // crossed to the other side of the molecule without meeting the boundary
        if ((startX == 0 && startY / p[1] <= 0) || (startY == 0 && startX / p[0] <= 0) ||
            (startX / p[0] <= 0 && startY / p[1] <= 0))
          break;
        std::copy(p, p + 3, pp);
        for (int k = 0; k < 3; k++) p[k] += vel[k];
      }
    }
    for (const auto &h : hits)
      if (!(h[0] == 0 && h[1] == 0 && h[2] == 0)) pts.push_back(h);
  }

  // least-squares ellipsoid through the points (:560-640)
  double m4[3] = {0, 0, 0}, m22[3] = {0, 0, 0}, m2[3] = {0, 0, 0};  // x4 y4 z4; x2y2 x2z2 y2z2; x2 y2 z2
  for (const auto &p : pts) {
    const double x2 = p[0] * p[0], y2 = p[1] * p[1], z2 = p[2] * p[2];
    m4[0] += x2 * x2; m4[1] += y2 * y2; m4[2] += z2 * z2;
    m22[0] += x2 * y2; m22[1] += x2 * z2; m22[2] += y2 * z2;
    m2[0] += x2; m2[1] += y2; m2[2] += z2;
  }
  const double mu4 = m4[0], nu4 = m4[1], ep4 = m4[2], de = m22[0], si = m22[1], rh = m22[2];
  const double al = m2[0], be = m2[1], ga = m2[2];
  const double det = ep4 * mu4 * nu4 - ep4 * de * de - mu4 * rh * rh + 2 * de * rh * si - nu4 * si * si;
  const double A = (al * (nu4 * ep4 - rh * rh) + de * (rh * ga - be * ep4) + si * (be * rh - nu4 * ga)) / det;
  const double B = (mu4 * (be * ep4 - ga * rh) + al * (rh * si - de * ep4) + si * (de * ga - be * si)) / det;
  const double C = (mu4 * (nu4 * ga - be * rh) + de * (be * si - de * ga) + al * (de * rh - nu4 * si)) / det;
  a = 1.0 / std::sqrt(A);
  b = 1.0 / std::sqrt(B);
  c = 1.0 / std::sqrt(C);
  const double npts = (double)pts.size();
  const double rmsd = std::sqrt((A * A * mu4 + B * B * nu4 + C * C * ep4 +
                                 2 * (A * B * de + B * C * rh + A * C * si - A * al - B * be - C * ga) + npts) /
                                (npts - 1));
  const double r2 = 2 * rmsd * rmsd;
  const double caa = r2 * (ep4 * nu4 - rh * rh) * a * a / (4 * A * A * det);
  const double cbb = r2 * (ep4 * mu4 - si * si) * b * b / (4 * B * B * det);
  const double ccc = r2 * (mu4 * nu4 - de * de) * c * c / (4 * C * C * det);
  const double cab = r2 * (rh * si - de * ep4) * a * b / (4 * A * B * det);
  const double cac = r2 * (de * rh - nu4 * si) * a * c / (4 * A * C * det);
  const double cbc = r2 * (de * si - mu4 * rh) * b * c / (4 * B * C * det);
  const double ua = (a / A) * std::sqrt((ep4 * nu4 - rh * rh) * 2 / det) * rmsd / 2;
  const double ub = (b / B) * std::sqrt((ep4 * mu4 - si * si) * 2 / det) * rmsd / 2;
  const double uc = (c / C) * std::sqrt((mu4 * nu4 - de * de) * 2 / det) * rmsd / 2;
  const double avg = (a + b + c) / 3.0;
  const double avgU = std::sqrt(caa + cbb + ccc + 2 * (cab + cac + cbc)) / 3.0;
  const double P = 1.6075;
  const double f = (std::pow(a * b, P) + std::pow(a * c, P) + std::pow(b * c, P)) / 3;
  const double area = 4 * M_PI * std::pow(f, 1.0 / P);
  const double da = area * std::pow(a, P - 1) * (std::pow(b, P) + std::pow(c, P)) / (3 * f);
  const double db = area * std::pow(b, P - 1) * (std::pow(a, P) + std::pow(c, P)) / (3 * f);
  const double dc = area * std::pow(c, P - 1) * (std::pow(a, P) + std::pow(b, P)) / (3 * f);
  const double areaU = std::sqrt(da * da * caa + db * db * cbb + dc * dc * ccc +
                                 2 * (da * db * cab + da * dc * cac + db * dc * cbc));
  if (print) {  // Equipotential::print (:643-666)
    std::cout << "*********************************************************" << std::endl;
    std::cout << "Equipotential Ellipsoid: " << std::endl;
    std::cout << "*********************************************************" << std::endl;
    std::cout << "Axis Length: " << a << "  " << b << "  " << c << "  Ang" << std::endl;
    std::cout << "Uncertainy: " << ua << "  " << ub << "  " << uc << std::endl;
    std::cout << "Percent Uncert: " << ua * 100 / a << "  " << ub * 100 / b << "  " << uc * 100 / b << std::endl;
    std::cout << "RMSD: " << rmsd << std::endl;
    std::cout << "Covariance matrix: " << rmsd << std::endl;
    std::cout << "{  " << caa << "  " << cab << "  " << cac << "  }" << std::endl;
    std::cout << "{  " << cab << "  " << cbb << "  " << cbc << "  }" << std::endl;
    std::cout << "{  " << cac << "  " << cbc << "  " << ccc << "  }" << std::endl;
    std::cout << "Average ellipsoid axes: " << avg << " +/- " << avgU << " Ang" << std::endl;
    std::cout << "Ellipsoid surface area: " << area << " +/- " << areaU << " Ang^2" << std::endl;
  }

  // grow until every boundary point is inside, at most to three times a (:668-715)
  const double a0 = a;
  for (bool grown = true; grown;) {
    grown = false;
    if (a > 3 * a0) break;
    for (const auto &p : pts) {
      if (p[0] * p[0] / (a * a) + p[1] * p[1] / (b * b) + p[2] * p[2] / (c * c) > 1) {
        a += 0.01;
        b += 0.01;
        c += 0.01;
        grown = true;
        break;
      }
    }
  }
  if (print) std::cout << "Ellipsoid axes further expanded by: " << a - a0 << " Ang" << std::endl;
}

}  // namespace massccs
