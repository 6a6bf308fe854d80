// setup.h -- host side of massccs_b200: the reference's input, gas, target
// and system set-up (cces-cepid/massccs src/Input.cpp, src/GasBuffer.cpp,
// src/MoleculeTarget.cpp, src/System.cpp:19-144), re-implemented for the
// GPU engine.  The trajectory loop itself runs on the device (ccs_run).
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace massccs {

// input.json (Input.cpp:49-263): a flat object of strings and numbers.
struct Input {
  std::string targetFilename, user_ff;
  unsigned nProbe = 10000, nIter = 10, seed = 20162104, nthreads = 1;
  double dt = 10.0, temperatureTarget = 298.0, skin = 0.01;
  double lj_cutoff = 12.0, coul_cutoff = 25.0, alpha = 0.0;
  int gas_buffer_flag = 1, equipotential_flag = 0, short_range_cutoff = 1, long_range_flag = 0,
      long_range_cutoff = 1, polarizability_flag = 1, user_ff_flag = 0;
  std::string gas_str = "He", equip_str = "no", short_str = "yes", long_str = "no", long_cut_str = "yes",
              polar_str = "yes";
  bool ref_quirks = false;   // extension key "ref_quirks": reproduce the CO2 reference-velocity bug
  std::string precision = "fp32";  // extension key "precision": "fp32" or "fp64"
  unsigned fp64_check = 2000;      // extension key "fp64_check": FP32 runs rerun this many trajectories in FP64
  std::vector<int> devices;        // extension key "devices": a count N (GPUs 0..N-1) or a list "0,2,3"
  std::string setup_device = "auto";  // extension key "setup_device": where the equipotential rays run:
                                      // "cpu", "gpu", or "auto" (the GPU from 20,000 atoms on)

  explicit Input(const std::string &path);
  void print() const;  // Input::printReadInput (Input.cpp:313-345)
};

// Probe sites (GasBuffer.cpp:58-192).
struct GasBuffer {
  int natoms = 1;
  std::string type;
  double x[3] = {0, 0, 0}, y[3] = {0, 0, 0}, z[3] = {0, 0, 0};
  double q[3] = {0, 0, 0}, m[3] = {0, 0, 0}, eps[3] = {0, 0, 0}, sig[3] = {0, 0, 0};
  double mass = 0, d = 0;
  explicit GasBuffer(int flag);
};

// Target molecule in the principal-axis frame (MoleculeTarget.cpp:19-931).
struct MoleculeTarget {
  int natoms = 0;
  std::vector<std::string> name;
  std::vector<double> x, y, z, q, m, eps, sig, eps_c, sig_c;
  double mass = 0, Q = 0, maxX = 0, maxY = 0, maxZ = 0, radius = 0;
  double inertia[3][3] = {}, vectors[3][3] = {};
  bool diagonal = false;
  // force-field table
  std::vector<std::string> ff_name;
  std::vector<double> ff_m, ff_eps, ff_sig;

  MoleculeTarget(const std::string &file, int gas_flag, const std::string &user_ff, bool user_ff_flag,
                 int force_type);
  void printFF(int gas_flag) const;
  void print() const;

 private:
  int gas_flag_ = 1;
  bool user_ff_flag_ = false;
  void defaultFF();
  void readUserFF(const std::string &path);
  void readXYZ(const std::string &path, int force_type);
  void readPQR(const std::string &path);
  void assign(int i, const std::string &sym);
  bool assign_found(int i, const std::string &sym);  // false: type not in the force field
  [[noreturn]] void unknown_type() const;
  void moveToCenterOfMass();
  void calculateMoleculeRadius();
  void orientateMolecule();
  void setInertia();
};

// System::System up to the trajectory loop (System.cpp:19-144).
struct SystemSetup {
  Input in;
  GasBuffer gas;
  MoleculeTarget target;
  int force_type = 2;
  double mu = 0, alpha = 0, gas_inertia = 0, d_bond = 0;
  double a = 0, b = 0, c = 0, bmax = 0;
  double lx = 0, ly = 0, lz = 0;  // half box
  int Nx = 0, Ny = 0, Nz = 0;
  double cell_size = 0;
  double t_orient = 0, t_ellipsoid = 0, t_cells = 0;

  SystemSetup(const std::string &json_path, bool print);

 private:
  void geometric_ellipsoid(bool print);
};

// the equipotential ellipsoid (Equipotential.cpp:19-715): a, b, c of the
// surface where the probe's potential is 1 % of a slow particle's kinetic energy
void equipotential_ellipsoid(const MoleculeTarget &t, int gas, int polarizability_flag, double temperature,
                             double mu, double alpha, int nthreads, bool print, double &a, double &b, double &c,
                             int gpu_device = -1);

int select_force_type(const Input &in);  // System.cpp:49-87
std::string resolve_path(const std::string &json_path, const std::string &file);

// the reference's pre-draw (System.cpp:184-197) into 9 rows of n
void predraw(const SystemSetup &S, uint32_t seed, size_t n, double *rnd);

struct Reduction {
  std::vector<double> omega;
  std::vector<int32_t> nfree, nscatter, nlost;
  double ccs = 0, err = 0;
};
// per-iteration reduction (System.cpp:287-321)
Reduction reduce(size_t niter, size_t nprobe, const int8_t *status, const double *omc, double bmax);

}  // namespace massccs
