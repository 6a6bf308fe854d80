// molecule.cpp -- probe gases and the target molecule (cces-cepid/massccs
// src/GasBuffer.cpp:19-192, src/MoleculeTarget.cpp:19-931).
//
// The target is read from .xyz (4 columns, or 5 with charges) or .pqr, given
// the per-gas Lennard-Jones pair parameters of the built-in tables or of a
// user .ff file, moved to its centre of mass and rotated to its principal
// axes with the longest extent on z -- the frame the trajectory loop uses.
#include <charconv>
#include <cmath>
#include <cstring>
#include <string_view>
#include <fstream>
#include <iostream>
#include <sstream>
#include <vector>

#include "setup.h"

namespace massccs {

GasBuffer::GasBuffer(int flag) {
  switch (flag) {
    case 1:
      natoms = 1; type = "He"; m[0] = 4.0026; eps[0] = 0.0309008; sig[0] = 3.043;
      mass = m[0];
      break;
    case 2:  // two N atoms and a massless central charge
      natoms = 3; type = "N2";
      z[0] = 0.5488; z[1] = -0.5488;
      q[0] = q[1] = -0.4825; q[2] = 0.965;
      m[0] = m[1] = 14.007;
      eps[0] = eps[1] = 1.0;
      mass = m[0] + m[1];
      d = std::fabs(z[0] - z[1]);
      break;
    case 3:  // O - C - O, Harris and Yung
      natoms = 3; type = "CO2";
      z[0] = -1.149; z[2] = 1.149;
      q[0] = q[2] = -0.3256; q[1] = 0.6512;
      m[0] = m[2] = 15.999; m[1] = 12.011;
      eps[0] = eps[2] = 0.159; eps[1] = 0.055;
      sig[0] = sig[2] = 3.033; sig[1] = 2.757;
      mass = m[0] + m[1] + m[2];
      d = std::fabs(z[0] - z[2]);
      break;
    case 4:
      natoms = 1; type = "Ar"; m[0] = 39.948; eps[0] = 0.185; sig[0] = 3.446;
      mass = m[0];
      break;
    case 5:
      natoms = 1; type = "co2"; m[0] = 44.0098; eps[0] = 0.4008; sig[0] = 4.444;
      mass = m[0];
      break;
    default:
      throw std::invalid_argument("unknown gas buffer");
  }
}

namespace {
struct FFRow {
  const char *sym;
  double m, eps, sig;
};
}  // namespace

// MoleculeTarget::defaultFF (MoleculeTarget.cpp:372-538)
void MoleculeTarget::defaultFF() {
  static const FFRow he[] = {{"C", 12.011, 0.0309, 3.043}, {"N", 14.007, 0.0309, 3.043},
                             {"H", 1.008, 0.0150, 2.38},   {"O", 15.999, 0.0309, 3.043},
                             {"S", 32.06, 0.0311, 3.5}};
  static const FFRow n2[] = {{"C", 12.011, 0.0824736, 3.2255}, {"N", 14.007, 0.0758527, 3.5719},
                             {"H", 1.008, 0.0362711, 1.8986},  {"O", 15.999, 0.062323, 3.0750},
                             {"S", 32.06, 0.138032, 3.4237},   {"P", 30.9738, 0.145372, 3.47},
                             {"F", 18.9984, 0.04649, 3.1285}};
  static const FFRow uff[] = {{"C", 12.011, 0.10499, 3.43085}, {"N", 14.007, 0.06899, 3.26069},
                              {"H", 1.008, 0.04399, 2.57113},  {"O", 15.999, 0.05999, 3.11815},
                              {"S", 32.06, 0.27399, 3.59478},  {"P", 30.9738, 0.30499, 3.69456}};
  static const FFRow imos[] = {{"C", 12.011, 0.09759, 3.58140}, {"N", 14.007, 0.05579, 3.25500},
                               {"H", 1.008, 0.01892, 1.24090},  {"O", 15.999, 0.08279, 4.39200},
                               {"S", 32.06, 0.05999, 3.50000},  {"P", 30.9738, 0.05999, 3.50000},
                               {"K", 39.0983, 0.05999, 3.50000}};
  const FFRow *rows;
  size_t n;
  if (gas_flag_ == 1) { rows = he; n = 5; }
  else if (gas_flag_ == 2) { rows = n2; n = 7; }
  else if (gas_flag_ == 3 || gas_flag_ == 4) { rows = uff; n = 6; }
  else { rows = imos; n = 7; }
  for (size_t i = 0; i < n; i++) {
    ff_name.push_back(rows[i].sym);
    ff_m.push_back(rows[i].m);
    ff_eps.push_back(rows[i].eps);
    ff_sig.push_back(rows[i].sig);
  }
}

// MoleculeTarget::readUserFF (MoleculeTarget.cpp:321-370)
void MoleculeTarget::readUserFF(const std::string &path) {
  std::ifstream f(path);
  std::string line;
  int n = 0;
  if (!f || !std::getline(f, line) || !(std::istringstream(line) >> n) || n < 0)
    throw std::invalid_argument("Error: reading force-field parameters file " + path);
  std::getline(f, line);  // comment
  for (int i = 0; i < n; i++) {
    std::string sym;
    double m, e, s;
    if (!std::getline(f, line) || !(std::istringstream(line) >> sym >> m >> e >> s))
      throw std::invalid_argument("Error: reading force-field parameters file " + path);
    ff_name.push_back(sym);
    ff_m.push_back(m);
    ff_eps.push_back(e);
    ff_sig.push_back(s);
  }
}

// MoleculeTarget::assignedParameter (MoleculeTarget.cpp:540-570): pair
// parameters per gas; Lorentz-Berthelot mixing for CO2 (O and C sites) and Ar.
void MoleculeTarget::assign(int i, const std::string &sym) {
  if (!assign_found(i, sym)) unknown_type();
}

void MoleculeTarget::unknown_type() const {
  throw std::invalid_argument(user_ff_flag_ ? "Atom type not found in the file user force field"
                                            : "Atom type not found in the default data base ");
}

// the lookup itself: reads the tables only, so atoms may be assigned in parallel
bool MoleculeTarget::assign_found(int i, const std::string &sym) {
  for (size_t k = 0; k < ff_name.size(); k++) {
    if (sym != ff_name[k]) continue;
    m[i] = ff_m[k];
    if (gas_flag_ == 3) {
      eps[i] = std::sqrt(ff_eps[k] * 0.159);
      sig[i] = 0.5 * (ff_sig[k] + 3.033);
      eps_c[i] = std::sqrt(ff_eps[k] * 0.055);
      sig_c[i] = 0.5 * (ff_sig[k] + 2.757);
    } else if (gas_flag_ == 4) {
      eps[i] = std::sqrt(ff_eps[k] * 0.185);
      sig[i] = 0.5 * (ff_sig[k] + 3.446);
    } else {
      eps[i] = ff_eps[k];
      sig[i] = ff_sig[k];
    }
    return true;
  }
  return false;
}

namespace {
void resize_all(MoleculeTarget &t, int n) {
  t.natoms = n;
  t.name.assign(n, "");
  for (auto *v : {&t.x, &t.y, &t.z, &t.q, &t.m, &t.eps, &t.sig, &t.eps_c, &t.sig_c}) v->assign(n, 0.0);
}
}  // namespace

// Fast text input for multi-million-atom targets: the file is read whole and
// split into lines and whitespace tokens in place; numbers go through
// std::from_chars (correctly rounded, as the stream extraction the format
// was defined with).  A line whose tokens are not plain numbers where numbers
// are expected is parsed again with std::istringstream, so every input reads
// exactly as with stream extraction.
namespace {
bool slurp(const std::string &path, std::string &buf) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return false;
  f.seekg(0, std::ios::end);
  const std::streamoff size = f.tellg();
  if (size < 0) return false;
  buf.resize((size_t)size);
  f.seekg(0, std::ios::beg);
  return size == 0 || (bool)f.read(&buf[0], size);
}

// std::getline's lines: split at '\n', the '\n' dropped, a last line kept
// only if it holds characters
struct Lines {
  const char *p, *end;
  bool next(std::string_view &line) {
    if (p >= end) return false;
    const char *q = static_cast<const char *>(std::memchr(p, '\n', (size_t)(end - p)));
    const char *stop = q ? q : end;
    line = std::string_view(p, (size_t)(stop - p));
    p = q ? q + 1 : end;
    return true;
  }
};

inline bool space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; }

// the whitespace tokens of a line: up to maxt stored, all counted
int tokens(std::string_view line, std::string_view *tok, int maxt) {
  int n = 0;
  size_t i = 0;
  while (true) {
    while (i < line.size() && space(line[i])) i++;
    if (i >= line.size()) return n;
    const size_t j = i;
    while (i < line.size() && !space(line[i])) i++;
    if (n < maxt) tok[n] = line.substr(j, i - j);
    n++;
  }
}

// a whole token that is a plain decimal number (what stream extraction reads
// the same way); anything else returns false and the caller falls back
bool plain_double(std::string_view t, double &v) {
  if (!t.empty() && t[0] == '+') t.remove_prefix(1);
  if (t.empty()) return false;
  const char c = t[0];
  if (!(c == '-' || c == '.' || (c >= '0' && c <= '9'))) return false;
  if (c == '-' && (t.size() < 2 || !(t[1] == '.' || (t[1] >= '0' && t[1] <= '9')))) return false;
  const auto r = std::from_chars(t.data(), t.data() + t.size(), v);
  return r.ec == std::errc() && r.ptr == t.data() + t.size();
}
bool plain_long(std::string_view t, long &v) {
  if (!t.empty() && t[0] == '+') t.remove_prefix(1);
  if (t.empty() || t[0] == '+') return false;
  const auto r = std::from_chars(t.data(), t.data() + t.size(), v);
  return r.ec == std::errc() && r.ptr == t.data() + t.size();
}
}  // namespace

// MoleculeTarget::readXYZfile (MoleculeTarget.cpp:148-319): atom count, a
// comment line, then "Sym x y z" or "Sym x y z q" (charges dropped for force
// types 1 and 2); every line must carry the same number of items.
void MoleculeTarget::readXYZ(const std::string &path, int force_type) {
  std::string buf;
  if (!slurp(path, buf)) throw std::invalid_argument("Error: missing number ot atoms in xyz file");
  Lines L{buf.data(), buf.data() + buf.size()};
  std::string_view line;
  int n = 0;
  if (!L.next(line) || !(std::istringstream(std::string(line)) >> n) || n < 0)
    throw std::invalid_argument("Error: missing number ot atoms in xyz file");
  L.next(line);  // comment
  std::vector<std::string_view> lines;
  lines.reserve((size_t)n);
  while (L.next(line)) lines.push_back(line);
  // every line must carry as many items as the first one (lines are
  // independent: counted in parallel)
  const long nl = (long)lines.size();
  std::string_view tok0[5];
  const int items0 = nl ? tokens(lines[0], tok0, 5) : -1;
  long bad = 0;
#pragma omp parallel for schedule(static) reduction(+ : bad)
  for (long i = 1; i < nl; i++) {
    std::string_view tk[5];
    bad += tokens(lines[(size_t)i], tk, 5) != items0;
  }
  if (bad) throw std::invalid_argument("Error: numbers of items by lines in the xyz file");
  if ((int)lines.size() != n)
    throw std::invalid_argument("Error: numbers of lines and natoms are differens in the xyz file");
  const bool charges = items0 != 4;
  resize_all(*this, n);
  // atoms are parsed in parallel (each writes only its own entries); the
  // totals are then summed in atom order, as the reference does
  int unknown = 0;
#pragma omp parallel for schedule(static) reduction(+ : unknown)
  for (int i = 0; i < n; i++) {
    std::string_view tok[5];
    std::string sym;
    double xi = 0, yi = 0, zi = 0, qi = 0;
    const int nt = tokens(lines[(size_t)i], tok, 5);
    if (nt >= 4 && plain_double(tok[1], xi) && plain_double(tok[2], yi) && plain_double(tok[3], zi) &&
        (!charges || (nt >= 5 && plain_double(tok[4], qi)))) {
      sym = std::string(tok[0]);
    } else {  // stream extraction, as the format defines it
      xi = yi = zi = qi = 0;
      std::istringstream is{std::string(lines[(size_t)i])};
      is >> sym >> xi >> yi >> zi;
      if (charges) is >> qi;
    }
    if (!charges || force_type == 1 || force_type == 2) qi = 0.0;
    name[i] = sym;
    unknown += !assign_found(i, sym);
    x[i] = xi; y[i] = yi; z[i] = zi; q[i] = qi;
  }
  if (unknown) unknown_type();
  for (int i = 0; i < n; i++) {
    mass += m[i];
    Q += q[i];
  }
}

// MoleculeTarget::readPQRfile (MoleculeTarget.cpp:60-146): whitespace fields
// "ATOM serial name resName resSeq x y z q r"; the element is the first
// letter of the atom name unless a user force field is given.
void MoleculeTarget::readPQR(const std::string &path) {
  std::string buf;
  if (!slurp(path, buf)) throw std::invalid_argument("Error: reading pqr file " + path);
  Lines L{buf.data(), buf.data() + buf.size()};
  std::string_view line;
  std::vector<std::string_view> atoms;
  std::string_view tok[9];
  while (L.next(line))
    if (tokens(line, tok, 1) > 0 && tok[0] == "ATOM") atoms.push_back(line);
  resize_all(*this, (int)atoms.size());
  // records parsed in parallel (each writes only its own entries); totals
  // summed in atom order, as the reference does
  long first_unknown = natoms, first_bad = natoms;
#pragma omp parallel for schedule(static) reduction(min : first_unknown, first_bad)
  for (int i = 0; i < natoms; i++) {
    std::string_view tk[9];
    std::string aname;
    long serial, chain;
    double xi = 0, yi = 0, zi = 0, qi = 0;
    if (tokens(atoms[(size_t)i], tk, 9) >= 9 && plain_long(tk[1], serial) && plain_long(tk[4], chain) &&
        plain_double(tk[5], xi) && plain_double(tk[6], yi) && plain_double(tk[7], zi) &&
        plain_double(tk[8], qi)) {
      aname = std::string(tk[2]);
    } else {  // stream extraction, as the format defines it
      std::istringstream is{std::string(atoms[(size_t)i])};
      std::string rec, res;
      if (!(is >> rec >> serial >> aname >> res >> chain >> xi >> yi >> zi >> qi)) {
        first_bad = std::min(first_bad, (long)i);
        continue;
      }
    }
    const std::string sym = user_ff_flag_ ? aname : aname.substr(0, 1);
    name[i] = sym;
    if (!assign_found(i, sym)) first_unknown = std::min(first_unknown, (long)i);
    x[i] = xi; y[i] = yi; z[i] = zi; q[i] = qi;
  }
  // the error of the first failing record in file order, as a sequential read reports it
  if (first_bad < first_unknown)
    throw std::invalid_argument("Error: unsupported PQR ATOM record: " + std::string(atoms[(size_t)first_bad]));
  if (first_unknown < natoms) unknown_type();
  for (int i = 0; i < natoms; i++) {
    mass += m[i];
    Q += q[i];
  }
}

void MoleculeTarget::moveToCenterOfMass() {  // MoleculeTarget.cpp:596-620
  double r[3] = {0, 0, 0};
  for (int i = 0; i < natoms; i++) {
    r[0] += m[i] * x[i];
    r[1] += m[i] * y[i];
    r[2] += m[i] * z[i];
  }
  for (double &c : r) c /= mass;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < natoms; i++) {
    x[i] -= r[0];
    y[i] -= r[1];
    z[i] -= r[2];
  }
}

void MoleculeTarget::calculateMoleculeRadius() {  // MoleculeTarget.cpp:905-931
  double rmax = 0.0;
  int id = 0;
  for (int i = 0; i < natoms; i++) {
    const double r = std::sqrt(x[i] * x[i] + y[i] * y[i] + z[i] * z[i]);
    if (r > rmax) { id = i; rmax = r; }
  }
  radius = std::sqrt(x[id] * x[id] + y[id] * y[id] + z[id] * z[id]);
}

// MoleculeTarget::orientateMolecule (MoleculeTarget.cpp:623-698): used when
// the inertia tensor is already diagonal or its eigenvectors are degenerate.
void MoleculeTarget::orientateMolecule() {
  double rmax = 0.0, theta = 0.0;
  int id = 0;
  for (int i = 0; i < natoms; i++) {
    const double r = std::sqrt(x[i] * x[i] + y[i] * y[i] + z[i] * z[i]);
    if (r > rmax) { id = i; rmax = r; }
  }
  if ((x[id] != 0.0) & (y[id] != 0.0)) theta = std::atan2(y[id], x[id]);
  double phi = std::acos(z[id] / rmax);
  theta *= -1.0;
  for (int i = 0; i < natoms; i++) {
    const double xi = x[i], yi = y[i];
    x[i] = std::cos(theta) * xi - std::sin(theta) * yi;
    y[i] = std::sin(theta) * xi + std::cos(theta) * yi;
  }
  phi *= -1.0;
  for (int i = 0; i < natoms; i++) {
    const double xi = x[i], zi = z[i];
    x[i] = std::sin(phi) * zi + std::cos(phi) * xi;
    z[i] = std::cos(phi) * zi - std::sin(phi) * xi;
  }
  rmax = 0.0;
  for (int i = 0; i < natoms; i++) {
    const double r = std::sqrt(x[i] * x[i] + y[i] * y[i]);
    if (r > rmax) { id = i; rmax = r; }
  }
  const double gamma = -std::atan2(y[id], x[id]);
  for (int i = 0; i < natoms; i++) {
    const double xi = x[i], yi = y[i];
    x[i] = std::cos(gamma) * xi - std::sin(gamma) * yi;
    y[i] = std::sin(gamma) * xi + std::cos(gamma) * yi;
  }
}

namespace {
// closed-form roots of the characteristic cubic (MoleculeTarget.cpp:812-850)
void eigenvalues3(double A[3][3], double ev[3]) {
  double a0 = A[0][0] * A[1][1] * A[2][2] - A[0][0] * A[1][2] * A[2][1] - A[1][1] * A[0][2] * A[2][0] -
              A[2][2] * A[0][1] * A[1][0] + A[0][1] * A[1][2] * A[2][0] + A[0][2] * A[2][1] * A[1][0];
  double a1 = A[0][1] * A[1][0] + A[0][2] * A[2][0] + A[1][2] * A[2][1] - A[0][0] * A[1][1] -
              A[1][1] * A[2][2] - A[2][2] * A[0][0];
  double a2 = A[0][0] + A[1][1] + A[2][2];
  a0 = -a0; a1 = -a1; a2 = -a2;
  const double p = (3 * a1 - a2 * a2) / 3;
  const double q = (9 * a1 * a2 - 27 * a0 - 2 * a2 * a2 * a2) / 27;
  const double Qv = p / 3, Rv = q / 2, D = Qv * Qv * Qv + Rv * Rv;
  double a, b;
  if (D < 0) { a = Rv; b = std::sqrt(-D); }
  else { a = Rv + std::sqrt(D); b = 0; }
  const double phase = std::atan2(b, a);
  const double mag = std::pow(a * a + b * b, 1.0 / 6.0);
  ev[0] = -(a2 / 3) + mag * 2 * std::cos(phase / 3.0);
  ev[1] = -(a2 / 3) - mag * (std::cos(phase / 3.0) + std::sqrt(3.0) * std::sin(phase / 3.0));
  ev[2] = -(a2 / 3) - mag * (std::cos(phase / 3.0) - std::sqrt(3.0) * std::sin(phase / 3.0));
}
// eigenvectors from the first two roots; the third is their cross product
// (MoleculeTarget.cpp:852-878)
void eigenvectors3(double A[3][3], const double l[3], double V[3][3]) {
  double det = l[0] * l[0] - l[0] * A[1][1] - A[1][2] * A[1][2] - l[0] * A[2][2] + A[1][1] * A[2][2];
  double y = (l[0] * A[1][0] - A[2][2] * A[1][0] + A[1][2] * A[2][0]) / det;
  double z = (A[2][1] * A[1][0] + l[0] * A[2][0] - A[1][1] * A[2][0]) / det;
  double nf = std::sqrt(1 + y * y + z * z);
  V[0][0] = 1.0 / nf; V[0][1] = y / nf; V[0][2] = z / nf;
  det = l[1] * l[1] - l[1] * A[0][0] - A[0][2] * A[0][2] - l[1] * A[2][2] + A[0][0] * A[2][2];
  const double x = (l[1] * A[0][1] + A[0][2] * A[2][1] - A[0][1] * A[2][2]) / det;
  z = (A[0][1] * A[0][2] + (l[1] - A[0][0]) * A[2][1]) / det;
  nf = std::sqrt(1 + x * x + z * z);
  V[1][0] = x / nf; V[1][1] = 1 / nf; V[1][2] = z / nf;
  V[2][0] = V[0][1] * V[1][2] - V[0][2] * V[1][1];
  V[2][1] = V[0][2] * V[1][0] - V[0][0] * V[1][2];
  V[2][2] = V[0][0] * V[1][1] - V[0][1] * V[1][0];
}
double dot(const double *a, const double *b) {
  double r = 0.0;
  r += a[0] * b[0];
  r += a[1] * b[1];
  r += a[2] * b[2];
  return r;
}
}  // namespace

// MoleculeTarget::setInertia (MoleculeTarget.cpp:701-805)
void MoleculeTarget::setInertia() {
  for (auto &row : inertia)
    for (double &v : row) v = 0.0;
  for (int i = 0; i < natoms; i++) {
    const double r[3] = {x[i], y[i], z[i]};
    const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) inertia[a][b] += m[i] * (r2 * (a == b ? 1.0 : 0.0) - r[a] * r[b]);
  }
  auto small = [](double v) { return std::fabs(v) < 1.e-12; };
  diagonal = false;
  if (small(inertia[0][1]) && small(inertia[1][0]) && small(inertia[1][2]) && small(inertia[2][1]) &&
      small(inertia[2][0]) && small(inertia[0][2])) {
    orientateMolecule();
    diagonal = true;
  } else {
    double ev[3];
    eigenvalues3(inertia, ev);
    eigenvectors3(inertia, ev, vectors);
    double d = std::sqrt(std::pow(dot(vectors[0], vectors[1]), 2.0));
    d = std::fmax(std::sqrt(std::pow(dot(vectors[0], vectors[2]), 2.0)), d);
    d = std::fmax(std::sqrt(std::pow(dot(vectors[1], vectors[2]), 2.0)), d);
    if (d > 1e-6) {
      orientateMolecule();
    } else {
#pragma omp parallel for schedule(static)
      for (int i = 0; i < natoms; i++) {
        const double xi = x[i], yi = y[i], zi = z[i];
        x[i] = xi * vectors[0][0] + yi * vectors[0][1] + zi * vectors[0][2];
        y[i] = xi * vectors[1][0] + yi * vectors[1][1] + zi * vectors[1][2];
        z[i] = xi * vectors[2][0] + yi * vectors[2][1] + zi * vectors[2][2];
      }
    }
  }
  double mx = 0, my = 0, mz = 0;
  for (int i = 0; i < natoms; i++) {
    mx = std::fmax(mx, std::fabs(x[i]));
    my = std::fmax(my, std::fabs(y[i]));
    mz = std::fmax(mz, std::fabs(z[i]));
  }
  // longest extent on z
  if (mx > my && mx > mz) {
    for (int i = 0; i < natoms; i++) {
      const double xi = x[i];
      x[i] = -z[i];
      z[i] = xi;
    }
  } else if (my > mx && my > mz) {
    for (int i = 0; i < natoms; i++) {
      const double yi = y[i];
      y[i] = z[i];
      z[i] = -yi;
    }
  }
  maxX = maxY = maxZ = 0;  // signed coordinate of largest magnitude, as the reference keeps it
  for (int i = 0; i < natoms; i++) {
    if (std::fabs(x[i]) > std::fabs(maxX)) maxX = x[i];
    if (std::fabs(y[i]) > std::fabs(maxY)) maxY = y[i];
    if (std::fabs(z[i]) > std::fabs(maxZ)) maxZ = z[i];
  }
}

MoleculeTarget::MoleculeTarget(const std::string &file, int gas_flag, const std::string &user_ff,
                               bool user_ff_flag, int force_type)
    : gas_flag_(gas_flag), user_ff_flag_(user_ff_flag) {
  if (user_ff_flag) readUserFF(user_ff);
  else defaultFF();
  const size_t dotp = file.find_last_of('.');
  const std::string ext = dotp == std::string::npos ? "" : file.substr(dotp + 1);
  if (ext == "pqr") readPQR(file);
  else if (ext == "xyz") readXYZ(file, force_type);
  else throw std::invalid_argument("Error: only acceptable PQR or XYZ or XYZ-Q format");
  if (natoms == 0) throw std::invalid_argument("Error: the target has no atoms");
  moveToCenterOfMass();
  calculateMoleculeRadius();
  setInertia();
}

void MoleculeTarget::printFF(int gas_flag) const {  // MoleculeTarget.cpp:572-594
  std::cout << "*********************************************************" << std::endl;
  std::cout << "Force Field parameters: " << std::endl;
  std::cout << "*********************************************************" << std::endl;
  std::cout << "Symbol  mass (amu)  epsilon (kcal/mol)  sigma(Angstroms) " << std::endl;
  if (gas_flag == 3) {
    for (size_t i = 0; i < ff_name.size(); i++)
      std::cout << ff_name[i] << "-C  " << ff_m[i] << "   " << std::sqrt(ff_eps[i] * 0.055) << "   "
                << 0.5 * (ff_sig[i] + 2.757) << std::endl;
    for (size_t i = 0; i < ff_name.size(); i++)
      std::cout << ff_name[i] << "-O  " << ff_m[i] << "   " << std::sqrt(ff_eps[i] * 0.159) << "   "
                << 0.5 * (ff_sig[i] + 3.033) << std::endl;
  } else {
    for (size_t i = 0; i < ff_name.size(); i++)
      std::cout << ff_name[i] << "   " << ff_m[i] << "   " << ff_eps[i] << "   " << ff_sig[i] << std::endl;
  }
}

void MoleculeTarget::print() const {  // MoleculeTarget.cpp:887-903
  std::cout << "*********************************************************" << std::endl;
  std::cout << "MOLECULE:: orientation around the inertia principal axis " << std::endl;
  std::cout << "*********************************************************" << std::endl;
  std::cout << "Inertia matrix a.u. Ang^2: " << std::endl;
  for (const auto &row : inertia)
    std::cout << "{  " << row[0] << "  " << row[1] << "  " << row[2] << "  }" << std::endl;
  if (!diagonal) {
    std::cout << "Rotation matrix applied to molecule: " << std::endl;
    for (const auto &row : vectors)
      std::cout << "{  " << row[0] << "  " << row[1] << "  " << row[2] << "  }" << std::endl;
  }
  std::cout << "Molecule radius: " << radius << " Ang " << std::endl;
}

}  // namespace massccs
