// input.cpp -- input.json reader (cces-cepid/massccs src/Input.cpp:49-263).
// A small reader for the flat JSON object the reference accepts; the
// reference uses rapidjson for the same keys and defaults.
#include <cctype>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <algorithm>
#include <map>
#include <sstream>
#include <thread>

#include "setup.h"

namespace massccs {
namespace {

struct JsonValue {
  std::string text;
  bool is_string = false;
};

std::map<std::string, JsonValue> parse_flat_json(const std::string &src) {
  std::map<std::string, JsonValue> out;
  size_t p = 0;
  auto skip = [&]() {
    while (p < src.size() && std::isspace((unsigned char)src[p])) p++;
  };
  skip();
  if (p >= src.size() || src[p] != '{') throw std::invalid_argument("input.json: not a JSON object");
  p++;
  for (;;) {
    skip();
    while (p < src.size() && src[p] == ',') { p++; skip(); }
    if (p >= src.size()) throw std::invalid_argument("input.json: unterminated object");
    if (src[p] == '}') break;
    if (src[p] != '"') throw std::invalid_argument("input.json: expected a key");
    size_t e = src.find('"', p + 1);
    if (e == std::string::npos) throw std::invalid_argument("input.json: bad key");
    std::string key = src.substr(p + 1, e - p - 1);
    p = e + 1;
    skip();
    if (p >= src.size() || src[p] != ':') throw std::invalid_argument("input.json: expected ':'");
    p++;
    skip();
    JsonValue v;
    if (p < src.size() && src[p] == '"') {
      e = src.find('"', p + 1);
      if (e == std::string::npos) throw std::invalid_argument("input.json: unterminated string");
      v.text = src.substr(p + 1, e - p - 1);
      v.is_string = true;
      p = e + 1;
    } else {
      size_t s = p;
      while (p < src.size() && src[p] != ',' && src[p] != '}' && !std::isspace((unsigned char)src[p])) p++;
      v.text = src.substr(s, p - s);
    }
    out[key] = v;
  }
  return out;
}

double number(const JsonValue &v, const std::string &key) {
  if (v.is_string) throw std::invalid_argument("Error input.json: " + key + " format error");
  size_t used = 0;
  double d = std::stod(v.text, &used);
  if (used != v.text.size()) throw std::invalid_argument("Error input.json: " + key + " format error");
  return d;
}

unsigned unsigned_number(const JsonValue &v, const std::string &key) {
  const double d = number(v, key);
  if (d < 0 || d != (double)(unsigned)d) throw std::invalid_argument("Error input.json: " + key + " format error");
  return (unsigned)d;
}

}  // namespace

Input::Input(const std::string &path) {
  std::ifstream f(path);
  if (!f) throw std::invalid_argument("cannot open " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  auto d = parse_flat_json(ss.str());
  auto has = [&](const char *k) { return d.count(k) != 0; };
  if (!has("targetFileName") || !d["targetFileName"].is_string)
    throw std::invalid_argument("Error input.json: targetFileName not found");
  targetFilename = d["targetFileName"].text;
  nProbe = has("numberProbe") ? unsigned_number(d["numberProbe"], "numberProbe") : 10000;
  nIter = has("nIter") ? unsigned_number(d["nIter"], "nIter") : 10;
  seed = has("seed") ? unsigned_number(d["seed"], "seed") : 20162104u;
  nthreads = has("nthreads") ? unsigned_number(d["nthreads"], "nthreads") : std::max(1u, std::thread::hardware_concurrency());
  dt = has("dt") ? number(d["dt"], "dt") : 10.0;
  temperatureTarget = has("Temp") ? number(d["Temp"], "Temp") : 298.0;
  skin = has("skin") ? number(d["skin"], "skin") : 0.01;
  if (has("GasBuffer")) {
    gas_str = d["GasBuffer"].text;
    if (gas_str == "He") gas_buffer_flag = 1;
    else if (gas_str == "N2") gas_buffer_flag = 2;
    else if (gas_str == "CO2") gas_buffer_flag = 3;
    else if (gas_str == "Ar") gas_buffer_flag = 4;
    else if (gas_str == "co2") gas_buffer_flag = 5;
    else throw std::invalid_argument("only available the follow gas buffer types: He Ar N2 CO2");
  }
  auto yesno = [&](const char *key, std::string &str, int &flag, const char *def, int defflag) {
    if (has(key)) {
      str = d[key].text;
      if (str == "yes") flag = 1;
      else if (str == "no") flag = 0;
      else throw std::invalid_argument(std::string("need to choice ") + key + ": yes or no");
    } else {
      str = def;
      flag = defflag;
    }
  };
  yesno("Equipotential", equip_str, equipotential_flag, "no", 0);
  yesno("Short-range cutoff", short_str, short_range_cutoff, "yes", 1);
  lj_cutoff = has("LJ-cutoff") ? number(d["LJ-cutoff"], "LJ-cutoff") : 12.0;
  yesno("Long-range forces", long_str, long_range_flag, "no", 0);
  yesno("Long-range cutoff", long_cut_str, long_range_cutoff, "yes", 1);
  coul_cutoff = has("Coul-cutoff") ? number(d["Coul-cutoff"], "Coul-cutoff") : 25.0;
  if (gas_buffer_flag == 1) yesno("polarizability", polar_str, polarizability_flag, "yes", 1);
  else yesno("polarizability", polar_str, polarizability_flag, "no", 0);
  if (has("alpha")) {
    alpha = number(d["alpha"], "alpha");
  } else if (polarizability_flag == 1) {  // Constants.h:79-83
    static const double tab[6] = {0.0, 0.204956, 1.710, 2.911, 1.6411, 2.911};
    alpha = tab[gas_buffer_flag];
  }
  if (has("force-field")) {
    user_ff = d["force-field"].text;
    user_ff_flag = 1;
  }
  if (has("ref_quirks")) ref_quirks = d["ref_quirks"].text == "yes";
  if (has("precision")) {
    precision = d["precision"].text;
    if (precision != "fp32" && precision != "fp64")
      throw std::invalid_argument("precision must be fp32 or fp64");
  }
  if (has("fp64_check")) fp64_check = unsigned_number(d["fp64_check"], "fp64_check");
  if (has("setup_device")) {
    setup_device = d["setup_device"].text;
    if (setup_device != "cpu" && setup_device != "gpu" && setup_device != "auto")
      throw std::invalid_argument("setup_device must be cpu, gpu or auto");
  }
  if (has("devices")) {  // one job split over several GPUs: a count, or a comma-separated list of GPU numbers
    const std::string &t = d["devices"].text;
    devices.clear();
    if (t.find(',') == std::string::npos) {
      const unsigned nd = unsigned_number(d["devices"], "devices");
      for (unsigned k = 0; k < nd; k++) devices.push_back((int)k);
    } else {
      size_t s = 0;
      while (s <= t.size()) {
        const size_t e = std::min(t.find(',', s), t.size());
        const std::string item = t.substr(s, e - s);
        size_t used = 0;
        int v = -1;
        try { v = std::stoi(item, &used); } catch (const std::exception &) { used = 0; }
        if (used == 0 || used != item.size() || v < 0) throw std::invalid_argument("Error input.json: devices format error");
        devices.push_back(v);
        s = e + 1;
      }
    }
    if (devices.empty()) throw std::invalid_argument("Error input.json: devices must name at least one GPU");
  }
}

void Input::print() const {
  std::cout << "*********************************************************" << std::endl;
  std::cout << "INPUT:: Simulation Parameters " << std::endl;
  std::cout << "*********************************************************" << std::endl;
  std::cout << "target filename                  : " << targetFilename << std::endl;
  std::cout << "number of probe                  : " << nProbe << std::endl;
  std::cout << "number of iterarions             : " << nIter << std::endl;
  std::cout << "number of threads                : " << nthreads << std::endl;
  std::cout << "seed number                      : " << seed << std::endl;
  std::cout << "gas buffer                       : " << gas_str << std::endl;
  std::cout << "Target Temperature (K)           : " << temperatureTarget << std::endl;
  std::cout << "timestep (fs)                    : " << dt << std::endl;
  std::cout << "Skin cell size (Ang)             : " << skin << std::endl;
  std::cout << "Equipotential                    : " << equip_str << std::endl;
  std::cout << "Cut short-range interaction      : " << short_str << std::endl;
  if (short_range_cutoff == 1) std::cout << "LJ cutoff (Ang)                  : " << lj_cutoff << std::endl;
  std::cout << "Apply long-range interaction     : " << long_str << std::endl;
  std::cout << "Cut long-range interaction       : " << long_cut_str << std::endl;
  if (long_range_cutoff == 1) std::cout << "Coulomb cutoff (Ang)             : " << coul_cutoff << std::endl;
  std::cout << "Apply induced-dipole interaction : " << polar_str << std::endl;
  if (polarizability_flag == 1) std::cout << "alpha (Ang^3)                    : " << alpha << std::endl;
  if (user_ff_flag == 1) std::cout << "force-field                      : " << user_ff << std::endl;
}

}  // namespace massccs
