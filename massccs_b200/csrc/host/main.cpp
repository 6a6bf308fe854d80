// main.cpp -- the drop-in CLI: `massccs input.json` (cces-cepid/massccs
// src/main.cpp:20-34) with the trajectory loop on the B200.
#include <algorithm>
#include <chrono>
#include <iostream>

#include "massccs_host.h"

int main(int argc, char *argv[]) {
  if (argc < 2) {
    std::cout << "Usage: " << argv[0] << " input.json" << std::endl;
    return 1;
  }
  const auto t0 = std::chrono::steady_clock::now();
  char err[512] = {0};
  mh_system *sys = nullptr;
  int rc = mh_open(&sys, argv[1], 1, err, sizeof err);
  if (rc) {
    std::cerr << "massccs: " << err << std::endl;
    return 1;
  }
  int devs[64];
  size_t nd = 0;
  mh_get_devices(sys, devs, 64, &nd);  // "devices" in input.json: one job over several GPUs
  rc = nd > 1 ? mh_run_devices(sys, std::min<size_t>(nd, 64), devs, nullptr, 1, nullptr, nullptr, nullptr)
              : mh_run(sys, nd == 1 ? devs[0] : 0, nullptr, 1, nullptr, nullptr, nullptr);
  mh_close(sys);
  if (rc) {
    std::cerr << "massccs: " << ccs_status_string(rc) << std::endl;
    return 1;
  }
  std::cout << "Total time: " << std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count()
            << " s" << std::endl;
  std::cout << "Program finished..." << std::endl;
  return 0;
}
