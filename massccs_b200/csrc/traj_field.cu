// traj_field.cu -- the trajectory kernels with the learned field (their SURR
// instantiations), compiled apart from ccs_engine.cu so the two build in
// parallel.  The kernels themselves are in ccs_device.cuh; the launches in
// ccs_engine.cu pick these when a context's field is on.
#include <cuda_runtime.h>

#include "engine_ctx.h"

using namespace ccs;

namespace {
template <int GAS, bool HASQ> ccs_internal::KernelFn traj_g(int G) {
  switch (G) {
    case 1: return traj_kernel<float, 1, GAS, HASQ, false, true>;
    case 8: return traj_kernel<float, 8, GAS, HASQ, false, true>;
    case 16: return traj_kernel<float, 16, GAS, HASQ, false, true>;
    default: return traj_kernel<float, 32, GAS, HASQ, false, true>;
  }
}
template <int GAS, bool HASQ> ccs_internal::KernelFn resume_nt(int nt) {
  return nt == 32 ? resume_kernel<float, GAS, HASQ, 32, false, true>
                  : nt == 128 ? resume_kernel<float, GAS, HASQ, 128, false, true>
                              : resume_kernel<float, GAS, HASQ, 64, false, true>;
}
}  // namespace

ccs_internal::KernelFn ccs_internal::pick_traj_field(int gas, bool hasq, int G) {
  if (G == 4) G = 8;  // no 4-lane instantiation with the field
  if (gas == GAS_ATOM) return hasq ? traj_g<GAS_ATOM, true>(G) : traj_g<GAS_ATOM, false>(G);
  if (gas == GAS_N2) return hasq ? traj_g<GAS_N2, true>(G) : traj_g<GAS_N2, false>(G);
  return hasq ? traj_g<GAS_CO2, true>(G) : traj_g<GAS_CO2, false>(G);
}

ccs_internal::KernelFn ccs_internal::pick_resume_field(int gas, bool hasq, int nt) {
  if (gas == GAS_ATOM) return hasq ? resume_nt<GAS_ATOM, true>(nt) : resume_nt<GAS_ATOM, false>(nt);
  if (gas == GAS_N2) return hasq ? resume_nt<GAS_N2, true>(nt) : resume_nt<GAS_N2, false>(nt);
  return hasq ? resume_nt<GAS_CO2, true>(nt) : resume_nt<GAS_CO2, false>(nt);
}
