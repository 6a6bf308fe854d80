/*
 * massccs_host.h -- C-ABI of the host side (libmassccs_host.so).
 *
 * The set-up and reduction that surround the GPU trajectory loop, kept in the
 * reference's form so that massccs_b200 drops in for cces-cepid/massccs:
 *   mh_open     <- System::System up to the trajectory loop (src/System.cpp:19-144):
 *                  Input (src/Input.cpp:49-263), GasBuffer (src/GasBuffer.cpp:19-192),
 *                  MoleculeTarget (src/MoleculeTarget.cpp:19-931), the geometric
 *                  ellipsoid (src/System.cpp:1640-1698) and the cell box
 *                  (src/LinkedCell.cpp:48-90)
 *   mh_predraw  <- the serial mt19937 pre-draw (src/System.cpp:184-197)
 *   mh_reduce   <- the per-iteration reduction (src/System.cpp:287-321)
 *   mh_run      <- the whole run with the report of the reference's stdout
 * The trajectory loop itself is ccs_run (include/massccs_gpu.h).
 */
#ifndef MASSCCS_HOST_H
#define MASSCCS_HOST_H

#include <stddef.h>
#include <stdint.h>

#include "massccs_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mh_system mh_system;

/* Scalars of a built system (the System members of src/System.h:57-100). */
typedef struct {
  int32_t gas_flag, force_type, natoms, gas_natoms;
  uint32_t nprobe, niter, seed, nthreads;
  int32_t short_range_cutoff, long_range_flag, long_range_cutoff, polarizability_flag;
  int32_t equipotential_flag, user_ff_flag;
  double dt, temperature, skin, lj_cutoff, coul_cutoff;
  double alpha;            /* kcal/mol units (System.cpp:117) */
  double mu, target_mass, target_charge, gas_mass, gas_inertia, d_bond;
  double a, b, c, bmax;
  double lx, ly, lz;       /* half box lengths */
  int32_t Nx, Ny, Nz, Ncells;
  double cell_size;
  double max_x, max_y, max_z, radius;
} mh_info;

/* Read input.json and build the system.  Paths inside input.json are taken
 * relative to the json file's directory.  print: echo the reference's set-up
 * report on stdout.  Returns a ccs_status; err receives a message. */
int mh_open(mh_system **out, const char *input_json, int print, char *err, size_t errlen);
void mh_close(mh_system *sys);
int mh_get_info(const mh_system *sys, mh_info *info);

/* Oriented target arrays (any pointer may be NULL). */
int mh_get_target(const mh_system *sys, double *x, double *y, double *z, double *q, double *m,
                  double *eps, double *sig, double *eps_c, double *sig_c);

/* Engine parameters for this system (gas, force type, cutoffs, ellipsoid, box). */
int mh_fill_params(const mh_system *sys, ccs_params *p);

/* The reference's pre-draw for ntraj trajectories into rnd (9 rows of ntraj). */
int mh_predraw(const mh_system *sys, uint32_t seed, size_t ntraj, double *rnd);

/* Per-iteration reduction; omega/nfree/nscatter/nlost have niter entries. */
int mh_reduce(size_t niter, size_t nprobe, const int8_t *status, const double *one_minus_cos,
              double bmax, double *omega, int32_t *nfree, int32_t *nscatter, int32_t *nlost,
              double *ccs, double *err);

/* The whole run on a device: pre-draw, ccs_run, reduction and (print) the
 * report lines of System.cpp:201-325.  ccs/err/seconds may be NULL;
 * seconds is the reference's "CCS time" span (pre-draw to reduction). */
int mh_run(mh_system *sys, int device, const ccs_params *overrides, int print, double *ccs,
           double *err, double *seconds);

/* The same run as one job split over several GPUs (no counterpart in the
 * reference, whose OpenMP loop shares one host's cores): one pre-draw,
 * contiguous slices of the trajectory numbers per GPU (one context and one
 * host thread each), the reduction in the reference's fixed order over all of
 * them.  Every trajectory keeps its random numbers, so the result equals the
 * one-GPU run's whenever the lanes per force evaluation agree: with
 * lanes_per_traj = 0 they are tuned once, on the first GPU, and used by all.
 * A GPU number may repeat (several contexts on one GPU). */
int mh_run_devices(mh_system *sys, size_t ndevices, const int *devices, const ccs_params *overrides, int print,
                   double *ccs, double *err, double *seconds);

/* The GPUs the input.json's "devices" key names (count 0: the key is absent). */
int mh_get_devices(const mh_system *sys, int *devices, size_t cap, size_t *count);

#ifdef __cplusplus
}
#endif
#endif
