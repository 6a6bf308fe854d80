/*
 * massccs_gpu.h -- C-ABI of the B200 trajectory engine (libmassccs_gpu.so).
 *
 * The drop-in boundary for the reference's trajectory loop.  In the reference
 * (cces-cepid/massccs) the hot path is the body of the OpenMP loop in
 * System::System (src/System.cpp:204-285): per trajectory, System::setup
 * (src/System.cpp:1397-1518), then run_He / run_N2 / run_CO2
 * (src/System.cpp:338-1392), which call the Force::*_LC routines
 * (src/Force.cpp:34-1725) over the LinkedCell tables (src/LinkedCell.cpp:19-440).
 * The reference has no FFI of its own; these entry points are what a host that
 * keeps the reference's set-up (Input, MoleculeTarget, ellipsoid, RNG pre-draw)
 * and its reduction (src/System.cpp:287-321) binds in place of that loop.
 *
 * Conventions
 *  - Plain C types only; every function returns a ccs_status (0 = success).
 *  - The host owns every input and output array; the library copies them and
 *    owns all device memory of a context.
 *  - One host thread per context; calls on one context are serialised.
 *  - No exceptions cross the ABI; ccs_last_error() describes the last failure.
 *  - Units are the reference's: Angstrom, fs, amu, kcal/mol, e.
 */
#ifndef MASSCCS_GPU_H
#define MASSCCS_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CCS_ABI_VERSION 2

typedef enum {
  CCS_OK = 0,
  CCS_ERR_INVALID = -1,     /* bad argument or call order */
  CCS_ERR_NOMEM = -2,       /* host or device allocation failed */
  CCS_ERR_CUDA = -3,        /* CUDA runtime error (message in ccs_last_error) */
  CCS_ERR_TIMEOUT = -4,     /* the device watchdog stopped the kernel */
  CCS_ERR_NODEVICE = -5,    /* no usable CUDA device / not built for it */
  CCS_ERR_UNSUPPORTED = -6  /* a configuration this engine does not implement */
} ccs_status;

/* Buffer gases, numbered as Input.cpp:134-150 (gas_buffer_flag). */
typedef enum {
  CCS_GAS_HE = 1,   /* 1 site */
  CCS_GAS_N2 = 2,   /* 2 N + massless central charge (GasBuffer.cpp:79-115) */
  CCS_GAS_CO2 = 3,  /* O-C-O, Harris-Yung (GasBuffer.cpp:116-165) */
  CCS_GAS_AR = 4,   /* 1 site */
  CCS_GAS_CO2_1SITE = 5 /* "co2": 1 site (GasBuffer.cpp:178-190) */
} ccs_gas;

typedef enum {
  CCS_PREC_FP32 = 0, /* forces and integration in FP32; 1-cos(chi) in FP64 */
  CCS_PREC_FP64 = 1  /* everything in FP64 (the oracle-matching mode) */
} ccs_precision;

/* Trajectory status, as the reference classifies trajectories (System.cpp:217-227). */
typedef enum {
  CCS_TRAJ_FREE = 0,    /* missed the ellipsoid: counted, dOmega = 0 */
  CCS_TRAJ_SCATTER = 1, /* left the ellipsoid/box within the energy tolerance */
  CCS_TRAJ_LOST = 2,    /* ran out of retries: excluded from the denominator */
  CCS_TRAJ_CAPPED = 3   /* hit the per-try step cap (the reference would not end) */
} ccs_traj_status;

/* quirks bits */
#define CCS_QUIRK_CO2_VCM 1 /* reproduce System.cpp:1012 (vcm[0] = gasProbe->vcm[1]) */

/* Run parameters: the scalars System passes to setup/run_* and Force
 * (System.h:57-100, Force.cpp:20-26), plus engine knobs.  Fill with
 * ccs_params_default() first. */
typedef struct {
  int32_t gas;              /* ccs_gas */
  int32_t force_type;       /* 1..6, System.cpp:49-87 */
  double dt;                /* fs */
  double temperature;       /* K */
  double mu;                /* amu: reduced mass (atomic gases) or gas mass (N2, CO2) */
  double gas_inertia;       /* amu A^2, sum m z^2 of the gas sites (System.cpp:109-112) */
  double d_bond;            /* A, constrained pair distance (GasBuffer d) */
  double alpha;             /* polarizability already in kcal/mol units (System.cpp:117) */
  double lj_cutoff;         /* A */
  double coul_cutoff;       /* A */
  double skin;              /* A, the reference cell edge is lj_cutoff + skin */
  double a, b, c;           /* ellipsoid semi-axes, A */
  double bmax;              /* maximal impact parameter, A */
  double lx, ly, lz;        /* half box lengths (System.cpp:142-144), A */
  int32_t precision;        /* ccs_precision */
  int32_t quirks;           /* CCS_QUIRK_* bits */
  double cell_size;         /* engine cell edge in A; 0 = automatic */
  int32_t lanes_per_traj;   /* 0 = autotuned, else 1, 4, 8, 16 or 32 lanes per force evaluation */
  int32_t block_size;       /* 0 = automatic (multiple of 32) */
  uint32_t max_steps_per_try; /* 0 = 2,000,000 */
  double watchdog_s;        /* kernel wall-time budget, 0 = 600 s */
  int32_t schedule;         /* 0 = index order, 1 = longest expected trajectories first,
                               2 = index order, and a trajectory past park_steps moves to the
                               warp pass only once every trajectory has been taken (which ones
                               move then depends on timing: FP32 results can differ between runs
                               at rounding level, the two passes summing forces in different
                               orders) */
  uint32_t park_steps;      /* steps after which a trajectory moves to the warp pass; 0 = 2048 */
  int32_t resume_block;     /* threads per trajectory in the warp pass: 32, 64 or 128; 0 = 32 for
                               N2/CO2 in FP32 on targets whose candidate lists fit 2048 entries,
                               else 64 */
  int32_t spec_tries;       /* failed tries after which a warp-pass trajectory runs its remaining
                               tries at once (2..8); 0 = default, < 0 = never */
} ccs_params;

/* Per-run statistics. */
typedef struct {
  uint64_t ntraj, nfree, nscatter, nlost, ncapped;
  uint64_t steps;           /* integration steps, all tries */
  uint64_t visits;          /* site x atom pairs the engine evaluated */
  uint64_t parked;          /* trajectories finished by the warp pass (the long ones) */
  double kernel_ms;         /* device time of both trajectory passes (CUDA events) */
  double h2d_ms, d2h_ms;    /* copy times of ccs_run (CUDA events) */
  int32_t lanes_per_traj, block_size, grid_size;
  int32_t speculated;       /* warp-pass trajectories whose remaining tries ran at once */
  double lane_ms, warp_ms;  /* the lane pass and the warp pass separately */
} ccs_stats;

typedef struct ccs_ctx ccs_ctx;

/* Library version and the ABI it implements. */
int ccs_version(int32_t *abi_version);

/* Create a context on a CUDA device (replaces the per-trajectory `new Force` /
 * `new GasBuffer` of System.cpp:211-213 with one long-lived device context). */
int ccs_create(ccs_ctx **out, int device);
void ccs_destroy(ccs_ctx *ctx);

/* Defaults for every field of ccs_params (He, force_type 4, reference defaults). */
void ccs_params_default(ccs_params *p);

/* Target atoms (MoleculeTarget arrays, MoleculeTarget.h:74-92, in the
 * reference's oriented frame).  eps/sig are the pair parameters for the
 * probe's LJ sites exactly as MoleculeTarget::assignedParameter produces them
 * (MoleculeTarget.cpp:540-570); eps_c/sig_c the CO2 carbon-site parameters
 * (NULL unless gas = CO2).  The library builds its own cell grid from them
 * (LinkedCell.cpp:19-440 is the reference counterpart).  Call ccs_set_params
 * first: the grid depends on the cutoffs and force type. */
int ccs_set_target(ccs_ctx *ctx, size_t natoms, const double *x, const double *y, const double *z,
                   const double *q, const double *eps, const double *sig, const double *eps_c,
                   const double *sig_c);

/* Scalar parameters (System.cpp:19-144 results).  Resets the target grid. */
int ccs_set_params(ccs_ctx *ctx, const ccs_params *p);

/* Run ntraj trajectories (System.cpp:204-285).  rnd[k] are the reference's
 * pre-drawn arrays rnd_vec1..9 (System.cpp:184-197): rnd[0] = sqrt(bmax^2 u1),
 * rnd[1..4] = u2..u5, rnd[5..8] = u6..u9 (only read for N2/CO2, may be NULL
 * otherwise).  Outputs (host arrays of ntraj; steps/visits may be NULL):
 * status (ccs_traj_status), one_minus_cos = 1 - cos(chi) for scatter else 0,
 * steps = integration steps over all tries, visits = engine pair visits.
 * Synchronous. */
int ccs_run(ccs_ctx *ctx, size_t ntraj, const double *const rnd[9], int8_t *status,
            double *one_minus_cos, uint32_t *steps, uint32_t *visits, ccs_stats *stats);

/* Many ions in one launch of each pass (batched ions of uneven size).  No
 * counterpart in the reference, which runs one ion per process: a caller with
 * several ions replaces their separate System::System runs
 * (src/System.cpp:146-321) by one call.  ions[i] is a context set up for ion
 * i (ccs_set_params + ccs_set_target), all on one device, with one precision,
 * and all atomic or all molecular gases; ntraj[i] its trajectory count.
 * rnd[k] holds row k of every ion's pre-draw back to back (ion 0 first), and
 * status / one_minus_cos / steps / visits are laid out the same way.  The
 * first context's stream, scratch and statistics carry the run; lanes per
 * force evaluation are its lanes_per_traj (8, 16 or 32), else autotuned on a
 * sub-batch of every ion's first trajectories.  Synchronous. */
int ccs_run_batch(ccs_ctx *const *ions, size_t nions, const size_t *ntraj, const double *const rnd[9],
                  int8_t *status, double *one_minus_cos, uint32_t *steps, uint32_t *visits,
                  ccs_stats *stats);

/* Same on device buffers, asynchronous on `stream` (a cudaStream_t, NULL =
 * the context's stream): the host does not wait for the GPU (the watchdog
 * deadline is set on the device; the first run of a context with lanes_per_traj
 * = 0 waits once for its autotuning).  d_rnd holds 9 rows of `stride` doubles.
 * Statistics are accumulated on the device and read back by ccs_sync_stats,
 * which waits for the run and returns CCS_ERR_TIMEOUT if the watchdog
 * stopped it. */
int ccs_run_device(ccs_ctx *ctx, size_t ntraj, const double *d_rnd, size_t stride,
                   int8_t *d_status, double *d_one_minus_cos, uint32_t *d_steps,
                   uint32_t *d_visits, void *stream);
int ccs_sync_stats(ccs_ctx *ctx, ccs_stats *stats);

/* ccs_run_device without any device allocation.  No counterpart in the
 * reference (whose CPU loop allocates per trajectory): it is for callers that
 * cannot allocate device memory while they run -- a host whose allocator owns
 * the whole device heap, a service with a memory budget fixed at start-up, or
 * code where an allocation would synchronise the device.  The run's scratch
 * (work counter, statistics, watchdog deadline, launch-parameter copy, park
 * buffer of long trajectories) is a 40 MiB static device array that every GPU
 * loading the library holds until exit; inputs and outputs are the caller's
 * device buffers, as for ccs_run_device, and the results are the same bit for
 * bit (the park buffer has ccs_run_device's capacity at every allowed size).
 *  - at most 262144 trajectories per call (CCS_ERR_INVALID beyond that);
 *  - the first call on a device looks up the array's device address; make it
 *    before any stream capture;
 *  - the array is shared by every call on a device and keeps the last call's
 *    contents: calls whose work overlaps on the GPU (other streams, other
 *    threads, other contexts on the same device) race, so serialise them;
 *  - lanes per force evaluation: the configured value, else the one the
 *    context already tuned, else 32 (no autotuning run);
 *  - stats == NULL: the call returns without waiting for the GPU; a later
 *    ccs_sync_stats(ctx) waits for the run, fills the statistics from the
 *    array and returns CCS_ERR_TIMEOUT if the watchdog stopped it (before
 *    another call on the same device reuses the array);
 *  - stats given: the call waits for the run, fills stats and returns
 *    CCS_ERR_TIMEOUT if the watchdog stopped it. */
int ccs_run_device_noalloc(ccs_ctx *ctx, size_t ntraj, const double *d_rnd, size_t stride,
                           int8_t *d_status, double *d_one_minus_cos, uint32_t *d_steps,
                           uint32_t *d_visits, void *stream, ccs_stats *stats);

/* Force on gas site `site` at npts positions (pos: npts x 3), as the
 * reference's per-site dispatch picks the routine (System.cpp:371-379,
 * 594-637, 1028-1065 -> Force.cpp).  Same device code as the trajectory
 * kernel.  Outputs: f (npts x 3), U (npts), visits (npts, may be NULL). */
int ccs_eval_site_forces(ccs_ctx *ctx, size_t npts, int site, const double *pos, double *f,
                         double *U, uint32_t *visits);

/* Initial conditions of System::setup (System.cpp:1397-1518) for ntraj
 * trajectories: hit flags and site positions/velocities (ntraj x 3 sites x 3). */
int ccs_eval_setup(ccs_ctx *ctx, size_t ntraj, const double *const rnd[9], int8_t *hit,
                   double *pos, double *vel);

/* Engine description after ccs_set_target: grid and reach actually used. */
typedef struct {
  int32_t nx, ny, nz, natoms;
  double cell_size, reach;
  double origin[3];
  int32_t charged, allpairs, max_cell_atoms, vel_table_len;
  int32_t sm_count, reserved;
} ccs_info;
int ccs_get_info(ccs_ctx *ctx, ccs_info *info);

/* Measurement helper with no counterpart in the reference: the device's
 * sustained FP32 FMA throughput (TFLOP/s, 2 flops per FMA), measured by an
 * FMA-chain kernel over all SMs for about `ms` milliseconds.  The trajectory
 * kernels are bound by the FP32 pipe, so this is their roofline denominator. */
int ccs_measure_fp32_peak(int device, double ms, double *tflops);

/* ---- Learned field ---------------------------------------------------------
 * No counterpart in the reference, which evaluates every force of every step
 * with the linked-cell sums (src/Force.cpp:34-1725); the learned field
 * replaces most of those sums.  Range separation: every pair term is split
 * by a smooth switch S(r) (1 below r_in, 0 above r_out) into a near part,
 * summed exactly over the atoms within r_out, and a far part, which is smooth
 * in the site position and is learned.  Per context (target + gas): a
 * 16-level hash-grid encoding of the site position (2 features per level,
 * smoothstep blending) feeding an MLP 32 -> 64 -> 64 -> nf fields: the far
 * potential of each gas site type and, with the induced dipole, the three
 * far-field components; far forces and the far field's Jacobian are minus the
 * fields' gradients.  It is trained on the GPU (ccs_field_train: samples
 * labelled by the engine's own cell grid and tables, the project's
 * forward/backward and Adam kernels) and evaluated in the lane pass by
 * tcgen05 BF16 tensor-core MMAs with FP32 accumulation.  A position is
 * evaluated fully exactly when it lies within fallback_radius of an atom,
 * outside the field's domain, or in a voxel whose validation error exceeds
 * err_threshold.  FP32 precision, force types 2, 4 and 6. */
typedef struct {
  int64_t samples;          /* training samples (default 4,000,000) */
  int32_t iterations;       /* Adam steps (default 6000) */
  int32_t batch;            /* samples per step (default 32768) */
  int32_t log2_table;       /* rows per level = 2^log2_table (default 20, at most 22) */
  int32_t base_res;         /* coarsest grid resolution over the domain (default 8) */
  int32_t finest_res;       /* finest grid resolution (default 128) */
  int32_t validation;       /* validation samples for the error voxels (default 1,048,576) */
  double fallback_radius;   /* A: exact evaluation within this distance of any atom (default 2.0:
                               the pair terms within r_out are always exact, so contact forces
                               are; this zone only keeps the network off the unreachable core) */
  double voxel;             /* A: edge of the exact-evaluation bitmap's voxels (default 0.5) */
  double err_voxel;         /* A: edge of the validation-error voxels (default 2.0) */
  double err_threshold;     /* force error |G - G*| / g of a field (g: the RMS of its gradient
                               labels) above which a validation voxel is evaluated exactly; 0 (the
                               default) flags none.  A probe crossing into an exact voxel sees the
                               learned far part's error as a jump in its potential energy, which
                               the energy test (0.5 % of the collision energy) can reject */
  double near_fraction;     /* share of samples drawn in the shell around atoms (default 0.5) */
  double near_shell;        /* A: that shell's thickness beyond fallback_radius (default 6.0) */
  double lr;                /* Adam learning rate, decayed tenfold over the run (default 1e-2) */
  double lam_u, u0, f0;     /* loss per field: lam_u (u-U*)^2/(U*^2+(u0 s)^2) + |G-G*|^2/(|G*|^2+(f0 g)^2),
                               s and g the RMS of the field's values and gradients
                               (defaults 0.1, 0.05, 0.05) */
  uint64_t seed;            /* sampling, initialisation and batch order (default 2104) */
  double r_in, r_out;       /* A: the range-separation switch (defaults 6 and 12) */
} ccs_field_params;

typedef struct {
  double domain_lo[3], domain_side;   /* the field's domain cube, A */
  int32_t levels, dense_levels, nfields, log2_table;
  int32_t res[16];                    /* grid resolution per level */
  int64_t samples;                    /* training samples drawn */
  double output_scale[5];             /* per field: values are s_f * (network output) */
  double gradient_scale[5];           /* per field: RMS of the gradient labels */
  double sample_ms, label_ms, train_ms, validate_ms;
  double first_loss, final_loss;      /* mean training loss of the first and last steps */
  double val_force_rel_rms;           /* validation: RMS over samples of the largest
                                         |G - G*| / g of the fields */
  double val_force_rel_p99;
  double val_u_rel_rms;               /* RMS of the largest |u - U*| / s of the fields */
  double exact_fraction;              /* share of the domain's voxels evaluated exactly */
  int64_t err_voxels;                 /* validation voxels above err_threshold */
} ccs_field_report;

void ccs_field_params_default(ccs_field_params *p);

/* Sample, label, train and validate the learned field of the context's
 * current target and parameters (call after ccs_set_target; a later
 * ccs_set_params or ccs_set_target discards it).  Synchronous.  Does not
 * switch it on: see ccs_field_enable.  report may be NULL. */
int ccs_field_train(ccs_ctx *ctx, const ccs_field_params *p, ccs_field_report *report);

/* Runs of this context use the learned field (on = 1) or exact forces only
 * (on = 0, the default).  CCS_ERR_INVALID if no field is trained. */
int ccs_field_enable(ccs_ctx *ctx, int on);

/* Inference of the fields gas site `site` uses (its far potential; at the
 * dipole's site also the three far-field components: nfields = 1 or 4) at
 * npts positions (pos: npts x 3): u (npts x 4: the values, nfields used),
 * g (npts x 4 x 3: minus each field's gradient -- for a potential the far
 * force), exact[i] = 1 where the trajectory kernels evaluate that position
 * fully exactly (the field's values are still returned).  path 0: the
 * tensor-core kernel of the lane pass (128 positions per CTA); path 1: the
 * warp kernel of the warp pass.  exact and nfields may be NULL. */
int ccs_field_eval(ccs_ctx *ctx, size_t npts, int site, const double *pos, int path, double *u, double *g,
                   int8_t *exact, int32_t *nfields);

/* Test hooks of the training kernels (the checker compares them with its
 * own restatement).  Parameters in FP32: table [16][2^log2_table][2], mlp =
 * W1 [64][32], b1 [64], W2 [64][64], b2 [64], W3 [nf][64], b3 [nf];
 * scales: nf output scales, then nf gradient scales (the loss floors).
 * ccs_field_setup prepares a context's field geometry without training
 * (domain, grids, exact-evaluation bitmap) with random parameters;
 * ccs_field_get/set_weights read or replace the parameters (set also
 * refreshes the inference copies); ccs_field_loss_grad runs the training
 * forward/backward on n given samples (pos n x 3, labels n x nf x 4: U, Fx,
 * Fy, Fz: a potential's force, i.e. minus the gradient) and returns the mean
 * loss and its gradients. */
int ccs_field_setup(ccs_ctx *ctx, const ccs_field_params *p, ccs_field_report *report);
int ccs_field_get_weights(ccs_ctx *ctx, float *table, float *mlp, double *scales);
int ccs_field_set_weights(ccs_ctx *ctx, const float *table, const float *mlp, const double *scales);
int ccs_field_loss_grad(ccs_ctx *ctx, size_t n, const float *pos, const float *labels, double *loss,
                        float *dtable, float *dmlp);
/* The training labels at n positions: every field's far part and minus its
 * gradient, labels n x nf x 4 (the engine's cell grid and FP32 tables). */
int ccs_field_labels(ccs_ctx *ctx, size_t n, const double *pos, double *labels);

/* The equipotential ellipsoid's boundary points on the GPU
 * (src/Equipotential.cpp:86-200 with the all-atom potentials of :203-557):
 * the z-extent march from (0, 0, |max_z| + 20) in 0.5 A steps, then
 * max(25, ceil(zmax)) + 1 z-levels of 20 rays towards the z-axis in 0.1 A
 * steps; each step's potential is an FP64 sum over all atoms (one CTA per
 * ray, fixed-order reduction).  Threshold ek in kcal/mol; alpha in kcal/mol
 * units; eps/sig as for ccs_set_target (eps_c/sig_c for CO2).  Writes every
 * ray's crossing point (0, 0, 0: none) in (level, rotation) order into pts
 * (cap rows of 3) and their count into npts (CCS_ERR_INVALID with npts set
 * when cap is too small); zmax receives the widened z extent (x 1.3).  The
 * least-squares fit is the caller's (the host library does it). */
int ccs_equipotential_points(int device, size_t natoms, const double *x, const double *y, const double *z,
                             const double *q, const double *eps, const double *sig, const double *eps_c,
                             const double *sig_c, int gas, int polar, double alpha, double ek, double max_x,
                             double max_y, double max_z, size_t cap, double *pts, size_t *npts, double *zmax);

/* Human-readable strings. */
const char *ccs_status_string(int status);
const char *ccs_last_error(ccs_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif
