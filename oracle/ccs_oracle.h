/*
 * ccs_oracle.h -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * A plain-C, FP64 restatement of the reference's trajectory-method CCS path
 * (cces-cepid/massccs).  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg may load it.  Every function cites the reference file:line
 * it restates.  Beyond the reference it exposes per-trajectory outputs
 * (status, 1-cos(chi), steps, atom visits) so the GPU engine can be checked
 * trajectory by trajectory on identical initial conditions.
 *
 * Parity is pinned by replaying the reference's shipped logs (ccs_He.log,
 * ccs_Ar.log, ccs.out, ccs_N2.log) and by comparison against the reference
 * binary built from its own sources into oracle/_ref/.
 */
#ifndef CCS_ORACLE_H
#define CCS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_system orc_system;

/* Scalar state of a built system (System.h:57-100 members after System.cpp:19-144). */
typedef struct {
  int gas_flag;            /* He=1 N2=2 CO2=3 Ar=4 co2=5 (Input.cpp:134-150) */
  int force_type;          /* 1..6, System.cpp:49-87 */
  int natoms;              /* target atoms */
  int gas_natoms;          /* probe sites */
  unsigned nprobe, niter, seed, nthreads;
  int short_range_cutoff, long_range_flag, long_range_cutoff, polarizability_flag;
  int equipotential_flag, user_ff_flag;
  double dt, temperature, skin, lj_cutoff, coul_cutoff;
  double alpha;            /* already multiplied by ALPHA_TO_KCAL_MOL (System.cpp:117) */
  double mu, target_mass, target_charge, gas_mass, gas_inertia, d_bond;
  double a, b, c, bmax;    /* ellipsoid semi-axes and maximal impact parameter */
  double lx, ly, lz;       /* half box lengths (System.cpp:142-144) */
  int Nx, Ny, Nz, Ncells;
  double cell_size;        /* lj_cutoff + skin */
  double max_x, max_y, max_z, radius;
} orc_params;

/* Build the full set-up of System::System (System.cpp:19-144) from an input.json.
 * print: 0 silent, 1 echo the reference's set-up report to stdout.
 * Returns NULL and fills err on failure. */
orc_system *orc_open(const char *json_path, int print, char *err, int errlen);
void orc_close(orc_system *s);
void orc_get_params(const orc_system *s, orc_params *p);

/* Target arrays in the reference's final order (oriented, then sorted by cell:
 * LinkedCell.cpp:132-225).  Any pointer may be NULL.  eps_c/sig_c are only
 * meaningful for CO2. */
void orc_get_target(const orc_system *s, double *x, double *y, double *z, double *q,
                    double *m, double *eps, double *sig, double *eps_c, double *sig_c);

/* The serial mt19937 pre-draw (System.cpp:184-197) for ntraj trajectories.
 * rnd is 9*ntraj doubles laid out as rnd[k*ntraj + j]; row 0 already holds
 * sqrt(bmax^2 u) as the reference stores it.  Rows 5..8 stay 0 for atomic gases. */
void orc_predraw(const orc_system *s, unsigned seed, size_t ntraj, double *rnd);

/* First n outputs of std::mt19937(seed) (RandomNumber.cpp:19-29), raw 32-bit. */
void orc_mt19937(unsigned seed, size_t n, uint32_t *out);

/* quirks bit 0: reproduce the reference's CO2 reference-velocity bug
 * (System.cpp:1012, vcm[0] = gasProbe->vcm[1]).  Without it the fixed vcm[0]. */
#define ORC_QUIRK_CO2_VCM 1

/* Run trajectories j in [0,n) (the body of System.cpp:204-285) with nthreads
 * OpenMP threads (0 = all).  rnd as in orc_predraw with row stride `stride`.
 * Outputs (any may be NULL): status 0 free / 1 scatter / 2 lost,
 * one_minus_cos = 1 - cos(chi) for scatter else 0, steps = integration steps
 * over all tries, visits = target-atom visits summed over every stencil cell
 * the force routines walked (the work unit of the performance model). */
void orc_run(const orc_system *s, size_t n, const double *rnd, size_t stride, int quirks,
             int nthreads, int8_t *status, double *one_minus_cos, uint32_t *steps,
             uint64_t *visits);

/* Initial conditions only (System::setup, System.cpp:1397-1518) for one
 * trajectory: writes site positions/velocities (3 sites x 3, row-major),
 * rcm, vcm, returns hit (1) or free (0). */
int orc_setup_one(const orc_system *s, const double rnd9[9], double pos[9], double vel[9],
                  double rcm[3], double vcm[3]);

/* Speed sampler (System::velGenerator, System.cpp:1537-1555) for one uniform. */
double orc_vel_generator(const orc_system *s, double u);

/* Force on probe site iatom at position pos as the reference's dispatch picks it
 * (System.cpp:371-379, 594-637, 1028-1065).  Returns 0, or -1 for a bad site. */
int orc_site_force(const orc_system *s, int iatom, const double pos[3], double f[3],
                   double *U, uint64_t *visits);

/* Per-iteration reduction and CCS estimate (System.cpp:287-321). */
void orc_reduce(size_t niter, size_t nprobe, const int8_t *status, const double *one_minus_cos,
                double bmax, double *omega, int *nfree, int *nscatter, int *nlost,
                double *ccs, double *err);

/* Whole reference run: pre-draw, trajectories, reduction and the report lines
 * of System.cpp:201-325 (print=1). ccs/err may be NULL. */
int orc_run_system(orc_system *s, int nthreads, int quirks, int print, double *ccs, double *err);

#ifdef __cplusplus
}
#endif
#endif
