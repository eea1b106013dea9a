/*
 * mz_oracle.h -- TEST ORACLE.  A plain-C, FP64, single-threaded restatement
 * of the reference's objective for the spline EAM/MEAM/GMEAM/JMEAM/pair styles.  It exists to
 * check the CUDA evaluator: only tests, the smoke check and the benchmark's
 * CPU-baseline leg call it.  The product never links it.
 *
 * It follows the reference loop by loop, in the reference's own order:
 *   PotMEAMSpline::fast_compute   src/pots/pot_meam_spline/pot_meam_spline.cpp:102-283
 *   PotEAMSpline::fast_compute    src/pots/pot_eam_spline/pot_eam_spline.cpp:100-223
 *   PotGMEAMSpline::fast_compute  src/pots/pot_gmeam_spline/pot_gmeam_spline.cpp:103-290
 *   PotPairSpline::fast_compute   src/pots/pot_pair_spline/pot_pair_spline.cpp:71-139
 *   PotJMEAMSpline::fast_compute  src/pots/pot_jmeam_spline/pot_jmeam_spline.cpp:103-306
 *   PotJMEAM2Spline::fast_compute src/pots/pot_jmeam2_spline/pot_jmeam2_spline.cpp
 *   Potential::accumulate_error   src/potential.cpp:415-491
 *   Spline3Eq::refresh_basis      src/spline3eq.cpp:192-225
 *   Spline3Eq::splint_comb        src/spline3eq.h:110-122, 204-236
 *   Spline5Eq::refresh_basis      src/spline5eq.cpp:209-293 (own Gaussian elimination
 *                                 with partial pivoting in place of LAPACK dgesv)
 *   Spline5Eq::splint_comb        src/spline5eq.h:110-127, 226-255
 *   Spline::get_knotshift         src/spline.cpp:74-99 (triplet cos knots)
 *   Triplet::setup_triplet        src/triplet.cpp:34-40
 *   Config::find_triplets         src/config.cpp:240-285 (all j<k pairs)
 * with forces scattered to neighbours as the reference does
 * (atom_j.force -= ...).  Its input is the neighbour list of the
 * evaluator's builder (pair order = the reference's); the reference program
 * itself, compiled by oracle/Makefile, pins both.
 */
#ifndef MZ_ORACLE_H
#define MZ_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int nknots;
  double left, right;
  int nat[2], grad_fixed[2];
  double grad[2];
  const int *y_fixed;
  const double *y;
  int quintic;      /* spline5eq (spline5eq.cpp) */
  double grad2[2];  /* spline5eq: y'' at the ends */
} mzo_spline;

typedef struct {
  int style;     /* 0 eam/spline, 1 meam/spline, 2 gmeam/spline, 3 pair/spline, 4 jmeam/spline,
                    5 jmeam2/spline */
  int ntypes;
  int nsplines;  /* group-major: phi, rho, U [, f, g] */
  const mzo_spline *splines;
  int embed_extrap;
  double energy_weight, stress_weight;
  int omit_punishments; /* leave the style punishments out (a database shard past the first) */
} mzo_pot;

typedef struct {
  int ncells, natoms;
  int64_t npairs;
  const int *cell_atom0;
  const double *cell_vol, *cell_weight, *cell_eweight, *cell_sweight, *cell_energy0, *cell_stress0;
  const int *atom_type, *atom_cell;
  const double *atom_force0;
  const int64_t *pair_off;
  const int *pair_nbr;
  const double *pair_r, *pair_u;  /* u [npairs][3] */
  const int8_t *pair_knot;        /* [npairs][nfun] phi rho f (p p2) */
  const double *pair_shift;       /* [npairs][nfun] */
  int nfun;                       /* radial functions per slot: phi, rho, f (+ p, p2) */
} mzo_db;

/* Objective of the coefficient vector `coeffs` (Potential::coeff order).
 * Outputs (nullable): errvec [esize], forces [natoms][3], energy [ncells]
 * (per atom), stress [ncells][6], dens [natoms] (unclamped densities).
 * Returns the objective (NaN propagates as in the reference). */
double mzo_objective(const mzo_db *db, const mzo_pot *pot, const double *coeffs, double *errvec,
                     double *forces, double *energy, double *stress, double *dens);

/* The objective of `coeffs` and, in *dobj, its exact derivative along the
 * direction `dir` [ncoeff] (tangent-linear restatement of mzo_objective:
 * forward-mode differentiation statement by statement, no finite
 * differences).  Returns the objective. */
double mzo_objective_tangent(const mzo_db *db, const mzo_pot *pot, const double *coeffs, const double *dir,
                             double *dobj);

/* Length of the residual vector. */
int mzo_esize(const mzo_db *db, const mzo_pot *pot);

/* Number of adjustable coefficients. */
int mzo_ncoeff(const mzo_pot *pot);

#ifdef __cplusplus
}
#endif

#endif
