/*
 * mz_b200.h -- C ABI of the B200 evaluator for the spline EAM/MEAM fitting
 * objective.
 *
 * The reference program evaluates its objective through the polymorphic C++
 * class Potential (src/potential.h:35-109).  Every optimizer (Powell,
 * simulated annealing, genetic algorithm) calls
 *     double Potential::compute(const Comm&, ErrorVec* = nullptr)   potential.h:67
 * which, for the spline styles, runs PotMEAMSpline::fast_compute<Spline3Eq>
 * (src/pots/pot_meam_spline/pot_meam_spline.cpp:102-283) or
 * PotEAMSpline::fast_compute<Spline3Eq>
 * (src/pots/pot_eam_spline/pot_eam_spline.cpp:100-223).
 *
 * This header is the drop-in boundary for that call.  It carries plain
 * pointers and sizes only.  No C++ exception crosses it: every function
 * returns an mz_status (0 = success) and mz_last_error() returns the message
 * of the last failure on the calling thread.  Host buffers are owned by the
 * caller; the evaluator context owns its device memory, stream and graphs.
 * One context may be used by one host thread at a time.
 *
 * File formats are the reference's own (potential file pot_list.cpp:101-142
 * and spline3eq.cpp:54-106, configuration file cell.cpp:39-136), and the
 * parameter vector layout is the reference's Potential::coeff order
 * (potential.cpp:192-206 -> pot_fns.cpp:209-218 -> spline.cpp:105-114 ->
 * spline3eq.cpp:376-382): for each function group in file order, for each
 * alloy spline, the free knot values in ascending knot order, then the free
 * end slopes (left, right).
 */
#ifndef MZ_B200_H
#define MZ_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int mz_status;

enum {
  MZ_OK = 0,
  MZ_ERR_ARG = 1,          /* bad argument (null pointer, size mismatch)          */
  MZ_ERR_IO = 2,           /* file cannot be opened                              */
  MZ_ERR_FORMAT = 3,       /* malformed potential / configuration file           */
  MZ_ERR_RANGE = 4,        /* pair closer than a spline's first knot, cell too    */
                           /* small, or a neighbour row beyond the kernel limit   */
  MZ_ERR_UNSUPPORTED = 5,  /* potential style / basis not implemented            */
  MZ_ERR_CUDA = 6,         /* CUDA runtime error (message has the CUDA text)      */
  MZ_ERR_NOMEM = 7,        /* host or device allocation failed                   */
  MZ_ERR_TIMEOUT = 8       /* a bounded device wait gave up                      */
};

/* arithmetic of an evaluation */
enum {
  MZ_FP64 = 0,   /* everything in FP64 (reference parity path)                    */
  MZ_MIXED = 1   /* FP32 spline and triplet arithmetic, FP64 per-atom densities,  */
                 /* energies, virials, residuals and gradient sums                */
};

/* potential styles (the #T string of the potential file) */
enum {
  MZ_STYLE_EAM_SPLINE = 0,
  MZ_STYLE_MEAM_SPLINE = 1,
  MZ_STYLE_GMEAM_SPLINE = 2,
  MZ_STYLE_PAIR_SPLINE = 3,
  MZ_STYLE_JMEAM_SPLINE = 4,   /* MEAM + sum p_ij p_ik q(cos) in the energy             */
  MZ_STYLE_JMEAM2_SPLINE = 5   /* MEAM + two such terms (p, q) and (p2, q2)             */
};

typedef struct mz_pot mz_pot;  /* a potential: splines + parameter layout        */
typedef struct mz_db mz_db;    /* configuration database + neighbour lists       */
typedef struct mz_ctx mz_ctx;  /* device-resident evaluator                      */

/* Message of the last failed call on this thread ("" if none). */
const char *mz_last_error(void);

/* ---------------------------------------------------------------- potential */

/* Read a potential file (first #P block).  Replaces PotList::init
 * (src/pot_list.cpp:84-177) + Potential::read_pot (potential.cpp:153-161)
 * for the eam/spline, meam/spline, gmeam/spline, jmeam/spline, jmeam2/spline and
 * pair/spline styles with spline3eq bases. */
mz_status mz_pot_read(const char *path, mz_pot **out);
/* Same from the file's text held in memory. */
mz_status mz_pot_parse(const char *text, mz_pot **out);
void mz_pot_free(mz_pot *pot);
/* An independent copy of a potential (Potential::clone, src/potential.h:43). */
mz_status mz_pot_clone(const mz_pot *pot, mz_pot **out);
/* Style (MZ_STYLE_*), number of atom types, number of splines. */
mz_status mz_pot_info(const mz_pot *pot, int *style, int *ntypes, int *nsplines);
/* Number of adjustable coefficients: Potential::get_ncoeff (potential.h:59). */
mz_status mz_pot_ncoeff(const mz_pot *pot, int *ncoeff);
/* Read / write all coefficients in Potential::coeff(i) order (potential.h:60). */
mz_status mz_pot_get_coeffs(const mz_pot *pot, double *coeffs);
mz_status mz_pot_set_coeffs(mz_pot *pot, const double *coeffs);
/* Write the potential in the reference format (Potential::write_pot,
 * potential.cpp:299-319; Spline3Eq::write_basis_fn, spline3eq.cpp:248-273). */
mz_status mz_pot_write(const mz_pot *pot, const char *path);
/* Evaluate spline s of the potential at x: value and slope.  Mirrors
 * Spline3Eq::splint_comb(double, double*) (spline3eq.h:204-236), linear
 * extrapolation outside the knots (spline5eq: spline5eq.h:226-255, quadratic
 * outside).  Host-side, for tests and tools. */
mz_status mz_pot_spline_eval(const mz_pot *pot, int spline, double x, double *val, double *grad);

/* Potential::rescale (src/potential.h:68) for the spline styles, in place:
 * PotMEAM::rescale (pot_meam.cpp:281-375, with rescale_3body :497-525) or
 * PotEAM::rescale (pot_eam.cpp:257-389, with the U'(mid) = 0 gauge).  The
 * per-atom densities of the potential's current coefficients (mz_densities)
 * and the database's atom types drive it; flag as the reference's (< 0
 * never, 0 when needed, 1 always).  *rescaled = the reference's return value;
 * factors[4]: embedding scale a, MEAM f scale b, JMEAM p and p2 scales
 * (0 where unused).
 * U's knot grid changes, so evaluators must be re-created afterwards.
 * pair/spline never rescales (Potential::rescale, potential.cpp:258-261). */
mz_status mz_pot_rescale(mz_pot *pot, const mz_db *db, const double *densities, int flag, int *rescaled,
                         double *factors);

/* Potential::write_data (src/potential.cpp:325-342): the .rho, .energy,
 * .stress, .force, .error and .punish files of one evaluated potential
 * (<prefix>.<ext>, or <prefix>.<ext>.<num> when num >= 0), formatted as the
 * reference writes them, from the outputs of one FP64 mz_objective call
 * (errvec, per-cell energy per atom and stress, forces) and mz_densities.
 * pair/spline writes no .rho and no .punish file; densities may be NULL. */
mz_status mz_write_data(const mz_db *db, const mz_pot *pot, double energy_weight, double stress_weight,
                        const double *errvec, const double *energy, const double *stress, const double *forces,
                        const double *densities, const char *prefix, int num);

/* ----------------------------------------------------------------- database */

/* Cells given as arrays (all host memory, copied).  Atoms are in cell order.
 * Replaces the parsed result of Cell::read_cell (src/cell.cpp:39-136). */
typedef struct {
  int ncells;
  int natoms;
  const int *cell_natoms;      /* [ncells]                                   */
  const double *cell_lattice;  /* [ncells][3][3] rows = #X #Y #Z vectors    */
  const double *cell_energy0;  /* [ncells] target energy per atom (#E)      */
  const double *cell_stress0;  /* [ncells][6] xx yy zz xy yz zx (#S)        */
  const double *cell_weight;   /* [ncells] (#W, default 1)  nullable        */
  const double *cell_eweight;  /* [ncells] (#EW, default 1) nullable        */
  const double *cell_sweight;  /* [ncells] (#SW, default 1) nullable        */
  const int *atom_type;        /* [natoms]                                   */
  const double *atom_pos;      /* [natoms][3]                                */
  const double *atom_force0;   /* [natoms][3] target forces                  */
} mz_cells_desc;

/* Build the database and its neighbour lists for a potential.  Replaces
 * Config::init (config.cpp:46-119): Cell::find_scale (cell.cpp:158-170),
 * Config::find_pairs (config.cpp:143-234, full double-counted list), the
 * per-pair knot/shift set-up of check_pair (pair_meam_spline.cpp:50-99,
 * pair_eam_spline.cpp:50-86) and, for MEAM, find_triplets
 * (config.cpp:240-285) whose triplets are enumerated implicitly as the j<k
 * pairs of each atom's row.  Fails with MZ_ERR_RANGE where the reference
 * throws (pair shorter than a spline's first knot). */
mz_status mz_db_build(const mz_cells_desc *cells, const mz_pot *pot, mz_db **out);
/* Read a configuration file (#N/#X/#Y/#Z/#E/#S/#W/#EW/#SW/#F) and build. */
mz_status mz_db_read(const char *config_path, const mz_pot *pot, mz_db **out);
/* The same two, with the periodic-image pair search and knot / shift set-up
 * run on GPU `device` (one thread per atom, the host builder's loop order and
 * rounding): the resulting database is identical, array for array, to
 * mz_db_build's, and the same errors are reported. */
mz_status mz_db_build_device(const mz_cells_desc *cells, const mz_pot *pot, int device, mz_db **out);
mz_status mz_db_read_device(const char *config_path, const mz_pot *pot, int device, mz_db **out);
void mz_db_free(mz_db *db);

typedef struct {
  int ncells;
  int natoms;
  int64_t npairs;       /* entries of the full neighbour list (pair/spline: */
                        /* each pair once, config.cpp:181-185)            */
  int64_t ntriplets;    /* j<k pairs of every row (= reference triplets)  */
  int max_row;          /* longest neighbour row                          */
  int esize;            /* residual entries of the cells: 8 ncells + 3    */
                        /* natoms, 7 ncells + 3 natoms for pair/spline    */
                        /* (the style penalties add 1 for MEAM, ntypes    */
                        /* for EAM, one per f spline for GMEAM, 2 / 3 for */
                        /* JMEAM / JMEAM2)                                */
} mz_db_stats;
mz_status mz_db_info(const mz_db *db, mz_db_stats *stats);

/* Read-only view of the built database (pointers into the mz_db, valid
 * until mz_db_free).  Pair data of atom i occupy slots
 * [pair_off[i], pair_off[i+1]) in the reference's pair order; pair_knot and
 * pair_shift hold nfun values per slot -- phi, rho, f (+ p for jmeam/spline,
 * + p, p2 for jmeam2/spline) -- knot -1 where the reference's is -1 (f unused
 * for EAM, rho and f for pair/spline).  in_off/in_slot list, per atom, the
 * slots whose neighbour it is. */
typedef struct {
  int ncells, natoms;
  int64_t npairs;
  const int *cell_atom0;  /* [ncells+1] */
  const double *cell_vol, *cell_weight, *cell_eweight, *cell_sweight, *cell_energy0;
  const double *cell_stress0;  /* [ncells][6] */
  const double *cell_lattice;  /* [ncells][9] */
  const int *atom_type, *atom_cell;
  const double *atom_pos, *atom_force0;  /* [natoms][3] */
  const int64_t *pair_off;               /* [natoms+1] */
  const int *pair_nbr;
  const double *pair_r, *pair_u;         /* u: [npairs][3] */
  const int8_t *pair_knot;               /* [npairs][nfun] */
  const double *pair_shift;              /* [npairs][nfun] */
  const int64_t *in_off, *in_slot;
  int nfun;                              /* radial functions per slot: 3, 4 or 5 */
} mz_db_view;
mz_status mz_db_get_view(const mz_db *db, mz_db_view *view);

/* One spline of a potential as read (group-major order: phi..., rho...,
 * U..., f..., g...).  Pointers valid until the potential changes. */
typedef struct {
  int group, alloy, nknots;
  double left, right;
  int nat[2];         /* natural end (bc -1)       */
  int grad_fixed[2];  /* end slope fixed (bc 1)    */
  double grad[2];
  const int *y_fixed;
  const double *y;
  const double *x;    /* knot positions [nknots] (rescale moves them)  */
  double step;        /* knot spacing                                   */
  int quintic;        /* spline5eq basis (spline5eq.cpp)                */
  double grad2[2];    /* spline5eq: y'' at the ends                      */
} mz_spline_view;
mz_status mz_pot_get_spline(const mz_pot *pot, int spline, mz_spline_view *view);

/* Replace the targets (energy per atom, stress, forces) of every cell. */
mz_status mz_db_set_targets(mz_db *db, const double *energy0, const double *stress0,
                            const double *force0);

/* ---------------------------------------------------------------- evaluator */

typedef struct {
  double energy_weight;   /* param key energy_weight (config.cpp:50), default 0 */
  double stress_weight;   /* param key stress_weight (config.cpp:51), default 0 */
  int embed_extrap;       /* param key embed_extrap (pot_eam.cpp:71), default 0 */
  int device;             /* CUDA device ordinal                               */
  int max_candidates;     /* largest ncand per call (sizes device buffers)     */
  int omit_punishments;   /* nonzero: leave out the style punishment entries   */
                          /* (f-max for MEAM, U'(mid) for EAM; their ErrorVec */
                          /* entries read 0) -- for all but one shard of a    */
                          /* database split over several evaluators           */
} mz_settings;

/* Copy the database and the potential's fixed structure to the device. */
mz_status mz_create(const mz_db *db, const mz_pot *pot, const mz_settings *settings, mz_ctx **out);
void mz_destroy(mz_ctx *ctx);

/* Objective of ncand parameter vectors (params[ncand][ncoeff], host).
 * obj[ncand] receives the weighted sum of squares that Potential::compute
 * returns.  Optional outputs (nullable, host):
 *   errvec [ncand][esize]     the ErrorVec, layout of accumulate_error
 *                             (potential.cpp:415-491) + the style penalty
 *                             entries (pot_meam_spline.cpp:274-278 or
 *                             pot_eam_spline.cpp:211-218; none for
 *                             pair/spline)
 *   forces [ncand][natoms][3] per-atom forces in configuration order
 *   energy [ncand][ncells]    energy per atom of each cell
 *   stress [ncand][ncells][6] stress of each cell (xx yy zz xy yz zx)
 * precision is MZ_FP64 or MZ_MIXED. */
mz_status mz_objective(mz_ctx *ctx, int ncand, const double *params, int precision, double *obj,
                       double *errvec, double *forces, double *energy, double *stress);

/* Objective and its gradient with respect to every coefficient
 * (grad[ncand][ncoeff]), by a hand-written adjoint pass.  The reference has
 * no gradient; its optimizers take forward differences of compute()
 * (opt_powell.cpp:348-389). */
mz_status mz_objective_grad(mz_ctx *ctx, int ncand, const double *params, int precision,
                            double *obj, double *grad);

/* Embedding densities of every atom for one parameter vector (dens[natoms],
 * configuration order).  Mirrors fast_compute_densities
 * (pot_meam_spline.cpp:289-349, pot_eam_spline.cpp:229-268). */
mz_status mz_densities(mz_ctx *ctx, const double *params, double *dens);

/* Same as mz_objective with device pointers (params, obj, errvec, forces on
 * the device; any output may be null) enqueued on the context's stream; the
 * call returns before the work completes.  mz_sync waits for it. */
mz_status mz_objective_device(mz_ctx *ctx, int ncand, const double *d_params, int precision,
                              double *d_obj, double *d_errvec, double *d_forces);
mz_status mz_objective_grad_device(mz_ctx *ctx, int ncand, const double *d_params, int precision,
                                   double *d_obj, double *d_grad);
mz_status mz_sync(mz_ctx *ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that time or order
 * work against it. */
void *mz_stream(mz_ctx *ctx);

/* Products of two row sets over a long shared axis, FP64, on the device:
 *   out[i][j] = sum over k < n of A[i][k] * B[j][k]   (i < na, j < nb)
 * with row i of A at d_a + i * lda and row j of B at d_b + j * ldb (device
 * pointers, lda and ldb >= n), out[na][nb] on the device.  Enqueued on the
 * context's stream like mz_objective_device.  With the residual vectors'
 * derivatives as the rows of A this gives Powell's linear system
 * gamma^T gamma (A == B) and its right-hand side gamma^T e (B = the ErrorVec,
 * nb = 1) (OptPowell::lineqsys_init / lineqsys_update,
 * opt_powell.cpp:438-493, which sum k in one sequential host loop).  Sums
 * run in a fixed order: bit-reproducible on a device for given shapes; when
 * d_a == d_b with the same stride and count, out is exactly symmetric.  The
 * first call of a larger shape grows a context-owned workspace.  No
 * reference counterpart as an entry point. */
mz_status mz_gram_device(mz_ctx *ctx, int na, const double *d_a, int64_t lda, int nb, const double *d_b,
                         int64_t ldb, int64_t n, double *d_out);

/* Counters since mz_create: kernel launches issued by this context. */
mz_status mz_launch_count(const mz_ctx *ctx, int64_t *launches);

/* Which mixed-precision MEAM forward the context runs: 1 = the tensor-core
 * (tcgen05, TF32 split) triplet sums, opted into with the environment variable
 * MZ_TC=1 when the context is created; 0 = the CUDA-core one-pass forward.
 * No reference counterpart. */
mz_status mz_tensor_core_forward(const mz_ctx *ctx, int *on);

/* Launch variants chosen by the context's autotuner (no reference
 * counterpart).  The first objective call of a precision, with or without
 * the gradient, times on the caller's own candidates the forward kernel at
 * three atom-block sizes (blocks of at most 256, 192 or 128 pair slots, a
 * quarter as many atoms) and, for the gradient, the adjoint at the same three
 * sizes and two persistent-grid sizes, and keeps the fastest for the
 * context's lifetime (contexts of the same workload in one process share the
 * choice).  For meam/spline in mixed precision the forward and the adjoint
 * are also timed with two candidates per CTA (the triplet geometry shared,
 * both candidates' arithmetic as packed FP32 pairs).  The environment variable MZ_TUNE=0 at
 * mz_create keeps the first variant of each, MZ_TUNE=2 the first with two
 * candidates per CTA where that applies.  Block sizes leave the results
 * unchanged; two candidates per CTA change the order of FP32 additions
 * inside chunks of 8 partners, and the gradient's table sums follow the block
 * partition, so those may differ in the last bits between variants.
 * choice[5] = {forward slots per block, adjoint slots per block, adjoint
 * CTAs, forward candidates per CTA, adjoint candidates per CTA}, zeros
 * before the first call. */
mz_status mz_tuning(mz_ctx *ctx, int precision, int grad, int *choice);

/* Kernels of the evaluator, for per-kernel timing. */
enum {
  MZ_K_PREP = 0,    /* coefficients -> knot and evaluation tables          */
  MZ_K_ATOMS,       /* densities, embedding, per-slot reaction vectors      */
  MZ_K_GATHER,      /* per-atom forces, force residuals                     */
  MZ_K_CELLS,       /* per-cell energy, stress, residual entries            */
  MZ_K_FINAL,       /* sum of squares + punishments                         */
  MZ_K_ADJ,         /* adjoint pass over the neighbour rows                 */
  MZ_K_GRAD_FINAL,  /* table gradient -> coefficient gradient               */
  /* mixed-precision meam/spline over triplet moments (the "FM" path):       */
  MZ_K_FM_COEF,     /* candidates' B-spline coefficients and their products */
  MZ_K_FM_FWD,      /* contraction of the moments: G, Y1, Y2 per slot       */
  MZ_K_FM_EPI,      /* densities, embedding, reaction vectors               */
  MZ_K_FM_PRE,      /* adjoint weights, pair-function and U gradients       */
  MZ_K_FM_ADJ,      /* transposed contraction: moment-space gradient        */
  MZ_K_FM_GRAD,     /* moment-space and B-spline gradients -> knot table    */
  MZ_NKERNELS
};
const char *mz_kernel_name(int kernel);
/* With on != 0 the context brackets every kernel it launches with CUDA
 * events on its own stream.  mz_kernel_times waits for the stream, adds the
 * elapsed times of the launches recorded since the last call to ms[kernel]
 * and their count to launches[kernel] (arrays of MZ_NKERNELS, zeroed by the
 * caller), and forgets them. */
mz_status mz_profile(mz_ctx *ctx, int on);
/* 1 when the tuned launches of (precision, grad) use the triplet-moment
 * path for mixed-precision meam/spline (the candidates' triplet sums as
 * contractions of per-slot moments built once per database: MZ_K_FM_*), 2
 * when they do and its forward contraction runs on the tensor cores in
 * integers (tcgen05 kind::i8 over four 8-bit digits of each operand, exact
 * 32-bit sums), 3 when its adjoint contraction does too (MZ_FM8ADJ=0 keeps
 * that one on the CUDA cores), 0 when they use the row kernels.  MZ_FM=0 in the
 * environment at mz_create keeps the row kernels, MZ_FM=2 always takes the
 * moment path where it applies, the default lets the tuner time both;
 * MZ_FM8=0 keeps the moment path's forward on the CUDA cores (the default
 * uses the tensor cores where the digits fit in device memory).  No
 * reference counterpart. */
mz_status mz_moment_path(const mz_ctx *ctx, int precision, int grad, int *on);
mz_status mz_kernel_times(mz_ctx *ctx, double *ms, int64_t *launches);

/* Objective of one coefficient vector without allocating any device memory.
 *
 * This entry point has no counterpart in the reference.  It exists for
 * callers that cannot call cudaMalloc: code running where the device
 * allocator is off limits (inside another framework's memory pool or
 * allocator hooks, in processes with a fixed device-memory budget, or on a
 * path that must not add allocations).  Instead
 * of the context's buffers it uses one file-scope device array of
 * MZ_NOALLOC_SCRATCH_BYTES (64 MiB) that every GPU loading the library holds
 * until exit; the database, the potential's tables and all per-slot and
 * per-atom scratch are staged there.  Databases that do not fit are rejected
 * with MZ_ERR_RANGE (roughly up to 1e5 atoms / 2e5 pairs).
 *
 * Inputs and outputs are host memory: params[ncoeff] in, obj (the value
 * Potential::compute returns) and, if non-null, forces[natoms][3] out.  FP64,
 * on the device named by settings->device (checked against the device count
 * first; the caller's current device is restored on return).  Every call is
 * synchronous: it copies with cudaMemcpy and launches on the legacy default
 * stream, which synchronises with all blocking streams, so no call may run
 * while a stream capture is in progress in any thread.  The first call on a
 * device also looks up the array's device address (once per device).  Every
 * call reuses the same array and leaves the last call's contents in it, so
 * calls that overlap on the GPU (from several host threads) race: serialise
 * them. */
#define MZ_NOALLOC_SCRATCH_BYTES (64u << 20)
mz_status mz_objective_noalloc(const mz_db *db, const mz_pot *pot, const mz_settings *settings,
                               const double *params, double *obj, double *forces);

/* Measured CUDA-core throughput of the device (dependent-free FMA streams in
 * FP64 or FP32, MZ_FP64 / MZ_MIXED), in TFLOP/s (2 flops per FMA). */
mz_status mz_alu_peak(int device, int precision, double *tflops);

#ifdef __cplusplus
}
#endif

#endif /* MZ_B200_H */
