// Host-side model of the potential and the configuration database.
//
// These are the B200 evaluator's own data structures; the arithmetic that
// fixes parity with the reference (knot grid, knot/shift bisection, second
// derivative refresh, periodic image search) is restated here from the
// reference files cited at each function.  Compile this code with
// -ffp-contract=off: the neighbour distances and shifts must round exactly
// as the reference's do, so that the lists are identical.
#pragma once

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "mz_b200.h"

namespace mzb {

// Second derivatives (and, for the quintic basis, fourth derivatives) that a
// spline carries between refreshes.  The reference's rescale evaluates splines
// whose y was scaled after their last refresh, so these travel separately.
struct SplineDerivs {
  std::vector<double> ypp, yp4;
};

struct Spline3 {
  // Definition read from the file (spline3eq.cpp:54-106; spline5eq.cpp:57-115
  // for the quintic basis, whose ends also carry y'').
  double left = 0, right = 0;
  int nknots = 0;
  int quintic = 0;             // spline5eq
  int nat[2] = {0, 0};         // natural end (bc -1)
  int grad_fixed[2] = {1, 1};  // end slope fixed (bc 1) ; bc 0 -> free
  double grad[2] = {0, 0};
  double grad2[2] = {0, 0};    // spline5eq: y'' at the ends
  std::vector<int> y_fixed;
  std::vector<double> y;
  // Knot grid exactly as Spline3Eq::set_spline (spline3eq.cpp:354-370).
  double step = 0, invstep = 0;
  std::vector<double> x;

  void set_grid();
  int ncoeff() const;
  // Bisection knot + shift (Spline::get_knotshift, spline.cpp:74-99); -1 if
  // r lies beyond the last knot by more than the reference's 1e-8 slack.
  int knotshift(double r, double *shift) const;
  // Second derivatives (Spline3Eq::refresh_basis, spline3eq.cpp:192-225).
  void refresh(std::vector<double> &ypp) const;
  // Value + slope at x with linear extrapolation (spline3eq.h:204-236).
  double eval(const std::vector<double> &ypp, double xv, double *g) const;
  // spline5eq: y'' and y'''' from the 2n x 2n system of
  // Spline5Eq::refresh_basis (spline5eq.cpp:209-293), solved by Gaussian
  // elimination with partial pivoting.
  void refresh5(std::vector<double> &ypp, std::vector<double> &yp4) const;
  // Either basis: refresh, value + slope (+ y'') at x (spline5eq.h:205-291
  // for the quintic, quadratic beyond the ends).
  void refresh_any(SplineDerivs &d) const;
  double eval_any(const SplineDerivs &d, double xv, double *g) const;
  double eval_grad2_any(const SplineDerivs &d, double xv) const;

  // Operations of the reference's rescale (spline3eq.cpp:112-186, 301-350):
  // new end knots with values re-interpolated, x scaled (reversed when the
  // factor is negative), y scaled, a spline added (values / slopes of `rhs`
  // evaluated with the second derivatives `rhs_ypp` it carries), a*x added.
  void readjust_x(double left, double right);
  void rescale_x(double scale);
  void scale_y(double f);
  void divide_y(double f);
  void add(const Spline3 &rhs, const SplineDerivs &rhs_d);
  void add_linear(double a);
  double max_y_mag() const;  // Spline::get_max_y_mag (spline.cpp:58-67)
};

// Function groups in file order.  MEAM: phi(Pair_ij) rho(Pair_j) U(Atom/Pair_i)
// f(Pair_ij) g(Triplet_i) (pot_meam.cpp:31-47, pot_eam.cpp:30-46,
// pot_pair.cpp:25-37).  EAM: the first three.
// JMEAM adds p (Pair_ij, radial) and q (Triplet_i) after g, JMEAM2 a second
// pair p2, q2 (pot_jmeam.cpp:31-45, pot_jmeam2.cpp:31-45).
enum Group { G_PHI = 0, G_RHO = 1, G_U = 2, G_F = 3, G_G = 4, G_P1 = 5, G_Q1 = 6, G_P2 = 7, G_Q2 = 8 };

// MEAM and GMEAM share the skeleton (three-body f f g); GMEAM indexes g by
// the types of i and of the pair j, k (Triplet_i_jk, pot_fns.cpp:166-168) and
// punishes every f spline (pot_gmeam_spline.cpp:173-178).
inline bool style_meam(int style) {
  return style == MZ_STYLE_MEAM_SPLINE || style == MZ_STYLE_GMEAM_SPLINE || style == MZ_STYLE_JMEAM_SPLINE ||
         style == MZ_STYLE_JMEAM2_SPLINE;
}
// Direct three-body energy terms sum_{j<k} p_ij p_ik q_i(cos) of the JMEAM
// styles (PotJMEAMSpline::fast_compute, pot_jmeam_spline.cpp:208-219):
// jmeam/spline one (p, q), jmeam2/spline two.
inline int style_nj(int style) {
  return style == MZ_STYLE_JMEAM_SPLINE ? 1 : style == MZ_STYLE_JMEAM2_SPLINE ? 2 : 0;
}
// pair/spline (PotPair, pot_pair.cpp:25-37; PotPairSpline::fast_compute,
// pot_pair_spline.cpp:71-139): phi only, each pair once (dbl_cnt_pair_ = 0,
// config.cpp:181-185), no embedding, no constraint or punishment entries.
inline bool style_pair(int style) { return style == MZ_STYLE_PAIR_SPLINE; }
// Entries after the per-cell constraints: MEAM 1, GMEAM one per f spline, EAM one per type.
inline int style_npen(int style, int ntypes) {
  return style_nj(style) > 0              ? 1 + style_nj(style)  // f-max, then p-max per (p, q)
         : style == MZ_STYLE_MEAM_SPLINE  ? 1
         : style == MZ_STYLE_GMEAM_SPLINE ? ntypes * (ntypes + 1) / 2
         : style == MZ_STYLE_PAIR_SPLINE  ? 0
                                          : ntypes;
}
// ErrorVec length: per cell E, 6 S, 3 F per atom (potential.cpp:423-444), the
// per-cell density constraints of the embedding styles, the punishments.
inline int style_esize(int style, int ntypes, int ncells, int natoms) {
  return 7 * ncells + 3 * natoms + (style_pair(style) ? 0 : ncells) + style_npen(style, ntypes);
}

struct Pot {
  int style = MZ_STYLE_MEAM_SPLINE;
  int ntypes = 1;
  std::string comment, type_name;
  int ngroups = 5;
  std::vector<std::vector<Spline3>> groups;  // [group][alloy index]

  // Flattened spline list (group-major) and the coefficient layout.
  int nsplines() const;
  const Spline3 &spline(int s) const;
  Spline3 &spline(int s);
  int spline_index(int group, int alloy) const;
  int ncoeff() const;
  void get_coeffs(double *out) const;
  void set_coeffs(const double *in);
  // The coefficient order as (spline, slot): slot k < n is knot y[k], n + e
  // the end slope grad[e], n + 2 + e the quintic y''[e].  Potential::coeff
  // walks free knots, then per free end its slope (and for spline5eq its
  // y'', Spline5Eq::bc_coeff spline5eq.cpp:459-468), while get_ncoeff counts
  // one per free end (spline5eq.cpp:81-85); the first ncoeff() of the walk
  // are the coefficients.
  std::vector<std::pair<int, int>> coeff_slots() const;
  double max_rcut() const;  // Potential::get_max_rcut (potential.cpp:72-82), radial groups

  // alloy indices (pot_fns.cpp:240-296)
  int idx_pair_ij(int ti, int tj) const {
    return (ti <= tj) ? ti * ntypes + tj - (ti * (ti + 1)) / 2 : tj * ntypes + ti - (tj * (tj + 1)) / 2;
  }
};

// Configuration database in CSR / structure-of-arrays form, atoms in
// configuration order.  Each atom's neighbour row is the reference's pair
// list for that atom in the same order (config.cpp:186-228).
struct Db {
  int style = -1;  // potential style the lists were built for (pair/spline: each pair once)
  int nfun = 3;    // radial functions per pair in pair_knot / pair_shift: phi, rho, f (+ p, p2)
  int ncells = 0, natoms = 0;
  int64_t npairs = 0, ntriplets = 0;
  int max_row = 0;
  // cells
  std::vector<int> cell_atom0;     // [ncells+1]
  std::vector<double> cell_vol, cell_weight, cell_eweight, cell_sweight, cell_energy0;
  std::vector<double> cell_stress0;  // [6*ncells]
  std::vector<double> cell_lattice;  // [9*ncells]
  // atoms
  std::vector<int> atom_type, atom_cell;
  std::vector<double> atom_pos, atom_force0;  // [3N]
  std::vector<int64_t> pair_off;              // [N+1]
  // pairs
  std::vector<int> pair_nbr;                  // neighbour atom index
  std::vector<double> pair_r, pair_u;         // r, unit vector [3Np]
  std::vector<int8_t> pair_knot;              // [Np][nfun] phi, rho, f (f: MEAM only), p, p2 (JMEAM)
  std::vector<double> pair_shift;             // [Np][nfun]
  // incoming lists: for every atom, the pair slots whose neighbour it is
  std::vector<int64_t> in_off;                // [N+1]
  std::vector<int64_t> in_slot;               // [Np]
};

// Potential::rescale for the spline styles (PotMEAM::rescale
// pot_meam.cpp:281-375 with rescale_3body :497-525; PotEAM::rescale
// pot_eam.cpp:257-389) from per-atom densities of the current potential.
// Returns 1 when the potential changed; factors = {embedding a, MEAM f b}.
int rescale_pot(Pot &pot, const int *atom_type, int natoms, const double *densities, int flag, double factors[2]);

// Potential::write_data's text files (potential.cpp:325-342 and the writers it calls).
void write_data_files(const Db &db, const Pot &pot, double energy_weight, double stress_weight, const double *errvec,
                      const double *energy, const double *stress, const double *forces, const double *densities,
                      const std::string &prefix, int num);

// Build lists (throws std::runtime_error with an mz status prefix).
void build_db(const mz_cells_desc &cells, const Pot &pot, Db &db);
// The same lists from the GPU (mz_nbr.cu); identical arrays.
void build_db_device(const mz_cells_desc &cells, const Pot &pot, Db &db, int device);
// Pieces shared by both builders: cells / atoms / validation, the periodic
// image range of one cell (false when the cell is too small), the incoming
// lists, and the reference's error texts.
void build_db_setup(const mz_cells_desc &cells, const Pot &pot, Db &db);
bool cell_scale(const double *lattice9, double max_rcut, double *vol, int s[3]);
void build_incoming(Db &db);
std::string cell_too_small_msg(int ci);
std::string pair_too_short_msg(const Pot &pot, int q, double rr, int ti, int tj, int ci, int i, int j);
void parse_pot(const std::string &text, Pot &pot);
std::string write_pot_text(const Pot &pot);
void read_config_file(const std::string &path, int ntypes, std::vector<int> &cell_natoms,
                      std::vector<double> &lattice, std::vector<double> &e0,
                      std::vector<double> &s0, std::vector<double> &w, std::vector<double> &ew,
                      std::vector<double> &sw, std::vector<int> &types, std::vector<double> &pos,
                      std::vector<double> &f0);

struct Failure {
  int status;
  std::string msg;
};

void set_error(const std::string &msg);

}  // namespace mzb

// Opaque handles of the C ABI.
struct mz_pot {
  mzb::Pot pot;
};
struct mz_db {
  mzb::Db db;
};
