// Device-side data layout and shared helpers of the evaluator.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mzb {

constexpr int MAX_SPLINES = 64;     // splines in one potential (8 types MEAM: 36+8+8+36+8)
constexpr int BLOCK_SLOTS = 256;    // pair slots (threads) of one atom block
constexpr int BLOCK_ATOMS = 64;     // atoms of one atom block
constexpr int MAX_G_KNOTS = 16;     // g spline knots the adjoint's per-thread tables hold
constexpr int ADJ_WARPS = BLOCK_SLOTS / 32;

// Geometry of one spline, shared by every candidate (knot positions never
// change: Potential::check_if_similar, pot_list.cpp:165-174).
struct SplineGeom {
  double x0, xN, step, invstep;
  double cut;   // xN * (1 + 1e-8): knot == -1 beyond it (spline.cpp:79)
  float cutf;   // the same cut for FP32 cosines, widened by 4 FP32 ulps
  int n;        // knots
  int toff;     // offset of this spline in a candidate's table
  int moff;     // offset of its refresh matrix d(ypp)/d(y, grad) [n][n+2]
                // (spline5eq: d(ypp, y'''')/d(y, grad, y''_end) [2n][n+4])
  int poff;     // offset of its per-interval polynomial coefficients [n-1][4] (spline5eq [n-1][6]),
                // a multiple of 4
  int q5;       // spline5eq (quintic pieces)
};

// A candidate's table, per spline at toff: y[n], ypp[n], grad[2], and for
// spline5eq also yp4[n] (y''''), grad2[2] (y'' at the ends) (total tab_stride
// doubles per candidate).  Its evaluation table, per spline at poff: for each
// knot interval k the polynomial in the shift b,
//   S = c0 + b (c1 + b (c2 + b c3)),   dS/dr = (c1 + b (2 c2 + 3 b c3)) / h,
// (quintic: six coefficients, the same Horner form) (pow_stride doubles per
// candidate), computed in FP64 from y, ypp (and yp4).

struct DevDb {
  int ncells, natoms, nblocks;
  int64_t npairs;
  // cells
  const int *cell_atom0;          // [ncells+1]
  const double *cell_vol, *cell_w, *cell_ew, *cell_sw, *cell_e0, *cell_s0;
  // atoms
  const int *atom_type, *atom_cell;
  const double *force0;           // [3N]
  const int *pair_off;            // [N+1]
  const int *in_off, *in_slot;    // incoming lists
  // pairs
  const int *pair_nbr;
  const double *pair_r, *pair_ux, *pair_uy, *pair_uz;
  const double *pair_shift;       // [nfun][Np] phi, rho, f (+ p, p2 for JMEAM)
  const int *pair_knot;           // packed: (phi+1) | (rho+1) << 8 | (f+1) << 16 | (p+1) << 24
  const signed char *pair_knot_p2;  // JMEAM2: knot of p2 (-1: none), else null
  const float *pair_rf, *pair_uxf, *pair_uyf, *pair_uzf, *pair_shiftf;  // FP32 copies
  // atom blocks
  const int *blk_atom0;           // [nblocks+1]
  // atom blocks of the adjoint: atoms grouped by type (adj_atoms, a
  // permutation), each block of one type, <= BLOCK_SLOTS slots and
  // <= BLOCK_ATOMS atoms; block b holds adj_atoms[adj_blk0[b] .. adj_blk0[b+1])
  int adj_nblocks;
  const int *adj_atoms;
  const int *adj_blk0;
  // descriptor of adjoint block b at adj_desc[adj_blk0[b] + b + a], a = 0..na:
  // (atom, first slot in the block, na | type << 8, cell) for a < na, and
  // (0, slot count, na | type << 8, 0) for a = na; adj_amax = max na + 1
  const int4 *adj_desc;
  int adj_amax;
  // FP64 adjoint: runs of adj_group consecutive blocks (of the 256-slot
  // partition) form one group, whose table gradients are summed on their own
  // and stored as one partial; the partials are summed in group order
  int adj_group;
};

struct DevPot {
  int style;          // MZ_STYLE_*
  int ntypes;
  int nsplines;
  int tab_stride;     // doubles per candidate table
  int pow_stride;     // doubles per candidate evaluation table
  int s_phi, s_rho, s_U, s_f, s_g;  // first spline of each group
  int embed_extrap;
  int g_nmax;         // largest g-spline knot count (MEAM)
  int g_q5;           // an angular spline (g, q, q2) is spline5eq: the adjoint's quintic accumulators
  int omit_pen;       // leave out the style punishments (sharded databases)
  int gmeam;          // g indexed by (i; j, k) types and one f punishment per f spline
  int npair;          // ntypes (ntypes + 1) / 2
  int pair;           // pair/spline: phi only over each pair once (self images at 1/2),
                      // no embedding, no constraint or punishment entries
  int nj;             // JMEAM direct three-body terms sum p_ij p_ik q_i(cos): 0, 1 or 2
  int s_p[2], s_q[2]; // first spline of p, q (p2, q2)
  int aux_rows;       // per-slot adjoint sums kept per candidate: 5 (1 + nj)
  double energy_weight, stress_weight;
};

}  // namespace mzb
