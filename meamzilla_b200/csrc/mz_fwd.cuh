// Forward kernels of the objective (see mz_device.cu for the call sequence).
#pragma once

#include "mz_spline.cuh"

namespace mzb {

// Per-atom outputs, [cand][AO_COUNT][natoms].
enum { AO_AX = 0, AO_AY, AO_AZ, AO_E, AO_S0, AO_PEN = AO_S0 + 6, AO_RHO, AO_FSQ, AO_COUNT };
// Per-slot triplet sums kept for the adjoint, [cand][aux_rows][npairs]:
//   G_p = sum_k g f_k,  H_p = sum_k g' f_k cos,  vk_p = sum_k g' f_k u_k,
// and for each JMEAM term m the same with (q_m, p_m) at rows AUX_COUNT (1 + m) + ...
enum { AUX_G = 0, AUX_H, AUX_VX, AUX_VY, AUX_VZ, AUX_COUNT };
// Per-cell adjoint seeds, [cand][CS_COUNT][ncells]: dF/dE_atom, dF/dS (6), dF/dpen.
enum { CS_EPS = 0, CS_MU0, CS_KAPPA = CS_MU0 + 6, CS_COUNT };

// ------------------------------------------------------------------ k_prep

// Coefficient vectors -> per-candidate knot tables.  cmap has the table's
// layout: cmap[toff+k] (knot k) and cmap[toff+2n+e] (end e) hold the
// coefficient index, or -1 where the value is fixed and comes from base.
__global__ void k_prep(int ncand, int P, const double *__restrict__ params, const double *__restrict__ base,
                       const int *__restrict__ cmap, const SplineGeom *__restrict__ geom,
                       const int *__restrict__ nat, int nsplines, int stride, double *__restrict__ tabs,
                       int pstride, double *__restrict__ ptabs, float *__restrict__ ptabf = nullptr,
                       float *__restrict__ wtab = nullptr, int s_g = 0, int ng = 0, int nbp = 0,
                       const double *__restrict__ M = nullptr) {
  const int c = blockIdx.x;
  const int s = threadIdx.x;
  if (c >= ncand || s >= nsplines) return;
  const SplineGeom g = geom[s];
  const double *pc = params + (size_t)c * P;
  double *t = tabs + (size_t)c * stride + g.toff;
  const double *bt = base + g.toff;
  const int *cm = cmap + g.toff;
  const int n = g.n;
  for (int k = 0; k < n; ++k) t[k] = cm[k] >= 0 ? pc[cm[k]] : bt[k];
  for (int e = 0; e < 2; ++e) t[2 * n + e] = cm[2 * n + e] >= 0 ? pc[cm[2 * n + e]] : bt[2 * n + e];
  if (g.q5) {
    // spline5eq: y'' at the ends, then (ypp, yp4) = M (y, grad, grad2) -- the
    // refresh of Spline5Eq::refresh_basis (spline5eq.cpp:209-293) is linear
    // in them; M is solved once on the host
    double *g2 = t + 3 * n + 2, *yp4 = t + 2 * n + 2;
    for (int e = 0; e < 2; ++e) g2[e] = cm[3 * n + 2 + e] >= 0 ? pc[cm[3 * n + 2 + e]] : bt[3 * n + 2 + e];
    const double *Ms = M + g.moff;
    const int nc = n + 4;
    for (int r = 0; r < 2 * n; ++r) {
      const double *row = Ms + (size_t)r * nc;
      double acc = 0.0;
      for (int c = 0; c < n; ++c) acc += row[c] * t[c];
      acc += row[n] * t[2 * n] + row[n + 1] * t[2 * n + 1] + row[n + 2] * g2[0] + row[n + 3] * g2[1];
      if (r < n) t[n + r] = acc;
      else yp4[r - n] = acc;
    }
    double *pc6 = ptabs + (size_t)c * pstride + g.poff;
    const double H2 = g.step * g.step / 6.0, H4 = g.step * g.step * g.step * g.step / 360.0;
    for (int k = 0; k < n - 1; ++k) {
      const double p1 = t[k], p2 = t[k + 1], d21 = t[n + k], d22 = t[n + k + 1], d41 = yp4[k], d42 = yp4[k + 1];
      double *q = pc6 + 6 * k;
      q[0] = p1;
      q[1] = p2 - p1 + H2 * (-2.0 * d21 - d22) + H4 * (8.0 * d41 + 7.0 * d42);
      q[2] = 3.0 * H2 * d21;
      q[3] = H2 * (d22 - d21) + H4 * (-20.0 * d41 - 10.0 * d42);
      q[4] = 15.0 * H4 * d41;
      q[5] = H4 * (3.0 * d42 - 3.0 * d41);
    }
    if (ptabf) {
      float *pf = ptabf + (size_t)c * pstride + g.poff;
      for (int k = 0; k < 6 * (n - 1); ++k) pf[k] = (float)pc6[k];
    }
    return;
  }
  // Spline3Eq::refresh_basis (spline3eq.cpp:192-225)
  double u[64];
  double *y = t, *ypp = t + n;
  const double inv = g.invstep;
  const double gl = t[2 * n], gr = t[2 * n + 1];
  if (nat[2 * s]) {
    ypp[0] = 0;
    u[0] = 0;
  } else {
    ypp[0] = -0.5;
    u[0] = (3.0 * inv) * ((y[1] - y[0]) * inv - gl);
  }
  for (int i = 1; i < n - 1; ++i) {
    double p = 0.5 * ypp[i - 1] + 2.0;
    ypp[i] = (-0.5) / p;
    double ui = (y[i + 1] - y[i]) * inv - (y[i] - y[i - 1]) * inv;
    u[i] = (6.0 * ui * 0.5 * inv - 0.5 * u[i - 1]) / p;
  }
  double qn, un;
  if (nat[2 * s + 1]) {
    qn = un = 0.0;
  } else {
    qn = 0.5;
    un = (3.0 * inv) * (gr - (y[n - 1] - y[n - 2]) * inv);
  }
  ypp[n - 1] = (un - qn * u[n - 2]) / (qn * ypp[n - 2] + 1.0);
  for (int k = n - 2; k >= 0; --k) ypp[k] = ypp[k] * ypp[k + 1] + u[k];
  // evaluation table: the cubic of every interval in its shift
  double *pc4 = ptabs + (size_t)c * pstride + g.poff;
  const double H = g.step * g.step / 6.0;
  for (int k = 0; k < n - 1; ++k) {
    pc4[4 * k] = y[k];
    pc4[4 * k + 1] = y[k + 1] - y[k] - (2.0 * ypp[k] + ypp[k + 1]) * H;
    pc4[4 * k + 2] = 3.0 * ypp[k] * H;
    pc4[4 * k + 3] = (ypp[k + 1] - ypp[k]) * H;
  }
  if (ptabf) {  // FP32 copy of the evaluation table (mixed precision)
    float *pf = ptabf + (size_t)c * pstride + g.poff;
    for (int k = 0; k < 4 * (n - 1); ++k) pf[k] = (float)pc4[k];
  }
  if (wtab && s >= s_g && s < s_g + ng) {
    // Cubic B-spline coefficients of g on its uniform grid (basis function m
    // centred on knot m-1): S(x_i) = (w_i + 4 w_i+1 + w_i+2)/6 and
    // S''(x_i) = (w_i - 2 w_i+1 + w_i+2)/h^2 give w_i+1 = y_i - h^2/6 y''_i,
    // and the two outer coefficients follow from S'' at the end knots.
    // Their differences are the coefficients of g' (times h) in the
    // quadratic B-spline basis; both are stored: [w_0 .. w_nbp-1, dw_0 .. dw_nbp-2].
    float *w = wtab + ((size_t)c * ng + (s - s_g)) * (2 * nbp - 1);
    const double h2 = g.step * g.step;
    double wm[66];
    for (int i = 0; i < n; ++i) wm[i + 1] = y[i] - h2 / 6.0 * ypp[i];
    wm[0] = h2 * ypp[0] + 2.0 * wm[1] - wm[2];
    wm[n + 1] = h2 * ypp[n - 1] + 2.0 * wm[n] - wm[n - 1];
    for (int i = 0; i < nbp; ++i) w[i] = i < n + 2 ? (float)wm[i] : 0.f;
    for (int i = 0; i + 1 < nbp; ++i) w[nbp + i] = i + 1 < n + 2 ? (float)(wm[i + 1] - wm[i]) : 0.f;
  }
}

// ----------------------------------------------------------- atom blocks

// Shared state of one atom block, common to the forward and adjoint kernels.
struct BlockRows {
  int atom_lo, na, slot_lo, nslot;
};

__device__ __forceinline__ BlockRows block_rows(const DevDb &db, int blk) {
  BlockRows b;
  b.atom_lo = db.blk_atom0[blk];
  b.na = db.blk_atom0[blk + 1] - b.atom_lo;
  b.slot_lo = db.pair_off[b.atom_lo];
  b.nslot = db.pair_off[b.atom_lo + b.na] - b.slot_lo;
  return b;
}

// Owner atom of slot t: the last a with a_lo[a] <= t.
__device__ __forceinline__ int slot_owner(const int *a_lo, int na, int t) {
  int lo = 0, hi = na;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (a_lo[mid] <= t) lo = mid;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ int pair_ij_index(int ti, int tj, int nt) {
  return (ti <= tj) ? ti * nt + tj - (ti * (ti + 1)) / 2 : tj * nt + ti - (tj * (tj + 1)) / 2;
}

// Share of phi(r_p) in atom i's energy and forces: 1/2 in the double-counted
// lists; in pair/spline's single list 1, or 1/2 for an image of atom i itself
// (its two images +n and -n are both listed, pot_pair_spline.cpp:106-113).
__device__ __forceinline__ double phi_share(const DevPot &pot, bool self) {
  return pot.pair && !self ? 1.0 : 0.5;
}

// Pair functions of one slot: phi, rho, f with slopes (pot_meam_spline.cpp:152-191).
template <bool MEAM, typename R>
struct PairEval {
  R ux, uy, uz, r, invr;
  R phi, dphi, rho, drho, f, df;
  int kphi, krho, kf, tj, pij;
  R bphi, brho, bf;
  R p[2], dp[2], bp[2];  // JMEAM p (p2) (pot_jmeam_spline.cpp:196-202)
  int kp[2];
};

template <bool MEAM, typename R, bool Q5 = false>
__device__ __forceinline__ PairEval<MEAM, R> eval_pair(const DevDb &db, const DevPot &pot, const SplineGeom *sg,
                                                      const R *ptab, int64_t gs, int ti) {
  PairEval<MEAM, R> p;
  const int64_t Np = db.npairs;
  if (sizeof(R) == 8) {
    p.ux = (R)db.pair_ux[gs]; p.uy = (R)db.pair_uy[gs]; p.uz = (R)db.pair_uz[gs]; p.r = (R)db.pair_r[gs];
  } else {
    p.ux = (R)db.pair_uxf[gs]; p.uy = (R)db.pair_uyf[gs]; p.uz = (R)db.pair_uzf[gs]; p.r = (R)db.pair_rf[gs];
  }
  p.invr = R(1) / p.r;
  const int kn = db.pair_knot[gs];
  p.kphi = (kn & 0xff) - 1;
  p.krho = ((kn >> 8) & 0xff) - 1;
  p.kf = ((kn >> 16) & 0xff) - 1;
  p.tj = db.atom_type[db.pair_nbr[gs]];
  p.pij = pair_ij_index(ti, p.tj, pot.ntypes);
  p.phi = p.dphi = p.rho = p.drho = p.f = p.df = R(0);
  p.bphi = p.brho = p.bf = R(0);
  if (p.kphi >= 0) {
    const SplineGeom &g = sg[pot.s_phi + p.pij];
    p.bphi = sizeof(R) == 8 ? (R)db.pair_shift[gs] : (R)db.pair_shiftf[gs];
    p.phi = piece_val_grad<Q5, R>(ptab + g.poff, p.kphi, p.bphi, (R)g.invstep, p.dphi, g.q5);
  }
  if (p.krho >= 0) {
    const SplineGeom &g = sg[pot.s_rho + p.tj];
    p.brho = sizeof(R) == 8 ? (R)db.pair_shift[Np + gs] : (R)db.pair_shiftf[Np + gs];
    p.rho = piece_val_grad<Q5, R>(ptab + g.poff, p.krho, p.brho, (R)g.invstep, p.drho, g.q5);
  }
  if (MEAM && p.kf >= 0) {
    const SplineGeom &g = sg[pot.s_f + p.pij];
    p.bf = sizeof(R) == 8 ? (R)db.pair_shift[2 * Np + gs] : (R)db.pair_shiftf[2 * Np + gs];
    p.f = piece_val_grad<Q5, R>(ptab + g.poff, p.kf, p.bf, (R)g.invstep, p.df, g.q5);
  }
  return p;
}

// The JMEAM radial functions p (p2) of one slot.
template <bool MEAM, typename R, bool Q5 = false>
__device__ __forceinline__ void eval_pair_p(const DevDb &db, const DevPot &pot, const SplineGeom *sg, const R *ptab,
                                            int64_t gs, PairEval<MEAM, R> &p) {
  const int64_t Np = db.npairs;
  const int kn = db.pair_knot[gs];
  p.kp[0] = ((kn >> 24) & 0xff) - 1;
  p.kp[1] = pot.nj > 1 ? (int)db.pair_knot_p2[gs] : -1;
  for (int m = 0; m < 2; ++m) {
    p.p[m] = p.dp[m] = p.bp[m] = R(0);
    if (m < pot.nj && p.kp[m] >= 0) {
      const SplineGeom &g = sg[pot.s_p[m] + p.pij];
      p.bp[m] = sizeof(R) == 8 ? (R)db.pair_shift[(3 + m) * Np + gs] : (R)db.pair_shiftf[(3 + m) * Np + gs];
      p.p[m] = piece_val_grad<Q5, R>(ptab + g.poff, p.kp[m], p.bp[m], (R)g.invstep, p.dp[m], g.q5);
    }
  }
}

// ------------------------------------------------------------------ k_atoms

// Shared-memory layout of k_atoms (dynamic), see atoms_smem_bytes():
//   double red[10][BLOCK_SLOTS]       per-slot partials for the per-atom sums
//   double a_dF[BLOCK_ATOMS], a_U[BLOCK_ATOMS]
//   SplineGeom sg[nsplines]
//   int a_lo[BLOCK_ATOMS+2]
//   R ptab[pstride]                    this candidate's evaluation table
//   R4 srow[BLOCK_SLOTS]               (u_x, u_y, u_z, f) of every slot of the block
//   int stype[BLOCK_SLOTS+8]           neighbour type of every slot (GMEAM)
//   R spv[nj][BLOCK_SLOTS+8]           JMEAM p (p2) of every slot
template <typename R>
struct Vec4;
template <>
struct Vec4<float> {
  using T = float4;
};
template <>
struct Vec4<double> {
  using T = double4;
};

template <typename R>
__host__ __device__ inline size_t atoms_smem_bytes(int nsplines, int pstride, int nj = 0) {
  size_t b = sizeof(double) * (10 * BLOCK_SLOTS + 2 * BLOCK_ATOMS);
  b += sizeof(SplineGeom) * nsplines;
  b += sizeof(int) * (BLOCK_ATOMS + 2);
  b = (b + 31) & ~size_t(31);
  b += sizeof(R) * (pstride + 4);
  b = (b + 31) & ~size_t(31);
  b += 4 * sizeof(R) * (BLOCK_SLOTS + 8);
  b += sizeof(int) * (BLOCK_SLOTS + 8);  // neighbour type of every slot (GMEAM's g index)
  b += sizeof(R) * (size_t)nj * (BLOCK_SLOTS + 8);
  return b;
}

// g spline of the triplet (i; j, k) in GMEAM: Triplet_i_jk
// (PotFns::get_3body_alloy_idx, pot_fns.cpp:166-168).
__device__ __forceinline__ int gmeam_g_index(const DevPot &pot, int ti, int tj, int tk) {
  return pot.s_g + ti * pot.npair + pair_ij_index(tj, tk, pot.ntypes);
}

// Dot product of unit vectors: exact (no fused multiply-add, as the
// reference computes Triplet::cos) in FP64, fused in FP32.
__device__ __forceinline__ double cos_dot(double ax, double ay, double az, double bx, double by, double bz) {
  return cos_exact(ax, ay, az, bx, by, bz);
}
__device__ __forceinline__ float cos_dot(float ax, float ay, float az, float bx, float by, float bz) {
  return fmaf(ax, bx, fmaf(ay, by, az * bz));
}

// Row sums of one angular channel for slot `tid`: with w_k the partner's
// radial weight (f_k for g, p_k for a JMEAM q) and s the channel's spline,
//   S = sum_k s(cos) w_k,  T = sum_k s'(cos) w_k cos,  v = sum_k s'(cos) w_k u_k
// over the row's other slots whose cosine has a knot of s.  FP32 chunks of 8
// terms are added to FP64 totals (as the g loop of k_atoms).
template <bool Q5, typename R, typename R4, class W>
__device__ __forceinline__ void channel_row_sums(const R4 *srow, W weight, int row_lo, int row_hi, int tid, R ux,
                                                 R uy, R uz, const SplineGeom &gs, const R *spc, double &S, double &T,
                                                 double &vx, double &vy, double &vz) {
  const R x0 = (R)gs.x0, inv = (R)gs.invstep, cut = g_cut<R>(gs);
  S = T = vx = vy = vz = 0.0;
  for (int kb = row_lo; kb < row_hi; kb += 8) {
    R s8 = 0, t8 = 0, x8 = 0, y8 = 0, z8 = 0;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int k = kb + u;
      const R4 o = srow[k];
      const R cs = cos_dot(ux, uy, uz, o.x, o.y, o.z);
      const bool ok = (k < row_hi) && (k != tid) && (cs < cut);
      const R wk = ok ? weight(k) : R(0);
      R b;
      const int kk = g_knot<R>(cs, x0, inv, gs.n, b);
      R ds;
      const R sv = piece_val_grad<Q5, R>(spc, kk, b, inv, ds, gs.q5);
      const R dsw = ds * wk;
      s8 += sv * wk;
      t8 += dsw * cs;
      x8 += dsw * o.x;
      y8 += dsw * o.y;
      z8 += dsw * o.z;
    }
    S += (double)s8;
    T += (double)t8;
    vx += (double)x8;
    vy += (double)y8;
    vz += (double)z8;
  }
}


// Warp-cooperative sum over the slots [lo, hi) of `n` per-slot arrays
// red[q * BLOCK_SLOTS + s]; the result is valid on lane 0.  Fixed order.
template <int NQ>
__device__ __forceinline__ void warp_slot_sums(const double *red, int lo, int hi, int lane, double *out) {
#pragma unroll
  for (int q = 0; q < NQ; ++q) out[q] = 0.0;
  for (int s = lo + lane; s < hi; s += 32) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) out[q] += red[q * BLOCK_SLOTS + s];
  }
#pragma unroll
  for (int q = 0; q < NQ; ++q)
    for (int o = 16; o > 0; o >>= 1) out[q] += __shfl_down_sync(0xffffffffu, out[q], o);
}

// One CTA per (atom block, candidate), one thread per pair slot.  A single
// pass over each slot's row gives G_p, H_p and vk_p; the density
// rho_i = sum_p rho_p + 1/2 sum_p f_p G_p (each j<k triplet seen from both
// ends) and every force term follow from them (pot_meam_spline.cpp:143-269):
//   V_p = u_p (phi'_p/2 + rho'_p U') + U' [u_p (f'_p G_p - f_p H_p / r_p)
//                                          + f_p vk_p / r_p]
// is the force atom i's terms add to atom i along slot p; the neighbour
// receives -V_p (k_gather).  In FP32 the row sums are taken in chunks of 8
// terms, each chunk added to an FP64 total.
template <bool MEAM, typename R, bool AUX, bool GM = false, bool JM = false, bool Q5 = false>
__global__ void __launch_bounds__(BLOCK_SLOTS, JM ? 2 : sizeof(R) == 4 ? 4 : 3)
    k_atoms(DevDb db, DevPot pot, const SplineGeom *__restrict__ geom, const double *__restrict__ tabs,
            const double *__restrict__ ptabs, double *__restrict__ Vout, double *__restrict__ aout,
            double *__restrict__ aux) {
  using R4 = typename Vec4<R>::T;
  extern __shared__ __align__(32) unsigned char smem_raw[];
  const int cand = blockIdx.y;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
  const int N = db.natoms;
  const int64_t Np = db.npairs;

  double *red = reinterpret_cast<double *>(smem_raw);
  double *a_dF = red + 10 * BLOCK_SLOTS;
  double *a_U = a_dF + BLOCK_ATOMS;
  SplineGeom *sg = reinterpret_cast<SplineGeom *>(a_U + BLOCK_ATOMS);
  int *a_lo = reinterpret_cast<int *>(sg + pot.nsplines);
  size_t off = sizeof(double) * (10 * BLOCK_SLOTS + 2 * BLOCK_ATOMS) + sizeof(SplineGeom) * pot.nsplines +
               sizeof(int) * (BLOCK_ATOMS + 2);
  off = (off + 31) & ~size_t(31);
  R *ptab = reinterpret_cast<R *>(smem_raw + off);
  off += sizeof(R) * (pot.pow_stride + 4);
  off = (off + 31) & ~size_t(31);
  R4 *srow = reinterpret_cast<R4 *>(smem_raw + off);
  int *stype = reinterpret_cast<int *>(srow + BLOCK_SLOTS + 8);
  R *spv = reinterpret_cast<R *>(stype + BLOCK_SLOTS + 8);

  const BlockRows br = block_rows(db, blockIdx.x);
  const double *tc = tabs + (size_t)cand * pot.tab_stride;
  const double *pc = ptabs + (size_t)cand * pot.pow_stride;
  for (int i = tid; i < pot.pow_stride; i += blockDim.x) ptab[i] = (R)pc[i];
  for (int i = tid; i < pot.nsplines; i += blockDim.x) sg[i] = geom[i];
  for (int a = tid; a <= br.na; a += blockDim.x) a_lo[a] = db.pair_off[br.atom_lo + a] - br.slot_lo;
  __syncthreads();

  const bool have = tid < br.nslot;
  const int me = have ? slot_owner(a_lo, br.na, tid) : 0;
  const int ti = db.atom_type[br.atom_lo + me];
  const int64_t gs = (int64_t)br.slot_lo + tid;

  PairEval<MEAM, R> pe;
  {
    R4 v;
    v.x = v.y = v.z = v.w = R(0);
    if (have) {
      pe = eval_pair<MEAM, R, Q5>(db, pot, sg, ptab, gs, ti);
      v.x = pe.ux; v.y = pe.uy; v.z = pe.uz; v.w = pe.f;
    }
    srow[tid] = v;
    if (tid < 8) srow[BLOCK_SLOTS + tid] = R4{};
    if (GM) {
      stype[tid] = have ? pe.tj : 0;
      if (tid < 8) stype[BLOCK_SLOTS + tid] = 0;
    }
    if (JM) {
      if (have) eval_pair_p<MEAM, R, Q5>(db, pot, sg, ptab, gs, pe);
      for (int m = 0; m < pot.nj; ++m) {
        spv[m * (BLOCK_SLOTS + 8) + tid] = have ? pe.p[m] : R(0);
        if (tid < 8) spv[m * (BLOCK_SLOTS + 8) + BLOCK_SLOTS + tid] = R(0);
      }
    }
  }
  __syncthreads();

  // ---- the one pass over the row: G_p, H_p, vk_p
  double G = 0, H = 0, vkx = 0, vky = 0, vkz = 0;
  if (GM && have && (AUX || pe.f != R(0) || pe.df != R(0))) {
    // GMEAM: the g spline depends on the partner's neighbour type as well
    const int row_lo = a_lo[me], row_hi = a_lo[me + 1];
    for (int kb = row_lo; kb < row_hi; kb += 8) {
      R g8 = 0, h8 = 0, x8 = 0, y8 = 0, z8 = 0;
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int k = kb + u;
        const R4 o = srow[k];
        const SplineGeom &g2 = sg[gmeam_g_index(pot, ti, pe.tj, stype[k])];
        const R ginv = (R)g2.invstep;
        const R cs = cos_dot(pe.ux, pe.uy, pe.uz, o.x, o.y, o.z);
        const bool ok = (k < row_hi) && (k != tid) && (cs < g_cut<R>(g2));  // triplet_meam_spline.cpp:66-70
        const R fk = ok ? o.w : R(0);
        R b;
        const int kk = g_knot<R>(cs, (R)g2.x0, ginv, g2.n, b);
        R dg;
        const R gv = piece_val_grad<Q5, R>(ptab + g2.poff, kk, b, ginv, dg, g2.q5);
        const R dgfk = dg * fk;
        g8 += gv * fk;
        h8 += dgfk * cs;
        x8 += dgfk * o.x;
        y8 += dgfk * o.y;
        z8 += dgfk * o.z;
      }
      G += (double)g8;
      H += (double)h8;
      vkx += (double)x8;
      vky += (double)y8;
      vkz += (double)z8;
    }
    if (AUX) {
      double *ax = aux + (size_t)cand * (JM ? pot.aux_rows : (int)AUX_COUNT) * Np;
      ax[AUX_G * Np + gs] = G;
      ax[AUX_H * Np + gs] = H;
      ax[AUX_VX * Np + gs] = vkx;
      ax[AUX_VY * Np + gs] = vky;
      ax[AUX_VZ * Np + gs] = vkz;
    }
  } else if (!GM && MEAM && have && (AUX || pe.f != R(0) || pe.df != R(0))) {
    const SplineGeom gg = sg[pot.s_g + ti];
    const R *gpc = ptab + gg.poff;
    const R gx0 = (R)gg.x0, ginv = (R)gg.invstep;
    const R gcut = g_cut<R>(gg);
    const int row_lo = a_lo[me], row_hi = a_lo[me + 1];
    for (int kb = row_lo; kb < row_hi; kb += 8) {
      R g8 = 0, h8 = 0, x8 = 0, y8 = 0, z8 = 0;
      // Branch-free chunk of 8 partners: a partner that is this slot, past
      // the row, or not a triplet contributes with weight zero.  srow is
      // padded with zero rows past the block's last slot.
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int k = kb + u;
        const R4 o = srow[k];
        const R cs = cos_dot(pe.ux, pe.uy, pe.uz, o.x, o.y, o.z);
        const bool ok = (k < row_hi) && (k != tid) && (cs < gcut);  // triplet_meam_spline.cpp:66-70
        const R fk = ok ? o.w : R(0);
        R b;
        const int kk = g_knot<R>(cs, gx0, ginv, gg.n, b);
        R dg;
        const R gv = piece_val_grad<Q5, R>(gpc, kk, b, ginv, dg, gg.q5);
        const R dgfk = dg * fk;
        g8 += gv * fk;
        h8 += dgfk * cs;
        x8 += dgfk * o.x;
        y8 += dgfk * o.y;
        z8 += dgfk * o.z;
      }
      G += (double)g8;
      H += (double)h8;
      vkx += (double)x8;
      vky += (double)y8;
      vkz += (double)z8;
    }
    if (AUX) {
      double *ax = aux + (size_t)cand * (JM ? pot.aux_rows : (int)AUX_COUNT) * Np;
      ax[AUX_G * Np + gs] = G;
      ax[AUX_H * Np + gs] = H;
      ax[AUX_VX * Np + gs] = vkx;
      ax[AUX_VY * Np + gs] = vky;
      ax[AUX_VZ * Np + gs] = vkz;
    }
  }
  // ---- JMEAM: the same row sums for each (p, q) term (pot_jmeam_spline.cpp:208-219)
  double G2[2] = {0, 0}, H2[2] = {0, 0}, v2x[2] = {0, 0}, v2y[2] = {0, 0}, v2z[2] = {0, 0};
  if (JM && have) {
    for (int m = 0; m < pot.nj; ++m) {
      if (!AUX && pe.p[m] == R(0) && pe.dp[m] == R(0)) continue;
      const SplineGeom qg = sg[pot.s_q[m] + ti];
      const R *wm = spv + m * (BLOCK_SLOTS + 8);
      channel_row_sums<Q5, R>(srow, [&](int k) { return wm[k]; }, a_lo[me], a_lo[me + 1], tid, pe.ux, pe.uy, pe.uz,
                          qg, ptab + qg.poff, G2[m], H2[m], v2x[m], v2y[m], v2z[m]);
      if (AUX) {
        double *ax = aux + ((size_t)cand * pot.aux_rows + AUX_COUNT * (1 + m)) * Np;
        ax[AUX_G * Np + gs] = G2[m];
        ax[AUX_H * Np + gs] = H2[m];
        ax[AUX_VX * Np + gs] = v2x[m];
        ax[AUX_VY * Np + gs] = v2y[m];
        ax[AUX_VZ * Np + gs] = v2z[m];
      }
    }
  }
  if (have) red[tid] = (double)pe.rho + (MEAM ? 0.5 * (double)pe.f * G : 0.0);
  __syncthreads();

  // ---- embedding (pot_meam_spline.cpp:208-223): one warp per atom
  for (int a = warp; a < br.na; a += nwarp) {
    double rho;
    warp_slot_sums<1>(red, a_lo[a], a_lo[a + 1], lane, &rho);
    if (lane == 0 && pot.pair) {
      double *ao = aout + (size_t)cand * AO_COUNT * N;
      a_dF[a] = a_U[a] = 0.0;
      ao[AO_PEN * N + br.atom_lo + a] = 0.0;
      ao[AO_RHO * N + br.atom_lo + a] = 0.0;
    } else if (lane == 0) {
      const int ia = br.atom_lo + a;
      const SplineGeom &gU = sg[pot.s_U + db.atom_type[ia]];
      const double w = db.cell_w[db.atom_cell[ia]];
      double pen = 0.0;
      const double lo = gU.x0, hi = gU.xN;
      const double rho_raw = rho;
      if (rho < lo) {
        pen = w * 100.0 * 10. * (lo - rho) * (lo - rho);
        if (!pot.embed_extrap) rho = lo;
      } else if (rho > hi) {
        pen = w * 100.0 * 10. * (rho - hi) * (rho - hi);
        if (!pot.embed_extrap) rho = hi;
      }
      const PointEval U = spl_point_t<Q5>(tc, gU, rho);  // FP64 table of this candidate
      a_dF[a] = U.grad;
      a_U[a] = U.val;
      double *ao = aout + (size_t)cand * AO_COUNT * N;
      ao[AO_PEN * N + ia] = pen;
      ao[AO_RHO * N + ia] = rho_raw;
    }
  }
  __syncthreads();

  // ---- V_p and the slot's stress (stress.h:134-137; pot_meam_spline.cpp:171-173, 234-236, 265-268)
  if (have) {
    const double dF = a_dF[me];
    const double ux = (double)pe.ux, uy = (double)pe.uy, uz = (double)pe.uz;
    const double sp = MEAM ? 0.5 : phi_share(pot, db.pair_nbr[gs] == br.atom_lo + me);
    double cu = sp * (double)pe.dphi + (double)pe.drho * dF;
    double Vx = 0, Vy = 0, Vz = 0;
    double e3 = 0.0;  // JMEAM: 1/2 sum_m p_m G2_m, this slot's share of the p p q energy
    if (MEAM) {
      const double ip = (double)pe.invr, fp = (double)pe.f;
      cu += dF * ((double)pe.df * G - fp * ip * H);
      const double ck = dF * fp * ip;
      Vx = ck * vkx;
      Vy = ck * vky;
      Vz = ck * vkz;
      if (JM)
        for (int m = 0; m < pot.nj; ++m) {
          // the q terms' dfj without U' (pot_jmeam_spline.cpp:263-273)
          const double pm = (double)pe.p[m];
          cu += (double)pe.dp[m] * G2[m] - pm * ip * H2[m];
          Vx += pm * ip * v2x[m];
          Vy += pm * ip * v2y[m];
          Vz += pm * ip * v2z[m];
          e3 += 0.5 * pm * G2[m];
        }
    }
    Vx += ux * cu;
    Vy += uy * cu;
    Vz += uz * cu;
    double *Vc = Vout + (size_t)cand * 3 * Np + 3 * gs;  // (x, y, z) per slot
    Vc[0] = Vx;
    Vc[1] = Vy;
    Vc[2] = Vz;
    const double rr = db.pair_r[gs];
    const double dx = db.pair_ux[gs], dy = db.pair_uy[gs], dz = db.pair_uz[gs];
    red[0 * BLOCK_SLOTS + tid] = Vx;
    red[1 * BLOCK_SLOTS + tid] = Vy;
    red[2 * BLOCK_SLOTS + tid] = Vz;
    red[3 * BLOCK_SLOTS + tid] = sp * (double)pe.phi + e3;
    red[4 * BLOCK_SLOTS + tid] = -(dx * (Vx * rr));
    red[5 * BLOCK_SLOTS + tid] = -(dy * (Vy * rr));
    red[6 * BLOCK_SLOTS + tid] = -(dz * (Vz * rr));
    red[7 * BLOCK_SLOTS + tid] = -(dx * (Vy * rr));
    red[8 * BLOCK_SLOTS + tid] = -(dy * (Vz * rr));
    red[9 * BLOCK_SLOTS + tid] = -(dz * (Vx * rr));
  }
  __syncthreads();
  for (int a = warp; a < br.na; a += nwarp) {
    double acc[10];
    warp_slot_sums<10>(red, a_lo[a], a_lo[a + 1], lane, acc);
    if (lane == 0) {
      const int ia = br.atom_lo + a;
      double *ao = aout + (size_t)cand * AO_COUNT * N;
      ao[AO_AX * N + ia] = acc[0];
      ao[AO_AY * N + ia] = acc[1];
      ao[AO_AZ * N + ia] = acc[2];
      ao[AO_E * N + ia] = acc[3] + a_U[a];
#pragma unroll
      for (int q = 0; q < 6; ++q) ao[(AO_S0 + q) * N + ia] = acc[4 + q];
    }
  }
}

// ----------------------------------------------------------------- k_gather

// F_i = sum of V over the atom's own slots - sum of V over the slots whose
// neighbour is i; then the force residual w (F - F0) (potential.cpp:468-478)
// and, for the adjoint, lambda_i = dF/dF_i = 2 w e_i.
__global__ void k_gather(DevDb db, const double *__restrict__ V, double *__restrict__ aout,
                         double *__restrict__ forces, double *__restrict__ errvec, int esize,
                         double *__restrict__ lam) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  const int N = db.natoms;
  if (i >= N) return;
  const int64_t Np = db.npairs;
  double *ao = aout + (size_t)c * AO_COUNT * N;
  const double *Vc = V + (size_t)c * 3 * Np;  // (x, y, z) per slot: one or two 32-byte sectors a read
  double fx = ao[AO_AX * N + i], fy = ao[AO_AY * N + i], fz = ao[AO_AZ * N + i];
  for (int q = db.in_off[i]; q < db.in_off[i + 1]; ++q) {
    const double *v = Vc + 3 * (int64_t)db.in_slot[q];
    fx -= v[0];
    fy -= v[1];
    fz -= v[2];
  }
  const int cell = db.atom_cell[i];
  const double w = db.cell_w[cell];
  const double rx = w * (fx - db.force0[3 * i]);
  const double ry = w * (fy - db.force0[3 * i + 1]);
  const double rz = w * (fz - db.force0[3 * i + 2]);
  ao[AO_FSQ * N + i] = rx * rx + ry * ry + rz * rz;
  if (forces) {
    double *F = forces + (size_t)c * 3 * N;
    F[3 * i] = fx;
    F[3 * i + 1] = fy;
    F[3 * i + 2] = fz;
  }
  if (errvec) {
    const int a0 = db.cell_atom0[cell];
    double *e = errvec + (size_t)c * esize + 7 * (cell + 1) + 3 * a0 + 3 * (i - a0);
    e[0] = rx;
    e[1] = ry;
    e[2] = rz;
  }
  if (lam) {
    double *L = lam + (size_t)c * 3 * N;
    L[i] = 2.0 * w * rx;
    L[N + i] = 2.0 * w * ry;
    L[2 * N + i] = 2.0 * w * rz;
  }
}

// ------------------------------------------------------------------ k_cells

// One warp per cell (potential.cpp:450-485); with `seeds`, also the adjoint
// seeds dF/dE_atom, dF/dS_cell and dF/dpen of the cell.
__global__ void k_cells(DevDb db, DevPot pot, const double *__restrict__ aout, double *__restrict__ cellobj,
                        double *__restrict__ errvec, int esize, double *__restrict__ energy,
                        double *__restrict__ stress, double *__restrict__ seeds) {
  const int cell = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  const int c = blockIdx.y;
  if (cell >= db.ncells) return;
  const int N = db.natoms;
  const double *ao = aout + (size_t)c * AO_COUNT * N;
  const int a0 = db.cell_atom0[cell], a1 = db.cell_atom0[cell + 1];
  double v[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) v[q] = 0.0;
  for (int a = a0 + lane; a < a1; a += 32) {
    v[0] += ao[AO_E * N + a];
#pragma unroll
    for (int q = 0; q < 6; ++q) v[1 + q] += ao[(AO_S0 + q) * N + a];
    v[7] += ao[AO_PEN * N + a];
    v[8] += ao[AO_FSQ * N + a];
  }
#pragma unroll
  for (int q = 0; q < 9; ++q)
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
  if (lane == 0) {
    const int na = a1 - a0;
    const double w = db.cell_w[cell];
    const double E = v[0] / na;
    const double ew = w * db.cell_ew[cell] * pot.energy_weight;
    const double eE = ew * na * (E - db.cell_e0[cell]);
    double sum = eE * eE;
    double eS[6], sig[6];
    const double sw = w * db.cell_sw[cell] * pot.stress_weight;
    for (int q = 0; q < 6; ++q) {
      sig[q] = v[1 + q] / db.cell_vol[cell];
      eS[q] = sw * (sig[q] - db.cell_s0[6 * cell + q]);
      sum += eS[q] * eS[q];
    }
    sum += v[8];
    const double cons = v[7];
    sum += cons * cons;
    cellobj[(size_t)c * db.ncells + cell] = sum;
    if (errvec) {
      double *e = errvec + (size_t)c * esize + 7 * cell + 3 * a0;
      e[0] = eE;
      for (int q = 0; q < 6; ++q) e[1 + q] = eS[q];
      if (!pot.pair) errvec[(size_t)c * esize + 7 * db.ncells + 3 * N + cell] = cons;
    }
    if (energy) energy[(size_t)c * db.ncells + cell] = E;
    if (stress)
      for (int q = 0; q < 6; ++q) stress[((size_t)c * db.ncells + cell) * 6 + q] = sig[q];
    if (seeds) {
      double *sd = seeds + (size_t)c * CS_COUNT * db.ncells;
      sd[CS_EPS * db.ncells + cell] = 2.0 * eE * ew;
      for (int q = 0; q < 6; ++q) sd[(CS_MU0 + q) * db.ncells + cell] = 2.0 * eS[q] * sw / db.cell_vol[cell];
      sd[CS_KAPPA * db.ncells + cell] = 2.0 * cons;
    }
  }
}

// ------------------------------------------------------------------ k_final

// Sum of squares over cells + the style's punishment entries.
// Signed largest-|y| knot of one spline (Spline::get_max_y_mag, spline.cpp:58-67).
__device__ __forceinline__ double spline_max_y(const SplineGeom &g, const double *tab, int *which) {
  double sm = 0.0;
  int sat = -1;
  for (int k = 0; k < g.n; ++k) {
    const double y = tab[g.toff + k];
    if (fabs(sm) < fabs(y)) {
      sm = y;
      sat = g.toff + k;
    }
  }
  if (which) *which = sat;
  return sm;
}
// Signed largest-|y| knot over a Pair_ij group (PotFns::get_max_y_mag,
// pot_fns.cpp:100-111) whose first spline is s0: f, or JMEAM's p (p2).
__device__ __forceinline__ double group_max_y(const DevPot &pot, int s0, const SplineGeom *geom, const double *tab,
                                              int *which) {
  double my = 0.0;
  int at = -1;
  const int nf = pot.ntypes * (pot.ntypes + 1) / 2;
  for (int f = 0; f < nf; ++f) {
    int sat;
    const double sm = spline_max_y(geom[s0 + f], tab, &sat);
    if (fabs(my) < fabs(sm)) {
      my = sm;
      at = sat;
    }
  }
  if (which) *which = at;
  return my;
}

__global__ void k_final(DevDb db, DevPot pot, const SplineGeom *__restrict__ geom,
                        const double *__restrict__ tabs, const double *__restrict__ cellobj,
                        double *__restrict__ obj, double *__restrict__ errvec, int esize) {
  __shared__ double part[256];
  const int c = blockIdx.x;
  const int t = threadIdx.x;
  double s = 0.0;
  for (int i = t; i < db.ncells; i += blockDim.x) s += cellobj[(size_t)c * db.ncells + i];
  part[t] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (t < o) part[t] += part[t + o];
    __syncthreads();
  }
  if (t == 0) {
    double total = part[0];
    const double *tab = tabs + (size_t)c * pot.tab_stride;
    double *ev = errvec ? errvec + (size_t)c * esize + 8 * db.ncells + 3 * db.natoms : nullptr;
    if (pot.pair) {
      // no punishments (PotPairSpline::fast_compute, pot_pair_spline.cpp:133)
    } else if (pot.omit_pen) {
      if (ev) {
        const int npen = pot.style == MZ_STYLE_MEAM_SPLINE ? 1
                         : pot.nj > 0                     ? 1 + pot.nj
                         : pot.gmeam                      ? pot.npair
                                                          : pot.ntypes;
        for (int q = 0; q < npen; ++q) ev[q] = 0.0;
      }
    } else if (pot.gmeam) {
      // one f-magnitude punishment per f spline (pot_gmeam_spline.cpp:173-178)
      for (int f = 0; f < pot.npair; ++f) {
        const double m = fabs(spline_max_y(geom[pot.s_f + f], tab, nullptr));
        const double fe = 100. * 25. * (1.0 - m) * (1.0 - m);
        total += fe * fe;
        if (ev) ev[f] = fe;
      }
    } else if (pot.style == MZ_STYLE_MEAM_SPLINE || pot.nj > 0) {
      // f-potential magnitude punishment (pot_meam_spline.cpp:274-278), and
      // JMEAM's p (p2) magnitude punishments (pot_jmeam_spline.cpp:286-299)
      for (int q = 0; q <= pot.nj; ++q) {
        const double m = fabs(group_max_y(pot, q == 0 ? pot.s_f : pot.s_p[q - 1], geom, tab, nullptr));
        const double fe = 100. * 25. * (1.0 - m) * (1.0 - m);
        total += fe * fe;
        if (ev) ev[q] = fe;
      }
    } else {
      // U'(mid-range) punishment per type (pot_eam_spline.cpp:211-218)
      for (int ty = 0; ty < pot.ntypes; ++ty) {
        const SplineGeom &g = geom[pot.s_U + ty];
        const double e = 100. * spl_point_any(tab, g, 0.5 * (g.x0 + g.xN)).grad;
        total += e * e;
        if (ev) ev[ty] = e;
      }
    }
    obj[c] = total;
  }
}

}  // namespace mzb
