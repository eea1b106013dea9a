// B200 evaluator of the spline EAM/MEAM fitting objective: device context,
// kernels and the evaluator half of the C ABI (include/mz_b200.h).
//
// Work decomposition (one launch sequence per objective call):
//   k_prep    one thread per (candidate, spline): coefficients -> knot table,
//             second derivatives by the reference's tridiagonal solve
//             (Spline3Eq::refresh_basis, spline3eq.cpp:192-225).
//   k_atoms   one CTA per (atom block, candidate), one thread per pair slot.
//             The atom block's neighbour rows are staged in shared memory;
//             triplets are enumerated implicitly as the other slots of the
//             same row, so nothing per triplet is stored.  It computes, per
//             atom, the embedding density, U and U', and per pair slot the
//             reaction vector V_p that the atom's terms apply to the
//             neighbour (PotMEAMSpline::fast_compute, pot_meam_spline.cpp:
//             143-270; PotEAMSpline::fast_compute, pot_eam_spline.cpp:135-207).
//   k_gather  one thread per atom: F_i = sum_p V_p(own row) - sum V(incoming
//             slots) -- the reference's "atom_j.force -= ..." scatter,
//             written as a gather so no atomics are needed.
//   k_cells   one warp per cell: energy per atom, stress / volume, constraint
//             and the residual vector entries (Potential::accumulate_error,
//             potential.cpp:415-491).
//   k_final   one CTA per candidate: sum of squares + style penalties
//             (pot_meam_spline.cpp:274-278, pot_eam_spline.cpp:211-218).
// All reductions run in a fixed order: results are bit-reproducible.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "mz_b200.h"
#include "mz_device.cuh"
#include "mz_host.hpp"

namespace mzb {

// ------------------------------------------------------------- spline math

template <typename R>
__device__ __forceinline__ R spl_val_grad(const R *y, const R *ypp, int k, R b, R step6, R stepsq6,
                                          R invstep, R &grad) {
  // Spline3Eq::splint_comb(int, double, double*) (spline3eq.h:110-122)
  const R a = R(1) - b;
  const R p1 = y[k], p2 = y[k + 1], d1 = ypp[k], d2 = ypp[k + 1];
  grad = (p2 - p1) * invstep + ((R(3) * b * b - R(1)) * d2 - (R(3) * a * a - R(1)) * d1) * step6;
  return a * p1 + b * p2 + ((a * a * a - a) * d1 + (b * b * b - b) * d2) * stepsq6;
}

template <typename R>
__device__ __forceinline__ R spl_val(const R *y, const R *ypp, int k, R b, R stepsq6) {
  const R a = R(1) - b;
  return a * y[k] + b * y[k + 1] + ((a * a * a - a) * ypp[k] + (b * b * b - b) * ypp[k + 1]) * stepsq6;
}

// Value + slope at a point with linear extrapolation
// (Spline3Eq::splint_comb(double, double*), spline3eq.h:204-236).  FP64.
__device__ __forceinline__ double spl_point(const double *tab, const SplineGeom &g, double r, double *grad) {
  const double *y = tab + g.toff, *ypp = y + g.n, *ge = y + 2 * g.n;
  const double xN = g.xN;
  if (r < g.x0) {
    *grad = ge[0];
    return y[0] + ge[0] * (r - g.x0);
  } else if (r > xN) {
    *grad = ge[1];
    return y[g.n - 1] + ge[1] * (r - xN);
  }
  double dr = r - g.x0;
  int k = (dr < 0) ? 0 : int(dr * g.invstep);
  if (k >= g.n - 1) k = g.n - 2;
  double b = (dr - k * g.step) * g.invstep;
  return spl_val_grad<double>(y, ypp, k, b, g.step / 6.0, g.step * g.step / 6.0, g.invstep, *grad);
}

// Knot + shift of cos(theta) on the g grid.  The reference bisects
// (spline.cpp:74-99); the interval found here is the same except within an
// ulp of a knot, where the spline's value and slope agree to rounding.
template <typename R>
__device__ __forceinline__ int g_knot(R c, R x0, R invstep, int n, R &b) {
  R t = (c - x0) * invstep;
  int k = (int)floor(t);
  k = k < 0 ? 0 : (k > n - 2 ? n - 2 : k);
  b = t - R(k);
  return k;
}

// cos(theta) exactly as Triplet::setup_triplet: x*x' + y*y' + z*z' with no
// fused multiply-add (triplet.cpp:34-40, vect.h:137-141).
__device__ __forceinline__ double cos_exact(double ax, double ay, double az, double bx, double by, double bz) {
  return __dadd_rn(__dadd_rn(__dmul_rn(ax, bx), __dmul_rn(ay, by)), __dmul_rn(az, bz));
}
__device__ __forceinline__ float cos_exact(float ax, float ay, float az, float bx, float by, float bz) {
  return __fadd_rn(__fadd_rn(__fmul_rn(ax, bx), __fmul_rn(ay, by)), __fmul_rn(az, bz));
}

// --------------------------------------------------------------- k_prep

// Coefficient vectors -> per-candidate knot tables.  cmap has the table's
// layout: cmap[toff+k] (knot k) and cmap[toff+2n+e] (end e) hold the
// coefficient index, or -1 where the value is fixed and comes from base.
__global__ void k_prep(int ncand, int P, const double *__restrict__ params, const double *__restrict__ base,
                       const int *__restrict__ cmap, const SplineGeom *__restrict__ geom,
                       const int *__restrict__ nat, int nsplines, int stride, double *__restrict__ tabs) {
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
  // Spline3Eq::refresh_basis (spline3eq.cpp:192-225); u lives in registers
  // of a fixed-size local array (n <= 64).
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
}

// -------------------------------------------------------------- k_atoms

// Per-atom outputs, [cand][AO_COUNT][natoms].
enum { AO_AX = 0, AO_AY, AO_AZ, AO_E, AO_S0, AO_PEN = AO_S0 + 6, AO_RHO, AO_FSQ, AO_COUNT };

// Shared-memory layout of k_atoms (dynamic), see atoms_smem_bytes():
//   double red[10][BLOCK_SLOTS]   per-slot partials for the per-atom sums
//   double a_dF[BLOCK_ATOMS], a_U[BLOCK_ATOMS]
//   SplineGeom sg[nsplines]
//   int a_lo[BLOCK_ATOMS+1]
//   R tab[stride]                  this candidate's knot tables
//   R sx,sy,sz,sf,sdf[BLOCK_SLOTS] pair data of the block
template <typename R>
__host__ __device__ inline size_t atoms_smem_bytes(int nsplines, int stride) {
  size_t b = sizeof(double) * (10 * BLOCK_SLOTS + 2 * BLOCK_ATOMS);
  b += sizeof(SplineGeom) * nsplines;
  b += sizeof(int) * (BLOCK_ATOMS + 2);
  b = (b + 15) & ~size_t(15);
  b += sizeof(R) * (stride + 1);
  b = (b + 15) & ~size_t(15);
  b += sizeof(R) * 5 * BLOCK_SLOTS;
  return b;
}

template <bool MEAM, typename R>
__global__ void __launch_bounds__(BLOCK_SLOTS)
    k_atoms(DevDb db, DevPot pot, const SplineGeom *__restrict__ geom, const double *__restrict__ tabs,
            double *__restrict__ Vout, double *__restrict__ aout) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int cand = blockIdx.y;
  const int blk = blockIdx.x;
  const int tid = threadIdx.x;
  const int N = db.natoms;
  const int64_t Np = db.npairs;

  double *red = reinterpret_cast<double *>(smem_raw);
  double *a_dF = red + 10 * BLOCK_SLOTS;
  double *a_U = a_dF + BLOCK_ATOMS;
  SplineGeom *sg = reinterpret_cast<SplineGeom *>(a_U + BLOCK_ATOMS);
  int *a_lo = reinterpret_cast<int *>(sg + pot.nsplines);
  size_t off = sizeof(double) * (10 * BLOCK_SLOTS + 2 * BLOCK_ATOMS) + sizeof(SplineGeom) * pot.nsplines +
               sizeof(int) * (BLOCK_ATOMS + 2);
  off = (off + 15) & ~size_t(15);
  R *tab = reinterpret_cast<R *>(smem_raw + off);
  off += sizeof(R) * (pot.tab_stride + 1);
  off = (off + 15) & ~size_t(15);
  R *sx = reinterpret_cast<R *>(smem_raw + off);
  R *sy = sx + BLOCK_SLOTS, *sz = sy + BLOCK_SLOTS, *sf = sz + BLOCK_SLOTS, *sdf = sf + BLOCK_SLOTS;

  const int atom_lo = db.blk_atom0[blk], atom_hi = db.blk_atom0[blk + 1];
  const int na = atom_hi - atom_lo;
  const int slot_lo = db.pair_off[atom_lo];
  const int nslot = db.pair_off[atom_hi] - slot_lo;

  const double *tc = tabs + (size_t)cand * pot.tab_stride;
  for (int i = tid; i < pot.tab_stride; i += blockDim.x) tab[i] = (R)tc[i];
  for (int i = tid; i < pot.nsplines; i += blockDim.x) sg[i] = geom[i];
  for (int a = tid; a <= na; a += blockDim.x) a_lo[a] = db.pair_off[atom_lo + a] - slot_lo;
  __syncthreads();

  const bool have = tid < nslot;
  // owner atom of my slot: last a with a_lo[a] <= tid
  int me = 0;
  if (have) {
    int lo = 0, hi = na;  // a_lo[lo] <= tid < a_lo[hi]
    while (hi - lo > 1) {
      int mid = (lo + hi) >> 1;
      if (a_lo[mid] <= tid) lo = mid;
      else hi = mid;
    }
    me = lo;
  }
  const int ti = db.atom_type[atom_lo + me];

  // ---- pair phase: phi, rho, f of my slot (pot_meam_spline.cpp:152-191)
  const int64_t gs = (int64_t)slot_lo + tid;
  R ux = 0, uy = 0, uz = 0, r = 0, fv = 0, dfv = 0, drho = 0, phig = 0, invr = 0;
  double e_half = 0.0, rho_p = 0.0;
  if (have) {
    if (sizeof(R) == 8) {
      ux = (R)db.pair_ux[gs]; uy = (R)db.pair_uy[gs]; uz = (R)db.pair_uz[gs]; r = (R)db.pair_r[gs];
    } else {
      ux = (R)db.pair_uxf[gs]; uy = (R)db.pair_uyf[gs]; uz = (R)db.pair_uzf[gs]; r = (R)db.pair_rf[gs];
    }
    invr = R(1) / r;
    const int kn = db.pair_knot[gs];
    const int kphi = (kn & 0xff) - 1, krho = ((kn >> 8) & 0xff) - 1, kf = ((kn >> 16) & 0xff) - 1;
    const int tj = db.atom_type[db.pair_nbr[gs]];
    const int pij = (ti <= tj) ? ti * pot.ntypes + tj - (ti * (ti + 1)) / 2 : tj * pot.ntypes + ti - (tj * (tj + 1)) / 2;
    if (kphi >= 0) {
      const SplineGeom &g = sg[pot.s_phi + pij];
      const R b = sizeof(R) == 8 ? (R)db.pair_shift[gs] : (R)db.pair_shiftf[gs];
      R gr;
      const R v = spl_val_grad<R>(tab + g.toff, tab + g.toff + g.n, kphi, b, (R)(g.step / 6.0),
                                  (R)(g.step * g.step / 6.0), (R)g.invstep, gr);
      e_half = 0.5 * (double)v;
      phig = R(0.5) * gr;
    }
    if (krho >= 0) {
      const SplineGeom &g = sg[pot.s_rho + tj];
      const R b = sizeof(R) == 8 ? (R)db.pair_shift[Np + gs] : (R)db.pair_shiftf[Np + gs];
      R gr;
      const R v = spl_val_grad<R>(tab + g.toff, tab + g.toff + g.n, krho, b, (R)(g.step / 6.0),
                                  (R)(g.step * g.step / 6.0), (R)g.invstep, gr);
      rho_p = (double)v;
      drho = gr;
    }
    if (MEAM && kf >= 0) {
      const SplineGeom &g = sg[pot.s_f + pij];
      const R b = sizeof(R) == 8 ? (R)db.pair_shift[2 * Np + gs] : (R)db.pair_shiftf[2 * Np + gs];
      R gr;
      fv = spl_val_grad<R>(tab + g.toff, tab + g.toff + g.n, kf, b, (R)(g.step / 6.0),
                           (R)(g.step * g.step / 6.0), (R)g.invstep, gr);
      dfv = gr;
    }
    sx[tid] = ux; sy[tid] = uy; sz[tid] = uz; sf[tid] = fv; sdf[tid] = dfv;
  }
  __syncthreads();

  // ---- density phase: rho_i = sum_j rho(r_ij) + sum_{j<k} f_ij f_ik g(cos)
  //      (pot_meam_spline.cpp:177-206).  Each slot p sums f_k g(cos_pk) over
  //      the other slots of its row; every triplet is seen twice, hence 1/2.
  const int row_lo = have ? a_lo[me] : 0, row_hi = have ? a_lo[me + 1] : 0;
  SplineGeom gg;
  if (MEAM) gg = sg[pot.s_g + ti];
  if (MEAM && have && fv != R(0)) {
    const R *gy = tab + gg.toff, *gypp = gy + gg.n;
    const R gx0 = (R)gg.x0, ginv = (R)gg.invstep, gsq6 = (R)(gg.step * gg.step / 6.0);
    const R gcut = (R)gg.cut;
    double acc = 0.0;
    for (int k = row_lo; k < row_hi; ++k) {
      if (k == tid) continue;
      const R fk = sf[k];
      const R cs = cos_exact(ux, uy, uz, sx[k], sy[k], sz[k]);
      if (!(cs < gcut)) continue;  // g_knot == -1: not a triplet (triplet_meam_spline.cpp:66-70)
      R b;
      const int kk = g_knot<R>(cs, gx0, ginv, gg.n, b);
      acc += (double)(fk * spl_val<R>(gy, gypp, kk, b, gsq6));
    }
    rho_p += 0.5 * (double)fv * acc;
  }
  if (have) red[tid] = rho_p;
  __syncthreads();

  // ---- embedding (pot_meam_spline.cpp:208-223): one thread per atom
  if (tid < na) {
    const int ia = atom_lo + tid;
    double rho = 0.0;
    for (int s = a_lo[tid]; s < a_lo[tid + 1]; ++s) rho += red[s];
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
    double dF;
    const double U = spl_point(tc, gU, rho, &dF);  // FP64 table of this candidate
    a_dF[tid] = dF;
    a_U[tid] = U;
    double *ao = aout + (size_t)cand * AO_COUNT * N;
    ao[AO_PEN * N + ia] = pen;
    ao[AO_RHO * N + ia] = rho_raw;
  }
  __syncthreads();

  // ---- force phase (pot_meam_spline.cpp:226-269).  V_p is the force the
  //      atom's terms add to atom i along slot p; the neighbour gets -V_p.
  double Vx = 0, Vy = 0, Vz = 0;
  if (have) {
    const double dF = a_dF[me];
    const double c0 = (double)phig + (double)drho * dF;  // pair and embedding terms
    Vx = (double)ux * c0; Vy = (double)uy * c0; Vz = (double)uz * c0;
    if (MEAM && (fv != R(0) || dfv != R(0))) {
      const R *gy = tab + gg.toff, *gypp = gy + gg.n;
      const R gx0 = (R)gg.x0, ginv = (R)gg.invstep, g6 = (R)(gg.step / 6.0),
              gsq6 = (R)(gg.step * gg.step / 6.0);
      const R gcut = (R)gg.cut;
      double sa = 0, sb = 0, vkx = 0, vky = 0, vkz = 0;
      for (int k = row_lo; k < row_hi; ++k) {
        if (k == tid) continue;
        const R fk = sf[k];
        if (fk == R(0)) continue;
        const R kx = sx[k], ky = sy[k], kz = sz[k];
        const R cs = cos_exact(ux, uy, uz, kx, ky, kz);
        if (!(cs < gcut)) continue;
        R b;
        const int kk = g_knot<R>(cs, gx0, ginv, gg.n, b);
        R dg;
        const R gv = spl_val_grad<R>(gy, gypp, kk, b, g6, gsq6, ginv, dg);
        const R gfk = gv * fk, dgfk = dg * fk;
        sa += (double)gfk;
        sb += (double)(dgfk * cs);
        vkx += (double)(dgfk * kx);
        vky += (double)(dgfk * ky);
        vkz += (double)(dgfk * kz);
      }
      // dfj = u_p (g f'_p f_k - g' f_p f_k cos / r_p) dF + u_k g' f_p f_k dF / r_p
      const double fp = (double)fv, dfp = (double)dfv, ip = (double)invr;
      const double cu = dF * (dfp * sa - fp * ip * sb);
      const double ck = dF * fp * ip;
      Vx += (double)ux * cu + ck * vkx;
      Vy += (double)uy * cu + ck * vky;
      Vz += (double)uz * cu + ck * vkz;
    }
    double *Vc = Vout + (size_t)cand * 3 * Np;
    Vc[gs] = Vx;
    Vc[Np + gs] = Vy;
    Vc[2 * Np + gs] = Vz;
    // stress contribution of slot p: -(u (x) V r), components xx yy zz xy yz zx
    // (stress.h:134-137; pot_meam_spline.cpp:171-173, 234-236, 265-268)
    const double rr = db.pair_r[gs];
    const double dx = db.pair_ux[gs], dy = db.pair_uy[gs], dz = db.pair_uz[gs];
    red[0 * BLOCK_SLOTS + tid] = Vx;
    red[1 * BLOCK_SLOTS + tid] = Vy;
    red[2 * BLOCK_SLOTS + tid] = Vz;
    red[3 * BLOCK_SLOTS + tid] = e_half;
    red[4 * BLOCK_SLOTS + tid] = -(dx * (Vx * rr));
    red[5 * BLOCK_SLOTS + tid] = -(dy * (Vy * rr));
    red[6 * BLOCK_SLOTS + tid] = -(dz * (Vz * rr));
    red[7 * BLOCK_SLOTS + tid] = -(dx * (Vy * rr));
    red[8 * BLOCK_SLOTS + tid] = -(dy * (Vz * rr));
    red[9 * BLOCK_SLOTS + tid] = -(dz * (Vx * rr));
  }
  __syncthreads();
  if (tid < na) {
    const int ia = atom_lo + tid;
    double acc[10];
#pragma unroll
    for (int q = 0; q < 10; ++q) acc[q] = 0.0;
    for (int s = a_lo[tid]; s < a_lo[tid + 1]; ++s) {
#pragma unroll
      for (int q = 0; q < 10; ++q) acc[q] += red[q * BLOCK_SLOTS + s];
    }
    double *ao = aout + (size_t)cand * AO_COUNT * N;
    ao[AO_AX * N + ia] = acc[0];
    ao[AO_AY * N + ia] = acc[1];
    ao[AO_AZ * N + ia] = acc[2];
    ao[AO_E * N + ia] = acc[3] + a_U[tid];
#pragma unroll
    for (int q = 0; q < 6; ++q) ao[(AO_S0 + q) * N + ia] = acc[4 + q];
  }
}

// ------------------------------------------------------------- k_gather

// F_i = sum of V over the atom's own slots - sum of V over the slots whose
// neighbour is i; then the force residual w (F - F0) (potential.cpp:468-478).
__global__ void k_gather(DevDb db, const double *__restrict__ V, double *__restrict__ aout,
                         double *__restrict__ forces, double *__restrict__ errvec, int esize) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  const int N = db.natoms;
  if (i >= N) return;
  const int64_t Np = db.npairs;
  double *ao = aout + (size_t)c * AO_COUNT * N;
  const double *Vc = V + (size_t)c * 3 * Np;
  double fx = ao[AO_AX * N + i], fy = ao[AO_AY * N + i], fz = ao[AO_AZ * N + i];
  for (int q = db.in_off[i]; q < db.in_off[i + 1]; ++q) {
    const int s = db.in_slot[q];
    fx -= Vc[s];
    fy -= Vc[Np + s];
    fz -= Vc[2 * Np + s];
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
}

// -------------------------------------------------------------- k_cells

// One warp per cell (potential.cpp:450-485).
__global__ void k_cells(DevDb db, DevPot pot, const double *__restrict__ aout, double *__restrict__ cellobj,
                        double *__restrict__ errvec, int esize, double *__restrict__ energy,
                        double *__restrict__ stress) {
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
    const double eE = w * db.cell_ew[cell] * pot.energy_weight * na * (E - db.cell_e0[cell]);
    double sum = eE * eE;
    double eS[6], sig[6];
    for (int q = 0; q < 6; ++q) {
      sig[q] = v[1 + q] / db.cell_vol[cell];
      eS[q] = w * db.cell_sw[cell] * pot.stress_weight * (sig[q] - db.cell_s0[6 * cell + q]);
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
      errvec[(size_t)c * esize + 7 * db.ncells + 3 * N + cell] = cons;
    }
    if (energy) energy[(size_t)c * db.ncells + cell] = E;
    if (stress)
      for (int q = 0; q < 6; ++q) stress[((size_t)c * db.ncells + cell) * 6 + q] = sig[q];
  }
}

// -------------------------------------------------------------- k_final

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
    if (pot.style == MZ_STYLE_MEAM_SPLINE) {
      // f-potential magnitude punishment (pot_meam_spline.cpp:274-278):
      // signed largest-|y| knot over the f splines (spline.cpp:58-67,
      // pot_fns.cpp:223-234).
      double my = 0.0;
      const int nf = pot.ntypes * (pot.ntypes + 1) / 2;
      for (int f = 0; f < nf; ++f) {
        const SplineGeom &g = geom[pot.s_f + f];
        double sm = 0.0;
        for (int k = 0; k < g.n; ++k) {
          double y = tab[g.toff + k];
          if (fabs(sm) < fabs(y)) sm = y;
        }
        if (fabs(my) < fabs(sm)) my = sm;
      }
      const double m = fabs(my);
      const double fe = 100. * 25. * (1.0 - m) * (1.0 - m);
      total += fe * fe;
      if (ev) ev[0] = fe;
    } else {
      // U'(mid-range) punishment per type (pot_eam_spline.cpp:211-218)
      for (int ty = 0; ty < pot.ntypes; ++ty) {
        const SplineGeom &g = geom[pot.s_U + ty];
        double gr;
        spl_point(tab, g, 0.5 * (g.x0 + g.xN), &gr);
        const double e = 100. * gr;
        total += e * e;
        if (ev) ev[ty] = e;
      }
    }
    obj[c] = total;
  }
}

}  // namespace mzb

// ================================================================= context

using namespace mzb;

struct mz_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  DevDb db{};
  DevPot pot{};
  int P = 0, nsplines = 0, stride = 0, esize = 0, npen = 0;
  int max_cand = 1, cand_cap = 1;
  int natoms = 0, ncells = 0;
  int64_t npairs = 0;
  int64_t launches = 0;
  std::vector<void *> allocs;
  SplineGeom *d_geom = nullptr;
  double *d_base = nullptr;
  int *d_cmap = nullptr, *d_nat = nullptr;
  double *d_params = nullptr, *d_tabs = nullptr, *d_V = nullptr, *d_aout = nullptr;
  double *d_forces = nullptr, *d_cellobj = nullptr, *d_obj = nullptr, *d_errvec = nullptr;
  double *d_energy = nullptr, *d_stress = nullptr;
  size_t smem64 = 0, smem32 = 0;
};

namespace {

struct CudaFail {
  std::string msg;
};

void ck(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw Failure{MZ_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

template <class T>
T *dalloc(mz_ctx *ctx, size_t n) {
  void *p = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc(&p, n * sizeof(T));
  if (e != cudaSuccess)
    throw Failure{MZ_ERR_NOMEM, std::string("device allocation of ") + std::to_string(n * sizeof(T)) +
                                    " bytes failed: " + cudaGetErrorString(e)};
  ctx->allocs.push_back(p);
  return static_cast<T *>(p);
}

template <class T>
T *dupload(mz_ctx *ctx, const T *h, size_t n) {
  T *d = dalloc<T>(ctx, n);
  if (n) ck(cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy H2D");
  return d;
}

template <class F>
mz_status guarded(F &&f) {
  try {
    f();
    set_error("");
    return MZ_OK;
  } catch (const Failure &e) {
    set_error(e.msg);
    return e.status;
  } catch (const std::bad_alloc &) {
    set_error("host allocation failed");
    return MZ_ERR_NOMEM;
  } catch (const std::exception &e) {
    set_error(e.what());
    return MZ_ERR_ARG;
  }
}

void release(mz_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (void *p : ctx->allocs) cudaFree(p);
  ctx->allocs.clear();
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  ctx->stream = nullptr;
}

// Enqueue one objective evaluation of n candidates whose coefficient
// vectors are already on the device.
void enqueue_objective(mz_ctx *ctx, int n, const double *d_params, int precision, double *d_obj,
                       double *d_errvec, double *d_forces, double *d_energy, double *d_stress) {
  cudaStream_t st = ctx->stream;
  k_prep<<<n, std::max(32, ((ctx->nsplines + 31) / 32) * 32), 0, st>>>(
      n, ctx->P, d_params, ctx->d_base, ctx->d_cmap, ctx->d_geom, ctx->d_nat, ctx->nsplines, ctx->stride,
      ctx->d_tabs);
  ck(cudaGetLastError(), "k_prep launch");
  dim3 ga(ctx->db.nblocks, n);
  const bool meam = ctx->pot.style == MZ_STYLE_MEAM_SPLINE;
  if (precision == MZ_MIXED) {
    if (meam)
      k_atoms<true, float><<<ga, BLOCK_SLOTS, ctx->smem32, st>>>(ctx->db, ctx->pot, ctx->d_geom, ctx->d_tabs,
                                                                  ctx->d_V, ctx->d_aout);
    else
      k_atoms<false, float><<<ga, BLOCK_SLOTS, ctx->smem32, st>>>(ctx->db, ctx->pot, ctx->d_geom, ctx->d_tabs,
                                                                   ctx->d_V, ctx->d_aout);
  } else {
    if (meam)
      k_atoms<true, double><<<ga, BLOCK_SLOTS, ctx->smem64, st>>>(ctx->db, ctx->pot, ctx->d_geom, ctx->d_tabs,
                                                                   ctx->d_V, ctx->d_aout);
    else
      k_atoms<false, double><<<ga, BLOCK_SLOTS, ctx->smem64, st>>>(ctx->db, ctx->pot, ctx->d_geom, ctx->d_tabs,
                                                                    ctx->d_V, ctx->d_aout);
  }
  ck(cudaGetLastError(), "k_atoms launch");
  dim3 gg((ctx->natoms + 255) / 256, n);
  k_gather<<<gg, 256, 0, st>>>(ctx->db, ctx->d_V, ctx->d_aout, d_forces, d_errvec, ctx->esize);
  ck(cudaGetLastError(), "k_gather launch");
  dim3 gc((ctx->ncells + 7) / 8, n);
  k_cells<<<gc, 256, 0, st>>>(ctx->db, ctx->pot, ctx->d_aout, ctx->d_cellobj, d_errvec, ctx->esize, d_energy,
                              d_stress);
  ck(cudaGetLastError(), "k_cells launch");
  k_final<<<n, 256, 0, st>>>(ctx->db, ctx->pot, ctx->d_geom, ctx->d_tabs, ctx->d_cellobj, d_obj, d_errvec,
                             ctx->esize);
  ck(cudaGetLastError(), "k_final launch");
  ctx->launches += 5;
}

}  // namespace

extern "C" {

mz_status mz_create(const mz_db *dbh, const mz_pot *poth, const mz_settings *set, mz_ctx **out) {
  mz_ctx *ctx = nullptr;
  mz_status st = guarded([&] {
    if (!dbh || !poth || !set || !out) throw Failure{MZ_ERR_ARG, "null argument"};
    const Db &db = dbh->db;
    const Pot &pot = poth->pot;
    if (db.npairs >= (int64_t(1) << 31)) throw Failure{MZ_ERR_RANGE, "more than 2^31 pairs"};
    if (db.max_row > BLOCK_SLOTS)
      throw Failure{MZ_ERR_RANGE, "neighbour row of " + std::to_string(db.max_row) + " pairs exceeds the kernel limit of " +
                                      std::to_string(BLOCK_SLOTS)};
    if (pot.nsplines() > MAX_SPLINES) throw Failure{MZ_ERR_RANGE, "too many splines"};
    ctx = new mz_ctx;
    ctx->device = set->device;
    ck(cudaSetDevice(ctx->device), "cudaSetDevice");
    ck(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    ctx->natoms = db.natoms;
    ctx->ncells = db.ncells;
    ctx->npairs = db.npairs;
    ctx->max_cand = std::max(1, set->max_candidates);

    // ---- potential structure
    const int ns = pot.nsplines();
    std::vector<SplineGeom> geom(ns);
    std::vector<int> nat(2 * ns);
    int toff = 0;
    for (int s = 0; s < ns; ++s) {
      const Spline3 &sp = pot.spline(s);
      SplineGeom &g = geom[s];
      g.x0 = sp.x[0];
      g.xN = sp.x[sp.nknots - 1];
      g.step = sp.step;
      g.invstep = sp.invstep;
      g.cut = sp.x.back() * (1. + 1.e-8);
      g.n = sp.nknots;
      g.toff = toff;
      toff += 2 * sp.nknots + 2;
      nat[2 * s] = sp.nat[0];
      nat[2 * s + 1] = sp.nat[1];
    }
    const int stride = toff;
    std::vector<double> base(stride, 0.0);
    std::vector<int> cmap(stride, -1);
    int ci = 0;
    for (int s = 0; s < ns; ++s) {
      const Spline3 &sp = pot.spline(s);
      const int o = geom[s].toff, n = sp.nknots;
      for (int k = 0; k < n; ++k) {
        base[o + k] = sp.y[k];
        if (!sp.y_fixed[k]) cmap[o + k] = ci++;
      }
      for (int e = 0; e < 2; ++e) {
        base[o + 2 * n + e] = sp.grad[e];
        if (!sp.grad_fixed[e] && !sp.nat[e]) cmap[o + 2 * n + e] = ci++;
      }
    }
    ctx->P = ci;
    ctx->nsplines = ns;
    ctx->stride = stride;
    ctx->d_geom = dupload(ctx, geom.data(), ns);
    ctx->d_nat = dupload(ctx, nat.data(), nat.size());
    ctx->d_base = dupload(ctx, base.data(), base.size());
    ctx->d_cmap = dupload(ctx, cmap.data(), cmap.size());
    DevPot &dp = ctx->pot;
    dp.style = pot.style;
    dp.ntypes = pot.ntypes;
    dp.nsplines = ns;
    dp.tab_stride = stride;
    dp.s_phi = pot.spline_index(G_PHI, 0);
    dp.s_rho = pot.spline_index(G_RHO, 0);
    dp.s_U = pot.spline_index(G_U, 0);
    dp.s_f = pot.style == MZ_STYLE_MEAM_SPLINE ? pot.spline_index(G_F, 0) : 0;
    dp.s_g = pot.style == MZ_STYLE_MEAM_SPLINE ? pot.spline_index(G_G, 0) : 0;
    dp.embed_extrap = set->embed_extrap;
    dp.energy_weight = set->energy_weight;
    dp.stress_weight = set->stress_weight;
    ctx->npen = pot.style == MZ_STYLE_MEAM_SPLINE ? 1 : pot.ntypes;
    ctx->esize = 8 * db.ncells + 3 * db.natoms + ctx->npen;

    // ---- database
    const int N = db.natoms;
    const int64_t Np = db.npairs;
    DevDb &d = ctx->db;
    d.ncells = db.ncells;
    d.natoms = N;
    d.npairs = Np;
    d.cell_atom0 = dupload(ctx, db.cell_atom0.data(), db.cell_atom0.size());
    d.cell_vol = dupload(ctx, db.cell_vol.data(), db.cell_vol.size());
    d.cell_w = dupload(ctx, db.cell_weight.data(), db.cell_weight.size());
    d.cell_ew = dupload(ctx, db.cell_eweight.data(), db.cell_eweight.size());
    d.cell_sw = dupload(ctx, db.cell_sweight.data(), db.cell_sweight.size());
    d.cell_e0 = dupload(ctx, db.cell_energy0.data(), db.cell_energy0.size());
    d.cell_s0 = dupload(ctx, db.cell_stress0.data(), db.cell_stress0.size());
    d.atom_type = dupload(ctx, db.atom_type.data(), db.atom_type.size());
    d.atom_cell = dupload(ctx, db.atom_cell.data(), db.atom_cell.size());
    d.force0 = dupload(ctx, db.atom_force0.data(), db.atom_force0.size());
    std::vector<int> off32(N + 1), inoff32(N + 1), inslot32(Np), knot32(Np);
    for (int i = 0; i <= N; ++i) {
      off32[i] = (int)db.pair_off[i];
      inoff32[i] = (int)db.in_off[i];
    }
    for (int64_t s = 0; s < Np; ++s) {
      inslot32[s] = (int)db.in_slot[s];
      knot32[s] = (db.pair_knot[3 * s] + 1) | ((db.pair_knot[3 * s + 1] + 1) << 8) |
                  ((db.pair_knot[3 * s + 2] + 1) << 16);
    }
    d.pair_off = dupload(ctx, off32.data(), off32.size());
    d.in_off = dupload(ctx, inoff32.data(), inoff32.size());
    d.in_slot = dupload(ctx, inslot32.data(), inslot32.size());
    d.pair_knot = dupload(ctx, knot32.data(), knot32.size());
    d.pair_nbr = dupload(ctx, db.pair_nbr.data(), db.pair_nbr.size());
    {
      std::vector<double> ux(Np), uy(Np), uz(Np), sh(3 * Np);
      std::vector<float> rf(Np), uxf(Np), uyf(Np), uzf(Np), shf(3 * Np);
      for (int64_t s = 0; s < Np; ++s) {
        ux[s] = db.pair_u[3 * s];
        uy[s] = db.pair_u[3 * s + 1];
        uz[s] = db.pair_u[3 * s + 2];
        rf[s] = (float)db.pair_r[s];
        uxf[s] = (float)ux[s];
        uyf[s] = (float)uy[s];
        uzf[s] = (float)uz[s];
        for (int q = 0; q < 3; ++q) {
          sh[q * Np + s] = db.pair_shift[3 * s + q];
          shf[q * Np + s] = (float)db.pair_shift[3 * s + q];
        }
      }
      d.pair_r = dupload(ctx, db.pair_r.data(), Np);
      d.pair_ux = dupload(ctx, ux.data(), Np);
      d.pair_uy = dupload(ctx, uy.data(), Np);
      d.pair_uz = dupload(ctx, uz.data(), Np);
      d.pair_shift = dupload(ctx, sh.data(), 3 * Np);
      d.pair_rf = dupload(ctx, rf.data(), Np);
      d.pair_uxf = dupload(ctx, uxf.data(), Np);
      d.pair_uyf = dupload(ctx, uyf.data(), Np);
      d.pair_uzf = dupload(ctx, uzf.data(), Np);
      d.pair_shiftf = dupload(ctx, shf.data(), 3 * Np);
    }
    // atom blocks: consecutive atoms, <= BLOCK_SLOTS slots and <= BLOCK_ATOMS atoms
    std::vector<int> blk(1, 0);
    {
      int slots = 0, atoms = 0;
      for (int i = 0; i < N; ++i) {
        const int n = (int)(db.pair_off[i + 1] - db.pair_off[i]);
        if (atoms > 0 && (slots + n > BLOCK_SLOTS || atoms + 1 > BLOCK_ATOMS)) {
          blk.push_back(i);
          slots = 0;
          atoms = 0;
        }
        slots += n;
        atoms += 1;
      }
      blk.push_back(N);
    }
    d.nblocks = (int)blk.size() - 1;
    d.blk_atom0 = dupload(ctx, blk.data(), blk.size());

    // ---- work buffers: candidates per launch bounded by device memory
    size_t freeb = 0, totalb = 0;
    ck(cudaMemGetInfo(&freeb, &totalb), "cudaMemGetInfo");
    const size_t per_cand = sizeof(double) * ((size_t)3 * Np + (size_t)AO_COUNT * N + (size_t)3 * N +
                                              (size_t)ctx->esize + (size_t)7 * db.ncells + stride + ctx->P + 1);
    size_t budget = (size_t)(0.6 * (double)freeb);
    int cap = (int)std::max<size_t>(1, budget / std::max<size_t>(per_cand, 1));
    ctx->cand_cap = std::min(ctx->max_cand, cap);
    const size_t C = ctx->cand_cap;
    ctx->d_params = dalloc<double>(ctx, C * ctx->P);
    ctx->d_tabs = dalloc<double>(ctx, C * stride);
    ctx->d_V = dalloc<double>(ctx, C * 3 * Np);
    ctx->d_aout = dalloc<double>(ctx, C * AO_COUNT * N);
    ctx->d_forces = dalloc<double>(ctx, C * 3 * N);
    ctx->d_cellobj = dalloc<double>(ctx, C * db.ncells);
    ctx->d_obj = dalloc<double>(ctx, C);
    ctx->d_errvec = dalloc<double>(ctx, C * ctx->esize);
    ctx->d_energy = dalloc<double>(ctx, C * db.ncells);
    ctx->d_stress = dalloc<double>(ctx, C * 6 * db.ncells);
    ctx->smem64 = atoms_smem_bytes<double>(ns, stride);
    ctx->smem32 = atoms_smem_bytes<float>(ns, stride);
    ck(cudaFuncSetAttribute(k_atoms<true, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ctx->smem64),
       "smem attr");
    ck(cudaFuncSetAttribute(k_atoms<false, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ctx->smem64),
       "smem attr");
    ck(cudaFuncSetAttribute(k_atoms<true, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ctx->smem32),
       "smem attr");
    ck(cudaFuncSetAttribute(k_atoms<false, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ctx->smem32),
       "smem attr");
    *out = ctx;
  });
  if (st != MZ_OK && ctx) {
    release(ctx);
    delete ctx;
  }
  return st;
}

void mz_destroy(mz_ctx *ctx) {
  if (!ctx) return;
  release(ctx);
  delete ctx;
}

mz_status mz_objective(mz_ctx *ctx, int ncand, const double *params, int precision, double *obj, double *errvec,
                       double *forces, double *energy, double *stress) {
  return guarded([&] {
    if (!ctx || !params || !obj || ncand <= 0) throw Failure{MZ_ERR_ARG, "bad argument"};
    if (precision != MZ_FP64 && precision != MZ_MIXED) throw Failure{MZ_ERR_ARG, "unknown precision"};
    ck(cudaSetDevice(ctx->device), "cudaSetDevice");
    const int P = ctx->P, E = ctx->esize, N = ctx->natoms, NC = ctx->ncells;
    for (int c0 = 0; c0 < ncand; c0 += ctx->cand_cap) {
      const int n = std::min(ctx->cand_cap, ncand - c0);
      ck(cudaMemcpyAsync(ctx->d_params, params + (size_t)c0 * P, sizeof(double) * n * P, cudaMemcpyHostToDevice,
                         ctx->stream),
         "params H2D");
      enqueue_objective(ctx, n, ctx->d_params, precision, ctx->d_obj, errvec ? ctx->d_errvec : nullptr,
                        forces ? ctx->d_forces : nullptr, energy ? ctx->d_energy : nullptr,
                        stress ? ctx->d_stress : nullptr);
      ck(cudaMemcpyAsync(obj + c0, ctx->d_obj, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream), "obj D2H");
      if (errvec)
        ck(cudaMemcpyAsync(errvec + (size_t)c0 * E, ctx->d_errvec, sizeof(double) * n * E, cudaMemcpyDeviceToHost,
                           ctx->stream),
           "errvec D2H");
      if (forces)
        ck(cudaMemcpyAsync(forces + (size_t)c0 * 3 * N, ctx->d_forces, sizeof(double) * n * 3 * N,
                           cudaMemcpyDeviceToHost, ctx->stream),
           "forces D2H");
      if (energy)
        ck(cudaMemcpyAsync(energy + (size_t)c0 * NC, ctx->d_energy, sizeof(double) * n * NC, cudaMemcpyDeviceToHost,
                           ctx->stream),
           "energy D2H");
      if (stress)
        ck(cudaMemcpyAsync(stress + (size_t)c0 * 6 * NC, ctx->d_stress, sizeof(double) * n * 6 * NC,
                           cudaMemcpyDeviceToHost, ctx->stream),
           "stress D2H");
      ck(cudaStreamSynchronize(ctx->stream), "objective");
    }
  });
}

mz_status mz_objective_device(mz_ctx *ctx, int ncand, const double *d_params, int precision, double *d_obj,
                              double *d_errvec, double *d_forces) {
  return guarded([&] {
    if (!ctx || !d_params || !d_obj || ncand <= 0) throw Failure{MZ_ERR_ARG, "bad argument"};
    if (ncand > ctx->cand_cap)
      throw Failure{MZ_ERR_RANGE, "ncand exceeds the candidates one launch can hold (" + std::to_string(ctx->cand_cap) + ")"};
    if (precision != MZ_FP64 && precision != MZ_MIXED) throw Failure{MZ_ERR_ARG, "unknown precision"};
    ck(cudaSetDevice(ctx->device), "cudaSetDevice");
    enqueue_objective(ctx, ncand, d_params, precision, d_obj, d_errvec, d_forces, nullptr, nullptr);
  });
}

mz_status mz_objective_grad(mz_ctx *ctx, int ncand, const double *params, int precision, double *obj, double *grad) {
  return guarded([&] { throw Failure{MZ_ERR_UNSUPPORTED, "gradient not built yet"}; });
}

mz_status mz_objective_grad_device(mz_ctx *ctx, int ncand, const double *d_params, int precision, double *d_obj,
                                   double *d_grad) {
  return guarded([&] { throw Failure{MZ_ERR_UNSUPPORTED, "gradient not built yet"}; });
}

mz_status mz_densities(mz_ctx *ctx, const double *params, double *dens) {
  return guarded([&] {
    if (!ctx || !params || !dens) throw Failure{MZ_ERR_ARG, "bad argument"};
    ck(cudaSetDevice(ctx->device), "cudaSetDevice");
    ck(cudaMemcpyAsync(ctx->d_params, params, sizeof(double) * ctx->P, cudaMemcpyHostToDevice, ctx->stream),
       "params H2D");
    enqueue_objective(ctx, 1, ctx->d_params, MZ_FP64, ctx->d_obj, nullptr, nullptr, nullptr, nullptr);
    ck(cudaMemcpyAsync(dens, ctx->d_aout + (size_t)AO_RHO * ctx->natoms, sizeof(double) * ctx->natoms,
                       cudaMemcpyDeviceToHost, ctx->stream),
       "dens D2H");
    ck(cudaStreamSynchronize(ctx->stream), "densities");
  });
}

mz_status mz_sync(mz_ctx *ctx) {
  return guarded([&] {
    if (!ctx) throw Failure{MZ_ERR_ARG, "null context"};
    ck(cudaStreamSynchronize(ctx->stream), "sync");
  });
}

void *mz_stream(mz_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

mz_status mz_launch_count(const mz_ctx *ctx, int64_t *launches) {
  return guarded([&] {
    if (!ctx || !launches) throw Failure{MZ_ERR_ARG, "null argument"};
    *launches = ctx->launches;
  });
}

}  // extern "C"
