// Adjoint of the objective with respect to every knot value and end slope.
//
// The objective is F = sum of squared residuals.  With the residuals'
// sensitivities frozen as seeds -- lambda_i = dF/dF_i (k_gather),
// eps_c = dF/dE_atom, mu_c = dF/dS_c, kappa_c = dF/dpen (k_cells) -- the
// gradient is that of
//   L = sum_i [eps E_i + kappa pen(rho_i)] + sum_p Lambda_p . V_p
// with Lambda_p = lambda_i - lambda_nbr(p) + m_p(mu_c)  (the force gather and
// the slot's stress term transposed).  Per atom, with a_p = Lambda_p . u_p,
//   Lambda_p . V_p = a_p phi'_p/2 + U'(rho) k_p,
//   k_p = a_p rho'_p + a_p f'_p G_p - a_p f_p H_p / r_p + f_p J_p / r_p,
//   J_p = Lambda_p . vk_p,   K_i = sum_p k_p,
// so one more pass over each row (for d K / d f and the g table) is all the
// adjoint needs; G, H and vk come from the forward pass.  Densities and
// embedding derivatives are recomputed, nothing per triplet is stored.
// JMEAM's terms sum p_j p_k q(cos) enter E_i directly and V_p without U':
// each is the g channel with (chi, U', f, g) replaced by (eps, 1, p, q) and
// runs as one more pass over the row with the same shared-memory rows.
#pragma once

#include <type_traits>

#include "mz_fwd.cuh"
#include "mz_fwd2.cuh"

namespace mzb {

// g-table gradient of one knot interval in the cubic's power basis:
// dc_q accumulates dF/dc_q of S(b) = c0 + c1 b + c2 b^2 + c3 b^3.  Its map to
// the knot table follows from c0 = y_m, c1 = y_m+1 - y_m - (2 y''_m + y''_m+1) H,
// c2 = 3 y''_m H, c3 = (y''_m+1 - y''_m) H with H = h^2/6.
template <class Add>
__device__ __forceinline__ void power_to_table(const SplineGeom &g, int m, double d0, double d1, double d2,
                                               double d3, Add add) {
  const double H = g.step * g.step / 6.0;
  add(m, d0 - d1);
  add(m + 1, d1);
  add(g.n + m, -2.0 * H * d1 + 3.0 * H * d2 - H * d3);
  add(g.n + m + 1, -H * d1 + H * d3);
}

// spline5eq: the same for the quintic's six power coefficients, from
// c0 = y_m, c1 = y_m+1 - y_m + H2 (-2 y''_m - y''_m+1) + H4 (8 y4_m + 7 y4_m+1),
// c2 = 3 H2 y''_m, c3 = H2 (y''_m+1 - y''_m) + H4 (-20 y4_m - 10 y4_m+1),
// c4 = 15 H4 y4_m, c5 = 3 H4 (y4_m+1 - y4_m), H2 = h^2/6, H4 = h^4/360.
template <class Add>
__device__ __forceinline__ void power_to_table5(const SplineGeom &g, int m, const double *d, Add add) {
  const double H2 = g.step * g.step / 6.0, H4 = g.step * g.step * g.step * g.step / 360.0;
  add(m, d[0] - d[1]);
  add(m + 1, d[1]);
  add(g.n + m, H2 * (-2.0 * d[1] + 3.0 * d[2] - d[3]));
  add(g.n + m + 1, H2 * (-d[1] + d[3]));
  add(2 * g.n + 2 + m, H4 * (8.0 * d[1] - 20.0 * d[3] + 15.0 * d[4] - 3.0 * d[5]));
  add(2 * g.n + 3 + m, H4 * (7.0 * d[1] - 10.0 * d[3] + 3.0 * d[5]));
}

constexpr int GACC_FLUSH_BLOCKS = 32;  // atom blocks between flushes of the per-thread g tables
// atom blocks between flushes of the per-warp FP32 tables into FP64 (mixed
// precision; the FP64 kernels flush after every block)
constexpr int FT_FLUSH_BLOCKS = 8;
// The adjoint walks type-pure atom blocks (DevDb::adj_*), so each thread keeps
// one g table (its block's type), flushed when the CTA moves to a block of
// another type and every GACC_FLUSH_BLOCKS blocks.

// Mixed precision: per-warp FP64 table gradients live in global memory, one
// slice per (candidate, CTA, warp) of wglob [ncand][gridDim.x][ADJ_WARPS][stride]
// (lane 0 / distinct lanes write them, and the slices are summed in a fixed
// order); keeping them out of shared memory lets four CTAs share an SM.  The
// pair-function and embedding gradients enter the warp's FP32 shared table
// with shared-memory atomics (the order of same-address additions is not
// fixed, so the mixed gradient can differ run to run at FP32 rounding level).
//
// FP64 (R = double): every table sum is FP64 and in a fixed order.  The
// warp's table is FP64 in shared memory; each of its entries has an owner lane
// (entry mod 32) that adds the warp's contributions in slot order; the
// per-thread g tables are flushed into it after every block; and the blocks of
// each group of db.adj_group consecutive blocks (256-slot partition, the one
// partition the FP64 launches use) are summed into one partial per group, the
// partials in group order.  The gradient is then bit-identical from call to
// call and for any number of CTAs.
// Shared-memory layout of k_adj (dynamic), see adj_smem_bytes():
//   FT     ftab[ADJ_WARPS][stride]          per-warp pair-function gradients (FP32; FP64 for R = double)
//   R4 gacc[gtabs][ng-1][BLOCK_SLOTS]       per-thread g-table gradients, power basis: one table
//                                           (the block's type) for MEAM; one per partner type for
//                                           GMEAM, flushed every block
//   R2 gacc5[gtabs][ng-1][BLOCK_SLOTS]      spline5eq angular splines: the b^4, b^5 coefficients
//   double red[BLOCK_SLOTS], a_chi[BLOCK_ATOMS], a_dF[BLOCK_ATOMS]
//   SplineGeom sg[nsplines]; int a_lo[BLOCK_ATOMS+2], a_idx[BLOCK_ATOMS+2], a_cell[BLOCK_ATOMS+2],
//                            a_na (atom count | type << 8)
//   R ptab[pstride]
//   R4 srow[BLOCK_SLOTS+8]  (u_x, u_y, u_z, f)              of every slot (zero padded)
//   R4 sadj[BLOCK_SLOTS+8]  (a f', a f / r, Q_x, Q_y)        with Q = f Lambda / r
//   R  sqz[BLOCK_SLOTS+8]   Q_z
//   int stype[BLOCK_SLOTS+8] neighbour type of every slot (GMEAM)
template <typename R>
__host__ __device__ inline size_t adj_smem_bytes(int nsplines, int stride, int pstride, bool meam, int gtabs,
                                                 int ng, bool gq5 = false) {
  size_t b = (sizeof(R) == 8 ? sizeof(double) : sizeof(float)) * (size_t)ADJ_WARPS * stride;
  b = (b + 31) & ~size_t(31);
  if (meam) b += (gq5 ? 6 : 4) * sizeof(R) * (size_t)gtabs * (ng - 1) * BLOCK_SLOTS;
  b += sizeof(double) * (BLOCK_SLOTS + 2 * BLOCK_ATOMS);
  b += sizeof(SplineGeom) * nsplines;
  b += sizeof(int) * (3 * BLOCK_ATOMS + 8);
  b = (b + 31) & ~size_t(31);
  b += sizeof(R) * (pstride + 4);
  b = (b + 31) & ~size_t(31);
  b += 9 * sizeof(R) * (BLOCK_SLOTS + 8);
  b += sizeof(int) * (BLOCK_SLOTS + 8);
  return b;
}

// g_knot<float> from t = (c - x0) / h: interval (clamped to [0, nmax]) and shift
__device__ __forceinline__ int knot_of_t(float t, int nmax, float &b) {
  int k = __float_as_int(t + 8388607.5f) - 0x4B000000;
  k = k < 0 ? 0 : (k > nmax ? nmax : k);
  b = t - (__int_as_float(k + 0x4B000000) - 8388608.0f);
  return k;
}

template <bool MEAM, typename R, bool GM = false, bool JM = false, bool Q5 = false>
__global__ void __launch_bounds__(BLOCK_SLOTS, JM || sizeof(R) == 8 ? 2 : (GM || Q5) ? 3 : 4)
    k_adj(DevDb db, DevPot pot, const SplineGeom *__restrict__ geom, const double *__restrict__ tabs,
          const double *__restrict__ ptabs, const double *__restrict__ aout, const double *__restrict__ aux,
          const double *__restrict__ lam, const double *__restrict__ seeds, double *__restrict__ partial,
          double *__restrict__ wglob) {
  using R4 = typename Vec4<R>::T;
  extern __shared__ __align__(32) unsigned char smem_raw[];
  const int cand = blockIdx.y;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
  const int N = db.natoms, NC = db.ncells;
  const int64_t Np = db.npairs;
  const int stride = pot.tab_stride;
  const int ng = MEAM ? pot.g_nmax : 2;  // per-thread tables sized by the largest g spline
  const int nint = ng - 1;
  const int gtabs = GM ? pot.ntypes : 1;

  constexpr bool DET = sizeof(R) == 8;  // FP64: fixed-order FP64 table sums (see above)
  using FT = typename std::conditional<DET, double, float>::type;
  double *wtab = DET ? nullptr : wglob + ((size_t)cand * gridDim.x + blockIdx.x) * ADJ_WARPS * stride;
  FT *ftab = reinterpret_cast<FT *>(smem_raw);
  size_t off = sizeof(FT) * (size_t)ADJ_WARPS * stride;
  off = (off + 31) & ~size_t(31);
  using R2 = typename std::conditional<sizeof(R) == 4, float2, double2>::type;
  R4 *gacc = reinterpret_cast<R4 *>(smem_raw + off);
  if (MEAM) off += 4 * sizeof(R) * (size_t)gtabs * nint * BLOCK_SLOTS;
  R2 *gacc5 = reinterpret_cast<R2 *>(smem_raw + off);
  const bool gq5 = Q5 && pot.g_q5;  // quintic accumulators of the angular splines
  if (MEAM && gq5) off += 2 * sizeof(R) * (size_t)gtabs * nint * BLOCK_SLOTS;
  double *red = reinterpret_cast<double *>(smem_raw + off);
  double *a_chi = red + BLOCK_SLOTS;
  double *a_dF = a_chi + BLOCK_ATOMS;
  SplineGeom *sg = reinterpret_cast<SplineGeom *>(a_dF + BLOCK_ATOMS);
  int *a_lo = reinterpret_cast<int *>(sg + pot.nsplines);
  int *a_idx = a_lo + BLOCK_ATOMS + 2;
  int *a_cell = a_idx + BLOCK_ATOMS + 2;
  int *a_na = a_cell + BLOCK_ATOMS + 2;
  off = reinterpret_cast<unsigned char *>(a_na + 2) - smem_raw;
  off = (off + 31) & ~size_t(31);
  R *ptab = reinterpret_cast<R *>(smem_raw + off);
  off += sizeof(R) * (pot.pow_stride + 4);
  off = (off + 31) & ~size_t(31);
  R4 *srow = reinterpret_cast<R4 *>(smem_raw + off);
  R4 *sadj = srow + BLOCK_SLOTS + 8;
  R *sqz = reinterpret_cast<R *>(sadj + BLOCK_SLOTS + 8);
  int *stype = reinterpret_cast<int *>(sqz + BLOCK_SLOTS + 8);
  // meam/spline, spline3eq, FP32: the rows as pairs of slots (2 p, 2 p + 1),
  // in the same storage -- rowA[p] = (u_x, u_x', u_y, u_y'), rowB[p] =
  // (u_z, u_z', f, f'), adjA[p] = (a f', a f', -a f / r, -a f' / r'),
  // adjB[p] = (Q_x, Q_x', Q_y, Q_y'), qz2[p] = (Q_z, Q_z')
  constexpr bool PK = MEAM && !GM && !JM && !Q5 && sizeof(R) == 4;
  constexpr int HP = (BLOCK_SLOTS + 8) / 2;
  float4 *rowA = reinterpret_cast<float4 *>(srow), *rowB = rowA + HP;
  float4 *adjA = reinterpret_cast<float4 *>(sadj), *adjB = adjA + HP;
  const float2 *qz2 = reinterpret_cast<const float2 *>(sqz);
  auto put_pair_row = [&](int k, float ux, float uy, float uz, float f, float qx, float qy, float qX, float qY,
                          float qZ) {
    float *fa = reinterpret_cast<float *>(rowA), *fb = reinterpret_cast<float *>(rowB);
    float *ga = reinterpret_cast<float *>(adjA), *gb = reinterpret_cast<float *>(adjB);
    const int o = 4 * (k >> 1) + (k & 1);
    fa[o] = ux;
    fa[o + 2] = uy;
    fb[o] = uz;
    fb[o + 2] = f;
    ga[o] = qx;
    ga[o + 2] = -qy;
    gb[o] = qX;
    gb[o + 2] = qY;
    reinterpret_cast<float *>(sqz)[k] = qZ;
  };

  const double *tc = tabs + (size_t)cand * stride;
  const double *pcand = ptabs + (size_t)cand * pot.pow_stride;
  for (int i = tid; i < pot.pow_stride; i += blockDim.x) ptab[i] = (R)pcand[i];
  for (int i = tid; i < ADJ_WARPS * stride; i += blockDim.x) {
    if (!DET) wtab[i] = 0.0;
    ftab[i] = FT(0);
  }
  if (MEAM)
    for (int i = tid; i < gtabs * nint * BLOCK_SLOTS; i += blockDim.x) gacc[i] = R4{};
  if (MEAM && gq5)
    for (int i = tid; i < gtabs * nint * BLOCK_SLOTS; i += blockDim.x) gacc5[i] = R2{};
  for (int i = tid; i < pot.nsplines; i += blockDim.x) sg[i] = geom[i];
  FT *ft = ftab + (size_t)warp * stride;
  double *wt = DET ? reinterpret_cast<double *>(ft) : wtab + (size_t)warp * stride;
  // Table contributions of this thread's slot.  Mixed: FP32 shared atomics.
  // FP64: kept per thread (phi, rho, f and JMEAM's p, p2: four entries each,
  // six for a quintic piece, at most 30) and added by det_flush.
  constexpr int NCONTRIB = DET ? (JM && Q5 ? 30 : 24) : 1;
  int c_idx[NCONTRIB];
  double c_val[NCONTRIB];
  int c_n = 0;
  auto add_f = [&](int idx, double v) {
    if constexpr (DET) {
      c_idx[c_n] = idx;
      c_val[c_n] = v;
      ++c_n;
    } else {
      atomicAdd(ft + idx, (float)v);
    }
  };
  // Every lane of the warp: the contributions of lanes 0..31 in order, each
  // entry added by its owner lane (idx mod 32), so each table entry receives
  // its additions in a fixed order.
  auto det_flush = [&]() {
    if constexpr (DET) {
      __syncwarp();
      for (int src = 0; src < 32; ++src) {
        const int n = __shfl_sync(0xffffffffu, c_n, src);
        for (int e = 0; e < n; ++e) {
          const int idx = __shfl_sync(0xffffffffu, e < c_n ? c_idx[e] : 0, src);
          const double v = __shfl_sync(0xffffffffu, e < c_n ? c_val[e] : 0.0, src);
          if ((idx & 31) == lane) ft[idx] += v;
        }
      }
      c_n = 0;
      __syncwarp();
    }
  };

  const double *ao = aout + (size_t)cand * AO_COUNT * N;
  const double *ax = aux + (size_t)cand * (JM ? pot.aux_rows : (int)AUX_COUNT) * Np;
  const double *L = lam + (size_t)cand * 3 * N;
  const double *sd = seeds + (size_t)cand * CS_COUNT * NC;

  // Flush of the per-thread g table of type t (power basis) into the warp's
  // FP64 table: one warp-wide sum per (interval, coefficient).
  auto flush_gacc_spline = [&](int s) {
    const SplineGeom &gg = sg[s];
    for (int m = 0; m < gg.n - 1; ++m) {
      const R4 v = gacc[m * BLOCK_SLOTS + tid];
      double d[6] = {(double)v.x, (double)v.y, (double)v.z, (double)v.w, 0.0, 0.0};
      if (gq5) {
        const R2 v5 = gacc5[m * BLOCK_SLOTS + tid];
        d[4] = (double)v5.x;
        d[5] = (double)v5.y;
      }
#pragma unroll
      for (int q = 0; q < (Q5 ? 6 : 4); ++q)
        for (int o = 16; o > 0; o >>= 1) d[q] += __shfl_down_sync(0xffffffffu, d[q], o);
      if (lane == 0) {
        if (quintic_of<Q5>(gg)) power_to_table5(gg, m, d, [&](int idx, double x) { wt[gg.toff + idx] += x; });
        else power_to_table(gg, m, d[0], d[1], d[2], d[3], [&](int idx, double x) { wt[gg.toff + idx] += x; });
      }
    }
    for (int m = 0; m < nint; ++m) gacc[m * BLOCK_SLOTS + tid] = R4{};
    if (gq5)
      for (int m = 0; m < nint; ++m) gacc5[m * BLOCK_SLOTS + tid] = R2{};
  };
  auto flush_gacc = [&](int t) { flush_gacc_spline(pot.s_g + t); };
  // GMEAM: this thread's table tk holds triplets (i; j, k) with j its slot's
  // neighbour type (tj_mine) and k of type tk, i.e. g spline (t; tj_mine, tk).
  auto flush_gacc_gm = [&](int t, bool have_t, int tj_mine) {
    for (int v = 0; v < pot.ntypes; ++v)
      for (int tk = 0; tk < pot.ntypes; ++tk) {
        const SplineGeom &g2 = sg[gmeam_g_index(pot, t, v, tk)];
        for (int m = 0; m < g2.n - 1; ++m) {
          R4 val = R4{};
          R2 val5 = R2{};
          if (have_t && tj_mine == v) {
            val = gacc[(tk * nint + m) * BLOCK_SLOTS + tid];
            if (gq5) val5 = gacc5[(tk * nint + m) * BLOCK_SLOTS + tid];
          }
          double d[6] = {(double)val.x, (double)val.y, (double)val.z, (double)val.w, (double)val5.x,
                         (double)val5.y};
#pragma unroll
          for (int q = 0; q < (Q5 ? 6 : 4); ++q)
            for (int o = 16; o > 0; o >>= 1) d[q] += __shfl_down_sync(0xffffffffu, d[q], o);
          if (lane == 0) {
            if (quintic_of<Q5>(g2)) power_to_table5(g2, m, d, [&](int idx, double x) { wt[g2.toff + idx] += x; });
            else power_to_table(g2, m, d[0], d[1], d[2], d[3], [&](int idx, double x) { wt[g2.toff + idx] += x; });
          }
        }
      }
    for (int i = 0; i < gtabs * nint; ++i) gacc[i * BLOCK_SLOTS + tid] = R4{};
    if (gq5)
      for (int i = 0; i < gtabs * nint; ++i) gacc5[i * BLOCK_SLOTS + tid] = R2{};
  };

  // the warp's FP32 sums into its FP64 table (global memory): a lane's loads
  // are all issued before its adds and stores
  auto flush_ft = [&]() {
    __syncwarp();
    for (int e0 = lane; e0 < stride; e0 += 32 * 8) {
      double v[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) v[q] = e0 + 32 * q < stride ? wt[e0 + 32 * q] : 0.0;
#pragma unroll
      for (int q = 0; q < 8; ++q)
        if (e0 + 32 * q < stride) {
          wt[e0 + 32 * q] = v[q] + (double)ft[e0 + 32 * q];
          ft[e0 + 32 * q] = 0.f;
        }
    }
    __syncwarp();
  };

  // Block descriptors (atom, first slot, atom count | type << 8, cell; one more
  // entry holds the slot count) are loaded a block ahead, and the start of the
  // block after that two blocks ahead, so that no global load stands between
  // the barriers of a block's prologue.  Threads past the block's count load
  // entries of the following blocks, which nobody reads.
  const int ndesc = N + db.adj_nblocks, amax = db.adj_amax;
  // Block order of this CTA: blocks blockIdx.x + k gridDim.x (mixed), or the
  // groups blockIdx.x + k gridDim.x of db.adj_group consecutive blocks (FP64).
  const int GB = DET ? max(db.adj_group, 1) : 1;
  const int ngroups = (db.adj_nblocks + GB - 1) / GB;
  auto next_blk = [&](int b) {
    if (!DET) return b + (int)gridDim.x;
    const int nx = b + 1;
    return (nx % GB) ? nx : nx + ((int)gridDim.x - 1) * GB;
  };
  const int first_blk = DET ? (int)blockIdx.x * GB : (int)blockIdx.x;
  int4 dn = make_int4(0, 0, 0, 0);
  int nb = first_blk;
  if (nb < db.adj_nblocks) {
    const int base = db.adj_blk0[nb] + nb;
    if (tid < amax && base + tid < ndesc) dn = db.adj_desc[base + tid];
  }
  nb = next_blk(nb);
  int nbase = nb < db.adj_nblocks ? db.adj_blk0[nb] + nb : 0;

  int since_flush = 0, since_ft = 0, tab_t = -1;
  for (int blk = first_blk; blk < db.adj_nblocks; blk = next_blk(blk)) {
    __syncthreads();  // previous block done with the shared arrays
    if (tid < amax) {
      a_idx[tid] = dn.x;
      a_lo[tid] = dn.y;
      a_cell[tid] = dn.w;
    }
    if (tid == 0) a_na[0] = dn.z;
    __syncthreads();
    if (nb < db.adj_nblocks) {  // the next block's descriptor, the start of the one after
      if (tid < amax && nbase + tid < ndesc) dn = db.adj_desc[nbase + tid];
      nb = next_blk(nb);
      nbase = nb < db.adj_nblocks ? db.adj_blk0[nb] + nb : 0;
    }
    const int na = a_na[0] & 255;
    const int nslot = a_lo[na];
    const int ti = a_na[0] >> 8;  // every atom of the block
    if (!DET && MEAM && !GM && tab_t >= 0 && ti != tab_t) {
      flush_gacc(tab_t);
      since_flush = 0;
    }
    tab_t = ti;

    const bool have = tid < nslot;
    const int me = have ? slot_owner(a_lo, na, tid) : 0;
    const int ia = a_idx[me];
    const int64_t gs = (int64_t)db.pair_off[ia] + (tid - a_lo[me]);
    const int cell = a_cell[me];

    PairEval<MEAM, R> pe;
    double Lx = 0, Ly = 0, Lz = 0, a_p = 0, G = 0, H = 0, J = 0;
    if (PK) {  // zero rows for idle threads and the padding
      put_pair_row(tid, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f);
      if (tid < 8) put_pair_row(BLOCK_SLOTS + tid, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f);
    } else if (MEAM) {  // zero rows for idle threads and the padding
      srow[tid] = R4{};
      sadj[tid] = R4{};
      sqz[tid] = R(0);
      if (GM) stype[tid] = 0;
      if (tid < 8) {
        srow[BLOCK_SLOTS + tid] = R4{};
        sadj[BLOCK_SLOTS + tid] = R4{};
        sqz[BLOCK_SLOTS + tid] = R(0);
        if (GM) stype[BLOCK_SLOTS + tid] = 0;
      }
    }
    if (have) {
      pe = eval_pair<MEAM, R, Q5>(db, pot, sg, ptab, gs, ti);
      const int j = db.pair_nbr[gs];
      const double ux = db.pair_ux[gs], uy = db.pair_uy[gs], uz = db.pair_uz[gs], r = db.pair_r[gs];
      // m_p: the slot's stress term -r (u_x V_x, u_y V_y, u_z V_z, u_x V_y, u_y V_z, u_z V_x) transposed
      const double mxx = sd[(CS_MU0 + 0) * NC + cell], myy = sd[(CS_MU0 + 1) * NC + cell],
                   mzz = sd[(CS_MU0 + 2) * NC + cell], mxy = sd[(CS_MU0 + 3) * NC + cell],
                   myz = sd[(CS_MU0 + 4) * NC + cell], mzx = sd[(CS_MU0 + 5) * NC + cell];
      Lx = L[ia] - L[j] - r * (mxx * ux + mzx * uz);
      Ly = L[N + ia] - L[N + j] - r * (myy * uy + mxy * ux);
      Lz = L[2 * N + ia] - L[2 * N + j] - r * (mzz * uz + myz * uy);
      a_p = Lx * ux + Ly * uy + Lz * uz;
      double kp = a_p * (double)pe.drho;
      if (MEAM) {
        G = ax[AUX_G * Np + gs];
        H = ax[AUX_H * Np + gs];
        J = Lx * ax[AUX_VX * Np + gs] + Ly * ax[AUX_VY * Np + gs] + Lz * ax[AUX_VZ * Np + gs];
        const double ip = (double)pe.invr, fp = (double)pe.f;
        kp += a_p * (double)pe.df * G - a_p * fp * ip * H + fp * ip * J;
        if constexpr (PK) {
          put_pair_row(tid, pe.ux, pe.uy, pe.uz, pe.f, (float)(a_p * (double)pe.df), (float)(a_p * fp * ip),
                       (float)(fp * ip * Lx), (float)(fp * ip * Ly), (float)(fp * ip * Lz));
        } else {
          R4 v;
          v.x = pe.ux; v.y = pe.uy; v.z = pe.uz; v.w = pe.f;
          srow[tid] = v;
          R4 q;
          q.x = (R)(a_p * (double)pe.df);
          q.y = (R)(a_p * fp * ip);
          q.z = (R)(fp * ip * Lx);
          q.w = (R)(fp * ip * Ly);
          sadj[tid] = q;
          sqz[tid] = (R)(fp * ip * Lz);
          if (GM) stype[tid] = pe.tj;
        }
      }
      red[tid] = kp;
    }
    __syncthreads();

    // ---- per atom (one warp each): K_i, rho, U', U'', chi = dL/drho; U table gradient
    for (int a = warp; a < na; a += nwarp) {
      double K;
      warp_slot_sums<1>(red, a_lo[a], a_lo[a + 1], lane, &K);
      if (lane == 0 && pot.pair) {
        a_chi[a] = a_dF[a] = 0.0;
      } else if (lane == 0) {
        const int i = a_idx[a];
        const double rho = ao[AO_RHO * N + i];
        const int c = a_cell[a];
        const SplineGeom &gU = sg[pot.s_U + ti];
        const double w = db.cell_w[c];
        double rt = rho, dpen = 0.0, drt = 1.0;
        if (rho < gU.x0) {
          dpen = -w * 100.0 * 10. * 2.0 * (gU.x0 - rho);
          if (!pot.embed_extrap) { rt = gU.x0; drt = 0.0; }
        } else if (rho > gU.xN) {
          dpen = w * 100.0 * 10. * 2.0 * (rho - gU.xN);
          if (!pot.embed_extrap) { rt = gU.xN; drt = 0.0; }
        }
        const PointEval U = spl_point_t<Q5>(tc, gU, rt);
        const double eps = sd[CS_EPS * NC + c], kap = sd[CS_KAPPA * NC + c];
        a_chi[a] = (eps * U.grad + U.grad2 * K) * drt + kap * dpen;
        a_dF[a] = U.grad;
        // into the warp's FP32 table (lane 0 alone writes it in this phase), so
        // that no global read-modify-write stands before the barrier
        FT *ftU = ft + gU.toff;
        if (quintic_of<Q5>(gU)) spl_point_adjoint5(gU, U, rt, eps, K, [&](int idx, double v) { ftU[idx] += (FT)v; });
        else spl_point_adjoint(gU, U, rt, eps, K, [&](int idx, double v) { ftU[idx] += (FT)v; });
      }
    }
    __syncthreads();

    if (have) {
      const double chi = a_chi[me], dF = a_dF[me];
      double dKdf = 0.0;
      if (GM) {
        // GMEAM: g spline (i; j, k) per partner, table by the partner's type
        const double fp = (double)pe.f, ip = (double)pe.invr;
        const R gam = (R)(0.5 * chi * fp + dF * a_p * (double)pe.df);
        const R del = (R)(dF * fp * ip);
        const R lx = (R)Lx, ly = (R)Ly, lz = (R)Lz, ap = (R)a_p;
        const int row_lo = a_lo[me], row_hi = a_lo[me + 1];
        for (int kb = row_lo; kb < row_hi; kb += 8) {
          R dk8 = 0;
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const int k = kb + u;
            const R4 o = srow[k];
            const R4 q = sadj[k];
            const int tk = stype[k];
            const SplineGeom &g2 = sg[gmeam_g_index(pot, ti, pe.tj, tk)];
            const R ginv = (R)g2.invstep;
            const R cs = cos_dot(pe.ux, pe.uy, pe.uz, o.x, o.y, o.z);
            const bool ok = (k < row_hi) && (k != tid) && (cs < g_cut<R>(g2));
            const R wk = ok ? R(1) : R(0);
            R b;
            const int m = g_knot<R>(cs, (R)g2.x0, ginv, g2.n, b);
            R dg;
            const R gv = piece_val_grad<Q5, R>(ptab + g2.poff, m, b, ginv, dg, g2.q5);
            const R qu = q.z * pe.ux + q.w * pe.uy + sqz[k] * pe.uz;
            dk8 += wk * (q.x * gv - q.y * dg * cs + dg * qu);
            const R bpk = lx * o.x + ly * o.y + lz * o.z;
            const R fk = wk * o.w;
            const R cg = fk * gam;
            const R cs1 = fk * del * (bpk - ap * cs) * ginv;
            const R b2 = b * b;
            R4 *ga = gacc + (size_t)(tk * nint + m) * BLOCK_SLOTS + tid;
            R4 d = *ga;
            d.x += cg;
            d.y += cg * b + cs1;
            d.z += cg * b2 + R(2) * cs1 * b;
            d.w += cg * b2 * b + R(3) * cs1 * b2;
            *ga = d;
            if (quintic_of<Q5>(g2)) {  // quintic pieces: the b^4 and b^5 coefficients
              R2 *g5 = gacc5 + (size_t)(tk * nint + m) * BLOCK_SLOTS + tid;
              R2 e = *g5;
              const R b3 = b2 * b;
              e.x += cg * b3 * b + R(4) * cs1 * b3;
              e.y += cg * b3 * b2 + R(5) * cs1 * b3 * b;
              *g5 = e;
            }
          }
          dKdf += (double)dk8;
        }
        dKdf += ip * (J - a_p * H);
      } else if constexpr (PK) {
        // Two partners per step as packed FP32 pairs (sm_100 __ffma2_rn and
        // friends); per partner the arithmetic of the branch below, with the
        // interval search of g_knot<float> and the pieces evaluated one by one.
        const SplineGeom gg = sg[pot.s_g + ti];
        const float *gpc = ptab + gg.poff;
        const float ginv = (float)gg.invstep, gcut = g_cut<float>(gg);
        const int nmax = gg.n - 2;
        const double fp = (double)pe.f, ip = (double)pe.invr;
        const float2 UX = bcast2(pe.ux), UY = bcast2(pe.uy), UZ = bcast2(pe.uz);
        const float2 LX = bcast2((float)Lx), LY = bcast2((float)Ly), LZ = bcast2((float)Lz);
        const float2 NAP = bcast2(-(float)a_p);
        const float2 GAM = bcast2((float)(0.5 * chi * fp + dF * a_p * (double)pe.df));
        const float2 DELH = bcast2((float)(dF * fp * ip) * ginv);
        const float2 GINV = bcast2(ginv), NX0 = bcast2(-(float)gg.x0);
        float4 *ga = reinterpret_cast<float4 *>(gacc) + tid;
        const int row_lo = a_lo[me], row_hi = a_lo[me + 1];
        // steps of 2 pairs: at most 3 masked partners at the end of a row
        for (int pb = row_lo >> 1; 2 * pb < row_hi; pb += 2) {
          float2 dk2 = bcast2(0.f);
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            const int p = pb + u, k0 = 2 * p, k1 = k0 + 1;
            const float4 ra = rowA[p], rb = rowB[p], qa = adjA[p], qb = adjB[p];
            const float2 ox = pair2(ra.x, ra.y), oy = pair2(ra.z, ra.w), oz = pair2(rb.x, rb.y);
            const float2 cs = fma2(UX, ox, fma2(UY, oy, mul2(UZ, oz)));
            // k0 >= row_lo - 1 and k1 >= row_lo by the start of the loop
            const bool ok0 = k0 >= row_lo && k0 < row_hi && k0 != tid && cs.x < gcut;
            const bool ok1 = k1 < row_hi && k1 != tid && cs.y < gcut;
            const float2 w = pair2(ok0 ? 1.f : 0.f, ok1 ? 1.f : 0.f);
            const float2 t = mul2(add2(cs, NX0), GINV);
            float b0, b1;
            const int m0 = knot_of_t(t.x, nmax, b0), m1 = knot_of_t(t.y, nmax, b1);
            const float2 b = pair2(b0, b1);
            float dg0, dg1;
            const float gv0 = cubic_val_grad<float>(gpc, m0, b0, ginv, dg0);
            const float gv1 = cubic_val_grad<float>(gpc, m1, b1, ginv, dg1);
            const float2 gv = pair2(gv0, gv1), dg = pair2(dg0, dg1);
            // d K / d f_p from the triplet terms of slot k
            const float2 qu = fma2(pair2(qb.x, qb.y), UX, fma2(pair2(qb.z, qb.w), UY, mul2(qz2[p], UZ)));
            dk2 = fma2(w, fma2(pair2(qa.x, qa.y), gv, mul2(dg, fma2(pair2(qa.z, qa.w), cs, qu))), dk2);
            // g table (power basis): value weight cg, slope weight cs1 / h
            const float2 bpk = fma2(LX, ox, fma2(LY, oy, mul2(LZ, oz)));
            const float2 fk = mul2(w, pair2(rb.z, rb.w));
            const float2 cg = mul2(fk, GAM);
            const float2 cs1 = mul2(mul2(fk, DELH), fma2(NAP, cs, bpk));
            // cg b^j + j cs1 b^(j-1), j = 0..3
            const float2 c1 = fma2(cg, b, cs1);
            const float2 c2 = mul2(b, add2(c1, cs1));
            const float2 c3 = mul2(mul2(b, b), add2(c1, add2(cs1, cs1)));
            float4 d = ga[m0 * BLOCK_SLOTS];
            d.x += cg.x;
            d.y += c1.x;
            d.z += c2.x;
            d.w += c3.x;
            ga[m0 * BLOCK_SLOTS] = d;
            d = ga[m1 * BLOCK_SLOTS];
            d.x += cg.y;
            d.y += c1.y;
            d.z += c2.y;
            d.w += c3.y;
            ga[m1 * BLOCK_SLOTS] = d;
          }
          dKdf += (double)dk2.x + (double)dk2.y;
        }
        dKdf += ip * (J - a_p * H);
      } else if (MEAM) {
        const SplineGeom gg = sg[pot.s_g + ti];
        const R *gpc = ptab + gg.poff;
        const R gx0 = (R)gg.x0, ginv = (R)gg.invstep;
        const R gcut = g_cut<R>(gg);
        const int ngt = gg.n;
        const double fp = (double)pe.f, ip = (double)pe.invr;
        const R gam = (R)(0.5 * chi * fp + dF * a_p * (double)pe.df);
        const R del = (R)(dF * fp * ip);
        const R lx = (R)Lx, ly = (R)Ly, lz = (R)Lz, ap = (R)a_p;
        R4 *ga = gacc + tid;
        const int row_lo = a_lo[me], row_hi = a_lo[me + 1];
        for (int kb = row_lo; kb < row_hi; kb += 8) {
          R dk8 = 0;
          // Branch-free chunk of 8 partners (zero weight when not a triplet
          // of this row; the shared rows are padded with zeros).
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const int k = kb + u;
            const R4 o = srow[k];
            const R4 q = sadj[k];
            const R cs = cos_dot(pe.ux, pe.uy, pe.uz, o.x, o.y, o.z);
            const bool ok = (k < row_hi) && (k != tid) && (cs < gcut);
            const R wk = ok ? R(1) : R(0);
            R b;
            const int m = g_knot<R>(cs, gx0, ginv, ngt, b);
            R dg;
            const R gv = piece_val_grad<Q5, R>(gpc, m, b, ginv, dg, gg.q5);
            // d K / d f_p from the triplet terms of slot k
            const R qu = q.z * pe.ux + q.w * pe.uy + sqz[k] * pe.uz;
            dk8 += wk * (q.x * gv - q.y * dg * cs + dg * qu);
            // g table (power basis): value weight cg, slope weight cgp / h
            const R bpk = lx * o.x + ly * o.y + lz * o.z;
            const R fk = wk * o.w;
            const R cg = fk * gam;
            const R cs1 = fk * del * (bpk - ap * cs) * ginv;
            const R b2 = b * b;
            R4 d = ga[m * BLOCK_SLOTS];
            d.x += cg;
            d.y += cg * b + cs1;
            d.z += cg * b2 + R(2) * cs1 * b;
            d.w += cg * b2 * b + R(3) * cs1 * b2;
            ga[m * BLOCK_SLOTS] = d;
            if (quintic_of<Q5>(gg)) {  // quintic pieces: the b^4 and b^5 coefficients
              R2 e = gacc5[m * BLOCK_SLOTS + tid];
              const R b3 = b2 * b;
              e.x += cg * b3 * b + R(4) * cs1 * b3;
              e.y += cg * b3 * b2 + R(5) * cs1 * b3 * b;
              gacc5[m * BLOCK_SLOTS + tid] = e;
            }
          }
          dKdf += (double)dk8;
        }
        dKdf += ip * (J - a_p * H);
      }
      // ---- pair-function tables: phi (energy + force), rho (density + force), f
      auto pair_adj = [&](int s, int k, R b, double cv, double cd) {
        const SplineGeom &g = sg[s];
        if (quintic_of<Q5>(g)) {
          const SplW5<double> w = spl_weights5<double>((double)b, g.step, g.invstep);
          add_f(g.toff + k, cv * w.wa + cd * w.da);
          add_f(g.toff + k + 1, cv * w.wb + cd * w.db);
          add_f(g.toff + g.n + k, cv * w.wA + cd * w.dA);
          add_f(g.toff + g.n + k + 1, cv * w.wB + cd * w.dB);
          add_f(g.toff + 2 * g.n + 2 + k, cv * w.w4a + cd * w.d4a);
          add_f(g.toff + 2 * g.n + 3 + k, cv * w.w4b + cd * w.d4b);
          return;
        }
        const SplW<double> w = spl_weights<double>((double)b, g.step, g.invstep);
        add_f(g.toff + k, cv * w.wa + cd * w.da);
        add_f(g.toff + k + 1, cv * w.wb + cd * w.db);
        add_f(g.toff + g.n + k, cv * w.wA + cd * w.dA);
        add_f(g.toff + g.n + k + 1, cv * w.wB + cd * w.dB);
      };
      const double eps = sd[CS_EPS * NC + cell];
      const double sp = MEAM ? 0.5 : phi_share(pot, db.pair_nbr[gs] == ia);
      if (pe.kphi >= 0) pair_adj(pot.s_phi + pe.pij, pe.kphi, pe.bphi, sp * eps, sp * a_p);
      if (pe.krho >= 0) pair_adj(pot.s_rho + pe.tj, pe.krho, pe.brho, chi, dF * a_p);
      if (MEAM && pe.kf >= 0) pair_adj(pot.s_f + pe.pij, pe.kf, pe.bf, chi * G + dF * dKdf, dF * a_p * G);
    }
    if (JM) {
      // ---- JMEAM (p, q) terms: the per-thread tables hold this block's g
      // gradients; flush them, then one pass per term with the rows of p
      flush_gacc(tab_t);
      since_flush = 0;
      if (have) eval_pair_p<MEAM, R, Q5>(db, pot, sg, ptab, gs, pe);
      const double eps = sd[CS_EPS * NC + cell];
      for (int ch = 0; ch < pot.nj; ++ch) {
        const double *axm = ax + (size_t)AUX_COUNT * (1 + ch) * Np;
        double G2 = 0, H2 = 0, J2 = 0;
        const double pm = have ? (double)pe.p[ch] : 0.0, ip = have ? (double)pe.invr : 0.0;
        __syncthreads();  // every thread is done with the previous rows
        if (have) {
          G2 = axm[AUX_G * Np + gs];
          H2 = axm[AUX_H * Np + gs];
          J2 = Lx * axm[AUX_VX * Np + gs] + Ly * axm[AUX_VY * Np + gs] + Lz * axm[AUX_VZ * Np + gs];
          R4 v;
          v.x = pe.ux; v.y = pe.uy; v.z = pe.uz; v.w = pe.p[ch];
          srow[tid] = v;
          R4 q;
          q.x = (R)(a_p * (double)pe.dp[ch]);
          q.y = (R)(a_p * pm * ip);
          q.z = (R)(pm * ip * Lx);
          q.w = (R)(pm * ip * Ly);
          sadj[tid] = q;
          sqz[tid] = (R)(pm * ip * Lz);
        }
        __syncthreads();
        const SplineGeom qg = sg[pot.s_q[ch] + ti];
        if (have) {
          const R *qpc = ptab + qg.poff;
          const R qx0 = (R)qg.x0, qinv = (R)qg.invstep, qcut = g_cut<R>(qg);
          const R gam = (R)(0.5 * eps * pm + a_p * (double)pe.dp[ch]);
          const R del = (R)(pm * ip);
          const R lx = (R)Lx, ly = (R)Ly, lz = (R)Lz, ap = (R)a_p;
          R4 *ga = gacc + tid;
          const int row_lo = a_lo[me], row_hi = a_lo[me + 1];
          double dKdp = 0.0;
          for (int kb = row_lo; kb < row_hi; kb += 8) {
            R dk8 = 0;
#pragma unroll
            for (int u = 0; u < 8; ++u) {
              const int k = kb + u;
              const R4 o = srow[k];
              const R4 q = sadj[k];
              const R cs = cos_dot(pe.ux, pe.uy, pe.uz, o.x, o.y, o.z);
              const bool ok = (k < row_hi) && (k != tid) && (cs < qcut);
              const R wk = ok ? R(1) : R(0);
              R b;
              const int m = g_knot<R>(cs, qx0, qinv, qg.n, b);
              R dq;
              const R qv = piece_val_grad<Q5, R>(qpc, m, b, qinv, dq, qg.q5);
              const R qu = q.z * pe.ux + q.w * pe.uy + sqz[k] * pe.uz;
              dk8 += wk * (q.x * qv - q.y * dq * cs + dq * qu);
              const R bpk = lx * o.x + ly * o.y + lz * o.z;
              const R pk = wk * o.w;
              const R cg = pk * gam;
              const R cs1 = pk * del * (bpk - ap * cs) * qinv;
              const R b2 = b * b;
              R4 d = ga[m * BLOCK_SLOTS];
              d.x += cg;
              d.y += cg * b + cs1;
              d.z += cg * b2 + R(2) * cs1 * b;
              d.w += cg * b2 * b + R(3) * cs1 * b2;
              ga[m * BLOCK_SLOTS] = d;
              if (quintic_of<Q5>(qg)) {  // quintic pieces: the b^4 and b^5 coefficients
                R2 e = gacc5[m * BLOCK_SLOTS + tid];
                const R b3 = b2 * b;
                e.x += cg * b3 * b + R(4) * cs1 * b3;
                e.y += cg * b3 * b2 + R(5) * cs1 * b3 * b;
                gacc5[m * BLOCK_SLOTS + tid] = e;
              }
            }
            dKdp += (double)dk8;
          }
          dKdp += ip * (J2 - a_p * H2);
          if (pe.kp[ch] >= 0) {
            const SplineGeom &g = sg[pot.s_p[ch] + pe.pij];
            const double cv = eps * G2 + dKdp, cd = a_p * G2;
            const int kp = pe.kp[ch];
            if (quintic_of<Q5>(g)) {
              const SplW5<double> w = spl_weights5<double>((double)pe.bp[ch], g.step, g.invstep);
              add_f(g.toff + kp, cv * w.wa + cd * w.da);
              add_f(g.toff + kp + 1, cv * w.wb + cd * w.db);
              add_f(g.toff + g.n + kp, cv * w.wA + cd * w.dA);
              add_f(g.toff + g.n + kp + 1, cv * w.wB + cd * w.dB);
              add_f(g.toff + 2 * g.n + 2 + kp, cv * w.w4a + cd * w.d4a);
              add_f(g.toff + 2 * g.n + 3 + kp, cv * w.w4b + cd * w.d4b);
            } else {
              const SplW<double> w = spl_weights<double>((double)pe.bp[ch], g.step, g.invstep);
              add_f(g.toff + kp, cv * w.wa + cd * w.da);
              add_f(g.toff + kp + 1, cv * w.wb + cd * w.db);
              add_f(g.toff + g.n + kp, cv * w.wA + cd * w.dA);
              add_f(g.toff + g.n + kp + 1, cv * w.wB + cd * w.dB);
            }
          }
        }
        flush_gacc_spline(pot.s_q[ch] + ti);
      }
    }
    if constexpr (DET) {
      det_flush();
      if (GM) flush_gacc_gm(tab_t, have, have ? pe.tj : 0);
      else if (MEAM) flush_gacc(tab_t);
      if ((blk + 1) % GB == 0 || blk + 1 == db.adj_nblocks) {
        // end of a group: its partial, the warp tables summed in warp order
        __syncthreads();
        double *out = partial + ((size_t)cand * ngroups + blk / GB) * stride;
        for (int e = tid; e < stride; e += blockDim.x) {
          double s = 0.0;
          for (int w = 0; w < ADJ_WARPS; ++w) s += (double)ftab[(size_t)w * stride + e];
          out[e] = s;
        }
        __syncthreads();
        for (int i = tid; i < ADJ_WARPS * stride; i += blockDim.x) ftab[i] = FT(0);
      }
    } else {
      if (++since_ft == FT_FLUSH_BLOCKS) {
        flush_ft();
        since_ft = 0;
      }
      if (GM) {
        flush_gacc_gm(tab_t, have, have ? pe.tj : 0);
      } else if (MEAM && ++since_flush == GACC_FLUSH_BLOCKS) {
        flush_gacc(tab_t);
        since_flush = 0;
      }
    }
  }
  if constexpr (!DET) {
    if (since_ft > 0) flush_ft();
    __syncthreads();
    if (MEAM && !GM && since_flush > 0 && tab_t >= 0) {
      flush_gacc(tab_t);
      __syncthreads();
    }
    double *out = partial + ((size_t)cand * gridDim.x + blockIdx.x) * stride;
    for (int e = tid; e < stride; e += blockDim.x) {
      double s = 0.0;
      for (int w = 0; w < ADJ_WARPS; ++w) s += wtab[(size_t)w * stride + e];
      out[e] = s;
    }
  }
}

// Sum the CTA partials, add the punishment terms, and map the table
// gradient (y, ypp, end slopes) to the coefficients through the transposed
// refresh: ypp = M [y; slope_left; slope_right] (Spline3Eq::refresh_basis is
// linear in them, spline3eq.cpp:192-225).
__global__ void k_grad_final(DevPot pot, const SplineGeom *__restrict__ geom, const double *__restrict__ tabs,
                             const double *__restrict__ partial, int nparts, const double *__restrict__ M,
                             const int *__restrict__ cmap, int P, double *__restrict__ grad) {
  extern __shared__ double ext[];
  const int c = blockIdx.x;
  const int t = threadIdx.x;
  const int stride = pot.tab_stride;
  for (int e = t; e < stride; e += blockDim.x) {
    double s = 0.0;
    const double *p = partial + (size_t)c * nparts * stride + e;
    for (int b = 0; b < nparts; ++b) s += p[(size_t)b * stride];
    ext[e] = s;
  }
  __syncthreads();
  const double *tab = tabs + (size_t)c * stride;
  if (t == 0 && !pot.omit_pen && !pot.pair) {
    if (pot.gmeam) {
      for (int f = 0; f < pot.npair; ++f) {
        int at = -1;
        const double my = spline_max_y(geom[pot.s_f + f], tab, &at);
        const double m = fabs(my);
        const double fe = 100. * 25. * (1.0 - m) * (1.0 - m);
        if (at >= 0) ext[at] += 2.0 * fe * (-5000.0) * (1.0 - m) * (my > 0 ? 1.0 : (my < 0 ? -1.0 : 0.0));
      }
    } else if (pot.style == MZ_STYLE_MEAM_SPLINE || pot.nj > 0) {
      for (int q = 0; q <= pot.nj; ++q) {  // f, then JMEAM's p (p2)
        int at = -1;
        const double my = group_max_y(pot, q == 0 ? pot.s_f : pot.s_p[q - 1], geom, tab, &at);
        const double m = fabs(my);
        const double fe = 100. * 25. * (1.0 - m) * (1.0 - m);
        if (at >= 0) ext[at] += 2.0 * fe * (-5000.0) * (1.0 - m) * (my > 0 ? 1.0 : (my < 0 ? -1.0 : 0.0));
      }
    } else {
      for (int ty = 0; ty < pot.ntypes; ++ty) {
        const SplineGeom &g = geom[pot.s_U + ty];
        const double mid = 0.5 * (g.x0 + g.xN);
        const PointEval e = spl_point_any(tab, g, mid);
        const double ev = 100. * e.grad;
        const int to = g.toff;
        if (g.q5) spl_point_adjoint5(g, e, mid, 0.0, 2.0 * ev * 100.0, [&](int idx, double v) { ext[to + idx] += v; });
        else spl_point_adjoint(g, e, mid, 0.0, 2.0 * ev * 100.0, [&](int idx, double v) { ext[to + idx] += v; });
      }
    }
  }
  __syncthreads();
  double *gc = grad + (size_t)c * P;
  for (int s = t; s < pot.nsplines; s += blockDim.x) {
    const SplineGeom g = geom[s];
    const int n = g.n;
    if (g.q5) {
      // spline5eq: (ypp, yp4) = M (y, grad, grad2), M [2n][n+4]
      for (int col = 0; col < n + 4; ++col) {
        const int te = col < n ? g.toff + col : col < n + 2 ? g.toff + 2 * n + (col - n) : g.toff + 3 * n + 2 + (col - n - 2);
        double acc = ext[te];
        for (int r = 0; r < n; ++r) acc += M[g.moff + r * (n + 4) + col] * ext[g.toff + n + r];
        for (int r = 0; r < n; ++r) acc += M[g.moff + (n + r) * (n + 4) + col] * ext[g.toff + 2 * n + 2 + r];
        const int ci = cmap[te];
        if (ci >= 0) gc[ci] = acc;
      }
      continue;
    }
    for (int col = 0; col < n + 2; ++col) {
      double acc = col < n ? ext[g.toff + col] : ext[g.toff + 2 * n + (col - n)];
      for (int r = 0; r < n; ++r) acc += M[g.moff + r * (n + 2) + col] * ext[g.toff + n + r];
      const int ci = col < n ? cmap[g.toff + col] : cmap[g.toff + 2 * n + (col - n)];
      if (ci >= 0) gc[ci] = acc;
    }
  }
}

}  // namespace mzb
