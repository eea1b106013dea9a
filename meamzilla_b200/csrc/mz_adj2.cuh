// Adjoint of the mixed-precision MEAM objective with two candidates per CTA.
//
// The structure is k_adj's (mz_adj.cuh) for meam/spline with spline3eq
// pieces: persistent CTAs over type-pure atom blocks, one thread per pair
// slot, one pass over each row for d K / d f and the g-table gradient.  Each
// (slot, partner) computes the triplet geometry -- cosine, g interval,
// shift -- once and both candidates' arithmetic as packed FP32 pairs
// (__ffma2_rn).  Per candidate the per-thread g tables live in shared memory
// as coefficient pairs ((x_A, x_B, y_A, y_B), (z_A, z_B, w_A, w_B) per
// interval); the per-warp FP64 tables, which the per-thread tables and the
// pair-function sums are flushed into, live in global memory (one slice per
// candidate, CTA and warp, summed in a fixed order at the end), so that two
// candidates fit the shared memory of two CTAs per SM.  Each candidate's
// gradient equals k_adj's up to the order of FP32 and FP64 additions.
#pragma once

#include "mz_adj.cuh"
#include "mz_fwd2.cuh"

namespace mzb {

// Shared-memory layout of k_adj2 (dynamic), see adj2_smem_bytes():
//   float4 gacc[nint][2][BLOCK_SLOTS]     per-thread g-table gradients of both candidates
//   float  ftab[2][ADJ_WARPS][stride]     per-warp pair-function gradients of one block
//   double red[2][BLOCK_SLOTS], a_chi[2][BLOCK_ATOMS], a_dF[2][BLOCK_ATOMS]
//   SplineGeom sg[nsplines]; int a_lo[BLOCK_ATOMS+2], a_idx[BLOCK_ATOMS], a_len[BLOCK_ATOMS]
//   float4 pt2[2][pstride / 4 + 1]       both candidates' evaluation tables, interleaved
//   float4 srow[BLOCK_SLOTS+8]           (u_x, u_y, u_z, 0)
//   float2 sf[BLOCK_SLOTS+8]             (f_A, f_B)
//   float4 sq0[BLOCK_SLOTS+8]            (a f'_A, a f'_B, a f / r _A, a f / r _B)
//   float4 sq1[BLOCK_SLOTS+8]            (Q_x A, Q_x B, Q_y A, Q_y B),  Q = f Lambda / r
//   float2 sqz[BLOCK_SLOTS+8]            (Q_z A, Q_z B)
__host__ __device__ inline size_t adj2_smem_bytes(int nsplines, int stride, int pstride, int ng) {
  size_t b = sizeof(float4) * 2 * (size_t)(ng - 1) * BLOCK_SLOTS;
  b += sizeof(float) * 2 * (size_t)ADJ_WARPS * stride;
  b = (b + 31) & ~size_t(31);
  b += sizeof(double) * (2 * BLOCK_SLOTS + 4 * BLOCK_ATOMS);
  b += sizeof(SplineGeom) * nsplines;
  b += sizeof(int) * (3 * BLOCK_ATOMS + 2);
  b = (b + 31) & ~size_t(31);
  b += sizeof(float4) * 2 * ((size_t)pstride / 4 + 1);
  b = (b + 31) & ~size_t(31);
  b += (3 * sizeof(float4) + 2 * sizeof(float2)) * (BLOCK_SLOTS + 8);
  return b;
}

// wglob: [ncand][gridDim.x][ADJ_WARPS][stride] FP64 per-warp tables (zeroed
// here); partial: [ncand][gridDim.x][stride] as k_adj writes it.
__global__ void __launch_bounds__(BLOCK_SLOTS, 2)
    k_adj2(DevDb db, DevPot pot, const SplineGeom *__restrict__ geom, const double *__restrict__ tabs,
           const double *__restrict__ ptabs, const double *__restrict__ aout, const double *__restrict__ aux,
           const double *__restrict__ lam, const double *__restrict__ seeds, double *__restrict__ wglob,
           double *__restrict__ partial, int ncand) {
  extern __shared__ __align__(32) unsigned char smem_raw[];
  const int cA = 2 * blockIdx.y;
  const bool twoc = cA + 1 < ncand;
  const int cB = twoc ? cA + 1 : cA;
  const int nc = twoc ? 2 : 1;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
  const int N = db.natoms, NC = db.ncells;
  const int64_t Np = db.npairs;
  const int stride = pot.tab_stride;
  const int nint = pot.g_nmax - 1;

  float4 *gacc = reinterpret_cast<float4 *>(smem_raw);
  float *ftab = reinterpret_cast<float *>(gacc + 2 * (size_t)nint * BLOCK_SLOTS);
  size_t off = sizeof(float4) * 2 * (size_t)nint * BLOCK_SLOTS + sizeof(float) * 2 * (size_t)ADJ_WARPS * stride;
  off = (off + 31) & ~size_t(31);
  double *red = reinterpret_cast<double *>(smem_raw + off);  // [2][BLOCK_SLOTS]
  double *a_chi = red + 2 * BLOCK_SLOTS;                      // [2][BLOCK_ATOMS]
  double *a_dF = a_chi + 2 * BLOCK_ATOMS;                     // [2][BLOCK_ATOMS]
  SplineGeom *sg = reinterpret_cast<SplineGeom *>(a_dF + 2 * BLOCK_ATOMS);
  int *a_lo = reinterpret_cast<int *>(sg + pot.nsplines);
  int *a_idx = a_lo + BLOCK_ATOMS + 2;
  int *a_len = a_idx + BLOCK_ATOMS;
  off = reinterpret_cast<unsigned char *>(a_len + BLOCK_ATOMS) - smem_raw;
  off = (off + 31) & ~size_t(31);
  float4 *pt2 = reinterpret_cast<float4 *>(smem_raw + off);
  const int npiece = pot.pow_stride / 4;
  off += sizeof(float4) * 2 * ((size_t)npiece + 1);
  off = (off + 31) & ~size_t(31);
  float4 *srow = reinterpret_cast<float4 *>(smem_raw + off);
  float4 *sq0 = srow + BLOCK_SLOTS + 8;
  float4 *sq1 = sq0 + BLOCK_SLOTS + 8;
  float2 *sf = reinterpret_cast<float2 *>(sq1 + BLOCK_SLOTS + 8);
  float2 *sqz = sf + BLOCK_SLOTS + 8;

  load_pt2(pt2, ptabs + (size_t)cA * pot.pow_stride, ptabs + (size_t)cB * pot.pow_stride, pot.pow_stride);
  for (int i = tid; i < 2 * ADJ_WARPS * stride; i += blockDim.x) ftab[i] = 0.f;
  for (int i = tid; i < 2 * nint * BLOCK_SLOTS; i += blockDim.x) gacc[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int i = tid; i < pot.nsplines; i += blockDim.x) sg[i] = geom[i];
  double *wt[2];
  float *ft[2];
  for (int c = 0; c < 2; ++c) {
    wt[c] = wglob + (((size_t)(c ? cB : cA) * gridDim.x + blockIdx.x) * ADJ_WARPS + warp) * stride;
    ft[c] = ftab + ((size_t)c * ADJ_WARPS + warp) * stride;
  }
  for (int e = lane; e < stride; e += 32) {
    wt[0][e] = 0.0;
    if (twoc) wt[1][e] = 0.0;
  }
  const double *tcs[2] = {tabs + (size_t)cA * stride, tabs + (size_t)cB * stride};
  const double *aos[2] = {aout + (size_t)cA * AO_COUNT * N, aout + (size_t)cB * AO_COUNT * N};
  const double *axs[2] = {aux + (size_t)cA * AUX_COUNT * Np, aux + (size_t)cB * AUX_COUNT * Np};
  const double *Ls[2] = {lam + (size_t)cA * 3 * N, lam + (size_t)cB * 3 * N};
  const double *sds[2] = {seeds + (size_t)cA * CS_COUNT * NC, seeds + (size_t)cB * CS_COUNT * NC};

  // per-thread g tables of type t into the warps' FP64 tables
  auto flush_gacc = [&](int t) {
    const SplineGeom &gg = sg[pot.s_g + t];
    for (int m = 0; m < gg.n - 1; ++m) {
      const float4 lo = gacc[(2 * m) * BLOCK_SLOTS + tid], hi = gacc[(2 * m + 1) * BLOCK_SLOTS + tid];
      double d[8] = {(double)lo.x, (double)lo.z, (double)hi.x, (double)hi.z,
                     (double)lo.y, (double)lo.w, (double)hi.y, (double)hi.w};
#pragma unroll
      for (int q = 0; q < 8; ++q)
        for (int o = 16; o > 0; o >>= 1) d[q] += __shfl_down_sync(0xffffffffu, d[q], o);
      if (lane == 0)
        for (int c = 0; c < nc; ++c)
          power_to_table(gg, m, d[4 * c], d[4 * c + 1], d[4 * c + 2], d[4 * c + 3],
                         [&](int idx, double x) { wt[c][gg.toff + idx] += x; });
    }
    for (int m = 0; m < 2 * nint; ++m) gacc[m * BLOCK_SLOTS + tid] = make_float4(0.f, 0.f, 0.f, 0.f);
  };

  // the warp's FP32 sums into its FP64 tables (in global memory): all loads
  // of a lane issued before its adds and stores
  auto flush_ft = [&]() {
    __syncwarp();
    for (int c = 0; c < nc; ++c) {
      double *__restrict__ w = wt[c];
      float *__restrict__ fl = ft[c];
      for (int e0 = lane; e0 < stride; e0 += 32 * 8) {
        double v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int e = e0 + 32 * q;
          v[q] = e < stride ? w[e] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int e = e0 + 32 * q;
          if (e < stride) {
            w[e] = v[q] + (double)fl[e];
            fl[e] = 0.f;
          }
        }
      }
    }
    __syncwarp();
  };

  int since_flush = 0, since_ft = 0, tab_t = -1;
  for (int blk = blockIdx.x; blk < db.adj_nblocks; blk += gridDim.x) {
    const int b0 = db.adj_blk0[blk], na = db.adj_blk0[blk + 1] - b0;
    __syncthreads();  // previous block done with the shared arrays
    if (tid < na) {
      const int at = db.adj_atoms[b0 + tid];
      a_idx[tid] = at;
      a_len[tid] = db.pair_off[at + 1] - db.pair_off[at];
    }
    __syncthreads();
    if (warp == 0) {  // row starts in the block's slot numbering (na <= 64: two atoms per lane)
      const int v0 = 2 * lane < na ? a_len[2 * lane] : 0, v1 = 2 * lane + 1 < na ? a_len[2 * lane + 1] : 0;
      int inc = v0 + v1;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
      }
      const int exc = inc - v0 - v1;
      if (2 * lane <= na) a_lo[2 * lane] = exc;
      if (2 * lane + 1 <= na) a_lo[2 * lane + 1] = exc + v0;
      if (lane == 31) a_lo[na] = inc;
    }
    __syncthreads();
    const int nslot = a_lo[na];
    const int ti = db.atom_type[a_idx[0]];  // every atom of the block
    if (tab_t >= 0 && ti != tab_t) {
      flush_gacc(tab_t);
      since_flush = 0;
    }
    tab_t = ti;

    const bool have = tid < nslot;
    const int me = have ? slot_owner(a_lo, na, tid) : 0;
    const int ia = a_idx[me];
    const int64_t gs = (int64_t)db.pair_off[ia] + (tid - a_lo[me]);
    const int cell = db.atom_cell[ia];

    // zero rows for idle threads and the padding
    srow[tid] = make_float4(0.f, 0.f, 0.f, 0.f);
    sq0[tid] = srow[tid];
    sq1[tid] = srow[tid];
    sf[tid] = bcast2(0.f);
    sqz[tid] = bcast2(0.f);
    if (tid < 8) {
      srow[BLOCK_SLOTS + tid] = make_float4(0.f, 0.f, 0.f, 0.f);
      sq0[BLOCK_SLOTS + tid] = srow[BLOCK_SLOTS + tid];
      sq1[BLOCK_SLOTS + tid] = srow[BLOCK_SLOTS + tid];
      sf[BLOCK_SLOTS + tid] = bcast2(0.f);
      sqz[BLOCK_SLOTS + tid] = bcast2(0.f);
    }

    // ---- the slot's pair functions of both candidates, Lambda_p, a_p, k_p
    float fux = 0.f, fuy = 0.f, fuz = 0.f, invr = 0.f;
    float2 dphi = bcast2(0.f), drho = dphi, f = dphi, df = dphi;
    int kphi = -1, krho = -1, kf = -1, pij = 0, tj = 0;
    float bphi = 0.f, brho = 0.f, bf = 0.f;
    double Lx[2] = {0, 0}, Ly[2] = {0, 0}, Lz[2] = {0, 0}, ap[2] = {0, 0}, G[2] = {0, 0}, H[2] = {0, 0},
           J[2] = {0, 0};
    if (have) {
      fux = db.pair_uxf[gs];
      fuy = db.pair_uyf[gs];
      fuz = db.pair_uzf[gs];
      invr = 1.f / db.pair_rf[gs];
      const int kn = db.pair_knot[gs];
      kphi = (kn & 0xff) - 1;
      krho = ((kn >> 8) & 0xff) - 1;
      kf = ((kn >> 16) & 0xff) - 1;
      const int j = db.pair_nbr[gs];
      tj = db.atom_type[j];
      pij = pair_ij_index(ti, tj, pot.ntypes);
      if (kphi >= 0) {
        const SplineGeom &g = sg[pot.s_phi + pij];
        bphi = db.pair_shiftf[gs];
        cubic2_val_grad(pt2, npiece, g.poff, kphi, bphi, (float)g.invstep, dphi);
      }
      if (krho >= 0) {
        const SplineGeom &g = sg[pot.s_rho + tj];
        brho = db.pair_shiftf[Np + gs];
        cubic2_val_grad(pt2, npiece, g.poff, krho, brho, (float)g.invstep, drho);
      }
      if (kf >= 0) {
        const SplineGeom &g = sg[pot.s_f + pij];
        bf = db.pair_shiftf[2 * Np + gs];
        f = cubic2_val_grad(pt2, npiece, g.poff, kf, bf, (float)g.invstep, df);
      }
      const double ux = db.pair_ux[gs], uy = db.pair_uy[gs], uz = db.pair_uz[gs], r = db.pair_r[gs];
      const double ip = (double)invr;
      float qa[2], qb[2], qx[2], qy[2], qzz[2];
      for (int c = 0; c < 2; ++c) {
        const double *sd = sds[c], *L = Ls[c], *ax = axs[c];
        // m_p: the slot's stress term -r (u_x V_x, u_y V_y, u_z V_z, u_x V_y, u_y V_z, u_z V_x) transposed
        const double mxx = sd[(CS_MU0 + 0) * NC + cell], myy = sd[(CS_MU0 + 1) * NC + cell],
                     mzz = sd[(CS_MU0 + 2) * NC + cell], mxy = sd[(CS_MU0 + 3) * NC + cell],
                     myz = sd[(CS_MU0 + 4) * NC + cell], mzx = sd[(CS_MU0 + 5) * NC + cell];
        Lx[c] = L[ia] - L[j] - r * (mxx * ux + mzx * uz);
        Ly[c] = L[N + ia] - L[N + j] - r * (myy * uy + mxy * ux);
        Lz[c] = L[2 * N + ia] - L[2 * N + j] - r * (mzz * uz + myz * uy);
        ap[c] = Lx[c] * ux + Ly[c] * uy + Lz[c] * uz;
        G[c] = ax[AUX_G * Np + gs];
        H[c] = ax[AUX_H * Np + gs];
        J[c] = Lx[c] * ax[AUX_VX * Np + gs] + Ly[c] * ax[AUX_VY * Np + gs] + Lz[c] * ax[AUX_VZ * Np + gs];
        const double fp = c ? (double)f.y : (double)f.x, dfp = c ? (double)df.y : (double)df.x;
        const double drp = c ? (double)drho.y : (double)drho.x;
        red[c * BLOCK_SLOTS + tid] = ap[c] * drp + ap[c] * dfp * G[c] - ap[c] * fp * ip * H[c] + fp * ip * J[c];
        qa[c] = (float)(ap[c] * dfp);
        qb[c] = (float)(ap[c] * fp * ip);
        qx[c] = (float)(fp * ip * Lx[c]);
        qy[c] = (float)(fp * ip * Ly[c]);
        qzz[c] = (float)(fp * ip * Lz[c]);
      }
      srow[tid] = make_float4(fux, fuy, fuz, 0.f);
      sf[tid] = f;
      sq0[tid] = make_float4(qa[0], qa[1], qb[0], qb[1]);
      sq1[tid] = make_float4(qx[0], qx[1], qy[0], qy[1]);
      sqz[tid] = pair2(qzz[0], qzz[1]);
    }
    __syncthreads();

    // ---- per atom (one warp each, per candidate): K_i, rho, U', U'', chi; U table gradient
    for (int a = warp; a < na; a += nwarp) {
      double K[2];
      warp_slot_sums<2>(red, a_lo[a], a_lo[a + 1], lane, K);
      if (lane == 0) {
        const int i = a_idx[a];
        const int c0 = db.atom_cell[i];
        const SplineGeom &gU = sg[pot.s_U + db.atom_type[i]];
        const double w = db.cell_w[c0];
        for (int c = 0; c < nc; ++c) {
          const double rho = aos[c][AO_RHO * N + i];
          double rt = rho, dpen = 0.0, drt = 1.0;
          if (rho < gU.x0) {
            dpen = -w * 100.0 * 10. * 2.0 * (gU.x0 - rho);
            if (!pot.embed_extrap) { rt = gU.x0; drt = 0.0; }
          } else if (rho > gU.xN) {
            dpen = w * 100.0 * 10. * 2.0 * (rho - gU.xN);
            if (!pot.embed_extrap) { rt = gU.xN; drt = 0.0; }
          }
          const PointEval U = spl_point(tcs[c], gU, rt);
          const double eps = sds[c][CS_EPS * NC + c0], kap = sds[c][CS_KAPPA * NC + c0];
          a_chi[c * BLOCK_ATOMS + a] = (eps * U.grad + U.grad2 * K[c]) * drt + kap * dpen;
          a_dF[c * BLOCK_ATOMS + a] = U.grad;
          // into the warp's FP32 table (lane 0 alone writes it in this phase)
          float *fU = ft[c] + gU.toff;
          spl_point_adjoint(gU, U, rt, eps, K[c], [&](int idx, double v) { fU[idx] += (float)v; });
        }
        if (!twoc) {  // keep the unused half defined
          a_chi[BLOCK_ATOMS + a] = a_chi[a];
          a_dF[BLOCK_ATOMS + a] = a_dF[a];
        }
      }
    }
    __syncthreads();

    if (have) {
      double chi[2], dF[2];
      for (int c = 0; c < 2; ++c) {
        chi[c] = a_chi[c * BLOCK_ATOMS + me];
        dF[c] = a_dF[c * BLOCK_ATOMS + me];
      }
      const double ip = (double)invr;
      const float2 gam = pair2((float)(0.5 * chi[0] * (double)f.x + dF[0] * ap[0] * (double)df.x),
                               (float)(0.5 * chi[1] * (double)f.y + dF[1] * ap[1] * (double)df.y));
      const SplineGeom gg = sg[pot.s_g + ti];
      const int goff = gg.poff;
      const float gx0 = (float)gg.x0, ginv = (float)gg.invstep, gcut = gg.cutf;
      const int ngt = gg.n;
      // slope weight per candidate: dF f / r / h
      const float2 delh = pair2((float)(dF[0] * (double)f.x * ip) * ginv, (float)(dF[1] * (double)f.y * ip) * ginv);
      const float2 lx = pair2((float)Lx[0], (float)Lx[1]), ly = pair2((float)Ly[0], (float)Ly[1]),
                   lz = pair2((float)Lz[0], (float)Lz[1]);
      const float2 nap = pair2(-(float)ap[0], -(float)ap[1]);
      const float2 ux2 = bcast2(fux), uy2 = bcast2(fuy), uz2 = bcast2(fuz);
      float4 *ga = gacc + tid;
      const int row_lo = a_lo[me], row_hi = a_lo[me + 1];
      double dKdf[2] = {0.0, 0.0};
      const float2 zero = bcast2(0.f);
      for (int kb = row_lo; kb < row_hi; kb += 8) {
        float2 dk8 = zero;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int k = kb + u;
          const float4 o = srow[k];
          const float cs = cos_dot(fux, fuy, fuz, o.x, o.y, o.z);
          const bool ok = (k < row_hi) && (k != tid) && (cs < gcut);
          float b;
          const int m = g_knot<float>(cs, gx0, ginv, ngt, b);
          float2 dg;
          const float2 gv = cubic2_val_grad(pt2, npiece, goff, m, b, ginv, dg);
          const float4 q0 = sq0[k], q1 = sq1[k];
          const float2 qz = sqz[k];
          const float2 cs2 = bcast2(cs);
          // d K / d f_p from the triplet terms of slot k:
          //   a_k f'_k g - (a_k f_k / r_k) g' cos + g' (Q_k . u_p)
          const float2 qu = fma2(pair2(q1.x, q1.y), ux2, fma2(pair2(q1.z, q1.w), uy2, mul2(qz, uz2)));
          const float2 inner = fma2(mul2(pair2(q0.z, q0.w), cs2), bcast2(-1.f), qu);
          const float2 term = fma2(pair2(q0.x, q0.y), gv, mul2(dg, inner));
          const float2 fk = ok ? sf[k] : zero;
          if (ok) dk8 = add2(dk8, term);
          // g table (power basis): value weight cg = f_k gam, slope weight cs1 / h
          const float2 bpk = fma2(lx, bcast2(o.x), fma2(ly, bcast2(o.y), mul2(lz, bcast2(o.z))));
          const float2 cg = mul2(fk, gam);
          const float2 cs1 = mul2(mul2(fk, delh), fma2(nap, cs2, bpk));
          const float b2 = b * b;
          float4 d0 = ga[(2 * m) * BLOCK_SLOTS], d1 = ga[(2 * m + 1) * BLOCK_SLOTS];
          float2 dx = pair2(d0.x, d0.y), dy = pair2(d0.z, d0.w), dz = pair2(d1.x, d1.y), dw = pair2(d1.z, d1.w);
          dx = add2(dx, cg);
          dy = fma2(cg, bcast2(b), add2(dy, cs1));
          dz = fma2(cg, bcast2(b2), fma2(cs1, bcast2(2.f * b), dz));
          dw = fma2(cg, bcast2(b2 * b), fma2(cs1, bcast2(3.f * b2), dw));
          ga[(2 * m) * BLOCK_SLOTS] = make_float4(dx.x, dx.y, dy.x, dy.y);
          ga[(2 * m + 1) * BLOCK_SLOTS] = make_float4(dz.x, dz.y, dw.x, dw.y);
        }
        dKdf[0] += (double)dk8.x;
        dKdf[1] += (double)dk8.y;
      }
      // ---- pair-function tables of each candidate: phi (energy + force), rho (density + force), f
      for (int c = 0; c < nc; ++c) {
        dKdf[c] += ip * (J[c] - ap[c] * H[c]);
        float *ftc = ft[c];
        auto pair_adj = [&](int s, int k, float b, double cv, double cd) {
          const SplineGeom &g = sg[s];
          const SplW<double> w = spl_weights<double>((double)b, g.step, g.invstep);
          atomicAdd(ftc + g.toff + k, (float)(cv * w.wa + cd * w.da));
          atomicAdd(ftc + g.toff + k + 1, (float)(cv * w.wb + cd * w.db));
          atomicAdd(ftc + g.toff + g.n + k, (float)(cv * w.wA + cd * w.dA));
          atomicAdd(ftc + g.toff + g.n + k + 1, (float)(cv * w.wB + cd * w.dB));
        };
        const double eps = sds[c][CS_EPS * NC + cell];
        if (kphi >= 0) pair_adj(pot.s_phi + pij, kphi, bphi, 0.5 * eps, 0.5 * ap[c]);
        if (krho >= 0) pair_adj(pot.s_rho + tj, krho, brho, chi[c], dF[c] * ap[c]);
        if (kf >= 0) pair_adj(pot.s_f + pij, kf, bf, chi[c] * G[c] + dF[c] * dKdf[c], dF[c] * ap[c] * G[c]);
      }
    }
    if (++since_ft == FT_FLUSH_BLOCKS) {
      flush_ft();
      since_ft = 0;
    }
    if (++since_flush == GACC_FLUSH_BLOCKS) {
      flush_gacc(tab_t);
      since_flush = 0;
    }
  }
  if (since_ft > 0) flush_ft();
  __syncthreads();
  if (since_flush > 0 && tab_t >= 0) flush_gacc(tab_t);
  __threadfence_block();
  __syncthreads();
  // this CTA's partial of each candidate: the warps' tables summed in order
  for (int c = 0; c < nc; ++c) {
    const int cand = c ? cB : cA;
    const double *w0 = wglob + ((size_t)cand * gridDim.x + blockIdx.x) * ADJ_WARPS * stride;
    double *out = partial + ((size_t)cand * gridDim.x + blockIdx.x) * stride;
    for (int e = tid; e < stride; e += blockDim.x) {
      double s = 0.0;
      for (int w = 0; w < ADJ_WARPS; ++w) s += w0[(size_t)w * stride + e];
      out[e] = s;
    }
  }
}

}  // namespace mzb
