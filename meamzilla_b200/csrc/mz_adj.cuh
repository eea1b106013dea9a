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
#pragma once

#include "mz_fwd.cuh"

namespace mzb {

// Shared-memory layout of k_adj (dynamic), see adj_smem_bytes().
template <typename R>
__host__ __device__ inline size_t adj_smem_bytes(int nsplines, int stride, int pstride, bool meam) {
  size_t b = sizeof(double) * (size_t)ADJ_WARPS * stride;               // per-warp gradient tables
  if (meam) b += sizeof(double) * 2 * MAX_G_KNOTS * BLOCK_SLOTS;         // per-thread g tables
  b += sizeof(double) * (BLOCK_SLOTS + 2 * BLOCK_ATOMS);                 // red, a_chi, a_dF
  b += sizeof(SplineGeom) * nsplines;
  b += sizeof(int) * (BLOCK_ATOMS + 2);
  b = (b + 15) & ~size_t(15);
  b += sizeof(R) * (pstride + 4);
  b = (b + 15) & ~size_t(15);
  b += sizeof(R) * 9 * BLOCK_SLOTS;
  return b;
}

template <bool MEAM, typename R>
__global__ void __launch_bounds__(BLOCK_SLOTS)
    k_adj(DevDb db, DevPot pot, const SplineGeom *__restrict__ geom, const double *__restrict__ tabs,
          const double *__restrict__ ptabs, const double *__restrict__ aout, const double *__restrict__ aux, const double *__restrict__ lam,
          const double *__restrict__ seeds, double *__restrict__ partial) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int cand = blockIdx.y;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int N = db.natoms, NC = db.ncells;
  const int64_t Np = db.npairs;
  const int stride = pot.tab_stride;

  double *wtab = reinterpret_cast<double *>(smem_raw);
  double *gpriv = wtab + (size_t)ADJ_WARPS * stride;
  double *red = gpriv + (MEAM ? 2 * MAX_G_KNOTS * BLOCK_SLOTS : 0);
  double *a_chi = red + BLOCK_SLOTS;
  double *a_dF = a_chi + BLOCK_ATOMS;
  SplineGeom *sg = reinterpret_cast<SplineGeom *>(a_dF + BLOCK_ATOMS);
  int *a_lo = reinterpret_cast<int *>(sg + pot.nsplines);
  size_t off = reinterpret_cast<unsigned char *>(a_lo + BLOCK_ATOMS + 2) - smem_raw;
  off = (off + 15) & ~size_t(15);
  R *ptab = reinterpret_cast<R *>(smem_raw + off);
  off += sizeof(R) * (pot.pow_stride + 4);
  off = (off + 15) & ~size_t(15);
  R *sx = reinterpret_cast<R *>(smem_raw + off);
  R *sy = sx + BLOCK_SLOTS, *sz = sy + BLOCK_SLOTS, *sf = sz + BLOCK_SLOTS, *sal = sf + BLOCK_SLOTS,
    *sbe = sal + BLOCK_SLOTS, *sqx = sbe + BLOCK_SLOTS, *sqy = sqx + BLOCK_SLOTS, *sqz = sqy + BLOCK_SLOTS;

  const double *tc = tabs + (size_t)cand * stride;
  const double *pcand = ptabs + (size_t)cand * pot.pow_stride;
  for (int i = tid; i < pot.pow_stride; i += blockDim.x) ptab[i] = (R)pcand[i];
  for (int i = tid; i < ADJ_WARPS * stride; i += blockDim.x) wtab[i] = 0.0;
  if (MEAM)
    for (int i = tid; i < 2 * MAX_G_KNOTS * BLOCK_SLOTS; i += blockDim.x) gpriv[i] = 0.0;
  for (int i = tid; i < pot.nsplines; i += blockDim.x) sg[i] = geom[i];
  double *wt = wtab + (size_t)warp * stride;
  auto add_w = [&](int idx, double v) { atomicAdd(wt + idx, v); };

  const double *ao = aout + (size_t)cand * AO_COUNT * N;
  const double *ax = aux + (size_t)cand * AUX_COUNT * Np;
  const double *L = lam + (size_t)cand * 3 * N;
  const double *sd = seeds + (size_t)cand * CS_COUNT * NC;

  for (int blk = blockIdx.x; blk < db.nblocks; blk += gridDim.x) {
    const BlockRows br = block_rows(db, blk);
    __syncthreads();  // previous block done with the shared arrays
    for (int a = tid; a <= br.na; a += blockDim.x) a_lo[a] = db.pair_off[br.atom_lo + a] - br.slot_lo;
    __syncthreads();

    const bool have = tid < br.nslot;
    const int me = have ? slot_owner(a_lo, br.na, tid) : 0;
    const int ia = br.atom_lo + me;
    const int ti = db.atom_type[ia];
    const int64_t gs = (int64_t)br.slot_lo + tid;
    const int cell = db.atom_cell[ia];

    PairEval<MEAM, R> pe;
    double Lx = 0, Ly = 0, Lz = 0, a_p = 0, G = 0, H = 0, J = 0;
    if (have) {
      pe = eval_pair<MEAM, R>(db, pot, sg, ptab, gs, ti);
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
        sx[tid] = pe.ux; sy[tid] = pe.uy; sz[tid] = pe.uz; sf[tid] = pe.f;
        sal[tid] = (R)(a_p * (double)pe.df);
        sbe[tid] = (R)(a_p * fp * ip);
        sqx[tid] = (R)(fp * ip * Lx);
        sqy[tid] = (R)(fp * ip * Ly);
        sqz[tid] = (R)(fp * ip * Lz);
      }
      red[tid] = kp;
    }
    __syncthreads();

    // ---- per atom: K_i, rho, U', U'', chi = dL/drho; U table gradient
    if (tid < br.na) {
      const int i = br.atom_lo + tid;
      double K = 0.0;
      for (int s = a_lo[tid]; s < a_lo[tid + 1]; ++s) K += red[s];
      const double rho = ao[AO_RHO * N + i];
      const int c = db.atom_cell[i];
      const SplineGeom &gU = sg[pot.s_U + db.atom_type[i]];
      const double w = db.cell_w[c];
      double rt = rho, dpen = 0.0, drt = 1.0;
      if (rho < gU.x0) {
        dpen = -w * 100.0 * 10. * 2.0 * (gU.x0 - rho);
        if (!pot.embed_extrap) { rt = gU.x0; drt = 0.0; }
      } else if (rho > gU.xN) {
        dpen = w * 100.0 * 10. * 2.0 * (rho - gU.xN);
        if (!pot.embed_extrap) { rt = gU.xN; drt = 0.0; }
      }
      const PointEval U = spl_point(tc, gU, rt);
      const double eps = sd[CS_EPS * NC + c], kap = sd[CS_KAPPA * NC + c];
      a_chi[tid] = (eps * U.grad + U.grad2 * K) * drt + kap * dpen;
      a_dF[tid] = U.grad;
      const int toffU = gU.toff;
      spl_point_adjoint(gU, U, rt, eps, K, [&](int idx, double v) { add_w(toffU + idx, v); });
    }
    __syncthreads();

    if (have) {
      const double chi = a_chi[me], dF = a_dF[me];
      double dKdf = 0.0;
      if (MEAM) {
        const SplineGeom gg = sg[pot.s_g + ti];
        const R *gpc = ptab + gg.poff;
        const R gx0 = (R)gg.x0, ginv = (R)gg.invstep, gst = (R)gg.step;
        const R gcut = g_cut<R>(gg);
        const int ng = gg.n;
        const double fp = (double)pe.f, ip = (double)pe.invr;
        const double gam = 0.5 * chi * fp + dF * a_p * (double)pe.df;
        const double del = dF * fp * ip;
        double *gp = gpriv + tid;
        const int row_lo = a_lo[me], row_hi = a_lo[me + 1];
        for (int k = row_lo; k < row_hi; ++k) {
          if (k == tid) continue;
          const R fk = sf[k], alk = sal[k];
          if (fk == R(0) && alk == R(0)) continue;
          const R kx = sx[k], ky = sy[k], kz = sz[k];
          const R cs = cos_exact(pe.ux, pe.uy, pe.uz, kx, ky, kz);
          if (!(cs < gcut)) continue;
          R b;
          const int m = g_knot<R>(cs, gx0, ginv, ng, b);
          R dg;
          const R gv = cubic_val_grad<R>(gpc, m, b, ginv, dg);
          // d K / d f_p from the triplet terms of slot k
          const R qu = sqx[k] * pe.ux + sqy[k] * pe.uy + sqz[k] * pe.uz;
          dKdf += (double)(alk * gv - sbe[k] * dg * cs + dg * qu);
          // g table: value weight cg, slope weight cgp of this ordered pair
          const double bpk = Lx * (double)kx + Ly * (double)ky + Lz * (double)kz;
          const double cg = (double)fk * gam;
          const double cgp = (double)fk * del * (bpk - a_p * (double)cs);
          const SplW<R> w = spl_weights<R>(b, gst, ginv);
          gp[m * BLOCK_SLOTS] += cg * (double)w.wa + cgp * (double)w.da;
          gp[(m + 1) * BLOCK_SLOTS] += cg * (double)w.wb + cgp * (double)w.db;
          gp[(ng + m) * BLOCK_SLOTS] += cg * (double)w.wA + cgp * (double)w.dA;
          gp[(ng + m + 1) * BLOCK_SLOTS] += cg * (double)w.wB + cgp * (double)w.dB;
        }
        dKdf += ip * (J - a_p * H);
      }
      // ---- pair-function tables: phi (energy + force), rho (density + force), f
      auto pair_adj = [&](int s, int k, R b, double cv, double cd) {
        const SplineGeom &g = sg[s];
        const SplW<double> w = spl_weights<double>((double)b, g.step, g.invstep);
        add_w(g.toff + k, cv * w.wa + cd * w.da);
        add_w(g.toff + k + 1, cv * w.wb + cd * w.db);
        add_w(g.toff + g.n + k, cv * w.wA + cd * w.dA);
        add_w(g.toff + g.n + k + 1, cv * w.wB + cd * w.dB);
      };
      const double eps = sd[CS_EPS * NC + cell];
      if (pe.kphi >= 0) pair_adj(pot.s_phi + pe.pij, pe.kphi, pe.bphi, 0.5 * eps, 0.5 * a_p);
      if (pe.krho >= 0) pair_adj(pot.s_rho + pe.tj, pe.krho, pe.brho, chi, dF * a_p);
      if (MEAM && pe.kf >= 0) pair_adj(pot.s_f + pe.pij, pe.kf, pe.bf, chi * G + dF * dKdf, dF * a_p * G);
    }
    __syncwarp();
    if (MEAM) {
      // flush the per-thread g tables into the warp's table, per g spline
      for (int t = 0; t < pot.ntypes; ++t) {
        const SplineGeom &gg = sg[pot.s_g + t];
        const int ng = gg.n;
        for (int e = 0; e < 2 * ng; ++e) {
          double v = (have && ti == t) ? gpriv[e * BLOCK_SLOTS + tid] : 0.0;
          for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
          if (lane == 0 && v != 0.0) wt[gg.toff + e] += v;
        }
      }
      if (have) {
        const int ng = sg[pot.s_g + ti].n;
        for (int e = 0; e < 2 * ng; ++e) gpriv[e * BLOCK_SLOTS + tid] = 0.0;
      }
    }
  }
  __syncthreads();
  double *out = partial + ((size_t)cand * gridDim.x + blockIdx.x) * stride;
  for (int e = tid; e < stride; e += blockDim.x) {
    double s = 0.0;
    for (int w = 0; w < ADJ_WARPS; ++w) s += wtab[(size_t)w * stride + e];
    out[e] = s;
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
  if (t == 0) {
    if (pot.style == MZ_STYLE_MEAM_SPLINE) {
      int at = -1;
      const double my = f_max_y(pot, geom, tab, &at);
      const double m = fabs(my);
      const double fe = 100. * 25. * (1.0 - m) * (1.0 - m);
      if (at >= 0) ext[at] += 2.0 * fe * (-5000.0) * (1.0 - m) * (my > 0 ? 1.0 : (my < 0 ? -1.0 : 0.0));
    } else {
      for (int ty = 0; ty < pot.ntypes; ++ty) {
        const SplineGeom &g = geom[pot.s_U + ty];
        const double mid = 0.5 * (g.x0 + g.xN);
        const PointEval e = spl_point(tab, g, mid);
        const double ev = 100. * e.grad;
        const int to = g.toff;
        spl_point_adjoint(g, e, mid, 0.0, 2.0 * ev * 100.0, [&](int idx, double v) { ext[to + idx] += v; });
      }
    }
  }
  __syncthreads();
  double *gc = grad + (size_t)c * P;
  for (int s = t; s < pot.nsplines; s += blockDim.x) {
    const SplineGeom g = geom[s];
    const int n = g.n;
    for (int col = 0; col < n + 2; ++col) {
      double acc = col < n ? ext[g.toff + col] : ext[g.toff + 2 * n + (col - n)];
      for (int r = 0; r < n; ++r) acc += M[g.moff + r * (n + 2) + col] * ext[g.toff + n + r];
      const int ci = col < n ? cmap[g.toff + col] : cmap[g.toff + 2 * n + (col - n)];
      if (ci >= 0) gc[ci] = acc;
    }
  }
}

}  // namespace mzb
