// Mixed-precision MEAM forward with two candidates per CTA.
//
// Every triplet's geometry -- the cosine, its g interval and shift, the
// triplet mask -- is the same for all candidates; only the spline pieces and
// the partners' f values differ.  This kernel computes the geometry once per
// (slot, partner) and evaluates both candidates' pieces and row sums as FP32
// pairs with the sm_100 packed instructions (__ffma2_rn and friends, one
// instruction for two lanes of arithmetic).  The two candidates' evaluation
// tables are interleaved in shared memory -- for piece i (over all splines)
// lo[i] = (c0 A, c0 B, c1 A, c1 B) and hi[i] = (c2 A, c2 B, c3 A, c3 B) in two
// arrays with a 16-byte stride -- so that one 16-byte load brings two
// coefficient pairs of both.  Results per candidate are those of k_atoms'
// mixed path up to the order of FP32 additions inside each chunk of 8
// partners (the chunk sums are added to FP64 totals as there).
//
// Scope: meam/spline with spline3eq pieces (the g of Triplet_i); the other
// styles keep the one-candidate kernel.
#pragma once

#include <type_traits>

#include "mz_fwd.cuh"

namespace mzb {

__device__ __forceinline__ float2 pair2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 bcast2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }

// Value and slope of piece k of the spline at evaluation-table offset `off`
// (a multiple of 4), for both candidates of the interleaved table pt2: lo
// pairs at pt2[i], hi pairs at pt2[npiece + i], i = off / 4 + k.
__device__ __forceinline__ float2 cubic2_val_grad(const float4 *pt2, int npiece, int off, int k, float b, float inv,
                                                  float2 &grad) {
  const int i = (off >> 2) + k;
  const float4 lo = pt2[i];           // c0A c0B c1A c1B
  const float4 hi = pt2[npiece + i];  // c2A c2B c3A c3B
  const float2 c0 = pair2(lo.x, lo.y), c1 = pair2(lo.z, lo.w), c2 = pair2(hi.x, hi.y), c3 = pair2(hi.z, hi.w);
  const float2 bb = bcast2(b);
  const float2 slope = fma2(bb, fma2(bcast2(3.f * b), c3, add2(c2, c2)), c1);  // c1 + b (2 c2 + 3 b c3)
  grad = mul2(slope, bcast2(inv));
  return fma2(bb, fma2(bb, fma2(bb, c3, c2), c1), c0);
}

// Shared-memory layout of k_atoms2 (dynamic), see atoms2_smem_bytes():
//   double red[10][BLOCK_SLOTS]        per-slot partials for the per-atom sums
//   double a_dF[2][BLOCK_ATOMS], a_U[2][BLOCK_ATOMS]
//   SplineGeom sg[nsplines]
//   int a_lo[BLOCK_ATOMS+2]
//   float4 pt2[2][pstride / 4 + 1]     the two candidates' evaluation tables, interleaved
//   float4 srow[BLOCK_SLOTS+8]         (u_x, u_y, u_z, 0) of every slot
//   float2 sf[BLOCK_SLOTS+8]           (f of candidate A, f of candidate B) of every slot
__host__ __device__ inline size_t atoms2_smem_bytes(int nsplines, int pstride) {
  size_t b = sizeof(double) * (10 * BLOCK_SLOTS + 4 * BLOCK_ATOMS);
  b += sizeof(SplineGeom) * nsplines;
  b += sizeof(int) * (BLOCK_ATOMS + 2);
  b = (b + 31) & ~size_t(31);
  b += sizeof(float4) * 2 * ((size_t)pstride / 4 + 1);
  b = (b + 31) & ~size_t(31);
  b += sizeof(float4) * (BLOCK_SLOTS + 8);
  b += sizeof(float2) * (BLOCK_SLOTS + 8);
  return b;
}

// Both candidates' evaluation tables into the interleaved layout.
__device__ __forceinline__ void load_pt2(float4 *pt2, const double *pcA, const double *pcB, int pstride) {
  const int np = pstride / 4;
  for (int i = threadIdx.x; i < np; i += blockDim.x) {
    const double *a = pcA + 4 * i, *b = pcB + 4 * i;
    pt2[i] = make_float4((float)a[0], (float)b[0], (float)a[1], (float)b[1]);
    pt2[np + i] = make_float4((float)a[2], (float)b[2], (float)a[3], (float)b[3]);
  }
}

// One CTA per (atom block, candidate pair), one thread per pair slot;
// candidates 2 y and 2 y + 1 (the last CTA of an odd count evaluates its
// single candidate twice and writes it once).  The arithmetic of each
// candidate follows k_atoms (pot_meam_spline.cpp:143-269).
template <bool AUX>
__global__ void __launch_bounds__(BLOCK_SLOTS, 4)
    k_atoms2(DevDb db, DevPot pot, const SplineGeom *__restrict__ geom, const double *__restrict__ tabs,
             const double *__restrict__ ptabs, double *__restrict__ Vout, double *__restrict__ aout,
             double *__restrict__ aux, int ncand) {
  extern __shared__ __align__(32) unsigned char smem_raw[];
  const int cA = 2 * blockIdx.y;
  const bool twoc = cA + 1 < ncand;
  const int cB = twoc ? cA + 1 : cA;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
  const int N = db.natoms;
  const int64_t Np = db.npairs;

  double *red = reinterpret_cast<double *>(smem_raw);
  double *a_dF = red + 10 * BLOCK_SLOTS;   // [2][BLOCK_ATOMS]
  double *a_U = a_dF + 2 * BLOCK_ATOMS;    // [2][BLOCK_ATOMS]
  SplineGeom *sg = reinterpret_cast<SplineGeom *>(a_U + 2 * BLOCK_ATOMS);
  int *a_lo = reinterpret_cast<int *>(sg + pot.nsplines);
  size_t off = sizeof(double) * (10 * BLOCK_SLOTS + 4 * BLOCK_ATOMS) + sizeof(SplineGeom) * pot.nsplines +
               sizeof(int) * (BLOCK_ATOMS + 2);
  off = (off + 31) & ~size_t(31);
  float4 *pt2 = reinterpret_cast<float4 *>(smem_raw + off);
  const int npiece = pot.pow_stride / 4;
  off += sizeof(float4) * 2 * ((size_t)npiece + 1);
  off = (off + 31) & ~size_t(31);
  float4 *srow = reinterpret_cast<float4 *>(smem_raw + off);
  float2 *sf = reinterpret_cast<float2 *>(srow + BLOCK_SLOTS + 8);

  const BlockRows br = block_rows(db, blockIdx.x);
  load_pt2(pt2, ptabs + (size_t)cA * pot.pow_stride, ptabs + (size_t)cB * pot.pow_stride, pot.pow_stride);
  for (int i = tid; i < pot.nsplines; i += blockDim.x) sg[i] = geom[i];
  for (int a = tid; a <= br.na; a += blockDim.x) a_lo[a] = db.pair_off[br.atom_lo + a] - br.slot_lo;
  __syncthreads();

  const bool have = tid < br.nslot;
  const int me = have ? slot_owner(a_lo, br.na, tid) : 0;
  const int ti = db.atom_type[br.atom_lo + me];
  const int64_t gs = (int64_t)br.slot_lo + tid;

  // ---- the slot's pair functions for both candidates (pot_meam_spline.cpp:152-191)
  float ux = 0.f, uy = 0.f, uz = 0.f, invr = 0.f;
  float2 phi = bcast2(0.f), dphi = phi, rho = phi, drho = phi, f = phi, df = phi;
  if (have) {
    ux = db.pair_uxf[gs];
    uy = db.pair_uyf[gs];
    uz = db.pair_uzf[gs];
    invr = 1.f / db.pair_rf[gs];
    const int kn = db.pair_knot[gs];
    const int kphi = (kn & 0xff) - 1, krho = ((kn >> 8) & 0xff) - 1, kf = ((kn >> 16) & 0xff) - 1;
    const int tj = db.atom_type[db.pair_nbr[gs]];
    const int pij = pair_ij_index(ti, tj, pot.ntypes);
    if (kphi >= 0) {
      const SplineGeom &g = sg[pot.s_phi + pij];
      phi = cubic2_val_grad(pt2, npiece, g.poff, kphi, db.pair_shiftf[gs], (float)g.invstep, dphi);
    }
    if (krho >= 0) {
      const SplineGeom &g = sg[pot.s_rho + tj];
      rho = cubic2_val_grad(pt2, npiece, g.poff, krho, db.pair_shiftf[Np + gs], (float)g.invstep, drho);
    }
    if (kf >= 0) {
      const SplineGeom &g = sg[pot.s_f + pij];
      f = cubic2_val_grad(pt2, npiece, g.poff, kf, db.pair_shiftf[2 * Np + gs], (float)g.invstep, df);
    }
  }
  srow[tid] = make_float4(ux, uy, uz, 0.f);
  sf[tid] = f;
  if (tid < 8) {
    srow[BLOCK_SLOTS + tid] = make_float4(0.f, 0.f, 0.f, 0.f);
    sf[BLOCK_SLOTS + tid] = bcast2(0.f);
  }
  __syncthreads();

  // ---- the one pass over the row: G_p, H_p, vk_p of both candidates
  double G[2] = {0, 0}, H[2] = {0, 0}, vx[2] = {0, 0}, vy[2] = {0, 0}, vz[2] = {0, 0};
  if (have && (AUX || f.x != 0.f || f.y != 0.f || df.x != 0.f || df.y != 0.f)) {
    const SplineGeom gg = sg[pot.s_g + ti];
    const int goff = gg.poff;
    const float gx0 = (float)gg.x0, ginv = (float)gg.invstep, gcut = gg.cutf;
    const int row_lo = a_lo[me], row_hi = a_lo[me + 1];
    const float2 zero = bcast2(0.f);
    auto chunk = [&](int kb, auto NK) {
      constexpr int nk = decltype(NK)::value;
      float2 g8 = zero, h8 = zero, x8 = zero, y8 = zero, z8 = zero;
#pragma unroll
      for (int u = 0; u < nk; ++u) {
        const int k = kb + u;
        const float4 o = srow[k];
        const float cs = cos_dot(ux, uy, uz, o.x, o.y, o.z);
        const bool ok = (k < row_hi) && (k != tid) && (cs < gcut);  // triplet_meam_spline.cpp:66-70
        const float2 fk = ok ? sf[k] : zero;
        float b;
        const int kk = g_knot<float>(cs, gx0, ginv, gg.n, b);
        float2 dg;
        const float2 gv = cubic2_val_grad(pt2, npiece, goff, kk, b, ginv, dg);
        const float2 dgfk = mul2(dg, fk);
        g8 = fma2(gv, fk, g8);
        h8 = fma2(dgfk, bcast2(cs), h8);
        x8 = fma2(dgfk, bcast2(o.x), x8);
        y8 = fma2(dgfk, bcast2(o.y), y8);
        z8 = fma2(dgfk, bcast2(o.z), z8);
      }
      G[0] += (double)g8.x;
      G[1] += (double)g8.y;
      H[0] += (double)h8.x;
      H[1] += (double)h8.y;
      vx[0] += (double)x8.x;
      vx[1] += (double)x8.y;
      vy[0] += (double)y8.x;
      vy[1] += (double)y8.y;
      vz[0] += (double)z8.x;
      vz[1] += (double)z8.y;
    };
    // steps of 8 partners, the rest of the row in steps of 4
    int kb = row_lo;
    for (; kb + 8 <= row_hi; kb += 8) chunk(kb, std::integral_constant<int, 8>{});
    if (kb + 4 <= row_hi) {
      chunk(kb, std::integral_constant<int, 4>{});
      kb += 4;
    }
    if (kb < row_hi) chunk(kb, std::integral_constant<int, 4>{});
    if (AUX)
      for (int c = 0; c < (twoc ? 2 : 1); ++c) {
        double *ax = aux + (size_t)(cA + c) * AUX_COUNT * Np;
        ax[AUX_G * Np + gs] = G[c];
        ax[AUX_H * Np + gs] = H[c];
        ax[AUX_VX * Np + gs] = vx[c];
        ax[AUX_VY * Np + gs] = vy[c];
        ax[AUX_VZ * Np + gs] = vz[c];
      }
  }
  if (have) {
    red[tid] = (double)rho.x + 0.5 * (double)f.x * G[0];
    red[BLOCK_SLOTS + tid] = (double)rho.y + 0.5 * (double)f.y * G[1];
  }
  __syncthreads();

  // ---- embedding of both candidates (pot_meam_spline.cpp:208-223): one warp per atom
  for (int a = warp; a < br.na; a += nwarp) {
    double rr[2];
    warp_slot_sums<2>(red, a_lo[a], a_lo[a + 1], lane, rr);
    if (lane == 0) {
      const int ia = br.atom_lo + a;
      const SplineGeom &gU = sg[pot.s_U + db.atom_type[ia]];
      const double w = db.cell_w[db.atom_cell[ia]];
      for (int c = 0; c < 2; ++c) {
        double r = rr[c], pen = 0.0;
        const double raw = r;
        if (r < gU.x0) {
          pen = w * 100.0 * 10. * (gU.x0 - r) * (gU.x0 - r);
          if (!pot.embed_extrap) r = gU.x0;
        } else if (r > gU.xN) {
          pen = w * 100.0 * 10. * (r - gU.xN) * (r - gU.xN);
          if (!pot.embed_extrap) r = gU.xN;
        }
        const PointEval U = spl_point(tabs + (size_t)(cA + (c ? cB - cA : 0)) * pot.tab_stride, gU, r);
        a_dF[c * BLOCK_ATOMS + a] = U.grad;
        a_U[c * BLOCK_ATOMS + a] = U.val;
        if (c == 0 || twoc) {
          double *ao = aout + (size_t)(cA + c) * AO_COUNT * N;
          ao[AO_PEN * N + ia] = pen;
          ao[AO_RHO * N + ia] = raw;
        }
      }
    }
  }
  __syncthreads();

  // ---- V_p and the slot's stress, one candidate after the other
  for (int c = 0; c < (twoc ? 2 : 1); ++c) {
    const int cand = cA + c;
    if (have) {
      const double dF = a_dF[c * BLOCK_ATOMS + me];
      const double fp = c ? (double)f.y : (double)f.x, dfp = c ? (double)df.y : (double)df.x;
      const double ip = (double)invr;
      double cu = 0.5 * (c ? (double)dphi.y : (double)dphi.x) + (c ? (double)drho.y : (double)drho.x) * dF;
      cu += dF * (dfp * G[c] - fp * ip * H[c]);
      const double ck = dF * fp * ip;
      const double Vx = ck * vx[c] + (double)ux * cu, Vy = ck * vy[c] + (double)uy * cu,
                   Vz = ck * vz[c] + (double)uz * cu;
      double *Vc = Vout + (size_t)cand * 3 * Np + 3 * gs;  // (x, y, z) per slot
      Vc[0] = Vx;
      Vc[1] = Vy;
      Vc[2] = Vz;
      const double r = db.pair_r[gs];
      const double dx = db.pair_ux[gs], dy = db.pair_uy[gs], dz = db.pair_uz[gs];
      red[0 * BLOCK_SLOTS + tid] = Vx;
      red[1 * BLOCK_SLOTS + tid] = Vy;
      red[2 * BLOCK_SLOTS + tid] = Vz;
      red[3 * BLOCK_SLOTS + tid] = 0.5 * (c ? (double)phi.y : (double)phi.x);
      red[4 * BLOCK_SLOTS + tid] = -(dx * (Vx * r));
      red[5 * BLOCK_SLOTS + tid] = -(dy * (Vy * r));
      red[6 * BLOCK_SLOTS + tid] = -(dz * (Vz * r));
      red[7 * BLOCK_SLOTS + tid] = -(dx * (Vy * r));
      red[8 * BLOCK_SLOTS + tid] = -(dy * (Vz * r));
      red[9 * BLOCK_SLOTS + tid] = -(dz * (Vx * r));
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
        ao[AO_E * N + ia] = acc[3] + a_U[c * BLOCK_ATOMS + a];
#pragma unroll
        for (int q = 0; q < 6; ++q) ao[(AO_S0 + q) * N + ia] = acc[4 + q];
      }
    }
    __syncthreads();
  }
}

}  // namespace mzb
