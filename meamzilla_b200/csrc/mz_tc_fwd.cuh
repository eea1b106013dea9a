// Mixed-precision MEAM forward pass with the triplet sums on the tensor
// cores (tcgen05, kind::tf32, accumulator in tensor memory).
//
// For slot j of atom i the triplet sums of the one-pass forward are
//   G_j    = sum_k g(cos_jk) f_k
//   vkp_j  = sum_k g'(cos_jk) f_k (u_k - cos_jk u_j)      (the part of vk
//            perpendicular to u_j; the parallel part cancels in V_j)
// Written in the cubic B-spline basis of g (g(x) = sum_n w_n B_n(x), the
// w_n follow from the knot table: w_{i+1} = y_i - h^2/6 y''_i), every sum
// splits into candidate coefficients times geometry:
//   G_j   = sum_n w_n  sum_k f_k B_n(cos_jk)                 = sum_n w_n D[(j,n)]
//   vkp_j = 1/h sum_n dw_n sum_k f_k Q_n(cos_jk) (u_k.e1_j, u_k.e2_j)
// with (e1_j, e2_j) an orthonormal pair perpendicular to u_j, and g' in the
// quadratic B-spline basis Q_n with coefficients dw_n = w_n+1 - w_n (formed
// in FP64: contracting the cubic basis' slopes, which sum to zero, with
// w_n near 1 would cancel).  For all
// candidates of the CTA at once, D = F Phi^T with
//   F   [candidate][k]        f of partner k under each candidate (the A operand)
//   Phi [(j, feature)][k]     B_n, Q_n u.e1, Q_n u.e2 of each pair (j, k) (the B operand)
// one MMA of M = 128 rows, N = 28 features x 8 slots, K = 8 partners per
// instruction.  FP32 accuracy from TF32 operands: F and Phi are split
// x = hi + lo (both TF32); rows 0-63 of A hold F_hi, rows 64-127 F_lo, and
// two MMAs (B = Phi_hi, Phi_lo) give hi*hi + hi*lo + lo*hi + lo*lo, summed
// over the two row halves in the epilogue.  The epilogue (one thread per
// TMEM lane = candidate) contracts D with the candidate's w_n.  Everything
// after the triplet sums (density, U, reaction vectors, per-atom sums) is
// the one-pass forward's arithmetic (k_atoms) with one warp per
// (candidate, 32 slots).
//
// The reference computes the same sums triplet by triplet
// (PotMEAMSpline::fast_compute, pot_meam_spline.cpp:143-269).
#pragma once

#include <algorithm>

#include "mz_fwd.cuh"
#include "mz_tc.cuh"

namespace mzb {

constexpr int TC_CANDS = 64;    // candidates of one CTA (MMA rows: hi 0-63, lo 64-127)
constexpr int TC_THREADS = 256;
constexpr int TC_MAX_KC = 3;    // 32-partner K chunks: rows of at most 96 slots
constexpr int TC_TMEM_COLS = 256;
constexpr int TC_NB = 10;       // B-spline coefficients of the g splines the kernel is built for (8 knots)
constexpr uint32_t TC_WAIT_LIMIT = 1u << 22;

// Launch geometry and shared-memory carve-up (byte offsets from the 1 KiB
// aligned base), filled on the host by tc_plan().
struct TcParams {
  int kc;        // K chunks for the longest row
  int smax;      // kc * 32
  int J;         // slots per j-group (N = J * 3 NB <= 256)
  int gp_pitch;  // floats per candidate row of the G / psi array (odd)
  int off_a, off_bhi, off_blo, off_gp, off_geo, off_w, off_sg, off_part, off_u, off_bar;
  int smem_bytes;
};

template <int NB>
struct TcShape {
  static constexpr int F = 3 * NB - 2;                   // features per slot: NB values, 2 x (NB-1) slopes
  static constexpr int NW = 2 * NB - 1;                  // coefficients per g spline: w, dw
  static constexpr int NLD = (F + 15) / 16;              // 16-column TMEM loads per slot
};

// Per-slot geometry staged in shared memory (16 floats):
//   [0..3] u_x u_y u_z r   [4..6] e1   [7] phi shift   [8..10] e2  [11] rho shift
//   [12] f shift  [13] packed knots (int)  [14] neighbour type (int)  [15] -
constexpr int TC_GEO = 16;

__device__ __forceinline__ void perp_pair(float ux, float uy, float uz, float *e1, float *e2) {
  const float ax = fabsf(ux), ay = fabsf(uy), az = fabsf(uz);
  float x, y, z;  // u x (the axis of the smallest component of u)
  if (ax <= ay && ax <= az) {
    x = 0.f; y = uz; z = -uy;
  } else if (ay <= az) {
    x = -uz; y = 0.f; z = ux;
  } else {
    x = uy; y = -ux; z = 0.f;
  }
  const float inv = rsqrtf(x * x + y * y + z * z);
  e1[0] = x * inv; e1[1] = y * inv; e1[2] = z * inv;
  e2[0] = uy * e1[2] - uz * e1[1];
  e2[1] = uz * e1[0] - ux * e1[2];
  e2[2] = ux * e1[1] - uy * e1[0];
}

// FP32 cubic of one pair function at a staged slot (value and slope).
__device__ __forceinline__ float tc_pair_fn(const float *ptab, const SplineGeom &g, int k, float b, float &d) {
  const float4 c = __ldg(reinterpret_cast<const float4 *>(ptab + g.poff + 4 * k));
  const float inv = (float)g.invstep;
  d = (c.y + b * (2.f * c.z + 3.f * b * c.w)) * inv;
  return c.x + b * (c.y + b * (c.z + b * c.w));
}

template <int NB, bool AUX>
__global__ void __launch_bounds__(TC_THREADS, 1)
    k_atoms_tc(DevDb db, DevPot pot, TcParams tp, const SplineGeom *__restrict__ geom,
               const double *__restrict__ tabs, const float *__restrict__ ptabf, const float *__restrict__ wtab,
               int ncand, double *__restrict__ Vout, double *__restrict__ aout, double *__restrict__ aux,
               int *__restrict__ err) {
  constexpr int F = TcShape<NB>::F;
  extern __shared__ __align__(1024) unsigned char tc_raw[];
  unsigned char *base = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(tc_raw) + 1023) &
                                                          ~static_cast<uintptr_t>(1023));
  unsigned char *sA = base + tp.off_a;
  unsigned char *sBh = base + tp.off_bhi;
  unsigned char *sBl = base + tp.off_blo;
  float *gp = reinterpret_cast<float *>(base + tp.off_gp);
  float *geo = reinterpret_cast<float *>(base + tp.off_geo);
  float *wsm = reinterpret_cast<float *>(base + tp.off_w);
  SplineGeom *sg = reinterpret_cast<SplineGeom *>(base + tp.off_sg);
  double *part = reinterpret_cast<double *>(base + tp.off_part);
  double *sU = reinterpret_cast<double *>(base + tp.off_u);  // [0,64) U, [64,128) U'
  uint64_t *bar = reinterpret_cast<uint64_t *>(base + tp.off_bar);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int cg = blockIdx.y * TC_CANDS;
  const int C = min(TC_CANDS, ncand - cg);
  const int N = db.natoms;
  const int64_t Np = db.npairs;
  const int nt = pot.ntypes;
  const int pitch = tp.gp_pitch;

  for (int i = tid; i < pot.nsplines; i += TC_THREADS) sg[i] = geom[i];
  constexpr int NW = TcShape<NB>::NW;
  for (int i = tid; i < TC_CANDS * nt * NW; i += TC_THREADS) {
    const int c = i / (nt * NW);
    wsm[i] = c < C ? wtab[(size_t)(cg + c) * nt * NW + (i - c * nt * NW)] : 0.f;
  }
  {  // B tiles start zeroed; each (j-slot, partner) column is then cleared and rewritten incrementally
    float4 *b4 = reinterpret_cast<float4 *>(sBh);
    const int nb4 = (tp.off_gp - tp.off_bhi) / 16;
    for (int i = tid; i < nb4; i += TC_THREADS) b4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  if (tid == 0) tc::mbar_init(bar, 1);
  if (warp == 0) tc::tmem_alloc(tslot, TC_TMEM_COLS);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tm = *tslot;
  uint32_t phase = 0;
  int prev_kk = -1;  // rows this thread's feature column holds nonzeros at (interval), -1 none

  for (int ia = blockIdx.x; ia < N; ia += gridDim.x) {
    const int s0 = db.pair_off[ia];
    const int n = db.pair_off[ia + 1] - s0;
    const int ti = db.atom_type[ia];
    const int kcu = (n + 31) >> 5;
    __syncthreads();  // the previous atom is done with the shared arrays

    // ---- stage the row: FP32 geometry, perpendicular pair, shifts, knots
    for (int k = tid; k < kcu * 32; k += TC_THREADS) {
      float *q = geo + k * TC_GEO;
      if (k < n) {
        const int64_t s = (int64_t)s0 + k;
        const float ux = db.pair_uxf[s], uy = db.pair_uyf[s], uz = db.pair_uzf[s];
        float e1[3], e2[3];
        perp_pair(ux, uy, uz, e1, e2);
        q[0] = ux; q[1] = uy; q[2] = uz; q[3] = db.pair_rf[s];
        q[4] = e1[0]; q[5] = e1[1]; q[6] = e1[2]; q[7] = db.pair_shiftf[s];
        q[8] = e2[0]; q[9] = e2[1]; q[10] = e2[2]; q[11] = db.pair_shiftf[Np + s];
        q[12] = db.pair_shiftf[2 * Np + s];
        q[13] = __int_as_float(db.pair_knot[s]);
        q[14] = __int_as_float(db.atom_type[db.pair_nbr[s]]);
        q[15] = 0.f;
      } else {
#pragma unroll
        for (int u = 0; u < TC_GEO; ++u) q[u] = 0.f;
      }
    }
    for (int i = tid; i < TC_CANDS * pitch; i += TC_THREADS) gp[i] = 0.f;
    __syncthreads();

    // ---- A operand: f of every partner under every candidate, split hi / lo
    for (int i = tid; i < TC_CANDS * kcu * 32; i += TC_THREADS) {
      const int c = i / (kcu * 32), k = i - c * (kcu * 32);
      float f = 0.f;
      if (c < C && k < n) {
        const float *q = geo + k * TC_GEO;
        const int kn = __float_as_int(q[13]);
        const int kf = ((kn >> 16) & 0xff) - 1;
        if (kf >= 0) {
          const int pij = pair_ij_index(ti, __float_as_int(q[14]), nt);
          float d;
          f = tc_pair_fn(ptabf + (size_t)(cg + c) * pot.pow_stride, sg[pot.s_f + pij], kf, q[12], d);
        }
      }
      float hi, lo;
      tc::split_tf32(f, hi, lo);
      unsigned char *A = sA + (k >> 5) * 16384;
      *reinterpret_cast<float *>(A + tc::sw128_off(c, k & 31)) = hi;
      *reinterpret_cast<float *>(A + tc::sw128_off(64 + c, k & 31)) = lo;
    }

    // epilogue constants of this thread's TMEM lane (candidate c, row half)
    const int quarter = warp & 3;
    const int c_ep = (32 * quarter + lane) & 63;
    float wr[NW];
#pragma unroll
    for (int u = 0; u < NW; ++u) wr[u] = wsm[(c_ep * nt + ti) * NW + u];
    const SplineGeom gg = sg[pot.s_g + ti];
    const float gx0 = (float)gg.x0, ginv = (float)gg.invstep, gcut = g_cut<float>(gg);

    for (int j0 = 0; j0 < n; j0 += tp.J) {
      const int jc = min(tp.J, n - j0);
      const int npad = ((jc * F + 15) / 16) * 16;
      for (int q = 0; q < kcu; ++q) {
        // ---- B operand: warp = slot of the group, lane = partner of the chunk
        if (warp < tp.J) {
          const int j = j0 + warp, k = 32 * q + lane;
          const int rb = warp * F;
          if (prev_kk >= 0) {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              const uint32_t o = tc::sw128_off(rb + prev_kk + u, lane);
              *reinterpret_cast<float *>(sBh + o) = 0.f;
              *reinterpret_cast<float *>(sBl + o) = 0.f;
            }
#pragma unroll
            for (int u = 0; u < 3; ++u)
#pragma unroll
              for (int sct = 0; sct < 2; ++sct) {
                const uint32_t o = tc::sw128_off(rb + NB + sct * (NB - 1) + prev_kk + u, lane);
                *reinterpret_cast<float *>(sBh + o) = 0.f;
                *reinterpret_cast<float *>(sBl + o) = 0.f;
              }
            prev_kk = -1;
          }
          if (warp < jc && k < n && k != j) {
            const float *pj = geo + j * TC_GEO, *pk = geo + k * TC_GEO;
            const float cs = cos_dot(pj[0], pj[1], pj[2], pk[0], pk[1], pk[2]);
            if (cs < gcut) {  // triplet_meam_spline.cpp:66-70
              float b;
              const int kk = g_knot<float>(cs, gx0, ginv, gg.n, b);
              const float a = 1.f - b;
              const float bv[4] = {a * a * a * (1.f / 6.f), (2.f / 3.f) - b * b + 0.5f * b * b * b,
                                   (2.f / 3.f) - a * a + 0.5f * a * a * a, b * b * b * (1.f / 6.f)};
              // quadratic B-splines: d/db sum_u w_kk+u B_u = sum_u dw_kk+u Q_u
              const float qv[3] = {0.5f * a * a, 0.5f + b * a, 0.5f * b * b};
              const float p1 = pk[0] * pj[4] + pk[1] * pj[5] + pk[2] * pj[6];
              const float p2 = pk[0] * pj[8] + pk[1] * pj[9] + pk[2] * pj[10];
#pragma unroll
              for (int u = 0; u < 4; ++u) {
                float hi, lo;
                tc::split_tf32(bv[u], hi, lo);
                const uint32_t o = tc::sw128_off(rb + kk + u, lane);
                *reinterpret_cast<float *>(sBh + o) = hi;
                *reinterpret_cast<float *>(sBl + o) = lo;
              }
#pragma unroll
              for (int u = 0; u < 3; ++u) {
                const float vals[2] = {qv[u] * p1, qv[u] * p2};
#pragma unroll
                for (int sct = 0; sct < 2; ++sct) {
                  float hi, lo;
                  tc::split_tf32(vals[sct], hi, lo);
                  const uint32_t o = tc::sw128_off(rb + NB + sct * (NB - 1) + kk + u, lane);
                  *reinterpret_cast<float *>(sBh + o) = hi;
                  *reinterpret_cast<float *>(sBl + o) = lo;
                }
              }
              prev_kk = kk;
            }
          }
        }
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
          tc::fence_after_sync();
          const int ksteps = min(4, (n - 32 * q + 7) >> 3);
          const uint32_t idesc = tc::idesc_tf32(128, npad, 0, 0);
          const uint32_t a0 = tc::smem_u32(sA + q * 16384), bh0 = tc::smem_u32(sBh), bl0 = tc::smem_u32(sBl);
          for (int s = 0; s < ksteps; ++s) {
            const uint64_t ad = tc::desc_sw128(a0 + 32 * s, 16, 1024);
            tc::mma_tf32(tm, ad, tc::desc_sw128(bh0 + 32 * s, 16, 1024), idesc, (q | s) != 0);
            tc::mma_tf32(tm, ad, tc::desc_sw128(bl0 + 32 * s, 16, 1024), idesc, 1u);
          }
          tc::commit(bar);
        }
        if (!tc::mbar_wait(bar, phase, TC_WAIT_LIMIT) && lane == 0) atomicExch(err, 1);
        phase ^= 1u;
      }
      tc::fence_after_sync();
      // ---- epilogue: contract the features with the candidate's B-spline coefficients
      for (int jj = warp >> 2; jj < jc; jj += 2) {
        float v[16 * TcShape<NB>::NLD];
        const uint32_t ta = tm + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(jj * F);
#pragma unroll
        for (int l = 0; l < TcShape<NB>::NLD; ++l) tc::tmem_ld16(ta + 16 * l, v + 16 * l);
        tc::tmem_wait_ld();
        float G = 0.f, a1 = 0.f, a2 = 0.f;
#pragma unroll
        for (int u = 0; u < NB; ++u) G = fmaf(wr[u], v[u], G);
#pragma unroll
        for (int u = 0; u < NB - 1; ++u) {
          a1 = fmaf(wr[NB + u], v[NB + u], a1);
          a2 = fmaf(wr[NB + u], v[2 * NB - 1 + u], a2);
        }
        if (c_ep < C) {
          float *g = gp + c_ep * pitch + 3 * (j0 + jj);
          atomicAdd(g, G);
          atomicAdd(g + 1, a1 * ginv);
          atomicAdd(g + 2, a2 * ginv);
        }
      }
      tc::fence_before_sync();
      __syncthreads();
    }

    // ---- density: rho_i = sum_j rho_j + 1/2 f_j G_j, one warp per (candidate, 32 slots)
    const int ntask = C * kcu;
    for (int t2 = warp; t2 < ntask; t2 += TC_THREADS / 32) {
      const int c = t2 / kcu, h = t2 - c * kcu, j = 32 * h + lane;
      double term = 0.0;
      if (j < n) {
        const float *q = geo + j * TC_GEO;
        const int kn = __float_as_int(q[13]);
        const int tj = __float_as_int(q[14]);
        const float *pt = ptabf + (size_t)(cg + c) * pot.pow_stride;
        const int krho = ((kn >> 8) & 0xff) - 1, kf = ((kn >> 16) & 0xff) - 1;
        float d, rho = 0.f, f = 0.f;
        if (krho >= 0) rho = tc_pair_fn(pt, sg[pot.s_rho + tj], krho, q[11], d);
        if (kf >= 0) f = tc_pair_fn(pt, sg[pot.s_f + pair_ij_index(ti, tj, nt)], kf, q[12], d);
        term = (double)rho + 0.5 * (double)f * (double)gp[c * pitch + 3 * j];
      }
      for (int o = 16; o > 0; o >>= 1) term += __shfl_down_sync(0xffffffffu, term, o);
      if (lane == 0) part[t2] = term;
    }
    __syncthreads();
    // ---- embedding (pot_meam_spline.cpp:208-223), one thread per candidate
    if (tid < C) {
      double rho = 0.0;
      for (int h = 0; h < kcu; ++h) rho += part[tid * kcu + h];
      const int cand = cg + tid;
      const SplineGeom &gU = sg[pot.s_U + ti];
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
      const PointEval U = spl_point(tabs + (size_t)cand * pot.tab_stride, gU, rho);
      sU[tid] = U.val;
      sU[TC_CANDS + tid] = U.grad;
      double *ao = aout + (size_t)cand * AO_COUNT * N;
      ao[AO_PEN * N + ia] = pen;
      ao[AO_RHO * N + ia] = rho_raw;
    }
    __syncthreads();
    // ---- reaction vectors, stress and energy terms of every slot
    for (int t2 = warp; t2 < ntask; t2 += TC_THREADS / 32) {
      const int c = t2 / kcu, h = t2 - c * kcu, j = 32 * h + lane;
      const int cand = cg + c;
      double acc[10];
#pragma unroll
      for (int u = 0; u < 10; ++u) acc[u] = 0.0;
      if (j < n) {
        const int64_t s = (int64_t)s0 + j;
        const float *q = geo + j * TC_GEO;
        const int kn = __float_as_int(q[13]);
        const int tj = __float_as_int(q[14]);
        const int pij = pair_ij_index(ti, tj, nt);
        const float *pt = ptabf + (size_t)cand * pot.pow_stride;
        const int kphi = (kn & 0xff) - 1, krho = ((kn >> 8) & 0xff) - 1, kf = ((kn >> 16) & 0xff) - 1;
        float phi = 0.f, dphi = 0.f, drho = 0.f, f = 0.f, df = 0.f;
        if (kphi >= 0) phi = tc_pair_fn(pt, sg[pot.s_phi + pij], kphi, q[7], dphi);
        if (krho >= 0) tc_pair_fn(pt, sg[pot.s_rho + tj], krho, q[11], drho);
        if (kf >= 0) f = tc_pair_fn(pt, sg[pot.s_f + pij], kf, q[12], df);
        const float *g3 = gp + c * pitch + 3 * j;
        const double G = g3[0];
        const double dF = sU[TC_CANDS + c];
        const double ux = q[0], uy = q[1], uz = q[2];
        const double ip = 1.0 / (double)q[3];
        // vk perpendicular to u_j in the lab frame
        const double vx = (double)g3[1] * q[4] + (double)g3[2] * q[8];
        const double vy = (double)g3[1] * q[5] + (double)g3[2] * q[9];
        const double vz = (double)g3[1] * q[6] + (double)g3[2] * q[10];
        const double cu = 0.5 * (double)dphi + (double)drho * dF + dF * (double)df * G;
        const double ck = dF * (double)f * ip;
        const double Vx = ux * cu + ck * vx, Vy = uy * cu + ck * vy, Vz = uz * cu + ck * vz;
        double *Vc = Vout + (size_t)cand * 3 * Np + 3 * (int64_t)s;  // (x, y, z) per slot
        Vc[0] = Vx;
        Vc[1] = Vy;
        Vc[2] = Vz;
        if (AUX) {
          double *ax = aux + (size_t)cand * AUX_COUNT * Np;
          ax[AUX_G * Np + s] = G;
          ax[AUX_H * Np + s] = 0.0;  // H_j = u_j . vk_j; with vk taken perpendicular it is 0
          ax[AUX_VX * Np + s] = vx;
          ax[AUX_VY * Np + s] = vy;
          ax[AUX_VZ * Np + s] = vz;
        }
        const double rr = db.pair_r[s];
        const double dx = db.pair_ux[s], dy = db.pair_uy[s], dz = db.pair_uz[s];
        acc[0] = Vx;
        acc[1] = Vy;
        acc[2] = Vz;
        acc[3] = 0.5 * (double)phi;
        acc[4] = -(dx * (Vx * rr));
        acc[5] = -(dy * (Vy * rr));
        acc[6] = -(dz * (Vz * rr));
        acc[7] = -(dx * (Vy * rr));
        acc[8] = -(dy * (Vz * rr));
        acc[9] = -(dz * (Vx * rr));
      }
#pragma unroll
      for (int u = 0; u < 10; ++u)
        for (int o = 16; o > 0; o >>= 1) acc[u] += __shfl_down_sync(0xffffffffu, acc[u], o);
      if (lane == 0)
#pragma unroll
        for (int u = 0; u < 10; ++u) part[t2 * 10 + u] = acc[u];
    }
    __syncthreads();
    if (tid < C) {
      double acc[10];
#pragma unroll
      for (int u = 0; u < 10; ++u) acc[u] = 0.0;
      for (int h = 0; h < kcu; ++h)
#pragma unroll
        for (int u = 0; u < 10; ++u) acc[u] += part[(tid * kcu + h) * 10 + u];
      double *ao = aout + (size_t)(cg + tid) * AO_COUNT * N;
      ao[AO_AX * N + ia] = acc[0];
      ao[AO_AY * N + ia] = acc[1];
      ao[AO_AZ * N + ia] = acc[2];
      ao[AO_E * N + ia] = acc[3] + sU[tid];
#pragma unroll
      for (int u = 0; u < 6; ++u) ao[(AO_S0 + u) * N + ia] = acc[4 + u];
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tm, TC_TMEM_COLS);
}

// Shared-memory plan of k_atoms_tc for rows of at most max_row slots and
// NB B-spline coefficients per g spline; smem_bytes = 0 when it cannot run.
inline TcParams tc_plan(int max_row, int nb, int ntypes, int nsplines, int smem_limit) {
  TcParams p{};
  const int F = 3 * nb - 2;
  p.kc = std::max(1, (max_row + 31) / 32);
  p.smax = 32 * p.kc;
  p.J = std::min(8, 256 / F);
  while (p.J > 1 && (p.J - 1) * F + 16 * ((F + 15) / 16) > TC_TMEM_COLS) --p.J;
  p.gp_pitch = 3 * p.smax + 1;
  const int brows = ((p.J * F + 15) / 16) * 16;
  size_t o = 0;
  auto take = [&](size_t bytes, size_t align) {
    o = (o + align - 1) / align * align;
    const size_t at = o;
    o += bytes;
    return (int)at;
  };
  p.off_a = take((size_t)p.kc * 16384, 1024);
  p.off_bhi = take((size_t)brows * 128, 1024);
  p.off_blo = take((size_t)brows * 128, 1024);
  p.off_gp = take(sizeof(float) * TC_CANDS * p.gp_pitch, 16);
  p.off_geo = take(sizeof(float) * TC_GEO * p.smax, 16);
  p.off_w = take(sizeof(float) * TC_CANDS * ntypes * (2 * nb - 1), 16);
  p.off_sg = take(sizeof(SplineGeom) * nsplines, 16);
  p.off_part = take(sizeof(double) * TC_CANDS * p.kc * 10, 16);
  p.off_u = take(sizeof(double) * 2 * TC_CANDS, 16);
  p.off_bar = take(16, 16);
  p.smem_bytes = (int)o + 1024;  // + alignment slack of the dynamic base
  if (max_row > 32 * TC_MAX_KC || p.smem_bytes > smem_limit) p.smem_bytes = 0;
  return p;
}

}  // namespace mzb
