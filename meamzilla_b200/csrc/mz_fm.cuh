// Batched mixed-precision meam/spline objective and gradient over triplet
// moments ("FM" path).
//
// The triplet sums of slot p = (i, j) that the forward needs,
//   G_p = sum_k f_ik(r_k) g_i(cos_pk),   vk_p = sum_k g_i'(cos_pk) f_ik(r_k) u_k
// (pot_meam_spline.cpp:194-206 and 240-269 enumerate the same triplets), are
// bilinear in the candidate's spline coefficients.  Written in the cubic
// B-spline bases of f and g (f = sum_a c_a B_a(r), g = sum_n w_n B_n(cos);
// both splines are C2 cubics on uniform knots, so these are exact
// re-parametrisations of the knot tables), with e1, e2 an orthonormal pair
// perpendicular to u_p:
//   G_p  = sum_{o,a,n} c^{(t_i,o)}_a w^{(t_i)}_n  X_p[0][o,a,n]
//   Y1_p = sum ... X_p[1][o,a,n],   Y2_p = sum ... X_p[2][o,a,n]
//   X_p[0][o,a,n]   = sum_k [type k = o] B_a(r_k) B_n(cos_pk)
//   X_p[1|2][o,a,n] = sum_k [type k = o] B_a(r_k) B_n'(cos_pk) (u_k . e1|e2)
// and vk_p - u_p (u_p . vk_p) = e1 Y1_p + e2 Y2_p, which is all of vk that the
// reaction vector V_p uses.  The moments X do not depend on the candidate:
// they are computed once per database (k_fm_features, FP64, stored FP32).
// Per launch the candidates' triplet work becomes two dense contractions of
// X with the candidates' products K[o,a,n] = c_a w_n:
//   forward   Y[q][t][c]   = sum_d X[t][d][q] K_s[d][c]        (k_fm_gemm_fwd)
//   adjoint   Kbar_s[d][c] = sum_{q,t} X[t][d][q] Ybar[q][t][c] (k_fm_gemm_adj)
// and everything per slot or per atom is a short epilogue (k_fm_epi,
// k_fm_adj_pre).  Precision is that of the mixed path: FP32 spline values and
// contractions, FP64 per-atom densities, energies, virials, residuals and
// gradient sums.
//
// Layouts (feature slots q: the atoms in type-sorted order, each row
// contiguous, each type's run padded to a multiple of FM_TILE):
//   X     [nch][3][FM_DC][Q]         moments, FM_DC features per chunk
//   E     [Q][8]                     e1, e2 of the slot (FP32)
//   Y     [ngroups][Q][3][CG]        G, Y1, Y2; the adjoint overwrites them with
//                                    dL/dG, dL/dY1, dL/dY2
//   V     [ngroups][Np][CG][3]       reaction vectors (FP64), global slot order
//   aoutF [ngroups][N][AO_COUNT][CG] per-atom outputs (FP64)
// with candidates in groups of CG (the launch's candidates rounded up to a
// power of two from 8 to 64).
#pragma once

#include "mz_adj.cuh"

namespace mzb {

constexpr int FM_TILE = 128;   // feature slots per contraction tile
constexpr int FM_DC = 24;      // features per chunk of the forward contraction
constexpr int FM_MAXT = 2;     // atom types
constexpr int FM_MAXN = 16;    // B-spline coefficients of a g spline (knots + 2)
constexpr int FM_MAXB = 24;    // B-spline coefficients of any spline the path reads (knots + 2)
constexpr int FM_SUB = 16;     // feature slots per sub-tile of the adjoint contraction
constexpr int FM_ROWS = 8;     // features per thread in the adjoint contraction
constexpr int FM_PCHUNK = 32;  // slots per chunk of the pair-function gradient

struct FmPlan {
  int nt;          // atom types
  int NA, NN;      // B-spline coefficients per f spline, per g spline (the largest)
  int D, Dpad;     // features per kind: nt NA NN, padded to a multiple of FM_DC
  int nch;         // Dpad / FM_DC
  int CG;          // candidates per group
  int64_t Q;       // feature slots
  int ntiles;      // Q / FM_TILE
  int tile0[FM_MAXT + 1];  // first tile of each type
  int nblk;        // atom blocks of the adjoint epilogue (type-pure, <= 256 slots, <= 64 atoms)
  const int *blk0;         // [nblk + 1] into adj_atoms
  const int *row0;         // [N] feature slot of each atom's first pair
  const float *X;
  const float *E;
  float *Y;
  const float *Kf;         // [ngroups][nt][Dpad][CG]
  const double *coef64;    // [ncand][nsplines][FM_MAXB]
  const float *coef32;     // [ngroups][nsplines][FM_MAXB][CG]
  double *V;
  double *aoutF;
  float *lamf;             // [ngroups][N][3][CG]
  double *seedF;           // [ngroups][NC][CS_COUNT][CG]
  double *Kbar;            // [ngroups][nctas_adj][nt][Dpad][CG]  FP64 partials of the adjoint contraction
  double *Pbar;            // [ngroups][nctas_pre][nsplines][FM_MAXB][CG]  pair-function B-spline gradients
  double *Tbar;            // [ngroups][nctas_pre][CG][stride]  embedding table gradients
  int nctas_adj, nctas_pre;
};

// ------------------------------------------------------------- helpers

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Uniform cubic B-spline basis on an interval at shift b: the weights of
// coefficients m .. m+3 (basis m centred on knot m-1) and their b-derivatives.
template <typename R>
__device__ __forceinline__ void bsp_basis(R b, R *N) {
  const R a = R(1) - b, b2 = b * b, b3 = b2 * b;
  N[0] = a * a * a / R(6);
  N[1] = (R(3) * b3 - R(6) * b2 + R(4)) / R(6);
  N[2] = (R(-3) * b3 + R(3) * b2 + R(3) * b + R(1)) / R(6);
  N[3] = b3 / R(6);
}
template <typename R>
__device__ __forceinline__ void bsp_dbasis(R b, R *N) {
  const R a = R(1) - b;
  N[0] = -a * a / R(2);
  N[1] = (R(3) * b * b - R(4) * b) / R(2);
  N[2] = (R(-3) * b * b + R(2) * b + R(1)) / R(2);
  N[3] = b * b / R(2);
}

// An orthonormal pair perpendicular to the unit vector u (FP64; used when
// the moments are built, and stored with them).
__device__ __forceinline__ void perp_frame(double ux, double uy, double uz, double *e1, double *e2) {
  const double ax = fabs(ux), ay = fabs(uy), az = fabs(uz);
  double vx, vy, vz;  // u x (the axis least aligned with u)
  if (ax <= ay && ax <= az) {
    vx = 0.0; vy = uz; vz = -uy;
  } else if (ay <= az) {
    vx = -uz; vy = 0.0; vz = ux;
  } else {
    vx = uy; vy = -ux; vz = 0.0;
  }
  const double inv = 1.0 / sqrt(vx * vx + vy * vy + vz * vz);
  e1[0] = vx * inv; e1[1] = vy * inv; e1[2] = vz * inv;
  e2[0] = uy * e1[2] - uz * e1[1];
  e2[1] = uz * e1[0] - ux * e1[2];
  e2[2] = ux * e1[1] - uy * e1[0];
}

__device__ __forceinline__ int fm_tile_type(const FmPlan &fp, int tile) {
  int s = 0;
  while (s + 1 < fp.nt && tile >= fp.tile0[s + 1]) ++s;
  return s;
}

// ---------------------------------------------------------- k_fm_features

// One CTA per atom (type-sorted order), one warp per slot of its row; lane L
// holds the moments of partner type o = L / NA and f coefficient a = L % NA
// for every g coefficient n and the three kinds.  Triplets as the FP64
// kernels take them: every other slot of the row whose cosine is below g's
// cut (triplet_meam_spline.cpp:65-70), the g interval by g_knot.
__global__ void __launch_bounds__(256) k_fm_features(DevDb db, DevPot pot, const SplineGeom *__restrict__ geom,
                                                     FmPlan fp, float *__restrict__ X, float *__restrict__ E) {
  __shared__ double su[3][BLOCK_SLOTS], sbf[BLOCK_SLOTS];
  __shared__ int so[BLOCK_SLOTS], skf[BLOCK_SLOTS];
  const int i = db.adj_atoms[blockIdx.x];
  const int ti = db.atom_type[i];
  const int64_t p0 = db.pair_off[i];
  const int n = db.pair_off[i + 1] - (int)p0;
  const int64_t Np = db.npairs;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
  for (int k = tid; k < n; k += blockDim.x) {
    const int64_t gs = p0 + k;
    su[0][k] = db.pair_ux[gs];
    su[1][k] = db.pair_uy[gs];
    su[2][k] = db.pair_uz[gs];
    so[k] = db.atom_type[db.pair_nbr[gs]];
    skf[k] = ((db.pair_knot[gs] >> 16) & 0xff) - 1;
    sbf[k] = db.pair_shift[2 * Np + gs];
  }
  __syncthreads();
  const SplineGeom gg = geom[pot.s_g + ti];
  const int ol = lane / fp.NA, al = lane % fp.NA;
  const bool active = lane < fp.nt * fp.NA;
  const int64_t q0 = fp.row0[i];
  for (int p = warp; p < n; p += nwarp) {
    const double ux = su[0][p], uy = su[1][p], uz = su[2][p];
    double e1[3], e2[3];
    perp_frame(ux, uy, uz, e1, e2);
    double acc[3][FM_MAXN];
#pragma unroll
    for (int t = 0; t < 3; ++t)
#pragma unroll
      for (int m = 0; m < FM_MAXN; ++m) acc[t][m] = 0.0;
    for (int k = 0; k < n; ++k) {
      if (k == p) continue;
      const double vx = su[0][k], vy = su[1][k], vz = su[2][k];
      const double c = cos_exact(ux, uy, uz, vx, vy, vz);
      if (!(c < gg.cut)) continue;
      const int kf = skf[k];
      if (kf < 0) continue;
      double w = 0.0;
      if (active && so[k] == ol) {
        const int j = al - kf;
        if (j >= 0 && j < 4) {
          double Nf[4];
          bsp_basis<double>(sbf[k], Nf);
          w = j == 0 ? Nf[0] : j == 1 ? Nf[1] : j == 2 ? Nf[2] : Nf[3];
        }
      }
      if (w == 0.0) continue;
      double b;
      const int m = g_knot<double>(c, gg.x0, gg.invstep, gg.n, b);
      double Ng[4], Nd[4];
      bsp_basis<double>(b, Ng);
      bsp_dbasis<double>(b, Nd);
      const double p1 = (vx * e1[0] + vy * e1[1] + vz * e1[2]) * gg.invstep * w;
      const double p2 = (vx * e2[0] + vy * e2[1] + vz * e2[2]) * gg.invstep * w;
#pragma unroll
      for (int nn = 0; nn < FM_MAXN; ++nn) {
        const int j = nn - m;
        const double gv = j == 0 ? Ng[0] : j == 1 ? Ng[1] : j == 2 ? Ng[2] : j == 3 ? Ng[3] : 0.0;
        const double gd = j == 0 ? Nd[0] : j == 1 ? Nd[1] : j == 2 ? Nd[2] : j == 3 ? Nd[3] : 0.0;
        acc[0][nn] += w * gv;
        acc[1][nn] += p1 * gd;
        acc[2][nn] += p2 * gd;
      }
    }
    const int64_t q = q0 + p;
    if (active) {
#pragma unroll
      for (int t = 0; t < 3; ++t)
#pragma unroll
        for (int nn = 0; nn < FM_MAXN; ++nn)
          if (nn < fp.NN) {
            const int d = lane * fp.NN + nn, ch = d / FM_DC, din = d % FM_DC;
            X[((size_t)(ch * 3 + t) * FM_DC + din) * fp.Q + q] = (float)acc[t][nn];
          }
    }
    if (lane == 0) {
      float *e = E + (size_t)q * 8;
      e[0] = (float)e1[0]; e[1] = (float)e1[1]; e[2] = (float)e1[2];
      e[3] = (float)e2[0]; e[4] = (float)e2[1]; e[5] = (float)e2[2];
      e[6] = 0.f; e[7] = 0.f;
    }
  }
}

// ------------------------------------------------------------- k_fm_coef

// B-spline coefficients of every spline of every candidate from its FP64
// knot table: with the basis function m centred on knot m-1,
// y_i = (d_i + 4 d_i+1 + d_i+2) / 6 and y''_i = (d_i - 2 d_i+1 + d_i+2) / h^2,
// so d_i+1 = y_i - h^2/6 y''_i, and the outer two follow from y'' at the end
// knots.  FP64, and FP32 in the epilogues' candidate-fastest layout.
__global__ void k_fm_coef(int ncand, const SplineGeom *__restrict__ geom, int nsplines, int stride,
                          const double *__restrict__ tabs, FmPlan fp, double *__restrict__ coef64,
                          float *__restrict__ coef32) {
  const int c = blockIdx.x, s = threadIdx.x;
  if (c >= ncand || s >= nsplines) return;
  const SplineGeom g = geom[s];
  const double *y = tabs + (size_t)c * stride + g.toff, *ypp = y + g.n;
  const double h2 = g.step * g.step;
  const int n = g.n;
  double *o64 = coef64 + ((size_t)c * nsplines + s) * FM_MAXB;
  const int gy = c / fp.CG, cl = c % fp.CG;
  float *o32 = coef32 + ((size_t)gy * nsplines + s) * FM_MAXB * fp.CG + cl;
  for (int m = 0; m < FM_MAXB; ++m) {
    double d = 0.0;
    if (m >= 1 && m <= n) d = y[m - 1] - h2 / 6.0 * ypp[m - 1];
    else if (m == 0 && n >= 2) d = h2 * ypp[0] + 2.0 * (y[0] - h2 / 6.0 * ypp[0]) - (y[1] - h2 / 6.0 * ypp[1]);
    else if (m == n + 1 && n >= 2)
      d = h2 * ypp[n - 1] + 2.0 * (y[n - 1] - h2 / 6.0 * ypp[n - 1]) - (y[n - 2] - h2 / 6.0 * ypp[n - 2]);
    o64[m] = d;
    o32[(size_t)m * fp.CG] = (float)d;
  }
}

// K_s[d][c] = c^{f(s,o)}_a w^{g(s)}_n, d = (o NA + a) NN + n (FP64 products,
// rounded once); zero beyond D and for missing candidates.
__global__ void k_fm_kmat(int ncand, DevPot pot, FmPlan fp, const double *__restrict__ coef64,
                          float *__restrict__ Kf) {
  const int s = blockIdx.x, gy = blockIdx.y;
  const int total = fp.Dpad * fp.CG;
  for (int idx = blockIdx.z * blockDim.x + threadIdx.x; idx < total; idx += gridDim.z * blockDim.x) {
    const int d = idx / fp.CG, cl = idx % fp.CG, c = gy * fp.CG + cl;
    double v = 0.0;
    if (c < ncand && d < fp.D) {
      const int o = d / (fp.NA * fp.NN), a = (d / fp.NN) % fp.NA, nn = d % fp.NN;
      const int fs = pot.s_f + pair_ij_index(s, o, pot.ntypes), gs = pot.s_g + s;
      v = coef64[((size_t)c * pot.nsplines + fs) * FM_MAXB + a] *
          coef64[((size_t)c * pot.nsplines + gs) * FM_MAXB + nn];
    }
    Kf[((size_t)(gy * fp.nt + s) * fp.Dpad + d) * fp.CG + cl] = (float)v;
  }
}

// ---------------------------------------------------------- k_fm_gemm_fwd

// Y[q][t][c] = sum_d X[t][d][q] K_s[d][c] over one tile of FM_TILE feature
// slots (one atom type s) and one group of CG = 8 NW candidates.  Thread
// (lane, warp): slots 4 lane .. 4 lane + 3, candidates 8 warp .. 8 warp + 7,
// all three kinds -- 96 FP32 sums as packed pairs of slots.  The moments are
// streamed in chunks of FM_DC features through a double buffer filled by
// cp.async; K_s stays in shared memory for the whole tile.
template <int NW>
__host__ __device__ constexpr size_t fm_fwd_smem(int Dpad) {
  return sizeof(float) * ((size_t)Dpad * NW * 8 + 2 * 3 * FM_DC * FM_TILE);
}

template <int NW>
__global__ void __launch_bounds__(NW * 32, 1) k_fm_gemm_fwd(FmPlan fp) {
  extern __shared__ __align__(16) float fsm[];
  constexpr int CG = NW * 8;
  float *Ks = fsm;                        // [Dpad][CG]
  float *Xs = Ks + (size_t)fp.Dpad * CG;  // [2][3][FM_DC][FM_TILE]
  const int tile = blockIdx.x, gy = blockIdx.y;
  const int s = fm_tile_type(fp, tile);
  const int64_t qb = (int64_t)tile * FM_TILE;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const float *Kg = fp.Kf + (size_t)(gy * fp.nt + s) * fp.Dpad * CG;
  for (int i = tid * 4; i < fp.Dpad * CG; i += NW * 32 * 4) cp_async16(Ks + i, Kg + i);
  auto load_chunk = [&](int ch, int buf) {
    float *dst = Xs + (size_t)buf * 3 * FM_DC * FM_TILE;
    const float *src = fp.X + (size_t)ch * 3 * FM_DC * fp.Q + qb;
    for (int i = tid; i < 3 * FM_DC * (FM_TILE / 4); i += NW * 32) {
      const int row = i / (FM_TILE / 4), col = (i % (FM_TILE / 4)) * 4;
      cp_async16(dst + row * FM_TILE + col, src + (size_t)row * fp.Q + col);
    }
    cp_async_commit();
  };
  load_chunk(0, 0);
  float2 acc[3][2][8];  // [kind][slot pair][candidate]: (slot 2 sp, slot 2 sp + 1)
#pragma unroll
  for (int t = 0; t < 3; ++t)
#pragma unroll
    for (int sp = 0; sp < 2; ++sp)
#pragma unroll
      for (int c = 0; c < 8; ++c) acc[t][sp][c] = make_float2(0.f, 0.f);
  for (int ch = 0; ch < fp.nch; ++ch) {
    if (ch + 1 < fp.nch) {
      load_chunk(ch + 1, (ch + 1) & 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const float *xb = Xs + (size_t)(ch & 1) * 3 * FM_DC * FM_TILE + 4 * lane;
    const float *kb = Ks + (size_t)ch * FM_DC * CG + warp * 8;
#pragma unroll 2
    for (int din = 0; din < FM_DC; ++din) {
      const float4 k0 = *reinterpret_cast<const float4 *>(kb + din * CG);
      const float4 k1 = *reinterpret_cast<const float4 *>(kb + din * CG + 4);
      const float kk[8] = {k0.x, k0.y, k0.z, k0.w, k1.x, k1.y, k1.z, k1.w};
#pragma unroll
      for (int t = 0; t < 3; ++t) {
        const float4 xv = *reinterpret_cast<const float4 *>(xb + (t * FM_DC + din) * FM_TILE);
        const float2 x01 = make_float2(xv.x, xv.y), x23 = make_float2(xv.z, xv.w);
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const float2 kc = bcast2(kk[c]);
          acc[t][0][c] = fma2(x01, kc, acc[t][0][c]);
          acc[t][1][c] = fma2(x23, kc, acc[t][1][c]);
        }
      }
    }
    __syncthreads();
  }
  float *Yb = fp.Y + ((size_t)gy * fp.Q + qb + 4 * lane) * 3 * CG + warp * 8;
#pragma unroll
  for (int sl = 0; sl < 4; ++sl)
#pragma unroll
    for (int t = 0; t < 3; ++t) {
      float v[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) v[c] = (sl & 1) ? acc[t][sl >> 1][c].y : acc[t][sl >> 1][c].x;
      float *dst = Yb + ((size_t)sl * 3 + t) * CG;
      *reinterpret_cast<float4 *>(dst) = make_float4(v[0], v[1], v[2], v[3]);
      *reinterpret_cast<float4 *>(dst + 4) = make_float4(v[4], v[5], v[6], v[7]);
    }
}

// ------------------------------------------------------ per-slot helpers

// One pair function (FP32) of a slot from the candidate's B-spline
// coefficients: value and d/dr.
__device__ __forceinline__ float fm_pair_val(const float *coef, int CG, int k, float b, float inv, float &d) {
  float N[4], Nd[4];
  bsp_basis<float>(b, N);
  bsp_dbasis<float>(b, Nd);
  const float c0 = coef[(size_t)k * CG], c1 = coef[(size_t)(k + 1) * CG], c2 = coef[(size_t)(k + 2) * CG],
              c3 = coef[(size_t)(k + 3) * CG];
  d = (Nd[0] * c0 + Nd[1] * c1 + Nd[2] * c2 + Nd[3] * c3) * inv;
  return N[0] * c0 + N[1] * c1 + N[2] * c2 + N[3] * c3;
}

struct FmSlot {
  int64_t gs;
  int j, tj, pij;
  float ux, uy, uz, r, invr;
  int kphi, krho, kf;
  float bphi, brho, bf;
};

__device__ __forceinline__ FmSlot fm_slot(const DevDb &db, const DevPot &pot, int64_t gs, int ti) {
  FmSlot s;
  s.gs = gs;
  const int64_t Np = db.npairs;
  s.j = db.pair_nbr[gs];
  s.tj = db.atom_type[s.j];
  s.pij = pair_ij_index(ti, s.tj, pot.ntypes);
  s.ux = db.pair_uxf[gs];
  s.uy = db.pair_uyf[gs];
  s.uz = db.pair_uzf[gs];
  s.r = db.pair_rf[gs];
  s.invr = 1.f / s.r;
  const int kn = db.pair_knot[gs];
  s.kphi = (kn & 0xff) - 1;
  s.krho = ((kn >> 8) & 0xff) - 1;
  s.kf = ((kn >> 16) & 0xff) - 1;
  s.bphi = db.pair_shiftf[gs];
  s.brho = db.pair_shiftf[Np + gs];
  s.bf = db.pair_shiftf[2 * Np + gs];
  return s;
}

// phi, rho, f (values and slopes) of a slot for candidate cl of the group
struct FmPairVals {
  float phi, dphi, rho, drho, f, df;
};
__device__ __forceinline__ FmPairVals fm_pair_vals(const DevPot &pot, const SplineGeom *sg, const float *coefg,
                                                   int CG, const FmSlot &s) {
  FmPairVals v{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (s.kphi >= 0) {
    const int sp = pot.s_phi + s.pij;
    v.phi = fm_pair_val(coefg + (size_t)sp * FM_MAXB * CG, CG, s.kphi, s.bphi, (float)sg[sp].invstep, v.dphi);
  }
  if (s.krho >= 0) {
    const int sp = pot.s_rho + s.tj;
    v.rho = fm_pair_val(coefg + (size_t)sp * FM_MAXB * CG, CG, s.krho, s.brho, (float)sg[sp].invstep, v.drho);
  }
  if (s.kf >= 0) {
    const int sp = pot.s_f + s.pij;
    v.f = fm_pair_val(coefg + (size_t)sp * FM_MAXB * CG, CG, s.kf, s.bf, (float)sg[sp].invstep, v.df);
  }
  return v;
}

// ---------------------------------------------------------------- k_fm_epi

// Forward epilogue, thread = (atom in type order, candidate of group
// blockIdx.y): the density rho_i = sum_p rho_p + 1/2 f_p G_p and the pair
// energy in FP64 over the atom's row, the embedding (clamp and punishment,
// pot_meam_spline.cpp:208-223), then per slot the reaction vector
//   V_p = u_p (phi'_p / 2 + U' (rho'_p + f'_p G_p)) + U' f_p / r_p (e1 Y1 + e2 Y2)
// (the force atom i's terms put on it along slot p; the neighbour receives
// -V_p), with the atom's own force and virial sums.
__global__ void __launch_bounds__(256) k_fm_epi(DevDb db, DevPot pot, const SplineGeom *__restrict__ geom,
                                               const double *__restrict__ tabs, FmPlan fp, int ncand) {
  __shared__ SplineGeom sg[MAX_SPLINES];
  const int gy = blockIdx.y, CG = fp.CG;
  for (int s = threadIdx.x; s < pot.nsplines; s += blockDim.x) sg[s] = geom[s];
  __syncthreads();
  const int N = db.natoms;
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)N * CG) return;
  const int qa = (int)(idx / CG), cl = (int)(idx % CG);
  const int c = gy * CG + cl;
  if (c >= ncand) return;
  const float *coefg = fp.coef32 + (size_t)gy * pot.nsplines * FM_MAXB * CG + cl;
  const double *tc = tabs + (size_t)c * pot.tab_stride;
  const int i = db.adj_atoms[qa];
  const int ti = db.atom_type[i];
  const int64_t p0 = db.pair_off[i];
  const int n = db.pair_off[i + 1] - (int)p0;
  const int64_t q0 = fp.row0[i];
  const float *Yq = fp.Y + ((size_t)gy * fp.Q + q0) * 3 * CG + cl;
  double rho = 0.0, epair = 0.0;
  for (int p = 0; p < n; ++p) {
    const FmSlot s = fm_slot(db, pot, p0 + p, ti);
    const FmPairVals v = fm_pair_vals(pot, sg, coefg, CG, s);
    const float G = Yq[(size_t)p * 3 * CG];
    rho += (double)v.rho + 0.5 * (double)v.f * (double)G;
    epair += 0.5 * (double)v.phi;
  }
  // embedding
  const SplineGeom &gU = sg[pot.s_U + ti];
  const double w = db.cell_w[db.atom_cell[i]];
  double pen = 0.0, rt = rho;
  if (rho < gU.x0) {
    pen = w * 100.0 * 10. * (gU.x0 - rho) * (gU.x0 - rho);
    if (!pot.embed_extrap) rt = gU.x0;
  } else if (rho > gU.xN) {
    pen = w * 100.0 * 10. * (rho - gU.xN) * (rho - gU.xN);
    if (!pot.embed_extrap) rt = gU.xN;
  }
  const PointEval U = spl_point(tc, gU, rt);
  const float dF = (float)U.grad;
  double F[3] = {0, 0, 0}, S[6] = {0, 0, 0, 0, 0, 0};
  double *Vg = fp.V + (size_t)gy * db.npairs * CG * 3;
  for (int p = 0; p < n; ++p) {
    const FmSlot s = fm_slot(db, pot, p0 + p, ti);
    const FmPairVals v = fm_pair_vals(pot, sg, coefg, CG, s);
    const float *yp = Yq + (size_t)p * 3 * CG;
    const float G = yp[0], Y1 = yp[CG], Y2 = yp[2 * CG];
    const float4 e = *reinterpret_cast<const float4 *>(fp.E + (size_t)(q0 + p) * 8);
    const float2 e2 = *reinterpret_cast<const float2 *>(fp.E + (size_t)(q0 + p) * 8 + 4);
    const float A = 0.5f * v.dphi + dF * (v.drho + v.df * G);
    const float B = dF * v.f * s.invr;
    const double Vx = (double)(s.ux * A + B * (e.x * Y1 + e.w * Y2));
    const double Vy = (double)(s.uy * A + B * (e.y * Y1 + e2.x * Y2));
    const double Vz = (double)(s.uz * A + B * (e.z * Y1 + e2.y * Y2));
    double *Vd = Vg + ((size_t)s.gs * CG + cl) * 3;
    Vd[0] = Vx;
    Vd[1] = Vy;
    Vd[2] = Vz;
    const double rr = db.pair_r[s.gs], dx = db.pair_ux[s.gs], dy = db.pair_uy[s.gs], dz = db.pair_uz[s.gs];
    F[0] += Vx;
    F[1] += Vy;
    F[2] += Vz;
    S[0] -= dx * (Vx * rr);
    S[1] -= dy * (Vy * rr);
    S[2] -= dz * (Vz * rr);
    S[3] -= dx * (Vy * rr);
    S[4] -= dy * (Vz * rr);
    S[5] -= dz * (Vx * rr);
  }
  double *ao = fp.aoutF + ((size_t)gy * N + i) * AO_COUNT * CG + cl;
  ao[AO_AX * CG] = F[0];
  ao[AO_AY * CG] = F[1];
  ao[AO_AZ * CG] = F[2];
  ao[AO_E * CG] = epair + U.val;
#pragma unroll
  for (int q = 0; q < 6; ++q) ao[(AO_S0 + q) * CG] = S[q];
  ao[AO_PEN * CG] = pen;
  ao[AO_RHO * CG] = rho;
}

// ------------------------------------------------------------- k_fm_gather

// F_i = own-row sum - sum of V over the slots whose neighbour is i; the force
// residual w (F - F0) (potential.cpp:468-478) and lambda_i = 2 w e_i (FP32,
// for the adjoint).  Thread = (atom, candidate).
__global__ void k_fm_gather(DevDb db, FmPlan fp, int ncand, double *__restrict__ forces,
                            double *__restrict__ errvec, int esize, int want_lam) {
  const int CG = fp.CG, gy = blockIdx.y;
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int N = db.natoms;
  if (idx >= (int64_t)N * CG) return;
  const int i = (int)(idx / CG), cl = (int)(idx % CG), c = gy * CG + cl;
  if (c >= ncand) return;
  double *ao = fp.aoutF + ((size_t)gy * N + i) * AO_COUNT * CG + cl;
  const double *Vg = fp.V + (size_t)gy * db.npairs * CG * 3 + cl * 3;
  double fx = ao[AO_AX * CG], fy = ao[AO_AY * CG], fz = ao[AO_AZ * CG];
  for (int q = db.in_off[i]; q < db.in_off[i + 1]; ++q) {
    const double *v = Vg + (size_t)db.in_slot[q] * CG * 3;
    fx -= v[0];
    fy -= v[1];
    fz -= v[2];
  }
  const int cell = db.atom_cell[i];
  const double w = db.cell_w[cell];
  const double rx = w * (fx - db.force0[3 * i]);
  const double ry = w * (fy - db.force0[3 * i + 1]);
  const double rz = w * (fz - db.force0[3 * i + 2]);
  ao[AO_FSQ * CG] = rx * rx + ry * ry + rz * rz;
  if (forces) {
    double *Fo = forces + (size_t)c * 3 * N;
    Fo[3 * i] = fx;
    Fo[3 * i + 1] = fy;
    Fo[3 * i + 2] = fz;
  }
  if (errvec) {
    const int a0 = db.cell_atom0[cell];
    double *e = errvec + (size_t)c * esize + 7 * (cell + 1) + 3 * a0 + 3 * (i - a0);
    e[0] = rx;
    e[1] = ry;
    e[2] = rz;
  }
  if (want_lam) {
    float *L = fp.lamf + ((size_t)gy * N + i) * 3 * CG + cl;
    L[0] = (float)(2.0 * w * rx);
    L[CG] = (float)(2.0 * w * ry);
    L[2 * CG] = (float)(2.0 * w * rz);
  }
}

// -------------------------------------------------------------- k_fm_cells

// Potential::accumulate_error per cell (potential.cpp:450-485), thread =
// (cell, candidate); with want_seeds also the adjoint seeds dF/dE_atom,
// dF/dS_cell / volume and dF/dpen.
__global__ void k_fm_cells(DevDb db, DevPot pot, FmPlan fp, int ncand, double *__restrict__ cellobj,
                           double *__restrict__ errvec, int esize, double *__restrict__ energy,
                           double *__restrict__ stress, int want_seeds) {
  const int CG = fp.CG, gy = blockIdx.y;
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int NC = db.ncells, N = db.natoms;
  if (idx >= (int64_t)NC * CG) return;
  const int cell = (int)(idx / CG), cl = (int)(idx % CG), c = gy * CG + cl;
  if (c >= ncand) return;
  const int a0 = db.cell_atom0[cell], a1 = db.cell_atom0[cell + 1];
  double v[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) v[q] = 0.0;
  for (int a = a0; a < a1; ++a) {
    const double *ao = fp.aoutF + ((size_t)gy * N + a) * AO_COUNT * CG + cl;
    v[0] += ao[AO_E * CG];
#pragma unroll
    for (int q = 0; q < 6; ++q) v[1 + q] += ao[(AO_S0 + q) * CG];
    v[7] += ao[AO_PEN * CG];
    v[8] += ao[AO_FSQ * CG];
  }
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
  cellobj[(size_t)c * NC + cell] = sum;
  if (errvec) {
    double *e = errvec + (size_t)c * esize + 7 * cell + 3 * a0;
    e[0] = eE;
    for (int q = 0; q < 6; ++q) e[1 + q] = eS[q];
    errvec[(size_t)c * esize + 7 * NC + 3 * N + cell] = cons;
  }
  if (energy) energy[(size_t)c * NC + cell] = E;
  if (stress)
    for (int q = 0; q < 6; ++q) stress[((size_t)c * NC + cell) * 6 + q] = sig[q];
  if (want_seeds) {
    double *sd = fp.seedF + ((size_t)gy * NC + cell) * CS_COUNT * CG + cl;
    sd[CS_EPS * CG] = 2.0 * eE * ew;
    for (int q = 0; q < 6; ++q) sd[(CS_MU0 + q) * CG] = 2.0 * eS[q] * sw / db.cell_vol[cell];
    sd[CS_KAPPA * CG] = 2.0 * cons;
  }
}

// ------------------------------------------------------------ k_fm_adj_pre

// Adjoint epilogue, persistent CTAs over the atom blocks (type-pure, at most
// 256 slots and 64 atoms), candidate group blockIdx.y.  With the residual
// sensitivities frozen (lambda, eps, mu, kappa),
// L = sum_i [eps E_i + kappa pen_i] + sum_p Lambda_p . V_p and, per slot,
// Lambda_p = lambda_i - lambda_j - r_p M_cell u_p, a_p = Lambda_p . u_p:
//   k_p   = a_p (rho'_p + f'_p G_p) + f_p / r_p (Lambda.e1 Y1 + Lambda.e2 Y2)
//   K_i   = sum_p k_p,  chi_i = dL/drho_i = (eps U' + U'' K_i) [unclamped] + kappa dpen/drho
//   dL/dG_p = 1/2 f_p chi_i + a_p U' f'_p,  dL/dY1|2 = U' f_p / r_p Lambda.e1|2
// (written over Y for k_fm_gemm_adj), and the pair functions' (value, slope)
// weights
//   phi: (eps / 2, a_p / 2), rho: (chi, U' a_p),
//   f:   (chi G_p / 2 + U' (Lambda.e1 Y1 + Lambda.e2 Y2) / r_p, U' a_p G_p)
// (f's role as the partner k goes through the contraction).  The weights of
// FM_PCHUNK slots at a time are staged in shared memory and added into
// per-(function, candidate) FP32 B-spline coefficient sums by whole warps
// (the slot, hence the interval, is warp-uniform, so a switch picks the four
// coefficients), flushed to this CTA's FP64 partial at a change of atom type
// and every FM_PFLUSH blocks; the embedding table gradient (value weight
// eps, slope weight K_i) is added per atom, in atom order, by the thread of
// each candidate, in FP64.  Fixed order throughout.
constexpr int FM_ABLK = 64;   // atoms per block of the adjoint epilogue
constexpr int FM_PFLUSH = 4;  // blocks between flushes of the pair-function sums
struct FmAdjSmem {
  double chi[FM_ABLK][64];
  double dF[FM_ABLK][64];
  double K[FM_ABLK][64];
  float w[FM_PCHUNK][6][64];
  int sk[FM_PCHUNK][3];    // knots of phi, rho, f
  float sb[FM_PCHUNK][3];  // shifts
  int stj[FM_PCHUNK];      // neighbour type
  int satom[FM_ABLK];
  int arow[FM_ABLK + 1];   // block-local first slot of each atom
};

__device__ __forceinline__ void fm_lambda(const DevDb &db, const FmPlan &fp, int gy, int cl, int i, int cell,
                                          const FmSlot &s, float &lx, float &ly, float &lz) {
  const int CG = fp.CG, N = db.natoms;
  const float *Li = fp.lamf + ((size_t)gy * N + i) * 3 * CG + cl;
  const float *Lj = fp.lamf + ((size_t)gy * N + s.j) * 3 * CG + cl;
  const double *sd = fp.seedF + ((size_t)gy * db.ncells + cell) * CS_COUNT * CG + cl;
  const float mxx = (float)sd[(CS_MU0 + 0) * CG], myy = (float)sd[(CS_MU0 + 1) * CG],
              mzz = (float)sd[(CS_MU0 + 2) * CG], mxy = (float)sd[(CS_MU0 + 3) * CG],
              myz = (float)sd[(CS_MU0 + 4) * CG], mzx = (float)sd[(CS_MU0 + 5) * CG];
  lx = Li[0] - Lj[0] - s.r * (mxx * s.ux + mzx * s.uz);
  ly = Li[CG] - Lj[CG] - s.r * (myy * s.uy + mxy * s.ux);
  lz = Li[2 * CG] - Lj[2 * CG] - s.r * (mzz * s.uz + myz * s.uy);
}

// The spline of pair function F (0 phi, 1 rho, 2 f) for a centre of type ti
// and a neighbour of type tj.
__device__ __forceinline__ int fm_pair_spline(const DevPot &pot, int F, int ti, int tj) {
  return F == 1 ? pot.s_rho + tj : (F == 0 ? pot.s_phi : pot.s_f) + pair_ij_index(ti, tj, pot.ntypes);
}

__host__ __device__ inline size_t fm_pre_smem(int nsplines) {
  return sizeof(FmAdjSmem) + sizeof(SplineGeom) * (size_t)nsplines;
}

__global__ void __launch_bounds__(256, 1) k_fm_adj_pre(DevDb db, DevPot pot, const SplineGeom *__restrict__ geom,
                                                      const double *__restrict__ tabs, FmPlan fp, int ncand) {
  extern __shared__ __align__(16) unsigned char fm_raw[];
  FmAdjSmem &sm = *reinterpret_cast<FmAdjSmem *>(fm_raw);
  SplineGeom *sg = reinterpret_cast<SplineGeom *>(fm_raw + sizeof(FmAdjSmem));
  const int gy = blockIdx.y, CG = fp.CG, N = db.natoms, NC = db.ncells;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int s = tid; s < pot.nsplines; s += blockDim.x) sg[s] = geom[s];
  const int cl = tid % CG, set = tid / CG, nsets = blockDim.x / CG;
  const int c = gy * CG + cl;
  const bool live = c < ncand;
  const float *coefg = fp.coef32 + (size_t)gy * pot.nsplines * FM_MAXB * CG + cl;
  const double *tc = tabs + (size_t)(live ? c : 0) * pot.tab_stride;
  // pair-function lanes: function pF = warp / wpf, candidate pc
  const int wpf = (CG + 31) / 32;
  const int pF = warp / wpf, pc = (warp % wpf) * 32 + lane;
  const bool pworker = pF < 3 && pc < CG && gy * CG + pc < ncand;
  float pacc[FM_MAXT][FM_MAXB];
#pragma unroll
  for (int o = 0; o < FM_MAXT; ++o)
#pragma unroll
    for (int a = 0; a < FM_MAXB; ++a) pacc[o][a] = 0.f;
  double *Pb = fp.Pbar + ((size_t)gy * gridDim.x + blockIdx.x) * pot.nsplines * FM_MAXB * CG;
  double *Tb = fp.Tbar + ((size_t)gy * gridDim.x + blockIdx.x) * CG * pot.tab_stride;
  for (int i = tid; i < pot.nsplines * FM_MAXB * CG; i += blockDim.x) Pb[i] = 0.0;
  for (int i = tid; i < CG * pot.tab_stride; i += blockDim.x) Tb[i] = 0.0;
  auto flush_pairs = [&](int tf) {
    if (!pworker) return;
#pragma unroll
    for (int ot = 0; ot < FM_MAXT; ++ot)
      if (ot < pot.ntypes) {
        double *pb = Pb + (size_t)fm_pair_spline(pot, pF, tf, ot) * FM_MAXB * CG + pc;
#pragma unroll
        for (int a = 0; a < FM_MAXB; ++a) {
          pb[(size_t)a * CG] += (double)pacc[ot][a];
          pacc[ot][a] = 0.f;
        }
      }
  };
  __syncthreads();

  int pacc_t = -1, since = 0;
  for (int blk = blockIdx.x; blk < fp.nblk; blk += gridDim.x) {
    const int a0 = fp.blk0[blk], na = fp.blk0[blk + 1] - a0;
    __syncthreads();
    if (tid < na) sm.satom[tid] = db.adj_atoms[a0 + tid];
    __syncthreads();
    if (tid == 0) {
      int lo = 0;
      for (int a = 0; a < na; ++a) {
        sm.arow[a] = lo;
        lo += db.pair_off[sm.satom[a] + 1] - db.pair_off[sm.satom[a]];
      }
      sm.arow[na] = lo;
    }
    __syncthreads();
    const int nslot = sm.arow[na];
    const int ti = db.atom_type[sm.satom[0]];
    if (pacc_t >= 0 && (ti != pacc_t || since == FM_PFLUSH)) {
      flush_pairs(pacc_t);
      since = 0;
    }
    pacc_t = ti;
    ++since;
    const SplineGeom &gU = sg[pot.s_U + ti];
    // ---- per (atom, candidate): K_i, chi_i
    for (int a = set; a < na && live; a += nsets) {
      const int i = sm.satom[a];
      const int64_t p0 = db.pair_off[i];
      const int n = db.pair_off[i + 1] - (int)p0;
      const int cell = db.atom_cell[i];
      const int64_t q0 = fp.row0[i];
      const float *Yq = fp.Y + ((size_t)gy * fp.Q + q0) * 3 * CG + cl;
      const double rho = fp.aoutF[((size_t)gy * N + i) * AO_COUNT * CG + AO_RHO * CG + cl];
      const double w = db.cell_w[cell];
      double rt = rho, dpen = 0.0, drt = 1.0;
      if (rho < gU.x0) {
        dpen = -w * 100.0 * 10. * 2.0 * (gU.x0 - rho);
        if (!pot.embed_extrap) { rt = gU.x0; drt = 0.0; }
      } else if (rho > gU.xN) {
        dpen = w * 100.0 * 10. * 2.0 * (rho - gU.xN);
        if (!pot.embed_extrap) { rt = gU.xN; drt = 0.0; }
      }
      const PointEval U = spl_point(tc, gU, rt);
      double K = 0.0;
      for (int p = 0; p < n; ++p) {
        const FmSlot s = fm_slot(db, pot, p0 + p, ti);
        const FmPairVals v = fm_pair_vals(pot, sg, coefg, CG, s);
        const float *yp = Yq + (size_t)p * 3 * CG;
        const float4 e = *reinterpret_cast<const float4 *>(fp.E + (size_t)(q0 + p) * 8);
        const float2 e2 = *reinterpret_cast<const float2 *>(fp.E + (size_t)(q0 + p) * 8 + 4);
        float lx, ly, lz;
        fm_lambda(db, fp, gy, cl, i, cell, s, lx, ly, lz);
        const float ap = lx * s.ux + ly * s.uy + lz * s.uz;
        const float l1 = lx * e.x + ly * e.y + lz * e.z, l2 = lx * e.w + ly * e2.x + lz * e2.y;
        K += (double)(ap * (v.drho + v.df * yp[0]) + v.f * s.invr * (l1 * yp[CG] + l2 * yp[2 * CG]));
      }
      const double *sd = fp.seedF + ((size_t)gy * NC + cell) * CS_COUNT * CG + cl;
      const double eps = sd[CS_EPS * CG], kap = sd[CS_KAPPA * CG];
      sm.chi[a][cl] = (eps * U.grad + U.grad2 * K) * drt + kap * dpen;
      sm.dF[a][cl] = U.grad;
      sm.K[a][cl] = K;
    }
    __syncthreads();
    // ---- embedding table gradients: one thread per candidate, atoms in order
    if (set == 0 && live) {
      double *tb = Tb + (size_t)cl * pot.tab_stride + gU.toff;
      for (int a = 0; a < na; ++a) {
        const int i = sm.satom[a];
        const double rho = fp.aoutF[((size_t)gy * N + i) * AO_COUNT * CG + AO_RHO * CG + cl];
        const double rt = pot.embed_extrap ? rho : (rho < gU.x0 ? gU.x0 : (rho > gU.xN ? gU.xN : rho));
        const PointEval U = spl_point(tc, gU, rt);
        const double eps = fp.seedF[((size_t)gy * NC + db.atom_cell[i]) * CS_COUNT * CG + CS_EPS * CG + cl];
        spl_point_adjoint(gU, U, rt, eps, sm.K[a][cl], [&](int ix, double x) { tb[ix] += x; });
      }
    }
    // ---- dL/dY over Y and the pair-function weights, chunk by chunk
    for (int c0 = 0; c0 < nslot; c0 += FM_PCHUNK) {
      const int qn = min(FM_PCHUNK, nslot - c0);
      __syncthreads();  // the previous chunk's weights are consumed
      for (int qq = set; qq < qn; qq += nsets) {
        const int ql = c0 + qq;
        int a = 0;
        while (a + 1 < na && sm.arow[a + 1] <= ql) ++a;
        const int i = sm.satom[a];
        const int p = ql - sm.arow[a];
        const FmSlot s = fm_slot(db, pot, db.pair_off[i] + p, ti);
        if (cl == 0) {
          sm.sk[qq][0] = s.kphi;
          sm.sk[qq][1] = s.krho;
          sm.sk[qq][2] = s.kf;
          sm.sb[qq][0] = s.bphi;
          sm.sb[qq][1] = s.brho;
          sm.sb[qq][2] = s.bf;
          sm.stj[qq] = s.tj;
        }
        if (!live) continue;
        const int cell = db.atom_cell[i];
        const FmPairVals v = fm_pair_vals(pot, sg, coefg, CG, s);
        const int64_t q = fp.row0[i] + p;
        float *yp = fp.Y + ((size_t)gy * fp.Q + q) * 3 * CG + cl;
        const float G = yp[0], Y1 = yp[CG], Y2 = yp[2 * CG];
        const float4 e = *reinterpret_cast<const float4 *>(fp.E + (size_t)q * 8);
        const float2 e2 = *reinterpret_cast<const float2 *>(fp.E + (size_t)q * 8 + 4);
        float lx, ly, lz;
        fm_lambda(db, fp, gy, cl, i, cell, s, lx, ly, lz);
        const float ap = lx * s.ux + ly * s.uy + lz * s.uz;
        const float l1 = lx * e.x + ly * e.y + lz * e.z, l2 = lx * e.w + ly * e2.x + lz * e2.y;
        const float chi = (float)sm.chi[a][cl], dF = (float)sm.dF[a][cl];
        const float eps = (float)fp.seedF[((size_t)gy * NC + cell) * CS_COUNT * CG + CS_EPS * CG + cl];
        const float B = dF * v.f * s.invr;
        yp[0] = 0.5f * v.f * chi + ap * dF * v.df;
        yp[CG] = B * l1;
        yp[2 * CG] = B * l2;
        sm.w[qq][0][cl] = 0.5f * eps;
        sm.w[qq][1][cl] = 0.5f * ap;
        sm.w[qq][2][cl] = chi;
        sm.w[qq][3][cl] = dF * ap;
        sm.w[qq][4][cl] = 0.5f * chi * G + dF * (l1 * Y1 + l2 * Y2) * s.invr;
        sm.w[qq][5][cl] = dF * ap * G;
      }
      __syncthreads();
      if (pworker) {
        for (int qq = 0; qq < qn; ++qq) {
          const int k = sm.sk[qq][pF];
          if (k < 0) continue;  // warp-uniform
          const int ot = sm.stj[qq];
          const float b = sm.sb[qq][pF];
          float Nv[4], Nd[4];
          bsp_basis<float>(b, Nv);
          bsp_dbasis<float>(b, Nd);
          const float inv = (float)sg[fm_pair_spline(pot, pF, ti, ot)].invstep;
          const float wv = sm.w[qq][2 * pF][pc], wd = sm.w[qq][2 * pF + 1][pc] * inv;
          const float c0v = wv * Nv[0] + wd * Nd[0], c1v = wv * Nv[1] + wd * Nd[1], c2v = wv * Nv[2] + wd * Nd[2],
                      c3v = wv * Nv[3] + wd * Nd[3];
          switch (ot * FM_MAXB + k) {
#define FM_CASE(OT, K)      \
  case OT * FM_MAXB + K:    \
    pacc[OT][K] += c0v;     \
    pacc[OT][K + 1] += c1v; \
    pacc[OT][K + 2] += c2v; \
    pacc[OT][K + 3] += c3v; \
    break;
#define FM_CASES(OT)                                                                                       \
  FM_CASE(OT, 0) FM_CASE(OT, 1) FM_CASE(OT, 2) FM_CASE(OT, 3) FM_CASE(OT, 4) FM_CASE(OT, 5) FM_CASE(OT, 6) \
  FM_CASE(OT, 7) FM_CASE(OT, 8) FM_CASE(OT, 9) FM_CASE(OT, 10) FM_CASE(OT, 11) FM_CASE(OT, 12)             \
  FM_CASE(OT, 13) FM_CASE(OT, 14) FM_CASE(OT, 15) FM_CASE(OT, 16) FM_CASE(OT, 17) FM_CASE(OT, 18)          \
  FM_CASE(OT, 19) FM_CASE(OT, 20)
            FM_CASES(0)
            FM_CASES(1)
#undef FM_CASES
#undef FM_CASE
            default:
              break;
          }
        }
      }
    }
  }
  __syncthreads();
  if (pacc_t >= 0) flush_pairs(pacc_t);
}

// ---------------------------------------------------------- k_fm_gemm_adj

// Kbar_s[d][c] += sum_{q,t} X[t][d][q] Ybar[q][t][c] over this CTA's run of
// tiles, sub-tile by sub-tile of FM_SUB slots (all Dpad features of the three
// kinds in shared memory).  Thread: FM_ROWS consecutive features x 8
// candidates, FP32 sums flushed into this CTA's FP64 partial of the tile's
// atom type after every tile.
__host__ __device__ inline size_t fm_adj_smem(int Dpad, int CG) {
  return sizeof(float) * ((size_t)3 * Dpad * FM_SUB + (size_t)FM_SUB * 3 * CG);
}

__global__ void __launch_bounds__(256, 1) k_fm_gemm_adj(FmPlan fp) {
  extern __shared__ __align__(16) float asm_[];
  const int CG = fp.CG, gy = blockIdx.y;
  float *Xs = asm_;                               // [3 Dpad rows: (kind, feature)][FM_SUB]
  float *Ys = Xs + (size_t)3 * fp.Dpad * FM_SUB;  // [FM_SUB][3][CG]
  const int tid = threadIdx.x;
  const int ncs = CG / 8, nds = fp.Dpad / FM_ROWS;
  const int cs = tid % ncs, ds = tid / ncs;
  const bool worker = ds < nds;
  const int per = (fp.ntiles + gridDim.x - 1) / gridDim.x;
  const int tb = blockIdx.x * per, te = min(fp.ntiles, tb + per);
  double *Kb = fp.Kbar + ((size_t)gy * gridDim.x + blockIdx.x) * fp.nt * fp.Dpad * CG;
  for (int i = tid; i < fp.nt * fp.Dpad * CG; i += blockDim.x) Kb[i] = 0.0;
  float acc[FM_ROWS][8];
#pragma unroll
  for (int r = 0; r < FM_ROWS; ++r)
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[r][c] = 0.f;
  for (int tile = tb; tile < te; ++tile) {
    const int s = fm_tile_type(fp, tile);
    for (int sub = 0; sub < FM_TILE; sub += FM_SUB) {
      const int64_t qb = (int64_t)tile * FM_TILE + sub;
      __syncthreads();
      const int nrow = 3 * fp.Dpad;
      for (int i = tid; i < nrow * (FM_SUB / 4); i += blockDim.x) {
        const int row = i / (FM_SUB / 4), col = (i % (FM_SUB / 4)) * 4;
        const int t = row / fp.Dpad, d = row % fp.Dpad;
        const size_t grow = (size_t)((d / FM_DC) * 3 + t) * FM_DC + d % FM_DC;
        cp_async16(Xs + (size_t)row * FM_SUB + col, fp.X + grow * fp.Q + qb + col);
      }
      const float *ysrc = fp.Y + ((size_t)gy * fp.Q + qb) * 3 * CG;
      for (int i = tid * 4; i < FM_SUB * 3 * CG; i += blockDim.x * 4) cp_async16(Ys + i, ysrc + i);
      cp_async_commit();
      cp_async_wait<0>();
      __syncthreads();
      if (worker) {
#pragma unroll
        for (int t = 0; t < 3; ++t)
#pragma unroll
          for (int qg = 0; qg < FM_SUB; qg += 4) {
            float4 xv[FM_ROWS];
#pragma unroll
            for (int r = 0; r < FM_ROWS; ++r)
              xv[r] = *reinterpret_cast<const float4 *>(Xs + ((size_t)t * fp.Dpad + ds * FM_ROWS + r) * FM_SUB + qg);
#pragma unroll
            for (int qq = 0; qq < 4; ++qq) {
              const float *yq = Ys + ((size_t)(qg + qq) * 3 + t) * CG + cs * 8;
              const float4 y0 = *reinterpret_cast<const float4 *>(yq), y1 = *reinterpret_cast<const float4 *>(yq + 4);
              const float yv[8] = {y0.x, y0.y, y0.z, y0.w, y1.x, y1.y, y1.z, y1.w};
#pragma unroll
              for (int r = 0; r < FM_ROWS; ++r) {
                const float x = qq == 0 ? xv[r].x : qq == 1 ? xv[r].y : qq == 2 ? xv[r].z : xv[r].w;
#pragma unroll
                for (int c = 0; c < 8; ++c) acc[r][c] = fmaf(x, yv[c], acc[r][c]);
              }
            }
          }
      }
    }
    if (worker) {
      double *kb = Kb + ((size_t)s * fp.Dpad + ds * FM_ROWS) * CG + cs * 8;
#pragma unroll
      for (int r = 0; r < FM_ROWS; ++r)
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          kb[(size_t)r * CG + c] += (double)acc[r][c];
          acc[r][c] = 0.f;
        }
    }
  }
}

// -------------------------------------------------------------- k_fm_grad

// Per candidate: the CTA partials summed in order; the contraction's Kbar
// split into its factors (dL/dc_a = sum_n Kbar w_n, dL/dw_n = sum_a Kbar c_a);
// the B-spline coefficient gradients of phi, rho, f, g mapped to the knot
// table (the transpose of k_fm_coef's map); the embedding table gradients
// added.  The result is one table-gradient partial, which k_grad_final maps
// to the coefficients.
__global__ void k_fm_grad(DevPot pot, const SplineGeom *__restrict__ geom, FmPlan fp,
                          const double *__restrict__ coef64, double *__restrict__ out) {
  extern __shared__ double gsm[];
  const int c = blockIdx.x, CG = fp.CG, gy = c / CG, cl = c % CG;
  const int ns = pot.nsplines, stride = pot.tab_stride;
  double *bgrad = gsm;                         // [ns][FM_MAXB]
  double *tab = bgrad + (size_t)ns * FM_MAXB;  // [stride]
  double *kbar = tab + stride;                 // [nt][Dpad]
  for (int i = threadIdx.x; i < ns * FM_MAXB; i += blockDim.x) {
    const int s = i / FM_MAXB, a = i % FM_MAXB;
    double v = 0.0;
    for (int b = 0; b < fp.nctas_pre; ++b)
      v += fp.Pbar[(((size_t)gy * fp.nctas_pre + b) * ns + s) * FM_MAXB * CG + (size_t)a * CG + cl];
    bgrad[i] = v;
  }
  for (int e = threadIdx.x; e < stride; e += blockDim.x) {
    double v = 0.0;
    for (int b = 0; b < fp.nctas_pre; ++b) v += fp.Tbar[(((size_t)gy * fp.nctas_pre + b) * CG + cl) * stride + e];
    tab[e] = v;
  }
  for (int i = threadIdx.x; i < fp.nt * fp.Dpad; i += blockDim.x) {
    double v = 0.0;
    for (int b = 0; b < fp.nctas_adj; ++b)
      v += fp.Kbar[(((size_t)gy * fp.nctas_adj + b) * fp.nt * fp.Dpad + i) * CG + cl];
    kbar[i] = v;
  }
  __syncthreads();
  const double *cf = coef64 + (size_t)c * ns * FM_MAXB;
  if (threadIdx.x == 0) {
    // Kbar -> f and g coefficient gradients, in a fixed order
    for (int s = 0; s < fp.nt; ++s) {
      const int gs = pot.s_g + s;
      for (int o = 0; o < fp.nt; ++o) {
        const int fs = pot.s_f + pair_ij_index(s, o, pot.ntypes);
        for (int a = 0; a < fp.NA; ++a)
          for (int nn = 0; nn < fp.NN; ++nn) {
            const double kb = kbar[(size_t)s * fp.Dpad + (o * fp.NA + a) * fp.NN + nn];
            bgrad[(size_t)fs * FM_MAXB + a] += kb * cf[(size_t)gs * FM_MAXB + nn];
            bgrad[(size_t)gs * FM_MAXB + nn] += kb * cf[(size_t)fs * FM_MAXB + a];
          }
      }
    }
    // B-spline coefficient gradients -> (y, y'') table gradients of phi, rho, f, g
    for (int s = 0; s < ns; ++s) {
      if (s >= pot.s_U && s < pot.s_f) continue;  // U: table gradients already
      const SplineGeom g = geom[s];
      const int n = g.n;
      const double H = g.step * g.step / 6.0, h2 = g.step * g.step;
      const double *db = bgrad + (size_t)s * FM_MAXB;
      double *y = tab + g.toff, *ypp = y + n;
      // d_m+1 = y_m - H y''_m
      for (int m = 0; m < n; ++m) {
        y[m] += db[m + 1];
        ypp[m] -= H * db[m + 1];
      }
      // d_0 = h2 y''_0 + 2 (y_0 - H y''_0) - (y_1 - H y''_1)
      y[0] += 2.0 * db[0];
      ypp[0] += (h2 - 2.0 * H) * db[0];
      y[1] -= db[0];
      ypp[1] += H * db[0];
      // d_n+1 = h2 y''_n-1 + 2 (y_n-1 - H y''_n-1) - (y_n-2 - H y''_n-2)
      y[n - 1] += 2.0 * db[n + 1];
      ypp[n - 1] += (h2 - 2.0 * H) * db[n + 1];
      y[n - 2] -= db[n + 1];
      ypp[n - 2] += H * db[n + 1];
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < stride; e += blockDim.x) out[(size_t)c * stride + e] = tab[e];
}

}  // namespace mzb
