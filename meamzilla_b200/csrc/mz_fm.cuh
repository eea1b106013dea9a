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
//   E     [Q][8]                     e1, e2 of the slot (FP64)
//   Y     [ngroups][Q][3][CG]        G, Y1, Y2 (FP32)
//   Yb    [ngroups][Q][3][CG]        dL/dG, dL/dY1, dL/dY2 (FP32)
//   V     [ngroups][Np][CG][3]       reaction vectors (FP64), global slot order
//   aoutF [ngroups][N][AO_COUNT][CG] per-atom outputs (FP64)
// with candidates in groups of CG (the launch's candidates rounded up to a
// power of two from 8 to 64).
#pragma once

#include "mz_adj.cuh"

namespace mzb {

constexpr int FM_TILE = 64;    // feature slots per contraction tile
constexpr int FM_DC = 24;      // features per chunk of the forward contraction
constexpr int FM_MAXT = 2;     // atom types
constexpr int FM_MAXN = 16;    // B-spline coefficients of a g spline (knots + 2)
constexpr int FM_MAXB = 24;    // B-spline coefficients of any spline the path reads (knots + 2)
constexpr int FM_SUB = 16;     // feature slots per sub-tile of the adjoint contraction
constexpr int FM_ROWS = 8;     // features per thread in the adjoint contraction
constexpr int FM_PCHUNK = 32;  // slots per chunk of the pair-function gradient
constexpr int FM_PB = 4;       // slots per batch of loads in the row walks (the pre pass's second: 2 FM_PB)
constexpr int FM_PBW = 2 * FM_PB;

struct FmPlan {
  int nt;          // atom types
  int NA, NN;      // B-spline coefficients per f spline, per g spline (the largest)
  int D, Dpad;     // features per kind: nt NA NN, padded to a multiple of FM_DC
  int nch;         // Dpad / FM_DC
  int CG;          // candidates per group
  int64_t Q;       // feature slots
  int ntiles;      // Q / FM_TILE
  int tile0[FM_MAXT + 1];  // first tile of each type
  int64_t qend[FM_MAXT];   // end of each type's real slots (the rest of its last tile is padding)
  int NB;          // B-spline coefficients of the phi, rho and f splines (the largest)
  int utoff, ustride;  // the U splines' part of a knot table: its offset and length
  int nblk;        // atom blocks of the epilogues (type-pure, <= BLOCK_SLOTS slots, <= FM_ABLK atoms)
  const int *blk0;         // [nblk + 1] into adj_atoms
  const int *row0;         // [N] feature slot of each atom's first pair
  const float *X;
  const double *E;         // [Q][8] e1, e2 of each slot (FP64)
  float *Y;                // [ngroups][Q][3][CG] G, Y1, Y2 (the contraction's sums, rounded once to FP32)
  float *Yb;               // [ngroups][Q][3][CG] dL/dG, dL/dY1, dL/dY2 (FP32, the adjoint's operand)
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
  // the integer contraction (mz_fm8.cuh), when built
  const signed char *X8;   // [Q / 128][3][2][3][16 KB]
  const signed char *xe;   // [Q][4]
  signed char *K8;         // [ngroups][nt][2][3][8 KB]
  int *ke;                 // [ngroups][nt][64]
  int *zmax;               // [ngroups][Q / 128][64] exponent bounds of the adjoint operand per tile (or null)
};

// ------------------------------------------- digits of the integer contraction
// (the tensor-core forward of mz_fm8.cuh; constants and layouts described there)
constexpr int FM8_TM = 128;                      // slots per tile (MMA M)
constexpr int FM8_D = 256;                       // features per kind, padded (MMA K in bytes)
constexpr int FM8_NC = 64;                       // candidates per MMA (N), the group padded
constexpr int FM8_DIG = 4;                       // base-256 digits per number
constexpr int FM8_CLS = 4;                       // weight classes kept (i + j <= 3)
constexpr int FM8_XBLK = FM8_TM * 128;           // one (digit, kblock) block of a tile: 16 KB
constexpr int FM8_KBLK = FM8_NC * 128;           // one (digit, kblock) block of K8: 8 KB
constexpr int FM8_STAGE = FM8_DIG * FM8_XBLK;    // one (tile, kind, kblock): 64 KB
constexpr int FM8_BTYPE = 2 * FM8_DIG * FM8_KBLK;  // K8 of one type: 64 KB
constexpr int FM8_SHIFT = 30;                    // |X_int|, |K_int| <= 2^30
constexpr int FM8_NST = 8;                       // stages in the ring, one (tile, kind, kblock, digit) block each
constexpr int FM8_THREADS = 320;                 // producer, MMA, eight epilogue warps
constexpr uint32_t FM8_WAIT = 1u << 26;          // polls before a wait gives up
constexpr int FM8_SPAN_LOG = 3;
constexpr int FM8_SPAN = 1 << FM8_SPAN_LOG;      // tiles per exponent span of the integer adjoint's operand

// byte of (row r, byte k) in a SW128 K-major block
__host__ __device__ inline uint32_t sw128_byte(int r, int k) {
  return (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((((k >> 4) ^ r) & 7) << 4) + (k & 15));
}
// first byte of X8 block (tile T, kind t, kblock kb, digit l)
__host__ __device__ inline size_t x8_block(int64_t T, int t, int kb, int l) {
  return ((((size_t)T * 3 + t) * 2 + kb) * FM8_DIG + l) * FM8_XBLK;
}
// first byte of K8 block (group gy, type s, kblock kb, digit l)
__host__ __device__ inline size_t k8_block(int gy, int s, int nt, int kb, int l) {
  return ((((size_t)gy * nt + s) * 2 + kb) * FM8_DIG + l) * FM8_KBLK;
}

// Balanced base-256 digits of an integer |v| <= 2^30:
// v = d0 2^24 + d1 2^16 + d2 2^8 + d3, d1..d3 in [-128, 127], d0 in [-64, 64].
__host__ __device__ inline void digits256(long long v, signed char *d) {
#pragma unroll
  for (int l = FM8_DIG - 1; l > 0; --l) {
    const long long lo = ((v + 128) & 255) - 128;
    d[l] = (signed char)lo;
    v = (v - lo) / 256;
  }
  d[0] = (signed char)v;
}

// The binary exponent e with |v| < 2^e for the largest |v| of a row (0 for a
// zero row), kept in [-100, 100] (smaller rows quantise to zero).
__host__ __device__ inline int fm8_exponent(double amax) {
  if (!(amax > 0.0)) return 0;
  int e;
  frexp(amax, &e);
  return e < -100 ? -100 : (e > 100 ? 100 : e);
}

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
                                                     FmPlan fp, float *__restrict__ X, double *__restrict__ E,
                                                     signed char *__restrict__ X8, signed char *__restrict__ xe) {
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
    if (X && active) {
#pragma unroll
      for (int t = 0; t < 3; ++t)
#pragma unroll
        for (int nn = 0; nn < FM_MAXN; ++nn)
          if (nn < fp.NN) {
            const int d = lane * fp.NN + nn, ch = d / FM_DC, din = d % FM_DC;
            X[((size_t)(ch * 3 + t) * FM_DC + din) * fp.Q + q] = (float)acc[t][nn];
          }
    }
    if (X8) {  // the same moments as digits for the integer contraction (mz_fm8.cuh)
#pragma unroll
      for (int t = 0; t < 3; ++t) {
        double m = 0.0;
#pragma unroll
        for (int nn = 0; nn < FM_MAXN; ++nn)
          if (active && nn < fp.NN) m = fmax(m, fabs(acc[t][nn]));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        const int e = fm8_exponent(m);
        if (lane == 0) xe[q * 4 + t] = (signed char)e;
        if (active) {
          const int64_t T = q / FM8_TM;
          const int r = (int)(q % FM8_TM);
#pragma unroll
          for (int nn = 0; nn < FM_MAXN; ++nn)
            if (nn < fp.NN) {
              const int d = lane * fp.NN + nn;
              signed char dg[FM8_DIG];
              digits256(llrint(ldexp(acc[t][nn], FM8_SHIFT - e)), dg);
              const uint32_t o = sw128_byte(r, d & 127);
#pragma unroll
              for (int l = 0; l < FM8_DIG; ++l) X8[x8_block(T, t, d >> 7, l) + o] = dg[l];
            }
        }
      }
    }
    if (lane == 0) {
      double *e = E + (size_t)q * 8;
      e[0] = e1[0]; e[1] = e1[1]; e[2] = e1[2];
      e[3] = e2[0]; e[4] = e2[1]; e[5] = e2[2];
      e[6] = 0.0; e[7] = 0.0;
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
// (lane, warp): slots 2 lane and 2 lane + 1, candidates 8 warp .. 8 warp + 7,
// all three kinds.  Each chunk of FM_DC features is summed in FP32 (packed
// pairs of slots) and added to a compensated FP32 total (TwoSum: the total
// and the exact rounding error of each addition, packed pairs), stored as
// their FP64 sum, so a sum carries the rounding of FM_DC terms, not of all
// Dpad.  The moments stream through a double buffer
// filled by cp.async; K_s stays in shared memory for the whole tile.
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
  float2 tot[3][8], cmp[3][8];  // [kind][candidate]: (slot 2 lane, slot 2 lane + 1), total and its error
#pragma unroll
  for (int t = 0; t < 3; ++t)
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      tot[t][c] = make_float2(0.f, 0.f);
      cmp[t][c] = make_float2(0.f, 0.f);
    }
  for (int ch = 0; ch < fp.nch; ++ch) {
    if (ch + 1 < fp.nch) {
      load_chunk(ch + 1, (ch + 1) & 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const float *xb = Xs + (size_t)(ch & 1) * 3 * FM_DC * FM_TILE + 2 * lane;
    const float *kb = Ks + (size_t)ch * FM_DC * CG + warp * 8;
    float2 acc[3][8];  // this chunk, (slot 2 lane, slot 2 lane + 1)
#pragma unroll
    for (int t = 0; t < 3; ++t)
#pragma unroll
      for (int c = 0; c < 8; ++c) acc[t][c] = make_float2(0.f, 0.f);
#pragma unroll 4
    for (int din = 0; din < FM_DC; ++din) {
      const float4 k0 = *reinterpret_cast<const float4 *>(kb + din * CG);
      const float4 k1 = *reinterpret_cast<const float4 *>(kb + din * CG + 4);
      const float kk[8] = {k0.x, k0.y, k0.z, k0.w, k1.x, k1.y, k1.z, k1.w};
#pragma unroll
      for (int t = 0; t < 3; ++t) {
        const float2 xv = *reinterpret_cast<const float2 *>(xb + (t * FM_DC + din) * FM_TILE);
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[t][c] = fma2(xv, bcast2(kk[c]), acc[t][c]);
      }
    }
    // TwoSum (Knuth): s = a + b exactly as s + err
#pragma unroll
    for (int t = 0; t < 3; ++t)
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const float2 a = tot[t][c], b = acc[t][c];
        const float2 sum = add2(a, b);
        const float2 bb = add2(sum, make_float2(-a.x, -a.y));
        const float2 err = add2(add2(a, make_float2(-(sum.x - bb.x), -(sum.y - bb.y))), add2(b, make_float2(-bb.x, -bb.y)));
        tot[t][c] = sum;
        cmp[t][c] = add2(cmp[t][c], err);
      }
    __syncthreads();
  }
  float *Yo = fp.Y + ((size_t)gy * fp.Q + qb + 2 * lane) * 3 * CG + warp * 8;
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int t = 0; t < 3; ++t) {
      float *dst = Yo + ((size_t)h * 3 + t) * CG;
#pragma unroll
      for (int c = 0; c < 8; c += 2) {
        const double v0 = h ? (double)tot[t][c].y + (double)cmp[t][c].y : (double)tot[t][c].x + (double)cmp[t][c].x;
        const double v1 =
            h ? (double)tot[t][c + 1].y + (double)cmp[t][c + 1].y : (double)tot[t][c + 1].x + (double)cmp[t][c + 1].x;
        *reinterpret_cast<float2 *>(dst + c) = make_float2((float)v0, (float)v1);
      }
    }
}

// ------------------------------------------------------ block staging

// The epilogues walk the type-pure atom blocks (at most BLOCK_SLOTS slots
// and FM_ABLK atoms).  Everything of a block that does not depend on the
// candidate is staged once in shared memory: per slot its global index,
// neighbour, neighbour type, knots, the FP32 unit vector and 1/r, the FP64
// frame (e1, e2), and the B-spline basis values (and d/dr) of phi, rho and f
// at its shifts; and the pair splines' B-spline coefficients of the block's
// atom type for the group's candidates.
constexpr int FM_ABLK = 4;   // atoms per block of the epilogues: 4 x 64 candidates fill 256 threads

template <typename R>
struct FmStage {
  int *satom, *arow;  // [FM_ABLK], [FM_ABLK + 1]
  int *gs, *nbr, *tj, *kn;  // [BLOCK_SLOTS]
  int *ctype;         // type whose coefficients are staged (-1: none yet)
  float4 *uf;         // [BLOCK_SLOTS] (ux, uy, uz, 1/r)
  double *e;          // [BLOCK_SLOTS][6] e1 / r, e2 / r (FP32 stages keep e1, e2 as floats in the same space)
  double4 *ur;        // [BLOCK_SLOTS] (ux, uy, uz, r) in FP64
  R *bas;             // [BLOCK_SLOTS][3][8] basis N0..N3 and d/dr N0'..N3' of phi, rho, f
  R *coef;            // [3][nt][NB][CG]
};

template <typename R>
__host__ __device__ inline size_t fm_stage_bytes(int nt, int NB, int CG) {
  return sizeof(int) * (2 * FM_ABLK + 2 + 4 * BLOCK_SLOTS) + 16 + (sizeof(R) == 4 ? sizeof(float4) * BLOCK_SLOTS : 0) +
         sizeof(double4) * BLOCK_SLOTS + sizeof(double) * 6 * BLOCK_SLOTS + sizeof(R) * 24 * BLOCK_SLOTS +
         sizeof(R) * 3 * nt * NB * CG;
}

// carves the staging arrays out of shared memory at `base` (16-byte aligned)
template <typename R>
__device__ __forceinline__ FmStage<R> fm_stage_carve(unsigned char *base, const FmPlan &fp) {
  FmStage<R> st;
  double4 *ur = reinterpret_cast<double4 *>(base);
  st.ur = ur;
  double *e = reinterpret_cast<double *>(ur + BLOCK_SLOTS);
  st.e = e;
  // the FP32 unit vectors only where the FP32 epilogue reads them
  float4 *uf = reinterpret_cast<float4 *>(e + 6 * BLOCK_SLOTS);
  st.uf = uf;
  R *bas = reinterpret_cast<R *>(uf + (sizeof(R) == 4 ? BLOCK_SLOTS : 0));
  st.bas = bas;
  R *coef = bas + 24 * BLOCK_SLOTS;
  st.coef = coef;
  int *ip = reinterpret_cast<int *>(coef + 3 * fp.nt * fp.NB * fp.CG);
  st.satom = ip;
  st.arow = ip + FM_ABLK;
  st.gs = st.arow + FM_ABLK + 1;
  st.nbr = st.gs + BLOCK_SLOTS;
  st.tj = st.nbr + BLOCK_SLOTS;
  st.kn = st.tj + BLOCK_SLOTS;
  st.ctype = st.kn + BLOCK_SLOTS;
  return st;
}

// The spline of pair function F (0 phi, 1 rho, 2 f) for a centre of type ti
// and a neighbour of type tj.
__device__ __forceinline__ int fm_pair_spline(const DevPot &pot, int F, int ti, int tj) {
  return F == 1 ? pot.s_rho + tj : (F == 0 ? pot.s_phi : pot.s_f) + pair_ij_index(ti, tj, pot.ntypes);
}

// Stages block blk; returns its slot count (all threads; barriers inside).
// FP32 coefficients come from the group's FP32 table, FP64 ones from the
// candidates' FP64 coefficients.
template <typename R>
__device__ int fm_stage_block(const DevDb &db, const DevPot &pot, const SplineGeom *sg, const FmPlan &fp,
                              const FmStage<R> &st, int blk, int gy, int ncand, int &na_out, int &ti_out) {
  const int tid = threadIdx.x, T = blockDim.x, CG = fp.CG;
  const int a0 = fp.blk0[blk], na = fp.blk0[blk + 1] - a0;
  __syncthreads();  // the previous block is done with the staging
  if (tid < na) st.satom[tid] = db.adj_atoms[a0 + tid];
  __syncthreads();
  if (tid == 0) {
    int lo = 0;
    for (int a = 0; a < na; ++a) {
      st.arow[a] = lo;
      lo += db.pair_off[st.satom[a] + 1] - db.pair_off[st.satom[a]];
    }
    st.arow[na] = lo;
  }
  __syncthreads();
  const int nslot = st.arow[na];
  const int ti = db.atom_type[st.satom[0]];
  const int64_t Np = db.npairs;
  for (int ql = tid; ql < nslot; ql += T) {
    const int a = slot_owner(st.arow, na, ql);
    const int i = st.satom[a], p = ql - st.arow[a];
    const int64_t gs = db.pair_off[i] + p;
    const int j = db.pair_nbr[gs];
    st.gs[ql] = (int)gs;
    st.nbr[ql] = j;
    const int tj = db.atom_type[j];
    st.tj[ql] = tj;
    const int kn = db.pair_knot[gs];
    st.kn[ql] = kn;
    if (sizeof(R) == 4) st.uf[ql] = make_float4(db.pair_uxf[gs], db.pair_uyf[gs], db.pair_uzf[gs], 1.f / db.pair_rf[gs]);
    st.ur[ql] = make_double4(db.pair_ux[gs], db.pair_uy[gs], db.pair_uz[gs], db.pair_r[gs]);
    const double *e = fp.E + (size_t)(fp.row0[i] + p) * 8;
    const double ir = 1.0 / db.pair_r[gs];  // the FP64 stage keeps e1 / r, e2 / r (its only use)
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      if (sizeof(R) == 4) reinterpret_cast<float *>(st.e)[ql * 6 + k] = (float)e[k];
      else st.e[ql * 6 + k] = e[k] * ir;
    }
#pragma unroll
    for (int F = 0; F < 3; ++F) {
      const int k = ((kn >> (8 * F)) & 0xff) - 1;
      R *bs = st.bas + (ql * 3 + F) * 8;
      if (k >= 0) {
        const R b = sizeof(R) == 8 ? (R)db.pair_shift[(int64_t)F * Np + gs] : (R)db.pair_shiftf[(int64_t)F * Np + gs];
        bsp_basis<R>(b, bs);
        bsp_dbasis<R>(b, bs + 4);
        const R inv = (R)sg[fm_pair_spline(pot, F, ti, tj)].invstep;
#pragma unroll
        for (int q = 4; q < 8; ++q) bs[q] *= inv;
      } else {
#pragma unroll
        for (int q = 0; q < 8; ++q) bs[q] = R(0);
      }
    }
  }
  // the pair coefficients of the block's type (consecutive blocks of a CTA
  // are mostly of one type: restaged only at a change)
  const bool restage = *st.ctype != ti;
  __syncthreads();
  const int ncf = restage ? 3 * fp.nt * fp.NB * CG : 0;
  if (restage && tid == 0) *st.ctype = ti;
  for (int idx = tid; idx < ncf; idx += T) {
    const int cl = idx % CG, a = (idx / CG) % fp.NB, o = (idx / (CG * fp.NB)) % fp.nt, F = idx / (CG * fp.NB * fp.nt);
    const int sp = fm_pair_spline(pot, F, ti, o);
    if (sizeof(R) == 8) {
      const int c = gy * CG + cl;
      st.coef[idx] = c < ncand ? (R)fp.coef64[((size_t)c * pot.nsplines + sp) * FM_MAXB + a] : R(0);
    } else {
      st.coef[idx] = (R)fp.coef32[(((size_t)gy * pot.nsplines + sp) * FM_MAXB + a) * CG + cl];
    }
  }
  __syncthreads();
  na_out = na;
  ti_out = ti;
  return nslot;
}

// phi, rho, f (values and d/dr) of staged slot ql for candidate cl
template <typename R>
struct FmPairVals {
  R phi, dphi, rho, drho, f, df;
};
// the staged basis of slot ql for pair function F: N0..N3, then their d/dr
// (16-byte shared loads, the same address in every lane)
__device__ __forceinline__ void fm_bas(const FmStage<float> &st, int ql, int F, float *b) {
  const float4 *p = reinterpret_cast<const float4 *>(st.bas + (ql * 3 + F) * 8);
  const float4 x = p[0], y = p[1];
  b[0] = x.x; b[1] = x.y; b[2] = x.z; b[3] = x.w;
  b[4] = y.x; b[5] = y.y; b[6] = y.z; b[7] = y.w;
}
__device__ __forceinline__ void fm_bas(const FmStage<double> &st, int ql, int F, double *b) {
  const double2 *p = reinterpret_cast<const double2 *>(st.bas + (ql * 3 + F) * 8);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const double2 x = p[i];
    b[2 * i] = x.x;
    b[2 * i + 1] = x.y;
  }
}

// value and d/dr of pair function F at staged slot ql for candidate cl
template <typename R>
__device__ __forceinline__ void fm_pair_val(const FmStage<R> &st, const FmPlan &fp, int ql, int cl, int F, int kn,
                                            int tj, R &v, R &d) {
  const int k = ((kn >> (8 * F)) & 0xff) - 1;
  R bs[8];
  fm_bas(st, ql, F, bs);
  const int CG = fp.CG;
  const R *cf = st.coef + ((size_t)(F * fp.nt + tj) * fp.NB + (k < 0 ? 0 : k)) * CG + cl;
  const R c0 = cf[0], c1 = cf[CG], c2 = cf[2 * CG], c3 = cf[3 * CG];
  v = bs[0] * c0 + bs[1] * c1 + bs[2] * c2 + bs[3] * c3;  // zero basis where k < 0
  d = bs[4] * c0 + bs[5] * c1 + bs[6] * c2 + bs[7] * c3;
}

// only the value (d = 0) or only d/dr (d = 1) of pair function F
template <typename R>
__device__ __forceinline__ R fm_pair_one(const FmStage<R> &st, const FmPlan &fp, int ql, int cl, int F, int kn, int tj,
                                         int d) {
  const int k = ((kn >> (8 * F)) & 0xff) - 1;
  const R *bs = st.bas + (ql * 3 + F) * 8 + 4 * d;
  R b[4];
  if (sizeof(R) == 4) {
    const float4 x = *reinterpret_cast<const float4 *>(bs);
    b[0] = x.x; b[1] = x.y; b[2] = x.z; b[3] = x.w;
  } else {
    const double2 x = reinterpret_cast<const double2 *>(bs)[0], y = reinterpret_cast<const double2 *>(bs)[1];
    b[0] = x.x; b[1] = x.y; b[2] = y.x; b[3] = y.y;
  }
  const int CG = fp.CG;
  const R *cf = st.coef + ((size_t)(F * fp.nt + tj) * fp.NB + (k < 0 ? 0 : k)) * CG + cl;
  return b[0] * cf[0] + b[1] * cf[CG] + b[2] * cf[2 * CG] + b[3] * cf[3 * CG];  // zero basis where k < 0
}

template <typename R>
__device__ __forceinline__ FmPairVals<R> fm_pair_vals(const FmStage<R> &st, const FmPlan &fp, int ql, int cl) {
  R v[3], d[3];
  const int kn = st.kn[ql], tj = st.tj[ql];
#pragma unroll
  for (int F = 0; F < 3; ++F) fm_pair_val(st, fp, ql, cl, F, kn, tj, v[F], d[F]);
  return FmPairVals<R>{v[0], d[0], v[1], d[1], v[2], d[2]};
}

// ---------------------------------------------------------------- k_fm_epi

// Forward epilogue, persistent CTAs over the atom blocks, one task per
// (atom, candidate of group blockIdx.y): the density
// rho_i = sum_p rho_p + 1/2 f_p G_p and the pair energy in FP64 over the
// atom's row, the embedding (clamp and punishment,
// pot_meam_spline.cpp:208-223), then per slot the reaction vector, in FP64,
//   V_p = u_p (phi'_p / 2 + U' (rho'_p + f'_p G_p)) + U' f_p / r_p (e1 Y1 + e2 Y2)
// (the force atom i's terms put on it along slot p; the neighbour receives
// -V_p), with the atom's own force and virial sums.  The pair functions are
// evaluated in FP64 here (from the candidates' FP64 B-spline coefficients):
// the forces are sums of reaction vectors much larger than they are.
__host__ __device__ inline size_t fm_epi_smem(int nsplines, int nt, int NB, int CG) {
  return ((fm_stage_bytes<double>(nt, NB, CG) + 15) & ~size_t(15)) + sizeof(SplineGeom) * (size_t)nsplines;
}

__global__ void __launch_bounds__(256) k_fm_epi(DevDb db, DevPot pot, const SplineGeom *__restrict__ geom,
                                               const double *__restrict__ tabs, FmPlan fp, int ncand) {
  extern __shared__ __align__(16) unsigned char fm_raw[];
  const FmStage<double> st = fm_stage_carve<double>(fm_raw, fp);
  SplineGeom *sg = reinterpret_cast<SplineGeom *>(
      fm_raw + ((fm_stage_bytes<double>(fp.nt, fp.NB, fp.CG) + 15) & ~size_t(15)));
  const int gy = blockIdx.y, CG = fp.CG, N = db.natoms;
  const int tid = threadIdx.x, T = blockDim.x;
  for (int s = tid; s < pot.nsplines; s += T) sg[s] = geom[s];
  if (tid == 0) *st.ctype = -1;
  const int cl = tid % CG;
  const int c = gy * CG + cl;
  const bool live = c < ncand;
  const double *tc = tabs + (size_t)(live ? c : 0) * pot.tab_stride;
  double *__restrict__ Vg = fp.V + (size_t)gy * db.npairs * CG * 3 + cl * 3;
  for (int blk = blockIdx.x; blk < fp.nblk; blk += gridDim.x) {
    int na, ti;
    const int nslot = fm_stage_block<double>(db, pot, sg, fp, st, blk, gy, ncand, na, ti);
    (void)nslot;
    if (!live) continue;
    const SplineGeom &gU = sg[pot.s_U + ti];
    for (int task = tid; task < na * CG; task += T) {
      const int a = task / CG;
      const int i = st.satom[a], lo = st.arow[a], n = st.arow[a + 1] - lo;
      const float *Yq = fp.Y + ((size_t)gy * fp.Q + fp.row0[i]) * 3 * CG + cl;
      double rho = 0.0, epair = 0.0;
#pragma unroll 4
      for (int p = 0; p < n; ++p) {
        const int ql = lo + p, kn = st.kn[ql], tj = st.tj[ql];
        const double phi = fm_pair_one<double>(st, fp, ql, cl, 0, kn, tj, 0);
        const double rv = fm_pair_one<double>(st, fp, ql, cl, 1, kn, tj, 0);
        const double fv = fm_pair_one<double>(st, fp, ql, cl, 2, kn, tj, 0);
        rho += rv + 0.5 * fv * (double)Yq[(size_t)p * 3 * CG];
        epair += 0.5 * phi;
      }
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
      const double dF = U.grad;
      double F[3] = {0, 0, 0}, S[6] = {0, 0, 0, 0, 0, 0};
      // slots in batches of FM_PB, every load of a batch before its stores
      for (int p0 = 0; p0 < n; p0 += FM_PB) {
        float yv[FM_PB][3];
#pragma unroll
        for (int j = 0; j < FM_PB; ++j) {
          const float *yp = Yq + (size_t)min(p0 + j, n - 1) * 3 * CG;
          yv[j][0] = yp[0];
          yv[j][1] = yp[CG];
          yv[j][2] = yp[2 * CG];
        }
#pragma unroll
      for (int j = 0; j < FM_PB; ++j) {
        const int p = p0 + j;
        if (p >= n) break;
        const int ql = lo + p;
        FmPairVals<double> v;
        {
          const int kn = st.kn[ql], tj = st.tj[ql];
          v.dphi = fm_pair_one<double>(st, fp, ql, cl, 0, kn, tj, 1);
          v.drho = fm_pair_one<double>(st, fp, ql, cl, 1, kn, tj, 1);
          fm_pair_val<double>(st, fp, ql, cl, 2, kn, tj, v.f, v.df);
        }
        const double G = yv[j][0], Y1 = yv[j][1], Y2 = yv[j][2];  // FP32 sums, FP64 arithmetic
        const double *e = st.e + ql * 6;
        const int64_t gs = st.gs[ql];
        const double4 ur = st.ur[ql];
        const double rr = ur.w, dx = ur.x, dy = ur.y, dz = ur.z;
        const double A = 0.5 * v.dphi + dF * (v.drho + v.df * G);
        const double B = dF * v.f;  // the staged frames carry the 1 / r
        const double Vx = dx * A + B * (e[0] * Y1 + e[3] * Y2);
        const double Vy = dy * A + B * (e[1] * Y1 + e[4] * Y2);
        const double Vz = dz * A + B * (e[2] * Y1 + e[5] * Y2);
        double *Vd = Vg + (size_t)gs * CG * 3;
        Vd[0] = Vx;
        Vd[1] = Vy;
        Vd[2] = Vz;
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
  }
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

// Adjoint epilogue, persistent CTAs over the atom blocks, candidate group
// blockIdx.y.  With the residual sensitivities frozen (lambda, eps, mu,
// kappa), L = sum_i [eps E_i + kappa pen_i] + sum_p Lambda_p . V_p and, per
// slot, Lambda_p = lambda_i - lambda_j - r_p M_cell u_p, a_p = Lambda_p . u_p:
//   k_p   = a_p (rho'_p + f'_p G_p) + f_p / r_p (Lambda.e1 Y1 + Lambda.e2 Y2)
//   K_i   = sum_p k_p,  chi_i = dL/drho_i = (eps U' + U'' K_i) [unclamped] + kappa dpen/drho
//   dL/dG_p = 1/2 f_p chi_i + a_p U' f'_p,  dL/dY1|2 = U' f_p / r_p Lambda.e1|2
// (into Yb for k_fm_gemm_adj), and the pair functions' (value, slope) weights
//   phi: (eps / 2, a_p / 2), rho: (chi, U' a_p),
//   f:   (chi G_p / 2 + U' (Lambda.e1 Y1 + Lambda.e2 Y2) / r_p, U' a_p G_p)
// (f's role as the partner k goes through the contraction).  One task per
// (atom, candidate) walks the atom's row twice: K_i and chi_i, then dL/dY and
// the pair-function weights times the slot's four B-spline basis values,
// added into the CTA's FP32 coefficient sums in shared memory; the embedding
// table gradient (value weight eps, slope weight K_i) goes into the CTA's
// FP64 table sums.  Both use shared-memory atomics (the lanes of a warp add
// to different candidates' words; the order of additions from different
// warps is not fixed, so this gradient is reproducible to FP32 rounding, not
// bit for bit).  The sums go to this CTA's FP64 partials at a change of atom
// type, every FM_PFLUSH blocks and at the end.
constexpr int FM_PFLUSH = 4;  // blocks between flushes of the pair-function sums

__host__ __device__ inline size_t fm_pre_smem(int nsplines, int CG, int nt, int NB, int ustride) {
  size_t b = (fm_stage_bytes<float>(nt, NB, CG) + 15) & ~size_t(15);
  b += sizeof(SplineGeom) * (size_t)nsplines;
  b = (b + 15) & ~size_t(15);
  b += sizeof(double) * (size_t)ustride * CG;
  b += sizeof(float) * (size_t)3 * nt * NB * CG;
  return b;
}

__global__ void __launch_bounds__(256, 2) k_fm_adj_pre(DevDb db, DevPot pot, const SplineGeom *__restrict__ geom,
                                                      const double *__restrict__ tabs, FmPlan fp, int ncand) {
  extern __shared__ __align__(16) unsigned char fm_raw[];
  const int gy = blockIdx.y, CG = fp.CG, N = db.natoms, NC = db.ncells;
  const int tid = threadIdx.x, T = blockDim.x;
  const FmStage<float> st = fm_stage_carve<float>(fm_raw, fp);
  size_t off = (fm_stage_bytes<float>(fp.nt, fp.NB, CG) + 15) & ~size_t(15);
  SplineGeom *sg = reinterpret_cast<SplineGeom *>(fm_raw + off);
  off += sizeof(SplineGeom) * (size_t)pot.nsplines;
  off = (off + 15) & ~size_t(15);
  // embedding tables of the candidates: the U splines' slices, [CG][ustride]
  double *utab = reinterpret_cast<double *>(fm_raw + off);
  float *pacc = reinterpret_cast<float *>(utab + (size_t)fp.ustride * CG);  // [3][nt][NB][CG]
  const int npe = 3 * fp.nt * fp.NB;
  const int64_t nspan8 = ((fp.Q >> 7) + FM8_SPAN - 1) >> FM8_SPAN_LOG;  // spans of the integer adjoint's exponents
  for (int sidx = tid; sidx < pot.nsplines; sidx += T) sg[sidx] = geom[sidx];
  if (tid == 0) *st.ctype = -1;
  for (int e = tid; e < npe * CG; e += T) pacc[e] = 0.f;
  for (int e = tid; e < fp.ustride * CG; e += T) utab[e] = 0.0;
  double *Pb = fp.Pbar + ((size_t)gy * gridDim.x + blockIdx.x) * pot.nsplines * FM_MAXB * CG;
  double *Tb = fp.Tbar + ((size_t)gy * gridDim.x + blockIdx.x) * CG * pot.tab_stride;
  for (int i = tid; i < pot.nsplines * FM_MAXB * CG; i += T) Pb[i] = 0.0;
  for (int i = tid; i < CG * pot.tab_stride; i += T) Tb[i] = 0.0;
  // the CTA's sums of atom type tf into its FP64 partials
  auto flush_pairs = [&](int tf) {
    __syncthreads();
    for (int idx = tid; idx < npe * CG; idx += T) {
      const int e = idx / CG, c2 = idx % CG;
      const int F = e / (fp.nt * fp.NB), o = (e / fp.NB) % fp.nt, a = e % fp.NB;
      Pb[((size_t)fm_pair_spline(pot, F, tf, o) * FM_MAXB + a) * CG + c2] += (double)pacc[idx];
      pacc[idx] = 0.f;
    }
    __syncthreads();
  };
  __syncthreads();

  int pacc_t = -1, since = 0;
  for (int blk = blockIdx.x; blk < fp.nblk; blk += gridDim.x) {
    // the block's type decides the pair splines of the sums: flush before staging
    const int ti_next = db.atom_type[db.adj_atoms[fp.blk0[blk]]];
    if (pacc_t >= 0 && (ti_next != pacc_t || since == FM_PFLUSH)) {
      flush_pairs(pacc_t);
      since = 0;
    }
    int na, ti;
    fm_stage_block<float>(db, pot, sg, fp, st, blk, gy, ncand, na, ti);
    pacc_t = ti;
    ++since;
    const SplineGeom &gU = sg[pot.s_U + ti];
    for (int task = tid; task < na * CG; task += T) {
      const int a = task / CG, cl = task % CG;
      const int c = gy * CG + cl;
      if (c >= ncand) continue;
      const double *tc = tabs + (size_t)c * pot.tab_stride;
      const int i = st.satom[a], lo = st.arow[a], n = st.arow[a + 1] - lo;
      const int cell = db.atom_cell[i];
      const int64_t q0 = fp.row0[i];
      float *Yq = fp.Y + ((size_t)gy * fp.Q + q0) * 3 * CG + cl;
      float *Ybq = fp.Yb + ((size_t)gy * fp.Q + q0) * 3 * CG + cl;
      // the atom's and its cell's candidate data
      const float *Li = fp.lamf + ((size_t)gy * N + i) * 3 * CG + cl;
      const float lix = Li[0], liy = Li[CG], liz = Li[2 * CG];
      const double *sd = fp.seedF + ((size_t)gy * NC + cell) * CS_COUNT * CG + cl;
      const float mxx = (float)sd[(CS_MU0 + 0) * CG], myy = (float)sd[(CS_MU0 + 1) * CG],
                  mzz = (float)sd[(CS_MU0 + 2) * CG], mxy = (float)sd[(CS_MU0 + 3) * CG],
                  myz = (float)sd[(CS_MU0 + 4) * CG], mzx = (float)sd[(CS_MU0 + 5) * CG];
      const double eps = sd[CS_EPS * CG], kap = sd[CS_KAPPA * CG];
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
      auto lam = [&](const float *Lj, const float4 &u, float &lx, float &ly, float &lz) {
        const float r = __frcp_rn(u.w);
        lx = lix - Lj[0] - r * (mxx * u.x + mzx * u.z);
        ly = liy - Lj[1] - r * (myy * u.y + mxy * u.x);
        lz = liz - Lj[2] - r * (mzz * u.z + myz * u.y);
      };
      // the integer adjoint's operand Z = 2^(e_q - 30) dL/dY: its exponent
      // bound per (span of FM8_SPAN 128-slot tiles, candidate),
      // |v| < 2^(field - 126), kept as the running maximum of the span
      int64_t zspan = -1;
      int zexp = -1000;
      // FP32 exponent field of v plus e_q (a value's bound before the
      // constant -126 - 30), far below every bound for v = 0
      auto zfield = [](float v, int eq) { return v != 0.f ? (int)((__float_as_uint(v) >> 23) & 255) + eq : -100000; };
      auto zbound = [&](int64_t q, int fe) {
        const int64_t sp = q >> (7 + FM8_SPAN_LOG);
        if (sp != zspan) {
          if (zspan >= 0 && zexp > -1000) atomicMax(fp.zmax + ((size_t)gy * nspan8 + zspan) * 64 + cl, zexp);
          zspan = sp;
          zexp = -1000;
        }
        zexp = max(zexp, fe - 126 - FM8_SHIFT);
      };
      auto zflush = [&]() {
        if (zspan >= 0 && zexp > -1000) atomicMax(fp.zmax + ((size_t)gy * nspan8 + zspan) * 64 + cl, zexp);
        zspan = -1;
        zexp = -1000;
      };
      const float dF = (float)U.grad;
      // ---- pass 1: K_i, dL/dY1 and dL/dY2 (they do not depend on chi_i), and
      // per slot (a_p, G_p, U' (Lambda.e1 Y1 + Lambda.e2 Y2) / r_p) for pass 2,
      // kept as FP32 in the slot's own Y words (Y is not read again)
      double K = 0.0;
      // slots in batches of FM_PB: every load of a batch is issued before its
      // stores (the stores go to the same arrays, so the compiler would
      // otherwise keep each slot's loads behind the previous slot's stores)
      for (int p0 = 0; p0 < n; p0 += FM_PB) {
        float yv[FM_PB][3];
        float lj[FM_PB][3];
#pragma unroll
        for (int j = 0; j < FM_PB; ++j) {
          const int p = min(p0 + j, n - 1);  // past the row: the last slot again, not used
          const float *yp = Yq + (size_t)p * 3 * CG;
          yv[j][0] = yp[0];
          yv[j][1] = yp[CG];
          yv[j][2] = yp[2 * CG];
          const float *Lj = fp.lamf + ((size_t)gy * N + st.nbr[lo + p]) * 3 * CG + cl;
          lj[j][0] = __ldg(Lj);
          lj[j][1] = __ldg(Lj + CG);
          lj[j][2] = __ldg(Lj + 2 * CG);
        }
#pragma unroll
        for (int j = 0; j < FM_PB; ++j) {
          const int p = p0 + j;
          if (p >= n) break;
          const int ql = lo + p;
          const FmPairVals<float> v = fm_pair_vals<float>(st, fp, ql, cl);
          float *yp = Yq + (size_t)p * 3 * CG;
          const float G = yv[j][0], Y1 = yv[j][1], Y2 = yv[j][2];
          const float4 u = st.uf[ql];
          const float *e = reinterpret_cast<const float *>(st.e) + ql * 6;
          float lx, ly, lz;
          lam(lj[j], u, lx, ly, lz);
          const float ap = lx * u.x + ly * u.y + lz * u.z;
          const float l1 = lx * e[0] + ly * e[1] + lz * e[2], l2 = lx * e[3] + ly * e[4] + lz * e[5];
          const float t12 = (l1 * Y1 + l2 * Y2) * u.w;
          // the slot's term in FP32, the atom's sum in FP64
          K += (double)(ap * (v.drho + v.df * G) + v.f * t12);
          const float B = dF * v.f * u.w, y1 = B * l1, y2 = B * l2;
          float *yb = Ybq + (size_t)p * 3 * CG;
          yb[CG] = y1;
          yb[2 * CG] = y2;
          yp[0] = ap;
          yp[CG] = G;
          yp[2 * CG] = dF * t12;
          if (fp.zmax) {
            const char4 eq = *reinterpret_cast<const char4 *>(fp.xe + (q0 + p) * 4);
            zbound(q0 + p, max(zfield(y1, eq.y), zfield(y2, eq.z)));
          }
        }
      }
      const float ch = (float)((eps * U.grad + U.grad2 * K) * drt + kap * dpen);
      spl_point_adjoint(gU, U, rt, eps, K,
                        [&](int ix, double x) { atomicAdd(utab + (size_t)cl * fp.ustride + (gU.toff - fp.utoff) + ix, x); });
      // ---- pass 2: dL/dG and the pair-function gradients
      const float epsf = (float)eps;
      for (int p0 = 0; p0 < n; p0 += FM_PBW) {
        float2 aGv[FM_PBW];
        float svv[FM_PBW];
#pragma unroll
        for (int j = 0; j < FM_PBW; ++j) {
          const float *yp = Yq + (size_t)min(p0 + j, n - 1) * 3 * CG;
          aGv[j] = make_float2(yp[0], yp[CG]);
          svv[j] = yp[2 * CG];
        }
#pragma unroll
      for (int j = 0; j < FM_PBW; ++j) {
        const int p = p0 + j;
        if (p >= n) break;
        const int ql = lo + p;
        const float ap = aGv[j].x, G = aGv[j].y, sv = svv[j];
        const int kn = st.kn[ql], tj = st.tj[ql];
        float bs[3][8];
#pragma unroll
        for (int F = 0; F < 3; ++F) fm_bas(st, ql, F, bs[F]);
        float f, df;
        {
          const int k = ((kn >> 16) & 0xff) - 1;
          const float *cf = st.coef + ((size_t)(2 * fp.nt + tj) * fp.NB + (k < 0 ? 0 : k)) * CG + cl;
          const float c0 = cf[0], c1 = cf[CG], c2 = cf[2 * CG], c3 = cf[3 * CG];
          f = bs[2][0] * c0 + bs[2][1] * c1 + bs[2][2] * c2 + bs[2][3] * c3;  // zero basis where k < 0
          df = bs[2][4] * c0 + bs[2][5] * c1 + bs[2][6] * c2 + bs[2][7] * c3;
        }
        const float y0 = 0.5f * f * ch + ap * dF * df;
        Ybq[(size_t)p * 3 * CG] = y0;
        if (fp.zmax) zbound(q0 + p, zfield(y0, (int)fp.xe[(q0 + p) * 4]));
        const float wv[3] = {0.5f * epsf, ch, 0.5f * ch * G + sv};
        const float wd[3] = {0.5f * ap, dF * ap, dF * ap * G};
#pragma unroll
        for (int F = 0; F < 3; ++F) {
          const int k = ((kn >> (8 * F)) & 0xff) - 1;
          if (k < 0) continue;
          float *pe = pacc + ((size_t)(F * fp.nt + tj) * fp.NB + k) * CG + cl;
          atomicAdd(pe, wv[F] * bs[F][0] + wd[F] * bs[F][4]);
          atomicAdd(pe + CG, wv[F] * bs[F][1] + wd[F] * bs[F][5]);
          atomicAdd(pe + 2 * CG, wv[F] * bs[F][2] + wd[F] * bs[F][6]);
          atomicAdd(pe + 3 * CG, wv[F] * bs[F][3] + wd[F] * bs[F][7]);
        }
      }
      }
      if (fp.zmax) zflush();
    }
  }
  if (pacc_t >= 0) flush_pairs(pacc_t);
  // the embedding table sums into this CTA's partial
  for (int idx = tid; idx < fp.ustride * CG; idx += T) {
    const int c2 = idx / fp.ustride, e = idx % fp.ustride;
    Tb[(size_t)c2 * pot.tab_stride + fp.utoff + e] = utab[idx];
  }
}

// ---------------------------------------------------------- k_fm_gemm_adj

// Kbar_s[d][c] += sum_{q,t} X[t][d][q] Ybar[q][t][c] over this CTA's run of
// tiles, sub-tile by sub-tile of FM_SUB slots (all Dpad features of the three
// kinds in shared memory at an 80-byte row stride, two sub-tiles in flight:
// cp.async fills one while the other is consumed).  Thread: FM_ROWS features
// (every nds-th, so that the threads of a warp read neighbouring rows) x 8
// candidates (four from each half of the group, so that the threads of a
// warp read one contiguous 128-byte run) as packed pairs of candidates; the FP32 sums of a tile are added to this CTA's FP64
// partial of the tile's atom type.  The operand of padding slots (past a
// type's last real slot) is taken as zero.
//
// With DIG8 the moments come from the integer forward's digits (X8, xe; no
// FP32 copy is kept): each sub-tile's digit rows (16 rows of every (kind,
// kblock, digit) block, 2 KB contiguous each, 48 KB in all) are copied raw
// into one staging buffer and turned into the FP32 operand, X_int 2^(e - 30)
// rounded once, before the sub-tile is consumed; the copy of the next
// sub-tile's digits overlaps the arithmetic.
constexpr int FM_XS = FM_SUB + 4;  // shared-memory row stride of the moments (80 B: no bank aliasing)
constexpr int FM8_SUBRAW = 3 * 2 * FM8_DIG * FM_SUB * 128;  // digit rows of one sub-tile: 48 KB
__host__ __device__ inline size_t fm_adj_smem(int Dpad, int CG, bool dig8 = false) {
  return 2 * sizeof(float) * ((size_t)3 * Dpad * FM_XS + (size_t)FM_SUB * 3 * CG) +
         (dig8 ? (size_t)FM8_SUBRAW + sizeof(double) * 3 * FM_SUB : 0);
}

template <bool DIG8>
__global__ void __launch_bounds__(256, 1) k_fm_gemm_adj(FmPlan fp) {
  extern __shared__ __align__(16) float asm_[];
  const int CG = fp.CG, gy = blockIdx.y;
  const size_t xsz = (size_t)3 * fp.Dpad * FM_XS, ysz = (size_t)FM_SUB * 3 * CG;
  unsigned char *raw = reinterpret_cast<unsigned char *>(asm_ + 2 * (xsz + ysz));  // DIG8: digit rows
  double *rsc = reinterpret_cast<double *>(raw + FM8_SUBRAW);                      // DIG8: [3][FM_SUB] scales
  const int tid = threadIdx.x;
  const int ncs = CG / 8, nds = fp.Dpad / FM_ROWS;
  const int cs = tid % ncs, ds = tid / ncs;
  const bool worker = ds < nds;
  const int per = (fp.ntiles + gridDim.x - 1) / gridDim.x;
  const int tb = blockIdx.x * per, te = min(fp.ntiles, tb + per);
  constexpr int NSUB = FM_TILE / FM_SUB;
  const int total = te > tb ? (te - tb) * NSUB : 0;
  double *Kb = fp.Kbar + ((size_t)gy * gridDim.x + blockIdx.x) * fp.nt * fp.Dpad * CG;
  for (int i = tid; i < fp.nt * fp.Dpad * CG; i += blockDim.x) Kb[i] = 0.0;
  auto load = [&](int k, float *bx) {
    const int64_t qb = (int64_t)(tb + k / NSUB) * FM_TILE + (k % NSUB) * FM_SUB;
    if constexpr (DIG8) {
      // the 16 digit rows of every (kind, kblock, digit) block: 2 KB each
      const int64_t T = qb / FM8_TM;
      const int r0 = (int)(qb % FM8_TM);
      for (int i = tid; i < 3 * 2 * FM8_DIG * 128; i += blockDim.x) {
        const int blk = i >> 7, ch = i & 127;  // blk = (t * 2 + kb) * FM8_DIG + l
        const size_t src = (size_t)T * 3 * 2 * FM8_STAGE + (size_t)blk * FM8_XBLK + (size_t)(r0 >> 3) * 1024 + ch * 16;
        cp_async16(raw + (size_t)blk * 2048 + ch * 16, fp.X8 + src);
      }
    } else {
      const int nrow = 3 * fp.Dpad;
      for (int i = tid; i < nrow * (FM_SUB / 4); i += blockDim.x) {
        const int row = i / (FM_SUB / 4), col = (i % (FM_SUB / 4)) * 4;
        const int t = row / fp.Dpad, d = row % fp.Dpad;
        const size_t grow = (size_t)((d / FM_DC) * 3 + t) * FM_DC + d % FM_DC;
        cp_async16(bx + (size_t)row * FM_XS + col, fp.X + grow * fp.Q + qb + col);
      }
    }
    const float *ysrc = fp.Yb + ((size_t)gy * fp.Q + qb) * 3 * CG;
    float *by = bx + xsz;
    const int64_t qe = fp.qend[fm_tile_type(fp, (int)(qb / FM_TILE))];
    for (int i = tid * 4; i < (int)ysz; i += blockDim.x * 4) {
      if (qb + i / (3 * CG) < qe) cp_async16(by + i, ysrc + i);
      else *reinterpret_cast<float4 *>(by + i) = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    cp_async_commit();
  };
  float2 acc[FM_ROWS][4];
#pragma unroll
  for (int r = 0; r < FM_ROWS; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[r][c] = make_float2(0.f, 0.f);
  // DIG8: the staged digits of sub-tile k -> its FP32 operand
  auto dequant = [&](int k, float *bx) {
    const int64_t qb = (int64_t)(tb + k / NSUB) * FM_TILE + (k % NSUB) * FM_SUB;
    for (int i = tid; i < 3 * FM_SUB; i += blockDim.x) {  // the block can be a single warp
      const int t = i / FM_SUB, j = i % FM_SUB;
      rsc[i] = ldexp(1.0, (int)fp.xe[(qb + j) * 4 + t] - FM8_SHIFT);
    }
    __syncthreads();
    const int nd4 = fp.Dpad / 4;
    for (int i = tid; i < 3 * nd4 * FM_SUB; i += blockDim.x) {
      const int j = i % FM_SUB, d4 = (i / FM_SUB) % nd4, t = i / (FM_SUB * nd4);
      const int d = 4 * d4, kb = d >> 7;
      const uint32_t o = sw128_byte(j, d & 127);
      uint32_t w[FM8_DIG];
#pragma unroll
      for (int l = 0; l < FM8_DIG; ++l)
        w[l] = *reinterpret_cast<const uint32_t *>(raw + (size_t)((t * 2 + kb) * FM8_DIG + l) * 2048 + o);
      const double sc = rsc[t * FM_SUB + j];
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        int v = 0;
#pragma unroll
        for (int l = 0; l < FM8_DIG; ++l) v = v * 256 + (int)(signed char)(w[l] >> (8 * b));
        bx[((size_t)t * fp.Dpad + d + b) * FM_XS + j] = (float)((double)v * sc);
      }
    }
  };
  if constexpr (DIG8) {
    if (total > 0) {
      load(0, asm_);
      cp_async_wait<0>();
      __syncthreads();
      dequant(0, asm_);
    }
  } else if (total > 0) {
    load(0, asm_);
  }
  for (int k = 0; k < total; ++k) {
    if constexpr (DIG8) {
      __syncthreads();  // the digits of sub-tile k are in its operand; the staging buffer is free
      if (k + 1 < total) load(k + 1, asm_ + ((k + 1) & 1) * (xsz + ysz));
    } else {
      if (k + 1 < total) {
        load(k + 1, asm_ + ((k + 1) & 1) * (xsz + ysz));
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      __syncthreads();
    }
    const float *Xs = asm_ + (k & 1) * (xsz + ysz), *Ys = Xs + xsz;
    if (worker) {
#pragma unroll
      for (int t = 0; t < 3; ++t)
#pragma unroll
        for (int qg = 0; qg < FM_SUB; qg += 4) {
          float4 xv[FM_ROWS];
#pragma unroll
          for (int r = 0; r < FM_ROWS; ++r)
            xv[r] = *reinterpret_cast<const float4 *>(Xs + ((size_t)t * fp.Dpad + r * nds + ds) * FM_XS + qg);
#pragma unroll
          for (int qq = 0; qq < 4; ++qq) {
            // candidates 4 cs .. 4 cs + 3 and CG/2 + 4 cs .. CG/2 + 4 cs + 3
            const float *yq = Ys + ((size_t)(qg + qq) * 3 + t) * CG + cs * 4;
            const float4 y0 = *reinterpret_cast<const float4 *>(yq),
                         y1 = *reinterpret_cast<const float4 *>(yq + CG / 2);
            const float2 yv[4] = {make_float2(y0.x, y0.y), make_float2(y0.z, y0.w), make_float2(y1.x, y1.y),
                                  make_float2(y1.z, y1.w)};
#pragma unroll
            for (int r = 0; r < FM_ROWS; ++r) {
              const float x = qq == 0 ? xv[r].x : qq == 1 ? xv[r].y : qq == 2 ? xv[r].z : xv[r].w;
              const float2 xx = bcast2(x);
#pragma unroll
              for (int c = 0; c < 4; ++c) acc[r][c] = fma2(xx, yv[c], acc[r][c]);
            }
          }
        }
    }
    if ((k + 1) % NSUB == 0 && worker) {  // end of a tile: into the FP64 partial of its type
      const int s = fm_tile_type(fp, tb + k / NSUB);
      double *kb = Kb + ((size_t)s * fp.Dpad + ds) * CG + cs * 4;
#pragma unroll
      for (int r = 0; r < FM_ROWS; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const int cc = (c < 2 ? 0 : CG / 2) + 2 * (c & 1);
          kb[(size_t)r * nds * CG + cc] += (double)acc[r][c].x;
          kb[(size_t)r * nds * CG + cc + 1] += (double)acc[r][c].y;
          acc[r][c] = make_float2(0.f, 0.f);
        }
    }
    if constexpr (DIG8) {
      if (k + 1 < total) {  // the next sub-tile's digits have landed: its operand
        cp_async_wait<0>();
        __syncthreads();
        dequant(k + 1, asm_ + ((k + 1) & 1) * (xsz + ysz));
      }
    }
    __syncthreads();
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
