// The forward moment contraction on the tensor cores, exactly in integers
// (tcgen05.mma.kind::i8, S32 accumulators in tensor memory).
//
//   Y[q][t][c] = sum_d X[t][d][q] K_s[d][c]            (k_fm_gemm_fwd's sum)
//
// Both operands are written as 31-bit fixed-point numbers with a power-of-two
// scale: the moments per (slot q, kind t) over the row's features,
// X = 2^(e_q - 30) X_int, and the candidates' products per (type s,
// candidate c) over the features, K = 2^(e_c - 30) K_int, with |X_int|,
// |K_int| <= 2^30 (e: the binary exponent of the row's or column's largest
// magnitude).  Each integer is four balanced base-256 digits
//   X_int = a0 2^24 + a1 2^16 + a2 2^8 + a3,  a_i in [-128, 127] (a0 in [-64, 64]),
// so X_int K_int = sum_{i,j} a_i b_j 2^(48 - 8 (i + j)).  The digit products
// of the weight classes m = i + j = 0..3 (ten pairs; the classes 4..6 weigh
// at most 2^-38 of the scale and are left out) are summed over the
// features by the MMA exactly in 32 bits (at most 4 x 256 x 128^2 < 2^31),
// and the epilogue forms, exactly in FP64 up to one final rounding,
//   Y = 2^(e_q + e_c - 60) (acc_0 2^48 + acc_1 2^40 + acc_2 2^32 + acc_3 2^24).
// The moments' digits are built once per database from their FP64 values
// (k_fm_features); so the roundings are the two 31-bit quantisations,
// relative to the row's and the column's largest entries, and there is no
// accumulation error (the FP32 contraction rounds every addition).
//
// Layouts (each block a 128-byte-swizzled K-major tile, the image the MMA
// reads from shared memory; rows of 128 bytes, 8-row groups 1 KiB apart,
// 16-byte chunk j of row r at chunk j ^ (r % 8)):
//   X8 [ntile8][3 kinds][2 kblocks][4 digits][128 slots x 128 B]   16 KB blocks
//   xe [Q][4]                               e_q of kinds 0..2 (int8)
//   K8 [ngroups][nt][2 kblocks][4 digits][64 candidates x 128 B]   8 KB blocks
//   ke [ngroups][nt][64]                    e_c (int32)
// Feature d of a row sits in kblock d / 128 at byte d % 128; features past
// the potential's D are zero.  One (tile, kind, kblock) is 64 KB contiguous:
// one bulk copy.
//
// k_fm_gemm_fwd8: persistent, one CTA per SM over a contiguous run of 128-slot
// tiles (type-pure: each type's slots are padded to 128).  Warp 0 streams the
// tiles' 16 KB digit blocks into an eight-stage ring (cp.async.bulk, completion
// on an mbarrier), warp 1 issues the MMAs (M = 128 slots, K = 32 bytes; per K
// step one MMA per digit i of the moments, N = (4 - i) x 64 over the
// candidates' stacked digit blocks, written from column 64 i so that its
// column block j lands in the class accumulator i + j; four classes of 64
// columns) and commits them to mbarriers, warps 2-9 read the accumulators of
// the previous (tile, kind) out of tensor memory (two sets of 256 columns, so
// the MMAs of the next kind overlap the epilogue) and store Y.  The
// candidates' digit blocks of the current atom type sit in shared memory and
// are reloaded where a CTA's run of tiles crosses into the next type.  Every
// wait is bounded: a wait that gives up sets the context's error flag and its
// role stops; the producer then waits for its copies in flight and the MMA
// thread for its MMAs before tensor memory is freed.
#pragma once

#include "mz_fm.cuh"
#include "mz_tc.cuh"

namespace mzb {

// ---------------------------------------------------------- k_fm_kmat8

// K8 and ke of one (type s, group gy): K_s[d][c] = c^{f(s,o)}_a w^{g(s)}_n in
// FP64 (as k_fm_kmat), the column exponent over d, the digits.  Candidates
// past ncand and features past D are zero.
__global__ void __launch_bounds__(256) k_fm_kmat8(int ncand, DevPot pot, FmPlan fp,
                                                  const double *__restrict__ coef64, signed char *__restrict__ K8,
                                                  int *__restrict__ ke) {
  __shared__ int se[FM8_NC];
  const int s = blockIdx.x, gy = blockIdx.y;
  const int nt = fp.nt;
  auto kval = [&](int d, int cl) -> double {
    const int c = gy * fp.CG + cl;
    if (cl >= fp.CG || c >= ncand || d >= fp.D) return 0.0;
    const int o = d / (fp.NA * fp.NN), a = (d / fp.NN) % fp.NA, nn = d % fp.NN;
    const int fs = pot.s_f + pair_ij_index(s, o, pot.ntypes), gs = pot.s_g + s;
    return coef64[((size_t)c * pot.nsplines + fs) * FM_MAXB + a] *
           coef64[((size_t)c * pot.nsplines + gs) * FM_MAXB + nn];
  };
  // column maxima: one warp per candidate, lanes over the features
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int cl = warp; cl < FM8_NC; cl += blockDim.x >> 5) {
    double m = 0.0;
    for (int d = lane; d < FM8_D; d += 32) m = fmax(m, fabs(kval(d, cl)));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) se[cl] = fm8_exponent(m);
  }
  __syncthreads();
  if (threadIdx.x < FM8_NC) ke[((size_t)gy * nt + s) * FM8_NC + threadIdx.x] = se[threadIdx.x];
  for (int idx = threadIdx.x; idx < FM8_NC * FM8_D; idx += blockDim.x) {
    const int cl = idx % FM8_NC, d = idx / FM8_NC;
    const long long v = llrint(ldexp(kval(d, cl), FM8_SHIFT - se[cl]));
    signed char dg[FM8_DIG];
    digits256(v, dg);
    const int kb = d >> 7;
    const uint32_t o = sw128_byte(cl, d & 127);
#pragma unroll
    for (int l = 0; l < FM8_DIG; ++l) K8[k8_block(gy, s, nt, kb, l) + o] = dg[l];
  }
}

// ---------------------------------------------------------- k_fm_gemm_fwd8

__host__ __device__ constexpr size_t fm8_smem(int nt) {
  return 1024 + (size_t)FM8_NST * FM8_XBLK + (size_t)FM8_BTYPE + sizeof(double) * FM_MAXT * FM8_NC +
         sizeof(uint64_t) * (2 * FM8_NST + 8) + 16;
}

__global__ void __launch_bounds__(FM8_THREADS, 1) k_fm_gemm_fwd8(FmPlan fp, int *__restrict__ err) {
  extern __shared__ __align__(16) unsigned char sm8raw[];
  const uint32_t raw = tc::smem_u32(sm8raw);
  unsigned char *sA = sm8raw + (((raw + 1023u) & ~1023u) - raw);  // 1 KiB aligned
  unsigned char *sB = sA + FM8_NST * FM8_XBLK;                     // K8 of the current type
  double *ssc = reinterpret_cast<double *>(sB + FM8_BTYPE);        // [nt][64] 2^(e_c - 60)
  uint64_t *full = reinterpret_cast<uint64_t *>(ssc + FM_MAXT * FM8_NC);
  uint64_t *empty = full + FM8_NST;
  uint64_t *accf = empty + FM8_NST;  // [2] accumulators of a (tile, kind) complete
  uint64_t *acce = accf + 2;         // [2] accumulators read out
  uint64_t *bload = acce + 2;        // K8 of a type landed
  uint64_t *bfree = bload + 1;       // the MMAs reading the previous type's K8 are done
  uint64_t *mdone = bfree + 1;       // every MMA of the CTA is done
  uint32_t *tslot = reinterpret_cast<uint32_t *>(mdone + 1);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gy = blockIdx.y, CG = fp.CG, nt = fp.nt;
  const int64_t ntile8 = fp.Q / FM8_TM;
  const int64_t per = (ntile8 + gridDim.x - 1) / gridDim.x;
  const int64_t tb = (int64_t)blockIdx.x * per, te = min(ntile8, tb + per);

  if (tid == 0) {
    for (int i = 0; i < FM8_NST; ++i) {
      tc::mbar_init(full + i, 1);
      tc::mbar_init(empty + i, 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(accf + b, 1);
      tc::mbar_init(acce + b, 8);
    }
    tc::mbar_init(bload, 1);
    tc::mbar_init(bfree, 1);
    tc::mbar_init(mdone, 1);
  }
  for (int i = tid; i < nt * FM8_NC; i += blockDim.x)
    ssc[i] = ldexp(1.0, fp.ke[(size_t)gy * nt * FM8_NC + i] - FM8_SHIFT);
  if (warp == 1) tc::tmem_alloc(tslot, 512);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tm = *tslot;

  if (warp == 0) {
    // ---------------- producer: K8 of each type as the tiles reach it, the tiles' digit blocks
    if (lane == 0 && tb < te) {
      int cur = fm_tile_type(fp, (int)(2 * tb)), nb = 0;
      tc::mbar_expect_tx(bload, FM8_BTYPE);
      tc::bulk_g2s(sB, fp.K8 + k8_block(gy, cur, nt, 0, 0), FM8_BTYPE, bload);
      ++nb;
      int64_t it = 0;
      bool ok = true;
      for (int64_t T = tb; T < te && ok; ++T) {
        const int s = fm_tile_type(fp, (int)(2 * T));
        if (s != cur) {  // the next type's K8, once the MMAs have left the current one
          if (!tc::mbar_wait(bfree, (uint32_t)((nb - 1) & 1), FM8_WAIT)) {
            atomicExch(err, 2);
            ok = false;
            break;
          }
          tc::mbar_expect_tx(bload, FM8_BTYPE);
          tc::bulk_g2s(sB, fp.K8 + k8_block(gy, s, nt, 0, 0), FM8_BTYPE, bload);
          ++nb;
          cur = s;
        }
        for (int t = 0; t < 3 && ok; ++t)
          for (int kb = 0; kb < 2 && ok; ++kb)
            for (int l = 0; l < FM8_DIG; ++l, ++it) {
              const int st = (int)(it % FM8_NST);
              if (it >= FM8_NST && !tc::mbar_wait(empty + st, (uint32_t)(((it / FM8_NST) & 1) ^ 1), FM8_WAIT)) {
                atomicExch(err, 2);
                ok = false;
                break;
              }
              tc::mbar_expect_tx(full + st, FM8_XBLK);
              tc::bulk_g2s(sA + st * FM8_XBLK, fp.X8 + x8_block(T, t, kb, l), FM8_XBLK, full + st);
            }
      }
      // copies in flight land before the CTA can exit
      for (int64_t j = it > FM8_NST ? it - FM8_NST : 0; j < it; ++j)
        if (!tc::mbar_wait(full + (int)(j % FM8_NST), (uint32_t)((j / FM8_NST) & 1), FM8_WAIT)) atomicExch(err, 2);
      if (!tc::mbar_wait(bload, (uint32_t)((nb - 1) & 1), FM8_WAIT)) atomicExch(err, 2);
    }
  } else if (warp == 1) {
    // ---------------- MMA issue
    if (lane == 0) {
      bool ok = true;
      int64_t it = 0, seq = 0;
      int cur = -1, nb = 0;
      const uint32_t b0 = tc::smem_u32(sB);
      for (int64_t T = tb; T < te && ok; ++T) {
        const int s = fm_tile_type(fp, (int)(2 * T));
        if (s != cur) {
          if (cur >= 0) tc::commit(bfree);  // after the last MMAs on the previous type's K8
          if (!tc::mbar_wait(bload, (uint32_t)(nb & 1), FM8_WAIT)) {
            atomicExch(err, 3);
            ok = false;
            break;
          }
          ++nb;
          cur = s;
        }
        for (int t = 0; t < 3 && ok; ++t, ++seq) {
          const int buf = (int)(seq & 1);
          if (seq >= 2 && !tc::mbar_wait(acce + buf, (uint32_t)(((seq >> 1) & 1) ^ 1), FM8_WAIT)) {
            atomicExch(err, 3);
            ok = false;
            break;
          }
          tc::fence_after_sync();
          // one stage per digit i of the moments.  The candidates' digit blocks
          // j = 0..3 lie one after another (64 rows each), so one MMA of
          // N = (4 - i) 64 takes the pairs (i, j), j <= 3 - i, at once; written
          // from column 64 i, its column block j lands in class i + j.  The
          // MMA of digit 0 starts every class's sum.
          for (int kb = 0; kb < 2 && ok; ++kb)
            for (int i = 0; i < FM8_DIG; ++i, ++it) {
              const int st = (int)(it % FM8_NST);
              if (!tc::mbar_wait(full + st, (uint32_t)((it / FM8_NST) & 1), FM8_WAIT)) {
                atomicExch(err, 3);
                ok = false;
                break;
              }
              tc::fence_after_sync();
              const uint32_t a0 = tc::smem_u32(sA + st * FM8_XBLK);
              const uint32_t idesc_i = tc::idesc_s8(FM8_TM, (FM8_DIG - i) * FM8_NC);
              const uint32_t d = tm + (uint32_t)(buf * 256 + i * FM8_NC);
#pragma unroll
              for (int kk = 0; kk < 4; ++kk) {
                const uint64_t ad = tc::desc_sw128(a0 + 32 * kk, 16, 1024);
                const uint64_t bd = tc::desc_sw128(b0 + kb * FM8_DIG * FM8_KBLK + 32 * kk, 16, 1024);
                tc::mma_s8(d, ad, bd, idesc_i, (kb == 0 && kk == 0 && i == 0) ? 0u : 1u);
              }
              tc::commit(empty + st);  // the stage is free once these MMAs are done
            }
          if (ok) tc::commit(accf + buf);
        }
      }
      tc::commit(mdone);
      if (!tc::mbar_wait(mdone, 0, FM8_WAIT)) atomicExch(err, 3);
    }
  } else {
    // ---------------- epilogue: warps 2..9, TMEM lane quarter warp % 4, candidate
    // half (warp - 2) / 4
    const int quarter = warp & 3, r = 32 * quarter + lane, ch = (warp - 2) >> 2;
    int64_t seq = 0;
    bool ok = true;
    for (int64_t T = tb; T < te && ok; ++T) {
      const int s = fm_tile_type(fp, (int)(2 * T));
      const int64_t q = T * FM8_TM + r;
      const char4 eq = *reinterpret_cast<const char4 *>(fp.xe + q * 4);  // the slot's three exponents, early
      for (int t = 0; t < 3; ++t, ++seq) {
        const int buf = (int)(seq & 1);
        if (!tc::mbar_wait(accf + buf, (uint32_t)((seq >> 1) & 1), FM8_WAIT)) {
          atomicExch(err, 4);
          ok = false;
          break;
        }
        tc::fence_after_sync();
        const int e = t == 0 ? eq.x : (t == 1 ? eq.y : eq.z);
        const double sq = __longlong_as_double((long long)(e - FM8_SHIFT + 1023) << 52);  // 2^(e - 30)
        float *yo = fp.Y + (((size_t)gy * fp.Q + q) * 3 + t) * CG;
        const uint32_t ta = tm + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(buf * 256);
        for (int cb = 2 * ch; cb < 2 * ch + 2 && cb * 16 < CG; ++cb) {
          int v[FM8_CLS][16];
#pragma unroll
          for (int m = 0; m < FM8_CLS; ++m) tc::tmem_ld16i(ta + m * FM8_NC + cb * 16, v[m]);
          tc::tmem_wait_ld();
#pragma unroll
          for (int u = 0; u < 16; u += 2) {
            double y2[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              // X_int K_int = sum_m acc_m 2^(48 - 8 m), scaled by 2^(e_q - 30) 2^(e_c - 30)
              const double a = ((double)v[0][u + h] * 281474976710656.0 + (double)v[1][u + h] * 1099511627776.0) +
                               ((double)v[2][u + h] * 4294967296.0 + (double)v[3][u + h] * 16777216.0);
              y2[h] = a * sq * ssc[s * FM8_NC + cb * 16 + u + h];
            }
            if (cb * 16 + u + 1 < CG) *reinterpret_cast<float2 *>(yo + cb * 16 + u) = make_float2((float)y2[0], (float)y2[1]);
          }
        }
        tc::fence_before_sync();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(acce + buf);
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 1) tc::tmem_dealloc(tm, 512);
}

}  // namespace mzb

namespace mzb {

// ------------------------------------------------------- integer adjoint
//
//   Kbar_s[d][c] = sum_{t,q} X[t][q][d] Ybar[q][t][c]                 (k_fm_gemm_adj's sum)
//
// With X = 2^(e_q - 30) X_int the row scale folds into the other operand,
// Z[t][q][c] = 2^(e_q - 30) Ybar[q][t][c], so Kbar = sum X_int Z.  Z is
// written as four balanced base-256 digits of a 31-bit integer with one
// power-of-two scale per (span of FM8_SPAN tiles, candidate),
// Z = 2^(e_Sc - 30) Z_int; the adjoint pre pass leaves the bound e_Sc
// (|Z| < 2^e_Sc over the span) in fp.zmax.  The digits never reach global
// memory: sixteen converter warps read Ybar (FP32) of each (tile, kind) and
// write Z's digits straight into the shared-memory stage the MMA reads, a
// K-major operand (64 candidates per digit block, the four blocks stacked
// along N; K = slots, rows of 128 slot bytes).
// The MMA reads the moments' digit blocks as they are stored for the
// forward -- 128 slot rows of 128 feature bytes -- as an MN-major operand
// (M = 128 features, K = slots: 8-row groups 1 KiB apart).  One tile's three
// kinds are 3 x 4 K steps of 32 slots per 128-feature half, with one MMA per
// digit i of the moments (N = (4 - i) x 64 over Z's stacked digit blocks, as
// in the forward), into the four class accumulators of each half (all 512
// TMEM columns).  The accumulators carry the sums of a whole segment -- the tiles
// of one span and one atom type in this CTA's run -- exactly (at most
// 4 x 384 x FM8_SPAN x 128^2 < 2^31), and at its end the same sixteen warps
// (lane quarter x feature half x candidate half) read them out and add
//   2^(e_Sc - 30) (acc_0 2^48 + acc_1 2^40 + acc_2 2^32 + acc_3 2^24)
// to the CTA's FP64 partial of the type (each (feature, candidate) word has
// one owner thread).  Padding slots (past a type's last real slot) and
// absent candidates give zero digits.

constexpr int FM8_ZBLK = FM8_NC * 128;          // one (tile, kind, digit) block of Z: 8 KB
constexpr int FM8_ZSTAGE = FM8_DIG * FM8_ZBLK;  // one (tile, kind): 32 KB
constexpr int FM8_ATHREADS = 576;               // producer, MMA, sixteen converter / epilogue warps

static_assert(4LL * 3 * FM8_TM * FM8_SPAN * 128 * 128 < (1LL << 31), "segment class sums must stay exact in S32");

// spans of the adjoint operand's exponents
__host__ __device__ inline int64_t fm8_nspan(int64_t Q) { return (Q / FM8_TM + FM8_SPAN - 1) >> FM8_SPAN_LOG; }

// The span exponent of a bound from the pre pass (|Z| < 2^zm; below -1000:
// no non-zero value), kept in [-100, ...).
__device__ __forceinline__ int fm8_span_exp(int zm) { return zm > -1000 ? max(-100, zm) : 0; }

__host__ __device__ constexpr size_t fm8_adj_smem() {
  return 1024 + (size_t)FM8_NST * FM8_XBLK + 2 * (size_t)FM8_ZSTAGE + sizeof(uint64_t) * (2 * FM8_NST + 8) + 16;
}

__global__ void __maxnreg__(96) k_fm_gemm_adj8(FmPlan fp, int ncand, int *__restrict__ err) {
  extern __shared__ __align__(16) unsigned char sm8raw[];
  const uint32_t raw = tc::smem_u32(sm8raw);
  unsigned char *sA = sm8raw + (((raw + 1023u) & ~1023u) - raw);  // [NST][16 KB] moments' digits (tile, kind, half, digit)
  unsigned char *sB = sA + FM8_NST * FM8_XBLK;                     // [2][32 KB] Z digits (tile, kind)
  uint64_t *afull = reinterpret_cast<uint64_t *>(sB + 2 * FM8_ZSTAGE);
  uint64_t *aempty = afull + FM8_NST, *bfull = aempty + FM8_NST, *bempty = bfull + 2;
  uint64_t *accf = bempty + 2, *acce = accf + 1, *mdone = acce + 1;
  uint32_t *tslot = reinterpret_cast<uint32_t *>(mdone + 1);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gy = blockIdx.y, CG = fp.CG, nt = fp.nt;
  const int64_t ntile8 = fp.Q / FM8_TM, nspan = fm8_nspan(fp.Q);
  const int64_t per = (ntile8 + gridDim.x - 1) / gridDim.x;
  const int64_t tb = (int64_t)blockIdx.x * per, te = min(ntile8, tb + per);
  double *Kb = fp.Kbar + ((size_t)gy * gridDim.x + blockIdx.x) * nt * fp.Dpad * CG;
  for (int i = tid; i < nt * fp.Dpad * CG; i += blockDim.x) Kb[i] = 0.0;
  // a segment ends at the last tile of a span, before a change of atom type
  // and at the end of the CTA's run
  auto seg_end = [&](int64_t T) {
    return T + 1 >= te || ((T + 1) & (FM8_SPAN - 1)) == 0 ||
           fm_tile_type(fp, (int)(2 * (T + 1))) != fm_tile_type(fp, (int)(2 * T));
  };

  if (tid == 0) {
    for (int i = 0; i < FM8_NST; ++i) {
      tc::mbar_init(afull + i, 1);
      tc::mbar_init(aempty + i, 1);
    }
    for (int i = 0; i < 2; ++i) {
      tc::mbar_init(bfull + i, 16);
      tc::mbar_init(bempty + i, 1);
    }
    tc::mbar_init(accf, 1);
    tc::mbar_init(acce, 16);
    tc::mbar_init(mdone, 1);
  }
  if (warp == 1) tc::tmem_alloc(tslot, 512);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tm = *tslot;

  if (warp == 0) {
    // ---------------- producer: per (tile, kind, half) the moments' four 16 KB digit blocks
    if (lane == 0) {
      int64_t ia = 0;
      bool ok = true;
      for (int64_t T = tb; T < te && ok; ++T)
        for (int t = 0; t < 3 && ok; ++t)
          for (int kb = 0; kb < 2 && ok; ++kb)
            for (int l = 0; l < FM8_DIG; ++l) {
              const int ast = (int)(ia % FM8_NST);
              if (ia >= FM8_NST && !tc::mbar_wait(aempty + ast, (uint32_t)(((ia / FM8_NST) & 1) ^ 1), FM8_WAIT)) {
                atomicExch(err, 5);
                ok = false;
                break;
              }
              tc::mbar_expect_tx(afull + ast, FM8_XBLK);
              tc::bulk_g2s(sA + ast * FM8_XBLK, fp.X8 + x8_block(T, t, kb, l), FM8_XBLK, afull + ast);
              ++ia;
            }
      // copies in flight land before the CTA can exit
      for (int64_t j = ia > FM8_NST ? ia - FM8_NST : 0; j < ia; ++j)
        if (!tc::mbar_wait(afull + (int)(j % FM8_NST), (uint32_t)((j / FM8_NST) & 1), FM8_WAIT)) atomicExch(err, 5);
    }
  } else if (warp == 1) {
    // ---------------- MMA issue: A = moments (MN-major), B = Z (K-major)
    if (lane == 0) {
      bool ok = true, fresh = true;  // fresh: the next tile starts a segment
      int64_t ia = 0, ib = 0, seg = 0;
      for (int64_t T = tb; T < te && ok; ++T) {
        if (fresh && seg >= 1 && !tc::mbar_wait(acce, (uint32_t)((seg - 1) & 1), FM8_WAIT)) {
          atomicExch(err, 6);
          ok = false;
          break;
        }
        tc::fence_after_sync();
        for (int t = 0; t < 3 && ok; ++t) {
          const int bst = (int)(ib & 1);
          if (!tc::mbar_wait(bfull + bst, (uint32_t)((ib >> 1) & 1), FM8_WAIT)) {
            atomicExch(err, 6);
            ok = false;
            break;
          }
          tc::fence_after_sync();
          const uint32_t b0 = tc::smem_u32(sB + bst * FM8_ZSTAGE);
          // one stage per digit i of the moments; Z's digit blocks j = 0..3 lie
          // one after another (64 rows each), so one MMA of N = (4 - i) 64
          // takes the pairs (i, j), j <= 3 - i, with its column block j in
          // class i + j (written from column 64 i); digit 0 starts the sums
          for (int kb = 0; kb < 2 && ok; ++kb)
            for (int i = 0; i < FM8_DIG; ++i) {
              const int ast = (int)(ia % FM8_NST);
              if (!tc::mbar_wait(afull + ast, (uint32_t)((ia / FM8_NST) & 1), FM8_WAIT)) {
                atomicExch(err, 6);
                ok = false;
                break;
              }
              tc::fence_after_sync();
              const uint32_t a0 = tc::smem_u32(sA + ast * FM8_XBLK);
              const uint32_t idesc_i = tc::idesc_s8(FM8_TM, (FM8_DIG - i) * FM8_NC, 1, 0);
              const uint32_t d = tm + (uint32_t)(kb * 256 + i * FM8_NC);
#pragma unroll
              for (int kk = 0; kk < 4; ++kk) {
                // 32 slot rows per K step: 4 groups of 8 rows, 1 KiB apart
                const uint64_t ad = tc::desc_sw128(a0 + 4096 * kk, FM8_STAGE, 1024);
                const uint64_t bd = tc::desc_sw128(b0 + 32 * kk, 16, 1024);
                tc::mma_s8(d, ad, bd, idesc_i, (fresh && t == 0 && kk == 0 && i == 0) ? 0u : 1u);
              }
              tc::commit(aempty + ast);
              ++ia;
            }
          if (!ok) break;
          tc::commit(bempty + bst);
          ++ib;
        }
        if (!ok) break;
        fresh = seg_end(T);
        if (fresh) {
          tc::commit(accf);
          ++seg;
        }
      }
      tc::commit(mdone);
      if (!tc::mbar_wait(mdone, 0, FM8_WAIT)) atomicExch(err, 6);
    }
  } else {
    // ---------------- converters / epilogue: warps 2..17
    // conversion: candidate cc, slots 16 g .. 16 g + 15 of each (tile, kind)
    const int ct = tid - 64, cc = ct & (FM8_NC - 1), g = ct >> 6;
    const bool live = cc < CG && gy * CG + cc < ncand;
    const float *Ybase = fp.Yb + (size_t)gy * fp.Q * 3 * CG + cc;
    // read-out: TMEM lane quarter warp % 4, feature half and candidate half from (warp - 2) / 4
    constexpr int NCH = FM8_NC / 2;
    const int grp = (warp - 2) >> 2, quarter = warp & 3, half = grp & 1, c0 = (grp >> 1) * NCH;
    const int d = half * FM8_TM + 32 * quarter + lane;
    int64_t ib = 0, seg = 0, pend = -1, cspan = -1;
    int e = 0;
    bool ok = true;
    auto drain = [&](int64_t Tend) {
      if (!tc::mbar_wait(accf, (uint32_t)(seg & 1), FM8_WAIT)) {
        atomicExch(err, 7);
        ok = false;
        return;
      }
      tc::fence_after_sync();
      const int s = fm_tile_type(fp, (int)(2 * Tend));
      const int *zm = fp.zmax + ((size_t)gy * nspan + (Tend >> FM8_SPAN_LOG)) * FM8_NC + c0;
      double *kbp = Kb + ((size_t)s * fp.Dpad + d) * CG + c0;
      const uint32_t ta = tm + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(half * 256 + c0);
#pragma unroll 1
      for (int cb = 0; cb < NCH / 8; ++cb) {
        int v[FM8_CLS][8];
#pragma unroll
        for (int m = 0; m < FM8_CLS; ++m) tc::tmem_ld8i(ta + m * FM8_NC + cb * 8, v[m]);
        const int4 z0 = *reinterpret_cast<const int4 *>(zm + cb * 8), z1 = *reinterpret_cast<const int4 *>(zm + cb * 8 + 4);
        tc::tmem_wait_ld();
        const int e8[8] = {z0.x, z0.y, z0.z, z0.w, z1.x, z1.y, z1.z, z1.w};
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int c = c0 + cb * 8 + u;
          if (d < fp.Dpad && c < CG) {
            const double a = ((double)v[0][u] * 281474976710656.0 + (double)v[1][u] * 1099511627776.0) +
                             ((double)v[2][u] * 4294967296.0 + (double)v[3][u] * 16777216.0);
            // 2^(e - 30), e in [-100, 100]: a normal double built from its exponent field
            kbp[cb * 8 + u] += a * __longlong_as_double((long long)(fm8_span_exp(e8[u]) - FM8_SHIFT + 1023) << 52);
          }
        }
      }
      tc::fence_before_sync();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(acce);
      ++seg;
    };
    float yn[16];  // the next (tile, kind)'s operand, loaded ahead
    if (tb < te) {
      const int64_t q0 = tb * FM8_TM + 16 * g, qend = fp.qend[fm_tile_type(fp, (int)(2 * tb))];
#pragma unroll
      for (int k = 0; k < 16; ++k) yn[k] = (live && q0 + k < qend) ? Ybase[(size_t)(q0 + k) * 3 * CG] : 0.f;
    }
    for (int64_t T = tb; T < te && ok; ++T) {
      const int64_t sp = T >> FM8_SPAN_LOG;
      if (sp != cspan) {
        cspan = sp;
        e = live ? fm8_span_exp(fp.zmax[((size_t)gy * nspan + sp) * FM8_NC + cc]) : 0;
      }
      const int s = fm_tile_type(fp, (int)(2 * T));
      const int64_t q0 = T * FM8_TM + 16 * g, qend = fp.qend[s];
      for (int t = 0; t < 3 && ok; ++t) {
        const int bst = (int)(ib & 1);
        float y[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) y[k] = yn[k];
        {  // the next item's loads in flight while this one is converted
          const int tn = t == 2 ? 0 : t + 1;
          const int64_t qn = t == 2 ? q0 + FM8_TM : q0;
          const bool more = t < 2 || T + 1 < te;
          const int64_t qendn = t == 2 && more ? fp.qend[fm_tile_type(fp, (int)(2 * (T + 1)))] : qend;
#pragma unroll
          for (int k = 0; k < 16; ++k)
            yn[k] = (more && live && qn + k < qendn) ? Ybase[((size_t)(qn + k) * 3 + tn) * CG] : 0.f;
        }
        // the 16 slots' row exponents (kinds 0..2 in bytes 0..2 of each word)
        int xw[16];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int4 x4 = *reinterpret_cast<const int4 *>(fp.xe + q0 * 4 + 16 * k);
          xw[4 * k] = x4.x;
          xw[4 * k + 1] = x4.y;
          xw[4 * k + 2] = x4.z;
          xw[4 * k + 3] = x4.w;
        }
        if (ib >= 2 && !tc::mbar_wait(bempty + bst, (uint32_t)(((ib >> 1) & 1) ^ 1), FM8_WAIT)) {
          atomicExch(err, 7);
          ok = false;
          break;
        }
        // Z_int = Ybar 2^(e_q - e): a power-of-two scaling in two exact FP32
        // steps (each factor a normal float for |e_q - e| <= 252, below which
        // every value rounds to zero; the product neither overflows,
        // |Z_int| <= 2^30, nor underflows where it rounds to a non-zero
        // integer), one rounding to int32.  Its balanced base-256 digits are
        // the bytes of (Z_int + 0x808080) ^ 0x808080 (the offset makes the
        // three lower digits + 128 the bytes, without carries; the top byte is
        // the top digit); a 4 x 4 byte transpose then gathers one digit of four
        // slots per 32-bit word of that digit's 16-byte chunk
        uint32_t w[FM8_DIG][4];
#pragma unroll
        for (int k4 = 0; k4 < 4; ++k4) {
          uint32_t v[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int k = 4 * k4 + u;
            const int sh = max(-252, (int)(signed char)((xw[k] >> (8 * t)) & 255) - e), h1 = sh >> 1;
            const float s1 = __int_as_float((h1 + 127) << 23), s2 = __int_as_float((sh - h1 + 127) << 23);
            v[u] = ((uint32_t)__float2int_rn((y[k] * s1) * s2) + 0x808080u) ^ 0x808080u;
          }
          const uint32_t ablo = __byte_perm(v[0], v[1], 0x5140), abhi = __byte_perm(v[0], v[1], 0x7362);
          const uint32_t cdlo = __byte_perm(v[2], v[3], 0x5140), cdhi = __byte_perm(v[2], v[3], 0x7362);
          w[3][k4] = __byte_perm(ablo, cdlo, 0x5410);  // least significant digit
          w[2][k4] = __byte_perm(ablo, cdlo, 0x7632);
          w[1][k4] = __byte_perm(abhi, cdhi, 0x5410);
          w[0][k4] = __byte_perm(abhi, cdhi, 0x7632);  // most significant digit
        }
        unsigned char *zb = sB + bst * FM8_ZSTAGE + sw128_byte(cc, 16 * g);
#pragma unroll
        for (int l = 0; l < FM8_DIG; ++l)
          *reinterpret_cast<uint4 *>(zb + l * FM8_ZBLK) = make_uint4(w[l][0], w[l][1], w[l][2], w[l][3]);
        tc::fence_async_smem();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(bfull + bst);
        ++ib;
        // the previous segment's read-out once the next tile's first kind is
        // staged (the MMAs wait for both)
        if (t == 0 && pend >= 0) {
          drain(pend);
          pend = -1;
        }
      }
      if (ok && seg_end(T)) pend = T;
    }
    if (ok && pend >= 0) drain(pend);
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 1) tc::tmem_dealloc(tm, 512);
}

}  // namespace mzb
