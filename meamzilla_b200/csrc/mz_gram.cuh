// FP64 products of row sets over a long shared axis, for Powell's normal
// equations: out[i][j] = sum_k A[i][k] * B[j][k] (i < na, j < nb, k < n).
//
// Powell's linear system is lineqsys = gamma^T gamma and p = -gamma^T e
// (OptPowell::lineqsys_init, opt_powell.cpp:438-472) with one row and p
// redone after each secant update (OptPowell::lineqsys_update,
// opt_powell.cpp:476-493).  gamma is esize x ncoeff; here its columns are
// the rows of A (ncoeff rows of esize doubles, one per coefficient, which is
// how the forward-difference residual vectors come out of the evaluator), so
// every read walks a row and is coalesced.  The reference sums k in one
// sequential loop; here k is cut into S contiguous ranges (one per CTA
// column of the grid), each summed in a fixed order, and k_gram_sum adds the
// S partials in rank order: the result is bit-reproducible for a given
// (na, nb, n, S), and S depends only on the shapes and the SM count.
//
//   k_gram_tile  nb > GRAM_VEC: 64 x 64 output tiles, 256 threads with a
//                4 x 4 register tile each, k staged through shared memory in
//                slices of 32; when A and B are the same rows only the tiles
//                on or above the diagonal run (the lower ones are mirrored by
//                k_gram_sum, exactly, since a*b == b*a).
//   k_gram_vec   nb <= GRAM_VEC (the update's one or two columns): chunks of
//                1024 k with B's chunk in shared memory, one warp per A row,
//                lanes striding k, a fixed shuffle tree per row and chunk.
//   k_gram_sum   one thread per output: sum of the S partials in order.
//
// Bytes: k_gram_vec reads A once; k_gram_tile reads each 64-row block of A
// once per output tile it takes part in (ceil(nb / 64) times in all).  The
// vector form is HBM-bound, the square form FP64-FMA-bound.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace mzb {

constexpr int GRAM_T = 64;      // output tile edge of k_gram_tile
constexpr int GRAM_BK = 32;     // k slice staged per step
constexpr int GRAM_VEC = 4;     // largest nb served by k_gram_vec
constexpr int GRAM_VK = 1024;   // k chunk of k_gram_vec

struct GramArgs {
  const double *A;
  const double *B;
  int64_t lda, ldb, n;
  int na, nb;
  int sym;      // A and B are the same rows: upper tiles only
  int S;        // k ranges (grid.y of k_gram_tile, grid.x of k_gram_vec)
  int64_t kper; // k per range (multiple of GRAM_BK / GRAM_VK)
  double *partial;  // [S][na][nb]
  double *out;      // [na][nb]
};

// Tile index t of the upper triangle (row-major over tile rows) -> (bi, bj).
__device__ __forceinline__ void gram_upper_tile(int t, int T, int &bi, int &bj) {
  bi = 0;
  int rowlen = T;
  while (t >= rowlen) {
    t -= rowlen;
    ++bi;
    --rowlen;
  }
  bj = bi + t;
}

__global__ void __launch_bounds__(256) k_gram_tile(GramArgs g) {
  __shared__ double As[GRAM_BK][GRAM_T + 1];
  __shared__ double Bs[GRAM_BK][GRAM_T + 1];
  const int T = (g.nb + GRAM_T - 1) / GRAM_T;
  int bi, bj;
  if (g.sym) {
    gram_upper_tile(blockIdx.x, T, bi, bj);
  } else {
    bi = blockIdx.x / T;
    bj = blockIdx.x % T;
  }
  const int s = blockIdx.y;
  const int64_t k0 = (int64_t)s * g.kper;
  const int64_t k1 = min(g.n, k0 + g.kper);
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int i0 = bi * GRAM_T, j0 = bj * GRAM_T;
  double acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[r][c] = 0.0;
  // loader: lane = k within the slice, 8 rows per pass
  const int lk = tid & 31, lr = tid >> 5;
  for (int64_t kb = k0; kb < k1; kb += GRAM_BK) {
    const int64_t k = kb + lk;
    const bool kin = k < k1;
#pragma unroll
    for (int q = 0; q < GRAM_T / 8; ++q) {
      const int row = lr + 8 * q;
      const int ia = i0 + row, jb = j0 + row;
      As[lk][row] = (kin && ia < g.na) ? __ldg(g.A + (int64_t)ia * g.lda + k) : 0.0;
      Bs[lk][row] = (kin && jb < g.nb) ? __ldg(g.B + (int64_t)jb * g.ldb + k) : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < GRAM_BK; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) a[r] = As[kk][ty + 16 * r];
#pragma unroll
      for (int c = 0; c < 4; ++c) b[c] = Bs[kk][tx + 16 * c];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = fma(a[r], b[c], acc[r][c]);
    }
    __syncthreads();
  }
  double *P = g.partial + (size_t)s * g.na * g.nb;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int i = i0 + ty + 16 * r;
    if (i >= g.na) continue;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int j = j0 + tx + 16 * c;
      if (j < g.nb) P[(size_t)i * g.nb + j] = acc[r][c];
    }
  }
}

__global__ void __launch_bounds__(256) k_gram_vec(GramArgs g) {
  __shared__ double Bs[GRAM_VEC][GRAM_VK];
  const int s = blockIdx.x;
  const int64_t k0 = (int64_t)s * g.kper;
  const int64_t k1 = min(g.n, k0 + g.kper);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  // this CTA's sums, row i owned by warp i % nw (its lane 0 alone adds)
  double *P = g.partial + (size_t)s * g.na * g.nb;
  for (int i = warp; i < g.na; i += nw)
    if (lane < g.nb) P[(size_t)i * g.nb + lane] = 0.0;
  for (int64_t kb = k0; kb < k1; kb += GRAM_VK) {
    const int len = (int)min((int64_t)GRAM_VK, k1 - kb);
    __syncthreads();  // the previous chunk's reads of Bs are done
    for (int j = 0; j < g.nb; ++j)
      for (int t = threadIdx.x; t < GRAM_VK; t += blockDim.x)
        Bs[j][t] = t < len ? __ldg(g.B + (int64_t)j * g.ldb + kb + t) : 0.0;
    __syncthreads();
    for (int i = warp; i < g.na; i += nw) {
      const double *a = g.A + (int64_t)i * g.lda + kb;
      double acc[GRAM_VEC] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
      for (int t = lane; t < GRAM_VK; t += 32) {
        const double av = t < len ? __ldg(a + t) : 0.0;
#pragma unroll
        for (int j = 0; j < GRAM_VEC; ++j)
          if (j < g.nb) acc[j] = fma(av, Bs[j][t], acc[j]);
      }
#pragma unroll
      for (int j = 0; j < GRAM_VEC; ++j) {
        double v = acc[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0 && j < g.nb) P[(size_t)i * g.nb + j] += v;
      }
    }
  }
}

__global__ void k_gram_sum(GramArgs g) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.na * g.nb) return;
  int i = t / g.nb, j = t % g.nb;
  if (g.sym && j / GRAM_T < i / GRAM_T) {  // lower tile: its mirror was computed
    const int x = i;
    i = j;
    j = x;
  }
  const size_t o = (size_t)i * g.nb + j, stride = (size_t)g.na * g.nb;
  double v = 0.0;
  for (int s = 0; s < g.S; ++s) v += g.partial[s * stride + o];
  g.out[t] = v;
}

}  // namespace mzb
