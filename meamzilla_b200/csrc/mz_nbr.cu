// Neighbour lists on the GPU: the periodic-image pair search of
// Config::find_pairs (config.cpp:143-234; the full double-counted list, or
// each pair once for pair/spline) with the per-pair knot / shift set-up of
// check_pair (pair_meam_spline.cpp:50-99, pair_eam_spline.cpp:50-86,
// pair_pair_spline.cpp:48-72, Spline::get_knotshift spline.cpp:74-99).
//
// One thread per atom walks its cell's atoms and images in the reference's
// order (neighbour j, then ix, iy, iz), so every row holds the same pairs in
// the same order as the host builder's.  All FP64 arithmetic is written with
// explicitly rounded operations in the host's evaluation order (no fused
// multiply-add), so r, the unit vectors and the shifts are bit-identical.
// Two passes: count (and detect the reference's "pair too short" error),
// then fill at the row offsets.  The row-offset scan and the incoming lists
// run on the host.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <string>
#include <vector>

#include "mz_host.hpp"

namespace mzb {
namespace {

struct NbrParams {
  int natoms;
  int nq;            // radial functions checked per pair: phi (rho, f, p, p2)
  int nf;            // values stored per pair (Db::nfun)
  int half;          // each pair once: neighbours j >= i of the cell (config.cpp:181-185)
  int ntypes;
  double max_rcut;
  int s[5];          // first spline of phi, rho, f, p, p2
  const double *x;   // knot grids of all splines, concatenated
  const int *xoff;   // [nsplines] offset of each grid in x
  const int *xn;     // [nsplines] knots of each grid
};

__device__ __forceinline__ double dmag(double x, double y, double z) {
  return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
}

// Spline::get_knotshift (spline.cpp:74-99): bisection for the lower knot,
// -1 at or beyond x_N (1 + 1e-8).
__device__ __forceinline__ int knotshift(const double *x, int n, double r, double *shift) {
  int knot = -1;
  if (r < __dmul_rn(x[n - 1], 1. + 1.e-8)) {
    int klo = 0, khi = n - 1;
    while (khi - klo > 1) {
      const int k = (khi + klo) >> 1;
      if (x[k] > r) khi = k;
      else klo = k;
    }
    knot = klo;
    const double h = __dsub_rn(x[khi], x[klo]);
    *shift = __ddiv_rn(__dsub_rn(r, x[klo]), h);
  }
  return knot;
}

__device__ __forceinline__ int pair_ij(int ti, int tj, int nt) {
  return (ti <= tj) ? ti * nt + tj - (ti * (ti + 1)) / 2 : tj * nt + ti - (tj * (tj + 1)) / 2;
}

template <bool FILL>
__global__ void k_find_pairs(NbrParams p, const int *__restrict__ cell_atom0, const int *__restrict__ atom_cell,
                             const double *__restrict__ lat, const int *__restrict__ img,
                             const int *__restrict__ types, const double *__restrict__ pos,
                             int *__restrict__ count, const int64_t *__restrict__ off, int *__restrict__ nbr,
                             double *__restrict__ r_out, double *__restrict__ u_out, int8_t *__restrict__ knot_out,
                             double *__restrict__ shift_out, int *__restrict__ fail_atom, int *__restrict__ fail_info,
                             double *__restrict__ fail_r) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= p.natoms) return;
  const int ci = atom_cell[a];
  const int sx = img[3 * ci], sy = img[3 * ci + 1], sz = img[3 * ci + 2];
  int row = 0;
  if (sx > 0 && sy > 0 && sz > 0) {  // a too-small cell is reported by the host
    const int a_lo = cell_atom0[ci], na = cell_atom0[ci + 1] - a_lo, i = a - a_lo;
    const double *A = lat + 9 * (size_t)ci;
    const double a0x = A[0], a0y = A[1], a0z = A[2], a1x = A[3], a1y = A[4], a1z = A[5];
    const double a2x = A[6], a2y = A[7], a2z = A[8];
    const double pix = pos[3 * (size_t)a], piy = pos[3 * (size_t)a + 1], piz = pos[3 * (size_t)a + 2];
    const int ti = types[a];
    const double rc = p.max_rcut;
    const double rc2 = rc * rc * (1.0 + 1e-6);  // prefilter only; the test below is the reference's
    const int nq = p.nq;
    const int64_t o = FILL ? off[a] : 0;
    for (int j = p.half ? i : 0; j < na; ++j) {
      const double *pj = pos + 3 * (size_t)(a_lo + j);
      const double pjx = pj[0], pjy = pj[1], pjz = pj[2];
      const int tj = types[a_lo + j];
      const int pij = pair_ij(ti, tj, p.ntypes);
      const int sidx[5] = {p.s[0] + pij, p.s[1] + tj, p.s[2] + pij, p.s[3] + pij, p.s[4] + pij};
      for (int ix = -sx; ix <= sx; ++ix)
        for (int iy = -sy; iy <= sy; ++iy)
          for (int iz = -sz; iz <= sz; ++iz) {
            if (i == j && ix == 0 && iy == 0 && iz == 0) continue;
            const double fx = (double)ix, fy = (double)iy, fz = (double)iz;
            // pj + ix a0 + iy a1 + iz a2 - pi, left to right (config.cpp:204-210)
            const double dx = __dsub_rn(
                __dadd_rn(__dadd_rn(__dadd_rn(pjx, __dmul_rn(fx, a0x)), __dmul_rn(fy, a1x)), __dmul_rn(fz, a2x)), pix);
            const double dy = __dsub_rn(
                __dadd_rn(__dadd_rn(__dadd_rn(pjy, __dmul_rn(fx, a0y)), __dmul_rn(fy, a1y)), __dmul_rn(fz, a2y)), piy);
            const double dz = __dsub_rn(
                __dadd_rn(__dadd_rn(__dadd_rn(pjz, __dmul_rn(fx, a0z)), __dmul_rn(fy, a1z)), __dmul_rn(fz, a2z)), piz);
            if (dx * dx + dy * dy + dz * dz > rc2) continue;
            const double r = dmag(dx, dy, dz);
            if (r >= rc) continue;
            int kn[5] = {-1, -1, -1, -1, -1};
            double sh[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
            for (int q = 0; q < nq; ++q) {
              const double *x = p.x + p.xoff[sidx[q]];
              if (r < x[0]) {  // check_pair throws (pair_meam_spline.cpp:61-65)
                if (!FILL) {
                  atomicMin(fail_atom, a);
                  fail_info[2 * a] = j;
                  fail_info[2 * a + 1] = q;
                  fail_r[a] = r;
                  count[a] = row;
                }
                return;
              }
              kn[q] = knotshift(x, p.xn[sidx[q]], r, &sh[q]);
            }
            if (kn[0] == -1 && kn[1] == -1 && kn[2] == -1 && kn[3] == -1 && kn[4] == -1) continue;
            if (FILL) {
              const int64_t s = o + row;
              nbr[s] = a_lo + j;
              r_out[s] = r;
              u_out[3 * s] = __ddiv_rn(dx, r);
              u_out[3 * s + 1] = __ddiv_rn(dy, r);
              u_out[3 * s + 2] = __ddiv_rn(dz, r);
              for (int q = 0; q < p.nf; ++q) {
                knot_out[p.nf * s + q] = (int8_t)kn[q];
                shift_out[p.nf * s + q] = kn[q] >= 0 ? sh[q] : 0.0;
              }
            }
            ++row;
          }
    }
  }
  if (!FILL) count[a] = row;
}

void ck(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw Failure{MZ_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

// Device buffers released on every exit path.
struct DevBufs {
  std::vector<void *> p;
  template <class T>
  T *alloc(size_t n) {
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(1, n) * sizeof(T));
    if (e != cudaSuccess)
      throw Failure{MZ_ERR_NOMEM, "device allocation of " + std::to_string(n * sizeof(T)) + " bytes failed"};
    p.push_back(q);
    return static_cast<T *>(q);
  }
  template <class T>
  T *upload(const T *h, size_t n) {
    T *d = alloc<T>(n);
    if (n) ck(cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice), "list builder H2D");
    return d;
  }
  ~DevBufs() {
    for (void *q : p) cudaFree(q);
  }
};

}  // namespace

void build_db_device(const mz_cells_desc &c, const Pot &pot, Db &db, int device) {
  build_db_setup(c, pot, db);
  const bool meam = style_meam(pot.style);
  const double max_rcut = pot.max_rcut();
  const int N = c.natoms, NC = c.ncells;
  // image ranges per cell (host, as the host builder)
  std::vector<int> img(3 * (size_t)NC, 0);
  int first_small = -1;
  for (int ci = 0; ci < NC; ++ci) {
    int s[3];
    if (cell_scale(c.cell_lattice + 9 * (size_t)ci, max_rcut, &db.cell_vol[ci], s)) {
      img[3 * ci] = s[0];
      img[3 * ci + 1] = s[1];
      img[3 * ci + 2] = s[2];
    } else if (first_small < 0) {
      first_small = ci;
    }
  }
  // knot grids of every spline
  const int ns = pot.nsplines();
  std::vector<double> xs;
  std::vector<int> xoff(ns), xn(ns);
  for (int s = 0; s < ns; ++s) {
    const Spline3 &sp = pot.spline(s);
    xoff[s] = (int)xs.size();
    xn[s] = sp.nknots;
    xs.insert(xs.end(), sp.x.begin(), sp.x.end());
  }

  ck(cudaSetDevice(device), "cudaSetDevice");
  DevBufs B;
  NbrParams p{};
  p.natoms = N;
  p.half = style_pair(pot.style) ? 1 : 0;
  const int nj = style_nj(pot.style);
  p.nq = p.half ? 1 : meam ? 3 + nj : 2;
  p.nf = db.nfun;
  p.ntypes = pot.ntypes;
  p.max_rcut = max_rcut;
  p.s[0] = pot.spline_index(G_PHI, 0);
  p.s[1] = p.half ? 0 : pot.spline_index(G_RHO, 0);
  p.s[2] = meam ? pot.spline_index(G_F, 0) : 0;
  p.s[3] = nj > 0 ? pot.spline_index(G_P1, 0) : 0;
  p.s[4] = nj > 1 ? pot.spline_index(G_P2, 0) : 0;
  p.x = B.upload(xs.data(), xs.size());
  p.xoff = B.upload(xoff.data(), xoff.size());
  p.xn = B.upload(xn.data(), xn.size());
  const int *d_c0 = B.upload(db.cell_atom0.data(), db.cell_atom0.size());
  const int *d_ac = B.upload(db.atom_cell.data(), db.atom_cell.size());
  const double *d_lat = B.upload(c.cell_lattice, 9 * (size_t)NC);
  const int *d_img = B.upload(img.data(), img.size());
  const int *d_ty = B.upload(c.atom_type, (size_t)N);
  const double *d_pos = B.upload(c.atom_pos, 3 * (size_t)N);
  int *d_cnt = B.alloc<int>(N);
  int *d_fa = B.alloc<int>(1);
  int *d_fi = B.alloc<int>(2 * (size_t)N);
  double *d_fr = B.alloc<double>(N);
  const int big = INT_MAX;
  ck(cudaMemcpy(d_fa, &big, sizeof(int), cudaMemcpyHostToDevice), "list builder H2D");
  const int T = 128, G = (N + T - 1) / T;
  k_find_pairs<false><<<G, T>>>(p, d_c0, d_ac, d_lat, d_img, d_ty, d_pos, d_cnt, nullptr, nullptr, nullptr, nullptr,
                                nullptr, nullptr, d_fa, d_fi, d_fr);
  ck(cudaGetLastError(), "pair count launch");
  std::vector<int> cnt(N);
  int fa = big;
  ck(cudaMemcpy(cnt.data(), d_cnt, sizeof(int) * N, cudaMemcpyDeviceToHost), "pair count");
  ck(cudaMemcpy(&fa, d_fa, sizeof(int), cudaMemcpyDeviceToHost), "pair count");
  // the reference reports the first failing cell in order
  if (fa != big || first_small >= 0) {
    const int cs = fa != big ? db.atom_cell[fa] : INT_MAX;
    if (first_small >= 0 && first_small <= cs) throw Failure{MZ_ERR_RANGE, cell_too_small_msg(first_small)};
    int info[2];
    double rr;
    ck(cudaMemcpy(info, d_fi + 2 * (size_t)fa, sizeof(info), cudaMemcpyDeviceToHost), "failure record");
    ck(cudaMemcpy(&rr, d_fr + fa, sizeof(double), cudaMemcpyDeviceToHost), "failure record");
    const int a_lo = db.cell_atom0[cs];
    throw Failure{MZ_ERR_RANGE, pair_too_short_msg(pot, info[1], rr, c.atom_type[fa], c.atom_type[a_lo + info[0]], cs,
                                                   fa - a_lo, info[0])};
  }
  db.pair_off.assign(N + 1, 0);
  db.max_row = 0;
  db.ntriplets = 0;
  for (int a = 0; a < N; ++a) {
    db.pair_off[a + 1] = db.pair_off[a] + cnt[a];
    db.max_row = std::max(db.max_row, cnt[a]);
    if (meam) db.ntriplets += (int64_t)cnt[a] * (cnt[a] - 1) / 2;
  }
  const int64_t np = db.pair_off[N];
  db.npairs = np;
  const int64_t *d_off = B.upload(db.pair_off.data(), db.pair_off.size());
  int *d_nbr = B.alloc<int>(np);
  double *d_r = B.alloc<double>(np);
  double *d_u = B.alloc<double>(3 * (size_t)np);
  const size_t nf = (size_t)db.nfun;
  int8_t *d_kn = B.alloc<int8_t>(nf * np);
  double *d_sh = B.alloc<double>(nf * np);
  k_find_pairs<true><<<G, T>>>(p, d_c0, d_ac, d_lat, d_img, d_ty, d_pos, nullptr, d_off, d_nbr, d_r, d_u, d_kn, d_sh,
                               nullptr, nullptr, nullptr);
  ck(cudaGetLastError(), "pair fill launch");
  db.pair_nbr.resize(np);
  db.pair_r.resize(np);
  db.pair_u.resize(3 * (size_t)np);
  db.pair_knot.resize(nf * np);
  db.pair_shift.resize(nf * np);
  ck(cudaMemcpy(db.pair_nbr.data(), d_nbr, sizeof(int) * np, cudaMemcpyDeviceToHost), "pair lists D2H");
  ck(cudaMemcpy(db.pair_r.data(), d_r, sizeof(double) * np, cudaMemcpyDeviceToHost), "pair lists D2H");
  ck(cudaMemcpy(db.pair_u.data(), d_u, sizeof(double) * 3 * np, cudaMemcpyDeviceToHost), "pair lists D2H");
  ck(cudaMemcpy(db.pair_knot.data(), d_kn, nf * np, cudaMemcpyDeviceToHost), "pair lists D2H");
  ck(cudaMemcpy(db.pair_shift.data(), d_sh, sizeof(double) * nf * np, cudaMemcpyDeviceToHost), "pair lists D2H");
  build_incoming(db);
}

}  // namespace mzb
