// B200 evaluator of the spline EAM/MEAM fitting objective: device context
// and the evaluator half of the C ABI (include/mz_b200.h).
//
// Launch sequence of one objective call (kernels in mz_fwd.cuh / mz_adj.cuh):
//   k_prep    one thread per (candidate, spline): coefficients -> knot table,
//             second derivatives by the reference's tridiagonal solve
//             (Spline3Eq::refresh_basis, spline3eq.cpp:192-225).
//   k_atoms   one CTA per (atom block, candidate), one thread per pair slot.
//             The block's neighbour rows are staged in shared memory and
//             triplets are enumerated implicitly as the other slots of the
//             same row (nothing per triplet is stored).  One pass over the
//             row gives the density, U, U' and the reaction vector V_p of
//             every slot (PotMEAMSpline::fast_compute,
//             pot_meam_spline.cpp:143-270; PotEAMSpline::fast_compute,
//             pot_eam_spline.cpp:135-207).
//   k_gather  one thread per atom: F_i = sum_p V_p(own row) - sum V(incoming
//             slots) -- the reference's "atom_j.force -= ..." scatter as a
//             gather, no atomics.
//   k_cells   one warp per cell: energy per atom, stress / volume, constraint
//             and the residual vector entries (Potential::accumulate_error,
//             potential.cpp:415-491).
//   k_final   one CTA per candidate: sum of squares + style punishments
//             (pot_meam_spline.cpp:274-278, pot_eam_spline.cpp:211-218).
// and for the gradient:
//   k_adj        persistent CTAs over atom blocks, one thread per slot
//   k_grad_final partial sums, punishment terms, transposed refresh.
// Forward reductions run in a fixed order (bit-reproducible objective).  The
// FP64 gradient's table sums are FP64 in a fixed order (bit-reproducible, for
// any launch variant); the mixed-precision adjoint adds its pair-function and
// embedding gradients with FP32 shared-memory atomics.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "mz_b200.h"
#include "mz_device.cuh"
#include "mz_host.hpp"
#include "mz_adj.cuh"
#include "mz_fwd2.cuh"
#include "mz_adj2.cuh"
#include "mz_tc_fwd.cuh"
#include "mz_fm.cuh"
#include "mz_fm8.cuh"
#include "mz_gram.cuh"

// ================================================================= context

using namespace mzb;

struct mz_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  DevDb db{};
  DevPot pot{};
  int P = 0, nsplines = 0, stride = 0, pstride = 0, esize = 0, npen = 0;
  int max_cand = 1, cand_cap = 1;
  int natoms = 0, ncells = 0;
  int64_t npairs = 0;
  int64_t launches = 0;
  int adj_ctas = 0;
  std::vector<void *> allocs;
  SplineGeom *d_geom = nullptr;
  double *d_base = nullptr, *d_M = nullptr;
  int *d_cmap = nullptr, *d_nat = nullptr;
  double *d_params = nullptr, *d_tabs = nullptr, *d_ptabs = nullptr, *d_V = nullptr, *d_aout = nullptr;
  double *d_forces = nullptr, *d_cellobj = nullptr, *d_obj = nullptr, *d_errvec = nullptr;
  double *d_energy = nullptr, *d_stress = nullptr;
  double *d_aux = nullptr, *d_lam = nullptr, *d_seeds = nullptr, *d_partial = nullptr, *d_grad = nullptr;
  float *d_ptabf = nullptr, *d_wtab = nullptr;  // FP32 evaluation tables, g B-spline coefficients
  int *d_err = nullptr;                         // device-side failure flag (bounded waits)
  TcParams tc{};                                // tensor-core forward plan
  bool tc_ok = false;
  bool q5 = false;  // spline5eq potential: objective only (no adjoint)
  int nsm = 1;
  // Kernel sequences of the host-buffer entry points captured as CUDA graphs,
  // one per (candidates, precision, outputs); replayed on later calls.
  bool use_graphs = true;
  struct Graph {
    cudaGraphExec_t exec;
    int64_t kernels;
  };
  std::map<uint64_t, Graph> graphs;
  size_t smem_atoms[2] = {0, 0};  // [FP64, MIXED]
  size_t smem_adj[2] = {0, 0};
  bool adj_fits[2] = {true, true};  // the adjoint's shared-memory tables fit [FP64, MIXED]
  // Launch variants the autotuner picks from, per (precision, gradient):
  // atoms per block of the forward and of the adjoint (partitions capped at
  // TUNE_CAPS[i] pair slots and a quarter as many atoms) and the adjoint's
  // persistent CTAs.  Every variant gives the same objective; the adjoint's
  // FP64 table sums follow the partition (rounding-level differences).
  static constexpr int NCAPS = 3;
  const int *d_blk[NCAPS] = {};
  int nblk[NCAPS] = {};
  const int *d_adjblk[NCAPS] = {};
  int nadjblk[NCAPS] = {};
  const int4 *d_adjdesc[NCAPS] = {};
  int adjamax[NCAPS] = {};
  int adj_ctas_max = 1, adj_per_sm = 1;
  struct Tune {
    bool done = false;
    bool fm = false;  // mixed meam/spline: the triplet-moment path
    int fwd = 0, adj = 0, ctas = 0;
    int nc = 1;      // candidates per CTA of the forward (2: k_atoms2, mixed meam/spline)
    int adj_nc = 1;  // candidates per CTA of the adjoint (2: k_adj2)
  };
  size_t smem_atoms2 = 0, smem_adj2 = 0;
  bool nc2_ok = false;  // k_atoms2 / k_adj2 apply (meam/spline, spline3eq, CUDA-core forward)
  int adj2_per_sm = 1;
  double *d_wglob = nullptr;  // the adjoint kernels' per-warp FP64 tables
  int fwd_nc = 1, adj_nc = 1;  // the variants in force
  Tune tune[2][2];  // [precision][gradient]
  int autotune = 1;  // MZ_TUNE: 1 time the variants, 0 the first variant, 2 the first with two candidates per CTA
  int adj_ctas_force = 0;  // MZ_ADJ_CTAS: persistent CTAs of the adjoint, fixed (0: the tuner's)
  bool profiling = false;
  // Mixed-precision meam/spline over triplet moments (mz_fm.cuh): eligible
  // from the potential's shape; the moments are built at the first mixed
  // launch that uses the path; MZ_FM=0 never uses it, 2 always, 1 (default)
  // lets the tuner time it against the row kernels.
  struct Fm {
    bool eligible = false, ready = false, failed = false;
    bool tc8 = false;   // the forward contraction on the tensor cores (mz_fm8.cuh)
    bool tc8a = false;  // and the adjoint contraction
    FmPlan plan{};
    int CGmax = 8, ngroups_max = 1;
    size_t smem_pre = 0;
  } fm;
  int fm_mode = 1;
  int fm8_mode = 1;  // MZ_FM8=0 keeps the forward contraction on the CUDA cores
  int fm8a_mode = 1;  // MZ_FM8ADJ=0 keeps the adjoint contraction on the CUDA cores
  int smem_optin = 0;  // largest dynamic shared memory a block may opt into
  bool fm_on = false;  // the moment path in force for mixed launches
  double *d_gram = nullptr;  // partial sums of mz_gram_device, grown on demand
  size_t gram_cap = 0;       // doubles
  struct Mark {
    int kernel;
    cudaEvent_t start, stop;
  };
  std::vector<Mark> marks;
};

namespace {

// Atom-block caps (pair slots per block) the autotuner chooses among.
constexpr int TUNE_CAPS[3] = {BLOCK_SLOTS, BLOCK_SLOTS * 3 / 4, BLOCK_SLOTS / 2};

void ck(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw Failure{MZ_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

template <class T>
T *dalloc(mz_ctx *ctx, size_t n) {
  void *p = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc(&p, n * sizeof(T));
  if (e != cudaSuccess)
    throw Failure{MZ_ERR_NOMEM, std::string("device allocation of ") + std::to_string(n * sizeof(T)) +
                                    " bytes failed: " + cudaGetErrorString(e)};
  ctx->allocs.push_back(p);
  return static_cast<T *>(p);
}

template <class T>
T *dupload(mz_ctx *ctx, const T *h, size_t n) {
  T *d = dalloc<T>(ctx, n);
  if (n) ck(cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy H2D");
  return d;
}

template <class F>
mz_status guarded(F &&f) {
  try {
    f();
    set_error("");
    return MZ_OK;
  } catch (const Failure &e) {
    set_error(e.msg);
    return e.status;
  } catch (const std::bad_alloc &) {
    set_error("host allocation failed");
    return MZ_ERR_NOMEM;
  } catch (const std::exception &e) {
    set_error(e.what());
    return MZ_ERR_ARG;
  }
}

void release(mz_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto &m : ctx->marks) {
    cudaEventDestroy(m.start);
    cudaEventDestroy(m.stop);
  }
  ctx->marks.clear();
  for (auto &g : ctx->graphs) cudaGraphExecDestroy(g.second.exec);
  ctx->graphs.clear();
  for (void *p : ctx->allocs) cudaFree(p);
  ctx->allocs.clear();
  if (ctx->d_gram) cudaFree(ctx->d_gram);
  ctx->d_gram = nullptr;
  ctx->gram_cap = 0;
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  ctx->stream = nullptr;
}

// A kernel that gave up on a bounded wait sets the context's flag.
void check_device_flag(mz_ctx *ctx) {
  int e = 0;
  ck(cudaMemcpy(&e, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost), "flag D2H");
  if (e) {
    ck(cudaMemset(ctx->d_err, 0, sizeof(int)), "flag reset");
    throw Failure{MZ_ERR_CUDA, "a tensor-core completion wait timed out on the device"};
  }
}

// The gradient needs the adjoint's shared-memory tables, sized by the
// potential (per-thread angular tables, per-warp tables of every spline).
void check_adjoint(const mz_ctx *ctx, int precision) {
  if (!ctx->adj_fits[precision == MZ_FP64 ? 0 : 1])
    throw Failure{MZ_ERR_RANGE, std::string("potential too large for the adjoint's shared-memory tables in ") +
                                    (precision == MZ_FP64 ? "FP64" : "mixed precision") +
                                    " (the objective is available)"};
}

// Brackets one kernel launch with events when the context is profiling.
struct Bracket {
  mz_ctx *ctx;
  mz_ctx::Mark m{};
  Bracket(mz_ctx *c, int kernel) : ctx(c) {
    ctx->launches += 1;
    if (!ctx->profiling) return;
    m.kernel = kernel;
    ck(cudaEventCreate(&m.start), "cudaEventCreate");
    ck(cudaEventCreate(&m.stop), "cudaEventCreate");
    ck(cudaEventRecord(m.start, ctx->stream), "cudaEventRecord");
  }
  ~Bracket() {
    if (!ctx->profiling) return;
    cudaEventRecord(m.stop, ctx->stream);
    ctx->marks.push_back(m);
  }
};

template <bool MEAM, typename R, bool AUX>
void launch_atoms(mz_ctx *ctx, int n, size_t smem) {
  dim3 ga(ctx->db.nblocks, n);
  if constexpr (MEAM && sizeof(R) == 4) {
    if (ctx->fwd_nc == 2 && ctx->nc2_ok) {  // two candidates per CTA, packed FP32 pairs
      dim3 g2(ctx->db.nblocks, (n + 1) / 2);
      k_atoms2<AUX><<<g2, BLOCK_SLOTS, ctx->smem_atoms2, ctx->stream>>>(
          ctx->db, ctx->pot, ctx->d_geom, ctx->d_tabs, ctx->d_ptabs, ctx->d_V, ctx->d_aout, ctx->d_aux, n);
      return;
    }
  }
  if (ctx->q5) {  // spline5eq pieces where a spline's basis is spline5eq
    if (MEAM && ctx->pot.nj > 0)
      k_atoms<MEAM, R, AUX, false, true, true><<<ga, BLOCK_SLOTS, smem, ctx->stream>>>(
          ctx->db, ctx->pot, ctx->d_geom, ctx->d_tabs, ctx->d_ptabs, ctx->d_V, ctx->d_aout, ctx->d_aux);
    else if (MEAM && ctx->pot.gmeam)
      k_atoms<MEAM, R, AUX, true, false, true><<<ga, BLOCK_SLOTS, smem, ctx->stream>>>(
          ctx->db, ctx->pot, ctx->d_geom, ctx->d_tabs, ctx->d_ptabs, ctx->d_V, ctx->d_aout, ctx->d_aux);
    else
      k_atoms<MEAM, R, AUX, false, false, true><<<ga, BLOCK_SLOTS, smem, ctx->stream>>>(
          ctx->db, ctx->pot, ctx->d_geom, ctx->d_tabs, ctx->d_ptabs, ctx->d_V, ctx->d_aout, ctx->d_aux);
    return;
  }
  if constexpr (MEAM) {
    if (ctx->pot.nj > 0) {
      k_atoms<MEAM, R, AUX, false, true><<<ga, BLOCK_SLOTS, smem, ctx->stream>>>(
          ctx->db, ctx->pot, ctx->d_geom, ctx->d_tabs, ctx->d_ptabs, ctx->d_V, ctx->d_aout, ctx->d_aux);
      return;
    }
  }
  if (MEAM && ctx->pot.gmeam)
    k_atoms<MEAM, R, AUX, true><<<ga, BLOCK_SLOTS, smem, ctx->stream>>>(ctx->db, ctx->pot, ctx->d_geom, ctx->d_tabs,
                                                                       ctx->d_ptabs, ctx->d_V, ctx->d_aout,
                                                                       ctx->d_aux);
  else
    k_atoms<MEAM, R, AUX><<<ga, BLOCK_SLOTS, smem, ctx->stream>>>(ctx->db, ctx->pot, ctx->d_geom, ctx->d_tabs,
                                                                   ctx->d_ptabs, ctx->d_V, ctx->d_aout, ctx->d_aux);
}

template <bool MEAM, typename R>
void launch_adj(mz_ctx *ctx, int n, size_t smem) {
  dim3 ga(ctx->adj_ctas, n);
  if (ctx->q5) {  // spline5eq pieces where a spline's basis is spline5eq
    if (MEAM && ctx->pot.nj > 0)
      k_adj<MEAM, R, false, true, true><<<ga, BLOCK_SLOTS, smem, ctx->stream>>>(
          ctx->db, ctx->pot, ctx->d_geom, ctx->d_tabs, ctx->d_ptabs, ctx->d_aout, ctx->d_aux, ctx->d_lam,
          ctx->d_seeds, ctx->d_partial, ctx->d_wglob);
    else if (MEAM && ctx->pot.gmeam)
      k_adj<MEAM, R, true, false, true><<<ga, BLOCK_SLOTS, smem, ctx->stream>>>(
          ctx->db, ctx->pot, ctx->d_geom, ctx->d_tabs, ctx->d_ptabs, ctx->d_aout, ctx->d_aux, ctx->d_lam,
          ctx->d_seeds, ctx->d_partial, ctx->d_wglob);
    else
      k_adj<MEAM, R, false, false, true><<<ga, BLOCK_SLOTS, smem, ctx->stream>>>(
          ctx->db, ctx->pot, ctx->d_geom, ctx->d_tabs, ctx->d_ptabs, ctx->d_aout, ctx->d_aux, ctx->d_lam,
          ctx->d_seeds, ctx->d_partial, ctx->d_wglob);
    return;
  }
  if constexpr (MEAM && sizeof(R) == 4) {
    if (ctx->adj_nc == 2 && ctx->nc2_ok) {  // two candidates per CTA, packed FP32 pairs
      dim3 g2(ctx->adj_ctas, (n + 1) / 2);
      k_adj2<<<g2, BLOCK_SLOTS, ctx->smem_adj2, ctx->stream>>>(ctx->db, ctx->pot, ctx->d_geom, ctx->d_tabs,
                                                               ctx->d_ptabs, ctx->d_aout, ctx->d_aux, ctx->d_lam,
                                                               ctx->d_seeds, ctx->d_wglob, ctx->d_partial, n);
      return;
    }
  }
  if constexpr (MEAM) {
    if (ctx->pot.nj > 0) {
      k_adj<MEAM, R, false, true><<<ga, BLOCK_SLOTS, smem, ctx->stream>>>(
          ctx->db, ctx->pot, ctx->d_geom, ctx->d_tabs, ctx->d_ptabs, ctx->d_aout, ctx->d_aux, ctx->d_lam,
          ctx->d_seeds, ctx->d_partial, ctx->d_wglob);
      return;
    }
  }
  if (MEAM && ctx->pot.gmeam)
    k_adj<MEAM, R, true><<<ga, BLOCK_SLOTS, smem, ctx->stream>>>(ctx->db, ctx->pot, ctx->d_geom, ctx->d_tabs,
                                                                  ctx->d_ptabs, ctx->d_aout, ctx->d_aux, ctx->d_lam,
                                                                  ctx->d_seeds, ctx->d_partial, ctx->d_wglob);
  else
    k_adj<MEAM, R><<<ga, BLOCK_SLOTS, smem, ctx->stream>>>(ctx->db, ctx->pot, ctx->d_geom, ctx->d_tabs, ctx->d_ptabs,
                                                            ctx->d_aout, ctx->d_aux, ctx->d_lam, ctx->d_seeds,
                                                            ctx->d_partial, ctx->d_wglob);
}

template <class K>
void smem_attr(K kernel, size_t bytes) {
  ck(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes), "smem attribute");
}

// ------------------------------------------------------- triplet moments

// Candidates per group of the moment path's layouts for a launch of n.
int fm_cg(int n) {
  int cg = 8;
  while (cg < n && cg < 64) cg *= 2;
  return cg;
}

template <int NW>
void fm_fwd_launch(mz_ctx *ctx, const FmPlan &fp, int G) {
  k_fm_gemm_fwd<NW><<<dim3(fp.ntiles, G), NW * 32, fm_fwd_smem<NW>(fp.Dpad), ctx->stream>>>(fp);
}

// The moments, the slots' frames and the path's buffers, at the first
// launch that uses the path.  Buffers of the row kernels are reused where
// they are large enough for the path's layouts.  False (and the path stays
// off for the context) when the device memory is not there.
bool fm_prepare(mz_ctx *ctx) {
  auto &fm = ctx->fm;
  if (fm.ready) return true;
  if (fm.failed || !fm.eligible) return false;
  FmPlan &fp = fm.plan;
  const size_t C = ctx->cand_cap;
  fm.CGmax = fm_cg((int)std::min<size_t>(C, 64));
  fm.ngroups_max = (int)((C + fm.CGmax - 1) / fm.CGmax);
  const size_t G = fm.ngroups_max, CG = fm.CGmax, Cp = G * CG;
  const size_t Q = fp.Q, N = ctx->natoms, NC = ctx->ncells, Np = ctx->npairs, ns = ctx->nsplines;
  const size_t stride = ctx->stride;
  // the pre pass's persistent grid: as many CTAs as are resident at once (a
  // second wave would run a fixed share of the blocks on a half-empty GPU);
  // launches of fewer candidates stage less and stay resident as well
  fm.smem_pre = fm_pre_smem(ctx->nsplines, 64, fp.nt, fp.NB, fp.ustride);
  smem_attr(k_fm_adj_pre, fm.smem_pre);
  {
    int occ = 0;
    ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_fm_adj_pre, 256, fm.smem_pre), "occupancy");
    fp.nctas_pre = std::max(1, std::min(fp.nblk, std::max(1, occ) * ctx->nsm));
  }
  fp.nctas_adj = std::max(1, std::min(fp.ntiles, ctx->nsm));
  const size_t aux_rows = (size_t)ctx->pot.aux_rows;
  struct Need {
    void *have;
    size_t have_bytes, need_bytes;
  };
  Need need[] = {
      {ctx->d_aux, sizeof(double) * C * aux_rows * Np, 2 * sizeof(float) * G * Q * 3 * CG},  // Y, Yb
      {ctx->d_V, sizeof(double) * C * 3 * Np, sizeof(double) * Cp * Np * 3},                   // V
      {ctx->d_aout, sizeof(double) * C * AO_COUNT * N, sizeof(double) * Cp * AO_COUNT * N},    // aoutF
      {ctx->d_lam, sizeof(double) * C * 3 * N, sizeof(float) * Cp * 3 * N},                    // lamf
      {ctx->d_seeds, sizeof(double) * C * CS_COUNT * NC, sizeof(double) * Cp * CS_COUNT * NC}, // seedF
  };
  size_t extra = sizeof(float) * 3 * (size_t)fp.Dpad * Q + sizeof(double) * 8 * Q + sizeof(float) * G * fp.nt * fp.Dpad * CG +
                 sizeof(double) * C * ns * FM_MAXB + sizeof(float) * G * ns * FM_MAXB * CG +
                 sizeof(double) * G * CG *
                     ((size_t)fp.nctas_adj * fp.nt * fp.Dpad + (size_t)fp.nctas_pre * (ns * FM_MAXB + stride));
  for (auto &x : need)
    if (x.need_bytes > x.have_bytes) extra += x.need_bytes;
  size_t freeb = 0, totalb = 0;
  ck(cudaMemGetInfo(&freeb, &totalb), "cudaMemGetInfo");
  if (extra > (size_t)(0.85 * (double)freeb)) {
    fm.failed = true;
    return false;
  }
  // the integer contraction's digits, in place of the FP32 moments, when they fit
  const size_t ntile8 = Q / FM8_TM;
  const size_t bytes8 = ntile8 * 3 * 2 * FM8_STAGE + 4 * Q + G * fp.nt * FM8_BTYPE + sizeof(int) * G * fp.nt * FM8_NC;
  const size_t bytesX = sizeof(float) * 3 * (size_t)fp.Dpad * Q;
  fm.tc8 = ctx->fm8_mode != 0 && fp.D <= FM8_D && Q % FM8_TM == 0 &&
           extra - bytesX + bytes8 <= (size_t)(0.85 * (double)freeb) &&
           fm8_smem(fp.nt) <= (size_t)ctx->smem_optin &&
           fm_adj_smem(fp.Dpad, 64, true) <= (size_t)ctx->smem_optin;
  // the kernels' own limits (registers x threads) allow their block sizes
  {
    cudaFuncAttributes fa{};
    if (fm.tc8 && (cudaFuncGetAttributes(&fa, k_fm_gemm_fwd8) != cudaSuccess || fa.maxThreadsPerBlock < FM8_THREADS))
      fm.tc8 = false;
  }
  bool adj8_ok = false;
  {
    cudaFuncAttributes fa{};
    adj8_ok = cudaFuncGetAttributes(&fa, k_fm_gemm_adj8) == cudaSuccess && fa.maxThreadsPerBlock >= FM8_ATHREADS;
  }
  // the adjoint on the tensor cores as well: its operand's exponent bounds per (span, candidate)
  const size_t bytesZ = sizeof(int) * G * (size_t)fm8_nspan((int64_t)Q) * FM8_NC;
  fm.tc8a = fm.tc8 && adj8_ok && ctx->fm8a_mode != 0 && extra - bytesX + bytes8 + bytesZ <= (size_t)(0.85 * (double)freeb) &&
            fm8_adj_smem() <= (size_t)ctx->smem_optin;
  auto pick = [&](Need &x) -> void * {
    return x.need_bytes <= x.have_bytes ? x.have : (void *)dalloc<unsigned char>(ctx, x.need_bytes);
  };
  fp.Y = static_cast<float *>(pick(need[0]));
  fp.Yb = fp.Y + G * Q * 3 * CG;
  fp.V = static_cast<double *>(pick(need[1]));
  fp.aoutF = static_cast<double *>(pick(need[2]));
  fp.lamf = static_cast<float *>(pick(need[3]));
  fp.seedF = static_cast<double *>(pick(need[4]));
  float *X = fm.tc8 ? nullptr : dalloc<float>(ctx, 3 * (size_t)fp.Dpad * Q);
  double *E = dalloc<double>(ctx, 8 * Q);
  fp.X = X;
  fp.E = E;
  fp.Kf = dalloc<float>(ctx, G * fp.nt * fp.Dpad * CG);
  double *coef64 = dalloc<double>(ctx, C * ns * FM_MAXB);
  float *coef32 = dalloc<float>(ctx, G * ns * FM_MAXB * CG);
  fp.coef64 = coef64;
  fp.coef32 = coef32;
  fp.Kbar = dalloc<double>(ctx, G * fp.nctas_adj * fp.nt * fp.Dpad * CG);
  fp.Pbar = dalloc<double>(ctx, G * fp.nctas_pre * ns * FM_MAXB * CG);
  fp.Tbar = dalloc<double>(ctx, G * fp.nctas_pre * CG * stride);
  if (X) ck(cudaMemsetAsync(X, 0, sizeof(float) * 3 * (size_t)fp.Dpad * Q, ctx->stream), "memset");
  ck(cudaMemsetAsync(E, 0, sizeof(double) * 8 * Q, ctx->stream), "memset");
  ck(cudaMemsetAsync(coef64, 0, sizeof(double) * C * ns * FM_MAXB, ctx->stream), "memset");
  ck(cudaMemsetAsync(coef32, 0, sizeof(float) * G * ns * FM_MAXB * CG, ctx->stream), "memset");
  signed char *X8 = nullptr, *xe = nullptr;
  if (fm.tc8) {
    X8 = dalloc<signed char>(ctx, ntile8 * 3 * 2 * FM8_STAGE);
    xe = dalloc<signed char>(ctx, 4 * Q);
    fp.K8 = dalloc<signed char>(ctx, G * fp.nt * FM8_BTYPE);
    fp.ke = dalloc<int>(ctx, G * fp.nt * FM8_NC);
    ck(cudaMemsetAsync(X8, 0, ntile8 * 3 * 2 * FM8_STAGE, ctx->stream), "memset");
    ck(cudaMemsetAsync(xe, 0, 4 * Q, ctx->stream), "memset");
    fp.X8 = X8;
    fp.xe = xe;
    smem_attr(k_fm_gemm_fwd8, fm8_smem(fp.nt));
    if (fm.tc8a) {
      fp.zmax = dalloc<int>(ctx, G * (size_t)fm8_nspan((int64_t)Q) * FM8_NC);
      smem_attr(k_fm_gemm_adj8, fm8_adj_smem());
    }
  }
  fp.CG = fm.CGmax;
  k_fm_features<<<ctx->natoms, 256, 0, ctx->stream>>>(ctx->db, ctx->pot, ctx->d_geom, fp, X, E, X8, xe);
  ck(cudaGetLastError(), "k_fm_features launch");
  ck(cudaStreamSynchronize(ctx->stream), "moments");
  smem_attr(k_fm_gemm_fwd<1>, fm_fwd_smem<1>(fp.Dpad));
  smem_attr(k_fm_gemm_fwd<2>, fm_fwd_smem<2>(fp.Dpad));
  smem_attr(k_fm_gemm_fwd<4>, fm_fwd_smem<4>(fp.Dpad));
  smem_attr(k_fm_gemm_fwd<8>, fm_fwd_smem<8>(fp.Dpad));
  smem_attr(k_fm_epi, fm_epi_smem(ctx->nsplines, fp.nt, fp.NB, 64));
  smem_attr(k_fm_gemm_adj<false>, fm_adj_smem(fp.Dpad, 64));
  if (fm.tc8) smem_attr(k_fm_gemm_adj<true>, fm_adj_smem(fp.Dpad, 64, true));
  fm.ready = true;
  return true;
}

// The moment path's launch sequence (after k_prep): objective, and with
// d_grad the gradient.
void enqueue_fm(mz_ctx *ctx, int n, double *d_obj, double *d_errvec, double *d_forces, double *d_energy,
                double *d_stress, double *d_grad) {
  cudaStream_t st = ctx->stream;
  FmPlan fp = ctx->fm.plan;
  fp.CG = fm_cg(std::min(n, 64));
  const int G = (n + fp.CG - 1) / fp.CG, CG = fp.CG;
  const int ns = ctx->nsplines, N = ctx->natoms, NC = ctx->ncells;
  const bool grad = d_grad != nullptr;
  {
    Bracket b(ctx, MZ_K_FM_COEF);
    k_fm_coef<<<n, std::max(32, ((ns + 31) / 32) * 32), 0, st>>>(n, ctx->d_geom, ns, ctx->stride, ctx->d_tabs, fp,
                                                                  const_cast<double *>(fp.coef64),
                                                                  const_cast<float *>(fp.coef32));
    ck(cudaGetLastError(), "k_fm_coef launch");
  }
  if (ctx->fm.tc8) {  // the forward contraction in integers on the tensor cores
    {
      Bracket b(ctx, MZ_K_FM_COEF);
      k_fm_kmat8<<<dim3(fp.nt, G), 256, 0, st>>>(n, ctx->pot, fp, fp.coef64, fp.K8, fp.ke);
      ck(cudaGetLastError(), "k_fm_kmat8 launch");
    }
    Bracket b(ctx, MZ_K_FM_FWD);
    const int ntile8 = (int)(fp.Q / FM8_TM);
    k_fm_gemm_fwd8<<<dim3(std::min(ntile8, ctx->nsm), G), FM8_THREADS, fm8_smem(fp.nt), st>>>(fp, ctx->d_err);
    ck(cudaGetLastError(), "k_fm_gemm_fwd8 launch");
  } else {
    {
      Bracket b(ctx, MZ_K_FM_COEF);
      const int zs = std::max(1, std::min(64, fp.Dpad * CG / 2048));
      k_fm_kmat<<<dim3(fp.nt, G, zs), 256, 0, st>>>(n, ctx->pot, fp, fp.coef64, const_cast<float *>(fp.Kf));
      ck(cudaGetLastError(), "k_fm_kmat launch");
    }
    Bracket b(ctx, MZ_K_FM_FWD);
    switch (CG / 8) {
      case 1: fm_fwd_launch<1>(ctx, fp, G); break;
      case 2: fm_fwd_launch<2>(ctx, fp, G); break;
      case 4: fm_fwd_launch<4>(ctx, fp, G); break;
      default: fm_fwd_launch<8>(ctx, fp, G); break;
    }
    ck(cudaGetLastError(), "k_fm_gemm_fwd launch");
  }
  const unsigned ablocks = (unsigned)(((int64_t)N * CG + 255) / 256);
  {
    Bracket b(ctx, MZ_K_FM_EPI);
    // persistent CTAs, as many as are resident at once
    const size_t esm = fm_epi_smem(ns, fp.nt, fp.NB, CG);
    int occ = 0;
    ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_fm_epi, 256, esm), "occupancy");
    const int eb = std::max(1, std::min(fp.nblk, std::max(1, occ) * ctx->nsm));
    k_fm_epi<<<dim3(eb, G), 256, esm, st>>>(ctx->db, ctx->pot, ctx->d_geom,
                                                                         ctx->d_tabs, fp, n);
    ck(cudaGetLastError(), "k_fm_epi launch");
  }
  {
    Bracket b(ctx, MZ_K_GATHER);
    k_fm_gather<<<dim3(ablocks, G), 256, 0, st>>>(ctx->db, fp, n, d_forces, d_errvec, ctx->esize, grad ? 1 : 0);
    ck(cudaGetLastError(), "k_fm_gather launch");
  }
  {
    Bracket b(ctx, MZ_K_CELLS);
    const unsigned cblocks = (unsigned)(((int64_t)NC * CG + 255) / 256);
    k_fm_cells<<<dim3(cblocks, G), 256, 0, st>>>(ctx->db, ctx->pot, fp, n, ctx->d_cellobj, d_errvec, ctx->esize,
                                                 d_energy, d_stress, grad ? 1 : 0);
    ck(cudaGetLastError(), "k_fm_cells launch");
  }
  {
    Bracket b(ctx, MZ_K_FINAL);
    k_final<<<n, 256, 0, st>>>(ctx->db, ctx->pot, ctx->d_geom, ctx->d_tabs, ctx->d_cellobj, d_obj, d_errvec,
                               ctx->esize);
    ck(cudaGetLastError(), "k_final launch");
  }
  if (!grad) return;
  if (fp.zmax)  // the pre pass's per-span exponent bounds start below every bound
    ck(cudaMemsetAsync(fp.zmax, 0x80, sizeof(int) * (size_t)G * fm8_nspan(fp.Q) * FM8_NC, st), "memset");
  {
    Bracket b(ctx, MZ_K_FM_PRE);
    k_fm_adj_pre<<<dim3(fp.nctas_pre, G), 256, fm_pre_smem(ns, CG, fp.nt, fp.NB, fp.ustride), st>>>(
        ctx->db, ctx->pot, ctx->d_geom, ctx->d_tabs, fp, n);
    ck(cudaGetLastError(), "k_fm_adj_pre launch");
  }
  {
    Bracket b(ctx, MZ_K_FM_ADJ);
    const int threads = ((fp.Dpad / FM_ROWS) * (CG / 8) + 31) / 32 * 32;
    if (ctx->fm.tc8a) {
      k_fm_gemm_adj8<<<dim3(fp.nctas_adj, G), FM8_ATHREADS, fm8_adj_smem(), st>>>(fp, n, ctx->d_err);
    } else if (ctx->fm.tc8)
      k_fm_gemm_adj<true><<<dim3(fp.nctas_adj, G), std::min(threads, 256), fm_adj_smem(fp.Dpad, CG, true), st>>>(fp);
    else
      k_fm_gemm_adj<false><<<dim3(fp.nctas_adj, G), std::min(threads, 256), fm_adj_smem(fp.Dpad, CG), st>>>(fp);
    ck(cudaGetLastError(), "k_fm_gemm_adj launch");
  }
  {
    Bracket b(ctx, MZ_K_FM_GRAD);
    const size_t sm = sizeof(double) * ((size_t)ns * FM_MAXB + ctx->stride + (size_t)fp.nt * fp.Dpad);
    k_fm_grad<<<n, 256, sm, st>>>(ctx->pot, ctx->d_geom, fp, fp.coef64, ctx->d_partial);
    ck(cudaGetLastError(), "k_fm_grad launch");
  }
  {
    Bracket b(ctx, MZ_K_GRAD_FINAL);
    k_grad_final<<<n, 256, sizeof(double) * ctx->stride, st>>>(ctx->pot, ctx->d_geom, ctx->d_tabs, ctx->d_partial,
                                                                1, ctx->d_M, ctx->d_cmap, ctx->P, d_grad);
    ck(cudaGetLastError(), "k_grad_final launch");
  }
}

// Enqueue the objective (and, with d_grad, its gradient) of n candidates
// whose coefficient vectors are already on the device.
void enqueue(mz_ctx *ctx, int n, const double *d_params, int precision, double *d_obj, double *d_errvec,
             double *d_forces, double *d_energy, double *d_stress, double *d_grad) {
  cudaStream_t st = ctx->stream;
  const bool meam = style_meam(ctx->pot.style);
  const bool mixed = precision == MZ_MIXED;
  const bool grad = d_grad != nullptr;
  {
    Bracket b(ctx, MZ_K_PREP);
    k_prep<<<n, std::max(32, ((ctx->nsplines + 31) / 32) * 32), 0, st>>>(
        n, ctx->P, d_params, ctx->d_base, ctx->d_cmap, ctx->d_geom, ctx->d_nat, ctx->nsplines, ctx->stride,
        ctx->d_tabs, ctx->pstride, ctx->d_ptabs, ctx->d_ptabf, ctx->tc_ok ? ctx->d_wtab : nullptr, ctx->pot.s_g,
        ctx->pot.ntypes, TC_NB, ctx->d_M);
    ck(cudaGetLastError(), "k_prep launch");
  }
  if (mixed && meam && ctx->fm_on && ctx->fm.ready) {
    enqueue_fm(ctx, n, d_obj, d_errvec, d_forces, d_energy, d_stress, d_grad);
    return;
  }
  {
    Bracket b(ctx, MZ_K_ATOMS);
    const size_t sa = ctx->smem_atoms[mixed ? 1 : 0];
    if (meam && mixed && ctx->tc_ok) {
      dim3 gt(std::min(ctx->nsm, ctx->natoms), (n + TC_CANDS - 1) / TC_CANDS);
      const size_t st_bytes = (size_t)ctx->tc.smem_bytes;
      if (grad)
        k_atoms_tc<TC_NB, true><<<gt, TC_THREADS, st_bytes, st>>>(ctx->db, ctx->pot, ctx->tc, ctx->d_geom, ctx->d_tabs,
                                                                 ctx->d_ptabf, ctx->d_wtab, n, ctx->d_V,
                                                                 ctx->d_aout, ctx->d_aux, ctx->d_err);
      else
        k_atoms_tc<TC_NB, false><<<gt, TC_THREADS, st_bytes, st>>>(ctx->db, ctx->pot, ctx->tc, ctx->d_geom,
                                                                  ctx->d_tabs, ctx->d_ptabf, ctx->d_wtab, n,
                                                                  ctx->d_V, ctx->d_aout, ctx->d_aux, ctx->d_err);
    } else if (meam) {
      if (mixed) grad ? launch_atoms<true, float, true>(ctx, n, sa) : launch_atoms<true, float, false>(ctx, n, sa);
      else grad ? launch_atoms<true, double, true>(ctx, n, sa) : launch_atoms<true, double, false>(ctx, n, sa);
    } else {
      if (mixed) launch_atoms<false, float, false>(ctx, n, sa);
      else launch_atoms<false, double, false>(ctx, n, sa);
    }
    ck(cudaGetLastError(), "k_atoms launch");
  }
  {
    Bracket b(ctx, MZ_K_GATHER);
    dim3 gg((ctx->natoms + 255) / 256, n);
    k_gather<<<gg, 256, 0, st>>>(ctx->db, ctx->d_V, ctx->d_aout, d_forces, d_errvec, ctx->esize,
                                 grad ? ctx->d_lam : nullptr);
    ck(cudaGetLastError(), "k_gather launch");
  }
  {
    Bracket b(ctx, MZ_K_CELLS);
    dim3 gc((ctx->ncells + 7) / 8, n);
    k_cells<<<gc, 256, 0, st>>>(ctx->db, ctx->pot, ctx->d_aout, ctx->d_cellobj, d_errvec, ctx->esize, d_energy,
                                d_stress, grad ? ctx->d_seeds : nullptr);
    ck(cudaGetLastError(), "k_cells launch");
  }
  {
    Bracket b(ctx, MZ_K_FINAL);
    k_final<<<n, 256, 0, st>>>(ctx->db, ctx->pot, ctx->d_geom, ctx->d_tabs, ctx->d_cellobj, d_obj, d_errvec,
                               ctx->esize);
    ck(cudaGetLastError(), "k_final launch");
  }
  if (!grad) return;
  {
    Bracket b(ctx, MZ_K_ADJ);
    const size_t sj = ctx->smem_adj[mixed ? 1 : 0];
    if (meam) mixed ? launch_adj<true, float>(ctx, n, sj) : launch_adj<true, double>(ctx, n, sj);
    else mixed ? launch_adj<false, float>(ctx, n, sj) : launch_adj<false, double>(ctx, n, sj);
    ck(cudaGetLastError(), "k_adj launch");
  }
  {
    Bracket b(ctx, MZ_K_GRAD_FINAL);
    // FP64: one partial per group of adj_group blocks; mixed: one per CTA
    const int nparts = mixed ? ctx->adj_ctas
                             : (ctx->db.adj_nblocks + ctx->db.adj_group - 1) / std::max(ctx->db.adj_group, 1);
    k_grad_final<<<n, 256, sizeof(double) * ctx->stride, st>>>(ctx->pot, ctx->d_geom, ctx->d_tabs, ctx->d_partial,
                                                                nparts, ctx->d_M, ctx->d_cmap, ctx->P, d_grad);
    ck(cudaGetLastError(), "k_grad_final launch");
  }
}

// Independent FMA streams: 8 accumulators per thread, no memory traffic.
template <typename T>
__global__ void k_fma_peak(T *out, int iters, T a, T b) {
  T x[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) x[q] = (T)(threadIdx.x + q);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int q = 0; q < 8; ++q) x[q] = fma(x[q], a, b);
  }
  T s = 0;
#pragma unroll
  for (int q = 0; q < 8; ++q) s += x[q];
  if (s == (T)-1.2345) out[0] = s;  // keeps the chain alive
}


// d(ypp)/d(y, slope_left, slope_right) of one spline: the refresh is linear,
// so its columns are the refresh of unit inputs.
void refresh_matrix(const Spline3 &sp, std::vector<double> &M) {
  const int n = sp.nknots;
  M.assign((size_t)n * (n + 2), 0.0);
  Spline3 s = sp;
  std::vector<double> ypp;
  for (int col = 0; col < n + 2; ++col) {
    std::fill(s.y.begin(), s.y.end(), 0.0);
    s.grad[0] = s.grad[1] = 0.0;
    if (col < n) s.y[col] = 1.0;
    else s.grad[col - n] = 1.0;
    s.refresh(ypp);
    for (int r = 0; r < n; ++r) M[(size_t)r * (n + 2) + col] = ypp[r];
  }
}

// d(ypp, yp4)/d(y, slope_left, slope_right, y''_left, y''_right) of one
// spline5eq spline, [2n][n+4]: Spline5Eq::refresh_basis is linear in them.
void refresh_matrix5(const Spline3 &sp, std::vector<double> &M) {
  const int n = sp.nknots, nc = n + 4;
  M.assign((size_t)2 * n * nc, 0.0);
  Spline3 s = sp;
  std::vector<double> ypp, yp4;
  for (int col = 0; col < nc; ++col) {
    std::fill(s.y.begin(), s.y.end(), 0.0);
    s.grad[0] = s.grad[1] = s.grad2[0] = s.grad2[1] = 0.0;
    if (col < n) s.y[col] = 1.0;
    else if (col < n + 2) s.grad[col - n] = 1.0;
    else s.grad2[col - n - 2] = 1.0;
    s.refresh5(ypp, yp4);
    for (int r = 0; r < n; ++r) {
      M[(size_t)r * nc + col] = ypp[r];
      M[(size_t)(n + r) * nc + col] = yp4[r];
    }
  }
}

// Host image of a potential's structure for the device: per-spline geometry
// (offsets of its knot table, evaluation table and refresh matrix), natural
// ends, the fixed table values and the coefficient map (table entry ->
// coefficient index in Potential::coeff's order, -1 where fixed).
struct PotImage {
  std::vector<SplineGeom> geom;
  std::vector<int> nat;
  std::vector<double> base, M;
  std::vector<int> cmap;
  int stride = 0, pstride = 0, P = 0;
};

PotImage pot_image(const Pot &pot) {
  PotImage im;
  const int ns = pot.nsplines();
  im.geom.resize(ns);
  im.nat.resize(2 * ns);
  int toff = 0, poff = 0;
  for (int s = 0; s < ns; ++s) {
    const Spline3 &sp = pot.spline(s);
    SplineGeom &g = im.geom[s];
    g.x0 = sp.x[0];
    g.xN = sp.x[sp.nknots - 1];
    g.step = sp.step;
    g.invstep = sp.invstep;
    g.cut = sp.x.back() * (1. + 1.e-8);
    float cf = (float)g.cut;
    for (int u = 0; u < 4; ++u) cf = std::nextafter(cf, INFINITY);
    g.cutf = cf;
    g.n = sp.nknots;
    g.q5 = sp.quintic;
    g.toff = toff;
    toff += (sp.quintic ? 3 : 2) * sp.nknots + (sp.quintic ? 4 : 2);
    // every spline's pieces start on 4 entries (16 bytes in FP32): cubic
    // pieces are loaded as float4 / double2 pairs, quintic ones as pairs, and
    // a mixed-basis potential puts cubic splines after quintic ones
    poff = (poff + 3) & ~3;
    g.poff = poff;
    poff += (sp.quintic ? 6 : 4) * (sp.nknots - 1);
    im.nat[2 * s] = sp.nat[0];
    im.nat[2 * s + 1] = sp.nat[1];
    std::vector<double> M;
    if (sp.quintic) refresh_matrix5(sp, M);
    else refresh_matrix(sp, M);
    g.moff = (int)im.M.size();
    im.M.insert(im.M.end(), M.begin(), M.end());
  }
  im.stride = toff;
  im.pstride = (poff + 3) & ~3;  // candidates' tables start on 16 bytes too
  im.base.assign(toff, 0.0);
  im.cmap.assign(toff, -1);
  for (int s = 0; s < ns; ++s) {
    const Spline3 &sp = pot.spline(s);
    const int o = im.geom[s].toff, n = sp.nknots;
    for (int k = 0; k < n; ++k) im.base[o + k] = sp.y[k];
    for (int e = 0; e < 2; ++e) im.base[o + 2 * n + e] = sp.grad[e];
    if (sp.quintic)
      for (int e = 0; e < 2; ++e) im.base[o + 3 * n + 2 + e] = sp.grad2[e];
  }
  int ci = 0;
  for (auto &cs : pot.coeff_slots()) {
    const int o = im.geom[cs.first].toff, n = im.geom[cs.first].n, slot = cs.second;
    const int at = slot < n ? o + slot : slot < n + 2 ? o + 2 * n + (slot - n) : o + 3 * n + 2 + (slot - n - 2);
    im.cmap[at] = ci++;
  }
  im.P = ci;
  return im;
}

// Knots of slot s packed as the kernels read them:
// (phi+1) | (rho+1) << 8 | (f+1) << 16 | (p+1) << 24.
int packed_knots(const Db &db, int64_t s) {
  const int nf = db.nfun;
  return (db.pair_knot[nf * s] + 1) | ((db.pair_knot[nf * s + 1] + 1) << 8) | ((db.pair_knot[nf * s + 2] + 1) << 16) |
         (nf > 3 ? (db.pair_knot[nf * s + 3] + 1) << 24 : 0);
}

// ---------------------------------------------------------------- autotuner

// Choices by workload, shared by the contexts of one process, so that
// evaluators of the same database and potential structure launch the same
// variants (and give bit-identical gradients).
std::mutex g_tune_mu;
std::map<std::vector<int64_t>, mz_ctx::Tune> g_tune_cache;

void apply_variant(mz_ctx *ctx, const mz_ctx::Tune &t) {
  ctx->fm_on = t.fm;
  ctx->fwd_nc = t.nc;
  ctx->adj_nc = t.adj_nc;
  ctx->db.nblocks = ctx->nblk[t.fwd];
  ctx->db.blk_atom0 = ctx->d_blk[t.fwd];
  ctx->db.adj_nblocks = ctx->nadjblk[t.adj];
  ctx->db.adj_blk0 = ctx->d_adjblk[t.adj];
  ctx->db.adj_desc = ctx->d_adjdesc[t.adj];
  ctx->db.adj_amax = ctx->adjamax[t.adj];
  ctx->adj_ctas = ctx->adj_ctas_force > 0 ? std::min(ctx->adj_ctas_force, ctx->adj_ctas_max) : t.ctas;
}

int adj_ctas_for(const mz_ctx *ctx, int v, int per_sm) {
  return std::max(1, std::min(ctx->nadjblk[v], ctx->nsm * per_sm));
}

// One objective (+ gradient) with events around every kernel: the device
// time of `kernel` in ms (of all of them for kernel < 0).  The caller's
// profiling marks are kept aside.
double trial(mz_ctx *ctx, int n, const double *d_params, int precision, bool grad, int kernel) {
  std::vector<mz_ctx::Mark> keep;
  keep.swap(ctx->marks);
  const bool prof = ctx->profiling;
  ctx->profiling = true;
  auto restore = [&] {
    for (auto &m : ctx->marks) {
      cudaEventDestroy(m.start);
      cudaEventDestroy(m.stop);
    }
    ctx->marks.swap(keep);
    ctx->profiling = prof;
  };
  double ms = 0.0;
  try {
    enqueue(ctx, n, d_params, precision, ctx->d_obj, nullptr, nullptr, nullptr, nullptr,
            grad ? ctx->d_grad : nullptr);
    ck(cudaStreamSynchronize(ctx->stream), "autotune trial");
    for (auto &m : ctx->marks) {
      float t = 0.f;
      ck(cudaEventElapsedTime(&t, m.start, m.stop), "cudaEventElapsedTime");
      if (m.kernel == kernel || kernel < 0) ms += t;
    }
  } catch (...) {
    restore();
    throw;
  }
  restore();
  return ms;
}

// Picks, once per (precision, gradient), the forward's atoms per block, then
// the adjoint's atoms per block and persistent CTAs, by timing each on the
// caller's own candidates; MZ_TUNE=0 keeps the first variant of each.
void tune_variant(mz_ctx *ctx, int n, const double *d_params, int precision, bool grad) {
  mz_ctx::Tune &t = ctx->tune[precision][grad ? 1 : 0];
  if (!t.done) {
    const std::vector<int64_t> key = {ctx->device,     ctx->natoms,    ctx->npairs, ctx->ncells, ctx->pot.style,
                                      ctx->pot.ntypes, ctx->P,         precision,   grad,        ctx->q5,
                                      ctx->autotune,   ctx->nblk[0],   ctx->nadjblk[0], ctx->fm_mode};
    bool cached = false;
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      auto it = g_tune_cache.find(key);
      if (it != g_tune_cache.end()) {
        t = it->second;
        cached = true;
      }
    }
    if (cached && t.fm && !fm_prepare(ctx)) t.fm = false;
    if (!cached) {
      mz_ctx::Tune best;
      best.ctas = adj_ctas_for(ctx, 0, ctx->adj_per_sm);
      if (ctx->autotune == 2 && precision == MZ_MIXED && ctx->nc2_ok) {
        best.nc = 2;
        best.adj_nc = 2;
        best.ctas = adj_ctas_for(ctx, 0, ctx->adj2_per_sm);
      }
      if (ctx->autotune == 1) {
        const int64_t l0 = ctx->launches;
        apply_variant(ctx, best);
        trial(ctx, n, d_params, precision, grad, MZ_K_ATOMS);  // warm-up
        double bt = 1e300;
        const int ncs = (precision == MZ_MIXED && ctx->nc2_ok && n > 1) ? 2 : 1;
        for (int nc = 1; nc <= ncs; ++nc)
          for (int v = 0; v < mz_ctx::NCAPS; ++v) {
            mz_ctx::Tune c = best;
            c.fwd = v;
            c.nc = nc;
            apply_variant(ctx, c);
            const double x = trial(ctx, n, d_params, precision, grad, MZ_K_ATOMS);
            if (x < bt) {
              bt = x;
              best.fwd = v;
              best.nc = nc;
            }
          }
        if (grad) {
          double ba = 1e300;
          const int ancs = (precision == MZ_MIXED && ctx->nc2_ok && n > 1) ? 2 : 1;
          for (int anc = 1; anc <= ancs; ++anc) {
            const int pmax = anc == 2 ? ctx->adj2_per_sm : ctx->adj_per_sm;
            // the FP64 gradient's sums follow the 256-slot partition only
            const int nv = precision == MZ_FP64 ? 1 : mz_ctx::NCAPS;
            for (int v = 0; v < nv; ++v)
              for (int per = pmax; per >= std::max(1, pmax - 1); --per) {
                mz_ctx::Tune c = best;
                c.adj = v;
                c.adj_nc = anc;
                c.ctas = adj_ctas_for(ctx, v, per);
                apply_variant(ctx, c);
                const double x = trial(ctx, n, d_params, precision, grad, MZ_K_ADJ);
                if (x < ba) {
                  ba = x;
                  best.adj = v;
                  best.adj_nc = anc;
                  best.ctas = c.ctas;
                }
              }
          }
        }
        ctx->launches = l0;  // trials are not the caller's launches
      }
      // mixed meam/spline: the triplet-moment path, against the row kernels'
      // best (whole call), or always with MZ_FM=2
      if (precision == MZ_MIXED && ctx->fm.eligible && ctx->fm_mode > 0 &&
          (ctx->fm_mode == 2 || ctx->autotune == 1) && fm_prepare(ctx)) {
        if (ctx->fm_mode == 2) {
          best.fm = true;
        } else {
          const int64_t l0 = ctx->launches;
          mz_ctx::Tune c = best;
          apply_variant(ctx, c);
          trial(ctx, n, d_params, precision, grad, -1);
          const double t_rows = trial(ctx, n, d_params, precision, grad, -1);
          c.fm = true;
          apply_variant(ctx, c);
          trial(ctx, n, d_params, precision, grad, -1);
          const double t_fm = trial(ctx, n, d_params, precision, grad, -1);
          best.fm = t_fm < t_rows;
          ctx->launches = l0;
        }
      }
      best.done = true;
      t = best;
      std::lock_guard<std::mutex> lk(g_tune_mu);
      g_tune_cache.emplace(key, best);
    }
    t.done = true;
  }
  apply_variant(ctx, t);
}

// The kernels of one objective call on the context's own buffers: captured
// into a CUDA graph the first time a shape is seen, replayed afterwards (not
// while profiling, whose per-kernel events are recorded around launches).
constexpr size_t MAX_GRAPHS = 32;
void launch_objective(mz_ctx *ctx, int n, int precision, bool ev, bool fo, bool en, bool st, bool gr) {
  tune_variant(ctx, n, ctx->d_params, precision, gr);
  auto go = [&] {
    enqueue(ctx, n, ctx->d_params, precision, ctx->d_obj, ev ? ctx->d_errvec : nullptr, fo ? ctx->d_forces : nullptr,
            en ? ctx->d_energy : nullptr, st ? ctx->d_stress : nullptr, gr ? ctx->d_grad : nullptr);
  };
  if (!ctx->use_graphs || ctx->profiling) {
    go();
    return;
  }
  const uint64_t key = ((uint64_t)n << 8) | ((uint64_t)precision << 5) | ((uint64_t)ev << 4) | ((uint64_t)fo << 3) |
                       ((uint64_t)en << 2) | ((uint64_t)st << 1) | (uint64_t)gr;
  auto it = ctx->graphs.find(key);
  if (it == ctx->graphs.end()) {
    if (ctx->graphs.size() >= MAX_GRAPHS) {
      go();
      return;
    }
    const int64_t l0 = ctx->launches;
    cudaGraph_t g = nullptr;
    ck(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal), "graph capture");
    try {
      go();
    } catch (...) {
      cudaStreamEndCapture(ctx->stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    ck(cudaStreamEndCapture(ctx->stream, &g), "graph capture end");
    cudaGraphExec_t ex = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    ck(ie, "graph instantiate");
    const int64_t nk = ctx->launches - l0;
    ctx->launches = l0;
    it = ctx->graphs.emplace(key, mz_ctx::Graph{ex, nk}).first;
  }
  ck(cudaGraphLaunch(it->second.exec, ctx->stream), "graph launch");
  ctx->launches += it->second.kernels;
}

void run_host(mz_ctx *ctx, int ncand, const double *params, int precision, double *obj, double *errvec,
              double *forces, double *energy, double *stress, double *grad) {
  if (!ctx || !params || !obj || ncand <= 0) throw Failure{MZ_ERR_ARG, "bad argument"};
  if (precision != MZ_FP64 && precision != MZ_MIXED) throw Failure{MZ_ERR_ARG, "unknown precision"};
  if (grad) check_adjoint(ctx, precision);
  ck(cudaSetDevice(ctx->device), "cudaSetDevice");
  const int P = ctx->P, E = ctx->esize, N = ctx->natoms, NC = ctx->ncells;
  for (int c0 = 0; c0 < ncand; c0 += ctx->cand_cap) {
    const int n = std::min(ctx->cand_cap, ncand - c0);
    ck(cudaMemcpyAsync(ctx->d_params, params + (size_t)c0 * P, sizeof(double) * n * P, cudaMemcpyHostToDevice,
                       ctx->stream),
       "params H2D");
    launch_objective(ctx, n, precision, errvec != nullptr, forces != nullptr, energy != nullptr, stress != nullptr,
                     grad != nullptr);
    ck(cudaMemcpyAsync(obj + c0, ctx->d_obj, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream), "obj D2H");
    if (grad)
      ck(cudaMemcpyAsync(grad + (size_t)c0 * P, ctx->d_grad, sizeof(double) * n * P, cudaMemcpyDeviceToHost,
                         ctx->stream),
         "grad D2H");
    if (errvec)
      ck(cudaMemcpyAsync(errvec + (size_t)c0 * E, ctx->d_errvec, sizeof(double) * n * E, cudaMemcpyDeviceToHost,
                         ctx->stream),
         "errvec D2H");
    if (forces)
      ck(cudaMemcpyAsync(forces + (size_t)c0 * 3 * N, ctx->d_forces, sizeof(double) * n * 3 * N,
                         cudaMemcpyDeviceToHost, ctx->stream),
         "forces D2H");
    if (energy)
      ck(cudaMemcpyAsync(energy + (size_t)c0 * NC, ctx->d_energy, sizeof(double) * n * NC, cudaMemcpyDeviceToHost,
                         ctx->stream),
         "energy D2H");
    if (stress)
      ck(cudaMemcpyAsync(stress + (size_t)c0 * 6 * NC, ctx->d_stress, sizeof(double) * n * 6 * NC,
                         cudaMemcpyDeviceToHost, ctx->stream),
         "stress D2H");
    ck(cudaStreamSynchronize(ctx->stream), "objective");
    check_device_flag(ctx);
  }
}

}  // namespace

extern "C" {

mz_status mz_create(const mz_db *dbh, const mz_pot *poth, const mz_settings *set, mz_ctx **out) {
  mz_ctx *ctx = nullptr;
  mz_status st = guarded([&] {
    if (!dbh || !poth || !set || !out) throw Failure{MZ_ERR_ARG, "null argument"};
    const Db &db = dbh->db;
    const Pot &pot = poth->pot;
    if (db.npairs >= (int64_t(1) << 31)) throw Failure{MZ_ERR_RANGE, "more than 2^31 pairs"};
    if (db.max_row > BLOCK_SLOTS)
      throw Failure{MZ_ERR_RANGE, "neighbour row of " + std::to_string(db.max_row) +
                                      " pairs exceeds the kernel limit of " + std::to_string(BLOCK_SLOTS)};
    if (pot.nsplines() > MAX_SPLINES) throw Failure{MZ_ERR_RANGE, "too many splines"};
    const bool meam = style_meam(pot.style);
    if (style_pair(db.style) != style_pair(pot.style) || (meam && !style_meam(db.style)))
      throw Failure{MZ_ERR_ARG, "the database's lists were built for another potential style"};
    if (meam)
      for (int gi : {(int)G_G, (int)G_Q1, (int)G_Q2})
        if (gi < (int)pot.groups.size())
          for (auto &g : pot.groups[gi]) {
            if (g.nknots > MAX_G_KNOTS)
              throw Failure{MZ_ERR_RANGE, "angular spline with more than " + std::to_string(MAX_G_KNOTS) + " knots"};
          }
    ctx = new mz_ctx;
    ctx->device = set->device;
    ck(cudaSetDevice(ctx->device), "cudaSetDevice");
    ck(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    ctx->natoms = db.natoms;
    ctx->ncells = db.ncells;
    ctx->npairs = db.npairs;
    ctx->max_cand = std::max(1, set->max_candidates);

    // ---- potential structure
    const int ns = pot.nsplines();
    const PotImage im = pot_image(pot);
    const std::vector<SplineGeom> &geom = im.geom;
    const std::vector<int> &nat = im.nat, &cmap = im.cmap;
    const std::vector<double> &base = im.base, &Mall = im.M;
    const int stride = im.stride;
    ctx->pstride = im.pstride;
    ctx->P = im.P;
    ctx->q5 = false;  // any spline5eq spline: the kernels built for per-spline bases
    for (int s = 0; s < ns; ++s) ctx->q5 = ctx->q5 || pot.spline(s).quintic;
    ctx->nsplines = ns;
    ctx->stride = stride;
    ctx->d_geom = dupload(ctx, geom.data(), ns);
    ctx->d_nat = dupload(ctx, nat.data(), nat.size());
    ctx->d_base = dupload(ctx, base.data(), base.size());
    ctx->d_cmap = dupload(ctx, cmap.data(), cmap.size());
    ctx->d_M = dupload(ctx, Mall.data(), Mall.size());
    DevPot &dp = ctx->pot;
    dp.style = pot.style;
    dp.ntypes = pot.ntypes;
    dp.nsplines = ns;
    dp.tab_stride = stride;
    dp.pow_stride = ctx->pstride;
    dp.pair = style_pair(pot.style) ? 1 : 0;
    dp.s_phi = pot.spline_index(G_PHI, 0);
    dp.s_rho = dp.pair ? 0 : pot.spline_index(G_RHO, 0);
    dp.s_U = dp.pair ? 0 : pot.spline_index(G_U, 0);
    dp.s_f = meam ? pot.spline_index(G_F, 0) : 0;
    dp.s_g = meam ? pot.spline_index(G_G, 0) : 0;
    dp.embed_extrap = set->embed_extrap;
    dp.energy_weight = set->energy_weight;
    dp.stress_weight = set->stress_weight;
    dp.omit_pen = set->omit_punishments;
    dp.gmeam = pot.style == MZ_STYLE_GMEAM_SPLINE;
    dp.npair = pot.ntypes * (pot.ntypes + 1) / 2;
    dp.nj = style_nj(pot.style);
    for (int m = 0; m < 2; ++m) {
      dp.s_p[m] = m < dp.nj ? pot.spline_index(m == 0 ? G_P1 : G_P2, 0) : 0;
      dp.s_q[m] = m < dp.nj ? pot.spline_index(m == 0 ? G_Q1 : G_Q2, 0) : 0;
    }
    dp.aux_rows = AUX_COUNT * (1 + dp.nj);
    ctx->npen = style_npen(pot.style, pot.ntypes);
    ctx->esize = style_esize(pot.style, pot.ntypes, db.ncells, db.natoms);

    // ---- database
    const int N = db.natoms;
    const int64_t Np = db.npairs;
    DevDb &d = ctx->db;
    d.ncells = db.ncells;
    d.natoms = N;
    d.npairs = Np;
    d.cell_atom0 = dupload(ctx, db.cell_atom0.data(), db.cell_atom0.size());
    d.cell_vol = dupload(ctx, db.cell_vol.data(), db.cell_vol.size());
    d.cell_w = dupload(ctx, db.cell_weight.data(), db.cell_weight.size());
    d.cell_ew = dupload(ctx, db.cell_eweight.data(), db.cell_eweight.size());
    d.cell_sw = dupload(ctx, db.cell_sweight.data(), db.cell_sweight.size());
    d.cell_e0 = dupload(ctx, db.cell_energy0.data(), db.cell_energy0.size());
    d.cell_s0 = dupload(ctx, db.cell_stress0.data(), db.cell_stress0.size());
    d.atom_type = dupload(ctx, db.atom_type.data(), db.atom_type.size());
    d.atom_cell = dupload(ctx, db.atom_cell.data(), db.atom_cell.size());
    d.force0 = dupload(ctx, db.atom_force0.data(), db.atom_force0.size());
    const int nf = db.nfun;
    std::vector<int> off32(N + 1), inoff32(N + 1), inslot32(Np), knot32(Np);
    std::vector<signed char> knotp2(nf > 4 ? Np : 0);
    for (int i = 0; i <= N; ++i) {
      off32[i] = (int)db.pair_off[i];
      inoff32[i] = (int)db.in_off[i];
    }
    for (int64_t s = 0; s < Np; ++s) {
      inslot32[s] = (int)db.in_slot[s];
      knot32[s] = packed_knots(db, s);
      if (nf > 4) knotp2[s] = db.pair_knot[nf * s + 4];
    }
    d.pair_knot_p2 = nf > 4 ? dupload(ctx, knotp2.data(), knotp2.size()) : nullptr;
    d.pair_off = dupload(ctx, off32.data(), off32.size());
    d.in_off = dupload(ctx, inoff32.data(), inoff32.size());
    d.in_slot = dupload(ctx, inslot32.data(), inslot32.size());
    d.pair_knot = dupload(ctx, knot32.data(), knot32.size());
    d.pair_nbr = dupload(ctx, db.pair_nbr.data(), db.pair_nbr.size());
    {
      std::vector<double> ux(Np), uy(Np), uz(Np), sh(nf * Np);
      std::vector<float> rf(Np), uxf(Np), uyf(Np), uzf(Np), shf(nf * Np);
      for (int64_t s = 0; s < Np; ++s) {
        ux[s] = db.pair_u[3 * s];
        uy[s] = db.pair_u[3 * s + 1];
        uz[s] = db.pair_u[3 * s + 2];
        rf[s] = (float)db.pair_r[s];
        uxf[s] = (float)ux[s];
        uyf[s] = (float)uy[s];
        uzf[s] = (float)uz[s];
        for (int q = 0; q < nf; ++q) {
          sh[q * Np + s] = db.pair_shift[nf * s + q];
          shf[q * Np + s] = (float)db.pair_shift[nf * s + q];
        }
      }
      d.pair_r = dupload(ctx, db.pair_r.data(), Np);
      d.pair_ux = dupload(ctx, ux.data(), Np);
      d.pair_uy = dupload(ctx, uy.data(), Np);
      d.pair_uz = dupload(ctx, uz.data(), Np);
      d.pair_shift = dupload(ctx, sh.data(), nf * Np);
      d.pair_rf = dupload(ctx, rf.data(), Np);
      d.pair_uxf = dupload(ctx, uxf.data(), Np);
      d.pair_uyf = dupload(ctx, uyf.data(), Np);
      d.pair_uzf = dupload(ctx, uzf.data(), Np);
      d.pair_shiftf = dupload(ctx, shf.data(), nf * Np);
    }
    // atom blocks: consecutive atoms, <= cap slots and <= cap / 4 atoms, for
    // each of the autotuner's caps (a row longer than the cap is a block of its own)
    for (int v = 0; v < mz_ctx::NCAPS; ++v) {
      const int cap = TUNE_CAPS[v], acap = std::max(1, cap / 4);
      std::vector<int> blk(1, 0);
      int slots = 0, atoms = 0;
      for (int i = 0; i < N; ++i) {
        const int n = (int)(db.pair_off[i + 1] - db.pair_off[i]);
        if (atoms > 0 && (slots + n > cap || atoms + 1 > acap)) {
          blk.push_back(i);
          slots = 0;
          atoms = 0;
        }
        slots += n;
        atoms += 1;
      }
      blk.push_back(N);
      ctx->nblk[v] = (int)blk.size() - 1;
      ctx->d_blk[v] = dupload(ctx, blk.data(), blk.size());
    }
    d.nblocks = ctx->nblk[0];
    d.blk_atom0 = ctx->d_blk[0];
    // type-pure atom blocks of the adjoint (one g-table type per block)
    {
      std::vector<int> order(N);
      for (int i = 0; i < N; ++i) order[i] = i;
      std::stable_sort(order.begin(), order.end(),
                       [&](int a, int b) { return db.atom_type[a] < db.atom_type[b]; });
      d.adj_atoms = dupload(ctx, order.data(), order.size());
      for (int v = 0; v < mz_ctx::NCAPS; ++v) {
        const int cap = TUNE_CAPS[v], acap = std::max(1, cap / 4);
        std::vector<int> b0(1, 0);
        int slots = 0, atoms = 0, ty = -1;
        for (int q = 0; q < N; ++q) {
          const int i = order[q];
          const int n = (int)(db.pair_off[i + 1] - db.pair_off[i]);
          if (atoms > 0 && (db.atom_type[i] != ty || slots + n > cap || atoms + 1 > acap)) {
            b0.push_back(q);
            slots = 0;
            atoms = 0;
          }
          ty = db.atom_type[i];
          slots += n;
          atoms += 1;
        }
        b0.push_back(N);
        ctx->nadjblk[v] = (int)b0.size() - 1;
        ctx->d_adjblk[v] = dupload(ctx, b0.data(), b0.size());
        // descriptors: na + 1 entries per block at b0[b] + b
        std::vector<int4> desc;
        desc.reserve((size_t)N + b0.size());
        int amax = 1;
        for (size_t b = 0; b + 1 < b0.size(); ++b) {
          const int na = b0[b + 1] - b0[b];
          const int tb = db.atom_type[order[b0[b]]];
          int lo = 0;
          for (int q = b0[b]; q < b0[b + 1]; ++q) {
            const int i = order[q];
            desc.push_back(make_int4(i, lo, na | tb << 8, db.atom_cell[i]));
            lo += (int)(db.pair_off[i + 1] - db.pair_off[i]);
          }
          desc.push_back(make_int4(0, lo, na | tb << 8, 0));
          amax = std::max(amax, na + 1);
        }
        ctx->adjamax[v] = amax;
        ctx->d_adjdesc[v] = dupload(ctx, desc.data(), desc.size());
      }
      d.adj_nblocks = ctx->nadjblk[0];
      d.adj_blk0 = ctx->d_adjblk[0];
      d.adj_desc = ctx->d_adjdesc[0];
      d.adj_amax = ctx->adjamax[0];
      // FP64 adjoint groups: at most about 1024 partials per candidate
      d.adj_group = std::max(1, ctx->nadjblk[0] / 1024);

      // ---- triplet-moment path (mixed meam/spline): shape, feature slots
      // (the type-sorted rows, each type's run padded to FM_TILE)
      if (pot.style == MZ_STYLE_MEAM_SPLINE && !ctx->q5 && pot.ntypes <= FM_MAXT) {
        int NA = 0, NN = 0, PB = 0, NBp = 0;
        for (int t = 0; t < dp.npair; ++t) NA = std::max(NA, pot.spline(dp.s_f + t).nknots + 2);
        for (int t = 0; t < pot.ntypes; ++t) NN = std::max(NN, pot.spline(dp.s_g + t).nknots + 2);
        for (int s = 0; s < ns; ++s)
          if (s < dp.s_U || s >= dp.s_f) PB = std::max(PB, pot.spline(s).nknots + 2);
        for (int s = 0; s < dp.s_g; ++s)
          if (s < dp.s_U || s >= dp.s_f) NBp = std::max(NBp, pot.spline(s).nknots + 2);
        if (pot.ntypes * NA <= 32 && NN <= FM_MAXN && PB <= 23 && db.max_row <= BLOCK_SLOTS) {
          FmPlan &fp = ctx->fm.plan;
          fp.nt = pot.ntypes;
          fp.NA = NA;
          fp.NN = NN;
          fp.NB = NBp;
          // the U splines are consecutive in the knot table
          fp.utoff = im.geom[dp.s_U].toff;
          fp.ustride = im.geom[dp.s_U + pot.ntypes - 1].toff + 2 * im.geom[dp.s_U + pot.ntypes - 1].n + 2 - fp.utoff;
          fp.D = pot.ntypes * NA * NN;
          fp.Dpad = (fp.D + FM_DC - 1) / FM_DC * FM_DC;
          fp.nch = fp.Dpad / FM_DC;
          std::vector<int> row0(N, 0);
          int64_t q = 0;
          int tix = 0;
          for (int t = 0; t < pot.ntypes; ++t) {
            fp.tile0[t] = (int)(q / FM_TILE);
            for (; tix < N && db.atom_type[order[tix]] == t; ++tix) {
              const int i = order[tix];
              row0[i] = (int)q;
              q += db.pair_off[i + 1] - db.pair_off[i];
            }
            fp.qend[t] = q;
            q = (q + FM8_TM - 1) / FM8_TM * FM8_TM;  // type runs on 128-slot tiles (mz_fm8.cuh)
          }
          fp.Q = q;
          fp.ntiles = (int)(q / FM_TILE);
          for (int t = pot.ntypes; t <= FM_MAXT; ++t) fp.tile0[t] = fp.ntiles;
          if (q < (int64_t(1) << 31) && tix == N) {
            fp.row0 = dupload(ctx, row0.data(), row0.size());
            // the epilogues' atom blocks: type-pure runs of the type-sorted
            // order, <= BLOCK_SLOTS slots and <= FM_ABLK atoms
            std::vector<int> b0(1, 0);
            int slots = 0, atoms = 0, ty = -1;
            for (int qa = 0; qa < N; ++qa) {
              const int i = order[qa];
              const int nr = (int)(db.pair_off[i + 1] - db.pair_off[i]);
              if (atoms > 0 && (db.atom_type[i] != ty || slots + nr > BLOCK_SLOTS || atoms + 1 > FM_ABLK)) {
                b0.push_back(qa);
                slots = 0;
                atoms = 0;
              }
              ty = db.atom_type[i];
              slots += nr;
              atoms += 1;
            }
            b0.push_back(N);
            fp.nblk = (int)b0.size() - 1;
            fp.blk0 = dupload(ctx, b0.data(), b0.size());
            ctx->fm.eligible = true;
          }
        }
      }
    }

    // ---- shared memory of the kernels
    ctx->smem_atoms[0] = atoms_smem_bytes<double>(ns, ctx->pstride, dp.nj);
    ctx->smem_atoms[1] = atoms_smem_bytes<float>(ns, ctx->pstride, dp.nj);
    int ng = 2;  // the adjoint's per-thread tables hold the largest angular spline (g, q, q2)
    bool gq5 = false;
    if (meam)
      for (int gi : {(int)G_G, (int)G_Q1, (int)G_Q2})
        if (gi < (int)pot.groups.size())
          for (auto &g : pot.groups[gi]) {
            ng = std::max(ng, g.nknots);
            gq5 = gq5 || g.quintic;
          }
    dp.g_nmax = ng;
    dp.g_q5 = gq5 ? 1 : 0;
    const int gtabs = dp.gmeam ? pot.ntypes : 1;
    ctx->smem_adj[0] = adj_smem_bytes<double>(ns, stride, ctx->pstride, meam, gtabs, ng, gq5);
    ctx->smem_adj[1] = adj_smem_bytes<float>(ns, stride, ctx->pstride, meam, gtabs, ng, gq5);
    int smem_max = 0;
    ck(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device), "attribute");
    ctx->smem_optin = smem_max;
    if (ctx->smem_atoms[0] > (size_t)smem_max)
      throw Failure{MZ_ERR_RANGE, "potential too large for the kernels' shared-memory tables"};
    // the gradient of a precision whose adjoint tables do not fit is refused at the call
    ctx->adj_fits[0] = ctx->smem_adj[0] <= (size_t)smem_max;
    ctx->adj_fits[1] = ctx->smem_adj[1] <= (size_t)smem_max;
    smem_attr(k_atoms<true, double, false>, ctx->smem_atoms[0]);
    smem_attr(k_atoms<true, double, true>, ctx->smem_atoms[0]);
    smem_attr(k_atoms<false, double, false>, ctx->smem_atoms[0]);
    smem_attr(k_atoms<true, float, false>, ctx->smem_atoms[1]);
    smem_attr(k_atoms<true, float, true>, ctx->smem_atoms[1]);
    smem_attr(k_atoms<false, float, false>, ctx->smem_atoms[1]);
    if (ctx->adj_fits[0]) smem_attr(k_adj<true, double>, ctx->smem_adj[0]);
    if (ctx->adj_fits[0]) smem_attr(k_adj<false, double>, ctx->smem_adj[0]);
    if (ctx->adj_fits[1]) smem_attr(k_adj<true, float>, ctx->smem_adj[1]);
    if (ctx->adj_fits[1]) smem_attr(k_adj<false, float>, ctx->smem_adj[1]);
    smem_attr(k_atoms<true, double, false, true>, ctx->smem_atoms[0]);
    smem_attr(k_atoms<true, double, true, true>, ctx->smem_atoms[0]);
    smem_attr(k_atoms<true, float, false, true>, ctx->smem_atoms[1]);
    smem_attr(k_atoms<true, float, true, true>, ctx->smem_atoms[1]);
    if (ctx->adj_fits[0]) smem_attr(k_adj<true, double, true>, ctx->smem_adj[0]);
    if (ctx->adj_fits[1]) smem_attr(k_adj<true, float, true>, ctx->smem_adj[1]);
    smem_attr(k_atoms<true, double, false, false, true>, ctx->smem_atoms[0]);
    smem_attr(k_atoms<true, double, true, false, true>, ctx->smem_atoms[0]);
    smem_attr(k_atoms<true, float, false, false, true>, ctx->smem_atoms[1]);
    smem_attr(k_atoms<true, float, true, false, true>, ctx->smem_atoms[1]);
    if (ctx->adj_fits[0]) smem_attr(k_adj<true, double, false, true>, ctx->smem_adj[0]);
    if (ctx->adj_fits[1]) smem_attr(k_adj<true, float, false, true>, ctx->smem_adj[1]);
    ctx->smem_atoms2 = atoms2_smem_bytes(ns, ctx->pstride);
    ctx->smem_adj2 = adj2_smem_bytes(ns, stride, ctx->pstride, ng);
    ctx->nc2_ok = pot.style == MZ_STYLE_MEAM_SPLINE && !ctx->q5 && ctx->smem_atoms2 <= (size_t)smem_max &&
                  ctx->smem_adj2 <= (size_t)smem_max;
    if (ctx->nc2_ok) {
      smem_attr(k_atoms2<true>, ctx->smem_atoms2);
      smem_attr(k_atoms2<false>, ctx->smem_atoms2);
      smem_attr(k_adj2, ctx->smem_adj2);
    }
    smem_attr(k_atoms<true, double, true, false, false, true>, ctx->smem_atoms[0]);
    smem_attr(k_atoms<true, float, true, false, false, true>, ctx->smem_atoms[1]);
    if (ctx->adj_fits[0]) smem_attr(k_adj<true, double, false, false, true>, ctx->smem_adj[0]);
    if (ctx->adj_fits[0]) smem_attr(k_adj<false, double, false, false, true>, ctx->smem_adj[0]);
    if (ctx->adj_fits[1]) smem_attr(k_adj<true, float, false, false, true>, ctx->smem_adj[1]);
    if (ctx->adj_fits[1]) smem_attr(k_adj<false, float, false, false, true>, ctx->smem_adj[1]);
    smem_attr(k_atoms<true, double, false, false, false, true>, ctx->smem_atoms[0]);
    smem_attr(k_atoms<false, double, false, false, false, true>, ctx->smem_atoms[0]);
    smem_attr(k_atoms<true, float, false, false, false, true>, ctx->smem_atoms[1]);
    smem_attr(k_atoms<false, float, false, false, false, true>, ctx->smem_atoms[1]);
    // spline5eq in gmeam/spline and jmeam[2]/spline potentials
    smem_attr(k_atoms<true, double, false, true, false, true>, ctx->smem_atoms[0]);
    smem_attr(k_atoms<true, double, true, true, false, true>, ctx->smem_atoms[0]);
    smem_attr(k_atoms<true, float, false, true, false, true>, ctx->smem_atoms[1]);
    smem_attr(k_atoms<true, float, true, true, false, true>, ctx->smem_atoms[1]);
    smem_attr(k_atoms<true, double, false, false, true, true>, ctx->smem_atoms[0]);
    smem_attr(k_atoms<true, double, true, false, true, true>, ctx->smem_atoms[0]);
    smem_attr(k_atoms<true, float, false, false, true, true>, ctx->smem_atoms[1]);
    smem_attr(k_atoms<true, float, true, false, true, true>, ctx->smem_atoms[1]);
    if (ctx->adj_fits[0]) smem_attr(k_adj<true, double, true, false, true>, ctx->smem_adj[0]);
    if (ctx->adj_fits[1]) smem_attr(k_adj<true, float, true, false, true>, ctx->smem_adj[1]);
    if (ctx->adj_fits[0]) smem_attr(k_adj<true, double, false, true, true>, ctx->smem_adj[0]);
    if (ctx->adj_fits[1]) smem_attr(k_adj<true, float, false, true, true>, ctx->smem_adj[1]);
    int nsm = 0, per_sm = 0;
    ck(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device), "attribute");
    if (ctx->adj_fits[1])
      ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_adj<true, float>, BLOCK_SLOTS, ctx->smem_adj[1]),
         "occupancy");
    ctx->adj_per_sm = std::max(1, per_sm);
    if (ctx->nc2_ok) {
      int p2 = 0;
      ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p2, k_adj2, BLOCK_SLOTS, ctx->smem_adj2), "occupancy");
      ctx->adj2_per_sm = std::max(1, p2);
    }
    int most_blocks = 0;
    for (int v = 0; v < mz_ctx::NCAPS; ++v) most_blocks = std::max(most_blocks, ctx->nadjblk[v]);
    ctx->adj_ctas_max = std::max(1, std::min(most_blocks, nsm * ctx->adj_per_sm));
    ctx->adj_ctas = std::max(1, std::min(d.adj_nblocks, nsm * ctx->adj_per_sm));
    ctx->nsm = nsm;
    {
      const char *env = std::getenv("MZ_TUNE");
      ctx->autotune = (env && env[0] == '0') ? 0 : (env && env[0] == '2') ? 2 : 1;
    }
    {
      const char *env = std::getenv("MZ_GRAPH");
      ctx->use_graphs = !(env && env[0] == '0');
    }
    {
      const char *env = std::getenv("MZ_ADJ_CTAS");
      ctx->adj_ctas_force = env ? std::max(0, std::atoi(env)) : 0;
    }
    {
      const char *env = std::getenv("MZ_FM");
      ctx->fm_mode = (env && env[0] == '0') ? 0 : (env && env[0] == '2') ? 2 : 1;
    }
    {
      const char *env = std::getenv("MZ_FM8");
      ctx->fm8_mode = (env && env[0] == '0') ? 0 : 1;
    }
    {
      const char *env = std::getenv("MZ_FM8ADJ");
      ctx->fm8a_mode = (env && env[0] == '0') ? 0 : 1;
    }
    // tensor-core forward (mixed precision, MEAM with TC_NB B-spline coefficients per g spline)
    {
      const char *env = std::getenv("MZ_TC");  // opt-in: "1"
      const bool allowed = env && env[0] == '1';
      ctx->tc = tc_plan(db.max_row, TC_NB, pot.ntypes, ns, smem_max);
      ctx->tc_ok =
          allowed && pot.style == MZ_STYLE_MEAM_SPLINE && !ctx->q5 && ng + 2 == TC_NB && ctx->tc.smem_bytes > 0;
      if (ctx->tc_ok) {
        smem_attr(k_atoms_tc<TC_NB, false>, (size_t)ctx->tc.smem_bytes);
        smem_attr(k_atoms_tc<TC_NB, true>, (size_t)ctx->tc.smem_bytes);
      }
    }

    // ---- work buffers: candidates per launch bounded by device memory
    size_t freeb = 0, totalb = 0;
    ck(cudaMemGetInfo(&freeb, &totalb), "cudaMemGetInfo");
    const size_t per_cand =
        sizeof(double) * ((size_t)(3 + (meam ? dp.aux_rows : 0)) * Np + (size_t)(AO_COUNT + 3 + 3) * N +
                          (size_t)ctx->esize + (size_t)(8 + 1 + CS_COUNT) * db.ncells + 2 * (size_t)stride + ctx->pstride +
                          (size_t)ctx->adj_ctas_max * stride * (1 + ADJ_WARPS) + (size_t)2048 * stride +
                          2 * (size_t)ctx->P + 1);
    const size_t budget = (size_t)(0.6 * (double)freeb);
    const int cap = (int)std::max<size_t>(1, budget / std::max<size_t>(per_cand, 1));
    ctx->cand_cap = std::min(ctx->max_cand, cap);
    const size_t C = ctx->cand_cap;
    ctx->d_params = dalloc<double>(ctx, C * ctx->P);
    ctx->d_tabs = dalloc<double>(ctx, C * stride);
    ctx->d_ptabs = dalloc<double>(ctx, C * ctx->pstride);
    ctx->d_V = dalloc<double>(ctx, C * 3 * Np);
    ctx->d_aout = dalloc<double>(ctx, C * AO_COUNT * N);
    ctx->d_forces = dalloc<double>(ctx, C * 3 * N);
    ctx->d_cellobj = dalloc<double>(ctx, C * db.ncells);
    ctx->d_obj = dalloc<double>(ctx, C);
    ctx->d_errvec = dalloc<double>(ctx, C * ctx->esize);
    ctx->d_energy = dalloc<double>(ctx, C * db.ncells);
    ctx->d_stress = dalloc<double>(ctx, C * 6 * db.ncells);
    ctx->d_aux = meam ? dalloc<double>(ctx, C * dp.aux_rows * Np) : nullptr;
    ctx->d_lam = dalloc<double>(ctx, C * 3 * N);
    ctx->d_seeds = dalloc<double>(ctx, C * CS_COUNT * db.ncells);
    const size_t nparts = std::max<size_t>(ctx->adj_ctas_max, (ctx->nadjblk[0] + d.adj_group - 1) / d.adj_group);
    ctx->d_partial = dalloc<double>(ctx, C * nparts * stride);
    ctx->d_wglob = dalloc<double>(ctx, C * (size_t)ctx->adj_ctas_max * ADJ_WARPS * stride);
    ctx->d_grad = dalloc<double>(ctx, C * ctx->P);
    ctx->d_ptabf = dalloc<float>(ctx, C * ctx->pstride);
    ctx->d_wtab = meam ? dalloc<float>(ctx, C * pot.ntypes * (2 * TC_NB - 1)) : nullptr;
    ctx->d_err = dalloc<int>(ctx, 1);
    ck(cudaMemset(ctx->d_err, 0, sizeof(int)), "flag init");
    *out = ctx;
  });
  if (st != MZ_OK && ctx) {
    release(ctx);
    delete ctx;
  }
  return st;
}

void mz_destroy(mz_ctx *ctx) {
  if (!ctx) return;
  release(ctx);
  delete ctx;
}

mz_status mz_objective(mz_ctx *ctx, int ncand, const double *params, int precision, double *obj, double *errvec,
                       double *forces, double *energy, double *stress) {
  return guarded([&] { run_host(ctx, ncand, params, precision, obj, errvec, forces, energy, stress, nullptr); });
}

mz_status mz_objective_grad(mz_ctx *ctx, int ncand, const double *params, int precision, double *obj, double *grad) {
  return guarded([&] {
    if (!grad) throw Failure{MZ_ERR_ARG, "null gradient buffer"};
    run_host(ctx, ncand, params, precision, obj, nullptr, nullptr, nullptr, nullptr, grad);
  });
}

mz_status mz_objective_device(mz_ctx *ctx, int ncand, const double *d_params, int precision, double *d_obj,
                              double *d_errvec, double *d_forces) {
  return guarded([&] {
    if (!ctx || !d_params || !d_obj || ncand <= 0) throw Failure{MZ_ERR_ARG, "bad argument"};
    if (ncand > ctx->cand_cap)
      throw Failure{MZ_ERR_RANGE,
                    "ncand exceeds the candidates one launch can hold (" + std::to_string(ctx->cand_cap) + ")"};
    if (precision != MZ_FP64 && precision != MZ_MIXED) throw Failure{MZ_ERR_ARG, "unknown precision"};
    ck(cudaSetDevice(ctx->device), "cudaSetDevice");
    tune_variant(ctx, ncand, d_params, precision, false);
    enqueue(ctx, ncand, d_params, precision, d_obj, d_errvec, d_forces, nullptr, nullptr, nullptr);
  });
}

mz_status mz_objective_grad_device(mz_ctx *ctx, int ncand, const double *d_params, int precision, double *d_obj,
                                   double *d_grad) {
  return guarded([&] {
    if (!ctx || !d_params || !d_obj || !d_grad || ncand <= 0) throw Failure{MZ_ERR_ARG, "bad argument"};
    if (ncand > ctx->cand_cap)
      throw Failure{MZ_ERR_RANGE,
                    "ncand exceeds the candidates one launch can hold (" + std::to_string(ctx->cand_cap) + ")"};
    if (precision != MZ_FP64 && precision != MZ_MIXED) throw Failure{MZ_ERR_ARG, "unknown precision"};
    check_adjoint(ctx, precision);
    ck(cudaSetDevice(ctx->device), "cudaSetDevice");
    tune_variant(ctx, ncand, d_params, precision, true);
    enqueue(ctx, ncand, d_params, precision, d_obj, nullptr, nullptr, nullptr, nullptr, d_grad);
  });
}

mz_status mz_densities(mz_ctx *ctx, const double *params, double *dens) {
  return guarded([&] {
    if (!ctx || !params || !dens) throw Failure{MZ_ERR_ARG, "bad argument"};
    if (ctx->pot.pair)  // PotPair has no compute_densities (pot_pair.h:25-42)
      throw Failure{MZ_ERR_UNSUPPORTED, "pair/spline has no embedding densities"};
    ck(cudaSetDevice(ctx->device), "cudaSetDevice");
    ck(cudaMemcpyAsync(ctx->d_params, params, sizeof(double) * ctx->P, cudaMemcpyHostToDevice, ctx->stream),
       "params H2D");
    tune_variant(ctx, 1, ctx->d_params, MZ_FP64, false);
    enqueue(ctx, 1, ctx->d_params, MZ_FP64, ctx->d_obj, nullptr, nullptr, nullptr, nullptr, nullptr);
    ck(cudaMemcpyAsync(dens, ctx->d_aout + (size_t)AO_RHO * ctx->natoms, sizeof(double) * ctx->natoms,
                       cudaMemcpyDeviceToHost, ctx->stream),
       "dens D2H");
    ck(cudaStreamSynchronize(ctx->stream), "densities");
  });
}

mz_status mz_sync(mz_ctx *ctx) {
  return guarded([&] {
    if (!ctx) throw Failure{MZ_ERR_ARG, "null context"};
    ck(cudaStreamSynchronize(ctx->stream), "sync");
    check_device_flag(ctx);
  });
}

void *mz_stream(mz_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

mz_status mz_gram_device(mz_ctx *ctx, int na, const double *d_a, int64_t lda, int nb, const double *d_b,
                         int64_t ldb, int64_t n, double *d_out) {
  return guarded([&] {
    if (!ctx || !d_a || !d_b || !d_out || na <= 0 || nb <= 0 || n <= 0 || lda < n || ldb < n)
      throw Failure{MZ_ERR_ARG, "bad argument"};
    if ((int64_t)na * nb > (int64_t)1 << 26) throw Failure{MZ_ERR_RANGE, "na * nb too large"};
    ck(cudaSetDevice(ctx->device), "cudaSetDevice");
    GramArgs g{};
    g.A = d_a;
    g.B = d_b;
    g.lda = lda;
    g.ldb = ldb;
    g.n = n;
    g.na = na;
    g.nb = nb;
    g.sym = (d_a == d_b && lda == ldb && na == nb) ? 1 : 0;
    g.out = d_out;
    const bool vec = nb <= GRAM_VEC;
    const int64_t unit = vec ? GRAM_VK : GRAM_BK;
    const int64_t units = (n + unit - 1) / unit;
    const int Ti = (na + GRAM_T - 1) / GRAM_T, Tj = (nb + GRAM_T - 1) / GRAM_T;
    const int ntiles = vec ? 1 : (g.sym ? Tj * (Tj + 1) / 2 : Ti * Tj);
    // about four CTAs per SM over all tiles and k ranges
    const int64_t want = std::max<int64_t>(1, (4 * (int64_t)ctx->nsm + ntiles - 1) / ntiles);
    int64_t S = std::min(units, want);
    const int64_t per = (units + S - 1) / S;
    S = (units + per - 1) / per;  // no empty range
    g.S = (int)S;
    g.kper = per * unit;
    const size_t need = (size_t)S * na * nb;
    if (need > ctx->gram_cap) {
      ck(cudaStreamSynchronize(ctx->stream), "gram workspace");
      if (ctx->d_gram) cudaFree(ctx->d_gram);
      ctx->d_gram = nullptr;
      ctx->gram_cap = 0;
      void *p = nullptr;
      cudaError_t e = cudaMalloc(&p, need * sizeof(double));
      if (e != cudaSuccess)
        throw Failure{MZ_ERR_NOMEM, std::string("gram workspace: ") + cudaGetErrorString(e)};
      ctx->d_gram = static_cast<double *>(p);
      ctx->gram_cap = need;
    }
    g.partial = ctx->d_gram;
    if (vec)
      k_gram_vec<<<(unsigned)S, 256, 0, ctx->stream>>>(g);
    else
      k_gram_tile<<<dim3((unsigned)ntiles, (unsigned)S), 256, 0, ctx->stream>>>(g);
    ck(cudaGetLastError(), "k_gram");
    const int outs = na * nb;
    k_gram_sum<<<(outs + 255) / 256, 256, 0, ctx->stream>>>(g);
    ck(cudaGetLastError(), "k_gram_sum");
    ctx->launches += 2;
  });
}

const char *mz_kernel_name(int k) {
  static const char *names[MZ_NKERNELS] = {"k_prep",   "k_atoms",      "k_gather",  "k_cells",  "k_final",
                                           "k_adj",    "k_grad_final", "k_fm_coef", "k_fm_fwd", "k_fm_epi",
                                           "k_fm_pre", "k_fm_adj",     "k_fm_grad"};
  return (k >= 0 && k < MZ_NKERNELS) ? names[k] : "?";
}

mz_status mz_tuning(mz_ctx *ctx, int precision, int grad, int *choice) {
  return guarded([&] {
    if (!ctx || !choice || (precision != MZ_FP64 && precision != MZ_MIXED)) throw Failure{MZ_ERR_ARG, "bad argument"};
    const mz_ctx::Tune &t = ctx->tune[precision][grad ? 1 : 0];
    choice[0] = t.done ? TUNE_CAPS[t.fwd] : 0;
    choice[1] = t.done ? TUNE_CAPS[t.adj] : 0;
    choice[2] = t.done ? t.ctas : 0;
    choice[3] = t.done ? t.nc : 0;
    choice[4] = t.done ? t.adj_nc : 0;
  });
}

mz_status mz_moment_path(const mz_ctx *ctx, int precision, int grad, int *on) {
  return guarded([&] {
    if (!ctx || !on || (precision != MZ_FP64 && precision != MZ_MIXED)) throw Failure{MZ_ERR_ARG, "bad argument"};
    const mz_ctx::Tune &t = ctx->tune[precision][grad ? 1 : 0];
    *on = (t.done && t.fm && ctx->fm.ready) ? (ctx->fm.tc8a ? 3 : ctx->fm.tc8 ? 2 : 1) : 0;
  });
}

mz_status mz_profile(mz_ctx *ctx, int on) {
  return guarded([&] {
    if (!ctx) throw Failure{MZ_ERR_ARG, "null context"};
    ctx->profiling = on != 0;
  });
}

mz_status mz_kernel_times(mz_ctx *ctx, double *ms, int64_t *launches) {
  return guarded([&] {
    if (!ctx || !ms || !launches) throw Failure{MZ_ERR_ARG, "null argument"};
    ck(cudaSetDevice(ctx->device), "cudaSetDevice");
    ck(cudaStreamSynchronize(ctx->stream), "sync");
    for (auto &m : ctx->marks) {
      float t = 0.f;
      ck(cudaEventElapsedTime(&t, m.start, m.stop), "cudaEventElapsedTime");
      ms[m.kernel] += t;
      launches[m.kernel] += 1;
      cudaEventDestroy(m.start);
      cudaEventDestroy(m.stop);
    }
    ctx->marks.clear();
  });
}

mz_status mz_alu_peak(int device, int precision, double *tflops) {
  return guarded([&] {
    if (!tflops) throw Failure{MZ_ERR_ARG, "null argument"};
    ck(cudaSetDevice(device), "cudaSetDevice");
    int nsm = 0;
    ck(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device), "attribute");
    const int threads = 256, blocks = nsm * 8, iters = 1 << 14;
    void *out = nullptr;
    ck(cudaMalloc(&out, 64), "cudaMalloc");
    cudaEvent_t a, b;
    ck(cudaEventCreate(&a), "event");
    ck(cudaEventCreate(&b), "event");
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
      cudaEventRecord(a);
      if (precision == MZ_FP64)
        k_fma_peak<double><<<blocks, threads>>>((double *)out, iters, 0.999999, 1e-7);
      else
        k_fma_peak<float><<<blocks, threads>>>((float *)out, iters, 0.999999f, 1e-7f);
      cudaEventRecord(b);
      ck(cudaEventSynchronize(b), "fma peak");
      float t = 0.f;
      cudaEventElapsedTime(&t, a, b);
      if (rep > 0) best = std::min(best, t);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    *tflops = 2.0 * 8.0 * (double)iters * threads * blocks / (best * 1e-3) / 1e12;
  });
}

mz_status mz_tensor_core_forward(const mz_ctx *ctx, int *on) {
  return guarded([&] {
    if (!ctx || !on) throw Failure{MZ_ERR_ARG, "null argument"};
    *on = ctx->tc_ok ? 1 : 0;
  });
}

mz_status mz_launch_count(const mz_ctx *ctx, int64_t *launches) {
  return guarded([&] {
    if (!ctx || !launches) throw Failure{MZ_ERR_ARG, "null argument"};
    *launches = ctx->launches;
  });
}

}  // extern "C"

// ======================================================== no-allocation path

// The one device array of mz_objective_noalloc.  In host code its name is
// only a host-side stand-in; kernels get the device address looked up once
// per device below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[MZ_NOALLOC_SCRATCH_BYTES];

namespace {

std::mutex g_noalloc_mutex;
void *g_noalloc_addr[64] = {nullptr};

// Sub-array placement inside the scratch array: 256-byte aligned slots.
struct Carve {
  size_t used = 0;
  template <class T>
  size_t take(size_t n) {
    const size_t at = (used + 255) & ~size_t(255);
    used = at + std::max<size_t>(n, 1) * sizeof(T);
    return at;
  }
};

}  // namespace

// Makes `device` current for its lifetime and then restores the caller's
// current device, on every exit path.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int device) {
    ck(cudaGetDevice(&prev), "cudaGetDevice");
    ck(cudaSetDevice(device), "cudaSetDevice");
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

extern "C" mz_status mz_objective_noalloc(const mz_db *dbh, const mz_pot *poth, const mz_settings *set,
                                          const double *params, double *obj, double *forces) {
  return guarded([&] {
    if (!dbh || !poth || !set || !params || !obj) throw Failure{MZ_ERR_ARG, "null argument"};
    int ndev = 0;
    ck(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
    if (set->device < 0 || set->device >= ndev || set->device >= 64)
      throw Failure{MZ_ERR_ARG, "device ordinal out of range"};
    const Db &db = dbh->db;
    const Pot &pot = poth->pot;
    const bool meam = pot.style == MZ_STYLE_MEAM_SPLINE;
    bool any_quintic = false;
    for (int s = 0; s < pot.nsplines(); ++s) any_quintic = any_quintic || pot.spline(s).quintic;
    if (pot.style == MZ_STYLE_GMEAM_SPLINE || style_nj(pot.style) > 0 || any_quintic)
      throw Failure{MZ_ERR_UNSUPPORTED,
                    "the no-allocation objective supports eam/spline, meam/spline and pair/spline with spline3eq"};
    if (style_pair(db.style) != style_pair(pot.style) || (meam && !style_meam(db.style)))
      throw Failure{MZ_ERR_ARG, "the database's lists were built for another potential style"};
    if (db.max_row > BLOCK_SLOTS)
      throw Failure{MZ_ERR_RANGE, "neighbour row of " + std::to_string(db.max_row) +
                                      " pairs exceeds the kernel limit of " + std::to_string(BLOCK_SLOTS)};
    if (pot.nsplines() > MAX_SPLINES) throw Failure{MZ_ERR_RANGE, "too many splines"};
    const int N = db.natoms, NC = db.ncells, ns = pot.nsplines();
    const int64_t Np = db.npairs;

    // ---- host images of the potential structure (the same as mz_create's)
    const PotImage im = pot_image(pot);
    const std::vector<SplineGeom> &geom = im.geom;
    const std::vector<int> &nat = im.nat, &cmap = im.cmap;
    const std::vector<double> &base = im.base;
    const int stride = im.stride, pstride = im.pstride, P = im.P;
    DevPot dp{};
    dp.style = pot.style;
    dp.ntypes = pot.ntypes;
    dp.nsplines = ns;
    dp.tab_stride = stride;
    dp.pow_stride = pstride;
    dp.pair = style_pair(pot.style) ? 1 : 0;
    dp.s_phi = pot.spline_index(G_PHI, 0);
    dp.s_rho = dp.pair ? 0 : pot.spline_index(G_RHO, 0);
    dp.s_U = dp.pair ? 0 : pot.spline_index(G_U, 0);
    dp.s_f = meam ? pot.spline_index(G_F, 0) : 0;
    dp.s_g = meam ? pot.spline_index(G_G, 0) : 0;
    dp.embed_extrap = set->embed_extrap;
    dp.energy_weight = set->energy_weight;
    dp.stress_weight = set->stress_weight;
    dp.omit_pen = set->omit_punishments;
    dp.gmeam = 0;
    dp.npair = pot.ntypes * (pot.ntypes + 1) / 2;

    // ---- host images of the database
    std::vector<int> off32(N + 1), inoff32(N + 1), inslot32(Np), knot32(Np);
    for (int i = 0; i <= N; ++i) {
      off32[i] = (int)db.pair_off[i];
      inoff32[i] = (int)db.in_off[i];
    }
    std::vector<double> ux(Np), uy(Np), uz(Np), sh(3 * Np);
    for (int64_t q = 0; q < Np; ++q) {
      inslot32[q] = (int)db.in_slot[q];
      knot32[q] = packed_knots(db, q);
      ux[q] = db.pair_u[3 * q];
      uy[q] = db.pair_u[3 * q + 1];
      uz[q] = db.pair_u[3 * q + 2];
      for (int k = 0; k < 3; ++k) sh[k * Np + q] = db.pair_shift[db.nfun * q + k];
    }
    std::vector<int> blk(1, 0);
    {
      int slots = 0, atoms = 0;
      for (int i = 0; i < N; ++i) {
        const int n = (int)(db.pair_off[i + 1] - db.pair_off[i]);
        if (atoms > 0 && (slots + n > BLOCK_SLOTS || atoms + 1 > BLOCK_ATOMS)) {
          blk.push_back(i);
          slots = 0;
          atoms = 0;
        }
        slots += n;
        atoms += 1;
      }
      blk.push_back(N);
    }
    const int nblocks = (int)blk.size() - 1;

    // ---- placement inside the scratch array (size check before any device work)
    Carve cv;
    const size_t o_params = cv.take<double>(P), o_tabs = cv.take<double>(stride), o_ptabs = cv.take<double>(pstride),
                 o_base = cv.take<double>(stride), o_cmap = cv.take<int>(stride), o_nat = cv.take<int>(2 * ns),
                 o_geom = cv.take<SplineGeom>(ns);
    const size_t o_atom0 = cv.take<int>(NC + 1), o_vol = cv.take<double>(NC), o_w = cv.take<double>(NC),
                 o_ew = cv.take<double>(NC), o_sw = cv.take<double>(NC), o_e0 = cv.take<double>(NC),
                 o_s0 = cv.take<double>(6 * (size_t)NC);
    const size_t o_type = cv.take<int>(N), o_cell = cv.take<int>(N), o_f0 = cv.take<double>(3 * (size_t)N),
                 o_off = cv.take<int>(N + 1), o_inoff = cv.take<int>(N + 1), o_inslot = cv.take<int>(Np),
                 o_knot = cv.take<int>(Np), o_nbr = cv.take<int>(Np), o_r = cv.take<double>(Np),
                 o_ux = cv.take<double>(Np), o_uy = cv.take<double>(Np), o_uz = cv.take<double>(Np),
                 o_sh = cv.take<double>(3 * (size_t)Np), o_blk = cv.take<int>(nblocks + 1);
    const size_t o_V = cv.take<double>(3 * (size_t)Np), o_aout = cv.take<double>((size_t)AO_COUNT * N),
                 o_forces = cv.take<double>(3 * (size_t)N), o_cellobj = cv.take<double>(NC),
                 o_obj = cv.take<double>(1);
    if (cv.used > (size_t)MZ_NOALLOC_SCRATCH_BYTES)
      throw Failure{MZ_ERR_RANGE, "database needs " + std::to_string(cv.used) +
                                      " bytes of scratch; the no-allocation entry point holds " +
                                      std::to_string((size_t)MZ_NOALLOC_SCRATCH_BYTES)};

    // ---- per-device set-up: the array's device address, with that device current
    // (the caller's current device is restored on return)
    DeviceGuard dev(set->device);
    unsigned char *base_ptr = nullptr;
    {
      std::lock_guard<std::mutex> lk(g_noalloc_mutex);
      if (!g_noalloc_addr[set->device]) {
        void *p = nullptr;
        ck(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress");
        g_noalloc_addr[set->device] = p;
      }
      base_ptr = static_cast<unsigned char *>(g_noalloc_addr[set->device]);
    }
    const size_t sa = atoms_smem_bytes<double>(ns, pstride);
    ck(cudaFuncSetAttribute(meam ? (const void *)k_atoms<true, double, false> : (const void *)k_atoms<false, double, false>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sa),
       "smem attribute");
    auto put = [&](size_t at, const void *src, size_t bytes) {
      if (bytes) ck(cudaMemcpy(base_ptr + at, src, bytes, cudaMemcpyHostToDevice), "cudaMemcpy H2D");
    };
    put(o_params, params, sizeof(double) * P);
    put(o_base, base.data(), sizeof(double) * stride);
    put(o_cmap, cmap.data(), sizeof(int) * stride);
    put(o_nat, nat.data(), sizeof(int) * 2 * ns);
    put(o_geom, geom.data(), sizeof(SplineGeom) * ns);
    put(o_atom0, db.cell_atom0.data(), sizeof(int) * (NC + 1));
    put(o_vol, db.cell_vol.data(), sizeof(double) * NC);
    put(o_w, db.cell_weight.data(), sizeof(double) * NC);
    put(o_ew, db.cell_eweight.data(), sizeof(double) * NC);
    put(o_sw, db.cell_sweight.data(), sizeof(double) * NC);
    put(o_e0, db.cell_energy0.data(), sizeof(double) * NC);
    put(o_s0, db.cell_stress0.data(), sizeof(double) * 6 * NC);
    put(o_type, db.atom_type.data(), sizeof(int) * N);
    put(o_cell, db.atom_cell.data(), sizeof(int) * N);
    put(o_f0, db.atom_force0.data(), sizeof(double) * 3 * N);
    put(o_off, off32.data(), sizeof(int) * (N + 1));
    put(o_inoff, inoff32.data(), sizeof(int) * (N + 1));
    put(o_inslot, inslot32.data(), sizeof(int) * Np);
    put(o_knot, knot32.data(), sizeof(int) * Np);
    put(o_nbr, db.pair_nbr.data(), sizeof(int) * Np);
    put(o_r, db.pair_r.data(), sizeof(double) * Np);
    put(o_ux, ux.data(), sizeof(double) * Np);
    put(o_uy, uy.data(), sizeof(double) * Np);
    put(o_uz, uz.data(), sizeof(double) * Np);
    put(o_sh, sh.data(), sizeof(double) * 3 * Np);
    put(o_blk, blk.data(), sizeof(int) * (nblocks + 1));
    // Nothing else needs clearing: every slot, atom and cell output below is
    // written by its kernel before it is read.

    auto D = [&](size_t at) { return static_cast<void *>(base_ptr + at); };
    DevDb d{};
    d.ncells = NC;
    d.natoms = N;
    d.npairs = Np;
    d.nblocks = nblocks;
    d.cell_atom0 = (const int *)D(o_atom0);
    d.cell_vol = (const double *)D(o_vol);
    d.cell_w = (const double *)D(o_w);
    d.cell_ew = (const double *)D(o_ew);
    d.cell_sw = (const double *)D(o_sw);
    d.cell_e0 = (const double *)D(o_e0);
    d.cell_s0 = (const double *)D(o_s0);
    d.atom_type = (const int *)D(o_type);
    d.atom_cell = (const int *)D(o_cell);
    d.force0 = (const double *)D(o_f0);
    d.pair_off = (const int *)D(o_off);
    d.in_off = (const int *)D(o_inoff);
    d.in_slot = (const int *)D(o_inslot);
    d.pair_nbr = (const int *)D(o_nbr);
    d.pair_r = (const double *)D(o_r);
    d.pair_ux = (const double *)D(o_ux);
    d.pair_uy = (const double *)D(o_uy);
    d.pair_uz = (const double *)D(o_uz);
    d.pair_shift = (const double *)D(o_sh);
    d.pair_knot = (const int *)D(o_knot);
    d.blk_atom0 = (const int *)D(o_blk);
    const SplineGeom *dgeom = (const SplineGeom *)D(o_geom);
    double *tabs = (double *)D(o_tabs), *ptabs = (double *)D(o_ptabs), *V = (double *)D(o_V),
           *aout = (double *)D(o_aout), *dforces = (double *)D(o_forces), *cellobj = (double *)D(o_cellobj),
           *dobj = (double *)D(o_obj);

    k_prep<<<1, std::max(32, ((ns + 31) / 32) * 32)>>>(1, P, (const double *)D(o_params), (const double *)D(o_base),
                                                       (const int *)D(o_cmap), dgeom, (const int *)D(o_nat), ns,
                                                       stride, tabs, pstride, ptabs);
    ck(cudaGetLastError(), "k_prep launch");
    dim3 ga(nblocks, 1);
    if (meam)
      k_atoms<true, double, false><<<ga, BLOCK_SLOTS, sa>>>(d, dp, dgeom, tabs, ptabs, V, aout, nullptr);
    else
      k_atoms<false, double, false><<<ga, BLOCK_SLOTS, sa>>>(d, dp, dgeom, tabs, ptabs, V, aout, nullptr);
    ck(cudaGetLastError(), "k_atoms launch");
    k_gather<<<dim3((N + 255) / 256, 1), 256>>>(d, V, aout, dforces, nullptr, 0, nullptr);
    ck(cudaGetLastError(), "k_gather launch");
    k_cells<<<dim3((NC + 7) / 8, 1), 256>>>(d, dp, aout, cellobj, nullptr, 0, nullptr, nullptr, nullptr);
    ck(cudaGetLastError(), "k_cells launch");
    k_final<<<1, 256>>>(d, dp, dgeom, tabs, cellobj, dobj, nullptr, 0);
    ck(cudaGetLastError(), "k_final launch");
    ck(cudaMemcpy(obj, dobj, sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy D2H");
    if (forces) ck(cudaMemcpy(forces, dforces, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost), "cudaMemcpy D2H");
  });
}
