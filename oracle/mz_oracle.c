/* TEST ORACLE -- see mz_oracle.h.  CPU restatement of the reference
 * objective used only to check the CUDA evaluator.  Compiled with
 * -ffp-contract=off so its arithmetic rounds like the reference's parity
 * build (oracle/Makefile). */
#include "mz_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define DUMMY_WEIGHT 100.0 /* PotPair::DUMMY_WEIGHT, pot_pair.h:39 */

typedef struct {
  int n, quintic;
  double step, invstep;
  double *x, *y, *ypp, *yp4;
  double grad[2], grad2[2];
  int nat[2];
} sp_t;

/* Spline5Eq::refresh_basis (spline5eq.cpp:209-293): the 2n x 2n system for
 * h^2 y'' and -h^4 y'''', solved here by Gaussian elimination with partial
 * pivoting (the reference calls LAPACK dgesv; the solutions agree to
 * rounding). */
static void sp_refresh5(sp_t *s) {
  const int n = s->n, m = 2 * n;
  double *A = (double *)calloc((size_t)m * m, sizeof(double)), *b = (double *)calloc(m, sizeof(double));
  const double *y = s->y, step = s->step, inv = s->invstep;
  int i, k, r, c;
#define AA(r, c) A[(size_t)(r) * m + (c)]
  for (i = 1; i < n - 1; ++i) {
    AA(i, i - 1) = 1. / 12; AA(i, i) = 10. / 12; AA(i, i + 1) = 1. / 12;
    AA(i, n + i - 1) = 1. / 180; AA(i, n + i) = -1. / 90; AA(i, n + i + 1) = 1. / 180;
    AA(n + i, i - 1) = 1.; AA(n + i, i) = -2.; AA(n + i, i + 1) = 1.;
    AA(n + i, n + i - 1) = 1. / 6; AA(n + i, n + i) = 2. / 3; AA(n + i, n + i + 1) = 1. / 6;
    b[i] = y[i + 1] - 2 * y[i] + y[i - 1];
  }
  if (s->nat[0]) {
    AA(0, 0) = -1.; AA(0, 1) = 1.; AA(0, n) = 1. / 3; AA(0, n + 1) = 1. / 6; b[0] = 0.;
    AA(n, n) = 1.; b[n] = 0.;
  } else {
    AA(0, 0) = 1. / 3; AA(0, 1) = 1. / 6; AA(0, n) = 1. / 45; AA(0, n + 1) = 7. / 360;
    b[0] = y[1] - y[0] - s->grad[0] * step;
    AA(n, 0) = 1.; b[n] = s->grad2[0] * (step * step);
  }
  if (s->nat[1]) {
    AA(n - 1, n - 2) = -1.; AA(n - 1, n - 1) = 1.; AA(n - 1, 2 * n - 2) = -1. / 6; AA(n - 1, 2 * n - 1) = -1. / 3;
    b[n - 1] = 0.;
    AA(2 * n - 1, 2 * n - 1) = 1.; b[2 * n - 1] = 0.;
  } else {
    AA(n - 1, n - 2) = -1. / 6; AA(n - 1, n - 1) = -1. / 3; AA(n - 1, 2 * n - 2) = -7. / 360;
    AA(n - 1, 2 * n - 1) = -1. / 45;
    b[n - 1] = y[n - 1] - y[n - 2] - s->grad[1] * step;
    AA(2 * n - 1, n - 1) = 1.; b[2 * n - 1] = s->grad2[1] * (step * step);
  }
  for (k = 0; k < m; ++k) {
    int p = k;
    for (r = k + 1; r < m; ++r)
      if (fabs(AA(r, k)) > fabs(AA(p, k))) p = r;
    if (p != k) {
      for (c = 0; c < m; ++c) { double t = AA(k, c); AA(k, c) = AA(p, c); AA(p, c) = t; }
      { double t = b[k]; b[k] = b[p]; b[p] = t; }
    }
    if (AA(k, k) == 0.0) continue;
    for (r = k + 1; r < m; ++r) {
      double f = AA(r, k) / AA(k, k);
      if (f == 0.0) continue;
      for (c = k + 1; c < m; ++c) AA(r, c) -= f * AA(k, c);
      b[r] -= f * b[k];
    }
  }
  for (k = m - 1; k >= 0; --k) {
    double acc = b[k];
    for (c = k + 1; c < m; ++c) acc -= AA(k, c) * b[c];
    b[k] = AA(k, k) != 0.0 ? acc / AA(k, k) : 0.0;
  }
#undef AA
  for (i = 0; i < n; ++i) {
    s->ypp[i] = b[i] * (inv * inv);
    s->yp4[i] = -b[n + i] * (inv * inv * inv * inv);
  }
  free(A);
  free(b);
}

/* Spline3Eq::set_spline (spline3eq.cpp:354-370) + coefficients in
 * Spline::coeff / Spline3Eq::bc_coeff order (spline.cpp:105-114,
 * spline3eq.cpp:376-382) + Spline3Eq::refresh_basis (spline3eq.cpp:192-225). */
static void sp_setup(sp_t *s, const mzo_spline *in, const double *coeffs, int *ci, int ncoeff) {
  int n = in->nknots, i, k;
  s->n = n;
  s->quintic = in->quintic;
  s->x = (double *)malloc(sizeof(double) * n);
  s->y = (double *)malloc(sizeof(double) * n);
  s->ypp = (double *)malloc(sizeof(double) * n);
  s->yp4 = (double *)calloc(n, sizeof(double));
  s->step = (in->right - in->left) / (n - 1);
  s->invstep = 1. / s->step;
  s->x[0] = in->left;
  s->x[n - 1] = in->right;
  for (i = 1; i < n - 1; ++i) s->x[i] = in->left + s->step * i;
  for (k = 0; k < n; ++k) s->y[k] = in->y[k];
  s->grad[0] = in->grad[0];
  s->grad[1] = in->grad[1];
  s->grad2[0] = in->grad2[0];
  s->grad2[1] = in->grad2[1];
  s->nat[0] = in->nat[0];
  s->nat[1] = in->nat[1];
  if (coeffs) {
    /* Potential::coeff's walk: free knots, then per free end its slope and
     * (spline5eq, Spline5Eq::bc_coeff spline5eq.cpp:459-468) its y''; only
     * the first get_ncoeff() entries of the walk are coefficients */
    for (k = 0; k < n; ++k)
      if (!in->y_fixed[k] && *ci < ncoeff) s->y[k] = coeffs[(*ci)++];
    for (i = 0; i < 2; ++i)
      if (!in->grad_fixed[i] && !in->nat[i]) {
        if (*ci < ncoeff) s->grad[i] = coeffs[(*ci)++];
        if (s->quintic && *ci < ncoeff) s->grad2[i] = coeffs[(*ci)++];
      }
  }
  if (s->quintic) {
    sp_refresh5(s);
    return;
  }
  {
    double p, qn, un;
    double *u = (double *)calloc(n, sizeof(double));
    double *ypp = s->ypp, *y = s->y, invstep = s->invstep;
    if (s->nat[0]) {
      ypp[0] = 0;
    } else {
      ypp[0] = -0.5;
      u[0] = (3.0 * invstep) * ((y[1] - y[0]) * invstep - s->grad[0]);
    }
    for (i = 1; i < n - 1; ++i) {
      p = 0.5 * ypp[i - 1] + 2.0;
      ypp[i] = (-0.5) / p;
      u[i] = (y[i + 1] - y[i]) * invstep - (y[i] - y[i - 1]) * invstep;
      u[i] = (6.0 * u[i] * 0.5 * invstep - 0.5 * u[i - 1]) / p;
    }
    if (s->nat[1]) {
      qn = un = 0.0;
    } else {
      qn = 0.5;
      un = (3.0 * invstep) * (s->grad[1] - (y[n - 1] - y[n - 2]) * invstep);
    }
    ypp[n - 1] = (un - qn * u[n - 2]) / (qn * ypp[n - 2] + 1.0);
    for (k = n - 2; k >= 0; --k) ypp[k] = ypp[k] * ypp[k + 1] + u[k];
    free(u);
  }
}

static void sp_free(sp_t *s) {
  free(s->x);
  free(s->y);
  free(s->ypp);
  free(s->yp4);
}

/* Spline::get_knotshift (spline.cpp:74-99) */
static int sp_knotshift(const sp_t *s, double r, double *shift) {
  int knot = -1;
  if (r < s->x[s->n - 1] * (1. + 1.e-8)) {
    int klo = 0, khi = s->n - 1;
    while (khi - klo > 1) {
      int k = (khi + klo) >> 1;
      if (s->x[k] > r) khi = k;
      else klo = k;
    }
    knot = klo;
    *shift = (r - s->x[klo]) / (s->x[khi] - s->x[klo]);
  }
  return knot;
}

/* Spline5Eq::splint_comb(int, double, double*) (spline5eq.h:110-127) */
static double sp_comb_k5(const sp_t *s, int knot, double shift, double *grad) {
  double a = 1.0 - shift, h = s->step;
  double p1 = s->y[knot], d21 = s->ypp[knot], d41 = s->yp4[knot];
  double p2 = s->y[knot + 1], d22 = s->ypp[knot + 1], d42 = s->yp4[knot + 1];
  *grad = (p2 - p1) * s->invstep + ((3 * shift * shift - 1) * d22 - (3 * a * a - 1) * d21) * h / 6.0 +
          ((15 * shift * shift * shift * shift - 30 * shift * shift + 7) * d42 -
           (15 * a * a * a * a - 30 * a * a + 7) * d41) * (h * h * h) / 360.0;
  return a * p1 + shift * p2 + ((a * a * a - a) * d21 + (shift * shift * shift - shift) * d22) * (h * h) / 6.0 +
         ((3 * a * a * a * a * a - 10 * a * a * a + 7 * a) * d41 +
          (3 * shift * shift * shift * shift * shift - 10 * shift * shift * shift + 7 * shift) * d42) *
             (h * h * h * h) / 360.0;
}

/* Spline3Eq::splint_comb(int, double, double*) (spline3eq.h:110-122) */
static double sp_comb_k(const sp_t *s, int knot, double shift, double *grad) {
  if (s->quintic) return sp_comb_k5(s, knot, shift, grad);
  double a = 1.0 - shift;
  double p1 = s->y[knot], d21 = s->ypp[knot];
  double p2 = s->y[knot + 1], d22 = s->ypp[knot + 1];
  *grad = (p2 - p1) * s->invstep + ((3 * shift * shift - 1) * d22 - (3 * a * a - 1) * d21) * s->step / 6.0;
  return a * p1 + shift * p2 + ((a * a * a - a) * d21 + (shift * shift * shift - shift) * d22) * s->step * s->step / 6.0;
}

/* Spline3Eq::splint_comb(double, double*) (spline3eq.h:204-236) */
static double sp_comb_x(const sp_t *s, double r, double *grad) {
  int n = s->n, k;
  double dr, b, a, p1, d21, p2, d22;
  if (s->quintic) { /* Spline5Eq::splint_comb(double, double*) (spline5eq.h:226-255) */
    if (r < s->x[0]) {
      *grad = s->grad[0] + s->grad2[0] * (r - s->x[0]);
      return s->y[0] + s->grad[0] * (r - s->x[0]) + 0.5 * s->grad2[0] * (r - s->x[0]) * (r - s->x[0]);
    } else if (r > s->x[n - 1]) {
      *grad = s->grad[1] + s->grad2[1] * (r - s->x[n - 1]);
      return s->y[n - 1] + s->grad[1] * (r - s->x[n - 1]) + 0.5 * s->grad2[1] * (r - s->x[n - 1]) * (r - s->x[n - 1]);
    }
    dr = r - s->x[0];
    if (dr < 0) k = 0;
    else {
      k = (int)(dr * s->invstep);
      if (k >= n - 1) k = n - 2;
    }
    b = (dr - k * s->step) * s->invstep;
    return sp_comb_k5(s, k, b, grad);
  }
  if (r < s->x[0]) {
    *grad = s->grad[0];
    return s->y[0] + s->grad[0] * (r - s->x[0]);
  } else if (r > s->x[n - 1]) {
    *grad = s->grad[1];
    return s->y[n - 1] + s->grad[1] * (r - s->x[n - 1]);
  }
  dr = r - s->x[0];
  if (dr < 0) k = 0;
  else {
    k = (int)(dr * s->invstep);
    if (k >= n - 1) k = n - 2;
  }
  b = (dr - k * s->step) * s->invstep;
  a = 1.0 - b;
  p1 = s->y[k];
  d21 = s->ypp[k];
  p2 = s->y[k + 1];
  d22 = s->ypp[k + 1];
  *grad = (p2 - p1) * s->invstep + ((3 * (b * b) - 1) * d22 - (3 * (a * a) - 1) * d21) * s->step / 6.0;
  return a * p1 + b * p2 + ((a * a * a - a) * d21 + (b * b * b - b) * d22) * (s->step * s->step) / 6.0;
}

static int pair_ij(int nt, int ti, int tj) {
  return (ti <= tj) ? ti * nt + tj - (ti * (ti + 1)) / 2 : tj * nt + ti - (tj * (tj + 1)) / 2;
}

int mzo_ncoeff(const mzo_pot *pot) {
  int n = 0, s, k, e;
  for (s = 0; s < pot->nsplines; ++s) {
    const mzo_spline *sp = &pot->splines[s];
    for (k = 0; k < sp->nknots; ++k) n += sp->y_fixed[k] ? 0 : 1;
    for (e = 0; e < 2; ++e) n += (!sp->grad_fixed[e] && !sp->nat[e]) ? 1 : 0;
  }
  return n;
}

int mzo_esize(const mzo_db *db, const mzo_pot *pot) {
  /* MEAM: one f punishment; GMEAM: one per f spline (pot_gmeam_spline.cpp:173-178); EAM: one per type;
   * pair/spline: neither density constraints nor punishments (pot_pair_spline.cpp:133) */
  if (pot->style == 3) return 7 * db->ncells + 3 * db->natoms;
  /* JMEAM: f and p magnitudes; JMEAM2: f, p and p2 (pot_jmeam_spline.cpp:286-299) */
  if (pot->style == 4 || pot->style == 5) return 8 * db->ncells + 3 * db->natoms + (pot->style == 4 ? 2 : 3);
  return 8 * db->ncells + 3 * db->natoms +
         (pot->style == 1 ? 1 : pot->style == 2 ? pot->ntypes * (pot->ntypes + 1) / 2 : pot->ntypes);
}

double mzo_objective(const mzo_db *db, const mzo_pot *pot, const double *coeffs, double *errvec_out,
                     double *forces_out, double *energy_out, double *stress_out, double *dens_out) {
  const int meam = pot->style == 1 || pot->style == 2 || pot->style == 4 || pot->style == 5;
  const int gmeam = pot->style == 2, pairpot = pot->style == 3;
  const int nj = pot->style == 4 ? 1 : pot->style == 5 ? 2 : 0; /* (p, q) pairs of JMEAM / JMEAM2 */
  const int nf = db->nfun;
  const int nt = pot->ntypes, npair = nt * (nt + 1) / 2;
  const int N = db->natoms, NC = db->ncells;
  int s, ci = 0, i;
  sp_t *sp = (sp_t *)malloc(sizeof(sp_t) * pot->nsplines);
  const int P = mzo_ncoeff(pot);
  for (s = 0; s < pot->nsplines; ++s) sp_setup(&sp[s], &pot->splines[s], coeffs, &ci, P);
  const sp_t *phi = sp, *rho = pairpot ? NULL : sp + npair, *U = pairpot ? NULL : sp + npair + nt;
  const sp_t *ff = meam ? sp + npair + 2 * nt : NULL, *gg = meam ? sp + 2 * npair + 2 * nt : NULL;
  /* JMEAM groups after g: p (Pair_ij), q (Triplet_i) [, p2, q2] (pot_jmeam.cpp:31-45) */
  const sp_t *pp[2] = {NULL, NULL}, *qq[2] = {NULL, NULL};
  int m;
  for (m = 0; m < nj; ++m) {
    pp[m] = sp + 2 * npair + 3 * nt + m * (npair + nt);
    qq[m] = pp[m] + npair;
  }

  /* initialize_compute (potential.cpp:388-408) */
  double *energy = (double *)calloc(NC, sizeof(double));
  double *stress = (double *)calloc(6 * (size_t)NC, sizeof(double));
  double *force = (double *)calloc(3 * (size_t)N, sizeof(double));
  double *constraint = (double *)calloc(NC, sizeof(double));
  int maxrow = 0;
  for (i = 0; i < N; ++i) {
    int n = (int)(db->pair_off[i + 1] - db->pair_off[i]);
    if (n > maxrow) maxrow = n;
  }
  double *drho = (double *)calloc(maxrow + 1, sizeof(double));
  double *fv = (double *)calloc(maxrow + 1, sizeof(double));
  double *dfv = (double *)calloc(maxrow + 1, sizeof(double));
  double *pv = (double *)calloc(2 * (size_t)(maxrow + 1), sizeof(double));
  double *dpv = (double *)calloc(2 * (size_t)(maxrow + 1), sizeof(double));
  size_t maxtrip = (size_t)maxrow * (maxrow > 0 ? maxrow - 1 : 0) / 2 + 1;
  double *tq = (double *)malloc(sizeof(double) * 2 * maxtrip), *tdq = (double *)malloc(sizeof(double) * 2 * maxtrip);
  int *tj_ = (int *)malloc(sizeof(int) * maxtrip), *tk_ = (int *)malloc(sizeof(int) * maxtrip);
  double *tg = (double *)malloc(sizeof(double) * maxtrip), *tdg = (double *)malloc(sizeof(double) * maxtrip);
  double *tcos = (double *)malloc(sizeof(double) * maxtrip);

  /* loop over atoms (pot_meam_spline.cpp:143-270) */
  for (i = 0; i < N; ++i) {
    const int cell = db->atom_cell[i], ti = db->atom_type[i];
    const int64_t p0 = db->pair_off[i];
    const int n = (int)(db->pair_off[i + 1] - p0);
    double *Fi = force + 3 * (size_t)i, *S = stress + 6 * (size_t)cell;
    double rho_val = 0.0, dF = 0.0;
    int p, ntrip = 0, t;
    for (p = 0; p < n; ++p) {
      const int64_t q = p0 + p;
      const int j = db->pair_nbr[q], tj = db->atom_type[j];
      const double *u = db->pair_u + 3 * q, r = db->pair_r[q];
      const int kphi = db->pair_knot[nf * q], krho = db->pair_knot[nf * q + 1], kf = db->pair_knot[nf * q + 2];
      double *Fj = force + 3 * (size_t)j;
      if (kphi != -1) {
        double phigrad, tmp[3], tr[3], phival;
        if (pairpot) {
          /* each pair once; half for an image of atom i itself (pot_pair_spline.cpp:100-113) */
          phival = sp_comb_k(&phi[pair_ij(nt, ti, tj)], kphi, db->pair_shift[nf * q], &phigrad);
          if (j == i) {
            phival *= 0.5;
            phigrad *= 0.5;
          }
        } else {
          phival = 0.5 * sp_comb_k(&phi[pair_ij(nt, ti, tj)], kphi, db->pair_shift[nf * q], &phigrad);
          phigrad *= 0.5;
        }
        energy[cell] += phival;
        tmp[0] = u[0] * phigrad; tmp[1] = u[1] * phigrad; tmp[2] = u[2] * phigrad;
        Fi[0] += tmp[0]; Fi[1] += tmp[1]; Fi[2] += tmp[2];
        Fj[0] -= tmp[0]; Fj[1] -= tmp[1]; Fj[2] -= tmp[2];
        tr[0] = tmp[0] * r; tr[1] = tmp[1] * r; tr[2] = tmp[2] * r;
        /* Stress operator& (stress.h:134-137) */
        S[0] -= u[0] * tr[0]; S[1] -= u[1] * tr[1]; S[2] -= u[2] * tr[2];
        S[3] -= u[0] * tr[1]; S[4] -= u[1] * tr[2]; S[5] -= u[2] * tr[0];
      }
      if (!pairpot && krho != -1) rho_val += sp_comb_k(&rho[tj], krho, db->pair_shift[nf * q + 1], &drho[p]);
      else drho[p] = 0.0;
      if (meam) {
        if (kf != -1) fv[p] = sp_comb_k(&ff[pair_ij(nt, ti, tj)], kf, db->pair_shift[nf * q + 2], &dfv[p]);
        else fv[p] = dfv[p] = 0.0;
      }
      for (m = 0; m < nj; ++m) { /* p (p2): pot_jmeam_spline.cpp:196-202 */
        const int kp = db->pair_knot[nf * q + 3 + m];
        if (kp != -1) pv[2 * p + m] = sp_comb_k(&pp[m][pair_ij(nt, ti, tj)], kp, db->pair_shift[nf * q + 3 + m],
                                                &dpv[2 * p + m]);
        else pv[2 * p + m] = dpv[2 * p + m] = 0.0;
      }
    }
    if (meam) {
      /* Config::find_triplets (config.cpp:262-281) with
       * TripletMEAMSpline::check_triplet (triplet_meam_spline.cpp:49-73):
       * every j<k pair whose cos has a g knot. */
      int j, k;
      for (j = 0; j < n - 1; ++j)
        for (k = j + 1; k < n; ++k) {
          /* GMEAM: g of (i; j, k) types, Triplet_i_jk (pot_fns.cpp:166-168) */
          const sp_t *g = gmeam ? &gg[ti * npair + pair_ij(nt, db->atom_type[db->pair_nbr[p0 + j]],
                                                             db->atom_type[db->pair_nbr[p0 + k]])]
                                : &gg[ti];
          const double *uj = db->pair_u + 3 * (p0 + j), *uk = db->pair_u + 3 * (p0 + k);
          double c = uj[0] * uk[0] + uj[1] * uk[1] + uj[2] * uk[2];
          double gs, qs[2];
          int gk = sp_knotshift(g, c, &gs), qk[2] = {-1, -1}, anyq = 0;
          for (m = 0; m < nj; ++m) {
            qk[m] = sp_knotshift(&qq[m][ti], c, &qs[m]);
            anyq |= qk[m] != -1;
          }
          /* TripletJMEAMSpline::check_triplet (triplet_jmeam_spline.cpp:49-86): a
           * triplet when g or q has a knot.  Where one of them has none the
           * reference evaluates that spline at knot -1 (out of its table); here
           * that term is zero. */
          if (gk == -1 && !anyq) continue;
          tj_[ntrip] = j;
          tk_[ntrip] = k;
          tcos[ntrip] = c;
          if (gk != -1) tg[ntrip] = sp_comb_k(g, gk, gs, &tdg[ntrip]);
          else tg[ntrip] = tdg[ntrip] = 0.0;
          for (m = 0; m < nj; ++m) {
            if (qk[m] != -1) tq[2 * ntrip + m] = sp_comb_k(&qq[m][ti], qk[m], qs[m], &tdq[2 * ntrip + m]);
            else tq[2 * ntrip + m] = tdq[2 * ntrip + m] = 0.0;
          }
          rho_val += fv[j] * fv[k] * tg[ntrip];
          /* pot_jmeam_spline.cpp:216-219 */
          for (m = 0; m < nj; ++m) energy[cell] += pv[2 * j + m] * pv[2 * k + m] * tq[2 * ntrip + m];
          ++ntrip;
        }
    }
    if (dens_out) dens_out[i] = rho_val;
    if (pairpot) continue;
    /* embedding (pot_meam_spline.cpp:208-223) */
    {
      const sp_t *Ui = &U[ti];
      const double w = db->cell_weight[cell];
      if (rho_val < Ui->x[0]) {
        double rho_i = Ui->x[0];
        constraint[cell] += w * DUMMY_WEIGHT * 10. * (rho_i - rho_val) * (rho_i - rho_val);
        if (!pot->embed_extrap) rho_val = rho_i;
      } else if (rho_val > Ui->x[Ui->n - 1]) {
        double rho_f = Ui->x[Ui->n - 1];
        constraint[cell] += w * DUMMY_WEIGHT * 10. * (rho_val - rho_f) * (rho_val - rho_f);
        if (!pot->embed_extrap) rho_val = rho_f;
      }
      energy[cell] += sp_comb_x(Ui, rho_val, &dF);
    }
    /* 2nd loop over pairs (pot_meam_spline.cpp:226-237) */
    for (p = 0; p < n; ++p) {
      const int64_t q = p0 + p;
      const int j = db->pair_nbr[q];
      const double *u = db->pair_u + 3 * q, r = db->pair_r[q];
      double *Fj = force + 3 * (size_t)j, tmp[3], tr[3];
      tmp[0] = u[0] * drho[p] * dF; tmp[1] = u[1] * drho[p] * dF; tmp[2] = u[2] * drho[p] * dF;
      Fi[0] += tmp[0]; Fi[1] += tmp[1]; Fi[2] += tmp[2];
      Fj[0] -= tmp[0]; Fj[1] -= tmp[1]; Fj[2] -= tmp[2];
      tr[0] = tmp[0] * r; tr[1] = tmp[1] * r; tr[2] = tmp[2] * r;
      S[0] -= u[0] * tr[0]; S[1] -= u[1] * tr[1]; S[2] -= u[2] * tr[2];
      S[3] -= u[0] * tr[1]; S[4] -= u[1] * tr[2]; S[5] -= u[2] * tr[0];
    }
    /* 2nd loop over triplets (pot_meam_spline.cpp:240-269) */
    for (t = 0; t < ntrip; ++t) {
      const int j = tj_[t], k = tk_[t];
      const int64_t qj = p0 + j, qk = p0 + k;
      const double *uj = db->pair_u + 3 * qj, *uk = db->pair_u + 3 * qk;
      const double rj = db->pair_r[qj], rk = db->pair_r[qk];
      const double invrj = 1.0 / rj, invrk = 1.0 / rk;
      double *Fj = force + 3 * (size_t)db->pair_nbr[qj], *Fk = force + 3 * (size_t)db->pair_nbr[qk];
      double dV3j = tg[t] * dfv[j] * fv[k] * dF;
      double dV3k = tg[t] * fv[j] * dfv[k] * dF;
      double V3 = tdg[t] * fv[j] * fv[k] * dF;
      /* pot_jmeam_spline.cpp:263-265 */
      for (m = 0; m < nj; ++m) {
        dV3j += tq[2 * t + m] * dpv[2 * j + m] * pv[2 * k + m];
        dV3k += tq[2 * t + m] * pv[2 * j + m] * dpv[2 * k + m];
        V3 += tdq[2 * t + m] * pv[2 * j + m] * pv[2 * k + m];
      }
      double vlj = V3 * invrj, vlk = V3 * invrk;
      double vv3j = dV3j - vlj * tcos[t], vv3k = dV3k - vlk * tcos[t];
      double dfj[3], dfk[3];
      int d;
      for (d = 0; d < 3; ++d) {
        dfj[d] = uj[d] * vv3j + uk[d] * vlj;
        dfk[d] = uk[d] * vv3k + uj[d] * vlk;
        Fi[d] += dfj[d] + dfk[d];
        Fj[d] -= dfj[d];
        Fk[d] -= dfk[d];
      }
      for (d = 0; d < 3; ++d) {
        dfj[d] *= rj;
        dfk[d] *= rk;
      }
      S[0] -= uj[0] * dfj[0]; S[1] -= uj[1] * dfj[1]; S[2] -= uj[2] * dfj[2];
      S[3] -= uj[0] * dfj[1]; S[4] -= uj[1] * dfj[2]; S[5] -= uj[2] * dfj[0];
      S[0] -= uk[0] * dfk[0]; S[1] -= uk[1] * dfk[1]; S[2] -= uk[2] * dfk[2];
      S[3] -= uk[0] * dfk[1]; S[4] -= uk[1] * dfk[2]; S[5] -= uk[2] * dfk[0];
    }
  }

  /* accumulate_error (potential.cpp:415-491) */
  const int esize = mzo_esize(db, pot);
  double *ev = (double *)malloc(sizeof(double) * esize);
  double sum = 0.0;
  int c, idx = 0;
  for (c = 0; c < NC; ++c) {
    const int a0 = db->cell_atom0[c], na = db->cell_atom0[c + 1] - a0;
    const double w = db->cell_weight[c];
    int q, a, d;
    energy[c] = energy[c] / na;
    ev[idx] = w * db->cell_eweight[c] * pot->energy_weight * na * (energy[c] - db->cell_energy0[c]);
    sum += ev[idx] * ev[idx];
    ++idx;
    for (q = 0; q < 6; ++q) {
      stress[6 * c + q] = stress[6 * c + q] / db->cell_vol[c];
      ev[idx] = w * db->cell_sweight[c] * pot->stress_weight * (stress[6 * c + q] - db->cell_stress0[6 * c + q]);
      sum += ev[idx] * ev[idx];
      ++idx;
    }
    for (a = a0; a < a0 + na; ++a)
      for (d = 0; d < 3; ++d) {
        ev[idx] = w * (force[3 * a + d] - db->atom_force0[3 * a + d]);
        sum += ev[idx] * ev[idx];
        ++idx;
      }
  }
  for (c = 0; c < NC && !pairpot; ++c) {
    ev[idx] = constraint[c];
    sum += ev[idx] * ev[idx];
    ++idx;
  }
  if (pairpot) {
    /* no punishments */
  } else if (pot->omit_punishments) {
    /* a shard past the first: its punishment entries are zero */
    int q, npen = gmeam ? npair : meam ? 1 + nj : nt;
    for (q = 0; q < npen; ++q) ev[idx++] = 0.0;
  } else if (gmeam) {
    /* pot_gmeam_spline.cpp:173-178: one punishment per f spline */
    int f, k;
    for (f = 0; f < npair; ++f) {
      double m = 0.0;
      for (k = 0; k < ff[f].n; ++k)
        if (fabs(m) < fabs(ff[f].y[k])) m = ff[f].y[k];
      double mag = fabs(m);
      double fe = DUMMY_WEIGHT * 25. * (1.0 - mag) * (1.0 - mag);
      sum += fe * fe;
      ev[idx++] = fe;
    }
  } else if (meam) {
    /* pot_meam_spline.cpp:274-278 with PotFns::get_max_y_mag (pot_fns.cpp:223-234)
     * and Spline::get_max_y_mag (spline.cpp:58-67); JMEAM adds the same for
     * p (and p2), pot_jmeam_spline.cpp:286-299 */
    int grp;
    for (grp = 0; grp <= nj; ++grp) {
      const sp_t *G = grp == 0 ? ff : pp[grp - 1];
      double my = 0.0;
      int f, k;
      for (f = 0; f < npair; ++f) {
        double mm = 0.0;
        for (k = 0; k < G[f].n; ++k)
          if (fabs(mm) < fabs(G[f].y[k])) mm = G[f].y[k];
        if (fabs(my) < fabs(mm)) my = mm;
      }
      double mag = fabs(my);
      double fe = DUMMY_WEIGHT * 25. * (1.0 - mag) * (1.0 - mag);
      sum += fe * fe;
      ev[idx++] = fe;
    }
  } else {
    /* pot_eam_spline.cpp:211-218 */
    int t;
    for (t = 0; t < nt; ++t) {
      double g, mid = 0.5 * (U[t].x[0] + U[t].x[U[t].n - 1]);
      sp_comb_x(&U[t], mid, &g);
      double e = DUMMY_WEIGHT * g;
      sum += e * e;
      ev[idx++] = e;
    }
  }
  if (errvec_out) memcpy(errvec_out, ev, sizeof(double) * esize);
  if (forces_out) memcpy(forces_out, force, sizeof(double) * 3 * (size_t)N);
  if (energy_out) memcpy(energy_out, energy, sizeof(double) * NC);
  if (stress_out) memcpy(stress_out, stress, sizeof(double) * 6 * (size_t)NC);

  free(ev);
  free(tj_); free(tk_); free(tg); free(tdg); free(tcos);
  free(drho); free(fv); free(dfv); free(pv); free(dpv); free(tq); free(tdq);
  free(energy); free(stress); free(force); free(constraint);
  for (s = 0; s < pot->nsplines; ++s) sp_free(&sp[s]);
  free(sp);
  return sum;
}

/* ------------------------------------------------------------------------
 * Tangent-linear restatement: the objective and its exact derivative along
 * one direction of the coefficient vector (forward-mode differentiation of
 * mzo_objective, statement by statement).  Every spline's knot table is
 * linear in its coefficients (Spline3Eq::refresh_basis spline3eq.cpp:192-225
 * and Spline5Eq::refresh_basis spline5eq.cpp:209-293 solve linear systems
 * whose right-hand sides are linear in y and the end derivatives), so the
 * derivative of a spline value at a fixed knot and shift is the value of the
 * "tangent spline" whose coefficients are the direction; at a variable point
 * x(t) the chain rule adds S'(x) x'. */

/* S''(x) of Spline3Eq / Spline5Eq::splint_comb(double, double*)
 * (spline3eq.h:204-236, spline5eq.h:226-255): zero (cubic) or the end y''
 * (quintic) on the extrapolated ranges. */
static double sp_second_x(const sp_t *s, double r) {
  int n = s->n, k;
  double dr, b, a;
  if (r < s->x[0]) return s->quintic ? s->grad2[0] : 0.0;
  if (r > s->x[n - 1]) return s->quintic ? s->grad2[1] : 0.0;
  dr = r - s->x[0];
  if (dr < 0) k = 0;
  else {
    k = (int)(dr * s->invstep);
    if (k >= n - 1) k = n - 2;
  }
  b = (dr - k * s->step) * s->invstep;
  a = 1.0 - b;
  if (!s->quintic) return a * s->ypp[k] + b * s->ypp[k + 1];
  /* d^2/dx^2 of the quintic piece of sp_comb_k5 */
  return a * s->ypp[k] + b * s->ypp[k + 1] +
         ((a * a * a - a) * s->yp4[k] + (b * b * b - b) * s->yp4[k + 1]) * (s->step * s->step) / 6.0;
}

/* The tangent spline of `in` along `dir`: zero knots and end values, the
 * direction's entries at the coefficient positions, refreshed. */
static void sp_setup_tangent(sp_t *t, const mzo_spline *in, const double *dir, int *ci, int ncoeff) {
  mzo_spline z = *in;
  double *zy = (double *)calloc(in->nknots, sizeof(double));
  z.y = zy;
  z.grad[0] = z.grad[1] = 0.0;
  z.grad2[0] = z.grad2[1] = 0.0;
  sp_setup(t, &z, dir, ci, ncoeff);
  free(zy);
}

/* value and derivative of a spline at a fixed knot and shift, and their tangents */
static double tcomb_k(const sp_t *s, const sp_t *ts, int knot, double shift, double *grad, double *tval,
                      double *tgrad) {
  *tval = sp_comb_k(ts, knot, shift, tgrad);
  return sp_comb_k(s, knot, shift, grad);
}

double mzo_objective_tangent(const mzo_db *db, const mzo_pot *pot, const double *coeffs, const double *dir,
                             double *dobj) {
  const int meam = pot->style == 1 || pot->style == 2 || pot->style == 4 || pot->style == 5;
  const int gmeam = pot->style == 2, pairpot = pot->style == 3;
  const int nj = pot->style == 4 ? 1 : pot->style == 5 ? 2 : 0;
  const int nf = db->nfun;
  const int nt = pot->ntypes, npair = nt * (nt + 1) / 2;
  const int N = db->natoms, NC = db->ncells;
  int s, ci = 0, cj = 0, i, m, d;
  sp_t *sp = (sp_t *)malloc(sizeof(sp_t) * pot->nsplines);
  sp_t *tsp = (sp_t *)malloc(sizeof(sp_t) * pot->nsplines);
  const int P = mzo_ncoeff(pot);
  for (s = 0; s < pot->nsplines; ++s) {
    sp_setup(&sp[s], &pot->splines[s], coeffs, &ci, P);
    sp_setup_tangent(&tsp[s], &pot->splines[s], dir, &cj, P);
  }
#define SPL(base, idx) (&sp[(base) + (idx)])
#define TSPL(base, idx) (&tsp[(base) + (idx)])
  const int o_phi = 0, o_rho = npair, o_U = npair + nt, o_f = npair + 2 * nt, o_g = 2 * npair + 2 * nt;
  int o_p[2] = {0, 0}, o_q[2] = {0, 0};
  for (m = 0; m < nj; ++m) {
    o_p[m] = 2 * npair + 3 * nt + m * (npair + nt);
    o_q[m] = o_p[m] + npair;
  }

  double *energy = (double *)calloc(NC, sizeof(double)), *tenergy = (double *)calloc(NC, sizeof(double));
  double *stress = (double *)calloc(6 * (size_t)NC, sizeof(double));
  double *tstress = (double *)calloc(6 * (size_t)NC, sizeof(double));
  double *force = (double *)calloc(3 * (size_t)N, sizeof(double));
  double *tforce = (double *)calloc(3 * (size_t)N, sizeof(double));
  double *constraint = (double *)calloc(NC, sizeof(double)), *tconstraint = (double *)calloc(NC, sizeof(double));
  int maxrow = 0;
  for (i = 0; i < N; ++i) {
    int n = (int)(db->pair_off[i + 1] - db->pair_off[i]);
    if (n > maxrow) maxrow = n;
  }
  const size_t R1 = (size_t)maxrow + 1;
  double *drho = (double *)calloc(R1, sizeof(double)), *tdrho = (double *)calloc(R1, sizeof(double));
  double *fv = (double *)calloc(R1, sizeof(double)), *tfv = (double *)calloc(R1, sizeof(double));
  double *dfv = (double *)calloc(R1, sizeof(double)), *tdfv = (double *)calloc(R1, sizeof(double));
  double *pv = (double *)calloc(2 * R1, sizeof(double)), *tpv = (double *)calloc(2 * R1, sizeof(double));
  double *dpv = (double *)calloc(2 * R1, sizeof(double)), *tdpv = (double *)calloc(2 * R1, sizeof(double));
  size_t maxtrip = (size_t)maxrow * (maxrow > 0 ? maxrow - 1 : 0) / 2 + 1;
  double *tq = (double *)malloc(sizeof(double) * 2 * maxtrip), *tdq = (double *)malloc(sizeof(double) * 2 * maxtrip);
  double *ttq = (double *)malloc(sizeof(double) * 2 * maxtrip), *ttdq = (double *)malloc(sizeof(double) * 2 * maxtrip);
  int *tj_ = (int *)malloc(sizeof(int) * maxtrip), *tk_ = (int *)malloc(sizeof(int) * maxtrip);
  double *tg = (double *)malloc(sizeof(double) * maxtrip), *tdg = (double *)malloc(sizeof(double) * maxtrip);
  double *ttg = (double *)malloc(sizeof(double) * maxtrip), *ttdg = (double *)malloc(sizeof(double) * maxtrip);
  double *tcos = (double *)malloc(sizeof(double) * maxtrip);

  for (i = 0; i < N; ++i) {
    const int cell = db->atom_cell[i], ti = db->atom_type[i];
    const int64_t p0 = db->pair_off[i];
    const int n = (int)(db->pair_off[i + 1] - p0);
    double *Fi = force + 3 * (size_t)i, *S = stress + 6 * (size_t)cell;
    double *tFi = tforce + 3 * (size_t)i, *tS = tstress + 6 * (size_t)cell;
    double rho_val = 0.0, trho = 0.0, dF = 0.0, tdF = 0.0;
    int p, ntrip = 0, t;
    for (p = 0; p < n; ++p) {
      const int64_t q = p0 + p;
      const int j = db->pair_nbr[q], tj = db->atom_type[j];
      const double *u = db->pair_u + 3 * q, r = db->pair_r[q];
      const int kphi = db->pair_knot[nf * q], krho = db->pair_knot[nf * q + 1], kf = db->pair_knot[nf * q + 2];
      double *Fj = force + 3 * (size_t)j, *tFj = tforce + 3 * (size_t)j;
      if (kphi != -1) {
        const int pij = pair_ij(nt, ti, tj);
        double phigrad, tphigrad, tphival, phival, tmp[3], ttmp[3];
        phival = tcomb_k(SPL(o_phi, pij), TSPL(o_phi, pij), kphi, db->pair_shift[nf * q], &phigrad, &tphival,
                         &tphigrad);
        if (!pairpot || j == i) {
          phival *= 0.5; phigrad *= 0.5; tphival *= 0.5; tphigrad *= 0.5;
        }
        energy[cell] += phival;
        tenergy[cell] += tphival;
        for (d = 0; d < 3; ++d) {
          tmp[d] = u[d] * phigrad;
          ttmp[d] = u[d] * tphigrad;
          Fi[d] += tmp[d]; Fj[d] -= tmp[d];
          tFi[d] += ttmp[d]; tFj[d] -= ttmp[d];
        }
        S[0] -= u[0] * (tmp[0] * r); S[1] -= u[1] * (tmp[1] * r); S[2] -= u[2] * (tmp[2] * r);
        S[3] -= u[0] * (tmp[1] * r); S[4] -= u[1] * (tmp[2] * r); S[5] -= u[2] * (tmp[0] * r);
        tS[0] -= u[0] * (ttmp[0] * r); tS[1] -= u[1] * (ttmp[1] * r); tS[2] -= u[2] * (ttmp[2] * r);
        tS[3] -= u[0] * (ttmp[1] * r); tS[4] -= u[1] * (ttmp[2] * r); tS[5] -= u[2] * (ttmp[0] * r);
      }
      if (!pairpot && krho != -1) {
        double tv;
        rho_val += tcomb_k(SPL(o_rho, tj), TSPL(o_rho, tj), krho, db->pair_shift[nf * q + 1], &drho[p], &tv,
                           &tdrho[p]);
        trho += tv;
      } else {
        drho[p] = tdrho[p] = 0.0;
      }
      if (meam) {
        const int pij = pair_ij(nt, ti, tj);
        if (kf != -1)
          fv[p] = tcomb_k(SPL(o_f, pij), TSPL(o_f, pij), kf, db->pair_shift[nf * q + 2], &dfv[p], &tfv[p], &tdfv[p]);
        else
          fv[p] = dfv[p] = tfv[p] = tdfv[p] = 0.0;
      }
      for (m = 0; m < nj; ++m) {
        const int kp = db->pair_knot[nf * q + 3 + m], pij = pair_ij(nt, ti, tj);
        if (kp != -1)
          pv[2 * p + m] = tcomb_k(SPL(o_p[m], pij), TSPL(o_p[m], pij), kp, db->pair_shift[nf * q + 3 + m],
                                  &dpv[2 * p + m], &tpv[2 * p + m], &tdpv[2 * p + m]);
        else
          pv[2 * p + m] = dpv[2 * p + m] = tpv[2 * p + m] = tdpv[2 * p + m] = 0.0;
      }
    }
    if (meam) {
      int j, k;
      for (j = 0; j < n - 1; ++j)
        for (k = j + 1; k < n; ++k) {
          const int gi = gmeam ? ti * npair + pair_ij(nt, db->atom_type[db->pair_nbr[p0 + j]],
                                                      db->atom_type[db->pair_nbr[p0 + k]])
                               : ti;
          const sp_t *g = SPL(o_g, gi), *tgs = TSPL(o_g, gi);
          const double *uj = db->pair_u + 3 * (p0 + j), *uk = db->pair_u + 3 * (p0 + k);
          double c = uj[0] * uk[0] + uj[1] * uk[1] + uj[2] * uk[2];
          double gsh, qs[2];
          int gk = sp_knotshift(g, c, &gsh), qk[2] = {-1, -1}, anyq = 0;
          for (m = 0; m < nj; ++m) {
            qk[m] = sp_knotshift(SPL(o_q[m], ti), c, &qs[m]);
            anyq |= qk[m] != -1;
          }
          if (gk == -1 && !anyq) continue;
          tj_[ntrip] = j;
          tk_[ntrip] = k;
          tcos[ntrip] = c;
          if (gk != -1) tg[ntrip] = tcomb_k(g, tgs, gk, gsh, &tdg[ntrip], &ttg[ntrip], &ttdg[ntrip]);
          else tg[ntrip] = tdg[ntrip] = ttg[ntrip] = ttdg[ntrip] = 0.0;
          for (m = 0; m < nj; ++m) {
            const size_t e = 2 * (size_t)ntrip + m;
            if (qk[m] != -1)
              tq[e] = tcomb_k(SPL(o_q[m], ti), TSPL(o_q[m], ti), qk[m], qs[m], &tdq[e], &ttq[e], &ttdq[e]);
            else tq[e] = tdq[e] = ttq[e] = ttdq[e] = 0.0;
          }
          rho_val += fv[j] * fv[k] * tg[ntrip];
          trho += tfv[j] * fv[k] * tg[ntrip] + fv[j] * tfv[k] * tg[ntrip] + fv[j] * fv[k] * ttg[ntrip];
          for (m = 0; m < nj; ++m) {
            const size_t e = 2 * (size_t)ntrip + m;
            energy[cell] += pv[2 * j + m] * pv[2 * k + m] * tq[e];
            tenergy[cell] += tpv[2 * j + m] * pv[2 * k + m] * tq[e] + pv[2 * j + m] * tpv[2 * k + m] * tq[e] +
                             pv[2 * j + m] * pv[2 * k + m] * ttq[e];
          }
          ++ntrip;
        }
    }
    if (pairpot) continue;
    {
      const sp_t *Ui = SPL(o_U, ti), *tUi = TSPL(o_U, ti);
      const double w = db->cell_weight[cell];
      double tUv, tUg;
      if (rho_val < Ui->x[0]) {
        double rho_i = Ui->x[0];
        constraint[cell] += w * DUMMY_WEIGHT * 10. * (rho_i - rho_val) * (rho_i - rho_val);
        tconstraint[cell] += w * DUMMY_WEIGHT * 10. * 2.0 * (rho_i - rho_val) * (-trho);
        if (!pot->embed_extrap) { rho_val = rho_i; trho = 0.0; }
      } else if (rho_val > Ui->x[Ui->n - 1]) {
        double rho_f = Ui->x[Ui->n - 1];
        constraint[cell] += w * DUMMY_WEIGHT * 10. * (rho_val - rho_f) * (rho_val - rho_f);
        tconstraint[cell] += w * DUMMY_WEIGHT * 10. * 2.0 * (rho_val - rho_f) * trho;
        if (!pot->embed_extrap) { rho_val = rho_f; trho = 0.0; }
      }
      energy[cell] += sp_comb_x(Ui, rho_val, &dF);
      tUv = sp_comb_x(tUi, rho_val, &tUg);
      tenergy[cell] += tUv + dF * trho;
      tdF = tUg + sp_second_x(Ui, rho_val) * trho;
    }
    for (p = 0; p < n; ++p) {
      const int64_t q = p0 + p;
      const int j = db->pair_nbr[q];
      const double *u = db->pair_u + 3 * q, r = db->pair_r[q];
      double *Fj = force + 3 * (size_t)j, *tFj = tforce + 3 * (size_t)j, tmp[3], ttmp[3];
      for (d = 0; d < 3; ++d) {
        tmp[d] = u[d] * drho[p] * dF;
        ttmp[d] = u[d] * (tdrho[p] * dF + drho[p] * tdF);
        Fi[d] += tmp[d]; Fj[d] -= tmp[d];
        tFi[d] += ttmp[d]; tFj[d] -= ttmp[d];
      }
      S[0] -= u[0] * (tmp[0] * r); S[1] -= u[1] * (tmp[1] * r); S[2] -= u[2] * (tmp[2] * r);
      S[3] -= u[0] * (tmp[1] * r); S[4] -= u[1] * (tmp[2] * r); S[5] -= u[2] * (tmp[0] * r);
      tS[0] -= u[0] * (ttmp[0] * r); tS[1] -= u[1] * (ttmp[1] * r); tS[2] -= u[2] * (ttmp[2] * r);
      tS[3] -= u[0] * (ttmp[1] * r); tS[4] -= u[1] * (ttmp[2] * r); tS[5] -= u[2] * (ttmp[0] * r);
    }
    for (t = 0; t < ntrip; ++t) {
      const int j = tj_[t], k = tk_[t];
      const int64_t qj = p0 + j, qk = p0 + k;
      const double *uj = db->pair_u + 3 * qj, *uk = db->pair_u + 3 * qk;
      const double rj = db->pair_r[qj], rk = db->pair_r[qk];
      const double invrj = 1.0 / rj, invrk = 1.0 / rk;
      double *Fj = force + 3 * (size_t)db->pair_nbr[qj], *Fk = force + 3 * (size_t)db->pair_nbr[qk];
      double *tFj = tforce + 3 * (size_t)db->pair_nbr[qj], *tFk = tforce + 3 * (size_t)db->pair_nbr[qk];
      double dV3j = tg[t] * dfv[j] * fv[k] * dF;
      double dV3k = tg[t] * fv[j] * dfv[k] * dF;
      double V3 = tdg[t] * fv[j] * fv[k] * dF;
      double tdV3j = ttg[t] * dfv[j] * fv[k] * dF + tg[t] * tdfv[j] * fv[k] * dF + tg[t] * dfv[j] * tfv[k] * dF +
                     tg[t] * dfv[j] * fv[k] * tdF;
      double tdV3k = ttg[t] * fv[j] * dfv[k] * dF + tg[t] * tfv[j] * dfv[k] * dF + tg[t] * fv[j] * tdfv[k] * dF +
                     tg[t] * fv[j] * dfv[k] * tdF;
      double tV3 = ttdg[t] * fv[j] * fv[k] * dF + tdg[t] * tfv[j] * fv[k] * dF + tdg[t] * fv[j] * tfv[k] * dF +
                   tdg[t] * fv[j] * fv[k] * tdF;
      for (m = 0; m < nj; ++m) {
        const size_t e = 2 * (size_t)t + m;
        const double pj = pv[2 * j + m], pk = pv[2 * k + m], dpj = dpv[2 * j + m], dpk = dpv[2 * k + m];
        const double tpj = tpv[2 * j + m], tpk = tpv[2 * k + m], tdpj = tdpv[2 * j + m], tdpk = tdpv[2 * k + m];
        dV3j += tq[e] * dpj * pk;
        dV3k += tq[e] * pj * dpk;
        V3 += tdq[e] * pj * pk;
        tdV3j += ttq[e] * dpj * pk + tq[e] * tdpj * pk + tq[e] * dpj * tpk;
        tdV3k += ttq[e] * pj * dpk + tq[e] * tpj * dpk + tq[e] * pj * tdpk;
        tV3 += ttdq[e] * pj * pk + tdq[e] * tpj * pk + tdq[e] * pj * tpk;
      }
      const double vlj = V3 * invrj, vlk = V3 * invrk, tvlj = tV3 * invrj, tvlk = tV3 * invrk;
      const double vv3j = dV3j - vlj * tcos[t], vv3k = dV3k - vlk * tcos[t];
      const double tvv3j = tdV3j - tvlj * tcos[t], tvv3k = tdV3k - tvlk * tcos[t];
      double dfj[3], dfk[3], tdfj[3], tdfk[3];
      for (d = 0; d < 3; ++d) {
        dfj[d] = uj[d] * vv3j + uk[d] * vlj;
        dfk[d] = uk[d] * vv3k + uj[d] * vlk;
        tdfj[d] = uj[d] * tvv3j + uk[d] * tvlj;
        tdfk[d] = uk[d] * tvv3k + uj[d] * tvlk;
        Fi[d] += dfj[d] + dfk[d];
        Fj[d] -= dfj[d];
        Fk[d] -= dfk[d];
        tFi[d] += tdfj[d] + tdfk[d];
        tFj[d] -= tdfj[d];
        tFk[d] -= tdfk[d];
      }
      for (d = 0; d < 3; ++d) {
        dfj[d] *= rj; dfk[d] *= rk; tdfj[d] *= rj; tdfk[d] *= rk;
      }
      S[0] -= uj[0] * dfj[0]; S[1] -= uj[1] * dfj[1]; S[2] -= uj[2] * dfj[2];
      S[3] -= uj[0] * dfj[1]; S[4] -= uj[1] * dfj[2]; S[5] -= uj[2] * dfj[0];
      S[0] -= uk[0] * dfk[0]; S[1] -= uk[1] * dfk[1]; S[2] -= uk[2] * dfk[2];
      S[3] -= uk[0] * dfk[1]; S[4] -= uk[1] * dfk[2]; S[5] -= uk[2] * dfk[0];
      tS[0] -= uj[0] * tdfj[0]; tS[1] -= uj[1] * tdfj[1]; tS[2] -= uj[2] * tdfj[2];
      tS[3] -= uj[0] * tdfj[1]; tS[4] -= uj[1] * tdfj[2]; tS[5] -= uj[2] * tdfj[0];
      tS[0] -= uk[0] * tdfk[0]; tS[1] -= uk[1] * tdfk[1]; tS[2] -= uk[2] * tdfk[2];
      tS[3] -= uk[0] * tdfk[1]; tS[4] -= uk[1] * tdfk[2]; tS[5] -= uk[2] * tdfk[0];
    }
  }

  /* accumulate_error (potential.cpp:415-491) and its tangent: F = sum e^2, dF = 2 sum e de */
  double sum = 0.0, tsum = 0.0;
  int c;
  for (c = 0; c < NC; ++c) {
    const int a0 = db->cell_atom0[c], na = db->cell_atom0[c + 1] - a0;
    const double w = db->cell_weight[c];
    const double ew = w * db->cell_eweight[c] * pot->energy_weight * na;
    const double sw = w * db->cell_sweight[c] * pot->stress_weight;
    int q, a;
    double e = ew * (energy[c] / na - db->cell_energy0[c]), te = ew * (tenergy[c] / na);
    sum += e * e;
    tsum += 2.0 * e * te;
    for (q = 0; q < 6; ++q) {
      e = sw * (stress[6 * c + q] / db->cell_vol[c] - db->cell_stress0[6 * c + q]);
      te = sw * (tstress[6 * c + q] / db->cell_vol[c]);
      sum += e * e;
      tsum += 2.0 * e * te;
    }
    for (a = a0; a < a0 + na; ++a)
      for (d = 0; d < 3; ++d) {
        e = w * (force[3 * a + d] - db->atom_force0[3 * a + d]);
        te = w * tforce[3 * a + d];
        sum += e * e;
        tsum += 2.0 * e * te;
      }
  }
  for (c = 0; c < NC && !pairpot; ++c) {
    sum += constraint[c] * constraint[c];
    tsum += 2.0 * constraint[c] * tconstraint[c];
  }
  if (pairpot || pot->omit_punishments) {
    /* no punishments */
  } else if (meam) {
    /* signed largest-|y| knot (Spline::get_max_y_mag spline.cpp:58-67 over the
     * group, PotFns::get_max_y_mag pot_fns.cpp:223-234; GMEAM per f spline):
     * fe = 2500 (1 - |m|)^2, dfe = -5000 (1 - |m|) sign(m) dm */
    int grp, ngrp = gmeam ? npair : 1 + nj;
    for (grp = 0; grp < ngrp; ++grp) {
      const int base = gmeam ? o_f + grp : (grp == 0 ? o_f : o_p[grp - 1]);
      const int nspl = gmeam ? 1 : npair;
      double my = 0.0, tmy = 0.0;
      int f, k;
      for (f = 0; f < nspl; ++f) {
        double mm = 0.0, tmm = 0.0;
        for (k = 0; k < sp[base + f].n; ++k)
          if (fabs(mm) < fabs(sp[base + f].y[k])) {
            mm = sp[base + f].y[k];
            tmm = tsp[base + f].y[k];
          }
        if (fabs(my) < fabs(mm)) {
          my = mm;
          tmy = tmm;
        }
      }
      const double mag = fabs(my);
      const double fe = DUMMY_WEIGHT * 25. * (1.0 - mag) * (1.0 - mag);
      const double sg = my > 0 ? 1.0 : (my < 0 ? -1.0 : 0.0);
      const double tfe = DUMMY_WEIGHT * 25. * 2.0 * (1.0 - mag) * (-sg * tmy);
      sum += fe * fe;
      tsum += 2.0 * fe * tfe;
    }
  } else {
    int t;
    for (t = 0; t < nt; ++t) {
      double g, tgv, mid = 0.5 * (sp[o_U + t].x[0] + sp[o_U + t].x[sp[o_U + t].n - 1]);
      sp_comb_x(&sp[o_U + t], mid, &g);
      sp_comb_x(&tsp[o_U + t], mid, &tgv);
      const double e = DUMMY_WEIGHT * g, te = DUMMY_WEIGHT * tgv;
      sum += e * e;
      tsum += 2.0 * e * te;
    }
  }
#undef SPL
#undef TSPL
  if (dobj) *dobj = tsum;
  free(tj_); free(tk_); free(tg); free(tdg); free(ttg); free(ttdg); free(tcos);
  free(drho); free(tdrho); free(fv); free(tfv); free(dfv); free(tdfv);
  free(pv); free(tpv); free(dpv); free(tdpv); free(tq); free(tdq); free(ttq); free(ttdq);
  free(energy); free(tenergy); free(stress); free(tstress); free(force); free(tforce);
  free(constraint); free(tconstraint);
  for (s = 0; s < pot->nsplines; ++s) {
    sp_free(&sp[s]);
    sp_free(&tsp[s]);
  }
  free(sp);
  free(tsp);
  return sum;
}
