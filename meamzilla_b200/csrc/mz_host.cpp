// Host side of the evaluator: potential files, parameter layout, spline
// arithmetic shared with the device tables, configuration files and the
// periodic neighbour-list builder.  Built with -ffp-contract=off (see
// mz_host.hpp).
#include "mz_host.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <stdexcept>
#include <thread>

namespace mzb {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

[[noreturn]] static void fail(int status, const std::string &msg) { throw Failure{status, msg}; }

// ------------------------------------------------------------------ Spline3

void Spline3::set_grid() {
  // Spline3Eq::set_spline (spline3eq.cpp:354-370)
  step = (right - left) / (nknots - 1);
  invstep = 1. / step;
  x.assign(nknots, 0.0);
  x[0] = left;
  x[nknots - 1] = right;
  for (int i = 1; i < nknots - 1; ++i) x[i] = left + step * i;
}

int Spline3::ncoeff() const {
  int n = 0;
  for (int k = 0; k < nknots; ++k) n += y_fixed[k] ? 0 : 1;
  for (int i = 0; i < 2; ++i) n += (!grad_fixed[i] && !nat[i]) ? 1 : 0;
  return n;
}

int Spline3::knotshift(double r, double *shift) const {
  // Spline::get_knotshift (spline.cpp:74-99)
  int knot = -1;
  if (r < x.back() * (1. + 1.e-8)) {
    int klo = 0, khi = nknots - 1;
    while (khi - klo > 1) {
      int k = (khi + klo) >> 1;
      if (x[k] > r) khi = k;
      else klo = k;
    }
    knot = klo;
    double h = x[khi] - x[klo];
    *shift = (r - x[klo]) / h;
  }
  return knot;
}

void Spline3::refresh(std::vector<double> &ypp) const {
  // Tridiagonal solve of Spline3Eq::refresh_basis (spline3eq.cpp:192-225):
  // clamped ends use the end slope, natural ends a zero second derivative.
  const int n = nknots;
  std::vector<double> u(n, 0.0);
  ypp.assign(n, 0.0);
  if (nat[0]) {
    ypp[0] = 0;
  } else {
    ypp[0] = -0.5;
    u[0] = (3.0 * invstep) * ((y[1] - y[0]) * invstep - grad[0]);
  }
  for (int i = 1; i < n - 1; ++i) {
    double p = 0.5 * ypp[i - 1] + 2.0;
    ypp[i] = (-0.5) / p;
    u[i] = (y[i + 1] - y[i]) * invstep - (y[i] - y[i - 1]) * invstep;
    u[i] = (6.0 * u[i] * 0.5 * invstep - 0.5 * u[i - 1]) / p;
  }
  double qn, un;
  if (nat[1]) {
    qn = un = 0.0;
  } else {
    qn = 0.5;
    un = (3.0 * invstep) * (grad[1] - (y[n - 1] - y[n - 2]) * invstep);
  }
  ypp[n - 1] = (un - qn * u[n - 2]) / (qn * ypp[n - 2] + 1.0);
  for (int k = n - 2; k >= 0; --k) ypp[k] = ypp[k] * ypp[k + 1] + u[k];
}

double Spline3::eval(const std::vector<double> &ypp, double r, double *g) const {
  // Spline3Eq::splint_comb(double, double*) (spline3eq.h:204-236)
  if (r < x[0]) {
    *g = grad[0];
    return y[0] + grad[0] * (r - x[0]);
  } else if (r > x[nknots - 1]) {
    *g = grad[1];
    return y[nknots - 1] + grad[1] * (r - x[nknots - 1]);
  }
  double dr = r - x[0];
  int k = (dr < 0) ? 0 : int(dr * invstep);
  if (k >= nknots - 1) k = nknots - 2;
  double b = (dr - k * step) * invstep, a = 1.0 - b;
  double p1 = y[k], d21 = ypp[k], p2 = y[k + 1], d22 = ypp[k + 1];
  *g = (p2 - p1) * invstep + ((3 * (b * b) - 1) * d22 - (3 * (a * a) - 1) * d21) * step / 6.0;
  return a * p1 + b * p2 + ((a * a * a - a) * d21 + (b * b * b - b) * d22) * (step * step) / 6.0;
}

void Spline3::refresh5(std::vector<double> &ypp, std::vector<double> &yp4) const {
  // Spline5Eq::refresh_basis (spline5eq.cpp:209-293): unknowns h^2 y'' (rows
  // 0..n-1) and -h^4 y'''' (n..2n-1); interior rows are the continuity of
  // y' and y''' of the quintic pieces, end rows natural (y''' = y'''' = 0)
  // or clamped (y' and y'' given).
  const int n = nknots, m = 2 * n;
  std::vector<double> A((size_t)m * m, 0.0), b(m, 0.0);
  auto a = [&](int r, int c) -> double & { return A[(size_t)r * m + c]; };
  for (int i = 1; i < n - 1; ++i) {
    a(i, i - 1) = 1. / 12;
    a(i, i) = 10. / 12;
    a(i, i + 1) = 1. / 12;
    a(i, n + i - 1) = 1. / 180;
    a(i, n + i) = -1. / 90;
    a(i, n + i + 1) = 1. / 180;
    a(n + i, i - 1) = 1.;
    a(n + i, i) = -2.;
    a(n + i, i + 1) = 1.;
    a(n + i, n + i - 1) = 1. / 6;
    a(n + i, n + i) = 2. / 3;
    a(n + i, n + i + 1) = 1. / 6;
    b[i] = y[i + 1] - 2 * y[i] + y[i - 1];
    b[n + i] = 0.;
  }
  if (nat[0]) {
    a(0, 0) = -1.;
    a(0, 1) = 1.;
    a(0, n) = 1. / 3;
    a(0, n + 1) = 1. / 6;
    b[0] = 0.;
    a(n, n) = 1.;
    b[n] = 0.;
  } else {
    a(0, 0) = 1. / 3;
    a(0, 1) = 1. / 6;
    a(0, n) = 1. / 45;
    a(0, n + 1) = 7. / 360;
    b[0] = y[1] - y[0] - grad[0] * step;
    a(n, 0) = 1.;
    b[n] = grad2[0] * (step * step);
  }
  if (nat[1]) {
    a(n - 1, n - 2) = -1.;
    a(n - 1, n - 1) = 1.;
    a(n - 1, 2 * n - 2) = -1. / 6;
    a(n - 1, 2 * n - 1) = -1. / 3;
    b[n - 1] = 0.;
    a(2 * n - 1, 2 * n - 1) = 1.;
    b[2 * n - 1] = 0.;
  } else {
    a(n - 1, n - 2) = -1. / 6;
    a(n - 1, n - 1) = -1. / 3;
    a(n - 1, 2 * n - 2) = -7. / 360;
    a(n - 1, 2 * n - 1) = -1. / 45;
    b[n - 1] = y[n - 1] - y[n - 2] - grad[1] * step;
    a(2 * n - 1, n - 1) = 1.;
    b[2 * n - 1] = grad2[1] * (step * step);
  }
  // elimination with row pivoting on the largest |entry| of each column
  for (int k = 0; k < m; ++k) {
    int p = k;
    for (int r = k + 1; r < m; ++r)
      if (std::abs(a(r, k)) > std::abs(a(p, k))) p = r;
    if (p != k) {
      for (int c = 0; c < m; ++c) std::swap(a(k, c), a(p, c));
      std::swap(b[k], b[p]);
    }
    const double piv = a(k, k);
    if (piv == 0.0) continue;  // singular column: left as is (the reference does not check either)
    for (int r = k + 1; r < m; ++r) {
      const double f = a(r, k) / piv;
      if (f == 0.0) continue;
      for (int c = k + 1; c < m; ++c) a(r, c) -= f * a(k, c);
      b[r] -= f * b[k];
    }
  }
  for (int k = m - 1; k >= 0; --k) {
    double s = b[k];
    for (int c = k + 1; c < m; ++c) s -= a(k, c) * b[c];
    b[k] = a(k, k) != 0.0 ? s / a(k, k) : 0.0;
  }
  ypp.assign(n, 0.0);
  yp4.assign(n, 0.0);
  for (int i = 0; i < n; ++i) {
    ypp[i] = b[i] * (invstep * invstep);
    yp4[i] = -b[n + i] * (invstep * invstep * invstep * invstep);
  }
}

void Spline3::refresh_any(SplineDerivs &d) const {
  if (quintic) refresh5(d.ypp, d.yp4);
  else {
    refresh(d.ypp);
    d.yp4.assign(nknots, 0.0);
  }
}

double Spline3::eval_any(const SplineDerivs &d, double r, double *g) const {
  if (!quintic) return eval(d.ypp, r, g);
  // Spline5Eq::splint_comb(double, double*) (spline5eq.h:226-255)
  const int n = nknots;
  if (r < x[0]) {
    *g = grad[0] + grad2[0] * (r - x[0]);
    return y[0] + grad[0] * (r - x[0]) + 0.5 * grad2[0] * (r - x[0]) * (r - x[0]);
  } else if (r > x[n - 1]) {
    *g = grad[1] + grad2[1] * (r - x[n - 1]);
    return y[n - 1] + grad[1] * (r - x[n - 1]) + 0.5 * grad2[1] * (r - x[n - 1]) * (r - x[n - 1]);
  }
  double dr = r - x[0];
  int k = (dr < 0) ? 0 : int(dr * invstep);
  if (k >= n - 1) k = n - 2;
  double b = (dr - k * step) * invstep, a = 1.0 - b;
  double p1 = y[k], d21 = d.ypp[k], d41 = d.yp4[k], p2 = y[k + 1], d22 = d.ypp[k + 1], d42 = d.yp4[k + 1];
  *g = (p2 - p1) * invstep + ((3 * b * b - 1) * d22 - (3 * a * a - 1) * d21) * step / 6.0 +
       ((15 * b * b * b * b - 30 * b * b + 7) * d42 - (15 * a * a * a * a - 30 * a * a + 7) * d41) *
           (step * step * step) / 360.0;
  return a * p1 + b * p2 + ((a * a * a - a) * d21 + (b * b * b - b) * d22) * (step * step) / 6.0 +
         ((3 * a * a * a * a * a - 10 * a * a * a + 7 * a) * d41 + (3 * b * b * b * b * b - 10 * b * b * b + 7 * b) * d42) *
             (step * step * step * step) / 360.0;
}

double Spline3::eval_grad2_any(const SplineDerivs &d, double r) const {
  // Spline5Eq::splint_grad2(double) (spline5eq.h:260-291); cubic: the
  // interpolated y'' (spline3eq.h:241-266), 0 beyond the ends
  const int n = nknots;
  if (r < x[0]) return quintic ? grad2[0] : 0.0;
  if (r > x[n - 1]) return quintic ? grad2[1] : 0.0;
  double dr = r - x[0];
  int k = (dr < 0) ? 0 : int(dr * invstep);
  if (k >= n - 1) k = n - 2;
  double b = (dr - k * step) * invstep, a = 1.0 - b;
  double d21 = d.ypp[k], d22 = d.ypp[k + 1];
  if (!quintic) return a * d21 + b * d22;
  double d41 = d.yp4[k], d42 = d.yp4[k + 1];
  return a * d21 + b * d22 + ((a * a * a - a) * d41 + (b * b * b - b) * d42) * (step * step) / 6.0;
}

void Spline3::readjust_x(double l, double r) {
  // Spline3Eq::readjust_x (spline3eq.cpp:112-143), Spline5Eq::readjust_x
  // (spline5eq.cpp:121-157: the ends' y'' re-evaluated as well)
  SplineDerivs d;
  refresh_any(d);
  const Spline3 old = *this;
  step = (r - l) / (nknots - 1);
  invstep = 1.0 / step;
  x[0] = l;
  x[nknots - 1] = r;
  for (int i = 1; i < nknots - 1; ++i) x[i] = l + i * step;
  double g;
  for (int i = 0; i < nknots; ++i) y[i] = old.eval_any(d, x[i], &g);
  if (!nat[0]) {
    old.eval_any(d, l, &g);
    grad[0] = g;
    if (quintic) grad2[0] = old.eval_grad2_any(d, l);
  }
  if (!nat[1]) {
    old.eval_any(d, r, &g);
    grad[1] = g;
    if (quintic) grad2[1] = old.eval_grad2_any(d, r);
  }
  left = x[0];
  right = x[nknots - 1];
}

void Spline3::rescale_x(double scale) {
  // Spline3Eq::rescale_x (spline3eq.cpp:150-171), Spline5Eq::rescale_x
  // (spline5eq.cpp:163-189).  For a negative factor the reference reverses
  // x, y and the knot flags; its reversals of the two-element end arrays
  // (natural flags, slopes, slope flags) span one element and leave them
  // as they are, and so does this.
  step *= std::abs(scale);
  invstep = 1.0 / step;
  for (int i = 0; i < nknots; ++i) x[i] *= scale;
  if (!nat[0]) {
    grad[0] /= scale;
    if (quintic) grad2[0] /= scale * scale;
  }
  if (!nat[1]) {
    grad[1] /= scale;
    if (quintic) grad2[1] /= scale * scale;
  }
  if (scale < 0.0) {
    std::reverse(x.begin(), x.end());
    std::reverse(y.begin(), y.end());
    std::reverse(y_fixed.begin(), y_fixed.end());
  }
  left = x[0];
  right = x[nknots - 1];
}

void Spline3::scale_y(double f) {
  // Spline3Eq::operator*= (spline3eq.cpp:301-313), Spline5Eq::operator*=
  // (spline5eq.cpp:381-396, the ends' y'' too)
  for (int i = 0; i < nknots; ++i) y[i] *= f;
  if (!nat[0]) {
    grad[0] *= f;
    if (quintic) grad2[0] *= f;
  }
  if (!nat[1]) {
    grad[1] *= f;
    if (quintic) grad2[1] *= f;
  }
}

void Spline3::divide_y(double f) {
  // Spline3Eq::operator/= (spline3eq.cpp:318-330), Spline5Eq::operator/=
  for (int i = 0; i < nknots; ++i) y[i] /= f;
  if (!nat[0]) {
    grad[0] /= f;
    if (quintic) grad2[0] /= f;
  }
  if (!nat[1]) {
    grad[1] /= f;
    if (quintic) grad2[1] /= f;
  }
}

void Spline3::add(const Spline3 &rhs, const SplineDerivs &rhs_d) {
  // Spline3Eq::operator+= (spline3eq.cpp:335-348), Spline5Eq::operator+=
  // (spline5eq.cpp:424-441: y'' at the ends as well)
  const double rmax = rhs.x.back();
  double g;
  for (int i = 0; i < nknots; ++i) y[i] += (x[i] < rmax) ? rhs.eval_any(rhs_d, x[i], &g) : 0.;
  if (!nat[0]) {
    double v = 0.;
    if (x[0] < rmax) {
      rhs.eval_any(rhs_d, x[0], &g);
      v = g;
    }
    grad[0] += v;
    if (quintic) grad2[0] += (x[0] < rmax) ? rhs.eval_grad2_any(rhs_d, x[0]) : 0.;
  }
  if (!nat[1]) {
    double v = 0.;
    if (x.back() < rmax) {
      rhs.eval_any(rhs_d, x.back(), &g);
      v = g;
    }
    grad[1] += v;
    if (quintic) grad2[1] += (x.back() < rmax) ? rhs.eval_grad2_any(rhs_d, x.back()) : 0.;
  }
}

void Spline3::add_linear(double a) {
  // Spline3Eq::add_linear (spline3eq.cpp:177-186)
  for (int i = 0; i < nknots; ++i) y[i] += a * x[i];
  if (!nat[0]) grad[0] += a;
  if (!nat[1]) grad[1] += a;
}

double Spline3::max_y_mag() const {
  double m = 0.0;
  for (double v : y)
    if (std::abs(m) < std::abs(v)) m = v;
  return m;
}

// ---------------------------------------------------------------------- Pot

int Pot::nsplines() const {
  int n = 0;
  for (auto &g : groups) n += (int)g.size();
  return n;
}
int Pot::spline_index(int group, int alloy) const {
  int s = 0;
  for (int g = 0; g < group; ++g) s += (int)groups[g].size();
  return s + alloy;
}
const Spline3 &Pot::spline(int s) const {
  for (auto &g : groups) {
    if (s < (int)g.size()) return g[s];
    s -= (int)g.size();
  }
  fail(MZ_ERR_ARG, "spline index out of range");
}
Spline3 &Pot::spline(int s) { return const_cast<Spline3 &>(static_cast<const Pot *>(this)->spline(s)); }

int Pot::ncoeff() const {
  int n = 0;
  for (auto &g : groups)
    for (auto &s : g) n += s.ncoeff();
  return n;
}

// Coefficient order: Potential::coeff -> PotFns::coeff -> Spline::coeff ->
// Spline3Eq::bc_coeff (potential.cpp:192-206, pot_fns.cpp:209-218,
// spline.cpp:105-114, spline3eq.cpp:376-382).
std::vector<std::pair<int, int>> Pot::coeff_slots() const {
  std::vector<std::pair<int, int>> w;
  const int nc = ncoeff();
  int si = 0;
  for (auto &g : groups)
    for (auto &s : g) {
      for (int k = 0; k < s.nknots; ++k)
        if (!s.y_fixed[k]) w.emplace_back(si, k);
      for (int e = 0; e < 2; ++e)
        if (!s.grad_fixed[e] && !s.nat[e]) {
          w.emplace_back(si, s.nknots + e);
          if (s.quintic) w.emplace_back(si, s.nknots + 2 + e);
        }
      ++si;
    }
  w.resize(std::min<size_t>(w.size(), (size_t)nc));
  return w;
}
static double &slot_ref(Spline3 &s, int slot) {
  return slot < s.nknots ? s.y[slot] : slot < s.nknots + 2 ? s.grad[slot - s.nknots] : s.grad2[slot - s.nknots - 2];
}
void Pot::get_coeffs(double *out) const {
  Pot &self = const_cast<Pot &>(*this);
  int i = 0;
  for (auto &c : coeff_slots()) out[i++] = slot_ref(self.spline(c.first), c.second);
}
void Pot::set_coeffs(const double *in) {
  int i = 0;
  for (auto &c : coeff_slots()) slot_ref(spline(c.first), c.second) = in[i++];
}

double Pot::max_rcut() const {
  // radial groups: phi, rho, (MEAM) f, (JMEAM) p, p2
  double m = 0.0;
  for (int gi = 0; gi < (int)groups.size(); ++gi) {
    if (gi == G_U || gi == G_G || gi == G_Q1 || gi == G_Q2) continue;
    for (auto &s : groups[gi]) m = std::max(m, s.x.back());
  }
  return m;
}

static std::vector<std::string> split_lines(const std::string &text) {
  // Universe::read_file (universe.cpp:145-165): strip CR, drop blank lines.
  std::vector<std::string> out;
  std::istringstream is(text);
  std::string line;
  while (std::getline(is, line)) {
    size_t cr = line.find('\r');
    if (cr != std::string::npos) line.erase(cr, 1);
    for (char c : line)
      if (!std::isspace((unsigned char)c)) { out.push_back(line); break; }
  }
  return out;
}

static std::string read_text(const std::string &path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) fail(MZ_ERR_IO, "cannot open file: " + path);
  std::ostringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

void parse_pot(const std::string &text, Pot &pot) {
  // PotList::init (pot_list.cpp:84-142) for one #P block.
  std::vector<std::string> L = split_lines(text);
  if (L.empty()) fail(MZ_ERR_FORMAT, "empty potential file");
  size_t ln = 0;
  pot.comment = L[ln++];
  if (ln >= L.size() || L[ln].substr(0, 2) != "#T") fail(MZ_ERR_FORMAT, "potential type line (#T ...) missing");
  {
    std::istringstream is(L[ln++]);
    std::string lab;
    is >> lab >> pot.type_name >> pot.ntypes;
    if (is.fail()) fail(MZ_ERR_FORMAT, "pot type line (#T ...) is incorrect");
  }
  if (pot.ntypes < 1 || pot.ntypes > 8) fail(MZ_ERR_FORMAT, "number of atom types must be 1..8");
  int nt = pot.ntypes, npair = nt * (nt + 1) / 2;
  std::vector<int> nalloy;
  if (pot.type_name == "meam/spline") {
    pot.style = MZ_STYLE_MEAM_SPLINE;
    nalloy = {npair, nt, nt, npair, nt};
  } else if (pot.type_name == "gmeam/spline") {
    // g_i_jk: n * n (n + 1) / 2 splines (pot_gmeam.cpp:31-36)
    pot.style = MZ_STYLE_GMEAM_SPLINE;
    nalloy = {npair, nt, nt, npair, nt * npair};
  } else if (pot.type_name == "eam/spline") {
    pot.style = MZ_STYLE_EAM_SPLINE;
    nalloy = {npair, nt, nt};
  } else if (pot.type_name == "jmeam/spline") {
    // + p (Pair_ij), q (Triplet_i) (pot_jmeam.cpp:31-45)
    pot.style = MZ_STYLE_JMEAM_SPLINE;
    nalloy = {npair, nt, nt, npair, nt, npair, nt};
  } else if (pot.type_name == "jmeam2/spline") {
    // + p2, q2 (pot_jmeam2.cpp:31-45)
    pot.style = MZ_STYLE_JMEAM2_SPLINE;
    nalloy = {npair, nt, nt, npair, nt, npair, nt, npair, nt};
  } else if (pot.type_name == "pair/spline") {
    pot.style = MZ_STYLE_PAIR_SPLINE;
    nalloy = {npair};
  } else {
    fail(MZ_ERR_UNSUPPORTED, "potential style \"" + pot.type_name +
                                 "\" is not implemented (eam/spline, meam/spline, gmeam/spline, jmeam/spline, "
                                 "jmeam2/spline, pair/spline)");
  }
  pot.ngroups = (int)nalloy.size();
  if (ln >= L.size() || L[ln++].substr(0, 2) != "#P") fail(MZ_ERR_FORMAT, "potential line (#P ...) missing");
  pot.groups.assign(pot.ngroups, {});
  bool quintic = false;
  for (int g = 0; g < pot.ngroups; ++g) {
    for (int a = 0; a < nalloy[g]; ++a) {
      // PotFns::read_pot_fns (pot_fns.cpp:439-465) + Spline3Eq::read_basis
      if (ln >= L.size() || L[ln].substr(0, 2) != "#B") fail(MZ_ERR_FORMAT, "potential line (#B ...) missing");
      {
        std::istringstream is(L[ln++]);
        std::string lab, basis;
        is >> lab >> basis;
        if (is.fail()) fail(MZ_ERR_FORMAT, "incorrect basis definition, use format (#B <basis type>)");
        if (basis != "spline3eq" && basis != "spline5eq")
          fail(MZ_ERR_UNSUPPORTED, "basis \"" + basis + "\" is not implemented (spline3eq, spline5eq)");
        quintic = basis == "spline5eq";  // per function (pot_fns.cpp:439-465): bases may be mixed
      }
      Spline3 s;
      s.quintic = quintic ? 1 : 0;
      if (ln + 2 >= L.size()) fail(MZ_ERR_FORMAT, "unexpected end of potential file");
      {
        std::istringstream is(L[ln++]);
        is >> s.left >> s.right >> s.nknots;
        if (is.fail()) fail(MZ_ERR_FORMAT, "incorrect spline definition, use format (<left x> <right x> <nknots>)");
      }
      if (s.nknots < 3 || s.nknots > 64) fail(MZ_ERR_FORMAT, "spline knot count must be 3..64");
      {
        std::istringstream is(L[ln++]);
        int lc, rc;
        is >> lc >> rc;
        if (is.fail()) fail(MZ_ERR_FORMAT, "incorrect boundary condition constraint line");
        int c[2] = {lc, rc};
        for (int e = 0; e < 2; ++e) {
          if (c[e] == -1) s.nat[e] = 1;
          else if (c[e] == 0) s.grad_fixed[e] = 0;
          else if (c[e] == 1) s.grad_fixed[e] = 1;
          else fail(MZ_ERR_FORMAT, "boundary condition constraint line has an incorrect constraint value");
        }
      }
      {
        std::istringstream is(L[ln++]);
        is >> s.grad[0] >> s.grad[1];
        if (is.fail()) fail(MZ_ERR_FORMAT, "incorrect boundary condition line, format is (<left grad> <right grad>)");
      }
      if (s.quintic) {  // Spline5Eq::read_basis (spline5eq.cpp:97-102)
        if (ln >= L.size()) fail(MZ_ERR_FORMAT, "unexpected end of potential file");
        std::istringstream is(L[ln++]);
        is >> s.grad2[0] >> s.grad2[1];
        if (is.fail())
          fail(MZ_ERR_FORMAT, "incorrect boundary condition line, format is (<left grad2> <right grad2>)");
      }
      s.y.assign(s.nknots, 0.0);
      s.y_fixed.assign(s.nknots, 0);
      for (int k = 0; k < s.nknots; ++k) {
        if (ln >= L.size()) fail(MZ_ERR_FORMAT, "unexpected end of potential file");
        std::istringstream is(L[ln++]);
        is >> s.y_fixed[k] >> s.y[k];
        if (is.fail()) fail(MZ_ERR_FORMAT, "incorrect spline knot line, format is (<is y fixed?> <y-value>)");
      }
      s.set_grid();
      pot.groups[g].push_back(std::move(s));
    }
  }
}

std::string write_pot_text(const Pot &pot) {
  // Potential::write_pots (potential.cpp:721-732) + Spline3Eq::write_basis_fn
  // (spline3eq.cpp:248-273): scientific, 15 digits.
  std::ostringstream os;
  os << pot.comment << "\n#T " << pot.type_name << " " << pot.ntypes << "\n#P\n";
  char buf[128];
  for (auto &g : pot.groups)
    for (auto &s : g) {
      os << (s.quintic ? "#B spline5eq\n" : "#B spline3eq\n");
      std::snprintf(buf, sizeof buf, "%.15e %.15e %d\n", s.x[0], s.x[s.nknots - 1], s.nknots);
      os << buf;
      int c[2];
      for (int e = 0; e < 2; ++e) c[e] = s.nat[e] ? -1 : s.grad_fixed[e];
      os << c[0] << " " << c[1] << "\n";
      std::snprintf(buf, sizeof buf, "%.15e %.15e\n", s.grad[0], s.grad[1]);
      os << buf;
      if (s.quintic) {  // Spline5Eq::write_basis_fn (spline5eq.cpp:305-331)
        std::snprintf(buf, sizeof buf, "%.15e %.15e\n", s.grad2[0], s.grad2[1]);
        os << buf;
      }
      for (int k = 0; k < s.nknots; ++k) {
        std::snprintf(buf, sizeof buf, "%d %.15e\n", s.y_fixed[k], s.y[k]);
        os << buf;
      }
      os << "\n";
    }
  os << "\n";
  return os.str();
}

// ------------------------------------------------------------ configuration

void read_config_file(const std::string &path, int ntypes, std::vector<int> &cell_natoms,
                      std::vector<double> &lattice, std::vector<double> &e0,
                      std::vector<double> &s0, std::vector<double> &w, std::vector<double> &ew,
                      std::vector<double> &sw, std::vector<int> &types, std::vector<double> &pos,
                      std::vector<double> &f0) {
  // Cell::read_cell (cell.cpp:39-136), cell after cell until the end.
  std::vector<std::string> L = split_lines(read_text(path));
  size_t ln = 0, end = L.size();
  int cell = 0;
  auto err = [&](const std::string &m) {
    fail(MZ_ERR_FORMAT, m + " - cell=" + std::to_string(cell) + " (file=" + path + ")");
  };
  while (ln < end) {
    std::istringstream is(L[ln]);
    std::string lab;
    int n = 0, useforce = 1;
    is >> lab >> n >> useforce;
    if (lab != "#N") err("ERROR: number line (#N ...) is missing");
    if (is.fail()) err("ERROR: number line (#N ...) is incorrect");
    if (ln + 1 == end) err("ERROR: unexpected end of config file");
    double a[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, E = 0, S[6] = {0, 0, 0, 0, 0, 0}, W = 1, EW = 1, SW = 1;
    while (L[++ln].substr(0, 2) != "#F") {
      if (ln + 1 == end) err("ERROR: unexpected end of config file");
      std::istringstream hs(L[ln]);
      hs >> lab;
      if (lab == "#X") { hs >> a[0] >> a[1] >> a[2]; if (hs.fail()) err("ERROR: box_x vector (#X ...) incorrect"); }
      else if (lab == "#Y") { hs >> a[3] >> a[4] >> a[5]; if (hs.fail()) err("ERROR: box_y vector (#Y ...) incorrect"); }
      else if (lab == "#Z") { hs >> a[6] >> a[7] >> a[8]; if (hs.fail()) err("ERROR: box_z vector (#Z ...) incorrect"); }
      else if (lab == "#E") { hs >> E; if (hs.fail()) err("ERROR: energy (#E ...) incorrect"); }
      else if (lab == "#S") {
        for (int k = 0; k < 6; ++k) hs >> S[k];
        if (hs.fail()) err("ERROR: stress tensor (#S ...) incorrect");
      } else if (lab == "#W") { hs >> W; if (hs.fail()) err("ERROR: configuration weight (#W ...) incorrect"); }
      else if (lab == "#EW") { hs >> EW; if (hs.fail()) err("ERROR: configuration energy weight (#EW ...) incorrect"); }
      else if (lab == "#SW") { hs >> SW; if (hs.fail()) err("ERROR: configuration stress weight (#SW ...) incorrect"); }
    }
    if (ln + n >= end) err("ERROR: unexpected end of config file");
    cell_natoms.push_back(n);
    lattice.insert(lattice.end(), a, a + 9);
    e0.push_back(E);
    s0.insert(s0.end(), S, S + 6);
    w.push_back(W);
    ew.push_back(EW);
    sw.push_back(SW);
    for (int i = 0; i < n; ++i) {
      const std::string &al = L[++ln];
      if (al[0] == '#') err("ERROR: too few atoms");
      std::istringstream as(al);
      int t;
      double p[3], f[3];
      as >> t >> p[0] >> p[1] >> p[2] >> f[0] >> f[1] >> f[2];
      if (as.fail()) err("ERROR: atom line incorrect - atom=" + std::to_string(i));
      if (t < 0 || t >= ntypes) err("ERROR: incorrect atom type specified - atom=" + std::to_string(i));
      types.push_back(t);
      pos.insert(pos.end(), p, p + 3);
      f0.insert(f0.end(), f, f + 3);
    }
    ++ln;
    if (ln < end && L[ln].substr(0, 2) != "#N") err("ERROR: too many atoms");
    ++cell;
  }
}

// ------------------------------------------------------------------ rescale

int rescale_pot(Pot &pot, const int *atom_type, int natoms, const double *dens, int flag, double factors[4]) {
  // PotMEAM::rescale (pot_meam.cpp:281-375) / PotEAM::rescale (pot_eam.cpp:257-389)
  factors[0] = factors[1] = factors[2] = factors[3] = 0.0;
  if (flag < 0 || style_pair(pot.style)) return 0;  // PotPair: Potential::rescale (potential.cpp:258-261)
  const bool meam = style_meam(pot.style);
  std::vector<Spline3> &F = pot.groups[G_U];
  const int Fs = (int)F.size();
  std::vector<double> minrho(Fs, 1e100), maxrho(Fs, -1e100);
  for (int i = 0; i < natoms; ++i) {
    const int t = atom_type[i];
    maxrho[t] = std::max(dens[i], maxrho[t]);
    minrho[t] = std::min(dens[i], minrho[t]);
  }
  double min_density = 1e100, max_density = -1e100;
  int min_idx = -1, max_idx = -1;
  for (int i = 0; i < Fs; ++i) {
    if (maxrho[i] > max_density) {
      max_density = maxrho[i];
      max_idx = i;
    }
    if (minrho[i] < min_density) {
      min_density = minrho[i];
      min_idx = i;
    }
  }
  if (max_idx < 0 || min_idx < 0) return 0;  // no atoms: nothing to measure
  const int sign = (max_density >= -min_density) ? 1 : -1;
  std::vector<double> L(Fs), R(Fs);
  for (int i = 0; i < Fs; ++i) {
    const double rho_i = F[i].x[0], rho_f = F[i].x.back(), length = rho_f - rho_i;
    L[i] = minrho[i] - 0.01 * length;
    R[i] = maxrho[i] + 0.01 * length;
    if (flag || minrho[i] - rho_i < 0. || minrho[i] - rho_i > 0.05 * length || maxrho[i] - rho_f > 0. ||
        maxrho[i] - rho_f < -0.05 * length)
      flag = 1;
    if (R[i] - rho_f > 100.0 || L[i] - rho_i < -100.0) return 0;  // bounds too big
  }
  const double a = (sign == 1) ? 1.0 / R[max_idx] : 1.0 / L[min_idx];
  if (flag || std::abs(a) > 1.05 || std::abs(a) < 0.95) flag = 1;
  if (meam && flag && pot.style == MZ_STYLE_GMEAM_SPLINE) {
    // PotGMEAM::rescale_3body (pot_gmeam.cpp:301-345): each f_ij by its own
    // b = 1 / signed largest-|y| knot, and every g_i_jk whose f_ij or f_ik it
    // is divided by b (twice when j and k give the same f)
    const int nt = pot.ntypes;
    std::vector<Spline3> &fg = pot.groups[G_F], &gg = pot.groups[G_G];
    for (int fi = 0; fi < (int)fg.size(); ++fi) {
      const double b = 1.0 / fg[fi].max_y_mag();
      fg[fi].scale_y(b);
      for (int i = 0; i < nt; ++i)
        for (int j = 0; j < nt; ++j)
          for (int k = j; k < nt; ++k) {
            const int ijk = i * nt * (nt + 1) / 2 + pot.idx_pair_ij(j, k);
            if (fi == pot.idx_pair_ij(i, j)) gg[ijk].divide_y(b);
            if (fi == pot.idx_pair_ij(i, k)) gg[ijk].divide_y(b);
          }
      if (fi == 0) factors[1] = b;
    }
  } else if (meam && flag) {
    // PotMEAM::rescale_3body (pot_meam.cpp:497-525): f*f*g = (b f)(b f)(g / b^2),
    // b = 1 / signed largest-|y| knot of the f group (PotFns::get_max_y_mag, pot_fns.cpp:100-111)
    double m = 0.0;
    for (const Spline3 &sp : pot.groups[G_F]) {
      const double v = sp.max_y_mag();
      if (std::abs(m) < std::abs(v)) m = v;
    }
    const double b = 1.0 / m;
    for (Spline3 &sp : pot.groups[G_F]) sp.scale_y(b);
    for (Spline3 &sp : pot.groups[G_G]) sp.divide_y(b * b);
    factors[1] = b;
    // PotJMEAM::rescale_3body (pot_jmeam.cpp:375-401), PotJMEAM2::rescale_3body
    // (pot_jmeam2.cpp:416-442): p p q = (b p)(b p)(q / b^2) likewise, b from the p (p2) group
    for (int t = 0; t < style_nj(pot.style); ++t) {
      const int gp = t == 0 ? G_P1 : G_P2, gq = t == 0 ? G_Q1 : G_Q2;
      double mp = 0.0;
      for (const Spline3 &sp : pot.groups[gp]) {
        const double v = sp.max_y_mag();
        if (std::abs(mp) < std::abs(v)) mp = v;
      }
      const double bp = 1.0 / mp;
      for (Spline3 &sp : pot.groups[gp]) sp.scale_y(bp);
      for (Spline3 &sp : pot.groups[gq]) sp.divide_y(bp * bp);
      factors[2 + t] = bp;
    }
  }
  if (!flag) return 0;
  for (int i = 0; i < Fs; ++i) {
    F[i].readjust_x(L[i], R[i]);
    F[i].rescale_x(a);
  }
  for (Spline3 &sp : pot.groups[G_RHO]) sp.scale_y(a);
  if (meam)
    for (Spline3 &sp : pot.groups[G_G]) sp.scale_y(a);
  factors[0] = a;
  if (!meam) {
    // Gauge U'(mid) = 0 (pot_eam.cpp:336-383): lambda_i = U_i'(mid of its range),
    // phi_ij += lambda_j rho_i + lambda_i rho_j, U_i -= lambda_i n.  The
    // reference adds a copy of rho scaled in y whose second derivatives are
    // the unscaled rho's; so does this.
    std::vector<Spline3> &rho = pot.groups[G_RHO];
    std::vector<Spline3> &phi = pot.groups[G_PHI];
    std::vector<SplineDerivs> rho_d(rho.size());
    for (size_t i = 0; i < rho.size(); ++i) rho[i].refresh_any(rho_d[i]);
    std::vector<double> lam(Fs);
    for (int i = 0; i < Fs; ++i) {
      SplineDerivs d;
      F[i].refresh_any(d);
      double g;
      F[i].eval_any(d, 0.5 * (F[i].x[0] + F[i].x.back()), &g);
      lam[i] = g;
    }
    int count = 0;
    for (int i = 0; i < Fs; ++i)
      for (int j = i; j < Fs; ++j) {
        Spline3 t = rho[i];
        t.scale_y(lam[j]);
        phi[count].add(t, rho_d[i]);
        Spline3 t2 = rho[j];
        t2.scale_y(lam[i]);
        phi[count].add(t2, rho_d[j]);
        ++count;
      }
    for (int i = 0; i < Fs; ++i) F[i].add_linear(-1.0 * lam[i]);
  }
  return 1;
}

// -------------------------------------------------------------- data files

namespace {
std::string data_name(const std::string &prefix, const char *ext, int num) {
  std::ostringstream oss;
  oss << prefix << ext;
  if (num >= 0) oss << "." << num;
  return oss.str();
}
std::ofstream open_out(const std::string &path) {
  std::ofstream f(path, std::ios_base::out);
  if (!f) throw Failure{MZ_ERR_IO, "cannot write " + path};
  return f;
}
}  // namespace

void write_data_files(const Db &db, const Pot &pot, double energy_weight, double stress_weight, const double *e,
                      const double *energy, const double *stress, const double *force, const double *dens,
                      const std::string &prefix, int num) {
  // Potential::write_data (potential.cpp:325-342): .rho (PotEAM::write_densities
  // pot_eam.cpp:506-540), .energy (:497-543), .stress (:548-592), .force
  // (:597-642), .error (:647-708), .punish (PotEAM / PotMEAM::write_punish).
  // pair/spline writes neither .rho nor .punish (Potential::write_extras and
  // write_punish do nothing, potential.cpp:713-725).
  const int NC = db.ncells, N = db.natoms;
  const bool meam = style_meam(pot.style), pair = style_pair(pot.style);
  const int esize = style_esize(pot.style, pot.ntypes, NC, N);
  if (!pair) {
    std::ofstream f = open_out(data_name(prefix, ".rho", num));
    f << std::setw(6) << std::right << "conf:" << std::setw(5) << std::right << "atom" << std::setw(8) << std::right
      << "type" << std::setw(15) << std::right << "rho" << std::endl;
    for (int c = 0; c < NC; ++c)
      for (int i = 0; i < db.cell_atom0[c + 1] - db.cell_atom0[c]; ++i) {
        const int a = db.cell_atom0[c] + i;
        f << std::setw(5) << std::right << c << ":" << std::setw(5) << std::right << i << std::setw(8) << std::right
          << db.atom_type[a] << std::setw(15) << std::right << std::fixed << dens[a] << std::endl;
      }
  }
  {
    std::ofstream f = open_out(data_name(prefix, ".energy", num));
    f << "Global energy weight is " << std::fixed << energy_weight << std::endl;
    f << std::setw(3) << std::right << "#" << std::setw(11) << std::right << "conf_w" << std::setw(11) << std::right
      << "conf_ew" << std::setw(9) << std::right << "natoms" << std::setw(15) << std::right << "energy error"
      << std::setw(18) << std::right << "e" << std::setw(18) << std::right << "e0" << std::setw(15) << std::right
      << "|e-e0|" << std::setw(15) << std::right << "e-e0" << std::setw(15) << std::right << "de/e0" << std::endl;
    int idx = 0;
    for (int c = 0; c < NC; ++c) {
      const int na = db.cell_atom0[c + 1] - db.cell_atom0[c];
      const double en = energy[c], e0 = db.cell_energy0[c];
      f << std::setw(3) << std::right << c << std::fixed << std::setw(11) << std::right << std::setprecision(4)
        << db.cell_weight[c] << std::setw(11) << std::right << std::setprecision(4) << db.cell_eweight[c]
        << std::setw(9) << std::right << na << std::setw(15) << std::right << std::setprecision(6) << e[idx] * e[idx]
        << std::setw(18) << std::right << std::setprecision(10) << en << std::setw(18) << std::right
        << std::setprecision(10) << e0 << std::setw(15) << std::right << std::setprecision(6) << std::abs(en - e0)
        << std::setw(15) << std::right << std::setprecision(6) << en - e0;
      if (e0 == 0) f << std::setw(15) << std::right << "inf";
      else f << std::setw(15) << std::right << std::setprecision(6) << (e0 - en) / e0;
      f << std::endl;
      idx += 7 + 3 * na;
    }
  }
  {
    std::ofstream f = open_out(data_name(prefix, ".stress", num));
    f << "Global stress weight is " << std::fixed << stress_weight << std::endl;
    f << std::setw(3) << std::right << "#" << std::setw(11) << std::right << "conf_w" << std::setw(11) << std::right
      << "conf_sw" << std::setw(15) << std::right << "stress error" << std::setw(18) << std::right << "s"
      << std::setw(18) << std::right << "s0" << std::setw(15) << std::right << "ds/s0" << std::endl;
    int idx = 0;
    for (int c = 0; c < NC; ++c) {
      ++idx;
      for (int d = 0; d < 6; ++d) {
        const double s = stress[6 * c + d], s0 = db.cell_stress0[6 * c + d];
        f << std::setw(3) << std::right << c << std::fixed << std::setw(11) << std::right << std::setprecision(4)
          << db.cell_weight[c] << std::setw(11) << std::right << std::setprecision(4) << db.cell_sweight[c]
          << std::setw(15) << std::right << std::setprecision(6) << e[idx] * e[idx] << std::setw(18) << std::right
          << std::setprecision(10) << s << std::setw(18) << std::right << std::setprecision(10) << s0;
        if (s0 == 0) f << std::setw(15) << std::right << "inf";
        else f << std::setw(15) << std::right << std::setprecision(6) << (s0 - s) / s0;
        f << std::endl;
        ++idx;
      }
      idx += 3 * (db.cell_atom0[c + 1] - db.cell_atom0[c]);
    }
  }
  {
    std::ofstream f = open_out(data_name(prefix, ".force", num));
    f << std::setw(6) << std::right << "conf:" << std::setw(5) << std::right << "atom" << std::setw(8) << std::right
      << "type" << std::setw(15) << std::right << "force error" << std::setw(15) << std::right << "f"
      << std::setw(15) << std::right << "f0" << std::setw(15) << std::right << "df/f0" << std::endl;
    int idx = 0;
    for (int c = 0; c < NC; ++c) {
      idx += 7;
      for (int i = 0; i < db.cell_atom0[c + 1] - db.cell_atom0[c]; ++i) {
        const int a = db.cell_atom0[c] + i;
        for (int d = 0; d < 3; ++d) {
          const double fv = force[3 * a + d], f0 = db.atom_force0[3 * a + d];
          f << std::setw(5) << std::right << c << ":" << std::setw(5) << std::right << i << std::setw(8) << std::right
            << db.atom_type[a] << std::setw(15) << std::right << std::fixed << e[idx] * e[idx] << std::setw(15)
            << std::right << std::fixed << fv << std::setw(15) << std::right << std::fixed << f0;
          if (f0 == 0) f << std::setw(15) << std::right << "inf";
          else f << std::setw(15) << std::right << std::fixed << (f0 - fv) / f0;
          f << std::endl;
          ++idx;
        }
      }
    }
  }
  {
    double se = 0.0, ss = 0.0, sf = 0.0, sp = 0.0;
    int idx = 0;
    for (int c = 0; c < NC; ++c) {
      se += e[idx] * e[idx];
      ++idx;
      for (int d = 0; d < 6; ++d, ++idx) ss += e[idx] * e[idx];
      for (int i = 0; i < 3 * (db.cell_atom0[c + 1] - db.cell_atom0[c]); ++i, ++idx) sf += e[idx] * e[idx];
    }
    for (int i = idx; i < esize; ++i) sp += e[i] * e[i];
    const double total = se + ss + sf + sp;
    const int npunish = esize - 3 * N - 6 * NC - NC;
    std::ofstream f = open_out(data_name(prefix, ".error", num));
    f << "Total error sum " << std::fixed << total << " count " << esize << " (" << 3 * N << " forces, " << 6 * NC
      << " stresses, " << NC << " energies";
    if (npunish == 0) f << ")" << std::endl;
    else f << ", " << npunish << " punishments)" << std::endl;
    f << "Sum of force errors  = " << std::fixed << sf << std::endl;
    f << "Sum of energy errors = " << std::fixed << se << std::endl;
    f << "Sum of stress errors = " << std::fixed << ss << std::endl;
    if (npunish) f << "Sum of punish errors = " << std::fixed << sp << std::endl;
  }
  if (!pair) {
    std::ofstream f = open_out(data_name(prefix, ".punish", num));
    f << "Limiting constraints (atomic density lies inside F boundaries)" << std::endl;
    f << std::setw(3) << std::right << "#" << std::setw(11) << std::right << "conf_w" << std::setw(15) << std::right
      << "punish error" << std::setw(15) << std::right << "punishment" << std::endl;
    int idx = 7 * NC + 3 * N;
    for (int c = 0; c < NC; ++c, ++idx)
      f << std::setw(3) << std::right << c << std::fixed << std::setw(11) << std::right << std::setprecision(4)
        << db.cell_weight[c] << std::setw(15) << std::right << std::setprecision(6) << e[idx] * e[idx]
        << std::setw(15) << std::right << std::setprecision(6) << e[idx] / db.cell_weight[c] << std::endl;
    if (pot.style == MZ_STYLE_GMEAM_SPLINE) {
      // PotGMEAM::write_punish (pot_gmeam.cpp:246-296): one line per f spline
      f << std::endl << "Dummy constraints (|f_max(r)| = 1)" << std::endl;
      f << std::setw(15) << std::right << "punish error" << std::setw(15) << std::right << "|f_max(r)|" << std::endl;
      for (const Spline3 &sp : pot.groups[G_F]) {
        f << std::fixed << std::setw(15) << std::right << std::setprecision(6) << e[idx] * e[idx] << std::setw(15)
          << std::right << std::setprecision(6) << std::abs(std::abs(sp.max_y_mag())) << std::endl;
        ++idx;
      }
    } else if (meam) {
      // PotMEAM::write_punish; PotJMEAM / PotJMEAM2::write_punish add the p
      // (p2) magnitudes (pot_jmeam.cpp:309-366, pot_jmeam2.cpp:337-410)
      static const char *name[3] = {"f", "p", "p2"};
      const int grp[3] = {G_F, G_P1, G_P2};
      for (int t = 0; t <= style_nj(pot.style); ++t, ++idx) {
        double m = 0.0;
        for (const Spline3 &sp : pot.groups[grp[t]]) {
          const double v = sp.max_y_mag();
          if (std::abs(m) < std::abs(v)) m = v;
        }
        f << std::endl << "Dummy constraints (|" << name[t] << "_max(r)| = 1)" << std::endl;
        f << std::setw(15) << std::right << "punish error" << std::setw(15) << std::right
          << (std::string("|") + name[t] + "_max(r)|") << std::endl;
        f << std::fixed << std::setw(15) << std::right << std::setprecision(6) << e[idx] * e[idx] << std::setw(15)
          << std::right << std::setprecision(6) << std::abs(std::abs(m)) << std::endl;
      }
    } else {
      f << std::endl << "Dummy constraints (F'(n_avg) = 0)" << std::endl;
      f << std::setw(7) << std::right << "element" << std::setw(15) << std::right << "punish error" << std::setw(15)
        << std::right << "F'(n_avg)" << std::endl;
      for (int t = 0; t < pot.ntypes; ++t, ++idx)
        f << std::setw(7) << std::right << t << std::fixed << std::setw(15) << std::right << std::setprecision(6)
          << e[idx] * e[idx] << std::setw(15) << std::right << std::setprecision(6) << e[idx] / 100. << std::endl;
    }
  }
}

// --------------------------------------------------------------- neighbours

namespace {
struct V3 {
  double x, y, z;
};
inline double dot(const V3 &a, const V3 &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(const V3 &a, const V3 &b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline double mag(const V3 &v) { return std::sqrt(dot(v, v)); }

struct CellPairs {
  std::vector<int> nbr;
  std::vector<double> r, u, shift;
  std::vector<int8_t> knot;
  std::vector<int> row_len;
  int status = MZ_OK;
  std::string msg;
};
}  // namespace

void build_db_setup(const mz_cells_desc &c, const Pot &pot, Db &db) {
  if (c.ncells <= 0 || c.natoms <= 0 || !c.cell_natoms || !c.cell_lattice || !c.atom_type || !c.atom_pos)
    fail(MZ_ERR_ARG, "empty or incomplete cell description");
  const bool meam = style_meam(pot.style);
  db.style = pot.style;
  db.nfun = 3 + style_nj(pot.style);
  db.ncells = c.ncells;
  db.natoms = c.natoms;
  db.cell_atom0.assign(c.ncells + 1, 0);
  for (int i = 0; i < c.ncells; ++i) {
    if (c.cell_natoms[i] <= 0) fail(MZ_ERR_FORMAT, "cell with no atoms: cell=" + std::to_string(i));
    db.cell_atom0[i + 1] = db.cell_atom0[i] + c.cell_natoms[i];
  }
  if (db.cell_atom0[c.ncells] != c.natoms) fail(MZ_ERR_ARG, "cell atom counts do not sum to natoms");
  auto opt = [&](const double *p, int i, double d) { return p ? p[i] : d; };
  db.cell_vol.resize(c.ncells);
  db.cell_weight.resize(c.ncells);
  db.cell_eweight.resize(c.ncells);
  db.cell_sweight.resize(c.ncells);
  db.cell_energy0.resize(c.ncells);
  db.cell_stress0.assign(6 * (size_t)c.ncells, 0.0);
  db.cell_lattice.assign(c.cell_lattice, c.cell_lattice + 9 * (size_t)c.ncells);
  for (int i = 0; i < c.ncells; ++i) {
    db.cell_weight[i] = opt(c.cell_weight, i, 1.0);
    db.cell_eweight[i] = opt(c.cell_eweight, i, 1.0);
    db.cell_sweight[i] = opt(c.cell_sweight, i, 1.0);
    db.cell_energy0[i] = opt(c.cell_energy0, i, 0.0);
    for (int k = 0; k < 6; ++k) db.cell_stress0[6 * i + k] = c.cell_stress0 ? c.cell_stress0[6 * i + k] : 0.0;
  }
  db.atom_type.assign(c.atom_type, c.atom_type + c.natoms);
  db.atom_cell.resize(c.natoms);
  db.atom_pos.assign(c.atom_pos, c.atom_pos + 3 * (size_t)c.natoms);
  if (c.atom_force0) db.atom_force0.assign(c.atom_force0, c.atom_force0 + 3 * (size_t)c.natoms);
  else db.atom_force0.assign(3 * (size_t)c.natoms, 0.0);
  for (int i = 0; i < c.ncells; ++i)
    for (int a = db.cell_atom0[i]; a < db.cell_atom0[i + 1]; ++a) {
      if (db.atom_type[a] < 0 || db.atom_type[a] >= pot.ntypes)
        fail(MZ_ERR_FORMAT, "incorrect atom type specified - cell=" + std::to_string(i));
      db.atom_cell[a] = i;
    }
}

bool cell_scale(const double *A, double max_rcut, double *vol, int s[3]) {
  // Cell::compute_vol (cell.cpp:191-194) and Cell::find_scale (cell.cpp:158-170)
  V3 a0{A[0], A[1], A[2]}, a1{A[3], A[4], A[5]}, a2{A[6], A[7], A[8]};
  *vol = std::abs(dot(a0, cross(a1, a2)));
  double ihx = mag(cross(a1, a2)) / *vol, ihy = mag(cross(a2, a0)) / *vol, ihz = mag(cross(a0, a1)) / *vol;
  s[0] = int(std::ceil(max_rcut * ihx));
  s[1] = int(std::ceil(max_rcut * ihy));
  s[2] = int(std::ceil(max_rcut * ihz));
  return s[0] > 0 && s[1] > 0 && s[2] > 0;
}

std::string cell_too_small_msg(int ci) {
  return "ERROR: Cell #" + std::to_string(ci) + " is too small or potential is too big";
}

std::string pair_too_short_msg(const Pot &pot, int q, double rr, int ti, int tj, int ci, int i, int j) {
  static const char *nm[5] = {"phi", "rho", "f", "p", "p2"};
  char buf[256];
  std::snprintf(buf, sizeof buf,
                "ERROR: Pair distance too short for potential (r=%g, pot=%s[%d]) - cell=%d atom=%d neigh=%d", rr,
                nm[q], q == 1 ? tj : pot.idx_pair_ij(ti, tj), ci, i, j);
  return buf;
}

void build_incoming(Db &db) {
  // Incoming lists (counting sort by neighbour, slot order kept).
  const int64_t np = db.npairs;
  db.in_off.assign(db.natoms + 1, 0);
  for (int64_t s = 0; s < np; ++s) db.in_off[db.pair_nbr[s] + 1]++;
  for (int a = 0; a < db.natoms; ++a) db.in_off[a + 1] += db.in_off[a];
  db.in_slot.resize(np);
  std::vector<int64_t> fill(db.in_off.begin(), db.in_off.end() - 1);
  for (int64_t s = 0; s < np; ++s) db.in_slot[fill[db.pair_nbr[s]]++] = s;
}

void build_db(const mz_cells_desc &c, const Pot &pot, Db &db) {
  build_db_setup(c, pot, db);
  const bool meam = style_meam(pot.style), half = style_pair(pot.style);
  const int nj = style_nj(pot.style), nf = db.nfun;
  // radial functions checked per pair: phi (rho, f, p, p2)
  const int nq = half ? 1 : meam ? 3 + nj : 2;
  const double max_rcut = pot.max_rcut();
  const int sphi0 = pot.spline_index(G_PHI, 0), srho0 = half ? -1 : pot.spline_index(G_RHO, 0);
  const int sf0 = meam ? pot.spline_index(G_F, 0) : -1;
  const int sp0[2] = {nj > 0 ? pot.spline_index(G_P1, 0) : -1, nj > 1 ? pot.spline_index(G_P2, 0) : -1};

  std::vector<CellPairs> per(c.ncells);
  std::atomic<int> next(0);
  auto work = [&]() {
    for (;;) {
      int ci = next.fetch_add(1);
      if (ci >= c.ncells) return;
      CellPairs &out = per[ci];
      const double *A = c.cell_lattice + 9 * (size_t)ci;
      V3 a0{A[0], A[1], A[2]}, a1{A[3], A[4], A[5]}, a2{A[6], A[7], A[8]};
      int sc[3];
      if (!cell_scale(A, max_rcut, &db.cell_vol[ci], sc)) {
        out.status = MZ_ERR_RANGE;
        out.msg = cell_too_small_msg(ci);
        return;
      }
      const int sx = sc[0], sy = sc[1], sz = sc[2];
      const int a_lo = db.cell_atom0[ci], na = db.cell_atom0[ci + 1] - a_lo;
      // Config::find_pairs (config.cpp:143-234): double counted (j0 = 0), or
      // for pair/spline each pair once (j0 = the atom's own index)
      for (int i = 0; i < na && out.status == MZ_OK; ++i) {
        const double *pi = c.atom_pos + 3 * (size_t)(a_lo + i);
        const int ti = c.atom_type[a_lo + i];
        int row = 0;
        for (int j = half ? i : 0; j < na; ++j) {
          const double *pj = c.atom_pos + 3 * (size_t)(a_lo + j);
          const int tj = c.atom_type[a_lo + j];
          for (int ix = -sx; ix <= sx; ++ix)
            for (int iy = -sy; iy <= sy; ++iy)
              for (int iz = -sz; iz <= sz; ++iz) {
                if (i == j && ix == 0 && iy == 0 && iz == 0) continue;
                V3 d;
                d.x = pj[0] + ix * a0.x + iy * a1.x + iz * a2.x - pi[0];
                d.y = pj[1] + ix * a0.y + iy * a1.y + iz * a2.y - pi[1];
                d.z = pj[2] + ix * a0.z + iy * a1.z + iz * a2.z - pi[2];
                double r = mag(d);
                if (r >= max_rcut) continue;
                // Pair::setup_pair (pair.cpp:35-42)
                double rr = mag(d);
                V3 u{d.x / rr, d.y / rr, d.z / rr};
                // check_pair (pair_meam_spline.cpp:50-99 / pair_eam_spline.cpp:50-86 /
                // pair_pair_spline.cpp:48-72 / pair_jmeam_spline.cpp:48-110)
                const int pij = pot.idx_pair_ij(ti, tj);
                int sidx[5] = {sphi0 + pij, srho0 + tj, meam ? sf0 + pij : -1, sp0[0] + pij, sp0[1] + pij};
                int kn[5] = {-1, -1, -1, -1, -1};
                double sh[5] = {0, 0, 0, 0, 0};
                bool bad = false;
                for (int q = 0; q < nq; ++q) {
                  const Spline3 &sp = pot.spline(sidx[q]);
                  if (rr < sp.x[0]) {
                    out.status = MZ_ERR_RANGE;
                    out.msg = pair_too_short_msg(pot, q, rr, ti, tj, ci, i, j);
                    bad = true;
                    break;
                  }
                  kn[q] = sp.knotshift(rr, &sh[q]);
                }
                if (bad) return;
                if (kn[0] == -1 && kn[1] == -1 && kn[2] == -1 && kn[3] == -1 && kn[4] == -1) continue;
                out.nbr.push_back(a_lo + j);
                out.r.push_back(rr);
                out.u.push_back(u.x);
                out.u.push_back(u.y);
                out.u.push_back(u.z);
                for (int q = 0; q < nf; ++q) {
                  out.knot.push_back((int8_t)kn[q]);
                  out.shift.push_back(kn[q] >= 0 ? sh[q] : 0.0);
                }
                ++row;
              }
        }
        out.row_len.push_back(row);
      }
    }
  };
  unsigned nth = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
  std::vector<std::thread> th;
  for (unsigned t = 0; t < nth; ++t) th.emplace_back(work);
  for (auto &t : th) t.join();
  for (int ci = 0; ci < c.ncells; ++ci)
    if (per[ci].status != MZ_OK) fail(per[ci].status, per[ci].msg);

  // Concatenate rows in atom order.
  db.pair_off.assign(c.natoms + 1, 0);
  int64_t np = 0;
  db.max_row = 0;
  db.ntriplets = 0;
  for (int ci = 0; ci < c.ncells; ++ci) {
    const int a_lo = db.cell_atom0[ci];
    for (size_t i = 0; i < per[ci].row_len.size(); ++i) {
      int n = per[ci].row_len[i];
      db.pair_off[a_lo + i + 1] = db.pair_off[a_lo + i] + n;
      db.max_row = std::max(db.max_row, n);
      if (meam) db.ntriplets += (int64_t)n * (n - 1) / 2;
    }
    np += (int64_t)per[ci].nbr.size();
  }
  db.npairs = np;
  db.pair_nbr.resize(np);
  db.pair_r.resize(np);
  db.pair_u.resize(3 * np);
  db.pair_knot.resize(nf * np);
  db.pair_shift.resize(nf * np);
  int64_t o = 0;
  for (int ci = 0; ci < c.ncells; ++ci) {
    CellPairs &p = per[ci];
    size_t n = p.nbr.size();
    std::copy(p.nbr.begin(), p.nbr.end(), db.pair_nbr.begin() + o);
    std::copy(p.r.begin(), p.r.end(), db.pair_r.begin() + o);
    std::copy(p.u.begin(), p.u.end(), db.pair_u.begin() + 3 * o);
    std::copy(p.knot.begin(), p.knot.end(), db.pair_knot.begin() + nf * o);
    std::copy(p.shift.begin(), p.shift.end(), db.pair_shift.begin() + nf * o);
    o += (int64_t)n;
    CellPairs().nbr.swap(p.nbr);
  }
  build_incoming(db);
}

}  // namespace mzb

// ------------------------------------------------------------------ C ABI

using namespace mzb;

template <class F>
static mz_status guarded(F &&f) {
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

extern "C" {

const char *mz_last_error(void) { return g_last_error.c_str(); }

mz_status mz_pot_clone(const mz_pot *pot, mz_pot **out) {
  return guarded([&] {
    if (!pot || !out) fail(MZ_ERR_ARG, "null argument");
    *out = new mz_pot(*pot);
  });
}

mz_status mz_pot_parse(const char *text, mz_pot **out) {
  return guarded([&] {
    if (!text || !out) fail(MZ_ERR_ARG, "null argument");
    auto *p = new mz_pot;
    try {
      parse_pot(text, p->pot);
    } catch (...) {
      delete p;
      throw;
    }
    *out = p;
  });
}

mz_status mz_pot_read(const char *path, mz_pot **out) {
  return guarded([&] {
    if (!path || !out) fail(MZ_ERR_ARG, "null argument");
    std::string t = read_text(path);
    auto *p = new mz_pot;
    try {
      parse_pot(t, p->pot);
    } catch (...) {
      delete p;
      throw;
    }
    *out = p;
  });
}

void mz_pot_free(mz_pot *pot) { delete pot; }

mz_status mz_pot_info(const mz_pot *pot, int *style, int *ntypes, int *nsplines) {
  return guarded([&] {
    if (!pot) fail(MZ_ERR_ARG, "null potential");
    if (style) *style = pot->pot.style;
    if (ntypes) *ntypes = pot->pot.ntypes;
    if (nsplines) *nsplines = pot->pot.nsplines();
  });
}

mz_status mz_pot_ncoeff(const mz_pot *pot, int *n) {
  return guarded([&] {
    if (!pot || !n) fail(MZ_ERR_ARG, "null argument");
    *n = pot->pot.ncoeff();
  });
}

mz_status mz_pot_get_coeffs(const mz_pot *pot, double *x) {
  return guarded([&] {
    if (!pot || !x) fail(MZ_ERR_ARG, "null argument");
    pot->pot.get_coeffs(x);
  });
}

mz_status mz_pot_set_coeffs(mz_pot *pot, const double *x) {
  return guarded([&] {
    if (!pot || !x) fail(MZ_ERR_ARG, "null argument");
    pot->pot.set_coeffs(x);
  });
}

mz_status mz_pot_write(const mz_pot *pot, const char *path) {
  return guarded([&] {
    if (!pot || !path) fail(MZ_ERR_ARG, "null argument");
    std::ofstream f(path);
    if (!f) fail(MZ_ERR_IO, std::string("cannot write ") + path);
    f << write_pot_text(pot->pot);
  });
}

mz_status mz_pot_spline_eval(const mz_pot *pot, int s, double x, double *val, double *grad) {
  return guarded([&] {
    if (!pot || !val || !grad) fail(MZ_ERR_ARG, "null argument");
    if (s < 0 || s >= pot->pot.nsplines()) fail(MZ_ERR_ARG, "spline index out of range");
    const Spline3 &sp = pot->pot.spline(s);
    SplineDerivs d;
    sp.refresh_any(d);
    *val = sp.eval_any(d, x, grad);
  });
}

static void build_any(const mz_cells_desc &c, const mz_pot *pot, int device, mz_db **out) {
  auto *d = new mz_db;
  try {
    if (device >= 0) build_db_device(c, pot->pot, d->db, device);
    else build_db(c, pot->pot, d->db);
  } catch (...) {
    delete d;
    throw;
  }
  *out = d;
}

mz_status mz_pot_rescale(mz_pot *pot, const mz_db *db, const double *densities, int flag, int *rescaled,
                         double *factors) {
  return guarded([&] {
    if (!pot || !db || !densities || !rescaled || !factors) fail(MZ_ERR_ARG, "null argument");
    for (auto &g : pot->pot.groups)
      for (auto &sp : g)
        if (sp.nknots < 2) fail(MZ_ERR_ARG, "spline with fewer than two knots");
    *rescaled = rescale_pot(pot->pot, db->db.atom_type.data(), db->db.natoms, densities, flag, factors);
  });
}

mz_status mz_write_data(const mz_db *db, const mz_pot *pot, double energy_weight, double stress_weight,
                        const double *errvec, const double *energy, const double *stress, const double *forces,
                        const double *densities, const char *prefix, int num) {
  return guarded([&] {
    if (!db || !pot || !errvec || !energy || !stress || !forces || !prefix ||
        (!densities && !style_pair(pot->pot.style)))
      fail(MZ_ERR_ARG, "null argument");
    write_data_files(db->db, pot->pot, energy_weight, stress_weight, errvec, energy, stress, forces, densities,
                     prefix, num);
  });
}

mz_status mz_db_build(const mz_cells_desc *cells, const mz_pot *pot, mz_db **out) {
  return guarded([&] {
    if (!cells || !pot || !out) fail(MZ_ERR_ARG, "null argument");
    build_any(*cells, pot, -1, out);
  });
}

mz_status mz_db_build_device(const mz_cells_desc *cells, const mz_pot *pot, int device, mz_db **out) {
  return guarded([&] {
    if (!cells || !pot || !out || device < 0) fail(MZ_ERR_ARG, "null argument or negative device");
    build_any(*cells, pot, device, out);
  });
}

static void read_any(const char *path, const mz_pot *pot, int device, mz_db **out) {
  {
    std::vector<int> cn, types;
    std::vector<double> lat, e0, s0, w, ew, sw, pos, f0;
    read_config_file(path, pot->pot.ntypes, cn, lat, e0, s0, w, ew, sw, types, pos, f0);
    mz_cells_desc c;
    c.ncells = (int)cn.size();
    c.natoms = (int)types.size();
    c.cell_natoms = cn.data();
    c.cell_lattice = lat.data();
    c.cell_energy0 = e0.data();
    c.cell_stress0 = s0.data();
    c.cell_weight = w.data();
    c.cell_eweight = ew.data();
    c.cell_sweight = sw.data();
    c.atom_type = types.data();
    c.atom_pos = pos.data();
    c.atom_force0 = f0.data();
    build_any(c, pot, device, out);
  }
}

mz_status mz_db_read(const char *path, const mz_pot *pot, mz_db **out) {
  return guarded([&] {
    if (!path || !pot || !out) fail(MZ_ERR_ARG, "null argument");
    read_any(path, pot, -1, out);
  });
}

mz_status mz_db_read_device(const char *path, const mz_pot *pot, int device, mz_db **out) {
  return guarded([&] {
    if (!path || !pot || !out || device < 0) fail(MZ_ERR_ARG, "null argument or negative device");
    read_any(path, pot, device, out);
  });
}

void mz_db_free(mz_db *db) { delete db; }

mz_status mz_db_info(const mz_db *db, mz_db_stats *st) {
  return guarded([&] {
    if (!db || !st) fail(MZ_ERR_ARG, "null argument");
    st->ncells = db->db.ncells;
    st->natoms = db->db.natoms;
    st->npairs = db->db.npairs;
    st->ntriplets = db->db.ntriplets;
    st->max_row = db->db.max_row;
    // + the style's punishment entries
    st->esize = 7 * db->db.ncells + 3 * db->db.natoms + (style_pair(db->db.style) ? 0 : db->db.ncells);
  });
}

mz_status mz_db_get_view(const mz_db *dbh, mz_db_view *v) {
  return guarded([&] {
    if (!dbh || !v) fail(MZ_ERR_ARG, "null argument");
    const Db &d = dbh->db;
    v->ncells = d.ncells;
    v->natoms = d.natoms;
    v->npairs = d.npairs;
    v->cell_atom0 = d.cell_atom0.data();
    v->cell_vol = d.cell_vol.data();
    v->cell_weight = d.cell_weight.data();
    v->cell_eweight = d.cell_eweight.data();
    v->cell_sweight = d.cell_sweight.data();
    v->cell_energy0 = d.cell_energy0.data();
    v->cell_stress0 = d.cell_stress0.data();
    v->cell_lattice = d.cell_lattice.data();
    v->atom_type = d.atom_type.data();
    v->atom_cell = d.atom_cell.data();
    v->atom_pos = d.atom_pos.data();
    v->atom_force0 = d.atom_force0.data();
    v->pair_off = d.pair_off.data();
    v->pair_nbr = d.pair_nbr.data();
    v->pair_r = d.pair_r.data();
    v->pair_u = d.pair_u.data();
    v->pair_knot = d.pair_knot.data();
    v->pair_shift = d.pair_shift.data();
    v->in_off = d.in_off.data();
    v->in_slot = d.in_slot.data();
    v->nfun = d.nfun;
  });
}

mz_status mz_pot_get_spline(const mz_pot *pot, int s, mz_spline_view *v) {
  return guarded([&] {
    if (!pot || !v) fail(MZ_ERR_ARG, "null argument");
    if (s < 0 || s >= pot->pot.nsplines()) fail(MZ_ERR_ARG, "spline index out of range");
    int g = 0, a = s;
    while (a >= (int)pot->pot.groups[g].size()) a -= (int)pot->pot.groups[g++].size();
    const Spline3 &sp = pot->pot.spline(s);
    v->group = g;
    v->alloy = a;
    v->nknots = sp.nknots;
    v->left = sp.left;
    v->right = sp.right;
    v->nat[0] = sp.nat[0];
    v->nat[1] = sp.nat[1];
    v->grad_fixed[0] = sp.grad_fixed[0];
    v->grad_fixed[1] = sp.grad_fixed[1];
    v->grad[0] = sp.grad[0];
    v->grad[1] = sp.grad[1];
    v->quintic = sp.quintic;
    v->grad2[0] = sp.grad2[0];
    v->grad2[1] = sp.grad2[1];
    v->y_fixed = sp.y_fixed.data();
    v->y = sp.y.data();
    v->x = sp.x.data();
    v->step = sp.step;
  });
}

mz_status mz_db_set_targets(mz_db *db, const double *e0, const double *s0, const double *f0) {
  return guarded([&] {
    if (!db) fail(MZ_ERR_ARG, "null database");
    if (e0) std::copy(e0, e0 + db->db.ncells, db->db.cell_energy0.begin());
    if (s0) std::copy(s0, s0 + 6 * (size_t)db->db.ncells, db->db.cell_stress0.begin());
    if (f0) std::copy(f0, f0 + 3 * (size_t)db->db.natoms, db->db.atom_force0.begin());
  });
}

}  // extern "C"
