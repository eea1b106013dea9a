// Device-side equidistant cubic spline arithmetic (value, slope, second
// derivative, and the weights of each with respect to the knot table), plus
// the exact triplet cosine.
#pragma once

#include <cuda_runtime.h>

#include "mz_device.cuh"

namespace mzb {

// Value and slope from (knot, shift): Spline3Eq::splint_comb(int, double,
// double*) (spline3eq.h:110-122).
template <typename R>
__device__ __forceinline__ R spl_val_grad(const R *y, const R *ypp, int k, R b, R step6, R stepsq6,
                                          R invstep, R &grad) {
  const R a = R(1) - b;
  const R p1 = y[k], p2 = y[k + 1], d1 = ypp[k], d2 = ypp[k + 1];
  grad = (p2 - p1) * invstep + ((R(3) * b * b - R(1)) * d2 - (R(3) * a * a - R(1)) * d1) * step6;
  return a * p1 + b * p2 + ((a * a * a - a) * d1 + (b * b * b - b) * d2) * stepsq6;
}

// Value and slope from the per-interval cubic c = (c0, c1, c2, c3) of the
// evaluation table -- the same polynomial as above, with
//   c0 = y[k], c1 = y[k+1] - y[k] - (2 ypp[k] + ypp[k+1]) h^2/6,
//   c2 = 3 ypp[k] h^2/6, c3 = (ypp[k+1] - ypp[k]) h^2/6,
// formed once in FP64 so that FP32 evaluation rounds only once per term.
__device__ __forceinline__ void load_cubic(const float *c, float &c0, float &c1, float &c2, float &c3) {
  const float4 q = *reinterpret_cast<const float4 *>(c);
  c0 = q.x; c1 = q.y; c2 = q.z; c3 = q.w;
}
__device__ __forceinline__ void load_cubic(const double *c, double &c0, double &c1, double &c2, double &c3) {
  const double2 q0 = *reinterpret_cast<const double2 *>(c), q1 = *reinterpret_cast<const double2 *>(c + 2);
  c0 = q0.x; c1 = q0.y; c2 = q1.x; c3 = q1.y;
}
template <typename R>
__device__ __forceinline__ R cubic_val_grad(const R *ptab, int k, R b, R invstep, R &grad) {
  R c0, c1, c2, c3;
  load_cubic(ptab + 4 * k, c0, c1, c2, c3);
  grad = (c1 + b * (R(2) * c2 + R(3) * b * c3)) * invstep;
  return c0 + b * (c1 + b * (c2 + b * c3));
}
template <typename R>
__device__ __forceinline__ R cubic_val(const R *ptab, int k, R b) {
  R c0, c1, c2, c3;
  load_cubic(ptab + 4 * k, c0, c1, c2, c3);
  return c0 + b * (c1 + b * (c2 + b * c3));
}

// spline5eq: the quintic of each interval (Spline5Eq::splint_comb,
// spline5eq.h:110-127) as six coefficients c0..c5 in the shift b, formed in
// FP64; loaded as 8-byte pairs (an interval starts on 24 or 48 bytes).
__device__ __forceinline__ void load_quintic(const float *c, float *q) {
  const float2 a = *reinterpret_cast<const float2 *>(c), b = *reinterpret_cast<const float2 *>(c + 2),
               d = *reinterpret_cast<const float2 *>(c + 4);
  q[0] = a.x; q[1] = a.y; q[2] = b.x; q[3] = b.y; q[4] = d.x; q[5] = d.y;
}
__device__ __forceinline__ void load_quintic(const double *c, double *q) {
  const double2 a = *reinterpret_cast<const double2 *>(c), b = *reinterpret_cast<const double2 *>(c + 2),
                d = *reinterpret_cast<const double2 *>(c + 4);
  q[0] = a.x; q[1] = a.y; q[2] = b.x; q[3] = b.y; q[4] = d.x; q[5] = d.y;
}
template <typename R>
__device__ __forceinline__ R quintic_val_grad(const R *ptab, int k, R b, R invstep, R &grad) {
  R c[6];
  load_quintic(ptab + 6 * k, c);
  grad = (c[1] + b * (R(2) * c[2] + b * (R(3) * c[3] + b * (R(4) * c[4] + R(5) * b * c[5])))) * invstep;
  return c[0] + b * (c[1] + b * (c[2] + b * (c[3] + b * (c[4] + b * c[5]))));
}
// The piece of a spline: cubic, or -- in kernels built with Q5, for
// potentials with spline5eq splines -- quintic where the spline's own basis
// is spline5eq (`q5`, its SplineGeom flag; the reference picks the basis per
// function, pot_fns.cpp:439-465, with the virtual Spline path for mixed
// potentials, pot_meam_spline.cpp:56-73).
template <bool Q5, typename R>
__device__ __forceinline__ R piece_val_grad(const R *ptab, int k, R b, R invstep, R &grad, int q5) {
  if constexpr (Q5) {
    if (q5) return quintic_val_grad<R>(ptab, k, b, invstep, grad);
  }
  return cubic_val_grad<R>(ptab, k, b, invstep, grad);
}
// The spline's basis is quintic (only in kernels built with Q5).
template <bool Q5>
__device__ __forceinline__ bool quintic_of(const SplineGeom &g) {
  if constexpr (Q5) return g.q5 != 0;
  else return false;
}

// Weights of the value (w*) and of the slope (d*) on the table entries
// y[k], y[k+1], ypp[k], ypp[k+1] at shift b -- the transposes of the two
// formulas above, used by the adjoint.
template <typename R>
struct SplW {
  R wa, wb, wA, wB, da, db, dA, dB;
};
template <typename R>
__device__ __forceinline__ SplW<R> spl_weights(R b, R step, R invstep) {
  SplW<R> w;
  const R a = R(1) - b, h6 = step / R(6), hh6 = step * step / R(6);
  w.wa = a;
  w.wb = b;
  w.wA = (a * a * a - a) * hh6;
  w.wB = (b * b * b - b) * hh6;
  w.da = -invstep;
  w.db = invstep;
  w.dA = -(R(3) * a * a - R(1)) * h6;
  w.dB = (R(3) * b * b - R(1)) * h6;
  return w;
}

// Point evaluation with linear extrapolation beyond the end knots:
// Spline3Eq::splint_comb(double, double*) (spline3eq.h:204-236) and
// Spline3Eq::splint_grad2(double) (spline3eq.h:241-266).  FP64.
struct PointEval {
  double val, grad, grad2;
  int k;          // interval, or -1 left / -2 right of the knots
  double b;       // shift inside the interval
};
__device__ __forceinline__ PointEval spl_point5(const double *tab, const SplineGeom &g, double r) {
  // Spline5Eq::splint_comb(double, double*) and splint_grad2(double)
  // (spline5eq.h:226-291): quadratic beyond the end knots
  const double *y = tab + g.toff, *ypp = y + g.n, *ge = y + 2 * g.n, *yp4 = ge + 2, *g2 = yp4 + g.n;
  PointEval e;
  e.b = 0.0;
  if (r < g.x0) {
    e.grad = ge[0] + g2[0] * (r - g.x0);
    e.val = y[0] + ge[0] * (r - g.x0) + 0.5 * g2[0] * (r - g.x0) * (r - g.x0);
    e.grad2 = g2[0];
    e.k = -1;
    return e;
  } else if (r > g.xN) {
    e.grad = ge[1] + g2[1] * (r - g.xN);
    e.val = y[g.n - 1] + ge[1] * (r - g.xN) + 0.5 * g2[1] * (r - g.xN) * (r - g.xN);
    e.grad2 = g2[1];
    e.k = -2;
    return e;
  }
  const double dr = r - g.x0;
  int k = (dr < 0) ? 0 : int(dr * g.invstep);
  if (k >= g.n - 1) k = g.n - 2;
  const double b = (dr - k * g.step) * g.invstep, a = 1.0 - b, h = g.step;
  const double p1 = y[k], p2 = y[k + 1], d21 = ypp[k], d22 = ypp[k + 1], d41 = yp4[k], d42 = yp4[k + 1];
  e.grad = (p2 - p1) * g.invstep + ((3 * b * b - 1) * d22 - (3 * a * a - 1) * d21) * h / 6.0 +
           ((15 * b * b * b * b - 30 * b * b + 7) * d42 - (15 * a * a * a * a - 30 * a * a + 7) * d41) * (h * h * h) /
               360.0;
  e.val = a * p1 + b * p2 + ((a * a * a - a) * d21 + (b * b * b - b) * d22) * (h * h) / 6.0 +
          ((3 * a * a * a * a * a - 10 * a * a * a + 7 * a) * d41 + (3 * b * b * b * b * b - 10 * b * b * b + 7 * b) * d42) *
              (h * h * h * h) / 360.0;
  e.grad2 = a * d21 + b * d22 + ((a * a * a - a) * d41 + (b * b * b - b) * d42) * (h * h) / 6.0;
  e.k = k;
  e.b = b;
  return e;
}

__device__ __forceinline__ PointEval spl_point(const double *tab, const SplineGeom &g, double r) {
  const double *y = tab + g.toff, *ypp = y + g.n, *ge = y + 2 * g.n;
  PointEval e;
  if (r < g.x0) {
    e.grad = ge[0];
    e.val = y[0] + ge[0] * (r - g.x0);
    e.grad2 = 0.0;
    e.k = -1;
    e.b = 0.0;
    return e;
  } else if (r > g.xN) {
    e.grad = ge[1];
    e.val = y[g.n - 1] + ge[1] * (r - g.xN);
    e.grad2 = 0.0;
    e.k = -2;
    e.b = 0.0;
    return e;
  }
  const double dr = r - g.x0;
  int k = (dr < 0) ? 0 : int(dr * g.invstep);
  if (k >= g.n - 1) k = g.n - 2;
  const double b = (dr - k * g.step) * g.invstep;
  e.val = spl_val_grad<double>(y, ypp, k, b, g.step / 6.0, g.step * g.step / 6.0, g.invstep, e.grad);
  e.grad2 = (1.0 - b) * ypp[k] + b * ypp[k + 1];
  e.k = k;
  e.b = b;
  return e;
}

// The basis from the spline (kernels built with Q5) or cubic.
template <bool Q5>
__device__ __forceinline__ PointEval spl_point_t(const double *tab, const SplineGeom &g, double r) {
  if constexpr (Q5) {
    if (g.q5) return spl_point5(tab, g, r);
  }
  return spl_point(tab, g, r);
}
__device__ __noinline__ PointEval spl_point_any(const double *tab, const SplineGeom &g, double r) {
  return g.q5 ? spl_point5(tab, g, r) : spl_point(tab, g, r);
}

// spline5eq: weights of the value and the slope on y[k], y[k+1], ypp[k],
// ypp[k+1], yp4[k], yp4[k+1] at shift b (the transposes of the quintic
// piece, spline5eq.h:110-127).
template <typename R>
struct SplW5 {
  R wa, wb, wA, wB, w4a, w4b, da, db, dA, dB, d4a, d4b;
};
template <typename R>
__device__ __forceinline__ SplW5<R> spl_weights5(R b, R step, R invstep) {
  SplW5<R> w;
  const R a = R(1) - b, h = step;
  const R h6 = h / R(6), hh6 = h * h / R(6), h3 = h * h * h / R(360), h4 = h * h * h * h / R(360);
  w.wa = a;
  w.wb = b;
  w.wA = (a * a * a - a) * hh6;
  w.wB = (b * b * b - b) * hh6;
  w.w4a = (R(3) * a * a * a * a * a - R(10) * a * a * a + R(7) * a) * h4;
  w.w4b = (R(3) * b * b * b * b * b - R(10) * b * b * b + R(7) * b) * h4;
  w.da = -invstep;
  w.db = invstep;
  w.dA = -(R(3) * a * a - R(1)) * h6;
  w.dB = (R(3) * b * b - R(1)) * h6;
  w.d4a = -(R(15) * a * a * a * a - R(30) * a * a + R(7)) * h3;
  w.d4b = (R(15) * b * b * b * b - R(30) * b * b + R(7)) * h3;
  return w;
}

// Adds cv * d(value)/d(table) + cd * d(slope)/d(table) of a spline5eq point
// evaluation (quadratic beyond the ends) to the table gradient; table slice
// layout y[n], ypp[n], grad[2], yp4[n], grad2[2].
template <class Add>
__device__ __forceinline__ void spl_point_adjoint5(const SplineGeom &g, const PointEval &e, double r, double cv,
                                                   double cd, Add add) {
  const int n = g.n;
  if (e.k == -1) {  // y0 + g0 (r - x0) + g2_0 (r - x0)^2 / 2
    const double d = r - g.x0;
    add(0, cv);
    add(2 * n, cv * d + cd);
    add(3 * n + 2, cv * 0.5 * d * d + cd * d);
  } else if (e.k == -2) {
    const double d = r - g.xN;
    add(n - 1, cv);
    add(2 * n + 1, cv * d + cd);
    add(3 * n + 3, cv * 0.5 * d * d + cd * d);
  } else {
    const SplW5<double> w = spl_weights5<double>(e.b, g.step, g.invstep);
    add(e.k, cv * w.wa + cd * w.da);
    add(e.k + 1, cv * w.wb + cd * w.db);
    add(n + e.k, cv * w.wA + cd * w.dA);
    add(n + e.k + 1, cv * w.wB + cd * w.dB);
    add(2 * n + 2 + e.k, cv * w.w4a + cd * w.d4a);
    add(2 * n + 3 + e.k, cv * w.w4b + cd * w.d4b);
  }
}

// Adds cv * d(value)/d(table) + cd * d(slope)/d(table) of a point evaluation
// to the spline's table gradient `acc` (same layout as its table slice).
template <class Add>
__device__ __forceinline__ void spl_point_adjoint(const SplineGeom &g, const PointEval &e, double r, double cv,
                                                  double cd, Add add) {
  const int n = g.n;
  if (e.k == -1) {  // y0 + grad0 (r - x0)
    add(0, cv);
    add(2 * n, cv * (r - g.x0) + cd);
  } else if (e.k == -2) {
    add(n - 1, cv);
    add(2 * n + 1, cv * (r - g.xN) + cd);
  } else {
    const SplW<double> w = spl_weights<double>(e.b, g.step, g.invstep);
    add(e.k, cv * w.wa + cd * w.da);
    add(e.k + 1, cv * w.wb + cd * w.db);
    add(n + e.k, cv * w.wA + cd * w.dA);
    add(n + e.k + 1, cv * w.wB + cd * w.dB);
  }
}

// Knot + shift of cos(theta) on the g grid.  The reference bisects
// (spline.cpp:74-99); the interval found here is the same except within an
// ulp of a knot, where the spline's value and slope agree to rounding.
template <typename R>
__device__ __forceinline__ int g_knot(R c, R x0, R invstep, int n, R &b) {
  const R t = (c - x0) * invstep;
  int k = (int)floor(t);
  k = k < 0 ? 0 : (k > n - 2 ? n - 2 : k);
  b = t - R(k);
  return k;
}
// FP32: floor through the float format instead of conversion instructions.
// For 0 <= t < 2^22, t + (2^23 - 1/2) rounds to the integer 2^23 + floor(t)
// (exact halves, where t is an integer, round to even: the interval below
// with b = 1, which evaluates to the same spline value); its bit pattern
// minus that of 2^23 is floor(t).  t slightly below 0 gives -1, clamped.
template <>
__device__ __forceinline__ int g_knot<float>(float c, float x0, float invstep, int n, float &b) {
  const float t = (c - x0) * invstep;
  int k = __float_as_int(t + 8388607.5f) - 0x4B000000;
  k = k < 0 ? 0 : (k > n - 2 ? n - 2 : k);
  b = t - (__int_as_float(k + 0x4B000000) - 8388608.0f);
  return k;
}

// cos(theta) exactly as Triplet::setup_triplet: x*x' + y*y' + z*z' with no
// fused multiply-add (triplet.cpp:34-40, vect.h:137-141).
__device__ __forceinline__ double cos_exact(double ax, double ay, double az, double bx, double by, double bz) {
  return __dadd_rn(__dadd_rn(__dmul_rn(ax, bx), __dmul_rn(ay, by)), __dmul_rn(az, bz));
}
__device__ __forceinline__ float cos_exact(float ax, float ay, float az, float bx, float by, float bz) {
  return __fadd_rn(__fadd_rn(__fmul_rn(ax, bx), __fmul_rn(ay, by)), __fmul_rn(az, bz));
}

// Upper cut of the g grid in the kernel's arithmetic.  FP64 uses the
// reference's x_N (1 + 1e-8) (spline.cpp:79).  In FP32 a cosine of
// collinear neighbours rounds to 1.0f, which must stay a triplet as it is in
// FP64, so the cut is widened by a few FP32 ulps.
template <typename R>
__device__ __forceinline__ R g_cut(const SplineGeom &g);
template <>
__device__ __forceinline__ double g_cut<double>(const SplineGeom &g) {
  return g.cut;
}
template <>
__device__ __forceinline__ float g_cut<float>(const SplineGeom &g) {
  return g.cutf;
}

}  // namespace mzb
