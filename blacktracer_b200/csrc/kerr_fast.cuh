// kerr_fast.cuh -- "fast" FP64 form of the Kerr geodesic integrator.
//
// The reference's method unchanged (Cash-Karp 5(4), its step control,
// tolerance, end point and capture test), all in FP64, with the equations
// of motion (BT/Metric.h:198-226) rewritten around three reciprocals --
// 1/rho^2, 1/Delta, 1/sin(theta) -- instead of the sixteen divisions of the
// reference's expression, and compiled with FMA contraction.  Each term is
// the reference's term with its divisions turned into products:
//   f2 = (2aP - (2a - 2b) Delta) / (2 rho^2 Delta) + b cos^2 / (sin^2 rho^2)
//   f3 = (rtwo (Theta - partR) + 4 r P) / (2 rho^2 Delta) - p_r^2 rtwo / (2 rho^2)
//        + p_th^2 r / rho^4 - (r - 1) W / (rho^2 Delta^2) + p_r^2 r Delta / rho^4
//        - r W / (rho^4 Delta)
//   f4 = (cos sin (b^2/sin^2 - a^2) + b^2 cos^3/sin^3) / rho^2
//        - a^2 cos sin (p_th^2 + p_r^2 Delta) / rho^4 + a^2 cos sin W / (rho^4 Delta)
// with W = Theta Delta + R.  Within a step, sin and cos of each stage's theta
// come from those at the start of the step by angle addition (rotate), the
// slope at the start of a step is kept across a rejected attempt, the
// step-size factor and the error ratio are computed in FP32, and the three
// reciprocals use an approximate reciprocal refined by Newton-Raphson.
// Results agree with the plain form to rounding level (they are not
// bit-identical).
#pragma once

#include "kerr_plain.cuh"

namespace bt {
namespace fast {

// 1/x by the hardware's approximate reciprocal (PTX rcp.approx.ftz.f64)
// refined by one Newton-Raphson step, r <- r + r (1 - x r), which squares
// its relative error: two dependent FMAs instead of a correctly rounded
// division.  A second step changed the C2 grid by less than its rounding
// (p99 against the plain form 1.4e-10 rad with it, 1.9e-10 without, the same
// topology) and cost 1.5-2% of the build time.
__device__ __forceinline__ double rcp_nr(double x) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  return fma(r, fma(-x, r, 1.0), r);
}

// The equations of motion from sin and cos of theta (theta itself enters
// only through them).
static __device__ __forceinline__ plain::Slope eom_fast_sc(double r, double sinv, double cosv,
                                                        double pr, double pt, double b,
                                                        double q, double a, double asq) {
  const double cossq = cosv * cosv;
  const double bsq = b * b;
  const double delta = r * r - 2. * r + asq;
  const double rosq = r * r + asq * cossq;
  const double P = r * r + asq - a * b;
  const double prsq = pr * pr, ptsq = pt * pt;
  const double R = P * P - delta * ((b - a) * (b - a) + q);
  const double partR = q + (a - b) * (a - b);
  const double ir = rcp_nr(rosq), id = rcp_nr(delta), is = rcp_nr(sinv);
  const double is2 = is * is;
  const double ir2 = ir * ir;
  const double bth = q - cossq * (bsq * is2 - asq);
  const double W = bth * delta + R;
  const double rtwo = 2. * r - 2.;
  const double acs = asq * cosv * sinv;
  const double hrd = 0.5 * ir * id;
  plain::Slope o;
  o.f0 = delta * ir * pr;
  o.f1 = ir * pt;
  o.f2 = (2. * a * P - (2. * a - 2. * b) * delta) * hrd + b * cossq * is2 * ir;
  o.f3 = (rtwo * (bth - partR) + 4. * r * P) * hrd - 0.5 * prsq * rtwo * ir +
         ptsq * r * ir2 - (r - 1.) * W * ir * id * id + prsq * r * delta * ir2 -
         r * W * ir2 * id;
  o.f4 = (cosv * sinv * (bsq * is2 - asq) + bsq * cossq * cosv * is2 * is) * ir -
         acs * (ptsq + prsq * delta) * ir2 + acs * W * ir2 * id;
  return o;
}

__device__ __forceinline__ void put(const plain::Slope& s, double* o) {
  o[0] = s.f0;
  o[1] = s.f1;
  o[2] = s.f2;
  o[3] = s.f3;
  o[4] = s.f4;
}

// Per-ray state: odeint1's, plus the slope at the start of the step and sin
// and cos of its theta, kept across a rejected attempt (the state does not
// change; the reference recomputes the same values).
struct FastState : plain::RayState {
  double d[5];
  double sn, cs;  // sin, cos of y[1]
  bool dv;
};

// Stage increments of theta above this take a full sincos.
constexpr double kRotMax = 0.125;

// sin and cos of theta + dt from those of theta, by the angle-addition
// formulas with the Taylor series of sin(dt) and cos(dt) - 1 (through dt^7
// and dt^8: the next terms are below 2.1e-14 and 2.7e-16 for |dt| <= 1/8).
// The stages of a step move theta by small amounts; this replaces five of
// the six FP64 sincos evaluations of an attempt.
__device__ __forceinline__ void rotate(double sn, double cs, double dt, double& s, double& c) {
  const double x2 = dt * dt;
  const double sd = dt * (1. + x2 * (-1. / 6. + x2 * (1. / 120. + x2 * (-1. / 5040.))));
  const double cm1 = x2 * (-0.5 + x2 * (1. / 24. + x2 * (-1. / 720. + x2 * (1. / 40320.))));
  s = sn + (sn * cm1 + cs * sd);
  c = cs + (cs * cm1 - sn * sd);
}

// Slope at stage point t whose theta is theta_0 + dt.
__device__ __forceinline__ void stage_slope(const double* t, double dt, double sn0,
                                            double cs0, double b, double q, double a,
                                            double asq, double* o) {
  double sn, cs;
  if (fabs(dt) <= kRotMax) {
    rotate(sn0, cs0, dt, sn, cs);
  } else {
    sincos(t[1], &sn, &cs);
  }
  put(eom_fast_sc(t[0], sn, cs, t[3], t[4], b, q, a, asq), o);
}

// One Cash-Karp attempt (BT/Metric.h:228-251) in the fast form.
__device__ __forceinline__ void ck_attempt(const FastState& S, double h, double* yo,
                                           double* err, double a, double asq) {
  using namespace plain;
  const double* y = S.y;
  const double* d = S.d;
  const double b = S.b, q = S.q;
  double k1[5], k2[5], k3[5], k4[5], k5[5], t[5], dt;
#pragma unroll
  for (int i = 0; i < 5; i++) t[i] = y[i] + b21 * h * d[i];
  dt = b21 * h * d[1];
  stage_slope(t, dt, S.sn, S.cs, b, q, a, asq, k1);
#pragma unroll
  for (int i = 0; i < 5; i++) t[i] = y[i] + h * (b31 * d[i] + b32 * k1[i]);
  dt = h * (b31 * d[1] + b32 * k1[1]);
  stage_slope(t, dt, S.sn, S.cs, b, q, a, asq, k2);
#pragma unroll
  for (int i = 0; i < 5; i++)
    t[i] = y[i] + h * (b41 * d[i] + b42 * k1[i] + b43 * k2[i]);
  dt = h * (b41 * d[1] + b42 * k1[1] + b43 * k2[1]);
  stage_slope(t, dt, S.sn, S.cs, b, q, a, asq, k3);
#pragma unroll
  for (int i = 0; i < 5; i++)
    t[i] = y[i] + h * (b51 * d[i] + b52 * k1[i] + b53 * k2[i] + b54 * k3[i]);
  dt = h * (b51 * d[1] + b52 * k1[1] + b53 * k2[1] + b54 * k3[1]);
  stage_slope(t, dt, S.sn, S.cs, b, q, a, asq, k4);
#pragma unroll
  for (int i = 0; i < 5; i++)
    t[i] = y[i] + h * (b61 * d[i] + b62 * k1[i] + b63 * k2[i] + b64 * k3[i] + b65 * k4[i]);
  dt = h * (b61 * d[1] + b62 * k1[1] + b63 * k2[1] + b64 * k3[1] + b65 * k4[1]);
  stage_slope(t, dt, S.sn, S.cs, b, q, a, asq, k5);
#pragma unroll
  for (int i = 0; i < 5; i++) {
    yo[i] = y[i] + h * (c1 * d[i] + c3 * k2[i] + c4 * k3[i] + c6 * k5[i]);
    err[i] = h * (dc1 * d[i] + dc3 * k2[i] + dc4 * k3[i] + dc5 * k4[i] + dc6 * k5[i]);
  }
}

__device__ __forceinline__ bool begin_ray(const RayParams& p, double th, double ph,
                                          FastState& s, double& tho, double& pho,
                                          int32_t& steps, uint8_t& status) {
  s.dv = false;
  return plain::begin_ray(p, th, ph, s, tho, pho, steps, status);
}

__device__ __forceinline__ void start_ray(const RayParams& p, const plain::RayStart& rs,
                                          FastState& s) {
  s.dv = false;
  plain::start_ray(p, rs, s);
}

// One quality-controlled attempt (odeint1 loop body + rkqs, BT/Metric.h
// :291-302, 253-270) in the fast form.
__device__ __forceinline__ bool attempt(const RayParams& p, FastState& s) {
  using namespace plain;
  double scal[5], yt[5], err[5];
  if (!s.dv) {
    sincos(s.y[1], &s.sn, &s.cs);
    put(eom_fast_sc(s.y[0], s.sn, s.cs, s.y[3], s.y[4], s.b, s.q, p.a, p.asq), s.d);
    s.dv = true;
  }
#pragma unroll
  for (int i = 0; i < 5; i++) scal[i] = fabs(s.y[i]) + fabs(s.d[i] * s.h) + kTiny;
  ck_attempt(s, s.h, yt, err, p.a, p.asq);
  // the error ratio only decides acceptance and steers the step size:
  // FP32 (~1e-7 relative) instead of five FP64 divisions
  float em = 0.f;
#pragma unroll
  for (int i = 0; i < 5; i++) em = fmaxf(em, fabsf((float)err[i] / (float)scal[i]));
  const double errmax = (double)(em / (float)p.eps);
  if (errmax <= 1.0) {
    s.z += s.h;
#pragma unroll
    for (int i = 0; i < 5; i++) s.y[i] = yt[i];
    s.dv = false;
  }
  // rkqs's step-size update (BT/Metric.h:262-268) with the growth / shrink
  // factor errmax^-0.2 / errmax^-0.25 in FP32: the factor only steers the
  // next step (its error is that of the step-size heuristic, ~1e-7
  // relative), and an FP64 pow is the longest dependent chain of an attempt
  const bool ok = errmax <= 1.0;
  const double pw = (double)powf((float)errmax, ok ? -0.2f : -0.25f);
  if (ok) s.h = errmax > kErrCon ? kSafety * s.h * pw : kAdaptive * s.h;
  else s.h = fmin(kSafety * s.h * pw, 0.1 * s.h);
  s.step = s.nstp;
  s.nstp++;
  return s.z <= p.z_end || s.nstp >= p.maxstp;
}

}  // namespace fast
}  // namespace bt
