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
// with W = Theta Delta + R.  Results agree with the plain form to rounding
// level (they are not bit-identical).
#pragma once

#include "kerr_plain.cuh"

namespace bt {
namespace fast {

static __device__ __noinline__ plain::Slope eom_fast(double r, double th, double pr,
                                                     double pt, double b, double q,
                                                     double a, double asq) {
  double sinv, cosv;
  sincos(th, &sinv, &cosv);
  const double cossq = cosv * cosv;
  const double bsq = b * b;
  const double delta = r * r - 2. * r + asq;
  const double rosq = r * r + asq * cossq;
  const double P = r * r + asq - a * b;
  const double prsq = pr * pr, ptsq = pt * pt;
  const double R = P * P - delta * ((b - a) * (b - a) + q);
  const double partR = q + (a - b) * (a - b);
  const double ir = 1. / rosq, id = 1. / delta, is = 1. / sinv;
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

struct EomFast {
  static __device__ __forceinline__ void f(const double* y, double* o, double b, double q,
                                           double a, double asq) {
    const plain::Slope s = eom_fast(y[0], y[1], y[3], y[4], b, q, a, asq);
    o[0] = s.f0;
    o[1] = s.f1;
    o[2] = s.f2;
    o[3] = s.f3;
    o[4] = s.f4;
  }
};

__device__ __forceinline__ bool attempt(const RayParams& p, plain::RayState& s) {
  return plain::attempt<EomFast>(p, s);
}

__device__ __forceinline__ void integrate_ray(const RayParams& p, double th, double ph,
                                              double& tho, double& pho, int32_t& steps,
                                              uint8_t& status) {
  plain::RayState s;
  if (!plain::begin_ray(p, th, ph, s, tho, pho, steps, status)) return;
  if (p.maxstp > 0)
    while (!attempt(p, s)) {
    }
  plain::finish_ray(p, s, tho, pho, steps, status);
}

}  // namespace fast
}  // namespace bt
