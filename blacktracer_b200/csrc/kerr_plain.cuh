// kerr_plain.cuh -- FP64 Kerr null-geodesic integrator, "plain" form.
//
// Device restatement of the reference integrator (annemiekie/BlackTracer
// BT/Metric.h:198-324 and the ray set-up of BT/Grid.h:524-554) that keeps
// the reference's arithmetic expression trees term for term, so that with
// FMA contraction disabled (this header is only compiled with --fmad=false)
// every +, -, *, /, sqrt rounds exactly as the reference's host build.  The
// only differences come from the device libm's sin/cos/pow, which may differ
// from the host libm by an ulp.  The Cash-Karp tableau is the published one
// (Numerical Recipes, BT/Metric.h:41-49).
//
// State layout: y[0..4] = {r, theta, phi, p_r, p_theta}; b = p_phi, q = the
// Carter constant.  One ray per thread; everything lives in registers.
#pragma once

#include "bt_internal.h"

namespace bt {
namespace plain {

// Step control (BT/Metric.h:27-33).
constexpr double kSafety = 0.9, kPGrow = -0.2, kPShrnk = -0.25;
constexpr double kErrCon = 1.89e-4, kTiny = 1.0e-30, kAdaptive = 5.0;

// Cash-Karp 5(4) tableau.
constexpr double b21 = 0.2, b31 = 3.0 / 40.0, b32 = 9.0 / 40.0, b41 = 0.3,
                 b42 = -0.9, b43 = 1.2, b51 = -11.0 / 54.0, b52 = 2.5,
                 b53 = -70.0 / 27.0, b54 = 35.0 / 27.0,
                 b61 = 1631.0 / 55296.0, b62 = 175.0 / 512.0,
                 b63 = 575.0 / 13824.0, b64 = 44275.0 / 110592.0,
                 b65 = 253.0 / 4096.0, c1 = 37.0 / 378.0, c3 = 250.0 / 621.0,
                 c4 = 125.0 / 594.0, c6 = 512.0 / 1771.0,
                 dc5 = -277.00 / 14336.0;
constexpr double dc1 = 37.0 / 378.0 - 2825.0 / 27648.0,
                 dc3 = 250.0 / 621.0 - 18575.0 / 48384.0,
                 dc4 = 125.0 / 594.0 - 13525.0 / 55296.0,
                 dc6 = 512.0 / 1771.0 - 0.25;

__device__ __forceinline__ double sqd(double x) { return x * x; }

// Equations of motion (BT/Metric.h:198-226).  Sub-expressions keep the
// reference's association: Delta = (r^2 - 2r) + a^2, rho^2 = r^2 + a^2 cos^2,
// P = (r^2 + a^2) - a b, R = P^2 - Delta((b-a)^2 + q),
// Theta = q - cos^2 (b^2/sin^2 - a^2).
//
// Kept out of line: an attempt evaluates it five times (and the step start
// once more), and each evaluation holds about sixteen IEEE divisions and a
// sincos, so inlining every call site makes the ray loop larger than the
// instruction cache.  One copy, called six times, keeps it resident; the
// arithmetic is the same either way.
struct Slope {
  double f0, f1, f2, f3, f4;
};

static __device__ __noinline__ Slope eom_call(double r, double th, double pr, double pt,
                                       double b, double q, double a, double asq) {
  double f[5];
  double sinv, cosv;
  sincos(th, &sinv, &cosv);
  const double cossq = sqd(cosv);
  const double sinsq = sqd(sinv);
  const double bsq = sqd(b);
  const double delta = sqd(r) - 2. * r + asq;
  const double rosq = sqd(r) + asq * sqd(cosv);
  const double P = sqd(r) + asq - a * b;
  const double prsq = sqd(pr);
  const double ptsq = sqd(pt);
  const double R = sqd(P) - delta * (sqd((b - a)) + q);
  const double partR = (q + sqd(a - b));
  const double bth = q - sqd(cosv) * (sqd(b) / sqd(sinv) - asq);
  const double rosqsq = sqd(2 * rosq);
  const double sqrosqdel = (sqd(rosq) * delta);
  const double acs = asq * cosv * sinv;
  const double rtwo = 2 * r - 2;

  f[0] = delta / rosq * pr;
  f[1] = 1. / rosq * pt;
  f[2] = (2 * a * P - (2 * a - 2 * b) * delta + (2 * b * cossq * delta) / sinsq) /
         (rosq * 2 * delta);
  f[3] = (rtwo * bth - rtwo * partR + 4 * r * P) / (rosq * (2 * delta)) -
         (prsq * rtwo) / (2 * rosq) + (4 * ptsq * r) / rosqsq -
         ((4 * r - 4) * (bth * (delta) + R)) / (rosq * sqd(2 * delta)) +
         (4 * prsq * r * (delta)) / rosqsq - (r * (bth * delta + R)) / sqrosqdel;
  f[4] = ((2 * cosv * sinv * (bsq / sinsq - asq) +
           (2 * bsq * (cosv * cosv * cosv)) / (sinv * sinv * sinv)) * delta) /
             (rosq * 2 * delta) -
         (4 * acs * ptsq) / rosqsq - (4 * acs * prsq * delta) / rosqsq +
         (acs * (bth * delta + R)) / sqrosqdel;
  return Slope{f[0], f[1], f[2], f[3], f[4]};
}

__device__ __forceinline__ void eom(const double* y, double* f, double b,
                                    double q, double a, double asq) {
  const Slope s = eom_call(y[0], y[1], y[3], y[4], b, q, a, asq);
  f[0] = s.f0;
  f[1] = s.f1;
  f[2] = s.f2;
  f[3] = s.f3;
  f[4] = s.f4;
}

// The equations of motion an attempt uses (the reference's by default).
struct EomPlain {
  static __device__ __forceinline__ void f(const double* y, double* o, double b, double q,
                                           double a, double asq) {
    eom(y, o, b, q, a, asq);
  }
};

// One Cash-Karp attempt (BT/Metric.h:228-251).  Stage slopes k1..k5 are
// the reference's aks[0..4], [5..9], ..., [20..24].
template <class E = EomPlain>
__device__ __forceinline__ void ck_attempt(const double* y, const double* d,
                                           double h, double* yo, double* err,
                                           double b, double q, double a,
                                           double asq) {
  double k1[5], k2[5], k3[5], k4[5], k5[5], t[5];
#pragma unroll
  for (int i = 0; i < 5; i++) t[i] = y[i] + b21 * h * d[i];
  E::f(t, k1, b, q, a, asq);
#pragma unroll
  for (int i = 0; i < 5; i++) t[i] = y[i] + h * (b31 * d[i] + b32 * k1[i]);
  E::f(t, k2, b, q, a, asq);
#pragma unroll
  for (int i = 0; i < 5; i++)
    t[i] = y[i] + h * (b41 * d[i] + b42 * k1[i] + b43 * k2[i]);
  E::f(t, k3, b, q, a, asq);
#pragma unroll
  for (int i = 0; i < 5; i++)
    t[i] = y[i] + h * (b51 * d[i] + b52 * k1[i] + b53 * k2[i] + b54 * k3[i]);
  E::f(t, k4, b, q, a, asq);
#pragma unroll
  for (int i = 0; i < 5; i++)
    t[i] = y[i] + h * (b61 * d[i] + b62 * k1[i] + b63 * k2[i] + b64 * k3[i] +
                       b65 * k4[i]);
  E::f(t, k5, b, q, a, asq);
#pragma unroll
  for (int i = 0; i < 5; i++) {
    yo[i] = y[i] + h * (c1 * d[i] + c3 * k2[i] + c4 * k3[i] + c6 * k5[i]);
    err[i] = h * (dc1 * d[i] + dc3 * k2[i] + dc4 * k3[i] + dc5 * k4[i] +
                  dc6 * k5[i]);
  }
}

// Capture classification (BT/Metric.h:110-174).  Returns 1 = celestial
// (integrate), 0 = captured, -1 = Newton loop exceeded its cap.
constexpr int kNewtonCap = 100000;
constexpr int kGoldCap = 200;

__device__ __forceinline__ double Rpot(double r, double b, double q, double a,
                                       double asq) {
  const double P = sqd(r) + asq - a * b;
  return sqd(P) - (sqd(r) - 2. * r + asq) * (sqd((b - a)) + q);
}

__device__ __forceinline__ int celestial(const RayParams& p, double pR,
                                         double b, double q,
                                         double* r0_out = nullptr) {
  const double a = p.a, asq = p.asq;
  // checkB_Q: Newton for the spherical photon orbit radius r0 with b0(r0)=b
  double r0 = 2.0, bcheck = 100;
  int it = 0;
  while (fabs(b - bcheck) > 0.0000001) {
    if (++it > kNewtonCap) return -1;
    bcheck = -(r0 * r0 * r0 - 3. * sqd(r0) + asq * r0 + asq) / (a * (r0 - 1.));
    const double bd =
        (asq + a - 2. * r0 * (sqd(r0) - 3. * r0 + 3.)) / (a * sqd(r0 - 1.));
    const double rn = r0 - (bcheck - b) / bd;
    r0 = rn < 1 ? 1.0001 : rn;
  }
  const double qb = -(r0 * r0 * r0) *
                    (r0 * r0 * r0 - 6. * sqd(r0) + 9. * r0 - 4. * asq) /
                    (asq * sqd(r0 - 1.));
  if (r0_out) *r0_out = r0;
  const bool c1 = (p.b_lo >= b) || (p.b_hi <= b) || (q >= qb);
  if (!c1) return pR < 0 ? 1 : 0;
  // checkRup: golden-section minimum of R on [r, 4r]; R(min) >= 0 -> turns
  if (a == 0) return 0;
  const double gr = (sqrt(5.0) + 1.) / 2.;
  double lo = p.rS, hi = 4 * p.rS;
  double c = hi - (hi - lo) / gr;
  double dd = lo + (hi - lo) / gr;
  int g = 0;
  while (fabs(c - dd) > 0.00001 && g++ < kGoldCap) {
    if (Rpot(c, b, q, a, asq) < Rpot(dd, b, q, a, asq)) hi = dd;
    else lo = c;
    c = hi - (hi - lo) / gr;
    dd = lo + (hi - lo) / gr;
  }
  return Rpot((lo + hi) / 2, b, q, a, asq) >= 0 ? 1 : 0;
}

// wrapToPi (BT/Metric.h:176-185).  The reference's `while (phi < 0)
// phi += 2pi` never ends for phi = -inf and takes ~|phi|/2pi turns; here it
// is bounded (identical results whenever it ends within 4096 turns).
constexpr int kWrapCap = 4096;
__device__ __forceinline__ void wrap_to_pi(double& th, double& ph) {
  th = fmod(th, kPi2);
  while (th < 0) th += kPi2;
  if (th > kPi) {
    th -= 2 * (th - kPi);
    ph += kPi;
  }
  for (int it = 0; ph < 0; it++) {
    if (it == kWrapCap) {
      ph = fmod(ph, kPi2) + kPi2;  // NaN for -inf
      break;
    }
    ph += kPi2;
  }
  ph = fmod(ph, kPi2);
}

// Initial momenta of a camera-sky direction (BT/Grid.h:524-547):
// camera frame -> boosted FIDO frame -> rotated by (br, btheta, bphi).
__device__ __forceinline__ void ray_setup(const RayParams& p, double th,
                                          double ph, double& pR,
                                          double& pTheta, double& b,
                                          double& q) {
  double st, ct, sp_, cp;
  sincos(th, &st, &ct);
  sincos(ph, &sp_, &cp);
  const double xCam = st * cp;
  const double yCam = st * sp_;
  const double zCam = ct;
  const double sp = p.sp;
  const double yFido = (-yCam + sp) / (1 - sp * yCam);
  const double xFido = -p.sqrt_1msp2 * xCam / (1 - sp * yCam);
  const double zFido = -p.sqrt_1msp2 * zCam / (1 - sp * yCam);
  const double k = p.kb;
  const double rFido =
      xFido * p.bphi / k + p.br * yFido + p.br * p.btheta / k * zFido;
  const double thetaFido = p.btheta * yFido - k * zFido;
  const double phiFido =
      -xFido * p.br / k + p.bphi * yFido + p.bphi * p.btheta / k * zFido;
  const double eF = 1. / (p.alpha + p.w * p.wbar * phiFido);
  pR = eF * p.ro * rFido / p.sqrtf_delta;
  pTheta = eF * p.ro * thetaFido;
  const double pPhi = eF * p.wbar * phiFido;
  b = pPhi;
  q = pTheta * pTheta + p.cosS2 * (b * b / p.sinS2 - p.asq);
}

// Per-ray integration state of odeint1 (BT/Metric.h:276-303).
struct RayState {
  double y[5];
  double z, h, b, q;
  int32_t nstp, step;
};

// The result of a ray's set-up and capture test when it must be integrated:
// initial momenta, the constants of motion and the spherical photon-orbit
// radius of its b (the capture test's Newton solution).
struct RayStart {
  double pR, pTheta, b, q, r0;
};

// Set-up + capture test of one ray (BT/Grid.h:524-552).  Returns true when
// the ray must be integrated (rs filled); otherwise tho/pho/steps/status are
// final.
__device__ __forceinline__ bool setup_ray(const RayParams& p, double th, double ph,
                                          RayStart& rs, double& tho, double& pho,
                                          int32_t& steps, uint8_t& status) {
  double pR, pTheta, b, q;
  ray_setup(p, th, ph, pR, pTheta, b, q);
  tho = -1;
  pho = -1;
  steps = 0;
  double r0 = 0;
  const int cel = celestial(p, pR, b, q, &r0);
  if (cel <= 0) {
    status = cel < 0 ? BT_RAY_NONCONVERGED : BT_RAY_CAPTURED;
    return false;
  }
  rs.pR = pR;
  rs.pTheta = pTheta;
  rs.b = b;
  rs.q = q;
  rs.r0 = r0;
  return true;
}

// odeint1's start state (BT/Metric.h:276-281, rkckIntegrate1 :307-324).
__device__ __forceinline__ void start_ray(const RayParams& p, const RayStart& rs,
                                          RayState& s) {
  s.y[0] = p.rS; s.y[1] = p.thetaS; s.y[2] = p.phiS; s.y[3] = rs.pR;
  s.y[4] = rs.pTheta;
  s.z = 0.0;
  s.h = p.h1 * (p.z_end > 0 ? 1 : (p.z_end < 0 ? -1 : 0));
  s.b = rs.b;
  s.q = rs.q;
  s.nstp = 0;
  s.step = 0;
}

__device__ __forceinline__ bool begin_ray(const RayParams& p, double th,
                                          double ph, RayState& s, double& tho,
                                          double& pho, int32_t& steps,
                                          uint8_t& status,
                                          double* r0_out = nullptr) {
  RayStart rs;
  if (!setup_ray(p, th, ph, rs, tho, pho, steps, status)) return false;
  if (r0_out) *r0_out = rs.r0;
  start_ray(p, rs, s);
  return true;
}

// One quality-controlled attempt (odeint1 loop body + rkqs,
// BT/Metric.h:291-302, 253-270).  Returns true when the ray is finished
// (end point reached or attempt cap hit).
template <class E = EomPlain>
__device__ __forceinline__ bool attempt(const RayParams& p, RayState& s) {
  double d[5], scal[5], yt[5], err[5];
  E::f(s.y, d, s.b, s.q, p.a, p.asq);
#pragma unroll
  for (int i = 0; i < 5; i++) scal[i] = fabs(s.y[i]) + fabs(d[i] * s.h) + kTiny;
  ck_attempt<E>(s.y, d, s.h, yt, err, s.b, s.q, p.a, p.asq);
  double errmax = 0.0;
#pragma unroll
  for (int i = 0; i < 5; i++) errmax = fmax(errmax, fabs(err[i] / scal[i]));
  errmax /= p.eps;
  if (errmax <= 1.0) {
    s.z += s.h;
#pragma unroll
    for (int i = 0; i < 5; i++) s.y[i] = yt[i];
    s.h = errmax > kErrCon ? kSafety * s.h * pow(errmax, kPGrow)
                           : kAdaptive * s.h;
  } else {
    s.h = fmin(kSafety * s.h * pow(errmax, kPShrnk), 0.1 * s.h);
  }
  s.step = s.nstp;
  s.nstp++;
  return s.z <= p.z_end || s.nstp >= p.maxstp;
}

// odeint1's state plus the slope at the start of the step.  After a
// rejected attempt the state is unchanged, and the reference's next
// iteration recomputes derivs from the same values (BT/Metric.h:292): the
// slope is kept instead, which gives the same results.
struct CachedState : RayState {
  double d[5];
  bool dv;  // d holds the slope of y
};

__device__ __forceinline__ bool begin_ray_cached(const RayParams& p, double th, double ph,
                                                 CachedState& s, double& tho, double& pho,
                                                 int32_t& steps, uint8_t& status) {
  s.dv = false;
  return begin_ray(p, th, ph, s, tho, pho, steps, status);
}

__device__ __forceinline__ void start_ray_cached(const RayParams& p, const RayStart& rs,
                                                 CachedState& s) {
  s.dv = false;
  start_ray(p, rs, s);
}

// Step-size update of rkqs (BT/Metric.h:262-268) with one pow for both
// outcomes, so that lanes that accept and lanes that reject do not run it
// one after the other (the values are those of the two separate calls).
__device__ __forceinline__ void update_step(RayState& s, double errmax) {
  const bool ok = errmax <= 1.0;
  const double pw = pow(errmax, ok ? kPGrow : kPShrnk);
  if (ok) s.h = errmax > kErrCon ? kSafety * s.h * pw : kAdaptive * s.h;
  else s.h = fmin(kSafety * s.h * pw, 0.1 * s.h);
}

template <class E = EomPlain>
__device__ __forceinline__ bool attempt_cached(const RayParams& p, CachedState& s) {
  double scal[5], yt[5], err[5];
  if (!s.dv) {
    E::f(s.y, s.d, s.b, s.q, p.a, p.asq);
    s.dv = true;
  }
#pragma unroll
  for (int i = 0; i < 5; i++) scal[i] = fabs(s.y[i]) + fabs(s.d[i] * s.h) + kTiny;
  ck_attempt<E>(s.y, s.d, s.h, yt, err, s.b, s.q, p.a, p.asq);
  double errmax = 0.0;
#pragma unroll
  for (int i = 0; i < 5; i++) errmax = fmax(errmax, fabs(err[i] / scal[i]));
  errmax /= p.eps;
  if (errmax <= 1.0) {
    s.z += s.h;
#pragma unroll
    for (int i = 0; i < 5; i++) s.y[i] = yt[i];
    s.dv = false;
  }
  update_step(s, errmax);
  s.step = s.nstp;
  s.nstp++;
  return s.z <= p.z_end || s.nstp >= p.maxstp;
}

// Outputs of a finished ray.  odeint1 copies the state back only when z
// reached the end point; otherwise the start angles come back
// (BT/Metric.h:298-302).  Then wrapToPi (BT/Metric.h:322).
__device__ __forceinline__ void finish_ray(const RayParams& p,
                                           const RayState& s, double& tho,
                                           double& pho, int32_t& steps,
                                           uint8_t& status) {
  const bool done = s.z <= p.z_end;
  double to = done ? s.y[1] : p.thetaS;
  double po = done ? s.y[2] : p.phiS;
  wrap_to_pi(to, po);
  tho = to;
  pho = po;
  steps = s.step;
  status = done ? BT_RAY_ESCAPED : BT_RAY_MAXSTEP;
}

}  // namespace plain
}  // namespace bt
