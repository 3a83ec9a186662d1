// kerr_mixed.cuh -- mixed-precision form of the Kerr geodesic integrator.
//
// Same method as the reference (BT/Metric.h: Cash-Karp 5(4), the same
// step-control constants, tolerance and end point, the same analytic capture
// test) with the arithmetic split by where precision matters:
//   * FP64: the state y, the affine parameter z and the step h (so phi
//     accumulates over many windings in FP64), the capture classification
//     (plain::celestial), and whole attempts that
//       - start or end within fp64_band of the ray's spherical photon-orbit
//         radius r0 (from the capture test's Newton solve),
//       - cross a radial or polar turning point (p_r or p_theta changes sign,
//         i.e. R(r) or Theta(theta) passes through zero),
//       - start beyond r = 1e8 (FP32 range guard).
//   * FP32: everything else -- the six equation-of-motion evaluations of an
//     attempt, the stage combinations, the error estimate and the step-size
//     power law.  The FP32 equations use 3 reciprocals instead of 17
//     divisions and are ordered so that no intermediate overflows for
//     r < 1e8.
#pragma once

#include "kerr_plain.cuh"

namespace bt {
namespace mixed {

__device__ __forceinline__ float sqf(float x) { return x * x; }

// Equations of motion in FP32 (physics of BT/Metric.h:198-226).
__device__ __forceinline__ void eom_f(const float* y, float* f, float b,
                                      float q, float a, float asq) {
  const float r = y[0], pr = y[3], pt = y[4];
  float sn, cs;
  sincosf(y[1], &sn, &cs);
  const float cs2 = cs * cs;
  const float sn2 = sn * sn;
  const float isn2 = 1.0f / sn2;
  const float bsq = b * b;
  const float delta = r * r - 2.f * r + asq;
  const float rosq = r * r + asq * cs2;
  const float P = r * r + asq - a * b;
  const float R = P * P - delta * (sqf(b - a) + q);
  const float partR = q + sqf(a - b);
  const float bth = q - cs2 * (bsq * isn2 - asq);
  const float ir = 1.0f / rosq;
  const float id = 1.0f / delta;
  const float prsq = pr * pr, ptsq = pt * pt;
  const float acs = asq * cs * sn;
  const float rtwo = 2.f * r - 2.f;
  const float rir = r * ir;
  const float W = (bth * delta + R) * ir;  // (Theta Delta + R) / rho^2
  f[0] = delta * ir * pr;
  f[1] = ir * pt;
  f[2] = ((2.f * a * P - (2.f * a - 2.f * b) * delta) * id +
          2.f * b * cs2 * isn2) * (0.5f * ir);
  const float T1 = (rtwo * bth - rtwo * partR + 4.f * r * P) * ir * (0.5f * id);
  const float T2 = prsq * rtwo * (0.5f * ir);
  const float T3 = ptsq * ir * rir;
  const float T4 = ((r - 1.f) * id) * (W * id);
  const float T5 = prsq * rir * (delta * ir);
  const float T6 = rir * W * id;
  f[3] = T1 - T2 + T3 - T4 + T5 - T6;
  const float c3s3 = cs2 * cs * isn2 / sn;
  f[4] = (cs * sn * (bsq * isn2 - asq) + bsq * c3s3) * ir -
         acs * ptsq * ir * ir - acs * prsq * (delta * ir) * ir +
         acs * W * ir * id;
}

struct MixedState {
  plain::RayState s;
  float r0;      // spherical photon-orbit radius of this ray's b
  int32_t n64;   // attempts taken in FP64
};

// One attempt.  Returns true when the ray is finished.
__device__ __forceinline__ bool attempt(const RayParams& p, MixedState& m) {
  using namespace plain;
  plain::RayState& s = m.s;
  const float band = (float)p.fp64_band;
  bool use64 = s.y[0] > 1e8 || fabs(s.y[0] - (double)m.r0) < band;
  if (!use64) {
    float yf[5], d[5], k1[5], k2[5], k3[5], k4[5], k5[5], t[5];
#pragma unroll
    for (int i = 0; i < 5; i++) yf[i] = (float)s.y[i];
    const float hf = (float)s.h;
    const float bf = (float)s.b, qf = (float)s.q, af = (float)p.a,
                a2f = (float)p.asq;
    eom_f(yf, d, bf, qf, af, a2f);
#pragma unroll
    for (int i = 0; i < 5; i++) t[i] = yf[i] + hf * ((float)b21 * d[i]);
    eom_f(t, k1, bf, qf, af, a2f);
#pragma unroll
    for (int i = 0; i < 5; i++)
      t[i] = yf[i] + hf * ((float)b31 * d[i] + (float)b32 * k1[i]);
    eom_f(t, k2, bf, qf, af, a2f);
#pragma unroll
    for (int i = 0; i < 5; i++)
      t[i] = yf[i] + hf * ((float)b41 * d[i] + (float)b42 * k1[i] +
                           (float)b43 * k2[i]);
    eom_f(t, k3, bf, qf, af, a2f);
#pragma unroll
    for (int i = 0; i < 5; i++)
      t[i] = yf[i] + hf * ((float)b51 * d[i] + (float)b52 * k1[i] +
                           (float)b53 * k2[i] + (float)b54 * k3[i]);
    eom_f(t, k4, bf, qf, af, a2f);
#pragma unroll
    for (int i = 0; i < 5; i++)
      t[i] = yf[i] + hf * ((float)b61 * d[i] + (float)b62 * k1[i] +
                           (float)b63 * k2[i] + (float)b64 * k3[i] +
                           (float)b65 * k4[i]);
    eom_f(t, k5, bf, qf, af, a2f);
    float inc[5];
    float errmax = 0.f;
#pragma unroll
    for (int i = 0; i < 5; i++) {
      inc[i] = hf * ((float)c1 * d[i] + (float)c3 * k2[i] + (float)c4 * k3[i] +
                     (float)c6 * k5[i]);
      const float e = hf * ((float)dc1 * d[i] + (float)dc3 * k2[i] +
                            (float)dc4 * k3[i] + (float)dc5 * k4[i] +
                            (float)dc6 * k5[i]);
      const float sc = fabsf(yf[i]) + fabsf(d[i] * hf) + 1.0e-30f;
      errmax = fmaxf(errmax, fabsf(e / sc));
    }
    errmax /= (float)p.eps;
    const float rn = yf[0] + inc[0];
    const bool turn = (yf[3] + inc[3]) * yf[3] < 0.f ||
                      (yf[4] + inc[4]) * yf[4] < 0.f;
    const bool near = fabsf(rn - m.r0) < band;
    const bool finite = errmax <= 3.0e38f;  // false for NaN / inf
    if (finite && (errmax > 1.0f || !(turn || near))) {
      if (errmax <= 1.0f) {
        s.z += s.h;
#pragma unroll
        for (int i = 0; i < 5; i++) s.y[i] += (double)inc[i];
        s.h = errmax > (float)kErrCon
                  ? kSafety * s.h * (double)__powf(errmax, (float)kPGrow)
                  : kAdaptive * s.h;
      } else {
        s.h = fmin(kSafety * s.h * (double)__powf(errmax, (float)kPShrnk),
                   0.1 * s.h);
      }
      s.step = s.nstp;
      s.nstp++;
      return s.z <= p.z_end || s.nstp >= p.maxstp;
    }
  }
  m.n64++;
  return plain::attempt(p, s);
}

__device__ __forceinline__ bool begin_ray(const RayParams& p, double th,
                                          double ph, MixedState& m,
                                          double& tho, double& pho,
                                          int32_t& steps, uint8_t& status) {
  double r0 = 0;
  const bool go = plain::begin_ray(p, th, ph, m.s, tho, pho, steps, status, &r0);
  m.r0 = (float)r0;
  m.n64 = 0;
  return go;
}

__device__ __forceinline__ void start_ray(const RayParams& p, const plain::RayStart& rs,
                                          MixedState& m) {
  plain::start_ray(p, rs, m.s);
  m.r0 = (float)rs.r0;
  m.n64 = 0;
}

}  // namespace mixed
}  // namespace bt
