// map_math.cuh -- per-pixel map arithmetic (FP32), host+device.
//
// Restates the reference's device helpers (annemiekie/BlackTracer
// BT/kernel.cuh) in their FP32 operation order: grid interpolation
// (findBlock :736-752, interpolateSpline :940-968, interpolateHermite
// :891-938, findPoint :817-889, interpolateLinear :774-788, intersection
// :754-772, hermite :790-815, piCheck/piCheckTot :274-322, wrapToPi
// :694-703), solid angles (calcArea :586-610, calcAreax :612-649), pixel
// corners (retrievePixelCorners :652-672), Doppler/gravitational shift
// (redshift :348-365), lensing (findLensingRedshift :674-692) and the HSP
// colour model (RGBtoHSP/HSPtoRGB :388-524, D. R. Finley's public-domain
// formulas).  Compiled with FMA contraction off, every +,-,*,/ rounds as in
// the reference; sinf/cosf/atanf/powf come from the device libm.
//
// Grid reads are bounds-checked: where the reference indexes rows outside
// the grid (findPoint's neighbours 3 gaps away, :836-855 and :877-880, read
// memory around the buffer), this build reads an absent vertex (-2, -2).
#pragma once

#include <cuda_runtime.h>

#include "bt_internal.h"

namespace bt {
namespace mapm {

#define BT_HD __host__ __device__ __forceinline__

constexpr float PI = 3.141592653589793238f;
constexpr float PI2 = 6.283185307179586476f;
constexpr float Pr = .299f, Pg = .587f, Pb = .114f;

struct GridRef {
  const float2* g;  // GN x GM float2 (the map grid), (-2,-2) = absent
  int GM, GN;
  BT_HD float2 at(int i, int j) const {
    if (i < 0 || i >= GN || j < 0 || j >= GM) return make_float2(-2.f, -2.f);
    return g[(size_t)i * GM + j];
  }
};

BT_HD bool pi_check(float* p, float factor) {
  float factor1 = PI2 * (1.f - factor);
  bool check = false;
  for (int q = 0; q < 4; q++)
    if (p[q] > factor1) {
      check = true;
      break;
    }
  if (!check) return false;
  check = false;
  float factor2 = PI2 * factor;
  for (int q = 0; q < 4; q++)
    if (p[q] < factor2) {
      p[q] += PI2;
      check = true;
    }
  return check;
}

BT_HD bool pi_check_tot(float2* tp, float factor, int size) {
  float factor1 = PI2 * (1.f - factor);
  bool check = false;
  for (int q = 0; q < size; q++)
    if (tp[q].y > factor1) {
      check = true;
      break;
    }
  if (!check) return false;
  check = false;
  float factor2 = PI2 * factor;
  for (int q = 0; q < size; q++)
    if (tp[q].y < factor2) {
      tp[q].y += PI2;
      check = true;
    }
  return check;
}

// wrapToPi (float); the phi loop is bounded like the FP64 one.
BT_HD void wrap_to_pi(float& th, float& ph) {
  th = fmodf(th, PI2);
  while (th < 0.f) th += PI2;
  if (th > PI) {
    th -= 2.f * (th - PI);
    ph += PI;
  }
  for (int it = 0; ph < 0.f; it++) {
    if (it == 4096) {
      ph = fmodf(ph, PI2) + PI2;
      break;
    }
    ph += PI2;
  }
  ph = fmodf(ph, PI2);
}

BT_HD float2 hermite(float v, float2 x0, float2 x1, float2 x2, float2 x3) {
  const float aTension = 0.f, aBias = 0.f;
  float const v2 = v * v;
  float const v3 = v * v2;
  float const aa = (1.f + aBias) * (1.f - aTension) / 2.f;
  float const bb = (1.f - aBias) * (1.f - aTension) / 2.f;
  float const m0T = aa * (x1.x - x0.x) + bb * (x2.x - x1.x);
  float const m0P = aa * (x1.y - x0.y) + bb * (x2.y - x1.y);
  float const m1T = aa * (x2.x - x1.x) + bb * (x3.x - x2.x);
  float const m1P = aa * (x2.y - x1.y) + bb * (x3.y - x2.y);
  float const u0 = 2.f * v3 - 3.f * v2 + 1.f;
  float const u1 = v3 - 2.f * v2 + v;
  float const u2 = v3 - v2;
  float const u3 = -2.f * v3 + 3.f * v2;
  return make_float2(u0 * x1.x + u1 * m0T + u2 * m1T + u3 * x2.x,
                     u0 * x1.y + u1 * m0P + u2 * m1P + u3 * x2.y);
}

BT_HD float2 intersection(float ax, float ay, float bx, float by, float cx,
                          float cy, float dx, float dy) {
  double a1 = by - ay;
  double b1 = ax - bx;
  double c1 = a1 * (ax) + b1 * (ay);
  double a2 = dy - cy;
  double b2 = cx - dx;
  double c2 = a2 * (cx) + b2 * (cy);
  double determinant = a1 * b2 - a2 * b1;
  if (determinant == 0) return make_float2(-1.f, -1.f);
  double x = (b2 * c1 - b1 * c2) / determinant;
  double y = (a1 * c2 - a2 * c1) / determinant;
  return make_float2((float)x, (float)y);
}

BT_HD float2 interpolate_linear(float percDown, float percRight,
                                const float2* cc) {
  float phi[4] = {cc[0].y, cc[1].y, cc[2].y, cc[3].y};
  float theta[4] = {cc[0].x, cc[1].x, cc[2].x, cc[3].x};
  pi_check(phi, 0.2f);
  float leftT = theta[0] + percDown * (theta[2] - theta[0]);
  float leftP = phi[0] + percDown * (phi[2] - phi[0]);
  float rightT = theta[1] + percDown * (theta[3] - theta[1]);
  float rightP = phi[1] + percDown * (phi[3] - phi[1]);
  float upT = theta[0] + percRight * (theta[1] - theta[0]);
  float upP = phi[0] + percRight * (phi[1] - phi[0]);
  float downT = theta[2] + percRight * (theta[3] - theta[2]);
  float downP = phi[2] + percRight * (phi[3] - phi[2]);
  return intersection(upT, upP, downT, downP, leftT, leftP, rightT, rightP);
}

BT_HD float2 interpolate_hermite(const GridRef& G, int i, int j, int gap,
                                 float percDown, float percRight, float2* cc,
                                 int count);

// findPoint: a neighbour sample, reconstructed when the vertex is absent.
BT_HD float2 find_point(const GridRef& G, int i, int j, int offver, int offhor,
                        int gap, int count) {
  const int GM = G.GM, GN = G.GN;
  float2 gridpt = G.at(i, j);
  if (gridpt.x == -2 && gridpt.y == -2) {
    int j2 = (j + offhor * gap + GM) % GM;
    int i2 = i + offver * gap;
    float2 ij2 = G.at(i2, j2);
    if (ij2.x == -1 && ij2.y == -1) return make_float2(-1.f, -1.f);
    if (ij2.x != -2 && ij2.y != -2) {
      int j0 = (j - offhor * gap + GM) % GM;
      int i0 = (i - offver * gap);
      float2 ij0 = G.at(i0, j0);
      if (ij0.x < 0) return make_float2(-1.f, -1.f);
      int jprev = (j - 3 * offhor * gap + GM) % GM;
      int jnext = (j + 3 * offhor * gap + GM) % GM;
      int iprev = i - offver * 3 * gap;
      int inext = i + offver * 3 * gap;
      if (offver != 0) {
        if (i2 == 0) {
          jnext = (j0 + GM / 2) % GM;
          inext = i0;
        } else if (i0 == GN - 1) {
          jprev = (j0 + GM / 2) % GM;
          iprev = i2;
        } else if (i2 == GN - 1) {
          inext = i0;
          jnext = (j0 + GM / 2) % GM;
        }
      }
      float2 ijprev = G.at(iprev, jprev);
      float2 ijnext = G.at(inext, jnext);
      if (ijprev.x > -2 && ijnext.x > -2) {
        float2 pt[4] = {ijprev, ij0, ij2, ijnext};
        if (pt[0].x != -1 && pt[3].x != -1) {
          pi_check_tot(pt, 0.2f, 4);
          return hermite(0.5f, pt[0], pt[1], pt[2], pt[3]);
        }
      }
      float2 pt[2] = {ij2, ij0};
      pi_check_tot(pt, 0.2f, 2);
      return make_float2(.5f * (pt[0].x + pt[1].x), .5f * (pt[0].y + pt[1].y));
    }
    if (count > 0) return make_float2(-1.f, -1.f);
    int j0 = (j + gap) % GM;
    int j1 = (j - gap + GM) % GM;
    if (i - gap < 0) return make_float2(-1.f, -1.f);
    float2 cc2[12];
    cc2[0] = G.at(i + gap, j0);
    cc2[1] = G.at(i - gap, j0);
    cc2[2] = G.at(i - gap, j1);
    cc2[3] = G.at(i + gap, j1);
    for (int q = 0; q < 4; q++)
      if (cc2[q].x == -1 || cc2[q].x == -2) return make_float2(-1.f, -1.f);
    return interpolate_hermite(G, i - gap, j1, 2 * gap, .5f, .5f, cc2, 1);
  }
  return gridpt;
}

BT_HD float2 interpolate_hermite(const GridRef& G, int i, int j, int gap,
                                 float percDown, float percRight, float2* cc,
                                 int count) {
  const int GM = G.GM, GN = G.GN;
  int k = i + gap;
  int l = (j + gap) % GM;
  int imin1 = i - gap;
  int kplus1 = k + gap;
  int jmin1 = (j - gap + GM) % GM;
  int lplus1 = (l + gap) % GM;
  int jx = j, jy = j, lx = l, ly = l;
  if (i == 0) {
    jx = (j + GM / 2) % GM;
    lx = (jx + gap) % GM;
    imin1 = k;
  } else if (k == GN - 1) {
    jy = (j + GM / 2) % GM;
    ly = (jy + gap) % GM;
    kplus1 = i;
  }
  cc[4] = find_point(G, i, jmin1, 0, -1, gap, count);
  cc[5] = find_point(G, i, lplus1, 0, 1, gap, count);
  cc[6] = find_point(G, k, jmin1, 0, -1, gap, count);
  cc[7] = find_point(G, k, lplus1, 0, 1, gap, count);
  cc[8] = find_point(G, imin1, jx, -1, 0, gap, count);
  cc[9] = find_point(G, imin1, lx, -1, 0, gap, count);
  cc[10] = find_point(G, kplus1, jy, 1, 0, gap, count);
  cc[11] = find_point(G, kplus1, ly, 1, 0, gap, count);
  for (int q = 4; q < 12; q++)
    if (cc[q].x == -1) return interpolate_linear(percDown, percRight, cc);
  pi_check_tot(cc, 0.2f, 12);
  float2 up = hermite(percRight, cc[4], cc[0], cc[1], cc[5]);
  float2 down = hermite(percRight, cc[6], cc[2], cc[3], cc[7]);
  float2 upup = make_float2(cc[8].x + (cc[9].x - cc[8].x) * percRight,
                            cc[8].y + (cc[9].y - cc[8].y) * percRight);
  float2 downdown = make_float2(cc[10].x + (cc[11].x - cc[10].x) * percRight,
                                cc[10].y + (cc[11].y - cc[10].y) * percRight);
  return hermite(percDown, upup, up, down, downdown);
}

// interpolatePix (BT/MakeImageKernel.cu:328-351) for the G = 1 case:
// celestial (theta, phi) of one camera-sky direction, and the block size.
BT_HD float2 interpolate_pix(const GridRef& G, float theta, float phi,
                             int gridlvl, int& gap_out) {
  const int GM = G.GM;
  int half = (phi < PI) ? 0 : 1;
  int a = 0;
  int b = half * GM / 2;
  int gap = GM / 2;
  // findBlock
  for (int s = 0; s < gridlvl + 1; s++) {
    int ngap = gap / 2;
    int k = a + ngap;
    int l = b + ngap;
    if (gap <= 1 || G.at(k, l).x == -2.f) break;
    float thHalf = PI2 * k / (1.f * GM);
    float phHalf = PI2 * l / (1.f * GM);
    if (thHalf <= theta) a = k;
    if (phHalf <= phi) b = l;
    gap = ngap;
  }
  gap_out = gap;
  int k = a + gap;
  int l = b + gap;
  float factor = PI2 / (1.f * GM);
  float cornersCam[4] = {factor * a, factor * b, factor * k, factor * l};
  l = l % GM;
  float2 cc[12];
  cc[0] = G.at(a, b);
  cc[1] = G.at(a, l);
  cc[2] = G.at(k, b);
  cc[3] = G.at(k, l);
  for (int q = 4; q < 12; q++) cc[q] = make_float2(-1.f, -1.f);
  // interpolateSpline
  float2 r;
  const float thetaUp = cornersCam[0], thetaDown = cornersCam[2];
  const float phiLeft = cornersCam[1], phiRight = cornersCam[3];
  bool done = false;
  if (thetaUp == theta) {
    if (phiLeft == phi) { r = cc[0]; done = true; }
    else if (phiRight == phi) { r = cc[1]; done = true; }
    else if (a == 0.f) { r = cc[0]; done = true; }
  } else if (thetaDown == theta) {
    if (phiLeft == phi) { r = cc[2]; done = true; }
    else if (phiRight == phi) { r = cc[3]; done = true; }
  }
  if (!done) {
    for (int q = 0; q < 4; q++)
      if (cc[q].x == -1 && cc[q].y == -1) {
        r = make_float2(-1.f, -1.f);
        done = true;
        break;
      }
  }
  if (!done) {
    float percDown = (theta - thetaUp) / (thetaDown - thetaUp);
    float percRight = (phi - phiLeft) / (phiRight - phiLeft);
    r = interpolate_hermite(G, a, b, gap, percDown, percRight, cc, 0);
  }
  if (!(r.x == -1 && r.y == -1)) wrap_to_pi(r.x, r.y);
  return r;
}

// Solid angle of a spherical quad, two triangles (calcArea).
BT_HD float calc_area(const float* t, const float* p) {
  float x[4], y[4], z[4];
  for (int q = 0; q < 4; q++) {
    float sint = sinf(t[q]);
    x[q] = sint * cosf(p[q]);
    y[q] = sint * sinf(p[q]);
    z[q] = cosf(t[q]);
  }
  float dotpr1 = 1.f;
  dotpr1 += x[0] * x[2] + y[0] * y[2] + z[0] * z[2];
  float dotpr2 = dotpr1;
  dotpr1 += x[2] * x[1] + y[2] * y[1] + z[2] * z[1];
  dotpr1 += x[0] * x[1] + y[0] * y[1] + z[0] * z[1];
  dotpr2 += x[0] * x[3] + y[0] * y[3] + z[0] * z[3];
  dotpr2 += x[2] * x[3] + y[2] * y[3] + z[2] * z[3];
  float triprod1 = fabsf(x[0] * (y[1] * z[2] - y[2] * z[1]) -
                         y[0] * (x[1] * z[2] - x[2] * z[1]) +
                         z[0] * (x[1] * y[2] - x[2] * y[1]));
  float triprod2 = fabsf(x[0] * (y[2] * z[3] - y[3] * z[2]) -
                         y[0] * (x[2] * z[3] - x[3] * z[2]) +
                         z[0] * (x[2] * y[3] - x[3] * y[2]));
  return 2.f * (atanf(triprod1 / dotpr1) + atanf(triprod2 / dotpr2));
}

// Solid angle of a spherical triangle, vertices reordered so the smallest
// dot product is not between the first two (calcAreax).
BT_HD float calc_areax(const float* t, const float* p) {
  float xi[3], yi[3], zi[3];
  for (int q = 0; q < 3; q++) {
    float sint = sinf(t[q]);
    xi[q] = sint * cosf(p[q]);
    yi[q] = sint * sinf(p[q]);
    zi[q] = cosf(t[q]);
  }
  float dot01 = xi[0] * xi[1] + yi[0] * yi[1] + zi[0] * zi[1];
  float dot02 = xi[0] * xi[2] + yi[0] * yi[2] + zi[0] * zi[2];
  float dot12 = xi[2] * xi[1] + yi[2] * yi[1] + zi[2] * zi[1];
  float x[3] = {xi[0], xi[1], xi[2]};
  float y[3] = {yi[0], yi[1], yi[2]};
  float z[3] = {zi[0], zi[1], zi[2]};
  if (dot01 < dot02 && dot01 < dot12) {
    x[0] = xi[2]; x[1] = xi[0]; x[2] = xi[1];
    y[0] = yi[2]; y[1] = yi[0]; y[2] = yi[1];
    z[0] = zi[2]; z[1] = zi[0]; z[2] = zi[1];
  } else if (dot02 < dot12 && dot02 < dot01) {
    x[0] = xi[1]; x[1] = xi[2]; x[2] = xi[0];
    y[0] = yi[1]; y[1] = yi[2]; y[2] = yi[0];
    z[0] = zi[1]; z[1] = zi[2]; z[2] = zi[0];
  }
  float dotpr1 = 1.f;
  dotpr1 += x[0] * x[2] + y[0] * y[2] + z[0] * z[2];
  dotpr1 += x[2] * x[1] + y[2] * y[1] + z[2] * z[1];
  dotpr1 += x[0] * x[1] + y[0] * y[1] + z[0] * z[1];
  float triprod1 = fabsf(x[0] * (y[1] * z[2] - y[2] * z[1]) -
                         y[0] * (x[1] * z[2] - x[2] * z[1]) +
                         z[0] * (x[1] * y[2] - x[2] * y[1]));
  return 2.f * (atanf(triprod1 / dotpr1));
}

// retrievePixelCorners: corners of pixel (i, j) from the (M+1)-wide corner
// array, in the reference's order {lower-left, upper-left, upper-right,
// lower-right}; false (ind = -1 in the reference) when a corner is captured.
BT_HD bool pixel_corners(const float2* thphi, int ind, int M, float* t,
                         float* p, bool& picheck, float offset) {
  const int M1 = M + 1;
  t[0] = thphi[ind + M1].x;
  t[1] = thphi[ind].x;
  t[2] = thphi[ind + 1].x;
  t[3] = thphi[ind + M1 + 1].x;
  p[0] = thphi[ind + M1].y;
  p[1] = thphi[ind].y;
  p[2] = thphi[ind + 1].y;
  p[3] = thphi[ind + M1 + 1].y;
  for (int q = 0; q < 4; q++) {
    if (p[q] < 0 || t[q] < 0) return false;
    p[q] = fmodf(p[q] + offset, PI2);
  }
  picheck = pi_check(p, .2f);
  return true;
}

BT_HD float pixel_solid_angle(const float* t, const float* p) {
  float th1[3] = {t[0], t[1], t[2]};
  float ph1[3] = {p[0], p[1], p[2]};
  float th2[3] = {t[0], t[2], t[3]};
  float ph2[3] = {p[0], p[2], p[3]};
  return calc_areax(th1, ph1) + calc_areax(th2, ph2);
}

// (1+z)^-1 ... the reference's redshift factor for a camera-sky direction.
BT_HD float redshift(float theta, float phi, const float* cam) {
  const float cam_speed = cam[0], cam_alpha = cam[1], cam_w = cam[2],
              cam_wbar = cam[3], cam_br = cam[4], cam_btheta = cam[5],
              cam_bphi = cam[6];
  float xCam = sinf(theta) * cosf(phi);
  float zCam = cosf(theta);
  float yCam = sinf(theta) * sinf(phi);
  float part = (1.f - cam_speed * yCam);
  float betaPart = sqrtf(1.f - cam_speed * cam_speed) / part;
  float xFido = -sqrtf(1.f - cam_speed * cam_speed) * xCam / part;
  float zFido = -sqrtf(1.f - cam_speed * cam_speed) * zCam / part;
  float yFido = (-yCam + cam_speed) / part;
  float k = sqrtf(1.f - cam_btheta * cam_btheta);
  float phiFido = -xFido * cam_br / k + cam_bphi * yFido + cam_bphi * cam_btheta / k * zFido;
  float eF = 1.f / (cam_alpha + cam_w * cam_wbar * phiFido);
  float b = eF * cam_wbar * phiFido;
  return 1.f / (betaPart * (1.f - b * cam_w) / cam_alpha);
}

// findLensingRedshift: magnification fraction and shift of pixel `ind`.
BT_HD void lensing_redshift(const float* t, const float* p, int M, int ind,
                            const float* cam, const float2* view, float& frac,
                            float& redshft, float solidAngle) {
  const int M1 = M + 1;
  if (solidAngle == 0.f) solidAngle = pixel_solid_angle(t, p);
  float ver4[4] = {view[ind].x, view[ind + 1].x, view[ind + M1 + 1].x, view[ind + M1].x};
  float hor4[4] = {view[ind].y, view[ind + 1].y, view[ind + M1 + 1].y, view[ind + M1].y};
  float pixArea = calc_area(ver4, hor4);
  frac = pixArea / solidAngle;
  float thetaCam = (ver4[0] + ver4[1] + ver4[2] + ver4[3]) * .25f;
  float phiCam = (hor4[0] + hor4[1] + hor4[2] + hor4[3]) * .25f;
  redshft = redshift(thetaCam, phiCam, cam);
}

BT_HD void rgb_to_hsp(float R, float G, float B, float& H, float& S, float& P) {
  P = sqrtf(R * R * Pr + G * G * Pg + B * B * Pb);
  if (R == G && R == B) {
    H = 0.f;
    S = 0.f;
    return;
  }
  if (R >= G && R >= B) {
    if (B >= G) {
      H = 6.f / 6.f - 1.f / 6.f * (B - G) / (R - G);
      S = 1.f - G / R;
    } else {
      H = 0.f / 6.f + 1.f / 6.f * (G - B) / (R - B);
      S = 1.f - B / R;
    }
  } else if (G >= R && G >= B) {
    if (R >= B) {
      H = 2.f / 6.f - 1.f / 6.f * (R - B) / (G - B);
      S = 1.f - B / G;
    } else {
      H = 2.f / 6.f + 1.f / 6.f * (B - R) / (G - R);
      S = 1.f - R / G;
    }
  } else {
    if (G >= R) {
      H = 4.f / 6.f - 1.f / 6.f * (G - R) / (B - R);
      S = 1.f - R / B;
    } else {
      H = 4.f / 6.f + 1.f / 6.f * (R - G) / (B - G);
      S = 1.f - G / B;
    }
  }
}

BT_HD void hsp_to_rgb(float H, float S, float P, float& R, float& G, float& B) {
  float part, minOverMax = 1.f - S;
  if (minOverMax > 0.f) {
    if (H < 1.f / 6.f) {
      H = 6.f * H;
      part = 1.f + H * (1.f / minOverMax - 1.f);
      B = P / sqrtf(Pr / minOverMax / minOverMax + Pg * part * part + Pb);
      R = B / minOverMax;
      G = B + H * (R - B);
    } else if (H < 2.f / 6.f) {
      H = 6.f * (-H + 2.f / 6.f);
      part = 1.f + H * (1.f / minOverMax - 1.f);
      B = P / sqrtf(Pg / minOverMax / minOverMax + Pr * part * part + Pb);
      G = B / minOverMax;
      R = B + H * (G - B);
    } else if (H < 3.f / 6.f) {
      H = 6.f * (H - 2.f / 6.f);
      part = 1.f + H * (1.f / minOverMax - 1.f);
      R = P / sqrtf(Pg / minOverMax / minOverMax + Pb * part * part + Pr);
      G = R / minOverMax;
      B = R + H * (G - R);
    } else if (H < 4.f / 6.f) {
      H = 6.f * (-H + 4.f / 6.f);
      part = 1.f + H * (1.f / minOverMax - 1.f);
      R = P / sqrtf(Pb / minOverMax / minOverMax + Pg * part * part + Pr);
      B = R / minOverMax;
      G = R + H * (B - R);
    } else if (H < 5.f / 6.f) {
      H = 6.f * (H - 4.f / 6.f);
      part = 1.f + H * (1.f / minOverMax - 1.f);
      G = P / sqrtf(Pb / minOverMax / minOverMax + Pr * part * part + Pg);
      B = G / minOverMax;
      R = G + H * (B - G);
    } else {
      H = 6.f * (-H + 6.f / 6.f);
      part = 1.f + H * (1.f / minOverMax - 1.f);
      G = P / sqrtf(Pr / minOverMax / minOverMax + Pb * part * part + Pg);
      R = G / minOverMax;
      B = G + H * (R - G);
    }
  } else {
    if (H < 1.f / 6.f) {
      H = 6.f * (H);
      R = sqrtf(P * P / (Pr + Pg * H * H));
      G = R * H;
      B = 0.f;
    } else if (H < 2.f / 6.f) {
      H = 6.f * (-H + 2.f / 6.f);
      G = sqrtf(P * P / (Pg + Pr * H * H));
      R = G * H;
      B = 0.f;
    } else if (H < .5f) {
      H = 6.f * (H - 2.f / 6.f);
      G = sqrtf(P * P / (Pg + Pb * H * H));
      B = G * H;
      R = 0.f;
    } else if (H < 4.f / 6.f) {
      H = 6.f * (-H + 4.f / 6.f);
      B = sqrtf(P * P / (Pb + Pg * H * H));
      G = B * H;
      R = 0.f;
    } else if (H < 5.f / 6.f) {
      H = 6.f * (H - 4.f / 6.f);
      B = sqrtf(P * P / (Pb + Pr * H * H));
      R = B * H;
      G = 0.f;
    } else {
      H = 6.f * (-H + 1.f);
      R = sqrtf(P * P / (Pr + Pb * H * H));
      B = R * H;
      G = 0.f;
    }
  }
}

#undef BT_HD

}  // namespace mapm
}  // namespace bt
