// Host-side check that the branch-free forms of the star path compute what
// the forms they replace compute, bit for bit:
//   * in_quad_edges (the pixel's edge terms, no short-circuit) against
//     in_quad (cross_pos edge by edge, starInPolygon, BT/kernel.cuh:245-266);
//   * in_pixel (the four quadrant cases as selects) against the quadrant
//     cases as branches (interpolate, BT/kernel.cuh:112-200).
// Compiled by nvcc as host code only: it launches nothing and needs no GPU.
// Prints "quad <mismatches> <cases>" and "bisect <mismatches> <cases>".
#include <cstdio>
#include <cstring>
#include <random>

#include "stars_pixel.cuh"

using namespace bt;

// The quadrant cases as branches, in the reference's order of operations.
static void in_pixel_branches(float t0, float t1, float t2, float t3, float p0, float p1,
                              float p2, float p3, float& st, float& sp, int sgn) {
  const float error = 0.00001f;
  float midT = (t0 + t1 + t2 + t3) * .25f;
  float midP = (p0 + p1 + p2 + p3) * .25f;
  float y = 0.5f, x = 0.5f, perc = 0.5f;
  for (int q = 0; q < 10; q++) {
    if ((fabsf(st - midT) < error) && (fabsf(sp - midP) < error)) break;
    const float h01T = (t0 + t1) * .5f, h23T = (t2 + t3) * .5f;
    const float h12T = (t2 + t1) * .5f, h03T = (t0 + t3) * .5f;
    const float h01P = (p0 + p1) * .5f, h23P = (p2 + p3) * .5f;
    const float h12P = (p2 + p1) * .5f, h03P = (p0 + p3) * .5f;
    const float l0123T = h23T - h01T, l0312T = h12T - h03T;
    const float l0123P = h23P - h01P, l0312P = h12P - h03P;
    const float l01sT = st - h01T, l03sT = st - h03T;
    const float l01sP = sp - h01P, l03sP = sp - h03P;
    const int a = (((l0312T * l03sP) - (l03sT * l0312P)) > 0.f) ? 1 : -1;
    const int b = (((l0123T * l01sP) - (l01sT * l0123P)) > 0.f) ? 1 : -1;
    perc *= 0.5f;
    if (sgn * a > 0) {
      if (sgn * b > 0) {
        t2 = h12T; t0 = h01T; t3 = midT; p2 = h12P; p0 = h01P; p3 = midP;
        x -= perc; y -= perc;
      } else {
        t2 = midT; t1 = h01T; t3 = h03T; p2 = midP; p1 = h01P; p3 = h03P;
        x -= perc; y += perc;
      }
    } else {
      if (sgn * b > 0) {
        t1 = h12T; t3 = h23T; t0 = midT; p1 = h12P; p3 = h23P; p0 = midP;
        x += perc; y -= perc;
      } else {
        t0 = h03T; t1 = midT; t2 = h23T; p0 = h03P; p1 = midP; p2 = h23P;
        x += perc; y += perc;
      }
    }
    midT = (t0 + t1 + t2 + t3) * .25f;
    midP = (p0 + p1 + p2 + p3) * .25f;
  }
  st = y;
  sp = x;
}

static bool same_bits(float a, float b) { return std::memcmp(&a, &b, sizeof(float)) == 0; }

int main() {
  std::mt19937 rng(20261203);
  std::uniform_real_distribution<float> centre_t(0.05f, 3.1f), centre_p(0.05f, 6.2f);
  std::uniform_real_distribution<float> unit(-1.f, 1.f);
  long quad_cases = 0, quad_bad = 0, bis_cases = 0, bis_bad = 0;
  for (int n = 0; n < 20000; n++) {
    // a pixel quad: four corners around a centre, sizes from 1e-5 to 0.3 rad,
    // corner order and winding as they come (the pixel set-up's orientation)
    const float ct = centre_t(rng), cp = centre_p(rng);
    const float size = std::pow(10.f, -5.f + 4.5f * (0.5f * (unit(rng) + 1.f)));
    PixelCore core{};
    const float base[4][2] = {{-1, -1}, {-1, 1}, {1, 1}, {1, -1}};
    const bool flip = unit(rng) > 0;
    for (int k = 0; k < 4; k++) {
      const int kk = flip ? 3 - k : k;
      core.t[k] = ct + size * (base[kk][0] + 0.4f * unit(rng));
      core.p[k] = cp + size * (base[kk][1] + 0.4f * unit(rng));
    }
    const float* t = core.t;
    const float* p = core.p;
    const float orient = (t[1] - t[0]) * (p[1] + p[0]) + (t[2] - t[1]) * (p[2] + p[1]) +
                         (t[3] - t[2]) * (p[3] + p[2]) + (t[0] - t[3]) * (p[0] + p[3]);
    core.bits = orient < 0 ? 2 : 0;
    PixelStars P;
    stars_of(core, 1, P);
    for (int s = 0; s < 16; s++) {
      // stars over the quad's bounding box and a margin around it
      const float st = ct + 1.6f * size * unit(rng);
      const float sp = cp + 1.6f * size * unit(rng);
      const bool a = in_quad_edges(P, st, sp);
      const bool b = in_quad(P.t, P.p, st, sp, P.sgn);
      quad_cases++;
      if (a != b) quad_bad++;
      if (!b) continue;
      float y1 = st, x1 = sp, y2 = st, x2 = sp;
      in_pixel(P.t[0], P.t[1], P.t[2], P.t[3], P.p[0], P.p[1], P.p[2], P.p[3], y1, x1, P.sgn);
      in_pixel_branches(P.t[0], P.t[1], P.t[2], P.t[3], P.p[0], P.p[1], P.p[2], P.p[3], y2,
                        x2, P.sgn);
      bis_cases++;
      if (!same_bits(y1, y2) || !same_bits(x1, x2)) bis_bad++;
    }
  }
  std::printf("quad %ld %ld\n", quad_bad, quad_cases);
  std::printf("bisect %ld %ld\n", bis_bad, bis_cases);
  return 0;
}
