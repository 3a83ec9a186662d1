// stars_pixel.cuh -- per-pixel star splatting, host+device.
//
// The arithmetic of distortStarMap (annemiekie/BlackTracer
// BT/MakeImageKernel.cu:206-326) for one pixel: search of the star kd-tree
// (searchTree :27-96), point-in-quad (starInPolygon, BT/kernel.cuh:245-266),
// in-pixel position (interpolate :112-200), magnitude with lensing and
// redshift, blackbody colour, Gaussian splat (gaussian :335-338) into the
// pixel's (2s+1)^2 cells.  Host+device so the same code can be checked
// against the reference on a CPU.
#pragma once

#include "blackbody_table.h"
#include "map_math.cuh"

namespace bt {

struct StarSet {
  int n, treeLevel;
  const float* pos;  // 2n (theta, phi) in tree order
  const float* mag;  // 2n (magnitude, B-V colour index)
  const int* tree;   // 2^(treeLevel+1)-1 cumulative counts
  const uchar3* psf; // diffraction sprite, psf_size^2 (may be NULL)
  int psf_size;
};

#define BT_HD __host__ __device__ __forceinline__

BT_HD int ffs_u32(unsigned x) {
#ifdef __CUDA_ARCH__
  return __ffs((int)x);
#else
  return __builtin_ffs((int)x);
#endif
}
BT_HD int imax(int a, int b) { return a > b ? a : b; }
BT_HD int imin(int a, int b) { return a < b ? a : b; }

using namespace mapm;

BT_HD float dist_sq(float ta, float tb, float pa, float pb) {
  return (ta - tb) * (ta - tb) + (pa - pb) * (pa - pb);
}

BT_HD float gaussian(float dist) {
  const float sigma = 1.f / 2.5f;
  return expf(-.5f * dist / (sigma * sigma)) * 1.f / (sigma * 2.506628274631f);
}

// checkCrossProduct; sgn is +-1 so the reference always takes its first arm.
BT_HD bool cross_pos(float ta, float tb, float pa, float pb,
                                          float st, float sp, int sgn) {
  const float c1t = (float)sgn * (ta - tb);
  const float c1p = (float)sgn * (pa - pb);
  const float c2t = sgn ? st - tb : st - ta;
  const float c2p = sgn ? sp - pb : sp - pa;
  return (c1t * c2p - c2t * c1p) > 0;
}

BT_HD bool in_quad(const float* t, const float* p, float st,
                                        float sp, int sgn) {
  return cross_pos(t[0], t[1], p[0], p[1], st, sp, sgn) &&
         cross_pos(t[1], t[2], p[1], p[2], st, sp, sgn) &&
         cross_pos(t[2], t[3], p[2], p[3], st, sp, sgn) &&
         cross_pos(t[3], t[0], p[3], p[0], st, sp, sgn);
}

// In-pixel position of a star by 10 halvings of the projected quad
// (interpolate, BT/kernel.cuh:112-200).  Returns (y, x) in [0,1]^2.
BT_HD void in_pixel(float t0, float t1, float t2, float t3, float p0,
                         float p1, float p2, float p3, float& st, float& sp,
                         int sgn) {
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

struct PixelStars {
  float t[4], p[4];
  int sgn;
  bool picheck;
  long tested, budget;  // star tests so far / allowed before deferring
  bool abort;
  float red, redshft, frac, maxDistSq;
  int step;
  float3* cells;  // (2s+1)^2 cells of this pixel
  bool any;
};

// Iterative search of the star kd-tree for nodes overlapping the pixel's
// bounding box (searchTree, BT/MakeImageKernel.cu:27-96, as called there
// with picheck = 0).  emit(node) is called in the reference's emission order;
// it returns false to stop the search.
template <class Emit>
BT_HD void tree_search(const StarSet& S, const float* mn, const float* mx,
                       Emit&& emit) {
  const int L = S.treeLevel;
  float nodeStart[2] = {0.f, 0.f};
  float nodeSize[2] = {PI, PI2};
  int node = 0;
  unsigned bitMask = (unsigned)powf(2, L);
  int level = 0, lvl = 0;
  int guard = 0;
  while (bitMask != 0 && guard++ < (1 << 22)) {
    bitMask &= ~(1u << (L - level));
    for (lvl = level + 1; lvl <= L; lvl++) {
      int star_n = S.tree[node];
      if (node != 0 && ((node + 1) & node) != 0) star_n -= S.tree[node - 1];
      const int tp = lvl & 1;
      const float x_overlap = fmaxf(0.f, fminf(mx[0], nodeStart[0] + nodeSize[0]) -
                                             fmaxf(mn[0], nodeStart[0]));
      const float y_overlap = fmaxf(0.f, fminf(mx[1], nodeStart[1] + nodeSize[1]) -
                                             fmaxf(mn[1], nodeStart[1]));
      const float overlapArea = x_overlap * y_overlap;
      const bool size = overlapArea / (nodeSize[0] * nodeSize[1]) > 0.8f;
      nodeSize[tp] = nodeSize[tp] * .5f;
      if (star_n == 0) {
        node = node * 2 + 1;
        break;
      }
      const float check = nodeStart[tp] + nodeSize[tp];
      const bool lu = mn[tp] < check;
      const bool rd = mx[tp] >= check;
      if (lvl == L || (rd && lu && size)) {
        if (rd && !emit(node * 2 + 2)) return;
        if (lu && !emit(node * 2 + 1)) return;
        node = node * 2 + 1;
        break;
      }
      node = node * 2 + 1;
      if (rd) bitMask |= 1u << (L - lvl);
      if (!lu) break;
    }
    level = L - ffs_u32(bitMask) + 1;
    if (level >= 0) {
      const int diff = lvl - level;
      for (int k = 0; k < diff; k++) {
        const int tp = (lvl - k) & 1;
        if (!(node & 1)) nodeStart[tp] -= nodeSize[tp];
        nodeSize[tp] = nodeSize[tp] * 2.f;
        node = (node - 1) / 2;
      }
      node++;
      const int tp = level & 1;
      nodeStart[tp] += nodeSize[tp];
    }
  }
}

// Per-pixel set-up of distortStarMap (BT/MakeImageKernel.cu:222-263):
// corners, bounding box, winding, lensing fraction and redshift.  Returns
// false for black-hole pixels.
BT_HD bool pixel_setup(const float2* thphi, const uint8_t* bh, const float* cam,
                       int M, int step, const float2* view, int lr,
                       const float* area, int i, int j, PixelStars& P, float* mn,
                       float* mx) {
  const size_t ij = (size_t)i * M + j;
  P.any = false;
  P.abort = false;
  P.tested = 0;
  P.step = step;
  if (bh[ij] != 0) return false;
  P.picheck = false;
  const int ind = i * (M + 1) + j;
  pixel_corners(thphi, ind, M, P.t, P.p, P.picheck, 0.f);
  mx[0] = fmaxf(fmaxf(P.t[0], P.t[1]), fmaxf(P.t[2], P.t[3]));
  mx[1] = fmaxf(fmaxf(P.p[0], P.p[1]), fmaxf(P.p[2], P.p[3]));
  mn[0] = fminf(fminf(P.t[0], P.t[1]), fminf(P.t[2], P.t[3]));
  mn[1] = fminf(fminf(P.p[0], P.p[1]), fminf(P.p[2], P.p[3]));
  const float* t = P.t;
  const float* p = P.p;
  const float orient = (t[1] - t[0]) * (p[1] + p[0]) + (t[2] - t[1]) * (p[2] + p[1]) +
                       (t[3] - t[2]) * (p[3] + p[2]) + (t[0] - t[3]) * (p[0] + p[3]);
  P.sgn = orient < 0 ? -1 : 1;
  P.redshft = 1.f;
  P.frac = 1.f;
  if (lr) lensing_redshift(P.t, P.p, M, ind, cam, view, P.frac, P.redshft, area[ij]);
  P.red = 4.f * log10f(P.redshft);
  P.maxDistSq = (step + .5f) * (step + .5f);
  return true;
}

// A star that passed the quad test: its in-pixel position and colour.
struct StarHit {
  float st, sp, part;
  float3 hsp;
};

// The quad test of star q (with the seam retry), BT/MakeImageKernel.cu:285-291.
BT_HD bool star_test(const PixelStars& P, const StarSet& S, int q, float& st,
                     float& sp) {
  st = S.pos[2 * q];
  sp = S.pos[2 * q + 1];
  bool in = in_quad(P.t, P.p, st, sp, P.sgn);
  if (P.picheck && !in && sp < PI2 * .2f) {
    sp += PI2;
    in = in_quad(P.t, P.p, st, sp, P.sgn);
  }
  return in;
}

// In-pixel position, magnitude and colour of a star inside the quad
// (BT/MakeImageKernel.cu:293-301).
BT_HD StarHit star_hit(const PixelStars& P, const StarSet& S, int q, float st,
                       float sp) {
  StarHit h;
  in_pixel(P.t[0], P.t[1], P.t[2], P.t[3], P.p[0], P.p[1], P.p[2], P.p[3], st, sp,
           P.sgn);
  h.st = st;
  h.sp = sp;
  h.part = S.mag[2 * q] + P.red;
  const float bv = S.mag[2 * q + 1];
  const float temp = 46.f / P.redshft *
                         ((1.f / ((0.92f * bv) + 1.7f)) + (1.f / ((0.92f * bv) + 0.62f))) -
                     10.f;
  // The reference clamps to 1170 (BT/MakeImageKernel.cu:297), the length of
  // the flattened table minus 3, then reads tempToRGB[3*index]: shifted
  // temperatures above 40000 K read past its 391 entries.  Clamped to the
  // last entry (40000 K) here.
  const int index = imax(0, imin((int)floorf(temp), kBlackbodyEntries - 1));
  rgb_to_hsp((float)blackbody(3 * index) / 255.f, (float)blackbody(3 * index + 1) / 255.f,
             (float)blackbody(3 * index + 2) / 255.f, h.hsp.x, h.hsp.y, h.hsp.z);
  return h;
}

// Contribution of a star to cell (u, v) of its pixel, squared RGB
// (BT/MakeImageKernel.cu:305-320).  Returns false outside the splat radius.
BT_HD bool cell_light(const PixelStars& P, const StarHit& h, int u, int v,
                      float3& out) {
  const float dist = dist_sq(-P.step + u + .5f, h.st, -P.step + v + .5f, h.sp);
  if (dist > P.maxDistSq) return false;
  const float appMag = h.part - 2.5f * log10f(P.frac * gaussian(dist));
  const float brightness = 100 * exp10f(-.4f * appMag);
  float r, g, b;
  hsp_to_rgb(h.hsp.x, h.hsp.y, h.hsp.z * brightness, r, g, b);
  r *= 255.f;
  g *= 255.f;
  b *= 255.f;
  out = make_float3(r * r, g * g, b * b);
  return true;
}

// Tests and splats the stars of one tree node (distortStarMap's inner loop,
// BT/MakeImageKernel.cu:278-324, without trails).
BT_HD void splat_node(PixelStars& P, const StarSet& S, int node) {
  int startN = 0;
  if (node != 0 && ((node + 1) & node) != 0) startN = S.tree[node - 1];
  const int endN = S.tree[node];
  P.tested += endN - startN;
  if (P.tested > P.budget) {
    P.abort = true;
    return;
  }
  const int fw = 2 * P.step + 1;
  for (int q = startN; q < endN; q++) {
    float st, sp;
    if (!star_test(P, S, q, st, sp)) continue;
    if (!P.any) {
      for (int c = 0; c < fw * fw; c++) P.cells[c] = make_float3(0.f, 0.f, 0.f);
      P.any = true;
    }
    const StarHit h = star_hit(P, S, q, st, sp);
    for (int u = 0; u <= 2 * P.step; u++)
      for (int v = 0; v <= 2 * P.step; v++) {
        float3 l;
        if (!cell_light(P, h, u, v, l)) continue;
        float3& c = P.cells[fw * u + v];
        c.x += l.x;
        c.y += l.y;
        c.z += l.z;
      }
  }
}

// The whole of distortStarMap for pixel (i, j) (no trails).  Returns 0 (no
// star), 1 (stars; cells written) or 2 (more than `budget` star tests:
// nothing written, the pixel is left to the warp-cooperative path).
BT_HD int pixel_stars(const float2* thphi, const uint8_t* bh, const StarSet& S,
                      const float* cam, int M, int N, int step, const float2* view,
                      int lr, const float* area, int i, int j, float3* cells,
                      long budget = 0x7fffffffffffL) {
  PixelStars P;
  float mn[2], mx[2];
  P.cells = cells;
  if (!pixel_setup(thphi, bh, cam, M, step, view, lr, area, i, j, P, mn, mx)) return 0;
  P.budget = budget;
  tree_search(S, mn, mx, [&](int node) {
    splat_node(P, S, node);
    return !P.abort;
  });
  if (P.abort) return 2;
  return P.any ? 1 : 0;
}

#undef BT_HD

}  // namespace bt
