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
  // The sprite's non-zero entries: offsets from its centre (row, column)
  // and values, in row-major order; psf_rnz = their largest |offset|.
  const short2* psf_nzoff;
  const float4* psf_nzval;
  int psf_nnz, psf_rnz;
  // Entries [0, psf_nsplit) lie at or before the centre in row-major order;
  // psf_centre = the sprite's value at its centre (index size/2, size/2).
  int psf_nsplit;
  float4 psf_centre;
  // The sprite resampled at footprint scales s_k = 0.25 * 2^(k/8), k = 0..32:
  // entry values = bilinear sample at (centre + offset / s_k) / s_k^2, non-zero
  // entries only, level k at [lvl_start[k], lvl_start[k + 1]).
  const short2* psf_lvoff;
  const float4* psf_lvval;
  const int* psf_lvstart;
  // Per blackbody entry: RGBtoHSP of its colour (h, s, p) and
  // 255 * HSPtoRGB(h, s, p), computed once on the device by the same code.
  // bb_n = 391: the reference's table (100 K steps, index floor(temp));
  // bb_n = 1024: an FP32 table over the same 1000-40000 K range, linearly
  // interpolated from the reference's entries (index round(temp * 1023/390)).
  const float4* bb_hsp;
  const float4* bb_rgb;
  int bb_n;
  // Bounding box of each node's stars, (theta_min, phi_min, theta_max,
  // phi_max); min > max for a node without stars.  Not part of the
  // reference's layout: derived from pos and tree when the set is created.
  const float4* box;
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
BT_HD int clz_u32(unsigned x) {
#ifdef __CUDA_ARCH__
  return __clz((int)x);
#else
  return x ? __builtin_clz(x) : 32;
#endif
}
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
  // kept rolled: the star kernels are bound by instruction fetch
#pragma unroll 1
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
    // The reference's four quadrant cases as selects (the same values, no
    // divergent branches between lanes):
    //   A  B : t2 = h12, t0 = h01, t3 = mid;  x -= perc, y -= perc
    //   A !B : t2 = mid, t1 = h01, t3 = h03;  x -= perc, y += perc
    //  !A  B : t1 = h12, t3 = h23, t0 = mid;  x += perc, y -= perc
    //  !A !B : t0 = h03, t1 = mid, t2 = h23;  x += perc, y += perc
    const bool A = sgn * a > 0, B = sgn * b > 0;
    const float n0T = A ? (B ? h01T : t0) : (B ? midT : h03T);
    const float n1T = A ? (B ? t1 : h01T) : (B ? h12T : midT);
    const float n2T = A ? (B ? h12T : midT) : (B ? t2 : h23T);
    const float n3T = A ? (B ? midT : h03T) : (B ? h23T : t3);
    const float n0P = A ? (B ? h01P : p0) : (B ? midP : h03P);
    const float n1P = A ? (B ? p1 : h01P) : (B ? h12P : midP);
    const float n2P = A ? (B ? h12P : midP) : (B ? p2 : h23P);
    const float n3P = A ? (B ? midP : h03P) : (B ? h23P : p3);
    t0 = n0T; t1 = n1T; t2 = n2T; t3 = n3T;
    p0 = n0P; p1 = n1P; p2 = n2P; p3 = n3P;
    x = A ? x - perc : x + perc;
    y = B ? y - perc : y + perc;
    midT = (t0 + t1 + t2 + t3) * .25f;
    midP = (p0 + p1 + p2 + p3) * .25f;
  }
  st = y;
  sp = x;
}

struct PixelStars {
  float t[4], p[4];
  int sgn;
  // Edge k of the quad test as cross_pos computes it: c1 = sgn * (corner k -
  // corner k+1), anchored at corner k+1.
  float et[4], ep[4];
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
  // nodeStart / nodeSize of the reference as scalars (axis 0: theta, 1: phi)
  // so that nothing is indexed by the run-time axis.
  const float mn0 = mn[0], mn1 = mn[1], mx0 = mx[0], mx1 = mx[1];
  const int L = S.treeLevel;
  float st0 = 0.f, st1 = 0.f;
  float sz0 = PI, sz1 = PI2;
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
      const float x_overlap = fmaxf(0.f, fminf(mx0, st0 + sz0) - fmaxf(mn0, st0));
      const float y_overlap = fmaxf(0.f, fminf(mx1, st1 + sz1) - fmaxf(mn1, st1));
      const float overlapArea = x_overlap * y_overlap;
      const bool size = overlapArea / (sz0 * sz1) > 0.8f;
      if (tp) sz1 = sz1 * .5f;
      else sz0 = sz0 * .5f;
      if (star_n == 0) {
        node = node * 2 + 1;
        break;
      }
      const float check = tp ? st1 + sz1 : st0 + sz0;
      const bool lu = (tp ? mn1 : mn0) < check;
      const bool rd = (tp ? mx1 : mx0) >= check;
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
        if ((lvl - k) & 1) {
          if (!(node & 1)) st1 -= sz1;
          sz1 = sz1 * 2.f;
        } else {
          if (!(node & 1)) st0 -= sz0;
          sz0 = sz0 * 2.f;
        }
        node = (node - 1) / 2;
      }
      node++;
      if (level & 1) st1 += sz1;
      else st0 += sz0;
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
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const int k1 = (k + 1) & 3;
    P.et[k] = (float)P.sgn * (t[k] - t[k1]);
    P.ep[k] = (float)P.sgn * (p[k] - p[k1]);
  }
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
  int bb;  // blackbody entry
};

// Blackbody entry of a star of colour index bv seen with redshift factor
// redshft (BT/MakeImageKernel.cu:294-297).
BT_HD int blackbody_index(float bv, float redshft, int n = kBlackbodyEntries) {
  const float temp = 46.f / redshft *
                         ((1.f / ((0.92f * bv) + 1.7f)) + (1.f / ((0.92f * bv) + 0.62f))) -
                     10.f;
  // The reference clamps to 1170 (BT/MakeImageKernel.cu:297), the length of
  // the flattened table minus 3, then reads tempToRGB[3*index]: shifted
  // temperatures above 40000 K read past its 391 entries.  Clamped to the
  // last entry (40000 K) here.
  if (n == kBlackbodyEntries) return imax(0, imin((int)floorf(temp), kBlackbodyEntries - 1));
  const float t = fminf(fmaxf(temp, 0.f), (float)(kBlackbodyEntries - 1));
  return imin((int)rintf(t * ((float)(n - 1) / (float)(kBlackbodyEntries - 1))), n - 1);
}

// RGBtoHSP of blackbody entry k (BT/MakeImageKernel.cu:298-301).
BT_HD float3 blackbody_hsp(int k) {
  float3 h;
  rgb_to_hsp((float)blackbody(3 * k) / 255.f, (float)blackbody(3 * k + 1) / 255.f,
             (float)blackbody(3 * k + 2) / 255.f, h.x, h.y, h.z);
  return h;
}

// in_quad from the pixel's edge terms: edge k is cross_pos(corner k, corner
// k+1) with c1 = (P.et[k], P.ep[k]) and c2 = star - corner k+1, the same
// products and differences in the same order, so the result is identical;
// the four edges are combined without short-circuit branches.
BT_HD bool in_quad_edges(const PixelStars& P, float st, float sp) {
  bool r = true;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const int k1 = (k + 1) & 3;
    r &= (P.et[k] * (sp - P.p[k1]) - (st - P.t[k1]) * P.ep[k]) > 0;
  }
  return r;
}

// The quad test of star q (with the seam retry), BT/MakeImageKernel.cu:285-291.
BT_HD bool star_test(const PixelStars& P, const StarSet& S, int q, float& st,
                     float& sp) {
  const float2 pq = reinterpret_cast<const float2*>(S.pos)[q];  // 8-byte aligned
  st = pq.x;
  sp = pq.y;
  bool in = in_quad_edges(P, st, sp);
  if (P.picheck && !in && sp < PI2 * .2f) {
    sp += PI2;
    in = in_quad_edges(P, st, sp);
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
  h.bb = blackbody_index(S.mag[2 * q + 1], P.redshft, S.bb_n);
  const float4 c = S.bb_hsp[h.bb];
  h.hsp = make_float3(c.x, c.y, c.z);
  return h;
}

// Contribution of a star to cell (u, v) of its pixel, squared RGB
// (BT/MakeImageKernel.cu:305-320).  Returns false outside the splat radius.
BT_HD bool cell_light_v(int step, float maxDistSq, float frac, float st, float sp,
                        float part, float hx, float hy, float hz, int u, int v,
                        float3& out) {
  const float dist = dist_sq(-step + u + .5f, st, -step + v + .5f, sp);
  if (dist > maxDistSq) return false;
  const float appMag = part - 2.5f * log10f(frac * gaussian(dist));
  const float brightness = 100 * exp10f(-.4f * appMag);
  float r, g, b;
  hsp_to_rgb(hx, hy, hz * brightness, r, g, b);
  r *= 255.f;
  g *= 255.f;
  b *= 255.f;
  out = make_float3(r * r, g * g, b * b);
  return true;
}

BT_HD bool cell_light(const PixelStars& P, const StarHit& h, int u, int v,
                      float3& out) {
  return cell_light_v(P.step, P.maxDistSq, P.frac, h.st, h.sp, h.part, h.hsp.x, h.hsp.y,
                      h.hsp.z, u, v, out);
}

// True when no star inside box b (theta/phi ranges) can pass the quad test
// of pixel P: for one of the four edges, every point of the box lies on the
// rejecting side by more than the rounding error of cross_pos's float
// evaluation.  cross_pos(k) is c1t*(sp - pb) - (st - tb)*c1p > 0, linear in
// the star position, so its maximum over the box is at a corner; that maximum
// is compared against a bound of the float evaluation's error.  Both that evaluation and this one (in float too) are within a few
// units of 2^-24 of the terms' magnitudes (mag); the margin is 1e-5 * mag.
BT_HD bool box_outside(const PixelStars& P, float tmin, float pmin, float tmax,
                       float pmax) {
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const int k1 = (k + 1) & 3;
    const float c1t = P.et[k], c1p = P.ep[k];
    const float tb = P.t[k1], pb = P.p[k1];
    const float sp = c1t > 0 ? pmax : pmin;
    const float st = c1p > 0 ? tmin : tmax;
    const float fmax = c1t * (sp - pb) - (st - tb) * c1p;
    const float mag = fabsf(c1t) * fmaxf(fabsf(pmax - pb), fabsf(pmin - pb)) +
                      fabsf(c1p) * fmaxf(fabsf(tmax - tb), fabsf(tmin - tb));
    if (fmax < -(1e-5f * mag + 1e-30f)) return true;
  }
  return false;
}

// True when star_test rejects every star of a node with bounding box b,
// including the seam retry at phi + 2pi that pixels straddling phi = 0 take
// for stars with phi < 0.2 * 2pi.
BT_HD bool node_excluded(const PixelStars& P, float4 b) {
  if (!(b.x <= b.z) || !(b.y <= b.w)) return true;  // no stars
  if (!box_outside(P, b.x, b.y, b.z, b.w)) return false;
  if (!P.picheck || !(b.y < PI2 * .2f)) return true;
  const float lo = b.y + PI2, hi = fminf(b.w, PI2 * .2f) + PI2;
  return box_outside(P, b.x, lo - 1e-5f, b.z, hi + 1e-5f);
}

// Visits, left to right, the leaves under `root` (a node at level `lvl`)
// that hold a star which may pass the pixel's quad test; subtrees whose
// bounding box excludes every star are skipped.  Leaf star ranges are
// contiguous in tree order, so the visited stars keep the order of a plain
// scan of root's range, minus stars the test rejects anyway.
template <class Visit>
BT_HD bool walk_leaves(PixelStars& P, const StarSet& S, int root, int lvl,
                       Visit&& visit) {
  const int L = S.treeLevel;
  int k = root, l = lvl;
  for (;;) {
    // a node test costs about as much as four star tests
    P.tested += 4;
    if (P.tested > P.budget) {
      P.abort = true;
      return false;
    }
    if (!node_excluded(P, S.box[k])) {
      if (l >= L) {
        if (!visit(k)) return false;
      } else {
        k = 2 * k + 1;
        l++;
        continue;
      }
    }
    // next node in pre-order inside root's subtree
    while (k != root && (k & 1) == 0) {
      k = (k - 1) >> 1;
      l--;
    }
    if (k == root) return true;
    k++;
  }
}

// Level of node k in the implicit complete binary tree.
BT_HD int node_level(int k) { return 31 - clz_u32((unsigned)k + 1u); }

// Star tests a node costs in a pixel's budget (about four star tests).
constexpr int kNodeCost = 4;

// Start and end of a node's star range.
BT_HD void node_range(const StarSet& S, int node, int& a0, int& a1) {
  a0 = (node != 0 && ((node + 1) & node) != 0) ? S.tree[node - 1] : 0;
  a1 = S.tree[node];
}

// The per-pixel values the star tests and the splat need, compact enough to
// pass between lanes through shared memory.
struct PixelCore {
  float t[4], p[4];
  float red, redshft, frac;
  int bits;  // bit 0: picheck, bit 1: sgn < 0
};

BT_HD PixelCore core_of(const PixelStars& P) {
  PixelCore c;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    c.t[k] = P.t[k];
    c.p[k] = P.p[k];
  }
  c.red = P.red;
  c.redshft = P.redshft;
  c.frac = P.frac;
  c.bits = (P.picheck ? 1 : 0) | (P.sgn < 0 ? 2 : 0);
  return c;
}

BT_HD void stars_of(const PixelCore& c, int step, PixelStars& P) {
#pragma unroll
  for (int k = 0; k < 4; k++) {
    P.t[k] = c.t[k];
    P.p[k] = c.p[k];
  }
  P.sgn = (c.bits & 2) ? -1 : 1;
  P.picheck = (c.bits & 1) != 0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const int k1 = (k + 1) & 3;
    P.et[k] = (float)P.sgn * (P.t[k] - P.t[k1]);
    P.ep[k] = (float)P.sgn * (P.p[k] - P.p[k1]);
  }
  P.red = c.red;
  P.redshft = c.redshft;
  P.frac = c.frac;
  P.step = step;
  P.maxDistSq = (step + .5f) * (step + .5f);
  P.tested = 0;
  P.budget = 0x7fffffffffffL;
  P.abort = false;
  P.any = false;
  P.cells = nullptr;
}

// Per-star factors of the splat in a cheaper form.  cell_light computes
//   100 * 10^(-0.4 * (part - 2.5 log10(frac * g))) = 100 * 10^(-0.4 part) * frac * g
// and HSPtoRGB(h, s, p * b) = b * HSPtoRGB(h, s, p) (the HSP model is
// linear in its perceived brightness), so a star's colour and brightness are
// computed once and each cell needs only its Gaussian.  The two forms agree
// to float rounding (relative ~1e-6).  `ok` is false where the rewrite could
// differ by more than rounding -- a magnification factor that is not a
// positive finite number, or a brightness large enough for HSPtoRGB's P*P to
// overflow -- and those stars take cell_light.
struct StarFast {
  float b0;          // 100 * 10^(-0.4 part) * frac
  float r0, g0, bl0; // 255 * HSPtoRGB(h, s, p)
  bool ok;
};

BT_HD StarFast star_fast(const PixelStars& P, const StarSet& S, const StarHit& h) {
  StarFast f;
  f.b0 = 100.f * exp10f(-.4f * h.part) * P.frac;
  const float4 c = S.bb_rgb[h.bb];
  f.r0 = c.x;
  f.g0 = c.y;
  f.bl0 = c.z;
  f.ok = P.frac > 0.f && f.b0 < 1e15f && f.b0 > 0.f && h.hsp.z <= 1.f;
  return f;
}

// cell_light kept out of line for the rare stars star_fast does not cover,
// so that the unrolled cell loops stay small.
#ifdef __CUDA_ARCH__
__device__ __noinline__
#else
inline
#endif
bool cell_light_slow(int step, float maxDistSq, float frac, float st, float sp, float part,
                     float hx, float hy, float hz, int u, int v, float3& out) {
  return cell_light_v(step, maxDistSq, frac, st, sp, part, hx, hy, hz, u, v, out);
}

BT_HD bool cell_light_fast(const PixelStars& P, const StarHit& h, const StarFast& f,
                           int u, int v, float3& out) {
  const float dist = dist_sq(-P.step + u + .5f, h.st, -P.step + v + .5f, h.sp);
  if (dist > P.maxDistSq) return false;
  // gaussian(dist) = exp(-dist / (2 sigma^2)) / (sigma sqrt(2 pi)), sigma = 0.4
#ifdef __CUDA_ARCH__
  const float gauss = __expf(-3.125f * dist) * 0.99735570f;
#else
  const float gauss = expf(-3.125f * dist) * 0.99735570f;
#endif
  const float b = f.b0 * gauss;
  const float r = f.r0 * b, g = f.g0 * b, bl = f.bl0 * b;
  out = make_float3(r * r, g * g, bl * bl);
  return true;
}

// A star's (2 kStep + 1)^2 cells added into acc: the per-star form where it
// applies (f.ok), else cell_light.  Two separate unrolled loops, so that the
// hot one carries none of the rare one's call set-up (the star kernels are
// bound by instruction fetch).
template <int kStep>
BT_HD void splat_cells(const PixelStars& P, const StarHit& h, const StarFast& f,
                       float3* acc) {
  constexpr int FW = 2 * kStep + 1, FW2 = FW * FW;
  if (f.ok) {
#pragma unroll
    for (int c = 0; c < FW2; c++) {
      float3 l;
      if (cell_light_fast(P, h, f, c / FW, c % FW, l)) {
        acc[c].x += l.x;
        acc[c].y += l.y;
        acc[c].z += l.z;
      }
    }
  } else {
#pragma unroll
    for (int c = 0; c < FW2; c++) {
      float3 l;
      if (cell_light_slow(P.step, P.maxDistSq, P.frac, h.st, h.sp, h.part, h.hsp.x,
                          h.hsp.y, h.hsp.z, c / FW, c % FW, l)) {
        acc[c].x += l.x;
        acc[c].y += l.y;
        acc[c].z += l.z;
      }
    }
  }
}

#undef BT_HD

}  // namespace bt
