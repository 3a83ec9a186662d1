// map.cu -- the per-pixel map on the device: grid interpolation, black-hole
// mask, solid angles and their smoothing, the environment map's summed-area
// table and its integration over each projected pixel, with lensing and
// redshift (annemiekie/BlackTracer BT/MakeImageKernel.cu:458-751 and the
// summed-area table of cudaPrep :1312-1330).
//
// Thread mapping: x -> column j, y -> row i, so consecutive lanes touch
// consecutive pixels (the reference maps x to rows, which strides every
// access by a full row).  Compiled with --fmad=false so the FP32 arithmetic
// rounds like the reference's (see map_math.cuh).
#include <cstring>
#include <new>

#include "bt_internal.h"
#include "map_math.cuh"
#include "map_internal.h"

namespace bt {

using namespace mapm;

constexpr int TX = 32, TY = 8;

static dim3 grid2(int w, int h) {
  return dim3((unsigned)((w + TX - 1) / TX), (unsigned)((h + TY - 1) / TY));
}

// Camera-sky corners of an equirectangular output, Viewer::makeSphereView
// (BT/Viewer.h:82-88): {i*PI/H, j*PI2/W} evaluated in double, stored float.
__global__ void k_view_sphere(float2* view, int W, int H) {
  const int j = blockIdx.x * TX + threadIdx.x;
  const int i = blockIdx.y * TY + threadIdx.y;
  if (i > H || j > W) return;
  view[(size_t)i * (W + 1) + j] =
      make_float2((float)(1.f * i * kPi / H), (float)(1.f * j * kPi2 / W));
}

// pixInterpolation, G = 1 (BT/MakeImageKernel.cu:458-515): celestial
// (theta, phi) and block size at every pixel corner.  Bound by the latency
// of its grid reads: six blocks per SM (40 registers) instead of three.
__global__ void __launch_bounds__(TX * TY, 6)
k_pixinterp(const float2* __restrict__ view, int M, int N,
                            GridRef G, int gridlvl, float hor, float ver,
                            float2* __restrict__ thphi, int* __restrict__ gap) {
  const int j = blockIdx.x * TX + threadIdx.x;
  const int i = blockIdx.y * TY + threadIdx.y;
  const int M1 = M + 1;
  if (i > N || j > M) return;
  const float2 v = view[(size_t)i * M1 + j];
  const float theta = v.x + ver;
  const float phi = fmodf(v.y + hor + PI2, PI2);
  int g = 0;
  thphi[(size_t)i * M1 + j] = interpolate_pix(G, theta, phi, gridlvl, g);
  gap[(size_t)i * M1 + j] = g;
}

// ---------------------------------------------------------- G = 2 blending
// Interpolation between two grids computed for neighbouring camera poses
// (the reference's movement between precomputed grids, BT/MakeImageKernel.cu
// camUpdate / findBhCenter / findBhBorders / smoothBorder :386-456 and the
// Gr > 1 branch of pixInterpolation :466-510).  The border of the black hole
// is found in both grids along kBlendAngles directions from the centre of the
// captured region; near the black hole each grid is read at a position
// stretched towards its own border so that the shadow moves smoothly.

// findBhCenter (:391-404): bounding box (in radians) of the captured
// vertices of either grid.  box = {theta_min, theta_max}, {phi_min, phi_max};
// the values are non-negative, so float order equals their bits' int order.
__global__ void k_bh_center(const float2* __restrict__ ga, const float2* __restrict__ gb,
                            int GM, int GN, float2* box) {
  const int j = blockIdx.x * TX + threadIdx.x;
  const int i = blockIdx.y * TY + threadIdx.y;
  if (i >= GN || j >= GM) return;
  const size_t q = (size_t)i * GM + j;
  if (ga[q].x == -1.f || gb[q].x == -1.f) {
    const float gridsize = PI / (1.f * GN);
    atomicMin((int*)&box[0].x, __float_as_int(gridsize * (float)i));
    atomicMax((int*)&box[0].y, __float_as_int(gridsize * (float)i));
    atomicMin((int*)&box[1].x, __float_as_int(gridsize * (float)j));
    atomicMax((int*)&box[1].y, __float_as_int(gridsize * (float)j));
  }
}

// findBhBorders (:406-430): from the centre of the box, walk outwards in
// lattice steps along direction k until a vertex with theta > 0 follows a
// captured one (-1); thread 2k walks grid a, 2k+1 grid b.  The reference's
// walk has no bound (and reads past the lattice when it misses the border);
// here it stops at the lattice edge, and such walks are counted in *edge.
__global__ void k_bh_borders(const float2* __restrict__ ga, const float2* __restrict__ gb,
                             int GM, int GN, int nang, float2* border, uint32_t* edge) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nang * 2) return;
  const int ii = i / 2;
  const float2* g = (i % 2) ? gb : ga;
  const float angle = PI2 / (1.f * nang) * 1.f * ii;
  const float thetaChange = -sinf(angle);
  const float phiChange = cosf(angle);
  float2 pt = {.5f * border[0].x + .5f * border[0].y, .5f * border[1].x + .5f * border[1].y};
  pt = {pt.x / PI2 * GM, pt.y / PI2 * GM};
  float2 gridB = {-2, -2}, gridA = {-2, -2};
  const int cap = 4 * (GM + GN);
  int it = 0;
  while (!(gridA.x > 0 && gridB.x == -1)) {
    gridB = gridA;
    pt.x += thetaChange;
    pt.y += phiChange;
    const int gx = int(pt.x), gy = int(pt.y);
    if (gx < 0 || gy < 0 || gx >= GN || gy >= GM || ++it > cap) {
      atomicAdd(edge, 1u);
      break;
    }
    gridA = g[(size_t)gx * GM + gy];
  }
  border[2 + i] = {(pt.x - thetaChange) * PI2 / (1.f * GM), (pt.y - phiChange) * PI2 / (1.f * GM)};
}

// smoothBorder (:444-456): each border point averaged with its two
// neighbours of the same grid.
__global__ void k_smooth_border(const float2* __restrict__ in, float2* __restrict__ out, int nang) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nang * 2) return;
  if (i == 0) {
    out[0] = in[0];
    out[1] = in[1];
  }
  const int prev = (i - 2 + 2 * nang) % (2 * nang);
  const int next = (i + 2) % (2 * nang);
  out[i + 2] = {1.f / 3.f * (in[prev + 2].x + in[i + 2].x + in[next + 2].x),
                1.f / 3.f * (in[prev + 2].y + in[i + 2].y + in[next + 2].y)};
}

// pixInterpolation with Gr > 1 (:466-510): grid a weighted 1 - alpha, grid b
// alpha; the block gap kept is grid b's (the reference's second call writes
// it last).
__global__ void k_pixinterp2(const float2* __restrict__ view, int M, int N, GridRef GA,
                             GridRef GB, int gridlvl, float hor, float ver,
                             const float2* __restrict__ bhBorder, int angleNum, float alpha,
                             float2* __restrict__ thphi, int* __restrict__ gap) {
  const int j = blockIdx.x * TX + threadIdx.x;
  const int i = blockIdx.y * TY + threadIdx.y;
  const int M1 = M + 1;
  if (i > N || j > M) return;
  const float2 v = view[(size_t)i * M1 + j];
  const float theta = v.x + ver;
  const float phi = fmodf(v.y + hor + PI2, PI2);
  const size_t q = (size_t)i * M1 + j;
  float2 A, B;
  int ga = 0, gb = 0;
  const float2 center = {.5f * bhBorder[0].x + .5f * bhBorder[0].y,
                         .5f * bhBorder[1].x + .5f * bhBorder[1].y};
  const float stretchRad =
      fmaxf(bhBorder[0].y - bhBorder[0].x, bhBorder[1].x - bhBorder[1].y) * 0.75f;
  const float centerdist =
      (theta - center.x) * (theta - center.x) + (phi - center.y) * (phi - center.y);
  if (centerdist < stretchRad * stretchRad) {
    float angle = atan2f(center.x - theta, phi - center.y);
    angle = fmodf(angle + PI2, PI2);
    const int angleSlot = angle / PI2 * angleNum;
    const float2 bA = bhBorder[2 * angleSlot + 2], bB = bhBorder[2 * angleSlot + 3];
    const float2 bhBorderNew = {(1.f - alpha) * bA.x + alpha * bB.x,
                                (1.f - alpha) * bA.y + alpha * bB.y};
    if (centerdist <= (bhBorderNew.x - center.x) * (bhBorderNew.x - center.x) +
                          (bhBorderNew.y - center.y) * (bhBorderNew.y - center.y)) {
      thphi[q] = {-1, -1};
      // the reference returns here without writing gapsave (an earlier
      // frame's value, or uninitialised memory); 0 keeps frames reproducible
      gap[q] = 0;
      return;
    }
    const float tStoB = (center.x - stretchRad * sinf(angle) - bhBorderNew.x);
    const float pStoB = (center.y + stretchRad * cosf(angle) - bhBorderNew.y);
    const float thetaPerc = fabsf(tStoB) < 1E-5 ? 0 : 1.f - (theta - bhBorderNew.x) / tStoB;
    const float phiPerc = fabsf(pStoB) < 1E-5 ? 0 : 1.f - (phi - bhBorderNew.y) / pStoB;
    const float thetaA = theta - thetaPerc * (bhBorderNew.x - bA.x);
    const float phiA = phi - phiPerc * (bhBorderNew.y - bA.y);
    const float thetaB = theta - thetaPerc * (bhBorderNew.x - bB.x);
    const float phiB = phi - phiPerc * (bhBorderNew.y - bB.y);
    A = interpolate_pix(GA, thetaA, phiA, gridlvl, ga);
    B = interpolate_pix(GB, thetaB, phiB, gridlvl, gb);
  } else {
    A = interpolate_pix(GA, theta, phi, gridlvl, ga);
    B = interpolate_pix(GB, theta, phi, gridlvl, gb);
  }
  gap[q] = gb;
  if (A.x == -1 || B.x == -1) {
    thphi[q] = {-1, -1};
  } else {
    if (A.y < .2f * PI2 && B.y > .8f * PI2) A.y += PI2;
    if (B.y < .2f * PI2 && A.y > .8f * PI2) B.y += PI2;
    thphi[q] = {(1.f - alpha) * A.x + alpha * B.x, fmodf((1.f - alpha) * A.y + alpha * B.y, PI2)};
  }
}

int blend_prepare(const float2* ga, const float2* gb, int GN, int GM, float2* border,
                  float2* border2, int nang, uint32_t* edge, cudaStream_t s) {
  // {100, 0} per axis, as the reference initialises its box (:1308-1310)
  const float2 init[2] = {{100.f, 0.f}, {100.f, 0.f}};
  BT_CUDA_TRY(cudaMemcpyAsync(border, init, sizeof(init), cudaMemcpyHostToDevice, s));
  BT_CUDA_TRY(cudaMemsetAsync(edge, 0, sizeof(uint32_t), s));
  k_bh_center<<<grid2(GM, GN), dim3(TX, TY), 0, s>>>(ga, gb, GM, GN, border);
  const unsigned nb = (unsigned)((2 * nang + 255) / 256);
  k_bh_borders<<<nb, 256, 0, s>>>(ga, gb, GM, GN, nang, border, edge);
  for (int r = 0; r < 2; r++) {
    k_smooth_border<<<nb, 256, 0, s>>>(border, border2, nang);
    k_smooth_border<<<nb, 256, 0, s>>>(border2, border, nang);
  }
  BT_CUDA_TRY(cudaGetLastError());
  return BT_OK;
}

// findBlackPixels + findArea (BT/MakeImageKernel.cu:539-568), fused.
__global__ void k_bh_area(const float2* __restrict__ thphi, int M, int N,
                          uint8_t* __restrict__ bh, float* __restrict__ area) {
  const int j = blockIdx.x * TX + threadIdx.x;
  const int i = blockIdx.y * TY + threadIdx.y;
  if (i >= N || j >= M) return;
  float t[4], p[4];
  bool picheck = false;
  const bool ok = pixel_corners(thphi, i * (M + 1) + j, M, t, p, picheck, 0.f);
  bh[(size_t)i * M + j] = ok ? 0 : 1;
  // the reference computes the area for captured pixels too, from the
  // partially wrapped corners; those values are never read
  area[(size_t)i * M + j] = ok ? pixel_solid_angle(t, p) : 0.f;
}

__device__ __forceinline__ int corner_gap(const int* gap, int i, int j, int M) {
  const int M1 = M + 1;
  return max(max(gap[i * M1 + j], gap[i * M1 + M1 + j]),
             max(gap[i * M1 + j + 1], gap[i * M1 + M1 + j + 1]));
}

// smoothAreaH (BT/MakeImageKernel.cu:570-591): box filter along the row,
// width max(corner gaps)/2, over non-black pixels; the column wraps.
__global__ void k_smooth_h(float* __restrict__ out, const float* __restrict__ area,
                           const uint8_t* __restrict__ bh, const int* __restrict__ gap,
                           int M, int N) {
  const int j = blockIdx.x * TX + threadIdx.x;
  const int i = blockIdx.y * TY + threadIdx.y;
  if (i >= N || j >= M) return;
  if (bh[(size_t)i * M + j] == 1) return;
  const int fs = corner_gap(gap, i, j, M) / 2;
  float sum = 0.f;
  int count = 0;
  const size_t row = (size_t)i * M;
  for (int h = -fs; h <= fs; h++) {
    int jj = (j + h) % M;
    if (jj < 0) jj += M;
    if (bh[row + jj] == 0) {
      sum += area[row + jj];
      count++;
    }
  }
  out[row + j] = sum / (1.f * count);
}

// smoothAreaV (BT/MakeImageKernel.cu:593-616): the same along the column,
// clamped at the image edges; writes back into `area`.
__global__ void k_smooth_v(const float* __restrict__ in, float* __restrict__ area,
                           const uint8_t* __restrict__ bh, const int* __restrict__ gap,
                           int M, int N) {
  const int j = blockIdx.x * TX + threadIdx.x;
  const int i = blockIdx.y * TY + threadIdx.y;
  if (i >= N || j >= M) return;
  if (bh[(size_t)i * M + j] == 1) return;
  const int fs = corner_gap(gap, i, j, M) / 2;
  float sum = 0.f;
  const int minv = max(0, i - fs);
  const int maxv = min(N - 1, i + fs);
  int count = 0;
  for (int h = minv; h <= maxv; h++) {
    if (bh[(size_t)h * M + j] == 0) {
      sum += in[(size_t)h * M + j];
      count++;
    }
  }
  area[(size_t)i * M + j] = sum / (1.f * count);
}

// Summed-area table of the environment map (cudaPrep, BT/MakeImageKernel.cu
// :1312-1330): per column, down the rows, the running float sums of
// B^2.2 A, G^2.2 A, R^2.2 A and A, A the cell's solid angle (calcArea,
// BT/kernel.cuh:586-610).  The reference computes it on the host, and a
// cell of a 2048- to 16384-column map is so small that calcArea's float
// result carries rounding noise of ~1e-3 relative which the host's sinf /
// cosf / atanf decide.  To give the reference's table, the cell areas take
// the host's sinf and cosf of the grid angles (every argument is pxsz * k,
// k integer: tables made by the host) and atanf as the double atan rounded
// to float (which equals the host's atanf on the arguments calcArea
// produces: checked on every cell of 2048- and sampled cells of 8192- and
// 16384-column maps), and byte^2.2 the host's powf (a 256-entry table); the
// float operations are calcArea's, FMA off.
//
// Pass 1: one thread per cell writes its four terms into the table.
__global__ void k_sat_terms(const uint8_t* __restrict__ bgr, int rows, int cols,
                            const float* __restrict__ sin_t, const float* __restrict__ cos_t,
                            const float* __restrict__ pow_t, float4* __restrict__ sat) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= cols) return;
  for (int p = blockIdx.y; p < rows; p += gridDim.y) {
    // theta = {pxsz (p+1), pxsz p, pxsz p, pxsz (p+1)}, phi = {pxsz q, pxsz q,
    // pxsz (q+1), pxsz (q+1)}
    const int it[4] = {p + 1, p, p, p + 1};
    const int ip[4] = {q, q, q + 1, q + 1};
    float x[4], y[4], z[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const float sint = sin_t[it[k]];
      x[k] = sint * cos_t[ip[k]];
      y[k] = sint * sin_t[ip[k]];
      z[k] = cos_t[it[k]];
    }
    float dotpr1 = 1.f;
    dotpr1 += x[0] * x[2] + y[0] * y[2] + z[0] * z[2];
    float dotpr2 = dotpr1;
    dotpr1 += x[2] * x[1] + y[2] * y[1] + z[2] * z[1];
    dotpr1 += x[0] * x[1] + y[0] * y[1] + z[0] * z[1];
    dotpr2 += x[0] * x[3] + y[0] * y[3] + z[0] * z[3];
    dotpr2 += x[2] * x[3] + y[2] * y[3] + z[2] * z[3];
    const float triprod1 = fabsf(x[0] * (y[1] * z[2] - y[2] * z[1]) -
                                 y[0] * (x[1] * z[2] - x[2] * z[1]) +
                                 z[0] * (x[1] * y[2] - x[2] * y[1]));
    const float triprod2 = fabsf(x[0] * (y[2] * z[3] - y[3] * z[2]) -
                                 y[0] * (x[2] * z[3] - x[3] * z[2]) +
                                 z[0] * (x[2] * y[3] - x[3] * y[2]));
    const float a1 = (float)atan((double)(triprod1 / dotpr1));
    const float a2 = (float)atan((double)(triprod2 / dotpr2));
    const float area = 2.f * (a1 + a2);
    const uint8_t* px = bgr + ((size_t)p * cols + q) * 3;
    sat[(size_t)p * cols + q] =
        make_float4(pow_t[px[0]] * area, pow_t[px[1]] * area, pow_t[px[2]] * area, area);
  }
}

// Pass 2: one thread per column adds the terms down the rows in place, in
// the reference's order.
__global__ void k_sat_scan(int rows, int cols, float4* __restrict__ sat) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= cols) return;
  float4 prev = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int p = 0; p < rows; p++) {
    const float4 t = sat[(size_t)p * cols + q];
    prev.x += t.x;
    prev.y += t.y;
    prev.z += t.z;
    prev.w += t.w;
    sat[(size_t)p * cols + q] = prev;
  }
}

// Summed-area table read at the reference's linear index.  The reference
// can index a row before the table (int(thMin/pixSize)-1 = -1, :664) and up
// to a row past it (theta = pi, or a phi that rounds to `cols`); such reads
// return zero here.
__device__ __forceinline__ float4 sat_lin(const float4* sat, long idx, long total) {
  if (idx < 0 || idx >= total) return make_float4(0.f, 0.f, 0.f, 0.f);
  return sat[idx];
}

// Colour of a pixel from its summed environment (B, G, R, solid angle):
// gamma, HSP, lensing and redshift (BT/MakeImageKernel.cu:725-750); BGRA8.
__device__ __forceinline__ uchar4 env_finish(float4 color, const float* t, const float* p,
                                             int M, int ind, const Cam7& cam,
                                             const float2* view, float solidangle, int lr) {
  color.x = fminf(255.f, powf(color.x / color.w, 1.f / 2.2f));
  color.y = fminf(255.f, powf(color.y / color.w, 1.f / 2.2f));
  color.z = fminf(255.f, powf(color.z / color.w, 1.f / 2.2f));
  float H, S, P;
  rgb_to_hsp(color.z / 255.f, color.y / 255.f, color.x / 255.f, H, S, P);
  if (lr) {
    float redshft, frac;
    lensing_redshift(t, p, M, ind, cam.v, view, frac, redshft, solidangle);
    P *= frac;
    P = powf(P, redshft);
  }
  hsp_to_rgb(H, S, fminf(1.f, P), color.z, color.y, color.x);
  return make_uchar4((unsigned char)min(255, int(color.x * 255)),
                     (unsigned char)min(255, int(color.y * 255)),
                     (unsigned char)min(255, int(color.z * 255)), 255);
}

// Columns of the environment map a projected pixel spans (BT/MakeImageKernel.cu:650-657).
struct EnvSpan {
  float pixSize;
  int pixMin, pixNum;
};

__device__ __forceinline__ EnvSpan env_span(const float* p, int rows) {
  EnvSpan e;
  e.pixSize = PI / float(rows);
  const float phMax = fmaxf(fmaxf(p[0], p[1]), fmaxf(p[2], p[3]));
  const float phMin = fminf(fminf(p[0], p[1]), fminf(p[2], p[3]));
  const int pixMax = int(phMax / e.pixSize);
  e.pixMin = int(phMin / e.pixSize);
  e.pixNum = pixMax - e.pixMin + 1;
  if (e.pixNum > 1 && pixMax * e.pixSize > phMax) e.pixNum -= 1;
  return e;
}

// Pixels spanning at least this many environment columns are integrated by
// a warp each (k_env_wide); next to the shadow a pixel can span all of them.
constexpr int kEnvWide = 48;

// distortEnvironmentMap (BT/MakeImageKernel.cu:631-751): integrate the
// environment over the projected pixel column by column with two
// summed-area reads per column, gamma, HSP, lensing and redshift; BGRA8.
// Pixels spanning kEnvWide columns or more are queued for k_env_wide.
__global__ void k_env(const float2* __restrict__ thphi, uchar4* __restrict__ out,
                      const uint8_t* __restrict__ bh, int rows, int cols, int M,
                      int N, const float4* __restrict__ sat, Cam7 cam,
                      const float* __restrict__ solidangle,
                      const float2* __restrict__ view, int lr,
                      uint32_t* __restrict__ wide, uint32_t* nwide) {
  const int j = blockIdx.x * TX + threadIdx.x;
  const int i = blockIdx.y * TY + threadIdx.y;
  if (i >= N || j >= M) return;
  const size_t ij = (size_t)i * M + j;
  const long total = (long)rows * cols;
  if (bh[ij] == 0) {
    float t[4], p[4];
    bool picheck = false;
    const int ind = i * (M + 1) + j;
    const bool ok = pixel_corners(thphi, ind, M, t, p, picheck, 0.f);
    if (ok && ind > 0) {  // pixel (0,0) is never coloured by the reference
      const EnvSpan e = env_span(p, rows);
      const float pixSize = e.pixSize;
      const int pixMin = e.pixMin, pixNum = e.pixNum;
      if (pixNum >= kEnvWide) {
        wide[atomicAdd(nwide, 1u)] = (uint32_t)ij;
        return;
      }
      float4 color = make_float4(0.f, 0.f, 0.f, 0.f);
      if (pixNum == 1) {
        const float thMax = fmaxf(fmaxf(t[0], t[1]), fmaxf(t[2], t[3]));
        const float thMin = fminf(fminf(t[0], t[1]), fminf(t[2], t[3]));
        const float4 mx = sat_lin(sat, (long)int(thMax / pixSize) * cols + pixMin, total);
        const float4 mn = sat_lin(sat, (long)(int(thMin / pixSize) - 1) * cols + pixMin, total);
        color.x += mx.x - mn.x;
        color.y += mx.y - mn.y;
        color.z += mx.z - mn.z;
        color.w += mx.w - mn.w;
      } else if (pixNum < cols) {
        // max2/min2 are running extremes over all boundaries so far, as in
        // the reference (they are not reset per column)
        float max1 = -100, min1 = cols + 1, max2 = -100, min2 = cols + 1;
        for (int s = 0; s <= pixNum; s++) {
          const float cp = (pixMin + s) * pixSize;
          for (int q = 0; q < 4; q++) {
            const float ap = p[q], bp = p[(q + 1) % 4];
            const float at = t[q], bt = t[(q + 1) % 4];
            if ((cp - ap) * (cp - bp) <= 0) {
              const float ct = at + (bt - at) / (bp - ap) * (cp - ap);
              min2 = ct < min2 ? ct : min2;
              max2 = ct > max2 ? ct : max2;
            }
          }
          if (s > 0) {
            const float max_ = fmaxf(max1, max2);
            const float min_ = fminf(min1, min2);
            const int col = (pixMin + s) % cols;
            const long index1 = (long)int(max_ / pixSize) * cols + col;
            const long index2 = (long)(int(min_ / pixSize) - 1) * cols + col;
            const float4 mx = sat_lin(sat, index1, total);
            const float4 mn = index2 > 0 ? sat_lin(sat, index2, total)
                                         : make_float4(0.f, 0.f, 0.f, 0.f);
            color.x += mx.x - mn.x;
            color.y += mx.y - mn.y;
            color.z += mx.z - mn.z;
            color.w += mx.w - mn.w;
          }
          max1 = max2;
          min1 = min2;
        }
      } else {
        const float thMax = fmaxf(fmaxf(t[0], t[1]), fmaxf(t[2], t[3]));
        const float thMin = fminf(fminf(t[0], t[1]), fminf(t[2], t[3]));
        const long thMaxPix = (long)int(thMax / pixSize) * cols;
        const long thMinPix = (long)int(thMin / pixSize) * cols;
        for (int q = 0; q < pixNum; q++) {
          const int col = (pixMin + q) % cols;
          const float4 mx = sat_lin(sat, thMaxPix + col, total);
          const float4 mn = sat_lin(sat, thMinPix + col, total);
          color.x += mx.x - mn.x;
          color.y += mx.y - mn.y;
          color.z += mx.z - mn.z;
          color.w += mx.w - mn.w;
        }
      }
      out[ij] = env_finish(color, t, p, M, ind, cam, view, solidangle[ij], lr);
      return;
    }
  }
  out[ij] = make_uchar4(0, 0, 0, 255);
}

// Adds the per-column differences d of 32 consecutive columns (one per lane,
// lane order = column order; lanes [first, last] valid) to `color` one after
// the other, as the reference's sequential loop does; every lane ends with
// the same color.  The values pass through the warp's 32 float4 of shared
// memory (one broadcast load per column instead of four shuffles; the
// kernel is bound by issue, and this sum is most of its instructions).
__device__ __forceinline__ void add_in_order(float4& color, float4 d, int first, int last,
                                             float4* sh) {
  const int lane = threadIdx.x & 31;
  __syncwarp();
  sh[lane] = d;
  __syncwarp();
  if (first == 0 && last == 31) {
#pragma unroll
    for (int b = 0; b < 32; b++) {
      const float4 v = sh[b];
      color.x += v.x;
      color.y += v.y;
      color.z += v.z;
      color.w += v.w;
    }
  } else {
    for (int b = first; b <= last; b++) {
      const float4 v = sh[b];
      color.x += v.x;
      color.y += v.y;
      color.z += v.z;
      color.w += v.w;
    }
  }
}

// The wide pixels of k_env, one warp each: 32 columns per step, the running
// theta extremes of the reference as a warp prefix max/min, column sums
// added in column order (bit-identical to the per-thread loop).
constexpr int kEnvWideThreads = 256;

__global__ void __launch_bounds__(kEnvWideThreads)
k_env_wide(const float2* __restrict__ thphi, uchar4* __restrict__ out,
                           int rows, int cols, int M, const float4* __restrict__ sat,
                           Cam7 cam, const float* __restrict__ solidangle,
                           const float2* __restrict__ view, int lr,
                           const uint32_t* __restrict__ wide, const uint32_t* nwide) {
  const int lane = threadIdx.x & 31;
  __shared__ float4 sh_d[kEnvWideThreads / 32][32];
  float4* sh = sh_d[threadIdx.x >> 5];
  const uint32_t n = *nwide;
  const long total = (long)rows * cols;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t item = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; item < n;
       item += warps) {
    const uint32_t ij = wide[item];
    const int i = ij / M, j = ij % M;
    float t[4], p[4];
    bool picheck = false;
    const int ind = i * (M + 1) + j;
    pixel_corners(thphi, ind, M, t, p, picheck, 0.f);
    const EnvSpan e = env_span(p, rows);
    const float pixSize = e.pixSize;
    const int pixMin = e.pixMin, pixNum = e.pixNum;
    float4 color = make_float4(0.f, 0.f, 0.f, 0.f);
    if (pixNum < cols) {
      float cmax = -100, cmin = cols + 1;  // running extremes before this step
      for (int s0 = 0; s0 <= pixNum; s0 += 32) {
        const int s = s0 + lane;
        float lmax = -100, lmin = cols + 1;
        if (s <= pixNum) {
          const float cp = (pixMin + s) * pixSize;
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const float ap = p[q], bp = p[(q + 1) & 3];
            const float at = t[q], bt = t[(q + 1) & 3];
            if ((cp - ap) * (cp - bp) <= 0) {
              const float ct = at + (bt - at) / (bp - ap) * (cp - ap);
              lmin = ct < lmin ? ct : lmin;
              lmax = ct > lmax ? ct : lmax;
            }
          }
        }
        // inclusive prefix max / min over the lanes, then the carry
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const float a = __shfl_up_sync(0xffffffffu, lmax, o);
          const float b = __shfl_up_sync(0xffffffffu, lmin, o);
          if (lane >= o) {
            lmax = a > lmax ? a : lmax;
            lmin = b < lmin ? b : lmin;
          }
        }
        lmax = lmax > cmax ? lmax : cmax;
        lmin = lmin < cmin ? lmin : cmin;
        float4 d = make_float4(0.f, 0.f, 0.f, 0.f);
        if (s >= 1 && s <= pixNum) {
          const int col = (pixMin + s) % cols;
          const long index1 = (long)int(lmax / pixSize) * cols + col;
          const long index2 = (long)(int(lmin / pixSize) - 1) * cols + col;
          const float4 mx = sat_lin(sat, index1, total);
          const float4 mn = index2 > 0 ? sat_lin(sat, index2, total)
                                       : make_float4(0.f, 0.f, 0.f, 0.f);
          d = make_float4(mx.x - mn.x, mx.y - mn.y, mx.z - mn.z, mx.w - mn.w);
        }
        // columns s >= 1 only: lane 0 of the first step holds boundary 0
        add_in_order(color, d, s0 == 0 ? 1 : 0, min(31, pixNum - s0), sh);
        cmax = __shfl_sync(0xffffffffu, lmax, 31);
        cmin = __shfl_sync(0xffffffffu, lmin, 31);
      }
    } else {
      const float thMax = fmaxf(fmaxf(t[0], t[1]), fmaxf(t[2], t[3]));
      const float thMin = fminf(fminf(t[0], t[1]), fminf(t[2], t[3]));
      const long thMaxPix = (long)int(thMax / pixSize) * cols;
      const long thMinPix = (long)int(thMin / pixSize) * cols;
      for (int q0 = 0; q0 < pixNum; q0 += 32) {
        const int q = q0 + lane;
        float4 d = make_float4(0.f, 0.f, 0.f, 0.f);
        if (q < pixNum) {
          const int col = (pixMin + q) % cols;
          const float4 mx = sat_lin(sat, thMaxPix + col, total);
          const float4 mn = sat_lin(sat, thMinPix + col, total);
          d = make_float4(mx.x - mn.x, mx.y - mn.y, mx.z - mn.z, mx.w - mn.w);
        }
        add_in_order(color, d, 0, min(31, pixNum - q0 - 1), sh);
      }
    }
    const uchar4 px = env_finish(color, t, p, M, ind, cam, view, solidangle[ij], lr);
    if (lane == 0) out[ij] = px;
  }
}

int map_run_env(MapScratch& S, const MapFrame& F, cudaStream_t s) {
  if (int rc = map_run_prep(S, F, s)) return rc;
  return map_run_envmap(S, F, s);
}

int map_run_prep(MapScratch& S, const MapFrame& F, cudaStream_t s) {
  const int M = S.M, N = S.N;
  GridRef G{F.grid, F.GM, F.GN};
  if (F.grid2) {
    GridRef G2{F.grid2, F.GM, F.GN};
    k_pixinterp2<<<grid2(M + 1, N + 1), dim3(TX, TY), 0, s>>>(
        F.view, M, N, G, G2, F.gridlvl, F.hor, F.ver, F.blend_border, F.blend_angles, F.alpha,
        S.thphi, S.gap);
  } else {
    k_pixinterp<<<grid2(M + 1, N + 1), dim3(TX, TY), 0, s>>>(
        F.view, M, N, G, F.gridlvl, F.hor, F.ver, S.thphi, S.gap);
  }
  k_bh_area<<<grid2(M, N), dim3(TX, TY), 0, s>>>(S.thphi, M, N, S.bh, S.area);
  k_smooth_h<<<grid2(M, N), dim3(TX, TY), 0, s>>>(S.area_tmp, S.area, S.bh, S.gap, M, N);
  k_smooth_v<<<grid2(M, N), dim3(TX, TY), 0, s>>>(S.area_tmp, S.area, S.bh, S.gap, M, N);
  BT_CUDA_TRY(cudaGetLastError());
  return BT_OK;
}

int map_run_envmap(MapScratch& S, const MapFrame& F, cudaStream_t s) {
  const int M = S.M, N = S.N;
  if (F.map && F.env) {
    BT_CUDA_TRY(cudaMemsetAsync(S.env_wide_count, 0, sizeof(uint32_t), s));
    k_env<<<grid2(M, N), dim3(TX, TY), 0, s>>>(
        S.thphi, (uchar4*)F.out_bg, S.bh, F.env->rows, F.env->cols, M, N,
        F.env->sat, F.cam, S.area, F.view, F.lr, S.env_wide, S.env_wide_count);
    k_env_wide<<<sm_count() * 8, kEnvWideThreads, 0, s>>>(
        S.thphi, (uchar4*)F.out_bg, F.env->rows, F.env->cols, M, F.env->sat, F.cam,
        S.area, F.view, F.lr, S.env_wide, S.env_wide_count);
    BT_CUDA_TRY(cudaGetLastError());
  }
  return BT_OK;
}

// Census of the environment pass of the last frame: per coloured pixel the
// environment columns it spans (pixNum, BT/MakeImageKernel.cu:650-657);
// sums pixNum + 1 and the pixels into out[0] and out[1].
__global__ void k_env_census(const float2* __restrict__ thphi, const uint8_t* __restrict__ bh,
                             int rows, int M, int N, unsigned long long* out) {
  const int j = blockIdx.x * TX + threadIdx.x;
  const int i = blockIdx.y * TY + threadIdx.y;
  unsigned long long cols = 0, px = 0;
  if (i < N && j < M && bh[(size_t)i * M + j] == 0) {
    float t[4], p[4];
    bool picheck = false;
    const int ind = i * (M + 1) + j;
    if (pixel_corners(thphi, ind, M, t, p, picheck, 0.f) && ind > 0) {
      cols = (unsigned long long)(env_span(p, rows).pixNum + 1);
      px = 1;
    }
  }
  for (int o = 16; o; o >>= 1) {
    cols += __shfl_down_sync(0xffffffffu, cols, o);
    px += __shfl_down_sync(0xffffffffu, px, o);
  }
  if ((threadIdx.x & 31) == 0 && (cols || px)) {
    atomicAdd(out, cols);
    atomicAdd(out + 1, px);
  }
}

int map_env_census(const MapScratch& S, int env_rows, unsigned long long* out, cudaStream_t s) {
  k_env_census<<<grid2(S.M, S.N), dim3(TX, TY), 0, s>>>(S.thphi, S.bh, env_rows, S.M, S.N, out);
  BT_CUDA_TRY(cudaGetLastError());
  return BT_OK;
}

int launch_view_sphere(float2* view, int W, int H, cudaStream_t s) {
  k_view_sphere<<<grid2(W + 1, H + 1), dim3(TX, TY), 0, s>>>(view, W, H);
  BT_CUDA_TRY(cudaGetLastError());
  return BT_OK;
}

int launch_sat(const uint8_t* bgr, int rows, int cols, const float* sin_t, const float* cos_t,
               const float* pow_t, float4* sat, cudaStream_t s) {
  k_sat_terms<<<dim3((cols + 127) / 128, rows < 65535 ? rows : 65535), 128, 0, s>>>(
      bgr, rows, cols, sin_t, cos_t, pow_t, sat);
  k_sat_scan<<<(cols + 127) / 128, 128, 0, s>>>(rows, cols, sat);
  BT_CUDA_TRY(cudaGetLastError());
  return BT_OK;
}

}  // namespace bt
