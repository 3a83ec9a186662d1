// ref_map_harness.cpp -- runs the REFERENCE's per-pixel map kernels on the
// host.  TEST INFRASTRUCTURE ONLY.
//
// oracle/Makefile extracts the kernel bodies of the reference
// (BT/MakeImageKernel.cu lines 27-853: the kernels only, no GL, no host
// driver) into oracle/_ref/mik_body.inc at build time and compiles them here
// for the host together with the reference's device helpers (BT/kernel.cuh),
// with CUDA's qualifiers and builtins defined away.  Nothing of the reference
// is copied into this repository.
//
// Each kernel is run once per valid pixel / corner (blockDim = 1, blockIdx =
// (i, j)), which is the reference's per-thread computation without the
// out-of-range threads its launch shapes create (distortEnvironmentMap,
// distortStarMap, sumStarLight, makePix and addStarsAndBackground have no
// bounds check and index past the image when N or M is not a multiple of
// their block shape).  The summed-area table of cudaPrep
// (BT/MakeImageKernel.cu:1312-1330) lives in the host driver outside that
// range, so it is restated below (btref_map_sat), calling the reference's
// calcArea.
#define _GNU_SOURCE 1
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <strings.h>
#include <sys/mman.h>
#include <chrono>
#include <vector>

#include <omp.h>

#include "opencv2/core/core.hpp"
// threadIdx & co become per-thread host variables the driver sets.
#define __STORAGE__ thread_local
#include "cuda_runtime.h"
#include "device_launch_parameters.h"

#undef __device__
#undef __global__
#undef __host__
#undef __constant__
#undef __forceinline__
#define __device__
#define __global__
#define __host__
#define __constant__
#define __forceinline__ inline

using namespace std;
typedef unsigned int uint;

// ---- device intrinsics used by the kernels, for one host thread ----
// int atomicAdd is a real atomic: the timing driver below runs pixels on
// several host threads (addTrails counts hits per star with it).
static inline int atomicAdd(int* p, int v) { return __atomic_fetch_add(p, v, __ATOMIC_RELAXED); }
static inline float atomicAdd(float* p, float v) { float o = *p; *p += v; return o; }
static inline int atomicMin(int* p, int v) { int o = *p; *p = std::min(o, v); return o; }
static inline int atomicMax(int* p, int v) { int o = *p; *p = std::max(o, v); return o; }
static inline unsigned atomicMin(unsigned* p, unsigned v) { unsigned o = *p; *p = std::min(o, v); return o; }
static inline unsigned atomicMax(unsigned* p, unsigned v) { unsigned o = *p; *p = std::max(o, v); return o; }
static inline int __ffs(unsigned x) { return ffs((int)x); }
static inline float __int_as_float(int x) { float f; memcpy(&f, &x, 4); return f; }
static inline int __float_as_int(float x) { int i; memcpy(&i, &x, 4); return i; }
static inline float __uint_as_float(unsigned x) { float f; memcpy(&f, &x, 4); return f; }
static inline unsigned __float_as_uint(float x) { unsigned i; memcpy(&i, &x, 4); return i; }

#include "kernel.cuh"
#define ij (i * M + j)
#include "mik_body.inc"
#undef ij

namespace {
inline void at(int i, int j) {
  blockIdx.x = i; blockIdx.y = j; blockIdx.z = 0;
  threadIdx.x = threadIdx.y = threadIdx.z = 0;
  blockDim.x = blockDim.y = blockDim.z = 1;
}
}  // namespace

namespace {
// Zero-filled memory reserved on first touch, for arrays indexed by pixel of
// which a sample touches only a few rows.
template <class T>
struct Lazy {
  T* p = nullptr;
  size_t bytes = 0;
  explicit Lazy(size_t n) : bytes(n * sizeof(T)) {
    void* m = mmap(nullptr, bytes, PROT_READ | PROT_WRITE,
                   MAP_PRIVATE | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
    p = m == MAP_FAILED ? nullptr : (T*)m;
  }
  ~Lazy() {
    if (p) munmap(p, bytes);
  }
};
double secs_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}
}  // namespace

extern "C" {

// pixInterpolation (G = 1) for every corner (N+1) x (M+1).
void btref_map_pixinterp(const float* view, int M, int N, const float* grid,
                         int GM, int GN1, int gridlvl, float hor, float ver,
                         float* thphi, int* gap) {
  float2 border[4] = {};
  for (int i = 0; i <= N; i++)
    for (int j = 0; j <= M; j++) {
      at(i, j);
      pixInterpolation((const float2*)view, M, N, 1, (float2*)thphi,
                       (const float2*)grid, GM, GN1, hor, ver, gap, gridlvl,
                       border, 1000, 0.f);
    }
}

// The Gr = 2 path: findBhCenter, findBhBorders, smoothBorder x 4
// (BT/MakeImageKernel.cu:391-456, as the reference sequences them) on two
// grids stored one after the other (2 x GN1 x GM float2), then
// pixInterpolation with Gr = 2 for every corner.  border: (2 + 2*angleNum)
// float2 out.  Only for grids where every border walk ends inside the
// lattice (the reference's walk has no bound).
void btref_map_pixinterp_blend(const float* view, int M, int N, const float* grid2,
                               int GM, int GN1, int gridlvl, float hor, float ver,
                               float alpha, float* thphi, int* gap, float* border_out) {
  const int angleNum = 1000;
  std::vector<float2> b1((size_t)(angleNum + 1) * 2), b2((size_t)(angleNum + 1) * 2);
  b1[0] = {100, 0};
  b1[1] = {100, 0};
  const float2* g = (const float2*)grid2;
  for (int i = 0; i < GN1; i++)
    for (int j = 0; j < GM; j++) {
      at(i, j);
      findBhCenter(GM, GN1, g, b1.data());
    }
  for (int i = 0; i < angleNum * 2; i++) {
    at(i, 0);
    findBhBorders(GM, GN1, g, angleNum, b1.data());
  }
  for (int r = 0; r < 2; r++) {
    for (int i = 0; i < angleNum * 2; i++) {
      at(i, 0);
      smoothBorder(b1.data(), b2.data(), angleNum);
    }
    for (int i = 0; i < angleNum * 2; i++) {
      at(i, 0);
      smoothBorder(b2.data(), b1.data(), angleNum);
    }
  }
  for (int i = 0; i <= N; i++)
    for (int j = 0; j <= M; j++) {
      at(i, j);
      pixInterpolation((const float2*)view, M, N, 2, (float2*)thphi, g, GM, GN1, hor, ver,
                       gap, gridlvl, b1.data(), angleNum, alpha);
    }
  memcpy(border_out, b1.data(), (size_t)(2 + 2 * angleNum) * sizeof(float2));
}

// findBlackPixels + findArea for every pixel.
void btref_map_bh_area(const float* thphi, int M, int N, unsigned char* bh,
                       float* area) {
  for (int i = 0; i < N; i++)
    for (int j = 0; j < M; j++) {
      at(i, j);
      findBlackPixels((const float2*)thphi, M, N, bh);
      findArea((const float2*)thphi, M, N, area);
    }
}

// smoothAreaH then smoothAreaV; area is updated in place (areaSmooth is the
// intermediate, as in cudaPrep).
void btref_map_smooth(float* area, float* areaSmooth, const unsigned char* bh,
                      const int* gap, int M, int N) {
  for (int i = 0; i < N; i++)
    for (int j = 0; j < M; j++) {
      at(i, j);
      smoothAreaH(areaSmooth, area, bh, gap, M, N);
    }
  for (int i = 0; i < N; i++)
    for (int j = 0; j < M; j++) {
      at(i, j);
      smoothAreaV(areaSmooth, area, bh, gap, M, N);
    }
}

// Summed-area table of cudaPrep (BT/MakeImageKernel.cu:1312-1330) over a BGR8
// image (cv::imread's channel order), rows x cols; out: rows*cols float4.
void btref_map_sat(const unsigned char* bgr, int rows, int cols, float* out) {
  float pxsz = PI2 / (1.f * cols);
  // columns are independent (each is summed down its rows)
#pragma omp parallel for schedule(static)
  for (int q = 0; q < cols; q++) {
    float prev[4] = {0.f, 0.f, 0.f, 0.f};
    float phi[4] = {pxsz * q, pxsz * q, pxsz * (q + 1), pxsz * (q + 1)};
    for (int p = 0; p < rows; p++) {
      float theta[4] = {pxsz * (p + 1), pxsz * p, pxsz * p, pxsz * (p + 1)};
      float area = calcArea(theta, phi);
      const unsigned char* px = bgr + ((size_t)p * cols + q) * 3;
      prev[0] += powf(px[0], 2.2f) * area;
      prev[1] += powf(px[1], 2.2f) * area;
      prev[2] += powf(px[2], 2.2f) * area;
      prev[3] += area;
      memcpy(out + ((size_t)p * cols + q) * 4, prev, sizeof(prev));
    }
  }
}

// distortEnvironmentMap for every pixel; out is BGRA8.
void btref_map_env(const float* thphi, unsigned char* out, const unsigned char* bh,
                   int rows, int cols, int M, int N, float* sat,
                   const float* cam7, const float* area, float* view, int lr) {
  int2 imsize = {rows, cols};
  for (int i = 0; i < N; i++)
    for (int j = 0; j < M; j++) {
      at(i, j);
      distortEnvironmentMap((const float2*)thphi, (uchar4*)out, bh, imsize, M, N,
                            0.f, (float4*)sat, cam7, 0, nullptr, area,
                            (float2*)view, lr != 0);
    }
}

// distortStarMap + sumStarLight (+ makePix) on frame 0 (no trails), per
// pixel.  starLight scratch: N*M*(2step+1)^2 float3; search: N*M*searchNr.
// out: BGRA8 star image; light: N*M float3 summed star light; cells_out
// (optional): the splat scratch after distortStarMap.
void btref_map_stars(const float* thphi, const unsigned char* bh,
                     const float* stars, const int* tree, int starSize,
                     const float* cam7, const float* mag, int treeLevel, int M,
                     int N, int step, const float* view, int lr,
                     const float* area, float* light, unsigned char* out,
                     float* cells_out) {
  const int filterW = 2 * step + 1;
  const int searchNr = (int)powf(2, treeLevel / 3 * 2);
  std::vector<float3> scratch((size_t)N * M * filterW * filterW);
  std::vector<int> search((size_t)N * M * searchNr + 64 * searchNr);
  const int trailnum = 30;
  std::vector<int2> stCache((size_t)2 * starSize * trailnum, int2{-1, -1});
  std::vector<int> stnums(starSize, 0);
  std::vector<float3> trail((size_t)N * M, float3{0.f, 0.f, 0.f});
  std::vector<float2> grad((size_t)(N + 1) * (M + 1), float2{0.f, 0.f});
  for (int i = 0; i < N; i++)
    for (int j = 0; j < M; j++) {
      at(i, j);
      distortStarMap(scratch.data(), (const float2*)thphi, bh, stars, tree,
                     starSize, cam7, mag, treeLevel, M, N, step, 0.f,
                     search.data(), searchNr, stCache.data(), stnums.data(),
                     trail.data(), trailnum, grad.data(), 0, (const float2*)view,
                     lr != 0, area);
    }
  if (cells_out)
    memcpy(cells_out, scratch.data(), scratch.size() * sizeof(float3));
  for (int i = 0; i < N; i++)
    for (int j = 0; j < M; j++) {
      at(i, j);
      sumStarLight(scratch.data(), trail.data(), (float3*)light, step, M, N, filterW);
    }
  for (int i = 0; i < N; i++)
    for (int j = 0; j < M; j++) {
      at(i, j);
      makePix((float3*)light, (uchar4*)out, M, N, nullptr);
    }
}

// addDiffraction (BT/MakeImageKernel.cu:775-800) for every pixel, one after
// the other in row-major order, on the summed star light (N*M float3, with
// one more row after it: the kernel's row bound lets the pixel at row
// N - filtersize/2 write one row past the image).  The sprite is
// filtersize^2 RGB8.  Run sequentially, a pixel sees every term added before
// it, including its own sprite centre's.
void btref_map_diffraction(float* light, int M, int N, const unsigned char* sprite,
                           int filtersize) {
  for (int i = 0; i < N; i++)
    for (int j = 0; j < M; j++) {
      at(i, j);
      addDiffraction((float3*)light, M, N, (const uchar3*)sprite, filtersize);
    }
}

// addStarsAndBackground per pixel (stars, background -> output, BGRA8).
void btref_map_compose(const unsigned char* stars, const unsigned char* bg,
                       unsigned char* out, int M, int N) {
  for (int i = 0; i < N; i++)
    for (int j = 0; j < M; j++) {
      at(i, j);
      addStarsAndBackground((uchar4*)stars, (uchar4*)bg, (uchar4*)out, M);
    }
}

// ---- CPU baseline: the reference's map kernels on host threads ----


// One frame of the reference's per-pixel map timed on `nthreads` host
// threads (OpenMP over rows; 0 = all): pixInterpolation over all corners,
// findBlackPixels + findArea + smoothAreaH/V over all pixels, then
// distortEnvironmentMap and distortStarMap over every row_stride-th row.
// secs: [corners, black/area/smooth, environment rows, star rows];
// returns the rows sampled.  sat points at the summed-area table with zero
// rows readable before and after it; grid at a map grid with absent rows
// readable around it (as ref_map_frame pads them).
int btref_map_time(const float* view, int M, int N, const float* grid, int GM, int GN1,
                   int gridlvl, const float* sat, int env_rows, int env_cols,
                   const float* stars, const int* tree, int starSize, const float* mag,
                   int treeLevel, const float* cam7, int step, int lr, int row_stride,
                   int nthreads, double* secs) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
  std::vector<float2> thphi((size_t)(N + 1) * (M + 1));
  std::vector<int> gap((size_t)(N + 1) * (M + 1));
  auto t = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic, 2)
  for (int i = 0; i <= N; i++) {
    float2 border[4] = {};
    for (int j = 0; j <= M; j++) {
      at(i, j);
      pixInterpolation((const float2*)view, M, N, 1, thphi.data(), (const float2*)grid, GM,
                       GN1, 0.f, 0.f, gap.data(), gridlvl, border, 1000, 0.f);
    }
  }
  secs[0] = secs_since(t);
  std::vector<unsigned char> bh((size_t)N * M);
  std::vector<float> area((size_t)N * M), areaS((size_t)N * M);
  t = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic, 2)
  for (int i = 0; i < N; i++)
    for (int j = 0; j < M; j++) {
      at(i, j);
      findBlackPixels(thphi.data(), M, N, bh.data());
      findArea(thphi.data(), M, N, area.data());
    }
#pragma omp parallel for schedule(dynamic, 2)
  for (int i = 0; i < N; i++)
    for (int j = 0; j < M; j++) {
      at(i, j);
      smoothAreaH(areaS.data(), area.data(), bh.data(), gap.data(), M, N);
    }
#pragma omp parallel for schedule(dynamic, 2)
  for (int i = 0; i < N; i++)
    for (int j = 0; j < M; j++) {
      at(i, j);
      smoothAreaV(areaS.data(), area.data(), bh.data(), gap.data(), M, N);
    }
  secs[1] = secs_since(t);
  std::vector<int> rows;
  for (int i = row_stride / 2; i < N; i += row_stride) rows.push_back(i);
  const int nr = (int)rows.size();
  std::vector<unsigned char> out((size_t)N * M * 4);
  int2 imsize = {env_rows, env_cols};
  t = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic, 1)
  for (int r = 0; r < nr; r++)
    for (int j = 0; j < M; j++) {
      at(rows[r], j);
      distortEnvironmentMap(thphi.data(), (uchar4*)out.data(), bh.data(), imsize, M, N, 0.f,
                            (float4*)sat, cam7, 0, nullptr, area.data(), (float2*)view,
                            lr != 0);
    }
  secs[2] = secs_since(t);
  const int filterW = 2 * step + 1;
  const int searchNr = (int)powf(2, treeLevel / 3 * 2);
  const int trailnum = 30;
  Lazy<float3> scratch((size_t)N * M * filterW * filterW);
  Lazy<int> search((size_t)N * M * searchNr + (size_t)4096 * searchNr);
  Lazy<int2> stCache((size_t)2 * starSize * trailnum);
  Lazy<int> stnums((size_t)starSize);
  Lazy<float3> trail((size_t)N * M);
  Lazy<float2> grad((size_t)(N + 1) * (M + 1));
  if (!scratch.p || !search.p || !stCache.p || !stnums.p || !trail.p || !grad.p) return -1;
  // frame 0: every cache entry empty (clearArrays)
  for (size_t q = 0; q < (size_t)2 * starSize * trailnum; q++) stCache.p[q] = int2{-1, -1};
  t = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic, 1)
  for (int r = 0; r < nr; r++)
    for (int j = 0; j < M; j++) {
      at(rows[r], j);
      distortStarMap(scratch.p, thphi.data(), bh.data(), stars, tree, starSize, cam7, mag,
                     treeLevel, M, N, step, 0.f, search.p, searchNr, stCache.p, stnums.p,
                     trail.p, trailnum, grad.p, 0, (const float2*)view, lr != 0, area.data());
    }
  secs[3] = secs_since(t);
  return nr;
}

// One frame of the reference's map kernels on host threads, with the colour
// passes restricted to the listed rows (all rows, or a sample of a frame too
// large to run whole).  pixInterpolation over every corner, findBlackPixels,
// findArea and smoothAreaH/V over every pixel (thphi, gap, bh and the
// smoothed area are returned whole); then for each listed row
// distortEnvironmentMap, and distortStarMap over the rows within `step` of a
// listed row followed by sumStarLight, makePix and addStarsAndBackground on
// the listed rows.  env_rows / star_rows / img_rows: nr x M BGRA8 (any may be
// NULL; img_rows needs both passes).  area_in (may be NULL): smoothed solid
// angles the colour passes use instead of the ones computed here (area_out
// still receives these).  sat and grid are padded as for btref_map_time.  Rows of the star pass run in chunks; chunks next to each
// other never run at the same time, so searchTree's writes past a pixel's
// slots (into the next pixel's) land where only the same thread reads.
// Returns 0, or -1 if scratch memory could not be reserved.
int btref_map_frame_rows(const float* view, int M, int N, const float* grid, int GM, int GN1,
                         int gridlvl, const float* sat, int env_rows, int env_cols,
                         const float* stars, const int* tree, int starSize, const float* mag,
                         int treeLevel, const float* cam7, int step, int lr,
                         const int* rows, int nr, int nthreads, float* thphi_out,
                         int* gap_out, unsigned char* bh_out, float* area_out,
                         const float* area_in, unsigned char* env_rows_out,
                         unsigned char* star_rows_out, unsigned char* img_rows_out) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
  float2* thphi = (float2*)thphi_out;
#pragma omp parallel for schedule(dynamic, 2)
  for (int i = 0; i <= N; i++) {
    float2 border[4] = {};
    for (int j = 0; j <= M; j++) {
      at(i, j);
      pixInterpolation((const float2*)view, M, N, 1, thphi, (const float2*)grid, GM, GN1, 0.f,
                       0.f, gap_out, gridlvl, border, 1000, 0.f);
    }
  }
  std::vector<float> areaS((size_t)N * M);
#pragma omp parallel for schedule(dynamic, 2)
  for (int i = 0; i < N; i++)
    for (int j = 0; j < M; j++) {
      at(i, j);
      findBlackPixels(thphi, M, N, bh_out);
      findArea(thphi, M, N, area_out);
    }
#pragma omp parallel for schedule(dynamic, 2)
  for (int i = 0; i < N; i++)
    for (int j = 0; j < M; j++) {
      at(i, j);
      smoothAreaH(areaS.data(), area_out, bh_out, gap_out, M, N);
    }
#pragma omp parallel for schedule(dynamic, 2)
  for (int i = 0; i < N; i++)
    for (int j = 0; j < M; j++) {
      at(i, j);
      smoothAreaV(areaS.data(), area_out, bh_out, gap_out, M, N);
    }
  const float* area_use = area_in ? area_in : area_out;
  // distortEnvironmentMap writes out[ij]: a full-frame buffer reserved lazily
  Lazy<uchar4> env_img((size_t)N * M);
  if (!env_img.p) return -1;
  if (env_rows_out || img_rows_out) {
    int2 imsize = {env_rows, env_cols};
#pragma omp parallel for schedule(dynamic, 1)
    for (int r = 0; r < nr; r++)
      for (int j = 0; j < M; j++) {
        at(rows[r], j);
        distortEnvironmentMap(thphi, env_img.p, bh_out, imsize, M, N, 0.f, (float4*)sat,
                              cam7, 0, nullptr, area_use, (float2*)view, lr != 0);
      }
    if (env_rows_out)
      for (int r = 0; r < nr; r++)
        memcpy(env_rows_out + (size_t)r * M * 4, env_img.p + (size_t)rows[r] * M, (size_t)M * 4);
  }
  if (star_rows_out || img_rows_out) {
    const int filterW = 2 * step + 1;
    const int searchNr = (int)powf(2, treeLevel / 3 * 2);
    const int trailnum = 30;
    Lazy<float3> scratch((size_t)N * M * filterW * filterW);
    Lazy<int> search((size_t)N * M * searchNr + (size_t)4096 * searchNr);
    Lazy<int2> stCache((size_t)2 * starSize * trailnum);
    Lazy<int> stnums((size_t)starSize);
    Lazy<float3> trail((size_t)N * M);
    Lazy<float2> grad((size_t)(N + 1) * (M + 1));
    Lazy<float3> light((size_t)N * M);
    Lazy<uchar4> simg((size_t)N * M);
    Lazy<uchar4> comp((size_t)N * M);
    if (!scratch.p || !search.p || !stCache.p || !stnums.p || !trail.p || !grad.p || !light.p ||
        !simg.p || !comp.p)
      return -1;
    for (size_t q = 0; q < (size_t)2 * starSize * trailnum; q++) stCache.p[q] = int2{-1, -1};
    // rows the star pass needs, as runs of consecutive rows cut into chunks
    std::vector<char> need(N, 0);
    for (int r = 0; r < nr; r++)
      for (int u = -step; u <= step; u++)
        if (rows[r] + u >= 0 && rows[r] + u < N) need[rows[r] + u] = 1;
    constexpr int kChunk = 4;
    std::vector<std::pair<int, int>> chunks[2];  // [first, last) by parity in their run
    for (int i = 0; i < N;) {
      if (!need[i]) { i++; continue; }
      int k = 0;
      while (i < N && need[i]) {
        int e = i;
        while (e < N && need[e] && e - i < kChunk) e++;
        chunks[k & 1].push_back({i, e});
        k++;
        i = e;
      }
    }
    for (int ph = 0; ph < 2; ph++) {
      const auto& C = chunks[ph];
#pragma omp parallel for schedule(dynamic, 1)
      for (int c = 0; c < (int)C.size(); c++)
        for (int i = C[c].first; i < C[c].second; i++)
          for (int j = 0; j < M; j++) {
            at(i, j);
            distortStarMap(scratch.p, thphi, bh_out, stars, tree, starSize, cam7, mag, treeLevel,
                           M, N, step, 0.f, search.p, searchNr, stCache.p, stnums.p, trail.p,
                           trailnum, grad.p, 0, (const float2*)view, lr != 0, area_use);
          }
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int r = 0; r < nr; r++)
      for (int j = 0; j < M; j++) {
        at(rows[r], j);
        sumStarLight(scratch.p, trail.p, light.p, step, M, N, filterW);
        makePix(light.p, simg.p, M, N, nullptr);
        if (img_rows_out) addStarsAndBackground(simg.p, env_img.p, comp.p, M);
      }
    for (int r = 0; r < nr; r++) {
      if (star_rows_out)
        memcpy(star_rows_out + (size_t)r * M * 4, simg.p + (size_t)rows[r] * M, (size_t)M * 4);
      if (img_rows_out)
        memcpy(img_rows_out + (size_t)r * M * 4, comp.p + (size_t)rows[r] * M, (size_t)M * 4);
    }
  }
  return 0;
}

// ---- trails (addTrails / makeGradField / clearArrays) ----
// One frame's star pass as the reference's driver runs it
// (BT/MakeImageKernel.cu:1481-1497): clearArrays, makeGradField,
// distortStarMap, then sumStarLight (which adds and clears the trail buffer).
// Pixels run in ascending order, so the per-star caches list pixels in that
// order.  thphi is read one element past the corner array by makeGradField;
// the caller pads it with an absent (-2) value.
struct TrailRun {
  int M, N, step, filterW, searchNr, trailnum, starSize;
  std::vector<float3> scratch;
  std::vector<int> search;
  std::vector<int2> stCache;
  std::vector<int> stnums;
  std::vector<float3> trail;
  std::vector<float2> grad;
};

static void trail_frame(TrailRun& R, int frame, const float* thphi, const unsigned char* bh,
                        const float* stars, const int* tree, const float* cam7,
                        const float* mag, int treeLevel, const float* view, int lr,
                        const float* area, float* trail_out, float* light, int with_sum) {
  const int M = R.M, N = R.N;
  for (int q = 0; q < R.starSize; q++) {
    at(q, 0);
    clearArrays(R.stnums.data(), R.stCache.data(), frame, R.trailnum, R.starSize);
  }
  for (int i = 0; i <= N; i++)
    for (int j = 0; j <= M; j++) {
      at(i, j);
      makeGradField((const float2*)thphi, M, N, R.grad.data());
    }
  for (int i = 0; i < N; i++)
    for (int j = 0; j < M; j++) {
      at(i, j);
      distortStarMap(R.scratch.data(), (const float2*)thphi, bh, stars, tree, R.starSize, cam7,
                     mag, treeLevel, M, N, R.step, 0.f, R.search.data(), R.searchNr,
                     R.stCache.data(), R.stnums.data(), R.trail.data(), R.trailnum,
                     R.grad.data(), frame, (const float2*)view, lr != 0, area);
    }
  if (trail_out) memcpy(trail_out, R.trail.data(), R.trail.size() * sizeof(float3));
  if (!with_sum) return;
  for (int i = 0; i < N; i++)
    for (int j = 0; j < M; j++) {
      at(i, j);
      sumStarLight(R.scratch.data(), R.trail.data(), (float3*)light, R.step, M, N, R.filterW);
    }
}

static void trail_init(TrailRun& R, int M, int N, int step, int treeLevel, int starSize,
                       int trailnum) {
  R.M = M; R.N = N; R.step = step; R.filterW = 2 * step + 1;
  R.searchNr = (int)powf(2, treeLevel / 3 * 2);
  R.trailnum = trailnum;
  R.starSize = starSize;
  R.scratch.assign((size_t)N * M * R.filterW * R.filterW, float3{0.f, 0.f, 0.f});
  R.search.assign((size_t)N * M * R.searchNr + 64 * R.searchNr, 0);
  R.stCache.assign((size_t)2 * starSize * trailnum, int2{-1, -1});
  R.stnums.assign(starSize, 0);
  R.trail.assign((size_t)N * M, float3{0.f, 0.f, 0.f});
  R.grad.assign((size_t)(N + 1) * (M + 1), float2{0.f, 0.f});
}

// Frame 0 only (no line is drawn at frame 0): the star caches it leaves --
// per star up to trailnum pixels (i, j) in ascending order -- and the number
// of hits per star.  Safe to run on any input.
void btref_trail_cache(const float* thphi, const unsigned char* bh, const float* stars,
                       const int* tree, int starSize, const float* cam7, const float* mag,
                       int treeLevel, int M, int N, int step, const float* view, int lr,
                       const float* area, int trailnum, int* cache_out, int* stnums_out) {
  TrailRun R;
  trail_init(R, M, N, step, treeLevel, starSize, trailnum);
  trail_frame(R, 0, thphi, bh, stars, tree, cam7, mag, treeLevel, view, lr, area, nullptr,
              nullptr, 0);
  for (int q = 0; q < starSize; q++) {
    stnums_out[q] = R.stnums[q];
    for (int w = 0; w < trailnum; w++) {
      const int2 c = R.stCache[2 * (trailnum * q) + w];  // parity 0
      cache_out[2 * (trailnum * q + w)] = c.x;
      cache_out[2 * (trailnum * q + w) + 1] = c.y;
    }
  }
}

// Frames 0 and 1 in sequence; the trail buffer of frame 1 before
// sumStarLight consumes it, and frame 1's summed star light.  Only for inputs
// where every line walk of frame 1 ends (the reference's walk can run on
// forever); the caller checks that first.
void btref_trail_frames(const float* thphi0, const unsigned char* bh0, const float* area0,
                        const float* cam0, const float* thphi1, const unsigned char* bh1,
                        const float* area1, const float* cam1, const float* stars,
                        const int* tree, int starSize, const float* mag, int treeLevel, int M,
                        int N, int step, const float* view, int lr, int trailnum,
                        float* trail_out, float* light_out) {
  TrailRun R;
  trail_init(R, M, N, step, treeLevel, starSize, trailnum);
  std::vector<float> light((size_t)N * M * 3);
  trail_frame(R, 0, thphi0, bh0, stars, tree, cam0, mag, treeLevel, view, lr, area0, nullptr,
              light.data(), 1);
  trail_frame(R, 1, thphi1, bh1, stars, tree, cam1, mag, treeLevel, view, lr, area1, trail_out,
              light_out, 1);
}

// searchTree for one bounding box (picheck = 0, as distortStarMap calls it).
int btref_search_tree(const int* tree, const float* mn, const float* mx,
                      int treeLevel, int* nodes, int cap) {
  std::vector<int> buf(1 << 20);
  int pos = 0;
  searchTree(tree, mn, mx, treeLevel, buf.data(), 0, pos, 0);
  for (int k = 0; k < pos && k < cap; k++) nodes[k] = buf[k];
  return pos;
}

// The reference's blackbody table (tempToRGB, BT/kernel.cuh:45): 391 RGB
// triplets, 1000-40000 K in 100 K steps.
void btref_blackbody(int* out) {
  for (int k = 0; k < 1173; k++) out[k] = (int)tempToRGB[k];
}

// The reference's device helpers, one call each (for unit checks).
int btref_star_in_polygon(const float* t, const float* p, float st, float sp, int sgn) {
  return starInPolygon(t, p, st, sp, sgn) ? 1 : 0;
}
void btref_interpolate(const float* t, const float* p, float* st, float* sp, int sgn) {
  interpolate(t[0], t[1], t[2], t[3], p[0], p[1], p[2], p[3], *st, *sp, sgn, 0, 0);
}
float btref_calc_area(const float* t4, const float* p4) {
  float t[4], p[4];
  memcpy(t, t4, sizeof(t));
  memcpy(p, p4, sizeof(p));
  return calcArea(t, p);
}
float btref_redshift(float theta, float phi, const float* cam7) {
  return redshift(theta, phi, cam7);
}
void btref_rgb_hsp(float r, float g, float b, float* hsp) {
  RGBtoHSP(r, g, b, hsp[0], hsp[1], hsp[2]);
}
void btref_hsp_rgb(float h, float s, float p, float* rgb) {
  HSPtoRGB(h, s, p, rgb[0], rgb[1], rgb[2]);
}

}  // extern "C"
