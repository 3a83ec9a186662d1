// stars.cu -- star splatting on the device (annemiekie/BlackTracer
// BT/MakeImageKernel.cu: searchTree :27-96, distortStarMap :206-326,
// sumStarLight :753-773, addDiffraction :775-800, makePix :802-835,
// addStarsAndBackground :837-853; helpers in BT/kernel.cuh: interpolate
// :112-200, starInPolygon :245-266, gaussian :335-338).
//
// Structure on the B200:
//   k_star_cells  one thread per pixel: corners, kd-tree search of the
//                 pixel's bounding box, point-in-quad, in-pixel bisection,
//                 magnitude/colour, splat into the pixel's own
//                 (2s+1)^2 cells.  Nodes are processed as the search emits
//                 them (no per-pixel node list in memory).  A pixel writes
//                 its cells only when it holds a star and flags itself, so
//                 a sparse sky costs no scratch traffic.
//   k_star_gather gathers the mirrored cells of the flagged neighbours in
//                 the reference's (u, v) order (bit-identical sums), then
//                 makePix and the composite with the environment, fused.
//   k_diff_*      diffraction: bright pixels are collected, then their PSF
//                 is scattered with atomics into a copy of the star light.
//                 The reference's kernel reads a pixel while other threads
//                 add into it (a data race, :781-797); here every read
//                 happens before any add (snapshot semantics).
// Trails (addTrails, :98-174) are a multi-frame effect and are not part of
// a single frame: on the first frame they leave the image unchanged.
#include <cstring>
#include <new>
#include <vector>

#include "bt_internal.h"
#include "map_internal.h"
#include "stars_pixel.cuh"

namespace bt {

}  // namespace bt

struct bt_stars {
  bt::StarSet s;
  float* pos;
  float* mag;
  int* tree;
  uchar3* psf;
};

namespace bt {

const StarSet* stars_internal(const bt_stars* s) { return &s->s; }

constexpr int TX = 32, TY = 8;
static dim3 grid2(int w, int h) {
  return dim3((unsigned)((w + TX - 1) / TX), (unsigned)((h + TY - 1) / TY));
}

// Star tests a pixel may spend in k_star_cells before it is handed to the
// warp-cooperative kernel.  Pixels next to the shadow project onto slivers
// whose bounding boxes cover most of the sky (hundreds of thousands of
// candidate stars); one such lane would stall its warp for the whole frame.
constexpr long kStarBudget = 2048;

// distortStarMap without trails: splat cells + flag per pixel; pixels over
// the budget are queued for k_star_heavy.
__global__ void k_star_cells(const float2* __restrict__ thphi,
                             const uint8_t* __restrict__ bh, StarSet S, Cam7 cam,
                             int M, int N, int step, const float2* __restrict__ view,
                             int lr, const float* __restrict__ area,
                             float3* __restrict__ cells, uint8_t* __restrict__ flag,
                             uint32_t* __restrict__ heavy, uint32_t* nheavy) {
  const int j = blockIdx.x * TX + threadIdx.x;
  const int i = blockIdx.y * TY + threadIdx.y;
  if (i >= N || j >= M) return;
  const size_t ij = (size_t)i * M + j;
  const int fw = 2 * step + 1;
  const int r = pixel_stars(thphi, bh, S, cam.v, M, N, step, view, lr, area, i, j,
                            cells + ij * fw * fw, kStarBudget);
  flag[ij] = r == 1 ? 1 : 0;
  if (r == 2) heavy[atomicAdd(nheavy, 1u)] = (uint32_t)ij;
}

constexpr int kHeavyThreads = 256;  // one block per deferred pixel
constexpr int kHeavyNodes = 2048;   // nodes per search pass (shared memory)
constexpr int kMaxCells = 25;       // (2s+1)^2 for step <= 2 in registers

// The deferred pixels, one block each.  Thread 0 walks the kd-tree (in
// passes of kHeavyNodes emitted nodes) into shared memory with a prefix sum
// of the nodes' star counts; then all threads sweep the concatenated star
// ranges, each accumulating its hits into its own cell registers, and a
// block reduction adds the partial cells.  Sums are reassociated (not in the
// reference's star order), which changes them only by float rounding.
__global__ void __launch_bounds__(kHeavyThreads)
k_star_heavy(const float2* __restrict__ thphi, const uint8_t* __restrict__ bh,
             StarSet S, Cam7 cam, int M, int N, int step,
             const float2* __restrict__ view, int lr, const float* __restrict__ area,
             float3* __restrict__ cells, uint8_t* __restrict__ flag,
             const uint32_t* __restrict__ heavy, const uint32_t* nheavy) {
  __shared__ int sh_node[kHeavyNodes];
  __shared__ int sh_end[kHeavyNodes];  // inclusive prefix of star counts
  __shared__ int sh_count, sh_more, sh_total;
  __shared__ float sh_red[kHeavyThreads / 32][kMaxCells * 3];
  __shared__ int sh_any;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const uint32_t n = *nheavy;
  const int fw = 2 * step + 1, fw2 = fw * fw;
  for (uint32_t item = blockIdx.x; item < n; item += gridDim.x) {
    const uint32_t ij = heavy[item];
    const int i = ij / M, j = ij % M;
    PixelStars P;
    float mn[2], mx[2];
    pixel_setup(thphi, bh, cam.v, M, step, view, lr, area, i, j, P, mn, mx);
    float3 acc[kMaxCells];
#pragma unroll
    for (int c = 0; c < kMaxCells; c++) acc[c] = make_float3(0.f, 0.f, 0.f);
    int any = 0;
    int skip = 0;
    for (;;) {
      if (tid == 0) {
        int emitted = 0, count = 0, more = 0, total = 0;
        tree_search(S, mn, mx, [&](int node) {
          if (emitted >= skip + kHeavyNodes) {
            more = 1;
            return false;
          }
          if (emitted >= skip) {
            int startN = 0;
            if (node != 0 && ((node + 1) & node) != 0) startN = S.tree[node - 1];
            total += S.tree[node] - startN;
            sh_node[count] = node;
            sh_end[count] = total;
            count++;
          }
          emitted++;
          return true;
        });
        sh_count = count;
        sh_more = more;
        sh_total = total;
      }
      __syncthreads();
      const int count = sh_count, total = sh_total;
      for (int k = tid; k < total; k += kHeavyThreads) {
        // node holding the k-th candidate: first end > k
        int lo = 0, hi = count - 1;
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (sh_end[mid] > k) hi = mid;
          else lo = mid + 1;
        }
        const int node = sh_node[lo];
        int startN = 0;
        if (node != 0 && ((node + 1) & node) != 0) startN = S.tree[node - 1];
        const int q = startN + (k - (lo ? sh_end[lo - 1] : 0));
        float st, sp;
        if (!star_test(P, S, q, st, sp)) continue;
        any = 1;
        const StarHit h = star_hit(P, S, q, st, sp);
#pragma unroll
        for (int c = 0; c < kMaxCells; c++) {
          if (c >= fw2) break;
          float3 l;
          if (cell_light(P, h, c / fw, c % fw, l)) {
            acc[c].x += l.x;
            acc[c].y += l.y;
            acc[c].z += l.z;
          }
        }
      }
      const int more = sh_more;
      __syncthreads();
      if (!more) break;
      skip += kHeavyNodes;
    }
    // block reduction of the cells
    any = __syncthreads_or(any);
    if (any) {
#pragma unroll
      for (int c = 0; c < kMaxCells; c++) {
        if (c >= fw2) break;
        float x = acc[c].x, y = acc[c].y, z = acc[c].z;
        for (int o = 16; o > 0; o >>= 1) {
          x += __shfl_xor_sync(0xffffffffu, x, o);
          y += __shfl_xor_sync(0xffffffffu, y, o);
          z += __shfl_xor_sync(0xffffffffu, z, o);
        }
        if (lane == 0) {
          sh_red[w][3 * c] = x;
          sh_red[w][3 * c + 1] = y;
          sh_red[w][3 * c + 2] = z;
        }
      }
      __syncthreads();
      if (tid < 3 * fw2) {
        float v = 0.f;
        for (int ww = 0; ww < kHeavyThreads / 32; ww++) v += sh_red[ww][tid];
        ((float*)(cells + (size_t)ij * fw2))[tid] = v;
      }
    }
    if (tid == 0) flag[ij] = any ? 1 : 0;
    __syncthreads();
  }
}

// sumStarLight (+ makePix + addStarsAndBackground when no diffraction).
template <bool kCompose>
__global__ void k_star_gather(const float3* __restrict__ cells,
                              const uint8_t* __restrict__ flag, int M, int N,
                              int step, float* __restrict__ light,
                              const uchar4* __restrict__ bg,
                              uchar4* __restrict__ out, int map) {
  const int j = blockIdx.x * TX + threadIdx.x;
  const int i = blockIdx.y * TY + threadIdx.y;
  if (i >= N || j >= M) return;
  const int fw = 2 * step + 1;
  const int fw2 = fw * fw;
  float3 b = make_float3(0.f, 0.f, 0.f);
  const int start = max(0, step - i);
  const int stop = min(2 * step, step + N - i - 1);
  const float factor = 20.f;
  for (int u = start; u <= stop; u++)
    for (int v = 0; v <= 2 * step; v++) {
      const size_t nb = (size_t)(i + u - step) * M + ((j + v - step + M) % M);
      if (!flag[nb]) continue;
      const float3 c = cells[fw2 * nb + fw2 - (fw * u + v + 1)];
      b.x += factor * c.x;
      b.y += factor * c.y;
      b.z += factor * c.z;
    }
  const size_t ij = (size_t)i * M + j;
  if (!kCompose) {
    light[3 * ij] = b.x;
    light[3 * ij + 1] = b.y;
    light[3 * ij + 2] = b.z;
    return;
  }
  // makePix (BT/MakeImageKernel.cu:802-835)
  float3 rgb = make_float3(sqrtf(b.x), sqrtf(b.y), sqrtf(b.z));
  const float mxc = fmaxf(fmaxf(rgb.x, rgb.y), rgb.z);
  if (mxc > 255.f) {
    float3 hsp;
    rgb_to_hsp(rgb.x / 255.f, rgb.y / 255.f, rgb.z / 255.f, hsp.x, hsp.y, hsp.z);
    hsp.z = 1.0f;
    hsp_to_rgb(hsp.x, hsp.y, hsp.z, rgb.x, rgb.y, rgb.z);
    rgb.x *= 255; rgb.y *= 255; rgb.z *= 255;
  }
  uchar4 st = make_uchar4((unsigned char)min(255, (int)(rgb.z)),
                          (unsigned char)min(255, (int)(rgb.y)),
                          (unsigned char)min(255, (int)(rgb.x)), 255);
  if (map) {
    // addStarsAndBackground (BT/MakeImageKernel.cu:837-853), p = 1
    const uchar4 g = bg[ij];
    const float sx = (float)st.x * st.x, sy = (float)st.y * st.y, sz = (float)st.z * st.z;
    const float gx = (float)g.x * g.x, gy = (float)g.y * g.y, gz = (float)g.z * g.z;
    const float p = 1.f;
    const float ox = sqrtf(p * sx + (2.f - p) * gx), oy = sqrtf(p * sy + (2.f - p) * gy),
                oz = sqrtf(p * sz + (2.f - p) * gz);
    st = make_uchar4((unsigned char)min((int)ox, 255), (unsigned char)min((int)oy, 255),
                     (unsigned char)min((int)oz, 255), 255);
  }
  out[ij] = st;
}

// Diffraction, pass 1: pixels brighter than 65025 in any channel.
__global__ void k_diff_mark(const float* __restrict__ light, int n,
                            uint32_t* __restrict__ list, uint32_t* count) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const float m = fmaxf(fmaxf(light[3 * q], light[3 * q + 1]), light[3 * q + 2]);
  if (m > 65025.f) list[atomicAdd(count, 1u)] = q;
}

// Diffraction, pass 2 (addDiffraction, BT/MakeImageKernel.cu:775-800): one
// block per bright pixel scatters the sprite, reading the snapshot `light`
// and adding into `acc`.
__global__ void k_diff_scatter(const float* __restrict__ light, float* acc,
                               const uint32_t* __restrict__ list,
                               const uint32_t* count, int M, int N,
                               const uchar3* __restrict__ psf, int fs) {
  const uint32_t n = *count;
  for (uint32_t b = blockIdx.x; b < n; b += gridDim.x) {
    const uint32_t ij = list[b];
    const int i = ij / M, j = ij % M;
    const float lx = light[3 * ij], ly = light[3 * ij + 1], lz = light[3 * ij + 2];
    const float mxv = fmaxf(fmaxf(lx, ly), lz);
    const int fh = fs / 2;
    int startx = 0, endx = fs;
    if (i < fh) startx = fh - i;
    if (i > (N - fh)) endx = N - i + fh;
    const float div = 10000 * powf(mxv, 0.6);
    for (int c = threadIdx.x; c < (endx - startx) * fs; c += blockDim.x) {
      const int q = startx + c / fs, p = c % fs;
      const int ti = i - fh + q;
      if (ti < 0 || ti >= N) continue;
      const uchar3 d = psf[q * fs + p];
      const float dx = lx / div * (float)d.x, dy = ly / div * (float)d.y,
                  dz = lz / div * (float)d.z;
      const size_t t = (size_t)ti * M + (j - fh + p + M) % M;
      atomicAdd(&acc[3 * t], fminf(65025.f, dx * dx));
      atomicAdd(&acc[3 * t + 1], fminf(65025.f, dy * dy));
      atomicAdd(&acc[3 * t + 2], fminf(65025.f, dz * dz));
    }
  }
}

// makePix + composite from a light buffer (after diffraction).
__global__ void k_makepix(const float* __restrict__ light, int M, int N,
                          const uchar4* __restrict__ bg, uchar4* __restrict__ out,
                          int map) {
  const int j = blockIdx.x * TX + threadIdx.x;
  const int i = blockIdx.y * TY + threadIdx.y;
  if (i >= N || j >= M) return;
  const size_t ij = (size_t)i * M + j;
  float3 rgb = make_float3(sqrtf(light[3 * ij]), sqrtf(light[3 * ij + 1]),
                           sqrtf(light[3 * ij + 2]));
  const float mxc = fmaxf(fmaxf(rgb.x, rgb.y), rgb.z);
  if (mxc > 255.f) {
    float3 hsp;
    rgb_to_hsp(rgb.x / 255.f, rgb.y / 255.f, rgb.z / 255.f, hsp.x, hsp.y, hsp.z);
    hsp.z = 1.0f;
    hsp_to_rgb(hsp.x, hsp.y, hsp.z, rgb.x, rgb.y, rgb.z);
    rgb.x *= 255; rgb.y *= 255; rgb.z *= 255;
  }
  uchar4 st = make_uchar4((unsigned char)min(255, (int)(rgb.z)),
                          (unsigned char)min(255, (int)(rgb.y)),
                          (unsigned char)min(255, (int)(rgb.x)), 255);
  if (map) {
    const uchar4 g = bg[ij];
    const float p = 1.f;
    const float ox = sqrtf(p * ((float)st.x * st.x) + (2.f - p) * ((float)g.x * g.x));
    const float oy = sqrtf(p * ((float)st.y * st.y) + (2.f - p) * ((float)g.y * g.y));
    const float oz = sqrtf(p * ((float)st.z * st.z) + (2.f - p) * ((float)g.z * g.z));
    st = make_uchar4((unsigned char)min((int)ox, 255), (unsigned char)min((int)oy, 255),
                     (unsigned char)min((int)oz, 255), 255);
  }
  out[ij] = st;
}

int map_run_stars(MapScratch& Sc, const MapFrame& F, cudaStream_t s) {
  const int M = Sc.M, N = Sc.N;
  const int fw = 2 * F.step + 1;
  const size_t np = (size_t)M * N;
  if (!Sc.cells || Sc.cells_fw < fw) {
    if (Sc.cells) cudaFree(Sc.cells);
    Sc.cells = nullptr;
    cudaError_t e = cudaMalloc((void**)&Sc.cells, np * fw * fw * sizeof(float3));
    if (e != cudaSuccess) {
      set_error("star cell scratch allocation failed: %s", cudaGetErrorString(e));
      return BT_ERR_NOMEM;
    }
    Sc.cells_fw = fw;
  }
  if (F.step > 2) {
    set_error("star splat step > 2 is not supported");
    return BT_ERR_ARG;
  }
  BT_CUDA_TRY(cudaMemsetAsync(Sc.heavy_count, 0, sizeof(uint32_t), s));
  k_star_cells<<<grid2(M, N), dim3(TX, TY), 0, s>>>(
      Sc.thphi, Sc.bh, *F.stars, F.cam, M, N, F.step, F.view, F.lr, Sc.area,
      Sc.cells, Sc.flag, Sc.heavy_list, Sc.heavy_count);
  k_star_heavy<<<sm_count() * 4, kHeavyThreads, 0, s>>>(
      Sc.thphi, Sc.bh, *F.stars, F.cam, M, N, F.step, F.view, F.lr, Sc.area,
      Sc.cells, Sc.flag, Sc.heavy_list, Sc.heavy_count);
  BT_CUDA_TRY(cudaGetLastError());
  const bool diff = F.diffraction && F.stars->psf && F.stars->psf_size > 0;
  if (!diff) {
    k_star_gather<true><<<grid2(M, N), dim3(TX, TY), 0, s>>>(
        Sc.cells, Sc.flag, M, N, F.step, Sc.light, (const uchar4*)F.out_bg,
        (uchar4*)F.out, F.map);
    BT_CUDA_TRY(cudaGetLastError());
    return BT_OK;
  }
  k_star_gather<false><<<grid2(M, N), dim3(TX, TY), 0, s>>>(
      Sc.cells, Sc.flag, M, N, F.step, Sc.light, nullptr, nullptr, F.map);
  BT_CUDA_TRY(cudaMemcpyAsync(Sc.light2, Sc.light, np * 3 * sizeof(float),
                              cudaMemcpyDeviceToDevice, s));
  BT_CUDA_TRY(cudaMemsetAsync(Sc.diff_count, 0, sizeof(uint32_t), s));
  k_diff_mark<<<(unsigned)((np + 255) / 256), 256, 0, s>>>(Sc.light, (int)np,
                                                          Sc.diff_list, Sc.diff_count);
  k_diff_scatter<<<sm_count() * 8, 256, 0, s>>>(Sc.light, Sc.light2, Sc.diff_list,
                                                Sc.diff_count, M, N, F.stars->psf,
                                                F.stars->psf_size);
  k_makepix<<<grid2(M, N), dim3(TX, TY), 0, s>>>(Sc.light2, M, N,
                                                 (const uchar4*)F.out_bg,
                                                 (uchar4*)F.out, F.map);
  BT_CUDA_TRY(cudaGetLastError());
  return BT_OK;
}

}  // namespace bt

using namespace bt;

namespace {

// StarProcessor::makeTree (BT/StarProcessor.h:172-212): recursive halving
// of (theta, phi) space, alternating axes, to depth treeLevel; leaves hold
// the stars, every node the cumulative count up to its end.
struct TreeBuilder {
  int L;
  std::vector<int>& tree;
  std::vector<float>& pos;
  std::vector<float>& mag;
  void make(std::vector<int>& idx, const float* th, const float* ph,
            const float* m, const float* bv, int level, float thphi[2],
            float size[2], int writePos) {
    const int stsize = (int)idx.size();
    int searchPos = 0;
    if (writePos != 0 && ((writePos + 1) & writePos) != 0)
      searchPos = tree[writePos - 1];
    tree[writePos] = searchPos + stsize;
    if (level == L) {
      for (int k = 0; k < stsize; k++) {
        const int s = idx[k];
        pos[(size_t)(k + searchPos) * 2] = th[s];
        pos[(size_t)(k + searchPos) * 2 + 1] = ph[s];
        mag[(size_t)(k + searchPos) * 2] = m[s];
        mag[(size_t)(k + searchPos) * 2 + 1] = bv[s];
      }
      return;
    }
    level++;
    const int n = level % 2;
    size[n] = size[n] * .5;
    std::vector<int> lu, rd;
    const float check = thphi[n] + size[n];
    for (int k = 0; k < stsize; k++) {
      const int s = idx[k];
      const float v = n == 0 ? th[s] : ph[s];
      if (v < check) lu.push_back(s);
      else rd.push_back(s);
    }
    std::vector<int>().swap(idx);
    float sizeNew[2] = {size[0], size[1]};
    float thphiNew[2] = {thphi[0], thphi[1]};
    make(lu, th, ph, m, bv, level, thphiNew, sizeNew, writePos * 2 + 1);
    float thphiNew2[2] = {thphi[0], thphi[1]};
    float sizeNew2[2] = {size[0], size[1]};
    thphiNew2[n] += size[n];
    make(rd, th, ph, m, bv, level, thphiNew2, sizeNew2, writePos * 2 + 2);
  }
};

}  // namespace

extern "C" {

int bt_stars_tree_size(int treeLevel) { return (1 << (treeLevel + 1)) - 1; }

int bt_stars_build_tree(const float* theta, const float* phi, const float* mag,
                        const float* bv, int n, int treeLevel, float magnitude_cut,
                        float* star_pos, float* star_mag, int* tree, int* n_kept) {
  clear_error();
  BT_ARG_CHECK(n >= 0 && treeLevel >= 1 && treeLevel <= 24, "invalid star set");
  BT_ARG_CHECK(star_pos && star_mag && tree && n_kept, "NULL output");
  BT_ARG_CHECK(n == 0 || (theta && phi && mag && bv), "NULL input");
  // StarProcessor ctor (BT/StarProcessor.h:34-64): stars fainter than the
  // cut are set aside; the rest go into the tree.
  std::vector<int> idx;
  idx.reserve(n);
  for (int k = 0; k < n; k++)
    if (!(mag[k] > magnitude_cut)) idx.push_back(k);
  const int kept = (int)idx.size();
  std::vector<int> t((size_t)bt_stars_tree_size(treeLevel));
  std::vector<float> p((size_t)kept * 2), m((size_t)kept * 2);
  TreeBuilder B{treeLevel, t, p, m};
  float thphi[2] = {0, 0};
  float size[2] = {(float)kPi, (float)kPi2};
  B.make(idx, theta, phi, mag, bv, 0, thphi, size, 0);
  std::memcpy(tree, t.data(), t.size() * sizeof(int));
  std::memcpy(star_pos, p.data(), p.size() * sizeof(float));
  std::memcpy(star_mag, m.data(), m.size() * sizeof(float));
  *n_kept = kept;
  return BT_OK;
}

int bt_stars_create(const float* star_pos, const float* star_mag, int n,
                    const int* tree, int treeLevel, const uint8_t* psf_rgb,
                    int psf_size, bt_stars** out, void* stream) {
  clear_error();
  BT_ARG_CHECK(out && tree && (n == 0 || (star_pos && star_mag)), "NULL pointer");
  BT_ARG_CHECK(treeLevel >= 1 && treeLevel <= 24 && n >= 0, "invalid star set");
  BT_ARG_CHECK(psf_size >= 0 && (psf_size == 0 || psf_rgb), "invalid sprite");
  *out = nullptr;
  bt_stars* st = new (std::nothrow) bt_stars;
  if (!st) return BT_ERR_NOMEM;
  std::memset(st, 0, sizeof(*st));
  const size_t tsize = (size_t)bt_stars_tree_size(treeLevel);
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaMalloc((void**)&st->pos, (size_t)2 * n * sizeof(float) + 16);
  if (e == cudaSuccess) e = cudaMalloc((void**)&st->mag, (size_t)2 * n * sizeof(float) + 16);
  if (e == cudaSuccess) e = cudaMalloc((void**)&st->tree, tsize * sizeof(int));
  if (e == cudaSuccess && psf_size)
    e = cudaMalloc((void**)&st->psf, (size_t)psf_size * psf_size * 3);
  if (e == cudaSuccess && n)
    e = cudaMemcpyAsync(st->pos, star_pos, (size_t)2 * n * sizeof(float),
                        cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && n)
    e = cudaMemcpyAsync(st->mag, star_mag, (size_t)2 * n * sizeof(float),
                        cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(st->tree, tree, tsize * sizeof(int), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && psf_size)
    e = cudaMemcpyAsync(st->psf, psf_rgb, (size_t)psf_size * psf_size * 3,
                        cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    cudaFree(st->pos); cudaFree(st->mag); cudaFree(st->tree); cudaFree(st->psf);
    delete st;
    set_error("star set upload failed: %s", cudaGetErrorString(e));
    return BT_ERR_CUDA;
  }
  st->s.n = n;
  st->s.treeLevel = treeLevel;
  st->s.pos = st->pos;
  st->s.mag = st->mag;
  st->s.tree = st->tree;
  st->s.psf = st->psf;
  st->s.psf_size = psf_size;
  *out = st;
  return BT_OK;
}

void bt_stars_destroy(bt_stars* st) {
  if (!st) return;
  cudaFree(st->pos);
  cudaFree(st->mag);
  cudaFree(st->tree);
  if (st->psf) cudaFree(st->psf);
  delete st;
}

}  // extern "C"
