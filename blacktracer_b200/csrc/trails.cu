// trails.cu -- star trails between consecutive frames.
//
// The reference draws, inside distortStarMap, a short fading line from where
// a star was seen in the previous frame to where it is now (addTrails,
// BT/MakeImageKernel.cu:98-174), guided by the gradient of the celestial
// theta over the camera sky (makeGradField :517-537); a per-star cache of up
// to trailnum = 30 pixels per frame, double-buffered by frame parity,
// remembers where each star was (clearArrays :618-629).  sumStarLight adds
// the trail buffer to the star light (:767-771).
//
// Here the same effect runs as a separate pass of the frame:
//   1. clear this frame's cache counts (both parities at frame 0) and the
//      trail buffer; makeGradField on this frame's corners;
//   2. k_trail_hits: every (pixel, star) pair that passes the quad test in a
//      pixel whose kd-tree search holds fewer than starSize/100 stars (the
//      reference's condition) appends a hit (key star << 32 | pixel);
//   3. the hits are sorted by key (CUB radix sort), which defines the order
//      the reference leaves to its atomics: a star's cache lists its pixels
//      in ascending pixel order;
//   4. k_trail_store fills this frame's cache from the sorted hits;
//      k_trail_draw runs addTrails's choice of the previous position for
//      every hit and walks the line.
// Differences from the reference, each deliberate: the line walk stops where
// it would leave the box spanned by its two end points (the reference's walk
// can step past its target and then never ends, writing outside the image:
// for a purely vertical displacement it walks away at once); pixels two lines
// cross keep the brighter value per channel (the reference keeps whichever
// thread wrote last); the gradient starts at zero (the reference's buffer is
// uninitialised device memory).
#include <algorithm>
#include <cstring>
#include <new>

#include <cub/cub.cuh>

#include "map_internal.h"
#include "stars_pixel.cuh"

using bt::clear_error;
using bt::set_error;

struct bt_trails {
  int n_stars, M, N, trailnum;
  size_t cap;
  int2* cache;        // [2][n_stars][trailnum]
  int32_t* count;     // [2][n_stars]
  float2* grad;       // (N+1)*(M+1)
  float* trail;       // N*M*3
  uint64_t* keys[2];  // hits, then sorted
  uint32_t* vals[2];  // hit index, then sorted
  float* part;        // per hit: magnitude + redshift term
  float* frac;        // per hit: lensing fraction of its pixel
  int32_t* bb;        // per hit: blackbody entry
  uint32_t* ctr;      // [0] hits appended, [1] walks cut
  uint32_t* ctr_host; // pinned
  void* tmp;
  size_t tmp_bytes;
  int64_t frame;
};

namespace {

using namespace bt;

constexpr int TX = 32, TY = 8;

// makeGradField (BT/MakeImageKernel.cu:517-537) at corner (i, j).  The
// reference's right neighbour of the last column is index i*M1 + M1, the first
// corner of the next row; past the last row that index lies outside the
// corner array and reads as absent here.
__global__ void k_trail_grad(const float2* __restrict__ thphi, int M, int N,
                             float2* __restrict__ grad) {
  const int j = blockIdx.x * TX + threadIdx.x;
  const int i = blockIdx.y * TY + threadIdx.y;
  const int M1 = M + 1, N1 = N + 1;
  if (i >= N1 || j >= M1) return;
  const float up = thphi[min(N, i + 1) * M1 + j].x;
  const float down = thphi[max(0, i - 1) * M1 + j].x;
  const float left = thphi[i * M1 + max(0, j - 1)].x;
  const long r = (long)i * M1 + min(M1, j + 1);
  const float right = r < (long)N1 * M1 ? thphi[r].x : -2.f;
  const float mid = thphi[i * M1 + j].x;
  if (mid > 0) {
    float xdir = 0;
    if (up > 0 && down > 0) xdir = .5f * (up - mid) - .5f * (down - mid);
    float ydir = 0;
    if (left > 0 && right > 0) ydir = .5f * (right - mid) - .5f * (left - mid);
    grad[i * M1 + j] = make_float2(-ydir, xdir);
  }
}

// Step 2: the (pixel, star) hits of distortStarMap's quad test in pixels
// whose search holds fewer than starSize / 100 stars.
__global__ void __launch_bounds__(TX * TY)
k_trail_hits(const float2* __restrict__ thphi, const uint8_t* __restrict__ bh, StarSet S,
             Cam7 cam, int M, int N, int step, const float2* __restrict__ view, int lr,
             const float* __restrict__ area, uint64_t* __restrict__ keys,
             uint32_t* __restrict__ vals, float* __restrict__ part, float* __restrict__ frac,
             int32_t* __restrict__ bbi, uint32_t* ctr, size_t cap) {
  const int j = blockIdx.x * TX + threadIdx.x;
  const int i = blockIdx.y * TY + threadIdx.y;
  if (i >= N || j >= M) return;
  PixelStars P;
  float mn[2], mx[2];
  if (!pixel_setup(thphi, bh, cam.v, M, step, view, lr, area, i, j, P, mn, mx)) return;
  P.budget = 0x7fffffffffffL;
  // starsToCheck: the stars of every node the search emits
  long to_check = 0;
  tree_search(S, mn, mx, [&](int node) {
    int a0, a1;
    node_range(S, node, a0, a1);
    to_check += a1 - a0;
    return true;
  });
  if (to_check == 0 || !(to_check < S.n / 100)) return;
  const uint64_t ij = (uint64_t)i * M + j;
  tree_search(S, mn, mx, [&](int node) {
    walk_leaves(P, S, node, node_level(node), [&](int leaf) {
      int a0, a1;
      node_range(S, leaf, a0, a1);
      for (int q = a0; q < a1; q++) {
        float st, sp;
        if (!star_test(P, S, q, st, sp)) continue;
        const uint32_t k = atomicAdd(ctr, 1u);
        if (k >= cap) continue;
        keys[k] = ((uint64_t)q << 32) | ij;
        vals[k] = k;
        part[k] = S.mag[2 * q] + P.red;
        frac[k] = P.frac;
        bbi[k] = blackbody_index(S.mag[2 * q + 1], P.redshft, S.bb_n);
      }
      return true;
    });
    return true;
  });
}

// First index of the sorted hits whose key is >= v.
__device__ __forceinline__ size_t lower_bound(const uint64_t* k, size_t n, uint64_t v) {
  size_t lo = 0, hi = n;
  while (lo < hi) {
    const size_t mid = (lo + hi) >> 1;
    if (k[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Step 4a: this frame's cache from the sorted hits (the stores of addTrails
// :102-104, in ascending pixel order per star).
__global__ void k_trail_store(const uint64_t* __restrict__ keys, size_t cap, int M,
                              int trailnum, int2* __restrict__ cache,
                              int32_t* __restrict__ count) {
  const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (k >= cap) return;
  const uint64_t key = keys[k];
  if (key == ~0ull) return;
  const uint64_t q = key >> 32;
  const uint32_t ij = (uint32_t)key;
  const size_t start = (k == 0 || (keys[k - 1] >> 32) != q) ? k : lower_bound(keys, k, q << 32);
  const size_t rank = k - start;
  if (rank < (size_t)trailnum)
    cache[q * trailnum + rank] = make_int2((int)(ij / (uint32_t)M), (int)(ij % (uint32_t)M));
  if (rank == 0) {
    const size_t end = lower_bound(keys, cap, (q + 1) << 32);
    count[q] = (int32_t)min(end - start, (size_t)trailnum);
  }
}

__device__ __forceinline__ void max_store(float* p, float v) {
  // non-negative floats order like their bit patterns
  atomicMax((unsigned int*)p, __float_as_uint(fmaxf(v, 0.f)));
}

// Step 4b: addTrails (BT/MakeImageKernel.cu:106-172) for every hit.
__global__ void k_trail_draw(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                             size_t cap, const float* __restrict__ part,
                             const float* __restrict__ frac, const int32_t* __restrict__ bbi,
                             const float4* __restrict__ bb_hsp, int M, int N, int trailnum,
                             const int2* __restrict__ prev_cache,
                             const int32_t* __restrict__ prev_count,
                             const float2* __restrict__ grad, float* __restrict__ trail,
                             uint32_t* cut) {
  const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (k >= cap) return;
  const uint64_t key = keys[k];
  if (key == ~0ull) return;
  const uint64_t q = key >> 32;
  const uint32_t ijp = (uint32_t)key;
  const int i = (int)(ijp / (uint32_t)M), j = (int)(ijp % (uint32_t)M);
  const int M1 = M + 1;
  float traildist = M;
  float angle = kPi2F;
  int2 prev = make_int2(0, 0);
  bool line = false;
  const int np = prev_count[q];
  for (int w = 0; w < np; w++) {
    const int2 pr = prev_cache[q * trailnum + w];
    const int dx = (pr.x - i);
    const int dy = (pr.y - j);
    const int dxx = dx * dx;
    const int dyy = dy * dy;
    if (dxx <= 1 && dyy <= 1) {
      line = false;
      break;
    }
    const float2 gr = grad[pr.x * M1 + pr.y];
    const float dist = sqrtf(dxx + dyy);
    if (dist > M / 25.f) continue;
    const float div = (dist * sqrtf(gr.x * gr.x + gr.y * gr.y));
    const float a1 = acosf((1.f * dx * gr.x + 1.f * dy * gr.y) / div);
    const float a2 = acosf((1.f * dx * -gr.x + 1.f * dy * -gr.y) / div);
    const float a = fminf(a1, a2);
    if (a > angle || a > kPiF * .25f) continue;
    else if (a < angle) {
      angle = a;
      traildist = dist;
      prev = pr;
      line = true;
    }
  }
  if (!line) return;
  const uint32_t v = vals[k];
  const float4 hsp = bb_hsp[bbi[v]];
  const float pt = part[v], fr = frac[v];
  const int deltax = i - prev.x;
  const int deltay = j - prev.y;
  const int sgnDeltaX = deltax < 0 ? -1 : 1;
  const int sgnDeltaY = deltay < 0 ? -1 : 1;
  const float deltaerr = deltay == 0.f ? fabsf(deltax) : fabsf(deltax / (1.f * deltay));
  const int xlo = min(prev.x, i), xhi = max(prev.x, i);
  const int ylo = min(prev.y, j), yhi = max(prev.y, j);
  float error = 0.f;
  int y = prev.y;
  int x = prev.x;
  while (y != j || x != i) {
    if (error < 1.f) {
      y += sgnDeltaY;
      error += deltaerr;
    }
    if (error >= 0.5f) {
      x += sgnDeltaX;
      error -= 1.f;
    }
    if (x < xlo || x > xhi || y < ylo || y > yhi) {  // past the target: stop
      atomicAdd(cut, 1u);
      break;
    }
    const float dist = dist_sq(x, i, y, j);
    const float appMag = pt - 2.5f * log10f(fr);
    float brightness = 100 * exp10f(-.4f * appMag);
    brightness *= ((traildist - sqrtf(dist)) * (traildist - sqrtf(dist))) / (traildist * traildist);
    float r, g, b;
    hsp_to_rgb(hsp.x, hsp.y, hsp.z * brightness, r, g, b);
    r *= 255.f;
    g *= 255.f;
    b *= 255.f;
    float* t = trail + 3 * ((size_t)x * M + y);
    max_store(t, r * r);
    max_store(t + 1, g * g);
    max_store(t + 2, b * b);
    if (dist <= 1.f) break;
  }
}

void trails_free(bt_trails* t) {
  void* p[] = {t->cache, t->count, t->grad, t->trail, t->keys[0], t->keys[1], t->vals[0],
               t->vals[1], t->part, t->frac, t->bb, t->ctr, t->tmp};
  for (void* x : p)
    if (x) cudaFree(x);
  if (t->ctr_host) cudaFreeHost(t->ctr_host);
}

}  // namespace

namespace bt {

int trails_run(bt_trails* t, MapScratch& Sc, const MapFrame& F, const StarSet& SS,
               cudaStream_t s) {
  if (t->M != Sc.M || t->N != Sc.N || t->n_stars != SS.n) {
    set_error("invalid argument: trails made for %d x %d and %d stars, frame is %d x %d "
              "with %d stars", t->M, t->N, t->n_stars, Sc.M, Sc.N, SS.n);
    return BT_ERR_ARG;
  }
  const int M = Sc.M, N = Sc.N;
  const int cur = (int)(t->frame & 1), prv = 1 - cur;
  // clearArrays: this parity's counts, both at frame 0
  if (t->frame == 0)
    BT_CUDA_TRY(cudaMemsetAsync(t->count, 0, 2 * (size_t)t->n_stars * sizeof(int32_t), s));
  else
    BT_CUDA_TRY(cudaMemsetAsync(t->count + (size_t)cur * t->n_stars, 0,
                                (size_t)t->n_stars * sizeof(int32_t), s));
  BT_CUDA_TRY(cudaMemsetAsync(t->trail, 0, (size_t)M * N * 3 * sizeof(float), s));
  BT_CUDA_TRY(cudaMemsetAsync(t->ctr, 0, 2 * sizeof(uint32_t), s));
  BT_CUDA_TRY(cudaMemsetAsync(t->keys[0], 0xff, t->cap * sizeof(uint64_t), s));
  k_trail_grad<<<dim3((M + 1 + TX - 1) / TX, (N + 1 + TY - 1) / TY), dim3(TX, TY), 0, s>>>(
      Sc.thphi, M, N, t->grad);
  k_trail_hits<<<dim3((M + TX - 1) / TX, (N + TY - 1) / TY), dim3(TX, TY), 0, s>>>(
      Sc.thphi, Sc.bh, SS, F.cam, M, N, F.step, F.view, F.lr, Sc.area, t->keys[0],
      t->vals[0], t->part, t->frac, t->bb, t->ctr, t->cap);
  BT_CUDA_TRY(cudaGetLastError());
  size_t bytes = t->tmp_bytes;
  BT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(t->tmp, bytes, t->keys[0], t->keys[1],
                                              t->vals[0], t->vals[1], (int64_t)t->cap, 0,
                                              64, s));
  const unsigned blocks = (unsigned)((t->cap + 255) / 256);
  k_trail_store<<<blocks, 256, 0, s>>>(t->keys[1], t->cap, M, t->trailnum,
                                       t->cache + (size_t)cur * t->n_stars * t->trailnum,
                                       t->count + (size_t)cur * t->n_stars);
  k_trail_draw<<<blocks, 256, 0, s>>>(t->keys[1], t->vals[1], t->cap, t->part, t->frac, t->bb,
                                      SS.bb_hsp, M, N, t->trailnum,
                                      t->cache + (size_t)prv * t->n_stars * t->trailnum,
                                      t->count + (size_t)prv * t->n_stars, t->grad, t->trail,
                                      t->ctr + 1);
  BT_CUDA_TRY(cudaGetLastError());
  BT_CUDA_TRY(cudaMemcpyAsync(t->ctr_host, t->ctr, 2 * sizeof(uint32_t),
                              cudaMemcpyDeviceToHost, s));
  t->frame++;
  return BT_OK;
}

const float* trails_buffer(const bt_trails* t) { return t->trail; }

}  // namespace bt

extern "C" {

int bt_trails_create(int n_stars, int width, int height, int trailnum, size_t max_hits,
                     bt_trails** out) {
  clear_error();
  BT_ARG_CHECK(out, "NULL pointer");
  BT_ARG_CHECK(n_stars > 0 && width > 0 && height > 0 && trailnum > 0 && trailnum <= 1024,
               "invalid trail sizes");
  BT_ARG_CHECK((size_t)width * height < ((size_t)1 << 32), "frame too large for trails");
  *out = nullptr;
  bt_trails* t = new (std::nothrow) bt_trails;
  if (!t) return BT_ERR_NOMEM;
  std::memset(t, 0, sizeof(*t));
  t->n_stars = n_stars;
  t->M = width;
  t->N = height;
  t->trailnum = trailnum;
  t->cap = max_hits ? max_hits : std::max((size_t)1 << 16, (size_t)width * height);
  const size_t M1N1 = (size_t)(width + 1) * (height + 1);
  cudaError_t e = cudaMalloc((void**)&t->cache, 2 * (size_t)n_stars * trailnum * sizeof(int2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&t->count, 2 * (size_t)n_stars * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMalloc((void**)&t->grad, M1N1 * sizeof(float2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&t->trail, (size_t)width * height * 3 * sizeof(float));
  for (int b = 0; b < 2 && e == cudaSuccess; b++) {
    e = cudaMalloc((void**)&t->keys[b], t->cap * sizeof(uint64_t));
    if (e == cudaSuccess) e = cudaMalloc((void**)&t->vals[b], t->cap * sizeof(uint32_t));
  }
  if (e == cudaSuccess) e = cudaMalloc((void**)&t->part, t->cap * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc((void**)&t->frac, t->cap * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc((void**)&t->bb, t->cap * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMalloc((void**)&t->ctr, 2 * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&t->ctr_host, 2 * sizeof(uint32_t));
  if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(
                            nullptr, t->tmp_bytes, t->keys[0], t->keys[1], t->vals[0],
                            t->vals[1], (int64_t)t->cap, 0, 64, (cudaStream_t)0);
  if (e == cudaSuccess) e = cudaMalloc(&t->tmp, t->tmp_bytes);
  if (e == cudaSuccess) e = cudaMemset(t->grad, 0, M1N1 * sizeof(float2));
  if (e == cudaSuccess) e = cudaMemset(t->ctr, 0, 2 * sizeof(uint32_t));
  if (e != cudaSuccess) {
    set_error("trail buffers: %s", cudaGetErrorString(e));
    trails_free(t);
    delete t;
    return BT_ERR_NOMEM;
  }
  t->ctr_host[0] = t->ctr_host[1] = 0;
  *out = t;
  return BT_OK;
}

void bt_trails_destroy(bt_trails* t) {
  if (!t) return;
  cudaDeviceSynchronize();
  trails_free(t);
  delete t;
}

int bt_trails_reset(bt_trails* t) {
  clear_error();
  BT_ARG_CHECK(t, "NULL pointer");
  t->frame = 0;
  return BT_OK;
}

int bt_trails_query(bt_trails* t, bt_trails_info* info, void* stream) {
  clear_error();
  BT_ARG_CHECK(t && info, "NULL pointer");
  BT_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  info->frame = t->frame;
  const uint32_t h = t->ctr_host[0];
  info->hits = (uint32_t)std::min((size_t)h, t->cap);
  info->dropped = h > t->cap ? (uint32_t)(h - t->cap) : 0;
  info->walks_cut = t->ctr_host[1];
  info->trail = t->trail;
  return BT_OK;
}

}  // extern "C"
