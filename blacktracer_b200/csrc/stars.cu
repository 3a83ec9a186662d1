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
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
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
  float4* box;
  float4* bb;    // 2 * kBlackbodyEntries: HSP, then RGB at unit brightness
  float4* bb1k;  // the same for the 1024-entry FP32 table
  uchar3* psf;
  short2* psf_nzoff;
  float4* psf_nzval;
  short2* psf_lvoff;
  float4* psf_lvval;
  int* psf_lvstart;
};

namespace bt {

constexpr int kBlackbody1k = 1024;

const StarSet* stars_internal(const bt_stars* s) { return &s->s; }

StarSet stars_for_frame(const bt_stars* s, int bb_table) {
  StarSet o = s->s;
  if (bb_table == 1) {
    o.bb_hsp = s->bb1k;
    o.bb_rgb = s->bb1k + kBlackbody1k;
    o.bb_n = kBlackbody1k;
  }
  return o;
}

constexpr int TX = 32, TY = 8;
static dim3 grid2(int w, int h) {
  return dim3((unsigned)((w + TX - 1) / TX), (unsigned)((h + TY - 1) / TY));
}

// pixel_setup kept out of line where it runs once per lane ahead of a hot
// loop: its lensing and redshift code is large, and inlined it crowds the
// loop out of the instruction cache.
__device__ __noinline__ bool pixel_setup_ool(const float2* thphi, const uint8_t* bh,
                                             const float* cam, int M, int step,
                                             const float2* view, int lr, const float* area,
                                             int i, int j, PixelStars& P, float* mn,
                                             float* mx) {
  return pixel_setup(thphi, bh, cam, M, step, view, lr, area, i, j, P, mn, mx);
}

// Star tests (node tests count kNodeCost) a pixel may spend in the warp
// path before it is handed to k_star_heavy, and the number of kd-tree
// leaves it may list.  Pixels next to the shadow project onto quads that
// hold up to hundreds of thousands of stars; they get a whole block.
constexpr long kStarBudget = 2048;
constexpr int kLeaves = 32;
constexpr int kWarps = TX * TY / 32;

// Broadcast of a star hit from lane b.
__device__ __forceinline__ StarHit shfl_hit(const StarHit& h, int b) {
  StarHit o;
  o.st = __shfl_sync(0xffffffffu, h.st, b);
  o.sp = __shfl_sync(0xffffffffu, h.sp, b);
  o.part = __shfl_sync(0xffffffffu, h.part, b);
  o.hsp.x = __shfl_sync(0xffffffffu, h.hsp.x, b);
  o.hsp.y = __shfl_sync(0xffffffffu, h.hsp.y, b);
  o.hsp.z = __shfl_sync(0xffffffffu, h.hsp.z, b);
  return o;
}

// distortStarMap without trails, one warp per 32 pixels of a row.
// Phase A, lane = pixel: corners, lensing, redshift, kd-tree search; the
// leaves whose stars may fall inside the pixel's quad are listed in shared
// memory (pixels over the budget go to the heavy list).  Phase B, for each
// pixel of the warp in turn: the warp tests the listed stars 32 at a time
// and appends the hits, in star order, to a queue of the warp.  A queue that
// cannot take a test step's hits (and the queue at the end) is drained: each
// lane places one queued star in its pixel (bisection) and colours it, then
// the stars' cells are computed a few stars per warp step and added in queue
// order, so each cell of each pixel sums its stars in the order the
// reference does and is bit-identical to the reference's.  Queueing across
// pixels lets the bisection run on up to 32 hits at once instead of on the
// one or two lanes of a test step that hold a hit.
__global__ void __launch_bounds__(TX * TY)
k_star_cells(const float2* __restrict__ thphi, const uint8_t* __restrict__ bh,
             StarSet S, Cam7 cam, int M, int N, int step,
             const float2* __restrict__ view, int lr, const float* __restrict__ area,
             float3* __restrict__ cells, uint8_t* __restrict__ flag,
             uint32_t* __restrict__ heavy, uint32_t* nheavy) {
  __shared__ int sh_leaf[kWarps][kLeaves][32];
  __shared__ PixelCore sh_core[kWarps][32];
  const int lane = threadIdx.x, w = threadIdx.y;
  const int j = blockIdx.x * TX + lane;
  const int i = blockIdx.y * TY + w;
  const bool valid = i < N && j < M;
  const size_t ij = valid ? (size_t)i * M + j : 0;
  const int fw = 2 * step + 1, fw2 = fw * fw;

  // ---- phase A: this lane's pixel ----
  int nleaf = 0;
  if (valid) {
    PixelStars P;
    float mn[2], mx[2];
    if (pixel_setup_ool(thphi, bh, cam.v, M, step, view, lr, area, i, j, P, mn, mx)) {
      P.budget = kStarBudget;
      tree_search(S, mn, mx, [&](int node) {
        walk_leaves(P, S, node, node_level(node), [&](int leaf) {
          int a0, a1;
          node_range(S, leaf, a0, a1);
          P.tested += a1 - a0;
          if (P.tested > P.budget || nleaf == kLeaves) {
            P.abort = true;
            return false;
          }
          sh_leaf[w][nleaf++][lane] = leaf;
          return true;
        });
        return !P.abort;
      });
      if (P.abort) {
        heavy[atomicAdd(nheavy, 1u)] = (uint32_t)ij;
        nleaf = 0;
      } else if (nleaf) {
        sh_core[w][lane] = core_of(P);
      }
    }
  }
  __syncwarp();

  // ---- phase B: the warp tests the stars of each listed pixel; hits wait
  // in a per-warp queue of 32 in test order, which is drained (placed and
  // splatted, one hit per lane) when a test step's hits would not fit ----
  __shared__ int sh_hq[kWarps][32];
  __shared__ float2 sh_hpos[kWarps][32];
  __shared__ uint8_t sh_hpx[kWarps][32];
  const float maxDistSq = (step + .5f) * (step + .5f);
  int my_any = 0;
  int qn = 0;
  int cur = -1;  // the pixel whose cells acc holds
  float3 acc = make_float3(0.f, 0.f, 0.f);
  auto flush_cells = [&]() {
    if (cur >= 0) {
      const size_t pij = (size_t)i * M + (blockIdx.x * TX + cur);
      if (lane < fw2) cells[pij * fw2 + lane] = acc;
      if (lane == cur) my_any = 1;
    }
  };
  auto drain = [&](int count) {
    StarHit h{};
    int hpx = 0;
    if (lane < count) {
      hpx = sh_hpx[w][lane];
      PixelStars Q;
      stars_of(sh_core[w][hpx], step, Q);
      const float2 pos = sh_hpos[w][lane];
      h = star_hit(Q, S, sh_hq[w][lane], pos.x, pos.y);
    }
    // The cells of G = 32 / (2s+1)^2 queued stars per step: lane
    // g * (2s+1)^2 + c computes cell c of star e0 + g, then lane c adds the G
    // results in queue order.  A cell outside the splat radius yields +0, which leaves the sum
    // unchanged (the sums start at +0 and add squares), so every cell sums
    // exactly what the star-by-star loop of the reference sums.
    const int G = 32 / fw2;
    const int g = lane / fw2, c = lane - g * fw2;
    for (int e0 = 0; e0 < count; e0 += G) {
      const bool mine = g < G && e0 + g < count;
      const int src = mine ? e0 + g : 0;
      const StarHit hb = shfl_hit(h, src);
      const int pl = __shfl_sync(0xffffffffu, hpx, src);
      float3 l = make_float3(0.f, 0.f, 0.f);
      if (mine && !cell_light_v(step, maxDistSq, sh_core[w][pl].frac, hb.st, hb.sp, hb.part,
                                hb.hsp.x, hb.hsp.y, hb.hsp.z, c / fw, c % fw, l))
        l = make_float3(0.f, 0.f, 0.f);
      const int ng = min(G, count - e0);
      for (int k = 0; k < ng; k++) {
        const int pe = __shfl_sync(0xffffffffu, hpx, e0 + k);
        if (pe != cur) {
          flush_cells();
          cur = pe;
          acc = make_float3(0.f, 0.f, 0.f);
        }
        const int from = min(k * fw2 + lane, 31);
        const float lx = __shfl_sync(0xffffffffu, l.x, from);
        const float ly = __shfl_sync(0xffffffffu, l.y, from);
        const float lz = __shfl_sync(0xffffffffu, l.z, from);
        if (lane < fw2) {
          acc.x += lx;
          acc.y += ly;
          acc.z += lz;
        }
      }
    }
  };
  // One loop over the warp's pixels, leaves and star steps with the drain at
  // a single call site (the kernel's hot code is what bounds it; a second
  // inlined copy of the drain for the last hits doubled it).  A step whose
  // hits would not fit waits in registers while the queue drains.
  PixelStars P;
  int px = -1, n = 0, k = 0;  // pixel, its leaves, the next leaf
  int base = 0, a1 = 0;       // star range left of the current leaf
  bool pend = false, in = false;  // a tested step waiting for room; its lane result
  int q = 0, cnt = 0;
  unsigned ball = 0;
  float st = 0.f, sp = 0.f;
  for (;;) {
    bool done = false;
    for (;;) {
      if (pend) {
        if (qn + cnt > 32) break;  // drain first
        if (in) {
          const int at = qn + __popc(ball & ((1u << lane) - 1u));
          sh_hq[w][at] = q;
          sh_hpos[w][at] = make_float2(st, sp);
          sh_hpx[w][at] = (uint8_t)px;
        }
        qn += cnt;
        pend = false;
      }
      if (base < a1) {
        q = base + lane;
        base += 32;
        st = 0.f;
        sp = 0.f;
        in = q < a1 && star_test(P, S, q, st, sp);
        ball = __ballot_sync(0xffffffffu, in);
        cnt = __popc(ball);
        pend = cnt != 0;
      } else if (k < n) {
        node_range(S, sh_leaf[w][k][px], base, a1);
        k++;
      } else if (px < 31) {
        px++;
        n = __shfl_sync(0xffffffffu, nleaf, px);
        k = 0;
        if (n) stars_of(sh_core[w][px], step, P);
      } else {
        done = true;
        break;
      }
    }
    if (qn) {
      __syncwarp();
      drain(qn);
      __syncwarp();
      qn = 0;
    }
    if (done) break;
  }
  flush_cells();
  // heavy pixels are written 0 here and flagged again by k_star_heavy
  if (valid) flag[ij] = (uint8_t)my_any;
}

constexpr int kHeavyNodes = 1024;   // nodes per search pass (shared memory)
// Candidate leaves box-tested per batch of a deferred pixel.
constexpr int kHeavyBatch = 2048;

// heavy_count layout: [0] deferred pixels, [1] and [2] the two queues of
// k_star_heavy (front and back of `order`; the unit path fills only the
// first, with the pixels that did not fit its node pool), [3] its shared
// item counter.
enum { kHcDeferred = 0, kHcGiant = 1, kHcOther = 2, kHcNext = 3, kHcWords = 4 };

// ---- Deferred pixels in units of candidate leaves ----
// A deferred pixel's kd-tree search emits nodes; the leaves under them, laid
// end to end in emission order, are the pixel's candidate leaves.  All
// deferred pixels' candidate leaves are cut into units of U leaves (one
// pixel per unit) that warps take from a counter: a pixel of a million
// candidate stars spreads over every SM instead of holding one block.  Each
// unit's cell sums go to its own slot, and a last pass adds a pixel's units
// in unit order, so frames are reproducible.  Pixels whose nodes do not fit
// the node pool go to the block-per-pixel kernel (k_star_heavy).
enum { kHvUnits = 0, kHvUnitLeaves = 1, kHvFetch = 2, kHvWords = 4 };
// Rounds of 32 leaves per unit, at least (more when the unit slots run out).
constexpr int kUnitRounds = 1;
// Emitted nodes per deferred pixel the first pass keeps (a 4K frame's
// deferred pixels emit up to ~570); a pixel that emits more is searched
// again by the second pass.
constexpr uint32_t kHvSlab = 1024;

// Pass 1, one thread per deferred pixel: the nodes its search emits and the
// leaves under them.
__global__ void k_hv_count(const float2* __restrict__ thphi, const uint8_t* __restrict__ bh,
                           StarSet S, Cam7 cam, int M, int step,
                           const float2* __restrict__ view, int lr,
                           const float* __restrict__ area, const uint32_t* __restrict__ heavy,
                           const uint32_t* __restrict__ hc, uint32_t* __restrict__ nn,
                           uint32_t* __restrict__ nl, int* __restrict__ slab,
                           uint32_t slab_pixels) {
  const uint32_t n = hc[kHcDeferred];
  const int L = S.treeLevel;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += gridDim.x * blockDim.x) {
    const uint32_t ij = heavy[k];
    PixelStars P;
    float mn[2], mx[2];
    uint32_t nodes = 0, leaves = 0;
    int* keep = k < slab_pixels ? slab + (size_t)k * kHvSlab : nullptr;
    if (pixel_setup(thphi, bh, cam.v, M, step, view, lr, area, ij / M, ij % M, P, mn, mx))
      tree_search(S, mn, mx, [&](int node) {
        if (keep && nodes < kHvSlab) keep[nodes] = node;
        nodes++;
        leaves += 1u << (L - node_level(node));  // disjoint nodes: at most 2^L leaves
        return true;
      });
    nn[k] = nodes;
    nl[k] = leaves;
  }
}

// Exclusive scan of one value per thread of a 1024-thread block; *total
// receives the block's sum.  sh: 32 words of shared memory.
__device__ __forceinline__ unsigned long long block_scan(unsigned long long v,
                                                         unsigned long long* sh,
                                                         unsigned long long* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned long long x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[w] = x;
  __syncthreads();
  if (w == 0) {
    unsigned long long t = sh[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    sh[lane] = t;
  }
  __syncthreads();
  const unsigned long long before = w ? sh[w - 1] : 0ull;
  *total = sh[31];
  __syncthreads();
  return before + x - v;
}

// Pass 2, one block: node offsets (noff, n + 1 entries), the unit size and
// unit offsets (uoff).  The first `ok` pixels are kept: ok is the first
// pixel whose nodes would end past node_cap, and at most unit_cap / 2; the
// others go to the fallback queue (order, as k_star_heavy's giant queue)
// with no nodes and no units.  U = 32 R leaves with R = ceil(kept leaves /
// (32 (unit_cap - ok))): each pixel's last unit may be partial, so the
// units number at most kept / U + ok <= unit_cap.
__global__ void __launch_bounds__(1024)
k_hv_scan(const uint32_t* __restrict__ heavy, uint32_t* hc, const uint32_t* __restrict__ nn,
          const uint32_t* __restrict__ nl, uint32_t* __restrict__ noff,
          uint32_t* __restrict__ uoff, uint32_t* __restrict__ order, uint32_t* ctl,
          uint32_t node_cap, uint32_t unit_cap) {
  __shared__ unsigned long long sh[32];
  __shared__ uint32_t sh_ok, sh_nodes;
  const uint32_t n = hc[kHcDeferred];
  // pixels [0, ok) keep their nodes
  if (threadIdx.x == 0) sh_ok = min(n, unit_cap / 2);
  unsigned long long base = 0;
  for (uint32_t c = 0; c < n; c += blockDim.x) {
    const uint32_t k = c + threadIdx.x;
    const unsigned long long v = k < n ? nn[k] : 0ull;
    unsigned long long tot;
    const unsigned long long off = base + block_scan(v, sh, &tot);
    if (k < n && off + v > node_cap) atomicMin(&sh_ok, k);
    base += tot;
    if (k < n) noff[k] = (uint32_t)(off < node_cap ? off : node_cap);
  }
  __syncthreads();
  const uint32_t ok = sh_ok;
  // the kept pixels' leaves, and the fallback queue
  unsigned long long kept = 0;
  for (uint32_t c = 0; c < n; c += blockDim.x) {
    const uint32_t k = c + threadIdx.x;
    const unsigned long long lv = (k < ok) ? nl[k] : 0ull;
    unsigned long long tot;
    block_scan(lv, sh, &tot);
    kept += tot;
    if (k < n && k >= ok) order[k - ok] = heavy[k];
  }
  const unsigned long long slots = 32ull * (unit_cap - ok);  // ok <= unit_cap / 2
  const unsigned long long R = kept > slots ? (kept + slots - 1) / slots : 1ull;
  const unsigned long long U = 32ull * (R > (unsigned long long)kUnitRounds ? R : kUnitRounds);
  unsigned long long ubase = 0;
  for (uint32_t c = 0; c < n; c += blockDim.x) {
    const uint32_t k = c + threadIdx.x;
    const unsigned long long u = (k < ok) ? (nl[k] + U - 1) / U : 0ull;
    unsigned long long tot;
    const unsigned long long off = ubase + block_scan(u, sh, &tot);
    ubase += tot;
    if (k < n) uoff[k] = (uint32_t)off;
  }
  if (threadIdx.x == 0) sh_nodes = ok > 0 ? noff[ok - 1] + nn[ok - 1] : 0u;
  __syncthreads();
  const uint32_t nodes_ok = sh_nodes;
  for (uint32_t k = ok + threadIdx.x; k <= n; k += blockDim.x) noff[k] = nodes_ok;
  if (threadIdx.x == 0) {
    uoff[n] = (uint32_t)ubase;
    ctl[kHvUnits] = (uint32_t)ubase;
    ctl[kHvUnitLeaves] = (uint32_t)U;
    ctl[kHvFetch] = 0;
    // k_star_heavy takes the fallback pixels as its giant queue
    hc[kHcGiant] = n - ok;
    hc[kHcOther] = 0;
    hc[kHcNext] = 0;
  }
}

// Pass 3, one thread per kept deferred pixel: its search again, the nodes
// into the pool with the leaves up to each (within the pixel).
__global__ void k_hv_nodes(const float2* __restrict__ thphi, const uint8_t* __restrict__ bh,
                           StarSet S, Cam7 cam, int M, int step,
                           const float2* __restrict__ view, int lr,
                           const float* __restrict__ area, const uint32_t* __restrict__ heavy,
                           const uint32_t* __restrict__ hc, const uint32_t* __restrict__ noff,
                           const int* __restrict__ slab, uint32_t slab_pixels,
                           int* __restrict__ pool, uint32_t* __restrict__ pend) {
  const uint32_t n = hc[kHcDeferred];
  const int L = S.treeLevel;
  const unsigned lane = threadIdx.x & 31u;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < n; k += warps) {
    const uint32_t b0 = noff[k], b1 = noff[k + 1];
    if (b0 == b1) continue;
    if (k < slab_pixels && b1 - b0 <= kHvSlab) {
      // the first pass kept them: copy, the leaves up to each node as a
      // warp prefix sum
      const int* src = slab + (size_t)k * kHvSlab;
      uint32_t carry = 0;
      for (uint32_t e0 = b0; e0 < b1; e0 += 32) {
        const uint32_t e = e0 + lane;
        const int node = e < b1 ? src[e - b0] : 0;
        uint32_t c = e < b1 ? 1u << (L - node_level(node)) : 0u;
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t y = __shfl_up_sync(0xffffffffu, c, o);
          if (lane >= (unsigned)o) c += y;
        }
        if (e < b1) {
          pool[e] = node;
          pend[e] = carry + c;
        }
        carry += __shfl_sync(0xffffffffu, c, 31);
      }
      continue;
    }
    // more nodes than the slab holds (or past its pixels): lane 0 searches
    // again while the warp waits, so that every lane stays on this pixel
    if (lane == 0) {
      const uint32_t ij = heavy[k];
      PixelStars P;
      float mn[2], mx[2];
      pixel_setup(thphi, bh, cam.v, M, step, view, lr, area, ij / M, ij % M, P, mn, mx);
      uint32_t e = b0, cum = 0;
      tree_search(S, mn, mx, [&](int node) {
        if (e >= b1) return false;  // the same search as pass 1: never taken
        cum += 1u << (L - node_level(node));
        pool[e] = node;
        pend[e] = cum;
        e++;
        return true;
      });
    }
    __syncwarp();
  }
}

// Pass 4: warps take units.  A unit is leaves [f0, f0 + U) of its pixel's
// candidate leaves; lane l box-tests leaf f0 + 32 r + l, the warp sweeps the
// survivors' stars 32 at a time, queues the hits and splats them 32 at a
// time, one per lane, into the lane's cell registers (the per-star form of
// the brightness, star_fast); the warp's sums go to the unit's slot.
// Three blocks per SM (85 registers, a few spilled): the kernel is bound by
// instruction fetch and more resident warps hide it (13.7 -> 13.2 ms per 4K
// frame against two blocks; four blocks spilled too much to gain more).
template <int kStep>
__global__ void __launch_bounds__(256, 3)
k_star_units(const float2* __restrict__ thphi, const uint8_t* __restrict__ bh, StarSet S,
             Cam7 cam, int M, const float2* __restrict__ view, int lr,
             const float* __restrict__ area, const uint32_t* __restrict__ heavy,
             const uint32_t* __restrict__ hc, const uint32_t* __restrict__ noff,
             const uint32_t* __restrict__ uoff, const int* __restrict__ pool,
             const uint32_t* __restrict__ pend, uint32_t* ctl, float* __restrict__ partial,
             uint8_t* __restrict__ uany) {
  constexpr int FW = 2 * kStep + 1, FW2 = FW * FW;
  constexpr int kWarps = 256 / 32;
  __shared__ int sh_q[kWarps][64];
  __shared__ float2 sh_qpos[kWarps][64];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int L = S.treeLevel;
  const uint32_t n = hc[kHcDeferred];
  const uint32_t total = ctl[kHvUnits];
  const uint32_t U = ctl[kHvUnitLeaves];
  for (;;) {
    uint32_t u = 0;
    if (lane == 0) u = atomicAdd(&ctl[kHvFetch], 1u);
    u = __shfl_sync(0xffffffffu, u, 0);
    if (u >= total) break;
    // the unit's pixel: the last k with uoff[k] <= u (pixels without units
    // share their offset with the next pixel)
    uint32_t lo = 0, hi = n - 1;
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (uoff[mid] <= u) lo = mid;
      else hi = mid - 1;
    }
    const uint32_t k = lo;
    const uint32_t ij = heavy[k];
    PixelStars P;
    float mn[2], mx[2];
    pixel_setup(thphi, bh, cam.v, M, kStep, view, lr, area, ij / M, ij % M, P, mn, mx);
    const uint32_t n0 = noff[k], n1 = noff[k + 1];
    const uint32_t f0 = (u - uoff[k]) * U;
    const uint32_t f1 = min(f0 + U, pend[n1 - 1]);
    float3 acc[FW2];
#pragma unroll
    for (int c = 0; c < FW2; c++) acc[c] = make_float3(0.f, 0.f, 0.f);
    int any = 0, qn = 0;
    auto splat_queued = [&](int q_at) {
      const int q = sh_q[w][q_at];
      const float2 pos = sh_qpos[w][q_at];
      const StarHit h = star_hit(P, S, q, pos.x, pos.y);
      splat_cells<kStep>(P, h, star_fast(P, S, h), acc);
    };
    // One loop that tests until 32 hits are queued (or the unit is done) and
    // then splats them, so that the splat has a single call site: the kernel
    // is bound by instruction fetch, and a second inlined copy of the splat
    // for the last hits doubled its hot code.
    uint32_t f = f0;     // next batch of 32 candidate leaves
    unsigned keep = 0;   // batch lanes whose leaf survived the box test
    int leaf = -1;       // this lane's leaf of the batch
    int qb = 0, a1 = 0;  // star range left of the current leaf
    for (;;) {
      bool done = false;
      while (qn < 32) {
        if (qb < a1) {
          const int q = qb + lane;
          qb += 32;
          float st = 0.f, sp = 0.f;
          const bool in = q < a1 && star_test(P, S, q, st, sp);
          const unsigned ball = __ballot_sync(0xffffffffu, in);
          if (!ball) continue;
          any = 1;
          if (in) {
            const int at = qn + __popc(ball & ((1u << lane) - 1u));
            sh_q[w][at] = q;
            sh_qpos[w][at] = make_float2(st, sp);
          }
          qn += __popc(ball);
        } else if (keep) {
          const int src = __ffs(keep) - 1;
          keep &= keep - 1;
          node_range(S, __shfl_sync(0xffffffffu, leaf, src), qb, a1);
        } else if (f < f1) {
          const uint32_t kk = f + lane;
          f += 32;
          leaf = -1;
          if (kk < f1) {
            uint32_t a = n0, b = n1 - 1;  // first node whose leaves reach past kk
            while (a < b) {
              const uint32_t mid = (a + b) >> 1;
              if (pend[mid] > kk) b = mid;
              else a = mid + 1;
            }
            const int node = pool[a];
            const int d = L - node_level(node);
            const uint32_t start = a > n0 ? pend[a - 1] : 0u;
            leaf = (int)((((long long)node + 1) << d) - 1 + (kk - start));
            if (node_excluded(P, S.box[leaf])) leaf = -1;
          }
          keep = __ballot_sync(0xffffffffu, leaf >= 0);
        } else {
          done = true;
          break;
        }
      }
      if (qn == 0) break;
      __syncwarp();
      if (lane < qn) splat_queued(lane);
      __syncwarp();
      if (qn > 32) {
        if (lane < qn - 32) {
          sh_q[w][lane] = sh_q[w][lane + 32];
          sh_qpos[w][lane] = sh_qpos[w][lane + 32];
        }
        qn -= 32;
      } else {
        qn = 0;
      }
      __syncwarp();
      if (done && qn == 0) break;
    }
    float* out = partial + (size_t)u * (FW2 * 3);
#pragma unroll
    for (int c = 0; c < FW2; c++) {
      float x = acc[c].x, y = acc[c].y, z = acc[c].z;
      for (int o = 16; o > 0; o >>= 1) {
        x += __shfl_xor_sync(0xffffffffu, x, o);
        y += __shfl_xor_sync(0xffffffffu, y, o);
        z += __shfl_xor_sync(0xffffffffu, z, o);
      }
      if (lane == 0) {
        out[3 * c] = x;
        out[3 * c + 1] = y;
        out[3 * c + 2] = z;
      }
    }
    if (lane == 0) uany[u] = any ? 1 : 0;
  }
}

// Pass 5, one warp per deferred pixel with units: its cells are the sums of
// its units' slots in unit order (lane c adds component c), its flag whether
// any unit splatted a star.
template <int kStep>
__global__ void k_star_units_sum(const uint32_t* __restrict__ heavy,
                                 const uint32_t* __restrict__ hc,
                                 const uint32_t* __restrict__ uoff,
                                 const float* __restrict__ partial,
                                 const uint8_t* __restrict__ uany, float* __restrict__ cells,
                                 uint8_t* __restrict__ flag) {
  constexpr int FW = 2 * kStep + 1, C = FW * FW * 3;
  const uint32_t n = hc[kHcDeferred];
  const int lane = threadIdx.x & 31;
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); k < n; k += warps) {
    const uint32_t u0 = uoff[k], u1 = uoff[k + 1];
    if (u0 == u1) continue;  // no candidates, or a fallback pixel
    int a = 0;
    for (uint32_t u = u0 + lane; u < u1; u += 32) a |= uany[u];
    const bool any = __any_sync(0xffffffffu, a != 0);
    const uint32_t ij = heavy[k];
    if (any)
      for (int c = lane; c < C; c += 32) {
        float v = 0.f;
        for (uint32_t u = u0; u < u1; u++) v += partial[(size_t)u * C + c];
        cells[(size_t)ij * C + c] = v;
      }
    if (lane == 0) flag[ij] = any ? 1 : 0;
  }
}

// Deferred pixels that did not fit the unit path's node pool, one block at a
// time each, taken from the queues by a shared counter; kThreads-thread
// blocks.  Thread 0
// walks the kd-tree (in passes of kHeavyNodes emitted nodes) into shared
// memory with a prefix sum of the number of leaves under each node.  The
// block then takes that flat range of candidate leaves kHeavyBatch at a time:
// thread t box-tests leaves t, t + kThreads, ... of the batch against the
// pixel's quad, each warp lists its survivors in its own segment, and after
// one barrier the warps sweep the survivors round-robin, one leaf at a time,
// 32 stars per step.  Hits wait in a per-warp queue and are splatted 32 at a
// time, one per lane, into the lane's (2s+1)^2 cell registers with the
// per-star form of the brightness (star_fast); the threads' cells are added
// by a block reduction at the end.  Sums are reassociated relative to the
// reference's star order, which changes them only by float rounding; the
// order is fixed, so frames are reproducible.
template <int kStep, int kThreads>
__global__ void __launch_bounds__(kThreads, 512 / kThreads)
k_star_heavy(const float2* __restrict__ thphi, const uint8_t* __restrict__ bh,
             StarSet S, Cam7 cam, int M, int N, const float2* __restrict__ view,
             int lr, const float* __restrict__ area, float3* __restrict__ cells,
             uint8_t* __restrict__ flag, const uint32_t* __restrict__ order,
             uint32_t* hc, uint32_t np) {
  constexpr int FW = 2 * kStep + 1, FW2 = FW * FW;
  constexpr int kWarps = kThreads / 32;
  constexpr int kPer = kHeavyBatch / kThreads;  // leaves per thread per batch
  __shared__ int sh_node[kHeavyNodes];
  __shared__ long long sh_end[kHeavyNodes];  // inclusive prefix of leaf counts
  __shared__ int sh_count, sh_more;
  __shared__ long long sh_total;
  __shared__ int sh_surv[kWarps][kPer * 32];
  __shared__ int sh_wcount[kWarps];
  __shared__ float3 sh_red[kWarps][FW2];
  __shared__ uint32_t sh_item;
  __shared__ int sh_q[kWarps][64];
  __shared__ float2 sh_qpos[kWarps][64];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int L = S.treeLevel;
  for (;;) {
    if (tid == 0) sh_item = atomicAdd(&hc[kHcNext], 1u);
    __syncthreads();
    const uint32_t item = sh_item;
    const uint32_t ng = hc[kHcGiant], no = hc[kHcOther];
    __syncthreads();
    if (item >= ng + no) break;
    const uint32_t ij = item < ng ? order[item] : order[np - 1 - (item - ng)];
    const int i = ij / M, j = ij % M;
    PixelStars P;
    float mn[2], mx[2];
    pixel_setup(thphi, bh, cam.v, M, kStep, view, lr, area, i, j, P, mn, mx);
    float3 acc[FW2];
#pragma unroll
    for (int c = 0; c < FW2; c++) acc[c] = make_float3(0.f, 0.f, 0.f);
    int any = 0;
    int skip = 0;
    // Stars that passed the quad test wait in a per-warp queue and are
    // placed, coloured and splatted 32 at a time, one per lane.
    int qn = 0;
    auto splat_queued = [&](int k) {
      const int q = sh_q[w][k];
      const float2 pos = sh_qpos[w][k];
      const StarHit h = star_hit(P, S, q, pos.x, pos.y);
      splat_cells<kStep>(P, h, star_fast(P, S, h), acc);
    };
    for (;;) {
      if (tid == 0) {
        int emitted = 0, count = 0, more = 0;
        long long total = 0;
        tree_search(S, mn, mx, [&](int node) {
          if (emitted >= skip + kHeavyNodes) {
            more = 1;
            return false;
          }
          if (emitted >= skip) {
            total += 1ll << (L - node_level(node));
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
      const int count = sh_count;
      const long long total = sh_total;
      for (long long base = 0; base < total; base += kHeavyBatch) {
        // box tests: this warp's survivors, in (round, lane) order
        int wn = 0;
#pragma unroll 1
        for (int r = 0; r < kPer; r++) {
          const long long k = base + (long long)r * kThreads + tid;
          int leaf = -1;
          if (k < total) {
            int lo = 0, hi = count - 1;
            while (lo < hi) {
              const int mid = (lo + hi) >> 1;
              if (sh_end[mid] > k) hi = mid;
              else lo = mid + 1;
            }
            const int node = sh_node[lo];
            const int d = L - node_level(node);
            leaf = (int)((((long long)node + 1) << d) - 1 + (k - (lo ? sh_end[lo - 1] : 0)));
            if (node_excluded(P, S.box[leaf])) leaf = -1;
          }
          const unsigned keep = __ballot_sync(0xffffffffu, leaf >= 0);
          if (leaf >= 0) sh_surv[w][wn + __popc(keep & ((1u << lane) - 1u))] = leaf;
          wn += __popc(keep);
        }
        if (lane == 0) sh_wcount[w] = wn;
        __syncthreads();
        int ns = 0;
        for (int ww = 0; ww < kWarps; ww++) ns += sh_wcount[ww];
        // sweep: survivor s (over the warps' segments in order) to warp s % kWarps
        int seg = 0, segbase = 0;
        for (int s = w; s < ns; s += kWarps) {
          while (s >= segbase + sh_wcount[seg]) segbase += sh_wcount[seg++];
          int a0, a1;
          node_range(S, sh_surv[seg][s - segbase], a0, a1);
          for (int qb = a0; qb < a1; qb += 32) {
            const int q = qb + lane;
            float st = 0.f, sp = 0.f;
            const bool in = q < a1 && star_test(P, S, q, st, sp);
            const unsigned ball = __ballot_sync(0xffffffffu, in);
            if (!ball) continue;
            any = 1;
            if (in) {
              const int at = qn + __popc(ball & ((1u << lane) - 1u));
              sh_q[w][at] = q;
              sh_qpos[w][at] = make_float2(st, sp);
            }
            qn += __popc(ball);
            if (qn >= 32) {
              __syncwarp();
              splat_queued(lane);
              __syncwarp();
              if (lane < qn - 32) {
                sh_q[w][lane] = sh_q[w][lane + 32];
                sh_qpos[w][lane] = sh_qpos[w][lane + 32];
              }
              qn -= 32;
              __syncwarp();
            }
          }
        }
        __syncthreads();
      }
      const int more = sh_more;
      __syncthreads();
      if (!more) break;
      skip += kHeavyNodes;
    }
    if (lane < qn) splat_queued(lane);
    __syncwarp();
    any = __syncthreads_or(any);
    if (any) {
#pragma unroll
      for (int c = 0; c < FW2; c++) {
        float x = acc[c].x, y = acc[c].y, z = acc[c].z;
        for (int o = 16; o > 0; o >>= 1) {
          x += __shfl_xor_sync(0xffffffffu, x, o);
          y += __shfl_xor_sync(0xffffffffu, y, o);
          z += __shfl_xor_sync(0xffffffffu, z, o);
        }
        if (lane == 0) sh_red[w][c] = make_float3(x, y, z);
      }
      __syncthreads();
      if (tid < FW2) {
        float3 v = make_float3(0.f, 0.f, 0.f);
        for (int ww = 0; ww < kWarps; ww++) {
          v.x += sh_red[ww][tid].x;
          v.y += sh_red[ww][tid].y;
          v.z += sh_red[ww][tid].z;
        }
        cells[(size_t)ij * FW2 + tid] = v;
      }
    }
    if (tid == 0) flag[ij] = any ? 1 : 0;
    __syncthreads();
  }
}

// The per-entry colour tables of StarSet (bb_hsp, bb_rgb).
__global__ void k_blackbody_tables(float4* __restrict__ bb) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= kBlackbodyEntries) return;
  const float3 h = blackbody_hsp(k);
  float r, g, b;
  hsp_to_rgb(h.x, h.y, h.z, r, g, b);
  bb[k] = make_float4(h.x, h.y, h.z, 0.f);
  bb[kBlackbodyEntries + k] = make_float4(255.f * r, 255.f * g, 255.f * b, 0.f);
}

// The 1024-entry FP32 table: entry k lies at k * 390/1023 on the reference's
// 100 K grid and is the linear interpolation of its two neighbouring entries.
__global__ void k_blackbody_tables_1k(float4* __restrict__ bb) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= kBlackbody1k) return;
  const float t = (float)k * ((float)(kBlackbodyEntries - 1) / (float)(kBlackbody1k - 1));
  const int i0 = imin((int)t, kBlackbodyEntries - 2);
  const float f = t - (float)i0;
  float c[3];
  for (int q = 0; q < 3; q++)
    c[q] = ((1.f - f) * (float)blackbody(3 * i0 + q) + f * (float)blackbody(3 * i0 + 3 + q)) /
           255.f;
  float3 h;
  rgb_to_hsp(c[0], c[1], c[2], h.x, h.y, h.z);
  float r, g, b;
  hsp_to_rgb(h.x, h.y, h.z, r, g, b);
  bb[k] = make_float4(h.x, h.y, h.z, 0.f);
  bb[kBlackbody1k + k] = make_float4(255.f * r, 255.f * g, 255.f * b, 0.f);
}

// Threads per block of k_star_heavy; the launch fills the SMs with as many
// blocks as are resident at once.
constexpr int kHeavyThreads = 512;

// Buffers of the unit path (lazy): per-pixel counts and offsets, the node
// pool (max(2^21, N*M) entries) and the unit slots (max(2^18, N*M/8) units
// of (2s+1)^2 cells), sized for splat width fw.
// The unit path's scratch for np pixels and a (2s+1)^2 splat: per-pixel
// counts and offsets, the node pool, the units' cell sums and flags, the
// first pass's slab.  Small frames get small floors (a frame's deferred
// pixels that do not fit take the block-per-pixel kernel, and a pixel past
// the slab is searched twice), so that a server can hold many of them.
static size_t units_node_cap(size_t np) { return std::max<size_t>((size_t)1 << 18, np); }
static size_t units_unit_cap(size_t np) { return std::max<size_t>((size_t)1 << 15, np / 8); }
static uint32_t units_slab_pixels(size_t np) {
  return (uint32_t)std::min<size_t>(std::max<size_t>(np / 512, 1024), 32768);
}

size_t map_star_scratch_bytes(size_t np, int fw) {
  return 4 * (np + 1) * sizeof(uint32_t) + units_node_cap(np) * (sizeof(int) + sizeof(uint32_t)) +
         units_unit_cap(np) * ((size_t)fw * fw * 3 * sizeof(float) + 1) +
         (size_t)units_slab_pixels(np) * kHvSlab * sizeof(int) + kHvWords * sizeof(uint32_t);
}

static int ensure_units(MapScratch& Sc, int fw) {
  const size_t np = (size_t)Sc.M * Sc.N;
  if (Sc.hv_ctl && Sc.hv_fw >= fw) return BT_OK;
  cudaFree(Sc.hv_nn); cudaFree(Sc.hv_nl); cudaFree(Sc.hv_noff); cudaFree(Sc.hv_uoff);
  cudaFree(Sc.hv_pool); cudaFree(Sc.hv_pend); cudaFree(Sc.hv_partial); cudaFree(Sc.hv_uany);
  cudaFree(Sc.hv_ctl); cudaFree(Sc.hv_slab);
  Sc.hv_nn = Sc.hv_nl = Sc.hv_noff = Sc.hv_uoff = Sc.hv_pend = Sc.hv_ctl = nullptr;
  Sc.hv_pool = Sc.hv_slab = nullptr;
  Sc.hv_slab_pixels = 0;
  Sc.hv_partial = nullptr;
  Sc.hv_uany = nullptr;
  Sc.hv_fw = 0;
  if (!Sc.hv_node_cap) Sc.hv_node_cap = units_node_cap(np);
  if (!Sc.hv_unit_cap) Sc.hv_unit_cap = units_unit_cap(np);
  cudaError_t e = cudaSuccess;
#define HV_ALLOC(p, bytes) \
  if (e == cudaSuccess) e = cudaMalloc((void**)&(p), (bytes));
  HV_ALLOC(Sc.hv_nn, np * sizeof(uint32_t));
  HV_ALLOC(Sc.hv_nl, np * sizeof(uint32_t));
  HV_ALLOC(Sc.hv_noff, (np + 1) * sizeof(uint32_t));
  HV_ALLOC(Sc.hv_uoff, (np + 1) * sizeof(uint32_t));
  HV_ALLOC(Sc.hv_pool, Sc.hv_node_cap * sizeof(int));
  HV_ALLOC(Sc.hv_pend, Sc.hv_node_cap * sizeof(uint32_t));
  HV_ALLOC(Sc.hv_partial, Sc.hv_unit_cap * fw * fw * 3 * sizeof(float));
  HV_ALLOC(Sc.hv_uany, Sc.hv_unit_cap);
  HV_ALLOC(Sc.hv_ctl, kHvWords * sizeof(uint32_t));
  const uint32_t slab_px = Sc.hv_slab_req < 0 ? units_slab_pixels(np) : (uint32_t)Sc.hv_slab_req;
  if (slab_px) HV_ALLOC(Sc.hv_slab, (size_t)slab_px * kHvSlab * sizeof(int));
  if (e == cudaSuccess) Sc.hv_slab_pixels = slab_px;
#undef HV_ALLOC
  if (e != cudaSuccess) {
    set_error("star unit scratch allocation failed: %s", cudaGetErrorString(e));
    return BT_ERR_NOMEM;
  }
  Sc.hv_fw = fw;
  return BT_OK;
}

// Deferred pixels whose first-pass nodes the slab keeps (< 0: the default);
// the unit path's buffers are released and reserved again at the next frame.
int map_set_star_slab(MapScratch& Sc, int pixels) {
  const size_t nodes = Sc.hv_node_cap, units = Sc.hv_unit_cap;
  if (int rc = map_set_star_capacity(Sc, nodes, units)) return rc;
  Sc.hv_slab_req = pixels;
  return BT_OK;
}

// Capacities of the unit path (0: the defaults); its buffers are released
// and reserved again at the next frame.
int map_set_star_capacity(MapScratch& Sc, size_t nodes, size_t units) {
  BT_CUDA_TRY(cudaDeviceSynchronize());
  cudaFree(Sc.hv_nn); cudaFree(Sc.hv_nl); cudaFree(Sc.hv_noff); cudaFree(Sc.hv_uoff);
  cudaFree(Sc.hv_pool); cudaFree(Sc.hv_pend); cudaFree(Sc.hv_partial); cudaFree(Sc.hv_uany);
  cudaFree(Sc.hv_ctl); cudaFree(Sc.hv_slab);
  Sc.hv_nn = Sc.hv_nl = Sc.hv_noff = Sc.hv_uoff = Sc.hv_pend = Sc.hv_ctl = nullptr;
  Sc.hv_pool = Sc.hv_slab = nullptr;
  Sc.hv_slab_pixels = 0;
  Sc.hv_partial = nullptr;
  Sc.hv_uany = nullptr;
  Sc.hv_fw = 0;
  Sc.hv_node_cap = nodes;
  Sc.hv_unit_cap = units;
  return BT_OK;
}

template <int kStep>
void launch_units(MapScratch& Sc, const MapFrame& F, const StarSet& SS, cudaStream_t s) {
  static int per_sm = 0;
  if (!per_sm) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_star_units<kStep>, 256, 0);
    if (per_sm < 1) per_sm = 1;
  }
  k_star_units<kStep><<<sm_count() * per_sm, 256, 0, s>>>(
      Sc.thphi, Sc.bh, SS, F.cam, Sc.M, F.view, F.lr, Sc.area, Sc.heavy_list, Sc.heavy_count,
      Sc.hv_noff, Sc.hv_uoff, Sc.hv_pool, Sc.hv_pend, Sc.hv_ctl, Sc.hv_partial, Sc.hv_uany);
  k_star_units_sum<kStep><<<sm_count() * 4, 256, 0, s>>>(
      Sc.heavy_list, Sc.heavy_count, Sc.hv_uoff, Sc.hv_partial, Sc.hv_uany, (float*)Sc.cells,
      Sc.flag);
}

template <int kStep>
void launch_heavy(MapScratch& Sc, const MapFrame& F, const StarSet& SS, cudaStream_t s) {
  static int per_sm = 0;
  if (!per_sm) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_star_heavy<kStep, kHeavyThreads>,
                                                  kHeavyThreads, 0);
    if (per_sm < 1) per_sm = 1;
  }
  k_star_heavy<kStep, kHeavyThreads><<<sm_count() * per_sm, kHeavyThreads, 0, s>>>(
      Sc.thphi, Sc.bh, SS, F.cam, Sc.M, Sc.N, F.view, F.lr, Sc.area, Sc.cells,
      Sc.flag, Sc.heavy_order, Sc.heavy_count, (uint32_t)((size_t)Sc.M * Sc.N));
}

// sumStarLight (+ makePix + addStarsAndBackground when no diffraction).
template <bool kCompose>
__global__ void k_star_gather(const float3* __restrict__ cells,
                              const uint8_t* __restrict__ flag, int M, int N,
                              int step, float* __restrict__ light,
                              const uchar4* __restrict__ bg,
                              uchar4* __restrict__ out, int map,
                              const float* __restrict__ trail) {
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
  if (trail) {  // factor2 = 1, BT/MakeImageKernel.cu:766-770
    b.x += 1.f * trail[3 * ij];
    b.y += 1.f * trail[3 * ij + 1];
    b.z += 1.f * trail[3 * ij + 2];
  }
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

// Light of a bright pixel as the reference's thread reads it after adding
// the sprite's centre term (value `centre`) to its own pixel.
__device__ __forceinline__ float psf_term_light(float l, float div, float centre) {
  const float d = l / div * centre;
  return l + fminf(65025.f, d * d);
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
// and adding into `acc`.  The reference's thread reads its pixel again for
// every sprite entry, so the entries after the centre see the centre's term
// it added to its own pixel (psf_term_light).
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
    const uchar3 dc = psf[fh * fs + fh];
    const float lx2 = psf_term_light(lx, div, (float)dc.x),
                ly2 = psf_term_light(ly, div, (float)dc.y),
                lz2 = psf_term_light(lz, div, (float)dc.z);
    for (int c = threadIdx.x; c < (endx - startx) * fs; c += blockDim.x) {
      const int q = startx + c / fs, p = c % fs;
      const int ti = i - fh + q;
      if (ti < 0 || ti >= N) continue;
      const uchar3 d = psf[q * fs + p];
      const bool post = q > fh || (q == fh && p > fh);
      const float dx = (post ? lx2 : lx) / div * (float)d.x,
                  dy = (post ? ly2 : ly) / div * (float)d.y,
                  dz = (post ? lz2 : lz) / div * (float)d.z;
      const size_t t = (size_t)ti * M + (j - fh + p + M) % M;
      atomicAdd(&acc[3 * t], fminf(65025.f, dx * dx));
      atomicAdd(&acc[3 * t + 1], fminf(65025.f, dy * dy));
      atomicAdd(&acc[3 * t + 2], fminf(65025.f, dz * dz));
    }
  }
}

// Diffraction as a gather (addDiffraction, BT/MakeImageKernel.cu:775-800).
// A bright pixel (any channel of its summed star light above 65025) adds
// min(65025, (light / (10000 max^0.6) * sprite)^2) per channel around
// itself; written from the receiving side, pixel t gathers that term from
// every bright pixel t - o for the sprite's non-zero offsets o.  Pass 1
// stores each pixel's coefficient light / (10000 max^0.6) (zero for the
// others); pass 2 reads a tile of coefficients with its halo from shared
// memory.  No atomics: the frame is deterministic.  The reference's
// arithmetic per term is kept (coefficient times sprite value, squared,
// clamped); only the summation order differs.
//
// What each term reads: the reference's thread reads its own pixel again for
// every sprite entry, after adding the entries before it, and the centre
// entry lands on that pixel.  So the entries up to the centre (row-major)
// use the pixel's light, the entries after it its light plus the centre's
// term: two coefficients per pixel.  Other bright pixels' terms that land on
// a bright pixel are read or not depending on thread timing in the
// reference; here every pixel's coefficients come from the light before any
// term is added.
__global__ void k_diff_coef(const float* __restrict__ light, int n, float4 centre,
                            float3* __restrict__ coef, float3* __restrict__ coef_post) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const float lx = light[3 * q], ly = light[3 * q + 1], lz = light[3 * q + 2];
  const float m = fmaxf(fmaxf(lx, ly), lz);
  float3 c = make_float3(0.f, 0.f, 0.f), c2 = c;
  if (m > 65025.f) {
    const float div = 10000 * powf(m, 0.6);
    c = make_float3(lx / div, ly / div, lz / div);
    c2 = make_float3(psf_term_light(lx, div, centre.x) / div,
                     psf_term_light(ly, div, centre.y) / div,
                     psf_term_light(lz, div, centre.z) / div);
  }
  coef[q] = c;
  coef_post[q] = c2;
}

constexpr int kDiffTX = 32, kDiffTY = 8;

// Loads the coefficient tile of a kDiffTX x kDiffTY output tile with a halo
// of H on every side into shared memory (rows outside the image: zero;
// columns wrap around the sphere).
__device__ __forceinline__ void load_coef_tile(const float3* __restrict__ coef, int M, int N,
                                               int i0, int j0, int H, float3* tile,
                                               int ty = kDiffTY) {
  const int TW = kDiffTX + 2 * H, TH = ty + 2 * H;
  const int tid = threadIdx.y * kDiffTX + threadIdx.x;
  for (int k = tid; k < TW * TH; k += kDiffTX * ty) {
    const int r = k / TW, c = k % TW;
    const int i = i0 - H + r;
    const int j = ((j0 - H + c) % M + M) % M;
    tile[k] = (i >= 0 && i < N) ? coef[(size_t)i * M + j] : make_float3(0.f, 0.f, 0.f);
  }
}

// Sprite entries [k0, k1) gathered from the coefficient tile into a.
__device__ __forceinline__ void diff_gather_range(const float3* tile, int base, int TW, int k0,
                                                  int k1, const short2* __restrict__ nzoff,
                                                  const float4* __restrict__ nzval,
                                                  float& ax, float& ay, float& az) {
  for (int k = k0; k < k1; k++) {
    const short2 o = nzoff[k];  // source = target - offset
    const float3 c = tile[base - o.x * TW - o.y];
    if (c.x == 0.f && c.y == 0.f && c.z == 0.f) continue;
    const float4 v = nzval[k];
    const float dx = c.x * v.x, dy = c.y * v.y, dz = c.z * v.z;
    ax += fminf(65025.f, dx * dx);
    ay += fminf(65025.f, dy * dy);
    az += fminf(65025.f, dz * dz);
  }
}

// The sprite entries up to its centre from the tile of `coef`, then the tile
// is reloaded with `coef_post` for the entries after the centre.
__global__ void __launch_bounds__(kDiffTX * kDiffTY)
k_diff_gather(const float3* __restrict__ coef, const float3* __restrict__ coef_post,
              const float* __restrict__ light, float* __restrict__ out, int M, int N,
              const short2* __restrict__ nzoff, const float4* __restrict__ nzval, int nsplit,
              int nnz, int H) {
  extern __shared__ float3 tile[];
  const int i0 = blockIdx.y * kDiffTY, j0 = blockIdx.x * kDiffTX;
  const int ti = i0 + threadIdx.y, tj = j0 + threadIdx.x;
  const bool in = ti < N && tj < M;
  const int TW = kDiffTX + 2 * H;
  const int base = (threadIdx.y + H) * TW + threadIdx.x + H;
  float ax = 0.f, ay = 0.f, az = 0.f;
  load_coef_tile(coef, M, N, i0, j0, H, tile);
  __syncthreads();
  if (in) diff_gather_range(tile, base, TW, 0, nsplit, nzoff, nzval, ax, ay, az);
  __syncthreads();
  load_coef_tile(coef_post, M, N, i0, j0, H, tile);
  __syncthreads();
  if (!in) return;
  diff_gather_range(tile, base, TW, nsplit, nnz, nzoff, nzval, ax, ay, az);
  const size_t t = (size_t)ti * M + tj;
  out[3 * t] = light[3 * t] + ax;
  out[3 * t + 1] = light[3 * t + 1] + ay;
  out[3 * t + 2] = light[3 * t + 2] + az;
}

// Footprint scale levels of the scaled gather: s_k = 0.25 * 2^(k/8).
constexpr int kPsfLevels = 33;
// Its output tiles are 32 x 32 (1024 threads): the halo of the largest
// footprints (~45 pixels) is shared by four times the pixels of a 32 x 8
// tile, and an SM keeps 32 warps resident.
constexpr int kDiffTYS = 32;

// The same with the sprite's footprint scaled at the receiving pixel by
// s = sqrt(magnification) (its camera-sky area over its celestial solid
// angle, as lensing uses), s clamped to [0.25, 4] and rounded to the nearest
// level s_k (9% steps): the term from offset o is the sprite sampled
// bilinearly at (centre + o / s_k) divided by s_k^2 -- a scale keeps the
// sprite's total light -- read from the level's precomputed entries.  The
// reference has no scaled footprint; every term of this one uses the
// source's light before any term is added (the coefficients of pass 1).
__global__ void __launch_bounds__(kDiffTX * kDiffTYS)
k_diff_gather_scaled(const float3* __restrict__ coef, const float* __restrict__ light,
                     float* __restrict__ out, int M, int N, const short2* __restrict__ lvoff,
                     const float4* __restrict__ lvval, const int* __restrict__ lvstart,
                     int maxlevel, int H, const float2* __restrict__ view,
                     const float* __restrict__ area) {
  extern __shared__ float3 tile[];
  const int i0 = blockIdx.y * kDiffTYS, j0 = blockIdx.x * kDiffTX;
  load_coef_tile(coef, M, N, i0, j0, H, tile, kDiffTYS);
  __syncthreads();
  const int ti = i0 + threadIdx.y, tj = j0 + threadIdx.x;
  if (ti >= N || tj >= M) return;
  const size_t t = (size_t)ti * M + tj;
  const int M1 = M + 1, ind = ti * M1 + tj;
  float ver4[4] = {view[ind].x, view[ind + 1].x, view[ind + M1 + 1].x, view[ind + M1].x};
  float hor4[4] = {view[ind].y, view[ind + 1].y, view[ind + M1 + 1].y, view[ind + M1].y};
  const float sa = area[t];
  const float mag = sa > 0.f ? calc_area(ver4, hor4) / sa : 1.f;
  // level of s = sqrt(mag): k = 8 log2(s / 0.25) = 4 log2(mag) + 16
  const float kf = mag > 0.f ? 4.f * log2f(mag) + 16.f : 0.f;
  const int k = imin(maxlevel, imax(0, (int)rintf(kf == kf ? kf : 16.f)));
  const int TW = kDiffTX + 2 * H;
  const int base = (threadIdx.y + H) * TW + threadIdx.x + H;
  float ax = 0.f, ay = 0.f, az = 0.f;
  for (int e = lvstart[k]; e < lvstart[k + 1]; e++) {
    const short2 o = lvoff[e];
    const float3 c = tile[base - o.x * TW - o.y];
    if (c.x == 0.f && c.y == 0.f && c.z == 0.f) continue;
    const float4 v = lvval[e];
    const float dx = c.x * v.x, dy = c.y * v.y, dz = c.z * v.z;
    ax += fminf(65025.f, dx * dx);
    ay += fminf(65025.f, dy * dy);
    az += fminf(65025.f, dz * dz);
  }
  out[3 * t] = light[3 * t] + ax;
  out[3 * t + 1] = light[3 * t + 1] + ay;
  out[3 * t + 2] = light[3 * t + 2] + az;
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

// Census of the star pass of the last frame, per pixel outside the shadow:
// the stars in the kd-tree nodes the search emits (the reference tests all
// of them, its starsToCheck) and the stars in the leaves left after the
// node-box pruning (the candidates tested here), and the stars that pass
// the quad test (hits, each placed in the pixel and splatted).  Sums into
// out[0..3]: pixels, reference candidates, candidates, hits; out[4..5]: the
// candidates and hits of the pixels with more than 2048 candidates.
__global__ void k_star_census(const float2* __restrict__ thphi, const uint8_t* __restrict__ bh,
                              StarSet S, Cam7 cam, int M, int N, int step,
                              const float2* __restrict__ view, int lr,
                              const float* __restrict__ area, unsigned long long* out) {
  const int j = blockIdx.x * TX + threadIdx.x;
  const int i = blockIdx.y * TY + threadIdx.y;
  unsigned long long px = 0, ref = 0, ours = 0, hits = 0, big_c = 0, big_h = 0;
  if (i < N && j < M) {
    PixelStars P;
    float mn[2], mx[2];
    if (pixel_setup(thphi, bh, cam.v, M, step, view, lr, area, i, j, P, mn, mx)) {
      px = 1;
      P.budget = 0x7fffffffffffL;
      tree_search(S, mn, mx, [&](int node) {
        int a0, a1;
        node_range(S, node, a0, a1);
        ref += (unsigned long long)(a1 - a0);
        walk_leaves(P, S, node, node_level(node), [&](int leaf) {
          int b0, b1;
          node_range(S, leaf, b0, b1);
          ours += (unsigned long long)(b1 - b0);
          for (int q = b0; q < b1; q++) {
            float st, sp;
            if (star_test(P, S, q, st, sp)) hits++;
          }
          return true;
        });
        return true;
      });
      if (ours > (unsigned long long)kStarBudget) {
        big_c = ours;
        big_h = hits;
      }
    }
  }
  for (int o = 16; o; o >>= 1) {
    px += __shfl_down_sync(0xffffffffu, px, o);
    ref += __shfl_down_sync(0xffffffffu, ref, o);
    ours += __shfl_down_sync(0xffffffffu, ours, o);
    hits += __shfl_down_sync(0xffffffffu, hits, o);
    big_c += __shfl_down_sync(0xffffffffu, big_c, o);
    big_h += __shfl_down_sync(0xffffffffu, big_h, o);
  }
  if ((threadIdx.x & 31) == 0 && px) {
    atomicAdd(out, px);
    atomicAdd(out + 1, ref);
    atomicAdd(out + 2, ours);
    atomicAdd(out + 3, hits);
    atomicAdd(out + 4, big_c);
    atomicAdd(out + 5, big_h);
  }
}

int map_star_census(const MapScratch& Sc, const MapFrame& F, unsigned long long* out,
                    cudaStream_t s) {
  const StarSet SS = stars_for_frame(F.stars, F.bb_table);
  k_star_census<<<grid2(Sc.M, Sc.N), dim3(TX, TY), 0, s>>>(
      Sc.thphi, Sc.bh, SS, F.cam, Sc.M, Sc.N, F.step, F.view, F.lr, Sc.area, out);
  BT_CUDA_TRY(cudaGetLastError());
  return BT_OK;
}

// The star cells of a splat of width fw: N*M*fw^2 float3, and at least two
// per pixel (the diffraction coefficients reuse them).
static int ensure_cells(MapScratch& Sc, int fw) {
  const size_t np = (size_t)Sc.M * Sc.N;
  if (Sc.cells && Sc.cells_fw >= fw) return BT_OK;
  if (Sc.cells) cudaFree(Sc.cells);
  Sc.cells = nullptr;
  Sc.cells_fw = 0;
  cudaError_t e = cudaMalloc((void**)&Sc.cells, np * imax(fw * fw, 2) * sizeof(float3));
  if (e != cudaSuccess) {
    set_error("star cell scratch allocation failed: %s", cudaGetErrorString(e));
    return BT_ERR_NOMEM;
  }
  Sc.cells_fw = fw;
  return BT_OK;
}

// addDiffraction (BT/MakeImageKernel.cu:775-800) of a star-light buffer
// (N*M*3 floats) into out (not the same buffer); the coefficients go into the
// star cells.  psf_scale: footprint scaled by the receiving pixel's
// magnification, from view and the smoothed solid angles `area`.
int map_diffract(MapScratch& Sc, const StarSet& SS, const float* light, float* out,
                 int psf_scale, const float2* view, const float* area, cudaStream_t s) {
  const int M = Sc.M, N = Sc.N;
  const size_t np = (size_t)M * N;
  if (int rc = ensure_cells(Sc, 1)) return rc;
  float3* coef = Sc.cells;
  float3* coef_post = Sc.cells + np;
  k_diff_coef<<<(unsigned)((np + 255) / 256), 256, 0, s>>>(light, (int)np, SS.psf_centre, coef,
                                                           coef_post);
  const dim3 dgrid((unsigned)((M + kDiffTX - 1) / kDiffTX), (unsigned)((N + kDiffTY - 1) / kDiffTY));
  const dim3 dblock(kDiffTX, kDiffTY);
  constexpr int kMaxHalo = 52;  // (8 + 104) x (32 + 104) float3 = 183 KB of shared memory
  auto tile_bytes = [](int H, int ty = kDiffTY) {
    return (size_t)(kDiffTX + 2 * H) * (ty + 2 * H) * sizeof(float3);
  };
  if (psf_scale && SS.psf_lvstart) {
    // the highest level whose footprint fits the shared-memory halo
    int maxlevel = kPsfLevels - 1;
    while (maxlevel > 0 &&
           (int)ceilf(imax(1, SS.psf_rnz) * 0.25f * exp2f(maxlevel / 8.f)) + 1 > kMaxHalo)
      maxlevel--;
    const int H = imin(kMaxHalo, (int)ceilf(imax(1, SS.psf_rnz) * 0.25f * exp2f(maxlevel / 8.f)) + 1);
    BT_CUDA_TRY(cudaFuncSetAttribute(k_diff_gather_scaled,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)tile_bytes(H, kDiffTYS)));
    const dim3 sgrid((unsigned)((M + kDiffTX - 1) / kDiffTX),
                     (unsigned)((N + kDiffTYS - 1) / kDiffTYS));
    k_diff_gather_scaled<<<sgrid, dim3(kDiffTX, kDiffTYS), tile_bytes(H, kDiffTYS), s>>>(
        coef, light, out, M, N, SS.psf_lvoff, SS.psf_lvval, SS.psf_lvstart, maxlevel, H, view,
        area);
  } else if (SS.psf_rnz <= kMaxHalo) {
    const int H = imax(1, SS.psf_rnz);
    BT_CUDA_TRY(cudaFuncSetAttribute(k_diff_gather, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)tile_bytes(kMaxHalo)));
    k_diff_gather<<<dgrid, dblock, tile_bytes(H), s>>>(coef, coef_post, light, out, M, N,
                                                       SS.psf_nzoff, SS.psf_nzval, SS.psf_nsplit,
                                                       SS.psf_nnz, H);
  } else {
    // sprites wider than the shared-memory halo: scatter with atomics
    BT_CUDA_TRY(cudaMemcpyAsync(out, light, np * 3 * sizeof(float), cudaMemcpyDeviceToDevice, s));
    BT_CUDA_TRY(cudaMemsetAsync(Sc.diff_count, 0, sizeof(uint32_t), s));
    k_diff_mark<<<(unsigned)((np + 255) / 256), 256, 0, s>>>(light, (int)np, Sc.diff_list,
                                                            Sc.diff_count);
    k_diff_scatter<<<sm_count() * 8, 256, 0, s>>>(light, out, Sc.diff_list, Sc.diff_count, M, N,
                                                  SS.psf, SS.psf_size);
  }
  BT_CUDA_TRY(cudaGetLastError());
  return BT_OK;
}

int map_diffract_light(MapScratch& Sc, const bt_stars* stars, const float* light, float* out,
                       cudaStream_t s) {
  const StarSet& SS = stars->s;
  if (!SS.psf || SS.psf_size <= 0) {
    set_error("invalid argument: the star set has no diffraction sprite");
    return BT_ERR_ARG;
  }
  return map_diffract(Sc, SS, light, out, 0, nullptr, nullptr, s);
}

int map_run_stars(MapScratch& Sc, const MapFrame& F, cudaStream_t s) {
  const int M = Sc.M, N = Sc.N;
  const StarSet SS = stars_for_frame(F.stars, F.bb_table);
  const int fw = 2 * F.step + 1;
  if (F.step > 2) {
    set_error("star splat step > 2 is not supported");
    return BT_ERR_ARG;
  }
  if (int rc = ensure_cells(Sc, fw)) return rc;
  if (int rc = ensure_units(Sc, fw)) return rc;
  BT_CUDA_TRY(cudaMemsetAsync(Sc.heavy_count, 0, kHcWords * sizeof(uint32_t), s));
  k_star_cells<<<grid2(M, N), dim3(TX, TY), 0, s>>>(
      Sc.thphi, Sc.bh, SS, F.cam, M, N, F.step, F.view, F.lr, Sc.area,
      Sc.cells, Sc.flag, Sc.heavy_list, Sc.heavy_count + kHcDeferred);
  // deferred pixels: in units of candidate leaves, the pixels past the node
  // pool in k_star_heavy
  k_hv_count<<<sm_count() * 2, 128, 0, s>>>(Sc.thphi, Sc.bh, SS, F.cam, M, F.step, F.view,
                                            F.lr, Sc.area, Sc.heavy_list, Sc.heavy_count,
                                            Sc.hv_nn, Sc.hv_nl, Sc.hv_slab, Sc.hv_slab_pixels);
  k_hv_scan<<<1, 1024, 0, s>>>(Sc.heavy_list, Sc.heavy_count, Sc.hv_nn, Sc.hv_nl, Sc.hv_noff,
                               Sc.hv_uoff, Sc.heavy_order, Sc.hv_ctl,
                               (uint32_t)std::min<size_t>(Sc.hv_node_cap, 0xffffffffu),
                               (uint32_t)std::min<size_t>(Sc.hv_unit_cap, 0xffffffffu));
  k_hv_nodes<<<sm_count() * 2, 128, 0, s>>>(Sc.thphi, Sc.bh, SS, F.cam, M, F.step, F.view,
                                            F.lr, Sc.area, Sc.heavy_list, Sc.heavy_count,
                                            Sc.hv_noff, Sc.hv_slab, Sc.hv_slab_pixels,
                                            Sc.hv_pool, Sc.hv_pend);
  if (F.step == 0) launch_units<0>(Sc, F, SS, s);
  else if (F.step == 1) launch_units<1>(Sc, F, SS, s);
  else launch_units<2>(Sc, F, SS, s);
  if (F.step == 0) launch_heavy<0>(Sc, F, SS, s);
  else if (F.step == 1) launch_heavy<1>(Sc, F, SS, s);
  else launch_heavy<2>(Sc, F, SS, s);
  BT_CUDA_TRY(cudaGetLastError());
  const float* trail = nullptr;
  if (F.trails) {
    if (int rc = trails_run(F.trails, Sc, F, SS, s)) return rc;
    trail = trails_buffer(F.trails);
  }
  const bool diff = F.diffraction && SS.psf && SS.psf_size > 0;
  if (!diff) {
    if (F.bg_ready) BT_CUDA_TRY(cudaStreamWaitEvent(s, F.bg_ready, 0));
    k_star_gather<true><<<grid2(M, N), dim3(TX, TY), 0, s>>>(
        Sc.cells, Sc.flag, M, N, F.step, Sc.light, (const uchar4*)F.out_bg,
        (uchar4*)F.out, F.map, trail);
    BT_CUDA_TRY(cudaGetLastError());
    return BT_OK;
  }
  k_star_gather<false><<<grid2(M, N), dim3(TX, TY), 0, s>>>(
      Sc.cells, Sc.flag, M, N, F.step, Sc.light, nullptr, nullptr, F.map, trail);
  // the star cells are consumed: their buffer holds the coefficients
  if (int rc = map_diffract(Sc, SS, Sc.light, Sc.light2, F.psf_scale, F.view, Sc.area, s))
    return rc;
  if (F.bg_ready) BT_CUDA_TRY(cudaStreamWaitEvent(s, F.bg_ready, 0));
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

// Bounding box of every node's stars (theta_min, phi_min, theta_max,
// phi_max), leaves from their star ranges, inner nodes from their children.
// NaN coordinates are left out: the quad test rejects such stars.  Returns
// false when the tree's cumulative counts do not describe ranges inside
// [0, n) -- the kernels would read past the star arrays.
bool node_boxes(const float* pos, int n, const int* tree, int L,
                std::vector<float4>& box) {
  const size_t nodes = ((size_t)2 << L) - 1;
  const float inf = std::numeric_limits<float>::infinity();
  box.assign(nodes, make_float4(inf, inf, -inf, -inf));
  const size_t first = ((size_t)1 << L) - 1;
  int prev = 0;
  for (size_t k = first; k < nodes; k++) {
    const int start = k == first ? 0 : prev;
    const int end = tree[k];
    if (end < start || end > n) return false;
    prev = end;
    float4 b = box[k];
    for (int q = start; q < end; q++) {
      const float t = pos[2 * (size_t)q], p = pos[2 * (size_t)q + 1];
      if (t != t || p != p) continue;
      b.x = std::min(b.x, t); b.y = std::min(b.y, p);
      b.z = std::max(b.z, t); b.w = std::max(b.w, p);
    }
    box[k] = b;
  }
  for (size_t k = first; k-- > 0;) {
    const float4 a = box[2 * k + 1], c = box[2 * k + 2];
    box[k] = make_float4(std::min(a.x, c.x), std::min(a.y, c.y), std::max(a.z, c.z),
                         std::max(a.w, c.w));
  }
  return true;
}

// The sprite resampled at the footprint scales s_k = 0.25 * 2^(k/8),
// k = 0..kPsfLevels-1 (StarSet::psf_lvoff): level k lists the offsets
// (dq, dp) within R_k = ceil(max(1, rnz) s_k) + 1 of the centre whose
// bilinear sample of the sprite at (centre + offset / s_k), divided by s_k^2,
// is non-zero in some channel; level k is [lvstart[k], lvstart[k + 1]).
void psf_levels(const uint8_t* psf_rgb, int psf_size, int rnz, std::vector<short2>& lvoff,
                std::vector<float4>& lvval, std::vector<int>& lvstart) {
  lvoff.clear();
  lvval.clear();
  lvstart.assign(1, 0);
  if (psf_size < 2) return;
  const float c0 = (float)(psf_size / 2);
  auto px = [&](int q, int p, int ch) {
    return (float)psf_rgb[((size_t)q * psf_size + p) * 3 + ch];
  };
  for (int k = 0; k < kPsfLevels; k++) {
    const float sc = 0.25f * std::exp2((float)k / 8.f), is = 1.f / sc;
    const int R = (int)std::ceil(std::max(1, rnz) * sc) + 1;
    for (int dq = -R; dq <= R; dq++)
      for (int dp = -R; dp <= R; dp++) {
        const float u = c0 + dq * is, v = c0 + dp * is;
        if (u < 0.f || v < 0.f || u > psf_size - 1 || v > psf_size - 1) continue;
        const int u0 = std::min((int)u, psf_size - 2), v0 = std::min((int)v, psf_size - 2);
        const float fu = u - u0, fv = v - v0;
        float val[3];
        for (int ch = 0; ch < 3; ch++)
          val[ch] = ((1 - fu) * (1 - fv) * px(u0, v0, ch) + (1 - fu) * fv * px(u0, v0 + 1, ch) +
                     fu * (1 - fv) * px(u0 + 1, v0, ch) + fu * fv * px(u0 + 1, v0 + 1, ch)) *
                    is * is;
        if (val[0] == 0.f && val[1] == 0.f && val[2] == 0.f) continue;
        lvoff.push_back(make_short2((short)dq, (short)dp));
        lvval.push_back(make_float4(val[0], val[1], val[2], 0.f));
      }
    lvstart.push_back((int)lvoff.size());
  }
}

}  // namespace

extern "C" {

int bt_stars_tree_size(int treeLevel) { return (1 << (treeLevel + 1)) - 1; }

int bt_psf_levels(const uint8_t* psf_rgb, int psf_size, int level, int16_t* offsets,
                  float* values, int capacity, int* count) {
  clear_error();
  BT_ARG_CHECK(psf_rgb && count && psf_size >= 2, "invalid sprite");
  BT_ARG_CHECK(level >= 0 && level < kPsfLevels, "level must be in [0, 32]");
  int rnz = 0;
  for (int q = 0; q < psf_size; q++)
    for (int p = 0; p < psf_size; p++) {
      const uint8_t* v = psf_rgb + ((size_t)q * psf_size + p) * 3;
      if (v[0] || v[1] || v[2])
        rnz = std::max(rnz, std::max(std::abs(q - psf_size / 2), std::abs(p - psf_size / 2)));
    }
  std::vector<short2> off;
  std::vector<float4> val;
  std::vector<int> start;
  psf_levels(psf_rgb, psf_size, rnz, off, val, start);
  const int n = start[level + 1] - start[level];
  *count = n;
  if (!offsets || !values || capacity < n) return BT_OK;
  for (int e = 0; e < n; e++) {
    const short2 o = off[start[level] + e];
    const float4 v = val[start[level] + e];
    offsets[2 * e] = o.x;
    offsets[2 * e + 1] = o.y;
    values[3 * e] = v.x;
    values[3 * e + 1] = v.y;
    values[3 * e + 2] = v.z;
  }
  return BT_OK;
}

int bt_stars_blackbody(const bt_stars* st, int table, float* hsp, float* rgb, int capacity,
                       int* count, void* stream) {
  clear_error();
  BT_ARG_CHECK(st && count, "NULL pointer");
  BT_ARG_CHECK(table == 0 || table == 1, "table must be 0 (391 entries) or 1 (1024)");
  const int n = table ? kBlackbody1k : kBlackbodyEntries;
  *count = n;
  if (!hsp || !rgb || capacity < n) return BT_OK;
  const float4* dev = table ? st->bb1k : st->bb;
  std::vector<float4> h(2 * (size_t)n);
  cudaStream_t s = (cudaStream_t)stream;
  BT_CUDA_TRY(cudaMemcpyAsync(h.data(), dev, 2 * n * sizeof(float4), cudaMemcpyDeviceToHost, s));
  BT_CUDA_TRY(cudaStreamSynchronize(s));
  for (int k = 0; k < n; k++) {
    hsp[3 * k] = h[k].x; hsp[3 * k + 1] = h[k].y; hsp[3 * k + 2] = h[k].z;
    rgb[3 * k] = h[n + k].x; rgb[3 * k + 1] = h[n + k].y; rgb[3 * k + 2] = h[n + k].z;
  }
  return BT_OK;
}

int bt_psf_airy(int size, float first_zero, uint8_t* rgb) {
  clear_error();
  BT_ARG_CHECK(rgb && size >= 3 && size <= 1025 && (size & 1) && first_zero > 0.f,
               "invalid sprite arguments (odd size in [3, 1025], first_zero > 0)");
  // first zero of J1 at x = 3.8317...; channel wavelengths relative to 550 nm
  const double j1z = 3.8317059702075123, lam[3] = {610. / 550., 550. / 550., 465. / 550.};
  const int h = size / 2;
  for (int y = 0; y < size; y++)
    for (int x = 0; x < size; x++) {
      const double r = std::sqrt((double)(x - h) * (x - h) + (double)(y - h) * (y - h));
      for (int c = 0; c < 3; c++) {
        const double z = j1z * r / (first_zero * lam[c]);
        const double I = z < 1e-9 ? 1.0 : std::pow(2.0 * std::cyl_bessel_j(1.0, z) / z, 2.0);
        // RGB order, as the reference loads its sprite (stbi_load,
        // BT/MakeImageKernel.cu:1281-1286): channel c scales star light c
        rgb[((size_t)y * size + x) * 3 + c] = (uint8_t)std::lround(255.0 * I);
      }
    }
  return BT_OK;
}

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
  std::vector<float4> box;
  if (!node_boxes(star_pos, n, tree, treeLevel, box)) {
    delete st;
    set_error("invalid argument: the star tree's counts do not match %d stars", n);
    return BT_ERR_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaMalloc((void**)&st->pos, (size_t)2 * n * sizeof(float) + 16);
  if (e == cudaSuccess) e = cudaMalloc((void**)&st->mag, (size_t)2 * n * sizeof(float) + 16);
  if (e == cudaSuccess) e = cudaMalloc((void**)&st->tree, tsize * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc((void**)&st->box, box.size() * sizeof(float4));
  if (e == cudaSuccess) e = cudaMalloc((void**)&st->bb, 2 * kBlackbodyEntries * sizeof(float4));
  if (e == cudaSuccess) e = cudaMalloc((void**)&st->bb1k, 2 * kBlackbody1k * sizeof(float4));
  if (e == cudaSuccess) {
    k_blackbody_tables<<<(kBlackbodyEntries + 127) / 128, 128, 0, s>>>(st->bb);
    k_blackbody_tables_1k<<<kBlackbody1k / 128, 128, 0, s>>>(st->bb1k);
    e = cudaGetLastError();
  }
  // the sprite's non-zero entries, offsets from its centre (index size/2)
  std::vector<short2> nzoff;
  std::vector<float4> nzval;
  int rnz = 0, nsplit = 0;
  float4 centre = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int q = 0; q < psf_size; q++)
    for (int p = 0; p < psf_size; p++) {
      const uint8_t* v = psf_rgb + ((size_t)q * psf_size + p) * 3;
      const int dq = q - psf_size / 2, dp = p - psf_size / 2;
      if (dq == 0 && dp == 0) centre = make_float4((float)v[0], (float)v[1], (float)v[2], 0.f);
      if (!v[0] && !v[1] && !v[2]) continue;
      nzoff.push_back(make_short2((short)dq, (short)dp));
      nzval.push_back(make_float4((float)v[0], (float)v[1], (float)v[2], 0.f));
      if (dq < 0 || (dq == 0 && dp <= 0)) nsplit = (int)nzoff.size();
      rnz = std::max(rnz, std::max(std::abs(dq), std::abs(dp)));
    }
  // resampled levels for the magnification-scaled footprint
  std::vector<short2> lvoff;
  std::vector<float4> lvval;
  std::vector<int> lvstart(1, 0);
  psf_levels(psf_rgb, psf_size, rnz, lvoff, lvval, lvstart);
  if (e == cudaSuccess && psf_size)
    e = cudaMalloc((void**)&st->psf, (size_t)psf_size * psf_size * 3);
  if (e == cudaSuccess && !lvoff.empty()) {
    e = cudaMalloc((void**)&st->psf_lvoff, lvoff.size() * sizeof(short2));
    if (e == cudaSuccess) e = cudaMalloc((void**)&st->psf_lvval, lvval.size() * sizeof(float4));
    if (e == cudaSuccess) e = cudaMalloc((void**)&st->psf_lvstart, lvstart.size() * sizeof(int));
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(st->psf_lvoff, lvoff.data(), lvoff.size() * sizeof(short2),
                          cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(st->psf_lvval, lvval.data(), lvval.size() * sizeof(float4),
                          cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(st->psf_lvstart, lvstart.data(), lvstart.size() * sizeof(int),
                          cudaMemcpyHostToDevice, s);
  }
  if (e == cudaSuccess && !nzoff.empty())
    e = cudaMalloc((void**)&st->psf_nzoff, nzoff.size() * sizeof(short2));
  if (e == cudaSuccess && !nzoff.empty())
    e = cudaMalloc((void**)&st->psf_nzval, nzval.size() * sizeof(float4));
  if (e == cudaSuccess && !nzoff.empty())
    e = cudaMemcpyAsync(st->psf_nzoff, nzoff.data(), nzoff.size() * sizeof(short2),
                        cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && !nzoff.empty())
    e = cudaMemcpyAsync(st->psf_nzval, nzval.data(), nzval.size() * sizeof(float4),
                        cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(st->box, box.data(), box.size() * sizeof(float4),
                        cudaMemcpyHostToDevice, s);
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
    cudaFree(st->pos); cudaFree(st->mag); cudaFree(st->tree); cudaFree(st->box);
    cudaFree(st->bb); cudaFree(st->bb1k); cudaFree(st->psf);
    cudaFree(st->psf_nzoff); cudaFree(st->psf_nzval);
    cudaFree(st->psf_lvoff); cudaFree(st->psf_lvval); cudaFree(st->psf_lvstart);
    delete st;
    set_error("star set upload failed: %s", cudaGetErrorString(e));
    return BT_ERR_CUDA;
  }
  st->s.n = n;
  st->s.treeLevel = treeLevel;
  st->s.pos = st->pos;
  st->s.mag = st->mag;
  st->s.tree = st->tree;
  st->s.box = st->box;
  st->s.bb_hsp = st->bb;
  st->s.bb_rgb = st->bb + kBlackbodyEntries;
  st->s.bb_n = kBlackbodyEntries;
  st->s.psf = st->psf;
  st->s.psf_size = psf_size;
  st->s.psf_nzoff = st->psf_nzoff;
  st->s.psf_nzval = st->psf_nzval;
  st->s.psf_nnz = (int)nzoff.size();
  st->s.psf_rnz = rnz;
  st->s.psf_nsplit = nsplit;
  st->s.psf_centre = centre;
  st->s.psf_lvoff = st->psf_lvoff;
  st->s.psf_lvval = st->psf_lvval;
  st->s.psf_lvstart = st->psf_lvstart;
  *out = st;
  return BT_OK;
}

void bt_stars_destroy(bt_stars* st) {
  if (!st) return;
  cudaFree(st->pos);
  cudaFree(st->mag);
  cudaFree(st->tree);
  cudaFree(st->box);
  cudaFree(st->bb);
  cudaFree(st->bb1k);
  if (st->psf) cudaFree(st->psf);
  cudaFree(st->psf_nzoff);
  cudaFree(st->psf_nzval);
  cudaFree(st->psf_lvoff);
  cudaFree(st->psf_lvval);
  cudaFree(st->psf_lvstart);
  delete st;
}

}  // extern "C"
