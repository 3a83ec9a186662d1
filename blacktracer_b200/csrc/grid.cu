// grid.cu -- the adaptive camera-sky grid, built on the device.
//
// Replaces Grid::Grid (annemiekie/BlackTracer BT/Grid.h:605-624): raytrace,
// integrateFirst, adaptiveBlockIntegration (level-synchronous refinement,
// :291-505), fixTvertices (:103-204) and the GPU hand-off (saveAsGpuHash
// :642 + makeGrid, BT/MakeImageKernel.cu:369-384).
//
// The reference keeps the grid in hash maps keyed by i<<32|j.  Here it is a
// dense N x M lattice in HBM (vertex (i,j) at i*M+j): vflag marks the keys
// the map would hold, blevel the block levels.  Refinement is one kernel per
// level over the level's block list; new vertices are deduplicated with an
// atomicCAS on vflag (the reference's set semantics), appended to a trace
// list and integrated by the persistent trace kernel.  No step needs the
// host: every launch reads its work count from device memory, so a whole
// build is asynchronous and graph-capturable.
//
// Grids are built in sets (bt_batch): G grids of the same size, each with
// its own camera and spin, advance through the levels together -- every
// build kernel covers all G grids (blockIdx.y = grid), and each level's rays
// of all grids go through one persistent trace launch with a shared work
// queue, so that the long rays of one grid overlap the work of the others.
// A lone grid (bt_grid_create) is a set of one.  The launch sequence of a
// set depends only on its shape, start level, precision and trace launch
// shape, so it can be captured once as a CUDA graph and replayed; cameras
// and spins reach the kernels through device-resident descriptors.
//
// The T-vertex fix of the reference iterates an unordered_map, so its result
// depends on the hash table's iteration order.  This build fixes blocks in a
// canonical order -- level ascending, then key i<<32|j ascending, then edge
// (left, top, right, bottom) -- and computes that sequential result in
// parallel: per level, every edge is fixed by one thread; a value owned by an
// edge that precedes the reader in the canonical order is taken from the
// previous pass, any other foreign value from the level's input.  Because a
// fix only reads the near ends of its collinear neighbours, a few passes
// reach the fixed point, which is exactly the sequential result.
//
// Compiled with --fmad=false (the fix's FP64 Hermite must round like the
// reference's host build).
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "bt_internal.h"
#include "grid_flow.cuh"

namespace bt {

constexpr int kMaxTfixPasses = 8;
constexpr int kParamSlots = 2;  // pinned descriptor staging slots

}  // namespace bt

struct bt_batch;

struct bt_grid {
  bt_batch* set;               // the build set this grid belongs to
  int index;                   // position in the set
  bt::LatticeView L;           // slices of the set's arrays
  bt::GridCounters* ctr;       // device (slice)
  bt::GridCounters* ctr_host;  // pinned mirror (slice)
  bt::RayParams params;
  bt_camera cam;
  double a;
  int built;
  float2* mapgrid;  // float2 export for the map (lazy)
  uint32_t* rowv;   // compact export: per-row vertex / block counts + totals
  uint32_t* rowb;
  uint64_t* totals;
  uint64_t* totals_host;
  char* compact;    // compact export staging (device), lazily sized
  size_t compact_bytes;
  int32_t map_rows;
  int sym;
};

struct bt_batch {
  int G, N, M, eq, maxlevel;
  size_t NM;
  int standalone;  // created by bt_grid_create (a set of one)
  bt_grid* grids;
  // arrays of all members; member g at offset g*NM (lists: 4 per member,
  // fix buffers: 2 per member)
  double2* thphi;
  int32_t* steps;
  uint8_t* vflag;
  uint8_t* vstat;
  int8_t* blevel;
  uint32_t* lists;
  double2* X;
  bt::GridCounters* ctr;
  bt::GridCounters* ctr_host;
  bt::GridDesc* D;        // device descriptors
  bt::GridDesc* Dh[bt::kParamSlots];  // pinned staging
  cudaEvent_t Dev[bt::kParamSlots];   // staging slot reusable once passed
  int slot;
  uint32_t* qoff;         // G + 1
  uint32_t* qfetch;
  bt::TraceShape shape;
  int startlevel, precision;
  int launches;           // kernels of the last build
  int built;
  int built_n;            // members built by the last build (the first built_n)
  // timing of the trace launches (eager builds only)
  int timing;
  cudaEvent_t ev[2 * 16];
  int n_ev;
  // graph replay
  int graph;
  cudaStream_t cap_stream;
  cudaGraphExec_t exec;
  int exec_n, exec_startlevel, exec_precision, exec_tfix_passes;
  bt::TraceShape exec_shape;
  // Jacobi passes of the T-vertex fix per level (kMaxTfixPasses unless a
  // test lowers it with bt_grid_set_tfix_passes)
  int tfix_passes;
  // 1: the fix of a level as one cooperative launch when the set fits the
  // device at once (k_tfix_level); 0: a launch per pass (bt_grid_set_tfix_launch)
  int tfix_coop, exec_tfix_coop;
  // the refinement levels as one persistent launch (bt_batch_set_flow; flow =
  // its blocks per SM, 0 = off): its check, hot-trace and hot-set-up queues
  // (G*NM slots each), block bytes (G*NM per level below the max that blocks
  // wait on, flow_bw_levels of them) and control block; the set-up and trace
  // queues and the sync words reuse the block lists
  int flow, exec_flow;
  int flow_bw_levels;
  int flow_early;  // refine blocks early in the flow (on unless a test turns it off)
  int flow_drop;  // diagnostic: the next flow build loses one ray (bt_grid_set_flow_drop)
  // set-wide "changed" flag per T-vertex pass of k_tfix_level (16 words)
  uint32_t* tfix_changed;
  uint32_t* flow_q;
  uint8_t* flow_bw;
  bt::FlowCtl* flow_ctl;
};

namespace bt {

__device__ __forceinline__ uint32_t pow2u(int e) { return 1u << e; }

// ------------------------------------------------------------ seeding
// raytrace + integrateFirst (BT/Grid.h:291-338): the poles, the start-level
// lattice and the first block list.
//   trace list: [north pole, south pole if eq, rows i = gap..(<N-eq) x cols]
//   check list: [top-row blocks (0, j)], then the blocks of rows i != N-1
//   (none when maxlevel == startlevel: those get blevel = startlevel here).
struct SeedShape {
  uint32_t gap, cols, rows, brows, npole;
};

static SeedShape seed_shape(const LatticeView& L) {
  SeedShape s;
  s.gap = 1u << (L.maxlevel - L.startlevel);
  s.cols = (uint32_t)L.M / s.gap;
  s.rows = ((uint32_t)L.N - (uint32_t)L.eq - 1u) / s.gap;  // i in [gap, N-eq)
  s.brows = L.eq ? s.rows : s.rows - 1;  // the equator row N-1 has no block
  s.npole = L.eq ? 2 : 1;
  return s;
}

__global__ void k_seed(const GridDesc* __restrict__ D, SeedShape S) {
  const GridDesc& d = D[blockIdx.y];
  const LatticeView L = d.L;
  uint32_t* trace = d.trace;
  uint32_t* check = d.list[0];
  GridCounters* ctr = d.ctr;
  const uint32_t M = L.M;
  const bool uniform = L.maxlevel == L.startlevel;
  const uint32_t total = S.rows * S.cols;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total + S.cols;
       t += gridDim.x * blockDim.x) {
    if (t < S.cols) {
      check[t] = t * S.gap;
      continue;
    }
    const uint32_t q = t - S.cols;
    const uint32_t r = q / S.cols;
    const uint32_t i = S.gap * (1 + r), j = S.gap * (q % S.cols);
    const uint32_t key = i * M + j;
    trace[S.npole + q] = key;
    L.vflag[key] = 2;
    if (r < S.brows) {
      if (uniform) L.blevel[key] = (int8_t)L.startlevel;
      else check[S.cols + q] = key;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    trace[0] = 0;
    L.vflag[0] = 2;
    if (L.eq) {
      trace[1] = ((uint32_t)L.N - 1) * M;
      L.vflag[((uint32_t)L.N - 1) * M] = 2;
    }
    ctr->n_trace = S.npole + total;
    ctr->n_hot = S.npole + total;
    ctr->n_cold = 0;
    ctr->n_check = S.cols + (uniform ? 0 : S.brows * S.cols);
    ctr->n_next = 0;
    ctr->fetch = 0;
    ctr->tfix_flags[1] = 1;
  }
}

// Pole copies of raytrace (BT/Grid.h:303-315), after the poles are traced.
__global__ void k_pole_copy(const GridDesc* __restrict__ D) {
  const LatticeView L = D[blockIdx.y].L;
  const uint32_t gap = pow2u(L.maxlevel - L.startlevel);
  const uint32_t M = L.M, N = L.N;
  for (uint32_t j = (blockIdx.x * blockDim.x + threadIdx.x) * gap; j < M;
       j += gridDim.x * blockDim.x * gap) {
    if (j == 0) continue;
    L.thphi[j] = L.thphi[0];
    L.steps[j] = L.steps[0];
    L.vstat[j] = L.vstat[0];
    L.vflag[j] = 1;
    if (L.eq) {
      const size_t s0 = (size_t)(N - 1) * M;
      L.thphi[s0 + j] = L.thphi[s0];
      L.steps[s0 + j] = L.steps[0];  // the reference copies steps[0] (:312)
      L.vstat[s0 + j] = L.vstat[s0];
      L.vflag[s0 + j] = 1;
    }
  }
}

// Queue offsets of the next trace launch: qoff[g] = rays of grids < g.
__global__ void k_queue(const GridDesc* __restrict__ D, int G, uint32_t* qoff,
                        uint32_t* qfetch) {
  __shared__ uint32_t s[1024];
  const int t = threadIdx.x, T = blockDim.x;
  uint32_t carry = 0;
  for (int base = 0; base < G; base += T) {
    const uint32_t v = base + t < G ? *(volatile uint32_t*)&D[base + t].ctr->n_trace : 0u;
    s[t] = v;
    __syncthreads();
    for (int o = 1; o < T; o <<= 1) {
      const uint32_t a = t >= o ? s[t - o] : 0u;
      __syncthreads();
      s[t] += a;
      __syncthreads();
    }
    if (base + t < G) qoff[base + t + 1] = carry + s[t];
    carry += s[T - 1];
    __syncthreads();
  }
  if (t == 0) {
    qoff[0] = 0;
    *qfetch = 0;
  }
}

// ------------------------------------------------------------ refinement
// A hot new vertex (kHotSteps) goes to the front of the trace list, else to
// the back: the trace kernel takes the front first, so the longest rays of a
// level start first instead of whenever a lane happens to reach them.  The
// order changes no result.

__device__ __forceinline__ void claim_vertex(const LatticeView& L, uint32_t i,
                                             uint32_t j, uint32_t* trace,
                                             GridCounters* ctr, bool hot) {
  const uint32_t key = i * (uint32_t)L.M + j;
  // 32-bit CAS on the aligned word that holds the byte
  uint32_t* word = (uint32_t*)((uintptr_t)(L.vflag + key) & ~(uintptr_t)3);
  const uint32_t sh = ((uintptr_t)(L.vflag + key) & 3) * 8;
  uint32_t old = *(volatile uint32_t*)word;
  for (;;) {
    if ((old >> sh) & 0xffu) return;  // exists or already claimed
    const uint32_t nw = old | (2u << sh);
    const uint32_t got = atomicCAS(word, old, nw);
    if (got == old) break;
    old = got;
  }
  atomicAdd(&ctr->n_trace, 1u);
  if (hot) {
    trace[atomicAdd(&ctr->n_hot, 1u)] = key;
  } else {
    const uint32_t cap = (uint32_t)L.N * (uint32_t)L.M;
    trace[cap - 1u - atomicAdd(&ctr->n_cold, 1u)] = key;
  }
}

// One level of adaptiveBlockIntegration (BT/Grid.h:476-497) with
// refineCheck (:410-445) and fillVector (:453-459).
__global__ void k_refine(const GridDesc* __restrict__ D, int level, int cur) {
  const GridDesc& d = D[blockIdx.y];
  const LatticeView L = d.L;
  const uint32_t* check = d.list[cur];
  uint32_t* next = d.list[cur ^ 1];
  uint32_t* trace = d.trace;
  uint32_t* leaves = d.leaves;
  GridCounters* ctr = d.ctr;
  const uint32_t n = *(volatile uint32_t*)&ctr->n_check;
  const uint32_t M = L.M;
  const uint32_t gap = pow2u(L.maxlevel - level);
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += gridDim.x * blockDim.x) {
    const uint32_t key = check[t];
    const uint32_t i = key / M, j = key % M;
    const uint32_t k = i + gap, l = (j + gap) % M;
    const double2 v1 = L.thphi[(size_t)i * M + j];
    const double2 v2 = L.thphi[(size_t)k * M + j];
    const double2 v3 = L.thphi[(size_t)i * M + l];
    const double2 v4 = L.thphi[(size_t)k * M + l];
    const double diag = (v1.x - v4.x) * (v1.x - v4.x) + (v1.y - v4.y) * (v1.y - v4.y);
    const double diag2 = (v2.x - v3.x) * (v2.x - v3.x) + (v2.y - v3.y) * (v2.y - v3.y);
    const double mx = diag < diag2 ? diag2 : diag;  // std::max
    const bool refine = (level < 6 && mx > 1E-10) || (mx > 0.015);
    if (!refine) {
      L.blevel[key] = (int8_t)level;
      const uint32_t s = atomicAdd(&ctr->n_leaf, 1u);
      leaves[s] = key;
      continue;
    }
    const uint32_t kh = i + gap / 2, lh = j + gap / 2;
    const int32_t smax = max(max(L.steps[(size_t)i * M + j], L.steps[(size_t)k * M + j]),
                             max(L.steps[(size_t)i * M + l], L.steps[(size_t)k * M + l]));
    const bool hot = smax >= kHotSteps;
    claim_vertex(L, kh, j, trace, ctr, hot);
    claim_vertex(L, kh, lh, trace, ctr, hot);
    claim_vertex(L, i, lh, trace, ctr, hot);
    claim_vertex(L, i + gap, lh, trace, ctr, hot);
    claim_vertex(L, kh, (j + gap) % M, trace, ctr, hot);
    const uint32_t s = atomicAdd(&ctr->n_next, 4u);
    next[s + 0] = key;
    next[s + 1] = kh * M + j;
    next[s + 2] = kh * M + lh;
    next[s + 3] = i * M + lh;
  }
}

// Level hand-over, one thread per grid.  after_seed: only account the
// seeded rays; otherwise the next list becomes the check list and the leaf
// offset of `slot` is set.
__global__ void k_advance(const GridDesc* __restrict__ D, int G, int after_seed, int slot) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G) return;
  GridCounters* ctr = D[g].ctr;
  uint64_t t = ((uint64_t)ctr->traced_hi << 32 | ctr->traced_lo) + ctr->n_trace;
  ctr->traced_lo = (uint32_t)t;
  ctr->traced_hi = (uint32_t)(t >> 32);
  ctr->n_trace = 0;
  ctr->n_hot = 0;
  ctr->n_cold = 0;
  ctr->fetch = 0;
  if (!after_seed) {
    ctr->n_check = ctr->n_next;
    ctr->n_next = 0;
  }
  if (slot >= 0 && slot < 16) ctr->leaf_off[slot] = ctr->n_leaf;
}

// Blocks left at the last level get level = MAXLEVEL (BT/Grid.h:503-504).
__global__ void k_finalize(const GridDesc* __restrict__ D, int cur) {
  const GridDesc& d = D[blockIdx.y];
  const uint32_t n = *(volatile uint32_t*)&d.ctr->n_check;
  const uint32_t* check = d.list[cur];
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += gridDim.x * blockDim.x)
    d.L.blevel[check[t]] = (int8_t)d.L.maxlevel;
}

// ------------------------------------------------------------ T-vertex fix
struct TfixArgs {
  LatticeView L;
  int level;
  int pass;
  const uint32_t* leaves;
  uint32_t lo, hi_slot;  // leaf range: [leaf_off[lo], leaf_off[hi_slot])
  double2* Xcur;
  const double2* Xprev;
  GridCounters* ctr;
};

__device__ __forceinline__ uint64_t rank_of(uint32_t i, uint32_t j, int e) {
  return ((uint64_t)i << 34) | ((uint64_t)j << 2) | (uint64_t)e;
}

__device__ __forceinline__ bool vexists(const LatticeView& L, uint32_t i,
                                        uint32_t j) {
  return i < (uint32_t)L.N && j < (uint32_t)L.M &&
         L.vflag[(size_t)i * L.M + j] == 1;
}

// The level-`level` edge that writes vertex (ip, jp), if any: a vertex on a
// level line strictly inside an edge of a level-`level` leaf block (whose
// other side is finer).  Blocks whose top-left corner is captured skip the
// fix (BT/Grid.h:107) and write nothing.
__device__ bool owner_rank(const LatticeView& L, int level, uint32_t ip,
                           uint32_t jp, uint64_t& rank) {
  const uint32_t g = pow2u(L.maxlevel - level);
  const uint32_t M = L.M;
  const bool hi = (ip % g) == 0, hj = (jp % g) == 0;
  if (hi == hj) return false;
  uint32_t bi, bj;
  int e;
  if (hi) {
    const uint32_t j0 = jp - jp % g;
    if (L.blevel[(size_t)ip * M + j0] == level) {
      bi = ip; bj = j0; e = 1;
    } else if (ip >= g && L.blevel[(size_t)(ip - g) * M + j0] == level) {
      bi = ip - g; bj = j0; e = 3;
    } else {
      return false;
    }
  } else {
    const uint32_t i0 = ip - ip % g;
    const uint32_t jl = (jp + M - g) % M;
    if (L.blevel[(size_t)i0 * M + jp] == level) {
      bi = i0; bj = jp; e = 0;
    } else if (L.blevel[(size_t)i0 * M + jl] == level) {
      bi = i0; bj = jl; e = 2;
    } else {
      return false;
    }
  }
  if (L.thphi[(size_t)bi * M + bj].y < 0) return false;
  rank = rank_of(bi, bj, e);
  return true;
}

// hermite (BT/Grid.h:183-204), tension 0, bias 0
__device__ __forceinline__ double hermite1(double v, double x0, double x1,
                                           double x2, double x3) {
  const double aTension = 0., aBias = 0.;
  const double v2 = v * v;
  const double v3 = v * v2;
  const double aa = (1. + aBias) * (1. - aTension) / 2.;
  const double bb = (1. - aBias) * (1. - aTension) / 2.;
  const double m0 = aa * (x1 - x0) + bb * (x2 - x1);
  const double m1 = aa * (x2 - x1) + bb * (x3 - x2);
  const double u0 = 2. * v3 - 3. * v2 + 1.;
  const double u1 = v3 - 2. * v2 + v;
  const double u2 = v3 - v2;
  const double u3 = -2. * v3 + 3. * v2;
  return u0 * x1 + u1 * m0 + u2 * m1 + u3 * x2;
}

// check2PIcross + correct2PIcross with factor 5 (BT/Metric.h:333-364)
__device__ __forceinline__ void fix2pi(double* p, int n) {
  bool cross = false;
  for (int q = 0; q < n; q++)
    if (p[q] > kPi2 * (1. - 1. / 5.)) cross = true;
  if (!cross) return;
  for (int q = 0; q < n; q++)
    if (p[q] < kPi2 * (1. / 5.)) p[q] += kPi2;
}

struct Edge {
  uint32_t i0, j0;  // start vertex
  int udlr;         // 1 = vertical (down), 0 = horizontal (right)
  uint32_t g;       // length
  uint64_t rank;
};

// Value of vertex (ip, jp) as the sequential canonical order would see it
// while edge E processes its sub-edge [a_off, b_off].
__device__ double2 read_vertex(const TfixArgs& A, const Edge& E, uint32_t ip,
                               uint32_t jp, uint32_t a_off, uint32_t b_off) {
  const LatticeView& L = A.L;
  const size_t id = (size_t)ip * L.M + jp;
  // own interior vertex?
  uint32_t o = 0;
  bool own = false;
  if (E.udlr) {
    if (jp == E.j0 && ip > E.i0 && ip < E.i0 + E.g) { own = true; o = ip - E.i0; }
  } else {
    if (ip == E.i0 && jp > E.j0 && jp < E.j0 + E.g) { own = true; o = jp - E.j0; }
  }
  if (own) {
    // pre-order DFS: written = everything left of a, plus every endpoint of
    // an interval on the path from the edge to [a, b]
    bool written = o <= a_off || o == b_off;
    if (!written) {
      const uint32_t h = b_off - a_off;
      for (uint32_t len = 2 * h; len <= E.g; len *= 2) {
        const uint32_t y = (a_off / len + 1) * len;
        if (o == y) { written = true; break; }
      }
    }
    return written ? A.Xcur[id] : L.thphi[id];
  }
  if (A.pass > 1) {
    uint64_t r;
    if (owner_rank(L, A.level, ip, jp, r) && r < E.rank) return A.Xprev[id];
  }
  return L.thphi[id];
}

// One node of checkAdjacentBlock's walk (BT/Grid.h:132-177): the sub-edge
// [fa, fb] of edge E.  When its midpoint exists, writes the midpoint's value
// (hermite of the four values along the line, or the mean of the ends) to
// Xcur, sets `changed` if it differs from the previous pass, and returns
// true (the walk then visits both halves).
__device__ bool fix_node(const TfixArgs& A, const Edge& E, uint32_t fa, uint32_t fb,
                         bool& changed) {
  const LatticeView& L = A.L;
  const uint32_t M = L.M, N = L.N;
  const uint32_t h = fb - fa;
  const uint32_t ia = E.i0 + E.udlr * fa, ja = E.j0 + (1 - E.udlr) * fa;
  uint32_t ib, jb;
  if (fb == E.g) {
    ib = E.i0 + E.udlr * E.g;
    jb = (E.j0 + (1 - E.udlr) * E.g) % M;
  } else {
    ib = E.i0 + E.udlr * fb;
    jb = E.j0 + (1 - E.udlr) * fb;
  }
  const uint32_t im = ia + E.udlr * h / 2, jm = ja + (1 - E.udlr) * h / 2;
  if (!vexists(L, im, jm)) return false;
  uint32_t jprev = (ja - (1 - E.udlr) * h + M) % M;
  uint32_t jnext = (ja + (1 - E.udlr) * 2 * h) % M;
  uint32_t iprev = ia - E.udlr * h;
  uint32_t inext = ia + 2 * E.udlr * h;
  bool half = false;
  if (ia == 0) {
    jprev = (ja + M / 2) % M;
    iprev = h;
  } else if (inext > N - 1) {
    inext = ia;
    if (L.eq) jnext = (ja + M / 2) % M;
    else half = true;
  }
  double2 val;
  bool succes = false;
  const double2 va = read_vertex(A, E, ia, ja, fa, fb);
  const double2 vb = read_vertex(A, E, ib, jb, fa, fb);
  if (vexists(L, iprev, jprev) && vexists(L, inext, jnext)) {
    const double2 vp = read_vertex(A, E, iprev, jprev, fa, fb);
    const double2 vn = read_vertex(A, E, inext, jnext, fa, fb);
    if (!(vp.x == -1 && vp.y == -1) && !(vn.x == -1 && vn.y == -1)) {
      succes = true;
      double ct[4] = {vp.x, va.x, vb.x, vn.x};
      double cp[4] = {vp.y, va.y, vb.y, vn.y};
      if (half) ct[3] = kPi - ct[3];
      fix2pi(cp, 4);
      val.x = hermite1(0.5, ct[0], ct[1], ct[2], ct[3]);
      val.y = hermite1(0.5, cp[0], cp[1], cp[2], cp[3]);
    }
  }
  if (!succes) {
    double ct[2] = {va.x, vb.x};
    double cp[2] = {va.y, vb.y};
    fix2pi(cp, 2);
    val.x = 1. / 2. * (ct[1] + ct[0]);
    val.y = 1. / 2. * (cp[1] + cp[0]);
  }
  const size_t idm = (size_t)im * M + jm;
  if (A.pass > 1) {
    const double2 old = A.Xprev[idm];
    if (__double_as_longlong(old.x) != __double_as_longlong(val.x) ||
        __double_as_longlong(old.y) != __double_as_longlong(val.y))
      changed = true;
  }
  A.Xcur[idm] = val;
  return true;
}

// checkAdjacentBlock (BT/Grid.h:132-177) as an explicit pre-order DFS, one
// thread per edge.  Returns true if any written value differs from the
// previous pass.
__device__ bool fix_edge(const TfixArgs& A, const Edge& E) {
  const LatticeView& L = A.L;
  struct Frame { uint32_t a, b; int lv; };
  Frame stack[16];
  int sp = 0;
  stack[sp++] = {0u, E.g, A.level};
  bool changed = false;
  while (sp > 0) {
    const Frame f = stack[--sp];
    if (!fix_node(A, E, f.a, f.b, changed)) continue;
    if (f.lv + 1 == L.maxlevel) continue;
    const uint32_t mo = f.a + (f.b - f.a) / 2;
    if (sp + 2 <= 16) {
      stack[sp++] = {mo, f.b, f.lv + 1};  // right half after the left one
      stack[sp++] = {f.a, mo, f.lv + 1};
    } else {
      atomicOr(&A.ctr->err, 2u);
    }
  }
  return changed;
}

// The same walk by a team of T lanes (a power of two, T <= 16, teams aligned
// in the warp; every lane of the warp calls, `valid` false for a team without
// an edge), depth by depth: the sub-edges of one depth are independent, and
// every value a node reads (its ends and the points one length beyond them)
// sits at a multiple of its length, i.e. at a midpoint of an earlier depth,
// so the values are the DFS's.  read_vertex keeps the DFS's view of which
// points this pass has written.  g <= 64 (at most 32 sub-edges per depth).
__device__ bool fix_edge_team(const TfixArgs& A, const Edge& E, bool valid, uint32_t g,
                              unsigned T, unsigned t) {
  const int depths = __ffs((int)g) - 1;  // log2 g
  uint32_t vis = valid ? 1u : 0u;         // sub-edges of this depth the walk visits
  bool changed = false;
  for (int d = 0; d < depths; d++) {
    const uint32_t nd = 1u << d, h = g >> d;
    uint32_t wrote = 0;
    for (uint32_t k = t; k < nd; k += T)
      if (((vis >> k) & 1u) && fix_node(A, E, k * h, (k + 1) * h, changed)) wrote |= 1u << k;
    __syncwarp();  // this depth's values before the next depth reads them
    for (unsigned sft = 1; sft < T; sft <<= 1) wrote |= __shfl_xor_sync(0xffffffffu, wrote, sft);
    vis = 0;
    if (d + 1 < depths)
      for (uint32_t k = 0; k < nd; k++)
        if ((wrote >> k) & 1u) vis |= 3u << (2 * k);
  }
  return changed;
}

// One Jacobi pass of the fix over leaf edges [lo, hi) of grid A at side g, by
// all threads of the launch's blockIdx.y row (warps whole).  A pass takes
// about (rounds of edges over the threads) x (nodes walked one after another),
// each node a few dependent loads: one thread per edge walks up to g - 1
// nodes, a team of T = min(16, g / 2) lanes log2 g depths but takes T lanes
// per edge.  Edges of 4 to 64 vertices go to teams when that estimate is the
// smaller (a lone grid's coarse levels, whose long edges bound the pass);
// otherwise one thread walks each edge (a set of many grids, whose edges
// outnumber the threads).  Returns whether this thread wrote a changed value.
__device__ bool tfix_sweep(const TfixArgs& A, uint32_t lo, uint32_t hi, uint32_t g) {
  const LatticeView& L = A.L;
  const uint32_t M = L.M;
  const uint64_t n4 = 4ull * (hi - lo);
  auto edge_of = [&](uint64_t u, Edge& E) -> bool {
    const uint32_t key = A.leaves[lo + (uint32_t)(u >> 2)];
    const int e = (int)(u & 3u);
    const uint32_t i = key / M, j = key % M;
    if (L.thphi[key].y < 0) return false;  // BT/Grid.h:107
    const uint32_t k = i + g, l = (j + g) % M;
    E = e == 0   ? Edge{i, j, 1, g, rank_of(i, j, 0)}
        : e == 1 ? Edge{i, j, 0, g, rank_of(i, j, 1)}
        : e == 2 ? Edge{i, l, 1, g, rank_of(i, j, 2)}
                 : Edge{k, j, 0, g, rank_of(i, j, 3)};
    return true;
  };
  bool changed = false;
  const unsigned T = min(16u, g / 2);
  const uint64_t lanes = (uint64_t)gridDim.x * blockDim.x;
  const int depths = __ffs((int)g) - 1;
  const uint64_t team_cost = (n4 * T + lanes - 1) / lanes * (uint64_t)depths;
  const uint64_t walk_cost = (n4 + lanes - 1) / lanes * (uint64_t)(g - 1);
  if (g < 4 || g > 64 || team_cost >= walk_cost) {
    for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n4;
         u += (uint64_t)gridDim.x * blockDim.x) {
      Edge E;
      if (edge_of(u, E)) changed |= fix_edge(A, E);
    }
    return changed;
  }
  const unsigned lane = threadIdx.x & 31u;
  const unsigned tpw = 32u / T, team = lane / T, t = lane % T;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t w0 = warp * tpw; w0 < n4; w0 += nwarps * tpw) {  // warp-uniform
    const uint64_t u = w0 + team;
    Edge E{0u, 0u, 0, g, 0ull};
    const bool valid = u < n4 && edge_of(u, E);
    changed |= fix_edge_team(A, E, valid, g, T, t);
  }
  return changed;
}

__device__ __forceinline__ TfixArgs tfix_args(const GridDesc& d, int level, int pass,
                                              int lo, int hi_slot) {
  TfixArgs A;
  A.L = d.L;
  A.level = level;
  A.pass = pass;
  A.leaves = d.leaves;
  A.lo = lo;
  A.hi_slot = hi_slot;
  A.Xcur = d.X[pass & 1];
  A.Xprev = d.X[(pass - 1) & 1];
  A.ctr = d.ctr;
  return A;
}

__global__ void k_tfix_pass(const GridDesc* __restrict__ D, int level, int pass, int lo_slot,
                            int hi_slot) {
  const TfixArgs A = tfix_args(D[blockIdx.y], level, pass, lo_slot, hi_slot);
  GridCounters* ctr = A.ctr;
  if (A.pass > 1 && *(volatile uint32_t*)&ctr->tfix_flags[A.pass - 1] == 0)
    return;  // converged already
  const uint32_t lo = ctr->leaf_off[A.lo], hi = ctr->leaf_off[A.hi_slot];
  // an edge's T-vertices belong to it alone
  const bool changed = tfix_sweep(A, lo, hi, pow2u(A.L.maxlevel - A.level));
  if (__any_sync(0xffffffffu, changed) && (threadIdx.x & 31) == 0)
    atomicOr(&ctr->tfix_flags[A.pass], 1u);
}

// Copies the converged values of a level's T-vertices into the lattice (the
// last pass, `passes`, wrote X[passes & 1]; passes skipped after convergence
// left both buffers equal on every written vertex).
__global__ void k_tfix_commit(const GridDesc* __restrict__ D, int level, int lo_slot,
                              int hi_slot, int passes) {
  const GridDesc& d = D[blockIdx.y];
  GridCounters* ctr = d.ctr;
  const uint32_t lo = ctr->leaf_off[lo_slot], hi = ctr->leaf_off[hi_slot];
  const LatticeView L = d.L;
  const double2* X = d.X[passes & 1];
  const uint32_t M = L.M;
  const uint32_t g = pow2u(L.maxlevel - level);
  const uint64_t n4 = 4ull * (hi - lo);
  for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n4;
       u += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t key = d.leaves[lo + (uint32_t)(u >> 2)];
    const int e = (int)(u & 3u);
    const uint32_t i = key / M, j = key % M;
    if (L.thphi[key].y < 0) continue;
    const uint32_t k = i + g, l = (j + g) % M;
    const uint32_t si = e == 3 ? k : i, sj = e == 2 ? l : j;
    const int ud = (e == 0 || e == 2) ? 1 : 0;
    for (uint32_t o = 1; o < g; o++) {
      const uint32_t ip = si + ud * o, jp = sj + (1 - ud) * o;
      const size_t id = (size_t)ip * M + jp;
      if (L.vflag[id] == 1) L.thphi[id] = X[id];
    }
  }
}

__global__ void k_tfix_check(const GridDesc* __restrict__ D, int G, int passes) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G) return;
  GridCounters* ctr = D[g].ctr;
  bool conv = false;
  for (int t = 2; t <= passes; t++)
    if (ctr->tfix_flags[t] == 0) conv = true;
  if (!conv) ctr->err |= 1u;
  for (int t = 0; t < 16; t++) ctr->tfix_flags[t] = 0;
  ctr->tfix_flags[1] = 1;
}

// The T-vertex fix of one level for every grid of the set in one cooperative
// launch (blockIdx.y = grid): the Jacobi passes of k_tfix_pass separated by
// grid-wide barriers, stopping after the first pass in which no grid changed
// (at most `passes`), then k_tfix_commit and k_tfix_check.  The same passes
// and values as the launches it replaces, which cost a launch each even
// after convergence (40 launches and ~0.5 ms of a C2 build).  set_changed
// (16 words, zero on entry and left zero) is the set-wide "changed" flag per
// pass.
__global__ void __launch_bounds__(128)
k_tfix_level(const GridDesc* __restrict__ D, int level, int lo_slot, int hi_slot, int passes,
             uint32_t* set_changed) {
  cooperative_groups::grid_group grid = cooperative_groups::this_grid();
  const GridDesc& d = D[blockIdx.y];
  GridCounters* ctr = d.ctr;
  const uint32_t lo = ctr->leaf_off[lo_slot], hi = ctr->leaf_off[hi_slot];
  const LatticeView& L = d.L;
  const uint32_t M = L.M;
  const uint32_t g = pow2u(L.maxlevel - level);
  const uint64_t n4 = 4ull * (hi - lo);
  int pass = 1;
  for (; pass <= passes; pass++) {
    // a grid that did not change in the previous pass is converged
    if (pass == 1 || *(volatile uint32_t*)&ctr->tfix_flags[pass - 1] != 0) {
      const TfixArgs A = tfix_args(d, level, pass, lo_slot, hi_slot);
      const bool changed = tfix_sweep(A, lo, hi, g);
      if (__any_sync(0xffffffffu, changed) && (threadIdx.x & 31) == 0) {
        atomicOr(&ctr->tfix_flags[pass], 1u);
        atomicOr(&set_changed[pass], 1u);
      }
    }
    grid.sync();
    // the same decision in every block: stop when no grid changed
    if (pass > 1 && *(volatile uint32_t*)&set_changed[pass] == 0) break;
  }
  // commit (the values of the last pass; passes after a grid converged left
  // both buffers equal on every vertex it writes)
  const double2* X = d.X[passes & 1];
  for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n4;
       u += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t key = d.leaves[lo + (uint32_t)(u >> 2)];
    const int e = (int)(u & 3u);
    const uint32_t i = key / M, j = key % M;
    if (L.thphi[key].y < 0) continue;
    const uint32_t k = i + g, l = (j + g) % M;
    const uint32_t si = e == 3 ? k : i, sj = e == 2 ? l : j;
    const int ud = (e == 0 || e == 2) ? 1 : 0;
    for (uint32_t o = 1; o < g; o++) {
      const uint32_t ip = si + ud * o, jp = sj + (1 - ud) * o;
      const size_t id = (size_t)ip * M + jp;
      if (L.vflag[id] == 1) L.thphi[id] = X[id];
    }
  }
  grid.sync();
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    bool conv = false;
    for (int t = 2; t <= passes; t++)
      if (ctr->tfix_flags[t] == 0) conv = true;
    if (!conv) ctr->err |= 1u;
    for (int t = 0; t < 16; t++) ctr->tfix_flags[t] = 0;
    ctr->tfix_flags[1] = 1;
    if (blockIdx.y == 0)
      for (int t = 0; t < 16; t++) set_changed[t] = 0;
  }
}

// ------------------------------------------------------------ flow
// Sync words of the first n grids' vertices: traced where the seed level
// traced them (and the pole copies), else nothing yet.
__global__ void k_flow_sync(const GridDesc* __restrict__ D, size_t total, uint32_t NM,
                            uint32_t* __restrict__ vsync) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const uint32_t g = (uint32_t)(t / NM), key = (uint32_t)(t % NM);
    vsync[t] = D[g].L.vflag[key] == 1 ? kVTraced : 0u;
  }
}

// The start level's blocks of grid blockIdx.y (its check list) onto the
// check queue: their corners are all traced.
__global__ void k_flow_checks(const GridDesc* __restrict__ D, uint32_t NM,
                              uint32_t* __restrict__ q, FlowCtl* ctl) {
  const uint32_t g = blockIdx.y;
  const GridDesc& d = D[g];
  const uint32_t n = d.ctr->n_check;
  const unsigned lane = threadIdx.x & 31u;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const uint32_t t = base + threadIdx.x;
    const bool valid = t < n;
    const unsigned m = __ballot_sync(0xffffffffu, valid);
    unsigned long long at = 0;
    if (lane == 0 && m) {
      atomicAdd(&ctl->live.v, (unsigned long long)__popc(m));
      at = atomicAdd(&ctl->tail[kFqCheck].v, (unsigned long long)__popc(m));
    }
    at = __shfl_sync(0xffffffffu, at, 0);
    if (valid) q[at + __popc(m & ((1u << lane) - 1u))] = g * NM + d.list[0][t];
  }
}

// After the flow, one block per grid: its leaves (tagged with their level)
// sorted by level into the leaf list with the per-level offsets the T-vertex
// fix reads (the order within a level does not matter to it), the rays it
// traced counted, and the flow's error flags.
__global__ void k_flow_leaves(const GridDesc* __restrict__ D, int span,
                              const FlowCtl* __restrict__ ctl) {
  const GridDesc& d = D[blockIdx.x];
  GridCounters* ctr = d.ctr;
  const uint32_t n = ctr->n_leaf;
  __shared__ uint32_t cnt[16], off[16];
  if (threadIdx.x < 16) cnt[threadIdx.x] = 0;
  __syncthreads();
  uint32_t* tmp = d.trace;  // free once the flow has ended
  for (uint32_t t = threadIdx.x; t < n; t += blockDim.x) {
    const uint32_t v = d.leaves[t];
    tmp[t] = v;
    atomicAdd(&cnt[v >> kFlowKeyBits], 1u);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (int s = 0; s < 16; s++) {
      off[s] = acc;
      if (s <= span) ctr->leaf_off[s] = acc;
      acc += cnt[s];
    }
    const uint64_t tr = ((uint64_t)ctr->traced_hi << 32 | ctr->traced_lo) + ctr->n_trace;
    ctr->traced_lo = (uint32_t)tr;
    ctr->traced_hi = (uint32_t)(tr >> 32);
    ctr->n_trace = 0;
    ctr->err |= ctl->err;
  }
  __syncthreads();
  for (uint32_t t = threadIdx.x; t < n; t += blockDim.x) {
    const uint32_t v = tmp[t];
    d.leaves[atomicAdd(&off[v >> kFlowKeyBits], 1u)] = v & ((1u << kFlowKeyBits) - 1u);
  }
}

// ------------------------------------------------------------ exports
// makeGrid (BT/MakeImageKernel.cu:369-384) from the dense lattice: float2
// values, (-2,-2) where no vertex exists; with sym the lower hemisphere is
// mirrored (theta -> pi - theta).
__global__ void k_export_map(LatticeView L, float2* out, int rows, int sym) {
  const size_t NM = (size_t)L.N * L.M;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < NM;
       q += (size_t)gridDim.x * blockDim.x) {
    float2 v = make_float2(-2.f, -2.f);
    if (L.vflag[q] == 1) {
      const double2 d = L.thphi[q];
      v = make_float2((float)d.x, (float)d.y);
    }
    out[q] = v;
    if (sym) {
      const uint32_t i = (uint32_t)(q / L.M), j = (uint32_t)(q % L.M);
      if (v.x != -1 && v.x != -2) v.x = kPiF - v.x;
      out[(size_t)(rows - (int)i - 1) * L.M + j] = v;
    }
  }
}

__global__ void k_export_dense(LatticeView L, double* th, double* ph,
                               uint8_t* ex, int32_t* st, int8_t* bl,
                               uint8_t* vs) {
  const size_t NM = (size_t)L.N * L.M;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < NM;
       q += (size_t)gridDim.x * blockDim.x) {
    const bool e = L.vflag[q] == 1;
    const double2 d = L.thphi[q];
    if (th) th[q] = e ? d.x : -2.0;
    if (ph) ph[q] = e ? d.y : -2.0;
    if (ex) ex[q] = e ? 1 : 0;
    if (st) st[q] = L.steps[q];
    if (bl) bl[q] = L.blevel[q];
    if (vs) vs[q] = L.vstat[q];
  }
}

// Compact export in key order (i, then j): per-row counts, a row scan,
// then an ordered per-row compaction (one block per row).
__global__ void k_row_count(const uint8_t* __restrict__ vflag, const int8_t* __restrict__ bl,
                            int M, uint32_t* __restrict__ vcount,
                            uint32_t* __restrict__ bcount) {
  const int i = blockIdx.x;
  uint32_t v = 0, b = 0;
  for (int j = threadIdx.x; j < M; j += blockDim.x) {
    v += vflag[(size_t)i * M + j] == 1;
    b += bl[(size_t)i * M + j] >= 0;
  }
  for (int o = 16; o > 0; o >>= 1) {
    v += __shfl_xor_sync(0xffffffffu, v, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  __shared__ uint32_t sv[32], sb[32];
  if ((threadIdx.x & 31) == 0) {
    sv[threadIdx.x >> 5] = v;
    sb[threadIdx.x >> 5] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t tv = 0, tb = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      tv += sv[w];
      tb += sb[w];
    }
    vcount[i] = tv;
    bcount[i] = tb;
  }
}

// Exclusive scan of N row counts in one block: each thread scans a
// contiguous chunk, the chunk totals are scanned in shared memory.
__global__ void k_row_scan(uint32_t* vcount, uint32_t* bcount, int N, uint64_t* totals) {
  __shared__ uint64_t sv[1024], sb[1024];
  const int t = threadIdx.x, T = blockDim.x;
  const int chunk = (N + T - 1) / T;
  const int i0 = min(N, t * chunk), i1 = min(N, i0 + chunk);
  uint64_t v = 0, b = 0;
  for (int i = i0; i < i1; i++) {
    v += vcount[i];
    b += bcount[i];
  }
  sv[t] = v;
  sb[t] = b;
  __syncthreads();
  for (int o = 1; o < T; o <<= 1) {
    const uint64_t av = t >= o ? sv[t - o] : 0, ab = t >= o ? sb[t - o] : 0;
    __syncthreads();
    sv[t] += av;
    sb[t] += ab;
    __syncthreads();
  }
  uint64_t pv = sv[t] - v, pb = sb[t] - b;
  for (int i = i0; i < i1; i++) {
    const uint32_t cv = vcount[i], cb = bcount[i];
    vcount[i] = (uint32_t)pv;
    bcount[i] = (uint32_t)pb;
    pv += cv;
    pb += cb;
  }
  if (t == T - 1) {
    totals[0] = sv[t];
    totals[1] = sb[t];
  }
}

struct CompactOut {
  uint32_t* vi;
  uint32_t* vj;
  double* th;
  double* ph;
  int32_t* st;
  uint32_t* bi;
  uint32_t* bj;
  int8_t* blv;
};

__global__ void k_row_compact(LatticeView L, const uint32_t* __restrict__ voff,
                              const uint32_t* __restrict__ boff, CompactOut o) {
  const int i = blockIdx.x;
  const int M = L.M;
  __shared__ uint32_t base_v, base_b;
  __shared__ uint32_t wv[32], wb[32];
  if (threadIdx.x == 0) {
    base_v = voff[i];
    base_b = boff[i];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int j0 = 0; j0 < M; j0 += blockDim.x) {
    const int j = j0 + threadIdx.x;
    const size_t id = (size_t)i * M + j;
    const bool hv = j < M && L.vflag[id] == 1;
    const bool hb = j < M && L.blevel[id] >= 0;
    const unsigned mv = __ballot_sync(0xffffffffu, hv), mb = __ballot_sync(0xffffffffu, hb);
    if (lane == 0) {
      wv[w] = __popc(mv);
      wb[w] = __popc(mb);
    }
    __syncthreads();
    uint32_t pv = base_v, pb = base_b;
    for (int ww = 0; ww < w; ww++) {
      pv += wv[ww];
      pb += wb[ww];
    }
    const unsigned lt = (1u << lane) - 1u;
    if (hv) {
      const uint32_t k = pv + __popc(mv & lt);
      const double2 v = L.thphi[id];
      if (o.vi) o.vi[k] = i;
      if (o.vj) o.vj[k] = j;
      if (o.th) o.th[k] = v.x;
      if (o.ph) o.ph[k] = v.y;
      if (o.st) o.st[k] = L.steps[id];
    }
    if (hb) {
      const uint32_t k = pb + __popc(mb & lt);
      if (o.bi) o.bi[k] = i;
      if (o.bj) o.bj[k] = j;
      if (o.blv) o.blv[k] = L.blevel[id];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int ww = 0; ww < nw; ww++) {
        base_v += wv[ww];
        base_b += wb[ww];
      }
    }
    __syncthreads();
  }
}

static unsigned grid_blocks(size_t work, int threads) {
  size_t b = (work + threads - 1) / threads;
  const size_t cap = (size_t)sm_count() * 8;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (unsigned)b;
}

// Blocks per grid of a set-wide launch (grid dimension y = the G grids),
// so that the whole launch covers the device a few times over.
static unsigned set_blocks(size_t work, int threads, int G) {
  size_t b = (work + threads - 1) / threads;
  size_t cap = ((size_t)sm_count() * 8 + G - 1) / G;
  if (cap < 2) cap = 2;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (unsigned)b;
}

}  // namespace bt

using namespace bt;

namespace {

void batch_free(bt_batch* b) {
  if (!b) return;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
  if (b->timing)
    for (int k = 0; k < 2 * 16; k++) cudaEventDestroy(b->ev[k]);
  for (int k = 0; k < kParamSlots; k++) {
    if (b->Dev[k]) cudaEventDestroy(b->Dev[k]);
    if (b->Dh[k]) cudaFreeHost(b->Dh[k]);
  }
  if (b->grids) {
    for (int g = 0; g < b->G; g++) {
      bt_grid* m = &b->grids[g];
      void* ptrs[] = {m->mapgrid, m->rowv, m->rowb, m->totals, m->compact};
      for (void* p : ptrs)
        if (p) cudaFree(p);
      if (m->totals_host) cudaFreeHost(m->totals_host);
    }
    delete[] b->grids;
  }
  void* ptrs[] = {b->thphi, b->steps,   b->vflag,  b->vstat,   b->blevel, b->lists,
                  b->X,     b->ctr,     b->D,      b->qoff,    b->qfetch, b->flow_q,
                  b->flow_bw, b->flow_ctl, b->tfix_changed};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (b->ctr_host) cudaFreeHost(b->ctr_host);
  delete b;
}

int batch_create(int maxlevel, int angle, int count, bt_batch** out) {
  BT_ARG_CHECK(out != nullptr, "out is NULL");
  *out = nullptr;
  BT_ARG_CHECK(count >= 1 && count <= 65535, "set size out of [1, 65535]");
  int32_t N, M;
  if (int rc = bt_grid_dims(maxlevel, angle, &N, &M)) return rc;
  bt_batch* b = new (std::nothrow) bt_batch;
  if (!b) return BT_ERR_NOMEM;
  std::memset(b, 0, sizeof(*b));
  b->G = count;
  b->N = N;
  b->M = M;
  b->eq = angle ? 1 : 0;
  b->maxlevel = maxlevel;
  b->NM = (size_t)N * M;
  b->shape = TraceShape{128, 0, 0};
  b->tfix_passes = bt::kMaxTfixPasses;
  b->tfix_coop = 1;
  b->flow_early = 1;
  b->grids = new (std::nothrow) bt_grid[count];
  if (!b->grids) {
    delete b;
    return BT_ERR_NOMEM;
  }
  std::memset(b->grids, 0, sizeof(bt_grid) * count);
  const size_t G = (size_t)count, NM = b->NM;
  cudaError_t e = cudaSuccess;
#define GALLOC(ptr, bytes) \
  if (e == cudaSuccess) e = cudaMalloc((void**)&(ptr), (bytes));
  GALLOC(b->thphi, G * NM * sizeof(double2));
  GALLOC(b->steps, G * NM * sizeof(int32_t));
  GALLOC(b->vflag, G * NM + 4);
  GALLOC(b->vstat, G * NM);
  GALLOC(b->blevel, G * NM);
  GALLOC(b->lists, 4 * G * NM * sizeof(uint32_t));
  GALLOC(b->X, 2 * G * NM * sizeof(double2));
  GALLOC(b->ctr, G * sizeof(GridCounters));
  GALLOC(b->D, G * sizeof(GridDesc));
  GALLOC(b->qoff, (G + 1) * sizeof(uint32_t));
  GALLOC(b->qfetch, sizeof(uint32_t));
  GALLOC(b->tfix_changed, 16 * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMemset(b->tfix_changed, 0, 16 * sizeof(uint32_t));
  for (size_t g = 0; g < G; g++) {
    bt_grid* m = &b->grids[g];
    GALLOC(m->rowv, (size_t)N * sizeof(uint32_t));
    GALLOC(m->rowb, (size_t)N * sizeof(uint32_t));
    GALLOC(m->totals, 2 * sizeof(uint64_t));
    if (e == cudaSuccess) e = cudaMallocHost((void**)&m->totals_host, 2 * sizeof(uint64_t));
  }
#undef GALLOC
  if (e == cudaSuccess) e = cudaMallocHost((void**)&b->ctr_host, G * sizeof(GridCounters));
  for (int k = 0; k < kParamSlots && e == cudaSuccess; k++) {
    e = cudaMallocHost((void**)&b->Dh[k], G * sizeof(GridDesc));
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->Dev[k], cudaEventDisableTiming);
  }
  if (e != cudaSuccess) {
    set_error("grid set allocation (%d grids, N=%d M=%d) failed: %s", count, N, M,
              cudaGetErrorString(e));
    batch_free(b);
    return BT_ERR_NOMEM;
  }
  for (size_t g = 0; g < G; g++) {
    bt_grid* m = &b->grids[g];
    m->set = b;
    m->index = (int)g;
    m->L.N = N;
    m->L.M = M;
    m->L.eq = b->eq;
    m->L.maxlevel = maxlevel;
    m->L.thphi = b->thphi + g * NM;
    m->L.steps = b->steps + g * NM;
    m->L.vflag = b->vflag + g * NM;
    m->L.vstat = b->vstat + g * NM;
    m->L.blevel = b->blevel + g * NM;
    m->ctr = b->ctr + g;
    m->ctr_host = b->ctr_host + g;
  }
  *out = b;
  return BT_OK;
}

// Descriptor of member g for a build from `startlevel` with ray params p.
GridDesc member_desc(bt_batch* b, int g, int startlevel, const RayParams& p) {
  const size_t NM = b->NM, G = b->G;
  bt_grid* m = &b->grids[g];
  GridDesc d;
  d.L = m->L;
  d.L.startlevel = startlevel;
  d.p = p;
  d.list[0] = b->lists + (0 * G + g) * NM;
  d.list[1] = b->lists + (1 * G + g) * NM;
  d.trace = b->lists + (2 * G + g) * NM;
  d.leaves = b->lists + (3 * G + g) * NM;
  d.X[0] = b->X + (0 * G + g) * NM;
  d.X[1] = b->X + (1 * G + g) * NM;
  d.ctr = b->ctr + g;
  return d;
}

// The flow is used when switched on and its items fit in 28 bits.
static bool flow_usable(const bt_batch* b, int n) {
  return b->flow && b->flow_q && (uint64_t)n * b->NM < (1ull << kFlowKeyBits);
}

// The launch sequence of one build of the whole set (no host
// synchronisation).  Returns the number of kernels launched in *launches.
int batch_enqueue(bt_batch* b, int n, int startlevel, int precision, cudaStream_t s,
                  bool timing, int* launches) {
  const int G = n;  // the first n members
  const size_t NM = b->NM;
  int nk = 0;
  BT_CUDA_TRY(cudaMemsetAsync(b->vflag, 0, G * NM + 4, s));
  BT_CUDA_TRY(cudaMemsetAsync(b->vstat, 0, G * NM, s));
  BT_CUDA_TRY(cudaMemsetAsync(b->steps, 0, G * NM * sizeof(int32_t), s));
  BT_CUDA_TRY(cudaMemsetAsync(b->blevel, 0xff, G * NM, s));
  BT_CUDA_TRY(cudaMemsetAsync(b->ctr, 0, G * sizeof(GridCounters), s));
  b->n_ev = 0;
  auto trace = [&]() -> int {
    const bool t = timing && b->timing && b->n_ev + 2 <= 2 * 16;
    k_queue<<<1, 1024, 0, s>>>(b->D, G, b->qoff, b->qfetch);
    if (t) BT_CUDA_TRY(cudaEventRecord(b->ev[b->n_ev], s));
    const int rc = precision == BT_PRECISION_MIXED
                       ? launch_trace_mixed(b->D, G, b->qoff, b->qfetch, b->shape, s)
                   : precision == BT_PRECISION_FAST
                       ? launch_trace_fast(b->D, G, b->qoff, b->qfetch, b->shape, s)
                       : launch_trace_plain(b->D, G, b->qoff, b->qfetch, b->shape, s);
    if (t) {
      BT_CUDA_TRY(cudaEventRecord(b->ev[b->n_ev + 1], s));
      b->n_ev += 2;
    }
    nk += 2;
    return rc;
  };
  const unsigned ga = (G + 127) / 128;
  LatticeView L0 = b->grids[0].L;
  L0.startlevel = startlevel;
  const SeedShape S = seed_shape(L0);
  k_seed<<<dim3(set_blocks((size_t)(S.rows + 1) * S.cols, 256, G), G), 256, 0, s>>>(b->D, S);
  BT_CUDA_TRY(cudaGetLastError());
  nk++;
  if (int rc = trace()) return rc;
  k_pole_copy<<<dim3(set_blocks(S.cols, 256, G), G), 256, 0, s>>>(b->D);
  k_advance<<<ga, 128, 0, s>>>(b->D, G, 1, 0);
  BT_CUDA_TRY(cudaGetLastError());
  nk += 2;
  if (flow_usable(b, G) && startlevel < b->maxlevel) {
    // the refinement levels as one persistent launch
    const size_t GNM = (size_t)G * NM, gnm_full = (size_t)b->G * NM;
    uint32_t* vsync = b->lists + 1 * gnm_full;
    uint32_t* qsetup = b->lists + 0 * gnm_full;  // the check lists, once read
    uint32_t* qtrace = b->lists + 2 * gnm_full;  // the trace lists, free now
    // early refinement when the waiter bits of every level fit a sync word
    const int span = b->maxlevel - startlevel;
    const bool early = b->flow_early && span <= kFlowEarlySpan && span - 1 <= b->flow_bw_levels;
    const size_t bw_levels = early ? (size_t)(span - 1) : 1;
    BT_CUDA_TRY(cudaMemsetAsync(b->flow_ctl, 0, sizeof(FlowCtl), s));
    if (bw_levels) BT_CUDA_TRY(cudaMemsetAsync(b->flow_bw, 0, bw_levels * GNM, s));
    BT_CUDA_TRY(cudaMemsetAsync(b->flow_q, 0xff, 3 * GNM * sizeof(uint32_t), s));
    k_flow_sync<<<sm_count() * 8, 256, 0, s>>>(b->D, GNM, (uint32_t)NM, vsync);
    k_flow_checks<<<dim3(set_blocks(NM / 4, 256, G), G), 256, 0, s>>>(b->D, (uint32_t)NM,
                                                                      b->flow_q, b->flow_ctl);
    BT_CUDA_TRY(cudaMemsetAsync(qsetup, 0xff, GNM * sizeof(uint32_t), s));
    BT_CUDA_TRY(cudaMemsetAsync(qtrace, 0xff, GNM * sizeof(uint32_t), s));
    FlowArgs A;
    A.D = b->D;
    A.G = G;
    A.NM = (uint32_t)NM;
    A.M = (uint32_t)b->M;
    A.maxlevel = b->maxlevel;
    A.startlevel = startlevel;
    A.q[kFqCheck] = b->flow_q;
    A.q[kFqSetup] = qsetup;
    A.q[kFqTrace] = qtrace;
    A.q[kFqHot] = b->flow_q + GNM;
    A.q[kFqSetupHot] = b->flow_q + 2 * GNM;
    for (int k = 0; k < kFq; k++) A.cap[k] = GNM;
    A.vsync = vsync;
    A.bwait = b->flow_bw;
    A.bw_stride = early ? GNM : 0;
    A.early = early ? 1 : 0;
    A.ctl = b->flow_ctl;
    A.blocks_per_sm = b->flow;
    A.drop = b->flow_drop;
    b->flow_drop = 0;
    const bool t = timing && b->timing && b->n_ev + 2 <= 2 * 16;
    if (t) BT_CUDA_TRY(cudaEventRecord(b->ev[b->n_ev], s));
    const int rc = precision == BT_PRECISION_MIXED ? launch_flow_mixed(A, s)
                   : precision == BT_PRECISION_FAST ? launch_flow_fast(A, s)
                                                    : launch_flow_plain(A, s);
    if (rc) return rc;
    if (t) {
      BT_CUDA_TRY(cudaEventRecord(b->ev[b->n_ev + 1], s));
      b->n_ev += 2;
    }
    k_flow_leaves<<<G, 256, 0, s>>>(b->D, b->maxlevel - startlevel, b->flow_ctl);
    BT_CUDA_TRY(cudaGetLastError());
    nk += 5;
  } else {
  int cur = 0;
  for (int level = startlevel; level < b->maxlevel; level++) {
    k_refine<<<dim3(set_blocks(NM / 4, 256, G), G), 256, 0, s>>>(b->D, level, cur);
    BT_CUDA_TRY(cudaGetLastError());
    nk++;
    if (int rc = trace()) return rc;
    k_advance<<<ga, 128, 0, s>>>(b->D, G, 0, level - startlevel + 1);
    BT_CUDA_TRY(cudaGetLastError());
    nk++;
    cur ^= 1;
  }
  k_finalize<<<dim3(set_blocks(NM / 4, 256, G), G), 256, 0, s>>>(b->D, cur);
  BT_CUDA_TRY(cudaGetLastError());
  nk++;
  }
  // T-vertex fix, level by level (coarse to fine): one cooperative launch per
  // level when the set's blocks fit the device at once, else a launch per pass
  const unsigned nb = set_blocks(NM / 16, 128, G);
  static int coop_per_sm = -1;
  if (coop_per_sm < 0) {
    int dev = 0, coop = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    coop_per_sm = 0;
    if (coop) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&coop_per_sm, k_tfix_level, 128, 0);
  }
  const unsigned coop_x = std::min<unsigned>(nb, (unsigned)(coop_per_sm * sm_count()) / G);
  for (int level = startlevel; level < b->maxlevel; level++) {
    int lo = level - startlevel, hi = level - startlevel + 1;
    int passes = b->tfix_passes;
    if (b->tfix_coop && coop_x >= 1) {
      int lv = level;
      uint32_t* changed = b->tfix_changed;
      void* args[] = {(void*)&b->D, (void*)&lv, (void*)&lo, (void*)&hi, (void*)&passes,
                      (void*)&changed};
      BT_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)k_tfix_level, dim3(coop_x, G),
                                              dim3(128), args, 0, s));
      nk++;
      continue;
    }
    for (int pass = 1; pass <= passes; pass++)
      k_tfix_pass<<<dim3(nb, G), 128, 0, s>>>(b->D, level, pass, lo, hi);
    k_tfix_commit<<<dim3(nb, G), 128, 0, s>>>(b->D, level, lo, hi, passes);
    k_tfix_check<<<ga, 128, 0, s>>>(b->D, G, passes);
    BT_CUDA_TRY(cudaGetLastError());
    nk += passes + 2;
  }
  BT_CUDA_TRY(cudaMemcpyAsync(b->ctr_host, b->ctr, G * sizeof(GridCounters),
                              cudaMemcpyDeviceToHost, s));
  *launches = nk;
  return BT_OK;
}

int batch_build(bt_batch* b, const bt_camera* cams, const double* spins, int n,
                int startlevel, const bt_integ_opts* o, cudaStream_t s) {
  BT_ARG_CHECK(cams && spins, "NULL cameras or spins");
  BT_ARG_CHECK(n >= 1 && n <= b->G, "grid count out of [1, set size]");
  BT_ARG_CHECK(startlevel >= 1 && startlevel <= b->maxlevel,
               "startlevel out of [1, maxlevel]");
  BT_ARG_CHECK(b->maxlevel - startlevel <= 12, "maxlevel - startlevel > 12 is not supported");
  const int G = n;
  // descriptors into the next pinned staging slot, once its last copy ran
  const int slot = b->slot;
  b->slot = (slot + 1) % kParamSlots;
  BT_CUDA_TRY(cudaEventSynchronize(b->Dev[slot]));
  GridDesc* Dh = b->Dh[slot];
  int precision = -1;
  for (int g = 0; g < G; g++) {
    RayParams p;
    if (make_ray_params(&cams[g], spins[g], o, &p)) {
      set_error("invalid camera or integrator options (grid %d)", g);
      return BT_ERR_ARG;
    }
    precision = p.precision;
    Dh[g] = member_desc(b, g, startlevel, p);
    bt_grid* m = &b->grids[g];
    m->params = p;
    m->cam = cams[g];
    m->a = spins[g];
    m->L.startlevel = startlevel;
    m->built = 0;
  }
  b->built = 0;
  BT_CUDA_TRY(cudaMemcpyAsync(b->D, Dh, G * sizeof(GridDesc), cudaMemcpyHostToDevice, s));
  BT_CUDA_TRY(cudaEventRecord(b->Dev[slot], s));
  int launches = 0;
  if (b->graph) {
    const bool same = b->exec && b->exec_n == G && b->exec_startlevel == startlevel &&
                      b->exec_precision == precision &&
                      b->exec_tfix_passes == b->tfix_passes &&
                      b->exec_tfix_coop == b->tfix_coop &&
                      b->exec_flow == b->flow &&
                      b->exec_shape.threads == b->shape.threads &&
                      b->exec_shape.blocks_per_sm == b->shape.blocks_per_sm &&
                      b->exec_shape.refill == b->shape.refill;
    if (!same) {
      if (b->exec) cudaGraphExecDestroy(b->exec);
      b->exec = nullptr;
      if (!b->cap_stream)
        BT_CUDA_TRY(cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking));
      BT_CUDA_TRY(cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal));
      int rc = batch_enqueue(b, G, startlevel, precision, b->cap_stream, false, &launches);
      cudaGraph_t graph = nullptr;
      const cudaError_t e = cudaStreamEndCapture(b->cap_stream, &graph);
      if (rc == BT_OK && e != cudaSuccess) {
        set_error("build capture failed: %s", cudaGetErrorString(e));
        rc = BT_ERR_CUDA;
      }
      if (rc == BT_OK) {
        const cudaError_t ie = cudaGraphInstantiate(&b->exec, graph, 0);
        if (ie != cudaSuccess) {
          set_error("build graph instantiation failed: %s", cudaGetErrorString(ie));
          rc = BT_ERR_CUDA;
          b->exec = nullptr;
        }
      }
      if (graph) cudaGraphDestroy(graph);
      if (rc) return rc;
      b->exec_n = G;
      b->exec_startlevel = startlevel;
      b->exec_precision = precision;
      b->exec_tfix_passes = b->tfix_passes;
      b->exec_tfix_coop = b->tfix_coop;
      b->exec_flow = b->flow;
      b->exec_shape = b->shape;
      b->launches = launches;
    }
    BT_CUDA_TRY(cudaGraphLaunch(b->exec, s));
    b->n_ev = 0;
  } else {
    if (int rc = batch_enqueue(b, G, startlevel, precision, s, true, &launches)) return rc;
    b->launches = launches;
  }
  b->startlevel = startlevel;
  b->precision = precision;
  b->built = 1;
  b->built_n = G;
  for (int g = 0; g < b->G; g++) b->grids[g].built = g < G ? 1 : 0;
  return BT_OK;
}

float batch_trace_ms(const bt_batch* b) {
  float total = 0.f;
  for (int k = 0; k + 1 < b->n_ev; k += 2) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, b->ev[k], b->ev[k + 1]) == cudaSuccess) total += ms;
  }
  return total;
}

// The flow's buffers, reserved when it is switched on.
int batch_set_flow(bt_batch* b, int on) {
  if (on && !b->flow_q) {
    const size_t GNM = (size_t)b->G * b->NM;
    // block bytes for every level below the max that a build can have
    // blocks wait on (start level 1 or more), at most the early-refinement span
    const int lv = std::max(1, std::min(b->maxlevel - 2, kFlowBwLevels));
    cudaError_t e = cudaMalloc((void**)&b->flow_q, 3 * GNM * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc((void**)&b->flow_bw, (size_t)lv * GNM);
    if (e == cudaSuccess) e = cudaMalloc((void**)&b->flow_ctl, sizeof(FlowCtl));
    if (e != cudaSuccess) {
      cudaFree(b->flow_q);
      cudaFree(b->flow_bw);
      cudaFree(b->flow_ctl);
      b->flow_q = nullptr;
      b->flow_bw = nullptr;
      b->flow_ctl = nullptr;
      set_error("flow buffers (%zu vertices) failed: %s", GNM, cudaGetErrorString(e));
      return BT_ERR_NOMEM;
    }
    b->flow_bw_levels = lv;
  }
  b->flow = on > 0 ? on : 0;
  return BT_OK;
}

int batch_set_timing(bt_batch* b, int on) {
  if (on && !b->timing)
    for (int k = 0; k < 2 * 16; k++) BT_CUDA_TRY(cudaEventCreate(&b->ev[k]));
  if (!on && b->timing) {
    for (int k = 0; k < 2 * 16; k++) cudaEventDestroy(b->ev[k]);
    b->n_ev = 0;
  }
  b->timing = on ? 1 : 0;
  return BT_OK;
}

}  // namespace

namespace bt {
// The map grid of a built grid written into a caller's device buffer of
// map_rows x M float2 (as bt_grid_map_export returns it), without the
// grid's own export buffer.
int grid_map_export_into(const bt_grid* g, float* dst, cudaStream_t s) {
  const int GN = g->L.N, GM = g->L.M;
  const int symv = (float)GM / (float)GN > 3 ? 1 : 0;  // dev_sym, BT/MakeImageKernel.cu:1259-1260
  const int GN1 = symv ? 2 * GN - 1 : GN;
  k_export_map<<<grid_blocks((size_t)GN * GM, 256), 256, 0, s>>>(g->L, (float2*)dst, GN1, symv);
  BT_CUDA_TRY(cudaGetLastError());
  return BT_OK;
}
}  // namespace bt

extern "C" {

int bt_grid_dims(int maxlevel, int angle, int32_t* N, int32_t* M) {
  BT_ARG_CHECK(maxlevel >= 1 && maxlevel <= 14, "maxlevel out of [1, 14]");
  BT_ARG_CHECK(N && M, "NULL pointer");
  const int eq = angle ? 1 : 0;
  // BT/Grid.h:612-614
  *N = (int32_t)(uint32_t)std::round(std::pow(2, maxlevel) / (2 - eq) + 1);
  *M = (2 - eq) * 2 * (*N - 1);
  return BT_OK;
}

int bt_grid_create(int maxlevel, int angle, bt_grid** out) {
  clear_error();
  BT_ARG_CHECK(out != nullptr, "out is NULL");
  *out = nullptr;
  bt_batch* b = nullptr;
  if (int rc = batch_create(maxlevel, angle, 1, &b)) return rc;
  b->standalone = 1;
  *out = &b->grids[0];
  return BT_OK;
}

void bt_grid_destroy(bt_grid* g) {
  if (!g || !g->set->standalone) return;  // members go with their set
  batch_free(g->set);
}

int bt_grid_build(bt_grid* g, const bt_camera* cam, double a, int startlevel,
                  const bt_integ_opts* o, void* stream) {
  clear_error();
  BT_ARG_CHECK(g && cam, "NULL pointer");
  BT_ARG_CHECK(g->set->standalone, "the grid belongs to a set: build the set (bt_batch_build)");
  return batch_build(g->set, cam, &a, 1, startlevel, o, (cudaStream_t)stream);
}

int bt_grid_query(bt_grid* g, bt_grid_info* info, void* stream) {
  clear_error();
  BT_ARG_CHECK(g && info, "NULL pointer");
  BT_ARG_CHECK(g->built, "grid not built");
  BT_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  const GridCounters& c = *g->ctr_host;
  std::memset(info, 0, sizeof(*info));
  info->N = g->L.N;
  info->M = g->L.M;
  info->maxlevel = g->L.maxlevel;
  info->startlevel = g->L.startlevel;
  info->angle = g->L.eq;
  info->traced = ((int64_t)c.traced_hi << 32) | c.traced_lo;
  info->n_leaf_blocks = c.n_leaf + 0;
  info->flags = c.err | (c.overflow ? 4u : 0u);
  info->thphi = (double*)g->L.thphi;
  info->steps = g->L.steps;
  info->exists = g->L.vflag;
  info->blevel = g->L.blevel;
  info->status = g->L.vstat;
  info->launches = g->set->launches;
  info->trace_ms = batch_trace_ms(g->set);
  info->trace_launches = g->set->n_ev / 2;
  if (info->flags) {
    set_error("grid build flags 0x%x (1: T-vertex fix did not converge, "
              "2: fix stack overflow, 4: work list overflow, 8: the flow gave up waiting, "
              "16: the flow refined a block early that the level form would not)",
              info->flags);
    return BT_ERR_NUMERIC;
  }
  return BT_OK;
}

int bt_grid_set_timing(bt_grid* g, int on) {
  BT_ARG_CHECK(g != nullptr, "NULL grid");
  return batch_set_timing(g->set, on);
}

int bt_grid_set_graph(bt_grid* g, int on) {
  BT_ARG_CHECK(g != nullptr, "NULL grid");
  g->set->graph = on ? 1 : 0;
  return BT_OK;
}

int bt_grid_set_flow(bt_grid* g, int on) {
  clear_error();
  BT_ARG_CHECK(g != nullptr, "NULL grid");
  return batch_set_flow(g->set, on);
}

int bt_grid_set_shape(bt_grid* g, const bt_trace_shape* shape) {
  clear_error();
  BT_ARG_CHECK(g != nullptr, "NULL grid");
  return bt_batch_set_shape(g->set, shape);
}

int bt_grid_tune(bt_grid* g, const bt_integ_opts* o, double p99_target_rad, int repeats,
                 bt_tune_result* out, void* stream) {
  clear_error();
  BT_ARG_CHECK(g != nullptr, "NULL grid");
  BT_ARG_CHECK(g->set->standalone, "a member of a set: tune the set");
  BT_ARG_CHECK(g->built, "grid not built");
  const bt_camera cam = g->cam;
  const double a = g->a;
  return bt_batch_tune(g->set, &cam, &a, g->L.startlevel, o, p99_target_rad, repeats, out,
                       stream);
}

int bt_grid_set_tfix_passes(bt_grid* g, int passes) {
  clear_error();
  BT_ARG_CHECK(g != nullptr, "NULL grid");
  BT_ARG_CHECK(passes >= 1 && passes <= kMaxTfixPasses, "passes must be in [1, 8]");
  g->set->tfix_passes = passes;
  return BT_OK;
}

int bt_grid_set_flow_drop(bt_grid* g) {
  clear_error();
  BT_ARG_CHECK(g != nullptr, "NULL grid");
  BT_ARG_CHECK(g->set->flow, "the one-launch build is off (bt_grid_set_flow)");
  BT_ARG_CHECK(!g->set->graph, "graph replay is on: the drop applies to one eager build");
  g->set->flow_drop = 1;
  return BT_OK;
}

int bt_grid_set_tfix_launch(bt_grid* g, int cooperative) {
  clear_error();
  BT_ARG_CHECK(g != nullptr, "NULL grid");
  g->set->tfix_coop = cooperative ? 1 : 0;
  return BT_OK;
}

int bt_grid_export_dense(const bt_grid* g, double* theta, double* phi,
                         uint8_t* exists, int32_t* steps, int8_t* blevel,
                         uint8_t* status, void* stream) {
  clear_error();
  BT_ARG_CHECK(g != nullptr, "NULL grid");
  BT_ARG_CHECK(g->built, "grid not built");
  const size_t NM = (size_t)g->L.N * g->L.M;
  k_export_dense<<<grid_blocks(NM, 256), 256, 0, (cudaStream_t)stream>>>(
      g->L, theta, phi, exists, steps, blevel, status);
  BT_CUDA_TRY(cudaGetLastError());
  return BT_OK;
}

int bt_grid_export(bt_grid* g, bt_grid_export_t* out, void* stream) {
  clear_error();
  BT_ARG_CHECK(g && out, "NULL pointer");
  BT_ARG_CHECK(g->built, "grid not built");
  cudaStream_t s = (cudaStream_t)stream;
  const int N = g->L.N;
  k_row_count<<<N, 256, 0, s>>>(g->L.vflag, g->L.blevel, g->L.M, g->rowv, g->rowb);
  k_row_scan<<<1, 1024, 0, s>>>(g->rowv, g->rowb, N, g->totals);
  BT_CUDA_TRY(cudaGetLastError());
  BT_CUDA_TRY(cudaMemcpyAsync(g->totals_host, g->totals, 2 * sizeof(uint64_t),
                              cudaMemcpyDeviceToHost, s));
  BT_CUDA_TRY(cudaStreamSynchronize(s));
  const size_t nv = g->totals_host[0], nb = g->totals_host[1];
  out->n_vertices = nv;
  out->n_blocks = nb;
  if (nv > out->cap_vertices || nb > out->cap_blocks) {
    set_error("export capacity too small: need %zu vertices, %zu blocks", nv, nb);
    return BT_ERR_ARG;
  }
  // stage on the device in key order, then one copy per array to the
  // caller's buffers (host or device)
  const size_t need = nv * (4 + 4 + 8 + 8 + 4) + nb * (4 + 4 + 1) + 64;
  if (g->compact_bytes < need) {
    if (g->compact) cudaFree(g->compact);
    g->compact = nullptr;
    g->compact_bytes = 0;
    cudaError_t e = cudaMalloc((void**)&g->compact, need);
    if (e != cudaSuccess) {
      set_error("export staging allocation failed: %s", cudaGetErrorString(e));
      return BT_ERR_NOMEM;
    }
    g->compact_bytes = need;
  }
  CompactOut o;
  char* p = g->compact;
  o.th = (double*)p; p += nv * 8;
  o.ph = (double*)p; p += nv * 8;
  o.vi = (uint32_t*)p; p += nv * 4;
  o.vj = (uint32_t*)p; p += nv * 4;
  o.st = (int32_t*)p; p += nv * 4;
  o.bi = (uint32_t*)p; p += nb * 4;
  o.bj = (uint32_t*)p; p += nb * 4;
  o.blv = (int8_t*)p;
  k_row_compact<<<N, 256, 0, s>>>(g->L, g->rowv, g->rowb, o);
  BT_CUDA_TRY(cudaGetLastError());
  struct { void* dst; const void* src; size_t bytes; } cp[] = {
      {out->theta, o.th, nv * 8}, {out->phi, o.ph, nv * 8}, {out->vi, o.vi, nv * 4},
      {out->vj, o.vj, nv * 4},    {out->steps, o.st, nv * 4}, {out->bi, o.bi, nb * 4},
      {out->bj, o.bj, nb * 4},    {out->level, o.blv, nb}};
  for (auto& c : cp)
    if (c.dst && c.bytes)
      BT_CUDA_TRY(cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDefault, s));
  return BT_OK;
}


int bt_grid_map_export(bt_grid* g, const float** grid_out, int32_t* rows,
                       int32_t* cols, int32_t* sym, void* stream) {
  clear_error();
  BT_ARG_CHECK(g && grid_out, "NULL pointer");
  BT_ARG_CHECK(g->built, "grid not built");
  const int GN = g->L.N, GM = g->L.M;
  // dev_sym, BT/MakeImageKernel.cu:1259-1260
  const int symv = (float)GM / (float)GN > 3 ? 1 : 0;
  const int GN1 = symv ? 2 * GN - 1 : GN;
  if (!g->mapgrid) {
    cudaError_t e = cudaMalloc((void**)&g->mapgrid, (size_t)GN1 * GM * sizeof(float2));
    if (e != cudaSuccess) {
      set_error("map grid allocation failed: %s", cudaGetErrorString(e));
      return BT_ERR_NOMEM;
    }
  }
  g->sym = symv;
  g->map_rows = GN1;
  k_export_map<<<grid_blocks((size_t)GN * GM, 256), 256, 0, (cudaStream_t)stream>>>(
      g->L, g->mapgrid, GN1, symv);
  BT_CUDA_TRY(cudaGetLastError());
  *grid_out = (const float*)g->mapgrid;
  if (rows) *rows = GN1;
  if (cols) *cols = GM;
  if (sym) *sym = symv;
  return BT_OK;
}


int bt_batch_create(int maxlevel, int angle, int count, bt_batch** out) {
  clear_error();
  return batch_create(maxlevel, angle, count, out);
}

void bt_batch_destroy(bt_batch* b) {
  if (b && !b->standalone) batch_free(b);
}

int bt_batch_build(bt_batch* b, const bt_camera* cams, const double* spins, int startlevel,
                   const bt_integ_opts* o, void* stream) {
  clear_error();
  BT_ARG_CHECK(b != nullptr, "NULL set");
  return batch_build(b, cams, spins, b->G, startlevel, o, (cudaStream_t)stream);
}

int bt_batch_build_first(bt_batch* b, int n, const bt_camera* cams, const double* spins,
                         int startlevel, const bt_integ_opts* o, void* stream) {
  clear_error();
  BT_ARG_CHECK(b != nullptr, "NULL set");
  return batch_build(b, cams, spins, n, startlevel, o, (cudaStream_t)stream);
}

bt_grid* bt_batch_grid(bt_batch* b, int k) {
  if (!b || k < 0 || k >= b->G) return nullptr;
  return &b->grids[k];
}

int bt_batch_set_graph(bt_batch* b, int on) {
  BT_ARG_CHECK(b != nullptr, "NULL set");
  b->graph = on ? 1 : 0;
  return BT_OK;
}

int bt_batch_set_flow(bt_batch* b, int on) {
  clear_error();
  BT_ARG_CHECK(b != nullptr, "NULL set");
  return batch_set_flow(b, on);
}

int bt_batch_set_timing(bt_batch* b, int on) {
  BT_ARG_CHECK(b != nullptr, "NULL set");
  return batch_set_timing(b, on);
}

int bt_batch_set_shape(bt_batch* b, const bt_trace_shape* shape) {
  clear_error();
  BT_ARG_CHECK(b && shape, "NULL pointer");
  BT_ARG_CHECK(shape->threads == 64 || shape->threads == 128 || shape->threads == 256,
               "threads must be 64, 128 or 256");
  BT_ARG_CHECK(shape->blocks_per_sm >= 0 && shape->blocks_per_sm <= 32,
               "blocks_per_sm out of [0, 32]");
  BT_ARG_CHECK(shape->refill >= 0 && shape->refill <= 32, "refill out of [0, 32]");
  b->shape = TraceShape{shape->threads, shape->blocks_per_sm, shape->refill};
  return BT_OK;
}

int bt_batch_query(bt_batch* b, bt_batch_info* info, void* stream) {
  clear_error();
  BT_ARG_CHECK(b && info, "NULL pointer");
  BT_ARG_CHECK(b->built, "set not built");
  BT_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  std::memset(info, 0, sizeof(*info));
  info->count = b->built_n;
  for (int g = 0; g < b->built_n; g++) {
    const GridCounters& c = b->ctr_host[g];
    info->traced += ((int64_t)c.traced_hi << 32) | c.traced_lo;
    info->flags |= c.err | (c.overflow ? 4u : 0u);
  }
  info->trace_ms = batch_trace_ms(b);
  info->trace_launches = b->n_ev / 2;
  info->launches = b->launches;
  info->graph = b->graph;
  info->shape.threads = b->shape.threads;
  info->shape.blocks_per_sm = b->shape.blocks_per_sm;
  info->shape.refill = b->shape.refill;
  if (info->flags) {
    set_error("grid set build flags 0x%x", info->flags);
    return BT_ERR_NUMERIC;
  }
  return BT_OK;
}

int bt_batch_autotune(bt_batch* b, const bt_camera* cams, const double* spins, int startlevel,
                      const bt_integ_opts* o, int repeats, bt_trace_shape* best,
                      float* best_ms, void* stream) {
  clear_error();
  BT_ARG_CHECK(b != nullptr, "NULL set");
  BT_ARG_CHECK(repeats >= 1 && repeats <= 100, "repeats out of [1, 100]");
  cudaStream_t s = (cudaStream_t)stream;
  const TraceShape saved = b->shape;
  const int graph = b->graph;
  b->graph = 0;  // time eager builds; the chosen shape is captured later
  static const TraceShape cand[] = {{128, 0}, {128, 4}, {128, 5}, {64, 0}, {256, 0}};
  cudaEvent_t e0, e1;
  BT_CUDA_TRY(cudaEventCreate(&e0));
  BT_CUDA_TRY(cudaEventCreate(&e1));
  float best_t = 3.4e38f;
  TraceShape best_s = saved;
  int rc = BT_OK;
  for (const TraceShape& c : cand) {
    b->shape = c;
    if ((rc = batch_build(b, cams, spins, b->G, startlevel, o, s))) break;  // warm-up
    float t_min = 3.4e38f;
    for (int r = 0; r < repeats && rc == BT_OK; r++) {
      cudaEventRecord(e0, s);
      rc = batch_build(b, cams, spins, b->G, startlevel, o, s);
      cudaEventRecord(e1, s);
      if (cudaEventSynchronize(e1) != cudaSuccess) rc = BT_ERR_CUDA;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms < t_min) t_min = ms;
    }
    if (rc) break;
    if (t_min < best_t) {
      best_t = t_min;
      best_s = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->graph = graph;
  b->shape = rc == BT_OK ? best_s : saved;
  if (rc) return rc;
  if (best) {
    best->threads = best_s.threads;
    best->blocks_per_sm = best_s.blocks_per_sm;
    best->refill = best_s.refill;
  }
  if (best_ms) *best_ms = best_t;
  return BT_OK;
}

}  // extern "C"

namespace {

constexpr double kTunePi = 3.14159265358979323846;

// splitmix64: the tuner's seeded sample directions.
uint64_t tune_mix(uint64_t& x) {
  uint64_t z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// p99 of max(|d theta|, |d phi| wrapped to [-pi, pi]) over the rays that
// escaped in both runs; -1 when there are none.
double tune_p99(const std::vector<double>& t0, const std::vector<double>& p0,
                const std::vector<uint8_t>& s0, const std::vector<double>& t1,
                const std::vector<double>& p1, const std::vector<uint8_t>& s1) {
  std::vector<double> e;
  e.reserve(t0.size());
  for (size_t k = 0; k < t0.size(); k++) {
    if (s0[k] != BT_RAY_ESCAPED || s1[k] != BT_RAY_ESCAPED) continue;
    double dp = std::fabs(p0[k] - p1[k]);
    dp = std::fmod(dp, 2 * kTunePi);
    if (dp > kTunePi) dp = 2 * kTunePi - dp;
    e.push_back(std::max(std::fabs(t0[k] - t1[k]), dp));
  }
  if (e.empty()) return -1;
  const size_t at = std::min(e.size() - 1, (size_t)std::ceil(0.99 * (double)e.size()) - 1);
  std::nth_element(e.begin(), e.begin() + at, e.end());
  return e[at];
}

// The MIXED form's FP64 band by accuracy (see bt_batch_tune).
int tune_band(const bt_camera* cams, const double* spins, int G, const bt_integ_opts& o,
              double target, cudaStream_t s, double* band, double* p99, int* met) {
  static const double cand[] = {0.05, 0.1, 0.2, 0.5, 1.0, 2.0, 5.0};
  const int ncam = std::min(G, 8), per = 2048;
  const size_t n = (size_t)ncam * per;
  std::vector<double> th(n), ph(n);
  uint64_t seed = 20261204;
  for (size_t k = 0; k < n; k++) {
    const double u = (double)(tune_mix(seed) >> 11) * 0x1.0p-53;
    const double v = (double)(tune_mix(seed) >> 11) * 0x1.0p-53;
    th[k] = std::acos(1 - 2 * u);
    ph[k] = 2 * kTunePi * v;
  }
  double* d = nullptr;  // th, ph, theta out, phi out
  int32_t* steps = nullptr;
  uint8_t* st = nullptr;
  cudaError_t e = cudaMalloc((void**)&d, 4 * n * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc((void**)&steps, n * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMalloc((void**)&st, n);
  if (e != cudaSuccess) {
    cudaFree(d);
    cudaFree(steps);
    set_error("tuner sample buffers: %s", cudaGetErrorString(e));
    return BT_ERR_NOMEM;
  }
  int rc = BT_OK;
  auto run = [&](const bt_integ_opts& oo, std::vector<double>& to, std::vector<double>& po,
                 std::vector<uint8_t>& so) -> int {
    for (int c = 0; c < ncam; c++) {
      const size_t at = (size_t)c * per;
      if (int r = bt_integrate_rays(&cams[c], spins[c], d + at, d + n + at, per, d + 2 * n + at,
                                    d + 3 * n + at, steps + at, st + at, &oo, s))
        return r;
    }
    to.resize(n);
    po.resize(n);
    so.resize(n);
    if (cudaMemcpyAsync(to.data(), d + 2 * n, n * sizeof(double), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaMemcpyAsync(po.data(), d + 3 * n, n * sizeof(double), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaMemcpyAsync(so.data(), st, n, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      set_error("tuner sample copies failed");
      return BT_ERR_CUDA;
    }
    return BT_OK;
  };
  std::vector<double> t0, p0, t1, p1;
  std::vector<uint8_t> s0, s1;
  if (cudaMemcpyAsync(d, th.data(), n * sizeof(double), cudaMemcpyHostToDevice, s) !=
          cudaSuccess ||
      cudaMemcpyAsync(d + n, ph.data(), n * sizeof(double), cudaMemcpyHostToDevice, s) !=
          cudaSuccess) {
    set_error("tuner sample copies failed");
    rc = BT_ERR_CUDA;
  }
  bt_integ_opts op = o;
  op.precision = BT_PRECISION_PLAIN;
  if (rc == BT_OK) rc = run(op, t0, p0, s0);
  double best_e = 3.4e38;
  *met = 0;
  for (double c : cand) {
    if (rc) break;
    bt_integ_opts om = o;
    om.fp64_band = c;
    if ((rc = run(om, t1, p1, s1))) break;
    const double q = tune_p99(t0, p0, s0, t1, p1, s1);
    if (q >= 0 && q <= target) {
      *band = c;
      *p99 = q;
      *met = 1;
      break;
    }
    if (q >= 0 && q < best_e) {
      best_e = q;
      *band = c;
      *p99 = q;
    }
  }
  cudaFree(d);
  cudaFree(steps);
  cudaFree(st);
  return rc;
}

}  // namespace

extern "C" {

int bt_batch_tune(bt_batch* b, const bt_camera* cams, const double* spins, int startlevel,
                  const bt_integ_opts* o, double p99_target_rad, int repeats,
                  bt_tune_result* out, void* stream) {
  clear_error();
  BT_ARG_CHECK(b && cams && spins && out, "NULL pointer");
  BT_ARG_CHECK(repeats >= 1 && repeats <= 100, "repeats out of [1, 100]");
  BT_ARG_CHECK(p99_target_rad > 0, "p99 target must be positive");
  cudaStream_t s = (cudaStream_t)stream;
  bt_integ_opts opt;
  if (o) opt = *o;
  else bt_integ_opts_default(&opt);
  std::memset(out, 0, sizeof(*out));
  out->fp64_band = opt.fp64_band;
  out->band_p99_rad = -1;
  if (opt.precision == BT_PRECISION_MIXED) {
    if (int rc = tune_band(cams, spins, b->G, opt, p99_target_rad, s, &out->fp64_band,
                           &out->band_p99_rad, &out->band_met))
      return rc;
    opt.fp64_band = out->fp64_band;
  }
  // configurations: level builds (shape x refill), then one-launch builds
  struct Conf {
    TraceShape shape;
    int flow;
  };
  std::vector<Conf> conf;
  // as many blocks as fit, the capped register budgets, and fewer warps per
  // SM (a lone grid's longest rays run faster on lightly loaded SMs)
  static const TraceShape shapes[] = {{128, 0, 0}, {128, 4, 0}, {128, 5, 0}, {64, 0, 0},
                                      {256, 0, 0}, {128, 2, 0}, {128, 1, 0}};
  for (const TraceShape& sh : shapes)
    for (int r : {4, 8, 16}) conf.push_back({TraceShape{sh.threads, sh.blocks_per_sm, r}, 0});
  for (int f : {1, 2}) conf.push_back({b->shape, f});
  const TraceShape saved = b->shape;
  const int saved_flow = b->flow, graph = b->graph;
  b->graph = 0;  // time eager builds; the chosen configuration is captured later
  cudaEvent_t e0, e1;
  BT_CUDA_TRY(cudaEventCreate(&e0));
  BT_CUDA_TRY(cudaEventCreate(&e1));
  float best_t = 3.4e38f, best_level = 3.4e38f, best_flow = 3.4e38f;
  Conf best = {saved, saved_flow};
  int rc = BT_OK;
  for (const Conf& c : conf) {
    b->shape = c.shape;
    if (c.flow) {
      if (batch_set_flow(b, c.flow) != BT_OK) {  // no room for its buffers: skip
        clear_error();
        b->flow = 0;
        continue;
      }
    } else {
      b->flow = 0;
    }
    if ((rc = batch_build(b, cams, spins, b->G, startlevel, &opt, s))) break;  // warm-up
    float t_min = 3.4e38f;
    for (int r = 0; r < repeats && rc == BT_OK; r++) {
      cudaEventRecord(e0, s);
      rc = batch_build(b, cams, spins, b->G, startlevel, &opt, s);
      cudaEventRecord(e1, s);
      if (cudaEventSynchronize(e1) != cudaSuccess) rc = BT_ERR_CUDA;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms < t_min) t_min = ms;
    }
    if (rc) break;
    out->candidates++;
    if (c.flow) best_flow = std::min(best_flow, t_min);
    else best_level = std::min(best_level, t_min);
    if (t_min < best_t) {
      best_t = t_min;
      best = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->graph = graph;
  if (rc) {
    b->shape = saved;
    b->flow = saved_flow;
    return rc;
  }
  b->shape = best.shape;
  b->flow = best.flow;
  out->shape.threads = best.shape.threads;
  out->shape.blocks_per_sm = best.shape.blocks_per_sm;
  out->shape.refill = best.shape.refill;
  out->flow = best.flow;
  out->best_ms = best_t;
  out->level_ms = best_level < 3.4e38f ? best_level : 0.f;
  out->flow_ms = best_flow < 3.4e38f ? best_flow : 0.f;
  return BT_OK;
}

}  // extern "C"
