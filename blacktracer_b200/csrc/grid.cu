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
#include <cmath>
#include <cstring>
#include <new>

#include "bt_internal.h"

namespace bt {

constexpr int kMaxTfixPasses = 8;

struct GridBuffers {
  uint32_t* list[2];  // block lists of consecutive levels (ping-pong)
  uint32_t* trace;    // vertices to trace this level
  uint32_t* leaves;   // leaf blocks (level < max) in level order
  double2* X[2];      // T-vertex fix pass buffers
  size_t cap;         // capacity of each list (entries)
};

}  // namespace bt

struct bt_grid {
  bt::LatticeView L;
  bt::GridBuffers B;
  bt::GridCounters* ctr;       // device
  bt::GridCounters* ctr_host;  // pinned mirror
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
  int launches;     // kernels launched by the last build
  int timing;       // record CUDA events around the trace launches
  cudaEvent_t ev[2 * 16];
  int n_ev;
  int32_t map_rows;
  int sym;
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

__global__ void k_seed(LatticeView L, SeedShape S, uint32_t* trace,
                       uint32_t* check, GridCounters* ctr) {
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
    ctr->n_check = S.cols + (uniform ? 0 : S.brows * S.cols);
    ctr->n_next = 0;
    ctr->fetch = 0;
    ctr->tfix_flags[1] = 1;
  }
}

// Pole copies of raytrace (BT/Grid.h:303-315), after the poles are traced.
__global__ void k_pole_copy(LatticeView L) {
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

// ------------------------------------------------------------ refinement
__device__ __forceinline__ void claim_vertex(const LatticeView& L, uint32_t i,
                                             uint32_t j, uint32_t* trace,
                                             GridCounters* ctr) {
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
  const uint32_t slot = atomicAdd(&ctr->n_trace, 1u);
  trace[slot] = key;
}

// One level of adaptiveBlockIntegration (BT/Grid.h:476-497) with
// refineCheck (:410-445) and fillVector (:453-459).
__global__ void k_refine(LatticeView L, int level, const uint32_t* check,
                         uint32_t* next, uint32_t* trace, uint32_t* leaves,
                         GridCounters* ctr) {
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
    claim_vertex(L, kh, j, trace, ctr);
    claim_vertex(L, kh, lh, trace, ctr);
    claim_vertex(L, i, lh, trace, ctr);
    claim_vertex(L, i + gap, lh, trace, ctr);
    claim_vertex(L, kh, (j + gap) % M, trace, ctr);
    const uint32_t s = atomicAdd(&ctr->n_next, 4u);
    next[s + 0] = key;
    next[s + 1] = kh * M + j;
    next[s + 2] = kh * M + lh;
    next[s + 3] = i * M + lh;
  }
}

// Level hand-over.  after_seed: only account the seeded rays; otherwise the
// next list becomes the check list and the leaf offset of `slot` is set.
__global__ void k_advance(GridCounters* ctr, int after_seed, int slot) {
  uint64_t t = ((uint64_t)ctr->traced_hi << 32 | ctr->traced_lo) + ctr->n_trace;
  ctr->traced_lo = (uint32_t)t;
  ctr->traced_hi = (uint32_t)(t >> 32);
  ctr->n_trace = 0;
  ctr->fetch = 0;
  if (!after_seed) {
    ctr->n_check = ctr->n_next;
    ctr->n_next = 0;
  }
  if (slot >= 0 && slot < 16) ctr->leaf_off[slot] = ctr->n_leaf;
}

// Blocks left at the last level get level = MAXLEVEL (BT/Grid.h:503-504).
__global__ void k_finalize(LatticeView L, const uint32_t* check,
                           GridCounters* ctr) {
  const uint32_t n = *(volatile uint32_t*)&ctr->n_check;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += gridDim.x * blockDim.x)
    L.blevel[check[t]] = (int8_t)L.maxlevel;
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

// checkAdjacentBlock (BT/Grid.h:132-177) as an explicit pre-order DFS.
// Returns true if any written value differs from the previous pass.
__device__ bool fix_edge(const TfixArgs& A, const Edge& E) {
  const LatticeView& L = A.L;
  const uint32_t M = L.M, N = L.N;
  struct Frame { uint32_t a, b; int lv; };
  Frame stack[16];
  int sp = 0;
  stack[sp++] = {0u, E.g, A.level};
  bool changed = false;
  while (sp > 0) {
    const Frame f = stack[--sp];
    const uint32_t h = f.b - f.a;
    const uint32_t ia = E.i0 + E.udlr * f.a, ja = E.j0 + (1 - E.udlr) * f.a;
    uint32_t ib, jb;
    if (f.b == E.g) {
      ib = E.i0 + E.udlr * E.g;
      jb = (E.j0 + (1 - E.udlr) * E.g) % M;
    } else {
      ib = E.i0 + E.udlr * f.b;
      jb = E.j0 + (1 - E.udlr) * f.b;
    }
    const uint32_t im = ia + E.udlr * h / 2, jm = ja + (1 - E.udlr) * h / 2;
    if (!vexists(L, im, jm)) continue;
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
    const double2 va = read_vertex(A, E, ia, ja, f.a, f.b);
    const double2 vb = read_vertex(A, E, ib, jb, f.a, f.b);
    if (vexists(L, iprev, jprev) && vexists(L, inext, jnext)) {
      const double2 vp = read_vertex(A, E, iprev, jprev, f.a, f.b);
      const double2 vn = read_vertex(A, E, inext, jnext, f.a, f.b);
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
    if (f.lv + 1 == L.maxlevel) continue;
    const uint32_t mo = f.a + h / 2;
    if (sp + 2 <= 16) {
      stack[sp++] = {mo, f.b, f.lv + 1};  // right half after the left one
      stack[sp++] = {f.a, mo, f.lv + 1};
    } else {
      atomicOr(&A.ctr->err, 2u);
    }
  }
  return changed;
}

__global__ void k_tfix_pass(TfixArgs A) {
  GridCounters* ctr = A.ctr;
  if (A.pass > 1 && *(volatile uint32_t*)&ctr->tfix_flags[A.pass - 1] == 0)
    return;  // converged already
  const uint32_t lo = ctr->leaf_off[A.lo], hi = ctr->leaf_off[A.hi_slot];
  const LatticeView& L = A.L;
  const uint32_t M = L.M;
  const uint32_t g = pow2u(L.maxlevel - A.level);
  bool changed = false;
  for (uint32_t t = lo + blockIdx.x * blockDim.x + threadIdx.x; t < hi;
       t += gridDim.x * blockDim.x) {
    const uint32_t key = A.leaves[t];
    const uint32_t i = key / M, j = key % M;
    if (L.thphi[key].y < 0) continue;  // BT/Grid.h:107
    const uint32_t k = i + g, l = (j + g) % M;
    Edge e0 = {i, j, 1, g, rank_of(i, j, 0)};
    Edge e1 = {i, j, 0, g, rank_of(i, j, 1)};
    Edge e2 = {i, l, 1, g, rank_of(i, j, 2)};
    Edge e3 = {k, j, 0, g, rank_of(i, j, 3)};
    changed |= fix_edge(A, e0);
    changed |= fix_edge(A, e1);
    changed |= fix_edge(A, e2);
    changed |= fix_edge(A, e3);
  }
  if (__any_sync(0xffffffffu, changed) && (threadIdx.x & 31) == 0)
    atomicOr(&ctr->tfix_flags[A.pass], 1u);
}

// Copies the converged values of a level's T-vertices into the lattice.
__global__ void k_tfix_commit(TfixArgs A) {
  GridCounters* ctr = A.ctr;
  const uint32_t lo = ctr->leaf_off[A.lo], hi = ctr->leaf_off[A.hi_slot];
  const LatticeView& L = A.L;
  const uint32_t M = L.M;
  const uint32_t g = pow2u(L.maxlevel - A.level);
  for (uint32_t t = lo + blockIdx.x * blockDim.x + threadIdx.x; t < hi;
       t += gridDim.x * blockDim.x) {
    const uint32_t key = A.leaves[t];
    const uint32_t i = key / M, j = key % M;
    if (L.thphi[key].y < 0) continue;
    const uint32_t k = i + g, l = (j + g) % M;
    const uint32_t si[4] = {i, i, i, k}, sj[4] = {j, j, l, j};
    const int ud[4] = {1, 0, 1, 0};
    for (int e = 0; e < 4; e++)
      for (uint32_t o = 1; o < g; o++) {
        const uint32_t ip = si[e] + ud[e] * o, jp = sj[e] + (1 - ud[e]) * o;
        const size_t id = (size_t)ip * M + jp;
        if (L.vflag[id] == 1) L.thphi[id] = A.Xcur[id];
      }
  }
}

__global__ void k_tfix_check(GridCounters* ctr, int passes) {
  bool conv = false;
  for (int t = 2; t <= passes; t++)
    if (ctr->tfix_flags[t] == 0) conv = true;
  if (!conv) ctr->err |= 1u;
  for (int t = 0; t < 16; t++) ctr->tfix_flags[t] = 0;
  ctr->tfix_flags[1] = 1;
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

// Exclusive scan of N row counts in one block (N <= 16385 rows).
__global__ void k_row_scan(uint32_t* vcount, uint32_t* bcount, int N, uint64_t* totals) {
  if (threadIdx.x != 0) return;
  uint64_t sv = 0, sb = 0;
  for (int i = 0; i < N; i++) {
    const uint32_t v = vcount[i], b = bcount[i];
    vcount[i] = (uint32_t)sv;
    bcount[i] = (uint32_t)sb;
    sv += v;
    sb += b;
  }
  totals[0] = sv;
  totals[1] = sb;
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

}  // namespace bt

using namespace bt;

static void grid_free_buffers(bt_grid* g) {
  void* ptrs[] = {g->L.thphi, g->L.steps, g->L.vflag, g->L.vstat, g->L.blevel,
                  g->B.list[0], g->B.list[1], g->B.trace, g->B.leaves,
                  g->B.X[0], g->B.X[1], g->ctr, g->mapgrid,
                  g->rowv, g->rowb, g->totals, g->compact};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (g->ctr_host) cudaFreeHost(g->ctr_host);
  if (g->totals_host) cudaFreeHost(g->totals_host);
}

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
  int32_t N, M;
  int rc = bt_grid_dims(maxlevel, angle, &N, &M);
  if (rc) return rc;
  bt_grid* g = new (std::nothrow) bt_grid;
  if (!g) return BT_ERR_NOMEM;
  std::memset(g, 0, sizeof(*g));
  g->L.N = N;
  g->L.M = M;
  g->L.eq = angle ? 1 : 0;
  g->L.maxlevel = maxlevel;
  const size_t NM = (size_t)N * M;
  g->B.cap = NM;
  cudaError_t e = cudaSuccess;
#define GALLOC(ptr, bytes)                                   \
  if (e == cudaSuccess) e = cudaMalloc((void**)&(ptr), (bytes));
  GALLOC(g->L.thphi, NM * sizeof(double2));
  GALLOC(g->L.steps, NM * sizeof(int32_t));
  GALLOC(g->L.vflag, NM + 4);
  GALLOC(g->L.vstat, NM);
  GALLOC(g->L.blevel, NM);
  GALLOC(g->B.list[0], NM * sizeof(uint32_t));
  GALLOC(g->B.list[1], NM * sizeof(uint32_t));
  GALLOC(g->B.trace, NM * sizeof(uint32_t));
  GALLOC(g->B.leaves, NM * sizeof(uint32_t));
  GALLOC(g->B.X[0], NM * sizeof(double2));
  GALLOC(g->B.X[1], NM * sizeof(double2));
  GALLOC(g->ctr, sizeof(GridCounters));
  GALLOC(g->rowv, (size_t)N * sizeof(uint32_t));
  GALLOC(g->rowb, (size_t)N * sizeof(uint32_t));
  GALLOC(g->totals, 2 * sizeof(uint64_t));
#undef GALLOC
  if (e == cudaSuccess) e = cudaMallocHost((void**)&g->ctr_host, sizeof(GridCounters));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&g->totals_host, 2 * sizeof(uint64_t));
  if (e != cudaSuccess) {
    set_error("grid allocation (N=%d M=%d) failed: %s", N, M, cudaGetErrorString(e));
    grid_free_buffers(g);
    delete g;
    return BT_ERR_NOMEM;
  }
  *out = g;
  return BT_OK;
}

void bt_grid_destroy(bt_grid* g) {
  if (!g) return;
  if (g->timing)
    for (int k = 0; k < 2 * 16; k++) cudaEventDestroy(g->ev[k]);
  grid_free_buffers(g);
  delete g;
}

int bt_grid_build(bt_grid* g, const bt_camera* cam, double a, int startlevel,
                  const bt_integ_opts* o, void* stream) {
  clear_error();
  BT_ARG_CHECK(g && cam, "NULL pointer");
  BT_ARG_CHECK(startlevel >= 1 && startlevel <= g->L.maxlevel,
               "startlevel out of [1, maxlevel]");
  BT_ARG_CHECK(g->L.maxlevel - startlevel <= 12,
               "maxlevel - startlevel > 12 is not supported");
  RayParams p;
  if (make_ray_params(cam, a, o, &p)) {
    set_error("invalid camera or integrator options");
    return BT_ERR_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  g->params = p;
  g->cam = *cam;
  g->a = a;
  g->L.startlevel = startlevel;
  g->built = 0;
  LatticeView L = g->L;
  const size_t NM = (size_t)L.N * L.M;
  BT_CUDA_TRY(cudaMemsetAsync(L.vflag, 0, NM + 4, s));
  BT_CUDA_TRY(cudaMemsetAsync(L.vstat, 0, NM, s));
  BT_CUDA_TRY(cudaMemsetAsync(L.steps, 0, NM * sizeof(int32_t), s));
  BT_CUDA_TRY(cudaMemsetAsync(L.blevel, 0xff, NM, s));
  BT_CUDA_TRY(cudaMemsetAsync(g->ctr, 0, sizeof(GridCounters), s));
  g->n_ev = 0;
  auto trace = [&]() -> int {
    const bool t = g->timing && g->n_ev + 2 <= 2 * 16;
    if (t) BT_CUDA_TRY(cudaEventRecord(g->ev[g->n_ev], s));
    const int rc = p.precision == BT_PRECISION_MIXED
                       ? launch_trace_mixed(p, L, g->B.trace, g->ctr, s)
                       : launch_trace_plain(p, L, g->B.trace, g->ctr, s);
    if (t) {
      BT_CUDA_TRY(cudaEventRecord(g->ev[g->n_ev + 1], s));
      g->n_ev += 2;
    }
    return rc;
  };
  const SeedShape S = seed_shape(L);
  k_seed<<<grid_blocks((size_t)(S.rows + 1) * S.cols, 256), 256, 0, s>>>(
      L, S, g->B.trace, g->B.list[0], g->ctr);
  BT_CUDA_TRY(cudaGetLastError());
  if (int rc = trace()) return rc;
  k_pole_copy<<<grid_blocks(S.cols, 256), 256, 0, s>>>(L);
  k_advance<<<1, 1, 0, s>>>(g->ctr, 1, 0);
  BT_CUDA_TRY(cudaGetLastError());
  int cur = 0;
  for (int level = startlevel; level < L.maxlevel; level++) {
    k_refine<<<grid_blocks(NM / 4, 256), 256, 0, s>>>(
        L, level, g->B.list[cur], g->B.list[cur ^ 1], g->B.trace, g->B.leaves,
        g->ctr);
    BT_CUDA_TRY(cudaGetLastError());
    if (int rc = trace()) return rc;
    k_advance<<<1, 1, 0, s>>>(g->ctr, 0, level - startlevel + 1);
    BT_CUDA_TRY(cudaGetLastError());
    cur ^= 1;
  }
  k_finalize<<<grid_blocks(NM / 4, 256), 256, 0, s>>>(L, g->B.list[cur], g->ctr);
  BT_CUDA_TRY(cudaGetLastError());
  // T-vertex fix, level by level (coarse to fine)
  for (int level = startlevel; level < L.maxlevel; level++) {
    TfixArgs A;
    A.L = L;
    A.level = level;
    A.leaves = g->B.leaves;
    A.lo = level - startlevel;
    A.hi_slot = level - startlevel + 1;
    A.ctr = g->ctr;
    const unsigned nb = grid_blocks(NM / 16, 128);
    for (int pass = 1; pass <= kMaxTfixPasses; pass++) {
      A.pass = pass;
      A.Xcur = g->B.X[pass & 1];
      A.Xprev = g->B.X[(pass - 1) & 1];
      k_tfix_pass<<<nb, 128, 0, s>>>(A);
      BT_CUDA_TRY(cudaGetLastError());
    }
    A.Xcur = g->B.X[0];
    k_tfix_commit<<<nb, 128, 0, s>>>(A);
    k_tfix_check<<<1, 1, 0, s>>>(g->ctr, kMaxTfixPasses);
    BT_CUDA_TRY(cudaGetLastError());
  }
  BT_CUDA_TRY(cudaMemcpyAsync(g->ctr_host, g->ctr, sizeof(GridCounters),
                              cudaMemcpyDeviceToHost, s));
  // seed, pole copy, finalize; per level: refine + trace + advance (the
  // start level adds one trace and one advance); per fixed level: passes,
  // commit, check
  const int nlev = L.maxlevel - startlevel;
  g->launches = 3 + 3 * nlev + 2 + nlev * (kMaxTfixPasses + 2);
  g->built = 1;
  return BT_OK;
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
  info->launches = g->launches;
  info->trace_ms = 0.f;
  info->trace_launches = g->n_ev / 2;
  for (int k = 0; k + 1 < g->n_ev; k += 2) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, g->ev[k], g->ev[k + 1]) == cudaSuccess)
      info->trace_ms += ms;
  }
  if (info->flags) {
    set_error("grid build flags 0x%x (1: T-vertex fix did not converge, "
              "2: fix stack overflow, 4: work list overflow)", info->flags);
    return BT_ERR_NUMERIC;
  }
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

int bt_grid_set_timing(bt_grid* g, int on) {
  BT_ARG_CHECK(g != nullptr, "NULL grid");
  if (on && !g->timing)
    for (int k = 0; k < 2 * 16; k++) BT_CUDA_TRY(cudaEventCreate(&g->ev[k]));
  g->timing = on ? 1 : g->timing;
  if (!on) g->timing = 0;
  return BT_OK;
}

int bt_grid_export(bt_grid* g, bt_grid_export_t* out, void* stream) {
  clear_error();
  BT_ARG_CHECK(g && out, "NULL pointer");
  BT_ARG_CHECK(g->built, "grid not built");
  cudaStream_t s = (cudaStream_t)stream;
  const int N = g->L.N;
  k_row_count<<<N, 256, 0, s>>>(g->L.vflag, g->L.blevel, g->L.M, g->rowv, g->rowb);
  k_row_scan<<<1, 32, 0, s>>>(g->rowv, g->rowb, N, g->totals);
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

}  // extern "C"
