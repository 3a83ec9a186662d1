// grid_flow.cuh -- the refinement levels of a grid set as one persistent
// launch, driven by data instead of level barriers.
//
// The reference refines level by level (adaptiveBlockIntegration,
// BT/Grid.h:465-505): every block of a level is checked (refineCheck,
// :410-445) once all of the level's rays are traced, so each level waits for
// its longest ray and the device idles behind it.  Here a block is checked as
// soon as its own four corners are traced, and a new vertex is set up and
// traced as soon as a check creates it, all inside one launch:
//
//   check queue   blocks whose four corners are traced: refineCheck; a leaf
//                 records its level, a refined block claims its five new
//                 vertices (-> setup queue) and creates its four children,
//                 which wait for their corners (or, at the max level, are
//                 leaves at once)
//   setup queue   new vertices: ray set-up and capture test; captured rays
//                 are final, the others leave their start state and go to
//                 the trace queue
//   trace queue   rays to integrate, one per lane, lanes refilled eight at a
//                 time
//
// Each block of the launch has one manager warp (checks first, then
// set-ups, 32 per step) and tracer warps.  A finished vertex sets the traced
// bit of its sync word and, for each child block that registered on it (one
// waiter bit per corner position), decrements the block's count of untraced
// corners; the decrement that reaches zero queues the block.  A child is
// created with a count of five (four corners and a guard): it registers on
// each corner, counts down the corners already traced, then drops the guard.
// The traced bit and the waiter bits share one word, so exactly one of the
// tracer and the registering block sees the other.  A vertex's waiters are
// blocks of its native level (the level at which its lattice position first
// appears): it is created by a refinement into that level, and blocks of
// later levels are only created after it is traced.
//
// Decisions depend only on corner values, so the grids are the ones the
// level-by-level build gives, bit for bit; only the order of work differs.
// The launch ends when no queued or running item is left (a count of items
// pushed and not finished).  Every wait is bounded: a warp that finds no
// work sleeps and retries, and gives up (error flag 8) after about two
// seconds without progress anywhere (the longest legitimate wait, one ray
// alone, is a few milliseconds); a queue slot taken before its producer
// wrote it is waited for the same way.
#pragma once

#include "bt_internal.h"
#include "kerr_plain.cuh"
#include "trace_kernel.cuh"

namespace bt {

constexpr uint32_t kVTraced = 0x80000000u;  // sync word: the vertex is final
constexpr uint32_t kQEmpty = 0xffffffffu;   // queue slot not written yet
enum { kFqCheck = 0, kFqSetup = 1, kFqTrace = 2, kFq = 3 };
// Items: grid g's vertex or block origin key as g * NM + key (< 2^28); a
// check item carries (level - startlevel) in its top four bits.
constexpr uint32_t kFlowKeyBits = 28;
constexpr int kFlowThreads = 256;  // one manager warp and seven tracer warps
constexpr long long kFlowIdleCap = 8000000;  // ~2 s of 256 ns sleeps

struct FlowCtl {
  unsigned long long head[kFq];
  unsigned long long tail[kFq];
  unsigned long long live;  // items pushed and not finished
  unsigned long long progress;  // items finished (for the idle bound)
  uint32_t err;
  uint32_t pad;
};

struct FlowArgs {
  const GridDesc* D;
  int G;
  uint32_t NM, M;
  int maxlevel, startlevel;
  uint32_t* q[kFq];
  unsigned long long cap[kFq];  // slots of each queue
  uint32_t* vsync;  // G * NM: traced bit + waiter bits
  uint8_t* bwait;   // G * NM: untraced corners of the block at this origin
  FlowCtl* ctl;
};

__device__ __forceinline__ void flow_push(const FlowArgs& A, int qi, uint32_t item) {
  atomicAdd(&A.ctl->live, 1ull);
  const unsigned long long t = atomicAdd(&A.ctl->tail[qi], 1ull);
  if (t >= A.cap[qi]) {  // cannot happen: each queue holds one slot per vertex
    atomicOr(&A.ctl->err, 4u);
    return;
  }
  __threadfence();  // the item's data before its slot
  atomicExch(&A.q[qi][t], item);
}

// Takes up to `want` items of queue qi for the calling (uniform) warp: the
// index of the first in *base, the count returned.  Only items already
// counted in tail are taken, so every taken slot is being written.
__device__ __forceinline__ unsigned flow_take(const FlowArgs& A, int qi, unsigned want,
                                              unsigned long long* base) {
  const unsigned lane = threadIdx.x & 31u;
  unsigned long long b = 0;
  unsigned n = 0;
  if (lane == 0 && want) {
    unsigned long long h = *(volatile unsigned long long*)&A.ctl->head[qi];
    for (int tries = 0; tries < 64; tries++) {
      unsigned long long t = *(volatile unsigned long long*)&A.ctl->tail[qi];
      if (t > A.cap[qi]) t = A.cap[qi];  // slots past the capacity were never written
      if (t <= h) break;
      const unsigned take = (unsigned)min((unsigned long long)want, t - h);
      const unsigned long long old = atomicCAS(&A.ctl->head[qi], h, h + take);
      if (old == h) {
        b = h;
        n = take;
        break;
      }
      h = old;
    }
  }
  *base = __shfl_sync(0xffffffffu, b, 0);
  return __shfl_sync(0xffffffffu, n, 0);
}

// The item in slot k of queue qi, once its producer has written it (bounded).
__device__ __forceinline__ uint32_t flow_read(const FlowArgs& A, int qi,
                                              unsigned long long k) {
  uint32_t v = *(volatile uint32_t*)&A.q[qi][k];
  for (long long it = 0; v == kQEmpty && it < kFlowIdleCap; it++) {
    __nanosleep(256);
    v = *(volatile uint32_t*)&A.q[qi][k];
  }
  if (v == kQEmpty) atomicOr(&A.ctl->err, 8u);
  __threadfence();  // the item's data after its slot
  return v;
}

// Native level of lattice vertex (i, j): the level at which its position
// first appears, i.e. maxlevel minus the common power-of-two factor of i and
// j, at most maxlevel - startlevel.
__device__ __forceinline__ int native_level(const FlowArgs& A, uint32_t i, uint32_t j) {
  const int span = A.maxlevel - A.startlevel;
  const int ti = i ? __ffs((int)i) - 1 : span, tj = j ? __ffs((int)j) - 1 : span;
  return A.maxlevel - min(min(ti, tj), span);
}

// One of a block's untraced-corner count comes off; the one that empties it
// queues the block's check (levels below the maximum only register).
__device__ __forceinline__ void block_corner_done(const FlowArgs& A, uint32_t g,
                                                  uint32_t origin, int level) {
  const uint32_t gk = g * A.NM + origin;
  uint32_t* word = (uint32_t*)((uintptr_t)(A.bwait + gk) & ~(uintptr_t)3);
  const uint32_t sh = ((uintptr_t)(A.bwait + gk) & 3) * 8;
  const uint32_t old = atomicSub(word, 1u << sh);
  if (((old >> sh) & 0xffu) == 1u)
    flow_push(A, kFqCheck, ((uint32_t)(level - A.startlevel) << kFlowKeyBits) | gk);
}

// Vertex key of grid g is final (its lattice values written): set its traced
// bit and release the blocks that waited on it.
__device__ __forceinline__ void vertex_done(const FlowArgs& A, uint32_t g, uint32_t key) {
  __threadfence();  // the vertex's values before its traced bit
  const uint32_t old = atomicOr(&A.vsync[g * A.NM + key], kVTraced);
  const uint32_t waiters = old & 0xfu;
  if (!waiters) return;
  const uint32_t i = key / A.M, j = key % A.M;
  const int level = native_level(A, i, j);
  const uint32_t gap = 1u << (A.maxlevel - level);
  for (int p = 0; p < 4; p++) {
    if (!(waiters & (1u << p))) continue;
    const uint32_t oi = (p & 2) ? i - gap : i;
    const uint32_t oj = (p & 1) ? (j + A.M - gap) % A.M : j;
    block_corner_done(A, g, oi * A.M + oj, level);
  }
}

// A child block at `level` with origin (oi, oj) and side gap: counted to five,
// registered on its corners, the traced ones counted down, the guard dropped.
__device__ __forceinline__ void block_create(const FlowArgs& A, uint32_t g, uint32_t oi,
                                             uint32_t oj, uint32_t gap, int level) {
  const uint32_t origin = oi * A.M + oj;
  {
    const uint32_t gk = g * A.NM + origin;
    uint32_t* word = (uint32_t*)((uintptr_t)(A.bwait + gk) & ~(uintptr_t)3);
    const uint32_t sh = ((uintptr_t)(A.bwait + gk) & 3) * 8;
    // the byte is zero (never used, or the finished parent's): add five
    atomicAdd(word, 5u << sh);
  }
  const uint32_t oj2 = (oj + gap) % A.M;
  const uint32_t corner[4] = {origin, oi * A.M + oj2, (oi + gap) * A.M + oj,
                              (oi + gap) * A.M + oj2};
  for (int p = 0; p < 4; p++) {
    const uint32_t old = atomicOr(&A.vsync[g * A.NM + corner[p]], 1u << p);
    if (old & kVTraced) block_corner_done(A, g, origin, level);
  }
  block_corner_done(A, g, origin, level);  // the guard
}

// claim_vertex of the level form for the flow: a vertex no block claimed yet
// becomes claimed (flag 2) and goes to the setup queue.
__device__ __forceinline__ void flow_claim(const FlowArgs& A, const GridDesc& d, uint32_t g,
                                           uint32_t i, uint32_t j) {
  const uint32_t key = i * A.M + j;
  uint32_t* word = (uint32_t*)((uintptr_t)(d.L.vflag + key) & ~(uintptr_t)3);
  const uint32_t sh = ((uintptr_t)(d.L.vflag + key) & 3) * 8;
  uint32_t old = *(volatile uint32_t*)word;
  for (;;) {
    if ((old >> sh) & 0xffu) return;  // exists or already claimed
    const uint32_t got = atomicCAS(word, old, old | (2u << sh));
    if (got == old) break;
    old = got;
  }
  atomicAdd(&d.ctr->n_trace, 1u);
  flow_push(A, kFqSetup, g * A.NM + key);
}

// refineCheck of a block (BT/Grid.h:410-445) and, when it refines, the claims
// and children of adaptiveBlockIntegration (:476-497).
__device__ __forceinline__ void flow_check(const FlowArgs& A, uint32_t item) {
  const int level = A.startlevel + (int)(item >> kFlowKeyBits);
  const uint32_t gk = item & ((1u << kFlowKeyBits) - 1u);
  const uint32_t g = gk / A.NM, key = gk % A.NM;
  const GridDesc& d = A.D[g];
  const LatticeView& L = d.L;
  const uint32_t M = A.M;
  const uint32_t gap = 1u << (A.maxlevel - level);
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
    // leaves below the max level, tagged with their level for the T-vertex fix
    const uint32_t s = atomicAdd(&d.ctr->n_leaf, 1u);
    d.leaves[s] = ((uint32_t)(level - A.startlevel) << kFlowKeyBits) | key;
    return;
  }
  const uint32_t h = gap / 2, kh = i + h, lh = j + h;
  flow_claim(A, d, g, kh, j);
  flow_claim(A, d, g, kh, lh);
  flow_claim(A, d, g, i, lh);
  flow_claim(A, d, g, i + gap, lh);
  flow_claim(A, d, g, kh, (j + gap) % M);
  const int lc = level + 1;
  const uint32_t co[4][2] = {{i, j}, {kh, j}, {kh, lh}, {i, lh}};
  for (int c = 0; c < 4; c++) {
    if (lc == A.maxlevel) {
      L.blevel[co[c][0] * M + co[c][1]] = (int8_t)lc;  // k_finalize's leaves
    } else {
      block_create(A, g, co[c][0], co[c][1], h, lc);
    }
  }
}

// Set-up and capture test of a new vertex (as k_setup_lattice).
template <class Policy>
__device__ __forceinline__ void flow_setup(const FlowArgs& A, uint32_t item) {
  const uint32_t g = item / A.NM, key = item % A.NM;
  const GridDesc& d = A.D[g];
  double th, ph, to, po;
  int32_t s;
  uint8_t ss;
  lattice_seed(d.L, key, th, ph);
  plain::RayStart rs;
  const bool go = plain::setup_ray(d.p, th, ph, rs, to, po, s, ss);
  if (go && d.p.maxstp > 0) {
    d.X[0][key] = make_double2(rs.pR, rs.pTheta);
    d.X[1][key] = make_double2(rs.b, rs.q);
    reinterpret_cast<float*>(d.L.steps)[key] = (float)rs.r0;
    flow_push(A, kFqTrace, item);
    return;
  }
  if (go) {
    typename Policy::State st;
    Policy::start(d.p, rs, st);
    Policy::finish(d.p, st, to, po, s, ss);
  }
  d.L.thphi[key] = make_double2(to, po);
  d.L.steps[key] = s;
  d.L.vstat[key] = ss;
  d.L.vflag[key] = 1;
  vertex_done(A, g, key);
}

__device__ __forceinline__ void flow_finished(const FlowArgs& A) {
  atomicAdd(&A.ctl->progress, 1ull);
  atomicAdd(&A.ctl->live, (unsigned long long)-1ll);
}

// The flow.  Warp 0 of each block manages (checks, then set-ups, one item per
// lane); the others trace.  A warp with nothing to do sleeps and looks again
// until no item is live anywhere.
template <class Policy>
__global__ void __launch_bounds__(kFlowThreads, 2) k_flow(FlowArgs A) {
  const unsigned lane = threadIdx.x & 31u;
  const bool manager = (threadIdx.x >> 5) == 0;
  long long idle = 0;
  unsigned long long seen = 0;
  // tracer lane state
  uint32_t item = 0;
  bool busy = false;
  typename Policy::State st;
  for (;;) {
    bool worked = false;
    if (manager) {
      unsigned long long base;
      unsigned n = flow_take(A, kFqCheck, 32, &base);
      if (n) {
        if (lane < n) {
          flow_check(A, flow_read(A, kFqCheck, base + lane));
          flow_finished(A);
        }
        worked = true;
      } else if ((n = flow_take(A, kFqSetup, 32, &base)) != 0) {
        if (lane < n) {
          flow_setup<Policy>(A, flow_read(A, kFqSetup, base + lane));
          flow_finished(A);
        }
        worked = true;
      }
    } else {
      const unsigned idle_m = __ballot_sync(0xffffffffu, !busy);
      const unsigned busy_m = ~idle_m;
      if (idle_m && (__popc(idle_m) >= kRefillMin || !busy_m)) {
        unsigned long long base;
        const unsigned n = flow_take(A, kFqTrace, __popc(idle_m), &base);
        if (n) {
          const unsigned rank = __popc(idle_m & ((1u << lane) - 1u));
          if (!busy && rank < n) {
            item = flow_read(A, kFqTrace, base + rank);
            const GridDesc& d = A.D[item / A.NM];
            Policy::start(d.p, lattice_start(d, item % A.NM), st);
            busy = true;
          }
          worked = true;
        }
      }
      if (busy) {
        worked = true;
        const uint32_t g = item / A.NM, key = item % A.NM;
        const GridDesc& d = A.D[g];
        if (Policy::attempt(d.p, st)) {
          double to, po;
          int32_t s;
          uint8_t ss;
          Policy::finish(d.p, st, to, po, s, ss);
          d.L.thphi[key] = make_double2(to, po);
          d.L.steps[key] = s;
          d.L.vstat[key] = ss;
          d.L.vflag[key] = 1;
          vertex_done(A, g, key);
          flow_finished(A);
          busy = false;
        }
      }
      worked = __any_sync(0xffffffffu, worked);
    }
    if (worked) {
      idle = 0;
      continue;
    }
    // nothing here: done when no item is live, else wait (bounded)
    if (*(volatile unsigned long long*)&A.ctl->live == 0ull) break;
    const unsigned long long pr = *(volatile unsigned long long*)&A.ctl->progress;
    if (pr != seen) {
      seen = pr;
      idle = 0;
    }
    if (++idle > kFlowIdleCap || *(volatile uint32_t*)&A.ctl->err) {
      if (lane == 0) atomicOr(&A.ctl->err, 8u);
      break;
    }
    __nanosleep(256);
  }
}

// The flow's launch: the resident blocks only (all must be able to run at
// once only for speed; a block that has not started holds no work).
template <class Policy>
int launch_flow(const FlowArgs& A, cudaStream_t s) {
  static int per_sm = 0;
  if (!per_sm) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_flow<Policy>, kFlowThreads, 0);
    if (per_sm < 1) per_sm = 1;
  }
  k_flow<Policy><<<sm_count() * per_sm, kFlowThreads, 0, s>>>(A);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("flow launch: %s", cudaGetErrorString(e));
    return BT_ERR_CUDA;
  }
  return BT_OK;
}

}  // namespace bt
