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
// Each block of the launch has a worker warp (checks first, then set-ups,
// one per lane), a service warp that feeds the block's tracer lanes and
// collects their rays, and tracer warps.  A finished vertex sets the traced
// bit of its sync word and, for each block that registered on it (a waiter
// bit per corner position and level), sets that corner's bit in the block's
// byte; the bit that completes the four queues the block's check.  A block
// registers on each of its corners when it is created and sets the bits of
// the corners already traced itself.  The traced bit and the waiter bits
// share one word, so exactly one of the tracer and the registering block
// sees the other.
//
// Early refinement: refineCheck refines a block when the larger of its two
// diagonals' squared separations is above the threshold, so a traced
// diagonal above it decides the block without its other two corners.  The
// bit that completes a diagonal reads its two corners and, when they are far
// enough apart, queues the block as refined at once: its children are
// created, and their new rays start, while the block's slow corner is still
// being integrated (a chain of slow rays no longer runs level after level).
// The one case where the larger-of-two rule can differ from the diagonal
// alone is a NaN separation on the (0, 3) diagonal when the (1, 2) diagonal
// decided: std::max then keeps the NaN and the block is a leaf.  A block
// refined early on (1, 2) is therefore checked again by whoever completes its
// corners, and a disagreement is reported (error flag 16: rebuild in the
// level form).  Blocks of several levels then wait on one vertex (a child can
// exist before its parent's corners are traced), so the waiter bits carry
// the level (four per level above the vertex's native one, 28 bits in all:
// early refinement needs maxlevel - startlevel <= 7) and every level below
// the max has its own array of block bytes.
//
// The manager's queues (checks, set-ups) hand out tickets: a lane reserves
// the next slot with a fetch-and-add (one per warp) and polls that slot, its
// own address, until the producer has written it.  Taking only items already
// written by compare-and-swap on a shared head let one warp in the whole
// device succeed per round trip to L2 and made the flow ten times slower than
// the level builds.  Rays are taken (by fetch-and-add) only when already
// pushed, hot rays first (set-ups of vertices whose parent block holds a slow
// ray, kHotSteps, go to a queue of their own), so that a tracer lane is free
// when a hot ray arrives instead of being bound to a ray far back in the
// queue: the longest chain of rays, level after level, bounds a single
// grid's build.
//
// Decisions depend only on corner values, so the grids are the ones the
// level-by-level build gives, bit for bit (flag 16 aside); only the order of
// work differs.
// The launch ends when no queued or running item is left (a count of items
// pushed and not finished).  Every wait is bounded: a warp with nothing to do
// backs off and looks again, and gives up (error flag 8) after two seconds in
// which nothing anywhere moved (no item pushed or finished, no tracer warp
// reporting attempts).
#pragma once

#include "bt_internal.h"
#include "kerr_plain.cuh"
#include "trace_kernel.cuh"

namespace bt {

constexpr uint32_t kVTraced = 0x80000000u;  // sync word: the vertex is final
constexpr uint32_t kQEmpty = 0xffffffffu;   // queue slot not written yet
enum { kFqCheck = 0, kFqSetup = 1, kFqTrace = 2, kFqHot = 3, kFqSetupHot = 4, kFq = 5 };
// Items: grid g's vertex or block origin key as g * NM + key (< 2^28); a
// check item carries (level - startlevel) in its top four bits (with early
// refinement: bits 28-30, and bit 31 for a block refined early), a set-up
// item the vertex's hot bit (kHotSteps) in bit 28.
constexpr uint32_t kFlowKeyBits = 28;
constexpr uint32_t kFlowKeyMask = (1u << kFlowKeyBits) - 1u;
constexpr uint32_t kFlowEarly = 0x80000000u;
// Early refinement: the most levels below the max that blocks wait on.
constexpr int kFlowEarlySpan = 7;
constexpr int kFlowBwLevels = kFlowEarlySpan - 1;
// A block's byte: its corners traced (bit p = corner p: 0 origin, 1 right,
// 2 below, 3 diagonal), checked or refined early, refined on (1, 2).
constexpr uint32_t kBCorners = 0xfu;
constexpr uint32_t kBDecided = 0x10u;
constexpr uint32_t kBByDiag2 = 0x20u;
// A block: one service warp, kFlowWorkers worker warps, kFlowSlots tracer warps.
constexpr int kFlowWorkers = 1;
constexpr int kFlowSlots = 6;  // tracer warps = tracer lanes per service lane
constexpr int kFlowTracers = 32 * kFlowSlots;
constexpr int kFlowThreads = 32 * (1 + kFlowWorkers) + kFlowTracers;
// A warp gives up after this long with nothing to do while nothing anywhere
// moved (no item pushed or finished, no tracer warp reporting attempts).
constexpr unsigned long long kFlowIdleNs = 2000000000ull;
constexpr unsigned kFlowBeat = 1024;  // tracer loop steps between progress reports

// Every counter on a line of its own: each is hit by warps all over the
// device, and sharing a line would queue their atomics behind each other.
struct alignas(128) FlowCounter {
  unsigned long long v;
};

struct FlowCtl {
  FlowCounter head[kFq];  // tickets handed out
  FlowCounter tail[kFq];  // slots reserved by producers
  FlowCounter live;       // items pushed and not finished
  FlowCounter progress;   // tracer warps' heartbeats
  uint32_t err;
  uint32_t dropped;       // diagnostic: the ray already lost (FlowArgs::drop)
};

struct FlowArgs {
  const GridDesc* D;
  int G;
  uint32_t NM, M;
  int maxlevel, startlevel;
  uint32_t* q[kFq];
  unsigned long long cap[kFq];  // slots of each queue
  uint32_t* vsync;  // G * NM: traced bit + waiter bits
  // block bytes: of level l at (l - startlevel - 1) * bw_stride + g * NM +
  // origin; bw_stride 0 (early refinement off): one array for all levels
  uint8_t* bwait;
  size_t bw_stride;
  int early;  // refine a block as soon as one diagonal decides it
  FlowCtl* ctl;
  int blocks_per_sm;  // of the launch (capped by the occupancy limit)
  // Diagnostic (bt_grid_set_flow_drop): the first ray to be traced is
  // counted as live but never handed to a tracer, so that nothing can
  // finish the flow and its bounded wait runs out (error flag 8).
  int drop;
};

__device__ __forceinline__ unsigned long long flow_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// One item onto queue qi from one lane.  live counts it before it can be
// seen, so live reaches zero only when every item pushed has finished.
__device__ __forceinline__ void flow_push(const FlowArgs& A, int qi, uint32_t item) {
  atomicAdd(&A.ctl->live.v, 1ull);
  __threadfence();
  const unsigned long long t = atomicAdd(&A.ctl->tail[qi].v, 1ull);
  if (t >= A.cap[qi]) {  // cannot happen: each queue holds one slot per vertex
    atomicOr(&A.ctl->err, 4u);
    return;
  }
  __threadfence();  // the item's data before its slot
  *(volatile uint32_t*)&A.q[qi][t] = item;
}

// Up to five items per lane onto queue qi, one reservation for the warp (the
// whole warp calls).
__device__ __forceinline__ void flow_push_warp(const FlowArgs& A, int qi, const uint32_t* items,
                                               unsigned n) {
  const unsigned lane = threadIdx.x & 31u;
  unsigned incl = n;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= (unsigned)o) incl += v;
  }
  const unsigned total = __shfl_sync(0xffffffffu, incl, 31);
  if (!total) return;
  unsigned long long t0 = 0;
  if (lane == 0) {
    atomicAdd(&A.ctl->live.v, (unsigned long long)total);
    __threadfence();
    t0 = atomicAdd(&A.ctl->tail[qi].v, (unsigned long long)total);
  }
  t0 = __shfl_sync(0xffffffffu, t0, 0) + (incl - n);
  if (n) __threadfence();  // the items' data before their slots
  for (unsigned k = 0; k < n; k++) {
    if (t0 + k >= A.cap[qi]) {
      atomicOr(&A.ctl->err, 4u);
      break;
    }
    *(volatile uint32_t*)&A.q[qi][t0 + k] = items[k];
  }
}

// Tickets of queue qi for the lanes of `want` (the whole warp calls): ticket t
// is slot t, which the lane polls until its producer has written it.  Items
// are handed out in queue order with one atomic per warp and no retries; a
// ticket past the queue's capacity (< 2^28) can never be written (its lane
// stops asking).
__device__ __forceinline__ void flow_tickets(const FlowArgs& A, int qi, bool want,
                                             uint32_t& ticket, bool& have, bool& dead) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned m = __ballot_sync(0xffffffffu, want);
  if (!m) return;
  unsigned long long b = 0;
  if (lane == 0) b = atomicAdd(&A.ctl->head[qi].v, (unsigned long long)__popc(m));
  b = __shfl_sync(0xffffffffu, b, 0);
  if (want) {
    const unsigned long long t = b + __popc(m & ((1u << lane) - 1u));
    if (t < A.cap[qi]) {
      ticket = (uint32_t)t;
      have = true;
    } else {
      dead = true;
    }
  }
}

// Up to one item for each lane of `mask` from queue qi, taking only items
// already pushed: the count read before the fetch-and-add can be overtaken by
// another warp, so a few tickets may lead their producers (those lanes poll
// their slots like any ticket).  Returns the lanes of `mask` left without
// one.  The whole warp calls.
__device__ __forceinline__ unsigned flow_take(const FlowArgs& A, int qi, unsigned mask,
                                              uint32_t& ticket, bool& have, int& tq) {
  const unsigned lane = threadIdx.x & 31u;
  unsigned k = 0;
  unsigned long long b = 0;
  if (lane == 0) {
    unsigned long long t = *(volatile unsigned long long*)&A.ctl->tail[qi].v;
    if (t > A.cap[qi]) t = A.cap[qi];
    const unsigned long long h = *(volatile unsigned long long*)&A.ctl->head[qi].v;
    if (t > h) {
      k = (unsigned)min((unsigned long long)__popc(mask), t - h);
      b = atomicAdd(&A.ctl->head[qi].v, (unsigned long long)k);
    }
  }
  k = __shfl_sync(0xffffffffu, k, 0);
  if (!k) return mask;
  b = __shfl_sync(0xffffffffu, b, 0);
  const unsigned rank = __popc(mask & ((1u << lane) - 1u));
  if (((mask >> lane) & 1u) && rank < k && b + rank < A.cap[qi]) {
    ticket = (uint32_t)(b + rank);
    have = true;
    tq = qi;
  }
  for (unsigned r = 0; r < k; r++) mask &= mask - 1u;  // the k lowest lanes took one
  return mask;
}

// The item of a lane's ticket, or kQEmpty while it is not written.
__device__ __forceinline__ uint32_t flow_poll(const FlowArgs& A, int qi, uint32_t ticket) {
  const uint32_t v = *(volatile uint32_t*)&A.q[qi][ticket];
  if (v != kQEmpty) __threadfence();  // the item's data after its slot
  return v;
}

// Idle state of a warp (lane 0's, in shared memory): backoff and the bound on
// waiting.
struct FlowIdle {
  unsigned long long since, live_seen, beat_seen;
  unsigned ns, it;
};

__device__ __forceinline__ void flow_busy(FlowIdle& w) {
  if ((threadIdx.x & 31u) == 0) {
    w.ns = 32;
    w.it = 0;
  }
}

// Called by the whole warp when it did nothing this step: false when the
// flow is over (no live item), failed, or stalled (error flag 8), else
// sleeps (32 ns doubling up to max_ns) and returns true.
__device__ __forceinline__ bool flow_wait(const FlowArgs& A, FlowIdle& w, unsigned max_ns) {
  const unsigned lane = threadIdx.x & 31u;
  int stop = 0;
  unsigned ns = 0;
  if (lane == 0) {
    if ((w.it++ & 1u) == 0u) {
      const unsigned long long live = *(volatile unsigned long long*)&A.ctl->live.v;
      const unsigned long long beat = *(volatile unsigned long long*)&A.ctl->progress.v;
      const uint32_t err = *(volatile uint32_t*)&A.ctl->err;
      const unsigned long long now = flow_now();
      if (live == 0ull || err) {
        stop = 1;
      } else if (w.it == 1u || live != w.live_seen || beat != w.beat_seen) {
        w.live_seen = live;
        w.beat_seen = beat;
        w.since = now;
      } else if (now - w.since > kFlowIdleNs) {
        atomicOr(&A.ctl->err, 8u);
        stop = 1;
      }
    }
    ns = w.ns;
    if (w.ns < max_ns) w.ns *= 2u;
  }
  if (__shfl_sync(0xffffffffu, stop, 0)) return false;
  __nanosleep(__shfl_sync(0xffffffffu, ns, 0));
  return true;
}

// Items finished by the warp this step come off live, after the items they
// pushed went on (the whole warp calls).
__device__ __forceinline__ void flow_finished(const FlowArgs& A, unsigned n) {
  if (!n) return;
  __syncwarp();
  if ((threadIdx.x & 31u) == 0) {
    __threadfence();
    atomicAdd(&A.ctl->live.v, (unsigned long long)(0ull - n));
  }
}

// Native level of lattice vertex (i, j): the level at which its position
// first appears, i.e. maxlevel minus the common power-of-two factor of i and
// j, at most maxlevel - startlevel.
__device__ __forceinline__ int native_level(const FlowArgs& A, uint32_t i, uint32_t j) {
  const int span = A.maxlevel - A.startlevel;
  const int ti = i ? __ffs((int)i) - 1 : span, tj = j ? __ffs((int)j) - 1 : span;
  return A.maxlevel - min(min(ti, tj), span);
}

// Squared separation of two lattice values, rounded as refineCheck's
// expression is without contraction (the level form's k_refine is compiled
// with --fmad=false; the flow is also built into units that contract).
__device__ __forceinline__ double flow_sep(const double2 u, const double2 v) {
  const double dx = u.x - v.x, dy = u.y - v.y;
  return __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
}

// refineCheck's threshold (BT/Grid.h:437-440).
__device__ __forceinline__ bool flow_refines(double mx, int level) {
  return (level < 6 && mx > 1E-10) || (mx > 0.015);
}

// refineCheck (BT/Grid.h:410-445) of the block at (i, j) with side gap: the
// larger of its diagonals' squared separations against the threshold.
__device__ __forceinline__ bool flow_rule(const LatticeView& L, uint32_t M, uint32_t i,
                                          uint32_t j, uint32_t gap, int level) {
  const uint32_t k = i + gap, l = (j + gap) % M;
  const double diag = flow_sep(L.thphi[(size_t)i * M + j], L.thphi[(size_t)k * M + l]);
  const double diag2 = flow_sep(L.thphi[(size_t)k * M + j], L.thphi[(size_t)i * M + l]);
  const double mx = diag < diag2 ? diag2 : diag;  // std::max
  return flow_refines(mx, level);
}

// The byte of the block of `level` (above the start level) at gk = g * NM +
// origin: its aligned 32-bit word, and the byte's shift in it.
__device__ __forceinline__ uint32_t* block_word(const FlowArgs& A, uint32_t gk, int level,
                                                uint32_t& sh) {
  const size_t lv = A.bw_stride ? (size_t)(level - A.startlevel - 1) : 0;
  uint8_t* byte = A.bwait + lv * A.bw_stride + gk;
  sh = (uint32_t)((uintptr_t)byte & 3) * 8;
  return (uint32_t*)((uintptr_t)byte & ~(uintptr_t)3);
}

// Corner p of the block of `level` at origin (grid g) is traced.  The bit
// that completes the four queues the block's check; with early refinement,
// the bit that completes a diagonal whose separation alone refines the block
// queues it as refined.  Exactly one of them decides (kBDecided).
__device__ __forceinline__ void block_corner_done(const FlowArgs& A, uint32_t g,
                                                  uint32_t origin, int level, int p) {
  const uint32_t gk = g * A.NM + origin;
  uint32_t sh;
  uint32_t* word = block_word(A, gk, level, sh);
  const uint32_t old = (atomicOr(word, (1u << p) << sh) >> sh) & 0xffu;
  const uint32_t now = old | (1u << p);
  const uint32_t tag = (uint32_t)(level - A.startlevel) << kFlowKeyBits;
  const uint32_t M = A.M, i = origin / M, j = origin % M;
  const uint32_t gap = 1u << (A.maxlevel - level);
  if ((now & kBCorners) == kBCorners) {
    uint32_t prev = old;
    if (!(old & kBDecided)) {
      prev = (atomicOr(word, kBDecided << sh) >> sh) & 0xffu;
      if (!(prev & kBDecided)) {
        flow_push(A, kFqCheck, tag | gk);
        return;
      }
    }
    // refined early on the (1, 2) diagonal: the full rule must agree (it
    // does unless the (0, 3) separation is NaN)
    if (prev & kBByDiag2) {
      __threadfence();  // the corners' values after their traced bits
      if (!flow_rule(A.D[g].L, M, i, j, gap, level)) atomicOr(&A.ctl->err, 16u);
    }
    return;
  }
  if (!A.early || (old & kBDecided)) return;
  const bool d03 = (now & 9u) == 9u && (old & 9u) != 9u;
  const bool d12 = (now & 6u) == 6u && (old & 6u) != 6u;
  if (!d03 && !d12) return;
  __threadfence();  // the corners' values after their traced bits
  const LatticeView& L = A.D[g].L;
  const uint32_t k = i + gap, l = (j + gap) % M;
  const double sep = d03 ? flow_sep(L.thphi[(size_t)i * M + j], L.thphi[(size_t)k * M + l])
                         : flow_sep(L.thphi[(size_t)k * M + j], L.thphi[(size_t)i * M + l]);
  if (!flow_refines(sep, level)) return;
  const uint32_t mark = kBDecided | (d03 ? 0u : kBByDiag2);
  const uint32_t prev = (atomicOr(word, mark << sh) >> sh) & 0xffu;
  if (prev & kBDecided) return;  // checked or refined meanwhile
  flow_push(A, kFqCheck, kFlowEarly | tag | gk);
}

// Vertex key of grid g is final (its lattice values written): set its traced
// bit and release the blocks that waited on it (waiter bit 4 e + p: corner p
// of a block e levels above the vertex's native one).
__device__ __forceinline__ void vertex_done(const FlowArgs& A, uint32_t g, uint32_t key) {
  __threadfence();  // the vertex's values before its traced bit
  const uint32_t old = atomicOr(&A.vsync[g * A.NM + key], kVTraced);
  uint32_t waiters = old & ~kVTraced;
  if (!waiters) return;
  const uint32_t i = key / A.M, j = key % A.M;
  const int native = native_level(A, i, j);
  while (waiters) {
    const int b = __ffs((int)waiters) - 1;
    waiters &= waiters - 1u;
    const int level = native + (b >> 2), p = b & 3;
    const uint32_t gap = 1u << (A.maxlevel - level);
    const uint32_t oi = (p & 2) ? i - gap : i;
    const uint32_t oj = (p & 1) ? (j + A.M - gap) % A.M : j;
    block_corner_done(A, g, oi * A.M + oj, level, p);
  }
}

// A child block at `level` with origin (oi, oj) and side gap: registered on
// its corners, the traced ones set at once.  Its byte is zero (its level's
// array is cleared for each build; with one array, the checked parent at the
// same origin cleared it).
__device__ __forceinline__ void block_create(const FlowArgs& A, uint32_t g, uint32_t oi,
                                             uint32_t oj, uint32_t gap, int level) {
  const uint32_t origin = oi * A.M + oj;
  const uint32_t oj2 = (oj + gap) % A.M;
  const uint32_t ci[4] = {oi, oi, oi + gap, oi + gap}, cj[4] = {oj, oj2, oj, oj2};
  for (int p = 0; p < 4; p++) {
    uint32_t* sw = &A.vsync[g * A.NM + ci[p] * A.M + cj[p]];
    const int e = level - native_level(A, ci[p], cj[p]);
    if (!A.early && e > 0) {
      // without early refinement a corner of an older level was traced
      // before the parent's check
      if (*(volatile uint32_t*)sw & kVTraced) block_corner_done(A, g, origin, level, p);
      else atomicOr(&A.ctl->err, 4u);
      continue;
    }
    const uint32_t old = atomicOr(sw, 1u << (4 * e + p));
    if (old & kVTraced) block_corner_done(A, g, origin, level, p);
  }
}

// claim_vertex of the level form for the flow: a vertex no block claimed yet
// becomes claimed (flag 2); true when this call claimed it.
__device__ __forceinline__ bool flow_claim(const GridDesc& d, uint32_t M, uint32_t i,
                                           uint32_t j) {
  const uint32_t key = i * M + j;
  uint32_t* word = (uint32_t*)((uintptr_t)(d.L.vflag + key) & ~(uintptr_t)3);
  const uint32_t sh = ((uintptr_t)(d.L.vflag + key) & 3) * 8;
  uint32_t old = *(volatile uint32_t*)word;
  for (;;) {
    if ((old >> sh) & 0xffu) return false;  // exists or already claimed
    const uint32_t got = atomicCAS(word, old, old | (2u << sh));
    if (got == old) break;
    old = got;
  }
  atomicAdd(&d.ctr->n_trace, 1u);
  return true;
}

// refineCheck of a block (BT/Grid.h:410-445) and, when it refines, the claims
// and children of adaptiveBlockIntegration (:476-497).  The new vertices'
// set-up items go to `claimed` (at most five); their count is returned.
__device__ __forceinline__ unsigned flow_check(const FlowArgs& A, uint32_t item,
                                              uint32_t* claimed) {
  const bool early = A.early && (item & kFlowEarly);
  const int level =
      A.startlevel + (int)((item >> kFlowKeyBits) & (A.early ? 7u : 15u));
  const uint32_t gk = item & kFlowKeyMask;
  const uint32_t g = gk / A.NM, key = gk % A.NM;
  const GridDesc& d = A.D[g];
  const LatticeView& L = d.L;
  const uint32_t M = A.M;
  const uint32_t gap = 1u << (A.maxlevel - level);
  const uint32_t i = key / M, j = key % M;
  const uint32_t k = i + gap, l = (j + gap) % M;
  // refined early: a traced diagonal decided it (its other corners may still
  // be in flight)
  if (!early && !flow_rule(L, M, i, j, gap, level)) {
    L.blevel[key] = (int8_t)level;
    // leaves below the max level, tagged with their level for the T-vertex fix
    const uint32_t s = atomicAdd(&d.ctr->n_leaf, 1u);
    d.leaves[s] = ((uint32_t)(level - A.startlevel) << kFlowKeyBits) | key;
    return 0;
  }
  const uint32_t h = gap / 2, kh = i + h, lh = j + h;
  // hot: a slow corner (a block refined early waits for one)
  bool slow = early;
  if (!early) {
    const int32_t smax = max(max(L.steps[(size_t)i * M + j], L.steps[(size_t)k * M + j]),
                             max(L.steps[(size_t)i * M + l], L.steps[(size_t)k * M + l]));
    slow = smax >= kHotSteps;
  }
  const uint32_t hot = slow ? 1u << kFlowKeyBits : 0u;
  const uint32_t nv[5][2] = {{kh, j}, {kh, lh}, {i, lh}, {i + gap, lh}, {kh, (j + gap) % M}};
  unsigned n = 0;
  for (int v = 0; v < 5; v++)
    if (flow_claim(d, M, nv[v][0], nv[v][1]))
      claimed[n++] = hot | (g * A.NM + nv[v][0] * M + nv[v][1]);
  const int lc = level + 1;
  if (!A.bw_stride && level > A.startlevel && lc < A.maxlevel) {
    // one array of block bytes: the child at this origin takes this byte,
    // and no corner of this block is left to set it
    uint32_t sh;
    uint32_t* word = block_word(A, gk, level, sh);
    atomicAnd(word, ~(0xffu << sh));
  }
  const uint32_t co[4][2] = {{i, j}, {kh, j}, {kh, lh}, {i, lh}};
  for (int c = 0; c < 4; c++) {
    if (lc == A.maxlevel) {
      L.blevel[co[c][0] * M + co[c][1]] = (int8_t)lc;  // k_finalize's leaves
    } else {
      block_create(A, g, co[c][0], co[c][1], h, lc);
    }
  }
  return n;
}

// Set-up and capture test of a new vertex (as k_setup_lattice); true when
// its ray is to be traced (its start state left in the fix buffers).
template <class Policy>
__device__ __forceinline__ bool flow_setup(const FlowArgs& A, uint32_t item) {
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
    return true;
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
  return false;
}

// The mailboxes between a block's service warp and its tracer lanes (slot t =
// tracer lane t): the service hands a ray's start state and item over and
// takes its result back, so tracer lanes never touch the queues, the sync
// words or a fence.  With that traffic in the tracers' own loop, every
// attempt of a warp waited for a round trip to L2 and the longest rays ran
// at 4.3 us per attempt instead of 1.8.
struct FlowMail {
  double start[5][kFlowTracers];  // pR, pTheta, b, q, r0
  double out[2][kFlowTracers];    // theta, phi
  int32_t steps[kFlowTracers];
  uint32_t item[kFlowTracers];  // service -> tracer: the ray to trace (kQEmpty: none)
  uint32_t done[kFlowTracers];  // tracer -> service: the ray traced (kQEmpty: none)
  uint8_t stat[kFlowTracers];
  FlowIdle idle[1 + kFlowWorkers];
  uint32_t stop;  // set by the service when the flow is over
};

// The worker warps of each block: checks and set-ups.  Each lane holds a
// ticket of the check queue and one of each set-up queue (hot, other) and
// serves what is written (a check, then a hot set-up before another); a
// set-up's ray goes to the hot or the other trace queue.
template <class Policy>
__device__ __forceinline__ void flow_worker(const FlowArgs& A, FlowIdle& w) {
  uint32_t tc = 0, th = 0, ts = 0;
  bool hc = false, hh = false, hs = false, dc = false, dh = false, ds = false;
  for (;;) {
    flow_tickets(A, kFqCheck, !hc && !dc, tc, hc, dc);
    flow_tickets(A, kFqSetupHot, !hh && !dh, th, hh, dh);
    flow_tickets(A, kFqSetup, !hs && !ds, ts, hs, ds);
    const uint32_t ci = hc ? flow_poll(A, kFqCheck, tc) : kQEmpty;
    if (ci != kQEmpty) hc = false;
    uint32_t claimed[5];
    const unsigned nc = ci != kQEmpty ? flow_check(A, ci, claimed) : 0u;
    // a check's new vertices: hot ones (all or none) to the hot set-up queue
    const bool chot = nc && (claimed[0] >> kFlowKeyBits);
    flow_push_warp(A, kFqSetupHot, claimed, chot ? nc : 0u);
    flow_push_warp(A, kFqSetup, claimed, chot ? 0u : nc);
    // one set-up per lane and pass, a hot one when there is one
    uint32_t si = hh ? flow_poll(A, kFqSetupHot, th) : kQEmpty;
    if (si != kQEmpty) {
      hh = false;
    } else {
      si = hs ? flow_poll(A, kFqSetup, ts) : kQEmpty;
      if (si != kQEmpty) hs = false;
    }
    const uint32_t sk = si & kFlowKeyMask;
    const bool trace = si != kQEmpty && flow_setup<Policy>(A, sk);
    const bool hot = (si >> kFlowKeyBits) & 1u;
    bool lose = false;
    if (A.drop && trace && atomicCAS(&A.ctl->dropped, 0u, 1u) == 0u) {
      atomicAdd(&A.ctl->live.v, 1ull);  // live for good: never pushed, never finished
      lose = true;
    }
    flow_push_warp(A, kFqHot, &sk, trace && hot && !lose ? 1u : 0u);
    flow_push_warp(A, kFqTrace, &sk, trace && !hot && !lose ? 1u : 0u);
    const unsigned done = __popc(__ballot_sync(0xffffffffu, ci != kQEmpty)) +
                          __popc(__ballot_sync(0xffffffffu, si != kQEmpty));
    flow_finished(A, done);
    if (done) {
      flow_busy(w);
      continue;
    }
    if (!flow_wait(A, w, 1024u)) break;
  }
}

// Warp 0 of each block: the tracer lanes' service.  Lane l owns slot l of
// each tracer warp.  It writes traced rays into the lattice and releases
// their blocks (vertex_done), and fills free slots with rays already pushed,
// hot ones first (one per lane and pass).
__device__ __forceinline__ void flow_service(const FlowArgs& A, FlowMail& S) {
  const unsigned lane = threadIdx.x & 31u;
  FlowIdle& w = S.idle[0];
  uint32_t occ = 0;  // slots holding a ray (handed over or being traced)
  uint32_t ticket = 0;
  bool have = false;
  int tq = kFqTrace;
  unsigned beat = 0;
  for (;;) {
    unsigned nfin = 0, nstart = 0;
    bool lost = false;
    for (int k = 0; k < kFlowSlots; k++) {
      if (!((occ >> k) & 1u)) continue;
      const int t = (int)lane + 32 * k;
      const uint32_t it = *(volatile uint32_t*)&S.done[t];
      if (it == kQEmpty) continue;
      __threadfence_block();
      const uint32_t g = it / A.NM, key = it % A.NM;
      const GridDesc& d = A.D[g];
      d.L.thphi[key] = make_double2(S.out[0][t], S.out[1][t]);
      d.L.steps[key] = S.steps[t];
      d.L.vstat[key] = S.stat[t];
      d.L.vflag[key] = 1;
      *(volatile uint32_t*)&S.done[t] = kQEmpty;
      occ &= ~(1u << k);
      vertex_done(A, g, key);
      nfin++;
    }
    const bool room = occ != (1u << kFlowSlots) - 1u;
    const unsigned wantm = __ballot_sync(0xffffffffu, room && !have);
    if (wantm) {
      const unsigned left = flow_take(A, kFqHot, wantm, ticket, have, tq);
      if (left) flow_take(A, kFqTrace, left, ticket, have, tq);
    }
    if (have) {
      const uint32_t it = flow_poll(A, tq, ticket);
      if (it != kQEmpty) {
        have = false;
        const int k = __ffs(~occ) - 1;  // free: a ticket is only taken with room
        if (k >= kFlowSlots) {  // cannot happen; the ray is lost, so the flow fails
          atomicOr(&A.ctl->err, 4u);
          lost = true;
        } else {
          const int t = (int)lane + 32 * k;
          const GridDesc& d = A.D[it / A.NM];
          const plain::RayStart rs = lattice_start(d, it % A.NM);
          S.start[0][t] = rs.pR;
          S.start[1][t] = rs.pTheta;
          S.start[2][t] = rs.b;
          S.start[3][t] = rs.q;
          S.start[4][t] = rs.r0;
          __threadfence_block();
          *(volatile uint32_t*)&S.item[t] = it;
          occ |= 1u << k;
          nstart++;
        }
      }
    }
    if (__any_sync(0xffffffffu, lost)) break;
    const unsigned fin = __reduce_add_sync(0xffffffffu, nfin);
    flow_finished(A, fin);
    if (fin || __any_sync(0xffffffffu, nstart != 0)) {
      flow_busy(w);
      continue;
    }
    if (__any_sync(0xffffffffu, occ != 0)) {
      // rays in the tracers: look again soon, and report that work goes on
      if (++beat == kFlowBeat) {
        beat = 0;
        if (lane == 0) atomicAdd(&A.ctl->progress.v, 1ull);
      }
      flow_busy(w);
      __nanosleep(64);
      continue;
    }
    if (!flow_wait(A, w, 1024u)) break;
  }
  if (lane == 0) *(volatile uint32_t*)&S.stop = 1u;
}

// Tracer lanes: integrate the ray in their slot, one attempt per pass.
template <class Policy>
__device__ __forceinline__ void flow_tracer(const FlowArgs& A, FlowMail& S, int t) {
  bool busy = false;
  uint32_t item = 0;
  const RayParams* p = nullptr;
  typename Policy::State st;
  unsigned ns = 32;
  for (;;) {
    if (!busy) {
      const uint32_t it = *(volatile uint32_t*)&S.item[t];
      if (it != kQEmpty) {
        __threadfence_block();
        plain::RayStart rs;
        rs.pR = S.start[0][t];
        rs.pTheta = S.start[1][t];
        rs.b = S.start[2][t];
        rs.q = S.start[3][t];
        rs.r0 = S.start[4][t];
        *(volatile uint32_t*)&S.item[t] = kQEmpty;
        item = it;
        p = &A.D[it / A.NM].p;
        Policy::start(*p, rs, st);
        busy = true;
      }
    }
    if (busy && Policy::attempt(*p, st)) {
      double to, po;
      int32_t s;
      uint8_t ss;
      Policy::finish(*p, st, to, po, s, ss);
      S.out[0][t] = to;
      S.out[1][t] = po;
      S.steps[t] = s;
      S.stat[t] = ss;
      __threadfence_block();
      *(volatile uint32_t*)&S.done[t] = item;
      busy = false;
    }
    if (__any_sync(0xffffffffu, busy)) {
      ns = 32;
      continue;
    }
    // no lane of the warp is tracing: wait for rays, or the end (the
    // service stops only when no ray is live, so none is handed over then)
    if (__shfl_sync(0xffffffffu, *(volatile uint32_t*)&S.stop, 0)) break;
    __nanosleep(ns);
    if (ns < 256u) ns *= 2u;
  }
}

// The flow: per block a service warp, worker warps and tracer warps.  A
// warp with nothing to do backs off and looks again until no item is live
// anywhere.
template <class Policy>
__global__ void __launch_bounds__(kFlowThreads, 2) k_flow(FlowArgs A) {
  __shared__ FlowMail S;
  for (int t = threadIdx.x; t < kFlowTracers; t += kFlowThreads) {
    S.item[t] = kQEmpty;
    S.done[t] = kQEmpty;
  }
  if (threadIdx.x == 0) S.stop = 0u;
  __syncthreads();
  const unsigned warp = threadIdx.x >> 5;
  if (warp == 0) {
    flow_busy(S.idle[0]);
    flow_service(A, S);
  } else if (warp <= kFlowWorkers) {
    flow_busy(S.idle[warp]);
    flow_worker<Policy>(A, S.idle[warp]);
  } else {
    flow_tracer<Policy>(A, S, (int)threadIdx.x - 32 * (1 + kFlowWorkers));
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
  const int bps = A.blocks_per_sm < 1 ? 1 : (A.blocks_per_sm > per_sm ? per_sm : A.blocks_per_sm);
  k_flow<Policy><<<sm_count() * bps, kFlowThreads, 0, s>>>(A);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("flow launch: %s", cudaGetErrorString(e));
    return BT_ERR_CUDA;
  }
  return BT_OK;
}

}  // namespace bt
