// trace_kernel.cuh -- persistent ray-tracing kernels with per-lane refill.
//
// One ray per lane.  Rays take from 1 to 1000 attempts, so a warp that ran
// each lane's ray to completion would idle most lanes behind the longest ray.
// Instead every lane whose ray finishes takes the next ray at once, so lanes
// stay busy until the work runs out; only the last rays leave idle lanes.
// Grid builds take rays from a work queue in device memory (warp-aggregated
// atomicAdd on its head); the ray-list form of bt_integrate_rays gives each
// warp a fixed stride of the caller's rays (no state outside the call).
//
// Policy supplies State, begin(), attempt(), finish() -- see PlainPolicy in
// integrate.cu and MixedPolicy / FastPolicy in mixed.cu.
#pragma once

#include "bt_internal.h"
#include "kerr_plain.cuh"

namespace bt {

constexpr uint32_t kLaneIdle = 0xffffffffu;  // needs a ray
constexpr uint32_t kLaneDone = 0xfffffffeu;  // queue exhausted

// A warp refills its idle lanes once at least this many are idle (or none is
// busy): a new ray's set-up and capture test (a Newton and a golden-section
// loop, about two attempts of FP64 work) runs for all refilled lanes at once
// while the warp's other lanes wait, instead of once per finishing lane.
constexpr int kRefillMin = 8;

// Ray seeds of lattice vertex (i, j), Grid::callKernel BT/Grid.h:388-389.
__device__ __forceinline__ void lattice_seed(const LatticeView& L, uint32_t key,
                                             double& th, double& ph) {
  const uint32_t i = key / (uint32_t)L.M, j = key % (uint32_t)L.M;
  th = (double)i / (L.N - 1) * kPi / (2 - L.eq);
  ph = (double)j / L.M * kPi2;
}

// Grid of queue entry k: the last g with qoff[g] <= k (empty grids have
// qoff[g] == qoff[g + 1] and are never chosen).
__device__ __forceinline__ int queue_grid(const uint32_t* __restrict__ qoff, int G,
                                          uint32_t k) {
  int lo = 0, hi = G - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (qoff[mid] <= k) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Vertex key of queue entry k: the front segment (n_hot entries) of grid
// g's trace list, then its back one.
__device__ __forceinline__ uint32_t queue_key(const GridDesc& d, uint32_t r) {
  const uint32_t nh = *(volatile const uint32_t*)&d.ctr->n_hot;
  return r < nh ? d.trace[r] : d.trace[(uint32_t)d.L.N * (uint32_t)d.L.M - 1u - (r - nh)];
}

// Set-up pass of a level: the set-up and capture test of every listed ray
// (ray_setup + checkCelest, BT/Grid.h:524-552), one thread each, so that the
// trace kernel's lanes only integrate.  A ray that must be integrated leaves
// its start in the grid's T-vertex buffers (free until the T-vertex fix
// runs): (p_r, p_theta) in X[0], (b, q) in X[1], and its photon-orbit radius
// as float in its steps slot (overwritten when it finishes); any other ray
// (captured, Newton cap, maxstp 0) is final here and marked traced.
template <class Policy>
__global__ void __launch_bounds__(128)
k_setup_lattice(const GridDesc* __restrict__ D, int G, const uint32_t* __restrict__ qoff) {
  const uint32_t n = qoff[G];
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += gridDim.x * blockDim.x) {
    const int g = queue_grid(qoff, G, k);
    const GridDesc& d = D[g];
    const uint32_t key = queue_key(d, k - qoff[g]);
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
    } else {
      if (go) {  // maxstp 0: odeint1's loop does not run (BT/Metric.h:283)
        typename Policy::State st;
        Policy::start(d.p, rs, st);
        Policy::finish(d.p, st, to, po, s, ss);
      }
      d.L.thphi[key] = make_double2(to, po);
      d.L.steps[key] = s;
      d.L.vstat[key] = ss;
      d.L.vflag[key] = 1;
    }
  }
}

// The start a set-up pass left for the ray of vertex key.
__device__ __forceinline__ plain::RayStart lattice_start(const GridDesc& d, uint32_t key) {
  const double2 a = d.X[0][key], b = d.X[1][key];
  plain::RayStart rs;
  rs.pR = a.x;
  rs.pTheta = a.y;
  rs.b = b.x;
  rs.q = b.y;
  rs.r0 = (double)reinterpret_cast<const float*>(d.L.steps)[key];
  return rs;
}

// Traces the listed vertices of G grids into their lattices, after their
// set-up pass.  Queue entry k is vertex trace[k - qoff[g]] of grid g; each
// grid's rays use that grid's camera and spin (D[g].p).
template <class Policy, int kThreads, int kMinBlocks>
__global__ void __launch_bounds__(kThreads, kMinBlocks)
k_trace_lattice(const GridDesc* __restrict__ D, int G,
                const uint32_t* __restrict__ qoff, uint32_t* qfetch, int refill) {
  const uint32_t n = qoff[G];
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt_mask = (1u << lane) - 1u;
  uint32_t slot = kLaneIdle;
  uint32_t key = 0;
  int g = 0;
  typename Policy::State st;
  for (;;) {
    const bool need = slot == kLaneIdle;
    const unsigned m = __ballot_sync(0xffffffffu, need);
    const unsigned busy = __ballot_sync(0xffffffffu, slot < kLaneDone);
    if (m && (__popc(m) >= refill || !busy)) {
      const int leader = __ffs(m) - 1;
      uint32_t base = 0;
      if ((int)lane == leader) base = atomicAdd(qfetch, (uint32_t)__popc(m));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (need) {
        const uint32_t k = base + (uint32_t)__popc(m & lt_mask);
        if (k < n) {
          g = queue_grid(qoff, G, k);
          const GridDesc& d = D[g];
          key = queue_key(d, k - qoff[g]);
          // rays the set-up pass finished need nothing more
          if (d.L.vflag[key] != 1) {
            Policy::start(d.p, lattice_start(d, key), st);
            slot = k;
          }
        } else {
          slot = kLaneDone;
        }
      }
    }
    if (__all_sync(0xffffffffu, slot == kLaneDone)) break;
    if (slot < kLaneDone) {
      const GridDesc& d = D[g];
      if (Policy::attempt(d.p, st)) {
        double to, po;
        int32_t s;
        uint8_t ss;
        Policy::finish(d.p, st, to, po, s, ss);
        d.L.thphi[key] = make_double2(to, po);
        d.L.steps[key] = s;
        d.L.vstat[key] = ss;
        d.L.vflag[key] = 1;
        slot = kLaneIdle;
      }
    }
  }
}

// Launch of a level's set-up pass and of k_trace_lattice: one block per SM
// times the requested (or the largest resident) number of blocks.  128-thread blocks come in three
// register budgets -- as compiled (3 blocks per SM), capped for 4 and for 5
// resident blocks (with a few spills) -- picked by blocks_per_sm 0-3, 4, 5+.
template <class Policy>
int launch_trace_shape(const GridDesc* D, int G, const uint32_t* qoff,
                       uint32_t* qfetch, TraceShape shape, cudaStream_t s) {
  static int resident[5] = {0, 0, 0, 0, 0};  // per variant, for this Policy
  auto go = [&](auto kernel, int threads, int variant) -> int {
    int& per_sm_max = resident[variant];
    if (!per_sm_max) {
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_max, kernel, threads, 0);
      if (per_sm_max < 1) per_sm_max = 1;
    }
    int per_sm = per_sm_max;
    if (shape.blocks_per_sm > 0 && shape.blocks_per_sm < per_sm) per_sm = shape.blocks_per_sm;
    k_setup_lattice<Policy><<<sm_count() * 8, 128, 0, s>>>(D, G, qoff);
    const int refill = shape.refill > 0 ? shape.refill : kRefillMin;
    kernel<<<sm_count() * per_sm, threads, 0, s>>>(D, G, qoff, qfetch, refill);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      set_error("trace launch: %s", cudaGetErrorString(e));
      return BT_ERR_CUDA;
    }
    return BT_OK;
  };
  switch (shape.threads) {
    case 64: return go(k_trace_lattice<Policy, 64, 1>, 64, 0);
    case 256: return go(k_trace_lattice<Policy, 256, 1>, 256, 1);
    default:
      if (shape.blocks_per_sm >= 5) return go(k_trace_lattice<Policy, 128, 5>, 128, 4);
      if (shape.blocks_per_sm == 4) return go(k_trace_lattice<Policy, 128, 4>, 128, 3);
      return go(k_trace_lattice<Policy, 128, 1>, 128, 2);
  }
}

// Ray-list form (bt_integrate_rays): rays 0..n-1 of caller arrays.  A
// persistent launch (the resident blocks only); warp w of the W warps owns
// rays w, w + W, w + 2W, ... and its idle lanes take them in that order (as
// the grid form, kRefillMin at a time): the warp's next-ray counter is a
// register every lane holds (all lanes add the same ballot count), so nothing
// outside the call's arrays is read or written and calls on different
// streams share no state.  Striding
// spreads each warp's rays over the whole list, so warps see similar mixes
// of short and long rays.
template <class Policy>
__global__ void __launch_bounds__(128)
k_trace_rays(const RayParams p, const double* __restrict__ th_in,
             const double* __restrict__ ph_in, size_t n,
             double* __restrict__ tho, double* __restrict__ pho,
             int32_t* __restrict__ steps, uint8_t* __restrict__ status) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt_mask = (1u << lane) - 1u;
  const size_t W = (size_t)gridDim.x * (blockDim.x >> 5);
  const size_t w = (size_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  size_t next = 0;  // warp-uniform
  bool idle = true, done = false;
  size_t r = 0;
  typename Policy::State st;
  for (;;) {
    const bool need = idle && !done;
    const unsigned m = __ballot_sync(0xffffffffu, need);
    const unsigned busy = __ballot_sync(0xffffffffu, !idle);
    if (m && (__popc(m) >= kRefillMin || !busy)) {
      if (need) {
        const size_t k = w + (next + (size_t)__popc(m & lt_mask)) * W;
        if (k < n) {
          r = k;
          double to, po;
          int32_t s;
          uint8_t ss;
          const bool go = Policy::begin(p, th_in[r], ph_in[r], st, to, po, s, ss);
          if (go && p.maxstp > 0) {
            idle = false;
          } else {
            if (go) Policy::finish(p, st, to, po, s, ss);
            tho[r] = to; pho[r] = po; steps[r] = s;
            if (status) status[r] = ss;
          }
        } else {
          done = true;
        }
      }
      next += (size_t)__popc(m);
    }
    if (__all_sync(0xffffffffu, done)) break;
    if (!idle) {
      if (Policy::attempt(p, st)) {
        double to, po;
        int32_t s;
        uint8_t ss;
        Policy::finish(p, st, to, po, s, ss);
        tho[r] = to; pho[r] = po; steps[r] = s;
        if (status) status[r] = ss;
        idle = true;
      }
    }
  }
}

// Launch of k_trace_rays: as many 128-thread blocks as are resident on the
// device at once, fewer when there are fewer rays than lanes.
template <class Policy>
int launch_trace_rays(const RayParams& p, const double* th, const double* ph, size_t n,
                      double* tho, double* pho, int32_t* steps, uint8_t* status,
                      cudaStream_t s) {
  if (n == 0) return BT_OK;
  static int per_sm = 0;  // per Policy
  if (!per_sm) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace_rays<Policy>, 128, 0);
    if (per_sm < 1) per_sm = 1;
  }
  size_t blocks = (size_t)sm_count() * per_sm;
  const size_t need = (n + 127) / 128;
  if (blocks > need) blocks = need;
  k_trace_rays<Policy><<<(unsigned)blocks, 128, 0, s>>>(p, th, ph, n, tho, pho, steps, status);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("ray launch: %s", cudaGetErrorString(e));
    return BT_ERR_CUDA;
  }
  return BT_OK;
}

}  // namespace bt
