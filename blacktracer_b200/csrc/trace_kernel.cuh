// trace_kernel.cuh -- persistent ray-tracing kernels with per-lane refill.
//
// One ray per lane.  Rays take from 1 to 1000 attempts, so a warp that ran
// each lane's ray to completion would idle most lanes behind the longest ray.
// Instead every lane whose ray finishes takes the next ray from a global work
// queue at once (warp-aggregated atomicAdd on the queue head), so lanes stay
// busy until the queue is empty; only the last rays leave idle lanes.
//
// Policy supplies State, begin(), attempt(), finish() -- see PlainPolicy in
// integrate.cu and MixedPolicy in mixed.cu.
#pragma once

#include "bt_internal.h"

namespace bt {

constexpr uint32_t kLaneIdle = 0xffffffffu;  // needs a ray
constexpr uint32_t kLaneDone = 0xfffffffeu;  // queue exhausted

// Ray seeds of lattice vertex (i, j), Grid::callKernel BT/Grid.h:388-389.
__device__ __forceinline__ void lattice_seed(const LatticeView& L, uint32_t key,
                                             double& th, double& ph) {
  const uint32_t i = key / (uint32_t)L.M, j = key % (uint32_t)L.M;
  th = (double)i / (L.N - 1) * kPi / (2 - L.eq);
  ph = (double)j / L.M * kPi2;
}

// Traces lattice vertices keys[0 .. ctr->n_trace) into the lattice.
template <class Policy>
__global__ void __launch_bounds__(128)
k_trace_lattice(const RayParams p, const LatticeView L,
                const uint32_t* __restrict__ keys, GridCounters* ctr) {
  const uint32_t n = *(volatile uint32_t*)&ctr->n_trace;
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt_mask = (1u << lane) - 1u;
  uint32_t slot = kLaneIdle;
  uint32_t key = 0;
  typename Policy::State st;
  for (;;) {
    const bool need = slot == kLaneIdle;
    const unsigned m = __ballot_sync(0xffffffffu, need);
    if (m) {
      const int leader = __ffs(m) - 1;
      uint32_t base = 0;
      if ((int)lane == leader) base = atomicAdd(&ctr->fetch, (uint32_t)__popc(m));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (need) {
        const uint32_t k = base + (uint32_t)__popc(m & lt_mask);
        if (k < n) {
          key = keys[k];
          double th, ph, to, po;
          int32_t s;
          uint8_t ss;
          lattice_seed(L, key, th, ph);
          if (Policy::begin(p, th, ph, st, to, po, s, ss)) {
            slot = k;
          } else {
            L.thphi[key] = make_double2(to, po);
            L.steps[key] = s;
            L.vstat[key] = ss;
            L.vflag[key] = 1;
          }
        } else {
          slot = kLaneDone;
        }
      }
    }
    if (__all_sync(0xffffffffu, slot == kLaneDone)) break;
    if (slot < kLaneDone) {
      if (Policy::attempt(p, st)) {
        double to, po;
        int32_t s;
        uint8_t ss;
        Policy::finish(p, st, to, po, s, ss);
        L.thphi[key] = make_double2(to, po);
        L.steps[key] = s;
        L.vstat[key] = ss;
        L.vflag[key] = 1;
        slot = kLaneIdle;
      }
    }
  }
}

// Ray-list form (bt_integrate_rays): rays 0..n-1, queue head in *fetch.
template <class Policy>
__global__ void __launch_bounds__(128)
k_trace_list(const RayParams p, const double* __restrict__ th_in,
             const double* __restrict__ ph_in, size_t n,
             double* __restrict__ tho, double* __restrict__ pho,
             int32_t* __restrict__ steps, uint8_t* __restrict__ status,
             unsigned long long* fetch) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt_mask = (1u << lane) - 1u;
  bool idle = true, done = false;
  size_t r = 0;
  typename Policy::State st;
  for (;;) {
    const bool need = idle && !done;
    const unsigned m = __ballot_sync(0xffffffffu, need);
    if (m) {
      const int leader = __ffs(m) - 1;
      unsigned long long base = 0;
      if ((int)lane == leader)
        base = atomicAdd(fetch, (unsigned long long)__popc(m));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (need) {
        const unsigned long long k = base + (unsigned)__popc(m & lt_mask);
        if (k < n) {
          r = (size_t)k;
          double to, po;
          int32_t s;
          uint8_t ss;
          if (Policy::begin(p, th_in[r], ph_in[r], st, to, po, s, ss)) {
            idle = false;
          } else {
            tho[r] = to; pho[r] = po; steps[r] = s;
            if (status) status[r] = ss;
          }
        } else {
          done = true;
        }
      }
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

}  // namespace bt
