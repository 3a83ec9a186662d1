// bt_internal.h -- shared host/device definitions of the library.
#pragma once

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>

#include <cuda_runtime.h>

#include "blacktracer.h"

namespace bt {

// Constants of the reference (BT/Const.h:2-4 for the host FP64 pair,
// BT/kernel.cuh:24-25 for the FP32 pair used by the per-pixel map).
constexpr double kPi = 3.141592653589793238;
constexpr double kPi2 = kPi * 2.;
constexpr float kPiF = 3.141592653589793238f;
constexpr float kPi2F = 6.283185307179586476f;

// Thread-local last-error message (bt_last_error).
void set_error(const char* fmt, ...);
void clear_error();

// Everything one ray integration needs besides its two seed angles.
// Host-computed scalars that depend only on the camera and the spin are
// evaluated once on the host (glibc libm), which keeps them bit-identical
// to the reference's host evaluation.
struct RayParams {
  // camera (BT/Camera.h:8-11)
  double thetaS, phiS, rS, sp;
  double br, btheta, bphi;
  double alpha, w, wbar, Delta, ro;
  double sqrt_1msp2;   // (double)sqrtf(1 - sp*sp)       BT/Grid.h:529-530
  double sqrtf_delta;  // (double)sqrtf(Delta)            BT/Grid.h:542
  double kb;           // sqrt(1 - btheta*btheta)         BT/Grid.h:532
  double cosS2;        // cos(thetaS)*cos(thetaS)         BT/Grid.h:547
  double sinS2;        // sin(thetaS)*sin(thetaS)
  // spin (BT/Metric.h:36-39)
  double a, asq;
  // capture-test thresholds of checkB_Q that depend only on a
  // (BT/Metric.h:146-147,164-165): b0(r2) and b0(r1)
  double b_lo, b_hi;
  // step control (BT/Metric.h:311-314)
  double eps, h1, z_end;
  int32_t maxstp;
  int32_t precision;
  double fp64_band;
  double r_ph_lo, r_ph_hi;  // prograde / retrograde equatorial photon orbits
};

// Fills RayParams from a camera, a spin and options (host, glibc libm).
int make_ray_params(const bt_camera* cam, double a, const bt_integ_opts* o,
                    RayParams* p);

int sm_count();

// Ray-list integration (integrate.cu / mixed.cu).
int launch_integrate(const RayParams& p, const double* th, const double* ph,
                     size_t n, double* tho, double* pho, int32_t* steps,
                     uint8_t* status, cudaStream_t s);
int launch_integrate_mixed(const RayParams& p, const double* th,
                           const double* ph, size_t n, double* tho,
                           double* pho, int32_t* steps, uint8_t* status,
                           cudaStream_t s);
int launch_integrate_fast(const RayParams& p, const double* th, const double* ph,
                          size_t n, double* tho, double* pho, int32_t* steps,
                          uint8_t* status, cudaStream_t s);

// Dense-lattice view of one grid on the device (grid.cu).  Vertex (i, j) of
// the reference's CamToCel map lives at index i*M + j.
struct LatticeView {
  int32_t N, M, eq, maxlevel, startlevel;
  double2* thphi;   // (theta, phi) of existing vertices
  int32_t* steps;   // the reference's steps vector (BT/Grid.h:577)
  uint8_t* vflag;   // 0 absent, 1 traced, 2 claimed (placeholder)
  uint8_t* vstat;   // BT_RAY_* of traced vertices
  int8_t* blevel;   // level of the leaf block with top-left (i, j), or -1
};

// Work counters of a grid build (device memory).
struct GridCounters {
  uint32_t n_check;   // blocks to examine at the current level
  uint32_t n_next;    // blocks for the next level
  uint32_t n_trace;   // vertices to trace: n_hot from the front of the
                      // trace list, the rest from its back
  uint32_t n_hot;     // vertices whose parent block holds a slow ray
  uint32_t n_cold;
  uint32_t fetch;     // work-queue head of the trace kernel
  uint32_t n_amb;     // mixed form: blocks whose decision waits for FP64
  uint32_t n_retrace; // mixed form: corners re-traced in FP64
  uint32_t overflow;  // a work list overflowed (should never happen)
  uint32_t traced_lo; // total rays traced (64-bit split)
  uint32_t traced_hi;
  uint32_t tfix_flags[16];  // T-vertex fix: "changed" flag per pass
  uint32_t leaf_off[16];    // T-vertex fix: leaf-list offset per level
  uint32_t n_leaf;
  uint32_t err;       // nonzero: a bounded loop gave up
};

// One grid of a build set as the build kernels see it (device memory, one
// entry per grid): lattice, ray parameters of its camera and spin, work
// lists and counters.
struct GridDesc {
  LatticeView L;
  RayParams p;
  uint32_t* list[2];  // block lists of consecutive levels (ping-pong)
  uint32_t* trace;    // vertices to trace this level
  uint32_t* leaves;   // leaf blocks (level < max) in level order
  double2* X[2];      // T-vertex fix pass buffers
  GridCounters* ctr;
};

// Launch shape of the ray-tracing kernel: threads per block (64, 128 or
// 256), resident blocks per SM (0 = as many as fit) and the number of idle
// lanes a warp waits for before it refills them (0 = kRefillMin).
struct TraceShape {
  int threads;
  int blocks_per_sm;
  int refill;
};

// Traces the listed vertices of all G grids in one persistent launch: the
// per-grid trace counts are laid end to end (qoff[g] = first queue entry of
// grid g, qoff[G] = total) and lanes take entries from the shared queue head
// *qfetch.  Plain form in integrate.cu, mixed form in mixed.cu.
int launch_trace_plain(const GridDesc* D, int G, const uint32_t* qoff,
                       uint32_t* qfetch, TraceShape shape, cudaStream_t s);
int launch_trace_mixed(const GridDesc* D, int G, const uint32_t* qoff,
                       uint32_t* qfetch, TraceShape shape, cudaStream_t s);
int launch_trace_fast(const GridDesc* D, int G, const uint32_t* qoff,
                      uint32_t* qfetch, TraceShape shape, cudaStream_t s);

// A new vertex is hot when its parent block has a corner whose ray took at
// least kHotSteps attempts (its own ray is then likely slow too): both build
// forms start hot rays first.
constexpr int32_t kHotSteps = 100;

// The refinement levels of a set as one persistent launch (grid_flow.cuh):
// the flow's queues and sync words, its control block, and its launch per
// form (integrate.cu, mixed.cu).
struct FlowArgs;
int launch_flow_plain(const FlowArgs& A, cudaStream_t s);
int launch_flow_mixed(const FlowArgs& A, cudaStream_t s);
int launch_flow_fast(const FlowArgs& A, cudaStream_t s);

// Map grid of a built grid into a caller's buffer (grid.cu).
int grid_map_export_into(const bt_grid* g, float* dst, cudaStream_t s);

}  // namespace bt

#define BT_CUDA_TRY(expr)                                                   \
  do {                                                                      \
    cudaError_t e_ = (expr);                                                \
    if (e_ != cudaSuccess) {                                                \
      bt::set_error("%s:%d %s: %s", __FILE__, __LINE__, #expr,              \
                    cudaGetErrorString(e_));                                \
      return BT_ERR_CUDA;                                                   \
    }                                                                       \
  } while (0)

#define BT_ARG_CHECK(cond, msg)                                             \
  do {                                                                      \
    if (!(cond)) {                                                          \
      bt::set_error("invalid argument: %s", msg);                           \
      return BT_ERR_ARG;                                                    \
    }                                                                       \
  } while (0)
