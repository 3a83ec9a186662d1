// mixed.cu -- launchers of the mixed-precision (kerr_mixed.cuh) and fast FP64
// (kerr_fast.cuh) integrators.  Compiled with FMA contraction on: these forms
// are not bit-matched to the reference; their error against the FP64 oracle
// is measured instead.
#include <algorithm>

#include "bt_internal.h"
#include "kerr_fast.cuh"
#include "kerr_mixed.cuh"
#include "trace_kernel.cuh"
#include "grid_flow.cuh"

namespace bt {

struct MixedPolicy {
  using State = mixed::MixedState;
  static __device__ __forceinline__ bool begin(const RayParams& p, double th,
                                               double ph, State& s, double& to,
                                               double& po, int32_t& st,
                                               uint8_t& ss) {
    return mixed::begin_ray(p, th, ph, s, to, po, st, ss);
  }
  static __device__ __forceinline__ void start(const RayParams& p, const plain::RayStart& rs,
                                               State& s) {
    mixed::start_ray(p, rs, s);
  }
  static __device__ __forceinline__ bool attempt(const RayParams& p, State& s) {
    return mixed::attempt(p, s);
  }
  static __device__ __forceinline__ void finish(const RayParams& p,
                                                const State& s, double& to,
                                                double& po, int32_t& st,
                                                uint8_t& ss) {
    plain::finish_ray(p, s.s, to, po, st, ss);
  }
};

struct FastPolicy {
  using State = fast::FastState;
  static __device__ __forceinline__ bool begin(const RayParams& p, double th,
                                               double ph, State& s, double& to,
                                               double& po, int32_t& st,
                                               uint8_t& ss) {
    return fast::begin_ray(p, th, ph, s, to, po, st, ss);
  }
  static __device__ __forceinline__ void start(const RayParams& p, const plain::RayStart& rs,
                                               State& s) {
    fast::start_ray(p, rs, s);
  }
  static __device__ __forceinline__ bool attempt(const RayParams& p, State& s) {
    return fast::attempt(p, s);
  }
  static __device__ __forceinline__ void finish(const RayParams& p,
                                                const State& s, double& to,
                                                double& po, int32_t& st,
                                                uint8_t& ss) {
    plain::finish_ray(p, s, to, po, st, ss);
  }
};

int launch_integrate_mixed(const RayParams& p, const double* th,
                           const double* ph, size_t n, double* tho,
                           double* pho, int32_t* steps, uint8_t* status,
                           cudaStream_t s) {
  return launch_trace_rays<MixedPolicy>(p, th, ph, n, tho, pho, steps, status, s);
}

int launch_trace_mixed(const GridDesc* D, int G, const uint32_t* qoff,
                       uint32_t* qfetch, TraceShape shape, cudaStream_t s) {
  return launch_trace_shape<MixedPolicy>(D, G, qoff, qfetch, shape, s);
}

int launch_integrate_fast(const RayParams& p, const double* th, const double* ph,
                          size_t n, double* tho, double* pho, int32_t* steps,
                          uint8_t* status, cudaStream_t s) {
  return launch_trace_rays<FastPolicy>(p, th, ph, n, tho, pho, steps, status, s);
}

int launch_trace_fast(const GridDesc* D, int G, const uint32_t* qoff,
                      uint32_t* qfetch, TraceShape shape, cudaStream_t s) {
  return launch_trace_shape<FastPolicy>(D, G, qoff, qfetch, shape, s);
}

int launch_flow_fast(const FlowArgs& A, cudaStream_t s) {
  return launch_flow<FastPolicy>(A, s);
}

int launch_flow_mixed(const FlowArgs& A, cudaStream_t s) {
  return launch_flow<MixedPolicy>(A, s);
}

}  // namespace bt

namespace bt {
namespace {
__global__ void k_probe_rcp(const double* __restrict__ x, double* __restrict__ out, size_t n) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x)
    out[k] = fast::rcp_nr(x[k]);
}
}  // namespace
}  // namespace bt

extern "C" int bt_probe_fast_rcp(const double* x, double* out, size_t n, void* stream) {
  bt::clear_error();
  BT_ARG_CHECK(x && out, "NULL pointer");
  if (n == 0) return BT_OK;
  bt::k_probe_rcp<<<(unsigned)std::min<size_t>((n + 255) / 256, 4096), 256, 0,
                    (cudaStream_t)stream>>>(x, out, n);
  BT_CUDA_TRY(cudaGetLastError());
  return BT_OK;
}
