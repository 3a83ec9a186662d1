// noalloc.cu -- ray integration with host buffers, without any allocation.
//
// bt_integrate_rays_host stages the rays in device memory that it allocates
// with cudaMalloc on first use and grows on demand.  Some callers cannot
// allow that: a render or serving thread that must never stall on the
// implicit device synchronisation of cudaMalloc/cudaFree, a plugin host that
// gives each plugin a fixed device-memory budget and rejects allocations
// beyond it, or middleware whose device memory is owned by another runtime's
// allocator.  bt_integrate_rays_host_static serves them: its staging area is
// a file-scope static __device__ array of fixed size (kStaticMaxRays rays),
// which every GPU that loads this library holds until the process exits.
#include <cstring>
#include <mutex>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "bt_internal.h"

namespace {

constexpr size_t kStaticMaxRays = 65536;
constexpr int kMaxDevices = 64;

// Layout: theta_in, phi_in, theta_out, phi_out (double each), steps (int32),
// status (uint8), each kStaticMaxRays long, in this order.
constexpr size_t kStageBytes = kStaticMaxRays * (4 * sizeof(double) + sizeof(int32_t) + 1);

static __device__ __align__(256) unsigned char g_static_stage[kStageBytes];

std::mutex g_stage_mu;
void* g_stage_addr[kMaxDevices] = {};
CUcontext g_stage_ctx[kMaxDevices] = {};
PFN_cuCtxGetCurrent_v4000 g_ctx_current = nullptr;

// The current context, through the driver entry point the runtime exposes
// (no link against the driver library); nullptr if it cannot be had.
CUcontext current_context() {
  if (!g_ctx_current) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    g_ctx_current = (PFN_cuCtxGetCurrent_v4000)fn;
  }
  CUcontext c = nullptr;
  return g_ctx_current(&c) == CUDA_SUCCESS ? c : nullptr;
}

// Device address of the static staging array on the current device.  In
// host code the symbol names a host-side stand-in, not device memory, so the
// address is looked up with the device current and kept, per device and per
// context: after cudaDeviceReset the device gets a new context, the module
// is loaded again, and the address is looked up again.
int stage_address(void** out) {
  int dev = 0;
  BT_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    bt::set_error("device ordinal %d is beyond the %d devices supported", dev, kMaxDevices);
    return BT_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(g_stage_mu);
  // No current context yet on this thread (the runtime makes the primary
  // context current on first use) also leads to a lookup, which does that.
  const CUcontext ctx = current_context();
  if (!g_stage_addr[dev] || ctx == nullptr || ctx != g_stage_ctx[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_stage);
    if (e != cudaSuccess || p == nullptr) {
      bt::set_error("cudaGetSymbolAddress of the static staging area failed: %s",
                    cudaGetErrorString(e));
      return BT_ERR_CUDA;
    }
    g_stage_addr[dev] = p;
    g_stage_ctx[dev] = current_context();
  }
  *out = g_stage_addr[dev];
  return BT_OK;
}

}  // namespace

extern "C" {

size_t bt_integrate_rays_host_static_capacity(void) { return kStaticMaxRays; }

int bt_integrate_rays_host_static(const bt_camera* cam, double a,
                                  const double* theta, const double* phi,
                                  size_t n, double* theta_out, double* phi_out,
                                  int32_t* steps, uint8_t* status,
                                  const bt_integ_opts* o, void* stream) {
  bt::clear_error();
  BT_ARG_CHECK(cam != nullptr, "cam is NULL");
  if (n == 0) return BT_OK;
  BT_ARG_CHECK(theta && phi && theta_out && phi_out && steps, "NULL array pointer");
  if (n > kStaticMaxRays) {
    bt::set_error("invalid argument: %zu rays exceed the static staging capacity of %zu rays "
                  "(call it in chunks, or use bt_integrate_rays_host)",
                  n, kStaticMaxRays);
    return BT_ERR_ARG;
  }
  bt::RayParams p;
  if (int rc = bt::make_ray_params(cam, a, o, &p)) {
    bt::set_error("invalid camera or integrator options");
    return rc;
  }
  void* base = nullptr;
  if (int rc = stage_address(&base)) return rc;
  double* dth = (double*)base;
  double* dph = dth + kStaticMaxRays;
  double* dto = dph + kStaticMaxRays;
  double* dpo = dto + kStaticMaxRays;
  int32_t* dst = (int32_t*)(dpo + kStaticMaxRays);
  uint8_t* dss = (uint8_t*)(dst + kStaticMaxRays);
  cudaStream_t s = (cudaStream_t)stream;
  // Every input and output slot of rays [0, n) is written before it is read,
  // so nothing left from an earlier call needs clearing.
  BT_CUDA_TRY(cudaMemcpyAsync(dth, theta, n * sizeof(double), cudaMemcpyHostToDevice, s));
  BT_CUDA_TRY(cudaMemcpyAsync(dph, phi, n * sizeof(double), cudaMemcpyHostToDevice, s));
  if (int rc = bt::launch_integrate(p, dth, dph, n, dto, dpo, dst, dss, s)) return rc;
  BT_CUDA_TRY(cudaMemcpyAsync(theta_out, dto, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  BT_CUDA_TRY(cudaMemcpyAsync(phi_out, dpo, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  BT_CUDA_TRY(cudaMemcpyAsync(steps, dst, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  if (status) BT_CUDA_TRY(cudaMemcpyAsync(status, dss, n, cudaMemcpyDeviceToHost, s));
  BT_CUDA_TRY(cudaStreamSynchronize(s));
  return BT_OK;
}

}  // extern "C"
