// noalloc.cu -- the reference's per-step norm of a device-resident field, computed without
// allocating anything.
//
// Who needs it.  Some callers cannot call cudaMalloc.  One is a host whose device memory
// is owned and budgeted by another runtime -- a Fortran/OpenACC driver or a framework
// memory pool that has already claimed the GPU's memory at start-up -- so a library that
// allocates on its own can fail or fragment that budget.  The other is a per-step
// diagnostic hook: the reference prints norm(v_r) after every step (cube.f90:77,
// auxiliary.f90:100-125), and such a hook must not pay the device-wide synchronisation
// that cudaMalloc / cudaFree can cause in the middle of a time loop.  For them,
// solar_gpu_norm_noalloc takes the field and the result slot as device pointers the
// caller already owns, and keeps its only scratch -- one partial sum per (zone, radial
// plane) -- in a fixed-size file-scope device array.
//
// Limits and sharing.  The array holds kNormMaxPlanes partials, so nr <= kNormMaxPlanes/6
// (2048); larger grids, and planes of more than INT_MAX points, are rejected with
// SOLAR_ERR_ARG before anything is launched.  Every GPU that loads the library
// holds the array (96 KiB) until the process exits.  All calls share it and it keeps the
// previous call's partials; each call overwrites exactly the partials it then reads, so
// nothing has to be cleared first.  Two calls whose kernels overlap on the GPU (different
// streams, same device) race on the array: serialise them.
//
// Set-up.  The array's device address is resolved with cudaGetSymbolAddress (which
// allocates nothing) on the first call in each CUDA context, with that context current,
// and cached together with the context's unique id: after a cudaDeviceReset the device
// gets a new primary context, the module is loaded again, and the next call resolves the
// new address instead of using a dead one.  That first call per context should come
// before any stream capture.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <climits>
#include <cstdio>
#include <mutex>

#include "../../include/solar_gpu.h"

namespace solar {
int report_error(int code, const char* msg);   // defined in solar_gpu.cu
}

namespace {

constexpr int kNormMaxPlanes = 6 * 2048;      // one partial per (zone, radial plane)
constexpr int kMaxDevices = 64;
constexpr int kThreads = 256;

static __device__ __align__(256) double g_norm_partials[kNormMaxPlanes];

// Device address of g_norm_partials per device, valid for the context whose id is cached
// beside it (nullptr until that device is set up).
double* g_partials[kMaxDevices] = {};
unsigned long long g_ctx_id[kMaxDevices] = {};
std::mutex g_setup_mutex;

// Unique id of the calling thread's current CUDA context (driver entry points reached
// through the runtime, so the library needs no -lcuda); 0 when unavailable.
unsigned long long current_context_id() {
  static PFN_cuCtxGetCurrent_v4000 get_current = nullptr;
  static PFN_cuCtxGetId_v12000 get_id = nullptr;
  static bool looked_up = false;
  if (!looked_up) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(p);
    p = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(p);
    looked_up = true;
  }
  if (!get_current || !get_id) return 0;
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// One CTA per (zone, plane): sum of f^2 over the plane in a fixed order.
__global__ void __launch_bounds__(kThreads) norm_plane_sums(const double* __restrict__ f, int plane,
                                                            double* __restrict__ part) {
  __shared__ double red[kThreads];
  const double* p = f + (long long)blockIdx.x * plane;
  double acc = 0.0;
  for (int i = threadIdx.x; i < plane; i += kThreads) acc += p[i] * p[i];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// One CTA: add the partials in a fixed order and apply auxiliary.f90:122.
__global__ void __launch_bounds__(kThreads) norm_finish(const double* __restrict__ part, int nparts, double scale,
                                                        double* __restrict__ out) {
  __shared__ double red[kThreads];
  double acc = 0.0;
  for (int i = threadIdx.x; i < nparts; i += kThreads) acc += part[i];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sqrt(red[0] * scale);
}

}  // namespace

extern "C" int solar_gpu_norm_noalloc(const double* d_field, int nx, int nr, double* d_out, void* stream) {
  if (!d_field || !d_out) return solar::report_error(SOLAR_ERR_ARG, "solar_gpu_norm_noalloc: null device pointer");
  if (nx < 1 || nr < 1) return solar::report_error(SOLAR_ERR_ARG, "solar_gpu_norm_noalloc: nx and nr must be >= 1");
  if ((long long)nx * nx > INT_MAX)
    return solar::report_error(SOLAR_ERR_ARG, "solar_gpu_norm_noalloc: nx * nx exceeds INT_MAX points per plane");
  if (6LL * nr > kNormMaxPlanes) {
    char msg[160];
    std::snprintf(msg, sizeof(msg),
                  "solar_gpu_norm_noalloc: nr = %d exceeds the fixed scratch of %d planes (nr <= %d)", nr,
                  kNormMaxPlanes, kNormMaxPlanes / 6);
    return solar::report_error(SOLAR_ERR_ARG, msg);
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return solar::report_error(SOLAR_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return solar::report_error(SOLAR_ERR_ARG, "solar_gpu_norm_noalloc: device ordinal too large");
  double* part = nullptr;
  {
    // First call in a context (that context current): resolve the array's device address.
    // The host-side name g_norm_partials is only a stand-in; kernels need this address.
    // (cudaGetSymbolAddress also creates the device's primary context if it does not exist
    // yet, so the id is read after it.)  Without a context id the address is resolved on
    // every call.
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    const unsigned long long id = current_context_id();
    if (g_partials[dev] && id != 0 && g_ctx_id[dev] == id) {
      part = g_partials[dev];
    } else {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_norm_partials);
      if (e != cudaSuccess) return solar::report_error(SOLAR_ERR_CUDA, cudaGetErrorString(e));
      part = static_cast<double*>(p);
      g_partials[dev] = part;
      g_ctx_id[dev] = current_context_id();
    }
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int planes = 6 * nr;
  const int plane = nx * nx;
  norm_plane_sums<<<planes, kThreads, 0, s>>>(d_field, plane, part);
  norm_finish<<<1, kThreads, 0, s>>>(part, planes, 6.0 / ((double)nx * nx * nr), d_out);
  e = cudaGetLastError();
  if (e != cudaSuccess) return solar::report_error(SOLAR_ERR_CUDA, cudaGetErrorString(e));
  return SOLAR_OK;
}
