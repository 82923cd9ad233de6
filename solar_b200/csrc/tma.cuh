// tma.cuh -- thin wrappers over the sm_100a tensor-memory-accelerator (TMA) tile loads
// and shared-memory mbarriers used by the streaming stencil kernels.
//
// Only plain (single-CTA) tile loads are used: every load reads this GPU's own memory.
//
// Every wait on an mbarrier is bounded: after the kernel's limit of polls (kWaitPolls, about
// a second or more -- each mbarrier.try_wait may suspend the thread for a while before it
// reports that the phase is still open) the waiting thread gets `false` and records an
// error code in the context's device error word, which the host turns into
// SOLAR_ERR_TIMEOUT.  A CTA whose wait gave up stops issuing loads, leaves its plane loop
// at the next CTA barrier and, before it exits, waits (bounded again) for every load it
// issued and did not consume, so that no bulk copy is still writing into its shared
// memory when the SM hands that memory to another CTA.  A copy that has not landed after
// a second limit is taken as lost.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace solar {

constexpr uint32_t kWaitPolls = 1u << 22;   // bound of one wait: polls of try_wait

// Codes a kernel leaves in the context's device error word.
enum DeviceError : int {
  kErrStageLead = 1,        // stage kernel: lead ring (p, v_r planes) wait gave up
  kErrStageTile = 2,        // stage kernel: tile ring wait gave up
  kErrFilterRing = 3,       // filter kernel: ring wait gave up
  kErrEdgeRing = 4,         // edge kernel: ring wait gave up
  kErrAdjointRing = 5,      // transposed stage kernel: ring wait gave up
  kErrForcingSample = 16,   // a forcing time sample outside the loaded samples was needed
};

// Kernels that take part in failure-injection tests (solar_gpu_inject_wait_timeout).
enum InjectKernel : int { kInjEdge = 1, kInjStage = 2, kInjFilter = 4, kInjAdjStage = 8 };

// Wait control carried in a kernel's arguments: the device error word, the bound of one
// wait in polls, and the injection switch of failure-detection tests (nonzero: the
// producer issues no loads, so the first wait runs out with nothing in flight).
struct WaitCtl {
  int* err;
  uint32_t polls;
  int no_loads;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait_u32(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  return mbar_try_wait_u32(smem_u32(bar), parity);
}

// Wait for the phase with the given parity to complete, at most `polls` tests.
__device__ __forceinline__ bool mbar_wait_polls(uint64_t* bar, uint32_t parity, uint32_t polls) {
  const uint32_t b = smem_u32(bar);
  for (uint32_t it = 0; it < polls; ++it)
    if (mbar_try_wait_u32(b, parity)) return true;
  return false;
}

// Consumer wait: on giving up, record `code` in the device error word.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, const WaitCtl& w, int code) {
  if (mbar_wait_polls(bar, parity, w.polls)) return true;
  if (w.err) atomicExch(w.err, code);
  return false;
}

// Before a CTA that gave up exits: wait (bounded) for the loads of planes [first, end) of a
// ring of `slots` mbarriers filled in plane order from plane `base` (plane m in slot
// (m - base) % slots, phase parity ((m - base) / slots) & 1).
__device__ __forceinline__ void mbar_drain(uint64_t* bars, int slots, int base, int first, int end, uint32_t polls) {
  for (int m = first; m < end; ++m) {
    const int q = m - base;
    mbar_wait_polls(&bars[q % slots], (uint32_t)((q / slots) & 1), polls);
  }
}

// 3-D tile load global -> shared, completion signalled on `bar` (transaction bytes).
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// Untiled bulk copy global -> shared of `bytes` bytes (both addresses 16-byte aligned,
// bytes a multiple of 16), completion signalled on `bar` (transaction bytes).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Programmatic dependent launch.  A kernel launched with programmatic stream serialization
// starts as its predecessor's last CTAs exit, before that grid has fully completed; it must
// call grid_dependency_wait() before it reads anything the predecessor (or an earlier
// kernel) wrote and before it writes anything, and only constant tables may be read before
// that.  (No kernel here triggers its successor earlier: successor CTAs waiting on SMs during
// a multi-wave stage kernel's last wave cost the FP32 step 1.5%.)
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

}  // namespace solar
