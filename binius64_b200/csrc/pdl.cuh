// Programmatic dependent launch for the chains of dependent kernels in the sumcheck round loops.
//
// A kernel launched through launch_pdl may be scheduled while the previous kernel on its stream is
// still running, which hides most of the ~3 us gap between dependent launches.  Such a kernel
// must call pdl_wait() before it touches memory the previous kernel writes: griddepcontrol.wait
// returns once the prerequisite grid has completed and its memory operations are visible (for a
// kernel launched without the attribute it returns at once).  pdl_trigger() lets the next kernel
// of the stream be launched early; it does not release the next kernel's pdl_wait(), so it may be
// called anywhere.
#pragma once
#include <cuda_runtime.h>

namespace bgpu {

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Whether the calling thread's launch_pdl calls use programmatic dependent launch (default on).
// A dependent grid scheduled early holds its CTAs' SM slots while it waits; a thread that
// proves beside others on the same GPU (a proving-queue worker) may launch plainly instead.
bool pdl_enabled();
void set_pdl_enabled(bool on);

template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                       cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

}  // namespace bgpu
