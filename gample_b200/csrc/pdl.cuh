// pdl.cuh -- programmatic dependent launch for chains of dependent kernels.
//
// A kernel launched with launch_pdl() may start while the kernel before it
// on the stream is finishing, so its launch latency overlaps that kernel's
// tail. It must call grid_dependency_wait() before its first global-memory
// access (griddepcontrol.wait returns once the previous grid has completed
// and its memory is visible; at once when there is no programmatic
// predecessor), and calls grid_dependents_launch() once it runs, which lets
// the next such kernel be scheduled. A kernel launched normally after one of
// these waits for its completion as usual.
#pragma once

#include <cuda_runtime.h>

#include "device.hpp"

namespace gample {

__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dependents_launch() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KArgs, typename... Args>
void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  GP_CUDA(cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...));
  GP_LAUNCH_CHECK();
}

}  // namespace gample
