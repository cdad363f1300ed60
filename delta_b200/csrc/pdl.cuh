// Programmatic dependent launch for the kernels of the replayed time step.
//
// A kernel launched with launch_dep(true, ...) may start while the kernel before it on
// the stream is still running (the launch attribute cudaLaunchAttributeProgrammatic-
// StreamSerialization; under stream capture it becomes a programmatic edge of the graph).
// Every such kernel calls dep_sync() as its first statement: griddepcontrol.wait returns
// once the previous kernel has completed and its memory operations are visible, so nothing
// the kernel reads or writes is touched before then; griddepcontrol.launch_dependents then
// lets the next kernel's launch begin.  What overlaps is the launch and block scheduling of
// a kernel with the end of the one before it.  Launched without the attribute (the stepped
// path), dep_sync() returns at once.  No kernel launched this way waits on another CTA, so
// CTAs of a dependent kernel that are resident early cannot hold up the kernel before it.
#pragma once

#include <cuda_runtime.h>

#include <utility>

namespace delta {

__device__ __forceinline__ void dep_sync() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// kernel<<<grid, block, smem, st>>>(args...), as a programmatic dependent launch when dep.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_dep(bool dep, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args &&...args) {
  if (!dep) {
    kernel<<<grid, block, smem, st>>>(std::forward<Args>(args)...);
    return cudaGetLastError();
  }
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace delta
