// Kernel launches with programmatic dependent launch.
//
// The kernels of the step and rebuild sequences call grid_dep_sync()
// (sc_common.cuh) before they touch what the kernel before them writes, so
// they may be launched with programmatic stream serialization: each one's
// blocks start as the previous kernel's retire instead of after its
// completion, in host-driven steps and inside captured graphs alike.  The
// attribute is on by default; SIMCORE_PDL=0 in the environment switches it
// off for the process, and a PdlOff object for the launches of its thread
// while it lives.
#pragma once

#include <cuda_runtime.h>

#include <utility>

namespace sc {

bool pdl_enabled();

struct PdlOff {
  bool prev;
  PdlOff();
  ~PdlOff();
};

template <typename... P, typename... A>
inline cudaError_t launch_pdl(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t st, A &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  if (pdl_enabled()) {
    cfg.attrs = at;
    cfg.numAttrs = 1;
  }
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

}  // namespace sc
