// Fast variant of the integrator for the mixed-precision step, compiled with
// --fmad=true: the algorithm of sc_step.cuh with FMA contraction, one
// reciprocal per shared denominator and rsqrt normalisation.  FP64
// throughout; not bit-identical to the reference (differences at the level
// of FP64 rounding), which the mixed path does not claim.
#include <cuda_runtime.h>

#include "sc_common.cuh"
#include "sc_kernels.h"
#include "sc_launch.h"
#include "sc_pair.cuh"
#include "sc_step.cuh"
#include "sc_step_warp.cuh"

namespace sc {

template <int ND, int MAXC>
static void set_attr_fast(size_t smem) {
  cudaFuncSetAttribute(k_integrate<ND, 1, true, MAXC, false>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaFuncSetAttribute(k_integrate<ND, 1, true, MAXC, true>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaFuncSetAttribute(k_integrate<ND, 1, true, MAXC, false, true>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaFuncSetAttribute(k_integrate<ND, 1, true, MAXC, true, true>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

// The block kernel compiled for up to MAXC sites, with compile-time offsets
// when the block has exactly MAXC.
template <int ND, bool FUSE, int MAXC>
static void launch_block_fast(const SysConst &k, const DevState &d, int nblocks, int C, size_t smem,
                              int midstep, int rbuf, int interaction, int capture, cudaStream_t st) {
  if (C == MAXC)
    launch_pdl(k_integrate<ND, 1, true, MAXC, FUSE, true>, dim3(nblocks), dim3(C), smem, st, k, d,
               midstep, rbuf, interaction, capture);
  else
    launch_pdl(k_integrate<ND, 1, true, MAXC, FUSE>, dim3(nblocks), dim3(C), smem, st, k, d,
               midstep, rbuf, interaction, capture);
}

void prepare_integrate_fast(int C) {
  size_t smem = integrate_smem_bytes(C, C / 2);
  if (C <= 128) {
    set_attr_fast<3, 128>(smem);
    set_attr_fast<2, 128>(smem);
  } else if (C <= 192) {
    set_attr_fast<3, 192>(smem);
    set_attr_fast<2, 192>(smem);
  } else if (C <= 256) {
    set_attr_fast<3, 256>(smem);
    set_attr_fast<2, 256>(smem);
  } else {
    set_attr_fast<3, 512>(smem);
    set_attr_fast<2, 512>(smem);
  }
}

template <int ND, bool FUSE>
static int launch_fast(const SysConst &k, const DevState &d, int nblocks, int C, int midstep,
                       int rbuf, int interaction, int capture, cudaStream_t st) {
  int launched = 0;
  if (d.n_wg > 0) {
    const int grid = (d.n_wg + kIntWarps - 1) / kIntWarps;
    launch_pdl(k_integrate_warp<ND, 1, true, FUSE>, dim3(grid), dim3(kIntWarps * 32), 0, st, k, d, midstep, rbuf,
                                                                        interaction, capture);
    ++launched;
  }
  if (nblocks == 0) return launched;
  const size_t smem = integrate_smem_bytes(C, d.blk_maxf);
  if (C <= 128)
    launch_block_fast<ND, FUSE, 128>(k, d, nblocks, C, smem, midstep, rbuf, interaction, capture, st);
  else if (C <= 192)
    launch_block_fast<ND, FUSE, 192>(k, d, nblocks, C, smem, midstep, rbuf, interaction, capture, st);
  else if (C <= 256)
    launch_block_fast<ND, FUSE, 256>(k, d, nblocks, C, smem, midstep, rbuf, interaction, capture, st);
  else
    launch_block_fast<ND, FUSE, 512>(k, d, nblocks, C, smem, midstep, rbuf, interaction, capture, st);
  return launched + 1;
}

int launch_integrate_fast(const SysConst &k, const DevState &d, int nblocks, int C,
                          int midstep, int rbuf, int interaction, int capture,
                          cudaStream_t st, bool fuse) {
  if (k.n_dim == 3)
    return fuse ? launch_fast<3, true>(k, d, nblocks, C, midstep, rbuf, interaction, capture, st)
                : launch_fast<3, false>(k, d, nblocks, C, midstep, rbuf, interaction, capture, st);
  return fuse ? launch_fast<2, true>(k, d, nblocks, C, midstep, rbuf, interaction, capture, st)
              : launch_fast<2, false>(k, d, nblocks, C, midstep, rbuf, interaction, capture, st);
}

}  // namespace sc
