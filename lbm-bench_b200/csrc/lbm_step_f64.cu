// FP64 step kernels. This translation unit is compiled with --fmad=false:
// every multiply and add rounds separately, in the reference's order, so
// the results are bit-identical to LBM-Bench's CPU kernels built with
// strict IEEE arithmetic (src/kernel_pull_soa.c:118-198).
#include "lbm_internal.h"

namespace lbm {

template <int KIND, bool FORCE, bool BRINK>
static cudaError_t go(const StepArgs<StoreF64> &a, dim3 grid, dim3 block, cudaStream_t st)
{
  step_kernel<StoreF64, KIND, FORCE, BRINK><<<grid, block, 0, st>>>(a);
  return cudaGetLastError();
}

template <int KIND>
static cudaError_t pick(bool force, bool brink, const StepArgs<StoreF64> &a, dim3 grid,
    dim3 block, cudaStream_t st)
{
  if (brink)
    return go<KIND, true, true>(a, grid, block, st);
  return force ? go<KIND, true, false>(a, grid, block, st)
               : go<KIND, false, false>(a, grid, block, st);
}

template <int KIND, bool FORCE, int G>
static cudaError_t go_tma(const TmaArgs<StoreF64> &a, int blocks, cudaStream_t st)
{
  // the opt-in shared-memory size is a per-kernel attribute: set it once
  // per instantiation for the largest size requested so far
  static size_t granted = 0;
  const size_t smem = (size_t)a.stages * a.stage_bytes;
  if (smem > granted) {
    cudaError_t e = cudaFuncSetAttribute(step_kernel_tma<StoreF64, KIND, FORCE, G>,
        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
      return e;
    granted = smem;
  }
  step_kernel_tma<StoreF64, KIND, FORCE, G><<<blocks, tma_threads(G), smem, st>>>(a);
  return cudaGetLastError();
}

template <int KIND, bool FORCE>
static cudaError_t go_tma_groups(const TmaArgs<StoreF64> &a, int groups, int blocks,
    cudaStream_t st)
{
  switch (groups) {
  case 1: return go_tma<KIND, FORCE, 1>(a, blocks, st);
  case 3: return go_tma<KIND, FORCE, 3>(a, blocks, st);
  default: return go_tma<KIND, FORCE, 2>(a, blocks, st);
  }
}

cudaError_t launch_step_tma_f64(int kind, bool force, const TmaArgs<StoreF64> &a, int groups,
    int blocks, cudaStream_t st)
{
  if (groups < 1 || groups > 3 || a.stages < groups || a.stages % groups != 0 || a.stages > 8)
    return cudaErrorInvalidValue; // each stage must belong to one consumer group
  switch (kind) {
  case kPullStep: return force ? go_tma_groups<kPullStep, true>(a, groups, blocks, st)
                               : go_tma_groups<kPullStep, false>(a, groups, blocks, st);
  case kPushStep: return force ? go_tma_groups<kPushStep, true>(a, groups, blocks, st)
                               : go_tma_groups<kPushStep, false>(a, groups, blocks, st);
  case kAAEvenStep: return force ? go_tma_groups<kAAEvenStep, true>(a, groups, blocks, st)
                                 : go_tma_groups<kAAEvenStep, false>(a, groups, blocks, st);
  case kAAOddStep: return force ? go_tma_groups<kAAOddStep, true>(a, groups, blocks, st)
                                : go_tma_groups<kAAOddStep, false>(a, groups, blocks, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_step_f64(int kind, bool force, bool brink, const StepArgs<StoreF64> &a,
    dim3 grid, dim3 block, cudaStream_t st)
{
  switch (kind) {
  case kPullStep: return pick<kPullStep>(force, brink, a, grid, block, st);
  case kPushStep: return pick<kPushStep>(force, brink, a, grid, block, st);
  case kAAEvenStep: return pick<kAAEvenStep>(force, brink, a, grid, block, st);
  case kAAOddStep: return pick<kAAOddStep>(force, brink, a, grid, block, st);
  }
  return cudaErrorInvalidValue;
}

} // namespace lbm
