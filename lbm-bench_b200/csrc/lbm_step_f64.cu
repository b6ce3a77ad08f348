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
