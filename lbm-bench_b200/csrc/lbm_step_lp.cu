// Reduced-precision step kernels: FP32 arithmetic on shifted populations
// g_d = f_d - w_d, stored as FP32 or as FP16 (scaled by a power of two).
// Multiply-add contraction is allowed here.
#include "lbm_internal.h"

namespace lbm {

template <class ST, int KIND, bool FORCE, bool BRINK>
static cudaError_t go(const StepArgs<ST> &a, dim3 grid, dim3 block, cudaStream_t st)
{
  step_kernel<ST, KIND, FORCE, BRINK><<<grid, block, 0, st>>>(a);
  return cudaGetLastError();
}

template <class ST, int KIND>
static cudaError_t pick(bool force, bool brink, const StepArgs<ST> &a, dim3 grid, dim3 block,
    cudaStream_t st)
{
  if (brink)
    return go<ST, KIND, true, true>(a, grid, block, st);
  return force ? go<ST, KIND, true, false>(a, grid, block, st)
               : go<ST, KIND, false, false>(a, grid, block, st);
}

template <class ST>
static cudaError_t launch(int kind, bool force, bool brink, const StepArgs<ST> &a, dim3 grid,
    dim3 block, cudaStream_t st)
{
  switch (kind) {
  case kPullStep: return pick<ST, kPullStep>(force, brink, a, grid, block, st);
  case kPushStep: return pick<ST, kPushStep>(force, brink, a, grid, block, st);
  case kAAEvenStep: return pick<ST, kAAEvenStep>(force, brink, a, grid, block, st);
  case kAAOddStep: return pick<ST, kAAOddStep>(force, brink, a, grid, block, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_step_f32(int kind, bool force, bool brink, const StepArgs<StoreF32> &a,
    dim3 grid, dim3 block, cudaStream_t st)
{
  return launch(kind, force, brink, a, grid, block, st);
}

cudaError_t launch_step_f16(int kind, bool force, bool brink, const StepArgs<StoreF16> &a,
    dim3 grid, dim3 block, cudaStream_t st)
{
  return launch(kind, force, brink, a, grid, block, st);
}

} // namespace lbm
