// Reduced-precision step kernels: FP32 arithmetic on shifted populations
// g_d = f_d - w_d, stored as FP32 or as FP16 (scaled by a power of two), two
// cells per thread (lbm_step_x2.cuh). Multiply-add contraction is allowed.
#include <type_traits>

#include "lbm_internal.h"
#include "lbm_step_x2.cuh"
#include "lbm_step_x2s.cuh"
#include "lbm_step_x4s.cuh"

namespace lbm {

// In FP16 storage without the Brinkman term the four-cell kernels serve AA
// even (pz % 4 == 0) and AA odd (nz a multiple of 128). The shuffle-aligned
// two-cell kernel serves the other shifted steps when nz is a multiple of
// 64; the rest uses the generic two-cell kernel.
template <class ST, int KIND, bool FORCE, bool BRINK>
static cudaError_t go(const StepArgs2<ST> &a, dim3 grid, dim3 block, cudaStream_t st)
{
  if constexpr (std::is_same<ST, StoreF16>::value && !BRINK) {
    if (KIND == kAAEvenStep && a.g.pz % 4 == 0 && !a.no_quad) {
      dim3 qg, qb;
      quad_launch_shape(a.g, qg, qb);
      qg.z = a.planes;
      step_kernel_even_quad<FORCE><<<qg, qb, 0, st>>>(a);
      return cudaGetLastError();
    }
    if constexpr (KIND == kAAOddStep) {
      if (a.g.nz % 128 == 0 && !a.no_quad && !a.no_shuffle) {
        dim3 qg, qb;
        quad_shuffle_launch_shape(a.g, qg, qb);
        qg.z = a.planes;
        step_kernel_x4s<KIND, FORCE><<<qg, qb, 0, st>>>(a);
        return cudaGetLastError();
      }
    }
  }
  if constexpr (KIND != kAAEvenStep) { // AA even is local: nothing to realign
    if (a.g.nz % 64 == 0 && !a.no_shuffle) {
      dim3 sg, sb;
      shuffle_launch_shape(a.g, sg, sb);
      sg.z = a.planes;
      step_kernel_x2s<ST, KIND, FORCE, BRINK><<<sg, sb, 0, st>>>(a);
      return cudaGetLastError();
    }
  }
  step_kernel_x2<ST, KIND, FORCE, BRINK><<<grid, block, 0, st>>>(a);
  return cudaGetLastError();
}

template <class ST, int KIND>
static cudaError_t pick(bool force, bool brink, const StepArgs2<ST> &a, dim3 grid, dim3 block,
    cudaStream_t st)
{
  if (brink)
    return go<ST, KIND, true, true>(a, grid, block, st);
  return force ? go<ST, KIND, true, false>(a, grid, block, st)
               : go<ST, KIND, false, false>(a, grid, block, st);
}

template <class ST>
static cudaError_t launch(int kind, bool force, bool brink, const StepArgs2<ST> &a,
    cudaStream_t st)
{
  dim3 grid, block;
  pair_launch_shape(a.g, grid, block);
  grid.z = a.planes;
  switch (kind) {
  case kPullStep: return pick<ST, kPullStep>(force, brink, a, grid, block, st);
  case kPushStep: return pick<ST, kPushStep>(force, brink, a, grid, block, st);
  case kAAEvenStep: return pick<ST, kAAEvenStep>(force, brink, a, grid, block, st);
  case kAAOddStep: return pick<ST, kAAOddStep>(force, brink, a, grid, block, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_step_x2_f32(int kind, bool force, bool brink, const StepArgs2<StoreF32> &a,
    cudaStream_t st)
{
  return launch(kind, force, brink, a, st);
}

cudaError_t launch_step_x2_f16(int kind, bool force, bool brink, const StepArgs2<StoreF16> &a,
    cudaStream_t st)
{
  return launch(kind, force, brink, a, st);
}

template <class ST, int KIND>
static cudaError_t go_cp(bool force, const StepArgs<ST> &a, dim3 grid, dim3 block,
    cudaStream_t st)
{
  if (KIND == kAAEvenStep) {
    if (a.cn == 0)
      return cudaSuccess;
    const unsigned nb = (a.cn + kStepThreads - 1) / kStepThreads;
    if (force)
      step_kernel_cp_local<ST, true><<<nb, kStepThreads, 0, st>>>(a);
    else
      step_kernel_cp_local<ST, false><<<nb, kStepThreads, 0, st>>>(a);
    return cudaGetLastError();
  }
  const bool zper = (a.g.per & 4) != 0;
  const bool off32 = (unsigned long long)Q * (unsigned long long)a.g.plane < (1ull << 32);
  if (off32) {
    if (force)
      zper ? step_kernel_cp<ST, KIND, true, true, uint32_t><<<grid, block, 0, st>>>(a)
           : step_kernel_cp<ST, KIND, true, false, uint32_t><<<grid, block, 0, st>>>(a);
    else
      zper ? step_kernel_cp<ST, KIND, false, true, uint32_t><<<grid, block, 0, st>>>(a)
           : step_kernel_cp<ST, KIND, false, false, uint32_t><<<grid, block, 0, st>>>(a);
  } else {
    if (force)
      zper ? step_kernel_cp<ST, KIND, true, true, uint64_t><<<grid, block, 0, st>>>(a)
           : step_kernel_cp<ST, KIND, true, false, uint64_t><<<grid, block, 0, st>>>(a);
    else
      zper ? step_kernel_cp<ST, KIND, false, true, uint64_t><<<grid, block, 0, st>>>(a)
           : step_kernel_cp<ST, KIND, false, false, uint64_t><<<grid, block, 0, st>>>(a);
  }
  return cudaGetLastError();
}

template <class ST>
static cudaError_t launch_cp(int kind, bool force, const StepArgs<ST> &a, dim3 grid, dim3 block,
    cudaStream_t st)
{
  switch (kind) {
  case kPullStep: return go_cp<ST, kPullStep>(force, a, grid, block, st);
  case kPushStep: return go_cp<ST, kPushStep>(force, a, grid, block, st);
  case kAAEvenStep: return go_cp<ST, kAAEvenStep>(force, a, grid, block, st);
  case kAAOddStep: return go_cp<ST, kAAOddStep>(force, a, grid, block, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_step_cp_f32(int kind, bool force, const StepArgs<StoreF32> &a, dim3 grid,
    dim3 block, cudaStream_t st)
{
  return launch_cp<StoreF32>(kind, force, a, grid, block, st);
}

cudaError_t launch_step_cp_f16(int kind, bool force, const StepArgs<StoreF16> &a, dim3 grid,
    dim3 block, cudaStream_t st)
{
  return launch_cp<StoreF16>(kind, force, a, grid, block, st);
}

} // namespace lbm
