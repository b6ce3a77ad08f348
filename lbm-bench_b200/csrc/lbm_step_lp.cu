// Reduced-precision step kernels: FP32 arithmetic on shifted populations
// g_d = f_d - w_d, stored as FP32 or as FP16 (scaled by a power of two), two
// cells per thread (lbm_step_x2.cuh). Multiply-add contraction is allowed.
#include <type_traits>

#include "lbm_internal.h"
#include "lbm_step_x2.cuh"
#include "lbm_step_x2s.cuh"
#include "lbm_step_x4s.cuh"
#include "lbm_step_cp2.cuh"

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
  cell_launch_shape(a.g, grid, block);
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

template <class ST, int KIND, bool FORCE>
static cudaError_t go_cp2(const StepArgs2<ST> &args, cudaStream_t st)
{
  StepArgs2<ST> a = args;
  if constexpr (KIND == kAAEvenStep) {
    constexpr uint32_t N = LocalCells<ST>::value;
    if (a.cn == 0)
      return cudaSuccess;
    const uint32_t end = a.c0 + a.cn;
    const uint32_t lo = (a.c0 + N - 1) / N * N, hi = end / N * N;
    if (hi > lo) {
      const uint32_t groups = (hi - lo) / N;
      step_kernel_cp2_local<ST, FORCE><<<(groups + kStepThreads - 1) / kStepThreads,
          kStepThreads, 0, st>>>(a);
    }
    if (a.c0 % N != 0 || end % N != 0)
      step_kernel_cp2_local_ends<ST, FORCE><<<1, 32, 0, st>>>(a);
    return cudaGetLastError();
  } else {
  const bool zper = (a.g.per & 4) != 0;
  const bool off32 = (unsigned long long)Q * (unsigned long long)a.g.plane < (1ull << 32);
  if constexpr (((LBM_CP2_PAIR_KINDS >> KIND) & 1) != 0) {
    // two cells per thread (z, z + 32): block (32, 4), one word pair per block column
    const dim3 block(32, 4, 1);
    const dim3 grid((unsigned)((a.g.W + 1) / 2), (unsigned)((a.g.ny + 3) / 4), (unsigned)a.planes);
    if (cp_prefetches<KIND, sizeof(typename ST::S)>())
      a.pf_planes = prefetch_planes(LBM_CP_PF_TENTHS, LBM_MINB_CP2_PAIR, grid.x * grid.y);
    if (off32)
      zper ? step_kernel_cp2_pair<ST, KIND, FORCE, true, uint32_t><<<grid, block, 0, st>>>(a)
           : step_kernel_cp2_pair<ST, KIND, FORCE, false, uint32_t><<<grid, block, 0, st>>>(a);
    else
      zper ? step_kernel_cp2_pair<ST, KIND, FORCE, true, uint64_t><<<grid, block, 0, st>>>(a)
           : step_kernel_cp2_pair<ST, KIND, FORCE, false, uint64_t><<<grid, block, 0, st>>>(a);
    return cudaGetLastError();
  }
  dim3 grid, block;
  cell_launch_shape(a.g, grid, block);
  grid.z = a.planes;
  if (off32)
    zper ? step_kernel_cp<CpMathUnits<ST>, KIND, FORCE, true, uint32_t><<<grid, block, 0, st>>>(a)
         : step_kernel_cp<CpMathUnits<ST>, KIND, FORCE, false, uint32_t><<<grid, block, 0, st>>>(a);
  else
    zper ? step_kernel_cp<CpMathUnits<ST>, KIND, FORCE, true, uint64_t><<<grid, block, 0, st>>>(a)
         : step_kernel_cp<CpMathUnits<ST>, KIND, FORCE, false, uint64_t><<<grid, block, 0, st>>>(a);
  return cudaGetLastError();
  }
}

template <class ST>
static cudaError_t launch_cp2(int kind, bool force, const StepArgs2<ST> &a, cudaStream_t st)
{
  switch (kind) {
  case kPullStep: return force ? go_cp2<ST, kPullStep, true>(a, st)
                               : go_cp2<ST, kPullStep, false>(a, st);
  case kPushStep: return force ? go_cp2<ST, kPushStep, true>(a, st)
                               : go_cp2<ST, kPushStep, false>(a, st);
  case kAAEvenStep: return force ? go_cp2<ST, kAAEvenStep, true>(a, st)
                                 : go_cp2<ST, kAAEvenStep, false>(a, st);
  case kAAOddStep: return force ? go_cp2<ST, kAAOddStep, true>(a, st)
                                : go_cp2<ST, kAAOddStep, false>(a, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_step_cp2_f32(int kind, bool force, const StepArgs2<StoreF32> &a,
    cudaStream_t st)
{
  return launch_cp2<StoreF32>(kind, force, a, st);
}

cudaError_t launch_step_cp2_f16(int kind, bool force, const StepArgs2<StoreF16> &a,
    cudaStream_t st)
{
  return launch_cp2<StoreF16>(kind, force, a, st);
}

} // namespace lbm
