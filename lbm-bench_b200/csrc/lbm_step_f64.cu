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

// Zou-He pressure boundary (src/lbm.c:676-785, kernelComputeBoundaryConditions),
// applied to the state after a step, one thread per (y, z) of the inlet
// plane (blockIdx.z = 0, x = 0) or the outlet plane (1, x = nx - 1) where
// `marks` flags a cell. Populations are read and written through the
// orientation of the current state, so the kernel serves every pattern.
// It fixes the five populations entering across the x face from the
// outside - E, NE, SE, TE, BE at the inlet, W, NW, SW, TW, BW at the outlet
// - from the fourteen known ones so that the cell's density is rho_in or
// rho_out. The arithmetic is the reference's, operation for operation and
// in FP64 (this unit has no multiply-add contraction), so the FP64 state is
// bit-identical to the reference's pull and push kernels followed by its
// boundary pass; shifted storage adds and removes w_d around it.
template <class ST>
__global__ void pressure_bc_kernel(Grid g, UserBox u, int orient, typename ST::S *state,
    const uint32_t *__restrict__ mask, const uint8_t *__restrict__ marks, double rho_in,
    double rho_out, float scale, float inv_scale)
{
  using V = typename ST::V;
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int side = blockIdx.z;
  if (z >= u.nz || y >= u.ny || !marks[((size_t)side * u.ny + y) * u.nz + z])
    return;
  const int x = side ? u.nx - 1 : 0;
  uint32_t cell, m;
  if (!locate(g, mask, x + u.ox, y + u.oy, z + u.oz, cell, m))
    return;
  const Nbr nb = make_nbr(g, x + u.ox, y + u.oy, z + u.oz, cell);
  auto at = [&](int d) {
    int p;
    uint32_t c;
    state_slot(orient, d, m, cell, nb, p, c);
    return state + (size_t)p * g.plane + c;
  };
  auto wgt = [](int d) {
    const int c = wclass(d);
    return c == 0 ? 1.0 / 3.0 : c == 1 ? 1.0 / 18.0 : 1.0 / 36.0;
  };
  auto get = [&](int d) {
    double v = (double)ST::decode(*at(d), (V)inv_scale);
    return ST::kShifted ? v + wgt(d) : v;
  };
  auto put = [&](int d, double v) {
    if (ST::kShifted)
      v -= wgt(d);
    ST::store(at(d), (V)v, (V)scale);
  };
  const double third = 1.0 / 3.0, quarter = 1.0 / 4.0, sixth = 1.0 / 6.0;
  const double fN = get(dN), fS = get(dS), fT = get(dT), fB = get(dB);
  const double rest = get(dC) + (fT + fB + fS + fN) + (get(dTS) + get(dBS) + get(dTN) + get(dBN));
  if (side == 0) {
    const double dens = rho_in;
    const double fW = get(dW), fSW = get(dSW), fNW = get(dNW), fTW = get(dTW), fBW = get(dBW);
    const double ux = 1.0 - (rest + 2.0 * (fSW + fTW + fW + fBW + fNW)) * (1.0 / rho_in);
    const double ind = sixth * dens * ux;
    put(dE, fW + third * dens * ux);
    put(dNE, fSW - quarter * (fN - fS) + ind);
    put(dSE, fNW + quarter * (fN - fS) + ind);
    put(dTE, fBW - quarter * (fT - fB) + ind);
    put(dBE, fTW + quarter * (fT - fB) + ind);
  } else {
    const double dens = rho_out;
    const double fE = get(dE), fNE = get(dNE), fSE = get(dSE), fTE = get(dTE), fBE = get(dBE);
    const double ux = -1.0 + (rest + 2.0 * (fNE + fBE + fE + fTE + fSE)) * (1.0 / rho_out);
    const double ind = sixth * dens * ux;
    put(dW, fE - third * dens * ux);
    put(dSW, fNE + quarter * (fN - fS) - ind);
    put(dNW, fSE - quarter * (fN - fS) - ind);
    put(dBW, fTE + quarter * (fT - fB) - ind);
    put(dTW, fBE - quarter * (fT - fB) - ind);
  }
}

cudaError_t launch_pressure_bc(int precision, const Grid &g, const UserBox &u, int orient,
    void *state, const uint32_t *mask, const uint8_t *marks, double rho_in, double rho_out,
    float scale, cudaStream_t st)
{
  dim3 block(32, 4, 1);
  dim3 grid((u.nz + 31) / 32, (u.ny + 3) / 4, 2);
  switch (precision) {
  case kF64:
    pressure_bc_kernel<StoreF64><<<grid, block, 0, st>>>(g, u, orient, (double *)state, mask,
        marks, rho_in, rho_out, 1.f, 1.f);
    break;
  case kF32:
    pressure_bc_kernel<StoreF32><<<grid, block, 0, st>>>(g, u, orient, (float *)state, mask,
        marks, rho_in, rho_out, 1.f, 1.f);
    break;
  default:
    pressure_bc_kernel<StoreF16><<<grid, block, 0, st>>>(g, u, orient, (__half *)state, mask,
        marks, rho_in, rho_out, scale, 1.f / scale);
  }
  return cudaGetLastError();
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

template <class ST, int KIND>
static cudaError_t go_cp(bool force, const StepArgs<ST> &args, dim3 grid, dim3 block,
    cudaStream_t st)
{
  StepArgs<ST> a = args;
  if constexpr (KIND == kAAEvenStep) {
    if (a.cn == 0)
      return cudaSuccess;
    const unsigned nb = (a.cn + kStepThreads - 1) / kStepThreads;
    if (force)
      step_kernel_cp_local<ST, true><<<nb, kStepThreads, 0, st>>>(a);
    else
      step_kernel_cp_local<ST, false><<<nb, kStepThreads, 0, st>>>(a);
    return cudaGetLastError();
  } else {
  if (cp_prefetches<KIND, sizeof(typename ST::S)>())
    a.pf_planes = prefetch_planes(LBM_CP_PF_TENTHS,
        CpOccupancy<KIND, sizeof(typename ST::S)>::value, grid.x * grid.y);
  const bool zper = (a.g.per & 4) != 0;
  const bool off32 = (unsigned long long)Q * (unsigned long long)a.g.plane < (1ull << 32);
  if (off32) {
    if (force)
      zper ? step_kernel_cp<CpMathDirect<ST>, KIND, true, true, uint32_t><<<grid, block, 0, st>>>(a)
           : step_kernel_cp<CpMathDirect<ST>, KIND, true, false, uint32_t><<<grid, block, 0, st>>>(a);
    else
      zper ? step_kernel_cp<CpMathDirect<ST>, KIND, false, true, uint32_t><<<grid, block, 0, st>>>(a)
           : step_kernel_cp<CpMathDirect<ST>, KIND, false, false, uint32_t><<<grid, block, 0, st>>>(a);
  } else {
    if (force)
      zper ? step_kernel_cp<CpMathDirect<ST>, KIND, true, true, uint64_t><<<grid, block, 0, st>>>(a)
           : step_kernel_cp<CpMathDirect<ST>, KIND, true, false, uint64_t><<<grid, block, 0, st>>>(a);
    else
      zper ? step_kernel_cp<CpMathDirect<ST>, KIND, false, true, uint64_t><<<grid, block, 0, st>>>(a)
           : step_kernel_cp<CpMathDirect<ST>, KIND, false, false, uint64_t><<<grid, block, 0, st>>>(a);
  }
  return cudaGetLastError();
  }
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

cudaError_t launch_step_cp_f64(int kind, bool force, const StepArgs<StoreF64> &a, dim3 grid,
    dim3 block, cudaStream_t st)
{
  return launch_cp<StoreF64>(kind, force, a, grid, block, st);
}

} // namespace lbm
